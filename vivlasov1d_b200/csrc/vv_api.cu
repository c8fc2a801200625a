// libvv: C ABI implementation (include/vv.h).
//
// Host-side responsibilities: grid set-up (coordinates, h0, FFT twiddles,
// the tensor-product preconditioner's eigenvalues and per-mode LU factors,
// the CFD4 Poisson symbol), launch configuration, and the two drivers that
// the reference delegates to PETSc: restarted GMRES (KSPGMRES semantics) and
// the Picard-over-phi time step of run_nonlinear_matrixfree_split_mp.py.
// All decisions of GMRES (Givens rotations, convergence tests) are taken on
// the device; the host only reads a 16-byte status block per iteration.
#include "vv.h"
#include "vv_common.cuh"
#include "vv_bracket.cuh"
#include "vv_pc.cuh"
#include "vv_vec.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <vector>

using cd = std::complex<double>;

struct vv_ctx {
    vv_grid g;
    int nx, nv, M, logM, nmodes, restart;
    size_t ncell;
    double hx, hv, ht_inv, hx_inv, hv_inv, hx2_inv, f1, f2;
    cudaStream_t st;
    int device;
    // device buffers
    double *v, *h0, *hxp, *Fh, *tmp, *bvec, *delta, *fl, *V, *part, *scal, *xscratch, *mom_part;
    double2 *spec, *tw, *lambda, *dinv;
    double *alpha, *gamma, *sym_inv;
    vv::GmresState* gm;
    // pinned host staging
    double* hpin;
    int* hstat;
    // launch configuration
    int npart, npart_max;
    int mom_S, mom_seg;
    int pcR;
    size_t smem_rfft, smem_irfft, smem_tri, smem_pois;
    bool pivot_differs;
    // timing of the JVP stencil kernel
    bool timing;
    std::vector<cudaEvent_t> ev;
    size_t ev_used;
    int64_t t_launches;
    double t_ms;
    int64_t launches;
};

namespace {

thread_local char g_err[256];

int fail_cuda(cudaError_t e, const char* what) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return VV_ERR_CUDA;
}

#define CK(call)                                             \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call); \
    } while (0)
#define CKL(c)                                                     \
    do {                                                           \
        (c)->launches++;                                           \
        cudaError_t e_ = cudaGetLastError();                       \
        if (e_ != cudaSuccess) return fail_cuda(e_, "kernel launch"); \
    } while (0)
#define TRY(x)                    \
    do {                          \
        int s_ = (x);             \
        if (s_ != VV_OK) return s_; \
    } while (0)

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

int ilog2(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

template <typename T>
int dalloc(T** p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        snprintf(g_err, sizeof g_err, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
        return VV_ERR_ALLOC;
    }
    return VV_OK;
}

inline unsigned grid1d(size_t n, int threads, unsigned cap = 4096) {
    size_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

vv::BracketParams bparams(const vv_ctx* c, double factor) {
    vv::BracketParams p;
    p.nx = c->nx;
    p.nv = c->nv;
    p.ht_inv = c->ht_inv;
    p.factor = factor;
    p.f1 = c->f1;
    p.f2 = c->f2;
    p.h0 = c->h0;
    p.hxp = c->hxp;
    return p;
}

vv::PcParams pcparams(const vv_ctx* c) {
    vv::PcParams p;
    p.nx = c->nx;
    p.nv = c->nv;
    p.M = c->M;
    p.logM = c->logM;
    p.R = c->pcR;
    p.tw = c->tw;
    return p;
}

// ---- timing helpers --------------------------------------------------------
cudaEvent_t next_event(vv_ctx* c) {
    if (c->ev_used == c->ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev.push_back(e);
    }
    return c->ev[c->ev_used++];
}

int drain_timing(vv_ctx* c) {
    if (c->ev_used == 0) return VV_OK;
    CK(cudaEventSynchronize(c->ev[c->ev_used - 1]));
    for (size_t k = 0; k + 1 < c->ev_used; k += 2) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]));
        c->t_ms += ms;
        c->t_launches++;
    }
    c->ev_used = 0;
    return VV_OK;
}

// ---- bracket launches -------------------------------------------------------
template <int SCHEME, int MODE>
int launch_bracket_s(vv_ctx* c, const double* X, const double* Xh, double* Y, double factor, double* sumsq) {
    dim3 grid((c->nx + vv::BX - 1) / vv::BX, (c->nv + vv::BY - 1) / vv::BY);
    dim3 block(vv::BX, vv::TY);
    vv::BracketParams p = bparams(c, factor);
    const bool timed = c->timing && MODE == vv::MODE_JVP;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timed) {
        if (c->ev_used + 2 > 8192) TRY(drain_timing(c));
        e0 = next_event(c);
        e1 = next_event(c);
        if (e0) cudaEventRecord(e0, c->st);
    }
    if (c->g.order == VV_ORDER_REFERENCE)
        vv::k_bracket_ref<SCHEME, MODE><<<grid, block, 0, c->st>>>(X, Xh, Y, p, sumsq);
    else
        vv::k_bracket_fac<SCHEME, MODE, double><<<grid, block, 0, c->st>>>(X, Xh, Y, p, sumsq);
    CKL(c);
    if (timed && e1) cudaEventRecord(e1, c->st);
    return VV_OK;
}

template <int MODE>
int launch_bracket(vv_ctx* c, const double* X, const double* Xh, double* Y, double factor, double* sumsq) {
    switch (c->g.bracket) {
        case VV_BRACKET_J1: return launch_bracket_s<1, MODE>(c, X, Xh, Y, factor, sumsq);
        case VV_BRACKET_J2: return launch_bracket_s<2, MODE>(c, X, Xh, Y, factor, sumsq);
        default: return launch_bracket_s<4, MODE>(c, X, Xh, Y, factor, sumsq);
    }
}

int bracket_tiles(const vv_ctx* c) {
    return ((c->nx + vv::BX - 1) / vv::BX) * ((c->nv + vv::BY - 1) / vv::BY);
}

// ---- reductions ---------------------------------------------------------------
// reduce np partials (1 column) into dst (device)
int reduce_to(vv_ctx* c, const double* part, int np, double* dst) {
    vv::k_reduce_cols<<<1, vv::RED_THREADS, 0, c->st>>>(part, np, 1, np, dst);
    CKL(c);
    return VV_OK;
}

int sumsq_to(vv_ctx* c, const double* x, double* dst) {
    vv::k_sumsq_partial<double><<<c->npart, vv::RED_THREADS, 0, c->st>>>(x, c->ncell, c->part);
    CKL(c);
    return reduce_to(c, c->part, c->npart, dst);
}

int read_scalar(vv_ctx* c, const double* dsrc, double* out) {
    CK(cudaMemcpyAsync(c->hpin, dsrc, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *out = c->hpin[0];
    return VV_OK;
}

// ---- preconditioner ---------------------------------------------------------
int pc_apply(vv_ctx* c, const double* X, double* Y) {
    vv::PcParams p = pcparams(c);
    const unsigned rows = (unsigned)((c->nv + c->pcR - 1) / c->pcR);
    vv::k_rfft_rows<double><<<rows, 256, c->smem_rfft, c->st>>>(X, c->spec, p);
    CKL(c);
    vv::TriParams t;
    t.nv = c->nv;
    t.nmodes = c->nmodes;
    t.lambda = c->lambda;
    t.alpha = c->alpha;
    t.gamma = c->gamma;
    t.dinv = c->dinv;
    vv::k_tridiag_modes<<<c->nmodes, vv::TRI_THREADS, c->smem_tri, c->st>>>(c->spec, t);
    CKL(c);
    vv::k_irfft_rows<double><<<rows, 256, c->smem_irfft, c->st>>>(c->spec, Y, p);
    CKL(c);
    return VV_OK;
}

// Y = P^-1 J X (or J X)
int apply_operator(vv_ctx* c, const double* X, double* Y) {
    if (c->g.preconditioner == VV_PC_TENSOR_KINETIC) {
        TRY(launch_bracket<vv::MODE_JVP>(c, X, nullptr, c->tmp, 0.5, nullptr));
        return pc_apply(c, c->tmp, Y);
    }
    return launch_bracket<vv::MODE_JVP>(c, X, nullptr, Y, 0.5, nullptr);
}

// ---- moments / Poisson ------------------------------------------------------
vv::PoissonParams pparams(const vv_ctx* c) {
    vv::PoissonParams p;
    p.nx = c->nx;
    p.M = c->M;
    p.logM = c->logM;
    p.S = c->mom_S;
    p.hv = c->hv;
    p.charge = c->g.charge;
    p.hx2_inv = c->hx2_inv;
    p.hx = c->hx;
    p.inv_nx = 1.0 / c->nx;
    p.tw = c->tw;
    p.sym_inv = c->sym_inv;
    return p;
}

int moments_poisson(vv_ctx* c, const double* F, double* n, double* u, double* e, double* a,
                    double* phi, double* h1, double* scal) {
    dim3 grid((c->nx + vv::MOM_TX - 1) / vv::MOM_TX, c->mom_S);
    dim3 block(vv::MOM_TX, vv::MOM_TY);
    vv::k_moments_partial<double><<<grid, block, 0, c->st>>>(F, c->nx, c->nv, c->mom_seg, c->v, c->mom_part);
    CKL(c);
    vv::k_moments_poisson<<<1, vv::POIS_THREADS, c->smem_pois, c->st>>>(c->mom_part, nullptr, n, u, e, a, phi, h1,
                                                                        scal, pparams(c));
    CKL(c);
    return VV_OK;
}

// Poisson apply: mode 0 rhs, 1 matvec, 2 function; optional ||y||^2 -> sumsq
__global__ void k_poisson_apply(const double* __restrict__ x, const double* __restrict__ n,
                                double* __restrict__ y, int nx, double hx2_inv, double charge, int mode,
                                double* __restrict__ sumsq) {
    __shared__ double red[32];
    __shared__ double nmean_s;
    double t = 0.0;
    if (mode != 1) {
        for (int i = threadIdx.x; i < nx; i += blockDim.x) t += n[i];
        t = block_sum(t, red);
        if (threadIdx.x == 0) nmean_s = t / nx;
        __syncthreads();
    }
    double r2 = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        double r;
        if (mode == 0) {
            r = -(n[i] - nmean_s) * charge;
        } else {
            const int im2 = (i - 2 + 2 * nx) % nx, im1 = (i - 1 + nx) % nx;
            const int ip1 = (i + 1) % nx, ip2 = (i + 2) % nx;
            r = (5. * x[im2] - 32. * x[im1] + 54. * x[i] - 32. * x[ip1] + 5. * x[ip2]) * hx2_inv / 12.;
            if (mode == 2) r = r + (n[i] - nmean_s) * charge;
        }
        if (y) y[i] = r;
        r2 += r * r;
    }
    r2 = block_sum(r2, red);
    if (threadIdx.x == 0 && sumsq) sumsq[0] = r2;
}

int poisson_apply(vv_ctx* c, const double* x, const double* n, double* y, int mode, double* sumsq) {
    k_poisson_apply<<<1, 1024, 0, c->st>>>(x, n, y, c->nx, c->hx2_inv, c->g.charge, mode, sumsq);
    CKL(c);
    return VV_OK;
}

// ---- GMRES driver ---------------------------------------------------------
struct GmHead {
    int it, its, reason, active;
};

int read_head(vv_ctx* c, GmHead* h) {
    CK(cudaMemcpyAsync(c->hstat, c->gm, sizeof(GmHead), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    std::memcpy(h, c->hstat, sizeof(GmHead));
    return VV_OK;
}

int gmres(vv_ctx* c, const double* b, double* x, const vv_ksp_opts* o, vv_ksp_result* res) {
    const int restart = (o->restart > 0) ? o->restart : c->restart;
    if (restart > c->restart || restart < 1) return VV_ERR_ARG;
    const size_t n = c->ncell;
    double* V = c->V;
    vv::GmresState hs;
    std::memset(&hs, 0, offsetof(vv::GmresState, hcol));
    hs.restart = restart;
    hs.max_it = o->max_it;
    hs.rtol = o->rtol;
    hs.atol = o->atol;
    hs.dtol = (o->dtol > 0.0) ? o->dtol : 1e5;
    hs.haptol = 1e-30;
    std::memcpy(c->hpin, &hs, offsetof(vv::GmresState, hcol));
    CK(cudaMemcpyAsync(c->gm, c->hpin, offsetof(vv::GmresState, hcol), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(x, 0, n * sizeof(double), c->st));
    const unsigned eg = grid1d(n, 256);
    bool guess_zero = true;
    GmHead h{};
    for (;;) {
        // r = b - A x  (KSPInitialResidual) into V0
        if (guess_zero) {
            CK(cudaMemcpyAsync(V, b, n * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        } else {
            TRY(apply_operator(c, x, V));
            vv::k_axpby<double><<<eg, 256, 0, c->st>>>(b, V, n, 1.0, -1.0);
            CKL(c);
        }
        TRY(sumsq_to(c, V, &c->gm->sumsq));
        vv::k_gmres_cycle_start<<<1, 32, 0, c->st>>>(c->gm);
        CKL(c);
        vv::k_scale<double, double><<<eg, 256, 0, c->st>>>(V, V, n, &c->gm->scale, 1.0);
        CKL(c);
        TRY(read_head(c, &h));
        int it = 0;
        while (h.active) {
            double* w = V + (size_t)(it + 1) * n;
            TRY(apply_operator(c, V + (size_t)it * n, w));
            // classical Gram-Schmidt: hcol = <w, v_j>, w -= sum hcol_j v_j
            const int m = it + 1;
            for (int q0 = 0; q0 < m; q0 += vv::MDOT_CHUNK) {
                vv::k_mdot_partial<double><<<c->npart, vv::RED_THREADS, 0, c->st>>>(w, V, n, q0, m, n, c->part,
                                                                                    c->npart_max);
                CKL(c);
            }
            vv::k_reduce_cols<<<1, vv::RED_THREADS, 0, c->st>>>(c->part, c->npart, m, c->npart_max, c->gm->hcol);
            CKL(c);
            double* part2 = c->part + (size_t)(vv::MAX_RESTART + 1) * c->npart_max;
            vv::k_maxpy<double><<<c->npart, vv::RED_THREADS, 0, c->st>>>(w, V, n, m, c->gm->hcol, -1.0, n, part2);
            CKL(c);
            TRY(reduce_to(c, part2, c->npart, &c->gm->sumsq));
            vv::k_gmres_arnoldi<<<1, 32, 0, c->st>>>(c->gm);
            CKL(c);
            vv::k_scale<double, double><<<eg, 256, 0, c->st>>>(w, w, n, &c->gm->scale, 1.0);
            CKL(c);
            TRY(read_head(c, &h));
            it = h.it;
        }
        vv::k_gmres_backsub<<<1, 32, 0, c->st>>>(c->gm);
        CKL(c);
        // number of coefficients to apply is in gm->pad
        int pad = 0;
        CK(cudaMemcpyAsync(c->hstat, &c->gm->pad, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        pad = c->hstat[0];
        if (pad > 0) {
            vv::k_maxpy<double><<<c->npart, vv::RED_THREADS, 0, c->st>>>(x, V, n, pad, c->gm->nrs, 1.0, n, nullptr);
            CKL(c);
        }
        TRY(read_head(c, &h));
        if (h.reason != 0) break;
        guess_zero = false;
    }
    double rn = 0.0;
    TRY(read_scalar(c, &c->gm->res, &rn));
    res->its = h.its;
    res->reason = h.reason;
    res->rnorm = rn;
    return VV_OK;
}

// ---- step helpers -----------------------------------------------------------
int copy_d(vv_ctx* c, double* dst, const double* src, size_t count) {
    if (!dst || !src || dst == src) return VV_OK;
    CK(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    return VV_OK;
}

int set_hxp(vv_ctx* c, const double* h1p, const double* h1h, const double* h2p, const double* h2h) {
    const double* src[4] = {h1p, h1h, h2p, h2h};
    for (int k = 0; k < 4; ++k) {
        double* dst = c->hxp + (size_t)k * c->nx;
        if (src[k]) {
            CK(cudaMemcpyAsync(dst, src[k], c->nx * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        } else {
            CK(cudaMemsetAsync(dst, 0, c->nx * sizeof(double), c->st));
        }
    }
    return VV_OK;
}

int residual_norm(vv_ctx* c, const double* F, double* Y, double* out) {
    const int tiles = bracket_tiles(c);
    TRY(launch_bracket<vv::MODE_RESIDUAL>(c, F, c->Fh, Y, 1.0, c->part));
    TRY(reduce_to(c, c->part, tiles, c->scal + 2));
    double s2 = 0.0;
    TRY(read_scalar(c, c->scal + 2, &s2));
    *out = std::sqrt(s2);
    return VV_OK;
}

int calc_residual(vv_ctx* c, vv_state* st, double* out) {
    double fnorm = 0.0;
    TRY(residual_norm(c, st->f, c->tmp, &fnorm));
    TRY(poisson_apply(c, st->phi, st->n, nullptr, 2, c->scal + 3));
    double p2 = 0.0;
    TRY(read_scalar(c, c->scal + 3, &p2));
    *out = fnorm + std::sqrt(p2);
    return VV_OK;
}

int calc_moments(vv_ctx* c, vv_state* st) {
    return moments_poisson(c, st->f, st->n, st->u, st->e, st->a, st->phi, st->h1c, c->scal);
}

}  // namespace

// =============================================================================
// C ABI
// =============================================================================
extern "C" {

int vv_version(void) { return 1; }

const char* vv_status_string(int status) {
    switch (status) {
        case VV_OK: return "ok";
        case VV_ERR_ARG: return "invalid argument";
        case VV_ERR_UNSUPPORTED: return "unsupported configuration";
        case VV_ERR_CUDA: return g_err[0] ? g_err : "CUDA error";
        case VV_ERR_ALLOC: return g_err[0] ? g_err : "device allocation failed";
        case VV_ERR_DIVERGED: return "nonlinear residual above the abort threshold";
        case VV_ERR_NAN: return "NaN or Inf encountered";
        case VV_ERR_TIMEOUT: return "bounded device wait gave up";
        default: return "unknown status";
    }
}

int vv_create(const vv_grid* grid, vv_ctx** out) {
    if (!grid || !out) return VV_ERR_ARG;
    *out = nullptr;
    const vv_grid& g = *grid;
    if (g.nx < 4 || g.nv < 5 || !(g.L > 0.0) || !(g.vmax > g.vmin) || !(g.ht > 0.0)) return VV_ERR_ARG;
    if (!is_pow2(g.nx)) {
        snprintf(g_err, sizeof g_err, "nx=%d: the x FFT kernels need a power of two", g.nx);
        return VV_ERR_UNSUPPORTED;
    }
    if (g.bracket != VV_BRACKET_J1 && g.bracket != VV_BRACKET_J2 && g.bracket != VV_BRACKET_J4) return VV_ERR_ARG;
    if (g.preconditioner != VV_PC_NONE && g.preconditioner != VV_PC_TENSOR_KINETIC) return VV_ERR_ARG;
    if (g.laplace != VV_LAPLACE_CFD4) return VV_ERR_UNSUPPORTED;
    const int restart = g.gmres_restart > 0 ? g.gmres_restart : 30;
    if (restart > vv::MAX_RESTART) return VV_ERR_ARG;

    vv_ctx* c = new vv_ctx();
    c->g = g;
    c->g.gmres_restart = restart;
    c->nx = g.nx;
    c->nv = g.nv;
    c->M = g.nx / 2;
    c->logM = ilog2(c->M);
    c->nmodes = c->M + 1;
    c->restart = restart;
    c->ncell = (size_t)g.nx * g.nv;
    c->st = 0;
    cudaGetDevice(&c->device);
    // grid (run_base.py:133-137, Grid.pyx:40-48)
    c->hx = g.L / g.nx;
    c->hv = (g.vmax - g.vmin) / (g.nv - 1);
    c->ht_inv = 1. / g.ht;
    c->hx_inv = 1. / c->hx;
    c->hv_inv = 1. / c->hv;
    c->hx2_inv = 1. / (c->hx * c->hx);
    c->f1 = c->hx_inv * c->hv_inv / 12.;  // PoissonBracket.pyx:344
    c->f2 = c->hx_inv * c->hv_inv / 24.;  // PoissonBracket.pyx:345

    const int nx = c->nx, nv = c->nv, M = c->M, nm = c->nmodes;
    const size_t n = c->ncell;
    c->npart_max = 592;  // 4 x 148 SMs
    {
        size_t b = (n + (size_t)vv::RED_THREADS * 8 - 1) / ((size_t)vv::RED_THREADS * 8);
        c->npart = (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)c->npart_max));
    }
    c->mom_seg = 64;
    c->mom_S = (nv + c->mom_seg - 1) / c->mom_seg;
    c->pcR = std::max(1, 4096 / nx);
    if (c->pcR > 64) c->pcR = 64;
    c->smem_rfft = (size_t)c->pcR * M * sizeof(double2);
    c->smem_irfft = (size_t)c->pcR * (2 * M + 1) * sizeof(double2);
    c->smem_tri = (size_t)nv * sizeof(double2);
    c->smem_pois = (size_t)M * sizeof(double2) + (size_t)nx * sizeof(double) + (size_t)(nx + 2) * sizeof(double);

    int s = VV_OK;
    const int tiles = bracket_tiles(c);
    const size_t part_count = std::max({(size_t)(vv::MAX_RESTART + 2) * c->npart_max, (size_t)tiles,
                                        (size_t)vv::INV_NPART * c->npart_max});
    if ((s = dalloc(&c->v, nv)) || (s = dalloc(&c->h0, nv)) || (s = dalloc(&c->hxp, 4 * (size_t)nx)) ||
        (s = dalloc(&c->Fh, n)) || (s = dalloc(&c->tmp, n)) || (s = dalloc(&c->bvec, n)) ||
        (s = dalloc(&c->delta, n)) || (s = dalloc(&c->fl, n)) || (s = dalloc(&c->V, (size_t)(restart + 1) * n)) ||
        (s = dalloc(&c->part, part_count)) || (s = dalloc(&c->scal, 64)) || (s = dalloc(&c->xscratch, 2 * (size_t)nx)) ||
        (s = dalloc(&c->mom_part, (size_t)c->mom_S * 3 * nx)) || (s = dalloc(&c->spec, (size_t)nm * nv)) ||
        (s = dalloc(&c->tw, (size_t)std::max(1, nx / 2))) || (s = dalloc(&c->lambda, nm)) ||
        (s = dalloc(&c->dinv, (size_t)nm * nv)) || (s = dalloc(&c->alpha, nv)) || (s = dalloc(&c->gamma, nv)) ||
        (s = dalloc(&c->sym_inv, nm)) || (s = dalloc(&c->gm, 1))) {
        vv_destroy(c);
        return s;
    }
    if (cudaMallocHost((void**)&c->hpin, sizeof(vv::GmresState) + 256) != cudaSuccess ||
        cudaMallocHost((void**)&c->hstat, 64) != cudaSuccess) {
        vv_destroy(c);
        return VV_ERR_ALLOC;
    }

    // ---- host precomputation ----
    std::vector<double> hv_(nv), h0_(nv), alpha(nv), gamma(nv);
    for (int j = 0; j < nv; ++j) {
        hv_[j] = g.vmin + (double)j * c->hv;              // vmin + j*hv
        h0_[j] = 0.5 * (hv_[j] * hv_[j]) * g.mass;        // Toolbox.pyx:187
    }
    const long double PI = 3.141592653589793238462643383279502884L;
    std::vector<double2> tw(std::max(1, nx / 2));
    for (int k = 0; k < nx / 2; ++k) {
        const long double a = 2.0L * PI * (long double)k / (long double)nx;
        tw[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
    }
    // eigenvalues (TensorProduct.pyx:109-116), including ifftshift
    std::vector<cd> e(nx), lam(nm);
    const double twopi = 2.0 * M_PI;
    for (int i = 0; i < nx; ++i) {
        const double t2 = (twopi * (double)i) / (double)nx;
        const double t1 = t2 * (double)(nx - 1);
        e[i] = cd(std::cos(t1), std::sin(t1)) - cd(std::cos(t2), std::sin(t2));
    }
    for (int k = 0; k < nm; ++k) lam[k] = e[(k + nx / 2) % nx];
    // band matrix (TensorProductKineticFast.pyx:248-272) and its LU without pivoting
    const double arak = 0.5 * c->hx_inv * c->hv_inv / 12.;
    const double hv2 = c->hv * c->hv;
    for (int j = 0; j < nv; ++j) {
        alpha[j] = 0.5 * (2. * c->hv * hv_[j] - hv2) * arak;
        gamma[j] = 0.5 * (2. * c->hv * hv_[j] + hv2) * arak;
    }
    std::vector<double2> dinv((size_t)nm * nv);
    std::vector<double2> lam2(nm);
    bool piv = false;
    for (int k = 0; k < nm; ++k) {
        const cd L = lam[k];
        lam2[k] = make_double2(L.real(), L.imag());
        cd dprev;
        for (int r = 0; r < nv; ++r) {
            const cd diag = L * 1.0 * (4. * c->hv * hv_[r]) * arak + c->ht_inv;
            cd d = diag;
            if (r > 0) {
                const cd sub = L * 0.5 * (2. * c->hv * hv_[r] - hv2) * arak;   // A[r, r-1]
                const cd sup = L * 0.5 * (2. * c->hv * hv_[r - 1] + hv2) * arak;  // A[r-1, r]
                // LAPACK's zgbtf2 pivots when |sub|_1 > |U_{r-1}|_1 (cabs1)
                if (std::fabs(sub.real()) + std::fabs(sub.imag()) > std::fabs(dprev.real()) + std::fabs(dprev.imag()))
                    piv = true;
                const cd l = sub * (1.0 / dprev);
                d = diag - l * sup;
            }
            if (d == cd(0.0, 0.0)) {
                snprintf(g_err, sizeof g_err, "zero pivot in preconditioner mode %d row %d", k, r);
                vv_destroy(c);
                return VV_ERR_ARG;
            }
            const cd di = 1.0 / d;
            dinv[(size_t)k * nv + r] = make_double2(di.real(), di.imag());
            dprev = d;
        }
    }
    c->pivot_differs = piv;
    // CFD4 symbol (PETScPoissonCFD4.pyx:130-134): (54 - 64 cos t + 10 cos 2t)/(12 hx^2)
    std::vector<double> sym(nm);
    for (int k = 0; k < nm; ++k) {
        const long double t = 2.0L * PI * (long double)k / (long double)nx;
        const long double s_ = (54.0L - 64.0L * cosl(t) + 10.0L * cosl(2.0L * t)) * (long double)c->hx2_inv / 12.0L;
        sym[k] = (k == 0) ? 0.0 : (double)(1.0L / s_);
    }
    std::vector<double2> lam_h(lam2);
    if (cudaMemcpy(c->v, hv_.data(), nv * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->h0, h0_.data(), nv * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->alpha, alpha.data(), nv * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->gamma, gamma.data(), nv * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->lambda, lam_h.data(), nm * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->dinv, dinv.data(), dinv.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->sym_inv, sym.data(), nm * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(c->hxp, 0, 4 * (size_t)nx * sizeof(double)) != cudaSuccess ||
        cudaMemset(c->Fh, 0, n * sizeof(double)) != cudaSuccess) {
        vv_destroy(c);
        return fail_cuda(cudaGetLastError(), "vv_create upload");
    }
    // dynamic shared memory limits
    if (cudaFuncSetAttribute(vv::k_rfft_rows<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)c->smem_rfft) != cudaSuccess ||
        cudaFuncSetAttribute(vv::k_irfft_rows<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)c->smem_irfft) != cudaSuccess ||
        cudaFuncSetAttribute(vv::k_tridiag_modes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)c->smem_tri) != cudaSuccess ||
        cudaFuncSetAttribute(vv::k_moments_poisson, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)c->smem_pois) != cudaSuccess) {
        vv_destroy(c);
        return fail_cuda(cudaGetLastError(), "cudaFuncSetAttribute");
    }
    *out = c;
    return VV_OK;
}

int vv_destroy(vv_ctx* c) {
    if (!c) return VV_OK;
    void* bufs[] = {c->v, c->h0, c->hxp, c->Fh, c->tmp, c->bvec, c->delta, c->fl, c->V, c->part, c->scal,
                    c->xscratch, c->mom_part, c->spec, c->tw, c->lambda, c->dinv, c->alpha, c->gamma,
                    c->sym_inv, c->gm};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (c->hpin) cudaFreeHost(c->hpin);
    if (c->hstat) cudaFreeHost(c->hstat);
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    delete c;
    return VV_OK;
}

int vv_set_stream(vv_ctx* c, void* stream) {
    if (!c) return VV_ERR_ARG;
    c->st = (cudaStream_t)stream;
    return VV_OK;
}

int vv_grid_vectors(vv_ctx* c, double* v_host, double* h0_host) {
    if (!c) return VV_ERR_ARG;
    if (v_host) CK(cudaMemcpy(v_host, c->v, c->nv * sizeof(double), cudaMemcpyDeviceToHost));
    if (h0_host) CK(cudaMemcpy(h0_host, c->h0, c->nv * sizeof(double), cudaMemcpyDeviceToHost));
    return VV_OK;
}

int vv_update_history(vv_ctx* c, const double* F) {
    if (!c || !F) return VV_ERR_ARG;
    return copy_d(c, c->Fh, F, c->ncell);
}

int vv_update_previous(vv_ctx* c, const double* h1p, const double* h1h, const double* h2p, const double* h2h) {
    if (!c) return VV_ERR_ARG;
    return set_hxp(c, h1p, h1h, h2p, h2h);
}

int vv_function(vv_ctx* c, const double* F, double* Y, int apply_pc) {
    if (!c || !F || !Y) return VV_ERR_ARG;
    const bool pc = apply_pc && c->g.preconditioner == VV_PC_TENSOR_KINETIC;
    TRY(launch_bracket<vv::MODE_RESIDUAL>(c, F, c->Fh, pc ? c->tmp : Y, 1.0, nullptr));
    if (pc) TRY(pc_apply(c, c->tmp, Y));
    return VV_OK;
}

int vv_jacobian(vv_ctx* c, const double* F, double* Y, int apply_pc) {
    if (!c || !F || !Y) return VV_ERR_ARG;
    const bool pc = apply_pc && c->g.preconditioner == VV_PC_TENSOR_KINETIC;
    TRY(launch_bracket<vv::MODE_JVP>(c, F, nullptr, pc ? c->tmp : Y, 0.5, nullptr));
    if (pc) TRY(pc_apply(c, c->tmp, Y));
    return VV_OK;
}

int vv_function_norm(vv_ctx* c, const double* F, double* Y, double* norm) {
    if (!c || !F || !Y || !norm) return VV_ERR_ARG;
    return residual_norm(c, F, Y, norm);
}

int vv_bracket(vv_ctx* c, const double* X, double* Y, double factor) {
    if (!c || !X || !Y) return VV_ERR_ARG;
    return launch_bracket<vv::MODE_ADD>(c, X, nullptr, Y, factor, nullptr);
}

int vv_pc_apply(vv_ctx* c, const double* X, double* Y) {
    if (!c || !X || !Y) return VV_ERR_ARG;
    if (c->g.preconditioner != VV_PC_TENSOR_KINETIC) return copy_d(c, Y, X, c->ncell);
    return pc_apply(c, X, Y);
}

int vv_moments(vv_ctx* c, const double* F, double* n, double* u, double* e, double* a) {
    if (!c || !F) return VV_ERR_ARG;
    return moments_poisson(c, F, n, u, e, a, nullptr, nullptr, nullptr);
}

int vv_potential_to_hamiltonian(vv_ctx* c, const double* phi, double* h1) {
    if (!c || !phi || !h1) return VV_ERR_ARG;
    vv::k_xprofile<<<1, 1024, 0, c->st>>>(phi, c->nx, c->g.charge, c->hx, h1, c->scal + 8);
    CKL(c);
    return VV_OK;
}

int vv_poisson_rhs(vv_ctx* c, const double* n, double* b) {
    if (!c || !n || !b) return VV_ERR_ARG;
    return poisson_apply(c, nullptr, n, b, 0, nullptr);
}

int vv_poisson_matvec(vv_ctx* c, const double* x, double* y) {
    if (!c || !x || !y) return VV_ERR_ARG;
    return poisson_apply(c, x, nullptr, y, 1, nullptr);
}

int vv_poisson_function(vv_ctx* c, const double* x, const double* n, double* y) {
    if (!c || !x || !n || !y) return VV_ERR_ARG;
    return poisson_apply(c, x, n, y, 2, nullptr);
}

int vv_poisson_solve(vv_ctx* c, const double* n, double* phi) {
    if (!c || !n || !phi) return VV_ERR_ARG;
    vv::k_moments_poisson<<<1, vv::POIS_THREADS, c->smem_pois, c->st>>>(nullptr, n, nullptr, nullptr, nullptr, nullptr,
                                                                        phi, nullptr, c->scal, pparams(c));
    CKL(c);
    return VV_OK;
}

int vv_gmres(vv_ctx* c, const double* b, double* x, const vv_ksp_opts* o, vv_ksp_result* r) {
    if (!c || !b || !x || !o || !r) return VV_ERR_ARG;
    return gmres(c, b, x, o, r);
}

int vv_calculate_moments(vv_ctx* c, vv_state* st) {
    if (!c || !st || !st->f) return VV_ERR_ARG;
    return calc_moments(c, st);
}

int vv_calculate_residual(vv_ctx* c, vv_state* st, double* out) {
    if (!c || !st || !out || !st->f || !st->phi || !st->n) return VV_ERR_ARG;
    return calc_residual(c, st, out);
}

int vv_run_init(vv_ctx* c, vv_state* st, int normalise) {
    if (!c || !st || !st->f || !st->phi || !st->h1c || !st->n) return VV_ERR_ARG;
    if (normalise) {
        // nave = sum(f)*hv/nx ; f *= 1/nave   (run_base.py:623-628)
        vv::k_sum_partial<double><<<c->npart, vv::RED_THREADS, 0, c->st>>>(st->f, c->ncell, c->part);
        CKL(c);
        TRY(reduce_to(c, c->part, c->npart, c->scal + 4));
        double sum = 0.0;
        TRY(read_scalar(c, c->scal + 4, &sum));
        const double nave = sum * c->hv / c->nx;
        vv::k_scale<double, double><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(st->f, st->f, c->ncell, nullptr,
                                                                            1. / nave);
        CKL(c);
    }
    TRY(calc_moments(c, st));
    CK(cudaStreamSynchronize(c->st));
    return VV_OK;
}

int vv_step(vv_ctx* c, vv_state* st, const vv_snes_opts* so, const vv_ksp_opts* ko, vv_step_report* rep) {
    if (!c || !st || !so || !ko || !rep || !st->f || !st->fh || !st->phi || !st->h1c || !st->h1h || !st->n)
        return VV_ERR_ARG;
    std::memset(rep, 0, sizeof(*rep));
    const size_t n = c->ncell;
    const int nx = c->nx;
    // make_history (run_base.py:749-763) + update_history (PETScVlasovSolver.pyx:135-140)
    TRY(copy_d(c, st->fh, st->f, n));
    TRY(copy_d(c, st->h1h, st->h1c, nx));
    if (st->h2c && st->h2h) TRY(copy_d(c, st->h2h, st->h2c, nx));
    if (st->phih) TRY(copy_d(c, st->phih, st->phi, nx));
    TRY(copy_d(c, c->Fh, st->f, n));
    // update_previous
    TRY(set_hxp(c, st->h1c, st->h1h, st->h2c, st->h2h));
    double pred = 0.0;
    TRY(calc_residual(c, st, &pred));
    rep->residual[0] = pred;
    int i = 0;
    for (;;) {
        ++i;
        TRY(copy_d(c, c->fl, st->f, n));
        // snes ksponly: b = P^-1 R(f); GMRES; f -= delta unless the solve failed.
        // calc_residual left R(f) -- evaluated with the same Fh and Have -- in tmp.
        if (c->g.preconditioner == VV_PC_TENSOR_KINETIC) TRY(pc_apply(c, c->tmp, c->bvec));
        else TRY(copy_d(c, c->bvec, c->tmp, n));
        vv_ksp_result kr{};
        TRY(gmres(c, c->bvec, c->delta, ko, &kr));
        if (i - 1 < VV_MAX_PICARD) {
            rep->gmres_its[i - 1] = kr.its;
            rep->ksp_reason[i - 1] = kr.reason;
        }
        rep->gmres_its_total += kr.its;
        if (kr.reason >= 0) {
            vv::k_axpby<double><<<grid1d(n, 256), 256, 0, c->st>>>(c->delta, st->f, n, -1.0, 1.0);
            CKL(c);
        } else {
            rep->ksp_failures++;
        }
        TRY(calc_moments(c, st));
        TRY(set_hxp(c, st->h1c, st->h1h, st->h2c, st->h2h));
        const double prev = pred;
        TRY(calc_residual(c, st, &pred));
        if (i < VV_MAX_PICARD + 1) rep->residual[i] = pred;
        const bool rose = pred > prev && i > 1;
        const bool small = pred < so->atol;
        const bool maxed = i >= so->max_iter || i >= VV_MAX_PICARD;
        if (rose || small || maxed) {
            rep->stop_rule = rose ? 1 : (small ? 2 : 3);
            if (pred > prev) {
                TRY(copy_d(c, st->f, c->fl, n));
                TRY(calc_moments(c, st));
                rep->reverted = 1;
            }
            break;
        }
    }
    rep->picard_its = i;
    CK(cudaStreamSynchronize(c->st));
    if (std::isnan(pred)) return VV_ERR_NAN;
    if (pred > so->abort_residual) {
        rep->aborted = 1;
        return VV_ERR_DIVERGED;
    }
    return VV_OK;
}

int vv_invariants(vv_ctx* c, const double* f, const double* phi, const double* h2, vv_invariant_set* out) {
    if (!c || !f || !phi || !out) return VV_ERR_ARG;
    double* h1 = c->xscratch;
    vv::k_xprofile<<<1, 1024, 0, c->st>>>(phi, c->nx, c->g.charge, c->hx, h1, c->scal + 16);
    CKL(c);
    vv::k_invariants_partial<<<c->npart, vv::RED_THREADS, 0, c->st>>>(f, c->nx, c->nv, c->v, c->h0, h1, h2, c->part);
    CKL(c);
    vv::k_invariants_final<<<1, vv::RED_THREADS, 0, c->st>>>(c->part, c->npart, c->scal + 20);
    CKL(c);
    CK(cudaMemcpyAsync(c->hpin, c->scal + 16, 24 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double fe = c->hpin[0];
    const double* s = c->hpin + 4;
    const double hx = c->hx, hv = c->hv, hxhv = hx * hv;
    out->mass = s[0] * 0.25 * hx * hv;
    out->L1 = hxhv * s[1];
    out->L2 = hxhv * s[2];
    out->L3 = hxhv * s[3];
    out->L4 = hxhv * s[4];
    out->L5 = hxhv * s[5];
    out->L6 = hxhv * s[6];
    out->L8 = hxhv * s[7];
    out->entropy = -hx * hv * s[8];
    out->E_kin = s[9] * hx * hv;
    out->E_pot = (s[10] + s[11]) * hx * hv;
    out->energy = out->E_kin + 0.5 * out->E_pot;
    out->momentum = s[12] * c->g.mass * hx * hv;
    out->Lmin = s[13] * hx * hv;
    out->Lmax = s[14] * hx * hv;
    out->field_energy = fe;
    return VV_OK;
}

int vv_timing_enable(vv_ctx* c, int enable) {
    if (!c) return VV_ERR_ARG;
    c->timing = enable != 0;
    return VV_OK;
}

int vv_timing_read(vv_ctx* c, int64_t* launches, double* total_ms, int reset) {
    if (!c) return VV_ERR_ARG;
    TRY(drain_timing(c));
    if (launches) *launches = c->t_launches;
    if (total_ms) *total_ms = c->t_ms;
    if (reset) {
        c->t_launches = 0;
        c->t_ms = 0.0;
    }
    return VV_OK;
}

int vv_launch_count(vv_ctx* c, int64_t* launches, int reset) {
    if (!c) return VV_ERR_ARG;
    if (launches) *launches = c->launches;
    if (reset) c->launches = 0;
    return VV_OK;
}

}  // extern "C"
