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
#include "vv_batch.cuh"
#include "vv_adjoint.cuh"
#include "vv_pcv.cuh"
#include "vv_coll.cuh"
#include "vv_pred.cuh"

#include <algorithm>
#include <array>
#include <cstdlib>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

using cd = std::complex<double>;

struct vv_ctx {
    vv_grid g;
    int nx, nv, M, logM, nmodes, restart;
    size_t ncell;
    double hx, hv, ht_inv, hx_inv, hv_inv, hx2_inv, f1, f2;
    double lap[4];   // the Laplacian: stencil a0, a1, a2 and denominator (x hx^-2)
    double ravg[4];  // the right-hand side's density average: r0, r1, r2, denominator
    int avg;         // the time derivative (vv::AvgKind; arakawa_J2 -> point)
    double tfac;     // ht_inv / divisor of the averaging stencil
    // collisions (vv::CollKind; none unless dissipation 'collisions' with
    // coll_freq != 0): the factors for the midpoint weight 1/2, the current
    // moments in use (the state's inside vv_step, mom_p after vv_set_moments)
    // and the history moments (mom_h, copied at make_history); n, U, a each
    int coll;
    double coll_drag_fac, coll_diff_fac;
    vv::CollMoments coll_p, coll_h;
    double *mom_p, *mom_h;
    // double bracket (dissipation_type = 'double_bracket'; 0 none, 1 ffh, 2 fhh,
    // FP64): nu = coll_freq, the residual's Fave (kept for the Jacobian) and
    // the inner bracket
    int db;
    double db_nu;
    double *db_fave, *db_b;
    // explicit predictor of the initial guess (vv_pred.cuh): method, iterations,
    // h fields (kinetic, potential or RK), bracket output, RK stages, stage
    // input, the saved iterate, collision-only residual partials
    int pred, pred_iter;
    double *pred_H, *pred_Hp, *pred_Y, *pred_K, *pred_S, *pred_fl, *pred_cpart, *pred_zero;
    // non-null: the bracket kernels run in the reference order with this h
    // field (the predictor's residual with a zero Have)
    const double* zero_h;
    // the potential preconditioner (VV_PC_TENSOR_POTENTIAL): v modes, eigenvalues
    // for n = nv, nv twiddles, transposed field, v spectrum, elimination
    // scratch (FP32 copies in the mixed mode), rows per CTA of the v FFT, phi
    int nmv, pvR;
    double2 *lamv, *twv, *pv_spec, *pv_scr;
    double *pv_xt, *phipc;
    float2 *twv32, *pv_spec32, *pv_scr32;
    float* pv_xt32;
    cudaStream_t st;      // the caller's stream
    int device;
    // device buffers
    double *v, *h0, *hxp, *Fh, *tmp, *bvec, *delta, *fl, *V, *part, *scal, *xscratch, *mom_part;
    double2 *spec, *tw, *lambda, *dinv;
    double *alpha, *gamma, *sym_inv;
    vv::DevState* ds;
    // single-precision operands of the mixed mode (GMRES basis, JVP, preconditioner)
    bool mixed;
    float *V32, *tmp32, *bvec32, *delta32, *alpha32, *gamma32;
    float2 *spec32, *tw32, *lambda32, *dinv32;
    size_t smem_rfft32, smem_irfft32, smem_tri32;
    bool tri_stage32;
    // kernel variants (picked by the autotuner at vv_create)
    int fft_kind;      // 0: shared-memory radix-2 per warp, 1: four-step register/shuffle FFT,
                       // 2: direct DFT (the only kind for nx that is not a power of two)
    bool pow2;         // nx a power of two
    int tri_kind;      // 0: one CTA per mode (block scan), 1: one warp per mode (lines staged in shared
                       // memory when tri_ws_smem fits smem_limit)
    int smem_limit;    // dynamic shared memory per block on this device
    int narrow_bracket;  // 1: 32x16 tiles instead of 64x32
    int march;           // Jacobian stencil: 0 tiles, 128 or 256 the strip width of the marching kernel
    // pinned host staging
    double* hpin;
    int* hstat;
    vv::DevState* hds;    // pinned copy of the device state (report read-back)
    // launch configuration
    int npart, npart_max;
    int mom_S, mom_seg;
    int pcR;
    size_t smem_rfft, smem_irfft, smem_tri, smem_pois;
    bool tri_stage;
    bool pivot_differs;
    // timing of the JVP stencil kernel (host-driven path)
    bool timing;
    std::vector<cudaEvent_t> ev;
    size_t ev_used;
    int64_t t_launches;
    double t_ms;
    int64_t launches;
    // graph of one time step
    bool use_graph;
    cudaStream_t cs[4];
    cudaGraph_t step_graph;
    cudaGraphExec_t step_exec;
    vv_state step_key;         // state pointers the graph was captured with
    unsigned long long hnd[5]; // h_gm_outer, h_gm_inner, h_gm_first, h_pic, h_revert
    cudaGraph_t cap_owner;     // top-level graph of the capture in progress
    bool opts_valid;           // last uploaded options still in the device state
    vv_ksp_opts last_ksp;
    vv_snes_opts last_snes;
    unsigned long long last_hnd[5];
    unsigned long long step_hnd[5];  // handles of this context's own step graph
    // kernels per region of the step graph (for launch accounting)
    int nk_top, nk_pic, nk_cycle, nk_restart, nk_arnoldi, nk_revert;
    // discrete adjoint (allocated at the first adjoint call): GMRES operator
    // switch, coefficient planes of J_H^T and J_Fbar^T, Poisson-chain scratch
    bool adj;
    double *adj_cH, *adj_cF, *adj_zpart, *adj_zbuf, *adj_q, *adj_hprof, *adj_h1a, *adj_h1b;
};

namespace {

thread_local char g_err[256];

int fail_cuda(cudaError_t e, const char* what) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return VV_ERR_CUDA;
}

template <typename... A>
int fail(int status, const char* fmt, A... args) {
    snprintf(g_err, sizeof g_err, fmt, args...);
    return status;
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
#define TRY(...)                    \
    do {                            \
        int s_ = (__VA_ARGS__);     \
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
    p.tfac = c->tfac;
    p.factor = factor;
    p.f1 = c->f1;
    p.f2 = c->f2;
    p.hx_inv = c->hx_inv;
    p.hv_inv = c->hv_inv;
    p.h0 = c->h0;
    p.hxp = c->hxp;
    p.xidx = nullptr;
    p.xstride = 0;
    p.hfield = nullptr;
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
    p.yidx = nullptr;
    p.yoff = 0;
    p.ystride = 0;
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
bool aligned16(const void* p) { return p == nullptr || ((uintptr_t)p & 15u) == 0; }

// the wide tiles; with an averaged time derivative or collisions only for
// the Jacobian (the residual, Xh != null, stages F - Fh in the narrow tiles,
// or takes its partial sums from the collision kernel's narrow tiling)
bool wide_ok(const vv_ctx* c, const void* X, const void* Xh, const void* Y) {
    return !c->narrow_bracket && c->nx % vv::WX == 0 && aligned16(X) && aligned16(Xh) && aligned16(Y) &&
           !((c->avg != vv::AVG_POINT || c->coll != vv::COLL_NONE || c->db != 0) && Xh != nullptr);
}

// the marching Jacobian stencil: about two waves of CTAs, segments of whole chunks
template <int SCHEME, typename T, int MW>
int launch_march(vv_ctx* c, const T* X, T* Y, const vv::BracketParams& p) {
    const size_t smem = vv::MarchRow<T, MW>::smem_bytes();
    constexpr int CH = vv::MarchShape<T>::CH;
    int per_sm = 0, nsm = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vv::k_bracket_march<SCHEME, T, MW>, MW, smem);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    const int strips = c->nx / MW;
    const long target = 2L * nsm * std::max(1, per_sm);
    const int nseg = (int)std::max<long>(1, (target + strips - 1) / strips);
    int seg = (c->nv + nseg - 1) / nseg;
    seg = std::max(CH, (seg + CH - 1) / CH * CH);
    const dim3 grid(strips, (c->nv + seg - 1) / seg);
    vv::k_bracket_march<SCHEME, T, MW><<<grid, MW, smem, c->st>>>(X, Y, p, seg);
    return VV_OK;
}

// X may be a GMRES basis base pointer with xidx -> the vector index in the state;
// AVG: the time derivative (vv::AvgKind)
template <int SCHEME, int MODE, typename T, int AVG>
int launch_bracket_a(vv_ctx* c, const T* X, const T* Xh, T* Y, double factor, double* sumsq, const int* xidx) {
    dim3 grid((c->nx + vv::BX - 1) / vv::BX, (c->nv + vv::BY - 1) / vv::BY);
    dim3 block(vv::BX, vv::TY);
    vv::BracketParams p = bparams(c, factor);
    p.xidx = xidx;
    p.xstride = xidx ? c->ncell : 0;
    const bool timed = c->timing && MODE == vv::MODE_JVP;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timed) {
        if (c->ev_used + 2 > 8192) TRY(drain_timing(c));
        e0 = next_event(c);
        e1 = next_event(c);
        if (e0) cudaEventRecord(e0, c->st);
    }
    bool done = false;
    if constexpr (std::is_same<T, double>::value) {
        if (c->g.order == VV_ORDER_REFERENCE || c->zero_h) {
            p.hfield = c->zero_h;
            vv::k_bracket_ref<SCHEME, MODE, AVG><<<grid, block, 0, c->st>>>(X, Xh, Y, p, sumsq);
            done = true;
        }
    }
    if (!done && MODE == vv::MODE_JVP && AVG == vv::AVG_POINT && c->march && c->g.order != VV_ORDER_REFERENCE &&
        c->nx % c->march == 0 && aligned16(X) && aligned16(Y)) {
        TRY(c->march == 256 ? launch_march<SCHEME, T, 256>(c, X, Y, p) : launch_march<SCHEME, T, 128>(c, X, Y, p));
        done = true;
    }
    if (!done) {
        if constexpr (AVG == vv::AVG_POINT || MODE == vv::MODE_JVP) {
            if (wide_ok(c, X, Xh, Y)) {
                dim3 gw(c->nx / vv::WX, (c->nv + vv::WY - 1) / vv::WY);
                vv::k_bracket_wide<SCHEME, MODE, T, AVG><<<gw, vv::WTHREADS, 0, c->st>>>(X, Xh, Y, p, sumsq);
                done = true;
            }
        }
        if (!done) vv::k_bracket_fac<SCHEME, MODE, T, AVG><<<grid, block, 0, c->st>>>(X, Xh, Y, p, sumsq);
    }
    CKL(c);
    if (timed && e1) cudaEventRecord(e1, c->st);
    return VV_OK;
}

// the Simpson bracket: one kernel in the reference's operation order for
// every order setting and precision (BX x BY tiles)
template <int MODE, typename T, int AVG>
int launch_simpson(vv_ctx* c, const T* X, const T* Xh, T* Y, double factor, double* sumsq, const int* xidx) {
    dim3 grid((c->nx + vv::BX - 1) / vv::BX, (c->nv + vv::BY - 1) / vv::BY);
    dim3 block(vv::BX, vv::TY);
    vv::BracketParams p = bparams(c, factor);
    p.xidx = xidx;
    p.xstride = xidx ? c->ncell : 0;
    if constexpr (std::is_same<T, double>::value) p.hfield = c->zero_h;
    vv::k_bracket_simpson<MODE, T, AVG><<<grid, block, 0, c->st>>>(X, Xh, Y, p, sumsq);
    CKL(c);
    return VV_OK;
}

template <int MODE, typename T, int AVG>
int launch_bracket_avg(vv_ctx* c, const T* X, const T* Xh, T* Y, double factor, double* sumsq, const int* xidx) {
    switch (c->g.bracket) {
        case VV_BRACKET_SIMPSON: return launch_simpson<MODE, T, AVG>(c, X, Xh, Y, factor, sumsq, xidx);
        case VV_BRACKET_J1: return launch_bracket_a<1, MODE, T, AVG>(c, X, Xh, Y, factor, sumsq, xidx);
        case VV_BRACKET_J2: return launch_bracket_a<2, MODE, T, AVG>(c, X, Xh, Y, factor, sumsq, xidx);
        default: return launch_bracket_a<4, MODE, T, AVG>(c, X, Xh, Y, factor, sumsq, xidx);
    }
}

// MODE_ADD (the bare bracket) has no time derivative
template <int MODE, typename T>
int launch_bracket_td(vv_ctx* c, const T* X, const T* Xh, T* Y, double factor, double* sumsq, const int* xidx) {
    if constexpr (MODE != vv::MODE_ADD) {
        switch (c->avg) {
            case vv::AVG_MIDPOINT:
                return launch_bracket_avg<MODE, T, vv::AVG_MIDPOINT>(c, X, Xh, Y, factor, sumsq, xidx);
            case vv::AVG_SIMPSON:
                return launch_bracket_avg<MODE, T, vv::AVG_SIMPSON>(c, X, Xh, Y, factor, sumsq, xidx);
            case vv::AVG_J4: return launch_bracket_avg<MODE, T, vv::AVG_J4>(c, X, Xh, Y, factor, sumsq, xidx);
            default: break;
        }
    }
    return launch_bracket_avg<MODE, T, vv::AVG_POINT>(c, X, Xh, Y, factor, sumsq, xidx);
}

// Y += C_p[X] (+ C_h[Xh]) after the bracket, per-tile sums of squares of Y on
// the narrow tiling (PETScNLVlasovMP.pyx:33-58 adds the collision operator
// after the bracket; CollisionOperator.pyx:72-110, :164-202)
template <typename T>
int launch_collision(vv_ctx* c, const T* X, const T* Xh, T* Y, double* sumsq, const int* xidx) {
    vv::CollParams p;
    p.nx = c->nx;
    p.nv = c->nv;
    p.kind = c->coll;
    p.drag_fac = c->coll_drag_fac;
    p.diff_fac = c->coll_diff_fac;
    p.v = c->v;
    p.xidx = xidx;
    p.xstride = xidx ? c->ncell : 0;
    dim3 grid((c->nx + vv::BX - 1) / vv::BX, (c->nv + vv::BY - 1) / vv::BY);
    vv::k_collision<T><<<grid, dim3(vv::BX, vv::TY), 0, c->st>>>(X, Xh, Y, p, c->coll_p, c->coll_h, sumsq);
    CKL(c);
    return VV_OK;
}

// Y += factor [X, H] in the reference order (FP64, narrow tiles) with H the
// profiles (hfield null) or a general field: the double bracket's brackets
int launch_bracket_gen(vv_ctx* c, const double* X, const int* xidx, double* Y, const double* hfield, double factor,
                       double* sumsq) {
    dim3 grid((c->nx + vv::BX - 1) / vv::BX, (c->nv + vv::BY - 1) / vv::BY);
    dim3 block(vv::BX, vv::TY);
    vv::BracketParams p = bparams(c, factor);
    p.xidx = xidx;
    p.xstride = xidx ? c->ncell : 0;
    p.hfield = hfield;
    switch (c->g.bracket) {
        case VV_BRACKET_SIMPSON:
            vv::k_bracket_simpson<vv::MODE_ADD, double><<<grid, block, 0, c->st>>>(X, nullptr, Y, p, sumsq);
            break;
        case VV_BRACKET_J1: vv::k_bracket_ref<1, vv::MODE_ADD><<<grid, block, 0, c->st>>>(X, nullptr, Y, p, sumsq); break;
        case VV_BRACKET_J2: vv::k_bracket_ref<2, vv::MODE_ADD><<<grid, block, 0, c->st>>>(X, nullptr, Y, p, sumsq); break;
        default: vv::k_bracket_ref<4, vv::MODE_ADD><<<grid, block, 0, c->st>>>(X, nullptr, Y, p, sumsq); break;
    }
    CKL(c);
    return VV_OK;
}

__global__ void k_fave(const double* __restrict__ F, const double* __restrict__ Fh, double* __restrict__ Fave, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        Fave[i] = __dadd_rn(__dmul_rn(0.5, Fh[i]), __dmul_rn(0.5, F[i]));   // Fave.set(0); axpy(.5, Fh); axpy(.5, F)
}

// the double bracket after the bracket (PETScNLVlasovMP.pyx:33-58): the
// residual stores Fave and adds DoubleBracket.function(Fave, Have, Y, 1);
// the Jacobian adds DoubleBracket.jacobian(X, Fave, Have, Y, 1/2)
// (DoubleBracket.pyx:69-97); sumsq from the last launch
int db_apply(vv_ctx* c, int mode, const double* X, const double* Xh, const int* xidx, double* Y, double* sumsq) {
    const size_t bytes = c->ncell * sizeof(double);
    double* B = c->db_b;
    const double* Fa = c->db_fave;
    if (mode == vv::MODE_RESIDUAL) {
        k_fave<<<grid1d(c->ncell, 256), 256, 0, c->st>>>(X, Xh, c->db_fave, c->ncell);
        CKL(c);
        CK(cudaMemsetAsync(B, 0, bytes, c->st));
        TRY(launch_bracket_gen(c, Fa, nullptr, B, nullptr, 1.0, nullptr));                 // B = [Fave, Have]
        if (c->db == 1) return launch_bracket_gen(c, Fa, nullptr, Y, B, -c->db_nu * 1.0, sumsq);   // [Fave, B]
        return launch_bracket_gen(c, B, nullptr, Y, nullptr, -c->db_nu * 1.0, sumsq);             // [B, Have]
    }
    const double f = -c->db_nu * 0.5;
    CK(cudaMemsetAsync(B, 0, bytes, c->st));
    if (c->db == 1) {
        TRY(launch_bracket_gen(c, Fa, nullptr, B, nullptr, 1.0, nullptr));    // B = [Fave, Have]
        TRY(launch_bracket_gen(c, X, xidx, Y, B, f, nullptr));                // Y += f [X, B]
        CK(cudaMemsetAsync(B, 0, bytes, c->st));
        TRY(launch_bracket_gen(c, X, xidx, B, nullptr, 1.0, nullptr));        // B = [X, Have]
        return launch_bracket_gen(c, Fa, nullptr, Y, B, f, sumsq);            // Y += f [Fave, B]
    }
    TRY(launch_bracket_gen(c, X, xidx, B, nullptr, 1.0, nullptr));            // B = [X, Have]
    return launch_bracket_gen(c, B, nullptr, Y, nullptr, f, sumsq);           // Y += f [B, Have]
}

// the residual (MODE_RESIDUAL) or Jacobian (MODE_JVP) of the chosen
// discretisation, or the bare bracket (MODE_ADD); with a double bracket or
// collisions the residual's partial sums come from the last kernel
template <int MODE, typename T>
int launch_bracket(vv_ctx* c, const T* X, const T* Xh, T* Y, double factor, double* sumsq,
                   const int* xidx = nullptr) {
    const bool coll = MODE != vv::MODE_ADD && c->coll != vv::COLL_NONE;
    const bool db = MODE != vv::MODE_ADD && c->db != 0 && std::is_same<T, double>::value;
    TRY(launch_bracket_td<MODE, T>(c, X, Xh, Y, factor, (coll || db) ? nullptr : sumsq, xidx));
    if constexpr (std::is_same<T, double>::value) {
        if (db) TRY(db_apply(c, MODE, X, Xh, xidx, Y, coll ? nullptr : sumsq));
    }
    if (coll) return launch_collision<T>(c, X, MODE == vv::MODE_RESIDUAL ? Xh : nullptr, Y, sumsq, xidx);
    return VV_OK;
}

// number of per-CTA partials a bracket launch writes for these operands
int bracket_tiles(const vv_ctx* c, const void* X = nullptr, const void* Xh = nullptr, const void* Y = nullptr) {
    if (c->g.order != VV_ORDER_REFERENCE && c->g.bracket != VV_BRACKET_SIMPSON && wide_ok(c, X, Xh, Y))
        return (c->nx / vv::WX) * ((c->nv + vv::WY - 1) / vv::WY);
    return ((c->nx + vv::BX - 1) / vv::BX) * ((c->nv + vv::BY - 1) / vv::BY);
}

// ---- reductions ---------------------------------------------------------------
int reduce_to(vv_ctx* c, const double* part, int np, double* dst) {
    vv::k_reduce_cols<<<1, vv::RED_THREADS, 0, c->st>>>(part, np, 1, np, dst);
    CKL(c);
    return VV_OK;
}

int read_scalar(vv_ctx* c, const double* dsrc, double* out) {
    CK(cudaMemcpyAsync(c->hpin, dsrc, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    *out = c->hpin[0];
    return VV_OK;
}

// ---- preconditioner ---------------------------------------------------------
// shared memory of the FFT kernels for a variant (bytes)
size_t fft_smem(int kind, int M, int R, size_t csz, bool inverse) {
    if (kind == 1) {
        const int E = M / 32;
        return (size_t)(M + R * (M + 1) + R * 32 * (E + 1)) * csz;
    }
    return inverse ? (size_t)(M + 2 * R * (M + 1)) * csz : (size_t)(M + R * (M + 1)) * csz;
}

bool four_step_ok(int M) { return M >= 32 && M <= 512; }

// shared memory of the direct-DFT kernels (any nx)
size_t rdft_smem(int nx, size_t csz) { return (size_t)nx * csz + (size_t)vv::DFT_ROWS * nx * (csz / 2); }
size_t irdft_smem(int nx, size_t csz) { return (size_t)nx * csz + (size_t)vv::DFT_ROWS * (nx / 2 + 1) * csz; }

template <typename TI, typename R>
int launch_rfft(vv_ctx* c, const TI* X, typename Cplx<R>::type* spec, const vv::PcParams& p, unsigned rows) {
    const size_t csz = sizeof(typename Cplx<R>::type);
    const int M = c->M;
    if (c->fft_kind == 2 || !c->pow2) {
        const unsigned g = (unsigned)((c->nv + vv::DFT_ROWS - 1) / vv::DFT_ROWS);
        vv::k_rdft_rows<TI, R><<<g, vv::DFT_THREADS, rdft_smem(c->nx, csz), c->st>>>(X, spec, p);
    } else if (c->fft_kind == 1 && four_step_ok(M)) {
        const size_t sm = fft_smem(1, M, c->pcR, csz, false);
        switch (M / 32) {
            case 1: vv::k_rfft4<TI, R, 1><<<rows, 32 * c->pcR, sm, c->st>>>(X, spec, p); break;
            case 2: vv::k_rfft4<TI, R, 2><<<rows, 32 * c->pcR, sm, c->st>>>(X, spec, p); break;
            case 4: vv::k_rfft4<TI, R, 4><<<rows, 32 * c->pcR, sm, c->st>>>(X, spec, p); break;
            case 8: vv::k_rfft4<TI, R, 8><<<rows, 32 * c->pcR, sm, c->st>>>(X, spec, p); break;
            default: vv::k_rfft4<TI, R, 16><<<rows, 32 * c->pcR, sm, c->st>>>(X, spec, p); break;
        }
    } else {
        vv::k_rfft_rows<TI, R><<<rows, 32 * c->pcR, fft_smem(0, M, c->pcR, csz, false), c->st>>>(X, spec, p);
    }
    CKL(c);
    return VV_OK;
}

template <typename R, typename TO>
int launch_irfft(vv_ctx* c, const typename Cplx<R>::type* spec, TO* Y, const vv::PcParams& p, unsigned rows) {
    const size_t csz = sizeof(typename Cplx<R>::type);
    const int M = c->M;
    if (c->fft_kind == 2 || !c->pow2) {
        const unsigned g = (unsigned)((c->nv + vv::DFT_ROWS - 1) / vv::DFT_ROWS);
        vv::k_irdft_rows<R, TO><<<g, vv::DFT_THREADS, irdft_smem(c->nx, csz), c->st>>>(spec, Y, p);
    } else if (c->fft_kind == 1 && four_step_ok(M)) {
        const size_t sm = fft_smem(1, M, c->pcR, csz, true);
        switch (M / 32) {
            case 1: vv::k_irfft4<R, TO, 1><<<rows, 32 * c->pcR, sm, c->st>>>(spec, Y, p); break;
            case 2: vv::k_irfft4<R, TO, 2><<<rows, 32 * c->pcR, sm, c->st>>>(spec, Y, p); break;
            case 4: vv::k_irfft4<R, TO, 4><<<rows, 32 * c->pcR, sm, c->st>>>(spec, Y, p); break;
            case 8: vv::k_irfft4<R, TO, 8><<<rows, 32 * c->pcR, sm, c->st>>>(spec, Y, p); break;
            default: vv::k_irfft4<R, TO, 16><<<rows, 32 * c->pcR, sm, c->st>>>(spec, Y, p); break;
        }
    } else {
        vv::k_irfft_rows<R, TO><<<rows, 32 * c->pcR, fft_smem(0, M, c->pcR, csz, true), c->st>>>(spec, Y, p);
    }
    CKL(c);
    return VV_OK;
}

// Dynamic shared memory limits are attributes of a kernel FUNCTION, shared
// by every context of the process on a device: a per-context value would let
// a later, smaller context lower the limit an earlier, larger one launches
// with.  They are raised once per device to the opt-in maximum less each
// kernel's static shared memory instead; each context then only checks that
// its own sizes fit under the smallest of those limits.
void smem_set(const void* f, int optin, int& lowest, cudaError_t& e) {
    cudaFuncAttributes fa;
    cudaError_t x = cudaFuncGetAttributes(&fa, f);
    const int limit = optin - (int)fa.sharedSizeBytes;
    if (x == cudaSuccess) x = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    if (e == cudaSuccess) e = x;
    lowest = std::min(lowest, limit);
}

template <typename R>
void smem_attributes(int optin, int& lowest, cudaError_t& e) {
    auto set = [&](const void* f) { smem_set(f, optin, lowest, e); };
    set((const void*)vv::k_rfft_rows<double, R>);
    set((const void*)vv::k_rfft_rows<float, R>);
    set((const void*)vv::k_irfft_rows<R, R>);
#define VV_SET4(E)                                   \
    set((const void*)vv::k_rfft4<double, R, E>);     \
    set((const void*)vv::k_rfft4<float, R, E>);      \
    set((const void*)vv::k_irfft4<R, R, E>);
    VV_SET4(1) VV_SET4(2) VV_SET4(4) VV_SET4(8) VV_SET4(16)
#undef VV_SET4
    set((const void*)vv::k_tridiag_modes<R, true>);
    set((const void*)vv::k_tridiag_modes<R, false>);
    set((const void*)vv::k_rdft_rows<double, R>);
    set((const void*)vv::k_rdft_rows<float, R>);
    set((const void*)vv::k_irdft_rows<R, R>);
    set((const void*)vv::k_tridiag_warp_staged<R>);
    set((const void*)vv::k_b_tridiag_w<R>);
    set((const void*)vv::k_b_rfftj<double, R>);
    set((const void*)vv::k_b_rfftj<float, R>);
    set((const void*)vv::k_b_irfftj<R, R>);
    set((const void*)vv::k_b_tridiagj<R>);
    set((const void*)vv::k_b_tridiagjs<R>);
    set((const void*)vv::k_b_tridiagjm<R, 2>);
    set((const void*)vv::k_b_tridiagjm<R, 4>);
    set((const void*)vv::k_b_tridiagjv<R>);
    set((const void*)vv::k_b_gm_mdot_p<R>);
#define VV_SETJ(S)                                                  \
    set((const void*)vv::k_b_jvp_rfftj<S, vv::BS_X, R>);           \
    set((const void*)vv::k_b_jvp_rfftj<S, vv::BS_VIT, R>);
    VV_SETJ(1) VV_SETJ(2) VV_SETJ(4)
#undef VV_SETJ
}

// dynamic shared memory of the staged warp-per-mode tridiagonal solve
size_t tri_ws_smem(int nv, size_t csz) {
    return (size_t)vv::TRIW_WARPS * 2 * vv::tri_ws_slots(nv) * csz + 2 * vv::tri_ws_slots(nv) * (csz / 2);
}

int raise_smem_limits(int* limit_out) {
    static std::mutex mu;
    static int limit_of[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(VV_ERR_ARG, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (limit_of[dev] == 0) {
        int optin = 0;
        if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
            return fail_cuda(e, "cudaDeviceGetAttribute (shared memory opt-in)");
        int lowest = optin;
        smem_attributes<double>(optin, lowest, e);
        smem_attributes<float>(optin, lowest, e);
        smem_set((const void*)vv::k_moments_poisson, optin, lowest, e);
        smem_set((const void*)vv::k_b_moments_poisson, optin, lowest, e);
        smem_set((const void*)vv::k_adj_poisson, optin, lowest, e);
#define VV_SET_MARCH(S)                                                              \
    smem_set((const void*)vv::k_bracket_march<S, double, 128>, optin, lowest, e);     \
    smem_set((const void*)vv::k_bracket_march<S, double, 256>, optin, lowest, e);     \
    smem_set((const void*)vv::k_bracket_march<S, float, 128>, optin, lowest, e);      \
    smem_set((const void*)vv::k_bracket_march<S, float, 256>, optin, lowest, e);
        VV_SET_MARCH(1) VV_SET_MARCH(2) VV_SET_MARCH(4)
#undef VV_SET_MARCH
        smem_set((const void*)vv::k_tridiag_modes_adjT, optin, lowest, e);
#define VV_SET_BFFT(FS)                                                         \
    smem_set((const void*)vv::k_b_rfft<double, double, FS>, optin, lowest, e);  \
    smem_set((const void*)vv::k_b_rfft<double, float, FS>, optin, lowest, e);   \
    smem_set((const void*)vv::k_b_rfft<float, float, FS>, optin, lowest, e);    \
    smem_set((const void*)vv::k_b_irfft<double, double, FS>, optin, lowest, e); \
    smem_set((const void*)vv::k_b_irfft<float, float, FS>, optin, lowest, e);
        VV_SET_BFFT(true)
        VV_SET_BFFT(false)
#undef VV_SET_BFFT
        smem_set((const void*)vv::k_b_tridiag<double, true>, optin, lowest, e);
        smem_set((const void*)vv::k_b_tridiag<float, true>, optin, lowest, e);
        smem_set((const void*)vv::k_b_tridiag<double, false>, optin, lowest, e);
        smem_set((const void*)vv::k_b_tridiag<float, false>, optin, lowest, e);
        if (e != cudaSuccess) return fail_cuda(e, "cudaFuncSetAttribute (dynamic shared memory)");
        limit_of[dev] = lowest;
    }
    *limit_out = limit_of[dev];
    return VV_OK;
}

// P^-1 with input type TI, arithmetic R (double: FP64 tables and spectrum,
// float: the mixed mode's FP32 copies) and output type TO.  Y may be a GMRES
// basis base pointer with yidx -> the vector index (+yoff).
template <typename TI, typename R, typename TO>
int pck_apply_t(vv_ctx* c, const TI* X, TO* Y, const int* yidx = nullptr, int yoff = 0) {
    constexpr bool D = std::is_same<R, double>::value;
    using C2 = typename Cplx<R>::type;
    vv::PcParams p = pcparams(c);
    C2* spec = D ? reinterpret_cast<C2*>(c->spec) : reinterpret_cast<C2*>(c->spec32);
    p.tw = D ? (const void*)c->tw : (const void*)c->tw32;
    const size_t sm_t = D ? c->smem_tri : c->smem_tri32;
    const bool stage = D ? c->tri_stage : c->tri_stage32;
    const unsigned rows = (unsigned)((c->nv + c->pcR - 1) / c->pcR);
    TRY(launch_rfft<TI, R>(c, X, spec, p, rows));
    vv::TriParams t;
    t.nv = c->nv;
    t.nmodes = c->nmodes;
    t.lambda = D ? (const void*)c->lambda : (const void*)c->lambda32;
    t.alpha = D ? (const void*)c->alpha : (const void*)c->alpha32;
    t.gamma = D ? (const void*)c->gamma : (const void*)c->gamma32;
    t.dinv = D ? (const void*)c->dinv : (const void*)c->dinv32;
    if (c->tri_kind == 1) {
        const unsigned g = (unsigned)((c->nmodes + vv::TRIW_WARPS - 1) / vv::TRIW_WARPS);
        const size_t sm = tri_ws_smem(c->nv, sizeof(typename Cplx<R>::type));
        if (sm <= (size_t)c->smem_limit)
            vv::k_tridiag_warp_staged<R><<<g, 32 * vv::TRIW_WARPS, sm, c->st>>>(spec, t);
        else
            vv::k_tridiag_warp<R><<<g, 32 * vv::TRIW_WARPS, 0, c->st>>>(spec, t);
    }
    else if (stage)
        vv::k_tridiag_modes<R, true><<<c->nmodes, vv::TRI_THREADS, sm_t, c->st>>>(spec, t);
    else
        vv::k_tridiag_modes<R, false><<<c->nmodes, vv::TRI_THREADS, sm_t, c->st>>>(spec, t);
    CKL(c);
    p.yidx = yidx;
    p.yoff = yoff;
    p.ystride = yidx ? c->ncell : 0;
    return launch_irfft<R, TO>(c, spec, Y, p, rows);
}

// The potential preconditioner: the v transforms as row transforms of the
// transposed field (radix-2 FFT for a power-of-two nv, else the direct DFT),
// the x-tridiagonal systems per v mode by elimination with partial pivoting
template <typename TI, typename R, typename TO>
int pcv_apply_t(vv_ctx* c, const TI* X, TO* Y, const int* yidx = nullptr, int yoff = 0) {
    constexpr bool D = std::is_same<R, double>::value;
    using C2 = typename Cplx<R>::type;
    const int nx = c->nx, nv = c->nv;
    R* xt = D ? reinterpret_cast<R*>(c->pv_xt) : reinterpret_cast<R*>(c->pv_xt32);
    C2* spec = D ? reinterpret_cast<C2*>(c->pv_spec) : reinterpret_cast<C2*>(c->pv_spec32);
    C2* scr = D ? reinterpret_cast<C2*>(c->pv_scr) : reinterpret_cast<C2*>(c->pv_scr32);
    const dim3 tb(32, 8);
    vv::k_transpose<TI, R><<<dim3((nx + 31) / 32, (nv + 31) / 32), tb, 0, c->st>>>(X, xt, nv, nx, nullptr, 0, 0);
    CKL(c);
    vv::PcParams p;
    p.nx = nv;   // rows of length nv ...
    p.nv = nx;   // ... one per x point
    p.M = nv / 2;
    p.logM = is_pow2(nv) ? ilog2(nv / 2) : -1;
    p.R = c->pvR;
    p.tw = D ? (const void*)c->twv : (const void*)c->twv32;
    p.yidx = nullptr;
    p.yoff = 0;
    p.ystride = 0;
    const size_t csz = sizeof(C2);
    const bool fft = is_pow2(nv);
    const unsigned gr = (unsigned)((nx + c->pvR - 1) / c->pvR), gd = (unsigned)((nx + vv::DFT_ROWS - 1) / vv::DFT_ROWS);
    if (fft) vv::k_rfft_rows<R, R><<<gr, 32 * c->pvR, fft_smem(0, nv / 2, c->pvR, csz, false), c->st>>>(xt, spec, p);
    else vv::k_rdft_rows<R, R><<<gd, vv::DFT_THREADS, rdft_smem(nv, csz), c->st>>>(xt, spec, p);
    CKL(c);
    vv::PotParams q;
    q.nx = nx;
    q.nmv = c->nmv;
    q.arak = 0.5 * c->hx_inv * c->hv_inv / 12.;   // TensorProductPotentialFast.pyx:237
    q.ht_inv = c->ht_inv;
    q.phi = c->phipc;
    q.lam = c->lamv;
    vv::k_pcv_solve<R><<<(unsigned)((c->nmv + 63) / 64), 64, 0, c->st>>>(spec, scr, q);
    CKL(c);
    if (fft) vv::k_irfft_rows<R, R><<<gr, 32 * c->pvR, fft_smem(0, nv / 2, c->pvR, csz, true), c->st>>>(spec, xt, p);
    else vv::k_irdft_rows<R, R><<<gd, vv::DFT_THREADS, irdft_smem(nv, csz), c->st>>>(spec, xt, p);
    CKL(c);
    vv::k_transpose<R, TO><<<dim3((nv + 31) / 32, (nx + 31) / 32), tb, 0, c->st>>>(xt, Y, nx, nv, yidx, yoff,
                                                                                   yidx ? c->ncell : 0);
    CKL(c);
    return VV_OK;
}

// P^-1 of the context's preconditioner
template <typename TI, typename R, typename TO>
int pc_apply_t(vv_ctx* c, const TI* X, TO* Y, const int* yidx = nullptr, int yoff = 0) {
    if (c->g.preconditioner == VV_PC_TENSOR_POTENTIAL) return pcv_apply_t<TI, R, TO>(c, X, Y, yidx, yoff);
    return pck_apply_t<TI, R, TO>(c, X, Y, yidx, yoff);
}

int pc_apply(vv_ctx* c, const double* X, double* Y, const int* yidx = nullptr, int yoff = 0) {
    return pc_apply_t<double, double, double>(c, X, Y, yidx, yoff);
}

// buffers of the GMRES solve in precision T
template <typename T> struct Buf;
template <> struct Buf<double> {
    static double* V(vv_ctx* c) { return c->V; }
    static double* tmp(vv_ctx* c) { return c->tmp; }
    static double* b(vv_ctx* c) { return c->bvec; }
    static double* x(vv_ctx* c) { return c->delta; }
};
template <> struct Buf<float> {
    static float* V(vv_ctx* c) { return c->V32; }
    static float* tmp(vv_ctx* c) { return c->tmp32; }
    static float* b(vv_ctx* c) { return c->bvec32; }
    static float* x(vv_ctx* c) { return c->delta32; }
};

// ---- discrete adjoint: A^T and P^-T (FP64) ----------------------------------
vv::PoissonParams pparams(const vv_ctx* c);
int copy_d(vv_ctx* c, double* dst, const double* src, size_t count);

vv::AdjParams adjparams(const vv_ctx* c) {
    vv::AdjParams p;
    p.nx = c->nx;
    p.nv = c->nv;
    p.ncell = c->ncell;
    p.ht_inv = c->ht_inv;
    p.f1 = c->f1;
    p.f2 = c->f2;
    p.hv = c->hv;
    return p;
}

// Y = A^T X (X may be a basis base pointer with xidx)
int adj_apply(vv_ctx* c, const double* X, const int* xidx, double* Y) {
    const vv::AdjParams p = adjparams(c);
    dim3 grid((c->nx + vv::ADJ_TX - 1) / vv::ADJ_TX, c->mom_S);
    vv::k_adj_apply<<<grid, dim3(vv::ADJ_TX, vv::ADJ_TY), 0, c->st>>>(p, c->adj_cH, c->adj_cF, X, xidx, Y, c->mom_seg,
                                                                      c->adj_zpart);
    CKL(c);
    vv::k_adj_poisson<<<1, vv::POIS_THREADS, c->smem_pois, c->st>>>(c->adj_zpart, c->mom_S, c->adj_zbuf, c->adj_q,
                                                                    pparams(c));
    CKL(c);
    vv::k_adj_bcast<<<grid1d(c->ncell, 256), 256, 0, c->st>>>(p, c->adj_q, Y);
    CKL(c);
    return VV_OK;
}

// Y = P^-T X: the same FFT pair, conjugate-transposed mode solves
// (the kinetic factors for the potential preconditioner too: any fixed P
// serves the transposed solve, and P^-T of the potential preconditioner is
// not built)
int pcT_apply(vv_ctx* c, const double* X, double* Y, const int* yidx = nullptr, int yoff = 0) {
    if (c->g.preconditioner == VV_PC_NONE) {
        if (yidx) return VV_ERR_UNSUPPORTED;
        return copy_d(c, Y, X, c->ncell);
    }
    vv::PcParams p = pcparams(c);
    p.tw = c->tw;
    const unsigned rows = (unsigned)((c->nv + c->pcR - 1) / c->pcR);
    TRY(launch_rfft<double, double>(c, X, c->spec, p, rows));
    vv::TriParams t;
    t.nv = c->nv;
    t.nmodes = c->nmodes;
    t.lambda = c->lambda;
    t.alpha = c->alpha;
    t.gamma = c->gamma;
    t.dinv = c->dinv;
    const int ch = (c->nv + vv::TRI_THREADS - 1) / vv::TRI_THREADS;
    const size_t sm = ((size_t)c->nv + (c->nv + ch - 1) / ch) * sizeof(double2);
    vv::k_tridiag_modes_adjT<<<c->nmodes, vv::TRI_THREADS, sm, c->st>>>(c->spec, t);
    CKL(c);
    p.yidx = yidx;
    p.yoff = yoff;
    p.ystride = yidx ? c->ncell : 0;
    return launch_irfft<double, double>(c, c->spec, Y, p, rows);
}

// Y = P^-1 J X (or J X) in precision T
template <typename T>
int apply_operator_t(vv_ctx* c, const T* X, T* Y) {
    if constexpr (std::is_same<T, double>::value) {
        if (c->adj) {   // the adjoint solve: P^-T A^T
            TRY(adj_apply(c, X, nullptr, c->tmp));
            return pcT_apply(c, c->tmp, Y);
        }
    }
    if (c->g.preconditioner != VV_PC_NONE) {
        TRY(launch_bracket<vv::MODE_JVP, T>(c, X, nullptr, Buf<T>::tmp(c), 0.5, nullptr));
        return pc_apply_t<T, T, T>(c, Buf<T>::tmp(c), Y);
    }
    return launch_bracket<vv::MODE_JVP, T>(c, X, nullptr, Y, 0.5, nullptr);
}

int apply_operator(vv_ctx* c, const double* X, double* Y) { return apply_operator_t<double>(c, X, Y); }

template <typename T>
__global__ void k_copy_to_slot(const T* __restrict__ src, T* __restrict__ V, const int* __restrict__ idx,
                               size_t n) {
    T* dst = V + (size_t)(*idx + 1) * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// Arnoldi operator V[it] -> V[it+1], it read from the device state
template <typename T>
int apply_operator_state(vv_ctx* c) {
    const int* itp = &c->ds->it;
    T* V = Buf<T>::V(c);
    if constexpr (std::is_same<T, double>::value) {
        if (c->adj) {   // the adjoint solve: V[it+1] = P^-T A^T V[it]
            TRY(adj_apply(c, V, itp, c->tmp));
            if (c->g.preconditioner != VV_PC_NONE) return pcT_apply(c, c->tmp, V, itp, 1);
            k_copy_to_slot<double><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->tmp, V, itp, c->ncell);
            CKL(c);
            return VV_OK;
        }
    }
    TRY(launch_bracket<vv::MODE_JVP, T>(c, V, nullptr, Buf<T>::tmp(c), 0.5, nullptr, itp));
    if (c->g.preconditioner != VV_PC_NONE) return pc_apply_t<T, T, T>(c, Buf<T>::tmp(c), V, itp, 1);
    k_copy_to_slot<T><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(Buf<T>::tmp(c), V, itp, c->ncell);
    CKL(c);
    return VV_OK;
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
    p.la0 = c->lap[0];
    p.la1 = c->lap[1];
    p.la2 = c->lap[2];
    p.lden = c->lap[3];
    p.ravg = c->ravg[3] != 1.0 ? 1 : 0;
    p.ra0 = c->ravg[0];
    p.ra1 = c->ravg[1];
    p.ra2 = c->ravg[2];
    p.rden = c->ravg[3];
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

__global__ void k_poisson_apply(const double* __restrict__ x, const double* __restrict__ n,
                                double* __restrict__ y, int mode, double* __restrict__ sumsq, vv::PoissonParams p) {
    vv::poisson_apply_cta(x, n, y, p.nx, p.hx2_inv, p.charge, mode, sumsq, p.la0, p.la1, p.la2, p.lden, p.ravg, p.ra0,
                          p.ra1, p.ra2, p.rden);
}

int poisson_apply(vv_ctx* c, const double* x, const double* n, double* y, int mode, double* sumsq) {
    k_poisson_apply<<<1, 1024, 0, c->st>>>(x, n, y, mode, sumsq, pparams(c));
    CKL(c);
    return VV_OK;
}

// ---- small copies -----------------------------------------------------------
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

// ---- GMRES: kernel sequences shared by the host-driven and graph paths ------
// state header written by the host before a solve / step (the option fields)
int upload_options(vv_ctx* c, const vv_ksp_opts* o, const vv_snes_opts* so) {
    if (c->opts_valid && so && std::memcmp(&c->last_ksp, o, sizeof *o) == 0 &&
        std::memcmp(&c->last_snes, so, sizeof *so) == 0 && std::memcmp(c->last_hnd, c->hnd, sizeof c->hnd) == 0)
        return VV_OK;
    c->opts_valid = so != nullptr;
    c->last_ksp = *o;
    if (so) c->last_snes = *so;
    std::memcpy(c->last_hnd, c->hnd, sizeof c->hnd);
    vv::DevState* h = c->hds;
    h->restart = (o->restart > 0) ? o->restart : c->restart;
    h->max_it = o->max_it;
    h->rtol = o->rtol;
    if (so && c->mixed) h->rtol = std::max(o->rtol, c->g.mixed_rtol > 0.0 ? c->g.mixed_rtol : 1e-2);
    h->atol = o->atol;
    h->dtol = (o->dtol > 0.0) ? o->dtol : 1e5;
    h->haptol = 1e-30;
    if (so) {
        h->snes_atol = so->atol;
        h->pic_max_iter = so->max_iter;
        h->abort_residual = so->abort_residual;
    }
    h->h_gm_outer = c->hnd[0];
    h->h_gm_inner = c->hnd[1];
    h->h_gm_first = c->hnd[2];
    h->h_pic = c->hnd[3];
    h->h_revert = c->hnd[4];
    h->cnt[0] = h->cnt[1] = h->cnt[2] = h->cnt[3] = 0u;
    // one copy of the header (everything before the report arrays)
    CK(cudaMemcpyAsync(c->ds, h, offsetof(vv::DevState, gmres_its), cudaMemcpyHostToDevice, c->st));
    return VV_OK;
}

template <typename T>
int gm_init(vv_ctx* c, T* x) {
    vv::k_gm_init<T><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->ds, x, c->ncell);
    CKL(c);
    return VV_OK;
}

template <typename T>
int copy_t(vv_ctx* c, T* dst, const T* src, size_t count) {
    if (!dst || !src || dst == src) return VV_OK;
    CK(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToDevice, c->st));
    return VV_OK;
}

// V0 = b (first cycle) or b - A x (restart)
template <typename T>
int gm_cycle_head(vv_ctx* c, const T* b, const T* x, bool first) {
    T* V = Buf<T>::V(c);
    if (first) return copy_t<T>(c, V, b, c->ncell);
    TRY(apply_operator_t<T>(c, x, V));
    vv::k_axpby<T><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(b, V, c->ncell, 1.0, -1.0);
    CKL(c);
    return VV_OK;
}

template <typename T>
int gm_cycle_start(vv_ctx* c) {
    T* V = Buf<T>::V(c);
    vv::k_gm_cycle<T><<<c->npart, vv::RED_THREADS, 0, c->st>>>(c->ds, V, c->ncell, c->part);
    CKL(c);
    vv::k_gm_scale<T><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->ds, V, c->ncell, c->ncell);
    CKL(c);
    return VV_OK;
}

template <typename T>
int gm_arnoldi(vv_ctx* c) {
    T* V = Buf<T>::V(c);
    TRY(apply_operator_state<T>(c));
    vv::k_gm_mdot<T><<<c->npart, vv::RED_THREADS, 0, c->st>>>(c->ds, V, c->ncell, c->ncell, c->part, c->npart_max);
    CKL(c);
    vv::k_gm_maxpy<T><<<c->npart, vv::RED_THREADS, 0, c->st>>>(c->ds, V, c->ncell, c->ncell, c->part);
    CKL(c);
    vv::k_gm_scale<T><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->ds, V, c->ncell, c->ncell);
    CKL(c);
    return VV_OK;
}

template <typename T>
int gm_finish(vv_ctx* c, T* x) {
    vv::k_gm_finish<T><<<c->npart, vv::RED_THREADS, 0, c->st>>>(c->ds, Buf<T>::V(c), c->ncell, x, c->ncell);
    CKL(c);
    return VV_OK;
}

struct GmHead {
    int it, its, reason, active;
};

int read_head(vv_ctx* c, GmHead* h) {
    CK(cudaMemcpyAsync(c->hstat, c->ds, sizeof(GmHead), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    std::memcpy(h, c->hstat, sizeof(GmHead));
    return VV_OK;
}

// Host-driven GMRES: the same kernels, with the host reading the 16-byte
// status block after every Arnoldi step.
template <typename T>
int gmres_host(vv_ctx* c, const T* b, T* x, vv_ksp_result* res) {
    TRY(gm_init<T>(c, x));
    bool first = true;
    GmHead h{};
    for (;;) {
        TRY(gm_cycle_head<T>(c, b, x, first));
        TRY(gm_cycle_start<T>(c));
        TRY(read_head(c, &h));
        while (h.active) {
            TRY(gm_arnoldi<T>(c));
            TRY(read_head(c, &h));
        }
        TRY(gm_finish<T>(c, x));
        TRY(read_head(c, &h));
        if (h.reason != 0) break;
        first = false;
    }
    if (res) {
        double rn = 0.0;
        TRY(read_scalar(c, &c->ds->res, &rn));
        res->its = h.its;
        res->reason = h.reason;
        res->rnorm = rn;
    }
    return VV_OK;
}

// ---- graph capture helpers ----------------------------------------------------
// Add a conditional node at the current position of the capture on `cs`.
// *handle_out: a handle created earlier on `owner`, or 0 to create one on the
// top-level graph `owner` (handles may serve conditional nodes of child
// graphs) with a default applied at every launch.
int add_conditional(cudaGraph_t owner, cudaStream_t cs, cudaGraphConditionalNodeType type, unsigned size,
                    unsigned defval, unsigned long long* handle_out, cudaGraph_t* bodies) {
    static const bool dbg = getenv("VV_DEBUG") != nullptr;
    if (dbg) {
        fprintf(stderr, "[vv] add_conditional type=%d size=%u\n", (int)type, size);
        fflush(stderr);
    }
    cudaStreamCaptureStatus status;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraph_t g = nullptr;
    CK(cudaStreamGetCaptureInfo(cs, &status, nullptr, &g, &deps, &nd));
    if (status != cudaStreamCaptureStatusActive) return VV_ERR_CUDA;
    cudaGraphConditionalHandle h = (cudaGraphConditionalHandle)*handle_out;   // an existing handle, or a new one
    if (!h) CK(cudaGraphConditionalHandleCreate(&h, owner, defval, cudaGraphCondAssignDefault));
    cudaGraphNodeParams prm = {cudaGraphNodeTypeConditional};
    prm.conditional.handle = h;
    prm.conditional.type = type;
    prm.conditional.size = size;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &prm));
    for (unsigned k = 0; k < size; ++k) bodies[k] = prm.conditional.phGraph_out[k];
    CK(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
    *handle_out = (unsigned long long)h;
    return VV_OK;
}

// Capture `fn` into `body` on capture stream `s`, with c->st pointing at it.
template <typename F>
int capture_body(vv_ctx* c, cudaStream_t s, cudaGraph_t body, int* nkernels, F fn) {
    const cudaStream_t saved = c->st;
    const int64_t l0 = c->launches;
    CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    c->st = s;
    int r = fn();
    c->st = saved;
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &out);
    if (r != VV_OK) return r;
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture");
    if (nkernels) *nkernels = (int)(c->launches - l0);
    return VV_OK;
}

// GMRES solve b -> x into the graph being captured on c->st (level = depth of c->st)
template <typename T>
int capture_gmres(vv_ctx* c, int level, const T* b, T* x) {
    TRY(gm_init<T>(c, x));
    cudaGraph_t outer[1];
    TRY(add_conditional(c->cap_owner, c->st, cudaGraphCondTypeWhile, 1, 1, &c->hnd[0], outer));
    const int l1 = level + 1;
    return capture_body(c, c->cs[l1], outer[0], &c->nk_cycle, [&]() -> int {
        cudaGraph_t br[2];
        TRY(add_conditional(c->cap_owner, c->cs[l1], cudaGraphCondTypeIf, 2, 1, &c->hnd[2], br));
        TRY(capture_body(c, c->cs[l1 + 1], br[0], nullptr, [&]() { return gm_cycle_head<T>(c, b, x, true); }));
        TRY(capture_body(c, c->cs[l1 + 1], br[1], &c->nk_restart,
                         [&]() { return gm_cycle_head<T>(c, b, x, false); }));
        TRY(gm_cycle_start<T>(c));
        cudaGraph_t inner[1];
        TRY(add_conditional(c->cap_owner, c->cs[l1], cudaGraphCondTypeWhile, 1, 0, &c->hnd[1], inner));
        TRY(capture_body(c, c->cs[l1 + 1], inner[0], &c->nk_arnoldi, [&]() { return gm_arnoldi<T>(c); }));
        return gm_finish<T>(c, x);
    });
}

// ---- residual / moments helpers of the step ---------------------------------
int residual_norm(vv_ctx* c, const double* F, double* Y, double* out) {
    const int tiles = bracket_tiles(c, F, c->Fh, Y);
    TRY(launch_bracket<vv::MODE_RESIDUAL, double>(c, F, c->Fh, Y, 1.0, c->part));
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

// residual of f into tmp + tile partials, Poisson residual into ds->pnorm2,
// then the Picard decision kernel (phase 0: initial residual)
int step_residual(vv_ctx* c, vv_state* st, int phase) {
    const int tiles = bracket_tiles(c, st->f, c->Fh, c->tmp);
    TRY(launch_bracket<vv::MODE_RESIDUAL, double>(c, st->f, c->Fh, c->tmp, 1.0, c->part));
    TRY(poisson_apply(c, st->phi, st->n, nullptr, 2, &c->ds->pnorm2));
    vv::k_pic_residual<<<1, 32, 0, c->st>>>(c->ds, c->part, tiles, phase);
    CKL(c);
    return VV_OK;
}

// ---- explicit predictors of the initial guess (vv_pred.cuh) ------------------
// Y = -[X, H] (zeroed first) in the reference-order kernels with a general h
int pred_bracket(vv_ctx* c, const double* X, const double* H, double* Y) {
    CK(cudaMemsetAsync(Y, 0, c->ncell * sizeof(double), c->st));
    return launch_bracket_gen(c, X, nullptr, Y, H, -1.0, nullptr);
}

// kinetic / potential substep: X += factor * ht / niter * (-[X, H])
int pred_substep(vv_ctx* c, double* X, const double* H, double factor) {
    TRY(pred_bracket(c, X, H, c->pred_Y));
    const double s = factor * c->g.ht / (double)c->pred_iter;
    vv::k_pred_axpy<<<grid1d(c->ncell, 256), 256, 0, c->st>>>(X, c->pred_Y, s, c->ncell);
    CKL(c);
    return VV_OK;
}

// Y = the predictor applied to F (Y may alias F), with H0 and the history
// profiles h1h, h2h (run_base.py:811-912)
int pred_run(vv_ctx* c, const double* F, const double* h1h, const double* h2h, double* Y) {
    const size_t n = c->ncell;
    const int nx = c->nx, nv = c->nv;
    const unsigned gr = grid1d(n, 256);
    const double ht = c->g.ht, niter = (double)c->pred_iter;
    TRY(copy_d(c, Y, F, n));
    if (c->pred == VV_GUESS_SYMPLECTIC2 || c->pred == VV_GUESS_SYMPLECTIC4) {
        vv::k_pred_hfield<<<gr, 256, 0, c->st>>>(c->h0, h1h, h2h, c->pred_H, nx, nv, 0);
        vv::k_pred_hfield<<<gr, 256, 0, c->st>>>(c->h0, h1h, h2h, c->pred_Hp, nx, nv, 1);
        CKL(c);
        // run_base.py:887-898
        const double fac2 = std::pow(2., 1. / 3.);
        const double c1 = 0.5 / (2. - fac2), c2 = c1 * (1. - fac2);
        const double d1 = 1. / (2. - fac2), d2 = -d1 * fac2;
        for (int it = 0; it < c->pred_iter; ++it) {
            if (c->pred == VV_GUESS_SYMPLECTIC2) {   // run_base.py:866-877
                TRY(pred_substep(c, Y, c->pred_H, 0.5));
                TRY(pred_substep(c, Y, c->pred_Hp, 1.0));
                TRY(pred_substep(c, Y, c->pred_H, 0.5));
            } else {                                // run_base.py:900-912
                TRY(pred_substep(c, Y, c->pred_H, c1));
                TRY(pred_substep(c, Y, c->pred_Hp, d1));
                TRY(pred_substep(c, Y, c->pred_H, c2));
                TRY(pred_substep(c, Y, c->pred_Hp, d2));
                TRY(pred_substep(c, Y, c->pred_H, c2));
                TRY(pred_substep(c, Y, c->pred_Hp, d1));
                TRY(pred_substep(c, Y, c->pred_H, c1));
            }
        }
        return VV_OK;
    }
    vv::k_pred_hfield<<<gr, 256, 0, c->st>>>(c->h0, h1h, h2h, c->pred_H, nx, nv, 2);
    CKL(c);
    double* K1 = c->pred_K;
    double* K2 = K1 + n;
    double* K3 = K2 + n;
    double* K4 = K3 + n;
    double* S = c->pred_S;
    const double b = ht / niter;
    for (int it = 0; it < c->pred_iter; ++it) {
        TRY(pred_bracket(c, Y, c->pred_H, K1));
        if (c->pred == VV_GUESS_RK4_16) {           // PETScArakawaRungeKutta.pyx:20-58
            const double a = 0.5 * ht / niter;
            vv::k_pred_stage<<<gr, 256, 0, c->st>>>(Y, K1, nullptr, nullptr, S, a, 0.0, 0, n);
            TRY(pred_bracket(c, S, c->pred_H, K2));
            vv::k_pred_stage<<<gr, 256, 0, c->st>>>(Y, K2, nullptr, nullptr, S, a, 0.0, 0, n);
            TRY(pred_bracket(c, S, c->pred_H, K3));
            vv::k_pred_stage<<<gr, 256, 0, c->st>>>(Y, K3, nullptr, nullptr, S, 1.0 * ht / niter, 0.0, 0, n);
            TRY(pred_bracket(c, S, c->pred_H, K4));
            vv::k_pred_rk_final<<<gr, 256, 0, c->st>>>(Y, K1, K2, K3, K4, b, 2., 6., n);
        } else {                                    // PETScArakawaRungeKutta.pyx:61-100
            const double a = 1. / 3. * ht / niter;
            vv::k_pred_stage<<<gr, 256, 0, c->st>>>(Y, K1, nullptr, nullptr, S, a, 0.0, 0, n);
            TRY(pred_bracket(c, S, c->pred_H, K2));
            vv::k_pred_stage<<<gr, 256, 0, c->st>>>(Y, K1, K2, nullptr, S, a, b, 1, n);
            TRY(pred_bracket(c, S, c->pred_H, K3));
            vv::k_pred_stage<<<gr, 256, 0, c->st>>>(Y, K1, K2, K3, S, 0.0, b, 2, n);
            TRY(pred_bracket(c, S, c->pred_H, K4));
            vv::k_pred_rk_final<<<gr, 256, 0, c->st>>>(Y, K1, K2, K3, K4, b, 3., 8., n);
        }
        CKL(c);
    }
    return VV_OK;
}

// the guard's residual (phase 0: of the current f, 1: of the prediction),
// with the Have of the last update_previous and, for a solver whose Have is
// still the zero vector of its construction (no update_previous yet; the
// device flag decides), with a zero Have: the time derivative and the
// collision terms (the brackets and the double bracket of a zero h vanish)
int pred_residual(vv_ctx* c, vv_state* st, int phase) {
    const int tiles = bracket_tiles(c, st->f, c->Fh, c->tmp);
    TRY(launch_bracket<vv::MODE_RESIDUAL, double>(c, st->f, c->Fh, c->tmp, 1.0, c->part));
    TRY(poisson_apply(c, st->phi, st->n, nullptr, 2, &c->ds->pnorm2));
    const bool coll = c->coll != vv::COLL_NONE;
    c->zero_h = c->pred_zero;
    const int r = launch_bracket_td<vv::MODE_RESIDUAL, double>(c, st->f, c->Fh, c->pred_Y, 1.0,
                                                                coll ? nullptr : c->pred_cpart, nullptr);
    c->zero_h = nullptr;
    TRY(r);
    if (coll) TRY(launch_collision<double>(c, st->f, c->Fh, c->pred_Y, c->pred_cpart, nullptr));
    const int ncp = ((c->nx + vv::BX - 1) / vv::BX) * ((c->nv + vv::BY - 1) / vv::BY);
    vv::k_pred_norm<<<1, 32, 0, c->st>>>(c->ds, c->part, tiles, c->pred_cpart, ncp, phase);
    CKL(c);
    return VV_OK;
}

// initial_guess (run_base.py:786-808) after make_history, before update_previous
int pred_guess(vv_ctx* c, vv_state* st) {
    const size_t n = c->ncell;
    TRY(copy_d(c, c->pred_fl, st->f, n));
    TRY(pred_residual(c, st, 0));
    TRY(pred_run(c, st->f, st->h1h, st->h2h, st->f));
    TRY(calc_moments(c, st));
    TRY(pred_residual(c, st, 1));
    vv::k_pred_guard<<<grid1d(n, 256), 256, 0, c->st>>>(c->ds, st->f, c->pred_fl, n);
    CKL(c);
    return calc_moments(c, st);
}

// make_history + update_previous + initial residual
int step_prologue(vv_ctx* c, vv_state* st) {
    const size_t n = c->ncell;
    const int nx = c->nx;
    TRY(copy_d(c, st->fh, st->f, n));
    TRY(copy_d(c, st->h1h, st->h1c, nx));
    if (st->h2c && st->h2h) TRY(copy_d(c, st->h2h, st->h2c, nx));
    if (st->phih) TRY(copy_d(c, st->phih, st->phi, nx));
    TRY(copy_d(c, c->Fh, st->f, n));
    // update_history -> update_matrices of the potential preconditioner
    if (c->g.preconditioner == VV_PC_TENSOR_POTENTIAL) TRY(copy_d(c, c->phipc, st->phi, nx));
    // nc -> nh, uc -> uh, ac -> ah (run_base.py:757-760) for the collision operator
    if (c->coll != vv::COLL_NONE) {
        TRY(copy_d(c, c->mom_h, st->n, nx));
        TRY(copy_d(c, c->mom_h + nx, st->u, nx));
        TRY(copy_d(c, c->mom_h + 2 * nx, st->a, nx));
    }
    if (c->pred) TRY(pred_guess(c, st));
    TRY(set_hxp(c, st->h1c, st->h1h, st->h2c, st->h2h));
    return step_residual(c, st, 0);
}

// the preconditioned right-hand side of the ksponly solve: b = P^-1 R(f),
// with R(f) left in tmp by the last residual evaluation (same Fh and Have)
int step_rhs(vv_ctx* c, vv_state* st) {
    TRY(copy_d(c, c->fl, st->f, c->ncell));
    if (c->mixed) {   // FP64 residual -> FP32 right-hand side
        if (c->g.preconditioner != VV_PC_NONE) return pc_apply_t<double, float, float>(c, c->tmp, c->bvec32);
        vv::k_scale<double, float><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->tmp, c->bvec32, c->ncell, nullptr, 1.0);
        CKL(c);
        return VV_OK;
    }
    if (c->g.preconditioner != VV_PC_NONE) return pc_apply(c, c->tmp, c->bvec);
    return copy_d(c, c->bvec, c->tmp, c->ncell);
}

int step_after_solve(vv_ctx* c, vv_state* st) {
    if (c->mixed)
        vv::k_pic_apply<float, double><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->ds, c->delta32, st->f, c->ncell);
    else
        vv::k_pic_apply<double, double><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->ds, c->delta, st->f, c->ncell);
    CKL(c);
    TRY(calc_moments(c, st));
    TRY(copy_d(c, c->hxp, st->h1c, c->nx));   // update_previous: H1p <- h1c
    return step_residual(c, st, 1);
}

int step_revert(vv_ctx* c, vv_state* st) {
    TRY(copy_d(c, st->f, c->fl, c->ncell));
    return calc_moments(c, st);
}

bool same_state(const vv_state& a, const vv_state& b) { return std::memcmp(&a, &b, sizeof a) == 0; }

// ---- autotuner ---------------------------------------------------------------
// Times the candidate kernel variants of one grid shape on the context's own
// scratch buffers (CUDA events, a few launches each) and keeps the fastest:
// FFT kind x rows per CTA x tridiagonal kind for the preconditioner in the
// GMRES precision, and the bracket tile shape.  Results are cached per
// (nx, nv, precision, time derivative) for the life of the process.
struct TuneResult {
    int fft_kind, pcR, tri_kind, narrow, march;
};

std::vector<std::pair<std::array<int, 4>, TuneResult>>& tune_cache() {
    static std::vector<std::pair<std::array<int, 4>, TuneResult>> cache;
    return cache;
}

template <typename F>
int time_it(vv_ctx* c, F fn, int reps, float* ms) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int r = VV_OK;
    for (int k = 0; k < 2 && r == VV_OK; ++k) r = fn();
    cudaEventRecord(e0, c->st);
    for (int k = 0; k < reps && r == VV_OK; ++k) r = fn();
    cudaEventRecord(e1, c->st);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r != VV_OK) return r;
    if (e != cudaSuccess) return fail_cuda(e, "autotune timing");
    return VV_OK;
}

int autotune(vv_ctx* c) {
    const std::array<int, 4> key = {c->nx, c->nv, c->mixed ? 1 : 0, c->avg};
    for (auto& kv : tune_cache())
        if (kv.first == key) {
            c->fft_kind = kv.second.fft_kind;
            c->pcR = kv.second.pcR;
            c->tri_kind = kv.second.tri_kind;
            c->narrow_bracket = kv.second.narrow;
            c->march = kv.second.march;
            return VV_OK;
        }
    const size_t n = c->ncell;
    CK(cudaMemsetAsync(c->tmp, 0, n * sizeof(double), c->st));
    if (c->mixed) CK(cudaMemsetAsync(c->tmp32, 0, n * sizeof(float), c->st));
    TuneResult best{c->fft_kind, c->pcR, c->tri_kind, 0, 0};
    float best_ms = 1e30f;
    // FP64 complex size also in the mixed mode: the FP64 entry points
    // (vv_pc_apply) share the tuned rows-per-CTA
    const size_t csz = sizeof(double2);
    for (int kind = c->pow2 ? 0 : 2; kind <= 2; ++kind) {
        if (kind == 1 && !four_step_ok(c->M)) continue;
        if (kind == 2 && c->pow2) continue;   // the FFT kernels always beat the O(nx^2) DFT
        for (int R = 1; R <= (kind == 2 ? 1 : 8); R *= 2) {
            if (kind < 2 && fft_smem(kind, c->M, R, csz, true) > 200 * 1024) continue;
            for (int tk = 0; tk <= 1; ++tk) {
                c->fft_kind = kind;
                c->pcR = R;
                c->tri_kind = tk;
                float ms = 0.f;
                int r = c->mixed ? time_it(c, [&]() { return pc_apply_t<float, float, float>(c, c->tmp32, c->bvec32); },
                                           5, &ms)
                                 : time_it(c, [&]() { return pc_apply(c, c->tmp, c->bvec); }, 5, &ms);
                TRY(r);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = {kind, R, tk, 0, 0};
                }
            }
        }
    }
    c->fft_kind = best.fft_kind;
    c->pcR = best.pcR;
    c->tri_kind = best.tri_kind;
    if (c->nx % vv::WX == 0) {
        float t_wide = 0.f, t_narrow = 0.f;
        for (int nb = 0; nb <= 1; ++nb) {
            c->narrow_bracket = nb;
            float ms = 0.f;
            int r = c->mixed ? time_it(c, [&]() {
                                   return launch_bracket<vv::MODE_JVP, float>(c, c->tmp32, nullptr, c->bvec32, 0.5,
                                                                              nullptr);
                               }, 10, &ms)
                             : time_it(c, [&]() {
                                   return launch_bracket<vv::MODE_JVP, double>(c, c->tmp, nullptr, c->bvec, 0.5,
                                                                               nullptr);
                               }, 10, &ms);
            TRY(r);
            (nb ? t_narrow : t_wide) = ms;
        }
        best.narrow = t_narrow < t_wide ? 1 : 0;
    }
    c->narrow_bracket = best.narrow;
    // the Jacobian stencil: tiles (the choice above) or the marching kernel
    {
        float t_best = 1e30f;
        for (int mw : {0, 128, 256}) {
            if (mw && (c->nx % mw != 0 || c->g.order == VV_ORDER_REFERENCE || c->avg != vv::AVG_POINT)) continue;
            c->march = mw;
            float ms = 0.f;
            int r = c->mixed ? time_it(c, [&]() {
                                   return launch_bracket<vv::MODE_JVP, float>(c, c->tmp32, nullptr, c->bvec32, 0.5,
                                                                              nullptr);
                               }, 10, &ms)
                             : time_it(c, [&]() {
                                   return launch_bracket<vv::MODE_JVP, double>(c, c->tmp, nullptr, c->bvec, 0.5,
                                                                               nullptr);
                               }, 10, &ms);
            TRY(r);
            if (ms < t_best) {
                t_best = ms;
                best.march = mw;
            }
        }
    }
    c->march = best.march;
    c->launches = 0;
    tune_cache().push_back({key, best});
    return VV_OK;
}

// A fixed kernel shape "fft,R,tri,narrow[,march]" (the fields of TuneResult),
// checked against what the grid allows; VV_ERR_ARG when it does not fit.
int apply_shape(vv_ctx* c, const char* spec) {
    int v[5] = {0, 1, 0, 0, 0};
    const int n = sscanf(spec, "%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4]);
    if (n < 4) return fail(VV_ERR_ARG, "VV_SHAPE=\"%s\": expected fft,R,tri,narrow[,march]", spec);
    const int kind = v[0], R = v[1], tk = v[2], nb = v[3], mw = v[4];
    if (kind < 0 || kind > 2 || ((kind == 0 || kind == 1) && !c->pow2) || (kind == 1 && !four_step_ok(c->M)))
        return fail(VV_ERR_ARG, "VV_SHAPE: FFT kind %d does not fit nx %d", kind, c->nx);
    if (R != 1 && R != 2 && R != 4 && R != 8)
        return fail(VV_ERR_ARG, "VV_SHAPE: rows per CTA %d not in {1, 2, 4, 8}", R);
    if (kind < 2 && fft_smem(kind, c->M, R, sizeof(double2), true) > (size_t)c->smem_limit)
        return fail(VV_ERR_ARG, "VV_SHAPE: %d FFT rows per CTA need more shared memory than the limit", R);
    if (tk != 0 && tk != 1) return fail(VV_ERR_ARG, "VV_SHAPE: tridiagonal kind %d not in {0, 1}", tk);
    if (nb != 0 && nb != 1) return fail(VV_ERR_ARG, "VV_SHAPE: narrow flag %d not in {0, 1}", nb);
    if (mw != 0 && ((mw != 128 && mw != 256) || c->nx % mw != 0))
        return fail(VV_ERR_ARG, "VV_SHAPE: marching strip width %d does not fit nx %d", mw, c->nx);
    c->fft_kind = kind;
    c->pcR = kind == 2 ? 1 : R;
    c->tri_kind = tk;
    c->narrow_bracket = nb;
    c->march = mw;
    return VV_OK;
}

void destroy_graph(vv_ctx* c) {
    if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
    if (c->step_graph) cudaGraphDestroy(c->step_graph);
    c->step_exec = nullptr;
    c->step_graph = nullptr;
}

// Capture one time step of context c into the graph being captured on c->st
// (the top-level stream of this instance); conditional handles are created
// on `owner`, the top-level graph.  Body graphs are captured on c->cs[1..3].
int capture_step(vv_ctx* c, vv_state* st, cudaGraph_t owner) {
    for (int k = 1; k < 4; ++k)
        if (!c->cs[k]) CK(cudaStreamCreateWithFlags(&c->cs[k], cudaStreamNonBlocking));
    for (auto& h : c->hnd) h = 0;   // new handles on `owner`
    c->cap_owner = owner;
    const int64_t l0 = c->launches;
    TRY(step_prologue(c, st));
    cudaGraph_t pic[1];
    TRY(add_conditional(owner, c->st, cudaGraphCondTypeWhile, 1, 0, &c->hnd[3], pic));
    TRY(capture_body(c, c->cs[1], pic[0], &c->nk_pic, [&]() -> int {
        TRY(step_rhs(c, st));
        if (c->mixed) TRY(capture_gmres<float>(c, 1, c->bvec32, c->delta32));
        else TRY(capture_gmres<double>(c, 1, c->bvec, c->delta));
        return step_after_solve(c, st);
    }));
    cudaGraph_t rev[1];
    TRY(add_conditional(owner, c->st, cudaGraphCondTypeIf, 1, 0, &c->hnd[4], rev));
    TRY(capture_body(c, c->cs[1], rev[0], &c->nk_revert, [&]() { return step_revert(c, st); }));
    c->nk_top = (int)(c->launches - l0);
    c->launches = l0;   // captured, not executed
    c->step_key = *st;
    return VV_OK;
}

// Build the graph of one time step for the buffers in `st`.
int build_step_graph(vv_ctx* c, vv_state* st) {
    destroy_graph(c);
    if (!c->cs[0]) CK(cudaStreamCreateWithFlags(&c->cs[0], cudaStreamNonBlocking));
    CK(cudaGraphCreate(&c->step_graph, 0));
    const cudaStream_t saved = c->st;
    CK(cudaStreamBeginCaptureToGraph(c->cs[0], c->step_graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    c->st = c->cs[0];
    int r = capture_step(c, st, c->step_graph);
    c->st = saved;
    cudaGraph_t out = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->cs[0], &out);
    if (r == VV_OK && e != cudaSuccess) r = fail_cuda(e, "cudaStreamEndCapture");
    if (r != VV_OK) {
        destroy_graph(c);
        return r;
    }
    e = cudaGraphInstantiate(&c->step_exec, c->step_graph, 0);
    if (e != cudaSuccess) {
        destroy_graph(c);
        return fail_cuda(e, "cudaGraphInstantiate");
    }
    std::memcpy(c->step_hnd, c->hnd, sizeof c->hnd);
    return VV_OK;
}

// Read the step report of context c from its pinned state copy.
int fill_report(vv_ctx* c, const vv::DevState& d, int restart, vv_step_report* rep, double abort_residual,
                bool count_launches = true) {
    std::memset(rep, 0, sizeof(*rep));
    rep->picard_its = d.pic_i;
    rep->gmres_its_total = d.gmres_total;
    rep->reverted = d.pic_revert;
    rep->stop_rule = d.pic_stop_rule;
    rep->ksp_failures = d.ksp_failures;
    const int np = std::min(d.pic_i, VV_MAX_PICARD);
    for (int k = 0; k < np; ++k) {
        rep->gmres_its[k] = d.gmres_its[k];
        rep->ksp_reason[k] = d.ksp_reason[k];
    }
    for (int k = 0; k <= np; ++k) rep->residual[k] = d.residual[k];
    if (c->pred) {
        rep->guess_kept = d.guess_kept;
        rep->guess_prev = d.guess_prev;
        rep->guess_residual = d.guess_res;
    }
    (void)restart;
    if (c->use_graph && count_launches) {
        // kernels the graph executed: top level once, the Picard body per pass,
        // the GMRES cycle body per cycle (+ restart branch), the Arnoldi body per iteration
        const int64_t top = c->nk_top - c->nk_pic - c->nk_revert;
        const int64_t cycles = d.ncycles;
        c->launches += top + (int64_t)np * (c->nk_pic - c->nk_cycle) +
                       cycles * (c->nk_cycle - c->nk_arnoldi - c->nk_restart) + (cycles - np) * c->nk_restart +
                       (int64_t)d.gmres_total * c->nk_arnoldi + (d.pic_revert ? c->nk_revert : 0);
    }
    if (std::isnan(d.pred)) return VV_ERR_NAN;
    if (d.pred > abort_residual) {
        rep->aborted = 1;
        return VV_ERR_DIVERGED;
    }
    return VV_OK;
}

// Host-driven time step with the same kernel sequence.
int step_host(vv_ctx* c, vv_state* st) {
    TRY(step_prologue(c, st));
    for (;;) {
        TRY(step_rhs(c, st));
        if (c->mixed) TRY(gmres_host<float>(c, c->bvec32, c->delta32, nullptr));
        else TRY(gmres_host<double>(c, c->bvec, c->delta, nullptr));
        TRY(step_after_solve(c, st));
        int act = 0;
        CK(cudaMemcpyAsync(c->hstat, &c->ds->pic_active, sizeof(int), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
        act = c->hstat[0];
        if (!act) break;
    }
    int rev = 0;
    CK(cudaMemcpyAsync(c->hstat, &c->ds->pic_revert, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    rev = c->hstat[0];
    if (rev) TRY(step_revert(c, st));
    return VV_OK;
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
    if (g.bracket != VV_BRACKET_J1 && g.bracket != VV_BRACKET_J2 && g.bracket != VV_BRACKET_J4 &&
        g.bracket != VV_BRACKET_SIMPSON)
        return VV_ERR_ARG;
    if (g.preconditioner != VV_PC_NONE && g.preconditioner != VV_PC_TENSOR_KINETIC &&
        g.preconditioner != VV_PC_TENSOR_POTENTIAL)
        return VV_ERR_ARG;
    if (g.laplace != VV_LAPLACE_CFD4 && g.laplace != VV_LAPLACE_CFD2 && g.laplace != VV_LAPLACE_SIMPSON &&
        g.laplace != VV_LAPLACE_CFD2_AVE && g.laplace != VV_LAPLACE_SIMPSON_AVE)
        return VV_ERR_UNSUPPORTED;
    if (g.averaging != VV_AVERAGING_POINT && g.averaging != VV_AVERAGING_MIDPOINT &&
        g.averaging != VV_AVERAGING_ARAKAWA_J2 && g.averaging != VV_AVERAGING_ARAKAWA_J4 &&
        g.averaging != VV_AVERAGING_SIMPSON)
        return VV_ERR_ARG;
    if (g.collision != VV_COLLISION_NONE && g.collision != VV_COLLISION_T && g.collision != VV_COLLISION_E)
        return VV_ERR_ARG;
    if (g.double_bracket != VV_DOUBLE_BRACKET_NONE && g.double_bracket != VV_DOUBLE_BRACKET_FFH &&
        g.double_bracket != VV_DOUBLE_BRACKET_FHH)
        return VV_ERR_ARG;
    if (g.double_bracket != VV_DOUBLE_BRACKET_NONE && g.coll_freq != 0.0 && g.precision == VV_PRECISION_MIXED)
        return VV_ERR_UNSUPPORTED;   // the double bracket runs in FP64 only
    const int restart = g.gmres_restart > 0 ? g.gmres_restart : 30;
    if (restart > vv::MAX_RESTART) return VV_ERR_ARG;
    if (g.precision != VV_PRECISION_FP64 && g.precision != VV_PRECISION_MIXED) return VV_ERR_ARG;
    if (g.initial_guess < VV_GUESS_NONE || g.initial_guess > VV_GUESS_RK4_18) return VV_ERR_ARG;

    vv_ctx* c = new vv_ctx();
    c->g = g;
    c->g.gmres_restart = restart;
    c->nx = g.nx;
    c->nv = g.nv;
    c->M = g.nx / 2;
    c->pow2 = is_pow2(g.nx);
    c->logM = c->pow2 ? ilog2(c->M) : -1;   // -1: the Poisson solve takes its direct-DFT branch
    c->nmodes = c->M + 1;
    c->restart = restart;
    c->mixed = g.precision == VV_PRECISION_MIXED;
    c->ncell = (size_t)g.nx * g.nv;
    c->st = 0;
    cudaGetDevice(&c->device);
    {
        const char* e = getenv("VV_GRAPH");
        c->use_graph = !(e && e[0] == '0');
    }
    // grid (run_base.py:133-137, Grid.pyx:40-48)
    c->hx = g.L / g.nx;
    c->hv = (g.vmax - g.vmin) / (g.nv - 1);
    c->ht_inv = 1. / g.ht;
    c->hx_inv = 1. / c->hx;
    c->hv_inv = 1. / c->hv;
    c->hx2_inv = 1. / (c->hx * c->hx);
    // the time derivative (TimeDerivative.pyx:36-53): time_fac = ht_inv / divisor
    c->avg = g.averaging == VV_AVERAGING_MIDPOINT   ? vv::AVG_MIDPOINT
             : g.averaging == VV_AVERAGING_SIMPSON  ? vv::AVG_SIMPSON
             : g.averaging == VV_AVERAGING_ARAKAWA_J4 ? vv::AVG_J4
                                                      : vv::AVG_POINT;
    c->tfac = c->ht_inv / vv::avg_divisor(c->avg);
    // collisions (CollisionOperator.create, config.py:148-154: none unless coll_freq != 0);
    // the factors of the midpoint rule's 1/2 in CollisionOperator.pyx:80-81's order
    c->coll = (g.collision != VV_COLLISION_NONE && g.coll_freq != 0.0)
                  ? (g.collision == VV_COLLISION_T ? vv::COLL_T : vv::COLL_E)
                  : vv::COLL_NONE;
    c->coll_drag_fac = -0.5 * g.coll_freq * g.coll_drag * c->hv_inv * 0.5;
    c->coll_diff_fac = -0.5 * g.coll_freq * g.coll_diff * (1. / (c->hv * c->hv));
    // the double bracket (DoubleBracket.create, config.py:156-162: none unless coll_freq != 0)
    c->db = (g.double_bracket != VV_DOUBLE_BRACKET_NONE && g.coll_freq != 0.0) ? g.double_bracket : 0;
    c->db_nu = g.coll_freq;
    c->pred = g.initial_guess;
    c->pred_iter = g.initial_iter > 0 ? g.initial_iter : 1;
    {   // the Laplacian's stencil (matrix_mult of PETScPoissonCFD2/CFD4/Simpson.pyx; the Ave classes
        // keep CFD2's / Simpson's) and the density average of their formRHS (PETScPoissonCFD2Ave.pyx:
        // 0.25 (n_{i-1} + 2 n_i + n_{i+1}); PETScPoissonSimpsonAve.pyx: (n_{i-2} + 8 n_{i-1} + 18 n_i
        // + 8 n_{i+1} + n_{i+2}) / 36)
        const double cfd2[4] = {2., -1., 0., 1.}, cfd4[4] = {54., -32., 5., 12.}, simp[4] = {30., -16., 1., 12.};
        const bool c2 = g.laplace == VV_LAPLACE_CFD2 || g.laplace == VV_LAPLACE_CFD2_AVE;
        const bool sp = g.laplace == VV_LAPLACE_SIMPSON || g.laplace == VV_LAPLACE_SIMPSON_AVE;
        const double* l = c2 ? cfd2 : sp ? simp : cfd4;
        for (int k = 0; k < 4; ++k) c->lap[k] = l[k];
        const double none[4] = {1., 0., 0., 1.}, a2[4] = {2., 1., 0., 4.}, as[4] = {18., 8., 1., 36.};
        const double* r = g.laplace == VV_LAPLACE_CFD2_AVE ? a2 : g.laplace == VV_LAPLACE_SIMPSON_AVE ? as : none;
        for (int k = 0; k < 4; ++k) c->ravg[k] = r[k];
    }
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
    // rows (warps) per CTA of the x-FFT kernels: 4 consecutive v rows per
    // transposed 64-byte write, fewer when shared memory would exceed 200 KB
    c->pcR = 4;
    while (c->pcR > 1 && (size_t)(M + 2 * c->pcR * (M + 1)) * sizeof(double2) > 200 * 1024) c->pcR /= 2;
    c->smem_rfft = (size_t)(M + c->pcR * (M + 1)) * sizeof(double2);
    c->smem_irfft = (size_t)(M + 2 * c->pcR * (M + 1)) * sizeof(double2);
    {
        const int ch = (nv + vv::TRI_THREADS - 1) / vv::TRI_THREADS;
        const size_t np = (size_t)nv + (nv + ch - 1) / ch;
        c->tri_stage = np * 48 <= 200 * 1024;
        c->smem_tri = c->tri_stage ? np * 48 : np * sizeof(double2);
        c->tri_stage32 = np * 24 <= 200 * 1024;
        c->smem_tri32 = c->tri_stage32 ? np * 24 : np * sizeof(float2);
    }
    c->smem_rfft32 = (size_t)(M + c->pcR * (M + 1)) * sizeof(float2);
    c->smem_irfft32 = (size_t)(M + 2 * c->pcR * (M + 1)) * sizeof(float2);
    // moments_poisson_cta: M+1 complex, nx (padded to even) and nx + 2 doubles
    c->smem_pois = (size_t)(M + 1) * sizeof(double2) + (size_t)((nx + 1) & ~1) * sizeof(double) +
                   (size_t)(nx + 2) * sizeof(double);

    int s = VV_OK;
    const int tiles = ((nx + vv::BX - 1) / vv::BX) * ((nv + vv::BY - 1) / vv::BY);  // the largest grid
    const size_t part_count = std::max({(size_t)(vv::MAX_RESTART + 2) * c->npart_max, (size_t)tiles,
                                        (size_t)vv::INV_NPART * c->npart_max});
    if ((s = dalloc(&c->v, nv)) || (s = dalloc(&c->h0, nv)) || (s = dalloc(&c->hxp, 4 * (size_t)nx)) ||
        (s = dalloc(&c->Fh, n)) || (s = dalloc(&c->tmp, n)) || (s = dalloc(&c->bvec, n)) ||
        (s = dalloc(&c->delta, n)) || (s = dalloc(&c->fl, n)) ||
        (s = dalloc(&c->V, (size_t)(c->mixed ? 1 : restart + 1) * n)) ||
        (s = dalloc(&c->part, part_count)) || (s = dalloc(&c->scal, 64)) || (s = dalloc(&c->xscratch, 2 * (size_t)nx)) ||
        (s = dalloc(&c->mom_part, (size_t)c->mom_S * 3 * nx)) || (s = dalloc(&c->spec, (size_t)nm * nv)) ||
        (s = dalloc(&c->tw, (size_t)nx)) || (s = dalloc(&c->lambda, nm)) ||
        (s = dalloc(&c->dinv, (size_t)nm * nv)) || (s = dalloc(&c->alpha, nv)) || (s = dalloc(&c->gamma, nv)) ||
        (s = dalloc(&c->sym_inv, nm)) || (s = dalloc(&c->ds, 1))) {
        vv_destroy(c);
        return s;
    }
    if (c->mixed &&
        ((s = dalloc(&c->V32, (size_t)(restart + 1) * n)) || (s = dalloc(&c->tmp32, n)) || (s = dalloc(&c->bvec32, n)) ||
         (s = dalloc(&c->delta32, n)) || (s = dalloc(&c->alpha32, nv)) || (s = dalloc(&c->gamma32, nv)) ||
         (s = dalloc(&c->spec32, (size_t)nm * nv)) || (s = dalloc(&c->tw32, (size_t)nx)) ||
         (s = dalloc(&c->lambda32, nm)) || (s = dalloc(&c->dinv32, (size_t)nm * nv)))) {
        vv_destroy(c);
        return s;
    }
    if (cudaMallocHost((void**)&c->hpin, 4096) != cudaSuccess ||
        cudaMallocHost((void**)&c->hds, sizeof(vv::DevState)) != cudaSuccess ||
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
    std::vector<double2> tw(nx);   // W^k = exp(-2 pi i k / nx), k < nx
    for (int k = 0; k < nx; ++k) {
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
    // the Laplacian's symbol (e.g. CFD4, PETScPoissonCFD4.pyx:130-134: (54 - 64 cos t + 10 cos 2t)/(12 hx^2))
    // and, for the Ave operators, the symbol of the density average in the numerator
    std::vector<double> sym(nm);
    for (int k = 0; k < nm; ++k) {
        const long double t = 2.0L * PI * (long double)k / (long double)nx;
        const long double s_ = ((long double)c->lap[0] + 2.0L * (long double)c->lap[1] * cosl(t) +
                                2.0L * (long double)c->lap[2] * cosl(2.0L * t)) *
                               (long double)c->hx2_inv / (long double)c->lap[3];
        const long double a_ = ((long double)c->ravg[0] + 2.0L * (long double)c->ravg[1] * cosl(t) +
                                2.0L * (long double)c->ravg[2] * cosl(2.0L * t)) /
                               (long double)c->ravg[3];
        sym[k] = (k == 0) ? 0.0 : (double)(a_ / s_);
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
        cudaMemset(c->Fh, 0, n * sizeof(double)) != cudaSuccess ||
        cudaMemset(c->ds, 0, sizeof(vv::DevState)) != cudaSuccess) {
        vv_destroy(c);
        return fail_cuda(cudaGetLastError(), "vv_create upload");
    }
    if (c->mixed) {
        std::vector<float> a32(alpha.begin(), alpha.end()), g32(gamma.begin(), gamma.end());
        std::vector<float2> tw32(tw.size()), lam32(nm), dinv32(dinv.size());
        for (size_t k = 0; k < tw.size(); ++k) tw32[k] = make_float2((float)tw[k].x, (float)tw[k].y);
        for (int k = 0; k < nm; ++k) lam32[k] = make_float2((float)lam2[k].x, (float)lam2[k].y);
        for (size_t k = 0; k < dinv.size(); ++k) dinv32[k] = make_float2((float)dinv[k].x, (float)dinv[k].y);
        if (cudaMemcpy(c->alpha32, a32.data(), nv * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(c->gamma32, g32.data(), nv * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(c->tw32, tw32.data(), tw32.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(c->lambda32, lam32.data(), nm * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(c->dinv32, dinv32.data(), dinv32.size() * sizeof(float2), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
            vv_destroy(c);
            return fail_cuda(cudaGetLastError(), "vv_create upload (fp32)");
        }
    }
    // the potential preconditioner: eigenvalues for n = nv (TensorProduct.pyx:109-116
    // with the ifftshift), nv twiddles, buffers; phi starts at zero until
    // vv_pc_set_potential or a step's make_history sets it
    if (g.preconditioner == VV_PC_TENSOR_POTENTIAL) {
        const int nmv = nv / 2 + 1;
        c->nmv = nmv;
        c->pvR = 4;
        while (c->pvR > 1 && fft_smem(0, nv / 2, c->pvR, sizeof(double2), true) > 200 * 1024) c->pvR /= 2;
        if ((s = dalloc(&c->lamv, nmv)) || (s = dalloc(&c->twv, (size_t)nv)) || (s = dalloc(&c->pv_xt, n)) ||
            (s = dalloc(&c->pv_spec, (size_t)nmv * nx)) || (s = dalloc(&c->pv_scr, (size_t)3 * nmv * nx)) ||
            (s = dalloc(&c->phipc, (size_t)nx)) ||
            (c->mixed && ((s = dalloc(&c->twv32, (size_t)nv)) || (s = dalloc(&c->pv_xt32, n)) ||
                          (s = dalloc(&c->pv_spec32, (size_t)nmv * nx)) ||
                          (s = dalloc(&c->pv_scr32, (size_t)3 * nmv * nx))))) {
            vv_destroy(c);
            return s;
        }
        std::vector<cd> ev(nv);
        for (int i = 0; i < nv; ++i) {
            const double t2 = (twopi * (double)i) / (double)nv;
            const double t1 = t2 * (double)(nv - 1);
            ev[i] = cd(std::cos(t1), std::sin(t1)) - cd(std::cos(t2), std::sin(t2));
        }
        std::vector<double2> lv(nmv), twvh(nv);
        std::vector<float2> twv32h(nv);
        for (int k = 0; k < nmv; ++k) {
            const cd L = ev[(k + nv / 2) % nv];
            lv[k] = make_double2(L.real(), L.imag());
        }
        for (int k = 0; k < nv; ++k) {
            const long double a = 2.0L * PI * (long double)k / (long double)nv;
            twvh[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
            twv32h[k] = make_float2((float)twvh[k].x, (float)twvh[k].y);
        }
        if (cudaMemcpy(c->lamv, lv.data(), nmv * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(c->twv, twvh.data(), nv * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
            (c->mixed && cudaMemcpy(c->twv32, twv32h.data(), nv * sizeof(float2), cudaMemcpyHostToDevice) !=
                             cudaSuccess) ||
            cudaMemset(c->phipc, 0, nx * sizeof(double)) != cudaSuccess) {
            vv_destroy(c);
            return fail_cuda(cudaGetLastError(), "vv_create upload (potential preconditioner)");
        }
    }
    // double bracket: Fave and the inner bracket
    if (c->db && ((s = dalloc(&c->db_fave, n)) || (s = dalloc(&c->db_b, n)))) {
        vv_destroy(c);
        return s;
    }
    if (c->db && (cudaMemset(c->db_fave, 0, n * sizeof(double)) != cudaSuccess ||
                  cudaMemset(c->db_b, 0, n * sizeof(double)) != cudaSuccess)) {
        vv_destroy(c);
        return fail_cuda(cudaGetLastError(), "vv_create upload (double bracket)");
    }
    // the predictor's work fields
    if (c->pred) {
        const size_t ntile = (size_t)((nx + vv::BX - 1) / vv::BX) * ((nv + vv::BY - 1) / vv::BY);
        if ((s = dalloc(&c->pred_H, n)) || (s = dalloc(&c->pred_Hp, n)) || (s = dalloc(&c->pred_Y, n)) ||
            (s = dalloc(&c->pred_K, 4 * n)) || (s = dalloc(&c->pred_S, n)) || (s = dalloc(&c->pred_fl, n)) ||
            (s = dalloc(&c->pred_cpart, ntile)) || (s = dalloc(&c->pred_zero, n))) {
            vv_destroy(c);
            return s;
        }
        if (cudaMemset(c->pred_zero, 0, n * sizeof(double)) != cudaSuccess) {
            vv_destroy(c);
            return fail_cuda(cudaGetLastError(), "vv_create (predictor)");
        }
    }
    // collisions: current / history moment profiles (n, U, a)
    if (c->coll != vv::COLL_NONE) {
        if ((s = dalloc(&c->mom_p, (size_t)3 * nx)) || (s = dalloc(&c->mom_h, (size_t)3 * nx))) {
            vv_destroy(c);
            return s;
        }
        c->coll_p = {c->mom_p, c->mom_p + nx, c->mom_p + 2 * nx};
        c->coll_h = {c->mom_h, c->mom_h + nx, c->mom_h + 2 * nx};
        if (cudaMemset(c->mom_p, 0, 3 * nx * sizeof(double)) != cudaSuccess ||
            cudaMemset(c->mom_h, 0, 3 * nx * sizeof(double)) != cudaSuccess) {
            vv_destroy(c);
            return fail_cuda(cudaGetLastError(), "vv_create upload (collision moments)");
        }
    }
    // dynamic shared memory limits (process-wide, raised once per device)
    {
        int limit = 0;
        if ((s = raise_smem_limits(&limit)) != VV_OK) {
            vv_destroy(c);
            return s;
        }
        c->smem_limit = limit;
        const size_t need = std::max({c->smem_tri, c->mixed ? c->smem_tri32 : (size_t)0, c->smem_pois,
                                      c->pow2 ? fft_smem(0, M, c->pcR, sizeof(double2), true)
                                              : std::max(rdft_smem(nx, sizeof(double2)), irdft_smem(nx, sizeof(double2)))});
        if (need > (size_t)limit) {
            vv_destroy(c);
            return fail(VV_ERR_ARG, "grid %d x %d needs %zu bytes of shared memory per block (limit %d)", nx, nv,
                        need, limit);
        }
    }
    c->fft_kind = !c->pow2 ? 2 : four_step_ok(c->M) ? 1 : 0;
    c->tri_kind = c->nmodes >= 64 ? 1 : 0;
    c->narrow_bracket = 0;
    c->march = 0;
    {
        const char* e = getenv("VV_MARCH");   // fixed strip width (tests, profiling); the autotuner may override
        if (e) c->march = atoi(e);
    }
    {
        // VV_SHAPE="fft,R,tri,narrow[,march]" fixes the kernel variants (tests run each variant
        // explicitly; profiling); else the autotuner picks them by timing
        const char* sh = getenv("VV_SHAPE");
        if (sh && sh[0]) {
            if ((s = apply_shape(c, sh)) != VV_OK) {
                vv_destroy(c);
                return s;
            }
            *out = c;
            return VV_OK;
        }
    }
    {
        const char* e = getenv("VV_AUTOTUNE");
        if (!(e && e[0] == '0')) {
            if ((s = autotune(c)) != VV_OK) {
                vv_destroy(c);
                return s;
            }
        }
    }
    *out = c;
    return VV_OK;
}

int vv_destroy(vv_ctx* c) {
    if (!c) return VV_OK;
    void* bufs[] = {c->v, c->h0, c->hxp, c->Fh, c->tmp, c->bvec, c->delta, c->fl, c->V, c->part, c->scal,
                    c->xscratch, c->mom_part, c->spec, c->tw, c->lambda, c->dinv, c->alpha, c->gamma,
                    c->sym_inv, c->ds, c->V32, c->tmp32, c->bvec32, c->delta32, c->alpha32, c->gamma32,
                    c->spec32, c->tw32, c->lambda32, c->dinv32, c->adj_cH, c->adj_cF, c->adj_zpart,
                    c->adj_zbuf, c->adj_q, c->adj_hprof, c->adj_h1a, c->adj_h1b, c->lamv, c->twv, c->pv_spec,
                    c->pv_scr, c->pv_xt, c->phipc, c->twv32, c->pv_spec32, c->pv_scr32, c->pv_xt32,
                    c->mom_p, c->mom_h, c->db_fave, c->db_b, c->pred_H, c->pred_Hp, c->pred_Y, c->pred_K,
                    c->pred_S, c->pred_fl, c->pred_cpart, c->pred_zero};
    destroy_graph(c);
    for (int k = 0; k < 4; ++k)
        if (c->cs[k]) cudaStreamDestroy(c->cs[k]);
    if (c->hds) cudaFreeHost(c->hds);
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
    TRY(set_hxp(c, h1p, h1h, h2p, h2h));
    vv::k_set_have<<<1, 1, 0, c->st>>>(c->ds);
    CKL(c);
    return VV_OK;
}

int vv_predict(vv_ctx* c, const double* F, const double* h1h, const double* h2h, double* Y) {
    if (!c || !F || !Y || !c->pred) return VV_ERR_ARG;
    return pred_run(c, F, h1h, h2h, Y);
}

int vv_initial_guess(vv_ctx* c, vv_state* st, double* prev, double* guess, int32_t* kept) {
    if (!c || !st || !st->f || !st->phi || !st->n || !st->h1c || !c->pred) return VV_ERR_ARG;
    TRY(pred_guess(c, st));
    CK(cudaMemcpyAsync(c->hds, c->ds, offsetof(vv::DevState, hcol), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (prev) *prev = c->hds->guess_prev;
    if (guess) *guess = c->hds->guess_res;
    if (kept) *kept = c->hds->guess_kept;
    return VV_OK;
}

int vv_function(vv_ctx* c, const double* F, double* Y, int apply_pc) {
    if (!c || !F || !Y) return VV_ERR_ARG;
    const bool pc = apply_pc && c->g.preconditioner != VV_PC_NONE;
    TRY(launch_bracket<vv::MODE_RESIDUAL, double>(c, F, c->Fh, pc ? c->tmp : Y, 1.0, nullptr));
    if (pc) TRY(pc_apply(c, c->tmp, Y));
    return VV_OK;
}

int vv_jacobian(vv_ctx* c, const double* F, double* Y, int apply_pc) {
    if (!c || !F || !Y) return VV_ERR_ARG;
    const bool pc = apply_pc && c->g.preconditioner != VV_PC_NONE;
    TRY(launch_bracket<vv::MODE_JVP, double>(c, F, nullptr, pc ? c->tmp : Y, 0.5, nullptr));
    if (pc) TRY(pc_apply(c, c->tmp, Y));
    return VV_OK;
}

int vv_function_norm(vv_ctx* c, const double* F, double* Y, double* norm) {
    if (!c || !F || !Y || !norm) return VV_ERR_ARG;
    return residual_norm(c, F, Y, norm);
}

int vv_bracket(vv_ctx* c, const double* X, double* Y, double factor) {
    if (!c || !X || !Y) return VV_ERR_ARG;
    return launch_bracket<vv::MODE_ADD, double>(c, X, nullptr, Y, factor, nullptr);
}

int vv_pc_apply(vv_ctx* c, const double* X, double* Y) {
    if (!c || !X || !Y) return VV_ERR_ARG;
    if (c->g.preconditioner == VV_PC_NONE) return copy_d(c, Y, X, c->ncell);
    return pc_apply(c, X, Y);
}

int vv_set_moments(vv_ctx* c, const double* n_p, const double* u_p, const double* e_p, const double* a_p,
                   const double* n_h, const double* u_h, const double* e_h, const double* a_h) {
    (void)e_p;
    (void)e_h;   // the collision operators read n, U and a only
    if (!c || !n_p || !u_p || !a_p || !n_h || !u_h || !a_h) return VV_ERR_ARG;
    if (c->coll == vv::COLL_NONE) return VV_OK;
    const int nx = c->nx;
    TRY(copy_d(c, c->mom_p, n_p, nx));
    TRY(copy_d(c, c->mom_p + nx, u_p, nx));
    TRY(copy_d(c, c->mom_p + 2 * nx, a_p, nx));
    TRY(copy_d(c, c->mom_h, n_h, nx));
    TRY(copy_d(c, c->mom_h + nx, u_h, nx));
    TRY(copy_d(c, c->mom_h + 2 * nx, a_h, nx));
    c->coll_p = {c->mom_p, c->mom_p + nx, c->mom_p + 2 * nx};
    return VV_OK;
}

int vv_pc_set_potential(vv_ctx* c, const double* phi) {
    if (!c || !phi) return VV_ERR_ARG;
    if (c->g.preconditioner != VV_PC_TENSOR_POTENTIAL) return VV_OK;
    return copy_d(c, c->phipc, phi, c->nx);
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
    const int restart = (o->restart > 0) ? o->restart : c->restart;
    if (restart > c->restart || restart < 1 || o->max_it < 0) return VV_ERR_ARG;
    const unsigned long long saved[5] = {c->hnd[0], c->hnd[1], c->hnd[2], c->hnd[3], c->hnd[4]};
    for (auto& h : c->hnd) h = 0;   // host-driven: no conditional handles
    c->opts_valid = false;
    int s = upload_options(c, o, nullptr);
    c->opts_valid = false;
    for (int k = 0; k < 5; ++k) c->hnd[k] = saved[k];
    TRY(s);
    if (!c->mixed) return gmres_host<double>(c, b, x, r);
    // mixed: FP32 solve of the FP64 system, converted at the boundary
    vv::k_scale<double, float><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(b, c->bvec32, c->ncell, nullptr, 1.0);
    CKL(c);
    TRY(gmres_host<float>(c, c->bvec32, c->delta32, r));
    vv::k_scale<float, double><<<grid1d(c->ncell, 256), 256, 0, c->st>>>(c->delta32, x, c->ncell, nullptr, 1.0);
    CKL(c);
    return VV_OK;
}

}  // extern "C"

namespace {

int adj_buffers(vv_ctx* c) {
    if (c->adj_cH) return VV_OK;
    int s = VV_OK;
    const size_t nx = c->nx;
    if ((s = dalloc(&c->adj_cH, (size_t)vv::ADJ_NOFF * c->ncell)) || (s = dalloc(&c->adj_cF, (size_t)vv::ADJ_NOFF * c->ncell)) ||
        (s = dalloc(&c->adj_zpart, (size_t)c->mom_S * nx)) || (s = dalloc(&c->adj_zbuf, nx)) ||
        (s = dalloc(&c->adj_q, nx)) || (s = dalloc(&c->adj_hprof, nx)) || (s = dalloc(&c->adj_h1a, nx)) ||
        (s = dalloc(&c->adj_h1b, nx)))
        return s;
    return VV_OK;
}

template <int S>
int adj_coefs(vv_ctx* c, const double* F, const double* f) {
    const vv::AdjParams p = adjparams(c);
    const dim3 grid((c->nx + 255) / 256, c->nv);
    vv::k_adj_coef<S, 0><<<grid, 256, 0, c->st>>>(p, c->h0, c->adj_hprof, nullptr, nullptr, c->adj_cH);
    CKL(c);
    vv::k_adj_coef<S, 1><<<grid, 256, 0, c->st>>>(p, nullptr, nullptr, F, f, c->adj_cF);
    CKL(c);
    return VV_OK;
}

}  // namespace

extern "C" {

int vv_step_adjoint(vv_ctx* c, const double* F, const double* f, const double* h2p, const double* h2h,
                    const double* gF, double* gf, const vv_ksp_opts* o, vv_ksp_result* r) {
    if (!c || !F || !f || !gF || !gf || !o || !r) return VV_ERR_ARG;
    if (c->mixed) return VV_ERR_UNSUPPORTED;
    if (c->g.bracket == VV_BRACKET_SIMPSON)   // the transposed stencil is built for the Arakawa brackets
        return fail(VV_ERR_UNSUPPORTED, "vv_step_adjoint: the Simpson bracket has no transposed stencil here");
    if (c->avg != vv::AVG_POINT)   // the transposed operator is built for the point time derivative
        return fail(VV_ERR_UNSUPPORTED, "vv_step_adjoint: averaged time derivatives have no transposed stencil here");
    if (c->coll != vv::COLL_NONE || c->db)
        return fail(VV_ERR_UNSUPPORTED, "vv_step_adjoint: the dissipative terms have no transposed stencil here");
    const int restart = (o->restart > 0) ? o->restart : c->restart;
    if (restart > c->restart || restart < 1 || o->max_it < 0) return VV_ERR_ARG;
    TRY(adj_buffers(c));
    // H = h0 + (h1(F) + h1(f) + h2p + h2h)/2 and Fbar = (F + f)/2 as coefficient planes
    TRY(moments_poisson(c, F, nullptr, nullptr, nullptr, nullptr, nullptr, c->adj_h1a, nullptr));
    TRY(moments_poisson(c, f, nullptr, nullptr, nullptr, nullptr, nullptr, c->adj_h1b, nullptr));
    vv::k_adj_hprof<<<1, 256, 0, c->st>>>(c->nx, c->adj_h1a, c->adj_h1b, h2p, h2h, c->adj_hprof);
    CKL(c);
    switch (c->g.bracket) {
        case VV_BRACKET_J1: TRY(adj_coefs<1>(c, F, f)); break;
        case VV_BRACKET_J2: TRY(adj_coefs<2>(c, F, f)); break;
        default: TRY(adj_coefs<4>(c, F, f)); break;
    }
    // left-preconditioned transpose system  P^-T A^T lambda = P^-T gF
    TRY(pcT_apply(c, gF, c->bvec));
    const unsigned long long saved[5] = {c->hnd[0], c->hnd[1], c->hnd[2], c->hnd[3], c->hnd[4]};
    for (auto& h : c->hnd) h = 0;
    c->opts_valid = false;
    int s = upload_options(c, o, nullptr);
    c->opts_valid = false;
    for (int k = 0; k < 5; ++k) c->hnd[k] = saved[k];
    TRY(s);
    c->adj = true;
    s = gmres_host<double>(c, c->bvec, c->delta, r);
    c->adj = false;
    TRY(s);
    vv::k_adj_pull<<<grid1d(c->ncell, 256), 256, 0, c->st>>>(adjparams(c), gF, c->delta, gf);
    CKL(c);
    return VV_OK;
}

int vv_field_energy_grad(vv_ctx* c, const double* f, double* g) {
    if (!c || !f || !g) return VV_ERR_ARG;
    TRY(adj_buffers(c));
    // phi of f, then dW/dphi, then the transpose of the moments -> Poisson chain
    TRY(moments_poisson(c, f, nullptr, nullptr, nullptr, nullptr, c->adj_h1a, nullptr, nullptr));
    vv::k_adj_fe_gphi<<<1, 1024, 0, c->st>>>(c->nx, c->g.charge, c->hx, c->adj_h1a, c->adj_zpart);
    CKL(c);
    vv::k_adj_poisson<<<1, vv::POIS_THREADS, c->smem_pois, c->st>>>(c->adj_zpart, 1, c->adj_zbuf, c->adj_q, pparams(c));
    CKL(c);
    vv::k_adj_fill<<<grid1d(c->ncell, 256), 256, 0, c->st>>>(adjparams(c), c->adj_q, g);
    CKL(c);
    return VV_OK;
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
    const int restart = (ko->restart > 0) ? ko->restart : c->restart;
    if (restart > c->restart || restart < 1 || ko->max_it < 0 || so->max_iter < 1) return VV_ERR_ARG;
    if (c->coll != vv::COLL_NONE) {   // the collision operator reads the state's moments (set_moments nc, uc, ac)
        if (!st->u || !st->a) return VV_ERR_ARG;
        c->coll_p = {st->n, st->u, st->a};
    }
    std::memset(rep, 0, sizeof(*rep));
    if (c->use_graph) {
        if (!c->step_exec || !same_state(c->step_key, *st)) TRY(build_step_graph(c, st));
        std::memcpy(c->hnd, c->step_hnd, sizeof c->hnd);
        TRY(upload_options(c, ko, so));
        CK(cudaGraphLaunch(c->step_exec, c->st));
    } else {
        const unsigned long long saved[5] = {c->hnd[0], c->hnd[1], c->hnd[2], c->hnd[3], c->hnd[4]};
        for (auto& h : c->hnd) h = 0;
        int s = upload_options(c, ko, so);
        for (int k = 0; k < 5; ++k) c->hnd[k] = saved[k];
        TRY(s);
        TRY(step_host(c, st));
    }
    // report
    CK(cudaMemcpyAsync(c->hds, c->ds, offsetof(vv::DevState, hcol), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return fill_report(c, *c->hds, restart, rep, so->abort_residual);
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

int vv_time_kernel(vv_ctx* c, int which, int reps, double* avg_ms) {
    if (!c || !avg_ms || reps < 1 || reps > 100000 || which < 0 || which > 2) return VV_ERR_ARG;
    for (int k = 0; k < 4; ++k)
        if (!c->cs[k]) CK(cudaStreamCreateWithFlags(&c->cs[k], cudaStreamNonBlocking));
    const cudaStream_t saved = c->st;
    const int64_t l0 = c->launches;
    cudaGraph_t g = nullptr;
    CK(cudaStreamSynchronize(saved));
    CK(cudaStreamBeginCapture(c->cs[0], cudaStreamCaptureModeRelaxed));
    c->st = c->cs[0];
    int r = VV_OK;
    for (int k = 0; k < reps && r == VV_OK; ++k) {
        if (which == 0) {
            if (c->mixed) r = launch_bracket<vv::MODE_JVP, float>(c, c->V32, nullptr, c->tmp32, 0.5, nullptr);
            else r = launch_bracket<vv::MODE_JVP, double>(c, c->V, nullptr, c->tmp, 0.5, nullptr);
        } else if (which == 1) {
            r = launch_bracket<vv::MODE_RESIDUAL, double>(c, c->V, c->Fh, c->tmp, 1.0, nullptr);
        } else {
            if (c->mixed) r = pc_apply_t<float, float, float>(c, c->V32, c->tmp32);
            else r = pc_apply(c, c->V, c->tmp);
        }
    }
    c->st = saved;
    cudaError_t e = cudaStreamEndCapture(c->cs[0], &g);
    c->launches = l0;
    if (r != VV_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture");
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGraphInstantiate");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaGraphLaunch(ex, c->st);                    // warm-up
    cudaEventRecord(e0, c->st);
    cudaGraphLaunch(ex, c->st);
    cudaEventRecord(e1, c->st);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(ex);
    if (e != cudaSuccess) return fail_cuda(e, "vv_time_kernel");
    *avg_ms = (double)ms / reps;
    return VV_OK;
}

int vv_kernel_shape(vv_ctx* c, int32_t* shape) {
    if (!c || !shape) return VV_ERR_ARG;
    shape[0] = c->fft_kind;
    shape[1] = c->pcR;
    shape[2] = c->tri_kind;
    shape[3] = c->narrow_bracket;
    shape[4] = c->march;
    return VV_OK;
}

int vv_launch_count(vv_ctx* c, int64_t* launches, int reset) {
    if (!c) return VV_ERR_ARG;
    if (launches) *launches = c->launches;
    if (reset) c->launches = 0;
    return VV_OK;
}


// ---- batched sweep: lockstep over an instance table --------------------------
}  // extern "C"

// One graph (or host-driven loop) advances every instance of the batch by one
// time step.  Each kernel launch covers all instances with a persistent grid
// that walks the work list of the current mask; the Picard/GMRES loops run in
// lockstep, and the batch loop conditions are the OR of the instance flags
// (k_b_ctrl, which also rebuilds the work lists).
struct vv_batch {
    int n;
    std::vector<vv_ctx*> ctx;
    std::vector<vv_state> states;
    bool mixed;
    int scheme;
    int R;                       // FFT rows per CTA
    int fft4;                    // x-FFTs: 1 four-step register/shuffle, 0 radix-2
    int pcj;                     // 1: preconditioner in the v-major layout (vv_pcj.cuh); fft4/R unused
    int march;                   // 1: Jacobian stencil by the marching kernel, 0: 64 x 32 tiles
    bool pcj_ok;                 // every instance has M in 32..256 (the v-major kernels' lengths)
    void* dinvJ;                 // device: v-major LU reciprocals of every instance (GMRES precision)
    void* jtab;                  // device: every instance's Jacobian stencil coefficient tables (k_b_jcoef)
    size_t smem_fftj;            // dynamic shared memory of the v-major FFT blocks
    size_t smem_fjv;             // ... of the Jacobian stencil fused with the x-FFT (k_b_jvp_rfftj)
    int fuse;                    // 1: the GMRES operator's stencil runs inside the preconditioner's x-FFT
    int tri_kind;                // tridiagonal solves: 0 CTA per mode (tables staged), 1 warp per mode,
                                 // 2 CTA per mode (tables through L1); v-major: 0 lane per mode, 1 warp
                                 // per mode, 2/3 two/four warps per mode, 4 lanes by line length, 5 lane
                                 // per mode with chunk scans, 6 register-resident chunks
    size_t smem_tri_stage, smem_tri_plain, smem_tri_warp;
    size_t smem_tri_js;          // k_b_tridiagjs (padded warp slices)
    size_t smem_tri_jm2, smem_tri_jm4;   // k_b_tridiagjm, 2 and 4 warps per mode
    size_t smem_tri_jv;                  // k_b_tridiagjv (lanes per mode by line length)
    int nvmax;                   // largest velocity grid of the table
    int smem_limit;              // dynamic shared memory per block available to the batch kernels
    double* wpart;               // device: per-warp partial sums of every instance
    vv::BInst* tab;              // device instance table
    int* lists;                  // device work lists (vv::NLIST of them)
    size_t list_words;
    int tot[vv::NFAM];           // work items per family over all instances
    size_t smem_rfft, smem_irfft, smem_pois;
    unsigned int* counts;        // device: passes per control op
    int* flag;                   // device: last control result
    int* hflag;                  // pinned
    unsigned int* hcounts;       // pinned
    unsigned int* gather;        // device: n state headers
    unsigned int* hgather;       // pinned
    int words;                   // 32-bit words of a state header
    int nsm;                     // multiprocessors
    cudaStream_t st;             // stream of the kernels (the capture stream during capture)
    cudaStream_t user;
    cudaStream_t cs[4];
    cudaGraph_t g;
    cudaGraphExec_t ex;
    unsigned long long hnd[4];   // batch handles: pic, outer, inner, revert (index = BH_*)
    bool use_graph;
    int64_t launches;
    int64_t pending_l0 = 0;      // launch count before the uncollected launch
    int pending = 0;             // 1: a vv_batch_launch awaits its vv_batch_collect
    int nk_prologue, nk_pic_head, nk_cycle_head, nk_arnoldi, nk_cycle_tail, nk_pic_tail, nk_revert_ctrl, nk_revert;
};

namespace {

enum { BH_PIC = 0, BH_OUTER = 1, BH_INNER = 2, BH_REVERT = 3 };

// Persistent launch of a batch kernel over family `fam`: as many blocks as fit
// on the GPU at once (never more than the family's work items).
template <typename... KA, typename... A>
int blaunch(vv_batch* b, void (*k)(KA...), int fam, dim3 threads, size_t smem, A... args) {
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, (int)(threads.x * threads.y * threads.z),
                                                                  smem);
    if (e != cudaSuccess) return fail_cuda(e, "batch occupancy");
    const long cap = (long)std::max(1, per_sm) * b->nsm;
    const unsigned grid = (unsigned)std::max<long>(1, std::min<long>(cap, b->tot[fam]));
    k<<<grid, threads, smem, b->st>>>(args...);
    b->launches++;
    e = cudaGetLastError();
    return e == cudaSuccess ? VV_OK : fail_cuda(e, "batch kernel launch");
}

const int* blist(const vv_batch* b, int l) { return b->lists + (size_t)l * b->list_words; }

int b_ctrl(vv_batch* b, int op, int h) {
    vv::k_b_ctrl<<<1, vv::CTRL_THREADS, 0, b->st>>>(b->tab, b->n, op, (b->use_graph && h >= 0) ? b->hnd[h] : 0ull,
                                                     b->flag, b->counts, b->lists);
    b->launches++;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VV_OK : fail_cuda(e, "batch control launch");
}

int b_flag(vv_batch* b, int* out) {
    CK(cudaMemcpyAsync(b->hflag, b->flag, sizeof(int), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    *out = *b->hflag;
    return VV_OK;
}

// the tridiagonal stage of P^-1 (the tuned kernel) on the spectra of the
// instances in list L, in place
template <typename T>
int b_tri(vv_batch* b, const int* L) {
    const vv::BInst* tab = b->tab;
    if (b->pcj) {
        if (b->tri_kind == 1)
            return blaunch(b, vv::k_b_tridiagjs<T>, vv::F_MODES, 32 * vv::TRIW_WARPS, b->smem_tri_js, tab, L, b->n,
                           vv::tri_ws_slots(b->nvmax));
        if (b->tri_kind == 2)
            return blaunch(b, vv::k_b_tridiagjm<T, 2>, vv::F_MODES, 32 * vv::TRIW_WARPS * 2, b->smem_tri_jm2, tab, L,
                           b->n, b->nvmax);
        if (b->tri_kind == 3)
            return blaunch(b, vv::k_b_tridiagjm<T, 4>, vv::F_MODES, 32 * vv::TRIW_WARPS * 4, b->smem_tri_jm4, tab, L,
                           b->n, b->nvmax);
        if (b->tri_kind == 4)
            return blaunch(b, vv::k_b_tridiagjv<T>, vv::F_MODES, vv::TJV_THREADS, b->smem_tri_jv, tab, L, b->n);
        if (b->tri_kind == 5)
            return blaunch(b, vv::k_b_tridiagjc<T>, vv::F_MODES, vv::TJC_THREADS, 0, tab, L, b->n);
        if (b->tri_kind == 6)
            return blaunch(b, vv::k_b_tridiagjr<T>, vv::F_MODES, vv::TJR_THREADS, 0, tab, L, b->n);
        return blaunch(b, vv::k_b_tridiagj<T>, vv::F_MODES, 32,
                       (size_t)64 * vv::TJ_RING * sizeof(typename Cplx<T>::type), tab, L, b->n);
    }
    if (b->tri_kind == 1)
        return blaunch(b, vv::k_b_tridiag_w<T>, vv::F_MODES, 32 * vv::TRIW_WARPS, b->smem_tri_warp, tab, L, b->n,
                       vv::tri_ws_slots(b->nvmax));
    if (b->tri_kind == 2)
        return blaunch(b, vv::k_b_tridiag<T, false>, vv::F_MODES, vv::TRI_THREADS, b->smem_tri_plain, tab, L, b->n);
    return blaunch(b, vv::k_b_tridiag<T, true>, vv::F_MODES, vv::TRI_THREADS, b->smem_tri_stage, tab, L, b->n);
}

// P^-1 of every instance in list l: input FP64 tmp (right-hand side) or the
// GMRES-precision scratch; output b, V0 or V[it+1]
template <typename T>
int b_pc(vv_batch* b, int l, bool from_tmp64, int dst) {
    const vv::BInst* tab = b->tab;
    const int* L = blist(b, l);
    if (b->pcj) {
        const dim3 ft(vv::FJ_THREADS);
        if (from_tmp64) TRY(blaunch(b, vv::k_b_rfftj<double, T>, vv::F_ROWS, ft, b->smem_fftj, tab, L, b->n, 1));
        else TRY(blaunch(b, vv::k_b_rfftj<T, T>, vv::F_ROWS, ft, b->smem_fftj, tab, L, b->n, 0));
        TRY(b_tri<T>(b, L));
        return blaunch(b, vv::k_b_irfftj<T, T>, vv::F_ROWS, ft, b->smem_fftj, tab, L, b->n, dst);
    }
    const dim3 rt(32 * b->R);
    if (b->fft4) {
        if (from_tmp64) TRY(blaunch(b, vv::k_b_rfft<double, T, true>, vv::F_ROWS, rt, b->smem_rfft, tab, L, b->n, 1));
        else TRY(blaunch(b, vv::k_b_rfft<T, T, true>, vv::F_ROWS, rt, b->smem_rfft, tab, L, b->n, 0));
    } else {
        if (from_tmp64) TRY(blaunch(b, vv::k_b_rfft<double, T, false>, vv::F_ROWS, rt, b->smem_rfft, tab, L, b->n, 1));
        else TRY(blaunch(b, vv::k_b_rfft<T, T, false>, vv::F_ROWS, rt, b->smem_rfft, tab, L, b->n, 0));
    }
    TRY(b_tri<T>(b, L));
    if (b->fft4) return blaunch(b, vv::k_b_irfft<T, T, true>, vv::F_ROWS, rt, b->smem_irfft, tab, L, b->n, dst);
    return blaunch(b, vv::k_b_irfft<T, T, false>, vv::F_ROWS, rt, b->smem_irfft, tab, L, b->n, dst);
}

// the Jacobian stencil of every instance in list L (tiles or marching strips)
template <int S, int SRC, typename T>
int b_jvp(vv_batch* b, const int* L) {
    if (b->march)
        return blaunch(b, vv::k_b_bracket_march<S, SRC, T>, vv::F_MARCH, vv::MARCH_BW,
                       vv::MarchRow<T, vv::MARCH_BW>::smem_bytes(), (const vv::BInst*)b->tab, L, b->n);
    return blaunch(b, vv::k_b_bracket<S, SRC, T>, vv::F_TILE, vv::WTHREADS, 0, (const vv::BInst*)b->tab, L, b->n);
}

// P^-1 J x (SRC BS_X, into V0) or P^-1 J v_it (BS_VIT, into V[it+1]) of the
// instances of list l: the stencil fused into the x-FFT when the v-major
// layout runs with `fuse`, else the stencil kernel then P^-1
template <int S, int SRC, typename T>
int b_jvp_pc(vv_batch* b, int l, int dst) {
    const int* L = blist(b, l);
    if (b->pcj && b->fuse) {
        const vv::BInst* tab = b->tab;
        const dim3 ft(vv::FJ_THREADS);
        TRY(blaunch(b, vv::k_b_jvp_rfftj<S, SRC, T>, vv::F_ROWS, ft, b->smem_fjv, tab, L, b->n));
        TRY(b_tri<T>(b, L));
        return blaunch(b, vv::k_b_irfftj<T, T>, vv::F_ROWS, ft, b->smem_fftj, tab, L, b->n, dst);
    }
    TRY(b_jvp<S, SRC, T>(b, L));
    return b_pc<T>(b, l, false, dst);
}

template <typename T>
int b_jvp_all(vv_batch* b) {
    const int* L = blist(b, vv::L_ALL);
    switch (b->scheme) {
        case VV_BRACKET_J1: return b_jvp<1, vv::BS_X, T>(b, L);
        case VV_BRACKET_J2: return b_jvp<2, vv::BS_X, T>(b, L);
        default: return b_jvp<4, vv::BS_X, T>(b, L);
    }
}

template <int S, typename T>
int b_residual(vv_batch* b, int l, int phase) {
    const vv::BInst* tab = b->tab;
    const int* L = blist(b, l);
    TRY(blaunch(b, vv::k_b_poisson, vv::F_INST, 1024, 0, tab, L, b->n));
    TRY(blaunch(b, vv::k_b_bracket<S, vv::BS_RESIDUAL, T>, vv::F_TILE, vv::WTHREADS, 0, tab, L, b->n));
    TRY(blaunch(b, vv::k_b_pic_residual, vv::F_INST, 32, 0, tab, L, b->n, phase));
    return b_ctrl(b, vv::BC_PIC, BH_PIC);
}

template <int S, typename T>
int b_prologue(vv_batch* b) {
    TRY(blaunch(b, vv::k_b_prologue, vv::F_VEC, vv::RED_THREADS, 0, (const vv::BInst*)b->tab, blist(b, vv::L_ALL), b->n));
    return b_residual<S, T>(b, vv::L_ALL, 0);
}

template <int S, typename T>
int b_pic_head(vv_batch* b) {
    TRY(b_pc<T>(b, vv::L_PIC, true, vv::BD_B));
    TRY(blaunch(b, vv::k_b_gm_init<T>, vv::F_VEC, vv::RED_THREADS, 0, (const vv::BInst*)b->tab, blist(b, vv::L_PIC), b->n));
    return b_ctrl(b, vv::BC_GM_START, BH_OUTER);
}

template <int S, typename T>
int b_cycle_head(vv_batch* b) {
    const vv::BInst* tab = b->tab;
    const int* G = blist(b, vv::L_GM);
    TRY(b_jvp_pc<S, vv::BS_X, T>(b, vv::L_GMR, vv::BD_V0));
    TRY(blaunch(b, vv::k_b_gm_head<T>, vv::F_VEC, vv::RED_THREADS, 0, tab, G, b->n));
    TRY(blaunch(b, vv::k_b_gm_cycle_p<T>, vv::F_VEC, vv::RED_THREADS, 0, tab, G, b->n));
    TRY(blaunch(b, vv::k_b_gm_cycle_f, vv::F_INST, vv::CTRL_THREADS, 0, tab, G, b->n));
    return b_ctrl(b, vv::BC_INNER, BH_INNER);
}

template <int S, typename T>
int b_arnoldi(vv_batch* b) {
    const vv::BInst* tab = b->tab;
    const int* A = blist(b, vv::L_INNER);
    TRY(b_jvp_pc<S, vv::BS_VIT, T>(b, vv::L_INNER, vv::BD_VNEXT));
    TRY(blaunch(b, vv::k_b_gm_mdot_p<T>, vv::F_VEC, vv::RED_THREADS, vv::mdot_smem<T>(), tab, A, b->n));
    TRY(blaunch(b, vv::k_b_gm_mdot_f, vv::F_INST, vv::CTRL_THREADS, 0, tab, A, b->n));
    TRY(blaunch(b, vv::k_b_gm_maxpy_p<T>, vv::F_VEC, vv::RED_THREADS, 0, tab, A, b->n));
    // ||w||, Arnoldi bookkeeping and the BC_INNER control step in one launch
    return blaunch(b, vv::k_b_arnoldi_ctrl, vv::F_INST, vv::CTRL_THREADS, 0, tab, A, b->n,
                   (b->use_graph ? b->hnd[BH_INNER] : 0ull), b->flag, b->counts, b->lists, b->counts + vv::BN_DONE,
                   b->counts + vv::BN_DROPPED);
}

template <int S, typename T>
int b_cycle_tail(vv_batch* b) {
    const int* G = blist(b, vv::L_GM);
    TRY(blaunch(b, vv::k_b_gm_solve, vv::F_INST, 32, 0, (const vv::BInst*)b->tab, G, b->n));
    TRY(blaunch(b, vv::k_b_gm_update<T>, vv::F_VEC, vv::RED_THREADS, 0, (const vv::BInst*)b->tab, G, b->n));
    return b_ctrl(b, vv::BC_GM_FINISH, BH_OUTER);
}

int b_moments(vv_batch* b, int l) {
    const int* L = blist(b, l);
    TRY(blaunch(b, vv::k_b_moments_partial, vv::F_MOM, dim3(vv::MOM_TX, vv::MOM_TY), 0, (const vv::BInst*)b->tab, L, b->n));
    return blaunch(b, vv::k_b_moments_poisson, vv::F_INST, vv::POIS_THREADS, b->smem_pois, (const vv::BInst*)b->tab, L,
                   b->n);
}

template <int S, typename T>
int b_pic_tail(vv_batch* b) {
    TRY(blaunch(b, vv::k_b_pic_apply<T>, vv::F_VEC, vv::RED_THREADS, 0, (const vv::BInst*)b->tab, blist(b, vv::L_PIC), b->n));
    TRY(b_moments(b, vv::L_PIC));
    return b_residual<S, T>(b, vv::L_PIC, 1);
}

int b_revert_ctrl(vv_batch* b) { return b_ctrl(b, vv::BC_REVERT, BH_REVERT); }

int b_revert(vv_batch* b) {
    TRY(blaunch(b, vv::k_b_revert, vv::F_VEC, vv::RED_THREADS, 0, (const vv::BInst*)b->tab, blist(b, vv::L_REVERT), b->n));
    return b_moments(b, vv::L_REVERT);
}

// host-driven step (the same kernels; the host reads each loop flag)
template <int S, typename T>
int b_step_host(vv_batch* b) {
    int f = 0;
    TRY(b_prologue<S, T>(b));
    TRY(b_flag(b, &f));
    while (f) {
        TRY(b_pic_head<S, T>(b));
        int outer = 0;
        TRY(b_flag(b, &outer));
        while (outer) {
            TRY(b_cycle_head<S, T>(b));
            int inner = 0;
            TRY(b_flag(b, &inner));
            while (inner) {
                TRY(b_arnoldi<S, T>(b));
                TRY(b_flag(b, &inner));
            }
            TRY(b_cycle_tail<S, T>(b));
            TRY(b_flag(b, &outer));
        }
        TRY(b_pic_tail<S, T>(b));
        TRY(b_flag(b, &f));
    }
    TRY(b_revert_ctrl(b));
    TRY(b_flag(b, &f));
    if (f) TRY(b_revert(b));
    return VV_OK;
}

// body capture on a batch capture stream
template <typename F>
int b_body(vv_batch* b, int level, cudaGraph_t body, F fn) {
    const cudaStream_t saved = b->st;
    CK(cudaStreamBeginCaptureToGraph(b->cs[level], body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    b->st = b->cs[level];
    const int r = fn();
    b->st = saved;
    cudaGraph_t out = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cs[level], &out);
    if (r != VV_OK) return r;
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture (batch)");
    return VV_OK;
}

// Arnoldi steps per iteration of the batch graph's inner loop (VV_BATCH_UNROLL=1..4 overrides)
constexpr int INNER_UNROLL = 2;
int inner_unroll() {
    const char* e = getenv("VV_BATCH_UNROLL");
    const int u = e ? atoi(e) : INNER_UNROLL;
    return (u >= 1 && u <= 4) ? u : INNER_UNROLL;
}

template <int S, typename T>
int b_capture(vv_batch* b) {
    // the loop handles exist before the control kernels that set them are captured
    for (auto& h : b->hnd) {
        cudaGraphConditionalHandle ch;
        CK(cudaGraphConditionalHandleCreate(&ch, b->g, 0, cudaGraphCondAssignDefault));
        h = (unsigned long long)ch;
    }
    // kernels per sequence (for the launch count of graph steps)
    const int64_t l0 = b->launches;
    TRY(b_prologue<S, T>(b));
    b->nk_prologue = (int)(b->launches - l0);
    cudaGraph_t pic[1];
    TRY(add_conditional(b->g, b->st, cudaGraphCondTypeWhile, 1, 0, &b->hnd[BH_PIC], pic));
    TRY(b_body(b, 1, pic[0], [&]() -> int {
        int64_t m = b->launches;
        TRY(b_pic_head<S, T>(b));
        b->nk_pic_head = (int)(b->launches - m);
        cudaGraph_t outer[1];
        TRY(add_conditional(b->g, b->st, cudaGraphCondTypeWhile, 1, 0, &b->hnd[BH_OUTER], outer));
        TRY(b_body(b, 2, outer[0], [&]() -> int {
            int64_t q = b->launches;
            TRY(b_cycle_head<S, T>(b));
            b->nk_cycle_head = (int)(b->launches - q);
            cudaGraph_t inner[1];
            TRY(add_conditional(b->g, b->st, cudaGraphCondTypeWhile, 1, 0, &b->hnd[BH_INNER], inner));
            // INNER_UNROLL Arnoldi steps per iteration of the conditional loop
            // (each iteration costs about five kernel launches of its own); a
            // step after the one that emptied the inner list finds it empty and
            // does nothing (every kernel walks an empty list)
            TRY(b_body(b, 3, inner[0], [&]() -> int {
                const int64_t w = b->launches;
                const int unroll = inner_unroll();
                for (int u = 0; u < unroll; ++u) TRY(b_arnoldi<S, T>(b));
                b->nk_arnoldi = (int)(b->launches - w) / unroll;
                return VV_OK;
            }));
            q = b->launches;
            TRY(b_cycle_tail<S, T>(b));
            b->nk_cycle_tail = (int)(b->launches - q);
            return VV_OK;
        }));
        m = b->launches;
        TRY(b_pic_tail<S, T>(b));
        b->nk_pic_tail = (int)(b->launches - m);
        return VV_OK;
    }));
    int64_t m = b->launches;
    TRY(b_revert_ctrl(b));
    b->nk_revert_ctrl = (int)(b->launches - m);
    cudaGraph_t rev[1];
    TRY(add_conditional(b->g, b->st, cudaGraphCondTypeIf, 1, 0, &b->hnd[BH_REVERT], rev));
    TRY(b_body(b, 1, rev[0], [&]() -> int {
        const int64_t w = b->launches;
        TRY(b_revert(b));
        b->nk_revert = (int)(b->launches - w);
        return VV_OK;
    }));
    b->launches = l0;   // captured, not executed
    return VV_OK;
}

template <typename T>
int b_dispatch_capture(vv_batch* b) {
    switch (b->scheme) {
        case VV_BRACKET_J1: return b_capture<1, T>(b);
        case VV_BRACKET_J2: return b_capture<2, T>(b);
        default: return b_capture<4, T>(b);
    }
}

template <typename T>
int b_dispatch_host(vv_batch* b) {
    switch (b->scheme) {
        case VV_BRACKET_J1: return b_step_host<1, T>(b);
        case VV_BRACKET_J2: return b_step_host<2, T>(b);
        default: return b_step_host<4, T>(b);
    }
}

// Launch shape of the preconditioner kernels: rows per CTA of the x-FFTs,
// the tridiagonal variant and the FFT kind (work items per instance and
// shared memory).
void b_shape(vv_batch* b, std::vector<vv::BInst>& tab, int R, int tri_kind, int fft4, int pcj = 0) {
    b->R = R;
    b->tri_kind = tri_kind;
    b->fft4 = fft4;
    b->pcj = pcj && b->pcj_ok;
    const bool tri_warp = tri_kind == 1;
    const size_t csz = b->mixed ? sizeof(float2) : sizeof(double2);
    for (int f = 0; f < vv::NFAM; ++f) b->tot[f] = 0;
    b->smem_rfft = b->smem_irfft = 0;
    for (int i = 0; i < b->n; ++i) {
        vv::BInst& I = tab[i];
        const vv_ctx* c = b->ctx[i];
        I.pp.R = R;
        I.cnt[vv::F_ROWS] = (c->nv + R - 1) / R;
        I.cnt[vv::F_MODES] = tri_warp ? (c->nmodes + vv::TRIW_WARPS - 1) / vv::TRIW_WARPS : c->nmodes;
        if (b->pcj) {
            const int rb = vv::fj_rows_of(c->M);
            I.cnt[vv::F_ROWS] = (c->nv + rb - 1) / rb;
            const int items = (c->nmodes + vv::TRIW_WARPS - 1) / vv::TRIW_WARPS;
            const int tch = vv::tjr_ch(b->mixed ? 4 : 8);
            I.cnt[vv::F_MODES] = tri_kind == 6   ? (c->nmodes + vv::tjr_modes(c->nv, tch) - 1) / vv::tjr_modes(c->nv, tch)
                                 : tri_kind == 5 ? (c->nmodes + vv::TJC_MG - 1) / vv::TJC_MG
                                 : tri_kind == 4 ? (items + vv::tjv_group(c->nv) - 1) / vv::tjv_group(c->nv)
                                 : tri_kind >= 1 ? items
                                                 : (c->nmodes + 31) / 32;
        }
        for (int f = 0; f < vv::NFAM; ++f) b->tot[f] += I.cnt[f];
        b->smem_rfft = std::max(b->smem_rfft, fft_smem(0, c->M, R, csz, false));
        b->smem_irfft = std::max(b->smem_irfft, fft_smem(0, c->M, R, csz, true));
        if (fft4 && c->M >= 32 && c->M <= 128) {   // the lengths k_b_rfft/k_b_irfft run four-step
            b->smem_rfft = std::max(b->smem_rfft, fft_smem(1, c->M, R, csz, false));
            b->smem_irfft = std::max(b->smem_irfft, fft_smem(1, c->M, R, csz, true));
        }
    }
}

// upload the table in its current shape and rebuild the list of all instances
int b_apply_shape(vv_batch* b, const std::vector<vv::BInst>& tab) {
    CK(cudaMemcpyAsync(b->tab, tab.data(), tab.size() * sizeof(vv::BInst), cudaMemcpyHostToDevice, b->st));
    TRY(b_ctrl(b, vv::BC_ALL, -1));
    CK(cudaStreamSynchronize(b->st));
    return VV_OK;
}

// whether tridiagonal variant tw (layout pj) fits the device's shared memory
bool b_tri_fits(const vv_batch* b, int tw, int pj) {
    size_t need = 0;
    if (pj && tw == 6) return b->nvmax <= vv::tjr_nvmax(b->mixed ? 4 : 8);   // chunks held in registers
    if (pj)
        need = tw == 1 ? b->smem_tri_js : tw == 2 ? b->smem_tri_jm2 : tw == 3 ? b->smem_tri_jm4 : tw == 4 ? b->smem_tri_jv : 0;
    else if (tw == 1) need = b->smem_tri_warp;
    return need <= (size_t)b->smem_limit;
}

// whether the fused stencil + x-FFT kernel fits the device's shared memory
bool b_fuse_fits(const vv_batch* b) { return b->pcj_ok && b->smem_fjv <= (size_t)b->smem_limit; }

// Batch autotuner: times the whole-table preconditioner (the step's largest
// share) for FFT kind x FFT rows per CTA x tridiagonal variant and keeps the
// fastest.
template <typename T>
int b_autotune(vv_batch* b, std::vector<vv::BInst>& tab) {
    for (int i = 0; i < b->n; ++i) {
        const vv_ctx* c = b->ctx[i];
        CK(cudaMemsetAsync(b->mixed ? (void*)c->tmp32 : (void*)c->tmp, 0, c->ncell * sizeof(T), b->st));
    }
    // the lockstep tail: a few of the slowest instances run alone for most of
    // a step's GMRES iterations; the largest NTAIL instances stand in for it
    constexpr int NTAIL = 4;
    std::vector<int> member(b->n, 0), order(b->n);
    for (int i = 0; i < b->n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->ctx[a]->ncell > b->ctx[c]->ncell; });
    for (int i = 0; i < std::min(NTAIL, b->n); ++i) member[order[i]] = 1;
    int* dmember = nullptr;
    CK(cudaMalloc((void**)&dmember, b->n * sizeof(int)));
    if (cudaMemcpy(dmember, member.data(), b->n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(dmember);
        return fail_cuda(cudaGetLastError(), "batch autotune");
    }
    auto tail_list = [&]() -> int {
        vv::k_b_build_subset<<<1, vv::CTRL_THREADS, 0, b->st>>>(b->tab, b->n, b->lists, vv::L_TAIL, dmember);
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? VV_OK : fail_cuda(e, "batch autotune list");
    };
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // mean time of `reps` calls of fn after two untimed ones (1e30 on failure)
    auto timed = [&](auto fn, int reps, int& r) -> float {
        for (int k = 0; k < 2 && r == VV_OK; ++k) r = fn();
        cudaEventRecord(e0, b->st);
        for (int k = 0; k < reps && r == VV_OK; ++k) r = fn();
        cudaEventRecord(e1, b->st);
        float ms = 0.f;
        if (r != VV_OK || cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            return 1e30f;
        return ms / reps;
    };
    // weights of the lockstep profile of a step of the 256-instance sweep:
    // about 30 whole-table-equivalent GMRES iterations and 100 iterations in
    // which only the slowest instances are left
    constexpr float W_FULL = 30.f, W_TAIL = 100.f;
    float best = 1e30f;
    int bR = b->R, bW = b->tri_kind, bF = b->fft4, bJ = b->pcj, r = VV_OK;
    for (int pj = 0; pj <= (b->pcj_ok ? 1 : 0) && r == VV_OK; ++pj)
    for (int f4 = 0; f4 <= (pj ? 0 : 1) && r == VV_OK; ++f4)
    for (int tw = 0; tw <= (pj ? 6 : 2) && r == VV_OK; ++tw) {
        if (!b_tri_fits(b, tw, pj)) continue;
        for (int R = 2; R <= (pj ? 2 : 8) && r == VV_OK; R *= 2) {
            b_shape(b, tab, R, tw, f4, pj);
            if ((r = b_apply_shape(b, tab)) != VV_OK) break;
            if ((r = tail_list()) != VV_OK) break;
            const float tf = timed([&]() { return b_pc<T>(b, vv::L_ALL, false, vv::BD_B); }, 5, r);
            const float tt = timed([&]() { return b_pc<T>(b, vv::L_TAIL, false, vv::BD_B); }, 5, r);
            const float score = W_FULL * tf + W_TAIL * tt;
            if (getenv("VV_DEBUG"))
                fprintf(stderr, "[vv_batch] tune pcj=%d fft4=%d R=%d tri=%d: full %.1f us, tail %.1f us\n", pj, f4, R,
                        tw, tf * 1e3f, tt * 1e3f);
            if (r == VV_OK && score < best) {
                best = score;
                bR = R;
                bW = tw;
                bF = f4;
                bJ = pj;
            }
        }
    }
    if (r == VV_OK) {
        b_shape(b, tab, bR, bW, bF, bJ);
        r = b_apply_shape(b, tab);
    }
    if (r == VV_OK) r = tail_list();
    // Jacobian stencil: 64 x 32 tiles or marching strips before P^-1, or (v-major
    // layout) the stencil fused into the x-FFT; timed as the whole GMRES
    // operator P^-1 J on the table and on the tail, by the same weights
    float bestj = 1e30f;
    int bM = 0, bFu = 0;
    auto op = [&](int l) -> int {
        switch (b->scheme) {
            case VV_BRACKET_J1: return b_jvp_pc<1, vv::BS_X, T>(b, l, vv::BD_B);
            case VV_BRACKET_J2: return b_jvp_pc<2, vv::BS_X, T>(b, l, vv::BD_B);
            default: return b_jvp_pc<4, vv::BS_X, T>(b, l, vv::BD_B);
        }
    };
    for (int fu = 0; fu <= (b->pcj && b_fuse_fits(b) ? 1 : 0) && r == VV_OK; ++fu)
        for (int m = 0; m <= (fu ? 0 : 1) && r == VV_OK; ++m) {
            b->march = m;
            b->fuse = fu;
            const float tf = timed([&]() { return op(vv::L_ALL); }, 5, r);
            const float tt = timed([&]() { return op(vv::L_TAIL); }, 5, r);
            const float score = W_FULL * tf + W_TAIL * tt;
            if (getenv("VV_DEBUG"))
                fprintf(stderr, "[vv_batch] tune fuse=%d march=%d: full %.1f us, tail %.1f us\n", fu, m, tf * 1e3f,
                        tt * 1e3f);
            if (score < bestj) {
                bestj = score;
                bM = m;
                bFu = fu;
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dmember);
    TRY(r);
    b->march = bM;
    b->fuse = bFu;
    return VV_OK;
}

template <typename X>
int upload_vec(X** dst, const std::vector<X>& v) {
    if (cudaMalloc((void**)dst, std::max<size_t>(1, v.size()) * sizeof(X)) != cudaSuccess) return VV_ERR_ALLOC;
    if (!v.empty() && cudaMemcpy(*dst, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail_cuda(cudaGetLastError(), "batch table upload");
    return VV_OK;
}

}  // namespace

extern "C" {

int vv_batch_destroy(vv_batch* b) {
    if (!b) return VV_OK;
    if (b->pending && b->user) cudaStreamSynchronize(b->user);   // a launch never collected: let it finish
    for (auto s : b->cs) {
        cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
        if (s && cudaStreamIsCapturing(s, &cst) == cudaSuccess && cst != cudaStreamCaptureStatusNone) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(s, &junk);
            if (junk) cudaGraphDestroy(junk);
        }
    }
    cudaGetLastError();
    for (auto s : b->cs) if (s) cudaStreamDestroy(s);
    if (b->ex) cudaGraphExecDestroy(b->ex);
    if (b->g) cudaGraphDestroy(b->g);
    for (void* p : {(void*)b->tab, (void*)b->lists, (void*)b->counts, (void*)b->flag, (void*)b->gather, (void*)b->wpart,
                    b->dinvJ, b->jtab})
        if (p) cudaFree(p);
    if (b->hflag) cudaFreeHost(b->hflag);
    if (b->hcounts) cudaFreeHost(b->hcounts);
    if (b->hgather) cudaFreeHost(b->hgather);
    delete b;
    return VV_OK;
}

int vv_batch_create(int n, vv_ctx* const* ctxs, const vv_state* states, vv_batch** out) {
    if (n < 1 || !ctxs || !states || !out) return VV_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        const vv_state& s = states[i];
        if (!ctxs[i] || !s.f || !s.fh || !s.phi || !s.h1c || !s.h1h || !s.n) return VV_ERR_ARG;
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) return VV_ERR_ARG;   // one context per instance
    }
    const vv_ctx* c0 = ctxs[0];
    for (int i = 0; i < n; ++i) {
        const vv_ctx* c = ctxs[i];
        // one scheme, precision and preconditioner for the table; the wide
        // 64 x 32 stencil tiles (nx a multiple of 64); the factored order;
        // the point time derivative
        if (c->mixed != c0->mixed || c->g.bracket != c0->g.bracket ||
            c->g.preconditioner != VV_PC_TENSOR_KINETIC || c->g.order == VV_ORDER_REFERENCE ||
            c->g.bracket == VV_BRACKET_SIMPSON || c->avg != vv::AVG_POINT || c->coll != vv::COLL_NONE || c->db ||
            c->pred || c->nx % vv::WX != 0 || !c->pow2 || c->device != c0->device)
            return VV_ERR_UNSUPPORTED;
    }
    vv_batch* b = new vv_batch();   // value-initialised: pointers and counts start at zero
    b->n = n;
    b->ctx.assign(ctxs, ctxs + n);
    b->states.assign(states, states + n);
    b->mixed = c0->mixed;
    b->scheme = c0->g.bracket;
    b->R = 4;
    b->use_graph = c0->use_graph;
    auto fail_b = [&](int code) { vv_batch_destroy(b); return code; };
    if (cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, c0->device) != cudaSuccess)
        return fail_b(fail_cuda(cudaGetLastError(), "multiprocessor count"));
    std::vector<vv::BInst> tab(n);
    for (int i = 0; i < n; ++i) {
        vv_ctx* c = ctxs[i];
        const vv_state& s = states[i];
        vv::BInst& I = tab[i];
        std::memset(&I, 0, sizeof I);
        I.ds = c->ds;
        I.nx = c->nx;
        I.nv = c->nv;
        I.ncell = c->ncell;
        I.tiles_x = c->nx / vv::WX;
        // vector kernels: 2048 cells per block item (eight warp items of 256)
        I.vblk = (int)std::max<size_t>(1, std::min<size_t>((c->ncell + 2047) / 2048, (size_t)c->npart_max));
        I.mom_seg = c->mom_seg;
        I.mom_bx = (c->nx + vv::MOM_TX - 1) / vv::MOM_TX;
        I.mom_S = c->mom_S;
        I.cnt[vv::F_TILE] = I.tiles_x * ((c->nv + vv::WY - 1) / vv::WY);
        I.cnt[vv::F_MARCH] = (c->nx / vv::MARCH_BW) * ((c->nv + vv::MARCH_SEG - 1) / vv::MARCH_SEG);
        I.cnt[vv::F_VEC] = I.vblk;
        I.cnt[vv::F_MOM] = I.mom_bx * c->mom_S;
        I.cnt[vv::F_INST] = 1;
        I.bp = bparams(c, 0.5);
        I.pp = pcparams(c);
        I.pp.R = b->R;
        I.pp.tw = b->mixed ? (const void*)c->tw32 : (const void*)c->tw;
        I.tp.nv = c->nv;
        I.tp.nmodes = c->nmodes;
        I.tp.lambda = b->mixed ? (const void*)c->lambda32 : (const void*)c->lambda;
        I.tp.alpha = b->mixed ? (const void*)c->alpha32 : (const void*)c->alpha;
        I.tp.gamma = b->mixed ? (const void*)c->gamma32 : (const void*)c->gamma;
        I.tp.dinv = b->mixed ? (const void*)c->dinv32 : (const void*)c->dinv;
        I.po = pparams(c);
        I.f = s.f; I.fh = s.fh; I.phi = s.phi; I.phih = s.phih;
        I.h1c = s.h1c; I.h1h = s.h1h; I.h2c = s.h2c; I.h2h = s.h2h;
        I.n = s.n; I.u = s.u; I.e = s.e; I.a = s.a;
        I.Fh = c->Fh; I.tmp = c->tmp; I.fl = c->fl; I.part = c->part; I.mom_part = c->mom_part;
        I.hxp = c->hxp; I.v = c->v; I.scal = c->scal;
        if (b->mixed) {
            I.V = c->V32; I.tmpT = c->tmp32; I.bT = c->bvec32; I.xT = c->delta32; I.specT = c->spec32;
        } else {
            I.V = c->V; I.tmpT = c->tmp; I.bT = c->bvec; I.xT = c->delta; I.specT = c->spec;
        }
        {
            const int ch = (c->nv + vv::TRI_THREADS - 1) / vv::TRI_THREADS;
            const size_t np = (size_t)c->nv + (c->nv + ch - 1) / ch;
            b->smem_tri_stage = std::max(b->smem_tri_stage, np * (b->mixed ? 24 : 48));
            b->smem_tri_plain = std::max(b->smem_tri_plain, np * (b->mixed ? sizeof(float2) : sizeof(double2)));
            b->smem_tri_warp = std::max(b->smem_tri_warp, tri_ws_smem(c->nv, b->mixed ? sizeof(float2) : sizeof(double2)));
            b->nvmax = std::max(b->nvmax, c->nv);
            b->smem_tri_js = vv::tri_js_smem(b->nvmax, b->mixed ? sizeof(float2) : sizeof(double2));
            b->smem_tri_jm2 = vv::tri_jm_smem(b->nvmax, b->mixed ? sizeof(float2) : sizeof(double2), 2);
            b->smem_tri_jm4 = vv::tri_jm_smem(b->nvmax, b->mixed ? sizeof(float2) : sizeof(double2), 4);
            b->smem_tri_jv = std::max(b->smem_tri_jv, vv::tjv_smem_of(c->nv, b->mixed ? sizeof(float2) : sizeof(double2)));
        }
        b->smem_pois = std::max(b->smem_pois, c->smem_pois);
    }
    b_shape(b, tab, 8, 0, 1);   // the largest shared-memory shape, for the limit check
    {
        int limit = 0;
        int r = raise_smem_limits(&limit);
        if (r != VV_OK) return fail_b(r);
        b->smem_limit = limit;
        if (std::max({b->smem_rfft, b->smem_irfft, b->smem_tri_stage, b->smem_pois}) > (size_t)limit)
            return fail_b(VV_ERR_UNSUPPORTED);
    }
    // the v-major preconditioner layout: lengths, shared memory and the v-major LU tables
    {
        const size_t csz = b->mixed ? sizeof(float2) : sizeof(double2);
        b->pcj_ok = true;
        size_t words = 0;
        for (int i = 0; i < n; ++i) {
            const int slots = vv::fj_slots_of(ctxs[i]->M);
            if (slots < 0) b->pcj_ok = false;
            else {
                b->smem_fftj = std::max(b->smem_fftj, (size_t)slots * csz);
                b->smem_fjv = std::max(b->smem_fjv, vv::fjv_smem_of(ctxs[i]->M, csz / 2));
            }
            words += (size_t)ctxs[i]->nmodes * ctxs[i]->nv;
        }
        if (b->smem_fftj > (size_t)b->smem_limit) b->pcj_ok = false;
        if (b->pcj_ok) {
            if (cudaMalloc(&b->dinvJ, words * csz) != cudaSuccess) return fail_b(VV_ERR_ALLOC);
            size_t off = 0;
            for (int i = 0; i < n; ++i) {
                const vv_ctx* c = ctxs[i];
                const size_t cnt = (size_t)c->nmodes * c->nv;
                const unsigned g = (unsigned)((cnt + 255) / 256);
                char* dst = (char*)b->dinvJ + off * csz;
                if (b->mixed) vv::k_modes_to_vmajor<float2><<<g, 256>>>(c->dinv32, (float2*)dst, c->nmodes, c->nv);
                else vv::k_modes_to_vmajor<double2><<<g, 256>>>(c->dinv, (double2*)dst, c->nmodes, c->nv);
                tab[i].dinvJ = dst;
                off += cnt;
            }
            const cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return fail_b(fail_cuda(e, "v-major LU tables"));
            // the fused stencil's coefficient tables: (nx + nv) x 3 of the GMRES precision per
            // instance, 16-byte aligned; filled by k_b_jcoef once the table is on the device
            const size_t tsz = csz / 2;
            std::vector<size_t> jo(n);
            size_t jbytes = 0;
            for (int i = 0; i < n; ++i) {
                jo[i] = jbytes;
                jbytes += (3 * (size_t)(ctxs[i]->nx + ctxs[i]->nv) * tsz + 15) & ~(size_t)15;
            }
            if (cudaMalloc(&b->jtab, jbytes) != cudaSuccess) return fail_b(VV_ERR_ALLOC);
            const int js = b->scheme == VV_BRACKET_J1 ? 1 : b->scheme == VV_BRACKET_J2 ? 2 : 4;
            for (int i = 0; i < n; ++i) {
                char* base = (char*)b->jtab + jo[i];
                tab[i].jcol = base;
                tab[i].jrow = base + 3 * (size_t)ctxs[i]->nx * tsz;
                tab[i].jfp32 = b->mixed ? 1 : 0;
                tab[i].jscheme = js;
            }
        }
    }
    // per-warp partials: (restart + 2) columns of 8 vblk per instance
    {
        size_t words = 0;
        std::vector<size_t> off(n);
        for (int i = 0; i < n; ++i) {
            off[i] = words;
            words += (size_t)(ctxs[i]->restart + 2) * 8 * tab[i].vblk;
        }
        if (cudaMalloc((void**)&b->wpart, words * sizeof(double)) != cudaSuccess) return fail_b(VV_ERR_ALLOC);
        for (int i = 0; i < n; ++i) tab[i].wpart = b->wpart + off[i];
    }
    int r = VV_OK;
    if ((r = upload_vec(&b->tab, tab))) return fail_b(r);
    b->list_words = vv::blist_words(n);
    b->words = (int)(offsetof(vv::DevState, hcol) / sizeof(unsigned int));
    if (cudaMalloc((void**)&b->lists, (size_t)vv::NLIST * b->list_words * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&b->counts, vv::BN_WORDS * sizeof(unsigned int)) != cudaSuccess ||
        cudaMalloc((void**)&b->flag, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&b->gather, (size_t)n * b->words * sizeof(unsigned int)) != cudaSuccess)
        return fail_b(VV_ERR_ALLOC);
    if (cudaMallocHost((void**)&b->hflag, sizeof(int)) != cudaSuccess ||
        cudaMallocHost((void**)&b->hcounts, vv::BN_WORDS * sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost((void**)&b->hgather, (size_t)n * b->words * sizeof(unsigned int)) != cudaSuccess)
        return fail_b(VV_ERR_ALLOC);
    for (auto& s : b->cs)
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return fail_b(VV_ERR_CUDA);
    b->user = 0;
    b->st = b->cs[0];
    // empty lists, then the list of every instance
    if (cudaMemsetAsync(b->lists, 0, (size_t)vv::NLIST * b->list_words * sizeof(int), b->st) != cudaSuccess)
        return fail_b(fail_cuda(cudaGetLastError(), "batch lists"));
    if (b->jtab) {
        vv::k_b_jcoef<<<n, 1024, 0, b->st>>>(b->tab, n);
        if (cudaGetLastError() != cudaSuccess) return fail_b(VV_ERR_CUDA);
    }
    b_shape(b, tab, 4, 0, 0);
    if ((r = b_apply_shape(b, tab)) != VV_OK) return fail_b(r);
    {
        // VV_BATCH_SHAPE="R,tri,fft4[,vmajor[,march[,fuse]]]" fixes the shape (tests, profiling; fuse
        // defaults to 1 with the v-major layout); else the autotuner picks it
        const char* bs = getenv("VV_BATCH_SHAPE");
        int fR = 0, fT = 0, fF = 0, fJ = 0, fM = 0, fU = 1;
        const int nf = bs ? sscanf(bs, "%d,%d,%d,%d,%d,%d", &fR, &fT, &fF, &fJ, &fM, &fU) : 0;
        const bool fixed = nf >= 3 && (fR == 2 || fR == 4 || fR == 8) && fT >= 0 && fT <= (fJ ? 6 : 2) &&
                           (fF == 0 || fF == 1) && (fJ == 0 || (fJ == 1 && b->pcj_ok)) && b_tri_fits(b, fT, fJ);
        const char* at = getenv("VV_AUTOTUNE");
        if (fixed) {
            b->march = fM != 0;
            b_shape(b, tab, fR, fT, fF, fJ);
            b->fuse = (fU != 0 && b->pcj && b_fuse_fits(b)) ? 1 : 0;
            if ((r = b_apply_shape(b, tab)) != VV_OK) return fail_b(r);
        } else if (!(at && at[0] == '0')) {
            r = b->mixed ? b_autotune<float>(b, tab) : b_autotune<double>(b, tab);
            if (r != VV_OK) return fail_b(r);
        }
    }
    b->launches = 0;
    if (b->use_graph) {
        if (cudaGraphCreate(&b->g, 0) != cudaSuccess) return fail_b(VV_ERR_CUDA);
        if (cudaStreamBeginCaptureToGraph(b->cs[0], b->g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) !=
            cudaSuccess)
            return fail_b(VV_ERR_CUDA);
        r = b->mixed ? b_dispatch_capture<float>(b) : b_dispatch_capture<double>(b);
        cudaGraph_t outg = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->cs[0], &outg);
        if (r != VV_OK) return fail_b(r);
        if (e != cudaSuccess) return fail_b(fail_cuda(e, "batch capture"));
        cudaGraphInstantiateParams ip = {};
        const cudaError_t ie = cudaGraphInstantiateWithParams(&b->ex, b->g, &ip);
        if (ie != cudaSuccess) {
            cudaGraphNodeType t = cudaGraphNodeTypeEmpty;
            if (ip.errNode_out) cudaGraphNodeGetType(ip.errNode_out, &t);
            char what[128];
            snprintf(what, sizeof what, "batch instantiate (result %d, node type %d)", (int)ip.result_out, (int)t);
            return fail_b(fail_cuda(ie, what));
        }
    }
    *out = b;
    return VV_OK;
}

int vv_batch_set_stream(vv_batch* b, void* stream) {
    if (!b) return VV_ERR_ARG;
    b->user = (cudaStream_t)stream;
    return VV_OK;
}

int vv_batch_launch(vv_batch* b, const vv_snes_opts* so, const vv_ksp_opts* ko) {
    if (!b || !so || !ko) return VV_ERR_ARG;
    if (b->pending) return fail(VV_ERR_ARG, "vv_batch_launch: the previous launch was not collected");
    for (int i = 0; i < b->n; ++i) {
        vv_ctx* c = b->ctx[i];
        const int restart = (ko->restart > 0) ? ko->restart : c->restart;
        if (restart > c->restart || restart < 1 || ko->max_it < 0 || so->max_iter < 1) return VV_ERR_ARG;
        // the instance's own graph handles stay out of the batch graph
        for (auto& h : c->hnd) h = 0;
        const cudaStream_t saved = c->st;
        c->st = b->user;
        const int r = upload_options(c, ko, so);
        c->st = saved;
        TRY(r);
    }
    b->st = b->user;
    b->pending_l0 = b->launches;
    CK(cudaMemsetAsync(b->counts, 0, vv::BN_WORDS * sizeof(unsigned int), b->user));
    if (b->use_graph) {
        CK(cudaGraphLaunch(b->ex, b->user));
    } else {
        const int r = b->mixed ? b_dispatch_host<float>(b) : b_dispatch_host<double>(b);
        b->st = b->cs[0];
        TRY(r);
    }
    b->st = b->user;
    vv::k_b_gather_states<<<b->n, 128, 0, b->user>>>(b->tab, b->words, b->gather);
    b->launches++;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(b->hgather, b->gather, (size_t)b->n * b->words * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                       b->user));
    CK(cudaMemcpyAsync(b->hcounts, b->counts, vv::BN_WORDS * sizeof(unsigned int), cudaMemcpyDeviceToHost, b->user));
    b->st = b->cs[0];
    b->pending = 1;
    return VV_OK;
}

int vv_batch_collect(vv_batch* b, const vv_snes_opts* so, const vv_ksp_opts* ko, vv_step_report* reports,
                     int* statuses) {
    if (!b || !so || !ko || !reports) return VV_ERR_ARG;
    if (!b->pending) return fail(VV_ERR_ARG, "vv_batch_collect: nothing launched");
    b->pending = 0;
    CK(cudaStreamSynchronize(b->user));
    if (b->use_graph) {
        const unsigned* k = b->hcounts;
        b->launches = b->pending_l0 + 1 + b->nk_prologue + b->nk_revert_ctrl +
                      (int64_t)k[vv::BC_PIC] * (b->nk_pic_head + b->nk_pic_tail) +
                      (int64_t)(k[vv::BC_GM_START] + k[vv::BC_GM_FINISH]) * (b->nk_cycle_head + b->nk_cycle_tail) +
                      (int64_t)(k[vv::BC_INNER] + k[vv::BN_IDLE]) * b->nk_arnoldi +
                      (int64_t)k[vv::BC_REVERT] * b->nk_revert;
    }
    int first_bad = VV_OK;
    vv::DevState d;
    for (int i = 0; i < b->n; ++i) {
        vv_ctx* c = b->ctx[i];
        std::memcpy(&d, b->hgather + (size_t)i * b->words, (size_t)b->words * sizeof(unsigned int));
        const int restart = (ko->restart > 0) ? ko->restart : c->restart;
        const int s = fill_report(c, d, restart, &reports[i], so->abort_residual, false);
        if (statuses) statuses[i] = s;
        if (s != VV_OK && first_bad == VV_OK) first_bad = s;
    }
    return first_bad;
}

int vv_batch_step(vv_batch* b, const vv_snes_opts* so, const vv_ksp_opts* ko, vv_step_report* reports,
                  int* statuses) {
    if (!b || !so || !ko || !reports) return VV_ERR_ARG;
    TRY(vv_batch_launch(b, so, ko));
    return vv_batch_collect(b, so, ko, reports, statuses);
}

int vv_batch_time_kernel(vv_batch* b, int which, int it, int reps, double* avg_ms) {
    if (!b || !avg_ms || reps < 1 || which < 0 || which > 5 || it < 0) return VV_ERR_ARG;
    for (int i = 0; i < b->n; ++i)
        if (it + 1 >= b->ctx[i]->restart + 1) return VV_ERR_ARG;   // V[it+1] must exist
    const int64_t l0 = b->launches;
    b->st = b->cs[0];
    vv::k_b_set_it<<<1, 256, 0, b->st>>>(b->tab, b->n, it);
    CK(cudaGetLastError());
    const vv::BInst* tab = b->tab;
    const int* L = blist(b, vv::L_ALL);
    auto one = [&]() -> int {
        switch (which) {
            case 0:
                return b->mixed ? blaunch(b, vv::k_b_gm_mdot_p<float>, vv::F_VEC, vv::RED_THREADS,
                                          vv::mdot_smem<float>(), tab, L, b->n)
                                : blaunch(b, vv::k_b_gm_mdot_p<double>, vv::F_VEC, vv::RED_THREADS,
                                          vv::mdot_smem<double>(), tab, L, b->n);
            case 1: return b->mixed ? b_pc<float>(b, vv::L_ALL, false, vv::BD_B) : b_pc<double>(b, vv::L_ALL, false, vv::BD_B);
            case 2: return b->mixed ? b_jvp_all<float>(b) : b_jvp_all<double>(b);   // the tuned stencil kernel
            case 4: return b->mixed ? b_tri<float>(b, L) : b_tri<double>(b, L);     // the tuned tridiagonal stage
            case 5: {   // the GMRES operator P^-1 J as the step applies it (fused or not)
                auto op = [&](auto tag) -> int {
                    using TT = decltype(tag);
                    switch (b->scheme) {
                        case VV_BRACKET_J1: return b_jvp_pc<1, vv::BS_X, TT>(b, vv::L_ALL, vv::BD_B);
                        case VV_BRACKET_J2: return b_jvp_pc<2, vv::BS_X, TT>(b, vv::L_ALL, vv::BD_B);
                        default: return b_jvp_pc<4, vv::BS_X, TT>(b, vv::L_ALL, vv::BD_B);
                    }
                };
                return b->mixed ? op(0.0f) : op(0.0);
            }
            default:
                return b->mixed ? blaunch(b, vv::k_b_gm_maxpy_p<float>, vv::F_VEC, vv::RED_THREADS, 0, tab, L, b->n)
                                : blaunch(b, vv::k_b_gm_maxpy_p<double>, vv::F_VEC, vv::RED_THREADS, 0, tab, L, b->n);
        }
    };
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeRelaxed));
    int r = VV_OK;
    for (int k = 0; k < reps && r == VV_OK; ++k) r = one();
    cudaError_t e = cudaStreamEndCapture(b->st, &g);
    if (r == VV_OK && e != cudaSuccess) r = fail_cuda(e, "vv_batch_time_kernel capture");
    if (r == VV_OK && (e = cudaGraphInstantiate(&ex, g, 0)) != cudaSuccess) r = fail_cuda(e, "vv_batch_time_kernel instantiate");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float ms = 0.f;
    if (r == VV_OK) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        e = cudaGraphLaunch(ex, b->st);   // warm-up
        if (e == cudaSuccess) e = cudaEventRecord(e0, b->st);
        if (e == cudaSuccess) e = cudaGraphLaunch(ex, b->st);
        if (e == cudaSuccess) e = cudaEventRecord(e1, b->st);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) r = fail_cuda(e, "vv_batch_time_kernel");
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (ex) cudaGraphExecDestroy(ex);
    if (g) cudaGraphDestroy(g);
    b->launches = l0;
    TRY(r);
    *avg_ms = (double)ms / reps;
    return VV_OK;
}

int vv_batch_launch_count(vv_batch* b, int64_t* launches, int reset) {
    if (!b) return VV_ERR_ARG;
    if (launches) *launches = b->launches;
    if (reset) b->launches = 0;
    return VV_OK;
}

}  // extern "C"
