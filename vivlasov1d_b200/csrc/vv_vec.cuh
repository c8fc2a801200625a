// Vector kernels of the Newton/Picard-GMRES loop: deterministic two-stage
// reductions, the fused multi-dot / multi-axpy of classical Gram-Schmidt,
// the GMRES Hessenberg/Givens bookkeeping (one thread; PETSc's KSPGMRES
// algorithm), moments + Poisson + h1 in one pass pair, and the invariants.
#pragma once
#include "vv_common.cuh"
#include "vv_pc.cuh"

namespace vv {

constexpr int RED_THREADS = 256;
constexpr int MAX_RESTART = 64;
constexpr int MDOT_CHUNK = 8;

// ---------------------------------------------------------------------------
// Device-resident solver state: GMRES (PETSc KSP_GMRES arrays: hh = rotated
// Hessenberg, column-major with ld = restart+2; grs = rotated right-hand side;
// cc/ss = Givens; KSPConvergedDefault state) and the Picard loop of the time
// step, plus the step report.  Every loop decision is taken here, so a whole
// time step can run as one CUDA graph with conditional nodes; when a
// conditional handle is 0 the kernels run outside a graph (host-driven).
// ---------------------------------------------------------------------------
constexpr int MAX_PICARD_DEV = 64;

struct DevState {
    // GMRES control
    int it, its, reason, active;
    int restart, max_it, first, pad;
    unsigned int cnt[4];   // last-CTA counters: 0 cycle sumsq, 1 mdot, 2 maxpy, 3 spare
    double rtol, atol, dtol, haptol;
    double rnorm0, ttol, res, scale, sumsq;
    // Picard control
    int pic_i, pic_stop, pic_revert, pic_stop_rule;
    int pic_max_iter, ksp_failures, gmres_total, pic_active;
    int ncycles, gm_outer;   // gm_outer: in a GMRES solve (lockstep batch mask)
    double snes_atol, abort_residual, pred, prev, pnorm2;
    // conditional handles (0 outside a graph)
    unsigned long long h_gm_outer, h_gm_inner, h_gm_first, h_pic, h_revert;
    // report
    int gmres_its[MAX_PICARD_DEV];
    int ksp_reason[MAX_PICARD_DEV];
    double residual[MAX_PICARD_DEV + 1];
    // initial guess (after the option header, which the host uploads before a
    // step, and before the GMRES arrays: part of the report read-back)
    double guess_prev, guess_res;
    int guess_kept;
    int have_set;   // 1 once update_previous has run (before it the solver's Have is zero)
    // GMRES arrays
    double hcol[MAX_RESTART + 2];
    double grs[MAX_RESTART + 2];
    double cc[MAX_RESTART + 1], ss[MAX_RESTART + 1];
    double hh[(MAX_RESTART + 2) * (MAX_RESTART + 1)];
    // 1/||V_q|| of the basis vectors as produced (the lockstep batch keeps V_q
    // unnormalised and applies these factors where it reads the basis)
    double vsc[MAX_RESTART + 2];
};

// PETSc reasons
constexpr int R_ITERATING = 0, R_RTOL = 2, R_ATOL = 3, R_NULL = -2, R_ITS = -3, R_DTOL = -4,
              R_BREAKDOWN = -5, R_NANORINF = -9;

VV_DEV void set_cond(unsigned long long h, unsigned int v) {
    if (h) cudaGraphSetConditional((cudaGraphConditionalHandle)h, v);
}

VV_DEV int ksp_converged(DevState* s, int n, double rnorm) {
    if (n == 0) {
        s->rnorm0 = rnorm;
        s->ttol = fmax(s->rtol * rnorm, s->atol);
    }
    if (isnan(rnorm) || isinf(rnorm)) return R_NANORINF;
    if (rnorm <= s->ttol) return rnorm < s->atol ? R_ATOL : R_RTOL;
    if (rnorm >= s->dtol * s->rnorm0) return R_DTOL;
    return R_ITERATING;
}

// Last-CTA election (threadfence reduction): true in every thread of the
// block that finishes last; that block also resets the counter.  No waiting.
__device__ __forceinline__ bool last_block(unsigned int* counter, unsigned int nblk) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = atomicAdd(counter, 1u);
        am_last = (t == nblk - 1);
        if (am_last) *counter = 0u;
    }
    __syncthreads();
    if (am_last) __threadfence();
    return am_last;
}
__device__ __forceinline__ bool last_block(unsigned int* counter) { return last_block(counter, gridDim.x); }

// deterministic sum of part[0..np) by one warp
__device__ __forceinline__ double warp_reduce_parts(const double* part, int np) {
    const int lane = threadIdx.x & 31;
    double a = 0.0;
    for (int b = lane; b < np; b += 32) a += __ldcg(part + b);
    return warp_sum(a);
}

// ----- partial sums of squares / sums --------------------------------------
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
k_sumsq_partial(const T* __restrict__ x, size_t n, double* __restrict__ part) {
    __shared__ double sh[RED_THREADS / 32];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)RED_THREADS + threadIdx.x; i < n; i += (size_t)gridDim.x * RED_THREADS) {
        const double v = (double)x[i];
        acc += v * v;
    }
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
k_sum_partial(const T* __restrict__ x, size_t n, double* __restrict__ part) {
    __shared__ double sh[RED_THREADS / 32];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)RED_THREADS + threadIdx.x; i < n; i += (size_t)gridDim.x * RED_THREADS)
        acc += (double)x[i];
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Reduce `np` partials per column (m columns, stride ld) into out[m].
__global__ void __launch_bounds__(RED_THREADS)
k_reduce_cols(const double* __restrict__ part, int np, int m, int ld, double* __restrict__ out) {
    const int w = threadIdx.x >> 5;
    for (int q = w; q < m; q += RED_THREADS / 32) {
        const double t = warp_reduce_parts(part + (size_t)q * ld, np);
        if ((threadIdx.x & 31) == 0) out[q] = t;
    }
}

// y = s * x, s = *scale (device) ; if scale pointer is null uses sval
template <typename TI, typename TO>
__global__ void k_scale(const TI* __restrict__ x, TO* __restrict__ y, size_t n, const double* __restrict__ scale,
                        double sval) {
    const double s = scale ? *scale : sval;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = (TO)((double)x[i] * s);
}

// y = a*x + b*y
template <typename T>
__global__ void k_axpby(const T* __restrict__ x, T* __restrict__ y, size_t n, double a, double b) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = (T)(a * (double)x[i] + b * (double)y[i]);
}

// ----- GMRES kernels (state driven) ----------------------------------------
// Start of a solve: x = 0; its = 0; first cycle.
template <typename T>
__device__ __forceinline__ void gm_init_block(DevState* s, T* __restrict__ x, size_t n, int bid, int nblk) {
    for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)nblk * blockDim.x)
        x[i] = T(0);
    if (bid == 0 && threadIdx.x == 0) {
        s->its = 0;
        s->reason = R_ITERATING;
        s->first = 1;
        s->active = 0;
        s->it = 0;
        set_cond(s->h_gm_first, 1u);
        set_cond(s->h_gm_outer, 1u);
    }
}
template <typename T>
__global__ void k_gm_init(DevState* s, T* __restrict__ x, size_t n) {
    gm_init_block<T>(s, x, n, blockIdx.x, gridDim.x);
}

// state update of a cycle start from ||V0||^2 (one thread)
VV_DEV void gm_cycle_state(DevState* s, double ss2) {
    const double res = sqrt(ss2);
    s->ncycles += 1;
    s->it = 0;
    s->grs[0] = res;
    s->res = res;
    s->scale = (res != 0.0) ? 1.0 / res : 1.0;
    s->vsc[0] = s->scale;
    if (res == 0.0) {
        s->reason = R_ATOL;
        s->active = 0;
    } else {
        s->reason = ksp_converged(s, s->its, res);
        s->active = (s->reason == R_ITERATING && s->its < s->max_it) ? 1 : 0;
    }
    set_cond(s->h_gm_inner, (unsigned)s->active);
}

// Cycle start (KSPGMRESCycle top): ||V0||^2 partials; the last CTA computes
// res, the convergence test with n = its, the scale 1/res and `active`.
template <typename T>
__device__ __forceinline__ void gm_cycle_block(DevState* s, const T* __restrict__ V0, size_t n,
                                               double* __restrict__ part, int bid, int nblk) {
    __shared__ double sh[RED_THREADS / 32];
    double acc = 0.0;
    for (size_t i = bid * (size_t)RED_THREADS + threadIdx.x; i < n; i += (size_t)nblk * RED_THREADS) {
        const double v = (double)V0[i];
        acc += v * v;
    }
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[bid] = t;
    if (!last_block(&s->cnt[0], nblk)) return;
    if (threadIdx.x >= 32) return;
    const double ss2 = warp_reduce_parts(part, nblk);
    if (threadIdx.x != 0) return;
    gm_cycle_state(s, ss2);
}
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
k_gm_cycle(DevState* s, const T* __restrict__ V0, size_t n, double* __restrict__ part) {
    gm_cycle_block<T>(s, V0, n, part, blockIdx.x, gridDim.x);
}

// V[idx] *= scale, idx = s->it (the vector just produced)
template <typename T>
__device__ __forceinline__ void gm_scale_block(const DevState* s, T* __restrict__ V, size_t ldv, size_t n, int bid,
                                               int nblk) {
    T* v = V + (size_t)s->it * ldv;
    const double sc = s->scale;
    for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)nblk * blockDim.x)
        v[i] = (T)((double)v[i] * sc);
}
template <typename T>
__global__ void k_gm_scale(DevState* s, T* __restrict__ V, size_t ldv, size_t n) {
    gm_scale_block<T>(s, V, ldv, n, blockIdx.x, gridDim.x);
}

// hcol_q = <w, V_q>, q = 0..it, w = V[it+1]  (one multi-dot, last CTA reduces)
template <typename T>
__device__ __forceinline__ void gm_mdot_block(DevState* s, const T* __restrict__ V, size_t ldv, size_t n,
                                              double* __restrict__ part, int ld, int bid, int nblk) {
    static_assert(MDOT_CHUNK <= RED_THREADS / 32, "one warp per dot of a chunk");
    __shared__ double shc[MDOT_CHUNK][RED_THREADS / 32];
    const int it = s->it;
    const int m = it + 1;
    const T* w = V + (size_t)(it + 1) * ldv;
    for (int q0 = 0; q0 < m; q0 += MDOT_CHUNK) {
        double acc[MDOT_CHUNK];
#pragma unroll
        for (int c = 0; c < MDOT_CHUNK; ++c) acc[c] = 0.0;
        const int cnt = min(MDOT_CHUNK, m - q0);
        for (size_t i = bid * (size_t)RED_THREADS + threadIdx.x; i < n; i += (size_t)nblk * RED_THREADS) {
            const double wi = (double)w[i];
#pragma unroll
            for (int c = 0; c < MDOT_CHUNK; ++c)
                if (c < cnt) acc[c] += wi * (double)V[(size_t)(q0 + c) * ldv + i];
        }
        // block sums of the chunk's dots: warp sums, one barrier, then warp c
        // adds the warp sums of dot c (the order of block_sum)
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int c = 0; c < MDOT_CHUNK; ++c) {
            if (c < cnt) {
                const double t = warp_sum(acc[c]);
                if (lane == 0) shc[c][wid] = t;
            }
        }
        __syncthreads();
        if (wid < cnt) {
            double r = (lane < RED_THREADS / 32) ? shc[wid][lane] : 0.0;
            r = warp_sum(r);
            if (lane == 0) part[(size_t)(q0 + wid) * ld + bid] = r;
        }
        __syncthreads();
    }
    if (!last_block(&s->cnt[1], nblk)) return;
    const int wid = threadIdx.x >> 5;
    for (int q = wid; q < m; q += RED_THREADS / 32) {
        const double t = warp_reduce_parts(part + (size_t)q * ld, nblk);
        if ((threadIdx.x & 31) == 0) s->hcol[q] = t;
    }
}
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
k_gm_mdot(DevState* s, const T* __restrict__ V, size_t ldv, size_t n, double* __restrict__ part, int ld) {
    gm_mdot_block<T>(s, V, ldv, n, part, ld, blockIdx.x, gridDim.x);
}

// Arnoldi bookkeeping after tt = ||w|| (KSPGMRESCycle + UpdateHessenberg)
// hcol, cc, ss: the state's arrays or copies of them (the lockstep batch
// stages them in shared memory so that the rotation chain does not wait on
// global loads ordered after its own stores)
VV_DEV void gm_arnoldi(DevState* s, double tt, const double* hcol, const double* cc, const double* ss) {
    const int it = s->it;
    const int ld = s->restart + 2;
    double* hh = s->hh;
#define HH(a, b) hh[(b) * ld + (a)]
    s->scale = (tt != 0.0) ? 1.0 / tt : 1.0;
    s->vsc[it + 1] = s->scale;
    HH(it + 1, it) = tt;
    double hapbnd = fabs(tt / s->grs[it]);
    if (hapbnd > s->haptol) hapbnd = s->haptol;
    const bool hapend = tt < hapbnd;
    // apply the previous rotations to the new column hcol (KSPGMRES's
    // HH(j-1) <- c t + s HH(j), HH(j) <- c HH(j) - s t, t = HH(j-1)): the
    // value carried from row to row stays in a register and the loads of
    // hcol, cc and ss do not wait on the stores of earlier rows
    double hj = hcol[0];
    for (int j = 1; j <= it; ++j) {
        const double hn = hcol[j];
        const double c = cc[j - 1], sn = ss[j - 1];
        HH(j - 1, it) = c * hj + sn * hn;
        hj = c * hn - sn * hj;
    }
    HH(it, it) = hj;
    bool null = false;
    if (!hapend) {
        const double h1 = tt;
        const double t = sqrt(hj * hj + h1 * h1);
        if (t == 0.0) {
            s->reason = R_NULL;
            null = true;
        } else {
            const double c = hj / t, sn = h1 / t;
            s->cc[it] = c;
            s->ss[it] = sn;
            const double g = s->grs[it];
            s->grs[it + 1] = -(sn * g);
            s->grs[it] = c * g;
            HH(it, it) = c * hj + sn * h1;
            s->res = fabs(sn * g);
        }
    } else {
        s->res = 0.0;
    }
#undef HH
    s->it = it + 1;
    s->its += 1;
    if (!null) {
        s->reason = ksp_converged(s, s->its, s->res);
        if (hapend && s->reason == R_ITERATING) s->reason = R_BREAKDOWN;
    }
    s->active = (s->reason == R_ITERATING && s->it < s->restart && s->its < s->max_it) ? 1 : 0;
    set_cond(s->h_gm_inner, (unsigned)s->active);
}
VV_DEV void gm_arnoldi(DevState* s, double tt) { gm_arnoldi(s, tt, s->hcol, s->cc, s->ss); }

// w += sum_q (-hcol_q) V_q and ||w||^2 (classical Gram-Schmidt update,
// VecMAXPY with lhh = -<w,v>); the last CTA finishes the Arnoldi step.
template <typename T>
__device__ __forceinline__ void gm_maxpy_block(DevState* s, T* __restrict__ V, size_t ldv, size_t n,
                                               double* __restrict__ part, int bid, int nblk) {
    __shared__ double sh[RED_THREADS / 32];
    __shared__ double cf[MAX_RESTART + 2];
    const int it = s->it;
    const int m = it + 1;
    T* w = V + (size_t)(it + 1) * ldv;
    for (int q = threadIdx.x; q < m; q += RED_THREADS) cf[q] = -s->hcol[q];
    __syncthreads();
    double acc = 0.0;
    for (size_t i = bid * (size_t)RED_THREADS + threadIdx.x; i < n; i += (size_t)nblk * RED_THREADS) {
        double wi = (double)w[i];
        for (int q = 0; q < m; ++q) wi += cf[q] * (double)V[(size_t)q * ldv + i];
        w[i] = (T)wi;
        acc += wi * wi;
    }
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[bid] = t;
    if (!last_block(&s->cnt[2], nblk)) return;
    if (threadIdx.x >= 32) return;
    const double ss2 = warp_reduce_parts(part, nblk);
    if (threadIdx.x == 0) gm_arnoldi(s, sqrt(ss2));
}
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
k_gm_maxpy(DevState* s, T* __restrict__ V, size_t ldv, size_t n, double* __restrict__ part) {
    gm_maxpy_block<T>(s, V, ldv, n, part, blockIdx.x, gridDim.x);
}

// KSPGMRESBuildSoln: every CTA solves the small triangular system (thread 0,
// into shared memory) and updates its share of x += sum nrs_q V_q; CTA 0
// records the outcome and decides whether another cycle follows.
// KSPGMRESBuildSoln's triangular solve (one thread): nrs[0..npad) from the
// rotated Hessenberg and right-hand side; npad = 0 on breakdown or no step.
VV_DEV void gm_backsolve(const DevState* s, double* nrs, int* npad_out, int* breakdown_out) {
    const int last = s->it - 1;
    const int ld = s->restart + 2;
    const double* hh = s->hh;
#define HH(a, b) hh[(b) * ld + (a)]
    int npad = 0, breakdown = 0;
    if (last >= 0) {
        if (HH(last, last) == 0.0) {
            breakdown = 1;
        } else {
            nrs[last] = s->grs[last] / HH(last, last);
            for (int ii = 1; ii <= last && !breakdown; ++ii) {
                const int k = last - ii;
                double t = s->grs[k];
                for (int j = k + 1; j <= last; ++j) t = t - HH(k, j) * nrs[j];
                if (HH(k, k) == 0.0) breakdown = 1;
                else nrs[k] = t / HH(k, k);
            }
            if (!breakdown) npad = last + 1;
        }
    }
#undef HH
    *npad_out = npad;
    *breakdown_out = breakdown;
}

// outcome of a cycle after the solution update (one thread)
VV_DEV void gm_finish_state(DevState* s, int npad, int breakdown) {
    if (breakdown) s->reason = R_BREAKDOWN;
    if (s->its >= s->max_it && s->reason == R_ITERATING) s->reason = R_ITS;
    s->first = 0;
    s->pad = npad;
    set_cond(s->h_gm_outer, s->reason == R_ITERATING ? 1u : 0u);
    set_cond(s->h_gm_first, 0u);
}

template <typename T>
__device__ __forceinline__ void gm_finish_block(DevState* s, const T* __restrict__ V, size_t ldv, T* __restrict__ x,
                                                size_t n, int bid, int nblk) {
    __shared__ double nrs[MAX_RESTART + 1];
    __shared__ int npad, breakdown;
    if (threadIdx.x == 0) gm_backsolve(s, nrs, &npad, &breakdown);
    __syncthreads();
    const int m = npad;
    if (m > 0) {
        for (size_t i = bid * (size_t)RED_THREADS + threadIdx.x; i < n; i += (size_t)nblk * RED_THREADS) {
            double xi = (double)x[i];
            for (int q = 0; q < m; ++q) xi += nrs[q] * (double)V[(size_t)q * ldv + i];
            x[i] = (T)xi;
        }
    }
    if (bid == 0 && threadIdx.x == 0) gm_finish_state(s, m, breakdown);
}
template <typename T>
__global__ void __launch_bounds__(RED_THREADS)
k_gm_finish(DevState* s, const T* __restrict__ V, size_t ldv, T* __restrict__ x, size_t n) {
    gm_finish_block<T>(s, V, ldv, x, n, blockIdx.x, gridDim.x);
}

// ----- Picard-loop kernels -------------------------------------------------
// f -= delta unless the linear solve failed (SNES ksponly skips the update
// when the KSP reason is negative); record the solve in the report.
template <typename TF, typename TD>
__device__ __forceinline__ void pic_apply_block(DevState* s, const TF* __restrict__ delta, TD* __restrict__ f,
                                                size_t n, int bid, int nblk) {
    const bool ok = s->reason >= 0;
    if (ok) {
        for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)nblk * blockDim.x)
            f[i] = f[i] - (TD)delta[i];
    }
    if (bid == 0 && threadIdx.x == 0) {
        const int k = s->pic_i;
        if (k < MAX_PICARD_DEV) {
            s->gmres_its[k] = s->its;
            s->ksp_reason[k] = s->reason;
        }
        s->gmres_total += s->its;
        if (!ok) s->ksp_failures += 1;
    }
}
template <typename TF, typename TD>
__global__ void k_pic_apply(DevState* s, const TF* __restrict__ delta, TD* __restrict__ f, size_t n) {
    pic_apply_block<TF, TD>(s, delta, f, n, blockIdx.x, gridDim.x);
}

// Residual of the current iterate: ||R(f)|| from the bracket kernel's tile
// partials plus ||Poisson residual|| (s->pnorm2), then the stop rules of
// run_nonlinear_matrixfree_split_mp.py:158-163.  phase 0: the initial residual.
__device__ __forceinline__ void pic_residual_warp(DevState* s, const double* __restrict__ part, int np, int phase) {
    if (threadIdx.x >= 32) return;
    const double f2 = warp_reduce_parts(part, np);
    if (threadIdx.x != 0) return;
    const double pred = sqrt(f2) + sqrt(s->pnorm2);
    if (phase == 0) {
        s->have_set = 1;   // the step's prologue ran update_previous
        s->pred = pred;
        s->residual[0] = pred;
        s->pic_i = 0;
        s->pic_stop = 0;
        s->pic_revert = 0;
        s->pic_stop_rule = 0;
        s->gmres_total = 0;
        s->ksp_failures = 0;
        s->ncycles = 0;
        s->pic_active = 1;
        set_cond(s->h_pic, 1u);
        set_cond(s->h_revert, 0u);
        return;
    }
    const int i = s->pic_i + 1;
    s->pic_i = i;
    s->prev = s->pred;
    s->pred = pred;
    if (i <= MAX_PICARD_DEV) s->residual[i] = pred;
    const bool rose = pred > s->prev && i > 1;
    const bool small = pred < s->snes_atol;
    const bool maxed = i >= s->pic_max_iter || i >= MAX_PICARD_DEV;
    if (rose || small || maxed) {
        s->pic_stop_rule = rose ? 1 : (small ? 2 : 3);
        s->pic_revert = pred > s->prev ? 1 : 0;
        s->pic_stop = 1;
        s->pic_active = 0;
    }
    set_cond(s->h_pic, s->pic_active ? 1u : 0u);
    set_cond(s->h_revert, (unsigned)s->pic_revert);
}
__global__ void k_pic_residual(DevState* s, const double* __restrict__ part, int np, int phase) {
    pic_residual_warp(s, part, np, phase);
}

// ---------------------------------------------------------------------------
// moments: partial sums over v segments, then one CTA finishes moments,
// Poisson (spectral, CFD4 symbol) and h1 = phi - mean(phi).
// ---------------------------------------------------------------------------
constexpr int MOM_TX = 32, MOM_TY = 8;

template <typename T>
__device__ __forceinline__ void moments_partial_block(const T* __restrict__ F, int nx, int nv, int seg,
                                                      const double* __restrict__ v,
                                                      double* __restrict__ part /* [S][3][nx] */, int bx, int s) {
    __shared__ double sh[3][MOM_TY][MOM_TX + 1];
    const int i = bx * MOM_TX + threadIdx.x;
    const int ja = s * seg, jb = min(nv, ja + seg);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if (i < nx) {
        for (int j = ja + threadIdx.y; j < jb; j += MOM_TY) {
            const double f = (double)F[(size_t)j * nx + i];
            const double vj = v[j];
            a0 += f;
            a1 += vj * f;
            a2 += (vj * vj) * f;
        }
    }
    sh[0][threadIdx.y][threadIdx.x] = a0;
    sh[1][threadIdx.y][threadIdx.x] = a1;
    sh[2][threadIdx.y][threadIdx.x] = a2;
    __syncthreads();
    if (threadIdx.y < 3 && i < nx) {
        double t = 0.0;
        for (int y = 0; y < MOM_TY; ++y) t += sh[threadIdx.y][y][threadIdx.x];
        part[((size_t)s * 3 + threadIdx.y) * nx + i] = t;
    }
}
template <typename T>
__global__ void __launch_bounds__(MOM_TX * MOM_TY)
k_moments_partial(const T* __restrict__ F, int nx, int nv, int seg, const double* __restrict__ v,
                  double* __restrict__ part /* [S][3][nx] */) {
    moments_partial_block<T>(F, nx, nv, seg, v, part, blockIdx.x, blockIdx.y);
}

struct PoissonParams {
    int nx, M, logM, S;   // S = number of moment partials
    double hv, charge, hx2_inv, hx, inv_nx;
    const double2* tw;       // nx twiddles W^k (the FFT reads k < nx/2)
    const double* sym_inv;   // M+1 entries: (density-average symbol / Laplacian symbol)_k, 0 for k = 0
    // the Laplacian: periodic stencil (la2, la1, la0, la1, la2) / lden hx^-2
    double la0, la1, la2, lden;
    // the density in the right-hand side: (ra2, ra1, ra0, ra1, ra2) / rden
    // (PETScPoissonCFD2Ave/SimpsonAve.pyx; ravg = 0: n itself); the spectral
    // solve folds its symbol into sym_inv
    int ravg;
    double ra0, ra1, ra2, rden;
};

// the right-hand side's density at i: n_i, or its periodic 5-point average
// in the reference's order ((((r2 n_{i-2} + r1 n_{i-1}) + r0 n_i) + r1 n_{i+1})
// + r2 n_{i+2}) / rden
__device__ __forceinline__ double rhs_density(const double* __restrict__ n, int i, int nx, int ravg, double r0,
                                              double r1, double r2, double rden) {
    if (!ravg) return n[i];
    const int im2 = (i - 2 + 2 * nx) % nx, im1 = (i - 1 + nx) % nx;
    const int ip1 = (i + 1) % nx, ip2 = (i + 2) % nx;
    return ((((r2 * n[im2] + r1 * n[im1]) + r0 * n[i]) + r1 * n[ip1]) + r2 * n[ip2]) / rden;
}

constexpr int POIS_THREADS = 1024;

// Single CTA.  Inputs: moment partials (or n directly when part == nullptr).
// Outputs (each optional): n, u, e, a, phi, h1; scal[0] = ||Poisson residual||_2,
// scal[1] = sum(phi).
__device__ __forceinline__ void moments_poisson_cta(const double* __restrict__ part, const double* __restrict__ n_in,
                                                    double* __restrict__ n, double* __restrict__ u,
                                                    double* __restrict__ e, double* __restrict__ a,
                                                    double* __restrict__ phi, double* __restrict__ h1,
                                                    double* __restrict__ scal, const PoissonParams& p) {
    extern __shared__ double2 psm[];
    double2* buf = psm;                                   // M + 1 complex
    double* nn = reinterpret_cast<double*>(psm + p.M + 1);  // nx, padded to an even count
    double* ph = nn + ((p.nx + 1) & ~1);                  // nx + 2; 16-byte aligned (read as double2)
    __shared__ double red[POIS_THREADS / 32];
    const int nx = p.nx, M = p.M;
    // 1. moments
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        double s0, s1 = 0.0, s2 = 0.0;
        if (part) {
            s0 = 0.0;
            for (int s = 0; s < p.S; ++s) {
                s0 += part[((size_t)s * 3 + 0) * nx + i];
                s1 += part[((size_t)s * 3 + 1) * nx + i];
                s2 += part[((size_t)s * 3 + 2) * nx + i];
            }
            s0 *= p.hv; s1 *= p.hv; s2 *= p.hv;
            if (n) n[i] = s0;
            if (u) u[i] = s1;
            if (e) e[i] = s2;
            if (a) a[i] = s0 * s0 / (s0 * s2 - s1 * s1);   // Toolbox.pyx:164-165
        } else {
            s0 = n_in[i];
        }
        nn[i] = s0;
    }
    __syncthreads();
    if (!phi && !h1 && !scal) return;
    // 2. rhs b = -(n - mean n)*charge
    double t = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) t += nn[i];
    t = block_sum(t, red);
    __shared__ double nmean_s;
    if (threadIdx.x == 0) nmean_s = t * p.inv_nx;
    __syncthreads();
    const double nmean = nmean_s;
    double* phs;
    if (p.logM < 0) {
        // 3'. any nx: direct DFT of b, divide by the symbol, direct inverse
        //     (numpy's rfft / irfft conventions)
        double2* X2 = reinterpret_cast<double2*>(ph);   // M+1 complex <= nx + 2 doubles
        for (int k = threadIdx.x; k <= M; k += blockDim.x) {
            double re = 0.0, im = 0.0;
            int idx = 0;
            for (int m = 0; m < nx; ++m) {
                const double b = -(nn[m] - nmean) * p.charge;
                const double2 w = p.tw[idx];
                re += b * w.x;
                im += b * w.y;
                idx += k;
                if (idx >= nx) idx -= nx;
            }
            double2 Xk = make_double2(re * p.sym_inv[k], im * p.sym_inv[k]);
            if (k == 0 || 2 * k == nx) Xk.y = 0.0;
            X2[k] = Xk;
        }
        __syncthreads();
        phs = reinterpret_cast<double*>(buf);            // 2M + 2 >= nx doubles
        const int K = (nx - 1) / 2;
        for (int m = threadIdx.x; m < nx; m += blockDim.x) {
            double s = X2[0].x;
            int idx = 0;
            for (int k = 1; k <= K; ++k) {
                idx += m;
                if (idx >= nx) idx -= nx;
                const double2 w = p.tw[idx];
                s += 2.0 * (X2[k].x * w.x + X2[k].y * w.y);
            }
            if (!(nx & 1)) s += (m & 1) ? -X2[nx / 2].x : X2[nx / 2].x;
            phs[m] = s * p.inv_nx;
        }
        __syncthreads();
    } else {
    // 3. FFT of b (real, via M-point complex), divide by the symbol, inverse
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        const double b0 = -(nn[2 * m] - nmean) * p.charge;
        const double b1 = -(nn[2 * m + 1] - nmean) * p.charge;
        buf[bitrev(m, p.logM)] = make_double2(b0, b1);
    }
    __syncthreads();
    block_fft<-1>(buf, M, p.tw);
    // split into X_k (k = 0..M), divide, rebuild Z for the inverse in place:
    // every thread handles the pair (k, M-k) so the in-place update is safe.
    double2* X2 = reinterpret_cast<double2*>(ph);  // reuse ph storage: needs (M+1) complex = nx+2 doubles
    for (int k = threadIdx.x; k <= M; k += blockDim.x) {
        const double2 zk = buf[k == M ? 0 : k];
        const double2 zc = c_conj(buf[k == 0 ? 0 : M - k]);
        const double2 E = c_scale(c_add(zk, zc), 0.5);
        const double2 D = c_sub(zk, zc);
        const double2 O = make_double2(0.5 * D.y, -0.5 * D.x);
        const double2 w = (k < M) ? p.tw[k] : make_double2(-1.0, 0.0);
        double2 Xk = c_add(E, c_mul(w, O));
        Xk = c_scale(Xk, p.sym_inv[k]);
        if (k == 0 || k == M) Xk.y = 0.0;
        X2[k] = Xk;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < M; k += blockDim.x) {
        const double2 xk = X2[k];
        const double2 xc = c_conj(X2[M - k]);
        const double2 E = c_scale(c_add(xk, xc), 0.5);
        double2 w = p.tw[k];
        w.y = -w.y;
        const double2 O = c_mul(w, c_scale(c_sub(xk, xc), 0.5));
        buf[bitrev(k, p.logM)] = make_double2(E.x - O.y, E.y + O.x);
    }
    __syncthreads();
    block_fft<+1>(buf, M, p.tw);
    const double sc = 1.0 / (double)M;
    phs = reinterpret_cast<double*>(X2);  // overwrite: phi in smem
    __syncthreads();
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        phs[2 * m] = buf[m].x * sc;
        phs[2 * m + 1] = buf[m].y * sc;
    }
    __syncthreads();
    }
    // 4. mean of phi, h1 and Poisson residual A phi + (n - nmean) charge
    t = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) t += phs[i];
    t = block_sum(t, red);
    __shared__ double phimean_s, phisum_s;
    if (threadIdx.x == 0) { phisum_s = t; phimean_s = t * p.inv_nx; }
    __syncthreads();
    double r2 = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const double pc = phs[i];
        if (phi) phi[i] = pc;
        if (h1) h1[i] = pc - phimean_s;
        const int im2 = (i - 2 + 2 * nx) % nx, im1 = (i - 1 + nx) % nx;
        const int ip1 = (i + 1) % nx, ip2 = (i + 2) % nx;
        const double Ax =
            (p.la2 * phs[im2] + p.la1 * phs[im1] + p.la0 * pc + p.la1 * phs[ip1] + p.la2 * phs[ip2]) * p.hx2_inv / p.lden;
        const double r = Ax + (rhs_density(nn, i, nx, p.ravg, p.ra0, p.ra1, p.ra2, p.rden) - nmean) * p.charge;
        r2 += r * r;
    }
    r2 = block_sum(r2, red);
    if (threadIdx.x == 0 && scal) {
        scal[0] = sqrt(r2);
        scal[1] = phisum_s;
    }
}
__global__ void __launch_bounds__(POIS_THREADS)
k_moments_poisson(const double* __restrict__ part, const double* __restrict__ n_in,
                  double* __restrict__ n, double* __restrict__ u, double* __restrict__ e,
                  double* __restrict__ a, double* __restrict__ phi, double* __restrict__ h1,
                  double* __restrict__ scal, PoissonParams p) {
    moments_poisson_cta(part, n_in, n, u, e, a, phi, h1, scal, p);
}

// Poisson apply (one CTA): mode 0 rhs b = -(n~ - mean n) charge, 1 matvec
// (the stencil (a2, a1, a0, a1, a2) / den hx^-2 of the Laplacian), 2
// function (matvec + (n~ - mean n) charge), n~ = rhs_density; optional
// ||y||^2 -> sumsq (PETScPoissonSolver.pyx:58-74, PETScPoissonCFD4.pyx:64-101,
// PETScPoissonCFD2.pyx:64-101, PETScPoissonSimpson.pyx:62-101,
// PETScPoissonCFD2Ave.pyx, PETScPoissonSimpsonAve.pyx)
__device__ __forceinline__ void poisson_apply_cta(const double* __restrict__ x, const double* __restrict__ n,
                                                  double* __restrict__ y, int nx, double hx2_inv, double charge,
                                                  int mode, double* __restrict__ sumsq, double a0, double a1,
                                                  double a2, double den, int ravg, double ra0, double ra1,
                                                  double ra2, double rden) {
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
            r = -(rhs_density(n, i, nx, ravg, ra0, ra1, ra2, rden) - nmean_s) * charge;
        } else {
            const int im2 = (i - 2 + 2 * nx) % nx, im1 = (i - 1 + nx) % nx;
            const int ip1 = (i + 1) % nx, ip2 = (i + 2) % nx;
            r = (a2 * x[im2] + a1 * x[im1] + a0 * x[i] + a1 * x[ip1] + a2 * x[ip2]) * hx2_inv / den;
            if (mode == 2) r = r + (rhs_density(n, i, nx, ravg, ra0, ra1, ra2, rden) - nmean_s) * charge;
        }
        if (y) y[i] = r;
        r2 += r * r;
    }
    r2 = block_sum(r2, red);
    if (threadIdx.x == 0 && sumsq) sumsq[0] = r2;
}

// ---------------------------------------------------------------------------
// invariants (distribution_function.pyx:130-306, hamiltonian.pyx:67-124,
// potential.pyx:48-59), compensated FP64 sums
// ---------------------------------------------------------------------------
constexpr int INV_SUMS = 13;   // mass, L1..L6, L8, S, Ekin, Ep1, Ep2, P
constexpr int INV_NPART = INV_SUMS + 2;  // + min, max

// one CTA: h1 = phi - mean(phi) into h1out, field energy into fe[0]
__global__ void k_xprofile(const double* __restrict__ phi, int nx, double charge, double hx,
                           double* __restrict__ h1out, double* __restrict__ fe) {
    __shared__ double red[32];
    __shared__ double mean_s;
    double t = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) t += phi[i];
    t = block_sum(t, red);
    if (threadIdx.x == 0) mean_s = t / nx;
    __syncthreads();
    double w = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        h1out[i] = phi[i] - mean_s;
        const double d = phi[(i + 1) % nx] - phi[i];
        w += d * d;
    }
    w = block_sum(w, red);
    if (threadIdx.x == 0) fe[0] = 0.5 * charge * w / hx;
}

__global__ void __launch_bounds__(RED_THREADS)
k_invariants_partial(const double* __restrict__ f, int nx, int nv, const double* __restrict__ v,
                     const double* __restrict__ h0, const double* __restrict__ h1,
                     const double* __restrict__ h2, double* __restrict__ part) {
    __shared__ double sh[RED_THREADS / 32];
    KSum acc[INV_SUMS];
#pragma unroll
    for (int q = 0; q < INV_SUMS; ++q) acc[q].init();
    double fmn = INFINITY, fmx = -INFINITY;
    const size_t n = (size_t)nx * nv;
    for (size_t idx = blockIdx.x * (size_t)RED_THREADS + threadIdx.x; idx < n;
         idx += (size_t)gridDim.x * RED_THREADS) {
        const int j = (int)(idx / nx), i = (int)(idx - (size_t)j * nx);
        const double fv = f[idx];
        fmn = fmin(fmn, fv);
        fmx = fmax(fmx, fv);
        acc[9].add(fv * h0[j]);
        acc[10].add(fv * h1[i]);
        if (h2) acc[11].add(fv * h2[i]);
        if (j < nv - 1) {
            const int ip = (i + 1 == nx) ? 0 : i + 1;
            const double s4 = ((fv + f[(size_t)j * nx + ip]) + f[(size_t)(j + 1) * nx + ip]) + f[(size_t)(j + 1) * nx + i];
            acc[0].add(s4);
            const double f2 = fv * fv, f3 = f2 * fv, f4 = f2 * f2;
            acc[1].add(fabs(fv));
            acc[2].add(f2);
            acc[3].add(f3);
            acc[4].add(f4);
            acc[5].add(f4 * fv);
            acc[6].add(f3 * f3);
            acc[7].add(f4 * f4);
            const double fe = fv <= 0.0 ? 1e-15 : fv;
            acc[8].add(fe * log(fe));
            acc[12].add(fv * v[j]);
        }
    }
    for (int q = 0; q < INV_SUMS; ++q) {
        const double t = block_sum(acc[q].value(), sh);
        if (threadIdx.x == 0) part[(size_t)q * gridDim.x + blockIdx.x] = t;
        __syncthreads();
    }
    {
        double m = warp_min(fmn);
        __shared__ double shm[RED_THREADS / 32], shx[RED_THREADS / 32];
        double x = warp_max(fmx);
        if ((threadIdx.x & 31) == 0) { shm[threadIdx.x >> 5] = m; shx[threadIdx.x >> 5] = x; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < RED_THREADS / 32; ++w) { m = fmin(m, shm[w]); x = fmax(x, shx[w]); }
            part[(size_t)INV_SUMS * gridDim.x + blockIdx.x] = m;
            part[(size_t)(INV_SUMS + 1) * gridDim.x + blockIdx.x] = x;
        }
    }
}

// one CTA: out[q] for the 13 sums (compensated over partials), min, max
__global__ void __launch_bounds__(RED_THREADS)
k_invariants_final(const double* __restrict__ part, int np, double* __restrict__ out) {
    __shared__ double sh[RED_THREADS / 32];
    for (int q = 0; q < INV_SUMS; ++q) {
        KSum a; a.init();
        for (int b = threadIdx.x; b < np; b += RED_THREADS) a.add(part[(size_t)q * np + b]);
        const double t = block_sum(a.value(), sh);
        if (threadIdx.x == 0) out[q] = t;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double m = INFINITY, x = -INFINITY;
        for (int b = 0; b < np; ++b) {
            m = fmin(m, part[(size_t)INV_SUMS * np + b]);
            x = fmax(x, part[(size_t)(INV_SUMS + 1) * np + b]);
        }
        out[INV_SUMS] = m;
        out[INV_SUMS + 1] = x;
    }
}

}  // namespace vv
