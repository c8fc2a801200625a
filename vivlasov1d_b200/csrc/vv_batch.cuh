// Lockstep batch kernels: one launch serves every instance of a batch.
//
// A batch is a table of independent runs (any mix of grid sizes and initial
// data).  Each kernel of the time step is launched once for the whole table
// with a persistent grid (sized to fill the GPU once): its blocks loop over
// the work items of the instances that are active in the current pass --
// every item is (instance, local block), and runs the same body as the
// single-grid kernel does for that block.  Every instance keeps its own
// Picard and GMRES state (DevState).  The one-block control kernel k_b_ctrl
// applies the state transitions of the loop masks, folds them into the loop
// conditions of the batch graph and rebuilds the compacted work lists:
// for each mask, the active instances and, per kernel family, the prefix
// sums of their block counts.  Instances that converge early thus cost
// nothing in the passes the others still need.
#pragma once
#include "vv_bracket.cuh"
#include "vv_pc.cuh"
#include "vv_pcj.cuh"
#include "vv_vec.cuh"

namespace vv {

// kernel families (work items per instance)
enum BFam { F_TILE = 0, F_ROWS = 1, F_MODES = 2, F_VEC = 3, F_MOM = 4, F_INST = 5, F_MARCH = 6, NFAM = 7 };

// marching Jacobian stencil of the batch: strips of MARCH_BW columns (every
// batch nx is a multiple of 64), segments of MARCH_SEG rows
constexpr int MARCH_BW = 64, MARCH_SEG = 128;
// work lists (one per mask)
// L_TAIL: the batch autotuner's stand-in for the lockstep tail (the largest instances)
enum BList { L_ALL = 0, L_PIC = 1, L_GM = 2, L_GMR = 3, L_INNER = 4, L_REVERT = 5, L_TAIL = 6, NLIST = 7 };

// per-instance description read by the batched kernels (device-resident)
struct BInst {
    DevState* ds;
    int cnt[NFAM];               // work items per family
    int nx, nv, tiles_x, vblk;   // wide-stencil tiles along x; blocks of the vector kernels
    int mom_seg, mom_bx, mom_S;  // moments: v rows per segment, x blocks, segments
    size_t ncell;
    BracketParams bp;            // factor and xidx are set per launch
    PcParams pp;                 // FFT parameters in the GMRES precision (R = rows per CTA of the batch)
    TriParams tp;
    PoissonParams po;
    // run state (FP64, vv_state)
    double *f, *fh, *phi, *phih, *h1c, *h1h, *h2c, *h2h, *n, *u, *e, *a;
    // context work buffers (FP64)
    double *Fh, *tmp, *fl, *part, *mom_part, *hxp, *v, *scal;
    // GMRES buffers in the GMRES precision: basis, operator scratch, rhs, solution, spectrum
    void *V, *tmpT, *bT, *xT, *specT;
    // LU reciprocals of the preconditioner, v-major (dinvJ[j*(M+1) + k]; the v-major layout)
    const void* dinvJ;
    // per-warp partial sums of the GMRES reductions: (restart + 2) columns of 8 * vblk
    double* wpart;
    // the Jacobian stencil's coefficients in the GMRES precision (jfp32: FP32):
    // per column (B1, bm, bp) from the x profile of h (rewritten by k_b_poisson
    // every Picard pass), per row (A1, am, ap) from h0; jscheme: 1, 2 or 4
    void *jcol, *jrow;
    int jfp32, jscheme;
};

// layout of one work list: [nact][total per family][ids: n][prefix per family: n+1]
__host__ __device__ constexpr size_t blist_words(int n) { return 1 + NFAM + (size_t)n + (size_t)NFAM * (n + 1); }

// 16-byte vector of T (the batch kernels' vector loads)
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };

// active instances whose list a block stages in shared memory for the search
constexpr int BLIST_SMEM = 512;
constexpr int CTRL_THREADS = 1024;   // control blocks and the per-instance finalize kernels

// The list header of family F: the number of instances and of work items,
// and the first entries of the list's prefix and id arrays, loaded together
// in one round trip (the arrays' addresses do not depend on the header; a
// tail pass of a few instances needs nothing more).  Thread t holds pre[t]
// for t < list_npre() and ids[t] for t < list_nids() (within the arrays).
constexpr int LIST_SPEC = 32;
VV_DEV int list_npre() { return min(LIST_SPEC + 1, (int)blockDim.x); }
VV_DEV int list_nids() { return min(LIST_SPEC, (int)blockDim.x); }
struct ListHead {
    int nact, total, pre, id;
};
template <int F>
VV_DEV ListHead list_head(const int* __restrict__ L, int n) {
    const int* ids = L + 1 + NFAM;
    const int* pre = ids + n + (size_t)F * (n + 1);
    const int t = threadIdx.x;
    ListHead h;
    h.pre = (t < list_npre() && t <= n) ? pre[t] : 0;   // pre holds n + 1 entries
    h.id = (t < list_nids() && t < n) ? ids[t] : 0;
    h.nact = L[0];
    h.total = L[1 + F];
    return h;
}
// stage pre[0..nact] and ids[0..nact) in shared memory (nact <= BLIST_SMEM;
// the caller takes a barrier before reading them): the entries the header
// brought, then the rest
template <int F>
VV_DEV void list_stage(const int* __restrict__ L, int n, const ListHead& h, int* s_pre, int* s_ids) {
    const int* ids = L + 1 + NFAM;
    const int* pre = ids + n + (size_t)F * (n + 1);
    const int t = threadIdx.x, np = list_npre(), ni = list_nids();
    if (t < np && t <= h.nact) s_pre[t] = h.pre;
    if (t < ni && t < h.nact) s_ids[t] = h.id;
    for (int i = np + t; i <= h.nact; i += blockDim.x) s_pre[i] = pre[i];
    for (int i = ni + t; i < h.nact; i += blockDim.x) s_ids[i] = ids[i];
}

// Loop of a persistent block over the work items of family F in list L:
// body(instance, local block).  Block-uniform; a barrier separates items.
// Lists of up to STAGE_MAX instances are searched in shared memory.
template <int F, int STAGE_MAX = BLIST_SMEM, typename Body>
VV_DEV void for_work(const BInst* __restrict__ tab, const int* __restrict__ L, int n, Body body) {
    __shared__ int s_pre[STAGE_MAX + 1];
    __shared__ int s_ids[STAGE_MAX];
    const ListHead h = list_head<F>(L, n);
    const int nact = h.nact;
    const int total = h.total;
    if ((int)blockIdx.x >= total) return;
    const int* ids = L + 1 + NFAM;
    const int* pre = ids + n + (size_t)F * (n + 1);
    const bool staged = nact <= STAGE_MAX;
    if (staged) {
        list_stage<F>(L, n, h, s_pre, s_ids);
        __syncthreads();
        pre = s_pre;
        ids = s_ids;
    }
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        int lo = 0, hi = nact - 1;   // the last p with pre[p] <= w
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pre[mid] <= w) lo = mid;
            else hi = mid - 1;
        }
        body(tab[ids[lo]], w - pre[lo]);
        __syncthreads();
    }
}

// Warp-granular loop over the same work: block item b of an instance is the
// eight warp items 8 b .. 8 b + 7, and every warp walks the list's warp items
// on its own (body(instance, local warp item, part, split), warp-uniform),
// with no barrier between items, so the warps of an SM overlap one item's
// header loads with another's data.  With Split, a list with fewer warp items
// than the grid has warps gives each item to `split` warps (part 0 .. split
// - 1) to divide among them.  For bodies that use no shared memory per item;
// the block must have 8 warps.
constexpr int MAX_SPLIT = 8;
template <int F, bool Split = false, typename Body>
VV_DEV void for_warp_work(const BInst* __restrict__ tab, const int* __restrict__ L, int n, Body body) {
    __shared__ int s_pre[BLIST_SMEM + 1];
    __shared__ int s_ids[BLIST_SMEM];
    const ListHead h = list_head<F>(L, n);
    const int nact = h.nact;
    const int total = h.total;
    const int nw = gridDim.x * 8, wtotal = 8 * total;
    // split factor: when the list holds fewer warp items than the grid has
    // warps (a few instances left), every item is taken by `split` warps,
    // which the body divides its work among (body(instance, item, part))
    const int split = Split ? max(1, min(MAX_SPLIT, nw / max(1, wtotal))) : 1;
    if ((int)blockIdx.x * 8 >= wtotal * split) return;
    const int* ids = L + 1 + NFAM;
    const int* pre = ids + n + (size_t)F * (n + 1);
    if (nact <= BLIST_SMEM) {
        list_stage<F>(L, n, h, s_pre, s_ids);
        __syncthreads();
        pre = s_pre;
        ids = s_ids;
    }
    for (int e = blockIdx.x * 8 + (threadIdx.x >> 5); e < wtotal * split; e += nw) {
        const int w = e / split, part = e - w * split;
        const int bw = w >> 3;
        int lo = 0, hi = nact - 1;   // the last p with pre[p] <= bw
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pre[mid] <= bw) lo = mid;
            else hi = mid - 1;
        }
        body(tab[ids[lo]], w - 8 * pre[lo], part, split);
    }
}

// ---- stencil ----------------------------------------------------------------
enum BSrc { BS_RESIDUAL = 0, BS_X = 1, BS_VIT = 2 };

// RESIDUAL: tmp = R(f) (FP64) with tile partials; BS_X: tmpT = J x;
// BS_VIT: tmpT = J v_it, v_it = vsc[it] V[it] (the Arnoldi input; the
// operator is linear, so the factor scales its two coefficients)
template <int SCHEME, int SRC, typename T>
__global__ void __launch_bounds__(WTHREADS, 4) k_b_bracket(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_TILE>(tab, L, n, [&](const BInst& I, int local) {
        BracketParams p = I.bp;
        p.xidx = nullptr;
        const int bx = local % I.tiles_x, by = local / I.tiles_x;
        if (SRC == BS_RESIDUAL) {
            p.factor = 1.0;
            bracket_wide_tile<SCHEME, MODE_RESIDUAL, double>(I.f, I.Fh, I.tmp, p, I.part, bx, by, I.tiles_x);
        } else {
            p.factor = 0.5;
            if (SRC == BS_VIT) {
                const double sc = I.ds->vsc[I.ds->it];
                p.factor *= sc;
                p.ht_inv *= sc;
            }
            const T* X = (SRC == BS_X) ? (const T*)I.xT : (const T*)I.V + (size_t)I.ds->it * I.ncell;
            bracket_wide_tile<SCHEME, MODE_JVP, T>(X, nullptr, (T*)I.tmpT, p, nullptr, bx, by, I.tiles_x);
        }
    });
}

// The Jacobian stencil by the marching kernel (same arithmetic as the tiles,
// bit for bit): BS_X: tmpT = J x; BS_VIT: tmpT = J v_it
template <int SCHEME, int SRC, typename T>
__global__ void __launch_bounds__(MARCH_BW) k_b_bracket_march(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                             int n) {
    for_work<F_MARCH>(tab, L, n, [&](const BInst& I, int local) {
        BracketParams p = I.bp;
        p.xidx = nullptr;
        p.factor = 0.5;
        if (SRC == BS_VIT) {
            const double sc = I.ds->vsc[I.ds->it];
            p.factor *= sc;
            p.ht_inv *= sc;
        }
        const T* X = (SRC == BS_X) ? (const T*)I.xT : (const T*)I.V + (size_t)I.ds->it * I.ncell;
        const int strips = I.nx / MARCH_BW;
        bracket_march_item<SCHEME, T, MARCH_BW>(X, (T*)I.tmpT, p, MARCH_SEG, local % strips, local / strips);
    });
}

// ---- preconditioner ---------------------------------------------------------
// rFFT rows: input FP64 tmp (right-hand side) or the GMRES-precision scratch
// FS: the four-step register/shuffle FFT for rows of 64 to 256 points (a
// switch on each instance's half length M; longer rows would raise the
// register count of every instance's blocks), else the radix-2 warp FFT
template <typename TI, typename R, bool FS>
__global__ void k_b_rfft(const BInst* __restrict__ tab, const int* __restrict__ L, int n, int from_tmp64) {
    for_work<F_ROWS>(tab, L, n, [&](const BInst& I, int local) {
        const TI* X = from_tmp64 ? (const TI*)I.tmp : (const TI*)I.tmpT;
        auto* spec = (typename Cplx<R>::type*)I.specT;
        if (FS) {
            switch (I.pp.M) {
                case 32: rfft4_block<TI, R, 1>(X, spec, I.pp, local); return;
                case 64: rfft4_block<TI, R, 2>(X, spec, I.pp, local); return;
                case 128: rfft4_block<TI, R, 4>(X, spec, I.pp, local); return;
                default: break;
            }
        }
        rfft_rows_block<TI, R>(X, spec, I.pp, local);
    });
}

// tridiagonal solves: one CTA per mode (tables staged in shared memory or
// read through L1), or one warp per mode (an item is TRIW_WARPS modes); the
// batch autotuner picks the variant
template <typename R, bool STAGE>
__global__ void __launch_bounds__(TRI_THREADS) k_b_tridiag(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        tridiag_mode<R, STAGE>((typename Cplx<R>::type*)I.specT, I.tp, local);
    });
}

// warp per mode, lines staged in the warp's shared-memory slice and the
// instance's alpha/gamma tables in the CTA's (dynamic smem:
// TRIW_WARPS x 2 x tri_ws_slots(largest nv) complex + 2 x as many real)
template <typename R>
__global__ void __launch_bounds__(32 * TRIW_WARPS) k_b_tridiag_w(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                                int n, int nsmax) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int w = threadIdx.x >> 5;
        const int k = local * TRIW_WARPS + w;
        const int ns = tri_ws_slots(I.tp.nv);
        C* sb = reinterpret_cast<C*>(smem_raw) + (size_t)w * 2 * ns;
        R* sal = reinterpret_cast<R*>(reinterpret_cast<C*>(smem_raw) + (size_t)TRIW_WARPS * 2 * nsmax);
        R* sga = sal + ns;
        tri_ws_stage_tables<R>(I.tp, sal, sga);
        if (k < I.tp.nmodes) tri_ws_stage_line<R>((const C*)I.specT, I.tp, k, sb, sb + ns);
        cp_async_commit();
        cp_async_wait0();
        __syncthreads();
        if (k < I.tp.nmodes) tridiag_warp_staged<R>((C*)I.specT, I.tp, k, sb, sb + ns, sal, sga);
    });
}

enum BDst { BD_B = 0, BD_V0 = 1, BD_VNEXT = 2 };

// ---- preconditioner, v-major spectrum layout (vv_pcj.cuh) ---------------------
// x-FFTs of RB rows per work item (RB set by the instance's M = 32..256)
template <typename TI, typename R>
__global__ void __launch_bounds__(FJ_THREADS) k_b_rfftj(const BInst* __restrict__ tab, const int* __restrict__ L, int n,
                                                        int from_tmp64) {
    for_work<F_ROWS>(tab, L, n, [&](const BInst& I, int local) {
        const TI* X = from_tmp64 ? (const TI*)I.tmp : (const TI*)I.tmpT;
        auto* spec = (typename Cplx<R>::type*)I.specT;
        switch (I.pp.M) {
            case 32: rfftj_block<TI, R, 32>(X, spec, I.pp, local); break;
            case 64: rfftj_block<TI, R, 64>(X, spec, I.pp, local); break;
            case 128: rfftj_block<TI, R, 128>(X, spec, I.pp, local); break;
            default: rfftj_block<TI, R, 256>(X, spec, I.pp, local); break;
        }
    });
}

// LU solves: one lane per x mode, 32 modes per work item (dynamic smem:
// the warp's ring, 64 TJ_RING complex)
template <typename R>
__global__ void __launch_bounds__(32) k_b_tridiagj(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int k = local * 32 + (int)threadIdx.x;
        tridiagj_lane<R>((C*)I.specT, (const C*)I.dinvJ, I.tp, k, reinterpret_cast<C*>(smem_raw));
    });
}

// ---- the Jacobian stencil's coefficient tables --------------------------------
// The coefficient form of the J1/J2/J4 bracket (the wide tiles' srow / scol):
// per column i (B1, bm, bp) from b = the x profile of h at i-2..i+2
// (periodic), per row j (A1, am, ap) from h0 at j-2..j+2 (zero outside the
// grid), computed in FP64 and stored in the GMRES precision as three arrays
// each (jcol = B1[nx] bm[nx] bp[nx], jrow = A1[nv] am[nv] ap[nv]).  The row
// table is fixed; the column table follows the x profile, which changes only
// in k_b_prologue and k_b_poisson, and k_b_poisson (which follows every
// prologue) rewrites it.
template <int SCHEME, typename T>
VV_DEV void jcoef_cols_s(const BInst& I, const double* sb) {
    T* jc = reinterpret_cast<T*>(I.jcol);
    for (int i = threadIdx.x; i < I.nx; i += blockDim.x) {
        const int l = i + 2;
        double bm, bq;
        Coef<SCHEME>::col(sb[l] - sb[l - 1], sb[l + 1] - sb[l], sb[l + 1] - sb[l - 1], sb[l] - sb[l - 2],
                          sb[l + 2] - sb[l], bm, bq);
        jc[i] = T(sb[l + 1] - sb[l - 1]);
        jc[I.nx + i] = T(bm);
        jc[2 * I.nx + i] = T(bq);
    }
}
template <int SCHEME, typename T>
VV_DEV void jcoef_rows_s(const BInst& I) {
    T* jr = reinterpret_cast<T*>(I.jrow);
    const double* h0 = I.bp.h0;
    const int nv = I.nv;
    for (int j = threadIdx.x; j < nv; j += blockDim.x) {
        double a[5];
#pragma unroll
        for (int d = 0; d < 5; ++d) {
            const int jj = j - 2 + d;
            a[d] = (jj >= 0 && jj < nv) ? h0[jj] : 0.0;
        }
        double am, aq;
        Coef<SCHEME>::row(a[2] - a[1], a[3] - a[2], a[3] - a[1], a[2] - a[0], a[4] - a[2], am, aq);
        jr[j] = T(a[3] - a[1]);
        jr[nv + j] = T(am);
        jr[2 * nv + j] = T(aq);
    }
}
constexpr int JCOEF_NXMAX = 512;   // the longest rows of the v-major layout (M <= 256)
// block-uniform: the column table from the current x profile of h (and the
// row table when `rows`), for the instance's scheme and precision
VV_DEV void jcoef_block(const BInst& I, bool rows) {
    if (!I.jcol || I.nx > JCOEF_NXMAX) return;
    __shared__ double sb[JCOEF_NXMAX + 4];
    for (int c = threadIdx.x; c < I.nx + 4; c += blockDim.x) {
        int xi = c - 2;
        if (xi < 0) xi += I.nx;
        else if (xi >= I.nx) xi -= I.nx;
        sb[c] = b_fac(I.bp, xi);
    }
    __syncthreads();
    switch (I.jscheme * 2 + I.jfp32) {
        case 2: jcoef_cols_s<1, double>(I, sb); if (rows) jcoef_rows_s<1, double>(I); break;
        case 3: jcoef_cols_s<1, float>(I, sb); if (rows) jcoef_rows_s<1, float>(I); break;
        case 4: jcoef_cols_s<2, double>(I, sb); if (rows) jcoef_rows_s<2, double>(I); break;
        case 5: jcoef_cols_s<2, float>(I, sb); if (rows) jcoef_rows_s<2, float>(I); break;
        case 8: jcoef_cols_s<4, double>(I, sb); if (rows) jcoef_rows_s<4, double>(I); break;
        default: jcoef_cols_s<4, float>(I, sb); if (rows) jcoef_rows_s<4, float>(I); break;
    }
    __syncthreads();
}

// both tables of every instance (one block per instance; at batch creation)
__global__ void __launch_bounds__(1024) k_b_jcoef(const BInst* __restrict__ tab, int n) {
    if ((int)blockIdx.x < n) jcoef_block(tab[blockIdx.x], true);
}

// ---- Jacobian stencil fused with the x-FFT of the preconditioner -------------
// The GMRES operator applies the Jacobian stencil and then P^-1, whose first
// stage is the real FFT of every v row: one kernel computes the stencil of
// its RB rows from a band of RB + 4 input rows staged in shared memory
// (periodic halo of 2 in x) and transforms them in place of the row loads,
// so the stencil's output never goes through HBM and one launch per Arnoldi
// step is saved.  The stencil is the wide-tile kernel's expression (the
// coefficient form of the J1/J2/J4 bracket with the point time derivative),
// its coefficients read from the instance's tables (jcoef_block).
//
// Shared memory: the FFT's twiddles, then two regions that the stencil and
// the FFT use in turn (each region's next user starts after a barrier that
// follows its last read):
//   region 1, the pass-1 buffer A or: the RB rows' coefficients (3 x RB T)
//     and the band ((RB + 4) x (nx + 8) T, row r at band[r * (nx + 8) + 4 + i]);
//   region 2, the pass-2 buffer B or the stencil's output (RB rows of
//     2 SB >= nx T: the row stride of B, which keeps the first pass's 8-byte
//     reads of two rows per half-warp on distinct banks where SB is padded).
// The stencil runs one column per thread down the RB rows with a rolling
// register window (6 shared loads per output, as the wide tiles).
__host__ __device__ constexpr size_t fjv_align(size_t b) { return (b + 15) & ~(size_t)15; }
__host__ __device__ constexpr size_t fjv_band(int M, int rb, size_t tsz) {
    return fjv_align((size_t)rb * 3 * tsz) + fjv_align((size_t)(rb + 4) * (2 * M + 8) * tsz);
}
template <int M> __host__ __device__ constexpr size_t fjv_region1(size_t tsz) {
    constexpr int P1 = FftJ<M>::P1, P2 = FftJ<M>::P2, RB = fj_rows(P2);
    const size_t a = fjv_align((size_t)RB * fj_sa(P1, P2) * 2 * tsz), band = fjv_band(M, RB, tsz);
    return a > band ? a : band;
}
template <int M> __host__ __device__ constexpr size_t fjv_smem_t(size_t tsz) {
    constexpr int P2 = FftJ<M>::P2, RB = fj_rows(P2);
    return fjv_align((size_t)M * 2 * tsz) + fjv_region1<M>(tsz) + (size_t)RB * fj_sb(M, P2) * 2 * tsz;
}
inline size_t fjv_smem_of(int M, size_t tsz) {
    switch (M) {
        case 32: return fjv_smem_t<32>(tsz);
        case 64: return fjv_smem_t<64>(tsz);
        case 128: return fjv_smem_t<128>(tsz);
        case 256: return fjv_smem_t<256>(tsz);
        default: return 0;
    }
}

template <int SCHEME, typename T, int M>
VV_DEV void jvp_rfftj_block(const T* __restrict__ X, typename Cplx<T>::type* __restrict__ spec, const PcParams& pp,
                            const BracketParams& bp, const T* __restrict__ jcol, const T* __restrict__ jrow,
                            int item) {
    using C = typename Cplx<T>::type;
    constexpr int P1 = FftJ<M>::P1, P2 = FftJ<M>::P2, RB = fj_rows(P2);
    constexpr int NX = 2 * M, BS = NX + 8, YS = 2 * fj_sb(M, P2), VN = 16 / (int)sizeof(T);
    static_assert(YS >= NX, "a stencil output row fits a pass-2 row");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    unsigned char* r1 = smem_raw + fjv_align((size_t)M * sizeof(C));
    C* A = reinterpret_cast<C*>(r1);
    C* B = reinterpret_cast<C*>(r1 + fjv_region1<M>(sizeof(T)));
    T* sy = reinterpret_cast<T*>(B);
    T* srow = reinterpret_cast<T*>(r1);   // A1, am, ap of the RB rows: srow[k * RB + r]
    T* band = reinterpret_cast<T*>(r1 + fjv_align((size_t)RB * 3 * sizeof(T)));
    const int nv = pp.nv, j0 = item * RB;
    const C* tw = reinterpret_cast<const C*>(pp.tw);
    for (int k = threadIdx.x; k < M; k += FJ_THREADS) stw[k] = tw[k];
    // band rows j0 - 2 .. j0 + RB + 1 (zeros outside the grid): the interior by
    // 16-byte cp.async, every copy in flight at once (rows outside the grid
    // copy 0 bytes from the base and zero-fill), then the halo
    for (int q = threadIdx.x; q < (RB + 4) * (NX / VN); q += FJ_THREADS) {
        const int rr = q / (NX / VN), v = q - rr * (NX / VN);
        const int jj = j0 - 2 + rr;
        const bool in = jj >= 0 && jj < nv;
        cp_async_16(band + rr * BS + 4 + v * VN, in ? X + (size_t)jj * NX + v * VN : X, in ? 16 : 0);
    }
    cp_async_commit();
    for (int q = threadIdx.x; q < (RB + 4) * 4; q += FJ_THREADS) {
        const int rr = q >> 2, h = q & 3;
        const int jj = j0 - 2 + rr;
        const int c = h < 2 ? 2 + h : NX + 2 + h;     // band columns of x = NX - 2, NX - 1, 0, 1
        const int xi = h < 2 ? NX - 2 + h : h - 2;
        band[rr * BS + c] = (jj >= 0 && jj < nv) ? X[(size_t)jj * NX + xi] : T(0);
    }
    for (int q = threadIdx.x; q < 3 * RB; q += FJ_THREADS) {
        const int k = q / RB, j = j0 + q - k * RB;
        srow[q] = j < nv ? jrow[k * nv + j] : T(0);
    }
    cp_async_wait0();
    __syncthreads();
    const T tscale = T(((SCHEME == 2) ? bp.f2 : bp.f1) * bp.factor);
    const T htinv = T(bp.ht_inv);
    // the wide tile's expression, column i per thread, rows r = 0..RB-1 through
    // a register window: column i rows r-2..r+2, columns i+-1 rows r-1..r+1
    for (int i = threadIdx.x; i < NX; i += FJ_THREADS) {
        const T* bc = band + 4 + i;    // row rr of the band at bc[rr * BS]
        const T B1 = jcol[i], bm = jcol[NX + i], bq = jcol[2 * NX + i];
        T w0 = bc[0], w1 = bc[BS], w2 = bc[2 * BS], w3 = bc[3 * BS];
        T m0 = bc[BS - 1], m1 = bc[2 * BS - 1], q0 = bc[BS + 1], q1 = bc[2 * BS + 1];
#pragma unroll 4
        for (int r = 0; r < RB; ++r) {
            const T w4 = bc[(r + 4) * BS];
            const T m2 = bc[(r + 3) * BS - 1], q2 = bc[(r + 3) * BS + 1];
            const int j = j0 + r;
            T y = htinv * w2;
            if (j >= 2 && j < nv - 2) {
                const T A1 = srow[r], am = srow[RB + r], ap = srow[2 * RB + r];
                T s = T(0);
                if (Coef<SCHEME>::cA1 != 0.0 || Coef<SCHEME>::cA2 != 0.0) {
                    T ax = T(0), bx = T(0);
                    if (Coef<SCHEME>::cA1 != 0.0) {
                        ax = T(Coef<SCHEME>::cA1) * (q1 - m1);
                        bx = T(Coef<SCHEME>::cB1) * (w3 - w1);
                    }
                    if (Coef<SCHEME>::cA2 != 0.0) {
                        ax += T(Coef<SCHEME>::cA2) * (bc[(r + 2) * BS + 2] - bc[(r + 2) * BS - 2]);
                        bx += T(Coef<SCHEME>::cB2) * (w4 - w0);
                    }
                    s = A1 * ax - B1 * bx;
                }
                s += am * (m0 - q0);
                s += ap * (m2 - q2);
                s += bm * (m0 - m2);
                s += bq * (q0 - q2);
                y += tscale * s;
            }
            sy[r * YS + i] = y;
            w0 = w1; w1 = w2; w2 = w3; w3 = w4;
            m0 = m1; m1 = m2; q0 = q1; q1 = q2;
        }
    }
    __syncthreads();
    using T2 = typename Pair<T>::type;
    rfftj_rows<T, M>(spec, pp, item, stw, A, B, [&](int r, int, int nn) {
        const T2 v = *reinterpret_cast<const T2*>(sy + r * YS + 2 * nn);
        return c_make<C>(v.x, v.y);
    });
}

// Jacobian stencil + x-FFT of every active instance's RB-row items:
// BS_X: J x; BS_VIT: J v_it, v_it = vsc[it] V[it] (as k_b_bracket).  The
// list is staged for up to FJV_STAGE instances (larger lists are searched in
// global memory), which keeps the static shared memory small enough for
// five blocks per SM beside the largest stencil band.
constexpr int FJV_STAGE = 256;
template <int SCHEME, int SRC, typename T>
__global__ void __launch_bounds__(FJ_THREADS, 5) k_b_jvp_rfftj(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                            int n) {
    for_work<F_ROWS, FJV_STAGE>(tab, L, n, [&](const BInst& I, int local) {
        BracketParams p = I.bp;
        p.xidx = nullptr;
        p.factor = 0.5;
        if (SRC == BS_VIT) {
            const double sc = I.ds->vsc[I.ds->it];
            p.factor *= sc;
            p.ht_inv *= sc;
        }
        const T* X = (SRC == BS_X) ? (const T*)I.xT : (const T*)I.V + (size_t)I.ds->it * I.ncell;
        auto* spec = (typename Cplx<T>::type*)I.specT;
        const T* jc = (const T*)I.jcol;
        const T* jr = (const T*)I.jrow;
        switch (I.pp.M) {
            case 32: jvp_rfftj_block<SCHEME, T, 32>(X, spec, I.pp, p, jc, jr, local); break;
            case 64: jvp_rfftj_block<SCHEME, T, 64>(X, spec, I.pp, p, jc, jr, local); break;
            case 128: jvp_rfftj_block<SCHEME, T, 128>(X, spec, I.pp, p, jc, jr, local); break;
            default: jvp_rfftj_block<SCHEME, T, 256>(X, spec, I.pp, p, jc, jr, local); break;
        }
    });
}

template <typename R, typename TO>
__global__ void __launch_bounds__(FJ_THREADS) k_b_irfftj(const BInst* __restrict__ tab, const int* __restrict__ L, int n,
                                                         int dst) {
    for_work<F_ROWS>(tab, L, n, [&](const BInst& I, int local) {
        TO* Y = (TO*)I.bT;
        if (dst == BD_V0) Y = (TO*)I.V;
        else if (dst == BD_VNEXT) Y = (TO*)I.V + (size_t)(I.ds->it + 1) * I.ncell;
        const auto* spec = (const typename Cplx<R>::type*)I.specT;
        switch (I.pp.M) {
            case 32: irfftj_block<R, TO, 32>(spec, Y, I.pp, local); break;
            case 64: irfftj_block<R, TO, 64>(spec, Y, I.pp, local); break;
            case 128: irfftj_block<R, TO, 128>(spec, Y, I.pp, local); break;
            default: irfftj_block<R, TO, 256>(spec, Y, I.pp, local); break;
        }
    });
}

// pad between the warps' slices of k_b_tridiagjs (complex slots)
constexpr int TRIJS_PAD = 8;
__host__ __device__ constexpr size_t tri_js_smem(int nvmax, size_t csz) {
    return (size_t)TRIW_WARPS * (2 * tri_ws_slots(nvmax) + TRIJS_PAD) * csz + 2 * (size_t)tri_ws_slots(nvmax) * (csz / 2);
}

// LU solves on the v-major layout by the staged warp solve: TRIW_WARPS
// consecutive modes per work item, one warp per mode; the CTA stages the
// modes' columns together (a row's TRIW_WARPS values are one 32-byte sector
// in FP32) into the warps' slices and writes the solutions back the same
// way.  The warps' slices are 2 ns + TRIJS_PAD complex apart: with 8-byte
// elements a staging instruction writes 8 rows x TRIW_WARPS modes, and a
// slice stride of 8 (mod 16) complex spreads the four modes of a row over
// both halves of the banks (two wavefronts, the minimum) where a multiple of
// 16 put them on one bank pair.  Dynamic smem: tri_js_smem.
template <typename R>
__global__ void __launch_bounds__(32 * TRIW_WARPS) k_b_tridiagjs(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                                int n, int nsmax) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int nv = I.tp.nv, nm = I.tp.nmodes;
        const int CH = (nv + 31) / 32;
        const int ns = tri_ws_slots(nv);
        const int w = threadIdx.x >> 5;
        const int k0 = local * TRIW_WARPS;
        const int ws = 2 * ns + TRIJS_PAD;   // complex slots per warp slice
        C* base = reinterpret_cast<C*>(smem_raw);
        R* sal = reinterpret_cast<R*>(base + (size_t)TRIW_WARPS * (2 * nsmax + TRIJS_PAD));
        R* sga = sal + ns;
        C* spec = (C*)I.specT;
        const C* dj = (const C*)I.dinvJ;
        const FastDiv dch((unsigned)CH);
        tri_ws_stage_tables<R>(I.tp, sal, sga);
        for (int t = threadIdx.x; t < nv * TRIW_WARPS; t += blockDim.x) {
            const int j = t / TRIW_WARPS, m = t % TRIW_WARPS;
            const int k = k0 + m;
            if (k < nm) {
                C* sb = base + (size_t)m * ws;
                const int q = j + (int)dch((unsigned)j);
                cp_async_elem(&sb[q], &spec[(size_t)j * nm + k]);
                cp_async_elem(&sb[ns + q], &dj[(size_t)j * nm + k]);
            }
        }
        cp_async_commit();
        cp_async_wait0();
        __syncthreads();
        if (k0 + w < nm) {
            C* sb = base + (size_t)w * ws;
            tri_ws_solve<R>(sb, sb + ns, sal, sga, reinterpret_cast<const C*>(I.tp.lambda)[k0 + w], nv);
        }
        __syncthreads();
        for (int t = threadIdx.x; t < nv * TRIW_WARPS; t += blockDim.x) {
            const int j = t / TRIW_WARPS, m = t % TRIW_WARPS;
            const int k = k0 + m;
            if (k < nm) spec[(size_t)j * nm + k] = base[(size_t)m * ws + j + (int)dch((unsigned)j)];
        }
    });
}

// dst[j*nm + k] = src[k*nv + j]: the v-major copy of a mode-major table
template <typename C>
__global__ void k_modes_to_vmajor(const C* __restrict__ src, C* __restrict__ dst, int nm, int nv) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nm * nv) return;
    const int j = (int)(i / nm), k = (int)(i % nm);
    dst[i] = src[(size_t)k * nv + j];
}

template <typename R, typename TO, bool FS>
__global__ void k_b_irfft(const BInst* __restrict__ tab, const int* __restrict__ L, int n, int dst) {
    for_work<F_ROWS>(tab, L, n, [&](const BInst& I, int local) {
        TO* Y = (TO*)I.bT;
        if (dst == BD_V0) Y = (TO*)I.V;
        else if (dst == BD_VNEXT) Y = (TO*)I.V + (size_t)(I.ds->it + 1) * I.ncell;
        const auto* spec = (const typename Cplx<R>::type*)I.specT;
        if (FS) {
            switch (I.pp.M) {
                case 32: irfft4_block<R, TO, 1>(spec, Y, I.pp, local); return;
                case 64: irfft4_block<R, TO, 2>(spec, Y, I.pp, local); return;
                case 128: irfft4_block<R, TO, 4>(spec, Y, I.pp, local); return;
                default: break;
            }
        }
        irfft_rows_block<R, TO>(spec, Y, I.pp, local);
    });
}

// ---- step prologue: make_history + update_previous (run_base.py:749-763) ----
__global__ void k_b_prologue(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        const int nb = I.vblk;
        for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < I.ncell; i += (size_t)nb * blockDim.x) {
            const double fv = I.f[i];
            I.fh[i] = fv;
            I.Fh[i] = fv;
        }
        const int nx = I.nx;
        const bool h2both = I.h2c && I.h2h;
        for (int i = bid * blockDim.x + threadIdx.x; i < nx; i += nb * blockDim.x) {
            const double h1 = I.h1c[i];
            I.h1h[i] = h1;
            if (h2both) I.h2h[i] = I.h2c[i];
            if (I.phih) I.phih[i] = I.phi[i];
            I.hxp[i] = h1;
            I.hxp[nx + i] = h1;
            I.hxp[2 * nx + i] = I.h2c ? I.h2c[i] : 0.0;
            I.hxp[3 * nx + i] = I.h2h ? I.h2h[i] : 0.0;
        }
    });
}

// ---- Poisson residual of the current moments (and H1p <- h1c) -------------
__global__ void __launch_bounds__(1024) k_b_poisson(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        for (int i = threadIdx.x; i < I.nx; i += blockDim.x) I.hxp[i] = I.h1c[i];
        __syncthreads();
        jcoef_block(I, false);   // the pass's Jacobian column coefficients from the new profile
        poisson_apply_cta(I.phi, I.n, nullptr, I.nx, I.po.hx2_inv, I.po.charge, 2, &I.ds->pnorm2, I.po.la0, I.po.la1,
                          I.po.la2, I.po.lden, I.po.ravg, I.po.ra0, I.po.ra1, I.po.ra2, I.po.rden);
    });
}

__global__ void k_b_pic_residual(const BInst* __restrict__ tab, const int* __restrict__ L, int n, int phase) {
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        pic_residual_warp(I.ds, I.part, I.cnt[F_TILE], phase);
    });
}

// ---- moments + Poisson + h1 -------------------------------------------------
__global__ void __launch_bounds__(MOM_TX * MOM_TY)
k_b_moments_partial(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_MOM>(tab, L, n, [&](const BInst& I, int local) {
        const int bx = local % I.mom_bx, s = local / I.mom_bx;
        moments_partial_block<double>(I.f, I.nx, I.nv, I.mom_seg, I.v, I.mom_part, bx, s);
    });
}

__global__ void __launch_bounds__(POIS_THREADS) k_b_moments_poisson(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                                   int n) {
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        moments_poisson_cta(I.mom_part, nullptr, I.n, I.u, I.e, I.a, I.phi, I.h1c, I.scal, I.po);
    });
}

// ---- Picard pass ------------------------------------------------------------
// start of the linear solve: x = 0, GMRES state reset; fl <- f (the iterate
// a rejected pass reverts to)
template <typename T>
__global__ void k_b_gm_init(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        gm_init_block<T>(I.ds, (T*)I.xT, I.ncell, bid, I.vblk);
        for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < I.ncell; i += (size_t)I.vblk * blockDim.x)
            I.fl[i] = I.f[i];
    });
}

template <typename T>
__global__ void k_b_pic_apply(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        pic_apply_block<T, double>(I.ds, (const T*)I.xT, I.f, I.ncell, bid, I.vblk);
    });
}

__global__ void k_b_revert(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < I.ncell; i += (size_t)I.vblk * blockDim.x)
            I.f[i] = I.fl[i];
    });
}

// ---- GMRES ------------------------------------------------------------------
// The batch reductions work on warp items: block item `bid` of an instance is
// eight warp items wi = 8 bid + warp, and warp item wi covers the contiguous
// cells [256 (wi + nwi s), 256 (wi + nwi s) + 256) (nwi = 8 vblk warp items,
// s = 0, 1, ...), read with 16-byte vector loads: lane l holds vectors
// l + 32 t, t < WV.  Each warp writes its own partial sum (no barrier, no
// atomic); a one-block finalize kernel per instance reduces them in a fixed
// order.
VV_DEV int wi_count(const BInst& I) { return 8 * I.vblk; }

constexpr int WCELLS = 256;   // cells of a warp item
template <typename T> VV_DEV constexpr int vec_n() { return Vec16<T>::n; }
// elements of a 16-byte vector as double
VV_DEV void vload(const float* p, double (&o)[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
VV_DEV void vload(const double* p, double (&o)[2]) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    o[0] = v.x; o[1] = v.y;
}
VV_DEV void vstore(float* p, const double (&o)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4((float)o[0], (float)o[1], (float)o[2], (float)o[3]);
}
VV_DEV void vstore(double* p, const double (&o)[2]) { *reinterpret_cast<double2*>(p) = make_double2(o[0], o[1]); }

// deterministic sum of part[0..np) by one warp with eight loads in flight per
// lane (lane l adds part[l + 32 j] into accumulator j mod 8; fixed tree after)
VV_DEV double warp_reduce_parts8(const double* __restrict__ part, int np) {
    const int lane = threadIdx.x & 31;
    double a[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = 0.0;
    int b = lane;
    for (; b + 7 * 32 < np; b += 8 * 32)
#pragma unroll
        for (int u = 0; u < 8; ++u) a[u] += __ldcg(part + b + 32 * u);
#pragma unroll
    for (int u = 0; u < 8; ++u)
        if (b + 32 * u < np) a[u] += __ldcg(part + b + 32 * u);
    return warp_sum(((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7])));
}

// deterministic sum of part[0..np) by the whole block: warp w sums the w-th
// of blockDim/32 consecutive ranges, warp 0 the warp sums in order; every
// thread returns the sum (block-uniform call)
VV_DEV double block_reduce_parts(const double* __restrict__ part, int np) {
    __shared__ double ws[32];
    const int nwarp = blockDim.x >> 5, wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = (np + nwarp - 1) / nwarp;
    const int lo = min(np, wid * per), hi = min(np, lo + per);
    const double t = warp_reduce_parts8(part + lo, hi - lo);
    if (lane == 0) ws[wid] = t;
    __syncthreads();
    if (wid == 0) {
        const double r = warp_sum(lane < nwarp ? ws[lane] : 0.0);
        if (lane == 0) ws[0] = r;
    }
    __syncthreads();
    const double r = ws[0];
    __syncthreads();   // ws read by every thread before a next call writes it
    return r;
}

// cycle head: V0 = b (first cycle) or b - P^-1 J x (restart, P^-1 J x in V0)
template <typename T>
__global__ void k_b_gm_head(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        const T* b = (const T*)I.bT;
        T* v = (T*)I.V;
        const bool first = I.ds->first != 0;
        for (size_t i = bid * (size_t)blockDim.x + threadIdx.x; i < I.ncell; i += (size_t)I.vblk * blockDim.x)
            v[i] = first ? b[i] : (T)(1.0 * (double)b[i] + (-1.0) * (double)v[i]);
    });
}

// ||V0||^2 per warp item
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) k_b_gm_cycle_p(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    constexpr int VN = vec_n<T>(), WV = WCELLS / (32 * VN);
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        const int lane = threadIdx.x & 31, nwi = wi_count(I), wi = bid * 8 + (threadIdx.x >> 5);
        const T* V0 = (const T*)I.V;
        double acc = 0.0;
        for (size_t base = (size_t)wi * WCELLS; base < I.ncell; base += (size_t)nwi * WCELLS) {
#pragma unroll
            for (int t = 0; t < WV; ++t) {
                const size_t i = base + (size_t)(lane + 32 * t) * VN;
                if (i < I.ncell) {
                    double v[VN];
                    vload(V0 + i, v);
#pragma unroll
                    for (int e = 0; e < VN; ++e) acc += v[e] * v[e];
                }
            }
        }
        acc = warp_sum(acc);
        if (lane == 0) I.wpart[wi] = acc;
    });
}

// cycle start: res, convergence test, scale, `active` (CTRL_THREADS per instance)
__global__ void __launch_bounds__(CTRL_THREADS, 1) k_b_gm_cycle_f(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                              int n) {
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        const double ss2 = block_reduce_parts(I.wpart, wi_count(I));
        if (threadIdx.x == 0) gm_cycle_state(I.ds, ss2);
    });
}


// <w, V_q>, q = 0..it, w = V[it+1], per warp item (column q of the partials)
// basis vectors whose 16-byte loads a lane issues together before using them
// (the loads of a chunk are independent; issuing them first keeps a chunk's
// worth of bytes in flight per warp instead of one vector's)
template <typename T> VV_DEV constexpr int gs_chunk() { return sizeof(T) == 4 ? 4 : 2; }
template <typename T>
VV_DEV void vload_raw(const T* p, typename Vec16<T>::type& o) { o = *reinterpret_cast<const typename Vec16<T>::type*>(p); }
VV_DEV void vexpand(const float4& v, double (&o)[4]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
VV_DEV void vexpand(const double2& v, double (&o)[2]) { o[0] = v.x; o[1] = v.y; }

// dynamic shared memory of the multi-dot: two stages of a thread's CK basis
// chunks (16-byte pieces, thread-interleaved)
template <typename T> __host__ __device__ constexpr size_t mdot_smem() {
    return (size_t)2 * gs_chunk<T>() * (WCELLS / (32 * (16 / sizeof(T)))) * 16 * RED_THREADS;
}

template <typename T>
__global__ void __launch_bounds__(RED_THREADS, 3) k_b_gm_mdot_p(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    static_assert(RED_THREADS == 256, "eight warp items per block item");
    constexpr int VN = vec_n<T>(), WV = WCELLS / (32 * VN), CK = gs_chunk<T>();
    using V16 = typename Vec16<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V16* sbuf = reinterpret_cast<V16*>(smem_raw);   // piece (stage, c, t) of this thread at [((stage CK + c) WV + t) RED_THREADS + tid]
    for_warp_work<F_VEC, true>(tab, L, n, [&](const BInst& I, int wi, int part, int split) {
        const int lane = threadIdx.x & 31, nwi = wi_count(I);
        const int it = I.ds->it, m = it + 1;
        const size_t nc = I.ncell;
        const T* V = (const T*)I.V;
        const T* w = V + (size_t)(it + 1) * nc;
        if ((size_t)nwi * WCELLS >= nc) {
            // one cell range per item: w in registers, the item's basis chunks
            // streamed through two shared-memory stages by cp.async (a chunk's
            // copies in flight while the previous one is summed); each thread
            // reads back only its own pieces
            const size_t base = (size_t)wi * WCELLS;
            V16 wr[WV];
#pragma unroll
            for (int t = 0; t < WV; ++t) {
                const size_t i = base + (size_t)(lane + 32 * t) * VN;
                if (i < nc) vload_raw(w + i, wr[t]);
                else wr[t] = V16{};
            }
            auto issue = [&](int q0, int stage) {
#pragma unroll
                for (int c = 0; c < CK; ++c)
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        const size_t i = base + (size_t)(lane + 32 * t) * VN;
                        const bool in = q0 + c < m && i < nc;
                        cp_async_16(&sbuf[((stage * CK + c) * WV + t) * RED_THREADS + threadIdx.x],
                                    in ? (const void*)(V + (size_t)(q0 + c) * nc + i) : (const void*)V, in ? 16 : 0);
                    }
                cp_async_commit();
            };
            const int step = split * CK;
            int q0 = part * CK;
            if (q0 < m) issue(q0, 0);
            if (q0 + step < m) issue(q0 + step, 1);
            for (int k = 0; q0 < m; q0 += step, ++k) {
                if (q0 + step < m) cp_async_wait1();   // the next chunk's group may still be in flight
                else cp_async_wait0();
                const int stage = k & 1;
                double acc[CK];
#pragma unroll
                for (int c = 0; c < CK; ++c) {
                    acc[c] = 0.0;
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        double wv[VN], v[VN];
                        vexpand(wr[t], wv);
                        vexpand(sbuf[((stage * CK + c) * WV + t) * RED_THREADS + threadIdx.x], v);
#pragma unroll
                        for (int e = 0; e < VN; ++e) acc[c] += wv[e] * v[e];
                    }
                }
                if (q0 + 2 * step < m) issue(q0 + 2 * step, stage);   // after this stage's reads
                const int cnt = min(CK, m - q0);
#pragma unroll
                for (int c = 0; c < CK; ++c) {
                    if (c < cnt) {
                        const double t = warp_sum(acc[c]);
                        if (lane == 0) I.wpart[(size_t)(q0 + c) * nwi + wi] = t;
                    }
                }
            }
            return;
        }
        // chunks of CK columns, dealt round-robin to the item's `split` warps;
        // every partial is one warp's fixed-order sum whatever the split
        for (int q0 = part * CK; q0 < m; q0 += split * CK) {
            double acc[CK];
#pragma unroll
            for (int c = 0; c < CK; ++c) acc[c] = 0.0;
            const int cnt = min(CK, m - q0);
            for (size_t base = (size_t)wi * WCELLS; base < nc; base += (size_t)nwi * WCELLS) {
                V16 wr[WV], vr[CK][WV];
#pragma unroll
                for (int t = 0; t < WV; ++t) {
                    const size_t i = base + (size_t)(lane + 32 * t) * VN;
                    if (i < nc) vload_raw(w + i, wr[t]);
                    else wr[t] = V16{};
                }
#pragma unroll
                for (int c = 0; c < CK; ++c)
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        const size_t i = base + (size_t)(lane + 32 * t) * VN;
                        if (c < cnt && i < nc) vload_raw(V + (size_t)(q0 + c) * nc + i, vr[c][t]);
                        else vr[c][t] = V16{};
                    }
#pragma unroll
                for (int c = 0; c < CK; ++c) {
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        double wv[VN], v[VN];
                        vexpand(wr[t], wv);
                        vexpand(vr[c][t], v);
#pragma unroll
                        for (int e = 0; e < VN; ++e) acc[c] += wv[e] * v[e];
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CK; ++c) {
                if (c < cnt) {
                    const double t = warp_sum(acc[c]);
                    if (lane == 0) I.wpart[(size_t)(q0 + c) * nwi + wi] = t;
                }
            }
        }
    });
}

// hcol_q = vsc_q <w, V_q> = <w, v_q> from the partials (one warp per column,
// CTRL_THREADS per instance: every column at once for restarts up to 31).
// A separate kernel: a last-block reduction inside the multi-dot needs a
// device-scope fence per work item, which waits for the item's stores.
__global__ void __launch_bounds__(CTRL_THREADS, 1) k_b_gm_mdot_f(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        DevState* s = I.ds;
        const int m = s->it + 1, nwi = wi_count(I);
        for (int q = threadIdx.x >> 5; q < m; q += blockDim.x >> 5) {
            const double t = warp_reduce_parts8(I.wpart + (size_t)q * nwi, nwi);
            if ((threadIdx.x & 31) == 0) s->hcol[q] = t * s->vsc[q];
        }
    });
}

// w += sum_q (-hcol_q vsc_q) V_q and ||w||^2 per warp item
template <typename T>
__global__ void __launch_bounds__(RED_THREADS, 3) k_b_gm_maxpy_p(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    constexpr int VN = vec_n<T>(), WV = WCELLS / (32 * VN), CK = gs_chunk<T>();
    using V16 = typename Vec16<T>::type;
    __shared__ double cf[MAX_RESTART + 2];
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        const DevState* s = I.ds;
        const int m = s->it + 1;
        for (int q = threadIdx.x; q < m; q += blockDim.x) cf[q] = -s->hcol[q] * s->vsc[q];
        __syncthreads();
        const int lane = threadIdx.x & 31, nwi = wi_count(I), wi = bid * 8 + (threadIdx.x >> 5);
        const size_t nc = I.ncell;
        T* V = (T*)I.V;
        T* w = V + (size_t)m * nc;
        double acc = 0.0;
        for (size_t base = (size_t)wi * WCELLS; base < nc; base += (size_t)nwi * WCELLS) {
            double wv[WV][VN];
#pragma unroll
            for (int t = 0; t < WV; ++t) {
                const size_t i = base + (size_t)(lane + 32 * t) * VN;
                if (i < nc) vload(w + i, wv[t]);
            }
            // the loads of CK basis vectors issued together, the updates in
            // the order q = 0, 1, .. (the same sums as one vector at a time)
            int q = 0;
            for (; q + CK <= m; q += CK) {
                V16 vr[CK][WV];
#pragma unroll
                for (int c = 0; c < CK; ++c)
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        const size_t i = base + (size_t)(lane + 32 * t) * VN;
                        if (i < nc) vload_raw(V + (size_t)(q + c) * nc + i, vr[c][t]);
                        else vr[c][t] = V16{};
                    }
#pragma unroll
                for (int c = 0; c < CK; ++c) {
                    const double cc = cf[q + c];
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        double v[VN];
                        vexpand(vr[c][t], v);
#pragma unroll
                        for (int e = 0; e < VN; ++e) wv[t][e] += cc * v[e];
                    }
                }
            }
            for (; q < m; ++q) {
                const T* vq = V + (size_t)q * nc;
                const double c = cf[q];
#pragma unroll
                for (int t = 0; t < WV; ++t) {
                    const size_t i = base + (size_t)(lane + 32 * t) * VN;
                    if (i < nc) {
                        double v[VN];
                        vload(vq + i, v);
#pragma unroll
                        for (int e = 0; e < VN; ++e) wv[t][e] += c * v[e];
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < WV; ++t) {
                const size_t i = base + (size_t)(lane + 32 * t) * VN;
                if (i < nc) {
                    vstore(w + i, wv[t]);
#pragma unroll
                    for (int e = 0; e < VN; ++e) acc += wv[t][e] * wv[t][e];
                }
            }
        }
        acc = warp_sum(acc);
        if (lane == 0) I.wpart[wi] = acc;
    });
}

// end of a cycle: triangular solve once per instance (coefficients into
// hcol, their count into pad), then the solution update x += sum nrs_q V_q
__global__ void k_b_gm_solve(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        if (threadIdx.x != 0) return;
        DevState* s = I.ds;
        int npad = 0, breakdown = 0;
        gm_backsolve(s, s->hcol, &npad, &breakdown);
        gm_finish_state(s, npad, breakdown);
    });
}

template <typename T>
__global__ void __launch_bounds__(RED_THREADS, 3) k_b_gm_update(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    __shared__ double nrs[MAX_RESTART + 1];
    for_work<F_VEC>(tab, L, n, [&](const BInst& I, int bid) {
        const DevState* s = I.ds;
        const int m = s->pad;
        for (int q = threadIdx.x; q < m; q += blockDim.x) nrs[q] = s->hcol[q] * s->vsc[q];
        __syncthreads();
        if (m <= 0) return;
        const T* V = (const T*)I.V;
        T* x = (T*)I.xT;
        // warp items of WCELLS cells with 16-byte loads; the loads of CK basis
        // vectors issued together, the sums in the order q = 0, 1, ..
        constexpr int VN = vec_n<T>(), WV = WCELLS / (32 * VN), CK = gs_chunk<T>();
        using V16 = typename Vec16<T>::type;
        const int lane = threadIdx.x & 31, nwi = wi_count(I), wi = bid * 8 + (threadIdx.x >> 5);
        const size_t nc = I.ncell;
        for (size_t base = (size_t)wi * WCELLS; base < nc; base += (size_t)nwi * WCELLS) {
            double xv[WV][VN];
#pragma unroll
            for (int t = 0; t < WV; ++t) {
                const size_t i = base + (size_t)(lane + 32 * t) * VN;
                if (i < nc) vload(x + i, xv[t]);
            }
            int q = 0;
            for (; q + CK <= m; q += CK) {
                V16 vr[CK][WV];
#pragma unroll
                for (int c = 0; c < CK; ++c)
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        const size_t i = base + (size_t)(lane + 32 * t) * VN;
                        if (i < nc) vload_raw(V + (size_t)(q + c) * nc + i, vr[c][t]);
                        else vr[c][t] = V16{};
                    }
#pragma unroll
                for (int c = 0; c < CK; ++c) {
                    const double cc = nrs[q + c];
#pragma unroll
                    for (int t = 0; t < WV; ++t) {
                        double v[VN];
                        vexpand(vr[c][t], v);
#pragma unroll
                        for (int e = 0; e < VN; ++e) xv[t][e] += cc * v[e];
                    }
                }
            }
            for (; q < m; ++q) {
                const double cc = nrs[q];
#pragma unroll
                for (int t = 0; t < WV; ++t) {
                    const size_t i = base + (size_t)(lane + 32 * t) * VN;
                    if (i < nc) {
                        double v[VN];
                        vload(V + (size_t)q * nc + i, v);
#pragma unroll
                        for (int e = 0; e < VN; ++e) xv[t][e] += cc * v[e];
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < WV; ++t) {
                const size_t i = base + (size_t)(lane + 32 * t) * VN;
                if (i < nc) vstore(x + i, xv[t]);
            }
        }
    });
}

// ---- control ----------------------------------------------------------------
// One block.  Applies the mask transitions of `op` to every instance,
// rebuilds the work lists of the masks it changed, and folds the result into
// the batch loop condition: handle (0 outside a graph) and *flag (read by
// the host-driven loop).  counts[op] counts the passes.
enum BCtrl { BC_PIC = 0, BC_GM_START = 1, BC_INNER = 2, BC_GM_FINISH = 3, BC_REVERT = 4, BC_ALL = 5 };
// words of the batch's counter array after the passes per BCtrl op: the
// Arnoldi control's dropped-instance count and grid counter, and the Arnoldi
// steps that found the inner list empty (the unrolled loop body's idle
// copies, for the launch count)
enum BCount { BN_DROPPED = 6, BN_DONE = 7, BN_IDLE = 8, BN_WORDS = 9 };


// rebuild list `l` from the per-instance membership test `in(q)` over the
// candidates src(0..cnt-1) (every instance, or the list's own members when
// the list only shrinks: the build then compacts it in place -- a chunk reads
// its candidates before the barrier that precedes its writes, and every
// write lands at or before the position it was read from): one pass of warp
// scans over (member, work items per family) and one scan of the warp totals
// per value (CTRL_THREADS threads)
template <typename In, typename Src>
__device__ void ctrl_build_from(const BInst* __restrict__ tab, int n, int cnt, int* __restrict__ lists, int l, In in,
                                Src src) {
    constexpr int NV = NFAM + 1, NW = CTRL_THREADS / 32;
    static_assert(NV <= NW, "one warp per scanned value");
    int* L = lists + (size_t)l * blist_words(n);
    int* ids = L + 1 + NFAM;
    int* pre = ids + n;
    __shared__ int wsum[NV][NW];
    __shared__ int wtot[NV];
    __shared__ int carry[NV];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x < NV) carry[threadIdx.x] = 0;
    __syncthreads();
    for (int i0 = 0; i0 < cnt; i0 += CTRL_THREADS) {
        const int i = i0 + threadIdx.x;
        const int q = i < cnt ? src(i) : 0;
        const bool on = i < cnt && in(q);
        int v[NV], inc[NV];
        v[0] = on ? 1 : 0;
#pragma unroll
        for (int f = 0; f < NFAM; ++f) v[1 + f] = on ? tab[q].cnt[f] : 0;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            inc[k] = v[k];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(0xffffffffu, inc[k], d);
                if (lane >= d) inc[k] += o;
            }
            if (lane == 31) wsum[k][wid] = inc[k];
        }
        __syncthreads();
        if (wid < NV) {   // warp k: exclusive scan of the warp totals of value k
            const int x = wsum[wid][lane];
            int y = x;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(0xffffffffu, y, d);
                if (lane >= d) y += o;
            }
            wsum[wid][lane] = y - x;
            if (lane == 31) wtot[wid] = y;
        }
        __syncthreads();
        if (on) {
            const int pos = carry[0] + wsum[0][wid] + inc[0] - 1;
            ids[pos] = q;
#pragma unroll
            for (int f = 0; f < NFAM; ++f)
                pre[(size_t)f * (n + 1) + pos] = carry[1 + f] + wsum[1 + f][wid] + inc[1 + f] - v[1 + f];
        }
        __syncthreads();
        if (threadIdx.x < NV) carry[threadIdx.x] += wtot[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        L[0] = carry[0];
        for (int f = 0; f < NFAM; ++f) {
            L[1 + f] = carry[1 + f];
            pre[(size_t)f * (n + 1) + carry[0]] = carry[1 + f];
        }
    }
    __syncthreads();
}

template <typename In>
__device__ void ctrl_build(const BInst* __restrict__ tab, int n, int* __restrict__ lists, int l, In in) {
    ctrl_build_from(tab, n, n, lists, l, in, [](int i) { return i; });
}

// the control step by one block of CTRL_THREADS threads
__device__ void ctrl_run(const BInst* __restrict__ tab, int n, int op, unsigned long long handle, int* __restrict__ flag,
                         unsigned int* __restrict__ counts, int* __restrict__ lists) {
    // mask transitions (each instance by one thread)
    for (int q = threadIdx.x; q < n; q += CTRL_THREADS) {
        DevState* s = tab[q].ds;
        if (op == BC_GM_START) s->gm_outer = s->pic_active != 0 ? 1 : 0;
        else if (op == BC_GM_FINISH && s->gm_outer) s->gm_outer = s->reason == R_ITERATING ? 1 : 0;
    }
    __syncthreads();
    int l = L_PIC;
    switch (op) {
        case BC_ALL: l = L_ALL; ctrl_build(tab, n, lists, L_ALL, [&](int) { return true; }); break;
        case BC_PIC: ctrl_build(tab, n, lists, L_PIC, [&](int q) { return tab[q].ds->pic_active != 0; }); break;
        case BC_GM_START:
        case BC_GM_FINISH:
            l = L_GM;
            ctrl_build(tab, n, lists, L_GM, [&](int q) { return tab[q].ds->gm_outer != 0; });
            ctrl_build(tab, n, lists, L_GMR, [&](int q) {
                const DevState* s = tab[q].ds;
                return s->gm_outer != 0 && s->first == 0;
            });
            break;
        case BC_INNER:
            l = L_INNER;
            ctrl_build(tab, n, lists, L_INNER, [&](int q) {
                const DevState* s = tab[q].ds;
                return s->gm_outer != 0 && s->active != 0;
            });
            break;
        default:
            l = L_REVERT;
            ctrl_build(tab, n, lists, L_REVERT, [&](int q) { return tab[q].ds->pic_revert != 0; });
            break;
    }
    if (threadIdx.x == 0) {
        const int any = lists[(size_t)l * blist_words(n)] > 0 ? 1 : 0;
        set_cond(handle, any ? 1u : 0u);
        if (flag) *flag = any;
        if (any && counts) counts[op] += 1u;
    }
}

__global__ void __launch_bounds__(CTRL_THREADS)
k_b_ctrl(const BInst* __restrict__ tab, int n, int op, unsigned long long handle, int* __restrict__ flag,
         unsigned int* __restrict__ counts, int* __restrict__ lists) {
    ctrl_run(tab, n, op, handle, flag, counts, lists);
}

// list l of the instances q with member[q] != 0 (one block of CTRL_THREADS)
__global__ void __launch_bounds__(CTRL_THREADS)
k_b_build_subset(const BInst* __restrict__ tab, int n, int* __restrict__ lists, int l, const int* __restrict__ member) {
    ctrl_build(tab, n, lists, l, [&](int q) { return member[q] != 0; });
}

// End of an Arnoldi step: ||w|| and the Arnoldi bookkeeping of every
// instance of list L (one block per instance; vsc of the new vector), then the
// BC_INNER control step by the block that finishes last (`done`: a grid
// counter, zero on entry and on exit; `dropped`: the instances that left the
// inner loop in this step, zero on entry and on exit).  The blocks only write instance
// state before the counter, so the device-scope fence is short.
__global__ void __launch_bounds__(CTRL_THREADS)
k_b_arnoldi_ctrl(const BInst* __restrict__ tab, const int* __restrict__ L, int n, unsigned long long handle,
                 int* __restrict__ flag, unsigned int* __restrict__ counts, int* __restrict__ lists,
                 unsigned int* __restrict__ done, unsigned int* __restrict__ dropped) {
    __shared__ double s_h[MAX_RESTART + 2], s_c[MAX_RESTART + 1], s_s[MAX_RESTART + 1];
    __shared__ unsigned int s_dropped;
    // the blocks that get an item take part in the grid counter (block 0
    // always, for an empty list); read before any block arrives, so before
    // the last one compacts the list in place
    const int nb = max(1, min((int)gridDim.x, L[1 + F_INST]));
    for_work<F_INST>(tab, L, n, [&](const BInst& I, int) {
        DevState* s = I.ds;
        const int it = s->it;
        for (int j = threadIdx.x; j <= it; j += blockDim.x) {
            s_h[j] = s->hcol[j];
            if (j < it) {
                s_c[j] = s->cc[j];
                s_s[j] = s->ss[j];
            }
        }
        const double ss2 = block_reduce_parts(I.wpart, wi_count(I));   // its barriers publish the copies
        if (threadIdx.x == 0) {
            gm_arnoldi(s, sqrt(ss2), s_h, s_c, s_s);
            if (!s->active) atomicAdd(dropped, 1u);   // before this block's arrival at the counter
        }
    });
    // one participating block (an instance or none left: the lockstep tail)
    // is the last by itself and skips the grid counter's fence and atomic;
    // its own state writes are ordered by the barrier that ended its item
    if ((int)blockIdx.x >= nb || (nb > 1 && !last_block(done, nb))) return;
    // the inner loop only drops instances: compact the current L_INNER in
    // place instead of scanning the whole table (a tail pass with a few
    // instances left reads a few states, not n), and only when an instance
    // left it in this step
    int* LI = lists + (size_t)L_INNER * blist_words(n);
    const int cnt = LI[0];
    const int* ids = LI + 1 + NFAM;
    if (threadIdx.x == 0) {
        s_dropped = atomicExch(dropped, 0u);
        if (cnt == 0 && counts) counts[BN_IDLE] += 1u;   // an idle copy of the step
    }
    __syncthreads();
    if (s_dropped)
        ctrl_build_from(tab, n, cnt, lists, L_INNER, [&](int q) {
            const DevState* s = tab[q].ds;
            return s->gm_outer != 0 && s->active != 0;
        }, [&](int i) { return ids[i]; });
    if (threadIdx.x == 0) {
        const int any = LI[0] > 0 ? 1 : 0;
        set_cond(handle, any ? 1u : 0u);
        if (flag) *flag = any;
        if (any && counts) counts[BC_INNER] += 1u;
    }
}

// set the Arnoldi index of every instance (kernel timing)
__global__ void k_b_set_it(const BInst* __restrict__ tab, int n, int it) {
    for (int q = threadIdx.x; q < n; q += blockDim.x) tab[q].ds->it = it;
}



// copy the first `words` 32-bit words of every instance's state into out[n][words]
__global__ void k_b_gather_states(const BInst* __restrict__ tab, int words, unsigned int* __restrict__ out) {
    const unsigned int* src = reinterpret_cast<const unsigned int*>(tab[blockIdx.x].ds);
    unsigned int* dst = out + (size_t)blockIdx.x * words;
    for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
}

// ---- LU solves on the v-major layout, W warps per mode ------------------------
// k_b_tridiagjs with each mode's line split over W warps instead of one: lane
// l of sub-warp s owns the chunk c = 32 s + l of CH = ceil(nv / 32 W) rows, so
// the sequential chunk sweeps are W times shorter and a CTA of 4 modes runs
// 4 W warps on the same staged lines.  The chunks' affine maps are joined by
// a warp scan and then across the W sub-warps through shared memory.  Slot
// of row r: r + r / CH (one pad per chunk; CH + 1 odd for power-of-two lines,
// so the chunk-strided accesses are conflict-free).
__host__ __device__ constexpr int tri_jm_slots(int nv, int W) { return nv + 32 * W; }
__host__ __device__ constexpr size_t tri_jm_smem(int nvmax, size_t csz, int W) {
    return (size_t)TRIW_WARPS * (2 * tri_jm_slots(nvmax, W) + TRIJS_PAD) * csz +
           2 * (size_t)tri_jm_slots(nvmax, W) * (csz / 2);
}

// inclusive warp scan of affine maps in `forward` lane order; *ex gets the
// exclusive prefix (identity for the first lane)
template <typename C>
__device__ __forceinline__ Aff<C> warp_scan_aff_ie(Aff<C> a, bool forward, Aff<C>* ex) {
    const int lane = threadIdx.x & 31;
    const int pos = forward ? lane : 31 - lane;
    Aff<C> inc = a;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Aff<C> o = shfl_aff(inc, d, forward);
        if (pos >= d) inc = aff_combine(o, inc);
    }
    const Aff<C> prev = shfl_aff(inc, 1, forward);
    if (pos > 0) *ex = prev;
    else {
        ex->P = c_make<C>(1.0, 0.0);
        ex->Q = c_make<C>(0.0, 0.0);
    }
    return inc;
}

template <typename R, int W>
__global__ void __launch_bounds__(32 * TRIW_WARPS * W) k_b_tridiagjm(const BInst* __restrict__ tab,
                                                                    const int* __restrict__ L, int n, int nsmax) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Aff<C> tot[2][TRIW_WARPS][W];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int nv = I.tp.nv, nm = I.tp.nmodes;
        const int CH = (nv + 32 * W - 1) / (32 * W);
        const int ns = tri_jm_slots(nv, W);
        const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int m = wid / W, sw = wid % W;        // mode of the CTA's item, sub-warp within the mode
        const int k0 = local * TRIW_WARPS;
        const int ws = 2 * ns + TRIJS_PAD;
        C* base = reinterpret_cast<C*>(smem_raw);
        R* sal = reinterpret_cast<R*>(base + (size_t)TRIW_WARPS * (2 * tri_jm_slots(nsmax, W) + TRIJS_PAD));
        R* sga = sal + ns;
        C* spec = (C*)I.specT;
        const C* dj = (const C*)I.dinvJ;
        const FastDiv dch((unsigned)CH);
        {
            const R* al = reinterpret_cast<const R*>(I.tp.alpha);
            const R* ga = reinterpret_cast<const R*>(I.tp.gamma);
            for (int r = threadIdx.x; r < nv; r += blockDim.x) {
                const int q = r + (int)dch((unsigned)r);
                cp_async_elem(&sal[q], &al[r]);
                cp_async_elem(&sga[q], &ga[r]);
            }
        }
        for (int t = threadIdx.x; t < nv * TRIW_WARPS; t += blockDim.x) {
            const int j = t / TRIW_WARPS, mm = t % TRIW_WARPS;
            const int k = k0 + mm;
            if (k < nm) {
                C* sb = base + (size_t)mm * ws;
                const int q = j + (int)dch((unsigned)j);
                cp_async_elem(&sb[q], &spec[(size_t)j * nm + k]);
                cp_async_elem(&sb[ns + q], &dj[(size_t)j * nm + k]);
            }
        }
        cp_async_commit();
        cp_async_wait0();
        __syncthreads();
        const bool on = k0 + m < nm;
        C* sb = base + (size_t)m * ws;
        const C* sd = sb + ns;
        const C lam = on ? reinterpret_cast<const C*>(I.tp.lambda)[k0 + m] : c_make<C>(0.0, 0.0);
        const int chunk = sw * 32 + lane;
        const int r0 = chunk * CH;
        const int r1 = min(r0 + CH, nv);
        const int q0 = chunk * (CH + 1);
        // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
        Aff<C> a;
        a.P = c_make<C>(1.0, 0.0);
        a.Q = c_make<C>(0.0, 0.0);
        if (on)
            for (int r = r0, q = q0; r < r1; ++r, ++q) {
                Aff<C> mp;
                if (r == 0) mp.P = c_make<C>(0.0, 0.0);
                else {
                    const C dprev = sd[(r == r0) ? q - 2 : q - 1];   // row r0-1 sits before the previous pad slot
                    const C l = c_mul(c_rmul(lam, sal[q]), dprev);
                    mp.P = c_make<C>(-l.x, -l.y);
                }
                mp.Q = sb[q];
                a = aff_combine(a, mp);
            }
        Aff<C> ex;
        Aff<C> inc = warp_scan_aff_ie<C>(a, true, &ex);
        if (lane == 31) tot[0][m][sw] = inc;
        __syncthreads();
        Aff<C> pre;
        pre.P = c_make<C>(1.0, 0.0);
        pre.Q = c_make<C>(0.0, 0.0);
        for (int u = 0; u < sw; ++u) pre = aff_combine(pre, tot[0][m][u]);
        C y = aff_combine(pre, ex).Q;
        if (on)
            for (int r = r0, q = q0; r < r1; ++r, ++q) {
                const C b = sb[q];
                if (r == 0) y = b;
                else {
                    const C dprev = sd[(r == r0) ? q - 2 : q - 1];
                    const C l = c_mul(c_rmul(lam, sal[q]), dprev);
                    y = c_sub(b, c_mul(l, y));
                }
                sb[q] = y;
            }
        // backward: x_r = U_r^-1 (y_r - c_r x_{r+1}) == mu_r + nu_r x_{r+1}; each lane reads its own chunk only
        a.P = c_make<C>(1.0, 0.0);
        a.Q = c_make<C>(0.0, 0.0);
        if (on)
            for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
                Aff<C> mp;
                const C d = sd[q];
                mp.Q = c_mul(d, sb[q]);
                if (r == nv - 1) mp.P = c_make<C>(0.0, 0.0);
                else {
                    const C nu = c_mul(d, c_rmul(lam, sga[q]));
                    mp.P = c_make<C>(-nu.x, -nu.y);
                }
                a = aff_combine(a, mp);
            }
        inc = warp_scan_aff_ie<C>(a, false, &ex);
        if (lane == 0) tot[1][m][sw] = inc;
        __syncthreads();
        pre.P = c_make<C>(1.0, 0.0);
        pre.Q = c_make<C>(0.0, 0.0);
        for (int u = W - 1; u > sw; --u) pre = aff_combine(pre, tot[1][m][u]);
        C x = aff_combine(pre, ex).Q;
        if (on)
            for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
                const C d = sd[q];
                if (r == nv - 1) x = c_mul(d, sb[q]);
                else x = c_mul(d, c_sub(sb[q], c_mul(c_rmul(lam, sga[q]), x)));
                sb[q] = x;
            }
        __syncthreads();
        for (int t = threadIdx.x; t < nv * TRIW_WARPS; t += blockDim.x) {
            const int j = t / TRIW_WARPS, mm = t % TRIW_WARPS;
            const int k = k0 + mm;
            if (k < nm) spec[(size_t)j * nm + k] = base[(size_t)mm * ws + j + (int)dch((unsigned)j)];
        }
        __syncthreads();
    });
}

// ---- LU solves on the v-major layout, lanes per mode set by the line length ----
// The chunked solves cost a warp scan (and a sub-warp combine) per chunk on
// top of the per-row work, so short lines want fewer, longer chunks: each
// mode gets LPM = 8..64 lanes, enough for chunks of about TJV_CH rows, and a
// CTA of TJV_THREADS threads solves G = TJV_THREADS / (4 LPM) consecutive
// 4-mode items of one instance at once (G items x 4 modes x nv rows staged:
// about the same shared memory for every nv).  The lanes of a mode scan
// their chunks' affine maps with width-LPM warp shuffles (LPM <= 32) or a
// warp scan and a combine of the two sub-warps (LPM = 64).  The alpha/gamma
// tables are read through L1 in the chunk order.
constexpr int TJV_THREADS = 256, TJV_CH = 16;
__host__ __device__ constexpr int tjv_lpm(int nv) {
    return nv <= 8 * TJV_CH ? 8 : nv <= 16 * TJV_CH ? 16 : nv <= 32 * TJV_CH ? 32 : 64;
}
__host__ __device__ constexpr int tjv_group(int nv) { return TJV_THREADS / (TRIW_WARPS * tjv_lpm(nv)); }
__host__ __device__ constexpr int tjv_slots(int nv) { return nv + tjv_lpm(nv); }
// complex slots of one group's 4-mode item: 4 x (line + LU reciprocals) + pad
__host__ __device__ constexpr int tjv_item_slots(int nv) { return TRIW_WARPS * (2 * tjv_slots(nv) + TRIJS_PAD); }
__host__ __device__ constexpr size_t tjv_smem_of(int nv, size_t csz) {
    return (size_t)tjv_group(nv) * tjv_item_slots(nv) * csz;
}

template <typename C>
__device__ __forceinline__ C shfl_w(C v, int d, bool up, int width) {
    C r;
    r.x = up ? __shfl_up_sync(0xffffffffu, v.x, d, width) : __shfl_down_sync(0xffffffffu, v.x, d, width);
    r.y = up ? __shfl_up_sync(0xffffffffu, v.y, d, width) : __shfl_down_sync(0xffffffffu, v.y, d, width);
    return r;
}
// inclusive scan of affine maps over segments of `width` lanes in `forward`
// order; *ex gets the exclusive prefix (identity for a segment's first lane)
template <typename C>
__device__ __forceinline__ Aff<C> seg_scan_aff(Aff<C> a, bool forward, int width, Aff<C>* ex) {
    const int l = threadIdx.x & (width - 1);
    const int pos = forward ? l : width - 1 - l;
    Aff<C> inc = a;
    for (int d = 1; d < width; d <<= 1) {
        Aff<C> o;
        o.P = shfl_w(inc.P, d, forward, width);
        o.Q = shfl_w(inc.Q, d, forward, width);
        if (pos >= d) inc = aff_combine(o, inc);
    }
    Aff<C> prev;
    prev.P = shfl_w(inc.P, 1, forward, width);
    prev.Q = shfl_w(inc.Q, 1, forward, width);
    if (pos > 0) *ex = prev;
    else {
        ex->P = c_make<C>(1.0, 0.0);
        ex->Q = c_make<C>(0.0, 0.0);
    }
    return inc;
}

template <typename R>
__global__ void __launch_bounds__(TJV_THREADS) k_b_tridiagjv(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                             int n) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Aff<C> tot[2][TJV_THREADS / 32];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int nv = I.tp.nv, nm = I.tp.nmodes;
        const int lpm = tjv_lpm(nv), G = tjv_group(nv);
        const int CH = (nv + lpm - 1) / lpm;
        const int ns = tjv_slots(nv), is = tjv_item_slots(nv);
        const int ws = 2 * ns + TRIJS_PAD;
        const int tid = threadIdx.x;
        const int gi = tid / (TRIW_WARPS * lpm);               // item of the group
        const int m = (tid / lpm) % TRIW_WARPS;                 // mode within the item
        const int l = tid % lpm;                                // lane within the mode
        const int kbase = local * G * TRIW_WARPS;               // first mode of the CTA's group
        C* base = reinterpret_cast<C*>(smem_raw);
        C* spec = (C*)I.specT;
        const C* dj = (const C*)I.dinvJ;
        const R* al = reinterpret_cast<const R*>(I.tp.alpha);
        const R* ga = reinterpret_cast<const R*>(I.tp.gamma);
        const FastDiv dch((unsigned)CH);
        // stage G items: row j of an item's 4 modes is one 32-byte sector
        // (cols = 4 G is a power of two: shifts, no runtime division)
        const int cols = G * TRIW_WARPS;
        const int lc = __ffs(cols) - 1;
        for (int t = tid; t < nv * cols; t += TJV_THREADS) {
            const int j = t >> lc, c = t & (cols - 1);
            const int k = kbase + c;
            if (k < nm) {
                C* sb = base + (size_t)(c / TRIW_WARPS) * is + (size_t)(c % TRIW_WARPS) * ws;
                const int q = j + (int)dch((unsigned)j);
                cp_async_elem(&sb[q], &spec[(size_t)j * nm + k]);
                cp_async_elem(&sb[ns + q], &dj[(size_t)j * nm + k]);
            }
        }
        cp_async_commit();
        cp_async_wait0();
        __syncthreads();
        const int k = kbase + gi * TRIW_WARPS + m;
        const bool on = gi < G && k < nm;
        C* sb = base + (size_t)gi * is + (size_t)m * ws;
        const C* sd = sb + ns;
        const C lam = on ? reinterpret_cast<const C*>(I.tp.lambda)[k] : c_make<C>(0.0, 0.0);
        const int r0 = l * CH;
        const int r1 = min(r0 + CH, nv);
        const int q0 = l * (CH + 1);
        const int width = lpm < 32 ? lpm : 32;
        const int wid = tid >> 5;
        const bool two = lpm > 32;                              // two sub-warps per mode
        // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
        Aff<C> a;
        a.P = c_make<C>(1.0, 0.0);
        a.Q = c_make<C>(0.0, 0.0);
        if (on)
            for (int r = r0, q = q0; r < r1; ++r, ++q) {
                Aff<C> mp;
                if (r == 0) mp.P = c_make<C>(0.0, 0.0);
                else {
                    const C dprev = sd[(r == r0) ? q - 2 : q - 1];
                    const C lr = c_mul(c_rmul(lam, __ldg(al + r)), dprev);
                    mp.P = c_make<C>(-lr.x, -lr.y);
                }
                mp.Q = sb[q];
                a = aff_combine(a, mp);
            }
        Aff<C> ex;
        Aff<C> inc = seg_scan_aff<C>(a, true, width, &ex);
        if (two) {
            if ((tid & 31) == 31) tot[0][wid] = inc;
            __syncthreads();
            if (l >= 32) ex = aff_combine(tot[0][wid - 1], ex);
        }
        C y = ex.Q;
        if (on)
            for (int r = r0, q = q0; r < r1; ++r, ++q) {
                const C b = sb[q];
                if (r == 0) y = b;
                else {
                    const C dprev = sd[(r == r0) ? q - 2 : q - 1];
                    const C lr = c_mul(c_rmul(lam, __ldg(al + r)), dprev);
                    y = c_sub(b, c_mul(lr, y));
                }
                sb[q] = y;
            }
        // backward: x_r = U_r^-1 (y_r - c_r x_{r+1}) == mu_r + nu_r x_{r+1}
        a.P = c_make<C>(1.0, 0.0);
        a.Q = c_make<C>(0.0, 0.0);
        if (on)
            for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
                Aff<C> mp;
                const C d = sd[q];
                mp.Q = c_mul(d, sb[q]);
                if (r == nv - 1) mp.P = c_make<C>(0.0, 0.0);
                else {
                    const C nu = c_mul(d, c_rmul(lam, __ldg(ga + r)));
                    mp.P = c_make<C>(-nu.x, -nu.y);
                }
                a = aff_combine(a, mp);
            }
        inc = seg_scan_aff<C>(a, false, width, &ex);
        if (two) {
            if ((tid & 31) == 0) tot[1][wid] = inc;
            __syncthreads();
            if (l < 32) ex = aff_combine(tot[1][wid + 1], ex);
        }
        C x = ex.Q;
        if (on)
            for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
                const C d = sd[q];
                if (r == nv - 1) x = c_mul(d, sb[q]);
                else x = c_mul(d, c_sub(sb[q], c_mul(c_rmul(lam, __ldg(ga + r)), x)));
                sb[q] = x;
            }
        __syncthreads();
        for (int t = tid; t < nv * cols; t += TJV_THREADS) {
            const int j = t >> lc, c = t & (cols - 1);
            const int kk = kbase + c;
            if (kk < nm)
                spec[(size_t)j * nm + kk] =
                    base[(size_t)(c / TRIW_WARPS) * is + (size_t)(c % TRIW_WARPS) * ws + j + (int)dch((unsigned)j)];
        }
        __syncthreads();
    });
}

// ---- LU solves on the v-major layout: lane per mode, threads per row chunk ----
// A CTA takes TJC_MG consecutive x modes of one instance and splits their
// lines into TJC_NC chunks of CH = ceil(nv / TJC_NC) rows: thread (c, m)
// sweeps rows [c CH, (c+1) CH) of mode m.  The TJC_MG lanes of a chunk read
// one row of TJC_MG consecutive modes (64 contiguous bytes in FP32) straight
// from the spectrum and the LU reciprocals in global memory -- no staging, no
// pad slots -- and the chunk's affine maps are joined per mode by one warp
// scan over the TJC_NC chunks (a warp per mode, through shared memory).  The
// replay sweeps re-read their rows (L1/L2) and write y, then x, in place.
constexpr int TJC_MG = 8, TJC_NC = 32, TJC_THREADS = TJC_MG * TJC_NC;

template <typename R>
__global__ void __launch_bounds__(TJC_THREADS) k_b_tridiagjc(const BInst* __restrict__ tab, const int* __restrict__ L,
                                                             int n) {
    using C = typename Cplx<R>::type;
    static_assert(TJC_NC == 32 && TJC_MG <= TJC_THREADS / 32, "one warp scans the chunks of one mode");
    __shared__ Aff<C> tot[TJC_NC][TJC_MG];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int nv = I.tp.nv, nm = I.tp.nmodes;
        const int CH = (nv + TJC_NC - 1) / TJC_NC;
        const int tid = threadIdx.x;
        const int m = tid % TJC_MG, c = tid / TJC_MG;
        const int k = local * TJC_MG + m;
        const bool on = k < nm;
        C* col = (C*)I.specT + k;                         // row r at col[r * nm]
        const C* dcol = (const C*)I.dinvJ + k;
        const R* al = reinterpret_cast<const R*>(I.tp.alpha);
        const R* ga = reinterpret_cast<const R*>(I.tp.gamma);
        const C lam = on ? reinterpret_cast<const C*>(I.tp.lambda)[k] : c_make<C>(0.0, 0.0);
        const int r0 = c * CH, r1 = min(r0 + CH, nv);
        const size_t ld = (size_t)nm;
        // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
        Aff<C> a;
        a.P = c_make<C>(1.0, 0.0);
        a.Q = c_make<C>(0.0, 0.0);
        if (on) {
#pragma unroll 4
            for (int r = r0; r < r1; ++r) {
                Aff<C> mp;
                mp.Q = col[r * ld];
                if (r == 0) mp.P = c_make<C>(0.0, 0.0);
                else {
                    const C lr = c_mul(c_rmul(lam, __ldg(al + r)), dcol[(r - 1) * ld]);
                    mp.P = c_make<C>(-lr.x, -lr.y);
                }
                a = aff_combine(a, mp);
            }
        }
        tot[c][m] = a;
        __syncthreads();
        if (tid < TJC_MG * 32) {                           // warp w scans the chunks of mode w
            const int w = tid >> 5, lane = tid & 31;
            Aff<C> ex;
            warp_scan_aff_ie<C>(tot[lane][w], true, &ex);
            __syncwarp();
            tot[lane][w] = ex;
        }
        __syncthreads();
        C y = tot[c][m].Q;
        if (on) {
#pragma unroll 4
            for (int r = r0; r < r1; ++r) {
                const C b = col[r * ld];
                if (r == 0) y = b;
                else {
                    const C lr = c_mul(c_rmul(lam, __ldg(al + r)), dcol[(r - 1) * ld]);
                    y = c_sub(b, c_mul(lr, y));
                }
                col[r * ld] = y;
            }
        }
        __syncthreads();   // every chunk's exclusive prefix read before the maps are overwritten
        // backward: x_r = U_r^-1 (y_r - c_r x_{r+1}) == mu_r + nu_r x_{r+1}
        a.P = c_make<C>(1.0, 0.0);
        a.Q = c_make<C>(0.0, 0.0);
        if (on) {
#pragma unroll 4
            for (int r = r1 - 1; r >= r0; --r) {
                Aff<C> mp;
                const C d = dcol[r * ld];
                mp.Q = c_mul(d, col[r * ld]);
                if (r == nv - 1) mp.P = c_make<C>(0.0, 0.0);
                else {
                    const C nu = c_mul(d, c_rmul(lam, __ldg(ga + r)));
                    mp.P = c_make<C>(-nu.x, -nu.y);
                }
                a = aff_combine(a, mp);
            }
        }
        tot[c][m] = a;
        __syncthreads();
        if (tid < TJC_MG * 32) {                           // chunks in descending order
            const int w = tid >> 5, lane = tid & 31;
            Aff<C> ex;
            warp_scan_aff_ie<C>(tot[lane][w], false, &ex);
            __syncwarp();
            tot[lane][w] = ex;
        }
        __syncthreads();
        C x = tot[c][m].Q;
        if (on) {
#pragma unroll 4
            for (int r = r1 - 1; r >= r0; --r) {
                const C d = dcol[r * ld];
                const C yv = col[r * ld];
                if (r == nv - 1) x = c_mul(d, yv);
                else x = c_mul(d, c_sub(yv, c_mul(c_rmul(lam, __ldg(ga + r)), x)));
                col[r * ld] = x;
            }
        }
        __syncthreads();   // the prefixes read before the next item reuses the array
    });
}

// ---- LU solves on the v-major layout, chunks held in registers ---------------
// Every lane owns a chunk of CH <= tjr_ch rows of one mode and keeps its right
// hand side and LU reciprocals in registers from one load to the store of the
// solution: the four sweeps (compose and replay, forward and backward) read
// no memory, so a row costs its arithmetic and one global load or store per
// value.  A warp holds 4 consecutive modes x 8 chunks (lane = 4 c + m: the 8
// rows a warp loads at once are 32-byte runs of the v-major spectrum); G
// warps, a power of two up to TJR_G with 8 G CH >= nv, cover a mode group's
// lines, and a CTA of TJR_G warps solves TJR_G / G groups (64 / G modes).
// The chunks' affine maps are scanned with shuffles inside the warp and
// joined across the G warps by a shuffle tree over their totals in shared
// memory.  Chunks of 8 rows in FP32 and 4 in FP64 (registers).
constexpr int TJR_G = 16, TJR_THREADS = 32 * TJR_G;
__host__ __device__ constexpr int tjr_ch(size_t rsz) { return rsz == 4 ? 8 : 4; }
__host__ __device__ constexpr int tjr_nvmax(size_t rsz) { return 8 * TJR_G * tjr_ch(rsz); }
__host__ __device__ constexpr int tjr_g(int nv, int ch) {
    return nv <= 8 * ch ? 1 : nv <= 16 * ch ? 2 : nv <= 32 * ch ? 4 : nv <= 64 * ch ? 8 : 16;
}
__host__ __device__ constexpr int tjr_modes(int nv, int ch) { return 4 * (TJR_G / tjr_g(nv, ch)); }   // modes per CTA item

// shfl of an affine map from lane src (full warp)
template <typename C>
VV_DEV Aff<C> shfl_aff_idx(const Aff<C>& a, int src) {
    Aff<C> r;
    r.P.x = __shfl_sync(0xffffffffu, a.P.x, src);
    r.P.y = __shfl_sync(0xffffffffu, a.P.y, src);
    r.Q.x = __shfl_sync(0xffffffffu, a.Q.x, src);
    r.Q.y = __shfl_sync(0xffffffffu, a.Q.y, src);
    return r;
}

// the composition, in order, of the maps t[0..cnt) of a lane's mode (cnt <=
// 16; one value per 8 chunk lanes of stride 4): lane c composes t[2c], t[2c+1]
// and a tree over the 8 chunk lanes joins them; every lane gets the result
template <typename C>
VV_DEV Aff<C> tjr_join(const Aff<C>* t, int stride, int cnt, int c, int m) {
    Aff<C> id;
    id.P = c_make<C>(1.0, 0.0);
    id.Q = c_make<C>(0.0, 0.0);
    Aff<C> a = 2 * c < cnt ? t[(2 * c) * stride] : id;
    if (2 * c + 1 < cnt) a = aff_combine(a, t[(2 * c + 1) * stride]);
#pragma unroll
    for (int d = 1; d < 8; d <<= 1) {
        const Aff<C> o = shfl_aff(a, 4 * d, false);
        if ((c & (2 * d - 1)) == 0 && c + d < 8) a = aff_combine(a, o);
    }
    return shfl_aff_idx(a, m);
}

// ordered composition of the maps mp(0) .. mp(CH - 1) (mp(0) first) as two
// independent chains over the halves joined at the end: half the dependent
// depth of one chain for two more registers of live state
template <typename C, int CH, typename Map>
VV_DEV Aff<C> aff_two_chains(Map mp) {
    Aff<C> a = mp(0), b = mp(CH / 2);
#pragma unroll
    for (int j = 1; j < CH / 2; ++j) {
        a = aff_combine(a, mp(j));
        b = aff_combine(b, mp(CH / 2 + j));
    }
    return aff_combine(a, b);
}

// One lane's chunk: rows r0 .. r0 + n of mode k (FULL: n == CH for every lane
// of the CTA, no guards).  The forward multipliers l_r and then the backward
// products lambda gamma_r stay in registers between a sweep's compose and its
// replay.  Lanes without a mode run the same instructions on zeros (a
// branch around the work of idle warps keeps more state live across the
// barriers and spills).
template <typename R, bool FULL>
VV_DEV void tjr_chunk(const BInst& I, int k, bool on, int r0, int n, int G, int grp, int sw, int c, int m,
                      Aff<typename Cplx<R>::type> (*tot)[TJR_G][4]) {
    using C = typename Cplx<R>::type;
    constexpr int CH = tjr_ch(sizeof(R));
    const int nv = I.tp.nv;
    const size_t ld = (size_t)I.tp.nmodes;
    C* col = (C*)I.specT + k + (size_t)r0 * ld;       // row r0 + j at col[j * ld]
    const C* dcol = (const C*)I.dinvJ + k + (size_t)r0 * ld;
    const C zero = c_make<C>(0.0, 0.0);
    const bool first = r0 == 0, last = r0 + n == nv;   // the chunk holds row 0 / row nv - 1
    Aff<C> id;
    id.P = c_make<C>(1.0, 0.0);
    id.Q = zero;
    C lam = zero;
    C bb[CH], dd[CH], ll[CH];
    R gg[CH];
    Aff<C> ex = id;
    {
        const R* al = reinterpret_cast<const R*>(I.tp.alpha) + r0;
        const R* ga = reinterpret_cast<const R*>(I.tp.gamma) + r0;
        if (on) lam = reinterpret_cast<const C*>(I.tp.lambda)[k];
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const bool in = FULL || j < n;
            bb[j] = in ? col[j * ld] : zero;
            dd[j] = in ? dcol[j * ld] : zero;
            const R a = in ? __ldg(al + j) : (R)0;
            gg[j] = in ? __ldg(ga + j) : (R)0;
            ll[j] = c_rmul(lam, a);
        }
        const C dp0 = (n > 0 && !first) ? dcol[-(ptrdiff_t)ld] : zero;   // U^-1 of the row before the chunk
        // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
#pragma unroll
        for (int j = 0; j < CH; ++j) ll[j] = c_mul(ll[j], j == 0 ? dp0 : dd[j > 0 ? j - 1 : 0]);
        Aff<C> inc = aff_two_chains<C, CH>([&](int j) {
            Aff<C> mp;
            mp.Q = bb[j];
            mp.P = (j == 0 && first) ? zero : c_make<C>(-ll[j].x, -ll[j].y);
            return (FULL || j < n) ? mp : id;
        });
#pragma unroll
        for (int d = 1; d < 8; d <<= 1) {
            const Aff<C> o = shfl_aff(inc, 4 * d, true);
            if (c >= d) inc = aff_combine(o, inc);
        }
        ex = shfl_aff(inc, 4, true);
        if (c == 0) ex = id;
        if (c == 7) tot[0][grp * G + sw][m] = inc;
    }
    __syncthreads();
    {
        const Aff<C> pre = tjr_join<C>(&tot[0][grp * G][m], 4, sw, c, m);
        C y = aff_combine(pre, ex).Q;
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            if (FULL || j < n) {
                y = (j == 0 && first) ? bb[j] : c_sub(bb[j], c_mul(ll[j], y));
                bb[j] = y;
            }
        }
        // backward: x_r = U_r^-1 (y_r - c_r x_{r+1}) == mu_r + nu_r x_{r+1}; map i is row CH - 1 - i
#pragma unroll
        for (int j = 0; j < CH; ++j) ll[j] = c_rmul(lam, gg[j]);
        Aff<C> inc = aff_two_chains<C, CH>([&](int i) {
            const int j = CH - 1 - i;
            const C nu = c_mul(dd[j], ll[j]);
            Aff<C> mp;
            mp.Q = c_mul(dd[j], bb[j]);
            mp.P = (j == n - 1 && last) ? zero : c_make<C>(-nu.x, -nu.y);
            return (FULL || j < n) ? mp : id;
        });
#pragma unroll
        for (int d = 1; d < 8; d <<= 1) {
            const Aff<C> o = shfl_aff(inc, 4 * d, false);
            if (c + d < 8) inc = aff_combine(o, inc);
        }
        ex = shfl_aff(inc, 4, false);
        if (c == 7) ex = id;
        if (c == 0) tot[1][grp * G + sw][m] = inc;
    }
    __syncthreads();
    {
        // the warps above this one, highest first: tot[1][grp G + G - 1 - u], u < G - 1 - sw
        const Aff<C> post = tjr_join<C>(&tot[1][grp * G + G - 1][m], -4, G - 1 - sw, c, m);
        C x = aff_combine(post, ex).Q;
#pragma unroll
        for (int j = CH - 1; j >= 0; --j) {
            if (FULL || j < n) {
                x = (j == n - 1 && last) ? c_mul(dd[j], bb[j]) : c_mul(dd[j], c_sub(bb[j], c_mul(ll[j], x)));
                col[j * ld] = x;
            }
        }
    }
}

template <typename R>
__global__ void __launch_bounds__(TJR_THREADS, 1)
    k_b_tridiagjr(const BInst* __restrict__ tab, const int* __restrict__ L, int n) {
    using C = typename Cplx<R>::type;
    constexpr int CHM = tjr_ch(sizeof(R));
    __shared__ Aff<C> tot[2][TJR_G][4];
    for_work<F_MODES>(tab, L, n, [&](const BInst& I, int local) {
        const int nv = I.tp.nv, nm = I.tp.nmodes;
        const int G = tjr_g(nv, CHM), MPB = tjr_modes(nv, CHM);
        const int CH = (nv + 8 * G - 1) / (8 * G);
        const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int m = lane & 3, c = lane >> 2;
        const int grp = wid / G, sw = wid % G;
        const int k = local * MPB + 4 * grp + m;
        const bool on = k < nm;
        const int r0 = min((8 * sw + c) * CH, nv);
        const int cnt = on ? min(CH, nv - r0) : 0;
        // block-uniform choice (both paths hold barriers): every mode of the
        // item present and every chunk CHM rows long
        if ((local + 1) * MPB <= nm && nv == 8 * G * CHM)
            tjr_chunk<R, true>(I, k, true, r0, CHM, G, grp, sw, c, m, tot);
        else
            tjr_chunk<R, false>(I, on ? k : 0, on, r0, cnt, G, grp, sw, c, m, tot);
        __syncthreads();   // the totals read before the next item overwrites them
    });
}

}  // namespace vv
