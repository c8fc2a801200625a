// FFT tensor-product kinetic preconditioner  P^-1 = F_x^-1 (A_k^-1) F_x
// (TensorProductKinetic.pyx:345-359, TensorProductKineticFast.pyx:102-272).
//
//   k_rfft_rows    : real FFT along x of every v row (length nx, power of 2),
//                    via a half-length complex FFT in shared memory; writes
//                    the half spectrum TRANSPOSED, spec[k*nv + j], so every
//                    x mode's v line is contiguous (the reference's cax->cay
//                    scatter, TensorProductKinetic.pyx:183-188).
//   k_tridiag_modes: one CTA per x mode solves the complex tridiagonal system
//                    in v with the LU factors computed once at set-up
//                    (zgbtrf, TensorProductKineticFast.pyx:88-90).  The two
//                    bidiagonal sweeps are linear recurrences; each thread
//                    composes the affine maps of a chunk of rows, a block
//                    scan joins the chunks, and each thread replays its chunk.
//   k_irfft_rows   : inverse real FFT (normalised by 1/nx, the pyFFTW
//                    default) back to F[j*nx + i]; the imaginary parts of the
//                    mean and Nyquist modes are ignored, as by a c2r FFT.
#pragma once
#include "vv_common.cuh"

namespace vv {

struct PcParams {
    int nx, nv;
    int M;                 // nx/2: complex FFT length
    int logM;
    int R;                 // rows (warps) per CTA in the row kernels
    const void* tw;        // tw[k] = exp(-2 pi i k / nx), k < nx (double2 or float2); the FFT kernels read k < nx/2
    const int* yidx;       // optional: output is Y + (*yidx + yoff) * ystride
    int yoff;
    size_t ystride;
};

__device__ __forceinline__ int bitrev(int m, int logM) {
    return logM == 0 ? 0 : (int)(__brev((unsigned)m) >> (32 - logM));
}

// In-place radix-2 DIT FFT of one row of length M (bit-reversed input) by
// one warp; `stw` holds exp(-2 pi i k /(2M)), k < M, in shared memory.
// SIGN = -1 forward, +1 inverse (unnormalised).  Only __syncwarp between
// stages: the warps of a CTA transform their rows independently.
template <int SIGN, typename C>
__device__ __forceinline__ void warp_fft(C* buf, int M, int logM, const C* stw) {
    const int lane = threadIdx.x & 31;
    const int nb = M >> 1;
    for (int lh = 0; lh < logM; ++lh) {
        const int half = 1 << lh;
        const int tshift = logM - lh;          // twiddle index = pos * (M/half)
        for (int b = lane; b < nb; b += 32) {
            const int grp = b >> lh;
            const int pos = b & (half - 1);
            const int i0 = (grp << (lh + 1)) + pos;
            const int i1 = i0 + half;
            C w = stw[pos << tshift];
            if (SIGN > 0) w.y = -w.y;
            const C a = buf[i0];
            const C t = c_mul(w, buf[i1]);
            buf[i0] = c_add(a, t);
            buf[i1] = c_sub(a, t);
        }
        __syncwarp();
    }
}

// Block-wide in-place radix-2 DIT FFT of one row of length M (bit-reversed
// input), used by the single-CTA Poisson solve.  stw as in warp_fft.
template <int SIGN>
__device__ __forceinline__ void block_fft(double2* buf, int M, const double2* stw) {
    for (int half = 1; half < M; half <<= 1) {
        const int tstride = M / half;
        for (int b = threadIdx.x; b < (M >> 1); b += blockDim.x) {
            const int grp = b / half;
            const int pos = b - grp * half;
            const int i0 = grp * 2 * half + pos;
            const int i1 = i0 + half;
            double2 w = stw[pos * tstride];
            if (SIGN > 0) w.y = -w.y;
            const double2 a = buf[i0];
            const double2 t = c_mul(w, buf[i1]);
            buf[i0] = c_add(a, t);
            buf[i1] = c_sub(a, t);
        }
        __syncthreads();
    }
}

// Real FFT along x of R consecutive v rows (one warp per row), half
// spectrum written transposed: spec[k*nv + j], k = 0..M.
// dynamic smem: [M twiddles][R rows x (M+1) complex]
template <typename TI, typename R>
__device__ __forceinline__ void rfft_rows_block(const TI* __restrict__ X, typename Cplx<R>::type* __restrict__ spec,
                                                const PcParams& p, int bid) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    const int M = p.M, LD = M + 1;
    C* rows = stw + M;
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = tw[k];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j0 = bid * p.R;
    const int j = j0 + warp;
    C* buf = rows + warp * LD;
    __syncthreads();
    if (warp < p.R && j < p.nv) {
        const TI* row = X + (size_t)j * p.nx;
        for (int m = lane; m < M; m += 32)
            buf[bitrev(m, p.logM)] = c_make<C>((double)row[2 * m], (double)row[2 * m + 1]);
        __syncwarp();
        warp_fft<-1>(buf, M, p.logM, stw);
        // split: X_k = E_k + W_N^k O_k,  E = (Z_k + conj Z_{M-k})/2,  O = -i/2 (Z_k - conj Z_{M-k})
        // computed for the pair (k, M-k) by one lane so the update is in place
        for (int k = lane; k <= M / 2; k += 32) {
            const int kc = M - k;
            const C zk = buf[k == M ? 0 : k];
            const C zc = buf[k == 0 ? 0 : kc];
            C out_k, out_c;
            {
                const C zcc = c_conj(zc);
                const C E = c_scale(c_add(zk, zcc), (R)0.5);
                const C D = c_sub(zk, zcc);
                const C O = c_make<C>(0.5 * D.y, -0.5 * D.x);
                out_k = c_add(E, c_mul(stw[k], O));
            }
            {
                const C zkc = c_conj(zk);   // pair element kc: Z_kc and conj Z_{M-kc} = conj Z_k
                const C E = c_scale(c_add(zc, zkc), (R)0.5);
                const C D = c_sub(zc, zkc);
                const C O = c_make<C>(0.5 * D.y, -0.5 * D.x);
                const C w = (kc < M) ? stw[kc] : c_make<C>(-1.0, 0.0);
                out_c = c_add(E, c_mul(w, O));
            }
            if (k == 0) {           // k = 0 and k = M share Z_0
                buf[0] = out_k;
                buf[M] = out_c;
            } else if (k == kc) {
                buf[k] = out_k;
            } else {
                buf[k] = out_k;
                buf[kc] = out_c;
            }
        }
    }
    __syncthreads();
    // transposed, coalesced write: R consecutive j per mode k
    const int nrow = min(p.R, p.nv - j0);
    for (int idx = threadIdx.x; idx < (M + 1) * p.R; idx += blockDim.x) {
        const int k = idx / p.R, r = idx - k * p.R;
        if (r < nrow) spec[(size_t)k * p.nv + j0 + r] = rows[r * LD + k];
    }
}

template <typename TI, typename R>
__global__ void k_rfft_rows(const TI* __restrict__ X, typename Cplx<R>::type* __restrict__ spec, PcParams p) {
    rfft_rows_block<TI, R>(X, spec, p, blockIdx.x);
}

// spec[k*nv + j] (k = 0..M) -> rows of Y (one warp per row), scaled by 1/nx
// dynamic smem: [M twiddles][R rows x (M+1) spectrum][R rows x (M+1) work]
template <typename R, typename TO>
__device__ __forceinline__ void irfft_rows_block(const typename Cplx<R>::type* __restrict__ spec,
                                                 TO* __restrict__ Y, const PcParams& p, int bid) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    const int M = p.M, LD = M + 1;
    C* xs = stw + M;
    C* work = xs + p.R * LD;
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = tw[k];
    const int j0 = bid * p.R;
    const int nrow = min(p.R, p.nv - j0);
    for (int idx = threadIdx.x; idx < (M + 1) * p.R; idx += blockDim.x) {
        const int k = idx / p.R, r = idx - k * p.R;
        C v = c_make<C>(0.0, 0.0);
        if (r < nrow) v = spec[(size_t)k * p.nv + j0 + r];
        if (k == 0 || k == M) v.y = 0;   // c2r ignores these imaginary parts
        xs[r * LD + k] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= nrow) return;
    const C* xr = xs + warp * LD;
    C* buf = work + warp * LD;
    // Z_k = (X_k + conj X_{M-k})/2 + i W_N^{-k} (X_k - conj X_{M-k})/2
    for (int k = lane; k < M; k += 32) {
        const C xk = xr[k];
        const C xc = c_conj(xr[M - k]);
        const C E = c_scale(c_add(xk, xc), (R)0.5);
        C w = stw[k];
        w.y = -w.y;
        const C O = c_mul(w, c_scale(c_sub(xk, xc), (R)0.5));
        buf[bitrev(k, p.logM)] = c_make<C>(E.x - O.y, E.y + O.x);
    }
    __syncwarp();
    warp_fft<+1>(buf, M, p.logM, stw);
    const R s = (R)(1.0 / (double)M);   // (1/M) IDFT_M gives the 1/nx-normalised irfft
    TO* row = Y + (size_t)(j0 + warp) * p.nx;
    for (int m = lane; m < M; m += 32) {
        const C z = buf[m];
        row[2 * m] = (TO)(z.x * s);
        row[2 * m + 1] = (TO)(z.y * s);
    }
}

template <typename R, typename TO>
__global__ void k_irfft_rows(const typename Cplx<R>::type* __restrict__ spec, TO* __restrict__ Y, PcParams p) {
    if (p.yidx) Y += (size_t)(*p.yidx + p.yoff) * p.ystride;
    irfft_rows_block<R, TO>(spec, Y, p, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Four-step FFT by one warp, M = 32 E (E = 1..32): lane l holds z[l + 32 m2];
// an E-point DFT in registers, the twiddle W_M^{l k2}, then a 32-point DIF
// across lanes with xor shuffles.  Lane l ends with X[k2 + E bitrev5(l)].
// No shared memory and no barrier inside the transform.
// ---------------------------------------------------------------------------
// bit reversal of j over `bits` bits; a loop (not recursion) so that it folds
// to a constant inside unrolled loops and register arrays stay in registers
__host__ __device__ constexpr int crev(int j, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((j >> b) & 1) << (bits - 1 - b);
    return r;
}
__host__ __device__ constexpr int clog2(int n) { return n <= 1 ? 0 : 1 + clog2(n >> 1); }

// W_M^q (SIGN < 0) or its conjugate from the staged table stw[k] = W_N^k,
// k < M, N = 2M: W_M^q = W_N^{2q}, and W_N^{k+M} = -W_N^k.
template <int M, int SIGN, typename C>
__device__ __forceinline__ C tw_half(const C* stw, int q) {
    const int idx = 2 * q;
    C w = idx < M ? stw[idx] : stw[idx - M];
    if (idx >= M) { w.x = -w.x; w.y = -w.y; }
    if (SIGN > 0) w.y = -w.y;
    return w;
}

template <int E, int SIGN, typename C>
__device__ __forceinline__ void reg_fft(C (&a)[E], const C* stw) {
    constexpr int B = clog2(E);
    C t[E];
#pragma unroll
    for (int j = 0; j < E; ++j) t[crev(j, B)] = a[j];
#pragma unroll
    for (int h = 1; h < E; h <<= 1) {
#pragma unroll
        for (int g = 0; g < E; g += 2 * h) {
#pragma unroll
            for (int pos = 0; pos < h; ++pos) {
                const C w = tw_half<32 * E, SIGN>(stw, 32 * pos * (E / (2 * h)));  // W_E^{pos E/(2h)}
                const C u = t[g + pos];
                const C v = c_mul(w, t[g + pos + h]);
                t[g + pos] = c_add(u, v);
                t[g + pos + h] = c_sub(u, v);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < E; ++j) a[j] = t[j];
}

template <int E, int SIGN, typename C>
__device__ __forceinline__ void warp_fft4(C (&a)[E], const C* stw) {
    const int lane = threadIdx.x & 31;
    reg_fft<E, SIGN>(a, stw);
#pragma unroll
    for (int k2 = 1; k2 < E; ++k2) {                 // W_M^{lane k2}
        a[k2] = c_mul(a[k2], tw_half<32 * E, SIGN>(stw, lane * k2));
    }
#pragma unroll
    for (int span = 16; span >= 1; span >>= 1) {
        const bool upper = (lane & span) != 0;
        const int i = lane & (span - 1);
        const C w = tw_half<32 * E, SIGN>(stw, (i * (16 / span)) * E);  // W_32^{i 16/span}
#pragma unroll
        for (int k2 = 0; k2 < E; ++k2) {
            const C mine = a[k2];
            C other;
            other.x = __shfl_xor_sync(0xffffffffu, mine.x, span);
            other.y = __shfl_xor_sync(0xffffffffu, mine.y, span);
            a[k2] = upper ? c_mul(c_sub(other, mine), w) : c_add(mine, other);
        }
    }
}

// index in a warp's padded buffer of the value lane l holds as a[k2]
template <int E>
__device__ __forceinline__ int zslot(int lane, int k2) { return lane * (E + 1) + k2; }
// ... and of transform output k (k = k2 + E k1 lives in lane bitrev5(k1))
template <int E>
__device__ __forceinline__ int zslot_of(int k) {
    return (int)(__brev((unsigned)(k / E)) >> 27) * (E + 1) + (k % E);
}

// Real FFT along x (nx = 2M = 64 E) of RW rows per CTA, one warp per row,
// half spectrum written transposed: spec[k*nv + j].
// dynamic smem: [M twiddles][RW x (M+1) half spectra][RW x 32(E+1) transform slots]
template <typename TI, typename R, int E>
__device__ __forceinline__ void rfft4_block(const TI* __restrict__ X, typename Cplx<R>::type* __restrict__ spec,
                                            const PcParams& p, int bid) {
    using C = typename Cplx<R>::type;
    constexpr int M = 32 * E, LD = M + 1, ZS = 32 * (E + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    C* rows = stw + M;
    C* zb = rows + p.R * LD;
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = tw[k];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j0 = bid * p.R;
    const int j = j0 + warp;
    __syncthreads();
    if (warp < p.R && j < p.nv) {
        const TI* row = X + (size_t)j * p.nx;
        C a[E];
#pragma unroll
        for (int m2 = 0; m2 < E; ++m2) {
            const int m = lane + 32 * m2;
            a[m2] = c_make<C>((double)row[2 * m], (double)row[2 * m + 1]);
        }
        warp_fft4<E, -1>(a, stw);
        C* z = zb + warp * ZS;
#pragma unroll
        for (int k2 = 0; k2 < E; ++k2) z[zslot<E>(lane, k2)] = a[k2];
        __syncwarp();
        C* out = rows + warp * LD;
        for (int k = lane; k <= M / 2; k += 32) {
            const int kc = M - k;
            const C zk = z[zslot_of<E>(k == M ? 0 : k)];
            const C zc = z[zslot_of<E>(k == 0 ? 0 : kc)];
            const C zcc = c_conj(zc);
            C E1 = c_scale(c_add(zk, zcc), (R)0.5);
            C D = c_sub(zk, zcc);
            const C outk = c_add(E1, c_mul(stw[k], c_make<C>(0.5 * D.y, -0.5 * D.x)));
            const C zkc = c_conj(zk);
            E1 = c_scale(c_add(zc, zkc), (R)0.5);
            D = c_sub(zc, zkc);
            const C w = (kc < M) ? stw[kc] : c_make<C>(-1.0, 0.0);
            const C outc = c_add(E1, c_mul(w, c_make<C>(0.5 * D.y, -0.5 * D.x)));
            out[k] = outk;
            if (kc != k) out[kc] = outc;
        }
    }
    __syncthreads();
    const int nrow = min(p.R, p.nv - j0);
    for (int idx = threadIdx.x; idx < (M + 1) * p.R; idx += blockDim.x) {
        const int k = idx / p.R, r = idx - k * p.R;
        if (r < nrow) spec[(size_t)k * p.nv + j0 + r] = rows[r * LD + k];
    }
}

template <typename TI, typename R, int E>
__global__ void k_rfft4(const TI* __restrict__ X, typename Cplx<R>::type* __restrict__ spec, PcParams p) {
    rfft4_block<TI, R, E>(X, spec, p, blockIdx.x);
}

// spec[k*nv + j] -> RW rows of Y (one warp per row), normalised by 1/nx
// dynamic smem: [M twiddles][RW x (M+1) half spectra][RW x 32(E+1) transform slots]
template <typename R, typename TO, int E>
__device__ __forceinline__ void irfft4_block(const typename Cplx<R>::type* __restrict__ spec, TO* __restrict__ Y,
                                             const PcParams& p, int bid) {
    using C = typename Cplx<R>::type;
    constexpr int M = 32 * E, LD = M + 1, ZS = 32 * (E + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    C* rows = stw + M;
    C* zb = rows + p.R * LD;
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = tw[k];
    const int j0 = bid * p.R;
    const int nrow = min(p.R, p.nv - j0);
    for (int idx = threadIdx.x; idx < (M + 1) * p.R; idx += blockDim.x) {
        const int k = idx / p.R, r = idx - k * p.R;
        C v = c_make<C>(0.0, 0.0);
        if (r < nrow) v = spec[(size_t)k * p.nv + j0 + r];
        if (k == 0 || k == M) v.y = 0;   // c2r ignores these imaginary parts
        rows[r * LD + k] = v;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= nrow) return;
    const C* xr = rows + warp * LD;
    C a[E];
#pragma unroll
    for (int m2 = 0; m2 < E; ++m2) {
        const int k = lane + 32 * m2;
        const C xk = xr[k];
        const C xc = c_conj(xr[M - k]);
        const C E1 = c_scale(c_add(xk, xc), (R)0.5);
        C w = stw[k];
        w.y = -w.y;
        const C O = c_mul(w, c_scale(c_sub(xk, xc), (R)0.5));
        a[m2] = c_make<C>(E1.x - O.y, E1.y + O.x);      // Z_k = E + i O
    }
    warp_fft4<E, +1>(a, stw);
    C* z = zb + warp * ZS;
#pragma unroll
    for (int k2 = 0; k2 < E; ++k2) z[zslot<E>(lane, k2)] = a[k2];
    __syncwarp();
    const R s = (R)(1.0 / (double)M);
    TO* row = Y + (size_t)(j0 + warp) * p.nx;
    for (int m = lane; m < M; m += 32) {
        const C v = z[zslot_of<E>(m)];
        row[2 * m] = (TO)(v.x * s);
        row[2 * m + 1] = (TO)(v.y * s);
    }
}

template <typename R, typename TO, int E>
__global__ void k_irfft4(const typename Cplx<R>::type* __restrict__ spec, TO* __restrict__ Y, PcParams p) {
    if (p.yidx) Y += (size_t)(*p.yidx + p.yoff) * p.ystride;
    irfft4_block<R, TO, E>(spec, Y, p, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Direct real DFT along x for any nx (the lengths the FFT kernels do not
// take: odd and other non-power-of-two grids of the reference's example
// configurations).  O(nx^2) per row from the nx-entry twiddle table;
// numpy's rfft / irfft conventions (irfft ignores the imaginary parts of
// X_0 and, for even nx, X_{nx/2}).  DFT_ROWS rows per CTA.
// ---------------------------------------------------------------------------
constexpr int DFT_ROWS = 4, DFT_THREADS = 256;

// X_k = sum_n x_n W^{nk}, k = 0..nx/2, written mode-major spec[k*nv + j].
// dynamic smem: nx twiddles (complex R) + DFT_ROWS x nx (R)
template <typename TI, typename R>
__global__ void __launch_bounds__(DFT_THREADS)
k_rdft_rows(const TI* __restrict__ X, typename Cplx<R>::type* __restrict__ spec, PcParams p) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = p.nx, nm = N / 2 + 1;
    C* stw = reinterpret_cast<C*>(smem_raw);
    R* xs = reinterpret_cast<R*>(stw + N);
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < N; k += blockDim.x) stw[k] = tw[k];
    const int j0 = blockIdx.x * DFT_ROWS;
    for (int i = threadIdx.x; i < DFT_ROWS * N; i += blockDim.x) {
        const int r = i / N, n = i - r * N, j = j0 + r;
        xs[i] = (j < p.nv) ? (R)X[(size_t)j * N + n] : (R)0;
    }
    __syncthreads();
    for (int u = threadIdx.x; u < nm * DFT_ROWS; u += blockDim.x) {
        const int k = u / DFT_ROWS, r = u - k * DFT_ROWS, j = j0 + r;
        const R* xr = xs + r * N;
        R re = 0, im = 0;
        int idx = 0;
        for (int n = 0; n < N; ++n) {
            const C w = stw[idx];
            re += xr[n] * w.x;
            im += xr[n] * w.y;
            idx += k;
            if (idx >= N) idx -= N;
        }
        if (j < p.nv) spec[(size_t)k * p.nv + j] = c_make<C>((double)re, (double)im);
    }
}

// x_n = (1/nx) [Re X_0 + 2 sum_{k=1}^{(nx-1)/2} Re(X_k W^{-nk}) + (nx even) Re X_{nx/2} (-1)^n]
// dynamic smem: nx twiddles + DFT_ROWS x (nx/2 + 1) complex
template <typename R, typename TO>
__global__ void __launch_bounds__(DFT_THREADS)
k_irdft_rows(const typename Cplx<R>::type* __restrict__ spec, TO* __restrict__ Y, PcParams p) {
    using C = typename Cplx<R>::type;
    if (p.yidx) Y += (size_t)(*p.yidx + p.yoff) * p.ystride;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N = p.nx, nm = N / 2 + 1, K = (N - 1) / 2;
    C* stw = reinterpret_cast<C*>(smem_raw);
    C* xs = stw + N;
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < N; k += blockDim.x) stw[k] = tw[k];
    const int j0 = blockIdx.x * DFT_ROWS;
    for (int i = threadIdx.x; i < DFT_ROWS * nm; i += blockDim.x) {
        const int k = i / DFT_ROWS, r = i - k * DFT_ROWS, j = j0 + r;
        xs[r * nm + k] = (j < p.nv) ? spec[(size_t)k * p.nv + j] : c_make<C>(0.0, 0.0);
    }
    __syncthreads();
    const R inv = (R)(1.0 / (double)N);
    for (int u = threadIdx.x; u < DFT_ROWS * N; u += blockDim.x) {
        const int r = u / N, n = u - r * N, j = j0 + r;
        const C* xr = xs + r * nm;
        R s = xr[0].x;
        int idx = 0;
        for (int k = 1; k <= K; ++k) {
            idx += n;
            if (idx >= N) idx -= N;
            const C w = stw[idx];   // W^{nk} = (cos, -sin): Re(X e^{+i theta}) = X.x w.x + X.y w.y
            s += (R)2 * (xr[k].x * w.x + xr[k].y * w.y);
        }
        if (!(N & 1)) s += (n & 1) ? -xr[N / 2].x : xr[N / 2].x;
        if (j < p.nv) Y[(size_t)j * N + n] = (TO)(s * inv);
    }
}

// ---------------------------------------------------------------------------
// tridiagonal solves, one CTA per x mode
// ---------------------------------------------------------------------------
struct TriParams {
    int nv, nmodes;
    const void* lambda;  // per mode eigenvalue lambda_k (shifted, TensorProduct.pyx:109-116), complex R
    const void* alpha;   // nv (R): sub-diagonal  A[r,r-1] = lambda * alpha[r]
    const void* gamma;   // nv (R): super-diagonal A[r,r+1] = lambda * gamma[r]
    const void* dinv;    // nmodes*nv (complex R): 1 / U[r,r] of the LU factors
};

constexpr int TRI_THREADS = 256;

// affine map x -> P x + Q on complex numbers; combine(first, second) = second o first
template <typename C> struct Aff { C P, Q; };
template <typename C>
VV_DEV Aff<C> aff_combine(const Aff<C>& first, const Aff<C>& second) {
    Aff<C> r;
    r.P = c_mul(second.P, first.P);
    r.Q = c_add(c_mul(second.P, first.Q), second.Q);
    return r;
}
template <typename T>
VV_DEV T shfl_dir(T v, int d, bool up) {
    return up ? __shfl_up_sync(0xffffffffu, v, d) : __shfl_down_sync(0xffffffffu, v, d);
}
template <typename C>
VV_DEV Aff<C> shfl_aff(const Aff<C>& a, int d, bool up) {
    Aff<C> r;
    r.P.x = shfl_dir(a.P.x, d, up);
    r.P.y = shfl_dir(a.P.y, d, up);
    r.Q.x = shfl_dir(a.Q.x, d, up);
    r.Q.y = shfl_dir(a.Q.y, d, up);
    return r;
}

// Exclusive scan of affine maps across the block in thread order `pos`
// (pos = tid for the forward sweep, nthreads-1-tid for the backward sweep;
// both keep warps intact).  Returns the image of 0 under the composition of
// all earlier chunks.
template <typename C>
__device__ C block_scan_aff(Aff<C> a, bool forward, Aff<C>* sh) {
    const int pos = forward ? (int)threadIdx.x : TRI_THREADS - 1 - (int)threadIdx.x;
    const int lane = pos & 31, wid = pos >> 5;
    Aff<C> inc = a;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Aff<C> o = shfl_aff(inc, d, forward);   // the lane d earlier in pos order
        if (lane >= d) inc = aff_combine(o, inc);
    }
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    Aff<C> pre;
    pre.P = c_make<C>(1.0, 0.0);
    pre.Q = c_make<C>(0.0, 0.0);
    for (int w = 0; w < wid; ++w) pre = aff_combine(pre, sh[w]);
    const Aff<C> prev = shfl_aff(inc, 1, forward);
    Aff<C> ex = pre;
    if (lane > 0) ex = aff_combine(pre, prev);
    __syncthreads();
    return ex.Q;
}

// One CTA per x mode; each thread owns a chunk of C consecutive rows.  The
// right-hand side, LU reciprocals and the alpha/gamma tables are staged in
// shared memory with one pad slot per chunk (conflict-free chunk-strided
// access).  dynamic smem: 3 arrays of nv + nv/C complex/real slots.
template <typename R, bool STAGE>
__device__ __forceinline__ void tridiag_mode(typename Cplx<R>::type* __restrict__ spec, const TriParams& p, int k) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Aff<C> shw[TRI_THREADS / 32];
    const int nv = p.nv;
    const int CH = (nv + TRI_THREADS - 1) / TRI_THREADS;   // rows per thread
    const int NP = nv + (nv + CH - 1) / CH;               // padded length
    C* b = reinterpret_cast<C*>(smem_raw);
    C* di = b + NP;
    R* al = reinterpret_cast<R*>(di + NP);
    R* ga = al + NP;
    C* line = spec + (size_t)k * nv;
    const C* dinv_g = reinterpret_cast<const C*>(p.dinv) + (size_t)k * nv;
    const R* alpha_g = reinterpret_cast<const R*>(p.alpha);
    const R* gamma_g = reinterpret_cast<const R*>(p.gamma);
    const C lam = reinterpret_cast<const C*>(p.lambda)[k];
    const FastDiv dch((unsigned)CH);
    for (int r = threadIdx.x; r < nv; r += TRI_THREADS) {   // every copy in flight at once
        const int q = r + (int)dch((unsigned)r);
        cp_async_elem(&b[q], &line[r]);
        if (STAGE) {
            cp_async_elem(&di[q], &dinv_g[r]);
            cp_async_elem(&al[q], &alpha_g[r]);
            cp_async_elem(&ga[q], &gamma_g[r]);
        }
    }
    cp_async_commit();
    cp_async_wait0();
    __syncthreads();
    // accessors: row r at padded index q (tables staged or read through L1/L2)
    auto DI = [&](int r, int q) -> C { return STAGE ? di[q] : dinv_g[r]; };
    auto AL = [&](int r, int q) -> R { return STAGE ? al[q] : alpha_g[r]; };
    auto GA = [&](int r, int q) -> R { return STAGE ? ga[q] : gamma_g[r]; };
    const int r0 = threadIdx.x * CH;
    const int r1 = min(r0 + CH, nv);
    const int q0 = threadIdx.x * (CH + 1);       // padded index of r0
    // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
    Aff<C> a;
    a.P = c_make<C>(1.0, 0.0);
    a.Q = c_make<C>(0.0, 0.0);
    for (int r = r0, q = q0; r < r1; ++r, ++q) {
        Aff<C> m;
        if (r == 0) m.P = c_make<C>(0.0, 0.0);
        else {
            const C dprev = DI(r - 1, (r == r0) ? q - 2 : q - 1);   // r0-1 sits before the pad slot
            const C l = c_mul(c_rmul(lam, AL(r, q)), dprev);
            m.P = c_make<C>(-l.x, -l.y);
        }
        m.Q = b[q];
        a = aff_combine(a, m);
    }
    C y = block_scan_aff<C>(a, true, shw);
    for (int r = r0, q = q0; r < r1; ++r, ++q) {
        if (r == 0) y = b[q];
        else {
            const C dprev = DI(r - 1, (r == r0) ? q - 2 : q - 1);
            const C l = c_mul(c_rmul(lam, AL(r, q)), dprev);
            y = c_sub(b[q], c_mul(l, y));
        }
        b[q] = y;
    }
    __syncthreads();
    // backward: x_r = U_r^-1 (y_r - c_r x_{r+1})  ==  mu_r + nu_r x_{r+1}
    a.P = c_make<C>(1.0, 0.0);
    a.Q = c_make<C>(0.0, 0.0);
    for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
        Aff<C> m;
        const C d = DI(r, q);
        m.Q = c_mul(d, b[q]);
        if (r == nv - 1) m.P = c_make<C>(0.0, 0.0);
        else {
            const C nu = c_mul(d, c_rmul(lam, GA(r, q)));
            m.P = c_make<C>(-nu.x, -nu.y);
        }
        a = aff_combine(a, m);
    }
    C x = block_scan_aff<C>(a, false, shw);
    for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
        const C d = DI(r, q);
        if (r == nv - 1) x = c_mul(d, b[q]);
        else {
            const C cc = c_rmul(lam, GA(r, q));
            x = c_mul(d, c_sub(b[q], c_mul(cc, x)));
        }
        line[r] = x;
    }
}

template <typename R, bool STAGE>
__global__ void __launch_bounds__(TRI_THREADS)
k_tridiag_modes(typename Cplx<R>::type* __restrict__ spec, TriParams p) {
    tridiag_mode<R, STAGE>(spec, p, blockIdx.x);
}

// Warp-scan of affine maps (no shared memory): returns the image of 0 under
// the composition of the maps of all earlier lanes in `forward` order.
template <typename C>
__device__ __forceinline__ C warp_scan_aff(Aff<C> a, bool forward) {
    const int lane = threadIdx.x & 31;
    const int pos = forward ? lane : 31 - lane;
    Aff<C> inc = a;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Aff<C> o = shfl_aff(inc, d, forward);
        if (pos >= d) inc = aff_combine(o, inc);
    }
    const Aff<C> prev = shfl_aff(inc, 1, forward);
    return pos > 0 ? prev.Q : c_make<C>(0.0, 0.0);
}

// One warp per x mode (8 modes per CTA): lane l owns rows
// [l*CH, (l+1)*CH) of the mode's v line; the LU reciprocals and the
// alpha/gamma tables are read through L1 in the lane's own contiguous chunk.
// No shared memory, no block barrier.
constexpr int TRIW_WARPS = 4;

// shared-memory slots per warp and array of the staged warp solve: the line
// padded by one slot per lane chunk (at most 32 pads)
__host__ __device__ constexpr int tri_ws_slots(int nv) { return nv + 32; }

// mode k of the spectrum by the calling warp
template <typename R>
__device__ __forceinline__ void tridiag_warp_mode(typename Cplx<R>::type* __restrict__ spec, const TriParams& p,
                                                  int k) {
    using C = typename Cplx<R>::type;
    const int lane = threadIdx.x & 31;
    const int nv = p.nv;
    const int CH = (nv + 31) / 32;
    const int r0 = lane * CH;
    const int r1 = min(r0 + CH, nv);
    C* line = spec + (size_t)k * nv;
    const C* di = reinterpret_cast<const C*>(p.dinv) + (size_t)k * nv;
    const R* al = reinterpret_cast<const R*>(p.alpha);
    const R* ga = reinterpret_cast<const R*>(p.gamma);
    const C lam = reinterpret_cast<const C*>(p.lambda)[k];
    // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
    Aff<C> a;
    a.P = c_make<C>(1.0, 0.0);
    a.Q = c_make<C>(0.0, 0.0);
    for (int r = r0; r < r1; ++r) {
        Aff<C> m;
        if (r == 0) m.P = c_make<C>(0.0, 0.0);
        else {
            const C l = c_mul(c_rmul(lam, al[r]), di[r - 1]);
            m.P = c_make<C>(-l.x, -l.y);
        }
        m.Q = line[r];
        a = aff_combine(a, m);
    }
    C y = warp_scan_aff<C>(a, true);
    for (int r = r0; r < r1; ++r) {
        const C b = line[r];
        if (r == 0) y = b;
        else {
            const C l = c_mul(c_rmul(lam, al[r]), di[r - 1]);
            y = c_sub(b, c_mul(l, y));
        }
        line[r] = y;
    }
    __syncwarp();
    // backward: x_r = U_r^-1 (y_r - c_r x_{r+1})  ==  mu_r + nu_r x_{r+1}
    a.P = c_make<C>(1.0, 0.0);
    a.Q = c_make<C>(0.0, 0.0);
    for (int r = r1 - 1; r >= r0; --r) {
        Aff<C> m;
        const C d = di[r];
        m.Q = c_mul(d, line[r]);
        if (r == nv - 1) m.P = c_make<C>(0.0, 0.0);
        else {
            const C nu = c_mul(d, c_rmul(lam, ga[r]));
            m.P = c_make<C>(-nu.x, -nu.y);
        }
        a = aff_combine(a, m);
    }
    C x = warp_scan_aff<C>(a, false);
    for (int r = r1 - 1; r >= r0; --r) {
        const C d = di[r];
        const C yv = line[r];
        if (r == nv - 1) x = c_mul(d, yv);
        else x = c_mul(d, c_sub(yv, c_mul(c_rmul(lam, ga[r]), x)));
        line[r] = x;
    }
}

template <typename R>
__global__ void __launch_bounds__(32 * TRIW_WARPS)
k_tridiag_warp(typename Cplx<R>::type* __restrict__ spec, TriParams p) {
    const int k = blockIdx.x * TRIW_WARPS + (threadIdx.x >> 5);
    if (k >= p.nmodes) return;
    tridiag_warp_mode<R>(spec, p, k);
}

// One warp per x mode with the mode's line and its LU reciprocals staged in
// the warp's slice of shared memory (and the alpha/gamma tables in the CTA's,
// shared by its warps): coalesced cp.async copies of whole lines, then lane l
// sweeps rows [l*CH, (l+1)*CH) out of shared memory (row r at padded slot
// r + r/CH; CH + 1 is odd for power-of-two lines, so the lanes'
// chunk-strided accesses are free of bank conflicts), with the chunks joined
// by warp scans of affine maps.  Every slice holds tri_ws_slots(nv) slots.
//
// tri_ws_stage_tables (all threads of the CTA) and tri_ws_stage_line (the
// warp of mode k) issue the copies; the caller waits for them
// (cp_async_wait0 + __syncthreads) before tridiag_warp_staged.
template <typename R>
__device__ __forceinline__ void tri_ws_stage_tables(const TriParams& p, R* __restrict__ sal, R* __restrict__ sga) {
    const int nv = p.nv;
    const int CH = (nv + 31) / 32;
    const R* al = reinterpret_cast<const R*>(p.alpha);
    const R* ga = reinterpret_cast<const R*>(p.gamma);
    const FastDiv dch((unsigned)CH);
    for (int r = threadIdx.x; r < nv; r += blockDim.x) {
        const int q = r + (int)dch((unsigned)r);
        cp_async_elem(&sal[q], &al[r]);
        cp_async_elem(&sga[q], &ga[r]);
    }
}
template <typename R>
__device__ __forceinline__ void tri_ws_stage_line(const typename Cplx<R>::type* __restrict__ spec, const TriParams& p,
                                                  int k, typename Cplx<R>::type* __restrict__ sb,
                                                  typename Cplx<R>::type* __restrict__ sd) {
    using C = typename Cplx<R>::type;
    const int lane = threadIdx.x & 31;
    const int nv = p.nv;
    const int CH = (nv + 31) / 32;
    const C* line = spec + (size_t)k * nv;
    const C* dg = reinterpret_cast<const C*>(p.dinv) + (size_t)k * nv;
    const FastDiv dch((unsigned)CH);
    for (int r = lane; r < nv; r += 32) {   // every copy in flight at once
        const int q = r + (int)dch((unsigned)r);
        cp_async_elem(&sb[q], &line[r]);
        cp_async_elem(&sd[q], &dg[r]);
    }
}
// the solve of one mode by the calling warp out of its staged slices (the
// solution replaces the right-hand side in sb)
template <typename R>
__device__ __forceinline__ void tri_ws_solve(typename Cplx<R>::type* __restrict__ sb,
                                             const typename Cplx<R>::type* __restrict__ sd,
                                             const R* __restrict__ al, const R* __restrict__ ga,
                                             typename Cplx<R>::type lam, int nv) {
    using C = typename Cplx<R>::type;
    const int lane = threadIdx.x & 31;
    const int CH = (nv + 31) / 32;
    const int r0 = lane * CH;
    const int r1 = min(r0 + CH, nv);
    const int q0 = lane * (CH + 1);
    // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
    Aff<C> a;
    a.P = c_make<C>(1.0, 0.0);
    a.Q = c_make<C>(0.0, 0.0);
    for (int r = r0, q = q0; r < r1; ++r, ++q) {
        Aff<C> m;
        if (r == 0) m.P = c_make<C>(0.0, 0.0);
        else {
            const C dprev = sd[(r == r0) ? q - 2 : q - 1];   // r0-1 sits before the previous chunk's pad slot
            const C l = c_mul(c_rmul(lam, al[q]), dprev);
            m.P = c_make<C>(-l.x, -l.y);
        }
        m.Q = sb[q];
        a = aff_combine(a, m);
    }
    C y = warp_scan_aff<C>(a, true);
    for (int r = r0, q = q0; r < r1; ++r, ++q) {
        const C b = sb[q];
        if (r == 0) y = b;
        else {
            const C dprev = sd[(r == r0) ? q - 2 : q - 1];
            const C l = c_mul(c_rmul(lam, al[q]), dprev);
            y = c_sub(b, c_mul(l, y));
        }
        sb[q] = y;
    }
    // backward: x_r = U_r^-1 (y_r - c_r x_{r+1})  ==  mu_r + nu_r x_{r+1} (each lane reads its own chunk only)
    a.P = c_make<C>(1.0, 0.0);
    a.Q = c_make<C>(0.0, 0.0);
    for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
        Aff<C> m;
        const C d = sd[q];
        m.Q = c_mul(d, sb[q]);
        if (r == nv - 1) m.P = c_make<C>(0.0, 0.0);
        else {
            const C nu = c_mul(d, c_rmul(lam, ga[q]));
            m.P = c_make<C>(-nu.x, -nu.y);
        }
        a = aff_combine(a, m);
    }
    C x = warp_scan_aff<C>(a, false);
    for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
        const C d = sd[q];
        if (r == nv - 1) x = c_mul(d, sb[q]);
        else x = c_mul(d, c_sub(sb[q], c_mul(c_rmul(lam, ga[q]), x)));
        sb[q] = x;
    }
}

template <typename R>
__device__ __forceinline__ void tridiag_warp_staged(typename Cplx<R>::type* __restrict__ spec, const TriParams& p,
                                                    int k, typename Cplx<R>::type* __restrict__ sb,
                                                    const typename Cplx<R>::type* __restrict__ sd,
                                                    const R* __restrict__ al, const R* __restrict__ ga) {
    using C = typename Cplx<R>::type;
    const int lane = threadIdx.x & 31;
    const int nv = p.nv;
    const int CH = (nv + 31) / 32;
    C* line = spec + (size_t)k * nv;
    tri_ws_solve<R>(sb, sd, al, ga, reinterpret_cast<const C*>(p.lambda)[k], nv);
    __syncwarp();
    const FastDiv dch((unsigned)CH);
    for (int r = lane; r < nv; r += 32) line[r] = sb[r + (int)dch((unsigned)r)];
}

// dynamic smem: TRIW_WARPS x 2 x tri_ws_slots(nv) complex + 2 x tri_ws_slots(nv) real
template <typename R>
__global__ void __launch_bounds__(32 * TRIW_WARPS)
k_tridiag_warp_staged(typename Cplx<R>::type* __restrict__ spec, TriParams p) {
    using C = typename Cplx<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int w = threadIdx.x >> 5;
    const int k = blockIdx.x * TRIW_WARPS + w;
    const int ns = tri_ws_slots(p.nv);
    C* sb = reinterpret_cast<C*>(smem_raw) + (size_t)w * 2 * ns;
    R* sal = reinterpret_cast<R*>(reinterpret_cast<C*>(smem_raw) + (size_t)TRIW_WARPS * 2 * ns);
    R* sga = sal + ns;
    tri_ws_stage_tables<R>(p, sal, sga);
    if (k < p.nmodes) tri_ws_stage_line<R>(spec, p, k, sb, sb + ns);
    cp_async_commit();
    cp_async_wait0();
    __syncthreads();
    if (k < p.nmodes) tridiag_warp_staged<R>(spec, p, k, sb, sb + ns, sal, sga);
}

}  // namespace vv
