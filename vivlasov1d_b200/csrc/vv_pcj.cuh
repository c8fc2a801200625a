// Tensor-product kinetic preconditioner, v-major spectrum layout (the batch
// path's second layout): spec[j * (M + 1) + k] for velocity row j and x mode
// k = 0..M (M = nx/2).  Same operator as vv_pc.cuh (TensorProduct.pyx:
// 109-116 eigenvalues, TensorProductKineticFast.pyx:248-272 band matrix, LU
// without pivoting) with kernels shaped for the work instead of the layout:
//
//   x-FFTs  two-pass shared-memory Stockham FFT of the packed complex row
//           (M = P1 x P2): a P1-point DFT in registers per thread, the
//           twiddle W_M^(m2 k1), a P2-point DFT in registers; the register
//           DFTs use compile-time twiddles, the rows are read and written
//           whole (no transpose) and the real-FFT split is one more pass
//           through shared memory;
//   v-solve one lane per x mode, the LU forward and back substitution run
//           sequentially down the mode's column: a warp reads 32 consecutive
//           modes of a row (coalesced), the LU reciprocals come from a
//           v-major copy of the table (dinvJ[j * (M + 1) + k]); no scans.
#pragma once
#include "vv_common.cuh"
#include "vv_pc.cuh"

namespace vv {

// cos(k pi / 8) and sin(k pi / 8), k = 0..15 (values of the circle)
__host__ __device__ constexpr double cos_pi8(int k) {
    switch (k & 15) {
        case 0: return 1.0;
        case 1: return 0.92387953251128675613;
        case 2: return 0.70710678118654752440;
        case 3: return 0.38268343236508977173;
        case 4: return 0.0;
        case 5: return -0.38268343236508977173;
        case 6: return -0.70710678118654752440;
        case 7: return -0.92387953251128675613;
        case 8: return -1.0;
        case 9: return -0.92387953251128675613;
        case 10: return -0.70710678118654752440;
        case 11: return -0.38268343236508977173;
        case 12: return 0.0;
        case 13: return 0.38268343236508977173;
        case 14: return 0.70710678118654752440;
        default: return 0.92387953251128675613;
    }
}
__host__ __device__ constexpr double sin_pi8(int k) { return cos_pi8(k - 4); }

// v * exp(SIGN i pi k / 8), with the trivial angles done without multiplies
template <int SIGN, typename C>
VV_DEV C rot_pi8(C v, int k) {
    k &= 15;
    if (k == 0) return v;
    if (k == 8) return c_make<C>(-v.x, -v.y);
    if (k == 4) return SIGN > 0 ? c_make<C>(-v.y, v.x) : c_make<C>(v.y, -v.x);    // +-i v
    if (k == 12) return SIGN > 0 ? c_make<C>(v.y, -v.x) : c_make<C>(-v.y, v.x);   // -+i v
    using R = decltype(v.x);
    const R c = (R)cos_pi8(k), s = (R)(SIGN * sin_pi8(k));
    C r;
    r.x = v.x * c - v.y * s;
    r.y = v.x * s + v.y * c;
    return r;
}

// In-register DFT of P = 2, 4, 8 or 16 points, natural order in and out:
// X_k = sum_n a_n exp(SIGN 2 pi i n k / P) (radix-2, decimation in time).
template <int P, int SIGN, typename C>
VV_DEV void reg_dft(C (&a)[P]) {
    constexpr int B = clog2(P);
    static_assert(P >= 2 && P <= 16 && (P & (P - 1)) == 0, "register DFT of 2..16 points");
    C t[P];
#pragma unroll
    for (int j = 0; j < P; ++j) t[crev(j, B)] = a[j];
#pragma unroll
    for (int h = 1; h < P; h <<= 1) {
#pragma unroll
        for (int g = 0; g < P; g += 2 * h) {
#pragma unroll
            for (int pos = 0; pos < h; ++pos) {
                const C v = rot_pi8<SIGN>(t[g + pos + h], (8 * pos) / h);   // W_{2h}^pos
                const C u = t[g + pos];
                t[g + pos] = c_add(u, v);
                t[g + pos + h] = c_sub(u, v);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < P; ++j) a[j] = t[j];
}

constexpr int FJ_THREADS = 128;   // threads of the v-major FFT blocks

// factors of M and rows per work item (RB x P2 = FJ_THREADS threads in pass 1)
template <int M> struct FftJ;
template <> struct FftJ<32> { static constexpr int P1 = 8, P2 = 4; };
template <> struct FftJ<64> { static constexpr int P1 = 8, P2 = 8; };
template <> struct FftJ<128> { static constexpr int P1 = 16, P2 = 8; };
template <> struct FftJ<256> { static constexpr int P1 = 16, P2 = 16; };

// padded row strides (complex slots) of the two shared buffers: a row offset
// of P2 mod 16 slots keeps the rows a half-warp touches on distinct banks
__host__ __device__ constexpr int fj_pad(int base, int p2) { return p2 >= 16 ? base : base + ((p2 - base % 16 + 16) % 16); }
__host__ __device__ constexpr int fj_rows(int p2) { return FJ_THREADS / p2; }
__host__ __device__ constexpr int fj_sa(int p1, int p2) { return fj_pad(p1 * (p2 + 1), p2); }
__host__ __device__ constexpr int fj_sb(int m, int p2) { return fj_pad(m, p2); }
// shared memory of one block (complex slots): M twiddles + RB x SA + RB x SB
__host__ __device__ constexpr int fj_slots(int m, int p1, int p2) {
    return m + fj_rows(p2) * (fj_sa(p1, p2) + fj_sb(m, p2));
}
inline int fj_slots_of(int M) {
    switch (M) {
        case 32: return fj_slots(32, 8, 4);
        case 64: return fj_slots(64, 8, 8);
        case 128: return fj_slots(128, 16, 8);
        case 256: return fj_slots(256, 16, 16);
        default: return -1;
    }
}
inline int fj_rows_of(int M) {
    switch (M) {
        case 32: return fj_rows(4);
        case 64: case 128: return fj_rows(8);
        case 256: return fj_rows(16);
        default: return -1;
    }
}

template <typename T> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };

// Real FFT along x of rows [item*RB, item*RB + RB), half spectra written
// v-major: spec[j*(M+1) + k], k = 0..M.  load(r, j, n) returns the packed
// complex sample z_n = x_{2n} + i x_{2n+1} of row j = item*RB + r (j < nv);
// stw / A / B: the block's twiddle, pass-1 and pass-2 buffers, the twiddles
// staged and a barrier taken by the caller.
template <typename R, int M, typename Load>
VV_DEV void rfftj_rows(typename Cplx<R>::type* __restrict__ spec, const PcParams& p, int item,
                       const typename Cplx<R>::type* stw, typename Cplx<R>::type* A, typename Cplx<R>::type* B,
                       Load load) {
    using C = typename Cplx<R>::type;
    constexpr int P1 = FftJ<M>::P1, P2 = FftJ<M>::P2, RB = fj_rows(P2);
    constexpr int SA = fj_sa(P1, P2), SB = fj_sb(M, P2), H = M / 2 + 1;
    const int j0 = item * RB;
    {   // pass 1: thread = (row r, m2); z_n = x_{2n} + i x_{2n+1}, n = P2 m1 + m2
        const int r = threadIdx.x / P2, m2 = threadIdx.x % P2;
        const int j = j0 + r;
        C a[P1];
        if (j < p.nv) {
#pragma unroll
            for (int m1 = 0; m1 < P1; ++m1) a[m1] = load(r, j, P2 * m1 + m2);
        } else {
#pragma unroll
            for (int m1 = 0; m1 < P1; ++m1) a[m1] = c_make<C>(0.0, 0.0);
        }
        reg_dft<P1, -1>(a);
#pragma unroll
        for (int k1 = 1; k1 < P1; ++k1) a[k1] = c_mul(a[k1], tw_half<M, -1>(stw, m2 * k1));
        C* Ar = A + r * SA + m2;
#pragma unroll
        for (int k1 = 0; k1 < P1; ++k1) Ar[k1 * (P2 + 1)] = a[k1];
    }
    __syncthreads();
    // pass 2: unit = (row r, k1); Z_{k1 + P1 k2}
    for (int u = threadIdx.x; u < RB * P1; u += FJ_THREADS) {
        const int r = u / P1, k1 = u % P1;
        const C* Ar = A + r * SA + k1 * (P2 + 1);
        C b[P2];
#pragma unroll
        for (int m2 = 0; m2 < P2; ++m2) b[m2] = Ar[m2];
        reg_dft<P2, -1>(b);
        C* Br = B + r * SB + k1;
#pragma unroll
        for (int k2 = 0; k2 < P2; ++k2) Br[P1 * k2] = b[k2];
    }
    __syncthreads();
    // real split: unit = (row r, k), k = 0..M/2 writes X_k and X_{M-k}
    for (int u = threadIdx.x; u < RB * H; u += FJ_THREADS) {
        const int r = u / H, k = u % H;
        const int j = j0 + r;
        if (j >= p.nv) continue;
        const C* Br = B + r * SB;
        const int kc = M - k;
        const C zk = Br[k];
        const C zc = Br[k == 0 ? 0 : kc];
        const C zcc = c_conj(zc);
        C E1 = c_scale(c_add(zk, zcc), (decltype(zk.x))0.5);
        C D = c_sub(zk, zcc);
        const C outk = c_add(E1, c_mul(stw[k], c_make<C>(0.5 * D.y, -0.5 * D.x)));
        C* out = spec + (size_t)j * (M + 1);
        out[k] = outk;
        if (kc != k) {
            const C zkc = c_conj(zk);
            E1 = c_scale(c_add(zc, zkc), (decltype(zk.x))0.5);
            D = c_sub(zc, zkc);
            const C w = (kc < M) ? stw[kc] : c_make<C>(-1.0, 0.0);
            out[kc] = c_add(E1, c_mul(w, c_make<C>(0.5 * D.y, -0.5 * D.x)));
        }
    }
}

// Real FFT along x of rows [item*RB, item*RB + RB) of X (nv x nx, nx = 2M).
template <typename TI, typename R, int M>
VV_DEV void rfftj_block(const TI* __restrict__ X, typename Cplx<R>::type* __restrict__ spec, const PcParams& p,
                        int item) {
    using C = typename Cplx<R>::type;
    constexpr int P1 = FftJ<M>::P1, P2 = FftJ<M>::P2, RB = fj_rows(P2);
    constexpr int SA = fj_sa(P1, P2);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    C* A = stw + M;
    C* B = A + RB * SA;
    const C* tw = reinterpret_cast<const C*>(p.tw);
    for (int k = threadIdx.x; k < M; k += FJ_THREADS) stw[k] = tw[k];
    __syncthreads();
    rfftj_rows<R, M>(spec, p, item, stw, A, B, [&](int, int j, int nn) {
        const auto v = *reinterpret_cast<const typename Pair<TI>::type*>(X + (size_t)j * p.nx + 2 * nn);
        return c_make<C>((double)v.x, (double)v.y);
    });
}

// Inverse: half spectra spec[j*(M+1) + k] of rows [item*RB, item*RB + RB)
// -> rows of Y, normalised by 1/nx (numpy's irfft; the imaginary parts of
// X_0 and X_M are ignored).
template <typename R, typename TO, int M>
VV_DEV void irfftj_block(const typename Cplx<R>::type* __restrict__ spec, TO* __restrict__ Y, const PcParams& p,
                         int item) {
    using C = typename Cplx<R>::type;
    constexpr int P1 = FftJ<M>::P1, P2 = FftJ<M>::P2, RB = fj_rows(P2);
    constexpr int SA = fj_sa(P1, P2), SB = fj_sb(M, P2), H = M / 2 + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* stw = reinterpret_cast<C*>(smem_raw);
    C* A = stw + M;
    C* B = A + RB * SA;
    static_assert(SA >= M + 1 && RB % 2 == 0, "a row's half spectrum fits a pass-1 row; items start on even rows");
    const C* tw = reinterpret_cast<const C*>(p.tw);
    const int j0 = item * RB;
    {   // the item's half spectra are consecutive in the v-major layout: copy
        // them into A (free until pass 1; SA >= M + 1) with 16-byte cp.async,
        // every load in flight at once (j0 is even, so the source is 16-byte
        // aligned; an odd count of FP32 complex values leaves 8 bytes)
        const int rows = min(RB, p.nv - j0);
        const char* src = reinterpret_cast<const char*>(spec + (size_t)j0 * (M + 1));
        char* dst = reinterpret_cast<char*>(A);
        const int nb = rows * (M + 1) * (int)sizeof(C), n16 = nb / 16;
        for (int q = threadIdx.x; q < n16; q += FJ_THREADS) cp_async_16(dst + 16 * q, src + 16 * q, 16);
        if (threadIdx.x == 0 && (nb & 15)) cp_async_8(dst + 16 * n16, src + 16 * n16, 8);
        cp_async_commit();
    }
    for (int k = threadIdx.x; k < M; k += FJ_THREADS) stw[k] = tw[k];
    cp_async_wait0();
    __syncthreads();
    // unpack: Z_k = E + i O, E = (X_k + conj X_{M-k})/2, O = W_N^-k (X_k - conj X_{M-k})/2
    for (int u = threadIdx.x; u < RB * H; u += FJ_THREADS) {
        const int r = u / H, k = u % H;
        const int j = j0 + r;
        const int kc = M - k;
        C xk = c_make<C>(0.0, 0.0), xc = xk;
        if (j < p.nv) {
            const C* in = A + r * (M + 1);
            xk = in[k];
            xc = in[kc];
        }
        if (k == 0) {
            xk.y = 0;
            xc.y = 0;
        }
        C* Br = B + r * SB;
        {
            const C cc = c_conj(xc);
            const C E1 = c_scale(c_add(xk, cc), (decltype(xk.x))0.5);
            C w = stw[k];
            w.y = -w.y;
            const C O = c_mul(w, c_scale(c_sub(xk, cc), (decltype(xk.x))0.5));
            Br[k] = c_make<C>(E1.x - O.y, E1.y + O.x);
        }
        if (k != 0 && kc != k) {
            const C cc = c_conj(xk);
            const C E1 = c_scale(c_add(xc, cc), (decltype(xk.x))0.5);
            C w = stw[kc];
            w.y = -w.y;
            const C O = c_mul(w, c_scale(c_sub(xc, cc), (decltype(xk.x))0.5));
            Br[kc] = c_make<C>(E1.x - O.y, E1.y + O.x);
        }
    }
    __syncthreads();
    {   // pass 1 (inverse): thread = (row r, m2)
        const int r = threadIdx.x / P2, m2 = threadIdx.x % P2;
        const C* Br = B + r * SB + m2;
        C a[P1];
#pragma unroll
        for (int m1 = 0; m1 < P1; ++m1) a[m1] = Br[P2 * m1];
        reg_dft<P1, +1>(a);
#pragma unroll
        for (int k1 = 1; k1 < P1; ++k1) a[k1] = c_mul(a[k1], tw_half<M, +1>(stw, m2 * k1));
        C* Ar = A + r * SA + m2;
#pragma unroll
        for (int k1 = 0; k1 < P1; ++k1) Ar[k1 * (P2 + 1)] = a[k1];
    }
    __syncthreads();
    using RR = decltype(stw[0].x);
    const RR s = (RR)(1.0 / (double)M);
    for (int u = threadIdx.x; u < RB * P1; u += FJ_THREADS) {
        const int r = u / P1, k1 = u % P1;
        const int j = j0 + r;
        const C* Ar = A + r * SA + k1 * (P2 + 1);
        C b[P2];
#pragma unroll
        for (int m2 = 0; m2 < P2; ++m2) b[m2] = Ar[m2];
        reg_dft<P2, +1>(b);
        if (j < p.nv) {
            TO* row = Y + (size_t)j * p.nx;
#pragma unroll
            for (int k2 = 0; k2 < P2; ++k2) {
                typename Pair<TO>::type o;
                o.x = (TO)(b[k2].x * s);
                o.y = (TO)(b[k2].y * s);
                *reinterpret_cast<typename Pair<TO>::type*>(row + 2 * (k1 + P1 * k2)) = o;
            }
        }
    }
}

// LU solve of mode k (one lane) down its column of the v-major spectrum:
// forward y_j = b_j - lambda alpha_j U_{j-1}^-1 y_{j-1}, back substitution
// x_j = U_j^-1 (y_j - lambda gamma_j x_{j+1}), in place.  The sweep is a
// dependent chain per lane, so the lane streams its column through a private
// ring of TJ_RING rows in shared memory that cp.async keeps TJ_NCH chunks of
// TJ_CHK rows ahead (the copies of a lane are its own: no barrier).  ring:
// 32 lanes x TJ_RING rows x 2 complex (value, LU reciprocal) per warp.
constexpr int TJ_CHK = 8, TJ_NCH = 8, TJ_RING = TJ_CHK * TJ_NCH;

template <typename R>
VV_DEV void tridiagj_lane(typename Cplx<R>::type* __restrict__ spec, const typename Cplx<R>::type* __restrict__ dinvJ,
                          const TriParams& p, int k, typename Cplx<R>::type* __restrict__ ring) {
    using C = typename Cplx<R>::type;
    const int lane = threadIdx.x & 31;
    const bool on = k < p.nmodes;
    const int nm = p.nmodes, nv = p.nv;
    const R* al = reinterpret_cast<const R*>(p.alpha);
    const R* ga = reinterpret_cast<const R*>(p.gamma);
    const C lam = on ? reinterpret_cast<const C*>(p.lambda)[k] : c_make<C>(0.0, 0.0);
    C* col = spec + k;
    const C* dcol = dinvJ + k;
    C* rv = ring + lane;                 // slot s: value at rv[64 s], LU reciprocal at rv[64 s + 32]
    const int nch = (nv + TJ_CHK - 1) / TJ_CHK;
    // chunk c of the forward sweep holds rows c*CHK.., of the backward sweep rows nv-1-c*CHK down
    auto issue = [&](int c, bool fwd) {
        if (on && c < nch) {
#pragma unroll
            for (int u = 0; u < TJ_CHK; ++u) {
                const int i = c * TJ_CHK + u;
                const int j = fwd ? i : nv - 1 - i;
                if (i < nv) {
                    const int s = i % TJ_RING;
                    cp_async_elem(&rv[64 * s], &col[(size_t)j * nm]);
                    cp_async_elem(&rv[64 * s + 32], &dcol[(size_t)j * nm]);
                }
            }
        }
        cp_async_commit();
    };
    // forward
#pragma unroll
    for (int c = 0; c < TJ_NCH; ++c) issue(c, true);
    C y = c_make<C>(0.0, 0.0), dprev = y;
    for (int c = 0; c < nch; ++c) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(TJ_NCH - 1) : "memory");
#pragma unroll
        for (int u = 0; u < TJ_CHK; ++u) {
            const int j = c * TJ_CHK + u;
            if (j < nv) {
                const int s = j % TJ_RING;
                const C b = rv[64 * s];
                if (j == 0) y = b;
                else {
                    const C l = c_mul(c_rmul(lam, al[j]), dprev);
                    y = c_sub(b, c_mul(l, y));
                }
                dprev = rv[64 * s + 32];
                if (on) col[(size_t)j * nm] = y;
            }
        }
        issue(c + TJ_NCH, true);
    }
    cp_async_wait0();
    // the back substitution reads y through cp.async, which is not ordered
    // after this thread's plain stores of y without a fence
    __threadfence();
#pragma unroll
    for (int c = 0; c < TJ_NCH; ++c) issue(c, false);
    C x = c_make<C>(0.0, 0.0);
    for (int c = 0; c < nch; ++c) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(TJ_NCH - 1) : "memory");
#pragma unroll
        for (int u = 0; u < TJ_CHK; ++u) {
            const int i = c * TJ_CHK + u;
            if (i < nv) {
                const int j = nv - 1 - i;
                const int s = i % TJ_RING;
                const C yv = rv[64 * s];
                const C d = rv[64 * s + 32];
                if (i == 0) x = c_mul(d, yv);
                else x = c_mul(d, c_sub(yv, c_mul(c_rmul(lam, ga[j]), x)));
                if (on) col[(size_t)j * nm] = x;
            }
        }
        issue(c + TJ_NCH, false);
    }
    cp_async_wait0();
}

}  // namespace vv
