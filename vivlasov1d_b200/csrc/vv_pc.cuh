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
    int R;                 // rows per CTA in the row kernels
    const double2* tw;     // tw[k] = exp(-2 pi i k / nx), k < nx/2
    const int* yidx;       // optional: output is Y + (*yidx + yoff) * ystride
    int yoff;
    size_t ystride;
};

// In-place radix-2 DIT FFT of R rows of length M stored bit-reversed in smem.
// `stw` is the twiddle table exp(-2 pi i k / (2M)), k < M, in shared memory.
// sign = -1 forward, +1 inverse (unnormalised).
template <int SIGN>
__device__ __forceinline__ void smem_fft(double2* buf, int R, int M, const double2* stw) {
    const int nthr = blockDim.x;
    const int nb = R * (M >> 1);
    for (int half = 1; half < M; half <<= 1) {
        const int tstride = M / half;  // W_M^(pos*M/(2 half)) = stw[pos*M/half]
        for (int b = threadIdx.x; b < nb; b += nthr) {
            const int row = b / (M >> 1);
            const int bb = b - row * (M >> 1);
            const int grp = bb / half;
            const int pos = bb - grp * half;
            const int i0 = row * M + grp * 2 * half + pos;
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

__device__ __forceinline__ int bitrev(int m, int logM) {
    return logM == 0 ? 0 : (int)(__brev((unsigned)m) >> (32 - logM));
}

__device__ __forceinline__ void load_twiddles(double2* stw, const double2* __restrict__ tw, int M) {
    for (int k = threadIdx.x; k < M; k += blockDim.x) stw[k] = tw[k];
}

// rows j0 .. j0+R-1 of X -> spec[k*nv + j] for k = 0..M
// dynamic smem: [M twiddles][R*M buffer]
template <typename T>
__global__ void k_rfft_rows(const T* __restrict__ X, double2* __restrict__ spec, PcParams p) {
    extern __shared__ double2 smem[];
    const int M = p.M;
    double2* stw = smem;
    double2* buf = smem + M;
    const int j0 = blockIdx.x * p.R;
    const int nrow = min(p.R, p.nv - j0);
    load_twiddles(stw, p.tw, M);
    for (int idx = threadIdx.x; idx < p.R * M; idx += blockDim.x) {
        const int r = idx / M, m = idx - r * M;
        double2 z = make_double2(0.0, 0.0);
        if (r < nrow) {
            const T* row = X + (size_t)(j0 + r) * p.nx;
            z = make_double2((double)row[2 * m], (double)row[2 * m + 1]);
        }
        buf[r * M + bitrev(m, p.logM)] = z;
    }
    __syncthreads();
    smem_fft<-1>(buf, p.R, M, stw);
    // split: X_k = E_k + W_N^k O_k,  E = (Z_k + conj Z_{M-k})/2,  O = -i/2 (Z_k - conj Z_{M-k})
    for (int idx = threadIdx.x; idx < (M + 1) * p.R; idx += blockDim.x) {
        const int k = idx / p.R, r = idx - k * p.R;
        if (r >= nrow) continue;
        const double2 zk = buf[r * M + (k == M ? 0 : k)];
        const double2 zc = c_conj(buf[r * M + (k == 0 ? 0 : M - k)]);
        const double2 E = c_scale(c_add(zk, zc), 0.5);
        const double2 D = c_sub(zk, zc);
        const double2 O = make_double2(0.5 * D.y, -0.5 * D.x);  // -i/2 * D
        const double2 w = (k < M) ? stw[k] : make_double2(-1.0, 0.0);   // W_N^M = -1
        spec[(size_t)k * p.nv + j0 + r] = c_add(E, c_mul(w, O));
    }
}

// spec[k*nv + j] (k = 0..M) -> rows of Y, scaled by 1/nx
// dynamic smem: [M twiddles][R*M buffer][R*(M+1) spectrum]
template <typename T>
__global__ void k_irfft_rows(const double2* __restrict__ spec, T* __restrict__ Y, PcParams p) {
    if (p.yidx) Y += (size_t)(*p.yidx + p.yoff) * p.ystride;
    extern __shared__ double2 smem[];
    const int M = p.M;
    double2* stw = smem;
    double2* buf = smem + M;
    double2* xs = buf + p.R * M;
    const int j0 = blockIdx.x * p.R;
    const int nrow = min(p.R, p.nv - j0);
    load_twiddles(stw, p.tw, M);
    for (int idx = threadIdx.x; idx < (M + 1) * p.R; idx += blockDim.x) {
        const int k = idx / p.R, r = idx - k * p.R;
        double2 v = make_double2(0.0, 0.0);
        if (r < nrow) v = spec[(size_t)k * p.nv + j0 + r];
        if (k == 0 || k == M) v.y = 0.0;   // c2r ignores these imaginary parts
        xs[r * (M + 1) + k] = v;
    }
    __syncthreads();
    // Z_k = (X_k + conj X_{M-k})/2 + i W_N^{-k} (X_k - conj X_{M-k})/2
    for (int idx = threadIdx.x; idx < p.R * M; idx += blockDim.x) {
        const int r = idx / M, k = idx - r * M;
        const double2 xk = xs[r * (M + 1) + k];
        const double2 xc = c_conj(xs[r * (M + 1) + (M - k)]);
        const double2 E = c_scale(c_add(xk, xc), 0.5);
        double2 w = stw[k];
        w.y = -w.y;                            // W_N^{-k}
        const double2 O = c_mul(w, c_scale(c_sub(xk, xc), 0.5));
        buf[r * M + bitrev(k, p.logM)] = make_double2(E.x - O.y, E.y + O.x);  // E + i O
    }
    __syncthreads();
    smem_fft<+1>(buf, p.R, M, stw);
    const double s = 1.0 / (double)M;   // (1/M) IDFT_M gives the 1/nx-normalised irfft
    for (int idx = threadIdx.x; idx < p.R * M; idx += blockDim.x) {
        const int r = idx / M, m = idx - r * M;
        if (r >= nrow) continue;
        const double2 z = buf[r * M + m];
        T* row = Y + (size_t)(j0 + r) * p.nx;
        row[2 * m] = (T)(z.x * s);
        row[2 * m + 1] = (T)(z.y * s);
    }
}

// ---------------------------------------------------------------------------
// tridiagonal solves, one CTA per x mode
// ---------------------------------------------------------------------------
struct TriParams {
    int nv, nmodes;
    const double2* lambda;  // per mode eigenvalue lambda_k (shifted, TensorProduct.pyx:109-116)
    const double* alpha;    // nv: sub-diagonal  A[r,r-1] = lambda * alpha[r]
    const double* gamma;    // nv: super-diagonal A[r,r+1] = lambda * gamma[r]
    const double2* dinv;    // nmodes*nv: 1 / U[r,r] of the LU factors
};

constexpr int TRI_THREADS = 256;

// affine map x -> P x + Q on complex numbers; combine(first, second) = second o first
struct Aff { double2 P, Q; };
VV_DEV Aff aff_combine(const Aff& first, const Aff& second) {
    Aff r;
    r.P = c_mul(second.P, first.P);
    r.Q = c_add(c_mul(second.P, first.Q), second.Q);
    return r;
}
VV_DEV Aff shfl_aff(const Aff& a, int d, bool up) {
    Aff r;
    if (up) {
        r.P.x = __shfl_up_sync(0xffffffffu, a.P.x, d);
        r.P.y = __shfl_up_sync(0xffffffffu, a.P.y, d);
        r.Q.x = __shfl_up_sync(0xffffffffu, a.Q.x, d);
        r.Q.y = __shfl_up_sync(0xffffffffu, a.Q.y, d);
    } else {
        r.P.x = __shfl_down_sync(0xffffffffu, a.P.x, d);
        r.P.y = __shfl_down_sync(0xffffffffu, a.P.y, d);
        r.Q.x = __shfl_down_sync(0xffffffffu, a.Q.x, d);
        r.Q.y = __shfl_down_sync(0xffffffffu, a.Q.y, d);
    }
    return r;
}

// Exclusive scan of affine maps across the block in thread order `pos`
// (pos = tid for the forward sweep, nthreads-1-tid for the backward sweep;
// both keep warps intact).  Returns the image of 0 under the composition of
// all earlier chunks.
__device__ double2 block_scan_aff(Aff a, bool forward, Aff* sh) {
    const int pos = forward ? (int)threadIdx.x : TRI_THREADS - 1 - (int)threadIdx.x;
    const int lane = pos & 31, wid = pos >> 5;
    Aff inc = a;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Aff o = shfl_aff(inc, d, forward);   // the lane d earlier in pos order
        if (lane >= d) inc = aff_combine(o, inc);
    }
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    Aff pre;
    pre.P = make_double2(1.0, 0.0);
    pre.Q = make_double2(0.0, 0.0);
    for (int w = 0; w < wid; ++w) pre = aff_combine(pre, sh[w]);
    const Aff prev = shfl_aff(inc, 1, forward);
    Aff ex = pre;
    if (lane > 0) ex = aff_combine(pre, prev);
    __syncthreads();
    return ex.Q;
}

// One CTA per x mode.  STAGE: the mode's LU reciprocals and the alpha/gamma
// tables are staged in shared memory (nv <= 4096); otherwise read from L2.
// dynamic smem: [nv rhs][nv dinv][nv alpha][nv gamma] (the last three only if STAGE)
template <bool STAGE>
__global__ void __launch_bounds__(TRI_THREADS)
k_tridiag_modes(double2* __restrict__ spec, TriParams p) {
    extern __shared__ double2 sm[];
    __shared__ Aff shw[TRI_THREADS / 32];
    const int k = blockIdx.x;
    const int nv = p.nv;
    double2* b = sm;
    double2* line = spec + (size_t)k * nv;
    const double2* dinv_g = p.dinv + (size_t)k * nv;
    const double2* dinv = STAGE ? sm + nv : dinv_g;
    const double* alpha = STAGE ? reinterpret_cast<const double*>(sm + 2 * nv) : p.alpha;
    const double* gamma = STAGE ? reinterpret_cast<const double*>(sm + 2 * nv) + nv : p.gamma;
    const double2 lam = p.lambda[k];
    for (int r = threadIdx.x; r < nv; r += TRI_THREADS) {
        b[r] = line[r];
        if (STAGE) {
            sm[nv + r] = dinv_g[r];
            reinterpret_cast<double*>(sm + 2 * nv)[r] = p.alpha[r];
            reinterpret_cast<double*>(sm + 2 * nv)[nv + r] = p.gamma[r];
        }
    }
    __syncthreads();
    const int C = (nv + TRI_THREADS - 1) / TRI_THREADS;
    const int r0 = threadIdx.x * C;
    const int r1 = min(r0 + C, nv);
    // forward: y_r = b_r - l_r y_{r-1},  l_r = lambda alpha_r / U_{r-1}
    Aff a;
    a.P = make_double2(1.0, 0.0);
    a.Q = make_double2(0.0, 0.0);
    for (int r = r0; r < r1; ++r) {
        Aff m;
        if (r == 0) m.P = make_double2(0.0, 0.0);
        else {
            const double2 l = c_mul(c_rmul(lam, alpha[r]), dinv[r - 1]);
            m.P = make_double2(-l.x, -l.y);
        }
        m.Q = b[r];
        a = aff_combine(a, m);
    }
    double2 y = block_scan_aff(a, true, shw);
    for (int r = r0; r < r1; ++r) {
        if (r == 0) y = b[0];
        else {
            const double2 l = c_mul(c_rmul(lam, alpha[r]), dinv[r - 1]);
            y = c_sub(b[r], c_mul(l, y));
        }
        b[r] = y;
    }
    __syncthreads();
    // backward: x_r = U_r^-1 (y_r - c_r x_{r+1})  ==  mu_r + nu_r x_{r+1}
    a.P = make_double2(1.0, 0.0);
    a.Q = make_double2(0.0, 0.0);
    for (int r = r1 - 1; r >= r0; --r) {
        Aff m;
        const double2 di = dinv[r];
        m.Q = c_mul(di, b[r]);
        if (r == nv - 1) m.P = make_double2(0.0, 0.0);
        else {
            const double2 nu = c_mul(di, c_rmul(lam, gamma[r]));
            m.P = make_double2(-nu.x, -nu.y);
        }
        a = aff_combine(a, m);
    }
    double2 x = block_scan_aff(a, false, shw);
    for (int r = r1 - 1; r >= r0; --r) {
        const double2 di = dinv[r];
        if (r == nv - 1) x = c_mul(di, b[r]);
        else {
            const double2 c = c_rmul(lam, gamma[r]);
            x = c_mul(di, c_sub(b[r], c_mul(c, x)));
        }
        line[r] = x;
    }
}

}  // namespace vv
