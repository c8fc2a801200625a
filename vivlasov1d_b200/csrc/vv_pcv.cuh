// Tensor-product potential preconditioner (`tensor_potential`):
// TensorProductPotential.pyx:157-183 (the FFT - solve - iFFT sequence),
// TensorProductPotentialFast.pyx:43-266 (FFT along v, banded matrices from
// phi, zgbtrf/zgbtrs with KL = KU = 1), eigenvalues TensorProduct.pyx:109-116
// for n = nv.
//
//   P^-1 X = irFFT_v [ A_k^-1 (rFFT_v X)_k ],  k = 0..nv/2,
//
// A_k (nx x nx, tridiagonal, no periodic corner entries):
//   A[i][i-1] = lambda_k (phi_i - phi_{i-1}) a,
//   A[i][i]   = lambda_k 2 (phi_{i+1} - phi_{i-1}) a + 1/ht,
//   A[i][i+1] = lambda_k (phi_{i+1} - phi_i) a,     a = hx^-1 hv^-1 / 24,
// with periodic differences of phi, built from the phi of make_history.
//
// The v transforms run as the x-row kernels on the transposed field (rows of
// length nv); A_k is solved by Gaussian elimination with partial pivoting
// (the pivot rule of LAPACK's band LU: swap when |sub|_1 > |diag|_1), one
// thread per mode, rebuilt at every application from phi.
#pragma once
#include "vv_common.cuh"

namespace vv {

// dst[c*rows + r] = src[r*cols + c] (rows x cols -> cols x rows), 32 x 32
// tiles through shared memory, block (32, 8); dst may be a GMRES basis base
// pointer: dst += (*yidx + yoff) * ystride
template <typename TI, typename TO>
__global__ void k_transpose(const TI* __restrict__ src, TO* __restrict__ dst, int rows, int cols,
                            const int* __restrict__ yidx, int yoff, size_t ystride) {
    __shared__ TO t[32][33];
    if (yidx) dst += (size_t)(*yidx + yoff) * ystride;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[k][threadIdx.x] = (TO)src[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) dst[(size_t)c * rows + r] = t[threadIdx.x][k];
    }
}

struct PotParams {
    int nx, nmv;           // x points, v modes (nv/2 + 1)
    double arak, ht_inv;   // hx^-1 hv^-1 / 24, 1/ht
    const double* phi;     // nx: the potential of make_history
    const double2* lam;    // nmv: shifted eigenvalues for n = nv
};

template <typename C>
VV_DEV double c_abs1(C a) { return fabs((double)a.x) + fabs((double)a.y); }
template <typename C>
VV_DEV C c_div(C a, C b) {
    using R = decltype(a.x);
    const R den = b.x * b.x + b.y * b.y;
    C r;
    r.x = (a.x * b.x + a.y * b.y) / den;
    r.y = (a.y * b.x - a.x * b.y) / den;
    return r;
}

// A_k c = b for mode k = one thread, in place on spec[k*nx ..]; scr holds the
// thread's diagonal, super- and (fill-in) second super-diagonal, 3 nx complex.
// Elimination with partial pivoting as in a tridiagonal solver with row
// interchanges (the fill-in of an interchange sits in dl), then back
// substitution.
template <typename R>
__global__ void k_pcv_solve(typename Cplx<R>::type* __restrict__ spec, typename Cplx<R>::type* __restrict__ scr,
                            PotParams p) {
    using C = typename Cplx<R>::type;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.nmv) return;
    const int n = p.nx;
    C* b = spec + (size_t)k * n;
    C* d = scr + (size_t)k * 3 * n;
    C* du = d + n;
    C* dl = du + n;
    const double2 lam = p.lam[k];
    // bands (TensorProductPotentialFast.pyx:228-260): dl[i] = A[i+1][i], du[i] = A[i][i+1]
    for (int i = 0; i < n; ++i) {
        const int im = i == 0 ? n - 1 : i - 1, ip = i + 1 == n ? 0 : i + 1;
        const double2 dg = c_rmul(c_rmul(c_rmul(lam, 2.0), p.phi[ip] - p.phi[im]), p.arak);
        d[i] = c_make<C>(dg.x + p.ht_inv, dg.y);
        if (i + 1 < n) {
            const double2 up = c_rmul(c_rmul(c_rmul(lam, 1.0), p.phi[ip] - p.phi[i]), p.arak);
            const int i1 = i + 1, i1m = i;
            const double2 lo = c_rmul(c_rmul(c_rmul(lam, 1.0), p.phi[i1] - p.phi[i1m]), p.arak);
            du[i] = c_make<C>(up.x, up.y);
            dl[i] = c_make<C>(lo.x, lo.y);
        }
    }
    const C zero = c_make<C>(0.0, 0.0);
    for (int i = 0; i + 1 < n; ++i) {
        const bool last = i + 2 == n;
        if (c_abs1(d[i]) >= c_abs1(dl[i])) {   // no interchange
            const C fact = c_div(dl[i], d[i]);
            d[i + 1] = c_sub(d[i + 1], c_mul(fact, du[i]));
            b[i + 1] = c_sub(b[i + 1], c_mul(fact, b[i]));
            if (!last) dl[i] = zero;
        } else {                                   // rows i and i+1 interchanged
            const C fact = c_div(d[i], dl[i]);
            d[i] = dl[i];
            const C temp = d[i + 1];
            d[i + 1] = c_sub(du[i], c_mul(fact, temp));
            if (!last) {
                dl[i] = du[i + 1];
                du[i + 1] = c_make<C>(-(fact.x * dl[i].x - fact.y * dl[i].y), -(fact.x * dl[i].y + fact.y * dl[i].x));
            }
            du[i] = temp;
            const C tb = b[i];
            b[i] = b[i + 1];
            b[i + 1] = c_sub(tb, c_mul(fact, b[i + 1]));
        }
    }
    b[n - 1] = c_div(b[n - 1], d[n - 1]);
    if (n > 1) b[n - 2] = c_div(c_sub(b[n - 2], c_mul(du[n - 2], b[n - 1])), d[n - 2]);
    for (int i = n - 3; i >= 0; --i)
        b[i] = c_div(c_sub(c_sub(b[i], c_mul(du[i], b[i + 1])), c_mul(dl[i], b[i + 2])), d[i]);
}

}  // namespace vv
