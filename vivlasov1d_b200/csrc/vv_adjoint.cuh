// Discrete adjoint of the converged implicit step (FP64).
//
// A converged step F = Phi(f) satisfies G(F, f) = (F - f)/ht +
// M J((F + f)/2, H(F, f)) = 0 with H = h0 + (h1(F) + h1(f) + h2p + h2h)/2,
// h1 = L u the moments -> Poisson -> mean-removal chain and M the interior
// rows 2 <= j < nv-2 (PETScNLVlasovMP.pyx:43-58, PoissonBracket.pyx:335-389,
// Toolbox.pyx:38-74).  Its coupled Jacobian is
//   A u = u/ht + 1/2 M J(u, H) + 1/2 M J(Fbar, E L u),   Fbar = (F + f)/2,
// and since dG/df = A - (2/ht) I, a gradient gF with respect to F pulls back
// to gf = -gF + (2/ht) lambda with A^T lambda = gF, where
//   A^T lambda = lambda/ht + 1/2 J_H^T lambda - 1/2 L^T E^T J_Fbar^T lambda
// (J(x, h) = -J(h, x) pointwise for the Arakawa forms; J_h^T is the transpose
// of x -> M J(x, h); L^T p = hv E[-charge (I - mean) Pois^-1 (I - mean) p]).
// The transposes are built from the bracket's stencil form: for fixed h,
// M J(x, h)(i, j) = sum_t c_t(i, j) x(i + di_t, j + dj_t) over 12 offsets,
// the coefficients c_t formed term by term from the J1/J2 formulas
// (PoissonBracket.pyx:100-111, 221-232); then
//   J_h^T y (p) = sum_t c_t(p - off_t) y(p - off_t).
// The linear solve is preconditioned by P^-T = F^-1 diag(A_k^-H) F: the
// kinetic preconditioner with each mode's tridiagonal solve conjugate-
// transposed, from the same LU factors.
#pragma once
#include "vv_common.cuh"
#include "vv_pc.cuh"
#include "vv_vec.cuh"

namespace vv {

constexpr int ADJ_NOFF = 12;
// offsets (di, dj) of the stencil form, in the order of the coefficient planes
__host__ __device__ constexpr int adj_di(int t) {
    return t == 0 ? 1 : t == 1 ? -1 : t == 4 ? 1 : t == 5 ? -1 : t == 6 ? -1 : t == 7 ? 1 : t == 8 ? 2 : t == 9 ? -2 : 0;
}
__host__ __device__ constexpr int adj_dj(int t) {
    return t == 2 ? 1 : t == 3 ? -1 : t == 4 ? 1 : t == 5 ? -1 : t == 6 ? 1 : t == 7 ? -1 : t == 10 ? 2 : t == 11 ? -2 : 0;
}

struct AdjParams {
    int nx, nv;
    size_t ncell;
    double ht_inv, f1, f2, hv;
};

// Coefficient planes c_t (t < 12, plane stride ncell) of x -> M J(x, h) for
// h = h0(v) + hprof(x) (HK = 0, the separable Hamiltonian) or h = (F + f)/2
// (HK = 1); zero on the masked rows.  Grid: (ceil(nx/256), nv).
template <int SCHEME, int HK>
__global__ void k_adj_coef(AdjParams p, const double* __restrict__ h0, const double* __restrict__ hprof,
                           const double* __restrict__ F, const double* __restrict__ f, double* __restrict__ coef) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int nx = p.nx, nv = p.nv;
    if (i >= nx) return;
    double* c = coef + (size_t)j * nx + i;
    double cc[ADJ_NOFF];
#pragma unroll
    for (int t = 0; t < ADJ_NOFF; ++t) cc[t] = 0.0;
    if (j >= 2 && j < nv - 2) {
        auto H = [&](int di, int dj) -> double {
            int ii = i + di;
            ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
            const int jj = j + dj;
            if (HK == 0) return h0[jj] + hprof[ii];
            const size_t q = (size_t)jj * nx + ii;
            return 0.5 * F[q] + 0.5 * f[q];
        };
        if (SCHEME == 1 || SCHEME == 4) {
            const double a = p.f1 * (SCHEME == 4 ? 2.0 : 1.0);
            const double A = H(0, 1) - H(0, -1), B = H(1, 0) - H(-1, 0);
            cc[0] += a * A; cc[1] -= a * A; cc[2] -= a * B; cc[3] += a * B;                           // jpp
            cc[0] += a * (H(1, 1) - H(1, -1)); cc[1] -= a * (H(-1, 1) - H(-1, -1));                   // jpc
            cc[2] -= a * (H(1, 1) - H(-1, 1)); cc[3] += a * (H(1, -1) - H(-1, -1));
            cc[4] += a * (H(0, 1) - H(1, 0)); cc[5] -= a * (H(-1, 0) - H(0, -1));                     // jcp
            cc[6] -= a * (H(0, 1) - H(-1, 0)); cc[7] += a * (H(1, 0) - H(0, -1));
        }
        if (SCHEME == 2 || SCHEME == 4) {
            const double a = p.f2 * (SCHEME == 4 ? -1.0 : 1.0);
            const double C = H(-1, 1) - H(1, -1), D = H(1, 1) - H(-1, -1);
            cc[4] += a * C; cc[5] -= a * C; cc[6] -= a * D; cc[7] += a * D;                           // jcc
            cc[8] += a * (H(1, 1) - H(1, -1)); cc[9] -= a * (H(-1, 1) - H(-1, -1));                   // jpc
            cc[10] -= a * (H(1, 1) - H(-1, 1)); cc[11] += a * (H(1, -1) - H(-1, -1));
            cc[4] += a * (H(0, 2) - H(2, 0)); cc[5] -= a * (H(-2, 0) - H(0, -2));                     // jcp
            cc[6] -= a * (H(0, 2) - H(-2, 0)); cc[7] += a * (H(2, 0) - H(0, -2));
        }
    }
#pragma unroll
    for (int t = 0; t < ADJ_NOFF; ++t) c[(size_t)t * p.ncell] = cc[t];
}

constexpr int ADJ_TX = 32, ADJ_TY = 8;

// out = y/ht + 1/2 J_H^T y, and the v-sums of z = J_Fbar^T y per segment:
// zpart[s * nx + i] (segments of `seg` rows).  Grid (ceil(nx/32), S).
// y may be a GMRES basis base pointer with yidx -> the vector index.
__global__ void __launch_bounds__(ADJ_TX * ADJ_TY)
k_adj_apply(AdjParams p, const double* __restrict__ cH, const double* __restrict__ cF, const double* __restrict__ y,
            const int* __restrict__ yidx, double* __restrict__ out, int seg, double* __restrict__ zpart) {
    __shared__ double sz[ADJ_TY][ADJ_TX + 1];
    if (yidx) y += (size_t)(*yidx) * p.ncell;
    const int nx = p.nx, nv = p.nv;
    const int i = blockIdx.x * ADJ_TX + threadIdx.x;
    const int ja = blockIdx.y * seg, jb = min(nv, ja + seg);
    double zacc = 0.0;
    if (i < nx) {
        for (int j = ja + threadIdx.y; j < jb; j += ADJ_TY) {
            double aH = 0.0, aF = 0.0;
#pragma unroll
            for (int t = 0; t < ADJ_NOFF; ++t) {
                const int jj = j - adj_dj(t);
                if (jj < 2 || jj >= nv - 2) continue;   // the coefficients vanish on the masked rows
                int ii = i - adj_di(t);
                ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
                const size_t q = (size_t)jj * nx + ii;
                const double yv = __ldg(y + q);
                aH += __ldg(cH + (size_t)t * p.ncell + q) * yv;
                aF += __ldg(cF + (size_t)t * p.ncell + q) * yv;
            }
            const size_t g = (size_t)j * nx + i;
            out[g] = y[g] * p.ht_inv + 0.5 * aH;
            zacc += aF;
        }
    }
    sz[threadIdx.y][threadIdx.x] = zacc;
    __syncthreads();
    if (threadIdx.y == 0 && i < nx) {
        double t = 0.0;
        for (int r = 0; r < ADJ_TY; ++r) t += sz[r][threadIdx.x];
        zpart[(size_t)blockIdx.y * nx + i] = t;
    }
}

// One CTA: z = sum of the segment partials, q = -charge (I - mean) Pois^-1
// (I - mean) z (the Poisson chain of moments_poisson_cta with n = z).
// dynamic smem: as k_moments_poisson.
__global__ void __launch_bounds__(POIS_THREADS)
k_adj_poisson(const double* __restrict__ zpart, int S, double* __restrict__ zbuf, double* __restrict__ q,
              PoissonParams po) {
    for (int i = threadIdx.x; i < po.nx; i += blockDim.x) {
        double t = 0.0;
        for (int s = 0; s < S; ++s) t += zpart[(size_t)s * po.nx + i];
        zbuf[i] = t;
    }
    __syncthreads();
    moments_poisson_cta(nullptr, zbuf, nullptr, nullptr, nullptr, nullptr, nullptr, q, nullptr, po);
}

// out_ij -= 1/2 hv q_i (the broadcast of L^T), every row
__global__ void k_adj_bcast(AdjParams p, const double* __restrict__ q, double* __restrict__ out) {
    const double s = 0.5 * p.hv;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < p.ncell; e += (size_t)gridDim.x * blockDim.x)
        out[e] -= s * q[e % p.nx];
}

// gradient of the field energy W = 1/2 charge sum_i (phi_{i+1} - phi_i)^2 / hx
// with respect to phi: charge/hx (d_{i-1} - d_i), d_i = phi_{i+1} - phi_i (one CTA)
__global__ void k_adj_fe_gphi(int nx, double charge, double hx, const double* __restrict__ phi,
                              double* __restrict__ g) {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;
        const double d = phi[ip] - phi[i], dm = phi[i] - phi[im];
        g[i] = charge / hx * (dm - d);
    }
}

// out_ij = hv q_i, every row (L^T of a profile)
__global__ void k_adj_fill(AdjParams p, const double* __restrict__ q, double* __restrict__ out) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < p.ncell; e += (size_t)gridDim.x * blockDim.x)
        out[e] = p.hv * q[e % p.nx];
}

// gf = -gF + (2/ht) lambda
__global__ void k_adj_pull(AdjParams p, const double* __restrict__ gF, const double* __restrict__ lam,
                           double* __restrict__ gf) {
    const double s = 2.0 * p.ht_inv;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < p.ncell; e += (size_t)gridDim.x * blockDim.x)
        gf[e] = s * lam[e] - gF[e];
}

// hprof = (h1F + h1f + h2p + h2h) / 2 (h2 optional)
__global__ void k_adj_hprof(int nx, const double* __restrict__ a, const double* __restrict__ b,
                            const double* __restrict__ c, const double* __restrict__ d, double* __restrict__ out) {
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        double v = 0.5 * a[i] + 0.5 * b[i];
        if (c) v += 0.5 * c[i];
        if (d) v += 0.5 * d[i];
        out[i] = v;
    }
}

// Conjugate-transposed tridiagonal solve of mode k, A_k^H z = b, from the LU
// factors of A_k (diagonal reciprocals dinv, L sub-diagonal
// l_r = lambda alpha_r dinv_{r-1}, U super-diagonal c_r = lambda gamma_r):
//   U^H w = b : w_r = conj(dinv_r) (b_r - conj(c_{r-1}) w_{r-1})
//   L^H z = w : z_r = w_r - conj(l_{r+1}) z_{r+1}
// Each thread composes the affine maps of a chunk of rows; block scans join
// the chunks (the structure of tridiag_mode).  dynamic smem: nv + nv/CH complex.
__global__ void __launch_bounds__(TRI_THREADS) k_tridiag_modes_adjT(double2* __restrict__ spec, TriParams p) {
    using C = double2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ Aff<C> shw[TRI_THREADS / 32];
    const int k = blockIdx.x;
    const int nv = p.nv;
    const int CH = (nv + TRI_THREADS - 1) / TRI_THREADS;
    C* b = reinterpret_cast<C*>(smem_raw);
    C* line = spec + (size_t)k * nv;
    const C* di = reinterpret_cast<const C*>(p.dinv) + (size_t)k * nv;
    const double* al = reinterpret_cast<const double*>(p.alpha);
    const double* ga = reinterpret_cast<const double*>(p.gamma);
    const C lam = reinterpret_cast<const C*>(p.lambda)[k];
    for (int r = threadIdx.x; r < nv; r += TRI_THREADS) b[r + r / CH] = line[r];
    __syncthreads();
    const int r0 = threadIdx.x * CH;
    const int r1 = min(r0 + CH, nv);
    const int q0 = threadIdx.x * (CH + 1);
    // forward: U^H w = b
    Aff<C> a;
    a.P = make_double2(1.0, 0.0);
    a.Q = make_double2(0.0, 0.0);
    for (int r = r0, q = q0; r < r1; ++r, ++q) {
        const C dc = c_conj(di[r]);
        Aff<C> m;
        if (r == 0) m.P = make_double2(0.0, 0.0);
        else {
            const C cm = c_conj(c_rmul(lam, ga[r - 1]));
            const C t = c_mul(dc, cm);
            m.P = make_double2(-t.x, -t.y);
        }
        m.Q = c_mul(dc, b[q]);
        a = aff_combine(a, m);
    }
    C w = block_scan_aff<C>(a, true, shw);
    for (int r = r0, q = q0; r < r1; ++r, ++q) {
        const C dc = c_conj(di[r]);
        if (r == 0) w = c_mul(dc, b[q]);
        else w = c_mul(dc, c_sub(b[q], c_mul(c_conj(c_rmul(lam, ga[r - 1])), w)));
        b[q] = w;
    }
    __syncthreads();
    // backward: L^H z = w
    a.P = make_double2(1.0, 0.0);
    a.Q = make_double2(0.0, 0.0);
    for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
        Aff<C> m;
        m.Q = b[q];
        if (r == nv - 1) m.P = make_double2(0.0, 0.0);
        else {
            const C l = c_conj(c_mul(c_rmul(lam, al[r + 1]), di[r]));
            m.P = make_double2(-l.x, -l.y);
        }
        a = aff_combine(a, m);
    }
    C z = block_scan_aff<C>(a, false, shw);
    for (int r = r1 - 1, q = q0 + (r1 - 1 - r0); r >= r0; --r, --q) {
        if (r == nv - 1) z = b[q];
        else z = c_sub(b[q], c_mul(c_conj(c_mul(c_rmul(lam, al[r + 1]), di[r])), z));
        line[r] = z;
    }
}

}  // namespace vv
