// Explicit predictors of the step's initial guess (solvers/explicit/ as
// driven by run_base.py:786-912): the symplectic compositions of kinetic and
// potential bracket substeps (PETScArakawaSymplectic.pyx:62-92) and the two
// RK4 integrators (PETScArakawaRungeKutta.pyx:20-100).  The brackets run in
// the reference-order kernels with a general h field (vv_bracket.cuh); the
// kernels here build the h fields, form the stage inputs and the updates
// with every product and sum rounded separately in the order numpy
// evaluates the reference's expressions, and decide the residual guard.
#pragma once
#include "vv_common.cuh"
#include "vv_vec.cuh"

namespace vv {

// h field of a substep, F layout: mode 0 H0 (kinetic), 1 H1h + H2h
// (potential), 2 H0 + H1h + H2h (RK); h2 may be null (zero)
__global__ void k_pred_hfield(const double* __restrict__ h0, const double* __restrict__ h1,
                              const double* __restrict__ h2, double* __restrict__ H, int nx, int nv, int mode) {
    const size_t n = (size_t)nx * nv;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(g / nx), i = (int)(g - (size_t)j * nx);
        const double b2 = h2 ? h2[i] : 0.0;
        double v;
        if (mode == 0) v = h0[j];
        else if (mode == 1) v = __dadd_rn(h1[i], b2);
        else v = __dadd_rn(__dadd_rn(h0[j], h1[i]), b2);
        H[g] = v;
    }
}

// x[:,:] += s * y  (s = factor * ht / niter, formed on the host)
__global__ void k_pred_axpy(double* __restrict__ x, const double* __restrict__ y, double s, size_t n) {
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x)
        x[g] = __dadd_rn(x[g], __dmul_rn(s, y[g]));
}

// RK stage inputs: mode 0  x + a k1,  1  (x - a k1) + b k2,  2  ((x + b k1) - b k2) + b k3
__global__ void k_pred_stage(const double* __restrict__ x, const double* __restrict__ k1,
                             const double* __restrict__ k2, const double* __restrict__ k3, double* __restrict__ out,
                             double a, double b, int mode, size_t n) {
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        double v;
        if (mode == 0) v = __dadd_rn(x[g], __dmul_rn(a, k1[g]));
        else if (mode == 1) v = __dadd_rn(__dsub_rn(x[g], __dmul_rn(a, k1[g])), __dmul_rn(b, k2[g]));
        else
            v = __dadd_rn(__dsub_rn(__dadd_rn(x[g], __dmul_rn(b, k1[g])), __dmul_rn(b, k2[g])), __dmul_rn(b, k3[g]));
        out[g] = v;
    }
}

// RK update: x = x + b * (((k1 + w k2) + w k3) + k4) / d
__global__ void k_pred_rk_final(double* __restrict__ x, const double* __restrict__ k1, const double* __restrict__ k2,
                                const double* __restrict__ k3, const double* __restrict__ k4, double b, double w,
                                double d, size_t n) {
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        const double s = __dadd_rn(__dadd_rn(__dadd_rn(k1[g], __dmul_rn(w, k2[g])), __dmul_rn(w, k3[g])), k4[g]);
        x[g] = __dadd_rn(x[g], __ddiv_rn(__dmul_rn(b, s), d));
    }
}

// Residual norms of the guard (calculate_residual, run_base.py:631-637):
// ||R(f)|| from the residual kernel's partials plus ||Poisson residual||.
// Before the first update_previous the solver's Have is the zero vector of
// its construction: R then comes from the partials of the zero-Have residual
// (zpart).  phase 0: before the predictor; phase 1: the prediction's
// residual and the keep decision.
__global__ void k_pred_norm(DevState* s, const double* __restrict__ part, int np, const double* __restrict__ zpart,
                            int nzp, int phase) {
    if (threadIdx.x >= 32) return;
    const double f2 = s->have_set ? warp_reduce_parts(part, np) : warp_reduce_parts(zpart, nzp);
    if (threadIdx.x != 0) return;
    const double r = sqrt(f2) + sqrt(s->pnorm2);
    if (phase == 0) {
        s->guess_prev = r;
    } else {
        s->guess_res = r;
        s->guess_kept = r > s->guess_prev ? 0 : 1;
    }
}

// the guard: restore the previous iterate unless the prediction was kept
__global__ void k_pred_guard(const DevState* __restrict__ s, double* __restrict__ f, const double* __restrict__ fl,
                             size_t n) {
    if (s->guess_kept) return;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x)
        f[g] = fl[g];
}

__global__ void k_set_have(DevState* s) { s->have_set = 1; }

}  // namespace vv
