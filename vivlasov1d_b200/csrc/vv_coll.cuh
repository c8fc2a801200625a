// Collision operators of dissipation_type = 'collisions'
// (CollisionOperator.pyx:72-110 collT, :164-202 collE), added to the
// residual / Jacobian after the bracket as PETScNLVlasovMP.pyx:33-58 does:
//
//   Y += C_p[X]               (Jacobian: the current moments, factor 1/2)
//   Y += C_p[F] + C_h[Fh]     (residual: current and history moments)
//
// with, on the rows 2 <= j < nv-2 and u = U / n,
//   collT: drag_fac ((v+ - u) f+ - (v- - u) f-) a + diff_fac (f+ - 2 f + f-)
//   collE: drag_fac ((v+ - u) f+ - (v- - u) f-)   + diff_fac (f+ - 2 f + f-) / a
//   drag_fac = -factor nu drag / (2 hv),  diff_fac = -factor nu diff / hv^2.
// FP64 rounds every operation separately in the loop body's order (the
// reference's bits when the bracket part is too); FP32 for the mixed
// Jacobian.  The moments are frozen x profiles (n, U, a).  The grid is the
// bracket's narrow 32 x 16 tiling, so the per-tile sums of squares of the
// final Y (sumsq) line up with the residual norm's partials.
#pragma once
#include "vv_bracket.cuh"

namespace vv {

enum CollKind { COLL_NONE = 0, COLL_T = 1, COLL_E = 2 };

struct CollMoments {
    const double *n, *U, *a;   // density, velocity density, collision factor (nx each)
};

struct CollParams {
    int nx, nv, kind;
    double drag_fac, diff_fac;   // with the factor 1/2 of the midpoint rule
    const double* v;             // nv
    const int* xidx;             // optional: X is a GMRES basis base pointer + (*xidx) * xstride
    size_t xstride;
};

template <typename T>
VV_DEV T coll_term(int kind, T fp, T f0, T fm, T vp, T vm, T u, T a, T drag_fac, T diff_fac) {
    // ((v+ - u) f+ - (v- - u) f-) [a];  (f+ - 2 f) + f-  [/ a]
    T drag = rn_sub<T>(rn_mul<T>(rn_sub<T>(vp, u), fp), rn_mul<T>(rn_sub<T>(vm, u), fm));
    T diff = rn_add<T>(rn_sub<T>(fp, rn_mul<T>(T(2), f0)), fm);
    if (kind == COLL_T) drag = rn_mul<T>(drag, a);
    else diff = diff / a;
    return rn_add<T>(rn_mul<T>(drag_fac, drag), rn_mul<T>(diff_fac, diff));
}

// Y += C[X] (+ C_h[Xh] when Xh); optional per-tile sum of squares of Y
template <typename T>
__global__ void __launch_bounds__(BX * TY)
k_collision(const T* __restrict__ X, const T* __restrict__ Xh, T* __restrict__ Y, CollParams p, CollMoments mp,
            CollMoments mh, double* __restrict__ sumsq) {
    if (p.xidx) X += (size_t)(*p.xidx) * p.xstride;
    __shared__ double sred[BX * TY / 32];
    const int i = blockIdx.x * BX + threadIdx.x;
    const int nx = p.nx, nv = p.nv;
    double acc2 = 0.0;
    if (i < nx) {
        const T up = T(mp.U[i] / mp.n[i]), ap = T(mp.a[i]);
        T uh = T(0), ah = T(1);
        if (Xh) {
            uh = T(mh.U[i] / mh.n[i]);
            ah = T(mh.a[i]);
        }
        const T dr = T(p.drag_fac), df = T(p.diff_fac);
#pragma unroll
        for (int r = 0; r < BY / TY; ++r) {
            const int j = blockIdx.y * BY + threadIdx.y + r * TY;
            if (j >= nv) continue;
            const size_t g = (size_t)j * nx + i;
            T y = Y[g];
            if (j >= 2 && j < nv - 2) {
                const T vp = T(p.v[j + 1]), vm = T(p.v[j - 1]);
                y = rn_add<T>(y, coll_term<T>(p.kind, X[g + nx], X[g], X[g - nx], vp, vm, up, ap, dr, df));
                if (Xh) y = rn_add<T>(y, coll_term<T>(p.kind, Xh[g + nx], Xh[g], Xh[g - nx], vp, vm, uh, ah, dr, df));
                Y[g] = y;
            }
            acc2 += (double)y * (double)y;
        }
    }
    if (sumsq) {
        const double t = block_sum(acc2, sred);
        if (threadIdx.x == 0 && threadIdx.y == 0) sumsq[blockIdx.x + gridDim.x * blockIdx.y] = t;
    }
}

}  // namespace vv
