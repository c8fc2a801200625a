// Arakawa J1/J2/J4 bracket kernels: residual, Jacobian-vector product and
// bare bracket, with the time-derivative term fused in.
//
// Layout: fields are F[j*nx + i] (x fastest, periodic; v bounded).  A CTA
// owns a BX x BY tile of outputs and stages the input with a 2-cell halo in
// shared memory (x wraps periodically; rows outside [0, nv) are never read by
// interior outputs).  The Hamiltonian is regenerated in the CTA from the 1-D
// profiles h0(v) and the four x profiles of h1/h2 -- it never touches HBM.
//
// Two arithmetic orders:
//   * REFERENCE -- the exact expression trees of PoissonBracket.pyx:100-113
//     (J1), :221-234 (J2), :360-389 (J4) and PETScNLVlasovMP.pyx:33-58, with
//     every operation rounded separately (__dadd_rn/__dmul_rn, no FMA), and
//     h built in the axpy order of PETScVlasovSolver.pyx:145-149.  Results are
//     bit-identical to the reference loop.
//   * FACTORED -- h(x,v) = a(v) + b(x) is separable, so every stencil
//     coefficient of the bracket (the coefficient form of
//     PoissonBracket.pyx:168-181 and :290-301) is a sum of a v-difference of a
//     and an x-difference of b.  The J4 stencil then collapses to 8 input
//     differences and 6 products per output (~21 FP64 ops instead of ~60).
#pragma once
#include "vv_common.cuh"

namespace vv {

enum BracketMode { MODE_JVP = 0, MODE_RESIDUAL = 1, MODE_ADD = 2 };

struct BracketParams {
    int nx, nv;
    double ht_inv;   // 1/ht
    double tfac;     // ht_inv / divisor of the averaging stencil (unused for 'point')
    double factor;   // bracket factor (0.5 for the JVP, 1.0 residual)
    double f1;       // hx_inv*hv_inv/12
    double f2;       // hx_inv*hv_inv/24
    double hx_inv, hv_inv;
    const double* h0;   // nv: 0.5 v^2 mass
    const double* hxp;  // 4*nx: h1p, h1h, h2p, h2h profiles
    const int* xidx;    // optional: input is X + (*xidx) * xstride (GMRES basis vector)
    size_t xstride;
    const double* hfield;   // optional (MODE_ADD, reference-order kernels): a general h[j*nx + i]
                            // instead of the profiles (the double bracket's inner bracket)
};

template <typename T> VV_DEV T rn_add(T a, T b);
template <typename T> VV_DEV T rn_sub(T a, T b);
template <typename T> VV_DEV T rn_mul(T a, T b);
template <> VV_DEV double rn_add<double>(double a, double b) { return __dadd_rn(a, b); }
template <> VV_DEV double rn_sub<double>(double a, double b) { return __dsub_rn(a, b); }
template <> VV_DEV double rn_mul<double>(double a, double b) { return __dmul_rn(a, b); }
template <> VV_DEV float rn_add<float>(float a, float b) { return __fadd_rn(a, b); }
template <> VV_DEV float rn_sub<float>(float a, float b) { return __fsub_rn(a, b); }
template <> VV_DEV float rn_mul<float>(float a, float b) { return __fmul_rn(a, b); }

// Averaged time derivative (TimeDerivative.pyx:84-275).  On the rows
// 2 <= j < nv-2 the averaging operators replace ht_inv * x by
// (stencil sum of x) * ht_inv / divisor:
//   AVG 1  midpoint (also the arakawa_J1 class)  1 2 1 / 2 4 2 / 1 2 1, /16
//   AVG 5  Simpson                               1 4 1 / 4 16 4 / 1 4 1, /36
//   AVG 4  Arakawa J4: 13 points, (0,+-2) 1, diagonals 2, (+-1,0) and
//          (0,+-1) 8, (+-2,0) 1, centre 20, /64
// The terms are added in the order of the reference's loop body (v offset
// outer, x offset inner).  EXACT rounds every operation separately (the
// FP64 result is the reference's bits); otherwise the compiler may contract,
// which changes nothing for AVG 1 and 5 (their weights are powers of two).
// xs(di, dj) returns the input at x offset di, v offset dj.
enum AvgKind { AVG_POINT = 0, AVG_MIDPOINT = 1, AVG_J4 = 4, AVG_SIMPSON = 5 };

template <int AVG, bool EXACT, typename T, typename Get>
VV_DEV T avg_stencil(const Get& xs) {
    auto add = [](T a, T b) -> T {
        if constexpr (EXACT) return rn_add<T>(a, b);
        else return a + b;
    };
    auto mul = [](T w, T b) -> T {
        if constexpr (EXACT) return rn_mul<T>(w, b);
        else return w * b;
    };
    if constexpr (AVG == AVG_J4) {
        T s = xs(0, -2);
        s = add(s, mul(T(2), xs(-1, -1)));
        s = add(s, mul(T(8), xs(0, -1)));
        s = add(s, mul(T(2), xs(1, -1)));
        s = add(s, xs(-2, 0));
        s = add(s, mul(T(8), xs(-1, 0)));
        s = add(s, mul(T(20), xs(0, 0)));
        s = add(s, mul(T(8), xs(1, 0)));
        s = add(s, xs(2, 0));
        s = add(s, mul(T(2), xs(-1, 1)));
        s = add(s, mul(T(8), xs(0, 1)));
        s = add(s, mul(T(2), xs(1, 1)));
        s = add(s, xs(0, 2));
        return s;
    } else {
        constexpr double e = AVG == AVG_MIDPOINT ? 2.0 : 4.0, c = AVG == AVG_MIDPOINT ? 4.0 : 16.0;
        T s = xs(-1, -1);
        s = add(s, mul(T(e), xs(0, -1)));
        s = add(s, xs(1, -1));
        s = add(s, mul(T(e), xs(-1, 0)));
        s = add(s, mul(T(c), xs(0, 0)));
        s = add(s, mul(T(e), xs(1, 0)));
        s = add(s, xs(-1, 1));
        s = add(s, mul(T(e), xs(0, 1)));
        s = add(s, xs(1, 1));
        return s;
    }
}

// divisor of each averaging stencil
constexpr double avg_divisor(int avg) { return avg == AVG_J4 ? 64.0 : avg == AVG_SIMPSON ? 36.0 : 16.0; }

constexpr int BX = 32;
constexpr int BY = 16;
constexpr int TY = 8;             // threads in y; each thread handles BY/TY rows
constexpr int SX = BX + 4;
constexpr int SY = BY + 4;

__device__ __forceinline__ int wrapx(int i, int nx) {
    i %= nx;
    return i < 0 ? i + nx : i;
}

// h at (i, j) in the reference's axpy order: (((h0 + .5 h1p) + .5 h1h) + .5 h2p) + .5 h2h
__device__ __forceinline__ double h_ref(const BracketParams& p, int i, int j) {
    const int nx = p.nx;
    double h = p.h0[j];
    h = __dadd_rn(h, 0.5 * p.hxp[i]);
    h = __dadd_rn(h, 0.5 * p.hxp[nx + i]);
    h = __dadd_rn(h, 0.5 * p.hxp[2 * nx + i]);
    h = __dadd_rn(h, 0.5 * p.hxp[3 * nx + i]);
    return h;
}

// x part of h: ((.5 h1p + .5 h1h) + .5 h2p) + .5 h2h
__device__ __forceinline__ double b_fac(const BracketParams& p, int i) {
    const int nx = p.nx;
    double b = 0.5 * p.hxp[i] + 0.5 * p.hxp[nx + i];
    b += 0.5 * p.hxp[2 * nx + i];
    b += 0.5 * p.hxp[3 * nx + i];
    return b;
}

// Stage input and (reference order only) h into shared memory.
template <int MODE, bool STAGE_H>
__device__ __forceinline__ void stage_tile(const double* __restrict__ X, const double* __restrict__ Xh,
                                           const BracketParams& p, int i0, int j0,
                                           double (*sx)[SX + 1], double (*sh)[SX + 1]) {
    const int tid = threadIdx.x + BX * threadIdx.y;
    for (int s = tid; s < SX * SY; s += BX * TY) {
        const int ly = s / SX, lx = s - ly * SX;
        const int gi = wrapx(i0 - 2 + lx, p.nx);
        const int gj = j0 - 2 + ly;
        double xv = 0.0, hv = 0.0;
        if (gj >= 0 && gj < p.nv) {
            const size_t g = (size_t)gj * p.nx + gi;
            if (MODE == MODE_RESIDUAL) {
                // Fave = 0 + .5 Fh + .5 F   (PETScNLVlasovMP.pyx:49-51)
                xv = __dadd_rn(0.5 * Xh[g], 0.5 * X[g]);
            } else {
                xv = X[g];
            }
            if (STAGE_H) hv = p.hfield ? p.hfield[g] : h_ref(p, gi, gj);
        }
        sx[ly][lx] = xv;
        if (STAGE_H) sh[ly][lx] = hv;
    }
}

// Stage D = X - Xh (the residual's Fder, PETScNLVlasovMP.pyx:53-55) with the
// same 2-cell halo, for the averaged time derivative of the residual.
template <typename T, int LD>
__device__ __forceinline__ void stage_diff(const T* __restrict__ X, const T* __restrict__ Xh,
                                           const BracketParams& p, int i0, int j0, T (*sd)[LD],
                                           int sx_w, int sy_h, int nthreads, int tid) {
    for (int s = tid; s < sx_w * sy_h; s += nthreads) {
        const int ly = s / sx_w, lx = s - ly * sx_w;
        const int gi = wrapx(i0 - 2 + lx, p.nx);
        const int gj = j0 - 2 + ly;
        T d = T(0);
        if (gj >= 0 && gj < p.nv) {
            const size_t g = (size_t)gj * p.nx + gi;
            d = rn_sub<T>(X[g], Xh[g]);
        }
        sd[ly][lx] = d;
    }
}

#define R_ADD(a, b) __dadd_rn((a), (b))
#define R_SUB(a, b) __dsub_rn((a), (b))
#define R_MUL(a, b) __dmul_rn((a), (b))

// ---------------------------------------------------------------------------
// Reference operation order
// ---------------------------------------------------------------------------
template <int SCHEME, int MODE, int AVG = AVG_POINT>
__global__ void __launch_bounds__(BX * TY)
k_bracket_ref(const double* __restrict__ X, const double* __restrict__ Xh,
              double* __restrict__ Y, BracketParams p, double* __restrict__ sumsq) {
    constexpr bool DIFF = AVG != AVG_POINT && MODE == MODE_RESIDUAL;
    if (p.xidx) X += (size_t)(*p.xidx) * p.xstride;
    __shared__ double sx[SY][SX + 1];
    __shared__ double sh[SY][SX + 1];
    __shared__ double sd[DIFF ? SY : 1][SX + 1];
    __shared__ double sred[BX * TY / 32];
    const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY;
    stage_tile<MODE, true>(X, Xh, p, i0, j0, sx, sh);
    if constexpr (DIFF) stage_diff<double, SX + 1>(X, Xh, p, i0, j0, sd, SX, SY, BX * TY, threadIdx.x + BX * threadIdx.y);
    __syncthreads();

    double acc2 = 0.0;
    const int lx = threadIdx.x + 2;
    const int i = i0 + threadIdx.x;
#pragma unroll
    for (int r = 0; r < BY / TY; ++r) {
        const int ly = threadIdx.y + r * TY + 2;
        const int j = j0 + ly - 2;
        if (i >= p.nx || j >= p.nv) continue;
        const size_t g = (size_t)j * p.nx + i;
#define XS(di, dj) sx[ly + (dj)][lx + (di)]
#define HS(di, dj) sh[ly + (dj)][lx + (di)]
        double y;
        const bool inner = j >= 2 && j < p.nv - 2;
        if (AVG != AVG_POINT && MODE == MODE_JVP && inner) {
            y = __dmul_rn(avg_stencil<AVG, true, double>([&](int di, int dj) { return XS(di, dj); }), p.tfac);
        } else if (DIFF && inner) {
            y = __dmul_rn(avg_stencil<AVG, true, double>([&](int di, int dj) { return sd[ly + dj][lx + di]; }),
                          p.tfac);
        } else if (MODE == MODE_JVP) {
            y = R_MUL(p.ht_inv, X[g]);                 // Y.axpy(ht_inv, F)
        } else if (MODE == MODE_RESIDUAL) {
            y = R_MUL(p.ht_inv, R_SUB(X[g], Xh[g]));   // Y.axpy(ht_inv, F - Fh)
        } else {
            y = Y[g];
        }
        if (inner) {
            double s1 = 0.0, s2 = 0.0;
            if (SCHEME == 1 || SCHEME == 4) {
                const double jpp = R_SUB(R_MUL(R_SUB(XS(1, 0), XS(-1, 0)), R_SUB(HS(0, 1), HS(0, -1))),
                                         R_MUL(R_SUB(XS(0, 1), XS(0, -1)), R_SUB(HS(1, 0), HS(-1, 0))));
                const double jpc = R_ADD(R_SUB(R_SUB(R_MUL(XS(1, 0), R_SUB(HS(1, 1), HS(1, -1))),
                                                     R_MUL(XS(-1, 0), R_SUB(HS(-1, 1), HS(-1, -1)))),
                                               R_MUL(XS(0, 1), R_SUB(HS(1, 1), HS(-1, 1)))),
                                         R_MUL(XS(0, -1), R_SUB(HS(1, -1), HS(-1, -1))));
                const double jcp = R_ADD(R_SUB(R_SUB(R_MUL(XS(1, 1), R_SUB(HS(0, 1), HS(1, 0))),
                                                     R_MUL(XS(-1, -1), R_SUB(HS(-1, 0), HS(0, -1)))),
                                               R_MUL(XS(-1, 1), R_SUB(HS(0, 1), HS(-1, 0)))),
                                         R_MUL(XS(1, -1), R_SUB(HS(1, 0), HS(0, -1))));
                s1 = R_ADD(R_ADD(jpp, jpc), jcp);
            }
            if (SCHEME == 2 || SCHEME == 4) {
                const double jcc = R_SUB(R_MUL(R_SUB(XS(1, 1), XS(-1, -1)), R_SUB(HS(-1, 1), HS(1, -1))),
                                         R_MUL(R_SUB(XS(-1, 1), XS(1, -1)), R_SUB(HS(1, 1), HS(-1, -1))));
                const double jpc = R_ADD(R_SUB(R_SUB(R_MUL(XS(2, 0), R_SUB(HS(1, 1), HS(1, -1))),
                                                     R_MUL(XS(-2, 0), R_SUB(HS(-1, 1), HS(-1, -1)))),
                                               R_MUL(XS(0, 2), R_SUB(HS(1, 1), HS(-1, 1)))),
                                         R_MUL(XS(0, -2), R_SUB(HS(1, -1), HS(-1, -1))));
                const double jcp = R_ADD(R_SUB(R_SUB(R_MUL(XS(1, 1), R_SUB(HS(0, 2), HS(2, 0))),
                                                     R_MUL(XS(-1, -1), R_SUB(HS(-2, 0), HS(0, -2)))),
                                               R_MUL(XS(-1, 1), R_SUB(HS(0, 2), HS(-2, 0)))),
                                         R_MUL(XS(1, -1), R_SUB(HS(2, 0), HS(0, -2))));
                s2 = R_ADD(R_ADD(jcc, jpc), jcp);
            }
            double add;
            if (SCHEME == 1) {
                add = R_MUL(R_MUL(p.factor, s1), p.f1);      // factor*(..)*arakawa_factor
            } else if (SCHEME == 2) {
                add = R_MUL(R_MUL(p.factor, s2), p.f2);
            } else {
                const double r1 = R_MUL(s1, p.f1), r2 = R_MUL(s2, p.f2);
                add = R_MUL(p.factor, R_SUB(R_MUL(2.0, r1), r2));
            }
            y = R_ADD(y, add);
        }
#undef XS
#undef HS
        Y[g] = y;
        acc2 += y * y;
    }
    if (sumsq) {
        const double t = block_sum(acc2, sred);
        if (threadIdx.x == 0 && threadIdx.y == 0) sumsq[blockIdx.x + gridDim.x * blockIdx.y] = t;
    }
}

// ---------------------------------------------------------------------------
// Simpson bracket (PoissonBracket.pyx:405-492): four J1-pattern brackets at
// x/v spacings (1,1), (1,2), (2,1), (2,2), combined as
// (25 b11 - 10 b12 - 10 b21 + 4 b22) factor hx^-1 hv^-1 / 9, in the
// reference's operation order (round-to-nearest adds and multiplies: the
// FP64 result is the reference's bits); T = float for the mixed-precision
// Jacobian.
// ---------------------------------------------------------------------------

template <int MODE, typename T, int AVG = AVG_POINT>
__global__ void __launch_bounds__(BX * TY)
k_bracket_simpson(const T* __restrict__ X, const T* __restrict__ Xh, T* __restrict__ Y, BracketParams p,
                  double* __restrict__ sumsq) {
    constexpr bool DIFF = AVG != AVG_POINT && MODE == MODE_RESIDUAL;
    if (p.xidx) X += (size_t)(*p.xidx) * p.xstride;
    __shared__ T sx[SY][SX + 1];
    __shared__ T sh[SY][SX + 1];
    __shared__ T sd[DIFF ? SY : 1][SX + 1];
    __shared__ double sred[BX * TY / 32];
    const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY;
    const int tid = threadIdx.x + BX * threadIdx.y;
    for (int s = tid; s < SX * SY; s += BX * TY) {
        const int ly = s / SX, lx = s - ly * SX;
        const int gi = wrapx(i0 - 2 + lx, p.nx);
        const int gj = j0 - 2 + ly;
        T xv = T(0), hv = T(0);
        if (gj >= 0 && gj < p.nv) {
            const size_t g = (size_t)gj * p.nx + gi;
            // Fave = 0 + .5 Fh + .5 F  (PETScNLVlasovMP.pyx:49-51)
            xv = (MODE == MODE_RESIDUAL) ? rn_add<T>(rn_mul<T>(T(0.5), Xh[g]), rn_mul<T>(T(0.5), X[g])) : X[g];
            hv = T(p.hfield ? p.hfield[g] : h_ref(p, gi, gj));
        }
        sx[ly][lx] = xv;
        sh[ly][lx] = hv;
    }
    if constexpr (DIFF) stage_diff<T, SX + 1>(X, Xh, p, i0, j0, sd, SX, SY, BX * TY, tid);
    __syncthreads();
    const T sfac = T(((p.factor * p.hx_inv) * p.hv_inv) / 9.);   // simpson_factor
    const T htinv = T(p.ht_inv);
    double acc2 = 0.0;
    const int lx = threadIdx.x + 2;
    const int i = i0 + threadIdx.x;
#define A_(x, y) rn_add<T>((x), (y))
#define S_(x, y) rn_sub<T>((x), (y))
#define M_(x, y) rn_mul<T>((x), (y))
#pragma unroll
    for (int r = 0; r < BY / TY; ++r) {
        const int ly = threadIdx.y + r * TY + 2;
        const int j = j0 + ly - 2;
        if (i >= p.nx || j >= p.nv) continue;
        const size_t g = (size_t)j * p.nx + i;
#define XS(di, dj) sx[ly + (dj)][lx + (di)]
#define HS(di, dj) sh[ly + (dj)][lx + (di)]
        T y;
        const bool inner = j >= 2 && j < p.nv - 2;
        if (AVG != AVG_POINT && MODE == MODE_JVP && inner)
            y = rn_mul<T>(avg_stencil<AVG, true, T>([&](int di, int dj) { return XS(di, dj); }), T(p.tfac));
        else if (DIFF && inner)
            y = rn_mul<T>(avg_stencil<AVG, true, T>([&](int di, int dj) { return sd[ly + dj][lx + di]; }),
                          T(p.tfac));
        else if (MODE == MODE_JVP) y = M_(htinv, X[g]);                  // Y.axpy(ht_inv, F)
        else if (MODE == MODE_RESIDUAL) y = M_(htinv, S_(X[g], Xh[g]));  // Y.axpy(ht_inv, F - Fh)
        else y = Y[g];                                                   // bracket only: Y += factor [X, H]
        if (inner) {
            T t = M_(S_(XS(0, 2), XS(0, -2)), S_(HS(-2, 0), HS(2, 0)));
            t = A_(t, M_(S_(XS(2, 0), XS(-2, 0)), S_(HS(0, 2), HS(0, -2))));
            t = A_(t, M_(XS(0, 2), S_(HS(-2, 2), HS(2, 2))));
            t = A_(t, M_(XS(0, -2), S_(HS(2, -2), HS(-2, -2))));
            t = A_(t, M_(XS(2, 0), S_(HS(2, 2), HS(2, -2))));
            t = A_(t, M_(XS(-2, 0), S_(HS(-2, -2), HS(-2, 2))));
            t = A_(t, M_(XS(2, 2), S_(HS(0, 2), HS(2, 0))));
            t = A_(t, M_(XS(2, -2), S_(HS(2, 0), HS(0, -2))));
            t = A_(t, M_(XS(-2, 2), S_(HS(-2, 0), HS(0, 2))));
            t = A_(t, M_(XS(-2, -2), S_(HS(0, -2), HS(-2, 0))));
            const T b22 = t / T(48.);
            t = M_(S_(XS(0, 2), XS(0, -2)), S_(HS(-1, 0), HS(1, 0)));
            t = A_(t, M_(S_(XS(1, 0), XS(-1, 0)), S_(HS(0, 2), HS(0, -2))));
            t = A_(t, M_(XS(0, 2), S_(HS(-1, 2), HS(1, 2))));
            t = A_(t, M_(XS(0, -2), S_(HS(1, -2), HS(-1, -2))));
            t = A_(t, M_(XS(1, 0), S_(HS(1, 2), HS(1, -2))));
            t = A_(t, M_(XS(-1, 0), S_(HS(-1, -2), HS(-1, 2))));
            t = A_(t, M_(XS(1, 2), S_(HS(0, 2), HS(1, 0))));
            t = A_(t, M_(XS(1, -2), S_(HS(1, 0), HS(0, -2))));
            t = A_(t, M_(XS(-1, -2), S_(HS(0, -2), HS(-1, 0))));
            t = A_(t, M_(XS(-1, 2), S_(HS(-1, 0), HS(0, 2))));
            const T b12 = t / T(24.);
            t = M_(S_(XS(0, 1), XS(0, -1)), S_(HS(-2, 0), HS(2, 0)));
            t = A_(t, M_(S_(XS(2, 0), XS(-2, 0)), S_(HS(0, 1), HS(0, -1))));
            t = A_(t, M_(XS(0, 1), S_(HS(-2, 1), HS(2, 1))));
            t = A_(t, M_(XS(0, -1), S_(HS(2, -1), HS(-2, -1))));
            t = A_(t, M_(XS(2, 0), S_(HS(2, 1), HS(2, -1))));
            t = A_(t, M_(XS(-2, 0), S_(HS(-2, -1), HS(-2, 1))));
            t = A_(t, M_(XS(2, 1), S_(HS(0, 1), HS(2, 0))));
            t = A_(t, M_(XS(2, -1), S_(HS(2, 0), HS(0, -1))));
            t = A_(t, M_(XS(-2, 1), S_(HS(-2, 0), HS(0, 1))));
            t = A_(t, M_(XS(-2, -1), S_(HS(0, -1), HS(-2, 0))));
            const T b21 = t / T(24.);
            t = M_(S_(XS(0, 1), XS(0, -1)), S_(HS(-1, 0), HS(1, 0)));
            t = A_(t, M_(S_(XS(1, 0), XS(-1, 0)), S_(HS(0, 1), HS(0, -1))));
            t = A_(t, M_(XS(0, 1), S_(HS(-1, 1), HS(1, 1))));
            t = A_(t, M_(XS(0, -1), S_(HS(1, -1), HS(-1, -1))));
            t = A_(t, M_(XS(-1, 0), S_(HS(-1, -1), HS(-1, 1))));
            t = A_(t, M_(XS(1, 0), S_(HS(1, 1), HS(1, -1))));
            t = A_(t, M_(XS(1, 1), S_(HS(0, 1), HS(1, 0))));
            t = A_(t, M_(XS(1, -1), S_(HS(1, 0), HS(0, -1))));
            t = A_(t, M_(XS(-1, -1), S_(HS(0, -1), HS(-1, 0))));
            t = A_(t, M_(XS(-1, 1), S_(HS(-1, 0), HS(0, 1))));
            const T b11 = t / T(12.);
            const T c = A_(S_(S_(M_(T(25.), b11), M_(T(10.), b12)), M_(T(10.), b21)), M_(T(4.), b22));
            y = A_(y, M_(c, sfac));
        }
#undef XS
#undef HS
        Y[g] = y;
        acc2 += (double)y * (double)y;
    }
#undef A_
#undef S_
#undef M_
    if (sumsq) {
        const double t = block_sum(acc2, sred);
        if (threadIdx.x == 0 && threadIdx.y == 0) sumsq[blockIdx.x + gridDim.x * blockIdx.y] = t;
    }
}

// ---------------------------------------------------------------------------
// Factored (separable-h) form
// ---------------------------------------------------------------------------
// Per scheme constants of  y/scale = A1*(cA1*d10 + cA2*d20) - B1*(cB1*d01 + cB2*d02)
//                                    + am*dm + ap*dp + bm*em + bp*ep
template <int SCHEME> struct Coef;
template <> struct Coef<1> {
    static constexpr double cA1 = 2.0, cA2 = 0.0, cB1 = 2.0, cB2 = 0.0;
    // alpha_m = -Da_m ; alpha_p = -Da_p ; beta_m = Db_m ; beta_p = Db_p
    VV_DEV static void row(double Dam, double Dap, double A1, double Cm, double Cp, double& am, double& ap) {
        am = -Dam; ap = -Dap;
    }
    VV_DEV static void col(double Dbm, double Dbp, double B1, double Bm, double Bp, double& bm, double& bp) {
        bm = Dbm; bp = Dbp;
    }
};
template <> struct Coef<2> {
    static constexpr double cA1 = 0.0, cA2 = 1.0, cB1 = 0.0, cB2 = 1.0;
    VV_DEV static void row(double Dam, double Dap, double A1, double Cm, double Cp, double& am, double& ap) {
        am = -Cm - A1; ap = -Cp - A1;
    }
    VV_DEV static void col(double Dbm, double Dbp, double B1, double Bm, double Bp, double& bm, double& bp) {
        bm = Bm + B1; bp = Bp + B1;
    }
};
template <> struct Coef<4> {  // 2*J1 - 0.5*J2 in units of f1 (f2 = f1/2)
    static constexpr double cA1 = 4.0, cA2 = -0.5, cB1 = 4.0, cB2 = -0.5;
    VV_DEV static void row(double Dam, double Dap, double A1, double Cm, double Cp, double& am, double& ap) {
        am = -2.0 * Dam + 0.5 * (Cm + A1);
        ap = -2.0 * Dap + 0.5 * (Cp + A1);
    }
    VV_DEV static void col(double Dbm, double Dbp, double B1, double Bm, double Bp, double& bm, double& bp) {
        bm = 2.0 * Dbm - 0.5 * (Bm + B1);
        bp = 2.0 * Dbp - 0.5 * (Bp + B1);
    }
};

template <int SCHEME, int MODE, typename T, int AVG = AVG_POINT>
__global__ void __launch_bounds__(BX * TY)
k_bracket_fac(const T* __restrict__ X, const T* __restrict__ Xh, T* __restrict__ Y,
              BracketParams p, double* __restrict__ sumsq) {
    constexpr bool DIFF = AVG != AVG_POINT && MODE == MODE_RESIDUAL;
    if (p.xidx) X += (size_t)(*p.xidx) * p.xstride;
    __shared__ T sx[SY][SX + 1];
    __shared__ T sd[DIFF ? SY : 1][SX + 1];
    __shared__ double sa[SY];       // a(v) = h0 on the tile rows (with halo)
    __shared__ double sb[SX];       // b(x) on the tile columns (with halo)
    __shared__ double srow[BY][3];  // A1, alpha_m, alpha_p (scaled)
    __shared__ double scol[BX][3];  // B1, beta_m, beta_p (scaled)
    __shared__ double sred[BX * TY / 32];
    const int i0 = blockIdx.x * BX, j0 = blockIdx.y * BY;
    const int tid = threadIdx.x + BX * threadIdx.y;
    for (int s = tid; s < SX * SY; s += BX * TY) {
        const int ly = s / SX, lx = s - ly * SX;
        const int gi = wrapx(i0 - 2 + lx, p.nx);
        const int gj = j0 - 2 + ly;
        T xv = T(0);
        if (gj >= 0 && gj < p.nv) {
            const size_t g = (size_t)gj * p.nx + gi;
            if (MODE == MODE_RESIDUAL) xv = T(0.5) * Xh[g] + T(0.5) * X[g];
            else xv = X[g];
        }
        sx[ly][lx] = xv;
    }
    if constexpr (DIFF) stage_diff<T, SX + 1>(X, Xh, p, i0, j0, sd, SX, SY, BX * TY, tid);
    if (tid < SY) {
        const int gj = j0 - 2 + tid;
        sa[tid] = (gj >= 0 && gj < p.nv) ? p.h0[gj] : 0.0;
    } else if (tid >= 32 && tid < 32 + SX) {
        const int l = tid - 32;
        sb[l] = b_fac(p, wrapx(i0 - 2 + l, p.nx));
    }
    __syncthreads();
    const double scale = (SCHEME == 2) ? p.f2 : p.f1;
    if (tid < BY) {
        const int l = tid + 2;
        const double Dam = sa[l] - sa[l - 1], Dap = sa[l + 1] - sa[l];
        const double A1 = sa[l + 1] - sa[l - 1];
        const double Cm = sa[l] - sa[l - 2], Cp = sa[l + 2] - sa[l];
        double am, ap;
        Coef<SCHEME>::row(Dam, Dap, A1, Cm, Cp, am, ap);
        srow[tid][0] = A1; srow[tid][1] = am; srow[tid][2] = ap;
    } else if (tid >= 32 && tid < 32 + BX) {
        const int l = tid - 32 + 2;
        const double Dbm = sb[l] - sb[l - 1], Dbp = sb[l + 1] - sb[l];
        const double B1 = sb[l + 1] - sb[l - 1];
        const double Bm = sb[l] - sb[l - 2], Bp = sb[l + 2] - sb[l];
        double bm, bp;
        Coef<SCHEME>::col(Dbm, Dbp, B1, Bm, Bp, bm, bp);
        scol[tid - 32][0] = B1; scol[tid - 32][1] = bm; scol[tid - 32][2] = bp;
    }
    __syncthreads();

    const int lx = threadIdx.x + 2;
    const int i = i0 + threadIdx.x;
    const T B1 = T(scol[threadIdx.x][0]), bm = T(scol[threadIdx.x][1]), bp = T(scol[threadIdx.x][2]);
    const T tscale = T(scale * p.factor);
    double acc2 = 0.0;
#pragma unroll
    for (int r = 0; r < BY / TY; ++r) {
        const int ty = threadIdx.y + r * TY;
        const int ly = ty + 2;
        const int j = j0 + ty;
        if (i >= p.nx || j >= p.nv) continue;
        const size_t g = (size_t)j * p.nx + i;
#define XS(di, dj) sx[ly + (dj)][lx + (di)]
        T y;
        const bool inner = j >= 2 && j < p.nv - 2;
        if (AVG != AVG_POINT && MODE == MODE_JVP && inner)
            y = avg_stencil<AVG, false, T>([&](int di, int dj) { return XS(di, dj); }) * T(p.tfac);
        else if (DIFF && inner)
            y = avg_stencil<AVG, false, T>([&](int di, int dj) { return sd[ly + dj][lx + di]; }) * T(p.tfac);
        else if (MODE == MODE_JVP) y = T(p.ht_inv) * X[g];
        else if (MODE == MODE_RESIDUAL) y = T(p.ht_inv) * (X[g] - Xh[g]);
        else y = Y[g];
        if (inner) {
            const T A1 = T(srow[ty][0]), am = T(srow[ty][1]), ap = T(srow[ty][2]);
            const T xm1m1 = XS(-1, -1), xp1m1 = XS(1, -1), xm1p1 = XS(-1, 1), xp1p1 = XS(1, 1);
            T s = T(0);
            if (Coef<SCHEME>::cA1 != 0.0 || Coef<SCHEME>::cA2 != 0.0) {
                T ax = T(0), bx = T(0);
                if (Coef<SCHEME>::cA1 != 0.0) {
                    ax = T(Coef<SCHEME>::cA1) * (XS(1, 0) - XS(-1, 0));
                    bx = T(Coef<SCHEME>::cB1) * (XS(0, 1) - XS(0, -1));
                }
                if (Coef<SCHEME>::cA2 != 0.0) {
                    ax += T(Coef<SCHEME>::cA2) * (XS(2, 0) - XS(-2, 0));
                    bx += T(Coef<SCHEME>::cB2) * (XS(0, 2) - XS(0, -2));
                }
                s = A1 * ax - B1 * bx;
            }
            s += am * (xm1m1 - xp1m1);
            s += ap * (xm1p1 - xp1p1);
            s += bm * (xm1m1 - xm1p1);
            s += bp * (xp1m1 - xp1p1);
            y += tscale * s;
        }
#undef XS
        Y[g] = y;
        acc2 += (double)y * (double)y;
    }
    if (sumsq) {
        const double t = block_sum(acc2, sred);
        if (tid == 0) sumsq[blockIdx.x + gridDim.x * blockIdx.y] = t;
    }
}

// ---------------------------------------------------------------------------
// Factored form, wide tiles: 64 (x) x 32 (v) outputs per CTA, 256 threads,
// each thread one column and 8 consecutive rows (register window along v,
// 6 shared-memory loads per output).  Staging uses 16-byte loads; the
// periodic wrap is one conditional add/subtract.  Requires nx % 64 == 0 and
// 16-byte aligned fields (checked by the launcher; otherwise k_bracket_fac).
// ---------------------------------------------------------------------------
constexpr int WX = 64;
constexpr int WY = 32;
constexpr int WR = 8;                 // rows per thread
constexpr int WSX = WX + 4;           // 68
constexpr int WSY = WY + 4;           // 36
constexpr int WTHREADS = WX * (WY / WR);  // 256

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// One 64 x 32 output tile (bx, by) of the bracket; the tile grid is tiles_x
// wide (the per-tile sum of squares goes to sumsq[bx + tiles_x by]).  Shared
// by the single-grid kernel below and the batched kernels.
template <int SCHEME, int MODE, typename T, int AVG = AVG_POINT>
__device__ __forceinline__ void bracket_wide_tile(const T* __restrict__ X, const T* __restrict__ Xh,
                                                  T* __restrict__ Y, const BracketParams& p,
                                                  double* __restrict__ sumsq, int bx, int by, int tiles_x) {
    static_assert(AVG == AVG_POINT || MODE == MODE_JVP, "the wide tiles average the Jacobian only");
    using V2 = typename Vec2<T>::type;
    __shared__ __align__(16) T sx[WSY][WSX];
    __shared__ double sa[WSY];
    __shared__ double sb[WSX];
    __shared__ double srow[WY][3];
    __shared__ double scol[WX][3];
    __shared__ double sred[WTHREADS / 32];
    const int tid = threadIdx.x;
    const int i0 = bx * WX, j0 = by * WY;
    const int nx = p.nx, nv = p.nv;
    // ---- stage the input tile (x pairs) ----
    constexpr int NP = WSX / 2;   // 34 pairs per row
    for (int q = tid; q < NP * WSY; q += WTHREADS) {
        const int ly = q / NP, px = q - ly * NP;
        int gi = i0 - 2 + 2 * px;
        if (gi < 0) gi += nx;
        else if (gi >= nx) gi -= nx;
        const int gj = j0 - 2 + ly;
        V2 v;
        v.x = T(0); v.y = T(0);
        if (gj >= 0 && gj < nv) {
            const size_t g = (size_t)gj * nx + gi;
            const V2 a = *reinterpret_cast<const V2*>(X + g);
            if (MODE == MODE_RESIDUAL) {
                const V2 b = *reinterpret_cast<const V2*>(Xh + g);
                v.x = T(0.5) * b.x + T(0.5) * a.x;
                v.y = T(0.5) * b.y + T(0.5) * a.y;
            } else {
                v = a;
            }
        }
        *reinterpret_cast<V2*>(&sx[ly][2 * px]) = v;
    }
    if (tid < WSY) {
        const int gj = j0 - 2 + tid;
        sa[tid] = (gj >= 0 && gj < nv) ? p.h0[gj] : 0.0;
    } else if (tid >= 64 && tid < 64 + WSX) {
        const int l = tid - 64;
        int gi = i0 - 2 + l;
        if (gi < 0) gi += nx;
        else if (gi >= nx) gi -= nx;
        sb[l] = b_fac(p, gi);
    }
    __syncthreads();
    if (tid < WY) {
        const int l = tid + 2;
        double am, ap;
        Coef<SCHEME>::row(sa[l] - sa[l - 1], sa[l + 1] - sa[l], sa[l + 1] - sa[l - 1], sa[l] - sa[l - 2],
                          sa[l + 2] - sa[l], am, ap);
        srow[tid][0] = sa[l + 1] - sa[l - 1];
        srow[tid][1] = am;
        srow[tid][2] = ap;
    } else if (tid >= 64 && tid < 64 + WX) {
        const int c = tid - 64, l = c + 2;
        double bm, bp;
        Coef<SCHEME>::col(sb[l] - sb[l - 1], sb[l + 1] - sb[l], sb[l + 1] - sb[l - 1], sb[l] - sb[l - 2],
                          sb[l + 2] - sb[l], bm, bp);
        scol[c][0] = sb[l + 1] - sb[l - 1];
        scol[c][1] = bm;
        scol[c][2] = bp;
    }
    __syncthreads();
    // ---- compute: column tx, rows ty*8 .. ty*8+7, rolling register window ----
    const int tx = tid & (WX - 1), ty = tid / WX;
    const int lx = tx + 2;
    const int r0 = ty * WR;            // tile row of the first output
    const int i = i0 + tx;
    const T B1 = T(scol[tx][0]), bm = T(scol[tx][1]), bp = T(scol[tx][2]);
    const T tscale = T(((SCHEME == 2) ? p.f2 : p.f1) * p.factor);
    const T htinv = T(p.ht_inv);
    // window: column i rows j-2..j+2, columns i+-1 rows j-1..j+1
    T w0 = sx[r0][lx], w1 = sx[r0 + 1][lx], w2 = sx[r0 + 2][lx], w3 = sx[r0 + 3][lx];
    T m0 = sx[r0 + 1][lx - 1], m1 = sx[r0 + 2][lx - 1];
    T q0 = sx[r0 + 1][lx + 1], q1 = sx[r0 + 2][lx + 1];
    double acc2 = 0.0;
#pragma unroll
    for (int q = 0; q < WR; ++q) {
        const T w4 = sx[r0 + q + 4][lx];
        const T m2 = sx[r0 + q + 3][lx - 1];
        const T q2 = sx[r0 + q + 3][lx + 1];
        const int j = j0 + r0 + q;
        if (j < nv) {
            const size_t g = (size_t)j * nx + i;
            T y;
            const bool inner = j >= 2 && j < nv - 2;
            if (AVG != AVG_POINT && inner) {
                // the window holds every stencil point but (+-2, 0)
                y = avg_stencil<AVG, false, T>([&](int di, int dj) -> T {
                        if (di == 0) return dj == -2 ? w0 : dj == -1 ? w1 : dj == 0 ? w2 : dj == 1 ? w3 : w4;
                        if (di == -1) return dj == -1 ? m0 : dj == 0 ? m1 : m2;
                        if (di == 1) return dj == -1 ? q0 : dj == 0 ? q1 : q2;
                        return sx[r0 + q + 2][lx + di];
                    }) * T(p.tfac);
            } else if (MODE == MODE_JVP) y = htinv * w2;
            else if (MODE == MODE_RESIDUAL) y = htinv * (X[g] - Xh[g]);
            else y = Y[g];
            if (inner) {
                const T A1 = T(srow[r0 + q][0]), am = T(srow[r0 + q][1]), ap = T(srow[r0 + q][2]);
                T s = T(0);
                if (Coef<SCHEME>::cA1 != 0.0 || Coef<SCHEME>::cA2 != 0.0) {
                    T ax = T(0), bx = T(0);
                    if (Coef<SCHEME>::cA1 != 0.0) {
                        ax = T(Coef<SCHEME>::cA1) * (q1 - m1);
                        bx = T(Coef<SCHEME>::cB1) * (w3 - w1);
                    }
                    if (Coef<SCHEME>::cA2 != 0.0) {
                        ax += T(Coef<SCHEME>::cA2) * (sx[r0 + q + 2][lx + 2] - sx[r0 + q + 2][lx - 2]);
                        bx += T(Coef<SCHEME>::cB2) * (w4 - w0);
                    }
                    s = A1 * ax - B1 * bx;
                }
                s += am * (m0 - q0);     // (x(-1,-1) - x(+1,-1))
                s += ap * (m2 - q2);     // (x(-1,+1) - x(+1,+1))
                s += bm * (m0 - m2);     // (x(-1,-1) - x(-1,+1))
                s += bp * (q0 - q2);     // (x(+1,-1) - x(+1,+1))
                y += tscale * s;
            }
            Y[g] = y;
            acc2 += (double)y * (double)y;
        }
        w0 = w1; w1 = w2; w2 = w3; w3 = w4;
        m0 = m1; m1 = m2;
        q0 = q1; q1 = q2;
    }
    if (sumsq) {
        const double t = block_sum(acc2, sred);
        if (tid == 0) sumsq[bx + tiles_x * by] = t;
    }
}

// ---------------------------------------------------------------------------
// Marching Jacobian-vector product: a CTA owns a strip of MW columns (one
// thread per column) and a segment of rows, and walks down v through a ring
// of NR rows in shared memory (a power of two) that cp.async fills three
// chunks of CH rows ahead of the compute.  One block barrier per chunk: the
// ring holds the chunk being computed with its 2-row halos and the three
// chunks after it (NR = 4 CH + 4), so the copies of chunk k+3 go out right
// after the barrier that publishes chunk k -- every thread has passed it, so
// chunk k-1's rows are free -- and the row coefficients are double-buffered.  Each thread keeps its column's five-row
// window and its column's x-coefficients in registers; the v-coefficients of
// a chunk's rows are formed once per CTA.  A row costs 5 shared loads per
// output; the x halo is 4 of MW + 4 columns and the v halo 4 rows per segment.
// ---------------------------------------------------------------------------
// rows per chunk and ring rows (a power of two = 4 chunks + 4 halo rows)
template <typename T> struct MarchShape;
template <> struct MarchShape<double> { static constexpr int CH = 7, NR = 32; };
template <> struct MarchShape<float> { static constexpr int CH = 15, NR = 64; };


// ring row layout: [pad][2 left halo][MW columns][2 right halo][pad]; the
// main columns start at LP elements (16 bytes), every row is 16-byte aligned
template <typename T, int MW>
struct MarchRow {
    static constexpr int LP = 16 / (int)sizeof(T);
    static constexpr int RS = MW + 2 * LP;
    static constexpr size_t smem_bytes() {
        return (size_t)MarchShape<T>::NR * RS * sizeof(T) + (size_t)2 * MarchShape<T>::CH * 3 * sizeof(double);
    }
};

// rows [ra, rb] of the strip starting at column x0 into their ring slots
template <typename T, int MW>
VV_DEV void march_load(const T* __restrict__ X, T* ring, int nx, int nv, int x0, int ra, int rb) {
    using RW = MarchRow<T, MW>;
    constexpr int NR = MarchShape<T>::NR;
    constexpr int NMAIN = MW * (int)sizeof(T) / 16;     // 16-byte chunks of the main columns
    constexpr int NCH = NMAIN + 2;
    constexpr int EPC = 16 / (int)sizeof(T);             // elements per 16-byte chunk
    const int nrow = rb - ra + 1;
    const int xl = x0 == 0 ? nx - 2 : x0 - 2;           // periodic halo columns
    const int xr = x0 + MW == nx ? 0 : x0 + MW;
    for (int idx = threadIdx.x; idx < nrow * NCH; idx += blockDim.x) {
        const int rr = idx / NCH, c = idx - rr * NCH;
        const int r = ra + rr;
        T* row = ring + ((r + NR) & (NR - 1)) * RW::RS;
        const bool in = r >= 0 && r < nv;
        const T* src = X + (size_t)(in ? r : 0) * nx;
        if (c < NMAIN) {
            cp_async_16(row + RW::LP + c * EPC, src + x0 + c * EPC, in ? 16 : 0);
        } else {
            const int gx = c == NMAIN ? xl : xr;
            T* dst = c == NMAIN ? row + RW::LP - 2 : row + RW::LP + MW;
            if (sizeof(T) == 8) cp_async_16(dst, src + gx, in ? 16 : 0);
            else cp_async_8(dst, src + gx, in ? 8 : 0);
        }
    }
}

// one (strip, segment) item of the marching stencil by a CTA of MW threads
// (block-uniform; the ring is idle when it returns)
template <int SCHEME, typename T, int MW>
VV_DEV void bracket_march_item(const T* __restrict__ X, T* __restrict__ Y, const BracketParams& p, int seg,
                               int strip, int segi) {
    using RW = MarchRow<T, MW>;
    constexpr int CH = MarchShape<T>::CH, NR = MarchShape<T>::NR;
    static_assert(NR >= 4 * CH + 4 && (NR & (NR - 1)) == 0, "ring of four chunks and the halo, a power of two");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ring = reinterpret_cast<T*>(smem_raw);
    double* rcb = reinterpret_cast<double*>(smem_raw + (size_t)NR * RW::RS * sizeof(T));   // [2][CH][3] row coefficients
    const int nx = p.nx, nv = p.nv;
    const int tx = threadIdx.x;
    const int x0 = strip * MW;
    const int i = x0 + tx;
    const int j_start = segi * seg;
    const int j_end = min(nv, j_start + seg);
    if (j_start >= j_end) return;
    // column coefficients (fixed for the thread)
    double b[5];
#pragma unroll
    for (int d = 0; d < 5; ++d) {
        int gi = i - 2 + d;
        gi = gi < 0 ? gi + nx : (gi >= nx ? gi - nx : gi);
        b[d] = b_fac(p, gi);
    }
    double bm_d, bp_d;
    Coef<SCHEME>::col(b[2] - b[1], b[3] - b[2], b[3] - b[1], b[2] - b[0], b[4] - b[2], bm_d, bp_d);
    const T B1 = T(b[3] - b[1]), bm = T(bm_d), bp = T(bp_d);
    const T tscale = T(((SCHEME == 2) ? p.f2 : p.f1) * p.factor);
    const T htinv = T(p.ht_inv);
    auto hv0 = [&](int j) -> double { return (j >= 0 && j < nv) ? p.h0[j] : 0.0; };
    // prologue: the first chunk with its halo, then the next two chunks (three
    // copy groups in flight; the compute of a chunk waits for its own group)
    march_load<T, MW>(X, ring, nx, nv, x0, j_start - 2, min(j_start + CH + 1, j_end + 1));
    cp_async_commit();
    for (int k = 1; k <= 2; ++k) {
        const int ra = j_start + k * CH + 2, rb = min(j_start + (k + 1) * CH + 1, j_end + 1);
        if (ra <= rb) march_load<T, MW>(X, ring, nx, nv, x0, ra, rb);
        cp_async_commit();
    }
    const int lx = RW::LP + tx;
    auto rowp = [&](int r) -> const T* { return ring + ((r + NR) & (NR - 1)) * RW::RS + lx; };
    T w0, w1, w2, w3, m0, m1, q0, q1;
    bool primed = false;
    int par = 0;
    for (int jc = j_start; jc < j_end; jc += CH, par ^= 1) {
        const int jn = min(jc + CH, j_end);
        double* rc = rcb + par * 3 * CH;
        // the chunk's row coefficients (A1, am, ap), once per CTA (the other
        // buffer may still be read by threads computing the previous chunk)
        if (tx < jn - jc) {
            const int j = jc + tx;
            const double a0 = hv0(j - 2), a1 = hv0(j - 1), a2 = hv0(j), a3 = hv0(j + 1), a4 = hv0(j + 2);
            double am_d, ap_d;
            Coef<SCHEME>::row(a2 - a1, a3 - a2, a3 - a1, a2 - a0, a4 - a2, am_d, ap_d);
            rc[3 * tx] = a3 - a1;
            rc[3 * tx + 1] = am_d;
            rc[3 * tx + 2] = ap_d;
        }
        cp_async_wait2();
        __syncthreads();
        // the third chunk ahead into the slots of the previous chunk, which
        // every thread has finished (it passed this barrier after computing it)
        {
            const int ra = jc + 3 * CH + 2, rb = min(jc + 4 * CH + 1, j_end + 1);
            if (ra <= rb) march_load<T, MW>(X, ring, nx, nv, x0, ra, rb);
            cp_async_commit();
        }
        if (!primed) {
            w0 = rowp(jc - 2)[0]; w1 = rowp(jc - 1)[0]; w2 = rowp(jc)[0]; w3 = rowp(jc + 1)[0];
            m0 = rowp(jc - 1)[-1]; m1 = rowp(jc)[-1];
            q0 = rowp(jc - 1)[1]; q1 = rowp(jc)[1];
            primed = true;
        }
        T* yout = Y + (size_t)jc * nx + i;
        // one output row; the window shifts by renaming when the loop is unrolled
        auto row_out = [&](int j, T* yo) {
            const T* r2 = rowp(j + 2);
            const T* r1 = rowp(j + 1);
            const T w4 = r2[0];
            const T m2 = r1[-1];
            const T q2 = r1[1];
            T y = htinv * w2;
            if (j >= 2 && j < nv - 2) {
                const double* cj = rc + 3 * (j - jc);
                const T A1 = T(cj[0]), am = T(cj[1]), ap = T(cj[2]);
                T s = T(0);
                if (Coef<SCHEME>::cA1 != 0.0 || Coef<SCHEME>::cA2 != 0.0) {
                    T ax = T(0), bx = T(0);
                    if (Coef<SCHEME>::cA1 != 0.0) {
                        ax = T(Coef<SCHEME>::cA1) * (q1 - m1);
                        bx = T(Coef<SCHEME>::cB1) * (w3 - w1);
                    }
                    if (Coef<SCHEME>::cA2 != 0.0) {
                        const T* r0 = rowp(j);
                        ax += T(Coef<SCHEME>::cA2) * (r0[2] - r0[-2]);
                        bx += T(Coef<SCHEME>::cB2) * (w4 - w0);
                    }
                    s = A1 * ax - B1 * bx;
                }
                s += am * (m0 - q0);
                s += ap * (m2 - q2);
                s += bm * (m0 - m2);
                s += bp * (q0 - q2);
                y += tscale * s;
            }
            *yo = y;
            w0 = w1; w1 = w2; w2 = w3; w3 = w4;
            m0 = m1; m1 = m2;
            q0 = q1; q1 = q2;
        };
        if (jn - jc == CH) {
#pragma unroll
            for (int k = 0; k < CH; ++k) row_out(jc + k, yout + (size_t)k * nx);
        } else {
            for (int j = jc; j < jn; ++j, yout += nx) row_out(j, yout);
        }
    }
    cp_async_wait0();
    __syncthreads();   // the ring is idle for the next item
}

template <int SCHEME, typename T, int MW>
__global__ void __launch_bounds__(MW)
k_bracket_march(const T* __restrict__ X, T* __restrict__ Y, BracketParams p, int seg) {
    if (p.xidx) X += (size_t)(*p.xidx) * p.xstride;
    bracket_march_item<SCHEME, T, MW>(X, Y, p, seg, blockIdx.x, blockIdx.y);
}

template <int SCHEME, int MODE, typename T, int AVG = AVG_POINT>
__global__ void __launch_bounds__(WTHREADS, 4)
k_bracket_wide(const T* __restrict__ X, const T* __restrict__ Xh, T* __restrict__ Y,
               BracketParams p, double* __restrict__ sumsq) {
    if (p.xidx) X += (size_t)(*p.xidx) * p.xstride;
    bracket_wide_tile<SCHEME, MODE, T, AVG>(X, Xh, Y, p, sumsq, blockIdx.x, blockIdx.y, gridDim.x);
}

}  // namespace vv
