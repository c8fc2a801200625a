/*
 * vv_port.c -- C/OpenMP restatement of viVlasov1D's implicit midpoint step.
 *
 * TEST INFRASTRUCTURE ONLY: this is the CPU port used as the timed CPU
 * baseline (bench.py's cpu_baseline leg and --impl reference) and checked
 * against the numpy oracle in tests/.  The product never links it.
 *
 * It follows the same reference files as oracle/vlasov_oracle.py:
 *   bracket J4 in the loop's operation order     PoissonBracket.pyx:335-389
 *   residual / JVP                               PETScNLVlasovMP.pyx:33-58
 *   Have axpy chain                              PETScVlasovSolver.pyx:142-157
 *   tensor-product kinetic preconditioner        TensorProductKinetic.pyx:345-359,
 *                                                TensorProductKineticFast.pyx:102-272,
 *                                                TensorProduct.pyx:109-116
 *     (band LU of each x mode; the port checks that LAPACK's partial
 *      pivoting would not swap rows and then factors without pivoting)
 *   moments                                      Toolbox.pyx:79-165
 *   CFD4 Poisson (exact circulant inverse)       PETScPoissonCFD4.pyx:146-183
 *   GMRES(restart) as PETSc KSPGMRES             (see oracle/vlasov_oracle.py)
 *   Picard loop, stop/revert rules               run_nonlinear_matrixfree_split_mp.py:111-174
 * Arrays use the flat layout F[j*nx + i].
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

typedef struct port {
    int nx, nv, nmodes, restart, max_it, snes_max_iter;
    size_t n;
    double L, vmin, vmax, ht, hx, hv, ht_inv, hx_inv, hv_inv, hx2_inv, f1, f2, charge, mass;
    double ksp_rtol, ksp_atol, snes_atol;
    double *v, *h0, *f, *fh, *fl, *phi, *h1c, *h1h, *nn;
    double *tmp, *b, *x, *V, *H;  /* H: Have (nx*nv) */
    cplx *tw, *lam, *dinv, *spec;
    double *alpha, *gamma, *sym_inv;
    int pivot;
} port;

static double now_dot(const double* a, const double* b, size_t n) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* ---- FFT: iterative radix-2 complex FFT of length m (power of two) ---- */
static void fft_inplace(cplx* a, int m, const cplx* tw, int twstride, int inverse) {
    for (int i = 1, j = 0; i < m; ++i) {
        int bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { cplx t = a[i]; a[i] = a[j]; a[j] = t; }
    }
    for (int len = 2; len <= m; len <<= 1) {
        const int step = m / len;
        for (int i = 0; i < m; i += len)
            for (int k = 0; k < len / 2; ++k) {
                cplx w = tw[(size_t)k * step * twstride];
                if (inverse) w = conj(w);
                const cplx u = a[i + k], t = w * a[i + k + len / 2];
                a[i + k] = u + t;
                a[i + k + len / 2] = u - t;
            }
    }
}

/* real FFT of length nx via a complex FFT of length nx/2; out[0..nx/2] */
static void rfft_row(const port* p, const double* x, cplx* out, cplx* work) {
    const int M = p->nx / 2;
    for (int m = 0; m < M; ++m) work[m] = x[2 * m] + I * x[2 * m + 1];
    fft_inplace(work, M, p->tw, 2, 0);
    for (int k = 0; k <= M; ++k) {
        const cplx zk = work[k == M ? 0 : k], zc = conj(work[k == 0 ? 0 : M - k]);
        const cplx E = 0.5 * (zk + zc), O = -0.5 * I * (zk - zc);
        const cplx w = (k < M) ? p->tw[k] : -1.0;
        out[k] = E + w * O;
    }
}

static void irfft_row(const port* p, const cplx* Xin, double* y, cplx* work, cplx* X) {
    const int M = p->nx / 2;
    for (int k = 0; k <= M; ++k) X[k] = Xin[k];
    X[0] = creal(X[0]);
    X[M] = creal(X[M]);
    for (int k = 0; k < M; ++k) {
        const cplx xk = X[k], xc = conj(X[M - k]);
        const cplx E = 0.5 * (xk + xc), O = conj(p->tw[k]) * 0.5 * (xk - xc);
        work[k] = E + I * O;
    }
    fft_inplace(work, M, p->tw, 2, 1);
    const double s = 1.0 / M;
    for (int m = 0; m < M; ++m) {
        y[2 * m] = creal(work[m]) * s;
        y[2 * m + 1] = cimag(work[m]) * s;
    }
}

/* ---- preconditioner ---- */
static void pc_apply(port* p, const double* X, double* Y) {
    const int nx = p->nx, nv = p->nv, nm = p->nmodes;
#pragma omp parallel
    {
        cplx* work = malloc(sizeof(cplx) * (nx / 2 + 2));
        cplx* row = malloc(sizeof(cplx) * (nm + 1));
#pragma omp for schedule(static)
        for (int j = 0; j < nv; ++j) {
            rfft_row(p, X + (size_t)j * nx, row, work);
            for (int k = 0; k < nm; ++k) p->spec[(size_t)k * nv + j] = row[k];
        }
#pragma omp for schedule(static)
        for (int k = 0; k < nm; ++k) {
            cplx* b = p->spec + (size_t)k * nv;
            const cplx* di = p->dinv + (size_t)k * nv;
            const cplx lam = p->lam[k];
            for (int r = 1; r < nv; ++r) b[r] -= (lam * p->alpha[r] * di[r - 1]) * b[r - 1];
            b[nv - 1] = b[nv - 1] * di[nv - 1];
            for (int r = nv - 2; r >= 0; --r) b[r] = (b[r] - lam * p->gamma[r] * b[r + 1]) * di[r];
        }
#pragma omp for schedule(static)
        for (int j = 0; j < nv; ++j) {
            for (int k = 0; k < nm; ++k) row[k] = p->spec[(size_t)k * nv + j];
            cplx* X2 = malloc(sizeof(cplx) * (nm + 1));
            irfft_row(p, row, Y + (size_t)j * nx, work, X2);
            free(X2);
        }
        free(work);
        free(row);
    }
}

/* ---- bracket (J4, reference operation order) ---- */
#define XX(di, dj) x[(size_t)(j + (dj)) * nx + ((i + (di) + nx) % nx)]
#define HH(di, dj) h[(size_t)(j + (dj)) * nx + ((i + (di) + nx) % nx)]
static void bracket_j4(const port* p, const double* x, const double* h, double* y, double factor) {
    const int nx = p->nx, nv = p->nv;
    const double f1 = p->f1, f2 = p->f2;
#pragma omp parallel for schedule(static)
    for (int j = 2; j < nv - 2; ++j)
        for (int i = 0; i < nx; ++i) {
            const double jpp1 = (XX(1, 0) - XX(-1, 0)) * (HH(0, 1) - HH(0, -1)) - (XX(0, 1) - XX(0, -1)) * (HH(1, 0) - HH(-1, 0));
            const double jpc1 = XX(1, 0) * (HH(1, 1) - HH(1, -1)) - XX(-1, 0) * (HH(-1, 1) - HH(-1, -1)) -
                                XX(0, 1) * (HH(1, 1) - HH(-1, 1)) + XX(0, -1) * (HH(1, -1) - HH(-1, -1));
            const double jcp1 = XX(1, 1) * (HH(0, 1) - HH(1, 0)) - XX(-1, -1) * (HH(-1, 0) - HH(0, -1)) -
                                XX(-1, 1) * (HH(0, 1) - HH(-1, 0)) + XX(1, -1) * (HH(1, 0) - HH(0, -1));
            const double jcc2 = (XX(1, 1) - XX(-1, -1)) * (HH(-1, 1) - HH(1, -1)) - (XX(-1, 1) - XX(1, -1)) * (HH(1, 1) - HH(-1, -1));
            const double jpc2 = XX(2, 0) * (HH(1, 1) - HH(1, -1)) - XX(-2, 0) * (HH(-1, 1) - HH(-1, -1)) -
                                XX(0, 2) * (HH(1, 1) - HH(-1, 1)) + XX(0, -2) * (HH(1, -1) - HH(-1, -1));
            const double jcp2 = XX(1, 1) * (HH(0, 2) - HH(2, 0)) - XX(-1, -1) * (HH(-2, 0) - HH(0, -2)) -
                                XX(-1, 1) * (HH(0, 2) - HH(-2, 0)) + XX(1, -1) * (HH(2, 0) - HH(0, -2));
            const double r1 = (jpp1 + jpc1 + jcp1) * f1, r2 = (jcc2 + jpc2 + jcp2) * f2;
            y[(size_t)j * nx + i] += factor * (2. * r1 - r2);
        }
}
#undef XX
#undef HH

static void build_have(port* p) {
    const int nx = p->nx, nv = p->nv;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nv; ++j)
        for (int i = 0; i < nx; ++i) {
            double h = p->h0[j];
            h = h + 0.5 * p->h1c[i];
            h = h + 0.5 * p->h1h[i];
            p->H[(size_t)j * nx + i] = h;   /* h2 = 0 */
        }
}

static void residual(port* p, const double* F, double* Y) {
    const size_t n = p->n;
    double* Fave = p->fl == F ? NULL : NULL;
    (void)Fave;
    double* A = p->b;   /* scratch: Fave */
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < n; ++k) {
        A[k] = 0.5 * p->fh[k] + 0.5 * F[k];
        Y[k] = p->ht_inv * (F[k] - p->fh[k]);
    }
    bracket_j4(p, A, p->H, Y, 1.0);
}

static void jvp(port* p, const double* X, double* Y) {
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < p->n; ++k) Y[k] = p->ht_inv * X[k];
    bracket_j4(p, X, p->H, Y, 0.5);
}

static void op(port* p, const double* X, double* Y) {
    jvp(p, X, p->tmp);
    pc_apply(p, p->tmp, Y);
}

/* ---- moments + Poisson + h1 ---- */
static void moments_poisson(port* p) {
    const int nx = p->nx, nv = p->nv, M = nx / 2;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
        double s = 0.0;
        for (int j = 0; j < nv; ++j) s += p->f[(size_t)j * nx + i];
        p->nn[i] = s * p->hv;
    }
    double nmean = 0.0;
    for (int i = 0; i < nx; ++i) nmean += p->nn[i];
    nmean /= nx;
    double* bb = malloc(sizeof(double) * nx);
    cplx* work = malloc(sizeof(cplx) * (M + 2));
    cplx* X = malloc(sizeof(cplx) * (M + 2));
    cplx* X2 = malloc(sizeof(cplx) * (M + 2));
    for (int i = 0; i < nx; ++i) bb[i] = -(p->nn[i] - nmean) * p->charge;
    rfft_row(p, bb, X, work);
    for (int k = 0; k <= M; ++k) X[k] *= p->sym_inv[k];
    irfft_row(p, X, p->phi, work, X2);
    double s = 0.0;
    for (int i = 0; i < nx; ++i) s += p->phi[i];
    for (int i = 0; i < nx; ++i) p->h1c[i] = p->phi[i] - s / nx;
    free(bb); free(work); free(X); free(X2);
}

static double poisson_resnorm(const port* p) {
    const int nx = p->nx;
    double nmean = 0.0, r2 = 0.0;
    for (int i = 0; i < nx; ++i) nmean += p->nn[i];
    nmean /= nx;
    const double* x = p->phi;
    for (int i = 0; i < nx; ++i) {
        const double r = (5. * x[(i - 2 + 2 * nx) % nx] - 32. * x[(i - 1 + nx) % nx] + 54. * x[i] -
                          32. * x[(i + 1) % nx] + 5. * x[(i + 2) % nx]) * p->hx2_inv / 12. +
                         (p->nn[i] - nmean) * p->charge;
        r2 += r * r;
    }
    return sqrt(r2);
}

static double calc_residual(port* p) {
    residual(p, p->f, p->tmp);
    return sqrt(now_dot(p->tmp, p->tmp, p->n)) + poisson_resnorm(p);
}

/* ---- GMRES (PETSc semantics, zero initial guess) ---- */
static int gmres(port* p, const double* b, double* x, int* its_out) {
    const size_t n = p->n;
    const int R = p->restart;
    double* V = p->V;
    double *hh = calloc((size_t)(R + 2) * (R + 1), sizeof(double)), *grs = calloc(R + 2, sizeof(double));
    double *cc = calloc(R + 1, sizeof(double)), *ss = calloc(R + 1, sizeof(double)), *hcol = calloc(R + 2, sizeof(double));
    double *nrs = calloc(R + 1, sizeof(double));
#define HHm(a, c) hh[(size_t)(c) * (R + 2) + (a)]
    int its = 0, reason = 0, guess_zero = 1;
    double rnorm0 = 0.0, ttol = 0.0;
    memset(x, 0, n * sizeof(double));
    while (!reason) {
        if (guess_zero) memcpy(V, b, n * sizeof(double));
        else {
            op(p, x, V);
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < n; ++k) V[k] = b[k] - V[k];
        }
        double res = sqrt(now_dot(V, V, n));
        if (res != 0.0) {
            const double s = 1.0 / res;
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < n; ++k) V[k] *= s;
        }
        grs[0] = res;
        if (res == 0.0) { reason = 3; break; }
        if (its == 0) { rnorm0 = res; ttol = fmax(p->ksp_rtol * res, p->ksp_atol); }
        if (res <= ttol) reason = res < p->ksp_atol ? 3 : 2;
        else if (res >= 1e5 * rnorm0) reason = -4;
        int it = 0;
        while (!reason && it < R && its < p->max_it) {
            double* w = V + (size_t)(it + 1) * n;
            op(p, V + (size_t)it * n, w);
            for (int j = 0; j <= it; ++j) hcol[j] = now_dot(w, V + (size_t)j * n, n);
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < n; ++k) {
                double wk = w[k];
                for (int j = 0; j <= it; ++j) wk += -hcol[j] * V[(size_t)j * n + k];
                w[k] = wk;
            }
            for (int j = 0; j <= it; ++j) HHm(j, it) = hcol[j];
            const double tt = sqrt(now_dot(w, w, n));
            if (tt != 0.0) {
                const double s = 1.0 / tt;
#pragma omp parallel for schedule(static)
                for (size_t k = 0; k < n; ++k) w[k] *= s;
            }
            HHm(it + 1, it) = tt;
            double hapbnd = fabs(tt / grs[it]);
            if (hapbnd > 1e-30) hapbnd = 1e-30;
            const int hapend = tt < hapbnd;
            for (int j = 1; j <= it; ++j) {
                const double t = HHm(j - 1, it);
                HHm(j - 1, it) = cc[j - 1] * t + ss[j - 1] * HHm(j, it);
                HHm(j, it) = cc[j - 1] * HHm(j, it) - ss[j - 1] * t;
            }
            int null = 0;
            if (!hapend) {
                const double t = sqrt(HHm(it, it) * HHm(it, it) + HHm(it + 1, it) * HHm(it + 1, it));
                if (t == 0.0) { reason = -2; null = 1; }
                else {
                    cc[it] = HHm(it, it) / t;
                    ss[it] = HHm(it + 1, it) / t;
                    grs[it + 1] = -(ss[it] * grs[it]);
                    grs[it] = cc[it] * grs[it];
                    HHm(it, it) = cc[it] * HHm(it, it) + ss[it] * HHm(it + 1, it);
                    res = fabs(grs[it + 1]);
                }
            } else res = 0.0;
            ++it;
            ++its;
            if (null) break;
            if (isnan(res)) reason = -9;
            else if (res <= ttol) reason = res < p->ksp_atol ? 3 : 2;
            else if (res >= 1e5 * rnorm0) reason = -4;
            if (hapend && !reason) { reason = -5; break; }
        }
        const int last = it - 1;
        if (last >= 0 && HHm(last, last) != 0.0) {
            nrs[last] = grs[last] / HHm(last, last);
            for (int ii = 1; ii <= last; ++ii) {
                const int k = last - ii;
                double t = grs[k];
                for (int j = k + 1; j <= last; ++j) t -= HHm(k, j) * nrs[j];
                nrs[k] = t / HHm(k, k);
            }
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < n; ++k) {
                double s = 0.0;
                for (int j = 0; j <= last; ++j) s += nrs[j] * V[(size_t)j * n + k];
                x[k] += s;
            }
        }
        if (its >= p->max_it) { if (!reason) reason = -3; break; }
        guess_zero = 0;
    }
#undef HHm
    free(hh); free(grs); free(cc); free(ss); free(hcol); free(nrs);
    *its_out = its;
    return reason;
}

/* ---- public ---- */
port* vvp_create(int nx, int nv, double L, double vmin, double vmax, double ht, double charge, double mass,
                 double ksp_rtol, double ksp_atol, int ksp_max_it, double snes_atol, int snes_max_iter, int restart) {
    if (nx < 4 || (nx & (nx - 1)) || nv < 5) return NULL;
    port* p = calloc(1, sizeof(port));
    p->nx = nx; p->nv = nv; p->n = (size_t)nx * nv; p->nmodes = nx / 2 + 1;
    p->L = L; p->vmin = vmin; p->vmax = vmax; p->ht = ht; p->charge = charge; p->mass = mass;
    p->ksp_rtol = ksp_rtol; p->ksp_atol = ksp_atol; p->max_it = ksp_max_it;
    p->snes_atol = snes_atol; p->snes_max_iter = snes_max_iter; p->restart = restart;
    p->hx = L / nx; p->hv = (vmax - vmin) / (nv - 1);
    p->ht_inv = 1. / ht; p->hx_inv = 1. / p->hx; p->hv_inv = 1. / p->hv; p->hx2_inv = 1. / (p->hx * p->hx);
    p->f1 = p->hx_inv * p->hv_inv / 12.; p->f2 = p->hx_inv * p->hv_inv / 24.;
    const size_t n = p->n;
    p->v = malloc(nv * sizeof(double)); p->h0 = malloc(nv * sizeof(double));
    p->alpha = malloc(nv * sizeof(double)); p->gamma = malloc(nv * sizeof(double));
    p->f = calloc(n, sizeof(double)); p->fh = calloc(n, sizeof(double)); p->fl = calloc(n, sizeof(double));
    p->tmp = calloc(n, sizeof(double)); p->b = calloc(n, sizeof(double)); p->x = calloc(n, sizeof(double));
    p->H = calloc(n, sizeof(double)); p->V = calloc((size_t)(restart + 1) * n, sizeof(double));
    p->phi = calloc(nx, sizeof(double)); p->h1c = calloc(nx, sizeof(double)); p->h1h = calloc(nx, sizeof(double));
    p->nn = calloc(nx, sizeof(double));
    p->tw = malloc(sizeof(cplx) * (nx / 2)); p->lam = malloc(sizeof(cplx) * p->nmodes);
    p->dinv = malloc(sizeof(cplx) * p->nmodes * nv); p->spec = malloc(sizeof(cplx) * p->nmodes * nv);
    p->sym_inv = malloc(sizeof(double) * p->nmodes);
    for (int j = 0; j < nv; ++j) { p->v[j] = vmin + j * p->hv; p->h0[j] = 0.5 * (p->v[j] * p->v[j]) * mass; }
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < nx / 2; ++k) {
        const long double a = 2.0L * PI * k / nx;
        p->tw[k] = (double)cosl(a) - I * (double)sinl(a);
    }
    cplx* e = malloc(sizeof(cplx) * nx);
    for (int i = 0; i < nx; ++i) {
        const double t2 = (2.0 * M_PI * i) / nx, t1 = t2 * (nx - 1);
        e[i] = (cos(t1) + I * sin(t1)) - (cos(t2) + I * sin(t2));
    }
    for (int k = 0; k < p->nmodes; ++k) p->lam[k] = e[(k + nx / 2) % nx];
    free(e);
    const double arak = 0.5 * p->hx_inv * p->hv_inv / 12., hv2 = p->hv * p->hv;
    for (int j = 0; j < nv; ++j) {
        p->alpha[j] = 0.5 * (2. * p->hv * p->v[j] - hv2) * arak;
        p->gamma[j] = 0.5 * (2. * p->hv * p->v[j] + hv2) * arak;
    }
    for (int k = 0; k < p->nmodes; ++k) {
        cplx d = 0;
        for (int r = 0; r < nv; ++r) {
            const cplx diag = p->lam[k] * (4. * p->hv * p->v[r]) * arak + p->ht_inv;
            cplx dn = diag;
            if (r > 0) {
                const cplx sub = p->lam[k] * p->alpha[r], sup = p->lam[k] * p->gamma[r - 1];
                if (fabs(creal(sub)) + fabs(cimag(sub)) > fabs(creal(d)) + fabs(cimag(d))) p->pivot = 1;
                dn = diag - (sub / d) * sup;
            }
            d = dn;
            p->dinv[(size_t)k * nv + r] = 1.0 / d;
        }
    }
    for (int k = 0; k < p->nmodes; ++k) {
        const long double t = 2.0L * PI * k / nx;
        const long double s = (54.0L - 64.0L * cosl(t) + 10.0L * cosl(2.0L * t)) * p->hx2_inv / 12.0L;
        p->sym_inv[k] = k == 0 ? 0.0 : (double)(1.0L / s);
    }
    return p;
}

void vvp_destroy(port* p) {
    if (!p) return;
    void* b[] = {p->v, p->h0, p->alpha, p->gamma, p->f, p->fh, p->fl, p->tmp, p->b, p->x, p->H, p->V, p->phi,
                 p->h1c, p->h1h, p->nn, p->tw, p->lam, p->dinv, p->spec, p->sym_inv};
    for (size_t k = 0; k < sizeof b / sizeof b[0]; ++k) free(b[k]);
    free(p);
}

int vvp_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int vvp_pivot_needed(const port* p) { return p->pivot; }

/* set f (normalise as run_base.py:623-628 when asked), then moments/Poisson */
void vvp_set_f(port* p, const double* f, int normalise) {
    memcpy(p->f, f, p->n * sizeof(double));
    if (normalise) {
        double s = 0.0;
        for (size_t k = 0; k < p->n; ++k) s += p->f[k];
        const double nave = s * p->hv / p->nx, sc = 1. / nave;
        for (size_t k = 0; k < p->n; ++k) p->f[k] *= sc;
    }
    moments_poisson(p);
}

void vvp_get_f(const port* p, double* f) { memcpy(f, p->f, p->n * sizeof(double)); }
void vvp_get_phi(const port* p, double* phi) { memcpy(phi, p->phi, p->nx * sizeof(double)); }

/* one time step; returns Picard iterations, *gmres_total gets the GMRES sum */
int vvp_step(port* p, int* gmres_total) {
    memcpy(p->fh, p->f, p->n * sizeof(double));
    memcpy(p->h1h, p->h1c, p->nx * sizeof(double));
    build_have(p);
    double pred = calc_residual(p);
    int i = 0, tot = 0;
    for (;;) {
        ++i;
        memcpy(p->fl, p->f, p->n * sizeof(double));
        residual(p, p->f, p->tmp);
        pc_apply(p, p->tmp, p->b);
        double* bcopy = malloc(p->n * sizeof(double));
        memcpy(bcopy, p->b, p->n * sizeof(double));
        int its = 0;
        const int reason = gmres(p, bcopy, p->x, &its);
        free(bcopy);
        tot += its;
        if (reason >= 0) {
#pragma omp parallel for schedule(static)
            for (size_t k = 0; k < p->n; ++k) p->f[k] -= p->x[k];
        }
        moments_poisson(p);
        build_have(p);
        const double prev = pred;
        pred = calc_residual(p);
        if ((pred > prev && i > 1) || pred < p->snes_atol || i >= p->snes_max_iter) {
            if (pred > prev) {
                memcpy(p->f, p->fl, p->n * sizeof(double));
                moments_poisson(p);
            }
            break;
        }
    }
    if (gmres_total) *gmres_total = tot;
    return i;
}

/* one time step of n independent runs, the runs spread over the host threads
 * (each run single-threaded inside: the kernels' own parallel loops are nested
 * regions, which run on one thread) -- how a sweep of separate runs uses a
 * many-core host.  picard[i], gmres[i] get each run's counts. */
void vvp_step_many(port** ps, int n, int* picard, int* gmres_total) {
#ifdef _OPENMP
    const int saved = omp_get_max_active_levels();
    omp_set_max_active_levels(1);
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) {
        int g = 0;
        const int p = vvp_step(ps[i], &g);
        if (picard) picard[i] = p;
        if (gmres_total) gmres_total[i] = g;
    }
#ifdef _OPENMP
    omp_set_max_active_levels(saved);
#endif
}
