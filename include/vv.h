/*
 * vv.h -- C ABI of libvv, a B200 (sm_100a) implementation of viVlasov1D's
 * implicit variational (midpoint) time step for the 1D1V Vlasov-Poisson
 * system: Arakawa J1/J2/J4 bracket residual and Jacobian-vector product,
 * FFT tensor-product kinetic preconditioner, periodic CFD4 Poisson solve,
 * moments, restarted GMRES and the Picard-over-phi step, and the invariant
 * diagnostics.
 *
 * Conventions
 *   - Every entry point returns an int status (VV_OK == 0).  No call aborts
 *     the process and no device wait in the library is unbounded.
 *   - Field buffers are DEVICE pointers to nx*nv doubles in the reference's
 *     PETSc natural ordering: F[j*nx + i], x (i, periodic) fastest, v (j,
 *     bounded) slowest -- the layout of the DMDA ``da1`` global vector
 *     (vlasov/run/run_base.py:215-220).  x profiles (phi, h1, h2, n, u, e, a)
 *     are device pointers to nx doubles.
 *   - Work is enqueued on the stream set with vv_set_stream (default: the
 *     legacy default stream).  Calls that return a host scalar synchronise
 *     that stream.
 *   - The Hamiltonian is never stored as an nx*nv array: h = h0(v) + h1(x)
 *     (+ h2(x)) is separable, so the solver keeps the 1-D profiles and the
 *     kernels regenerate h on the fly.
 *
 * Every function names the reference interface it replaces (file:line,
 * relative to the viVlasov1D project root).
 */
#ifndef VIVLASOV1D_B200_VV_H
#define VIVLASOV1D_B200_VV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum vv_status {
    VV_OK = 0,
    VV_ERR_ARG = 1,          /* invalid argument or NULL pointer             */
    VV_ERR_UNSUPPORTED = 2,  /* configuration the library does not support  */
    VV_ERR_CUDA = 3,         /* a CUDA runtime call failed                   */
    VV_ERR_ALLOC = 4,        /* device allocation failed                     */
    VV_ERR_DIVERGED = 5,     /* Picard residual above the abort threshold    */
    VV_ERR_NAN = 6,          /* NaN/Inf met in a norm                        */
    VV_ERR_TIMEOUT = 7       /* a bounded device wait gave up                */
};

/* ---- discretisation choices (vlasov/core/config.py:63-126) ------------- */
enum vv_bracket {            /* solver.poisson_bracket                        */
    VV_BRACKET_J1 = 1,       /* PoissonBracket.pyx:68-186                      */
    VV_BRACKET_J2 = 2,       /* PoissonBracket.pyx:188-306                     */
    VV_BRACKET_J4 = 4,       /* PoissonBracket.pyx:309-403 (default)           */
    VV_BRACKET_SIMPSON = 5   /* PoissonBracket.pyx:405-492                     */
};
enum vv_preconditioner {     /* solver.preconditioner_scheme                  */
    VV_PC_NONE = 0,
    VV_PC_TENSOR_KINETIC = 1,   /* TensorProductKineticFast.pyx                */
    VV_PC_TENSOR_POTENTIAL = 2  /* TensorProductPotentialFast.pyx              */
};
enum vv_laplace {            /* solver.laplace_operator (run_base.py:93-94
                                imports PETScPoisson<laplace_operator>)       */
    VV_LAPLACE_CFD2 = 2,     /* PETScPoissonCFD2.pyx                           */
    VV_LAPLACE_CFD4 = 4,     /* PETScPoissonCFD4.pyx (default)                 */
    VV_LAPLACE_SIMPSON = 5,  /* PETScPoissonSimpson.pyx                        */
    VV_LAPLACE_CFD2_AVE = 12,   /* PETScPoissonCFD2Ave.pyx: the CFD2 Laplacian,
                                   density averaged (1 2 1)/4 in the RHS       */
    VV_LAPLACE_SIMPSON_AVE = 15 /* PETScPoissonSimpsonAve.pyx: the Simpson
                                   Laplacian, density (1 8 18 8 1)/36          */
};
enum vv_averaging {          /* solver.averaging_operator: the time derivative
                                (TimeDerivative.pyx:36-53; 0 for None/'none') */
    VV_AVERAGING_POINT = 0,     /* TimeDerivative: Y += F/ht (default)         */
    VV_AVERAGING_MIDPOINT = 1,  /* TimeDerivativeMidpoint (:84-157), also the
                                   arakawa_J1 class (:236-237)                 */
    VV_AVERAGING_ARAKAWA_J2 = 2,/* TimeDerivativeArakawaJ2 (:240-242) = point  */
    VV_AVERAGING_ARAKAWA_J4 = 4,/* TimeDerivativeArakawaJ4 (:245-321)          */
    VV_AVERAGING_SIMPSON = 5    /* TimeDerivativeSimpson (:160-233)            */
};
enum vv_collision {          /* solver.collision_operator with dissipation_type
                                = 'collisions' (CollisionOperator.pyx:44-58)  */
    VV_COLLISION_NONE = 0,
    VV_COLLISION_T = 1,      /* collT: CollisionOperator.pyx:68-157            */
    VV_COLLISION_E = 2       /* collE: CollisionOperator.pyx:160-250           */
};
enum vv_double_bracket {     /* solver.bracket_operator with dissipation_type
                                = 'double_bracket' (DoubleBracket.pyx:46-55)  */
    VV_DOUBLE_BRACKET_NONE = 0,
    VV_DOUBLE_BRACKET_FFH = 1,  /* DoubleBracketFFH: DoubleBracket.pyx:67-83   */
    VV_DOUBLE_BRACKET_FHH = 2   /* DoubleBracketFHH: DoubleBracket.pyx:86-97   */
};
enum vv_initial_guess {      /* solver.initial_guess: the explicit predictor of
                                the step's first iterate (run_base.py:173-181,
                                786-912; runspec.cfg:58 names)                 */
    VV_GUESS_NONE = 0,
    VV_GUESS_SYMPLECTIC2 = 1,   /* 'symplectic2': PETScArakawaSymplectic.pyx:62-92
                                   kinetic 1/2, potential 1, kinetic 1/2       */
    VV_GUESS_SYMPLECTIC4 = 2,   /* 'symplectic4': the 4th-order composition of
                                   run_base.py:887-912                         */
    VV_GUESS_RK4_16 = 3,        /* 'rk4_16': PETScArakawaRungeKutta.pyx:20-58   */
    VV_GUESS_RK4_18 = 4         /* 'rk4_18' and the option key 'rk4' (whose
                                   method calls the undefined rk18_J4):
                                   PETScArakawaRungeKutta.pyx:61-100, 3/8 rule */
};
enum vv_order {              /* arithmetic of the bracket kernels             */
    VV_ORDER_FACTORED = 0,   /* separable-h coefficient form (fast, default)   */
    VV_ORDER_REFERENCE = 1   /* the reference loop's operation order, no FMA   */
};
enum vv_precision {          /* arithmetic of the linear (GMRES) solve        */
    VV_PRECISION_FP64 = 0,   /* everything in FP64, as the reference           */
    VV_PRECISION_MIXED = 1   /* GMRES basis, JVP and preconditioner in FP32;
                                residual, Picard decisions, moments, Poisson
                                and invariants in FP64 (the Picard loop refines
                                the FP32 linear solves to the FP64 residual)   */
};

/* ---- grid and run parameters (runspec.cfg [grid], [initial_data]) ------- */
typedef struct vv_grid {
    int32_t nx;              /* points in x (periodic)                        */
    int32_t nv;              /* points in v (bounded), nv >= 5                */
    double  L;               /* x length; hx = L/nx                           */
    double  vmin, vmax;      /* hv = (vmax-vmin)/(nv-1)                       */
    double  ht;              /* time step                                     */
    double  charge;          /* particle charge (examples use -1)             */
    double  mass;            /* particle mass                                 */
    int32_t bracket;         /* enum vv_bracket                               */
    int32_t preconditioner;  /* enum vv_preconditioner                        */
    int32_t laplace;         /* enum vv_laplace                               */
    int32_t order;           /* enum vv_order                                 */
    int32_t gmres_restart;   /* restart length (PETSc default 30), <= 64      */
    int32_t precision;       /* enum vv_precision                             */
    double  mixed_rtol;      /* VV_PRECISION_MIXED only: relative tolerance of
                                the FP32 linear solves inside vv_step and the
                                batch step (<= 0: 1e-2; never below the KSP
                                rtol).  The FP64 Picard residual refines the
                                solution to the same fixed point, as in
                                mixed-precision iterative refinement; FP32
                                Krylov vectors cannot reduce a residual near
                                the FP64 round-off floor by 1e-4 cheaply.
                                vv_gmres always uses the rtol it is given.    */
    int32_t averaging;       /* enum vv_averaging (0: point).  The averaged
                                operators replace F/ht on the rows
                                2 <= j < nv-2 by a 9- or 13-point stencil of
                                F times 1/(ht d); they are supported by the
                                single-instance step, not by vv_batch_create
                                or vv_step_adjoint (VV_ERR_UNSUPPORTED).      */
    int32_t collision;       /* enum vv_collision (0: none); active only with
                                coll_freq != 0, as config.py:148-154.  The
                                residual and Jacobian then add the operator
                                with the moments of vv_set_moments (vv_step:
                                the state's n, u, a and their copies at
                                make_history).  Single runs only: not in
                                vv_batch_create or vv_step_adjoint.          */
    double  coll_freq;       /* runspec coll_freq (collision frequency)       */
    double  coll_diff;       /* runspec coll_diff (weight of diffusion, 1)    */
    double  coll_drag;       /* runspec coll_drag (weight of drag, 1)         */
    int32_t double_bracket;  /* enum vv_double_bracket (0: none); active only
                                with coll_freq != 0 (nu = coll_freq), as
                                config.py:156-162.  FP64 only (a mixed context
                                returns VV_ERR_UNSUPPORTED); its brackets run in
                                the reference's operation order; the Jacobian
                                uses the Fave of the last residual evaluation
                                (vv_function / the step's residual).  Single
                                runs only.                                    */
    int32_t initial_guess;   /* enum vv_initial_guess (0: none).  The
                                explicit classes of the reference compute no
                                bracket step as written; the predictor here
                                calls the bracket with the arguments in the
                                order of its signature (PoissonBracket.pyx:80;
                                the classes pass (x, y, h)), on cleared work
                                vectors, and with the sign of the implicit
                                residual, df/dt = -[f, h] (with the classes'
                                sign it steps backwards in time and the guard
                                discards every guess).  Single runs only (not
                                in vv_batch_create).                          */
    int32_t initial_iter;    /* runspec initial_iter: predictor iterations of
                                ht/initial_iter each (<= 0: 1)                */
} vv_grid;

typedef struct vv_ctx vv_ctx;

/* ---- lifetime ----------------------------------------------------------- */
/* Allocate a solver for one grid: the GMRES basis, spectra, reduction
 * scratch and the preconditioner's factorised band matrices.  Replaces the
 * construction of PETScVlasovSolver (PETScVlasovSolver.pyx:27-104) together
 * with TensorProductPreconditionerKineticFast (TensorProductKineticFast.pyx:
 * 25-93: eigenvalues, band matrices, one LU factorisation per x mode). */
int vv_create(const vv_grid* grid, vv_ctx** out);
int vv_destroy(vv_ctx* ctx);
int vv_set_stream(vv_ctx* ctx, void* cuda_stream);
const char* vv_status_string(int status);
int vv_version(void);
/* Velocity grid v_j and the kinetic Hamiltonian profile h0_j = 0.5 v_j^2 m
 * (Toolbox.pyx:175-187) copied to host arrays of nv doubles. */
int vv_grid_vectors(vv_ctx* ctx, double* v_host, double* h0_host);

/* ---- PETScVlasovSolver interface ---------------------------------------- */
/* update_history(F): Fh <- F                   PETScVlasovSolver.pyx:135-140 */
int vv_update_history(vv_ctx* ctx, const double* F);
/* update_previous: Have <- H0 + .5 H1p + .5 H1h + .5 H2p + .5 H2h
 * (PETScVlasovSolver.pyx:142-157).  Arguments are x profiles of h1/h2 at the
 * current Picard iterate (p) and the previous time level (h); NULL means
 * zero.  The profiles are copied (a snapshot, as the reference's Have). */
int vv_update_previous(vv_ctx* ctx, const double* h1p, const double* h1h,
                       const double* h2p, const double* h2h);
/* function(F, Y) / function_solver: Y = P^-1 R(F) or R(F) with
 * R(F) = (F - Fh)/ht + [ (F+Fh)/2, Have ]   PETScVlasovSolver.pyx:168-174,
 * PETScNLVlasovMP.pyx:43-58 */
int vv_function(vv_ctx* ctx, const double* F, double* Y, int apply_pc);
/* jacobian(F, Y) / jacobian_solver: Y = P^-1 J F or J F with
 * J F = F/ht + 0.5 [F, Have]      PETScVlasovSolver.pyx:160-166, 176-186,
 * PETScNLVlasovMP.pyx:33-40 (also mult/snes_mult/jacobian_mult) */
int vv_jacobian(vv_ctx* ctx, const double* F, double* Y, int apply_pc);
/* function_norm(F, Y): Y = R(F), *norm = ||Y||_2 (host scalar)
 *                                           PETScVlasovSolver.pyx:196-198 */
int vv_function_norm(vv_ctx* ctx, const double* F, double* Y, double* norm);
/* PoissonBracket.function: Y += factor * [X, Have] on rows 2 <= j < nv-2
 *                                   PoissonBracket.pyx:70-75, 325-330 */
int vv_bracket(vv_ctx* ctx, const double* X, double* Y, double factor);

/* ---- TensorProductPreconditioner ---------------------------------------- */
/* tensorProduct(X, Y): Y = P^-1 X     TensorProductKinetic.pyx:345-359,
 * TensorProductKineticFast.pyx:102-224.  X and Y may alias. */
int vv_pc_apply(vv_ctx* ctx, const double* X, double* Y);
/* update_matrices() of the potential preconditioner: its x-tridiagonal
 * matrices are built from phi (nx values; the solver's phi at update_history)
 * TensorProductPotentialFast.pyx:205-266, PETScVlasovSolver.pyx:135-140.
 * The time step (vv_step) takes phi at its own make_history.  A no-op for the
 * other preconditioners. */
int vv_pc_set_potential(vv_ctx* ctx, const double* phi);
/* PETScVlasovSolver.set_moments (PETScVlasovSolver.pyx:123-132): the current
 * (p) and history (h) moments the collision operator reads (device x
 * profiles, copied; e unused by the operators).  No-op without collisions.
 * vv_step takes the state's moments instead. */
int vv_set_moments(vv_ctx* ctx, const double* n_p, const double* u_p, const double* e_p, const double* a_p,
                   const double* n_h, const double* u_h, const double* e_h, const double* a_h);

/* ---- Toolbox ------------------------------------------------------------ */
/* compute_density / compute_velocity_density / compute_energy_density /
 * compute_collision_factor (Toolbox.pyx:79-165).  Any output may be NULL. */
int vv_moments(vv_ctx* ctx, const double* F, double* n, double* u, double* e, double* a);
/* potential_to_hamiltonian: h1_i = phi_i - sum(phi)/nx   Toolbox.pyx:38-74 */
int vv_potential_to_hamiltonian(vv_ctx* ctx, const double* phi, double* h1);

/* ---- PETScPoissonSolver (CFD4) ------------------------------------------ */
/* formRHS: b = -(n - mean n)*charge             PETScPoissonSolver.pyx:58-74 */
int vv_poisson_rhs(vv_ctx* ctx, const double* n, double* b);
/* matrix_mult: y = (5,-32,54,-32,5) x / (12 hx^2)  PETScPoissonCFD4.pyx:146-160 */
int vv_poisson_matvec(vv_ctx* ctx, const double* x, double* y);
/* function_mult: y = A x + (n - mean n)*charge    PETScPoissonCFD4.pyx:163-183 */
int vv_poisson_function(vv_ctx* ctx, const double* x, const double* n, double* y);
/* the KSP solve of A phi = b(n) on the mean-free subspace
 * (run/run_base.py:658-704, run_nonlinear_matrixfree_split_mp.py:56-80);
 * exact spectral inverse, phi has zero mean. */
int vv_poisson_solve(vv_ctx* ctx, const double* n, double* phi);

/* ---- GMRES (PETSc KSPGMRES as configured at
 *      run_nonlinear_matrixfree_split_mp.py:47-53, run_base.py:189-191) ---- */
typedef struct vv_ksp_opts {
    double  rtol;            /* petsc_ksp_rtol  (runspec default 1e-4)        */
    double  atol;            /* petsc_ksp_atol  (1e-50)                       */
    double  dtol;            /* divergence tolerance (PETSc default 1e5)      */
    int32_t max_it;          /* petsc_ksp_max_iter (1000)                     */
    int32_t restart;         /* 0 -> the context's gmres_restart              */
} vv_ksp_opts;
typedef struct vv_ksp_result {
    int32_t its;             /* KSPGetIterationNumber                         */
    int32_t reason;          /* KSPConvergedReason (PETSc numbering)          */
    double  rnorm;           /* last residual estimate                        */
} vv_ksp_result;
/* Solve (P^-1 J) x = b with zero initial guess; x and b are device fields. */
int vv_gmres(vv_ctx* ctx, const double* b, double* x, const vv_ksp_opts* opts,
             vv_ksp_result* result);

/* ---- the time step (run_nonlinear_matrixfree_split_mp.py:111-174) ------- */
typedef struct vv_state {    /* caller-owned device buffers                   */
    double* f;               /* nx*nv current distribution function (fc)    */
    double* fh;              /* nx*nv previous time level (fh)               */
    double* phi;             /* nx internal potential, current (pc_int)      */
    double* phih;            /* nx internal potential, previous (ph_int)     */
    double* h1c;             /* nx h1 profile, current                       */
    double* h1h;             /* nx h1 profile, previous                      */
    double* h2c;             /* nx external h2 profile, current (or NULL)    */
    double* h2h;             /* nx external h2 profile, previous (or NULL)   */
    double* n;               /* nx density of f (self.N)                     */
    double* u;               /* nx velocity density                          */
    double* e;               /* nx energy density                            */
    double* a;               /* nx collision factor                          */
} vv_state;
typedef struct vv_snes_opts {
    double  atol;            /* petsc_snes_atol: stop when residual < atol   */
    int32_t max_iter;        /* petsc_snes_max_iter                           */
    int32_t reserved;
    double  abort_residual;  /* abort threshold (reference: 10.)             */
} vv_snes_opts;
#define VV_MAX_PICARD 64
typedef struct vv_step_report {
    int32_t picard_its;      /* Picard (outer) iterations                    */
    int32_t gmres_its_total; /* sum of GMRES iterations                      */
    int32_t reverted;        /* 1 if the last iterate was rejected           */
    int32_t stop_rule;       /* 1 residual rose, 2 below atol, 3 max_iter    */
    int32_t ksp_failures;    /* linear solves with a negative reason         */
    int32_t aborted;         /* 1 if residual > abort threshold              */
    int32_t gmres_its[VV_MAX_PICARD];
    int32_t ksp_reason[VV_MAX_PICARD];
    double  residual[VV_MAX_PICARD + 1]; /* residual before/after each pass  */
    int32_t guess_kept;      /* initial guess: 1 if the predicted f was kept  */
    double  guess_prev;      /* residual before the predictor                 */
    double  guess_residual;  /* residual of the predicted f                   */
} vv_step_report;
/* Initial set-up of a run: optionally normalise f so that sum(f)*hv/nx == 1
 * (run_base.py:623-628), then moments, Poisson and h1 (run_base.py:506). */
int vv_run_init(vv_ctx* ctx, vv_state* st, int normalise);
/* calculate_moments: moments of st->f, Poisson, h1c (run_base.py:640-655). */
int vv_calculate_moments(vv_ctx* ctx, vv_state* st);
/* calculate_residual: ||R(f)||_2 + ||Poisson residual||_2 (run_base.py:631-637). */
int vv_calculate_residual(vv_ctx* ctx, vv_state* st, double* residual);
/* One implicit time step: make_history, the initial guess (when the grid
 * names a predictor), update_previous, Picard loop with one ksponly GMRES
 * solve per pass, revert/stop/abort rules. */
int vv_step(vv_ctx* ctx, vv_state* st, const vv_snes_opts* snes,
            const vv_ksp_opts* ksp, vv_step_report* report);
/* The predictor alone: Y = the grid's initial_guess method applied to F over
 * initial_iter iterations of ht/initial_iter, with H0, the history profiles
 * h1h and h2h (NULL: zero) and the grid's bracket in the reference's
 * operation order (PETScArakawaSymplectic.pyx:62-92,
 * PETScArakawaRungeKutta.pyx:20-100, run_base.py:811-912).  Y may alias F.
 * VV_ERR_ARG if the grid names no predictor. */
int vv_predict(vv_ctx* ctx, const double* F, const double* h1h, const double* h2h, double* Y);
/* initial_guess (run_base.py:786-808) on a state whose history is set
 * (after make_history): the residual of st->f (with the solver's Have of the
 * last update_previous, zero before the first), the predictor, moments, the
 * residual of the prediction; the prediction is kept unless its residual is
 * larger, else st->f is restored and its moments recomputed (the reference
 * keeps the prediction's potential there).  Host scalars: the two residuals
 * and whether the prediction was kept. */
int vv_initial_guess(vv_ctx* ctx, vv_state* st, double* prev, double* guess, int32_t* kept);

/* ---- batched sweep: many independent runs in lockstep -------------------- */
/* The reference runs one instance per process; a parameter sweep is many
 * processes.  A batch advances `n` independent runs (each its own context
 * and state, grids of different sizes) by one time step.  Every kernel of
 * the step is launched once for the whole table (each block serves one
 * instance), and the Picard and GMRES loops run in lockstep: each instance
 * keeps its own convergence tests and iteration counts, and an instance that
 * has converged is masked out of the later passes while the others
 * continue.  The step is one CUDA graph (batch-level conditional loops)
 * unless VV_GRAPH=0 at context creation, which drives the same kernels from
 * the host.  All instances must share the precision, bracket scheme and the
 * tensor_kinetic preconditioner, use the factored order and have nx a
 * multiple of 64; otherwise vv_batch_create returns VV_ERR_UNSUPPORTED.
 * Results equal each instance's own vv_step to rounding (the batch uses the
 * radix-2 x-FFT and 64 x 32 stencil tiles for every instance).  Contexts and
 * states stay owned by the caller and must outlive the batch. */
typedef struct vv_batch vv_batch;
int vv_batch_create(int n, vv_ctx* const* ctxs, const vv_state* states, vv_batch** out);
int vv_batch_destroy(vv_batch* batch);
int vv_batch_set_stream(vv_batch* batch, void* cuda_stream);
/* reports and statuses: arrays of n (statuses may be NULL); returns the
 * first non-OK instance status, VV_OK if all instances stepped.  Equals
 * vv_batch_launch followed by vv_batch_collect. */
int vv_batch_step(vv_batch* batch, const vv_snes_opts* snes, const vv_ksp_opts* ksp,
                  vv_step_report* reports, int* statuses);
/* The step in two halves, so that a caller can run several batches at once
 * on their own streams (a batch of the slowest instances beside one of the
 * rest: their lockstep loops then overlap instead of the slow instances
 * running alone at the end of every pass).  vv_batch_launch enqueues the
 * step and the read-back of the instance states on the batch's stream and
 * returns without waiting; vv_batch_collect waits for that stream and fills
 * the reports (the same arguments as vv_batch_step; snes and ksp as given
 * to the launch).  A launch must be collected before the next launch. */
int vv_batch_launch(vv_batch* batch, const vv_snes_opts* snes, const vv_ksp_opts* ksp);
int vv_batch_collect(vv_batch* batch, const vv_snes_opts* snes, const vv_ksp_opts* ksp,
                     vv_step_report* reports, int* statuses);
/* Number of kernels the batch has launched (graph nodes executed included). */
int vv_batch_launch_count(vv_batch* batch, int64_t* launches, int reset);
/* Device time of one whole-table launch of a batch kernel with every instance
 * active: `reps` launches are captured in a CUDA graph and timed with CUDA
 * events.  which: 0 Gram-Schmidt multi-dot (w and V_0..V_it read), 1
 * preconditioner (its three kernels), 2 Jacobian-vector-product stencil,
 * 3 Gram-Schmidt multi-axpy (w updated), 4 the preconditioner's tridiagonal
 * stage alone (in place on the spectra the last application left), 5 the
 * GMRES operator P^-1 J as the step applies it (the stencil fused into the
 * preconditioner's x-FFT when the batch runs fused).  it: the Arnoldi index
 * set in every instance first (it + 1 <= each context's restart).  Between
 * steps only: the GMRES scratch of every instance is overwritten. */
int vv_batch_time_kernel(vv_batch* batch, int which, int it, int reps, double* avg_ms);

/* ---- discrete adjoint of the converged step (no counterpart in the
 *      reference; built from its discrete operators) ---------------------
 * For a converged step f -> F (F = f^{n+1}, f = f^n, with the external
 * profiles h2p/h2h or NULL) and the gradient gF of a loss with respect to F,
 * writes the gradient with respect to f: gf = -gF + (2/ht) lambda with
 * A^T lambda = gF, A the coupled Jacobian of the step's residual (the
 * Jacobian-vector product of PETScNLVlasovMP.pyx:33-40 plus the f-phi
 * coupling through the moments and the Poisson solve,
 * solvers/full/PETScNLArakawaJ4.pyx:26-110).  The transpose system is solved
 * by GMRES preconditioned with the transposed kinetic preconditioner, to the
 * tolerances in opts; result reports its iterations.  FP64 contexts only
 * (VV_ERR_UNSUPPORTED for mixed).  The first call allocates the adjoint's
 * buffers (24 fields). */
int vv_step_adjoint(vv_ctx* ctx, const double* F, const double* f, const double* h2p,
                    const double* h2h, const double* gF, double* gf, const vv_ksp_opts* opts,
                    vv_ksp_result* result);
/* Gradient of the field energy 1/2 charge sum_i (phi_{i+1} - phi_i)^2 / hx
 * (potential.pyx:48-59) with respect to f. */
int vv_field_energy_grad(vv_ctx* ctx, const double* f, double* grad);

/* ---- invariants (vlasov/core/distribution_function.pyx:130-306,
 *      hamiltonian.pyx:67-124, potential.pyx:48-59) ---------------------- */
typedef struct vv_invariant_set {
    double mass, L1, L2, L3, L4, L5, L6, L8, Lmin, Lmax, entropy;
    double E_kin, E_pot, energy, momentum, field_energy;
} vv_invariant_set;
/* phi: internal potential (nx); h2: external profile or NULL.  Sums are
 * compensated FP64. */
int vv_invariants(vv_ctx* ctx, const double* f, const double* phi, const double* h2,
                  vv_invariant_set* out);

/* ---- timing of the dominant kernel (measurement support) --------------- */
/* When enabled, the library records CUDA events around every launch of the
 * Jacobian-vector-product stencil kernel on its stream; vv_timing_read
 * returns the number of launches and their summed device time (ms). */
int vv_timing_enable(vv_ctx* ctx, int enable);
int vv_timing_read(vv_ctx* ctx, int64_t* launches, double* total_ms, int reset);
/* Number of kernels the library has launched since the last reset
 * (kernels executed inside the time-step graph included). */
int vv_launch_count(vv_ctx* ctx, int64_t* launches, int reset);
/* Kernel variants the context runs, as five ints: FFT kind of the
 * preconditioner's x transforms (0 shared-memory radix-2, 1 four-step
 * register/shuffle, 2 direct DFT), FFT rows per CTA, tridiagonal kind (0 CTA
 * per mode, 1 warp per mode), narrow bracket tiles (1: 32 x 16 instead of
 * 64 x 32) and the marching Jacobian stencil's strip width (0: tiles).
 * vv_create picks them by timing the candidates on the device at hand, or
 * takes them from the environment variable VV_SHAPE="fft,R,tri,narrow[,march]"
 * (VV_ERR_ARG when they do not fit the grid).  No reference counterpart: the
 * reference has one implementation per operation. */
int vv_kernel_shape(vv_ctx* ctx, int32_t* shape);
/* Device time of one kernel on the context's own buffers: `reps` launches
 * are captured back to back in a CUDA graph and timed with CUDA events on the
 * context's stream.  which: 0 Jacobian-vector product (input: GMRES basis
 * vector 0, output: work field), 1 residual, 2 preconditioner apply (its
 * three kernels).  *avg_ms = time per launch (per apply for which == 2). */
int vv_time_kernel(vv_ctx* ctx, int which, int reps, double* avg_ms);

/* ---- invariants without a context or an allocation ----------------------
 * No counterpart in the reference: there the invariants are computed on the
 * host (distribution_function.pyx:130-306, hamiltonian.pyx:67-124,
 * potential.pyx:48-59).  Same results as vv_invariants (same sums, same
 * compensated FP64 order) for fields already on the device, but without a
 * vv_ctx: vv_create allocates the whole solver (GMRES basis, spectra,
 * preconditioner factors, scratch) and tunes it, which a diagnostics caller
 * cannot always afford -- a hook between the steps of a running solve, where
 * cudaMalloc/cudaFree would synchronise the device; a process whose device
 * memory a caching allocator already holds; analysis code with fields but no
 * solver.  This call performs no device allocation: its scratch is one fixed
 * array in the library's device memory (about 198 KiB per device).
 *   grid:   nx, nv, L, vmin, vmax, charge and mass are read (ht and the
 *           solver fields are not); f: nx*nv doubles, phi: nx doubles,
 *           h2: nx doubles or NULL; all device pointers.
 *   stream: the CUDA stream of the kernels (NULL: the legacy default
 *           stream); the call returns after synchronising it.
 * Limits and rules:
 *   nx > VV_NOALLOC_MAX_NX returns VV_ERR_UNSUPPORTED before any device
 *   work (the array holds the x profile of phi).
 *   The array is shared by all callers on a device: calls whose kernels can
 *   overlap in time (two host threads, or two unordered streams) race on it
 *   and must be serialised by the caller.
 *   The first call on each device (and the first after the device's CUDA
 *   context was destroyed and re-created, e.g. by cudaDeviceReset) does a
 *   one-time set-up: it looks up the array's device address in the current
 *   context, which may load the library's device code.  Make that first
 *   call before any stream capture begins on that device.
 *   Nothing in the array has to start at zero. */
#define VV_NOALLOC_MAX_NX 16384
int vv_invariants_noalloc(const vv_grid* grid, const double* f, const double* phi,
                          const double* h2, void* cuda_stream, vv_invariant_set* out);

#ifdef __cplusplus
}
#endif
#endif /* VIVLASOV1D_B200_VV_H */
