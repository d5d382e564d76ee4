/* cmsgpu.h -- C-ABI of the B200 (sm_100a) implicit-flow solver library libcmsgpu.so.
 *
 * The library replaces the linear-solver boundary of CMS-Flow's implicit
 * SIMPLEC step.  All arrays follow the reference's in-memory layout:
 *   - cells 1..ncells are active, ncells+1..ncellsD are dummy (ghost) cells;
 *   - cell2cell(k,i), acoef(k,i) are Fortran column-major [nmaxfaces][ncellsD]
 *     arrays: element (k,i) sits at offset (i-1)*nmaxfaces + (k-1);
 *   - neighbour indices are 1-based; ncface(i) faces are used per cell.
 * Every entry point returns a status: CMS_OK (0), CMS_NOT_CONVERGED (1),
 * CMS_NONFINITE (2), CMS_DEVICE_ERROR (3), CMS_BAD_ARGUMENT (4),
 * CMS_UNSUPPORTED (5).  The library never aborts the caller; the reference's
 * `iconv` global (source/solvers/solv_def.f90:8) is set by the caller from
 * the status (iconv = 0 for CMS_NONFINITE, 1 otherwise).
 *
 * Two calling styles are offered:
 *   - a handle API (cms_solver_*), reentrant per handle, one CUDA stream per
 *     handle;
 *   - the reference-shaped global API (cms_gpu_*) that mirrors the module
 *     state of solv_def: one implicit handle created by cms_gpu_init.
 */
#ifndef CMSGPU_H
#define CMSGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CMS_OK = 0,
  CMS_NOT_CONVERGED = 1,
  CMS_NONFINITE = 2,
  CMS_DEVICE_ERROR = 3,
  CMS_BAD_ARGUMENT = 4,
  CMS_UNSUPPORTED = 5
};

/* Unknown ordering used by the ILU(0) factor and its sweeps. */
enum {
  CMS_ORDER_MULTICOLOR = 0, /* greedy multicolour ordering: 2 colours on a Cartesian grid */
  CMS_ORDER_NATURAL = 1     /* the reference's natural order, level-scheduled sweeps */
};

/* Arithmetic of the Krylov solve. */
enum {
  CMS_PREC_FP64 = 0,        /* plain FP64 drop-in (ikind=8 build) */
  CMS_PREC_FP32_REFINE = 1, /* FP32 matrix/factor/SpMV/sweeps inside FP64 iterative refinement */
  CMS_PREC_FP32 = 2         /* FP32 throughout (ikind=4 build); dots accumulate in FP64 */
};

typedef struct cms_solver_opts {
  int ordering;      /* CMS_ORDER_*                                                    */
  int precision;     /* CMS_PREC_* (used by the *_d entry points; *_f is FP32)         */
  int norm;          /* BiCGStab stopping norm: 1 = L1 of the recursive residual
                        (pbicgstab.f90:95), 2 = L2                                     */
  double tol;        /* relative tolerance; the reference hard-codes 1e-3
                        (pbicgstab.f90:95, pgmres.f90:19)                              */
  int max_iters;     /* > 0 overrides the nswp argument                                */
  double inner_tol;  /* refinement: relative L2 reduction asked of each FP32 solve;
                        0 (default): 0.5 tol / (the outer relative residual before
                        the solve), kept within [1e-6, 1e-3]                         */
  int inner_max;     /* refinement: iteration cap of each FP32 solve; 0 (default):
                        the solve's remaining iteration budget (nswp or max_iters
                        minus the inner iterations so far); a cap > 0 is also
                        bounded by that budget                                       */
  int max_refine;    /* refinement: cap on FP64 residual/correction steps              */
  int verify;        /* 1: compute the FP64 true residual after the solve (one extra
                        pass); 0: skip it (true_relres = -1)                           */
  int multi_kernel;  /* 0: each BiCGStab solve is one persistent cooperative launch
                        (grid barriers between colour phases, dot products reduced
                        in the kernel); 1: one launch per phase with host polling.
                        Both run the same arithmetic.                                  */
  int inner_relax;   /* FP32 inner BiCGStab of refinement on a multicolour ordering:
                        2 (default) solves the reduced system on the rows of colours
                        >= 1 (Schur complement of the independent colour-0 block,
                        right-scaled by its diagonal), which is red/black ILU(0)
                        preconditioning in reduced form: no triangular sweeps, half
                        the unknowns; 1 factors the FP32 system without the
                        couplings among rows of colours >= 2, so its sweeps take two
                        phases like a red/black grid; 0: exact multicolour ILU(0).
                        The FP64 residual makes each converge to the same answer.   */
  double relaxsor;   /* SOR constant of nsolv 2 and 5 (SUCCESSIVE_OVER_RELAXATION_CONSTANT
                        card, default 1.8: flow.F90:131)                                */
  int nswp0_vel;     /* nswp0(2), the velocity iteration count the hybrid solver
                        (nsolv 5) triples for n = 4, 5 (solvers.f90:265); default 5  */
  int reduced_layout; /* block and row layout of the reduced inner solve: 0 auto
                        (= 5), 1 256 threads x 2 rows, 2 512 x 2, 3 512 x 4, 4 1024 x 2
                        (three phases, two grid barriers per iteration); 5 1024 x 2,
                        6 512 x 2, 7 256 x 2 in the single-reduction form (one
                        barrier per iteration; needs a structurally symmetric
                        reduced pattern, else the three-phase layout of the same
                        block size runs).  The tiles follow the layout's resident
                        block count; ensembles take the form of their members'
                        option at 256 threads x 2 rows                           */
} cms_solver_opts;

typedef struct cms_solve_info {
  int status;        /* CMS_*                                                          */
  int iters;         /* BiCGStab iterations or GMRES restarts (refinement: all inner)  */
  int inner;         /* GMRES Arnoldi steps (BiCGStab: iterations)                     */
  int refine_steps;  /* FP64 refinement steps (0 outside CMS_PREC_FP32_REFINE)         */
  double relres;     /* the ratio the stopping test last saw                           */
  double true_relres;/* ||b - A x||_2 / ||b - A x0||_2 in FP64 after the solve         */
  double rmom;       /* RMS of the normalised residual before the solve (solvers.f90:240) */
  int ncolors;       /* number of groups the sweeps run (colours or levels)            */
} cms_solve_info;

typedef struct cms_solver cms_solver;

/* Fills opts with the reference defaults: multicolour, FP64, L1, tol 1e-3. */
void cms_solver_default_opts(cms_solver_opts* opts);

/* solv_init (source/solvers/solvers.f90:93-202) + indexm (sparse.f90:2-70):
 * copies the connectivity, builds the unknown ordering, the ELL sparsity
 * pattern and the sweep schedule, and allocates all device buffers.
 * iwet may be NULL (all wet). */
int cms_solver_create(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                      const int* iwet, const cms_solver_opts* opts, cms_solver** out);

/* Replaces iwet (flow_wetdry output); the pattern is unchanged. */
int cms_solver_update_wet(cms_solver* s, const int* iwet);

int cms_solver_set_opts(cms_solver* s, const cms_solver_opts* opts);

/* solve(acoef,ss,sp,res,phi,n) (source/solvers/solvers.f90:205-304) with HOST
 * arrays: ap=(sum acoef - sp)/relax; ss += (1-relax)*phi*ap; res = normalised
 * residual; rmom = RMS(res); then BiCGStab (nsolv=3, pbicgstab.f90) or
 * GMRES(3) (nsolv=4, pgmres.f90) preconditioned by ILU(0) of the same matrix.
 * ss, res and phi are updated in place; nswp caps iterations (restarts). */
int cms_solver_solve_d(cms_solver* s, const double* acoef, double* ss, const double* sp, double* res, double* phi,
                       double relax, int nswp, int nsolv, cms_solve_info* info);
int cms_solver_solve_f(cms_solver* s, const float* acoef, float* ss, const float* sp, float* res, float* phi,
                       float relax, int nswp, int nsolv, cms_solve_info* info);

/* Same contract with DEVICE pointers (arrays already resident in HBM, same
 * layout).  The call is ordered on the handle's stream and returns after the
 * solve has finished. */
int cms_solver_solve_dev_d(cms_solver* s, const double* acoef, double* ss, const double* sp, double* res, double* phi,
                           double relax, int nswp, int nsolv, cms_solve_info* info);
int cms_solver_solve_dev_f(cms_solver* s, const float* acoef, float* ss, const float* sp, float* res, float* phi,
                           float relax, int nswp, int nsolv, cms_solve_info* info);

/* solve() with the variable index n (1 pressure correction, 2-3 velocity, 4
 * sediment, 5 salinity or heat; 0 none) for every MATRIX_SOLVER option
 * (solvers.f90:242-289): nsolv 0 (ADI) the prologue only, as solve() has no
 * branch for it; 1 Gauss-Seidel; 2 symmetric Gauss-Seidel, or
 * SSOR for n = 1 once rmom < 1e-3; 3 BiCGStab; 4 GMRES; 5 BiCGStab for n = 1
 * while rmom > 1e-4, else Gauss-Seidel with 4*nswp passes (n <= 3) or
 * 3*opts.nswp0_vel passes (n = 4, 5), SOR for n = 1; 6 SIP; 7 ICCG for n = 1,
 * else SIP; 8 ICCG for n = 1, else ICCGSTAB.  The Gauss-Seidel passes and the
 * incomplete Cholesky factor follow the handle's ordering (natural: the
 * reference's serial loops; multicolour: their multicolour form).  SIP, ICCG
 * and ICCGSTAB need exactly four faces per cell (a Cartesian grid), and SIP
 * the natural ordering of a grid numbered row by row from the south-west
 * (CMS_UNSUPPORTED otherwise).  Options other than 3 and 4 run in the type of
 * the call (CMS_PREC_FP32_REFINE is not applied to them).  The entry points
 * without n behave as n = 0. */
int cms_solver_solve_n_d(cms_solver* s, int n, const double* acoef, double* ss, const double* sp, double* res,
                         double* phi, double relax, int nswp, int nsolv, cms_solve_info* info);
int cms_solver_solve_n_f(cms_solver* s, int n, const float* acoef, float* ss, const float* sp, float* res, float* phi,
                         float relax, int nswp, int nsolv, cms_solve_info* info);
int cms_solver_solve_dev_n_d(cms_solver* s, int n, const double* acoef, double* ss, const double* sp, double* res,
                             double* phi, double relax, int nswp, int nsolv, cms_solve_info* info);
int cms_solver_solve_dev_n_f(cms_solver* s, int n, const float* acoef, float* ss, const float* sp, float* res,
                             float* phi, float relax, int nswp, int nsolv, cms_solve_info* info);

/* Number of groups the sweeps run and device bytes held by the handle. */
int cms_solver_ncolors(const cms_solver* s);
size_t cms_solver_device_bytes(const cms_solver* s);
/* Device-order permutation: perm[r] = natural 0-based cell of device row r. */
int cms_solver_get_perm(const cms_solver* s, int* perm);
/* Kernel launches issued by the handle since creation (counted on the host). */
long long cms_solver_launches(const cms_solver* s);
/* Refinements that finished on the exact multicolour ILU(0) inner solve
 * because a reduced or two-phase inner correction made the FP64 residual
 * more than 4 times larger or overflowed (the correction is undone first). */
long long cms_solver_refine_fallbacks(const cms_solver* s);
/* Kernel-class timing with CUDA events on the handle's stream.  Classes:
 * 0 prologue, 1 ILU(0) factor, 2 forward sweep, 3 backward sweep, 4 SpMV,
 * 5 vector/reduction kernels, 6 FP64 residual, 7 scalar kernels, 8 flow-step
 * assembly/correction kernels (a flow handle's solver), 9 persistent
 * BiCGStab (every iteration in one launch), 10 reduced-system build (the
 * inner solve's Schur complement), 11 persistent reduced BiCGStab.
 * profile_read fills ms[CMS_PROF_CLASSES], bytes[..] (algorithmic bytes:
 * every array a kernel touches counted once) and count[..] (launches);
 * reset=1 clears. */
#define CMS_PROF_CLASSES 12
int cms_solver_profile(cms_solver* s, int enable);
int cms_solver_profile_read(cms_solver* s, int reset, double* ms, double* bytes, long long* count);
/* Adjoint of solve() (no counterpart in the reference), FP64, device
 * pointers in the solve() layout (natural order, acoef [ncellsD][nmaxfaces]):
 * given the inputs of a forward solve (acoef, ss and sp as passed in, phi0 =
 * phi before the solve), its solution x (phi after the solve, ncellsD values,
 * dummies unchanged) and g = dL/dx, solves A^T lam = g (ILU(0)-BiCGStab to
 * ||r||2/||g||2 < tol, at most maxit iterations) and writes lam and the
 * gradients dL/dacoef, dL/dss, dL/dsp (rows of active cells; any output may be
 * NULL). */
int cms_solver_adjoint_dev_d(cms_solver* s, const double* acoef, const double* ss, const double* sp,
                             const double* phi0, const double* x, double relax, const double* g, double tol,
                             int maxit, double* lam, double* grad_acoef, double* grad_ss, double* grad_sp,
                             cms_solve_info* info);
/* Bottom-friction sink of the momentum equations and its adjoint (the
 * adjoint has no counterpart in the reference), FP64 device pointers over n
 * cells, on stream (a cudaStream_t, NULL: the legacy default stream; the
 * calls do not wait).  Forward: sp = spuv0 - Cd(n) |u| A with the Manning
 * closure Cd = g n^2 / max(min(10, h), 0.1 n)^0.3333 (fric_eval,
 * friction.F90:647-662, fric_lib.f90:965-966; the sink of coeffsourcesink_uv,
 * flow_imp.F90:409-574), coefman = n, uv = |u|, area = A.  Adjoint: given
 * grad_sp = dL/dsp (from cms_solver_adjoint_dev_d), writes
 * grad_coefman = dL/dn = -grad_sp |u| A dCd/dn with h, |u| and A held fixed. */
int cms_fric_sink_dev_d(int n, double grav, const double* coefman, const double* h, const double* uv,
                        const double* area, const double* spuv0, double* sp, void* stream);
int cms_fric_sink_adjoint_dev_d(int n, double grav, const double* coefman, const double* h, const double* uv,
                                const double* area, const double* grad_sp, double* grad_coefman, void* stream);
/* Momentum face coefficients and their adjoint (the adjoint has no
 * counterpart in the reference), FP64 device pointers in the solve() face
 * layout ([ncellsD][nmaxfaces], natural order; faces k < ncface(i) of the
 * ncells active cells), on stream (NULL: the legacy default stream; no
 * wait).  Forward: acoef = scheme(visk hk ds, flux) with the
 * ADVECTION_SCHEME coefficient function ndsch (0 none, 1 upwind, 2 hybrid,
 * 3 power law, 4 exponential; comp_lib.f90:40-109, as coeffsourcesink_uv
 * calls it, flow_imp.F90:120-126); other entries untouched.  Adjoint: given
 * grad_acoef = dL/dacoef (from cms_solver_adjoint_dev_d), writes dL/dvisk,
 * dL/dhk and dL/dflux for every face slot of the active cells (0 beyond
 * ncface); any of the three outputs may be NULL. */
int cms_momentum_coef_dev_d(int ncells, int nmaxfaces, int ndsch, const int* ncface, const double* visk,
                            const double* hk, const double* ds, const double* flux, double* acoef, void* stream);
int cms_momentum_coef_adjoint_dev_d(int ncells, int nmaxfaces, int ndsch, const int* ncface, const double* visk,
                                    const double* hk, const double* ds, const double* flux, const double* grad_acoef,
                                    double* grad_visk, double* grad_hk, double* grad_flux, void* stream);
/* Pressure-correction coefficients from the momentum coefficients and their
 * adjoint (the adjoint has no counterpart in the reference), FP64 device
 * pointers: cell2cell (1-based) and the face fields in the solve() layout
 * ([ncellsD][nmaxfaces]), iwet with ncellsD entries, acoef_u / sp_u the
 * momentum system (solve() layout), area, hk, ds, dn, fintp the cell area and
 * the face depth, length, centre distance and interpolation weight (fintp on
 * the two sides of a face adding to 1); on stream (NULL: the legacy default
 * stream; no wait).  Forward (coefsourcesink_pp, flow_imp.F90:577-794,
 * without the skewness correction): apu = iwet relax / max(sum acoef_u -
 * sp_u, 1e-6), ap = apu A, sumu = apu sum acoef_u, and on each face k <
 * ncface(i) to a wet cell a_pp = hk^2 ds ap_f / (1 - sumu_f) / dn, the face
 * values interpolated with fintp (the cell's own at a dummy neighbour); 0
 * across a dry side.  Adjoint: given grad_acoef_pp, writes dL/dacoef_u (the
 * same value on every face of a row), dL/dsp_u and dL/dhk; outputs may be
 * NULL. */
int cms_pp_coef_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet,
                      double relax, const double* acoef_u, const double* sp_u, const double* area, const double* hk,
                      const double* ds, const double* dn, const double* fintp, double* acoef_pp, void* stream);
int cms_pp_coef_adjoint_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet,
                              double relax, const double* acoef_u, const double* sp_u, const double* area,
                              const double* hk, const double* ds, const double* dn, const double* fintp,
                              const double* grad_acoef_pp, double* grad_acoef_u, double* grad_sp_u, double* grad_hk,
                              void* stream);
/* Right-hand side of the pressure-correction system and its adjoint (the
 * adjoint has no counterpart in the reference), same conventions as
 * cms_pp_coef_dev_d, plus idirface (face directions 1 N, 2 E, 3 S, 4 W, the
 * solve() face layout) and the cell fields u, v, h, dpx, dpy, p (p with
 * ncellsD entries: dummy values enter the boundary fluxes), sspp0, sppp0.
 * Forward (coefsourcesink_pp with the Rhie-Chow fluxes of
 * flow_imp_flux_noskew, flow_imp_flux.f90:361-409, wet cells, no skewness
 * correction): Hu = u + ap dpx h, Hv = v + ap dpy h, flux(k,i) =
 * hk ds (nx Hu_f + ny Hv_f - ap_f hk (p_c - p_i) / dn) with the face values
 * interpolated as in cms_pp_coef_dev_d, ss_pp = sspp0 - sum_k flux + p sppp0.
 * Adjoint: given grad_ss_pp, writes dL/dacoef_u, dL/dsp_u (through ap),
 * dL/dhk and dL/du, dL/dv (active cells); outputs may be NULL. */
int cms_pp_rhs_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface, const int* idirface,
                     const int* iwet, double relax, const double* acoef_u, const double* sp_u, const double* area,
                     const double* u, const double* v, const double* h, const double* dpx, const double* dpy,
                     const double* p, const double* hk, const double* ds, const double* dn, const double* fintp,
                     const double* sspp0, const double* sppp0, double* ss_pp, void* stream);
int cms_pp_rhs_adjoint_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface, const int* idirface,
                             const int* iwet, double relax, const double* acoef_u, const double* sp_u,
                             const double* area, const double* u, const double* v, const double* h, const double* dpx,
                             const double* dpy, const double* p, const double* hk, const double* ds, const double* dn,
                             const double* fintp, const double* grad_ss_pp, double* grad_acoef_u, double* grad_sp_u,
                             double* grad_hk, double* grad_u, double* grad_v, void* stream);
/* Blocks (tiles) of the handle's persistent BiCGStab launch: 0 restores the
 * default (the device's resident capacity, at most one block per 256 rows);
 * returns the count in use, or a negative CMS_* code. */
int cms_solver_set_tiles(cms_solver* s, int tiles);
/* The stream the handle runs on (a cudaStream_t). */
void* cms_solver_stream(cms_solver* s);

void cms_solver_destroy(cms_solver* s);

/* Host-only (no device calls): the unknown ordering a handle would use.
 * perm[r] = natural 0-based cell of device row r (ncells entries);
 * gstart[0..G] = device-row range of each sweep group (ncells+1 entries
 * available); kl_ku[0..1] = max lower / upper couplings per row.  Returns the
 * number of groups G (> 0) or -CMS_BAD_ARGUMENT. */
int cms_order_build(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface, int ordering,
                    int* perm, int* gstart, int* kl_ku);

/* ---- implicit flow step (flow_imp, source/flow/flow_imp.F90:29-312) ------
 * One SIMPLEC time step on the device: static sources, per outer iteration
 * momentum coefficients (exponential scheme) + skewness corrections + BCs,
 * u and v solves, pressure-correction coefficients + Rhie-Chow fluxes,
 * pp solve, velocity/flux/water-level correction, gradients, face values,
 * Manning friction, eddy viscosity and check_conv; then velface_eta and
 * the time-level update.  Cartesian and telescoping grids, ntsch = 1,
 * water-level (TH/H) strings on dummy faces, walls elsewhere.  Wetting and
 * drying is not handled: a step that would dry a cell returns
 * CMS_UNSUPPORTED.  Water levels of the string are inputs of each step
 * (the host keeps bnd_eval). */
typedef struct cms_flow cms_flow;

typedef struct cms_flow_opts {
  int nsolv;         /* MATRIX_SOLVER 0-8 as in solve() (cms_solver_solve_n_d);
                        4 GMRES by default (solvers.f90:8)                          */
  int ordering;      /* CMS_ORDER_*                                                */
  int precision;     /* CMS_PREC_FP64 or CMS_PREC_FP32_REFINE (the solves)         */
  int norm;          /* BiCGStab stopping norm (1 = L1 as the reference)           */
  double tol;        /* inner relative tolerance (reference 1e-3)                  */
  int nswp_pp;       /* iteration caps (flow.F90:779-792): pp 20/15, u/v 5         */
  int nswp_uv;
  int maxit;         /* outer iterations; 0: 20 + ncells/10000 (flow.F90:784,792)  */
  int skewcor;       /* skewness corrections on telescoping grids (flow.F90:108)   */
  double inner_tol;  /* refinement: as cms_solver_opts.inner_tol (0: adaptive)     */
  int inner_max;     /* refinement: as cms_solver_opts.inner_max (0: the budget)   */
  int multi_kernel;  /* solver kernels, as cms_solver_opts.multi_kernel            */
  double hdry;       /* drying depth (flow.F90:51, hmin = hdry); 0: 0.05 m          */
  int ponding;       /* keep isolated water bodies (flow.F90:54; default 0)         */
  int narrowchannels; /* keep one-cell-wide channels (flow.F90:55; default 0)       */
  double relaxsor;   /* SOR constant of nsolv 2 and 5 (flow.F90:131; default 1.8)   */
  int ndsch;         /* ADVECTION_SCHEME (flow.F90:533-545, definitions.F90:166-171):
                        0 NONE, 1 UPWIND, 2 HYBRID, 3 POWERLAW, 4 EXPONENTIAL
                        (default, flow.F90:111); the higher-order deferred-
                        correction schemes 5-18 give CMS_UNSUPPORTED             */
  int reduced_layout; /* cms_solver_opts.reduced_layout of the flow's solves (0 auto) */
} cms_flow_opts;

typedef struct cms_flow_info {
  int status;        /* CMS_*                                                      */
  int niter;         /* outer iterations run                                       */
  int iconv;         /* check_conv: 0 divergent, 1 continue (maxit reached), 2 converged */
  double rmom_p, rmom_u, rmom_v;  /* last normalised residuals (rmom(1:3))        */
  long long krylov_iters;         /* Krylov iterations of all solves of the step  */
  int nwet;          /* wet active cells during the step (number_wet_cells)        */
  int nchanged;      /* active cells whose wet state changed at the step's start   */
} cms_flow_info;

enum {
  CMS_FLOW_P = 0, CMS_FLOW_H = 1, CMS_FLOW_U = 2, CMS_FLOW_V = 3, CMS_FLOW_ETA = 4, CMS_FLOW_VIS = 5,
  CMS_FLOW_CFRICT = 6, CMS_FLOW_DPX = 7, CMS_FLOW_DPY = 8, CMS_FLOW_IWET = 9,
  CMS_FLOW_FLUX = 100, CMS_FLOW_VISK = 101, CMS_FLOW_HK = 102, CMS_FLOW_ACOEF = 103, CMS_FLOW_FINTP = 104,
  CMS_FLOW_ZBK = 105
};

void cms_flow_default_opts(cms_flow_opts* opts);
/* Grid in the reference layout: cell2cell/idirface [ncellsD][nmaxfaces]
 * (1-based ids, direction 1..4 = N,E,S,W), cell centres/sizes x,y,dx,dy and
 * bed elevation zb (ncellsD, zb = -depth), Manning n per active cell, and one
 * water-level string given as 1-based (cell, face) pairs whose faces lead to
 * dummy cells.  All other dummy faces are walls (geo_init_cart,
 * geospatial.F90:1400-1833; bnd_init). */
int cms_flow_create(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                    const int* idirface, const double* x, const double* y, const double* dx, const double* dy,
                    const double* zb, const double* coefman, int nth, const int* th_cells, const int* th_faces,
                    const cms_flow_opts* opts, cms_flow** out);
/* Cold start at rest from the water level eta0 (ncellsD values, natural
 * order), as prestart does (prestart.f90:302-325). */
int cms_flow_init(cms_flow* f, const double* eta0);
/* Hot start from the water pressure p (= g * water level) and velocities u, v
 * of all ncellsD cells, natural order, as a hot-start file holds them
 * (hot_read): hot_init (hot_start.F90:1125-1215: cells with h < hmin + 1e-5
 * dry and at rest, water-level string dummies copy their cell), then the rest
 * of prestart (prestart.f90:298-325): flow_wetdry(0) against hot_init's wet
 * set (dry-to-wet initialisation of the cells it wets), the wet-cell gradient
 * operator of the resulting wet set, bed slope, face values, face fluxes from
 * the velocities (flow_convflux, flow.F90:1879-1909) unless flux gives the
 * file's face fluxes ([ncellsD][nmaxfaces] like CMS_FLOW_FLUX; NULL: none),
 * friction, eddy viscosity.  Replaces cms_flow_init; stepping continues with
 * cms_flow_step. */
int cms_flow_init_hot(cms_flow* f, const double* p, const double* u, const double* v, const double* flux);
/* One time step of length dt; wsebnd holds the string's water levels at the
 * new time level (one per string entry), or NULL when the string's tide was
 * set with cms_flow_set_tide (then evaluated on the device).  The step starts
 * with wetting and drying (flow_wetdry(0), flow.F90:1231-1539, and
 * der_update, derivatives.f90:204-296) when any cell's depth class changed
 * since the last one. */
int cms_flow_step(cms_flow* f, double dt, const double* wsebnd, cms_flow_info* info);
/* The tidal/harmonic water-level string of bnd_eval (boundaries.F90:4098-4124)
 * evaluated on the device at the start of every step given wsebnd = NULL:
 * wse_j(t) = sum_k f_k amp_k cos(speed_k (t/3600 + dtj) + vu_k - phase_k +
 * psi_jk) + offset + wsevar_j, with ntc constituents (amp in m, speed in
 * radians per hour, phase, vu and psi in radians), nodal factors f (NULL: 1),
 * equilibrium arguments vu (NULL: 0; both NULL and dtj = 0 is the reference's
 * harmonic, non-tidal form), per-entry phase lags psi [nth][ntc] and level
 * variations wsevar [nth] (NULL: 0); t is the time after the step.  The
 * reference's ramp is 1 here (a ramped start passes its levels per step). */
int cms_flow_set_tide(cms_flow* f, int ntc, const double* amp, const double* speed, const double* phase,
                      const double* nodal, const double* vu, const double* psi, const double* wsevar, double dtj,
                      double offset);
/* Simulation time of the model's state in seconds (0 after cms_flow_init and
 * cms_flow_init_hot; the tide evaluation reads it; each step adds dt). */
int cms_flow_set_time(cms_flow* f, double t_seconds);
/* Wet set of flow_wetdry(0) (flow.F90:1231-1539; flow_pond 1807-1876) for the
 * water level eta (ncellsD values): depth rule, every dummy off the water-level
 * string closed (dry), narrow-channel removal (Cartesian rules; the one-cell
 * rule when narrowchannels is set), and flow_pond seeded by the string unless
 * ponding is set.  Host arrays only (no device work); hdry <= 0 means 0.05 m.
 * Grid arrays as in cms_flow_create; iwet receives ncellsD flags. */
int cms_wetdry_rules(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                     const int* idirface, const double* zb, const double* eta, int nth, const int* th_cells,
                     const int* th_faces, double hdry, int ponding, int narrowchannels, int* iwet);
/* Host copy (natural order) of a state array CMS_FLOW_*: ncellsD values for
 * cell arrays, [ncellsD][nmaxfaces] for face arrays. */
int cms_flow_get(cms_flow* f, int which, double* out);
int cms_flow_last_info(const cms_flow* f, cms_flow_info* info);
/* Solve records (u, v, pp) of the last outer iteration of the last step. */
int cms_flow_last_solves(const cms_flow* f, cms_solve_info* info3);
cms_solver* cms_flow_solver(cms_flow* f);
long long cms_flow_launches(const cms_flow* f);
size_t cms_flow_device_bytes(const cms_flow* f);
int cms_flow_njoint(const cms_flow* f);
/* Wet/dry updates run so far (steps that started with a changed wet set
 * candidate) and their host time in ms: ms3[0] depth-class read-back, ms3[1]
 * rules, ms3[2] application (flags, lists, dry-to-wet initialisation,
 * gradient-operator rows).  No counterpart in the reference. */
int cms_flow_wetdry_stats(const cms_flow* f, long long* updates, double* ms3);
/* Replay of the step's stage kernel sequences (pressure-correction assembly,
 * corrections and gradients) as CUDA graphs, captured per gradient-copy
 * state and again after every wet-set change: on = 1 turns it on (ensembles
 * do so for their members), 0 off (default: direct launches).  Graphs are
 * not used while the solver's profiling is on.  graph_stats gives the
 * replays and captures so far.  No counterpart in the reference. */
int cms_flow_set_graphs(cms_flow* f, int on);
int cms_flow_graph_stats(const cms_flow* f, long long* replays, long long* captures);
void cms_flow_destroy(cms_flow* f);

/* ---- Ensembles of independent flow models --------------------------------
 * (no counterpart in the reference: CMS-Flow runs one grid per process)
 * Members are cms_flow handles created as usual; an ensemble steps them
 * together.  When every member solves with BiCGStab in FP32 + refinement
 * (and the device can launch the persistent kernel), each of the three solves
 * of an outer iteration runs for all members in one batched persistent
 * launch; otherwise the members solve one after another.  Each member's
 * results are those of its own cms_flow_step up to rounding (dot products
 * are split over a different number of blocks). */
typedef struct cms_ensemble cms_ensemble;
int cms_ensemble_create(int nmembers, cms_flow* const* members, cms_ensemble** out);
/* Layout: blocks of the batched launch, split among members by unknowns
 * (0 = the device's resident capacity).  CMS_UNSUPPORTED when not batched. */
int cms_ensemble_set_tiles(cms_ensemble* e, int total_tiles);
/* Blocks of the batched launch in use; per_member (may be NULL) gets each
 * member's share. */
int cms_ensemble_tiles(const cms_ensemble* e, int* per_member);
int cms_ensemble_capacity(const cms_ensemble* e);
int cms_ensemble_batched(const cms_ensemble* e);
/* One time step of every member; wsebnd[i] holds member i's string levels
 * (NULL allowed for members without a string); infos: one per member. */
int cms_ensemble_step(cms_ensemble* e, double dt, const double* const* wsebnd, cms_flow_info* infos);
long long cms_ensemble_launches(const cms_ensemble* e);
/* Frees the ensemble, not its members. */
void cms_ensemble_destroy(cms_ensemble* e);

/* ---- reference-shaped global API (one implicit handle, like solv_def) ---- */

/* solv_init: source/solvers/solvers.f90:93-202. */
int cms_gpu_init(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet);
int cms_gpu_set_opts(const cms_solver_opts* opts);
int cms_gpu_update_wet(const int* iwet);
/* solve(acoef,ss,sp,res,phi,n): source/solvers/solvers.f90:205.  relax, nswp
 * and nsolv are the comvarbl values relax(n), nswp(n), nsolv; rmom receives
 * rmom(n).  Double for the ikind=8 build, float for ikind=4. */
int cms_gpu_solve_d(int n, const double* acoef, double* ss, const double* sp, double* res, double* phi, double relax,
                    int nswp, int nsolv, double* rmom);
int cms_gpu_solve_f(int n, const float* acoef, float* ss, const float* sp, float* res, float* phi, float relax,
                    int nswp, int nsolv, float* rmom);
/* The cms_solve_info of the last cms_gpu_solve_* call. */
int cms_gpu_last_info(cms_solve_info* info);
int cms_gpu_finalize(void);

/* ---- allocation-free entry point ------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they need it (a host that runs under a fixed device-memory
 * budget of its own pool, or that must not let cudaMalloc/cudaFree synchronise
 * the device in the middle of its time step): the solve() prologue of
 * source/solvers/solvers.f90:230-240 -- ap, the under-relaxed ss, the
 * normalised residual res and rmom = sqrt(sum res^2 / ncells) -- without a
 * solver handle and without any allocation.
 *
 * All array pointers are DEVICE pointers in the solve() layout (1-based
 * cell2cell, [ncellsD][nmaxfaces] acoef); ss is updated in place, res is
 * written, rmom is a HOST double.  stream is a cudaStream_t (NULL: the legacy
 * default stream); the call returns after the result is on the host.
 * Scratch is a fixed device array inside the library (about 0.5 MB per GPU,
 * held from load to exit); ncells above CMS_NOALLOC_MAX_CELLS is rejected with
 * CMS_BAD_ARGUMENT.  Every call resolves the array's address in the current
 * device's context (cudaGetSymbolAddress, no allocation), so the call works on
 * whichever device is current.  The call synchronises its stream and copies
 * rmom to the host, so it cannot be made during stream capture.  Every call
 * shares the one array, so calls that overlap on the GPU (other streams or
 * threads) race: serialise them.  cms_noalloc_last_error() gives the message of
 * the calling thread's last failed call. */
#define CMS_NOALLOC_MAX_CELLS 16777216
int cms_solve_residual_noalloc_d(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                                 const int* iwet, const double* acoef, double* ss, const double* sp, double* res,
                                 const double* phi, double relax, double* rmom, void* stream);
const char* cms_noalloc_last_error(void);

/* Failure-detection check of the bounded device waits: one block waits on a
 * progress flag that nothing sets, as the pipelined sweeps wait on a
 * neighbour row, and gives up after spin_limit polls.  Returns
 * CMS_DEVICE_ERROR with the wait's position in cms_gpu_last_error() -- the
 * expected result -- and leaves the handle usable. */
int cms_solver_wait_selftest(cms_solver* s, unsigned int spin_limit);
/* The same check for the persistent BiCGStab kernel's waits: which = 0 its
 * wait on a neighbour tile's progress counter, 1 its grid barrier, each run
 * by one block of a two-tile table whose other tile never runs, giving up
 * after spin_limit polls.  Returns CMS_DEVICE_ERROR with the message (the
 * expected result); the handle stays usable. */
int cms_solver_persist_wait_selftest(cms_solver* s, unsigned int spin_limit, int which);

/* Library version string. */
const char* cms_gpu_version(void);
/* Text of the last error a call reported (device or argument errors). */
const char* cms_gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CMSGPU_H */
