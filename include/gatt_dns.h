/*
 * gatt_dns.h -- C-ABI of the B200 (sm_100a) implementation of the GATT_DNS
 * per-RK4-stage hot path: compressible Navier-Stokes right-hand side, compact
 * derivative and filter line solves, RK4 stage update, SFD relaxation, boundary
 * conditions and the max-change residual.
 *
 * Drop-in boundary.  The reference Fortran solver (source/Fortran/main.F90) keeps
 * its time loop, CFL control, logging and I/O, and calls these entry points instead
 * of RK4_2D/RK4_3D, applyFilters2D/3D, the SFD block and applyBoundCond.  Every
 * array argument has the exact shape and meaning of the array main.F90 passes today
 * (column-major, 1-based indices inside index arrays); a Fortran
 * `interface ... bind(C)` module for these functions ships as include/gatt_dns_mod.f90.
 *
 * Conventions
 *  - Every function returns 0 (GATT_OK) or a GATT_ERR_* code; gatt_strerror() names it.
 *  - Host pointers are read during the call only; nothing is retained.
 *  - A context owns one CUDA stream (or the one given by gatt_set_stream); calls on
 *    one context must come from one host thread at a time.  Contexts are independent.
 *  - Fields are FP64, nx*ny*nz values, i fastest (Fortran order).  Variables are
 *    numbered U=0, V=1, W=2, R=3, E=4 (R = density, E = internal energy).
 *  - A context holds `nbatch` independent flow states that share the mesh,
 *    coefficients and boundary data; batch members are advanced together.
 */
#ifndef GATT_DNS_H
#define GATT_DNS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gatt_ctx gatt_ctx;

enum {
    GATT_OK = 0,
    GATT_ERR_CUDA = 1,      /* a CUDA runtime call failed (message in gatt_last_error) */
    GATT_ERR_BADARG = 2,    /* invalid argument: size, index box, direction, coverage */
    GATT_ERR_BADCOEF = 3,   /* non-finite coefficient or zero pivot in a matrix set */
    GATT_ERR_DIVERGED = 4,  /* max-change is NaN or all zero (main.F90:433-438) */
    GATT_ERR_TIMEOUT = 5,   /* a bounded device wait gave up */
    GATT_ERR_STATE = 6,     /* call out of order (e.g. step before matrices are set) */
    GATT_ERR_NOMEM = 7      /* device allocation failed */
};

enum { GATT_VAR_U = 0, GATT_VAR_V = 1, GATT_VAR_W = 2, GATT_VAR_R = 3, GATT_VAR_E = 4 };
enum { GATT_BC_DIRICHLET = 0, GATT_BC_NEUMANN = 1, GATT_BC_SECOND = 2 };
enum { GATT_DIST_LID_DRIVEN = 1, GATT_DIST_PERIODIC_SINE = 2, GATT_DIST_HOLD_INLET = 3 };

const char *gatt_strerror(int code);
/* Text of the last error raised on this host thread (CUDA message, argument name). */
const char *gatt_last_error(void);

/* Create a context for an nx*ny*nz grid (nz == 1 selects the 2-D equations of
 * nseq2d/RK4_2D) holding nbatch flow states.  Replaces the allocations of
 * main.F90:75-190 (decomp_2d_init on one rank: the whole grid is one pencil). */
int gatt_create(gatt_ctx **ctx, int nx, int ny, int nz, int nbatch);
void gatt_destroy(gatt_ctx *ctx);

/* Use the caller's CUDA stream (a cudaStream_t passed as void*) for all work. */
int gatt_set_stream(gatt_ctx *ctx, void *cuda_stream);

/* Physical parameters of parameters.F90 (writeFortranParameters.m:10-14). */
int gatt_set_physics(gatt_ctx *ctx, double Re, double Ma, double Pr, double gamma, double T0);

/* One direction's compact-scheme arrays, exactly as matrices.F90 allocates them
 * (writeFortranMatrices.m:73-110; consumed by derivs.F90:556-948):
 *   dir 1..3 = x, y, z; kind 0 = derivative (derivsA?.. derivsR?), 1 = filter (filterA?..)
 *   A(N-1,nTypes), B(N-periodic,nTypes), C(N-1,nTypes), D(N,nTypes) (periodic only,
 *   else may be NULL), R(N, 2*nRHS-1, nTypes); blocks(nBlocks,5) = derivBlocks? with
 *   1-based (type, a1, a2, b1, b2) line ranges.  The blocks must cover every line of the
 *   direction exactly once.  The filter uses the derivative blocks (main.F90:360), so
 *   kind 1 may pass nBlocks = 0 to reuse them.
 * Kinds 2..5 (no counterpart in the reference) hold the transposed operators the adjoint
 * needs, in the same factored form: a line operator L = LHS^-1 R has
 * L^T = R^T (LHS^T)^-1, so kind 2 = derivative LHS^T with an identity band, kind 3 =
 * identity LHS with the derivative R^T band, kinds 4 / 5 the same for the filter
 * (gatt_dns_b200/matrices.py: adjoint_sets emits them); they reuse the blocks. */
int gatt_set_matrices(gatt_ctx *ctx, int dir, int kind, int periodic, int nRHS, int nTypes,
                      const double *A, const double *B, const double *C, const double *D,
                      const double *R, int nBlocks, const int *blocks);

/* filterX/Y/Z and FilterCharTime of matrices.F90 / parameters.F90 (-1 = no blend). */
int gatt_set_filter(gatt_ctx *ctx, int filterX, int filterY, int filterZ, double filterCharTime);

/* timeStepping of parameters.F90, the integrator main.F90:304-352 selects: 1 RK4 (RK4_2D/3D,
 * the default), 2 Euler (EULER_2D/3D), 3 SSPRK3 (SSPRK3_2D/3D; timeIntegration.F90).
 * GATT_ERR_BADARG for any other value.  The tangent-linear and adjoint steps (gatt_jvp,
 * gatt_vjp) are RK4's and return GATT_ERR_STATE under the other two. */
int gatt_set_time_stepping(gatt_ctx *ctx, int timeStepping);

/* neumannCoeffs / neumann2Coeffs of matrices.F90 (getBoundaryConditions.m:75-80). */
int gatt_set_neumann(gatt_ctx *ctx, int neumannLength, const double *neumannCoeffs,
                     int neumann2Length, const double *neumann2Coeffs);

/* One boundary list of boundaryInfo.F90 (writeFortranBoundaries.m): var = U,V,W,E or
 * GATT_VAR_R for pressure (the reference's 'P' lists: iPd/vPd/iPn/dPn/iPs/dPs);
 * kind = Dirichlet (ind + val), Neumann or null-second-derivative (ind + dirs).
 * ind(n,6) holds 1-based [i1 i2 j1 j2 k1 k2]; dirs are 1..6 = xi,xf,yi,yf,zi,zf.
 * Replaces the nUd..dEs arguments of applyBoundCond (nseq.F90:327-345). */
int gatt_set_bc(gatt_ctx *ctx, int var, int kind, int n, const int *ind, const double *val,
                const int *dirs);

/* Corners: cN, cL(cN,6), cD(cN,3), cAdiabatic(cN) of boundaryInfo.F90 (nseq.F90:402-488). */
int gatt_set_corners(gatt_ctx *ctx, int cN, const int *cL, const int *cD, const int *cAdiabatic);

/* One generated disturbance call of runDisturbances.F90 (writeFortranDisturbances.m:35-90)
 * on the 1-based box ind[6], applied in the order added, with the box's x coordinates
 * x[ind[1]-ind[0]+1] and parameters par[npar]:
 * GATT_DIST_LID_DRIVEN = lidDrivenMovement(nx,ny,nz,x,y,z,t,u,U0)
 *   (source/disturbances/lidDrivenMovement.F90) on variable `var`, par = {U0};
 * GATT_DIST_PERIODIC_SINE = periodicSine(nx,ny,nz,x,y,z,t,u,omega,amplitude)
 *   (source/disturbances/periodicSine.F90) on variable `var`, par = {omega, amplitude}, at the
 *   time of each boundary-condition call (t + dt/2 or t + dt by stage, as timeIntegration.F90
 *   passes it; gatt_apply_bc's t);
 * GATT_DIST_HOLD_INLET = holdInlet(nx,ny,nz,x,y,z,t,u,v,r,w,e,holdDensity)
 *   (source/Fortran/holdInlet.F90) on U, V, W, E and, with par[0] > 0.5, R (var and x
 *   unused): the first gatt_apply_bc keeps their values on the box (main.F90:112 makes that
 *   call on the initial state), every later call puts them back.  Steps, the tangent-linear
 *   and the adjoint return GATT_ERR_STATE until that first call was made; adding or
 *   clearing disturbances that changes the held boxes drops the kept values. */
int gatt_add_disturbance(gatt_ctx *ctx, int type, int var, const int *ind, const double *x,
                         int npar, const double *par);
int gatt_clear_disturbances(gatt_ctx *ctx);

/* Forcings: the disturbances with forcing = true, which writeFortranDisturbances.m writes
 * into runForcings2D/3D.F90 and nseq2d/3d applies to the right-hand side it has formed
 * (nseq.F90:137, 321), in the order they are added, each on the 1-based box ind[6]:
 * GATT_FORCE_PRESSURE_GRADIENT = pressureGradient.F90 (par[0] = dpdx; dU += dpdx/R);
 * GATT_FORCE_TURBULENCE = turbulenceGenerator.F90 (par = {epsilon, e0}; 3-D only; box sums
 * of U*U + V*V + W*W, U, V, W, E of the right-hand side's input, then dU += 0.25*epsilon*
 * N/ET*U - 10*epsilon*Usum/N, likewise V and W, and dE -= 10*epsilon*(Esum/N - e0); one GPU
 * holds the whole box, as one rank does).  At most 4.  The tangent-linear and adjoint entry
 * points refuse contexts with forcings (GATT_ERR_STATE). */
#define GATT_FORCE_PRESSURE_GRADIENT 1
#define GATT_FORCE_TURBULENCE 2
int gatt_add_forcing(gatt_ctx *ctx, int type, const int *ind, int npar, const double *par);
int gatt_clear_forcings(gatt_ctx *ctx);

/* SFD (main.F90:122-164, 381-402): type 0 off, 1 constant chi = chiValue, 2 field chi
 * (nx*ny*nz, from calcSFDregion.m).  Delta <= 0 freezes the mean flow. */
int gatt_set_sfd(gatt_ctx *ctx, int type, double Delta, double chiValue, const double *chi);

/* Flow state of batch member b (host arrays of nx*ny*nz doubles each). */
int gatt_upload(gatt_ctx *ctx, int b, const double *U, const double *V, const double *W,
                const double *R, const double *E);
int gatt_download(gatt_ctx *ctx, int b, double *U, double *V, double *W, double *R, double *E);
/* SFD mean flow (Umean..Emean of main.F90:149-164). */
int gatt_upload_mean(gatt_ctx *ctx, int b, const double *U, const double *V, const double *W,
                     const double *R, const double *E);
int gatt_download_mean(gatt_ctx *ctx, int b, double *U, double *V, double *W, double *R,
                       double *E);
/* In 2-D, main.F90 keeps Wnew apart from W (it is never copied back); its value enters the
 * W max-change.  These move that array. */
int gatt_upload_wnew(gatt_ctx *ctx, int b, const double *Wnew);
int gatt_download_wnew(gatt_ctx *ctx, int b, double *Wnew);

/* Device pointer of a state field of member b (var 0..4), for callers that keep the flow
 * on the GPU between calls.  Valid until gatt_destroy. */
int gatt_state_device_ptr(gatt_ctx *ctx, int b, int var, double **dptr);

/* applyBoundCond on the device state at time t (nseq.F90:327-518), all members; the first
 * call keeps the holdInlet values (GATT_DIST_HOLD_INLET). */
int gatt_apply_bc(gatt_ctx *ctx, double t);

/* One compact line solve -- solveSystem{X,Y,Z}[per] (derivs.F90:556-948) -- of the host
 * field F into dF with the derivative (kind 0) or filter (kind 1) coefficients of dir, or
 * with one of the transposed-operator kinds 2..5. */
int gatt_deriv_dir(gatt_ctx *ctx, int dir, int kind, const double *F, double *dF);

/* Navier-Stokes right-hand side -- nseq2d / nseq3d (nseq.F90:10-323) -- of host fields;
 * in 2-D, W and dW are ignored. */
int gatt_rhs(gatt_ctx *ctx, const double *U, const double *V, const double *W, const double *R,
             const double *E, double *dU, double *dV, double *dW, double *dR, double *dE);

/* applyFilters2D/3D (derivs.F90:303-552) in place on the device state of all members;
 * blend = dt/FilterCharTime as main.F90:363 passes it. */
int gatt_filter(gatt_ctx *ctx, double blend);

/* One time step on the device state of all members: RK4_2D/RK4_3D, the filter, SFD,
 * applyBoundCond at t+dt, the max-change residual, and U = Unew (main.F90:255-465 minus the
 * CFL/dt control, logging and I/O).  maxChange receives 5*nbatch values (member-major);
 * it may be NULL.  Returns GATT_ERR_DIVERGED when a member's max-change is NaN or sums to
 * zero, as main.F90:433-438 stops. */
int gatt_step(gatt_ctx *ctx, double t, double dt, double *maxChange);

/* nsteps fixed-dt steps (t advances by dt each step, as main.F90:423 does) without a host
 * synchronisation per step; maxChange receives the last step's 5*nbatch values. */
int gatt_run(gatt_ctx *ctx, int nsteps, double t0, double dt, double *maxChange);

/* Jacobian-free Arnoldi, first-order variant of calcInstability.m:304-400, run for the
 * context's nbatch members as nbatch independent problems side by side (the Krylov index is
 * sequential within a problem; the batch advances every problem's step k together, each
 * member's arithmetic identical to a run of that member alone).
 *   base   host, 5*npts: U, V, W, R, E of the base flow, shared by all problems
 *   v0     host, nbatch*5*npts (member-major, then U, V, W, R, E): initial disturbances;
 *          zeta_1 = v0 restricted to the region and normalised (the reference passes its
 *          Gaussian bump unnormalised, calcInstability.m:309)
 *   region host npts bytes, nonzero = point in the flow region (calcInstability.m:137-141),
 *          or NULL for every point
 *   H      host, nbatch*(m+1)*m, column-major per member: H(i,k) at [b*(m+1)*m + k*(m+1) + i]
 * Vectors hold U, V, W, R, E (3-D) or U, V, R, E (2-D) over the region, N entries.  One
 * base run UM = Phi(base) (:327-340), then for k = 1..m: Phi(base + zeta_k*eps*sqrt(N))
 * over nsteps steps of dt from t0, B = (that - UM)/(eps*sqrt(N)), classical Gram-Schmidt
 * H(j,k) = zeta_j.B, H(k+1,k) = |B - sum H(j,k) zeta_j|, zeta_{k+1} (:364-400).  Leaves the
 * state at the last run's end; the basis stays on the device for gatt_arnoldi_vector.
 * m <= 512; device memory for the basis: nbatch*(m+1)*N doubles. */
int gatt_arnoldi(gatt_ctx *ctx, int m, int nsteps, double t0, double dt, double eps, const double *base,
                 const double *v0, const unsigned char *region, double *H);

/* Basis vector zeta_{j+1} (0 <= j <= m) of member b after gatt_arnoldi, as five host fields
 * U, V, W, R, E of npts each (W zero in 2-D, zero outside the region): the psiA = zeta*psiH
 * mode reconstruction of calcInstability.m:419 is left to the caller. */
int gatt_arnoldi_vector(gatt_ctx *ctx, int b, int j, double *out);

/* Tangent-linear and adjoint of the RHS and time step (no counterpart in the reference;
 * the reference linearises only by finite differences, calcInstability.m:353-390).  They
 * cover the whole step of 2-D and 3-D cases: RK4, boundary-condition program (lists,
 * corners, disturbances), filter and SFD; the adjoint also needs matrix kinds 2..5.  Arrays
 * are host, member-major: per member the five fields U, V, W, R, E of npts each (in 2-D the W
 * components are ignored on input and zero on output).  With SFD (gatt_set_sfd, type > 0)
 * the step maps the state and the mean, and the gatt_jvp / gatt_vjp vectors carry both:
 * per member U, V, W, R, E, then the mean's U, V, W, R, E (nbatch*10*npts); those two need
 * the mean set (gatt_upload_mean or a previous step), GATT_ERR_STATE otherwise.
 *   gatt_rhs_jvp: dk = F'(q) dq of nseq2d / nseq3d (nseq.F90:10-323), nbatch*5*npts arrays
 *   gatt_rhs_vjp: lam = F'(q)^T a
 *   gatt_jvp:     dqN = (dPhi/dq) dq0 over nsteps steps of dt from the context state (which
 *                 advances to the end state, as gatt_run)
 *   gatt_vjp:     lam0 = (dPhi/dq)^T lamN over nsteps steps from the context state, keeping a
 *                 checkpoint every checkpoint_every steps and recomputing each segment's
 *                 states for the reverse sweep; the context state ends at the end state. */
int gatt_rhs_jvp(gatt_ctx *ctx, const double *q, const double *dq, double *dk);
int gatt_rhs_vjp(gatt_ctx *ctx, const double *q, const double *a, double *lam);
int gatt_jvp(gatt_ctx *ctx, int nsteps, double t0, double dt, const double *dq0, double *dqN);
int gatt_vjp(gatt_ctx *ctx, int nsteps, double t0, double dt, int checkpoint_every, const double *lamN,
             double *lam0);

/* Autotuner (no counterpart in the reference): for every matrix set of the context, times
 * each applicable line-solve configuration on the context's grid -- the TMA-fed and the plain
 * register-resident solvers (16-row blocks) and the shared-tile solver at 8, 16, 32 and 64
 * rows per block -- over `reps` launches of one sweep of 5 (3-D) or 4 (2-D) scratch fields,
 * and keeps the fastest.  Per set (index dir*6 + kind, dir 0..2, kind 0..5), family[] gets
 * 0 shared tile, 1 register, 2 TMA-fed register (-1: no matrices), blocks[] the row-block
 * count and us[] the mean microseconds of one launch; any of them may be NULL.  Overwrites
 * the derivative scratch; call it after the matrices and before the first step. */
int gatt_autotune(gatt_ctx *ctx, int reps, int *family, int *blocks, double *us);

/* Self-test of the pipelined line solver's failure path (no counterpart in the reference):
 * runs one x-direction sweep whose copy barriers expect 16 bytes more than the copies
 * deliver, so that every bounded wait gives up (after 1 s; the real copies have landed by
 * then).  Returns the status the next synchronisation reports -- GATT_ERR_TIMEOUT when the
 * path works -- and leaves the context usable.  GATT_ERR_STATE when x lines do not use the
 * pipelined solver. */
int gatt_selftest_pipeline_timeout(gatt_ctx *ctx);

/* max|U|, max|V|, max|W| of every member (main.F90:196-204), for the caller's CFL. */
int gatt_max_velocity(gatt_ctx *ctx, double *vmax);

/* Wait for all work of the context. */
int gatt_synchronize(gatt_ctx *ctx);

/* Number of kernels this context launched since creation (for launch accounting). */
long long gatt_kernel_launches(gatt_ctx *ctx);

/* Profiling hook (no counterpart in the reference): runs nsteps uncaptured steps with a
 * CUDA event pair around every kernel launch and returns, per kernel class, the mean
 * device time of one launch in ms[GATT_NPROF] and the launches per step in
 * launches[GATT_NPROF].  Advances the state like gatt_run.  gatt_profile_name(i) names
 * class i. */
#define GATT_NPROF 17
int gatt_profile_kernels(gatt_ctx *ctx, double t0, double dt, int nsteps, double *ms, double *launches);
const char *gatt_profile_name(int cls);

/* Max-change residual that allocates nothing.  No counterpart in the reference (whose
 * max-change is the maxval reduction of main.F90:413-418): for callers that cannot call
 * cudaMalloc -- typically a host application whose own allocator owns all device memory
 * and forbids further allocations -- and so cannot create a context, but hold the fields
 * in device memory themselves.  For set s < nsets and variable v < nvar,
 * maxChange[s*nvar+v] = max_i |a[s*nvar+v][i] - b[s*nvar+v][i]| over n points, where a and
 * b are host arrays of device pointers; a NaN difference yields NaN.  The work runs on
 * `stream` (a cudaStream_t, NULL = default stream) and the call synchronises it and
 * returns the maxima in host memory; on a stream that is being captured it returns
 * GATT_ERR_STATE without enqueuing anything.
 * Limits: nvar <= 5 and nsets*nvar <= 160 (the accumulators are a 1280-byte static device
 * array that every GPU loading the library keeps until exit); larger requests return
 * GATT_ERR_BADARG.  The first call on a device looks up that array's address (the only
 * set-up, done once per device under a lock).  All calls share the array, so calls that
 * overlap on the GPU race; each call clears its accumulators first. */
int gatt_max_change_noalloc(int nsets, int nvar, long long n, const double *const *a, const double *const *b,
                            double *maxChange, void *stream);

#ifdef __cplusplus
}
#endif
#endif
