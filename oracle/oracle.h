/*
 * CPU oracle for the GATT_DNS per-RK4-stage hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference Fortran (source/Fortran/derivs.F90,
 * nseq.F90, timeIntegration.F90 and the filter / SFD / max-change block of
 * main.F90), with the same per-element operation order.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker or as the timed CPU baseline -- never as the product.
 *
 * Parity status: pinned to the reference's own Fortran.  The reference ships no tests
 * or golden outputs and cannot be compiled here (no Fortran compiler, no MPI, no
 * MATLAB), so tests/golden/make_reference_golden.py runs its unmodified derivs.F90,
 * nseq.F90 and timeIntegration.F90 through a Fortran-subset translator on small cases
 * and stores the outputs (tests/golden/reference_*.npz); tests/test_oracle_vs_reference.py
 * holds this restatement to them (line solves of every direction and kind, right-hand
 * side, boundary conditions, filters, one time step), besides known-answer tests
 * (spectral derivatives of trigonometric fields, filter transfer functions,
 * conservation on a periodic box).
 *
 * Arrays are Fortran column-major (i fastest), index blocks and boundary boxes are
 * 1-based exactly as matrices.F90 / boundaryInfo.F90 declare them.
 */
#ifndef GATT_ORACLE_H
#define GATT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One direction's coefficients, as the arrays matrices.F90 allocates
 * (writeFortranMatrices.m:73-110): A(N-1,nT), B(N-periodic,nT), C(N-1,nT),
 * D(N,nT) (periodic only), R(N,2*nR-1,nT); blocks(nBlocks,5). */
typedef struct {
    int periodic;
    int nR;
    int nTypes;
    int N;
    const double *A, *B, *C, *D, *R;
    int nBlocks;
    const int *blocks;
} orc_dir;

/* Boundary data, as boundaryInfo.F90 declares it (writeFortranBoundaries.m).
 * Variable order inside every [5] is U, V, W, P, E; kind order is d, n, s. */
typedef struct {
    int nx, ny, nz;
    double Re, Ma, Pr, gamma, T0;
    orc_dir dmat[3];
    orc_dir fmat[3];
    int filterDir[3];
    double filterCharTime;           /* parameters.F90 FilterCharTime (-1 = off) */
    int neumannLength, neumann2Length;
    const double *neumannCoeffs, *neumann2Coeffs;
    int nbc[3][5];
    const int *ibc[3][5];
    const double *vbc[5];
    const int *dbc[3][5];            /* only kinds n (1) and s (2) are used */
    int cN;
    const int *cL, *cD, *cAdiabatic; /* (cN,6), (cN,3), (cN) */
    int nDist;                       /* disturbances, type 1 = lidDrivenMovement */
    const int *distType, *distVar, *distInd; /* distInd (nDist,6) col-major */
    const double *distX;             /* x coordinates of every box, concatenated */
    const int *distXoff;             /* offset of box d's coordinates in distX */
    const double *distPar;           /* one parameter per disturbance (U0 for the lid) */
    int sfdType;                     /* 0 off, 1 constant, 2 field */
    double sfdDelta;
    const double *sfdChi;            /* nx*ny*nz field (type 1: filled by caller) */
    int timeStepping;                /* parameters.F90 timeStepping: 1 (or 0) RK4, 2 Euler, 3 SSPRK3 */
    /* forcings of runForcings2D/3D.F90, applied at the end of nseq (nseq.F90:137, 321) in
     * order: type 1 = pressureGradient (par dpdx; dU += dpdx/R), 2 = turbulenceGenerator
     * (par epsilon, e0; on U, V, W, E); forceInd (nForce,6) col-major 1-based boxes */
    int nForce;
    const int *forceType, *forceInd;
    const double *forcePar;          /* two per forcing */
    /* disturbances of types 2 = periodicSine (distPar = omega, distPar2 = amplitude; uses the
     * boundary-condition time) and 3 = holdInlet (distPar > 0.5: hold the density too; the
     * first call saves U, V, W, E (and R) on the box into holdSave + holdOff[d] and sets
     * holdSaved[d], later calls restore them) */
    const double *distPar2;
    double *holdSave;
    const long *holdOff;
    int *holdSaved;
} orc_case;

int orc_num_threads(void);
void orc_set_threads(int n);

/* solveSystem{X,Y,Z}[per] with a field F (derivs.F90:556-948).  kind 0 = derivative
 * coefficients, 1 = filter coefficients; dir 0,1,2 = x,y,z. */
void orc_solve(const orc_case *c, int dir, int kind, const double *F, double *dF);

/* nseq2d / nseq3d (nseq.F90:10-323).  In 2-D (nz == 1) W and dW are ignored. */
void orc_nseq(const orc_case *c, const double *U, const double *V, const double *W,
              const double *R, const double *E,
              double *dU, double *dV, double *dW, double *dR, double *dE);

/* applyBoundCond (nseq.F90:327-599) followed by the disturbances. */
void orc_apply_bc(const orc_case *c, double *U, double *V, double *W, double *R, double *E, double t);

/* RK4_2D / RK4_3D (timeIntegration.F90:8-156, 338-498).  In 2-D, W is updated in place
 * by the boundary conditions and Wn is untouched, as RK4_2D does. */
void orc_rk4(const orc_case *c, const double *U, const double *V, double *W, const double *R,
             const double *E, double *Un, double *Vn, double *Wn, double *Rn, double *En,
             double t, double dt);

/* applyFilters2D / applyFilters3D (derivs.F90:303-552); blend = dt/FilterCharTime. */
void orc_filters(const orc_case *c, double *U, double *V, double *W, double *R, double *E, double blend);

/* One time step of main.F90:255-465 minus the time control: RK4, filter, SFD,
 * boundary conditions, max-change, and U = Unew.  Wn is the persistent Wnew array
 * (its contents matter in 2-D, where main.F90 never copies it into W).
 * mean may be NULL when SFD is off. */
void orc_step(const orc_case *c, double *U, double *V, double *W, double *R, double *E,
              double *Wn, double *Um, double *Vm, double *Wm, double *Rm, double *Em,
              double t, double dt, double maxChange[5]);

#ifdef __cplusplus
}
#endif
#endif
