/*
 * CPU oracle for the GATT_DNS per-RK4-stage hot path -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the contract.  Pinned to the reference's own Fortran by golden vectors
 * (tests/golden/reference_*.npz: the unmodified derivs.F90, nseq.F90 and
 * timeIntegration.F90 run through a Fortran-subset translator).  Every function cites the
 * reference Fortran it restates; the element
 * operation order follows the Fortran expressions left to right (built with
 * -ffp-contract=off so no multiply-add is fused).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static int imod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

/* ------------------------------------------------------------------------- */
/* Line solves: derivs.F90:556-948                                            */
/* ------------------------------------------------------------------------- */

/* Solve one line.  F/dF point at the first element, s is the stride along the line.
 * Non-periodic: derivs.F90:583-611.  Periodic: derivs.F90:764-802. */
static void solve_line(const orc_dir *m, int t, const double *F, double *dF, long s)
{
    const int N = m->N, nR = m->nR;
    const int ldB = N - m->periodic;
    const double *R = m->R + (long)t * N * (2 * nR - 1);
    const double *A = m->A + (long)t * (N - 1);
    const double *B = m->B + (long)t * ldB;
    const double *C = m->C + (long)t * (N - 1);
    int i, l;
    /* RHS band product; the Fortran splits the rows in three ranges only to apply the
     * modulo where it can matter, so one modulo formula is equivalent. */
    for (i = 0; i < N; i++) {
        double acc = R[i + (long)(nR - 1) * N] * F[(long)i * s];
        for (l = 1; l <= nR - 1; l++) {
            acc = acc + R[i + (long)(nR - 1 + l) * N] * F[(long)imod(i + l, N) * s]
                      + R[i + (long)(nR - 1 - l) * N] * F[(long)imod(i - l, N) * s];
        }
        dF[(long)i * s] = acc;
    }
    if (!m->periodic) {
        dF[0] = dF[0] * B[0];
        for (i = 0; i < N - 1; i++)
            dF[(long)(i + 1) * s] = (dF[(long)(i + 1) * s] - A[i] * dF[(long)i * s]) * B[i + 1];
        for (i = N - 2; i >= 0; i--)
            dF[(long)i * s] = dF[(long)i * s] - C[i] * dF[(long)(i + 1) * s];
    } else {
        const double *D = m->D + (long)t * N;
        dF[0] = dF[0] * D[0];
        for (i = 1; i < N; i++) dF[0] = dF[0] + dF[(long)i * s] * D[i];
        dF[s] = dF[s] - A[0] * dF[0];
        dF[(long)(N - 1) * s] = dF[(long)(N - 1) * s] - C[0] * dF[0];
        dF[s] = dF[s] * B[0];
        for (i = 1; i < N - 1; i++)
            dF[(long)(i + 1) * s] = (dF[(long)(i + 1) * s] - A[i] * dF[(long)i * s]) * B[i];
        for (i = N - 2; i >= 1; i--)
            dF[(long)i * s] = dF[(long)i * s] - C[i] * dF[(long)(i + 1) * s];
    }
}

void orc_solve(const orc_case *c, int dir, int kind, const double *F, double *dF)
{
    const orc_dir *m = kind ? &c->fmat[dir] : &c->dmat[dir];
    const long nx = c->nx, ny = c->ny;
    const int nb = m->nBlocks;
    /* Flatten (block, line) pairs so OpenMP can spread the lines. */
    for (int bn = 0; bn < nb; bn++) {
        const int t = m->blocks[bn] - 1;
        const int a1 = m->blocks[bn + nb], a2 = m->blocks[bn + 2 * nb];
        const int b1 = m->blocks[bn + 3 * nb], b2 = m->blocks[bn + 4 * nb];
        const int na = a2 - a1 + 1, nbl = b2 - b1 + 1;
        #pragma omp parallel for schedule(static) if (na * nbl > 64)
        for (int q = 0; q < na * nbl; q++) {
            const long a = a1 - 1 + q % na, b = b1 - 1 + q / na;
            long base, s;
            if (dir == 0) { base = a * nx + b * nx * ny; s = 1; }          /* line (j,k) */
            else if (dir == 1) { base = a + b * nx * ny; s = nx; }         /* line (i,k) */
            else { base = a + b * nx; s = nx * ny; }                       /* line (i,j) */
            solve_line(m, t, F + base, dF + base, s);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Navier-Stokes right-hand side: nseq.F90:10-323                             */
/* ------------------------------------------------------------------------- */

/* Work arrays: the Fortran keeps its temporaries as automatic arrays, so a call pays no
 * allocation or first-touch cost after the first one.  Each call site owns fixed slots of a
 * persistent pool that grows to the largest grid seen (the oracle is not re-entrant). */
enum { SLOT_NSEQ = 0, SLOT_RK = 40, SLOT_BC = 50, SLOT_FILTER = 51, SLOT_STEP = 52, NSLOTS = 56 };
static double *g_pool[NSLOTS];
static long g_pool_n[NSLOTS];

static double *work_field(int slot, long n)
{
    if (g_pool_n[slot] < n) {
        free(g_pool[slot]);
        g_pool[slot] = (double *)malloc(sizeof(double) * (size_t)n);
        g_pool_n[slot] = n;
    }
    return g_pool[slot];
}

static void nseq2d(const orc_case *c, const double *U, const double *V, const double *R,
                   const double *E, double *dU, double *dV, double *dR, double *dE)
{
    const long n = (long)c->nx * c->ny * c->nz;
    const double g = c->gamma, Re = c->Re, Ma = c->Ma, Pr = c->Pr, T0 = c->T0;
    enum { DUx, DVx, DRx, DEx, DUy, DVy, DRy, DEy, TXX, TYY, TXY, DTXYX, DTXYY, DTXXX, DTYYY, QX, QY, HTX, HTY, MU, NT };
    double *w[NT];
    for (int k = 0; k < NT; k++) w[k] = work_field(SLOT_NSEQ + k, n);
    /* calcDerivsXY of U, V, R, E (nseq.F90:43-69) */
    orc_solve(c, 0, 0, U, w[DUx]); orc_solve(c, 1, 0, U, w[DUy]);
    orc_solve(c, 0, 0, V, w[DVx]); orc_solve(c, 1, 0, V, w[DVy]);
    orc_solve(c, 0, 0, R, w[DRx]); orc_solve(c, 1, 0, R, w[DRy]);
    orc_solve(c, 0, 0, E, w[DEx]); orc_solve(c, 1, 0, E, w[DEy]);
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < n; p++) {
        /* nseq.F90:77-85 */
        const double mu1 = (1.0 + 110.0 / T0) / (g * (g - 1.0) * Ma * Ma * E[p] + 110.0 / T0);
        const double mu2 = g * (g - 1.0) * Ma * Ma * E[p];
        const double mu = mu1 * mu2 * sqrt(mu2);
        const double dux = w[DUx][p], dvy = w[DVy][p];
        w[MU][p] = mu;
        w[TXX][p] = 1.0 / Re * mu * (2.0 * dux - 2.0 / 3.0 * (dux + dvy));
        w[TYY][p] = 1.0 / Re * mu * (2.0 * dvy - 2.0 / 3.0 * (dux + dvy));
        w[TXY][p] = 1.0 / Re * mu * (w[DUy][p] + w[DVx][p]);
        /* nseq.F90:109-110 */
        w[QX][p] = -g / Re / Pr * mu * w[DEx][p];
        w[QY][p] = -g / Re / Pr * mu * w[DEy][p];
    }
    orc_solve(c, 0, 0, w[TXY], w[DTXYX]); orc_solve(c, 1, 0, w[TXY], w[DTXYY]);
    orc_solve(c, 0, 0, w[TXX], w[DTXXX]);
    orc_solve(c, 1, 0, w[TYY], w[DTYYY]);
    orc_solve(c, 0, 0, w[QX], w[HTX]);
    orc_solve(c, 1, 0, w[QY], w[HTY]);
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < n; p++) {
        const double P = (g - 1.0) * R[p] * E[p];
        const double DPx = (g - 1.0) * (R[p] * w[DEx][p] + w[DRx][p] * E[p]);
        const double DPy = (g - 1.0) * (R[p] * w[DEy][p] + w[DRy][p] * E[p]);
        const double vtx = w[DTXXX][p] + w[DTXYY][p];
        const double vty = w[DTYYY][p] + w[DTXYX][p];
        const double dux = w[DUx][p], duy = w[DUy][p], dvx = w[DVx][p], dvy = w[DVy][p];
        /* nseq.F90:126-132 */
        dR[p] = -R[p] * (dux + dvy) - w[DRx][p] * U[p] - w[DRy][p] * V[p];
        dU[p] = -(dux * U[p] + duy * V[p]) + (vtx - DPx) / R[p];
        dV[p] = -(dvx * U[p] + dvy * V[p]) + (vty - DPy) / R[p];
        dE[p] = -(w[DEx][p] * U[p] + w[DEy][p] * V[p])
              + (-P * (dux + dvy) + w[TXX][p] * dux + w[TYY][p] * dvy + w[TXY][p] * (dvx + duy)
                 - w[HTX][p] - w[HTY][p]) / R[p];
    }
}

static void nseq3d(const orc_case *c, const double *U, const double *V, const double *W,
                   const double *R, const double *E,
                   double *dU, double *dV, double *dW, double *dR, double *dE)
{
    const long n = (long)c->nx * c->ny * c->nz;
    const double g = c->gamma, Re = c->Re, Ma = c->Ma, Pr = c->Pr, T0 = c->T0;
    enum { DUx, DUy, DUz, DVx, DVy, DVz, DWx, DWy, DWz, DRx, DRy, DRz, DEx, DEy, DEz,
           TXX, TYY, TZZ, TXY, TXZ, TYZ, QX, QY, QZ,
           DTXYX, DTXYY, DTXZX, DTXZZ, DTYZY, DTYZZ, DTXXX, DTYYY, DTZZZ, HTX, HTY, HTZ, NT };
    double *w[NT];
    for (int k = 0; k < NT; k++) w[k] = work_field(SLOT_NSEQ + k, n);
    const double *in[5] = {U, V, W, R, E};
    /* calcDerivsXYZ of U, V, W, R, E (nseq.F90:178-216) */
    for (int f = 0; f < 5; f++)
        for (int d = 0; d < 3; d++) orc_solve(c, d, 0, in[f], w[DUx + 3 * f + d]);
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < n; p++) {
        /* nseq.F90:225-239 */
        const double mu1 = (1.0 + 110.0 / T0) / (g * (g - 1.0) * Ma * Ma * E[p] + 110.0 / T0);
        const double mu2 = g * (g - 1.0) * Ma * Ma * E[p];
        const double mu = mu1 * mu2 * sqrt(mu2);
        double tzz = -2.0 / 3.0 * (w[DUx][p] + w[DVy][p] + w[DWz][p]);
        w[TXX][p] = 1.0 / Re * mu * (2.0 * w[DUx][p] + tzz);
        w[TYY][p] = 1.0 / Re * mu * (2.0 * w[DVy][p] + tzz);
        w[TZZ][p] = 1.0 / Re * mu * (2.0 * w[DWz][p] + tzz);
        w[TXY][p] = 1.0 / Re * mu * (w[DUy][p] + w[DVx][p]);
        w[TXZ][p] = 1.0 / Re * mu * (w[DUz][p] + w[DWx][p]);
        w[TYZ][p] = 1.0 / Re * mu * (w[DVz][p] + w[DWy][p]);
        /* nseq.F90:286-288 */
        w[QX][p] = -g / Re / Pr * mu * w[DEx][p];
        w[QY][p] = -g / Re / Pr * mu * w[DEy][p];
        w[QZ][p] = -g / Re / Pr * mu * w[DEz][p];
    }
    /* nseq.F90:241-306 */
    orc_solve(c, 0, 0, w[TXY], w[DTXYX]); orc_solve(c, 1, 0, w[TXY], w[DTXYY]);
    orc_solve(c, 0, 0, w[TXZ], w[DTXZX]); orc_solve(c, 2, 0, w[TXZ], w[DTXZZ]);
    orc_solve(c, 1, 0, w[TYZ], w[DTYZY]); orc_solve(c, 2, 0, w[TYZ], w[DTYZZ]);
    orc_solve(c, 0, 0, w[TXX], w[DTXXX]);
    orc_solve(c, 1, 0, w[TYY], w[DTYYY]);
    orc_solve(c, 2, 0, w[TZZ], w[DTZZZ]);
    orc_solve(c, 0, 0, w[QX], w[HTX]);
    orc_solve(c, 1, 0, w[QY], w[HTY]);
    orc_solve(c, 2, 0, w[QZ], w[HTZ]);
    #pragma omp parallel for schedule(static)
    for (long p = 0; p < n; p++) {
        const double P = (g - 1.0) * R[p] * E[p];
        const double DPx = (g - 1.0) * (R[p] * w[DEx][p] + w[DRx][p] * E[p]);
        const double DPy = (g - 1.0) * (R[p] * w[DEy][p] + w[DRy][p] * E[p]);
        const double DPz = (g - 1.0) * (R[p] * w[DEz][p] + w[DRz][p] * E[p]);
        const double vtx = w[DTXXX][p] + w[DTXYY][p] + w[DTXZZ][p];
        const double vty = w[DTYYY][p] + w[DTXYX][p] + w[DTYZZ][p];
        const double vtz = w[DTZZZ][p] + w[DTXZX][p] + w[DTYZY][p];
        const double dux = w[DUx][p], duy = w[DUy][p], duz = w[DUz][p];
        const double dvx = w[DVx][p], dvy = w[DVy][p], dvz = w[DVz][p];
        const double dwx = w[DWx][p], dwy = w[DWy][p], dwz = w[DWz][p];
        /* nseq.F90:310-318 */
        dR[p] = -R[p] * (dux + dvy + dwz) - w[DRx][p] * U[p] - w[DRy][p] * V[p] - w[DRz][p] * W[p];
        dU[p] = -(dux * U[p] + duy * V[p] + duz * W[p]) + (vtx - DPx) / R[p];
        dV[p] = -(dvx * U[p] + dvy * V[p] + dvz * W[p]) + (vty - DPy) / R[p];
        dW[p] = -(dwx * U[p] + dwy * V[p] + dwz * W[p]) + (vtz - DPz) / R[p];
        dE[p] = -(w[DEx][p] * U[p] + w[DEy][p] * V[p] + w[DEz][p] * W[p])
              + (-P * (dux + dvy + dwz) + w[TXX][p] * dux + w[TYY][p] * dvy + w[TZZ][p] * dwz
                 + w[TXY][p] * (dvx + duy) + w[TXZ][p] * (dwx + duz) + w[TYZ][p] * (dwy + dvz)
                 - w[HTX][p] - w[HTY][p] - w[HTZ][p]) / R[p];
    }
}

/* The forcings of runForcings2D/3D.F90 (writeFortranDisturbances.m writes one call per
 * forcing, on its box), in order, on the right-hand side nseq has formed. */
static void forcings(const orc_case *c, const double *U, const double *V, const double *W, const double *R,
                     const double *E, double *dU, double *dV, double *dW, double *dE)
{
    const long nx = c->nx, nxy = (long)c->nx * c->ny;
    for (int f = 0; f < c->nForce; f++) {
        int b[6];
        for (int q = 0; q < 6; q++) b[q] = c->forceInd[f + (long)q * c->nForce] - 1;
        const double *par = c->forcePar + 2 * f;
        if (c->forceType[f] == 1) {
            /* pressureGradient.F90: du = du + dpdx/r */
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) {
                        const long p = i + j * nx + k * nxy;
                        dU[p] = dU[p] + par[0] / R[p];
                    }
        } else if (c->forceType[f] == 2) {
            /* turbulenceGenerator.F90 on one rank: sums in array-element order, then
             * du = du + 0.25*epsilon*N/ET_sum*u - gamma*U_sum/N (gamma = 10*epsilon) */
            double ET = 0, Us = 0, Vs = 0, Ws = 0, Es = 0;
            long N = 0;
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) {
                        const long p = i + j * nx + k * nxy;
                        ET = ET + (U[p] * U[p] + V[p] * V[p] + W[p] * W[p]);
                        N++;
                    }
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) Us = Us + U[i + j * nx + k * nxy];
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) Vs = Vs + V[i + j * nx + k * nxy];
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) Ws = Ws + W[i + j * nx + k * nxy];
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) Es = Es + E[i + j * nx + k * nxy];
            const double eps = par[0], e0 = par[1], gamma = 10 * eps, Nd = (double)N;
            for (int k = b[4]; k <= b[5]; k++)
                for (int j = b[2]; j <= b[3]; j++)
                    for (int i = b[0]; i <= b[1]; i++) {
                        const long p = i + j * nx + k * nxy;
                        dU[p] = dU[p] + 0.25 * eps * Nd / ET * U[p] - gamma * Us / Nd;
                        dV[p] = dV[p] + 0.25 * eps * Nd / ET * V[p] - gamma * Vs / Nd;
                        dW[p] = dW[p] + 0.25 * eps * Nd / ET * W[p] - gamma * Ws / Nd;
                        dE[p] = dE[p] - gamma * (Es / Nd - e0);
                    }
        }
    }
}

void orc_nseq(const orc_case *c, const double *U, const double *V, const double *W,
              const double *R, const double *E,
              double *dU, double *dV, double *dW, double *dR, double *dE)
{
    if (c->nz == 1) nseq2d(c, U, V, R, E, dU, dV, dR, dE);
    else nseq3d(c, U, V, W, R, E, dU, dV, dW, dR, dE);
    if (c->nForce > 0) forcings(c, U, V, W, R, E, dU, dV, dW, dE);
}

/* ------------------------------------------------------------------------- */
/* Boundary conditions: nseq.F90:327-599                                      */
/* ------------------------------------------------------------------------- */

typedef struct { int i1, i2, j1, j2, k1, k2; } box_t;

static box_t box_of(const int *ind, int n, int row)
{
    box_t b;
    b.i1 = ind[row]; b.i2 = ind[row + n]; b.j1 = ind[row + 2 * n];
    b.j2 = ind[row + 3 * n]; b.k1 = ind[row + 4 * n]; b.k2 = ind[row + 5 * n];
    return b;
}

#define IDX(c, i, j, k) (((long)(i) - 1) + (long)(c)->nx * (((long)(j) - 1) + (long)(c)->ny * ((long)(k) - 1)))

/* getNeumannIndices (nseq.F90:520-550) */
static box_t neumann_box(box_t b, int dir, int len)
{
    switch (dir) {
    case 1: b.i2 += len; break;
    case 2: b.i1 -= len; break;
    case 3: b.j2 += len; break;
    case 4: b.j1 -= len; break;
    case 5: b.k2 += len; break;
    case 6: b.k1 -= len; break;
    }
    return b;
}

/* applyNeumann (nseq.F90:552-599) on the sub-array given by box b of field u. */
static void apply_neumann(const orc_case *c, double *u, box_t b, int dir, int len, const double *coef)
{
    int i, j, k, q;
    switch (dir) {
    case 1: case 2:
        for (k = b.k1; k <= b.k2; k++)
            for (j = b.j1; j <= b.j2; j++) {
                if (dir == 1) {
                    double v = coef[0] * u[IDX(c, b.i1 + 1, j, k)];
                    for (q = 2; q <= len; q++) v = v + coef[q - 1] * u[IDX(c, b.i1 + q, j, k)];
                    u[IDX(c, b.i1, j, k)] = v;
                } else {
                    double v = coef[0] * u[IDX(c, b.i1 + len - 1, j, k)];
                    for (q = 2; q <= len; q++) v = v + coef[q - 1] * u[IDX(c, b.i1 + len - q, j, k)];
                    u[IDX(c, b.i1 + len, j, k)] = v;
                }
            }
        break;
    case 3: case 4:
        for (k = b.k1; k <= b.k2; k++)
            for (i = b.i1; i <= b.i2; i++) {
                if (dir == 3) {
                    double v = coef[0] * u[IDX(c, i, b.j1 + 1, k)];
                    for (q = 2; q <= len; q++) v = v + coef[q - 1] * u[IDX(c, i, b.j1 + q, k)];
                    u[IDX(c, i, b.j1, k)] = v;
                } else {
                    double v = coef[0] * u[IDX(c, i, b.j1 + len - 1, k)];
                    for (q = 2; q <= len; q++) v = v + coef[q - 1] * u[IDX(c, i, b.j1 + len - q, k)];
                    u[IDX(c, i, b.j1 + len, k)] = v;
                }
            }
        break;
    case 5: case 6:
        for (j = b.j1; j <= b.j2; j++)
            for (i = b.i1; i <= b.i2; i++) {
                if (dir == 5) {
                    double v = coef[0] * u[IDX(c, i, j, b.k1 + 1)];
                    for (q = 2; q <= len; q++) v = v + coef[q - 1] * u[IDX(c, i, j, b.k1 + q)];
                    u[IDX(c, i, j, b.k1)] = v;
                } else {
                    double v = coef[0] * u[IDX(c, i, j, b.k1 + len - 1)];
                    for (q = 2; q <= len; q++) v = v + coef[q - 1] * u[IDX(c, i, j, b.k1 + len - q)];
                    u[IDX(c, i, j, b.k1 + len)] = v;
                }
            }
        break;
    }
}

#define FOR_BOX(b) \
    for (int k_ = (b).k1; k_ <= (b).k2; k_++) \
        for (int j_ = (b).j1; j_ <= (b).j2; j_++) \
            for (int i_ = (b).i1; i_ <= (b).i2; i_++)

/* periodicSine (source/disturbances/periodicSine.F90): pi and alpha are default reals
 * (single precision) there, so they are rounded to float here too. */
static void periodic_sine(const orc_case *c, double *u, box_t b, const double *x, double omega, double amp,
                          double t)
{
    const int n = b.i2 - b.i1 + 1;
    const float pi = (float)(4.0 * atan(1.0));
    const float alpha = (float)(2.0 * (double)pi / (x[n - 1] - x[0]));
    for (int k = b.k1; k <= b.k2; k++)
        for (int j = b.j1; j <= b.j2; j++)
            for (int i = 0; i < n; i++) {
                const long p = IDX(c, b.i1 + i, j, k);
                u[p] = u[p] + amp * sin((double)alpha * (x[i] - x[0])) * sin(omega * t);
            }
}

/* holdInlet (source/Fortran/holdInlet.F90): the first call keeps U, V, W, E (and R when the
 * density is held) on the box, every later call puts them back. */
static void hold_inlet(const orc_case *c, double *const *F, box_t b, double *save, int *saved, int holdR)
{
    const int order[5] = {0, 1, 2, 4, 3};  /* u, v, w, e, then r */
    const int nv = (*saved ? *saved - 1 : holdR) ? 5 : 4;
    long q = 0;
    for (int v = 0; v < nv; v++)
        FOR_BOX(b) {
            const long p = IDX(c, i_, j_, k_);
            if (*saved) F[order[v]][p] = save[q];
            else save[q] = F[order[v]][p];
            q++;
        }
    if (!*saved) *saved = 1 + holdR;  /* 1: U, V, W, E held; 2: R too */
}

/* lidDrivenMovement (source/disturbances/lidDrivenMovement.F90:1-19). */
static void lid_driven(const orc_case *c, double *u, box_t b, const double *x, double U0)
{
    const int n = b.i2 - b.i1 + 1;
    for (int k = b.k1; k <= b.k2; k++)
        for (int j = b.j1; j <= b.j2; j++)
            for (int i = 0; i < n; i++) {
                double s = 2 * (x[i] - x[0]) / (x[n - 1] - x[0]) - 1;
                double s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
                double p = 1 - s16 * s2;
                u[IDX(c, b.i1 + i, j, k)] = U0 * (p * p);
            }
}

void orc_apply_bc(const orc_case *c, double *U, double *V, double *W, double *R, double *E, double t)
{
    const long n = (long)c->nx * c->ny * c->nz;
    double *F[5] = {U, V, W, NULL, E};
    const double g = c->gamma;
    double *P = work_field(SLOT_BC, n);
    const int NL = c->neumannLength, N2 = c->neumann2Length;
    /* Dirichlet: nseq.F90:357-373 (U, V, W, E, then P) */
    const int dorder[4] = {0, 1, 2, 4};
    for (int q = 0; q < 4; q++) {
        const int v = dorder[q];
        for (int i = 0; i < c->nbc[0][v]; i++) {
            box_t b = box_of(c->ibc[0][v], c->nbc[0][v], i);
            FOR_BOX(b) F[v][IDX(c, i_, j_, k_)] = c->vbc[v][i];
        }
    }
    for (int i = 0; i < c->nbc[0][3]; i++) {
        box_t b = box_of(c->ibc[0][3], c->nbc[0][3], i);
        FOR_BOX(b) { long p = IDX(c, i_, j_, k_); R[p] = c->vbc[3][i] / (g - 1.0) / E[p]; }
    }
    /* Neumann: nseq.F90:377-400 (U, V, W, E, then P) */
    for (int q = 0; q < 4; q++) {
        const int v = dorder[q];
        for (int i = 0; i < c->nbc[1][v]; i++) {
            box_t b = box_of(c->ibc[1][v], c->nbc[1][v], i);
            const int d = c->dbc[1][v][i];
            apply_neumann(c, F[v], neumann_box(b, d, NL), d, NL, c->neumannCoeffs);
        }
    }
    for (int i = 0; i < c->nbc[1][3]; i++) {
        box_t b0 = box_of(c->ibc[1][3], c->nbc[1][3], i);
        const int d = c->dbc[1][3][i];
        box_t b = neumann_box(b0, d, NL);
        FOR_BOX(b) { long p = IDX(c, i_, j_, k_); P[p] = R[p] * E[p]; }
        apply_neumann(c, P, b, d, NL, c->neumannCoeffs);
        FOR_BOX(b0) { long p = IDX(c, i_, j_, k_); R[p] = P[p] / E[p]; }
    }
    /* Corners: nseq.F90:402-488 */
    for (int ci = 0; ci < c->cN; ci++) {
        box_t L = box_of(c->cL, c->cN, ci);
        int cd[3] = {c->cD[ci], c->cD[ci + c->cN], c->cD[ci + 2 * c->cN]};
        int nd = abs(cd[0]) + abs(cd[1]) + abs(cd[2]);
        if (c->cAdiabatic[ci] == 1) {
            FOR_BOX(L) E[IDX(c, i_, j_, k_)] = 0;
            for (int a = 0; a < 3; a++) {
                if (cd[a] == 0) continue;
                int d = cd[a] == 1 ? 2 * a + 1 : 2 * a + 2;
                box_t b = neumann_box(L, d, NL);
                FOR_BOX(b) { long p = IDX(c, i_, j_, k_); P[p] = E[p]; }
                apply_neumann(c, P, b, d, NL, c->neumannCoeffs);
                FOR_BOX(L) { long p = IDX(c, i_, j_, k_); E[p] = E[p] + P[p]; }
            }
            FOR_BOX(L) { long p = IDX(c, i_, j_, k_); E[p] = E[p] / nd; }
        }
        FOR_BOX(L) R[IDX(c, i_, j_, k_)] = 0;
        for (int a = 0; a < 3; a++) {
            if (cd[a] == 0) continue;
            int d = cd[a] == 1 ? 2 * a + 1 : 2 * a + 2;
            box_t b = neumann_box(L, d, NL);
            FOR_BOX(b) { long p = IDX(c, i_, j_, k_); P[p] = R[p] * E[p]; }
            apply_neumann(c, P, b, d, NL, c->neumannCoeffs);
            FOR_BOX(L) { long p = IDX(c, i_, j_, k_); R[p] = R[p] + P[p]; }
        }
        FOR_BOX(L) { long p = IDX(c, i_, j_, k_); R[p] = R[p] / E[p] / nd; }
    }
    /* Null second derivative: nseq.F90:491-513 */
    for (int q = 0; q < 4; q++) {
        const int v = dorder[q];
        for (int i = 0; i < c->nbc[2][v]; i++) {
            box_t b = box_of(c->ibc[2][v], c->nbc[2][v], i);
            const int d = c->dbc[2][v][i];
            apply_neumann(c, F[v], neumann_box(b, d, N2), d, N2, c->neumann2Coeffs);
        }
    }
    for (int i = 0; i < c->nbc[2][3]; i++) {
        box_t b0 = box_of(c->ibc[2][3], c->nbc[2][3], i);
        const int d = c->dbc[2][3][i];
        box_t b = neumann_box(b0, d, N2);
        FOR_BOX(b) { long p = IDX(c, i_, j_, k_); P[p] = R[p] * E[p]; }
        apply_neumann(c, P, b, d, N2, c->neumann2Coeffs);
        FOR_BOX(b0) { long p = IDX(c, i_, j_, k_); R[p] = P[p] / E[p]; }
    }
    /* Disturbances (runDisturbances.F90, generated by writeFortranDisturbances.m) */
    double *vars[5] = {U, V, W, R, E};
    for (int d = 0; d < c->nDist; d++) {
        box_t b = box_of(c->distInd, c->nDist, d);
        if (c->distType[d] == 1)
            lid_driven(c, vars[c->distVar[d]], b, c->distX + c->distXoff[d], c->distPar[d]);
        else if (c->distType[d] == 2)
            periodic_sine(c, vars[c->distVar[d]], b, c->distX + c->distXoff[d], c->distPar[d], c->distPar2[d], t);
        else if (c->distType[d] == 3)
            hold_inlet(c, vars, b, c->holdSave + c->holdOff[d], c->holdSaved + d, c->distPar[d] > 0.5);
    }
}

/* ------------------------------------------------------------------------- */
/* RK4: timeIntegration.F90:8-156 and 338-498                                 */
/* ------------------------------------------------------------------------- */

void orc_rk4(const orc_case *c, const double *U, const double *V, double *W, const double *R,
             const double *E, double *Un, double *Vn, double *Wn, double *Rn, double *En,
             double t, double dt)
{
    const long n = (long)c->nx * c->ny * c->nz;
    const int is3d = c->nz > 1;
    const double *q0[5] = {U, V, is3d ? W : NULL, R, E};
    double *qn[5] = {Un, Vn, is3d ? Wn : NULL, Rn, En};
    double *k[5], *delta[5];
    for (int f = 0; f < 5; f++) { k[f] = work_field(SLOT_RK + f, n); delta[f] = work_field(SLOT_RK + 5 + f, n); }
    /* In 2-D, the stage inputs carry the caller's W (RK4_2D passes W to applyBoundCond). */
    double *Wst = is3d ? Wn : W;
    /* Step 1 */
    orc_nseq(c, U, V, W, R, E, k[0], k[1], k[2], k[3], k[4]);
    for (int f = 0; f < 5; f++) {
        if (!is3d && f == 2) continue;
        #pragma omp parallel for schedule(static)
        for (long p = 0; p < n; p++) {
            delta[f][p] = dt / 6.0 * k[f][p];
            qn[f][p] = q0[f][p] + dt / 2.0 * k[f][p];
        }
    }
    for (int s = 2; s <= 4; s++) {
        const double tb = (s == 4) ? t + dt : t + dt / 2.0;
        orc_apply_bc(c, Un, Vn, Wst, Rn, En, tb);
        orc_nseq(c, Un, Vn, Wst, Rn, En, k[0], k[1], k[2], k[3], k[4]);
        for (int f = 0; f < 5; f++) {
            if (!is3d && f == 2) continue;
            #pragma omp parallel for schedule(static)
            for (long p = 0; p < n; p++) {
                if (s == 2) {
                    delta[f][p] = delta[f][p] + dt / 3.0 * k[f][p];
                    qn[f][p] = q0[f][p] + dt / 2.0 * k[f][p];
                } else if (s == 3) {
                    delta[f][p] = delta[f][p] + dt / 3.0 * k[f][p];
                    qn[f][p] = q0[f][p] + dt * k[f][p];
                } else {
                    qn[f][p] = q0[f][p] + delta[f][p] + dt / 6.0 * k[f][p];
                }
            }
        }
    }
    orc_apply_bc(c, Un, Vn, Wst, Rn, En, t + dt);
}

/* Euler: timeIntegration.F90:158-223 (2-D) and 500-567 (3-D).  The 3-D form applies the
 * boundary conditions at t, the 2-D form at t + dt (no time-dependent boundary data here). */
void orc_euler(const orc_case *c, const double *U, const double *V, double *W, const double *R,
               const double *E, double *Un, double *Vn, double *Wn, double *Rn, double *En,
               double t, double dt)
{
    const long n = (long)c->nx * c->ny * c->nz;
    const int is3d = c->nz > 1;
    const double *q0[5] = {U, V, is3d ? W : NULL, R, E};
    double *qn[5] = {Un, Vn, is3d ? Wn : NULL, Rn, En};
    double *k[5];
    for (int f = 0; f < 5; f++) k[f] = work_field(SLOT_RK + f, n);
    orc_nseq(c, U, V, W, R, E, k[0], k[1], k[2], k[3], k[4]);
    for (int f = 0; f < 5; f++) {
        if (!is3d && f == 2) continue;
        #pragma omp parallel for schedule(static)
        for (long p = 0; p < n; p++) qn[f][p] = q0[f][p] + dt * k[f][p];
    }
    orc_apply_bc(c, Un, Vn, is3d ? Wn : W, Rn, En, is3d ? t : t + dt);
}

/* SSPRK3: timeIntegration.F90:225-336 (2-D) and 569-680 (3-D): k1 at the step start, k2 at
 * q0 + dt k1, k3 at q0 + dt (k1 + k2) / 4, result q0 + dt (k1 + k2 + 4 k3) / 6, boundary
 * conditions after every stage.  acc holds k1, then k1 + k2. */
void orc_ssprk3(const orc_case *c, const double *U, const double *V, double *W, const double *R,
                const double *E, double *Un, double *Vn, double *Wn, double *Rn, double *En,
                double t, double dt)
{
    const long n = (long)c->nx * c->ny * c->nz;
    const int is3d = c->nz > 1;
    const double *q0[5] = {U, V, is3d ? W : NULL, R, E};
    double *qn[5] = {Un, Vn, is3d ? Wn : NULL, Rn, En};
    double *k[5], *acc[5];
    for (int f = 0; f < 5; f++) { k[f] = work_field(SLOT_RK + f, n); acc[f] = work_field(SLOT_RK + 5 + f, n); }
    double *Wst = is3d ? Wn : W;
    orc_nseq(c, U, V, W, R, E, k[0], k[1], k[2], k[3], k[4]);
    for (int s = 1; s <= 3; s++) {
        if (s > 1) orc_nseq(c, Un, Vn, Wst, Rn, En, k[0], k[1], k[2], k[3], k[4]);
        for (int f = 0; f < 5; f++) {
            if (!is3d && f == 2) continue;
            #pragma omp parallel for schedule(static)
            for (long p = 0; p < n; p++) {
                if (s == 1) {
                    acc[f][p] = k[f][p];
                    qn[f][p] = q0[f][p] + dt * k[f][p];
                } else if (s == 2) {
                    acc[f][p] = acc[f][p] + k[f][p];
                    qn[f][p] = q0[f][p] + dt * acc[f][p] / 4.0;
                } else {
                    qn[f][p] = q0[f][p] + dt * (acc[f][p] + 4.0 * k[f][p]) / 6.0;
                }
            }
        }
        orc_apply_bc(c, Un, Vn, Wst, Rn, En, s == 2 ? t + dt / 2.0 : t + dt);
    }
}

/* ------------------------------------------------------------------------- */
/* Filters: derivs.F90:303-552                                                */
/* ------------------------------------------------------------------------- */

void orc_filters(const orc_case *c, double *U, double *V, double *W, double *R, double *E, double blend)
{
    const long n = (long)c->nx * c->ny * c->nz;
    const int is3d = c->nz > 1;
    double *f[5] = {U, V, W, R, E};
    double *tmp = work_field(SLOT_FILTER, n);
    const int ndir = is3d ? 3 : 2;
    for (int d = 0; d < ndir; d++) {
        if (!c->filterDir[d]) continue;
        for (int q = 0; q < 5; q++) {
            if (!is3d && q == 2) continue;
            orc_solve(c, d, 1, f[q], tmp);
            if (blend > 0) {
                #pragma omp parallel for schedule(static)
                for (long p = 0; p < n; p++) tmp[p] = f[q][p] + blend * (tmp[p] - f[q][p]);
            }
            memcpy(f[q], tmp, sizeof(double) * (size_t)n);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* One step of the time loop: main.F90:255-465                                */
/* ------------------------------------------------------------------------- */

void orc_step(const orc_case *c, double *U, double *V, double *W, double *R, double *E,
              double *Wn, double *Um, double *Vm, double *Wm, double *Rm, double *Em,
              double t, double dt, double maxChange[5])
{
    const long n = (long)c->nx * c->ny * c->nz;
    const int is3d = c->nz > 1;
    double *Un = work_field(SLOT_STEP, n), *Vn = work_field(SLOT_STEP + 1, n), *Rn = work_field(SLOT_STEP + 2, n),
           *En = work_field(SLOT_STEP + 3, n);
    /* main.F90:304-352: the time integrator by parameters.F90 timeStepping */
    if (c->timeStepping == 2) orc_euler(c, U, V, W, R, E, Un, Vn, Wn, Rn, En, t, dt);
    else if (c->timeStepping == 3) orc_ssprk3(c, U, V, W, R, E, Un, Vn, Wn, Rn, En, t, dt);
    else orc_rk4(c, U, V, W, R, E, Un, Vn, Wn, Rn, En, t, dt);
    /* main.F90:357-378 -- the filter receives dt/FilterCharTime */
    orc_filters(c, Un, Vn, Wn, Rn, En, dt / c->filterCharTime);
    /* main.F90:381-402 */
    if (c->sfdType > 0) {
        double *qn[5] = {Un, Vn, Wn, Rn, En};
        double *qm[5] = {Um, Vm, Wm, Rm, Em};
        const int order[5] = {0, 1, 3, 4, 2};
        for (int q = 0; q < 5; q++) {
            const int f = order[q];
            if (f == 2 && !is3d) continue;
            if (c->sfdDelta > 0) {
                #pragma omp parallel for schedule(static)
                for (long p = 0; p < n; p++) qm[f][p] = qm[f][p] + dt / c->sfdDelta * (qn[f][p] - qm[f][p]);
            }
            #pragma omp parallel for schedule(static)
            for (long p = 0; p < n; p++) qn[f][p] = qn[f][p] - dt * c->sfdChi[p] * (qn[f][p] - qm[f][p]);
        }
    }
    /* main.F90:405-410 */
    orc_apply_bc(c, Un, Vn, Wn, Rn, En, t + dt);
    /* main.F90:413-418 */
    const double *a[5] = {Un, Vn, Wn, Rn, En};
    const double *b[5] = {U, V, W, R, E};
    for (int q = 0; q < 5; q++) {
        /* any NaN makes the result NaN, so a divergence is never masked */
        double m = 0;
        #pragma omp parallel
        {
            double mt = 0;
            #pragma omp for schedule(static) nowait
            for (long p = 0; p < n; p++) {
                double d = fabs(a[q][p] - b[q][p]);
                if (d > mt || d != d) mt = d;
            }
            #pragma omp critical
            if (mt > m || mt != mt) m = (m != m) ? m : mt;
        }
        maxChange[q] = m;
    }
    /* main.F90:459-465 */
    memcpy(U, Un, sizeof(double) * (size_t)n);
    memcpy(V, Vn, sizeof(double) * (size_t)n);
    memcpy(R, Rn, sizeof(double) * (size_t)n);
    memcpy(E, En, sizeof(double) * (size_t)n);
    if (is3d) memcpy(W, Wn, sizeof(double) * (size_t)n);
}
