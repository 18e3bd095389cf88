// Boundary conditions on the device: applyBoundCond (reference
// source/Fortran/nseq.F90:327-599) and the generated disturbance calls
// (runDisturbances.F90; source/disturbances/lidDrivenMovement.F90).
//
// The reference applies its lists strictly in order (Dirichlet U,V,W,E,P; Neumann
// U,V,W,E,P; corners; null second derivative U,V,W,E,P; disturbances), and later
// items read values earlier ones wrote.  The host flattens those lists into one
// program of box operations (BcOp) in that order; one CTA per batch member executes
// the program with a block barrier between dependent phases.  Boxes are boundary
// planes, so the whole program touches a small fraction of the field.
#pragma once

#include <cuda_runtime.h>
#include "pointwise.cuh"

namespace gatt {

enum BcOpCode {
    OP_SET = 0,        // F[var](box) = val
    OP_DIR_P = 1,      // R(box) = val/(gamma-1)/E(box)
    OP_NEU = 2,        // applyNeumann on F[var] over the extended box (face = first plane)
    OP_P_LOAD = 3,     // P(box) = R*E (box = extended box)
    OP_P_NEU = 4,      // applyNeumann on P over the extended box
    OP_R_FROM_P = 5,   // R(box) = P/E
    OP_CORNER_E0 = 6,  // E(box) = 0
    OP_P_FROM_E = 7,   // P(box) = E
    OP_E_ADD_P = 8,    // E(box) += P
    OP_E_DIV = 9,      // E(box) /= aux
    OP_R0 = 10,        // R(box) = 0
    OP_R_ADD_P = 11,   // R(box) += P
    OP_R_DIV_E = 12,   // R(box) = R/E/aux
    OP_LID = 13        // lidDrivenMovement on F[var](box), x coordinates at xoff, U0 = val
};

struct BcOp {
    int code;
    int var;        // 0..4 (U,V,W,R,E)
    int box[6];     // 1-based inclusive i1 i2 j1 j2 k1 k2
    int dir;        // 1..6 for Neumann
    int len;        // extrapolation length
    int coef;       // 0 = neumannCoeffs, 1 = neumann2Coeffs
    int aux;        // divisor for corner averages
    int xoff;       // offset of the box's x coordinates (OP_LID)
    double val;
};

struct BcProgram {
    const BcOp *ops;
    int nops;
    const double *coef1;  // neumannCoeffs
    const double *coef2;  // neumann2Coeffs
    const double *xs;     // disturbance coordinates
    double gamma;
    int nx, ny, nz;
};

__device__ __forceinline__ long long bidx(const BcProgram &pg, int i, int j, int k)
{
    return (long long)(i - 1) + (long long)pg.nx * ((long long)(j - 1) + (long long)pg.ny * (k - 1));
}

// Extrapolate the face of box b along dir from the next len nodes (applyNeumann,
// nseq.F90:552-599).  Threads stride over the face points.
__device__ void neumann_face(const BcProgram &pg, double *u, const int *b, int dir, int len, const double *c)
{
    int n1, n2;  // the two extents that span the face
    int a0, a1, c0, c1;
    if (dir <= 2) { a0 = b[2]; a1 = b[3]; c0 = b[4]; c1 = b[5]; }
    else if (dir <= 4) { a0 = b[0]; a1 = b[1]; c0 = b[4]; c1 = b[5]; }
    else { a0 = b[0]; a1 = b[1]; c0 = b[2]; c1 = b[3]; }
    n1 = a1 - a0 + 1; n2 = c1 - c0 + 1;
    const long long total = (long long)n1 * n2;
    for (long long q = threadIdx.x; q < total; q += blockDim.x) {
        const int a = a0 + (int)(q % n1), cc = c0 + (int)(q / n1);
        int i, j, k, di = 0, dj = 0, dk = 0;
        const bool lo = (dir & 1);               // odd dirs extrapolate at the low end
        const int s = lo ? 1 : -1;
        int face;
        if (dir <= 2) { face = lo ? b[0] : b[0] + len; di = s; j = a; k = cc; i = face; }
        else if (dir <= 4) { face = lo ? b[2] : b[2] + len; dj = s; i = a; k = cc; j = face; }
        else { face = lo ? b[4] : b[4] + len; dk = s; i = a; j = cc; k = face; }
        double v = c[0] * u[bidx(pg, i + di, j + dj, k + dk)];
        for (int m = 2; m <= len; m++) v = v + c[m - 1] * u[bidx(pg, i + m * di, j + m * dj, k + m * dk)];
        u[bidx(pg, i, j, k)] = v;
    }
}

// One CTA per batch member.  F: the five state arrays of this member (U,V,W,R,E);
// P: a scratch field of this member; x coordinates for disturbances in pg.xs.
__global__ void k_bc(BcProgram pg, StateSet q, double *Pbase, long long pstride)
{
    const int b = blockIdx.x;
    double *F[5];
#pragma unroll
    for (int f = 0; f < 5; f++) F[f] = q.v[f] + b * q.bstride;
    double *P = Pbase + b * pstride;
    double *Rr = F[3], *Ee = F[4];
    for (int o = 0; o < pg.nops; o++) {
        const BcOp op = pg.ops[o];
        if (op.code == OP_NEU || op.code == OP_P_NEU) {
            double *u = (op.code == OP_NEU) ? F[op.var] : P;
            neumann_face(pg, u, op.box, op.dir, op.len, op.coef ? pg.coef2 : pg.coef1);
            __syncthreads();
            continue;
        }
        const int ni = op.box[1] - op.box[0] + 1, nj = op.box[3] - op.box[2] + 1, nk = op.box[5] - op.box[4] + 1;
        const long long total = (long long)ni * nj * nk;
        for (long long q2 = threadIdx.x; q2 < total; q2 += blockDim.x) {
            const int i = op.box[0] + (int)(q2 % ni);
            const int j = op.box[2] + (int)((q2 / ni) % nj);
            const int k = op.box[4] + (int)(q2 / ((long long)ni * nj));
            const long long p = bidx(pg, i, j, k);
            switch (op.code) {
            case OP_SET: F[op.var][p] = op.val; break;
            case OP_DIR_P: Rr[p] = op.val / (pg.gamma - 1.0) / Ee[p]; break;
            case OP_P_LOAD: P[p] = Rr[p] * Ee[p]; break;
            case OP_R_FROM_P: Rr[p] = P[p] / Ee[p]; break;
            case OP_CORNER_E0: Ee[p] = 0.0; break;
            case OP_P_FROM_E: P[p] = Ee[p]; break;
            case OP_E_ADD_P: Ee[p] = Ee[p] + P[p]; break;
            case OP_E_DIV: Ee[p] = Ee[p] / (double)op.aux; break;
            case OP_R0: Rr[p] = 0.0; break;
            case OP_R_ADD_P: Rr[p] = Rr[p] + P[p]; break;
            case OP_R_DIV_E: Rr[p] = Rr[p] / Ee[p] / (double)op.aux; break;
            case OP_LID: {
                // lidDrivenMovement.F90:15-17
                const double *x = pg.xs + op.xoff;
                const double s = 2 * (x[i - op.box[0]] - x[0]) / (x[ni - 1] - x[0]) - 1;
                const double s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
                const double pp = 1 - s16 * s2;
                F[op.var][p] = op.val * (pp * pp);
                break;
            }
            default: break;
            }
        }
        // every item may read what the previous one wrote
        __syncthreads();
    }
}

}  // namespace gatt
