// Boundary conditions on the device: applyBoundCond (reference
// source/Fortran/nseq.F90:327-599) and the generated disturbance calls
// (runDisturbances.F90; source/disturbances/lidDrivenMovement.F90, periodicSine.F90,
// source/Fortran/holdInlet.F90).
//
// The reference applies its lists strictly in order (Dirichlet U,V,W,E,P; Neumann
// U,V,W,E,P; corners; null second derivative U,V,W,E,P; disturbances), and later
// items read values earlier ones wrote.  The host flattens those lists into one
// program of box operations (BcOp) in that order.  A cluster of CTAs (up to 16 SMs) per batch
// member executes the program, the points of each op spread over all its threads, with the
// cluster barrier (release/acquire at cluster scope: every write is visible after it) between
// dependent ops; where a cluster cannot be launched, one CTA per member with block barriers.
// Consecutive ops whose boxes and fields do not conflict form one phase without a barrier
// (the host sets BcOp::sync on the last op of each phase).  Boxes are boundary planes, so the whole program touches a small fraction of
// the field, but on one SM it cost half of a boundary-layer step.
#pragma once

#include <cooperative_groups.h>
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
    OP_LID = 13,       // lidDrivenMovement on F[var](box), x coordinates at xoff, U0 = val
    OP_SINE = 14,      // periodicSine: F[var](box) += xs[xoff + i - i1] * sin(val * t)
    OP_HOLD = 15       // holdInlet: aux fields (U, V, W, E, then R) of the box <-> hold + xoff
};

struct BcOp {
    int code;
    int var;        // 0..4 (U,V,W,R,E)
    int box[6];     // 1-based inclusive i1 i2 j1 j2 k1 k2
    int dir;        // 1..6 for Neumann
    int len;        // extrapolation length
    int coef;       // 0 = neumannCoeffs, 1 = neumann2Coeffs
    int aux;        // divisor for corner averages
    int xoff;       // offset of the box's x coordinates (OP_LID), of its x factors (OP_SINE), of
                    // its values in the member's hold buffer (OP_HOLD)
    int sync;       // barrier after this op (the next op depends on this op's phase)
    double val;
    long long tape; // adjoint tape: offset of this op's recorded base values (-1: none)
};

static_assert(sizeof(BcOp) % sizeof(long long) == 0, "ops are staged as 8-byte words");

struct BcProgram {
    const BcOp *ops;
    int nops;
    const double *coef1;  // neumannCoeffs
    const double *coef2;  // neumann2Coeffs
    const double *xs;     // disturbance coordinates (OP_LID) and x factors (OP_SINE)
    double gamma;
    int nx, ny, nz;
    // the time of the call: sp->t + tfac * sp->dt (the step's parameters on the device, so that
    // one captured program serves every step), or tfix when sp is null
    const StepParams *sp;
    double tfac, tfix;
    double *hold;         // holdInlet values, hstride per member
    long long hstride;
    int hold_save;        // 1: OP_HOLD keeps the fields (first call), 0: puts them back
};

__device__ __forceinline__ double bc_time(const BcProgram &pg)
{
    return pg.sp ? pg.sp->t + pg.tfac * pg.sp->dt : pg.tfix;
}

// periodicSine.F90:17-19: u + (amplitude sin(alpha (x_i - x_1))) sin(omega t), the x factor
// precomputed per point; the product and the sum rounded separately as the reference does
__device__ __forceinline__ double bc_sine(double u, double fx, double omega, double t)
{
    return __dadd_rn(u, __dmul_rn(fx, sin(omega * t)));
}

// holdInlet.F90 keeps u, v, w, e (and r with holdDensity): field of the v-th held value
__device__ __forceinline__ int bc_hold_field(int v) { return v < 3 ? v : (v == 3 ? 4 : 3); }

__device__ __forceinline__ long long bidx(const BcProgram &pg, int i, int j, int k)
{
    return (long long)(i - 1) + (long long)pg.nx * ((long long)(j - 1) + (long long)pg.ny * (k - 1));
}

// Extrapolate the face of box b along dir from the next len nodes (applyNeumann,
// nseq.F90:552-599).  Thread tid of nthr strides over the face points.
__device__ void neumann_face(const BcProgram &pg, double *u, const int *b, int dir, int len, const double *c,
                             int tid, int nthr)
{
    int n1, n2;  // the two extents that span the face
    int a0, a1, c0, c1;
    if (dir <= 2) { a0 = b[2]; a1 = b[3]; c0 = b[4]; c1 = b[5]; }
    else if (dir <= 4) { a0 = b[0]; a1 = b[1]; c0 = b[4]; c1 = b[5]; }
    else { a0 = b[0]; a1 = b[1]; c0 = b[2]; c1 = b[3]; }
    n1 = a1 - a0 + 1; n2 = c1 - c0 + 1;
    const long long total = (long long)n1 * n2;
    for (long long q = tid; q < total; q += nthr) {
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

// Largest program whose ops are staged in shared memory (48 KB, no opt-in needed); longer
// programs read their ops from global memory.
constexpr int kBcStagedOps = 48 * 1024 / (int)sizeof(BcOp);

// The program on one member: F the five state arrays (U,V,W,R,E), P a scratch field, thread
// tid of nthr; sync() is a barrier over all nthr threads that orders their memory accesses.
// sops: the ops copied to this CTA's shared memory (nullptr: read them from pg.ops).
template <typename Sync>
__device__ __forceinline__ void bc_run(const BcProgram &pg, const BcOp *sops, double *const *F, double *P, double *H,
                                       int tid, int nthr, Sync sync)
{
    double *Rr = F[3], *Ee = F[4];
    const BcOp *ops = sops ? sops : pg.ops;
    const double tnow = bc_time(pg);
    for (int o = 0; o < pg.nops; o++) {
        const BcOp op = ops[o];
        if (op.code == OP_NEU || op.code == OP_P_NEU) {
            double *u = (op.code == OP_NEU) ? F[op.var] : P;
            neumann_face(pg, u, op.box, op.dir, op.len, op.coef ? pg.coef2 : pg.coef1, tid, nthr);
            if (op.sync) sync();
            continue;
        }
        // 32-bit index arithmetic: a box holds fewer than 2^31 points (the grid does)
        const unsigned ni = op.box[1] - op.box[0] + 1, nj = op.box[3] - op.box[2] + 1, nk = op.box[5] - op.box[4] + 1;
        const unsigned nij = ni * nj, total = nij * nk;
        for (unsigned q2 = tid; q2 < total; q2 += nthr) {
            const unsigned kq = q2 / nij, r = q2 - kq * nij, jq = r / ni;
            const int i = op.box[0] + (int)(r - jq * ni);
            const int j = op.box[2] + (int)jq;
            const int k = op.box[4] + (int)kq;
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
            case OP_SINE: F[op.var][p] = bc_sine(F[op.var][p], pg.xs[op.xoff + i - op.box[0]], op.val, tnow); break;
            case OP_HOLD:
                for (int v = 0; v < op.aux; v++) {
                    double *h = H + op.xoff + (long long)v * total + q2;
                    if (pg.hold_save) *h = F[bc_hold_field(v)][p];
                    else F[bc_hold_field(v)][p] = *h;
                }
                break;
            default: break;
            }
        }
        // the next op reads or writes what this phase wrote (or writes what it read)
        if (op.sync) sync();
    }
}

// Copy the ops to shared memory (when they fit); every thread of the CTA calls it.
__device__ __forceinline__ const BcOp *bc_stage_ops(const BcProgram &pg, BcOp *sops)
{
    if (pg.nops > kBcStagedOps) return nullptr;
    const int n = pg.nops * (int)(sizeof(BcOp) / sizeof(long long));
    const long long *g = reinterpret_cast<const long long *>(pg.ops);
    long long *d = reinterpret_cast<long long *>(sops);
    for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = g[i];
    __syncthreads();
    return sops;
}

// One CTA per batch member (block barriers); dynamic shared memory: the staged ops.
__global__ void k_bc(BcProgram pg, StateSet q, double *Pbase, long long pstride)
{
    extern __shared__ BcOp bc_sops[];
    const int b = blockIdx.x;
    double *F[5];
#pragma unroll
    for (int f = 0; f < 5; f++) F[f] = q.v[f] + b * q.bstride;
    const BcOp *sops = bc_stage_ops(pg, bc_sops);
    double *H = pg.hold ? pg.hold + b * pg.hstride : nullptr;
    bc_run(pg, sops, F, Pbase + b * pstride, H, threadIdx.x, blockDim.x, [] { __syncthreads(); });
}

// One cluster of CTAs per batch member (cluster barriers); launched with a cluster dimension.
__global__ void k_bc_cluster(BcProgram pg, StateSet q, double *Pbase, long long pstride)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int b = blockIdx.x / (int)cl.num_blocks();
    double *F[5];
#pragma unroll
    for (int f = 0; f < 5; f++) F[f] = q.v[f] + b * q.bstride;
    extern __shared__ BcOp bc_sops[];
    const int nthr = (int)cl.num_threads();
    const int tid = (int)cl.block_rank() * blockDim.x + threadIdx.x;
    const BcOp *sops = bc_stage_ops(pg, bc_sops);
    double *H = pg.hold ? pg.hold + b * pg.hstride : nullptr;
    bc_run(pg, sops, F, Pbase + b * pstride, H, tid, nthr, [&] { cl.sync(); });
}

// ---- tangent-linear and adjoint of the program (no counterpart in the reference) -------
//
// The program is a sequence of in-place box updates; the nonlinear ones (pressure Dirichlet,
// P = R E, R = P / E, R = R / E / aux) need the base values they saw.  The tangent runs
// base and tangent side by side; the adjoint runs the ops in reverse with those base values
// read from a tape that k_bc_rec wrote while applying the program to the base state.
// Values recorded per box point, in the box's loop order: OP_DIR_P: E; OP_P_LOAD: R, E;
// OP_R_FROM_P: P, E; OP_R_DIV_E: R, E.

__host__ __device__ __forceinline__ int bc_tape_width(int code)
{
    return code == OP_DIR_P ? 1 : (code == OP_P_LOAD || code == OP_R_FROM_P || code == OP_R_DIV_E) ? 2 : 0;
}

// Face point q of a Neumann op: the face node and the unit step into the domain.
__device__ __forceinline__ void neumann_geom(const int *b, int dir, int len, long long q, int n1, int &i, int &j,
                                             int &k, int &di, int &dj, int &dk)
{
    int a0, c0;
    if (dir <= 2) { a0 = b[2]; c0 = b[4]; }
    else if (dir <= 4) { a0 = b[0]; c0 = b[4]; }
    else { a0 = b[0]; c0 = b[2]; }
    const int a = a0 + (int)(q % n1), cc = c0 + (int)(q / n1);
    const bool lo = (dir & 1);
    const int s = lo ? 1 : -1;
    di = dj = dk = 0;
    if (dir <= 2) { i = lo ? b[0] : b[0] + len; di = s; j = a; k = cc; }
    else if (dir <= 4) { j = lo ? b[2] : b[2] + len; dj = s; i = a; k = cc; }
    else { k = lo ? b[4] : b[4] + len; dk = s; i = a; j = cc; }
}

__device__ __forceinline__ void neumann_extent(const int *b, int dir, int &n1, int &n2)
{
    if (dir <= 2) { n1 = b[3] - b[2] + 1; n2 = b[5] - b[4] + 1; }
    else if (dir <= 4) { n1 = b[1] - b[0] + 1; n2 = b[5] - b[4] + 1; }
    else { n1 = b[1] - b[0] + 1; n2 = b[3] - b[2] + 1; }
}

// the forward program on the base, recording the tape (same arithmetic as k_bc)
template <typename Sync>
// member b, thread tid of nthr, sync(): a barrier over the nthr threads
__device__ __forceinline__ void k_bc_rec_run(int b, int tid, int nthr, Sync sync,
    BcProgram pg, StateSet q, double *Pbase, long long pstride, double *tape, long long tstride)
{
    double *F[5];
#pragma unroll
    for (int f = 0; f < 5; f++) F[f] = q.v[f] + b * q.bstride;
    double *P = Pbase + b * pstride;
    double *Rr = F[3], *Ee = F[4];
    double *tp = tape + b * tstride;
    double *H = pg.hold ? pg.hold + b * pg.hstride : nullptr;
    const double tnow = bc_time(pg);
    for (int o = 0; o < pg.nops; o++) {
        const BcOp op = pg.ops[o];
        if (op.code == OP_NEU || op.code == OP_P_NEU) {
            double *u = (op.code == OP_NEU) ? F[op.var] : P;
            neumann_face(pg, u, op.box, op.dir, op.len, op.coef ? pg.coef2 : pg.coef1, tid, nthr);
            sync();
            continue;
        }
        const int ni = op.box[1] - op.box[0] + 1, nj = op.box[3] - op.box[2] + 1, nk = op.box[5] - op.box[4] + 1;
        const long long total = (long long)ni * nj * nk;
        const int tw = bc_tape_width(op.code);
        for (long long q2 = tid; q2 < total; q2 += nthr) {
            const int i = op.box[0] + (int)(q2 % ni);
            const int j = op.box[2] + (int)((q2 / ni) % nj);
            const int k = op.box[4] + (int)(q2 / ((long long)ni * nj));
            const long long p = bidx(pg, i, j, k);
            double *t = tp + op.tape + tw * q2;
            switch (op.code) {
            case OP_SET: F[op.var][p] = op.val; break;
            case OP_DIR_P: t[0] = Ee[p]; Rr[p] = op.val / (pg.gamma - 1.0) / Ee[p]; break;
            case OP_P_LOAD: t[0] = Rr[p]; t[1] = Ee[p]; P[p] = Rr[p] * Ee[p]; break;
            case OP_R_FROM_P: t[0] = P[p]; t[1] = Ee[p]; Rr[p] = P[p] / Ee[p]; break;
            case OP_CORNER_E0: Ee[p] = 0.0; break;
            case OP_P_FROM_E: P[p] = Ee[p]; break;
            case OP_E_ADD_P: Ee[p] = Ee[p] + P[p]; break;
            case OP_E_DIV: Ee[p] = Ee[p] / (double)op.aux; break;
            case OP_R0: Rr[p] = 0.0; break;
            case OP_R_ADD_P: Rr[p] = Rr[p] + P[p]; break;
            case OP_R_DIV_E: t[0] = Rr[p]; t[1] = Ee[p]; Rr[p] = Rr[p] / Ee[p] / (double)op.aux; break;
            case OP_LID: {
                const double *x = pg.xs + op.xoff;
                const double sx = 2 * (x[i - op.box[0]] - x[0]) / (x[ni - 1] - x[0]) - 1;
                const double s2 = sx * sx, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
                const double pp = 1 - s16 * s2;
                F[op.var][p] = op.val * (pp * pp);
                break;
            }
            case OP_SINE: F[op.var][p] = bc_sine(F[op.var][p], pg.xs[op.xoff + i - op.box[0]], op.val, tnow); break;
            case OP_HOLD:  // the fields put back (the tangent and adjoint never run a first call)
                for (int v = 0; v < op.aux; v++) F[bc_hold_field(v)][p] = H[op.xoff + (long long)v * total + q2];
                break;
            default: break;
            }
        }
        sync();
    }
}

__global__ void k_bc_rec(
    BcProgram pg, StateSet q, double *Pbase, long long pstride, double *tape, long long tstride)
{
    k_bc_rec_run(blockIdx.x, threadIdx.x, blockDim.x, [] { __syncthreads(); }, pg, q, Pbase, pstride, tape, tstride);
}

__global__ void k_bc_rec_cluster(
    BcProgram pg, StateSet q, double *Pbase, long long pstride, double *tape, long long tstride)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    k_bc_rec_run(blockIdx.x / (int)cl.num_blocks(), (int)cl.block_rank() * blockDim.x + threadIdx.x, (int)cl.num_threads(),
           [&] { cl.sync(); }, pg, q, Pbase, pstride, tape, tstride);
}

// tangent: base q (updated as k_bc does) and tangent dq (P, dP scratch)
template <typename Sync>
// member b, thread tid of nthr, sync(): a barrier over the nthr threads
__device__ __forceinline__ void k_bc_tl_run(int b, int tid, int nthr, Sync sync,
    BcProgram pg, StateSet q, double *Pbase, StateSet dq, double *dPbase, long long pstride)
{
    double *F[5], *dF[5];
#pragma unroll
    for (int f = 0; f < 5; f++) { F[f] = q.v[f] + b * q.bstride; dF[f] = dq.v[f] + b * dq.bstride; }
    double *P = Pbase + b * pstride, *dP = dPbase + b * pstride;
    double *Rr = F[3], *Ee = F[4], *dR = dF[3], *dE = dF[4];
    double *H = pg.hold ? pg.hold + b * pg.hstride : nullptr;
    const double tnow = bc_time(pg);
    for (int o = 0; o < pg.nops; o++) {
        const BcOp op = pg.ops[o];
        if (op.code == OP_NEU || op.code == OP_P_NEU) {
            const double *cf = op.coef ? pg.coef2 : pg.coef1;
            neumann_face(pg, op.code == OP_NEU ? F[op.var] : P, op.box, op.dir, op.len, cf, tid, nthr);
            neumann_face(pg, op.code == OP_NEU ? dF[op.var] : dP, op.box, op.dir, op.len, cf, tid, nthr);
            sync();
            continue;
        }
        const int ni = op.box[1] - op.box[0] + 1, nj = op.box[3] - op.box[2] + 1, nk = op.box[5] - op.box[4] + 1;
        const long long total = (long long)ni * nj * nk;
        for (long long q2 = tid; q2 < total; q2 += nthr) {
            const int i = op.box[0] + (int)(q2 % ni);
            const int j = op.box[2] + (int)((q2 / ni) % nj);
            const int k = op.box[4] + (int)(q2 / ((long long)ni * nj));
            const long long p = bidx(pg, i, j, k);
            switch (op.code) {
            case OP_SET: F[op.var][p] = op.val; dF[op.var][p] = 0.0; break;
            case OP_DIR_P: {
                const double e = Ee[p], rn = op.val / (pg.gamma - 1.0) / e;
                dR[p] = -rn / e * dE[p];
                Rr[p] = rn;
                break;
            }
            case OP_P_LOAD: dP[p] = dR[p] * Ee[p] + Rr[p] * dE[p]; P[p] = Rr[p] * Ee[p]; break;
            case OP_R_FROM_P: {
                const double e = Ee[p], pv = P[p];
                dR[p] = dP[p] / e - pv * dE[p] / (e * e);
                Rr[p] = pv / e;
                break;
            }
            case OP_CORNER_E0: Ee[p] = 0.0; dE[p] = 0.0; break;
            case OP_P_FROM_E: P[p] = Ee[p]; dP[p] = dE[p]; break;
            case OP_E_ADD_P: Ee[p] = Ee[p] + P[p]; dE[p] = dE[p] + dP[p]; break;
            case OP_E_DIV: Ee[p] = Ee[p] / (double)op.aux; dE[p] = dE[p] / (double)op.aux; break;
            case OP_R0: Rr[p] = 0.0; dR[p] = 0.0; break;
            case OP_R_ADD_P: Rr[p] = Rr[p] + P[p]; dR[p] = dR[p] + dP[p]; break;
            case OP_R_DIV_E: {
                const double r = Rr[p], e = Ee[p], aux = (double)op.aux;
                dR[p] = dR[p] / e / aux - r * dE[p] / (e * e) / aux;
                Rr[p] = r / e / aux;
                break;
            }
            case OP_LID: {
                const double *x = pg.xs + op.xoff;
                const double sx = 2 * (x[i - op.box[0]] - x[0]) / (x[ni - 1] - x[0]) - 1;
                const double s2 = sx * sx, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
                const double pp = 1 - s16 * s2;
                F[op.var][p] = op.val * (pp * pp);
                dF[op.var][p] = 0.0;
                break;
            }
            // an additive forcing in time: the tangent passes through
            case OP_SINE: F[op.var][p] = bc_sine(F[op.var][p], pg.xs[op.xoff + i - op.box[0]], op.val, tnow); break;
            case OP_HOLD:  // held fields are constants
                for (int v = 0; v < op.aux; v++) {
                    F[bc_hold_field(v)][p] = H[op.xoff + (long long)v * total + q2];
                    dF[bc_hold_field(v)][p] = 0.0;
                }
                break;
            default: break;
            }
        }
        sync();
    }
}

__global__ void k_bc_tl(
    BcProgram pg, StateSet q, double *Pbase, StateSet dq, double *dPbase, long long pstride)
{
    k_bc_tl_run(blockIdx.x, threadIdx.x, blockDim.x, [] { __syncthreads(); }, pg, q, Pbase, dq, dPbase, pstride);
}

__global__ void k_bc_tl_cluster(
    BcProgram pg, StateSet q, double *Pbase, StateSet dq, double *dPbase, long long pstride)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    k_bc_tl_run(blockIdx.x / (int)cl.num_blocks(), (int)cl.block_rank() * blockDim.x + threadIdx.x, (int)cl.num_threads(),
           [&] { cl.sync(); }, pg, q, Pbase, dq, dPbase, pstride);
}

// adjoint of a Neumann face: g = lam[face]; lam[face] = 0; lam[face + m s] += c_{m-1} g
__device__ void neumann_face_adj(const BcProgram &pg, double *lam, const int *b, int dir, int len, const double *c,
                                 int tid, int nthr)
{
    int n1, n2;
    neumann_extent(b, dir, n1, n2);
    const long long total = (long long)n1 * n2;
    for (long long q = tid; q < total; q += nthr) {
        int i, j, k, di, dj, dk;
        neumann_geom(b, dir, len, q, n1, i, j, k, di, dj, dk);
        const long long pf = bidx(pg, i, j, k);
        const double g = lam[pf];
        lam[pf] = 0.0;
        for (int m = 1; m <= len; m++) lam[bidx(pg, i + m * di, j + m * dj, k + m * dk)] += c[m - 1] * g;
    }
}

// adjoint: lam (the five variables) and lP (the scratch's lambda, zero on entry), ops in reverse
template <typename Sync>
// member b, thread tid of nthr, sync(): a barrier over the nthr threads
__device__ __forceinline__ void k_bc_adj_run(int b, int tid, int nthr, Sync sync,
    BcProgram pg, StateSet lam, double *lPbase, long long pstride, const double *tape, long long tstride)
{
    double *L[5];
#pragma unroll
    for (int f = 0; f < 5; f++) L[f] = lam.v[f] + b * lam.bstride;
    double *lP = lPbase + b * pstride;
    double *lR = L[3], *lE = L[4];
    const double *tp = tape + b * tstride;
    for (int o = pg.nops - 1; o >= 0; o--) {
        const BcOp op = pg.ops[o];
        if (op.code == OP_NEU || op.code == OP_P_NEU) {
            neumann_face_adj(pg, op.code == OP_NEU ? L[op.var] : lP, op.box, op.dir, op.len,
                             op.coef ? pg.coef2 : pg.coef1, tid, nthr);
            sync();
            continue;
        }
        const int ni = op.box[1] - op.box[0] + 1, nj = op.box[3] - op.box[2] + 1, nk = op.box[5] - op.box[4] + 1;
        const long long total = (long long)ni * nj * nk;
        const int tw = bc_tape_width(op.code);
        for (long long q2 = tid; q2 < total; q2 += nthr) {
            const int i = op.box[0] + (int)(q2 % ni);
            const int j = op.box[2] + (int)((q2 / ni) % nj);
            const int k = op.box[4] + (int)(q2 / ((long long)ni * nj));
            const long long p = bidx(pg, i, j, k);
            const double *t = tp + op.tape + tw * q2;
            switch (op.code) {
            case OP_SET: L[op.var][p] = 0.0; break;
            case OP_DIR_P: {
                const double e = t[0], rn = op.val / (pg.gamma - 1.0) / e;
                lE[p] += -rn / e * lR[p];
                lR[p] = 0.0;
                break;
            }
            case OP_P_LOAD: lR[p] += t[1] * lP[p]; lE[p] += t[0] * lP[p]; lP[p] = 0.0; break;
            case OP_R_FROM_P: {
                const double pv = t[0], e = t[1];
                lP[p] += lR[p] / e;
                lE[p] += -pv / (e * e) * lR[p];
                lR[p] = 0.0;
                break;
            }
            case OP_CORNER_E0: lE[p] = 0.0; break;
            case OP_P_FROM_E: lE[p] += lP[p]; lP[p] = 0.0; break;
            case OP_E_ADD_P: lP[p] += lE[p]; break;
            case OP_E_DIV: lE[p] = lE[p] / (double)op.aux; break;
            case OP_R0: lR[p] = 0.0; break;
            case OP_R_ADD_P: lP[p] += lR[p]; break;
            case OP_R_DIV_E: {
                const double r = t[0], e = t[1], aux = (double)op.aux;
                lE[p] += -r / (e * e) / aux * lR[p];
                lR[p] = lR[p] / e / aux;
                break;
            }
            case OP_LID: L[op.var][p] = 0.0; break;
            case OP_SINE: break;
            case OP_HOLD:
                for (int v = 0; v < op.aux; v++) L[bc_hold_field(v)][p] = 0.0;
                break;
            default: break;
            }
        }
        sync();
    }
}

__global__ void k_bc_adj(
    BcProgram pg, StateSet lam, double *lPbase, long long pstride, const double *tape, long long tstride)
{
    k_bc_adj_run(blockIdx.x, threadIdx.x, blockDim.x, [] { __syncthreads(); }, pg, lam, lPbase, pstride, tape, tstride);
}

__global__ void k_bc_adj_cluster(
    BcProgram pg, StateSet lam, double *lPbase, long long pstride, const double *tape, long long tstride)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    k_bc_adj_run(blockIdx.x / (int)cl.num_blocks(), (int)cl.block_rank() * blockDim.x + threadIdx.x, (int)cl.num_threads(),
           [&] { cl.sync(); }, pg, lam, lPbase, pstride, tape, tstride);
}

}  // namespace gatt
