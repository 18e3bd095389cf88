// Compact line solves along x, y or z for sm_100a -- the B200 form of
// solveSystem{X,Y,Z}[per] (reference source/Fortran/derivs.F90:556-948).
//
// The reference solves every line with the precomputed Thomas factors of
// prepareThomas.m: a band product rhs = R*F, a forward recurrence
// y(i) = (rhs(i) - A y(i-1)) B and a backward recurrence x(i) = y(i) - C x(i+1); the cyclic
// variant first forms x(1) = D . rhs and then runs the same two recurrences on rows 2..N.
// Both recurrences are linear, so a line can be cut into P row blocks that run them
// concurrently from zero start values and are then recombined exactly:
//     y(i) = ytilde(i) + pi(i)  * y(start-1)     pi(i)  = prod_{k=start..i} (-A(k) B(k))
//     x(i) = xtilde(i) + rho(i) * x(end+1)       rho(i) = prod_{k=i..end}   (-C(k))
// where pi and rho depend only on the coefficients (precomputed per matrix type) and the
// block boundary values follow from a P-step prefix/suffix.  The recombination changes the
// floating-point order only for blocks after the first (forward) / before the last
// (backward); with P = 1 the kernel performs the reference's operations in its order.
//
// Mapping: one CTA = one tile of 32 lines and P warps; lane = line, warp = row block.
// The tile lives in shared memory as T[n][32] (row n, lane column): every per-row warp
// access is 32 consecutive doubles (conflict-free).
//  0. load: x-lines are contiguous, each lane reads 32-byte pieces of its own line;
//     y/z-lines are strided, each row is one 256-byte coalesced warp access.
//  1. halos to registers, then band product + forward recurrence of the block (in place)
//  2. (cyclic) x(1), the reduced forward recurrence
//  3. prefix of block boundary values, correction, backward recurrence (in place)
//  4. suffix, correction, store (optionally blended with the input: filter time relaxation)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gatt {

constexpr int kLanes = 32;   // lines per tile
constexpr int kMaxP = 16;    // largest number of row blocks per line
constexpr int kMaxPx = 25;   // row blocks of the pipelined x solver (wide form, 800 threads)
constexpr int kMaxPyz = 24;  // row blocks of the pipelined y/z solver (768 threads; 6-band: kMaxP)

enum SweepEpi { EPI_STORE = 0, EPI_BLEND = 1 };

// Division by a divisor fixed for a launch (the job decoding of the persistent solvers):
// floor(n / d) = (umulhi(n, m) + n) >> l for 0 <= n < 2^31, with l = ceil(log2 d) and
// m = floor(2^32 (2^l - d) / d) + 1 (Granlund and Montgomery, PLDI 1994) -- a multiply-high,
// an add and a shift instead of the twenty-odd instructions of a run-time integer division.
struct FastDiv {
    uint32_t d, m, l;
};
inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while ((1ull << l) < d) l++;
    f.l = l;
    f.m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
    return f;
}
__device__ __forceinline__ int fdiv(int n, const FastDiv &f)
{
    const uint32_t t = __umulhi((uint32_t)n, f.m);
    return (int)((t + (uint32_t)n) >> f.l);
}

// Per-row coefficient record, in the kernel's uniform row semantics:
//   forward  y(r) = (rhs(r) - fA(r) y(r-1)) * fB(r)
//   backward x(r) = y(r) - bC(r) x(r+1)
// plus the cyclic dot row D, the block propagators pi / rho, and (row 0 of a cyclic
// type) the corner couplings A(1) = LHS(1,N) and C(1) = LHS(N,1).
constexpr int kQ = 8;
// Pairs read together sit at even offsets: (fA, fB), (bC, pi), (cA, cC).
constexpr int kQfA = 0, kQfB = 1, kQbC = 2, kQpi = 3, kQD = 4, kQrho = 5, kQcA = 6, kQcC = 7;

struct SweepArgs {
    const double *in;        // base of the input field set
    double *out;             // base of the output field set
    long long in_bstride;    // elements between batch members (input)
    long long out_bstride;   // elements between batch members (output)
    long long npts;          // nx*ny*nz
    int in_slot[16];         // field slot (multiple of npts) per grid.y index
    int out_slot[16];
    int nx, ny, nz;
    int N;                   // line length
    int nlines;              // lines per field
    long long es;            // element stride along a strided line (y: nx, z: nx*ny)
    long long os;            // stride of the outer line index (y: nx*ny (k), z: nx (j))
    int tiles_per_row;       // strided: ceil(nx/32)
    const double *Rm;        // band coefficients [nTypes][N][Wp]
    const double *Q;         // row records [nTypes][N][kQ]
    int W;                   // 2*nR-1
    int Wp;                  // W padded to a multiple of 4
    const uint8_t *ltype;    // per-line matrix type (0-based)
    double blend;            // EPI_BLEND: out = in + blend*(solve - in) ...
    const double *blend_dt;  // ... or, when set, blend = *blend_dt / blend_fct (device dt)
    double blend_fct;
    int epi;                 // SweepEpi
    int P;                   // row blocks per line (1 .. kMaxP; kMaxPx for wide x lines); CTA = 32*P threads
    int stage;               // k_sweep: shared memory holds a coefficient copy (1) or not (0)
    // pipelined solver (k_psweep) only
    int dir;                 // 0 x, 1 y, 2 z
    int nf;                  // fields per launch
    int ntiles;              // tiles per field
    int njobs;               // ntiles * nf * members
    int ntypes;              // line types of the coefficient set
    int nst;                 // ring stages (1 .. kMaxStages)
    int Nreal;               // rows of a line that are stored (N, or fewer for padded lines)
    FastDiv fd_ntiles, fd_nf, fd_tpr;  // dividers by ntiles, nf and tiles_per_row
    // y and z lines in one launch (k_psweep, y/z form): parts = 2, part 1 the z lines.  The
    // jobs of one x-tile column run y then z, so the z tiles find their input in L2.
    int parts;               // 1, or 2
    int nout0, nout1;        // tiles per x-tile column of part 0 (y: nz) and part 1 (z: ny)
    FastDiv fd_nout;         // divider by nout0 + nout1
    int in_slot1[16], out_slot1[16];
    long long es1, os1;      // part 1's line and outer strides
    const double *Rm1, *Q1;  // part 1's coefficients
    const uint8_t *ltype1;
    int ntypes1;
    int box2;                // y/z lines past 256 rows: rows per tensor box (two boxes), else 0
    int tx_extra;            // bytes added to every copy barrier's expected count: 0, except in
                             // gatt_selftest_pipeline_timeout (its waits must run out)
    int *err;                // set to 1 when a pipeline wait gives up (host-mapped)
    // max-change epilogue (k_psweep, y/z form): the filter sweep that produces the step's final
    // state also reduces max |out - ref| per member and field into mc_acc[member * 5 + field
    // slot] (an unsigned 64-bit max on the IEEE bits, so a NaN wins); null: off
    // uniform band (k_psweep<..., UB = true>): every row of every line shares the band
    // coefficients band[0 .. W) (cyclic lines of one matrix type); the kernel reads them as
    // launch constants instead of per-row shared-memory records
    double band[16];
    double cac[2];           // uniform-band cyclic sets: the corner couplings (cA, cC) of row 0
    // x tiles field-inner and last tile first (xorder = 1): the launch's job cursor then runs
    // over (field, tile) instead of (tile, field) -- its "tiles" are the fields and its
    // "fields" the xtiles tiles -- so that each tile's fields are taken together, starting
    // from the points the preceding pointwise kernel wrote last (still in L2)
    int xorder, xtiles;
    int xchunk_store;        // x, two or more stages: one tensor store per warp (output box of 16 rows)
    unsigned long long *mc_acc;
    const double *mc_ref;    // the step's start state, field slots as in_slot
    long long mc_ref_bstride;
};

__device__ __forceinline__ double sweep_blend(const SweepArgs &a)
{
    return a.blend_dt ? *a.blend_dt / a.blend_fct : a.blend;
}

// Line data is read once per sweep: keep it out of L1 so the coefficient records stay there.
__device__ __forceinline__ void ld4_stream(const double *p, double *v)
{
    asm volatile("ld.global.L1::no_allocate.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}

__device__ __forceinline__ double ld_stream(const double *p)
{
    double v;
    asm volatile("ld.global.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ void st4(double *p, const double *v)
{
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
                 : "memory");
}

// First row of block p of a line of N rows cut into P blocks.
__host__ __device__ __forceinline__ int block_start(int p, int N, int P) { return (p * N) / P; }

__device__ __forceinline__ void ld4_coef(const double *p, double *v)
{
    asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}

// Rows per chunk of a recurrence pass: the chunk's coefficients are loaded before its
// dependent chain runs.
constexpr int kCh = 8;

// Shared memory of k_sweep, in doubles: the tile [N][32], the right halos of the row
// blocks [P][NR-1][32], the block-exchange values [3][P][32], then (stage) the coefficients
// of the tile's matrix type (band rows [N][Wp] and records [N][kQ]) when all its lines share
// one.  Long lines whose tile leaves no room for the coefficients read them through L1.
__host__ __device__ __forceinline__ size_t sweep_smem_doubles(int N, int P, int NR, int Wp, bool stage = true)
{
    return ((size_t)N + (size_t)P * (NR - 1) + 3 * (size_t)P) * kLanes + (stage ? (size_t)N * (Wp + kQ) : 0);
}

// BIG: instantiation for P > 4 (up to 32*kMaxP threads); otherwise at most 128 threads,
// which leaves the register allocator room for the chunk buffers.
template <bool XD, bool PER, int NR, bool BIG>
__global__ void __launch_bounds__(BIG ? 32 * kMaxP : 128) k_sweep(const SweepArgs a)
{
    constexpr int W = 2 * NR - 1;
    constexpr int NV = (W + 3) / 4;                          // 32-byte vectors per band row
    constexpr int RB = NR <= 4 ? 4 : (NR <= 7 ? 2 : 1);      // rows per chunk of the band pass
    extern __shared__ double T[];
    const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
    const int P = a.P;
    const int N = a.N;
    const int Wp = a.Wp;
    const double *F = a.in + (long long)blockIdx.z * a.in_bstride + (long long)a.in_slot[blockIdx.y] * a.npts;
    double *G = a.out + (long long)blockIdx.z * a.out_bstride + (long long)a.out_slot[blockIdx.y] * a.npts;
    long long base, s;
    int L;
    bool valid;
    if (XD) {
        L = blockIdx.x * kLanes + lane;
        valid = L < a.nlines;
        base = (long long)L * N;
        s = 1;
    } else {
        const int o = blockIdx.x / a.tiles_per_row;
        const int i = (blockIdx.x % a.tiles_per_row) * kLanes + lane;
        valid = i < a.nx;
        base = i + (long long)o * a.os;
        s = a.es;
        L = i + a.nx * o;
    }
    double *col = T + lane;
    double *halo = T + (size_t)N * kLanes + (size_t)p * (NR - 1) * kLanes + lane;   // this block's right halo
    double *xch = T + ((size_t)N + (size_t)P * (NR - 1)) * kLanes + lane;           // [3][P] (stride 32)
    const double *Fl = F + base;
    double *Gl = G + base;
    const bool vec = XD && (N % 4 == 0);

    // ---- 0. load the tile -------------------------------------------------------------
    if (valid) {
        if (vec) {
            // lane streams its own line in 32-byte pieces, 4 pieces in flight
            const int nj = N / 4;
            int j = p;
            for (; j + 3 * P < nj; j += 4 * P) {
                double v[4][4];
#pragma unroll
                for (int u = 0; u < 4; u++) ld4_stream(Fl + 4 * (j + u * P), v[u]);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    double *dst = col + 4 * (j + u * P) * kLanes;
                    dst[0] = v[u][0]; dst[kLanes] = v[u][1]; dst[2 * kLanes] = v[u][2]; dst[3 * kLanes] = v[u][3];
                }
            }
            for (; j < nj; j += P) {
                double v[4];
                ld4_stream(Fl + 4 * j, v);
                double *dst = col + 4 * j * kLanes;
                dst[0] = v[0]; dst[kLanes] = v[1]; dst[2 * kLanes] = v[2]; dst[3 * kLanes] = v[3];
            }
        } else {
            // one coalesced row per warp access, 16 rows in flight per lane
            const long long step = (long long)P * s;
            int n = p;
            for (; n + 15 * P < N; n += 16 * P) {
                double v[16];
                const double *src = Fl + (long long)n * s;
#pragma unroll
                for (int u = 0; u < 16; u++) v[u] = XD ? src[u * step] : ld_stream(src + u * step);
#pragma unroll
                for (int u = 0; u < 16; u++) col[(n + u * P) * kLanes] = v[u];
            }
            for (; n < N; n += P) col[n * kLanes] = XD ? Fl[n] : ld_stream(Fl + (long long)n * s);
        }
    }
    // coefficient staging: one copy of the tile's matrix type when every line shares it
    __shared__ int s_uniform;
    const int t = valid ? a.ltype[L] : -1;
    if (threadIdx.x < 32) {
        const int t0 = __shfl_sync(0xffffffffu, t, 0);
        const bool same = __all_sync(0xffffffffu, t == t0 || t < 0);
        if (lane == 0) s_uniform = same ? t0 : -1;
    }
    __syncthreads();
    const int tu = s_uniform;
    double *sR = T + ((size_t)N + (size_t)P * (NR - 1) + 3 * (size_t)P) * kLanes;
    double *sQ = sR + (size_t)N * Wp;
    const int sp = block_start(p, N, P), ep = block_start(p + 1, N, P) - 1;
    const double *Rm, *Q;
    if (tu >= 0 && a.stage) {
        // each warp copies the records of its own rows
        const double *gR = a.Rm + ((size_t)tu * N + sp) * Wp;
        const double *gQ = a.Q + ((size_t)tu * N + sp) * kQ;
        const int nR4 = (ep - sp + 1) * Wp / 4, nQ4 = (ep - sp + 1) * kQ / 4;
        for (int k = lane; k < nR4; k += kLanes) {
            double v[4];
            ld4_coef(gR + 4 * k, v);
            double *d = sR + (size_t)sp * Wp + 4 * k;
            d[0] = v[0]; d[1] = v[1]; d[2] = v[2]; d[3] = v[3];
        }
        for (int k = lane; k < nQ4; k += kLanes) {
            double v[4];
            ld4_coef(gQ + 4 * k, v);
            double *d = sQ + (size_t)sp * kQ + 4 * k;
            d[0] = v[0]; d[1] = v[1]; d[2] = v[2]; d[3] = v[3];
        }
        Rm = sR;
        Q = sQ;
        // other blocks' rows (cyclic corner terms in row 0, block-boundary propagators) are
        // read by every warp: wait for all warps' copies
        __syncthreads();
    } else {
        __syncthreads();
        Rm = a.Rm + (size_t)(t < 0 ? 0 : t) * N * Wp;
        Q = a.Q + (size_t)(t < 0 ? 0 : t) * N * kQ;
    }

    // ---- 1. halos, band product, forward recurrence ----------------------------------
    // window w = F(i-NR+1 .. i+NR-1).  Left halo -> registers, right halo -> the block's
    // shared halo rows; both are read before the barrier after which rows are overwritten.
    double w[W];
#pragma unroll
    for (int k = 0; k < NR - 1; k++) {
        int r = sp - (NR - 1) + k;
        r += r < 0 ? N : 0;
        w[k] = col[r * kLanes];
        int r2 = ep + 1 + k;
        r2 -= r2 >= N ? N : 0;
        const double hv = col[r2 * kLanes];
        __syncwarp();
        halo[k * kLanes] = hv;
    }
#pragma unroll
    for (int k = 0; k < NR; k++) w[NR - 1 + k] = col[(sp + k) * kLanes];
    __syncthreads();

    double yprev = 0.0, dot = 0.0;
    const double *rp = Rm + (size_t)sp * Wp;
    const double *qp = Q + (size_t)sp * kQ;
    double *cp = col + sp * kLanes;
    int i = sp;
    // full chunks: every incoming row i+NR is a row of this block (i + NR <= ep)
    const int nfull = (ep - NR + 1 - sp) / RB;
    for (int c = 0; c < nfull; c++) {
        double rc[RB][NV * 4], qc[RB][2], inc[RB];
#pragma unroll
        for (int u = 0; u < RB; u++) {
            const double2 *r2 = reinterpret_cast<const double2 *>(rp + u * Wp);
#pragma unroll
            for (int v = 0; v < NV * 2; v++) { const double2 x = r2[v]; rc[u][2 * v] = x.x; rc[u][2 * v + 1] = x.y; }
            if (!PER) {
                const double2 qa = *reinterpret_cast<const double2 *>(qp + u * kQ + kQfA);
                qc[u][kQfA] = qa.x; qc[u][kQfB] = qa.y;
            } else {
                qc[u][0] = qp[u * kQ + kQD];
            }
            inc[u] = cp[(u + NR) * kLanes];
        }
#pragma unroll
        for (int u = 0; u < RB; u++) {
            double acc = rc[u][NR - 1] * w[NR - 1];
#pragma unroll
            for (int l = 1; l < NR; l++) acc = acc + rc[u][NR - 1 + l] * w[NR - 1 + l] + rc[u][NR - 1 - l] * w[NR - 1 - l];
            if (!PER) {
                const double y = (acc - qc[u][kQfA] * yprev) * qc[u][kQfB];
                cp[u * kLanes] = y;
                yprev = y;
            } else {
                cp[u * kLanes] = acc;
                dot = (i + u == sp) ? acc * qc[u][0] : dot + acc * qc[u][0];
            }
#pragma unroll
            for (int k = 0; k < W - 1; k++) w[k] = w[k + 1];
            w[W - 1] = inc[u];
        }
        rp += RB * Wp; qp += RB * kQ; cp += RB * kLanes; i += RB;
    }
    // tail rows: the incoming row may come from the right halo
    for (; i <= ep; i++, rp += Wp, qp += kQ, cp += kLanes) {
        double rc[NV * 4], qc[2];
        {
            const double2 *r2 = reinterpret_cast<const double2 *>(rp);
#pragma unroll
            for (int v = 0; v < NV * 2; v++) { const double2 x = r2[v]; rc[2 * v] = x.x; rc[2 * v + 1] = x.y; }
            if (!PER) {
                const double2 qa = *reinterpret_cast<const double2 *>(qp + kQfA);
                qc[kQfA] = qa.x; qc[kQfB] = qa.y;
            } else {
                qc[0] = qp[kQD];
            }
        }
        const int r = i + NR;
        const double inc = r <= ep ? cp[NR * kLanes] : (r - ep - 1 < NR - 1 ? halo[(r - ep - 1) * kLanes] : 0.0);
        double acc = rc[NR - 1] * w[NR - 1];
#pragma unroll
        for (int l = 1; l < NR; l++) acc = acc + rc[NR - 1 + l] * w[NR - 1 + l] + rc[NR - 1 - l] * w[NR - 1 - l];
        if (!PER) {
            const double y = (acc - qc[kQfA] * yprev) * qc[kQfB];
            *cp = y;
            yprev = y;
        } else {
            *cp = acc;
            dot = (i == sp) ? acc * qc[0] : dot + acc * qc[0];
        }
#pragma unroll
        for (int k = 0; k < W - 1; k++) w[k] = w[k + 1];
        w[W - 1] = inc;
    }

    int r0 = sp;  // first row of this block in the recurrences (cyclic block 0 starts at row 1)
    if (PER) {
        xch[(2 * P + p) * kLanes] = dot;
        __syncthreads();
        // ---- 2. x(1) = D . rhs and the reduced forward recurrence (derivs.F90:786-799)
        double x1 = xch[(2 * P) * kLanes];
        for (int k = 1; k < P; k++) x1 = x1 + xch[(2 * P + k) * kLanes];
        if (p == 0) r0 = 1;
        const double cA = Q[kQcA], cC = Q[kQcC];
        // rows 1 and N-1 carry the corner terms (derivs.F90:792-793)
        if (r0 == 1) col[kLanes] = col[kLanes] - cA * x1;
        if (ep == N - 1) col[(N - 1) * kLanes] = col[(N - 1) * kLanes] - cC * x1;
        yprev = 0.0;
        const double *qq = Q + (size_t)r0 * kQ;
        double *cc = col + r0 * kLanes;
        int r = r0;
        for (; r + kCh - 1 <= ep; r += kCh, qq += kCh * kQ, cc += kCh * kLanes) {
            double qv[kCh][4], g[kCh];
#pragma unroll
            for (int u = 0; u < kCh; u++) {
                const double2 ab = *reinterpret_cast<const double2 *>(qq + u * kQ + kQfA);
                qv[u][kQfA] = ab.x;
                qv[u][kQfB] = ab.y;
                g[u] = cc[u * kLanes];
            }
#pragma unroll
            for (int u = 0; u < kCh; u++) {
                const double y = (g[u] - qv[u][kQfA] * yprev) * qv[u][kQfB];
                cc[u * kLanes] = y;
                yprev = y;
            }
        }
        for (; r <= ep; r++, qq += kQ, cc += kLanes) {
            const double y = (*cc - qq[kQfA] * yprev) * qq[kQfB];
            *cc = y;
            yprev = y;
        }
        if (p == 0) col[0] = x1;
    }
    xch[p * kLanes] = yprev;
    __syncthreads();

    // ---- 3. prefix, correction, backward recurrence ---------------------------------
    double Y = 0.0;
    for (int k = 0; k < p; k++) Y = xch[k * kLanes] + Q[(size_t)(block_start(k + 1, N, P) - 1) * kQ + kQpi] * Y;
    double xprev = 0.0;
    {
        const double *qq = Q + (size_t)ep * kQ;
        double *cc = col + ep * kLanes;
        int r = ep;
        for (; r - kCh + 1 >= r0; r -= kCh, qq -= kCh * kQ, cc -= kCh * kLanes) {
            double bc[kCh], pi[kCh], g[kCh];
#pragma unroll
            for (int u = 0; u < kCh; u++) {
                bc[u] = qq[-u * kQ + kQbC];
                pi[u] = qq[-u * kQ + kQpi];
                g[u] = cc[-u * kLanes];
            }
#pragma unroll
            for (int u = 0; u < kCh; u++) {
                const double y = g[u] + pi[u] * Y;  // Y = 0 in the first block
                const double x = y - bc[u] * xprev;
                cc[-u * kLanes] = x;
                xprev = x;
            }
        }
        for (; r >= r0; r--, qq -= kQ, cc -= kLanes) {
            const double y = *cc + qq[kQpi] * Y;
            const double x = y - qq[kQbC] * xprev;
            *cc = x;
            xprev = x;
        }
    }
    xch[(P + p) * kLanes] = xprev;
    __syncthreads();

    // ---- 4. suffix, correction, store --------------------------------------------------
    double X = 0.0;
    for (int k = P - 1; k > p; k--) X = xch[(P + k) * kLanes] + Q[(size_t)block_start(k, N, P) * kQ + kQrho] * X;
    if (!valid) return;
    const bool blend_on = a.epi == EPI_BLEND;
    const double blend = blend_on ? sweep_blend(a) : 0.0;
    const double *qq = Q + (size_t)sp * kQ + kQrho;  // X = 0 in the last block
    const double *cc = col + sp * kLanes;
    if (vec && (sp % 4 == 0) && ((ep + 1) % 4 == 0)) {
        for (int r = sp; r <= ep; r += 4, qq += 4 * kQ, cc += 4 * kLanes) {
            double v[4];
#pragma unroll
            for (int k = 0; k < 4; k++) v[k] = cc[k * kLanes] + qq[k * kQ] * X;
            if (PER && r == 0) v[0] = cc[0];  // x(1) is final
            if (blend_on) {
                double o[4];
                ld4_stream(Fl + r, o);
#pragma unroll
                for (int k = 0; k < 4; k++) v[k] = o[k] + blend * (v[k] - o[k]);
            }
            st4(Gl + r, v);
        }
    } else {
        double *gp = Gl + (long long)sp * s;
        const double *fp = Fl + (long long)sp * s;
#pragma unroll 4
        for (int r = sp; r <= ep; r++, qq += kQ, cc += kLanes, gp += s, fp += s) {
            double v = (PER && r == 0) ? *cc : *cc + (*qq) * X;
            if (blend_on) { const double o = *fp; v = o + blend * (v - o); }
            *gp = v;
        }
    }
}

// Fallback for lines too long for the shared tile (N > ~850) or band widths without an
// instantiation: one thread per line in the reference order, band product written to the
// output and the recurrences run in place there.  Requires in != out.
template <bool PER>
__global__ void k_sweep_global(const SweepArgs a, int nR)
{
    const int f = blockIdx.y, b = blockIdx.z;
    const int L = blockIdx.x * blockDim.x + threadIdx.x;
    if (L >= a.nlines) return;
    const int N = a.N;
    const double *__restrict__ F = a.in + (long long)b * a.in_bstride + (long long)a.in_slot[f] * a.npts;
    double *__restrict__ G = a.out + (long long)b * a.out_bstride + (long long)a.out_slot[f] * a.npts;
    long long base, s;
    if (a.es == 1) {  // x-lines
        base = (long long)L * N; s = 1;
    } else {
        const int i = L % a.nx, o = L / a.nx;
        base = i + (long long)o * a.os; s = a.es;
    }
    const int t = a.ltype[L];
    const double *Rt = a.Rm + (size_t)t * N * a.Wp;
    const double *Q = a.Q + (size_t)t * N * kQ;
    auto q = [&](int r, int fld) { return Q[(size_t)r * kQ + fld]; };
    for (int i = 0; i < N; i++) {
        const double *Ri = Rt + (size_t)i * a.Wp;
        double acc = Ri[nR - 1] * F[base + (long long)i * s];
        for (int l = 1; l < nR; l++) {
            int ip = i + l; ip -= (ip >= N) ? N : 0;
            int im = i - l; im += (im < 0) ? N : 0;
            acc = acc + Ri[nR - 1 + l] * F[base + (long long)ip * s] + Ri[nR - 1 - l] * F[base + (long long)im * s];
        }
        G[base + (long long)i * s] = acc;
    }
    double *g = G + base;
    int r0 = 0;
    if (PER) {
        double x1 = g[0] * q(0, kQD);
        for (int i = 1; i < N; i++) x1 = x1 + g[i * s] * q(i, kQD);
        g[0] = x1;
        g[s] = g[s] - q(0, kQcA) * x1;
        g[(N - 1) * s] = g[(N - 1) * s] - q(0, kQcC) * x1;
        r0 = 1;
    }
    double y = 0.0;
    for (int r = r0; r < N; r++) { y = (g[r * s] - q(r, kQfA) * y) * q(r, kQfB); g[r * s] = y; }
    double x = 0.0;
    for (int r = N - 1; r >= r0; r--) { x = g[r * s] - q(r, kQbC) * x; g[r * s] = x; }
    const double blend = a.epi == EPI_BLEND ? sweep_blend(a) : 0.0;
    if (blend > 0) {
        for (int i = 0; i < N; i++) {
            const double o = F[base + (long long)i * s];
            g[i * s] = o + blend * (g[i * s] - o);
        }
    }
}

}  // namespace gatt
