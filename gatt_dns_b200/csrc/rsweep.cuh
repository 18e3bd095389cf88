// Register-resident compact line solves for sm_100a: the fast forms of
// solveSystem{X,Y,Z}[per] (reference source/Fortran/derivs.F90:556-948) for lines whose
// length N is a multiple of the block height RPB (16 rows); k_psweep also takes non-cyclic
// y/z lines padded to such a length with identity rows (the host builds their records).
//
// Same algorithm and row records as k_sweep (sweep.cuh): band product, forward and backward
// Thomas recurrences, cut into P = N / RPB row blocks that run from zero start values and
// are recombined with the coefficient-only propagators pi / rho.  The difference is where
// the line lives: each thread keeps its RPB rows (plus NR-1 halo rows either side) in
// registers for the whole solve, and shared memory carries only the per-block boundary
// values (3*P*32 doubles).  Register slot k holds row p*RPB - (NR-1) + k before the band
// pass and row p*RPB + k after it; every register index is a compile-time constant.
//
// Two kernels feed the registers:
//  * k_rsweep: one tile per CTA, rows loaded straight from global memory (halo rows are
//    the neighbouring block's rows, L2 hits);
//  * k_psweep: persistent CTAs with a one- or two-stage shared-memory ring filled by the Tensor
//    Memory Accelerator -- one cp.async.bulk.tensor box {32 x N} per y/z tile (it lands
//    as [row][lane]) or one 128-byte-swizzled box per x tile (stored back the same way) --
//    so the next tile streams in while the current one is solved from registers and stored.
//    The coefficient records of all line types are copied to shared memory once per CTA.
//    Every mbarrier wait is bounded; a wait that gives up sets *err and the CTA returns.
#pragma once

#include <cuda.h>
#include "sweep.cuh"

namespace gatt {

// Largest band half-width + 1 the register kernels are instantiated for.
constexpr int kMaxNRreg = 7;
// Deepest shared-memory ring of k_psweep (the host picks 1 or 2 stages per launch).
constexpr int kMaxStages = 2;
// Longest mbarrier wait (ns) before a pipeline gives up.
constexpr unsigned long long kWaitNs = 1000000000ull;

// Shared memory of k_psweep in bytes: nst ring stages, the block exchange, the coefficient
// records of every line type (band rows [nTypes][N][Wp], records [nTypes][N][kQ]), the
// mbarriers.
__host__ __device__ __forceinline__ size_t psweep_stage_doubles(bool, int N) { return (size_t)N * kLanes; }
// cmp: the compact layout of the uniform-band x solver (records of kQc doubles, two exchange
// regions, no alignment slack: its shared window must start on the 1 KB swizzle period).
__host__ __device__ __forceinline__ size_t psweep_smem_bytes(bool xd, int N, int P, int ntypes, int Wp, int nst,
                                                            int ntypes1 = 0, bool cmp = false)
{
    return (nst * psweep_stage_doubles(xd, N) + (cmp ? 2 : 3) * (size_t)P * kLanes +
            (size_t)(ntypes + ntypes1) * N * (Wp + (cmp ? 6 : kQ))) *
               sizeof(double) +
           nst * 8 + (xd && !cmp ? 1024 : 0);  // x: room to align the ring to the 1 KB swizzle period
}

// Coefficient load: read-only data path (global records) or plain (shared-memory copy).
template <bool LDG, typename T>
__device__ __forceinline__ T ldc(const T *p)
{
    if constexpr (LDG) return __ldg(p);
    else return *p;
}

// ---- PTX helpers: mbarrier, bulk / tensor copies -----------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred q;\n mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n selp.u32 %0, 1, 0, q;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete; false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned long long limit_ns = kWaitNs)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

// 5-D tiled tensor load (no multicast) completing on an mbarrier.
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            int c4, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

// 5-D tiled tensor store shared -> global (bulk-group completion).
__device__ __forceinline__ void tma_store_5d(const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4, uint32_t src)
{
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(src)
                 : "memory");
}

// Contiguous global -> shared copy (16-byte aligned ends, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Contiguous shared -> global copy (bulk-group completion) and its group waits.
__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// ---- the solve of one row block from registers -------------------------------------------
// On entry w[k] = row p*RPB - (NR-1) + k of this thread's line; on return w[j] (j < RPB) =
// the solution at row p*RPB + j.  Every thread of the CTA calls it (three or four barriers).
// Rr: band rows of this block, Qt: the line type's row records, Qr = Qt + p*RPB records.
// CMP (compact shared memory, the uniform-band x solver): records of kQc doubles per row, the
// corner couplings (cA, cC) in cac[] (launch constants), two exchange regions of P x 32.
constexpr int kQc = 6;
template <bool PER, int NR, int RPB, bool LDG, bool UB = false, bool CMP = false>
__device__ __forceinline__ void solve_block(double (&w)[RPB + 2 * (NR - 1)], const double *Rr, const double *Qt,
                                            const double *Qr, double *xs, int lane, int p, int P,
                                            const double *band = nullptr, const double *cac = nullptr)
{
    constexpr int W = 2 * NR - 1;
    constexpr int H = NR - 1;
    constexpr int WP = (W + 3) / 4 * 4;
    constexpr int kQ = CMP ? kQc : ::gatt::kQ;  // record stride
    constexpr int DR = CMP ? 1 : 2;              // exchange region of the cyclic D-dot partials

    // ---- band product; forward recurrence (non-cyclic) or D-dot (cyclic) ----------------
    // row j's result goes to slot j: slot j is not read by rows after j.
    double yprev = 0.0, dot = 0.0;
#pragma unroll
    for (int j = 0; j < RPB; j++) {
        double rc[W + 1];
        if constexpr (UB) {
            // the same band on every row: launch constants (kernel parameter space)
#pragma unroll
            for (int v = 0; v < W; v++) rc[v] = band[v];
        } else {
            const double2 *r2 = reinterpret_cast<const double2 *>(Rr + j * WP);
#pragma unroll
            for (int v = 0; v < (W + 1) / 2; v++) {
                const double2 x = ldc<LDG>(r2 + v);
                rc[2 * v] = x.x;
                rc[2 * v + 1] = x.y;
            }
        }
        double acc = rc[NR - 1] * w[j + H];
#pragma unroll
        for (int l = 1; l < NR; l++) acc = acc + rc[NR - 1 + l] * w[j + H + l] + rc[NR - 1 - l] * w[j + H - l];
        if (!PER) {
            const double2 ab = ldc<LDG>(reinterpret_cast<const double2 *>(Qr + j * kQ + kQfA));
            const double y = (acc - ab.x * yprev) * ab.y;
            w[j] = y;
            yprev = y;
        } else {
            const double d = ldc<LDG>(Qr + j * kQ + kQD);
            dot = j == 0 ? acc * d : dot + acc * d;
            w[j] = acc;
        }
    }

    if (PER) {
        // ---- x(1) = D . rhs, corner terms, reduced forward recurrence (derivs.F90:786-799)
        // (the compact layout keeps the partials in the backward region: they are read before
        // the next barrier, and that region is written only after it)
        xs[(DR * P + p) * kLanes + lane] = dot;
        __syncthreads();
        double x1 = xs[(DR * P) * kLanes + lane];
        for (int k = 1; k < P; k++) x1 = x1 + xs[(DR * P + k) * kLanes + lane];
        double2 cc;  // row 0: (cA, cC)
        if constexpr (CMP) cc = make_double2(cac[0], cac[1]);
        else cc = ldc<LDG>(reinterpret_cast<const double2 *>(Qt + kQcA));
        yprev = 0.0;
#pragma unroll
        for (int j = 0; j < RPB; j++) {
            if (j == 0 && p == 0) continue;  // row 0 is x(1)
            double g = w[j];
            if (j == 1 && p == 0) g = g - cc.x * x1;
            if (j == RPB - 1 && p == P - 1) g = g - cc.y * x1;
            const double2 ab = ldc<LDG>(reinterpret_cast<const double2 *>(Qr + j * kQ + kQfA));
            const double y = (g - ab.x * yprev) * ab.y;
            w[j] = y;
            yprev = y;
        }
        if (p == 0) w[0] = x1;
    }
    xs[p * kLanes + lane] = yprev;
    __syncthreads();

    // ---- prefix of block-end values, correction, backward recurrence --------------------
    double Y = 0.0;
    for (int k = 0; k < p; k++) Y = xs[k * kLanes + lane] + ldc<LDG>(Qt + (size_t)((k + 1) * RPB - 1) * kQ + kQpi) * Y;
    double xprev = 0.0;
#pragma unroll
    for (int j = RPB - 1; j >= 0; j--) {
        if (PER && j == 0 && p == 0) break;  // x(1) is final
        const double2 cp = ldc<LDG>(reinterpret_cast<const double2 *>(Qr + j * kQ + kQbC));  // (bC, pi)
        const double y = w[j] + cp.y * Y;  // Y = 0 in the first block
        const double x = y - cp.x * xprev;
        w[j] = x;
        xprev = x;
    }
    xs[(P + p) * kLanes + lane] = xprev;
    __syncthreads();

    // ---- suffix of block-start values, correction ---------------------------------------
    double X = 0.0;
    for (int k = P - 1; k > p; k--) X = xs[(P + k) * kLanes + lane] + ldc<LDG>(Qt + (size_t)(k * RPB) * kQ + kQrho) * X;
#pragma unroll
    for (int j = 0; j < RPB; j++) {
        const double rho = ldc<LDG>(Qr + j * kQ + kQrho);
        w[j] = (PER && j == 0 && p == 0) ? w[0] : w[j] + rho * X;  // X = 0 in the last block
    }
}

// Line of a tile lane: start offset inside a field, element stride, line index.
struct LineRef {
    long long base, s;
    int L;
    bool valid;
};

template <bool XD>
__device__ __forceinline__ LineRef line_of(const SweepArgs &a, int tile, int lane)
{
    LineRef r;
    if (XD) {
        r.L = tile * kLanes + lane;
        r.valid = r.L < a.nlines;
        r.base = (long long)r.L * a.N;
        r.s = 1;
    } else {
        const int o = tile / a.tiles_per_row;
        const int i = (tile % a.tiles_per_row) * kLanes + lane;
        r.valid = i < a.nx;
        r.base = i + (long long)o * a.os;
        r.s = a.es;
        r.L = i + a.nx * o;
    }
    return r;
}

// Job j = tile + ntiles * (field + nf * member) of a persistent CTA, with the tile's outer
// index o and x-tile tx (y/z: tile = o * tiles_per_row + tx).  A CTA advances its job by the
// grid stride G; the stride is split the same way once, so that every later step is a few
// adds and compares instead of run-time integer divisions (about twenty instructions each).
struct JobCursor {
    int tile, f, b, o, tx, part;
};
struct JobStride {
    int gt, gf, gb, go, gx, nouter;
};
__device__ __forceinline__ JobCursor job_at(const SweepArgs &a, int j)
{
    JobCursor c;
    if (a.parts == 2) {
        // j = ((b * tiles_per_row + tx) * nf + f) * (nout0 + nout1) + r; r < nout0: y tile at
        // z = r, else z tile at y = r - nout0 -- x-tile column by column, all fields of one
        // column before the next
        const int g = fdiv(j, a.fd_nout);
        const int r = j - g * (a.nout0 + a.nout1);
        const int h = fdiv(g, a.fd_nf);
        c.f = g - h * a.nf;
        c.b = fdiv(h, a.fd_tpr);
        c.tx = h - c.b * a.tiles_per_row;
        c.part = r >= a.nout0;
        c.o = c.part ? r - a.nout0 : r;
        c.tile = c.o * a.tiles_per_row + c.tx;
        return c;
    }
    c.part = 0;
    const int fb = fdiv(j, a.fd_ntiles);
    c.tile = j - fb * a.ntiles;
    c.b = fdiv(fb, a.fd_nf);
    c.f = fb - c.b * a.nf;
    c.o = fdiv(c.tile, a.fd_tpr);
    c.tx = c.tile - c.o * a.tiles_per_row;
    return c;
}
__device__ __forceinline__ JobStride job_stride(const SweepArgs &a, int G)
{
    JobStride s;
    const int q = fdiv(G, a.fd_ntiles);
    s.gt = G - q * a.ntiles;
    s.gb = fdiv(q, a.fd_nf);
    s.gf = q - s.gb * a.nf;
    s.go = fdiv(s.gt, a.fd_tpr);
    s.gx = s.gt - s.go * a.tiles_per_row;
    s.nouter = fdiv(a.ntiles, a.fd_tpr);
    return s;
}
__device__ __forceinline__ void job_advance(JobCursor &c, const JobStride &s, const SweepArgs &a)
{
    c.tile += s.gt;
    c.o += s.go;
    c.tx += s.gx;
    if (c.tx >= a.tiles_per_row) { c.tx -= a.tiles_per_row; c.o++; }
    int carry = 0;
    if (c.tile >= a.ntiles) { c.tile -= a.ntiles; c.o -= s.nouter; carry = 1; }
    c.f += s.gf + carry;
    c.b += s.gb;
    if (c.f >= a.nf) { c.f -= a.nf; c.b++; }
    c.part = 0;
}

// The (tile, field) a cursor stands for: itself, or, for x tiles taken field-inner and last
// tile first (a.xorder), its fast index is the field and its slow index the reversed tile.
__device__ __forceinline__ JobCursor xjob(const SweepArgs &a, JobCursor c)
{
    if (a.xorder) {
        const int f = c.tile;
        c.tile = a.xtiles - 1 - c.f;
        c.f = f;
    }
    return c;
}

// Line of a tile lane from a cursor (line_of without divisions).
template <bool XD>
__device__ __forceinline__ LineRef line_at(const SweepArgs &a, const JobCursor &c, int lane)
{
    LineRef r;
    if (XD) {
        r.L = c.tile * kLanes + lane;
        r.valid = r.L < a.nlines;
        r.base = (long long)r.L * a.N;
        r.s = 1;
    } else {
        const int i = c.tx * kLanes + lane;
        r.valid = i < a.nx;
        r.base = i + (long long)c.o * (c.part ? a.os1 : a.os);
        r.s = c.part ? a.es1 : a.es;
        r.L = i + a.nx * c.o;
    }
    return r;
}

// Store the solved block (optionally blended with the input values `orig(j)`); with GUARD,
// y/z rows from nrows on (padding of non-cyclic lines) are not stored.
template <bool XD, int RPB, bool GUARD = false, typename Orig>
__device__ __forceinline__ void store_block(double *w, double *Gl, long long s, int sp, bool blend_on, double blend,
                                            Orig orig, int nrows)
{
    if (XD) {
#pragma unroll
        for (int q = 0; q < RPB / 4; q++) {
            double *v = &w[4 * q];
            if (blend_on) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const double o = orig(4 * q + k);
                    v[k] = o + blend * (v[k] - o);
                }
            }
            st4(Gl + sp + 4 * q, v);
        }
    } else {
#pragma unroll
        for (int j = 0; j < RPB; j++) {
            double v = w[j];
            if (blend_on) {
                const double o = orig(j);
                v = o + blend * (v - o);
            }
            if (!GUARD || sp + j < nrows) Gl[(long long)(sp + j) * s] = v;
        }
    }
}

// Halo row r of a line held at `ln` with element stride `st`: wraps for cyclic lines, zero
// outside a non-cyclic line (its band coefficients are zero there).
template <bool PER, typename Ld>
__device__ __forceinline__ double halo_row(int r, int N, Ld ld)
{
    if (PER) {
        r += r < 0 ? N : 0;
        r -= r >= N ? N : 0;
    } else if (r < 0 || r >= N) {
        return 0.0;
    }
    return ld(r);
}

// ---- one tile per CTA, rows from global memory ----------------------------------------
template <bool XD, bool PER, int NR, int RPB>
__global__ void __launch_bounds__(32 * kMaxP) k_rsweep(const SweepArgs a)
{
    constexpr int H = NR - 1;
    constexpr int WP = (2 * NR - 1 + 3) / 4 * 4;
    constexpr int NW = RPB + 2 * H;
    extern __shared__ __align__(16) double rxs[];  // [3][P][32]
    const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
    const int P = a.P;
    const int N = a.N;
    const int sp = p * RPB;
    const LineRef lr = line_of<XD>(a, blockIdx.x, lane);
    const double *Fl = a.in + (long long)blockIdx.z * a.in_bstride + (long long)a.in_slot[blockIdx.y] * a.npts + lr.base;
    double *Gl = a.out + (long long)blockIdx.z * a.out_bstride + (long long)a.out_slot[blockIdx.y] * a.npts + lr.base;
    const long long s = lr.s;
    const int t = lr.valid ? a.ltype[lr.L] : 0;
    const double *Qt = a.Q + (size_t)t * N * kQ;
    const double *Rr = a.Rm + ((size_t)t * N + sp) * WP;
    const double *Qr = Qt + (size_t)sp * kQ;

    auto ldg = [&](int r) { return ld_stream(Fl + (long long)r * s); };
    double w[NW];
    if (lr.valid) {
        if (XD) {
#pragma unroll
            for (int q = 0; q < RPB / 4; q++) ld4_stream(Fl + sp + 4 * q, &w[H + 4 * q]);
#pragma unroll
            for (int k = 0; k < H; k++) {
                w[k] = halo_row<PER>(sp - H + k, N, ldg);
                w[H + RPB + k] = halo_row<PER>(sp + RPB + k, N, ldg);
            }
        } else {
#pragma unroll
            for (int k = 0; k < NW; k++)
                w[k] = (k >= H && k < H + RPB) ? ldg(sp - H + k) : halo_row<PER>(sp - H + k, N, ldg);
        }
    } else {
#pragma unroll
        for (int k = 0; k < NW; k++) w[k] = 0.0;
    }
    solve_block<PER, NR, RPB, true>(w, Rr, Qt, Qr, rxs, lane, p, P);
    if (!lr.valid) return;
    const bool blend_on = a.epi == EPI_BLEND;
    const double blend = blend_on ? sweep_blend(a) : 0.0;
    store_block<XD, RPB>(w, Gl, s, sp, blend_on, blend, [&](int j) { return ldg(sp + j); }, N);
}

// ---- persistent CTAs, TMA-fed two-stage ring --------------------------------------------
// Job j = tile + ntiles * (field + nf * member); CTA b takes jobs b, b + G, b + 2G, ...
// y/z tiles: one tensor box {x: 32, line: N} of the 5-D map (x, y, z, field slot, member);
// x tiles: one tensor box {16 rows, 32 lines, N/16 row chunks} of the map (row in chunk, line,
// chunk, field slot, member) with the 128-byte swizzle -- it lands as [chunk][line][16 rows],
// the 16-byte pairs of rows of line L XOR-permuted by L % 8, so that a warp's 16-byte reads of
// its lines' row pairs are conflict-free -- and the solved tile leaves the same way through the
// output map (one tensor store; 32 line copies each way were bound by the number of copies).
// Register cap: the 768-thread bound holds a thread to 80 registers, which keeps three
// 256-thread CTAs resident (84 registers round up to two); the y/z 6-band filter spills at
// 80 and keeps the plain 512-thread bound.  WIDE (x lines of 25 row blocks, up to 400 points):
// an 800-thread bound, which holds a thread to 72 registers.
// UB: every row shares one band (a.band, launch constants; cyclic lines of one matrix type).
template <bool XD, bool PER, int NR, int RPB, bool WIDE = false, bool UB = false>
__global__ void __launch_bounds__(WIDE ? 32 * kMaxPx : ((NR == 6 && !XD) ? 32 * kMaxP : 768))
    k_psweep(const __grid_constant__ SweepArgs a, const __grid_constant__ CUtensorMap tmap,
             const __grid_constant__ CUtensorMap omap)
{
    constexpr int H = NR - 1;
    constexpr int WP = (2 * NR - 1 + 3) / 4 * 4;
    constexpr int NW = RPB + 2 * H;
    extern __shared__ __align__(128) double psm_raw[];
    const int lane = threadIdx.x & 31, p = threadIdx.x >> 5;
    const int P = a.P;
    const int N = a.N;
    const int sp = p * RPB;
    const size_t stage_d = psweep_stage_doubles(XD, N);
    const int nst = a.nst;
    // compact layout: the uniform-band x solver (records of kQc doubles, two exchange regions)
    constexpr bool CMP = UB && XD;
    constexpr int KQS = CMP ? kQc : kQ;
    // x: the swizzled ring starts on a 1 KB boundary (the host budgets the slack, except for
    // the compact layout, which needs the shared window itself to start there)
    const uint32_t pad = XD ? ((1024u - (smem_u32(psm_raw) & 1023u)) & 1023u) : 0u;
    if (CMP && pad) {
        if (threadIdx.x == 0) *(volatile int *)a.err = 2;
        return;
    }
    double *psm = psm_raw + pad / sizeof(double);
    double *xs = psm + nst * stage_d;
    constexpr int WPs = UB ? 0 : WP;                     // band rows in shared memory (none: UB)
    double *sRm = xs + (CMP ? 2 : 3) * P * kLanes;       // coefficient copy, all line types
    double *sQ = sRm + (size_t)a.ntypes * N * WPs;
    double *sRm1 = sQ + (size_t)a.ntypes * N * KQS;      // part 1 (z lines of a y+z launch)
    double *sQ1 = sRm1 + (size_t)(XD ? 0 : a.ntypes1) * N * WPs;
    const uint32_t st0 = smem_u32(psm);
    const uint32_t bar0 = smem_u32(sQ1 + (size_t)(XD ? 0 : a.ntypes1) * N * kQ);
    const int G = gridDim.x;
    if (st0 & 127u) {  // tensor copies need 128-byte aligned stages
        if (threadIdx.x == 0) *(volatile int *)a.err = 2;
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < nst; s++) mbar_init(bar0 + 8 * s, 1);
        fence_mbar_init();
    }
    __syncthreads();

    // thread 0: the copy of job c into stage s
    auto issue = [&](const JobCursor &c, int s) {
        const uint32_t bar = bar0 + 8 * s, dst = st0 + (uint32_t)(s * stage_d * sizeof(double));
        if (XD) {
            bulk_wait_read0();  // the tile stored out of this stage has been read
            fence_proxy_async();
            mbar_expect_tx(bar, (uint32_t)(N * kLanes * sizeof(double) + a.tx_extra));
            const JobCursor cx = xjob(a, c);
            tma_load_5d(dst, &tmap, 0, cx.tile * kLanes, 0, a.in_slot[cx.f], cx.b, bar);
        } else {
            fence_proxy_async();
            mbar_expect_tx(bar, (uint32_t)(N * kLanes * sizeof(double) + a.tx_extra));
            // part 1 of a y+z launch: z lines through the second map
            const bool ydir = a.dir == 1 && !c.part;
            const CUtensorMap *mp = c.part ? &omap : &tmap;
            const int slot = c.part ? a.in_slot1[c.f] : a.in_slot[c.f];
            tma_load_5d(dst, mp, c.tx * kLanes, ydir ? 0 : c.o, ydir ? c.o : 0, slot, c.b, bar);
            if (a.box2)  // second half of a line past one 256-row box
                tma_load_5d(dst + (uint32_t)(a.box2 * kLanes * sizeof(double)), mp, c.tx * kLanes,
                            ydir ? a.box2 : c.o, ydir ? c.o : a.box2, slot, c.b, bar);
        }
    };
    if (threadIdx.x == 0)
        for (int s = 0; s < nst; s++)
            if (blockIdx.x + s * G < a.njobs) issue(job_at(a, blockIdx.x + s * G), s);
    // the coefficient records are read by every tile: copy them once while the first tiles land
    {
        const int nR2 = UB ? 0 : a.ntypes * N * WP / 2, nQ2 = a.ntypes * N * KQS / 2;
        const double2 *gR = reinterpret_cast<const double2 *>(a.Rm);
        const double2 *gQ = reinterpret_cast<const double2 *>(a.Q);
        for (int i = threadIdx.x; i < nR2; i += blockDim.x) reinterpret_cast<double2 *>(sRm)[i] = __ldg(gR + i);
        for (int i = threadIdx.x; i < nQ2; i += blockDim.x) {
            // compact: the first kQc doubles of every kQ-double record
            const int gi = CMP ? (i / (kQc / 2)) * (kQ / 2) + i % (kQc / 2) : i;
            reinterpret_cast<double2 *>(sQ)[i] = __ldg(gQ + gi);
        }
        if (!XD && a.parts == 2) {
            const int mR2 = UB ? 0 : a.ntypes1 * N * WP / 2, mQ2 = a.ntypes1 * N * kQ / 2;
            const double2 *hR = reinterpret_cast<const double2 *>(a.Rm1);
            const double2 *hQ = reinterpret_cast<const double2 *>(a.Q1);
            for (int i = threadIdx.x; i < mR2; i += blockDim.x) reinterpret_cast<double2 *>(sRm1)[i] = __ldg(hR + i);
            for (int i = threadIdx.x; i < mQ2; i += blockDim.x) reinterpret_cast<double2 *>(sQ1)[i] = __ldg(hQ + i);
        }
    }
    __syncthreads();

    const bool blend_on = a.epi == EPI_BLEND;
    const double blend = blend_on ? sweep_blend(a) : 0.0;
    // cursors of this job and of the job nst strides ahead (the next copy into this stage):
    // advanced by adds where registers allow (x tiles, wide bands; measured 3-9 % faster
    // there), recomputed by division in the y/z narrow-band solvers, which sit at the
    // register cap and ran 5 % slower with two live cursors
    constexpr bool kIncr = XD || NR >= 6;
    const JobStride gs = job_stride(a, G);
    JobCursor cur = job_at(a, blockIdx.x), ahead = job_at(a, min(blockIdx.x + nst * G, a.njobs));
    int s = 0;
    uint32_t par = 0;
    // x with two or more stages: every warp stores its own 16-row chunk of the solved tile (no
    // block barrier before the store); the stage is refilled at the top of the next job, once
    // every warp's store has read it (the refill still lands a whole job ahead of its use)
    const bool wstore = XD && nst > 1 && a.xchunk_store;
    for (int j = blockIdx.x; j < a.njobs; j += G, s = (s + 1 == nst) ? 0 : s + 1, par ^= (s == 0) ? 1u : 0u) {
        if constexpr (kIncr) {
            if (j != (int)blockIdx.x) {
                job_advance(cur, gs, a);
                if (!wstore) job_advance(ahead, gs, a);
            }
        } else {
            cur = job_at(a, j);
            if (threadIdx.x == 0 && j + nst * G < a.njobs) ahead = job_at(a, j + nst * G);
        }
        const JobCursor cj = XD ? xjob(a, cur) : cur;
        const int tile = cj.tile, f = cj.f, b = cj.b;
        const bool p1 = !XD && cur.part;  // z lines of a y+z launch
        const LineRef lr = line_at<XD>(a, cj, lane);
        // one line type (every uniform-band set): no per-line type lookup
        const int t = (UB || !lr.valid) ? 0 : (p1 ? a.ltype1 : a.ltype)[lr.L];
        const double *Qt = (p1 ? sQ1 : sQ) + (size_t)t * N * KQS;
        const double *Rr = (p1 ? sRm1 : sRm) + ((size_t)t * N + sp) * WP;
        const double *Qr = Qt + (size_t)sp * KQS;
        const double *stg = psm + s * stage_d;
        const bool late = !mbar_wait(bar0 + 8 * s, par);

        // window rows from the stage
        double w[NW];
        // x: row r of this lane's line sits in chunk r/16, line row `lane`, 16-byte unit
        // (r%16)/2 XOR (lane%8); y/z: row r at [r][lane]
        auto xoff = [&](int r) {
            return (((r >> 4) * kLanes + lane) << 4) + (((((r & 15) >> 1) ^ (lane & 7))) << 1) + (r & 1);
        };
        auto lds = [&](int r) { return XD ? stg[xoff(r)] : stg[r * kLanes + lane]; };
        // x: the 16-byte unit of rows sp+2q, sp+2q+1 (sp is a multiple of 16: one chunk)
        const int xrow = ((sp >> 4) * kLanes + lane) << 4;
        auto xpair = [&](int q) { return xrow + ((q ^ (lane & 7)) << 1); };
        if (XD) {
#pragma unroll
            for (int q = 0; q < RPB / 2; q++) {
                const double2 v = *reinterpret_cast<const double2 *>(stg + xpair(q));
                w[H + 2 * q] = v.x;
                w[H + 2 * q + 1] = v.y;
            }
#pragma unroll
            for (int kk = 0; kk < H; kk++) {
                w[kk] = halo_row<PER>(sp - H + kk, N, lds);
                w[H + RPB + kk] = halo_row<PER>(sp + RPB + kk, N, lds);
            }
        } else {
#pragma unroll
            for (int kk = 0; kk < NW; kk++)
                w[kk] = (kk >= H && kk < H + RPB) ? lds(sp - H + kk) : halo_row<PER>(sp - H + kk, N, lds);
        }
        if (wstore && lane == 0) bulk_wait_read0();  // this warp's last store has read its stage
        if (__syncthreads_or(late)) {
            // give up: report, let the other stage's copy land (bounded; with warp stores its
            // refill has not been issued yet), leave
            if (threadIdx.x == 0) {
                *(volatile int *)a.err = 1;
                const int s1 = (s + 1 == nst) ? 0 : s + 1;
                if (nst > 1 && !wstore && j + G < a.njobs) mbar_wait(bar0 + 8 * s1, par ^ (s1 == 0 ? 1u : 0u));
            }
            if (XD && lane == 0) bulk_wait0();  // stores already issued
            __syncthreads();
            return;
        }
        if (wstore && j != (int)blockIdx.x) {
            // the previous job's stage: its next tile is job j - G + nst * G (the cursor `ahead`)
            if (threadIdx.x == 0 && j + (nst - 1) * G < a.njobs) issue(ahead, s == 0 ? nst - 1 : s - 1);
            job_advance(ahead, gs, a);
        }
        // y/z: every warp has its rows, refill this stage now (blend keeps it for the epilogue);
        // x: the stage also carries the results out, it is refilled after the stores
        if (!XD && !blend_on && threadIdx.x == 0 && j + nst * G < a.njobs) issue(ahead, s);

        solve_block<PER, NR, RPB, false, UB, CMP>(w, Rr, Qt, Qr, xs, lane, p, P, a.band, a.cac);
        if (XD) {
            // results back into the stage (own rows, same swizzled places), then one tensor
            // store of the tile (lines past the last one are clipped by the copy engine)
            double *sw = const_cast<double *>(stg);
#pragma unroll
            for (int q = 0; q < RPB / 2; q++) {
                double2 v = make_double2(w[2 * q], w[2 * q + 1]);
                if (blend_on) {
                    const double2 o = *reinterpret_cast<const double2 *>(sw + xpair(q));
                    v.x = o.x + blend * (v.x - o.x);
                    v.y = o.y + blend * (v.y - o.y);
                }
                *reinterpret_cast<double2 *>(sw + xpair(q)) = v;
            }
            fence_proxy_async();
            if (wstore) {
                // this warp's rows sp .. sp+15 are chunk p of the tile: 32 lines x 128 bytes
                static_assert(!XD || RPB == 16, "x warp stores take one 16-row chunk per warp");
                __syncwarp();
                if (lane == 0) {
                    tma_store_5d(&omap, 0, tile * kLanes, p, a.out_slot[f], b,
                                 st0 + (uint32_t)(s * stage_d * sizeof(double)) + (uint32_t)p * (kLanes * 128));
                    bulk_commit();
                }
            } else {
                __syncthreads();
                if (threadIdx.x == 0) {
                    tma_store_5d(&omap, 0, tile * kLanes, 0, a.out_slot[f], b,
                                 st0 + (uint32_t)(s * stage_d * sizeof(double)));
                    bulk_commit();
                }
                if (threadIdx.x == 0 && j + nst * G < a.njobs) issue(ahead, s);
            }
        } else {
            if (lr.valid) {
                double *Gl = a.out + (long long)b * a.out_bstride +
                             (long long)(p1 ? a.out_slot1[f] : a.out_slot[f]) * a.npts + lr.base;
                store_block<XD, RPB, !PER>(w, Gl, lr.s, sp, blend_on, blend, [&](int jj) { return lds(sp + jj); },
                                           a.Nreal);
            }
            if (a.mc_acc) {
                // max |stored value - step start| over this warp's rows of the tile (the stage
                // still holds the input: with the blend epilogue it is refilled only below)
                unsigned long long mx = 0;
                if (lr.valid) {
                    const double *ref = a.mc_ref + (long long)b * a.mc_ref_bstride + (long long)a.in_slot[f] * a.npts +
                                        lr.base;
#pragma unroll
                    for (int jj = 0; jj < RPB; jj++) {
                        if (!PER && sp + jj >= a.Nreal) continue;
                        double v = w[jj];
                        if (blend_on) {
                            const double o = lds(sp + jj);
                            v = o + blend * (v - o);
                        }
                        const unsigned long long u = (unsigned long long)__double_as_longlong(
                            fabs(v - ref[(long long)(sp + jj) * lr.s]));
                        mx = u > mx ? u : mx;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const unsigned long long u = __shfl_xor_sync(0xffffffffu, mx, o);
                    mx = u > mx ? u : mx;
                }
                if (lane == 0) atomicMax(a.mc_acc + b * 5 + a.in_slot[f], mx);
            }
            if (blend_on) {
                __syncthreads();
                if (threadIdx.x == 0 && j + nst * G < a.njobs) issue(ahead, s);
            }
        }
    }
    if (XD && lane == 0) bulk_wait0();  // every store has landed before the CTA leaves
}

}  // namespace gatt
