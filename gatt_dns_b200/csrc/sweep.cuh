// Compact line solves along x, y or z for sm_100a -- the B200 form of
// solveSystem{X,Y,Z}[per] (reference source/Fortran/derivs.F90:556-948).
//
// Layout: fields are FP64, i fastest.  One warp owns a tile of 32 lines; the tile is
// staged in shared memory as T[n][33] (row n = position along the line, column = line,
// one double of padding so both the strided-line load and the per-line solve are free
// of bank conflicts).  Each lane then runs the reference Thomas recurrence on its own
// line in place -- one thread per line keeps the reference's operation order, so the
// result matches the Fortran to rounding.  y- and z-lines are loaded with the warp
// reading 32 neighbouring lines at one position (256 contiguous bytes); x-lines are
// contiguous, so the warp reads along a line and transposes through the padded tile.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gatt {

constexpr int kTileLines = 32;
constexpr int kPad = 33;  // row pitch of the shared tile, in doubles
constexpr int kChunk = 16;  // loads each lane keeps in flight while staging a tile

enum SweepEpi { EPI_STORE = 0, EPI_BLEND = 1 };

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
    const double *R;         // [nTypes][N][W]
    const double *A, *B, *C, *D;  // [nTypes][N]
    int W;                   // 2*nR-1
    const uint8_t *ltype;    // per-line matrix type (0-based)
    double blend;            // EPI_BLEND: out = in + blend*(solve - in) ...
    const double *blend_dt;  // ... or, when set, blend = *blend_dt / blend_fct (device dt)
    double blend_fct;
};

__device__ __forceinline__ double sweep_blend(const SweepArgs &a)
{
    return a.blend_dt ? *a.blend_dt / a.blend_fct : a.blend;
}

// Solve the line held in column `col` (stride kPad) in place.
// Rows N .. N+NR-2 of the column hold copies of rows 0 .. NR-2 (the periodic wrap of
// the band product).  Non-periodic: derivs.F90:583-611; periodic: derivs.F90:764-802.
template <bool PER, int NR>
__device__ __forceinline__ void solve_column(double *__restrict__ col, int N,
                                             const double *__restrict__ Rt,
                                             const double *__restrict__ At,
                                             const double *__restrict__ Bt,
                                             const double *__restrict__ Ct,
                                             const double *__restrict__ Dt)
{
    constexpr int W = 2 * NR - 1;
    double w[W];
    // window holds F[i-(NR-1) .. i+(NR-1)] (indices modulo N)
#pragma unroll
    for (int q = 0; q < W; q++) {
        int idx = q - (NR - 1);
        idx = idx < 0 ? idx + N : idx;
        w[q] = col[idx * kPad];
    }
    double dprev = 0.0, x1 = 0.0;
    for (int i = 0; i < N; i++) {
        const double *Ri = Rt + (size_t)i * W;
        double acc = __ldg(Ri + NR - 1) * w[NR - 1];
#pragma unroll
        for (int l = 1; l < NR; l++)
            acc = acc + __ldg(Ri + NR - 1 + l) * w[NR - 1 + l] + __ldg(Ri + NR - 1 - l) * w[NR - 1 - l];
        if (!PER) {
            const double d = (i == 0) ? acc * __ldg(Bt) : (acc - __ldg(At + i - 1) * dprev) * __ldg(Bt + i);
            col[i * kPad] = d;
            dprev = d;
        } else {
            col[i * kPad] = acc;
            x1 = (i == 0) ? acc * __ldg(Dt) : x1 + acc * __ldg(Dt + i);
        }
#pragma unroll
        for (int q = 0; q < W - 1; q++) w[q] = w[q + 1];
        if (i + 1 < N) w[W - 1] = col[(i + NR) * kPad];
    }
    if (!PER) {
        double dn = col[(N - 1) * kPad];
        for (int i = N - 2; i >= 0; i--) {
            const double d = col[i * kPad] - __ldg(Ct + i) * dn;
            col[i * kPad] = d;
            dn = d;
        }
    } else {
        col[0] = x1;
        double d = (col[kPad] - __ldg(At) * x1) * __ldg(Bt);
        col[(N - 1) * kPad] = col[(N - 1) * kPad] - __ldg(Ct) * x1;
        col[kPad] = d;
        for (int i = 1; i < N - 1; i++) {
            d = (col[(i + 1) * kPad] - __ldg(At + i) * d) * __ldg(Bt + i);
            col[(i + 1) * kPad] = d;
        }
        double dn = col[(N - 1) * kPad];
        for (int i = N - 2; i >= 1; i--) {
            const double e = col[i * kPad] - __ldg(Ct + i) * dn;
            col[i * kPad] = e;
            dn = e;
        }
    }
}

// One warp per CTA; grid = (tiles, fields, batch).  Dynamic shared memory:
// (N + NR) * kPad doubles.
template <bool XD, bool PER, int NR, int EPI>
__global__ void __launch_bounds__(32) k_sweep(const SweepArgs a)
{
    extern __shared__ double T[];
    const int lane = threadIdx.x;
    const int f = blockIdx.y, b = blockIdx.z;
    const int N = a.N;
    const double *__restrict__ F = a.in + (long long)b * a.in_bstride + (long long)a.in_slot[f] * a.npts;
    double *G = a.out + (long long)b * a.out_bstride + (long long)a.out_slot[f] * a.npts;

    long long base;
    int nvalid, L0;
    if (XD) {
        // the tile's 32 x-lines are one contiguous run of nvalid*N doubles
        L0 = blockIdx.x * kTileLines;
        nvalid = min(kTileLines, a.nlines - L0);
        base = (long long)L0 * N;
        const double *__restrict__ src = F + base;
        const int total = nvalid * N;
        int l = 0, n = lane;
        while (n >= N) { n -= N; l++; }
        for (int i0 = 0; i0 < total; i0 += 32 * kChunk) {
            double v[kChunk];
#pragma unroll
            for (int u = 0; u < kChunk; u++) {
                const int idx = i0 + u * 32 + lane;
                v[u] = idx < total ? src[idx] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kChunk; u++) {
                if (i0 + u * 32 + lane < total) T[n * kPad + l] = v[u];
                n += 32;
                while (n >= N) { n -= N; l++; }
            }
        }
    } else {
        const int o = blockIdx.x / a.tiles_per_row;
        const int i0 = (blockIdx.x % a.tiles_per_row) * kTileLines;
        nvalid = min(kTileLines, a.nx - i0);
        base = i0 + (long long)o * a.os;
        L0 = i0 + a.nx * o;
        if (lane < nvalid) {
            const double *__restrict__ src = F + base + lane;
            for (int n0 = 0; n0 < N; n0 += kChunk) {
                double v[kChunk];
#pragma unroll
                for (int u = 0; u < kChunk; u++) v[u] = (n0 + u < N) ? src[(long long)(n0 + u) * a.es] : 0.0;
#pragma unroll
                for (int u = 0; u < kChunk; u++)
                    if (n0 + u < N) T[(n0 + u) * kPad + lane] = v[u];
            }
        }
    }
    __syncwarp();
    if (lane < nvalid) {
        double *col = T + lane;
        // wrap rows for the band product
#pragma unroll
        for (int q = 0; q < NR - 1; q++) col[(N + q) * kPad] = col[q * kPad];
        const int t = a.ltype[L0 + lane];
        const size_t co = (size_t)t * N;
        solve_column<PER, NR>(col, N, a.R + co * a.W, a.A + co, a.B + co, a.C + co, PER ? a.D + co : nullptr);
    }
    __syncwarp();
    const double blend = (EPI == EPI_BLEND) ? sweep_blend(a) : 0.0;
    if (XD) {
        double *dst = G + base;
        const double *src = F + base;
        const int total = nvalid * N;
        int l = 0, n = lane;
        while (n >= N) { n -= N; l++; }
        for (int idx = lane; idx < total; idx += 32) {
            double v = T[n * kPad + l];
            if (EPI == EPI_BLEND) { const double o = src[idx]; v = o + blend * (v - o); }
            dst[idx] = v;
            n += 32;
            while (n >= N) { n -= N; l++; }
        }
    } else if (lane < nvalid) {
        double *dst = G + base + lane;
        const double *src = F + base + lane;
#pragma unroll 8
        for (int n = 0; n < N; n++) {
            double v = T[n * kPad + lane];
            if (EPI == EPI_BLEND) { const double o = src[(long long)n * a.es]; v = o + blend * (v - o); }
            dst[(long long)n * a.es] = v;
        }
    }
}

// Fallback for lines too long for the shared tile: one thread per line, band product
// written straight to the output and the Thomas recurrences run in place there.
// Requires in != out.
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
    const double *Rt = a.R + (size_t)t * N * a.W;
    const double *At = a.A + (size_t)t * N, *Bt = a.B + (size_t)t * N, *Ct = a.C + (size_t)t * N;
    for (int i = 0; i < N; i++) {
        const double *Ri = Rt + (size_t)i * a.W;
        double acc = Ri[nR - 1] * F[base + (long long)i * s];
        for (int l = 1; l < nR; l++) {
            int ip = i + l; ip -= (ip >= N) ? N : 0;
            int im = i - l; im += (im < 0) ? N : 0;
            acc = acc + Ri[nR - 1 + l] * F[base + (long long)ip * s] + Ri[nR - 1 - l] * F[base + (long long)im * s];
        }
        G[base + (long long)i * s] = acc;
    }
    double *g = G + base;
    if (!PER) {
        double d = g[0] * Bt[0];
        g[0] = d;
        for (int i = 0; i < N - 1; i++) { d = (g[(i + 1) * s] - At[i] * d) * Bt[i + 1]; g[(i + 1) * s] = d; }
        for (int i = N - 2; i >= 0; i--) { d = g[i * s] - Ct[i] * d; g[i * s] = d; }
    } else {
        const double *Dt = a.D + (size_t)t * N;
        double x1 = g[0] * Dt[0];
        for (int i = 1; i < N; i++) x1 = x1 + g[i * s] * Dt[i];
        g[0] = x1;
        double d = (g[s] - At[0] * x1) * Bt[0];
        g[(N - 1) * s] = g[(N - 1) * s] - Ct[0] * x1;
        g[s] = d;
        for (int i = 1; i < N - 1; i++) { d = (g[(i + 1) * s] - At[i] * d) * Bt[i]; g[(i + 1) * s] = d; }
        d = g[(N - 1) * s];
        for (int i = N - 2; i >= 1; i--) { d = g[i * s] - Ct[i] * d; g[i * s] = d; }
    }
    const double blend = sweep_blend(a);
    if (blend > 0) {
        for (int i = 0; i < N; i++) {
            const double o = F[base + (long long)i * s];
            g[i * s] = o + blend * (g[i * s] - o);
        }
    }
}

}  // namespace gatt
