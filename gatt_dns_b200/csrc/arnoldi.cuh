// Device side of the Jacobian-free Arnoldi driver: the vector work of the Krylov loop of the
// reference's calcInstability.m:347-400 (first-order variant), for nbatch independent
// problems at once (one per batch member).
//
// A Krylov vector holds nv variables (U, V, W, R, E in 3-D; U, V, R, E in 2-D, the order
// of flow2vec, calcInstability.m:457-488) over every grid point; entries at points outside
// the flow region are zero, so sums over all points equal the reference's sums over
// region points.  Layout: zeta[b][j][v][p].
//
// Reductions are deterministic and independent of nbatch: a fixed grid of kRedBlocks
// blocks per member, each summing a fixed slice of points in a fixed tree order, then one
// thread summing the block partials in block order.  A member therefore gets bit-identical
// results whether it runs alone or in a batch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pointwise.cuh"

namespace gatt {

constexpr int kRedBlocks = 256;   // partial sums per member and vector
constexpr int kRedThreads = 256;
constexpr int kMaxKrylov = 512;   // largest Krylov dimension of one call

// state variable f (U, V, W, R, E) -> vector variable, -1 when not part of the vector
__device__ __forceinline__ int arn_var(int f, bool is3d) { return is3d ? f : (f == 2 ? -1 : (f < 2 ? f : f - 1)); }

// q = base + (zeta_k * eps) * sqrt(N) on region points, base elsewhere
// (calcInstability.m:353-362: disturbance = vec2flow(zeta(:,k)*epsilon*sqrt(N))).
__global__ void k_arn_perturb(StateSet q, const double *base, const double *zeta, long long zstride_b,
                              const uint8_t *region, double eps, double sqrtN, bool is3d, long long n)
{
    const int b = blockIdx.y;
    const double *z = zeta + b * zstride_b;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const bool in = region ? region[p] != 0 : true;
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const int v = arn_var(f, is3d);
            double x = base[f * n + p];
            if (v >= 0 && in) x = x + z[v * n + p] * eps * sqrtN;
            q.v[f][b * q.bstride + p] = x;
        }
    }
}

// B = (UP - UM) / (eps*sqrt(N)) on region points, 0 elsewhere (calcInstability.m:364-390)
__global__ void k_arn_diff(StateSet q, const double *um, double *B, long long bstride_b, int nv,
                           const uint8_t *region, double den, bool is3d, long long n)
{
    const int b = blockIdx.y;
    double *Bb = B + b * bstride_b;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const bool in = region ? region[p] != 0 : true;
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const int v = arn_var(f, is3d);
            if (v < 0) continue;
            Bb[v * n + p] = in ? (q.v[f][b * q.bstride + p] - um[f * n + p]) / den : 0.0;
        }
    }
}

// block tree sum of one value per thread (kRedThreads threads) -> thread 0
__device__ __forceinline__ double block_sum(double x, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        x = l < kRedThreads / 32 ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    }
    return x;
}

// Partial dot products zeta_j . B for j = 0..k (classical Gram-Schmidt uses the original B
// for every j, calcInstability.m:394-397).  Block x of member b covers a fixed slice.
// part[b][j][x]
__global__ void __launch_bounds__(kRedThreads) k_arn_dots(const double *zeta, long long zstride_b,
                                                          const double *B, long long bstride_b, int k,
                                                          long long len, double *part, int part_stride_b)
{
    __shared__ double sh[kRedThreads / 32];
    const int b = blockIdx.y;
    const double *Bb = B + b * bstride_b;
    const long long chunk = (len + kRedBlocks - 1) / kRedBlocks;
    const long long lo = blockIdx.x * chunk, hi = min(len, lo + chunk);
    for (int j = 0; j <= k; j++) {
        const double *z = zeta + b * zstride_b + (long long)j * len;
        double s = 0.0;
        for (long long i = lo + threadIdx.x; i < hi; i += kRedThreads) s += z[i] * Bb[i];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) part[(long long)b * part_stride_b + j * kRedBlocks + blockIdx.x] = s;
    }
}

// Sum the partials of nvec vectors in block order: h[b][j] = sum_x part[b][j][x]
__global__ void k_arn_sum(const double *part, int part_stride_b, int nvec, double *h, int h_stride_b, bool take_sqrt)
{
    const int b = blockIdx.x, j = threadIdx.x;
    if (j >= nvec) return;
    const double *pp = part + (long long)b * part_stride_b + j * kRedBlocks;
    double s = 0.0;
    for (int x = 0; x < kRedBlocks; x++) s += pp[x];
    h[b * h_stride_b + j] = take_sqrt ? sqrt(s) : s;
}

// uPrime = B - sum_{j<=k} H(j,k) zeta_j (in j order, calcInstability.m:396), written to the
// next basis slot, with partial sums of uPrime^2 for its norm.
__global__ void __launch_bounds__(kRedThreads) k_arn_orth(double *zeta, long long zstride_b, const double *B,
                                                          long long bstride_b, const double *hcol, int h_stride_b,
                                                          int k, long long len, double *part, int part_stride_b)
{
    __shared__ double sh[kRedThreads / 32];
    const int b = blockIdx.y;
    const double *Bb = B + b * bstride_b;
    double *zb = zeta + b * zstride_b;
    double *out = zb + (long long)(k + 1) * len;
    const double *hb = hcol + b * h_stride_b;
    const long long chunk = (len + kRedBlocks - 1) / kRedBlocks;
    const long long lo = blockIdx.x * chunk, hi = min(len, lo + chunk);
    double s = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += kRedThreads) {
        double u = Bb[i];
        for (int j = 0; j <= k; j++) u = u - hb[j] * zb[(long long)j * len + i];
        out[i] = u;
        s += u * u;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[(long long)b * part_stride_b + blockIdx.x] = s;
}

// zeta_{k+1} = uPrime / H(k+1,k) (calcInstability.m:400); a zero norm leaves zeros.
__global__ void k_arn_scale(double *zeta, long long zstride_b, const double *hnorm, int h_stride_b, int k1,
                            long long len)
{
    const int b = blockIdx.y;
    double *z = zeta + b * zstride_b + (long long)k1 * len;
    const double h = hnorm[b * h_stride_b];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
        z[i] = h != 0.0 ? z[i] / h : 0.0;
}

}  // namespace gatt
