// Pointwise kernels of the Navier-Stokes right-hand side, the RK4 stage update, SFD
// and the max-change residual (reference source/Fortran/nseq.F90:10-323,
// timeIntegration.F90:8-156/338-498, main.F90:381-420).
//
// Field sets are [member][slot][point] arrays of FP64; every kernel is a grid-stride
// loop over points with the batch member in blockIdx.y.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gatt {

// slot numbering of the per-member scratch sets
// 3-D first derivatives: slot 3*f + d, f in U,V,W,R,E and d in x,y,z
enum { D3_UX = 0, D3_UY, D3_UZ, D3_VX, D3_VY, D3_VZ, D3_WX, D3_WY, D3_WZ,
       D3_RX, D3_RY, D3_RZ, D3_EX, D3_EY, D3_EZ, D3_N };
// 3-D stresses and heat fluxes
enum { T3_XX = 0, T3_YY, T3_ZZ, T3_XY, T3_XZ, T3_YZ, T3_QX, T3_QY, T3_QZ, T3_N };
// 3-D second-sweep results
enum { S3_TXYX = 0, S3_TXYY, S3_TXZX, S3_TXZZ, S3_TYZY, S3_TYZZ, S3_TXXX, S3_TYYY, S3_TZZZ,
       S3_HTX, S3_HTY, S3_HTZ, S3_N };
// 2-D first derivatives: slot 2*f + d, f in U,V,R,E
enum { D2_UX = 0, D2_UY, D2_VX, D2_VY, D2_RX, D2_RY, D2_EX, D2_EY, D2_N };
enum { T2_XX = 0, T2_YY, T2_XY, T2_QX, T2_QY, T2_N };
enum { S2_TXYX = 0, S2_TXYY, S2_TXXX, S2_TYYY, S2_HTX, S2_HTY, S2_N };

struct Phys {
    double Re, Ma, Pr, gamma, T0;
};

// Device-resident per-step parameters, written by one small copy before each step so
// that a captured graph replays with new values.
struct StepParams {
    double t, dt;
    long long slot;   // row of the max-change history to fill
};

// RK4 stage modes for the assembly epilogue (timeIntegration.F90:380-487)
// RK_EULER: the one stage of EULER_2D/3D; SSP_STAGE1..3: SSPRK3_2D/3D (timeIntegration.F90).
enum { RK_STORE_RHS = 0, RK_STAGE1 = 1, RK_STAGE2 = 2, RK_STAGE3 = 3, RK_STAGE4 = 4, RK_EULER = 5,
       SSP_STAGE1 = 6, SSP_STAGE2 = 7, SSP_STAGE3 = 8 };

// ---- forcings (runForcings2D/3D.F90: disturbances with forcing = true) ---------------------
// Applied to the right-hand side nseq forms, in order, on 0-based inclusive boxes:
// FORCE_PRESSURE_GRADIENT (pressureGradient.F90): du = du + dpdx/r; FORCE_TURBULENCE
// (turbulenceGenerator.F90, one rank): with the box sums ET = sum(u u + v v + w w), U..E of
// the right-hand side's input state and N points, du = du + 0.25*eps*N/ET*u - gamma*Usum/N
// (gamma = 10 eps, likewise v, w) and de = de - gamma*(Esum/N - e0).
constexpr int kMaxForcings = 4;
enum { FORCE_PRESSURE_GRADIENT = 1, FORCE_TURBULENCE = 2 };
struct Forcings {
    int n;
    int type[kMaxForcings];
    int box[kMaxForcings][6];
    double par[kMaxForcings][2];
    double N[kMaxForcings];   // points of each box
    const double *sums;       // [member][kMaxForcings][5]: ET, U, V, W, E sums (turbulence)
    int nx, ny;
};

// k[] in U, V, W, R, E order; mom / en: apply the momentum (U, V, W) / energy rows only.
__device__ __forceinline__ void apply_forcings(const Forcings &fs, int b, long long p, double u, double v,
                                               double w, double r, double e, double k[5], bool mom, bool en)
{
    const int i = (int)(p % fs.nx);
    const long long jk = p / fs.nx;
    const int j = (int)(jk % fs.ny), kz = (int)(jk / fs.ny);
    for (int f = 0; f < fs.n; f++) {
        const int *bx = fs.box[f];
        if (i < bx[0] || i > bx[1] || j < bx[2] || j > bx[3] || kz < bx[4] || kz > bx[5]) continue;
        if (fs.type[f] == FORCE_PRESSURE_GRADIENT) {
            if (mom) k[0] = k[0] + fs.par[f][0] / r;
        } else if (fs.type[f] == FORCE_TURBULENCE) {
            const double *S = fs.sums + ((size_t)b * kMaxForcings + f) * 5;
            const double eps = fs.par[f][0], e0 = fs.par[f][1], gamma = 10 * eps, N = fs.N[f];
            if (mom) {
                k[0] = k[0] + 0.25 * eps * N / S[0] * u - gamma * S[1] / N;
                k[1] = k[1] + 0.25 * eps * N / S[0] * v - gamma * S[2] / N;
                k[2] = k[2] + 0.25 * eps * N / S[0] * w - gamma * S[3] / N;
            }
            if (en) k[4] = k[4] - gamma * (S[4] / N - e0);
        }
    }
}

// Whether a stage update reads / writes the increment accumulator delta.
__host__ __device__ __forceinline__ bool mode_reads_delta(int m)
{
    return m == RK_STAGE2 || m == RK_STAGE3 || m == RK_STAGE4 || m == SSP_STAGE2 || m == SSP_STAGE3;
}
__host__ __device__ __forceinline__ bool mode_writes_delta(int m)
{
    return m == RK_STAGE1 || m == RK_STAGE2 || m == RK_STAGE3 || m == SSP_STAGE1 || m == SSP_STAGE2;
}

struct FieldSet {
    double *p;            // base
    long long bstride;    // elements between members
    long long npts;
    __device__ __forceinline__ double *f(int b, int slot) const { return p + b * bstride + slot * npts; }
};

// Pointers of the five state variables of one set (U, V, W, R, E); separate pointers
// because in 2-D the W of a stage is a different array than U/V/R/E.
struct StateSet {
    double *v[5];
    long long bstride;
};

// Box sums of every turbulence forcing: each CTA (blockIdx.x of gridDim.x, member
// blockIdx.y) sums its grid-stride share of the box points in a fixed order into
// part[((b * kMaxForcings + f) * gridDim.x + cta) * 5 + q]; k_forcing_final adds the CTAs'
// partials in CTA order, so the sums do not depend on timing.
__global__ void __launch_bounds__(256) k_forcing_sums(StateSet q, Forcings fs, double *part)
{
    __shared__ double red[5][256];
    const int b = blockIdx.y;
    const double *U = q.v[0] + b * q.bstride, *V = q.v[1] + b * q.bstride, *W = q.v[2] + b * q.bstride;
    const double *E = q.v[4] + b * q.bstride;
    for (int f = 0; f < fs.n; f++) {
        if (fs.type[f] != FORCE_TURBULENCE) continue;
        const int *bx = fs.box[f];
        const long long ni = bx[1] - bx[0] + 1, nj = bx[3] - bx[2] + 1, nk = bx[5] - bx[4] + 1;
        const long long m = ni * nj * nk;
        double s[5] = {0, 0, 0, 0, 0};
        for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < m; t += (long long)gridDim.x * blockDim.x) {
            const long long i = bx[0] + t % ni, j = bx[2] + (t / ni) % nj, kz = bx[4] + t / (ni * nj);
            const long long p = i + fs.nx * (j + (long long)fs.ny * kz);
            const double u = U[p], v = V[p], w = W[p];
            s[0] += u * u + v * v + w * w;
            s[1] += u;
            s[2] += v;
            s[3] += w;
            s[4] += E[p];
        }
        for (int c = 0; c < 5; c++) red[c][threadIdx.x] = s[c];
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h)
                for (int c = 0; c < 5; c++) red[c][threadIdx.x] += red[c][threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x < 5)
            part[(((size_t)b * kMaxForcings + f) * gridDim.x + blockIdx.x) * 5 + threadIdx.x] = red[threadIdx.x][0];
        __syncthreads();
    }
}

__global__ void k_forcing_final(const double *part, int nblocks, double *sums)
{
    // one thread per (member, forcing, quantity): blockIdx.x = member
    const int t = threadIdx.x;  // f * 5 + q
    if (t >= kMaxForcings * 5) return;
    const int f = t / 5, qd = t % 5;
    const double *pp = part + ((size_t)blockIdx.x * kMaxForcings + f) * nblocks * 5 + qd;
    double s = 0;
    for (int c = 0; c < nblocks; c++) s += pp[(size_t)c * 5];
    sums[((size_t)blockIdx.x * kMaxForcings + f) * 5 + qd] = s;
}


__device__ __forceinline__ double sutherland_mu(const Phys &ph, double E)
{
    // nseq.F90:225-228 (and 77-80 in 2-D)
    const double g = ph.gamma, Ma = ph.Ma, T0 = ph.T0;
    const double mu1 = (1.0 + 110.0 / T0) / (g * (g - 1.0) * Ma * Ma * E + 110.0 / T0);
    const double mu2 = g * (g - 1.0) * Ma * Ma * E;
    return mu1 * mu2 * sqrt(mu2);
}

// Viscous stresses from the velocity gradients, 3-D (nseq.F90:225-236).  One definition for
// k_visc3d (which stores them for the second sweeps) and k_assemble3d (which recomputes them
// from the gradients it reads anyway instead of reading six stored fields back).
struct Stress3 {
    double xx, yy, zz, xy, xz, yz;
};
__device__ __forceinline__ Stress3 stress3d(double c, double dux, double duy, double duz, double dvx, double dvy,
                                            double dvz, double dwx, double dwy, double dwz)
{
    const double tzz = -2.0 / 3.0 * (dux + dvy + dwz);
    Stress3 t;
    t.xx = c * (2.0 * dux + tzz);
    t.yy = c * (2.0 * dvy + tzz);
    t.zz = c * (2.0 * dwz + tzz);
    t.xy = c * (duy + dvx);
    t.xz = c * (duz + dwx);
    t.yz = c * (dvz + dwy);
    return t;
}

// Stresses and heat fluxes at one point, 3-D (nseq.F90:225-239, 286-288): out[] in T3_* order;
// ld(i) returns the gradient of slot i in D3_* order (the R gradients are not read).
template <typename Ld>
__device__ __forceinline__ void visc3d_point(const Phys &ph, double E, Ld ld, double out[T3_N])
{
    const double mu = sutherland_mu(ph, E);
    const double c = 1.0 / ph.Re * mu;
    const Stress3 t = stress3d(c, ld(D3_UX), ld(D3_UY), ld(D3_UZ), ld(D3_VX), ld(D3_VY), ld(D3_VZ), ld(D3_WX),
                               ld(D3_WY), ld(D3_WZ));
    out[T3_XX] = t.xx;
    out[T3_YY] = t.yy;
    out[T3_ZZ] = t.zz;
    out[T3_XY] = t.xy;
    out[T3_XZ] = t.xz;
    out[T3_YZ] = t.yz;
    const double h = -ph.gamma / ph.Re / ph.Pr * mu;
    out[T3_QX] = h * ld(D3_EX);
    out[T3_QY] = h * ld(D3_EY);
    out[T3_QZ] = h * ld(D3_EZ);
}

// Stresses and heat fluxes, 3-D, thread per point.
__global__ void __launch_bounds__(256) k_visc3d(Phys ph, StateSet q, FieldSet d1, FieldSet tq, long long n)
{
    const int b = blockIdx.y;
    const double *E = q.v[4] + b * q.bstride;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        double o[T3_N];
        visc3d_point(ph, E[p], [&](int i) { return d1.f(b, i)[p]; }, o);
#pragma unroll
        for (int i = 0; i < T3_N; i++) tq.f(b, i)[p] = o[i];
    }
}

// Stresses and heat fluxes, 3-D, two consecutive points per thread through 16-byte loads and
// stores (n even, every field 16-byte aligned); same arithmetic as k_visc3d.
__global__ void __launch_bounds__(256) k_visc3d_v2(Phys ph, StateSet q, FieldSet d1, FieldSet tq, long long n)
{
    const int b = blockIdx.y;
    const double2 *E = reinterpret_cast<const double2 *>(q.v[4] + b * q.bstride);
    const long long n2 = n >> 1;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n2; p += (long long)gridDim.x * blockDim.x) {
        double2 g[D3_N];
#pragma unroll
        for (int i = 0; i < D3_N; i++)
            if (i != D3_RX && i != D3_RY && i != D3_RZ) g[i] = reinterpret_cast<const double2 *>(d1.f(b, i))[p];
        const double2 e = E[p];
        double o0[T3_N], o1[T3_N];
        visc3d_point(ph, e.x, [&](int i) { return g[i].x; }, o0);
        visc3d_point(ph, e.y, [&](int i) { return g[i].y; }, o1);
#pragma unroll
        for (int i = 0; i < T3_N; i++) reinterpret_cast<double2 *>(tq.f(b, i))[p] = make_double2(o0[i], o1[i]);
    }
}

// Stresses and heat fluxes, 2-D (nseq.F90:77-85, 109-110)
__global__ void k_visc2d(Phys ph, StateSet q, FieldSet d1, FieldSet tq, long long n)
{
    const int b = blockIdx.y;
    const double *E = q.v[4] + b * q.bstride;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double mu = sutherland_mu(ph, E[p]);
        const double dux = d1.f(b, D2_UX)[p], dvy = d1.f(b, D2_VY)[p];
        const double c = 1.0 / ph.Re * mu;
        tq.f(b, T2_XX)[p] = c * (2.0 * dux - 2.0 / 3.0 * (dux + dvy));
        tq.f(b, T2_YY)[p] = c * (2.0 * dvy - 2.0 / 3.0 * (dux + dvy));
        tq.f(b, T2_XY)[p] = c * (d1.f(b, D2_UY)[p] + d1.f(b, D2_VX)[p]);
        const double h = -ph.gamma / ph.Re / ph.Pr * mu;
        tq.f(b, T2_QX)[p] = h * d1.f(b, D2_EX)[p];
        tq.f(b, T2_QY)[p] = h * d1.f(b, D2_EY)[p];
    }
}

// RK4 update of one variable at one point (timeIntegration.F90:393-487)
__device__ __forceinline__ void rk_update(int mode, double dt, double k, double q0, double *delta, double *qn)
{
    switch (mode) {
    case RK_STORE_RHS: *qn = k; break;
    case RK_STAGE1: *delta = dt / 6.0 * k; *qn = q0 + dt / 2.0 * k; break;
    case RK_STAGE2: *delta = *delta + dt / 3.0 * k; *qn = q0 + dt / 2.0 * k; break;
    case RK_STAGE3: *delta = *delta + dt / 3.0 * k; *qn = q0 + dt * k; break;
    case RK_STAGE4: *qn = q0 + *delta + dt / 6.0 * k; break;
    // timeIntegration.F90:553-557 (Euler); 623-627, 648-652, 673-677 (SSPRK3: delta holds k1,
    // then k1 + k2; U + dt*(Uk1 + Uk2)/4 and U + dt*(Uk1 + Uk2 + 4*Uk3)/6 left to right)
    case RK_EULER: *qn = q0 + dt * k; break;
    case SSP_STAGE1: *delta = k; *qn = q0 + dt * k; break;
    case SSP_STAGE2: *delta = *delta + k; *qn = q0 + dt * *delta / 4.0; break;
    case SSP_STAGE3: *qn = q0 + dt * (*delta + 4.0 * k) / 6.0; break;
    }
}

// Input slots of the 3-D assembly: the stage state U, V, W, R, E, the 15 first derivatives
// (D3_* order), the 12 second-sweep results (S3_* order).
enum { A3_Q = 0, A3_D1 = 5, A3_D2 = 20, A3_NIN = 32 };

// dU, dV, dW, dR of nseq.F90:310-317 at one point, k[] in U, V, W, R order; ld(i) returns
// input slot i.  One definition for both assembly kernels.
template <typename Ld>
__device__ __forceinline__ void assemble3d_mom(const Phys &ph, Ld ld, double k[4])
{
    const double g = ph.gamma;
    const double u = ld(A3_Q + 0), v = ld(A3_Q + 1), w = ld(A3_Q + 2), r = ld(A3_Q + 3), e = ld(A3_Q + 4);
    const double dux = ld(A3_D1 + D3_UX), duy = ld(A3_D1 + D3_UY), duz = ld(A3_D1 + D3_UZ);
    const double dvx = ld(A3_D1 + D3_VX), dvy = ld(A3_D1 + D3_VY), dvz = ld(A3_D1 + D3_VZ);
    const double dwx = ld(A3_D1 + D3_WX), dwy = ld(A3_D1 + D3_WY), dwz = ld(A3_D1 + D3_WZ);
    const double drx = ld(A3_D1 + D3_RX), dry = ld(A3_D1 + D3_RY), drz = ld(A3_D1 + D3_RZ);
    const double dex = ld(A3_D1 + D3_EX), dey = ld(A3_D1 + D3_EY), dez = ld(A3_D1 + D3_EZ);
    const double DPx = (g - 1.0) * (r * dex + drx * e);
    const double DPy = (g - 1.0) * (r * dey + dry * e);
    const double DPz = (g - 1.0) * (r * dez + drz * e);
    const double vtx = ld(A3_D2 + S3_TXXX) + ld(A3_D2 + S3_TXYY) + ld(A3_D2 + S3_TXZZ);
    const double vty = ld(A3_D2 + S3_TYYY) + ld(A3_D2 + S3_TXYX) + ld(A3_D2 + S3_TYZZ);
    const double vtz = ld(A3_D2 + S3_TZZZ) + ld(A3_D2 + S3_TXZX) + ld(A3_D2 + S3_TYZY);
    k[3] = -r * (dux + dvy + dwz) - drx * u - dry * v - drz * w;
    k[0] = -(dux * u + duy * v + duz * w) + (vtx - DPx) / r;
    k[1] = -(dvx * u + dvy * v + dvz * w) + (vty - DPy) / r;
    k[2] = -(dwx * u + dwy * v + dwz * w) + (vtz - DPz) / r;
}

// dE of nseq.F90:318 at one point.  The stresses are recomputed from the gradients
// (stress3d) rather than read back.
template <typename Ld>
__device__ __forceinline__ double assemble3d_energy(const Phys &ph, Ld ld)
{
    const double g = ph.gamma;
    const double u = ld(A3_Q + 0), v = ld(A3_Q + 1), w = ld(A3_Q + 2), r = ld(A3_Q + 3), e = ld(A3_Q + 4);
    const double dux = ld(A3_D1 + D3_UX), duy = ld(A3_D1 + D3_UY), duz = ld(A3_D1 + D3_UZ);
    const double dvx = ld(A3_D1 + D3_VX), dvy = ld(A3_D1 + D3_VY), dvz = ld(A3_D1 + D3_VZ);
    const double dwx = ld(A3_D1 + D3_WX), dwy = ld(A3_D1 + D3_WY), dwz = ld(A3_D1 + D3_WZ);
    const double dex = ld(A3_D1 + D3_EX), dey = ld(A3_D1 + D3_EY), dez = ld(A3_D1 + D3_EZ);
    const double P = (g - 1.0) * r * e;
    const Stress3 t = stress3d(1.0 / ph.Re * sutherland_mu(ph, e), dux, duy, duz, dvx, dvy, dvz, dwx, dwy, dwz);
    return -(dex * u + dey * v + dez * w)
         + (-P * (dux + dvy + dwz) + t.xx * dux + t.yy * dvy
            + t.zz * dwz + t.xy * (dvx + duy)
            + t.xz * (dwx + duz) + t.yz * (dwy + dvz)
            - ld(A3_D2 + S3_HTX) - ld(A3_D2 + S3_HTY) - ld(A3_D2 + S3_HTZ)) / r;
}

// All five: k[] in U, V, W, R, E order.
template <typename Ld>
__device__ __forceinline__ void assemble3d_rhs(const Phys &ph, Ld ld, double k[5])
{
    assemble3d_mom(ph, ld, k);
    k[4] = assemble3d_energy(ph, ld);
}

// Assembly of dR, dU, dV, dW, dE (nseq.F90:310-318) fused with the RK4 stage update.
// q: stage input; q0: step start; out: stage output (may alias q: pointwise in place).
__global__ void __launch_bounds__(256, 3) k_assemble3d(Phys ph, StateSet q, StateSet q0, StateSet out, FieldSet delta,
                                                       FieldSet d1, FieldSet d2, long long n, int mode,
                                                       const StepParams *sp, Forcings fs)
{
    const int b = blockIdx.y;
    const double dt = sp ? sp->dt : 0.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        auto ld = [&](int i) {
            return i < A3_D1 ? q.v[i][b * q.bstride + p] : i < A3_D2 ? d1.f(b, i - A3_D1)[p] : d2.f(b, i - A3_D2)[p];
        };
        double k[5];
        assemble3d_rhs(ph, ld, k);
        if (fs.n) apply_forcings(fs, b, p, ld(A3_Q + 0), ld(A3_Q + 1), ld(A3_Q + 2), ld(A3_Q + 3), ld(A3_Q + 4), k, true, true);
#pragma unroll
        for (int f = 0; f < 5; f++) {
            double *dl = delta.p ? delta.f(b, f) + p : nullptr;
            double q0v = (mode != RK_STORE_RHS) ? q0.v[f][b * q0.bstride + p] : 0.0;
            double res;
            double dtmp = (dl && mode_reads_delta(mode)) ? *dl : 0.0;  // stage 1 overwrites delta
            rk_update(mode, dt, k[f], q0v, &dtmp, &res);
            if (dl && mode_writes_delta(mode)) *dl = dtmp;
            out.v[f][b * out.bstride + p] = res;
        }
    }
}

// 2-D assembly (nseq.F90:126-132) fused with the RK4 stage update.  W is left alone.
__global__ void k_assemble2d(Phys ph, StateSet q, StateSet q0, StateSet out, FieldSet delta,
                             FieldSet d1, FieldSet tq, FieldSet d2, long long n, int mode,
                             const StepParams *sp, Forcings fs)
{
    const int b = blockIdx.y;
    const double dt = sp ? sp->dt : 0.0;
    const double g = ph.gamma;
    const double *U = q.v[0] + b * q.bstride, *V = q.v[1] + b * q.bstride;
    const double *R = q.v[3] + b * q.bstride, *E = q.v[4] + b * q.bstride;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double u = U[p], v = V[p], r = R[p], e = E[p];
        const double dux = d1.f(b, D2_UX)[p], duy = d1.f(b, D2_UY)[p];
        const double dvx = d1.f(b, D2_VX)[p], dvy = d1.f(b, D2_VY)[p];
        const double drx = d1.f(b, D2_RX)[p], dry = d1.f(b, D2_RY)[p];
        const double dex = d1.f(b, D2_EX)[p], dey = d1.f(b, D2_EY)[p];
        const double P = (g - 1.0) * r * e;
        const double DPx = (g - 1.0) * (r * dex + drx * e);
        const double DPy = (g - 1.0) * (r * dey + dry * e);
        const double vtx = d2.f(b, S2_TXXX)[p] + d2.f(b, S2_TXYY)[p];
        const double vty = d2.f(b, S2_TYYY)[p] + d2.f(b, S2_TXYX)[p];
        const double kR = -r * (dux + dvy) - drx * u - dry * v;
        const double kU = -(dux * u + duy * v) + (vtx - DPx) / r;
        const double kV = -(dvx * u + dvy * v) + (vty - DPy) / r;
        const double kE = -(dex * u + dey * v)
                        + (-P * (dux + dvy) + tq.f(b, T2_XX)[p] * dux + tq.f(b, T2_YY)[p] * dvy
                           + tq.f(b, T2_XY)[p] * (dvx + duy) - d2.f(b, S2_HTX)[p] - d2.f(b, S2_HTY)[p]) / r;
        double k[5] = {kU, kV, 0.0, kR, kE};
        if (fs.n) apply_forcings(fs, b, p, u, v, 0.0, r, e, k, true, true);  // pressure gradient (2-D)
#pragma unroll
        for (int f = 0; f < 5; f++) {
            if (f == 2) continue;
            double *dl = delta.p ? delta.f(b, f) + p : nullptr;
            double q0v = (mode != RK_STORE_RHS) ? q0.v[f][b * q0.bstride + p] : 0.0;
            double res;
            double dtmp = (dl && mode_reads_delta(mode)) ? *dl : 0.0;  // stage 1 overwrites delta
            rk_update(mode, dt, k[f], q0v, &dtmp, &res);
            if (dl && mode_writes_delta(mode)) *dl = dtmp;
            out.v[f][b * out.bstride + p] = res;
        }
    }
}

// SFD relaxation (main.F90:381-402)
__global__ void k_sfd(StateSet q, FieldSet mean, const double *chi, double delta_sfd, int nvar,
                      long long n, const StepParams *sp)
{
    const int b = blockIdx.y;
    const double dt = sp->dt;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double x = chi[p];
        for (int f = 0; f < 5; f++) {
            if (nvar == 4 && f == 2) continue;
            double *qm = mean.f(b, f) + p;
            double *qq = q.v[f] + b * q.bstride + p;
            double m = *qm, v = *qq;
            if (delta_sfd > 0) { m = m + dt / delta_sfd * (v - m); *qm = m; }
            *qq = v - dt * x * (v - m);
        }
    }
}

// max|a - b| per variable, accumulated with an unsigned 64-bit max on the IEEE bits of
// the (non-negative) differences; a NaN (positive payload) wins over every number.
__global__ void k_maxchange(StateSet a, StateSet bset, unsigned long long *acc, long long n)
{
    const int b = blockIdx.y;
    __shared__ unsigned long long red[5][32];
    unsigned long long m[5] = {0, 0, 0, 0, 0};
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const double d = fabs(a.v[f][b * a.bstride + p] - bset.v[f][b * bset.bstride + p]);
            const unsigned long long u = (unsigned long long)__double_as_longlong(d);
            m[f] = u > m[f] ? u : m[f];
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int f = 0; f < 5; f++) {
        unsigned long long v = m[f];
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        if (lane == 0) red[f][wid] = v;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int f = 0; f < 5; f++) {
            unsigned long long v = lane < nw ? red[f][lane] : 0ull;
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w > v ? w : v;
            }
            if (lane == 0) atomicMax(acc + b * 5 + f, v);
        }
    }
}

// Max-change over independent (a, b) pointer sets: set s, variable v compares
// a[s*nvar+v] with b[s*nvar+v] over n points into acc[s*nvar+v] (blockIdx.y = set).
// (160 slots = 32 sets of the 5 variables; the pointer table is a 2.5 KB kernel parameter)
constexpr int kMaxChangeSlots = 160;
struct PtrSets {
    const double *a[kMaxChangeSlots];
    const double *b[kMaxChangeSlots];
};

__global__ void k_maxchange_sets(PtrSets ps, int nvar, unsigned long long *acc, long long n)
{
    const int s = blockIdx.y;
    for (int v = 0; v < nvar; v++) {
        const double *a = ps.a[s * nvar + v], *b = ps.b[s * nvar + v];
        unsigned long long m = 0;
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
            const unsigned long long u = (unsigned long long)__double_as_longlong(fabs(a[p] - b[p]));
            m = u > m ? u : m;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
            m = w > m ? w : m;
        }
        if ((threadIdx.x & 31) == 0) atomicMax(acc + s * nvar + v, m);
    }
}

// max|U|, max|V|, max|W| (main.F90:196-204), same bit trick
__global__ void k_maxvel(StateSet a, unsigned long long *acc, long long n)
{
    const int b = blockIdx.y;
    unsigned long long m[3] = {0, 0, 0};
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 3; f++) {
            const double d = fabs(a.v[f][b * a.bstride + p]);
            const unsigned long long u = (unsigned long long)__double_as_longlong(d);
            m[f] = u > m[f] ? u : m[f];
        }
    }
#pragma unroll
    for (int f = 0; f < 3; f++) {
        unsigned long long v = m[f];
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        if ((threadIdx.x & 31) == 0) atomicMax(acc + b * 3 + f, v);
    }
}

// Copy the accumulated max-change of this step into row `slot` of the history.
__global__ void k_store_maxchange(const unsigned long long *acc, double *hist, int nvals, const StepParams *sp)
{
    for (int i = threadIdx.x; i < nvals; i += blockDim.x)
        hist[sp->slot * nvals + i] = __longlong_as_double((long long)acc[i]);
}

__global__ void k_copy(double *dst, const double *src, long long n)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        dst[p] = src[p];
}

}  // namespace gatt
