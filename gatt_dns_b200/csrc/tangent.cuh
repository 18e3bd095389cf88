// Tangent-linear and adjoint pointwise kernels of the 3-D right-hand side (nseq.F90:142-323).
//
// The RHS is F(q) = Asm(q, D1 q, D2 T(E, D1 q)) with D1, D2 the line operators (linear), T the
// stresses and heat fluxes (k_visc3d / stress3d) and Asm the assembly (k_assemble3d).  The
// tangent runs the line operators on tangent fields and needs these pointwise derivatives:
//   k_tl_tau3d       dT = T_E dE + T_d1 dd1
//   k_tl_assemble3d  dk = Asm_q dq + Asm_d1 dd1 + Asm_d2 dd2 (stresses recomputed), then the
//                    same RK4 stage update as the forward on tangent arrays
// The adjoint runs the transposed line operators and these:
//   k_adj_asm3d      Asm^T a -> lambda on q, on the gradients, on the stresses (through the
//                    dissipation), on vtx/vty/vtz/ht (fed to the transposed second sweeps)
//   k_adj_tau3d      adds the transposed second sweeps, applies T^T (to gradients and E)
//   k_adj_q3d        adds the transposed first sweeps to lambda on q
// Layouts: d1 D3_*, tau T3_*, d2 S3_* (pointwise.cuh); adjoint sweep outputs S2[12] =
// x: (txx, txy, txz, qx) y: (txy, tyy, tyz, qy) z: (txz, tyz, tzz, qz) contributions, and
// S1[15] = [direction][U, V, W, R, E].
#pragma once

#include "pointwise.cuh"

namespace gatt {

// mu(E) of nseq.F90:225-228 and its derivative: mu = (1+S) x^{3/2} / (x+S), x = g(g-1)Ma^2 E,
// S = 110/T0  =>  dmu/dE = (1+S) g(g-1)Ma^2 sqrt(x) (x/2 + 3S/2) / (x+S)^2.
__device__ __forceinline__ double sutherland_dmu(const Phys &ph, double E)
{
    const double a = ph.gamma * (ph.gamma - 1.0) * ph.Ma * ph.Ma, S = 110.0 / ph.T0;
    const double x = a * E, den = x + S;
    return (1.0 + S) * a * sqrt(x) * (0.5 * x + 1.5 * S) / (den * den);
}

// tangent of stress3d: dc (tangent of c), gradients and their tangents
__device__ __forceinline__ Stress3 stress3d_tl(double c, double dc, double ux, double uy, double uz, double vx,
                                               double vy, double vz, double wx, double wy, double wz, double dux,
                                               double duy, double duz, double dvx, double dvy, double dvz, double dwx,
                                               double dwy, double dwz)
{
    const double tzz0 = -2.0 / 3.0 * (ux + vy + wz), dtzz0 = -2.0 / 3.0 * (dux + dvy + dwz);
    Stress3 t;
    t.xx = dc * (2.0 * ux + tzz0) + c * (2.0 * dux + dtzz0);
    t.yy = dc * (2.0 * vy + tzz0) + c * (2.0 * dvy + dtzz0);
    t.zz = dc * (2.0 * wz + tzz0) + c * (2.0 * dwz + dtzz0);
    t.xy = dc * (uy + vx) + c * (duy + dvx);
    t.xz = dc * (uz + wx) + c * (duz + dwx);
    t.yz = dc * (vz + wy) + c * (dvz + dwy);
    return t;
}

#define GATT_LOAD_D1(s, P)                                                                               \
    const double P##ux = s.f(b, D3_UX)[p], P##uy = s.f(b, D3_UY)[p], P##uz = s.f(b, D3_UZ)[p];           \
    const double P##vx = s.f(b, D3_VX)[p], P##vy = s.f(b, D3_VY)[p], P##vz = s.f(b, D3_VZ)[p];           \
    const double P##wx = s.f(b, D3_WX)[p], P##wy = s.f(b, D3_WY)[p], P##wz = s.f(b, D3_WZ)[p];           \
    const double P##rx = s.f(b, D3_RX)[p], P##ry = s.f(b, D3_RY)[p], P##rz = s.f(b, D3_RZ)[p];           \
    const double P##ex = s.f(b, D3_EX)[p], P##ey = s.f(b, D3_EY)[p], P##ez = s.f(b, D3_EZ)[p];

// dT = T_E dE + T_d1 dd1 (stresses and heat fluxes of k_visc3d, linearised)
__global__ void __launch_bounds__(256) k_tl_tau3d(Phys ph, StateSet q, FieldSet d1, StateSet dq, FieldSet dd1,
                                                  FieldSet dtq, long long n)
{
    const int b = blockIdx.y;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double e = q.v[4][b * q.bstride + p], de = dq.v[4][b * dq.bstride + p];
        const double mu = sutherland_mu(ph, e), dmu = sutherland_dmu(ph, e) * de;
        const double c = 1.0 / ph.Re * mu, dc = 1.0 / ph.Re * dmu;
        GATT_LOAD_D1(d1, )
        GATT_LOAD_D1(dd1, d)
        const Stress3 t = stress3d_tl(c, dc, ux, uy, uz, vx, vy, vz, wx, wy, wz, dux, duy, duz, dvx, dvy, dvz, dwx,
                                      dwy, dwz);
        dtq.f(b, T3_XX)[p] = t.xx;
        dtq.f(b, T3_YY)[p] = t.yy;
        dtq.f(b, T3_ZZ)[p] = t.zz;
        dtq.f(b, T3_XY)[p] = t.xy;
        dtq.f(b, T3_XZ)[p] = t.xz;
        dtq.f(b, T3_YZ)[p] = t.yz;
        const double hf = -ph.gamma / ph.Re / ph.Pr;
        const double h = hf * mu, dh = hf * dmu;
        dtq.f(b, T3_QX)[p] = dh * ex + h * dex;
        dtq.f(b, T3_QY)[p] = dh * ey + h * dey;
        dtq.f(b, T3_QZ)[p] = dh * ez + h * dez;
    }
}

// dk of the assembly, then the RK4 stage update on tangent arrays (same rk_update as the
// forward: the update is linear).  q: base stage input; dq: tangent stage input; dq0, dout,
// ddelta: tangent step start, output and increment.
__global__ void __launch_bounds__(256, 2) k_tl_assemble3d(Phys ph, StateSet q, FieldSet d1, FieldSet d2,
                                                          StateSet dq, FieldSet dd1, FieldSet dd2, StateSet dq0,
                                                          StateSet dout, FieldSet ddelta, long long n, int mode,
                                                          const StepParams *sp)
{
    const int b = blockIdx.y;
    const double dt = sp ? sp->dt : 0.0;
    const double g1 = ph.gamma - 1.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double u = q.v[0][b * q.bstride + p], v = q.v[1][b * q.bstride + p], w = q.v[2][b * q.bstride + p];
        const double r = q.v[3][b * q.bstride + p], e = q.v[4][b * q.bstride + p];
        const double du = dq.v[0][b * dq.bstride + p], dv = dq.v[1][b * dq.bstride + p];
        const double dw = dq.v[2][b * dq.bstride + p], dr = dq.v[3][b * dq.bstride + p];
        const double de = dq.v[4][b * dq.bstride + p];
        GATT_LOAD_D1(d1, )
        GATT_LOAD_D1(dd1, d)
        const double div = ux + vy + wz, ddiv = dux + dvy + dwz;
        const double P = g1 * r * e, dP = g1 * (dr * e + r * de);
        const double DPx = g1 * (r * ex + rx * e), DPy = g1 * (r * ey + ry * e), DPz = g1 * (r * ez + rz * e);
        const double dDPx = g1 * (dr * ex + r * dex + drx * e + rx * de);
        const double dDPy = g1 * (dr * ey + r * dey + dry * e + ry * de);
        const double dDPz = g1 * (dr * ez + r * dez + drz * e + rz * de);
        const double vtx = d2.f(b, S3_TXXX)[p] + d2.f(b, S3_TXYY)[p] + d2.f(b, S3_TXZZ)[p];
        const double vty = d2.f(b, S3_TYYY)[p] + d2.f(b, S3_TXYX)[p] + d2.f(b, S3_TYZZ)[p];
        const double vtz = d2.f(b, S3_TZZZ)[p] + d2.f(b, S3_TXZX)[p] + d2.f(b, S3_TYZY)[p];
        const double ht = d2.f(b, S3_HTX)[p] + d2.f(b, S3_HTY)[p] + d2.f(b, S3_HTZ)[p];
        const double dvtx = dd2.f(b, S3_TXXX)[p] + dd2.f(b, S3_TXYY)[p] + dd2.f(b, S3_TXZZ)[p];
        const double dvty = dd2.f(b, S3_TYYY)[p] + dd2.f(b, S3_TXYX)[p] + dd2.f(b, S3_TYZZ)[p];
        const double dvtz = dd2.f(b, S3_TZZZ)[p] + dd2.f(b, S3_TXZX)[p] + dd2.f(b, S3_TYZY)[p];
        const double dht = dd2.f(b, S3_HTX)[p] + dd2.f(b, S3_HTY)[p] + dd2.f(b, S3_HTZ)[p];
        const double mu = sutherland_mu(ph, e), c = 1.0 / ph.Re * mu;
        const double dc = 1.0 / ph.Re * (sutherland_dmu(ph, e) * de);
        const Stress3 t = stress3d(c, ux, uy, uz, vx, vy, vz, wx, wy, wz);
        const Stress3 dtt = stress3d_tl(c, dc, ux, uy, uz, vx, vy, vz, wx, wy, wz, dux, duy, duz, dvx, dvy, dvz, dwx,
                                        dwy, dwz);
        const double Phi = t.xx * ux + t.yy * vy + t.zz * wz + t.xy * (vx + uy) + t.xz * (wx + uz) + t.yz * (wy + vz);
        const double dPhi = dtt.xx * ux + t.xx * dux + dtt.yy * vy + t.yy * dvy + dtt.zz * wz + t.zz * dwz +
                            dtt.xy * (vx + uy) + t.xy * (dvx + duy) + dtt.xz * (wx + uz) + t.xz * (dwx + duz) +
                            dtt.yz * (wy + vz) + t.yz * (dwy + dvz);
        const double ir = 1.0 / r, ir2 = ir * ir;
        const double kR = -(dr * div + r * ddiv) - (drx * u + rx * du) - (dry * v + ry * dv) - (drz * w + rz * dw);
        const double kU = -(dux * u + ux * du + duy * v + uy * dv + duz * w + uz * dw) + (dvtx - dDPx) * ir -
                          (vtx - DPx) * dr * ir2;
        const double kV = -(dvx * u + vx * du + dvy * v + vy * dv + dvz * w + vz * dw) + (dvty - dDPy) * ir -
                          (vty - DPy) * dr * ir2;
        const double kW = -(dwx * u + wx * du + dwy * v + wy * dv + dwz * w + wz * dw) + (dvtz - dDPz) * ir -
                          (vtz - DPz) * dr * ir2;
        const double kE = -(dex * u + ex * du + dey * v + ey * dv + dez * w + ez * dw) +
                          (-dP * div - P * ddiv + dPhi - dht) * ir - (-P * div + Phi - ht) * dr * ir2;
        const double k[5] = {kU, kV, kW, kR, kE};
#pragma unroll
        for (int f = 0; f < 5; f++) {
            double *dl = ddelta.p ? ddelta.f(b, f) + p : nullptr;
            const double q0v = (mode != RK_STORE_RHS) ? dq0.v[f][b * dq0.bstride + p] : 0.0;
            double res;
            double dtmp = (dl && mode >= RK_STAGE2) ? *dl : 0.0;
            rk_update(mode, dt, k[f], q0v, &dtmp, &res);
            if (dl && mode != RK_STAGE4 && mode != RK_STORE_RHS) *dl = dtmp;
            dout.v[f][b * dout.bstride + p] = res;
        }
    }
}

// Asm^T a.  Outputs (overwritten): lq (5), ld1 (15, D3_*), ltau (9, T3_*: stresses through the
// dissipation, heat fluxes zero), lvt (4: vtx, vty, vtz, ht).
__global__ void __launch_bounds__(256, 2) k_adj_asm3d(Phys ph, StateSet q, FieldSet d1, FieldSet d2, StateSet a,
                                                      FieldSet lq, FieldSet ld1, FieldSet ltau, FieldSet lvt,
                                                      long long n)
{
    const int b = blockIdx.y;
    const double g1 = ph.gamma - 1.0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double u = q.v[0][b * q.bstride + p], v = q.v[1][b * q.bstride + p], w = q.v[2][b * q.bstride + p];
        const double r = q.v[3][b * q.bstride + p], e = q.v[4][b * q.bstride + p];
        const double aU = a.v[0][b * a.bstride + p], aV = a.v[1][b * a.bstride + p], aW = a.v[2][b * a.bstride + p];
        const double aR = a.v[3][b * a.bstride + p], aE = a.v[4][b * a.bstride + p];
        GATT_LOAD_D1(d1, )
        const double div = ux + vy + wz;
        const double P = g1 * r * e;
        const double DPx = g1 * (r * ex + rx * e), DPy = g1 * (r * ey + ry * e), DPz = g1 * (r * ez + rz * e);
        const double vtx = d2.f(b, S3_TXXX)[p] + d2.f(b, S3_TXYY)[p] + d2.f(b, S3_TXZZ)[p];
        const double vty = d2.f(b, S3_TYYY)[p] + d2.f(b, S3_TXYX)[p] + d2.f(b, S3_TYZZ)[p];
        const double vtz = d2.f(b, S3_TZZZ)[p] + d2.f(b, S3_TXZX)[p] + d2.f(b, S3_TYZY)[p];
        const double ht = d2.f(b, S3_HTX)[p] + d2.f(b, S3_HTY)[p] + d2.f(b, S3_HTZ)[p];
        const double c = 1.0 / ph.Re * sutherland_mu(ph, e);
        const Stress3 t = stress3d(c, ux, uy, uz, vx, vy, vz, wx, wy, wz);
        const double Phi = t.xx * ux + t.yy * vy + t.zz * wz + t.xy * (vx + uy) + t.xz * (wx + uz) + t.yz * (wy + vz);
        const double ir = 1.0 / r, ir2 = ir * ir;
        // kR = -r div - rx u - ry v - rz w
        double lr = -div * aR, ldiv = -r * aR;
        double lu = -rx * aR, lv = -ry * aR, lw = -rz * aR;
        double lrx = -u * aR, lry = -v * aR, lrz = -w * aR;
        // kU, kV, kW: convective terms and (vt - DP)/r
        double lux = -u * aU, luy = -v * aU, luz = -w * aU;
        lu += -ux * aU; lv += -uy * aU; lw += -uz * aU;
        double lvx = -u * aV, lvy = -v * aV, lvz = -w * aV;
        lu += -vx * aV; lv += -vy * aV; lw += -vz * aV;
        double lwx = -u * aW, lwy = -v * aW, lwz = -w * aW;
        lu += -wx * aW; lv += -wy * aW; lw += -wz * aW;
        const double lvtx = aU * ir, lvty = aV * ir, lvtz = aW * ir;
        const double lDPx = -aU * ir, lDPy = -aV * ir, lDPz = -aW * ir;
        lr += -(vtx - DPx) * aU * ir2 - (vty - DPy) * aV * ir2 - (vtz - DPz) * aW * ir2;
        // kE = -(ex u + ey v + ez w) + (-P div + Phi - ht)/r
        double lex = -u * aE, ley = -v * aE, lez = -w * aE;
        lu += -ex * aE; lv += -ey * aE; lw += -ez * aE;
        const double gE = aE * ir;
        const double lP = -div * gE;
        ldiv += -P * gE;
        const double lPhi = gE, lht = -gE;
        lr += -(-P * div + Phi - ht) * aE * ir2;
        // Phi = t:grad u with the stresses as separate inputs
        lux += t.xx * lPhi; lvy += t.yy * lPhi; lwz += t.zz * lPhi;
        lvx += t.xy * lPhi; luy += t.xy * lPhi;
        lwx += t.xz * lPhi; luz += t.xz * lPhi;
        lwy += t.yz * lPhi; lvz += t.yz * lPhi;
        // P = (g-1) r e; DP = (g-1)(r grad e + e grad r)
        lr += g1 * e * lP;
        double le = g1 * r * lP;
        lr += g1 * (ex * lDPx + ey * lDPy + ez * lDPz);
        lex += g1 * r * lDPx; ley += g1 * r * lDPy; lez += g1 * r * lDPz;
        lrx += g1 * e * lDPx; lry += g1 * e * lDPy; lrz += g1 * e * lDPz;
        le += g1 * (rx * lDPx + ry * lDPy + rz * lDPz);
        // div
        lux += ldiv; lvy += ldiv; lwz += ldiv;
        lq.f(b, 0)[p] = lu; lq.f(b, 1)[p] = lv; lq.f(b, 2)[p] = lw; lq.f(b, 3)[p] = lr; lq.f(b, 4)[p] = le;
        ld1.f(b, D3_UX)[p] = lux; ld1.f(b, D3_UY)[p] = luy; ld1.f(b, D3_UZ)[p] = luz;
        ld1.f(b, D3_VX)[p] = lvx; ld1.f(b, D3_VY)[p] = lvy; ld1.f(b, D3_VZ)[p] = lvz;
        ld1.f(b, D3_WX)[p] = lwx; ld1.f(b, D3_WY)[p] = lwy; ld1.f(b, D3_WZ)[p] = lwz;
        ld1.f(b, D3_RX)[p] = lrx; ld1.f(b, D3_RY)[p] = lry; ld1.f(b, D3_RZ)[p] = lrz;
        ld1.f(b, D3_EX)[p] = lex; ld1.f(b, D3_EY)[p] = ley; ld1.f(b, D3_EZ)[p] = lez;
        ltau.f(b, T3_XX)[p] = ux * lPhi; ltau.f(b, T3_YY)[p] = vy * lPhi; ltau.f(b, T3_ZZ)[p] = wz * lPhi;
        ltau.f(b, T3_XY)[p] = (vx + uy) * lPhi; ltau.f(b, T3_XZ)[p] = (wx + uz) * lPhi;
        ltau.f(b, T3_YZ)[p] = (wy + vz) * lPhi;
        ltau.f(b, T3_QX)[p] = 0.0; ltau.f(b, T3_QY)[p] = 0.0; ltau.f(b, T3_QZ)[p] = 0.0;
        lvt.f(b, 0)[p] = lvtx; lvt.f(b, 1)[p] = lvty; lvt.f(b, 2)[p] = lvtz; lvt.f(b, 3)[p] = lht;
    }
}

// lambda on the stresses = direct part + transposed second sweeps (S2), then T^T: adds to the
// gradients' lambda (ld1) and to lambda on E (lq slot 4).
__global__ void __launch_bounds__(256) k_adj_tau3d(Phys ph, StateSet q, FieldSet d1, FieldSet ltau, FieldSet s2,
                                                   FieldSet ld1, FieldSet lq, long long n)
{
    const int b = blockIdx.y;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double e = q.v[4][b * q.bstride + p];
        GATT_LOAD_D1(d1, )
        const double ltxx = ltau.f(b, T3_XX)[p] + s2.f(b, 0)[p];
        const double ltxy = ltau.f(b, T3_XY)[p] + s2.f(b, 1)[p] + s2.f(b, 4)[p];
        const double ltxz = ltau.f(b, T3_XZ)[p] + s2.f(b, 2)[p] + s2.f(b, 8)[p];
        const double ltyy = ltau.f(b, T3_YY)[p] + s2.f(b, 5)[p];
        const double ltyz = ltau.f(b, T3_YZ)[p] + s2.f(b, 6)[p] + s2.f(b, 9)[p];
        const double ltzz = ltau.f(b, T3_ZZ)[p] + s2.f(b, 10)[p];
        const double lqx = ltau.f(b, T3_QX)[p] + s2.f(b, 3)[p];
        const double lqy = ltau.f(b, T3_QY)[p] + s2.f(b, 7)[p];
        const double lqz = ltau.f(b, T3_QZ)[p] + s2.f(b, 11)[p];
        const double mu = sutherland_mu(ph, e), dmu = sutherland_dmu(ph, e);
        const double c = 1.0 / ph.Re * mu, cp = 1.0 / ph.Re * dmu;
        const double hf = -ph.gamma / ph.Re / ph.Pr;
        const double h = hf * mu, hp = hf * dmu;
        const double tzz0 = -2.0 / 3.0 * (ux + vy + wz);
        const double lc = (2.0 * ux + tzz0) * ltxx + (2.0 * vy + tzz0) * ltyy + (2.0 * wz + tzz0) * ltzz +
                          (uy + vx) * ltxy + (uz + wx) * ltxz + (vz + wy) * ltyz;
        const double ltzz0 = c * (ltxx + ltyy + ltzz);
        ld1.f(b, D3_UX)[p] += 2.0 * c * ltxx - 2.0 / 3.0 * ltzz0;
        ld1.f(b, D3_VY)[p] += 2.0 * c * ltyy - 2.0 / 3.0 * ltzz0;
        ld1.f(b, D3_WZ)[p] += 2.0 * c * ltzz - 2.0 / 3.0 * ltzz0;
        ld1.f(b, D3_UY)[p] += c * ltxy;
        ld1.f(b, D3_VX)[p] += c * ltxy;
        ld1.f(b, D3_UZ)[p] += c * ltxz;
        ld1.f(b, D3_WX)[p] += c * ltxz;
        ld1.f(b, D3_VZ)[p] += c * ltyz;
        ld1.f(b, D3_WY)[p] += c * ltyz;
        ld1.f(b, D3_EX)[p] += h * lqx;
        ld1.f(b, D3_EY)[p] += h * lqy;
        ld1.f(b, D3_EZ)[p] += h * lqz;
        const double lh = ex * lqx + ey * lqy + ez * lqz;
        lq.f(b, 4)[p] += cp * lc + hp * lh;
    }
}

// G = lq + the transposed first sweeps of the gradients' lambda (S1[direction][var])
__global__ void k_adj_q3d(FieldSet lq, FieldSet s1, StateSet G, long long n)
{
    const int b = blockIdx.y;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 5; f++)
            G.v[f][b * G.bstride + p] = lq.f(b, f)[p] + s1.f(b, f)[p] + s1.f(b, 5 + f)[p] + s1.f(b, 10 + f)[p];
    }
}

// out = alpha x + beta y over five fields (y may be null: out = alpha x)
__global__ void k_axpby5(StateSet out, StateSet x, StateSet y, double alpha, double beta, bool has_y, long long n)
{
    const int b = blockIdx.y;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const double xv = x.v[f][b * x.bstride + p];
            double r = alpha * xv;
            if (has_y) r = r + beta * y.v[f][b * y.bstride + p];
            out.v[f][b * out.bstride + p] = r;
        }
    }
}

// filter-blend adjoint: lam = lam + blend * (z - lam), blend = dt / fct (the forward's
// o + blend*(v - o) is linear in (o, v))
__global__ void k_adj_blend5(StateSet lam, StateSet z, const StepParams *sp, double fct, long long n)
{
    const int b = blockIdx.y;
    const double bl = sp->dt / fct;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int f = 0; f < 5; f++) {
            const double o = lam.v[f][b * lam.bstride + p];
            lam.v[f][b * lam.bstride + p] = o + bl * (z.v[f][b * z.bstride + p] - o);
        }
    }
}

// Adjoint of the SFD relaxation (k_sfd, main.F90:381-402).  Per point and variable, with
// x = dt chi and a = dt / Delta, the forward is m' = m + a (v - m), v' = v - x (v - m')
// (Delta > 0; otherwise m' = m).  From the sensitivities (lv, lm) of (v', m') it returns
// those of (v, m): with t = lm + x lv, lv <- (1 - x) lv + a t and lm <- (1 - a) t
// (Delta > 0); lv <- (1 - x) lv and lm <- t (Delta <= 0).  The tangent is k_sfd itself (the
// relaxation is linear in the state and the mean).
__global__ void k_sfd_adj(StateSet lq, FieldSet lmean, const double *chi, double delta_sfd, int nvar, long long n,
                          const StepParams *sp)
{
    const int b = blockIdx.y;
    const double dt = sp->dt;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double x = dt * chi[p];
        for (int f = 0; f < 5; f++) {
            if (nvar == 4 && f == 2) continue;
            double *lmp = lmean.f(b, f) + p;
            double *lvp = lq.v[f] + b * lq.bstride + p;
            const double lv = *lvp, t = *lmp + x * *lvp;
            if (delta_sfd > 0) {
                const double a = dt / delta_sfd;
                *lvp = (1.0 - x) * lv + a * t;
                *lmp = (1.0 - a) * t;
            } else {
                *lvp = (1.0 - x) * lv;
                *lmp = t;
            }
        }
    }
}

#undef GATT_LOAD_D1

}  // namespace gatt
