// Pointwise kernels fed by tensor copies (sm_100a).
//
// The 3-D assembly (nseq.F90:310-318 + the RK4 stage update, timeIntegration.F90:393-487)
// reads 32 to 42 fields per point.  Loaded by threads, every value in flight holds a register,
// and at 80 registers a thread the kernel stalls on memory latency well below the bandwidth
// (72 % of the copy peak).  Here persistent CTAs of 2*kPwC threads walk chunks of kPwC points;
// one thread issues the chunk's inputs as one tensor copy per field set -- a box of kPwC
// points by the set's slots (state 5, first derivatives 15, second sweeps 12, step start 5,
// increments 5), which lands slot-major in the ring stage -- into a two-stage shared-memory
// ring, so that the next chunk streams in, register-free, while the current one is computed
// from shared memory and stored.  (One 2 KB copy per field was bound by the number of copies
// the copy engine takes per SM, not by bytes.)  Two threads share a point (one the
// momentum and continuity rows, one the energy row) so that 16 warps compute while the ring
// holds two chunks.  The arithmetic is assemble3d_mom / assemble3d_energy, the same code as
// k_assemble3d.
//
// Requirements (checked by the host, which otherwise launches k_assemble3d): every set's
// fields equally spaced (a tensor map of dims {points, slots, members}), 16-byte aligned
// starts and an even number of points (tensor-map strides are multiples of 16 bytes).  A
// chunk past the last point reads zeros there and stores nothing.  Every mbarrier wait is
// bounded; a wait that gives up sets *err and the CTA returns after the copies it still has
// in flight land (bounded too).
#pragma once

#include "pointwise.cuh"
#include "rsweep.cuh"

namespace gatt {

// Points per chunk (the widest tensor box, 256 elements; threads per CTA: 2 * kPwC) and ring
// stages: 128-point chunks in four stages measured slower (more copies per byte).
constexpr int kPwC = 256;
constexpr int kPwSlots = A3_NIN + 10;          // inputs + step start (5) + increments (5)
constexpr int kPwStages = 2;

__host__ __device__ __forceinline__ size_t pw_smem_bytes(int nst)
{
    return (size_t)nst * kPwSlots * kPwC * sizeof(double) + 8 * (size_t)nst;
}

// Tensor maps of the assembly's input sets, each 5-D {points, slots, members, 1, 1}.
enum { PW_Q = 0, PW_D1, PW_D2, PW_Q0, PW_DL, PW_NMAPS };
struct PwMaps {
    CUtensorMap m[PW_NMAPS];
};

struct PwArgs {
    long long n;        // points per member
    long long nchunks;  // chunks per member
    long long njobs;    // chunks over all members
    int nst;            // ring stages
    int use_q0;         // step start read from its own arrays (else it is the stage input)
    int use_delta;      // increments read (stages 2-4)
    int mode;           // RK_* of the stage update
    int *err;           // set to 1 when a wait gives up
    Forcings fs;        // runForcings (none: fs.n = 0)
};

__global__ void __launch_bounds__(2 * kPwC, 1) k_assemble3d_pipe(Phys ph, StateSet out, FieldSet delta, PwArgs a,
                                                                 const StepParams *sp,
                                                                 const __grid_constant__ PwMaps maps)
{
    extern __shared__ __align__(128) double pw[];
    const int nst = a.nst;
    const uint32_t st0 = smem_u32(pw);
    const uint32_t bar0 = st0 + (uint32_t)(nst * kPwSlots * kPwC * sizeof(double));
    const long long G = gridDim.x;
    if (st0 & 127u) {  // tensor copies need 128-byte aligned stages
        if (threadIdx.x == 0) *(volatile int *)a.err = 2;
        return;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < nst; s++) mbar_init(bar0 + 8 * s, 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int nin = A3_NIN + (a.use_q0 ? 5 : 0) + (a.use_delta ? 5 : 0);
    // thread 0: the copies of chunk job j into stage s (full boxes: the tail's zero fill counts)
    auto issue = [&](long long j, int s) {
        const int b = (int)(j / a.nchunks);
        const int p0 = (int)((j % a.nchunks) * kPwC);
        const uint32_t bar = bar0 + 8 * s;
        const uint32_t dst = st0 + (uint32_t)(s * kPwSlots * kPwC * sizeof(double));
        constexpr uint32_t slot_bytes = kPwC * sizeof(double);
        fence_proxy_async();
        mbar_expect_tx(bar, (uint32_t)nin * slot_bytes);
        tma_load_5d(dst + A3_Q * slot_bytes, &maps.m[PW_Q], p0, 0, b, 0, 0, bar);
        tma_load_5d(dst + A3_D1 * slot_bytes, &maps.m[PW_D1], p0, 0, b, 0, 0, bar);
        tma_load_5d(dst + A3_D2 * slot_bytes, &maps.m[PW_D2], p0, 0, b, 0, 0, bar);
        if (a.use_q0) tma_load_5d(dst + A3_NIN * slot_bytes, &maps.m[PW_Q0], p0, 0, b, 0, 0, bar);
        if (a.use_delta) tma_load_5d(dst + (A3_NIN + 5) * slot_bytes, &maps.m[PW_DL], p0, 0, b, 0, 0, bar);
    };
    if (threadIdx.x == 0)
        for (int s = 0; s < nst; s++)
            if (blockIdx.x + s * G < a.njobs) issue(blockIdx.x + s * G, s);

    const double dt = sp ? sp->dt : 0.0;
    const int mode = a.mode;
    // two threads per point: the first kPwC threads the momentum and continuity rows, the
    // others the energy row
    const int pt = threadIdx.x % kPwC;
    const bool energy = threadIdx.x >= kPwC;
    int k = 0;
    for (long long j = blockIdx.x; j < a.njobs; j += G, k++) {
        const int s = k % nst;
        const uint32_t par = (uint32_t)(k / nst) & 1u;
        const bool late = !mbar_wait(bar0 + 8 * s, par);
        if (__syncthreads_or(late)) {
            // give up: report, let the other stages' copies land (bounded), leave
            if (threadIdx.x == 0) {
                *(volatile int *)a.err = 1;
                for (int t = 1; t < nst; t++)
                    if (j + t * G < a.njobs)
                        mbar_wait(bar0 + 8 * ((k + t) % nst), (uint32_t)((k + t) / nst) & 1u);
            }
            __syncthreads();
            return;
        }
        const int b = (int)(j / a.nchunks);
        const long long p0 = (j % a.nchunks) * kPwC;
        const double *S = pw + (size_t)s * kPwSlots * kPwC + pt;
        if (p0 + pt < a.n) {
            const long long p = p0 + pt;
            auto ld = [&](int i) { return S[i * kPwC]; };
            auto epi = [&](int v, double kv) {  // RK4 stage update of variable v
                const double q0v = mode == RK_STORE_RHS ? 0.0 : S[(a.use_q0 ? A3_NIN + v : A3_Q + v) * kPwC];
                double dtmp = a.use_delta ? S[(A3_NIN + 5 + v) * kPwC] : 0.0;  // stage 1 overwrites delta
                double res;
                rk_update(mode, dt, kv, q0v, &dtmp, &res);
                if (delta.p && mode_writes_delta(mode)) delta.f(b, v)[p] = dtmp;
                out.v[v][b * out.bstride + p] = res;
            };
            if (energy) {
                double kk[5];
                kk[4] = assemble3d_energy(ph, ld);
                if (a.fs.n) apply_forcings(a.fs, b, p, ld(0), ld(1), ld(2), ld(3), ld(4), kk, false, true);
                epi(4, kk[4]);
            } else {
                double kk[5];
                assemble3d_mom(ph, ld, kk);
                if (a.fs.n) apply_forcings(a.fs, b, p, ld(0), ld(1), ld(2), ld(3), ld(4), kk, true, false);
#pragma unroll
                for (int v = 0; v < 4; v++) epi(v, kk[v]);
            }
        }
        __syncthreads();  // every thread is done with stage s
        if (threadIdx.x == 0 && j + nst * G < a.njobs) issue(j + nst * G, s);
    }
}

}  // namespace gatt
