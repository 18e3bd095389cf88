// C-ABI implementation of the B200 GATT_DNS hot path (see include/gatt_dns.h).
//
// One context = one grid, `nbatch` flow states, one CUDA stream.  Device memory per
// member is laid out [member][slot][point]; the time step is captured once into a
// CUDA graph (one per state-buffer parity) and replayed with per-step {t, dt} copied
// into a device parameter block, so a step costs one small copy plus one graph launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/gatt_dns.h"
#include "arnoldi.cuh"
#include "tangent.cuh"
#include "bc.cuh"
#include "pointwise.cuh"
#include "pwpipe.cuh"
#include "rsweep.cuh"
#include "sweep.cuh"

using namespace gatt;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(e_ == cudaErrorMemoryAllocation ? GATT_ERR_NOMEM : GATT_ERR_CUDA,          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
    } while (0)

#define TRY(expr)                     \
    do {                              \
        int r_ = (expr);              \
        if (r_ != GATT_OK) return r_; \
    } while (0)

// Line-solve kernel families: shared-memory tile (any N), register-resident rows loaded
// from global memory, register-resident rows fed by a TMA ring (persistent CTAs).
enum SweepFamily { FAM_TILE = 0, FAM_REG = 1, FAM_PIPE = 2 };

// Matrix kinds per direction: 0 derivative, 1 filter, 2/3 derivative transpose (LHS^T solve,
// then R^T band), 4/5 filter transpose (same split); see gatt_set_matrices.
constexpr int kMatKinds = 6;

struct DevDir {
    bool set = false;
    int periodic = 0, nR = 0, nTypes = 0, N = 0, W = 0, Wp = 0, P = 1;
    int Np = 0;            // line length the pipelined solver runs: N, or N padded to 16 rows
    int rows = 0;          // rows of the kernel records uploaded (N, or Np for the padded solver)
    int rpb = 0;           // rows per block of the register-resident solver (0: shared-tile solver)
    bool uband = false;    // cyclic, one type, every row the same band: the uniform-band solver
    double band[16] = {};  // that band
    double cac[2] = {};    // and the corner couplings (cA, cC) of its row 0
    int family = 0;        // SweepFamily
    // the factors as given, repacked [type][row] ([type][row][diag] for R): kept to rebuild
    // the kernel records for another row-block partition (gatt_autotune)
    std::vector<double> hA, hB, hC, hD, hR;
    double *Rm = nullptr;  // band coefficients [nTypes][N][Wp]
    double *Q = nullptr;   // row records [nTypes][N][kQ] (see sweep.cuh)
};

struct HostBC {
    std::vector<int> ind;     // n*6, Fortran (n,6) column-major
    std::vector<double> val;  // Dirichlet values
    std::vector<int> dirs;    // Neumann / second-derivative directions
    int n = 0;
};

struct Dist {
    int type, var, ind[6], xoff;  // xoff: x coordinates (lid) or x factors (periodic sine) in distx
    double par;
};

constexpr int kBlock = 256;

// kernel classes reported by gatt_profile_kernels (names in gatt_profile_name)
enum {
    PC_D1X = 0, PC_D1Y, PC_D1Z, PC_VISC, PC_D2X, PC_D2Y, PC_D2Z, PC_ASSEMBLE, PC_BC,
    PC_FX, PC_FY, PC_FZ, PC_SFD, PC_MAXCHANGE, PC_OTHER, PC_D1YZ, PC_D2YZ, PC_N
};
const char *const kProfNames[PC_N] = {
    "sweep_d1_x", "sweep_d1_y", "sweep_d1_z", "visc", "sweep_d2_x", "sweep_d2_y", "sweep_d2_z",
    "assemble_rk", "bc", "filter_x", "filter_y", "filter_z", "sfd", "maxchange", "other",
    "sweep_d1_yz", "sweep_d2_yz"};

}  // namespace

struct gatt_ctx {
    int nx, ny, nz, nb;
    long long npts;
    bool is3d;
    Phys ph{};
    bool phys_set = false;
    DevDir mat[3][kMatKinds];  // kinds: derivative, filter, and the four transposed operators
    uint8_t *ltype[3] = {nullptr, nullptr, nullptr};
    bool lt_set[3] = {false, false, false};
    int lt_max[3] = {0, 0, 0};  // largest 0-based type in each direction's map
    int filt[3] = {0, 0, 0};
    double fct = -1.0;
    // boundary data (host) and the device program built from it
    HostBC bc[3][5];
    std::vector<int> cL, cD, cAd;
    int cN = 0;
    std::vector<double> coef1, coef2;
    std::vector<Dist> dists;
    std::vector<double> distx;
    BcOp *d_ops = nullptr;
    int nops = 0;
    double *d_coef1 = nullptr, *d_coef2 = nullptr, *d_xs = nullptr;
    // holdInlet: the values the first gatt_apply_bc kept, hold_len per member, laid out as the
    // program's OP_HOLD ops say (hold_sig: their boxes and field counts)
    double *d_hold = nullptr;
    long long hold_len = 0;
    std::vector<int> hold_sig;
    bool hold_saved = false;
    bool bc_dirty = true;
    // SFD
    int sfd_type = 0;
    double sfd_delta = 0;
    double *chi = nullptr;
    // state and scratch
    double *qA = nullptr, *qB = nullptr, *delta = nullptr, *mean = nullptr;
    double *d1 = nullptr, *tq = nullptr, *d2 = nullptr, *P = nullptr, *tmp = nullptr;
    double *tin = nullptr, *tout = nullptr;  // host-facing scratch (rhs / deriv entry points)
    // Jacobian-free Arnoldi (gatt_arnoldi): basis [b][j][v][p], B, base and base-run states,
    // reduction partials, Hessenberg columns, region mask
    double *arn_zeta = nullptr, *arn_B = nullptr, *arn_base = nullptr, *arn_um = nullptr;
    double *arn_part = nullptr, *arn_h = nullptr;
    uint8_t *arn_region = nullptr;
    int arn_m = 0;       // basis vectors held: m + 1 per member
    bool arn_have_region = false;
    // tangent-linear / adjoint work arrays (5-field sets unless noted), allocated on first use
    double *dx[5] = {};                  // base states: step start and stage states
    double *dy[3] = {};                  // tangent states
    double *t_delta = nullptr, *t_d1 = nullptr, *t_tq = nullptr, *t_d2 = nullptr;  // tangent RK increment, 15, 9, 12
    double *a_lam = nullptr, *a_acc = nullptr, *a_arg = nullptr, *a_prev = nullptr, *a_g = nullptr;
    double *a_lq = nullptr, *a_ld1 = nullptr, *a_ltau = nullptr, *a_lvt = nullptr;  // 5, 15, 9, 4
    double *a_s1 = nullptr, *a_s2 = nullptr, *a_scr = nullptr;                       // 15, 12, 5
    double *a_ckpt = nullptr, *a_seg = nullptr;
    int a_nckpt = 0, a_nseg = 0;
    bool a_ckpt_sfd = false, a_seg_sfd = false;  // checkpoint / segment slots hold a mean too
    long long tape_len = 0;              // doubles of the boundary-program tape per member
    double *t_P = nullptr, *a_lP = nullptr, *a_tape = nullptr, *a_tmp = nullptr;
    // 2-D cases: the base gradients, stresses and second sweeps of the tangent / adjoint in the
    // 3-D layouts (z slots zero); 3-D cases use d1 / tq / d2
    double *g_d1 = nullptr, *g_tq = nullptr, *g_d2 = nullptr;
    // SFD cases: the base mean of the step, the tangent mean, the adjoint mean and a scratch mean
    double *dxm = nullptr, *dym = nullptr, *a_lm = nullptr, *a_mscr = nullptr;
    long long a_tape_cap = 0;
    bool mean_init = false;                  // SFD mean uploaded or copied from the state
    int cur = 0;
    unsigned long long *acc = nullptr;
    double *hist = nullptr;
    int hist_cap = 0;
    StepParams *d_params = nullptr;
    StepParams *h_params = nullptr;  // pinned, hist_cap entries
    cudaStream_t stream = nullptr;
    // side stream: an x sweep runs on it beside the y/z sweeps of the same operand set (fork
    // and join through the two events; captured as parallel graph branches)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    double *tmp_side = nullptr;  // the side stream's scratch field (the global-memory line solver)
    bool own_stream = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_kernels[2] = {0, 0};
    bool capturing = false;
    int capture_count = 0;
    long long launches = 0;
    int nsm = 148;
    int *h_err = nullptr;   // pipeline wait give-up flag (pinned, device-mapped)
    int *d_err = nullptr;
    bool pw_pipe = true;    // 3-D assembly fed by bulk copies (GATT_PW=plain: thread loads)
    bool merge_yz = true;   // y and z derivative sweeps in one launch where their sets allow (GATT_MERGE_YZ=0: no)
    bool fuse_mc = true;    // max-change in the last filter sweep where nothing follows it (GATT_FUSE_MC=0: no)
    bool uband_on = true;   // uniform-band solver where a set allows it (GATT_UBAND=0: no)
    bool x_order = true;    // x tiles field-inner, last tile first (GATT_X_ORDER=0: tile-inner, first first)
    bool visc_v2 = true;    // stresses two points per thread (GATT_VISC_V2=0: one)
    bool x_compact = true;  // compact shared memory for the uniform-band x solver (GATT_X_COMPACT=0: no)
    bool x_wstore = true;   // x tiles stored chunk by chunk by their warps (GATT_X_WSTORE=0: by one thread)
    int time_stepping = 1;  // parameters.F90 timeStepping: 1 RK4, 2 Euler, 3 SSPRK3
    Forcings fc{};          // runForcings (fc.n = 0: none); boxes 0-based
    double *fsum = nullptr, *fpart = nullptr;  // turbulence box sums, per-CTA partials
    int fblocks = 0;        // CTAs of the sums kernel (fixed: the sums do not depend on timing)
    bool fork_x = true;     // x sweeps beside the y/z sweeps, filter field chains side by side
                            // (GATT_FORK_X=0: everything on one stream)
    bool fz_rev = true;     // last filter direction takes the fields in reverse order (GATT_FZ_REV=0: no)
    bool mc_done = false;   // set when a filter launch ran the max-change epilogue
    int bc_cluster = 0;     // CTAs per member for the boundary program (0: one CTA, k_bc)
    int bc_cluster_rec = 0, bc_cluster_tl = 0, bc_cluster_adj = 0;  // same, tape / tangent / adjoint
    long long bc_points = 0;  // point updates of one application of the program (sum over ops)
    // per-kernel-class timing (gatt_profile_kernels): events around every launch
    bool profiling = false;
    int prof_cls = -1;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_cls;  // class of each begin/end event pair
};

namespace {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------

// Synchronize the context's stream and report a line-solve pipeline that gave up waiting.
int sync_stream(gatt_ctx *c)
{
    CU(cudaStreamSynchronize(c->stream));
    if (c->h_err && *(volatile int *)c->h_err) {
        *(volatile int *)c->h_err = 0;
        return fail(GATT_ERR_TIMEOUT, "a copy pipeline gave up (tile wait timed out or misaligned ring)");
    }
    return GATT_OK;
}

int grid_for(const gatt_ctx *c, long long n)
{
    long long g = (n + kBlock - 1) / kBlock;
    long long cap = (long long)c->nsm * 8;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// Mark the start of a launch of kernel class `cls` (only records when profiling).
int before_launch(gatt_ctx *c, int cls)
{
    c->prof_cls = cls;
    if (!c->profiling) return GATT_OK;
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    CU(cudaEventRecord(e, c->stream));
    c->ev_pool.push_back(e);
    return GATT_OK;
}

int after_launch(gatt_ctx *c)
{
    if (c->profiling && c->prof_cls >= 0) {
        cudaEvent_t e;
        CU(cudaEventCreate(&e));
        CU(cudaEventRecord(e, c->stream));
        c->ev_pool.push_back(e);
        c->ev_cls.push_back(c->prof_cls);
    }
    c->prof_cls = -1;
    if (c->capturing) c->capture_count++;
    else c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GATT_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return GATT_OK;
}

int line_len(const gatt_ctx *c, int d) { return d == 0 ? c->nx : (d == 1 ? c->ny : c->nz); }
int nlines(const gatt_ctx *c, int d)
{
    return d == 0 ? c->ny * c->nz : (d == 1 ? c->nx * c->nz : c->nx * c->ny);
}

// State set of the current (which = 0) or next (which = 1) buffer.  In 2-D, slot W of
// buffer A is the caller's W and slot W of buffer B is main.F90's Wnew, never swapped.
StateSet state_set(const gatt_ctx *c, int which)
{
    double *buf = ((c->cur ^ which) == 0) ? c->qA : c->qB;
    StateSet s;
    for (int f = 0; f < 5; f++) s.v[f] = buf + f * c->npts;
    if (!c->is3d) s.v[2] = (which == 0 ? c->qA : c->qB) + 2 * c->npts;
    s.bstride = 5 * c->npts;
    return s;
}

FieldSet fset(const gatt_ctx *c, double *p, int nslots)
{
    FieldSet f;
    f.p = p;
    f.bstride = (long long)nslots * c->npts;
    f.npts = c->npts;
    return f;
}

int nd1(const gatt_ctx *c) { return c->is3d ? (int)D3_N : (int)D2_N; }
int ntq(const gatt_ctx *c) { return c->is3d ? (int)T3_N : (int)T2_N; }
int nd2(const gatt_ctx *c) { return c->is3d ? (int)S3_N : (int)S2_N; }

// ---------------------------------------------------------------------------
// line-solve dispatch
// ---------------------------------------------------------------------------

template <bool XD, bool PER, bool BIG>
void *pick_kernel(int nR)
{
    switch (nR) {
    case 2: return (void *)k_sweep<XD, PER, 2, BIG>;
    case 3: return (void *)k_sweep<XD, PER, 3, BIG>;
    case 4: return (void *)k_sweep<XD, PER, 4, BIG>;
    case 5: return (void *)k_sweep<XD, PER, 5, BIG>;
    case 6: return (void *)k_sweep<XD, PER, 6, BIG>;
    case 7: return (void *)k_sweep<XD, PER, 7, BIG>;
    case 8: return (void *)k_sweep<XD, PER, 8, BIG>;
    case 9: return (void *)k_sweep<XD, PER, 9, BIG>;
    case 10: return (void *)k_sweep<XD, PER, 10, BIG>;
    case 11: return (void *)k_sweep<XD, PER, 11, BIG>;
    default: return nullptr;
    }
}

void *sweep_kernel(bool xd, bool per, int nR, bool big)
{
    if (big) {
        if (xd) return per ? pick_kernel<true, true, true>(nR) : pick_kernel<true, false, true>(nR);
        return per ? pick_kernel<false, true, true>(nR) : pick_kernel<false, false, true>(nR);
    }
    if (xd) return per ? pick_kernel<true, true, false>(nR) : pick_kernel<true, false, false>(nR);
    return per ? pick_kernel<false, true, false>(nR) : pick_kernel<false, false, false>(nR);
}

// Register-resident solvers: 16-row blocks (32-row blocks spill registers for most bands).
constexpr int kRPB = 16;

template <bool XD, bool PER, bool PIPE>
void *pick_reg_kernel(int nR)
{
#define GATT_REG_CASE(n) \
    case n: return PIPE ? (void *)k_psweep<XD, PER, n, kRPB> : (void *)k_rsweep<XD, PER, n, kRPB>;
    switch (nR) {
    GATT_REG_CASE(2) GATT_REG_CASE(3) GATT_REG_CASE(4) GATT_REG_CASE(5) GATT_REG_CASE(6) GATT_REG_CASE(7)
    default: return nullptr;
    }
#undef GATT_REG_CASE
}

// The pipelined solver of cyclic lines whose rows all share one band (launch constants).
template <bool XD>
void *pick_ub_kernel(int nR)
{
    switch (nR) {
    case 2: return (void *)k_psweep<XD, true, 2, kRPB, false, true>;
    case 3: return (void *)k_psweep<XD, true, 3, kRPB, false, true>;
    case 4: return (void *)k_psweep<XD, true, 4, kRPB, false, true>;
    case 5: return (void *)k_psweep<XD, true, 5, kRPB, false, true>;
    case 6: return (void *)k_psweep<XD, true, 6, kRPB, false, true>;
    case 7: return (void *)k_psweep<XD, true, 7, kRPB, false, true>;
    default: return nullptr;
    }
}

// The pipelined x solver for more than 24 row blocks (800-thread bound).
template <bool PER>
void *pick_wide_kernel(int nR)
{
    switch (nR) {
    case 2: return (void *)k_psweep<true, PER, 2, kRPB, true>;
    case 3: return (void *)k_psweep<true, PER, 3, kRPB, true>;
    case 4: return (void *)k_psweep<true, PER, 4, kRPB, true>;
    case 5: return (void *)k_psweep<true, PER, 5, kRPB, true>;
    case 6: return (void *)k_psweep<true, PER, 6, kRPB, true>;
    case 7: return (void *)k_psweep<true, PER, 7, kRPB, true>;
    default: return nullptr;
    }
}

void *reg_kernel(bool pipe, bool xd, bool per, int nR, bool wide = false)
{
    if (wide) return (pipe && xd) ? (per ? pick_wide_kernel<true>(nR) : pick_wide_kernel<false>(nR)) : nullptr;
    if (pipe) {
        if (xd) return per ? pick_reg_kernel<true, true, true>(nR) : pick_reg_kernel<true, false, true>(nR);
        return per ? pick_reg_kernel<false, true, true>(nR) : pick_reg_kernel<false, false, true>(nR);
    }
    if (xd) return per ? pick_reg_kernel<true, true, false>(nR) : pick_reg_kernel<true, false, false>(nR);
    return per ? pick_reg_kernel<false, true, false>(nR) : pick_reg_kernel<false, false, false>(nR);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled()
{
    static EncodeTiledFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (EncodeTiledFn)f;
    }();
    return fn;
}

// Resident CTAs per SM of a kernel at a block size and dynamic shared memory (cached).
int resident_ctas(const void *k, int threads, size_t smem)
{
    static std::mutex mu;
    static std::map<std::tuple<const void *, int, size_t>, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_tuple(k, threads, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, threads, smem) != cudaSuccess) n = 0;
    cache[key] = n;
    return n;
}

// Line-solve family for new matrices: GATT_SWEEP = tile | reg | pipe (default pipe).
int choose_family()
{
    const char *e = getenv("GATT_SWEEP");
    if (e && strcmp(e, "tile") == 0) return FAM_TILE;
    if (e && strcmp(e, "reg") == 0) return FAM_REG;
    return FAM_PIPE;
}

// Shared memory a CTA may use (the opt-in maximum less a margin).
constexpr size_t kMaxSmem = 227 * 1024 - 256;

// Padded line length for the pipelined solver: non-cyclic y/z lines whose length is not a
// multiple of kRPB run as lines of the next multiple, the extra rows identity rows (A = C = 0,
// reciprocal pivot 1, zero band) that the tile copy fills with zeros past the grid edge and
// the store skips; the real rows' results are those of the unpadded line (the last real row
// has no super-diagonal, the first padded one no sub-diagonal).  Returns N when that does not
// apply (cyclic or x lines, more rows than the y/z solver's 24 blocks, layouts the tensor map
// cannot describe).
int padded_rows(const gatt_ctx *c, int d, int N, int nR, int periodic)
{
    if (N % kRPB == 0 || periodic || d == 0 || nR < 2 || nR > kMaxNRreg) return N;
    const int np = (N + kRPB - 1) / kRPB * kRPB;
    if (np / kRPB > kMaxPyz || (c->nx & 1) || (c->npts & 1)) return N;
    return np;
}

// Block height of the register-resident solvers for lines of Np rows (Np: N or its padded
// length) and band nR, or 0 when the shared-tile solver handles them (length not a multiple of
// kRPB, too many blocks, or a band wider than kMaxNRreg).  Padded lines and x lines of more
// than kMaxP blocks (up to kMaxPx) need the pipelined solver, and its shared memory must fit.
int choose_rpb(int d, int N, int Np, int nR, int nTypes, int Wp)
{
    if (choose_family() == FAM_TILE) return 0;
    if (nR < 2 || nR > kMaxNRreg || Np % kRPB) return 0;
    const int P = Np / kRPB;
    if (P <= kMaxP && Np == N) return kRPB;
    const bool pipe = choose_family() == FAM_PIPE;
    // thread bounds of the pipelined instantiations: x wide form 800, y/z 768 (512 for the
    // 6-band filter)
    const int maxp = d == 0 ? kMaxPx : (nR == 6 ? kMaxP : kMaxPyz);
    if (!pipe || P > maxp) return 0;
    return psweep_smem_bytes(d == 0, Np, P, nTypes, Wp, 1) <= kMaxSmem ? kRPB : 0;
}

size_t sweep_smem(int N, int P, int nR, int Wp, bool stage = true)
{
    return sweep_smem_doubles(N, P, nR, Wp, stage) * sizeof(double);
}
// 227 KB per block, less a margin for the kernel's few static shared variables
constexpr int kMaxNR = 11;  // widest band the shared-tile solver is instantiated for

// Row blocks per line: about 32 rows per block (shorter dependency chains, more warps per
// tile), a power of two up to kMaxP, every block at least nR+1 rows long, and few enough
// that the shared tile fits (long lines: fewer blocks, halo and exchange rows).
int choose_blocks(int N, int nR, int Wp, int rows = 0)
{
    if (rows < 4) {
        const char *e = getenv("GATT_BLOCK_ROWS");
        const int v = e ? atoi(e) : 0;
        rows = v >= 4 ? v : 32;
    }
    int P = 1;
    while (P * 2 <= kMaxP && N / (P * 2) >= rows && N / (P * 2) >= nR + 1) P *= 2;
    while (P > 1 && sweep_smem(N, P, nR, Wp, false) > kMaxSmem) P /= 2;
    return P;
}

// Allow every line-solve instantiation the full shared-memory budget once per context,
// outside any stream capture.
int set_sweep_attributes()
{
    for (int big = 0; big < 2; big++)
        for (int xd = 0; xd < 2; xd++)
            for (int per = 0; per < 2; per++)
                for (int nR = 2; nR <= kMaxNR; nR++) {
                    void *k = sweep_kernel(xd != 0, per != 0, nR, big != 0);
                    CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
                }
    for (int xd = 0; xd < 2; xd++)
        for (int per = 0; per < 2; per++)
            for (int nR = 2; nR <= kMaxNRreg; nR++)
                for (int wide = 0; wide < 2; wide++) {
                    void *k = reg_kernel(true, xd != 0, per != 0, nR, wide != 0);
                    if (!k) continue;
                    CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
                    CU(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
                }
    for (int xd = 0; xd < 2; xd++)  // the uniform-band instantiations
        for (int nR = 2; nR <= kMaxNRreg; nR++) {
            void *k = xd ? pick_ub_kernel<true>(nR) : pick_ub_kernel<false>(nR);
            if (!k) continue;
            CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
            CU(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        }
    CU(cudaFuncSetAttribute((const void *)k_assemble3d_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)pw_smem_bytes(kPwStages)));
    return GATT_OK;
}

// Kernel row records (sweep.cuh) of a matrix set for a partition into P row blocks: the
// reference's factors in uniform row semantics plus the block propagators of the partitioned
// recurrences (long double products).  Allocates the device arrays on first use.
int upload_records(gatt_ctx *c, DevDir &m, int P, int rows = 0)
{
    const int N0 = m.N, W = m.W, Wp = m.Wp, nTypes = m.nTypes;
    const int N = rows > 0 ? rows : N0;  // records for N rows: rows past N0 are identity rows
    const bool periodic = m.periodic != 0;
    if (N != N0 && periodic) return fail(GATT_ERR_STATE, "cyclic lines cannot be padded");
    std::vector<double> hRm((size_t)nTypes * N * Wp, 0.0), hQ((size_t)nTypes * N * kQ, 0.0);
    for (int t = 0; t < nTypes; t++) {
        const double *tA = &m.hA[(size_t)t * N0], *tB = &m.hB[(size_t)t * N0], *tC = &m.hC[(size_t)t * N0];
        double *q = &hQ[(size_t)t * N * kQ];
        for (int r = 0; r < N; r++) {
            double *qr = q + (size_t)r * kQ;
            if (r >= N0) {  // padding: x = 0 whatever comes before or after
                qr[kQfB] = 1.0;
                continue;
            }
            if (!periodic) {
                qr[kQfA] = r > 0 ? tA[r - 1] : 0.0;       // derivs.F90:607
                qr[kQfB] = tB[r];
                qr[kQbC] = r < N0 - 1 ? tC[r] : 0.0;      // derivs.F90:610
            } else {
                qr[kQfA] = r >= 2 ? tA[r - 1] : 0.0;      // derivs.F90:798
                qr[kQfB] = r >= 1 ? tB[r - 1] : 0.0;      // derivs.F90:796-798
                qr[kQbC] = (r >= 1 && r <= N - 2) ? tC[r] : 0.0;  // derivs.F90:801
                qr[kQD] = m.hD[(size_t)t * N + r];        // derivs.F90:786-789
            }
            for (int k = 0; k < W; k++) hRm[((size_t)t * N + r) * Wp + k] = m.hR[((size_t)t * N0 + r) * W + k];
        }
        if (periodic) { q[kQcA] = tA[0]; q[kQcC] = tC[0]; }  // derivs.F90:792-793
        for (int p = 0; p < P; p++) {
            const int s0 = block_start(p, N, P), e0 = block_start(p + 1, N, P) - 1;
            const int rs = (periodic && p == 0) ? 1 : s0;
            long double prod = 1.0L;
            for (int r = rs; r <= e0; r++) {
                prod *= -(long double)q[(size_t)r * kQ + kQfA] * (long double)q[(size_t)r * kQ + kQfB];
                q[(size_t)r * kQ + kQpi] = (double)prod;
            }
            prod = 1.0L;
            for (int r = e0; r >= rs; r--) {
                prod *= -(long double)q[(size_t)r * kQ + kQbC];
                q[(size_t)r * kQ + kQrho] = (double)prod;
            }
        }
    }
    // uniform band: cyclic, one type, every row's band equal to row 0's
    m.uband = periodic && nTypes == 1 && W <= 16 && N == N0;
    for (int r = 1; m.uband && r < N0; r++)
        for (int k = 0; k < W; k++)
            if (m.hR[(size_t)r * W + k] != m.hR[k]) m.uband = false;
    memset(m.band, 0, sizeof(m.band));
    if (m.uband) {
        for (int k = 0; k < W; k++) m.band[k] = m.hR[k];
        m.cac[0] = m.hA[0];  // derivs.F90:792-793
        m.cac[1] = m.hC[0];
    }
    TRY(sync_stream(c));
    if (!m.Rm) CU(cudaMalloc(&m.Rm, hRm.size() * sizeof(double)));
    if (!m.Q) CU(cudaMalloc(&m.Q, hQ.size() * sizeof(double)));
    CU(cudaMemcpy(m.Rm, hRm.data(), hRm.size() * sizeof(double), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(m.Q, hQ.data(), hQ.size() * sizeof(double), cudaMemcpyHostToDevice));
    m.P = P;
    m.rows = N;
    return GATT_OK;
}

// Pipelined register solver: build the tensor map (y/z), size the persistent grid, launch.
// Returns GATT_ERR_STATE (without launching) when the layout does not meet the copy engine's
// alignment rules, so that the caller falls back to k_rsweep.
int launch_psweep(gatt_ctx *c, const DevDir &m, int d, SweepArgs &a, int nmembers, int cls, const DevDir *m1 = nullptr)
{
    const int N = m.rows;  // padded y/z lines: the box covers the padding (zero fill)
    const bool xd = d == 0;
    const int nt1 = m1 ? m1->nTypes : 0;  // part 1 (z lines of a y+z launch)
    // uniform band (both parts the same band): launch constants instead of shared records
    bool ub = m.uband && m.periodic && m.P <= 24 && c->uband_on;
    if (ub && m1) ub = m1->uband && !memcmp(m.band, m1->band, sizeof(m.band));
    void *k = ub ? (xd ? pick_ub_kernel<true>(m.nR) : pick_ub_kernel<false>(m.nR))
                 : reg_kernel(true, xd, m.periodic != 0, m.nR, m.P > 24);  // 25 blocks: the 800-thread form
    if (ub) {
        memcpy(a.band, m.band, sizeof(a.band));
        memcpy(a.cac, m.cac, sizeof(a.cac));
    }
    const bool cmp = ub && xd && c->x_compact;  // the compact shared-memory layout
    if (!k) return GATT_ERR_STATE;
    // ring depth: the deepest ring that keeps the most CTAs resident (one stage suffices
    // when a tile's solve outlasts the next tile's copy)
    int nst = 0, per_sm = 0;
    size_t smem = 0;
    const int wps = ub ? 0 : m.Wp;  // the uniform-band solver keeps no band rows in shared memory
    for (int st = kMaxStages; st >= 1; st--) {
        const size_t b = psweep_smem_bytes(xd, N, m.P, m.nTypes, wps, st, nt1, cmp);
        if (b > kMaxSmem) continue;
        const int r = resident_ctas(k, 32 * m.P, b);
        if (r > per_sm) { per_sm = r; nst = st; smem = b; }
    }
    // x tiles hold their stage through the solve and the tensor store, so only a second stage
    // lets the next tile load meanwhile: among rings of two stages or more, the most resident
    // CTAs, then the deepest ring (128^3: x sweeps 7-14 % faster at two CTAs and two stages
    // than at three and one)
    if (xd) {
        int best = 0;
        for (int st = kMaxStages; st >= 2; st--) {
            const size_t b = psweep_smem_bytes(xd, N, m.P, m.nTypes, wps, st, 0, cmp);
            const int r = b <= kMaxSmem ? resident_ctas(k, 32 * m.P, b) : 0;
            if (r > best) { best = per_sm = r; nst = st; smem = b; }
        }
    }
    if (nst == 0 || per_sm < 1) return GATT_ERR_STATE;
    a.nst = nst;
    // 16-byte aligned field starts, even strides (tensor maps)
    if ((reinterpret_cast<uintptr_t>(a.in) & 15) || (c->npts & 1) || (a.in_bstride & 1)) return GATT_ERR_STATE;
    CUtensorMap map, omap;
    memset(&map, 0, sizeof(map));
    memset(&omap, 0, sizeof(omap));
    if (xd) {
        // {row in chunk, line, chunk of 16 rows, field slot, member}, 128-byte swizzle: a box
        // {16, 32, N/16} is one tile of 32 lines
        if ((N & 15) || (reinterpret_cast<uintptr_t>(a.out) & 15) || (a.out_bstride & 1)) return GATT_ERR_STATE;
        EncodeTiledFn enc = encode_tiled();
        if (!enc) return GATT_ERR_STATE;
        // the output map of warp stores copies one 16-row chunk (a box of {16, 32, 1})
        a.xchunk_store = nst > 1 && c->x_wstore;
        auto xmap = [&](CUtensorMap *mp, const double *base, const int *slots, long long bstride, bool chunk) {
            int nslots = 1;
            for (int f = 0; f < a.nf; f++) nslots = std::max(nslots, slots[f] + 1);
            const long long mstride = nmembers > 1 ? bstride : (long long)nslots * c->npts;
            cuuint64_t dims[5] = {16, (cuuint64_t)a.nlines, (cuuint64_t)(N / 16), (cuuint64_t)nslots,
                                  (cuuint64_t)nmembers};
            cuuint64_t strides[4] = {(cuuint64_t)N * 8, 128, (cuuint64_t)c->npts * 8, (cuuint64_t)mstride * 8};
            cuuint32_t box[5] = {16, (cuuint32_t)kLanes, chunk ? 1u : (cuuint32_t)(N / 16), 1, 1};
            cuuint32_t estr[5] = {1, 1, 1, 1, 1};
            return enc(mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double *>(base), dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        };
        if (!xmap(&map, a.in, a.in_slot, a.in_bstride, false) ||
            !xmap(&omap, a.out, a.out_slot, a.out_bstride, a.xchunk_store != 0))
            return GATT_ERR_STATE;
    } else {
        // one box of N rows, or two of N/2 for lines past the copy engine's 256-row box
        if (N > 512 || (N > 256 && (N & 1)) || (c->nx & 1)) return GATT_ERR_STATE;
        a.box2 = N > 256 ? N / 2 : 0;
        EncodeTiledFn enc = encode_tiled();
        if (!enc) return GATT_ERR_STATE;
        int nslots = 1;
        for (int f = 0; f < a.nf; f++) {
            nslots = std::max(nslots, a.in_slot[f] + 1);
            if (m1) nslots = std::max(nslots, a.in_slot1[f] + 1);
        }
        const long long mstride = nmembers > 1 ? a.in_bstride : (long long)nslots * c->npts;
        cuuint64_t dims[5] = {(cuuint64_t)c->nx, (cuuint64_t)c->ny, (cuuint64_t)c->nz, (cuuint64_t)nslots,
                              (cuuint64_t)nmembers};
        cuuint64_t strides[4] = {(cuuint64_t)c->nx * 8, (cuuint64_t)c->nx * c->ny * 8, (cuuint64_t)c->npts * 8,
                                 (cuuint64_t)mstride * 8};
        const int brows = a.box2 ? a.box2 : N;
        // map of direction dd: a box of 32 x-points by `brows` rows of its lines
        auto yzmap = [&](CUtensorMap *mp, int dd) {
            cuuint32_t box[5] = {(cuuint32_t)kLanes, (cuuint32_t)(dd == 1 ? brows : 1), (cuuint32_t)(dd == 2 ? brows : 1),
                                 1, 1};
            cuuint32_t estr[5] = {1, 1, 1, 1, 1};
            return enc(mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double *>(a.in), dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        };
        if (!yzmap(&map, d)) return GATT_ERR_STATE;
        if (m1 && !yzmap(&omap, 2)) return GATT_ERR_STATE;  // part 1: the z lines
    }
    if (xd && c->x_order && a.nf > 1) {
        // x tiles field-inner, last tile first: the cursor's fast index runs over the fields
        a.xorder = 1; a.xtiles = a.ntiles;
        a.ntiles = a.nf; a.nf = a.xtiles;
        a.fd_ntiles = make_fastdiv(a.ntiles); a.fd_nf = make_fastdiv(a.nf);
    }
    const int grid = std::min(a.njobs, per_sm * c->nsm);
    void *args[] = {&a, &map, &omap};
    TRY(before_launch(c, cls));
    CU(cudaLaunchKernel(k, dim3(grid), dim3(32 * m.P), args, smem, c->stream));
    if (a.mc_acc) c->mc_done = true;
    return after_launch(c);
}

// Run one compact solve (direction d, coefficient kind) over nf fields.
// in/out are set bases with per-member strides; slots index fields inside a set.
// blend_dt: device dt for the filter blend (NULL = use `blend`).
int sweep(gatt_ctx *c, int d, int kind, const double *in, long long in_bs, const int *in_slots,
          double *out, long long out_bs, const int *out_slots, int nf, int nmembers, double blend,
          const double *blend_dt, int cls = PC_OTHER, const StateSet *mc_ref = nullptr)
{
    const DevDir &m = c->mat[d][kind];
    if (!m.set || !c->lt_set[d]) return fail(GATT_ERR_STATE, "matrices not set for this direction");
    if (c->lt_max[d] >= m.nTypes) return fail(GATT_ERR_STATE, "line types exceed this matrix set's nTypes");
    if (nf > 16) return fail(GATT_ERR_BADARG, "too many fields in one sweep");
    SweepArgs a;
    memset(&a, 0, sizeof(a));
    a.in = in; a.out = out; a.in_bstride = in_bs; a.out_bstride = out_bs; a.npts = c->npts;
    for (int f = 0; f < nf; f++) { a.in_slot[f] = in_slots[f]; a.out_slot[f] = out_slots[f]; }
    a.nx = c->nx; a.ny = c->ny; a.nz = c->nz;
    a.N = m.rows; a.Nreal = m.N; a.nlines = nlines(c, d);
    a.es = d == 1 ? c->nx : (long long)c->nx * c->ny;
    a.os = d == 1 ? (long long)c->nx * c->ny : c->nx;
    a.tiles_per_row = (c->nx + kLanes - 1) / kLanes;
    a.Rm = m.Rm; a.Q = m.Q; a.W = m.W; a.Wp = m.Wp; a.P = m.P;
    a.ltype = c->ltype[d];
    a.blend = blend; a.blend_dt = blend_dt; a.blend_fct = c->fct;
    a.epi = (blend_dt != nullptr || blend > 0) ? EPI_BLEND : EPI_STORE;
    a.dir = d;
    a.nf = nf;
    a.ntiles = d == 0 ? (a.nlines + kLanes - 1) / kLanes : a.tiles_per_row * (d == 1 ? c->nz : c->ny);
    a.njobs = a.ntiles * nf * nmembers;
    a.fd_ntiles = make_fastdiv(a.ntiles); a.fd_nf = make_fastdiv(nf); a.fd_tpr = make_fastdiv(a.tiles_per_row);
    a.err = c->d_err;
    a.ntypes = m.nTypes;
    if (mc_ref && d > 0) {  // the max-change epilogue: only the pipelined y/z solver has it
        a.mc_acc = c->acc; a.mc_ref = mc_ref->v[0]; a.mc_ref_bstride = mc_ref->bstride;
    }
    if (m.family == FAM_PIPE && m.rpb) {
        int r = launch_psweep(c, m, d, a, nmembers, cls);
        if (r != GATT_ERR_STATE) return r;  // GATT_ERR_STATE: layout not expressible, use k_rsweep
        // padded lines: only the pipelined solver zero-fills past the grid edge
        if (m.rows != m.N || m.P > kMaxP)
            return fail(GATT_ERR_STATE, "padded or long lines need the pipelined solver (layout refused)");
    }
    a.stage = !m.rpb && sweep_smem(m.N, m.P, m.nR, m.Wp, true) <= kMaxSmem;
    const size_t smem = m.rpb ? (size_t)3 * m.P * kLanes * sizeof(double) : sweep_smem(m.N, m.P, m.nR, m.Wp, a.stage);
    void *k = m.rpb ? reg_kernel(false, d == 0, m.periodic != 0, m.nR)
                    : sweep_kernel(d == 0, m.periodic != 0, m.nR, m.P > 4);
    if (k && smem <= kMaxSmem && m.N >= 2) {
        dim3 grid(d == 0 ? (a.nlines + kLanes - 1) / kLanes
                         : a.tiles_per_row * (d == 1 ? c->nz : c->ny),
                  nf, nmembers);
        void *args[] = {&a};
        TRY(before_launch(c, cls));
        CU(cudaLaunchKernel(k, grid, dim3(32 * m.P), args, smem, c->stream));
        return after_launch(c);
    }
    // long lines: global-memory variant, out of place through the scratch field
    for (int b = 0; b < nmembers; b++) {
        for (int f = 0; f < nf; f++) {
            SweepArgs g = a;
            g.in = in + b * in_bs; g.in_bstride = 0; g.in_slot[0] = in_slots[f];
            g.out = c->tmp; g.out_bstride = 0; g.out_slot[0] = 0;
            g.es = d == 0 ? 1 : a.es;
            dim3 grid((a.nlines + 127) / 128, 1, 1);
            TRY(before_launch(c, cls));
            if (m.periodic) k_sweep_global<true><<<grid, 128, 0, c->stream>>>(g, m.nR);
            else k_sweep_global<false><<<grid, 128, 0, c->stream>>>(g, m.nR);
            TRY(after_launch(c));
            TRY(before_launch(c, cls));
            k_copy<<<grid_for(c, c->npts), kBlock, 0, c->stream>>>(out + b * out_bs + (long long)out_slots[f] * c->npts,
                                                                  c->tmp, c->npts);
            TRY(after_launch(c));
        }
    }
    return GATT_OK;
}

// The y and z derivative sweeps of nf fields (input slots sy / sz, output slots oy / oz),
// in one launch of the pipelined solver where both directions' sets allow it: x-tile column
// by column, each field's y tiles and then its z tiles, which find the column's field in L2
// (128^3: a column of one field is 4 MB).  Otherwise two launches.
int sweep_yz(gatt_ctx *c, const double *in, long long in_bs, const int *sy, const int *sz, double *out,
             long long out_bs, const int *oy, const int *oz, int nf, int nmembers, int cls_y, int cls_z, int cls_yz)
{
    const DevDir &my = c->mat[1][0], &mz = c->mat[2][0];
    const bool merge = c->merge_yz && c->is3d && my.set && mz.set && c->lt_set[1] && c->lt_set[2] &&
                       c->lt_max[1] < my.nTypes && c->lt_max[2] < mz.nTypes && my.family == FAM_PIPE &&
                       mz.family == FAM_PIPE && my.rpb && mz.rpb && my.rows == my.N && mz.rows == mz.N &&
                       my.rows == mz.rows && my.P == mz.P && my.nR == mz.nR && my.nR < 6 && my.Wp == mz.Wp &&
                       my.periodic == mz.periodic && my.rows <= 256 && nf <= 16;
    if (merge) {
        SweepArgs a;
        memset(&a, 0, sizeof(a));
        a.in = in; a.out = out; a.in_bstride = in_bs; a.out_bstride = out_bs; a.npts = c->npts;
        for (int f = 0; f < nf; f++) {
            a.in_slot[f] = sy[f]; a.out_slot[f] = oy[f];
            a.in_slot1[f] = sz[f]; a.out_slot1[f] = oz[f];
        }
        a.nx = c->nx; a.ny = c->ny; a.nz = c->nz;
        a.N = my.rows; a.Nreal = my.N; a.nlines = nlines(c, 1);
        a.es = c->nx; a.os = (long long)c->nx * c->ny;   // y lines: x stride nx, outer index z
        a.es1 = (long long)c->nx * c->ny; a.os1 = c->nx;  // z lines: stride nx*ny, outer index y
        a.tiles_per_row = (c->nx + kLanes - 1) / kLanes;
        a.Rm = my.Rm; a.Q = my.Q; a.W = my.W; a.Wp = my.Wp; a.P = my.P;
        a.ltype = c->ltype[1]; a.ntypes = my.nTypes;
        a.Rm1 = mz.Rm; a.Q1 = mz.Q; a.ltype1 = c->ltype[2]; a.ntypes1 = mz.nTypes;
        a.epi = EPI_STORE;
        a.dir = 1;
        a.nf = nf;
        a.parts = 2;
        a.nout0 = c->nz; a.nout1 = c->ny;
        a.ntiles = a.tiles_per_row * (c->nz + c->ny);
        a.njobs = a.ntiles * nf * nmembers;
        a.fd_ntiles = make_fastdiv(a.ntiles); a.fd_nf = make_fastdiv(nf); a.fd_tpr = make_fastdiv(a.tiles_per_row);
        a.fd_nout = make_fastdiv(c->nz + c->ny);
        a.err = c->d_err;
        const int r = launch_psweep(c, my, 1, a, nmembers, cls_yz, &mz);
        if (r != GATT_ERR_STATE) return r;  // GATT_ERR_STATE: layout refused, two launches
    }
    TRY(sweep(c, 1, 0, in, in_bs, sy, out, out_bs, oy, nf, nmembers, 0, nullptr, cls_y));
    return sweep(c, 2, 0, in, in_bs, sz, out, out_bs, oz, nf, nmembers, 0, nullptr, cls_z);
}

// ---------------------------------------------------------------------------
// right-hand side + stage update
// ---------------------------------------------------------------------------

// Tensor map {points, slots, members, 1, 1} of `nslots` fields starting at base[0..nslots)
// (equally spaced, checked) with member stride bstride; false when the layout does not fit the
// copy engine's rules (16-byte aligned start, strides multiples of 16 bytes).
bool pw_map(const gatt_ctx *c, CUtensorMap *map, const double *const *base, int nslots, long long bstride, int nmem)
{
    const long long n = c->npts;
    const long long sstride = nslots > 1 ? (long long)(base[1] - base[0]) : n;
    for (int f = 1; f < nslots; f++)
        if (base[f] != base[0] + f * sstride) return false;
    if ((reinterpret_cast<uintptr_t>(base[0]) & 15) || (n & 1) || (sstride & 1) || sstride < n) return false;
    if (nmem > 1 && ((bstride & 1) || bstride < sstride * nslots)) return false;
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    memset(map, 0, sizeof(*map));
    cuuint64_t dims[5] = {(cuuint64_t)n, (cuuint64_t)nslots, (cuuint64_t)nmem, 1, 1};
    const long long ms = nmem > 1 ? bstride : sstride * nslots;
    cuuint64_t strides[4] = {(cuuint64_t)sstride * 8, (cuuint64_t)ms * 8, (cuuint64_t)ms * nmem * 8,
                             (cuuint64_t)ms * nmem * 8};
    cuuint32_t box[5] = {(cuuint32_t)kPwC, (cuuint32_t)nslots, 1, 1, 1};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double *>(base[0]), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The forcings as the assembly kernels take them, and the box sums of the turbulence
// forcings over stage input q (runForcings: turbulenceGenerator sums its input fields).
Forcings forcing_args(const gatt_ctx *c)
{
    Forcings f = c->fc;
    f.sums = c->fsum;
    f.nx = c->nx;
    f.ny = c->ny;
    return f;
}

int forcing_sums(gatt_ctx *c, const StateSet &q, int nmem)
{
    bool turb = false;
    for (int f = 0; f < c->fc.n; f++) turb |= c->fc.type[f] == FORCE_TURBULENCE;
    if (!turb) return GATT_OK;
    TRY(before_launch(c, PC_OTHER));
    k_forcing_sums<<<dim3(c->fblocks, nmem), 256, 0, c->stream>>>(q, forcing_args(c), c->fpart);
    TRY(after_launch(c));
    TRY(before_launch(c, PC_OTHER));
    k_forcing_final<<<nmem, 32, 0, c->stream>>>(c->fpart, c->fblocks, c->fsum);
    return after_launch(c);
}

// 3-D assembly fed by tensor copies (pwpipe.cuh).  Returns GATT_ERR_STATE without launching
// when a set's layout does not fit the tensor maps; the caller then runs k_assemble3d.
int launch_assemble3d_pipe(gatt_ctx *c, const StateSet &q, const StateSet &q0, const StateSet &out,
                           const FieldSet &delta, const FieldSet &d1, const FieldSet &d2, int mode, int nmem)
{
    if (!c->pw_pipe || (c->npts & 1)) return GATT_ERR_STATE;
    PwArgs a;
    memset(&a, 0, sizeof(a));
    a.n = c->npts;
    a.nchunks = (a.n + kPwC - 1) / kPwC;
    a.njobs = a.nchunks * nmem;
    a.nst = kPwStages;
    a.mode = mode;
    a.use_delta = delta.p && mode_reads_delta(mode);
    a.use_q0 = 0;
    if (mode != RK_STORE_RHS)
        for (int f = 0; f < 5; f++)
            if (q0.v[f] != q.v[f] || q0.bstride != q.bstride) a.use_q0 = 1;
    a.err = c->d_err;
    a.fs = forcing_args(c);
    PwMaps maps;
    memset(&maps, 0, sizeof(maps));
    const double *qb[5], *q0b[5], *d1b[D3_N], *d2b[S3_N], *dlb[5];
    for (int f = 0; f < 5; f++) { qb[f] = q.v[f]; q0b[f] = q0.v[f]; dlb[f] = delta.p ? delta.p + f * delta.npts : nullptr; }
    for (int f = 0; f < D3_N; f++) d1b[f] = d1.p + f * d1.npts;
    for (int f = 0; f < S3_N; f++) d2b[f] = d2.p + f * d2.npts;
    if (!pw_map(c, &maps.m[PW_Q], qb, 5, q.bstride, nmem) || !pw_map(c, &maps.m[PW_D1], d1b, D3_N, d1.bstride, nmem) ||
        !pw_map(c, &maps.m[PW_D2], d2b, S3_N, d2.bstride, nmem))
        return GATT_ERR_STATE;
    if (a.use_q0 && !pw_map(c, &maps.m[PW_Q0], q0b, 5, q0.bstride, nmem)) return GATT_ERR_STATE;
    if (a.use_delta && !pw_map(c, &maps.m[PW_DL], dlb, 5, delta.bstride, nmem)) return GATT_ERR_STATE;
    const size_t smem = pw_smem_bytes(a.nst);
    const int per_sm = resident_ctas((const void *)k_assemble3d_pipe, 2 * kPwC, smem);
    if (per_sm < 1) return GATT_ERR_STATE;
    const long long grid = std::min<long long>(a.njobs, (long long)per_sm * c->nsm);
    TRY(before_launch(c, PC_ASSEMBLE));
    k_assemble3d_pipe<<<(unsigned)grid, 2 * kPwC, smem, c->stream>>>(c->ph, out, delta, a, c->d_params, maps);
    return after_launch(c);
}

// The 3-D assembly + RK4 stage update from gradients d1 and second sweeps d2 (tensor-copy
// fed where the layouts allow, else thread loads).
int assemble3d(gatt_ctx *c, const StateSet &q, const StateSet &q0, const StateSet &out, int mode, int nmem, double *d1,
               double *d2, double *delta)
{
    const long long n = c->npts;
    const FieldSet fd = fset(c, delta, 5), f1 = fset(c, d1, D3_N), f2 = fset(c, d2, S3_N);
    TRY(forcing_sums(c, q, nmem));
    const int pr = launch_assemble3d_pipe(c, q, q0, out, fd, f1, f2, mode, nmem);
    if (pr != GATT_ERR_STATE) return pr;
    TRY(before_launch(c, PC_ASSEMBLE));
    k_assemble3d<<<dim3(grid_for(c, n), nmem), kBlock, 0, c->stream>>>(c->ph, q, q0, out, fd, f1, f2, n, mode,
                                                                      c->d_params, forcing_args(c));
    return after_launch(c);
}

// Launches on the side stream: the context's stream and scratch field exchanged with the
// side stream's for the lifetime of the scope (two streams never share the scratch field).
struct OnSide {
    gatt_ctx *c;
    explicit OnSide(gatt_ctx *cc) : c(cc) { flip(); }
    ~OnSide() { flip(); }
    void flip() { std::swap(c->stream, c->side); std::swap(c->tmp, c->tmp_side); }
};

// The x sweep and the y/z sweeps of one operand set are independent: the x sweep runs on the
// side stream, forked from and joined back into the context's stream, so that each one's
// last partial wave of tiles overlaps the other (not while per-kernel events are recorded).
template <typename F>
int beside(gatt_ctx *c, F &&launch_x)
{
    if (!c->fork_x || c->profiling || !c->side) return launch_x();
    CU(cudaEventRecord(c->ev_fork, c->stream));
    CU(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    int r;
    {
        OnSide on(c);
        r = launch_x();
    }
    TRY(r);
    CU(cudaEventRecord(c->ev_join, c->side));
    return GATT_OK;
}
int join_side(gatt_ctx *c)
{
    if (!c->fork_x || c->profiling || !c->side) return GATT_OK;
    CU(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return GATT_OK;
}

// nseq2d/nseq3d on stage input q, fused with the RK4 update into out (mode).
int rhs_stage(gatt_ctx *c, const StateSet &q, const StateSet &q0, const StateSet &out, int mode, int nmem,
              double *d1, double *tq, double *d2, double *delta, bool assemble = true)
{
    const long long n = c->npts;
    const double *qin = q.v[0];
    const long long qbs = q.bstride;
    const StepParams *sp = c->d_params;
    if (c->is3d) {
        const long long bd1 = D3_N * n, btq = T3_N * n, bd2 = S3_N * n;
        // first derivatives of U, V, W, R, E (nseq.F90:178-216)
        const int fin[5] = {0, 1, 2, 3, 4};
        const int ox[5] = {D3_UX, D3_VX, D3_WX, D3_RX, D3_EX};
        const int oy[5] = {D3_UY, D3_VY, D3_WY, D3_RY, D3_EY};
        const int oz[5] = {D3_UZ, D3_VZ, D3_WZ, D3_RZ, D3_EZ};
        TRY(beside(c, [&] { return sweep(c, 0, 0, qin, qbs, fin, d1, bd1, ox, 5, nmem, 0, nullptr, PC_D1X); }));
        TRY(sweep_yz(c, qin, qbs, fin, fin, d1, bd1, oy, oz, 5, nmem, PC_D1Y, PC_D1Z, PC_D1YZ));
        TRY(join_side(c));
        TRY(before_launch(c, PC_VISC));
        if (c->visc_v2 && !(n & 1) && !(q.bstride & 1) && !((uintptr_t)q.v[4] & 15) && !((uintptr_t)d1 & 15) &&
            !((uintptr_t)tq & 15))
            k_visc3d_v2<<<dim3(grid_for(c, n / 2), nmem), kBlock, 0, c->stream>>>(c->ph, q, fset(c, d1, D3_N),
                                                                             fset(c, tq, T3_N), n);
        else
            k_visc3d<<<dim3(grid_for(c, n), nmem), kBlock, 0, c->stream>>>(c->ph, q, fset(c, d1, D3_N),
                                                                          fset(c, tq, T3_N), n);
        TRY(after_launch(c));
        // second sweeps (nseq.F90:241-306)
        const int ix[4] = {T3_XX, T3_XY, T3_XZ, T3_QX}, sx[4] = {S3_TXXX, S3_TXYX, S3_TXZX, S3_HTX};
        const int iy[4] = {T3_XY, T3_YY, T3_YZ, T3_QY}, sy[4] = {S3_TXYY, S3_TYYY, S3_TYZY, S3_HTY};
        const int iz[4] = {T3_XZ, T3_YZ, T3_ZZ, T3_QZ}, sz[4] = {S3_TXZZ, S3_TYZZ, S3_TZZZ, S3_HTZ};
        TRY(beside(c, [&] { return sweep(c, 0, 0, tq, btq, ix, d2, bd2, sx, 4, nmem, 0, nullptr, PC_D2X); }));
        TRY(sweep_yz(c, tq, btq, iy, iz, d2, bd2, sy, sz, 4, nmem, PC_D2Y, PC_D2Z, PC_D2YZ));
        TRY(join_side(c));
        if (!assemble) return GATT_OK;  // the gradients and second sweeps only (tangent / adjoint)
        return assemble3d(c, q, q0, out, mode, nmem, d1, d2, delta);
    }
    const long long bd1 = D2_N * n, btq = T2_N * n, bd2 = S2_N * n;
    const int fin[4] = {0, 1, 3, 4};
    const int ox[4] = {D2_UX, D2_VX, D2_RX, D2_EX};
    const int oy[4] = {D2_UY, D2_VY, D2_RY, D2_EY};
    TRY(beside(c, [&] { return sweep(c, 0, 0, qin, qbs, fin, d1, bd1, ox, 4, nmem, 0, nullptr, PC_D1X); }));
    TRY(sweep(c, 1, 0, qin, qbs, fin, d1, bd1, oy, 4, nmem, 0, nullptr, PC_D1Y));
    TRY(join_side(c));
    TRY(before_launch(c, PC_VISC));
    k_visc2d<<<dim3(grid_for(c, n), nmem), kBlock, 0, c->stream>>>(c->ph, q, fset(c, d1, D2_N), fset(c, tq, T2_N), n);
    TRY(after_launch(c));
    const int ix[3] = {T2_XY, T2_XX, T2_QX}, sx[3] = {S2_TXYX, S2_TXXX, S2_HTX};
    const int iy[3] = {T2_XY, T2_YY, T2_QY}, sy[3] = {S2_TXYY, S2_TYYY, S2_HTY};
    TRY(beside(c, [&] { return sweep(c, 0, 0, tq, btq, ix, d2, bd2, sx, 3, nmem, 0, nullptr, PC_D2X); }));
    TRY(sweep(c, 1, 0, tq, btq, iy, d2, bd2, sy, 3, nmem, 0, nullptr, PC_D2Y));
    TRY(join_side(c));
    TRY(before_launch(c, PC_ASSEMBLE));
    k_assemble2d<<<dim3(grid_for(c, n), nmem), kBlock, 0, c->stream>>>(
        c->ph, q, q0, out, fset(c, delta, 5), fset(c, d1, D2_N), fset(c, tq, T2_N), fset(c, d2, S2_N), n, mode, sp,
        forcing_args(c));
    return after_launch(c);
}

// ---------------------------------------------------------------------------
// boundary program
// ---------------------------------------------------------------------------

int check_box(const gatt_ctx *c, const int *b)
{
    if (b[0] < 1 || b[1] > c->nx || b[0] > b[1] || b[2] < 1 || b[3] > c->ny || b[2] > b[3] || b[4] < 1 ||
        b[5] > c->nz || b[4] > b[5])
        return fail(GATT_ERR_BADARG, "boundary box outside the grid: [" + std::to_string(b[0]) + " " +
                                         std::to_string(b[1]) + " " + std::to_string(b[2]) + " " +
                                         std::to_string(b[3]) + " " + std::to_string(b[4]) + " " +
                                         std::to_string(b[5]) + "]");
    return GATT_OK;
}

// getNeumannIndices (nseq.F90:520-550)
void neumann_box(const int *in, int dir, int len, int *out)
{
    for (int q = 0; q < 6; q++) out[q] = in[q];
    switch (dir) {
    case 1: out[1] += len; break;
    case 2: out[0] -= len; break;
    case 3: out[3] += len; break;
    case 4: out[2] -= len; break;
    case 5: out[5] += len; break;
    case 6: out[4] -= len; break;
    }
}

int build_bc_program(gatt_ctx *c)
{
    std::vector<BcOp> ops;
    auto mk = [&](int code, int var, const int *box) {
        BcOp o;
        memset(&o, 0, sizeof(o));
        o.code = code; o.var = var;
        for (int q = 0; q < 6; q++) o.box[q] = box[q];
        return o;
    };
    auto row = [&](const HostBC &h, int i, int *box) {
        for (int q = 0; q < 6; q++) box[q] = h.ind[i + (size_t)h.n * q];
    };
    const int NL = (int)c->coef1.size(), N2 = (int)c->coef2.size();
    const int order[4] = {GATT_VAR_U, GATT_VAR_V, GATT_VAR_W, GATT_VAR_E};
    int box[6], ext[6];
    // Dirichlet (nseq.F90:357-373)
    for (int v : order) {
        const HostBC &h = c->bc[GATT_BC_DIRICHLET][v];
        for (int i = 0; i < h.n; i++) {
            row(h, i, box); TRY(check_box(c, box));
            BcOp o = mk(OP_SET, v, box); o.val = h.val[i]; ops.push_back(o);
        }
    }
    {
        const HostBC &h = c->bc[GATT_BC_DIRICHLET][GATT_VAR_R];
        for (int i = 0; i < h.n; i++) {
            row(h, i, box); TRY(check_box(c, box));
            BcOp o = mk(OP_DIR_P, GATT_VAR_R, box); o.val = h.val[i]; ops.push_back(o);
        }
    }
    // Neumann (kind 1, nseq.F90:377-400) and null second derivative (kind 2, :491-513)
    auto neumann_lists = [&](int kind, int len, int coefsel) -> int {
        if (len < 1 && (c->bc[kind][0].n || c->bc[kind][1].n || c->bc[kind][2].n || c->bc[kind][3].n ||
                        c->bc[kind][4].n))
            return fail(GATT_ERR_STATE, "Neumann coefficients not set");
        for (int v : order) {
            const HostBC &h = c->bc[kind][v];
            for (int i = 0; i < h.n; i++) {
                row(h, i, box);
                const int d = h.dirs[i];
                if (d < 1 || d > 6) return fail(GATT_ERR_BADARG, "Neumann direction must be 1..6");
                neumann_box(box, d, len, ext); TRY(check_box(c, ext));
                BcOp o = mk(OP_NEU, v, ext); o.dir = d; o.len = len; o.coef = coefsel; ops.push_back(o);
            }
        }
        const HostBC &h = c->bc[kind][GATT_VAR_R];
        for (int i = 0; i < h.n; i++) {
            row(h, i, box);
            const int d = h.dirs[i];
            if (d < 1 || d > 6) return fail(GATT_ERR_BADARG, "Neumann direction must be 1..6");
            neumann_box(box, d, len, ext); TRY(check_box(c, ext)); TRY(check_box(c, box));
            ops.push_back(mk(OP_P_LOAD, 3, ext));
            BcOp o = mk(OP_P_NEU, 3, ext); o.dir = d; o.len = len; o.coef = coefsel; ops.push_back(o);
            ops.push_back(mk(OP_R_FROM_P, 3, box));
        }
        return GATT_OK;
    };
    TRY(neumann_lists(GATT_BC_NEUMANN, NL, 0));
    // corners (nseq.F90:402-488)
    for (int i = 0; i < c->cN; i++) {
        for (int q = 0; q < 6; q++) box[q] = c->cL[i + (size_t)c->cN * q];
        TRY(check_box(c, box));
        int cd[3] = {c->cD[i], c->cD[i + c->cN], c->cD[i + 2 * c->cN]};
        const int nd = std::abs(cd[0]) + std::abs(cd[1]) + std::abs(cd[2]);
        if (nd == 0) return fail(GATT_ERR_BADARG, "corner without direction");
        if (NL < 1) return fail(GATT_ERR_STATE, "Neumann coefficients not set");
        if (c->cAd[i] == 1) {
            ops.push_back(mk(OP_CORNER_E0, 4, box));
            for (int a = 0; a < 3; a++) {
                if (cd[a] != 1 && cd[a] != -1) continue;
                const int d = cd[a] == 1 ? 2 * a + 1 : 2 * a + 2;
                neumann_box(box, d, NL, ext); TRY(check_box(c, ext));
                ops.push_back(mk(OP_P_FROM_E, 4, ext));
                BcOp o = mk(OP_P_NEU, 4, ext); o.dir = d; o.len = NL; o.coef = 0; ops.push_back(o);
                ops.push_back(mk(OP_E_ADD_P, 4, box));
            }
            BcOp o = mk(OP_E_DIV, 4, box); o.aux = nd; ops.push_back(o);
        }
        ops.push_back(mk(OP_R0, 3, box));
        for (int a = 0; a < 3; a++) {
            if (cd[a] != 1 && cd[a] != -1) continue;
            const int d = cd[a] == 1 ? 2 * a + 1 : 2 * a + 2;
            neumann_box(box, d, NL, ext); TRY(check_box(c, ext));
            ops.push_back(mk(OP_P_LOAD, 3, ext));
            BcOp o = mk(OP_P_NEU, 3, ext); o.dir = d; o.len = NL; o.coef = 0; ops.push_back(o);
            ops.push_back(mk(OP_R_ADD_P, 3, box));
        }
        BcOp o = mk(OP_R_DIV_E, 3, box); o.aux = nd; ops.push_back(o);
    }
    TRY(neumann_lists(GATT_BC_SECOND, N2, 1));
    // disturbances (runDisturbances.F90)
    long long hold_len = 0;
    std::vector<int> hold_sig;
    for (const Dist &d : c->dists) {
        TRY(check_box(c, d.ind));
        if (d.type == GATT_DIST_HOLD_INLET) {
            BcOp o = mk(OP_HOLD, 0, d.ind);
            o.aux = d.par > 0.5 ? 5 : 4;
            const long long n = (long long)(d.ind[1] - d.ind[0] + 1) * (d.ind[3] - d.ind[2] + 1) * (d.ind[5] - d.ind[4] + 1);
            if (hold_len + o.aux * n > INT_MAX) return fail(GATT_ERR_BADARG, "holdInlet boxes too large");
            o.xoff = (int)hold_len;
            hold_len += o.aux * n;
            hold_sig.insert(hold_sig.end(), d.ind, d.ind + 6);
            hold_sig.push_back(o.aux);
            ops.push_back(o);
        } else {
            BcOp o = mk(d.type == GATT_DIST_PERIODIC_SINE ? OP_SINE : OP_LID, d.var, d.ind);
            o.xoff = d.xoff; o.val = d.par; ops.push_back(o);
        }
    }
    // phases: an op joins the running phase unless it reads or writes a field point that an op
    // of the phase writes, or writes one that it reads (fields U, V, W, R, E and the P scratch;
    // boxes compared as index ranges, the Neumann ones over their extended box)
    {
        auto access = [](const BcOp &o, unsigned &rd, unsigned &wr) {
            const unsigned U = 1u << o.var, R = 1u << 3, E = 1u << 4, P = 1u << 5;
            rd = wr = 0;
            switch (o.code) {
            case OP_SET: case OP_LID: wr = U; break;
            case OP_SINE: rd = wr = U; break;
            case OP_HOLD: rd = wr = 0x17u | (o.aux == 5 ? R : 0u); break;  // U V W E (R)
            case OP_DIR_P: rd = E; wr = R; break;
            case OP_NEU: rd = wr = U; break;
            case OP_P_LOAD: rd = R | E; wr = P; break;
            case OP_P_NEU: rd = wr = P; break;
            case OP_R_FROM_P: rd = P | E; wr = R; break;
            case OP_CORNER_E0: wr = E; break;
            case OP_P_FROM_E: rd = E; wr = P; break;
            case OP_E_ADD_P: rd = E | P; wr = E; break;
            case OP_E_DIV: rd = wr = E; break;
            case OP_R0: wr = R; break;
            case OP_R_ADD_P: rd = R | P; wr = R; break;
            case OP_R_DIV_E: rd = R | E; wr = R; break;
            default: rd = wr = 0x3f; break;
            }
        };
        auto overlap = [](const BcOp &a, const BcOp &b) {
            for (int q = 0; q < 3; q++)
                if (a.box[2 * q + 1] < b.box[2 * q] || b.box[2 * q + 1] < a.box[2 * q]) return false;
            return true;
        };
        size_t start = 0;
        for (size_t i = 0; i < ops.size(); i++) {
            unsigned rb, wb;
            access(ops[i], rb, wb);
            bool dep = false;
            for (size_t k = start; k < i && !dep; k++) {
                unsigned ra, wa;
                access(ops[k], ra, wa);
                dep = ((wa & (rb | wb)) || (ra & wb)) && overlap(ops[k], ops[i]);
            }
            if (dep) {
                ops[i - 1].sync = 1;
                start = i;
            }
        }
        if (!ops.empty()) ops.back().sync = 1;
    }
    // adjoint tape offsets (base values of the nonlinear ops, per box point)
    long long tape = 0;
    for (BcOp &o : ops) {
        const int tw = bc_tape_width(o.code);
        o.tape = tape;
        if (o.code != OP_NEU && o.code != OP_P_NEU && tw > 0)
            tape += (long long)tw * (o.box[1] - o.box[0] + 1) * (o.box[3] - o.box[2] + 1) * (o.box[5] - o.box[4] + 1);
    }
    c->tape_len = tape;
    c->bc_points = 0;
    for (const BcOp &o : ops) {
        const long long ni = o.box[1] - o.box[0] + 1, nj = o.box[3] - o.box[2] + 1, nk = o.box[5] - o.box[4] + 1;
        c->bc_points += (o.code == OP_NEU || o.code == OP_P_NEU) ? (o.dir <= 2 ? nj * nk : o.dir <= 4 ? ni * nk : ni * nj)
                                                                 : ni * nj * nk;
    }
    cudaFree(c->d_ops); c->d_ops = nullptr;
    cudaFree(c->d_coef1); c->d_coef1 = nullptr;
    cudaFree(c->d_coef2); c->d_coef2 = nullptr;
    cudaFree(c->d_xs); c->d_xs = nullptr;
    c->nops = (int)ops.size();
    if (!ops.empty()) {
        CU(cudaMalloc(&c->d_ops, ops.size() * sizeof(BcOp)));
        CU(cudaMemcpy(c->d_ops, ops.data(), ops.size() * sizeof(BcOp), cudaMemcpyHostToDevice));
    }
    if (!c->coef1.empty()) {
        CU(cudaMalloc(&c->d_coef1, c->coef1.size() * sizeof(double)));
        CU(cudaMemcpy(c->d_coef1, c->coef1.data(), c->coef1.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (!c->coef2.empty()) {
        CU(cudaMalloc(&c->d_coef2, c->coef2.size() * sizeof(double)));
        CU(cudaMemcpy(c->d_coef2, c->coef2.data(), c->coef2.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (!c->distx.empty()) {
        CU(cudaMalloc(&c->d_xs, c->distx.size() * sizeof(double)));
        CU(cudaMemcpy(c->d_xs, c->distx.data(), c->distx.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (hold_sig != c->hold_sig || (hold_len > 0 && !c->d_hold)) {  // a new hold layout: saved afresh
        cudaFree(c->d_hold); c->d_hold = nullptr;
        if (hold_len > 0) CU(cudaMalloc(&c->d_hold, sizeof(double) * (size_t)hold_len * c->nb));
        c->hold_len = hold_len;
        c->hold_sig = hold_sig;
        c->hold_saved = false;
    }
    c->bc_dirty = false;
    return GATT_OK;
}

// The program as the kernels take it, at time t + tfac dt of the step parameters on the device
BcProgram bc_program(const gatt_ctx *c, double tfac)
{
    BcProgram pg;
    pg.ops = c->d_ops; pg.nops = c->nops; pg.coef1 = c->d_coef1; pg.coef2 = c->d_coef2; pg.xs = c->d_xs;
    pg.gamma = c->ph.gamma; pg.nx = c->nx; pg.ny = c->ny; pg.nz = c->nz;
    pg.sp = c->d_params; pg.tfac = tfac; pg.tfix = 0.0;
    pg.hold = c->d_hold; pg.hstride = c->hold_len; pg.hold_save = 0;
    return pg;
}

// holdInlet puts back what the first boundary-condition call kept (main.F90:112 makes that
// call on the initial state): steps need it made
int check_hold(gatt_ctx *c)
{
    if (c->bc_dirty) TRY(build_bc_program(c));
    if (c->hold_len > 0 && !c->hold_saved)
        return fail(GATT_ERR_STATE, "holdInlet: call gatt_apply_bc on the initial state before stepping");
    return GATT_OK;
}

void invalidate_graphs(gatt_ctx *c)
{
    if (c->stream && (c->graph[0] || c->graph[1])) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < 2; i++) {
        if (c->graph[i]) cudaGraphExecDestroy(c->graph[i]);
        c->graph[i] = nullptr;
    }
}

// Cluster size for a boundary-program kernel: 16 CTAs (non-portable size) when the GPU can
// schedule such a cluster of 512-thread CTAs, else 8, else 0 (one CTA per member).
int bc_cluster_size(const void *k)
{
    if (cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) cudaGetLastError();
    for (int cs : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cs);
        cfg.blockDim = dim3(512);
        cfg.dynamicSmemBytes = 48 * 1024;  // the staged ops, at most
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) == cudaSuccess && n >= 1) return cs;
        cudaGetLastError();
    }
    return 0;
}

// Cluster sizes of the boundary-program kernels (GATT_BC_CLUSTER=0: one CTA per member).
// Host queries only: called at creation.
int choose_bc_cluster(gatt_ctx *c)
{
    c->bc_cluster = c->bc_cluster_rec = c->bc_cluster_tl = c->bc_cluster_adj = 0;
    const char *e = getenv("GATT_BC_CLUSTER");
    if (e && !strcmp(e, "0")) return GATT_OK;
    c->bc_cluster = bc_cluster_size((const void *)k_bc_cluster);
    c->bc_cluster_rec = bc_cluster_size((const void *)k_bc_rec_cluster);
    c->bc_cluster_tl = bc_cluster_size((const void *)k_bc_tl_cluster);
    c->bc_cluster_adj = bc_cluster_size((const void *)k_bc_adj_cluster);
    return GATT_OK;
}

// Launch a boundary-program kernel for nmem members: the cluster form with cs CTAs per
// member, cs the largest power of two up to the schedulable size cs_max that keeps the
// clusters of all members within the SMs and gives every CTA about 2048 point updates (small
// or many-member programs gain nothing from more CTAs and pay a barrier per op); with cs < 2
// the one-CTA form.
template <typename... KArgs, typename... Args>
int launch_bc(gatt_ctx *c, void (*kblock)(KArgs...), void (*kcluster)(KArgs...), int cs_max, int nmem, size_t smem,
              Args &&...args)
{
    const long long by_work = (c->bc_points + 2047) / 2048;
    const long long by_sms = std::max(1, c->nsm / std::max(1, nmem));
    int cs = 1;
    while (cs * 2 <= cs_max && cs * 2 <= by_work && cs * 2 <= by_sms) cs *= 2;
    if (cs >= 2) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(nmem * cs);
        cfg.blockDim = dim3(512);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = c->stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cs;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        CU(cudaLaunchKernelEx(&cfg, kcluster, std::forward<Args>(args)...));
    } else {
        kblock<<<nmem, 512, smem, c->stream>>>(std::forward<Args>(args)...);
    }
    return GATT_OK;
}

// applyBoundCond at time t + tfac dt of the step (timeIntegration.F90 passes t + dt/2 or
// t + dt by stage); fixed: at time tfix, keeping the holdInlet values on a first call
int apply_bc(gatt_ctx *c, const StateSet &q, int nmem, double tfac, bool fixed = false, double tfix = 0.0)
{
    if (c->bc_dirty) TRY(build_bc_program(c));
    if (c->nops == 0) return GATT_OK;
    BcProgram pg = bc_program(c, tfac);
    if (fixed) {
        pg.sp = nullptr; pg.tfix = tfix;
        pg.hold_save = c->hold_saved ? 0 : 1;
    } else if (c->hold_len > 0 && !c->hold_saved) {
        return fail(GATT_ERR_STATE, "holdInlet: call gatt_apply_bc on the initial state before stepping");
    }
    const size_t smem = c->nops <= kBcStagedOps ? (size_t)c->nops * sizeof(BcOp) : 0;  // staged ops
    TRY(before_launch(c, PC_BC));
    TRY(launch_bc(c, k_bc, k_bc_cluster, c->bc_cluster, nmem, smem, pg, q, c->P, (long long)c->npts));
    return after_launch(c);
}

// applyFilters2D/3D in place on set q (derivs.F90:303-552)
// With mc_ref, the last filtered direction also reduces the max-change against mc_ref into
// c->acc (when its launch can: c->mc_done tells).
int filter_set(gatt_ctx *c, const StateSet &q, int nmem, double blend, const double *blend_dt,
               const StateSet *mc_ref = nullptr)
{
    const int f3[5] = {0, 1, 2, 3, 4}, f2[4] = {0, 1, 3, 4};
    const int *fl = c->is3d ? f3 : f2;
    const int nf = c->is3d ? 5 : 4;
    const int ndir = c->is3d ? 3 : 2;
    int last = -1;
    for (int d = 0; d < ndir; d++)
        if (c->filt[d]) last = d;
    c->mc_done = false;
    // a filter direction after another takes the fields in the reverse order: its first
    // fields are the ones the previous direction wrote last (still in L2)
    const int r3[5] = {4, 3, 2, 1, 0}, r2[4] = {4, 3, 1, 0};
    const int *rl = c->is3d ? r3 : r2;
    auto chain = [&](const int *fwd, const int *rev, int n) -> int {
        int nth = 0;
        for (int d = 0; d < ndir; d++) {
            if (!c->filt[d]) continue;
            const int *sl = (c->fz_rev && (nth++ & 1)) ? rev : fwd;
            TRY(sweep(c, d, 1, q.v[0], q.bstride, sl, q.v[0], q.bstride, sl, n, nmem, blend, blend_dt, PC_FX + d,
                      d == last ? mc_ref : nullptr));
        }
        return GATT_OK;
    };
    if (!c->fork_x || c->profiling || !c->side) return chain(fl, rl, nf);
    // the fields' filters are independent -- U, V (and W) on the context's stream, R, E beside
    // them on the side stream, so that each direction's last partial wave overlaps the other
    // chain's launches
    const int fa3[3] = {0, 1, 2}, ra3[3] = {2, 1, 0}, fa2[2] = {0, 1}, ra2[2] = {1, 0}, fb[2] = {3, 4}, rb[2] = {4, 3};
    const int *fa = c->is3d ? fa3 : fa2, *ra = c->is3d ? ra3 : ra2;
    const int na = c->is3d ? 3 : 2;
    CU(cudaEventRecord(c->ev_fork, c->stream));
    CU(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    int r;
    {
        OnSide on(c);
        r = chain(fb, rb, 2);
    }
    TRY(r);
    CU(cudaEventRecord(c->ev_join, c->side));
    TRY(chain(fa, ra, na));
    CU(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return GATT_OK;
}

int check_ready(const gatt_ctx *c, bool need_filter)
{
    if (!c->phys_set) return fail(GATT_ERR_STATE, "gatt_set_physics not called");
    const int ndir = c->is3d ? 3 : 2;
    for (int d = 0; d < ndir; d++) {
        if (!c->mat[d][0].set || !c->lt_set[d]) return fail(GATT_ERR_STATE, "derivative matrices missing for a direction");
        if (c->lt_max[d] >= c->mat[d][0].nTypes) return fail(GATT_ERR_STATE, "block types exceed the derivative nTypes");
        if (need_filter && c->filt[d] && !c->mat[d][1].set)
            return fail(GATT_ERR_STATE, "filter matrices missing for a filtered direction");
        if (need_filter && c->filt[d] && c->lt_max[d] >= c->mat[d][1].nTypes)
            return fail(GATT_ERR_STATE, "block types exceed the filter nTypes");
    }
    return GATT_OK;
}

// The whole of main.F90:255-420 for all members, enqueued on the stream.
int step_body(gatt_ctx *c)
{
    const StateSet q0 = state_set(c, 0), qs = state_set(c, 1);
    StateSet qst = qs;  // stage BC set: in 2-D RK4_2D hands the caller's W to applyBoundCond
    if (!c->is3d) qst.v[2] = q0.v[2];
    const int nm = c->nb;
    CU(cudaMemsetAsync(c->acc, 0, sizeof(unsigned long long) * 5 * nm, c->stream));
    // the time integrator (main.F90:304-352 by timeStepping): every stage forms the RHS of its
    // input, updates the stage state and applies the boundary conditions
    if (c->time_stepping == 2) {  // EULER_2D/3D (timeIntegration.F90:158-223, 500-567)
        TRY(rhs_stage(c, q0, q0, qs, RK_EULER, nm, c->d1, c->tq, c->d2, c->delta));
        TRY(apply_bc(c, qst, nm, c->is3d ? 0.0 : 1.0));  // EULER_3D passes t, EULER_2D t + dt
    } else if (c->time_stepping == 3) {  // SSPRK3_2D/3D (timeIntegration.F90:225-336, 569-680)
        for (int s = 0; s < 3; s++) {
            TRY(rhs_stage(c, s == 0 ? q0 : qs, q0, qs, SSP_STAGE1 + s, nm, c->d1, c->tq, c->d2, c->delta));
            TRY(apply_bc(c, qst, nm, s == 1 ? 0.5 : 1.0));
        }
    } else {  // RK4_2D/3D (timeIntegration.F90:8-156, 338-498)
        for (int s = 1; s <= 4; s++) {
            TRY(rhs_stage(c, s == 1 ? q0 : qs, q0, qs, s, nm, c->d1, c->tq, c->d2, c->delta));
            TRY(apply_bc(c, qst, nm, s <= 2 ? 0.5 : 1.0));
        }
    }
    // nothing after the filter (no SFD, no boundary program): its last sweep can take the
    // max-change (main.F90:413-418) in its epilogue; the state sets must be equally spaced
    const bool mc_in_filter = c->fuse_mc && c->sfd_type == 0 && c->nops == 0 && c->is3d &&
                              qs.v[1] - qs.v[0] == c->npts && q0.v[1] - q0.v[0] == c->npts;
    if (c->fct > 0) TRY(filter_set(c, qs, nm, 0.0, &c->d_params->dt, mc_in_filter ? &q0 : nullptr));
    else TRY(filter_set(c, qs, nm, 0.0, nullptr, mc_in_filter ? &q0 : nullptr));
    const bool mc_done = mc_in_filter && c->mc_done;
    if (c->sfd_type > 0) {
        TRY(before_launch(c, PC_SFD));
        k_sfd<<<dim3(grid_for(c, c->npts), nm), kBlock, 0, c->stream>>>(qs, fset(c, c->mean, 5), c->chi, c->sfd_delta,
                                                                          c->is3d ? 5 : 4, c->npts, c->d_params);
        TRY(after_launch(c));
    }
    TRY(apply_bc(c, qs, nm, 1.0));  // main.F90:405, at t + dt
    if (!mc_done) {
        TRY(before_launch(c, PC_MAXCHANGE));
        k_maxchange<<<dim3(grid_for(c, c->npts), nm), kBlock, 0, c->stream>>>(qs, q0, c->acc, c->npts);
        TRY(after_launch(c));
    }
    TRY(before_launch(c, PC_MAXCHANGE));
    k_store_maxchange<<<1, 5 * nm < 1024 ? 5 * nm : 1024, 0, c->stream>>>(c->acc, c->hist, 5 * nm, c->d_params);
    return after_launch(c);
}

int ensure_graph(gatt_ctx *c)
{
    const int g = c->cur;
    if (c->graph[g]) return GATT_OK;
    if (c->bc_dirty) TRY(build_bc_program(c));
    cudaGraph_t graph;
    c->capturing = true;
    c->capture_count = 0;
    CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = step_body(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    c->capturing = false;
    if (rc != GATT_OK) { if (e == cudaSuccess) cudaGraphDestroy(graph); return rc; }
    CU(e);
    cudaError_t ei = cudaGraphInstantiate(&c->graph[g], graph, 0);
    cudaGraphDestroy(graph);
    CU(ei);
    c->graph_kernels[g] = c->capture_count;
    return GATT_OK;
}

int ensure_hist(gatt_ctx *c, int n)
{
    if (n <= c->hist_cap) return GATT_OK;
    int cap = c->hist_cap ? c->hist_cap : 64;
    while (cap < n) cap *= 2;
    TRY(sync_stream(c));
    cudaFree(c->hist);
    cudaFreeHost(c->h_params);
    c->hist = nullptr; c->h_params = nullptr;
    CU(cudaMalloc(&c->hist, sizeof(double) * 5 * c->nb * (size_t)cap));
    CU(cudaMallocHost(&c->h_params, sizeof(StepParams) * (size_t)cap));
    c->hist_cap = cap;
    invalidate_graphs(c);  // graphs hold the history pointer
    return GATT_OK;
}

int run_steps(gatt_ctx *c, int nsteps, double t0, double dt, double *maxChange, bool check_each)
{
    TRY(check_ready(c, true));
    if (nsteps < 1) return fail(GATT_ERR_BADARG, "nsteps < 1");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(GATT_ERR_BADARG, "dt must be positive and finite");
    if (c->sfd_type > 0 && !c->chi) return fail(GATT_ERR_STATE, "SFD field not set");
    TRY(check_hold(c));
    TRY(ensure_hist(c, nsteps));
    if (c->sfd_type > 0 && !c->mean_init) {
        // Umean = U when no mean flow was given (main.F90:158-163)
        const StateSet q = state_set(c, 0);
        for (int b = 0; b < c->nb; b++)
            for (int f = 0; f < 5; f++)
                CU(cudaMemcpyAsync(c->mean + ((size_t)b * 5 + f) * c->npts, q.v[f] + b * q.bstride,
                                   sizeof(double) * c->npts, cudaMemcpyDeviceToDevice, c->stream));
        c->mean_init = true;
    }
    double t = t0;
    for (int s = 0; s < nsteps; s++) {
        c->h_params[s].t = t; c->h_params[s].dt = dt; c->h_params[s].slot = s;
        TRY(ensure_graph(c));
        CU(cudaMemcpyAsync(c->d_params, &c->h_params[s], sizeof(StepParams), cudaMemcpyHostToDevice, c->stream));
        CU(cudaGraphLaunch(c->graph[c->cur], c->stream));
        c->launches += c->graph_kernels[c->cur];
        c->cur ^= 1;
        t = t + dt;  // main.F90:423
    }
    const int nv = 5 * c->nb;
    std::vector<double> h((size_t)nv * nsteps);
    CU(cudaMemcpyAsync(h.data(), c->hist, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    TRY(sync_stream(c));
    if (maxChange) memcpy(maxChange, h.data() + (size_t)nv * (nsteps - 1), sizeof(double) * nv);
    // divergence test of main.F90:433-438, per member and step
    for (int s = check_each ? 0 : nsteps - 1; s < nsteps; s++)
        for (int b = 0; b < c->nb; b++) {
            const double *m = h.data() + (size_t)nv * s + 5 * b;
            double sum = 0;
            bool nan = false;
            for (int f = 0; f < 5; f++) { nan |= std::isnan(m[f]); sum += m[f]; }
            if (nan || sum == 0)
                return fail(GATT_ERR_DIVERGED, "flow diverged (member " + std::to_string(b) + ", step " +
                                                   std::to_string(s) + ")");
        }
    return GATT_OK;
}

int alloc_fields(gatt_ctx *c, double **p, int nslots, int members)
{
    CU(cudaMalloc(p, sizeof(double) * (size_t)c->npts * nslots * members));
    CU(cudaMemsetAsync(*p, 0, sizeof(double) * (size_t)c->npts * nslots * members, c->stream));
    return GATT_OK;
}

int ensure_host_scratch(gatt_ctx *c)
{
    if (!c->tin) TRY(alloc_fields(c, &c->tin, 5, 1));
    if (!c->tout) TRY(alloc_fields(c, &c->tout, 5, 1));
    return GATT_OK;
}

int check_member(const gatt_ctx *c, int b)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (b < 0 || b >= c->nb) return fail(GATT_ERR_BADARG, "batch member out of range");
    return GATT_OK;
}

// ---------------------------------------------------------------------------
// allocation-free max-change: the accumulators live in a file-scope device array
// ---------------------------------------------------------------------------

// Every GPU that loads this library holds this array (160 x 8 = 1280 bytes) until the
// process exits.  Host code must not pass the symbol itself to a kernel: it names a
// host-side stand-in.  The device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned long long g_noalloc_maxchange[kMaxChangeSlots];

namespace {
constexpr int kMaxDevices = 64;
unsigned long long *g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mu;  // guards the per-device address cache

int noalloc_scratch(unsigned long long **out)
{
    int dev = 0;
    CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(GATT_ERR_BADARG, "device ordinal beyond the supported range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        CU(cudaGetSymbolAddress(&p, g_noalloc_maxchange));
        g_noalloc_ptr[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return GATT_OK;
}
}  // namespace

// ---------------------------------------------------------------------------
// Jacobian-free Arnoldi (calcInstability.m:304-400, first-order variant), nbatch problems
// ---------------------------------------------------------------------------

int arn_nv(const gatt_ctx *c) { return c->is3d ? 5 : 4; }

int arn_alloc(gatt_ctx *c, int m)
{
    const long long len = (long long)arn_nv(c) * c->npts;
    if (c->arn_m < m) {
        cudaFree(c->arn_zeta);
        c->arn_zeta = nullptr;
        c->arn_m = 0;
        CU(cudaMalloc(&c->arn_zeta, sizeof(double) * (size_t)c->nb * (m + 1) * len));
        cudaFree(c->arn_part);
        c->arn_part = nullptr;
        CU(cudaMalloc(&c->arn_part, sizeof(double) * (size_t)c->nb * (m + 2) * kRedBlocks));
        cudaFree(c->arn_h);
        c->arn_h = nullptr;
        CU(cudaMalloc(&c->arn_h, sizeof(double) * (size_t)c->nb * (m + 2)));
        c->arn_m = m;
    }
    if (!c->arn_B) CU(cudaMalloc(&c->arn_B, sizeof(double) * (size_t)c->nb * len));
    if (!c->arn_base) CU(cudaMalloc(&c->arn_base, sizeof(double) * 5 * (size_t)c->npts));
    if (!c->arn_um) CU(cudaMalloc(&c->arn_um, sizeof(double) * 5 * (size_t)c->npts));
    if (!c->arn_region) CU(cudaMalloc(&c->arn_region, (size_t)c->npts));
    return GATT_OK;
}

// Sum the partials of nvec vectors per member into arn_h[b][0..nvec) (sqrt when asked)
int arn_sum(gatt_ctx *c, int part_stride, int nvec, double *h, int h_stride, bool take_sqrt)
{
    TRY(before_launch(c, PC_OTHER));
    k_arn_sum<<<c->nb, (nvec + 31) / 32 * 32, 0, c->stream>>>(c->arn_part, part_stride, nvec, h, h_stride, take_sqrt);
    return after_launch(c);
}

int arnoldi(gatt_ctx *c, int m, int nsteps, double t0, double dt, double eps, const double *base,
            const double *v0, const unsigned char *region, double *H)
{
    TRY(check_ready(c, true));
    if (m < 1 || m > kMaxKrylov) return fail(GATT_ERR_BADARG, "Krylov dimension must be 1 .. " + std::to_string(kMaxKrylov));
    if (nsteps < 1) return fail(GATT_ERR_BADARG, "nsteps < 1");
    if (!(dt > 0) || !std::isfinite(dt) || !(eps > 0) || !std::isfinite(eps))
        return fail(GATT_ERR_BADARG, "dt and eps must be positive and finite");
    if (!base || !v0 || !H) return fail(GATT_ERR_BADARG, "null base, v0 or H");
    const long long n = c->npts;
    const int nv = arn_nv(c);
    const long long len = (long long)nv * n;
    TRY(arn_alloc(c, m));
    const long long zs = (long long)(c->arn_m + 1) * len;  // basis stride between members
    const int ps = (c->arn_m + 2) * kRedBlocks, hs = c->arn_m + 2;
    // flow region: the points whose values enter the vectors (calcInstability.m:137-141)
    long long nreg = n;
    if (region) {
        nreg = 0;
        for (long long p = 0; p < n; p++) nreg += region[p] != 0;
        if (nreg == 0) return fail(GATT_ERR_BADARG, "empty flow region");
        CU(cudaMemcpyAsync(c->arn_region, region, (size_t)n, cudaMemcpyHostToDevice, c->stream));
    }
    const uint8_t *reg = region ? c->arn_region : nullptr;
    const double sqrtN = std::sqrt((double)nv * (double)nreg);
    const double den = eps * sqrtN;
    CU(cudaMemcpyAsync(c->arn_base, base, sizeof(double) * 5 * n, cudaMemcpyHostToDevice, c->stream));
    // zeta_1 = v0 restricted to the region (flow2vec), normalised
    {
        std::vector<double> tmp((size_t)n);
        for (int b = 0; b < c->nb; b++)
            for (int f = 0; f < 5; f++) {
                const int v = c->is3d ? f : (f == 2 ? -1 : (f < 2 ? f : f - 1));
                if (v < 0) continue;
                const double *src = v0 + ((size_t)b * 5 + f) * n;
                for (long long p = 0; p < n; p++) tmp[p] = (!region || region[p]) ? src[p] : 0.0;
                CU(cudaMemcpyAsync(c->arn_zeta + b * zs + v * n, tmp.data(), sizeof(double) * n,
                                   cudaMemcpyHostToDevice, c->stream));
                CU(cudaStreamSynchronize(c->stream));  // tmp is reused
            }
    }
    const dim3 rgrid(kRedBlocks, c->nb);
    TRY(before_launch(c, PC_OTHER));
    k_arn_dots<<<rgrid, kRedThreads, 0, c->stream>>>(c->arn_zeta, zs, c->arn_zeta, zs, 0, len, c->arn_part, ps);
    TRY(after_launch(c));
    TRY(arn_sum(c, ps, 1, c->arn_h, hs, true));
    TRY(before_launch(c, PC_OTHER));
    k_arn_scale<<<dim3(grid_for(c, len), c->nb), kBlock, 0, c->stream>>>(c->arn_zeta, zs, c->arn_h, hs, 0, len);
    TRY(after_launch(c));

    auto evolve = [&](int k, double e) -> int {
        // state = base + (zeta_k * e) * sqrt(N); SFD mean restarts from it (main.F90:158-163)
        TRY(before_launch(c, PC_OTHER));
        k_arn_perturb<<<dim3(grid_for(c, n), c->nb), kBlock, 0, c->stream>>>(state_set(c, 0), c->arn_base,
                                                                             c->arn_zeta + k * len, zs, reg, e,
                                                                             sqrtN, c->is3d, n);
        TRY(after_launch(c));
        c->mean_init = false;
        return run_steps(c, nsteps, t0, dt, nullptr, true);
    };
    // UM: the base flow's own run (calcInstability.m:327-340); every member runs the base
    // (a zero disturbance), member 0's result is kept
    TRY(evolve(0, 0.0));
    {
        const StateSet q = state_set(c, 0);
        for (int f = 0; f < 5; f++)
            CU(cudaMemcpyAsync(c->arn_um + f * n, q.v[f], sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    }
    memset(H, 0, sizeof(double) * (size_t)c->nb * (m + 1) * m);
    std::vector<double> hc((size_t)c->nb * hs);
    for (int k = 0; k < m; k++) {
        // B = (Phi(base + disturbance) - UM) / (eps sqrt(N))
        TRY(evolve(k, eps));
        TRY(before_launch(c, PC_OTHER));
        k_arn_diff<<<dim3(grid_for(c, n), c->nb), kBlock, 0, c->stream>>>(state_set(c, 0), c->arn_um, c->arn_B, len, nv,
                                                                          reg, den, c->is3d, n);
        TRY(after_launch(c));
        // classical Gram-Schmidt: H(j,k) = zeta_j . B, uPrime = B - sum H(j,k) zeta_j
        TRY(before_launch(c, PC_OTHER));
        k_arn_dots<<<rgrid, kRedThreads, 0, c->stream>>>(c->arn_zeta, zs, c->arn_B, len, k, len, c->arn_part, ps);
        TRY(after_launch(c));
        TRY(arn_sum(c, ps, k + 1, c->arn_h, hs, false));
        TRY(before_launch(c, PC_OTHER));
        k_arn_orth<<<rgrid, kRedThreads, 0, c->stream>>>(c->arn_zeta, zs, c->arn_B, len, c->arn_h, hs, k, len,
                                                          c->arn_part, ps);
        TRY(after_launch(c));
        // H(k+1,k) = |uPrime|, zeta_{k+1} = uPrime / H(k+1,k)
        TRY(arn_sum(c, ps, 1, c->arn_h + k + 1, hs, true));
        TRY(before_launch(c, PC_OTHER));
        k_arn_scale<<<dim3(grid_for(c, len), c->nb), kBlock, 0, c->stream>>>(c->arn_zeta, zs, c->arn_h + k + 1, hs,
                                                                             k + 1, len);
        TRY(after_launch(c));
        CU(cudaMemcpyAsync(hc.data(), c->arn_h, sizeof(double) * hc.size(), cudaMemcpyDeviceToHost, c->stream));
        TRY(sync_stream(c));
        for (int b = 0; b < c->nb; b++)
            for (int i = 0; i <= k + 1; i++) {
                const double h = hc[(size_t)b * hs + i];
                if (!std::isfinite(h)) return fail(GATT_ERR_DIVERGED, "non-finite Hessenberg entry (member " +
                                                                          std::to_string(b) + ")");
                H[(size_t)b * (m + 1) * m + (size_t)k * (m + 1) + i] = h;
            }
    }
    return GATT_OK;
}


// ---------------------------------------------------------------------------
// Tangent-linear and adjoint of the step (no counterpart in the reference)
// ---------------------------------------------------------------------------
// Both run the 3-D data flow in the 3-D layouts.  A 2-D case runs it with no z direction:
// the z gradients and z second sweeps stay zero and W is zero, so the 3-D expressions reduce
// to nseq2d's (nseq.F90:10-139) and the W components of every vector are zero.  With SFD
// (main.F90:381-402) the step maps the state and the mean, so the tangent and adjoint carry
// both: a vector of a member is then its 5 state fields followed by its 5 mean fields.

StateSet set5(const gatt_ctx *c, double *p)
{
    StateSet s;
    for (int f = 0; f < 5; f++) s.v[f] = p + f * c->npts;
    s.bstride = 5 * c->npts;
    return s;
}

int copy_set5(gatt_ctx *c, double *dst, const double *src)
{
    CU(cudaMemcpyAsync(dst, src, sizeof(double) * 5 * (size_t)c->npts * c->nb, cudaMemcpyDeviceToDevice, c->stream));
    return GATT_OK;
}

// zero slot W of every member of a 5-field set (2-D cases)
int zero_w(gatt_ctx *c, double *set)
{
    if (c->is3d) return GATT_OK;
    CU(cudaMemset2DAsync(set + 2 * c->npts, sizeof(double) * 5 * (size_t)c->npts, 0, sizeof(double) * (size_t)c->npts,
                         c->nb, c->stream));
    return GATT_OK;
}

// copy between a context state slot (separate per-variable pointers) and a 5-field set; in
// 2-D the set's W is zero and the state's W (the caller's) is never overwritten
int state_to_set(gatt_ctx *c, const StateSet &q, double *dst, bool to_set)
{
    for (int b = 0; b < c->nb; b++)
        for (int f = 0; f < 5; f++) {
            if (!c->is3d && f == 2) continue;
            double *sp = q.v[f] + b * q.bstride, *dp = dst + ((size_t)b * 5 + f) * c->npts;
            if (to_set) CU(cudaMemcpyAsync(dp, sp, sizeof(double) * c->npts, cudaMemcpyDeviceToDevice, c->stream));
            else CU(cudaMemcpyAsync(sp, dp, sizeof(double) * c->npts, cudaMemcpyDeviceToDevice, c->stream));
        }
    if (to_set) TRY(zero_w(c, dst));
    return GATT_OK;
}

bool diff_sfd(const gatt_ctx *c) { return c->sfd_type > 0; }

// Vector fields per member of gatt_jvp / gatt_vjp: the state, and with SFD the mean.
int diff_nv(const gatt_ctx *c) { return diff_sfd(c) ? 10 : 5; }

int check_diff(gatt_ctx *c, bool adjoint, bool step = false)
{
    TRY(check_ready(c, true));
    if (step && c->time_stepping != 1)
        return fail(GATT_ERR_STATE, "the tangent-linear and adjoint steps are those of RK4 (timeStepping 1)");
    if (c->fc.n > 0) return fail(GATT_ERR_STATE, "the tangent-linear and adjoint do not cover forcings");
    if (step) TRY(check_hold(c));  // the right-hand side alone applies no boundary conditions
    else if (c->bc_dirty) TRY(build_bc_program(c));
    if (step && diff_sfd(c) && (!c->mean || !c->mean_init))
        return fail(GATT_ERR_STATE, "SFD: upload the mean (gatt_upload_mean) or run a step before the tangent/adjoint");
    const int ndir = c->is3d ? 3 : 2;
    if (adjoint)
        for (int d = 0; d < ndir; d++) {
            if (!c->mat[d][2].set || !c->mat[d][3].set)
                return fail(GATT_ERR_STATE, "transposed derivative matrices (kinds 2, 3) missing");
            if (c->filt[d] && (!c->mat[d][4].set || !c->mat[d][5].set))
                return fail(GATT_ERR_STATE, "transposed filter matrices (kinds 4, 5) missing");
        }
    return GATT_OK;
}

// allocate a set of nslots fields per member, zeroed (the 2-D z slots are never written)
int alloc_zeroed(gatt_ctx *c, double **p, int nslots)
{
    if (*p) return GATT_OK;
    TRY(alloc_fields(c, p, nslots, c->nb));
    CU(cudaMemsetAsync(*p, 0, sizeof(double) * nslots * (size_t)c->npts * c->nb, c->stream));
    return GATT_OK;
}

int diff_alloc(gatt_ctx *c, bool adjoint)
{
    for (double *&p : c->dx) TRY(alloc_zeroed(c, &p, 5));
    if (!c->is3d) {
        TRY(alloc_zeroed(c, &c->g_d1, D3_N));
        TRY(alloc_zeroed(c, &c->g_tq, T3_N));
        TRY(alloc_zeroed(c, &c->g_d2, S3_N));
    }
    if (diff_sfd(c)) TRY(alloc_zeroed(c, &c->dxm, 5));
    if (!adjoint) {
        if (!c->t_P) TRY(alloc_fields(c, &c->t_P, 1, c->nb));
        for (double *&p : c->dy) TRY(alloc_zeroed(c, &p, 5));
        TRY(alloc_zeroed(c, &c->t_delta, 5));
        TRY(alloc_zeroed(c, &c->t_d1, D3_N));
        TRY(alloc_zeroed(c, &c->t_tq, T3_N));
        TRY(alloc_zeroed(c, &c->t_d2, S3_N));
        if (diff_sfd(c)) TRY(alloc_zeroed(c, &c->dym, 5));
        return GATT_OK;
    }
    double **five[] = {&c->a_lam, &c->a_acc, &c->a_arg, &c->a_prev, &c->a_g, &c->a_lq, &c->a_scr};
    for (double **p : five) TRY(alloc_zeroed(c, p, 5));
    TRY(alloc_zeroed(c, &c->a_ld1, D3_N));
    TRY(alloc_zeroed(c, &c->a_ltau, T3_N));
    TRY(alloc_zeroed(c, &c->a_lvt, 4));
    TRY(alloc_zeroed(c, &c->a_s1, 15));
    TRY(alloc_zeroed(c, &c->a_s2, 12));
    if (!c->a_lP) TRY(alloc_fields(c, &c->a_lP, 1, c->nb));
    TRY(alloc_zeroed(c, &c->a_tmp, 5));
    if (diff_sfd(c)) {
        TRY(alloc_zeroed(c, &c->a_lm, 5));
        TRY(alloc_zeroed(c, &c->a_mscr, 5));
    }
    // five boundary-program tapes per step (after each stage and after the filter / SFD)
    const long long need = 5 * std::max(1LL, c->tape_len) * c->nb;
    if (c->a_tape_cap < need) {
        cudaFree(c->a_tape);
        c->a_tape = nullptr;
        c->a_tape_cap = 0;
        CU(cudaMalloc(&c->a_tape, sizeof(double) * (size_t)need));
        c->a_tape_cap = need;
    }
    return GATT_OK;
}

// boundary program on base x and tangent y together, at time t + tfac dt
int bc_tl(gatt_ctx *c, const StateSet &x, const StateSet &y, double tfac)
{
    if (c->nops == 0) return GATT_OK;
    TRY(before_launch(c, PC_BC));
    TRY(launch_bc(c, k_bc_tl, k_bc_tl_cluster, c->bc_cluster_tl, c->nb, 0, bc_program(c, tfac), x, c->P, y, c->t_P,
                  (long long)c->npts));
    return after_launch(c);
}

// boundary program on base x at time t + tfac dt, recording tape number `which` (0..4)
int bc_rec(gatt_ctx *c, const StateSet &x, int which, double tfac)
{
    if (c->nops == 0) return GATT_OK;
    const long long ts = std::max(1LL, c->tape_len);
    TRY(before_launch(c, PC_BC));
    TRY(launch_bc(c, k_bc_rec, k_bc_rec_cluster, c->bc_cluster_rec, c->nb, 0, bc_program(c, tfac), x, c->P,
                  (long long)c->npts, c->a_tape + which * ts * c->nb, ts));
    return after_launch(c);
}

// transposed boundary program on lambda, from tape `which`
int bc_adj(gatt_ctx *c, const StateSet &lam, int which)
{
    if (c->nops == 0) return GATT_OK;
    const long long ts = std::max(1LL, c->tape_len);
    CU(cudaMemsetAsync(c->a_lP, 0, sizeof(double) * (size_t)c->npts * c->nb, c->stream));
    TRY(before_launch(c, PC_BC));
    TRY(launch_bc(c, k_bc_adj, k_bc_adj_cluster, c->bc_cluster_adj, c->nb, 0, bc_program(c, 1.0), lam, c->a_lP,
                  (long long)c->npts, (const double *)(c->a_tape + which * ts * c->nb), ts));
    return after_launch(c);
}

int set_params(gatt_ctx *c, int slot, double t, double dt)
{
    TRY(ensure_hist(c, slot + 1));
    c->h_params[slot].t = t; c->h_params[slot].dt = dt; c->h_params[slot].slot = slot;
    CU(cudaMemcpyAsync(c->d_params, &c->h_params[slot], sizeof(StepParams), cudaMemcpyHostToDevice, c->stream));
    return GATT_OK;
}

// The base data the tangent / adjoint kernels read, in the 3-D layouts
double *diff_d1(gatt_ctx *c) { return c->is3d ? c->d1 : c->g_d1; }
double *diff_d2(gatt_ctx *c) { return c->is3d ? c->d2 : c->g_d2; }

// rhs_stage for the tangent and adjoint on 5-field sets: in 3-D the forward itself; in 2-D the
// 3-D data flow without the z direction (x and y sweeps into the 3-D slots, the z slots stay
// zero), so the stage matches nseq2d + RK4_2D to rounding and leaves the base data in the
// 3-D layouts.
int rhs_stage_d(gatt_ctx *c, const StateSet &q, const StateSet &q0, const StateSet &out, int mode,
                bool assemble = true)
{
    const int nm = c->nb;
    if (c->is3d) return rhs_stage(c, q, q0, out, mode, nm, c->d1, c->tq, c->d2, c->delta, assemble);
    const long long n = c->npts;
    const long long bd1 = D3_N * n, btq = T3_N * n, bd2 = S3_N * n;
    const int fin[5] = {0, 1, 2, 3, 4};
    const int ox[5] = {D3_UX, D3_VX, D3_WX, D3_RX, D3_EX};
    const int oy[5] = {D3_UY, D3_VY, D3_WY, D3_RY, D3_EY};
    TRY(sweep(c, 0, 0, q.v[0], q.bstride, fin, c->g_d1, bd1, ox, 5, nm, 0, nullptr, PC_D1X));
    TRY(sweep(c, 1, 0, q.v[0], q.bstride, fin, c->g_d1, bd1, oy, 5, nm, 0, nullptr, PC_D1Y));
    TRY(before_launch(c, PC_VISC));
    k_visc3d<<<dim3(grid_for(c, n), nm), kBlock, 0, c->stream>>>(c->ph, q, fset(c, c->g_d1, D3_N),
                                                                fset(c, c->g_tq, T3_N), n);
    TRY(after_launch(c));
    const int ix[4] = {T3_XX, T3_XY, T3_XZ, T3_QX}, sx[4] = {S3_TXXX, S3_TXYX, S3_TXZX, S3_HTX};
    const int iy[4] = {T3_XY, T3_YY, T3_YZ, T3_QY}, sy[4] = {S3_TXYY, S3_TYYY, S3_TYZY, S3_HTY};
    TRY(sweep(c, 0, 0, c->g_tq, btq, ix, c->g_d2, bd2, sx, 4, nm, 0, nullptr, PC_D2X));
    TRY(sweep(c, 1, 0, c->g_tq, btq, iy, c->g_d2, bd2, sy, 4, nm, 0, nullptr, PC_D2Y));
    if (!assemble) return GATT_OK;
    return assemble3d(c, q, q0, out, mode, nm, c->g_d1, c->g_d2, c->delta);
}

// Tangent of one RK stage (mode 1..4, or RK_STORE_RHS for the bare RHS): the base stage
// xin -> xout (the forward kernels), then the tangent yin -> yout.
int tl_stage(gatt_ctx *c, const StateSet &xin, const StateSet &x0, const StateSet &xout, const StateSet &yin,
             const StateSet &y0, const StateSet &yout, int mode)
{
    const int nm = c->nb;
    const long long n = c->npts;
    TRY(rhs_stage_d(c, xin, x0, xout, mode));
    double *d1 = diff_d1(c), *d2 = diff_d2(c);
    const long long bd1 = D3_N * n, btq = T3_N * n, bd2 = S3_N * n;
    const int fin[5] = {0, 1, 2, 3, 4};
    const int ox[5] = {D3_UX, D3_VX, D3_WX, D3_RX, D3_EX};
    const int oy[5] = {D3_UY, D3_VY, D3_WY, D3_RY, D3_EY};
    const int oz[5] = {D3_UZ, D3_VZ, D3_WZ, D3_RZ, D3_EZ};
    TRY(sweep(c, 0, 0, yin.v[0], yin.bstride, fin, c->t_d1, bd1, ox, 5, nm, 0, nullptr, PC_D1X));
    TRY(sweep(c, 1, 0, yin.v[0], yin.bstride, fin, c->t_d1, bd1, oy, 5, nm, 0, nullptr, PC_D1Y));
    if (c->is3d) TRY(sweep(c, 2, 0, yin.v[0], yin.bstride, fin, c->t_d1, bd1, oz, 5, nm, 0, nullptr, PC_D1Z));
    TRY(before_launch(c, PC_VISC));
    k_tl_tau3d<<<dim3(grid_for(c, n), nm), kBlock, 0, c->stream>>>(c->ph, xin, fset(c, d1, D3_N), yin,
                                                                  fset(c, c->t_d1, D3_N), fset(c, c->t_tq, T3_N), n);
    TRY(after_launch(c));
    const int ix[4] = {T3_XX, T3_XY, T3_XZ, T3_QX}, sx[4] = {S3_TXXX, S3_TXYX, S3_TXZX, S3_HTX};
    const int iy[4] = {T3_XY, T3_YY, T3_YZ, T3_QY}, sy[4] = {S3_TXYY, S3_TYYY, S3_TYZY, S3_HTY};
    const int iz[4] = {T3_XZ, T3_YZ, T3_ZZ, T3_QZ}, sz[4] = {S3_TXZZ, S3_TYZZ, S3_TZZZ, S3_HTZ};
    TRY(sweep(c, 0, 0, c->t_tq, btq, ix, c->t_d2, bd2, sx, 4, nm, 0, nullptr, PC_D2X));
    TRY(sweep(c, 1, 0, c->t_tq, btq, iy, c->t_d2, bd2, sy, 4, nm, 0, nullptr, PC_D2Y));
    if (c->is3d) TRY(sweep(c, 2, 0, c->t_tq, btq, iz, c->t_d2, bd2, sz, 4, nm, 0, nullptr, PC_D2Z));
    TRY(before_launch(c, PC_ASSEMBLE));
    k_tl_assemble3d<<<dim3(grid_for(c, n), nm), kBlock, 0, c->stream>>>(
        c->ph, xin, fset(c, d1, D3_N), fset(c, d2, S3_N), yin, fset(c, c->t_d1, D3_N), fset(c, c->t_d2, S3_N), y0,
        yout, fset(c, c->t_delta, 5), n, mode, c->d_params);
    return after_launch(c);
}

// SFD relaxation of a 5-field set with the mean `mean` (a 5-field set), the forward kernel
int sfd_set(gatt_ctx *c, const StateSet &q, double *mean)
{
    TRY(before_launch(c, PC_SFD));
    k_sfd<<<dim3(grid_for(c, c->npts), c->nb), kBlock, 0, c->stream>>>(q, fset(c, mean, 5), c->chi, c->sfd_delta,
                                                                     c->is3d ? 5 : 4, c->npts, c->d_params);
    return after_launch(c);
}

// One step of base and tangent: dx[0], dy[0] (and with SFD the means dxm, dym) = step start
// -> step end (same arrays)
int tl_step(gatt_ctx *c)
{
    const StateSet X0 = set5(c, c->dx[0]), XA = set5(c, c->dx[1]), XB = set5(c, c->dx[2]);
    const StateSet Y0 = set5(c, c->dy[0]), YA = set5(c, c->dy[1]), YB = set5(c, c->dy[2]);
    // boundary conditions after every stage (timeIntegration.F90:406-491) and after the filter
    TRY(tl_stage(c, X0, X0, XA, Y0, Y0, YA, RK_STAGE1));
    TRY(bc_tl(c, XA, YA, 0.5));
    TRY(tl_stage(c, XA, X0, XB, YA, Y0, YB, RK_STAGE2));
    TRY(bc_tl(c, XB, YB, 0.5));
    TRY(tl_stage(c, XB, X0, XA, YB, Y0, YA, RK_STAGE3));
    TRY(bc_tl(c, XA, YA, 1.0));
    TRY(tl_stage(c, XA, X0, XB, YA, Y0, YB, RK_STAGE4));
    TRY(bc_tl(c, XB, YB, 1.0));
    // the filter is linear: the same sweeps act on the tangent (main.F90:357-378)
    const double *bdt = c->fct > 0 ? &c->d_params->dt : nullptr;
    TRY(filter_set(c, XB, c->nb, 0.0, bdt));
    TRY(filter_set(c, YB, c->nb, 0.0, bdt));
    // SFD (main.F90:381-402) is linear in the state and the mean: k_sfd is its own tangent
    if (diff_sfd(c)) {
        TRY(sfd_set(c, XB, c->dxm));
        TRY(sfd_set(c, YB, c->dym));
    }
    TRY(bc_tl(c, XB, YB, 1.0));
    TRY(copy_set5(c, c->dx[0], c->dx[2]));
    return copy_set5(c, c->dy[0], c->dy[2]);
}

// transposed line operator L^T = R^T (LHS^T)^-1 of direction d over nf fields: kind k0 (the
// LHS^T solve) into the scratch, then kind k0+1 (the R^T band) into the output slots
int sweep_T(gatt_ctx *c, int d, int k0, const double *in, long long in_bs, const int *in_slots, double *out,
            long long out_bs, const int *out_slots, int nf)
{
    int sl[16];
    for (int f = 0; f < nf; f++) sl[f] = f;
    TRY(sweep(c, d, k0, in, in_bs, in_slots, c->a_scr, 5 * c->npts, sl, nf, c->nb, 0.0, nullptr, PC_OTHER));
    return sweep(c, d, k0 + 1, c->a_scr, 5 * c->npts, sl, out, out_bs, out_slots, nf, c->nb, 0.0, nullptr, PC_OTHER);
}

// G = F'(q)^T a (the adjoint of the RHS at state q)
int adj_rhs(gatt_ctx *c, const StateSet &q, const StateSet &a, const StateSet &G)
{
    const int nm = c->nb;
    const long long n = c->npts;
    const int ndir = c->is3d ? 3 : 2;  // 2-D: no z direction, its slots of a_s1 / a_s2 stay zero
    TRY(rhs_stage_d(c, q, q, q, RK_STORE_RHS, false));
    double *d1 = diff_d1(c), *d2 = diff_d2(c);
    TRY(before_launch(c, PC_OTHER));
    k_adj_asm3d<<<dim3(grid_for(c, n), nm), kBlock, 0, c->stream>>>(
        c->ph, q, fset(c, d1, D3_N), fset(c, d2, S3_N), a, fset(c, c->a_lq, 5), fset(c, c->a_ld1, D3_N),
        fset(c, c->a_ltau, T3_N), fset(c, c->a_lvt, 4), n);
    TRY(after_launch(c));
    // transposed second sweeps: (vtx, vty, vtz, ht) -> stress / heat-flux contributions
    const int v4[4] = {0, 1, 2, 3};
    for (int d = 0; d < ndir; d++) {
        const int o4[4] = {4 * d, 4 * d + 1, 4 * d + 2, 4 * d + 3};
        TRY(sweep_T(c, d, 2, c->a_lvt, 4 * n, v4, c->a_s2, 12 * n, o4, 4));
    }
    TRY(before_launch(c, PC_OTHER));
    k_adj_tau3d<<<dim3(grid_for(c, n), nm), kBlock, 0, c->stream>>>(c->ph, q, fset(c, d1, D3_N),
                                                                   fset(c, c->a_ltau, T3_N), fset(c, c->a_s2, 12),
                                                                   fset(c, c->a_ld1, D3_N), fset(c, c->a_lq, 5), n);
    TRY(after_launch(c));
    // transposed first sweeps: gradient lambdas -> state lambdas
    for (int d = 0; d < ndir; d++) {
        const int i5[5] = {D3_UX + d, D3_VX + d, D3_WX + d, D3_RX + d, D3_EX + d};
        const int o5[5] = {5 * d, 5 * d + 1, 5 * d + 2, 5 * d + 3, 5 * d + 4};
        TRY(sweep_T(c, d, 2, c->a_ld1, (long long)D3_N * n, i5, c->a_s1, 15 * n, o5, 5));
    }
    TRY(before_launch(c, PC_OTHER));
    k_adj_q3d<<<dim3(grid_for(c, n), nm), kBlock, 0, c->stream>>>(fset(c, c->a_lq, 5), fset(c, c->a_s1, 15), G, n);
    return after_launch(c);
}

int axpby5(gatt_ctx *c, double *out, const double *x, const double *y, double alpha, double beta)
{
    TRY(before_launch(c, PC_OTHER));
    k_axpby5<<<dim3(grid_for(c, c->npts), c->nb), kBlock, 0, c->stream>>>(
        set5(c, out), set5(c, const_cast<double *>(x)), set5(c, const_cast<double *>(y ? y : x)), alpha, beta,
        y != nullptr, c->npts);
    return after_launch(c);
}

// Adjoint of one step: a_lam (and with SFD a_lm) holds lambda at the step end; dx[0] (and
// dxm) the step's start state.  Reverse of: 4 RK stages (timeIntegration.F90:338-498), the
// x -> y -> z filter, SFD, the boundary conditions.
int adj_step(gatt_ctx *c, double dt)
{
    const StateSet X[5] = {set5(c, c->dx[0]), set5(c, c->dx[1]), set5(c, c->dx[2]), set5(c, c->dx[3]),
                           set5(c, c->dx[4])};
    // recompute the stage states q1..q4 (after their boundary conditions) and the end state,
    // recording the boundary program's tapes: 0..3 after the stages, 4 after filter and SFD
    for (int s = 1; s <= 4; s++) {
        TRY(rhs_stage_d(c, X[s - 1], X[0], X[s], s));
        TRY(bc_rec(c, X[s], s - 1, s <= 2 ? 0.5 : 1.0));
    }
    if (c->nops > 0) {
        TRY(copy_set5(c, c->a_tmp, c->dx[4]));
        TRY(filter_set(c, set5(c, c->a_tmp), c->nb, 0.0, c->fct > 0 ? &c->d_params->dt : nullptr));
        if (diff_sfd(c)) {
            TRY(copy_set5(c, c->a_mscr, c->dxm));
            TRY(sfd_set(c, set5(c, c->a_tmp), c->a_mscr));
        }
        TRY(bc_rec(c, set5(c, c->a_tmp), 4, 1.0));
    }
    TRY(bc_adj(c, set5(c, c->a_lam), 4));
    if (diff_sfd(c)) {
        TRY(before_launch(c, PC_OTHER));
        k_sfd_adj<<<dim3(grid_for(c, c->npts), c->nb), kBlock, 0, c->stream>>>(
            set5(c, c->a_lam), fset(c, c->a_lm, 5), c->chi, c->sfd_delta, c->is3d ? 5 : 4, c->npts, c->d_params);
        TRY(after_launch(c));
    }
    // filter^T, z -> y -> x; with the time blend lam = lam + b (F^T lam - lam)
    const int f5[5] = {0, 1, 2, 3, 4};
    for (int d = (c->is3d ? 2 : 1); d >= 0; d--) {
        if (!c->filt[d]) continue;
        if (c->fct > 0) {
            TRY(sweep_T(c, d, 4, c->a_lam, 5 * c->npts, f5, c->a_g, 5 * c->npts, f5, 5));
            TRY(before_launch(c, PC_OTHER));
            k_adj_blend5<<<dim3(grid_for(c, c->npts), c->nb), kBlock, 0, c->stream>>>(
                set5(c, c->a_lam), set5(c, c->a_g), c->d_params, c->fct, c->npts);
            TRY(after_launch(c));
        } else {
            TRY(sweep_T(c, d, 4, c->a_lam, 5 * c->npts, f5, c->a_lam, 5 * c->npts, f5, 5));
        }
    }
    TRY(zero_w(c, c->a_lam));  // 2-D: the filter leaves W alone
    // RK4: q4 = q0 + dt/6 k1 + dt/3 k2 + dt/3 k3 + dt/6 k4, q1 = q0 + dt/2 k1,
    // q2 = q0 + dt/2 k2, q3 = q0 + dt k3, k_s = F(q_{s-1})
    const StateSet A = set5(c, c->a_arg), G = set5(c, c->a_g);
    TRY(bc_adj(c, set5(c, c->a_lam), 3));  // the boundary conditions after stage 4
    TRY(copy_set5(c, c->a_acc, c->a_lam));
    const double wl[4] = {dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0};  // weight of lambda4 in a_s (s = 4..1)
    const double wp[4] = {0.0, dt, dt / 2.0, dt / 2.0};             // weight of lambda_{q_s}
    for (int i = 0; i < 4; i++) {
        const int s = 3 - i;  // stage state q_s feeds k_{s+1}
        TRY(axpby5(c, c->a_arg, c->a_lam, i ? c->a_prev : nullptr, wl[i], wp[i]));
        TRY(adj_rhs(c, X[s], A, G));
        if (s > 0) TRY(bc_adj(c, G, s - 1));  // q_s came out of the boundary conditions of stage s
        TRY(axpby5(c, c->a_acc, c->a_acc, c->a_g, 1.0, 1.0));
        if (s > 0) TRY(copy_set5(c, c->a_prev, c->a_g));
    }
    TRY(copy_set5(c, c->a_lam, c->a_acc));
    return zero_w(c, c->a_lam);
}

// host vector [member][nv fields][point] <-> device sets: the state part into / from `q`
// (a 5-field set), with SFD the mean part into / from `m`
int upload_vec(gatt_ctx *c, double *q, double *m, const double *host)
{
    const int nv = diff_nv(c);
    const size_t f5 = sizeof(double) * 5 * (size_t)c->npts, fv = sizeof(double) * nv * (size_t)c->npts;
    CU(cudaMemcpy2DAsync(q, f5, host, fv, f5, c->nb, cudaMemcpyHostToDevice, c->stream));
    if (nv == 10) CU(cudaMemcpy2DAsync(m, f5, host + 5 * c->npts, fv, f5, c->nb, cudaMemcpyHostToDevice, c->stream));
    TRY(zero_w(c, q));
    return nv == 10 ? zero_w(c, m) : GATT_OK;
}

int download_vec(gatt_ctx *c, double *host, const double *q, const double *m)
{
    const int nv = diff_nv(c);
    const size_t f5 = sizeof(double) * 5 * (size_t)c->npts, fv = sizeof(double) * nv * (size_t)c->npts;
    CU(cudaMemcpy2DAsync(host, fv, q, f5, f5, c->nb, cudaMemcpyDeviceToHost, c->stream));
    if (nv == 10) CU(cudaMemcpy2DAsync(host + 5 * c->npts, fv, m, f5, f5, c->nb, cudaMemcpyDeviceToHost, c->stream));
    return sync_stream(c);
}

int upload5(gatt_ctx *c, double *dst, const double *host)
{
    CU(cudaMemcpyAsync(dst, host, sizeof(double) * 5 * (size_t)c->npts * c->nb, cudaMemcpyHostToDevice, c->stream));
    return zero_w(c, dst);
}

int download5(gatt_ctx *c, double *host, const double *src)
{
    CU(cudaMemcpyAsync(host, src, sizeof(double) * 5 * (size_t)c->npts * c->nb, cudaMemcpyDeviceToHost, c->stream));
    return sync_stream(c);
}

int rhs_jvp(gatt_ctx *c, const double *q, const double *dq, double *dk)
{
    TRY(check_diff(c, false));
    TRY(diff_alloc(c, false));
    TRY(upload5(c, c->dx[0], q));
    TRY(upload5(c, c->dy[0], dq));
    const StateSet X0 = set5(c, c->dx[0]), Y0 = set5(c, c->dy[0]);
    TRY(tl_stage(c, X0, X0, set5(c, c->dx[1]), Y0, Y0, set5(c, c->dy[1]), RK_STORE_RHS));
    return download5(c, dk, c->dy[1]);
}

int rhs_vjp(gatt_ctx *c, const double *q, const double *a, double *lam)
{
    TRY(check_diff(c, true));
    TRY(diff_alloc(c, true));
    TRY(upload5(c, c->dx[0], q));
    TRY(upload5(c, c->a_arg, a));
    TRY(adj_rhs(c, set5(c, c->dx[0]), set5(c, c->a_arg), set5(c, c->a_g)));
    TRY(zero_w(c, c->a_g));
    return download5(c, lam, c->a_g);
}

int jvp(gatt_ctx *c, int nsteps, double t0, double dt, const double *dq0, double *dqN)
{
    TRY(check_diff(c, false, true));
    if (nsteps < 1 || !(dt > 0) || !dq0 || !dqN) return fail(GATT_ERR_BADARG, "bad nsteps, dt or arrays");
    TRY(diff_alloc(c, false));
    TRY(state_to_set(c, state_set(c, 0), c->dx[0], true));
    if (diff_sfd(c)) TRY(copy_set5(c, c->dxm, c->mean));
    TRY(upload_vec(c, c->dy[0], c->dym, dq0));
    double t = t0;
    for (int s = 0; s < nsteps; s++) {
        TRY(set_params(c, 0, t, dt));
        TRY(tl_step(c));
        TRY(sync_stream(c));  // the parameter slot is reused
        t = t + dt;
    }
    TRY(state_to_set(c, state_set(c, 0), c->dx[0], false));
    if (diff_sfd(c)) TRY(copy_set5(c, c->mean, c->dxm));
    return download_vec(c, dqN, c->dy[0], c->dym);
}

// Checkpointed reverse sweep: states (and SFD means) every `every` steps are kept on the
// forward pass; each segment is recomputed from its checkpoint (storing every step's start
// state), then its steps are reversed.  Leaves the context state at the end of the forward run.
int vjp(gatt_ctx *c, int nsteps, double t0, double dt, int every, const double *lamN, double *lam0)
{
    TRY(check_diff(c, true, true));
    if (nsteps < 1 || every < 1 || !(dt > 0) || !lamN || !lam0) return fail(GATT_ERR_BADARG, "bad nsteps, dt or arrays");
    TRY(diff_alloc(c, true));
    const bool sfd = diff_sfd(c);
    const int nck = (nsteps + every - 1) / every, seg = std::min(every, nsteps);
    const size_t s5 = 5 * (size_t)c->npts * c->nb;  // one 5-field set of every member
    const size_t st = (sfd ? 2 : 1) * s5;           // a checkpoint: state, then the SFD mean
    if (c->a_nckpt < nck + 1 || (sfd && c->a_ckpt_sfd == false)) {
        cudaFree(c->a_ckpt);
        c->a_ckpt = nullptr;
        c->a_nckpt = 0;
        CU(cudaMalloc(&c->a_ckpt, sizeof(double) * st * (nck + 1)));
        c->a_nckpt = nck + 1;
        c->a_ckpt_sfd = sfd;
    }
    if (c->a_nseg < seg || (sfd && c->a_seg_sfd == false)) {
        cudaFree(c->a_seg);
        c->a_seg = nullptr;
        c->a_nseg = 0;
        CU(cudaMalloc(&c->a_seg, sizeof(double) * st * seg));
        c->a_nseg = seg;
        c->a_seg_sfd = sfd;
    }
    auto save = [&](double *dst) -> int {
        TRY(state_to_set(c, state_set(c, 0), dst, true));
        return sfd ? copy_set5(c, dst + s5, c->mean) : GATT_OK;
    };
    auto restore = [&](const double *src) -> int {
        TRY(state_to_set(c, state_set(c, 0), const_cast<double *>(src), false));
        return sfd ? copy_set5(c, c->mean, src + s5) : GATT_OK;
    };
    // forward: checkpoints at steps 0, every, 2*every, ...; slot nck keeps the final state
    for (int k = 0; k < nck; k++) {
        TRY(save(c->a_ckpt + st * k));
        const int len = std::min(every, nsteps - k * every);
        TRY(run_steps(c, len, t0 + (double)(k * every) * dt, dt, nullptr, false));
    }
    TRY(save(c->a_ckpt + st * nck));
    TRY(upload_vec(c, c->a_lam, c->a_lm, lamN));
    for (int k = nck - 1; k >= 0; k--) {
        const int len = std::min(every, nsteps - k * every);
        TRY(restore(c->a_ckpt + st * k));
        for (int i = 0; i < len; i++) {
            TRY(save(c->a_seg + st * i));
            if (i + 1 < len) TRY(run_steps(c, 1, t0 + (double)(k * every + i) * dt, dt, nullptr, false));
        }
        for (int i = len - 1; i >= 0; i--) {
            TRY(copy_set5(c, c->dx[0], c->a_seg + st * i));
            if (sfd) TRY(copy_set5(c, c->dxm, c->a_seg + st * i + s5));
            TRY(set_params(c, 0, t0 + (double)(k * every + i) * dt, dt));
            TRY(adj_step(c, dt));
            TRY(sync_stream(c));
        }
    }
    TRY(restore(c->a_ckpt + st * nck));
    return download_vec(c, lam0, c->a_lam, c->a_lm);
}


// ---------------------------------------------------------------------------
// Autotuner: line-solve kernel family and row-block partition per matrix set
// ---------------------------------------------------------------------------

// Candidates for a matrix set: the two register-resident families (16-row blocks) where the
// line length allows them, and the shared-tile solver at 8, 16, 32 and 64 rows per block.
struct TuneCand {
    int family, rpb, P;
};

std::vector<TuneCand> tune_candidates(const DevDir &m)
{
    std::vector<TuneCand> out;
    if (m.N % kRPB == 0 && m.N / kRPB <= kMaxP && m.nR >= 2 && m.nR <= kMaxNRreg) {
        out.push_back({FAM_PIPE, kRPB, m.N / kRPB});
        out.push_back({FAM_REG, kRPB, m.N / kRPB});
    } else if (m.Np > m.N || (m.N % kRPB == 0 && m.N / kRPB > kMaxP && m.family == FAM_PIPE && m.rpb)) {
        out.push_back({FAM_PIPE, kRPB, m.Np / kRPB});  // padded or long lines: the pipelined solver only
    }
    for (int rows : {8, 16, 32, 64}) {
        const int P = choose_blocks(m.N, m.nR, m.Wp, rows);
        bool dup = false;
        for (const TuneCand &t : out) dup |= (t.family == FAM_TILE && t.P == P);
        if (!dup) out.push_back({FAM_TILE, 0, P});
    }
    return out;
}

// Time every candidate on the context's grid (nf fields of scratch through one sweep, `reps`
// launches after a warm-up, CUDA events on the context's stream) and keep the fastest.
int autotune(gatt_ctx *c, int reps, int *family, int *blocks, double *us)
{
    TRY(check_ready(c, false));
    if (reps < 1) reps = 3;
    const int nf = c->is3d ? 5 : 4, ns = nd1(c);  // inputs in d1 slots 0..nf-1, outputs after them
    CU(cudaMemsetAsync(c->d1, 0, sizeof(double) * (size_t)ns * c->npts * c->nb, c->stream));
    int in[5], outs[5];
    for (int f = 0; f < nf; f++) { in[f] = f; outs[f] = nf + f; }
    const long long bs = (long long)ns * c->npts;
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    int rc = GATT_OK;
    const int ndir = c->is3d ? 3 : 2;
    for (int d = 0; d < 3 && rc == GATT_OK; d++)
        for (int k = 0; k < kMatKinds && rc == GATT_OK; k++) {
            const int slot = d * kMatKinds + k;
            if (family) family[slot] = -1;
            if (blocks) blocks[slot] = 0;
            if (us) us[slot] = 0.0;
            DevDir &m = c->mat[d][k];
            if (d >= ndir || !m.set || m.N < 2) continue;
            TuneCand best{m.family, m.rpb, m.P};
            float best_ms = -1.0f;
            for (const TuneCand &t : tune_candidates(m)) {
                m.family = t.family; m.rpb = t.rpb;
                rc = upload_records(c, m, t.P, t.rpb ? t.P * t.rpb : m.N);
                if (rc != GATT_OK) break;
                rc = sweep(c, d, k, c->d1, bs, in, c->d1, bs, outs, nf, c->nb, 0.0, nullptr);
                if (rc != GATT_OK) break;
                cudaEventRecord(e0, c->stream);
                for (int r = 0; r < reps && rc == GATT_OK; r++)
                    rc = sweep(c, d, k, c->d1, bs, in, c->d1, bs, outs, nf, c->nb, 0.0, nullptr);
                cudaEventRecord(e1, c->stream);
                if (rc != GATT_OK) break;
                cudaEventSynchronize(e1);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= reps;
                if (best_ms < 0 || ms < best_ms) { best_ms = ms; best = t; }
            }
            if (rc != GATT_OK) break;
            m.family = best.family; m.rpb = best.rpb;
            rc = upload_records(c, m, best.P, best.rpb ? best.P * best.rpb : m.N);
            if (family) family[slot] = best.family;
            if (blocks) blocks[slot] = best.P;
            if (us) us[slot] = 1e3 * best_ms;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    invalidate_graphs(c);
    TRY(rc);
    return sync_stream(c);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char *gatt_strerror(int code)
{
    switch (code) {
    case GATT_OK: return "ok";
    case GATT_ERR_CUDA: return "CUDA error";
    case GATT_ERR_BADARG: return "invalid argument";
    case GATT_ERR_BADCOEF: return "invalid coefficient (non-finite value or zero pivot)";
    case GATT_ERR_DIVERGED: return "flow diverged";
    case GATT_ERR_TIMEOUT: return "device wait timed out";
    case GATT_ERR_STATE: return "call out of order";
    case GATT_ERR_NOMEM: return "out of device memory";
    default: return "unknown error";
    }
}

const char *gatt_last_error(void) { return g_err.c_str(); }

int gatt_create(gatt_ctx **out, int nx, int ny, int nz, int nbatch)
{
    if (!out) return fail(GATT_ERR_BADARG, "null output pointer");
    *out = nullptr;
    if (nx < 2 || ny < 2 || nz < 1 || nbatch < 1) return fail(GATT_ERR_BADARG, "grid must be at least 2x2x1, nbatch >= 1");
    if ((long long)nx * ny * nz > (1LL << 31)) return fail(GATT_ERR_BADARG, "grid too large");
    if (nbatch > 65535) return fail(GATT_ERR_BADARG, "nbatch too large");
    gatt_ctx *c = new gatt_ctx();
    c->nx = nx; c->ny = ny; c->nz = nz; c->nb = nbatch;
    c->npts = (long long)nx * ny * nz;
    c->is3d = nz > 1;
    {
        const char *pw = getenv("GATT_PW");
        c->pw_pipe = !(pw && !strcmp(pw, "plain"));
        const char *my = getenv("GATT_MERGE_YZ");
        c->merge_yz = !(my && !strcmp(my, "0"));
        const char *fm = getenv("GATT_FUSE_MC");
        c->fuse_mc = !(fm && !strcmp(fm, "0"));
        const char *ubs = getenv("GATT_UBAND");
        c->uband_on = !(ubs && !strcmp(ubs, "0"));
        const char *xos = getenv("GATT_X_ORDER");
        c->x_order = !(xos && !strcmp(xos, "0"));
        const char *v2s = getenv("GATT_VISC_V2");
        c->visc_v2 = !(v2s && !strcmp(v2s, "0"));
        const char *xcs = getenv("GATT_X_COMPACT");
        c->x_compact = !(xcs && !strcmp(xcs, "0"));
        const char *xws = getenv("GATT_X_WSTORE");
        c->x_wstore = !(xws && !strcmp(xws, "0"));
        const char *fxs = getenv("GATT_FORK_X");
        c->fork_x = !(fxs && !strcmp(fxs, "0"));
        const char *fzs = getenv("GATT_FZ_REV");
        c->fz_rev = !(fzs && !strcmp(fzs, "0"));
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev);
    int rc = GATT_OK;
    auto chk = [&](int r) { if (rc == GATT_OK) rc = r; };
    if (e != cudaSuccess) rc = fail(GATT_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (rc == GATT_OK) {
        cudaError_t es = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (es != cudaSuccess) rc = fail(GATT_ERR_CUDA, cudaGetErrorString(es));
        else c->own_stream = true;
        if (es == cudaSuccess) es = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
        if (es == cudaSuccess) es = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
        if (es == cudaSuccess) es = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
        if (es != cudaSuccess && rc == GATT_OK) rc = fail(GATT_ERR_CUDA, cudaGetErrorString(es));
    }
    if (rc == GATT_OK) {
        chk(alloc_fields(c, &c->qA, 5, nbatch));
        chk(alloc_fields(c, &c->qB, 5, nbatch));
        chk(alloc_fields(c, &c->delta, 5, nbatch));
        chk(alloc_fields(c, &c->d1, nd1(c), nbatch));
        chk(alloc_fields(c, &c->tq, ntq(c), nbatch));
        chk(alloc_fields(c, &c->d2, nd2(c), nbatch));
        chk(alloc_fields(c, &c->P, 1, nbatch));
        chk(alloc_fields(c, &c->tmp, 1, 1));
        chk(alloc_fields(c, &c->tmp_side, 1, 1));
    }
    if (rc == GATT_OK) {
        cudaError_t ea = cudaMalloc(&c->acc, sizeof(unsigned long long) * 5 * nbatch);
        if (ea == cudaSuccess) ea = cudaMalloc(&c->d_params, sizeof(StepParams));
        if (ea == cudaSuccess) ea = cudaMemsetAsync(c->d_params, 0, sizeof(StepParams), c->stream);
        if (ea == cudaSuccess) ea = cudaHostAlloc(&c->h_err, sizeof(int), cudaHostAllocMapped);
        if (ea == cudaSuccess) { *c->h_err = 0; ea = cudaHostGetDevicePointer(&c->d_err, c->h_err, 0); }
        if (ea != cudaSuccess) rc = fail(GATT_ERR_NOMEM, cudaGetErrorString(ea));
    }
    if (rc == GATT_OK) chk(set_sweep_attributes());
    if (rc == GATT_OK) chk(choose_bc_cluster(c));
    if (rc == GATT_OK) chk(ensure_hist(c, 64));
    if (rc == GATT_OK) {
        cudaError_t es = cudaStreamSynchronize(c->stream);
        if (es != cudaSuccess) rc = fail(GATT_ERR_CUDA, cudaGetErrorString(es));
    }
    if (rc != GATT_OK) { gatt_destroy(c); return rc; }
    *out = c;
    return GATT_OK;
}

void gatt_destroy(gatt_ctx *c)
{
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    invalidate_graphs(c);
    for (int d = 0; d < 3; d++) {
        for (int k = 0; k < kMatKinds; k++) {
            DevDir &m = c->mat[d][k];
            cudaFree(m.Rm);
            cudaFree(m.Q);
        }
        cudaFree(c->ltype[d]);
    }
    double *bufs[] = {c->qA, c->qB, c->delta, c->mean, c->d1, c->tq, c->d2, c->P, c->tmp, c->tmp_side, c->tin, c->tout, c->chi, c->hist,
                      c->d_coef1, c->d_coef2, c->d_xs, c->d_hold, c->arn_zeta, c->arn_B, c->arn_base, c->arn_um,
                      c->arn_part, c->arn_h};
    cudaFree(c->arn_region);
    for (double *p : c->dx) cudaFree(p);
    for (double *p : c->dy) cudaFree(p);
    double *dbufs[] = {c->t_delta, c->t_d1, c->t_tq, c->t_d2, c->a_lam, c->a_acc, c->a_arg, c->a_prev, c->a_g,
                       c->a_lq, c->a_ld1, c->a_ltau, c->a_lvt, c->a_s1, c->a_s2, c->a_scr, c->a_ckpt, c->a_seg,
                       c->t_P, c->a_lP, c->a_tape, c->a_tmp, c->g_d1, c->g_tq, c->g_d2, c->dxm, c->dym,
                       c->a_lm, c->a_mscr};
    for (double *p : dbufs) cudaFree(p);
    for (double *p : bufs) cudaFree(p);
    cudaFree(c->d_ops); cudaFree(c->acc); cudaFree(c->d_params);
    cudaFree(c->fsum); cudaFree(c->fpart);
    if (c->h_params) cudaFreeHost(c->h_params);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    delete c;
}

int gatt_set_stream(gatt_ctx *c, void *s)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    TRY(sync_stream(c));
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->own_stream = false;
    c->stream = (cudaStream_t)s;
    if (!s) {
        CU(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_physics(gatt_ctx *c, double Re, double Ma, double Pr, double gamma, double T0)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    const double v[5] = {Re, Ma, Pr, gamma, T0};
    for (double x : v)
        if (!std::isfinite(x) || x <= 0) return fail(GATT_ERR_BADARG, "physical parameters must be positive and finite");
    if (gamma <= 1) return fail(GATT_ERR_BADARG, "gamma must exceed 1");
    c->ph.Re = Re; c->ph.Ma = Ma; c->ph.Pr = Pr; c->ph.gamma = gamma; c->ph.T0 = T0;
    c->phys_set = true;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_matrices(gatt_ctx *c, int dir, int kind, int periodic, int nRHS, int nTypes, const double *A,
                      const double *B, const double *C, const double *D, const double *R, int nBlocks,
                      const int *blocks)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (dir < 1 || dir > 3 || kind < 0 || kind >= kMatKinds)
        return fail(GATT_ERR_BADARG, "dir must be 1..3 and kind 0..5");
    const int d = dir - 1;
    const int N = line_len(c, d);
    if (periodic != 0 && periodic != 1) return fail(GATT_ERR_BADARG, "periodic must be 0 or 1");
    if (nTypes < 1 || nTypes > 255) return fail(GATT_ERR_BADARG, "nTypes must be 1..255");
    // the band wraps around a line at most once (derivs.F90:583-602 index F(i +- l), l < nRHS)
    if (nRHS < 1 || nRHS > N) return fail(GATT_ERR_BADARG, "nRHS out of range (1..N)");
    if (N < 2) return fail(GATT_ERR_BADARG, "direction has a single node; it has no matrices");
    if (!A || !B || !C || !R || (periodic && !D)) return fail(GATT_ERR_BADARG, "missing coefficient array");
    if (nBlocks < 0 || (nBlocks > 0 && !blocks)) return fail(GATT_ERR_BADARG, "bad block list");
    if (nBlocks == 0 && !c->lt_set[d]) return fail(GATT_ERR_BADARG, "no blocks given and none set for this direction");
    const int W = 2 * nRHS - 1;
    const int nA = N - 1, nB = N - periodic;
    // repack to [type][row] (and [type][row][diag] for R), checking every value
    std::vector<double> hA((size_t)nTypes * N, 0.0), hB((size_t)nTypes * N, 0.0), hC((size_t)nTypes * N, 0.0),
        hD((size_t)nTypes * N, 0.0), hR((size_t)nTypes * N * W, 0.0);
    for (int t = 0; t < nTypes; t++) {
        for (int i = 0; i < nA; i++) {
            hA[(size_t)t * N + i] = A[i + (size_t)nA * t];
            hC[(size_t)t * N + i] = C[i + (size_t)nA * t];
        }
        for (int i = 0; i < nB; i++) hB[(size_t)t * N + i] = B[i + (size_t)nB * t];
        if (periodic)
            for (int i = 0; i < N; i++) hD[(size_t)t * N + i] = D[i + (size_t)N * t];
        for (int i = 0; i < N; i++)
            for (int q = 0; q < W; q++) hR[((size_t)t * N + i) * W + q] = R[i + (size_t)N * q + (size_t)N * W * t];
    }
    for (const std::vector<double> *v : {&hA, &hB, &hC, &hD, &hR})
        for (double x : *v)
            if (!std::isfinite(x)) return fail(GATT_ERR_BADCOEF, "non-finite coefficient (a zero pivot gives an infinite B)");
    for (int t = 0; t < nTypes; t++)
        for (int i = 0; i < nB; i++)
            if (hB[(size_t)t * N + i] == 0.0) return fail(GATT_ERR_BADCOEF, "zero reciprocal pivot in B");
    // type map from the blocks (derivs.F90:572-580: blocks(bn,1..5) = t, a1, a2, b1, b2)
    std::vector<uint8_t> lt;
    if (nBlocks > 0) {
        const int na = d == 0 ? c->ny : c->nx;
        const int nbd = d == 2 ? c->ny : c->nz;
        lt.assign((size_t)na * nbd, 0);
        std::vector<uint8_t> seen((size_t)na * nbd, 0);
        for (int bn = 0; bn < nBlocks; bn++) {
            const int t = blocks[bn], a1 = blocks[bn + nBlocks], a2 = blocks[bn + 2 * nBlocks];
            const int b1 = blocks[bn + 3 * nBlocks], b2 = blocks[bn + 4 * nBlocks];
            if (t < 1 || t > nTypes) return fail(GATT_ERR_BADARG, "block type out of range");
            if (a1 < 1 || a2 > na || a1 > a2 || b1 < 1 || b2 > nbd || b1 > b2)
                return fail(GATT_ERR_BADARG, "block line range outside the grid");
            for (int bb = b1; bb <= b2; bb++)
                for (int aa = a1; aa <= a2; aa++) {
                    const size_t L = (size_t)(aa - 1) + (size_t)na * (bb - 1);
                    if (seen[L]) return fail(GATT_ERR_BADARG, "blocks cover a line twice");
                    seen[L] = 1;
                    lt[L] = (uint8_t)(t - 1);
                }
        }
        for (uint8_t s : seen)
            if (!s) return fail(GATT_ERR_BADARG, "blocks leave a line uncovered");
    } else {
        // reuse the type map already set; its types must exist in this matrix set
        std::vector<uint8_t> cur((size_t)nlines(c, d));
        CU(cudaMemcpy(cur.data(), c->ltype[d], cur.size(), cudaMemcpyDeviceToHost));
        for (uint8_t t : cur)
            if (t >= nTypes) return fail(GATT_ERR_BADARG, "existing block types exceed nTypes");
    }
    const int Np = padded_rows(c, d, N, nRHS, periodic);
    const int rpb = choose_rpb(d, N, Np, nRHS, nTypes, (W + 3) / 4 * 4);
    const int P = rpb ? Np / rpb : choose_blocks(N, nRHS, (W + 3) / 4 * 4);
    TRY(sync_stream(c));
    DevDir &m = c->mat[d][kind];
    cudaFree(m.Rm);
    cudaFree(m.Q);
    m = DevDir();
    m.periodic = periodic; m.nR = nRHS; m.nTypes = nTypes; m.N = N; m.W = W; m.Wp = (W + 3) / 4 * 4;
    m.hA = std::move(hA); m.hB = std::move(hB); m.hC = std::move(hC); m.hD = std::move(hD); m.hR = std::move(hR);
    m.Np = rpb ? Np : N;  // a padded length the solver does not take is not kept
    TRY(upload_records(c, m, P, rpb ? Np : N));
    m.rpb = rpb;
    m.family = rpb ? choose_family() : FAM_TILE;
    m.set = true;
    if (nBlocks > 0) {
        if (!c->ltype[d]) CU(cudaMalloc(&c->ltype[d], lt.size()));
        CU(cudaMemcpy(c->ltype[d], lt.data(), lt.size(), cudaMemcpyHostToDevice));
        c->lt_set[d] = true;
        int mx = 0;
        for (uint8_t t : lt) mx = t > mx ? t : mx;
        c->lt_max[d] = mx;
    }
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_time_stepping(gatt_ctx *c, int scheme)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (scheme < 1 || scheme > 3) return fail(GATT_ERR_BADARG, "timeStepping must be 1 (RK4), 2 (Euler) or 3 (SSPRK3)");
    c->time_stepping = scheme;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_filter(gatt_ctx *c, int fx, int fy, int fz, double fct)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (!std::isfinite(fct) || fct == 0) return fail(GATT_ERR_BADARG, "FilterCharTime must be finite and non-zero (-1 = off)");
    c->filt[0] = fx != 0; c->filt[1] = fy != 0; c->filt[2] = (fz != 0) && c->is3d;
    c->fct = fct;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_neumann(gatt_ctx *c, int n1, const double *c1, int n2, const double *c2)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (n1 < 0 || n2 < 0 || (n1 && !c1) || (n2 && !c2)) return fail(GATT_ERR_BADARG, "bad Neumann coefficient arrays");
    c->coef1.assign(c1, c1 + n1);
    c->coef2.assign(c2, c2 + n2);
    c->bc_dirty = true;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_bc(gatt_ctx *c, int var, int kind, int n, const int *ind, const double *val, const int *dirs)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (var < 0 || var > 4 || kind < 0 || kind > 2 || n < 0) return fail(GATT_ERR_BADARG, "bad var/kind/count");
    if (n > 0 && !ind) return fail(GATT_ERR_BADARG, "missing index array");
    if (n > 0 && kind == GATT_BC_DIRICHLET && !val) return fail(GATT_ERR_BADARG, "missing Dirichlet values");
    if (n > 0 && kind != GATT_BC_DIRICHLET && !dirs) return fail(GATT_ERR_BADARG, "missing directions");
    HostBC &h = c->bc[kind][var];
    h.n = n;
    h.ind.assign(ind, ind + (size_t)6 * n);
    if (kind == GATT_BC_DIRICHLET) { h.val.assign(val, val + n); h.dirs.clear(); }
    else { h.dirs.assign(dirs, dirs + n); h.val.clear(); }
    c->bc_dirty = true;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_corners(gatt_ctx *c, int cN, const int *cL, const int *cD, const int *cAd)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (cN < 0 || (cN > 0 && (!cL || !cD || !cAd))) return fail(GATT_ERR_BADARG, "bad corner arrays");
    c->cN = cN;
    c->cL.assign(cL, cL + (size_t)6 * cN);
    c->cD.assign(cD, cD + (size_t)3 * cN);
    c->cAd.assign(cAd, cAd + cN);
    c->bc_dirty = true;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_add_disturbance(gatt_ctx *c, int type, int var, const int *ind, const double *x, int npar, const double *par)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (type != GATT_DIST_LID_DRIVEN && type != GATT_DIST_PERIODIC_SINE && type != GATT_DIST_HOLD_INLET)
        return fail(GATT_ERR_BADARG, "unsupported disturbance type");
    const bool hold = type == GATT_DIST_HOLD_INLET;
    const int need = type == GATT_DIST_PERIODIC_SINE ? 2 : 1;
    if ((!hold && (var < 0 || var > 4 || !x)) || !ind || npar < need || !par)
        return fail(GATT_ERR_BADARG, "bad disturbance arguments");
    Dist d;
    d.type = type; d.var = hold ? 0 : var;
    for (int q = 0; q < 6; q++) d.ind[q] = ind[q];
    for (int q = 0; q < 3; q++)
        if (d.ind[2 * q + 1] < d.ind[2 * q]) return fail(GATT_ERR_BADARG, "empty disturbance box");
    const int nxb = d.ind[1] - d.ind[0] + 1;
    d.xoff = (int)c->distx.size();
    d.par = par[0];
    if (type == GATT_DIST_LID_DRIVEN) {
        if (nxb > 1 && x[nxb - 1] == x[0]) return fail(GATT_ERR_BADARG, "degenerate disturbance coordinates");
        c->distx.insert(c->distx.end(), x, x + nxb);
    } else if (type == GATT_DIST_PERIODIC_SINE) {
        // periodicSine.F90:14-19: pi and alpha are default (single precision) reals there; the
        // factor amplitude*sin(alpha*(x_i - x_1)) of each x is formed here once
        if (nxb < 2 || x[nxb - 1] == x[0]) return fail(GATT_ERR_BADARG, "degenerate disturbance coordinates");
        const float pi = (float)(4.0 * atan(1.0));
        const float alpha = (float)(2.0 * (double)pi / (x[nxb - 1] - x[0]));
        for (int i = 0; i < nxb; i++) c->distx.push_back(par[1] * sin((double)alpha * (x[i] - x[0])));
    }
    c->dists.push_back(d);
    c->bc_dirty = true;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_add_forcing(gatt_ctx *c, int type, const int *ind, int npar, const double *par)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (type != GATT_FORCE_PRESSURE_GRADIENT && type != GATT_FORCE_TURBULENCE)
        return fail(GATT_ERR_BADARG, "forcing type must be GATT_FORCE_PRESSURE_GRADIENT or GATT_FORCE_TURBULENCE");
    if (c->fc.n >= kMaxForcings) return fail(GATT_ERR_BADARG, "at most 4 forcings");
    if (type == GATT_FORCE_TURBULENCE && !c->is3d)
        return fail(GATT_ERR_BADARG, "turbulenceGenerator acts on U, V, W, E: 3-D only");
    const int need = type == GATT_FORCE_TURBULENCE ? 2 : 1;
    if (!ind || npar < need || !par) return fail(GATT_ERR_BADARG, "forcing needs its box and parameters");
    const int lim[3] = {c->nx, c->ny, c->nz};
    for (int d = 0; d < 3; d++)
        if (ind[2 * d] < 1 || ind[2 * d + 1] > lim[d] || ind[2 * d] > ind[2 * d + 1])
            return fail(GATT_ERR_BADARG, "forcing box outside the grid");
    if (!c->fsum) {
        c->fblocks = 2 * c->nsm;
        CU(cudaMalloc(&c->fsum, sizeof(double) * (size_t)c->nb * kMaxForcings * 5));
        CU(cudaMalloc(&c->fpart, sizeof(double) * (size_t)c->nb * kMaxForcings * c->fblocks * 5));
    }
    const int f = c->fc.n++;
    c->fc.type[f] = type;
    for (int q = 0; q < 6; q++) c->fc.box[f][q] = ind[q] - 1;
    c->fc.par[f][0] = par[0];
    c->fc.par[f][1] = need > 1 ? par[1] : 0.0;
    c->fc.N[f] = (double)((long long)(ind[1] - ind[0] + 1) * (ind[3] - ind[2] + 1) * (ind[5] - ind[4] + 1));
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_clear_forcings(gatt_ctx *c)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    c->fc.n = 0;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_clear_disturbances(gatt_ctx *c)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    c->dists.clear();
    c->distx.clear();
    c->bc_dirty = true;
    invalidate_graphs(c);
    return GATT_OK;
}

int gatt_set_sfd(gatt_ctx *c, int type, double Delta, double chiValue, const double *chi)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (type < 0 || type > 2) return fail(GATT_ERR_BADARG, "SFD type must be 0, 1 or 2");
    if (type == 2 && !chi) return fail(GATT_ERR_BADARG, "SFD type 2 needs the chi field");
    if (!std::isfinite(Delta)) return fail(GATT_ERR_BADARG, "SFD Delta must be finite (-1 = frozen mean)");
    c->sfd_type = type;
    c->sfd_delta = Delta;
    invalidate_graphs(c);
    if (type == 0) return GATT_OK;
    if (!c->chi) CU(cudaMalloc(&c->chi, sizeof(double) * c->npts));
    if (type == 1) {
        std::vector<double> h(c->npts, chiValue);
        CU(cudaMemcpy(c->chi, h.data(), sizeof(double) * c->npts, cudaMemcpyHostToDevice));
    } else {
        CU(cudaMemcpy(c->chi, chi, sizeof(double) * c->npts, cudaMemcpyHostToDevice));
    }
    if (!c->mean) TRY(alloc_fields(c, &c->mean, 5, c->nb));
    return GATT_OK;
}

static int copy_state(gatt_ctx *c, int b, int which, double *const *host, bool up)
{
    TRY(check_member(c, b));
    const StateSet q = state_set(c, which);
    for (int f = 0; f < 5; f++) {
        if (!host[f]) continue;
        double *dp = q.v[f] + b * q.bstride;
        if (up) CU(cudaMemcpyAsync(dp, host[f], sizeof(double) * c->npts, cudaMemcpyHostToDevice, c->stream));
        else CU(cudaMemcpyAsync(host[f], dp, sizeof(double) * c->npts, cudaMemcpyDeviceToHost, c->stream));
    }
    TRY(sync_stream(c));
    return GATT_OK;
}

int gatt_upload(gatt_ctx *c, int b, const double *U, const double *V, const double *W, const double *R, const double *E)
{
    double *h[5] = {(double *)U, (double *)V, (double *)W, (double *)R, (double *)E};
    return copy_state(c, b, 0, h, true);
}

int gatt_download(gatt_ctx *c, int b, double *U, double *V, double *W, double *R, double *E)
{
    double *h[5] = {U, V, W, R, E};
    return copy_state(c, b, 0, h, false);
}

static int copy_mean(gatt_ctx *c, int b, double *const *host, bool up)
{
    TRY(check_member(c, b));
    if (!c->mean) TRY(alloc_fields(c, &c->mean, 5, c->nb));
    for (int f = 0; f < 5; f++) {
        if (!host[f]) continue;
        double *dp = c->mean + ((size_t)b * 5 + f) * c->npts;
        if (up) CU(cudaMemcpyAsync(dp, host[f], sizeof(double) * c->npts, cudaMemcpyHostToDevice, c->stream));
        else CU(cudaMemcpyAsync(host[f], dp, sizeof(double) * c->npts, cudaMemcpyDeviceToHost, c->stream));
    }
    TRY(sync_stream(c));
    return GATT_OK;
}

int gatt_upload_mean(gatt_ctx *c, int b, const double *U, const double *V, const double *W, const double *R, const double *E)
{
    double *h[5] = {(double *)U, (double *)V, (double *)W, (double *)R, (double *)E};
    TRY(copy_mean(c, b, h, true));
    c->mean_init = true;
    return GATT_OK;
}

int gatt_download_mean(gatt_ctx *c, int b, double *U, double *V, double *W, double *R, double *E)
{
    double *h[5] = {U, V, W, R, E};
    return copy_mean(c, b, h, false);
}

int gatt_upload_wnew(gatt_ctx *c, int b, const double *Wn)
{
    TRY(check_member(c, b));
    double *h[5] = {nullptr, nullptr, (double *)Wn, nullptr, nullptr};
    return copy_state(c, b, 1, h, true);
}

int gatt_download_wnew(gatt_ctx *c, int b, double *Wn)
{
    TRY(check_member(c, b));
    double *h[5] = {nullptr, nullptr, Wn, nullptr, nullptr};
    return copy_state(c, b, 1, h, false);
}

int gatt_state_device_ptr(gatt_ctx *c, int b, int var, double **dptr)
{
    TRY(check_member(c, b));
    if (var < 0 || var > 4 || !dptr) return fail(GATT_ERR_BADARG, "bad variable or output pointer");
    const StateSet q = state_set(c, 0);
    *dptr = q.v[var] + b * q.bstride;
    return GATT_OK;
}

int gatt_apply_bc(gatt_ctx *c, double t)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (!c->phys_set) return fail(GATT_ERR_STATE, "gatt_set_physics not called");
    if (!std::isfinite(t)) return fail(GATT_ERR_BADARG, "t must be finite");
    TRY(apply_bc(c, state_set(c, 0), c->nb, 0.0, true, t));
    TRY(sync_stream(c));
    if (c->hold_len > 0) c->hold_saved = true;
    return GATT_OK;
}

int gatt_deriv_dir(gatt_ctx *c, int dir, int kind, const double *F, double *dF)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    if (dir < 1 || dir > 3 || kind < 0 || kind >= kMatKinds || !F || !dF) return fail(GATT_ERR_BADARG, "bad arguments");
    if (line_len(c, dir - 1) < 2) return fail(GATT_ERR_BADARG, "direction has a single node");
    TRY(ensure_host_scratch(c));
    CU(cudaMemcpyAsync(c->tin, F, sizeof(double) * c->npts, cudaMemcpyHostToDevice, c->stream));
    const int s0 = 0;
    TRY(sweep(c, dir - 1, kind, c->tin, 0, &s0, c->tout, 0, &s0, 1, 1, 0.0, nullptr));
    CU(cudaMemcpyAsync(dF, c->tout, sizeof(double) * c->npts, cudaMemcpyDeviceToHost, c->stream));
    TRY(sync_stream(c));
    return GATT_OK;
}

int gatt_rhs(gatt_ctx *c, const double *U, const double *V, const double *W, const double *R, const double *E,
             double *dU, double *dV, double *dW, double *dR, double *dE)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    TRY(check_ready(c, false));
    if (!U || !V || !R || !E || !dU || !dV || !dR || !dE || (c->is3d && (!W || !dW)))
        return fail(GATT_ERR_BADARG, "missing field");
    TRY(ensure_host_scratch(c));
    const double *in[5] = {U, V, W, R, E};
    for (int f = 0; f < 5; f++) {
        if (!in[f]) continue;
        CU(cudaMemcpyAsync(c->tin + f * c->npts, in[f], sizeof(double) * c->npts, cudaMemcpyHostToDevice, c->stream));
    }
    StateSet q, o;
    for (int f = 0; f < 5; f++) { q.v[f] = c->tin + f * c->npts; o.v[f] = c->tout + f * c->npts; }
    q.bstride = o.bstride = 5 * c->npts;
    TRY(rhs_stage(c, q, q, o, RK_STORE_RHS, 1, c->d1, c->tq, c->d2, nullptr));
    double *out[5] = {dU, dV, dW, dR, dE};
    for (int f = 0; f < 5; f++) {
        if (!out[f] || (!c->is3d && f == 2)) continue;
        CU(cudaMemcpyAsync(out[f], c->tout + f * c->npts, sizeof(double) * c->npts, cudaMemcpyDeviceToHost, c->stream));
    }
    TRY(sync_stream(c));
    return GATT_OK;
}

int gatt_filter(gatt_ctx *c, double blend)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    TRY(check_ready(c, true));
    TRY(filter_set(c, state_set(c, 0), c->nb, blend > 0 ? blend : 0.0, nullptr));
    TRY(sync_stream(c));
    return GATT_OK;
}

int gatt_step(gatt_ctx *c, double t, double dt, double *maxChange)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    return run_steps(c, 1, t, dt, maxChange, true);
}

int gatt_run(gatt_ctx *c, int nsteps, double t0, double dt, double *maxChange)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    return run_steps(c, nsteps, t0, dt, maxChange, true);
}

int gatt_max_velocity(gatt_ctx *c, double *vmax)
{
    if (!c || !vmax) return fail(GATT_ERR_BADARG, "null argument");
    CU(cudaMemsetAsync(c->acc, 0, sizeof(unsigned long long) * 3 * c->nb, c->stream));
    TRY(before_launch(c, PC_OTHER));
    k_maxvel<<<dim3(grid_for(c, c->npts), c->nb), kBlock, 0, c->stream>>>(state_set(c, 0), c->acc, c->npts);
    TRY(after_launch(c));
    std::vector<unsigned long long> h(3 * c->nb);
    CU(cudaMemcpyAsync(h.data(), c->acc, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    TRY(sync_stream(c));
    for (size_t i = 0; i < h.size(); i++) memcpy(&vmax[i], &h[i], sizeof(double));
    return GATT_OK;
}

int gatt_arnoldi(gatt_ctx *c, int m, int nsteps, double t0, double dt, double eps, const double *base,
                 const double *v0, const unsigned char *region, double *H)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    return arnoldi(c, m, nsteps, t0, dt, eps, base, v0, region, H);
}

int gatt_arnoldi_vector(gatt_ctx *c, int b, int j, double *out)
{
    if (!c || !out) return fail(GATT_ERR_BADARG, "null argument");
    TRY(check_member(c, b));
    if (!c->arn_zeta || j < 0 || j > c->arn_m) return fail(GATT_ERR_BADARG, "no such basis vector");
    const long long n = c->npts, len = (long long)arn_nv(c) * n;
    const double *z = c->arn_zeta + (long long)b * (c->arn_m + 1) * len + (long long)j * len;
    for (int f = 0; f < 5; f++) {
        const int v = c->is3d ? f : (f == 2 ? -1 : (f < 2 ? f : f - 1));
        if (v < 0) memset(out + f * n, 0, sizeof(double) * n);
        else CU(cudaMemcpyAsync(out + f * n, z + v * n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    }
    TRY(sync_stream(c));
    return GATT_OK;
}

int gatt_rhs_jvp(gatt_ctx *c, const double *q, const double *dq, double *dk)
{
    if (!c || !q || !dq || !dk) return fail(GATT_ERR_BADARG, "null argument");
    return rhs_jvp(c, q, dq, dk);
}

int gatt_rhs_vjp(gatt_ctx *c, const double *q, const double *a, double *lam)
{
    if (!c || !q || !a || !lam) return fail(GATT_ERR_BADARG, "null argument");
    return rhs_vjp(c, q, a, lam);
}

int gatt_jvp(gatt_ctx *c, int nsteps, double t0, double dt, const double *dq0, double *dqN)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    return jvp(c, nsteps, t0, dt, dq0, dqN);
}

int gatt_vjp(gatt_ctx *c, int nsteps, double t0, double dt, int checkpoint_every, const double *lamN, double *lam0)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    return vjp(c, nsteps, t0, dt, checkpoint_every, lamN, lam0);
}

int gatt_autotune(gatt_ctx *c, int reps, int *family, int *blocks, double *us)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    return autotune(c, reps, family, blocks, us);
}

int gatt_selftest_pipeline_timeout(gatt_ctx *c)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    TRY(check_ready(c, false));
    TRY(sync_stream(c));
    // one x-direction first-derivative sweep of member 0's U through the copy ring, every
    // barrier expecting 16 bytes that never come
    const DevDir &m = c->mat[0][0];
    if (!m.set || m.family != FAM_PIPE) return fail(GATT_ERR_STATE, "x lines do not use the pipelined solver");
    SweepArgs a;
    memset(&a, 0, sizeof(a));
    const StateSet q = state_set(c, 0);
    a.in = q.v[0]; a.out = c->tmp; a.npts = c->npts;
    a.nx = c->nx; a.ny = c->ny; a.nz = c->nz; a.N = m.rows; a.Nreal = m.N; a.nlines = nlines(c, 0);
    a.es = 1; a.os = 0; a.tiles_per_row = (c->nx + kLanes - 1) / kLanes;
    a.Rm = m.Rm; a.Q = m.Q; a.W = m.W; a.Wp = m.Wp; a.P = m.P; a.ltype = c->ltype[0];
    a.epi = EPI_STORE; a.dir = 0; a.nf = 1; a.ntiles = (a.nlines + kLanes - 1) / kLanes; a.njobs = a.ntiles;
    a.fd_ntiles = make_fastdiv(a.ntiles); a.fd_nf = make_fastdiv(1); a.fd_tpr = make_fastdiv(a.tiles_per_row);
    a.err = c->d_err; a.ntypes = m.nTypes; a.tx_extra = 16;
    const int r = launch_psweep(c, m, 0, a, 1, PC_OTHER);
    if (r != GATT_OK) return r;
    return sync_stream(c);  // GATT_ERR_TIMEOUT when every wait gave up as intended
}

int gatt_synchronize(gatt_ctx *c)
{
    if (!c) return fail(GATT_ERR_BADARG, "null context");
    TRY(sync_stream(c));
    return GATT_OK;
}

long long gatt_kernel_launches(gatt_ctx *c) { return c ? c->launches : -1; }

int gatt_max_change_noalloc(int nsets, int nvar, long long n, const double *const *a, const double *const *b,
                            double *maxChange, void *stream)
{
    if (nsets < 1 || nvar < 1 || nvar > 5 || n < 1 || !a || !b || !maxChange)
        return fail(GATT_ERR_BADARG, "gatt_max_change_noalloc: need nsets >= 1, 1 <= nvar <= 5, n >= 1 and all arrays");
    if ((long long)nsets * nvar > kMaxChangeSlots)
        return fail(GATT_ERR_BADARG, "gatt_max_change_noalloc: nsets*nvar exceeds the " + std::to_string(kMaxChangeSlots) +
                                         " accumulators of its static scratch");
    cudaStream_t st = (cudaStream_t)stream;
    // the result comes back through a synchronised copy, which a capturing stream refuses
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CU(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(GATT_ERR_STATE, "gatt_max_change_noalloc: the stream is being captured; the call synchronises "
                                    "it and returns host values, so it cannot run inside a capture");
    PtrSets ps;
    for (int k = 0; k < nsets * nvar; k++) {
        if (!a[k] || !b[k]) return fail(GATT_ERR_BADARG, "gatt_max_change_noalloc: null field pointer");
        ps.a[k] = a[k];
        ps.b[k] = b[k];
    }
    unsigned long long *acc = nullptr;
    TRY(noalloc_scratch(&acc));
    // the array keeps the previous call's maxima: start this call from zero
    CU(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * nsets * nvar, st));
    int dev = 0, nsm = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    long long g = (n + kBlock - 1) / kBlock;
    if (g > (long long)nsm * 8) g = (long long)nsm * 8;
    k_maxchange_sets<<<dim3((unsigned)g, nsets), kBlock, 0, st>>>(ps, nvar, acc, n);
    CU(cudaGetLastError());
    unsigned long long h[kMaxChangeSlots];
    CU(cudaMemcpyAsync(h, acc, sizeof(unsigned long long) * nsets * nvar, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    for (int k = 0; k < nsets * nvar; k++) memcpy(&maxChange[k], &h[k], sizeof(double));
    return GATT_OK;
}

const char *gatt_profile_name(int cls) { return (cls >= 0 && cls < PC_N) ? kProfNames[cls] : nullptr; }

int gatt_profile_kernels(gatt_ctx *c, double t0, double dt, int nsteps, double *ms, double *launches)
{
    if (!c || !ms || !launches || nsteps < 1) return fail(GATT_ERR_BADARG, "bad arguments");
    TRY(check_ready(c, true));
    TRY(ensure_hist(c, 1));
    if (c->sfd_type > 0 && !c->mean_init) return fail(GATT_ERR_STATE, "run a step before profiling with SFD");
    TRY(check_hold(c));
    for (int i = 0; i < PC_N; i++) { ms[i] = 0; launches[i] = 0; }
    double t = t0;
    int rc = GATT_OK;
    for (int s = 0; s < nsteps && rc == GATT_OK; s++) {
        c->h_params[0].t = t; c->h_params[0].dt = dt; c->h_params[0].slot = 0;
        CU(cudaMemcpyAsync(c->d_params, &c->h_params[0], sizeof(StepParams), cudaMemcpyHostToDevice, c->stream));
        c->profiling = true;
        rc = step_body(c);
        c->profiling = false;
        TRY(sync_stream(c));
        size_t q = 0;
        for (size_t i = 0; i < c->ev_cls.size(); i++, q += 2) {
            float e = 0;
            cudaEventElapsedTime(&e, c->ev_pool[q], c->ev_pool[q + 1]);
            ms[c->ev_cls[i]] += e;
            launches[c->ev_cls[i]] += 1;
        }
        for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
        c->ev_pool.clear();
        c->ev_cls.clear();
        c->cur ^= 1;
        t = t + dt;
    }
    for (int i = 0; i < PC_N; i++) {
        if (launches[i] > 0) ms[i] /= launches[i];
        launches[i] /= nsteps;
    }
    return rc;
}

}  // extern "C"
