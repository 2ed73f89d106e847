// mps_internal.cuh -- context layout and device helpers shared by the
// solver's translation units.
//
// Layout in HBM: structure-of-arrays, particles in cell order (re-sorted
// every step by (Laplacian-grid cell, x, original id); NEIGHBOR's counting
// sort, functions.cu:2820-2852, orders a cell by id alone, and that order is
// formed when the permutation is downloaded).  Neighbour lists and the PPE matrix are
// row-major with a fixed row capacity: entry k of row i lives at i*cap + k.
// Kernels over the Laplacian-radius list (about 300 entries per row in 3D)
// give each row a whole warp; kernels over the PND-radius list (about 50)
// give each row a group of GS lanes; either way a row streams contiguously.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <thread>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/voxarmps.h"

// NVTX range over a host scope (stages, graph capture and replay, I/O): a
// profiler's timeline shows them; without one attached they cost nothing
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace vmps {

constexpr int kBlock = 256;

// Cell grid of one support radius, NEIGHBOR's (functions.cu:2790-2802): x and
// y cells of size re, z cells of size re + DELTA (3D).
struct Grid {
    int ncx, ncy, ncz, tnc;
    double re, rez;
    double xmin, ymin, zmin;
};

// NEIGHBOR's cell grid for support radius re over the box of f: each axis
// count int((max - min) / size) + 1 (functions.cu:2790-2802).  The quotients
// are checked in floating point before the conversion and the product is
// formed in 64 bits, so a box that is not finite, inverted, or holds more
// than max_cells cells (in total or along one axis) returns false instead of
// wrapping around.
inline bool grid_for(double xmin, double xmax, double ymin, double ymax, double zmin,
                     double zmax, int dim, double re, double delta, long long max_cells,
                     Grid* out)
{
    if (!(re > 0)) return false;
    auto axis = [&](double lo, double hi, double size, int* n) {
        const double q = (hi - lo) / size;
        if (!(q >= 0.0) || !(q < (double)max_cells)) return false;  // NaN fails as well
        *n = (int)q + 1;
        return (long long)*n <= max_cells;
    };
    Grid g;
    g.re = re;
    g.rez = dim == 3 ? re + delta : re;
    g.xmin = xmin;
    g.ymin = ymin;
    g.zmin = zmin;
    g.ncz = 1;
    if (!axis(xmin, xmax, re, &g.ncx) || !axis(ymin, ymax, re, &g.ncy)) return false;
    if (dim == 3 && !axis(zmin, zmax, g.rez, &g.ncz)) return false;
    const long long t = (long long)g.ncx * g.ncy * g.ncz;
    if (t > max_cells) return false;
    g.tnc = (int)t;
    *out = g;
    return true;
}

// Squared-distance thresholds equivalent to the reference's sqrt() compares
// (sqrt is correctly rounded on host and device, so the equivalence is exact).
struct Cutoff {
    double d2;       // 2D: d2 < d2 (strict); 3D: d2 <= d2
    int dim;
};

struct DeviceError {
    unsigned int bits;
};

// 2D cutoffs:  sqrt(d2) <  c  <=>  d2 <  sqrt_cut(c, true)
// 3D cutoffs:  sqrt(d2) <= c  <=>  d2 <= sqrt_cut(c, false)
// sqrt is correctly rounded on the host and on the device, so comparing the
// squared distance with these thresholds takes the reference's decisions.
inline double sqrt_cut(double c, bool strict)
{
    double s = c * c;
    if (strict) {
        while (std::sqrt(s) < c) s = std::nextafter(s, INFINITY);
        while (s > 0 && std::sqrt(std::nextafter(s, 0.0)) >= c) s = std::nextafter(s, 0.0);
    } else {
        while (std::sqrt(s) > c) s = std::nextafter(s, 0.0);
        while (std::sqrt(std::nextafter(s, INFINITY)) <= c) s = std::nextafter(s, INFINITY);
    }
    return s;
}

// Kernel function W() of one radius in the form the stage kernels evaluate:
// support tests on d2 against exact thresholds (q < 1 <=> d2 < lt, q <= 1
// <=> d2 <= le), magnitudes from rD = rsqrt(d2).
struct WK {
    double re, inv_re, lt, le;
    int ktype;
};

inline WK make_wk(int ktype, double re)
{
    WK k;
    k.re = re;
    k.inv_re = 1.0 / re;
    k.lt = sqrt_cut(re, true);
    k.le = sqrt_cut(re, false);
    k.ktype = ktype;
    return k;
}

}  // namespace vmps

struct vmps_gnn;  // learned CG initial guess (mps_gnn.cu)

struct mps_ctx {
    mps_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;   // captures the CG loop body into its while node
    std::string msg;
    int n = 0, pitch = 0;
    int gp = 0, wp = 0, fp = 0;
    int fp2 = 0;  // particles of the second fluid (ptype 2)
    bool p4s_bcon = false;  // P4s.w holds bcon (BCON ran after the last PREDICTION)
    vmps::Grid gl{}, gs{};
    double cut_l = 0, cut_s = 0;  // squared-distance thresholds
    int cap_l = 0, cap_s = 0;
    double n0_s = 0, n0_l = 0, lambda_l = 0;
    vmps_gnn* gnn = nullptr;
    // launch shapes picked by mps_autotune / mps_set_tuning
    int tune_small_wide = 0;  // lanes per PND-radius row: SmallG (0) or twice that (1)
    int tune_cg_bps = 0;      // CG grid blocks per SM (0: as many as fit, at most 8)
    int cg_iters = 0;
    int cg_loop_kernels = 4, cg_nspmv = 0;
    bool ppe_pending = false;
    int ppe_warm = 1;  // initial guess of the last assembly (0: zero)
    // CUDA graph of one step per buffer parity (the reorder double-buffers
    // the persistent state, so the step's pointers alternate with period 2)
    // (and per mps_step_io form: index parity + 2 when the step applies the
    // velocities and pressure that mps_step_io copied in beside it)
    bool use_graph = false;
    cudaGraphExec_t gexec[4] = {nullptr, nullptr, nullptr, nullptr};
    long gkernels[4] = {0, 0, 0, 0};
    int gdefer[4] = {0, 0, 0, 0};  // the deferred-field mask each graph applies
    // mps_step_io: u, v, w, p travel on their own stream while the neighbour
    // search runs and are applied after its reorder (bit k: field k of
    // x, y, z, u, v, w, p; ev_state marks the end of their copies)
    cudaStream_t stream_io = nullptr;
    cudaEvent_t ev_io = nullptr, ev_state = nullptr;
    cudaEvent_t ev_out[7] = {};  // mps_get_state: field k permuted, its copy may start
    int state_defer = 0;
    long swaps = 0;
    double cg_relres = 0;
    double cg_r0 = 0;  // relative residual of the CG starting point
    long steps = 0;
    bool initialized = false;
    unsigned int host_err = 0;

    // persistent particle state, cell order (double-buffered for the reorder)
    double *x = nullptr, *y = nullptr, *z = nullptr, *u = nullptr, *v = nullptr, *w = nullptr;
    double *p = nullptr, *pnew = nullptr, *phat = nullptr, *un = nullptr, *vn = nullptr,
           *wn = nullptr, *rho = nullptr, *nd = nullptr, *pold = nullptr;
    int *ptype = nullptr, *oid = nullptr, *scene = nullptr;
    // slab decomposition: 1 for the particles this context owns, 0 for ghost
    // copies of a neighbouring rank's particles (all 1 in a single context)
    int* own = nullptr;
    // rows outside this context's PPE system: bcon != 0 or a ghost (the CG
    // kernels' row mask; equal to bcon when every particle is owned)
    int* sysmask = nullptr;
    int* stage_ids = nullptr;  // H2D staging of particle indices (row exchanges)
    int* slot_of = nullptr;    // slot of each caller-order particle index
    // batched scenes (nscenes == 1: one scene, the global box)
    int nscenes = 1;
    double* sbox = nullptr;     // 6 per scene
    double* spmax = nullptr;    // per scene
    int *sfirst = nullptr, *slast = nullptr;  // slot range of each scene
    double* sbb = nullptr;      // per-scene b.b
    double* srr = nullptr;      // per-scene r.r
    int* sok = nullptr;         // per-scene converged flag
    // per-step scratch fields
    double *xs = nullptr, *ys = nullptr, *zs = nullptr, *us = nullptr, *vs = nullptr,
           *ws = nullptr, *nds = nullptr, *C = nullptr, *meu = nullptr, *neut = nullptr,
           *t1 = nullptr, *t2 = nullptr, *t3 = nullptr, *source = nullptr, *diag = nullptr;
    int* bcon = nullptr;
    // SPS strain tensor (6 comps) and collision outputs (swapped with the state)
    double* S6 = nullptr;
    double *xc = nullptr, *yc = nullptr, *zc = nullptr, *uc = nullptr, *vc = nullptr,
           *wc = nullptr;
    // packed gathers: positions (x, y, z, ptype), predicted positions,
    // collision output, velocities (u, v, w, -) and (pnew, phat) pairs
    double4 *P4 = nullptr, *P4s = nullptr, *P4c = nullptr, *U4 = nullptr;
    double4* PP4 = nullptr;  // (x, y, z, previous pressure) for PREDICTION's pressure sums
    float4* P4f = nullptr;   // positions relative to the box minimum, FP32, w = ptype
    float4* U4f = nullptr;   // velocities, FP32 (mixed precision's viscous sums)
    float4* P4sf = nullptr;  // precision 2: predicted positions relative to the box, FP32
    float2* PH32 = nullptr;  // precision 2: (pnew, phat) in FP32
    double screen_abs = 0;   // bound on |d2_fp32 - d2_exact| for the screening test
    double2* PH = nullptr;
    // sort / cells
    int *cell_l = nullptr, *cell_s = nullptr;      // per slot, 1-based Cnum
    int *bpos_l = nullptr, *bpos_s = nullptr;      // position inside the bucket
    int *cnt_l = nullptr, *cst_l = nullptr;        // per cell count / start
    int *cnt_s = nullptr, *cst_s = nullptr;
    int *bslot_l = nullptr, *boid_l = nullptr;     // bucketed slots / ids
    unsigned long long* bx_l = nullptr;            // order keys of x, bucketed (primary grid)
    unsigned long long* bx_s = nullptr;            // the same on the PND grid
    unsigned long long* key_s = nullptr;           // order keys of x in the PND grid's order
    int *bslot_s = nullptr, *boid_s = nullptr;
    int *src = nullptr, *inv = nullptr;            // new slot <- old slot, old -> new
    int *perm_s = nullptr, *perm_s_tmp = nullptr;  // small-grid cell order (slots)
    // lists (slot-major)
    int *nbr_l = nullptr, *len_l = nullptr, *nbr_s = nullptr, *len_s = nullptr;
    // PPE matrix (compact slot-major ELL) and CG vectors
    int *mcol = nullptr, *mlen = nullptr, *moff = nullptr;  // CSR: row i at moff[i]
    int2* mrow = nullptr;  // (moff, mlen) per row, mlen -1 for rows outside the system
    double* mval = nullptr;
    double *pres_x = nullptr, *pres_y = nullptr, *pres_z = nullptr;  // prediction pressure sums
    double *cg_r = nullptr, *cg_z = nullptr, *cg_p = nullptr, *cg_s = nullptr;
    // mixed precision (precision 1): FP32 copy of the matrix values and the
    // FP32 inner-CG vectors (correction d, residual, z, direction, A p)
    int2* mcv32 = nullptr;  // mixed precision: FP32 CSR copy, (column, value bits) per entry
    float *ir_d = nullptr, *ir_r = nullptr, *ir_z = nullptr, *ir_p = nullptr, *ir_s = nullptr;
    int cg_outer = 0;
    double* cg_part = nullptr;   // block partial sums
    size_t cg_part_cap = 0;      // doubles in cg_part
    double* cg_scal = nullptr;   // device scalars (rz, bb, rr, ...)
    int* cg_flag = nullptr;      // [0] done, [1] iterations
    unsigned int* cg_bar = nullptr;  // k_cg_loop's grid barrier: arrivals, monotonic per launch
    int* cg_flag_host = nullptr; // pinned
    double* red_host = nullptr;  // pinned scratch for scalars
    unsigned int* d_err = nullptr;
    unsigned int* h_err = nullptr;  // pinned
    int* len_max = nullptr;         // [0] max len_l, [1] max len_s (diagnostics)
    unsigned long long* d_max = nullptr;  // atomic max of a non-negative double
    int* scan_tmp = nullptr;        // tile sums of the cell-count scans
    double* stage_in = nullptr;     // H2D staging for mps_set_field / mps_set_rows
    double* stage_io = nullptr;     // 7 x pitch: mps_set_state / mps_get_state staging
    // profiling (CUDA events on the context stream)
    bool profile = false;
    cudaEvent_t ev[8] = {};
    std::vector<cudaEvent_t> ev_spmv;
    double ms_stage[5] = {0, 0, 0, 0, 0};
    double spmv_ms = 0, lists_ms = 0;
    long spmv_launches = 0, lists_launches = 0;
    // reorder double-buffers (same shapes as the persistent fields)
    std::vector<void*> alts;
    std::vector<void*> owned;
    std::vector<void*> pinned;
    // asynchronous VTU snapshots: pinned host copies (8 fields) filled by
    // device-to-host copies on the stream, written by a host thread
    double* snap = nullptr;
    int snap_n = 0;
    cudaEvent_t snap_ev = nullptr;
    std::thread snap_thread;
    int snap_status = 0;
};

namespace vmps {

// ---------------- device helpers (exact IEEE FP64, no contraction) ----------
// Every FP64 translation unit is compiled with -fmad=false so that a*b + c is
// two roundings, as in the reference's x86 build.

__host__ __device__ inline double kernel_w(double R, int ktype, int dim, double re)
{
    // W(), functions.cu:32-74
    double w = 0.0;
    double q = R / re;
    switch (ktype) {
    case 1:
        if (q < 0.5) w = 2.0 - 4.0 * (q * q);
        else if (q <= 1.0) w = (2 * q - 2) * (2 * q - 2);
        else w = 0;
        break;
    case 2:
        if (q < 1.0) w = (1 / q) - 1;
        else w = 0;
        break;
    case 3: {
        double Cc = 0.0;
        if (dim == 1) Cc = 0.6666;
        if (dim == 2) Cc = 1.43 * 3.14;
        if (dim == 3) Cc = 1 / 3.14;
        if (R < re) w = Cc / pow(re, (double)dim) * (1 - 1.5 * (q * q) + 0.75 * pow(q, 3.0));
        else if (R >= re && R < (2.0 * re)) w = Cc / pow(re, (double)dim) * (0.25 * pow(2.0 - q, 3.0));
        else w = 0;
        break;
    }
    case 5:
        if (q <= 1.0) w = 1.5 * log(1 / (q + 0.000001));
        else w = 0;
        break;
    case 6:
        if (q <= 1.0) w = pow((1 - q), 3.0);
        else w = 0;
        break;
    }
    return w;
}

template <int DIM>
__device__ __forceinline__ double dist2(double dx, double dy, double dz)
{
    // pow(dx,2)+pow(dy,2)[+pow(dz,2)] as the reference's -O2 build evaluates it
    if (DIM == 3) return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

__device__ __forceinline__ void set_error(unsigned int* e, unsigned int bit)
{
    atomicOr(e, bit);
}

// Cell of a position in one grid (functions.cu:2823-2835); returns false when
// the reference's int() would leave [1, nc] on some axis.
template <int DIM>
__device__ __forceinline__ bool cell_coords(const Grid& g, double x, double y, double z, int& ic,
                                            int& jc, int& kc)
{
    double fx = __ddiv_rn(x - g.xmin, g.re);
    double fy = __ddiv_rn(y - g.ymin, g.re);
    bool ok = (fx > -1.0) && (fx < (double)g.ncx) && (fy > -1.0) && (fy < (double)g.ncy);
    ic = ok ? (int)fx + 1 : 1;
    jc = ok ? (int)fy + 1 : 1;
    kc = 1;
    if (DIM == 3) {
        double fz = __ddiv_rn(z - g.zmin, g.rez);
        bool okz = (fz > -1.0) && (fz < (double)g.ncz);
        kc = okz ? (int)fz + 1 : 1;
        ok = ok && okz;
    }
    return ok;
}

inline int grid_blocks(long n) { return (int)((n + kBlock - 1) / kBlock); }

// W() of functions.cu:32-74 from d2 and rD = rsqrt(d2)
template <int DIM>
__device__ __forceinline__ double w_fast(const WK& k, double d2, double rD)
{
    if (k.ktype == 2) return d2 < k.lt ? k.re * rD - 1.0 : 0.0;
    double R = d2 * rD, q = R * k.inv_re;
    switch (k.ktype) {
    case 6:
        if (d2 <= k.le) {
            double t = 1.0 - q;
            return t * t * t;
        }
        return 0.0;
    case 1:
        if (q < 0.5) return 2.0 - 4.0 * (q * q);
        if (d2 <= k.le) {
            double t = 2 * q - 2;
            return t * t;
        }
        return 0.0;
    case 5:
        return d2 <= k.le ? 1.5 * log(1 / (q + 0.000001)) : 0.0;
    default:
        return kernel_w(R, k.ktype, DIM, k.re);
    }
}

__device__ __forceinline__ double rsq(double d2) { return rsqrt(d2); }

// W() in FP32 (mixed precision): same support tests on float thresholds
struct WKf {
    float re, inv_re, lt, le;
    int ktype;
};
inline WKf make_wkf(const WK& k)
{
    return WKf{(float)k.re, (float)k.inv_re, (float)k.lt, (float)k.le, k.ktype};
}
template <int DIM>
__device__ __forceinline__ float w_fast32(const WKf& k, float d2)
{
    const float rD = rsqrtf(d2);
    if (k.ktype == 2) return d2 < k.lt ? __fmaf_rn(k.re, rD, -1.f) : 0.f;
    const float R = d2 * rD, q = R * k.inv_re;
    switch (k.ktype) {
    case 6:
        if (d2 <= k.le) {
            const float t = 1.f - q;
            return t * t * t;
        }
        return 0.f;
    case 1:
        if (q < 0.5f) return 2.f - 4.f * (q * q);
        if (d2 <= k.le) {
            const float t = 2.f * q - 2.f;
            return t * t;
        }
        return 0.f;
    case 5:
        return d2 <= k.le ? 1.5f * logf(1.f / (q + 0.000001f)) : 0.f;
    default:
        return (float)kernel_w((double)R, k.ktype, DIM, (double)k.re);
    }
}

// A group of G consecutive lanes (G divides 32) that cooperates on one row.
template <int G>
struct Grp {
    int lane;       // 0..G-1
    long gid;       // global group index
    unsigned mask;  // this group's lanes inside the warp
    unsigned base;  // first warp lane of the group
    __device__ __forceinline__ Grp()
    {
        long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
        lane = (int)(t % G);
        gid = t / G;
        base = (threadIdx.x & 31u) - (unsigned)lane;
        mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << base);
    }
    // sum over the group, result in every lane (fixed butterfly order)
    __device__ __forceinline__ double sum(double v) const
    {
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        return v;
    }
    __device__ __forceinline__ float sumf(float v) const
    {
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        return v;
    }
    __device__ __forceinline__ double min(double v) const
    {
        for (int o = G / 2; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(mask, v, o));
        return v;
    }
    // ballot restricted to the group, bit k = group lane k
    __device__ __forceinline__ unsigned ballot(bool p) const
    {
        unsigned m = __ballot_sync(mask, p);
        return (G == 32) ? m : (m >> base) & ((1u << G) - 1u);
    }
};

// lanes per PND-radius row
template <int DIM>
struct SmallG {
    // 4 lanes in 2D and 3D (3D measured: 8 lanes cost 0.8 ms more per step on
    // the 1.6 M-particle dam, 2 lanes slow the list build); the autotuner may
    // double it
    static constexpr int G = 4;
};

}  // namespace vmps

// host-side helpers implemented in mps_context.cu
int vmps_check(mps_ctx* ctx, cudaError_t e, const char* what);
#define VMPS_CUDA(ctx, call)                                   \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return vmps_check(ctx, _e, #call); \
    } while (0)

// stage launchers (defined in the kernel translation units)
int vmps_neighbors(mps_ctx* ctx);
// track_max: also the largest value into ctx->d_max (n0 at mps_init)
int vmps_pnd(mps_ctx* ctx, int at_star, int correct, int which_list, double* out,
             bool track_max = false);
int vmps_max_reduce(mps_ctx* ctx, const double* a, double* result);
int vmps_sps(mps_ctx* ctx);
int vmps_vfraction(mps_ctx* ctx);
int vmps_viscosity(mps_ctx* ctx);
int vmps_predict(mps_ctx* ctx);
int vmps_bcon(mps_ctx* ctx);
int vmps_pressure_wc(mps_ctx* ctx);
int vmps_ppe(mps_ctx* ctx);
int vmps_ppe_finish(mps_ctx* ctx);
int vmps_ppe_apply(mps_ctx* ctx, const double* x, double* y);
int vmps_gnn_guess(mps_ctx* ctx);
int vmps_gnn_prepare(mps_ctx* ctx);
bool vmps_gnn_in_use(const mps_ctx* ctx);
void vmps_gnn_reset(mps_ctx* ctx);
void vmps_gnn_free(mps_ctx* ctx);
void vmps_drop_graphs(mps_ctx* ctx);
void vmps_reorder_swap(mps_ctx* ctx);
int vmps_phat(mps_ctx* ctx);
int vmps_pressgrad(mps_ctx* ctx);
int vmps_integrate(mps_ctx* ctx);
int vmps_collision(mps_ctx* ctx);
int vmps_commit(mps_ctx* ctx);
int vmps_count_launch(int k);
int vmps_pack(mps_ctx* ctx);
int vmps_pack_u(mps_ctx* ctx);
int vmps_state_apply(mps_ctx* ctx);
int vmps_scan(mps_ctx* ctx, int m, const int* in, int* out);
