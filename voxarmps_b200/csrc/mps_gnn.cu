// mps_gnn.cu -- learned initial guess for the PPE's conjugate gradients.
//
// A small message-passing network on the PND-radius neighbour graph (the
// lists NEIGHBOR builds for n, n* and the gradient) predicts the pressure
// increment of the coming solve from per-particle inputs: the PND deviation
// (n* - n0) / n0, the previous pressure, and the particle kind.  The
// prediction replaces the previous pressure as CG's starting point; CG still
// runs to the same relative residual, so the network changes the iteration
// count and never the answer.  There is no counterpart in the reference,
// whose CG starts from zero (functions.cu:2503) or, on its GPU path, from
// the previous pressure.
//
// Network (hidden width H = 64, L layers, inputs padded to F = 8):
//   h0 = relu(We f + be)
//   m_l = mean over the list of i of h_(l-1) of the neighbours
//   h_l = h_(l-1) + relu(W_l [h_(l-1), m_l] + b_l)          l = 1..L
//   y   = wd . h_L + bd,   guess = p_prev + pref * y   (unknown rows)
// with pref = max(rms of p_prev over the unknown rows, rho1 |g| l0).
//
// Precision: weights and activations are stored in BF16; sums accumulate
// in FP32.  Each layer's product W [h, m] is one [nodes x 128] x [128 x 64]
// BF16 GEMM on the tensor cores (tcgen05.mma, FP32 accumulator in tensor
// memory, k_gnn_layer_tc); the aggregation, encoder, decoder and the
// backward pass are CUDA-core kernels with sums in a fixed order.  Training
// keeps FP32 master weights, takes Adam steps on the chosen objective and
// reduces weight gradients through fixed per-block partials
// (deterministic).
#include <cuda_bf16.h>

#include "mps_internal.cuh"

using namespace vmps;

namespace {

constexpr int H = 64;
constexpr int F = 8;
constexpr int kMaxLayers = 8;
constexpr int kThreads = 256;
constexpr int kWgradBlocks = 296;  // 2 per SM: fixed, so partial sums are deterministic
constexpr int kTile = 16;          // nodes staged per tile in the weight-gradient kernel
constexpr int kMaxE = 2 * H * H + H;
constexpr int kPerThread = (kMaxE + kThreads - 1) / kThreads;

typedef __nv_bfloat16 bf16;
typedef __nv_bfloat162 bf162;

struct Layout {
    int L = 0, P = 0;
    int We = 0, be = 0, W[kMaxLayers] = {}, b[kMaxLayers] = {}, wd = 0, bd = 0;
};

Layout make_layout(int L)
{
    Layout y;
    y.L = L;
    int o = 0;
    y.We = o;
    o += H * F;
    y.be = o;
    o += H;
    for (int l = 0; l < L; l++) {
        y.W[l] = o;
        o += H * 2 * H;
        y.b[l] = o;
        o += H;
    }
    y.wd = o;
    o += H;
    y.bd = o;
    o += 1;
    y.P = o;
    return y;
}

}  // namespace

struct vmps_gnn {
    Layout lay;
    unsigned long long seed = 0;
    float *w = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;  // FP32 master, Adam, grad
    bf16* w16 = nullptr;                                           // BF16 copy used by kernels
    float* part = nullptr;                                         // weight-gradient partials
    int n_cap = 0;
    float *feat = nullptr, *tgt = nullptr, *y = nullptr;
    double *pprev = nullptr, *x0 = nullptr, *ax = nullptr;  // residual objective
    bf16 *h = nullptr, *mm = nullptr, *z = nullptr;
    float *dh = nullptr, *dh2 = nullptr, *dz = nullptr, *dm = nullptr;
    double* red = nullptr;  // reduction partials (kWgradBlocks x 2)
    float* scal = nullptr;  // [0] pref, [1] count of unknown fluid rows, [2] loss
    float* host = nullptr;  // pinned copy of scal
    long t = 0;             // Adam steps taken
    bool have_feat = false, use = false;
    std::vector<void*> owned, pinned;
};

namespace {

// the PPE's unknowns (fluid and wall particles that are not on the free surface)
__device__ __forceinline__ bool unknown_fluid(int bcon, int ptype) { return bcon == 0; }

// rms of p_prev and the count over the unknown rows: fixed-grid partials
__global__ void k_gnn_pref_part(int n, const double* __restrict__ p, const int* __restrict__ bcon,
                                const int* __restrict__ ptype, double* __restrict__ red)
{
    __shared__ double s0[kThreads], s1[kThreads];
    double a = 0, c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (unknown_fluid(bcon[i], ptype[i])) {
            a += p[i] * p[i];
            c += 1.0;
        }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = c;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s0[threadIdx.x] += s0[threadIdx.x + o];
            s1[threadIdx.x] += s1[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        red[2 * blockIdx.x] = s0[0];
        red[2 * blockIdx.x + 1] = s1[0];
    }
}

__global__ void k_gnn_pref_final(int nparts, const double* __restrict__ red, double floor_p,
                                 float* scal)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0, c = 0;
    for (int b = 0; b < nparts; b++) {
        a += red[2 * b];
        c += red[2 * b + 1];
    }
    double rms = c > 0 ? sqrt(a / c) : 0.0;
    scal[0] = (float)fmax(rms, floor_p);
    scal[1] = (float)c;
}

// inputs: PND deviation (x20), p_prev / pref, fluid, Dirichlet, wall, dummy
__global__ void k_gnn_feat(int n, const double* __restrict__ nstar, double n0,
                           const double* __restrict__ p, const int* __restrict__ bcon,
                           const int* __restrict__ ptype, const float* __restrict__ scal,
                           float* __restrict__ feat, double* __restrict__ pprev)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double pref = scal[0];
    pprev[i] = p[i];
    const int pt = ptype[i], bc = bcon[i];
    float* f = feat + (size_t)i * F;
    f[0] = (float)((nstar[i] - n0) / n0 * 20.0);
    f[1] = (float)(p[i] / pref);
    f[2] = pt > 0 ? 1.f : 0.f;
    f[3] = bc == 1 ? 1.f : 0.f;
    f[4] = pt == 0 ? 1.f : 0.f;
    f[5] = pt < 0 ? 1.f : 0.f;
    f[6] = 0.f;
    f[7] = 0.f;
}

// h0 = relu(We f + be); warp per node, lane owns channels 2l, 2l+1
__global__ void k_gnn_enc(int n, const float* __restrict__ feat, const bf16* __restrict__ w16,
                          Layout Y, bf16* __restrict__ h0, bf16* __restrict__ z0)
{
    Grp<32> q;
    const int i = (int)q.gid;
    if (i >= n) return;
    const int c0 = 2 * q.lane, c1 = c0 + 1;
    float a0 = __bfloat162float(w16[Y.be + c0]), a1 = __bfloat162float(w16[Y.be + c1]);
    const float* f = feat + (size_t)i * F;
    for (int k = 0; k < F; k++) {
        const float fk = f[k];
        a0 = a0 + __bfloat162float(w16[Y.We + c0 * F + k]) * fk;
        a1 = a1 + __bfloat162float(w16[Y.We + c1 * F + k]) * fk;
    }
    const size_t o = (size_t)i * H + c0;
    *(bf162*)(z0 + o) = __floats2bfloat162_rn(a0, a1);
    *(bf162*)(h0 + o) = __floats2bfloat162_rn(fmaxf(a0, 0.f), fmaxf(a1, 0.f));
}

// m_i = (sum over the list of i of h_j) / len_i, list order, FP32 sums.  A
// warp per node, two channels per lane: the row's entries are loaded once
// (a lane per entry) and handed out by shuffles, and four neighbours' rows
// are gathered before they are added, so four gathers are in flight.
__global__ void k_gnn_agg(int n, int cap, const int* __restrict__ nbr, const int* __restrict__ len,
                          const bf16* __restrict__ hin, bf16* __restrict__ mout)
{
    Grp<32> q;
    const int i = (int)q.gid;
    if (i >= n) return;
    const int L = len[i];
    const int* row = nbr + (size_t)i * cap;
    float s0 = 0.f, s1 = 0.f;
    for (int b = 0; b < L; b += 32) {
        const int mine = b + q.lane < L ? row[b + q.lane] : 0;
        const int cnt = min(32, L - b);
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
            float2 v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = __shfl_sync(0xffffffffu, mine, k + u);
                v[u] = __bfloat1622float2(*(const bf162*)(hin + (size_t)j * H + 2 * q.lane));
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                s0 = s0 + v[u].x;
                s1 = s1 + v[u].y;
            }
        }
        for (; k < cnt; k++) {
            const int j = __shfl_sync(0xffffffffu, mine, k);
            const float2 v = __bfloat1622float2(*(const bf162*)(hin + (size_t)j * H + 2 * q.lane));
            s0 = s0 + v.x;
            s1 = s1 + v.y;
        }
    }
    if (L > 0) {
        s0 = s0 / (float)L;
        s1 = s1 / (float)L;
    }
    *(bf162*)(mout + (size_t)i * H + 2 * q.lane) = __floats2bfloat162_rn(s0, s1);
}

// ---- the layer on the tensor cores ---------------------------------------
// h_out = h_in + relu(W [h_in, m] + b), z_out = W [h_in, m] + b for 128 nodes
// at a time: the node tile [h, m] (128 x 128 BF16) and W (64 x 128 BF16) sit
// in shared memory, one thread issues a chain of eight tcgen05.mma (K = 16
// each) into a 128 x 64 FP32 accumulator in tensor memory (node r in TMEM
// lane r), and four warps -- one per 32 lanes -- read it back for the bias,
// ReLU and residual epilogue.  Blocks loop over the node tiles.
constexpr int kTcM = 128;          // nodes per tile, the MMA's M
constexpr int kTcK = 2 * H;        // the inputs [h, m]
constexpr int kTcThreads = 128;    // four warps
constexpr uint32_t kTcCols = 64;   // TMEM columns of the accumulator (N = H)
constexpr unsigned kTcWaitLimit = 1u << 22;  // mbarrier polls before giving up

struct TcSmem {
    unsigned char a[kTcM * kTcK * 2];  // node tile, core-matrix layout (32 KB)
    unsigned char w[H * kTcK * 2];     // W, core-matrix layout (16 KB)
    float bias[H];
    unsigned long long bar;            // MMA completion
    uint32_t tmem;                     // accumulator address from tcgen05.alloc
};
constexpr size_t kTcSmemBytes = sizeof(TcSmem) + 128;

// Byte offset of element (r, k) of an R-row, K-major BF16 operand in the
// no-swizzle layout of tcgen05: core matrices of 8 rows x 16 bytes (8 K
// values) are 128 contiguous bytes; the R/8 core matrices of one 8-wide K
// chunk follow one another, then the next K chunk.  Core matrices adjacent
// in K are R*16 bytes apart (the descriptor's leading byte offset), adjacent
// in rows 128 bytes apart (its stride byte offset).
__device__ __forceinline__ uint32_t core_offset(int r, int k, int R)
{
    return (uint32_t)(((((k >> 3) * (R >> 3)) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// tcgen05 shared-memory matrix descriptor: start address, leading and stride
// byte offsets (each in 16-byte units), descriptor version 1 (bits 46-47),
// base offset 0, no swizzling
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D in FP32 (bits 4-5 = 1), A and B in
// BF16 (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at
// bit 24
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(H >> 3) << 17) |
                              ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// bounded wait for the given phase parity of an mbarrier
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (unsigned it = 0; it < kTcWaitLimit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kTcThreads) k_gnn_layer_tc(
    int n, const bf16* __restrict__ w16, int offW, int offb, const bf16* __restrict__ hin,
    const bf16* __restrict__ min_, bf16* __restrict__ hout, bf16* __restrict__ zout,
    unsigned int* err)
{
    extern __shared__ unsigned char tc_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 127) &
                                           ~(uintptr_t)127);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t a_addr = smem_addr(S.a), w_addr = smem_addr(S.w), bar = smem_addr(&S.bar);
    // W[c][k] (row-major, K fastest) into the core-matrix layout, 16 bytes at a time
    for (int e = tid; e < H * (kTcK / 8); e += kTcThreads) {
        const int c = e / (kTcK / 8), k8 = e % (kTcK / 8);
        const uint4 v = *reinterpret_cast<const uint4*>(w16 + offW + c * kTcK + k8 * 8);
        *reinterpret_cast<uint4*>(S.w + core_offset(c, k8 * 8, H)) = v;
    }
    for (int c = tid; c < H; c += kTcThreads) S.bias[c] = __bfloat162float(w16[offb + c]);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&S.tmem)),
                     "r"(kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = S.tmem;
    const int tiles = (n + kTcM - 1) / kTcM;
    uint32_t parity = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int node0 = t * kTcM;
        // [h, m] of the tile's nodes; rows past n are zero
        for (int e = tid; e < kTcM * (kTcK / 8); e += kTcThreads) {
            const int k8 = e / kTcM, r = e % kTcM, node = node0 + r;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (node < n)
                v = *reinterpret_cast<const uint4*>(k8 < H / 8 ? hin + (size_t)node * H + k8 * 8
                                                             : min_ + (size_t)node * H + (k8 - H / 8) * 8);
            *reinterpret_cast<uint4*>(S.a + core_offset(r, k8 * 8, kTcM)) = v;
        }
        // the tile's shared-memory writes become visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < kTcK / 16; s++) {
                const uint64_t ad = umma_desc(a_addr + s * 2 * (kTcM * 16), kTcM * 16, 128);
                const uint64_t bd = umma_desc(w_addr + s * 2 * (H * 16), H * 16, 128);
                const uint32_t acc = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                    :
                    : "r"(tmem), "l"(ad), "l"(bd), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u),
                      "r"(0u), "r"(0u));
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    bar));
        }
        failed = !mbar_wait(bar, parity);
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        // epilogue: node r of the tile is TMEM lane r, warp w reads lanes 32w..32w+31
        const int r = warp * 32 + lane, node = node0 + r;
#pragma unroll
        for (int cb = 0; cb < H; cb += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                  "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                  "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (node < n) {
                __align__(16) bf16 zo[16], ho[16];
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int c = cb + j;
                    const float zv = __uint_as_float(v[j]) + S.bias[c];
                    const float hv = __bfloat162float(
                        *reinterpret_cast<const bf16*>(S.a + core_offset(r, c, kTcM)));
                    zo[j] = __float2bfloat16_rn(zv);
                    ho[j] = __float2bfloat16_rn(hv + fmaxf(zv, 0.f));
                }
                const size_t o = (size_t)node * H + cb;
                if (zout) {
                    *reinterpret_cast<uint4*>(zout + o) = *reinterpret_cast<const uint4*>(zo);
                    *reinterpret_cast<uint4*>(zout + o + 8) = *reinterpret_cast<const uint4*>(zo + 8);
                }
                *reinterpret_cast<uint4*>(hout + o) = *reinterpret_cast<const uint4*>(ho);
                *reinterpret_cast<uint4*>(hout + o + 8) = *reinterpret_cast<const uint4*>(ho + 8);
            }
        }
        // the tile's shared memory and accumulator are free again
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
    }
    if (failed) {
        // an MMA that never signalled: flag it, give it one more bounded wait
        // before its accumulator is released
        if (tid == 0) atomicOr(err, (unsigned)MPS_ERR_CUDA);
        mbar_wait(bar, parity ^ 1u);
    }
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTcCols));
}

// ---- the backward products on the tensor cores (TF32) -------------------
// The gradients are FP32, so both backward products run tcgen05.mma of
// kind::tf32 (FP32 operands rounded to TF32's 10-bit mantissa, FP32
// accumulation): du = W^T dz per node tile (k_gnn_layer_b_tc) and the
// weight gradient sum over nodes of dz u^T per block of nodes
// (k_gnn_wgrad_tc).  Operands use the same no-swizzle K-major layout as the
// forward with 4-byte elements: a core matrix is 8 rows x 4 values.
__device__ __forceinline__ uint32_t core_offset32(int r, int k, int R)
{
    return (uint32_t)(((((k >> 2) * (R >> 3)) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 3) << 2));
}

// kind::tf32 instruction descriptor: D FP32, A and B TF32 (format 2), K-major
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                         uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot_addr, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_addr),
                 "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        bar));
}

constexpr uint32_t kTbCols = 2 * H;  // du: 128 FP32 columns
struct TbSmem {
    float a[kTcM * H];       // dz of the node tile (M = 128 nodes, K = 64)
    float b[2 * H * H];      // W^T (N = 128 inputs, K = 64 outputs)
    unsigned long long bar;
    uint32_t tmem;
};
constexpr size_t kTbSmemBytes = sizeof(TbSmem) + 128;

// Backward through h_out = h_in + relu(z), z = W [h_in, m] + b, for 128
// nodes at a time: dz = dh_out * [z > 0] (also written out for the weight
// gradient), du = W^T dz on the tensor cores, dself = dh_out + du[0, H),
// dm = du[H, 2H).
__global__ void __launch_bounds__(kTcThreads) k_gnn_layer_b_tc(
    int n, const bf16* __restrict__ w16, int offW, const bf16* __restrict__ z,
    const float* __restrict__ dhout, float* __restrict__ dz, float* __restrict__ dself,
    float* __restrict__ dm, unsigned int* err)
{
    extern __shared__ unsigned char tc_raw[];
    TbSmem& S = *reinterpret_cast<TbSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 127) &
                                           ~(uintptr_t)127);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t a_addr = smem_addr(S.a), b_addr = smem_addr(S.b), bar = smem_addr(&S.bar);
    // B: row k (input), column c (output) = W[c][k]
    for (int e = tid; e < 2 * H * H; e += kTcThreads) {
        const int c = e / (2 * H), k = e % (2 * H);
        *reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(S.b) + core_offset32(k, c, 2 * H)) =
            __bfloat162float(w16[offW + e]);
    }
    if (warp == 0) tmem_alloc(smem_addr(&S.tmem), kTbCols);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = S.tmem;
    const int tiles = (n + kTcM - 1) / kTcM;
    uint32_t parity = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int node0 = t * kTcM;
        // dz of the tile, four outputs at a time; rows past n are zero
        for (int e = tid; e < kTcM * (H / 4); e += kTcThreads) {
            const int c4 = e / kTcM, r = e % kTcM, node = node0 + r;
            float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
            if (node < n) {
                const size_t o = (size_t)node * H + 4 * c4;
                const float4 g = *reinterpret_cast<const float4*>(dhout + o);
                const float2 z01 = __bfloat1622float2(*reinterpret_cast<const bf162*>(z + o));
                const float2 z23 = __bfloat1622float2(*reinterpret_cast<const bf162*>(z + o + 2));
                d = make_float4(z01.x > 0.f ? g.x : 0.f, z01.y > 0.f ? g.y : 0.f,
                                z23.x > 0.f ? g.z : 0.f, z23.y > 0.f ? g.w : 0.f);
                *reinterpret_cast<float4*>(dz + o) = d;
            }
            *reinterpret_cast<float4*>(reinterpret_cast<unsigned char*>(S.a) +
                                       core_offset32(r, 4 * c4, kTcM)) = d;
        }
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < H / 8; s++)
                mma_tf32(tmem, umma_desc(a_addr + s * 2 * (kTcM * 16), kTcM * 16, 128),
                         umma_desc(b_addr + s * 2 * (2 * H * 16), 2 * H * 16, 128),
                         tf32_idesc(kTcM, 2 * H), s > 0 ? 1u : 0u);
            umma_commit(bar);
        }
        failed = !mbar_wait(bar, parity);
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        const int r = warp * 32 + lane, node = node0 + r;
#pragma unroll
        for (int kb = 0; kb < 2 * H; kb += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)kb, v);
            if (node < n) {
#pragma unroll
                for (int j = 0; j < 16; j += 4) {
                    const int k = kb + j;
                    const float4 du = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                  __uint_as_float(v[j + 2]),
                                                  __uint_as_float(v[j + 3]));
                    if (k < H) {
                        const size_t o = (size_t)node * H + k;
                        const float4 g = *reinterpret_cast<const float4*>(dhout + o);
                        *reinterpret_cast<float4*>(dself + o) =
                            make_float4(g.x + du.x, g.y + du.y, g.z + du.z, g.w + du.w);
                    } else {
                        *reinterpret_cast<float4*>(dm + (size_t)node * H + (k - H)) = du;
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
    }
    if (failed) {
        if (tid == 0) atomicOr(err, (unsigned)MPS_ERR_CUDA);
        mbar_wait(bar, parity ^ 1u);
    }
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kTbCols);
}

// Weight gradient of a layer (C = H outputs, K = 2H inputs [h, m]) over the
// block's fixed range of nodes, 32 nodes per MMA chunk: D[k][c] = sum over
// nodes of u[k] dz[c] in a 128 x 64 FP32 accumulator (M = the inputs, N =
// the outputs, K = the nodes; both operands transposed into K-major tiles as
// they are staged).  gb[c] = sum over nodes of dz[c] in FP32, fixed order.
// Writes the block's partial in the parameters' layout (W row-major, then
// b) for k_gnn_reduce.
constexpr int kWgChunk = 32;  // nodes per MMA chunk (four K = 8 steps)
struct WgSmem {
    float a[2 * H * kWgChunk];  // u^T: M = 128 inputs, K = 32 nodes
    float b[H * kWgChunk];      // dz^T: N = 64 outputs, K = 32 nodes
    float bsum[kTcThreads][4];  // per-thread bias partials
    unsigned long long bar;
    uint32_t tmem;
};
constexpr size_t kWgSmemBytes = sizeof(WgSmem) + 128;

__global__ void __launch_bounds__(kTcThreads) k_gnn_wgrad_tc(
    int n, const float* __restrict__ dz, const bf16* __restrict__ u0, const bf16* __restrict__ u1,
    float* __restrict__ part, unsigned int* err)
{
    extern __shared__ unsigned char tc_raw[];
    WgSmem& S = *reinterpret_cast<WgSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 127) &
                                           ~(uintptr_t)127);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int C = H, K = 2 * H, E = C * K + C;
    const uint32_t a_addr = smem_addr(S.a), b_addr = smem_addr(S.b), bar = smem_addr(&S.bar);
    const int per = ((n + gridDim.x - 1) / gridDim.x + kWgChunk - 1) / kWgChunk * kWgChunk;
    const int i0 = min(n, blockIdx.x * per), i1 = min(n, i0 + per);
    if (warp == 0) tmem_alloc(smem_addr(&S.tmem), (uint32_t)H);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = S.tmem;
    // bias partials: thread t sums outputs 4 (t % 16) .. +3 over the nodes
    // t / 16, t / 16 + 8, ... of every chunk, in chunk order
    float bs[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t parity = 0;
    bool failed = false, any = false;
    for (int c0 = i0; c0 < i1; c0 += kWgChunk) {
        // u^T: 8 inputs of one node per item (BF16 -> FP32)
        for (int e = tid; e < kWgChunk * (K / 8); e += kTcThreads) {
            const int a = e % kWgChunk, k8 = e / kWgChunk, node = c0 + a;
            float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (node < i1) {
                const bf16* src = k8 < H / 8 ? u0 + (size_t)node * H + 8 * k8
                                             : u1 + (size_t)node * H + 8 * (k8 - H / 8);
                const uint4 raw = *reinterpret_cast<const uint4*>(src);
                const bf162* h2 = reinterpret_cast<const bf162*>(&raw);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 f = __bfloat1622float2(h2[q]);
                    v[2 * q] = f.x;
                    v[2 * q + 1] = f.y;
                }
            }
#pragma unroll
            for (int q = 0; q < 8; q++)
                *reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(S.a) +
                                          core_offset32(8 * k8 + q, a, K)) = v[q];
        }
        // dz^T: 4 outputs of one node per item
        for (int e = tid; e < kWgChunk * (C / 4); e += kTcThreads) {
            const int c4 = e % (C / 4), a = e / (C / 4), node = c0 + a;
            float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
            if (node < i1) d = *reinterpret_cast<const float4*>(dz + (size_t)node * C + 4 * c4);
            const float dv[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
            for (int q = 0; q < 4; q++) {
                *reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(S.b) +
                                          core_offset32(4 * c4 + q, a, C)) = dv[q];
                bs[q] += dv[q];
            }
        }
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < kWgChunk / 8; s++)
                mma_tf32(tmem, umma_desc(a_addr + s * 2 * (K * 16), K * 16, 128),
                         umma_desc(b_addr + s * 2 * (C * 16), C * 16, 128), tf32_idesc(K, C),
                         (any || s > 0) ? 1u : 0u);
            umma_commit(bar);
        }
        any = true;
        failed = !mbar_wait(bar, parity);
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        // the chunk's tiles are free again for the next chunk
    }
    // bias: the 8 threads of each output group in thread order
#pragma unroll
    for (int q = 0; q < 4; q++) S.bsum[tid][q] = bs[q];
    __syncthreads();
    float* out = part + (size_t)blockIdx.x * E;
    if (tid < C / 4) {
        float g[4] = {0.f, 0.f, 0.f, 0.f};
        for (int t = tid; t < kTcThreads; t += C / 4)
            for (int q = 0; q < 4; q++) g[q] += S.bsum[t][q];
        for (int q = 0; q < 4; q++) out[C * K + 4 * tid + q] = g[q];
    }
    // W: input k = TMEM lane k, output c = column c
    if (!failed) {
        const int k = warp * 32 + lane;
#pragma unroll
        for (int cb = 0; cb < C; cb += 16) {
            uint32_t v[16];
            tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
#pragma unroll
            for (int j = 0; j < 16; j++) out[(size_t)(cb + j) * K + k] = any ? __uint_as_float(v[j]) : 0.f;
        }
    } else {
        if (tid == 0) atomicOr(err, (unsigned)MPS_ERR_CUDA);
        mbar_wait(bar, parity ^ 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, (uint32_t)H);
}

// y = bd + wd . h_L, sequential over channels; thread per node
__global__ void k_gnn_dec(int n, const bf16* __restrict__ w16, Layout Y, const bf16* __restrict__ hL,
                          float* __restrict__ y)
{
    __shared__ float wd[H + 1];
    for (int c = threadIdx.x; c <= H; c += blockDim.x) wd[c] = __bfloat162float(w16[Y.wd + c]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = wd[H];
    const bf16* hr = hL + (size_t)i * H;
    for (int c = 0; c < H; c++) a = a + wd[c] * __bfloat162float(hr[c]);
    y[i] = a;
}

// the guess: p_prev + pref * y on the unknown fluid rows
__global__ void k_gnn_guess(int n, const float* __restrict__ y, const int* __restrict__ bcon,
                            const int* __restrict__ ptype, const float* __restrict__ scal,
                            double* __restrict__ p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !unknown_fluid(bcon[i], ptype[i])) return;
    p[i] = p[i] + (double)scal[0] * (double)y[i];
}

// target increment after the solve: (p_solved - p_prev) / pref
__global__ void k_gnn_target(int n, const double* __restrict__ psol, const float* __restrict__ feat,
                             const float* __restrict__ scal, float* __restrict__ tgt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    tgt[i] = (float)(psol[i] / (double)scal[0]) - feat[(size_t)i * F + 1];
}

// Objective 0 (increment): loss = mean over the unknown rows of (y - t)^2,
// dy = 2 (y - t) / count.  Loss partials per block.
__global__ void k_gnn_dy_mse(int n, const float* __restrict__ y, const float* __restrict__ tgt,
                             const int* __restrict__ bcon, const int* __restrict__ ptype,
                             const float* __restrict__ scal, float* __restrict__ dy,
                             double* __restrict__ red)
{
    __shared__ double sl[kThreads];
    double loss = 0;
    const float cnt = fmaxf(scal[1], 1.f);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float d = 0.f;
        if (unknown_fluid(bcon[i], ptype[i])) {
            const float e = y[i] - tgt[i];
            d = 2.f * e / cnt;
            loss += (double)e * (double)e / (double)cnt;
        }
        dy[i] = d;
    }
    sl[threadIdx.x] = loss;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sl[threadIdx.x] += sl[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) red[blockIdx.x] = sl[0];
}

__global__ void k_gnn_loss_final(int nparts, const double* __restrict__ red, float* scal)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double a = 0;
    for (int b = 0; b < nparts; b++) a += red[b];
    scal[2] = (float)a;
}

// dh_L = wd dy (decoder backward to the last hidden layer)
__global__ void k_gnn_dh_dec(int n, const bf16* __restrict__ w16, Layout Y,
                             const float* __restrict__ dy, float* __restrict__ dh)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)n * H) return;
    dh[e] = __bfloat162float(w16[Y.wd + (int)(e % H)]) * dy[e / H];
}

// Objective 1 (residual): x0 = p_prev + pref y on the unknown rows
__global__ void k_gnn_x0(int n, const double* __restrict__ pprev, const float* __restrict__ y,
                         const int* __restrict__ bcon, const int* __restrict__ ptype,
                         const float* __restrict__ scal, double* __restrict__ x0)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x0[i] = unknown_fluid(bcon[i], ptype[i]) ? pprev[i] + (double)scal[0] * (double)y[i] : 0.0;
}

// r = b - A x0 on the unknown rows (into ax), partials of r.r and b.b
__global__ void k_gnn_resid(int n, const double* __restrict__ b, const int* __restrict__ bcon,
                            const int* __restrict__ ptype, double* __restrict__ ax,
                            double* __restrict__ red)
{
    __shared__ double s0[kThreads], s1[kThreads];
    double rr = 0, bb = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double r = 0.0;
        if (unknown_fluid(bcon[i], ptype[i])) {
            r = b[i] - ax[i];
            rr += r * r;
            bb += b[i] * b[i];
        }
        ax[i] = r;
    }
    s0[threadIdx.x] = rr;
    s1[threadIdx.x] = bb;
    __syncthreads();
    for (int o = kThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s0[threadIdx.x] += s0[threadIdx.x + o];
            s1[threadIdx.x] += s1[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        red[2 * blockIdx.x] = s0[0];
        red[2 * blockIdx.x + 1] = s1[0];
    }
}

// loss = r.r / b.b -> scal[2], 1 / b.b -> scal[3]
__global__ void k_gnn_resid_final(int nparts, const double* __restrict__ red, float* scal)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double rr = 0, bb = 0;
    for (int k = 0; k < nparts; k++) {
        rr += red[2 * k];
        bb += red[2 * k + 1];
    }
    scal[2] = bb > 0 ? (float)(rr / bb) : 0.f;
    scal[3] = bb > 0 ? (float)(1.0 / bb) : 0.f;
}

// dy = d(r.r / b.b)/dy = -2 pref (A r)_i / b.b on the unknown rows (A = A^T)
__global__ void k_gnn_dy_resid(int n, const double* __restrict__ ar, const int* __restrict__ bcon,
                               const int* __restrict__ ptype, const float* __restrict__ scal,
                               float* __restrict__ dy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dy[i] = unknown_fluid(bcon[i], ptype[i])
                ? (float)(-2.0 * (double)scal[0] * ar[i] * (double)scal[3])
                : 0.f;
}

// transpose of the mean aggregation on a symmetric list:
// dh_prev_j = dself_j + sum over the list of j of dm_i / len_i
__global__ void k_gnn_agg_b(int n, int cap, const int* __restrict__ nbr, const int* __restrict__ len,
                            const float* __restrict__ dself, const float* __restrict__ dm,
                            float* __restrict__ dprev)
{
    Grp<32> q;
    const int j = (int)q.gid;
    if (j >= n) return;
    const int L = len[j];
    const int* row = nbr + (size_t)j * cap;
    const size_t o = (size_t)j * H + 2 * q.lane;
    float s0 = 0.f, s1 = 0.f;
    // the row handed out by shuffles, four neighbours' gathers in flight,
    // added in list order
    for (int b = 0; b < L; b += 32) {
        const int mine = b + q.lane < L ? row[b + q.lane] : 0;
        const float lmine = b + q.lane < L ? (float)max(len[mine], 1) : 1.f;
        const int cnt = min(32, L - b);
        int k = 0;
        for (; k + 4 <= cnt; k += 4) {
            float2 v[4];
            float li[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int i = __shfl_sync(0xffffffffu, mine, k + u);
                li[u] = __shfl_sync(0xffffffffu, lmine, k + u);
                v[u] = *(const float2*)(dm + (size_t)i * H + 2 * q.lane);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                s0 = s0 + v[u].x / li[u];
                s1 = s1 + v[u].y / li[u];
            }
        }
        for (; k < cnt; k++) {
            const int i = __shfl_sync(0xffffffffu, mine, k);
            const float li = __shfl_sync(0xffffffffu, lmine, k);
            const float2 v = *(const float2*)(dm + (size_t)i * H + 2 * q.lane);
            s0 = s0 + v.x / li;
            s1 = s1 + v.y / li;
        }
    }
    const float2 g = *(const float2*)(dself + o);
    *(float2*)(dprev + o) = make_float2(g.x + s0, g.y + s1);
}

// encoder backward: dz0 = dh0 * [z0 > 0], in place
__global__ void k_gnn_relu_b(long count, const bf16* __restrict__ z, float* __restrict__ d)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    if (!(__bfloat162float(z[e]) > 0.f)) d[e] = 0.f;
}

// Weight gradients of one affine map with C outputs and K inputs:
// gW[c][k] = sum_i dz_i[c] u_i[k], gb[c] = sum_i dz_i[c], entries laid out
// as the parameters (W row-major, then b).  u is [u0 | u1] (BF16, H each)
// or uf (FP32, K wide).  Block b reduces a fixed chunk of nodes.
__global__ void __launch_bounds__(kThreads) k_gnn_wgrad(int n, int C, int K, const float* __restrict__ dz,
                                                        int dz_stride, const bf16* __restrict__ u0,
                                                        const bf16* __restrict__ u1,
                                                        const float* __restrict__ uf,
                                                        float* __restrict__ part)
{
    __shared__ float ds[kTile][H];
    __shared__ float us[kTile][2 * H];
    const int E = C * K + C;
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int i0 = blockIdx.x * chunk, i1 = min(n, i0 + chunk);
    float acc[kPerThread];
#pragma unroll
    for (int r = 0; r < kPerThread; r++) acc[r] = 0.f;
    for (int t0 = i0; t0 < i1; t0 += kTile) {
        const int nt = min(kTile, i1 - t0);
        __syncthreads();
        for (int e = threadIdx.x; e < nt * C; e += blockDim.x) {
            const int a = e / C, c = e % C;
            ds[a][c] = dz[(size_t)(t0 + a) * dz_stride + c];
        }
        for (int e = threadIdx.x; e < nt * K; e += blockDim.x) {
            const int a = e / K, k = e % K;
            float val;
            if (uf) val = uf[(size_t)(t0 + a) * K + k];
            else if (k < H) val = __bfloat162float(u0[(size_t)(t0 + a) * H + k]);
            else val = __bfloat162float(u1[(size_t)(t0 + a) * H + (k - H)]);
            us[a][k] = val;
        }
        __syncthreads();
        for (int a = 0; a < nt; a++) {
#pragma unroll
            for (int r = 0; r < kPerThread; r++) {
                const int e = threadIdx.x + r * kThreads;
                if (e < C * K) acc[r] = acc[r] + ds[a][e / K] * us[a][e % K];
                else if (e < E) acc[r] = acc[r] + ds[a][e - C * K];
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kPerThread; r++) {
        const int e = threadIdx.x + r * kThreads;
        if (e < E) part[(size_t)blockIdx.x * E + e] = acc[r];
    }
}

// g[off + e] = sum over blocks of part[b][e], fixed order
__global__ void k_gnn_reduce(int nparts, int E, const float* __restrict__ part, float* __restrict__ g)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    float a = 0.f;
    for (int b = 0; b < nparts; b++) a = a + part[(size_t)b * E + e];
    g[e] = a;
}

// Adam (Kingma & Ba 2015) with bias correction; refreshes the BF16 copy
__global__ void k_gnn_adam(int P, float* __restrict__ w, const float* __restrict__ g,
                           float* __restrict__ m, float* __restrict__ v, bf16* __restrict__ w16,
                           float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float wk = w[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    w[k] = wk;
    w16[k] = __float2bfloat16_rn(wk);
}

__global__ void k_gnn_to16(int P, const float* __restrict__ w, bf16* __restrict__ w16)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < P) w16[k] = __float2bfloat16_rn(w[k]);
}

// ------------------------------------------------------------------ host

template <typename T>
int galloc(mps_ctx* c, vmps_gnn* G, T** p, size_t count)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, (count > 0 ? count : 1) * sizeof(T));
    if (e != cudaSuccess) return vmps_check(c, e, "cudaMalloc (network)");
    e = cudaMemsetAsync(q, 0, (count > 0 ? count : 1) * sizeof(T), c->stream);
    if (e != cudaSuccess) return vmps_check(c, e, "cudaMemsetAsync (network)");
    G->owned.push_back(q);
    *p = (T*)q;
    return MPS_OK;
}

#define GTRY(x)                        \
    do {                               \
        int _r = (x);                  \
        if (_r != MPS_OK) return _r;   \
    } while (0)

void free_acts(vmps_gnn* G)
{
    // activation buffers are the owned entries after the first eight
    // (w, m, v, g, w16, part, red, scal) -- see vmps_gnn_create
    while (G->owned.size() > 8) {
        cudaFree(G->owned.back());
        G->owned.pop_back();
    }
    G->feat = G->tgt = G->y = nullptr;
    G->h = G->mm = G->z = nullptr;
    G->dh = G->dh2 = G->dz = G->dm = nullptr;
    G->pprev = G->x0 = G->ax = nullptr;
    G->n_cap = 0;
}

int ensure_acts(mps_ctx* c, vmps_gnn* G)
{
    const int n = c->n;
    if (G->n_cap >= n) return MPS_OK;
    free_acts(G);
    const size_t N = (size_t)n, L = (size_t)G->lay.L;
    GTRY(galloc(c, G, &G->feat, N * F));
    GTRY(galloc(c, G, &G->tgt, N));
    GTRY(galloc(c, G, &G->y, N));
    GTRY(galloc(c, G, &G->h, (L + 1) * N * H));
    GTRY(galloc(c, G, &G->mm, L * N * H));
    GTRY(galloc(c, G, &G->z, (L + 1) * N * H));
    GTRY(galloc(c, G, &G->dh, N * H));
    GTRY(galloc(c, G, &G->dh2, N * H));
    GTRY(galloc(c, G, &G->dz, N * H));
    GTRY(galloc(c, G, &G->dm, N * H));
    GTRY(galloc(c, G, &G->pprev, N));
    GTRY(galloc(c, G, &G->x0, N));
    GTRY(galloc(c, G, &G->ax, N));
    G->n_cap = n;
    G->have_feat = false;
    return MPS_OK;
}

inline int warp_blocks(int n) { return (int)(((long)n * 32 + kThreads - 1) / kThreads); }

// inputs at the current state: pref, features (needs bcon, n* and p_prev)
int features(mps_ctx* c, vmps_gnn* G)
{
    const int n = c->n;
    cudaStream_t st = c->stream;
    const mps_config& f = c->cfg;
    const double floor_p =
        f.rho1 * sqrt(f.gx * f.gx + f.gy * f.gy + f.gz * f.gz) * f.l0 + 1e-30;
    k_gnn_pref_part<<<kWgradBlocks, kThreads, 0, st>>>(n, c->pnew, c->bcon, c->ptype, G->red);
    k_gnn_pref_final<<<1, 32, 0, st>>>(kWgradBlocks, G->red, floor_p, G->scal);
    k_gnn_feat<<<grid_blocks(n), kThreads, 0, st>>>(n, c->nds, c->n0_s, c->pnew, c->bcon, c->ptype,
                                                    G->scal, G->feat, G->pprev);
    vmps_count_launch(3);
    G->have_feat = true;
    return MPS_OK;
}

// the tensor-core layer needs more than the default 48 KB of dynamic shared
// memory; set once per device, outside any stream capture
int tc_prepare(mps_ctx* c)
{
    static bool done[64] = {};
    if (c->device >= 0 && c->device < 64 && done[c->device]) return MPS_OK;
    VMPS_CUDA(c, cudaFuncSetAttribute(k_gnn_layer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemBytes));
    VMPS_CUDA(c, cudaFuncSetAttribute(k_gnn_layer_b_tc,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTbSmemBytes));
    VMPS_CUDA(c, cudaFuncSetAttribute(k_gnn_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kWgSmemBytes));
    if (c->device >= 0 && c->device < 64) done[c->device] = true;
    return MPS_OK;
}

int forward(mps_ctx* c, vmps_gnn* G)
{
    const int n = c->n;
    const size_t NH = (size_t)n * H;
    const Layout& Y = G->lay;
    cudaStream_t st = c->stream;
    k_gnn_enc<<<warp_blocks(n), kThreads, 0, st>>>(n, G->feat, G->w16, Y, G->h, G->z);
    vmps_count_launch(1);
    int sms = 0;
    VMPS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    // node tiles of the tensor-core layer: up to three resident blocks per SM
    const int tc_blocks = std::max(1, std::min((n + kTcM - 1) / kTcM, sms * 3));
    for (int l = 0; l < Y.L; l++) {
        k_gnn_agg<<<warp_blocks(n), kThreads, 0, st>>>(n, c->cap_s, c->nbr_s, c->len_s,
                                                       G->h + l * NH, G->mm + l * NH);
        k_gnn_layer_tc<<<tc_blocks, kTcThreads, kTcSmemBytes, st>>>(
            n, G->w16, Y.W[l], Y.b[l], G->h + l * NH, G->mm + l * NH, G->h + (l + 1) * NH,
            G->z + (l + 1) * NH, c->d_err);
        vmps_count_launch(2);
    }
    k_gnn_dec<<<grid_blocks(n), kThreads, 0, st>>>(n, G->w16, Y, G->h + Y.L * NH, G->y);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int wgrad(mps_ctx* c, vmps_gnn* G, int C, int K, const float* dz, int dz_stride, const bf16* u0,
          const bf16* u1, const float* uf, int off)
{
    cudaStream_t st = c->stream;
    const int E = C * K + C;
    k_gnn_wgrad<<<kWgradBlocks, kThreads, 0, st>>>(c->n, C, K, dz, dz_stride, u0, u1, uf, G->part);
    k_gnn_reduce<<<(E + kThreads - 1) / kThreads, kThreads, 0, st>>>(kWgradBlocks, E, G->part,
                                                                    G->g + off);
    vmps_count_launch(2);
    return MPS_OK;
}

// gradient of the loss at the captured features (into G->g).  objective 0:
// squared error of the increment against the solved one; objective 1: the
// relative squared residual |b - A x0|^2 / |b|^2 the guess leaves in the
// last PPE's system (what CG has to remove).
int backward(mps_ctx* c, vmps_gnn* G, int objective)
{
    const int n = c->n;
    const size_t NH = (size_t)n * H;
    const Layout& Y = G->lay;
    cudaStream_t st = c->stream;
    if (objective == 0) {
        k_gnn_dy_mse<<<kWgradBlocks, kThreads, 0, st>>>(n, G->y, G->tgt, c->bcon, c->ptype, G->scal,
                                                        G->dz, G->red);
        k_gnn_loss_final<<<1, 32, 0, st>>>(kWgradBlocks, G->red, G->scal);
        vmps_count_launch(2);
    } else {
        k_gnn_x0<<<grid_blocks(n), kThreads, 0, st>>>(n, G->pprev, G->y, c->bcon, c->ptype, G->scal,
                                                      G->x0);
        vmps_count_launch(1);
        GTRY(vmps_ppe_apply(c, G->x0, G->ax));
        k_gnn_resid<<<kWgradBlocks, kThreads, 0, st>>>(n, c->source, c->bcon, c->ptype, G->ax,
                                                        G->red);
        k_gnn_resid_final<<<1, 32, 0, st>>>(kWgradBlocks, G->red, G->scal);
        vmps_count_launch(2);
        GTRY(vmps_ppe_apply(c, G->ax, G->x0));  // A r (x0 is free again)
        k_gnn_dy_resid<<<grid_blocks(n), kThreads, 0, st>>>(n, G->x0, c->bcon, c->ptype, G->scal,
                                                            G->dz);
        vmps_count_launch(1);
    }
    k_gnn_dh_dec<<<(int)((NH + kThreads - 1) / kThreads), kThreads, 0, st>>>(n, G->w16, Y, G->dz,
                                                                            G->dh);
    vmps_count_launch(1);
    // decoder: dz holds dy (stride 1), inputs h_L
    GTRY(wgrad(c, G, 1, H, G->dz, 1, G->h + Y.L * NH, nullptr, nullptr, Y.wd));
    int sms = 0;
    VMPS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    const int tc_blocks = std::max(1, std::min((n + kTcM - 1) / kTcM, sms * 3));
    float* d_out = G->dh;   // gradient w.r.t. h_l
    float* d_self = G->dh2;
    for (int l = Y.L - 1; l >= 0; l--) {
        k_gnn_layer_b_tc<<<tc_blocks, kTcThreads, kTbSmemBytes, st>>>(
            n, G->w16, Y.W[l], G->z + (l + 1) * NH, d_out, G->dz, d_self, G->dm, c->d_err);
        k_gnn_wgrad_tc<<<kWgradBlocks, kTcThreads, kWgSmemBytes, st>>>(
            n, G->dz, G->h + l * NH, G->mm + l * NH, G->part, c->d_err);
        k_gnn_reduce<<<(2 * H * H + H + kThreads - 1) / kThreads, kThreads, 0, st>>>(
            kWgradBlocks, 2 * H * H + H, G->part, G->g + Y.W[l]);
        vmps_count_launch(3);
        // d_out <- dself + transpose-aggregated dm (gradient w.r.t. h_(l-1))
        k_gnn_agg_b<<<warp_blocks(n), kThreads, 0, st>>>(n, c->cap_s, c->nbr_s, c->len_s, d_self,
                                                         G->dm, d_out);
        vmps_count_launch(1);
    }
    // encoder
    k_gnn_relu_b<<<(int)((NH + kThreads - 1) / kThreads), kThreads, 0, st>>>((long)NH, G->z, d_out);
    vmps_count_launch(1);
    GTRY(wgrad(c, G, H, F, d_out, H, nullptr, nullptr, G->feat, Y.We));
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

// SplitMix64 stream -> uniform in [-a, a) (weights' initial values)
__host__ float uniform_pm(unsigned long long& s, float a)
{
    s += 0x9E3779B97F4A7C15ull;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)(((double)(z >> 11) / 9007199254740992.0) * 2.0 - 1.0) * a;
}

}  // namespace

// ------------------------------------------------------------------ internal API

void vmps_gnn_free(mps_ctx* c)
{
    if (!c->gnn) return;
    vmps_gnn* G = c->gnn;
    for (void* q : G->owned) cudaFree(q);
    for (void* q : G->pinned) cudaFreeHost(q);
    delete G;
    c->gnn = nullptr;
}

// before the PPE's assembly: the network's guess replaces the previous
// pressure on the unknown fluid rows (features are kept for training)
int vmps_gnn_guess(mps_ctx* c)
{
    vmps_gnn* G = c->gnn;
    if (!G) {
        c->msg = "learned guess requested without a network (mps_gnn_create)";
        return MPS_ERR_ARG;
    }
    GTRY(ensure_acts(c, G));
    GTRY(features(c, G));
    if (!G->use) return MPS_OK;
    GTRY(forward(c, G));
    k_gnn_guess<<<grid_blocks(c->n), kThreads, 0, c->stream>>>(c->n, G->y, c->bcon, c->ptype,
                                                              G->scal, c->pnew);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

bool vmps_gnn_in_use(const mps_ctx* c) { return c->gnn != nullptr && c->gnn->use; }

// device buffers sized by the particle count, outside any stream capture
int vmps_gnn_prepare(mps_ctx* c) { return c->gnn ? ensure_acts(c, c->gnn) : MPS_OK; }

// a new upload invalidates captured features
void vmps_gnn_reset(mps_ctx* c)
{
    if (c->gnn) c->gnn->have_feat = false;
}

// ------------------------------------------------------------------ C-ABI

extern "C" {

int mps_gnn_create(mps_ctx* c, int layers, unsigned long long seed)
{
    if (!c || layers < 1 || layers > kMaxLayers) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    vmps_gnn_free(c);
    vmps_gnn* G = new vmps_gnn();
    c->gnn = G;
    G->lay = make_layout(layers);
    G->seed = seed;
    const int P = G->lay.P;
    // the first eight owned buffers persist across uploads (free_acts)
    GTRY(galloc(c, G, &G->w, P));
    GTRY(galloc(c, G, &G->m, P));
    GTRY(galloc(c, G, &G->v, P));
    GTRY(galloc(c, G, &G->g, P));
    GTRY(galloc(c, G, &G->w16, P));
    GTRY(tc_prepare(c));
    GTRY(galloc(c, G, &G->part, (size_t)kWgradBlocks * kMaxE));
    GTRY(galloc(c, G, &G->red, (size_t)2 * kWgradBlocks));
    GTRY(galloc(c, G, &G->scal, 4));
    float* hp = nullptr;
    if (cudaMallocHost(&hp, 4 * sizeof(float)) != cudaSuccess) return MPS_ERR_CUDA;
    G->pinned.push_back(hp);
    G->host = hp;
    // He-uniform weights (fan-in), zero biases, zero decoder: the untrained
    // network's guess is the previous pressure
    std::vector<float> w(P, 0.f);
    unsigned long long s = seed;
    const Layout& Y = G->lay;
    const float ae = sqrtf(6.f / 6.f), al = sqrtf(6.f / (2.f * H));
    for (int k = 0; k < H * F; k++) w[Y.We + k] = (k % F) < 6 ? uniform_pm(s, ae) : 0.f;
    for (int l = 0; l < Y.L; l++)
        for (int k = 0; k < 2 * H * H; k++) w[Y.W[l] + k] = uniform_pm(s, al) * 0.5f;
    VMPS_CUDA(c, cudaMemcpyAsync(G->w, w.data(), sizeof(float) * P, cudaMemcpyHostToDevice,
                                 c->stream));
    k_gnn_to16<<<(P + kThreads - 1) / kThreads, kThreads, 0, c->stream>>>(P, G->w, G->w16);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

int mps_gnn_use(mps_ctx* c, int on)
{
    if (!c || !c->gnn) return MPS_ERR_ARG;
    c->gnn->use = on != 0;
    vmps_drop_graphs(c);
    return MPS_OK;
}

int mps_gnn_params(mps_ctx* c, float* get, const float* set, int* count)
{
    if (!c || !c->gnn) return MPS_ERR_ARG;
    vmps_gnn* G = c->gnn;
    const int P = G->lay.P;
    if (count) *count = P;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    if (set) {
        VMPS_CUDA(c, cudaMemcpyAsync(G->w, set, sizeof(float) * P, cudaMemcpyHostToDevice,
                                     c->stream));
        k_gnn_to16<<<(P + kThreads - 1) / kThreads, kThreads, 0, c->stream>>>(P, G->w, G->w16);
        vmps_count_launch(1);
        VMPS_CUDA(c, cudaMemsetAsync(G->m, 0, sizeof(float) * P, c->stream));
        VMPS_CUDA(c, cudaMemsetAsync(G->v, 0, sizeof(float) * P, c->stream));
        G->t = 0;
    }
    if (get)
        VMPS_CUDA(c, cudaMemcpyAsync(get, G->w, sizeof(float) * P, cudaMemcpyDeviceToHost,
                                     c->stream));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

// The whole training state: FP32 parameters, Adam's two moments and its step
// count (as a float), 3P + 1 values.  Moving it between contexts trains one
// network on several scenes' PPE snapshots with one Adam trajectory.
int mps_gnn_state(mps_ctx* c, float* get, const float* set, int* count)
{
    if (!c || !c->gnn) return MPS_ERR_ARG;
    vmps_gnn* G = c->gnn;
    const int P = G->lay.P;
    if (count) *count = 3 * P + 1;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    if (set) {
        const double t = set[3 * P];
        if (!(t >= 0.0 && t < 1e15)) {
            c->msg = "network state: bad Adam step count";
            return MPS_ERR_ARG;
        }
        VMPS_CUDA(c, cudaMemcpyAsync(G->w, set, sizeof(float) * P, cudaMemcpyHostToDevice,
                                     c->stream));
        VMPS_CUDA(c, cudaMemcpyAsync(G->m, set + P, sizeof(float) * P, cudaMemcpyHostToDevice,
                                     c->stream));
        VMPS_CUDA(c, cudaMemcpyAsync(G->v, set + 2 * P, sizeof(float) * P,
                                     cudaMemcpyHostToDevice, c->stream));
        k_gnn_to16<<<(P + kThreads - 1) / kThreads, kThreads, 0, c->stream>>>(P, G->w, G->w16);
        vmps_count_launch(1);
        G->t = (long)t;
    }
    if (get) {
        VMPS_CUDA(c, cudaMemcpyAsync(get, G->w, sizeof(float) * P, cudaMemcpyDeviceToHost,
                                     c->stream));
        VMPS_CUDA(c, cudaMemcpyAsync(get + P, G->m, sizeof(float) * P, cudaMemcpyDeviceToHost,
                                     c->stream));
        VMPS_CUDA(c, cudaMemcpyAsync(get + 2 * P, G->v, sizeof(float) * P,
                                     cudaMemcpyDeviceToHost, c->stream));
    }
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    if (get) get[3 * P] = (float)G->t;
    return MPS_OK;
}

// Features of the current state (as the next PPE would see them: call after
// mps_step has produced n* and bcon, i.e. for the step just taken they are
// the ones captured inside it).  Exposed for tests and offline training.
int mps_gnn_features(mps_ctx* c)
{
    if (!c || !c->gnn || !c->initialized) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    GTRY(ensure_acts(c, c->gnn));
    return features(c, c->gnn);
}

// `iters` Adam steps on the features captured by the last PPE and, for
// objective 0, the pressure it solved for (objective 1 needs only its matrix
// and right-hand side); *loss = the loss before the last step's update.
// grad_only != 0 computes the gradient (mps_gnn_download "grad") and takes
// no step.
int mps_gnn_train(mps_ctx* c, int iters, float lr, int objective, int grad_only, float* loss)
{
    if (!c || !c->gnn || iters < 1 || !(lr > 0) || objective < 0 || objective > 1)
        return MPS_ERR_ARG;
    vmps_gnn* G = c->gnn;
    if (!G->have_feat || G->n_cap < c->n) {
        c->msg = "no captured features: take a step with the network attached first";
        return MPS_ERR_ARG;
    }
    VMPS_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const int n = c->n;
    k_gnn_target<<<grid_blocks(n), kThreads, 0, st>>>(n, c->pnew, G->feat, G->scal, G->tgt);
    vmps_count_launch(1);
    const int P = G->lay.P;
    for (int it = 0; it < iters; it++) {
        GTRY(forward(c, G));
        GTRY(backward(c, G, objective));
        if (grad_only) break;
        G->t++;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - powf(b1, (float)G->t), c2 = 1.f - powf(b2, (float)G->t);
        k_gnn_adam<<<(P + kThreads - 1) / kThreads, kThreads, 0, st>>>(P, G->w, G->g, G->m, G->v,
                                                                      G->w16, lr, b1, b2, 1e-8f,
                                                                      c1, c2);
        vmps_count_launch(1);
    }
    VMPS_CUDA(c, cudaMemcpyAsync(G->host, G->scal, 4 * sizeof(float), cudaMemcpyDeviceToHost, st));
    VMPS_CUDA(c, cudaStreamSynchronize(st));
    if (loss) *loss = G->host[2];
    return MPS_OK;
}

// Network data in slot (cell) order: "feat" (n x 8), "target", "y" (n),
// "grad" (P), "pref" (1), "count" (1), "nbr" (n x cap_s ints, row-major),
// "len", "bcon", "ptype" (n ints), "cap" (1 int).
int mps_gnn_download(mps_ctx* c, const char* what, void* out, long* count)
{
    if (!c || !c->gnn || !what) return MPS_ERR_ARG;
    vmps_gnn* G = c->gnn;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    std::string s(what);
    const void* src = nullptr;
    size_t bytes = 0;
    long cnt = 0;
    const long n = c->n;
    if (s == "feat") { src = G->feat; cnt = n * F; bytes = cnt * sizeof(float); }
    else if (s == "target") { src = G->tgt; cnt = n; bytes = cnt * sizeof(float); }
    else if (s == "y") { src = G->y; cnt = n; bytes = cnt * sizeof(float); }
    else if (s == "grad") { src = G->g; cnt = G->lay.P; bytes = cnt * sizeof(float); }
    else if (s == "pref") { src = G->scal; cnt = 1; bytes = sizeof(float); }
    else if (s == "count") { src = G->scal + 1; cnt = 1; bytes = sizeof(float); }
    else if (s == "nbr") { src = c->nbr_s; cnt = n * c->cap_s; bytes = cnt * sizeof(int); }
    else if (s == "len") { src = c->len_s; cnt = n; bytes = cnt * sizeof(int); }
    else if (s == "bcon") { src = c->bcon; cnt = n; bytes = cnt * sizeof(int); }
    else if (s == "ptype") { src = c->ptype; cnt = n; bytes = cnt * sizeof(int); }
    else if (s == "cap") {
        if (count) *count = 1;
        if (out) *(int*)out = c->cap_s;
        return MPS_OK;
    } else return MPS_ERR_ARG;
    if (count) *count = cnt;
    if (!out) return MPS_OK;
    if (!src) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

// forward pass only, on the captured features (fills "y")
int mps_gnn_forward(mps_ctx* c)
{
    if (!c || !c->gnn || !c->gnn->have_feat) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    GTRY(forward(c, c->gnn));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

}  // extern "C"
