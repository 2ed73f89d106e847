// mps_noalloc.cu -- cell numbers and cell order without device allocation.
//
// Some programs cannot let a library call cudaMalloc: for example an
// application whose memory manager has already reserved the whole device
// heap for its own pool, or a time-critical loop whose rules forbid any
// allocation after start-up.  For them mps_cell_order_noalloc() bins
// particles (the first half of NEIGHBOR, functions.cu:2790-2852) using only
// the caller's buffers and the fixed scratch area below.
//
// The scratch area is a file-scope __device__ array.  Every GPU that loads
// this library holds it (kNoAllocScratchBytes, about 4 MiB) until the
// process exits.  Host code cannot use the array's name as a device
// address, so every call made outside a stream capture looks the address up
// with cudaGetSymbolAddress while the device is current (the module can be
// reloaded at a new address after cudaDeviceReset) and keeps it per device;
// a call made during a capture uses the kept address, so make the first call
// on each device before any stream capture.  All calls share the one area
// and it keeps the previous call's contents: the counters are cleared at
// the start of every call, and calls that overlap on the GPU (two streams at
// once) race.
#include <mutex>

#include "mps_internal.cuh"

using namespace vmps;

namespace {

constexpr int kNoAllocMaxParticles = 1 << 18;  // 262,144 particles
constexpr int kNoAllocMaxCells = 1 << 18;      // cell counters (tnc + 2 <= 262,144)
constexpr int kNoAllocScanThreads = 1024;

struct NoAllocScratch {
    int cnt[kNoAllocMaxCells];       // particles per cell
    int cst[kNoAllocMaxCells];       // first sorted slot of each cell
    int bpos[kNoAllocMaxParticles];  // arrival position inside the cell
    int bslot[kNoAllocMaxParticles]; // particle index, bucketed by cell
};
constexpr size_t kNoAllocScratchBytes = sizeof(NoAllocScratch);

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

template <int DIM>
__global__ void k_na_hash(int n, Grid g, const double* __restrict__ x,
                          const double* __restrict__ y, const double* __restrict__ z,
                          int* __restrict__ cell, NoAllocScratch* S, unsigned int* bad)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a, b, c;
    bool ok = cell_coords<DIM>(g, x[i], y[i], DIM == 3 ? z[i] : 0.0, a, b, c);
    if (!ok) atomicOr(bad, 1u);
    int C = a + (b - 1) * g.ncx + (c - 1) * g.ncx * g.ncy;
    cell[i] = C;
    S->bpos[i] = atomicAdd(&S->cnt[C], 1);
}

// exclusive scan of m <= kNoAllocMaxCells counters in one block
__global__ void k_na_scan(int m, NoAllocScratch* S)
{
    __shared__ int sh[kNoAllocScanThreads];
    const int per = (m + kNoAllocScanThreads - 1) / kNoAllocScanThreads;
    const int b = threadIdx.x * per;
    int local = 0;
    for (int k = b; k < b + per && k < m; k++) local += S->cnt[k];
    sh[threadIdx.x] = local;
    __syncthreads();
    for (int o = 1; o < kNoAllocScanThreads; o <<= 1) {
        int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += t;
        __syncthreads();
    }
    int run = sh[threadIdx.x] - local;
    for (int k = b; k < b + per && k < m; k++) {
        S->cst[k] = run;
        run += S->cnt[k];
    }
}

__global__ void k_na_scatter(int n, const int* __restrict__ cell, NoAllocScratch* S)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    S->bslot[S->cst[cell[i]] + S->bpos[i]] = i;
}

// inside a cell the order is ascending particle index (the reference's
// stable insertion, functions.cu:2820-2852)
__global__ void k_na_rank(int n, const int* __restrict__ cell, const NoAllocScratch* S,
                          int* __restrict__ perm)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int me = S->bslot[q];
    int c = cell[me];
    int b = S->cst[c], e = b + S->cnt[c], r = 0;
    for (int t = b; t < e; t++) r += (S->bslot[t] < me);
    perm[b + r] = me;
}

// the device address of the scratch area on the current device: looked up
// again outside a capture, the kept one during a capture
int scratch_for_device(cudaStream_t st, NoAllocScratch** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MPS_ERR_CUDA;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return MPS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return MPS_ERR_CUDA;
        g_scratch_ptr[dev] = p;
    }
    if (!g_scratch_ptr[dev]) return MPS_ERR_CUDA;  // first call inside a capture
    *out = (NoAllocScratch*)g_scratch_ptr[dev];
    return MPS_OK;
}

}  // namespace

extern "C" int mps_cell_order_noalloc(const mps_config* cfg, double re, int n, const double* x,
                                      const double* y, const double* z, int* cell, int* perm,
                                      unsigned int* out_of_grid, void* stream)
{
    if (!cfg || n <= 0 || !x || !y || !cell || !perm || !out_of_grid || !(re > 0) ||
        (cfg->dim == 3 && !z) || (cfg->dim != 2 && cfg->dim != 3))
        return MPS_ERR_ARG;
    if (n > kNoAllocMaxParticles) return MPS_ERR_ARG;
    // every axis count and the total are checked before they are multiplied
    Grid g;
    if (!grid_for(cfg->xmin, cfg->xmax, cfg->ymin, cfg->ymax, cfg->zmin, cfg->zmax, cfg->dim, re,
                  cfg->delta, kNoAllocMaxCells - 2, &g))
        return MPS_ERR_ARG;
    NoAllocScratch* S = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    int r = scratch_for_device(st, &S);
    if (r != MPS_OK) return r;
    const int m = g.tnc + 2;
    if (cudaMemsetAsync(S->cnt, 0, sizeof(int) * m, st) != cudaSuccess) return MPS_ERR_CUDA;
    if (cudaMemsetAsync(out_of_grid, 0, sizeof(unsigned int), st) != cudaSuccess)
        return MPS_ERR_CUDA;
    int nb = grid_blocks(n);
    if (cfg->dim == 3)
        k_na_hash<3><<<nb, kBlock, 0, st>>>(n, g, x, y, z, cell, S, out_of_grid);
    else
        k_na_hash<2><<<nb, kBlock, 0, st>>>(n, g, x, y, z, cell, S, out_of_grid);
    k_na_scan<<<1, kNoAllocScanThreads, 0, st>>>(m, S);
    k_na_scatter<<<nb, kBlock, 0, st>>>(n, cell, S);
    k_na_rank<<<nb, kBlock, 0, st>>>(n, cell, S, perm);
    vmps_count_launch(4);
    return cudaGetLastError() == cudaSuccess ? MPS_OK : MPS_ERR_CUDA;
}
