// mps_neighbors.cu -- hash, sort, reorder and neighbour lists (NEIGHBOR,
// functions.cu:2788-2929; the reference GPU path's calcHash / sort_by_key /
// findCellStart / createNeighbourArrays, neighbour_parallel.cu:37-199).
//
// Per step:
//   1. k_hash      exact FP64 cell number of every particle on both grids
//                  (Laplacian grid = primary order, PND grid = index only),
//                  bucket counts by atomics;
//   2. scan        exclusive prefix sums of the counts (cell starts);
//   3. k_scatter   particles into their cell bucket (arbitrary order);
//   4. k_rank      order inside a bucket by (x, original id) on both grids,
//                  so that every x-triple of cells is sorted by x; NEIGHBOR's
//                  own order, (cell, id) -- the stable counting sort of the
//                  reference's insertion loop (functions.cu:2820) -- is
//                  formed when a permutation is downloaded;
//   5. k_gather    reorder the persistent particle state into cell order;
//   6. k_lists     both lists, membership decided with the reference's exact
//                  FP64 arithmetic; Q particles of one cell per warp for the
//                  Laplacian radius (x-windowed runs), GS lanes per particle
//                  for the PND radius.  Exported rows are put back in the
//                  reference's scan order (x offset outermost, then y, z;
//                  ascending id inside a cell).
#include <cmath>
#include <cstdio>

#include "mps_internal.cuh"

using namespace vmps;

namespace {

template <int DIM>
__global__ void k_hash(int n, Grid gl, Grid gs, const double* __restrict__ x,
                       const double* __restrict__ y, const double* __restrict__ z,
                       int* __restrict__ cell_l, int* __restrict__ cell_s,
                       int* __restrict__ cnt_l, int* __restrict__ cnt_s,
                       int* __restrict__ bpos_l, int* __restrict__ bpos_s, unsigned int* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
    int a, b, c;
    bool ok = cell_coords<DIM>(gl, xi, yi, zi, a, b, c);
    int Cl = a + (b - 1) * gl.ncx + (c - 1) * gl.ncx * gl.ncy;
    ok = cell_coords<DIM>(gs, xi, yi, zi, a, b, c) && ok;
    int Cs = a + (b - 1) * gs.ncx + (c - 1) * gs.ncx * gs.ncy;
    if (!ok) set_error(err, MPS_ERR_CELL);
    cell_l[i] = Cl;
    cell_s[i] = Cs;
    bpos_l[i] = atomicAdd(&cnt_l[Cl], 1);
    bpos_s[i] = atomicAdd(&cnt_s[Cs], 1);
}

// three-phase exclusive scan (tile sums, scan of tile sums, tile rescans)
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* sh, int* total)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int s = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
        int si = s;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        sh[lane] = si - s;
        if (lane == 31) sh[32] = si;
    }
    __syncthreads();
    int r = inc - v + sh[wid];
    if (total) *total = sh[32];
    __syncthreads();
    return r;
}

__global__ void k_scan_tiles(int m, const int* __restrict__ in, int* __restrict__ tile_sum)
{
    __shared__ int sh[33];
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int s = 0;
    for (int k = 0; k < kScanItems; k++)
        if (base + k < m) s += in[base + k];
    int tot;
    block_exclusive_scan(s, sh, &tot);
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = tot;
}

__global__ void k_scan_sums(int tiles, int* tile_sum)
{
    __shared__ int sh[33];
    int carry = 0;
    for (int base = 0; base < tiles; base += kScanThreads) {
        int i = base + threadIdx.x;
        int v = i < tiles ? tile_sum[i] : 0;
        int tot;
        int e = block_exclusive_scan(v, sh, &tot);
        if (i < tiles) tile_sum[i] = e + carry;
        carry += tot;
        __syncthreads();
    }
}

__global__ void k_scan_apply(int m, const int* __restrict__ in, const int* __restrict__ tile_sum,
                             int* __restrict__ out)
{
    __shared__ int sh[33];
    int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int vals[kScanItems];
    int s = 0;
    for (int k = 0; k < kScanItems; k++) {
        vals[k] = (base + k < m) ? in[base + k] : 0;
        s += vals[k];
    }
    int e = block_exclusive_scan(s, sh, nullptr) + tile_sum[blockIdx.x];
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < m) out[base + k] = e;
        e += vals[k];
    }
}

// Unsigned key whose integer order is the order of the doubles (-0 just
// below +0, NaNs at the ends), so that (key, id) is a strict total order
// even on a state that has gone non-finite: every bucket position is taken
// exactly once.
__device__ __forceinline__ unsigned long long order_key(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void k_scatter(int n, const int* __restrict__ cell_l, const int* __restrict__ cell_s,
                          const int* __restrict__ bpos_l, const int* __restrict__ bpos_s,
                          const int* __restrict__ cst_l, const int* __restrict__ cst_s,
                          const int* __restrict__ oid, const double* __restrict__ x,
                          int* __restrict__ bslot_l, int* __restrict__ boid_l,
                          unsigned long long* __restrict__ bx_l, int* __restrict__ bslot_s,
                          int* __restrict__ boid_s, unsigned long long* __restrict__ bx_s)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int o = oid[i];
    int q = cst_l[cell_l[i]] + bpos_l[i];
    bslot_l[q] = i;
    boid_l[q] = o;
    const unsigned long long key = order_key(x[i]);
    bx_l[q] = key;
    int qs = cst_s[cell_s[i]] + bpos_s[i];
    bslot_s[qs] = i;
    boid_s[qs] = o;
    bx_s[qs] = key;
}

// Rank inside the bucket by (x, original id) on both grids, so that every
// cell's particles lie in ascending x and each x-triple of cells is sorted
// by x (the list passes window their candidate runs on x).  Laplacian grid
// (the memory order): src[new] = old slot and inv[old] = new.  PND grid:
// perm_tmp[position] = old slot and key_s[position] = x's order key.
// NEIGHBOR's own orders, (cell, id) on each grid (the stable counting sort
// of the reference's insertion loop, functions.cu:2820), are formed when
// the permutations are downloaded.
__global__ void k_rank(int n, const int* __restrict__ cell_l, const int* __restrict__ cell_s,
                       const int* __restrict__ cst_l, const int* __restrict__ cnt_l,
                       const int* __restrict__ cst_s, const int* __restrict__ cnt_s,
                       const int* __restrict__ bslot_l, const int* __restrict__ boid_l,
                       const unsigned long long* __restrict__ bx_l,
                       const int* __restrict__ bslot_s, const int* __restrict__ boid_s,
                       const unsigned long long* __restrict__ bx_s,
                       int* __restrict__ src, int* __restrict__ inv, int* __restrict__ perm_tmp,
                       unsigned long long* __restrict__ key_s)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    {
        int s = bslot_l[q], me = boid_l[q];
        const unsigned long long xm = bx_l[q];
        int c = cell_l[s];
        int b = cst_l[c], e = b + cnt_l[c], r = 0;
        for (int t = b; t < e; t++) {
            const unsigned long long xt = bx_l[t];
            r += (xt < xm || (xt == xm && boid_l[t] < me));
        }
        src[b + r] = s;
        inv[s] = b + r;
    }
    {
        int s = bslot_s[q], me = boid_s[q];
        const unsigned long long xm = bx_s[q];
        int c = cell_s[s];
        int b = cst_s[c], e = b + cnt_s[c], r = 0;
        for (int t = b; t < e; t++) {
            const unsigned long long xt = bx_s[t];
            r += (xt < xm || (xt == xm && boid_s[t] < me));
        }
        perm_tmp[b + r] = s;
        key_s[b + r] = xm;
    }
}

struct GatherSet {
    const void* from[24];
    void* to[24];
    int elem[24];
    int count;
};

__global__ void k_gather(int n, const int* __restrict__ src, GatherSet g)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int s = src[k];
    for (int a = 0; a < g.count; a++) {
        if (g.elem[a] == 8)
            ((double*)g.to[a])[k] = ((const double*)g.from[a])[s];
        else
            ((int*)g.to[a])[k] = ((const int*)g.from[a])[s];
    }
}

__global__ void k_scene_ranges_init(int ns, int n, int* __restrict__ first, int* __restrict__ last)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ns) { first[k] = n; last[k] = 0; }
}

// slot range [first, last) of each scene after the reorder
__global__ void k_scene_ranges(int n, const int* __restrict__ scene, int* __restrict__ first,
                               int* __restrict__ last)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int s = scene[k];
    atomicMin(&first[s], k);
    atomicMax(&last[s], k + 1);
}

__global__ void k_translate(int n, const int* __restrict__ inv, const int* __restrict__ in,
                            int* __restrict__ out)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = inv[in[k]];
}

// One list, G lanes per particle, row-major.  Membership is the reference's
// exact FP64 rule (3D: d <= cut, self included; 2D: d < cut, self excluded)
// over the 3x3(x3) cells around the particle's cell (functions.cu:2854-2918).
// The three cells of one (y, z) offset are consecutive in the grid's order
// (cells are numbered x fastest), so they are scanned as one range; cells
// whose box lies farther than the cutoff from the particle are left out.
// Inside a cell the order is by x, so a range is sorted by x and shrinks to
// the x-window [x_i - r, x_i + r], r the largest |dx| that the particle's
// distance to the range's (y, z) cells leaves under the cutoff
// (conservative margins); the lanes of the group find the windows of their
// runs (lane l: runs l, l + G, ...) by binary searches over the order keys
// of x.  Rows are stored in scan order (y, z outer, memory order inside);
// the reference's own order (x offset outermost, ascending id per cell) is
// restored when lists are exported (mps_download_lists).
// 6 resident blocks per SM (40 registers): with the warp's groups stepping
// together, the neighbour stage 4.51 ms on the 1.6 M-particle dam against
// 4.61 ms at 8 blocks (32 registers, spills) and 4.69 ms for divergent groups
template <int DIM, int G>
__global__ void __launch_bounds__(256, 6) k_lists(int n, Grid g, double cut, float cut_lo, float cut_hi, int cap,
                        const double4* __restrict__ P4, const float4* __restrict__ P4f,
                        const int* __restrict__ cell, const int* __restrict__ cst,
                        const int* __restrict__ cnt, const int* __restrict__ perm,
                        const unsigned long long* __restrict__ keys,
                        int* __restrict__ out, int* __restrict__ len, int* len_max, int which,
                        unsigned int* err)
{
    // The warp's 32 / G groups step through their runs together (every
    // loop trip count is the warp's largest, lanes past their own run's end
    // idle): divergent groups would replay each ballot and shuffle once per
    // group.  Groups past the last row take part with empty runs.
    Grp<G> q;
    const bool live = q.gid < n;
    const int i = live ? (int)q.gid : 0;
    double4 pi = P4[i];
    float4 fi = P4f[i];
    int C = cell[i] - 1;
    int ic = C % g.ncx + 1, jc = (C / g.ncx) % g.ncy + 1, kc = C / (g.ncx * g.ncy) + 1;
    int m1 = (ic == 1) ? 0 : -1, m2 = (ic == g.ncx) ? 0 : 1;
    int m3 = (jc == 1) ? 0 : -1, m4 = (jc == g.ncy) ? 0 : 1;
    int m5 = 0, m6 = 0;
    if (DIM == 3) { m5 = (kc == 1) ? 0 : -1; m6 = (kc == g.ncz) ? 0 : 1; }
    // distances from the particle to the faces of its own cell; a margin of
    // 1e-9 cell sizes keeps the culling conservative under rounding
    const double mx = 1e-9 * g.re, mz = 1e-9 * g.rez;
    double lox = pi.x - (g.xmin + (ic - 1) * g.re) - mx, hix = (g.xmin + ic * g.re) - pi.x - mx;
    double loy = pi.y - (g.ymin + (jc - 1) * g.re) - mx, hiy = (g.ymin + jc * g.re) - pi.y - mx;
    double loz = 0, hiz = 0;
    if (DIM == 3) {
        loz = pi.z - (g.zmin + (kc - 1) * g.rez) - mz;
        hiz = (g.zmin + kc * g.rez) - pi.z - mz;
    }
    auto gap2 = [](int off, double lo, double hi) {
        double d = off < 0 ? lo : (off > 0 ? hi : 0.0);
        return d > 0 ? d * d : 0.0;
    };
    const double gxl = gap2(-1, lox, hix), gxh = gap2(1, lox, hix);
    const int ndp = m6 - m5 + 1, nt = live ? (m4 - m3 + 1) * ndp : 0;
    // the windows of this lane's runs t = lane, lane + G, ...
    constexpr int NT = DIM == 3 ? 9 : 3;
    constexpr int R = (NT + G - 1) / G;
    int wb[R], we[R];
#pragma unroll
    for (int u = 0; u < R; u++) {
        const int t = q.lane + u * G;
        wb[u] = 0;
        we[u] = 0;
        if (t >= nt) continue;
        const int cu = m3 + t / ndp, dp = m5 + t % ndp;
        const double gyz = gap2(cu, loy, hiy) + (DIM == 3 ? gap2(dp, loz, hiz) : 0.0);
        if (gyz > cut) continue;
        const int rlo = (m1 < 0 && gyz + gxl <= cut) ? -1 : 0;
        const int rhi = (m2 > 0 && gyz + gxh <= cut) ? 1 : 0;
        const int Cr = ic + (jc - 1 + cu) * g.ncx + (kc - 1 + dp) * g.ncx * g.ncy;
        // |dx| above r puts the pair beyond the cutoff with room for every
        // rounding of the distance
        const double r = sqrt(cut - gyz) * (1.0 + 1e-12) + mx;
        const unsigned long long klo = order_key(pi.x - r), khi = order_key(pi.x + r);
        int lo_a = cst[Cr + rlo], hi_a = cst[Cr + rhi] + cnt[Cr + rhi];
        int lo_b = lo_a, hi_b = hi_a;
        while (lo_a < hi_a || lo_b < hi_b) {
            const int ma = (lo_a + hi_a) >> 1, mb = (lo_b + hi_b) >> 1;
            const bool sa = lo_a < hi_a, sb = lo_b < hi_b;
            const unsigned long long va = sa ? keys[ma] : 0ull, vb = sb ? keys[mb] : 0ull;
            if (sa) { if (va < klo) lo_a = ma + 1; else hi_a = ma; }
            if (sb) { if (vb <= khi) lo_b = mb + 1; else hi_b = mb; }
        }
        wb[u] = lo_a;
        we[u] = max(lo_a, lo_b);
    }
    int* row = out + (size_t)i * cap;
    int k = 0;
    const unsigned full = 0xffffffffu;
#pragma unroll
    for (int t = 0; t < NT; t++) {
        const int src_lane = (int)q.base + t % G;
        const int b = __shfl_sync(full, wb[t / G], src_lane);
        const int e = __shfl_sync(full, we[t / G], src_lane);
        const int trips = __reduce_max_sync(full, (e - b + G - 1) / G);
        for (int it = 0; it < trips; it++) {
            const int jj = b + it * G + q.lane;
            const bool valid = jj < e;
            bool in = false;
            int j = 0;
            if (valid) {
                j = perm[jj];
                // FP32 screen; the exact FP64 rule decides only inside
                // the screening margin [cut_lo, cut_hi]
                const float4 fj = P4f[j];
                const float ex = fj.x - fi.x, ey = fj.y - fi.y,
                            ez = DIM == 3 ? fj.z - fi.z : 0.f;
                // fused multiply-adds: fewer roundings than the bound assumes
                const float f2 = __fmaf_rn(ez, ez, __fmaf_rn(ey, ey, __fmul_rn(ex, ex)));
                if (f2 < cut_lo) {
                    in = (DIM == 3) || (j != i);
                } else if (f2 <= cut_hi) {
                    const double4 pj = P4[j];
                    const double d2 = dist2<DIM>(pj.x - pi.x, pj.y - pi.y,
                                                 DIM == 3 ? pj.z - pi.z : 0.0);
                    in = (DIM == 3) ? (d2 <= cut) : (j != i && d2 < cut);
                }
            }
            const unsigned m = (__ballot_sync(full, in) >> q.base) & ((1u << G) - 1u);
            if (in) {
                const int pos = k + __popc(m & ((1u << q.lane) - 1u));
                if (pos < cap) row[pos] = j;
            }
            k += __popc(m);
        }
    }
    // the longest row: one atomic per warp instead of one per particle
    const int km = __reduce_max_sync(full, live ? k : 0);
    if ((threadIdx.x & 31) == 0) atomicMax(&len_max[which], km);
    if (live && q.lane == 0) {
        if (k > cap) {
            set_error(err, MPS_ERR_LIST_OVERFLOW);
            k = cap;
        }
        len[i] = k;
    }
}

// The same lists for Q particles of one cell at a time, one warp: each
// candidate's packed position is loaded once and tested against the Q
// particles, so the load, the loop and the index work are shared.  Inside a
// cell particles are ordered by x, so each (y, z) run of three cells is
// sorted by x, and a run's candidates for the Q particles lie in one
// contiguous x-window: [min_q(x_q - r_q), max_q(x_q + r_q)], r_q the largest
// |dx| that the particle's distance to the run's (y, z) cells leaves under
// the cutoff (conservative margin).  Lane t finds run t's window by two
// interleaved binary searches over x.  Members keep their memory order, and
// a window a particle's neighbours cannot lie outside of drops only
// non-members, so every row receives exactly the entries, in exactly the
// order, of the one-particle scan of the whole run.  Groups whose particles
// sit in different cells are done one particle at a time.
template <int DIM, int Q>
__device__ __forceinline__ void list_rows(int lane, int i0, int nq, int C, const Grid& g,
                                          double cut, float cut_lo, float cut_hi, int cap,
                                          const double4* __restrict__ P4,
                                          const float4* __restrict__ P4f,
                                          const double* __restrict__ xs,
                                          const int* __restrict__ cst, const int* __restrict__ cnt,
                                          int* __restrict__ out, int* __restrict__ len,
                                          int* len_max, int which, unsigned int* err)
{
    const int c0 = C - 1;
    const int ic = c0 % g.ncx + 1, jc = (c0 / g.ncx) % g.ncy + 1, kc = c0 / (g.ncx * g.ncy) + 1;
    const int m1 = (ic == 1) ? 0 : -1, m2 = (ic == g.ncx) ? 0 : 1;
    const int m3 = (jc == 1) ? 0 : -1, m4 = (jc == g.ncy) ? 0 : 1;
    int m5 = 0, m6 = 0;
    if (DIM == 3) { m5 = (kc == 1) ? 0 : -1; m6 = (kc == g.ncz) ? 0 : 1; }
    const double mx = 1e-9 * g.re, mz = 1e-9 * g.rez;
    auto gap2 = [](int off, double lo, double hi) {
        double d = off < 0 ? lo : (off > 0 ? hi : 0.0);
        return d > 0 ? d * d : 0.0;
    };
    // lane t < nt owns (y, z) run t: whether any particle needs it, whether
    // any needs its x-1 / x+1 cell, and the union of their x-windows
    const int ndp = m6 - m5 + 1, nt = (m4 - m3 + 1) * ndp;
    const int cu = m3 + lane / ndp, dp = m5 + lane % ndp;
    bool scan_me = false, lo_me = false, hi_me = false;
    double xlo = INFINITY, xhi = -INFINITY;
    unsigned lt_mask;  // lanes below this one
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt_mask));
    float4 fi[Q];
    int k[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) {
        k[q] = 0;
        if (q >= nq) continue;
        const double4 pi = P4[i0 + q];
        fi[q] = P4f[i0 + q];
        if (lane >= nt) continue;
        const double lox = pi.x - (g.xmin + (ic - 1) * g.re) - mx;
        const double hix = (g.xmin + ic * g.re) - pi.x - mx;
        const double loy = pi.y - (g.ymin + (jc - 1) * g.re) - mx;
        const double hiy = (g.ymin + jc * g.re) - pi.y - mx;
        double gyz = gap2(cu, loy, hiy);
        if (DIM == 3) {
            const double loz = pi.z - (g.zmin + (kc - 1) * g.rez) - mz;
            const double hiz = (g.zmin + kc * g.rez) - pi.z - mz;
            gyz += gap2(dp, loz, hiz);
        }
        if (gyz > cut) continue;
        scan_me = true;
        if (m1 < 0 && gyz + gap2(-1, lox, hix) <= cut) lo_me = true;
        if (m2 > 0 && gyz + gap2(1, lox, hix) <= cut) hi_me = true;
        // |dx| above r puts the pair beyond the cutoff with room for every
        // rounding of the distance
        const double r = sqrt(cut - gyz) * (1.0 + 1e-12) + mx;
        xlo = fmin(xlo, pi.x - r);
        xhi = fmax(xhi, pi.x + r);
    }
    const unsigned scan_t = __ballot_sync(0xffffffffu, scan_me);
    // one batch of 32 candidates against the Q particles
    auto batch = [&](int j, bool valid, float4 fj) {
#pragma unroll
        for (int q = 0; q < Q; q++) {
            if (q >= nq) break;
            const int i = i0 + q;
            bool in = false;
            if (valid) {
                const float ex = fj.x - fi[q].x, ey = fj.y - fi[q].y,
                            ez = DIM == 3 ? fj.z - fi[q].z : 0.f;
                const float f2 = __fmaf_rn(ez, ez, __fmaf_rn(ey, ey, __fmul_rn(ex, ex)));
                if (f2 < cut_lo) {
                    in = (DIM == 3) || (j != i);
                } else if (f2 <= cut_hi) {
                    const double4 pi = P4[i], pj = P4[j];
                    const double d2 = dist2<DIM>(pj.x - pi.x, pj.y - pi.y,
                                                 DIM == 3 ? pj.z - pi.z : 0.0);
                    in = (DIM == 3) ? (d2 <= cut) : (j != i && d2 < cut);
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, in);
            if (m) {  // warp-uniform: many batches hold no member of this particle
                if (in) {
                    const int pos = k[q] + __popc(m & lt_mask);
                    if (pos < cap) out[(size_t)i * cap + pos] = j;
                }
                k[q] += __popc(m);
            }
        }
    };
    auto scan = [&](int b, int e) {
        for (int base = b; base < e; base += 32) {
            const int j = base + lane;
            const bool valid = j < e;
            batch(j, valid, valid ? P4f[j] : make_float4(0.f, 0.f, 0.f, 0.f));
        }
    };
    // the candidate window of every scanned (y, z) run, found at once (lane
    // t holds run t's [b, e)): first position with x >= xlo, first with
    // x > xhi, both searches advancing together
    int rb = 0, rend = 0;
    if (scan_me) {
        const int Cr = ic + (jc - 1 + cu) * g.ncx + (kc - 1 + dp) * g.ncx * g.ncy;
        const int rlo = lo_me ? -1 : 0, rhi = hi_me ? 1 : 0;
        const int b = cst[Cr + rlo], e = cst[Cr + rhi] + cnt[Cr + rhi];
        int lo_a = b, hi_a = e, lo_b = b, hi_b = e;
        while (lo_a < hi_a || lo_b < hi_b) {
            const int ma = (lo_a + hi_a) >> 1, mb = (lo_b + hi_b) >> 1;
            const bool sa = lo_a < hi_a, sb = lo_b < hi_b;
            const double va = sa ? xs[ma] : 0.0, vb = sb ? xs[mb] : 0.0;
            if (sa) { if (va < xlo) lo_a = ma + 1; else hi_a = ma; }
            if (sb) { if (vb <= xhi) lo_b = mb + 1; else hi_b = mb; }
        }
        rb = lo_a;
        rend = max(lo_a, lo_b);
    }
    for (int t = 0; t < nt; t++) {
        if (!(scan_t >> t & 1u)) continue;
        scan(__shfl_sync(0xffffffffu, rb, t), __shfl_sync(0xffffffffu, rend, t));
    }
    if (lane == 0) {
        int km = 0;
#pragma unroll
        for (int q = 0; q < Q; q++)
            if (q < nq) km = max(km, k[q]);
        atomicMax(&len_max[which], km);
#pragma unroll
        for (int q = 0; q < Q; q++) {
            if (q >= nq) break;
            int kq = k[q];
            if (kq > cap) {
                set_error(err, MPS_ERR_LIST_OVERFLOW);
                kq = cap;
            }
            len[i0 + q] = kq;
        }
    }
}

// 4 resident blocks per SM (at most 64 registers; 66 without the bound
// would leave 3)
template <int DIM, int Q>
__global__ void __launch_bounds__(256, 4) k_lists_q(int n, Grid g, double cut, float cut_lo, float cut_hi, int cap,
                          const double4* __restrict__ P4, const float4* __restrict__ P4f,
                          const double* __restrict__ xs,
                          const int* __restrict__ cell, const int* __restrict__ cst,
                          const int* __restrict__ cnt, int* __restrict__ out,
                          int* __restrict__ len, int* len_max, int which, unsigned int* err)
{
    const int lane = threadIdx.x & 31;
    const long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w * Q >= n) return;  // whole warps leave together
    const int i0 = (int)(w * Q);
    const int nq = min(Q, n - i0);
    const int C = cell[i0];
    bool same = true;
    for (int q = 1; q < nq; q++) same = same && cell[i0 + q] == C;
    if (same) {
        list_rows<DIM, Q>(lane, i0, nq, C, g, cut, cut_lo, cut_hi, cap, P4, P4f, xs, cst, cnt,
                          out, len, len_max, which, err);
    } else {
        for (int q = 0; q < nq; q++)
            list_rows<DIM, Q>(lane, i0 + q, 1, cell[i0 + q], g, cut, cut_lo, cut_hi, cap, P4, P4f,
                              xs, cst, cnt, out, len, len_max, which, err);
    }
}

// particles per warp in the Laplacian list (measured on the 1.6 M-particle
// dam: 2 and 4 equal, 8 slower)
constexpr int kListQ = 4;

int scan(mps_ctx* ctx, int m, const int* in, int* out, int* tile_sum)
{
    int tiles = (m + kScanTile - 1) / kScanTile;
    k_scan_tiles<<<tiles, kScanThreads, 0, ctx->stream>>>(m, in, tile_sum);
    k_scan_sums<<<1, kScanThreads, 0, ctx->stream>>>(tiles, tile_sum);
    k_scan_apply<<<tiles, kScanThreads, 0, ctx->stream>>>(m, in, tile_sum, out);
    vmps_count_launch(3);
    return MPS_OK;
}

}  // namespace

int vmps_scan(mps_ctx* ctx, int m, const int* in, int* out)
{
    return scan(ctx, m, in, out, ctx->scan_tmp);
}

// Persistent fields carried through the reorder (all other fields are
// recomputed each step before use).
static void persistent_set(mps_ctx* ctx, GatherSet& g, std::vector<void**>& slots,
                           std::vector<void*>& alts)
{
    g.count = 0;
    slots.clear();
    double** d[] = {&ctx->x, &ctx->y, &ctx->z, &ctx->u, &ctx->v, &ctx->w, &ctx->p, &ctx->pnew,
                    &ctx->phat, &ctx->un, &ctx->vn, &ctx->wn, &ctx->rho, &ctx->nd, &ctx->pold};
    int** ii[] = {&ctx->ptype, &ctx->oid, &ctx->cell_l, &ctx->cell_s, &ctx->scene, &ctx->own};
    for (auto f : d) {
        g.from[g.count] = *f;
        g.elem[g.count] = 8;
        slots.push_back((void**)f);
        g.count++;
    }
    for (auto f : ii) {
        g.from[g.count] = *f;
        g.elem[g.count] = 4;
        slots.push_back((void**)f);
        g.count++;
    }
    for (int a = 0; a < g.count; a++) g.to[a] = alts[a];
}

// Alternate buffers for the reorder live in ctx->owned after the primaries;
// they are registered by vmps_alloc_reorder() in mps_context.cu.
extern std::vector<void*>& vmps_reorder_alts(mps_ctx* ctx);

// Exchange the persistent fields with their alternates (the reorder wrote
// the alternates).  A replayed step graph skips the capture-time host code,
// so the graph path calls this once per replay.
void vmps_reorder_swap(mps_ctx* ctx)
{
    GatherSet g;
    std::vector<void**> slots;
    std::vector<void*>& alts = vmps_reorder_alts(ctx);
    persistent_set(ctx, g, slots, alts);
    for (int a = 0; a < g.count; a++) {
        void* old = *slots[a];
        *slots[a] = alts[a];
        alts[a] = old;
    }
    ctx->swaps++;
}

int vmps_neighbors(mps_ctx* ctx)
{
    const int n = ctx->n;
    cudaStream_t st = ctx->stream;
    int nb = grid_blocks(n);
    VMPS_CUDA(ctx, cudaMemsetAsync(ctx->cnt_l, 0, sizeof(int) * (ctx->gl.tnc + 2), st));
    VMPS_CUDA(ctx, cudaMemsetAsync(ctx->cnt_s, 0, sizeof(int) * (ctx->gs.tnc + 2), st));
    VMPS_CUDA(ctx, cudaMemsetAsync(ctx->len_max, 0, sizeof(int) * 2, st));
    if (ctx->cfg.dim == 3)
        k_hash<3><<<nb, kBlock, 0, st>>>(n, ctx->gl, ctx->gs, ctx->x, ctx->y, ctx->z, ctx->cell_l,
                                         ctx->cell_s, ctx->cnt_l, ctx->cnt_s, ctx->bpos_l,
                                         ctx->bpos_s, ctx->d_err);
    else
        k_hash<2><<<nb, kBlock, 0, st>>>(n, ctx->gl, ctx->gs, ctx->x, ctx->y, ctx->z, ctx->cell_l,
                                         ctx->cell_s, ctx->cnt_l, ctx->cnt_s, ctx->bpos_l,
                                         ctx->bpos_s, ctx->d_err);
    vmps_count_launch(1);
    scan(ctx, ctx->gl.tnc + 2, ctx->cnt_l, ctx->cst_l, ctx->scan_tmp);
    scan(ctx, ctx->gs.tnc + 2, ctx->cnt_s, ctx->cst_s, ctx->scan_tmp);
    k_scatter<<<nb, kBlock, 0, st>>>(n, ctx->cell_l, ctx->cell_s, ctx->bpos_l, ctx->bpos_s,
                                     ctx->cst_l, ctx->cst_s, ctx->oid, ctx->x, ctx->bslot_l,
                                     ctx->boid_l, ctx->bx_l, ctx->bslot_s, ctx->boid_s,
                                     ctx->bx_s);
    k_rank<<<nb, kBlock, 0, st>>>(n, ctx->cell_l, ctx->cell_s, ctx->cst_l, ctx->cnt_l, ctx->cst_s,
                                  ctx->cnt_s, ctx->bslot_l, ctx->boid_l, ctx->bx_l,
                                  ctx->bslot_s, ctx->boid_s, ctx->bx_s, ctx->src, ctx->inv,
                                  ctx->perm_s_tmp, ctx->key_s);
    vmps_count_launch(2);
    // reorder persistent state into cell order
    GatherSet g;
    std::vector<void**> slots;
    std::vector<void*>& alts = vmps_reorder_alts(ctx);
    persistent_set(ctx, g, slots, alts);
    k_gather<<<nb, kBlock, 0, st>>>(n, ctx->src, g);
    vmps_count_launch(1);
    vmps_reorder_swap(ctx);
    k_translate<<<nb, kBlock, 0, st>>>(n, ctx->inv, ctx->perm_s_tmp, ctx->perm_s);
    vmps_count_launch(1);
    if (ctx->nscenes > 1) {
        k_scene_ranges_init<<<grid_blocks(ctx->nscenes), kBlock, 0, st>>>(ctx->nscenes, n,
                                                                          ctx->sfirst, ctx->slast);
        k_scene_ranges<<<nb, kBlock, 0, st>>>(n, ctx->scene, ctx->sfirst, ctx->slast);
        vmps_count_launch(2);
    }
    {
        int r = vmps_pack(ctx);
        if (r != MPS_OK) return r;
    }
    if (ctx->profile) VMPS_CUDA(ctx, cudaEventRecord(ctx->ev[6], st));
    {
        // Laplacian list: kListQ particles per warp
        const int nq32 = (int)((((long)n + kListQ - 1) / kListQ * 32 + kBlock - 1) / kBlock);
        // screening window, rounded outwards to float
        auto lo = [&](double c) { return std::nextafter((float)(c - ctx->screen_abs), 0.f); };
        auto hi = [&](double c) { return std::nextafter((float)(c + ctx->screen_abs), INFINITY); };
        float lo_l = lo(ctx->cut_l), hi_l = hi(ctx->cut_l), lo_s = lo(ctx->cut_s), hi_s = hi(ctx->cut_s);
        if (ctx->cfg.dim == 3) {
            constexpr int GS = SmallG<3>::G;
            k_lists_q<3, kListQ><<<nq32, kBlock, 0, st>>>(
                n, ctx->gl, ctx->cut_l, lo_l, hi_l, ctx->cap_l, ctx->P4, ctx->P4f, ctx->x,
                ctx->cell_l, ctx->cst_l, ctx->cnt_l, ctx->nbr_l, ctx->len_l, ctx->len_max, 0, ctx->d_err);
            if (ctx->tune_small_wide)
                k_lists<3, 2 * GS><<<(int)(((long)n * 2 * GS + kBlock - 1) / kBlock), kBlock, 0, st>>>(
                    n, ctx->gs, ctx->cut_s, lo_s, hi_s, ctx->cap_s, ctx->P4, ctx->P4f, ctx->cell_s,
                    ctx->cst_s, ctx->cnt_s, ctx->perm_s, ctx->key_s, ctx->nbr_s, ctx->len_s, ctx->len_max, 1,
                    ctx->d_err);
            else
                k_lists<3, GS><<<(int)(((long)n * GS + kBlock - 1) / kBlock), kBlock, 0, st>>>(
                    n, ctx->gs, ctx->cut_s, lo_s, hi_s, ctx->cap_s, ctx->P4, ctx->P4f, ctx->cell_s,
                    ctx->cst_s, ctx->cnt_s, ctx->perm_s, ctx->key_s, ctx->nbr_s, ctx->len_s, ctx->len_max, 1,
                    ctx->d_err);
        } else {
            constexpr int GS = SmallG<2>::G;
            k_lists_q<2, kListQ><<<nq32, kBlock, 0, st>>>(
                n, ctx->gl, ctx->cut_l, lo_l, hi_l, ctx->cap_l, ctx->P4, ctx->P4f, ctx->x,
                ctx->cell_l, ctx->cst_l, ctx->cnt_l, ctx->nbr_l, ctx->len_l, ctx->len_max, 0, ctx->d_err);
            if (ctx->tune_small_wide)
                k_lists<2, 2 * GS><<<(int)(((long)n * 2 * GS + kBlock - 1) / kBlock), kBlock, 0, st>>>(
                    n, ctx->gs, ctx->cut_s, lo_s, hi_s, ctx->cap_s, ctx->P4, ctx->P4f, ctx->cell_s,
                    ctx->cst_s, ctx->cnt_s, ctx->perm_s, ctx->key_s, ctx->nbr_s, ctx->len_s, ctx->len_max, 1,
                    ctx->d_err);
            else
                k_lists<2, GS><<<(int)(((long)n * GS + kBlock - 1) / kBlock), kBlock, 0, st>>>(
                    n, ctx->gs, ctx->cut_s, lo_s, hi_s, ctx->cap_s, ctx->P4, ctx->P4f, ctx->cell_s,
                    ctx->cst_s, ctx->cnt_s, ctx->perm_s, ctx->key_s, ctx->nbr_s, ctx->len_s, ctx->len_max, 1,
                    ctx->d_err);
        }
    }
    vmps_count_launch(2);
    if (ctx->profile) {
        VMPS_CUDA(ctx, cudaEventRecord(ctx->ev[7], st));
        VMPS_CUDA(ctx, cudaEventSynchronize(ctx->ev[7]));
        float ms = 0;
        VMPS_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[6], ctx->ev[7]));
        ctx->lists_ms += ms;
        ctx->lists_launches++;
    }
    // mps_step_io's velocities and pressure, copied while the lists were
    // built, go into the new order (nothing above reads them)
    if (ctx->state_defer) {
        int r = vmps_state_apply(ctx);
        if (r != MPS_OK) return r;
    }
    VMPS_CUDA(ctx, cudaGetLastError());
    return MPS_OK;
}
