// mps_ppe.cu -- pressure Poisson equation: assembly and CG (PRESSURECALC
// Method 1, functions.cu:2465-2549; MATRIX functions.cu:869-1005; CGM
// functions.cu:506-716).
//
// Assembly keeps the reference's coefficients and diagonal (including the
// 1e-7/dt^2 compressibility term) but stores only the columns that can be
// non-zero in A*x: unknown (bcon == 0) neighbours with a non-zero weight.
// Dirichlet columns (bcon == 1, p fixed at 0) add to the diagonal only.
//
// The solver is Jacobi-preconditioned (or plain) CG on the unknown rows,
// stopped on the relative residual ||r||/||b|| <= cg_tol.  Dot products
// reduce in FP64 through fixed per-block partials that every consumer block
// re-reduces in the same order: deterministic, no atomics, no host sync per
// iteration.  A device flag ends the iteration; the host checks it every few
// iterations.
#include "mps_internal.cuh"

using namespace vmps;

namespace {

enum {
    S_BB = 0, S_RZ, S_RR, S_ZERO, S_NEWRZ, S_NEWRR, S_DONE, S_WORST,
    // mixed precision: inner r.r, its value at the sweep's start, the sweep's
    // target reduction (squared), the staged inner stop, staged inner r.r
    S_RIN, S_RIN0, S_ETA2, S_INDONE, S_NEWRIN,
    S_RR0,  // r.r of the initial guess
    S_COUNT
};
static_assert(S_COUNT <= 16, "cg_scal and red_host hold 16 doubles");
constexpr int kRedThreads = 256;
// lanes per row, measured on the 1.6 M-particle dam: the SpMV keeps a whole
// warp per row (16 or 8 lanes: 0.69 ms against 0.61 ms per launch); the
// assembly runs 16 lanes per row (PPE stage 12.4 ms against 12.8 ms at 32)
constexpr int kRowG = 32;
// systems of at most this many rows run their FP64 products with 16 lanes
// per row (two rows per warp): the 86,118-particle two-phase scene 2.04
// against 2.38 ms per step (rows of ~50 entries leave a warp's second half
// idle, and two rows per warp halve each warp's chain of dependent rows);
// the 1.6 M-particle dam keeps whole warps (0.61 against 0.69 ms per SpMV)
constexpr int kNarrowMaxRows = 262144;
constexpr int kAsmG = 16;
// lanes per row of the mixed-precision products (inner FP32 and refinement):
// 16 (config 2 at 19.37 ms/step against 19.63 ms with 32 or 8 lanes)
constexpr int kIrG = 16;

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) r += sh[k];
        sh[32] = r;
    }
    __syncthreads();
    r = sh[32];
    __syncthreads();
    return r;
}

// every block reduces the same partials in the same order
__device__ __forceinline__ double reduce_parts(const double* part, int nparts, double* sh)
{
    double v = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) v += part[k];
    return block_sum(v, sh);
}

struct Asm {
    WK wk;
    double cw;    // 2*DIM/lambda/n0_l/rho: coefficient of W (functions.cu:915)
    double cm;    // (3 or 2)*re/n0_l/rho: HL coefficient of 1/d^3 (functions.cu:901-910)
    double reg;   // 1e-7/dt/dt (functions.cu:921)
    double tiny2; // fabs(d) <= 1e-15  <=>  d2 <= tiny2
    double n0_s, dt;
    int matopt, srcopt;
};

// The w slot of the predicted positions for an assembly that forms CG's
// starting residual: the guess (pnew) of an unknown (bcon 0), a NaN whose
// low bits code the status otherwise (1: Dirichlet, 2: outside, bcon -1).
// A pressure that has gone NaN reads as an unknown with a NaN guess, as a
// separate gather of it would.
__device__ __forceinline__ double wguess_code(int b)
{
    return __longlong_as_double((long long)(0x7FF8000000000000ull | (b == 1 ? 1ull : 2ull)));
}

__device__ __forceinline__ int wguess_status(double w)
{
    if (w == w) return 0;
    const unsigned long long code = (unsigned long long)__double_as_longlong(w) & 3ull;
    return code == 1 ? 1 : (code == 2 ? -1 : 0);
}

__global__ void k_pack_wguess(int n, const int* __restrict__ bcon, const double* __restrict__ pnew,
                              double4* __restrict__ P4s)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bcon[i];
    reinterpret_cast<double*>(P4s + i)[3] = b == 0 ? pnew[i] : wguess_code(b);
}

// one lane group (kAsmG lanes) per row; the non-zero columns are compacted in list order into
// the row's CSR segment (capacity = the row's list length)
template <int DIM>
// 6 resident blocks per SM (40 registers, a few bytes of spills): measured
// 0.2 ms per step faster than 5 on the 1.6 M-particle dam, 8 spills too much
__global__ void __launch_bounds__(256, 6) k_assemble(int n, int cap, Asm A, const int* __restrict__ nbr,
                           const int* __restrict__ len, const int* __restrict__ bcon,
                           const double4* __restrict__ P4, const double* __restrict__ nsrc,
                           int warm, double* __restrict__ pnew, double* __restrict__ pold,
                           const int* __restrict__ moff,
                           int* __restrict__ mcol, double* __restrict__ mval,
                           int2* __restrict__ mcv32, int* __restrict__ mlen,
                           double* __restrict__ diag, double* __restrict__ source, int w_bcon,
                           int2* __restrict__ mrow, const int* __restrict__ own,
                           int* __restrict__ sysmask, double* __restrict__ r0)
{
    // The warp's two row groups step through their rows together (the trip
    // count is the warp's largest; lanes past their row's end idle), so the
    // ballot is one warp instruction rather than one per diverged group;
    // groups past the last row, and rows outside the system, take part with
    // no entries.
    Grp<kAsmG> q;
    const bool live = q.gid < n;
    const int i = live ? (int)q.gid : 0;
    const int bi = bcon[i];
    const bool mine = own[i] != 0;
    const bool work = live && bi == 0 && mine;
    if (live && q.lane == 0) {
        sysmask[i] = (bi != 0 || !mine) ? 1 : 0;
        if (bi != 0) {
            mlen[i] = 0;
            mrow[i] = make_int2(moff[i], -1);
            diag[i] = 0.0;
            source[i] = 0.0;
            if (warm == 2) pold[i] = pnew[i];
            // with r0 the rows read every neighbour's guess: CG's start
            // zeroes this one instead
            if (!r0) pnew[i] = 0.0;
        } else if (!mine) {  // a ghost: its row belongs to its owner's system, its
            mlen[i] = 0;     // value arrives from the owner (a column here, not a row)
            mrow[i] = make_int2(moff[i], -1);
            diag[i] = 0.0;
            source[i] = 0.0;
        }
    }
    const double4 pi = P4[i];
    const int* row = nbr + (size_t)i * cap;
    int* crow = mcol + moff[i];
    double* vrow = mval + moff[i];
    double dg = 0.0, ax = 0.0;
    int cnt = 0;
    const int L = work ? len[i] : 0;
    const int trips = __reduce_max_sync(0xffffffffu, (L + kAsmG - 1) / kAsmG);
    for (int it = 0; it < trips; it++) {
        int k = it * kAsmG + q.lane;
        double v = 0.0, xj = 0.0;
        int j = -1;
        bool keep = false;
        if (k < L) {
            j = row[k];
            double4 pj;
            int bj;
            if (w_bcon == 2) {  // w: the guess of an unknown, a coded NaN otherwise
                pj = P4[j];
                xj = pj.w;
                bj = wguess_status(pj.w);
                if (j == i) bj = -1;
            } else if (w_bcon) {  // P4's w slot holds bcon: one gather
                if (r0) xj = pnew[j];  // the initial guess, read beside the position
                pj = P4[j];
                bj = j == i ? -1 : (int)pj.w;
            } else {
                if (r0) xj = pnew[j];
                bj = j == i ? -1 : bcon[j];
                if (bj != -1) pj = P4[j];
            }
            if (bj != -1) {
                double d2 = dist2<DIM>(pj.x - pi.x, pj.y - pi.y, DIM == 3 ? pj.z - pi.z : 0.0);
                if (d2 > A.tiny2) {
                    double rD = rsq(d2);
                    v = A.matopt ? A.cm * (rD * rD * rD) : A.cw * w_fast<DIM>(A.wk, d2, rD);
                    keep = (bj == 0 && v != 0.0);
                }
            }
        }
        dg += v;
        const unsigned m = (__ballot_sync(0xffffffffu, keep) >> q.base) & ((1u << kAsmG) - 1u);
        if (keep) {
            int pos = cnt + __popc(m & ((1u << q.lane) - 1u));
            crow[pos] = j;
            vrow[pos] = -v;
            if (mcv32) mcv32[moff[i] + pos] = make_int2(j, __float_as_int((float)(-v)));
            ax += (-v) * xj;
        }
        cnt += __popc(m);
    }
    dg = q.sum(dg);
    if (r0) ax = q.sum(ax);
    if (work && q.lane == 0) {
        diag[i] = dg + A.reg;
        mlen[i] = cnt;
        mrow[i] = make_int2(moff[i], cnt);
        if (!A.srcopt) source[i] = 1.0 / A.dt / A.dt * (nsrc[i] - A.n0_s) / A.n0_s;
        // CG's starting residual b - A x0 of this row, from the entries just
        // formed (x0 = the previous pressure, which this pass leaves as is)
        if (r0) r0[i] = source[i] - ((dg + A.reg) * pnew[i] + ax);
        // initial guess: 0, the previous pressure, or the linear extrapolation
        // 2 p^n - p^(n-1) (pold keeps p^n for the next step)
        if (!warm) {
            pnew[i] = 0.0;
        } else if (warm == 2) {
            double pn = pnew[i];
            pnew[i] = 2.0 * pn - pold[i];
            pold[i] = pn;
        }
    }
}

// HS + ECS source (functions.cu:924-988) is a sequential recurrence over
// particle ids (source[i-1]); it runs as one thread walking the ids.
template <int DIM>
__global__ void k_source_hs(int n, int cap, double re, double n0, double dt,
                            const int* __restrict__ inv_id, const int* __restrict__ nbr,
                            const int* __restrict__ len, const int* __restrict__ bcon,
                            const int* __restrict__ ptype, const double* __restrict__ nstar,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ u,
                            const double* __restrict__ v, const double* __restrict__ w,
                            double* __restrict__ source)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double prev = 0.0;  // source of the previous id (0 unless written this call)
    for (int id = 0; id < n; id++) {
        int i = inv_id[id];
        double out = source[i];
        if (ptype[i] == -1) {
            prev = 0.0;
            continue;
        }
        if (bcon[i] == 0) {
            double alpha = 0.0, beta = 0.0, ECS = 0.0;
            if (id > 0) {
                alpha = (nstar[i] - n0) / n0;
                beta = (dt / n0) * (prev / (-1.0 / (n0 * dt)));
                ECS = fabs(alpha) * (beta / dt) + fabs(beta) * (alpha / dt);
            }
            double sum = 0.0;
            for (int k = 0; k < len[i]; k++) {
                int j = nbr[(size_t)i * cap + k];
                if (ptype[j] <= -1 || i == j) continue;
                double d = sqrt(dist2<DIM>(x[j] - x[i], y[j] - y[i], DIM == 3 ? z[j] - z[i] : 0.0));
                if (fabs(d) <= 1.0e-15) continue;
                double du = u[i] - u[j], dv = v[i] - v[j];
                if (DIM == 3) {
                    double dw = w[i] - w[j];
                    sum += (re / (d * d * d)) *
                           ((x[i] - x[j]) * du + (y[i] - y[j]) * dv + (z[i] - z[j]) * dw);
                } else {
                    sum += (re / (d * d * d)) * ((x[i] - x[j]) * du + (y[i] - y[j]) * dv);
                }
            }
            out = (-1.25 / (n0 * dt)) * sum + ECS;
            if (fabs(out) < 0.99) out = 0;
        } else if (bcon[i] == 1) {
            out = 0.0;
        } else {
            out = 0.0;
        }
        source[i] = out;
        prev = out;
    }
}

struct CG {
    const int* __restrict__ mcol;
    const double* __restrict__ mval;
    const int* __restrict__ mlen;
    const int* __restrict__ moff;
    const double* __restrict__ diag;
    const int* __restrict__ bcon;
    int cap, n, precond, nparts;
    int x0_zero;  // the initial guess is zero: r = b without a product
    const int2* __restrict__ mrow;  // (offset, length) per row; length -1: not an unknown
};

// (A v)_i with one warp on row i of the CSR matrix: coalesced column/value
// streams, two independent accumulators per lane, gathers of v from L2,
// butterfly sum in a fixed order; every lane returns the row's value.  (This
// plain form runs at 32 registers; restructured or deeper-unrolled variants
// measured 15-70% slower on B200.)  The column/value streams are read once
// per product and loaded evict-first (ld.global.cs), which keeps the
// gathered vector in L1/L2: 0.61 against 0.755 ms per launch after 700 steps
// of the 1.6 M-particle dam, equal on its first steps.
template <typename V, int G = kRowG>
__device__ __forceinline__ double spmv_row(const CG& A, const Grp<G>& q,
                                           const V* __restrict__ v, int i, int off, int L)
{
    const int* __restrict__ c = A.mcol + off;
    const double* __restrict__ a = A.mval + off;
    double acc0 = 0.0, acc1 = 0.0;
    int k = q.lane;
    for (; k + G < L; k += 2 * G) {
        int c0 = __ldcs(c + k), c1 = __ldcs(c + k + G);
        double a0 = __ldcs(a + k), a1 = __ldcs(a + k + G);
        acc0 += a0 * (double)v[c0];
        acc1 += a1 * (double)v[c1];
    }
    if (k < L) acc0 += __ldcs(a + k) * (double)v[__ldcs(c + k)];
    double acc = q.sum(acc0 + acc1);
    return A.diag[i] * (double)v[i] + acc;
}

template <typename V, int G = kRowG>
__device__ __forceinline__ double spmv_row_warp(const CG& A, const Grp<G>& q,
                                                const V* __restrict__ v, int i)
{
    return spmv_row(A, q, v, i, A.moff[i], A.mlen[i]);
}

// (A32 v)_i for the inner solve of the mixed-precision path: FP32 values,
// FP32 products and accumulation, same warp-per-row layout.  The FP32 copy
// interleaves each entry's column and value bits (one 8-byte load per
// entry), and each lane keeps four entries in flight.
template <int G = kRowG>
__device__ __forceinline__ float spmv_row_warp32(const CG& A, const int2* __restrict__ cv,
                                                 const Grp<G>& q, const float* __restrict__ v,
                                                 int i, int off, int L)
{
    const int2* __restrict__ e = cv + off;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
    int k = q.lane;
    for (; k + 3 * G < L; k += 4 * G) {
        const int2 e0 = __ldcs(e + k), e1 = __ldcs(e + k + G), e2 = __ldcs(e + k + 2 * G),
                   e3 = __ldcs(e + k + 3 * G);
        acc0 = __fmaf_rn(__int_as_float(e0.y), v[e0.x], acc0);
        acc1 = __fmaf_rn(__int_as_float(e1.y), v[e1.x], acc1);
        acc2 = __fmaf_rn(__int_as_float(e2.y), v[e2.x], acc2);
        acc3 = __fmaf_rn(__int_as_float(e3.y), v[e3.x], acc3);
    }
    for (; k + G < L; k += 2 * G) {
        const int2 e0 = __ldcs(e + k), e1 = __ldcs(e + k + G);
        acc0 = __fmaf_rn(__int_as_float(e0.y), v[e0.x], acc0);
        acc1 = __fmaf_rn(__int_as_float(e1.y), v[e1.x], acc1);
    }
    if (k < L) {
        const int2 e0 = __ldcs(e + k);
        acc2 = __fmaf_rn(__int_as_float(e0.y), v[e0.x], acc2);
    }
    float acc = q.sumf((acc0 + acc1) + (acc2 + acc3));
    return __fmaf_rn((float)A.diag[i], v[i], acc);
}

// r = b - A x, z = M^-1 r, p = z; partials of b.b, r.z, r.r
// 8 resident blocks per SM (32 registers): the grid is 8 blocks per SM and
// every block must be resident, or a second wave doubles the time
template <int G>
__global__ void __launch_bounds__(256, 8) k_cg_start(CG A, const double* __restrict__ b, const double* __restrict__ x,
                           double* __restrict__ r, double* __restrict__ zv, double* __restrict__ p,
                           double* __restrict__ part)
{
    __shared__ double sh[33];
    Grp<G> q;
    const long nwarps = (long)gridDim.x * blockDim.x / G;
    double bb = 0, rz = 0, rr = 0;
    for (long w = q.gid; w < A.n; w += nwarps) {
        int i = (int)w;
        double ri = 0, zi = 0;
        if (A.bcon[i] == 0) {
            double bi = b[i];
            ri = A.x0_zero ? bi : bi - spmv_row_warp(A, q, x, i);
            zi = A.precond ? ri / A.diag[i] : ri;
            if (q.lane == 0) {
                bb += bi * bi;
                rz += ri * zi;
                rr += ri * ri;
            }
        }
        if (q.lane == 0) {
            r[i] = ri;
            zv[i] = zi;
            p[i] = zi;
        }
    }
    bb = block_sum(bb, sh);
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bb;
        part[A.nparts + blockIdx.x] = rz;
        part[2 * A.nparts + blockIdx.x] = rr;
    }
}

// The same start when the assembly has already formed r = b - A x0 (in r):
// z = M^-1 r, p = z and the partials b.b, r.z, r.r, one thread per row; rows
// outside the system get r = z = p = 0 and Dirichlet rows their pressure 0
// (the assembly left the guess untouched for its neighbours to read).
__global__ void __launch_bounds__(256, 8) k_cg_start_rows(CG A, const double* __restrict__ b,
                                                          const int* __restrict__ bcon,
                                                          double* __restrict__ x,
                                                          double* __restrict__ r,
                                                          double* __restrict__ zv,
                                                          double* __restrict__ p,
                                                          double* __restrict__ part)
{
    __shared__ double sh[33];
    double bb = 0, rz = 0, rr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        double ri = 0, zi = 0;
        if (A.bcon[i] == 0) {
            const double bi = b[i];
            ri = r[i];
            zi = A.precond ? ri / A.diag[i] : ri;
            bb += bi * bi;
            rz += ri * zi;
            rr += ri * ri;
        } else {
            r[i] = 0.0;
            if (bcon[i] != 0) x[i] = 0.0;
        }
        zv[i] = zi;
        p[i] = zi;
    }
    bb = block_sum(bb, sh);
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bb;
        part[A.nparts + blockIdx.x] = rz;
        part[2 * A.nparts + blockIdx.x] = rr;
    }
}

__global__ void k_cg_start_scalars(int nparts, const double* __restrict__ part, double tol2,
                                   double* scal, int* flag, int use_cond,
                                   cudaGraphConditionalHandle cond)
{
    __shared__ double sh[33];
    double bb = reduce_parts(part, nparts, sh);
    double rz = reduce_parts(part + nparts, nparts, sh);
    double rr = reduce_parts(part + 2 * nparts, nparts, sh);
    if (threadIdx.x == 0) {
        scal[S_BB] = bb;
        scal[S_RZ] = rz;
        scal[S_RR] = rr;
        scal[S_RR0] = rr;
        scal[S_ZERO] = (bb == 0.0) ? 1.0 : 0.0;
        flag[0] = (bb == 0.0 || rr <= tol2 * bb) ? 1 : 0;
        flag[1] = 0;
        // inside a CUDA graph the CG loop is a while node on this value
        if (use_cond) cudaGraphSetConditional(cond, flag[0] ? 0u : 1u);
    }
}

// s = A p and partial p.s; G lanes per row (a whole warp, or half of one
// for the systems of up to kNarrowMaxRows rows)
template <int G>
__global__ void k_cg_spmv(CG A, const double* __restrict__ p, double* __restrict__ s,
                          double* __restrict__ part, const int* __restrict__ flag)
{
    __shared__ double sh[33];
    if (flag[0]) return;
    Grp<G> q;
    const long nwarps = (long)gridDim.x * blockDim.x / G;
    double ps = 0;
    // one 8-byte load of (offset, length) per row; length -1 marks rows
    // outside the system (measured 0.569 against 0.574 ms per launch with
    // bcon, mlen and moff read separately; prefetching the next row's pair
    // costs 0.64 ms)
    for (long w = q.gid; w < A.n; w += nwarps) {
        int i = (int)w;
        const int2 m = A.mrow[i];
        double si = 0;
        if (m.y >= 0) {
            si = spmv_row(A, q, p, i, m.x, m.y);
            if (q.lane == 0) ps += p[i] * si;
        }
        if (q.lane == 0) s[i] = si;
    }
    ps = block_sum(ps, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = ps;
}

// alpha = rz / p.s; x += alpha p; r -= alpha s; z = M^-1 r; partials r.z, r.r
__global__ void __launch_bounds__(256, 8) k_cg_update(CG A, double* __restrict__ x, double* __restrict__ r,
                            double* __restrict__ zv, const double* __restrict__ p,
                            const double* __restrict__ s, const double* __restrict__ part_ps,
                            double* __restrict__ part, const double* __restrict__ scal,
                            const int* __restrict__ flag)
{
    __shared__ double sh[33];
    if (flag[0]) return;
    double ps = reduce_parts(part_ps, A.nparts, sh);
    double alpha = scal[S_RZ] / ps;
    double rz = 0, rr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        if (A.bcon[i] != 0) continue;
        double xi = x[i] + alpha * p[i];
        double ri = r[i] - alpha * s[i];
        double zi = A.precond ? ri / A.diag[i] : ri;
        x[i] = xi;
        r[i] = ri;
        zv[i] = zi;
        rz += ri * zi;
        rr += ri * ri;
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = rz;
        part[A.nparts + blockIdx.x] = rr;
    }
}

// beta = rz'/rz; p = z + beta p.  Every block reaches the same decision from
// the same partials; block 0 stages rz', r.r and the decision for k_cg_commit
// (nothing read by this kernel is written by it).
__global__ void k_cg_direction(CG A, const double* __restrict__ zv, double* __restrict__ p,
                               const double* __restrict__ part, double* scal,
                               const int* __restrict__ flag, double tol2, int maxit,
                               int nscenes, const int* __restrict__ sok)
{
    __shared__ double sh[33];
    if (flag[0]) return;
    double rz = reduce_parts(part, A.nparts, sh);
    double rr = reduce_parts(part + A.nparts, A.nparts, sh);
    double beta = rz / scal[S_RZ];
    int it = flag[1] + 1;
    bool conv = rr <= tol2 * scal[S_BB];
    if (nscenes > 1) {  // every scene to its own relative residual
        conv = true;
        for (int k = 0; k < nscenes; k++) conv = conv && (sok[k] != 0);
    }
    bool done = conv || it >= maxit || !(rr == rr);
    if (!done) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x)
            if (A.bcon[i] == 0) p[i] = zv[i] + beta * p[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scal[S_NEWRZ] = rz;
        scal[S_NEWRR] = rr;
        scal[S_DONE] = done ? 1.0 : 0.0;
    }
}

// Batched scenes: per-scene sums over each scene's slot range (one block per
// scene, fixed order).  mode 0: b.b -> sbb; mode 1: r.r -> srr and the
// scene's converged flag sok = (r.r <= tol2 * b.b).
__global__ void k_scene_sums(int mode, const int* __restrict__ first, const int* __restrict__ last,
                             const int* __restrict__ scene, const int* __restrict__ bcon,
                             const double* __restrict__ v, double tol2, double* __restrict__ sbb,
                             double* __restrict__ srr, int* __restrict__ sok,
                             const int* __restrict__ flag)
{
    __shared__ double sh[33];
    if (flag && flag[0]) return;
    if (mode == 2 && flag[2] != 1) return;  // mixed precision: refinements only
    int k = blockIdx.x;
    double acc = 0.0;
    for (int i = first[k] + threadIdx.x; i < last[k]; i += blockDim.x)
        if (scene[i] == k && bcon[i] == 0) acc += v[i] * v[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) {
        if (mode == 0) {
            sbb[k] = acc;
        } else {
            srr[k] = acc;
            sok[k] = (sbb[k] == 0.0 || acc <= tol2 * sbb[k]) ? 1 : 0;
        }
    }
}

__global__ void k_invert(int n, const int* __restrict__ oid, int* __restrict__ inv_id)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv_id[oid[i]] = i;
}

// commits the iteration; inside a graph it also sets the while-node
// condition (the iteration cap in k_cg_direction bounds the loop)
__global__ void k_cg_commit(double* scal, int* flag, int use_cond,
                            cudaGraphConditionalHandle cond)
{
    if (!flag[0]) {
        scal[S_RZ] = scal[S_NEWRZ];
        scal[S_RR] = scal[S_NEWRR];
        flag[1] += 1;
        if (scal[S_DONE] != 0.0) flag[0] = 1;
    }
    if (use_cond) cudaGraphSetConditional(cond, flag[0] ? 0u : 1u);
}

// Grid-wide barrier of k_cg_loop (a cooperative launch: every block is
// resident).  Thread 0 of each block adds its arrival to a counter that
// grows by the grid size per barrier and waits for the count of this
// barrier, at most kBarSpins polls (about a second); past that it sets
// MPS_ERR_NOT_CONVERGED and the block reports failure, so a lost block ends
// the solve instead of hanging the GPU.
constexpr long kBarSpins = 1L << 24;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& target, unsigned* err,
                                             int* sh_ok)
{
    __syncthreads();
    target += gridDim.x;
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(bar, 1u);
        long spins = 0;
        while (ld_acquire_u32(bar) < target) {
            if (++spins > kBarSpins) {
                set_error(err, MPS_ERR_NOT_CONVERGED);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        *sh_ok = ok;
    }
    __syncthreads();
    return *sh_ok != 0;
}

// The whole Jacobi-PCG loop in one cooperative launch, for systems small
// enough that the loop's launches, not its bytes, set the time: each
// iteration runs k_cg_spmv, k_cg_update, k_cg_direction and k_cg_commit's
// work in that order with a grid barrier between them, over the same grid
// and the same fixed-order block partials, so it takes the same steps with
// the same bits as the four kernels.  The iteration state (r.z, the count)
// lives in registers, identical in every block; block 0 commits it at the
// end.  The barrier counter is zeroed before the launch.
template <int G>
__global__ void __launch_bounds__(kRedThreads) k_cg_loop(CG A, double* __restrict__ x,
        double* __restrict__ r, double* __restrict__ zv, double* __restrict__ p,
        double* __restrict__ s, double* __restrict__ part, double* scal, int* flag, double tol2,
        int maxit, unsigned* bar, unsigned* err)
{
    __shared__ double sh[33];
    __shared__ int sh_ok;
    if (flag[0]) return;
    Grp<G> q;
    const long nwarps = (long)gridDim.x * blockDim.x / G;
    const int np = A.nparts;
    double* part_ps = part + 4 * np;
    const double bb = scal[S_BB];
    double rz_old = scal[S_RZ];
    int it = flag[1];
    unsigned target = 0;
    for (;;) {
        // s = A p, partial p.s (k_cg_spmv)
        double ps = 0;
        for (long w = q.gid; w < A.n; w += nwarps) {
            const int i = (int)w;
            const int2 m = A.mrow[i];
            double si = 0;
            if (m.y >= 0) {
                si = spmv_row(A, q, p, i, m.x, m.y);
                if (q.lane == 0) ps += p[i] * si;
            }
            if (q.lane == 0) s[i] = si;
        }
        ps = block_sum(ps, sh);
        if (threadIdx.x == 0) part_ps[blockIdx.x] = ps;
        if (!grid_barrier(bar, target, err, &sh_ok)) return;
        // x += alpha p, r -= alpha s, z = M^-1 r, partials r.z, r.r (k_cg_update)
        const double alpha = rz_old / reduce_parts(part_ps, np, sh);
        double rz = 0, rr = 0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
            if (A.bcon[i] != 0) continue;
            const double xi = x[i] + alpha * p[i];
            const double ri = r[i] - alpha * s[i];
            const double zi = A.precond ? ri / A.diag[i] : ri;
            x[i] = xi;
            r[i] = ri;
            zv[i] = zi;
            rz += ri * zi;
            rr += ri * ri;
        }
        rz = block_sum(rz, sh);
        rr = block_sum(rr, sh);
        if (threadIdx.x == 0) {
            part[blockIdx.x] = rz;
            part[np + blockIdx.x] = rr;
        }
        if (!grid_barrier(bar, target, err, &sh_ok)) return;
        // beta, the stop test, p = z + beta p (k_cg_direction, k_cg_commit)
        const double rzn = reduce_parts(part, np, sh);
        const double rrn = reduce_parts(part + np, np, sh);
        const double beta = rzn / rz_old;
        it++;
        const bool done = rrn <= tol2 * bb || it >= maxit || !(rrn == rrn);
        if (!done) {
            for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n;
                 i += gridDim.x * blockDim.x)
                if (A.bcon[i] == 0) p[i] = zv[i] + beta * p[i];
        }
        rz_old = rzn;
        if (done) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                scal[S_RZ] = rzn;
                scal[S_RR] = rrn;
                flag[1] = it;
                flag[0] = 1;
            }
            return;
        }
        if (!grid_barrier(bar, target, err, &sh_ok)) return;
    }
}

// worst relative residual over batched scenes -> scal[S_WORST]
__global__ void k_scene_worst(int nscenes, const double* __restrict__ sbb,
                              const double* __restrict__ srr, double* scal)
{
    if (threadIdx.x != 0) return;
    double worst = 0.0;
    for (int k = 0; k < nscenes; k++)
        if (sbb[k] > 0) worst = fmax(worst, sqrt(srr[k] / sbb[k]));
    scal[S_WORST] = worst;
}

// clamp (functions.cu:2534-2547); a zero right-hand side gives p = 0
__global__ void k_clamp(int n, double pmin, double pmax, const double* __restrict__ scal,
                        double* __restrict__ pnew, const int* __restrict__ scene,
                        const double* __restrict__ spmax, const double* __restrict__ sbb)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = scal[S_ZERO] != 0.0 ? 0.0 : pnew[i];
    if (scene) {  // batched: the scene's own cap, zero where its right-hand side is zero
        int k = scene[i];
        pmax = spmax[k];
        if (sbb[k] == 0.0) v = 0.0;
    }
    if (v < pmin) v = pmin;
    if (v > pmax || v * 0.0 != 0.0) v = pmax;
    pnew[i] = v;
}


// ---------------------------------------------------------------------------
// Mixed precision (precision 1): iterative refinement.  The outer loop keeps
// x and r = b - A x in FP64 (r is updated as r -= A64 d with the FP64 matrix,
// so its accuracy is FP64's); each sweep solves A32 d = r approximately by
// Jacobi-PCG in FP32 (FP32 matrix copy, FP32 vectors, FP32 SpMV sums) with
// FP64 dot products, until the inner residual has fallen by the sweep's
// target factor.  The stop test is the FP64 one: ||r||/||b|| <= cg_tol.
//
// Both loops are one device state machine so that the graph's single while
// node (or the eager host loop) drives them: flag[2] = 0 runs an inner CG
// iteration, flag[2] = 1 runs a refinement; flag[1] counts inner iterations
// and flag[3] refinements.
struct IR {
    const int2* __restrict__ cv;    // FP32 copy of the CSR: (column, value bits)
    float* __restrict__ d;          // correction of this sweep
    float* __restrict__ r;          // inner residual
    float* __restrict__ z;
    float* __restrict__ p;
    float* __restrict__ s;
};

constexpr int kMaxSweeps = 40;  // refinement sweeps per solve (bound)

__host__ __device__ __forceinline__ double sweep_target(double tol2, double bb, double rr)
{
    // reduce the inner residual by what the FP64 test still needs (with a
    // factor 2 margin), at least 10x and at most to 1e-5 (FP32's floor)
    double e = rr > 0 ? 0.25 * tol2 * bb / rr : 1e-10;
    return fmin(1e-2, fmax(1e-10, e));
}

// r64 = b - A64 x; r32 = r64; z = M^-1 r32; p = z; d = 0; partials b.b,
// r32.z, r64.r64, r32.r32
__global__ void k_ir_start(CG A, IR I, const double* __restrict__ b, const double* __restrict__ x,
                           double* __restrict__ r64, double* __restrict__ part)
{
    __shared__ double sh[33];
    Grp<kRowG> q;
    const long nwarps = (long)gridDim.x * blockDim.x / kRowG;
    double bb = 0, rz = 0, rr = 0, rin = 0;
    for (long w = q.gid; w < A.n; w += nwarps) {
        int i = (int)w;
        double ri = 0;
        float r32 = 0.f, z32 = 0.f;
        if (A.bcon[i] == 0) {
            double bi = b[i];
            ri = A.x0_zero ? bi : bi - spmv_row_warp(A, q, x, i);
            r32 = (float)ri;
            z32 = A.precond ? r32 / (float)A.diag[i] : r32;
            if (q.lane == 0) {
                bb += bi * bi;
                rr += ri * ri;
                rz += (double)r32 * (double)z32;
                rin += (double)r32 * (double)r32;
            }
        }
        if (q.lane == 0) {
            r64[i] = ri;
            I.r[i] = r32;
            I.z[i] = z32;
            I.p[i] = z32;
            I.d[i] = 0.f;
            I.s[i] = 0.f;
        }
    }
    bb = block_sum(bb, sh);
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    rin = block_sum(rin, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bb;
        part[A.nparts + blockIdx.x] = rz;
        part[2 * A.nparts + blockIdx.x] = rr;
        part[3 * A.nparts + blockIdx.x] = rin;
    }
}

// The same start when the assembly has already formed r64 = b - A64 x (in
// r64): one thread per row; rows outside the system get zeros and
// Dirichlet rows their pressure 0 (the assembly left the guess untouched
// for its neighbours to read).
__global__ void __launch_bounds__(256, 8) k_ir_start_rows(CG A, IR I, const double* __restrict__ b,
                                                          const int* __restrict__ bcon,
                                                          double* __restrict__ x,
                                                          double* __restrict__ r64,
                                                          double* __restrict__ part)
{
    __shared__ double sh[33];
    double bb = 0, rz = 0, rr = 0, rin = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        float r32 = 0.f, z32 = 0.f;
        if (A.bcon[i] == 0) {
            const double bi = b[i], ri = r64[i];
            r32 = (float)ri;
            z32 = A.precond ? r32 / (float)A.diag[i] : r32;
            bb += bi * bi;
            rr += ri * ri;
            rz += (double)r32 * (double)z32;
            rin += (double)r32 * (double)r32;
        } else {
            r64[i] = 0.0;
            if (bcon[i] != 0) x[i] = 0.0;
        }
        I.r[i] = r32;
        I.z[i] = z32;
        I.p[i] = z32;
        I.d[i] = 0.f;
        I.s[i] = 0.f;
    }
    bb = block_sum(bb, sh);
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    rin = block_sum(rin, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bb;
        part[A.nparts + blockIdx.x] = rz;
        part[2 * A.nparts + blockIdx.x] = rr;
        part[3 * A.nparts + blockIdx.x] = rin;
    }
}

__global__ void k_ir_start_scalars(int nparts, const double* __restrict__ part, double tol2,
                                   double* scal, int* flag, int use_cond,
                                   cudaGraphConditionalHandle cond)
{
    __shared__ double sh[33];
    double bb = reduce_parts(part, nparts, sh);
    double rz = reduce_parts(part + nparts, nparts, sh);
    double rr = reduce_parts(part + 2 * nparts, nparts, sh);
    double rin = reduce_parts(part + 3 * nparts, nparts, sh);
    if (threadIdx.x == 0) {
        scal[S_BB] = bb;
        scal[S_RZ] = rz;
        scal[S_RR] = rr;
        scal[S_RR0] = rr;
        scal[S_RIN] = rin;
        scal[S_RIN0] = rin;
        scal[S_ETA2] = sweep_target(tol2, bb, rr);
        scal[S_ZERO] = (bb == 0.0) ? 1.0 : 0.0;
        flag[0] = (bb == 0.0 || rr <= tol2 * bb) ? 1 : 0;
        flag[1] = 0;
        flag[2] = 0;
        flag[3] = 0;
        if (use_cond) cudaGraphSetConditional(cond, flag[0] ? 0u : 1u);
    }
}

// inner: s = A32 p, partial p.s.  refinement: r64 -= A64 d, x += d, partial
// r64.r64 (each row writes only its own x and r; d is read-only here)
__global__ void k_ir_spmv(CG A, IR I, double* __restrict__ r64, double* __restrict__ x,
                          double* __restrict__ part, const int* __restrict__ flag)
{
    __shared__ double sh[33];
    if (flag[0]) return;
    const int phase = flag[2];
    Grp<kIrG> q;
    const long nwarps = (long)gridDim.x * blockDim.x / kIrG;
    double acc = 0;
    for (long w = q.gid; w < A.n; w += nwarps) {
        int i = (int)w;
        const int2 m = A.mrow[i];  // (offset, length); length -1: outside the system
        if (m.y < 0) {
            if (phase == 0 && q.lane == 0) I.s[i] = 0.f;
            continue;
        }
        if (phase == 0) {
            float si = spmv_row_warp32(A, I.cv, q, I.p, i, m.x, m.y);
            if (q.lane == 0) {
                I.s[i] = si;
                acc += (double)I.p[i] * (double)si;
            }
        } else {
            double t = spmv_row(A, q, I.d, i, m.x, m.y);
            if (q.lane == 0) {
                double ri = r64[i] - t;
                r64[i] = ri;
                x[i] = x[i] + (double)I.d[i];
                acc += ri * ri;
            }
        }
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// inner: alpha = rz / p.s; d += alpha p; r -= alpha s.  refinement: r32 =
// r64, d = 0.  Then z = M^-1 r32 and partials r32.z, r32.r32 (FP64 sums).
__global__ void k_ir_update(CG A, IR I, const double* __restrict__ r64,
                            const double* __restrict__ part_ps, double* __restrict__ part,
                            const double* __restrict__ scal, const int* __restrict__ flag)
{
    __shared__ double sh[33];
    if (flag[0]) return;
    const int phase = flag[2];
    float alpha = 0.f;
    if (phase == 0) {
        double ps = reduce_parts(part_ps, A.nparts, sh);
        alpha = (float)(scal[S_RZ] / ps);
    }
    double rz = 0, rin = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        if (A.bcon[i] != 0) continue;
        float ri;
        if (phase == 0) {
            I.d[i] = I.d[i] + alpha * I.p[i];
            ri = I.r[i] - alpha * I.s[i];
        } else {
            I.d[i] = 0.f;
            ri = (float)r64[i];
        }
        float zi = A.precond ? ri / (float)A.diag[i] : ri;
        I.r[i] = ri;
        I.z[i] = zi;
        rz += (double)ri * (double)zi;
        rin += (double)ri * (double)ri;
    }
    rz = block_sum(rz, sh);
    rin = block_sum(rin, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = rz;
        part[A.nparts + blockIdx.x] = rin;
    }
}

// inner: beta = rz'/rz, p = z + beta p unless the sweep ends.  refinement:
// the FP64 stop test (per scene when batched); p = z starts the next sweep.
__global__ void k_ir_direction(CG A, IR I, const double* __restrict__ part,
                               const double* __restrict__ part_rr, double* scal,
                               const int* __restrict__ flag, double tol2, int maxit, int nscenes,
                               const int* __restrict__ sok)
{
    __shared__ double sh[33];
    if (flag[0]) return;
    const int phase = flag[2];
    double rz = reduce_parts(part, A.nparts, sh);
    double rin = reduce_parts(part + A.nparts, A.nparts, sh);
    bool restart = false, indone = false, done = false;
    double rr = 0, beta = 0;
    if (phase == 0) {
        beta = rz / scal[S_RZ];
        int it = flag[1] + 1;
        indone = rin <= scal[S_ETA2] * scal[S_RIN0] || it >= maxit || !(rin == rin);
    } else {
        rr = reduce_parts(part_rr, A.nparts, sh);
        bool conv = rr <= tol2 * scal[S_BB];
        if (nscenes > 1) {
            conv = true;
            for (int k = 0; k < nscenes; k++) conv = conv && (sok[k] != 0);
        }
        done = conv || flag[1] >= maxit || flag[3] + 1 >= kMaxSweeps || !(rr == rr);
        restart = !done;
    }
    if ((phase == 0 && !indone) || restart) {
        const float b32 = (float)beta;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x)
            if (A.bcon[i] == 0) I.p[i] = restart ? I.z[i] : I.z[i] + b32 * I.p[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scal[S_NEWRZ] = rz;
        scal[S_NEWRIN] = rin;
        scal[S_INDONE] = indone ? 1.0 : 0.0;
        if (phase == 1) {
            scal[S_NEWRR] = rr;
            scal[S_DONE] = done ? 1.0 : 0.0;
        }
    }
}

__global__ void k_ir_commit(double* scal, int* flag, double tol2, int use_cond,
                            cudaGraphConditionalHandle cond)
{
    if (!flag[0]) {
        scal[S_RZ] = scal[S_NEWRZ];
        scal[S_RIN] = scal[S_NEWRIN];
        if (flag[2] == 0) {
            flag[1] += 1;
            if (scal[S_INDONE] != 0.0) flag[2] = 1;
        } else {
            scal[S_RR] = scal[S_NEWRR];
            scal[S_RIN0] = scal[S_NEWRIN];
            scal[S_ETA2] = sweep_target(tol2, scal[S_BB], scal[S_RR]);
            flag[3] += 1;
            flag[2] = 0;
            if (scal[S_DONE] != 0.0) flag[0] = 1;
        }
    }
    if (use_cond) cudaGraphSetConditional(cond, flag[0] ? 0u : 1u);
}

// y = A x on the unknown rows (0 elsewhere), with the last assembled matrix
__global__ void k_apply(CG A, const double* __restrict__ x, double* __restrict__ y)
{
    Grp<kRowG> q;
    const long nwarps = (long)gridDim.x * blockDim.x / kRowG;
    for (long w = q.gid; w < A.n; w += nwarps) {
        const int i = (int)w;
        double yi = 0.0;
        if (A.bcon[i] == 0) yi = spmv_row_warp(A, q, x, i);
        if (q.lane == 0) y[i] = yi;
    }
}

}  // namespace

// y = A x with the matrix of the last PPE (used to train the learned guess
// on the residual it leaves)
int vmps_ppe_apply(mps_ctx* c, const double* x, double* y)
{
    int sms = 0;
    VMPS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    CG G{c->mcol, c->mval, c->mlen, c->moff, c->diag, c->sysmask, c->cap_l, c->n, 0, 0, 0, c->mrow};
    k_apply<<<sms * 8, kRedThreads, 0, c->stream>>>(G, x, y);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

// PRESSURECALC's assembly part (MATRIX, source, initial guess); the solve
// follows in vmps_ppe or, for a scene split between contexts, in the
// host-driven CG entry points below.  *warm_out: the initial guess used
// (0: zero, the start kernels then skip the product).
static int ppe_assemble(mps_ctx* c, int* warm_out, double* r0 = nullptr, bool* fused = nullptr)
{
    const mps_config& f = c->cfg;
    cudaStream_t st = c->stream;
    const int n = c->n;
    const double *ax = c->x, *ay = c->y, *az = c->z, *nsrc = c->nd;
    const double4* P4 = c->P4;
    if (f.ppe_at_predicted) { ax = c->xs; ay = c->ys; az = c->zs; nsrc = c->nds; P4 = c->P4s; }
    Asm A;
    A.wk = make_wk(f.ktype, f.re_l);
    A.cw = 2.0 * f.dim / c->lambda_l / c->n0_l / f.rho1;
    A.cm = ((f.dim == 2) ? 3.0 * f.re_l : 2.0 * f.re_l) / c->n0_l / f.rho1;
    A.reg = (1.00e-7) / f.dt / f.dt;
    A.tiny2 = sqrt_cut(1.0e-15, false);
    A.n0_s = c->n0_s;
    A.dt = f.dt;
    A.matopt = f.matopt;
    A.srcopt = f.srcopt;
    // learned initial guess: the network's prediction replaces the previous
    // pressure (features are captured for training whenever a network exists)
    int warm = f.warm_start;
    if (c->gnn) {
        int r = vmps_gnn_guess(c);
        if (r != MPS_OK) return r;
        if (vmps_gnn_in_use(c)) warm = 1;
    }
    // CSR row offsets: exclusive scan of the Laplacian list lengths (each
    // row's non-zeros are a subset of its list)
    {
        int r = vmps_scan(c, n, c->len_l, c->moff);
        if (r != MPS_OK) return r;
    }
    // CG's starting residual in the same pass: a guess the pass does not
    // change (the previous pressure or the network's) and a source known
    // per row (not the sequential HS + ECS recurrence)
    if (fused) *fused = r0 && warm == 1 && !f.srcopt;
    if (!fused || !*fused) r0 = nullptr;
    const int wblocks = (int)(((long)n * kAsmG + kBlock - 1) / kBlock);
    // the predicted positions carry bcon in their w slot when BCON ran after
    // the last PREDICTION (always within a step; the per-stage entry points
    // may be called out of order)
    int w_bcon = (f.ppe_at_predicted && c->p4s_bcon) ? 1 : 0;
    if (r0 && f.ppe_at_predicted) {
        // with the residual formed here every kept column also needs its
        // guess: the w slot carries it for the unknowns and a coded NaN for
        // the other kinds, so one gather brings position, status and guess
        k_pack_wguess<<<grid_blocks(n), kBlock, 0, st>>>(n, c->bcon, c->pnew, c->P4s);
        vmps_count_launch(1);
        w_bcon = 2;
        c->p4s_bcon = false;  // the w slot no longer holds bcon alone
    }
    if (f.dim == 3)
        k_assemble<3><<<wblocks, kBlock, 0, st>>>(n, c->cap_l, A, c->nbr_l, c->len_l, c->bcon, P4,
                                                  nsrc, warm, c->pnew, c->pold, c->moff, c->mcol,
                                                  c->mval, c->mcv32, c->mlen, c->diag, c->source,
                                                  w_bcon, c->mrow, c->own, c->sysmask, r0);
    else
        k_assemble<2><<<wblocks, kBlock, 0, st>>>(n, c->cap_l, A, c->nbr_l, c->len_l, c->bcon, P4,
                                                  nsrc, warm, c->pnew, c->pold, c->moff, c->mcol,
                                                  c->mval, c->mcv32, c->mlen, c->diag, c->source,
                                                  w_bcon, c->mrow, c->own, c->sysmask, r0);
    vmps_count_launch(1);
    if (f.srcopt) {
        // slot of particle id k: inv_id[k] (the sort's inv buffer is free here)
        k_invert<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, c->inv);
        vmps_count_launch(1);
        if (f.dim == 3)
            k_source_hs<3><<<1, 32, 0, st>>>(n, c->cap_s, f.re_s, c->n0_s, f.dt, c->inv, c->nbr_s,
                                             c->len_s, c->bcon, c->ptype, c->nds, ax, ay, az, c->us,
                                             c->vs, c->ws, c->source);
        else
            k_source_hs<2><<<1, 32, 0, st>>>(n, c->cap_s, f.re_s, c->n0_s, f.dt, c->inv, c->nbr_s,
                                             c->len_s, c->bcon, c->ptype, c->nds, ax, ay, az, c->us,
                                             c->vs, c->ws, c->source);
        vmps_count_launch(1);
    }
    *warm_out = warm;
    return MPS_OK;
}

// grid of the CG kernels: blocks per SM from the autotuner, else as many as
// fit (at most 8); cg_part holds [0,3*nblk) start/update partials and
// [4*nblk,5*nblk) p.s
// Systems of at most this many rows solve in k_cg_loop (FP64, one scene):
// there the four launches per iteration and their gaps, not the bytes, set
// the iteration's time.  Measured: the 2D dam of 1,928 particles 0.272
// against 0.352 ms per step; the 86,118-particle two-phase scene 2.77
// against 2.28 ms (three grid barriers per iteration over 592 blocks cost
// more than the graph's kernel boundaries), the 1.6 M dam 27.1 against 20.3.
constexpr int kLoopMaxRows = 16384;

static bool use_cg_loop(mps_ctx* c)
{
    if (c->cfg.precision >= 1 || c->nscenes > 1 || c->n > kLoopMaxRows) return false;
    int coop = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return coop != 0;
}

static int cg_grid(mps_ctx* c, int* out, bool loop = false, int g = kRowG)
{
    int nblk = 0, occ = 0;
    VMPS_CUDA(c, cudaDeviceGetAttribute(&nblk, cudaDevAttrMultiProcessorCount, c->device));
    VMPS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                     &occ, g == 16 ? k_cg_spmv<16> : k_cg_spmv<kRowG>, kRedThreads, 0));
    const int sms = nblk;
    if (loop) {  // the cooperative loop needs its whole grid resident
        int occ_loop = 0;
        VMPS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                         &occ_loop, g == 16 ? k_cg_loop<16> : k_cg_loop<kRowG>, kRedThreads, 0));
        occ = std::min(occ, occ_loop);
    }
    const int bps = c->tune_cg_bps > 0 ? c->tune_cg_bps : 8;
    nblk *= std::max(1, std::min(occ, bps));
    // the loop's barriers wait for every block: no more blocks than the
    // rows' warps need, at least one per SM
    if (loop) nblk = std::min(nblk, std::max(sms, (c->n + kRedThreads / g - 1) / (kRedThreads / g)));
    if ((size_t)5 * nblk > c->cg_part_cap) {
        c->msg = "CG partial buffer too small for the launch grid";
        return MPS_ERR_ARG;
    }
    *out = nblk;
    return MPS_OK;
}

int vmps_ppe(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    cudaStream_t st = c->stream;
    const int n = c->n;
    const bool mixed = f.precision >= 1;
    int warm = 0, nblk = 0;
    bool fused = false;
    // small systems: the loop in one cooperative launch, over a grid that
    // the four-kernel loop (profiled runs) shares, so both give the same bits
    const bool loop_grid = use_cg_loop(c);
    const bool narrow = n <= kNarrowMaxRows;  // 16 lanes per row in the FP64 products
    {
        int r = ppe_assemble(c, &warm, c->cg_r, &fused);
        if (r != MPS_OK) return r;
        r = cg_grid(c, &nblk, loop_grid, narrow ? 16 : kRowG);
        if (r != MPS_OK) return r;
    }
    // zero initial guess (the assembly zeroed pnew): r = b exactly, so the
    // start kernels skip the product A x0
    CG G{c->mcol, c->mval, c->mlen, c->moff, c->diag, c->sysmask, c->cap_l, n,
         f.solver == 1 ? 1 : 0, nblk, warm == 0 ? 1 : 0, c->mrow};
    double tol2 = f.cg_tol * f.cg_tol;
    const bool batched = c->nscenes > 1;
    // Inside a stream capture (graph mode) the loop becomes a conditional
    // while node: no host synchronisation anywhere in the solve.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaGraph_t cgraph = nullptr;
    VMPS_CUDA(c, cudaStreamGetCaptureInfo(st, &cap, nullptr, &cgraph, nullptr, nullptr));
    const bool graph = cap == cudaStreamCaptureStatusActive;
    cudaGraphConditionalHandle cond = 0;
    const bool loop = loop_grid && !c->profile;  // profiling times each SpMV launch
    if (graph && !loop)
        VMPS_CUDA(c, cudaGraphConditionalHandleCreate(&cond, cgraph, 1, cudaGraphCondAssignDefault));
    const int use_cond = graph && !loop ? 1 : 0;
    IR I{c->mcv32, c->ir_d, c->ir_r, c->ir_z, c->ir_p, c->ir_s};
    if (mixed && fused) {
        k_ir_start_rows<<<nblk, kRedThreads, 0, st>>>(G, I, c->source, c->bcon, c->pnew, c->cg_r,
                                                      c->cg_part);
        k_ir_start_scalars<<<1, kRedThreads, 0, st>>>(nblk, c->cg_part, tol2, c->cg_scal,
                                                      c->cg_flag, use_cond, cond);
    } else if (mixed) {
        k_ir_start<<<nblk, kRedThreads, 0, st>>>(G, I, c->source, c->pnew, c->cg_r, c->cg_part);
        k_ir_start_scalars<<<1, kRedThreads, 0, st>>>(nblk, c->cg_part, tol2, c->cg_scal,
                                                      c->cg_flag, use_cond, cond);
    } else if (fused) {
        k_cg_start_rows<<<nblk, kRedThreads, 0, st>>>(G, c->source, c->bcon, c->pnew, c->cg_r,
                                                      c->cg_z, c->cg_p, c->cg_part);
        k_cg_start_scalars<<<1, kRedThreads, 0, st>>>(nblk, c->cg_part, tol2, c->cg_scal,
                                                      c->cg_flag, use_cond, cond);
    } else {
        (narrow ? k_cg_start<16> : k_cg_start<kRowG>)<<<nblk, kRedThreads, 0, st>>>(
            G, c->source, c->pnew, c->cg_r, c->cg_z,
                                                 c->cg_p, c->cg_part);
        k_cg_start_scalars<<<1, kRedThreads, 0, st>>>(nblk, c->cg_part, tol2, c->cg_scal,
                                                      c->cg_flag, use_cond, cond);
    }
    vmps_count_launch(2);
    if (batched) {
        k_scene_sums<<<c->nscenes, kRedThreads, 0, st>>>(0, c->sfirst, c->slast, c->scene, c->sysmask,
                                                         c->source, tol2, c->sbb, nullptr, nullptr,
                                                         nullptr);
        vmps_count_launch(1);
    }
    // one CG iteration on stream s (profiling events only outside graphs)
    auto iteration = [&](cudaStream_t s, int k) -> int {
        if (c->profile && !graph) {
            while ((int)c->ev_spmv.size() < 2 * (k + 1)) {
                cudaEvent_t e;
                VMPS_CUDA(c, cudaEventCreate(&e));
                c->ev_spmv.push_back(e);
            }
            VMPS_CUDA(c, cudaEventRecord(c->ev_spmv[2 * k], s));
        }
        if (mixed) {
            k_ir_spmv<<<nblk, kRedThreads, 0, s>>>(G, I, c->cg_r, c->pnew, c->cg_part + 4 * nblk,
                                                   c->cg_flag);
            if (c->profile && !graph) VMPS_CUDA(c, cudaEventRecord(c->ev_spmv[2 * k + 1], s));
            if (batched)
                k_scene_sums<<<c->nscenes, kRedThreads, 0, s>>>(2, c->sfirst, c->slast, c->scene,
                                                                c->sysmask, c->cg_r, tol2, c->sbb,
                                                                c->srr, c->sok, c->cg_flag);
            k_ir_update<<<nblk, kRedThreads, 0, s>>>(G, I, c->cg_r, c->cg_part + 4 * nblk,
                                                     c->cg_part, c->cg_scal, c->cg_flag);
            k_ir_direction<<<nblk, kRedThreads, 0, s>>>(G, I, c->cg_part, c->cg_part + 4 * nblk,
                                                        c->cg_scal, c->cg_flag, tol2, f.cg_max,
                                                        c->nscenes, c->sok);
            k_ir_commit<<<1, 1, 0, s>>>(c->cg_scal, c->cg_flag, tol2, graph ? 1 : 0, cond);
            VMPS_CUDA(c, cudaGetLastError());
            return MPS_OK;
        }
        (narrow ? k_cg_spmv<16> : k_cg_spmv<kRowG>)<<<nblk, kRedThreads, 0, s>>>(
            G, c->cg_p, c->cg_s, c->cg_part + 4 * nblk,
                                               c->cg_flag);
        if (c->profile && !graph) VMPS_CUDA(c, cudaEventRecord(c->ev_spmv[2 * k + 1], s));
        k_cg_update<<<nblk, kRedThreads, 0, s>>>(G, c->pnew, c->cg_r, c->cg_z, c->cg_p, c->cg_s,
                                                 c->cg_part + 4 * nblk, c->cg_part, c->cg_scal,
                                                 c->cg_flag);
        if (batched)
            k_scene_sums<<<c->nscenes, kRedThreads, 0, s>>>(1, c->sfirst, c->slast, c->scene,
                                                            c->sysmask, c->cg_r, tol2, c->sbb,
                                                            c->srr, c->sok, c->cg_flag);
        k_cg_direction<<<nblk, kRedThreads, 0, s>>>(G, c->cg_z, c->cg_p, c->cg_part, c->cg_scal,
                                                    c->cg_flag, tol2, f.cg_max, c->nscenes,
                                                    c->sok);
        k_cg_commit<<<1, 1, 0, s>>>(c->cg_scal, c->cg_flag, use_cond, cond);
        VMPS_CUDA(c, cudaGetLastError());
        return MPS_OK;
    };
    c->cg_loop_kernels = batched ? 5 : 4;
    c->cg_nspmv = 0;
    if (loop) {
        VMPS_CUDA(c, cudaMemsetAsync(c->cg_bar, 0, sizeof(unsigned), st));
        double* xp = c->pnew;
        double *rp = c->cg_r, *zp = c->cg_z, *pp = c->cg_p, *sp = c->cg_s, *part = c->cg_part,
               *scal = c->cg_scal;
        int* flag = c->cg_flag;
        int maxit = f.cg_max;
        unsigned *bar = c->cg_bar, *err = c->d_err;
        void* args[] = {&G, &xp, &rp, &zp, &pp, &sp, &part, &scal, &flag, &tol2, &maxit, &bar, &err};
        const void* fn = narrow ? (const void*)k_cg_loop<16> : (const void*)k_cg_loop<kRowG>;
        VMPS_CUDA(c, cudaLaunchCooperativeKernel(fn, dim3(nblk),
                                                 dim3(kRedThreads), args, 0, st));
        vmps_count_launch(1);
        c->cg_loop_kernels = 0;
        c->cg_nspmv = 1;
    } else if (graph) {
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        VMPS_CUDA(c, cudaStreamGetCaptureInfo(st, &cap, nullptr, &cgraph, &deps, &ndeps));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = cond;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        VMPS_CUDA(c, cudaGraphAddNode(&node, cgraph, deps, ndeps, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        VMPS_CUDA(c, cudaStreamUpdateCaptureDependencies(st, &node, 1,
                                                         cudaStreamSetCaptureDependencies));
        if (!c->stream2)
            VMPS_CUDA(c, cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking));
        VMPS_CUDA(c, cudaStreamBeginCaptureToGraph(c->stream2, body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeRelaxed));
        int r = iteration(c->stream2, 0);
        cudaGraph_t done_body = nullptr;
        VMPS_CUDA(c, cudaStreamEndCapture(c->stream2, &done_body));
        if (r != MPS_OK) return r;
    } else {
        const int check = 4;
        // the mixed path's body alternates inner iterations and refinements
        const int bound = mixed ? f.cg_max + kMaxSweeps : f.cg_max;
        for (int it = 0; it < bound; it++) {
            int r = iteration(st, it);
            if (r != MPS_OK) return r;
            vmps_count_launch(c->cg_loop_kernels);
            c->cg_nspmv++;
            if ((it + 1) % check == 0 || it + 1 == bound) {
                VMPS_CUDA(c, cudaMemcpyAsync(c->cg_flag_host, c->cg_flag, 4 * sizeof(int),
                                             cudaMemcpyDeviceToHost, st));
                VMPS_CUDA(c, cudaStreamSynchronize(st));
                if (c->cg_flag_host[0]) break;
            }
        }
    }
    if (batched) {
        k_scene_worst<<<1, 32, 0, st>>>(c->nscenes, c->sbb, c->srr, c->cg_scal);
        vmps_count_launch(1);
    }
    k_clamp<<<grid_blocks(n), kBlock, 0, st>>>(n, f.pmin, f.pmax, c->cg_scal, c->pnew,
                                               batched ? c->scene : nullptr, c->spmax, c->sbb);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaMemcpyAsync(c->cg_flag_host, c->cg_flag, 4 * sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
    VMPS_CUDA(c, cudaMemcpyAsync(c->red_host, c->cg_scal, S_COUNT * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    VMPS_CUDA(c, cudaGetLastError());
    c->ppe_pending = true;
    return MPS_OK;
}

// After the stream has been synchronised: iteration count, residual, status.
int vmps_ppe_finish(mps_ctx* c)
{
    if (!c->ppe_pending) return MPS_OK;
    c->ppe_pending = false;
    const mps_config& f = c->cfg;
    c->cg_iters = c->cg_flag_host[1];
    c->cg_outer = f.precision >= 1 ? c->cg_flag_host[3] : 0;
    if (c->profile) {
        // launches after convergence exit at once: count the working ones
        const int working = c->cg_iters + c->cg_outer;
        for (int k = 0; k < c->cg_nspmv && k < working; k++) {
            float ms = 0;
            VMPS_CUDA(c, cudaEventElapsedTime(&ms, c->ev_spmv[2 * k], c->ev_spmv[2 * k + 1]));
            c->spmv_ms += ms;
            c->spmv_launches++;
        }
    }
    double bb = c->red_host[S_BB], rr = c->red_host[S_RR];
    c->cg_relres = bb > 0 ? sqrt(rr / bb) : 0.0;
    c->cg_r0 = bb > 0 ? sqrt(c->red_host[S_RR0] / bb) : 0.0;
    if (c->nscenes > 1) c->cg_relres = c->red_host[S_WORST];
    if (!(c->cg_relres <= f.cg_tol)) c->host_err |= MPS_ERR_NOT_CONVERGED;
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

// ---------------------------------------------------------------------------
// Host-driven Jacobi-PCG over this context's rows, for a scene split between
// contexts (slab decomposition, voxarmps_b200/slab.py).  Each entry point
// runs one part of an iteration on the rows this context owns and returns
// the rank-local sums it formed (fixed-order block partials, then a fixed
// order over the blocks); the caller adds them over the ranks, forms alpha
// and beta, and between the calls exchanges the ghost entries of the CG
// vectors (mps_get_rows / mps_set_rows on "pnew" and "cg_p").  With one
// context the sequence reproduces vmps_ppe's FP64 Jacobi-PCG.
namespace {

__global__ void k_local_sums(int nparts, int count, const double* __restrict__ part,
                             double* __restrict__ out)
{
    __shared__ double sh[33];
    for (int k = 0; k < count; k++) {
        const double v = reduce_parts(part + (size_t)k * nparts, nparts, sh);
        if (threadIdx.x == 0) out[k] = v;
    }
}

// x += alpha p; r -= alpha s; z = M^-1 r; partials r.z, r.r (rows of this context)
__global__ void __launch_bounds__(256, 8) k_dcg_update(CG A, double alpha, double* __restrict__ x,
                                                       double* __restrict__ r,
                                                       double* __restrict__ zv,
                                                       const double* __restrict__ p,
                                                       const double* __restrict__ s,
                                                       double* __restrict__ part)
{
    __shared__ double sh[33];
    double rz = 0, rr = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        if (A.bcon[i] != 0) continue;
        const double xi = x[i] + alpha * p[i];
        const double ri = r[i] - alpha * s[i];
        const double zi = A.precond ? ri / A.diag[i] : ri;
        x[i] = xi;
        r[i] = ri;
        zv[i] = zi;
        rz += ri * zi;
        rr += ri * ri;
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = rz;
        part[A.nparts + blockIdx.x] = rr;
    }
}

// p = z + beta p on the rows of this context
__global__ void k_dcg_direction(CG A, double beta, const double* __restrict__ zv,
                                double* __restrict__ p)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x)
        if (A.bcon[i] == 0) p[i] = zv[i] + beta * p[i];
}

__global__ void k_set_zero_flag(double* scal, double bb)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) scal[S_ZERO] = (bb == 0.0) ? 1.0 : 0.0;
}

CG dcg_args(mps_ctx* c, int nblk)
{
    return CG{c->mcol, c->mval, c->mlen, c->moff, c->diag, c->sysmask, c->cap_l, c->n,
              c->cfg.solver == 1 ? 1 : 0, nblk, c->ppe_warm == 0 ? 1 : 0, c->mrow};
}

// the first `count` partial arrays of part, summed, to the host
int local_sums_to_host(mps_ctx* c, int nblk, const double* part, int count, double* out)
{
    // cg_scal / red_host slots 16..19 (the device loop's scalars use 0..15)
    k_local_sums<<<1, kRedThreads, 0, c->stream>>>(nblk, count, part, c->cg_scal + 16);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaMemcpyAsync(c->red_host + 16, c->cg_scal + 16, sizeof(double) * count,
                                 cudaMemcpyDeviceToHost, c->stream));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < count; k++) out[k] = c->red_host[16 + k];
    return MPS_OK;
}

}  // namespace

#define DCG_NEED(c)                                                                 \
    do {                                                                            \
        if (!(c) || !(c)->initialized || (c)->cfg.method == 3 || (c)->cfg.precision != 0) \
            return MPS_ERR_ARG;                                                     \
    } while (0)

extern "C" {

int mps_ppe_assemble(mps_ctx* c)
{
    DCG_NEED(c);
    VMPS_CUDA(c, cudaSetDevice(c->device));
    int warm = 0;
    int r = ppe_assemble(c, &warm);
    if (r != MPS_OK) return r;
    c->ppe_warm = warm;
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

int mps_dcg_start(mps_ctx* c, double* local3)
{
    DCG_NEED(c);
    if (!local3) return MPS_ERR_ARG;
    int nblk = 0;
    int r = cg_grid(c, &nblk);
    if (r != MPS_OK) return r;
    const CG G = dcg_args(c, nblk);
    VMPS_CUDA(c, cudaMemsetAsync(c->cg_flag, 0, 4 * sizeof(int), c->stream));
    k_cg_start<kRowG><<<nblk, kRedThreads, 0, c->stream>>>(G, c->source, c->pnew, c->cg_r, c->cg_z,
                                                     c->cg_p, c->cg_part);
    vmps_count_launch(1);
    return local_sums_to_host(c, nblk, c->cg_part, 3, local3);  // b.b, r.z, r.r
}

int mps_dcg_spmv(mps_ctx* c, double* local_ps)
{
    DCG_NEED(c);
    if (!local_ps) return MPS_ERR_ARG;
    int nblk = 0;
    int r = cg_grid(c, &nblk);
    if (r != MPS_OK) return r;
    const CG G = dcg_args(c, nblk);
    k_cg_spmv<kRowG><<<nblk, kRedThreads, 0, c->stream>>>(G, c->cg_p, c->cg_s, c->cg_part + 4 * nblk,
                                                    c->cg_flag);
    vmps_count_launch(1);
    return local_sums_to_host(c, nblk, c->cg_part + 4 * nblk, 1, local_ps);
}

int mps_dcg_update(mps_ctx* c, double alpha, double* local2)
{
    DCG_NEED(c);
    if (!local2) return MPS_ERR_ARG;
    int nblk = 0;
    int r = cg_grid(c, &nblk);
    if (r != MPS_OK) return r;
    const CG G = dcg_args(c, nblk);
    k_dcg_update<<<nblk, kRedThreads, 0, c->stream>>>(G, alpha, c->pnew, c->cg_r, c->cg_z,
                                                       c->cg_p, c->cg_s, c->cg_part);
    vmps_count_launch(1);
    return local_sums_to_host(c, nblk, c->cg_part, 2, local2);  // r.z, r.r
}

int mps_dcg_direction(mps_ctx* c, double beta)
{
    DCG_NEED(c);
    int nblk = 0;
    int r = cg_grid(c, &nblk);
    if (r != MPS_OK) return r;
    k_dcg_direction<<<nblk, kRedThreads, 0, c->stream>>>(dcg_args(c, nblk), beta, c->cg_z, c->cg_p);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int mps_dcg_finish(mps_ctx* c, int iters, double relres, double bb)
{
    DCG_NEED(c);
    const mps_config& f = c->cfg;
    k_set_zero_flag<<<1, 32, 0, c->stream>>>(c->cg_scal, bb);
    k_clamp<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, f.pmin, f.pmax, c->cg_scal, c->pnew,
                                                          nullptr, c->spmax, c->sbb);
    vmps_count_launch(2);
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->cg_iters = iters;
    c->cg_outer = 0;
    c->cg_relres = relres;
    c->ppe_pending = false;
    if (!(relres <= f.cg_tol)) {
        c->host_err |= MPS_ERR_NOT_CONVERGED;
        return MPS_ERR_NOT_CONVERGED;
    }
    return MPS_OK;
}

}  // extern "C"
