// mps_stages.cu -- explicit per-particle stages of one MPS step (FP64).
//
// Each particle's neighbour row is walked by a group of lanes.  Every
// support / cutoff decision the reference takes with sqrt() is taken here on
// the squared distance against an exact threshold (same decision, see
// sqrt_cut), and magnitudes use one rsqrt per pair instead of the
// reference's sqrt and four divisions (functions.cu:32-89, 245-428), so each
// term differs from the reference's by a few ulps at most.  Positions and
// velocities are gathered as packed double4.  Lists are row-major (see
// mps_internal.cuh): a group of G lanes walks one row, entries k = lane,
// lane + G, ..., and the group's partial sums meet in a fixed butterfly.
// Reference routines are cited on each kernel.
#include "mps_internal.cuh"

using namespace vmps;

namespace {

struct Lists {
    const int* __restrict__ nbr;
    const int* __restrict__ len;
    int cap;
};

__device__ __forceinline__ const int* row_of(const Lists& L, int i)
{
    return L.nbr + (size_t)i * L.cap;
}

template <int DIM>
__device__ __forceinline__ double d2of(const double4& a, const double4& b, double& dx, double& dy,
                                       double& dz)
{
    dx = b.x - a.x;
    dy = b.y - a.y;
    dz = DIM == 3 ? b.z - a.z : 0.0;
    return dist2<DIM>(dx, dy, dz);
}

// positions (x, y, z, ptype) when ptype != nullptr, else (a, b, c, 0)
// positions with the previous pressure, for the explicit pressure sums
__global__ void k_pack_pp(int n, const double* __restrict__ x, const double* __restrict__ y,
                          const double* __restrict__ z, const double* __restrict__ p,
                          double4* __restrict__ PP4)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) PP4[i] = make_double4(x[i], y[i], z[i], p[i]);
}

__global__ void k_pack(int n, const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, const int* __restrict__ ptype,
                       double4* __restrict__ P4)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) P4[i] = make_double4(x[i], y[i], z[i], ptype ? (double)ptype[i] : 0.0);
}

// PNUM / PNUMSTAR (functions.cu:94-122, 157-179)
template <int DIM, int G>
__global__ void k_pnd(int n, Lists L, const double4* __restrict__ P4, WK wk, int correct,
                      double ncorr, double* __restrict__ out, unsigned long long* dmax)
{
    Grp<G> q;
    int i = (int)q.gid;
    if (i >= n) return;
    double4 pi = P4[i];
    const int* row = row_of(L, i);
    int len = L.len[i];
    double sum = 0.0;
    for (int k = q.lane; k < len; k += G) {
        int j = row[k];
        if (i == j) continue;
        double dx, dy, dz;
        double d2 = d2of<DIM>(pi, P4[j], dx, dy, dz);
        sum += w_fast<DIM>(wk, d2, rsq(d2));
    }
    sum = q.sum(sum);
    if (q.lane == 0) {
        if (correct && wk.ktype != 2) sum = sum * ncorr;
        out[i] = sum;
        // non-negative doubles order as their bit patterns
        if (dmax && sum > 0.0) atomicMax(dmax, (unsigned long long)__double_as_longlong(sum));
    }
}

// BCON (functions.cu:433-445)
// P4w (the predicted positions the PPE is assembled at, or null): its w
// slot, unread after PNUMSTAR, takes bcon so that the assembly finds each
// neighbour's position and status in one gather
__global__ void k_bcon(int n, const int* __restrict__ ptype, const double* __restrict__ nd,
                       double n0, double dirichlet, int* __restrict__ bcon,
                       double4* __restrict__ P4w)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b;
    if (ptype[i] <= -1) b = -1;
    else if (nd[i] / n0 < dirichlet) b = 1;
    else b = 0;
    bcon[i] = b;
    if (P4w) reinterpret_cast<double*>(P4w + i)[3] = (double)b;
}

// V_FRACTION (functions.cu:2580-2638)
template <int DIM, int G>
__global__ void k_vfraction(int n, Lists L, const int* __restrict__ ptype,
                            const double4* __restrict__ P4, WK wk, int method,
                            double* __restrict__ C)
{
    Grp<G> q;
    int I = (int)q.gid;
    if (I >= n) return;
    double sum1 = 0, sum2 = 0;
    double4 pi = P4[I];
    const int* row = row_of(L, I);
    int len = L.len[I];
    for (int k = q.lane; k < len; k += G) {
        int J = row[k];
        int pj = ptype[J];
        if (I == J || pj <= 0) continue;
        double w = 1.0;
        if (method != 1) {
            double dx, dy, dz;
            double d2 = d2of<DIM>(pi, P4[J], dx, dy, dz);
            w = w_fast<DIM>(wk, d2, rsq(d2));
        }
        sum1 += w;
        if (pj == 2) sum2 += w;
    }
    sum1 = q.sum(sum1);
    sum2 = q.sum(sum2);
    if (q.lane == 0) {
        double c = sum2 / sum1;
        if (sum1 == 0) c = 0;
        C[I] = c;
    }
}

// velocity-gradient sums of VISCOSITY / SPS (functions.cu:2096-2117, 1734-1756);
// mind2 < 0: every pair (VISCOSITY); else pairs with d2 > mind2 (SPS d > coll/10).
// Returns the group-reduced sums in every lane.
template <int DIM, int G>
__device__ __forceinline__ void grad_sums(const Grp<G>& q, const Lists& L, int I,
                                          const double4* P4, const double* un, const double* vn,
                                          const double* wn, const WK& wk, double mind2, double* s)
{
    for (int k = 0; k < 9; k++) s[k] = 0.0;
    const int* row = row_of(L, I);
    int len = L.len[I];
    double4 pi = P4[I];
    double ui = un[I], vi = vn[I], wi = DIM == 3 ? wn[I] : 0.0;
    for (int k = q.lane; k < len; k += G) {
        int j = row[k];
        if (I == j) continue;
        double dx, dy, dz;
        double d2 = d2of<DIM>(pi, P4[j], dx, dy, dz);
        if (!(mind2 < 0 || d2 > mind2)) continue;
        double rD = rsq(d2);
        double f = w_fast<DIM>(wk, d2, rD) * rD * rD;
        double du = un[j] - ui, dv = vn[j] - vi;
        s[0] += du * dx * f;
        s[1] += dv * dy * f;
        s[2] += du * dy * f;
        s[3] += dv * dx * f;
        if (DIM == 3) {
            double dw = wn[j] - wi;
            s[4] += dw * dz * f;
            s[5] += du * dz * f;
            s[6] += dv * dz * f;
            s[7] += dw * dx * f;
            s[8] += dw * dy * f;
        }
    }
    for (int k = 0; k < (DIM == 3 ? 9 : 4); k++) s[k] = q.sum(s[k]);
}

// strain tensor S11 S12 S22 S13 S23 S33 (functions.cu:2118-2146)
template <int DIM>
__device__ __forceinline__ void strain(double n0, const double* s, double* S)
{
    double Uxx = (2.0 / n0) * s[0], Uyy = (2.0 / n0) * s[1];
    double Uxy = (2.0 / n0) * s[2], Uyx = (2.0 / n0) * s[3];
    S[1] = 0.5 * (Uxy + Uyx);
    S[0] = 0.5 * (Uxx + Uxx);
    S[2] = 0.5 * (Uyy + Uyy);
    S[3] = S[4] = S[5] = 0.0;
    if (DIM == 3) {
        double Uzz = (2.0 / n0) * s[4], Uxz = (2.0 / n0) * s[5], Uyz = (2.0 / n0) * s[6];
        double Uzx = (2.0 / n0) * s[7], Uzy = (2.0 / n0) * s[8];
        S[5] = 0.5 * (Uzz + Uzz);
        S[3] = 0.5 * (Uxz + Uzx);
        S[4] = 0.5 * (Uyz + Uzy);
    }
}

struct Phys {
    double rho1, rho2, nu1, nu2, n0, meu0, n_pl, phi, cohes, cs, l0, mind2;
    int fluid2_type;
    WK wk;
};

// VISCOSITY (functions.cu:2053-2184); reads C[i] where the reference reads
// C[0] (identical whenever phi == 0)
template <int DIM, int G>
__global__ void k_viscosity(int n, Lists L, Phys P, const int* __restrict__ ptype,
                            const double4* __restrict__ P4, const double* __restrict__ un,
                            const double* __restrict__ vn, const double* __restrict__ wn,
                            const double* __restrict__ C, const double* __restrict__ phat,
                            double* __restrict__ meu)
{
    Grp<G> q;
    int i = (int)q.gid;
    if (i >= n) return;
    int pt = ptype[i];
    if (P.fluid2_type == 0) {
        if (q.lane == 0) {
            if (pt <= 1) meu[i] = P.nu1 * P.rho1;
            if (pt == 2) meu[i] = P.nu2 * P.rho2;
        }
        return;
    }
    if (pt == 1) {
        if (q.lane == 0) meu[i] = P.nu1 * P.rho1;
        return;
    }
    double s[9], S[6];
    grad_sums<DIM, G>(q, L, i, P4, un, vn, wn, P.wk, -1.0, s);
    if (q.lane != 0) return;
    strain<DIM>(P.n0, s, S);
    double phi = (C[i] - 0.25) * P.phi / (1 - 0.25);
    if (C[i] < 0.25) phi = 0;
    double yield_stress = P.cohes * cos(phi) + phat[i] * sin(phi);
    double S11 = S[0], S12 = S[1], S22 = S[2], S13 = S[3], S23 = S[4], S33 = S[5];
    double II;
    if (DIM == 3)
        II = fabs((S11 * S22 * S33 + S12 * S23 * S13 + S13 * S12 * S23) -
                  (S13 * S22 * S13 + S11 * S23 * S23 + S12 * S12 * S33));
    else
        II = fabs(S11 * S22 - S12 * S12);
    double m = yield_stress / 2 / sqrt(II) + P.meu0 * pow(4 * II, (P.n_pl - 1) / 2);
    if (II == 0 || m > 200) m = 200;
    meu[i] = m;
}

// SPS pass 1: strain tensor and eddy viscosity (functions.cu:1731-1790)
template <int DIM, int G>
__global__ void k_sps1(int n, Lists L, Phys P, const int* __restrict__ ptype,
                       const double4* __restrict__ P4, const double* __restrict__ un,
                       const double* __restrict__ vn, const double* __restrict__ wn,
                       double* __restrict__ S6, double* __restrict__ neut)
{
    Grp<G> q;
    int i = (int)q.gid;
    if (i >= n || ptype[i] < 0) return;
    double s[9], S[6];
    grad_sums<DIM, G>(q, L, i, P4, un, vn, wn, P.wk, P.mind2, s);
    if (q.lane != 0) return;
    strain<DIM>(P.n0, s, S);
    for (int c = 0; c < 6; c++) S6[(size_t)c * n + i] = S[c];
    double S11 = S[0], S12 = S[1], S22 = S[2], S13 = S[3], S23 = S[4], S33 = S[5];
    double Sm;
    if (DIM == 3)
        Sm = sqrt(2 * S11 * S11) + 2 * sqrt(2 * S12 * S12) + sqrt(2 * S22 * S22) +
             sqrt(2 * S33 * S33) + 2 * sqrt(2 * S13 * S13) + 2 * sqrt(2 * S23 * S23);
    else
        Sm = sqrt(2 * S11 * S11) + 2 * sqrt(2 * S12 * S12) + sqrt(2 * S22 * S22);
    double cd = P.cs * P.l0;
    neut[i] = (cd * cd) * Sm;
}

// SPS pass 2: divergence of the SPS stress (functions.cu:1793-1830)
template <int DIM, int G>
__global__ void k_sps2(int n, Lists L, Phys P, const int* __restrict__ ptype,
                       const double4* __restrict__ P4, const double* __restrict__ S6,
                       const double* __restrict__ neut, double* __restrict__ t1,
                       double* __restrict__ t2, double* __restrict__ t3)
{
    Grp<G> q;
    int i = (int)q.gid;
    if (i >= n || ptype[i] < 0) return;
    double sum1 = 0, sum2 = 0, sum3 = 0;
    const int* row = row_of(L, i);
    int len = L.len[i];
    double ni = neut[i];
    double4 pi = P4[i];
    for (int k = q.lane; k < len; k += G) {
        int j = row[k];
        if (i == j) continue;
        double dx, dy, dz;
        double d2 = d2of<DIM>(pi, P4[j], dx, dy, dz);
        if (!(d2 > P.mind2)) continue;
        double rD = rsq(d2);
        double f = (neut[j] - ni) * w_fast<DIM>(P.wk, d2, rD) * rD * rD;
        sum1 += dx * f;
        sum2 += dy * f;
        if (DIM == 3) sum3 += dz * f;
    }
    sum1 = q.sum(sum1);
    sum2 = q.sum(sum2);
    sum3 = q.sum(sum3);
    if (q.lane != 0) return;
    double S11 = S6[i], S12 = S6[(size_t)n + i], S22 = S6[2 * (size_t)n + i];
    double S13 = S6[3 * (size_t)n + i], S23 = S6[4 * (size_t)n + i], S33 = S6[5 * (size_t)n + i];
    if (DIM == 3) {
        t1[i] = (2.0 / P.n0) * (2 * S11 * sum1 + 2 * S12 * sum2 + 2 * S13 * sum3);
        t2[i] = (2.0 / P.n0) * (2 * S12 * sum1 + 2 * S22 * sum2 + 2 * S23 * sum3);
        t3[i] = (2.0 / P.n0) * (2 * S13 * sum1 + 2 * S23 * sum2 + 2 * S33 * sum3);
    } else {
        t1[i] = (2.0 / P.n0) * (2 * S11 * sum1 + 2 * S12 * sum2);
        t2[i] = (2.0 / P.n0) * (2 * S12 * sum1 + 2 * S22 * sum2);
    }
}

struct PredArgs {
    WK ws, wl;
    double n0_s, visc_coef, dt, gx, gy, gz, relaxp, rho1, rho2;
    // Newtonian fluids: VISCOSITY sets meu by particle kind (nu1 rho1 for
    // kinds <= 1, nu2 rho2 for kind 2), so a neighbour's meu follows from the
    // kind its packed position carries, without a gather of meu
    int meu_by_kind;
    double meu1, meu2;
};

// PREDICTION (functions.cu:2283-2369), first part: the explicit pressure
// sums over the PND list, scaled by (1-relaxp)*2*dt/(n0*rho) (fluid rows).
// 5 resident blocks per SM (48 registers, no spills; 68 without the bound):
// with k_pressgrad's, 0.12 ms per step faster on the 1.6 M-particle dam
template <int DIM, int G>
__global__ void __launch_bounds__(256, 5) k_predict_p(int n, Lists Ls, PredArgs A, const double4* __restrict__ P4,
                            const double4* __restrict__ PP4, const double* __restrict__ phat,
                            const double* __restrict__ rho, double* __restrict__ px,
                            double* __restrict__ py, double* __restrict__ pz)
{
    Grp<G> q;
    int I = (int)q.gid;
    if (I >= n) return;
    if (P4[I].w <= 0) return;
    const double4 pi = PP4[I];
    double sum1 = 0, sum2 = 0, sum3 = 0;
    double ph = phat[I];
    const int* row = row_of(Ls, I);
    int len = Ls.len[I];
    for (int k = q.lane; k < len; k += G) {
        int J = row[k];
        if (I == J) continue;
        double dx, dy, dz;
        const double4 pj = PP4[J];  // position and previous pressure in one gather
        double d2 = d2of<DIM>(pi, pj, dx, dy, dz);
        if (!(d2 > 0)) continue;
        double rD = rsq(d2);
        double f = (pj.w - ph) * w_fast<DIM>(A.ws, d2, rD) * rD * rD;
        sum1 += dx * f;
        sum2 += dy * f;
        if (DIM == 3) sum3 += dz * f;
    }
    sum1 = q.sum(sum1);
    sum2 = q.sum(sum2);
    if (DIM == 3) sum3 = q.sum(sum3);
    if (q.lane != 0) return;
    double pc = (1 - A.relaxp) * (2.0 * A.dt / A.n0_s / rho[I]);
    px[I] = pc * sum1;
    py[I] = pc * sum2;
    if (DIM == 3) pz[I] = pc * sum3;
}

// lanes per particle of the FP32 viscous sums (measured: 8 lanes 3.9 ms of
// explicit stages on the 1.6 M-particle dam, 16 lanes 4.1, a warp 4.4)
constexpr int kPred32G = 8;
// Mixed precision: the viscous Laplacian's neighbour sums in FP32 (FP32
// positions relative to the box, FP32 velocities, FP32 weights and sums);
// u* and x* are then formed in FP64 exactly as in k_predict.
// TURB: the eddy-viscosity sums (sum7..9, times neut) are kept only with
// SPS on; without it neut is 0 and they add nothing.
template <int DIM, bool TURB>
// 4 blocks per SM: the two-entries-in-flight loop needs the registers
// (measured 4.4 ms explicit stages on the 1.6 M dam against 5.1 at 5 blocks)
__global__ void __launch_bounds__(256, 4)
k_predict32(int n, Lists Ll, PredArgs A, WKf wl, const double* __restrict__ meu,
            const double4* __restrict__ P4, const double4* __restrict__ U4,
            const float4* __restrict__ P4f, const float4* __restrict__ U4f,
            const double* __restrict__ px, const double* __restrict__ py,
            const double* __restrict__ pz, const double* __restrict__ neut,
            const double* __restrict__ t1, const double* __restrict__ t2,
            const double* __restrict__ t3, double* __restrict__ xs, double* __restrict__ ys,
            double* __restrict__ zs, double* __restrict__ us, double* __restrict__ vs,
            double* __restrict__ ws, double4* __restrict__ P4s, float4* __restrict__ P4sf,
            double3 box0)
{
    Grp<kPred32G> q;
    int I = (int)q.gid;
    if (I >= n) return;
    double4 pi = P4[I], ui4 = U4[I];
    int pI = (int)pi.w;
    // precision 2: the predicted positions in FP32 too, relative to the box
    auto put_f = [&](const double4& o) {
        if (P4sf)
            P4sf[I] = make_float4((float)(o.x - box0.x), (float)(o.y - box0.y),
                                  DIM == 3 ? (float)(o.z - box0.z) : 0.f, o.w);
    };
    if (pI <= 0) {
        if (q.lane == 0) {
            xs[I] = pi.x; ys[I] = pi.y; us[I] = ui4.x; vs[I] = ui4.y;
            if (DIM == 3) { zs[I] = pi.z; ws[I] = ui4.z; }
            P4s[I] = pi;
            put_f(pi);
        }
        return;
    }
    const float4 fi = P4f[I], vi = U4f[I];
    float s4 = 0.f, s5 = 0.f, s6 = 0.f, s7 = 0.f, s8 = 0.f, s9 = 0.f;
    const double mI = meu[I];
    const double rhoI = (pI == 1) ? A.rho1 : A.rho2;
    const float neu_same = (float)(mI / rhoI);
    const int* row = row_of(Ll, I);
    int len = Ll.len[I];
    auto add = [&](int J, const float4& fj, const float4& vj) {
        if (I == J) return;
        const float dx = fj.x - fi.x, dy = fj.y - fi.y, dz = DIM == 3 ? fj.z - fi.z : 0.f;
        const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (!(d2 > 0.f)) return;
        const float W = w_fast32<DIM>(wl, d2);
        float NEU = neu_same;
        if ((int)fj.w != pI) {
            const double mJ = A.meu_by_kind ? ((int)fj.w == 2 ? A.meu2 : A.meu1) : meu[J];
            NEU = (float)(2 * mI * mJ / (mI + mJ) / rhoI);
        }
        const float du = W * (vj.x - vi.x), dv = W * (vj.y - vi.y);
        s4 = __fmaf_rn(du, NEU, s4);
        s5 = __fmaf_rn(dv, NEU, s5);
        if (TURB) {
            s7 += du;
            s8 += dv;
        }
        if (DIM == 3) {
            const float dw = W * (vj.z - vi.z);
            s6 = __fmaf_rn(dw, NEU, s6);
            if (TURB) s9 += dw;
        }
    };
    // two entries per lane in flight (k, k + G); the sums see them in list order
    for (int k = q.lane; k < len; k += 2 * kPred32G) {
        const bool two = k + kPred32G < len;
        const int J0 = row[k], J1 = two ? row[k + kPred32G] : I;
        const float4 f0 = P4f[J0], f1 = P4f[J1], v0 = U4f[J0], v1 = U4f[J1];
        add(J0, f0, v0);
        add(J1, f1, v1);
    }
    double sum4 = q.sum((double)s4), sum5 = q.sum((double)s5), sum7 = 0, sum8 = 0, sum6 = 0,
           sum9 = 0;
    if (TURB) { sum7 = q.sum((double)s7); sum8 = q.sum((double)s8); }
    if (DIM == 3) sum6 = q.sum((double)s6);
    if (DIM == 3 && TURB) sum9 = q.sum((double)s9);
    if (q.lane != 0) return;
    double DT = A.dt, nt = TURB ? neut[I] : 0.0;
    double uS = ui4.x + A.gx * DT + A.visc_coef * (sum4 + nt * sum7) + DT * t1[I] - px[I];
    double vS = ui4.y + A.gy * DT + A.visc_coef * (sum5 + nt * sum8) + DT * t2[I] - py[I];
    double4 o = pi;
    o.x = pi.x + DT * uS;
    o.y = pi.y + DT * vS;
    us[I] = uS;
    vs[I] = vS;
    xs[I] = o.x;
    ys[I] = o.y;
    if (DIM == 3) {
        double wS = ui4.z + A.gz * DT + A.visc_coef * (sum6 + nt * sum9) + DT * t3[I] - pz[I];
        ws[I] = wS;
        o.z = pi.z + DT * wS;
        zs[I] = o.z;
    }
    P4s[I] = o;
    put_f(o);
}

// PREDICTION, second part: viscous Laplacian over the Laplacian list, one
// group of kPredG lanes per particle, then u* and x*.
// lanes per particle of the viscous sums: 8 (explicit stages 5.0 ms on the
// 1.6 M-particle dam against 5.5 ms with a whole warp; 4 is no better)
constexpr int kPredG = 8;
// TURB: the eddy-viscosity sums (sum7..9, times neut) are kept only with
// SPS on; without it neut is 0 and they add nothing (explicit stages 0.19
// ms faster on the 1.6 M-particle dam; 6 blocks per SM at 40 registers lose)
template <int DIM, bool TURB>
__global__ void __launch_bounds__(256, 5)
k_predict(int n, Lists Ll, PredArgs A, const double* __restrict__ meu,
          const double4* __restrict__ P4, const double4* __restrict__ U4,
          const double* __restrict__ px, const double* __restrict__ py,
          const double* __restrict__ pz, const double* __restrict__ neut,
          const double* __restrict__ t1, const double* __restrict__ t2,
          const double* __restrict__ t3, double* __restrict__ xs, double* __restrict__ ys,
          double* __restrict__ zs, double* __restrict__ us, double* __restrict__ vs,
          double* __restrict__ ws, double4* __restrict__ P4s)
{
    Grp<kPredG> q;
    int I = (int)q.gid;
    if (I >= n) return;
    double4 pi = P4[I], ui4 = U4[I];
    int pI = (int)pi.w;
    if (pI <= 0) {
        if (q.lane == 0) {
            xs[I] = pi.x; ys[I] = pi.y; us[I] = ui4.x; vs[I] = ui4.y;
            if (DIM == 3) { zs[I] = pi.z; ws[I] = ui4.z; }
            P4s[I] = pi;
        }
        return;
    }
    double sum4 = 0, sum5 = 0, sum6 = 0, sum7 = 0, sum8 = 0, sum9 = 0;
    double mI = meu[I];
    double rhoI = (pI == 1) ? A.rho1 : A.rho2;
    double neu_same = mI / rhoI;
    const int* row = row_of(Ll, I);
    int len = Ll.len[I];
    for (int k = q.lane; k < len; k += kPredG) {
        int J = row[k];
        if (I == J) continue;
        double4 pj = P4[J];
        double dx, dy, dz;
        double d2 = d2of<DIM>(pi, pj, dx, dy, dz);
        if (!(d2 > 0)) continue;
        double W = w_fast<DIM>(A.wl, d2, rsq(d2));
        double NEU = neu_same;
        if ((int)pj.w != pI) {
            const double mJ = A.meu_by_kind ? ((int)pj.w == 2 ? A.meu2 : A.meu1) : meu[J];
            NEU = 2 * mI * mJ / (mI + mJ) / rhoI;
        }
        double4 uj = U4[J];
        double du = W * (uj.x - ui4.x), dv = W * (uj.y - ui4.y);
        sum4 += du * NEU;
        sum5 += dv * NEU;
        if (TURB) {
            sum7 += du;
            sum8 += dv;
        }
        if (DIM == 3) {
            double dw = W * (uj.z - ui4.z);
            sum6 += dw * NEU;
            if (TURB) sum9 += dw;
        }
    }
    sum4 = q.sum(sum4); sum5 = q.sum(sum5);
    if (TURB) { sum7 = q.sum(sum7); sum8 = q.sum(sum8); }
    if (DIM == 3) sum6 = q.sum(sum6);
    if (DIM == 3 && TURB) sum9 = q.sum(sum9);
    if (q.lane != 0) return;
    double DT = A.dt, nt = TURB ? neut[I] : 0.0;
    double uS = ui4.x + A.gx * DT + A.visc_coef * (sum4 + nt * sum7) + DT * t1[I] - px[I];
    double vS = ui4.y + A.gy * DT + A.visc_coef * (sum5 + nt * sum8) + DT * t2[I] - py[I];
    double4 o = pi;
    o.x = pi.x + DT * uS;
    o.y = pi.y + DT * vS;
    us[I] = uS;
    vs[I] = vS;
    xs[I] = o.x;
    ys[I] = o.y;
    if (DIM == 3) {
        double wS = ui4.z + A.gz * DT + A.visc_coef * (sum6 + nt * sum9) + DT * t3[I] - pz[I];
        ws[I] = wS;
        o.z = pi.z + DT * wS;
        zs[I] = o.z;
    }
    P4s[I] = o;
}

// weakly compressible EOS (functions.cu:2467-2500)
__global__ void k_pressure_wc(int n, const int* __restrict__ ptype, const double* __restrict__ C,
                              const double* __restrict__ nstar, double n0, double beta, double c01,
                              double c02, double rho1, double rho2, double pmin, double pmax,
                              double* __restrict__ pnew)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n || ptype[I] < 0) return;
    double c0 = (ptype[I] == 2) ? c02 : c01;
    double Rho = rho2 * C[I] + rho1 * (1 - C[I]);
    double p;
    if (nstar[I] < beta * n0) p = 0.0;
    else p = (c0 * c0 * Rho / 7.0) * (pow(nstar[I] / n0, 7.0) - 1);
    if (p < pmin) p = pmin;
    if (p > pmax) p = pmax;
    pnew[I] = p;
}

// PHATCALC (functions.cu:207-224); also packs (pnew, phat) for the gradient
template <int G>
__global__ void k_phat(int n, Lists L, const double* __restrict__ pnew, double* __restrict__ phat,
                       double2* __restrict__ PH, float2* __restrict__ PH32)
{
    Grp<G> q;
    int I = (int)q.gid;
    if (I >= n) return;
    double mn = 999999999999999;
    const int* row = row_of(L, I);
    int len = L.len[I];
    for (int k = q.lane; k < len; k += G) {
        double pj = pnew[row[k]];
        if (pj < mn) mn = pj;
    }
    mn = q.min(mn);
    if (q.lane == 0) {
        phat[I] = mn;
        PH[I] = make_double2(pnew[I], mn);
        if (PH32) PH32[I] = make_float2((float)pnew[I], (float)mn);
    }
}

struct GradArgs {
    WK wk;
    double coef, vmax;
    int kh;
};

// PRESSGRAD (functions.cu:245-355), CPU semantics (p^_i + p^_j)
// 5 resident blocks per SM (48 registers, no spills; 70 without the bound)
template <int DIM, int G>
__global__ void __launch_bounds__(256, 5) k_pressgrad(int n, Lists L, GradArgs A, const int* __restrict__ ptype,
                            const double2* __restrict__ PH, const double4* __restrict__ P4s,
                            const double* __restrict__ rho, const double* __restrict__ us,
                            const double* __restrict__ vs, const double* __restrict__ ws,
                            double* __restrict__ un, double* __restrict__ vn,
                            double* __restrict__ wn)
{
    Grp<G> q;
    int I = (int)q.gid;
    if (I >= n || ptype[I] <= 0) return;
    double sum1 = 0, sum2 = 0, sum3 = 0;
    double4 pi = P4s[I];
    double2 phI = PH[I];
    const int* row = row_of(L, I);
    int len = L.len[I];
    for (int k = q.lane; k < len; k += G) {
        int J = row[k];
        if (I == J) continue;
        double dx, dy, dz;
        double d2 = d2of<DIM>(pi, P4s[J], dx, dy, dz);
        double rD = rsq(d2);
        double2 phJ = PH[J];
        double pp = (A.kh == 1) ? phJ.x + phI.x - (phI.y + phJ.y) : phJ.x - phI.y;
        double f = pp * w_fast<DIM>(A.wk, d2, rD) * rD * rD;
        sum1 += dx * f;
        sum2 += dy * f;
        if (DIM == 3) sum3 += dz * f;
    }
    sum1 = q.sum(sum1);
    sum2 = q.sum(sum2);
    if (DIM == 3) sum3 = q.sum(sum3);
    if (q.lane != 0) return;
    double c = A.coef / rho[I], VMAX = A.vmax, coeff = 2.0;
    double uN = us[I] - c * sum1;
    double vN = vs[I] - c * sum2;
    if (fabs(uN) > coeff * VMAX) uN = VMAX;
    if (vN > coeff * VMAX) vN = coeff * VMAX;
    if (vN < -coeff * VMAX) vN = -coeff * VMAX;
    un[I] = uN;
    vn[I] = vN;
    if (DIM == 3) {
        double wN = ws[I] - c * sum3;
        if (fabs(wN) > coeff * VMAX) wN = VMAX;
        wn[I] = wN;
    }
}

// Precision 2: PNUMSTAR (functions.cu:157-201) with FP32 positions relative
// to the box, FP32 weights and an FP32 sum; n* is stored in FP64 and the
// source (n* - n0) / n0 is formed from it in FP64.
template <int DIM, int G>
__global__ void k_pnd32(int n, Lists L, const float4* __restrict__ P4f, WKf wk,
                        double* __restrict__ out)
{
    Grp<G> q;
    int i = (int)q.gid;
    if (i >= n) return;
    const float4 pi = P4f[i];
    const int* row = row_of(L, i);
    int len = L.len[i];
    float sum = 0.f;
    for (int k = q.lane; k < len; k += G) {
        int j = row[k];
        if (i == j) continue;
        const float4 pj = P4f[j];
        const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = DIM == 3 ? pj.z - pi.z : 0.f;
        const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (d2 > 0.f) sum += w_fast32<DIM>(wk, d2);
    }
    sum = q.sumf(sum);
    if (q.lane == 0) out[i] = (double)sum;
}

// Precision 2: PRESSGRAD (functions.cu:245-355) with FP32 positions,
// pressures, weights and sums; u^{n+1} = u* - c * sum formed in FP64.
template <int DIM, int G>
__global__ void __launch_bounds__(256, 5) k_pressgrad32(int n, Lists L, GradArgs A, WKf wk,
                            const int* __restrict__ ptype, const float2* __restrict__ PH32,
                            const float4* __restrict__ P4sf, const double* __restrict__ rho,
                            const double* __restrict__ us, const double* __restrict__ vs,
                            const double* __restrict__ ws, double* __restrict__ un,
                            double* __restrict__ vn, double* __restrict__ wn)
{
    Grp<G> q;
    int I = (int)q.gid;
    if (I >= n || ptype[I] <= 0) return;
    float s1 = 0.f, s2 = 0.f, s3 = 0.f;
    const float4 pi = P4sf[I];
    const float2 phI = PH32[I];
    const int* row = row_of(L, I);
    int len = L.len[I];
    for (int k = q.lane; k < len; k += G) {
        int J = row[k];
        if (I == J) continue;
        const float4 pj = P4sf[J];
        const float dx = pj.x - pi.x, dy = pj.y - pi.y, dz = DIM == 3 ? pj.z - pi.z : 0.f;
        const float d2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
        if (!(d2 > 0.f)) continue;
        const float2 phJ = PH32[J];
        const float pp = (A.kh == 1) ? phJ.x + phI.x - (phI.y + phJ.y) : phJ.x - phI.y;
        const float f = pp * w_fast32<DIM>(wk, d2) / d2;
        s1 = __fmaf_rn(dx, f, s1);
        s2 = __fmaf_rn(dy, f, s2);
        if (DIM == 3) s3 = __fmaf_rn(dz, f, s3);
    }
    const double sum1 = q.sum((double)s1), sum2 = q.sum((double)s2);
    const double sum3 = DIM == 3 ? q.sum((double)s3) : 0.0;
    if (q.lane != 0) return;
    double c = A.coef / rho[I], VMAX = A.vmax, coeff = 2.0;
    double uN = us[I] - c * sum1;
    double vN = vs[I] - c * sum2;
    if (fabs(uN) > coeff * VMAX) uN = VMAX;
    if (vN > coeff * VMAX) vN = coeff * VMAX;
    if (vN < -coeff * VMAX) vN = -coeff * VMAX;
    un[I] = uN;
    vn[I] = vN;
    if (DIM == 3) {
        double wN = ws[I] - c * sum3;
        if (fabs(wN) > coeff * VMAX) wN = VMAX;
        wn[I] = wN;
    }
}

struct Box {
    double xmin, xmax, ymin, ymax, zmin, zmax, dl, dt, cc;
    const int* scene;     // per-particle scene, or nullptr for one scene
    const double* sbox;   // 6 per scene
};

// the box of particle I: its scene's when scenes are batched
__device__ __forceinline__ void box_of(const Box& B, int I, double* b)
{
    if (B.scene) {
        const double* q = B.sbox + 6 * B.scene[I];
        for (int k = 0; k < 6; k++) b[k] = q[k];
    } else {
        b[0] = B.xmin; b[1] = B.xmax; b[2] = B.ymin; b[3] = B.ymax; b[4] = B.zmin; b[5] = B.zmax;
    }
}

// EULERINTEGRATION + BOUNDARIE (functions.cu:1963-2021)
template <int DIM>
__global__ void k_integrate(int n, Box B, const int* __restrict__ ptype, double* __restrict__ x,
                            double* __restrict__ y, double* __restrict__ z,
                            double* __restrict__ un, double* __restrict__ vn,
                            double* __restrict__ wn, double4* __restrict__ P4)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n || ptype[I] <= 0) return;
    double DT = B.dt, DL = B.dl, CC = B.cc;
    double bx[6];
    box_of(B, I, bx);
    double xi = x[I] + un[I] * DT, yi = y[I] + vn[I] * DT;
    double ui = un[I], vi = vn[I];
    if (yi < bx[2] + DL * 3.0) { vi = fabs(vi) * CC; yi = bx[2] + DL * 3.0; }
    if (yi > bx[3] - DL * 3.0) { vi = -fabs(vi) * CC; yi = bx[3] - DL * 3.0; }
    if (xi < bx[0] + DL * 3.0) { ui = fabs(ui) * CC; xi = bx[0] + DL * 3.0; }
    if (xi > bx[1] - DL * 3.0) { ui = -fabs(ui) * CC; xi = bx[1] - DL * 3.0; }
    double zi = 0.0;
    if (DIM == 3) {
        double wi = wn[I];
        zi = z[I] + wn[I] * DT;
        if (zi < bx[4] + DL * 3.0) { wi = fabs(wi) * CC; zi = bx[4] + DL * 3.0; }
        if (zi > bx[5] - DL * 3.0) { wi = -fabs(wi) * CC; zi = bx[5] - DL * 3.0; }
        z[I] = zi;
        wn[I] = wi;
    }
    x[I] = xi; y[I] = yi; un[I] = ui; vn[I] = vi;
    P4[I] = make_double4(xi, yi, zi, P4[I].w);
}

struct CollArgs {
    double coll2, cc, dt, rho1, rho2;
};

// One visit of COLLISION2's pair loop (functions.cu:1536-1599) from i's list
// to its neighbour j, on register copies s = {u, v, w, x, y, z} of the two
// states: the reference's expressions in the reference's order.
template <int DIM>
__device__ __forceinline__ void coll_visit(const CollArgs& A, int pti, int ptj, double* si,
                                           double* sj)
{
    const double m1 = (pti == 1) ? A.rho1 : A.rho2, m2 = (ptj == 1) ? A.rho1 : A.rho2;
    const double ex = sj[3] - si[3], ey = sj[4] - si[4], ez = DIM == 3 ? sj[5] - si[5] : 0.0;
    const double d2 = dist2<DIM>(ex, ey, ez);
    if (!(d2 < A.coll2)) return;
    const double d = sqrt(d2);
    const double ug = (m1 * si[0] + m2 * sj[0]) / (m1 + m2);
    const double vg = (m1 * si[1] + m2 * sj[1]) / (m1 + m2);
    const double ur = m1 * (si[0] - ug), vr = m1 * (si[1] - vg);
    double vabs;
    if (DIM == 3) {
        const double wg = (m1 * si[2] + m2 * sj[2]) / (m1 + m2);
        const double wr = m1 * (si[2] - wg);
        vabs = (ur * ex + vr * ey + wr * ez) / d;
    } else {
        vabs = (ur * ex + vr * ey) / d;
    }
    if (!(vabs > 0)) return;
    const double um = (1.0 + A.cc) * vabs * ex / d;
    const double vm = (1.0 + A.cc) * vabs * ey / d;
    const double wm = DIM == 3 ? (1.0 + A.cc) * vabs * ez / d : 0.0;
    if (pti > 0) {
        si[0] = si[0] - um / m1; si[1] = si[1] - vm / m1;
        si[3] = si[3] - A.dt * um / m1; si[4] = si[4] - A.dt * vm / m1;
        if (DIM == 3) { si[2] = si[2] - wm / m1; si[5] = si[5] - A.dt * wm / m1; }
    }
    if (ptj > 0) {
        sj[0] = sj[0] + um / m2; sj[1] = sj[1] + vm / m2;
        sj[3] = sj[3] + A.dt * um / m2; sj[4] = sj[4] + A.dt * vm / m2;
        if (DIM == 3) { sj[2] = sj[2] + wm / m2; sj[5] = sj[5] + A.dt * wm / m2; }
    }
}

// COLLISION2 (functions.cu:1523-1601) in an order-independent form.  The
// reference walks every particle, walls and dummies included, in id order
// and updates pairs in place, so a pair (a, b), a < b, is visited twice:
// from a's list, then from b's list with the state the first visit left (a
// fluid-wall pair can be pushed twice; a fluid-fluid pair separates after
// the first push).  Each fluid particle here replays, for every neighbour
// closer than coll in the pre-collision state, that pair's two visits in
// registers.  With one such neighbour the particle takes the replayed state
// -- COLLISION2's own result, bit for bit, as nothing else touches the pair
// in between; with several it takes the pre-collision state plus the sum of
// the pairs' changes.  The new states go to the *o arrays, and
// k_collision_apply copies them over once every particle has read the
// pre-collision state (no buffer swap, so the step's buffers stay fixed).
template <int DIM, int G>
__global__ void __launch_bounds__(256, 3) k_collision(int n, Lists L, CollArgs A, const int* __restrict__ ptype,
                            const int* __restrict__ oid, const double4* __restrict__ P4,
                            const double* __restrict__ un, const double* __restrict__ vn,
                            const double* __restrict__ wn, double* __restrict__ xo,
                            double* __restrict__ yo, double* __restrict__ zo,
                            double* __restrict__ uo, double* __restrict__ vo,
                            double* __restrict__ wo)
{
    Grp<G> q;
    const int i = (int)q.gid;
    if (i >= n) return;  // whole groups leave together
    const int pti = ptype[i];
    if (pti <= 0) return;
    const double4 pi = P4[i];
    const double s0[6] = {un[i], vn[i], DIM == 3 ? wn[i] : 0.0, pi.x, pi.y, DIM == 3 ? pi.z : 0.0};
    // the replay of pair (i, j) into si
    auto replay = [&](int j, const double4& pj, double* si) {
        double sj[6] = {un[j], vn[j], DIM == 3 ? wn[j] : 0.0, pj.x, pj.y, DIM == 3 ? pj.z : 0.0};
#pragma unroll
        for (int t = 0; t < 6; t++) si[t] = s0[t];
        const int ptj = ptype[j];
        if (oid[j] < oid[i]) {
            coll_visit<DIM>(A, ptj, pti, sj, si);
            coll_visit<DIM>(A, pti, ptj, si, sj);
        } else {
            coll_visit<DIM>(A, pti, ptj, si, sj);
            coll_visit<DIM>(A, ptj, pti, sj, si);
        }
    };
    // the hot loop only finds the neighbours closer than coll (rare); the
    // replays run after it
    int hits = 0, jhit = -1;
    const int* row = row_of(L, i);
    const int len = L.len[i];
    for (int k = q.lane; k < len; k += G) {
        const int j = row[k];
        if (i == j) continue;
        double ex, ey, ez;
        if (d2of<DIM>(pi, P4[j], ex, ey, ez) < A.coll2) {
            hits++;
            jhit = j;
        }
    }
    int total = hits;
    for (int o = G / 2; o > 0; o >>= 1) total += __shfl_xor_sync(q.mask, total, o);
    double* const outs[6] = {uo, vo, wo, xo, yo, zo};
    if (total == 1) {  // the lane that met the one neighbour writes its replayed state
        if (hits == 1) {
            double si[6];
            replay(jhit, P4[jhit], si);
            for (int t = 0; t < 6; t++)
                if (DIM == 3 || (t != 2 && t != 5)) outs[t][i] = si[t];
        }
        return;
    }
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (total > 1) {  // several: the pre-collision state plus the sum of the replays' changes
        for (int k = q.lane; k < len; k += G) {
            const int j = row[k];
            if (i == j) continue;
            double ex, ey, ez;
            const double4 pj = P4[j];
            if (!(d2of<DIM>(pi, pj, ex, ey, ez) < A.coll2)) continue;
            double si[6];
            replay(j, pj, si);
#pragma unroll
            for (int t = 0; t < 6; t++) acc[t] += si[t] - s0[t];
        }
#pragma unroll
        for (int t = 0; t < 6; t++) acc[t] = q.sum(acc[t]);
    }
    if (q.lane != 0) return;
    for (int t = 0; t < 6; t++)
        if (DIM == 3 || (t != 2 && t != 5)) outs[t][i] = total > 1 ? s0[t] + acc[t] : s0[t];
}

template <int DIM>
__global__ void k_collision_apply(int n, const int* __restrict__ ptype, double* __restrict__ x,
                                  double* __restrict__ y, double* __restrict__ z,
                                  double* __restrict__ un, double* __restrict__ vn,
                                  double* __restrict__ wn, const double* __restrict__ xo,
                                  const double* __restrict__ yo, const double* __restrict__ zo,
                                  const double* __restrict__ uo, const double* __restrict__ vo,
                                  const double* __restrict__ wo, double4* __restrict__ P4)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || ptype[i] <= 0) return;
    double4 pi = P4[i];
    pi.x = xo[i];
    pi.y = yo[i];
    x[i] = pi.x;
    y[i] = pi.y;
    un[i] = uo[i];
    vn[i] = vo[i];
    if (DIM == 3) {
        pi.z = zo[i];
        z[i] = pi.z;
        wn[i] = wo[i];
    }
    P4[i] = pi;
}

// PREPDATA (functions.cu:2688-2746): roll state, flag ERROR#1 / ERROR#2
template <int DIM>
__global__ void k_commit(int n, Box B, const int* __restrict__ ptype,
                         const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, double* __restrict__ u,
                         double* __restrict__ v, double* __restrict__ w, double* __restrict__ p,
                         const double* __restrict__ un, const double* __restrict__ vn,
                         const double* __restrict__ wn, const double* __restrict__ pnew,
                         unsigned int* err)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    double pI = pnew[I];
    p[I] = pI;
    double uI = u[I], vI = v[I], wI = DIM == 3 ? w[I] : 0.0;
    if (ptype[I] > 0) {
        uI = un[I]; vI = vn[I];
        u[I] = uI; v[I] = vI;
        if (DIM == 3) { wI = wn[I]; w[I] = wI; }
    }
    bool bad = pI * 0 != 0 || uI * 0 != 0 || vI * 0 != 0 || (DIM == 3 && wI * 0 != 0);
    double bx[6];
    box_of(B, I, bx);
    double xi = x[I], yi = y[I];
    bool out = xi >= bx[1] || yi >= bx[3] || xi <= bx[0] || yi <= bx[2];
    if (DIM == 3) out = out || z[I] >= bx[5] || z[I] <= bx[4];
    if (bad) set_error(err, MPS_ERR_NAN);
    if (out) set_error(err, MPS_ERR_BOX);
}

Lists lists(mps_ctx* c, int which)
{
    Lists L;
    L.cap = which == 0 ? c->cap_l : c->cap_s;
    L.nbr = which == 0 ? c->nbr_l : c->nbr_s;
    L.len = which == 0 ? c->len_l : c->len_s;
    return L;
}

Phys phys(mps_ctx* c)
{
    Phys P;
    const mps_config& f = c->cfg;
    P.rho1 = f.rho1; P.rho2 = f.rho2; P.nu1 = f.nu1; P.nu2 = f.nu2; P.n0 = c->n0_s;
    P.meu0 = f.meu0; P.n_pl = f.n_pl; P.phi = f.phi; P.cohes = f.cohes; P.cs = f.cs; P.l0 = f.l0;
    P.mind2 = sqrt_cut(f.coll / 10, false);
    P.fluid2_type = f.fluid2_type;
    P.wk = make_wk(f.ktype, f.re_s);
    return P;
}

Box box(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    Box B{f.xmin, f.xmax, f.ymin, f.ymax, f.zmin, f.zmax, f.l0, f.dt, f.velcor,
          c->nscenes > 1 ? c->scene : nullptr, c->sbox};
    return B;
}

#define LAUNCH_DIM(kern, ...)                                                             \
    do {                                                                                  \
        if (c->cfg.dim == 3) kern<3><<<grid_blocks(c->n), kBlock, 0, c->stream>>>(__VA_ARGS__); \
        else kern<2><<<grid_blocks(c->n), kBlock, 0, c->stream>>>(__VA_ARGS__);           \
        vmps_count_launch(1);                                                             \
    } while (0)

inline int group_blocks(long n, int G) { return (int)((n * G + kBlock - 1) / kBlock); }

// G lanes per PND-radius row: SmallG, or twice that when the autotuner
// chose the wide form (ctx->tune_small_wide)
#define LAUNCH_SMALL(kern, ...)                                                           \
    do {                                                                                  \
        constexpr int G3 = SmallG<3>::G, G2 = SmallG<2>::G;                               \
        const bool wide = c->tune_small_wide != 0;                                        \
        if (c->cfg.dim == 3) {                                                            \
            if (wide) kern<3, 2 * G3><<<group_blocks(c->n, 2 * G3), kBlock, 0, c->stream>>>(__VA_ARGS__); \
            else kern<3, G3><<<group_blocks(c->n, G3), kBlock, 0, c->stream>>>(__VA_ARGS__); \
        } else {                                                                          \
            if (wide) kern<2, 2 * G2><<<group_blocks(c->n, 2 * G2), kBlock, 0, c->stream>>>(__VA_ARGS__); \
            else kern<2, G2><<<group_blocks(c->n, G2), kBlock, 0, c->stream>>>(__VA_ARGS__); \
        }                                                                                 \
        vmps_count_launch(1);                                                             \
    } while (0)
#define LAUNCH_GROUP(G, kern, ...)                                                        \
    do {                                                                                  \
        if (c->cfg.dim == 3)                                                              \
            kern<3><<<group_blocks(c->n, G), kBlock, 0, c->stream>>>(__VA_ARGS__);        \
        else                                                                              \
            kern<2><<<group_blocks(c->n, G), kBlock, 0, c->stream>>>(__VA_ARGS__);        \
        vmps_count_launch(1);                                                             \
    } while (0)
#define LAUNCH_WARP(kern, ...)                                                            \
    do {                                                                                  \
        if (c->cfg.dim == 3)                                                              \
            kern<3><<<group_blocks(c->n, 32), kBlock, 0, c->stream>>>(__VA_ARGS__);       \
        else                                                                              \
            kern<2><<<group_blocks(c->n, 32), kBlock, 0, c->stream>>>(__VA_ARGS__);       \
        vmps_count_launch(1);                                                             \
    } while (0)

}  // namespace

// FP32 copies relative to (x0, y0, z0); w = ptype when given, else 0
__global__ void k_pack_f(int n, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, double x0, double y0, double z0,
                         const int* __restrict__ ptype, float4* __restrict__ P4f)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        P4f[i] = make_float4((float)(x[i] - x0), (float)(y[i] - y0), (float)(z[i] - z0),
                             ptype ? (float)ptype[i] : 0.f);
}

int vmps_pack(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    k_pack_f<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->x, c->y, c->z, f.xmin, f.ymin,
                                                          f.dim == 3 ? f.zmin : 0.0, c->ptype,
                                                          c->P4f);
    vmps_count_launch(1);
    if (f.precision >= 1) {
        k_pack_f<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->u, c->v, c->w, 0.0, 0.0,
                                                              0.0, nullptr, c->U4f);
        vmps_count_launch(1);
    }
    k_pack<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->x, c->y, c->z, c->ptype, c->P4);
    k_pack<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->u, c->v, c->w, nullptr, c->U4);
    vmps_count_launch(2);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

// the packed velocities alone (mps_step_io's deferred velocities)
int vmps_pack_u(mps_ctx* c)
{
    if (c->cfg.precision >= 1) {
        k_pack_f<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->u, c->v, c->w, 0.0, 0.0,
                                                              0.0, nullptr, c->U4f);
        vmps_count_launch(1);
    }
    k_pack<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->u, c->v, c->w, nullptr, c->U4);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_pnd(mps_ctx* c, int at_star, int correct, int which, double* out, bool track_max)
{
    double re = which == 0 ? c->cfg.re_l : c->cfg.re_s;
    // the maximum is wanted once (n0); per step its atomics would all hit
    // one address
    unsigned long long* dmax = track_max ? c->d_max : nullptr;
    const double4* P = at_star ? c->P4s : c->P4;
    WK wk = make_wk(c->cfg.ktype, re);
    if (which == 0) {
        if (c->cfg.dim == 3)
            k_pnd<3, 32><<<group_blocks(c->n, 32), kBlock, 0, c->stream>>>(
                c->n, lists(c, 0), P, wk, correct, c->cfg.ncorrection, out, dmax);
        else
            k_pnd<2, 32><<<group_blocks(c->n, 32), kBlock, 0, c->stream>>>(
                c->n, lists(c, 0), P, wk, correct, c->cfg.ncorrection, out, dmax);
        vmps_count_launch(1);
    } else if (at_star && !correct && c->cfg.precision == 2 && c->P4sf) {
        // precision 2: n* from the FP32 predicted positions
        LAUNCH_SMALL(k_pnd32, c->n, lists(c, 1), c->P4sf, make_wkf(wk), out);
    } else {
        LAUNCH_SMALL(k_pnd, c->n, lists(c, 1), P, wk, correct, c->cfg.ncorrection, out, dmax);
    }
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_bcon(mps_ctx* c)
{
    k_bcon<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(
        c->n, c->ptype, c->nds, c->n0_s, c->cfg.dirichlet, c->bcon,
        c->cfg.ppe_at_predicted ? c->P4s : nullptr);
    c->p4s_bcon = c->cfg.ppe_at_predicted != 0;
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_vfraction(mps_ctx* c)
{
    // without second-fluid particles every sum2 is 0, so C = 0 everywhere
    // (sum1 = 0 also gives 0): no neighbour pass
    if (c->fp2 == 0) {
        VMPS_CUDA(c, cudaMemsetAsync(c->C, 0, sizeof(double) * c->n, c->stream));
        return MPS_OK;
    }
    LAUNCH_SMALL(k_vfraction, c->n, lists(c, 1), c->ptype, c->P4, make_wk(c->cfg.ktype, c->cfg.re_s),
               c->cfg.fraction_method, c->C);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_viscosity(mps_ctx* c)
{
    LAUNCH_SMALL(k_viscosity, c->n, lists(c, 1), phys(c), c->ptype, c->P4, c->un, c->vn, c->wn, c->C,
               c->phat, c->meu);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_sps(mps_ctx* c)
{
    Phys P = phys(c);
    LAUNCH_SMALL(k_sps1, c->n, lists(c, 1), P, c->ptype, c->P4, c->un, c->vn, c->wn, c->S6, c->neut);
    LAUNCH_SMALL(k_sps2, c->n, lists(c, 1), P, c->ptype, c->P4, c->S6, c->neut, c->t1, c->t2, c->t3);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_predict(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    PredArgs A;
    A.ws = make_wk(f.ktype, f.re_s);
    A.wl = make_wk(f.ktype, f.re_l);
    A.n0_s = c->n0_s;
    // 4*DT/(lambda*n0) of the viscous term (functions.cu:2361; "4" is the
    // reference's 2*d with d = 2, kept in 3D as well)
    A.visc_coef = 4 * f.dt / (c->lambda_l * c->n0_l);
    A.dt = f.dt; A.gx = f.gx; A.gy = f.gy; A.gz = f.gz; A.relaxp = f.relaxp;
    A.rho1 = f.rho1; A.rho2 = f.rho2;
    // the same products VISCOSITY forms (k_viscosity, fluid2_type 0)
    A.meu_by_kind = f.fluid2_type == 0 ? 1 : 0;
    A.meu1 = f.nu1 * f.rho1;
    A.meu2 = f.nu2 * f.rho2;
    k_pack_pp<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->x, c->y, c->z, c->pnew, c->PP4);
    vmps_count_launch(1);
    LAUNCH_SMALL(k_predict_p, c->n, lists(c, 1), A, c->P4, c->PP4, c->phat, c->rho, c->pres_x,
                 c->pres_y, c->pres_z);
    // without SPS, neut is 0 and the eddy-viscosity sums are left out
#define PRED32(D, T)                                                                          \
    k_predict32<D, T><<<group_blocks(c->n, kPred32G), kBlock, 0, c->stream>>>(                 \
        c->n, lists(c, 0), A, make_wkf(A.wl), c->meu, c->P4, c->U4, c->P4f, c->U4f, c->pres_x, \
        c->pres_y, c->pres_z, c->neut, c->t1, c->t2, c->t3, c->xs, c->ys, c->zs, c->us, c->vs,  \
        c->ws, c->P4s, c->P4sf, make_double3(f.xmin, f.ymin, f.dim == 3 ? f.zmin : 0.0))
#define PRED64(D, T)                                                                          \
    k_predict<D, T><<<group_blocks(c->n, kPredG), kBlock, 0, c->stream>>>(                     \
        c->n, lists(c, 0), A, c->meu, c->P4, c->U4, c->pres_x, c->pres_y, c->pres_z, c->neut,  \
        c->t1, c->t2, c->t3, c->xs, c->ys, c->zs, c->us, c->vs, c->ws, c->P4s)
    const bool turb = f.turb != 0;
    c->p4s_bcon = false;  // P4s.w is ptype again until BCON
    if (f.precision >= 1) {  // FP32 neighbour sums
        if (f.dim == 3) { if (turb) PRED32(3, true); else PRED32(3, false); }
        else { if (turb) PRED32(2, true); else PRED32(2, false); }
    } else {
        if (f.dim == 3) { if (turb) PRED64(3, true); else PRED64(3, false); }
        else { if (turb) PRED64(2, true); else PRED64(2, false); }
    }
#undef PRED32
#undef PRED64
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_pressure_wc(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    k_pressure_wc<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(
        c->n, c->ptype, c->C, c->nds, c->n0_s, f.beta_fs, f.c01, f.c02, f.rho1, f.rho2, f.pmin,
        f.pmax, c->pnew);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_phat(mps_ctx* c)
{
    const int G = (c->cfg.dim == 3 ? SmallG<3>::G : SmallG<2>::G) * (c->tune_small_wide ? 2 : 1);
    if (G == 16)
        k_phat<16><<<group_blocks(c->n, 16), kBlock, 0, c->stream>>>(c->n, lists(c, 1), c->pnew,
                                                                     c->phat, c->PH, c->PH32);
    else if (G == 8)
        k_phat<8><<<group_blocks(c->n, 8), kBlock, 0, c->stream>>>(c->n, lists(c, 1), c->pnew,
                                                                   c->phat, c->PH, c->PH32);
    else
        k_phat<4><<<group_blocks(c->n, 4), kBlock, 0, c->stream>>>(c->n, lists(c, 1), c->pnew,
                                                                   c->phat, c->PH, c->PH32);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_pressgrad(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    GradArgs A;
    A.wk = make_wk(f.ktype, f.re_s);
    A.coef = f.relaxp * (2.0 * f.dt / c->n0_s);
    A.vmax = f.vmax;
    A.kh = f.kh;
    if (f.precision == 2)
        LAUNCH_SMALL(k_pressgrad32, c->n, lists(c, 1), A, make_wkf(A.wk), c->ptype, c->PH32,
                     c->P4sf, c->rho, c->us, c->vs, c->ws, c->un, c->vn, c->wn);
    else
        LAUNCH_SMALL(k_pressgrad, c->n, lists(c, 1), A, c->ptype, c->PH, c->P4s, c->rho, c->us,
                     c->vs, c->ws, c->un, c->vn, c->wn);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_integrate(mps_ctx* c)
{
    LAUNCH_DIM(k_integrate, c->n, box(c), c->ptype, c->x, c->y, c->z, c->un, c->vn, c->wn, c->P4);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_collision(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    CollArgs A{sqrt_cut(f.coll, true), f.cc, f.dt, f.rho1, f.rho2};
    // new states to the *c scratch arrays, then copied over in place
    LAUNCH_SMALL(k_collision, c->n, lists(c, 1), A, c->ptype, c->oid, c->P4, c->un, c->vn, c->wn,
                 c->xc, c->yc, c->zc, c->uc, c->vc, c->wc);
    LAUNCH_DIM(k_collision_apply, c->n, c->ptype, c->x, c->y, c->z, c->un, c->vn, c->wn, c->xc,
               c->yc, c->zc, c->uc, c->vc, c->wc, c->P4);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_commit(mps_ctx* c)
{
    LAUNCH_DIM(k_commit, c->n, box(c), c->ptype, c->x, c->y, c->z, c->u, c->v, c->w, c->p, c->un,
               c->vn, c->wn, c->pnew, c->d_err);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}
