// mps_stages.cu -- explicit per-particle stages of one MPS step.
//
// One thread per particle, neighbours visited in list order and accumulated
// in FP64 with the reference's evaluation order (this unit is compiled with
// -fmad=false), so each stage reproduces the oracle's sums.  Lists are the
// slot-major ELL built by mps_neighbors.cu.  Reference routines are cited on
// each kernel.
#include "mps_internal.cuh"

using namespace vmps;

namespace {

struct Lists {
    const int* __restrict__ nbr;
    const int* __restrict__ len;
    int pitch;
};

__device__ __forceinline__ int nb(const Lists& L, int k, int i)
{
    return L.nbr[(size_t)k * L.pitch + i];
}

template <int DIM>
__device__ __forceinline__ double dist_ij(const double* x, const double* y, const double* z, int i,
                                          int j)
{
    double dz = DIM == 3 ? z[j] - z[i] : 0.0;
    return sqrt(dist2<DIM>(x[j] - x[i], y[j] - y[i], dz));
}

// PNUM / PNUMSTAR (functions.cu:94-122, 157-179)
template <int DIM>
__global__ void k_pnd(int n, Lists L, const double* __restrict__ x, const double* __restrict__ y,
                      const double* __restrict__ z, double re, int ktype, int correct,
                      double ncorr, double* __restrict__ out, unsigned long long* dmax)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sum = 0.0;
    int len = L.len[i];
    for (int k = 0; k < len; k++) {
        int j = nb(L, k, i);
        double d = dist_ij<DIM>(x, y, z, i, j);
        if (i != j) sum = sum + kernel_w(d, ktype, DIM, re);
    }
    if (correct && ktype != 2) sum = sum * ncorr;
    out[i] = sum;
    if (dmax && sum > 0.0) atomicMax(dmax, (unsigned long long)__double_as_longlong(sum));
}

// BCON (functions.cu:433-445)
__global__ void k_bcon(int n, const int* __restrict__ ptype, const double* __restrict__ nd,
                       double n0, double dirichlet, int* __restrict__ bcon)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int b;
    if (ptype[i] <= -1) b = -1;
    else if (nd[i] / n0 < dirichlet) b = 1;
    else b = 0;
    bcon[i] = b;
}

// V_FRACTION (functions.cu:2580-2638)
template <int DIM>
__global__ void k_vfraction(int n, Lists L, const int* __restrict__ ptype,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, double re, int ktype, int method,
                            double* __restrict__ C)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    double sum1 = 0, sum2 = 0;
    int len = L.len[I];
    for (int k = 0; k < len; k++) {
        int J = nb(L, k, I);
        int pj = ptype[J];
        if (method == 1) {
            if (I != J && pj > 0) {
                sum1 = sum1 + 1;
                if (pj == 2) sum2 = sum2 + 1;
            }
        } else {
            double d = dist_ij<DIM>(x, y, z, I, J);
            if (I != J && pj > 0) {
                double w = kernel_w(d, ktype, DIM, re);
                sum1 = sum1 + w;
                if (pj == 2) sum2 = sum2 + w;
            }
        }
    }
    double c = sum2 / sum1;
    if (sum1 == 0) c = 0;
    C[I] = c;
}

// velocity-gradient sums of VISCOSITY / SPS (functions.cu:2096-2117, 1734-1756)
template <int DIM>
__device__ __forceinline__ void grad_sums(const Lists& L, int I, const double* x, const double* y,
                                          const double* z, const double* un, const double* vn,
                                          const double* wn, double re, int ktype, double mind,
                                          double* s)
{
    for (int k = 0; k < 9; k++) s[k] = 0.0;
    int len = L.len[I];
    double xi = x[I], yi = y[I], zi = DIM == 3 ? z[I] : 0.0;
    double ui = un[I], vi = vn[I], wi = DIM == 3 ? wn[I] : 0.0;
    for (int k = 0; k < len; k++) {
        int j = nb(L, k, I);
        double dx = x[j] - xi, dy = y[j] - yi, dz = DIM == 3 ? z[j] - zi : 0.0;
        double d = sqrt(dist2<DIM>(dx, dy, dz));
        if (I != j && (mind < 0 || d > mind)) {
            double w = kernel_w(d, ktype, DIM, re);
            double du = un[j] - ui, dv = vn[j] - vi;
            s[0] = s[0] + du * dx * w / d / d;
            s[1] = s[1] + dv * dy * w / d / d;
            s[2] = s[2] + du * dy * w / d / d;
            s[3] = s[3] + dv * dx * w / d / d;
            if (DIM == 3) {
                double dw = wn[j] - wi;
                s[4] = s[4] + dw * dz * w / d / d;
                s[5] = s[5] + du * dz * w / d / d;
                s[6] = s[6] + dv * dz * w / d / d;
                s[7] = s[7] + dw * dx * w / d / d;
                s[8] = s[8] + dw * dy * w / d / d;
            }
        }
    }
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
    double rho1, rho2, nu1, nu2, n0, meu0, n_pl, phi, cohes, cs, l0, mind;
    int ktype, fluid2_type;
    double re;
};

// VISCOSITY (functions.cu:2053-2184); reads C[i] where the reference reads
// C[0] (identical whenever phi == 0)
template <int DIM>
__global__ void k_viscosity(int n, Lists L, Phys P, const int* __restrict__ ptype,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ un,
                            const double* __restrict__ vn, const double* __restrict__ wn,
                            const double* __restrict__ C, const double* __restrict__ phat,
                            double* __restrict__ meu)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int pt = ptype[i];
    if (P.fluid2_type == 0) {
        if (pt <= 1) meu[i] = P.nu1 * P.rho1;
        if (pt == 2) meu[i] = P.nu2 * P.rho2;
        return;
    }
    if (pt == 1) {
        meu[i] = P.nu1 * P.rho1;
        return;
    }
    double s[9], S[6];
    grad_sums<DIM>(L, i, x, y, z, un, vn, wn, P.re, P.ktype, -1.0, s);
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
template <int DIM>
__global__ void k_sps1(int n, Lists L, Phys P, const int* __restrict__ ptype,
                       const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, const double* __restrict__ un,
                       const double* __restrict__ vn, const double* __restrict__ wn,
                       double* __restrict__ S6, double* __restrict__ neut)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || ptype[i] < 0) return;
    double s[9], S[6];
    grad_sums<DIM>(L, i, x, y, z, un, vn, wn, P.re, P.ktype, P.mind, s);
    strain<DIM>(P.n0, s, S);
    for (int c = 0; c < 6; c++) S6[(size_t)c * n + i] = S[c];
    double S11 = S[0], S12 = S[1], S22 = S[2], S13 = S[3], S23 = S[4], S33 = S[5];
    double Sm;
    if (DIM == 3)
        Sm = pow(2 * S11 * S11, 0.5) + 2 * pow(2 * S12 * S12, 0.5) + pow(2 * S22 * S22, 0.5) +
             pow(2 * S33 * S33, 0.5) + 2 * pow(2 * S13 * S13, 0.5) + 2 * pow(2 * S23 * S23, 0.5);
    else
        Sm = pow(2 * S11 * S11, 0.5) + 2 * pow(2 * S12 * S12, 0.5) + pow(2 * S22 * S22, 0.5);
    double cd = P.cs * P.l0;
    neut[i] = (cd * cd) * Sm;
}

// SPS pass 2: divergence of the SPS stress (functions.cu:1793-1830)
template <int DIM>
__global__ void k_sps2(int n, Lists L, Phys P, const int* __restrict__ ptype,
                       const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, const double* __restrict__ S6,
                       const double* __restrict__ neut, double* __restrict__ t1,
                       double* __restrict__ t2, double* __restrict__ t3)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || ptype[i] < 0) return;
    double sum1 = 0, sum2 = 0, sum3 = 0;
    int len = L.len[i];
    double ni = neut[i];
    for (int k = 0; k < len; k++) {
        int j = nb(L, k, i);
        double dx = x[j] - x[i], dy = y[j] - y[i], dz = DIM == 3 ? z[j] - z[i] : 0.0;
        double d = sqrt(dist2<DIM>(dx, dy, dz));
        if (i != j && d > P.mind) {
            double w = kernel_w(d, P.ktype, DIM, P.re);
            sum1 = sum1 + (neut[j] - ni) * dx * w / d / d;
            sum2 = sum2 + (neut[j] - ni) * dy * w / d / d;
            if (DIM == 3) sum3 = sum3 + (neut[j] - ni) * dz * w / d / d;
        }
    }
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
    double re_s, n0_s, re_l, n0_l, lambda_l, dt, gx, gy, gz, relaxp, rho1, rho2;
    int ktype;
};

// PREDICTION (functions.cu:2283-2369): explicit pressure sums over the PND
// list, viscous Laplacian over the Laplacian list.
template <int DIM>
__global__ void k_predict(int n, Lists Ls, Lists Ll, PredArgs A, const int* __restrict__ ptype,
                          const double* __restrict__ meu, const double* __restrict__ x,
                          const double* __restrict__ y, const double* __restrict__ z,
                          const double* __restrict__ u, const double* __restrict__ v,
                          const double* __restrict__ w, const double* __restrict__ pnew,
                          const double* __restrict__ phat, const double* __restrict__ neut,
                          const double* __restrict__ t1, const double* __restrict__ t2,
                          const double* __restrict__ t3, const double* __restrict__ rho,
                          double* __restrict__ xs, double* __restrict__ ys,
                          double* __restrict__ zs, double* __restrict__ us,
                          double* __restrict__ vs, double* __restrict__ ws)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    int pI = ptype[I];
    if (pI <= 0) {
        xs[I] = x[I]; ys[I] = y[I]; us[I] = u[I]; vs[I] = v[I];
        if (DIM == 3) { zs[I] = z[I]; ws[I] = w[I]; }
        return;
    }
    double xi = x[I], yi = y[I], zi = DIM == 3 ? z[I] : 0.0;
    double sum1 = 0, sum2 = 0, sum3 = 0, sum4 = 0, sum5 = 0, sum6 = 0, sum7 = 0, sum8 = 0, sum9 = 0;
    double ph = phat[I];
    int len = Ls.len[I];
    for (int k = 0; k < len; k++) {
        int J = nb(Ls, k, I);
        double dx = x[J] - xi, dy = y[J] - yi, dz = DIM == 3 ? z[J] - zi : 0.0;
        double D = sqrt(dist2<DIM>(dx, dy, dz));
        if (I != J && D > 0) {
            double W = kernel_w(D, A.ktype, DIM, A.re_s);
            double pp = pnew[J] - ph;
            sum1 = sum1 + pp * dx * W / D / D;
            sum2 = sum2 + pp * dy * W / D / D;
            if (DIM == 3) sum3 = sum3 + pp * dz * W / D / D;
        }
    }
    double mI = meu[I], uI = u[I], vI = v[I], wI = DIM == 3 ? w[I] : 0.0;
    len = Ll.len[I];
    for (int k = 0; k < len; k++) {
        int J = nb(Ll, k, I);
        double dx = x[J] - xi, dy = y[J] - yi, dz = DIM == 3 ? z[J] - zi : 0.0;
        double D = sqrt(dist2<DIM>(dx, dy, dz));
        if (I != J && D > 0) {
            double NEU;
            if (pI == ptype[J]) {
                NEU = (pI == 1) ? mI / A.rho1 : mI / A.rho2;
            } else {
                double mJ = meu[J];
                NEU = (pI == 1) ? 2 * mI * mJ / (mI + mJ) / A.rho1 : 2 * mI * mJ / (mI + mJ) / A.rho2;
            }
            double W = kernel_w(D, A.ktype, DIM, A.re_l);
            double du = u[J] - uI, dv = v[J] - vI;
            sum4 = sum4 + W * du * NEU;
            sum5 = sum5 + W * dv * NEU;
            sum7 = sum7 + W * du;
            sum8 = sum8 + W * dv;
            if (DIM == 3) {
                double dw = w[J] - wI;
                sum6 = sum6 + W * dw * NEU;
                sum9 = sum9 + W * dw;
            }
        }
    }
    double DT = A.dt, rp = 1 - A.relaxp, nt = neut[I], r = rho[I];
    double uS = uI + A.gx * DT + 4 * DT * (sum4 + nt * sum7) / (A.lambda_l * A.n0_l) + DT * t1[I] -
                rp * (2.0 * DT / A.n0_s / r) * sum1;
    double vS = vI + A.gy * DT + 4 * DT * (sum5 + nt * sum8) / (A.lambda_l * A.n0_l) + DT * t2[I] -
                rp * (2.0 * DT / A.n0_s / r) * sum2;
    us[I] = uS;
    vs[I] = vS;
    xs[I] = xi + DT * uS;
    ys[I] = yi + DT * vS;
    if (DIM == 3) {
        double wS = wI + A.gz * DT + 4 * DT * (sum6 + nt * sum9) / (A.lambda_l * A.n0_l) +
                    DT * t3[I] - rp * (2.0 * DT / A.n0_s / r) * sum3;
        ws[I] = wS;
        zs[I] = zi + DT * wS;
    }
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

// PHATCALC (functions.cu:207-224)
__global__ void k_phat(int n, Lists L, const double* __restrict__ pnew, double* __restrict__ phat)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n) return;
    double mn = 999999999999999;
    int len = L.len[I];
    for (int k = 0; k < len; k++) {
        double pj = pnew[nb(L, k, I)];
        if (pj < mn) mn = pj;
    }
    phat[I] = mn;
}

struct GradArgs {
    double re, n0, dt, relaxp, vmax;
    int ktype, kh;
};

// PRESSGRAD (functions.cu:245-355), CPU semantics (p^_i + p^_j)
template <int DIM>
__global__ void k_pressgrad(int n, Lists L, GradArgs A, const int* __restrict__ ptype,
                            const double* __restrict__ pnew, const double* __restrict__ phat,
                            const double* __restrict__ xs, const double* __restrict__ ys,
                            const double* __restrict__ zs, const double* __restrict__ rho,
                            const double* __restrict__ us, const double* __restrict__ vs,
                            const double* __restrict__ ws, double* __restrict__ un,
                            double* __restrict__ vn, double* __restrict__ wn)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n || ptype[I] <= 0) return;
    double sum1 = 0, sum2 = 0, sum3 = 0;
    double xi = xs[I], yi = ys[I], zi = DIM == 3 ? zs[I] : 0.0;
    double pi = pnew[I], phi = phat[I];
    int len = L.len[I];
    for (int k = 0; k < len; k++) {
        int J = nb(L, k, I);
        double dx = xs[J] - xi, dy = ys[J] - yi, dz = DIM == 3 ? zs[J] - zi : 0.0;
        double D = sqrt(dist2<DIM>(dx, dy, dz));
        if (I != J) {
            double w = kernel_w(D, A.ktype, DIM, A.re);
            double pp = (A.kh == 1) ? pnew[J] + pi - (phi + phat[J]) : pnew[J] - phi;
            sum1 = sum1 + pp * dx * w / D / D;
            sum2 = sum2 + pp * dy * w / D / D;
            if (DIM == 3) sum3 = sum3 + pp * dz * w / D / D;
        }
    }
    double Rho = rho[I], DT = A.dt, VMAX = A.vmax, coeff = 2.0;
    double uN = us[I] - A.relaxp * (2.0 * DT / A.n0 / Rho) * sum1;
    double vN = vs[I] - A.relaxp * (2.0 * DT / A.n0 / Rho) * sum2;
    if (fabs(uN) > coeff * VMAX) uN = VMAX;
    if (vN > coeff * VMAX) vN = coeff * VMAX;
    if (vN < -coeff * VMAX) vN = -coeff * VMAX;
    un[I] = uN;
    vn[I] = vN;
    if (DIM == 3) {
        double wN = ws[I] - A.relaxp * (2.0 * DT / A.n0 / Rho) * sum3;
        if (fabs(wN) > coeff * VMAX) wN = VMAX;
        wn[I] = wN;
    }
}

struct Box {
    double xmin, xmax, ymin, ymax, zmin, zmax, dl, dt, cc;
};

// EULERINTEGRATION + BOUNDARIE (functions.cu:1963-2021)
template <int DIM>
__global__ void k_integrate(int n, Box B, const int* __restrict__ ptype, double* __restrict__ x,
                            double* __restrict__ y, double* __restrict__ z,
                            double* __restrict__ un, double* __restrict__ vn,
                            double* __restrict__ wn)
{
    int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= n || ptype[I] <= 0) return;
    double DT = B.dt, DL = B.dl, CC = B.cc;
    double xi = x[I] + un[I] * DT, yi = y[I] + vn[I] * DT;
    double ui = un[I], vi = vn[I];
    if (yi < B.ymin + DL * 3.0) { vi = fabs(vi) * CC; yi = B.ymin + DL * 3.0; }
    if (yi > B.ymax - DL * 3.0) { vi = -fabs(vi) * CC; yi = B.ymax - DL * 3.0; }
    if (xi < B.xmin + DL * 3.0) { ui = fabs(ui) * CC; xi = B.xmin + DL * 3.0; }
    if (xi > B.xmax - DL * 3.0) { ui = -fabs(ui) * CC; xi = B.xmax - DL * 3.0; }
    if (DIM == 3) {
        double zi = z[I] + wn[I] * DT, wi = wn[I];
        if (zi < B.zmin + DL * 3.0) { wi = fabs(wi) * CC; zi = B.zmin + DL * 3.0; }
        if (zi > B.zmax - DL * 3.0) { wi = -fabs(wi) * CC; zi = B.zmax - DL * 3.0; }
        z[I] = zi;
        wn[I] = wi;
    }
    x[I] = xi; y[I] = yi; un[I] = ui; vn[I] = vi;
}

struct CollArgs {
    double coll, cc, dt, rho1, rho2;
};

// COLLISION2 (functions.cu:1523-1601) in its order-independent form: each
// fluid particle gathers the impulse of every approaching pair (d < coll)
// from the pre-collision state.  Writes the new state to the *o arrays.
template <int DIM>
__global__ void k_collision(int n, Lists L, CollArgs A, const int* __restrict__ ptype,
                            const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ un,
                            const double* __restrict__ vn, const double* __restrict__ wn,
                            double* __restrict__ xo, double* __restrict__ yo,
                            double* __restrict__ zo, double* __restrict__ uo,
                            double* __restrict__ vo, double* __restrict__ wo)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xi = x[i], yi = y[i], zi = DIM == 3 ? z[i] : 0.0;
    double ui = un[i], vi = vn[i], wi = DIM == 3 ? wn[i] : 0.0;
    int pi = ptype[i];
    double du = 0, dv = 0, dw = 0, ddx = 0, ddy = 0, ddz = 0;
    if (pi > 0) {
        double m1 = (pi == 1) ? A.rho1 : A.rho2;
        int len = L.len[i];
        for (int k = 0; k < len; k++) {
            int j = nb(L, k, i);
            double ex = x[j] - xi, ey = y[j] - yi, ez = DIM == 3 ? z[j] - zi : 0.0;
            double d = sqrt(dist2<DIM>(ex, ey, ez));
            if (i == j || !(d < A.coll)) continue;
            double m2 = (ptype[j] == 1) ? A.rho1 : A.rho2;
            double ug = (m1 * ui + m2 * un[j]) / (m1 + m2);
            double vg = (m1 * vi + m2 * vn[j]) / (m1 + m2);
            double ur = m1 * (ui - ug), vr = m1 * (vi - vg), vabs;
            double wr = 0;
            if (DIM == 3) {
                double wg = (m1 * wi + m2 * wn[j]) / (m1 + m2);
                wr = m1 * (wi - wg);
                vabs = (ur * ex + vr * ey + wr * ez) / d;
            } else {
                vabs = (ur * ex + vr * ey) / d;
            }
            if (!(vabs > 0)) continue;
            double um = (1.0 + A.cc) * vabs * ex / d;
            double vm = (1.0 + A.cc) * vabs * ey / d;
            du -= um / m1; dv -= vm / m1;
            ddx -= A.dt * um / m1; ddy -= A.dt * vm / m1;
            if (DIM == 3) {
                double wm = (1.0 + A.cc) * vabs * ez / d;
                dw -= wm / m1; ddz -= A.dt * wm / m1;
            }
        }
    }
    xo[i] = xi + ddx; yo[i] = yi + ddy; uo[i] = ui + du; vo[i] = vi + dv;
    if (DIM == 3) { zo[i] = zi + ddz; wo[i] = wi + dw; }
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
    double xi = x[I], yi = y[I];
    bool out = xi >= B.xmax || yi >= B.ymax || xi <= B.xmin || yi <= B.ymin;
    if (DIM == 3) out = out || z[I] >= B.zmax || z[I] <= B.zmin;
    if (bad) set_error(err, MPS_ERR_NAN);
    if (out) set_error(err, MPS_ERR_BOX);
}

Lists lists(mps_ctx* c, int which)
{
    Lists L;
    L.pitch = c->pitch;
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
    P.mind = f.coll / 10; P.ktype = f.ktype; P.fluid2_type = f.fluid2_type; P.re = f.re_s;
    return P;
}

Box box(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    Box B{f.xmin, f.xmax, f.ymin, f.ymax, f.zmin, f.zmax, f.l0, f.dt, f.velcor};
    return B;
}

#define LAUNCH_DIM(kern, ...)                                                             \
    do {                                                                                  \
        if (c->cfg.dim == 3) kern<3><<<grid_blocks(c->n), kBlock, 0, c->stream>>>(__VA_ARGS__); \
        else kern<2><<<grid_blocks(c->n), kBlock, 0, c->stream>>>(__VA_ARGS__);           \
        vmps_count_launch(1);                                                             \
    } while (0)

}  // namespace

int vmps_pnd(mps_ctx* c, int at_star, int correct, int which, double* out)
{
    const double *x = at_star ? c->xs : c->x, *y = at_star ? c->ys : c->y,
                 *z = at_star ? c->zs : c->z;
    double re = which == 0 ? c->cfg.re_l : c->cfg.re_s;
    LAUNCH_DIM(k_pnd, c->n, lists(c, which), x, y, z, re, c->cfg.ktype, correct,
               c->cfg.ncorrection, out, c->d_max);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_bcon(mps_ctx* c)
{
    k_bcon<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->ptype, c->nds, c->n0_s,
                                                        c->cfg.dirichlet, c->bcon);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_vfraction(mps_ctx* c)
{
    LAUNCH_DIM(k_vfraction, c->n, lists(c, 1), c->ptype, c->x, c->y, c->z, c->cfg.re_s,
               c->cfg.ktype, c->cfg.fraction_method, c->C);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_viscosity(mps_ctx* c)
{
    LAUNCH_DIM(k_viscosity, c->n, lists(c, 1), phys(c), c->ptype, c->x, c->y, c->z, c->un, c->vn,
               c->wn, c->C, c->phat, c->meu);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_sps(mps_ctx* c)
{
    Phys P = phys(c);
    LAUNCH_DIM(k_sps1, c->n, lists(c, 1), P, c->ptype, c->x, c->y, c->z, c->un, c->vn, c->wn,
               c->S6, c->neut);
    LAUNCH_DIM(k_sps2, c->n, lists(c, 1), P, c->ptype, c->x, c->y, c->z, c->S6, c->neut, c->t1,
               c->t2, c->t3);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_predict(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    PredArgs A{f.re_s, c->n0_s, f.re_l, c->n0_l, c->lambda_l, f.dt, f.gx, f.gy, f.gz, f.relaxp,
               f.rho1, f.rho2, f.ktype};
    LAUNCH_DIM(k_predict, c->n, lists(c, 1), lists(c, 0), A, c->ptype, c->meu, c->x, c->y, c->z,
               c->u, c->v, c->w, c->pnew, c->phat, c->neut, c->t1, c->t2, c->t3, c->rho, c->xs,
               c->ys, c->zs, c->us, c->vs, c->ws);
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
    k_phat<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, lists(c, 1), c->pnew, c->phat);
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_pressgrad(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    GradArgs A{f.re_s, c->n0_s, f.dt, f.relaxp, f.vmax, f.ktype, f.kh};
    LAUNCH_DIM(k_pressgrad, c->n, lists(c, 1), A, c->ptype, c->pnew, c->phat, c->xs, c->ys, c->zs,
               c->rho, c->us, c->vs, c->ws, c->un, c->vn, c->wn);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_integrate(mps_ctx* c)
{
    LAUNCH_DIM(k_integrate, c->n, box(c), c->ptype, c->x, c->y, c->z, c->un, c->vn, c->wn);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int vmps_collision(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    CollArgs A{f.coll, f.cc, f.dt, f.rho1, f.rho2};
    // the new state goes to the *c buffers, which then swap roles with it
    LAUNCH_DIM(k_collision, c->n, lists(c, 1), A, c->ptype, c->x, c->y, c->z, c->un, c->vn, c->wn,
               c->xc, c->yc, c->zc, c->uc, c->vc, c->wc);
    VMPS_CUDA(c, cudaGetLastError());
    std::swap(c->x, c->xc);
    std::swap(c->y, c->yc);
    std::swap(c->un, c->uc);
    std::swap(c->vn, c->vc);
    if (c->cfg.dim == 3) {
        std::swap(c->z, c->zc);
        std::swap(c->wn, c->wc);
    }
    return MPS_OK;
}

int vmps_commit(mps_ctx* c)
{
    LAUNCH_DIM(k_commit, c->n, box(c), c->ptype, c->x, c->y, c->z, c->u, c->v, c->w, c->p, c->un,
               c->vn, c->wn, c->pnew, c->d_err);
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}
