/*
 * mps_oracle.c -- CPU restatement of the VoxarMPS per-step pipeline.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): loaded by
 * tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py.
 *
 * Every routine cites the reference routine it restates
 * (VoxarMPS/VoxarMPS/functions.cu or main.cu).  Floating-point expressions
 * keep the reference's evaluation order so that, with re_s == re_l and the
 * reference's semantics switches, the results are the reference's bits.
 * gcc -O2 folds pow(x, 2.0) to x*x, exactly as in the reference's own -O2
 * build, so squared differences are written as products here.
 */
#include "mps_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* kernel function, functions.cu:32-74                                 */
/* ------------------------------------------------------------------ */
double mo_W(double R, int ktype, int dim, double re)
{
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
        double C = 0.0;
        if (dim == 1) C = 0.6666;
        if (dim == 2) C = 1.43 * 3.14;
        if (dim == 3) C = 1 / 3.14;
        if (R < re) w = C / pow(re, dim) * (1 - 1.5 * (q * q) + 0.75 * pow(q, 3.0));
        else if (R >= re && R < (2.0 * re)) w = C / pow(re, dim) * (0.25 * pow(2.0 - q, 3.0));
        else w = 0;
        break;
    }
    case 5:
        if (q <= 1.0) w = 1.5 * log(1 / (q + 0.000001));
        else w = 0;
        break;
    case 6:
        if (q <= 1.0) w = pow((1 - q), 3);
        else w = 0;
        break;
    }
    return w;
}

/* main.cu:491-494 */
double mo_lambda(int ktype, double re)
{
    if (ktype == 1) return 0.22143 * (re * re);
    if (ktype == 2) return 0.16832 * (re * re);
    if (ktype == 5) return 0.250 * (re * re);
    if (ktype == 6) return 0.14288 * (re * re);
    return 0.0;
}

/* dist2d / dist3d, functions.cu:76-89: sqrt(pow(dx,2)+pow(dy,2)[+pow(dz,2)]) */
static inline double dist(int dim, int i, int j, const double* x, const double* y,
                          const double* z)
{
    double dx = x[j] - x[i], dy = y[j] - y[i];
    if (dim == 3) {
        double dz = z[j] - z[i];
        return sqrt(dx * dx + dy * dy + dz * dz);
    }
    return sqrt(dx * dx + dy * dy);
}

/* ------------------------------------------------------------------ */
/* neighbour search, functions.cu:2788-2929                            */
/* ------------------------------------------------------------------ */
int mo_grid(const mo_params* P, double re, int* ncx, int* ncy, int* ncz)
{
    *ncx = (int)((P->xmax - P->xmin) / (re)) + 1;
    *ncy = (int)((P->ymax - P->ymin) / (re)) + 1;
    if (P->dim == 3) {
        *ncz = (int)((P->zmax - P->zmin) / (re + P->delta)) + 1;
        return (*ncx) * (*ncy) * (*ncz);
    }
    *ncz = 1;
    return (*ncx) * (*ncy);
}

/* Cell coordinates of one particle (functions.cu:2823-2835).  Returns 0 when
   the coordinate lies outside the grid, which the reference does not check. */
static int cell_of(const mo_params* P, double re, int ncx, int ncy, int ncz, double xi,
                   double yi, double zi, int* ic, int* jc, int* kc)
{
    double fx = (xi - P->xmin) / (re), fy = (yi - P->ymin) / (re);
    if (!(fx > -1.0 && fx < (double)ncx) || !(fy > -1.0 && fy < (double)ncy)) return 0;
    *ic = (int)fx + 1;
    *jc = (int)fy + 1;
    *kc = 1;
    if (P->dim == 3) {
        double fz = (zi - P->zmin) / (re + P->delta);
        if (!(fz > -1.0 && fz < (double)ncz)) return 0;
        *kc = (int)fz + 1;
    }
    return (*ic >= 1 && *ic <= ncx && *jc >= 1 && *jc <= ncy && *kc >= 1 && *kc <= ncz);
}

int mo_neighbor(const mo_params* P, double re, int n, const double* x, const double* y,
                const double* z, int* cell, int* perm, int* off, int* nbr, int cap)
{
    int ncx, ncy, ncz;
    int tnc = mo_grid(P, re, &ncx, &ncy, &ncz);
    int* cnt = (int*)calloc((size_t)tnc + 2, sizeof(int));
    int* cst = (int*)calloc((size_t)tnc + 2, sizeof(int));
    int* ci = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1) * 3);
    int bad = 0;
    for (int k = 0; k < n; k++) {
        int a, b, c;
        if (!cell_of(P, re, ncx, ncy, ncz, x[k], y[k], P->dim == 3 ? z[k] : 0.0, &a, &b, &c)) {
            bad = 1;
            a = b = c = 1;
        }
        ci[3 * k] = a; ci[3 * k + 1] = b; ci[3 * k + 2] = c;
        int Cnum = a + (b - 1) * ncx + (c - 1) * ncx * ncy;
        cell[k] = Cnum;
        cnt[Cnum]++;
    }
    if (bad) { free(cnt); free(cst); free(ci); return MO_ERR_CELL; }
    /* The reference's insertion loop (functions.cu:2820-2852) is a stable
       counting sort: ip[] lists particles by cell, ascending index in a cell. */
    int acc = 0;
    for (int c = 1; c <= tnc; c++) { cst[c] = acc; acc += cnt[c]; }
    cst[tnc + 1] = acc;
    {
        int* fill = (int*)calloc((size_t)tnc + 2, sizeof(int));
        for (int k = 0; k < n; k++) perm[cst[cell[k]] + fill[cell[k]]++] = k;
        free(fill);
    }
    /* scan: row (x) outer, colu (y), dep (z) inner (functions.cu:2854-2918) */
    int total = 0;
    int over = 0;
    double cut3 = re + P->delta;
    for (int I = 0; I < n; I++) {
        int icell = ci[3 * I], jcell = ci[3 * I + 1], kcell = ci[3 * I + 2];
        int m1 = (icell == 1) ? 0 : -1, m2 = (icell == ncx) ? 0 : 1;
        int m3 = (jcell == 1) ? 0 : -1, m4 = (jcell == ncy) ? 0 : 1;
        off[I] = total;
        if (P->dim == 3) {
            int m5 = (kcell == 1) ? 0 : -1, m6 = (kcell == ncz) ? 0 : 1;
            for (int row = m1; row <= m2; row++)
                for (int colu = m3; colu <= m4; colu++)
                    for (int dep = m5; dep <= m6; dep++) {
                        int Cnum = icell + row + (jcell - 1 + colu) * ncx +
                                   (kcell - 1 + dep) * ncx * ncy;
                        for (int JJ = cst[Cnum]; JJ < cst[Cnum] + cnt[Cnum]; JJ++) {
                            int J = perm[JJ];
                            if (dist(3, I, J, x, y, z) <= cut3) {
                                if (total < cap) nbr[total] = J; else over = 1;
                                total++;
                            }
                        }
                    }
        } else {
            for (int row = m1; row <= m2; row++)
                for (int colu = m3; colu <= m4; colu++) {
                    int Cnum = icell + row + (jcell - 1 + colu) * ncx;
                    for (int JJ = cst[Cnum]; JJ < cst[Cnum] + cnt[Cnum]; JJ++) {
                        int J = perm[JJ];
                        if (I == J) continue;
                        if (dist(2, I, J, x, y, z) < re) {
                            if (total < cap) nbr[total] = J; else over = 1;
                            total++;
                        }
                    }
                }
        }
    }
    off[n] = total;
    free(cnt); free(cst); free(ci);
    return over ? -total : total;
}

/* ------------------------------------------------------------------ */
/* PND, functions.cu:94-122 (PNUM) and 157-179 (PNUMSTAR)              */
/* ------------------------------------------------------------------ */
void mo_pnd(const mo_params* P, double re, int n, const int* off, const int* nbr,
            const double* x, const double* y, const double* z, int correct, double* nd)
{
    for (int I = 0; I < n; I++) {
        double sum = 0.0;
        for (int l = off[I]; l < off[I + 1]; l++) {
            int J = nbr[l];
            double d = dist(P->dim, I, J, x, y, z);
            if (I != J) sum = sum + mo_W(d, P->ktype, P->dim, re);
        }
        if (correct && P->ktype != 2) sum = sum * P->ncorrection;
        nd[I] = sum;
    }
}

double mo_max(int n, const double* a)
{
    double m = 0.0; /* MAX[0] starts at 0 (main.cu:400) */
    for (int i = 0; i < n; i++) if (a[i] > m) m = a[i];
    return m;
}

/* BCON, functions.cu:433-445 */
void mo_bcon(int n, const int* ptype, const double* nd, double n0, double dirichlet, int* bcon)
{
    for (int i = 0; i < n; i++) {
        if (ptype[i] <= -1) bcon[i] = -1;
        else if (nd[i] / n0 < dirichlet) bcon[i] = 1;
        else bcon[i] = 0;
    }
}

/* ------------------------------------------------------------------ */
/* PPE matrix, functions.cu:869-922 (Method 1 branch).                 */
/* diag[i] = poiss[i][1]; val[l] = poiss[i][slot l] (negative values).  */
/* ------------------------------------------------------------------ */
void mo_matrix(const mo_params* P, double re, double lambda, double n0, int n, const int* off,
               const int* nbr, const double* x, const double* y, const double* z,
               const int* bcon, double* diag, double* val)
{
    int dim = P->dim;
    double Rho = P->rho1; /* PRESSURECALC passes Rho1 (main.cu:1149) */
    for (int i = 0; i < n; i++) {
        diag[i] = 0.0;
        for (int l = off[i]; l < off[i + 1]; l++) val[l] = 0.0;
        if (bcon[i] != 0) continue;
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (i == j) continue;
            if (bcon[j] == -1) { val[l] = 0.0; continue; }
            double d = dist(dim, i, j, x, y, z);
            if (fabs(d) <= 1.0e-15) continue;
            double v;
            if (P->matopt) {
                v = (dim == 2) ? 3.0 * re : 2.0 * re;
                v = v / (d * d * d);
                v = v / n0;
                v = v / Rho;
            } else {
                v = 2.0 * dim / lambda * mo_W(d, P->ktype, dim, re) / n0 / Rho;
            }
            val[l] = -v;
            diag[i] += v;
        }
        diag[i] += (1.00e-7) / P->dt / P->dt;
    }
}

/* source without srcopt, functions.cu:990-1003 (nsrc = n on the CPU path,
   n* on the GPU path, functions.cu:1126) */
void mo_source(const mo_params* P, double n0, int n, const int* ptype, const int* bcon,
               const double* nsrc, double* source)
{
    double DT = P->dt;
    for (int i = 0; i < n; i++) {
        if (ptype[i] == -1) continue;
        if (bcon[i] == 0) source[i] = 1.0 / DT / DT * (nsrc[i] - n0) / n0;
        else if (bcon[i] == 1) source[i] = 0.0;
    }
}

/* HS + ECS source (srcopt), functions.cu:924-988.  Sequential: each row
   reads the finished value of the previous particle's source.  alpha uses
   n* on both reference paths (MATRIX receives nstar, functions.cu:936). */
void mo_source_hs(const mo_params* P, double re, double n0, int n, const int* off,
                  const int* nbr, const int* ptype, const int* bcon, const double* nstar,
                  const double* x, const double* y, const double* z, const double* u,
                  const double* v, const double* w, double* source)
{
    double DT = P->dt;
    int dim = P->dim;
    for (int i = 0; i < n; i++) {
        if (ptype[i] == -1) continue;
        if (bcon[i] == 0) {
            double alpha = 0.0, beta = 0.0, ECS = 0.0;
            if (i > 0) {
                alpha = (nstar[i] - n0) / n0;
                beta = (DT / n0) * (source[i - 1] / (-1.0 / (n0 * DT)));
                ECS = fabs(alpha) * (beta / DT) + fabs(beta) * (alpha / DT);
            }
            double sum = 0.0;
            for (int l = off[i]; l < off[i + 1]; l++) {
                int j = nbr[l];
                if (ptype[j] <= -1 || i == j) continue;
                double d = dist(dim, i, j, x, y, z);
                if (fabs(d) <= 1.0e-15) continue;
                double du = u[i] - u[j], dv = v[i] - v[j];
                if (dim == 3) {
                    double dw = w[i] - w[j];
                    sum += (re / (d * d * d)) *
                           ((x[i] - x[j]) * du + (y[i] - y[j]) * dv + (z[i] - z[j]) * dw);
                } else {
                    sum += (re / (d * d * d)) * ((x[i] - x[j]) * du + (y[i] - y[j]) * dv);
                }
            }
            source[i] = (-1.25 / (n0 * DT)) * sum + ECS;
            if (fabs(source[i]) < 0.99) source[i] = 0;
        } else if (bcon[i] == 1) {
            source[i] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------ */
/* incomplete Cholesky, functions.cu:1139-1200                         */
/* ------------------------------------------------------------------ */
static int slot_of(const int* off, const int* nbr, int row, int col)
{
    for (int m = off[row]; m < off[row + 1]; m++) if (nbr[m] == col) return m;
    return -1;
}

void mo_incdecom(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
                 const double* val, double* icd, double* icv)
{
    memset(icd, 0, sizeof(double) * (size_t)n);
    memset(icv, 0, sizeof(double) * (size_t)off[n]);
    for (int i = 0; i < n; i++) {
        if (bcon[i] != 0) continue;
        double sum = diag[i];
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (j > i) continue;
            if (bcon[j] != 0) continue;
            sum = sum - icv[l] * icv[l];
        }
        icd[i] = sqrt(sum);
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (j < i) continue;
            if (bcon[j] != 0) continue;
            sum = val[l];
            for (int mj = off[j]; mj < off[j + 1]; mj++) {
                int kj = nbr[mj];
                if (kj >= i) continue;
                if (bcon[kj] != 0) continue;
                for (int mi = off[i]; mi < off[i + 1]; mi++) {
                    if (nbr[mi] == kj) { sum = sum - icv[mi] * icv[mj]; break; }
                }
            }
            icv[l] = sum / icd[i];
            int mj = slot_of(off, nbr, j, i);
            if (mj >= 0) icv[mj] = icv[l];
        }
    }
}

/* A*x in the reference's row order and slot order (functions.cu:516-527) */
void mo_spmv(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
             const double* val, const double* xin, double* s)
{
    for (int i = 0; i < n; i++) {
        if (bcon[i] != 0) { s[i] = 0.0; continue; }
        double acc = diag[i] * xin[i];
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (bcon[j] == -1) continue;
            acc = acc + val[l] * xin[j];
        }
        s[i] = acc;
    }
}

static void ic_solve(int n, const int* off, const int* nbr, const int* bcon, const double* icd,
                     const double* icv, const double* rin, double* q, double* aux)
{
    /* forward substitution (functions.cu:533-546) */
    memcpy(aux, rin, sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) {
        if (bcon[i] != 0) continue;
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (j > i) continue;
            if (bcon[j] != 0) continue;
            aux[i] = aux[i] - icv[l] * q[j];
        }
        q[i] = aux[i] / icd[i];
    }
    /* backward substitution (functions.cu:548-563) */
    memcpy(aux, q, sizeof(double) * (size_t)n);
    for (int i = n - 1; i >= 0; i--) {
        if (bcon[i] != 0) continue;
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (j < i) continue;
            if (bcon[j] != 0) continue;
            aux[i] = aux[i] - icv[l] * q[j];
        }
        q[i] = aux[i] / icd[i];
    }
}

/* ICCG with the reference's stop rule, functions.cu:506-716 */
int mo_cgm_ref(const mo_params* P, int n, const int* off, const int* nbr, const int* bcon,
               const double* diag, const double* val, const double* icd, const double* icv,
               const double* b, double* x)
{
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* r = (double*)calloc(1, sz);
    double* p = (double*)calloc(1, sz);
    double* q = (double*)calloc(1, sz);
    double* s = (double*)calloc(1, sz);
    double* aux = (double*)calloc(1, sz);
    double dt = P->dt;
    int iters = 0;
    mo_spmv(n, off, nbr, bcon, diag, val, x, s);
    for (int i = 0; i < n; i++) r[i] = b[i] - s[i];
    ic_solve(n, off, nbr, bcon, icd, icv, r, q, aux);
    memcpy(p, q, sz);
    double rqo = 0.0;
    for (int i = 0; i < n; i++) if (bcon[i] == 0) rqo += r[i] * q[i];
    for (int k = 0; k < P->imax; k++) {
        mo_spmv(n, off, nbr, bcon, diag, val, p, s);
        double ps = 0.0;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) ps += p[i] * s[i];
        double aa = rqo / ps;
        for (int i = 0; i < n; i++) x[i] = x[i] + aa * p[i];
        for (int i = 0; i < n; i++) r[i] = r[i] - aa * s[i];
        ic_solve(n, off, nbr, bcon, icd, icv, r, q, aux);
        double rqn = 0.0;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) rqn += r[i] * q[i];
        double bb = rqn / rqo;
        rqo = rqn;
        for (int i = 0; i < n; i++) p[i] = q[i] + bb * p[i];
        int j = 0;
        for (int i = 0; i < n; i++) {
            if (bcon[i] != 0) continue;
            double err1 = (r[i] > 0) ? r[i] * dt * dt : -r[i] * dt * dt;
            if (err1 > P->eps) j++;
        }
        iters = k + 1;
        if (j == 0 && k >= P->imin) break;
    }
    free(r); free(p); free(q); free(s); free(aux);
    return iters;
}

/* The reference's ICCG iteration (functions.cu:506-716: IC(0) factor from
   INCDECOM, forward and backward substitution as preconditioner) stopped on
   the relative residual ||b-Ax||/||b|| <= tol like mo_cg, so that its
   iteration count compares with the Jacobi-PCG of the CUDA path at the same
   tolerance.  Rows with bcon != 0 are held at 0. */
int mo_iccg(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
            const double* val, const double* icd, const double* icv, const double* b, double* x,
            double tol, int maxit, double* relres_out)
{
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* r = (double*)calloc(1, sz);
    double* p = (double*)calloc(1, sz);
    double* q = (double*)calloc(1, sz);
    double* s = (double*)calloc(1, sz);
    double* aux = (double*)calloc(1, sz);
    for (int i = 0; i < n; i++) if (bcon[i] != 0) x[i] = 0.0;
    mo_spmv(n, off, nbr, bcon, diag, val, x, s);
    double bb = 0.0, rr = 0.0;
    for (int i = 0; i < n; i++) {
        if (bcon[i] != 0) continue;
        r[i] = b[i] - s[i];
        bb += b[i] * b[i];
        rr += r[i] * r[i];
    }
    ic_solve(n, off, nbr, bcon, icd, icv, r, q, aux);
    for (int i = 0; i < n; i++) p[i] = bcon[i] == 0 ? q[i] : 0.0;
    double rq = 0.0;
    for (int i = 0; i < n; i++) if (bcon[i] == 0) rq += r[i] * q[i];
    int it = 0;
    const double thr = tol * tol * bb;
    while (rr > thr && it < maxit) {
        mo_spmv(n, off, nbr, bcon, diag, val, p, s);
        double ps = 0.0;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) ps += p[i] * s[i];
        double a = rq / ps;
        rr = 0.0;
        for (int i = 0; i < n; i++) {
            if (bcon[i] != 0) continue;
            x[i] += a * p[i];
            r[i] -= a * s[i];
            rr += r[i] * r[i];
        }
        ic_solve(n, off, nbr, bcon, icd, icv, r, q, aux);
        double rqn = 0.0;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) rqn += r[i] * q[i];
        double beta = rqn / rq;
        rq = rqn;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) p[i] = q[i] + beta * p[i];
        it++;
    }
    if (relres_out) *relres_out = mo_relres(n, off, nbr, bcon, diag, val, b, x);
    free(r); free(p); free(q); free(s); free(aux);
    return it;
}

double mo_relres(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
                 const double* val, const double* b, const double* x)
{
    double* s = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    mo_spmv(n, off, nbr, bcon, diag, val, x, s);
    double rr = 0.0, bb = 0.0;
    for (int i = 0; i < n; i++) {
        if (bcon[i] != 0) continue;
        double r = b[i] - s[i];
        rr += r * r;
        bb += b[i] * b[i];
    }
    free(s);
    if (bb == 0.0) return rr == 0.0 ? 0.0 : INFINITY;
    return sqrt(rr / bb);
}

/* Plain (precond=0) or Jacobi-preconditioned (precond=1) CG in FP64, stopped on
   the relative residual ||b-Ax||/||b|| <= tol.  This is the solver that the
   GPU path runs; rows with bcon != 0 are held at 0 (Dirichlet / excluded). */
int mo_cg(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
          const double* val, const double* b, double* x, double tol, int maxit, int precond,
          double* relres_out)
{
    size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
    double* r = (double*)calloc(1, sz);
    double* p = (double*)calloc(1, sz);
    double* z = (double*)calloc(1, sz);
    double* s = (double*)calloc(1, sz);
    for (int i = 0; i < n; i++) if (bcon[i] != 0) x[i] = 0.0;
    mo_spmv(n, off, nbr, bcon, diag, val, x, s);
    double bb = 0.0, rz = 0.0, rr = 0.0;
    for (int i = 0; i < n; i++) {
        if (bcon[i] != 0) continue;
        r[i] = b[i] - s[i];
        z[i] = precond ? r[i] / diag[i] : r[i];
        p[i] = z[i];
        bb += b[i] * b[i];
        rz += r[i] * z[i];
        rr += r[i] * r[i];
    }
    int it = 0;
    double thr = tol * tol * bb;
    while (rr > thr && it < maxit) {
        mo_spmv(n, off, nbr, bcon, diag, val, p, s);
        double ps = 0.0;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) ps += p[i] * s[i];
        double a = rz / ps;
        double rzn = 0.0;
        rr = 0.0;
        for (int i = 0; i < n; i++) {
            if (bcon[i] != 0) continue;
            x[i] += a * p[i];
            r[i] -= a * s[i];
            z[i] = precond ? r[i] / diag[i] : r[i];
            rzn += r[i] * z[i];
            rr += r[i] * r[i];
        }
        double beta = rzn / rz;
        rz = rzn;
        for (int i = 0; i < n; i++) if (bcon[i] == 0) p[i] = z[i] + beta * p[i];
        it++;
    }
    if (relres_out) *relres_out = mo_relres(n, off, nbr, bcon, diag, val, b, x);
    free(r); free(p); free(z); free(s);
    return it;
}

/* WC equation of state, functions.cu:2467-2500 */
void mo_pressure_wc(const mo_params* P, double n0, int n, const int* ptype, const double* C,
                    const double* nstar, double* pnew)
{
    for (int I = 0; I < n; I++) {
        if (ptype[I] < 0) continue; /* I = GP+1..TP */
        double c0 = (ptype[I] == 2) ? P->c02 : P->c01;
        double Rho = P->rho2 * C[I] + P->rho1 * (1 - C[I]);
        if (nstar[I] < P->beta_fs * n0) pnew[I] = 0.0;
        else pnew[I] = (c0 * c0 * Rho / 7.0) * (pow(nstar[I] / n0, 7.0) - 1);
        if (pnew[I] < P->pmin) pnew[I] = P->pmin;
        if (pnew[I] > P->pmax) pnew[I] = P->pmax;
    }
}

/* PHATCALC, functions.cu:207-224 */
void mo_phat(int n, const int* off, const int* nbr, const double* pnew, double* phat)
{
    for (int I = 0; I < n; I++) {
        double mn = 999999999999999;
        for (int l = off[I]; l < off[I + 1]; l++) {
            int J = nbr[l];
            if (pnew[J] < mn) mn = pnew[J];
        }
        phat[I] = mn;
    }
}

/* PRESSGRAD, functions.cu:245-355 (CPU semantics: KH uses p^_i + p^_j) */
void mo_pressgrad(const mo_params* P, double re, double n0, int n, const int* off,
                  const int* nbr, const int* ptype, const double* pnew, const double* phat,
                  const double* xs, const double* ys, const double* zs, const double* rho,
                  const double* us, const double* vs, const double* ws, double* un, double* vn,
                  double* wn)
{
    int dim = P->dim;
    double DT = P->dt, VMAX = P->vmax;
    for (int I = 0; I < n; I++) {
        if (ptype[I] <= 0) continue; /* I = GP+WP+1..TP */
        double sum1 = 0, sum2 = 0, sum3 = 0;
        if (P->kh == 1) {
            for (int l = off[I]; l < off[I + 1]; l++) {
                int J = nbr[l];
                double D = dist(dim, I, J, xs, ys, zs);
                if (I != J) {
                    double w = mo_W(D, P->ktype, dim, re);
                    double pp = pnew[J] + pnew[I] - (phat[I] + phat[J]);
                    sum1 = sum1 + pp * (xs[J] - xs[I]) * w / D / D;
                    sum2 = sum2 + pp * (ys[J] - ys[I]) * w / D / D;
                    if (dim == 3) sum3 = sum3 + pp * (zs[J] - zs[I]) * w / D / D;
                }
            }
        } else {
            for (int l = off[I]; l < off[I + 1]; l++) {
                int J = nbr[l];
                double D = dist(dim, I, J, xs, ys, zs);
                if (I != J) {
                    double w = mo_W(D, P->ktype, dim, re);
                    sum1 = sum1 + (pnew[J] - phat[I]) * (xs[J] - xs[I]) * w / D / D;
                    sum2 = sum2 + (pnew[J] - phat[I]) * (ys[J] - ys[I]) * w / D / D;
                    if (dim == 3) sum3 = sum3 + (pnew[J] - phat[I]) * (zs[J] - zs[I]) * w / D / D;
                }
            }
        }
        double Rho = rho[I];
        un[I] = us[I] - P->relaxp * (2.0 * DT / n0 / Rho) * sum1;
        vn[I] = vs[I] - P->relaxp * (2.0 * DT / n0 / Rho) * sum2;
        if (dim == 3) wn[I] = ws[I] - P->relaxp * (2.0 * DT / n0 / Rho) * sum3;
        double coeff = 2.0; /* damper, functions.cu:345-351 */
        if (fabs(un[I]) > coeff * VMAX) un[I] = VMAX;
        if (vn[I] > coeff * VMAX) vn[I] = coeff * VMAX;
        if (vn[I] < -coeff * VMAX) vn[I] = -coeff * VMAX;
        if (dim == 3)
            if (fabs(wn[I]) > coeff * VMAX) wn[I] = VMAX;
    }
}

/* PREDICTION, functions.cu:2283-2369.  The explicit pressure sums run over
   the PND list/radius, the viscous Laplacian over the Laplacian list/radius;
   with one list and one radius this is the reference loop exactly. */
void mo_prediction(const mo_params* P, double re_s, double n0_s, const int* off_s,
                   const int* nbr_s, double re_l, double n0_l, double lambda_l,
                   const int* off_l, const int* nbr_l, int n, const int* ptype,
                   const double* meu, const double* x, const double* y, const double* z,
                   const double* u, const double* v, const double* w, const double* pnew,
                   const double* phat, const double* neut, const double* t1, const double* t2,
                   const double* t3, const double* rho, double* xs, double* ys, double* zs,
                   double* us, double* vs, double* ws)
{
    int dim = P->dim, kt = P->ktype;
    double DT = P->dt;
    for (int I = 0; I < n; I++) {
        if (ptype[I] <= 0) {
            xs[I] = x[I]; ys[I] = y[I]; us[I] = u[I]; vs[I] = v[I];
            if (dim == 3) { zs[I] = z[I]; ws[I] = w[I]; }
            continue;
        }
        double sum1 = 0, sum2 = 0, sum3 = 0, sum4 = 0, sum5 = 0, sum6 = 0, sum7 = 0, sum8 = 0,
               sum9 = 0;
        for (int l = off_s[I]; l < off_s[I + 1]; l++) {
            int J = nbr_s[l];
            double D = dist(dim, I, J, x, y, z);
            if (I != J && D > 0) {
                double W = mo_W(D, kt, dim, re_s);
                sum1 = sum1 + (pnew[J] - phat[I]) * (x[J] - x[I]) * W / D / D;
                sum2 = sum2 + (pnew[J] - phat[I]) * (y[J] - y[I]) * W / D / D;
                if (dim == 3) sum3 = sum3 + (pnew[J] - phat[I]) * (z[J] - z[I]) * W / D / D;
            }
        }
        for (int l = off_l[I]; l < off_l[I + 1]; l++) {
            int J = nbr_l[l];
            double D = dist(dim, I, J, x, y, z);
            if (I != J && D > 0) {
                double NEU;
                if (ptype[I] == ptype[J]) {
                    if (ptype[I] == 1) NEU = meu[I] / P->rho1;
                    else NEU = meu[I] / P->rho2;
                } else {
                    if (ptype[I] == 1) NEU = 2 * meu[I] * meu[J] / (meu[I] + meu[J]) / P->rho1;
                    else NEU = 2 * meu[I] * meu[J] / (meu[I] + meu[J]) / P->rho2;
                }
                double W = mo_W(D, kt, dim, re_l);
                sum4 = sum4 + W * (u[J] - u[I]) * NEU;
                sum5 = sum5 + W * (v[J] - v[I]) * NEU;
                if (dim == 3) sum6 = sum6 + W * (w[J] - w[I]) * NEU;
                sum7 = sum7 + W * (u[J] - u[I]);
                sum8 = sum8 + W * (v[J] - v[I]);
                if (dim == 3) sum9 = sum9 + W * (w[J] - w[I]);
            }
        }
        double rp = 1 - P->relaxp;
        us[I] = u[I] + P->gx * DT + 4 * DT * (sum4 + neut[I] * sum7) / (lambda_l * n0_l) +
                DT * t1[I] - rp * (2.0 * DT / n0_s / rho[I]) * sum1;
        vs[I] = v[I] + P->gy * DT + 4 * DT * (sum5 + neut[I] * sum8) / (lambda_l * n0_l) +
                DT * t2[I] - rp * (2.0 * DT / n0_s / rho[I]) * sum2;
        if (dim == 3)
            ws[I] = w[I] + P->gz * DT + 4 * DT * (sum6 + neut[I] * sum9) / (lambda_l * n0_l) +
                    DT * t3[I] - rp * (2.0 * DT / n0_s / rho[I]) * sum3;
        xs[I] = x[I] + DT * us[I];
        ys[I] = y[I] + DT * vs[I];
        if (dim == 3) zs[I] = z[I] + DT * ws[I];
    }
}

/* velocity-gradient sums shared by VISCOSITY and SPS (functions.cu:2096-2117,
   1734-1756): out[0..8] = sum1..sum9 */
static void grad_sums(int dim, double re, int kt, int I, const int* off, const int* nbr,
                      const double* x, const double* y, const double* z, const double* un,
                      const double* vn, const double* wn, double mind, double* s)
{
    for (int k = 0; k < 9; k++) s[k] = 0;
    for (int l = off[I]; l < off[I + 1]; l++) {
        int j = nbr[l];
        double d = dist(dim, I, j, x, y, z);
        if (I != j && (mind < 0 || d > mind)) {
            double w = mo_W(d, kt, dim, re);
            s[0] = s[0] + (un[j] - un[I]) * (x[j] - x[I]) * w / d / d;
            s[1] = s[1] + (vn[j] - vn[I]) * (y[j] - y[I]) * w / d / d;
            s[2] = s[2] + (un[j] - un[I]) * (y[j] - y[I]) * w / d / d;
            s[3] = s[3] + (vn[j] - vn[I]) * (x[j] - x[I]) * w / d / d;
            if (dim == 3) {
                s[4] = s[4] + (wn[j] - wn[I]) * (z[j] - z[I]) * w / d / d;
                s[5] = s[5] + (un[j] - un[I]) * (z[j] - z[I]) * w / d / d;
                s[6] = s[6] + (vn[j] - vn[I]) * (z[j] - z[I]) * w / d / d;
                s[7] = s[7] + (wn[j] - wn[I]) * (x[j] - x[I]) * w / d / d;
                s[8] = s[8] + (wn[j] - wn[I]) * (y[j] - y[I]) * w / d / d;
            }
        }
    }
}

/* strain-rate tensor from the sums (functions.cu:2118-2146) */
static void strain(int dim, double n0, const double* s, double* S)
{
    double Uxx = (2.0 / n0) * s[0], Uyy = (2.0 / n0) * s[1];
    double Uxy = (2.0 / n0) * s[2], Uyx = (2.0 / n0) * s[3];
    S[1] = 0.5 * (Uxy + Uyx); /* S12 */
    S[0] = 0.5 * (Uxx + Uxx); /* S11 */
    S[2] = 0.5 * (Uyy + Uyy); /* S22 */
    S[3] = S[4] = S[5] = 0.0;
    if (dim == 3) {
        double Uzz = (2.0 / n0) * s[4], Uxz = (2.0 / n0) * s[5], Uyz = (2.0 / n0) * s[6];
        double Uzx = (2.0 / n0) * s[7], Uzy = (2.0 / n0) * s[8];
        S[5] = 0.5 * (Uzz + Uzz); /* S33 */
        S[3] = 0.5 * (Uxz + Uzx); /* S13 */
        S[4] = 0.5 * (Uyz + Uzy); /* S23 */
    }
}

/* VISCOSITY, functions.cu:2053-2184.  The reference reads C[I] with I the
   host-global 0 (functions.cu:2154); this restatement reads C[i].  The two
   agree whenever PHI == 0, which every shipped configuration uses. */
void mo_viscosity(const mo_params* P, double re, double n0, int n, const int* off,
                  const int* nbr, const int* ptype, const double* x, const double* y,
                  const double* z, const double* un, const double* vn, const double* wn,
                  const double* C, const double* phat, double* meu)
{
    int dim = P->dim;
    if (P->fluid2_type == 0) {
        for (int i = 0; i < n; i++) {
            if (ptype[i] <= 1) meu[i] = P->nu1 * P->rho1;
            if (ptype[i] == 2) meu[i] = P->nu2 * P->rho2;
        }
        return;
    }
    for (int i = 0; i < n; i++) {
        if (ptype[i] == 1) { meu[i] = P->nu1 * P->rho1; continue; }
        double s[9], S[6];
        grad_sums(dim, re, P->ktype, i, off, nbr, x, y, z, un, vn, wn, -1.0, s);
        strain(dim, n0, s, S);
        double phi = (C[i] - 0.25) * P->phi / (1 - 0.25);
        if (C[i] < 0.25) phi = 0;
        double yield_stress = P->cohes * cos(phi) + phat[i] * sin(phi);
        double II;
        double S11 = S[0], S12 = S[1], S22 = S[2], S13 = S[3], S23 = S[4], S33 = S[5];
        if (dim == 3)
            II = fabs((S11 * S22 * S33 + S12 * S23 * S13 + S13 * S12 * S23) -
                      (S13 * S22 * S13 + S11 * S23 * S23 + S12 * S12 * S33));
        else
            II = fabs(S11 * S22 - S12 * S12);
        meu[i] = yield_stress / 2 / sqrt(II) + P->meu0 * pow(4 * II, (P->n_pl - 1) / 2);
        if (II == 0 || meu[i] > 200) meu[i] = 200;
    }
}

/* SPS-LES, functions.cu:1719-1841 */
void mo_sps(const mo_params* P, double re, double n0, int n, const int* off, const int* nbr,
            const int* ptype, const double* x, const double* y, const double* z,
            const double* un, const double* vn, const double* wn, double* neut, double* t1,
            double* t2, double* t3)
{
    int dim = P->dim;
    double* S = (double*)calloc((size_t)(n > 0 ? n : 1) * 6, sizeof(double));
    double mind = P->coll / 10;
    for (int i = 0; i < n; i++) {
        if (ptype[i] < 0) continue; /* i = GP+1..TP */
        double s[9];
        grad_sums(dim, re, P->ktype, i, off, nbr, x, y, z, un, vn, wn, mind, s);
        double* Si = S + 6 * (size_t)i;
        strain(dim, n0, s, Si);
        double S11 = Si[0], S12 = Si[1], S22 = Si[2], S13 = Si[3], S23 = Si[4], S33 = Si[5];
        double Sm;
        if (dim == 3)
            Sm = pow(2 * S11 * S11, 0.5) + 2 * pow(2 * S12 * S12, 0.5) + pow(2 * S22 * S22, 0.5) +
                 pow(2 * S33 * S33, 0.5) + 2 * pow(2 * S13 * S13, 0.5) + 2 * pow(2 * S23 * S23, 0.5);
        else
            Sm = pow(2 * S11 * S11, 0.5) + 2 * pow(2 * S12 * S12, 0.5) + pow(2 * S22 * S22, 0.5);
        double cd = P->cs * P->l0;
        neut[i] = (cd * cd) * Sm;
    }
    for (int i = 0; i < n; i++) {
        if (ptype[i] < 0) continue;
        double sum1 = 0, sum2 = 0, sum3 = 0;
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            double d = dist(dim, i, j, x, y, z);
            if (i != j && d > mind) {
                double w = mo_W(d, P->ktype, dim, re);
                sum1 = sum1 + (neut[j] - neut[i]) * (x[j] - x[i]) * w / d / d;
                sum2 = sum2 + (neut[j] - neut[i]) * (y[j] - y[i]) * w / d / d;
                if (dim == 3) sum3 = sum3 + (neut[j] - neut[i]) * (z[j] - z[i]) * w / d / d;
            }
        }
        const double* Si = S + 6 * (size_t)i;
        double S11 = Si[0], S12 = Si[1], S22 = Si[2], S13 = Si[3], S23 = Si[4], S33 = Si[5];
        if (dim == 3) {
            t1[i] = (2.0 / n0) * (2 * S11 * sum1 + 2 * S12 * sum2 + 2 * S13 * sum3);
            t2[i] = (2.0 / n0) * (2 * S12 * sum1 + 2 * S22 * sum2 + 2 * S23 * sum3);
            t3[i] = (2.0 / n0) * (2 * S13 * sum1 + 2 * S23 * sum2 + 2 * S33 * sum3);
        } else {
            t1[i] = (2.0 / n0) * (2 * S11 * sum1 + 2 * S12 * sum2);
            t2[i] = (2.0 / n0) * (2 * S12 * sum1 + 2 * S22 * sum2);
        }
    }
    free(S);
}

/* V_FRACTION, functions.cu:2580-2638 */
void mo_vfraction(const mo_params* P, double re, int n, const int* off, const int* nbr,
                  const int* ptype, const double* x, const double* y, const double* z,
                  double* C)
{
    int dim = P->dim;
    for (int I = 0; I < n; I++) {
        double sum1 = 0, sum2 = 0;
        for (int l = off[I]; l < off[I + 1]; l++) {
            int J = nbr[l];
            if (P->fraction_method == 1) {
                if (I != J && ptype[J] > 0) {
                    sum1 = sum1 + 1;
                    if (ptype[J] == 2) sum2 = sum2 + 1;
                }
            } else {
                double d = dist(dim, I, J, x, y, z);
                if (I != J && ptype[J] > 0) {
                    sum1 = sum1 + mo_W(d, P->ktype, dim, re);
                    if (ptype[J] == 2) sum2 = sum2 + mo_W(d, P->ktype, dim, re);
                }
            }
        }
        C[I] = sum2 / sum1;
        if (sum1 == 0) C[I] = 0;
    }
}

/* COLLISION2, functions.cu:1523-1601: sequential, mutates i and j in place */
void mo_collision(const mo_params* P, int n, const int* off, const int* nbr, const int* ptype,
                  double* un, double* vn, double* wn, double* x, double* y, double* z)
{
    int dim = P->dim;
    double DT = P->dt, cc = P->cc;
    for (int i = 0; i < n; i++) {
        double m1 = (ptype[i] == 1) ? P->rho1 : P->rho2;
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            double m2 = (ptype[j] == 1) ? P->rho1 : P->rho2;
            double d = dist(dim, i, j, x, y, z);
            if (i != j && d < P->coll) {
                double ug = (m1 * un[i] + m2 * un[j]) / (m1 + m2);
                double vg = (m1 * vn[i] + m2 * vn[j]) / (m1 + m2);
                double wg = 0, wr = 0, wm = 0, vabs;
                if (dim == 3) wg = (m1 * wn[i] + m2 * wn[j]) / (m1 + m2);
                double ur = m1 * (un[i] - ug);
                double vr = m1 * (vn[i] - vg);
                if (dim == 3) wr = m1 * (wn[i] - wg);
                if (dim == 3)
                    vabs = (ur * (x[j] - x[i]) + vr * (y[j] - y[i]) + wr * (z[j] - z[i])) / d;
                else
                    vabs = (ur * (x[j] - x[i]) + vr * (y[j] - y[i])) / d;
                double um = (1.0 + cc) * vabs * (x[j] - x[i]) / d;
                double vm = (1.0 + cc) * vabs * (y[j] - y[i]) / d;
                if (dim == 3) wm = (1.0 + cc) * vabs * (z[j] - z[i]) / d;
                if (vabs > 0) {
                    if (ptype[i] > 0) {
                        un[i] = un[i] - um / m1;
                        vn[i] = vn[i] - vm / m1;
                        x[i] = x[i] - DT * um / m1;
                        y[i] = y[i] - DT * vm / m1;
                        if (dim == 3) { wn[i] = wn[i] - wm / m1; z[i] = z[i] - DT * wm / m1; }
                    }
                    if (ptype[j] > 0) {
                        un[j] = un[j] + um / m2;
                        vn[j] = vn[j] + vm / m2;
                        x[j] = x[j] + DT * um / m2;
                        y[j] = y[j] + DT * vm / m2;
                        if (dim == 3) { wn[j] = wn[j] + wm / m2; z[j] = z[j] + DT * wm / m2; }
                    }
                }
            }
        }
    }
}

/* One visit of COLLISION2's pair loop (functions.cu:1536-1599) from particle
   i's list to its neighbour j, on local copies of their states
   s = {u, v, w, x, y, z}: the same expressions, in the same order, as the
   reference's in-place update of unew/vnew/wnew and x/y/z. */
static void coll_visit(const mo_params* P, int dim, int pti, int ptj, double* si, double* sj)
{
    double m1 = (pti == 1) ? P->rho1 : P->rho2;
    double m2 = (ptj == 1) ? P->rho1 : P->rho2;
    double DT = P->dt, cc = P->cc;
    double dx = sj[3] - si[3], dy = sj[4] - si[4], dz = 0, d;
    if (dim == 3) {
        dz = sj[5] - si[5];
        d = sqrt(dx * dx + dy * dy + dz * dz);
    } else {
        d = sqrt(dx * dx + dy * dy);
    }
    if (!(d < P->coll)) return;
    double ug = (m1 * si[0] + m2 * sj[0]) / (m1 + m2);
    double vg = (m1 * si[1] + m2 * sj[1]) / (m1 + m2);
    double wg = 0, wr = 0, wm = 0, vabs;
    if (dim == 3) wg = (m1 * si[2] + m2 * sj[2]) / (m1 + m2);
    double ur = m1 * (si[0] - ug);
    double vr = m1 * (si[1] - vg);
    if (dim == 3) wr = m1 * (si[2] - wg);
    if (dim == 3)
        vabs = (ur * dx + vr * dy + wr * dz) / d;
    else
        vabs = (ur * dx + vr * dy) / d;
    double um = (1.0 + cc) * vabs * dx / d;
    double vm = (1.0 + cc) * vabs * dy / d;
    if (dim == 3) wm = (1.0 + cc) * vabs * dz / d;
    if (!(vabs > 0)) return;
    if (pti > 0) {
        si[0] = si[0] - um / m1; si[1] = si[1] - vm / m1;
        si[3] = si[3] - DT * um / m1; si[4] = si[4] - DT * vm / m1;
        if (dim == 3) { si[2] = si[2] - wm / m1; si[5] = si[5] - DT * wm / m1; }
    }
    if (ptj > 0) {
        sj[0] = sj[0] + um / m2; sj[1] = sj[1] + vm / m2;
        sj[3] = sj[3] + DT * um / m2; sj[4] = sj[4] + DT * vm / m2;
        if (dim == 3) { sj[2] = sj[2] + wm / m2; sj[5] = sj[5] + DT * wm / m2; }
    }
}

/* Order-independent collision.  COLLISION2 walks every particle (walls and
   dummies included) in id order and updates pairs in place, so a pair
   (a, b), a < b, is visited twice: from a's list, then from b's list with
   the state the first visit left.  A fluid-fluid pair's second visit finds
   the pair separating and does nothing; a fluid-wall pair can be pushed
   again, because the wall keeps its velocity.  Here every fluid particle
   replays, for each neighbour closer than coll in the pre-collision state,
   that pair's two visits on private copies.  With one such neighbour the
   particle takes the replayed state itself -- bit for bit COLLISION2's,
   since nothing else touches the pair in between; with several it takes
   the pre-collision state plus the sum of the pairs' changes, in list
   order, where the sequential result would depend on the visiting order. */
void mo_collision_gather(const mo_params* P, int n, const int* off, const int* nbr,
                         const int* ptype, double* un, double* vn, double* wn, double* x,
                         double* y, double* z)
{
    int dim = P->dim;
    size_t sz = sizeof(double) * 6 * (size_t)(n > 0 ? n : 1);
    double* out = (double*)malloc(sz);
    for (int i = 0; i < n; i++) {
        double s0[6] = {un[i], vn[i], dim == 3 ? wn[i] : 0.0, x[i], y[i], dim == 3 ? z[i] : 0.0};
        double acc[6] = {0, 0, 0, 0, 0, 0}, last[6];
        int hits = 0;
        for (int k = 0; k < 6; k++) { out[6 * (size_t)i + k] = s0[k]; last[k] = s0[k]; }
        if (ptype[i] <= 0) continue;
        for (int l = off[i]; l < off[i + 1]; l++) {
            int j = nbr[l];
            if (j == i || !(dist(dim, i, j, x, y, z) < P->coll)) continue;
            double si[6] = {s0[0], s0[1], s0[2], s0[3], s0[4], s0[5]};
            double sj[6] = {un[j], vn[j], dim == 3 ? wn[j] : 0.0, x[j], y[j],
                            dim == 3 ? z[j] : 0.0};
            if (j < i) {
                coll_visit(P, dim, ptype[j], ptype[i], sj, si);
                coll_visit(P, dim, ptype[i], ptype[j], si, sj);
            } else {
                coll_visit(P, dim, ptype[i], ptype[j], si, sj);
                coll_visit(P, dim, ptype[j], ptype[i], sj, si);
            }
            for (int k = 0; k < 6; k++) { acc[k] += si[k] - s0[k]; last[k] = si[k]; }
            hits++;
        }
        for (int k = 0; k < 6; k++)
            out[6 * (size_t)i + k] = hits == 1 ? last[k] : (hits > 1 ? s0[k] + acc[k] : s0[k]);
    }
    for (int i = 0; i < n; i++) {
        const double* o = out + 6 * (size_t)i;
        un[i] = o[0]; vn[i] = o[1]; x[i] = o[3]; y[i] = o[4];
        if (dim == 3) { wn[i] = o[2]; z[i] = o[5]; }
    }
    free(out);
}

/* EULERINTEGRATION + BOUNDARIE (dam test), functions.cu:1963-2021 */
void mo_euler(const mo_params* P, int n, const int* ptype, double* x, double* y, double* z,
              double* un, double* vn, double* wn)
{
    double DT = P->dt, DL = P->l0, CC = P->velcor;
    for (int I = 0; I < n; I++) {
        if (ptype[I] <= 0) continue;
        x[I] = x[I] + un[I] * DT;
        y[I] = y[I] + vn[I] * DT;
        if (P->dim == 3) z[I] = z[I] + wn[I] * DT;
        if (y[I] < P->ymin + DL * 3.0) { vn[I] = fabs(vn[I]) * CC; y[I] = P->ymin + DL * 3.0; }
        if (y[I] > P->ymax - DL * 3.0) { vn[I] = -fabs(vn[I]) * CC; y[I] = P->ymax - DL * 3.0; }
        if (x[I] < P->xmin + DL * 3.0) { un[I] = fabs(un[I]) * CC; x[I] = P->xmin + DL * 3.0; }
        if (x[I] > P->xmax - DL * 3.0) { un[I] = -fabs(un[I]) * CC; x[I] = P->xmax - DL * 3.0; }
        if (P->dim == 3) {
            if (z[I] < P->zmin + DL * 3.0) { wn[I] = fabs(wn[I]) * CC; z[I] = P->zmin + DL * 3.0; }
            if (z[I] > P->zmax - DL * 3.0) { wn[I] = -fabs(wn[I]) * CC; z[I] = P->zmax - DL * 3.0; }
        }
    }
}

/* PREPDATA, functions.cu:2688-2746.  Returns error bits: 1 = non-finite
   state (ERROR#1), 2 = particle outside the box (ERROR#2). */
int mo_prepdata(const mo_params* P, int n, const int* ptype, const double* x, const double* y,
                const double* z, double* u, double* v, double* w, double* p, const double* un,
                const double* vn, const double* wn, const double* pnew)
{
    int err = 0;
    for (int I = 0; I < n; I++) {
        p[I] = pnew[I];
        if (ptype[I] > 0) {
            u[I] = un[I]; v[I] = vn[I];
            if (P->dim == 3) w[I] = wn[I];
        }
        if (P->dim == 3) {
            if (p[I] * 0 != 0 || u[I] * 0 != 0 || v[I] * 0 != 0 || w[I] * 0 != 0) err |= 1;
            if (x[I] >= P->xmax || y[I] >= P->ymax || z[I] >= P->zmax || x[I] <= P->xmin ||
                y[I] <= P->ymin || z[I] <= P->zmin)
                err |= 2;
        } else {
            if (p[I] * 0 != 0 || u[I] * 0 != 0 || v[I] * 0 != 0) err |= 1;
            if (x[I] >= P->xmax || y[I] >= P->ymax || x[I] <= P->xmin || y[I] <= P->ymin) err |= 2;
        }
    }
    return err;
}

/* ------------------------------------------------------------------ */
/* whole pipeline                                                      */
/* ------------------------------------------------------------------ */
struct mo_state {
    mo_params P;
    int n;
    double *x, *y, *z, *u, *v, *w, *p, *pnew, *phat, *un, *vn, *wn, *xs, *ys, *zs, *us, *vs,
        *ws, *nd, *nds, *C, *meu, *neut, *t1, *t2, *t3, *rho, *source, *diag, *val, *pold;
    int *ptype, *bcon;
    int *cell_s, *perm_s, *off_s, *nbr_s, cap_s;
    int *cell_l, *perm_l, *off_l, *nbr_l, cap_l;
    double n0_s, n0_l, lambda_l, relres;
    int cg_iters, have_lists, last_err;
};

static int build_list(mo_state* S, double re, int** cell, int** perm, int** off, int** nbr,
                      int* cap)
{
    for (;;) {
        int r = mo_neighbor(&S->P, re, S->n, S->x, S->y, S->z, *cell, *perm, *off, *nbr, *cap);
        if (r == MO_ERR_CELL) return 4;
        if (r >= 0) return 0;
        *cap = -r + 16;
        free(*nbr);
        *nbr = (int*)malloc(sizeof(int) * (size_t)(*cap));
    }
}

static int single_radius(const mo_state* S) { return S->P.re_s == S->P.re_l; }

static int rebuild_lists(mo_state* S)
{
    int e = build_list(S, S->P.re_s, &S->cell_s, &S->perm_s, &S->off_s, &S->nbr_s, &S->cap_s);
    if (e) return e;
    if (single_radius(S)) {
        if (S->cap_l < S->off_s[S->n]) {
            free(S->nbr_l);
            S->cap_l = S->off_s[S->n] + 16;
            S->nbr_l = (int*)malloc(sizeof(int) * (size_t)S->cap_l);
        }
        memcpy(S->cell_l, S->cell_s, sizeof(int) * (size_t)S->n);
        memcpy(S->perm_l, S->perm_s, sizeof(int) * (size_t)S->n);
        memcpy(S->off_l, S->off_s, sizeof(int) * (size_t)(S->n + 1));
        memcpy(S->nbr_l, S->nbr_s, sizeof(int) * (size_t)S->off_s[S->n]);
        return 0;
    }
    return build_list(S, S->P.re_l, &S->cell_l, &S->perm_l, &S->off_l, &S->nbr_l, &S->cap_l);
}

mo_state* mo_create(const mo_params* P, int n, const double* x, const double* y,
                    const double* z, const int* ptype, const double* u, const double* v,
                    const double* w, const double* p)
{
    mo_state* S = (mo_state*)calloc(1, sizeof(mo_state));
    S->P = *P;
    S->n = n;
    size_t nd = (size_t)(n > 0 ? n : 1);
    double** dbl[] = {&S->x,  &S->y,  &S->z,  &S->u,    &S->v,    &S->w,    &S->p,     &S->pnew,
                      &S->phat, &S->un, &S->vn, &S->wn, &S->xs,   &S->ys,   &S->zs,    &S->us,
                      &S->vs, &S->ws, &S->nd, &S->nds, &S->C,   &S->meu,  &S->neut,  &S->t1,
                      &S->t2, &S->t3, &S->rho, &S->source, &S->diag, &S->pold};
    for (size_t k = 0; k < sizeof(dbl) / sizeof(dbl[0]); k++)
        *dbl[k] = (double*)calloc(nd, sizeof(double));
    S->ptype = (int*)calloc(nd, sizeof(int));
    S->bcon = (int*)calloc(nd, sizeof(int));
    S->cell_s = (int*)calloc(nd, sizeof(int));
    S->perm_s = (int*)calloc(nd, sizeof(int));
    S->off_s = (int*)calloc(nd + 1, sizeof(int));
    S->cell_l = (int*)calloc(nd, sizeof(int));
    S->perm_l = (int*)calloc(nd, sizeof(int));
    S->off_l = (int*)calloc(nd + 1, sizeof(int));
    S->cap_s = 64 * (int)nd;
    S->nbr_s = (int*)malloc(sizeof(int) * (size_t)S->cap_s);
    S->cap_l = 64 * (int)nd;
    S->nbr_l = (int*)malloc(sizeof(int) * (size_t)S->cap_l);
    S->val = NULL;
    memcpy(S->x, x, sizeof(double) * (size_t)n);
    memcpy(S->y, y, sizeof(double) * (size_t)n);
    if (z) memcpy(S->z, z, sizeof(double) * (size_t)n);
    memcpy(S->ptype, ptype, sizeof(int) * (size_t)n);
    if (u) memcpy(S->u, u, sizeof(double) * (size_t)n);
    if (v) memcpy(S->v, v, sizeof(double) * (size_t)n);
    if (w) memcpy(S->w, w, sizeof(double) * (size_t)n);
    if (p) memcpy(S->p, p, sizeof(double) * (size_t)n);
    /* density assignment, main.cu:972-977 */
    for (int i = 0; i < n; i++) S->rho[i] = (S->ptype[i] == 2) ? P->rho2 : P->rho1;
    S->lambda_l = mo_lambda(P->ktype, P->re_l);
    return S;
}

void mo_destroy(mo_state* S)
{
    if (!S) return;
    double* dbl[] = {S->x,  S->y,  S->z,  S->u,  S->v,   S->w,  S->p,   S->pnew, S->phat, S->un,
                     S->vn, S->wn, S->xs, S->ys, S->zs,  S->us, S->vs,  S->ws,   S->nd,   S->nds,
                     S->C,  S->meu, S->neut, S->t1, S->t2, S->t3, S->rho, S->source, S->diag,
                     S->val, S->pold};
    for (size_t k = 0; k < sizeof(dbl) / sizeof(dbl[0]); k++) free(dbl[k]);
    free(S->ptype); free(S->bcon);
    free(S->cell_s); free(S->perm_s); free(S->off_s); free(S->nbr_s);
    free(S->cell_l); free(S->perm_l); free(S->off_l); free(S->nbr_l);
    free(S);
}

/* pre-iteration work, main.cu:980-1012: lists, n (with pnew = p), n0 */
int mo_init(mo_state* S)
{
    int e = rebuild_lists(S);
    if (e) return e;
    S->have_lists = 1;
    mo_pnd(&S->P, S->P.re_s, S->n, S->off_s, S->nbr_s, S->x, S->y, S->z, 1, S->nd);
    for (int i = 0; i < S->n; i++) S->pnew[i] = S->p[i];
    for (int i = 0; i < S->n; i++) S->pold[i] = S->p[i];
    S->n0_s = mo_max(S->n, S->nd);
    if (single_radius(S)) {
        S->n0_l = S->n0_s;
    } else {
        double* tmp = (double*)malloc(sizeof(double) * (size_t)(S->n > 0 ? S->n : 1));
        mo_pnd(&S->P, S->P.re_l, S->n, S->off_l, S->nbr_l, S->x, S->y, S->z, 1, tmp);
        S->n0_l = mo_max(S->n, tmp);
        free(tmp);
    }
    return 0;
}

/* One time step in main.cu's order (main.cu:1027-1349).
 *   ppe_at_predicted = 0: reference CPU semantics -- A at x, b from the PND n
 *     computed at step start with the previous step's list (main.cu:1036-1047,
 *     1149-1150; functions.cu:997).
 *   ppe_at_predicted = 1: A at x*, b from n* (the reference GPU path,
 *     main.cu:1165, functions.cu:1126), the semantics the CUDA path uses. */
int mo_step(mo_state* S)
{
    mo_params* P = &S->P;
    int n = S->n, err = 0;
    if (P->method != 3 && !P->ppe_at_predicted)
        mo_pnd(P, P->re_s, n, S->off_s, S->nbr_s, S->x, S->y, S->z, 1, S->nd);
    err |= rebuild_lists(S);
    if (err) return err;
    if (P->turb)
        mo_sps(P, P->re_s, S->n0_s, n, S->off_s, S->nbr_s, S->ptype, S->x, S->y, S->z, S->un,
               S->vn, S->wn, S->neut, S->t1, S->t2, S->t3);
    mo_vfraction(P, P->re_s, n, S->off_s, S->nbr_s, S->ptype, S->x, S->y, S->z, S->C);
    mo_viscosity(P, P->re_s, S->n0_s, n, S->off_s, S->nbr_s, S->ptype, S->x, S->y, S->z, S->un,
                 S->vn, S->wn, S->C, S->phat, S->meu);
    mo_prediction(P, P->re_s, S->n0_s, S->off_s, S->nbr_s, P->re_l, S->n0_l, S->lambda_l,
                  S->off_l, S->nbr_l, n, S->ptype, S->meu, S->x, S->y, S->z, S->u, S->v, S->w,
                  S->pnew, S->phat, S->neut, S->t1, S->t2, S->t3, S->rho, S->xs, S->ys, S->zs,
                  S->us, S->vs, S->ws);
    mo_pnd(P, P->re_s, n, S->off_s, S->nbr_s, S->xs, S->ys, S->zs, 0, S->nds);
    if (P->method == 3) {
        mo_pressure_wc(P, S->n0_s, n, S->ptype, S->C, S->nds, S->pnew);
    } else {
        mo_bcon(n, S->ptype, S->nds, S->n0_s, P->dirichlet, S->bcon);
        int nnz = S->off_l[n];
        free(S->val);
        S->val = (double*)calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
        const double *ax = S->x, *ay = S->y, *az = S->z, *nsrc = S->nd;
        if (P->ppe_at_predicted) { ax = S->xs; ay = S->ys; az = S->zs; nsrc = S->nds; }
        mo_matrix(P, P->re_l, S->lambda_l, S->n0_l, n, S->off_l, S->nbr_l, ax, ay, az, S->bcon,
                  S->diag, S->val);
        memset(S->source, 0, sizeof(double) * (size_t)n);
        if (P->srcopt)
            mo_source_hs(P, P->re_s, S->n0_s, n, S->off_s, S->nbr_s, S->ptype, S->bcon, S->nds,
                         ax, ay, az, S->us, S->vs, S->ws, S->source);
        else
            mo_source(P, S->n0_s, n, S->ptype, S->bcon, nsrc, S->source);
        if (P->warm_start == 2) {
            /* linear extrapolation 2 p^n - p^(n-1) on unknown rows */
            for (int i = 0; i < n; i++) {
                double pn = S->pnew[i];
                S->pnew[i] = (S->bcon[i] != 0) ? 0.0 : 2.0 * pn - S->pold[i];
                S->pold[i] = pn;
            }
        } else if (P->warm_start) {
            for (int i = 0; i < n; i++) if (S->bcon[i] != 0) S->pnew[i] = 0.0;
        } else {
            memset(S->pnew, 0, sizeof(double) * (size_t)n);
        }
        if (P->solver == 0) {
            double* icd = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
            double* icv = (double*)calloc((size_t)(nnz > 0 ? nnz : 1), sizeof(double));
            mo_incdecom(n, S->off_l, S->nbr_l, S->bcon, S->diag, S->val, icd, icv);
            S->cg_iters = mo_cgm_ref(P, n, S->off_l, S->nbr_l, S->bcon, S->diag, S->val, icd,
                                     icv, S->source, S->pnew);
            free(icd); free(icv);
            S->relres = mo_relres(n, S->off_l, S->nbr_l, S->bcon, S->diag, S->val, S->source,
                                  S->pnew);
        } else {
            S->cg_iters = mo_cg(n, S->off_l, S->nbr_l, S->bcon, S->diag, S->val, S->source,
                                S->pnew, P->cg_tol, P->cg_max, P->solver == 1, &S->relres);
            if (!(S->relres <= P->cg_tol * 1.0001)) err |= 8;
        }
        /* clamp, functions.cu:2534-2547 */
        for (int I = 0; I < n; I++) {
            if (S->pnew[I] < P->pmin) S->pnew[I] = P->pmin;
            if (S->pnew[I] > P->pmax || S->pnew[I] * 0.0 != 0.0) S->pnew[I] = P->pmax;
        }
    }
    mo_phat(n, S->off_s, S->nbr_s, S->pnew, S->phat);
    mo_pressgrad(P, P->re_s, S->n0_s, n, S->off_s, S->nbr_s, S->ptype, S->pnew, S->phat, S->xs,
                 S->ys, S->zs, S->rho, S->us, S->vs, S->ws, S->un, S->vn, S->wn);
    mo_euler(P, n, S->ptype, S->x, S->y, S->z, S->un, S->vn, S->wn);
    if (P->collision_gather)
        mo_collision_gather(P, n, S->off_s, S->nbr_s, S->ptype, S->un, S->vn, S->wn, S->x, S->y,
                            S->z);
    else
        mo_collision(P, n, S->off_s, S->nbr_s, S->ptype, S->un, S->vn, S->wn, S->x, S->y, S->z);
    err |= mo_prepdata(P, n, S->ptype, S->x, S->y, S->z, S->u, S->v, S->w, S->p, S->un, S->vn,
                       S->wn, S->pnew);
    S->last_err = err;
    return err;
}

static void* field(mo_state* S, const char* name, int* is_int, long* count)
{
    long n = S->n;
    *is_int = 0;
    *count = n;
#define F(nm, ptr) if (!strcmp(name, nm)) return (void*)(ptr)
    F("x", S->x); F("y", S->y); F("z", S->z); F("u", S->u); F("v", S->v); F("w", S->w);
    F("p", S->p); F("pnew", S->pnew); F("phat", S->phat); F("un", S->un); F("vn", S->vn);
    F("wn", S->wn); F("xs", S->xs); F("ys", S->ys); F("zs", S->zs); F("us", S->us);
    F("vs", S->vs); F("ws", S->ws); F("n", S->nd); F("nstar", S->nds); F("C", S->C);
    F("meu", S->meu); F("neut", S->neut); F("t1", S->t1); F("t2", S->t2); F("t3", S->t3);
    F("rho", S->rho); F("source", S->source); F("diag", S->diag);
    if (!strcmp(name, "val")) { *count = S->off_l[n]; return S->val; }
    *is_int = 1;
    F("ptype", S->ptype); F("bcon", S->bcon); F("cell_s", S->cell_s); F("perm_s", S->perm_s);
    F("cell_l", S->cell_l); F("perm_l", S->perm_l);
    if (!strcmp(name, "off_s")) { *count = n + 1; return S->off_s; }
    if (!strcmp(name, "off_l")) { *count = n + 1; return S->off_l; }
    if (!strcmp(name, "nbr_s")) { *count = S->off_s[n]; return S->nbr_s; }
    if (!strcmp(name, "nbr_l")) { *count = S->off_l[n]; return S->nbr_l; }
#undef F
    return NULL;
}

long mo_get(mo_state* S, const char* name, void* out)
{
    int is_int;
    long count;
    void* src = field(S, name, &is_int, &count);
    if (!src) return -1;
    if (out) memcpy(out, src, (size_t)count * (is_int ? sizeof(int) : sizeof(double)));
    return count;
}

long mo_set(mo_state* S, const char* name, const void* in)
{
    int is_int;
    long count;
    void* dst = field(S, name, &is_int, &count);
    if (!dst || !strncmp(name, "nbr", 3) || !strncmp(name, "off", 3) || !strcmp(name, "val"))
        return -1;
    memcpy(dst, in, (size_t)count * (is_int ? sizeof(int) : sizeof(double)));
    return count;
}

double mo_scalar(mo_state* S, const char* name)
{
    if (!strcmp(name, "n0_s")) return S->n0_s;
    if (!strcmp(name, "n0_l")) return S->n0_l;
    if (!strcmp(name, "lambda_l")) return S->lambda_l;
    if (!strcmp(name, "cg_iters")) return (double)S->cg_iters;
    if (!strcmp(name, "cg_relres")) return S->relres;
    if (!strcmp(name, "nnz_s")) return (double)S->off_s[S->n];
    if (!strcmp(name, "nnz_l")) return (double)S->off_l[S->n];
    if (!strcmp(name, "err")) return (double)S->last_err;
    return NAN;
}
