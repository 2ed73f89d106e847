/*
 * ref_harness.cpp -- drives the reference's OWN CPU stage functions
 * (VoxarMPS/VoxarMPS/functions.cu, compiled unmodified except for the two
 * build patches listed in oracle/Makefile) in the order of main.cu's time
 * loop, with the physical parameters passed in instead of main()'s
 * hard-coded constants.
 *
 * TEST INFRASTRUCTURE ONLY: it pins the C restatement (mps_oracle.c)
 * against the reference and times the reference's CPU path for bench.py's
 * reference arm.  It is built into oracle/_ref/, which stays out of git.
 *
 * Departures from main(), each a parameter the reference hard-codes:
 *   - dt is taken from the parameters; DTcalculation (functions.cu:1684) is
 *     not called (it would force COURANT*DL/c0);
 *   - DL, re, g, Cs, PMAX and the CGM bounds come from the parameters;
 *   - inputs arrive as arrays instead of a .grd path.
 * The reference has a single support radius: this harness uses re_s.
 */
#include "functions.cuh"

#include <omp.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../mps_oracle.h"

namespace {

struct RefState {
    mo_params P;
    int TP, GP, WP, FP;
    double *x, *y, *z, *u, *v, *w, *p;
    int* PTYPE;
    double *xstar, *ystar, *zstar, *ustar, *vstar, *wstar, *pnew, *phat, *unew, *vnew, *wnew;
    double *NEUt, *TURB1, *TURB2, *TURB3, *n, *nstar, *MEU, *C, *RHO, *SFX, *SFY;
    int** neighb;
    int* bcon;
    double *source, **poiss, **ic;
    double* MAX;
    double n0, lambda;
    int KTYPE, DIM;
    std::string codeOpt, test;
    int nthreads;
};

double* dnew(int TP) { return new double[TP + 1](); }

}  // namespace

extern "C" {

void* rh_create(const mo_params* P, int n, const double* x, const double* y, const double* z,
                const int* ptype, const double* u, const double* v, const double* w,
                const double* p, int nthreads)
{
    RefState* S = new RefState();
    S->P = *P;
    S->nthreads = nthreads > 0 ? nthreads : 1;
    S->codeOpt = (S->nthreads > 1) ? "openmp" : "sequential";
    S->test = "dam";
    int TP = n;
    S->TP = TP;
    S->x = dnew(TP); S->y = dnew(TP); S->z = dnew(TP);
    S->u = dnew(TP); S->v = dnew(TP); S->w = dnew(TP); S->p = dnew(TP);
    S->PTYPE = new int[TP + 1]();
    S->GP = S->WP = S->FP = 0;
    for (int I = 1; I <= TP; I++) {
        S->x[I] = x[I - 1]; S->y[I] = y[I - 1];
        if (z) S->z[I] = z[I - 1];
        S->PTYPE[I] = ptype[I - 1];
        if (u) S->u[I] = u[I - 1];
        if (v) S->v[I] = v[I - 1];
        if (w) S->w[I] = w[I - 1];
        if (p) S->p[I] = p[I - 1];
        if (S->PTYPE[I] < 0) S->GP++;
        if (S->PTYPE[I] == 0) S->WP++;
        if (S->PTYPE[I] > 0) S->FP++;
    }
    /* main.cu:726-770 */
    S->neighb = new int*[TP + 1]();
    for (int m = 0; m <= TP; m++) S->neighb[m] = new int[NEIGHBORS + 1]();
    S->pnew = dnew(TP);
    S->bcon = new int[TP + 1]();
    S->source = dnew(TP);
    S->poiss = new double*[TP + 1]();
    S->ic = new double*[TP + 1]();
    if (P->method != 3) {
        for (int m = 1; m <= TP; m++) S->poiss[m] = new double[NEIGHBORS + 1]();
        for (int m = 1; m <= TP; m++) S->ic[m] = new double[NEIGHBORS + 1]();
    }
    S->xstar = dnew(TP); S->ystar = dnew(TP); S->zstar = dnew(TP);
    S->ustar = dnew(TP); S->vstar = dnew(TP); S->wstar = dnew(TP);
    S->phat = dnew(TP); S->unew = dnew(TP); S->vnew = dnew(TP); S->wnew = dnew(TP);
    S->n = dnew(TP); S->nstar = dnew(TP); S->NEUt = dnew(TP);
    S->TURB1 = dnew(TP); S->TURB2 = dnew(TP); S->TURB3 = dnew(TP);
    S->C = dnew(TP); S->MEU = dnew(TP); S->RHO = dnew(TP); S->SFX = dnew(TP); S->SFY = dnew(TP);
    S->MAX = new double[1]();
    S->KTYPE = P->ktype;
    S->DIM = P->dim;
    /* main.cu:491-494 */
    double re = P->re_s;
    if (P->ktype == 1) S->lambda = 0.22143 * pow(re, 2);
    if (P->ktype == 2) S->lambda = 0.16832 * pow(re, 2);
    if (P->ktype == 5) S->lambda = 0.250 * pow(re, 2);
    if (P->ktype == 6) S->lambda = 0.14288 * pow(re, 2);
    for (int I = 1; I <= TP; I++) S->RHO[I] = (S->PTYPE[I] == 2) ? P->rho2 : P->rho1;
    return S;
}

int rh_init(void* h)
{
    RefState* S = (RefState*)h;
    const mo_params& P = S->P;
    omp_set_num_threads(S->nthreads);
    NEIGHBOR(P.xmax, P.xmin, P.ymax, P.ymin, P.zmax, P.zmin, P.re_s, P.delta, S->TP, S->x, S->y,
             S->z, S->neighb, S->DIM, S->codeOpt);
    S->MAX[0] = 0.0;
    PNUM(0, S->KTYPE, S->DIM, S->TP, P.re_s, S->neighb, S->x, S->y, S->z, P.ncorrection, S->n,
         S->MAX, S->pnew, S->p, false, S->codeOpt);
    S->n0 = S->MAX[0];
    return 0;
}

/* one pass of main.cu:1027-1349 (CPU branch of every stage) */
int rh_step(void* h)
{
    RefState* S = (RefState*)h;
    const mo_params& P = S->P;
    omp_set_num_threads(S->nthreads);
    int TP = S->TP, GP = S->GP, WP = S->WP, FP = S->FP, DIM = S->DIM, KTYPE = S->KTYPE;
    double re = P.re_s, DT = P.dt, n0 = S->n0;
    double c0 = 0.0, Rho = 0.0, II = 0, yield_stress = 0, correction = 0, MAXresi = 0.001;
    int IterMax = 100, Fluid2_type = P.fluid2_type, I = 0;
    const std::string& codeOpt = S->codeOpt;
    if (P.method != 3)
        PNUM(I, KTYPE, DIM, TP, re, S->neighb, S->x, S->y, S->z, P.ncorrection, S->n, S->MAX,
             S->pnew, S->p, true, codeOpt);
    NEIGHBOR(P.xmax, P.xmin, P.ymax, P.ymin, P.zmax, P.zmin, re, P.delta, TP, S->x, S->y, S->z,
             S->neighb, DIM, codeOpt);
    if (P.turb)
        SPS(re, TP, GP, S->neighb, S->x, S->y, S->z, P.coll, KTYPE, S->unew, S->vnew, S->wnew, n0,
            S->NEUt, P.cs, P.l0, S->TURB1, S->TURB2, S->TURB3, DIM, codeOpt);
    V_FRACTION(re, P.fraction_method, TP, S->neighb, S->PTYPE, S->C, KTYPE, S->x, S->y, S->z, DIM,
               codeOpt);
    VISCOSITY(re, TP, Fluid2_type, S->PTYPE, S->MEU, P.nu1, P.nu2, P.rho1, P.rho2, S->neighb,
              S->x, S->y, S->z, KTYPE, S->unew, S->vnew, S->wnew, n0, S->C, P.phi, I, P.cohes,
              II, yield_stress, S->phat, P.meu0, P.n_pl, DIM, codeOpt);
    PREDICTION(re, S->xstar, S->ystar, S->zstar, S->ustar, S->vstar, S->wstar, S->u, S->v, S->w,
               TP, S->PTYPE, S->MEU, P.rho1, P.rho2, S->neighb, S->x, S->y, S->z, KTYPE, n0,
               S->phat, S->pnew, P.gx, P.gy, P.gz, DT, S->NEUt, S->lambda, S->TURB1, S->TURB2,
               S->TURB3, P.relaxp, S->RHO, S->SFX, S->SFY, DIM, codeOpt);
    PNUMSTAR(KTYPE, DIM, TP, re, S->neighb, S->xstar, S->ystar, S->zstar, S->nstar, codeOpt);
    if (P.method != 3) BCON(S->PTYPE, S->bcon, S->nstar, n0, P.dirichlet, TP, codeOpt);
    PRESSURECALC(P.method, GP, FP, WP, TP, S->PTYPE, c0, P.c01, P.c02, P.rho1, P.rho2, S->C,
                 S->nstar, P.beta_fs, n0, S->pnew, P.pmin, P.pmax, IterMax, MAXresi, re, S->x,
                 S->y, S->z, P.coll, KTYPE, correction, Rho, P.relaxp, S->lambda, DT, S->p, S->n,
                 DIM, S->neighb, S->poiss, S->bcon, S->source, S->ic, P.imin, P.imax, P.eps,
                 S->ustar, S->vstar, S->wstar, P.matopt != 0, P.srcopt != 0, codeOpt);
    PHATCALC(TP, S->neighb, S->pnew, S->phat, codeOpt);
    PRESSGRAD(GP, WP, P.kh, TP, S->pnew, S->neighb, S->xstar, S->ystar, S->zstar, S->phat, KTYPE,
              re, S->RHO, S->ustar, S->vstar, S->wstar, DT, S->unew, S->vnew, S->wnew, P.relaxp,
              n0, P.vmax, DIM, codeOpt, S->nstar);
    EULERINTEGRATION(GP, WP, TP, DT, S->x, S->y, S->z, S->unew, S->vnew, S->wnew, P.l0, P.xmax,
                     P.xmin, P.ymax, P.ymin, P.zmax, P.zmin, I, P.velcor, DIM, S->test, codeOpt);
    COLLISION2(TP, P.coll, S->PTYPE, P.rho1, P.rho2, S->neighb, P.cc, S->unew, S->vnew, S->wnew,
               S->x, S->y, S->z, DT, DIM, codeOpt);
    PREPDATA(TP, FP, S->x, S->y, S->z, S->u, S->v, S->w, S->p, S->unew, S->vnew, S->wnew,
             S->pnew, P.xmin, P.ymin, P.xmax, P.ymax, P.zmin, P.zmax, DIM, S->test, codeOpt);
    return 0;
}

/* Copy a field out in 0-based order.  Lists come out as CSR: "off" (n+1)
   and "nbr" (0-based indices, the reference's slot order). */
long rh_get(void* h, const char* name, void* out)
{
    RefState* S = (RefState*)h;
    int TP = S->TP;
    if (!strcmp(name, "off") || !strcmp(name, "nbr")) {
        long total = 0;
        int* o = (int*)out;
        for (int I = 1; I <= TP; I++) {
            int cnt = S->neighb[I][1] - 1;
            if (!strcmp(name, "off")) {
                if (o) o[I - 1] = (int)total;
            } else if (o) {
                for (int l = 0; l < cnt; l++) o[total + l] = S->neighb[I][l + 2] - 1;
            }
            total += cnt;
        }
        if (!strcmp(name, "off")) {
            if (o) o[TP] = (int)total;
            return TP + 1;
        }
        return total;
    }
    struct { const char* nm; double* a; } dbl[] = {
        {"x", S->x}, {"y", S->y}, {"z", S->z}, {"u", S->u}, {"v", S->v}, {"w", S->w},
        {"p", S->p}, {"pnew", S->pnew}, {"phat", S->phat}, {"un", S->unew}, {"vn", S->vnew},
        {"wn", S->wnew}, {"xs", S->xstar}, {"ys", S->ystar}, {"zs", S->zstar},
        {"us", S->ustar}, {"vs", S->vstar}, {"ws", S->wstar}, {"n", S->n},
        {"nstar", S->nstar}, {"C", S->C}, {"meu", S->MEU}, {"neut", S->NEUt},
        {"t1", S->TURB1}, {"t2", S->TURB2}, {"t3", S->TURB3}, {"rho", S->RHO},
        {"source", S->source}};
    for (auto& d : dbl)
        if (!strcmp(name, d.nm)) {
            if (out) memcpy(out, d.a + 1, sizeof(double) * (size_t)TP);
            return TP;
        }
    if (!strcmp(name, "bcon") || !strcmp(name, "ptype")) {
        int* src = !strcmp(name, "bcon") ? S->bcon : S->PTYPE;
        if (out) memcpy(out, src + 1, sizeof(int) * (size_t)TP);
        return TP;
    }
    if (!strcmp(name, "diag") && S->P.method != 3) {
        double* o = (double*)out;
        if (o) for (int I = 1; I <= TP; I++) o[I - 1] = S->poiss[I][1];
        return TP;
    }
    return -1;
}

/* Overwrite one double field (0-based input) between stage calls, as
   main.cu's caller-owned arrays allow.  Returns the count or -1. */
long rh_set(void* h, const char* name, const void* in)
{
    RefState* S = (RefState*)h;
    struct { const char* nm; double* a; } dbl[] = {
        {"x", S->x}, {"y", S->y}, {"z", S->z}, {"u", S->u}, {"v", S->v}, {"w", S->w},
        {"p", S->p}, {"pnew", S->pnew}, {"un", S->unew}, {"vn", S->vnew}, {"wn", S->wnew}};
    for (auto& d : dbl)
        if (!strcmp(name, d.nm)) {
            memcpy(d.a + 1, in, sizeof(double) * (size_t)S->TP);
            return S->TP;
        }
    return -1;
}

/* One reference routine on the harness state: "NEIGHBOR" (at re_s, the
   harness radius) or "COLLISION2" (functions.cu:2788, 1523), called with
   main.cu's arguments.  Returns 0, or -1 for an unknown name. */
int rh_stage(void* h, const char* name)
{
    RefState* S = (RefState*)h;
    const mo_params& P = S->P;
    omp_set_num_threads(S->nthreads);
    if (!strcmp(name, "NEIGHBOR")) {
        NEIGHBOR(P.xmax, P.xmin, P.ymax, P.ymin, P.zmax, P.zmin, P.re_s, P.delta, S->TP, S->x,
                 S->y, S->z, S->neighb, S->DIM, S->codeOpt);
        return 0;
    }
    if (!strcmp(name, "COLLISION2")) {
        COLLISION2(S->TP, P.coll, S->PTYPE, P.rho1, P.rho2, S->neighb, P.cc, S->unew, S->vnew,
                   S->wnew, S->x, S->y, S->z, P.dt, S->DIM, S->codeOpt);
        return 0;
    }
    return -1;
}

/* the reference's kernel function itself (functions.cu:32-74) */
double rh_W(double r, int ktype, int dim, double re) { return W(r, ktype, dim, re); }

double rh_scalar(void* h, const char* name)
{
    RefState* S = (RefState*)h;
    if (!strcmp(name, "n0")) return S->n0;
    if (!strcmp(name, "lambda")) return S->lambda;
    if (!strcmp(name, "neighbors_cap")) return (double)NEIGHBORS;
    return NAN;
}

void rh_destroy(void* h)
{
    RefState* S = (RefState*)h;
    if (!S) return;
    for (int m = 0; m <= S->TP; m++) delete[] S->neighb[m];
    delete[] S->neighb;
    if (S->P.method != 3) {
        for (int m = 1; m <= S->TP; m++) { delete[] S->poiss[m]; delete[] S->ic[m]; }
    }
    delete[] S->poiss; delete[] S->ic;
    double* arrs[] = {S->x, S->y, S->z, S->u, S->v, S->w, S->p, S->xstar, S->ystar, S->zstar,
                      S->ustar, S->vstar, S->wstar, S->pnew, S->phat, S->unew, S->vnew, S->wnew,
                      S->NEUt, S->TURB1, S->TURB2, S->TURB3, S->n, S->nstar, S->MEU, S->C,
                      S->RHO, S->SFX, S->SFY, S->source};
    for (double* a : arrs) delete[] a;
    delete[] S->PTYPE; delete[] S->bcon; delete[] S->MAX;
    delete S;
}

}  // extern "C"
