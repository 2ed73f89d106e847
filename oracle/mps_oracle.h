/*
 * mps_oracle.h -- CPU restatement of the VoxarMPS per-step MPS pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  The product library
 * (voxarmps_b200/) never links, loads or calls it.
 *
 * Every function restates one reference routine in plain C99, in double
 * precision, with the reference's operation order kept wherever it decides
 * the bits of the result.  Citations are to VoxarMPS/VoxarMPS/<file>:<line>.
 *
 * Conventions that differ from the reference (layout only, not semantics):
 *   - arrays are 0-based (the reference is 1-based);
 *   - neighbour lists are CSR (off[n+1], nbr[]) holding 0-based particle
 *     indices in the reference's own list order (functions.cu:2854-2918);
 *   - the reference's single support radius is split into a PND/gradient
 *     radius (re_s) and a Laplacian radius (re_l).  With re_s == re_l the
 *     pipeline is the reference's, bit for bit (pinned by the golden tests).
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mo_params {
    int dim;              /* 2 or 3 */
    int ktype;            /* kernel type: 1,2,3,5,6 (functions.cu:32-74) */
    int method;           /* 1: fully incompressible PPE, 3: weakly compressible EOS */
    double l0;            /* DL, particle spacing */
    double re_s;          /* PND / gradient / collision list radius */
    double re_l;          /* Laplacian (PPE, viscosity) radius */
    double delta;         /* DELTA: 3D z-cell expansion and 3D cutoff slack */
    double dt;
    double gx, gy, gz;
    double rho1, rho2, nu1, nu2;
    double beta_fs;       /* WC free-surface threshold BETA (main.cu:254) */
    double dirichlet;     /* BCON threshold (main.cu:226) */
    double relaxp;
    int kh;               /* KHcorrection (main.cu:354) */
    double vmax;
    double coll;          /* collision distance */
    double cc;            /* collision coefficient */
    double velcor;        /* wall reflection factor passed to BOUNDARIE (main.cu:1293) */
    double ncorrection;   /* n0 correction for ktype != 2 */
    double pmin, pmax;
    double c01, c02;      /* WC sound speeds */
    int turb;             /* SPS-LES on/off */
    double cs;            /* Smagorinsky constant */
    int fluid2_type;      /* 0 Newtonian, 1 Herschel-Bulkley */
    double n_pl, meu0, phi, cohes;
    int matopt, srcopt;
    int fraction_method;  /* 1 linear, 2 smoothed */
    /* PPE semantics switches (reference CPU path vs GPU path, see the header
       of mo_step): ppe_at_predicted=1 assembles A at x* and b from n*. */
    int ppe_at_predicted;
    int warm_start;       /* 0: zero, 1: previous pressure, 2: 2 p^n - p^(n-1) */
    int solver;           /* 0: reference ICCG with its absolute per-row stop rule,
                             1: Jacobi-preconditioned CG to a relative residual,
                             2: unpreconditioned CG to a relative residual */
    double cg_tol;        /* relative residual for solver 1/2 */
    int cg_max;           /* iteration cap for solver 1/2 */
    int imin, imax;       /* reference CGM bounds (main.cu:229) */
    double eps;           /* reference CGM per-row tolerance (main.cu:230) */
    int collision_gather; /* 1: order-independent (Jacobi) collision */
    double xmin, xmax, ymin, ymax, zmin, zmax;  /* grown bounding box */
} mo_params;

/* ---- kernel function and geometry (functions.cu:32-89) ---- */
double mo_W(double r, int ktype, int dim, double re);
double mo_lambda(int ktype, double re);            /* main.cu:491-494 */

/* ---- neighbour search (functions.cu:2788-2929) ----
 * cell[i]: 1-based Cnum of particle i; perm[k]: particle index at sorted
 * slot k (the reference's ip[], stable by cell).  Lists are written in the
 * reference's scan order.  Returns the number of list entries, or
 * -(needed) when cap is too small, or -1-INT_MAX... on a cell out of range
 * (return value MO_ERR_CELL). */
#define MO_ERR_CELL (-2147483647)
int mo_grid(const mo_params* P, double re, int* ncx, int* ncy, int* ncz);
int mo_neighbor(const mo_params* P, double re, int n, const double* x, const double* y,
                const double* z, int* cell, int* perm, int* off, int* nbr, int cap);

/* ---- per-stage routines ---- */
/* correct != 0: PNUM (applies Ncorrection for ktype != 2); correct == 0:
   PNUMSTAR, which never applies it (functions.cu:157-179). */
void mo_pnd(const mo_params* P, double re, int n, const int* off, const int* nbr,
            const double* x, const double* y, const double* z, int correct, double* nd);
double mo_max(int n, const double* a);
void mo_bcon(int n, const int* ptype, const double* nd, double n0, double dirichlet, int* bcon);
void mo_matrix(const mo_params* P, double re, double lambda, double n0, int n, const int* off,
               const int* nbr, const double* x, const double* y, const double* z,
               const int* bcon, double* diag, double* val);
void mo_source(const mo_params* P, double n0, int n, const int* ptype, const int* bcon,
               const double* nsrc, double* source);
void mo_source_hs(const mo_params* P, double re, double n0, int n, const int* off,
                  const int* nbr, const int* ptype, const int* bcon, const double* nstar,
                  const double* x, const double* y, const double* z, const double* u,
                  const double* v, const double* w, double* source);
void mo_incdecom(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
                 const double* val, double* icd, double* icv);
int mo_cgm_ref(const mo_params* P, int n, const int* off, const int* nbr, const int* bcon,
               const double* diag, const double* val, const double* icd, const double* icv,
               const double* b, double* x);
int mo_cg(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
          const double* val, const double* b, double* x, double tol, int maxit, int precond,
          double* relres_out);
int mo_iccg(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
            const double* val, const double* icd, const double* icv, const double* b, double* x,
            double tol, int maxit, double* relres_out);
void mo_spmv(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
             const double* val, const double* xin, double* s);
double mo_relres(int n, const int* off, const int* nbr, const int* bcon, const double* diag,
                 const double* val, const double* b, const double* x);
void mo_pressure_wc(const mo_params* P, double n0, int n, const int* ptype, const double* C,
                    const double* nstar, double* pnew);
void mo_phat(int n, const int* off, const int* nbr, const double* pnew, double* phat);
void mo_pressgrad(const mo_params* P, double re, double n0, int n, const int* off,
                  const int* nbr, const int* ptype, const double* pnew, const double* phat,
                  const double* xs, const double* ys, const double* zs, const double* rho,
                  const double* us, const double* vs, const double* ws, double* un, double* vn,
                  double* wn);
void mo_prediction(const mo_params* P, double re_s, double n0_s, const int* off_s,
                   const int* nbr_s, double re_l, double n0_l, double lambda_l,
                   const int* off_l, const int* nbr_l, int n, const int* ptype,
                   const double* meu, const double* x, const double* y, const double* z,
                   const double* u, const double* v, const double* w, const double* pnew,
                   const double* phat, const double* neut, const double* t1, const double* t2,
                   const double* t3, const double* rho, double* xs, double* ys, double* zs,
                   double* us, double* vs, double* ws);
void mo_viscosity(const mo_params* P, double re, double n0, int n, const int* off,
                  const int* nbr, const int* ptype, const double* x, const double* y,
                  const double* z, const double* un, const double* vn, const double* wn,
                  const double* C, const double* phat, double* meu);
void mo_sps(const mo_params* P, double re, double n0, int n, const int* off, const int* nbr,
            const int* ptype, const double* x, const double* y, const double* z,
            const double* un, const double* vn, const double* wn, double* neut, double* t1,
            double* t2, double* t3);
void mo_vfraction(const mo_params* P, double re, int n, const int* off, const int* nbr,
                  const int* ptype, const double* x, const double* y, const double* z,
                  double* C);
void mo_collision(const mo_params* P, int n, const int* off, const int* nbr, const int* ptype,
                  double* un, double* vn, double* wn, double* x, double* y, double* z);
void mo_collision_gather(const mo_params* P, int n, const int* off, const int* nbr,
                         const int* ptype, double* un, double* vn, double* wn, double* x,
                         double* y, double* z);
void mo_euler(const mo_params* P, int n, const int* ptype, double* x, double* y, double* z,
              double* un, double* vn, double* wn);
int mo_prepdata(const mo_params* P, int n, const int* ptype, const double* x, const double* y,
                const double* z, double* u, double* v, double* w, double* p, const double* un,
                const double* vn, const double* wn, const double* pnew);

/* ---- whole pipeline, main.cu:1027-1363 ---- */
typedef struct mo_state mo_state;
mo_state* mo_create(const mo_params* P, int n, const double* x, const double* y,
                    const double* z, const int* ptype, const double* u, const double* v,
                    const double* w, const double* p);
void mo_destroy(mo_state* S);
int mo_init(mo_state* S);      /* lists + n0 (main.cu:980-1012) */
int mo_step(mo_state* S);      /* one time step, returns 0 or an error code */
/* copy a named field into out (doubles or ints); returns element count or -1 */
long mo_get(mo_state* S, const char* name, void* out);
long mo_set(mo_state* S, const char* name, const void* in);
double mo_scalar(mo_state* S, const char* name);

#ifdef __cplusplus
}
#endif
#endif
