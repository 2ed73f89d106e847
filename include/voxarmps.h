/*
 * voxarmps.h -- C-ABI of the Blackwell-native (sm_100a) MPS solver core.
 *
 * Drop-in for the per-step entry points of VoxarMPS (declared in
 * VoxarMPS/VoxarMPS/functions.cuh:56-111 and driven by main.cu:1027-1363).
 * The reference passes 1-based host arrays to free functions that mutate
 * them; here a context owns every device buffer, the caller's host arrays
 * are borrowed only for the duration of a call, and every call returns a
 * status code instead of printing (functions.cu:2720-2743) or exit()ing.
 *
 * Particle arrays crossing this boundary are 0-based and in the caller's
 * particle order (the reference's id order).  Inside the context particles
 * live in cell order; downloads translate back.
 *
 * Thread safety: one context per host thread / stream; no global state.
 */
#ifndef VOXARMPS_H
#define VOXARMPS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (bit flags; a call may return several) ---------------- */
#define MPS_OK 0
#define MPS_ERR_ARG 1             /* bad argument / call order */
#define MPS_ERR_CUDA 2            /* CUDA runtime error (message: mps_last_message) */
#define MPS_ERR_NAN 4             /* non-finite p/u/v/w, reference ERROR#1 (functions.cu:2720) */
#define MPS_ERR_BOX 8             /* particle at/outside the box, ERROR#2 (functions.cu:2725) */
#define MPS_ERR_CELL 16           /* particle outside the cell grid (unchecked in NEIGHBOR) */
#define MPS_ERR_LIST_OVERFLOW 32  /* a neighbour list exceeded its capacity (inOut.h:30) */
#define MPS_ERR_NOT_CONVERGED 64  /* PPE did not reach cg_tol within cg_max iterations */
#define MPS_ERR_IO 128            /* file could not be read / written */

/* ---- configuration ------------------------------------------------------ *
 * Every constant main.cu hard-codes (main.cu:211-394) is a field.  The
 * Python mirror is voxarmps_b200.config.FIELDS (same order). */
typedef struct mps_config {
    int dim;              /* 2 or 3 (main.cu:186) */
    int ktype;            /* kernel function type 1,2,3,5,6 (functions.cu:32-74) */
    int method;           /* 1 fully incompressible PPE, 3 weakly compressible (main.cu:338) */
    double l0;            /* particle spacing DL */
    double re_s;          /* PND / gradient / collision support radius */
    double re_l;          /* Laplacian (PPE, viscous term) support radius */
    double delta;         /* DELTA: 3D z-cell expansion and 3D cutoff slack (main.cu:283) */
    double dt;
    double gx, gy, gz;
    double rho1, rho2, nu1, nu2;
    double beta_fs;       /* WC free-surface threshold */
    double dirichlet;     /* free surface where n_star / n0 < dirichlet (main.cu:226) */
    double relaxp;
    int kh;               /* Khayyer-Gotoh pressure-gradient correction */
    double vmax;
    double coll;          /* collision distance */
    double cc;            /* collision restitution coefficient */
    double velcor;        /* wall reflection factor (main.cu:1293) */
    double ncorrection;   /* PND correction for ktype != 2 */
    double pmin, pmax;
    double c01, c02;      /* WC sound speeds */
    int turb;             /* SPS-LES turbulence */
    double cs;            /* Smagorinsky constant */
    int fluid2_type;      /* 0 Newtonian, 1 Herschel-Bulkley second fluid */
    double n_pl, meu0, phi, cohes;
    int matopt, srcopt;   /* HL Laplacian, HS+ECS source */
    int fraction_method;  /* 1 linear, 2 kernel-smoothed */
    int ppe_at_predicted; /* 1: A at x*, b from n* (reference GPU path); 0: CPU path */
    int warm_start;       /* CG initial guess: 0 zero, 1 previous pressure, 2 2p^n - p^(n-1) */
    int solver;           /* 1 Jacobi-PCG, 2 unpreconditioned CG (relative residual) */
    double cg_tol;        /* relative residual ||b-Ax||/||b|| */
    int cg_max;
    int imin, imax;       /* kept for layout parity with the oracle; unused here */
    double eps;
    int collision_gather; /* must be 1: order-independent collision */
    double xmin, xmax, ymin, ymax, zmin, zmax;  /* grown bounding box (main.cu:692-715) */
    /* B200 path knobs (no reference counterpart) */
    int precision;        /* 0 FP64 throughout; 1 mixed PPE (FP32 inner CG, FP64 dots and
                             refinement) and FP32 viscous sums; 2 as 1, with PNUMSTAR and
                             the pressure gradient in FP32 as well */
    int list_cap_s;       /* neighbour-list capacity per particle, 0 = automatic */
    int list_cap_l;
} mps_config;

typedef struct mps_ctx mps_ctx;

/* Lifecycle.  Replaces main.cu's allocation block (main.cu:726-921). */
int mps_create(const mps_config* cfg, int device, mps_ctx** out);
int mps_destroy(mps_ctx* ctx);

/* Host -> device particle upload (main.cu:947-962).  z, w may be NULL in
 * 2D; u, v, w, p may be NULL (zero).  Arrays are borrowed for the call. */
int mps_upload(mps_ctx* ctx, int n, const double* x, const double* y, const double* z,
               const int* ptype, const double* u, const double* v, const double* w,
               const double* p);
/* Read a .grd file (main.cu:496-684 format) and upload it. */
int mps_load_grd(mps_ctx* ctx, const char* path);

/* Batched independent scenes (no reference counterpart: the reference runs
 * one scene per process).  Call after mps_upload and before mps_init.
 * scene[i] in [0, nscenes): the scene of particle i (caller order); boxes:
 * 6 doubles per scene (xmin xmax ymin ymax zmin zmax, the grown box of
 * main.cu:692-715); pmax: one per scene (main.cu:548).  Scenes share one
 * cell grid and must be separated by more than re_l so that no list
 * crosses scenes; they must share spacing, radii and kernel (one n0).
 * Wall clamps, the box check and the pressure cap use each particle's
 * scene; the PPE is solved until every scene's own relative residual is
 * <= cg_tol. */
int mps_set_scenes(mps_ctx* ctx, int nscenes, const int* scene, const double* boxes,
                   const double* pmax);

/* Pre-iteration work (main.cu:964-1012): density, lists, n0 = max PND. */
int mps_init(mps_ctx* ctx);

/* Per-stage entry points, one per reference routine, in main.cu's order. */
int mps_pnd(mps_ctx* ctx);                /* PNUM           functions.cu:94   */
int mps_neighbors(mps_ctx* ctx);          /* NEIGHBOR       functions.cu:2788 */
int mps_sps(mps_ctx* ctx);                /* SPS            functions.cu:1719 */
int mps_vfraction(mps_ctx* ctx);          /* V_FRACTION     functions.cu:2580 */
int mps_viscosity(mps_ctx* ctx);          /* VISCOSITY      functions.cu:2053 */
int mps_predict(mps_ctx* ctx);            /* PREDICTION     functions.cu:2283 */
int mps_pnd_star(mps_ctx* ctx);           /* PNUMSTAR       functions.cu:157  */
int mps_bcon(mps_ctx* ctx);               /* BCON           functions.cu:433  */
int mps_pressure(mps_ctx* ctx, int* iters, double* relres); /* PRESSURECALC functions.cu:2465 */
int mps_phat(mps_ctx* ctx);               /* PHATCALC       functions.cu:207  */
int mps_pressure_gradient(mps_ctx* ctx);  /* PRESSGRAD      functions.cu:245  */
int mps_integrate(mps_ctx* ctx);          /* EULERINTEGRATION functions.cu:2004 */
int mps_collision(mps_ctx* ctx);          /* COLLISION2     functions.cu:1523 */
int mps_commit(mps_ctx* ctx);             /* PREPDATA       functions.cu:2688 */

/* One full time step (main.cu:1027-1349 loop body) / several steps. */
int mps_step(mps_ctx* ctx);
int mps_run(mps_ctx* ctx, int steps);

/* Device -> host.  Field names: x y z u v w p pnew phat un vn wn xs ys zs us vs
 * ws n nstar C meu neut t1 t2 t3 rho source diag (double); ptype bcon (int);
 * cell_s cell_l (int, 1-based Cnum per particle, NEIGHBOR's cell number);
 * perm_s perm_l (int, particle ids in cell order: NEIGHBOR's ip[]).
 * Returns MPS_OK; *count (optional) receives the element count. */
int mps_download(mps_ctx* ctx, const char* field, void* out, long* count);
/* Neighbour lists in particle-id space, CSR: which 0 = PND radius, 1 =
 * Laplacian radius.  off has n+1 entries; nbr needs off[n] (query with
 * nbr == NULL first: *total receives the entry count). */
int mps_download_lists(mps_ctx* ctx, int which, int* off, int* nbr, long* total);
/* Overwrite / read the particle state between steps, host arrays in the
 * caller's particle order (the reference keeps x..p in caller-owned host
 * arrays across steps, main.cu:554-563).  NULL arrays are skipped; set_state
 * also sets pnew = p as PREPDATA leaves it (functions.cu:2700). */
int mps_set_state(mps_ctx* ctx, const double* x, const double* y, const double* z,
                  const double* u, const double* v, const double* w, const double* p);
int mps_get_state(mps_ctx* ctx, double* x, double* y, double* z, double* u, double* v,
                  double* w, double* p);
/* mps_set_state, mps_step and mps_get_state in one call: in[k] and out[k]
 * are the caller-order host arrays of x y z u v w p (NULL skips one; in and
 * out may be the same arrays).  The same results as the three calls; the
 * copy of u, v, w, p runs on a second stream while the step's neighbour
 * search runs, and they are applied after its reorder.  No counterpart in
 * the reference, whose loop (main.cu:1027-1363) keeps the state in host
 * arrays across steps: this is that loop's step with its host copies
 * overlapped.  Returns mps_step's status bits with mps_get_state's. */
int mps_step_io(mps_ctx* ctx, const double* const* in, double* const* out);
/* Overwrite one state array between stage calls, host doubles in the caller's
 * particle order: x y z u v w (the packed copies the stages read follow),
 * p, pnew, un vn wn (the corrected velocity COLLISION2 and PREPDATA read),
 * phat (the previous step's, read by PREDICTION), pold (p^(n-1)).
 * The reference's caller owns these arrays and may write them between any
 * two calls of main.cu's loop (main.cu:1027-1363); this is that write. */
int mps_set_field(mps_ctx* ctx, const char* field, const double* in);
/* ---- one scene split between contexts (slab decomposition) -------------- *
 * No counterpart in the reference (one process, one scene).  Each context
 * holds the particles of one slab of the scene plus ghost copies of its
 * neighbours' particles near the slab faces (voxarmps_b200/slab.py drives
 * it).  mps_set_owned: 1 for the particles this context owns, 0 for ghosts
 * (caller order; all 1 after mps_upload); ghost rows stay out of this
 * context's PPE system but remain columns of the owned rows.  mps_set_n0
 * replaces n0 (the scene's, formed over all contexts).  mps_get_rows /
 * mps_set_rows read / write one double field (names as mps_download, plus
 * "cg_p", the CG direction) at the given caller-order indices: the ghost
 * exchanges.  The PPE then runs host-driven, FP64 Jacobi-PCG only
 * (precision 0, method 1): mps_ppe_assemble (MATRIX, source, initial
 * guess), mps_dcg_start (local b.b, r.z, r.r), and per iteration
 * mps_dcg_spmv (local p.s), mps_dcg_update (local r.z, r.r after x += a p,
 * r -= a s), mps_dcg_direction (p = z + b p); the caller sums the local
 * values over the contexts and exchanges the ghost entries of pnew and
 * cg_p between the calls; mps_dcg_finish clamps and records the outcome
 * (bb: the scene's b.b). */
int mps_set_owned(mps_ctx* ctx, const int* owned);
int mps_set_n0(mps_ctx* ctx, double n0_s, double n0_l);
int mps_get_rows(mps_ctx* ctx, const char* field, int count, const int* ids, double* out);
int mps_set_rows(mps_ctx* ctx, const char* field, int count, const int* ids, const double* in);
int mps_ppe_assemble(mps_ctx* ctx);
int mps_dcg_start(mps_ctx* ctx, double* local3);
int mps_dcg_spmv(mps_ctx* ctx, double* local_ps);
int mps_dcg_update(mps_ctx* ctx, double alpha, double* local2);
int mps_dcg_direction(mps_ctx* ctx, double beta);
int mps_dcg_finish(mps_ctx* ctx, int iters, double relres, double bb);

/* Per-stage device timing with CUDA events (off by default).  While on,
 * scalars ms_neighbors ms_explicit ms_ppe ms_post ms_step (last step) and
 * spmv_ms / spmv_launches, lists_ms (accumulated) are available. */
int mps_set_profile(mps_ctx* ctx, int on);

/* Graph mode (no reference counterpart; the reference launches every stage
 * from the host).  When on, mps_step captures the whole step, the PPE's CG
 * loop included as a conditional while node, into a CUDA graph on its first
 * call for each of the two reorder buffer sets and replays it afterwards:
 * one graph launch and one host synchronisation per step.  Results are
 * identical to eager mode.  Off while profiling (mps_set_profile). */
int mps_set_graph(mps_ctx* ctx, int on);

/* ---- launch-shape autotuning (no reference counterpart) ------------------ *
 * small_lanes: lanes per row of the PND-radius list in the list build and
 * every stage over that list (4 or 8; sums over a row
 * change order with it, results stay within rounding).  cg_blocks_per_sm:
 * grid of the CG kernels (1..8, 0 = as many as fit). */
typedef struct mps_tuning {
    int small_lanes;
    int cg_blocks_per_sm;
} mps_tuning;
int mps_get_tuning(mps_ctx* ctx, mps_tuning* out);
int mps_set_tuning(mps_ctx* ctx, const mps_tuning* in);
/* Time every candidate over `steps` steps each (CUDA events, eager launches;
 * these are real steps that advance the simulation), keep the fastest per
 * parameter and return it.  Call it in place of the first warm-up steps. */
int mps_autotune(mps_ctx* ctx, int steps, mps_tuning* chosen);

/* ---- learned CG initial guess (no reference counterpart) ---------------- *
 * A message-passing network on the PND-radius neighbour graph (hidden width
 * 64, `layers` residual layers, BF16 weights/activations, FP32 sums) maps
 * per-particle inputs (PND deviation, previous pressure, particle kind) to
 * the pressure increment of the coming solve.  While a network exists every
 * PPE captures its inputs; mps_gnn_train then fits the network to the
 * pressure that PPE solved for.  With mps_gnn_use(ctx, 1) the prediction is
 * CG's starting point; CG still runs to cg_tol, so only the iteration count
 * changes.  Weights start from SplitMix64(seed) with a zero output layer
 * (the untrained guess is the previous pressure). */
int mps_gnn_create(mps_ctx* ctx, int layers, unsigned long long seed);
int mps_gnn_use(mps_ctx* ctx, int on);
/* `iters` Adam steps (learning rate lr) on the last PPE.  objective 0: mean
 * squared error of the scaled pressure increment against the solved one;
 * objective 1: relative squared residual |b - A x0|^2/|b|^2 that the guess
 * x0 leaves in that PPE's system.  grad_only != 0 only computes the
 * gradient.  *loss = the objective before the last update. */
int mps_gnn_train(mps_ctx* ctx, int iters, float lr, int objective, int grad_only, float* loss);
/* copy the FP32 parameters out (get) and/or in (set, resets Adam); *count = P */
int mps_gnn_params(mps_ctx* ctx, float* get, const float* set, int* count);
/* the whole training state out and/or in: parameters, Adam's first and
 * second moments (P each) and its step count; *count = 3P + 1.  Passing it
 * from context to context trains one network on several scenes. */
int mps_gnn_state(mps_ctx* ctx, float* get, const float* set, int* count);
/* inputs of the current state / forward pass on the captured inputs */
int mps_gnn_features(mps_ctx* ctx);
int mps_gnn_forward(mps_ctx* ctx);
/* network data in slot (cell) order: "feat", "target", "y", "grad", "pref",
 * "count", "nbr", "len", "bcon", "ptype", "cap" */
int mps_gnn_download(mps_ctx* ctx, const char* what, void* out, long* count);
/* Scalars: n0_s n0_l lambda_l cg_iters cg_relres n nnz_s nnz_l nnz_a steps
 * cap_s cap_l len_max_s len_max_l launches pmax and the profile timings. */
int mps_get_scalar(mps_ctx* ctx, const char* name, double* out);
/* Accumulated MPS_ERR_* bits since the last call (then cleared). */
int mps_get_error(mps_ctx* ctx);
const char* mps_last_message(mps_ctx* ctx);
/* VTU writer (inOut.cpp:104-336 format, ASCII UnstructuredGrid). */
int mps_write_vtu(mps_ctx* ctx, const char* path, int fluid_only);
/* Binary VTU snapshot: VTK XML UnstructuredGrid with raw appended data
 * (Float32 position/velocity/pressure, Int32 partType).  The state is copied
 * device-to-host on the context's stream and the file is written by a host
 * thread while later steps run; mps_wait_io joins that thread and returns
 * its status.  One snapshot is in flight at a time. */
int mps_snapshot_vtu(mps_ctx* ctx, const char* path, int fluid_only);
int mps_wait_io(mps_ctx* ctx);

/* Binary checkpoint of the full persistent state (replaces the reference's
 * disabled VTU read-back, inOut.cpp:25-102, main.cu:393): configuration,
 * n0, step count, every field carried between steps, scenes; checksummed.
 * mps_load_checkpoint replaces the context's configuration and state; the
 * resumed run continues bit for bit. */
int mps_save_checkpoint(mps_ctx* ctx, const char* path);
int mps_load_checkpoint(mps_ctx* ctx, const char* path);

/* Device stream the context launches on (cudaStream_t as void*). */
void* mps_stream(mps_ctx* ctx);

/* Allocation-free binning: the 1-based cell number of every particle and
 * the particles in cell order (ascending index inside a cell), for the grid
 * of support radius re over the box in cfg -- the first half of NEIGHBOR --
 * written to caller-owned device buffers.  For callers that may not
 * allocate device memory (an application that owns the whole device heap
 * through its own pool, or a loop that forbids allocation after start-up).
 * It has no counterpart in the reference.  x, y, z (z unused in 2D): device
 * positions; cell, perm: device outputs of n ints; out_of_grid: device word
 * set non-zero when a particle lies outside the grid; stream: cudaStream_t
 * or NULL.  Limits: n <= 262,144 particles and at most 262,142 cells;
 * larger inputs return MPS_ERR_ARG.  Scratch is a fixed static device area
 * shared by all calls (calls that overlap on the GPU race); a call outside
 * a stream capture looks its address up (again after a cudaDeviceReset), a
 * call during a capture reuses the last address found on that device, so
 * the first call on each device should come before any stream capture.
 * Asynchronous on stream. */
int mps_cell_order_noalloc(const mps_config* cfg, double re, int n, const double* x,
                           const double* y, const double* z, int* cell, int* perm,
                           unsigned int* out_of_grid, void* stream);

#ifdef __cplusplus
}
#endif
#endif
