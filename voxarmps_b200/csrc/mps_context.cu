// mps_context.cu -- the C-ABI (include/voxarmps.h): context lifecycle,
// device memory, host<->device transfers in the caller's particle order,
// the step driver in main.cu's stage order, .grd input and VTU output.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "mps_internal.cuh"

using namespace vmps;

static std::atomic<long long> g_launches{0};
int vmps_count_launch(int k)
{
    g_launches += k;
    return 0;
}

int vmps_check(mps_ctx* ctx, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return MPS_OK;
    if (ctx) ctx->msg = std::string(what) + ": " + cudaGetErrorString(e);
    return MPS_ERR_CUDA;
}

namespace {

template <typename T>
int dalloc(mps_ctx* c, T** p, size_t count)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, (count > 0 ? count : 1) * sizeof(T));
    if (e != cudaSuccess) return vmps_check(c, e, "cudaMalloc");
    e = cudaMemsetAsync(q, 0, (count > 0 ? count : 1) * sizeof(T), c->stream);
    if (e != cudaSuccess) return vmps_check(c, e, "cudaMemsetAsync");
    c->owned.push_back(q);
    *p = (T*)q;
    return MPS_OK;
}

template <typename T>
int halloc(mps_ctx* c, T** p, size_t count)
{
    void* q = nullptr;
    cudaError_t e = cudaMallocHost(&q, (count > 0 ? count : 1) * sizeof(T));
    if (e != cudaSuccess) return vmps_check(c, e, "cudaMallocHost");
    memset(q, 0, (count > 0 ? count : 1) * sizeof(T));
    c->pinned.push_back(q);
    *p = (T*)q;
    return MPS_OK;
}

// Step graphs hold the buffer addresses they were captured with.
void drop_graphs(mps_ctx* c)
{
    for (int k = 0; k < 4; k++) {
        if (c->gexec[k]) cudaGraphExecDestroy(c->gexec[k]);
        c->gexec[k] = nullptr;
        c->gkernels[k] = 0;
        c->gdefer[k] = 0;
    }
}

void snap_join(mps_ctx* c)
{
    if (c->snap_thread.joinable()) c->snap_thread.join();
}

void free_all(mps_ctx* c)
{
    snap_join(c);
    if (c->device >= 0) cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->snap = nullptr;  // pinned, freed below
    c->snap_n = 0;
    drop_graphs(c);
    c->swaps = 0;
    for (void* q : c->owned) cudaFree(q);
    for (void* q : c->pinned) cudaFreeHost(q);
    c->owned.clear();
    c->pinned.clear();
    c->alts.clear();
}

// NEIGHBOR's grid (functions.cu:2790-2802); false when the box holds more
// than 2^30 cells or is not a finite, non-inverted box
constexpr long long kMaxCells = 1LL << 30;
bool make_grid(const mps_config& f, double re, Grid* g)
{
    return grid_for(f.xmin, f.xmax, f.ymin, f.ymax, f.zmin, f.zmax, f.dim, re, f.delta,
                    kMaxCells, g);
}

int lattice_count(int dim, double ratio, bool inclusive)
{
    int r = (int)std::ceil(ratio) + 1, cnt = 0;
    double lim = ratio * ratio;
    for (int a = -r; a <= r; a++)
        for (int b = -r; b <= r; b++)
            for (int k = (dim == 3 ? -r : 0); k <= (dim == 3 ? r : 0); k++) {
                double d2 = (double)a * a + (double)b * b + (double)k * k;
                if (inclusive ? d2 <= lim : d2 < lim) cnt++;
            }
    return cnt;
}

// row capacity: 1.5x the lattice count plus slack, rows 32-byte aligned
int auto_cap(const mps_config& f, double re)
{
    bool three = f.dim == 3;
    double ratio = (three ? re + f.delta : re) / f.l0;
    int c = lattice_count(f.dim, ratio, three);
    int cap = (int)std::ceil(c * 1.5) + 8;
    return (cap + 7) / 8 * 8;
}

int validate(const mps_config& f, std::string& why)
{
    if (f.dim != 2 && f.dim != 3) { why = "dim must be 2 or 3"; return MPS_ERR_ARG; }
    if (f.method != 1 && f.method != 3) { why = "method must be 1 or 3"; return MPS_ERR_ARG; }
    if (!(f.l0 > 0) || !(f.re_s > 0) || !(f.re_l > 0) || !(f.dt > 0)) {
        why = "l0, re_s, re_l and dt must be positive";
        return MPS_ERR_ARG;
    }
    if (f.ktype != 1 && f.ktype != 2 && f.ktype != 3 && f.ktype != 5 && f.ktype != 6) {
        why = "ktype must be 1, 2, 3, 5 or 6";
        return MPS_ERR_ARG;
    }
    if (f.solver != 1 && f.solver != 2) { why = "solver must be 1 (Jacobi-PCG) or 2 (CG)"; return MPS_ERR_ARG; }
    if (f.warm_start < 0 || f.warm_start > 2) { why = "warm_start must be 0, 1 or 2"; return MPS_ERR_ARG; }
    if (f.precision < 0 || f.precision > 2) {
        why = "precision must be 0 (FP64), 1 (mixed PPE) or 2 (mixed PPE, FP32 PND* and gradient)";
        return MPS_ERR_ARG;
    }
    return MPS_OK;
}

__global__ void k_unpermute_d(int n, const int* __restrict__ oid, const double* __restrict__ a,
                              double* __restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[oid[i]] = a[i];
}

// The caller-order state of mps_get_state / mps_set_state in one pass over
// the particles: up to seven fields between cell order and the staging
// area (field k at stage + k * pitch), so that the host copies run back to
// back with one synchronisation.
struct StateIO {
    double* f[7];  // cell-order fields (null: not transferred)
    double* pnew;  // set: also receives p
};

__global__ void k_state_out(int n, long pitch, const int* __restrict__ oid, StateIO s,
                            double* __restrict__ stage)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = oid[i];
#pragma unroll
    for (int k = 0; k < 7; k++)
        if (s.f[k]) stage[k * pitch + o] = s.f[k][i];
}

__global__ void k_state_in(int n, long pitch, const int* __restrict__ oid, StateIO s,
                           const double* __restrict__ stage)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = oid[i];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        if (!s.f[k]) continue;
        const double v = stage[k * pitch + o];
        s.f[k][i] = v;
        if (k == 6 && s.pnew) s.pnew[i] = v;
    }
}

__global__ void k_unpermute_i(int n, const int* __restrict__ oid, const int* __restrict__ a,
                              int* __restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[oid[i]] = a[i];
}

__global__ void k_perm_ids(int n, const int* __restrict__ oid, const int* __restrict__ slots,
                           int* __restrict__ out)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = slots ? oid[slots[k]] : oid[k];
}

__global__ void k_permute_in(int n, const int* __restrict__ oid, const double* __restrict__ in,
                             double* __restrict__ a, double* __restrict__ b)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = in[oid[i]];
    a[i] = v;
    if (b) b[i] = v;
}

__global__ void k_permute_in_i(int n, const int* __restrict__ oid, const int* __restrict__ in,
                               int* __restrict__ a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = in[oid[i]];
}

__global__ void k_slot_of(int n, const int* __restrict__ oid, int* __restrict__ slot_of)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) slot_of[oid[i]] = i;
}

// rows by particle index; an index outside [0, n) is reported, not followed
__global__ void k_rows(int count, int n, const int* __restrict__ ids,
                       const int* __restrict__ slot_of, double* __restrict__ a,
                       double* __restrict__ vals, int set, unsigned int* err)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int id = ids[k];
    if (id < 0 || id >= n) {
        atomicOr(err, (unsigned)MPS_ERR_ARG);
        return;
    }
    const int s = slot_of[id];
    if (set) a[s] = vals[k];
    else vals[k] = a[s];
}

__global__ void k_iota(int n, int* a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

__global__ void k_fill_i(int n, int v, int* a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

__global__ void k_density(int n, const int* __restrict__ ptype, double rho1, double rho2,
                          double* __restrict__ rho)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rho[i] = (ptype[i] == 2) ? rho2 : rho1;
}

int collect_errors(mps_ctx* c)
{
    VMPS_CUDA(c, cudaMemcpyAsync(c->h_err, c->d_err, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                 c->stream));
    VMPS_CUDA(c, cudaMemsetAsync(c->d_err, 0, sizeof(unsigned int), c->stream));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->host_err |= *c->h_err;
    return (int)(*c->h_err);
}

int device_max(mps_ctx* c, double* out)
{
    unsigned long long h = 0;
    VMPS_CUDA(c, cudaMemcpyAsync(&h, c->d_max, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    double d;
    memcpy(&d, &h, sizeof(d));
    *out = d;
    return MPS_OK;
}

#define TRY(x)                     \
    do {                           \
        int _r = (x);              \
        if (_r != MPS_OK) return _r; \
    } while (0)

int allocate(mps_ctx* c)
{
    const size_t P = (size_t)c->pitch;
    double** dfields[] = {&c->x, &c->y, &c->z, &c->u, &c->v, &c->w, &c->p, &c->pnew,
                          &c->phat, &c->un, &c->vn, &c->wn, &c->rho, &c->nd, &c->pold, &c->xs, &c->ys,
                          &c->zs, &c->us, &c->vs, &c->ws, &c->nds, &c->C, &c->meu, &c->neut,
                          &c->t1, &c->t2, &c->t3, &c->source, &c->diag, &c->cg_r, &c->cg_z,
                          &c->cg_p, &c->cg_s, &c->xc, &c->yc, &c->zc, &c->uc, &c->vc, &c->wc,
                          &c->pres_x, &c->pres_y, &c->pres_z};
    for (auto f : dfields) TRY(dalloc(c, f, P));
    int** ifields[] = {&c->ptype, &c->oid, &c->scene, &c->own, &c->sysmask, &c->stage_ids,
                       &c->slot_of,
                       &c->bcon, &c->cell_l, &c->cell_s, &c->bpos_l,
                       &c->bpos_s, &c->bslot_l, &c->boid_l, &c->bslot_s, &c->boid_s, &c->src,
                       &c->inv, &c->perm_s, &c->perm_s_tmp, &c->len_l, &c->len_s, &c->mlen,
                       &c->moff};
    for (auto f : ifields) TRY(dalloc(c, f, P));
    TRY(dalloc(c, &c->S6, 6 * P));
    TRY(dalloc(c, &c->bx_l, P));
    TRY(dalloc(c, &c->bx_s, P));
    TRY(dalloc(c, &c->key_s, P));
    TRY(dalloc(c, &c->stage_in, P));
    TRY(dalloc(c, &c->stage_io, 7 * (size_t)P));
    TRY(dalloc(c, &c->P4, P));
    TRY(dalloc(c, &c->P4s, P));
    TRY(dalloc(c, &c->P4c, P));
    TRY(dalloc(c, &c->U4, P));
    TRY(dalloc(c, &c->PP4, P));
    TRY(dalloc(c, &c->P4f, P));
    if (c->cfg.precision >= 1) TRY(dalloc(c, &c->U4f, P));
    if (c->cfg.precision == 2) {
        TRY(dalloc(c, &c->P4sf, P));
        TRY(dalloc(c, &c->PH32, P));
    }
    TRY(dalloc(c, &c->PH, P));
    TRY(dalloc(c, &c->cnt_l, (size_t)c->gl.tnc + 2));
    TRY(dalloc(c, &c->cst_l, (size_t)c->gl.tnc + 2));
    TRY(dalloc(c, &c->cnt_s, (size_t)c->gs.tnc + 2));
    TRY(dalloc(c, &c->cst_s, (size_t)c->gs.tnc + 2));
    size_t tiles = (size_t)std::max(std::max(c->gl.tnc, c->gs.tnc), c->n) / 8192 + 4;
    TRY(dalloc(c, &c->scan_tmp, tiles));
    // row-major lists and matrix: row i at i * cap
    TRY(dalloc(c, &c->nbr_l, (size_t)c->cap_l * P));
    TRY(dalloc(c, &c->nbr_s, (size_t)c->cap_s * P));
    TRY(dalloc(c, &c->mrow, P));
    TRY(dalloc(c, &c->mcol, (size_t)c->cap_l * P));
    TRY(dalloc(c, &c->mval, (size_t)c->cap_l * P));
    if (c->cfg.precision >= 1) {
        TRY(dalloc(c, &c->mcv32, (size_t)c->cap_l * P));
        float** ffields[] = {&c->ir_d, &c->ir_r, &c->ir_z, &c->ir_p, &c->ir_s};
        for (auto f : ffields) TRY(dalloc(c, f, P));
    }
    int sms = 0;
    VMPS_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    // CG partials: 5 arrays of one value per block, at most 8 blocks per SM
    c->cg_part_cap = (size_t)5 * 8 * sms;
    TRY(dalloc(c, &c->cg_part, c->cg_part_cap));
    TRY(dalloc(c, &c->cg_scal, 32));
    TRY(dalloc(c, &c->cg_flag, 4));
    TRY(dalloc(c, &c->cg_bar, 4));
    TRY(dalloc(c, &c->d_err, 1));
    TRY(dalloc(c, &c->len_max, 2));
    TRY(dalloc(c, &c->d_max, 1));
    TRY(halloc(c, &c->cg_flag_host, 4));
    TRY(halloc(c, &c->red_host, 32));
    TRY(halloc(c, &c->h_err, 1));
    // alternates of the persistent fields for the reorder (same order as
    // persistent_set in mps_neighbors.cu: 15 doubles then 6 ints)
    c->alts.clear();
    for (int k = 0; k < 15; k++) {
        double* q;
        TRY(dalloc(c, &q, P));
        c->alts.push_back(q);
    }
    for (int k = 0; k < 6; k++) {
        int* q;
        TRY(dalloc(c, &q, P));
        c->alts.push_back(q);
    }
    return MPS_OK;
}

double* field_d(mps_ctx* c, const std::string& f)
{
    struct { const char* n; double* p; } t[] = {
        {"x", c->x}, {"y", c->y}, {"z", c->z}, {"u", c->u}, {"v", c->v}, {"w", c->w},
        {"p", c->p}, {"pnew", c->pnew}, {"phat", c->phat}, {"un", c->un}, {"vn", c->vn},
        {"wn", c->wn}, {"xs", c->xs}, {"ys", c->ys}, {"zs", c->zs}, {"us", c->us},
        {"vs", c->vs}, {"ws", c->ws}, {"n", c->nd}, {"nstar", c->nds}, {"C", c->C},
        {"meu", c->meu}, {"neut", c->neut}, {"t1", c->t1}, {"t2", c->t2}, {"t3", c->t3},
        {"rho", c->rho}, {"source", c->source}, {"diag", c->diag}, {"pold", c->pold},
        {"cg_p", c->cg_p}};
    for (auto& e : t)
        if (f == e.n) return e.p;
    return nullptr;
}

}  // namespace

void vmps_drop_graphs(mps_ctx* c) { drop_graphs(c); }

std::vector<void*>& vmps_reorder_alts(mps_ctx* ctx) { return ctx->alts; }

// mps_step_io's deferred fields (bits 3..6 of state_defer: u, v, w, p; p also
// sets pnew) from the staging area into the current cell order, after the
// copies on the I/O stream have ended; then the packed velocities.  Inside a
// step graph the wait is an external event node: each replay waits for the
// copies recorded before its launch.
int vmps_state_apply(mps_ctx* c)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    VMPS_CUDA(c, cudaStreamIsCapturing(c->stream, &cs));
    VMPS_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_state,
                                     cs == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0));
    double* dst[7] = {c->x, c->y, c->z, c->u, c->v, c->w, c->p};
    StateIO io{};
    for (int k = 3; k < 7; k++)
        if (c->state_defer >> k & 1) io.f[k] = dst[k];
    io.pnew = (c->state_defer >> 6 & 1) ? c->pnew : nullptr;
    k_state_in<<<grid_blocks(c->n), kBlock, 0, c->stream>>>(c->n, c->pitch, c->oid, io,
                                                            c->stage_io);
    vmps_count_launch(1);
    return vmps_pack_u(c);
}

// ------------------------------------------------------------------ C-ABI

extern "C" {

int mps_create(const mps_config* cfg, int device, mps_ctx** out)
{
    if (!cfg || !out) return MPS_ERR_ARG;
    *out = nullptr;
    std::string why;
    int r = validate(*cfg, why);
    if (r != MPS_OK) {
        fprintf(stderr, "voxarmps: %s\n", why.c_str());
        return r;
    }
    mps_ctx* c = new mps_ctx();
    c->cfg = *cfg;
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        fprintf(stderr, "voxarmps: %s\n", cudaGetErrorString(e));
        delete c;
        return MPS_ERR_CUDA;
    }
    *out = c;
    return MPS_OK;
}

int mps_destroy(mps_ctx* c)
{
    if (!c) return MPS_OK;
    free_all(c);  // joins a snapshot write in flight
    vmps_gnn_free(c);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : c->ev_spmv) cudaEventDestroy(e);
    if (c->snap_ev) cudaEventDestroy(c->snap_ev);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->stream_io) cudaStreamDestroy(c->stream_io);
    if (c->ev_io) cudaEventDestroy(c->ev_io);
    if (c->ev_state) cudaEventDestroy(c->ev_state);
    for (auto e : c->ev_out)
        if (e) cudaEventDestroy(e);
    delete c;
    return MPS_OK;
}

int mps_upload(mps_ctx* c, int n, const double* x, const double* y, const double* z,
               const int* ptype, const double* u, const double* v, const double* w,
               const double* p)
{
    if (!c || n <= 0 || !x || !y || !ptype || (c->cfg.dim == 3 && !z)) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    free_all(c);
    vmps_gnn_reset(c);
    mps_config& f = c->cfg;
    c->n = n;
    c->nscenes = 1;
    c->pitch = (n + 31) / 32 * 32;
    c->gp = c->wp = c->fp = c->fp2 = 0;
    c->p4s_bcon = false;
    for (int i = 0; i < n; i++) {
        if (ptype[i] < 0) c->gp++;
        else if (ptype[i] == 0) c->wp++;
        else c->fp++;
        if (ptype[i] == 2) c->fp2++;
    }
    if (!(f.xmin < f.xmax)) {
        // grown bounding box and PMAX of main.cu:612-715, 548
        double mn[3] = {99999999, 99999999, 99999999}, mx[3] = {-99999999, -99999999, -99999999};
        for (int i = 0; i < n; i++) {
            double q[3] = {x[i], y[i], f.dim == 3 ? z[i] : 0.0};
            for (int a = 0; a < f.dim; a++) {
                if (q[a] < mn[a]) mn[a] = q[a];
                if (q[a] > mx[a]) mx[a] = q[a];
            }
        }
        f.xmin = mn[0] - f.l0; f.xmax = mx[0] + f.l0;
        f.ymin = mn[1] - f.l0; f.ymax = mx[1] + f.l0;
        if (f.dim == 3) { f.zmin = mn[2] - f.l0; f.zmax = mx[2] + f.l0; }
        else { f.zmin = 99999999; f.zmax = -99999999; }
        f.pmax = (double)n * 4.50;
    }
    if (!make_grid(f, f.re_l, &c->gl) || !make_grid(f, f.re_s, &c->gs)) {
        c->msg = "cell grid too large (over 2^30 cells) or box not finite";
        return MPS_ERR_ARG;
    }
    // FP32 screening bound: coordinates stored relative to the box minimum
    // carry an absolute error e <= extent * 2^-24 each, a difference of two
    // at most 2e + |dx| 2^-24; the squared distance of a pair near the cutoff
    // c is off by at most sum(2|dx| de + de^2) + 3 c^2 2^-23 (the sum of
    // squares is formed with fused multiply-adds, at most three roundings).
    // The bound used is four times that, with c the larger cutoff.
    {
        double ext = std::max(f.xmax - f.xmin, f.ymax - f.ymin);
        if (f.dim == 3) ext = std::max(ext, f.zmax - f.zmin);
        double cmax = std::max(f.re_l, f.re_s) + (f.dim == 3 ? f.delta : 0.0);
        double u = std::ldexp(1.0, -24);
        double de = 2 * ext * u + cmax * u;
        c->screen_abs = 4.0 * (3 * (2 * cmax * de + de * de) + 3 * cmax * cmax * 2 * u);
    }
    bool strict = f.dim == 2;
    c->cut_l = sqrt_cut(strict ? f.re_l : f.re_l + f.delta, strict);
    c->cut_s = sqrt_cut(strict ? f.re_s : f.re_s + f.delta, strict);
    c->cap_l = f.list_cap_l > 0 ? (f.list_cap_l + 7) / 8 * 8 : auto_cap(f, f.re_l);
    c->cap_s = f.list_cap_s > 0 ? (f.list_cap_s + 7) / 8 * 8 : auto_cap(f, f.re_s);
    c->lambda_l = 0.0;  // main.cu:491-494 at the Laplacian radius
    double re = f.re_l;
    if (f.ktype == 1) c->lambda_l = 0.22143 * (re * re);
    if (f.ktype == 2) c->lambda_l = 0.16832 * (re * re);
    if (f.ktype == 5) c->lambda_l = 0.250 * (re * re);
    if (f.ktype == 6) c->lambda_l = 0.14288 * (re * re);
    TRY(allocate(c));
    cudaStream_t st = c->stream;
    auto up = [&](double* d, const double* h) -> cudaError_t {
        if (!h) return cudaMemsetAsync(d, 0, sizeof(double) * n, st);
        return cudaMemcpyAsync(d, h, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    };
    VMPS_CUDA(c, up(c->x, x));
    VMPS_CUDA(c, up(c->y, y));
    VMPS_CUDA(c, up(c->z, f.dim == 3 ? z : nullptr));
    VMPS_CUDA(c, up(c->u, u));
    VMPS_CUDA(c, up(c->v, v));
    VMPS_CUDA(c, up(c->w, f.dim == 3 ? w : nullptr));
    VMPS_CUDA(c, up(c->p, p));
    VMPS_CUDA(c, cudaMemcpyAsync(c->ptype, ptype, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    k_iota<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid);
    k_fill_i<<<grid_blocks(n), kBlock, 0, st>>>(n, 1, c->own);
    k_density<<<grid_blocks(n), kBlock, 0, st>>>(n, c->ptype, f.rho1, f.rho2, c->rho);
    vmps_count_launch(3);
    VMPS_CUDA(c, cudaStreamSynchronize(st));
    c->initialized = false;
    c->steps = 0;
    c->host_err = 0;
    return MPS_OK;
}

int mps_set_scenes(mps_ctx* c, int nscenes, const int* scene, const double* boxes,
                   const double* pmax)
{
    // particles must still be in caller order: after mps_upload, before mps_init
    if (!c || c->n == 0 || c->initialized || nscenes < 1 || !scene || !boxes || !pmax)
        return MPS_ERR_ARG;
    for (int i = 0; i < c->n; i++)
        if (scene[i] < 0 || scene[i] >= nscenes) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    drop_graphs(c);
    c->nscenes = nscenes;
    TRY(dalloc(c, &c->sbox, (size_t)6 * nscenes));
    TRY(dalloc(c, &c->spmax, (size_t)nscenes));
    TRY(dalloc(c, &c->sfirst, (size_t)nscenes));
    TRY(dalloc(c, &c->slast, (size_t)nscenes));
    TRY(dalloc(c, &c->sbb, (size_t)nscenes));
    TRY(dalloc(c, &c->srr, (size_t)nscenes));
    TRY(dalloc(c, &c->sok, (size_t)nscenes));
    cudaStream_t st = c->stream;
    VMPS_CUDA(c, cudaMemcpyAsync(c->sbox, boxes, sizeof(double) * 6 * nscenes,
                                 cudaMemcpyHostToDevice, st));
    VMPS_CUDA(c, cudaMemcpyAsync(c->spmax, pmax, sizeof(double) * nscenes, cudaMemcpyHostToDevice,
                                 st));
    // scene of slot i: the upload left particles in caller order (oid = i)
    VMPS_CUDA(c, cudaMemcpyAsync(c->scene, scene, sizeof(int) * c->n, cudaMemcpyHostToDevice, st));
    VMPS_CUDA(c, cudaStreamSynchronize(st));
    return MPS_OK;
}

int mps_load_grd(mps_ctx* c, const char* path)
{
    if (!c || !path) return MPS_ERR_ARG;
    std::ifstream in(path);
    if (!in.is_open()) {
        c->msg = std::string("cannot open ") + path;
        return MPS_ERR_IO;
    }
    int n = 0;
    in >> n;
    if (n <= 0) return MPS_ERR_IO;
    bool three = c->cfg.dim == 3;
    std::vector<double> x(n), y(n), z(n), u(n), v(n), w(n), p(n);
    std::vector<int> pt(n);
    for (int i = 0; i < n; i++) {  // main.cu:629-661
        in >> x[i] >> y[i];
        if (three) in >> z[i];
        in >> pt[i] >> u[i] >> v[i];
        if (three) in >> w[i];
        in >> p[i];
        if (!in) {
            c->msg = "truncated .grd file";
            return MPS_ERR_IO;
        }
    }
    return mps_upload(c, n, x.data(), y.data(), z.data(), pt.data(), u.data(), v.data(), w.data(),
                      p.data());
}

int mps_neighbors(mps_ctx* c)
{
    if (!c || c->n == 0) return MPS_ERR_ARG;
    return vmps_neighbors(c);
}

int mps_init(mps_ctx* c)
{
    if (!c || c->n == 0) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    drop_graphs(c);
    TRY(vmps_neighbors(c));
    VMPS_CUDA(c, cudaMemsetAsync(c->d_max, 0, sizeof(unsigned long long), c->stream));
    TRY(vmps_pnd(c, 0, 1, 1, c->nd, true));
    TRY(device_max(c, &c->n0_s));
    if (c->cfg.re_s == c->cfg.re_l) {
        c->n0_l = c->n0_s;
    } else {
        VMPS_CUDA(c, cudaMemsetAsync(c->d_max, 0, sizeof(unsigned long long), c->stream));
        TRY(vmps_pnd(c, 0, 1, 0, c->nds, true));
        TRY(device_max(c, &c->n0_l));
    }
    VMPS_CUDA(c, cudaMemcpyAsync(c->pnew, c->p, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                                 c->stream));
    VMPS_CUDA(c, cudaMemcpyAsync(c->pold, c->p, sizeof(double) * c->n, cudaMemcpyDeviceToDevice,
                                 c->stream));
    c->initialized = true;
    int e = collect_errors(c);
    return e;
}

#define NEED_INIT(c)                                   \
    do {                                               \
        if (!(c) || !(c)->initialized) return MPS_ERR_ARG; \
    } while (0)

int mps_pnd(mps_ctx* c) { NEED_INIT(c); return vmps_pnd(c, 0, 1, 1, c->nd); }
int mps_sps(mps_ctx* c) { NEED_INIT(c); return vmps_sps(c); }
int mps_vfraction(mps_ctx* c) { NEED_INIT(c); return vmps_vfraction(c); }
int mps_viscosity(mps_ctx* c) { NEED_INIT(c); return vmps_viscosity(c); }
int mps_predict(mps_ctx* c) { NEED_INIT(c); return vmps_predict(c); }
int mps_pnd_star(mps_ctx* c) { NEED_INIT(c); return vmps_pnd(c, 1, 0, 1, c->nds); }
int mps_bcon(mps_ctx* c) { NEED_INIT(c); return vmps_bcon(c); }
int mps_phat(mps_ctx* c) { NEED_INIT(c); return vmps_phat(c); }
int mps_pressure_gradient(mps_ctx* c) { NEED_INIT(c); return vmps_pressgrad(c); }
int mps_integrate(mps_ctx* c) { NEED_INIT(c); return vmps_integrate(c); }
int mps_collision(mps_ctx* c) { NEED_INIT(c); return vmps_collision(c); }
int mps_commit(mps_ctx* c)
{
    NEED_INIT(c);
    TRY(vmps_commit(c));
    return collect_errors(c);
}

int mps_pressure(mps_ctx* c, int* iters, double* relres)
{
    NEED_INIT(c);
    if (c->cfg.method == 3) {
        TRY(vmps_pressure_wc(c));
        c->cg_iters = 0;
        c->cg_relres = 0;
    } else {
        TRY(vmps_ppe(c));
        VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
        TRY(vmps_ppe_finish(c));
    }
    if (iters) *iters = c->cg_iters;
    if (relres) *relres = c->cg_relres;
    return MPS_OK;
}

// The stage sequence of one loop iteration (main.cu:1036-1337), enqueued
// on the context's stream without host synchronisation in graph mode.
static int enqueue_step(mps_ctx* c)
{
    const mps_config& f = c->cfg;
    auto mark = [&](int k) -> int {
        if (c->profile) VMPS_CUDA(c, cudaEventRecord(c->ev[k], c->stream));
        return MPS_OK;
    };
    TRY(mark(0));
    {
        NvtxRange r("mps.neighbors");
        if (f.method != 3 && !f.ppe_at_predicted) TRY(vmps_pnd(c, 0, 1, 1, c->nd));
        TRY(vmps_neighbors(c));
    }
    TRY(mark(1));
    {
        NvtxRange r("mps.explicit");
        if (f.turb) TRY(vmps_sps(c));
        TRY(vmps_vfraction(c));
        TRY(vmps_viscosity(c));
        TRY(vmps_predict(c));
        TRY(vmps_pnd(c, 1, 0, 1, c->nds));
        if (f.method != 3) TRY(vmps_bcon(c));
    }
    TRY(mark(2));
    {
        NvtxRange r("mps.pressure");
        if (f.method != 3) TRY(vmps_ppe(c));
        else TRY(vmps_pressure_wc(c));
    }
    TRY(mark(3));
    {
        NvtxRange r("mps.post");
        TRY(vmps_phat(c));
        TRY(vmps_pressgrad(c));
        TRY(vmps_integrate(c));
        TRY(vmps_collision(c));
        TRY(vmps_commit(c));
    }
    TRY(mark(4));
    return MPS_OK;
}

// One step as a CUDA graph.  The reorder alternates the persistent fields
// between two buffer sets, so a graph is captured per buffer parity and
// replayed afterwards; the CG loop inside is a conditional while node.
static int graph_step(mps_ctx* c)
{
    const int par = (int)(c->swaps & 1) + (c->state_defer ? 2 : 0);
    if (c->gexec[par] && c->gdefer[par] != c->state_defer) {  // another set of fields
        cudaGraphExecDestroy(c->gexec[par]);
        c->gexec[par] = nullptr;
    }
    if (!c->stream2) VMPS_CUDA(c, cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking));
    TRY(vmps_gnn_prepare(c));  // no allocation inside the capture
    if (!c->gexec[par]) {
        NvtxRange nr("mps.graph_capture");
        const long long l0 = g_launches.load();
        VMPS_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
        int r = enqueue_step(c);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (r != MPS_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            if (r != MPS_OK) return r;
            VMPS_CUDA(c, e);
        }
        cudaError_t ie = cudaGraphInstantiate(&c->gexec[par], g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) c->gexec[par] = nullptr;
        VMPS_CUDA(c, ie);
        c->gkernels[par] = (long)(g_launches.load() - l0);
        c->gdefer[par] = c->state_defer;
    } else {
        // the host side of a replay: the reorder's buffer exchange
        vmps_reorder_swap(c);
        vmps_count_launch((int)c->gkernels[par]);
        c->ppe_pending = c->cfg.method != 3;
    }
    VMPS_CUDA(c, cudaGraphLaunch(c->gexec[par], c->stream));
    return MPS_OK;
}

int mps_step(mps_ctx* c)
{
    NEED_INIT(c);
    NvtxRange nr("mps.step");
    VMPS_CUDA(c, cudaSetDevice(c->device));
    unsigned int before = c->host_err;
    const bool graph = c->use_graph && !c->profile;
    if (graph) TRY(graph_step(c));
    else TRY(enqueue_step(c));
    c->steps++;
    int e = collect_errors(c);
    TRY(vmps_ppe_finish(c));
    if (graph && c->cfg.method != 3)
        vmps_count_launch((c->cg_iters + c->cg_outer) * c->cg_loop_kernels);
    if (c->profile) {
        for (int k = 0; k < 4; k++) {
            float ms = 0;
            VMPS_CUDA(c, cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]));
            c->ms_stage[k] = ms;
        }
        float ms = 0;
        VMPS_CUDA(c, cudaEventElapsedTime(&ms, c->ev[0], c->ev[4]));
        c->ms_stage[4] = ms;
    }
    return e | (int)(c->host_err & ~before);
}

static int small_base(const mps_ctx*) { return SmallG<2>::G; }

int mps_get_tuning(mps_ctx* c, mps_tuning* out)
{
    if (!c || !out) return MPS_ERR_ARG;
    out->small_lanes = small_base(c) * (c->tune_small_wide ? 2 : 1);
    out->cg_blocks_per_sm = c->tune_cg_bps;
    return MPS_OK;
}

int mps_set_tuning(mps_ctx* c, const mps_tuning* in)
{
    if (!c || !in) return MPS_ERR_ARG;
    const int b = small_base(c);
    if ((in->small_lanes != b && in->small_lanes != 2 * b) || in->cg_blocks_per_sm < 0 ||
        in->cg_blocks_per_sm > 8) {
        c->msg = "tuning: small_lanes must be the base width or twice it, cg_blocks_per_sm 0..8";
        return MPS_ERR_ARG;
    }
    const int wide = in->small_lanes == 2 * b ? 1 : 0;
    if (wide != c->tune_small_wide || in->cg_blocks_per_sm != c->tune_cg_bps) drop_graphs(c);
    c->tune_small_wide = wide;
    c->tune_cg_bps = in->cg_blocks_per_sm;
    return MPS_OK;
}

static int autotune_search(mps_ctx* c, int steps, mps_tuning& t)
{
    auto median = [](std::vector<double> v) {
        std::sort(v.begin(), v.end());
        return v[v.size() / 2];
    };
    auto measure = [&](double* ppe_per_iter, double* rest) -> int {
        std::vector<double> a, b;
        for (int k = 0; k < steps; k++) {
            int r = mps_step(c);
            if (r & (MPS_ERR_ARG | MPS_ERR_CUDA)) return r;
            const double its = std::max(1, c->cg_iters + c->cg_outer);
            a.push_back(c->ms_stage[2] / its);
            b.push_back(c->ms_stage[4] - c->ms_stage[2]);
        }
        *ppe_per_iter = median(a);
        *rest = median(b);
        return MPS_OK;
    };
    if (c->cfg.method != 3) {
        int best = t.cg_blocks_per_sm;
        double best_ms = 1e300;
        for (int bps : {1, 2, 4, 8}) {
            t.cg_blocks_per_sm = bps;
            TRY(mps_set_tuning(c, &t));
            double ppe = 0, rest = 0;
            TRY(measure(&ppe, &rest));
            if (ppe < best_ms) {
                best_ms = ppe;
                best = bps;
            }
        }
        t.cg_blocks_per_sm = best;
        TRY(mps_set_tuning(c, &t));
    }
    const int b = small_base(c);
    int best = t.small_lanes;
    double best_ms = 1e300;
    for (int lanes : {b, 2 * b}) {
        t.small_lanes = lanes;
        TRY(mps_set_tuning(c, &t));
        double ppe = 0, rest = 0;
        TRY(measure(&ppe, &rest));
        if (rest < best_ms) {
            best_ms = rest;
            best = lanes;
        }
    }
    t.small_lanes = best;
    return mps_set_tuning(c, &t);
}

// Coordinate search: the CG grid by the PPE time per CG iteration, then the
// PND-radius lane width by the time of the rest of the step.  Each candidate
// runs `steps` profiled steps; the median step decides.  On failure the
// previous tuning and profiling state are restored.
int mps_autotune(mps_ctx* c, int steps, mps_tuning* chosen)
{
    NEED_INIT(c);
    if (steps < 1) return MPS_ERR_ARG;
    const bool prof = c->profile;
    mps_tuning before, t;
    TRY(mps_get_tuning(c, &before));
    t = before;
    TRY(mps_set_profile(c, 1));
    const int r = autotune_search(c, steps, t);
    if (r != MPS_OK) mps_set_tuning(c, &before);
    const int rp = mps_set_profile(c, prof ? 1 : 0);
    if (r != MPS_OK) return r;
    TRY(rp);
    if (chosen) *chosen = t;
    return MPS_OK;
}

int mps_set_graph(mps_ctx* c, int on)
{
    if (!c) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    if (!on) drop_graphs(c);
    c->use_graph = on != 0;
    return MPS_OK;
}

int mps_run(mps_ctx* c, int steps)
{
    int acc = 0;
    for (int s = 0; s < steps; s++) {
        int r = mps_step(c);
        if (r & (MPS_ERR_ARG | MPS_ERR_CUDA)) return r;
        acc |= r;
    }
    return acc;
}

int mps_set_state(mps_ctx* c, const double* x, const double* y, const double* z,
                  const double* u, const double* v, const double* w, const double* p)
{
    NEED_INIT(c);
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n;
    const long P = c->pitch;
    const double* src[7] = {x, y, z, u, v, w, p};
    double* dst[7] = {c->x, c->y, c->z, c->u, c->v, c->w, c->p};
    StateIO io{};
    for (int k = 0; k < 7; k++) {
        if (!src[k] || (c->cfg.dim == 2 && (k == 2 || k == 5))) continue;
        VMPS_CUDA(c, cudaMemcpyAsync(c->stage_io + k * P, src[k], sizeof(double) * n,
                                     cudaMemcpyHostToDevice, c->stream));
        io.f[k] = dst[k];
    }
    io.pnew = c->pnew;
    k_state_in<<<grid_blocks(n), kBlock, 0, c->stream>>>(n, P, c->oid, io, c->stage_io);
    vmps_count_launch(1);
    TRY(vmps_pack(c));
    VMPS_CUDA(c, cudaGetLastError());
    return MPS_OK;
}

int mps_set_field(mps_ctx* c, const char* field, const double* in)
{
    NEED_INIT(c);
    if (!field || !in) return MPS_ERR_ARG;
    static const char* const kSettable[] = {"x", "y", "z",  "u",  "v",  "w",    "p",
                                            "pnew", "un", "vn", "wn", "phat", "pold"};
    std::string f(field);
    bool ok = false;
    for (const char* s : kSettable) ok = ok || f == s;
    if (!ok || (c->cfg.dim == 2 && (f == "z" || f == "w" || f == "wn"))) {
        c->msg = "mps_set_field: field " + f + " cannot be set";
        return MPS_ERR_ARG;
    }
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n;
    VMPS_CUDA(c, cudaMemcpyAsync(c->stage_in, in, sizeof(double) * n, cudaMemcpyHostToDevice,
                                 c->stream));
    k_permute_in<<<grid_blocks(n), kBlock, 0, c->stream>>>(n, c->oid, c->stage_in, field_d(c, f),
                                                           nullptr);
    vmps_count_launch(1);
    // the packed copies the stages gather from follow the fields they pack
    if (f == "x" || f == "y" || f == "z" || f == "u" || f == "v" || f == "w") TRY(vmps_pack(c));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

// ---- slab decomposition support --------------------------------------------

int mps_set_owned(mps_ctx* c, const int* owned)
{
    NEED_INIT(c);
    if (!owned) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n;
    VMPS_CUDA(c, cudaMemcpyAsync(c->stage_ids, owned, sizeof(int) * n, cudaMemcpyHostToDevice,
                                 c->stream));
    k_permute_in_i<<<grid_blocks(n), kBlock, 0, c->stream>>>(n, c->oid, c->stage_ids, c->own);
    vmps_count_launch(1);
    drop_graphs(c);
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

int mps_set_n0(mps_ctx* c, double n0_s, double n0_l)
{
    NEED_INIT(c);
    if (!(n0_s > 0) || !(n0_l > 0)) return MPS_ERR_ARG;
    c->n0_s = n0_s;
    c->n0_l = n0_l;
    drop_graphs(c);
    return MPS_OK;
}

// rows by caller-order index: out[k] = field[particle ids[k]] (get) or
// field[particle ids[k]] = in[k] (set)
static int rows_io(mps_ctx* c, const char* field, int count, const int* ids, double* out,
                   const double* in)
{
    NEED_INIT(c);
    double* a = field ? field_d(c, field) : nullptr;
    if (!a || count < 0 || count > c->n || (count > 0 && !ids) || (count > 0 && !out && !in)) {
        c->msg = std::string("rows: bad field or arguments");
        return MPS_ERR_ARG;
    }
    if (count == 0) return MPS_OK;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const int n = c->n;
    k_slot_of<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, c->slot_of);
    VMPS_CUDA(c, cudaMemcpyAsync(c->stage_ids, ids, sizeof(int) * count, cudaMemcpyHostToDevice,
                                 st));
    if (in)
        VMPS_CUDA(c, cudaMemcpyAsync(c->stage_in, in, sizeof(double) * count,
                                     cudaMemcpyHostToDevice, st));
    k_rows<<<grid_blocks(count), kBlock, 0, st>>>(count, n, c->stage_ids, c->slot_of, a,
                                                  c->stage_in, in ? 1 : 0, c->d_err);
    vmps_count_launch(2);
    if (out)
        VMPS_CUDA(c, cudaMemcpyAsync(out, c->stage_in, sizeof(double) * count,
                                     cudaMemcpyDeviceToHost, st));
    VMPS_CUDA(c, cudaStreamSynchronize(st));
    if (in && (!strcmp(field, "x") || !strcmp(field, "y") || !strcmp(field, "z") ||
               !strcmp(field, "u") || !strcmp(field, "v") || !strcmp(field, "w")))
        TRY(vmps_pack(c));
    return MPS_OK;
}

int mps_get_rows(mps_ctx* c, const char* field, int count, const int* ids, double* out)
{
    if (!out && count > 0) return MPS_ERR_ARG;
    return rows_io(c, field, count, ids, out, nullptr);
}

int mps_set_rows(mps_ctx* c, const char* field, int count, const int* ids, const double* in)
{
    if (!in && count > 0) return MPS_ERR_ARG;
    return rows_io(c, field, count, ids, nullptr, in);
}

int mps_get_state(mps_ctx* c, double* x, double* y, double* z, double* u, double* v, double* w,
                  double* p)
{
    NEED_INIT(c);
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n;
    const long P = c->pitch;
    double* out[7] = {x, y, z, u, v, w, p};
    double* from[7] = {c->x, c->y, c->z, c->u, c->v, c->w, c->p};
    if (!c->stream_io) VMPS_CUDA(c, cudaStreamCreateWithFlags(&c->stream_io, cudaStreamNonBlocking));
    // one field at a time: its permutation into caller order on the
    // context's stream, its copy to the host on the I/O stream, so that each
    // copy overlaps the next field's permutation
    for (int k = 0; k < 7; k++) {
        if (!out[k] || (c->cfg.dim == 2 && (k == 2 || k == 5))) continue;
        if (!c->ev_out[k]) VMPS_CUDA(c, cudaEventCreateWithFlags(&c->ev_out[k], cudaEventDisableTiming));
        StateIO io{};
        io.f[k] = from[k];
        k_state_out<<<grid_blocks(n), kBlock, 0, c->stream>>>(n, P, c->oid, io, c->stage_io);
        vmps_count_launch(1);
        VMPS_CUDA(c, cudaEventRecord(c->ev_out[k], c->stream));
        VMPS_CUDA(c, cudaStreamWaitEvent(c->stream_io, c->ev_out[k], 0));
        VMPS_CUDA(c, cudaMemcpyAsync(out[k], c->stage_io + k * P, sizeof(double) * n,
                                     cudaMemcpyDeviceToHost, c->stream_io));
    }
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream_io));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

int mps_step_io(mps_ctx* c, const double* const* in, double* const* out)
{
    NEED_INIT(c);
    if (!in || !out) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    if (!c->stream_io) VMPS_CUDA(c, cudaStreamCreateWithFlags(&c->stream_io, cudaStreamNonBlocking));
    if (!c->ev_io) VMPS_CUDA(c, cudaEventCreateWithFlags(&c->ev_io, cudaEventDisableTiming));
    if (!c->ev_state) VMPS_CUDA(c, cudaEventCreateWithFlags(&c->ev_state, cudaEventDisableTiming));
    const int n = c->n;
    const long P = c->pitch;
    const mps_config& f = c->cfg;
    // the staging area is free once the context's stream has passed its
    // earlier work
    VMPS_CUDA(c, cudaEventRecord(c->ev_io, c->stream));
    VMPS_CUDA(c, cudaStreamWaitEvent(c->stream_io, c->ev_io, 0));
    double* dst[7] = {c->x, c->y, c->z, c->u, c->v, c->w, c->p};
    StateIO pos{};
    int defer = 0;
    for (int k = 0; k < 7; k++) {
        if (!in[k] || (f.dim == 2 && (k == 2 || k == 5))) continue;
        // positions first on the context's stream (the neighbour search
        // starts from them), the rest beside it
        VMPS_CUDA(c, cudaMemcpyAsync(c->stage_io + k * P, in[k], sizeof(double) * n,
                                     cudaMemcpyHostToDevice, k < 3 ? c->stream : c->stream_io));
        if (k < 3) pos.f[k] = dst[k];
        else defer |= 1 << k;
    }
    k_state_in<<<grid_blocks(n), kBlock, 0, c->stream>>>(n, P, c->oid, pos, c->stage_io);
    vmps_count_launch(1);
    // PNUM before the neighbour search reads the packed positions
    if (f.method != 3 && !f.ppe_at_predicted) TRY(vmps_pack(c));
    if (defer) VMPS_CUDA(c, cudaEventRecord(c->ev_state, c->stream_io));
    c->state_defer = defer;
    const int r = mps_step(c);
    c->state_defer = 0;
    if (r & (MPS_ERR_ARG | MPS_ERR_CUDA)) {
        // the step stopped before taking the fields: leave no copy pending
        cudaStreamSynchronize(c->stream_io);
        return r;
    }
    return r | mps_get_state(c, out[0], out[1], out[2], out[3], out[4], out[5], out[6]);
}

int mps_set_profile(mps_ctx* c, int on)
{
    if (!c) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    if (on && !c->ev[0])
        for (auto& e : c->ev) VMPS_CUDA(c, cudaEventCreate(&e));
    c->profile = on != 0;
    c->spmv_ms = c->lists_ms = 0;
    c->spmv_launches = c->lists_launches = 0;
    return MPS_OK;
}

int mps_download(mps_ctx* c, const char* field, void* out, long* count)
{
    if (!c || !field || c->n == 0) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n;
    std::string f(field);
    cudaStream_t st = c->stream;
    if (count) *count = n;
    if (!out) return MPS_OK;
    // S6 column-0 area doubles as the staging buffer (6 * pitch doubles)
    double* stage = c->S6;
    int* istage = (int*)c->S6;
    if (double* a = field_d(c, f)) {
        k_unpermute_d<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, a, stage);
        VMPS_CUDA(c, cudaMemcpyAsync(out, stage, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    } else if (f == "ptype" || f == "bcon" || f == "cell_l" || f == "cell_s" || f == "scene") {
        const int* a = f == "ptype" ? c->ptype : f == "bcon" ? c->bcon : f == "cell_l" ? c->cell_l
                       : f == "cell_s" ? c->cell_s : c->scene;
        k_unpermute_i<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, a, istage);
        VMPS_CUDA(c, cudaMemcpyAsync(out, istage, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    } else if (f == "perm_l" || f == "perm_s") {
        // the context orders a cell's particles by (x, id); NEIGHBOR's
        // permutations by id alone (functions.cu:2820): ids and cells in
        // the grid's order, then each cell's run sorted
        const bool pnd = f == "perm_s";
        std::vector<int> cl(n);
        int* o = (int*)out;
        k_perm_ids<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, pnd ? c->perm_s : nullptr, istage);
        k_perm_ids<<<grid_blocks(n), kBlock, 0, st>>>(n, pnd ? c->cell_s : c->cell_l,
                                                       pnd ? c->perm_s : nullptr, istage + n);
        vmps_count_launch(2);
        VMPS_CUDA(c, cudaMemcpyAsync(o, istage, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
        VMPS_CUDA(c, cudaMemcpyAsync(cl.data(), istage + n, sizeof(int) * n,
                                     cudaMemcpyDeviceToHost, st));
        VMPS_CUDA(c, cudaStreamSynchronize(st));
        for (int a = 0; a < n;) {
            int b = a + 1;
            while (b < n && cl[b] == cl[a]) b++;
            std::sort(o + a, o + b);
            a = b;
        }
        return MPS_OK;
    } else {
        c->msg = "unknown field " + f;
        return MPS_ERR_ARG;
    }
    vmps_count_launch(1);
    VMPS_CUDA(c, cudaStreamSynchronize(st));
    return MPS_OK;
}

int mps_download_lists(mps_ctx* c, int which, int* off, int* nbr, long* total)
{
    if (!c || c->n == 0 || (which != 0 && which != 1)) return MPS_ERR_ARG;
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n, P = c->pitch;
    int cap = which == 0 ? c->cap_s : c->cap_l;  // rows i*cap .. i*cap+len-1
    const int* dl = which == 0 ? c->len_s : c->len_l;
    const int* dn = which == 0 ? c->nbr_s : c->nbr_l;
    std::vector<int> len(n), oid(n), cell(n), ent((size_t)cap * P);
    VMPS_CUDA(c, cudaMemcpy(len.data(), dl, sizeof(int) * n, cudaMemcpyDeviceToHost));
    VMPS_CUDA(c, cudaMemcpy(oid.data(), c->oid, sizeof(int) * n, cudaMemcpyDeviceToHost));
    VMPS_CUDA(c, cudaMemcpy(cell.data(), which == 0 ? c->cell_s : c->cell_l, sizeof(int) * n,
                            cudaMemcpyDeviceToHost));
    VMPS_CUDA(c, cudaMemcpy(ent.data(), dn, sizeof(int) * ent.size(), cudaMemcpyDeviceToHost));
    const Grid& g = which == 0 ? c->gs : c->gl;
    std::vector<int> slot_of(n);
    for (int i = 0; i < n; i++) slot_of[oid[i]] = i;
    long tot = 0;
    for (int q = 0; q < n; q++) tot += len[slot_of[q]];
    if (total) *total = tot;
    if (!off) return MPS_OK;
    // rows are stored in scan order; the reference's order is x offset
    // outermost, then y, then z, ascending id inside a cell (functions.cu:2858)
    auto coords = [&](int C, int& a, int& b, int& k) {
        C -= 1;
        a = C % g.ncx;
        b = (C / g.ncx) % g.ncy;
        k = C / (g.ncx * g.ncy);
    };
    std::vector<std::pair<long, int>> keyed;
    long acc = 0;
    for (int q = 0; q < n; q++) {
        int i = slot_of[q];
        off[q] = (int)acc;
        if (nbr) {
            int ai, bi, ki;
            coords(cell[i], ai, bi, ki);
            keyed.clear();
            for (int k = 0; k < len[i]; k++) {
                int j = ent[(size_t)i * cap + k];
                int aj, bj, kj;
                coords(cell[j], aj, bj, kj);
                long rank = (long)(aj - ai + 1) * 9 + (bj - bi + 1) * 3 + (kj - ki + 1);
                keyed.emplace_back(rank * (long)n + oid[j], oid[j]);
            }
            std::sort(keyed.begin(), keyed.end());
            for (int k = 0; k < len[i]; k++) nbr[acc + k] = keyed[k].second;
        }
        acc += len[i];
    }
    off[n] = (int)acc;
    return MPS_OK;
}

int mps_get_scalar(mps_ctx* c, const char* name, double* out)
{
    if (!c || !name || !out) return MPS_ERR_ARG;
    std::string s(name);
    if (s == "n0_s") *out = c->n0_s;
    else if (s == "n0_l") *out = c->n0_l;
    else if (s == "lambda_l") *out = c->lambda_l;
    else if (s == "cg_iters") *out = c->cg_iters;
    else if (s == "cg_relres") *out = c->cg_relres;
    else if (s == "cg_r0") *out = c->cg_r0;
    else if (s == "cg_outer") *out = c->cg_outer;
    else if (s == "n") *out = c->n;
    else if (s == "steps") *out = (double)c->steps;
    else if (s == "cap_s") *out = c->cap_s;
    else if (s == "cap_l") *out = c->cap_l;
    else if (s == "launches") *out = (double)g_launches.load();
    else if (s == "ms_neighbors") *out = c->ms_stage[0];
    else if (s == "ms_explicit") *out = c->ms_stage[1];
    else if (s == "ms_ppe") *out = c->ms_stage[2];
    else if (s == "ms_post") *out = c->ms_stage[3];
    else if (s == "ms_step") *out = c->ms_stage[4];
    else if (s == "spmv_ms") *out = c->spmv_ms;
    else if (s == "spmv_launches") *out = (double)c->spmv_launches;
    else if (s == "lists_ms") *out = c->lists_ms;
    else if (s == "lists_launches") *out = (double)c->lists_launches;
    else if (s == "pmax") *out = c->cfg.pmax;
    else if (s == "xmin") *out = c->cfg.xmin;
    else if (s == "xmax") *out = c->cfg.xmax;
    else if (s == "ymin") *out = c->cfg.ymin;
    else if (s == "ymax") *out = c->cfg.ymax;
    else if (s == "zmin") *out = c->cfg.zmin;
    else if (s == "zmax") *out = c->cfg.zmax;
    else if (s == "len_max_l" || s == "len_max_s") {
        int h[2] = {0, 0};
        VMPS_CUDA(c, cudaMemcpy(h, c->len_max, sizeof(h), cudaMemcpyDeviceToHost));
        *out = s == "len_max_l" ? h[0] : h[1];
    } else if (s == "nnz_l" || s == "nnz_s" || s == "nnz_a") {
        std::vector<int> len(c->n);
        const int* d = s == "nnz_l" ? c->len_l : s == "nnz_s" ? c->len_s : c->mlen;
        VMPS_CUDA(c, cudaMemcpy(len.data(), d, sizeof(int) * c->n, cudaMemcpyDeviceToHost));
        double t = 0;
        for (int v : len) t += v;
        *out = t;
    } else {
        return MPS_ERR_ARG;
    }
    return MPS_OK;
}

int mps_get_error(mps_ctx* c)
{
    if (!c) return MPS_ERR_ARG;
    int e = (int)c->host_err;
    c->host_err = 0;
    return e;
}

const char* mps_last_message(mps_ctx* c) { return c ? c->msg.c_str() : ""; }

void* mps_stream(mps_ctx* c) { return c ? (void*)c->stream : nullptr; }


// ------------------------------------------------------------------ checkpoints
//
// Binary checkpoint (replaces the reference's disabled VTU read-back,
// inOut.cpp:25-102 / main.cu:393).  Little-endian layout:
//   char magic[8] = "VXMPSCK1"; uint32 version = 1; uint32 config_bytes;
//   mps_config (config_bytes); int32 n, nscenes; int64 steps;
//   double n0_s, n0_l;
//   15 double fields, n each, in the caller's particle order:
//     x y z u v w p pnew phat un vn wn rho n pold
//   int32 ptype[n], scene[n]; then, when nscenes > 1, double boxes[6 ns],
//   pmax[ns];  uint64 FNV-1a hash of every preceding byte.
// Resuming replays the counting sort by (cell, x, id) at the next step,
// which does not depend on the slot order before it, so a resumed run
// continues bit for bit.

static const char kCkMagic[8] = {'V', 'X', 'M', 'P', 'S', 'C', 'K', '1'};
static const char* kCkFields[15] = {"x",  "y",  "z",  "u",   "v", "w", "p", "pnew",
                                    "phat", "un", "vn", "wn", "rho", "n", "pold"};

struct Fnv {
    unsigned long long h = 14695981039346656037ull;  // FNV-1a 64-bit offset basis
    void add(const void* p, size_t k)
    {
        const unsigned char* b = (const unsigned char*)p;
        for (size_t i = 0; i < k; i++) h = (h ^ b[i]) * 1099511628211ull;
    }
};

int mps_save_checkpoint(mps_ctx* c, const char* path)
{
    NvtxRange nr("mps.save_checkpoint");
    NEED_INIT(c);
    if (!path) return MPS_ERR_ARG;
    const int n = c->n, ns = c->nscenes;
    std::vector<double> buf((size_t)n);
    std::vector<int> ib((size_t)n);
    FILE* fp = fopen(path, "wb");
    if (!fp) {
        c->msg = std::string("cannot write ") + path;
        return MPS_ERR_IO;
    }
    Fnv h;
    bool ok = true;
    auto put = [&](const void* p, size_t k) {
        h.add(p, k);
        ok = ok && fwrite(p, 1, k, fp) == k;
    };
    const unsigned version = 1, cb = (unsigned)sizeof(mps_config);
    const long long steps = c->steps;
    put(kCkMagic, 8);
    put(&version, 4);
    put(&cb, 4);
    put(&c->cfg, cb);
    put(&n, 4);
    put(&ns, 4);
    put(&steps, 8);
    put(&c->n0_s, 8);
    put(&c->n0_l, 8);
    int r = MPS_OK;
    for (const char* f : kCkFields) {
        r = mps_download(c, f, buf.data(), nullptr);
        if (r != MPS_OK) break;
        put(buf.data(), sizeof(double) * n);
    }
    for (const char* f : {"ptype", "scene"}) {
        if (r != MPS_OK) break;
        r = mps_download(c, f, ib.data(), nullptr);
        if (r == MPS_OK) put(ib.data(), sizeof(int) * n);
    }
    if (r == MPS_OK && ns > 1) {
        std::vector<double> boxes((size_t)6 * ns), pm((size_t)ns);
        cudaError_t e = cudaMemcpy(boxes.data(), c->sbox, sizeof(double) * 6 * ns,
                                   cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(pm.data(), c->spmax, sizeof(double) * ns, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) r = vmps_check(c, e, "checkpoint scenes");
        put(boxes.data(), sizeof(double) * 6 * ns);
        put(pm.data(), sizeof(double) * ns);
    }
    const unsigned long long sum = h.h;
    ok = ok && fwrite(&sum, 1, 8, fp) == 8;
    ok = (fclose(fp) == 0) && ok;
    if (r != MPS_OK) return r;
    return ok ? MPS_OK : MPS_ERR_IO;
}

int mps_load_checkpoint(mps_ctx* c, const char* path)
{
    NvtxRange nr("mps.load_checkpoint");
    if (!c || !path) return MPS_ERR_ARG;
    FILE* fp = fopen(path, "rb");
    if (!fp) {
        c->msg = std::string("cannot open ") + path;
        return MPS_ERR_IO;
    }
    std::vector<unsigned char> all;
    {
        unsigned char tmp[1 << 16];
        size_t k;
        while ((k = fread(tmp, 1, sizeof(tmp), fp)) > 0) all.insert(all.end(), tmp, tmp + k);
        fclose(fp);
    }
    size_t pos = 0;
    auto get = [&](void* p, size_t k) {
        if (pos + k > all.size()) return false;
        memcpy(p, all.data() + pos, k);
        pos += k;
        return true;
    };
    auto bad = [&](const char* why) {
        c->msg = std::string("checkpoint ") + path + ": " + why;
        return MPS_ERR_IO;
    };
    if (all.size() < 8 + 8) return bad("truncated");
    Fnv h;
    h.add(all.data(), all.size() - 8);
    unsigned long long sum = 0;
    memcpy(&sum, all.data() + all.size() - 8, 8);
    if (sum != h.h) return bad("checksum mismatch");
    char magic[8];
    unsigned version = 0, cb = 0;
    if (!get(magic, 8) || memcmp(magic, kCkMagic, 8) != 0) return bad("not a checkpoint");
    if (!get(&version, 4) || version != 1) return bad("unsupported version");
    if (!get(&cb, 4) || cb != sizeof(mps_config)) return bad("configuration layout differs");
    mps_config cfg;
    int n = 0, ns = 0;
    long long steps = 0;
    double n0s = 0, n0l = 0;
    if (!get(&cfg, cb) || !get(&n, 4) || !get(&ns, 4) || !get(&steps, 8) || !get(&n0s, 8) ||
        !get(&n0l, 8) || n <= 0 || ns < 1)
        return bad("bad header");
    std::string why;
    if (validate(cfg, why) != MPS_OK) return bad(why.c_str());
    std::vector<std::vector<double>> d(15, std::vector<double>((size_t)n));
    for (auto& a : d)
        if (!get(a.data(), sizeof(double) * n)) return bad("truncated fields");
    std::vector<int> pt((size_t)n), sc((size_t)n);
    if (!get(pt.data(), sizeof(int) * n) || !get(sc.data(), sizeof(int) * n))
        return bad("truncated fields");
    std::vector<double> boxes, pm;
    if (ns > 1) {
        boxes.resize((size_t)6 * ns);
        pm.resize((size_t)ns);
        if (!get(boxes.data(), sizeof(double) * 6 * ns) || !get(pm.data(), sizeof(double) * ns))
            return bad("truncated scenes");
    }
    // the payload must end exactly where the checksum starts
    if (pos != all.size() - 8) return bad("trailing bytes before the checksum");
    c->cfg = cfg;
    TRY(mps_upload(c, n, d[0].data(), d[1].data(), d[2].data(), pt.data(), d[3].data(),
                   d[4].data(), d[5].data(), d[6].data()));
    if (ns > 1) TRY(mps_set_scenes(c, ns, sc.data(), boxes.data(), pm.data()));
    // right after the upload the slots are in caller order
    double* dst[15] = {c->x,  c->y,  c->z,  c->u,  c->v,   c->w,  c->p,   c->pnew,
                       c->phat, c->un, c->vn, c->wn, c->rho, c->nd, c->pold};
    for (int k = 0; k < 15; k++)
        VMPS_CUDA(c, cudaMemcpyAsync(dst[k], d[k].data(), sizeof(double) * n,
                                     cudaMemcpyHostToDevice, c->stream));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    c->n0_s = n0s;
    c->n0_l = n0l;
    c->steps = steps;
    c->initialized = true;
    TRY(vmps_pack(c));
    VMPS_CUDA(c, cudaStreamSynchronize(c->stream));
    return MPS_OK;
}

// ------------------------------------------------------------------ binary VTU
//
// VTK XML UnstructuredGrid with raw appended data (UInt64 block headers):
// positions and velocities as 3-component Float32 (all three components in
// 3D), pressure Float32, partType Int32, vertex cells.  The snapshot is
// taken on the stream (unpermute kernels + device-to-host copies into
// pinned buffers) and written by a host thread while the device steps on;
// mps_wait_io joins it.

static int write_vtu_binary(const char* path, int n, const double* s, bool three, bool fluid_only)
{
    const double *x = s, *y = s + n, *z = s + 2 * (size_t)n, *u = s + 3 * (size_t)n,
                 *v = s + 4 * (size_t)n, *w = s + 5 * (size_t)n, *p = s + 6 * (size_t)n;
    const int* pt = (const int*)(s + 7 * (size_t)n);
    std::vector<int> keep;
    keep.reserve(n);
    for (int i = 0; i < n; i++)
        if (!fluid_only || pt[i] > 0) keep.push_back(i);
    const unsigned long long m = keep.size();
    std::vector<float> pos(3 * m), vel(3 * m), pr(m);
    std::vector<int> ty(m), conn(m), offs(m);
    std::vector<unsigned char> cell(m, 1);
    for (size_t k = 0; k < m; k++) {
        const int i = keep[k];
        pos[3 * k] = (float)x[i];
        pos[3 * k + 1] = (float)y[i];
        pos[3 * k + 2] = three ? (float)z[i] : 0.f;
        vel[3 * k] = (float)u[i];
        vel[3 * k + 1] = (float)v[i];
        vel[3 * k + 2] = three ? (float)w[i] : 0.f;
        pr[k] = (float)p[i];
        ty[k] = pt[i];
        conn[k] = (int)k;
        offs[k] = (int)k + 1;
    }
    struct Block { const void* p; unsigned long long bytes; };
    Block blocks[7] = {{pos.data(), 12 * m}, {vel.data(), 12 * m}, {pr.data(), 4 * m},
                       {ty.data(), 4 * m},   {conn.data(), 4 * m}, {offs.data(), 4 * m},
                       {cell.data(), m}};
    unsigned long long off[7], o = 0;
    for (int b = 0; b < 7; b++) {
        off[b] = o;
        o += 8 + blocks[b].bytes;
    }
    FILE* fp = fopen(path, "wb");
    if (!fp) return MPS_ERR_IO;
    fprintf(fp, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" "
                "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n <UnstructuredGrid>\n"
                "  <Piece NumberOfPoints=\"%llu\" NumberOfCells=\"%llu\">\n   <Points>\n"
                "    <DataArray type=\"Float32\" NumberOfComponents=\"3\" Name=\"Position\" "
                "format=\"appended\" offset=\"%llu\"/>\n   </Points>\n   <PointData>\n"
                "    <DataArray type=\"Float32\" NumberOfComponents=\"3\" Name=\"Velocity\" "
                "format=\"appended\" offset=\"%llu\"/>\n"
                "    <DataArray type=\"Float32\" Name=\"Pressure\" format=\"appended\" offset=\"%llu\"/>\n"
                "    <DataArray type=\"Int32\" Name=\"partType\" format=\"appended\" offset=\"%llu\"/>\n"
                "   </PointData>\n   <Cells>\n"
                "    <DataArray type=\"Int32\" Name=\"connectivity\" format=\"appended\" offset=\"%llu\"/>\n"
                "    <DataArray type=\"Int32\" Name=\"offsets\" format=\"appended\" offset=\"%llu\"/>\n"
                "    <DataArray type=\"UInt8\" Name=\"types\" format=\"appended\" offset=\"%llu\"/>\n"
                "   </Cells>\n  </Piece>\n </UnstructuredGrid>\n <AppendedData encoding=\"raw\">\n_",
            m, m, off[0], off[1], off[2], off[3], off[4], off[5], off[6]);
    bool ok = true;
    for (auto& b : blocks) {
        ok = ok && fwrite(&b.bytes, 8, 1, fp) == 1;
        if (b.bytes) ok = ok && fwrite(b.p, 1, b.bytes, fp) == b.bytes;
    }
    fprintf(fp, "\n </AppendedData>\n</VTKFile>\n");
    ok = ok && !ferror(fp);
    ok = (fclose(fp) == 0) && ok;
    return ok ? MPS_OK : MPS_ERR_IO;
}

int mps_snapshot_vtu(mps_ctx* c, const char* path, int fluid_only)
{
    NvtxRange nr("mps.snapshot_vtu");
    NEED_INIT(c);
    if (!path) return MPS_ERR_ARG;
    snap_join(c);  // one snapshot in flight: its buffers are reused
    VMPS_CUDA(c, cudaSetDevice(c->device));
    const int n = c->n;
    if (c->snap_n < n) {
        // 7 double fields + ptype (ints in the space of one double field)
        double* q = nullptr;
        VMPS_CUDA(c, cudaMallocHost(&q, sizeof(double) * 8 * (size_t)n));
        c->pinned.push_back(q);
        c->snap = q;
        c->snap_n = n;
    }
    if (!c->snap_ev) VMPS_CUDA(c, cudaEventCreateWithFlags(&c->snap_ev, cudaEventDisableTiming));
    cudaStream_t st = c->stream;
    const char* names[7] = {"x", "y", "z", "u", "v", "w", "p"};
    double* stage = c->S6;  // 6 * pitch doubles of scratch
    for (int k = 0; k < 7; k++) {
        double* a = field_d(c, names[k]);
        double* slot = stage + (size_t)(k % 6) * c->pitch;
        k_unpermute_d<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, a, slot);
        VMPS_CUDA(c, cudaMemcpyAsync(c->snap + (size_t)k * n, slot, sizeof(double) * n,
                                     cudaMemcpyDeviceToHost, st));
    }
    int* istage = (int*)(stage + (size_t)1 * c->pitch);  // after the 7th copy was queued
    k_unpermute_i<<<grid_blocks(n), kBlock, 0, st>>>(n, c->oid, c->ptype, istage);
    VMPS_CUDA(c, cudaMemcpyAsync(c->snap + (size_t)7 * n, istage, sizeof(int) * n,
                                 cudaMemcpyDeviceToHost, st));
    vmps_count_launch(8);
    VMPS_CUDA(c, cudaEventRecord(c->snap_ev, st));
    const std::string file(path);
    const bool three = c->cfg.dim == 3, fo = fluid_only != 0;
    double* data = c->snap;
    cudaEvent_t ev = c->snap_ev;
    c->snap_status = MPS_OK;
    c->snap_thread = std::thread([c, file, n, data, three, fo, ev]() {
        if (cudaEventSynchronize(ev) != cudaSuccess) {
            c->snap_status = MPS_ERR_CUDA;
            return;
        }
        c->snap_status = write_vtu_binary(file.c_str(), n, data, three, fo);
    });
    return MPS_OK;
}

int mps_wait_io(mps_ctx* c)
{
    if (!c) return MPS_ERR_ARG;
    snap_join(c);
    return c->snap_status;
}

int mps_write_vtu(mps_ctx* c, const char* path, int fluid_only)
{
    if (!c || !path || c->n == 0) return MPS_ERR_ARG;
    const int n = c->n;
    std::vector<double> x(n), y(n), z(n), u(n), v(n), w(n), p(n);
    std::vector<int> pt(n);
    const char* names[] = {"x", "y", "z", "u", "v", "w", "p"};
    double* dst[] = {x.data(), y.data(), z.data(), u.data(), v.data(), w.data(), p.data()};
    for (int k = 0; k < 7; k++) TRY(mps_download(c, names[k], dst[k], nullptr));
    TRY(mps_download(c, "ptype", pt.data(), nullptr));
    std::vector<int> keep;
    for (int i = 0; i < n; i++)
        if (!fluid_only || pt[i] > 0) keep.push_back(i);
    FILE* fp = fopen(path, "w");
    if (!fp) return MPS_ERR_IO;
    // inOut.cpp:122-216 layout; all three components are written in 3D (the
    // reference drops z and w there, inOut.cpp:135,154)
    int m = (int)keep.size();
    bool three = c->cfg.dim == 3;
    fprintf(fp, "<?xml version='1.0' encoding='UTF-8'?>\n");
    fprintf(fp, "<VTKFile xmlns='VTK' byte_order='LittleEndian' version='0.1' type='UnstructuredGrid'>\n");
    fprintf(fp, " <UnstructuredGrid>\n  <Piece NumberOfCells='%d' NumberOfPoints='%d'>\n", m, m);
    fprintf(fp, "   <Points>\n    <DataArray NumberOfComponents='3' type='Float32' Name='Position' format='ascii'>\n");
    for (int i : keep) fprintf(fp, "%.9g %.9g %.9g ", x[i], y[i], three ? z[i] : 0.0);
    fprintf(fp, "\n    </DataArray>\n   </Points>\n   <PointData>\n");
    fprintf(fp, "    <DataArray NumberOfComponents='3' type='Float32' Name='Velocity' format='ascii'>\n");
    for (int i : keep) fprintf(fp, "%.9g %.9g %.9g ", u[i], v[i], three ? w[i] : 0.0);
    fprintf(fp, "\n    </DataArray>\n    <DataArray NumberOfComponents='1' type='Float32' Name='Pressure' format='ascii'>\n");
    for (int i : keep) fprintf(fp, "%.9g ", p[i]);
    fprintf(fp, "\n    </DataArray>\n    <DataArray NumberOfComponents='1' type='Int32' Name='partType' format='ascii'>\n");
    for (int i : keep) fprintf(fp, "%d ", pt[i]);
    fprintf(fp, "\n    </DataArray>\n   </PointData>\n   <Cells>\n    <DataArray type='Int32' Name='connectivity' format='ascii'>\n");
    for (int b = 0; b < m; b++) fprintf(fp, "%d ", b);
    fprintf(fp, "\n    </DataArray>\n    <DataArray type='Int32' Name='offsets' format='ascii'>\n");
    for (int b = 1; b <= m; b++) fprintf(fp, "%d ", b);
    fprintf(fp, "\n    </DataArray>\n    <DataArray type='UInt8' Name='types' format='ascii'>\n");
    for (int b = 0; b < m; b++) fprintf(fp, "1 ");
    fprintf(fp, "\n    </DataArray>\n   </Cells>\n  </Piece>\n </UnstructuredGrid>\n</VTKFile>");
    int bad = ferror(fp);
    fclose(fp);
    return bad ? MPS_ERR_IO : MPS_OK;
}

}  // extern "C"
