// C ABI of the SIMP hot path (include/simp_gpu.h): context lifecycle, state
// transfer in the reference's Fortran layouts, and the per-step driver.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "ctx.h"

using namespace simp;

int simp_fail(simp_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int simp_cuda_check(simp_ctx *c, cudaError_t e, const char *what) {
    return simp_fail(c, SIMP_ERR_CUDA, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

namespace {

constexpr int kB = 256;
constexpr int kSnapRing = 3;
inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

__global__ void k_deinterleave(int n, const double *__restrict__ in, double *__restrict__ a,
                               double *__restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = in[2 * i];
    b[i] = in[2 * i + 1];
}

// out (original order) <- cell-order arrays
__global__ void k_to_orig2(int n, const int *__restrict__ id, const double *__restrict__ a,
                           const double *__restrict__ b, double *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = id[k];
    out[2 * o] = a[k];
    out[2 * o + 1] = b[k];
}

__global__ void k_to_orig1(int n, const int *__restrict__ id, const double *__restrict__ a,
                           double *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[id[k]] = a[k];
}

// Whole state to original order in one pass: stage = [x,y interleaved | vx,vy
// interleaved | mass | rho | hsml | A | h], 9 n doubles.
__global__ void k_pack_state(int n, const int *__restrict__ id, State s, double *__restrict__ stage) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t o = (size_t)id[k], N = (size_t)n;
    stage[2 * o] = s.x[k];
    stage[2 * o + 1] = s.y[k];
    stage[2 * N + 2 * o] = s.vx[k];
    stage[2 * N + 2 * o + 1] = s.vy[k];
    stage[4 * N + o] = s.m[k];
    stage[5 * N + o] = s.rho[k];
    stage[6 * N + o] = s.hs[k];
    stage[7 * N + o] = s.A[k];
    stage[8 * N + o] = s.h[k];
}

__global__ void k_init_ids(int n, int *id, const double *m, const double *rho, double *mor) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    id[k] = k;
    mor[k] = m[k] / rho[k];
}

__global__ void k_set_time(Scalars *sc, double t) { sc->t = t; }

Phys make_phys(const simp_params &p, double max_hsml) {
    Phys P{};
    P.skf = p.skf;
    P.scale_h = (p.skf == SIMP_SKF_CUBIC) ? 2 : 1;
    P.viscosity = p.viscosity;
    P.pressure_force = p.pressure_force;
    P.eos_alg = p.eos_alg;
    P.wind_force = p.wind_force;
    P.water_force = p.water_force;
    P.wind_kind = p.wind_kind;
    P.boundary_pressure = p.boundary_pressure;
    P.sle = p.sle;
    P.den_alg = p.den_alg;
    P.mass_from_area = p.mass_from_area;
    P.tse = p.tse;
    P.hsml_multiplicity = p.hsml_multiplicity;
    P.max_ind_int = p.max_ind_int;
    P.P_star = p.P_star;
    P.c_eos = p.c_eos;
    P.e = p.e;
    P.delta_min = p.delta_min;
    P.k_t = p.k_t;
    P.rho_ice = p.rho_ice;
    P.rho_air = p.rho_air;
    P.rho_water = p.rho_water;
    P.c_wind = p.c_wind;
    P.c_water = p.c_water;
    P.b_length = p.b_length;
    P.kappa_n = p.kappa_n;
    P.alpha = p.alpha;
    P.wind_u = p.wind_u;
    P.wind_v = p.wind_v;
    P.current_u = p.current_u;
    P.current_v = p.current_v;
    P.vortex_x = p.vortex_x;
    P.vortex_y = p.vortex_y;
    P.vortex_umax = p.vortex_umax;
    P.vortex_radius = p.vortex_radius;
    P.max_hsml = max_hsml;
    return P;
}

int check_params(simp_ctx *c, const simp_params &p) {
    auto bad = [&](const char *what) { return simp_fail(c, SIMP_ERR_BADARG, std::string("unsupported switch: ") + what); };
    if (p.int_algorithm != 2) return bad("int_algorithm (only 2, predictor-corrector, is on this path)");
    if (p.nnps_algorithm != 1 && p.nnps_algorithm != 2) return bad("nnps_algorithm (1 or 2)");
    if (p.sle != 0 && p.sle != 2) return bad("sle (0 or 2)");
    if (p.tse != 0 && p.tse != 2) return bad("tse (0 or 2)");
    if (p.rheology != 1) return bad("rheology (only 1, elliptical)");
    if (p.eos_alg != 1 && p.eos_alg != 3) return bad("eos_alg (1 or 3)");
    if (p.pa_sph != 1) return bad("pa_sph (only 1)");
    if (p.skf != SIMP_SKF_WENDLAND_C6 && p.skf != SIMP_SKF_CUBIC) return bad("skf (6 or 9)");
    if (p.den_alg != 3) return bad("den_alg (3 in the step; the summation density is simp_gpu_sum_density)");
    if (p.bfa != 1) return bad("bfa (only 1, Monaghan)");
    if (p.boundary_friction) return bad("boundary_friction");
    if (p.precision != SIMP_PREC_FP64) return bad("precision (this context type is FP64)");
    if (!(p.e > 0.0) || !(p.rho_ice > 0.0) || !(p.b_length > 0.0)) return bad("material constants");
    return SIMP_OK;
}

template <class T>
int dalloc(simp_ctx *c, T **p, size_t count) {
    if (count == 0) count = 1;
    if (cudaMalloc((void **)p, count * sizeof(T)) != cudaSuccess)
        return simp_fail(c, SIMP_ERR_NOMEM, "device allocation failed");
    return SIMP_OK;
}

#define TRY(expr)                       \
    do {                                \
        int _rc = (expr);               \
        if (_rc != SIMP_OK) return _rc; \
    } while (0)

void free_all(simp_ctx *c) {
    void *ptrs[] = {c->s0.x, c->s0.y, c->s0.vx, c->s0.vy, c->s0.m, c->s0.rho, c->s0.mor, c->s0.h,
                    c->s0.A, c->s0.hs, c->s1.x, c->s1.y, c->s1.vx, c->s1.vy, c->s1.rho, c->s1.mor,
                    c->s1.h, c->s1.A, c->mass1, c->xr, c->yr, c->xl, c->yl, c->cell, c->id, c->inv_id,
                    c->tau11, c->tau12, c->tau22, c->div, c->diag, c->rates, c->bx, c->by, c->bm,
                    c->bid, c->bcell, c->bcell_start, c->cell_start, c->cnt, c->perm, c->tmp,
                    c->itmp, c->scan_tmp, c->sc, c->pair_cnt, c->bpair_cnt, c->pair_buf_i,
                    c->pair_buf_j, c->pair_buf_r, c->pair_buf_h, c->nbr, c->nbr_count,
                    c->pair_j, c->pair_count,
                    c->s0.xf, c->s0.yf, c->s0.hsf, c->s1.xf, c->s1.yf};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c->sc_host) cudaFreeHost(c->sc_host);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    for (cudaEvent_t e : c->prof_ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
}

// Verlet-list skin: the parameter when given, else 10% of max(hsml).
double list_skin(const simp_ctx *c, double hmax) {
    return (c->prm.skin >= 0.0) ? c->prm.skin : 0.1 * hmax;
}

// Grid sizing from host-side extents.  Cell side = 1.15 (hsml + skin);
// the grid covers the particles and walls with a margin; the cell count is
// capped (a larger side only adds candidates, never drops pairs).
int size_grid(simp_ctx *c, double xmin, double xmax, double ymin, double ymax, double hmax) {
    // cell side: the Verlet-list reach (hsml + skin) plus 15% for motion
    // between sorts
    double cs = (hmax + list_skin(c, hmax)) * 1.15;
    if (!(cs > 0.0)) cs = 1.0;
    const double ext = std::max(xmax - xmin, ymax - ymin);
    const double margin = std::max(2.0 * cs, 0.02 * ext);
    const double x0 = xmin - margin, y0 = ymin - margin;
    const double w = xmax - xmin + 2.0 * margin, h = ymax - ymin + 2.0 * margin;
    const double cap = std::max(4.0 * (double)c->maxn, 65536.0);
    while (std::ceil(w / cs) * std::ceil(h / cs) > cap) cs *= 1.25;
    Grid &g = c->grid;
    c->grid_hmax = hmax;
    g.x0 = x0;
    g.y0 = y0;
    g.cs = cs;
    g.inv_cs = 1.0 / cs;
    g.ncx = std::max(1, (int)std::ceil(w / cs));
    g.ncy = std::max(1, (int)std::ceil(h / cs));
    const size_t ncells = (size_t)g.ncx * g.ncy;
    if (ncells + 1 > c->cell_cap) {
        if (c->cell_start) cudaFree(c->cell_start);
        if (c->cnt) cudaFree(c->cnt);
        if (c->bcell_start) cudaFree(c->bcell_start);
        if (c->scan_tmp) cudaFree(c->scan_tmp);
        c->cell_start = c->cnt = c->bcell_start = nullptr;
        c->scan_tmp = nullptr;
        const size_t capn = ncells + 1;
        TRY(dalloc(c, &c->cell_start, capn));
        TRY(dalloc(c, &c->cnt, capn));
        TRY(dalloc(c, &c->bcell_start, capn));
        const size_t sb = scan_tmp_bytes((int)std::max<size_t>(capn, (size_t)std::max(c->maxn, c->maxnb) + 1));
        if (cudaMalloc(&c->scan_tmp, sb) != cudaSuccess) return simp_fail(c, SIMP_ERR_NOMEM, "device allocation failed");
        c->scan_tmp_bytes = sb;
        c->cell_cap = capn;
    }
    g.cell_start = c->cell_start;
    return SIMP_OK;
}

// Walls never move: bin them on the host (stable by wall index).
int bin_walls(simp_ctx *c, int nb, const double *xb, const double *massb) {
    const Grid &g = c->grid;
    const size_t ncells = (size_t)g.ncx * g.ncy;
    std::vector<int> key(nb), order(nb);
    for (int b = 0; b < nb; ++b) {
        const int cx = clampi((int)std::floor((xb[2 * b] - g.x0) * g.inv_cs), 0, g.ncx - 1);
        const int cy = clampi((int)std::floor((xb[2 * b + 1] - g.y0) * g.inv_cs), 0, g.ncy - 1);
        key[b] = cy * g.ncx + cx;
    }
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    std::vector<double> hx(nb), hy(nb), hm(nb);
    std::vector<int> hid(nb), hcell(nb);
    std::vector<int> start(ncells + 1, 0);
    for (int k = 0; k < nb; ++k) {
        const int b = order[k];
        hx[k] = xb[2 * b];
        hy[k] = xb[2 * b + 1];
        hm[k] = massb[b];
        hid[k] = b;
        hcell[k] = key[b];
        start[key[b] + 1] += 1;
    }
    for (size_t k = 0; k < ncells; ++k) start[k + 1] += start[k];
    cudaStream_t s = c->stream;
    if (nb > 0) {
        SIMP_CUDA(c, cudaMemcpyAsync(c->bx, hx.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->by, hy.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->bm, hm.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->bid, hid.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->bcell, hcell.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    }
    SIMP_CUDA(c, cudaMemcpyAsync(c->bcell_start, start.data(), sizeof(int) * (ncells + 1),
                                 cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    return SIMP_OK;
}

int upload_interleaved(simp_ctx *c, const double *h2, double *a, double *b, int n, double *stage) {
    SIMP_CUDA(c, cudaMemcpyAsync(stage, h2, sizeof(double) * 2 * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    k_deinterleave<<<nblk(n, kB), kB, 0, c->stream>>>(n, stage, a, b);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    return SIMP_OK;
}

int download2(simp_ctx *c, const double *a, const double *b, double *h2) {
    double *stage = c->tmp;
    k_to_orig2<<<nblk(c->n, kB), kB, 0, c->stream>>>(c->n, c->id, a, b, stage);
    c->launches += 1;
    SIMP_CUDA(c, cudaMemcpyAsync(h2, stage, sizeof(double) * 2 * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    return SIMP_OK;
}

int download1(simp_ctx *c, const double *a, double *h1) {
    double *stage = c->tmp;
    k_to_orig1<<<nblk(c->n, kB), kB, 0, c->stream>>>(c->n, c->id, a, stage);
    c->launches += 1;
    SIMP_CUDA(c, cudaMemcpyAsync(h1, stage, sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    return SIMP_OK;
}

int read_scalars(simp_ctx *c) {
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc_host, c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    return SIMP_OK;
}

// One predictor-corrector step (time_integration.f90:263-390).
// One predictor-corrector step (time_integration.f90:263-390).  With
// profiling on, external event records between the kernels time each one.
void enqueue_step(simp_ctx *c, bool diag, bool prof) {
    auto mark = [&](int k) {
        if (prof) cudaEventRecordWithFlags(c->prof_ev[k], c->stream, cudaEventRecordExternal);
    };
    mark(0);
    launch_kinematic(c, c->s0, false);
    mark(1);
    launch_stress(c, c->s0, c->s0, EPI_PREDICT);
    mark(2);
    launch_kinematic(c, c->s1, diag);
    mark(3);
    launch_stress(c, c->s1, c->s0, EPI_CORRECT);
    mark(4);
    launch_step_finish(c);
    mark(5);
}

int ensure_graph(simp_ctx *c, bool diag) {
    const bool prof = c->profile;
    if (c->step_graph && c->graph_diag == diag && c->graph_profiled == prof) return SIMP_OK;
    if (c->step_graph) {
        cudaGraphExecDestroy(c->step_graph);
        c->step_graph = nullptr;
    }
    if (prof && !c->prof_ev[0])
        for (auto &e : c->prof_ev) SIMP_CUDA(c, cudaEventCreate(&e));
    cudaGraph_t g = nullptr;
    const long long before = c->launches;
    SIMP_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c, diag, prof);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->graph_kernels = c->launches - before;   // captured, not yet launched
    c->launches = before;
    if (e != cudaSuccess) return simp_cuda_check(c, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&c->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return simp_cuda_check(c, e, "cudaGraphInstantiate");
    c->graph_diag = diag;
    c->graph_profiled = prof;
    return SIMP_OK;
}

void invalidate_graph(simp_ctx *c) {
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
}

double disp_of(const Scalars &s) {
    double d2;
    std::memcpy(&d2, &s.dmax2_bits, sizeof(double));
    return std::sqrt(std::max(0.0, d2));
}

// Re-sort when the device-side stencil would grow past one cell ring.
bool wants_rebuild(const simp_ctx *c, const Scalars &s) {
    return (s.hmax + s.skin + 2.0 * disp_of(s)) * c->grid.inv_cs > 0.98;
}

// Resize the grid when hsml grew 5% past the bound the grid was sized for
// (sle = 2); until then the device-side stencil radius covers the growth.
bool wants_regrid(const simp_ctx *c, const Scalars &s) { return s.hmax > 1.05 * c->grid_hmax; }

int size_grid(simp_ctx *c, double xmin, double xmax, double ymin, double ymax, double hmax);
int bin_walls(simp_ctx *c, int nb, const double *xb, const double *massb);
int download2(simp_ctx *c, const double *a, const double *b, double *h2);

// New grid from the current extents and hsml bound, then a full re-sort.
int regrid(simp_ctx *c) {
    TRY(read_scalars(c));
    const double hmax = c->sc_host->hmax;
    std::vector<double> xy(2 * (size_t)c->n);
    TRY(download2(c, c->s0.x, c->s0.y, xy.data()));
    double xmin = xy[0], xmax = xy[0], ymin = xy[1], ymax = xy[1];
    for (int i = 0; i < c->n; ++i) {
        xmin = std::min(xmin, xy[2 * i]);
        xmax = std::max(xmax, xy[2 * i]);
        ymin = std::min(ymin, xy[2 * i + 1]);
        ymax = std::max(ymax, xy[2 * i + 1]);
    }
    for (int b = 0; b < c->nb; ++b) {
        xmin = std::min(xmin, c->host_xb[2 * b]);
        xmax = std::max(xmax, c->host_xb[2 * b]);
        ymin = std::min(ymin, c->host_xb[2 * b + 1]);
        ymax = std::max(ymax, c->host_xb[2 * b + 1]);
    }
    invalidate_graph(c);
    TRY(size_grid(c, xmin, xmax, ymin, ymax, hmax));
    TRY(bin_walls(c, c->nb, c->host_xb.data(), c->host_massb.data()));
    return rebuild(c);
}

int check_after(simp_ctx *c) {
    const Scalars &s = *c->sc_host;
    if (s.flags & FLAG_NONFINITE)
        return simp_fail(c, SIMP_ERR_NONFINITE, "non-finite particle state after a step");
    if (s.maxip > c->prm.max_ind_int)
        return simp_fail(c, SIMP_ERR_IND_INT,
                         "Particle are too close to each other, this can lead to memory issue. Please "
                         "allow a higher maximum number of interaction for a single particle. "
                         "(nnps.f90:660-668)");
    return SIMP_OK;
}

}  // namespace

extern "C" {

const char *simp_gpu_version(void) { return "simp_b200 0.1 (sm_100a)"; }

void simp_params_reference_default(simp_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->int_algorithm = 2;
    p->nnps_algorithm = 2;
    p->sle = 2;
    p->tse = 2;
    p->rheology = 1;
    p->eos_alg = 3;
    p->pa_sph = 1;
    p->skf = SIMP_SKF_WENDLAND_C6;
    p->den_alg = 3;
    p->bfa = 1;
    p->viscosity = 1;
    p->pressure_force = 1;
    p->wind_force = 1;
    p->water_force = 1;
    p->boundary_pressure = 1;
    p->boundary_friction = 0;
    p->mass_from_area = 1;
    p->max_ind_int = 200;
    p->hsml_multiplicity = 3;
    p->wind_kind = SIMP_WIND_UNIFORM;
    p->precision = SIMP_PREC_FP64;
    p->P_star = 2.75e4;
    p->c_eos = 20.0;
    p->e = 2.0;
    p->delta_min = 2.0e-9;
    p->k_t = 0.0;
    p->rho_ice = 900.0;
    p->rho_air = (double)1.3f;
    p->rho_water = 1026.0;
    p->c_wind = 1.2e-3;
    p->c_water = 5.5e-3;
    p->b_length = 8000.0;
    p->kappa_n = 5.4e12;
    p->kappa_t = 5.0e-8;
    p->alpha = (double)(1.0f / 6.0f);
    p->wind_u = 0.0;
    p->wind_v = (double)(-5.3f);
    p->current_u = 0.0;
    p->current_v = 0.0;
    p->dt = 0.0;
    p->max_hsml = 0.0;
    p->skin = -1.0;
}

int32_t simp_gpu_create(const simp_params *params, int32_t maxn, int32_t maxnb, simp_ctx **out) {
    if (!out) return SIMP_ERR_BADARG;
    *out = nullptr;
    if (!params || maxn < 1 || maxnb < 0) return SIMP_ERR_BADARG;
    simp_ctx *c = new simp_ctx();
    c->prm = *params;
    int rc = check_params(c, c->prm);
    if (rc != SIMP_OK) {
        *out = c;  // caller can read last_error, then destroy
        return rc;
    }
    c->maxn = maxn;
    c->maxnb = std::max(maxnb, 1);
    cudaGetDevice(&c->device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        *out = c;
        return simp_fail(c, SIMP_ERR_CUDA, "cudaStreamCreate failed (no usable CUDA device?)");
    }
    const size_t M = (size_t)maxn, MB = (size_t)c->maxnb, MX = std::max(M, MB);
    double **d1[] = {&c->s0.x, &c->s0.y, &c->s0.vx, &c->s0.vy, &c->s0.m, &c->s0.rho, &c->s0.mor, &c->s0.h,
                     &c->s0.A, &c->s0.hs, &c->s1.x, &c->s1.y, &c->s1.vx, &c->s1.vy, &c->s1.rho,
                     &c->s1.mor, &c->s1.h, &c->s1.A, &c->xr, &c->yr, &c->xl, &c->yl,
                     &c->tau11, &c->tau12, &c->tau22,
                     &c->div};
    for (double **p : d1) {
        rc = dalloc(c, p, M);
        if (rc) { *out = c; return rc; }
    }
    if (c->prm.mass_from_area && c->prm.sle != 2) {
        rc = dalloc(c, &c->mass1, M);
        if (rc) { *out = c; return rc; }
        c->s1.m = c->mass1;
    } else {
        c->s1.m = c->s0.m;
    }
    c->s1.hs = c->s0.hs;
    float **f1[] = {&c->s0.xf, &c->s0.yf, &c->s0.hsf, &c->s1.xf, &c->s1.yf};
    for (float **p : f1) {
        rc = dalloc(c, p, M);
        if (rc) { *out = c; return rc; }
    }
    c->s1.hsf = c->s0.hsf;
    if ((rc = dalloc(c, &c->nbr, (size_t)kMaxNbr * M)) || (rc = dalloc(c, &c->nbr_count, M)) ||
        (rc = dalloc(c, &c->pair_j, (size_t)kMaxPairs * M)) || (rc = dalloc(c, &c->pair_count, M)) ||
        (rc = dalloc(c, &c->diag, 9 * M)) || (rc = dalloc(c, &c->rates, 4 * M)) ||
        (rc = dalloc(c, &c->cell, M)) || (rc = dalloc(c, &c->id, M)) || (rc = dalloc(c, &c->inv_id, M)) ||
        (rc = dalloc(c, &c->perm, M)) || (rc = dalloc(c, &c->tmp, 12 * MX)) ||
        (rc = dalloc(c, &c->itmp, 3 * MX)) || (rc = dalloc(c, &c->bx, MB)) || (rc = dalloc(c, &c->by, MB)) ||
        (rc = dalloc(c, &c->bm, MB)) || (rc = dalloc(c, &c->bid, MB)) || (rc = dalloc(c, &c->bcell, MB)) ||
        (rc = dalloc(c, &c->sc, 1)) || (rc = dalloc(c, &c->pair_cnt, M + 1)) ||
        (rc = dalloc(c, &c->bpair_cnt, MB + 1))) {
        *out = c;
        return rc;
    }
    if (cudaMallocHost((void **)&c->sc_host, sizeof(Scalars) * (1 + kSnapRing)) != cudaSuccess) {
        *out = c;
        return simp_fail(c, SIMP_ERR_NOMEM, "pinned host allocation failed");
    }
    std::memset(c->sc_host, 0, sizeof(Scalars) * (1 + kSnapRing));
    *out = c;
    return SIMP_OK;
}

int32_t simp_gpu_destroy(simp_ctx *c) {
    if (!c) return SIMP_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    delete c;
    return SIMP_OK;
}

int32_t simp_gpu_set_state(simp_ctx *c, int32_t ntotal, const double *x, const double *vx,
                           const double *mass, const double *rho, const double *hsml,
                           const double *A, const double *h, int32_t ntotalb, const double *xb,
                           const double *massb, double dt, double current_time) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->stream) return simp_fail(c, SIMP_ERR_STATE, "context was not created successfully");
    if (ntotal < 1 || ntotalb < 0 || !x || !vx || !mass || !rho || !hsml || !A || !h ||
        (ntotalb > 0 && (!xb || !massb)))
        return simp_fail(c, SIMP_ERR_BADARG, "set_state: bad sizes or null arrays");
    if (ntotal > c->maxn)
        return simp_fail(c, SIMP_ERR_MAXN,
                         "Resolution desired too high, the number of particles generated is higher "
                         "than the maximum allowed. (initialize.f90:156-163)");
    if (ntotalb > c->maxnb)
        return simp_fail(c, SIMP_ERR_MAXN,
                         "The number of boundary particles generated is higher than the maximum "
                         "allowed. (boundaries.f90:296-303)");
    invalidate_graph(c);
    const int n = ntotal;
    c->n = n;
    c->nb = ntotalb;
    cudaStream_t s = c->stream;
    // extents and hsml bounds (host)
    double xmin = x[0], xmax = x[0], ymin = x[1], ymax = x[1], hmin = hsml[0], hmax = hsml[0];
    for (int i = 0; i < n; ++i) {
        xmin = std::min(xmin, x[2 * i]);
        xmax = std::max(xmax, x[2 * i]);
        ymin = std::min(ymin, x[2 * i + 1]);
        ymax = std::max(ymax, x[2 * i + 1]);
        hmin = std::min(hmin, hsml[i]);
        hmax = std::max(hmax, hsml[i]);
        if (!(hsml[i] > 0.0) || !(rho[i] > 0.0) || !(h[i] > 0.0))
            return simp_fail(c, SIMP_ERR_BADARG, "set_state: hsml, rho and h must be positive");
    }
    for (int b = 0; b < ntotalb; ++b) {
        xmin = std::min(xmin, xb[2 * b]);
        xmax = std::max(xmax, xb[2 * b]);
        ymin = std::min(ymin, xb[2 * b + 1]);
        ymax = std::max(ymax, xb[2 * b + 1]);
    }
    if (!std::isfinite(xmin + xmax + ymin + ymax))
        return simp_fail(c, SIMP_ERR_BADARG, "set_state: non-finite positions");
    const double max_hsml = (c->prm.max_hsml > 0.0) ? c->prm.max_hsml : hmax * 10.0;  // initialize.f90:191
    c->phys = make_phys(c->prm, max_hsml);
    TRY(size_grid(c, xmin, xmax, ymin, ymax, hmax));
    // particle arrays (original order)
    TRY(upload_interleaved(c, x, c->s0.x, c->s0.y, n, c->tmp));
    TRY(upload_interleaved(c, vx, c->s0.vx, c->s0.vy, n, c->tmp + 2 * (size_t)n));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.m, mass, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.rho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.hs, hsml, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.A, A, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.h, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_init_ids<<<nblk(n, kB), kB, 0, s>>>(n, c->id, c->s0.m, c->s0.rho, c->s0.mor);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    c->host_xb.assign(xb, xb + 2 * (size_t)ntotalb);
    c->host_massb.assign(massb, massb + ntotalb);
    TRY(bin_walls(c, ntotalb, xb, massb));
    // scalars
    Scalars sc{};
    sc.dt = dt;
    sc.t = current_time;
    sc.hmin = hmin;
    sc.hmax = hmax;
    sc.bs = 2.0 * hmin;
    sc.dmax2_bits = 0ull;
    {
        // bound on |coordinate| for the FP32 prefilter (grows on the device)
        const double xa = std::max(std::max(std::fabs(xmin), std::fabs(xmax)),
                                   std::max(std::fabs(ymin), std::fabs(ymax)));
        std::memcpy(&sc.xabs_bits, &xa, sizeof(double));
    }
    {
        const double inf = INFINITY;
        std::memcpy(&sc.acc_hmin, &inf, sizeof(double));
        std::memcpy(&sc.acc_dt, &inf, sizeof(double));
    }
    sc.acc_hmax = 0ull;
    sc.minip = 0x7fffffff;
    sc.skin = list_skin(c, hmax);
    sc.dlist2_bits = 0ull;
    sc.list_scan = 1;
    sc.blocks_done = 0u;
    *c->sc_host = sc;
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc, c->sc_host, sizeof(Scalars), cudaMemcpyHostToDevice, s));
    TRY(rebuild(c));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    c->have_state = true;
    return SIMP_OK;
}

int32_t simp_gpu_get_state(simp_ctx *c, double *x, double *vx, double *mass, double *rho,
                           double *hsml, double *A, double *h, double *dt, double *current_time) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "get_state before set_state");
    const int n = c->n;
    const size_t N = (size_t)n;
    cudaStream_t s = c->stream;
    double *stage = c->tmp;  // 9 n doubles
    k_pack_state<<<nblk(n, kB), kB, 0, s>>>(n, c->id, c->s0, stage);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    struct Out { double *dst; size_t off, len; } outs[] = {
        {x, 0, 2 * N}, {vx, 2 * N, 2 * N}, {mass, 4 * N, N}, {rho, 5 * N, N},
        {hsml, 6 * N, N}, {A, 7 * N, N}, {h, 8 * N, N}};
    for (const Out &o : outs)
        if (o.dst)
            SIMP_CUDA(c, cudaMemcpyAsync(o.dst, stage + o.off, sizeof(double) * o.len,
                                         cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc_host, c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    if (dt) *dt = c->sc_host->dt;
    if (current_time) *current_time = c->sc_host->t;
    return SIMP_OK;
}

int32_t simp_gpu_keep_diag(simp_ctx *c, int32_t keep) {
    if (!c) return SIMP_ERR_BADARG;
    c->keep_diag = keep != 0;
    return SIMP_OK;
}

int32_t simp_gpu_get_diag(simp_ctx *c, double *eps11, double *eps12, double *eps22, double *zeta,
                          double *eta, double *p, double *sig11, double *sig12, double *sig22) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "get_diag before set_state");
    double *outs[9] = {eps11, eps12, eps22, zeta, eta, p, sig11, sig12, sig22};
    for (int k = 0; k < 9; ++k)
        if (outs[k]) TRY(download1(c, c->diag + (size_t)k * c->maxn, outs[k]));
    return SIMP_OK;
}

int32_t simp_gpu_nnps(simp_ctx *c, int32_t *nip, int32_t *p_i, int32_t *p_j, double *r_ij,
                      double *hsml_ij, int32_t cap, int32_t *bnip, int32_t *bp_i, int32_t *bp_j,
                      double *br_ij, int32_t bcap) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "nnps before set_state");
    return export_pairs(c, nip, p_i, p_j, r_ij, hsml_ij, cap, bnip, bp_i, bp_j, br_ij, bcap);
}

int32_t simp_gpu_interaction_stats(simp_ctx *c, int32_t *maxip, int32_t *minip, int64_t *sumip,
                                   int32_t *noip) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "interaction_stats before set_state");
    TRY(read_scalars(c));
    if (maxip) *maxip = c->sc_host->maxip;
    if (minip) *minip = c->sc_host->minip;
    if (sumip) *sumip = (int64_t)c->sc_host->sumip;
    if (noip) *noip = c->sc_host->noip;
    return SIMP_OK;
}

int32_t simp_gpu_single_step(simp_ctx *c, double current_time, double *dxdt, double *dvxdt,
                             double *dhdt, double *dAdt) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "single_step before set_state");
    cudaStream_t s = c->stream;
    k_set_time<<<1, 1, 0, s>>>(c->sc, current_time);
    c->launches += 1;
    launch_reset_stats(c);
    launch_kinematic(c, c->s0, true);
    launch_stress(c, c->s0, c->s0, EPI_RATES);
    SIMP_CUDA(c, cudaGetLastError());
    const size_t M = (size_t)c->maxn;
    if (dxdt) TRY(download2(c, c->s0.vx, c->s0.vy, dxdt));
    if (dvxdt) TRY(download2(c, c->rates, c->rates + M, dvxdt));
    if (dhdt) TRY(download1(c, c->rates + 2 * M, dhdt));
    if (dAdt) TRY(download1(c, c->rates + 3 * M, dAdt));
    TRY(read_scalars(c));
    return check_after(c);
}

int32_t simp_gpu_sum_density(simp_ctx *c, double *rho_out) {
    if (!c || !rho_out) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "sum_density before set_state");
    double *stage = c->tmp;
    TRY(sum_density(c, stage));
    SIMP_CUDA(c, cudaMemcpyAsync(rho_out, stage, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    return SIMP_OK;
}

int32_t simp_gpu_step(simp_ctx *c, int32_t nsteps, double *current_time, double *dt) {
    if (!c || nsteps < 0) return SIMP_ERR_BADARG;
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "step before set_state");
    cudaStream_t s = c->stream;
    // bounds read at the end of the previous call (or by set_state)
    if (wants_regrid(c, *c->sc_host)) TRY(regrid(c));
    else if (wants_rebuild(c, *c->sc_host)) TRY(rebuild(c));
    launch_reset_stats(c);
    TRY(ensure_graph(c, c->keep_diag));
    // The cell list stays exact between sorts (the stencil radius adapts on
    // the device); the host re-sorts when a recent snapshot of the bounds says
    // the stencil would outgrow one ring of cells.  Snapshots are read without
    // stalling the device: the host runs at most kLag steps ahead.
    constexpr int kLag = kSnapRing - 1;
    cudaEvent_t ev[kSnapRing];
    for (int k = 0; k < kSnapRing; ++k) cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
    int rc = SIMP_OK;
    int quiet = 0;  // steps to skip checks after a sort (older snapshots predate it)
    for (int st = 0; st < nsteps && rc == SIMP_OK; ++st) {
        if (st >= kLag) {
            const int slot = (st - kLag) % kSnapRing;
            cudaEventSynchronize(ev[slot]);
            if (quiet > 0) {
                --quiet;
            } else if (wants_regrid(c, c->sc_host[1 + slot])) {
                rc = regrid(c);
                if (rc != SIMP_OK) break;
                rc = ensure_graph(c, c->keep_diag);
                if (rc != SIMP_OK) break;
                quiet = kLag;
            } else if (wants_rebuild(c, c->sc_host[1 + slot])) {
                rc = rebuild(c);
                if (rc != SIMP_OK) break;
                quiet = kLag;
            }
        }
        cudaError_t e = cudaGraphLaunch(c->step_graph, s);
        if (e != cudaSuccess) { rc = simp_cuda_check(c, e, "cudaGraphLaunch"); break; }
        c->launches += c->graph_kernels;
        cudaMemcpyAsync(&c->sc_host[1 + st % kSnapRing], c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s);
        cudaEventRecord(ev[st % kSnapRing], s);
        c->steps_since_rebuild++;
        if (c->graph_profiled) {
            // timing mode: wait for this step and add up its kernel times
            e = cudaEventSynchronize(c->prof_ev[simp_ctx::kProfKernels]);
            if (e != cudaSuccess) { rc = simp_cuda_check(c, e, "profile event"); break; }
            for (int k = 0; k < simp_ctx::kProfKernels; ++k) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, c->prof_ev[k], c->prof_ev[k + 1]);
                c->prof_ms[k] += ms;
            }
            c->prof_steps += 1;
        }
    }
    cudaError_t e = cudaStreamSynchronize(s);
    for (int k = 0; k < kSnapRing; ++k) cudaEventDestroy(ev[k]);
    if (rc != SIMP_OK) return rc;
    if (e != cudaSuccess) return simp_cuda_check(c, e, "simp_gpu_step");
    TRY(read_scalars(c));
    if (current_time) *current_time = c->sc_host->t;
    if (dt) *dt = c->sc_host->dt;
    return check_after(c);
}

void *simp_gpu_stream(simp_ctx *c) { return c ? (void *)c->stream : nullptr; }

int64_t simp_gpu_kernel_launches(const simp_ctx *c) { return c ? (int64_t)c->launches : 0; }

int32_t simp_gpu_profile(simp_ctx *c, int32_t on) {
    if (!c) return SIMP_ERR_BADARG;
    c->profile = on != 0;
    for (double &v : c->prof_ms) v = 0.0;
    c->prof_steps = 0;
    return SIMP_OK;
}

int32_t simp_gpu_kernel_times(simp_ctx *c, double *ms, int32_t n_kernels, int64_t *steps_timed) {
    if (!c || !ms || n_kernels < 0) return SIMP_ERR_BADARG;
    for (int k = 0; k < n_kernels; ++k) ms[k] = (k < simp_ctx::kProfKernels) ? c->prof_ms[k] : 0.0;
    if (steps_timed) *steps_timed = c->prof_steps;
    return SIMP_OK;
}

const char *simp_gpu_last_error(const simp_ctx *c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"
