// C ABI of the SIMP hot path (include/simp_gpu.h): context lifecycle, basin
// (instance) admission and removal, state transfer in the reference's
// Fortran layouts, and the per-step driver.
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
constexpr int kIdShift = 21;   // batch particle ids: slot << 21 | local index
inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

#define TRY(expr)                       \
    do {                                \
        int _rc = (expr);               \
        if (_rc != SIMP_OK) return _rc; \
    } while (0)

__global__ void k_deinterleave(int n, const double *__restrict__ in, double *__restrict__ a,
                               double *__restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = in[2 * i];
    b[i] = in[2 * i + 1];
}

// Fields of a single basin into the caller's order; a null source is skipped.
__global__ void k_pack_fields(int n, int id_base, const int *__restrict__ id, const double *__restrict__ a,
                              const double *__restrict__ b, double *__restrict__ out_a, double *__restrict__ out_b) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = id[k] - id_base;
    if (!SIMP_IN_RANGE(o, 0, n, SITE_SORT)) return;
    if (a) out_a[o] = a[k];
    if (b) out_b[o] = b[k];
}

// Two fields of a single basin into one interleaved array in the caller's
// order (x(2,n), vx(2,n)).
__global__ void k_pack_pair(int n, int id_base, const int *__restrict__ id, const double *__restrict__ a,
                            const double *__restrict__ b, double *__restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = id[k] - id_base;
    if (!SIMP_IN_RANGE(o, 0, n, SITE_SORT)) return;
    out[2 * (size_t)o] = a[k];
    out[2 * (size_t)o + 1] = b[k];
}

// New particles [off, off + n): ids, instance, sort positions, m / rho, and
// the summation density's kept kernel_zero (initialize.f90:60).
__global__ void k_init_new(int n, int off, int id_base, int slot, int *id, int *pinst, State s, double *xr,
                           double *yr, int *nbr_count, double *k0) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = off + k;
    id[i] = id_base + k;
    pinst[i] = slot;
    nbr_count[i] = -1;   // its Verlet list is built by the next kinematic pass
    xr[i] = s.x[i];
    yr[i] = s.y[i];
    s.mor[i] = s.m[i] / s.rho[i];
    refresh_views(s, i);
    if (k0) k0[i] = 0.0;
}

__global__ void k_mark_removed(int n, int slot, int *pinst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && pinst[i] == slot) pinst[i] = -1;
}

__global__ void k_flag_inst(Inst *inst, int slot, int flag) { atomicOr(&inst[slot].flags, flag); }

// One instance's state to its own particle order: stage = [x,y interleaved |
// vx,vy interleaved | mass | rho | hsml | A | h], 9 n_k doubles.
__global__ void k_pack_state(int n, int slot, int id_base, int nk, const int *__restrict__ pinst,
                             const int *__restrict__ id, State s, double *__restrict__ stage) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n || pinst[k] != slot) return;
    const size_t o = (size_t)(id[k] - id_base), N = (size_t)nk;
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

// Cell-order arrays of instance 0 to its particle order (single basin).
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

__global__ void k_set_time0(Scalars *sc, Inst *inst, double t) {
    sc->t = t;
    inst[0].t = t;
}

// Extents and validity of an uploaded basin [off, off + n): per block
// xmin, -xmax, ymin, -ymax, hmin, -hmax (all minima), and the counts of
// non-positive hsml / rho / h and of non-finite positions.
constexpr int kRedBlocks = 296;
constexpr int kRedVals = 8;
__global__ void __launch_bounds__(256) k_extents(int n, int off, State s, double *part) {
    double v[kRedVals] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, 0.0, 0.0};
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = off + k;
        const double x = s.x[i], y = s.y[i], hs = s.hs[i];
        v[0] = fmin(v[0], x);
        v[1] = fmin(v[1], -x);
        v[2] = fmin(v[2], y);
        v[3] = fmin(v[3], -y);
        v[4] = fmin(v[4], hs);
        v[5] = fmin(v[5], -hs);
        if (!(hs > 0.0) || !(s.rho[i] > 0.0) || !(s.h[i] > 0.0)) v[6] += 1.0;
        if (!isfinite(x) || !isfinite(y)) v[7] += 1.0;
    }
    __shared__ double red[kRedVals][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kRedVals; ++q) {
        for (int o = 16; o > 0; o >>= 1) {
            const double t = __shfl_xor_sync(0xffffffffu, v[q], o);
            v[q] = (q < 6) ? fmin(v[q], t) : v[q] + t;
        }
        if (lane == 0) red[q][w] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < kRedVals) {
        const int q = threadIdx.x;
        double r = red[q][0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = (q < 6) ? fmin(r, red[q][k]) : r + red[q][k];
        part[blockIdx.x * kRedVals + q] = r;
    }
}

// Wall particles per cell key (for their cell-start offsets).
__global__ void k_count_walls(int nb, const int *__restrict__ key, int *__restrict__ cnt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nb) atomicAdd(&cnt[key[k]], 1);
}

__global__ void k_grow_xabs(Scalars *sc, double xa) {
    atomicMax(&sc->xabs_bits, (unsigned long long)__double_as_longlong(xa));
}

// set_state of a state that continues the resident basin (the same
// particles in the same caller order, the same hsml): the values go into
// the particles' current places in cell order, so the sort, the cell lists
// and the Verlet lists stay, and the displacement bounds grow as after a
// step.  stage = [x,y interleaved | vx,vy interleaved | mass | rho | hsml |
// A | h] in the caller's order, uploaded in the groups below; each group's
// kernel runs as soon as its part has landed, while the next part is
// copied.  Per block, each group reduces its own slots of `part`:
// [0] non-finite positions, [1] changed hsml, [2] max squared displacement
// since the sort, [3] since the lists were built, [4] max |coordinate|
// (positions); [5] max hsml, [6] -min hsml (hsml); [7] other invalid
// values (velocities, then mass and rho, then A and h, adding up in stream
// order).
enum ContGroup { CG_POS, CG_VEL, CG_MASS, CG_HSML, CG_AH, kContGroups };

template <int G>
__global__ void __launch_bounds__(256) k_continue_group(int n, const int *__restrict__ id,
                                                       const double *__restrict__ stage, State s,
                                                       const double *__restrict__ xr,
                                                       const double *__restrict__ yr, NbrList nl, double *part) {
    double v[kRedVals] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -INFINITY, 0.0};
    const size_t N = (size_t)n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!SIMP_IN_RANGE(id[i], 0, n, SITE_SORT)) continue;
        const size_t o = (size_t)id[i];
        if (G == CG_POS) {
            const double x = stage[2 * o], y = stage[2 * o + 1];
            if (isfinite(x) && isfinite(y)) {
                const double dxr = x - xr[i], dyr = y - yr[i];
                v[2] = fmax(v[2], dxr * dxr + dyr * dyr);
                if (nl.count[i] >= 0) {
                    const double dxl = x - nl.xl[i], dyl = y - nl.yl[i];
                    v[3] = fmax(v[3], dxl * dxl + dyl * dyl);
                }
                v[4] = fmax(v[4], fmax(fabs(x), fabs(y)));
            } else {
                v[0] += 1.0;
            }
            s.x[i] = x;
            s.y[i] = y;
            s.xy[i] = make_double2(x, y);
            s.pf[i] = make_float4((float)x, (float)y, s.hsf[i], 0.0f);
        } else if (G == CG_VEL) {
            const double vx = stage[2 * N + 2 * o], vy = stage[2 * N + 2 * o + 1];
            if (!(isfinite(vx) && isfinite(vy))) v[7] += 1.0;
            s.vx[i] = vx;
            s.vy[i] = vy;
            s.vxy[i] = make_double2(vx, vy);
        } else if (G == CG_MASS) {
            const double m = stage[4 * N + o], rho = stage[5 * N + o];
            if (!(isfinite(m) && isfinite(rho) && rho > 0.0)) v[7] += 1.0;
            const double mor = m / rho;
            s.m[i] = m;
            s.rho[i] = rho;
            s.mor[i] = mor;
            if (s.hmm) s.hmm[i] = make_float4(s.hsf[i], (float)m, (float)mor, 0.0f);
            else s.mm[i] = make_double2(m, mor);
        } else if (G == CG_HSML) {
            const double hs = stage[6 * N + o];
            if (!(hs == s.hs[i])) v[1] += 1.0;
            v[5] = fmax(v[5], hs);
            v[6] = fmax(v[6], -hs);
        } else {
            const double A = stage[7 * N + o], h = stage[8 * N + o];
            if (!(isfinite(A) && isfinite(h) && h > 0.0)) v[7] += 1.0;
            s.A[i] = A;
            s.h[i] = h;
        }
    }
    // the slots of this group: a bit mask over [0, kRedVals)
    constexpr unsigned own = G == CG_POS ? 0x1du : G == CG_HSML ? 0x62u : 0x80u;
    __shared__ double red[kRedVals][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kRedVals; ++q) {
        if (!((own >> q) & 1u)) continue;
        const bool sum = q == 0 || q == 1 || q == 7;
        for (int d = 16; d > 0; d >>= 1) {
            const double t = __shfl_xor_sync(0xffffffffu, v[q], d);
            v[q] = sum ? v[q] + t : fmax(v[q], t);
        }
        if (lane == 0) red[q][w] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < kRedVals && ((own >> threadIdx.x) & 1u)) {
        const int q = threadIdx.x;
        const bool sum = q == 0 || q == 1 || q == 7;
        double r = red[q][0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = sum ? r + red[q][k] : fmax(r, red[q][k]);
        double &slot = part[blockIdx.x * kRedVals + q];
        slot = (q == 7 && G != CG_VEL) ? slot + r : r;   // (the velocity group writes slot 7 first)
    }
}

// The bounds of a continued state, as the step epilogue would leave them.
// (hsml is unchanged, so are its bounds, the bucket size and the skin)
__global__ void k_continue_finish(Scalars *sc, Inst *inst, double dt, double t, double d2, double dl2,
                                  double xa, int hsml_evolves) {
    sc->dt = dt;
    sc->t = t;
    inst[0].t = t;
    const unsigned long long b2 = (unsigned long long)__double_as_longlong(d2);
    if (b2 > sc->dmax2_bits) sc->dmax2_bits = b2;
    if (b2 > inst[0].dmax2_bits) inst[0].dmax2_bits = b2;
    const unsigned long long bl = (unsigned long long)__double_as_longlong(dl2);
    if (bl > sc->dlist2_bits) sc->dlist2_bits = bl;
    const unsigned long long bx = (unsigned long long)__double_as_longlong(xa);
    if (bx > sc->xabs_bits) sc->xabs_bits = bx;
    // the rule of the stress pass's last block (lists_block_done)
    const double dl = sqrt(__longlong_as_double((long long)sc->dlist2_bits));
    if (hsml_evolves || !(dl < 0.75 * sc->skin)) sc->list_scan = 1;
}

Phys make_phys(const simp_params &p, double max_hsml) {
    Phys P{};
    P.skf = p.skf;
    P.scale_h = scale_h_of(p.skf);
    P.viscosity = p.viscosity;
    P.pressure_force = p.pressure_force;
    P.eos_alg = p.eos_alg;
    P.wind_force = p.wind_force;
    P.water_force = p.water_force;
    P.wind_kind = p.wind_kind;
    P.boundary_pressure = p.boundary_pressure;
    P.sle = p.sle;
    P.den_alg = p.den_alg;
    P.nnps = p.nnps_algorithm;
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
    P.current_u = p.current_u;
    P.current_v = p.current_v;
    P.max_hsml = max_hsml;
    P.rheology = p.rheology;
    P.pa_sph = p.pa_sph;
    P.int_algorithm = p.int_algorithm;
    P.zeta_max = p.zeta_max;
    P.eta_max = p.eta_max;
    P.mu = tan(p.phi * kPi / 180.0);   // data_variables.f90:180
    P.bfa = p.bfa;
    P.boundary_friction = p.boundary_friction;
    P.kappa_t = p.kappa_t;
    P.xi = p.xi;
    P.Y = p.Y;
    P.nu = p.nu;
    // regularization is called when either switch is on, and then applies
    // the artificial viscosity of art_visc_alg (regularization.f90:23-35)
    const bool reg = p.xsph_regularization || p.artificial_visc;
    P.xsph = p.xsph_regularization ? 1 : 0;
    P.art_visc = (reg && (p.art_visc_alg == 1 || p.art_visc_alg == 2)) ? p.art_visc_alg : 0;
    P.artificial_visc = p.artificial_visc ? 1 : 0;
    P.csound = (p.artificial_visc || p.tse == 1 || p.boundary_friction) ? 1 : 0;   // sound_speed.f90:21
    P.alpha_pi = p.alpha_pi;
    P.beta_pi = p.beta_pi;
    P.chi = p.chi;
    return P;
}

int check_params(simp_ctx *c, const simp_params &p, bool batch) {
    auto bad = [&](const char *what) { return simp_fail(c, SIMP_ERR_BADARG, std::string("unsupported switch: ") + what); };
    if (p.int_algorithm < 1 || p.int_algorithm > 3) return bad("int_algorithm (1 Euler, 2 predictor-corrector, 3 leap-frog)");
    if (p.nnps_algorithm != 1 && p.nnps_algorithm != 2) return bad("nnps_algorithm (1 or 2)");
    if (p.sle < 0 || p.sle > 2) return bad("sle (0, 1 or 2)");
    if (p.tse < 0 || p.tse > 2) return bad("tse (0 fixed, 1 Monaghan, 2 viscous-plastic)");
    if (p.rheology != 1 && p.rheology != 2) return bad("rheology (1 elliptical, 2 Mohr-Coulomb)");
    if (p.eos_alg < 1 || p.eos_alg > 3) return bad("eos_alg (1, 2 or 3)");
    if (p.pa_sph != 1 && p.pa_sph != 2) return bad("pa_sph (1 or 2)");
    if (!skf_known(p.skf)) return bad("skf (1 to 9)");
    if (p.den_alg < 1 || p.den_alg > 3) return bad("den_alg (1 summation, 2 continuity, 3 h rho_ice)");
    if (p.bfa < 1 || p.bfa > 3) return bad("bfa (1 Monaghan, 2 Wang, 3 Marquis)");
    if (p.bfa == 2 && batch) return bad("bfa = 2 (wall normals) in a batch");
    if (p.precision != SIMP_PREC_FP64 && p.precision != SIMP_PREC_MIXED) return bad("precision (0 FP64, 1 mixed)");
    if (!(p.e > 0.0) || !(p.rho_ice > 0.0) || !(p.b_length > 0.0)) return bad("material constants");
    if (batch && (p.tse != 0 || p.sle != 0)) return bad("batches need a fixed dt (tse = 0) and fixed hsml (sle = 0)");
    return SIMP_OK;
}

template <class T>
int dalloc(simp_ctx *c, T **p, size_t count) {
    if (count == 0) count = 1;
    if (cudaMalloc((void **)p, count * sizeof(T)) != cudaSuccess)
        return simp_fail(c, SIMP_ERR_NOMEM, "device allocation failed");
    return SIMP_OK;
}

void free_all(simp_ctx *c) {
    void *ptrs[] = {c->s0.x, c->s0.y, c->s0.vx, c->s0.vy, c->s0.m, c->s0.rho, c->s0.mor, c->s0.h,
                    c->s0.A, c->s0.hs, c->s1.x, c->s1.y, c->s1.vx, c->s1.vy, c->s1.rho, c->s1.mor,
                    c->s1.h, c->s1.A, c->mass1, c->xr, c->yr, c->xl, c->yl, c->cell, c->id, c->pinst,
                    c->tau11, c->tau12, c->tau22, c->div, c->diag, c->rates, c->bx, c->by, c->bm, c->bnx, c->bny,
                    c->bid, c->binst, c->bcell, c->bcell_start, c->cell_start, c->cnt, c->perm, c->tmp,
                    c->itmp, c->scan_tmp, c->sc, c->pair_cnt, c->bpair_cnt, c->pair_buf_i,
                    c->pair_buf_j, c->pair_buf_r, c->pair_buf_h, c->nbr, c->nbr_count,
                    c->pair_j, c->pair_count, c->nbr_tmp, c->s0.hsf,
                    c->inst_dev, c->row_map, c->chunk_cnt, c->chunk_off, c->chunks, c->s0.xy, c->s0.vxy,
                    c->s0.pf, c->s0.mm, c->s0.hmm, c->s1.xy, c->s1.vxy, c->s1.pf, c->s1.mm, c->s1.hmm,
                    c->tau_a, c->tau_b, c->tau_q, c->pair_dw, c->drhodt, c->k0, c->red_dev, c->reg,
                    c->early_stage};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c->sc_host) cudaFreeHost(c->sc_host);
    if (c->red_host) cudaFreeHost(c->red_host);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    if (c->sort_graph) cudaGraphExecDestroy(c->sort_graph);
    for (cudaEvent_t e : c->prof_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->sort_ev)
        if (e) cudaEventDestroy(e);
    if (c->ev_graph) cudaEventDestroy(c->ev_graph);
    for (cudaEvent_t e : c->ev_up)
        if (e) cudaEventDestroy(e);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
}

// The step graph captured kernel arguments that changed (sizes, grid,
// physics): the next step re-captures it and updates the instantiated graph
// in place when the kernels are the same ones (a new state of the same
// basin), else instantiates it anew.
void invalidate_graph(simp_ctx *c) { c->graph_stale = true; }

// Verlet-list skin: the parameter when given, else 10% of max(hsml).
double list_skin(const simp_ctx *c, double hmax) {
    return (c->prm.skin >= 0.0) ? c->prm.skin : 0.1 * hmax;
}

// Grid of one instance from its extents: cell side 1.15 (hsml + skin) (the
// Verlet-list reach plus room for motion between sorts); the cell count is
// capped (a larger side only adds candidates, never drops pairs).
void size_inst_grid(const simp_ctx *c, InstHost &h, double xmin, double xmax, double ymin, double ymax,
                    double hmax) {
    double cs = (hmax + list_skin(c, hmax)) * 1.15;
    if (!(cs > 0.0)) cs = 1.0;
    const double ext = std::max(xmax - xmin, ymax - ymin);
    const double margin = std::max(2.0 * cs, 0.02 * ext);
    const double w = xmax - xmin + 2.0 * margin, hh = ymax - ymin + 2.0 * margin;
    const double cap = std::max(4.0 * (double)h.n, 65536.0);
    while (std::ceil(w / cs) * std::ceil(hh / cs) > cap) cs *= 1.25;
    Inst &I = h.I;
    I.x0 = xmin - margin;
    I.y0 = ymin - margin;
    I.cs = cs;
    I.inv_cs = 1.0 / cs;
    I.ncx = std::max(1, (int)std::ceil(w / cs));
    I.ncy = std::max(1, (int)std::ceil(hh / cs));
    h.grid_hmax = hmax;
}

// Cell-key bases of the active instances, the device table, the cell-list
// capacity and the wall cells.  Reads the device table first: current_time,
// displacement bounds and flags evolve there.
int layout(simp_ctx *c) {
    cudaStream_t s = c->stream;
    std::vector<Inst> cur(c->max_inst);
    SIMP_CUDA(c, cudaMemcpyAsync(cur.data(), c->inst_dev, sizeof(Inst) * c->max_inst, cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    // cell-key bases in admission order, so that a new basin's keys come
    // after every resident one (it is appended in memory, nothing moves)
    std::vector<int> by_order;
    for (int q = 0; q < c->max_inst; ++q)
        if (c->insts[q].active) by_order.push_back(q);
    std::sort(by_order.begin(), by_order.end(),
              [&](int a, int b) { return c->insts[a].order < c->insts[b].order; });
    int base = 0, top = 0;
    for (int q : by_order) {
        InstHost &h = c->insts[q];
        if (h.I.base >= 0) {   // already on the device: keep its evolving fields
            h.I.t = cur[q].t;
            h.I.dmax2_bits = cur[q].dmax2_bits;
            h.I.flags = cur[q].flags;
            h.I.hmin = cur[q].hmin;
            h.I.hmax = cur[q].hmax;
            h.I.bs = cur[q].bs;
        }
        h.I.base = base;
        base += h.I.ncx * h.I.ncy;
        top = std::max(top, q + 1);
    }
    c->total_cells = base;
    c->ninst = std::max(top, 1);
    const size_t need = (size_t)base + 2;
    if (need > c->cell_cap) {
        // (grown at least twofold, from a reserve of maxn / 8 cells: a
        // batch that admits basin after basin reallocates rarely; cudaFree
        // waits for the device)
        cudaFree(c->cell_start);
        cudaFree(c->cnt);
        cudaFree(c->bcell_start);
        c->cell_start = c->cnt = c->bcell_start = nullptr;
        const size_t capn = std::max(2 * need, std::max(2 * c->cell_cap, (size_t)c->maxn / 8 + 4096));
        TRY(dalloc(c, &c->cell_start, capn));
        TRY(dalloc(c, &c->cnt, capn));
        TRY(dalloc(c, &c->bcell_start, capn));
        const size_t sb = scan_tmp_bytes((int)std::max<size_t>(capn, (size_t)std::max(c->maxn, c->maxnb) + 1));
        if (sb > c->scan_tmp_bytes) {
            cudaFree(c->scan_tmp);
            c->scan_tmp = nullptr;
            if (cudaMalloc(&c->scan_tmp, sb) != cudaSuccess) return simp_fail(c, SIMP_ERR_NOMEM, "device allocation failed");
            c->scan_tmp_bytes = sb;
        }
        c->cell_cap = capn;
    }
    // cell rows of all instances, for the chunks of the tiled passes
    std::vector<int2> rows;
    for (int q : by_order)
        for (int r = 0; r < c->insts[q].I.ncy; ++r) rows.push_back(make_int2(q, r));
    c->total_rows = (int)rows.size();
    const size_t need_chunks = (size_t)c->maxn / kMinTileThreads + rows.size() + 2;
    if (rows.size() + 2 > c->row_cap || need_chunks > c->chunk_cap) {
        cudaFree(c->row_map);
        cudaFree(c->chunk_cnt);
        cudaFree(c->chunk_off);
        cudaFree(c->chunks);
        c->row_map = nullptr;
        c->chunk_cnt = c->chunk_off = nullptr;
        c->chunks = nullptr;
        const size_t rcap = std::max(2 * (rows.size() + 2), std::max(2 * c->row_cap, (size_t)4096));
        TRY(dalloc(c, &c->row_map, rcap));
        TRY(dalloc(c, &c->chunk_cnt, rcap));
        TRY(dalloc(c, &c->chunk_off, rcap));
        const size_t ccap = (size_t)c->maxn / kMinTileThreads + rcap;
        TRY(dalloc(c, &c->chunks, ccap));
        c->row_cap = rcap;
        c->chunk_cap = ccap;
    }
    if (!rows.empty())
        SIMP_CUDA(c, cudaMemcpyAsync(c->row_map, rows.data(), sizeof(int2) * rows.size(), cudaMemcpyHostToDevice, s));
    std::vector<Inst> table(c->max_inst);
    for (int q = 0; q < c->max_inst; ++q) table[q] = c->insts[q].active ? c->insts[q].I : Inst{};
    SIMP_CUDA(c, cudaMemcpyAsync(c->inst_dev, table.data(), sizeof(Inst) * c->max_inst, cudaMemcpyHostToDevice, s));
    // walls of every active instance, sorted by cell key (stable): each
    // instance's walls sorted by their local cell once per grid, then the
    // instances in key-base order (their key ranges are disjoint)
    int nb = 0;
    for (int q : by_order) {
        InstHost &h = c->insts[q];
        const Inst &I = h.I;
        if (h.wall_grid_cs != I.cs || h.wall_grid_x0 != I.x0 || h.wall_grid_y0 != I.y0 ||
            h.wall_key.size() != (size_t)h.nb) {
            std::vector<std::pair<int, int>> kb((size_t)h.nb);
            for (int b = 0; b < h.nb; ++b) {
                const double xb = h.xb[2 * b], yb = h.xb[2 * b + 1];
                const int cx = clampi((int)std::floor((xb - I.x0) * I.inv_cs), 0, I.ncx - 1);
                const int cy = clampi((int)std::floor((yb - I.y0) * I.inv_cs), 0, I.ncy - 1);
                kb[(size_t)b] = {cy * I.ncx + cx, b};
            }
            std::stable_sort(kb.begin(), kb.end(),
                             [](const std::pair<int, int> &a, const std::pair<int, int> &b) { return a.first < b.first; });
            h.wall_key.resize((size_t)h.nb);
            h.wall_order.resize((size_t)h.nb);
            for (int k = 0; k < h.nb; ++k) {
                h.wall_key[(size_t)k] = kb[(size_t)k].first;
                h.wall_order[(size_t)k] = kb[(size_t)k].second;
            }
            h.wall_grid_cs = I.cs;
            h.wall_grid_x0 = I.x0;
            h.wall_grid_y0 = I.y0;
        }
        nb += h.nb;
    }
    std::vector<double> hx(nb), hy(nb), hm(nb), hnx(nb), hny(nb);
    std::vector<int> hid(nb), hinst(nb), hcell(nb);
    int k = 0;
    for (int q : by_order) {
        const InstHost &h = c->insts[q];
        const bool hn = h.bn.size() == 2 * (size_t)h.nb;
        for (int e = 0; e < h.nb; ++e, ++k) {
            const int b = h.wall_order[(size_t)e];
            hx[k] = h.xb[2 * b];
            hy[k] = h.xb[2 * b + 1];
            hm[k] = h.massb[b];
            hnx[k] = hn ? h.bn[2 * b] : 0.0;
            hny[k] = hn ? h.bn[2 * b + 1] : 0.0;
            hid[k] = b;
            hinst[k] = q;
            hcell[k] = h.I.base + h.wall_key[(size_t)e];
        }
    }
    if (nb > 0) {
        SIMP_CUDA(c, cudaMemcpyAsync(c->bx, hx.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->by, hy.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->bm, hm.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        if (c->bnx) {
            SIMP_CUDA(c, cudaMemcpyAsync(c->bnx, hnx.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
            SIMP_CUDA(c, cudaMemcpyAsync(c->bny, hny.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, s));
        }
        SIMP_CUDA(c, cudaMemcpyAsync(c->bid, hid.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->binst, hinst.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
        SIMP_CUDA(c, cudaMemcpyAsync(c->bcell, hcell.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, s));
    }
    // cell-start offsets of the walls, counted and scanned on the device
    SIMP_CUDA(c, cudaMemsetAsync(c->cnt, 0, sizeof(int) * ((size_t)base + 1), s));
    if (nb > 0) k_count_walls<<<nblk(nb, kB), kB, 0, s>>>(nb, c->bcell, c->cnt);
    launch_scan_i32(c->cnt, c->bcell_start, base, c->scan_tmp, s);
    c->launches += 1 + kScanKernels;
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    c->nb = nb;
    invalidate_graph(c);
    return SIMP_OK;
}

DueMask mask_of(int slot) {
    DueMask m{};
    if (slot >= 0) m.w[slot >> 6] |= 1ull << (slot & 63);
    return m;
}

// Uploads one basin's particles to [c->n, c->n + n) (nothing else changes
// until add_instance takes them) and reduces their extents on the device.
int stage_instance(simp_ctx *c, int n, const double *x, const double *vx, const double *mass,
                   const double *rho, const double *hsml, const double *A, const double *h, int nb,
                   const double *xb, const double *massb, Extents *e) {
    if (n < 1 || nb < 0 || !x || !vx || !mass || !rho || !hsml || !A || !h || (nb > 0 && (!xb || !massb)))
        return simp_fail(c, SIMP_ERR_BADARG, "bad sizes or null arrays");
    if (c->n + n > c->maxn)
        return simp_fail(c, SIMP_ERR_MAXN,
                         "Resolution desired too high, the number of particles generated is higher "
                         "than the maximum allowed. (initialize.f90:156-163)");
    if (c->nb + nb > c->maxnb)
        return simp_fail(c, SIMP_ERR_MAXN,
                         "The number of boundary particles generated is higher than the maximum "
                         "allowed. (boundaries.f90:296-303)");
    if (c->id_stride && n >= c->id_stride)
        return simp_fail(c, SIMP_ERR_BADARG, "a basin of a batch holds at most 2,097,151 particles");
    cudaStream_t s = c->stream;
    const int off = c->n;
    const size_t N = (size_t)n;
    double *stage = c->tmp;
    SIMP_CUDA(c, cudaMemcpyAsync(stage, x, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(stage + 2 * N, vx, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, s));
    k_deinterleave<<<nblk(n, kB), kB, 0, s>>>(n, stage, c->s0.x + off, c->s0.y + off);
    k_deinterleave<<<nblk(n, kB), kB, 0, s>>>(n, stage + 2 * N, c->s0.vx + off, c->s0.vy + off);
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.m + off, mass, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.rho + off, rho, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.hs + off, hsml, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.A + off, A, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->s0.h + off, h, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    const int rb = std::min(kRedBlocks, nblk(n, 256));
    k_extents<<<rb, 256, 0, s>>>(n, off, c->s0, c->red_dev);
    c->launches += 3;
    SIMP_CUDA(c, cudaGetLastError());
    SIMP_CUDA(c, cudaMemcpyAsync(c->red_host, c->red_dev, sizeof(double) * kRedVals * rb, cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    double v[kRedVals] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, 0.0, 0.0};
    for (int b = 0; b < rb; ++b)
        for (int q = 0; q < kRedVals; ++q) {
            const double t = c->red_host[b * kRedVals + q];
            v[q] = (q < 6) ? std::min(v[q], t) : v[q] + t;
        }
    if (v[6] > 0.0) return simp_fail(c, SIMP_ERR_BADARG, "hsml, rho and h must be positive");
    e->n = n;
    e->xmin = v[0];
    e->xmax = -v[1];
    e->ymin = v[2];
    e->ymax = -v[3];
    e->hmin = v[4];
    e->hmax = -v[5];
    e->finite = v[7] == 0.0;
    return SIMP_OK;
}

// Appends the staged basin after the current particles and sorts it in.
int flush_batch(simp_ctx *c, bool compact);

int add_instance(simp_ctx *c, int slot, const simp_forcing &f, const Extents &e, int nb, const double *xb,
                 const double *massb, double t0) {
    const int n = e.n;
    double xmin = e.xmin, xmax = e.xmax, ymin = e.ymin, ymax = e.ymax;
    const double hmin = e.hmin, hmax = e.hmax;
    const double pxa = std::max(std::max(std::fabs(xmin), std::fabs(xmax)), std::max(std::fabs(ymin), std::fabs(ymax)));
    if (!e.finite) return simp_fail(c, SIMP_ERR_BADARG, "non-finite positions");
    for (int b = 0; b < nb; ++b) {
        xmin = std::min(xmin, xb[2 * b]);
        xmax = std::max(xmax, xb[2 * b]);
        ymin = std::min(ymin, xb[2 * b + 1]);
        ymax = std::max(ymax, xb[2 * b + 1]);
    }
    if (!std::isfinite(xmin + xmax + ymin + ymax))
        return simp_fail(c, SIMP_ERR_BADARG, "non-finite positions");
    InstHost &ih = c->insts[slot];
    ih = InstHost{};
    ih.active = true;
    ih.n = n;
    ih.nb = nb;
    ih.id_base = c->id_stride * slot;
    ih.order = c->next_order++;
    ih.xb.assign(xb, xb + 2 * (size_t)nb);
    ih.massb.assign(massb, massb + nb);
    size_inst_grid(c, ih, xmin, xmax, ymin, ymax, hmax);
    Inst &I = ih.I;
    I.base = -1;   // not laid out yet
    I.wind_kind = f.wind_kind;
    I.wind_u = f.wind_u;
    I.wind_v = f.wind_v;
    I.vortex_x = f.vortex_x;
    I.vortex_y = f.vortex_y;
    I.vortex_umax = f.vortex_umax;
    I.vortex_radius = f.vortex_radius;
    I.b_length = c->prm.b_length;
    I.t = t0;
    I.hmin = hmin;
    I.hmax = hmax;
    I.bs = 2.0 * hmin;
    I.dmax2_bits = 0ull;
    I.flags = 0;
    // particle arrays at [off, off + n), staged by stage_instance
    cudaStream_t s = c->stream;
    const int off = c->n;
    k_init_new<<<nblk(n, kB), kB, 0, s>>>(n, off, ih.id_base, slot, c->id, c->pinst, c->s0, c->xr, c->yr,
                                          c->nbr_count, c->k0);
    k_grow_xabs<<<1, 1, 0, s>>>(c->sc, pxa);
    c->launches += 2;
    SIMP_CUDA(c, cudaGetLastError());
    c->n += n;
    c->nb += nb;
    // the new basin's keys come last: only its own range is sorted, and the
    // resident basins keep their places and their Verlet lists.  A batch lays
    // out and sorts the basins admitted since its last flush together, at
    // the next flush (the next step, or a read of a basin).
    c->pending_from = std::min(c->pending_from, off);
    if (c->pending_due.empty()) c->pending_due.assign(kMaxSlots / 64, 0ull);
    c->pending_due[(size_t)slot >> 6] |= 1ull << (slot & 63);
    if (c->max_inst == 1) return flush_batch(c, false);
    return SIMP_OK;
}

// First position of an instance in memory (instances lie in admission order).
int inst_offset(const simp_ctx *c, int slot) {
    int off = 0;
    for (const InstHost &h : c->insts)
        if (h.active && h.order < c->insts[slot].order) off += h.n;
    return off;
}

// A retired basin leaves the batch at once (it is neither searched nor
// stepped, and its slot reads as free), but its particles keep their places
// until a compaction drops all retired basins together: when they make up a
// quarter of the batch, or an admission needs their room or slot.  Every
// compaction moves the basins after the first retired one down, as one
// removal at a time would, so the survivors' results do not change.
int remove_instance(simp_ctx *c, int slot) {
    InstHost &h = c->insts[slot];
    if (!h.active || h.retired) return simp_fail(c, SIMP_ERR_BADARG, "slot is free");
    h.retired = true;
    h.I.flags |= FLAG_RETIRED;
    c->zombie_n += h.n;
    k_flag_inst<<<1, 1, 0, c->stream>>>(c->inst_dev, slot, FLAG_RETIRED);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    if (c->max_inst == 1) return flush_batch(c, true);
    return SIMP_OK;
}

// The deferred work of a batch: with `compact`, every retired basin's
// particles are dropped; the basins admitted since the last flush are laid
// out and sorted.  One layout and one sort from the first position that
// changes.
int flush_batch(simp_ctx *c, bool compact) {
    int from = c->pending_from;
    DueMask due{};
    for (size_t w = 0; w < c->pending_due.size() && w < (size_t)(kMaxSlots / 64); ++w) due.w[w] = c->pending_due[w];
    bool any = from != 0x7fffffff;
    if (compact && c->zombie_n > 0) {
        for (int q = 0; q < c->max_inst; ++q) {
            const InstHost &h = c->insts[q];
            if (!h.active || !h.retired) continue;
            from = std::min(from, inst_offset(c, q));   // (offsets before any is dropped)
            k_mark_removed<<<nblk(c->n, kB), kB, 0, c->stream>>>(c->n, q, c->pinst);
            c->launches += 1;
            due.w[q >> 6] &= ~(1ull << (q & 63));
        }
        for (InstHost &h : c->insts)
            if (h.active && h.retired) h = InstHost{};
        c->zombie_n = 0;
        any = true;
    }
    if (!any) return SIMP_OK;
    TRY(layout(c));
    TRY(rebuild(c, due, from, false));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    c->pending_from = 0x7fffffff;
    c->pending_due.clear();
    return SIMP_OK;
}

// Before a step: the pending admissions, and a compaction once retired
// basins hold a quarter of the batch's particles.
int flush_for_step(simp_ctx *c) { return flush_batch(c, c->zombie_n > 0 && 4 * c->zombie_n >= c->n); }

int reset_all(simp_ctx *c) {
    for (InstHost &h : c->insts) h = InstHost{};
    c->n = 0;
    c->nb = 0;
    return SIMP_OK;
}

int read_scalars(simp_ctx *c) {
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc_host, c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    return SIMP_OK;
}

int read_inst(simp_ctx *c, int slot, Inst *out) {
    SIMP_CUDA(c, cudaMemcpyAsync(out, c->inst_dev + slot, sizeof(Inst), cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
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

int get_instance_state(simp_ctx *c, int slot, double *x, double *vx, double *mass, double *rho, double *hsml,
                       double *A, double *h, double *t) {
    const InstHost &ih = c->insts[slot];
    const int nk = ih.n;
    const size_t N = (size_t)nk;
    cudaStream_t s = c->stream;
    double *stage = c->tmp;  // 9 n_k doubles
    k_pack_state<<<nblk(c->n, kB), kB, 0, s>>>(c->n, slot, ih.id_base, nk, c->pinst, c->id, c->s0, stage);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    struct Out { double *dst; size_t off, len; } outs[] = {
        {x, 0, 2 * N}, {vx, 2 * N, 2 * N}, {mass, 4 * N, N}, {rho, 5 * N, N},
        {hsml, 6 * N, N}, {A, 7 * N, N}, {h, 8 * N, N}};
    for (const Out &o : outs)
        if (o.dst)
            SIMP_CUDA(c, cudaMemcpyAsync(o.dst, stage + o.off, sizeof(double) * o.len, cudaMemcpyDeviceToHost, s));
    Inst I{};
    SIMP_CUDA(c, cudaMemcpyAsync(&I, c->inst_dev + slot, sizeof(Inst), cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    if (t) *t = I.t;
    return SIMP_OK;
}

// One step of the selected integrator.  With profiling on, external event
// records between the kernels time each one.
void enqueue_step(simp_ctx *c, bool diag, bool prof) {
    auto mark = [&](int k) {
        if (prof) cudaEventRecordWithFlags(c->prof_ev[k], c->stream, cudaEventRecordExternal);
    };
    // continuity density (den_alg 2) and Benz hsml (sle 1) add a density-rate
    // pass after an update (timed with the stress pass before it)
    // (and so does the Monaghan time step with artificial viscosity, whose
    // divergence takes the updated velocities)
    const bool den2 = c->prm.den_alg == 2, benz = c->prm.sle == 1;
    const bool tsdiv = c->prm.tse == 1 && c->prm.artificial_visc;
    // summation density (den_alg 1, density.f90:41-100) replaces the
    // update's density by a pass over the right-hand side's pairs with the
    // masses and densities of the reference's call; its last call of the
    // step also does the tail above
    const bool den1 = c->prm.den_alg == 1;
    State &s0 = c->s0, &s1 = c->s1;
    mark(0);
    if (c->prm.int_algorithm == 1) {
        // euler_scheme (time_integration.f90:86-148): one right-hand side
        launch_kinematic(c, s0, diag);
        launch_regularize(c, s0);
        mark(1);
        launch_stress(c, s0, s0, EPI_EULER);
        if (den1) launch_sum_density(c, s0, s1, s0.m, s0.rho, s1.rho, true);         // :128
        else if (den2 || benz || tsdiv) launch_density_rate(c, s0, s1, den2 ? 2 : 0, true);
        mark(2);
        launch_copy_s1_to_s0(c);
        mark(3);
        mark(4);
    } else {
        // predictor_corrector (:155-282) or leapfrog_scheme (:289-391): the
        // same first half step, a different final update
        const bool leap = c->prm.int_algorithm == 3;
        launch_kinematic(c, s0, false);
        launch_regularize(c, s0);
        mark(1);
        launch_stress(c, s0, s0, EPI_PREDICT);
        if (den1) launch_sum_density(c, s0, s1, s0.m, s0.rho, s1.rho, false);        // :217, :344
        else if (den2) launch_density_rate(c, s0, s1, 1, false);
        mark(2);
        launch_kinematic(c, s1, diag);
        launch_regularize(c, s1);
        mark(3);
        launch_stress(c, s1, s0, leap ? EPI_LEAP : EPI_CORRECT);
        if (den1 && leap) {
            launch_sum_density(c, s1, s0, s1.m, s1.rho, s0.rho, true);                // :372
        } else if (den1) {
            // two calls (:242 and :262) over the corrector's pairs, the
            // second reading the first's densities: the second writes
            // scratch (the half-step density, no longer read) and is
            // copied in after
            launch_sum_density(c, s1, s0, s1.m, s1.rho, s0.rho, false);
            launch_sum_density(c, s1, s0, s1.m, s0.rho, s1.rho, true);
            launch_commit_rho(c, s1.rho, s0);
        } else if (leap ? (den2 || benz || tsdiv) : (benz || tsdiv)) {
            launch_density_rate(c, s1, s0, (leap && den2) ? 2 : 0, true);
        }
        mark(4);
    }
    launch_step_finish(c);
    mark(5);
}

int ensure_graph(simp_ctx *c, bool diag) {
    const bool prof = c->profile;
    const bool same_kind = c->step_graph && c->graph_diag == diag && c->graph_profiled == prof;
    if (same_kind && !c->graph_stale) return SIMP_OK;
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
    if (same_kind) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(c->step_graph, g, &info) == cudaSuccess) {
            cudaGraphDestroy(g);
            c->graph_stale = false;
            return SIMP_OK;
        }
        cudaGetLastError();   // (a different topology: instantiate below)
    }
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    e = cudaGraphInstantiate(&c->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return simp_cuda_check(c, e, "cudaGraphInstantiate");
    c->graph_diag = diag;
    c->graph_profiled = prof;
    c->graph_stale = false;
    return SIMP_OK;
}

// A single basin whose hsml grew 5% past the size its grid was built for
// (sle = 1, 2) gets a new grid; until then the stencil radius covers it.
int maybe_regrid(simp_ctx *c, bool *done) {
    *done = false;
    if (c->max_inst != 1 || !c->insts[0].active || c->prm.sle == 0) return SIMP_OK;
    InstHost &h = c->insts[0];
    Inst I{};
    TRY(read_inst(c, 0, &I));
    if (!(I.hmax > 1.05 * h.grid_hmax)) return SIMP_OK;
    *done = true;
    std::vector<double> xy(2 * (size_t)c->n);
    TRY(download2(c, c->s0.x, c->s0.y, xy.data()));
    double xmin = xy[0], xmax = xy[0], ymin = xy[1], ymax = xy[1];
    for (int i = 0; i < c->n; ++i) {
        xmin = std::min(xmin, xy[2 * i]);
        xmax = std::max(xmax, xy[2 * i]);
        ymin = std::min(ymin, xy[2 * i + 1]);
        ymax = std::max(ymax, xy[2 * i + 1]);
    }
    for (int b = 0; b < h.nb; ++b) {
        xmin = std::min(xmin, h.xb[2 * b]);
        xmax = std::max(xmax, h.xb[2 * b]);
        ymin = std::min(ymin, h.xb[2 * b + 1]);
        ymax = std::max(ymax, h.xb[2 * b + 1]);
    }
    size_inst_grid(c, h, xmin, xmax, ymin, ymax, I.hmax);
    TRY(layout(c));
    TRY(rebuild(c, mask_of(0), c->n, false));
    h.steps_since_sort = 0;
    return SIMP_OK;
}

int check_after(simp_ctx *c) {
    if (const unsigned f = take_bounds_flags())
        return simp_fail(c, SIMP_ERR_BOUNDS, "device index check failed (sites " + std::to_string(f) +
                                                 ": 1 neighbour, 2 cell, 4 sort slot, 8 tile slot)");
    const Scalars &s = *c->sc_host;
    if ((s.flags & FLAG_NONFINITE) && c->max_inst == 1)   // batches flag the basin instead
        return simp_fail(c, SIMP_ERR_NONFINITE, "non-finite particle state after a step");
    if (s.maxip > c->prm.max_ind_int)
        return simp_fail(c, SIMP_ERR_IND_INT,
                         "Particle are too close to each other, this can lead to memory issue. Please "
                         "allow a higher maximum number of interaction for a single particle. "
                         "(nnps.f90:660-668)");
    return SIMP_OK;
}

int create(const simp_params *params, int32_t maxn, int32_t maxnb, int32_t max_inst, simp_ctx **out) {
    if (!out) return SIMP_ERR_BADARG;
    *out = nullptr;
    if (!params || maxn < 1 || maxnb < 0 || max_inst < 1 || max_inst > kMaxSlots) return SIMP_ERR_BADARG;
    simp_ctx *c = new simp_ctx();
    *out = c;   // on failure the caller can read last_error, then destroy
    c->prm = *params;
    TRY(check_params(c, c->prm, max_inst > 1));
    c->maxn = maxn;
    c->maxnb = std::max(maxnb, 1);
    c->max_inst = max_inst;
    c->id_stride = (max_inst > 1) ? (1 << kIdShift) : 0;
    c->insts.assign(max_inst, InstHost{});
    cudaGetDevice(&c->device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return simp_fail(c, SIMP_ERR_CUDA, "cudaStreamCreate failed (no usable CUDA device?)");
    const size_t M = (size_t)maxn, MB = (size_t)c->maxnb, MX = std::max(M, MB);
    double **d1[] = {&c->s0.x, &c->s0.y, &c->s0.vx, &c->s0.vy, &c->s0.m, &c->s0.rho, &c->s0.mor, &c->s0.h,
                     &c->s0.A, &c->s0.hs, &c->s1.x, &c->s1.y, &c->s1.vx, &c->s1.vy, &c->s1.rho,
                     &c->s1.mor, &c->s1.h, &c->s1.A, &c->xr, &c->yr, &c->xl, &c->yl,
                     &c->tau11, &c->tau12, &c->tau22, &c->div};
    for (double **p : d1) TRY(dalloc(c, p, M));
    if (c->prm.mass_from_area && c->prm.sle != 2) {
        TRY(dalloc(c, &c->mass1, M));
        c->s1.m = c->mass1;
    } else {
        c->s1.m = c->s0.m;
    }
    c->s1.hs = c->s0.hs;
    TRY(dalloc(c, &c->s0.hsf, M));
    c->s1.hsf = c->s0.hsf;
    // packed neighbour copies of both state sets, and the stress records
    for (State *st : {&c->s0, &c->s1}) {
        TRY(dalloc(c, &st->xy, M));
        TRY(dalloc(c, &st->vxy, M));
        TRY(dalloc(c, &st->pf, M));
        if (c->prm.precision == SIMP_PREC_MIXED) TRY(dalloc(c, &st->hmm, M));
        else TRY(dalloc(c, &st->mm, M));
    }
    if (c->prm.precision == SIMP_PREC_MIXED) {
        TRY(dalloc(c, &c->tau_q, M));
    } else {
        TRY(dalloc(c, &c->tau_a, M));
        TRY(dalloc(c, &c->tau_b, M));
    }
    TRY(dalloc(c, &c->nbr, (size_t)kMaxNbr * M));
    TRY(dalloc(c, &c->nbr_count, M));
    TRY(dalloc(c, &c->nbr_tmp, (size_t)kMaxNbr * M));
    TRY(dalloc(c, &c->pair_j, (size_t)kMaxPairs * M));
    TRY(dalloc(c, &c->pair_count, M));
    if (c->prm.precision == SIMP_PREC_MIXED) {
        // the mixed form keeps its pairs' kernel gradients for the stress
        // pass (measured: in the plain form the 16-byte records cost the
        // kinematic pass more than they save the stress pass)
        if (cudaMalloc(&c->pair_dw, (size_t)kDwRows * M * sizeof(float2)) != cudaSuccess)
            return simp_fail(c, SIMP_ERR_NOMEM, "device allocation failed");
    }
    TRY(dalloc(c, &c->diag, 9 * M));
    TRY(dalloc(c, &c->rates, 4 * M));
    if (c->max_inst == 1) {
        SIMP_CUDA(c, cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        SIMP_CUDA(c, cudaEventCreateWithFlags(&c->ev_graph, cudaEventDisableTiming));
        for (cudaEvent_t &e : c->ev_up) SIMP_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        TRY(dalloc(c, &c->early_stage, 2 * M));
    }
    if (c->prm.xsph_regularization || c->prm.artificial_visc) TRY(dalloc(c, &c->reg, 4 * M));
    TRY(dalloc(c, &c->cell, M));
    TRY(dalloc(c, &c->id, M));
    TRY(dalloc(c, &c->pinst, M));
    TRY(dalloc(c, &c->perm, M));
    TRY(dalloc(c, &c->tmp, 16 * MX));
    if (c->prm.sle == 1 && c->prm.den_alg != 2) TRY(dalloc(c, &c->drhodt, M));
    if (c->prm.den_alg == 1) TRY(dalloc(c, &c->k0, M));
    TRY(dalloc(c, &c->itmp, 5 * MX));
    TRY(dalloc(c, &c->bx, MB));
    TRY(dalloc(c, &c->by, MB));
    TRY(dalloc(c, &c->bm, MB));
    if (c->prm.bfa == 2) {
        TRY(dalloc(c, &c->bnx, MB));
        TRY(dalloc(c, &c->bny, MB));
    }
    TRY(dalloc(c, &c->bid, MB));
    TRY(dalloc(c, &c->binst, MB));
    TRY(dalloc(c, &c->bcell, MB));
    TRY(dalloc(c, &c->sc, 1));
    TRY(dalloc(c, &c->red_dev, (size_t)kRedBlocks * kRedVals));
    if (cudaMallocHost((void **)&c->red_host, sizeof(double) * kRedBlocks * kRedVals) != cudaSuccess)
        return simp_fail(c, SIMP_ERR_NOMEM, "pinned host allocation failed");
    TRY(dalloc(c, &c->pair_cnt, M + 1));
    TRY(dalloc(c, &c->bpair_cnt, MB + 1));
    TRY(dalloc(c, &c->inst_dev, (size_t)max_inst));
    if (cudaMallocHost((void **)&c->sc_host, sizeof(Scalars)) != cudaSuccess)
        return simp_fail(c, SIMP_ERR_NOMEM, "pinned host allocation failed");
    std::memset(c->sc_host, 0, sizeof(Scalars));
    SIMP_CUDA(c, cudaMemsetAsync(c->inst_dev, 0, sizeof(Inst) * (size_t)max_inst, c->stream));
    // scalars of an empty context
    Scalars &sc = *c->sc_host;
    sc.dt = c->prm.dt;
    const double inf = INFINITY;
    std::memcpy(&sc.acc_hmin, &inf, sizeof(double));
    std::memcpy(&sc.acc_dt, &inf, sizeof(double));
    sc.minip = 0x7fffffff;
    sc.list_scan = 1;
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc, c->sc_host, sizeof(Scalars), cudaMemcpyHostToDevice, c->stream));
    TRY(tiled_configure(c));
    TRY(layout(c));
    return SIMP_OK;
}

simp_forcing forcing_of(const simp_params &p) {
    simp_forcing f{};
    f.wind_kind = p.wind_kind;
    f.wind_u = p.wind_u;
    f.wind_v = p.wind_v;
    f.vortex_x = p.vortex_x;
    f.vortex_y = p.vortex_y;
    f.vortex_umax = p.vortex_umax;
    f.vortex_radius = p.vortex_radius;
    return f;
}

}  // namespace

namespace simp {

int complete_pending(simp_ctx *c) {
    if (!c->pending_check) return SIMP_OK;
    c->pending_check = false;
    TRY(read_scalars(c));
    return check_after(c);
}

// Flag words of the debug build's index checks (check.cuh), one reader per
// translation unit built with them.
static std::vector<unsigned (*)()> &bounds_readers() {
    static std::vector<unsigned (*)()> v;
    return v;
}
int register_bounds_reader(unsigned (*take)()) {
    bounds_readers().push_back(take);
    return 1;
}
unsigned take_bounds_flags() {
    unsigned f = 0u;
    for (auto take : bounds_readers()) f |= take();
    return f;
}


// bf_Wang reads b_normal (boundary_force.f90:146-147), which the reference
// sets with the walls (boundaries.f90:232-287): a basin with walls needs
// them before its first right-hand side.
int check_normals(simp_ctx *c) {
    if (c->prm.bfa != 2 || !c->prm.boundary_pressure) return SIMP_OK;
    const InstHost &h = c->insts[0];
    if (h.active && h.nb > 0 && h.bn.size() != 2 * (size_t)h.nb)
        return simp_fail(c, SIMP_ERR_STATE, "bfa = 2 needs the wall normals (simp_gpu_set_wall_normals)");
    return SIMP_OK;
}

// Device bytes per unit of maxn of a context with these parameters (the
// allocations of create() below, with room for its cell lists).
double bytes_per_particle(const simp_params &p, bool single_basin) {
    const bool mixed = p.precision == SIMP_PREC_MIXED;
    double b = 26 * 8.0;                                      // FP64 state sets and per-RHS fields
    if (p.mass_from_area && p.sle != 2) b += 8.0;             // half-step mass
    b += 4.0;                                                 // hsml in FP32
    b += 2 * (3 * 16.0 + 16.0);                               // packed neighbour copies, two sets
    b += mixed ? 16.0 : 32.0;                                 // stress records
    b += 2 * kMaxNbr * 4.0 + 4.0;                             // Verlet lists and their renaming copy
    b += kMaxPairs * 4.0 + 4.0;                               // pair lists
    b += mixed ? kDwRows * 8.0 : 0.0;                         // kept kernel gradients
    b += 9 * 8.0 + 4 * 8.0;                                   // diagnostics, rates
    if (p.sle == 1 && p.den_alg != 2) b += 8.0;               // Benz's kept drhodt
    if (p.xsph_regularization || p.artificial_visc) b += 4 * 8.0;   // regularisation terms
    if (p.den_alg == 1) b += 8.0;                             // kept kernel_zero
    b += 4 * 4.0 + 16 * 8.0 + 5 * 4.0 + 4.0;                  // sort keys, scratch
    b += 16.0 / kMinTileThreads + 48.0;                       // chunks, cell lists (worst case)
    if (single_basin) b += 2 * 8.0;                           // read-back stage of the fixed fields
    return b;
}

// Enqueues nsteps steps of every basin of the context on its stream without
// waiting for them (profiling mode waits step by step).
// A single basin's scheduled re-sort, replayed from a captured graph (one
// launch where the re-sort is some fifteen).  Its kernels capture the
// particle and cell counts, whether the Verlet lists are renamed, and the
// cell arrays, which a new layout can reallocate: a change of any of those
// captures it again.  Rebuild's host side for this case is that it counts
// one more re-sort (a single basin keeps all its particles, and the lists
// stay as valid as they were).
int sort_replayed(simp_ctx *c, const DueMask &due) {
    simp_ctx::SortKey k;
    k.n = c->n;
    k.total_cells = c->total_cells;
    k.keep_lists = c->lists_valid;
    k.cell_start = c->cell_start;
    k.scan_tmp = c->scan_tmp;
    if (!c->sort_graph || !(k == c->sort_key)) {
        if (c->sort_graph) cudaGraphExecDestroy(c->sort_graph);
        c->sort_graph = nullptr;
        const long long l0 = c->launches, r0 = c->rebuilds;
        const int n0 = c->n;
        const bool lv0 = c->lists_valid;
        cudaGraph_t g = nullptr;
        SIMP_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = rebuild(c, due, c->n, false);
        const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        const long long kernels = c->launches - l0;
        c->launches = l0;   // (the launch below counts them)
        c->rebuilds = r0;
        c->n = n0;
        c->lists_valid = lv0;
        if (rc != SIMP_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return rc != SIMP_OK ? rc : simp_cuda_check(c, e, "re-sort capture");
        }
        const cudaError_t ei = cudaGraphInstantiate(&c->sort_graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            c->sort_graph = nullptr;
            return simp_cuda_check(c, ei, "cudaGraphInstantiate (re-sort)");
        }
        c->sort_kernels = kernels;
        c->sort_key = k;
    }
    SIMP_CUDA(c, cudaGraphLaunch(c->sort_graph, c->stream));
    c->launches += c->sort_kernels;
    c->rebuilds += 1;
    return SIMP_OK;
}

int step_enqueue(simp_ctx *c, int nsteps) {
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "step before set_state");
    TRY(complete_pending(c));   // (this step resets the statistics those steps left)
    cudaStream_t s = c->stream;
    TRY(flush_for_step(c));
    if (c->n == 0 || nsteps == 0) return SIMP_OK;   // (an empty batch)
    TRY(check_normals(c));
    // (a grid outgrown by hsml is re-made only at the basin's scheduled
    // sorts, so the results do not depend on how the steps are split into
    // calls; until then the stencil radius covers the larger hsml)
    bool regridded = false;
    launch_reset_stats(c);
    TRY(ensure_graph(c, c->keep_diag));
    if (c->graph_profiled && !c->sort_ev[0])
        for (auto &e : c->sort_ev) SIMP_CUDA(c, cudaEventCreate(&e));
    for (int st = 0; st < nsteps; ++st) {
        DueMask due{};
        bool any = false;
        for (int q = 0; q < c->max_inst; ++q) {
            InstHost &h = c->insts[q];
            if (h.active && !h.retired && h.steps_since_sort >= kSortEvery) {
                due.w[q >> 6] |= 1ull << (q & 63);
                h.steps_since_sort = 0;
                any = true;
            }
        }
        if (any) {
            if (c->graph_profiled) SIMP_CUDA(c, cudaEventRecord(c->sort_ev[0], s));
            TRY(maybe_regrid(c, &regridded));   // hsml grew past the grid (sle = 2)
            if (regridded) TRY(ensure_graph(c, c->keep_diag));
            else if (c->max_inst == 1 && c->pass_impl != SIMP_PASSES_TILED) TRY(sort_replayed(c, due));
            else TRY(rebuild(c, due, c->n, false));
            if (c->graph_profiled) {
                SIMP_CUDA(c, cudaEventRecord(c->sort_ev[1], s));
                SIMP_CUDA(c, cudaEventSynchronize(c->sort_ev[1]));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, c->sort_ev[0], c->sort_ev[1]);
                c->prof_ms[simp_ctx::kProfKernels] += ms;
            }
        }
        if (c->ev_graph) SIMP_CUDA(c, cudaEventRecord(c->ev_graph, s));
        cudaError_t e = cudaGraphLaunch(c->step_graph, s);
        if (e != cudaSuccess) return simp_cuda_check(c, e, "cudaGraphLaunch");
        c->launches += c->graph_kernels;
        c->lists_valid = true;
        for (InstHost &h : c->insts)
            if (h.active && !h.retired) {
                ++h.steps_since_sort;
                ++h.steps_done;
            }
        if (c->graph_profiled) {
            // timing mode: wait for this step and add up its kernel times
            e = cudaEventSynchronize(c->prof_ev[simp_ctx::kProfKernels]);
            if (e != cudaSuccess) return simp_cuda_check(c, e, "profile event");
            for (int k = 0; k < simp_ctx::kProfKernels; ++k) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, c->prof_ev[k], c->prof_ev[k + 1]);
                c->prof_ms[k] += ms;
            }
            c->prof_steps += 1;
        }
    }
    return SIMP_OK;
}

// Waits for the enqueued steps and checks the step's status.
int step_complete(simp_ctx *c, double *current_time, double *dt) {
    if (!c->have_state) return simp_fail(c, SIMP_ERR_STATE, "step before set_state");
    if (c->n == 0) {
        if (current_time) *current_time = 0.0;
        if (dt) *dt = c->prm.dt;
        return SIMP_OK;
    }
    TRY(read_scalars(c));   // (one wait: the scalars queue behind the steps)
    if (current_time) *current_time = c->sc_host->t;
    if (dt) *dt = c->sc_host->dt;
    return check_after(c);
}

int batch_slot_state(simp_ctx *c, int slot, double *x, double *vx, double *mass, double *rho, double *hsml,
                     double *A, double *h, double *t) {
    if (!c->insts[slot].active || c->insts[slot].retired) return simp_fail(c, SIMP_ERR_BADARG, "slot is free");
    TRY(flush_batch(c, false));
    return get_instance_state(c, slot, x, vx, mass, rho, hsml, A, h, t);
}

// set_state of a state that continues the resident basin: the same particle
// count and walls, the same hsml, no particle farther than one cell from
// where it was sorted, a finite resident state.  The values are written in
// place (k_continue_group, per upload group) and the sort, cell lists, Verlet lists and step
// graph stay.  Returns kFreshState, with the resident state overwritten or
// not, when the state does not qualify; the caller then sets it up from
// scratch.  Left out: Benz's kept drhodt (a fresh state zeroes it) and the
// Wang force's wall normals (a fresh state needs them set again).
constexpr int kFreshState = -1;   // (not a SIMP_ERR_* code)
int continue_state(simp_ctx *c, int n, const double *x, const double *vx, const double *mass, const double *rho,
                   const double *hsml, const double *A, const double *h, int nb, const double *xb,
                   const double *massb, double dt, double t) {
    const InstHost &ih = c->insts[0];
    if (!c->have_state || !ih.active || ih.n != n || ih.nb != nb || c->drhodt || c->prm.bfa == 2)
        return kFreshState;
    if (!x || !vx || !mass || !rho || !hsml || !A || !h || (nb > 0 && (!xb || !massb))) return kFreshState;
    if (nb > 0 && (std::memcmp(ih.xb.data(), xb, sizeof(double) * 2 * (size_t)nb) != 0 ||
                   std::memcmp(ih.massb.data(), massb, sizeof(double) * (size_t)nb) != 0))
        return kFreshState;
    cudaStream_t s = c->stream;
    const size_t N = (size_t)n;
    double *stage = c->tmp;
    const int rb = std::min(kRedBlocks, nblk(n, 256));
    NbrList nl;
    nl.nbr = c->nbr;
    nl.count = c->nbr_count;
    nl.xl = c->xl;
    nl.yl = c->yl;
    nl.stride = c->maxn;
    // the upload on the side stream (after whatever the context stream has
    // queued), each group's kernel on the context stream once its part is in
    struct Part { const double *src; size_t off, len; int group; } parts[] = {
        {x, 0, 2 * N, CG_POS}, {vx, 2 * N, 2 * N, CG_VEL}, {mass, 4 * N, N, -1}, {rho, 5 * N, N, CG_MASS},
        {hsml, 6 * N, N, CG_HSML}, {A, 7 * N, N, -1}, {h, 8 * N, N, CG_AH}};
    SIMP_CUDA(c, cudaEventRecord(c->ev_up[kContGroups], s));
    SIMP_CUDA(c, cudaStreamWaitEvent(c->side, c->ev_up[kContGroups], 0));
    for (const Part &p : parts) {
        SIMP_CUDA(c, cudaMemcpyAsync(stage + p.off, p.src, sizeof(double) * p.len, cudaMemcpyHostToDevice, c->side));
        if (p.group < 0) continue;
        SIMP_CUDA(c, cudaEventRecord(c->ev_up[p.group], c->side));
        SIMP_CUDA(c, cudaStreamWaitEvent(s, c->ev_up[p.group], 0));
        switch (p.group) {
            case CG_POS: k_continue_group<CG_POS><<<rb, 256, 0, s>>>(n, c->id, stage, c->s0, c->xr, c->yr, nl, c->red_dev); break;
            case CG_VEL: k_continue_group<CG_VEL><<<rb, 256, 0, s>>>(n, c->id, stage, c->s0, c->xr, c->yr, nl, c->red_dev); break;
            case CG_MASS: k_continue_group<CG_MASS><<<rb, 256, 0, s>>>(n, c->id, stage, c->s0, c->xr, c->yr, nl, c->red_dev); break;
            case CG_HSML: k_continue_group<CG_HSML><<<rb, 256, 0, s>>>(n, c->id, stage, c->s0, c->xr, c->yr, nl, c->red_dev); break;
            default: k_continue_group<CG_AH><<<rb, 256, 0, s>>>(n, c->id, stage, c->s0, c->xr, c->yr, nl, c->red_dev);
        }
        c->launches += 1;
    }
    SIMP_CUDA(c, cudaGetLastError());
    SIMP_CUDA(c, cudaMemcpyAsync(c->red_host, c->red_dev, sizeof(double) * kRedVals * rb, cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc_host, c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    // v: [0] invalid values, [1] changed hsml, [2] d2 since the sort, [3]
    // since the lists, [4] max |coordinate|, [5] max hsml, [6] -min hsml
    double v[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -INFINITY};
    for (int b = 0; b < rb; ++b) {
        const double *u = c->red_host + (size_t)b * kRedVals;
        v[0] += u[0] + u[7];
        v[1] += u[1];
        for (int q = 2; q < 7; ++q) v[q] = std::max(v[q], u[q]);
    }
    const Scalars &sc = *c->sc_host;
    if (v[0] > 0.0 || v[1] > 0.0 || sc.flags != 0 || !(v[2] <= ih.I.cs * ih.I.cs)) return kFreshState;
    // a fresh state would take max_hsml from its own largest hsml: the run
    // continues only if that gives the physics constants in use
    const double max_hsml = (c->prm.max_hsml > 0.0) ? c->prm.max_hsml : v[5] * 10.0;   // initialize.f90:191
    const Phys P = make_phys(c->prm, max_hsml);
    if (std::memcmp(&P, &c->phys, sizeof(Phys)) != 0) return kFreshState;
    k_continue_finish<<<1, 1, 0, s>>>(c->sc, c->inst_dev, dt, t, v[2], v[3], v[4], c->prm.sle != 0 ? 1 : 0);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    // (a set state starts the kept kernel_zero again, initialize.f90:60)
    if (c->k0) SIMP_CUDA(c, cudaMemsetAsync(c->k0, 0, sizeof(double) * (size_t)c->maxn, s));
    return SIMP_OK;
}

}  // namespace simp

extern "C" {

const char *simp_gpu_version(void) { return "simp_b200 0.2 (sm_100a)"; }

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
    p->zeta_max = 0.0;   // data_variables.f90:154 declares them without a value
    p->eta_max = 0.0;
    p->phi = 45.0;       // data_variables.f90:159
    p->xi = (double)0.5225f;   // default-real literals (data_variables.f90:158, 175)
    p->Y = 1.0e9;
    p->nu = (double)0.3f;
    p->artificial_visc = 0;    // globals.f90:180-187
    p->xsph_regularization = 0;
    p->art_visc_alg = 1;       // globals.f90:103
    p->alpha_pi = 1.0;         // data_variables.f90:171-173
    p->beta_pi = 2.0;
    p->chi = (double)0.3f;
}

int32_t simp_gpu_create(const simp_params *params, int32_t maxn, int32_t maxnb, simp_ctx **out) {
    return create(params, maxn, maxnb, 1, out);
}

int32_t simp_gpu_create_batch(const simp_params *params, int32_t maxn, int32_t maxnb, int32_t max_instances,
                              simp_ctx **out) {
    return create(params, maxn, maxnb, max_instances, out);
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
    SIMP_RANGE("simp_gpu_set_state");
    if (!c->stream) return simp_fail(c, SIMP_ERR_STATE, "context was not created successfully");
    if (c->max_inst != 1) return simp_fail(c, SIMP_ERR_BADARG, "set_state is for single-basin contexts; use simp_gpu_batch_add");
    if (ntotal > c->maxn)
        return simp_fail(c, SIMP_ERR_MAXN,
                         "Resolution desired too high, the number of particles generated is higher "
                         "than the maximum allowed. (initialize.f90:156-163)");
    if (ntotalb > c->maxnb)
        return simp_fail(c, SIMP_ERR_MAXN,
                         "The number of boundary particles generated is higher than the maximum "
                         "allowed. (boundaries.f90:296-303)");
    // (refused before anything changes: the resident state stays)
    if (ntotal < 1 || ntotalb < 0 || !x || !vx || !mass || !rho || !hsml || !A || !h ||
        (ntotalb > 0 && (!xb || !massb)))
        return simp_fail(c, SIMP_ERR_BADARG, "set_state: bad sizes or null arrays");
    c->pending_check = false;   // (a new state replaces what steps without outputs left)
    const int cont = simp::continue_state(c, ntotal, x, vx, mass, rho, hsml, A, h, ntotalb, xb, massb, dt,
                                          current_time);
    if (cont != simp::kFreshState) return cont;   // continued in place, or a CUDA error
    reset_all(c);
    c->have_state = false;
    Extents e{};
    TRY(stage_instance(c, ntotal, x, vx, mass, rho, hsml, A, h, ntotalb, xb, massb, &e));
    const double hmax = e.hmax, hmin = e.hmin;
    const double max_hsml = (c->prm.max_hsml > 0.0) ? c->prm.max_hsml : hmax * 10.0;  // initialize.f90:191
    c->phys = make_phys(c->prm, max_hsml);
    // global scalars of the run
    Scalars &sc = *c->sc_host;
    std::memset(&sc, 0, sizeof(Scalars));
    sc.dt = dt;
    sc.t = current_time;
    sc.hmin = hmin;
    sc.hmax = hmax;
    sc.bs = 2.0 * hmin;
    const double inf = INFINITY;
    std::memcpy(&sc.acc_hmin, &inf, sizeof(double));
    std::memcpy(&sc.acc_dt, &inf, sizeof(double));
    sc.minip = 0x7fffffff;
    sc.skin = list_skin(c, hmax);
    sc.list_scan = 1;
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc, c->sc_host, sizeof(Scalars), cudaMemcpyHostToDevice, c->stream));
    SIMP_CUDA(c, cudaMemsetAsync(c->inst_dev, 0, sizeof(Inst), c->stream));
    if (c->drhodt) SIMP_CUDA(c, cudaMemsetAsync(c->drhodt, 0, sizeof(double) * (size_t)c->maxn, c->stream));
    if (c->k0) SIMP_CUDA(c, cudaMemsetAsync(c->k0, 0, sizeof(double) * (size_t)c->maxn, c->stream));
    TRY(add_instance(c, 0, forcing_of(c->prm), e, ntotalb, xb, massb, current_time));
    c->have_state = true;
    return SIMP_OK;
}

int32_t simp_gpu_batch_add(simp_ctx *c, const simp_forcing *forcing, int32_t ntotal, const double *x,
                           const double *vx, const double *mass, const double *rho, const double *hsml,
                           const double *A, const double *h, int32_t ntotalb, const double *xb,
                           const double *massb, int32_t *slot) {
    if (!c || !forcing || !slot) return SIMP_ERR_BADARG;
    if (!c->stream) return simp_fail(c, SIMP_ERR_STATE, "context was not created successfully");
    auto free_slot = [&]() {
        for (int k = 0; k < c->max_inst; ++k)
            if (!c->insts[k].active) return k;
        return -1;
    };
    int q = free_slot();
    // retired basins still hold their slots and room until a compaction,
    // which an admission runs when it needs them, or once they make up a
    // quarter of the batch
    if ((q < 0 || c->n + (long long)ntotal > c->maxn || c->nb + (long long)ntotalb > c->maxnb ||
         4 * c->zombie_n >= c->n) && c->zombie_n > 0) {
        TRY(flush_batch(c, true));
        q = free_slot();
    }
    if (q < 0) return simp_fail(c, SIMP_ERR_MAXN, "no free slot in the batch");
    Extents e{};
    TRY(stage_instance(c, ntotal, x, vx, mass, rho, hsml, A, h, ntotalb, xb, massb, &e));
    if (!c->have_state) {
        // first basin: physics constants and the list skin
        const double hmax = e.hmax;
        c->phys = make_phys(c->prm, c->prm.max_hsml > 0.0 ? c->prm.max_hsml : 10.0 * hmax);
        TRY(read_scalars(c));
        c->sc_host->skin = list_skin(c, hmax);
        c->sc_host->dt = c->prm.dt;
        SIMP_CUDA(c, cudaMemcpyAsync(c->sc, c->sc_host, sizeof(Scalars), cudaMemcpyHostToDevice, c->stream));
    }
    TRY(add_instance(c, q, *forcing, e, ntotalb, xb, massb, 0.0));
    c->have_state = true;
    *slot = q;
    return SIMP_OK;
}

int32_t simp_gpu_set_wall_normals(simp_ctx *c, int32_t ntotalb, const double *b_normal) {
    if (!c) return SIMP_ERR_BADARG;
    if (c->max_inst != 1) return simp_fail(c, SIMP_ERR_BADARG, "set_wall_normals is for single-basin contexts");
    InstHost &h = c->insts[0];
    if (!c->have_state || !h.active) return simp_fail(c, SIMP_ERR_STATE, "set_wall_normals before set_state");
    if (ntotalb != h.nb || (ntotalb > 0 && !b_normal))
        return simp_fail(c, SIMP_ERR_BADARG, "set_wall_normals: ntotalb differs from the state's walls");
    h.bn.assign(b_normal, b_normal + 2 * (size_t)ntotalb);
    if (c->bnx) TRY(layout(c));
    return SIMP_OK;
}

int32_t simp_gpu_set_forcing(simp_ctx *c, const simp_forcing *f) {
    if (!c || !f) return SIMP_ERR_BADARG;
    if (c->max_inst != 1) return simp_fail(c, SIMP_ERR_BADARG, "set_forcing is for single-basin contexts");
    if (f->wind_kind != SIMP_WIND_UNIFORM && f->wind_kind != SIMP_WIND_VORTEX)
        return simp_fail(c, SIMP_ERR_BADARG, "unknown wind_kind");
    c->prm.wind_kind = f->wind_kind;
    c->prm.wind_u = f->wind_u;
    c->prm.wind_v = f->wind_v;
    c->prm.vortex_x = f->vortex_x;
    c->prm.vortex_y = f->vortex_y;
    c->prm.vortex_umax = f->vortex_umax;
    c->prm.vortex_radius = f->vortex_radius;
    InstHost &h = c->insts[0];
    if (h.active) {
        Inst &I = h.I;
        I.wind_kind = f->wind_kind;
        I.wind_u = f->wind_u;
        I.wind_v = f->wind_v;
        I.vortex_x = f->vortex_x;
        I.vortex_y = f->vortex_y;
        I.vortex_umax = f->vortex_umax;
        I.vortex_radius = f->vortex_radius;
        TRY(layout(c));
    }
    return SIMP_OK;
}

int32_t simp_gpu_batch_remove(simp_ctx *c, int32_t slot) {
    if (!c || slot < 0 || slot >= c->max_inst) return SIMP_ERR_BADARG;
    return remove_instance(c, slot);
}

int32_t simp_gpu_batch_get_state(simp_ctx *c, int32_t slot, double *x, double *vx, double *mass, double *rho,
                                 double *hsml, double *A, double *h, double *current_time) {
    if (!c || slot < 0 || slot >= c->max_inst) return SIMP_ERR_BADARG;
    if (!c->insts[slot].active || c->insts[slot].retired) return simp_fail(c, SIMP_ERR_BADARG, "slot is free");
    TRY(flush_batch(c, false));
    return get_instance_state(c, slot, x, vx, mass, rho, hsml, A, h, current_time);
}

int32_t simp_gpu_batch_info(simp_ctx *c, int32_t slot, int32_t *ntotal, int64_t *steps, int32_t *flags) {
    if (!c || slot < 0 || slot >= c->max_inst) return SIMP_ERR_BADARG;
    const InstHost &h = c->insts[slot];
    const bool live = h.active && !h.retired;
    if (ntotal) *ntotal = live ? h.n : 0;
    if (steps) *steps = h.steps_done;
    if (flags) {
        *flags = 0;
        if (live) {
            TRY(flush_batch(c, false));
            Inst I{};
            TRY(read_inst(c, slot, &I));
            *flags = I.flags;
        }
    }
    return SIMP_OK;
}

int32_t simp_gpu_get_state(simp_ctx *c, double *x, double *vx, double *mass, double *rho,
                           double *hsml, double *A, double *h, double *dt, double *current_time) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state || !c->insts[0].active) return simp_fail(c, SIMP_ERR_STATE, "get_state before set_state");
    SIMP_RANGE("simp_gpu_get_state");
    // after steps enqueued without outputs: the fields no step writes are
    // read back while the steps run (the side stream starts at the last
    // step's graph, after any re-sort), the others after them
    const bool mass_fixed = !c->mass1, hsml_fixed = c->prm.sle == 0;
    double *early_m = (c->pending_check && c->side && mass && mass_fixed) ? mass : nullptr;
    double *early_h = (c->pending_check && c->side && hsml && hsml_fixed) ? hsml : nullptr;
    if (early_m || early_h) {
        const int n = c->n;
        const size_t N = (size_t)n;
        SIMP_CUDA(c, cudaStreamWaitEvent(c->side, c->ev_graph, 0));
        k_pack_fields<<<nblk(n, kB), kB, 0, c->side>>>(n, c->insts[0].id_base, c->id, early_m ? c->s0.m : nullptr,
                                                        early_h ? c->s0.hs : nullptr, c->early_stage,
                                                        c->early_stage + N);
        c->launches += 1;
        SIMP_CUDA(c, cudaGetLastError());
        if (early_m)
            SIMP_CUDA(c, cudaMemcpyAsync(early_m, c->early_stage, sizeof(double) * N, cudaMemcpyDeviceToHost, c->side));
        if (early_h)
            SIMP_CUDA(c, cudaMemcpyAsync(early_h, c->early_stage + N, sizeof(double) * N, cudaMemcpyDeviceToHost,
                                         c->side));
    }
    // the rest in groups: each group's reorder on the context stream, its
    // copy on the side stream while the next group is reordered
    const int n = c->n, id_base = c->insts[0].id_base;
    const size_t N = (size_t)n;
    cudaStream_t s = c->stream;
    double *stage = c->tmp;   // [x,y | vx,vy | mass | rho | hsml | A | h], caller's order
    const double *m_src = (mass && !early_m) ? c->s0.m : nullptr, *hs_src = (hsml && !early_h) ? c->s0.hs : nullptr;
    struct Out { double *dst; size_t off, len; };
    struct Group { Out a, b; } groups[5] = {
        {{x, 0, 2 * N}, {nullptr, 0, 0}},
        {{vx, 2 * N, 2 * N}, {nullptr, 0, 0}},
        {{m_src ? mass : nullptr, 4 * N, N}, {rho, 5 * N, N}},
        {{hs_src ? hsml : nullptr, 6 * N, N}, {A, 7 * N, N}},
        {{h, 8 * N, N}, {nullptr, 0, 0}}};
    for (int g = 0; g < 5; ++g) {
        const Group &G = groups[g];
        if (!G.a.dst && !G.b.dst) continue;
        if (g == 0) {
            k_pack_pair<<<nblk(n, kB), kB, 0, s>>>(n, id_base, c->id, c->s0.x, c->s0.y, stage);
        } else if (g == 1) {
            k_pack_pair<<<nblk(n, kB), kB, 0, s>>>(n, id_base, c->id, c->s0.vx, c->s0.vy, stage + 2 * N);
        } else {
            const double *sa = g == 2 ? m_src : g == 3 ? hs_src : c->s0.h;
            const double *sb = g == 2 ? (rho ? c->s0.rho : nullptr) : g == 3 ? (A ? c->s0.A : nullptr) : nullptr;
            k_pack_fields<<<nblk(n, kB), kB, 0, s>>>(n, id_base, c->id, sa, sb, stage + G.a.off, stage + G.b.off);
        }
        c->launches += 1;
        SIMP_CUDA(c, cudaGetLastError());
        SIMP_CUDA(c, cudaEventRecord(c->ev_up[g], s));
        SIMP_CUDA(c, cudaStreamWaitEvent(c->side, c->ev_up[g], 0));
        for (const Out &o : {G.a, G.b})
            if (o.dst)
                SIMP_CUDA(c, cudaMemcpyAsync(o.dst, stage + o.off, sizeof(double) * o.len, cudaMemcpyDeviceToHost,
                                             c->side));
    }
    SIMP_CUDA(c, cudaMemcpyAsync(c->sc_host, c->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s));
    SIMP_CUDA(c, cudaStreamSynchronize(s));
    SIMP_CUDA(c, cudaStreamSynchronize(c->side));
    if (dt) *dt = c->sc_host->dt;
    if (current_time) *current_time = c->sc_host->t;
    if (c->pending_check) {   // the status of steps enqueued without outputs
        c->pending_check = false;
        return check_after(c);
    }
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
    if (!c->have_state || c->max_inst != 1) return simp_fail(c, SIMP_ERR_STATE, "get_diag needs a single basin with state");
    double *outs[9] = {eps11, eps12, eps22, zeta, eta, p, sig11, sig12, sig22};
    for (int k = 0; k < 9; ++k)
        if (outs[k]) TRY(download1(c, c->diag + (size_t)k * c->maxn, outs[k]));
    return SIMP_OK;
}

int32_t simp_gpu_write_output(simp_ctx *c, const char *folder) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state || c->max_inst != 1) return simp_fail(c, SIMP_ERR_STATE, "write_output needs a single basin with state");
    const InstHost &h = c->insts[0];
    const size_t n = (size_t)h.n;
    std::vector<double> xv(4 * n), f(5 * n), dg(9 * n);
    double t = 0.0;
    TRY(simp_gpu_get_state(c, xv.data(), xv.data() + 2 * n, f.data(), nullptr, f.data() + n, f.data() + 2 * n,
                           f.data() + 3 * n, nullptr, &t));
    double *d[9];
    for (int k = 0; k < 9; ++k) d[k] = dg.data() + (size_t)k * n;
    TRY(simp_gpu_get_diag(c, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8]));
    const int rc = simp_csv_append_snapshot(folder, h.n, h.nb, t, xv.data(), xv.data() + 2 * n, f.data(), d[5],
                                            f.data() + n, f.data() + 2 * n, f.data() + 3 * n, d[0], d[1], d[2],
                                            d[6], d[7], d[8]);
    if (rc) return simp_fail(c, rc, simp_csv_last_error());
    return SIMP_OK;
}

int32_t simp_gpu_nnps(simp_ctx *c, int32_t *nip, int32_t *p_i, int32_t *p_j, double *r_ij,
                      double *hsml_ij, int32_t cap, int32_t *bnip, int32_t *bp_i, int32_t *bp_j,
                      double *br_ij, int32_t bcap) {
    if (!c) return SIMP_ERR_BADARG;
    if (!c->have_state || c->max_inst != 1) return simp_fail(c, SIMP_ERR_STATE, "nnps needs a single basin with state");
    SIMP_RANGE("simp_gpu_nnps");
    TRY(export_pairs(c, nip, p_i, p_j, r_ij, hsml_ij, cap, bnip, bp_i, bp_j, br_ij, bcap));
    if (const unsigned f = take_bounds_flags())
        return simp_fail(c, SIMP_ERR_BOUNDS, "device index check failed (sites " + std::to_string(f) + ")");
    return SIMP_OK;
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
    if (!c->have_state || c->max_inst != 1) return simp_fail(c, SIMP_ERR_STATE, "single_step needs a single basin with state");
    SIMP_RANGE("simp_gpu_single_step");
    TRY(complete_pending(c));
    TRY(check_normals(c));
    cudaStream_t s = c->stream;
    k_set_time0<<<1, 1, 0, s>>>(c->sc, c->inst_dev, current_time);
    c->launches += 1;
    launch_reset_stats(c);
    launch_kinematic(c, c->s0, true);
    launch_regularize(c, c->s0);
    launch_stress(c, c->s0, c->s0, EPI_RATES);
    // the right-hand side's pair loop also sets the summation density's kept
    // kernel_zero (kernel.f90:503): the density itself goes to scratch
    if (c->k0) launch_sum_density(c, c->s0, c->s0, c->s0.m, c->s0.rho, c->tmp, false);
    SIMP_CUDA(c, cudaGetLastError());
    c->lists_valid = true;
    const size_t M = (size_t)c->maxn;
    // dx/dt: the velocities, or with XSPH what the rates epilogue wrote
    if (dxdt && c->reg && c->prm.xsph_regularization) TRY(download2(c, c->reg + 2 * M, c->reg + 3 * M, dxdt));
    else if (dxdt) TRY(download2(c, c->s0.vx, c->s0.vy, dxdt));
    if (dvxdt) TRY(download2(c, c->rates, c->rates + M, dvxdt));
    if (dhdt) TRY(download1(c, c->rates + 2 * M, dhdt));
    if (dAdt) TRY(download1(c, c->rates + 3 * M, dAdt));
    TRY(read_scalars(c));
    return check_after(c);
}

int32_t simp_gpu_sum_density(simp_ctx *c, double *rho_out) {
    if (!c || !rho_out) return SIMP_ERR_BADARG;
    if (!c->have_state || c->max_inst != 1) return simp_fail(c, SIMP_ERR_STATE, "sum_density needs a single basin with state");
    SIMP_RANGE("simp_gpu_sum_density");
    double *stage = c->tmp;
    TRY(sum_density(c, stage));
    SIMP_CUDA(c, cudaMemcpyAsync(rho_out, stage, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    if (const unsigned f = take_bounds_flags())
        return simp_fail(c, SIMP_ERR_BOUNDS, "device index check failed (sites " + std::to_string(f) + ")");
    return SIMP_OK;
}

// time_integration.f90:38-71 for nsteps iterations of every basin.  Each
// basin is re-sorted into its grid every kSortEvery of its own steps; in
// between the device-side stencil radius keeps the cell list exact.
int32_t simp_gpu_step(simp_ctx *c, int32_t nsteps, double *current_time, double *dt) {
    if (!c || nsteps < 0) return SIMP_ERR_BADARG;
    SIMP_RANGE("simp_gpu_step");
    TRY(simp::step_enqueue(c, nsteps));
    if (!current_time && !dt && c->max_inst == 1 && c->n > 0 && nsteps > 0) {
        // no outputs: return once enqueued; the next get_state or step
        // reads the status in its own wait
        c->pending_check = true;
        return SIMP_OK;
    }
    return simp::step_complete(c, current_time, dt);
}

int32_t simp_gpu_set_passes(simp_ctx *c, int32_t impl, int32_t threads, int32_t cap) {
    if (!c) return SIMP_ERR_BADARG;
    if (impl < SIMP_PASSES_GATHER || impl > SIMP_PASSES_GATHER_TWO)
        return simp_fail(c, SIMP_ERR_BADARG, "unknown pair-pass implementation");
    if (threads < kMinTileThreads || threads > 256 || threads % 32 != 0 || cap < 64 || cap % 4 != 0 ||
        cap > 32767)
        return simp_fail(c, SIMP_ERR_BADARG, "tile shape out of range");
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t need = std::max(tiled_smem_bytes(c->prm.precision, 0, cap, threads),
                                 tiled_smem_bytes(c->prm.precision, 1, cap, threads));
    if (optin > 0 && need + 1024 > (size_t)optin)
        return simp_fail(c, SIMP_ERR_BADARG, "tile shape exceeds the shared memory of a block");
    const bool rechunk = threads != c->tile_threads || impl != c->pass_impl;
    c->pass_impl = impl;   // (both keep the Verlet lists the same way)
    c->tile_threads = threads;
    c->tile_cap = cap;
    TRY(tiled_configure(c));
    if (rechunk && c->n > 0) build_chunks(c);
    invalidate_graph(c);
    SIMP_CUDA(c, cudaStreamSynchronize(c->stream));
    return SIMP_OK;
}

int32_t simp_gpu_get_passes(const simp_ctx *c, int32_t *impl, int32_t *threads, int32_t *cap) {
    if (!c) return SIMP_ERR_BADARG;
    if (impl) *impl = c->pass_impl;
    if (threads) *threads = c->tile_threads;
    if (cap) *cap = c->tile_cap;
    return SIMP_OK;
}

// One right-hand side at the current state (kinematic pass + stress pass in
// rates mode: no state changes), timed with events.
static int time_rhs(simp_ctx *c, int reps, double *ms) {
    cudaEvent_t e0, e1;
    SIMP_CUDA(c, cudaEventCreate(&e0));
    SIMP_CUDA(c, cudaEventCreate(&e1));
    launch_kinematic(c, c->s0, false);          // warm-up
    launch_regularize(c, c->s0);
    launch_stress(c, c->s0, c->s0, EPI_RATES);
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps; ++r) {
        launch_kinematic(c, c->s0, false);
        launch_regularize(c, c->s0);
        launch_stress(c, c->s0, c->s0, EPI_RATES);
    }
    cudaEventRecord(e1, c->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return simp_cuda_check(c, e, "autotune timing");
    *ms = (double)t / std::max(1, reps);
    return SIMP_OK;
}

int32_t simp_gpu_autotune(simp_ctx *c, int32_t reps, double *ms_best) {
    if (!c || reps < 1) return SIMP_ERR_BADARG;
    if (!c->have_state || c->n == 0) return simp_fail(c, SIMP_ERR_STATE, "autotune needs particles");
    TRY(flush_batch(c, true));
    struct Cand { int impl, threads, cap; };
    const Cand cands[] = {
        {SIMP_PASSES_TILED, 128, 512},  {SIMP_PASSES_TILED, 128, 768},  {SIMP_PASSES_TILED, 128, 1024},
        {SIMP_PASSES_TILED, 256, 768},  {SIMP_PASSES_TILED, 256, 1024}, {SIMP_PASSES_TILED, 256, 1536},
        {SIMP_PASSES_TILED, 64, 384},   {SIMP_PASSES_TILED, 64, 512},   {SIMP_PASSES_GATHER_ONE, 256, 1024},
        {SIMP_PASSES_GATHER_TWO, 256, 1024}};
    const Cand keep{c->pass_impl, c->tile_threads, c->tile_cap};
    Cand best = keep;
    double tbest = INFINITY;
    for (const Cand &k : cands) {
        if (simp_gpu_set_passes(c, k.impl, k.threads, k.cap) != SIMP_OK) continue;   // shape does not fit
        double t = 0.0;
        TRY(time_rhs(c, reps, &t));
        if (t < tbest) {
            tbest = t;
            best = k;
        }
    }
    TRY(simp_gpu_set_passes(c, best.impl, best.threads, best.cap));
    (void)keep;
    c->err.clear();
    if (ms_best) *ms_best = tbest;
    return SIMP_OK;
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
    for (int k = 0; k < n_kernels; ++k) ms[k] = (k <= simp_ctx::kProfKernels) ? c->prof_ms[k] : 0.0;
    if (steps_timed) *steps_timed = c->prof_steps;
    return SIMP_OK;
}

const char *simp_gpu_last_error(const simp_ctx *c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"
