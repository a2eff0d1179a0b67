// Shared device code of the two pair passes of one right-hand-side evaluation (single_step.f90:5-109)
// and the predictor-corrector update fused into the second pass's epilogue.
//
// Kinematic pass (single_step.f90:50-84 + internal_stress.f90:20-42), per
// particle i, in two phases:
//   1. candidate scan of the cell stencil with an FP32 prefilter and the
//      exact FP64 criterion for undecided candidates (neighbors.cuh); the
//      accepted neighbours go to a per-thread list in shared memory and to
//      the neighbour list in HBM that the stress pass reuses;
//   2. FP64 pair math over the dense list:
//        wdvx = (v_i - v_j) (x) grad W_ij            (kernel.f90:515-518)
//        div_i  -= m_j (wdvx1 + wdvx4)               (vector_divergence.f90:27)
//        grad_i -= m_j wdvx / rho_j                  (vector_gradient.f90:56-69)
//   then strain (single_step.f90:80-84), strength, bulk and shear viscosity,
//   replacement pressure and stress (bulk_viscosity.f90:65-76,
//   shear_viscosity.f90:57, eos.f90:141-147, stress_tensor.f90:31-39).
//   Writes tau = sigma / rho^2 and div.
//
// Stress pass (internal_stress.f90:103-137 stress_1, boundary_kernel.f90 +
// boundary_force.f90:74-84, wind_forcing.f90:35-51, water_drag.f90:35-53,
// single_step.f90:104-106) over the kinematic pass's neighbour list:
//   a_i = rho_i / (rho_ice h_i) sum_j m_j (tau_i + tau_j) . grad W_ij
//         - sum_walls F_b / rho_i + wind + water drag
//   followed by one of three epilogues: the rates (single_step), the
//   predictor half step (time_integration.f90:204-227) or the corrector and
//   final update (:343-388).
//
// Each pair is evaluated from both sides (gather form, no atomics on the
// accumulations); grad W is odd in dx so both sides see the same per-pair
// terms as the reference's scatter loop, summed in a different order.
//
// Two implementations share this file's helpers: passes.cu gathers each
// particle's neighbours from HBM over Verlet lists; tiled.cu stages chunks of
// particles with their cell halo in shared memory.
#pragma once

#include <cmath>
#include <cstddef>

#include "ctx.h"
#include "neighbors.cuh"

namespace simp {
namespace pass {

// per-thread list of a particle's pairs: the whole pair list of a particle
// with up to kMaxPairs pairs (then written out row by row), flushed when full
constexpr int kListSlots = kMaxPairs + 1;

// Pair arithmetic type T: double for the plain form, float for the mixed
// form.  Positions and velocities stay FP64; their differences are formed in
// FP64 and rounded to T, after which the kernel gradient and the pair sums
// run in T (compensated when T is float).
__device__ __forceinline__ double rsq(double v) { return rsqrt(v); }
__device__ __forceinline__ float rsq(float v) { return rsqrtf(v); }

// Sum of pair terms a * b: plain FP64, or FP32 with Kahan compensation.
// Every multiply-add of the pair arithmetic is an explicit fma, so the
// rounding does not depend on which products a compiler chooses to fuse
// (both pass implementations then give the same bits).
template <class T>
struct Sum {
    double s = 0.0;
    __device__ __forceinline__ void madd(double a, double b) { s = fma(a, b, s); }
    __device__ __forceinline__ double get() const { return s; }
};
template <>
struct Sum<float> {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void madd(float a, float b) {
        const float y = fmaf(a, b, -c);
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double get() const { return (double)s - (double)c; }
};

// Per-pair geometry and kernel gradient: dw = gfac * (dx, dy).
// r = s * rsqrt(s) and 1/hsml_ij from the particle's own 1/hsml when the two
// smoothing lengths are equal (then hsml_ij = hsml_i exactly).
template <class T>
struct PairGeom {
    T dx, dy, gfac, w;
};

// dx, dy: x_i - x_j (differences of the FP64 positions, rounded to T);
// hi, inv_hi, hj: the smoothing lengths in T (the FP32 copies in the mixed
// form).
template <class T, bool WANT_W, int SKF = 0>
__device__ __forceinline__ PairGeom<T> pair_geom(const Phys &P, T dx, T dy, T hi, T inv_hi, T hj) {
    PairGeom<T> g;
    g.dx = dx;
    g.dy = dy;
    const T s = fma(g.dx, g.dx, g.dy * g.dy);
    const T rs = rsq(s);
    const T r = s * rs;
    const T inv_h = (hj == hi) ? inv_hi : T(2) / (hi + hj);
    const T sh = (T)P.scale_h;
    const T shh = sh * inv_h;
    const T q = r * shh;
    T gq, w = 0;
    kernel_wg<T, WANT_W, SKF>(P.skf, q, shh, inv_h, &w, &gq);
    if (WANT_W) g.w = w;
    g.gfac = gq * shh * rs;
    return g;
}

// What a pass needs to decide the reference criterion for particle i.
struct PairCtx {
    double xi, yi, hi;
    float xif, yif, hif;
    float margin;
    bool use_f32;
    BinRule br;
    Grid g;                     // the particle's instance grid
    double hmax;                // instance bounds for the stencil radius
    unsigned long long dmax2_bits;
};

__device__ __forceinline__ PairCtx pair_ctx(const State &s, const Scalars *sc, const Inst &I,
                                            const int *cell_start, int i) {
    PairCtx p;
    p.xi = s.x[i];
    p.yi = s.y[i];
    p.hi = s.hs[i];
    const float4 f = s.pf[i];
    p.xif = f.x;
    p.yif = f.y;
    p.hif = f.z;
    p.margin = prefilter_margin(bitsd(sc->xabs_bits), I.hmin);
    p.use_f32 = p.margin < 0.25f;
    p.br = make_bin_rule(I.bs, p.xi, p.yi, I.hmax);
    p.g = inst_grid(I, cell_start);
    p.hmax = I.hmax;
    p.dmax2_bits = I.dmax2_bits;
    return p;
}

// The reference criterion for candidate j, decided exactly: FP32 prefilter,
// the FP64 test of nnps.f90:277-281 when undecided, then the bucket rule.
// (f: candidate j's packed FP32 copy, already loaded; read when p.use_f32)
__device__ __forceinline__ bool is_pair_with(const State &s, const PairCtx &p, int j, float4 f) {
    int dec = 2;
    if (p.use_f32) dec = prefilter(p.xif - f.x, p.yif - f.y, 0.5f * (p.hif + f.z), p.margin);
    if (dec == 0) return false;
    if (dec == 2 || p.br.on) {
        const double2 q = __ldg(&s.xy[j]);
        const double xj = q.x, yj = q.y;
        if (dec == 2) {
            double r;
            const double mh = __dmul_rn(__dadd_rn(p.hi, __ldg(&s.hs[j])), 0.5);
            if (!pair_test(__dsub_rn(p.xi, xj), __dsub_rn(p.yi, yj), mh, &r)) return false;
        }
        if (!bin_rule_ok(p.br, xj, yj)) return false;
    }
    return true;
}

__device__ __forceinline__ bool is_pair(const State &s, const PairCtx &p, int j) {
    return is_pair_with(s, p, j, p.use_f32 ? __ldg(&s.pf[j]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f));
}

// Visits the cell-stencil candidates of particle i (cell order).
template <class F>
__device__ __forceinline__ void for_stencil(const Grid &g, int i, int ci, int R, F &&f) {
    for_stencil_rows(g, ci, R, [&](int j0, int j1) {
        for (int j = j0; j < j1; ++j)
            if (j != i) f(j);
    });
}

// Every current pair of particle i: from its Verlet list when that list
// still holds every pair, else from its cell stencil.  The lists were all
// built at the same positions (xl, yl) with members within mhsml + skin; a
// current pair (i, j) was then at most mhsml + |dx_i| + |dx_j| apart, so i's
// list is complete while |dx_i| + max_j |dx_j| < skin.
template <class F>
__device__ __forceinline__ void for_each_current_pair(const State &s, const NbrList &nl, const Scalars *sc,
                                                      int i, int ci, const PairCtx &p, F &&on_pair) {
    const int cnt = nl.count[i];
    const double dxl = p.xi - nl.xl[i], dyl = p.yi - nl.yl[i];
    const double own = sqrt(dxl * dxl + dyl * dyl);
    const double all = sqrt(bitsd(sc->dlist2_bits));
    const bool valid = (own + all) * (1.0 + 1e-9) < sc->skin;
    if (cnt >= 0 && cnt <= kMaxNbr && valid) {
        for (int k = 0; k < cnt; ++k) {
            const int j = __ldg(&nl.nbr[(size_t)k * nl.stride + i]);
            if (!SIMP_IN_RANGE(j, 0, nl.n, SITE_NEIGHBOUR)) continue;
            if (is_pair(s, p, j)) on_pair(j);
        }
    } else {
        for_stencil(p.g, i, ci, stencil_radius(p.hmax, p.dmax2_bits, p.g, 0.0), [&](int j) {
            if (is_pair(s, p, j)) on_pair(j);
        });
    }
}

// The same, with the list candidates taken kBatch at a time: their list
// entries, then their FP32 copies are loaded together, so one wait covers a
// whole batch.  before_batch() runs ahead of each batch (at most kBatch
// pairs follow it) and ahead of each stencil candidate.
constexpr int kBatch = 4;
template <class B, class F>
__device__ __forceinline__ void for_each_current_pair_batched(const State &s, const NbrList &nl, const Scalars *sc,
                                                              int i, int ci, const PairCtx &p, B &&before_batch,
                                                              F &&on_pair) {
    const int cnt = nl.count[i];
    const double dxl = p.xi - nl.xl[i], dyl = p.yi - nl.yl[i];
    const double own = sqrt(dxl * dxl + dyl * dyl);
    const double all = sqrt(bitsd(sc->dlist2_bits));
    const bool valid = (own + all) * (1.0 + 1e-9) < sc->skin;
    if (cnt >= 0 && cnt <= kMaxNbr && valid) {
        for (int k0 = 0; k0 < cnt; k0 += kBatch) {
            before_batch();
            int jj[kBatch];
            float4 ff[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                jj[u] = (k0 + u < cnt) ? __ldg(&nl.nbr[(size_t)(k0 + u) * nl.stride + i]) : -1;
                if (jj[u] >= 0 && !SIMP_IN_RANGE(jj[u], 0, nl.n, SITE_NEIGHBOUR)) jj[u] = -1;
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                ff[u] = (jj[u] >= 0 && p.use_f32) ? __ldg(&s.pf[jj[u]]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int u = 0; u < kBatch; ++u)
                if (jj[u] >= 0 && is_pair_with(s, p, jj[u], ff[u])) on_pair(jj[u]);
        }
    } else {
        for_stencil(p.g, i, ci, stencil_radius(p.hmax, p.dmax2_bits, p.g, 0.0), [&](int j) {
            before_batch();
            if (is_pair(s, p, j)) on_pair(j);
        });
    }
}

// Per-neighbour scalars in the pair arithmetic type: the FP64 arrays for
// the plain form, the packed FP32 copies for the mixed form.
template <class T>
struct KinNb {
    T h, m, mor;
};
template <class T>
struct StressNb {
    T h, m, t11, t12, t22;
};
// Packed stress-pass neighbour records written by the kinematic pass:
// plain form (tau11, tau12), (tau22, m); mixed form (tau11, tau12, tau22, m).
struct TauRec {
    double2 *ta, *tb;   // plain form
    float4 *tq;         // mixed form
};

template <class T>
struct Nb;
template <>
struct Nb<double> {
    static __device__ __forceinline__ double h(const State &s, int j) { return s.hs[j]; }
    // hu: the basin's hsml where every particle has the same (then hsml is
    // not gathered), else negative
    static __device__ __forceinline__ KinNb<double> kin(const State &s, int j, double hu) {
        const double2 q = __ldg(&s.mm[j]);
        return {hu > 0.0 ? hu : __ldg(&s.hs[j]), q.x, q.y};
    }
    static __device__ __forceinline__ StressNb<double> stress(const State &s, const TauRec &t, int j, double hu) {
        const double2 a = __ldg(&t.ta[j]), b = __ldg(&t.tb[j]);
        return {hu > 0.0 ? hu : __ldg(&s.hs[j]), b.y, a.x, a.y, b.x};
    }
    static __device__ __forceinline__ StressNb<double> stress_rec(const TauRec &t, int j) {
        const double2 a = __ldg(&t.ta[j]), b = __ldg(&t.tb[j]);
        return {0.0, b.y, a.x, a.y, b.x};
    }
};
template <>
struct Nb<float> {
    static __device__ __forceinline__ float h(const State &s, int j) { return s.hsf[j]; }
    static __device__ __forceinline__ KinNb<float> kin(const State &s, int j, float) {
        const float4 q = __ldg(&s.hmm[j]);   // (hsml comes in the same record)
        return {q.x, q.y, q.z};
    }
    static __device__ __forceinline__ StressNb<float> stress(const State &s, const TauRec &t, int j, float hu) {
        const float4 q = __ldg(&t.tq[j]);
        return {hu > 0.0f ? hu : __ldg(&s.hsf[j]), q.w, q.x, q.y, q.z};
    }
    static __device__ __forceinline__ StressNb<float> stress_rec(const TauRec &t, int j) {
        const float4 q = __ldg(&t.tq[j]);
        return {0.0f, q.w, q.x, q.y, q.z};
    }
};

// Kinematic-pass pair terms (kernel.f90:515-518, vector_divergence.f90:27,
// vector_gradient.f90:56-69): sums of -div and of the velocity gradient.
template <class T>
struct KinSums {
    Sum<T> dv, g1, g2, g3, g4;
    // grad W_ij = (dwx, dwy)
    __device__ __forceinline__ void add(T dwx, T dwy, T dvx, T dvy, T mj, T mrj) {
        const T w2 = dvy * dwx, w3 = dvx * dwy, w4 = dvy * dwy;
        const T w1 = dvx * dwx;
        dv.madd(mj, fma(dvx, dwx, w4));
        g1.madd(mrj, w1);
        g2.madd(mrj, w2);
        g3.madd(mrj, w3);
        g4.madd(mrj, w4);
    }
};

// Stress-pass pair terms (internal_stress.f90:103-137): sum_j m_j grad W
// and sum_j m_j tau_j . grad W.
template <class T>
struct StressSums {
    Sum<T> sx, sy, tx, ty;
    __device__ __forceinline__ void add(T dwx, T dwy, T mj, T t11, T t12, T t22) {
        sx.madd(mj, dwx);
        sy.madd(mj, dwy);
        tx.madd(mj, fma(t11, dwx, t12 * dwy));
        ty.madd(mj, fma(t12, dwx, t22 * dwy));
    }
};

// Vector of two values of the pair arithmetic type (the per-pair kernel
// gradients kept for the stress pass, common.cuh: kDwRows).
template <class T>
struct Vec2;
template <>
struct Vec2<double> {
    using type = double2;
    static __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
};
template <>
struct Vec2<float> {
    using type = float2;
    static __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
};

struct KinArgs {
    State s;
    const int *cell_start;
    const Inst *inst;
    const int *pinst;      // instance of each particle
    const int *cell;
    Phys P;
    Scalars *sc;
    double *tau11, *tau12, *tau22, *div;
    TauRec rec;            // the stress pass's neighbour records (written here)
    void *dw;              // grad W per pair row (Vec2<T>), kDwRows rows of stride pl.stride
    double *diag;
    NbrList nl;
    PairList pl;
    int n, maxn;
    // tiled implementation
    const Chunk *chunks;
    const int *nchunks;
    int cap;               // halo particles that fit in shared memory
};

// Strain rates, rheology and stress of particle i from its velocity
// divergence dv and velocity gradient g (single_step.f90:80-84,
// internal_stress.f90:20-42): writes tau = sigma / rho^2, div and the
// optional diagnostics.
__device__ __forceinline__ void kin_rheology(const KinArgs &a, int i, double dv, double g1, double g2,
                                             double g3, double g4) {
    const State &s = a.s;
    const Phys &P = a.P;
    // strain rates, single_step.f90:80-84
    const double e11 = g1, e22 = g4, e12 = 0.5 * (g2 + g3);
    // rheology, internal_stress.f90:20-42
    const double hh = s.h[i], AA = s.A[i];
    const double em2 = 1.0 / (P.e * P.e);
    const double Pstr = P.P_star * hh * exp(-(P.c_eos * (1.0 - AA)));
    const double delta = sqrt(fma(fma(e11, e11, e22 * e22), 1.0 + em2,
                                  fma(4.0 * em2, e12 * e12, 2.0 * e11 * e22 * (1.0 - em2))));
    const double dcap = (fabs(delta) < P.delta_min) ? P.delta_min : delta;
    double zeta = 0.0, eta = 0.0, p = 0.0;
    if (P.viscosity) {
        p = Pstr;
        if (P.rheology == 2) {
            // Mohr-Coulomb, bulk_viscosity.f90:86-145 and shear_viscosity.f90:67-124
            const double root = sqrt(fma(e11 - e22, e11 - e22, 4.0 * (e12 * e12)));
            const double eps1 = 0.5 * ((e11 + e22) + root), eps2 = 0.5 * ((e11 + e22) - root);
            const double zero = 1.0e-18;
            double epsI = fabs(eps1 + eps2);
            if (epsI < zero) epsI = zero;
            zeta = 0.5 * p * (1.0 + P.k_t) / epsI;
            if (zeta > P.zeta_max * p) zeta = P.zeta_max * p;
            double epsII = eps1 - eps2;
            if (fabs(epsII) < zero) epsII = zero;
            eta = P.mu * (0.5 * p * (1.0 + P.k_t) - zeta * (eps1 + eps2)) / epsII;
            if (eta > P.eta_max * p) eta = P.eta_max * p;
        } else {
            // elliptical, bulk_viscosity.f90:65-76 and shear_viscosity.f90:57
            zeta = 0.5 * Pstr * (1.0 + P.k_t) / dcap;
            eta = zeta / (P.e * P.e);
        }
    }
    if (P.pressure_force) {   // eos.f90:20-31
        if (P.eos_alg == 3) {
            p = zeta * 2.0 * delta / (1.0 + P.k_t);           // Kreyscher :141-147
        } else if (P.eos_alg == 2) {
            // Gutfraind :96-104 (rho_0 = rho_ice, rho_max = 934)
            const double rho = s.rho[i];
            const double gamma = 1.9e5 * hh * exp(-20.0 * (1.0 - AA));
            p = gamma * (rho - P.rho_ice) / (934.0 - rho);
            if (p < 0.0) p = 0.0;
        } else {
            p = Pstr;                                         // Hibler :59
        }
    }
    const double ph = p * (1.0 - P.k_t) / 2.0;
    const double s11 = fma(zeta + eta, e11, fma(zeta - eta, e22, -ph));
    const double s12 = 2.0 * eta * e12;
    const double s22 = fma(zeta + eta, e22, fma(zeta - eta, e11, -ph));
    const double rho = s.rho[i];
    // stress_1 pairs sigma / rho^2 with m; stress_2 pairs sigma with m / rho
    // (internal_stress.f90:103-137, 146-219)
    const double ir2 = (P.pa_sph == 2) ? 1.0 : 1.0 / (rho * rho);
    const double mw = (P.pa_sph == 2) ? s.mor[i] : s.m[i];
    a.tau11[i] = s11 * ir2;
    a.tau12[i] = s12 * ir2;
    a.tau22[i] = s22 * ir2;
    if (a.rec.tq) {
        a.rec.tq[i] = make_float4((float)(s11 * ir2), (float)(s12 * ir2), (float)(s22 * ir2), (float)mw);
    } else {
        a.rec.ta[i] = make_double2(s11 * ir2, s12 * ir2);
        a.rec.tb[i] = make_double2(s22 * ir2, mw);
    }
    a.div[i] = dv;
    if (a.diag) {
        const size_t M = (size_t)a.maxn;
        a.diag[i] = e11;
        a.diag[M + i] = e12;
        a.diag[2 * M + i] = e22;
        a.diag[3 * M + i] = zeta;
        a.diag[4 * M + i] = eta;
        a.diag[5 * M + i] = p;
        a.diag[6 * M + i] = s11;
        a.diag[7 * M + i] = s12;
        a.diag[8 * M + i] = s22;
    }
}

struct StressArgs {
    State rhs;     // state the right-hand side is evaluated at
    State base;    // step-start state (own values for the integrator)
    State out;     // state written by the epilogue
    const int *cell_start;
    Inst *inst;
    const int *pinst;
    const int *cell;
    const double *bx, *by, *bm;
    const double *bnx, *bny;   // wall normals (bfa = 2)
    const int *bstart;
    int nb;
    Phys P;
    Scalars *sc;
    const double *tau11, *tau12, *tau22, *div;
    TauRec rec;
    const void *dw;
    NbrList nl;
    PairList pl;
    double *rates;
    // regularisation terms of this right-hand side (k_regularize), 4 maxn:
    // the artificial-viscosity acceleration (x, y) and the XSPH sum (x, y),
    // which a rates epilogue replaces by dx/dt; null when both are off
    double *reg;
    const double *xr, *yr;
    double *hs_next;
    int n, maxn, mode;
    // tiled implementation
    const Chunk *chunks;
    const int *nchunks;
    int cap;
};

// Max of a per-instance 64-bit field over the lanes of a warp: one atomic per
// warp when the warp holds a single instance (the common case: instances are
// contiguous in cell order), one per lane otherwise.
__device__ __forceinline__ void inst_max_u64(Inst *inst, int k, size_t field, unsigned long long v) {
    const unsigned mask = __match_any_sync(0xffffffffu, k);
    if (mask == 0xffffffffu) {
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
            v = (t > v) ? t : v;
        }
        if ((threadIdx.x & 31) != 0) return;
    }
    atomicMax(reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(&inst[k]) + field), v);
}

// Block-wide max / min folded into one device atomic per block (the
// same-address atomics of every warp would serialise in L2).  Called by all
// threads of the block at the same point.
template <bool MAX>
__device__ __forceinline__ void block_reduce_u64(unsigned long long *dst, unsigned long long v) {
    __shared__ unsigned long long part[32];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = MAX ? (t > v ? t : v) : (t < v ? t : v);
    }
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = MAX ? (part[w] > v ? part[w] : v) : (part[w] < v ? part[w] : v);
        if (MAX) atomicMax(dst, v); else atomicMin(dst, v);
    }
    __syncthreads();
}
__device__ __forceinline__ void warp_max_u64(unsigned long long *dst, unsigned long long v) {
    block_reduce_u64<true>(dst, v);
}
__device__ __forceinline__ void warp_min_u64(unsigned long long *dst, unsigned long long v) {
    block_reduce_u64<false>(dst, v);
}
__device__ __forceinline__ void warp_max_i32(int *dst, int v) {
    __shared__ int part[32];
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = max(v, part[w]);
        atomicMax(dst, v);
    }
    __syncthreads();
}

// The per-step bounds of the stress pass in one block-wide reduction (a warp
// shuffle per value, one barrier, one atomic per value and block):
// maxip (max), the list displacement (max), max |coordinate| (max), the next
// hsml minimum and maximum, and the VP time step (min).  Values whose bit in
// `active` is clear are skipped.  Every thread of the block calls it.
constexpr int kBounds = 6;
__device__ __forceinline__ void block_bounds(Scalars *sc, unsigned active, unsigned long long (&v)[kBounds]) {
    __shared__ unsigned long long part[32][kBounds];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kBounds; ++q) {
        if (!((active >> q) & 1u)) continue;
        const bool mn = (q == 3 || q == 5);
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, v[q], o);
            v[q] = mn ? (t < v[q] ? t : v[q]) : (t > v[q] ? t : v[q]);
        }
        if (lane == 0) part[w][q] = v[q];
    }
    __syncthreads();
    const int q = threadIdx.x;
    if (q < kBounds && ((active >> q) & 1u)) {
        const bool mn = (q == 3 || q == 5);
        unsigned long long r = part[0][q];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            const unsigned long long t = part[k][q];
            r = mn ? (t < r ? t : r) : (t > r ? t : r);
        }
        switch (q) {
            case 0: atomicMax(&sc->maxip, (int)r); break;
            case 1: atomicMax(&sc->dlist2_bits, r); break;
            case 2: atomicMax(&sc->xabs_bits, r); break;
            case 3: atomicMin(&sc->acc_hmin, r); break;
            case 4: atomicMax(&sc->acc_hmax, r); break;
            default: atomicMin(&sc->acc_dt, r); break;
        }
    }
}

// The last block of a stress pass to finish decides whether the next
// kinematic pass rebuilds the Verlet lists: when the fastest particle moved
// 3/4 of the skin since they were built (lists are then complete only for
// particles that moved less than skin / 4), or when hsml changes (sle 1, 2).
// Threadfence reduction; no block waits on another.  Every block of the
// grid calls it once, with all its threads.
__device__ __forceinline__ void lists_block_done(const StressArgs &a) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&a.sc->blocks_done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const double dl = sqrt(bitsd(atomicAdd(&a.sc->dlist2_bits, 0ull)));
        const bool stale = (a.P.sle != 0) || !(dl < 0.75 * a.sc->skin);
        a.sc->list_scan = stale ? 1 : 0;
        a.sc->blocks_done = 0u;
    }
}

// Everything of the stress pass after the pair sums S = sum_j m_j grad W_ij
// and T = sum_j m_j tau_j . grad W_ij of particle i: internal force, walls,
// drag, rates and the integrator epilogue with the bounds reductions.
// Called by every thread of the block (dead lanes with live = false).
// `lists`: the Verlet-list implementation (displacement since the lists
// were built, and the last block's rebuild decision).
template <int SKF>
__device__ __forceinline__ void stress_finish(const StressArgs &a, int i, bool live, int ki, const Inst &I,
                                              bool dead, double xi, double yi, double hi, int ci, double Sx,
                                              double Sy, double Tx, double Ty, int cnt, bool lists) {
    const State &s = a.rhs;
    const Phys &P = a.P;
    const double rho = s.rho[i], hh = s.h[i], AA = s.A[i], mi = s.m[i];
    const double fi = (P.pa_sph == 2) ? 1.0 / P.rho_ice / hh : rho / P.rho_ice / hh;
    double ax = fi * fma(a.tau11[i], Sx, fma(a.tau12[i], Sy, Tx));
    double ay = fi * fma(a.tau12[i], Sx, fma(a.tau22[i], Sy, Ty));
    // boundary force, boundary_kernel.f90:5-45 calling boundary_force.f90
    // once per wall pair (bfa 1 bf_Monaghan :38-102, 2 bf_Wang :109-176,
    // 3 bf_Marquis :183-225)
    const double vxi = s.vx[i], vyi = s.vy[i];
    if ((P.boundary_pressure || P.boundary_friction) && a.nb > 0 && !dead) {
        const Grid g = inst_grid(I, a.cell_start);
        const double bl = I.b_length;
        const int Rb = wall_radius(I.dmax2_bits, g, bl);
        const BinRule bb = make_bin_rule(I.bs, xi, yi, bl);
        const double sh = (double)P.scale_h;
        const double dt = a.sc->dt;
        const double csnd = P.boundary_friction ? sound_speed(P, rho) : 0.0;
        double fx = 0.0, fy = 0.0;   // sum of F_b (Monaghan), applied as -F_b / rho
        double gx = 0.0, gy = 0.0;   // acceleration terms added as they are
        cnt += for_each_wall(a.bx, a.by, a.bstart, g, ci, Rb, bb, xi, yi, bl,
                             [&](int b, double bdx, double bdy, double d) {
                                 if (P.bfa == 1) {
                                     const double mb = a.bm[b];
                                     if (P.boundary_pressure) {
                                         const double bw = boundary_w<SKF>(P, d, hi);
                                         const double coef = P.kappa_n * bw * 2.0 * mb / ((mi + mb) * (d * d));
                                         fx += coef * bdx;
                                         fy += coef * bdy;
                                     }
                                     if (P.boundary_friction) {   // :85-100
                                         const double t = boundary_fdwdq<SKF>(P, d, hi) / bl;
                                         const double bwx = -(t * (bdx / d) * sh), bwy = -(t * (bdy / d) * sh);
                                         const double v_r = vxi * bdx + vyi * bdy;
                                         const double pi_aj = P.kappa_t * csnd * v_r / d / rho;
                                         gx += (-1.0 * mb * pi_aj * bwx) / rho;
                                         gy += (-1.0 * mb * pi_aj * bwy) / rho;
                                     }
                                 } else if (P.bfa == 2) {
                                     if (P.boundary_pressure) {   // :146-172
                                         const double nx = a.bnx[b], ny = a.bny[b];
                                         const double v1 = nx * vxi + ny * vyi;
                                         double v2 = sqrt(vxi * vxi + vyi * vyi) - v1;
                                         const double F1 = mi * v1 / dt;
                                         double F2 = mi * v2 / dt;
                                         if (P.boundary_friction && fabs(v2) > fabs(P.xi * v1)) {
                                             v2 = v2 * P.xi * fabs(F1 / F2);
                                             F2 = mi * v2 / dt;
                                         }
                                         gx += F1 * nx + F2 * ny;
                                         gy += F1 * ny - F2 * nx;
                                     }
                                 } else if (!P.boundary_pressure && P.boundary_friction) {   // :212-222
                                     gx -= vxi * (1.0 - d / bl);
                                     gy -= vyi * (1.0 - d / bl);
                                 }
                             });
        ax -= fx / rho;
        ay -= fy / rho;
        ax += gx;
        ay += gy;
    }
    // drag, wind_forcing.f90:35-51 and water_drag.f90:35-53 (off at t <= 0)
    const double tnow = I.t;
    if (P.wind_force && tnow > 0.0) {
        double wu, wv;
        wind_at(I, xi, yi, &wu, &wv);
        const double ru = wu - vxi, rv = wv - vyi;
        const double k = P.c_wind * P.rho_air / (hh * P.rho_ice);
        ax += k * ru * fabs(ru);
        ay += k * rv * fabs(rv);
    }
    if (P.water_force && tnow > 0.0) {
        const double ru = P.current_u - vxi, rv = P.current_v - vyi;
        const double k = P.c_water * P.rho_water / (hh * P.rho_ice);
        ax += k * ru * fabs(ru);
        ay += k * rv * fabs(rv);
    }
    // regularisation, single_step.f90:99-101 (after the drag): the
    // artificial viscosity into dv/dt, the XSPH sum into dx/dt
    // (regularization.f90:93, then single_step.f90:106: dxdt = -chi xsph + v)
    double dxdt = vxi, dydt = vyi;
    if (a.reg) {
        const size_t M = (size_t)a.maxn;
        if (P.art_visc == 1 || P.art_visc == 2) {
            ax += a.reg[i];
            ay += a.reg[M + i];
        }
        if (P.xsph) {
            dxdt = -(P.chi * a.reg[2 * M + i]) + vxi;
            dydt = -(P.chi * a.reg[3 * M + i]) + vyi;
        }
    }
    // prognostic rates, single_step.f90:104-106
    const double dv = a.div[i];
    const double dhdt = -hh * dv / rho;
    const double dAdt = -AA * dv / rho;
    if (a.mode == EPI_RATES) {
        warp_max_i32(&a.sc->maxip, live ? cnt : 0);
        if (live) {
            const size_t M = (size_t)a.maxn;
            a.rates[i] = ax;
            a.rates[M + i] = ay;
            a.rates[2 * M + i] = dhdt;
            a.rates[3 * M + i] = dAdt;
            if (a.reg && P.xsph) {   // dx/dt in place of the XSPH sum
                a.reg[2 * M + i] = dxdt;
                a.reg[3 * M + i] = dydt;
            }
        }
        return;
    }
    const double dt = a.sc->dt;
    const State &b = a.base;
    const double x0 = b.x[i], y0 = b.y[i], vx0 = b.vx[i], vy0 = b.vy[i], h0 = b.h[i], A0 = b.A[i];
    double xn, yn, vxn, vyn, hn, An;
    if (a.mode == EPI_PREDICT) {
        // time_integration.f90:207-215 (and the leap-frog's first half, :333-341)
        xn = x0 + dxdt * dt / 2.0;
        yn = y0 + dydt * dt / 2.0;
        vxn = vx0 + ax * dt / 2.0;
        vyn = vy0 + ay * dt / 2.0;
        hn = h0 + dhdt * dt / 2.0;
        An = A0 + dAdt * dt / 2.0;
    } else if (a.mode == EPI_EULER) {
        // euler_scheme, time_integration.f90:117-125
        xn = x0 + dxdt * dt;
        yn = y0 + dydt * dt;
        vxn = vx0 + ax * dt;
        vyn = vy0 + ay * dt;
        hn = h0 + dhdt * dt;
        An = A0 + dAdt * dt;
    } else if (a.mode == EPI_LEAP) {
        // leapfrog_scheme, time_integration.f90:361-369 (vx0: the step-start
        // velocity, dxdt: the half-step right-hand side's dx/dt)
        vxn = vx0 + ax * dt;
        vyn = vy0 + ay * dt;
        hn = h0 + dhdt * dt;
        xn = x0 + (vx0 + dxdt) * dt / 2.0;
        yn = y0 + (vy0 + dydt) * dt / 2.0;
        An = A0 + dAdt * dt;
    } else {
        // time_integration.f90:236-259
        const double x12 = x0 + dxdt * dt / 2.0, y12 = y0 + dydt * dt / 2.0;
        const double vx12 = vx0 + ax * dt / 2.0, vy12 = vy0 + ay * dt / 2.0;
        const double h12 = h0 + dhdt * dt / 2.0, A12 = A0 + dAdt * dt / 2.0;
        xn = 2.0 * x12 - x0;
        yn = 2.0 * y12 - y0;
        vxn = 2.0 * vx12 - vx0;
        vyn = 2.0 * vy12 - vy0;
        hn = 2.0 * h12 - h0;
        An = 2.0 * A12 - A0;
    }
    if (An > 1.0) An = 1.0;
    // the step's last update: hsml, VP time step (after the corrector, the
    // Euler step or the leap-frog's second half).  `tail_later`: a
    // density-rate pass (k_density_rate) follows and does them, because the
    // final density (con_density), Benz's hsml or the Monaghan time step
    // with artificial viscosity needs the updated velocities of the
    // neighbours.
    const bool final_update = a.mode == EPI_CORRECT || a.mode == EPI_EULER || a.mode == EPI_LEAP;
    const bool den2 = P.den_alg == 2, den1 = P.den_alg == 1;
    const bool tail_later = final_update && ((den2 && a.mode != EPI_CORRECT) || den1 || P.sle == 1 ||
                                             (P.tse == 1 && P.artificial_visc));
    double rhon;
    if (den1) {
        rhon = s.rho[i];   // the density of the call, until the summation pass replaces it
    } else if (!den2) {
        rhon = hn * P.rho_ice;                                // density.f90:192
    } else if (a.mode == EPI_CORRECT) {
        // time_integration.f90:242-266: drho/dt of the corrector's density
        // call (half-step velocities and pairs) is the negated divergence
        // sum of this right-hand side
        const double r0 = b.rho[i];
        const double r12 = r0 + (-dv) * dt / 2.0;
        rhon = 2.0 * r12 - r0;
    } else {
        rhon = b.rho[i];   // rho_1, until k_density_rate adds drho/dt dt
    }
    double mn = b.m[i];
    const double hs_old = b.hs[i];
    if (P.sle != 2 && P.mass_from_area) {                     // mass_evolution.f90:66-69
        const double ar = kPi * ((P.alpha * hs_old) * (P.alpha * hs_old));
        mn = P.rho_ice * An * hn * ar;
    }
    double hsn = hs_old;
    if (final_update && !tail_later && P.sle == 2) {          // smoothing_length.f90:136-142
        hsn = sqrt(mn / rhon) * (double)P.hsml_multiplicity;
        if (hsn > P.max_hsml) hsn = P.max_hsml;
    }
    // displacement since the instance's last sort, max per instance
    const double dxr = xn - a.xr[i], dyr = yn - a.yr[i];
    // (non-finite values stay out of these bounds: the basin is flagged below)
    double d2 = dxr * dxr + dyr * dyr;
    if (!live || !isfinite(d2)) d2 = 0.0;
    inst_max_u64(a.inst, ki, offsetof(Inst, dmax2_bits), dbits(d2));
    double dl2 = 0.0;
    if (lists) {
        const double dxl = xn - a.nl.xl[i], dyl = yn - a.nl.yl[i];
        dl2 = dxl * dxl + dyl * dyl;
        if (!live || !isfinite(dl2)) dl2 = 0.0;
    }
    // (dead lanes contribute neutral bounds: in place updates, the particle
    // they mirror may already have been written by its own thread)
    double xa = fmax(fabs(xn), fabs(yn));
    if (!live || !isfinite(xa)) xa = 0.0;
    const bool bad = !(isfinite(xn) && isfinite(yn) && isfinite(vxn) && isfinite(vyn) &&
                       isfinite(hn) && isfinite(An));
    if (live && bad) {
        atomicOr(&a.sc->flags, FLAG_NONFINITE);
        atomicOr(&a.inst[ki].flags, FLAG_NONFINITE);
    }
    if (live) {
        const State &o = a.out;
        const double morn = mn / rhon;
        o.x[i] = xn;
        o.y[i] = yn;
        o.vx[i] = vxn;
        o.vy[i] = vyn;
        o.h[i] = hn;
        o.A[i] = An;
        o.rho[i] = rhon;
        if (P.sle != 2 && P.mass_from_area) o.m[i] = mn;
        o.mor[i] = morn;
        const float hsf = (float)hs_old;
        o.xy[i] = make_double2(xn, yn);
        o.vxy[i] = make_double2(vxn, vyn);
        o.pf[i] = make_float4((float)xn, (float)yn, hsf, 0.0f);
        if (o.hmm) o.hmm[i] = make_float4(hsf, (float)mn, (float)morn, 0.0f);
        else o.mm[i] = make_double2(mn, morn);
        if (final_update && !tail_later && P.sle == 2) a.hs_next[i] = hsn;
    }
    // this step's bounds, one block-wide reduction
    const bool corr = final_update && !tail_later;
    unsigned active = 1u | (lists ? 2u : 0u) | 4u;
    unsigned long long v[kBounds] = {(unsigned long long)(live ? cnt : 0), dbits(dl2), dbits(xa), ~0ull, 0ull,
                                     ~0ull};
    if (corr && P.sle == 2) {                                   // smoothing_length.f90:136-142
        active |= 8u | 16u;
        if (live) {
            v[3] = dbits(hsn);
            v[4] = dbits(hsn);
        }
    }
    if (corr && P.tse != 0) {                                   // time_step.f90:20-26
        active |= 32u;
        if (live) v[5] = dbits(dt_candidate(P, hsn, ax * ax + ay * ay, rhon, 0.0));
    }
    if (tail_later && P.tse == 1 && live) a.rates[i] = ax * ax + ay * ay;   // for k_density_rate
    block_bounds(a.sc, active, v);
    if (lists) lists_block_done(a);
}

}  // namespace pass

// tiled.cu
void launch_kinematic_tiled(simp_ctx *c, const pass::KinArgs &a);
void launch_stress_tiled(simp_ctx *c, const pass::StressArgs &a);

}  // namespace simp
