// The two pair passes of one right-hand-side evaluation (single_step.f90:5-109)
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
//   predictor half step (time_integration.f90:314-338) or the corrector and
//   final update (:343-388).
//
// Each pair is evaluated from both sides (gather form, no atomics on the
// accumulations); grad W is odd in dx so both sides see the same per-pair
// terms as the reference's scatter loop, summed in a different order.
#include <cmath>

#include "ctx.h"
#include "neighbors.cuh"

namespace simp {

namespace {

constexpr int kBlock = 128;
// per-thread shared-memory list: the whole pair list of a particle with up
// to kMaxPairs pairs (then written out row by row), flushed when full
constexpr int kListSlots = kMaxPairs + 1;
// minimum resident blocks per SM (register caps 73 and 64): more warps in
// flight to hide the latency of the neighbour gathers
constexpr int kMinBlocksKin = 7;
constexpr int kMinBlocksStress = 8;

// Pair arithmetic type T: double for the plain form, float for the mixed
// form.  Positions and velocities stay FP64; their differences are formed in
// FP64 and rounded to T, after which the kernel gradient and the pair sums
// run in T (compensated when T is float).
__device__ __forceinline__ double rsq(double v) { return rsqrt(v); }
__device__ __forceinline__ float rsq(float v) { return rsqrtf(v); }

// Sum of pair terms: plain FP64, or FP32 with Kahan compensation.
template <class T>
struct Sum {
    double s = 0.0;
    __device__ __forceinline__ void add(double v) { s += v; }
    __device__ __forceinline__ double get() const { return s; }
};
template <>
struct Sum<float> {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add(float v) {
        const float y = v - c;
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

template <class T, bool WANT_W>
__device__ __forceinline__ PairGeom<T> pair_geom(const Phys &P, double xi, double yi, double hi, double inv_hi,
                                                 double xj, double yj, double hj) {
    PairGeom<T> g;
    g.dx = (T)(xi - xj);
    g.dy = (T)(yi - yj);
    const T s = g.dx * g.dx + g.dy * g.dy;
    const T rs = rsq(s);
    const T r = s * rs;
    const T inv_h = (T)((hj == hi) ? inv_hi : 2.0 / (hi + hj));
    const T sh = (T)P.scale_h;
    const T shh = sh * inv_h;
    const T q = r * shh;
    T gq;
    if (P.skf == SIMP_SKF_WENDLAND_C6) {
        const T factor = (T)(78.0 / (7.0 * kPi)) * (shh * shh);
        const T om = T(1) - q;
        const T om2 = om * om, om4 = om2 * om2;
        if (WANT_W) g.w = factor * (om4 * om4) * (((T(32) * q + T(25)) * q + T(8)) * q + T(1));
        gq = factor * (T(-22) * q * (om4 * om2 * om) * ((T(16) * q + T(7)) * q + T(1)));
    } else {
        const T factor = (T)(15.0 / (7.0 * kPi)) * (shh * shh);
        if (q <= T(1)) {
            if (WANT_W) g.w = factor * ((T)(2.0f / 3.0f) - q * q + T(0.5) * q * q * q);
            gq = factor * (T(-2) * q + T(1.5) * q * q);
        } else {
            const T u = T(2) - q;
            if (WANT_W) g.w = factor * ((T)(1.0f / 6.0f) * u * u * u);
            gq = factor * (T(-0.5) * u * u);
        }
    }
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
    p.xif = s.xf[i];
    p.yif = s.yf[i];
    p.hif = s.hsf[i];
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
__device__ __forceinline__ bool is_pair(const State &s, const PairCtx &p, int j) {
    int dec = 2;
    if (p.use_f32) dec = prefilter(p.xif - s.xf[j], p.yif - s.yf[j], 0.5f * (p.hif + s.hsf[j]), p.margin);
    if (dec == 0) return false;
    if (dec == 2 || p.br.on) {
        const double xj = s.x[j], yj = s.y[j];
        if (dec == 2) {
            double r;
            const double mh = __dmul_rn(__dadd_rn(p.hi, s.hs[j]), 0.5);
            if (!pair_test(__dsub_rn(p.xi, xj), __dsub_rn(p.yi, yj), mh, &r)) return false;
        }
        if (!bin_rule_ok(p.br, xj, yj)) return false;
    }
    return true;
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
    if (cnt <= kMaxNbr && valid) {
        for (int k = 0; k < cnt; ++k) {
            const int j = nl.nbr[(size_t)k * nl.stride + i];
            if (is_pair(s, p, j)) on_pair(j);
        }
    } else {
        for_stencil(p.g, i, ci, stencil_radius(p.hmax, p.dmax2_bits, p.g, 0.0), [&](int j) {
            if (is_pair(s, p, j)) on_pair(j);
        });
    }
}

struct KinArgs {
    State s;
    const int *cell_start;
    const Inst *inst;
    const int *pinst;      // instance of each particle
    const int *cell;
    Phys P;
    Scalars *sc;
    double *tau11, *tau12, *tau22, *div;
    double *diag;
    NbrList nl;
    PairList pl;
    int n, maxn;
};

template <class T>
__global__ void __launch_bounds__(kBlock, kMinBlocksKin) k_kinematic(KinArgs a) {
    __shared__ int s_list[kListSlots * kBlock];
    const int t = threadIdx.x;
    const int i = blockIdx.x * blockDim.x + t;
    if (i >= a.n) return;
    const State &s = a.s;
    const Phys &P = a.P;
    const Inst &I = a.inst[a.pinst[i]];
    // a basin whose state turned non-finite is not searched any more (its
    // stencil would span its whole grid); it is only carried until retired
    const bool dead = (I.flags & FLAG_NONFINITE) != 0;
    const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
    const double xi = pc.xi, yi = pc.yi, hi = pc.hi;
    const double vxi = s.vx[i], vyi = s.vy[i];
    const double inv_hi = 1.0 / hi;
    Sum<T> dvs, g1s, g2s, g3s, g4s;   // -div and the velocity gradient, negated
    int cnt = 0;       // entries in this thread's shared-memory list
    int npairs = 0;    // exact pairs found so far
    auto flush = [&]() {
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const int j = s_list[k * kBlock + t];
            const PairGeom<T> pg = pair_geom<T, false>(P, xi, yi, hi, inv_hi, s.x[j], s.y[j], s.hs[j]);
            const T dwx = pg.gfac * pg.dx, dwy = pg.gfac * pg.dy;
            const T dvx = (T)(vxi - s.vx[j]), dvy = (T)(vyi - s.vy[j]);
            const T w1 = dvx * dwx, w2 = dvy * dwx, w3 = dvx * dwy, w4 = dvy * dwy;
            const T mj = (T)s.m[j], mrj = (T)s.mor[j];
            dvs.add(mj * (w1 + w4));
            g1s.add(mrj * w1);
            g2s.add(mrj * w2);
            g3s.add(mrj * w3);
            g4s.add(mrj * w4);
        }
        cnt = 0;
    };
    auto on_pair = [&](int j) {
        s_list[cnt * kBlock + t] = j;
        ++npairs;
        if (++cnt == kListSlots) flush();   // more than kMaxPairs pairs: no pair list
    };
    if (a.sc->list_scan && i == 0) atomicExch(&a.sc->dlist2_bits, 0ull);
    if (dead) {
        if (a.sc->list_scan) {
            a.nl.count[i] = 0;
            a.nl.xl[i] = xi;
            a.nl.yl[i] = yi;
        }
    } else if (a.sc->list_scan) {
        // rebuild the Verlet list from the cell stencil: members are the
        // candidates not certainly beyond mhsml + skin (FP32, with margin)
        const double skin = a.sc->skin;
        const float skinf = (float)skin, grow = 1.0f + pc.margin;
        int total = 0;
        for_stencil(pc.g, i, a.cell[i], stencil_radius(pc.hmax, pc.dmax2_bits, pc.g, pc.hmax + skin), [&](int j) {
            const float dxf = pc.xif - s.xf[j], dyf = pc.yif - s.yf[j];
            const float lim = 0.5f * (pc.hif + s.hsf[j]) + skinf;
            if (dxf * dxf + dyf * dyf > lim * lim * grow) return;
            if (total < kMaxNbr) a.nl.nbr[(size_t)total * a.nl.stride + i] = j;
            ++total;
            if (is_pair(s, pc, j)) on_pair(j);
        });
        a.nl.count[i] = total;
        a.nl.xl[i] = xi;
        a.nl.yl[i] = yi;
    } else {
        for_each_current_pair(s, a.nl, a.sc, i, a.cell[i], pc, on_pair);
    }
    // the stress pass's pair list, one coalesced row per k
    if (npairs <= kMaxPairs)
        for (int k = 0; k < cnt; ++k) a.pl.pj[(size_t)k * a.pl.stride + i] = s_list[k * kBlock + t];
    a.pl.count[i] = npairs;
    flush();
    const double dv = -dvs.get();
    const double g1 = -g1s.get(), g2 = -g2s.get(), g3 = -g3s.get(), g4 = -g4s.get();
    // strain rates, single_step.f90:80-84
    const double e11 = g1, e22 = g4, e12 = 0.5 * (g2 + g3);
    // rheology, internal_stress.f90:20-42
    const double hh = s.h[i], AA = s.A[i];
    const double em2 = 1.0 / (P.e * P.e);
    const double Pstr = P.P_star * hh * exp(-(P.c_eos * (1.0 - AA)));
    const double delta = sqrt((e11 * e11 + e22 * e22) * (1.0 + em2) + 4.0 * em2 * (e12 * e12) +
                              2.0 * e11 * e22 * (1.0 - em2));
    const double dcap = (fabs(delta) < P.delta_min) ? P.delta_min : delta;
    double zeta = 0.0, eta = 0.0, p = 0.0;
    if (P.viscosity) {
        zeta = 0.5 * Pstr * (1.0 + P.k_t) / dcap;
        eta = zeta / (P.e * P.e);
        p = Pstr;
    }
    if (P.pressure_force) p = (P.eos_alg == 3) ? zeta * 2.0 * delta / (1.0 + P.k_t) : Pstr;
    const double ph = p * (1.0 - P.k_t) / 2.0;
    const double s11 = (zeta + eta) * e11 + (zeta - eta) * e22 - ph;
    const double s12 = 2.0 * eta * e12;
    const double s22 = (zeta + eta) * e22 + (zeta - eta) * e11 - ph;
    const double rho = s.rho[i];
    const double ir2 = 1.0 / (rho * rho);
    a.tau11[i] = s11 * ir2;
    a.tau12[i] = s12 * ir2;
    a.tau22[i] = s22 * ir2;
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
    const int *bstart;
    int nb;
    Phys P;
    Scalars *sc;
    const double *tau11, *tau12, *tau22, *div;
    NbrList nl;
    PairList pl;
    double *rates;
    const double *xr, *yr;
    double *hs_next;
    int n, maxn, mode;
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
    __shared__ unsigned long long part[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = MAX ? (t > v ? t : v) : (t < v ? t : v);
    }
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBlock / 32; ++w) v = MAX ? (part[w] > v ? part[w] : v) : (part[w] < v ? part[w] : v);
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
    __shared__ int part[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBlock / 32; ++w) v = max(v, part[w]);
        atomicMax(dst, v);
    }
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(kBlock, kMinBlocksStress) k_stress(StressArgs a) {
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i0 < a.n;
    const int i = live ? i0 : a.n - 1;   // dead lanes mirror the last particle for warp reductions
    const State &s = a.rhs;
    const Phys &P = a.P;
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const double inv_hi = 1.0 / hi;
    const int ci = a.cell[i];
    const int ki = a.pinst[i];
    const Inst &I = a.inst[ki];
    const bool dead = (I.flags & FLAG_NONFINITE) != 0;   // see k_kinematic
    Sum<T> Sxs, Sys, Txs, Tys;
    auto accumulate = [&](int j) {
        const PairGeom<T> pg = pair_geom<T, false>(P, xi, yi, hi, inv_hi, s.x[j], s.y[j], s.hs[j]);
        const T dwx = pg.gfac * pg.dx, dwy = pg.gfac * pg.dy;
        const T mj = (T)s.m[j];
        const T t11 = (T)a.tau11[j], t12 = (T)a.tau12[j], t22 = (T)a.tau22[j];
        Sxs.add(mj * dwx);
        Sys.add(mj * dwy);
        Txs.add(mj * (t11 * dwx + t12 * dwy));
        Tys.add(mj * (t12 * dwx + t22 * dwy));
    };
    int cnt = a.pl.count[i];
    if (cnt <= kMaxPairs) {
        // the kinematic pass of this right-hand side found the pairs
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) accumulate(a.pl.pj[(size_t)k * a.pl.stride + i]);
    } else if (dead) {
        cnt = 0;
    } else {
        cnt = 0;
        const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
        for_each_current_pair(s, a.nl, a.sc, i, ci, pc, [&](int j) {
            accumulate(j);
            ++cnt;
        });
    }
    const double Sx = Sxs.get(), Sy = Sys.get(), Tx = Txs.get(), Ty = Tys.get();
    const double rho = s.rho[i], hh = s.h[i], AA = s.A[i], mi = s.m[i];
    const double fi = rho / P.rho_ice / hh;
    double ax = fi * (a.tau11[i] * Sx + a.tau12[i] * Sy + Tx);
    double ay = fi * (a.tau12[i] * Sx + a.tau22[i] * Sy + Ty);
    // boundary force (bf_Monaghan normal component, boundary_force.f90:78-82)
    if (P.boundary_pressure && a.nb > 0 && !dead) {
        const Grid g = inst_grid(I, a.cell_start);
        const double bl = I.b_length;
        const int Rb = wall_radius(I.dmax2_bits, g, bl);
        const BinRule bb = make_bin_rule(I.bs, xi, yi, bl);
        double fx = 0.0, fy = 0.0;
        cnt += for_each_wall(a.bx, a.by, a.bstart, g, ci, Rb, bb, xi, yi, bl,
                             [&](int b, double bdx, double bdy, double d) {
                                 const double bw = boundary_w(P, d, hi);
                                 const double mb = a.bm[b];
                                 const double coef = P.kappa_n * bw * 2.0 * mb / ((mi + mb) * (d * d));
                                 fx += coef * bdx;
                                 fy += coef * bdy;
                             });
        ax -= fx / rho;
        ay -= fy / rho;
    }
    // drag, wind_forcing.f90:35-51 and water_drag.f90:35-53 (off at t <= 0)
    const double vxi = s.vx[i], vyi = s.vy[i];
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
    // prognostic rates, single_step.f90:104-106
    const double dv = a.div[i];
    const double dhdt = -hh * dv / rho;
    const double dAdt = -AA * dv / rho;
    warp_max_i32(&a.sc->maxip, live ? cnt : 0);

    if (a.mode == EPI_RATES) {
        if (live) {
            const size_t M = (size_t)a.maxn;
            a.rates[i] = ax;
            a.rates[M + i] = ay;
            a.rates[2 * M + i] = dhdt;
            a.rates[3 * M + i] = dAdt;
        }
        return;
    }
    const double dt = a.sc->dt;
    const State &b = a.base;
    const double x0 = b.x[i], y0 = b.y[i], vx0 = b.vx[i], vy0 = b.vy[i], h0 = b.h[i], A0 = b.A[i];
    double xn, yn, vxn, vyn, hn, An;
    if (a.mode == EPI_PREDICT) {
        // time_integration.f90:315-323
        xn = x0 + vxi * dt / 2.0;
        yn = y0 + vyi * dt / 2.0;
        vxn = vx0 + ax * dt / 2.0;
        vyn = vy0 + ay * dt / 2.0;
        hn = h0 + dhdt * dt / 2.0;
        An = A0 + dAdt * dt / 2.0;
    } else {
        // time_integration.f90:344-367
        const double x12 = x0 + vxi * dt / 2.0, y12 = y0 + vyi * dt / 2.0;
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
    const double rhon = hn * P.rho_ice;                       // density.f90:192
    double mn = b.m[i];
    const double hs_old = b.hs[i];
    if (P.sle != 2 && P.mass_from_area) {                     // mass_evolution.f90:66-69
        const double ar = kPi * ((P.alpha * hs_old) * (P.alpha * hs_old));
        mn = P.rho_ice * An * hn * ar;
    }
    double hsn = hs_old;
    if (a.mode == EPI_CORRECT && P.sle == 2) {                // smoothing_length.f90:136-142
        hsn = sqrt(mn / rhon) * (double)P.hsml_multiplicity;
        if (hsn > P.max_hsml) hsn = P.max_hsml;
    }
    // displacement since the instance's last sort, max per instance
    const double dxr = xn - a.xr[i], dyr = yn - a.yr[i];
    // (non-finite values stay out of these bounds: the basin is flagged below)
    double d2 = dxr * dxr + dyr * dyr;
    if (!live || !isfinite(d2)) d2 = 0.0;
    inst_max_u64(a.inst, ki, offsetof(Inst, dmax2_bits), dbits(d2));
    const double dxl = xn - a.nl.xl[i], dyl = yn - a.nl.yl[i];
    double dl2 = dxl * dxl + dyl * dyl;
    if (!live || !isfinite(dl2)) dl2 = 0.0;
    warp_max_u64(&a.sc->dlist2_bits, dbits(dl2));
    double xa = fmax(fabs(xn), fabs(yn));
    if (!isfinite(xa)) xa = 0.0;
    warp_max_u64(&a.sc->xabs_bits, dbits(xa));
    const bool bad = !(isfinite(xn) && isfinite(yn) && isfinite(vxn) && isfinite(vyn) &&
                       isfinite(hn) && isfinite(An));
    if (live && bad) {
        atomicOr(&a.sc->flags, FLAG_NONFINITE);
        atomicOr(&a.inst[ki].flags, FLAG_NONFINITE);
    }
    if (live) {
        const State &o = a.out;
        o.x[i] = xn;
        o.y[i] = yn;
        o.xf[i] = (float)xn;
        o.yf[i] = (float)yn;
        o.vx[i] = vxn;
        o.vy[i] = vyn;
        o.h[i] = hn;
        o.A[i] = An;
        o.rho[i] = rhon;
        if (P.sle != 2 && P.mass_from_area) o.m[i] = mn;
        o.mor[i] = mn / rhon;
        if (a.mode == EPI_CORRECT && P.sle == 2) a.hs_next[i] = hsn;
    }
    if (a.mode == EPI_CORRECT) {
        if (P.sle == 2) {
            warp_min_u64(&a.sc->acc_hmin, dbits(hsn));
            warp_max_u64(&a.sc->acc_hmax, dbits(hsn));
        }
        if (P.tse == 2) {                                       // time_step.f90:155
            const double v = P.rho_ice * (hsn * hsn) * P.delta_min / (P.P_star * (1.0 + P.k_t));
            warp_min_u64(&a.sc->acc_dt, dbits(v));
        }
    }
    // The last block to finish decides whether the next kinematic pass
    // rebuilds the Verlet lists: when the fastest particle moved 3/4 of the
    // skin since they were built (lists are then complete only for particles
    // that moved less than skin / 4), or when hsml changes (sle = 2).
    // Threadfence reduction; no block waits on another.
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
        const bool stale = (P.sle == 2) || !(dl < 0.75 * a.sc->skin);
        a.sc->list_scan = stale ? 1 : 0;
        a.sc->blocks_done = 0u;
    }
}

// New hsml of the next step (sle = 2) and its FP32 copy.
__global__ void k_commit_hsml(int n, const double *__restrict__ hs_next, double *__restrict__ hs,
                              float *__restrict__ hsf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = hs_next[i];
    hs[i] = v;
    hsf[i] = (float)v;
}

// End of a predictor-corrector step: time_step's new dt, current_time += dt
// (time_integration.f90:179, using the dt computed at the end of the step),
// and the new hsml bounds.
// (One basin per context when tse = 2 or sle = 2: instance 0 carries its
// hsml bounds.)  Every instance's current_time advances by the same dt.
constexpr int kFinishThreads = 256;
__global__ void __launch_bounds__(kFinishThreads) k_step_finish(Scalars *sc, Inst *inst, int ninst, int tse,
                                                                int sle) {
    __shared__ double dt;
    if (threadIdx.x == 0) {
        if (tse == 2) {
            sc->dt = bitsd(sc->acc_dt);
            sc->acc_dt = dbits(INFINITY);
        }
        dt = sc->dt;
        sc->t = sc->t + dt;
        if (sle == 2) {
            sc->hmin = bitsd(sc->acc_hmin);
            sc->hmax = fmax(sc->hmax, bitsd(sc->acc_hmax));
            sc->bs = 2.0 * sc->hmin;
            sc->acc_hmin = dbits(INFINITY);
            sc->acc_hmax = 0ull;
            inst[0].hmin = sc->hmin;
            inst[0].hmax = sc->hmax;
            inst[0].bs = sc->bs;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < ninst; k += kFinishThreads) inst[k].t = inst[k].t + dt;
}

__global__ void k_reset_stats(Scalars *sc) {
    sc->maxip = 0;
    sc->minip = 0x7fffffff;
    sc->sumip = 0ull;
    sc->noip = 0;
    sc->flags = 0;
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

NbrList nbr_list(simp_ctx *c) {
    NbrList nl;
    nl.nbr = c->nbr;
    nl.count = c->nbr_count;
    nl.xl = c->xl;
    nl.yl = c->yl;
    nl.stride = c->maxn;
    return nl;
}

PairList pair_list(simp_ctx *c) {
    PairList pl;
    pl.pj = c->pair_j;
    pl.count = c->pair_count;
    pl.stride = c->maxn;
    return pl;
}

}  // namespace

void launch_kinematic(simp_ctx *c, const State &s, bool diag) {
    KinArgs a;
    a.s = s;
    a.cell_start = c->cell_start;
    a.inst = c->inst_dev;
    a.pinst = c->pinst;
    a.cell = c->cell;
    a.P = c->phys;
    a.sc = c->sc;
    a.tau11 = c->tau11;
    a.tau12 = c->tau12;
    a.tau22 = c->tau22;
    a.div = c->div;
    a.diag = diag ? c->diag : nullptr;
    a.nl = nbr_list(c);
    a.pl = pair_list(c);
    a.n = c->n;
    a.maxn = c->maxn;
    if (c->prm.precision == SIMP_PREC_MIXED)
        k_kinematic<float><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    else
        k_kinematic<double><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_stress(simp_ctx *c, const State &rhs, const State &base, EpiMode mode) {
    StressArgs a;
    a.rhs = rhs;
    a.base = base;
    a.out = (mode == EPI_PREDICT) ? c->s1 : c->s0;
    a.cell_start = c->cell_start;
    a.inst = c->inst_dev;
    a.pinst = c->pinst;
    a.cell = c->cell;
    a.bx = c->bx;
    a.by = c->by;
    a.bm = c->bm;
    a.bstart = c->bcell_start;
    a.nb = c->nb;
    a.P = c->phys;
    a.sc = c->sc;
    a.tau11 = c->tau11;
    a.tau12 = c->tau12;
    a.tau22 = c->tau22;
    a.div = c->div;
    a.nl = nbr_list(c);
    a.pl = pair_list(c);
    a.rates = c->rates;
    a.xr = c->xr;
    a.yr = c->yr;
    a.hs_next = c->tmp;   // hsml of the next step (committed by launch_step_finish)
    a.n = c->n;
    a.maxn = c->maxn;
    a.mode = mode;
    if (c->prm.precision == SIMP_PREC_MIXED)
        k_stress<float><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    else
        k_stress<double><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_step_finish(simp_ctx *c) {
    if (c->prm.sle == 2) {
        k_commit_hsml<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->tmp, c->s0.hs, c->s0.hsf);
        c->launches += 1;
    }
    k_step_finish<<<1, kFinishThreads, 0, c->stream>>>(c->sc, c->inst_dev, c->ninst, c->prm.tse, c->prm.sle);
    c->launches += 1;
}

void launch_reset_stats(simp_ctx *c) {
    k_reset_stats<<<1, 1, 0, c->stream>>>(c->sc);
    c->launches += 1;
}

}  // namespace simp
