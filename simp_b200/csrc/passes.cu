// Pair passes, per-particle implementation: each thread gathers its
// particle's neighbours from HBM, over Verlet lists (candidates within
// mhsml + skin, rebuilt when the fastest particle moved 3/4 of the skin) or
// the cell stencil.  The physics of both passes is described in
// pass_common.cuh.
#include <cmath>

#include "pass_common.cuh"

namespace simp {

namespace {

using namespace pass;

#ifndef SIMP_PASS_BLOCK
#define SIMP_PASS_BLOCK 128
#endif
constexpr int kBlock = SIMP_PASS_BLOCK;   // threads per block of the gather passes
// Up to this many particles in a context the kinematic pass runs as two
// kernels (k_find_pairs, k_kin_sums), above it as one (k_kinematic), unless
// the context names one form (SIMP_PASSES_GATHER_ONE / _TWO).  The
// two-kernel pass writes and re-reads the pair list; it is the faster form
// up to this size, the slower one above it, also when it runs in chunks
// whose pair lists stay in L2 (1,048,576 particles in chunks of 131,072 to
// 400,000: FP64 274 -> 310..374 us, mixed 242 -> 300..314 us against the
// one-kernel pass).  Per pass, one kernel -> two (B200, basins of the
// 500 m lattice), FP64: 147,456 particles 64.6 -> 55.1 us, 262,144 96.4 ->
// 89.2, 409,600 143.0 -> 143.3, 524,176 170.5 -> 179.8, 1,048,576 305.7 ->
// 343.9; mixed: 147,456 66.5 -> 53.3, 262,144 100.1 -> 87.5, 409,600
// 134.7 -> 131.9, 1,048,576 241 -> 267.
constexpr int kSplitMaxParticles = 400000;
// minimum resident blocks per SM, per precision form and kernel, measured
// against 4..8: the FP64 sums kernel of the two-kernel pass keeps its pair
// math in registers (5 blocks, cap 102; 6 is 3% slower at cfg2); the
// one-kernel pass, which runs above kSplitMaxParticles, at 6 blocks (cfg3
// FP64: 274, 249, 261 us per pass at 5, 6, 7; the FP32 form at 7 blocks,
// 253, 235, 241 at 6, 7, 8); the stress passes at 7 (FP64: 6 and 8 are
// 23% and 9% slower at cfg2) and 8 (FP32: 6 and 7 are 10% and 9% slower at
// cfg3)
#ifndef SIMP_KIN_MIN_BLOCKS
#define SIMP_KIN_MIN_BLOCKS 6
#endif
#ifndef SIMP_SUMS_MIN_BLOCKS
#define SIMP_SUMS_MIN_BLOCKS 5
#endif
#ifndef SIMP_STRESS_MIN_BLOCKS
#define SIMP_STRESS_MIN_BLOCKS 7
#endif
#ifndef SIMP_KIN_MIN_BLOCKS_F32
#define SIMP_KIN_MIN_BLOCKS_F32 7
#endif
#ifndef SIMP_STRESS_MIN_BLOCKS_F32
#define SIMP_STRESS_MIN_BLOCKS_F32 8
#endif
template <class T>
struct MinBlocks {
    static constexpr int kin = SIMP_KIN_MIN_BLOCKS, sums = SIMP_SUMS_MIN_BLOCKS, stress = SIMP_STRESS_MIN_BLOCKS;
};
template <>
struct MinBlocks<float> {
    static constexpr int kin = SIMP_KIN_MIN_BLOCKS_F32, sums = SIMP_KIN_MIN_BLOCKS_F32, stress = SIMP_STRESS_MIN_BLOCKS_F32;
};
// per-thread pair list in shared memory: a typical particle's pairs fit;
// a longer list is processed in batches.  Kept small: the shared memory of
// the resident blocks comes out of the L1 cache that serves the gathers.
constexpr int kGatherSlots = 24;
#ifndef SIMP_FIND_MIN_BLOCKS
#define SIMP_FIND_MIN_BLOCKS 8
#endif

// The kinematic pass in one kernel: candidates go into a per-thread list in
// shared memory, then the pair arithmetic runs densely.
template <class T, int SKF>
__global__ void __launch_bounds__(kBlock, MinBlocks<T>::kin) k_kinematic(KinArgs a) {
    __shared__ int s_list[kGatherSlots * kBlock];
    const int t = threadIdx.x;
    const int i = blockIdx.x * blockDim.x + t;
    if (i >= a.n) return;
    const State &s = a.s;
    const Phys &P = a.P;
    const Inst &I = a.inst[a.pinst[i]];
    // a basin whose state turned non-finite is not searched any more (its
    // stencil would span its whole grid); it is only carried until retired
    const bool dead = inst_dead(I.flags);
    const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
    const double xi = pc.xi, yi = pc.yi, hi = pc.hi;
    const double vxi = s.vx[i], vyi = s.vy[i];
    const double inv_hi = 1.0 / hi;
    KinSums<T> ks;     // -div and the velocity gradient, negated
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    const T hu = (I.hmin == I.hmax) ? hiT : T(-1);   // (every neighbour's hsml is hi)
    typename Vec2<T>::type *dwr = reinterpret_cast<typename Vec2<T>::type *>(a.dw);
    int cnt = 0;       // entries in this thread's shared-memory list
    int npairs = 0;    // exact pairs found so far
    int done = 0;      // pairs already processed (and written to the pair list)
    auto flush = [&]() {
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const int j = s_list[k * kBlock + t];
            if (!SIMP_IN_RANGE(j, 0, a.n, SITE_NEIGHBOUR)) continue;
            if (done + k < kMaxPairs) a.pl.pj[(size_t)(done + k) * a.pl.stride + i] = j;
            const double2 q = __ldg(&s.xy[j]), v = __ldg(&s.vxy[j]);
            const KinNb<T> nb = Nb<T>::kin(s, j, hu);
            const PairGeom<T> pg = pair_geom<T, false, SKF>(P, (T)(xi - q.x), (T)(yi - q.y), hiT, inv_hiT, nb.h);
            const T dwx = pg.gfac * pg.dx, dwy = pg.gfac * pg.dy;
            if (dwr && done + k < kDwRows) dwr[(size_t)(done + k) * a.pl.stride + i] = Vec2<T>::make(dwx, dwy);
            ks.add(dwx, dwy, (T)(vxi - v.x), (T)(vyi - v.y), nb.m, nb.mor);
        }
        done += cnt;
        cnt = 0;
    };
    auto on_pair = [&](int j) {
        s_list[cnt * kBlock + t] = j;
        ++npairs;
        if (++cnt == kGatherSlots) flush();
    };
    if (a.sc->list_scan && i == 0) atomicExch(&a.sc->dlist2_bits, 0ull);
    // (a particle of a newly admitted basin builds its list on its own)
    const bool build = a.sc->list_scan || a.nl.count[i] < 0;
    if (dead) {
        if (build) {
            a.nl.count[i] = 0;
            a.nl.xl[i] = xi;
            a.nl.yl[i] = yi;
        }
    } else if (build) {
        // rebuild the Verlet list from the cell stencil: members are the
        // candidates not certainly beyond mhsml + skin (FP32, with margin)
        const double skin = a.sc->skin;
        const float skinf = (float)skin, grow = 1.0f + pc.margin;
        int total = 0;
        for_stencil(pc.g, i, a.cell[i], stencil_radius(pc.hmax, pc.dmax2_bits, pc.g, pc.hmax + skin), [&](int j) {
            const float4 f = __ldg(&s.pf[j]);
            const float dxf = pc.xif - f.x, dyf = pc.yif - f.y;
            const float lim = 0.5f * (pc.hif + f.z) + skinf;
            if (dxf * dxf + dyf * dyf > lim * lim * grow) return;
            if (total < kMaxNbr) a.nl.nbr[(size_t)total * a.nl.stride + i] = j;
            ++total;
            if (is_pair_with(s, pc, j, f)) on_pair(j);
        });
        a.nl.count[i] = total;
        a.nl.xl[i] = xi;
        a.nl.yl[i] = yi;
    } else {
        // (room for a whole batch in the list before each batch)
        for_each_current_pair_batched(s, a.nl, a.sc, i, a.cell[i], pc, [&]() {
            if (cnt > kGatherSlots - kBatch) flush();
        }, [&](int j) {
            s_list[cnt * kBlock + t] = j;
            ++npairs;
            ++cnt;
        });
    }
    flush();   // (also writes the stress pass's pair list, a coalesced row per k)
    a.pl.count[i] = npairs;
    kin_rheology(a, i, -ks.dv.get(), -ks.g1.get(), -ks.g2.get(), -ks.g3.get(), -ks.g4.get());
}

// The kinematic pass in two kernels.  k_find_pairs decides the exact pairs
// of each particle (Verlet candidates, or the cell stencil when the lists
// are rebuilt) and writes them as the pair list; it needs fewer registers
// than the FP64 pair arithmetic, so more warps hide its gather latency.
// k_kin_sums then does the pair arithmetic over those rows, in the order
// they were found, the order of the one-kernel pass: both give bitwise the
// same results.  launch_kinematic picks between them.
__global__ void __launch_bounds__(kBlock, SIMP_FIND_MIN_BLOCKS) k_find_pairs(KinArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Inst &I = a.inst[a.pinst[i]];
    // a basin whose state turned non-finite is not searched any more (its
    // stencil would span its whole grid); it is only carried until retired
    const bool dead = inst_dead(I.flags);
    const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
    int npairs = 0;
    auto on_pair = [&](int j) {
        if (npairs < kMaxPairs) a.pl.pj[(size_t)npairs * a.pl.stride + i] = j;
        ++npairs;
    };
    if (a.sc->list_scan && i == 0) atomicExch(&a.sc->dlist2_bits, 0ull);
    // (a particle of a newly admitted basin builds its list on its own)
    const bool build = a.sc->list_scan || a.nl.count[i] < 0;
    if (dead) {
        if (build) {
            a.nl.count[i] = 0;
            a.nl.xl[i] = pc.xi;
            a.nl.yl[i] = pc.yi;
        }
    } else if (build) {
        // rebuild the Verlet list from the cell stencil: members are the
        // candidates not certainly beyond mhsml + skin (FP32, with margin)
        const double skin = a.sc->skin;
        const float skinf = (float)skin, grow = 1.0f + pc.margin;
        int total = 0;
        for_stencil(pc.g, i, a.cell[i], stencil_radius(pc.hmax, pc.dmax2_bits, pc.g, pc.hmax + skin), [&](int j) {
            const float4 f = __ldg(&s.pf[j]);
            const float dxf = pc.xif - f.x, dyf = pc.yif - f.y;
            const float lim = 0.5f * (pc.hif + f.z) + skinf;
            if (dxf * dxf + dyf * dyf > lim * lim * grow) return;
            if (total < kMaxNbr) a.nl.nbr[(size_t)total * a.nl.stride + i] = j;
            ++total;
            if (is_pair_with(s, pc, j, f)) on_pair(j);
        });
        a.nl.count[i] = total;
        a.nl.xl[i] = pc.xi;
        a.nl.yl[i] = pc.yi;
    } else {
        for_each_current_pair_batched(s, a.nl, a.sc, i, a.cell[i], pc, [] {}, on_pair);
    }
    a.pl.count[i] = npairs;
}

template <class T, int SKF>
__global__ void __launch_bounds__(kBlock, MinBlocks<T>::sums) k_kin_sums(KinArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Phys &P = a.P;
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const double vxi = s.vx[i], vyi = s.vy[i];
    const double inv_hi = 1.0 / hi;
    KinSums<T> ks;     // -div and the velocity gradient, negated
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    typename Vec2<T>::type *dwr = reinterpret_cast<typename Vec2<T>::type *>(a.dw);
    auto pair = [&](int k, int j) {
        if (!SIMP_IN_RANGE(j, 0, a.n, SITE_NEIGHBOUR)) return;
        const double2 q = __ldg(&s.xy[j]), v = __ldg(&s.vxy[j]);
        const KinNb<T> nb = Nb<T>::kin(s, j, T(-1));
        const PairGeom<T> pg = pair_geom<T, false, SKF>(P, (T)(xi - q.x), (T)(yi - q.y), hiT, inv_hiT, nb.h);
        const T dwx = pg.gfac * pg.dx, dwy = pg.gfac * pg.dy;
        if (dwr && k < kDwRows) dwr[(size_t)k * a.pl.stride + i] = Vec2<T>::make(dwx, dwy);
        ks.add(dwx, dwy, (T)(vxi - v.x), (T)(vyi - v.y), nb.m, nb.mor);
    };
    const int cnt = a.pl.count[i];
    if (cnt <= kMaxPairs) {
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) pair(k, __ldg(&a.pl.pj[(size_t)k * a.pl.stride + i]));
    } else {
        // more pairs than list rows: found again, in the same order
        const PairCtx pc = pair_ctx(s, a.sc, a.inst[a.pinst[i]], a.cell_start, i);
        int k = 0;
        for_each_current_pair(s, a.nl, a.sc, i, a.cell[i], pc, [&](int j) { pair(k++, j); });
    }
    kin_rheology(a, i, -ks.dv.get(), -ks.g1.get(), -ks.g2.get(), -ks.g3.get(), -ks.g4.get());
}

template <class T, int SKF>
__global__ void __launch_bounds__(kBlock, MinBlocks<T>::stress) k_stress(StressArgs a) {
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
    const bool dead = inst_dead(I.flags);   // see k_kinematic
    StressSums<T> ss;
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    const T hu = (I.hmin == I.hmax) ? hiT : T(-1);   // (every neighbour's hsml is hi)
    auto accumulate = [&](int j) {
        if (!SIMP_IN_RANGE(j, 0, a.n, SITE_NEIGHBOUR)) return;
        const double2 q = __ldg(&s.xy[j]);
        const StressNb<T> nb = Nb<T>::stress(s, a.rec, j, hu);
        const PairGeom<T> pg = pair_geom<T, false, SKF>(P, (T)(xi - q.x), (T)(yi - q.y), hiT, inv_hiT, nb.h);
        ss.add(pg.gfac * pg.dx, pg.gfac * pg.dy, nb.m, nb.t11, nb.t12, nb.t22);
    };
    int cnt = a.pl.count[i];
    if (a.dw && cnt <= kDwRows && !dead) {
        // the kinematic pass kept these pairs' kernel gradients
        const typename Vec2<T>::type *dwr = reinterpret_cast<const typename Vec2<T>::type *>(a.dw);
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const size_t r = (size_t)k * a.pl.stride + i;
            const typename Vec2<T>::type g = __ldg(&dwr[r]);
            const int j = __ldg(&a.pl.pj[r]);
            if (!SIMP_IN_RANGE(j, 0, a.n, SITE_NEIGHBOUR)) continue;
            const StressNb<T> nb = Nb<T>::stress_rec(a.rec, j);
            ss.add(g.x, g.y, nb.m, nb.t11, nb.t12, nb.t22);
        }
    } else if (cnt <= kMaxPairs) {
        // the kinematic pass of this right-hand side found the pairs
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) accumulate(__ldg(&a.pl.pj[(size_t)k * a.pl.stride + i]));
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
    // (a retired basin's particles are not written any more: their state
    // stays as it was until the batch's next compaction drops them)
    stress_finish<SKF>(a, i, live && !(I.flags & FLAG_RETIRED), ki, I, dead, xi, yi, hi, ci, ss.sx.get(), ss.sy.get(),
                       ss.tx.get(), ss.ty.get(), cnt, true);
}

// Regularisation of a right-hand side (regularization.f90, called by
// single_step.f90:99-101), per particle i over the pairs the kinematic pass
// just found, in FP64 in both precision forms:
//   XSPH (:45-95)  xs_i = sum_j m_j (v_i - v_j) W_ij / ((rho_i + rho_j) / 2)
//   artificial viscosity, av_i = -sum_j m_j pi_ij grad_i W_ij with
//     Hernquist-Katz (:102-213): pi_ij = lv_i / rho_i^2 + lv_j / rho_j^2,
//       lv = (alpha_pi hsml c |d| + beta_pi (|d| hsml)^2) rho, d the
//       velocity divergence (the kinematic pass's sum over rho) where it is
//       negative, else 0;
//     Monaghan (:220-308): pi_ij = (beta_pi iota^2 - alpha_pi iota
//       (c_i + c_j) / 2) / ((rho_i + rho_j) / 2), iota = hsml_ij v_r /
//       (r_ij^2 + (0.01 hsml_ij)^2), v_r = (v_i - v_j) . (x_i - x_j);
//     for pairs with (v_i - v_j) . (x_i - x_j) <= 0, else pi_ij = 0.
// The reference runs both loops serially over its pair list, where pi_ij
// keeps the previous pair's value for a pair outside the criterion and XSPH
// adds the same-signed term to both particles; the gather here evaluates
// every pair on its own (zero outside the criterion, XSPH antisymmetric).
struct RegArgs {
    State s;
    const double *div;   // the kinematic pass's -sum_j m_j (v_i - v_j) . grad W
    PairList pl;
    NbrList nl;
    const int *cell_start, *cell, *pinst;
    const Inst *inst;
    Scalars *sc;
    Phys P;
    double *reg;
    int n, maxn;
};

// lv / rho^2 of the Hernquist-Katz viscosity of particle k
__device__ __forceinline__ double hk_lv_r2(const Phys &P, const State &s, const double *div, int k) {
    const double rho = s.rho[k], hs = s.hs[k];
    double d = div[k] / rho;
    if (d >= 0.0) d = 0.0;
    const double c = sound_speed_held(P, rho);
    const double ad = fabs(d);
    const double lv = (P.alpha_pi * hs * c * ad + P.beta_pi * ((ad * hs) * (ad * hs))) * rho;
    return lv / (rho * rho);
}

__global__ void __launch_bounds__(kBlock) k_regularize(RegArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Phys &P = a.P;
    const size_t M = (size_t)a.maxn;
    const Inst &I = a.inst[a.pinst[i]];
    const double2 xy = s.xy[i], v = s.vxy[i];
    const double xi = xy.x, yi = xy.y, vxi = v.x, vyi = v.y;
    const double hi = s.hs[i], inv_hi = 1.0 / hi, rhoi = s.rho[i];
    const double ci = sound_speed_held(P, rhoi);
    const double pii = (P.art_visc == 1) ? hk_lv_r2(P, s, a.div, i) : 0.0;
    Sum<double> avx, avy, xsx, xsy;
    auto pair = [&](int j) {
        if (!SIMP_IN_RANGE(j, 0, a.n, SITE_NEIGHBOUR)) return;
        const double2 q = s.xy[j], w = s.vxy[j];
        const double dx = xi - q.x, dy = yi - q.y;
        const double dvx = vxi - w.x, dvy = vyi - w.y;
        const double hj = s.hs[j], rhoj = s.rho[j], mj = s.m[j];
        const PairGeom<double> pg = pair_geom<double, true>(P, dx, dy, hi, inv_hi, hj);
        if (P.xsph) {
            const double rbar = 0.5 * (rhoi + rhoj);
            xsx.madd(mj * dvx * pg.w / rbar, 1.0);
            xsy.madd(mj * dvy * pg.w / rbar, 1.0);
        }
        const double vr = dvx * dx + dvy * dy;
        if ((P.art_visc == 1 || P.art_visc == 2) && vr <= 0.0) {
            double pij;
            if (P.art_visc == 1) {
                pij = pii + hk_lv_r2(P, s, a.div, j);
            } else {
                const double hij = __dmul_rn(__dadd_rn(hi, hj), 0.5);
                const double r = ref_distance(dx, dy);
                const double scor = (double)0.01f * hij;
                const double iota = hij * vr / (r * r + scor * scor);
                const double cj = sound_speed_held(P, rhoj);
                pij = (P.beta_pi * (iota * iota) - P.alpha_pi * iota * (ci + cj) / 2.0) / ((rhoi + rhoj) / 2.0);
            }
            avx.madd(-(mj * pij), pg.gfac * pg.dx);
            avy.madd(-(mj * pij), pg.gfac * pg.dy);
        }
    };
    const bool dead = inst_dead(I.flags);
    const int cnt = a.pl.count[i];
    if (dead) {
    } else if (cnt <= kMaxPairs) {
        for (int k = 0; k < cnt; ++k) pair(a.pl.pj[(size_t)k * a.pl.stride + i]);
    } else {
        const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
        for_each_current_pair(s, a.nl, a.sc, i, a.cell[i], pc, pair);
    }
    a.reg[i] = avx.get();
    a.reg[M + i] = avy.get();
    a.reg[2 * M + i] = xsx.get();
    a.reg[3 * M + i] = xsy.get();
}

// Density rate drho/dt_i = sum_j m_j (v_i - v_j) . grad_i W_ij over the
// pairs of the right-hand side just evaluated, with the velocities the
// integrator has just written: con_density (density.f90:107-165, called
// after each update, time_integration.f90:128-133, 218-223, 344-349, 372-377)
// and the same sum in Benz_hsml (smoothing_length.f90:62-80).  The pair
// geometry and hsml are those of the right-hand side's state (the reference
// reuses that right-hand side's p_i, p_j and dwdx); the masses are the
// current ones at the call: the right-hand side's for con_density (called
// before mass_evolution), the updated ones for Benz_hsml's own sum (called
// after it).  The sum is FP64 in both precision forms.
//   rho_upd: 0 none, 1 rho = rho_1 + drho/dt dt / 2, 2 rho = rho_1 + drho/dt dt;
//   tail: the step's final hsml (Benz, or Marquis with the new density),
//   its bounds and the VP time step, which the stress epilogue left out.
struct DensArgs {
    State g;             // right-hand side state (positions, hsml, masses)
    State v;             // updated state: velocities in, rho and views out
    const double *mj;    // neighbour masses of the sum
    const double *rho1;  // step-start density
    double *acc;         // Benz's drhodt when den_alg != 2 (kept across steps)
    const double *a2;    // |dv/dt|^2 of the last right-hand side (tse = 1)
    double *hs_next;
    PairList pl;
    const int *cell_start, *cell, *pinst;
    const Inst *inst;
    Scalars *sc;
    Phys P;
    int n, rho_upd, tail;
    int dt_div;          // the Monaghan time step's divergence (artificial viscosity)
    // summation density (den_alg = 1, density.f90:41-100): rho_out =
    // (k0 m_i + sum_j m_j W_ij) / (k0 m_i / rho_i + sum_j m_j W_ij / rho_j)
    // over the right-hand side's pairs and kernel values, with the masses
    // m_sum and densities rho_in at the reference's density call; rho_out
    // is o.rho (then m/rho and the packed copies follow) or a scratch array
    // that k_commit_rho copies in
    int sum_mode;
    const double *m_sum, *rho_in;
    double *rho_out;
    // its self term kernel_zero(i) m_i: the reference keeps kernel_zero per
    // particle and sets it in each right-hand side's pair loop for the p_i
    // of every pair, W(0) at the pair's hsml (kernel.f90:503, set to 0 by
    // initialize.f90:60), so a particle that is p_i of no pair keeps an
    // earlier value.  Which particle of a pair is p_i follows the search:
    // direct_find (nnps.f90:41-148) the lower index; the bucket search
    // (nnps.f90:259-411) the lower index within one bucket, else the
    // particle whose bucket has the other's to its right, above, above
    // right or above left.  Of several pairs the serial pair order's last
    // gives the value (it matters only where hsml varies)
    double *k0;
    const int *id;
};

__global__ void __launch_bounds__(kBlock) k_density_rate(DensArgs a) {
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = i0 < a.n ? i0 : a.n - 1;   // dead lanes mirror the last particle for the reductions
    const State &g = a.g;
    const Phys &P = a.P;
    const Inst &I = a.inst[a.pinst[i]];
    const bool live = i0 < a.n && !(I.flags & FLAG_RETIRED);   // (a retired basin is not written)
    const bool dead = inst_dead(I.flags);
    const double xi = g.x[i], yi = g.y[i], hi = g.hs[i];
    const double inv_hi = 1.0 / hi;
    const double vxi = a.v.vx[i], vyi = a.v.vy[i];
    Sum<double> r, rt, num, den;
    // p_i rule of the summation density's kernel_zero (DensArgs)
    const int idi = a.sum_mode ? a.id[i] : 0;
    const long long bxi = (a.sum_mode && P.nnps == 2) ? ref_bin(xi, I.bs) : 0;
    const long long byi = (a.sum_mode && P.nnps == 2) ? ref_bin(yi, I.bs) : 0;
    long long last = -1;   // (position in the serial pair order, category then index)
    double h_last = 0.0;
    auto add = [&](int j) {
        if (!SIMP_IN_RANGE(j, 0, a.n, SITE_NEIGHBOUR)) return;
        const double2 q = g.xy[j];
        PairGeom<double> pg;
        if (a.sum_mode) {
            pg = pair_geom<double, true>(P, xi - q.x, yi - q.y, hi, inv_hi, g.hs[j]);
            const double mw = a.m_sum[j] * pg.w;
            num.madd(mw, 1.0);
            den.madd(mw / a.rho_in[j], 1.0);
            const int idj = a.id[j];
            int cat = -1;
            if (P.nnps != 2) {
                cat = idj > idi ? 0 : -1;
            } else {
                const long long dx = ref_bin(q.x, I.bs) - bxi, dy = ref_bin(q.y, I.bs) - byi;
                if (dx == 0 && dy == 0) cat = idj > idi ? 0 : -1;
                else if (dy == 0 && dx == 1) cat = 1;     // right
                else if (dy == 1 && dx == 0) cat = 2;     // up
                else if (dy == 1 && dx == 1) cat = 3;     // up-right
                else if (dy == 1 && dx == -1) cat = 4;    // up-left
            }
            const long long key = cat < 0 ? -1 : ((long long)cat << 32) | (long long)(unsigned)idj;
            if (key > last) {
                last = key;
                h_last = g.hs[j];
            }
        } else {
            pg = pair_geom<double, false>(P, xi - q.x, yi - q.y, hi, inv_hi, g.hs[j]);
        }
        const double2 v = a.v.vxy[j];
        const double dvx = vxi - v.x, dvy = vyi - v.y;
        const double t = fma(dvx, pg.gfac * pg.dx, dvy * (pg.gfac * pg.dy));
        r.madd(a.mj[j], t);
        // time_step.f90:93-109: the current masses (after mass_evolution)
        if (a.dt_div) rt.madd(a.v.m[j], t);
    };
    const int cnt = a.pl.count[i];
    if (dead) {
    } else if (cnt <= kMaxPairs) {
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) add(a.pl.pj[(size_t)k * a.pl.stride + i]);
    } else {
        // (more pairs than the list holds: the cell stencil of the
        // right-hand side's positions, whose bounds the instance keeps)
        const PairCtx pc = pair_ctx(g, a.sc, I, a.cell_start, i);
        for_stencil(pc.g, i, a.cell[i], stencil_radius(pc.hmax, pc.dmax2_bits, pc.g, 0.0), [&](int j) {
            if (is_pair(g, pc, j)) add(j);
        });
    }
    const double drhodt = r.get();
    const double dt = a.sc->dt;
    const State &o = a.v;
    double rhon = o.rho[i];
    if (a.sum_mode) {
        double k0 = a.k0[i];
        if (last >= 0) k0 = kernel_zero(P, (hi + h_last) / 2.0);   // nnps.f90:278
        const double k0m = k0 * a.m_sum[i];
        rhon = (k0m + num.get()) / (k0m / a.rho_in[i] + den.get());
        if (live) {
            a.k0[i] = k0;
            a.rho_out[i] = rhon;
            if (a.rho_out == o.rho) {
                o.mor[i] = o.m[i] / rhon;
                refresh_views(o, i);
            }
        }
    } else if (a.rho_upd && live) {
        rhon = (a.rho_upd == 1) ? a.rho1[i] + drhodt * dt / 2.0 : a.rho1[i] + drhodt * dt;
        o.rho[i] = rhon;
        o.mor[i] = o.m[i] / rhon;
        refresh_views(o, i);
    }
    if (!a.tail) return;
    const double hs_old = g.hs[i];
    double hsn = hs_old;
    if (P.sle == 1) {
        // Benz_hsml, smoothing_length.f90:82-94.  Without con_density the
        // reference adds to its drhodt array, never cleared: kept per
        // particle across steps (and re-sorts) here.
        double d = drhodt;
        if (a.acc) {
            d = a.acc[i] + drhodt;
            if (live) a.acc[i] = d;
        }
        const double dhs = -hs_old * d / 2.0 / rhon;
        hsn = hs_old + dhs * dt;
        if (hsn < 0.0) hsn = hsn - dhs * dt;
    } else if (P.sle == 2) {                                   // smoothing_length.f90:136-142
        hsn = sqrt(o.m[i] / rhon) * (double)P.hsml_multiplicity;
        if (hsn > P.max_hsml) hsn = P.max_hsml;
    }
    if (live && P.sle != 0) a.hs_next[i] = hsn;
    // (dead lanes contribute neutral values: the particle they mirror may
    // already have been updated by its own thread)
    unsigned active = 0u;
    unsigned long long v[kBounds] = {0ull, 0ull, 0ull, ~0ull, 0ull, ~0ull};
    if (P.sle != 0) {
        active |= 8u | 16u;
        if (live) {
            v[3] = dbits(hsn);
            v[4] = dbits(hsn);
        }
    }
    if (P.tse != 0) {                                          // time_step.f90:20-26
        active |= 32u;
        // |div v| = |sum_j m_j (v_i - v_j) . grad W| / rho_i (time_step.f90:108-111)
        const double adiv = a.dt_div ? fabs(rt.get() / rhon) : 0.0;
        if (live) v[5] = dbits(dt_candidate(P, hsn, P.tse == 1 ? a.a2[i] : 0.0, rhon, adiv));
    }
    block_bounds(a.sc, active, v);
}

// The summation density written to scratch by the second of two passes
// into the state (the first pass read the state's density).
__global__ void k_commit_rho(int n, const double *__restrict__ src, State o, const int *__restrict__ pinst,
                             const Inst *__restrict__ inst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (inst[pinst[i]].flags & FLAG_RETIRED)) return;
    const double r = src[i];
    o.rho[i] = r;
    o.mor[i] = o.m[i] / r;
    refresh_views(o, i);
}

// New hsml of the next step (sle = 1, 2) and its FP32 copy.
__global__ void k_commit_hsml(int n, const double *__restrict__ hs_next, State s0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = hs_next[i];
    const float vf = (float)v;
    s0.hs[i] = v;
    s0.hsf[i] = vf;
    s0.pf[i].z = vf;
    if (s0.hmm) s0.hmm[i].x = vf;
}

// End of a predictor-corrector step: time_step's new dt, current_time += dt
// (time_integration.f90:71, using the dt computed at the end of the step),
// and the new hsml bounds.
// (One basin per context when tse = 2 or sle != 0: instance 0 carries its
// hsml bounds.)  Every instance's current_time advances by the same dt.
constexpr int kFinishThreads = 256;
__global__ void __launch_bounds__(kFinishThreads) k_step_finish(Scalars *sc, Inst *inst, int ninst, int tse,
                                                                int sle) {
    __shared__ double dt;
    if (threadIdx.x == 0) {
        if (tse != 0) {
            sc->dt = bitsd(sc->acc_dt);
            sc->acc_dt = dbits(INFINITY);
        }
        dt = sc->dt;
        sc->t = sc->t + dt;
        if (sle != 0) {
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

// The Euler step writes its result into S1 (S0 is read by the pair sums of
// the same pass); this copies it back, with the packed copies.
__global__ void k_copy_s1_to_s0(int n, State s1, State s0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    s0.x[i] = s1.x[i];
    s0.y[i] = s1.y[i];
    s0.vx[i] = s1.vx[i];
    s0.vy[i] = s1.vy[i];
    s0.h[i] = s1.h[i];
    s0.A[i] = s1.A[i];
    s0.rho[i] = s1.rho[i];
    s0.mor[i] = s1.mor[i];
    if (s1.m != s0.m) s0.m[i] = s1.m[i];
    s0.xy[i] = s1.xy[i];
    s0.vxy[i] = s1.vxy[i];
    s0.pf[i] = s1.pf[i];
    if (s0.hmm) s0.hmm[i] = s1.hmm[i];
    else s0.mm[i] = s1.mm[i];
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
    nl.n = c->n;
    return nl;
}

TauRec tau_rec(simp_ctx *c) {
    TauRec r;
    r.ta = c->tau_a;
    r.tb = c->tau_b;
    r.tq = c->tau_q;
    return r;
}

PairList pair_list(simp_ctx *c) {
    PairList pl;
    pl.pj = c->pair_j;
    pl.count = c->pair_count;
    pl.stride = c->maxn;
    pl.n = c->n;
    return pl;
}

}  // namespace

void launch_kinematic(simp_ctx *c, const State &s, bool diag) {
    SIMP_RANGE("kinematic pass");
    KinArgs a{};
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
    a.rec = tau_rec(c);
    a.dw = c->pair_dw;
    a.diag = diag ? c->diag : nullptr;
    a.nl = nbr_list(c);
    a.pl = pair_list(c);
    a.n = c->n;
    a.maxn = c->maxn;
    if (c->pass_impl == SIMP_PASSES_TILED) {
        launch_kinematic_tiled(c, a);
        return;
    }
    const int g = nblk(c->n, kBlock);
    const bool mixed = c->prm.precision == SIMP_PREC_MIXED;
    const bool two = c->pass_impl == SIMP_PASSES_GATHER_TWO ||
                     (c->pass_impl == SIMP_PASSES_GATHER && c->n <= kSplitMaxParticles);
    if (!two) {
        switch (skf_compiled(c->prm.skf)) {
            case SIMP_SKF_CUBIC:
                if (mixed) k_kinematic<float, SIMP_SKF_CUBIC><<<g, kBlock, 0, c->stream>>>(a);
                else k_kinematic<double, SIMP_SKF_CUBIC><<<g, kBlock, 0, c->stream>>>(a);
                break;
            case SIMP_SKF_WENDLAND_C6:
                if (mixed) k_kinematic<float, SIMP_SKF_WENDLAND_C6><<<g, kBlock, 0, c->stream>>>(a);
                else k_kinematic<double, SIMP_SKF_WENDLAND_C6><<<g, kBlock, 0, c->stream>>>(a);
                break;
            default:
                if (mixed) k_kinematic<float, 0><<<g, kBlock, 0, c->stream>>>(a);
                else k_kinematic<double, 0><<<g, kBlock, 0, c->stream>>>(a);
        }
        c->launches += 1;
        return;
    }
    k_find_pairs<<<g, kBlock, 0, c->stream>>>(a);
    switch (skf_compiled(c->prm.skf)) {
        case SIMP_SKF_CUBIC:
            if (mixed) k_kin_sums<float, SIMP_SKF_CUBIC><<<g, kBlock, 0, c->stream>>>(a);
            else k_kin_sums<double, SIMP_SKF_CUBIC><<<g, kBlock, 0, c->stream>>>(a);
            break;
        case SIMP_SKF_WENDLAND_C6:
            if (mixed) k_kin_sums<float, SIMP_SKF_WENDLAND_C6><<<g, kBlock, 0, c->stream>>>(a);
            else k_kin_sums<double, SIMP_SKF_WENDLAND_C6><<<g, kBlock, 0, c->stream>>>(a);
            break;
        default:
            if (mixed) k_kin_sums<float, 0><<<g, kBlock, 0, c->stream>>>(a);
            else k_kin_sums<double, 0><<<g, kBlock, 0, c->stream>>>(a);
    }
    c->launches += 2;
}

void launch_stress(simp_ctx *c, const State &rhs, const State &base, EpiMode mode) {
    SIMP_RANGE("stress pass");
    StressArgs a{};
    a.rhs = rhs;
    a.base = base;
    a.out = (mode == EPI_PREDICT || mode == EPI_EULER) ? c->s1 : c->s0;
    a.cell_start = c->cell_start;
    a.inst = c->inst_dev;
    a.pinst = c->pinst;
    a.cell = c->cell;
    a.bx = c->bx;
    a.by = c->by;
    a.bm = c->bm;
    a.bnx = c->bnx;
    a.bny = c->bny;
    a.bstart = c->bcell_start;
    a.nb = c->nb;
    a.P = c->phys;
    a.sc = c->sc;
    a.tau11 = c->tau11;
    a.tau12 = c->tau12;
    a.tau22 = c->tau22;
    a.div = c->div;
    a.rec = tau_rec(c);
    a.dw = c->pair_dw;
    a.nl = nbr_list(c);
    a.pl = pair_list(c);
    a.rates = c->rates;
    a.reg = c->reg;
    a.xr = c->xr;
    a.yr = c->yr;
    a.hs_next = c->tmp;   // hsml of the next step (committed by launch_step_finish)
    a.n = c->n;
    a.maxn = c->maxn;
    a.mode = mode;
    if (c->pass_impl == SIMP_PASSES_TILED) {
        launch_stress_tiled(c, a);
        return;
    }
    const bool mixed = c->prm.precision == SIMP_PREC_MIXED;
    const int g = nblk(c->n, kBlock);
    switch (skf_compiled(c->prm.skf)) {
        case SIMP_SKF_CUBIC:
            if (mixed) k_stress<float, SIMP_SKF_CUBIC><<<g, kBlock, 0, c->stream>>>(a);
            else k_stress<double, SIMP_SKF_CUBIC><<<g, kBlock, 0, c->stream>>>(a);
            break;
        case SIMP_SKF_WENDLAND_C6:
            if (mixed) k_stress<float, SIMP_SKF_WENDLAND_C6><<<g, kBlock, 0, c->stream>>>(a);
            else k_stress<double, SIMP_SKF_WENDLAND_C6><<<g, kBlock, 0, c->stream>>>(a);
            break;
        default:
            if (mixed) k_stress<float, 0><<<g, kBlock, 0, c->stream>>>(a);
            else k_stress<double, 0><<<g, kBlock, 0, c->stream>>>(a);
    }
    c->launches += 1;
}

void launch_regularize(simp_ctx *c, const State &s) {
    if (!c->reg) return;
    SIMP_RANGE("regularisation pass");
    RegArgs a{};
    a.s = s;
    a.div = c->div;
    a.pl = pair_list(c);
    a.nl = nbr_list(c);
    a.cell_start = c->cell_start;
    a.cell = c->cell;
    a.pinst = c->pinst;
    a.inst = c->inst_dev;
    a.sc = c->sc;
    a.P = c->phys;
    a.reg = c->reg;
    a.n = c->n;
    a.maxn = c->maxn;
    k_regularize<<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_density_rate(simp_ctx *c, const State &g, const State &v, int rho_upd, bool tail) {
    SIMP_RANGE("density-rate pass");
    DensArgs a{};
    a.g = g;
    a.v = v;
    a.rho1 = c->s0.rho;
    a.acc = c->drhodt;
    a.mj = c->drhodt ? v.m : g.m;
    a.a2 = c->rates;
    a.hs_next = c->tmp;
    a.pl = pair_list(c);
    a.cell_start = c->cell_start;
    a.cell = c->cell;
    a.pinst = c->pinst;
    a.inst = c->inst_dev;
    a.sc = c->sc;
    a.P = c->phys;
    a.n = c->n;
    a.rho_upd = rho_upd;
    a.tail = tail ? 1 : 0;
    a.dt_div = (tail && c->prm.tse == 1 && c->prm.artificial_visc) ? 1 : 0;
    k_density_rate<<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_sum_density(simp_ctx *c, const State &g, const State &v, const double *m_sum, const double *rho_in,
                        double *rho_out, bool tail) {
    SIMP_RANGE("summation-density pass");
    DensArgs a{};
    a.g = g;
    a.v = v;
    a.rho1 = c->s0.rho;
    a.acc = c->drhodt;
    a.mj = c->drhodt ? v.m : g.m;
    a.a2 = c->rates;
    a.hs_next = c->tmp;
    a.pl = pair_list(c);
    a.cell_start = c->cell_start;
    a.cell = c->cell;
    a.pinst = c->pinst;
    a.inst = c->inst_dev;
    a.sc = c->sc;
    a.P = c->phys;
    a.n = c->n;
    a.rho_upd = 0;
    a.tail = tail ? 1 : 0;
    a.dt_div = (tail && c->prm.tse == 1 && c->prm.artificial_visc) ? 1 : 0;
    a.sum_mode = 1;
    a.m_sum = m_sum;
    a.rho_in = rho_in;
    a.rho_out = rho_out;
    a.k0 = c->k0;
    a.id = c->id;
    k_density_rate<<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_commit_rho(simp_ctx *c, const double *src, const State &o) {
    k_commit_rho<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, src, o, c->pinst, c->inst_dev);
    c->launches += 1;
}

void launch_step_finish(simp_ctx *c) {
    if (c->prm.sle != 0) {
        k_commit_hsml<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->tmp, c->s0);
        c->launches += 1;
    }
    k_step_finish<<<1, kFinishThreads, 0, c->stream>>>(c->sc, c->inst_dev, c->ninst, c->prm.tse, c->prm.sle);
    c->launches += 1;
}

void launch_copy_s1_to_s0(simp_ctx *c) {
    k_copy_s1_to_s0<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->n, c->s1, c->s0);
    c->launches += 1;
}

void launch_reset_stats(simp_ctx *c) {
    k_reset_stats<<<1, 1, 0, c->stream>>>(c->sc);
    c->launches += 1;
}

}  // namespace simp
