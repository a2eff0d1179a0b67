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

constexpr int kBlock = 128;
// minimum resident blocks per SM (register caps 73 and 64): more warps in
// flight to hide the latency of the neighbour gathers
#ifndef SIMP_KIN_MIN_BLOCKS
#define SIMP_KIN_MIN_BLOCKS 7
#endif
#ifndef SIMP_STRESS_MIN_BLOCKS
#define SIMP_STRESS_MIN_BLOCKS 8
#endif
constexpr int kMinBlocksKin = SIMP_KIN_MIN_BLOCKS;
constexpr int kMinBlocksStress = SIMP_STRESS_MIN_BLOCKS;
// per-thread pair list in shared memory: a typical particle's pairs fit;
// a longer list is processed in batches.  Kept small: the shared memory of
// the resident blocks comes out of the L1 cache that serves the gathers.
constexpr int kGatherSlots = 24;

template <class T>
__global__ void __launch_bounds__(kBlock, kMinBlocksKin) k_kinematic(KinArgs a) {
    __shared__ int s_list[kGatherSlots * kBlock];
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
    KinSums<T> ks;     // -div and the velocity gradient, negated
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    typename Vec2<T>::type *dwr = reinterpret_cast<typename Vec2<T>::type *>(a.dw);
    int cnt = 0;       // entries in this thread's shared-memory list
    int npairs = 0;    // exact pairs found so far
    int done = 0;      // pairs already processed (and written to the pair list)
    auto flush = [&]() {
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const int j = s_list[k * kBlock + t];
            if (done + k < kMaxPairs) a.pl.pj[(size_t)(done + k) * a.pl.stride + i] = j;
            const double2 q = s.xy[j], v = s.vxy[j];
            const KinNb<T> nb = Nb<T>::kin(s, j);
            const PairGeom<T> pg = pair_geom<T, false>(P, (T)(xi - q.x), (T)(yi - q.y), hiT, inv_hiT, nb.h);
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
            const float4 f = s.pf[j];
            const float dxf = pc.xif - f.x, dyf = pc.yif - f.y;
            const float lim = 0.5f * (pc.hif + f.z) + skinf;
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
    flush();   // (also writes the stress pass's pair list, a coalesced row per k)
    a.pl.count[i] = npairs;
    kin_rheology(a, i, -ks.dv.get(), -ks.g1.get(), -ks.g2.get(), -ks.g3.get(), -ks.g4.get());
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
    StressSums<T> ss;
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    auto accumulate = [&](int j) {
        const double2 q = s.xy[j];
        const StressNb<T> nb = Nb<T>::stress(s, a.rec, j);
        const PairGeom<T> pg = pair_geom<T, false>(P, (T)(xi - q.x), (T)(yi - q.y), hiT, inv_hiT, nb.h);
        ss.add(pg.gfac * pg.dx, pg.gfac * pg.dy, nb.m, nb.t11, nb.t12, nb.t22);
    };
    int cnt = a.pl.count[i];
    if (a.dw && cnt <= kDwRows && !dead) {
        // the kinematic pass kept these pairs' kernel gradients
        const typename Vec2<T>::type *dwr = reinterpret_cast<const typename Vec2<T>::type *>(a.dw);
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const size_t r = (size_t)k * a.pl.stride + i;
            const typename Vec2<T>::type g = dwr[r];
            const StressNb<T> nb = Nb<T>::stress_rec(a.rec, a.pl.pj[r]);
            ss.add(g.x, g.y, nb.m, nb.t11, nb.t12, nb.t22);
        }
    } else if (cnt <= kMaxPairs) {
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
    stress_finish(a, i, live, ki, I, dead, xi, yi, hi, ci, ss.sx.get(), ss.sy.get(), ss.tx.get(), ss.ty.get(), cnt,
                  true);
}

// New hsml of the next step (sle = 2) and its FP32 copy.
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
    return pl;
}

}  // namespace

void launch_kinematic(simp_ctx *c, const State &s, bool diag) {
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
    if (c->prm.precision == SIMP_PREC_MIXED)
        k_kinematic<float><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    else
        k_kinematic<double><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_stress(simp_ctx *c, const State &rhs, const State &base, EpiMode mode) {
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
    if (c->prm.precision == SIMP_PREC_MIXED)
        k_stress<float><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    else
        k_stress<double><<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_step_finish(simp_ctx *c) {
    if (c->prm.sle == 2) {
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
