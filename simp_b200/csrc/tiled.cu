// Pair passes, tiled implementation.
//
// Work unit: a chunk of up to P consecutive particles of one cell row of one
// instance (P = threads per block).  Particles are stored in cell order and a
// cell row's particles are contiguous, so the chunk's halo (the cell rows
// row - R .. row + R over the chunk's columns widened by R) is 2R + 1
// contiguous index ranges.  A block stages its halo in shared memory with
// coalesced loads and then works out of shared memory only:
//   kinematic pass: phase 1 runs the FP32 prefilter (proven margin) over the
//     candidates, the particle's Verlet list or, when that is stale, its
//     cell stencil, into a per-thread list of shared-memory slots; phase 2
//     applies the exact FP64 reference criterion where the prefilter left
//     the pair undecided and runs the pair math.  The pairs also go to HBM
//     for the stress pass; a list-rebuild pass also writes the Verlet lists.
//   stress pass: the pair sums over that list.
// The pairs of a particle are visited in increasing index order, the order
// of the per-particle implementation (passes.cu), so both give the same bits.
// A chunk whose halo does not fit the shared-memory capacity, or whose
// stencil radius exceeds kMaxRadius, runs the same arithmetic from HBM.
#include <algorithm>
#include <cmath>

#include "pass_common.cuh"

namespace simp {

namespace {

using namespace pass;

constexpr int kMaxRadius = 4;
constexpr int kMaxSeg = 2 * kMaxRadius + 1;
constexpr int kMaxTileThreads = 256;

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

// ---- chunk list (after every sort) -----------------------------------------

__global__ void k_count_chunks(int nrows, const int2 *__restrict__ row_map, const Inst *__restrict__ inst,
                               const int *__restrict__ cell_start, int P, int *__restrict__ nch) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nrows) return;
    const int2 qr = row_map[g];
    const Inst &I = inst[qr.x];
    const int k0 = I.base + qr.y * I.ncx;
    const int cnt = cell_start[k0 + I.ncx] - cell_start[k0];
    nch[g] = (cnt + P - 1) / P;
}

__global__ void k_write_chunks(int nrows, const int2 *__restrict__ row_map, const Inst *__restrict__ inst,
                               const int *__restrict__ cell_start, int P, const int *__restrict__ off,
                               Chunk *__restrict__ chunks) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nrows) return;
    const int2 qr = row_map[g];
    const Inst &I = inst[qr.x];
    const int k0 = I.base + qr.y * I.ncx;
    const int a = cell_start[k0], b = cell_start[k0 + I.ncx];
    int o = off[g];
    for (int p = a; p < b; p += P, ++o) chunks[o] = Chunk{p, min(p + P, b), qr.x, qr.y};
}

// ---- halo of a chunk ---------------------------------------------------------

struct Halo {
    int nseg, r0, R, total;
    int lo[kMaxSeg], hi[kMaxSeg], off[kMaxSeg + 1];
};

// Thread 0 of the block: the halo ranges of chunk ch.  fits = 0 when the
// radius or the capacity rules the shared-memory path out.
__device__ void make_halo(const Chunk &ch, const Inst &I, const int *__restrict__ cell_start,
                          const int *__restrict__ cell, int cap, double extra, Halo &h, int &fits) {
    const Grid g = inst_grid(I, cell_start);
    const int R = stencil_radius(I.hmax, I.dmax2_bits, g, extra);
    const int rowbase = I.base + ch.row * I.ncx;
    const int cx0 = cell[ch.p0] - rowbase, cx1 = cell[ch.p1 - 1] - rowbase;
    const int clo = max(cx0 - R, 0), chi = min(cx1 + R, I.ncx - 1);
    const int r0 = max(ch.row - R, 0), r1 = min(ch.row + R, I.ncy - 1);
    h.R = R;
    h.r0 = r0;
    h.nseg = r1 - r0 + 1;
    fits = (R <= kMaxRadius) ? 1 : 0;
    int total = 0;
    if (fits) {
        for (int d = 0; d < h.nseg; ++d) {
            const int k = I.base + (r0 + d) * I.ncx;
            h.lo[d] = cell_start[k + clo];
            h.hi[d] = cell_start[k + chi + 1];
            h.off[d] = total;
            total += h.hi[d] - h.lo[d];
        }
        h.off[h.nseg] = total;
        if (total > cap) fits = 0;
    }
    h.total = total;
}

// Shared-memory slot of particle j (which the halo holds), or -1.
__device__ __forceinline__ int slot_of(const Halo &h, int j) {
    int d = 0;
    while (d < h.nseg - 1 && j >= h.hi[d]) ++d;
    return (j >= h.lo[d] && j < h.hi[d]) ? h.off[d] + (j - h.lo[d]) : -1;
}

__device__ __forceinline__ int index_of(const Halo &h, int slot) {
    int d = 0;
    while (d < h.nseg - 1 && slot >= h.off[d + 1]) ++d;
    return h.lo[d] + (slot - h.off[d]);
}

// Copies halo element k (k < total) with f(global index, slot).
template <class F>
__device__ __forceinline__ void for_halo(const Halo &h, F &&f) {
    for (int d = 0; d < h.nseg; ++d) {
        const int len = h.hi[d] - h.lo[d];
        for (int k = threadIdx.x; k < len; k += blockDim.x) f(h.lo[d] + k, h.off[d] + k);
    }
}

// Candidate slot ranges of particle i (column cx of row `row`): f(s0, s1).
template <class F>
__device__ __forceinline__ void for_candidate_rows(const Halo &h, const Inst &I, const int *__restrict__ cell_start,
                                                   int cx, F &&f) {
    const int c0 = max(cx - h.R, 0), c1 = min(cx + h.R, I.ncx - 1);
    for (int d = 0; d < h.nseg; ++d) {
        const int k = I.base + (h.r0 + d) * I.ncx;
        const int j0 = cell_start[k + c0], j1 = cell_start[k + c1 + 1];
        f(h.off[d] + (j0 - h.lo[d]), h.off[d] + (j1 - h.lo[d]));
    }
}

// ---- kinematic pass ------------------------------------------------------------

template <class T>
struct KinTile {
    double *x, *y, *hs, *vx, *vy;
    float4 *pf;          // FP32 x, y, hsml for the prefilter
    T *m, *mor, *hT;     // hT: hsml in the pair arithmetic type
    unsigned short *list;
};

template <class T>
__host__ __device__ inline size_t kin_smem_bytes(int cap, int threads) {
    return (size_t)cap * (5 * sizeof(double) + sizeof(float4) + 3 * sizeof(T)) +
           (size_t)kListSlots * threads * sizeof(unsigned short);
}

template <class T>
__device__ __forceinline__ KinTile<T> kin_tile(unsigned char *base, int cap) {
    KinTile<T> t;
    t.x = reinterpret_cast<double *>(base);
    t.y = t.x + cap;
    t.hs = t.y + cap;
    t.vx = t.hs + cap;
    t.vy = t.vx + cap;
    t.pf = reinterpret_cast<float4 *>(t.vy + cap);
    t.m = reinterpret_cast<T *>(t.pf + cap);
    t.mor = t.m + cap;
    t.hT = t.mor + cap;
    t.list = reinterpret_cast<unsigned short *>(t.hT + cap);
    return t;
}

// Candidate entries of the per-thread list: a shared-memory slot, with
// kExact set when the FP32 prefilter left the pair undecided (or the bucket
// rule applies): the exact FP64 test then runs with the pair math.
constexpr unsigned short kExact = 0x8000;

template <class T, int SKF>
__global__ void __launch_bounds__(kMaxTileThreads) k_kin_tiled(KinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Halo h;
    __shared__ int fits;
    if ((int)blockIdx.x >= *a.nchunks) return;
    const Chunk ch = a.chunks[blockIdx.x];
    const Inst &I = a.inst[ch.q];
    const int t = threadIdx.x;
    const int i = ch.p0 + t;
    const bool live = i < ch.p1;
    // this pass rebuilds every Verlet list, or the particle's own (a newly
    // admitted basin); the halo then reaches mhsml + skin
    const bool scan = a.sc->list_scan != 0 || (live && a.nl.count[i] < 0);
    const bool any_scan = __syncthreads_or(scan) != 0;
    const double skin = a.sc->skin;
    if (threadIdx.x == 0)
        make_halo(ch, I, a.cell_start, a.cell, a.cap, any_scan ? I.hmax + skin : 0.0, h, fits);
    __syncthreads();
    const State &s = a.s;
    const Phys &P = a.P;
    const bool dead = inst_dead(I.flags);
    const KinTile<T> tl = kin_tile<T>(smem, a.cap);
    if (fits) {
        for_halo(h, [&](int j, int k) {
            const double2 q = s.xy[j], v = s.vxy[j];
            const KinNb<T> nb = Nb<T>::kin(s, j, T(-1));
            tl.x[k] = q.x;
            tl.y[k] = q.y;
            tl.hs[k] = s.hs[j];
            tl.vx[k] = v.x;
            tl.vy[k] = v.y;
            tl.pf[k] = s.pf[j];
            tl.m[k] = nb.m;
            tl.mor[k] = nb.mor;
            tl.hT[k] = nb.h;
        });
    }
    __syncthreads();
    if (!live) return;
    if (a.sc->list_scan && i == 0) atomicExch(&a.sc->dlist2_bits, 0ull);
    const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
    const double xi = pc.xi, yi = pc.yi, hi = pc.hi;
    const double vxi = s.vx[i], vyi = s.vy[i];
    const double inv_hi = 1.0 / hi;
    const NbrList &nl = a.nl;
    const PairList &pl = a.pl;
    KinSums<T> ks;
    int npairs = 0;
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    typename Vec2<T>::type *dwr = reinterpret_cast<typename Vec2<T>::type *>(a.dw);
    // row: the pair's position in the particle's pair list (its kernel
    // gradient is kept for the stress pass when row < kDwRows)
    auto pair_terms = [&](int row, double xj, double yj, T hj, double vxj, double vyj, T mj, T mrj) {
        const PairGeom<T> pg = pair_geom<T, false, SKF>(P, (T)(xi - xj), (T)(yi - yj), hiT, inv_hiT, hj);
        const T dwx = pg.gfac * pg.dx, dwy = pg.gfac * pg.dy;
        if (dwr && row < kDwRows) dwr[(size_t)row * pl.stride + i] = Vec2<T>::make(dwx, dwy);
        ks.add(dwx, dwy, (T)(vxi - vxj), (T)(vyi - vyj), mj, mrj);
    };
    if (dead) {
        // a basin flagged non-finite is carried without a search
        if (scan) {
            nl.count[i] = 0;
            nl.xl[i] = xi;
            nl.yl[i] = yi;
        }
    } else if (fits) {
        const int own = slot_of(h, i);
        const bool pre = pc.use_f32;
        const float up = 1.0f + pc.margin, down = 1.0f - pc.margin;
        const unsigned short decided = pc.br.on ? kExact : 0;
        int cnt = 0;          // candidates in the list
        // Phase 2 over the list: exact test where needed, then the pair
        // math; the confirmed pairs are compacted to the list front (final
        // batch) or written out at once (a full list in mid-scan).
        auto flush = [&](bool final) {
            int kept = 0;
#pragma unroll 2
            for (int k = 0; k < cnt; ++k) {
                const unsigned short e = tl.list[k * blockDim.x + t];
                const int sl = e & 0x7fff;
                if (sl == own) continue;
                if (!SIMP_IN_RANGE(sl, 0, a.cap, SITE_TILE)) continue;
                const double xj = tl.x[sl], yj = tl.y[sl], hj = tl.hs[sl];
                if (e & kExact) {
                    double r;
                    const double mh = __dmul_rn(__dadd_rn(hi, hj), 0.5);
                    if (!pair_test(__dsub_rn(xi, xj), __dsub_rn(yi, yj), mh, &r)) continue;
                    if (!bin_rule_ok(pc.br, xj, yj)) continue;
                }
                if (final)
                    tl.list[kept * blockDim.x + t] = (unsigned short)sl;
                else if (npairs < kMaxPairs)
                    pl.pj[(size_t)npairs * pl.stride + i] = index_of(h, sl);
                pair_terms(npairs, xj, yj, tl.hT[sl], tl.vx[sl], tl.vy[sl], tl.m[sl], tl.mor[sl]);
                ++kept;
                ++npairs;
            }
            cnt = final ? kept : 0;
        };
        // Phase 1: FP32 prefilter of a candidate slot into the list.
        auto cand = [&](int sl) {
            const float4 q = tl.pf[sl];
            const float dx = pc.xif - q.x, dy = pc.yif - q.y;
            const float mf = 0.5f * (pc.hif + q.z);
            const float sf = fmaf(dx, dx, dy * dy), tf = mf * mf;
            if (pre && sf > tf * up) return;
            const unsigned short fl = (pre && sf < tf * down) ? decided : kExact;
            tl.list[cnt * blockDim.x + t] = (unsigned short)sl | fl;
            if (++cnt == kListSlots) flush(false);
        };
        const int cx = a.cell[i] - (I.base + ch.row * I.ncx);
        if (scan) {
            // rebuild the Verlet list: members are the candidates not
            // certainly beyond mhsml + skin (FP32, with margin)
            const float skinf = (float)skin, grow = up;
            int total = 0;
            for_candidate_rows(h, I, a.cell_start, cx, [&](int s0, int s1) {
                for (int sl = s0; sl < s1; ++sl) {
                    if (sl == own) continue;
                    const float4 q = tl.pf[sl];
                    const float dxf = pc.xif - q.x, dyf = pc.yif - q.y;
                    const float lim = 0.5f * (pc.hif + q.z) + skinf;
                    if (dxf * dxf + dyf * dyf > lim * lim * grow) continue;
                    if (total < kMaxNbr) nl.nbr[(size_t)total * nl.stride + i] = index_of(h, sl);
                    ++total;
                    cand(sl);
                }
            });
            nl.count[i] = total;
            nl.xl[i] = xi;
            nl.yl[i] = yi;
        } else {
            const int lcnt = nl.count[i];
            const double dxl = xi - nl.xl[i], dyl = yi - nl.yl[i];
            const double mine = sqrt(dxl * dxl + dyl * dyl);
            const double all = sqrt(bitsd(a.sc->dlist2_bits));
            if (lcnt <= kMaxNbr && (mine + all) * (1.0 + 1e-9) < skin) {
                // the list still holds every pair; a member outside the halo
                // is outside the stencil, so not a pair
#pragma unroll 4
                for (int k = 0; k < lcnt; ++k) {
                    const int sl = slot_of(h, nl.nbr[(size_t)k * nl.stride + i]);
                    if (sl >= 0) cand(sl);
                }
            } else {
                for_candidate_rows(h, I, a.cell_start, cx, [&](int s0, int s1) {
                    for (int sl = s0; sl < s1; ++sl) cand(sl);
                });
            }
        }
        const int before = npairs;
        flush(true);
        // the last batch's pairs, one coalesced row per k
        for (int k = 0; k < cnt; ++k) {
            const int row = before + k;
            if (row < kMaxPairs) pl.pj[(size_t)row * pl.stride + i] = index_of(h, tl.list[k * blockDim.x + t]);
        }
    } else {
        // halo too large for shared memory: the same pairs from HBM
        auto on_pair = [&](int j) {
            if (npairs < kMaxPairs) pl.pj[(size_t)npairs * pl.stride + i] = j;
            const double2 q = s.xy[j], v = s.vxy[j];
            const KinNb<T> nb = Nb<T>::kin(s, j, T(-1));
            pair_terms(npairs, q.x, q.y, nb.h, v.x, v.y, nb.m, nb.mor);
            ++npairs;
        };
        if (scan) {
            const float skinf = (float)skin, grow = 1.0f + pc.margin;
            int total = 0;
            const Grid g = inst_grid(I, a.cell_start);
            for_stencil(g, i, a.cell[i], stencil_radius(I.hmax, I.dmax2_bits, g, I.hmax + skin), [&](int j) {
                const float4 f = s.pf[j];
                const float dxf = pc.xif - f.x, dyf = pc.yif - f.y;
                const float lim = 0.5f * (pc.hif + f.z) + skinf;
                if (dxf * dxf + dyf * dyf > lim * lim * grow) return;
                if (total < kMaxNbr) nl.nbr[(size_t)total * nl.stride + i] = j;
                ++total;
                if (is_pair(s, pc, j)) on_pair(j);
            });
            nl.count[i] = total;
            nl.xl[i] = xi;
            nl.yl[i] = yi;
        } else {
            for_each_current_pair(s, nl, a.sc, i, a.cell[i], pc, on_pair);
        }
    }
    pl.count[i] = npairs;
    kin_rheology(a, i, -ks.dv.get(), -ks.g1.get(), -ks.g2.get(), -ks.g3.get(), -ks.g4.get());
}

// ---- stress pass ----------------------------------------------------------------

template <class T>
struct StressTile {
    double *x, *y;
    T *hT, *m, *t11, *t12, *t22;
};

template <class T>
__host__ __device__ inline size_t stress_smem_bytes(int cap) {
    return (size_t)cap * (2 * sizeof(double) + 5 * sizeof(T));
}

template <class T>
__device__ __forceinline__ StressTile<T> stress_tile(unsigned char *base, int cap) {
    StressTile<T> t;
    t.x = reinterpret_cast<double *>(base);
    t.y = t.x + cap;
    t.hT = reinterpret_cast<T *>(t.y + cap);
    t.m = t.hT + cap;
    t.t11 = t.m + cap;
    t.t12 = t.t11 + cap;
    t.t22 = t.t12 + cap;
    return t;
}

template <class T, int SKF>
__global__ void __launch_bounds__(kMaxTileThreads) k_stress_tiled(StressArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Halo h;
    __shared__ int fits;
    if ((int)blockIdx.x >= *a.nchunks) {
        if (a.mode != EPI_RATES) lists_block_done(a);   // every block counts
        return;
    }
    const Chunk ch = a.chunks[blockIdx.x];
    const Inst &I = a.inst[ch.q];
    if (threadIdx.x == 0) make_halo(ch, I, a.cell_start, a.cell, a.cap, 0.0, h, fits);
    __syncthreads();
    const State &s = a.rhs;
    const Phys &P = a.P;
    const StressTile<T> tl = stress_tile<T>(smem, a.cap);
    if (fits) {
        for_halo(h, [&](int j, int k) {
            const double2 q = s.xy[j];
            const StressNb<T> nb = Nb<T>::stress(s, a.rec, j, T(-1));
            tl.x[k] = q.x;
            tl.y[k] = q.y;
            tl.hT[k] = nb.h;
            tl.m[k] = nb.m;
            tl.t11[k] = nb.t11;
            tl.t12[k] = nb.t12;
            tl.t22[k] = nb.t22;
        });
    }
    __syncthreads();
    const int i0 = ch.p0 + (int)threadIdx.x;
    const bool live = i0 < ch.p1;
    const int i = live ? i0 : ch.p1 - 1;   // idle lanes mirror the chunk's last particle
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const double inv_hi = 1.0 / hi;
    const int ci = a.cell[i];
    const bool dead = inst_dead(I.flags);
    StressSums<T> ss;
    const T hiT = Nb<T>::h(s, i), inv_hiT = (T)inv_hi;
    auto terms = [&](double xj, double yj, T hj, T mj, T t11, T t12, T t22) {
        const PairGeom<T> pg = pair_geom<T, false, SKF>(P, (T)(xi - xj), (T)(yi - yj), hiT, inv_hiT, hj);
        ss.add(pg.gfac * pg.dx, pg.gfac * pg.dy, mj, t11, t12, t22);
    };
    auto global_terms = [&](int j) {
        const double2 q = s.xy[j];
        const StressNb<T> nb = Nb<T>::stress(s, a.rec, j, T(-1));
        terms(q.x, q.y, nb.h, nb.m, nb.t11, nb.t12, nb.t22);
    };
    auto any_terms = [&](int j) {
        const int sl = fits ? slot_of(h, j) : -1;
        if (sl >= 0) terms(tl.x[sl], tl.y[sl], tl.hT[sl], tl.m[sl], tl.t11[sl], tl.t12[sl], tl.t22[sl]);
        else global_terms(j);
    };
    int cnt = live ? a.pl.count[i] : 0;
    if (dead || !live) {
        cnt = 0;
    } else if (a.dw && cnt <= kDwRows) {
        // the kinematic pass kept these pairs' kernel gradients
        const typename Vec2<T>::type *dwr = reinterpret_cast<const typename Vec2<T>::type *>(a.dw);
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) {
            const size_t r = (size_t)k * a.pl.stride + i;
            const typename Vec2<T>::type g = dwr[r];
            const int j = a.pl.pj[r];
            const int sl = fits ? slot_of(h, j) : -1;
            if (sl >= 0) {
                ss.add(g.x, g.y, tl.m[sl], tl.t11[sl], tl.t12[sl], tl.t22[sl]);
            } else {
                const StressNb<T> nb = Nb<T>::stress_rec(a.rec, j);
                ss.add(g.x, g.y, nb.m, nb.t11, nb.t12, nb.t22);
            }
        }
    } else if (cnt <= kMaxPairs) {
#pragma unroll 4
        for (int k = 0; k < cnt; ++k) any_terms(a.pl.pj[(size_t)k * a.pl.stride + i]);
    } else {
        cnt = 0;
        const PairCtx pc = pair_ctx(s, a.sc, I, a.cell_start, i);
        const Grid g = inst_grid(I, a.cell_start);
        for_stencil(g, i, ci, stencil_radius(I.hmax, I.dmax2_bits, g, 0.0), [&](int j) {
            if (!is_pair(s, pc, j)) return;
            any_terms(j);
            ++cnt;
        });
    }
    // (a retired basin's particles are not written any more)
    stress_finish<SKF>(a, i, live && !(I.flags & FLAG_RETIRED), ch.q, I, dead, xi, yi, hi, ci, ss.sx.get(),
                       ss.sy.get(), ss.tx.get(), ss.ty.get(), cnt, true);
}

int chunk_bound(const simp_ctx *c) {
    return c->n / std::max(1, c->tile_threads) + c->total_rows + 1;
}

}  // namespace

// Chunk list of the current cell lists (after every sort).
void build_chunks(simp_ctx *c) {
    const int rows = c->total_rows;
    cudaStream_t s = c->stream;
    if (rows == 0) {
        cudaMemsetAsync(c->chunk_off, 0, sizeof(int), s);
        return;
    }
    const int P = c->tile_threads;
    k_count_chunks<<<nblk(rows, 256), 256, 0, s>>>(rows, c->row_map, c->inst_dev, c->cell_start, P, c->chunk_cnt);
    launch_scan_i32(c->chunk_cnt, c->chunk_off, rows, c->scan_tmp, s);
    k_write_chunks<<<nblk(rows, 256), 256, 0, s>>>(rows, c->row_map, c->inst_dev, c->cell_start, P, c->chunk_off,
                                                   c->chunks);
    c->launches += 2 + kScanKernels;
}

template <class T, int SKF>
cudaError_t set_tile_smem(size_t kb, size_t sb) {
    cudaError_t e = cudaFuncSetAttribute(k_kin_tiled<T, SKF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kb);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stress_tiled<T, SKF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
    return e;
}

template <class T, int SKF>
void launch_tiled(simp_ctx *c, int pass, int grid, size_t sm, const KinArgs *ka, const StressArgs *sa) {
    if (pass == 0) k_kin_tiled<T, SKF><<<grid, c->tile_threads, sm, c->stream>>>(*ka);
    else k_stress_tiled<T, SKF><<<grid, c->tile_threads, sm, c->stream>>>(*sa);
}

void launch_tiled_any(simp_ctx *c, int pass, int grid, size_t sm, const KinArgs *ka, const StressArgs *sa) {
    const bool mixed = c->prm.precision == SIMP_PREC_MIXED;
    switch (skf_compiled(c->prm.skf)) {
        case SIMP_SKF_CUBIC:
            if (mixed) launch_tiled<float, SIMP_SKF_CUBIC>(c, pass, grid, sm, ka, sa);
            else launch_tiled<double, SIMP_SKF_CUBIC>(c, pass, grid, sm, ka, sa);
            break;
        case SIMP_SKF_WENDLAND_C6:
            if (mixed) launch_tiled<float, SIMP_SKF_WENDLAND_C6>(c, pass, grid, sm, ka, sa);
            else launch_tiled<double, SIMP_SKF_WENDLAND_C6>(c, pass, grid, sm, ka, sa);
            break;
        default:
            if (mixed) launch_tiled<float, 0>(c, pass, grid, sm, ka, sa);
            else launch_tiled<double, 0>(c, pass, grid, sm, ka, sa);
    }
}

size_t tiled_smem_bytes(int precision, int pass, int cap, int threads) {
    if (pass == 0)
        return precision == SIMP_PREC_MIXED ? kin_smem_bytes<float>(cap, threads)
                                            : kin_smem_bytes<double>(cap, threads);
    return precision == SIMP_PREC_MIXED ? stress_smem_bytes<float>(cap) : stress_smem_bytes<double>(cap);
}

int tiled_configure(simp_ctx *c) {
    const size_t kb = tiled_smem_bytes(c->prm.precision, 0, c->tile_cap, c->tile_threads);
    const size_t sb = tiled_smem_bytes(c->prm.precision, 1, c->tile_cap, c->tile_threads);
    cudaError_t e;
    const bool mixed = c->prm.precision == SIMP_PREC_MIXED;
    switch (skf_compiled(c->prm.skf)) {
        case SIMP_SKF_CUBIC:
            e = mixed ? set_tile_smem<float, SIMP_SKF_CUBIC>(kb, sb) : set_tile_smem<double, SIMP_SKF_CUBIC>(kb, sb);
            break;
        case SIMP_SKF_WENDLAND_C6:
            e = mixed ? set_tile_smem<float, SIMP_SKF_WENDLAND_C6>(kb, sb)
                      : set_tile_smem<double, SIMP_SKF_WENDLAND_C6>(kb, sb);
            break;
        default:
            e = mixed ? set_tile_smem<float, 0>(kb, sb) : set_tile_smem<double, 0>(kb, sb);
    }
    if (e != cudaSuccess) return simp_cuda_check(c, e, "cudaFuncSetAttribute (tile shared memory)");
    return SIMP_OK;
}

void launch_kinematic_tiled(simp_ctx *c, const KinArgs &a0) {
    KinArgs a = a0;
    a.chunks = c->chunks;
    a.nchunks = c->chunk_off + c->total_rows;
    a.cap = c->tile_cap;
    const int grid = chunk_bound(c);
    const size_t sm = tiled_smem_bytes(c->prm.precision, 0, c->tile_cap, c->tile_threads);
    launch_tiled_any(c, 0, grid, sm, &a, nullptr);
    c->launches += 1;
}

void launch_stress_tiled(simp_ctx *c, const StressArgs &a0) {
    StressArgs a = a0;
    a.chunks = c->chunks;
    a.nchunks = c->chunk_off + c->total_rows;
    a.cap = c->tile_cap;
    const int grid = chunk_bound(c);
    const size_t sm = tiled_smem_bytes(c->prm.precision, 1, c->tile_cap, c->tile_threads);
    launch_tiled_any(c, 1, grid, sm, nullptr, &a);
    c->launches += 1;
}

}  // namespace simp
