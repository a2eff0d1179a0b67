// Cell list of the neighbour search (replaces nnps.f90:155-517 bucket_search).
//
// The reference bins particles into square buckets of side 2 * min(hsml)
// serially and scans a half stencil of buckets (nnps.f90:211-412).  Here the
// particles are sorted once into a uniform grid of side cs = (1 + skin) *
// max(hsml) and stay in that order; each pair pass scans the (2R+1)^2 cells
// around a particle, R computed on the device from the exact bounds hmax and
// the maximal displacement since the sort (common.cuh: stencil_radius), so
// the cell list is a superset of every pair at every step without a host
// round trip.  The exact reference criterion (and its bucket rule) is applied
// per candidate in the passes, so the pair set equals the reference's.
//
// Sort: counting sort on cell keys (one radix digit of width log2(ncells)):
// key histogram, exclusive prefix scan, scatter, then a per-cell sort by
// original particle index so the order is deterministic.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "ctx.h"

namespace simp {

namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

// Exclusive scan, phase 1: per-tile sums.
__global__ void scan_tile_sums(const int *__restrict__ in, int n, int *__restrict__ sums) {
    __shared__ int red[kScanBlock / 32];
    const int base = blockIdx.x * kScanTile;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + k * kScanBlock + threadIdx.x;
        s += (i < n) ? in[i] : 0;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < kScanBlock / 32) ? red[threadIdx.x] : 0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) sums[blockIdx.x] = s;
    }
}

// Block-wide exclusive scan of one value per thread; returns the total.
__device__ int block_exclusive_scan(int v, int *smem_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) smem_warp[warp] = incl;
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (warp == 0) {
        int w = (lane < nw) ? smem_warp[lane] : 0;
        int wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < nw) smem_warp[lane] = wi - w;
        if (lane == 31) smem_warp[32] = wi;
    }
    __syncthreads();
    const int res = smem_warp[warp] + incl - v;
    __syncthreads();
    return res;  // the block total stays in smem_warp[32] until the next call
}

// Phase 2: exclusive scan of the tile sums in one block (sequential chunks).
__global__ void scan_sums(int *sums, int nt) {
    __shared__ int sw[33];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nt; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = (i < nt) ? sums[i] : 0;
        const int ex = block_exclusive_scan(v, sw);
        const int tot = sw[32];
        __syncthreads();
        if (i < nt) sums[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

// Phase 3: scan within tiles plus tile offset; out has n + 1 entries.
__global__ void scan_tiles(const int *__restrict__ in, int n, const int *__restrict__ sums,
                           int *__restrict__ out) {
    __shared__ int sw[33];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int loc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + k;
        v[k] = (i < n) ? in[i] : 0;
        loc += v[k];
    }
    const int ex = block_exclusive_scan(loc, sw) + sums[blockIdx.x];
    int run = ex;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

__global__ void scan_total(const int *__restrict__ in, int n, int *__restrict__ out) {
    out[n] = (n > 0) ? out[n - 1] + in[n - 1] : 0;
}

// Cell key of each particle from its sort position and its instance's grid;
// particles being removed (instance -1) go to the dump key after all cells.
__global__ void k_keys(int n, const double *__restrict__ xr, const double *__restrict__ yr,
                       const int *__restrict__ pinst, const Inst *__restrict__ inst, int dump_key,
                       int *__restrict__ key, int *__restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int q = pinst[i];
    int k = dump_key;
    if (q >= 0) {
        const Inst &I = inst[q];
        const int cx = clampi((int)floor((xr[i] - I.x0) * I.inv_cs), 0, I.ncx - 1);
        const int cy = clampi((int)floor((yr[i] - I.y0) * I.inv_cs), 0, I.ncy - 1);
        k = I.base + cy * I.ncx + cx;
    }
    key[i] = k;
    atomicAdd(&cnt[k], 1);
}

// Instances due for a re-sort take their current positions as sort
// positions; a basin flagged non-finite keeps its old (finite) ones.
__global__ void k_refresh_sortpos(int n, const int *__restrict__ pinst, DueMask due, const Inst *__restrict__ inst,
                                  const double *__restrict__ x, const double *__restrict__ y,
                                  double *__restrict__ xr, double *__restrict__ yr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int q = pinst[i];
    if (q < 0 || !((due.w[q >> 6] >> (q & 63)) & 1ull)) return;
    if (inst_dead(inst[q].flags)) return;
    xr[i] = x[i];
    yr[i] = y[i];
}

__global__ void k_reset_inst_disp(Inst *inst, int ninst, DueMask due) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ninst) return;
    if ((due.w[q >> 6] >> (q & 63)) & 1ull) inst[q].dmax2_bits = 0ull;
}

__global__ void k_scatter(int n, const int *__restrict__ key, const int *__restrict__ start,
                          int *__restrict__ cnt, int *__restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    const int slot = atomicSub(&cnt[k], 1) - 1;
    const int pos = start[k] + slot;
    if (!SIMP_IN_RANGE(pos, 0, n, SITE_SORT)) return;
    perm[pos] = i;
}

// Sort each cell's entries by original particle index (insertion sort; a
// cell holds a few tens of particles).
__global__ void k_cell_sort(int ncells, const int *__restrict__ start, int *__restrict__ perm,
                            const int *__restrict__ id) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const int a = start[c], b = start[c + 1];
    for (int k = a + 1; k < b; ++k) {
        const int v = perm[k];
        const int kv = id[v];
        int j = k - 1;
        while (j >= a && id[perm[j]] > kv) { perm[j + 1] = perm[j]; --j; }
        perm[j + 1] = v;
    }
}

constexpr int kGathered = 14;   // (the last two only with Benz's kept drhodt and the kept kernel_zero)
struct Gather {
    const double *src[kGathered];
    double *dst[kGathered];
};

__device__ __forceinline__ bool is_due(const DueMask &m, int q) {
    return q >= 0 && ((m.w[q >> 6] >> (q & 63)) & 1ull);
}

// Positions of the new order whose particle may differ from the old one:
// every position from `from` on (an admission appends a basin there; a
// removal shifts the basins after it down), and those of the due basins
// (each basin keeps its range of positions; the others keep their order).
__device__ __forceinline__ bool moves(int from, const DueMask &due, const int *pinst, int k) {
    return k >= from || is_due(due, pinst[k]);
}

// New order into scratch; inv[old] = new for every moved particle.
__global__ void k_gather(int kept, int from, DueMask due, const int *__restrict__ perm, Gather gd,
                         const int *__restrict__ key, int *__restrict__ cell_out, const int *__restrict__ id_in,
                         int *__restrict__ id_out, const int *__restrict__ pinst_in, int *__restrict__ pinst_out,
                         int *__restrict__ inv) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kept || !moves(from, due, pinst_in, k)) return;
    const int o = perm[k];
#pragma unroll
    for (int a = 0; a < kGathered; ++a)
        if (gd.src[a]) gd.dst[a][k] = gd.src[a][o];
    cell_out[k] = key[o];
    id_out[k] = id_in[o];
    pinst_out[k] = pinst_in[o];
    inv[o] = k;
}

// Verlet-list rows of the moved particles: each entry renamed to the new
// index and the row re-sorted, so a row lists its members in increasing
// index order exactly as a fresh scan of the cell stencil would.  An entry
// whose new index cannot be confirmed (perm[inv[v]] != v) turns the row into
// an overflowed one, which the kinematic pass answers by a stencil scan.
__global__ void k_remap_lists(int kept, int from, DueMask due, const int *__restrict__ pinst,
                              const int *__restrict__ perm, const int *__restrict__ inv, int n_old,
                              NbrList nl, int *__restrict__ nbr_out, int *__restrict__ cnt_out,
                              double *__restrict__ xl_out, double *__restrict__ yl_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kept || !moves(from, due, pinst, k)) return;
    const int o = perm[k];
    int cnt = nl.count[o];
    xl_out[k] = nl.xl[o];
    yl_out[k] = nl.yl[o];
    if (cnt < 0) {
        // (a particle whose list is still to be built keeps that mark)
    } else if (cnt <= kMaxNbr) {
        int row[kMaxNbr];
        for (int e = 0; e < cnt; ++e) {
            const int v = nl.nbr[(size_t)e * nl.stride + o];
            int w = -1;
            if (v >= 0 && v < n_old) {
                w = inv[v];
                if (w < 0 || w >= kept || perm[w] != v) w = -1;
            }
            if (w < 0) { cnt = kMaxNbr + 1; break; }
            int j = e - 1;
            while (j >= 0 && row[j] > w) { row[j + 1] = row[j]; --j; }
            row[j + 1] = w;
        }
        if (cnt <= kMaxNbr)
            for (int e = 0; e < cnt; ++e) nbr_out[(size_t)e * nl.stride + k] = row[e];
    } else {
        cnt = kMaxNbr + 1;
    }
    cnt_out[k] = cnt;
}

__global__ void k_put_back_lists(int kept, int from, DueMask due, const int *__restrict__ pinst, NbrList nl,
                                 const int *__restrict__ nbr_in, const int *__restrict__ cnt_in,
                                 const double *__restrict__ xl_in, const double *__restrict__ yl_in) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kept || !moves(from, due, pinst, k)) return;
    const int cnt = cnt_in[k];
    nl.count[k] = cnt;
    nl.xl[k] = xl_in[k];
    nl.yl[k] = yl_in[k];
    for (int e = 0; e < cnt && cnt <= kMaxNbr; ++e) nl.nbr[(size_t)e * nl.stride + k] = nbr_in[(size_t)e * nl.stride + k];
}

// Scratch back into the state arrays (pointers stay fixed so the captured
// step graph remains valid), with the FP32 copies of the moved particles.
__global__ void k_put_back(int kept, int from, DueMask due, Gather gd, State s, const int *__restrict__ id_new,
                           int *__restrict__ id, const int *__restrict__ pinst_new, int *__restrict__ pinst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kept || !moves(from, due, pinst, k)) return;
#pragma unroll
    for (int a = 0; a < kGathered; ++a)
        if (gd.src[a]) const_cast<double *>(gd.src[a])[k] = gd.dst[a][k];
    id[k] = id_new[k];
    pinst[k] = pinst_new[k];
    refresh_views(s, k);
}

// After a sort: displacement since the sort restarts; the Verlet lists are
// rebuilt by the next kinematic pass unless they were renamed.
__global__ void k_reset_disp(Scalars *sc, int lists_kept) {
    sc->dmax2_bits = 0ull;
    if (!lists_kept) {
        sc->dlist2_bits = 0ull;
        sc->list_scan = 1;
    }
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

size_t scan_tmp_bytes(int n) {
    const int nt = (n + kScanTile - 1) / kScanTile;
    return (size_t)(nt + 1) * sizeof(int);
}

// Exclusive scan of n ints into out[0..n] (out[n] = total).
void launch_scan_i32(const int *in, int *out, int n, void *tmp, cudaStream_t s) {
    const int nt = std::max(1, (n + kScanTile - 1) / kScanTile);
    int *sums = (int *)tmp;
    scan_tile_sums<<<nt, kScanBlock, 0, s>>>(in, n, sums);
    scan_sums<<<1, 1024, 0, s>>>(sums, nt);
    scan_tiles<<<nt, kScanBlock, 0, s>>>(in, n, sums, out);
    scan_total<<<1, 1, 0, s>>>(in, n, out);
}

// Sorts the particles into cell order (instance-major keys, within a cell by
// global id).  Instances in `due` re-bin at their current positions; the
// others keep their sort positions, so their order does not change.
// Positions from `from` on are rewritten (after an admission or a removal:
// the first position whose basin changed), before it only the due
// instances' ranges move.  Particles of removed instances (instance -1) end
// up after all others and are dropped: c->n shrinks to the kept count.  The
// Verlet lists follow the particles unless `new_lists` (or no list was built
// yet), in which case the next kinematic pass rebuilds them all.
int rebuild(simp_ctx *c, const DueMask &due, int from, bool new_lists) {
    SIMP_RANGE("re-sort");
    const int n = c->n;
    cudaStream_t s = c->stream;
    const int B = 256;
    const int nkeys = c->total_cells + 1;   // + the dump key
    const size_t MX = (size_t)std::max(c->maxn, c->maxnb);
    int *key = c->itmp;
    int *id_new = c->itmp + MX;
    int *pinst_new = c->itmp + 2 * MX;
    int *inv = c->itmp + 3 * MX;
    int *cnt_new = c->itmp + 4 * MX;
    int kept = 0;
    for (const InstHost &h : c->insts)
        if (h.active) kept += h.n;
    const bool keep_lists = c->lists_valid && !new_lists;
    if (n > 0) {
        k_refresh_sortpos<<<nblk(n, B), B, 0, s>>>(n, c->pinst, due, c->inst_dev, c->s0.x, c->s0.y, c->xr, c->yr);
        k_reset_inst_disp<<<nblk(c->ninst, 128), 128, 0, s>>>(c->inst_dev, c->ninst, due);
        SIMP_CUDA(c, cudaMemsetAsync(c->cnt, 0, sizeof(int) * (size_t)nkeys, s));
        k_keys<<<nblk(n, B), B, 0, s>>>(n, c->xr, c->yr, c->pinst, c->inst_dev, c->total_cells, key, c->cnt);
        launch_scan_i32(c->cnt, c->cell_start, nkeys, c->scan_tmp, s);
        k_scatter<<<nblk(n, B), B, 0, s>>>(n, key, c->cell_start, c->cnt, c->perm);
        // (the dump key is not ordered: its particles are dropped)
        if (c->total_cells > 0)
            k_cell_sort<<<nblk(c->total_cells, 128), 128, 0, s>>>(c->total_cells, c->cell_start, c->perm, c->id);
        double *srcs[kGathered] = {c->s0.x, c->s0.y, c->s0.vx, c->s0.vy, c->s0.m, c->s0.rho,
                                   c->s0.mor, c->s0.h, c->s0.A, c->s0.hs, c->xr, c->yr, c->drhodt, c->k0};
        Gather gd;
        for (int a = 0; a < kGathered; ++a) {
            gd.src[a] = srcs[a];
            gd.dst[a] = c->tmp + (size_t)a * MX;
        }
        c->launches += 7 + kScanKernels;
        if (kept > 0) {
            k_gather<<<nblk(kept, B), B, 0, s>>>(kept, from, due, c->perm, gd, key, c->cell, c->id, id_new,
                                                 c->pinst, pinst_new, inv);
            c->launches += 1;
            if (keep_lists) {
                NbrList nl{c->nbr, c->nbr_count, c->xl, c->yl, c->maxn};
                double *xl_new = c->tmp + 14 * MX, *yl_new = c->tmp + 15 * MX;
                k_remap_lists<<<nblk(kept, 128), 128, 0, s>>>(kept, from, due, c->pinst, c->perm, inv, n, nl,
                                                              c->nbr_tmp, cnt_new, xl_new, yl_new);
                k_put_back_lists<<<nblk(kept, B), B, 0, s>>>(kept, from, due, c->pinst, nl, c->nbr_tmp, cnt_new,
                                                             xl_new, yl_new);
                c->launches += 2;
            }
            k_put_back<<<nblk(kept, B), B, 0, s>>>(kept, from, due, gd, c->s0, id_new, c->id, pinst_new, c->pinst);
            c->launches += 1;
        }
    } else {
        SIMP_CUDA(c, cudaMemsetAsync(c->cell_start, 0, sizeof(int) * (size_t)(nkeys + 1), s));
    }
    k_reset_disp<<<1, 1, 0, s>>>(c->sc, keep_lists ? 1 : 0);
    c->launches += 1;
    if (!keep_lists) c->lists_valid = false;
    c->n = kept;
    if (c->pass_impl == SIMP_PASSES_TILED) build_chunks(c);
    SIMP_CUDA(c, cudaGetLastError());
    c->rebuilds += 1;
    return SIMP_OK;
}

}  // namespace simp
