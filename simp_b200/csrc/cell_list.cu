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

__global__ void k_keys(int n, const double *__restrict__ x, const double *__restrict__ y,
                       Grid g, int *__restrict__ key, int *__restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cx = clampi((int)floor((x[i] - g.x0) * g.inv_cs), 0, g.ncx - 1);
    const int cy = clampi((int)floor((y[i] - g.y0) * g.inv_cs), 0, g.ncy - 1);
    const int k = cy * g.ncx + cx;
    key[i] = k;
    atomicAdd(&cnt[k], 1);
}

__global__ void k_scatter(int n, const int *__restrict__ key, const int *__restrict__ start,
                          int *__restrict__ cnt, int *__restrict__ perm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    const int slot = atomicSub(&cnt[k], 1) - 1;
    perm[start[k] + slot] = i;
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

struct Gather {
    const double *src[10];
    double *dst[10];
};

__global__ void k_gather(int n, const int *__restrict__ perm, Gather gd, int narr,
                         const int *__restrict__ key, int *__restrict__ cell_out,
                         const int *__restrict__ id_in, int *__restrict__ id_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = perm[k];
    for (int a = 0; a < narr; ++a) gd.dst[a][k] = gd.src[a][o];
    cell_out[k] = key[o];
    id_out[k] = id_in[o];
}

// Rebuild-time positions, inverse index and the FP32 copies of the sorted state.
__global__ void k_finish_rebuild(int n, State s, double *__restrict__ xr, double *__restrict__ yr,
                                 const int *__restrict__ id, int *__restrict__ inv_id) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double x = s.x[k], y = s.y[k];
    xr[k] = x;
    yr[k] = y;
    s.xf[k] = (float)x;
    s.yf[k] = (float)y;
    s.hsf[k] = (float)s.hs[k];
    inv_id[id[k]] = k;
}

// After a sort the cell-order indices in the Verlet lists are stale.
__global__ void k_reset_disp(Scalars *sc) {
    sc->dmax2_bits = 0ull;
    sc->dlist2_bits = 0ull;
    sc->list_scan = 1;
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

int rebuild(simp_ctx *c) {
    const int n = c->n;
    const Grid &g = c->grid;
    const int ncells = g.ncx * g.ncy;
    cudaStream_t s = c->stream;
    const int B = 256;
    int *key = c->itmp;                 // n ints
    int *id_new = c->itmp + c->maxn;    // n ints
    SIMP_CUDA(c, cudaMemsetAsync(c->cnt, 0, sizeof(int) * (size_t)ncells, s));
    k_keys<<<nblk(n, B), B, 0, s>>>(n, c->s0.x, c->s0.y, g, key, c->cnt);
    launch_scan_i32(c->cnt, c->cell_start, ncells, c->scan_tmp, s);
    k_scatter<<<nblk(n, B), B, 0, s>>>(n, key, c->cell_start, c->cnt, c->perm);
    k_cell_sort<<<nblk(ncells, 128), 128, 0, s>>>(ncells, c->cell_start, c->perm, c->id);
    // gather state into scratch, then copy back (pointers stay fixed so the
    // captured step graph remains valid)
    double *srcs[10] = {c->s0.x, c->s0.y, c->s0.vx, c->s0.vy, c->s0.m,
                        c->s0.rho, c->s0.mor, c->s0.h, c->s0.A, c->s0.hs};
    Gather gd;
    for (int a = 0; a < 10; ++a) { gd.src[a] = srcs[a]; gd.dst[a] = c->tmp + (size_t)a * c->maxn; }
    k_gather<<<nblk(n, B), B, 0, s>>>(n, c->perm, gd, 10, key, c->cell, c->id, id_new);
    for (int a = 0; a < 10; ++a)
        SIMP_CUDA(c, cudaMemcpyAsync(srcs[a], gd.dst[a], sizeof(double) * (size_t)n,
                                     cudaMemcpyDeviceToDevice, s));
    SIMP_CUDA(c, cudaMemcpyAsync(c->id, id_new, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    k_finish_rebuild<<<nblk(n, B), B, 0, s>>>(n, c->s0, c->xr, c->yr, c->id, c->inv_id);
    k_reset_disp<<<1, 1, 0, s>>>(c->sc);
    c->launches += 7 + kScanKernels;
    SIMP_CUDA(c, cudaGetLastError());
    c->steps_since_rebuild = 0;
    c->rebuilds += 1;
    return SIMP_OK;
}

}  // namespace simp
