// Pair-list export of the NNPS entry point and the density pair sum, for
// the context's single basin (instance 0).
//
// The reference's NNPS writes p_i, p_j, r_ij, hsml_ij (nnps.f90:284-288) and
// bp_i, bp_j, br_ij (:479-482) into global arrays, in an order that depends on
// the OpenMP schedule (:426-433).  The export here emits the same unordered
// pair set in a canonical order: (p_i, p_j) with p_i < p_j, sorted, 1-based
// original indices; wall pairs sorted by (bp_i, bp_j).  Counting pass, prefix
// scan over original indices, emit pass, then a per-segment sort.
#include <algorithm>
#include <vector>

#include "ctx.h"
#include "neighbors.cuh"

namespace simp {

namespace {

constexpr int kBlock = 128;

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

struct ExpArgs {
    State s;
    const Inst *inst;          // instance 0 (the basin)
    const int *cell_start;
    const int *cell;
    const int *id;
    const double *bx, *by;
    const int *bstart;
    int nb;
    Phys P;
    Scalars *sc;
    int n;
    int *up_cnt;     // by original index
    const int *up_off;
    int *oi, *oj;
    double *orr, *oh;
};

__global__ void __launch_bounds__(kBlock) k_count(ExpArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Inst &I = a.inst[0];
    const Grid g = inst_grid(I, a.cell_start);
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const int ci = a.cell[i];
    const int R = stencil_radius(I.hmax, I.dmax2_bits, g, 0.0);
    const BinRule br = make_bin_rule(I.bs, xi, yi, I.hmax);
    const int idi = a.id[i];
    int up = 0;
    int cnt = for_each_pair(s.x, s.y, s.hs, g, i, ci, R, br, xi, yi, hi,
                            [&](int j, double, double, double, double) { up += (a.id[j] > idi); });
    if (a.P.boundary_pressure && a.nb > 0) {
        const int Rb = wall_radius(I.dmax2_bits, g, I.b_length);
        const BinRule bb = make_bin_rule(I.bs, xi, yi, I.b_length);
        cnt += for_each_wall(a.bx, a.by, a.bstart, g, ci, Rb, bb, xi, yi, I.b_length,
                             [&](int, double, double, double) {});
    }
    a.up_cnt[idi] = up;
    atomicMax(&a.sc->maxip, cnt);
    atomicMin(&a.sc->minip, cnt);
    atomicAdd(&a.sc->sumip, (unsigned long long)cnt);
    if (cnt == 0) atomicAdd(&a.sc->noip, 1);
}

__global__ void __launch_bounds__(kBlock) k_emit(ExpArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Inst &I = a.inst[0];
    const Grid g = inst_grid(I, a.cell_start);
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const int R = stencil_radius(I.hmax, I.dmax2_bits, g, 0.0);
    const BinRule br = make_bin_rule(I.bs, xi, yi, I.hmax);
    const int idi = a.id[i];
    const int base = a.up_off[idi];
    int k = 0;
    for_each_pair(s.x, s.y, s.hs, g, i, a.cell[i], R, br, xi, yi, hi,
                  [&](int j, double, double, double r, double mh) {
                      const int idj = a.id[j];
                      if (idj <= idi) return;
                      a.oi[base + k] = idi + 1;
                      a.oj[base + k] = idj + 1;
                      a.orr[base + k] = r;
                      a.oh[base + k] = mh;
                      ++k;
                  });
    // sort the segment by p_j
    for (int u = base + 1; u < base + k; ++u) {
        const int vj = a.oj[u];
        const double vr = a.orr[u], vh = a.oh[u];
        int w = u - 1;
        while (w >= base && a.oj[w] > vj) {
            a.oj[w + 1] = a.oj[w];
            a.orr[w + 1] = a.orr[w];
            a.oh[w + 1] = a.oh[w];
            --w;
        }
        a.oj[w + 1] = vj;
        a.orr[w + 1] = vr;
        a.oh[w + 1] = vh;
    }
}

// Wall pairs from the wall side: fluid particles binned within the stencil.
struct WallArgs {
    State s;
    const Inst *inst;
    const int *cell_start;
    const int *id;
    const double *bx, *by;
    const int *bcell, *bid;
    int nb;
    int *cnt;        // by original wall index
    const int *off;
    int *oi, *oj;
    double *orr;
    int emit;
};

__global__ void __launch_bounds__(kBlock) k_wall(WallArgs a) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.nb) return;
    const Inst &I = a.inst[0];
    const Grid g = inst_grid(I, a.cell_start);
    const double xb = a.bx[b], yb = a.by[b];
    const int Rb = wall_radius(I.dmax2_bits, g, I.b_length);
    const BinRule bb = make_bin_rule(I.bs, xb, yb, I.b_length);
    const int idb = a.bid[b];
    const int base = a.emit ? a.off[idb] : 0;
    int k = 0;
    for_stencil_rows(g, a.bcell[b], Rb, [&](int j0, int j1) {
        for (int j = j0; j < j1; ++j) {
            const double xj = a.s.x[j], yj = a.s.y[j];
            const double d = ref_distance(__dsub_rn(xb, xj), __dsub_rn(yb, yj));
            if (!(d <= I.b_length)) continue;
            if (!bin_rule_ok(bb, xj, yj)) continue;
            if (a.emit) {
                a.oi[base + k] = idb + 1;
                a.oj[base + k] = a.id[j] + 1;
                a.orr[base + k] = d;
            }
            ++k;
        }
    });
    if (!a.emit) {
        a.cnt[idb] = k;
        return;
    }
    for (int u = base + 1; u < base + k; ++u) {
        const int vj = a.oj[u];
        const double vr = a.orr[u];
        int w = u - 1;
        while (w >= base && a.oj[w] > vj) {
            a.oj[w + 1] = a.oj[w];
            a.orr[w + 1] = a.orr[w];
            --w;
        }
        a.oj[w + 1] = vj;
        a.orr[w + 1] = vr;
    }
}

struct DenArgs {
    State s;
    const Inst *inst;
    const int *cell_start;
    const int *cell;
    const int *id;
    Phys P;
    int n;
    double *out;   // original order
};

// density.f90:74-98 (sum_density), kernel_zero from the particle's hsml.
__global__ void __launch_bounds__(kBlock) k_sum_density(DenArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Phys &P = a.P;
    const Inst &I = a.inst[0];
    const Grid g = inst_grid(I, a.cell_start);
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const int R = stencil_radius(I.hmax, I.dmax2_bits, g, 0.0);
    const BinRule br = make_bin_rule(I.bs, xi, yi, I.hmax);
    const double k0 = kernel_zero(P, hi);
    const double mi = s.m[i], rhoi = s.rho[i];
    double num = k0 * mi, den = k0 * mi / rhoi;
    for_each_pair(s.x, s.y, s.hs, g, i, a.cell[i], R, br, xi, yi, hi,
                  [&](int j, double, double, double r, double mh) {
                      double w, gf;
                      pair_kernel<true>(P, r, mh, &w, &gf);
                      const double mw = s.m[j] * w;
                      den += mw / s.rho[j];
                      num += mw;
                  });
    a.out[a.id[i]] = num / den;
}

}  // namespace

int export_pairs(simp_ctx *c, int32_t *nip, int32_t *p_i, int32_t *p_j, double *r_ij,
                 double *hsml_ij, int32_t cap, int32_t *bnip, int32_t *bp_i, int32_t *bp_j,
                 double *br_ij, int32_t bcap) {
    if (const int rc = complete_pending(c)) return rc;   // (the search resets the statistics)
    cudaStream_t st = c->stream;
    const int n = c->n;
    ExpArgs a{};
    a.s = c->s0;
    a.inst = c->inst_dev;
    a.cell_start = c->cell_start;
    a.cell = c->cell;
    a.id = c->id;
    a.bx = c->bx;
    a.by = c->by;
    a.bstart = c->bcell_start;
    a.nb = c->nb;
    a.P = c->phys;
    a.sc = c->sc;
    a.n = n;
    a.up_cnt = c->itmp;
    launch_reset_stats(c);
    k_count<<<nblk(n, kBlock), kBlock, 0, st>>>(a);
    launch_scan_i32(c->itmp, c->pair_cnt, n, c->scan_tmp, st);
    c->launches += 1 + kScanKernels;
    int total = 0;
    SIMP_CUDA(c, cudaMemcpyAsync(&total, c->pair_cnt + n, sizeof(int), cudaMemcpyDeviceToHost, st));
    SIMP_CUDA(c, cudaStreamSynchronize(st));
    // wall pair counts
    int btotal = 0;
    WallArgs w{};
    w.s = c->s0;
    w.inst = c->inst_dev;
    w.cell_start = c->cell_start;
    w.id = c->id;
    w.bx = c->bx;
    w.by = c->by;
    w.bcell = c->bcell;
    w.bid = c->bid;
    w.nb = c->nb;
    const bool walls = c->prm.boundary_pressure && c->nb > 0;
    if (walls) {
        w.cnt = c->itmp + (size_t)std::max(c->maxn, c->maxnb);
        w.emit = 0;
        k_wall<<<nblk(c->nb, kBlock), kBlock, 0, st>>>(w);
        launch_scan_i32(w.cnt, c->bpair_cnt, c->nb, c->scan_tmp, st);
        c->launches += 1 + kScanKernels;
        SIMP_CUDA(c, cudaMemcpyAsync(&btotal, c->bpair_cnt + c->nb, sizeof(int), cudaMemcpyDeviceToHost, st));
        SIMP_CUDA(c, cudaStreamSynchronize(st));
    }
    const size_t need = (size_t)std::max(total, btotal) + 1;
    if (need > c->pair_buf_cap) {
        cudaFree(c->pair_buf_i);
        cudaFree(c->pair_buf_j);
        cudaFree(c->pair_buf_r);
        cudaFree(c->pair_buf_h);
        c->pair_buf_i = c->pair_buf_j = nullptr;
        c->pair_buf_r = c->pair_buf_h = nullptr;
        c->pair_buf_cap = 0;
        const size_t capn = need + need / 8;
        if (cudaMalloc(&c->pair_buf_i, capn * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&c->pair_buf_j, capn * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&c->pair_buf_r, capn * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&c->pair_buf_h, capn * sizeof(double)) != cudaSuccess)
            return simp_fail(c, SIMP_ERR_NOMEM, "device allocation of the pair-list buffers failed");
        c->pair_buf_cap = capn;
    }
    a.up_off = c->pair_cnt;
    a.oi = c->pair_buf_i;
    a.oj = c->pair_buf_j;
    a.orr = c->pair_buf_r;
    a.oh = c->pair_buf_h;
    k_emit<<<nblk(n, kBlock), kBlock, 0, st>>>(a);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    if (nip) *nip = total;
    const int m = std::min(total, (int)std::max(cap, 0));
    if (m > 0) {
        if (p_i) SIMP_CUDA(c, cudaMemcpyAsync(p_i, c->pair_buf_i, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
        if (p_j) SIMP_CUDA(c, cudaMemcpyAsync(p_j, c->pair_buf_j, sizeof(int) * m, cudaMemcpyDeviceToHost, st));
        if (r_ij) SIMP_CUDA(c, cudaMemcpyAsync(r_ij, c->pair_buf_r, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
        if (hsml_ij) SIMP_CUDA(c, cudaMemcpyAsync(hsml_ij, c->pair_buf_h, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
    }
    SIMP_CUDA(c, cudaStreamSynchronize(st));
    if (bnip) *bnip = btotal;
    if (walls) {
        w.off = c->bpair_cnt;
        w.oi = c->pair_buf_i;
        w.oj = c->pair_buf_j;
        w.orr = c->pair_buf_r;
        w.emit = 1;
        k_wall<<<nblk(c->nb, kBlock), kBlock, 0, st>>>(w);
        c->launches += 1;
        SIMP_CUDA(c, cudaGetLastError());
        const int mb = std::min(btotal, (int)std::max(bcap, 0));
        if (mb > 0) {
            if (bp_i) SIMP_CUDA(c, cudaMemcpyAsync(bp_i, c->pair_buf_i, sizeof(int) * mb, cudaMemcpyDeviceToHost, st));
            if (bp_j) SIMP_CUDA(c, cudaMemcpyAsync(bp_j, c->pair_buf_j, sizeof(int) * mb, cudaMemcpyDeviceToHost, st));
            if (br_ij) SIMP_CUDA(c, cudaMemcpyAsync(br_ij, c->pair_buf_r, sizeof(double) * mb, cudaMemcpyDeviceToHost, st));
        }
        SIMP_CUDA(c, cudaStreamSynchronize(st));
    }
    if (total > cap || btotal > bcap)
        return simp_fail(c, SIMP_ERR_PAIR_CAP,
                         "Too much particle interaction please allocate more memory for arrays "
                         "in globals module. (nnps.f90:132-139)");
    return SIMP_OK;
}

int sum_density(simp_ctx *c, double *rho_out_dev) {
    DenArgs a{};
    a.s = c->s0;
    a.inst = c->inst_dev;
    a.cell_start = c->cell_start;
    a.cell = c->cell;
    a.id = c->id;
    a.P = c->phys;
    a.n = c->n;
    a.out = rho_out_dev;
    k_sum_density<<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
    SIMP_CUDA(c, cudaGetLastError());
    return SIMP_OK;
}

}  // namespace simp
