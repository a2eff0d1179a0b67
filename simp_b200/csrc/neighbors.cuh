// Gather-form neighbour iteration over the cell list.
//
// For particle i (cell order) this visits every j with the reference's pair
// criterion (nnps.f90:277-281) and, when it can matter, the reference's
// bucket rule: the reference only tests pairs whose buckets NINT(x / bs),
// bs = 2 min(hsml), differ by at most one in each axis (its 3x3 half
// stencil, nnps.f90:259-407).  A pair within mhsml <= max(hsml) can only fall
// outside that stencil when max(hsml) >= bs (its axis separation is then at
// least bs), so the rule is evaluated only when hmax >= 2 hmin (1 - 1e-6).
#pragma once

#include "common.cuh"

namespace simp {

struct BinRule {
    bool on;
    double bs;
    long long bx, by;
};

__device__ __forceinline__ BinRule make_bin_rule(double bs, double xi, double yi, double reach) {
    BinRule b;
    b.on = reach >= bs * (1.0 - 1e-6);
    b.bs = bs;
    b.bx = b.on ? ref_bin(xi, b.bs) : 0;
    b.by = b.on ? ref_bin(yi, b.bs) : 0;
    return b;
}

__device__ __forceinline__ bool bin_rule_ok(const BinRule &b, double xj, double yj) {
    if (!b.on) return true;
    const long long dx = ref_bin(xj, b.bs) - b.bx, dy = ref_bin(yj, b.bs) - b.by;
    return dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1;
}

// Visits the stencil rows of cell ci (a global key of grid g) within radius
// R: f(j0, j1) for each row's contiguous index range.
template <class F>
__device__ __forceinline__ void for_stencil_rows(const Grid &g, int ci, int R, F &&f) {
    const int local = ci - g.base;
    if (!SIMP_IN_RANGE(local, 0, (long long)g.ncx * g.ncy, SITE_CELL)) return;
    const int cx = local % g.ncx, cy = local / g.ncx;
    const int r0 = max(cy - R, 0), r1 = min(cy + R, g.ncy - 1);
    const int c0 = max(cx - R, 0), c1 = min(cx + R, g.ncx - 1);
    for (int row = r0; row <= r1; ++row) {
        const int k = g.base + row * g.ncx;
        f(g.cell_start[k + c0], g.cell_start[k + c1 + 1]);
    }
}

// f(j, dx, dy, r, mh): dx = x_i - x_j, r = reference distance, mh = hsml_ij.
template <class F>
__device__ __forceinline__ int for_each_pair(const double *__restrict__ X, const double *__restrict__ Y,
                                             const double *__restrict__ HS, const Grid &g, int i, int ci,
                                             int R, const BinRule &br, double xi, double yi, double hi,
                                             F &&f) {
    int count = 0;
    for_stencil_rows(g, ci, R, [&](int j0, int j1) {
        for (int j = j0; j < j1; ++j) {
            if (j == i) continue;
            const double xj = X[j], yj = Y[j];
            const double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj);
            const double mh = __dmul_rn(__dadd_rn(hi, HS[j]), 0.5);
            double r;
            if (!pair_test(dx, dy, mh, &r)) continue;
            if (!bin_rule_ok(br, xj, yj)) continue;
            ++count;
            f(j, dx, dy, r, mh);
        }
    });
    return count;
}

// Boundary pairs of particle i: wall particles b with
// |xb - x_i| <= b_length (nnps.f90:473-476).  f(b, bdx, bdy, br) with
// bdx = xb - x_i.
template <class F>
__device__ __forceinline__ int for_each_wall(const double *__restrict__ BX, const double *__restrict__ BY,
                                             const int *__restrict__ bstart, const Grid &g, int ci, int Rb,
                                             const BinRule &br, double xi, double yi, double b_length,
                                             F &&f) {
    Grid gb = g;
    gb.cell_start = bstart;
    int count = 0;
    for_stencil_rows(gb, ci, Rb, [&](int b0, int b1) {
        for (int b = b0; b < b1; ++b) {
            const double xb = BX[b], yb = BY[b];
            const double bdx = __dsub_rn(xb, xi), bdy = __dsub_rn(yb, yi);
            const double d = ref_distance(bdx, bdy);
            if (!(d <= b_length)) continue;
            if (!bin_rule_ok(br, xb, yb)) continue;
            ++count;
            f(b, bdx, bdy, d);
        }
    });
    return count;
}

// FP32 prefilter of the pair criterion.  The float copies of x, y, hsml are
// within X 2^-24 (X = max |coordinate|) and hsml 2^-24 of the doubles; the
// float subtraction of two nearby coordinates is exact.  So the float
// squared distance and squared mhsml differ from the exact ones by at most
// (5.7 X / hmin + 12) 2^-24 relative near the decision boundary (where
// mhsml >= hmin).  The returned margin doubles that bound; a candidate is
// decided in FP32 only outside the margin, otherwise by the exact FP64 test.
__device__ __forceinline__ float prefilter_margin(double xabs, double hmin) {
    return (float)((12.0 * xabs / hmin + 40.0) * 0x1p-24);
}

// 0: not a pair, 1: a pair, 2: undecided (use the FP64 test)
__device__ __forceinline__ int prefilter(float dxf, float dyf, float mf, float margin) {
    const float sf = dxf * dxf + dyf * dyf;
    const float tf = mf * mf;
    if (sf > tf * (1.0f + margin)) return 0;
    if (sf < tf * (1.0f - margin)) return 1;
    return 2;
}

// Stencil radius for wall pairs: walls are static, the particle moved at
// most sqrt(dmax2) since it was binned.
__device__ __forceinline__ int wall_radius(unsigned long long dmax2_bits, const Grid &g, double b_length) {
    const double dm = sqrt(bitsd(dmax2_bits));
    return clamp_radius(ceil((b_length + dm) * g.inv_cs * (1.0 + 1e-12) + 1e-9), g);
}

}  // namespace simp
