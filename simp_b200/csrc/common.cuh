// Shared device-side definitions of the SIMP hot path on sm_100a.
//
// Data layout in HBM (one basin, FP64 plain form):
//   particle state is structure-of-arrays, permanently stored in cell order
//   (the order of the last cell-list rebuild): x, y, vx, vy, m, rho, mor
//   (= m / rho), hs (hsml), h, A, cell (rebuild-time cell id), id (original
//   particle index).  Each RHS evaluation reads one state set and writes the
//   next (start-of-step set S0 and half-step set S1, see passes.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/simp_gpu.h"

namespace simp {

constexpr double kPi = 3.1415926535897932;  // globals.f90:199

// Structure-of-arrays particle state (device pointers, cell order).
struct State {
    double *x, *y, *vx, *vy;
    double *m, *rho, *mor, *h, *A;
    double *hs;   // hsml (shared by S0 and S1: updated only at step end)
    float *hsf;   // its FP32 copy (shared)
    // Packed copies that the pair passes gather per neighbour (one or two
    // vector loads per neighbour instead of one scalar load per array):
    double2 *xy, *vxy;   // (x, y), (vx, vy)
    float4 *pf;          // (x, y, hsml, 0) in FP32: the candidate prefilter
    double2 *mm;         // (m, m / rho): plain form (null in the mixed form)
    float4 *hmm;         // (hsml, m, m / rho, 0) in FP32: mixed form (null in the plain form)
};

// Rewrites the packed copies of particle k from the FP64 arrays.
__device__ __forceinline__ void refresh_views(const State &s, int k) {
    const double x = s.x[k], y = s.y[k], hs = s.hs[k], m = s.m[k], mor = s.mor[k];
    const float hsf = (float)hs;
    s.hsf[k] = hsf;
    s.xy[k] = make_double2(x, y);
    s.vxy[k] = make_double2(s.vx[k], s.vy[k]);
    s.pf[k] = make_float4((float)x, (float)y, hsf, 0.0f);
    if (s.hmm) s.hmm[k] = make_float4(hsf, (float)m, (float)mor, 0.0f);
    else s.mm[k] = make_double2(m, mor);
}

// Verlet neighbour lists (cell-order indices): nbr[k * stride + i],
// k < count[i], holding every j within mhsml + skin of i at the positions
// (xl, yl) where the list was built; a count above kMaxNbr means the list
// overflowed and that particle scans its cell stencil instead.
constexpr int kMaxNbr = 48;
struct NbrList {
    int *nbr;
    int *count;
    double *xl, *yl;
    int stride;
};

// The kernel gradients of a right-hand side's pairs, kept by the kinematic
// pass for the stress pass (same pairs, same state): row k, particle i, for
// the first kDwRows pairs of each particle (the others are recomputed).
constexpr int kDwRows = 32;

// Exact pairs of the current right-hand side, written by the kinematic pass
// and consumed by the stress pass: pj[k * stride + i], k < count[i]; a count
// above kMaxPairs means the stress pass finds that particle's pairs itself.
constexpr int kMaxPairs = 48;
struct PairList {
    int *pj;
    int *count;
    int stride;
};

// Uniform cell grid of one basin.  cell = clamp(floor((x - x0) * inv_cs));
// rows are y.  A batch gives every basin (instance) its own grid in one
// shared cell-key space: key = base + row * ncx + col, so instances never
// share a cell and never interact.
struct Grid {
    double x0, y0, cs, inv_cs;
    int ncx, ncy, base;
    const int *cell_start;  // global: total cells + 1 entries, cell-ordered ranges
};

// Per-instance data of a batch (device table, indexed by instance id).
struct Inst {
    double x0, y0, cs, inv_cs;   // grid of this instance
    int ncx, ncy, base;
    int wind_kind;
    double wind_u, wind_v, vortex_x, vortex_y, vortex_umax, vortex_radius;
    double b_length;
    double t;                    // this instance's current_time
    double hmin, hmax, bs;       // hsml bounds and reference bucket size
    unsigned long long dmax2_bits;  // max squared displacement since its last sort
    int flags;                   // FLAG_* seen in this instance
    int pad;
};

__host__ __device__ __forceinline__ Grid inst_grid(const Inst &I, const int *cell_start) {
    Grid g;
    g.x0 = I.x0;
    g.y0 = I.y0;
    g.cs = I.cs;
    g.inv_cs = I.inv_cs;
    g.ncx = I.ncx;
    g.ncy = I.ncy;
    g.base = I.base;
    g.cell_start = cell_start;
    return g;
}

// Particle chunk of the tiled pair passes: consecutive particles [p0, p1)
// of cell row `row` of instance q.
struct Chunk {
    int p0, p1, q, row;
};

// Device-resident integrator scalars and per-step reductions.
struct Scalars {
    double dt;            // time step used by the next step
    double t;             // current_time
    double hmin, hmax;    // exact min / max of the current hsml
    double bs;            // reference bucket size 2 * hmin (nnps.f90:211)
    unsigned long long dmax2_bits;  // max squared displacement since rebuild
    unsigned long long xabs_bits;   // max |coordinate| of any particle so far
    // Verlet neighbour lists: members within mhsml + skin when built; valid
    // while every particle moved less than skin / 2 since (and hsml fixed)
    unsigned long long dlist2_bits; // max squared displacement since the lists were built
    double skin;
    int list_scan;                  // 1: the next kinematic pass rebuilds the lists
    unsigned int blocks_done;       // last-block detection of the stress pass
    unsigned long long acc_hmin, acc_hmax;  // accumulators of the next hsml
    unsigned long long acc_dt;              // VP time step min accumulator
    int flags;            // bit 0: non-finite state seen
    int maxip;            // max interactions per particle seen
    int minip;
    int pad;
    unsigned long long sumip;
    int noip;
    int pad2;
};

enum : int { FLAG_NONFINITE = 1 };

// Ordered-bits helpers for non-negative doubles (bit order = value order).
__device__ __forceinline__ unsigned long long dbits(double v) {
    return (unsigned long long)__double_as_longlong(v);
}
__device__ __forceinline__ double bitsd(unsigned long long b) {
    return __longlong_as_double((long long)b);
}

// Compile-time physics switches and constants for the pair passes.
struct Phys {
    int skf;        // SIMP_SKF_*
    int scale_h;    // 1 (C6) or 2 (cubic)
    int viscosity, pressure_force, eos_alg;
    int wind_force, water_force, wind_kind;
    int boundary_pressure;
    int sle, den_alg, mass_from_area, tse, hsml_multiplicity;
    int max_ind_int;
    double P_star, c_eos, e, delta_min, k_t;
    double rho_ice, rho_air, rho_water, c_wind, c_water;
    double b_length, kappa_n, alpha;
    double wind_u, wind_v, current_u, current_v;
    double vortex_x, vortex_y, vortex_umax, vortex_radius;
    double max_hsml;
};

// Interaction-count bookkeeping for nnps.f90:613-670.
__device__ __forceinline__ void note_interactions(Scalars *sc, int cnt) {
    atomicMax(&sc->maxip, cnt);
    atomicMin(&sc->minip, cnt);
}

// ---------------------------------------------------------------------------
// Bit-exact pair criterion of nnps.f90:277-281:
//   d = SQRT((xi-xj)**2 + (yi-yj)**2), mhsml = (hsml_i + hsml_j) / 2,
//   pair iff d <= mhsml.
// Evaluated with round-to-nearest intrinsics (no FMA contraction).  The
// square root is taken only when the squared distance is within 2^-48 of
// mhsml^2; outside that band the comparison of squares decides exactly.
__device__ __forceinline__ bool pair_test(double dx, double dy, double mh, double *d_out) {
    const double s = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
    const double t = __dmul_rn(mh, mh);
    if (s > t * (1.0 + 0x1p-48)) return false;
    const double d = __dsqrt_rn(s);
    *d_out = d;
    return d <= mh;
}

// Distance of the reference (always exact) — used where d itself is output.
__device__ __forceinline__ double ref_distance(double dx, double dy) {
    return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

// Reference bucket index NINT(x / bin_size) (nnps.f90:249-250): nearest,
// halves away from zero.
__device__ __forceinline__ long long ref_bin(double v, double bs) {
    return (long long)round(__ddiv_rn(v, bs));
}

// ---------------------------------------------------------------------------
// Pair kernel gradient factor.  With q = r / hij * scale_h this returns
//   w      (kernel value)
//   gfac   such that dwdx = gfac * dx  (i.e. dW/dq-term / hij / r * scale_h)
// kernel.f90:498-508 (Wendland C6) and kernel.f90:324-340 (cubic spline,
// restored with factor = 15/(7 pi) (scale_h / hij)^2).
template <bool WANT_W>
__device__ __forceinline__ void pair_kernel(const Phys &P, double r, double hij,
                                            double *w, double *gfac) {
    const double sh = (double)P.scale_h;
    const double inv_h = 1.0 / hij;
    const double q = r * inv_h * sh;
    const double shh = sh * inv_h;
    if (P.skf == SIMP_SKF_WENDLAND_C6) {
        const double factor = (78.0 / (7.0 * kPi)) * (shh * shh);
        const double om = 1.0 - q;
        const double om2 = om * om, om4 = om2 * om2;
        const double om7 = om4 * om2 * om;
        if (WANT_W) *w = factor * (om4 * om4) * (((32.0 * q + 25.0) * q + 8.0) * q + 1.0);
        const double g = factor * (-22.0 * q * om7 * ((16.0 * q + 7.0) * q + 1.0));
        *gfac = g * shh / r;
    } else {
        const double factor = (15.0 / (7.0 * kPi)) * (shh * shh);
        const double c23 = (double)(2.0f / 3.0f), c16 = (double)(1.0f / 6.0f);
        double g, wt;
        if (q <= 1.0) {
            wt = factor * (c23 - q * q + 0.5 * q * q * q);
            g = factor * (-2.0 * q + 1.5 * q * q);
        } else {
            const double u = 2.0 - q;
            wt = factor * (c16 * u * u * u);
            g = factor * (-0.5 * u * u);
        }
        if (WANT_W) *w = wt;
        *gfac = g * shh / r;
    }
}

// Kernel value at q = 0 with smoothing length hij (kernel_zero, kernel.f90:503).
__device__ __forceinline__ double kernel_zero(const Phys &P, double hij) {
    const double sh = (double)P.scale_h;
    const double shh = sh / hij;
    if (P.skf == SIMP_SKF_WENDLAND_C6) return (78.0 / (7.0 * kPi)) * (shh * shh);
    return (15.0 / (7.0 * kPi)) * (shh * shh) * (double)(2.0f / 3.0f);
}

// Boundary kernel value bw at distance br (support b_length).
// Wendland C6: boundary_kernel.f90:489-494; its factor uses a particle-pair
// smoothing length (hsml_ij indexed by the boundary-pair index), for which the
// particle's own hsml stands here (identical whenever hsml is uniform).
// Cubic: b_Quadratic's form (boundary_kernel.f90:106-112) with the cubic
// spline, support b_length, scale_h = 2.
__device__ __forceinline__ double boundary_w(const Phys &P, double br, double hs_i) {
    const double sh = (double)P.scale_h;
    const double q = br / P.b_length * sh;
    if (P.skf == SIMP_SKF_WENDLAND_C6) {
        const double shh = sh / hs_i;
        const double factor = (78.0 / (7.0 * kPi)) * (shh * shh);
        const double om = 1.0 - q;
        const double om2 = om * om, om4 = om2 * om2;
        return factor * (om4 * om4) * (((32.0 * q + 25.0) * q + 8.0) * q + 1.0);
    }
    const double shb = sh / P.b_length;
    const double factor = (15.0 / (7.0 * kPi)) * (shb * shb);
    const double c23 = (double)(2.0f / 3.0f), c16 = (double)(1.0f / 6.0f);
    if (q <= 1.0) return factor * (c23 - q * q + 0.5 * q * q * q);
    if (q <= 2.0) { const double u = 2.0 - q; return factor * (c16 * u * u * u); }
    return 0.0;
}

// Wind at a particle of an instance: uniform (the reference hard-codes one,
// wind_forcing.f90:36-37) or a cyclonic vortex
// U(r) = Umax (r/R) exp((1 - r^2/R^2)/2), counter-clockwise.
__device__ __forceinline__ void wind_at(const Inst &I, double x, double y, double *wu, double *wv) {
    if (I.wind_kind == SIMP_WIND_VORTEX) {
        const double rx = x - I.vortex_x, ry = y - I.vortex_y;
        const double r = sqrt(rx * rx + ry * ry);
        if (r == 0.0) { *wu = 0.0; *wv = 0.0; return; }
        const double s = r / I.vortex_radius;
        const double U = I.vortex_umax * s * exp(0.5 * (1.0 - s * s));
        *wu = -U * ry / r;
        *wv = U * rx / r;
    } else {
        *wu = I.wind_u;
        *wv = I.wind_v;
    }
}

// Stencil radius in cells that is guaranteed to contain every pair at the
// current positions: pairs are at most hmax apart now, each particle moved at
// most sqrt(dmax2) since it was binned.
// The result is clamped to [1, max(ncx, ncy)] (a non-finite bound, which the
// step reports as an error, then scans the whole grid instead of overflowing).
__device__ __forceinline__ int clamp_radius(double Rd, const Grid &g) {
    const double lim = (double)(g.ncx > g.ncy ? g.ncx : g.ncy);
    if (!(Rd >= 1.0)) Rd = (Rd != Rd) ? lim : 1.0;
    if (Rd > lim) Rd = lim;
    return (int)Rd;
}

__device__ __forceinline__ int stencil_radius(double hmax, unsigned long long dmax2_bits, const Grid &g,
                                              double extra) {
    const double dm = sqrt(bitsd(dmax2_bits));
    const double reach = fmax(hmax, extra) + 2.0 * dm;
    return clamp_radius(ceil(reach * g.inv_cs * (1.0 + 1e-12) + 1e-9), g);
}

__host__ __device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace simp
