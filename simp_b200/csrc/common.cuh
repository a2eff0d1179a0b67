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
#include "check.cuh"

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
    int n = 0;   // particles in the context (the debug build's index checks)
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
    int n = 0;   // particles in the context (the debug build's index checks)
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

enum : int { FLAG_NONFINITE = 1, FLAG_RETIRED = 2 };

// A basin that is neither searched nor stepped: its state turned non-finite
// (it is carried until the caller retires it), or it was retired and its
// storage waits for the next compaction of the batch.
__host__ __device__ __forceinline__ bool inst_dead(int flags) {
    return (flags & (FLAG_NONFINITE | FLAG_RETIRED)) != 0;
}

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
    int scale_h;    // scale_h_of(skf)
    int viscosity, pressure_force, eos_alg;
    int wind_force, water_force, wind_kind;
    int boundary_pressure;
    int sle, den_alg, mass_from_area, tse, hsml_multiplicity;
    int rheology, pa_sph, int_algorithm;
    int max_ind_int;
    int nnps;       // 1 direct search, 2 bucket search (the pair orientation)
    double P_star, c_eos, e, delta_min, k_t;
    double rho_ice, rho_air, rho_water, c_wind, c_water;
    double b_length, kappa_n, alpha;
    double wind_u, wind_v, current_u, current_v;
    double vortex_x, vortex_y, vortex_umax, vortex_radius;
    double max_hsml;
    double zeta_max, eta_max, mu;   // Mohr-Coulomb caps and tan(phi)
    int bfa, boundary_friction;     // boundary force algorithm and its friction branch
    double kappa_t, xi, Y, nu;      // friction parameters; Young modulus and Poisson ratio
    // regularisation (regularization.f90): XSPH, the artificial viscosity
    // (0 none, 1 Hernquist-Katz, 2 Monaghan; applied whenever either switch
    // is on, as the reference's regularization does), its coefficients
    int xsph, art_visc, artificial_visc;
    int csound;                     // 1: c_yang is refreshed (sound_speed.f90:21-27), 0: c stays 0
    double alpha_pi, beta_pi, chi;
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
// Smoothing kernels (kernel.f90:5-633).  With q = r / hsml_ij * scale_h and
// shh = scale_h / hsml_ij, kernel_wg gives W and gq = factor * dW/dq, so that
// grad W = gq * shh * (dx / r).  The reference's default-real literals keep
// their single-precision values.
__host__ __device__ constexpr int scale_h_of(int skf) {   // initialize.f90:208-217
    return (skf == SIMP_SKF_WENDLAND_C2 || skf == SIMP_SKF_WENDLAND_C4 || skf == SIMP_SKF_WENDLAND_C6) ? 1
         : (skf == SIMP_SKF_QUADRATIC || skf == SIMP_SKF_CUBIC) ? 2 : 3;
}
__host__ __device__ constexpr bool skf_known(int skf) { return skf >= 1 && skf <= 9; }

__device__ __forceinline__ double kexp(double v) { return exp(v); }
__device__ __forceinline__ float kexp(float v) { return expf(v); }
__device__ __forceinline__ double ktanh(double v) { return tanh(v); }
__device__ __forceinline__ float ktanh(float v) { return tanhf(v); }
__device__ __forceinline__ double kcosh(double v) { return cosh(v); }
__device__ __forceinline__ float kcosh(float v) { return coshf(v); }
__device__ __forceinline__ double klog(double v) { return log(v); }
__device__ __forceinline__ float klog(float v) { return logf(v); }

// The reference's log(2.) takes a default-real argument: the single-precision
// logarithm of 2 (0.693147182464599609375), promoted.
constexpr double kLog2Real4 = 0.693147182464599609375;
constexpr double kMarquis2C1 = 10.0, kMarquis2C2 = 50.0;   // kernel.f90:602-603

// Kernel choice of a pass: SKF when the pass is compiled for one kernel
// (the cubic spline and the reference default, Wendland C6), else the
// runtime switch (SKF = 0).
template <int SKF>
__host__ __device__ constexpr int skf_of(int runtime) { return SKF ? SKF : runtime; }
// The kernels with their own compiled pair passes.
__host__ __device__ constexpr int skf_compiled(int skf) {
    return (skf == SIMP_SKF_CUBIC || skf == SIMP_SKF_WENDLAND_C6) ? skf : 0;
}

template <class T, bool WANT_W, int SKF = 0>
__device__ __forceinline__ void kernel_wg(int skf, T q, T shh, T inv_h, T *w, T *gq) {
    const T s2 = shh * shh;
    switch (skf_of<SKF>(skf)) {
        case SIMP_SKF_QUADRATIC: {   // kernel.f90:269-276
            const T f = (T)(2.0 / kPi) * s2;
            if (WANT_W) *w = f * fma(T(0.1875) * q, q, fma(T(-0.75), q, T(0.75)));
            *gq = f * fma(T(0.375), q, T(-0.75));
            break;
        }
        case SIMP_SKF_GAUSSIAN: {    // kernel.f90:136-144
            const T f = (T)(1.0 / kPi) * s2;
            const T e = kexp(-(q * q));
            if (WANT_W) *w = f * e;
            *gq = f * (T(-2) * q * e);
            break;
        }
        case SIMP_SKF_QUINTIC: {     // kernel.f90:193-219
            const T f = (T)(7.0 / (478.0 * kPi)) * s2;
            const T u3 = T(3) - q, u2 = T(2) - q, u1 = T(1) - q;
            const T a3 = u3 * u3, a2 = u2 * u2, a1 = u1 * u1;
            T wq = 0, g = 0;
            if (q <= T(1)) {
                wq = a3 * a3 * u3 - T(6) * a2 * a2 * u2 + T(15) * a1 * a1 * u1;
                g = T(-5) * a3 * a3 + T(30) * a2 * a2 - T(75) * a1 * a1;
            } else if (q <= T(2)) {
                wq = a3 * a3 * u3 - T(6) * a2 * a2 * u2;
                g = T(-5) * a3 * a3 + T(30) * a2 * a2;
            } else if (q <= T(3)) {
                wq = a3 * a3 * u3;
                g = T(-5) * a3 * a3;
            }
            if (WANT_W) *w = f * wq;
            *gq = f * g;
            break;
        }
        case SIMP_SKF_WENDLAND_C2: { // kernel.f90:387-393
            const T f = (T)(3.0 / (2.0 * kPi)) * s2;
            const T om = T(1) - q, om2 = om * om;
            if (WANT_W) *w = f * (om2 * om2 * fma(T(4), q, T(1)));
            *gq = f * (T(-20) * q * (om2 * om));
            break;
        }
        case SIMP_SKF_WENDLAND_C4: { // kernel.f90:443-450
            const T f = (T)(3.0 / kPi) * s2;
            const T om = T(1) - q, om2 = om * om, om4 = om2 * om2;
            if (WANT_W) *w = f * (om4 * om2 * fma(fma(T(35), q, T(18)), q, T(3)));
            *gq = f * (T(-56) * q * fma(T(5), q, T(1)) * (om4 * om));
            break;
        }
        case SIMP_SKF_MARQUIS: {     // kernel.f90:555-563
            const T f = (T)(1.0 / kPi) * s2;
            const T z = T(300) * (q - T(1));
            if (WANT_W) *w = f * (T(0.5) - T(0.5) * ktanh(z));
            const T c = kcosh(z);
            *gq = f * (T(-150) / (c * c));
            break;
        }
        case SIMP_SKF_MARQUIS2: {    // kernel.f90:612-620 (factor without scale_h)
            const T f = (T)(1.0 / ((double)34.1558f * kPi)) * (inv_h * inv_h);
            const T c1 = (T)kMarquis2C1, c2 = (T)kMarquis2C2;
            const T z = c1 * (T(1) - q);
            if (WANT_W) *w = f * c2 * (klog(kcosh(z)) / c1 - q + T(1) + (T)kLog2Real4 / c1);
            *gq = f * (-c2 * ktanh(z) - T(1));
            break;
        }
        case SIMP_SKF_WENDLAND_C6: { // kernel.f90:499-508
            const T f = (T)(78.0 / (7.0 * kPi)) * s2;
            const T om = T(1) - q;
            const T om2 = om * om, om4 = om2 * om2;
            if (WANT_W) *w = f * (om4 * om4) * (((T(32) * q + T(25)) * q + T(8)) * q + T(1));
            *gq = f * (T(-22) * q * (om4 * om2 * om) * ((T(16) * q + T(7)) * q + T(1)));
            break;
        }
        default: {                   // SIMP_SKF_CUBIC, kernel.f90:324-340 restored
            const T f = (T)(15.0 / (7.0 * kPi)) * s2;
            if (q <= T(1)) {
                if (WANT_W) *w = f * fma(T(0.5) * q * q, q, fma(-q, q, (T)(2.0f / 3.0f)));
                *gq = f * fma(T(1.5) * q, q, T(-2) * q);
            } else {
                const T u = T(2) - q;
                if (WANT_W) *w = f * ((T)(1.0f / 6.0f) * u * u * u);
                *gq = f * (T(-0.5) * u * u);
            }
            break;
        }
    }
}

// FP64 pair kernel: w and gfac with grad W = gfac * dx.
template <bool WANT_W>
__device__ __forceinline__ void pair_kernel(const Phys &P, double r, double hij,
                                            double *w, double *gfac) {
    const double sh = (double)P.scale_h;
    const double inv_h = 1.0 / hij;
    const double shh = sh * inv_h;
    const double q = r * shh;
    double gq;
    kernel_wg<double, WANT_W>(P.skf, q, shh, inv_h, w, &gq);
    *gfac = gq * shh / r;
}

// Kernel value at q = 0 with smoothing length hij (kernel_zero of each kernel).
__device__ __forceinline__ double kernel_zero(const Phys &P, double hij) {
    const double shh = (double)P.scale_h / hij;
    const double s2 = shh * shh;
    switch (P.skf) {
        case SIMP_SKF_QUADRATIC: return (2.0 / kPi) * s2 * 0.75;
        case SIMP_SKF_GAUSSIAN: return (1.0 / kPi) * s2;
        case SIMP_SKF_QUINTIC: return (7.0 / (478.0 * kPi)) * s2 * 66.0;
        case SIMP_SKF_WENDLAND_C2: return (3.0 / (2.0 * kPi)) * s2;
        case SIMP_SKF_WENDLAND_C4: return (3.0 / kPi) * s2 * 3.0;
        case SIMP_SKF_MARQUIS: return (1.0 / kPi) * s2 * 0.5;
        case SIMP_SKF_MARQUIS2: {
            const double f = 1.0 / ((double)34.1558f * kPi * hij * hij);
            return f * kMarquis2C2 * (log(cosh(kMarquis2C1)) / kMarquis2C1 + 1.0 + kLog2Real4 / kMarquis2C1);
        }
        case SIMP_SKF_WENDLAND_C6: return (78.0 / (7.0 * kPi)) * s2;
        default: return (15.0 / (7.0 * kPi)) * s2 * (double)(2.0f / 3.0f);
    }
}

// Boundary kernel value bw at distance br (support b_length),
// boundary_kernel.f90:20-45 dispatch: b_Quadratic :106-112, b_Gaussian
// :177-183 (also for the Marquis kernels), b_quintic_spline :250-276 (its
// factor is 15/(478 pi), not the particle kernel's 7/(478 pi)),
// b_Wendland_C2 :342-347, b_Wendland_C4 :416-420, b_Wendland_C6 :489-494.
// The C6 factor uses a particle-pair smoothing length (hsml_ij indexed by
// the boundary-pair index), for which the particle's own hsml stands here
// (identical whenever hsml is uniform).  Cubic: b_Quadratic's form with the
// cubic spline, support b_length, scale_h = 2.
template <int SKF = 0>
__device__ __forceinline__ double boundary_w(const Phys &P, double br, double hs_i) {
    const double sh = (double)P.scale_h;
    const double q = br / P.b_length * sh;
    const double shb = sh / P.b_length, s2 = shb * shb;
    switch (skf_of<SKF>(P.skf)) {
        case SIMP_SKF_QUADRATIC:
            return (2.0 / kPi) * s2 * (0.1875 * q * q - 0.75 * q + 0.75);
        case SIMP_SKF_GAUSSIAN:
        case SIMP_SKF_MARQUIS:
        case SIMP_SKF_MARQUIS2:
            return (1.0 / kPi) * s2 * exp(-(q * q));
        case SIMP_SKF_QUINTIC: {
            const double f = (15.0 / (478.0 * kPi)) * s2;
            const double u3 = 3.0 - q, u2 = 2.0 - q, u1 = 1.0 - q;
            const double p3 = u3 * u3 * u3 * u3 * u3, p2 = u2 * u2 * u2 * u2 * u2, p1 = u1 * u1 * u1 * u1 * u1;
            if (q <= 1.0) return f * (p3 - 6.0 * p2 + 15.0 * p1);
            if (q <= 2.0) return f * (p3 - 6.0 * p2);
            if (q <= 3.0) return f * p3;
            return 0.0;
        }
        case SIMP_SKF_WENDLAND_C2: {
            const double om = 1.0 - q, om2 = om * om;
            return (3.0 / (2.0 * kPi)) * s2 * (om2 * om2 * (1.0 + 4.0 * q));
        }
        case SIMP_SKF_WENDLAND_C4: {
            const double om = 1.0 - q, om2 = om * om;
            return (3.0 / kPi) * s2 * (om2 * om2 * om2 * ((35.0 * q + 18.0) * q + 3.0));
        }
        case SIMP_SKF_WENDLAND_C6: {
            const double shh = sh / hs_i;
            const double factor = (78.0 / (7.0 * kPi)) * (shh * shh);
            const double om = 1.0 - q;
            const double om2 = om * om, om4 = om2 * om2;
            return factor * (om4 * om4) * (((32.0 * q + 25.0) * q + 8.0) * q + 1.0);
        }
        default: {
            const double factor = (15.0 / (7.0 * kPi)) * s2;
            const double c23 = (double)(2.0f / 3.0f), c16 = (double)(1.0f / 6.0f);
            if (q <= 1.0) return factor * (c23 - q * q + 0.5 * q * q * q);
            if (q <= 2.0) { const double u = 2.0 - q; return factor * (c16 * u * u * u); }
            return 0.0;
        }
    }
}

// factor * dW/dq of the boundary kernel at q = br / b_length * scale_h
// (boundary_kernel.f90: b_Quadratic :111-112, b_Gaussian :182-184,
// b_quintic_spline :257-274, b_Wendland_C2 :348-349, b_Wendland_C4
// :422-423, b_Wendland_C6 :495-496; the cubic as its kernel's derivative).
// The kernel gradient is then bdwdx = -(f dW/dq) / b_length * (bdx / br) *
// scale_h, with bdx = xb - x_i.
template <int SKF = 0>
__device__ __forceinline__ double boundary_fdwdq(const Phys &P, double br, double hs_i) {
    const double sh = (double)P.scale_h;
    const double q = br / P.b_length * sh;
    const double shb = sh / P.b_length, s2 = shb * shb;
    switch (skf_of<SKF>(P.skf)) {
        case SIMP_SKF_QUADRATIC:
            return (2.0 / kPi) * s2 * (0.375 * q - 0.75);
        case SIMP_SKF_GAUSSIAN:
        case SIMP_SKF_MARQUIS:
        case SIMP_SKF_MARQUIS2:
            return (1.0 / kPi) * s2 * (-2.0 * q * exp(-(q * q)));
        case SIMP_SKF_QUINTIC: {
            const double f = (15.0 / (478.0 * kPi)) * s2;
            const double u3 = 3.0 - q, u2 = 2.0 - q, u1 = 1.0 - q;
            const double p3 = (u3 * u3) * (u3 * u3), p2 = (u2 * u2) * (u2 * u2), p1 = (u1 * u1) * (u1 * u1);
            if (q <= 1.0) return f * (-5.0 * p3 + 30.0 * p2 - 75.0 * p1);
            if (q <= 2.0) return f * (-5.0 * p3 + 30.0 * p2);
            if (q <= 3.0) return f * (-5.0 * p3);
            return 0.0;
        }
        case SIMP_SKF_WENDLAND_C2: {
            const double q2 = q * q;
            return (3.0 / (2.0 * kPi)) * s2 * (20.0 * (q2 * q2 - 3.0 * (q2 * q) + 3.0 * q2 - q));
        }
        case SIMP_SKF_WENDLAND_C4: {
            const double om = 1.0 - q, om2 = om * om;
            return (3.0 / kPi) * s2 * ((-56.0 * q) * (5.0 * q + 1.0) * (om2 * om2 * om));
        }
        case SIMP_SKF_WENDLAND_C6: {
            const double shh = sh / hs_i;
            const double factor = (78.0 / (7.0 * kPi)) * (shh * shh);
            const double om = 1.0 - q;
            const double om2 = om * om, om4 = om2 * om2;
            return factor * ((-22.0 * q) * (om4 * om2 * om) * ((16.0 * q + 7.0) * q + 1.0));
        }
        default: {
            const double factor = (15.0 / (7.0 * kPi)) * s2;
            if (q <= 1.0) return factor * (1.5 * q * q - 2.0 * q);
            if (q <= 2.0) { const double u = 2.0 - q; return factor * (-0.5 * u * u); }
            return 0.0;
        }
    }
}

// Sound speed c_yang (sound_speed.f90:54-55), evaluated from the current
// density: the reference refreshes c after every density update
// (initialize.f90:200, time_integration.f90:140, 230, 274, 355, 383).
__device__ __forceinline__ double sound_speed(const Phys &P, double rho) {
    return sqrt(P.Y * (1.0 - P.nu) / (rho * (1.0 + P.nu) * (1.0 - 2.0 * P.nu)));
}
// The value the reference's c(:) holds: c_yang when sound_speed refreshes it
// (artificial viscosity, Monaghan time step or boundary friction), else the
// zero it was never moved from.
__device__ __forceinline__ double sound_speed_held(const Phys &P, double rho) {
    return P.csound ? sound_speed(P, rho) : 0.0;
}

// Time-step candidate of one particle (time_step.f90:132-157 VP_time_step;
// :40-124 Monaghan_time_step, whose dt = min(0.25 sqrt(min hsml / |a|),
// min CFL) is the min over the particles of min(0.25 sqrt(hsml / |a|), CFL),
// sqrt being monotone).  CFL: hsml / c, or with artificial viscosity
// 0.3 hsml / (c + hsml |div| + 1.2 (alpha_pi c + beta_pi hsml |div|))
// (:111-115; 0.3 and 1.2 are default-real literals).
// hs: the new hsml, a2: |dv/dt|^2 of the last right-hand side, rho: the new
// density (c_yang is refreshed from it before time_step), adiv: |div v|
// with the new velocities (artificial viscosity only).
__device__ __forceinline__ double dt_candidate(const Phys &P, double hs, double a2, double rho, double adiv) {
    if (P.tse == 2) return P.rho_ice * (hs * hs) * P.delta_min / (P.P_star * (1.0 + P.k_t));
    const double acc = sqrt(a2);
    const double f = 0.25 * sqrt(hs / acc);
    const double c = sound_speed(P, rho);
    const double cfl = P.artificial_visc
        ? (double)0.3f * hs / (c + hs * adiv + (double)1.2f * (P.alpha_pi * c + P.beta_pi * hs * adiv))
        : hs / c;
    return f < cfl ? f : cfl;
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
