// The two pair passes of one right-hand-side evaluation (single_step.f90:5-109)
// and the predictor-corrector update fused into the second pass's epilogue.
//
// Kinematic pass (single_step.f90:50-84 + internal_stress.f90:20-42):
//   gather over neighbours j of i:
//     wdvx = (v_i - v_j) (x) grad W_ij             (kernel.f90:515-518)
//     div_i  -= m_j (wdvx1 + wdvx4)                (vector_divergence.f90:27)
//     grad_i -= m_j wdvx / rho_j                   (vector_gradient.f90:56-69)
//   then, per particle, strain (single_step.f90:80-84), strength, bulk and
//   shear viscosity, replacement pressure and stress (bulk_viscosity.f90:
//   65-76, shear_viscosity.f90:57, eos.f90:141-147, stress_tensor.f90:31-39).
//   Writes tau = sigma / rho^2 and div per particle.
//
// Stress pass (internal_stress.f90:103-137 stress_1, boundary_kernel.f90 +
// boundary_force.f90:74-84, wind_forcing.f90:35-51, water_drag.f90:35-53,
// single_step.f90:104-106):
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

struct KinArgs {
    State s;
    Grid g;
    const int *cell;
    Phys P;
    Scalars *sc;
    double *tau11, *tau12, *tau22, *div;
    double *diag;
    int n, maxn;
};

__global__ void __launch_bounds__(kBlock) k_kinematic(KinArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const State &s = a.s;
    const Phys &P = a.P;
    const double xi = s.x[i], yi = s.y[i], vxi = s.vx[i], vyi = s.vy[i], hi = s.hs[i];
    const int R = stencil_radius(a.sc, a.g, 0.0);
    const BinRule br = make_bin_rule(a.sc, xi, yi, a.sc->hmax);
    double dv = 0.0, g1 = 0.0, g2 = 0.0, g3 = 0.0, g4 = 0.0;
    for_each_pair(s.x, s.y, s.hs, a.g, i, a.cell[i], R, br, xi, yi, hi,
                  [&](int j, double dx, double dy, double r, double mh) {
                      double gf;
                      pair_kernel<false>(P, r, mh, nullptr, &gf);
                      const double dwx = gf * dx, dwy = gf * dy;
                      const double dvx = vxi - s.vx[j], dvy = vyi - s.vy[j];
                      const double w1 = dvx * dwx, w2 = dvy * dwx, w3 = dvx * dwy, w4 = dvy * dwy;
                      const double mj = s.m[j], mrj = s.mor[j];
                      dv -= mj * (w1 + w4);
                      g1 -= mrj * w1;
                      g2 -= mrj * w2;
                      g3 -= mrj * w3;
                      g4 -= mrj * w4;
                  });
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
    Grid g;
    const int *cell;
    const double *bx, *by, *bm;
    const int *bstart;
    int nb;
    Phys P;
    Scalars *sc;
    const double *tau11, *tau12, *tau22, *div;
    double *rates;
    const double *xr, *yr;
    double *hs_next;
    int n, maxn, mode;
};

__device__ __forceinline__ void warp_max_u64(unsigned long long *dst, unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = (t > v) ? t : v;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(dst, v);
}
__device__ __forceinline__ void warp_min_u64(unsigned long long *dst, unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = (t < v) ? t : v;
    }
    if ((threadIdx.x & 31) == 0) atomicMin(dst, v);
}
__device__ __forceinline__ void warp_max_i32(int *dst, int v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(dst, v);
}

__global__ void __launch_bounds__(kBlock) k_stress(StressArgs a) {
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i0 < a.n;
    const int i = live ? i0 : a.n - 1;   // dead lanes mirror the last particle for warp reductions
    const State &s = a.rhs;
    const Phys &P = a.P;
    const double xi = s.x[i], yi = s.y[i], hi = s.hs[i];
    const int ci = a.cell[i];
    const int R = stencil_radius(a.sc, a.g, 0.0);
    const BinRule br = make_bin_rule(a.sc, xi, yi, a.sc->hmax);
    double Sx = 0.0, Sy = 0.0, Tx = 0.0, Ty = 0.0;
    int cnt = for_each_pair(s.x, s.y, s.hs, a.g, i, ci, R, br, xi, yi, hi,
                            [&](int j, double dx, double dy, double r, double mh) {
                                double gf;
                                pair_kernel<false>(P, r, mh, nullptr, &gf);
                                const double dwx = gf * dx, dwy = gf * dy;
                                const double mj = s.m[j];
                                const double t11 = a.tau11[j], t12 = a.tau12[j], t22 = a.tau22[j];
                                Sx += mj * dwx;
                                Sy += mj * dwy;
                                Tx += mj * (t11 * dwx + t12 * dwy);
                                Ty += mj * (t12 * dwx + t22 * dwy);
                            });
    const double rho = s.rho[i], hh = s.h[i], AA = s.A[i], mi = s.m[i];
    const double fi = rho / P.rho_ice / hh;
    double ax = fi * (a.tau11[i] * Sx + a.tau12[i] * Sy + Tx);
    double ay = fi * (a.tau12[i] * Sx + a.tau22[i] * Sy + Ty);
    // boundary force (bf_Monaghan normal component, boundary_force.f90:78-82)
    if (P.boundary_pressure && a.nb > 0) {
        const int Rb = wall_radius(a.sc, a.g, P.b_length);
        const BinRule bb = make_bin_rule(a.sc, xi, yi, P.b_length);
        double fx = 0.0, fy = 0.0;
        cnt += for_each_wall(a.bx, a.by, a.bstart, a.g, ci, Rb, bb, xi, yi, P.b_length,
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
    const double tnow = a.sc->t;
    if (P.wind_force && tnow > 0.0) {
        double wu, wv;
        wind_at(P, xi, yi, &wu, &wv);
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
    const double dxr = xn - a.xr[i], dyr = yn - a.yr[i];
    const double d2 = live ? dxr * dxr + dyr * dyr : 0.0;
    warp_max_u64(&a.sc->dmax2_bits, dbits(d2));
    if (live) {
        const State &o = a.out;
        o.x[i] = xn;
        o.y[i] = yn;
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
        const bool bad = !(isfinite(xn) && isfinite(yn) && isfinite(vxn) && isfinite(vyn) &&
                           isfinite(hn) && isfinite(An));
        if (live && bad) atomicOr(&a.sc->flags, FLAG_NONFINITE);
    }
}

// End of a predictor-corrector step: time_step's new dt, current_time += dt
// (time_integration.f90:179, using the dt computed at the end of the step),
// and the new hsml bounds.
__global__ void k_step_finish(Scalars *sc, int tse, int sle) {
    if (tse == 2) {
        sc->dt = bitsd(sc->acc_dt);
        sc->acc_dt = dbits(INFINITY);
    }
    sc->t = sc->t + sc->dt;
    if (sle == 2) {
        sc->hmin = bitsd(sc->acc_hmin);
        sc->hmax = fmax(sc->hmax, bitsd(sc->acc_hmax));
        sc->bs = 2.0 * sc->hmin;
        sc->acc_hmin = dbits(INFINITY);
        sc->acc_hmax = 0ull;
    }
}

__global__ void k_reset_stats(Scalars *sc) {
    sc->maxip = 0;
    sc->minip = 0x7fffffff;
    sc->sumip = 0ull;
    sc->noip = 0;
    sc->flags = 0;
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

void launch_kinematic(simp_ctx *c, const State &s, bool diag) {
    KinArgs a;
    a.s = s;
    a.g = c->grid;
    a.cell = c->cell;
    a.P = c->phys;
    a.sc = c->sc;
    a.tau11 = c->tau11;
    a.tau12 = c->tau12;
    a.tau22 = c->tau22;
    a.div = c->div;
    a.diag = diag ? c->diag : nullptr;
    a.n = c->n;
    a.maxn = c->maxn;
    k_kinematic<<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_stress(simp_ctx *c, const State &rhs, const State &base, EpiMode mode) {
    StressArgs a;
    a.rhs = rhs;
    a.base = base;
    a.out = (mode == EPI_PREDICT) ? c->s1 : c->s0;
    a.g = c->grid;
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
    a.rates = c->rates;
    a.xr = c->xr;
    a.yr = c->yr;
    a.hs_next = c->tmp;   // hsml of the next step (copied back by the caller)
    a.n = c->n;
    a.maxn = c->maxn;
    a.mode = mode;
    k_stress<<<nblk(c->n, kBlock), kBlock, 0, c->stream>>>(a);
    c->launches += 1;
}

void launch_step_finish(simp_ctx *c) {
    if (c->prm.sle == 2)
        cudaMemcpyAsync(c->s0.hs, c->tmp, sizeof(double) * (size_t)c->n, cudaMemcpyDeviceToDevice,
                        c->stream);
    k_step_finish<<<1, 1, 0, c->stream>>>(c->sc, c->prm.tse, c->prm.sle);
    c->launches += 1;
}

void launch_reset_stats(simp_ctx *c) {
    k_reset_stats<<<1, 1, 0, c->stream>>>(c->sc);
    c->launches += 1;
}

}  // namespace simp
