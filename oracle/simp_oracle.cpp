// SIMP per-step hot path: CPU FP64 ORACLE.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, routine by routine and in
// the reference's arithmetic evaluation order, the Fortran code of SIMP
// (McGill-sea-ice/SIMP) that the GPU library replaces.  It is the checker for
// the CUDA path: tests/, the smoke entry and the bench's CPU-baseline leg may
// load it; the product library never links or calls it.
//
// Parity status: UNPINNED against the reference itself.  The reference is
// Fortran 2018 and no Fortran compiler exists on the build or GPU machines,
// and the reference ships no tests, fixtures or golden vectors
// (README.md:60-66).  The restatement is pinned instead to known-answer tests
// derived from the mathematics (tests/golden/kat_*.json): kernel
// normalisation, lattice neighbour counts, rigid-translation zero strain,
// momentum conservation of the stress pair sum and the free-drift speed.
//
// Arithmetic follows gfortran semantics for the shipped flags (Makefile:4, no
// -O, no FMA contraction): compile with -ffp-contract=off.  Default-real
// literals of the reference (e.g. rho_air = 1.3, 2./3. in the cubic kernel)
// keep their single-precision values.
//
// OpenMP regions mirror the reference's (nnps.f90:227-509,
// single_step.f90:50-77, internal_stress.f90:103-137,
// boundary_kernel.f90:477-502).  With one thread the pair order and the
// summation order equal the reference's single-thread order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <string>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/simp_gpu.h"

namespace {

const double PI = 3.1415926535897932;  // globals.f90:199

// Default-real (single precision) literals as gfortran stores them.
inline double real4(float v) { return (double)v; }

struct Orc {
    simp_params P;
    int maxn = 0, maxnb = 0;
    int ntotal = 0, ntotalb = 0;
    int scale_h = 1;
    int itimestep = 0;
    double dt = 0.0, current_time = 0.0, max_hsml = 0.0;
    // data_variables.f90:26-124, column-major x(2, n) stored interleaved
    std::vector<double> x, vx, mass, rho, p, hsml, A, h, c;
    std::vector<double> xb, massb, b_normal;
    std::vector<double> dvxdt, dxdt, dAdt, dhdt, drhodt;
    std::vector<double> kernel_zero;
    std::vector<double> eps11, eps12, eps22, zeta, eta, sig11, sig12, sig22;
    int nip = 0, bnip = 0;
    std::vector<int> p_i, p_j, bp_i, bp_j;      // 1-based like the reference
    std::vector<double> r_ij, hsml_ij, br_ij, w, dwdx;
    std::vector<int> count_np;
    std::string err;
    bool bad = false;   // the state blew up (no bucket grid could be built)
    // regularisation pair loops: 0 per pair (a pair outside the viscosity
    // criterion contributes nothing, XSPH antisymmetric: the library's
    // form); 1 the reference's serial loops literally (pi_ij keeps the last
    // pair's value, regularization.f90:193-196, 285-291; XSPH adds the same
    // signed term to both particles, :82-89)
    int reg_literal = 0;
};

// ---------------------------------------------------------------------------
// Integer powers as gfortran expands x**n for constant n (products).
inline double p2(double a) { return a * a; }
inline double p3(double a) { return (a * a) * a; }
inline double p7(double a) { double a2 = a * a; double a4 = a2 * a2; return a4 * (a2 * a); }
inline double p8(double a) { double a2 = a * a; double a4 = a2 * a2; return a4 * a4; }

// Fortran NINT: nearest integer, halves away from zero.
inline long fnint(double v) { return lround(v); }

int num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int thread_id() {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

// OpenMP reduction of an array over a pair loop, with the private copies on
// the heap (array-section reductions live on thread stacks).  Each thread
// accumulates into a zeroed copy; copies are added to dst in thread order,
// which with one thread reproduces the serial summation exactly.
template <class Body>
void reduce_pairs(int npairs, double *dst, size_t len, int chunk, Body body) {
    const int nthr = num_threads();
    std::vector<std::vector<double>> priv(nthr);
#pragma omp parallel num_threads(nthr)
    {
        std::vector<double> &acc = priv[thread_id()];
        acc.assign(len, 0.0);
#pragma omp for schedule(dynamic, chunk)
        for (int k = 0; k < npairs; ++k) body(k, acc.data());
    }
    for (int t = 0; t < nthr; ++t)
        if (!priv[t].empty())
            for (size_t i = 0; i < len; ++i) dst[i] = dst[i] + priv[t][i];
}

// ---------------------------------------------------------------------------
// scale_h of kernel skf, initialize.f90:208-217 (9: the restored cubic, 2).
int scale_h_of(int skf) {
    if (skf == 4 || skf == 5 || skf == 6) return 1;
    if (skf == 1 || skf == 9) return 2;
    return 3;
}

// Fortran's x ** n for a small integer n, by multiplication.
double ipow(double x, int n) {
    double r = 1.0;
    for (int k = 0; k < n; ++k) r *= x;
    return r;
}

// Pair kernel, kernel.f90:5-45 dispatch.
//   in : r, hij (hsml_ij), dx(2)  out: w, dw(2), k0 (kernel_zero value)
// Each kernel in the reference's own arithmetic; default-real literals keep
// their single-precision values (real4).  Cubic spline: kernel.f90:324-340
// (commented out in the reference), restored with factor = 15/(7 pi)
// (scale_h/hsml_ij)^2 so that it is normalised like the other kernels.
void pair_kernel(const Orc &o, double r, double hij, const double dx[2],
                 double *w, double dw[2], double *k0) {
    const double sh = (double)o.scale_h;
    const double q = r / hij * sh;
    double wt = 0.0, g = 0.0;
    switch (o.P.skf) {
        case 1: {   // Quadratic, kernel.f90:269-276
            const double factor = 2.0 / PI * p2(sh / hij);
            *k0 = factor * (3.0 / 4.0);
            wt = factor * (3.0 / 16.0 * p2(q) - 3.0 / 4.0 * q + 3.0 / 4.0);
            g = factor * (3.0 / 8.0 * q - 3.0 / 4.0);
            break;
        }
        case 2: {   // Gaussian, kernel.f90:136-144
            const double factor = 1.0 / PI * p2(sh / hij);
            *k0 = factor;
            wt = factor * std::exp(-p2(q));
            g = factor * (-2 * q * std::exp(-p2(q)));
            break;
        }
        case 3: {   // quintic spline, kernel.f90:193-219
            const double factor = 7.0 / (478.0 * PI) * p2(sh / hij);
            *k0 = factor * (243 - 6 * 32 + 15);
            if (q >= 0.0 && q <= 1.0) {
                wt = factor * (ipow(3 - q, 5) - 6 * ipow(2 - q, 5) + 15 * ipow(1 - q, 5));
                g = factor * (-5 * ipow(3 - q, 4) + 30 * ipow(2 - q, 4) - 75 * ipow(1 - q, 4));
            }
            if (q > 1.0 && q <= 2.0) {
                wt = factor * (ipow(3 - q, 5) - 6 * ipow(2 - q, 5));
                g = factor * (-5 * ipow(3 - q, 4) + 30 * ipow(2 - q, 4));
            }
            if (q > 2.0 && q <= 3.0) {
                wt = factor * ipow(3 - q, 5);
                g = factor * (-5 * ipow(3 - q, 4));
            }
            break;
        }
        case 4: {   // Wendland C2, kernel.f90:387-393
            const double factor = 3.0 / (2.0 * PI) * p2(sh / hij);
            *k0 = factor;
            wt = factor * (ipow(1.0 - q, 4) * (1 + 4 * q));
            g = factor * (20.0 * (ipow(q, 4) - 3 * p3(q) + 3 * p2(q) - q));
            break;
        }
        case 5: {   // Wendland C4, kernel.f90:443-450
            const double factor = 3.0 / PI * p2(sh / hij);
            *k0 = factor * 3;
            wt = factor * (ipow(1 - q, 6) * (35 * p2(q) + 18 * q + 3));
            g = factor * (-56 * q * (5 * q + 1) * ipow(1 - q, 5));
            break;
        }
        case 6: {   // Wendland C6, kernel.f90:498-508
            const double factor = 78.0 / (7.0 * PI) * p2(sh / hij);
            *k0 = factor;
            const double om = 1.0 - q;
            wt = factor * p8(om) * (32.0 * p3(q) + 25.0 * p2(q) + 8.0 * q + 1.0);
            g = factor * (-22.0 * q * p7(om) * (16.0 * p2(q) + 7.0 * q + 1.0));
            break;
        }
        case 7: {   // Marquis, kernel.f90:555-563
            const double factor = 1.0 / PI * p2(sh / hij);
            *k0 = factor * (0.5 - 0.5 * std::tanh(0.0));
            wt = factor * (0.5 - 0.5 * std::tanh(300 * (q - 1)));
            g = factor * (-150 * std::pow(std::cosh(300 * (-1 + q)), -2));
            break;
        }
        case 8: {   // Marquis2, kernel.f90:612-620 (log(2.) of a default real)
            const double C1 = 10.0, C2 = 50.0;
            const double l2 = (double)std::log(2.0f);
            const double factor = 1.0 / (real4(34.1558f) * PI * p2(hij));
            *k0 = factor * C2 * (std::log(std::cosh(C1)) / C1 + 1 + l2 / C1);
            wt = factor * C2 * (std::log(std::cosh(C1 * (1 - q))) / C1 - q + 1 + l2 / C1);
            g = factor * (-C2 * std::tanh(C1 * (1 - q)) - 1);
            break;
        }
        default: {  // 9, cubic spline
            const double factor = 15.0 / (7.0 * PI) * p2(sh / hij);
            const double c23 = real4(2.0f / 3.0f), c16 = real4(1.0f / 6.0f);
            *k0 = factor * c23;
            if (q >= 0.0 && q <= 1.0) {
                wt = factor * (c23 - p2(q) + 0.5 * p3(q));
                g = factor * (-2.0 * q + 1.5 * p2(q));
            }
            if (q > 1.0 && q <= 2.0) {
                wt = factor * (c16 * p3(2.0 - q));
                g = factor * (-0.5 * p2(2.0 - q));
            }
            break;
        }
    }
    *w = wt;
    for (int d = 0; d < 2; ++d) dw[d] = g / hij * (dx[d] / r) * sh;
}

// Boundary kernel value bw, boundary_kernel.f90:20-45 dispatch (the Marquis
// kernels use b_Gaussian there).
// Wendland C6: :489-494, with factor from hsml_ij(int_id) (the pair array of
// the particle NNPS indexed by the boundary-pair index, as the reference does).
// Cubic: in the style of b_Quadratic (:106-112), support b_length, scale_h = 2.
double boundary_w(const Orc &o, double br, int int_id) {
    const double sh = (double)o.scale_h;
    const double bl = o.P.b_length;
    const double q = br / bl * sh;
    switch (o.P.skf) {
        case 1:     // b_Quadratic, :106-108
            return 2.0 / PI * p2(sh / bl) * (3.0 / 16.0 * p2(q) - 3.0 / 4.0 * q + 3.0 / 4.0);
        case 2: case 7: case 8:   // b_Gaussian, :177-179
            return 1.0 / PI * p2(sh / bl) * std::exp(-p2(q));
        case 3: {   // b_quintic_spline, :250-269
            const double factor = 15.0 / (478.0 * PI) * p2(sh / bl);
            double bw = 0.0;
            if (q >= 0.0 && q <= 1.0) bw = factor * (ipow(3 - q, 5) - 6 * ipow(2 - q, 5) + 15 * ipow(1 - q, 5));
            if (q > 1.0 && q <= 2.0) bw = factor * (ipow(3 - q, 5) - 6 * ipow(2 - q, 5));
            if (q > 2.0 && q <= 3.0) bw = factor * ipow(3 - q, 5);
            return bw;
        }
        case 4:     // b_Wendland_C2, :342-344
            return 3.0 / (2.0 * PI) * p2(sh / bl) * (ipow(1.0 - q, 4) * (1 + 4 * q));
        case 5:     // b_Wendland_C4, :416-418
            return 3.0 / PI * p2(sh / bl) * (ipow(1 - q, 6) * (35 * p2(q) + 18 * q + 3));
        case 6: {
            const double hij = (int_id - 1 < (int)o.hsml_ij.size()) ? o.hsml_ij[int_id - 1] : 0.0;
            const double factor = 78.0 / (7.0 * PI) * p2(sh / hij);
            const double om = 1.0 - q;
            return factor * p8(om) * (32.0 * p3(q) + 25.0 * p2(q) + 8.0 * q + 1.0);
        }
        default: {
            const double factor = 15.0 / (7.0 * PI) * p2(sh / bl);
            const double c23 = real4(2.0f / 3.0f), c16 = real4(1.0f / 6.0f);
            double bw = 0.0;
            if (q >= 0.0 && q <= 1.0) bw = factor * (c23 - p2(q) + 0.5 * p3(q));
            if (q > 1.0 && q <= 2.0) bw = factor * (c16 * p3(2.0 - q));
            return bw;
        }
    }
}

// factor * dW/dq of the boundary kernels, from which boundary_kernel.f90
// forms bdwdx = -factor * (dW/dq) / b_length * (bdx / br) * scale_h
// (b_Quadratic :111-112, b_Gaussian :182-184, b_quintic_spline :257-274,
// b_Wendland_C2 :348-349, b_Wendland_C4 :422-423, b_Wendland_C6 :495-496;
// the restored cubic: its kernel's derivative).
double boundary_fdwdq(const Orc &o, double br, int int_id) {
    const double sh = (double)o.scale_h;
    const double bl = o.P.b_length;
    const double q = br / bl * sh;
    switch (o.P.skf) {
        case 1:
            return 2.0 / PI * p2(sh / bl) * (3.0 / 8.0 * q - 3.0 / 4.0);
        case 2: case 7: case 8:
            return 1.0 / PI * p2(sh / bl) * (-2 * q * std::exp(-p2(q)));
        case 3: {
            const double factor = 15.0 / (478.0 * PI) * p2(sh / bl);
            double d = 0.0;
            if (q >= 0.0 && q <= 1.0) d = factor * (-5 * ipow(3 - q, 4) + 30 * ipow(2 - q, 4) - 75 * ipow(1 - q, 4));
            if (q > 1.0 && q <= 2.0) d = factor * (-5 * ipow(3 - q, 4) + 30 * ipow(2 - q, 4));
            if (q > 2.0 && q <= 3.0) d = factor * (-5 * ipow(3 - q, 4));
            return d;
        }
        case 4:
            return 3.0 / (2.0 * PI) * p2(sh / bl) * (20.0 * (ipow(q, 4) - 3 * p3(q) + 3 * p2(q) - q));
        case 5:
            return 3.0 / PI * p2(sh / bl) * (-56 * q * (5 * q + 1) * ipow(1 - q, 5));
        case 6: {
            const double hij = (int_id - 1 < (int)o.hsml_ij.size()) ? o.hsml_ij[int_id - 1] : 0.0;
            const double factor = 78.0 / (7.0 * PI) * p2(sh / hij);
            return factor * (-22.0 * q * p7(1 - q) * (16 * p2(q) + 7.0 * q + 1));
        }
        default: {
            const double factor = 15.0 / (7.0 * PI) * p2(sh / bl);
            double d = 0.0;
            if (q >= 0.0 && q <= 1.0) d = factor * (1.5 * p2(q) - 2.0 * q);
            if (q > 1.0 && q <= 2.0) d = factor * (-0.5 * p2(2.0 - q));
            return d;
        }
    }
}

// ---------------------------------------------------------------------------
// NNPS: direct_find, nnps.f90:41-148.
void direct_find(Orc &o) {
    o.nip = 0; o.bnip = 0;
    o.p_i.clear(); o.p_j.clear(); o.r_ij.clear(); o.hsml_ij.clear();
    o.bp_i.clear(); o.bp_j.clear(); o.br_ij.clear();
    o.count_np.assign(o.ntotal, 0);
    const double *x = o.x.data();
    for (int i = 0; i < o.ntotal - 1; ++i) {
        for (int j = i + 1; j < o.ntotal; ++j) {
            const double ax = x[2 * i] - x[2 * j], ay = x[2 * i + 1] - x[2 * j + 1];
            const double d = std::sqrt(ax * ax + ay * ay);
            const double mh = (o.hsml[i] + o.hsml[j]) / 2.0;
            if (d <= mh) {
                o.p_i.push_back(i + 1); o.p_j.push_back(j + 1);
                o.r_ij.push_back(d); o.hsml_ij.push_back(mh);
                o.count_np[i]++; o.count_np[j]++;
            }
        }
    }
    o.nip = (int)o.p_i.size();
    if (o.P.boundary_pressure || o.P.boundary_friction) {
        for (int i = 0; i < o.ntotalb; ++i)
            for (int j = 0; j < o.ntotal; ++j) {
                const double ax = o.xb[2 * i] - x[2 * j], ay = o.xb[2 * i + 1] - x[2 * j + 1];
                const double d = std::sqrt(ax * ax + ay * ay);
                if (d <= o.P.b_length) {
                    o.bp_i.push_back(i + 1); o.bp_j.push_back(j + 1); o.br_ij.push_back(d);
                    o.count_np[j]++;
                }
            }
        o.bnip = (int)o.bp_i.size();
    }
}

// NNPS: bucket_search, nnps.f90:155-517.
void bucket_search(Orc &o) {
    const int n = o.ntotal, nb = o.ntotalb;
    const double *x = o.x.data(), *xb = o.xb.data();
    o.count_np.assign(n, 0);

    // :211-216
    double hmin = o.hsml[0];
    for (int i = 1; i < n; ++i) hmin = std::min(hmin, o.hsml[i]);
    const double bin_size = 2.0 * hmin;
    double mnx = x[0], mxx = x[0], mny = x[1], mxy = x[1];
    for (int i = 0; i < nb; ++i) {
        mnx = std::min(mnx, xb[2 * i]); mxx = std::max(mxx, xb[2 * i]);
        mny = std::min(mny, xb[2 * i + 1]); mxy = std::max(mxy, xb[2 * i + 1]);
    }
    for (int i = 0; i < n; ++i) {
        mnx = std::min(mnx, x[2 * i]); mxx = std::max(mxx, x[2 * i]);
        mny = std::min(mny, x[2 * i + 1]); mxy = std::max(mxy, x[2 * i + 1]);
    }
    // a state that blew up (non-finite or absurdly spread) has no bucket grid;
    // the reference would index out of its arrays here
    if (!std::isfinite(mnx + mxx + mny + mxy + bin_size) ||
        (mxx - mnx) / bin_size > 1e6 || (mxy - mny) / bin_size > 1e6) {
        o.bad = true;
        o.nip = o.bnip = 0;
        o.p_i.clear(); o.p_j.clear(); o.r_ij.clear(); o.hsml_ij.clear();
        o.bp_i.clear(); o.bp_j.clear(); o.br_ij.clear();
        return;
    }
    const long bc1 = fnint(mnx / bin_size), bc2 = fnint(mxx / bin_size);
    const long bc3 = fnint(mny / bin_size), bc4 = fnint(mxy / bin_size);
    const long kx0 = bc1 - 1, ky0 = bc3 - 1;
    const long nkx = bc2 - bc1 + 3, nky = bc4 - bc3 + 3;
    // number_bin / bins (:218-224); bins kept as growable lists (the
    // reference's max_ind_int per-bin capacity is a fixed array bound).
    std::vector<std::vector<int>> bins((size_t)(nkx * nky));
    auto B = [&](long k, long l) -> std::vector<int> & { return bins[(size_t)((l - ky0) * nkx + (k - kx0))]; };
    // :246-254 serial binning in index order
    for (int i = 0; i < n; ++i) {
        const long xbn = fnint(x[2 * i] / bin_size), ybn = fnint(x[2 * i + 1] / bin_size);
        B(xbn, ybn).push_back(i + 1);
    }

    struct Buf { std::vector<int> pi, pj; std::vector<double> r, hm; std::vector<int> cnt; };
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    std::vector<Buf> bufs(nthr);
    const long ncx = bc2 - bc1 + 1, ncy = bc4 - bc3 + 1;

    auto test_pair = [&](Buf &b, int id1, int id2) {
        const int a = id1 - 1, c = id2 - 1;
        const double ax = x[2 * a] - x[2 * c], ay = x[2 * a + 1] - x[2 * c + 1];
        const double d = std::sqrt(ax * ax + ay * ay);             // :277
        const double mh = (o.hsml[a] + o.hsml[c]) / 2.0;            // :278
        if (d <= mh) {                                              // :281
            b.pi.push_back(id1); b.pj.push_back(id2); b.r.push_back(d); b.hm.push_back(mh);
            b.cnt[a]++; b.cnt[c]++;
        }
    };

#pragma omp parallel num_threads(nthr)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        Buf &b = bufs[tid];
        b.cnt.assign(n, 0);
        // :259-411, COLLAPSE(2) over (l, k)
#pragma omp for schedule(dynamic, 1) collapse(2)
        for (long l = bc3; l <= bc4; ++l) {
            for (long k = bc1; k <= bc2; ++k) {
                const std::vector<int> &cell = B(k, l);
                const int nc = (int)cell.size();
                for (int i = 0; i < nc - 1; ++i)
                    for (int j = i + 1; j < nc; ++j) test_pair(b, cell[i], cell[j]);
                for (int i = 0; i < nc; ++i) {
                    const int id1 = cell[i];
                    for (int id2 : B(k + 1, l)) test_pair(b, id1, id2);      // right
                    for (int id2 : B(k, l + 1)) test_pair(b, id1, id2);      // up
                    for (int id2 : B(k + 1, l + 1)) test_pair(b, id1, id2);  // up-right
                    for (int id2 : B(k - 1, l + 1)) test_pair(b, id1, id2);  // up-left
                }
            }
        }
    }
    (void)ncx; (void)ncy;
    // :426-433 merge (thread order; one thread = reference serial order)
    o.p_i.clear(); o.p_j.clear(); o.r_ij.clear(); o.hsml_ij.clear();
    for (int t = 0; t < nthr; ++t) {
        Buf &b = bufs[t];
        o.p_i.insert(o.p_i.end(), b.pi.begin(), b.pi.end());
        o.p_j.insert(o.p_j.end(), b.pj.begin(), b.pj.end());
        o.r_ij.insert(o.r_ij.end(), b.r.begin(), b.r.end());
        o.hsml_ij.insert(o.hsml_ij.end(), b.hm.begin(), b.hm.end());
        for (int i = 0; i < n; ++i) o.count_np[i] += b.cnt[i];
    }
    o.nip = (int)o.p_i.size();

    // :440-507 boundary pairs, 3x3 bins around each boundary particle
    o.bp_i.clear(); o.bp_j.clear(); o.br_ij.clear();
    if (o.P.boundary_pressure || o.P.boundary_friction) {
        for (int i = 0; i < nb; ++i) {
            const long xbn = fnint(xb[2 * i] / bin_size), ybn = fnint(xb[2 * i + 1] / bin_size);
            for (long k = ybn - 1; k <= ybn + 1; ++k)
                for (long j = xbn - 1; j <= xbn + 1; ++j) {
                    if (j < kx0 || j >= kx0 + nkx || k < ky0 || k >= ky0 + nky) continue;
                    for (int id2 : B(j, k)) {
                        const int c = id2 - 1;
                        const double ax = xb[2 * i] - x[2 * c], ay = xb[2 * i + 1] - x[2 * c + 1];
                        const double d = std::sqrt(ax * ax + ay * ay);  // :473
                        if (d <= o.P.b_length) {                         // :476
                            o.bp_i.push_back(i + 1); o.bp_j.push_back(id2); o.br_ij.push_back(d);
                            o.count_np[c]++;
                        }
                    }
                }
        }
    }
    o.bnip = (int)o.bp_i.size();
}

void nnps(Orc &o) {
    if (o.P.nnps_algorithm == 1) direct_find(o); else bucket_search(o);
}

// ---------------------------------------------------------------------------
// internal_stress.f90:5-164 with bulk_viscosity.f90:35-79,
// shear_viscosity.f90:36-60, eos.f90:39-61 / 112-151, stress_tensor.f90:31-39
// and stress_1 (internal_stress.f90:62-139).
void internal_stress(Orc &o) {
    const int n = o.ntotal;
    const simp_params &P = o.P;
    const double em2 = 1.0 / (P.e * P.e);  // e ** (-2)
    if (P.viscosity) {
        for (int i = 0; i < n; ++i)
            o.p[i] = P.P_star * o.h[i] * std::exp(-(P.c_eos * (1.0 - o.A[i])));   // :24
        if (P.rheology == 2) {
            // Mohr-Coulomb: MC_bulk_viscosity (bulk_viscosity.f90:86-145) and
            // MC_shear_viscosity (shear_viscosity.f90:67-124); mu = tan(phi pi/180.)
            const double zero = 1.0e-18, mu = std::tan(P.phi * PI / 180.0);
            std::vector<double> e1(n), e2(n);
            for (int i = 0; i < n; ++i) {
                const double rt = std::sqrt(p2(o.eps11[i] - o.eps22[i]) + 4 * p2(o.eps12[i]));
                e1[i] = 0.5 * ((o.eps11[i] + o.eps22[i]) + rt);
                e2[i] = 0.5 * ((o.eps11[i] + o.eps22[i]) - rt);
                double eI = std::fabs(e1[i] + e2[i]);
                if (eI < zero) eI = zero;
                o.zeta[i] = 0.5 * o.p[i] * (1 + P.k_t) / eI;
                if (o.zeta[i] > P.zeta_max * o.p[i]) o.zeta[i] = P.zeta_max * o.p[i];
            }
            for (int i = 0; i < n; ++i) {
                double eII = e1[i] - e2[i];
                if (std::fabs(eII) < zero) eII = zero;
                o.eta[i] = mu * (0.5 * o.p[i] * (1 + P.k_t) - o.zeta[i] * (e1[i] + e2[i])) / eII;
                if (o.eta[i] > P.eta_max * o.p[i]) o.eta[i] = P.eta_max * o.p[i];
            }
        } else {
            for (int i = 0; i < n; ++i) {                                          // bulk :65-76
                double delta = std::pow((p2(o.eps11[i]) + p2(o.eps22[i])) * (1.0 + em2) +
                                        4.0 * em2 * p2(o.eps12[i]) +
                                        2.0 * o.eps11[i] * o.eps22[i] * (1.0 - em2), 0.5);
                if (std::fabs(delta) < P.delta_min) delta = P.delta_min;
                o.zeta[i] = 0.5 * o.p[i] * (1.0 + P.k_t) / delta;
            }
            for (int i = 0; i < n; ++i) o.eta[i] = o.zeta[i] / (P.e * P.e);        // shear :57
        }
    }
    if (P.pressure_force) {
        if (P.eos_alg == 1) {
            for (int i = 0; i < n; ++i)
                o.p[i] = P.P_star * o.h[i] * std::exp(-(P.c_eos * (1.0 - o.A[i])));
        } else if (P.eos_alg == 2) {  // gutfraind_eos :96-104
            const double rho_max = 934.0, rho_0 = P.rho_ice;
            for (int i = 0; i < n; ++i) {
                const double gamma = 1.9e5 * o.h[i] * std::exp(-20 * (1 - o.A[i]));
                o.p[i] = gamma * (o.rho[i] - rho_0) / (rho_max - o.rho[i]);
                if (o.p[i] < 0.0) o.p[i] = 0.0;
            }
        } else {  // kreyscher_eos :141-147
            for (int i = 0; i < n; ++i) {
                const double delta = std::pow((p2(o.eps11[i]) + p2(o.eps22[i])) * (1.0 + em2) +
                                              4.0 * em2 * p2(o.eps12[i]) +
                                              2.0 * o.eps11[i] * o.eps22[i] * (1.0 - em2), 0.5);
                o.p[i] = o.zeta[i] * 2.0 * delta / (1.0 + P.k_t);
            }
        }
    }
    for (int i = 0; i < n; ++i) {                                                   // stress_tensor
        o.sig11[i] = (o.zeta[i] + o.eta[i]) * o.eps11[i] + (o.zeta[i] - o.eta[i]) * o.eps22[i] -
                     o.p[i] * (1.0 - P.k_t) / 2.0;
        o.sig12[i] = 2.0 * o.eta[i] * o.eps12[i];
        o.sig22[i] = (o.zeta[i] + o.eta[i]) * o.eps22[i] + (o.zeta[i] - o.eta[i]) * o.eps11[i] -
                     o.p[i] * (1.0 - P.k_t) / 2.0;
    }
    const double rho_ice = P.rho_ice;
    if (P.pa_sph == 2) {
        // stress_2 :146-219
        reduce_pairs(o.nip, o.dvxdt.data(), 2 * (size_t)n, 4096, [&](int k, double *dv) {
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double g1 = o.dwdx[2 * k], g2 = o.dwdx[2 * k + 1];
            double cj = (o.sig11[j] * g1 + o.sig12[j] * g2);
            double ci = (o.sig11[i] * g1 + o.sig12[i] * g2);
            dv[2 * i] = dv[2 * i] + o.mass[j] / rho_ice / o.h[i] / o.rho[j] * (ci + cj);
            dv[2 * j] = dv[2 * j] - o.mass[i] / rho_ice / o.h[j] / o.rho[i] * (ci + cj);
            cj = (o.sig12[j] * g1 + o.sig22[j] * g2);
            ci = (o.sig12[i] * g1 + o.sig22[i] * g2);
            dv[2 * i + 1] = dv[2 * i + 1] + o.mass[j] / rho_ice / o.h[i] / o.rho[j] * (ci + cj);
            dv[2 * j + 1] = dv[2 * j + 1] - o.mass[i] / rho_ice / o.h[j] / o.rho[i] * (ci + cj);
        });
        return;
    }
    // stress_1 :103-137 (REDUCTION(+:dvxdt))
    reduce_pairs(o.nip, o.dvxdt.data(), 2 * (size_t)n, 4096, [&](int k, double *dv) {
        const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
        const double g1 = o.dwdx[2 * k], g2 = o.dwdx[2 * k + 1];
        double cj = (o.sig11[j] * g1 + o.sig12[j] * g2) / p2(o.rho[j]);
        double ci = (o.sig11[i] * g1 + o.sig12[i] * g2) / p2(o.rho[i]);
        dv[2 * i] = dv[2 * i] + o.rho[i] * o.mass[j] / rho_ice / o.h[i] * (ci + cj);
        dv[2 * j] = dv[2 * j] + o.rho[j] * o.mass[i] / rho_ice / o.h[j] * (-ci - cj);
        cj = (o.sig12[j] * g1 + o.sig22[j] * g2) / p2(o.rho[j]);
        ci = (o.sig12[i] * g1 + o.sig22[i] * g2) / p2(o.rho[i]);
        dv[2 * i + 1] = dv[2 * i + 1] + o.rho[i] * o.mass[j] / rho_ice / o.h[i] * (ci + cj);
        dv[2 * j + 1] = dv[2 * j + 1] + o.rho[j] * o.mass[i] / rho_ice / o.h[j] * (-ci - cj);
    });
}

// boundary_kernel.f90:477-502 + boundary_force.f90:74-84 (bf_Monaghan,
// normal force).  The reference updates dvxdt from a called routine inside a
// reduction region (a race with several threads); this loop is serial.
// boundary_kernel.f90:5-45 (one loop per kernel, the same for all) with
// boundary_force.f90 called per boundary pair: bfa 1 bf_Monaghan :38-102,
// 2 bf_Wang :109-176, 3 bf_Marquis :183-225.
void boundary_kernel(Orc &o) {
    const simp_params &P = o.P;
    const double sh = (double)o.scale_h;
    for (int k = 0; k < o.bnip; ++k) {
        const int ci = o.bp_j[k] - 1;  // particle
        const int cj = o.bp_i[k] - 1;  // boundary particle
        const double bdx[2] = {o.xb[2 * cj] - o.x[2 * ci], o.xb[2 * cj + 1] - o.x[2 * ci + 1]};
        const double br = o.br_ij[k];
        const double bw = boundary_w(o, br, k + 1);
        const double fd = boundary_fdwdq(o, br, k + 1);
        const double bdwdx[2] = {-fd / P.b_length * (bdx[0] / br) * sh, -fd / P.b_length * (bdx[1] / br) * sh};
        const double *v = &o.vx[2 * ci];
        if (P.bfa == 1) {
            if (P.boundary_pressure) {
                for (int d = 0; d < 2; ++d) {
                    const double Fb = P.kappa_n * bdx[d] * bw * 2.0 * o.massb[cj] /
                                      ((o.mass[ci] + o.massb[cj]) * p2(br));
                    o.dvxdt[2 * ci + d] = o.dvxdt[2 * ci + d] + (-1.0 * Fb) / o.rho[ci];
                }
            }
            if (P.boundary_friction) {                                    // :85-100
                const double v_r = v[0] * bdx[0] + v[1] * bdx[1];
                const double pi_aj = P.kappa_t * o.c[ci] * v_r / br / o.rho[ci];
                for (int d = 0; d < 2; ++d)
                    o.dvxdt[2 * ci + d] = o.dvxdt[2 * ci + d] + (-1.0 * o.massb[cj] * pi_aj * bdwdx[d]) / o.rho[ci];
            }
        } else if (P.bfa == 2) {
            if (P.boundary_pressure) {                                    // :146-172
                const double *bn = &o.b_normal[2 * cj];
                double vv[2];
                vv[0] = bn[0] * v[0] + bn[1] * v[1];
                vv[1] = std::sqrt(p2(v[0]) + p2(v[1])) - vv[0];
                double F[2] = {o.mass[ci] * vv[0] / o.dt, o.mass[ci] * vv[1] / o.dt};
                if (P.boundary_friction && std::fabs(vv[1]) > std::fabs(P.xi * vv[0])) {
                    vv[1] = vv[1] * P.xi * std::fabs(F[0] / F[1]);
                    F[1] = o.mass[ci] * vv[1] / o.dt;
                }
                o.dvxdt[2 * ci] = o.dvxdt[2 * ci] + (F[0] * bn[0] + F[1] * bn[1]);
                o.dvxdt[2 * ci + 1] = o.dvxdt[2 * ci + 1] + (F[0] * bn[1] - F[1] * bn[0]);
            }
        } else if (P.bfa == 3) {
            if (P.boundary_pressure) continue;                            // :208-210
            if (P.boundary_friction)                                      // :213-216
                for (int d = 0; d < 2; ++d)
                    o.dvxdt[2 * ci + d] = o.dvxdt[2 * ci + d] - v[d] * (1 - (br / P.b_length));
        }
    }
}

void wind_at(const Orc &o, int i, double W[2]) {
    const simp_params &P = o.P;
    if (P.wind_kind == SIMP_WIND_VORTEX) {
        const double rx = o.x[2 * i] - P.vortex_x, ry = o.x[2 * i + 1] - P.vortex_y;
        const double r = std::sqrt(rx * rx + ry * ry);
        if (r == 0.0) { W[0] = 0.0; W[1] = 0.0; return; }
        const double s = r / P.vortex_radius;
        const double U = P.vortex_umax * s * std::exp(0.5 * (1.0 - s * s));
        W[0] = -U * ry / r; W[1] = U * rx / r;
    } else {
        W[0] = P.wind_u; W[1] = P.wind_v;
    }
}

// wind_forcing.f90:35-51, water_drag.f90:35-53.
void external_forces(Orc &o) {
    const simp_params &P = o.P;
    if (P.wind_force && o.current_time > 0.0 * 3600.0) {
        for (int i = 0; i < o.ntotal; ++i) {
            double W[2]; wind_at(o, i, W);
            for (int d = 0; d < 2; ++d) {
                const double rel = W[d] - o.vx[2 * i + d];
                o.dvxdt[2 * i + d] = o.dvxdt[2 * i + d] +
                                     (P.c_wind * P.rho_air * rel * std::fabs(rel)) / (o.h[i] * P.rho_ice);
            }
        }
    }
    if (P.water_force && o.current_time > 0.0 * 3600.0) {
        const double C[2] = {P.current_u, P.current_v};
        for (int i = 0; i < o.ntotal; ++i)
            for (int d = 0; d < 2; ++d) {
                const double rel = C[d] - o.vx[2 * i + d];
                o.dvxdt[2 * i + d] = o.dvxdt[2 * i + d] +
                                     (P.c_water * P.rho_water * rel * std::fabs(rel)) / (o.h[i] * P.rho_ice);
            }
    }
}

// The sound speed the reference keeps in c(:): c_yang of the current density
// when sound_speed refreshes it (artificial viscosity, Monaghan time step or
// boundary friction, sound_speed.f90:21-27), else never set (zero).
bool sound_speed_on(const simp_params &P) {
    return P.artificial_visc || P.tse == 1 || P.boundary_friction;
}

// regularization.f90:5-310, called by single_step.f90:99-101 after the drag
// terms: XSPH (:45-95) when xsph_regularization, then the artificial
// viscosity of art_visc_alg (:29-35), Hernquist-Katz (:102-213) or Monaghan
// (:220-308), whichever of the two switches brought it here.  Both loops run
// serially over the pair list with the last right-hand side's w and dwdx.
void regularization(Orc &o) {
    const simp_params &P = o.P;
    const int n = o.ntotal;
    const bool lit = o.reg_literal != 0;
    if (P.xsph_regularization) {
        std::vector<double> xs(2 * (size_t)n, 0.0);
        for (int k = 0; k < o.nip; ++k) {
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
            const double rbar = 0.5 * (o.rho[i] + o.rho[j]);
            for (int d = 0; d < 2; ++d) {
                xs[2 * i + d] = xs[2 * i + d] + o.mass[j] * dvx[d] * o.w[k] / rbar;
                const double tj = o.mass[i] * dvx[d] * o.w[k] / rbar;
                xs[2 * j + d] = lit ? xs[2 * j + d] + tj : xs[2 * j + d] - tj;
            }
        }
        for (size_t q = 0; q < 2 * (size_t)n; ++q) o.dxdt[q] = o.dxdt[q] - P.chi * xs[q];   // :93
    }
    if (P.art_visc_alg == 1) {
        std::vector<double> div(n, 0.0), lv(n);
        for (int k = 0; k < o.nip; ++k) {                                 // :148-167
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
            const double w1 = dvx[0] * o.dwdx[2 * k], w4 = dvx[1] * o.dwdx[2 * k + 1];
            div[i] = div[i] - o.mass[j] * (w1 + w4) / o.rho[i];
            div[j] = div[j] - o.mass[i] * (w1 + w4) / o.rho[j];
        }
        for (int i = 0; i < n; ++i) {                                     // :170-176
            if (div[i] >= 0.0) div[i] = 0.0;
            lv[i] = (P.alpha_pi * o.hsml[i] * o.c[i] * std::fabs(div[i]) +
                     P.beta_pi * p2(std::fabs(div[i]) * o.hsml[i])) * o.rho[i];
        }
        double pi_ij = 0.0;
        for (int k = 0; k < o.nip; ++k) {                                 // :179-211
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double dx[2] = {o.x[2 * i] - o.x[2 * j], o.x[2 * i + 1] - o.x[2 * j + 1]};
            const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
            const double crit = dvx[0] * dx[0] + dvx[1] * dx[1];
            if (crit <= 0.0) pi_ij = lv[i] / p2(o.rho[i]) + lv[j] / p2(o.rho[j]);
            else if (!lit) pi_ij = 0.0;
            for (int d = 0; d < 2; ++d) {
                o.dvxdt[2 * i + d] = o.dvxdt[2 * i + d] - o.mass[j] * pi_ij * o.dwdx[2 * k + d];
                o.dvxdt[2 * j + d] = o.dvxdt[2 * j + d] + o.mass[i] * pi_ij * o.dwdx[2 * k + d];
            }
        }
    } else if (P.art_visc_alg == 2) {
        double pi_ij = 0.0;
        for (int k = 0; k < o.nip; ++k) {                                 // :268-306
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double dx[2] = {o.x[2 * i] - o.x[2 * j], o.x[2 * i + 1] - o.x[2 * j + 1]};
            const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
            const double v_r = dvx[0] * dx[0] + dvx[1] * dx[1];
            const double s_cor = real4(0.01f) * o.hsml_ij[k];
            if (v_r <= 0.0) {
                const double iota = o.hsml_ij[k] * v_r / (p2(o.r_ij[k]) + p2(s_cor));
                pi_ij = (P.beta_pi * p2(iota) - P.alpha_pi * iota * (o.c[i] + o.c[j]) / 2) /
                        ((o.rho[i] + o.rho[j]) / 2);
            } else if (!lit) {
                pi_ij = 0.0;
            }
            for (int d = 0; d < 2; ++d) {
                o.dvxdt[2 * i + d] = o.dvxdt[2 * i + d] - o.mass[j] * pi_ij * o.dwdx[2 * k + d];
                o.dvxdt[2 * j + d] = o.dvxdt[2 * j + d] + o.mass[i] * pi_ij * o.dwdx[2 * k + d];
            }
        }
    }
}

// single_step.f90:5-109.
void single_step(Orc &o) {
    const int n = o.ntotal;
    std::fill(o.dxdt.begin(), o.dxdt.begin() + 2 * n, 0.0);
    std::fill(o.dvxdt.begin(), o.dvxdt.begin() + 2 * n, 0.0);
    std::fill(o.dAdt.begin(), o.dAdt.begin() + n, 0.0);
    std::fill(o.dhdt.begin(), o.dhdt.begin() + n, 0.0);
    // div_v_sum (n) and grad_v_sum (4 n) in one buffer
    std::vector<double> dg(5 * (size_t)n, 0.0);
    double *div = dg.data(), *grad = dg.data() + n;
    std::fill(o.eps11.begin(), o.eps11.begin() + n, 0.0);
    std::fill(o.eps12.begin(), o.eps12.begin() + n, 0.0);
    std::fill(o.eps22.begin(), o.eps22.begin() + n, 0.0);

    nnps(o);                                                        // :47
    const int nip = o.nip;
    o.w.assign(nip, 0.0);
    o.dwdx.assign(2 * (size_t)nip, 0.0);
    double *kz = o.kernel_zero.data();
    // :50-77 kinematic pair loop, REDUCTION(-:div_v_sum, grad_v_sum)
    reduce_pairs(nip, dg.data(), dg.size(), 256, [&](int k, double *acc) {
        double *dv = acc, *gv = acc + n;
        const int ci = o.p_i[k] - 1, cj = o.p_j[k] - 1;
        const double dx[2] = {o.x[2 * ci] - o.x[2 * cj], o.x[2 * ci + 1] - o.x[2 * cj + 1]};
        const double dvx[2] = {o.vx[2 * ci] - o.vx[2 * cj], o.vx[2 * ci + 1] - o.vx[2 * cj + 1]};
        double w, dw[2], k0;
        pair_kernel(o, o.r_ij[k], o.hsml_ij[k], dx, &w, dw, &k0);
        kz[ci] = k0;
        o.w[k] = w; o.dwdx[2 * k] = dw[0]; o.dwdx[2 * k + 1] = dw[1];
        const double wdvx[4] = {dvx[0] * dw[0], dvx[1] * dw[0], dvx[0] * dw[1], dvx[1] * dw[1]};
        dv[ci] = dv[ci] - o.mass[cj] * (wdvx[0] + wdvx[3]);           // vector_divergence.f90:27
        dv[cj] = dv[cj] - o.mass[ci] * (wdvx[0] + wdvx[3]);           // :28
        for (int c = 0; c < 4; ++c) {                                  // vector_gradient.f90:56-69
            gv[4 * (size_t)ci + c] = gv[4 * (size_t)ci + c] - o.mass[cj] * wdvx[c] / o.rho[cj];
            gv[4 * (size_t)cj + c] = gv[4 * (size_t)cj + c] - o.mass[ci] * wdvx[c] / o.rho[ci];
        }
    });
    if (o.P.pressure_force || o.P.viscosity) {                      // :80-84
        for (int i = 0; i < n; ++i) {
            o.eps11[i] = grad[4 * (size_t)i];
            o.eps22[i] = grad[4 * (size_t)i + 3];
            o.eps12[i] = 0.5 * (grad[4 * (size_t)i + 1] + grad[4 * (size_t)i + 2]);
        }
    }
    internal_stress(o);                                             // :87
    if (o.P.boundary_pressure || o.P.boundary_friction) boundary_kernel(o);  // :90-92
    external_forces(o);                                             // :95-96
    if (o.P.xsph_regularization || o.P.artificial_visc) regularization(o);   // :99-101
    for (int i = 0; i < n; ++i) {                                   // :104-106
        o.dhdt[i] = -o.h[i] * div[i] / o.rho[i];
        o.dAdt[i] = -o.A[i] * div[i] / o.rho[i];
        o.dxdt[2 * i] = o.dxdt[2 * i] + o.vx[2 * i];
        o.dxdt[2 * i + 1] = o.dxdt[2 * i + 1] + o.vx[2 * i + 1];
    }
}

// density.f90:41-100 (sum_density).  k0_mode 0: the reference's kernel_zero
// array (set per pair for particle p_i, kernel.f90:503); 1: W(0) evaluated
// with the particle's own hsml.
void sum_density(Orc &o, int k0_mode, double *out) {
    const int n = o.ntotal;
    std::vector<double> num(n), den(n);
    for (int i = 0; i < n; ++i) {
        double k0 = o.kernel_zero[i];
        if (k0_mode == 1) {
            double w, dw[2];
            const double dx[2] = {0.0, 0.0};
            pair_kernel(o, 1.0, o.hsml[i], dx, &w, dw, &k0);
        }
        num[i] = k0 * o.mass[i];
        den[i] = k0 * o.mass[i] / o.rho[i];
    }
    for (int k = 0; k < o.nip; ++k) {
        const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
        den[i] = den[i] + o.mass[j] * o.w[k] / o.rho[j];
        den[j] = den[j] + o.mass[i] * o.w[k] / o.rho[i];
        num[i] = num[i] + o.mass[j] * o.w[k];
        num[j] = num[j] + o.mass[i] * o.w[k];
    }
    for (int i = 0; i < n; ++i) out[i] = num[i] / den[i];
}

// density.f90:107-165 (con_density): drhodt over the last NNPS's pairs and
// kernel gradients with the current velocities.
void con_density(Orc &o) {
    std::fill(o.drhodt.begin(), o.drhodt.begin() + o.ntotal, 0.0);
    for (int k = 0; k < o.nip; ++k) {
        const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
        const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
        const double w1 = dvx[0] * o.dwdx[2 * k], w4 = dvx[1] * o.dwdx[2 * k + 1];
        const double v_ij = w1 + w4;
        o.drhodt[i] = o.drhodt[i] + o.mass[j] * v_ij;
        o.drhodt[j] = o.drhodt[j] + o.mass[i] * v_ij;
    }
}

void density(Orc &o) {
    if (o.P.den_alg == 2) {
        con_density(o);
    } else if (o.P.den_alg == 1) {
        std::vector<double> r(o.ntotal);
        sum_density(o, 0, r.data());
        std::copy(r.begin(), r.end(), o.rho.begin());
    } else if (o.P.den_alg == 3) {
        for (int i = 0; i < o.ntotal; ++i) o.rho[i] = o.h[i] * o.P.rho_ice;   // :192
    }
}

// sound_speed.f90:20-27 with c_yang :54-55: only when something reads c.
void sound_speed(Orc &o) {
    const simp_params &P = o.P;
    if (!sound_speed_on(P)) return;
    for (int i = 0; i < o.ntotal; ++i)
        o.c[i] = std::pow(P.Y * (1 - P.nu) / (o.rho[i] * (1 + P.nu) * (1 - 2 * P.nu)), 0.5);
}

// mass_evolution.f90:20-71.
void mass_evolution(Orc &o) {
    if (o.P.sle == 2 || !o.P.mass_from_area) return;
    for (int i = 0; i < o.ntotal; ++i) {
        const double area = PI * p2(o.P.alpha * o.hsml[i]);
        o.mass[i] = o.P.rho_ice * o.A[i] * o.h[i] * area;
    }
}

// smoothing_length.f90:40-111 (Benz_hsml).  Without con_density the pair
// loop adds to drhodt, which nothing clears: it accumulates over the steps.
void benz_hsml(Orc &o) {
    const int n = o.ntotal;
    if (o.P.den_alg != 2) {
        for (int k = 0; k < o.nip; ++k) {
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
            const double w1 = dvx[0] * o.dwdx[2 * k], w4 = dvx[1] * o.dwdx[2 * k + 1];
            const double v_ij = w1 + w4;
            o.drhodt[i] = o.drhodt[i] + o.mass[j] * v_ij;
            o.drhodt[j] = o.drhodt[j] + o.mass[i] * v_ij;
        }
    }
    for (int i = 0; i < n; ++i) {
        const double dhsmldt = -o.hsml[i] * o.drhodt[i] / 2.0 / o.rho[i];   // dim = 2
        o.hsml[i] = o.hsml[i] + dhsmldt * o.dt;
        if (o.hsml[i] < 0.0) o.hsml[i] = o.hsml[i] - dhsmldt * o.dt;
    }
}

// smoothing_length.f90:118-145 (Marquis_hsml); sle = 0 keeps hsml.
void smoothing_length(Orc &o) {
    if (o.P.sle == 1) { benz_hsml(o); return; }
    if (o.P.sle != 2) return;
    for (int i = 0; i < o.ntotal; ++i) {
        o.hsml[i] = std::sqrt(o.mass[i] / o.rho[i]) * (double)o.P.hsml_multiplicity;
        if (o.hsml[i] > o.max_hsml) o.hsml[i] = o.max_hsml;
    }
}

// time_step.f90:40-124 (Monaghan_time_step): the force criterion from the
// last right-hand side's accelerations and the CFL criterion from the sound
// speed; with artificial viscosity the CFL criterion also takes the velocity
// divergence over the last right-hand side's pairs and kernel gradients with
// the current velocities, masses and densities (:89-115).
void monaghan_time_step(Orc &o) {
    const int n = o.ntotal;
    const simp_params &P = o.P;
    const double fF = 0.25;
    std::vector<double> div(n, 0.0);
    if (P.artificial_visc) {
        for (int k = 0; k < o.nip; ++k) {
            const int i = o.p_i[k] - 1, j = o.p_j[k] - 1;
            const double dvx[2] = {o.vx[2 * i] - o.vx[2 * j], o.vx[2 * i + 1] - o.vx[2 * j + 1]};
            const double w1 = dvx[0] * o.dwdx[2 * k], w4 = dvx[1] * o.dwdx[2 * k + 1];
            div[i] = div[i] - o.mass[j] * (w1 + w4) / o.rho[i];
            div[j] = div[j] - o.mass[i] * (w1 + w4) / o.rho[j];
        }
    }
    double mf = 0.0, mc = 0.0;
    for (int i = 0; i < n; ++i) {
        const double acc = std::pow(p2(o.dvxdt[2 * i]) + p2(o.dvxdt[2 * i + 1]), 0.5);
        const double a = o.hsml[i] / acc;
        const double c = P.artificial_visc
            ? real4(0.3f) * o.hsml[i] / (o.c[i] + o.hsml[i] * std::fabs(div[i]) +
                                         real4(1.2f) * (P.alpha_pi * o.c[i] + P.beta_pi * o.hsml[i] * std::fabs(div[i])))
            : o.hsml[i] / o.c[i];
        mf = (i == 0) ? a : std::min(mf, a);
        mc = (i == 0) ? c : std::min(mc, c);
    }
    const double dt_force = fF * std::pow(mf, 0.5);
    o.dt = std::min(dt_force, mc);
}

// time_step.f90:132-157 (VP_time_step); tse = 0 keeps dt.
void time_step(Orc &o) {
    if (o.P.tse == 1) { monaghan_time_step(o); return; }
    if (o.P.tse != 2) return;
    double m = 0.0;
    for (int i = 0; i < o.ntotal; ++i) {
        const double v = o.P.rho_ice * p2(o.hsml[i]) * o.P.delta_min / (o.P.P_star * (1.0 + o.P.k_t));
        m = (i == 0) ? v : std::min(m, v);
    }
    o.dt = m;
}

void clamp_A(Orc &o) {
    for (int i = 0; i < o.ntotal; ++i) if (o.A[i] > 1.0) o.A[i] = 1.0;
}

// time_integration.f90:155-282 (predictor_corrector).
void predictor_corrector(Orc &o) {
    const int n = o.ntotal;
    const double dt = o.dt;
    std::vector<double> x1(o.x.begin(), o.x.begin() + 2 * n), vx1(o.vx.begin(), o.vx.begin() + 2 * n);
    std::vector<double> h1(o.h.begin(), o.h.begin() + n), A1(o.A.begin(), o.A.begin() + n);
    std::vector<double> rho1(o.rho.begin(), o.rho.begin() + n);
    single_step(o);                                                  // :204
    for (int k = 0; k < 2 * n; ++k) {
        o.x[k] = o.x[k] + o.dxdt[k] * dt / 2.0;
        o.vx[k] = o.vx[k] + o.dvxdt[k] * dt / 2.0;
    }
    for (int i = 0; i < n; ++i) {
        o.h[i] = o.h[i] + o.dhdt[i] * dt / 2.0;
        o.A[i] = o.A[i] + o.dAdt[i] * dt / 2.0;
    }
    clamp_A(o);
    density(o);
    if (o.P.den_alg == 2)                                            // :220-223
        for (int i = 0; i < n; ++i) o.rho[i] = o.rho[i] + o.drhodt[i] * dt / 2.0;
    mass_evolution(o);
    sound_speed(o);
    single_step(o);                                                  // :233
    std::vector<double> x12(2 * n), vx12(2 * n), h12(n), A12(n), rho12(n);
    for (int k = 0; k < 2 * n; ++k) {
        x12[k] = x1[k] + o.dxdt[k] * dt / 2.0;
        vx12[k] = vx1[k] + o.dvxdt[k] * dt / 2.0;
    }
    for (int i = 0; i < n; ++i) {
        h12[i] = h1[i] + o.dhdt[i] * dt / 2.0;
        A12[i] = A1[i] + o.dAdt[i] * dt / 2.0;
    }
    density(o);                                                      // :242
    if (o.P.den_alg == 2)                                            // :245-247
        for (int i = 0; i < n; ++i) rho12[i] = rho1[i] + o.drhodt[i] * dt / 2.0;
    for (int k = 0; k < 2 * n; ++k) {
        o.x[k] = 2.0 * x12[k] - x1[k];
        o.vx[k] = 2.0 * vx12[k] - vx1[k];
    }
    for (int i = 0; i < n; ++i) {
        o.h[i] = 2.0 * h12[i] - h1[i];
        o.A[i] = 2.0 * A12[i] - A1[i];
    }
    clamp_A(o);
    density(o);
    if (o.P.den_alg == 2)                                            // :265-267
        for (int i = 0; i < n; ++i) o.rho[i] = 2.0 * rho12[i] - rho1[i];
    mass_evolution(o);
    sound_speed(o);
    smoothing_length(o);
    time_step(o);
}

// euler_scheme, time_integration.f90:86-148.
void euler_scheme(Orc &o) {
    const int n = o.ntotal;
    const double dt = o.dt;
    single_step(o);
    for (int k = 0; k < 2 * n; ++k) {
        o.x[k] = o.x[k] + o.dxdt[k] * dt;
        o.vx[k] = o.vx[k] + o.dvxdt[k] * dt;
    }
    for (int i = 0; i < n; ++i) {
        o.h[i] = o.h[i] + o.dhdt[i] * dt;
        o.A[i] = o.A[i] + o.dAdt[i] * dt;
    }
    clamp_A(o);
    density(o);
    if (o.P.den_alg == 2)                                            // :131-133
        for (int i = 0; i < n; ++i) o.rho[i] = o.rho[i] + o.drhodt[i] * dt;
    mass_evolution(o);
    sound_speed(o);
    smoothing_length(o);
    time_step(o);
}

// leapfrog_scheme, time_integration.f90:289-391.
void leapfrog_scheme(Orc &o) {
    const int n = o.ntotal;
    const double dt = o.dt;
    std::vector<double> x1(o.x.begin(), o.x.begin() + 2 * n), vx1(o.vx.begin(), o.vx.begin() + 2 * n);
    std::vector<double> h1(o.h.begin(), o.h.begin() + n), A1(o.A.begin(), o.A.begin() + n);
    std::vector<double> rho1(o.rho.begin(), o.rho.begin() + n);
    single_step(o);                                                  // :330
    for (int k = 0; k < 2 * n; ++k) {
        o.x[k] = o.x[k] + o.dxdt[k] * dt / 2;
        o.vx[k] = o.vx[k] + o.dvxdt[k] * dt / 2;
    }
    for (int i = 0; i < n; ++i) {
        o.h[i] = o.h[i] + o.dhdt[i] * dt / 2;
        o.A[i] = o.A[i] + o.dAdt[i] * dt / 2;
    }
    clamp_A(o);
    density(o);
    if (o.P.den_alg == 2)                                            // :347-349
        for (int i = 0; i < n; ++i) o.rho[i] = o.rho[i] + o.drhodt[i] * dt / 2;
    mass_evolution(o);
    sound_speed(o);
    single_step(o);                                                  // :358
    for (int k = 0; k < 2 * n; ++k) {
        o.vx[k] = vx1[k] + o.dvxdt[k] * dt;
        o.x[k] = x1[k] + (vx1[k] + o.dxdt[k]) * dt / 2;
    }
    for (int i = 0; i < n; ++i) {
        o.h[i] = h1[i] + o.dhdt[i] * dt;
        o.A[i] = A1[i] + o.dAdt[i] * dt;
    }
    clamp_A(o);
    density(o);
    if (o.P.den_alg == 2)                                            // :375-377
        for (int i = 0; i < n; ++i) o.rho[i] = rho1[i] + o.drhodt[i] * dt;
    mass_evolution(o);
    sound_speed(o);
    smoothing_length(o);
    time_step(o);
}

int fail(Orc *o, int code, const char *msg) { o->err = msg; return code; }

bool normals_ok(const Orc &o) {
    return !(o.P.bfa == 2 && o.P.boundary_pressure && o.ntotalb > 0 &&
             o.b_normal.size() != 2 * (size_t)o.ntotalb);
}

}  // namespace

extern "C" {

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void *orc_create(const simp_params *P, int maxn, int maxnb) {
    Orc *o = new Orc();
    o->P = *P;
    o->maxn = maxn; o->maxnb = maxnb;
    o->scale_h = scale_h_of(P->skf);   // initialize.f90:208-217
    return o;
}

void orc_destroy(void *h) { delete (Orc *)h; }

const char *orc_last_error(void *h) { return ((Orc *)h)->err.c_str(); }

int orc_set_state(void *hh, int n, const double *x, const double *vx, const double *mass,
                  const double *rho, const double *hsml, const double *A, const double *h,
                  int nb, const double *xb, const double *massb, double dt, double t) {
    Orc *o = (Orc *)hh;
    if (n > o->maxn) return fail(o, SIMP_ERR_MAXN, "Resolution desired too high, the number of particles generated is higher than the maximum allowed.");
    if (nb > o->maxnb) return fail(o, SIMP_ERR_MAXN, "The number of boundary particles generated is higher than the maximum allowed.");
    o->ntotal = n; o->ntotalb = nb;
    o->x.assign(x, x + 2 * (size_t)n); o->vx.assign(vx, vx + 2 * (size_t)n);
    o->mass.assign(mass, mass + n); o->rho.assign(rho, rho + n); o->hsml.assign(hsml, hsml + n);
    o->A.assign(A, A + n); o->h.assign(h, h + n);
    o->xb.assign(xb, xb + 2 * (size_t)nb); o->massb.assign(massb, massb + nb);
    o->p.assign(n, 0.0); o->c.assign(n, 0.0);
    o->dvxdt.assign(2 * (size_t)n, 0.0); o->dxdt.assign(2 * (size_t)n, 0.0);
    o->dAdt.assign(n, 0.0); o->dhdt.assign(n, 0.0); o->drhodt.assign(n, 0.0);
    o->kernel_zero.assign(n, 0.0);
    o->b_normal.clear();
    for (auto *v : {&o->eps11, &o->eps12, &o->eps22, &o->zeta, &o->eta, &o->sig11, &o->sig12, &o->sig22})
        v->assign(n, 0.0);
    o->dt = dt; o->current_time = t;
    double mh = 0.0;
    for (int i = 0; i < n; ++i) mh = std::max(mh, hsml[i]);
    o->max_hsml = (o->P.max_hsml > 0.0) ? o->P.max_hsml : mh * 10.0;  // initialize.f90:191
    o->nip = o->bnip = 0;
    sound_speed(*o);                                                   // initialize.f90:200
    return 0;
}

// Form of the regularisation pair loops: 0 per pair (the library's), 1 the
// reference's serial loops literally.
int orc_set_regularization_form(void *hh, int literal) {
    ((Orc *)hh)->reg_literal = literal ? 1 : 0;
    return 0;
}

// b_normal(2, nb) of the walls (boundaries.f90:232-287), read by bf_Wang.
int orc_set_wall_normals(void *hh, int nb, const double *bn) {
    Orc *o = (Orc *)hh;
    if (nb != o->ntotalb) return fail(o, SIMP_ERR_BADARG, "set_wall_normals: ntotalb differs from the state's walls");
    o->b_normal.assign(bn, bn + 2 * (size_t)nb);
    return 0;
}



int orc_get_state(void *hh, double *x, double *vx, double *mass, double *rho, double *hsml,
                  double *A, double *h, double *dt, double *t) {
    Orc *o = (Orc *)hh;
    const int n = o->ntotal;
    if (x) std::copy(o->x.begin(), o->x.begin() + 2 * n, x);
    if (vx) std::copy(o->vx.begin(), o->vx.begin() + 2 * n, vx);
    if (mass) std::copy(o->mass.begin(), o->mass.begin() + n, mass);
    if (rho) std::copy(o->rho.begin(), o->rho.begin() + n, rho);
    if (hsml) std::copy(o->hsml.begin(), o->hsml.begin() + n, hsml);
    if (A) std::copy(o->A.begin(), o->A.begin() + n, A);
    if (h) std::copy(o->h.begin(), o->h.begin() + n, h);
    if (dt) *dt = o->dt;
    if (t) *t = o->current_time;
    return 0;
}

// Runs NNPS on the current state and copies the pair lists out in the
// oracle's own order (one thread: the reference's serial order).
int orc_nnps(void *hh, int *nip, int *p_i, int *p_j, double *r_ij, double *hsml_ij, int cap,
             int *bnip, int *bp_i, int *bp_j, double *br_ij, int bcap) {
    Orc *o = (Orc *)hh;
    nnps(*o);
    if (nip) *nip = o->nip;
    if (bnip) *bnip = o->bnip;
    const int m = std::min(o->nip, cap), mb = std::min(o->bnip, bcap);
    for (int k = 0; k < m; ++k) {
        if (p_i) p_i[k] = o->p_i[k];
        if (p_j) p_j[k] = o->p_j[k];
        if (r_ij) r_ij[k] = o->r_ij[k];
        if (hsml_ij) hsml_ij[k] = o->hsml_ij[k];
    }
    for (int k = 0; k < mb; ++k) {
        if (bp_i) bp_i[k] = o->bp_i[k];
        if (bp_j) bp_j[k] = o->bp_j[k];
        if (br_ij) br_ij[k] = o->br_ij[k];
    }
    if (o->nip > cap || o->bnip > bcap) return fail(o, SIMP_ERR_PAIR_CAP, "Too much particle interaction please allocate more memory for arrays in globals module.");
    return 0;
}

int orc_interaction_stats(void *hh, int *maxip, int *minip, long long *sumip, int *noip) {
    Orc *o = (Orc *)hh;
    int mx = 0, mn = 0, no = 0; long long s = 0;
    for (int i = 0; i < o->ntotal; ++i) {
        const int c = o->count_np[i];
        mx = (i == 0) ? c : std::max(mx, c);
        mn = (i == 0) ? c : std::min(mn, c);
        s += c; no += (c == 0);
    }
    *maxip = mx; *minip = mn; *sumip = s; *noip = no;
    return 0;
}

int orc_single_step(void *hh, double t, double *dxdt, double *dvxdt, double *dhdt, double *dAdt) {
    Orc *o = (Orc *)hh;
    if (!normals_ok(*o)) return fail(o, SIMP_ERR_STATE, "bfa = 2 needs the wall normals");
    o->current_time = t;
    single_step(*o);
    const int n = o->ntotal;
    if (dxdt) std::copy(o->dxdt.begin(), o->dxdt.begin() + 2 * n, dxdt);
    if (dvxdt) std::copy(o->dvxdt.begin(), o->dvxdt.begin() + 2 * n, dvxdt);
    if (dhdt) std::copy(o->dhdt.begin(), o->dhdt.begin() + n, dhdt);
    if (dAdt) std::copy(o->dAdt.begin(), o->dAdt.begin() + n, dAdt);
    return 0;
}

int orc_get_diag(void *hh, double *e11, double *e12, double *e22, double *zeta, double *eta,
                 double *p, double *s11, double *s12, double *s22) {
    Orc *o = (Orc *)hh;
    const int n = o->ntotal;
    auto cp = [n](const std::vector<double> &v, double *d) { if (d) std::copy(v.begin(), v.begin() + n, d); };
    cp(o->eps11, e11); cp(o->eps12, e12); cp(o->eps22, e22); cp(o->zeta, zeta); cp(o->eta, eta);
    cp(o->p, p); cp(o->sig11, s11); cp(o->sig12, s12); cp(o->sig22, s22);
    return 0;
}

// Runs one NNPS + kinematic pass (to fill w and kernel_zero, as after a
// single_step) and then the density pair sum.
int orc_sum_density(void *hh, int k0_mode, double *rho_out) {
    Orc *o = (Orc *)hh;
    const double t = o->current_time;
    std::vector<double> saved_rho(o->rho);
    single_step(*o);
    o->current_time = t;
    sum_density(*o, k0_mode, rho_out);
    o->rho = saved_rho;
    return 0;
}

// time_integration.f90:38-71 for nsteps iterations.
int orc_step(void *hh, int nsteps, double *t, double *dt) {
    Orc *o = (Orc *)hh;
    if (!normals_ok(*o)) return fail(o, SIMP_ERR_STATE, "bfa = 2 needs the wall normals");
    for (int s = 0; s < nsteps && !o->bad; ++s) {
        if (o->P.int_algorithm == 1) euler_scheme(*o);              // time_integration.f90:47-55
        else if (o->P.int_algorithm == 3) leapfrog_scheme(*o);
        else predictor_corrector(*o);
        o->itimestep += 1;
        o->current_time = o->current_time + o->dt;
    }
    if (o->bad) return fail(o, SIMP_ERR_NONFINITE, "state blew up: no bucket grid can be built");
    if (t) *t = o->current_time;
    if (dt) *dt = o->dt;
    for (int i = 0; i < 2 * o->ntotal; ++i)
        if (!std::isfinite(o->x[i]) || !std::isfinite(o->vx[i]))
            return fail(o, SIMP_ERR_NONFINITE, "non-finite particle state after step");
    return 0;
}

// Single pair-kernel evaluation for known-answer tests.
int orc_kernel(const simp_params *P, double r, double hij, double dx, double dy,
               double *w, double *dwx, double *dwy, double *k0) {
    Orc o; o.P = *P; o.scale_h = scale_h_of(P->skf);
    const double d[2] = {dx, dy};
    double dw[2];
    pair_kernel(o, r, hij, d, w, dw, k0);
    *dwx = dw[0]; *dwy = dw[1];
    return 0;
}

double orc_boundary_w(const simp_params *P, double br) {
    Orc o; o.P = *P; o.scale_h = scale_h_of(P->skf);
    o.hsml_ij.assign(1, P->b_length);
    return boundary_w(o, br, 1);
}

// factor * dW/dq of the boundary kernel at distance br (hsml_ij = b_length
// for the Wendland C6 factor, as orc_boundary_w).
double orc_boundary_fdwdq(const simp_params *P, double br) {
    Orc o; o.P = *P; o.scale_h = scale_h_of(P->skf);
    o.hsml_ij.assign(1, P->b_length);
    return boundary_fdwdq(o, br, 1);
}

}  // extern "C"
