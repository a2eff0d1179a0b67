/*
 * Drives the C ABI the way SIMP's Fortran host would: module-global style
 * arrays in the reference's layout (x(2,n) interleaved, 1-based pair
 * indices), status codes checked after every call.  Exit code 0 = all checks
 * passed.  Built and run by tests/test_c_driver.py on a GPU machine.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "simp_gpu.h"

#define CHECK(call)                                                              \
    do {                                                                         \
        int32_t rc_ = (call);                                                    \
        if (rc_ != SIMP_OK) {                                                    \
            fprintf(stderr, "%s failed: %d %s\n", #call, rc_, simp_gpu_last_error(ctx)); \
            return 1;                                                            \
        }                                                                        \
    } while (0)

static double lcg(unsigned long long *s) {
    *s = *s * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(*s >> 11) / 9007199254740992.0;
}

int main(void) {
    const int side = 40, n = side * side;
    const double dx = 2000.0, L = side * dx;
    double *x = malloc(sizeof(double) * 2 * n), *vx = calloc(2 * n, sizeof(double));
    double *mass = malloc(sizeof(double) * n), *rho = malloc(sizeof(double) * n);
    double *hsml = malloc(sizeof(double) * n), *A = malloc(sizeof(double) * n), *h = malloc(sizeof(double) * n);
    unsigned long long seed = 12345;
    for (int j = 0; j < side; ++j)
        for (int i = 0; i < side; ++i) {
            const int k = j * side + i;
            x[2 * k] = (i + 0.5) * dx + (lcg(&seed) - 0.5) * 0.1 * dx;
            x[2 * k + 1] = (j + 0.5) * dx + (lcg(&seed) - 0.5) * 0.1 * dx;
            h[k] = 1.0;
            A[k] = 1.0;
            rho[k] = 900.0;
            mass[k] = 900.0 * dx * dx;
            hsml[k] = 2.4 * dx;
        }
    /* wall on +x at spacing b_length / 3 */
    const double b_length = 4.0 * dx, sp = b_length / 3.0;
    const int nb = (int)ceil((L + dx) / sp);
    double *xb = malloc(sizeof(double) * 2 * nb), *massb = malloc(sizeof(double) * nb);
    for (int b = 0; b < nb; ++b) {
        xb[2 * b] = L + 0.5 * dx;
        xb[2 * b + 1] = -0.5 * dx + (b + 0.5) * (L + dx) / nb;
        massb[b] = 900.0 * dx * dx;
    }

    simp_params p;
    simp_params_reference_default(&p);
    p.skf = SIMP_SKF_CUBIC;
    p.sle = 0;
    p.mass_from_area = 0;
    p.tse = 0;
    p.dt = 1.0;
    p.b_length = b_length;
    p.wind_u = 10.0;
    p.wind_v = 0.0;

    simp_ctx *ctx = NULL;
    CHECK(simp_gpu_create(&p, n, nb, &ctx));
    CHECK(simp_gpu_set_state(ctx, n, x, vx, mass, rho, hsml, A, h, nb, xb, massb, p.dt, 0.0));

    /* NNPS: canonical 1-based pair lists */
    const int cap = 40 * n;
    int32_t nip = 0, bnip = 0;
    int32_t *pi = malloc(sizeof(int32_t) * cap), *pj = malloc(sizeof(int32_t) * cap);
    int32_t *bpi = malloc(sizeof(int32_t) * cap), *bpj = malloc(sizeof(int32_t) * cap);
    double *r = malloc(sizeof(double) * cap), *hm = malloc(sizeof(double) * cap), *br = malloc(sizeof(double) * cap);
    CHECK(simp_gpu_nnps(ctx, &nip, pi, pj, r, hm, cap, &bnip, bpi, bpj, br, cap));
    if (nip < 8 * n || bnip < 1) { fprintf(stderr, "too few pairs %d %d\n", nip, bnip); return 1; }
    for (int k = 0; k < nip; ++k) {
        if (pi[k] < 1 || pj[k] > n || pi[k] >= pj[k]) { fprintf(stderr, "bad pair %d\n", k); return 1; }
        if (k && (pi[k] < pi[k - 1] || (pi[k] == pi[k - 1] && pj[k] <= pj[k - 1]))) {
            fprintf(stderr, "pairs not sorted at %d\n", k);
            return 1;
        }
        if (!(r[k] <= hm[k])) { fprintf(stderr, "pair beyond support %d\n", k); return 1; }
    }
    for (int k = 0; k < bnip; ++k)
        if (bpi[k] < 1 || bpi[k] > nb || bpj[k] < 1 || bpj[k] > n || !(br[k] <= b_length)) {
            fprintf(stderr, "bad wall pair %d\n", k);
            return 1;
        }
    /* capacity error keeps the true count */
    int32_t nip2 = 0, bnip2 = 0;
    if (simp_gpu_nnps(ctx, &nip2, pi, pj, r, hm, 10, &bnip2, bpi, bpj, br, cap) != SIMP_ERR_PAIR_CAP ||
        nip2 != nip) {
        fprintf(stderr, "pair capacity not reported\n");
        return 1;
    }

    /* single_step at rest: only the wall acts, away from the wall */
    double *dxdt = malloc(sizeof(double) * 2 * n), *dvxdt = malloc(sizeof(double) * 2 * n);
    double *dhdt = malloc(sizeof(double) * n), *dAdt = malloc(sizeof(double) * n);
    CHECK(simp_gpu_single_step(ctx, 0.0, dxdt, dvxdt, dhdt, dAdt));
    int pushed = 0;
    for (int k = 0; k < n; ++k) {
        if (dvxdt[2 * k] > 0.0) { fprintf(stderr, "wall pulls particle %d\n", k); return 1; }
        pushed += dvxdt[2 * k] < 0.0;
    }
    if (pushed == 0) { fprintf(stderr, "wall force missing\n"); return 1; }

    /* ten predictor-corrector steps, then read back */
    double t = 0.0, dt = 0.0;
    CHECK(simp_gpu_step(ctx, 10, &t, &dt));
    if (t != 10.0 || dt != 1.0) { fprintf(stderr, "time %g dt %g\n", t, dt); return 1; }
    CHECK(simp_gpu_get_state(ctx, x, vx, mass, rho, hsml, A, h, &dt, &t));
    double ke = 0.0;
    for (int k = 0; k < n; ++k) {
        if (!isfinite(x[2 * k]) || !isfinite(vx[2 * k]) || !(A[k] <= 1.0)) { fprintf(stderr, "bad state %d\n", k); return 1; }
        ke += vx[2 * k] * vx[2 * k] + vx[2 * k + 1] * vx[2 * k + 1];
    }
    if (!(ke > 0.0)) { fprintf(stderr, "nothing moved\n"); return 1; }

    /* a host that hands the state over every step: set_state of what
       get_state returned, a step without outputs, get_state with time and dt */
    for (int k = 0; k < 3; ++k) {
        CHECK(simp_gpu_set_state(ctx, n, x, vx, mass, rho, hsml, A, h, nb, xb, massb, dt, t));
        CHECK(simp_gpu_step(ctx, 1, NULL, NULL));
        CHECK(simp_gpu_get_state(ctx, x, vx, mass, rho, hsml, A, h, &dt, &t));
    }
    if (t != 13.0) { fprintf(stderr, "time after the host loop %g\n", t); return 1; }

    /* capacity error of set_state */
    if (simp_gpu_set_state(ctx, n + 1, x, vx, mass, rho, hsml, A, h, nb, xb, massb, 1.0, 0.0) != SIMP_ERR_MAXN) {
        fprintf(stderr, "maxn not reported\n");
        return 1;
    }
    CHECK(simp_gpu_destroy(ctx));
    printf("abi_driver ok: nip=%d bnip=%d t=%g\n", nip, bnip, t);
    return 0;
}
