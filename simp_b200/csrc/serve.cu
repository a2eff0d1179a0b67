// Served request stream (include/simp_serve.h): continuous batching of
// basins over one batch context, admission by a device-memory budget, FP64
// spot-check replicas in a second batch context on its own stream.  Host
// code only; every step goes through the batch driver of abi.cu.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ctx.h"
#include "../../include/simp_serve.h"

namespace {

// Wall capacity of a batch = particles / 4; bytes per wall slot.
constexpr int kWallsPerParticleDiv = 4;
constexpr double kBytesPerWall = 48.0;
constexpr int kSpotSlots = 64;            // FP64 replicas resident at once

struct Request {
    simp_forcing f{};
    int n = 0, nb = 0;
    const double *x = nullptr, *vx = nullptr, *mass = nullptr, *rho = nullptr, *hsml = nullptr,
                 *A = nullptr, *h = nullptr, *xb = nullptr, *massb = nullptr;
    double *x_out = nullptr, *vx_out = nullptr, *h_out = nullptr, *A_out = nullptr;
    int64_t nsteps = 0;
    double arrival = 0.0;
    // progress
    enum { PENDING, RESIDENT, DONE, FAILED, CANCELLED } state = PENDING;
    int slot = -1, spot_slot = -1;
    int64_t remaining = 0;
    simp_request_stats st{};
};

}  // namespace

struct simp_server {
    simp_params prm{};
    simp_server_config cfg{};
    simp_ctx *main = nullptr;
    simp_ctx *spot = nullptr;       // FP64 replicas
    int maxn_main = 0, maxn_spot = 0, maxnb_main = 0, maxnb_spot = 0;
    long long res_main = 0, res_spot = 0, resb_main = 0, resb_spot = 0;
    int spot_count = 0;
    std::vector<Request> reqs;
    std::vector<int> order;         // request ids by arrival
    size_t next = 0;                // next pending in `order`
    std::vector<int> resident;      // request ids on the device
    simp_server_stats stats{};
    std::string err;
    // cancellations asked for (request id, run time), possibly from another
    // thread while run() steps; applied at the scheduling decisions
    std::mutex cancel_mu;
    std::vector<std::pair<int64_t, double>> cancels;
};

namespace {

int fail(simp_server *s, int code, const std::string &msg) {
    s->err = msg;
    return code;
}

double rel_l2(const std::vector<double> &a, const std::vector<double> &b) {
    double num = 0.0, den = 0.0;
    for (size_t k = 0; k < a.size(); ++k) {
        const double d = a[k] - b[k];
        num += d * d;
        den += b[k] * b[k];
    }
    return den > 0.0 ? std::sqrt(num / den) : std::sqrt(num);
}

using clock_t_ = std::chrono::steady_clock;

int ctx_error(simp_server *s, simp_ctx *c, int rc) {
    return fail(s, rc, std::string("batch: ") + simp_gpu_last_error(c));
}

// Admits the arrived requests in arrival order while slots and budget last
// (strict first-come-first-served: a large request at the head waits for
// room rather than being overtaken).
int admit(simp_server *s, double now) {
    while (s->next < s->order.size()) {
        Request &r = s->reqs[s->order[s->next]];
        if (r.state == Request::CANCELLED) {   // cancelled before it was admitted
            s->next += 1;
            continue;
        }
        if (r.arrival > now) break;
        if ((int)s->resident.size() >= s->cfg.max_instances) break;
        if (s->res_main + r.n > s->maxn_main || s->resb_main + r.nb > s->maxnb_main) {
            if (s->resident.empty())   // could never fit
                return fail(s, SIMP_ERR_MAXN, "a request exceeds the served batch's capacity");
            break;
        }
        int32_t slot = -1;
        int rc = simp_gpu_batch_add(s->main, &r.f, r.n, r.x, r.vx, r.mass, r.rho, r.hsml, r.A, r.h, r.nb,
                                    r.xb, r.massb, &slot);
        if (rc != SIMP_OK) return ctx_error(s, s->main, rc);
        r.slot = slot;
        s->res_main += r.n;
        s->resb_main += r.nb;
        const int id = s->order[s->next];
        if (s->spot && s->cfg.spot_every > 0 && id % s->cfg.spot_every == 0 && s->spot_count < kSpotSlots &&
            s->res_spot + r.n <= s->maxn_spot && s->resb_spot + r.nb <= s->maxnb_spot) {
            rc = simp_gpu_batch_add(s->spot, &r.f, r.n, r.x, r.vx, r.mass, r.rho, r.hsml, r.A, r.h, r.nb,
                                    r.xb, r.massb, &slot);
            if (rc != SIMP_OK) return ctx_error(s, s->spot, rc);
            r.spot_slot = slot;
            s->spot_count += 1;
            s->res_spot += r.n;
            s->resb_spot += r.nb;
        }
        r.state = Request::RESIDENT;
        r.remaining = r.nsteps;
        s->resident.push_back(id);
        s->next += 1;
    }
    long long rp = 0;
    for (int id : s->resident) rp += s->reqs[id].n;
    s->stats.peak_resident_particles = std::max<int64_t>(s->stats.peak_resident_particles, rp);
    s->stats.peak_resident_requests = std::max<int32_t>(s->stats.peak_resident_requests, (int32_t)s->resident.size());
    return SIMP_OK;
}

// A finished request: results to the caller, the FP64 comparison, and its
// slots freed.
int retire(simp_server *s, int id) {
    Request &r = s->reqs[id];
    const size_t n = (size_t)r.n;
    std::vector<double> v(2 * n), hh(n);
    int rc = simp::batch_slot_state(s->main, r.slot, r.x_out, v.data(), nullptr, nullptr, nullptr, r.A_out,
                                    hh.data(), nullptr);
    if (rc != SIMP_OK) return ctx_error(s, s->main, rc);
    if (r.vx_out) std::memcpy(r.vx_out, v.data(), sizeof(double) * 2 * n);
    if (r.h_out) std::memcpy(r.h_out, hh.data(), sizeof(double) * n);
    if (r.spot_slot >= 0) {
        std::vector<double> v64(2 * n), h64(n);
        rc = simp::batch_slot_state(s->spot, r.spot_slot, nullptr, v64.data(), nullptr, nullptr, nullptr,
                                    nullptr, h64.data(), nullptr);
        if (rc != SIMP_OK) return ctx_error(s, s->spot, rc);
        r.st.spot_checked = 1;
        r.st.err_v = rel_l2(v, v64);
        r.st.err_h = rel_l2(hh, h64);
        rc = simp_gpu_batch_remove(s->spot, r.spot_slot);
        if (rc != SIMP_OK) return ctx_error(s, s->spot, rc);
        s->spot_count -= 1;
        s->res_spot -= r.n;
        s->resb_spot -= r.nb;
    }
    int32_t flags = 0;
    int64_t steps = 0;
    simp_gpu_batch_info(s->main, r.slot, nullptr, &steps, &flags);
    rc = simp_gpu_batch_remove(s->main, r.slot);
    if (rc != SIMP_OK) return ctx_error(s, s->main, rc);
    s->res_main -= r.n;
    s->resb_main -= r.nb;
    r.st.steps = steps;
    r.st.status = (flags & simp::FLAG_NONFINITE) ? SIMP_ERR_NONFINITE : SIMP_OK;
    r.state = (r.st.status == SIMP_OK) ? Request::DONE : Request::FAILED;
    if (r.state == Request::DONE) {
        s->stats.completed += 1;
        s->stats.particle_steps += (int64_t)r.n * steps;
    } else {
        s->stats.failed += 1;
    }
    return SIMP_OK;
}

// Cancellations that are due at `now`: a pending request is marked (admit
// skips it), a resident one leaves both batches between steps.
int apply_cancels(simp_server *s, double now) {
    std::vector<int64_t> due;
    {
        std::lock_guard<std::mutex> lk(s->cancel_mu);
        std::vector<std::pair<int64_t, double>> later;
        for (const auto &c : s->cancels) {
            if (c.second <= now) due.push_back(c.first);
            else later.push_back(c);
        }
        s->cancels.swap(later);
    }
    for (int64_t id : due) {
        Request &r = s->reqs[(size_t)id];
        if (r.state == Request::PENDING) {
            r.state = Request::CANCELLED;
        } else if (r.state == Request::RESIDENT) {
            if (r.spot_slot >= 0) {
                const int rc = simp_gpu_batch_remove(s->spot, r.spot_slot);
                if (rc != SIMP_OK) return ctx_error(s, s->spot, rc);
                s->spot_count -= 1;
                s->res_spot -= r.n;
                s->resb_spot -= r.nb;
                r.spot_slot = -1;
            }
            int64_t steps = 0;
            simp_gpu_batch_info(s->main, r.slot, nullptr, &steps, nullptr);
            const int rc = simp_gpu_batch_remove(s->main, r.slot);
            if (rc != SIMP_OK) return ctx_error(s, s->main, rc);
            s->res_main -= r.n;
            s->resb_main -= r.nb;
            r.st.steps = steps;
            r.state = Request::CANCELLED;
            s->resident.erase(std::find(s->resident.begin(), s->resident.end(), (int)id));
        } else {
            continue;   // completed or failed already
        }
        r.st.status = SIMP_ERR_CANCELLED;
        r.st.completed_s = now;
        s->stats.cancelled += 1;
    }
    return SIMP_OK;
}

}  // namespace

extern "C" {

int32_t simp_server_create(const simp_params *params, const simp_server_config *cfg, simp_server **out) {
    if (!out) return SIMP_ERR_BADARG;
    *out = nullptr;
    if (!params || !cfg || cfg->max_instances < 1 || cfg->max_instances > simp::kMaxSlots ||
        cfg->max_request_particles < 1 || cfg->quantum_steps < 1 || cfg->spot_every < 0 ||
        !(cfg->hbm_budget_bytes > 0.0))
        return SIMP_ERR_BADARG;
    simp_server *s = new simp_server();
    *out = s;
    s->prm = *params;
    s->cfg = *cfg;
    const double per = simp::bytes_per_particle(s->prm, cfg->max_instances == 1) + kBytesPerWall / kWallsPerParticleDiv;
    double budget = cfg->hbm_budget_bytes;
    if (cfg->spot_every > 0) {
        simp_params p64 = s->prm;
        p64.precision = SIMP_PREC_FP64;
        const double spot_n = 2.0 * cfg->max_request_particles;
        s->maxn_spot = (int)spot_n;
        s->maxnb_spot = std::max(1, s->maxn_spot / kWallsPerParticleDiv);
        // (a batch of one slot is a single-basin context, with its read-back stage)
        const bool single = std::min(cfg->max_instances, kSpotSlots) == 1;
        budget -= spot_n * (simp::bytes_per_particle(p64, single) + kBytesPerWall / kWallsPerParticleDiv);
    }
    const double cap = std::floor(budget / per);
    if (cap < cfg->max_request_particles)
        return fail(s, SIMP_ERR_NOMEM, "the budget does not hold the largest request");
    s->maxn_main = (int)std::min(cap, 2.0e9);
    s->maxnb_main = std::max(1, s->maxn_main / kWallsPerParticleDiv);
    s->stats.capacity_particles = (double)s->maxn_main;
    int rc = simp_gpu_create_batch(&s->prm, s->maxn_main, s->maxnb_main, cfg->max_instances, &s->main);
    if (rc != SIMP_OK) return fail(s, rc, s->main ? simp_gpu_last_error(s->main) : "create_batch failed");
    if (cfg->spot_every > 0) {
        simp_params p64 = s->prm;
        p64.precision = SIMP_PREC_FP64;
        rc = simp_gpu_create_batch(&p64, s->maxn_spot, s->maxnb_spot, std::min(cfg->max_instances, kSpotSlots), &s->spot);
        if (rc != SIMP_OK) return fail(s, rc, s->spot ? simp_gpu_last_error(s->spot) : "create_batch failed");
    }
    return SIMP_OK;
}

int32_t simp_server_destroy(simp_server *s) {
    if (!s) return SIMP_OK;
    if (s->main) simp_gpu_destroy(s->main);
    if (s->spot) simp_gpu_destroy(s->spot);
    delete s;
    return SIMP_OK;
}

int32_t simp_server_submit(simp_server *s, const simp_forcing *forcing, int32_t ntotal, const double *x,
                           const double *vx, const double *mass, const double *rho, const double *hsml,
                           const double *A, const double *h, int32_t ntotalb, const double *xb,
                           const double *massb, int64_t nsteps, double arrival_s, double *x_out,
                           double *vx_out, double *h_out, double *A_out, int64_t *request_id) {
    if (!s || !forcing || !request_id) return SIMP_ERR_BADARG;
    if (ntotal < 1 || ntotalb < 0 || nsteps < 0 || !(arrival_s >= 0.0) || !x || !vx || !mass || !rho ||
        !hsml || !A || !h || (ntotalb > 0 && (!xb || !massb)))
        return fail(s, SIMP_ERR_BADARG, "submit: bad sizes or null arrays");
    if (ntotal > s->cfg.max_request_particles)
        return fail(s, SIMP_ERR_MAXN, "submit: request larger than max_request_particles");
    Request r;
    r.f = *forcing;
    r.n = ntotal;
    r.nb = ntotalb;
    r.x = x; r.vx = vx; r.mass = mass; r.rho = rho; r.hsml = hsml; r.A = A; r.h = h;
    r.xb = xb; r.massb = massb;
    r.x_out = x_out; r.vx_out = vx_out; r.h_out = h_out; r.A_out = A_out;
    r.nsteps = nsteps;
    r.arrival = arrival_s;
    r.st.arrival_s = arrival_s;
    r.st.ntotal = ntotal;
    r.st.admitted_s = r.st.completed_s = -1.0;
    r.st.err_v = r.st.err_h = -1.0;
    *request_id = (int64_t)s->reqs.size();
    s->reqs.push_back(r);
    s->stats.submitted += 1;
    return SIMP_OK;
}

int32_t simp_server_run(simp_server *s) {
    if (!s || !s->main) return SIMP_ERR_BADARG;
    s->order.clear();
    for (size_t k = 0; k < s->reqs.size(); ++k)
        if (s->reqs[k].state == Request::PENDING) s->order.push_back((int)k);
    std::stable_sort(s->order.begin(), s->order.end(),
                     [&](int a, int b) { return s->reqs[a].arrival < s->reqs[b].arrival; });
    s->next = 0;
    const auto t0 = clock_t_::now();
    auto now = [&]() { return std::chrono::duration<double>(clock_t_::now() - t0).count(); };
    for (;;) {
        const double t = now();
        int rc = apply_cancels(s, t);
        if (rc != SIMP_OK) return rc;
        const size_t before = s->resident.size();
        rc = admit(s, t);
        if (rc != SIMP_OK) return rc;
        s->stats.admit_s += now() - t;
        for (size_t k = before; k < s->resident.size(); ++k) s->reqs[s->resident[k]].st.admitted_s = now();
        if (s->resident.empty()) {
            if (s->next >= s->order.size()) break;   // all done
            const double wait = s->reqs[s->order[s->next]].arrival - now();
            if (wait > 0.0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
            continue;
        }
        // requests with no steps left leave at once
        int64_t q = s->cfg.quantum_steps;
        for (int id : s->resident) q = std::min<int64_t>(q, s->reqs[id].remaining);
        const double ts = now();
        if (q > 0) {
            rc = simp::step_enqueue(s->main, (int)q);
            if (rc != SIMP_OK) return ctx_error(s, s->main, rc);
            const bool spot_busy = s->spot && s->res_spot > 0;
            if (spot_busy) {
                rc = simp::step_enqueue(s->spot, (int)q);
                if (rc != SIMP_OK) return ctx_error(s, s->spot, rc);
            }
            rc = simp::step_complete(s->main, nullptr, nullptr);
            if (rc != SIMP_OK) return ctx_error(s, s->main, rc);
            if (spot_busy) {
                rc = simp::step_complete(s->spot, nullptr, nullptr);
                if (rc != SIMP_OK) return ctx_error(s, s->spot, rc);
            }
            s->stats.batch_steps += q;
        }
        const double tr = now();
        s->stats.step_s += tr - ts;
        std::vector<int> keep;
        for (int id : s->resident) {
            Request &r = s->reqs[id];
            r.remaining -= q;
            if (r.remaining <= 0) {
                rc = retire(s, id);
                if (rc != SIMP_OK) return rc;
                r.st.completed_s = now();   // its results are on the host
                s->stats.makespan_s = std::max(s->stats.makespan_s, r.st.completed_s);
            } else {
                keep.push_back(id);
            }
        }
        s->resident.swap(keep);
        s->stats.retire_s += now() - tr;
    }
    return SIMP_OK;
}

int32_t simp_server_cancel(simp_server *s, int64_t id, double at_s) {
    if (!s || id < 0) return SIMP_ERR_BADARG;
    std::lock_guard<std::mutex> lk(s->cancel_mu);
    if (id >= (int64_t)s->reqs.size()) return fail(s, SIMP_ERR_BADARG, "cancel: unknown request");
    s->cancels.emplace_back(id, at_s < 0.0 ? -1.0 : at_s);
    return SIMP_OK;
}

int32_t simp_server_request(const simp_server *s, int64_t id, simp_request_stats *out) {
    if (!s || !out || id < 0 || id >= (int64_t)s->reqs.size()) return SIMP_ERR_BADARG;
    *out = s->reqs[id].st;
    return SIMP_OK;
}

int32_t simp_server_stats_get(const simp_server *s, simp_server_stats *out) {
    if (!s || !out) return SIMP_ERR_BADARG;
    *out = s->stats;
    return SIMP_OK;
}

const char *simp_server_last_error(const simp_server *s) { return s ? s->err.c_str() : "null server"; }

}  // extern "C"
