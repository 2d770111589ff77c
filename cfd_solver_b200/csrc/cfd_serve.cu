// cfd_serve.cu -- continuous-batching request loop over the batch slots (host code only).
//
// A serving session owns one batch whose slots have fixed geometry classes (n0 x n1,
// profile). Requests arrive over time; each waits in its class's FIFO until a slot of
// that class is free, is admitted (grid, state and set-up written into the slot while
// the other slots stay resident), is stepped together with every other active slot by
// the same launches (the step graph), and is retired -- its slot back-filled -- once its
// steady residual falls below the request's tolerance, it hits its step cap, or it
// diverges. Latency = retirement time - arrival time.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cfd_b200.h"

void cfd_internal_set_error(const char* msg);

namespace {
double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

extern "C" int cfd_serve(const cfd_serve_config* cfg, const cfd_request* reqs, int nreq, cfd_result* results,
                         cfd_serve_stats* stats) {
    if (!cfg || !reqs || nreq < 0 || !results || cfg->nclasses <= 0 || !cfg->class_grids || !cfg->class_profile) {
        cfd_internal_set_error("cfd_serve: bad arguments");
        return CFD_E_ARG;
    }
    const int nc = cfg->nclasses;
    // slots per class: given, or an equal share of the HBM budget
    std::vector<int> nslots(nc);
    for (int k = 0; k < nc; k++) {
        if (cfg->class_slots) {
            nslots[k] = cfg->class_slots[k];
            if (nslots[k] <= 0) {
                cfd_internal_set_error("cfd_serve: class_slots must be > 0");
                return CFD_E_ARG;
            }
        } else {
            const size_t per = cfd_case_bytes(cfg->class_grids[k].n0, cfg->class_grids[k].n1, cfg->class_profile[k]);
            nslots[k] = per ? (int)std::min<size_t>(4096, (cfg->hbm_budget / nc) / per) : 0;
        }
        if (nslots[k] <= 0) {
            cfd_internal_set_error("cfd_serve: a slot class gets no slot within the budget");
            return CFD_E_OOM;
        }
    }
    auto class_of = [&](const cfd_request& r) {
        for (int k = 0; k < nc; k++)
            if (r.grid->n0 == cfg->class_grids[k].n0 && r.grid->n1 == cfg->class_grids[k].n1 &&
                r.params.profile == cfg->class_profile[k])
                return k;
        return -1;
    };
    // every request names a grid of one of the slot classes, at the slots' precision; checked
    // before any device work, so a bad request costs no batch
    for (int i = 0; i < nreq; i++) {
        const char* why = nullptr;
        if (!reqs[i].grid)
            why = "has no grid";
        else if (class_of(reqs[i]) < 0)
            why = "matches no slot class";
        else if (reqs[i].params.precision != cfg->precision)
            why = "has another precision than the slots";
        if (why) {
            cfd_internal_set_error(("cfd_serve: request " + std::to_string(i) + " " + why).c_str());
            return CFD_E_ARG;
        }
    }
    std::vector<cfd_grid> tg;
    std::vector<cfd_params> tp;
    std::vector<int> slot_class;
    for (int k = 0; k < nc; k++)
        for (int s = 0; s < nslots[k]; s++) {
            tg.push_back(cfg->class_grids[k]);
            cfd_params p;
            cfd_params_default(&p);
            p.profile = cfg->class_profile[k];
            p.precision = cfg->precision;
            tp.push_back(p);
            slot_class.push_back(k);
        }
    const int nslot = (int)tg.size();
    cfd_batch* b = nullptr;
    int rc = cfd_batch_create(nslot, tg.data(), tp.data(), &b);
    if (rc) return rc;
    for (int s = 0; s < nslot && !rc; s++) rc = cfd_batch_set_active(b, s, 0);
    if (rc) {
        cfd_batch_destroy(b);
        return rc;
    }
    std::vector<int> order(nreq);
    for (int i = 0; i < nreq; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return reqs[a].arrival_s < reqs[c].arrival_s; });
    for (int i = 0; i < nreq; i++) {
        results[i] = cfd_result{};
        results[i].status = CFD_E_NOTCONV;
        results[i].slot = -1;
        results[i].arrival_s = reqs[i].arrival_s;
    }
    std::vector<std::deque<int>> queue(nc);
    std::vector<int> occupant(nslot, -1);
    std::vector<cfd_step_stats> st(nslot);
    const int tick = std::max(1, cfg->steps_per_tick);
    long long steps = 0, cell_updates = 0;
    int next = 0, done = 0, active = 0;
    const auto t0 = std::chrono::steady_clock::now();
    while (done < nreq) {
        const double t = now_s(t0);
        while (next < nreq && reqs[order[next]].arrival_s <= t) {
            queue[class_of(reqs[order[next]])].push_back(order[next]);
            next++;
        }
        // back-fill free slots from the queues
        for (int s = 0; s < nslot; s++) {
            if (occupant[s] >= 0 || queue[slot_class[s]].empty()) continue;
            const int r = queue[slot_class[s]].front();
            queue[slot_class[s]].pop_front();
            rc = cfd_batch_admit(b, s, reqs[r].grid, &reqs[r].params);
            if (rc) {
                cfd_batch_destroy(b);
                return rc;
            }
            occupant[s] = r;
            results[r].slot = s;
            results[r].admit_s = now_s(t0);
            active++;
        }
        if (active == 0) {
            if (next < nreq) {
                const double wait = reqs[order[next]].arrival_s - now_s(t0);
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
            }
            continue;
        }
        rc = cfd_batch_step(b, tick);
        if (!rc) rc = cfd_batch_fetch_stats(b, st.data(), nslot);
        if (rc) {
            cfd_batch_destroy(b);
            return rc;
        }
        steps += tick;
        for (int s = 0; s < nslot; s++) {
            const int r = occupant[s];
            if (r < 0) continue;
            cell_updates += (long long)tick * tg[s].n0 * tg[s].n1;
            const cfd_step_stats& x = st[s];
            const bool nan = (x.status & 4) != 0 || !(x.steady_res_rel == x.steady_res_rel);
            const bool conv = x.steps >= 2 && x.steady_res_rel <= reqs[r].tol;
            if (!(nan || conv || x.steps >= reqs[r].max_steps)) continue;
            cfd_result& o = results[r];
            o.status = nan ? CFD_E_DIVERGED : conv ? CFD_OK : CFD_E_NOTCONV;
            o.steps = x.steps;
            o.done_s = now_s(t0);
            o.latency_s = o.done_s - reqs[r].arrival_s;
            o.nu = x.nu;
            o.steady_res_rel = x.steady_res_rel;
            o.mass_res_rel = x.mass_res_rel;
            rc = cfd_batch_set_active(b, s, 0);
            if (rc) {
                cfd_batch_destroy(b);
                return rc;
            }
            occupant[s] = -1;
            active--;
            done++;
        }
    }
    const double makespan = now_s(t0);
    cfd_batch_destroy(b);
    if (stats) {
        std::vector<double> lat;
        int conv = 0;
        double sum = 0.0;
        for (int i = 0; i < nreq; i++) {
            lat.push_back(results[i].latency_s);
            sum += results[i].latency_s;
            conv += results[i].status == CFD_OK;
        }
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double q) {
            if (lat.empty()) return 0.0;
            const size_t k = (size_t)std::min<double>(lat.size() - 1, std::ceil(q * lat.size()) - 1);
            return lat[k];
        };
        *stats = cfd_serve_stats{};
        stats->makespan_s = makespan;
        stats->cases_per_s = makespan > 0 ? conv / makespan : 0.0;
        stats->p50_latency_s = pct(0.50);
        stats->p99_latency_s = pct(0.99);
        stats->mean_latency_s = nreq ? sum / nreq : 0.0;
        stats->steps = steps;
        stats->cell_updates = cell_updates;
        stats->converged = conv;
        stats->failed = nreq - conv;
        stats->slots = nslot;
    }
    return CFD_OK;
}
