// cfd_serve.cu -- continuous-batching request loop (host code only).
//
// Two forms of admission:
//  * by free device memory (cfg->class_slots == NULL): the session owns a slot pool
//    (cfd_pool_create) of cfg->hbm_budget bytes. Requests of any size wait in one
//    arrival-ordered queue; every tick each waiting request, oldest first, is placed if a
//    free region of the budget fits it (a smaller one may pass a larger one that does not
//    fit yet, until the oldest has waited kMaxPassTicks ticks: then nothing passes it, so
//    the memory retirements free goes to it). A retired case gives its memory back at once.
//  * by fixed slots (cfg->class_slots given): one batch whose slots have fixed geometry
//    classes (n0 x n1, profile); each request waits in its class's FIFO for a free slot.
// Either way an admitted case (grid, state and set-up written into its slot while the
// others stay resident) is stepped together with every other active case by the same
// launches (the step graph), and is retired once its steady residual falls below the
// request's tolerance, it hits its step cap, or it diverges. Latency = retirement time -
// arrival time.
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

constexpr int kMaxPassTicks = 20;  // ticks the oldest waiting request may be passed by smaller ones

void fill_serve_stats(const cfd_result* results, int nreq, double makespan, long long steps,
                      long long cell_updates, int nslot, cfd_serve_stats* stats) {
    if (!stats) return;
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

// retirement test of request r from its case's latest stats; fills its result when retired
bool retire_if_done(const cfd_request& q, const cfd_step_stats& x, double t, cfd_result& o) {
    const bool nan = (x.status & 4) != 0 || !(x.steady_res_rel == x.steady_res_rel);
    const bool conv = x.steps >= 2 && x.steady_res_rel <= q.tol;
    if (!(nan || conv || x.steps >= q.max_steps)) return false;
    o.status = nan ? CFD_E_DIVERGED : conv ? CFD_OK : CFD_E_NOTCONV;
    o.steps = x.steps;
    o.done_s = t;
    o.latency_s = t - q.arrival_s;
    o.nu = x.nu;
    o.steady_res_rel = x.steady_res_rel;
    o.mass_res_rel = x.mass_res_rel;
    return true;
}

// admission by free device memory over a slot pool of cfg->hbm_budget bytes
int serve_pool(const cfd_serve_config* cfg, const cfd_request* reqs, int nreq, cfd_result* results,
               cfd_serve_stats* stats) {
    size_t smallest = 0;
    for (int i = 0; i < nreq; i++) {
        const char* why = nullptr;
        int code = CFD_E_ARG;
        size_t need = 0;
        if (!reqs[i].grid)
            why = "has no grid";
        else if (reqs[i].params.precision != cfg->precision)
            why = "has another precision than the session";
        else if (!(need = cfd_pool_case_bytes(reqs[i].grid->n0, reqs[i].grid->n1, reqs[i].params.profile)))
            why = "has a grid too small";
        else if (need > cfg->hbm_budget) {
            why = "needs more device memory than the whole budget";
            code = CFD_E_OOM;
        }
        if (why) {
            cfd_internal_set_error(("cfd_serve: request " + std::to_string(i) + " " + why).c_str());
            return code;
        }
        smallest = smallest ? std::min(smallest, need) : need;
    }
    const int max_cases = (int)std::max<size_t>(1, std::min<size_t>(4096, smallest ? cfg->hbm_budget / smallest : 1));
    cfd_batch* b = nullptr;
    int rc = cfd_pool_create(cfg->hbm_budget, max_cases, cfg->precision, &b);
    if (rc) return rc;
    std::vector<int> order(nreq);
    for (int i = 0; i < nreq; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return reqs[a].arrival_s < reqs[c].arrival_s; });
    for (int i = 0; i < nreq; i++) {
        results[i] = cfd_result{};
        results[i].status = CFD_E_NOTCONV;
        results[i].slot = -1;
        results[i].arrival_s = reqs[i].arrival_s;
    }
    std::deque<int> wait;              // arrived, not yet admitted (arrival order)
    std::vector<int> occupant(max_cases, -1);
    std::vector<cfd_step_stats> st(max_cases);
    const int tick = std::max(1, cfg->steps_per_tick);
    long long steps = 0, cell_updates = 0;
    int next = 0, done = 0, active = 0, head_passed = 0;
    const auto t0 = std::chrono::steady_clock::now();
    auto finish = [&](int code) {
        cfd_batch_destroy(b);
        return code;
    };
    while (done < nreq) {
        const double t = now_s(t0);
        while (next < nreq && reqs[order[next]].arrival_s <= t) wait.push_back(order[next++]);
        // admission: oldest first; a request that does not fit is passed by later ones until
        // the oldest has been passed kMaxPassTicks times
        bool head_blocked = false;
        for (auto it = wait.begin(); it != wait.end();) {
            if (head_blocked) break;
            const int r = *it;
            int slot = -1;
            rc = cfd_pool_admit(b, reqs[r].grid, &reqs[r].params, &slot);
            if (rc == CFD_E_OOM) {
                if (it == wait.begin() && head_passed >= kMaxPassTicks) head_blocked = true;
                ++it;
                continue;
            }
            if (rc) return finish(rc);
            if (it == wait.begin()) head_passed = 0;
            occupant[slot] = r;
            results[r].slot = slot;
            results[r].admit_s = now_s(t0);
            active++;
            it = wait.erase(it);
        }
        if (!wait.empty()) head_passed++;
        if (active == 0) {
            if (!wait.empty()) {
                cfd_internal_set_error("cfd_serve: a waiting request fits no free region of an empty pool");
                return finish(CFD_E_OOM);
            }
            if (next < nreq) {
                const double w = reqs[order[next]].arrival_s - now_s(t0);
                if (w > 0) std::this_thread::sleep_for(std::chrono::duration<double>(w));
            }
            continue;
        }
        rc = cfd_batch_step(b, tick);
        if (!rc) rc = cfd_batch_fetch_stats(b, st.data(), max_cases);
        if (rc) return finish(rc);
        steps += tick;
        const double tn = now_s(t0);
        for (int s = 0; s < max_cases; s++) {
            const int r = occupant[s];
            if (r < 0) continue;
            cell_updates += (long long)tick * reqs[r].grid->n0 * reqs[r].grid->n1;
            if (!retire_if_done(reqs[r], st[s], tn, results[r])) continue;
            rc = cfd_pool_release(b, s);
            if (rc) return finish(rc);
            occupant[s] = -1;
            active--;
            done++;
        }
    }
    fill_serve_stats(results, nreq, now_s(t0), steps, cell_updates, max_cases, stats);
    return finish(CFD_OK);
}
}  // namespace

extern "C" int cfd_serve(const cfd_serve_config* cfg, const cfd_request* reqs, int nreq, cfd_result* results,
                         cfd_serve_stats* stats) {
    if (!cfg || !reqs || nreq < 0 || !results) {
        cfd_internal_set_error("cfd_serve: bad arguments");
        return CFD_E_ARG;
    }
    if (!cfg->class_slots) return serve_pool(cfg, reqs, nreq, results, stats);
    if (cfg->nclasses <= 0 || !cfg->class_grids || !cfg->class_profile) {
        cfd_internal_set_error("cfd_serve: bad arguments");
        return CFD_E_ARG;
    }
    const int nc = cfg->nclasses;
    std::vector<int> nslots(nc);
    for (int k = 0; k < nc; k++) {
        nslots[k] = cfg->class_slots[k];
        if (nslots[k] <= 0) {
            cfd_internal_set_error("cfd_serve: class_slots must be > 0");
            return CFD_E_ARG;
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
        const double tn = now_s(t0);
        for (int s = 0; s < nslot; s++) {
            const int r = occupant[s];
            if (r < 0) continue;
            cell_updates += (long long)tick * tg[s].n0 * tg[s].n1;
            if (!retire_if_done(reqs[r], st[s], tn, results[r])) continue;
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
    fill_serve_stats(results, nreq, makespan, steps, cell_updates, nslot, stats);
    return CFD_OK;
}
