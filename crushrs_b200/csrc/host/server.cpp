// server.cpp — the continuous-batching crash server of crush_server.h.
//
// Built only on the public C ABI of crush.h: a wave is a batched context
// (crush_batch_create), driven in chunks of steps by its own host thread on
// its own CUDA stream; finished slots are read with crush_batch_done and
// crush_batch_results_range and handed to the result queue immediately.
#include "crush_server.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "errors.hpp"

namespace {

// A deep copy of a model description (the server owns its requests).
struct OwnedModel {
    std::vector<double> positions, velocity;
    std::vector<uint32_t> hexes, fixed;
    std::vector<int32_t> hex_part;
    std::vector<crush_material> materials;
    std::vector<std::vector<uint32_t>> c_nodes, c_faces, v_nodes, v_front;
    std::vector<std::vector<double>> c_scale;
    std::vector<crush_contact> contacts;
    std::vector<crush_vehicle> vehicles;
    crush_model_desc desc{};

    explicit OwnedModel(const crush_model_desc& d) {
        positions.assign(d.positions, d.positions + 3 * d.n_nodes);
        if (d.initial_velocity) velocity.assign(d.initial_velocity, d.initial_velocity + 3 * d.n_nodes);
        hexes.assign(d.hexes, d.hexes + 8 * d.n_hexes);
        hex_part.assign(d.hex_part, d.hex_part + d.n_hexes);
        if (d.n_fixed > 0) fixed.assign(d.fixed_nodes, d.fixed_nodes + d.n_fixed);
        materials.assign(d.materials, d.materials + d.n_parts);
        contacts.resize(d.n_contacts);
        c_nodes.resize(d.n_contacts);
        c_faces.resize(d.n_contacts);
        c_scale.resize(d.n_contacts);
        for (int k = 0; k < d.n_contacts; ++k) {
            const crush_contact& s = d.contacts[k];
            c_nodes[k].assign(s.nodes, s.nodes + std::max<int64_t>(s.n_nodes, 0));
            c_faces[k].assign(s.faces, s.faces + 4 * std::max<int64_t>(s.n_faces, 0));
            if (s.node_scale) c_scale[k].assign(s.node_scale, s.node_scale + std::max<int64_t>(s.n_nodes, 0));
            contacts[k] = s;
            contacts[k].nodes = c_nodes[k].data();
            contacts[k].faces = c_faces[k].data();
            contacts[k].node_scale = s.node_scale ? c_scale[k].data() : nullptr;
        }
        vehicles.resize(d.n_vehicles);
        v_nodes.resize(d.n_vehicles);
        v_front.resize(d.n_vehicles);
        for (int k = 0; k < d.n_vehicles; ++k) {
            const crush_vehicle& s = d.vehicles[k];
            v_nodes[k].assign(s.nodes, s.nodes + std::max<int64_t>(s.n_nodes, 0));
            v_front[k].assign(s.front_nodes, s.front_nodes + std::max<int64_t>(s.n_front, 0));
            vehicles[k] = s;
            vehicles[k].nodes = v_nodes[k].data();
            vehicles[k].front_nodes = v_front[k].data();
        }
        desc = d;
        desc.positions = positions.data();
        desc.initial_velocity = d.initial_velocity ? velocity.data() : nullptr;
        desc.hexes = hexes.data();
        desc.hex_part = hex_part.data();
        desc.fixed_nodes = fixed.empty() ? nullptr : fixed.data();
        desc.materials = materials.data();
        desc.contacts = contacts.empty() ? nullptr : contacts.data();
        desc.vehicles = vehicles.empty() ? nullptr : vehicles.data();
    }
};

struct Request {
    uint64_t ticket;
    std::unique_ptr<OwnedModel> model;
    double submit_s;
    double bytes;
    int64_t elements;
    int check_key;  // models of one wave share the step schedule
};

double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int schedule_key(const crush_settings& s) {
    const bool adaptive = !(s.time_step > 0.0) && s.adaptive_check_steps > 0;
    return adaptive ? s.adaptive_check_steps : -1;
}

}  // namespace

struct crush_server {
    crush_server_config cfg{};
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> queue;
    std::deque<crush_server_result> done;
    std::thread scheduler;
    std::vector<std::pair<int, std::thread>> workers;  // (wave id, thread)
    std::vector<int> finished;                         // waves whose thread is ending (to join)
    double budget = 0.0, in_use = 0.0, peak = 0.0;
    int active = 0;
    bool stop = false;
    uint64_t next_ticket = 1;
    int64_t submitted = 0, completed = 0, waves = 0;

    void run_wave(std::vector<Request> wave, int wave_id, double bytes);
    void schedule();
};

extern "C" double crush_model_footprint(const crush_model_desc* d) {
    if (!d) return 0.0;
    double faces = 0.0, slaves = 0.0;
    for (int k = 0; k < d->n_contacts; ++k) {
        faces += (double)d->contacts[k].n_faces;
        slaves += (double)d->contacts[k].n_nodes;
    }
    // element planes, state, corner forces, incidence, f64 element arrays;
    // nine 3N and five N f64 node arrays; contact geometry, hit lists, grids
    return 1100.0 * (double)d->n_hexes + 300.0 * (double)d->n_nodes + 330.0 * faces + 120.0 * slaves + 8192.0;
}

void crush_server::run_wave(std::vector<Request> wave, int wave_id, double bytes) {
    const double start = now_s(t0);
    std::vector<const crush_model_desc*> descs(wave.size());
    for (size_t k = 0; k < wave.size(); ++k) descs[k] = &wave[k].model->desc;
    crush_ctx* ctx = nullptr;
    const int n = (int)wave.size();
    std::vector<crush_server_result> out;
    auto report = [&](int slot, int status, const crush_results* r) {
        crush_server_result x;
        std::memset(&x, 0, sizeof(x));
        x.ticket = wave[slot].ticket;
        x.status = status;
        x.wave = wave_id;
        x.submit_s = wave[slot].submit_s;
        x.start_s = start;
        x.finish_s = now_s(t0);
        if (r) x.results = *r;
        out.push_back(x);
    };
    auto flush = [&]() {
        if (out.empty()) return;
        std::lock_guard<std::mutex> lk(mu);
        for (auto& x : out) done.push_back(x);
        completed += (int64_t)out.size();
        out.clear();
        cv_done.notify_all();
    };
    int st = crush_batch_create(descs.data(), n, cfg.device, &ctx);
    if (st == CRUSH_OK) st = crush_run_begin(ctx);
    if (st == CRUSH_OK) {
        std::vector<int> flags(n, 0), reported(n, 0);
        std::vector<crush_results> rs;
        int remaining = n, all = 0;
        while (remaining > 0 && st == CRUSH_OK) {
            st = crush_run_steps(ctx, cfg.chunk_steps, &all);
            if (st != CRUSH_OK) break;
            st = crush_batch_done(ctx, flags.data(), &all);
            if (st != CRUSH_OK) break;
            int lo = n, hi = -1;
            for (int k = 0; k < n; ++k)
                if (flags[k] && !reported[k]) {
                    lo = std::min(lo, k);
                    hi = std::max(hi, k);
                }
            if (hi < lo) continue;
            rs.resize(hi - lo + 1);
            st = crush_batch_results_range(ctx, lo, hi - lo + 1, rs.data());
            if (st != CRUSH_OK) break;
            for (int k = lo; k <= hi; ++k)
                if (flags[k] && !reported[k]) {
                    reported[k] = 1;
                    --remaining;
                    report(k, rs[k - lo].status, &rs[k - lo]);
                }
            flush();
        }
        if (st != CRUSH_OK)
            for (int k = 0; k < n; ++k)
                if (!reported[k]) report(k, st, nullptr);
    } else {
        for (int k = 0; k < n; ++k) report(k, st, nullptr);
    }
    if (ctx) crush_destroy(ctx);
    wave.clear();
    flush();
    std::lock_guard<std::mutex> lk(mu);
    in_use -= bytes;
    --active;
    finished.push_back(wave_id);
    cv_work.notify_all();
    cv_done.notify_all();
}

// Joins the threads of finished waves (called with mu held; those threads
// only return after releasing it).
void join_finished(crush_server* s) {
    for (int id : s->finished)
        for (auto it = s->workers.begin(); it != s->workers.end(); ++it)
            if (it->first == id) {
                if (it->second.joinable()) it->second.join();
                s->workers.erase(it);
                break;
            }
    s->finished.clear();
}

void join_finished(crush_server* s);

void crush_server::schedule() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_work.wait(lk, [&] { return stop || !finished.empty() || (!queue.empty() && active < cfg.max_waves); });
        join_finished(this);
        if (queue.empty()) {
            if (stop) break;
            continue;
        }
        if (active >= cfg.max_waves) continue;
        // While the GPU is busy, give arrivals a moment to join this wave.
        if (active > 0 && cfg.gather_ms > 0.0 && !stop) {
            cv_work.wait_for(lk, std::chrono::duration<double, std::milli>(cfg.gather_ms), [&] { return stop; });
            if (queue.empty()) continue;
        }
        // Form a wave from the head of the queue: same step schedule, within
        // the slot, element and memory limits.
        const int key = queue.front().check_key;
        std::vector<Request> wave;
        double bytes = 0.0;
        int64_t elements = 0;
        for (auto it = queue.begin(); it != queue.end() && (int)wave.size() < cfg.max_wave_slots;) {
            const bool fits = in_use + bytes + it->bytes <= budget && elements + it->elements <= cfg.max_wave_elements;
            if (it->check_key == key && (fits || (wave.empty() && active == 0))) {
                bytes += it->bytes;
                elements += it->elements;
                wave.push_back(std::move(*it));
                it = queue.erase(it);
            } else if (!fits && it->check_key == key) {
                break;  // keep arrival order within a schedule class
            } else {
                ++it;
            }
        }
        if (wave.empty()) {
            // The head does not fit while other waves hold memory: wait for one to finish.
            cv_work.wait(lk, [&] { return stop || active == 0 || in_use + queue.front().bytes <= budget; });
            continue;
        }
        in_use += bytes;
        peak = std::max(peak, in_use);
        ++active;
        const int id = (int)waves++;
        workers.emplace_back(id, std::thread(&crush_server::run_wave, this, std::move(wave), id, bytes));
    }
}

extern "C" {

int crush_server_create(const crush_server_config* config, crush_server** out) {
    if (!out) return crush::fail(CRUSH_ERR_INVALID, "null output");
    *out = nullptr;
    crush_server* s = new crush_server();
    crush_server_config c{};
    c.device = 0;
    c.max_waves = 4;
    c.max_wave_slots = 2048;
    c.chunk_steps = 100;
    c.max_wave_elements = 8000000;
    c.hbm_budget_bytes = 0.0;
    c.gather_ms = 2.0;
    if (config) {
        c.device = config->device;
        if (config->max_waves > 0) c.max_waves = config->max_waves;
        if (config->max_wave_slots > 0) c.max_wave_slots = config->max_wave_slots;
        if (config->chunk_steps > 0) c.chunk_steps = config->chunk_steps;
        if (config->max_wave_elements > 0) c.max_wave_elements = config->max_wave_elements;
        if (config->hbm_budget_bytes > 0.0) c.hbm_budget_bytes = config->hbm_budget_bytes;
        if (config->gather_ms >= 0.0) c.gather_ms = config->gather_ms;
    }
    s->cfg = c;
    if (c.hbm_budget_bytes > 0.0) {
        s->budget = c.hbm_budget_bytes;
    } else {
        size_t fr = 0, total = 0;
        if (cudaSetDevice(c.device) != cudaSuccess || cudaMemGetInfo(&fr, &total) != cudaSuccess) {
            cudaGetLastError();
            delete s;
            return crush::fail(CRUSH_ERR_CUDA, "crush_server_create: cannot query device memory");
        }
        s->budget = 0.8 * (double)fr;
    }
    s->scheduler = std::thread(&crush_server::schedule, s);
    *out = s;
    return CRUSH_OK;
}

int crush_server_submit(crush_server* s, const crush_model_desc* desc, uint64_t* ticket) {
    if (!s || !desc) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    if (desc->n_nodes <= 0 || !desc->positions || desc->n_hexes < 0 || (desc->n_hexes > 0 && (!desc->hexes || !desc->hex_part)) ||
        desc->n_parts <= 0 || !desc->materials || (desc->n_contacts > 0 && !desc->contacts) || (desc->n_vehicles > 0 && !desc->vehicles) ||
        (desc->n_fixed > 0 && !desc->fixed_nodes))
        return crush::fail(CRUSH_ERR_INVALID, "invalid model description");
    Request r;
    r.model.reset(new OwnedModel(*desc));
    r.bytes = crush_model_footprint(desc);
    r.elements = desc->n_hexes;
    r.check_key = schedule_key(desc->settings);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return crush::fail(CRUSH_ERR_BUSY, "server is shutting down");
    r.ticket = s->next_ticket++;
    r.submit_s = now_s(s->t0);
    if (ticket) *ticket = r.ticket;
    s->queue.push_back(std::move(r));
    ++s->submitted;
    s->cv_work.notify_all();
    return CRUSH_OK;
}

int crush_server_poll(crush_server* s, crush_server_result* out, int max, int* n, int wait_ms) {
    if (!s || (!out && max > 0) || !n) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    int k = 0;
    while (k < max && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *n = k;
    return CRUSH_OK;
}

int crush_server_stats_get(crush_server* s, crush_server_stats* out) {
    if (!s || !out) return crush::fail(CRUSH_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->waves = s->waves;
    out->queued = (int64_t)s->queue.size();
    out->running = s->active;
    out->bytes_in_use = s->in_use;
    out->peak_bytes_in_use = s->peak;
    out->budget_bytes = s->budget;
    return CRUSH_OK;
}

void crush_server_destroy(crush_server* s) {
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // finish what was submitted
        s->cv_done.wait(lk, [&] { return s->queue.empty() && s->active == 0; });
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->scheduler.joinable()) s->scheduler.join();
    for (auto& w : s->workers)
        if (w.second.joinable()) w.second.join();
    delete s;
}

}  // extern "C"
