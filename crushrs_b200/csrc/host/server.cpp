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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
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

// CRUSH_TRACE=1: each serving context prints where its host thread spent
// its time when it ends (diagnostics only).
struct ContextTrace {
    bool on = std::getenv("CRUSH_TRACE") && std::getenv("CRUSH_TRACE")[0] == '1';
    std::chrono::steady_clock::time_point born = std::chrono::steady_clock::now(), t = born;
    double ms[6] = {};  // create + begin, issue, append, wait for the chunk, results, other
    long long chunks = 0, appends = 0, appended = 0;
    void lap(int what) {
        if (!on) return;
        auto now = std::chrono::steady_clock::now();
        ms[what] += std::chrono::duration<double, std::milli>(now - t).count();
        t = now;
    }
    void print(int id, size_t slots) const {
        if (!on) return;
        const double life = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - born).count();
        std::fprintf(stderr,
                     "[crush-serve] context %d: %zu crashes, %lld chunks, %lld appends (%lld crashes); ms: create %.1f issue %.1f "
                     "append %.1f chunk wait %.1f results %.1f other %.1f life %.1f\n",
                     id, slots, chunks, appends, appended, ms[0], ms[1], ms[2], ms[3], ms[4], ms[5], life);
    }
};

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
    std::vector<std::pair<int, std::thread>> workers;  // (context id, thread)
    std::vector<int> finished;                         // contexts whose thread is ending (to join)
    double budget = 0.0, in_use = 0.0, peak = 0.0;
    int active = 0;                   // running contexts
    std::map<int, int> accepting;     // schedule class -> running contexts of it that still take requests
    std::map<int, std::pair<int, int>> load;  // accepting context id -> (schedule class, crashes running)
    bool stop = false;
    uint64_t next_ticket = 1;
    int64_t submitted = 0, completed = 0, contexts = 0;

    void run_context(std::vector<Request> first, int id, double bytes, crush_capacity room);
    void schedule();
    // Requests from the head of the queue with schedule class `key` whose
    // elements fit `elements` (at least one when `at_least_one`), removed
    // from the queue; called with mu held.
    std::vector<Request> take(int key, int64_t elements, int max_slots, bool at_least_one);
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

namespace {

// The room of a serving context: `elements` hexahedra and `slots` crashes
// of the serving mix (per hexahedron about 1.3 nodes, 0.11 contact faces and
// 0.17 listed contact nodes, plus per crash a few hundred of each for its
// road and small blocks; 4 contacts per crash), with margin.
crush_capacity serving_room(int64_t elements, int slots) {
    crush_capacity r;
    r.slots = slots;
    r.contacts = 6 * slots;
    r.hexes = elements;
    r.nodes = 2 * elements + 1000ll * slots;
    r.faces = elements / 4 + 1200ll * slots;
    r.primary_nodes = elements / 3 + 600ll * slots;
    return r;
}

// Device bytes of a context with that room (the admission measure of the
// HBM budget): per hexahedron its planes, state, corner forces, incidence
// and f64 arrays; per node the f64 node arrays; per contact face its
// geometry, cells and grid room; per contact its table room; per listed
// contact node its hit, events and roles; per slot its control blocks.
double room_bytes(const crush_capacity& r) {
    return 1100.0 * (double)r.hexes + 300.0 * (double)r.nodes + 800.0 * (double)r.faces + 15500.0 * (double)r.contacts +
           270.0 * (double)r.primary_nodes + 10000.0 * (double)r.slots;
}

// The room of a new context: the configured one, or a smaller one of the
// same mix that fits `left` bytes (never below the first request).
crush_capacity room_within(int64_t elements, int slots, double left, int64_t first_elements) {
    crush_capacity r = serving_room(elements, slots);
    while (room_bytes(r) > left && elements > first_elements) {
        elements = std::max<int64_t>(first_elements, elements / 2);
        slots = std::max(1, slots / 2);
        r = serving_room(elements, slots);
    }
    return r;
}

}  // namespace

std::vector<Request> crush_server::take(int key, int64_t elements, int max_slots, bool at_least_one) {
    std::vector<Request> out;
    int64_t e = 0;
    for (auto it = queue.begin(); it != queue.end() && (int)out.size() < max_slots;) {
        if (it->check_key != key) {
            ++it;
            continue;
        }
        if (e + it->elements > elements && !(at_least_one && out.empty())) break;  // keep arrival order within a class
        e += it->elements;
        out.push_back(std::move(*it));
        it = queue.erase(it);
    }
    return out;
}

// One serving context: a batched context with room for more crashes,
// created from the first requests, driven in chunks of steps on its own
// stream by this thread. Between chunks (step-graph boundaries) it admits
// waiting requests of its schedule class into the open run
// (crush_batch_append, whose host set-up overlaps the chunk just issued),
// reports every crash the moment it stops, and ends once its room is spent
// (or no request came for a while) and its crashes have all stopped.
void crush_server::run_context(std::vector<Request> first, int id, double bytes, crush_capacity room) {
    const int key = first.front().check_key;
    std::vector<Request> slots;  // the context's requests, by slot
    std::vector<double> start;   // when each slot began
    std::vector<int> reported;
    std::vector<crush_server_result> out;
    crush_ctx* ctx = nullptr;
    auto report = [&](int slot, int status, const crush_results* r) {
        crush_server_result x;
        std::memset(&x, 0, sizeof(x));
        x.ticket = slots[slot].ticket;
        x.status = status;
        x.wave = id;
        x.submit_s = slots[slot].submit_s;
        x.start_s = start[slot];
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
    int64_t used = 0;  // hexahedra admitted
    auto add = [&](std::vector<Request>& batch) {
        for (auto& r : batch) {
            used += r.elements;
            slots.push_back(std::move(r));
            start.push_back(now_s(t0));
            reported.push_back(0);
        }
        batch.clear();
    };
    std::vector<const crush_model_desc*> descs;
    for (auto& r : first) descs.push_back(&r.model->desc);
    ContextTrace tr;
    int st = crush_batch_create_reserved(descs.data(), (int)descs.size(), cfg.device, &room, &ctx);
    add(first);
    if (st == CRUSH_OK) st = crush_run_begin(ctx);
    tr.lap(0);
    bool open = true;  // still takes requests
    const int chunk = std::max(20, cfg.chunk_steps / 20 * 20);
    std::vector<int> flags;
    std::vector<crush_results> rs;
    while (st == CRUSH_OK) {
        int running = 0;
        for (size_t k = 0; k < slots.size(); ++k) running += reported[k] ? 0 : 1;
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (running == 0) {
                // Nothing on the device: wait for requests of this class, or end.
                if (!open || stop) break;
                const bool got = cv_work.wait_for(lk, std::chrono::duration<double, std::milli>(cfg.idle_ms), [&] {
                    if (stop) return true;
                    for (auto& q : queue)
                        if (q.check_key == key) return true;
                    return false;
                });
                if (!got || stop) break;
            }
            if (open) {
                load[id] = {key, running};
                // With max_running crashes running here and room for another
                // context, new requests are left to it (a crash's latency is
                // its steps times its context's step, which grows with the
                // crashes beside it).
                const bool held = cfg.max_running > 0 && running >= cfg.max_running && active < cfg.max_waves;
                if (!held) batch = take(key, room.hexes - used, room.slots - (int)slots.size(), false);
                // A request of this class waits that does not fit the room
                // left: this context takes no more, so the scheduler opens
                // another for it.
                bool waits = false;
                for (auto& q : queue) waits = waits || q.check_key == key;
                if (!held && batch.empty() && waits) {
                    --accepting[key];
                    load.erase(id);
                    open = false;
                    cv_work.notify_all();
                }
            }
        }
        tr.lap(5);
        if (running == 0 && batch.empty()) continue;  // nothing on the device, nothing admitted
        // Requests are waiting: short chunks, so the next admission comes soon.
        const bool waiting = !batch.empty();
        if (running > 0) {
            st = crush_run_issue(ctx, waiting ? 20 : chunk);
            ++tr.chunks;
        }
        tr.lap(1);
        if (st != CRUSH_OK) break;
        if (!batch.empty()) {
            descs.clear();
            for (auto& r : batch) descs.push_back(&r.model->desc);
            const int a = crush_batch_append(ctx, descs.data(), (int)descs.size(), nullptr);
            tr.lap(2);
            if (a == CRUSH_OK) {
                ++tr.appends;
                tr.appended += (long long)batch.size();
                add(batch);
            } else {
                // No room (or not admissible here): back to the queue's head
                // for another context; this one takes no more.
                std::lock_guard<std::mutex> lk(mu);
                for (auto it = batch.rbegin(); it != batch.rend(); ++it) queue.push_front(std::move(*it));
                if (open) {
                    --accepting[key];
                    load.erase(id);
                }
                open = false;
                cv_work.notify_all();
                if (a != CRUSH_ERR_BUSY && a != CRUSH_ERR_UNSUPPORTED) {
                    st = a;
                    break;
                }
            }
        }
        flags.assign(slots.size(), 0);
        int all = 0;
        st = crush_batch_done(ctx, flags.data(), &all);
        tr.lap(3);
        if (st != CRUSH_OK) break;
        int lo = (int)slots.size(), hi = -1;
        for (int k = 0; k < (int)slots.size(); ++k)
            if (flags[k] && !reported[k]) {
                lo = std::min(lo, k);
                hi = std::max(hi, k);
            }
        if (hi >= lo) {
            rs.resize(hi - lo + 1);
            st = crush_batch_results_range(ctx, lo, hi - lo + 1, rs.data());
            if (st != CRUSH_OK) break;
            for (int k = lo; k <= hi; ++k)
                if (flags[k] && !reported[k]) {
                    reported[k] = 1;
                    report(k, rs[k - lo].status, &rs[k - lo]);
                }
            flush();
            tr.lap(4);
        }
        if (open && ((int)slots.size() >= room.slots || used >= room.hexes)) {
            std::lock_guard<std::mutex> lk(mu);
            --accepting[key];
            load.erase(id);
            open = false;
            cv_work.notify_all();
        }
        }
    for (size_t k = 0; k < slots.size(); ++k)
        if (!reported[k]) report((int)k, st == CRUSH_OK ? CRUSH_ERR_INVALID : st, nullptr);
    if (ctx) crush_destroy(ctx);
    flush();
    tr.lap(5);
    tr.print(id, slots.size());
    std::lock_guard<std::mutex> lk(mu);
    if (open) --accepting[key];
    load.erase(id);
    in_use -= bytes;
    --active;
    finished.push_back(id);
    cv_work.notify_all();
    cv_done.notify_all();
}

// Joins the threads of finished contexts (called with mu held; those threads
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

// Opens a context when requests wait that no open context takes: none is
// accepting (room spent) or none of their schedule class runs, within the
// context and HBM limits.
void crush_server::schedule() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_work.wait_for(lk, std::chrono::milliseconds(5));
        join_finished(this);
        if (stop && queue.empty()) break;
        if (queue.empty() || active >= cfg.max_waves) continue;
        // Classes that an accepting context serves take their requests
        // themselves; a request of another class (or with every context
        // full) opens a context.
        // (With max_running, also when every accepting context of the class
        // has that many crashes running.)
        auto served = [&](int key) {
            if (accepting[key] <= 0) return false;
            if (cfg.max_running <= 0) return true;
            for (auto& kv : load)
                if (kv.second.first == key && kv.second.second < cfg.max_running) return true;
            return false;
        };
        const Request& head = queue.front();
        if (served(head.check_key)) continue;
        // While other contexts run, give arrivals a moment to join this one.
        if (active > 0 && cfg.gather_ms > 0.0) {
            cv_work.wait_for(lk, std::chrono::duration<double, std::milli>(cfg.gather_ms));
            if (queue.empty() || served(queue.front().check_key)) continue;
        }
        const crush_capacity room = room_within(cfg.max_wave_elements, cfg.max_wave_slots, budget - in_use, queue.front().elements);
        const double bytes = room_bytes(room);
        if (in_use + bytes > budget && active > 0) continue;  // wait for a context to finish
        std::vector<Request> first = take(queue.front().check_key, room.hexes, room.slots, true);
        if (first.empty()) continue;
        in_use += bytes;
        peak = std::max(peak, in_use);
        ++active;
        ++accepting[first.front().check_key];
        const int id = (int)contexts++;
        load[id] = {first.front().check_key, (int)first.size()};
        workers.emplace_back(id, std::thread(&crush_server::run_context, this, std::move(first), id, bytes, room));
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
    c.max_wave_slots = 1024;
    c.chunk_steps = 100;
    c.max_wave_elements = 2000000;
    c.hbm_budget_bytes = 0.0;
    c.gather_ms = 2.0;
    c.idle_ms = 200.0;
    if (config) {
        c.device = config->device;
        if (config->max_waves > 0) c.max_waves = config->max_waves;
        if (config->max_wave_slots > 0) c.max_wave_slots = config->max_wave_slots;
        if (config->chunk_steps > 0) c.chunk_steps = config->chunk_steps;
        if (config->max_wave_elements > 0) c.max_wave_elements = config->max_wave_elements;
        if (config->hbm_budget_bytes > 0.0) c.hbm_budget_bytes = config->hbm_budget_bytes;
        if (config->gather_ms >= 0.0) c.gather_ms = config->gather_ms;
        if (config->idle_ms > 0.0) c.idle_ms = config->idle_ms;
        if (config->max_queue > 0) c.max_queue = config->max_queue;
        if (config->max_running > 0) c.max_running = config->max_running;
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
    auto full = [&]() { return s->cfg.max_queue > 0 && (int64_t)s->queue.size() >= (int64_t)s->cfg.max_queue; };
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (full()) return crush::fail(CRUSH_ERR_BUSY, "request queue full");
    }
    Request r;
    r.model.reset(new OwnedModel(*desc));
    r.bytes = crush_model_footprint(desc);
    r.elements = desc->n_hexes;
    r.check_key = schedule_key(desc->settings);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return crush::fail(CRUSH_ERR_BUSY, "server is shutting down");
    if (full()) return crush::fail(CRUSH_ERR_BUSY, "request queue full");
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
    out->waves = s->contexts;
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
