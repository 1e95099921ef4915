// Batched and served runs of many scenes on one GPU: a host layer over the
// library's own C ABI (sdr_solver_*, sdr_metrics_*).
//
// The reference simulates one scene per process: build the scene, then per
// frame Solver::step and MetricsCollector::record, then the summary
// (main.rs:215-386). Here every scene runs that loop on its own solver (its
// own device state and CUDA stream) in its own host thread, so the kernels of
// different scenes overlap on the GPU: a scene's pressure solve occupies one
// SM, and a B200 has 148. Scenes never share device memory, so a scene's
// result is the same alone and in any mix (every solver is deterministic).
//
// Threads wait for their streams with blocking synchronisation
// (SDR_SOLVER_BLOCKING_SYNC) so that many more scene threads than host cores
// do not spin.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "packed_engine.h"
#include "sdr_gpu.h"

void sdr_internal_set_error(const std::string& msg);

namespace {

using Clock = std::chrono::steady_clock;

// A scene whose SDF values the layer owns.
struct SceneCopy {
    sdr_scene_desc d{};
    std::vector<double> sdf;
    explicit SceneCopy(const sdr_scene_desc& s) : d(s) {
        size_t n = (size_t)(s.sdf.nx * s.sdf.ny * s.sdf.nz);
        sdf.assign(s.sdf.data, s.sdf.data + n);
        d.sdf.data = sdf.data();
    }
};

struct SceneResult {
    int status = SDR_ERR_INVALID;  // not run yet
    std::string error = "not run";
    sdr_summary summary{};
    sdr_solver_stats stats{};
    double seconds = 0.0;
};

bool valid_scene(const sdr_scene_desc* s, std::string& why) {
    if (!s) return why = "null scene", false;
    if (!s->sdf.data || s->sdf.nx < 2 || s->sdf.ny < 2 || s->sdf.nz < 2) return why = "SDF needs data and >= 2 nodes per axis", false;
    if (!(s->sdf.dx > 0.0) || !(s->sim_dx > 0.0)) return why = "dx must be positive", false;
    if (!(s->frame_dt > 0.0)) return why = "frame_dt must be positive", false;
    if (!(s->cavity_volume > 0.0)) return why = "cavity_volume must be positive", false;
    return true;
}

// Solver::new grid (solver.rs:185-190): the MAC grid covering the SDF bounds.
void grid_dims(const sdr_scene_desc& s, uint64_t& nx, uint64_t& ny, uint64_t& nz) {
    auto cells = [&](uint64_t n) {
        double span = (double)(n - 1) * s.sdf.dx;
        return (uint64_t)std::fmax(std::ceil(span / s.sim_dx), 1.0);
    };
    nx = cells(s.sdf.nx);
    ny = cells(s.sdf.ny);
    nz = cells(s.sdf.nz);
}

// Particles the run can hold: the dose (flow x injection time within the run)
// over the particle volume (solver.rs:225-228), with a margin.
uint64_t particle_capacity(const sdr_scene_desc& s) {
    if (s.max_particles) return s.max_particles;
    double run = (double)s.frames * s.frame_dt;
    double inject = std::fmax(0.0, std::fmin(s.needle.inject_until, run));
    double pv = s.sim_dx * s.sim_dx * s.sim_dx / (double)std::max<uint64_t>(s.fluid.particles_per_cell, 1);
    double n = s.needle.flow_rate > 0.0 ? s.needle.flow_rate * inject / pv : 0.0;
    return (uint64_t)std::ceil(n * 1.25) + 65536;
}

uint64_t footprint(const sdr_scene_desc& s) {
    uint64_t nx, ny, nz;
    grid_dims(s, nx, ny, nz);
    const uint64_t cells = nx * ny * nz, nodes = (nx + 1) * (ny + 1) * (nz + 1);
    const uint64_t sdf_nodes = s.sdf.nx * s.sdf.ny * s.sdf.nz;
    // per cell: labels, histograms, wavefront tables, PCG vectors (f64), pressure;
    // per node: the six face arrays and their scratch copies (f32); per
    // particle: positions and velocities (double-buffered float4), sort keys,
    // gather records; the SDF in f64 and f32; a fixed workspace.
    return 320 * cells + 64 * nodes + 160 * particle_capacity(s) + 12 * sdf_nodes + (16ull << 20);
}

// One scene end to end: create, frames x (step, record), summary, destroy.
// `shared`: other scenes run beside this one (SDR_SOLVER_SHARED_GPU); a scene
// alone on the GPU gets the default solver (cluster pressure solve).
SceneResult run_scene(const sdr_scene_desc& d, int32_t device, bool shared) {
    SceneResult r;
    const auto t0 = Clock::now();
    sdr_solver* s = nullptr;
    sdr_metrics* m = nullptr;
    auto fail = [&](int rc) {
        r.status = rc;
        r.error = sdr_last_error();
    };
    sdr_solver_options o{};
    o.max_particles = particle_capacity(d);
    o.device = device;
    o.flags = SDR_SOLVER_BLOCKING_SYNC | (shared ? SDR_SOLVER_SHARED_GPU : 0);
    int rc = sdr_solver_create(&d.sdf, d.sim_dx, &d.fluid, &d.needle, &o, &s);
    if (rc == SDR_OK && d.has_outlet) rc = sdr_solver_set_outlet(s, &d.outlet);
    if (rc == SDR_OK) rc = sdr_solver_set_solve_params(s, &d.solve);
    if (rc == SDR_OK) rc = sdr_metrics_create(s, d.cavity_volume, &m);
    for (uint64_t f = 0; rc == SDR_OK && f < d.frames; ++f) {
        rc = sdr_solver_step(s, d.frame_dt);
        sdr_frame_metrics fm;
        if (rc == SDR_OK) rc = sdr_metrics_record(m, s, f, &fm);
    }
    if (rc == SDR_OK) rc = sdr_metrics_summary(m, &r.summary);
    if (rc == SDR_OK) rc = sdr_solver_get_stats(s, &r.stats);
    if (rc != SDR_OK) {
        fail(rc);
    } else {
        r.status = SDR_OK;
        r.error.clear();
    }
    if (m) sdr_metrics_destroy(m);
    if (s) sdr_solver_destroy(s);
    r.seconds = std::chrono::duration<double>(Clock::now() - t0).count();
    return r;
}

void copy_error(const std::string& e, char* out, size_t cap) {
    if (!out || cap == 0) return;
    size_t n = std::min(cap - 1, e.size());
    std::memcpy(out, e.data(), n);
    out[n] = 0;
}

int invalid(const std::string& why) {
    sdr_internal_set_error(why);
    return SDR_ERR_INVALID;
}

}  // namespace

struct sdr_batch {
    int32_t device = -1;
    std::vector<std::unique_ptr<SceneCopy>> scenes;
    std::vector<SceneResult> results;
    uint64_t packed_launches = 0, packed_steps = 0, packed_captures = 0;  // of the last packed run
    int packed_ctas = 0;
};

struct Request {
    uint64_t id = 0;
    std::unique_ptr<SceneCopy> scene;
    uint64_t bytes = 0;
    Clock::time_point submitted;
    int32_t state = SDR_REQ_QUEUED;
    SceneResult result;
    double latency = 0.0;
};

struct sdr_server {
    int32_t device = -1;
    uint64_t budget = 0;
    uint32_t max_active = 1;
    std::mutex mu;
    std::condition_variable cv_admit;  // dispatcher: a request arrived or memory freed
    std::condition_variable cv_work;   // workers: a request was admitted
    std::deque<Request*> pending;      // arrival order
    std::deque<Request*> admitted;
    std::map<uint64_t, std::unique_ptr<Request>> requests;
    uint64_t next_id = 1;
    bool stopping = false;
    sdr_server_stats stats{};
    std::thread dispatcher;
    std::vector<std::thread> workers;
    bool packed = false;  // one engine thread advances every admitted scene in packed steps

    // Packed mode: admit between packed steps, step every live scene together,
    // hand finished scenes back. Requests that arrive while others run join at
    // the next step, as slots and budget free up.
    void engine_loop() {
        PackedEngine* e = packed_engine_create(device);
        std::vector<PackedDone> done;
        std::unique_lock<std::mutex> lk(mu);
        const std::string fail_msg = e ? "" : std::string("packed engine: ") + sdr_last_error();
        for (;;) {
            std::vector<Request*> start;
            while (head_fits()) {
                Request* r = pending.front();
                pending.pop_front();
                stats.bytes_in_use += r->bytes;
                stats.peak_bytes = std::max(stats.peak_bytes, stats.bytes_in_use);
                r->state = SDR_REQ_RUNNING;
                stats.active += 1;
                stats.peak_active = std::max(stats.peak_active, stats.active);
                start.push_back(r);
            }
            const size_t live = e ? packed_engine_live(e) : 0;
            if (start.empty() && live == 0) {
                if (stopping && pending.empty()) break;
                cv_admit.wait(lk, [&] { return (stopping && pending.empty()) || head_fits(); });
                continue;
            }
            lk.unlock();
            done.clear();
            for (Request* r : start) {
                if (e) {
                    packed_engine_add(e, r->scene->d, particle_capacity(r->scene->d), r->id, done);
                } else {
                    PackedDone d;
                    d.tag = r->id;
                    d.status = SDR_ERR_CUDA;
                    d.error = fail_msg;
                    done.push_back(d);
                }
            }
            if (e && packed_engine_live(e)) packed_engine_step(e, done);
            lk.lock();
            for (auto& d : done) {
                Request* r = requests[d.tag].get();
                r->result.status = d.status;
                r->result.error = d.error;
                r->result.summary = d.summary;
                r->result.stats = d.stats;
                r->latency = std::chrono::duration<double>(Clock::now() - r->submitted).count();
                r->state = d.status == SDR_OK ? SDR_REQ_DONE : SDR_REQ_FAILED;
                r->scene.reset();
                stats.active -= 1;
                stats.bytes_in_use -= r->bytes;
                if (r->state == SDR_REQ_DONE) stats.completed += 1;
                else stats.failed += 1;
            }
        }
        lk.unlock();
        packed_engine_destroy(e);
    }

    // Admit from the head of the queue while the head fits (arrival order: a
    // large request at the head is not overtaken by smaller ones behind it).
    bool head_fits() const {
        return !pending.empty() && stats.active + admitted.size() < max_active &&
               stats.bytes_in_use + pending.front()->bytes <= budget;
    }

    void dispatch_loop() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            // Sleep until the head fits, or until shutdown finds the queue empty
            // (queued requests are still run at shutdown; the finishing work wakes us).
            cv_admit.wait(lk, [&] { return (stopping && pending.empty()) || head_fits(); });
            if (stopping && pending.empty()) return;
            while (head_fits()) {
                Request* r = pending.front();
                pending.pop_front();
                stats.bytes_in_use += r->bytes;
                stats.peak_bytes = std::max(stats.peak_bytes, stats.bytes_in_use);
                admitted.push_back(r);
                cv_work.notify_one();
            }
        }
    }

    void worker_loop() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv_work.wait(lk, [&] { return !admitted.empty() || (stopping && pending.empty()); });
            if (admitted.empty()) return;
            Request* r = admitted.front();
            admitted.pop_front();
            r->state = SDR_REQ_RUNNING;
            stats.active += 1;
            stats.peak_active = std::max(stats.peak_active, stats.active);
            lk.unlock();
            SceneResult res = run_scene(r->scene->d, device, true);
            lk.lock();
            r->result = std::move(res);
            r->latency = std::chrono::duration<double>(Clock::now() - r->submitted).count();
            r->state = r->result.status == SDR_OK ? SDR_REQ_DONE : SDR_REQ_FAILED;
            r->scene.reset();  // the SDF copy is no longer needed
            stats.active -= 1;
            stats.bytes_in_use -= r->bytes;
            if (r->state == SDR_REQ_DONE) stats.completed += 1;
            else stats.failed += 1;
            cv_admit.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

int sdr_scene_footprint(const sdr_scene_desc* scene, uint64_t* bytes) {
    std::string why;
    if (!bytes) return invalid("null argument");
    if (!valid_scene(scene, why)) return invalid(why);
    *bytes = footprint(*scene);
    return SDR_OK;
}

int sdr_batch_create(const sdr_scene_desc* scenes, size_t n, int32_t device, sdr_batch** out) {
    if (!out || (n && !scenes)) return invalid("null argument");
    *out = nullptr;
    std::string why;
    for (size_t i = 0; i < n; ++i)
        if (!valid_scene(&scenes[i], why)) return invalid("scene " + std::to_string(i) + ": " + why);
    try {
        auto b = std::make_unique<sdr_batch>();
        b->device = device;
        for (size_t i = 0; i < n; ++i) b->scenes.push_back(std::make_unique<SceneCopy>(scenes[i]));
        b->results.resize(n);
        *out = b.release();
        return SDR_OK;
    } catch (const std::bad_alloc&) {
        sdr_internal_set_error("host allocation failed");
        return SDR_ERR_OOM;
    }
}

int sdr_batch_run(sdr_batch* b, uint32_t concurrency) {
    if (!b) return invalid("null batch");
    const size_t n = b->scenes.size();
    if (n == 0) return SDR_OK;
    const size_t threads = concurrency == 0 ? n : std::min<size_t>(concurrency, n);
    std::atomic<size_t> next{0};
    auto body = [&] {
        for (size_t i; (i = next.fetch_add(1)) < n;)
            b->results[i] = run_scene(b->scenes[i]->d, b->device, threads > 1);
    };
    std::vector<std::thread> pool;
    pool.reserve(threads);
    for (size_t t = 0; t < threads; ++t) pool.emplace_back(body);
    for (auto& t : pool) t.join();
    return SDR_OK;
}

int sdr_batch_run_packed(sdr_batch* b) {
    if (!b) return invalid("null batch");
    PackedEngine* e = packed_engine_create(b->device);
    if (!e) return SDR_ERR_CUDA;
    const auto t0 = Clock::now();
    std::vector<PackedDone> done;
    auto take = [&] {
        const double t = std::chrono::duration<double>(Clock::now() - t0).count();
        for (auto& d : done) {
            SceneResult& r = b->results[d.tag];
            r.status = d.status;
            r.error = d.error;
            r.summary = d.summary;
            r.stats = d.stats;
            r.seconds = t;
        }
        done.clear();
    };
    for (size_t i = 0; i < b->scenes.size(); ++i)
        packed_engine_add(e, b->scenes[i]->d, particle_capacity(b->scenes[i]->d), i, done);
    take();
    while (packed_engine_live(e)) {
        packed_engine_step(e, done);
        take();
    }
    packed_engine_counters(e, &b->packed_launches, &b->packed_steps, &b->packed_captures, &b->packed_ctas);
    packed_engine_destroy(e);
    return SDR_OK;
}

int sdr_batch_packed_counters(const sdr_batch* b, uint64_t* launches, uint64_t* steps, uint64_t* graph_captures,
                              int32_t* ctas_per_sm) {
    if (!b || !launches || !steps) return invalid("null argument");
    *launches = b->packed_launches;
    *steps = b->packed_steps;
    if (graph_captures) *graph_captures = b->packed_captures;
    if (ctas_per_sm) *ctas_per_sm = b->packed_ctas;
    return SDR_OK;
}

int sdr_batch_result(const sdr_batch* b, size_t i, int32_t* status, sdr_summary* summary,
                     sdr_solver_stats* stats_or_null, double* seconds_or_null, char* error, size_t error_cap) {
    if (!b || !status || !summary) return invalid("null argument");
    if (i >= b->results.size()) return invalid("scene index out of range");
    const SceneResult& r = b->results[i];
    *status = r.status;
    *summary = r.summary;
    if (stats_or_null) *stats_or_null = r.stats;
    if (seconds_or_null) *seconds_or_null = r.seconds;
    copy_error(r.error, error, error_cap);
    return SDR_OK;
}

int sdr_batch_destroy(sdr_batch* b) {
    delete b;
    return SDR_OK;
}

int sdr_server_create(int32_t device, uint64_t budget_bytes, uint32_t max_active, sdr_server** out) {
    if (!out) return invalid("null argument");
    if (budget_bytes == 0 || max_active == 0) return invalid("budget and max_active must be positive");
    *out = nullptr;
    try {
        auto s = std::make_unique<sdr_server>();
        s->device = device;
        s->budget = budget_bytes;
        s->max_active = max_active;
        s->dispatcher = std::thread([p = s.get()] { p->dispatch_loop(); });
        for (uint32_t i = 0; i < max_active; ++i) s->workers.emplace_back([p = s.get()] { p->worker_loop(); });
        *out = s.release();
        return SDR_OK;
    } catch (const std::exception& e) {
        sdr_internal_set_error(std::string("server start failed: ") + e.what());
        return SDR_ERR_INVALID;
    }
}

int sdr_server_create_packed(int32_t device, uint64_t budget_bytes, uint32_t max_active, sdr_server** out) {
    if (!out) return invalid("null argument");
    if (budget_bytes == 0 || max_active == 0) return invalid("budget and max_active must be positive");
    *out = nullptr;
    try {
        auto s = std::make_unique<sdr_server>();
        s->device = device;
        s->budget = budget_bytes;
        s->max_active = max_active;
        s->packed = true;
        s->dispatcher = std::thread([p = s.get()] { p->engine_loop(); });
        *out = s.release();
        return SDR_OK;
    } catch (const std::exception& e) {
        sdr_internal_set_error(std::string("server start failed: ") + e.what());
        return SDR_ERR_INVALID;
    }
}

int sdr_server_submit(sdr_server* s, const sdr_scene_desc* scene, uint64_t* ticket) {
    if (!s || !ticket) return invalid("null argument");
    std::string why;
    if (!valid_scene(scene, why)) return invalid(why);
    auto r = std::make_unique<Request>();
    r->scene = std::make_unique<SceneCopy>(*scene);
    r->bytes = footprint(*scene);
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return invalid("server is shutting down");
    r->id = s->next_id++;
    *ticket = r->id;
    s->stats.submitted += 1;
    if (r->bytes > s->budget) {  // can never be admitted
        r->state = SDR_REQ_FAILED;
        r->result.status = SDR_ERR_CAPACITY;
        r->result.error = "scene footprint " + std::to_string(r->bytes) + " bytes exceeds the server budget";
        r->scene.reset();
        s->stats.failed += 1;
    } else {
        s->pending.push_back(r.get());
        s->cv_admit.notify_all();
    }
    s->requests.emplace(r->id, std::move(r));
    return SDR_OK;
}

int sdr_server_poll(sdr_server* s, uint64_t ticket, int32_t* state, sdr_summary* summary_or_null,
                    double* seconds_or_null, char* error, size_t error_cap) {
    if (!s || !state) return invalid("null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return invalid("unknown ticket");
    const Request& r = *it->second;
    *state = r.state;
    if (r.state == SDR_REQ_DONE) {
        if (summary_or_null) *summary_or_null = r.result.summary;
        if (seconds_or_null) *seconds_or_null = r.latency;
    }
    if (r.state == SDR_REQ_FAILED) copy_error(r.result.error, error, error_cap);
    return SDR_OK;
}

int sdr_server_get_stats(sdr_server* s, sdr_server_stats* out) {
    if (!s || !out) return invalid("null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    return SDR_OK;
}

int sdr_server_destroy(sdr_server* s) {
    if (!s) return SDR_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_admit.notify_all();
    s->cv_work.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    s->cv_work.notify_all();  // the queue is drained: idle workers leave
    for (auto& t : s->workers)
        if (t.joinable()) t.join();
    delete s;
    return SDR_OK;
}

}  // extern "C"
