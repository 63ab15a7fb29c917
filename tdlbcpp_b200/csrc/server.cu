// Serving form: a request loop over resident, continuously batched tanks.
//
// Callers submit tank-solve requests (tank size, impeller tip speed,
// Reynolds number, step count, storage precision) from any thread. Two
// server threads share the GPU work:
//   * admission (helper thread) -- requests are taken in arrival order while
//     a slot is free and the tank's device bytes (tdlb_lattice_bytes) fit
//     both the free HBM (less a reserve) and the server's budget; an
//     admitted tank is built on its own stream, gets its Rushton turbine, is
//     initialised and forced once (main.cpp:305), all while the resident
//     tanks keep stepping;
//   * stepping (worker thread) -- between two chunks the built tanks join
//     the resident batch of their precision and streaming scheme
//     (tdlb_batch_adopt); all resident tanks advance together in chunks:
//     every batch runs the same number of steps (the smallest remaining
//     count, capped by chunk_steps) through tdlb_batch_run, the batches of
//     different precisions on their own streams at the same time;
//   * retirement -- a finished tank leaves its batch (tdlb_batch_detach) and
//     the helper copies out its FP64 diagnostics (mass, momentum, impeller
//     force and torque, power number) and, if asked, its density and
//     velocity fields, and frees its memory, while the next chunk runs.
// Requests that arrive while others run join at a chunk boundary, so their
// work overlaps with the tanks already on the GPU.
// A tank's arithmetic does not depend on its batch neighbours: its result
// equals the same request run alone.
#include "tdlb_b200.h"
#include "tdlb_geometry.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Active {
    tdlb_request req;
    tdlb_batch batch;
    tdlb_handle h;
    long long remaining;
    double t_submit, t_admit;
    long long bytes;
    double D, omega;      // impeller diameter and angular speed (rad per step)
};

struct Pending {
    tdlb_request req;
    double t_submit;
};

}  // namespace

struct tdlb_server_s {
    int device = 0;
    long long budget = 0;        // bytes (0: free HBM only)
    long long reserve = 1LL << 30;
    int max_active = 64;
    int chunk = 100;
    float alpha = 0.97f, beta = 1.9f;
    Clock::time_point t0;

    std::mutex mu;
    std::condition_variable cv, idle_cv;
    std::deque<Pending> queue;
    std::vector<tdlb_result> done;
    bool stop = false;
    std::string err = "no error";
    long long submitted = 0, completed = 0;

    // shared with the helper thread (under mu)
    std::thread helper;
    std::vector<Active> ready;      // built tanks waiting to join a batch (own streams)
    std::vector<Active> finished;   // finished tanks detached from their batches
    int holding = 0;                // tanks holding device memory: building, ready, resident, finished

    // stepping-thread-owned
    std::thread worker;
    std::map<int, tdlb_batch> batches;   // key: storage * 2 + streaming
    std::vector<Active> active;
    long long bytes_in_use = 0;
    double lattice_updates = 0, busy_s = 0;
    long long chunks = 0, admitted = 0;
    int n_active_snapshot = 0;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// FlowParams::calcNuAndRe_m (FlowParams.hpp:65-70) in the reference's float
// arithmetic, with the blade outer radius of the request's turbine.
double nu_of(double reynolds, double tip, int radius) {
    const float Re_m = (float)((float)reynolds * M_PI / 2.0);
    return (double)(float)((float)tip * (float)radius / Re_m);
}

tdlb_rushton spec_of(const tdlb_request& r) {
    tdlb_rushton s{};
    s.x = r.x;
    s.y = r.y;
    s.z = r.z;
    s.tip_speed = r.tip_speed;
    return s;
}

tdlb_config config_of(const tdlb_request& r, int radius) {
    tdlb_config c{};
    c.x = r.x;
    c.y = r.y;
    c.z = r.z;
    c.streaming = r.streaming;
    c.storage = r.storage;
    c.initialRho = 1.0;
    c.nu = nu_of(r.reynolds, r.tip_speed, radius);
    c.cs0 = 0.1;
    c.g3 = 0.8;
    c.alpha = 0.97;
    c.beta = 1.9;
    c.useLES = r.les;
    return c;
}

long long need_of(const tdlb_request& r) {
    tdlb_config c = config_of(r, 1);
    int64_t b = 0;
    if (tdlb_lattice_bytes(&c, &b) != TDLB_OK) return -1;
    return (long long)b;
}

void note(tdlb_server_s* s, const std::string& msg) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->err = msg;
}

void push_result(tdlb_server_s* s, const tdlb_result& res) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->done.push_back(res);
    s->completed++;
    s->idle_cv.notify_all();
}

tdlb_result failed(const tdlb_request& r, int code, double t_submit, double now) {
    tdlb_result res{};
    res.id = r.id;
    res.status = code;
    res.t_submit = t_submit;
    res.t_admit = now;
    res.t_done = now;
    return res;
}

tdlb_batch batch_for(tdlb_server_s* s, const tdlb_request& r) {
    const int key = r.storage * 2 + r.streaming;
    auto it = s->batches.find(key);
    if (it != s->batches.end()) return it->second;
    tdlb_batch b = nullptr;
    const int rc = tdlb_batch_create_empty(s->device, r.streaming, r.storage, &b);
    if (rc != TDLB_OK) return nullptr;
    s->batches[key] = b;
    return b;
}

int index_in(tdlb_batch b, tdlb_handle h) {
    int n = 0;
    tdlb_batch_size(b, &n);
    for (int t = 0; t < n; t++) {
        tdlb_handle x = nullptr;
        tdlb_batch_tank(b, t, &x);
        if (x == h) return t;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// Helper thread: admission and retirement, off the stepping thread, so that
// building a tank (allocation, geometry, marker schedule: tens of ms for a
// 256^3 tank) and freeing one never leave the GPU idle between chunks.
// ---------------------------------------------------------------------------

// Takes the next request if a slot is free and its bytes fit: 1 taken (slot
// and bytes reserved), 0 nothing to take now, 2 the request failed (result
// pushed).
int take_request(tdlb_server_s* s, Pending& p, long long& need) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->queue.empty() || s->stop) return 0;
    if (s->holding >= s->max_active) return 0;
    p = s->queue.front();
    need = need_of(p.req);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    long long avail = (long long)free_b - s->reserve;
    if (s->budget > 0) avail = std::min(avail, s->budget - s->bytes_in_use);
    if (need >= 0 && need <= avail) {
        s->queue.pop_front();
        s->holding++;
        s->bytes_in_use += need;
        return 1;
    }
    if (s->holding > 0 && need >= 0) return 0;   // wait for memory to free up
    s->queue.pop_front();
    s->done.push_back(failed(p.req, need < 0 ? TDLB_EINVAL : TDLB_ENOMEM, p.t_submit, s->now()));
    s->completed++;
    s->idle_cv.notify_all();
    return 2;
}

// Gives back a slot and its bytes.
void release_slot(tdlb_server_s* s, long long bytes) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->holding--;
    s->bytes_in_use -= bytes;
    s->cv.notify_all();
}

// Builds a taken request's tank on its own stream: created, impeller
// attached, initialised and forced once (main.cpp:305), then handed to the
// stepping thread, which adopts it into its batch between two chunks.
void build(tdlb_server_s* s, const Pending& p, long long need) {
    const tdlb_request& r = p.req;
    const tdlb_rushton spec = spec_of(r);
    const int radius = tdlb_rushton_blade_outer_radius(&spec);
    const tdlb_config c = config_of(r, radius < 1 ? 1 : radius);
    tdlb_handle h = nullptr;
    int rc = tdlb_create_config(&c, s->device, &h);
    const double d1 = tdlb_rushton_impeller_increment(&spec, 1);
    if (rc == TDLB_OK) rc = tdlb_attach_rushton(h, &spec, d1, d1, d1);
    if (rc == TDLB_OK) rc = tdlb_initialise(h, 1.0f);
    if (rc == TDLB_OK) rc = tdlb_forcing_resident(h, s->alpha, s->beta);
    if (rc == TDLB_OK) rc = tdlb_synchronize(h);
    if (rc != TDLB_OK) {
        note(s, std::string("tank setup: ") + tdlb_last_error(h));
        if (h) tdlb_destroy(h);
        release_slot(s, need);
        push_result(s, failed(r, rc, p.t_submit, s->now()));
        return;
    }
    Active a{};
    a.req = r;
    a.h = h;
    a.remaining = r.steps;
    a.t_submit = p.t_submit;
    a.t_admit = s->now();
    a.bytes = need;
    const tdlb::RushtonGeom G = tdlb::RushtonGeom::from(spec);
    a.D = G.D;
    a.omega = G.increment(1000000000ULL);
    std::lock_guard<std::mutex> lk(s->mu);
    s->ready.push_back(a);
    s->admitted++;
    s->cv.notify_all();
}

// A finished tank, detached from its batch and on its own stream again: its
// FP64 diagnostics and optional fields are read, its memory freed.
void retire(tdlb_server_s* s, Active& a) {
    tdlb_result res{};
    res.id = a.req.id;
    res.t_submit = a.t_submit;
    res.t_admit = a.t_admit;
    res.cells = a.req.x * a.req.y * a.req.z;
    res.steps = a.req.steps;
    double load[5] = {0, 0, 0, 0, 0};
    double red[4] = {0, 0, 0, 0};
    int rc = tdlb_impeller_load(a.h, load);
    if (rc == TDLB_OK) rc = tdlb_reduce_fp64(a.h, red);
    if (rc == TDLB_OK && (a.req.out_rho || a.req.out_ux || a.req.out_uy || a.req.out_uz))
        rc = tdlb_read_velocity_density(a.h, a.req.out_rho, a.req.out_ux, a.req.out_uy, a.req.out_uz);
    if (rc != TDLB_OK) note(s, std::string("retirement: ") + tdlb_last_error(a.h));
    res.status = rc;
    res.mass = red[0];
    for (int c = 0; c < 3; c++) {
        res.momentum[c] = red[1 + c];
        res.force[c] = load[c];
    }
    res.torque = load[3];
    // power number P / (rho N^3 D^5), P = torque * omega, N = omega / (2 pi)
    const double N = a.omega / (2.0 * M_PI);
    res.power_number = N > 0 ? std::fabs(res.torque * a.omega) / (N * N * N * std::pow(a.D, 5)) : 0.0;
    tdlb_destroy(a.h);
    a.h = nullptr;
    release_slot(s, a.bytes);
    res.t_done = s->now();
    push_result(s, res);
}

void helper_loop(tdlb_server_s* s) {
    cudaSetDevice(s->device);
    for (;;) {
        std::vector<Active> fin;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            fin.swap(s->finished);
        }
        for (Active& a : fin) retire(s, a);
        Pending p;
        long long need = 0;
        const int took = take_request(s, p, need);
        if (took == 1) build(s, p, need);
        if (took != 0 || !fin.empty()) continue;
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->stop && s->finished.empty()) break;
        // wake for finished tanks, new requests or freed slots
        const long long sub0 = s->submitted;
        const int hold0 = s->holding;
        s->cv.wait_for(lk, std::chrono::milliseconds(20), [&] {
            return s->stop || !s->finished.empty() || s->submitted != sub0 || s->holding != hold0;
        });
    }
}

// ---------------------------------------------------------------------------
// Stepping thread.
// ---------------------------------------------------------------------------

// Tanks the helper has built join the batch of their precision and scheme.
void adopt_ready(tdlb_server_s* s) {
    std::vector<Active> rd;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        rd.swap(s->ready);
    }
    for (Active& a : rd) {
        tdlb_batch b = batch_for(s, a.req);
        int idx = -1;
        const int rc = b ? tdlb_batch_adopt(b, a.h, &idx) : TDLB_ECUDA;
        if (rc != TDLB_OK) {
            note(s, std::string("admission: ") + (b ? tdlb_batch_last_error(b) : "no batch"));
            tdlb_destroy(a.h);
            release_slot(s, a.bytes);
            push_result(s, failed(a.req, rc, a.t_submit, s->now()));
            continue;
        }
        a.batch = b;
        s->active.push_back(a);
    }
}

// A resident tank that will not finish: it leaves its batch (destroyed)
// with `code` as its result.
void drop_active(tdlb_server_s* s, size_t k, int code) {
    Active& a = s->active[k];
    tdlb_result res = failed(a.req, code, a.t_submit, s->now());
    res.t_admit = a.t_admit;
    const int idx = index_in(a.batch, a.h);
    if (idx >= 0) tdlb_batch_remove(a.batch, idx);
    release_slot(s, a.bytes);
    s->active.erase(s->active.begin() + (long)k);
    push_result(s, res);
}

void step_chunk(tdlb_server_s* s) {
    long long chunk = s->chunk;
    for (const Active& a : s->active) chunk = std::min(chunk, a.remaining);
    const double t = s->now();
    int rc = TDLB_OK;
    std::string why;
    for (auto& kv : s->batches) {
        int n = 0;
        tdlb_batch_size(kv.second, &n);
        if (n && rc == TDLB_OK) {
            rc = tdlb_batch_run(kv.second, (int)chunk, s->alpha, s->beta);
            if (rc != TDLB_OK) why = tdlb_batch_last_error(kv.second);
        }
    }
    for (auto& kv : s->batches)
        if (tdlb_batch_synchronize(kv.second) != TDLB_OK && rc == TDLB_OK) {
            rc = TDLB_ECUDA;
            why = tdlb_batch_last_error(kv.second);
        }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc != TDLB_OK) s->err = "chunk failed: " + why;
        s->busy_s += s->now() - t;
        s->chunks++;
    }
    if (rc != TDLB_OK) {   // every resident tank fails with the error
        for (size_t k = s->active.size(); k-- > 0;) drop_active(s, k, rc);
        return;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Active& a : s->active) {
            a.remaining -= chunk;
            s->lattice_updates += (double)a.req.x * a.req.y * a.req.z * (double)chunk;
        }
    }
    // finished tanks leave their batches (not destroyed) and go to the
    // helper, which reads and frees them while the next chunk runs
    for (size_t k = s->active.size(); k-- > 0;) {
        Active& a = s->active[k];
        if (a.remaining > 0) continue;
        const int idx = index_in(a.batch, a.h);
        tdlb_handle h = nullptr;
        if (idx < 0 || tdlb_batch_detach(a.batch, idx, &h) != TDLB_OK) {
            drop_active(s, k, TDLB_ECUDA);
            continue;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->finished.push_back(a);
        s->active.erase(s->active.begin() + (long)k);
        s->cv.notify_all();
    }
}

void loop(tdlb_server_s* s) {
    cudaSetDevice(s->device);
    for (;;) {
        adopt_ready(s);
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->n_active_snapshot = (int)s->active.size();
            if (s->stop) break;
            if (s->active.empty()) {
                s->cv.wait_for(lk, std::chrono::milliseconds(20), [&] { return s->stop || !s->ready.empty(); });
                continue;
            }
        }
        step_chunk(s);
    }
    // stopping: resident tanks end unfinished
    for (size_t k = s->active.size(); k-- > 0;) drop_active(s, k, TDLB_ESTATE);
}

thread_local std::string g_server_error = "no error";

}  // namespace

extern "C" {

int tdlb_server_create(int device, int64_t hbm_budget_bytes, int max_active, int chunk_steps, tdlb_server* out) {
    if (!out || max_active < 1 || chunk_steps < 1 || hbm_budget_bytes < 0) {
        g_server_error = "bad arguments";
        return TDLB_EINVAL;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_server_error = "no CUDA device available (this library has no CPU path)";
        return TDLB_ECUDA;
    }
    if (device < 0 || device >= ndev) {
        g_server_error = "device index out of range";
        return TDLB_EINVAL;
    }
    auto* s = new tdlb_server_s();
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    s->chunk = chunk_steps;
    s->t0 = Clock::now();
    try {
        s->worker = std::thread(loop, s);
        s->helper = std::thread(helper_loop, s);
    } catch (const std::exception& e) {
        g_server_error = e.what();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
            s->cv.notify_all();
        }
        if (s->worker.joinable()) s->worker.join();
        delete s;
        return TDLB_EINVAL;
    }
    *out = s;
    return TDLB_OK;
}

const char* tdlb_server_last_error(tdlb_server s) {
    if (!s) return g_server_error.c_str();
    std::lock_guard<std::mutex> lk(s->mu);
    g_server_error = s->err;   // a per-thread copy the caller may read
    return g_server_error.c_str();
}

int tdlb_server_submit(tdlb_server s, const tdlb_request* r) {
    if (!s || !r) return TDLB_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (r->x < 8 || r->y < 8 || r->z < 8 || r->steps < 1 || r->tip_speed <= 0 || r->reynolds <= 0 ||
        r->storage < TDLB_STORAGE_FP32 || r->storage > TDLB_STORAGE_BF16 ||
        (r->streaming != TDLB_STREAMING_SIMPLE && r->streaming != TDLB_STREAMING_ESOTWIST)) {
        s->err = "bad request (sizes >= 8, steps >= 1, tip speed and Re > 0, known storage and streaming)";
        return TDLB_EINVAL;
    }
    if (s->stop) {
        s->err = "server is stopping";
        return TDLB_ESTATE;
    }
    s->queue.push_back(Pending{*r, s->now()});
    s->submitted++;
    s->cv.notify_all();
    return TDLB_OK;
}

int tdlb_server_poll(tdlb_server s, tdlb_result* out, int cap, int* n) {
    if (!s || !n || cap < 0 || (cap > 0 && !out)) return TDLB_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    const int k = std::min(cap, (int)s->done.size());
    std::copy(s->done.begin(), s->done.begin() + k, out);
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return TDLB_OK;
}

int tdlb_server_wait_idle(tdlb_server s, double timeout_s) {
    if (!s) return TDLB_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->idle_cv.wait_for(lk, std::chrono::duration<double>(timeout_s < 0 ? 0 : timeout_s),
                                        [&] { return s->completed >= s->submitted; });
    if (!ok) {
        s->err = "timed out waiting for the submitted requests";
        return TDLB_ESTATE;
    }
    return TDLB_OK;
}

int tdlb_server_get_stats(tdlb_server s, tdlb_server_stats* st) {
    if (!s || !st) return TDLB_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->queued = (int64_t)s->queue.size();
    st->active = s->n_active_snapshot;
    st->admitted = s->admitted;
    st->chunks = s->chunks;
    st->bytes_in_use = s->bytes_in_use;
    st->lattice_updates = s->lattice_updates;
    st->busy_s = s->busy_s;
    st->elapsed_s = s->now();
    return TDLB_OK;
}

int tdlb_server_destroy(tdlb_server s) {
    if (!s) return TDLB_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    if (s->helper.joinable()) s->helper.join();
    cudaSetDevice(s->device);
    // what the threads left: finished tanks are read out, built ones and
    // queued requests end unfinished
    for (Active& a : s->finished) retire(s, a);
    for (Active& a : s->ready) {
        tdlb_destroy(a.h);
        push_result(s, failed(a.req, TDLB_ESTATE, a.t_submit, s->now()));
    }
    while (!s->queue.empty()) {
        push_result(s, failed(s->queue.front().req, TDLB_ESTATE, s->queue.front().t_submit, s->now()));
        s->queue.pop_front();
    }
    for (auto& kv : s->batches) tdlb_batch_destroy(kv.second);
    delete s;
    return TDLB_OK;
}

}  // extern "C"
