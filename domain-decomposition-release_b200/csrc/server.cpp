// server.cpp -- a request server over libjv contexts (jv_server_* in jv/jv.h).
//
// A request is one shot of forward modelling or RTM on its own model and
// grid.  The server keeps a queue of requests and `slots` worker threads;
// a worker takes the first queued request that it can place: one for which
// an idle context of the same problem shape is pooled, or whose device
// footprint (footprint_bytes) fits the memory still free under the server's
// budget once idle pooled contexts are released, least recently used first.
// The request runs on that context (own stream, own device memory from the
// stream-ordered allocator); the results go to the request's host buffers
// and the context goes back to the pool.
//
// A pooled context keeps its buffers, tensor maps and captured time-loop
// graphs; the next request of its shape only uploads its model
// (jv_set_model), geometry and a cleared image stack.  Requests admitted
// together run concurrently on the GPU.  Each request's result does not
// depend on what else runs, nor on whether its context is new or pooled:
// every shot starts from cleared wavefields, memory variables and shot
// images, and a context's kernels touch only its own memory.  Every wait
// here is a host wait, bounded where the caller asks for a time limit.
//
// The reference has no counterpart: its driver runs the shots of one job
// in a loop (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:18-135,
// RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_rtm3d_model_mpi).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "engine.hpp"
#include "jv/jv.h"

namespace {

using clk = std::chrono::steady_clock;

// how many of the latest latencies the p50/p99 statistics are taken over
constexpr size_t kLatencyWindow = 1 << 16;
// finished requests the server still answers jv_server_poll/wait for; the
// oldest finished records beyond this are forgotten
constexpr size_t kFinishedKept = 1 << 16;

// what a context is created for: requests with equal keys share contexts
struct PoolKey {
    int nx, ny, nz, pml;
    float dx, dy, dz, dt, fm;
    int nt, rec_width, precision, kind, n_recv;
    auto tie() const {
        return std::tie(nx, ny, nz, pml, dx, dy, dz, dt, fm, nt, rec_width, precision, kind, n_recv);
    }
    bool operator==(const PoolKey &o) const { return tie() == o.tie(); }
};

PoolKey key_of(const jv_request &q) {
    return PoolKey{q.grid.nx, q.grid.ny, q.grid.nz, q.grid.pml, q.grid.dx, q.grid.dy, q.grid.dz, q.dt, q.fm,
                   q.nt, q.rec_width > 0 ? q.rec_width : 1, q.precision, q.kind, q.n_recv};
}

struct Req {
    jv_request r{};
    size_t bytes = 0;
    int state = JV_JOB_QUEUED;
    jv_status result = JV_OK;
    std::string msg;
    clk::time_point t_submit, t_done;
};

struct Idle {
    PoolKey key;
    jv_ctx *ctx;
    size_t bytes;
};

jv_status fail(jv_status c, const std::string &m) {
    jv::set_last_error(m);
    return c;
}

// The device's stream-ordered pool keeps up to the largest open server's
// budget cached while any server on that device is open (transient
// allocations of requests reuse it instead of mapping fresh memory).  The
// first server on a device records the threshold it found; the last one to
// close puts it back and trims the pool down to it.
struct PoolThreshold {
    int servers = 0;
    uint64_t before = 0, kept = 0;
};
std::mutex g_thr_mu;
std::map<int, PoolThreshold> g_thr;

void pool_threshold_open(int device, uint64_t budget) {
    std::lock_guard<std::mutex> l(g_thr_mu);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    PoolThreshold &t = g_thr[device];
    if (t.servers == 0) {
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &t.before) != cudaSuccess) {
            cudaGetLastError();
            g_thr.erase(device);
            return;
        }
        t.kept = t.before;
    }
    t.servers++;
    if (budget > t.kept) {
        t.kept = budget;
        if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &t.kept) != cudaSuccess)
            cudaGetLastError();
    }
}

void pool_threshold_close(int device) {
    std::lock_guard<std::mutex> l(g_thr_mu);
    auto it = g_thr.find(device);
    if (it == g_thr.end()) return;
    if (--it->second.servers > 0) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t before = it->second.before;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &before);
        cudaMemPoolTrimTo(pool, (size_t)before);
    }
    cudaGetLastError();
    g_thr.erase(it);
}

}  // namespace

struct jv_server {
    int device = 0;
    size_t budget = 0;
    size_t in_use = 0;  // footprints of running requests and of pooled idle contexts
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<long long> queue;
    std::map<long long, Req> reqs;
    std::deque<long long> finished;  // ids in the order they ended
    long long next_id = 1;
    int running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<double> latencies_ms;
    long long n_completed = 0, n_failed = 0, n_cancelled = 0, n_reused = 0;
    double device_ms = 0.0;  // device time of the completed requests' propagations
    std::list<Idle> idle;  // pooled contexts, most recently used first
    bool threshold_set = false;
};

namespace {

// marks a request ended (under s->mu) and forgets the oldest ended ones
void record_end(jv_server *s, long long id) {
    s->finished.push_back(id);
    while (s->finished.size() > kFinishedKept) {
        s->reqs.erase(s->finished.front());
        s->finished.pop_front();
    }
}

// one request on `c`: a pooled context of its shape, or (c == NULL) a new one
jv_status run_request(int device, const jv_request &q, jv_ctx **c) {
    jv_status st;
    if (*c) {
        st = jv_set_model(*c, q.vp, q.vs, q.rho);
        if (st == JV_OK) st = jv_image_reset(*c);
    } else {
        jv_options o;
        jv_options_default(&o);
        o.device = device;
        o.rec_width = q.rec_width > 0 ? q.rec_width : 1;
        o.precision = q.precision;
        st = jv_create(&q.grid, q.vp, q.vs, q.rho, q.dt, q.fm, q.nt, &o, c);
    }
    if (st != JV_OK) return st;
    st = jv_set_geometry(*c, 1, q.shot_xyz, q.n_recv, q.recv_xyz);
    if (st == JV_OK) {
        if (q.kind == JV_JOB_FORWARD) {
            st = jv_forward(*c, 0, q.out[0], q.out[1], q.out[2]);
        } else {
            // without observed traces the request models its own, which
            // stay on the device
            if (!q.obs[0] && !q.obs[1] && !q.obs[2])
                st = jv::rtm_self_modelled(*c, 0);
            else
                st = jv_rtm_shot(*c, 0, q.obs[0], q.obs[1], q.obs[2]);
            for (int k = 0; k < 5 && st == JV_OK; k++)
                if (q.image[k]) st = jv_image_get(*c, k, q.image[k]);
        }
    }
    return st;
}

void worker_main(jv_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        long long id = 0;
        jv_request q{};
        jv_ctx *ctx = nullptr;
        size_t bytes = 0;
        std::vector<jv_ctx *> evict;
        {
            std::unique_lock<std::mutex> l(s->mu);
            // The first queued request that can be placed: on a pooled idle
            // context of its shape, or on a new context whose footprint fits
            // the budget once idle contexts (least recently used first) are
            // released.
            auto pick = [&]() -> bool {
                size_t idle_bytes = 0;
                for (const Idle &d : s->idle) idle_bytes += d.bytes;
                for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
                    const Req &r = s->reqs[*it];
                    const PoolKey k = key_of(r.r);
                    for (auto d = s->idle.begin(); d != s->idle.end(); ++d)
                        if (d->key == k) {
                            ctx = d->ctx;
                            bytes = d->bytes;
                            s->idle.erase(d);
                            id = *it;
                            s->queue.erase(it);
                            s->n_reused++;
                            return true;
                        }
                    if (s->in_use - idle_bytes + r.bytes <= s->budget) {
                        while (s->in_use + r.bytes > s->budget && !s->idle.empty()) {
                            evict.push_back(s->idle.back().ctx);
                            s->in_use -= s->idle.back().bytes;
                            s->idle.pop_back();
                        }
                        bytes = r.bytes;
                        s->in_use += bytes;
                        id = *it;
                        s->queue.erase(it);
                        return true;
                    }
                }
                return false;
            };
            s->cv.wait(l, [&] { return s->stop || pick(); });
            if (id == 0) return;  // stop requested
            Req &r = s->reqs[id];
            r.state = JV_JOB_RUNNING;
            s->running++;
            q = r.r;
        }
        for (jv_ctx *c : evict) jv_close(c);  // their memory returns before the new context allocates
        jv_status st = run_request(s->device, q, &ctx);
        const std::string msg = st == JV_OK ? std::string() : jv_last_error();
        double dev_ms = 0.0;
        if (st == JV_OK) jv_last_timing(ctx, &dev_ms);
        if (st != JV_OK && ctx) {
            jv_close(ctx);  // a failed context is not pooled
            ctx = nullptr;
        }
        {
            std::lock_guard<std::mutex> l(s->mu);
            Req &r = s->reqs[id];
            r.state = JV_JOB_DONE;
            r.result = st;
            r.msg = msg;
            r.t_done = clk::now();
            if (ctx && !s->stop) {
                s->idle.push_front(Idle{key_of(q), ctx, bytes});
                ctx = nullptr;
            } else {
                s->in_use -= bytes;
            }
            s->running--;
            if (st == JV_OK) {
                // the latency record keeps the most recent requests only
                if (s->latencies_ms.size() >= kLatencyWindow)
                    s->latencies_ms.erase(s->latencies_ms.begin(), s->latencies_ms.begin() + kLatencyWindow / 2);
                s->latencies_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
                s->n_completed++;
                s->device_ms += dev_ms;
            } else {
                s->n_failed++;
            }
            record_end(s, id);
        }
        if (ctx) jv_close(ctx);  // the server is closing
        s->done_cv.notify_all();
        s->cv.notify_all();  // a context or memory came free: another request may be placed now
    }
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = p * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

jv_status jv_footprint(const jv_grid *grid, int nt, int rec_width, int kind, int n_recv, size_t *bytes) {
    if (!grid || !bytes) return fail(JV_EINVAL, "jv_footprint: NULL argument");
    if (grid->nx < 8 || grid->ny < 8 || grid->nz < 8 || grid->pml < 4 || nt < 1 || n_recv < 0)
        return fail(JV_EINVAL, "jv_footprint: bad problem");
    // the context's trace buffer: three components of every receiver
    *bytes = jv::footprint_bytes(*grid, nt, rec_width > 0 ? rec_width : 1, kind == JV_JOB_RTM, JV_FP32) +
             3 * (size_t)n_recv * (size_t)nt * sizeof(float);
    jv::set_last_error("");
    return JV_OK;
}

jv_status jv_server_create(int device, int slots, size_t hbm_budget, jv_server **out) {
    if (!out) return fail(JV_EINVAL, "jv_server_create: NULL argument");
    *out = nullptr;
    if (slots < 1 || slots > 64) return fail(JV_EINVAL, "slots must be in 1..64");
    size_t budget = hbm_budget;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        cudaSetDevice(device);
        cudaError_t e = cudaMemGetInfo(&fr, &tot);
        if (e != cudaSuccess) return fail(JV_ECUDA, std::string("cudaMemGetInfo: ") + cudaGetErrorString(e));
        budget = fr / 10 * 9;
    }
    jv_server *s = new jv_server();
    s->device = device;
    s->budget = budget;
    cudaSetDevice(device);
    pool_threshold_open(device, budget);
    s->threshold_set = true;
    for (int k = 0; k < slots; k++) s->workers.emplace_back(worker_main, s);
    *out = s;
    jv::set_last_error("");
    return JV_OK;
}

jv_status jv_server_submit(jv_server *s, const jv_request *r, long long *id) {
    if (!s || !r || !id) return fail(JV_EINVAL, "jv_server_submit: NULL argument");
    if (r->kind != JV_JOB_FORWARD && r->kind != JV_JOB_RTM) return fail(JV_EINVAL, "unknown request kind");
    if (!r->vp || !r->vs || !r->rho || (r->n_recv > 0 && !r->recv_xyz) || r->n_recv < 0)
        return fail(JV_EINVAL, "request model or receivers missing");
    if (r->precision != JV_FP32 && r->precision != JV_BF16 && r->precision != JV_FP16)
        return fail(JV_EINVAL, "request precision must be JV_FP32, JV_BF16 or JV_FP16");
    size_t bytes = 0;
    jv_status st = jv_footprint(&r->grid, r->nt, r->rec_width, r->kind, r->n_recv, &bytes);
    if (st != JV_OK) return st;
    if (r->precision != JV_FP32)  // a 16-bit store: the footprint with 2-byte records
        bytes = bytes - jv::footprint_bytes(r->grid, r->nt, r->rec_width > 0 ? r->rec_width : 1,
                                            r->kind == JV_JOB_RTM, JV_FP32) +
                jv::footprint_bytes(r->grid, r->nt, r->rec_width > 0 ? r->rec_width : 1, r->kind == JV_JOB_RTM,
                                    r->precision);
    std::lock_guard<std::mutex> l(s->mu);
    if (bytes > s->budget)
        return fail(JV_ENOMEM, "request needs about " + std::to_string(bytes >> 20) + " MiB, the server's budget is " +
                                   std::to_string(s->budget >> 20) + " MiB");
    if (s->stop) return fail(JV_ESTATE, "server is closing");
    *id = s->next_id++;
    Req q;
    q.r = *r;
    q.bytes = bytes;
    q.t_submit = clk::now();
    s->reqs[*id] = q;
    s->queue.push_back(*id);
    s->cv.notify_all();
    jv::set_last_error("");
    return JV_OK;
}

jv_status jv_server_poll(jv_server *s, long long id, int *state, jv_status *result) {
    if (!s || !state) return fail(JV_EINVAL, "jv_server_poll: NULL argument");
    std::lock_guard<std::mutex> l(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(JV_EINVAL, "no such request");
    *state = it->second.state;
    if (result) *result = it->second.result;
    jv::set_last_error(it->second.msg);
    return JV_OK;
}

jv_status jv_server_wait(jv_server *s, long long id, double timeout_s, jv_status *result) {
    if (!s) return fail(JV_EINVAL, "jv_server_wait: NULL server");
    std::unique_lock<std::mutex> l(s->mu);
    if (s->reqs.find(id) == s->reqs.end()) return fail(JV_EINVAL, "no such request");
    // looked up again on every wake: records of ended requests may be dropped meanwhile
    auto ended = [&] {
        auto it = s->reqs.find(id);
        return it == s->reqs.end() || it->second.state == JV_JOB_DONE || it->second.state == JV_JOB_CANCELLED;
    };
    if (timeout_s < 0) {
        s->done_cv.wait(l, ended);
    } else if (!s->done_cv.wait_for(l, std::chrono::duration<double>(timeout_s), ended)) {
        auto it = s->reqs.find(id);
        jv::set_last_error(it->second.state == JV_JOB_RUNNING ? "request still running" : "request still queued");
        return JV_ETIMEOUT;
    }
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(JV_EINVAL, "request ended and its record was dropped");
    if (result) *result = it->second.result;
    jv::set_last_error(it->second.msg);
    return JV_OK;
}

jv_status jv_server_cancel(jv_server *s, long long id) {
    if (!s) return fail(JV_EINVAL, "jv_server_cancel: NULL server");
    {
        std::lock_guard<std::mutex> l(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return fail(JV_EINVAL, "no such request");
        if (it->second.state != JV_JOB_QUEUED) return fail(JV_ESTATE, "request has already started");
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), id));
        it->second.state = JV_JOB_CANCELLED;
        it->second.result = JV_ECANCELED;
        it->second.msg = "cancelled before it started";
        s->n_cancelled++;
        record_end(s, id);
    }
    s->done_cv.notify_all();
    jv::set_last_error("");
    return JV_OK;
}

jv_status jv_server_get_stats(jv_server *s, jv_server_stats *out) {
    if (!s || !out) return fail(JV_EINVAL, "jv_server_get_stats: NULL argument");
    std::lock_guard<std::mutex> l(s->mu);
    out->submitted = s->next_id - 1;
    out->completed = s->n_completed;
    out->failed = s->n_failed;
    out->cancelled = s->n_cancelled;
    out->running = s->running;
    out->queued = (long long)s->queue.size();
    out->p50_ms = percentile(s->latencies_ms, 0.50);
    out->p99_ms = percentile(s->latencies_ms, 0.99);
    double sum = 0.0;
    for (double v : s->latencies_ms) sum += v;
    out->mean_ms = s->latencies_ms.empty() ? 0.0 : sum / (double)s->latencies_ms.size();
    out->bytes_in_use = s->in_use;
    out->reused = s->n_reused;
    out->pooled = (long long)s->idle.size();
    out->device_ms = s->device_ms;
    out->budget = s->budget;
    jv::set_last_error("");
    return JV_OK;
}

jv_status jv_server_close(jv_server *s) {
    if (!s) return JV_OK;
    {
        std::lock_guard<std::mutex> l(s->mu);
        s->stop = true;
        for (long long id : s->queue) {
            s->reqs[id].state = JV_JOB_CANCELLED;
            s->reqs[id].result = JV_ECANCELED;
            s->reqs[id].msg = "server closed";
            s->n_cancelled++;
        }
        s->queue.clear();
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
    for (std::thread &t : s->workers)
        if (t.joinable()) t.join();
    for (Idle &d : s->idle) jv_close(d.ctx);
    s->idle.clear();
    if (s->threshold_set) pool_threshold_close(s->device);
    delete s;
    return JV_OK;
}

}  // extern "C"
