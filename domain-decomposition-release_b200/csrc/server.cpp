// server.cpp -- a request server over libjv contexts (jv_server_* in jv/jv.h).
//
// A request is one shot of forward modelling or RTM on its own model and
// grid.  The server keeps a queue of requests and `slots` worker threads;
// a worker takes the first queued request whose device footprint
// (footprint_bytes) fits the memory still free under the server's budget,
// runs it on a context of its own (own stream, own device memory from the
// stream-ordered allocator), copies the results to the request's host
// buffers and releases the context.  Requests admitted together run
// concurrently on the GPU.  Each request's result does not depend on what
// else runs: a context's kernels touch only its own memory.  Every wait here
// is a host wait, bounded where the caller asks for a time limit.
//
// The reference has no counterpart: its driver runs the shots of one job
// in a loop (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:18-135,
// RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_rtm3d_model_mpi).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "jv/jv.h"

namespace {

using clk = std::chrono::steady_clock;

// how many of the latest latencies the p50/p99 statistics are taken over
constexpr size_t kLatencyWindow = 1 << 16;

struct Req {
    jv_request r{};
    size_t bytes = 0;
    int state = JV_JOB_QUEUED;
    jv_status result = JV_OK;
    std::string msg;
    clk::time_point t_submit, t_done;
};

jv_status fail(jv_status c, const std::string &m) {
    jv::set_last_error(m);
    return c;
}

}  // namespace

struct jv_server {
    int device = 0;
    size_t budget = 0, in_use = 0;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<long long> queue;
    std::map<long long, Req> reqs;
    long long next_id = 1;
    int running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    std::vector<double> latencies_ms;
    long long n_completed = 0, n_failed = 0, n_cancelled = 0;
    // the device's stream-ordered pool keeps up to the budget cached while
    // the server is open (contexts of later requests reuse it instead of
    // mapping fresh memory); the previous threshold is put back at close
    cudaMemPool_t pool = nullptr;
    uint64_t pool_threshold_before = 0;
};

namespace {

// one request on a context of its own
jv_status run_request(int device, const jv_request &q) {
    jv_options o;
    jv_options_default(&o);
    o.device = device;
    o.rec_width = q.rec_width > 0 ? q.rec_width : 1;
    o.precision = q.precision;
    jv_ctx *c = nullptr;
    jv_status st = jv_create(&q.grid, q.vp, q.vs, q.rho, q.dt, q.fm, q.nt, &o, &c);
    if (st != JV_OK) return st;
    st = jv_set_geometry(c, 1, q.shot_xyz, q.n_recv, q.recv_xyz);
    if (st == JV_OK) {
        if (q.kind == JV_JOB_FORWARD) {
            st = jv_forward(c, 0, q.out[0], q.out[1], q.out[2]);
        } else {
            // without observed traces the request models its own, which
            // stay on the device
            if (!q.obs[0] && !q.obs[1] && !q.obs[2])
                st = jv::rtm_self_modelled(c, 0);
            else
                st = jv_rtm_shot(c, 0, q.obs[0], q.obs[1], q.obs[2]);
            for (int k = 0; k < 5 && st == JV_OK; k++)
                if (q.image[k]) st = jv_image_get(c, k, q.image[k]);
        }
    }
    const std::string msg = st == JV_OK ? std::string() : jv_last_error();
    jv_close(c);
    if (st != JV_OK) jv::set_last_error(msg);
    return st;
}

void worker_main(jv_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        long long id = 0;
        jv_request q{};
        {
            std::unique_lock<std::mutex> l(s->mu);
            // the first queued request that fits the memory still free
            auto pick = [&]() -> bool {
                for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
                    const Req &r = s->reqs[*it];
                    if (s->in_use + r.bytes <= s->budget) {
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
            s->in_use += r.bytes;
            s->running++;
            q = r.r;
        }
        const jv_status st = run_request(s->device, q);
        const std::string msg = st == JV_OK ? std::string() : jv_last_error();
        {
            std::lock_guard<std::mutex> l(s->mu);
            Req &r = s->reqs[id];
            r.state = JV_JOB_DONE;
            r.result = st;
            r.msg = msg;
            r.t_done = clk::now();
            s->in_use -= r.bytes;
            s->running--;
            if (st == JV_OK) {
                // the latency record keeps the most recent requests only
                if (s->latencies_ms.size() >= kLatencyWindow)
                    s->latencies_ms.erase(s->latencies_ms.begin(), s->latencies_ms.begin() + kLatencyWindow / 2);
                s->latencies_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
                s->n_completed++;
            } else {
                s->n_failed++;
            }
        }
        s->done_cv.notify_all();
        s->cv.notify_all();  // memory came free: another request may fit now
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
    if (cudaDeviceGetDefaultMemPool(&s->pool, device) == cudaSuccess &&
        cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &s->pool_threshold_before) == cudaSuccess) {
        uint64_t keep = budget;
        if (cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) s->pool = nullptr;
    } else {
        s->pool = nullptr;
        cudaGetLastError();
    }
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
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(JV_EINVAL, "no such request");
    auto ended = [&] { return it->second.state == JV_JOB_DONE || it->second.state == JV_JOB_CANCELLED; };
    if (timeout_s < 0) {
        s->done_cv.wait(l, ended);
    } else if (!s->done_cv.wait_for(l, std::chrono::duration<double>(timeout_s), ended)) {
        jv::set_last_error(it->second.state == JV_JOB_RUNNING ? "request still running" : "request still queued");
        return JV_ETIMEOUT;
    }
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
    if (s->pool) {
        cudaSetDevice(s->device);
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &s->pool_threshold_before);
        cudaMemPoolTrimTo(s->pool, 0);  // hand the cached memory back
    }
    delete s;
    return JV_OK;
}

}  // extern "C"
