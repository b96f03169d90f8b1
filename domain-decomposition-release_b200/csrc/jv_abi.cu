// jv_abi.cu -- the extern "C" boundary of libjv (include/jv/jv.h).
// Every entry point converts the C++ engine's Status into a jv_status and
// keeps the message for jv_last_error(); nothing here aborts.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "jv/jv.h"
#include "project_io.hpp"

// the .fld header is the reference's Frame struct as x86-64 lays it out
static_assert(sizeof(jv_frame) == 72, "jv_frame must match the reference Frame's 72 bytes");

namespace {
thread_local std::string g_err;

jv_status ret(const jv::Status &s) {
    g_err = s.msg;
    return s.code;
}
jv_status fail(jv_status c, const std::string &m) {
    g_err = m;
    return c;
}
}  // namespace

namespace jv {
// lets other translation units of the library report through jv_last_error()
void set_last_error(const std::string &m) { g_err = m; }
}  // namespace jv

// One submitted job and what became of it.
struct JobRec {
    jv_job job{};
    int state = JV_JOB_QUEUED;
    jv_status result = JV_OK;
    std::string msg;
};

struct jv_ctx {
    std::unique_ptr<jv::Engine> eng;
    bool from_project = false;
    jv::ArgFile arg;
    std::vector<float> shots, recvs;
    // device trace buffers for host-pointer calls (the second one lets a
    // batch copy the next shot's traces while the current shot runs)
    float *d_tr[2] = {nullptr, nullptr};
    size_t d_tr_elems[2] = {0, 0};
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_copy[2] = {nullptr, nullptr};
    // job queue, served in submission order by one worker thread
    std::mutex mu;
    std::condition_variable cv;       // the worker waits for jobs / stop
    std::condition_variable done_cv;  // callers wait for jobs to end
    std::deque<long long> queue;
    std::map<long long, JobRec> jobs;
    long long next_id = 1;
    bool running = false, stop = false;
    std::thread worker;

    bool busy() {
        std::lock_guard<std::mutex> l(mu);
        return running || !queue.empty();
    }
    // cancels queued jobs, lets the running one finish, joins the worker
    void shutdown() {
        {
            std::lock_guard<std::mutex> l(mu);
            stop = true;
            for (long long id : queue) {
                jobs[id].state = JV_JOB_CANCELLED;
                jobs[id].result = JV_ECANCELED;
                jobs[id].msg = "context closed";
            }
            queue.clear();
        }
        cv.notify_all();
        done_cv.notify_all();
        if (worker.joinable()) worker.join();
    }
    ~jv_ctx() {
        shutdown();
        if (eng) cudaSetDevice(eng->device());
        for (int q = 0; q < 2; q++) {
            if (d_tr[q]) cudaFreeAsync(d_tr[q], eng->stream());
            if (ev_copy[q]) cudaEventDestroy(ev_copy[q]);
        }
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }
};

static jv_status ensure_traces(jv_ctx *c, size_t elems, int which = 0) {
    if (c->d_tr_elems[which] >= elems) return JV_OK;
    cudaSetDevice(c->eng->device());
    cudaStream_t s = c->eng->stream();
    if (c->d_tr[which]) cudaFreeAsync(c->d_tr[which], s);
    c->d_tr[which] = nullptr;
    c->d_tr_elems[which] = 0;
    if (elems == 0) return JV_OK;
    cudaError_t e = cudaMallocAsync(&c->d_tr[which], elems * sizeof(float), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(JV_ENOMEM, std::string("trace buffer: ") + cudaGetErrorString(e));
    }
    c->d_tr_elems[which] = elems;
    return JV_OK;
}

// calls that use the engine are refused while jobs are queued or running
#define JV_IDLE(c)                                                                           \
    do {                                                                                     \
        if (!(c)) return fail(JV_EINVAL, "NULL context");                                    \
        if ((c)->busy()) return fail(JV_ESTATE, "jobs are queued or running on this context"); \
    } while (0)

// host-pointer forward modelling / migration of one shot (no idle check)
static jv_status forward_host(jv_ctx *c, int shot, float *vx, float *vy, float *vz) {
    const size_t per = (size_t)c->eng->nrec() * c->eng->nt();
    jv_status st = ensure_traces(c, 3 * per);
    if (st != JV_OK) return st;
    float *d = c->d_tr[0];
    st = ret(c->eng->forward(shot, vx ? d : nullptr, vy ? d + per : nullptr, vz ? d + 2 * per : nullptr));
    if (st != JV_OK) return st;
    float *h[3] = {vx, vy, vz};
    for (int q = 0; q < 3; q++)
        if (h[q] && per) {
            cudaError_t e = cudaMemcpyAsync(h[q], d + q * per, per * sizeof(float), cudaMemcpyDeviceToHost,
                                            c->eng->stream());
            if (e != cudaSuccess) return fail(JV_ECUDA, cudaGetErrorString(e));
        }
    cudaError_t e = cudaStreamSynchronize(c->eng->stream());
    if (e != cudaSuccess) return fail(JV_ECUDA, cudaGetErrorString(e));
    return JV_OK;
}

// the copy stream of host-pointer RTM calls and its two events, made once
static jv_status ensure_copy_stream(jv_ctx *c) {
    if (c->copy_stream) return JV_OK;
    cudaSetDevice(c->eng->device());
    cudaError_t e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; b++) e = cudaEventCreateWithFlags(&c->ev_copy[b], cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(JV_ECUDA, std::string("copy stream: ") + cudaGetErrorString(e));
    return JV_OK;
}

// One shot from host traces: they are copied on the copy stream while the
// forward pass runs (it does not read them); the reverse loop waits for the
// copy.  The previous call has finished with the buffer, since every call
// returns after its shot.
static jv_status rtm_host(jv_ctx *c, int shot, const float *ox, const float *oy, const float *oz) {
    const size_t per = (size_t)c->eng->nrec() * c->eng->nt();
    if (per && (!ox || !oy || !oz)) return fail(JV_EINVAL, "observed traces must not be NULL");
    jv_status st = ensure_traces(c, 3 * per);
    if (st == JV_OK) st = ensure_copy_stream(c);
    if (st != JV_OK) return st;
    const float *h[3] = {ox, oy, oz};
    for (int q = 0; q < 3 && per; q++) {
        cudaError_t e = cudaMemcpyAsync(c->d_tr[0] + q * per, h[q], per * sizeof(float), cudaMemcpyHostToDevice,
                                        c->copy_stream);
        if (e != cudaSuccess) return fail(JV_ECUDA, cudaGetErrorString(e));
    }
    cudaError_t e = cudaEventRecord(c->ev_copy[0], c->copy_stream);
    if (e != cudaSuccess) return fail(JV_ECUDA, cudaGetErrorString(e));
    st = ret(c->eng->rtm_shot(shot, c->d_tr[0], c->d_tr[0] + per, c->d_tr[0] + 2 * per, c->ev_copy[0]));
    if (st != JV_OK) cudaStreamSynchronize(c->copy_stream);  // the buffer is free when the call returns
    return st;
}

namespace jv {
jv_status rtm_self_modelled(jv_ctx *c, int shot) {
    JV_IDLE(c);
    const size_t per = (size_t)c->eng->nrec() * c->eng->nt();
    jv_status st = ensure_traces(c, 3 * per);
    if (st != JV_OK) return st;
    float *d = c->d_tr[0];
    st = ret(c->eng->forward(shot, d, d + per, d + 2 * per));
    if (st != JV_OK) return st;
    const double fwd_ms = c->eng->last_ms();
    st = ret(c->eng->rtm_shot(shot, d, d + per, d + 2 * per));
    if (st == JV_OK) c->eng->set_last_ms(fwd_ms + c->eng->last_ms());  // both propagations
    return st;
}
}  // namespace jv

extern "C" {

void jv_options_default(jv_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->device = 0;
    o->rec_width = 1;
    o->precision = JV_FP32;
    o->store_mode = JV_STORE_AUTO;
    o->use_graphs = 1;
    o->graph_steps = 0;
    o->store_budget = 0;
    o->kernel_variant = 4;
    o->zchunk = 0;
    o->autotune = 1;
}

jv_status jv_create(const jv_grid *grid, const float *vp, const float *vs, const float *rho, float dt, float fm,
                    int nt, const jv_options *opt, jv_ctx **out) {
    if (!grid || !out) return fail(JV_EINVAL, "jv_create: NULL argument");
    *out = nullptr;
    jv_options o;
    jv_options_default(&o);
    if (opt) o = *opt;
    jv::Engine *e = nullptr;
    jv::Status s = jv::Engine::create(*grid, vp, vs, rho, dt, fm, nt, o, &e);
    if (!s) return ret(s);
    jv_ctx *c = new jv_ctx();
    c->eng.reset(e);
    *out = c;
    g_err.clear();
    return JV_OK;
}

jv_status jv_open(const char *proj_path, const jv_options *opt, jv_ctx **out) {
    if (!proj_path || !out) return fail(JV_EINVAL, "jv_open: NULL argument");
    *out = nullptr;
    jv::ArgFile a;
    std::string m = jv::read_argfile(proj_path, &a);
    if (!m.empty()) return fail(JV_EIO, m);
    if (a.x_divide_num > 1 || a.y_divide_num > 1 || a.z_divide_num > 1)
        return fail(JV_EINVAL, "x/y/z_divide_num must be 1: the whole model is resident on one GPU");
    jv::GmsModel g;
    m = a.vp_path.empty() ? jv::read_gms(a.model_path, &g) : jv::read_raw_model(a, &g);
    if (!m.empty()) return fail(JV_EIO, m);
    std::vector<float> shots, recvs;
    m = jv::read_points(a.shot_path, &shots);
    if (!m.empty()) return fail(JV_EIO, m);
    m = jv::read_points(a.recv_path, &recvs);
    if (!m.empty()) return fail(JV_EIO, m);
    jv_options o;
    jv_options_default(&o);
    if (opt) o = *opt;
    if (a.rec_width > 0) o.rec_width = a.rec_width;
    if (a.precision == "bf16") o.precision = JV_BF16;
    else if (a.precision == "fp16") o.precision = JV_FP16;
    jv_grid gr{g.nx, g.ny, g.nz, a.pml_num, g.dx, g.dy, g.dz};
    const int nt = jv::ntime(a.T, a.dt);
    jv_ctx *c = nullptr;
    jv_status st = jv_create(&gr, g.params[0].data(), g.params[1].data(), g.params[2].data(), a.dt, a.fm, nt, &o, &c);
    if (st != JV_OK) return st;
    c->from_project = true;
    c->arg = a;
    c->eng->output_path = a.output_path;
    st = jv_set_geometry(c, (int)(shots.size() / 3), shots.data(), (int)(recvs.size() / 3), recvs.data());
    if (st != JV_OK) {
        delete c;
        return st;
    }
    *out = c;
    return JV_OK;
}

jv_status jv_read_argfile(const char *proj_path, jv_argfile *out) {
    if (!proj_path || !out) return fail(JV_EINVAL, "jv_read_argfile: NULL argument");
    jv::ArgFile a;
    std::string m = jv::read_argfile(proj_path, &a);
    if (!m.empty()) return fail(JV_EIO, m);
    std::memset(out, 0, sizeof(*out));
    const std::string *src[4] = {&a.model_path, &a.shot_path, &a.recv_path, &a.output_path};
    char *dst[4] = {out->model_path, out->shot_path, out->rece_path, out->output_path};
    for (int q = 0; q < 4; q++) {
        if (src[q]->size() >= sizeof(out->model_path)) return fail(JV_EINVAL, "path too long: " + *src[q]);
        std::memcpy(dst[q], src[q]->c_str(), src[q]->size() + 1);
    }
    out->is_output = a.is_output ? 1 : 0;
    out->t_snap = a.t_snap;
    out->pml_num = a.pml_num;
    out->fm = a.fm;
    out->dt = a.dt;
    out->T = a.T;
    out->x_divide_num = a.x_divide_num;
    out->y_divide_num = a.y_divide_num;
    out->z_divide_num = a.z_divide_num;
    out->slots_per_node = a.slots_per_node;
    out->rec_width = a.rec_width;
    const std::string *rsrc[3] = {&a.vp_path, &a.vs_path, &a.rho_path};
    char *rdst[3] = {out->vp_path, out->vs_path, out->rho_path};
    for (int q = 0; q < 3; q++) {
        if (rsrc[q]->size() >= sizeof(out->vp_path)) return fail(JV_EINVAL, "path too long: " + *rsrc[q]);
        std::memcpy(rdst[q], rsrc[q]->c_str(), rsrc[q]->size() + 1);
    }
    out->n_rows = a.n_rows;
    out->n_cols = a.n_cols;
    out->n_slices = a.n_slices;
    out->d_rows = a.d_rows;
    out->d_cols = a.d_cols;
    out->d_slices = a.d_slices;
    out->save_fld = a.save_fld ? 1 : 0;
    g_err.clear();
    return JV_OK;
}

void jv_frame_make(uint64_t n_rows, uint32_t n_cols, uint32_t n_slices, float d_rows, float d_cols, float d_slices,
                   float l_rows, float l_cols, float l_slices, jv_frame *f) {
    if (!f) return;
    std::memset(f, 0, sizeof(*f));
    f->n_rows = n_rows;
    f->n_cols = n_cols;
    f->n_slices = n_slices;
    f->n_elem_slice = n_rows * n_cols;
    f->n_elem = n_rows * n_cols * n_slices;
    f->d_rows = d_rows; f->d_cols = d_cols; f->d_slices = d_slices;
    f->l_rows = l_rows; f->l_cols = l_cols; f->l_slices = l_slices;
    // an empty axis has l = r = 0
    if (n_rows > 0) f->r_rows = l_rows + (float)(n_rows - 1) * d_rows; else f->l_rows = 0.f;
    if (n_cols > 0) f->r_cols = l_cols + (float)(n_cols - 1) * d_cols; else f->l_cols = 0.f;
    if (n_slices > 0) f->r_slices = l_slices + (float)(n_slices - 1) * d_slices; else f->l_slices = 0.f;
    // Frame::Type: with a spacing the frame is a line/mesh/grid, else a vec/mat/cube
    const bool spaced = d_rows > 0 || d_cols > 0 || d_slices > 0;
    const bool one_axis = (n_rows == 1 && n_cols == 1) || (n_rows == 1 && n_slices == 1) || (n_cols == 1 && n_slices == 1);
    const bool two_axes = (n_rows > 1 && n_cols > 1 && n_slices == 1) || (n_rows > 1 && n_slices > 1 && n_cols == 1) ||
                          (n_cols > 1 && n_slices > 1 && n_rows == 1);
    const bool three_axes = n_rows > 1 && n_cols > 1 && n_slices > 1;
    if (one_axis) f->type = spaced ? 10 : 1;
    else if (two_axes) f->type = spaced ? 20 : 2;
    else if (three_axes) f->type = spaced ? 30 : 3;
}

jv_status jv_fld_write(const char *path_noext, const jv_frame *f, const float *data) {
    if (!path_noext || !f || (f->n_elem && !data)) return fail(JV_EINVAL, "jv_fld_write: NULL argument");
    const std::string path = std::string(path_noext) + ".fld";
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) return fail(JV_EIO, "cannot create " + path);
    bool ok = std::fwrite(f, sizeof(*f), 1, fp) == 1;
    if (ok && f->n_elem) ok = std::fwrite(data, sizeof(float), (size_t)f->n_elem, fp) == (size_t)f->n_elem;
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(JV_EIO, "short write " + path);
    g_err.clear();
    return JV_OK;
}

jv_status jv_fld_read(const char *path, jv_frame *f, float *data, size_t capacity) {
    if (!path || !f) return fail(JV_EINVAL, "jv_fld_read: NULL argument");
    const std::string p(path);
    if (p.size() < 4 || p.compare(p.size() - 4, 4, ".fld") != 0) return fail(JV_EINVAL, p + ": not a .fld file");
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return fail(JV_EIO, "cannot open " + p);
    jv_frame h;
    if (std::fread(&h, sizeof(h), 1, fp) != 1 || h.n_elem != h.n_rows * h.n_cols * h.n_slices) {
        std::fclose(fp);
        return fail(JV_EIO, p + ": bad frame header");
    }
    *f = h;
    if (data) {
        if (capacity < h.n_elem) {
            std::fclose(fp);
            return fail(JV_EINVAL, p + ": " + std::to_string(h.n_elem) + " values do not fit the buffer");
        }
        if (std::fread(data, sizeof(float), (size_t)h.n_elem, fp) != (size_t)h.n_elem) {
            std::fclose(fp);
            return fail(JV_EIO, p + ": truncated data");
        }
    }
    std::fclose(fp);
    g_err.clear();
    return JV_OK;
}

jv_status jv_raw_read(const char *path, size_t n, float *data) {
    if (!path || (n && !data)) return fail(JV_EINVAL, "jv_raw_read: NULL argument");
    std::string m = jv::read_raw(path, data, n);
    if (!m.empty()) return fail(JV_EIO, m);
    g_err.clear();
    return JV_OK;
}

jv_status jv_set_geometry(jv_ctx *c, int n_shot, const float *shot_xyz, int n_recv, const float *recv_xyz) {
    JV_IDLE(c);
    jv::Status s = c->eng->set_geometry(n_shot, shot_xyz, n_recv, recv_xyz);
    if (s) {
        c->shots.assign(shot_xyz, shot_xyz + 3 * (size_t)n_shot);
        c->recvs.assign(recv_xyz, recv_xyz + 3 * (size_t)n_recv);
    }
    return ret(s);
}

jv_status jv_rtm_forward_pass(jv_ctx *c, int shot) {
    JV_IDLE(c);
    return ret(c->eng->rtm_forward_pass(shot));
}

jv_status jv_rtm_reverse_begin(jv_ctx *c, int shot, const float *d_ox, const float *d_oy, const float *d_oz) {
    JV_IDLE(c);
    return ret(c->eng->rtm_reverse_begin(shot, d_ox, d_oy, d_oz));
}

jv_status jv_rtm_reverse_op(jv_ctx *c, int op, int it) {
    JV_IDLE(c);
    return ret(c->eng->rtm_reverse_op(op, it));
}

jv_status jv_rtm_reverse_end(jv_ctx *c) {
    JV_IDLE(c);
    return ret(c->eng->rtm_reverse_end());
}

jv_status jv_set_model(jv_ctx *c, const float *vp, const float *vs, const float *rho) {
    JV_IDLE(c);
    return ret(c->eng->set_model(vp, vs, rho));
}

jv_status jv_get_info(const jv_ctx *c, jv_info *info) {
    if (!c || !info) return fail(JV_EINVAL, "NULL argument");
    c->eng->info(info);
    return JV_OK;
}

jv_status jv_reconstruction_energy(const jv_ctx *c, double *e_forward_end, double *e_residual) {
    if (!c || !e_forward_end || !e_residual) return fail(JV_EINVAL, "NULL argument");
    c->eng->reconstruction_energy(e_forward_end, e_residual);
    return JV_OK;
}

jv_status jv_get_kernel_config(const jv_ctx *c, jv_options *out) {
    if (!c || !out) return fail(JV_EINVAL, "NULL argument");
    c->eng->kernel_config(out);
    return JV_OK;
}

jv_status jv_forward_device(jv_ctx *c, int shot, float *d_vx, float *d_vy, float *d_vz) {
    JV_IDLE(c);
    return ret(c->eng->forward(shot, d_vx, d_vy, d_vz));
}

jv_status jv_forward(jv_ctx *c, int shot, float *vx, float *vy, float *vz) {
    JV_IDLE(c);
    return forward_host(c, shot, vx, vy, vz);
}

jv_status jv_rtm_shot_device(jv_ctx *c, int shot, const float *d_ox, const float *d_oy, const float *d_oz) {
    JV_IDLE(c);
    return ret(c->eng->rtm_shot(shot, d_ox, d_oy, d_oz));
}

jv_status jv_rtm_shot(jv_ctx *c, int shot, const float *ox, const float *oy, const float *oz) {
    JV_IDLE(c);
    return rtm_host(c, shot, ox, oy, oz);
}

jv_status jv_rtm_batch(jv_ctx *c, int n, const int *shots, const float *const *obs) {
    JV_IDLE(c);
    if (n < 0 || (n > 0 && (!shots || !obs))) return fail(JV_EINVAL, "jv_rtm_batch: bad arguments");
    const size_t per = (size_t)c->eng->nrec() * c->eng->nt();
    for (int k = 0; k < n && per; k++)
        for (int q = 0; q < 3; q++)
            if (!obs[3 * k + q]) return fail(JV_EINVAL, "observed traces must not be NULL");
    for (int b = 0; b < 2 && n > b; b++) {
        jv_status st = ensure_traces(c, 3 * per, b);
        if (st != JV_OK) return st;
    }
    {
        jv_status st = ensure_copy_stream(c);
        if (st != JV_OK) return st;
    }
    // shot k's traces go to buffer k % 2 on the copy stream; buffer k % 2
    // is free once shot k - 2 has finished, which jv_rtm_shot waits for
    auto issue = [&](int k) -> jv_status {
        float *d = c->d_tr[k % 2];
        for (int q = 0; q < 3 && per; q++) {
            cudaError_t e = cudaMemcpyAsync(d + q * per, obs[3 * k + q], per * sizeof(float), cudaMemcpyHostToDevice,
                                            c->copy_stream);
            if (e != cudaSuccess) return fail(JV_ECUDA, cudaGetErrorString(e));
        }
        cudaError_t e = cudaEventRecord(c->ev_copy[k % 2], c->copy_stream);
        if (e != cudaSuccess) return fail(JV_ECUDA, cudaGetErrorString(e));
        return JV_OK;
    };
    jv_status st = n > 0 ? issue(0) : JV_OK;
    double total = 0.0;
    for (int k = 0; k < n && st == JV_OK; k++) {
        if (k + 1 < n) st = issue(k + 1);
        if (st != JV_OK) break;
        float *d = c->d_tr[k % 2];
        st = ret(c->eng->rtm_shot(shots[k], d, d + per, d + 2 * per, c->ev_copy[k % 2]));
        total += c->eng->last_ms();
    }
    cudaStreamSynchronize(c->copy_stream);
    if (st == JV_OK) c->eng->set_last_ms(total);
    return st;
}

// ---------------------------------------------------------------- jobs

static jv_status run_job(jv_ctx *c, const jv_job &j) {
    if (j.kind == JV_JOB_FORWARD) return forward_host(c, j.shot, j.out[0], j.out[1], j.out[2]);
    if (j.obs[0] || j.obs[1] || j.obs[2]) return rtm_host(c, j.shot, j.obs[0], j.obs[1], j.obs[2]);
    // no observed traces: model them on the device, then migrate them
    const size_t per = (size_t)c->eng->nrec() * c->eng->nt();
    jv_status st = ensure_traces(c, 3 * per);
    if (st != JV_OK) return st;
    float *d = c->d_tr[0];
    st = ret(c->eng->forward(j.shot, d, d + per, d + 2 * per));
    if (st != JV_OK) return st;
    return ret(c->eng->rtm_shot(j.shot, d, d + per, d + 2 * per));
}

static void worker_main(jv_ctx *c) {
    cudaSetDevice(c->eng->device());
    for (;;) {
        long long id;
        jv_job job;
        {
            std::unique_lock<std::mutex> l(c->mu);
            c->cv.wait(l, [&] { return c->stop || !c->queue.empty(); });
            if (c->queue.empty()) return;  // stop requested, nothing left
            id = c->queue.front();
            c->queue.pop_front();
            JobRec &r = c->jobs[id];
            r.state = JV_JOB_RUNNING;
            job = r.job;
            c->running = true;
        }
        const jv_status st = run_job(c, job);
        const std::string msg = st == JV_OK ? std::string() : g_err;
        {
            std::lock_guard<std::mutex> l(c->mu);
            JobRec &r = c->jobs[id];
            r.state = JV_JOB_DONE;
            r.result = st;
            r.msg = msg;
            c->running = false;
        }
        c->done_cv.notify_all();
    }
}

jv_status jv_submit(jv_ctx *c, const jv_job *job, long long *id) {
    if (!c || !job || !id) return fail(JV_EINVAL, "jv_submit: NULL argument");
    if (job->kind != JV_JOB_FORWARD && job->kind != JV_JOB_RTM) return fail(JV_EINVAL, "unknown job kind");
    jv_info inf;
    c->eng->info(&inf);
    if (job->shot < 0 || job->shot >= inf.n_shot) return fail(JV_EINVAL, "shot index out of range");
    {
        std::lock_guard<std::mutex> l(c->mu);
        if (c->stop) return fail(JV_ESTATE, "context is closing");
        *id = c->next_id++;
        JobRec r;
        r.job = *job;
        c->jobs[*id] = r;
        c->queue.push_back(*id);
        if (!c->worker.joinable()) c->worker = std::thread(worker_main, c);
    }
    c->cv.notify_one();
    g_err.clear();
    return JV_OK;
}

jv_status jv_poll(jv_ctx *c, long long id, int *state, jv_status *result) {
    if (!c || !state) return fail(JV_EINVAL, "jv_poll: NULL argument");
    std::lock_guard<std::mutex> l(c->mu);
    auto it = c->jobs.find(id);
    if (it == c->jobs.end()) return fail(JV_EINVAL, "no such job");
    *state = it->second.state;
    if (result) *result = it->second.result;
    g_err = it->second.msg;
    return JV_OK;
}

jv_status jv_wait(jv_ctx *c, long long id, double timeout_s, jv_status *result) {
    if (!c) return fail(JV_EINVAL, "jv_wait: NULL context");
    std::unique_lock<std::mutex> l(c->mu);
    auto it = c->jobs.find(id);
    if (it == c->jobs.end()) return fail(JV_EINVAL, "no such job");
    auto ended = [&] { return it->second.state == JV_JOB_DONE || it->second.state == JV_JOB_CANCELLED; };
    if (timeout_s < 0) {
        c->done_cv.wait(l, ended);
    } else if (!c->done_cv.wait_for(l, std::chrono::duration<double>(timeout_s), ended)) {
        g_err = "job still " + std::string(it->second.state == JV_JOB_RUNNING ? "running" : "queued");
        return JV_ETIMEOUT;
    }
    if (result) *result = it->second.result;
    g_err = it->second.msg;
    return JV_OK;
}

jv_status jv_cancel(jv_ctx *c, long long id) {
    if (!c) return fail(JV_EINVAL, "jv_cancel: NULL context");
    {
        std::lock_guard<std::mutex> l(c->mu);
        auto it = c->jobs.find(id);
        if (it == c->jobs.end()) return fail(JV_EINVAL, "no such job");
        if (it->second.state != JV_JOB_QUEUED) return fail(JV_ESTATE, "job has already started");
        for (auto q = c->queue.begin(); q != c->queue.end(); ++q)
            if (*q == id) {
                c->queue.erase(q);
                break;
            }
        it->second.state = JV_JOB_CANCELLED;
        it->second.result = JV_ECANCELED;
        it->second.msg = "cancelled before it started";
    }
    c->done_cv.notify_all();
    g_err.clear();
    return JV_OK;
}

jv_status jv_image_reset(jv_ctx *c) {
    JV_IDLE(c);
    return ret(c->eng->image_reset());
}

jv_status jv_image_get(jv_ctx *c, int kind, double *out) {
    JV_IDLE(c);
    return ret(c->eng->image_get(kind, out));
}

jv_status jv_image_finalize(jv_ctx *c, float *img_pp, float *img_ps, float *img_sp, float *img_ss, float *lap_pp,
                            float *lap_ps, float *lap_sp, float *lap_ss) {
    JV_IDLE(c);
    float *o[8] = {img_pp, img_ps, img_sp, img_ss, lap_pp, lap_ps, lap_sp, lap_ss};
    return ret(c->eng->image_finalize(o));
}

jv_status jv_image_get_device(jv_ctx *c, int kind, double *d_out) {
    JV_IDLE(c);
    return ret(c->eng->image_get_device(kind, d_out));
}

jv_status jv_image_set(jv_ctx *c, int kind, const double *in) {
    JV_IDLE(c);
    return ret(c->eng->image_set(kind, in, false));
}

jv_status jv_image_set_device(jv_ctx *c, int kind, const double *d_in) {
    JV_IDLE(c);
    return ret(c->eng->image_set(kind, d_in, true));
}

jv_status jv_set_profiling(jv_ctx *c, int on) {
    JV_IDLE(c);
    c->eng->set_profiling(on != 0);
    return JV_OK;
}

jv_status jv_profile_entry(const jv_ctx *c, int idx, const char **name, double *total_ms, long long *launches) {
    if (!c || !name || !total_ms || !launches) return fail(JV_EINVAL, "NULL argument");
    if (!c->eng->profile_entry(idx, name, total_ms, launches)) return fail(JV_EINVAL, "no such profile entry");
    return JV_OK;
}

jv_status jv_run_project(jv_ctx *c) { return jv_run_project_shard(c, 0, 1, nullptr, nullptr); }

jv_status jv_run_project_shard(jv_ctx *c, int rank, int world, jv_reduce_fn reduce, void *user) {
    JV_IDLE(c);
    if (!c->from_project) return fail(JV_ESTATE, "jv_run_project needs a context made by jv_open");
    if (world < 1 || rank < 0 || rank >= world) return fail(JV_EINVAL, "rank must be in [0, world)");
    if (world > 1 && !reduce) return fail(JV_EINVAL, "a job of several ranks needs a reduce function");
    jv_info inf;
    c->eng->info(&inf);
    const int nshot = inf.n_shot, nrec = inf.n_recv, nt = inf.nt;
    const size_t per = (size_t)nrec * nt;
    // this rank's shots: s % world == rank (every shot exactly once over the job)
    std::vector<int> mine;
    for (int s = rank; s < nshot; s += world) mine.push_back(s);
    // phase 1: model the shots, keep their traces (mpi_sub_rtm3d :20-38)
    std::vector<float> all(mine.size() * 3 * per);
    for (size_t q0 = 0; q0 < mine.size(); q0++) {
        const int s = mine[q0];
        float *t = all.data() + q0 * 3 * per;
        jv_status st = jv_forward(c, s, t, t + per, t + 2 * per);
        if (st != JV_OK) return st;
        if (nrec > 0) {
            const char *nm[3] = {"vx_seis_0_", "vy_seis_0_", "vz_seis_0_"};
            for (int q = 0; q < 3; q++) {
                std::string m = jv::write_traces(c->arg.output_path + nm[q] + std::to_string(s), t + q * per, nrec, nt);
                if (!m.empty()) return fail(JV_EIO, m);
            }
        }
    }
    // phase 2: migrate the shots into one stack (:45-122)
    jv_status st = jv_image_reset(c);
    if (st != JV_OK) return st;
    for (size_t q0 = 0; q0 < mine.size(); q0++) {
        float *t = all.data() + q0 * 3 * per;
        st = jv_rtm_shot(c, mine[q0], t, t + per, t + 2 * per);
        if (st != JV_OK) return st;
    }
    const size_t n = (size_t)inf.n_phy;
    // sum the partial stacks of all ranks, before the Laplacian and the
    // compensation (the reference applies both to the stack of all shots)
    if (world > 1) {
        std::vector<double> buf(n);
        for (int k = 0; k < 5; k++) {
            st = jv_image_get(c, k, buf.data());
            if (st != JV_OK) return st;
            if (reduce(buf.data(), n, user) != 0) return fail(JV_ECANCELED, "the reduce function failed");
            st = jv_image_set(c, k, buf.data());
            if (st != JV_OK) return st;
        }
    }
    if (rank != 0) return JV_OK;
    // Laplacian, compensation, save (:123-134)
    std::vector<float> im(8 * n);
    float *o[8];
    for (int q = 0; q < 8; q++) o[q] = im.data() + q * n;
    st = jv_image_finalize(c, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7]);
    if (st != JV_OK) return st;
    const std::string suf = jv::size_info(inf.grid.nx, inf.grid.ny, inf.grid.nz, 0.f, 0.f, 0.f) + ".raw";
    const char *names[6] = {"image_pp_0", "image_pp_laplace_0", "image_ps_0", "image_sp_0", "image_ss_0", nullptr};
    const float *srcs[5] = {o[0], o[4], o[1], o[2], o[3]};
    jv_frame fr;
    jv_frame_make((uint64_t)inf.grid.nx, (uint32_t)inf.grid.ny, (uint32_t)inf.grid.nz, inf.grid.dx, inf.grid.dy,
                  inf.grid.dz, 0.f, 0.f, 0.f, &fr);
    for (int q = 0; q < 5; q++) {
        std::string m = jv::write_raw(c->arg.output_path + names[q] + suf, srcs[q], n);
        if (!m.empty()) return fail(JV_EIO, m);
        if (c->arg.save_fld) {
            st = jv_fld_write((c->arg.output_path + names[q]).c_str(), &fr, srcs[q]);
            if (st != JV_OK) return st;
        }
    }
    // source illumination, as a float raw image
    std::vector<double> ip(n);
    st = jv_image_get(c, JV_IMG_IP, ip.data());
    if (st != JV_OK) return st;
    std::vector<float> ipf(ip.begin(), ip.end());
    std::string m = jv::write_raw(c->arg.output_path + "image_ipfd_0" + suf, ipf.data(), n);
    if (!m.empty()) return fail(JV_EIO, m);
    if (c->arg.save_fld) return jv_fld_write((c->arg.output_path + "image_ipfd_0").c_str(), &fr, ipf.data());
    return JV_OK;
}

jv_status jv_last_timing(const jv_ctx *c, double *ms) {
    if (!c || !ms) return fail(JV_EINVAL, "NULL argument");
    *ms = c->eng->last_ms();
    return JV_OK;
}

jv_status jv_sync(jv_ctx *c) {
    JV_IDLE(c);
    return ret(c->eng->sync());
}

jv_status jv_close(jv_ctx *c) {
    delete c;
    return JV_OK;
}

const char *jv_last_error(void) { return g_err.c_str(); }

const char *jv_build_info(void) {
    static char buf[128];
    std::snprintf(buf, sizeof(buf), "libjv abi %d, sm_100a, nvcc %d.%d", JV_ABI_VERSION, __CUDACC_VER_MAJOR__,
                  __CUDACC_VER_MINOR__);
    return buf;
}

}  // extern "C"
