// noalloc.cu -- forward modelling without any device allocation.
//
// Who needs this: callers that must not call cudaMalloc/cudaFree at the
// moment they model a shot.  Examples are a host application whose memory
// pool (a framework's caching allocator, a reserved arena) already owns all
// free device memory, so a fresh cudaMalloc would fail; latency-sensitive
// paths where an allocation or free could block or synchronise the device;
// and plug-in hosts that forbid a plug-in from owning device memory at all.
// They pass every input and output; the working memory (wavefield, CPML
// memory variables, extended model, tables, receiver indices, step state)
// is carved out of one fixed scratch array compiled into this library.
//
// The scratch array lives for as long as the library is loaded, on every
// GPU that loads it (kNoAllocScratchBytes, 64 MiB).  Every call shares it
// and finds the previous call's contents in it: each call rewrites the
// tables and clears the wavefield and memory variables before it starts.
// Two calls whose GPU work overlaps (two host threads, or two streams on
// one device) race on the same array and produce garbage; serialise them.
//
// Host code cannot use the array's name as a device address (in host code
// it is a host-side stand-in), so the first call on each device, with that
// device current, looks the address up with cudaGetSymbolAddress, uploads
// the finite-difference coefficients into constant memory (the same values
// every context uses) and caches both facts with the device's current
// context.  A later call that finds another context current on the device
// (after cudaDeviceReset, or a primary context torn down and created anew)
// repeats that set-up.  The set-up synchronises the device once, so make the
// first call on a device before any stream capture; later calls only queue
// copies, memsets and kernels on `stream` and wait for that stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine.hpp"
#include "jv/jv.h"
#include "jv_internal.hpp"

namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct DeviceSetup {
    void *ctx = nullptr;   // the context current when the set-up ran
    void *addr = nullptr;  // device address of g_noalloc_scratch in it
};
DeviceSetup g_setup[kMaxDevices];

jv_status fail(jv_status c, const std::string &m) {
    jv::set_last_error(m);
    return c;
}

// the calling thread's current context (driver API, reached through the
// runtime so that the library needs no -lcuda); nullptr if unavailable
void *current_context() {
    typedef int (*CtxGetCurrent)(void **);
    static CtxGetCurrent fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (CtxGetCurrent) nullptr;
        return (CtxGetCurrent)f;
    }();
    void *c = nullptr;
    if (fn && fn(&c) != 0) c = nullptr;
    return c;
}

// Per-device set-up, once per device and context, under g_mu: the device
// address of the scratch array and the constant-memory coefficients.
jv_status device_setup(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(JV_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceSetup &d = g_setup[dev];
    void *ctx = current_context();
    if (!ctx) {
        // no context bound to this thread yet: bind (and if need be create)
        // the device's primary context, the one the set-up below uses, so
        // that the context recorded is that one (a context the caller has
        // made current is left as it is)
        cudaError_t e0 = cudaSetDevice(dev);
        if (e0 != cudaSuccess) return fail(JV_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e0));
        ctx = current_context();
    }
    if (!d.addr || ctx != d.ctx) {
        d.addr = nullptr;
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(JV_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        if (jv::upload_all_coefficients() != 0) return fail(JV_ECUDA, "coefficient upload failed");
        d.ctx = ctx;
        d.addr = p;
    }
    *out = (unsigned char *)d.addr;
    return JV_OK;
}

// bump allocator over the scratch array (256-byte aligned pieces)
struct Carver {
    unsigned char *base;
    size_t used = 0, cap;
    template <class T>
    T *take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        size_t bytes = count * sizeof(T);
        if (off + bytes > cap) return nullptr;
        used = off + bytes;
        return reinterpret_cast<T *>(base + off);
    }
};

}  // namespace

extern "C" jv_status jv_forward_noalloc(const jv_grid *grid, const float *d_vp, const float *d_vs, const float *d_rho,
                                        float dt, float fm, int nt, const float *src_xyz, int n_recv,
                                        const float *recv_xyz, float *d_vx, float *d_vy, float *d_vz,
                                        int *n_kept, void *stream) {
    using namespace jv;
    if (!grid || !d_vp || !d_vs || !d_rho || !src_xyz || (n_recv > 0 && !recv_xyz) || !n_kept)
        return fail(JV_EINVAL, "jv_forward_noalloc: NULL argument");
    if (grid->nx < 8 || grid->ny < 8 || grid->nz < 8) return fail(JV_EINVAL, "gridphy must have >= 8 cells per axis");
    if (grid->pml < kPhyHalf) return fail(JV_EINVAL, "pml_num must be >= 4");
    if (!(grid->dx > 0) || !(grid->dy > 0) || !(grid->dz > 0) || !(dt > 0) || !(fm > 0) || nt < 1)
        return fail(JV_EINVAL, "spacing, dt, fm must be > 0 and nt >= 1");
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(JV_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));

    // layout and CPML slabs: the same as the context path
    const int m = grid->pml;
    size_t fe = 0;
    const GridDev g = make_layout(*grid, &fe);
    const size_t guard = 32;
    long long psi_total = 0;
    CpmlDev cp = make_pml_slabs(g, 1, &psi_total);
    cp.dt = dt;

    // receivers inside gridphy, in input order (as jv_set_geometry keeps them)
    const float rx = (float)(g.px - 1) * g.dx, ry = (float)(g.py - 1) * g.dy, rz = (float)(g.pz - 1) * g.dz;
    const float lx = -(float)m * g.dx, ly = -(float)m * g.dy, lz = -(float)m * g.dz;
    auto inside = [&](const float *q) {
        return q[0] >= 0.0f && q[0] <= rx && q[1] >= 0.0f && q[1] <= ry && q[2] >= 0.0f && q[2] <= rz;
    };
    auto elem = [&](const float *q) -> long long {
        return g.xoff + gap_num(lx, q[0], g.dx) + g.sy * gap_num(ly, q[1], g.dy) + g.sz * gap_num(lz, q[2], g.dz);
    };
    if (!inside(src_xyz)) return fail(JV_EINVAL, "source lies outside gridphy");
    std::vector<long long> rec;
    for (int r = 0; r < n_recv; r++)
        if (inside(recv_xyz + 3 * r)) rec.push_back(elem(recv_xyz + 3 * r));
    *n_kept = (int)rec.size();

    // carve the scratch array; refuse problems that do not fit
    unsigned char *base = nullptr;
    jv_status st = device_setup(dev, &base);
    if (st != JV_OK) return st;
    Carver cv{base, 0, kNoAllocScratchBytes};
    float *model = cv.take<float>(4 * fe + guard);
    float *wave = cv.take<float>(9 * fe + guard);
    float *psi = cv.take<float>((size_t)psi_total);
    float4 *tabs[3];
    for (int a = 0; a < 3; a++) tabs[a] = cv.take<float4>((size_t)(a == 0 ? g.nx : a == 1 ? g.ny : g.nz));
    float *wavelet = cv.take<float>((size_t)nt);
    StepState *state = cv.take<StepState>(1);
    long long *rec_d = cv.take<long long>(rec.size() + 1);
    if (!model || !wave || (psi_total && !psi) || !tabs[0] || !tabs[1] || !tabs[2] || !wavelet || !state || !rec_d)
        return fail(JV_EINVAL, "problem needs more than the " + std::to_string(kNoAllocScratchBytes >> 20) +
                                   " MiB no-allocation scratch; use jv_create/jv_forward");
    if (fe >= ((size_t)1 << 31)) return fail(JV_EINVAL, "grid too large");

    // host-side tables, copied into the scratch array
    std::vector<float4> t[3];
    pml_axis_tables(g, fm, t);
    std::vector<float> wl(nt);
    ricker(nt, fm, dt, wl.data());
    StepState hs{};
    hs.it = 0;
    hs.src = elem(src_xyz);
    hs.tr[0] = d_vx;
    hs.tr[1] = d_vy;
    hs.tr[2] = d_vz;

    auto ck = [&](cudaError_t ee, const char *what) -> jv_status {
        if (ee != cudaSuccess) return fail(JV_ECUDA, std::string(what) + ": " + cudaGetErrorString(ee));
        return JV_OK;
    };
    // on failure, wait for the work already queued on `s` (it still writes the
    // scratch array and the caller's trace buffers) before returning
#define NA_CK(expr)                                    \
    do {                                               \
        jv_status _s = ck((cudaError_t)(expr), #expr); \
        if (_s != JV_OK) {                             \
            (void)cudaStreamSynchronize(s);            \
            return _s;                                 \
        }                                              \
    } while (0)
    for (int a = 0; a < 3; a++)
        NA_CK(cudaMemcpyAsync(tabs[a], t[a].data(), t[a].size() * sizeof(float4), cudaMemcpyHostToDevice, s));
    NA_CK(cudaMemcpyAsync(wavelet, wl.data(), nt * sizeof(float), cudaMemcpyHostToDevice, s));
    NA_CK(cudaMemcpyAsync(state, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    if (!rec.empty()) NA_CK(cudaMemcpyAsync(rec_d, rec.data(), rec.size() * sizeof(long long), cudaMemcpyHostToDevice, s));
    // the previous call left its state here: clear what must start at zero
    NA_CK(cudaMemsetAsync(model, 0, (4 * fe + guard) * sizeof(float), s));
    NA_CK(cudaMemsetAsync(wave, 0, (9 * fe + guard) * sizeof(float), s));
    if (psi_total) NA_CK(cudaMemsetAsync(psi, 0, (size_t)psi_total * sizeof(float), s));

    float *mb = model + guard;
    float *vp = mb, *bdt = mb + fe, *lam = mb + 2 * fe, *mu = mb + 3 * fe;
    NA_CK(k_model_prep(g, d_vp, d_vs, d_rho, dt, vp, bdt, lam, mu, s));
    WaveDev w{};
    for (int f = 0; f < 9; f++) w.f[f] = wave + guard + f * fe;
    for (int a = 0; a < 3; a++) cp.ax[a] = tabs[a];
    cp.psi = psi;
    KCfg kc;
    kc.variant = 2;
    for (int it = 0; it < nt; it++) {
        NA_CK(k_vel_pml(g, cp, w, bdt, vp, kc, s));
        NA_CK(k_vel_phy(kFwd, g, w, bdt, dt, 1, nullptr, nullptr, kc, s));
        NA_CK(k_stress_pml(g, cp, w, lam, mu, vp, 0, kc, s));
        NA_CK(k_stress_phy(kFwd, g, w, lam, mu, dt, 1, wavelet, state, 0, kc, s));
        NA_CK(k_record(w, rec_d, (int)rec.size(), nt, state, 0, s));
        NA_CK(k_step_advance(state, +1, s));
    }
    NA_CK(cudaStreamSynchronize(s));
#undef NA_CK
    jv::set_last_error("");
    return JV_OK;
}
