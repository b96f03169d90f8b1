// engine.cu -- host orchestration of libjv (see engine.hpp).
//
// The time loops restate the reference's blend drivers:
//   modelling      FD/fdtd3d_3_model_mpi_blend/fdtd3d_blend_elastic_model_mpi_meat.hpp:44-88
//   RTM forward    same file :125-155 (VOWR pack after the CPML stress update)
//   time reverse   RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:64-113
// (FD = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_fdtd3d_model_mpi,
//  RTM = .../elastic_1_rtm3d_model_mpi, relative to the reference root).
#include "engine.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

namespace jv {

// ------------------------------------------------------------ helpers

void diff_coeff(int order, double *c) {
    for (int n = 0; n < order; n++) {
        double a1 = 1, a2 = 1, a3 = 1;
        for (int i = 0; i < order; i++) {
            if (i != n) a1 = a1 * (2 * i + 1) * (2 * i + 1);
            if (i < n) a2 = a2 * ((2 * n + 1) * (2 * n + 1) - (2 * i + 1) * (2 * i + 1));
            if (i > n) a3 = a3 * ((2 * i + 1) * (2 * i + 1) - (2 * n + 1) * (2 * n + 1));
        }
        a1 = a1 * ((n % 2) ? -1.0 : 1.0);
        c[n] = a1 / ((2 * n + 1) * a2 * a3);
    }
}

int gap_num(float l, float r, float d) {
    int n_l, n_r;
    float v = 1.0f / d;
    if (l > 0) n_l = (int)(l * v + 0.125f);
    else n_l = (int)(l * v - 0.125f);
    if (r > 0) n_r = (int)(r * v + 0.125f);
    else n_r = (int)(r * v - 0.125f);
    return n_r - n_l;
}

int ntime(float T, float dt) {
    volatile float q = T / dt;
    return (int)std::ceil(q);
}

void ricker(int nt, float fm, float dt, float *w) {
    const double pi = 3.14159265358979323846;
    float dura = 1.3f / fm;
    volatile float q = dura / dt + 0.5f;
    int n0 = (int)std::floor(q);
    for (int i = 0; i < nt; i++) {
        volatile float t = (float)(i - n0) * dt;
        double a = pi * (double)fm * (double)t;
        double a2 = a * a;
        w[i] = (float)(1.0e4 * (1.0 - 2.0 * a2) * std::exp(-a2));
    }
}

static long long round_up(long long v, long long a) { return (v + a - 1) / a * a; }

// Every pitched field arena starts with kGuard zero floats, so the 16-byte
// x groups of the CPML slabs may read a few cells before gridext (x >= -5)
// without leaving the allocation; each field also ends with >= 128 floats
// of slack for reads past the last row.
constexpr size_t kGuard = 32;

Status Engine::cu(cudaError_t e, const char *what) const {
    Status s;
    if (e != cudaSuccess) {
        s.code = (e == cudaErrorMemoryAllocation) ? JV_ENOMEM : JV_ECUDA;
        s.msg = std::string(what) + ": " + cudaGetErrorString(e);
    }
    return s;
}

static Status bad(jv_status c, const std::string &m) {
    Status s;
    s.code = c;
    s.msg = m;
    return s;
}

#define JV_TRY(expr)                  \
    do {                              \
        Status _s = (expr);           \
        if (!_s) return _s;           \
    } while (0)
#define JV_CU(expr) JV_TRY(cu((expr), #expr))
#define JV_K(expr) JV_TRY(cu((cudaError_t)(expr), #expr))

// Device memory comes from the stream-ordered allocator on the context's
// stream: neither allocating nor freeing waits for other contexts' work on
// the device, so contexts run concurrently (a plain cudaFree would wait
// for the whole device).  The stream is synchronised once the allocation
// is made, so the memory is also usable from synchronous copies.
Status Engine::alloc(void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return Status{};
    cudaError_t e = cudaMallocAsync(p, bytes, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (*p) cudaFreeAsync(*p, stream_);
        *p = nullptr;
        return bad(JV_ENOMEM, "allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
    }
    allocs_.push_back(*p);
    dev_bytes_ += bytes;
    return Status{};
}

Engine::~Engine() {
    if (stream_) {
        cudaSetDevice(dev_);
        cudaStreamSynchronize(stream_);
    }
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    for (cudaEvent_t e : prof_pool_) cudaEventDestroy(e);
    for (void *p : allocs_)
        if (p) cudaFreeAsync(p, stream_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (host_store_) cudaFreeHost(host_store_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

// ------------------------------------------------------------ layout helpers

GridDev make_layout(const jv_grid &grid, size_t *field_elems) {
    GridDev g{};
    const int m = grid.pml;
    g.m = m;
    g.px = grid.nx; g.py = grid.ny; g.pz = grid.nz;
    g.nx = grid.nx + 2 * m; g.ny = grid.ny + 2 * m; g.nz = grid.nz + 2 * m;
    g.xoff = (32 - (m % 32)) % 32;
    g.sy = round_up(g.xoff + g.nx, 32);
    g.sz = g.sy * g.ny;
    g.dx = grid.dx; g.dy = grid.dy; g.dz = grid.dz;
    *field_elems = (size_t)round_up(g.sz * g.nz + 128, 64);
    return g;
}

CpmlDev make_pml_slabs(const GridDev &g, int zp, long long *psi_total) {
    zp = zp == 2 ? 2 : 1;
    const int NX = g.nx, NY = g.ny, NZ = g.nz, m = g.m;
    // top, bottom (z); front, back (y, physical z); right, left (x, physical y and z)
    const int bx[6][6] = {
        {2, NX - 2, 2, NY - 2, 2, m},           {2, NX - 2, 2, NY - 2, NZ - m, NZ - 2},
        {2, NX - 2, 2, m, m, NZ - m},           {2, NX - 2, NY - m, NY - 2, m, NZ - m},
        {2, m, m, NY - m, m, NZ - m},           {NX - m, NX - 2, m, NY - m, m, NZ - m},
    };
    const int na[6] = {3, 3, 2, 2, 1, 1};
    CpmlDev c{};
    long long off = 0;
    int blocks = 0;
    for (int q = 0; q < 6; q++) {
        PmlSlab S{};
        S.x0 = bx[q][0]; S.x1 = bx[q][1]; S.y0 = bx[q][2]; S.y1 = bx[q][3]; S.z0 = bx[q][4]; S.z1 = bx[q][5];
        S.naxes = na[q];
        if (S.x1 <= S.x0 || S.y1 <= S.y0 || S.z1 <= S.z0) continue;
        S.gstart = S.x0 - (int)((g.xoff + S.x0) & 3);
        S.ngroups = (S.x1 - S.gstart + 3) / 4;
        S.pitch = 4 * S.ngroups;
        // up to 64 groups of a row per block, as many rows as fit 256 threads
        const int nb = (S.ngroups + 63) / 64;
        S.gx = (S.ngroups + nb - 1) / nb;
        S.gy = 256 / S.gx;
        S.bx = (S.ngroups + S.gx - 1) / S.gx;
        S.by = (S.y1 - S.y0 + S.gy - 1) / S.gy;
        S.first_block = blocks;
        blocks += S.bx * S.by * ((S.z1 - S.z0 + zp - 1) / zp);
        S.stride = (long long)S.pitch * (S.y1 - S.y0) * (S.z1 - S.z0);
        S.psi_off = off;
        off += 6LL * S.naxes * S.stride;
        c.s[c.nslab++] = S;
    }
    c.nblocks = blocks;
    c.zp = zp;
    *psi_total = off;
    return c;
}

void pml_axis_tables(const GridDev &g, float fm, std::vector<float4> t[3]) {
    // d = vp * K, K = log10(1/R) 7 (s/N)^2 / (2 N delta), R = 0.001
    const int m = g.m;
    const double N = (double)(m - kPmlHalf);
    const double l10x7 = (double)(std::log10(1.0f / 0.001f) * 7.0f);
    const float alpha_max = (float)(3.14159265358979323846 * (double)fm);
    const int nax[3] = {g.nx, g.ny, g.nz};
    const float del[3] = {g.dx, g.dy, g.dz};
    for (int a = 0; a < 3; a++) {
        const int n = nax[a];
        t[a].assign(n, make_float4(0.f, 0.f, 0.f, 0.f));
        for (int c = 0; c < n; c++) {
            double sI, sH;
            if (c >= kPmlHalf && c < m) {  // low side: integer node m-c, half node m-c-1/2
                sI = m - c;
                sH = m - c - 0.5;
            } else if (c >= n - m && c < n - kPmlHalf) {  // high side: the two swap
                sH = c - (n - m - 1);
                sI = sH - 0.5;
            } else {
                continue;
            }
            const double k0 = l10x7 / (2.0 * N * (double)del[a]);
            const float qI = (float)sI / (float)N, qH = (float)sH / (float)N;
            t[a][c].x = (float)(k0 * (double)qI * (double)qI);
            t[a][c].y = (float)(k0 * (double)qH * (double)qH);
            t[a][c].z = std::max(alpha_max * (1.0f - qI), 0.0f);
            t[a][c].w = std::max(alpha_max * (1.0f - qH), 0.0f);
        }
    }
}

int upload_all_coefficients() {
    float list[5][4] = {};
    for (int o = 1; o <= 4; o++) {
        double c[4];
        diff_coeff(o, c);
        for (int i = 0; i < o; i++) list[o][i] = (float)c[i];
    }
    double c2[2];
    diff_coeff(2, c2);
    const float dc2[2] = {(float)c2[0], (float)c2[1]};
    return upload_coefficients(list, dc2);
}

// VOWR face boxes (FD/fdtd3d_0_base_module/fdtd3d_base_5_wave_recon_meat.hpp:19-30;
// face frames .jarvis_0_meta/.jarvis_3_operator/jarvis_1_mpicu_halo_store_operator_meat.hpp:129-134),
// velocity fields first, with their offsets in the per-step record and their
// first 256-thread block
std::vector<SegDev> vowr_segments(const GridDev &g, int r, long long *per_step, long long *blocks, bool vec) {
    const int W[10][6] = {
        {r - 1, r, r - 1, r, r, r - 1}, {r - 1, r, r, r - 1, r - 1, r}, {r, r - 1, r - 1, r, r - 1, r},
        {0, 0, 0, 0, r - 1, r},         {0, 0, r - 1, r, 0, 0},         {r - 1, r, 0, 0, 0, 0},
        {r - 1, r, r - 1, r, r - 1, r}, {0, 0, r, r - 1, r, r - 1},     {r, r - 1, 0, 0, r, r - 1},
        {r, r - 1, r, r - 1, 0, 0}};
    const int flds[10] = {VX, VY, VZ, SXX, SYY, SZZ, SAU, SXY, SXZ, SYZ};
    const int m = g.m;
    const int X0 = m, X1 = m + g.px, Y0 = m, Y1 = m + g.py, Z0 = m, Z1 = m + g.pz;
    std::vector<SegDev> segs;
    long long off = 0, blk = 0;
    for (int f = 0; f < 10; f++)
        for (int face = 0; face < 6; face++) {
            int wd = W[f][face];
            if (wd <= 0) continue;
            int x0 = X0, x1 = X1, y0 = Y0, y1 = Y1, z0 = Z0, z1 = Z1;
            switch (face) {
            case 0: z0 = Z0 - wd; z1 = Z0; break;
            case 1: z0 = Z1; z1 = Z1 + wd; break;
            case 2: y0 = Y0 - wd; y1 = Y0; break;
            case 3: y0 = Y1; y1 = Y1 + wd; break;
            case 4: x0 = X0 - wd; x1 = X0; break;
            default: x0 = X1; x1 = X1 + wd; break;
            }
            SegDev sg{};
            sg.fld = flds[f];
            sg.x0 = x0; sg.nxb = x1 - x0; sg.y0 = y0; sg.nyb = y1 - y0; sg.z0 = z0; sg.nzb = z1 - z0;
            if (vec) off = (off + 3) / 4 * 4;  // 16-byte aligned box records
            sg.off = off;
            sg.nblk_first = blk;
            // rows of whole 16-byte x groups: 4 values a thread
            sg.vw = vec && sg.nxb % 4 == 0 && (g.xoff + x0) % 4 == 0 ? 4 : 1;
            long long cnt = (long long)sg.nxb * sg.nyb * sg.nzb;
            off += cnt;
            blk += (cnt + 256LL * sg.vw - 1) / (256LL * sg.vw);
            segs.push_back(sg);
        }
    if (vec) off = (off + 3) / 4 * 4;  // every step's record starts 16-byte aligned
    *per_step = off;
    *blocks = blk;
    return segs;
}

size_t footprint_bytes(const jv_grid &grid, int nt, int rec_width, bool rtm, int precision) {
    size_t fe = 0;
    const GridDev g = make_layout(grid, &fe);
    long long psi = 0;
    make_pml_slabs(g, 1, &psi);
    const size_t nphy = (size_t)grid.nx * grid.ny * grid.nz;
    size_t b = (4 * fe + 32) * sizeof(float);                 // model
    b += (kNumFld * fe + 32) * sizeof(float);                 // forward wavefield
    b += (size_t)psi * sizeof(float);                         // its memory variables
    b += (size_t)2 * fz_psi_floats(g) * sizeof(float);        // the full-gridext kernels' ones
    b += 5 * nphy * sizeof(double);                           // stacks
    b += 16 * ((size_t)grid.nx + grid.ny + grid.nz + 2 * grid.pml * 3) + (1 << 20);  // tables, state, slack
    if (rtm) {
        long long per = 0, blk = 0;
        const bool s16 = precision == JV_BF16 || precision == JV_FP16;
        const std::vector<SegDev> segs = vowr_segments(g, rec_width, &per, &blk, !s16);
        const size_t nslot = nt > 1 ? nt - 1 : 0;
        b += (kNumFld * fe + 32) * sizeof(float) + (size_t)(psi + 2 * fz_psi_floats(g)) * sizeof(float);  // receiver wavefield
        b += (size_t)per * nslot * (s16 ? sizeof(uint16_t) : sizeof(float));      // boundary store
        if (s16) b += (nslot + 2) * segs.size() * sizeof(float);                    // its per-box scales
        b += 5 * ((nphy + 63) / 64 * 64) * sizeof(float);                           // shot image
    }
    return b;
}

// ------------------------------------------------------------ creation

Status Engine::create(const jv_grid &grid, const float *vp, const float *vs, const float *rho, float dt, float fm,
                      int nt, const jv_options &opt, Engine **out) {
    *out = nullptr;
    if (grid.nx < 8 || grid.ny < 8 || grid.nz < 8)
        return bad(JV_EINVAL, "gridphy must have at least 8 cells per axis");
    if (grid.pml < kPhyHalf) return bad(JV_EINVAL, "pml_num must be >= 4 (the 8th-order stencil reaches 4 cells)");
    if (!(grid.dx > 0) || !(grid.dy > 0) || !(grid.dz > 0)) return bad(JV_EINVAL, "grid spacing must be > 0");
    if (!(dt > 0) || !(fm > 0)) return bad(JV_EINVAL, "dt and fm must be > 0");
    if (nt < 1) return bad(JV_EINVAL, "nt must be >= 1");
    if (!vp || !vs || !rho) return bad(JV_EINVAL, "model arrays must not be NULL");
    int rw = opt.rec_width == 0 ? 1 : opt.rec_width;
    if (rw < 1 || rw > kPhyHalf || rw > grid.pml) return bad(JV_EINVAL, "rec_width must be in 1..4 and <= pml_num");
    if (opt.precision != JV_FP32 && opt.precision != JV_BF16 && opt.precision != JV_FP16)
        return bad(JV_EINVAL, "precision must be JV_FP32, JV_BF16 or JV_FP16");
    if ((opt.min_blocks != 0 && opt.min_blocks != 3 && opt.min_blocks != 4) ||
        (opt.pml_min_blocks != 0 && opt.pml_min_blocks != 3 && opt.pml_min_blocks != 4))
        return bad(JV_EINVAL, "min_blocks and pml_min_blocks must be 0, 3 or 4");
    if (opt.planes_per_thread < 0 || opt.planes_per_thread > 2 || opt.pml_planes_per_thread < 0 ||
        opt.pml_planes_per_thread > 2)
        return bad(JV_EINVAL, "planes_per_thread and pml_planes_per_thread must be 0, 1 or 2");
    if (opt.kernel_variant < -1 || opt.kernel_variant > 4)
        return bad(JV_EINVAL, "kernel_variant must be 0..4, or -1 (measured choice)");
    if (opt.tile_gx < 0 || opt.tile_gy < 0 || opt.tile_gx * std::max(opt.tile_gy, 1) > 256)
        return bad(JV_EINVAL, "tile_gx * tile_gy must be <= 256");
    long long next = (long long)(grid.nx + 2 * grid.pml) * (grid.ny + 2 * grid.pml) * (grid.nz + 2 * grid.pml);
    if (next > (1LL << 34)) return bad(JV_EINVAL, "grid too large");

    Engine *E = new Engine();
    E->grid_ = grid;
    E->opt_ = opt;
    E->opt_.rec_width = rw;
    if (E->opt_.graph_steps <= 0) E->opt_.graph_steps = 32;
    E->dt_ = dt;
    E->fm_ = fm;
    E->nt_ = nt;
    E->dev_ = opt.device;
    // -1: the resources of variant 4 (a superset of 3's and 2's), then the
    // measured choice after allocation
    const bool tune = opt.kernel_variant < 0;
    E->kc_.variant = tune ? 4 : opt.kernel_variant;
    E->kc_.zchunk = opt.zchunk;
    E->kc_.gx = opt.tile_gx;
    E->kc_.gy = opt.tile_gy;
    if (opt.min_blocks) E->kc_.minb = opt.min_blocks;
    if (opt.pml_min_blocks) E->kc_.pml_minb = opt.pml_min_blocks;
    if (opt.planes_per_thread) E->kc_.zp = opt.planes_per_thread;
    if (opt.pml_planes_per_thread) E->kc_.pml_zp = opt.pml_planes_per_thread;
    if (opt.run_chunks > 0) E->kc_.fzq = opt.run_chunks;
    const char *cf = std::getenv("JV_CHECK_FINITE");
    E->check_finite_ = cf && cf[0] == '1';
    Status s = E->alloc_all(vp, vs, rho);
    // measured at creation: the full choice with kernel_variant -1, else
    // (autotune on, nothing fixed by hand) the result-neutral knobs only
    const bool neutral = !tune && opt.autotune && opt.run_chunks <= 0 && opt.tile_gx <= 0 && opt.tile_gy <= 0;
    if (s && (tune || neutral)) s = E->autotune(!tune);
    if (!s) {
        delete E;
        return s;
    }
    *out = E;
    return Status{};
}

// The measured kernel choice (kernel_variant -1): a few forward-modelling
// steps of each candidate on this grid -- variant 4 where its kernels
// apply, with the cost model's three best run chunkings (unless run_chunks
// fixes one), variant 3 where its stress kernel applies, variant 2 -- and,
// for the variants with separate absorbing-layer kernels, their register
// budget (3 or 4 blocks per SM).  Then, unless tile_gx / tile_gy were
// given, the float4 kernels' block shape: the default number of blocks per
// gridphy row and one fewer or one more, timed on the reverse loop's
// float4 velocity update and the backward stress update (the forward step
// of a one-tile grid does not run them).  The fastest wins; the choice is
// kept per grid shape and device for the contexts that follow.
Status Engine::autotune(bool neutral) {
    struct Cand {
        int variant, pml_minb, q;  // q: variant 4's run chunks
        int gx = 0;                // float4 kernels' x groups per block (0: the default shape)
    };
    const bool shape_free = opt_.tile_gx <= 0 && opt_.tile_gy <= 0;
    static std::mutex mu;
    static std::map<std::array<long long, 7>, Cand> cache;
    int dev = 0;
    JV_CU(cudaGetDevice(&dev));
    cudaDeviceProp prop{};
    JV_CU(cudaGetDeviceProperties(&prop, dev));
    const std::array<long long, 7> key = {grid_.nx, grid_.ny, grid_.nz, grid_.pml, prop.multiProcessorCount,
                                          (long long)prop.totalGlobalMem, neutral ? 1 : 0};
    Status st{};
    auto apply = [&](const Cand &c) {
        kc_.variant = c.variant;
        kc_.pml_minb = c.pml_minb;
        if (shape_free) {
            kc_.gx = c.gx;
            kc_.gy = 0;
        }
        if (c.variant == 4 && fullF_.ok && c.q > 0 && c.q != fullF_.geo.Q) {
            kc_.fzq = c.q;
            const int e = k_make_full_maps(g_, F_, lam_, mu_, vp_, bdt_, axis_d_, fzpsiF_, zm_err_, kc_.fzq, &fullF_);
            if (e != 0 || !fullF_.ok) st = bad(JV_ECUDA, "variant-4 descriptors for the measured choice");
        }
        use_full_ = c.variant == 4 && fullF_.ok;
        vel_full_ = use_full_ && fullF_.geo.NTX == 1;
    };
    {
        std::lock_guard<std::mutex> l(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            apply(it->second);
            return st;
        }
    }
    std::vector<Cand> cands;
    if (fullF_.ok) {
        if (kc_.fzq > 0) {
            cands.push_back({4, 4, fullF_.geo.Q});
        } else {
            for (int k = 0; k < 3; k++)
                if (fullF_.qcand[k] > 0) cands.push_back({4, 4, fullF_.qcand[k]});
        }
    }
    if (neutral) {
        // only what cannot change a result: variant 4's run chunking (which
        // CTA updates which cells) and, below, the float4 kernels' block
        // shape (which thread updates which group)
        if (cands.empty()) cands.push_back({kc_.variant, kc_.pml_minb, 0});
    } else {
        if (mapsF_.ok) {
            cands.push_back({3, 4, 0});
            cands.push_back({3, 3, 0});
        }
        cands.push_back({2, 4, 0});
        cands.push_back({2, 3, 0});
    }
    const long long src = (long long)g_.xoff + (g_.m + g_.px / 2) + g_.sy * (g_.m + g_.py / 2) +
                          g_.sz * (g_.m + g_.pz / 2);
    float best = -1.f;
    Cand pick = cands[0];
    const int warm = 2, steps = 6;
    for (const Cand &c : cands) {
        if (cands.size() == 1) break;  // nothing to choose between
        apply(c);
        JV_TRY(st);
        JV_TRY(zero_wave(F_, 9));
        JV_TRY(zero_psi(cpF_));
        JV_TRY(set_state(0, src, nullptr, nullptr));
        for (int i = 0; i < warm; i++) JV_TRY(launch_step(kStepModel, 0, true));
        JV_CU(cudaEventRecord(ev0_, stream_));
        for (int i = 0; i < steps; i++) JV_TRY(launch_step(kStepModel, 0, true));
        JV_CU(cudaEventRecord(ev1_, stream_));
        JV_CU(cudaEventSynchronize(ev1_));
        JV_TRY(check_zm_err());
        float ms = 0.f;
        JV_CU(cudaEventElapsedTime(&ms, ev0_, ev1_));
        if (best < 0.f || ms < best) {
            best = ms;
            pick = c;
        }
    }
    apply(pick);
    JV_TRY(st);
    if (shape_free) {
        const int ngx = (g_.px + 3) / 4, nb0 = (ngx + 63) / 64;
        float sbest = -1.f;
        for (int nb = std::max(1, nb0 - 1); nb <= nb0 + 1; nb++) {
            const int gx = (ngx + nb - 1) / nb;
            if (gx > 256) continue;
            kc_.gx = nb == nb0 ? 0 : gx;
            kc_.gy = 0;
            JV_TRY(zero_wave(F_, kNumFld));
            JV_TRY(set_state(0, src, nullptr, nullptr));
            for (int i = 0; i < warm + steps; i++) {
                if (i == warm) JV_CU(cudaEventRecord(ev0_, stream_));
                JV_K(k_vel_phy(kRev, g_, F_, bdt_, dt_, opt_.rec_width, nullptr, nullptr, kc_, stream_));
                JV_K(k_stress_phy(kBwd, g_, F_, lam_, mu_, -dt_, opt_.rec_width, wavelet_, st_, 0, kc_, stream_,
                                  &mapsF_));
            }
            JV_CU(cudaEventRecord(ev1_, stream_));
            JV_CU(cudaEventSynchronize(ev1_));
            JV_TRY(check_zm_err());
            float ms = 0.f;
            JV_CU(cudaEventElapsedTime(&ms, ev0_, ev1_));
            if (sbest < 0.f || ms < sbest) {
                sbest = ms;
                pick.gx = kc_.gx;
            }
        }
        apply(pick);
    }
    JV_TRY(zero_wave(F_, kNumFld));
    JV_TRY(zero_psi(cpF_));
    JV_CU(cudaStreamSynchronize(stream_));
    std::lock_guard<std::mutex> l(mu);
    cache[key] = pick;
    return Status{};
}

Status Engine::alloc_all(const float *vp, const float *vs, const float *rho) {
    JV_CU(cudaSetDevice(dev_));
    JV_CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    JV_CU(cudaEventCreate(&ev0_));
    JV_CU(cudaEventCreate(&ev1_));

    // coefficient tables (universal constants; uploaded per device)
    JV_K(upload_all_coefficients());

    // pitched gridext layout
    g_ = make_layout(grid_, &field_elems_);
    if (field_elems_ >= (size_t)1 << 31) return bad(JV_EINVAL, "gridext too large for 32-bit element offsets");

    // model
    void *p;
    JV_TRY(alloc(&p, (4 * field_elems_ + kGuard) * sizeof(float)));
    JV_CU(cudaMemsetAsync(p, 0, (4 * field_elems_ + kGuard) * sizeof(float), stream_));
    float *mb = (float *)p + kGuard;
    vp_ = mb; bdt_ = mb + field_elems_; lam_ = mb + 2 * field_elems_; mu_ = mb + 3 * field_elems_;
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    JV_TRY(upload_model(vp, vs, rho));

    // forward/backward wavefield (13 components, one arena)
    JV_TRY(alloc(&p, (kNumFld * field_elems_ + kGuard) * sizeof(float)));
    JV_CU(cudaMemsetAsync(p, 0, kGuard * sizeof(float), stream_));
    for (int f = 0; f < kNumFld; f++) F_.f[f] = (float *)p + kGuard + f * field_elems_;
    if (kc_.variant >= 3) {
        JV_TRY(alloc(&p, sizeof(int)));
        zm_err_ = (int *)p;
        JV_CU(cudaMemsetAsync(zm_err_, 0, sizeof(int), stream_));
        JV_K(k_make_wave_maps(g_, F_, lam_, mu_, zm_err_, &mapsF_));
    }

    // CPML geometry: six slabs covering gridext outside gridphy and outside
    // the 2-cell outer rim; the slab table and axis tables are shared by
    // both wavefields, the memory-variable arenas are per wavefield
    {
        cpml_proto_ = make_pml_slabs(g_, kc_.pml_zp, &psi_total_);
        std::vector<float4> t[3];
        pml_axis_tables(g_, fm_, t);
        for (int a = 0; a < 3; a++) {
            JV_TRY(alloc(&p, t[a].size() * sizeof(float4)));
            axis_d_[a] = (float4 *)p;
            JV_CU(cudaMemcpy(axis_d_[a], t[a].data(), t[a].size() * sizeof(float4), cudaMemcpyHostToDevice));
        }
        JV_TRY(alloc(&p, (size_t)psi_total_ * sizeof(float)));
        cpF_ = make_cpml((float *)p);
    }
    if (kc_.variant == 4) {
        fz_psi_total_ = 2 * fz_psi_floats(g_);  // velocity and stress sets
        JV_TRY(alloc(&p, (size_t)fz_psi_total_ * sizeof(float)));
        fzpsiF_ = (float *)p;
        JV_K(k_make_full_maps(g_, F_, lam_, mu_, vp_, bdt_, axis_d_, fzpsiF_, zm_err_, kc_.fzq, &fullF_));
        // the fused velocity update runs on one-tile grids, where it measured
        // faster than the split kernels; x-tiled grids keep the split ones
        use_full_ = fullF_.ok;
        vel_full_ = fullF_.ok && fullF_.geo.NTX == 1;
    }

    // wavelet and step state
    std::vector<float> w(nt_);
    ricker(nt_, fm_, dt_, w.data());
    JV_TRY(alloc(&p, nt_ * sizeof(float)));
    wavelet_ = (float *)p;
    JV_CU(cudaMemcpy(wavelet_, w.data(), nt_ * sizeof(float), cudaMemcpyHostToDevice));
    JV_TRY(alloc(&p, sizeof(StepState)));
    st_ = (StepState *)p;

    // images
    JV_TRY(alloc(&p, 5 * nphy * sizeof(double)));
    double *ib = (double *)p;
    img_.ip = ib; img_.pp = ib + nphy; img_.ps = ib + 2 * nphy; img_.sp = ib + 3 * nphy; img_.ss = ib + 4 * nphy;
    JV_CU(cudaMemsetAsync(ib, 0, 5 * nphy * sizeof(double), stream_));

    // VOWR face boxes
    {
        long long off = 0, blk = 0;
        segs_h_ = vowr_segments(g_, opt_.rec_width, &off, &blk, opt_.precision == JV_FP32);
        per_step_ = off;
        if (blk >= (1LL << 31) || per_step_ >= (1LL << 31)) return bad(JV_EINVAL, "boundary store too large");
        nslot_ = nt_ > 1 ? nt_ - 1 : 0;
        vowr_ = VowrDev{};
        vowr_.per_step = per_step_;
        vowr_.nslot = nslot_;
        vowr_.prec = opt_.precision;
        vowr_.nseg = (int)segs_h_.size();
        vowr_.all_blocks = (int)blk;
        if (segs_h_.size() > (size_t)kVowrMaxSegs) return bad(JV_EINVAL, "too many boundary boxes");
        for (size_t q = 0; q < segs_h_.size(); q++) {
            const SegDev &S = segs_h_[q];
            vowr_.seg[q] = S;
            const long long nb = ((long long)S.nxb * S.nyb * S.nzb + 256LL * S.vw - 1) / (256LL * S.vw);
            if (S.fld <= VZ) vowr_.vel_blocks = (int)(S.nblk_first + nb);
        }
    }
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}

// vp, vs, rho (host, gridphy) -> the extended model and lambda, mu on the
// device, in the buffers every kernel and tensor map of the context uses
Status Engine::upload_model(const float *vp, const float *vs, const float *rho) {
    if (!vp || !vs || !rho) return bad(JV_EINVAL, "model arrays must not be NULL");
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    float *tmp = nullptr;
    JV_CU(cudaMallocAsync(&tmp, 3 * nphy * sizeof(float), stream_));
    cudaError_t e1 = cudaMemcpyAsync(tmp, vp, nphy * sizeof(float), cudaMemcpyHostToDevice, stream_);
    cudaError_t e2 = cudaMemcpyAsync(tmp + nphy, vs, nphy * sizeof(float), cudaMemcpyHostToDevice, stream_);
    cudaError_t e3 = cudaMemcpyAsync(tmp + 2 * nphy, rho, nphy * sizeof(float), cudaMemcpyHostToDevice, stream_);
    int ek = k_model_prep(g_, tmp, tmp + nphy, tmp + 2 * nphy, dt_, vp_, bdt_, lam_, mu_, stream_);
    cudaFreeAsync(tmp, stream_);
    cudaError_t e4 = cudaStreamSynchronize(stream_);
    JV_CU(e1); JV_CU(e2); JV_CU(e3); JV_K(ek); JV_CU(e4);
    return Status{};
}

Status Engine::set_model(const float *vp, const float *vs, const float *rho) {
    JV_CU(cudaSetDevice(dev_));
    JV_CU(cudaStreamSynchronize(stream_));
    return upload_model(vp, vs, rho);
}

Status Engine::set_geometry(int n_shot, const float *shot_xyz, int n_recv, const float *recv_xyz) {
    if (n_shot < 0 || n_recv < 0 || (n_shot > 0 && !shot_xyz) || (n_recv > 0 && !recv_xyz))
        return bad(JV_EINVAL, "bad geometry arguments");
    JV_CU(cudaSetDevice(dev_));
    JV_CU(cudaStreamSynchronize(stream_));
    shots_.assign(shot_xyz, shot_xyz + 3 * (size_t)n_shot);
    nshot_ = n_shot;
    // receivers inside gridphy, file order (jarvis_device_geometry_meat.hpp:98-127)
    const float rx = (float)(grid_.nx - 1) * grid_.dx, ry = (float)(grid_.ny - 1) * grid_.dy,
                rz = (float)(grid_.nz - 1) * grid_.dz;
    const float lx = -(float)grid_.pml * grid_.dx, ly = -(float)grid_.pml * grid_.dy, lz = -(float)grid_.pml * grid_.dz;
    rec_h_.clear();
    for (int r = 0; r < n_recv; r++) {
        const float *q = recv_xyz + 3 * r;
        if (!(q[0] >= 0.0f && q[0] <= rx && q[1] >= 0.0f && q[1] <= ry && q[2] >= 0.0f && q[2] <= rz)) continue;
        int i = gap_num(lx, q[0], grid_.dx), j = gap_num(ly, q[1], grid_.dy), k = gap_num(lz, q[2], grid_.dz);
        rec_h_.push_back(g_.xoff + i + g_.sy * j + g_.sz * k);
    }
    // the same receiver count: the indices go into the buffer the captured
    // graphs already read, and the graphs stay valid
    if (rec_d_ && (int)rec_h_.size() == nrec_) {
        JV_CU(cudaMemcpy(rec_d_, rec_h_.data(), nrec_ * sizeof(long long), cudaMemcpyHostToDevice));
        return Status{};
    }
    if (!rec_d_ && rec_h_.empty() && nrec_ == 0) return Status{};
    nrec_ = (int)rec_h_.size();
    if (rec_d_) {
        cudaFreeAsync(rec_d_, stream_);
        cudaStreamSynchronize(stream_);
        for (auto &a : allocs_)
            if (a == rec_d_) a = nullptr;
        rec_d_ = nullptr;
    }
    if (nrec_ > 0) {
        void *p;
        JV_TRY(alloc(&p, nrec_ * sizeof(long long)));
        rec_d_ = (long long *)p;
        JV_CU(cudaMemcpy(rec_d_, rec_h_.data(), nrec_ * sizeof(long long), cudaMemcpyHostToDevice));
    }
    // the graphs bake the receiver count and pointer
    for (auto &kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    return Status{};
}

Status Engine::check_shot(int shot, long long *src) const {
    if (shot < 0 || shot >= nshot_) return bad(JV_EINVAL, "shot index out of range");
    const float *q = &shots_[3 * (size_t)shot];
    const float rx = (float)(grid_.nx - 1) * grid_.dx, ry = (float)(grid_.ny - 1) * grid_.dy,
                rz = (float)(grid_.nz - 1) * grid_.dz;
    if (!(q[0] >= 0.0f && q[0] <= rx && q[1] >= 0.0f && q[1] <= ry && q[2] >= 0.0f && q[2] <= rz))
        return bad(JV_EINVAL, "shot " + std::to_string(shot) + " lies outside gridphy");
    const float lx = -(float)grid_.pml * grid_.dx, ly = -(float)grid_.pml * grid_.dy, lz = -(float)grid_.pml * grid_.dz;
    int i = gap_num(lx, q[0], grid_.dx), j = gap_num(ly, q[1], grid_.dy), k = gap_num(lz, q[2], grid_.dz);
    *src = g_.xoff + i + g_.sy * j + g_.sz * k;
    return Status{};
}

Status Engine::set_state(int it, long long src, float *const tr[3], const float *const obs[3]) {
    StepState &h = h_state_;
    h = StepState{};
    h.it = it;
    h.src = src;
    for (int q = 0; q < 3; q++) {
        h.tr[q] = tr ? tr[q] : nullptr;
        h.obs[q] = obs ? obs[q] : nullptr;
    }
    JV_CU(cudaMemcpyAsync(st_, &h, sizeof(h), cudaMemcpyHostToDevice, stream_));
    return Status{};
}

Status Engine::zero_wave(const WaveDev &w, int nfld) {
    JV_CU(cudaMemsetAsync(w.f[0], 0, (size_t)nfld * field_elems_ * sizeof(float), stream_));
    return Status{};
}

CpmlDev Engine::make_cpml(float *psi) const {
    CpmlDev c = cpml_proto_;
    c.dt = dt_;
    for (int a = 0; a < 3; a++) c.ax[a] = axis_d_[a];
    c.psi = psi;
    return c;
}

Status Engine::zero_psi(const CpmlDev &c) {
    if (psi_total_ > 0) JV_CU(cudaMemsetAsync(c.psi, 0, (size_t)psi_total_ * sizeof(float), stream_));
    // the axis-major stress memory variables of the full-gridext kernel
    float *fz = c.psi == cpF_.psi ? fzpsiF_ : c.psi == cpR_.psi ? fzpsiR_ : nullptr;
    if (fz) JV_CU(cudaMemsetAsync(fz, 0, (size_t)fz_psi_total_ * sizeof(float), stream_));
    return Status{};
}

// ------------------------------------------------------------ stepping

int Engine::prof_id(const char *name) {
    for (size_t i = 0; i < prof_names_.size(); i++)
        if (prof_names_[i] == name) return (int)i;
    prof_names_.push_back(name);
    prof_ms_.push_back(0.0);
    prof_n_.push_back(0);
    return (int)prof_names_.size() - 1;
}

cudaEvent_t Engine::prof_event() {
    if (prof_used_ == prof_pool_.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        prof_pool_.push_back(e);
    }
    return prof_pool_[prof_used_++];
}

Status Engine::prof_collect() {
    if (prof_pending_.empty()) return Status{};
    JV_CU(cudaStreamSynchronize(stream_));
    for (const ProfRec &r : prof_pending_) {
        float ms = 0.f;
        JV_CU(cudaEventElapsedTime(&ms, r.a, r.b));
        prof_ms_[r.id] += ms;
        prof_n_[r.id] += 1;
    }
    prof_pending_.clear();
    prof_used_ = 0;
    return Status{};
}

void Engine::set_profiling(bool on) {
    prof_ = on;
    prof_names_.clear();
    prof_ms_.clear();
    prof_n_.clear();
    prof_pending_.clear();
    prof_used_ = 0;
}

bool Engine::profile_entry(int i, const char **name, double *ms, long long *launches) const {
    if (i < 0 || i >= (int)prof_names_.size()) return false;
    *name = prof_names_[i].c_str();
    *ms = prof_ms_[i];
    *launches = prof_n_[i];
    return true;
}

Status Engine::check_finite(const char *after) {
    if (!nf_) {
        void *p;
        JV_TRY(alloc(&p, 8 * sizeof(unsigned long long)));
        nf_ = (unsigned long long *)p;
    }
    JV_CU(cudaMemsetAsync(nf_, 0, 8 * sizeof(unsigned long long), stream_));
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    JV_K(k_count_nonfinite(F_.f[0], kNumFld * field_elems_, 0, nf_ + 0, stream_));
    if (R_.f[0]) JV_K(k_count_nonfinite(R_.f[0], kNumFld * field_elems_, 0, nf_ + 1, stream_));
    JV_K(k_count_nonfinite(img_.ip, 5 * nphy, 1, nf_ + 2, stream_));
    if (shot_img_.ip) JV_K(k_count_nonfinite(shot_img_.ip, 5 * shot_img_pitch_, 0, nf_ + 2, stream_));
    unsigned long long h[8];
    JV_CU(cudaMemcpyAsync(h, nf_, sizeof(h), cudaMemcpyDeviceToHost, stream_));
    JV_CU(cudaStreamSynchronize(stream_));
    if (h[0] || h[1] || h[2]) {
        StepState sh;
        JV_CU(cudaMemcpy(&sh, st_, sizeof(sh), cudaMemcpyDeviceToHost));
        int fld[2] = {-1, -1};
        for (int w = 0; w < 2; w++) {
            const WaveDev &W = w == 0 ? F_ : R_;
            if (!h[w] || !W.f[0]) continue;
            for (int f = 0; f < kNumFld && fld[w] < 0; f++) {
                JV_CU(cudaMemsetAsync(nf_ + 4, 0, sizeof(unsigned long long), stream_));
                JV_K(k_count_nonfinite(W.f[f], field_elems_, 0, nf_ + 4, stream_));
                unsigned long long c = 0;
                JV_CU(cudaMemcpy(&c, nf_ + 4, sizeof(c), cudaMemcpyDeviceToHost));
                if (c) fld[w] = f;
            }
        }
        return bad(JV_ECUDA, std::string("non-finite values after ") + after + " (step kind " +
                                 std::to_string(cur_kind_) + ", it " + std::to_string(sh.it) +
                                 "): F " + std::to_string(h[0]) + " (first field " + std::to_string(fld[0]) +
                                 "), R " + std::to_string(h[1]) + " (first field " + std::to_string(fld[1]) +
                                 "), images " + std::to_string(h[2]));
    }
    return Status{};
}

// launch one kernel, bracketed by timing events when profiling
#define JV_L(name, expr)                                                    \
    do {                                                                    \
        if (prof_) {                                                        \
            ProfRec _r{prof_id(name), prof_event(), prof_event()};          \
            JV_CU(cudaEventRecord(_r.a, stream_));                          \
            JV_K(expr);                                                     \
            JV_CU(cudaEventRecord(_r.b, stream_));                          \
            prof_pending_.push_back(_r);                                    \
        } else {                                                            \
            JV_K(expr);                                                     \
        }                                                                   \
        if (check_finite_) JV_TRY(check_finite(name));                      \
    } while (0)

// The kernels of one time step of `kind`.  They read the time step as
// st_->it + off; advance == true ends the step with st_->it += direction.
Status Engine::launch_step(int kind, int off, bool advance) {
    cur_kind_ = kind;
    void *s = (void *)stream_;
    const float dt = dt_;
    const int rw = opt_.rec_width;
    switch (kind) {
    case kStepModel:
        if (vel_full_) {
            JV_L("vel_fz_fwd", k_vel_full(g_, F_, dt, fullF_, s));
        } else {
            JV_L("vel_pml", k_vel_pml(g_, cpF_, F_, bdt_, vp_, kc_, s));
            JV_L("vel_phy_fwd", k_vel_phy(kFwd, g_, F_, bdt_, dt, rw, nullptr, nullptr, kc_, s));
        }
        if (use_full_) {
            JV_L("stress_fz_fwd", k_stress_full(kFwd, g_, F_, dt, wavelet_, st_, off, fullF_, s));
        } else {
            JV_L("stress_pml", k_stress_pml(g_, cpF_, F_, lam_, mu_, vp_, 0, kc_, s));
            JV_L("stress_phy_fwd",
                 k_stress_phy(kFwd, g_, F_, lam_, mu_, dt, rw, wavelet_, st_, off, kc_, s, &mapsF_));
        }
        JV_L("record", k_record(F_, rec_d_, nrec_, nt_, st_, off, s));
        if (advance) JV_L("step_advance", k_step_advance(st_, +1, s));
        break;
    case kStepRtmFwd:
        if (vel_full_) {
            JV_L("vel_fz_rtmfwd", k_vel_full(g_, F_, dt, fullF_, s));
        } else {
            JV_L("vel_pml", k_vel_pml(g_, cpF_, F_, bdt_, vp_, kc_, s));
            JV_L("vel_phy_rtmfwd", k_vel_phy(kRtmFwd, g_, F_, bdt_, dt, rw, nullptr, nullptr, kc_, s));
        }
        if (use_full_) {
            // the boundary boxes lie in the absorbing layers: pack them after their update
            JV_L("stress_fz_rtmfwd", k_stress_full(kRtmFwd, g_, F_, dt, wavelet_, st_, off, fullF_, s));
            JV_L("vowr_pack", k_vowr(g_, F_, vowr_, st_, off, 1, 0, s));
        } else {
            JV_L("stress_pml_sau", k_stress_pml(g_, cpF_, F_, lam_, mu_, vp_, 1, kc_, s));
            JV_L("vowr_pack", k_vowr(g_, F_, vowr_, st_, off, 1, 0, s));
            JV_L("stress_phy_rtmfwd",
                 k_stress_phy(kRtmFwd, g_, F_, lam_, mu_, dt, rw, wavelet_, st_, off, kc_, s, &mapsF_));
        }
        if (advance) JV_L("step_advance", k_step_advance(st_, +1, s));
        break;
    case kStepRtmRev:
        // UPDATE 1: source subtraction (fused) + backward stress, receiver
        // injection + reverse velocity, stress boundary layers of step it-1
        JV_L("inject_rec", k_inject_rec(R_, rec_d_, nrec_, nt_, st_, off, s));
        JV_L("stress_phy_bwd", k_stress_phy(kBwd, g_, F_, lam_, mu_, -dt, rw, wavelet_, st_, off, kc_, s, &mapsF_));
        // the receiver side's velocity update: absorbing layers, then gridphy
        // (with its P-wave velocities, the full-gridext form measured no
        // faster on cfg2 and slower on x-tiled grids)
        JV_L("vel_pml", k_vel_pml(g_, cpR_, R_, bdt_, vp_, kc_, s));
        JV_L("vel_phy_rev", k_vel_phy(kRev, g_, R_, bdt_, dt, rw, nullptr, nullptr, kc_, s));
        JV_L("vowr_unpack", k_vowr(g_, F_, vowr_, st_, off - 1, 0, 2, s));
        // UPDATE 2: backward velocity with the imaging condition fused,
        // reverse stress, velocity boundary layers of step it-1
        JV_L("vel_phy_bwd_image", k_vel_phy(kBwd, g_, F_, bdt_, -dt, rw, &R_, &shot_img_, kc_, s));
        if (fullR_.ok) {
            JV_L("stress_fz_rev", k_stress_full(kRev, g_, R_, dt, wavelet_, st_, off, fullR_, s));
        } else {
            JV_L("stress_pml_sau", k_stress_pml(g_, cpR_, R_, lam_, mu_, vp_, 1, kc_, s));
            JV_L("stress_phy_rev",
                 k_stress_phy(kRev, g_, R_, lam_, mu_, dt, rw, wavelet_, st_, off, kc_, s, &mapsR_));
        }
        JV_L("vowr_unpack", k_vowr(g_, F_, vowr_, st_, off - 1, 0, 1, s));
        if (advance) JV_L("step_advance", k_step_advance(st_, -1, s));
        break;
    default: return bad(JV_EINVAL, "unknown step kind");
    }
    return Status{};
}

Status Engine::run_loop(int kind, int nsteps) {
    if (nsteps <= 0) return Status{};
    if (!opt_.use_graphs || prof_ || check_finite_) {
        for (int i = 0; i < nsteps; i++) {
            JV_TRY(launch_step(kind, 0, true));
            if (prof_ && prof_pending_.size() > 4096) JV_TRY(prof_collect());
        }
        if (prof_) JV_TRY(prof_collect());
        return Status{};
    }
    const int S = opt_.graph_steps;
    auto get = [&](int steps, cudaGraphExec_t *ex) -> Status {
        long long key = (long long)kind * 1000000LL + steps;
        auto it = graphs_.find(key);
        if (it != graphs_.end()) {
            *ex = it->second;
            return Status{};
        }
        cudaGraph_t gr;
        JV_CU(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        Status st;
        // one capture of `steps` time steps: step i reads st_->it + dir*i,
        // and one advance by dir*steps ends the chunk
        const int dir = kind == kStepRtmRev ? -1 : +1;
        for (int i = 0; i < steps && st; i++) st = launch_step(kind, dir * i, false);
        if (st) {
            int ek = k_step_advance(st_, dir * steps, stream_);
            if (ek != 0) st = bad(JV_ECUDA, std::string("step_advance: ") + cudaGetErrorString((cudaError_t)ek));
        }
        cudaError_t e = cudaStreamEndCapture(stream_, &gr);
        if (!st) {
            if (e == cudaSuccess) cudaGraphDestroy(gr);
            return st;
        }
        JV_CU(e);
        cudaError_t ei = cudaGraphInstantiate(ex, gr, 0);
        cudaGraphDestroy(gr);
        JV_CU(ei);
        graphs_[key] = *ex;
        return Status{};
    };
    const int full = nsteps / S, rem = nsteps % S;
    if (full > 0) {
        cudaGraphExec_t ex;
        JV_TRY(get(S, &ex));
        for (int i = 0; i < full; i++) JV_CU(cudaGraphLaunch(ex, stream_));
    }
    if (rem > 0) {
        cudaGraphExec_t ex;
        JV_TRY(get(rem, &ex));
        JV_CU(cudaGraphLaunch(ex, stream_));
    }
    return Status{};
}

// ------------------------------------------------------------ public ops

Status Engine::forward(int shot, float *d_vx, float *d_vy, float *d_vz) {
    JV_CU(cudaSetDevice(dev_));
    long long src;
    JV_TRY(check_shot(shot, &src));
    float *tr[3] = {d_vx, d_vy, d_vz};
    JV_CU(cudaEventRecord(ev0_, stream_));
    JV_TRY(zero_wave(F_, 9));
    JV_TRY(zero_psi(cpF_));
    JV_TRY(set_state(0, src, tr, nullptr));
    JV_TRY(run_loop(kStepModel, nt_));
    JV_CU(cudaEventRecord(ev1_, stream_));
    JV_CU(cudaEventSynchronize(ev1_));
    JV_CU(cudaGetLastError());
    JV_TRY(check_zm_err());
    float ms = 0.f;
    JV_CU(cudaEventElapsedTime(&ms, ev0_, ev1_));
    last_ms_ = ms;
    return Status{};
}

// Device memory the RTM passes need beyond modelling, allocated with the
// first RTM shot: the receiver wavefield, the FP32 shot image, the VOWR
// boundary store and the two energies of the reconstruction check.
Status Engine::rtm_prepare() {
    // lazily allocate the receiver wavefield and the boundary store
    if (!R_.f[0]) {
        void *p;
        JV_TRY(alloc(&p, (kNumFld * field_elems_ + kGuard) * sizeof(float)));
        JV_CU(cudaMemsetAsync(p, 0, kGuard * sizeof(float), stream_));
        for (int f = 0; f < kNumFld; f++) R_.f[f] = (float *)p + kGuard + f * field_elems_;
        if (kc_.variant >= 3) JV_K(k_make_wave_maps(g_, R_, lam_, mu_, zm_err_, &mapsR_));
        JV_TRY(alloc(&p, (size_t)psi_total_ * sizeof(float)));
        cpR_ = make_cpml((float *)p);
        if (kc_.variant == 4) {
            JV_TRY(alloc(&p, (size_t)fz_psi_total_ * sizeof(float)));
            fzpsiR_ = (float *)p;
            JV_K(k_make_full_maps(g_, R_, lam_, mu_, vp_, bdt_, axis_d_, fzpsiR_, zm_err_, kc_.fzq, &fullR_));
        }
    }
    if (!shot_img_.ip) {
        // five arrays at a pitch of whole 256-byte lines, so that every
        // array starts 16-byte aligned (the image update uses float4 access)
        void *p;
        const size_t pitch = (size_t)round_up((long long)g_.px * g_.py * g_.pz, 64);
        JV_TRY(alloc(&p, 5 * pitch * sizeof(float)));
        float *b = (float *)p;
        shot_img_.ip = b; shot_img_.pp = b + pitch; shot_img_.ps = b + 2 * pitch; shot_img_.sp = b + 3 * pitch;
        shot_img_.ss = b + 4 * pitch;
        shot_img_pitch_ = pitch;
    }
    if (!store_ && !vowr_.store16 && per_step_ > 0 && nslot_ > 0) {
        const bool s16 = vowr_.prec != JV_FP32;
        size_t bytes = (size_t)per_step_ * nslot_ * (s16 ? sizeof(uint16_t) : sizeof(float));
        if (s16) bytes += (size_t)vowr_.nseg * (nslot_ + 2) * sizeof(float);
        size_t freeb = 0, totalb = 0;
        JV_CU(cudaMemGetInfo(&freeb, &totalb));
        size_t budget = opt_.store_budget ? opt_.store_budget : (freeb > (2ULL << 30) ? freeb - (2ULL << 30) : 0);
        const size_t nrec = (size_t)per_step_ * nslot_;
        const size_t rec_bytes = nrec * (s16 ? sizeof(uint16_t) : sizeof(float));
        // placement: the device when the store fits its budget, else (or
        // when asked) pinned host memory mapped into the device's address
        // space -- the pack and unpack kernels then write and read it across
        // the host link, each step's record in one contiguous range
        const bool on_host = opt_.store_mode == JV_STORE_HOST || (opt_.store_mode != JV_STORE_DEVICE && bytes > budget);
        if (!on_host && bytes > budget)
            return bad(JV_ENOMEM, "boundary store of " + std::to_string(bytes) + " bytes does not fit the device budget of " +
                                      std::to_string(budget) + " bytes (store_mode JV_STORE_HOST keeps it in host memory)");
        void *rec = nullptr, *p;
        if (on_host) {
            void *h = nullptr;
            cudaError_t e = cudaHostAlloc(&h, rec_bytes, cudaHostAllocMapped | cudaHostAllocPortable);
            if (e != cudaSuccess) {
                cudaGetLastError();
                return bad(JV_ENOMEM, "pinned host allocation of " + std::to_string(rec_bytes) +
                                          " bytes for the boundary store failed: " + cudaGetErrorString(e));
            }
            host_store_ = h;
            JV_CU(cudaHostGetDevicePointer(&rec, h, 0));
        } else {
            JV_TRY(alloc(&rec, rec_bytes));
        }
        store_on_host_ = on_host;
        if (s16) {
            // 16-bit records; on the device one FP32 scale per box and step,
            // then the two rows of largest magnitudes
            JV_TRY(alloc(&p, (size_t)vowr_.nseg * (nslot_ + 2) * sizeof(float)));
            vowr_.store16 = (uint16_t *)rec;
            vowr_.scales = (float *)p;
            vowr_.amax = (unsigned *)(vowr_.scales + (size_t)vowr_.nseg * nslot_);
            JV_CU(cudaMemsetAsync(vowr_.amax, 0, 2 * (size_t)vowr_.nseg * sizeof(unsigned), stream_));
        } else {
            store_ = (float *)rec;
            vowr_.store = store_;
        }
    }
    if (!energy_d_) {
        void *p;
        JV_TRY(alloc(&p, 2 * sizeof(double)));
        energy_d_ = (double *)p;
    }
    return Status{};
}

Status Engine::rtm_forward_pass(int shot) {
    JV_CU(cudaSetDevice(dev_));
    long long src;
    JV_TRY(check_shot(shot, &src));
    JV_TRY(rtm_prepare());
    // forward with boundary store (rtm_forward)
    JV_TRY(zero_wave(F_, kNumFld));
    JV_TRY(zero_psi(cpF_));
    JV_TRY(set_state(0, src, nullptr, nullptr));
    JV_TRY(run_loop(kStepRtmFwd, nt_));
    // reconstruction check: the source wavefield's FP64 energy over gridphy
    // where the reconstruction starts (and, at the end of the reverse loop,
    // what is left of it once carried back to its zero initial state)
    JV_CU(cudaMemsetAsync(energy_d_, 0, 2 * sizeof(double), stream_));
    JV_K(k_wave_energy(g_, F_, energy_d_, stream_));
    fwd_shot_ = shot;
    return Status{};
}

Status Engine::rtm_reverse_begin(int shot, const float *d_ox, const float *d_oy, const float *d_oz) {
    JV_CU(cudaSetDevice(dev_));
    long long src;
    JV_TRY(check_shot(shot, &src));
    if (nrec_ > 0 && (!d_ox || !d_oy || !d_oz)) return bad(JV_EINVAL, "observed traces must not be NULL");
    if (fwd_shot_ != shot) return bad(JV_ESTATE, "the time-reverse loop needs the forward pass of the same shot first");
    const float *obs[3] = {d_ox, d_oy, d_oz};
    // time reverse: backward (reconstruction) + reverse (receivers) + image
    JV_TRY(zero_wave(R_, kNumFld));
    JV_TRY(zero_psi(cpR_));
    JV_TRY(set_state(nt_ - 1, src, nullptr, obs));
    JV_CU(cudaMemsetAsync(shot_img_.ip, 0, 5 * shot_img_pitch_ * sizeof(float), stream_));
    rev_open_ = true;
    return Status{};
}

// One kernel of the time-reverse loop at time index `it` (for the boundary
// replays, the index of the record replayed), launched directly; the loop
// of rtm_shot launches the same kernels per step (launch_step kStepRtmRev).
Status Engine::rtm_reverse_op(int op, int it) {
    if (!rev_open_) return bad(JV_ESTATE, "no time-reverse loop is open (jv_rtm_reverse_begin)");
    JV_CU(cudaSetDevice(dev_));
    h_state_.it = it;
    JV_CU(cudaMemcpyAsync(st_, &h_state_, sizeof(h_state_), cudaMemcpyHostToDevice, stream_));
    void *s = (void *)stream_;
    const float dt = dt_;
    const int rw = opt_.rec_width;
    switch (op) {
    case JV_OP_INJECT_RECEIVERS: JV_K(k_inject_rec(R_, rec_d_, nrec_, nt_, st_, 0, s)); break;
    case JV_OP_BACKWARD_STRESS:
        JV_K(k_stress_phy(kBwd, g_, F_, lam_, mu_, -dt, rw, wavelet_, st_, 0, kc_, s, &mapsF_));
        break;
    case JV_OP_REVERSE_VEL_PML: JV_K(k_vel_pml(g_, cpR_, R_, bdt_, vp_, kc_, s)); break;
    case JV_OP_REVERSE_VEL: JV_K(k_vel_phy(kRev, g_, R_, bdt_, dt, rw, nullptr, nullptr, kc_, s)); break;
    case JV_OP_INJECT_BOUNDARY_STRESS: JV_K(k_vowr(g_, F_, vowr_, st_, 0, 0, 2, s)); break;
    case JV_OP_BACKWARD_VEL_IMAGE: JV_K(k_vel_phy(kBwd, g_, F_, bdt_, -dt, rw, &R_, &shot_img_, kc_, s)); break;
    case JV_OP_REVERSE_STRESS_PML:
        // folded into the full-gridext stress kernel where that one runs
        if (!fullR_.ok) JV_K(k_stress_pml(g_, cpR_, R_, lam_, mu_, vp_, 1, kc_, s));
        break;
    case JV_OP_REVERSE_STRESS:
        if (fullR_.ok) JV_K(k_stress_full(kRev, g_, R_, dt, wavelet_, st_, 0, fullR_, s));
        else JV_K(k_stress_phy(kRev, g_, R_, lam_, mu_, dt, rw, wavelet_, st_, 0, kc_, s, &mapsR_));
        break;
    case JV_OP_INJECT_BOUNDARY_VEL: JV_K(k_vowr(g_, F_, vowr_, st_, 0, 0, 1, s)); break;
    default: return bad(JV_EINVAL, "unknown time-reverse operation");
    }
    return Status{};
}

// the end of the time-reverse loop, queued: the reconstruction check's
// second energy, the shot image added to the FP64 stacks, both energies
// copied to the host
Status Engine::reverse_end_launch() {
    if (!rev_open_) return bad(JV_ESTATE, "no time-reverse loop is open (jv_rtm_reverse_begin)");
    JV_CU(cudaSetDevice(dev_));
    rev_open_ = false;
    JV_K(k_wave_energy(g_, F_, energy_d_ + 1, stream_));
    JV_K(k_image_stack(g_, shot_img_, img_, stream_));
    JV_CU(cudaMemcpyAsync(recon_energy_, energy_d_, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    return Status{};
}

Status Engine::rtm_reverse_end() {
    JV_TRY(reverse_end_launch());
    JV_CU(cudaStreamSynchronize(stream_));
    JV_CU(cudaGetLastError());
    JV_TRY(check_zm_err());
    return Status{};
}

Status Engine::rtm_shot(int shot, const float *d_ox, const float *d_oy, const float *d_oz, cudaEvent_t obs_ready) {
    JV_CU(cudaSetDevice(dev_));
    long long src;
    JV_TRY(check_shot(shot, &src));
    if (nrec_ > 0 && (!d_ox || !d_oy || !d_oz)) return bad(JV_EINVAL, "observed traces must not be NULL");
    JV_TRY(rtm_prepare());
    JV_CU(cudaEventRecord(ev0_, stream_));
    JV_TRY(rtm_forward_pass(shot));
    if (obs_ready) JV_CU(cudaStreamWaitEvent(stream_, obs_ready, 0));
    JV_TRY(rtm_reverse_begin(shot, d_ox, d_oy, d_oz));
    JV_TRY(run_loop(kStepRtmRev, nt_));
    JV_TRY(reverse_end_launch());
    JV_CU(cudaEventRecord(ev1_, stream_));
    JV_CU(cudaEventSynchronize(ev1_));
    JV_CU(cudaGetLastError());
    JV_TRY(check_zm_err());
    float ms = 0.f;
    JV_CU(cudaEventElapsedTime(&ms, ev0_, ev1_));
    last_ms_ = ms;
    return Status{};
}

Status Engine::image_reset() {
    JV_CU(cudaSetDevice(dev_));
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    JV_CU(cudaMemsetAsync(img_.ip, 0, 5 * nphy * sizeof(double), stream_));
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}

Status Engine::image_get(int kind, double *out) {
    JV_CU(cudaSetDevice(dev_));
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    double *src[5] = {img_.ip, img_.pp, img_.ps, img_.sp, img_.ss};
    if (kind < 0 || kind > 4 || !out) return bad(JV_EINVAL, "bad image kind / output");
    JV_CU(cudaMemcpyAsync(out, src[kind], nphy * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}

Status Engine::image_finalize(float *out[8]) {
    JV_CU(cudaSetDevice(dev_));
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    if (!fin_) {
        void *p;
        JV_TRY(alloc(&p, 8 * nphy * sizeof(float)));
        fin_ = (float *)p;
    }
    JV_K(k_image_finalize(g_, img_, fin_, stream_));
    for (int q = 0; q < 8; q++)
        if (out[q]) JV_CU(cudaMemcpyAsync(out[q], fin_ + q * nphy, nphy * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}

Status Engine::image_get_device(int kind, double *out) {
    JV_CU(cudaSetDevice(dev_));
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    double *src[5] = {img_.ip, img_.pp, img_.ps, img_.sp, img_.ss};
    if (kind < 0 || kind > 4 || !out) return bad(JV_EINVAL, "bad image kind / output");
    JV_CU(cudaMemcpyAsync(out, src[kind], nphy * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}

Status Engine::image_set(int kind, const double *src, bool src_on_device) {
    JV_CU(cudaSetDevice(dev_));
    const size_t nphy = (size_t)g_.px * g_.py * g_.pz;
    double *dst[5] = {img_.ip, img_.pp, img_.ps, img_.sp, img_.ss};
    if (kind < 0 || kind > 4 || !src) return bad(JV_EINVAL, "bad image kind / input");
    JV_CU(cudaMemcpyAsync(dst[kind], src, nphy * sizeof(double),
                          src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream_));
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}


Status Engine::check_zm_err() {
    if (!zm_err_) return Status{};
    int h = 0;
    JV_CU(cudaMemcpy(&h, zm_err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        JV_CU(cudaMemset(zm_err_, 0, sizeof(int)));
        return bad(JV_ETIMEOUT, "a shared-memory tile of the z-marching stress kernel did not arrive in time");
    }
    return Status{};
}

Status Engine::sync() {
    JV_CU(cudaSetDevice(dev_));
    JV_CU(cudaStreamSynchronize(stream_));
    return Status{};
}

void Engine::info(jv_info *i) const {
    memset(i, 0, sizeof(*i));
    i->grid = grid_;
    i->nt = nt_;
    i->n_shot = nshot_;
    i->n_recv = nrec_;
    i->rec_width = opt_.rec_width;
    i->precision = opt_.precision;
    i->n_ext = (long long)g_.nx * g_.ny * g_.nz;
    i->n_phy = (long long)g_.px * g_.py * g_.pz;
    i->store_bytes_per_step = (size_t)per_step_ * (opt_.precision == JV_FP32 ? sizeof(float) : sizeof(uint16_t));
    i->device_bytes = dev_bytes_;
    i->store_on_device = store_on_host_ ? 0 : 1;
}

}  // namespace jv
