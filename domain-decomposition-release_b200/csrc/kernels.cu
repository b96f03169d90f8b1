// kernels.cu -- sm_100a CUDA kernels of libjv: interior 8th-order staggered
// velocity/stress updates (with the rtm_backward variable-order rim and the
// fused imaging condition), the 4th-order CPML slab updates, receivers,
// VOWR pack/unpack, model preparation and the image epilogue.
//
// Reference kernels restated here (paths relative to the reference root,
// FD = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/
// elastic_1_fdtd3d_model_mpi, RTM = .../elastic_1_rtm3d_model_mpi):
//   interior velocity   FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_2_vel_kernel.hpp:7-2088
//   interior stress     FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_3_stress_kernel.hpp:7-1364
//   CPML                FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_2_kernel_device_{x,y,z}_meat.hpp
//   damping profile     FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_1_host_meat.hpp:147-620
//   receivers           FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:57-107
//   imaging             RTM/rtm3d_0_image_module/rtm3d_iamge_kernel.hpp:6-51,118-135,184-200
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "jv_internal.hpp"

namespace jv {

__constant__ float c_list[5][4];  // c_list[o] = staggered coefficients of half-order o (1..4)
__constant__ float c_dc2[2];      // half-order 2 (CPML)

namespace {

constexpr int kTX = 32, kTY = 8;

__device__ __forceinline__ float ld(const float *__restrict__ p, long long i) { return __ldg(p + i); }

// Dp f = sum_r c_r (f[i+(r+1)s] - f[i-rs]);  Dm f = sum_r c_r (f[i+rs] - f[i-(r+1)s])
template <int O>
__device__ __forceinline__ float dp(const float *__restrict__ f, long long i, long long s, const float *c) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < O; r++) t += c[r] * (ld(f, i + (r + 1) * s) - ld(f, i - r * s));
    return t;
}
template <int O>
__device__ __forceinline__ float dm(const float *__restrict__ f, long long i, long long s, const float *c) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < O; r++) t += c[r] * (ld(f, i + r * s) - ld(f, i - (r + 1) * s));
    return t;
}
// runtime order 1..4 (rtm_backward rim)
__device__ __forceinline__ float dpv(const float *__restrict__ f, long long i, long long s, const float *c, int o) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < 4; r++)
        if (r < o) t += c[r] * (ld(f, i + (r + 1) * s) - ld(f, i - r * s));
    return t;
}
__device__ __forceinline__ float dmv(const float *__restrict__ f, long long i, long long s, const float *c, int o) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < 4; r++)
        if (r < o) t += c[r] * (ld(f, i + r * s) - ld(f, i - (r + 1) * s));
    return t;
}

// Order of one axis in the rtm_backward rim: within 4 cells of a gridphy
// face the order drops to e+1 (e = distance to the face) but never below
// rec_width (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_2_vel_kernel.hpp:132-152,240-261).
__device__ __forceinline__ int rim_order(int p, int np, int w) {
    int e = p < kPhyHalf ? p : (np - 1 - p < kPhyHalf ? np - 1 - p : kPhyHalf);
    if (e >= kPhyHalf) return kPhyHalf;
    return e < w ? w : e + 1;
}

// dt / rho of a cell for a step of signed length dt, from the stored
// |dt| / rho (model_prep)
__device__ __forceinline__ float signed_bdt(float b, float dt) { return dt < 0.f ? -b : b; }

template <int MODE, bool IMG>
__global__ void __launch_bounds__(kTX *kTY) vel_phy(GridDev g, WaveDev w, const float *__restrict__ bdt, float dt,
                                                   int rec_w, WaveDev rv, ImageDev img) {
    const int pi = blockIdx.x * kTX + threadIdx.x;
    const int pj = blockIdx.y * kTY + threadIdx.y;
    const int pk = blockIdx.z;
    if (pi >= g.px || pj >= g.py) return;
    const long long sy = g.sy, sz = g.sz;
    const long long i = g.xoff + (pi + g.m) + sy * (pj + g.m) + sz * (pk + g.m);
    const float *sxx = w.f[SXX], *syy = w.f[SYY], *szz = w.f[SZZ];
    const float *sxy = w.f[SXY], *sxz = w.f[SXZ], *syz = w.f[SYZ];
    float sxx_x, syx_x, szx_x, sxy_y, syy_y, szy_y, sxz_z, syz_z, szz_z;
    float sau_x = 0.f, sau_y = 0.f, sau_z = 0.f;
    constexpr bool kP = (MODE == kBwd || MODE == kRev);
    if (MODE == kBwd) {
        const int ox = rim_order(pi, g.px, rec_w), oy = rim_order(pj, g.py, rec_w), oz = rim_order(pk, g.pz, rec_w);
        const float *cx = c_list[ox], *cy = c_list[oy], *cz = c_list[oz];
        sxx_x = dpv(sxx, i, 1, cx, ox);
        syx_x = dmv(sxy, i, 1, cx, ox);
        szx_x = dmv(sxz, i, 1, cx, ox);
        sxy_y = dmv(sxy, i, sy, cy, oy);
        syy_y = dpv(syy, i, sy, cy, oy);
        szy_y = dmv(syz, i, sy, cy, oy);
        sxz_z = dmv(sxz, i, sz, cz, oz);
        syz_z = dmv(syz, i, sz, cz, oz);
        szz_z = dpv(szz, i, sz, cz, oz);
        const float *sau = w.f[SAU];
        sau_x = dpv(sau, i, 1, cx, ox);
        sau_y = dpv(sau, i, sy, cy, oy);
        sau_z = dpv(sau, i, sz, cz, oz);
    } else {
        const float *c = c_list[kPhyHalf];
        sxx_x = dp<4>(sxx, i, 1, c);
        syx_x = dm<4>(sxy, i, 1, c);
        szx_x = dm<4>(sxz, i, 1, c);
        sxy_y = dm<4>(sxy, i, sy, c);
        syy_y = dp<4>(syy, i, sy, c);
        szy_y = dm<4>(syz, i, sy, c);
        sxz_z = dm<4>(sxz, i, sz, c);
        syz_z = dm<4>(syz, i, sz, c);
        szz_z = dp<4>(szz, i, sz, c);
        if (kP) {
            const float *sau = w.f[SAU];
            sau_x = dp<4>(sau, i, 1, c);
            sau_y = dp<4>(sau, i, sy, c);
            sau_z = dp<4>(sau, i, sz, c);
        }
    }
    const float dtr = signed_bdt(ld(bdt, i), dt);
    const float a = dtr / g.dx, b = dtr / g.dy, c = dtr / g.dz;
    const float vx = w.f[VX][i] + (a * sxx_x + b * sxy_y + c * sxz_z);
    const float vy = w.f[VY][i] + (a * syx_x + b * syy_y + c * syz_z);
    const float vz = w.f[VZ][i] + (a * szx_x + b * szy_y + c * szz_z);
    w.f[VX][i] = vx;
    w.f[VY][i] = vy;
    w.f[VZ][i] = vz;
    if (kP) {
        const float px = w.f[VXP][i] + a * sau_x;
        const float py = w.f[VYP][i] + b * sau_y;
        const float pz = w.f[VZP][i] + c * sau_z;
        w.f[VXP][i] = px;
        w.f[VYP][i] = py;
        w.f[VZP][i] = pz;
        if (IMG) {
            // zero-lag imaging: s = this (reconstructed source) wavefield,
            // r = the receiver wavefield, already advanced this step
            const float rpx = ld(rv.f[VXP], i), rpy = ld(rv.f[VYP], i), rpz = ld(rv.f[VZP], i);
            const float rsx = ld(rv.f[VX], i) - rpx, rsy = ld(rv.f[VY], i) - rpy, rsz = ld(rv.f[VZ], i) - rpz;
            const float ssx = vx - px, ssy = vy - py, ssz = vz - pz;
            const long long o = pi + (long long)g.px * (pj + (long long)g.py * pk);
            img.ip[o] += px * px + py * py + pz * pz;
            img.pp[o] += px * rpx + py * rpy + pz * rpz;
            img.ps[o] += px * rsx + py * rsy + pz * rsz;
            img.sp[o] += ssx * rpx + ssy * rpy + ssz * rpz;
            img.ss[o] += ssx * rsx + ssy * rsy + ssz * rsz;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(kTX *kTY) stress_phy(GridDev g, WaveDev w, const float *__restrict__ lam,
                                                      const float *__restrict__ mu, float dt, int rec_w,
                                                      const float *__restrict__ wavelet,
                                                      const StepState *__restrict__ st, int it_off) {
    const int pi = blockIdx.x * kTX + threadIdx.x;
    const int pj = blockIdx.y * kTY + threadIdx.y;
    const int pk = blockIdx.z;
    if (pi >= g.px || pj >= g.py) return;
    const long long sy = g.sy, sz = g.sz;
    const long long i = g.xoff + (pi + g.m) + sy * (pj + g.m) + sz * (pk + g.m);
    const float *vx = w.f[VX], *vy = w.f[VY], *vz = w.f[VZ];
    float vx_x, vy_x, vz_x, vx_y, vy_y, vz_y, vx_z, vy_z, vz_z;
    if (MODE == kBwd) {
        const int ox = rim_order(pi, g.px, rec_w), oy = rim_order(pj, g.py, rec_w), oz = rim_order(pk, g.pz, rec_w);
        const float *cx = c_list[ox], *cy = c_list[oy], *cz = c_list[oz];
        vx_x = dmv(vx, i, 1, cx, ox);
        vy_x = dpv(vy, i, 1, cx, ox);
        vz_x = dpv(vz, i, 1, cx, ox);
        vx_y = dpv(vx, i, sy, cy, oy);
        vy_y = dmv(vy, i, sy, cy, oy);
        vz_y = dpv(vz, i, sy, cy, oy);
        vx_z = dpv(vx, i, sz, cz, oz);
        vy_z = dpv(vy, i, sz, cz, oz);
        vz_z = dmv(vz, i, sz, cz, oz);
    } else {
        const float *c = c_list[kPhyHalf];
        vx_x = dm<4>(vx, i, 1, c);
        vy_x = dp<4>(vy, i, 1, c);
        vz_x = dp<4>(vz, i, 1, c);
        vx_y = dp<4>(vx, i, sy, c);
        vy_y = dm<4>(vy, i, sy, c);
        vz_y = dp<4>(vz, i, sy, c);
        vx_z = dp<4>(vx, i, sz, c);
        vy_z = dp<4>(vy, i, sz, c);
        vz_z = dm<4>(vz, i, sz, c);
    }
    const float a = dt / g.dx, b = dt / g.dy, c = dt / g.dz;
    const float l = ld(lam, i), m = ld(mu, i);
    const float l2m = l + 2.0f * m;
    float sxx = w.f[SXX][i], syy = w.f[SYY][i], szz = w.f[SZZ][i];
    if (MODE != kRev && i == st->src) {
        // explosive source, applied before the stress update of step it
        // (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_3_stress_kernel.hpp:1308-1364)
        const float s = wavelet[st->it + it_off];
        if (MODE == kBwd) {
            sxx -= s; syy -= s; szz -= s;
        } else {
            sxx += s; syy += s; szz += s;
        }
    }
    w.f[SXX][i] = sxx + (a * l2m * vx_x + b * l * vy_y + c * l * vz_z);
    w.f[SYY][i] = syy + (a * l * vx_x + b * l2m * vy_y + c * l * vz_z);
    w.f[SZZ][i] = szz + (a * l * vx_x + b * l * vy_y + c * l2m * vz_z);
    w.f[SXY][i] += a * m * vy_x + b * m * vx_y;
    w.f[SXZ][i] += a * m * vz_x + c * m * vx_z;
    w.f[SYZ][i] += b * m * vz_y + c * m * vy_z;
    if (MODE != kFwd) w.f[SAU][i] += a * l2m * vx_x + b * l2m * vy_y + c * l2m * vz_z;
}

// ------------------------------------------------- z-marching variants
//
// One thread per (x, y) column of a 32 x 8 tile, marching over a chunk of
// z planes.  The z-derivatives come from register windows holding planes
// k-4 .. k+4 of the fields that need them, so every value is loaded once
// per chunk; x/y neighbours are read through L1.

// window helpers: w[4] is plane k
__device__ __forceinline__ float win_dp(const float *w, const float *c, int o) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < 4; r++)
        if (r < o) t += c[r] * (w[4 + r + 1] - w[4 - r]);
    return t;
}
__device__ __forceinline__ float win_dm(const float *w, const float *c, int o) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < 4; r++)
        if (r < o) t += c[r] * (w[4 + r] - w[4 - r - 1]);
    return t;
}

template <int MODE, bool IMG>
__global__ void __launch_bounds__(kTX *kTY) vel_phy_zm(GridDev g, WaveDev w, const float *__restrict__ bdt, float dt,
                                                      int rec_w, WaveDev rv, ImageDev img, int zc) {
    const int pi = blockIdx.x * kTX + threadIdx.x;
    const int pj = blockIdx.y * kTY + threadIdx.y;
    const int k0 = blockIdx.z * zc;
    const int k1 = min(k0 + zc, g.pz);
    if (pi >= g.px || pj >= g.py || k0 >= k1) return;
    constexpr bool kP = (MODE == kBwd || MODE == kRev);
    const long long sy = g.sy, sz = g.sz;
    long long i = g.xoff + (pi + g.m) + sy * (pj + g.m) + sz * (k0 + g.m);
    const float *sxx = w.f[SXX], *syy = w.f[SYY], *szz = w.f[SZZ];
    const float *sxy = w.f[SXY], *sxz = w.f[SXZ], *syz = w.f[SYZ], *sau = w.f[SAU];
    float wzz[9], wxz[9], wyz[9], wau[9];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const long long o = i + (q - 4) * sz;
        wzz[q] = ld(szz, o);
        wxz[q] = ld(sxz, o);
        wyz[q] = ld(syz, o);
        if (kP) wau[q] = ld(sau, o);
    }
    int ox = kPhyHalf, oy = kPhyHalf;
    if (MODE == kBwd) {
        ox = rim_order(pi, g.px, rec_w);
        oy = rim_order(pj, g.py, rec_w);
    }
    const float *cx = c_list[ox], *cy = c_list[oy];
    const float rdx = 1.0f / g.dx;
    (void)rdx;
    for (int k = k0; k < k1; k++, i += sz) {
        const long long o = i + 4 * sz;
        wzz[8] = ld(szz, o);
        wxz[8] = ld(sxz, o);
        wyz[8] = ld(syz, o);
        if (kP) wau[8] = ld(sau, o);
        int oz = kPhyHalf;
        if (MODE == kBwd) oz = rim_order(k, g.pz, rec_w);
        const float *cz = c_list[oz];
        float sxx_x, syx_x, szx_x, sxy_y, syy_y, szy_y, sau_x = 0.f, sau_y = 0.f;
        if (MODE == kBwd) {
            sxx_x = dpv(sxx, i, 1, cx, ox);
            syx_x = dmv(sxy, i, 1, cx, ox);
            szx_x = dmv(sxz, i, 1, cx, ox);
            sxy_y = dmv(sxy, i, sy, cy, oy);
            syy_y = dpv(syy, i, sy, cy, oy);
            szy_y = dmv(syz, i, sy, cy, oy);
            sau_x = dpv(sau, i, 1, cx, ox);
            sau_y = dpv(sau, i, sy, cy, oy);
        } else {
            sxx_x = dp<4>(sxx, i, 1, cx);
            syx_x = dm<4>(sxy, i, 1, cx);
            szx_x = dm<4>(sxz, i, 1, cx);
            sxy_y = dm<4>(sxy, i, sy, cy);
            syy_y = dp<4>(syy, i, sy, cy);
            szy_y = dm<4>(syz, i, sy, cy);
            if (kP) {
                sau_x = dp<4>(sau, i, 1, cx);
                sau_y = dp<4>(sau, i, sy, cy);
            }
        }
        const float sxz_z = win_dm(wxz, cz, oz);
        const float syz_z = win_dm(wyz, cz, oz);
        const float szz_z = win_dp(wzz, cz, oz);
        const float sau_z = kP ? win_dp(wau, cz, oz) : 0.f;
        const float dtr = signed_bdt(ld(bdt, i), dt);
        const float a = dtr / g.dx, b = dtr / g.dy, c = dtr / g.dz;
        const float vx = w.f[VX][i] + (a * sxx_x + b * sxy_y + c * sxz_z);
        const float vy = w.f[VY][i] + (a * syx_x + b * syy_y + c * syz_z);
        const float vz = w.f[VZ][i] + (a * szx_x + b * szy_y + c * szz_z);
        w.f[VX][i] = vx;
        w.f[VY][i] = vy;
        w.f[VZ][i] = vz;
        if (kP) {
            const float px = w.f[VXP][i] + a * sau_x;
            const float py = w.f[VYP][i] + b * sau_y;
            const float pz = w.f[VZP][i] + c * sau_z;
            w.f[VXP][i] = px;
            w.f[VYP][i] = py;
            w.f[VZP][i] = pz;
            if (IMG) {
                const float rpx = ld(rv.f[VXP], i), rpy = ld(rv.f[VYP], i), rpz = ld(rv.f[VZP], i);
                const float rsx = ld(rv.f[VX], i) - rpx, rsy = ld(rv.f[VY], i) - rpy, rsz = ld(rv.f[VZ], i) - rpz;
                const float ssx = vx - px, ssy = vy - py, ssz = vz - pz;
                const long long q = pi + (long long)g.px * (pj + (long long)g.py * k);
                img.ip[q] += px * px + py * py + pz * pz;
                img.pp[q] += px * rpx + py * rpy + pz * rpz;
                img.ps[q] += px * rsx + py * rsy + pz * rsz;
                img.sp[q] += ssx * rpx + ssy * rpy + ssz * rpz;
                img.ss[q] += ssx * rsx + ssy * rsy + ssz * rsz;
            }
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            wzz[q] = wzz[q + 1];
            wxz[q] = wxz[q + 1];
            wyz[q] = wyz[q + 1];
            if (kP) wau[q] = wau[q + 1];
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(kTX *kTY) stress_phy_zm(GridDev g, WaveDev w, const float *__restrict__ lam,
                                                         const float *__restrict__ mu, float dt, int rec_w,
                                                         const float *__restrict__ wavelet,
                                                         const StepState *__restrict__ st, int zc, int it_off) {
    const int pi = blockIdx.x * kTX + threadIdx.x;
    const int pj = blockIdx.y * kTY + threadIdx.y;
    const int k0 = blockIdx.z * zc;
    const int k1 = min(k0 + zc, g.pz);
    if (pi >= g.px || pj >= g.py || k0 >= k1) return;
    const long long sy = g.sy, sz = g.sz;
    long long i = g.xoff + (pi + g.m) + sy * (pj + g.m) + sz * (k0 + g.m);
    const float *vxf = w.f[VX], *vyf = w.f[VY], *vzf = w.f[VZ];
    float wx[9], wy[9], wz[9];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const long long o = i + (q - 4) * sz;
        wx[q] = ld(vxf, o);
        wy[q] = ld(vyf, o);
        wz[q] = ld(vzf, o);
    }
    int ox = kPhyHalf, oy = kPhyHalf;
    if (MODE == kBwd) {
        ox = rim_order(pi, g.px, rec_w);
        oy = rim_order(pj, g.py, rec_w);
    }
    const float *cx = c_list[ox], *cy = c_list[oy];
    const long long src = (MODE != kRev) ? st->src : -1;
    const float a = dt / g.dx, b = dt / g.dy, c = dt / g.dz;
    for (int k = k0; k < k1; k++, i += sz) {
        const long long o = i + 4 * sz;
        wx[8] = ld(vxf, o);
        wy[8] = ld(vyf, o);
        wz[8] = ld(vzf, o);
        int oz = kPhyHalf;
        if (MODE == kBwd) oz = rim_order(k, g.pz, rec_w);
        const float *cz = c_list[oz];
        float vx_x, vy_x, vz_x, vx_y, vy_y, vz_y;
        if (MODE == kBwd) {
            vx_x = dmv(vxf, i, 1, cx, ox);
            vy_x = dpv(vyf, i, 1, cx, ox);
            vz_x = dpv(vzf, i, 1, cx, ox);
            vx_y = dpv(vxf, i, sy, cy, oy);
            vy_y = dmv(vyf, i, sy, cy, oy);
            vz_y = dpv(vzf, i, sy, cy, oy);
        } else {
            vx_x = dm<4>(vxf, i, 1, cx);
            vy_x = dp<4>(vyf, i, 1, cx);
            vz_x = dp<4>(vzf, i, 1, cx);
            vx_y = dp<4>(vxf, i, sy, cy);
            vy_y = dm<4>(vyf, i, sy, cy);
            vz_y = dp<4>(vzf, i, sy, cy);
        }
        const float vx_z = win_dp(wx, cz, oz);
        const float vy_z = win_dp(wy, cz, oz);
        const float vz_z = win_dm(wz, cz, oz);
        const float l = ld(lam, i), m = ld(mu, i);
        const float l2m = l + 2.0f * m;
        float sxx = w.f[SXX][i], syy = w.f[SYY][i], szz = w.f[SZZ][i];
        if (MODE != kRev && i == src) {
            const float s = wavelet[st->it + it_off];
            if (MODE == kBwd) {
                sxx -= s; syy -= s; szz -= s;
            } else {
                sxx += s; syy += s; szz += s;
            }
        }
        w.f[SXX][i] = sxx + (a * l2m * vx_x + b * l * vy_y + c * l * vz_z);
        w.f[SYY][i] = syy + (a * l * vx_x + b * l2m * vy_y + c * l * vz_z);
        w.f[SZZ][i] = szz + (a * l * vx_x + b * l * vy_y + c * l2m * vz_z);
        w.f[SXY][i] += a * m * vy_x + b * m * vx_y;
        w.f[SXZ][i] += a * m * vz_x + c * m * vx_z;
        w.f[SYZ][i] += b * m * vz_y + c * m * vy_z;
        if (MODE != kFwd) w.f[SAU][i] += a * l2m * vx_x + b * l2m * vy_y + c * l2m * vz_z;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            wx[q] = wx[q + 1];
            wy[q] = wy[q + 1];
            wz[q] = wz[q + 1];
        }
    }
}

// --------------------------------------------- x-vectorised variants
//
// Each thread updates four consecutive x cells (one 16-byte group; the
// first gridphy column is 128-byte aligned, so groups and their +-4 halo
// groups are float4-aligned).  x-derivatives come from a 12-value window
// (three float4 loads), y/z-derivatives from float4 loads of the stencil
// rows/planes, with 32-bit element offsets.  Partial groups at the +x end of
// gridphy compute all four lanes but store only the cells inside gridphy.


__device__ __forceinline__ float4 ld4(const float *__restrict__ f, int i) {
    return __ldg(reinterpret_cast<const float4 *>(f + i));
}
__device__ __forceinline__ float4 ldw4(const float *f, int i) { return *reinterpret_cast<const float4 *>(f + i); }
__device__ __forceinline__ void f4a(float *a, float4 v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w; }

// window w[0..11] = f[i0-4 .. i0+7]
__device__ __forceinline__ void xwin(const float *__restrict__ f, int i0, float *w) {
    f4a(w, ld4(f, i0 - 4));
    f4a(w + 4, ld4(f, i0));
    f4a(w + 8, ld4(f, i0 + 4));
}
// x-derivatives of the 4 cells from the window, coefficient rows cc[c]
__device__ __forceinline__ void xdp(const float *w, const float *const *cc, float *out) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float t = 0.f;
#pragma unroll
        for (int r = 0; r < 4; r++) t += cc[c][r] * (w[4 + c + r + 1] - w[4 + c - r]);
        out[c] = t;
    }
}
__device__ __forceinline__ void xdm(const float *w, const float *const *cc, float *out) {
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float t = 0.f;
#pragma unroll
        for (int r = 0; r < 4; r++) t += cc[c][r] * (w[4 + c + r] - w[4 + c - r - 1]);
        out[c] = t;
    }
}
// y or z derivatives of the 4 cells (stride s), one coefficient row
__device__ __forceinline__ void sdp(const float *__restrict__ f, int i0, int s, const float *cf, float *out) {
    float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const float4 a = ld4(f, i0 + (r + 1) * s), b = ld4(f, i0 - r * s);
        t[0] += cf[r] * (a.x - b.x);
        t[1] += cf[r] * (a.y - b.y);
        t[2] += cf[r] * (a.z - b.z);
        t[3] += cf[r] * (a.w - b.w);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) out[c] = t[c];
}
__device__ __forceinline__ void sdm(const float *__restrict__ f, int i0, int s, const float *cf, float *out) {
    float t[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const float4 a = ld4(f, i0 + r * s), b = ld4(f, i0 - (r + 1) * s);
        t[0] += cf[r] * (a.x - b.x);
        t[1] += cf[r] * (a.y - b.y);
        t[2] += cf[r] * (a.z - b.z);
        t[3] += cf[r] * (a.w - b.w);
    }
#pragma unroll
    for (int c = 0; c < 4; c++) out[c] = t[c];
}

// coefficient rows: full 8th order, or the rtm_backward rim orders
// (rows of c_list are zero past their order, so a 4-term sum is exact)
// (outside the rtm_backward rim every row is the constant c_list[4], which
// the compiler folds into constant-bank operands)
template <int MODE>
__device__ __forceinline__ void xcoefs(int pi0, int px, int rw, const float **cc) {
#pragma unroll
    for (int c = 0; c < 4; c++) cc[c] = c_list[(MODE == kBwd) ? rim_order(pi0 + c, px, rw) : kPhyHalf];
}
template <int MODE>
__device__ __forceinline__ const float *scoef(int p, int np, int rw) {
    return c_list[(MODE == kBwd) ? rim_order(p, np, rw) : kPhyHalf];
}

__device__ __forceinline__ void st4(float *f, int i0, const float *v, int nvalid) {
    if (nvalid >= 4) {
        *reinterpret_cast<float4 *>(f + i0) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < nvalid) f[i0 + c] = v[c];
    }
}

// The velocity update of one 4-cell group (x cells pi0..pi0+3 of row pj,
// plane pk) of wavefield w, stored, with the updated velocities left in
// v[3][4] and, for the modes that carry them, the P-wave velocities in
// p[3][4].
template <int MODE>
__device__ __forceinline__ void vel_update4(const GridDev &g, const WaveDev &w, const float *__restrict__ bdt,
                                            float dt, int rec_w, int pi0, int pj, int pk, float v[3][4],
                                            float p[3][4]) {
    constexpr bool kP = (MODE == kBwd || MODE == kRev);
    const int nvalid = min(4, g.px - pi0);
    const int sy = (int)g.sy, sz = (int)g.sz;
    const int i0 = (int)g.xoff + (pi0 + g.m) + sy * (pj + g.m) + sz * (pk + g.m);
    const float *cx[4];
    xcoefs<MODE>(pi0, g.px, rec_w, cx);
    const float *cy = scoef<MODE>(pj, g.py, rec_w);
    const float *cz = scoef<MODE>(pk, g.pz, rec_w);
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    float Dx[4], Dy[4], Dz[4], t[4], win[12];
    // vx: Dp_x sxx + Dm_y sxy + Dm_z sxz
    xwin(w.f[SXX], i0, win);
    xdp(win, cx, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dx[c] = t[c] * rdx;
    sdm(w.f[SXY], i0, sy, cy, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dx[c] += t[c] * rdy;
    sdm(w.f[SXZ], i0, sz, cz, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dx[c] += t[c] * rdz;
    // vy: Dm_x sxy + Dp_y syy + Dm_z syz
    xwin(w.f[SXY], i0, win);
    xdm(win, cx, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dy[c] = t[c] * rdx;
    sdp(w.f[SYY], i0, sy, cy, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dy[c] += t[c] * rdy;
    sdm(w.f[SYZ], i0, sz, cz, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dy[c] += t[c] * rdz;
    // vz: Dm_x sxz + Dm_y syz + Dp_z szz
    xwin(w.f[SXZ], i0, win);
    xdm(win, cx, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dz[c] = t[c] * rdx;
    sdm(w.f[SYZ], i0, sy, cy, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dz[c] += t[c] * rdy;
    sdp(w.f[SZZ], i0, sz, cz, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Dz[c] += t[c] * rdz;

    float dtr[4];
    {
        const float4 r4 = ld4(bdt, i0);
        if (MODE == kBwd) {
            // -b as b / -1 (exact): the backward update carries the imaging
            // and runs at the 64-register cap, and with the division in place
            // of a select ptxas keeps the schedule that spills least (24
            // against 44 bytes; 255 against 267 us on cfg2)
            float sg = dt < 0.f ? -1.0f : 1.0f;
            asm("mov.b32 %0, %0;" : "+f"(sg));
            dtr[0] = __fdiv_rn(r4.x, sg); dtr[1] = __fdiv_rn(r4.y, sg);
            dtr[2] = __fdiv_rn(r4.z, sg); dtr[3] = __fdiv_rn(r4.w, sg);
        } else {
            dtr[0] = signed_bdt(r4.x, dt); dtr[1] = signed_bdt(r4.y, dt);
            dtr[2] = signed_bdt(r4.z, dt); dtr[3] = signed_bdt(r4.w, dt);
        }
    }
    f4a(v[0], ldw4(w.f[VX], i0));
    f4a(v[1], ldw4(w.f[VY], i0));
    f4a(v[2], ldw4(w.f[VZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) {
        v[0][c] += dtr[c] * Dx[c];
        v[1][c] += dtr[c] * Dy[c];
        v[2][c] += dtr[c] * Dz[c];
    }
    st4(w.f[VX], i0, v[0], nvalid);
    st4(w.f[VY], i0, v[1], nvalid);
    st4(w.f[VZ], i0, v[2], nvalid);
    if (kP) {
        // P-wave velocity from the pressure-like field sau (Dp on every axis)
        xwin(w.f[SAU], i0, win);
        xdp(win, cx, t);
        f4a(p[0], ldw4(w.f[VXP], i0));
#pragma unroll
        for (int c = 0; c < 4; c++) p[0][c] += dtr[c] * (t[c] * rdx);
        sdp(w.f[SAU], i0, sy, cy, t);
        f4a(p[1], ldw4(w.f[VYP], i0));
#pragma unroll
        for (int c = 0; c < 4; c++) p[1][c] += dtr[c] * (t[c] * rdy);
        sdp(w.f[SAU], i0, sz, cz, t);
        f4a(p[2], ldw4(w.f[VZP], i0));
#pragma unroll
        for (int c = 0; c < 4; c++) p[2][c] += dtr[c] * (t[c] * rdz);
        st4(w.f[VXP], i0, p[0], nvalid);
        st4(w.f[VYP], i0, p[1], nvalid);
        st4(w.f[VZP], i0, p[2], nvalid);
    }
}

// Zero-lag imaging condition of one group (RTM/rtm3d_0_image_module/
// rtm3d_iamge_kernel.hpp:6-51): P = p, S = v - p of the reconstructed
// source (v, p) and of the receiver wavefield (rv, rp), added into the
// shot's FP32 images.
__device__ __forceinline__ void image4(const GridDev &g, const ImageDev &img, int pi0, int pj, int pk,
                                       const float v[3][4], const float p[3][4], const float rv[3][4],
                                       const float rp[3][4]) {
    const int nvalid = min(4, g.px - pi0);
    const long long o0 = pi0 + (long long)g.px * (pj + (long long)g.py * pk);
    float a[5][4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float rsx = rv[0][c] - rp[0][c], rsy = rv[1][c] - rp[1][c], rsz = rv[2][c] - rp[2][c];
        const float ssx = v[0][c] - p[0][c], ssy = v[1][c] - p[1][c], ssz = v[2][c] - p[2][c];
        a[0][c] = p[0][c] * p[0][c] + p[1][c] * p[1][c] + p[2][c] * p[2][c];
        a[1][c] = p[0][c] * rp[0][c] + p[1][c] * rp[1][c] + p[2][c] * rp[2][c];
        a[2][c] = p[0][c] * rsx + p[1][c] * rsy + p[2][c] * rsz;
        a[3][c] = ssx * rp[0][c] + ssy * rp[1][c] + ssz * rp[2][c];
        a[4][c] = ssx * rsx + ssy * rsy + ssz * rsz;
    }
    float *dst[5] = {img.ip, img.pp, img.ps, img.sp, img.ss};
    bool al = nvalid == 4;
#pragma unroll
    for (int q = 0; q < 5; q++) al = al && ((reinterpret_cast<uintptr_t>(dst[q] + o0) & 15) == 0);
    if (al) {
#pragma unroll
        for (int q = 0; q < 5; q++) {
            float4 *p4 = reinterpret_cast<float4 *>(dst[q] + o0);
            float4 s4 = *p4;
            s4.x += a[q][0]; s4.y += a[q][1]; s4.z += a[q][2]; s4.w += a[q][3];
            *p4 = s4;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 5; q++)
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c < nvalid) dst[q][o0 + c] += a[q][c];
    }
}

// L2 prefetch of the line holding f[i]; the address is formed inside the asm
// so that it does not stay live until the later load of the same element
__device__ __forceinline__ void pf_l2(const float *f, int i) {
    asm volatile("{\n\t.reg .u64 a;\n\tmad.wide.s32 a, %1, 4, %0;\n\tprefetch.global.L2 [a];\n\t}" ::"l"(f), "r"(i));
}

// The lines of a group that no earlier block of the launch has brought into
// L2 (blocks run in plane order): the pointwise arrays at the group, the
// fields read only in their own plane, and the leading plane of each z
// stencil.  Prefetched together, their DRAM latencies overlap instead of
// following the chain of dependent loads (measured on cfg2: 253 against
// 263-269 us for the backward update with imaging, 151 against 154 us for
// the receiver update).  The receiver wavefield's and the images' lines are
// left out: their prefetch addresses spill at 64 registers and cost more
// than they gain (337 us).
template <int MODE>
__device__ __forceinline__ void vel_prefetch4(const GridDev &g, const WaveDev &w, const float *__restrict__ bdt,
                                              int i0) {
    constexpr bool kP = (MODE == kBwd || MODE == kRev);
    const int sz = (int)g.sz;
    pf_l2(bdt, i0);
    pf_l2(w.f[VX], i0);
    pf_l2(w.f[VY], i0);
    pf_l2(w.f[VZ], i0);
    pf_l2(w.f[SXX], i0);
    pf_l2(w.f[SXY], i0);
    pf_l2(w.f[SYY], i0);
    pf_l2(w.f[SXZ], i0 + 3 * sz);
    pf_l2(w.f[SYZ], i0 + 3 * sz);
    pf_l2(w.f[SZZ], i0 + 4 * sz);
    if (kP) {
        pf_l2(w.f[SAU], i0 + 4 * sz);
        pf_l2(w.f[VXP], i0);
        pf_l2(w.f[VYP], i0);
        pf_l2(w.f[VZP], i0);
    }
}

// One 4-cell group of the velocity update of wavefield w; with IMG (the
// backward update) the imaging condition against the receiver wavefield rv
// follows.
template <int MODE, bool IMG>
__device__ __forceinline__ void vel_group4(const GridDev &g, const WaveDev &w, const float *__restrict__ bdt,
                                           float dt, int rec_w, const WaveDev &rv, const ImageDev &img, int pi0,
                                           int pj, int pk) {
    const int i0 = (int)g.xoff + (pi0 + g.m) + (int)g.sy * (pj + g.m) + (int)g.sz * (pk + g.m);
    vel_prefetch4<MODE>(g, w, bdt, i0);
    float v[3][4], p[3][4];
    vel_update4<MODE>(g, w, bdt, dt, rec_w, pi0, pj, pk, v, p);
    if (IMG) {
        float r[3][4], rp[3][4];
        f4a(r[0], ld4(rv.f[VX], i0));
        f4a(r[1], ld4(rv.f[VY], i0));
        f4a(r[2], ld4(rv.f[VZ], i0));
        f4a(rp[0], ld4(rv.f[VXP], i0));
        f4a(rp[1], ld4(rv.f[VYP], i0));
        f4a(rp[2], ld4(rv.f[VZP], i0));
        image4(g, img, pi0, pj, pk, v, p, r, rp);
    }
}

// Blocks of blockDim.x groups x blockDim.y rows x ZP planes; a thread
// updates its group in ZP consecutive planes.
template <int MODE, bool IMG, int MINB, int ZP>
__global__ void __launch_bounds__(256, MINB) vel_phy_v4(GridDev g, WaveDev w, const float *__restrict__ bdt,
                                                       float dt, int rec_w, WaveDev rv, ImageDev img) {
    const int pi0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int pj = blockIdx.y * blockDim.y + threadIdx.y;
    if (pi0 >= g.px || pj >= g.py) return;
#pragma unroll
    for (int zz = 0; zz < ZP; zz++) {
        const int pk = blockIdx.z * ZP + zz;
        if (pk < g.pz) vel_group4<MODE, IMG>(g, w, bdt, dt, rec_w, rv, img, pi0, pj, pk);
    }
}

// One 4-cell group of the stress update (source fused).
template <int MODE>
__device__ __forceinline__ void stress_group4(const GridDev &g, const WaveDev &w, const float *__restrict__ lam,
                                              const float *__restrict__ mu, float dt, int rec_w,
                                              const float *__restrict__ wavelet, const StepState *__restrict__ st,
                                              int it_off, int pi0, int pj, int pk) {
    const int nvalid = min(4, g.px - pi0);
    const int sy = (int)g.sy, sz = (int)g.sz;
    const int i0 = (int)g.xoff + (pi0 + g.m) + sy * (pj + g.m) + sz * (pk + g.m);
    // the group's DRAM-new lines, as in vel_prefetch4: the pointwise model
    // and stress arrays, and the leading plane of each z stencil
    pf_l2(lam, i0);
    pf_l2(mu, i0);
    pf_l2(w.f[SXX], i0);
    pf_l2(w.f[SYY], i0);
    pf_l2(w.f[SZZ], i0);
    pf_l2(w.f[SXY], i0);
    pf_l2(w.f[SXZ], i0);
    pf_l2(w.f[SYZ], i0);
    if (MODE != kFwd) pf_l2(w.f[SAU], i0);
    pf_l2(w.f[VX], i0 + 4 * sz);
    pf_l2(w.f[VY], i0 + 4 * sz);
    pf_l2(w.f[VZ], i0 + 3 * sz);
    const float *cx[4];
    xcoefs<MODE>(pi0, g.px, rec_w, cx);
    const float *cy = scoef<MODE>(pj, g.py, rec_w);
    const float *cz = scoef<MODE>(pk, g.pz, rec_w);
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    // normal derivatives Nx = d vx/dx, ...; shear sums Sxy = d vy/dx + d vx/dy, ...
    float Nx[4], Ny[4], Nz[4], Sxy[4], Sxz[4], Syz[4], t[4], win[12];
    xwin(w.f[VX], i0, win);
    xdm(win, cx, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Nx[c] = t[c] * rdx;
    sdp(w.f[VX], i0, sy, cy, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Sxy[c] = t[c] * rdy;
    sdp(w.f[VX], i0, sz, cz, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Sxz[c] = t[c] * rdz;
    xwin(w.f[VY], i0, win);
    xdp(win, cx, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Sxy[c] += t[c] * rdx;
    sdm(w.f[VY], i0, sy, cy, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Ny[c] = t[c] * rdy;
    sdp(w.f[VY], i0, sz, cz, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Syz[c] = t[c] * rdz;
    xwin(w.f[VZ], i0, win);
    xdp(win, cx, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Sxz[c] += t[c] * rdx;
    sdp(w.f[VZ], i0, sy, cy, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Syz[c] += t[c] * rdy;
    sdm(w.f[VZ], i0, sz, cz, t);
#pragma unroll
    for (int c = 0; c < 4; c++) Nz[c] = t[c] * rdz;

    float l[4], m[4], sxx[4], syy[4], szz[4];
    f4a(l, ld4(lam, i0));
    f4a(m, ld4(mu, i0));
    f4a(sxx, ldw4(w.f[SXX], i0));
    f4a(syy, ldw4(w.f[SYY], i0));
    f4a(szz, ldw4(w.f[SZZ], i0));
    if (MODE != kRev) {
        // explosive source, applied before the stress update of step it
        // (FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_3_stress_kernel.hpp:1308-1364)
        const long long src = st->src;
        const long long d = src - (long long)i0;
        if (d >= 0 && d < nvalid) {
            const float w0 = wavelet[st->it + it_off];
            const float sv = (MODE == kBwd) ? -w0 : w0;
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c == (int)d) {
                    sxx[c] += sv;
                    syy[c] += sv;
                    szz[c] += sv;
                }
        }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float l2m = l[c] + 2.0f * m[c];
        sxx[c] += dt * (l2m * Nx[c] + l[c] * Ny[c] + l[c] * Nz[c]);
        syy[c] += dt * (l[c] * Nx[c] + l2m * Ny[c] + l[c] * Nz[c]);
        szz[c] += dt * (l[c] * Nx[c] + l[c] * Ny[c] + l2m * Nz[c]);
    }
    st4(w.f[SXX], i0, sxx, nvalid);
    st4(w.f[SYY], i0, syy, nvalid);
    st4(w.f[SZZ], i0, szz, nvalid);
    float a[4];
    f4a(a, ldw4(w.f[SXY], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * m[c] * Sxy[c];
    st4(w.f[SXY], i0, a, nvalid);
    f4a(a, ldw4(w.f[SXZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * m[c] * Sxz[c];
    st4(w.f[SXZ], i0, a, nvalid);
    f4a(a, ldw4(w.f[SYZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * m[c] * Syz[c];
    st4(w.f[SYZ], i0, a, nvalid);
    if (MODE != kFwd) {
        f4a(a, ldw4(w.f[SAU], i0));
#pragma unroll
        for (int c = 0; c < 4; c++) a[c] += dt * (l[c] + 2.0f * m[c]) * (Nx[c] + Ny[c] + Nz[c]);
        st4(w.f[SAU], i0, a, nvalid);
    }
}

template <int MODE, int MINB, int ZP>
__global__ void __launch_bounds__(256, MINB) stress_phy_v4(GridDev g, WaveDev w, const float *__restrict__ lam,
                                                          const float *__restrict__ mu, float dt, int rec_w,
                                                          const float *__restrict__ wavelet,
                                                          const StepState *__restrict__ st, int it_off) {
    const int pi0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int pj = blockIdx.y * blockDim.y + threadIdx.y;
    if (pi0 >= g.px || pj >= g.py) return;
#pragma unroll
    for (int zz = 0; zz < ZP; zz++) {
        const int pk = blockIdx.z * ZP + zz;
        if (pk < g.pz) stress_group4<MODE>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off, pi0, pj, pk);
    }
}

// ------------------------------------------ z-marching stress (variant 3)
//
// One CTA per SM, persistent.  The (row tile, plane) items of gridphy are
// split evenly over the CTAs; a CTA marches its items in z, one pair of
// x cells per thread (tile = all px cells of kZmRows rows, float2 shared-
// memory and global accesses).  Everything an item reads
// comes through TMA (cp.async.bulk.tensor), two items ahead, into a double
// buffer: the planes of vx, vy, vz with a 4-cell x/y halo (x/y stencils),
// and core tiles of lam, mu, the stress values and the vx, vy, vz plane
// five above (the entry that the register window of z stencils takes in
// next).  Threads read only shared memory and registers, and store the
// updated stress straight to global memory.  Every wait on a TMA barrier is
// bounded: when it runs out the CTA sets *err and stops.

constexpr int kZmRows = 4;
constexpr int kZmHalo = 4;
constexpr int kZmCPT = 2;           // cells per thread (an x pair, float2 accesses)
constexpr int kZmMaxThreads = 512;  // ceil(px / 2) * kZmRows; the register budget is set for this block size

// the descriptors of one launch, passed as one kernel parameter
struct ZmMaps {
    CUtensorMap halo[3];
    CUtensorMap core[kZmCore];
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// true when the phase with this parity has completed, false after ~1 s
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 2000000000LL) return false;
    }
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// Shared-memory geometry, fixed so that stencil offsets are immediates:
// a halo plane is a 256-float-wide box (row pitch 256) of kZmRows + 8 rows;
// a core tile (px rounded up to 4 wide, dense rows) sits in a region of
// kZmRows * 256 floats.
constexpr int kZmPitch = 256;
constexpr int kZmBoxH = kZmRows + 2 * kZmHalo;
constexpr int kZmHB = kZmPitch * kZmBoxH;  // floats of one halo plane
constexpr int kZmCB = kZmPitch * kZmRows;  // floats of one core-tile region
constexpr int kZmStage = 3 * kZmHB + kZmCore * kZmCB;

template <int MODE>
__global__ void __launch_bounds__(kZmMaxThreads, 1)
    stress_zm3(GridDev g, const __grid_constant__ ZmMaps maps, WaveDev w, float dt, int rec_w,
               const float *__restrict__ wavelet, const StepState *__restrict__ st, int it_off, int corew,
               int ytiles, int ntx, int tpp, int *err) {
    constexpr int NC = (MODE == kFwd) ? kZmCore - 1 : kZmCore;  // sau is not read in forward modelling
    extern __shared__ __align__(128) float sm[];
    constexpr int hb = kZmHB, cb = kZmCB, stage = kZmStage, boxw = kZmPitch;
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_abort;
    const int total = ytiles * ntx * g.pz;  // items (y tile, x tile, plane), plane fastest
    const int w0 = (int)((long long)total * blockIdx.x / gridDim.x);
    const int w1 = (int)((long long)total * (blockIdx.x + 1) / gridDim.x);
    if (w0 >= w1) return;
    const int tid = threadIdx.x;
    const int r = tid / tpp, xl = 2 * (tid - r * tpp);  // row; the pair's first cell within an x tile
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const uint32_t bytes_all = (uint32_t)(3 * kZmHB + NC * corew * kZmRows) * 4u;
    const uint32_t bytes_feed = (uint32_t)(3 * corew * kZmRows) * 4u;  // the window feed's share
    const int m = g.m;
    // x tile xt covers the gridphy pairs [xt tpp, (xt+1) tpp); its core box
    // starts at gridphy column 2 xt tpp (tpp even with several tiles, so
    // every box origin is a multiple of 4 floats) and its halo box 4 before
    auto tile_of = [&](int item, int &xt, int &yt, int &z) {
        const int t = item / g.pz;
        z = item - t * g.pz;
        yt = t / ntx;
        xt = t - yt * ntx;
    };
    auto issue = [&](int item, int b) {
        int xt, yt, z;
        tile_of(item, xt, yt, z);
        const int XC = (int)g.xoff + m + 2 * xt * tpp, XH = XC - kZmHalo;
        const uint32_t bar = b ? bar1 : bar0;
        const int Y = m + yt * kZmRows, Z = m + z;
        float *base = sm + b * stage;
        // the window's next entry: vx, vy, vz five planes above; it exists
        // inside gridext except for the last plane when pml is 4, where
        // the run ends and nothing is fetched
        const bool feed = Z + 5 < g.nz;
        mbar_expect(bar, feed ? bytes_all : bytes_all - bytes_feed);
        for (int f = 0; f < 3; f++) tma_load_3d(smem_u32(base + f * hb), &maps.halo[f], XH, Y - kZmHalo, Z, bar);
        if (feed)
            for (int f = 0; f < 3; f++)
                tma_load_3d(smem_u32(base + 3 * hb + f * cb), &maps.core[f], XC, Y, Z + 5, bar);
        for (int f = 3; f < NC; f++) tma_load_3d(smem_u32(base + 3 * hb + f * cb), &maps.core[f], XC, Y, Z, bar);
    };
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        issue(w0, 0);
        if (w0 + 1 < w1) issue(w0 + 1, 1);
    }
    const int sy = (int)g.sy, sz = (int)g.sz;
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    float2 rv[3][9];  // z windows of the pair: planes z-4 .. z+4 of vx, vy, vz
    const float *fv[3] = {w.f[VX], w.f[VY], w.f[VZ]};
    int cur_t = -1, cur_z = -2;
    for (int k = w0; k < w1; k++) {
        int xt, yt, z;
        tile_of(k, xt, yt, z);
        const int tile = k / g.pz;
        const int x = 2 * xt * tpp + xl;              // the pair's first gridphy column
        const int nval = min(kZmCPT, g.px - x);      // 1 for the last pair of an odd row
        const float *cx[2] = {c_list[(MODE == kBwd) ? rim_order(x, g.px, rec_w) : kPhyHalf],
                              c_list[(MODE == kBwd) ? rim_order(min(x + 1, g.px - 1), g.px, rec_w) : kPhyHalf]};
        const int y = yt * kZmRows + r;
        const bool live = y < g.py && x < g.px;
        const int i0 = (int)g.xoff + (x + m) + sy * (y + m) + sz * (z + m);  // even: float2-aligned
        const int b = (k - w0) & 1;
        const uint32_t parity = (uint32_t)(((k - w0) >> 1) & 1);
        const float *base = sm + b * stage;
        const int cc = r * corew + xl;  // the pair in a core tile
        if (tile != cur_t || z != cur_z + 1) {
            // a new run of planes: fill the z windows from global memory
#pragma unroll
            for (int f = 0; f < 3; f++) {
#pragma unroll
                for (int q = 0; q < 9; q++)
                    rv[f][q] = live ? __ldg(reinterpret_cast<const float2 *>(fv[f] + i0 + (q - 4) * sz))
                                    : make_float2(0.f, 0.f);
            }
        }
        cur_t = tile;
        cur_z = z;
        if (!mbar_wait_bounded(b ? bar1 : bar0, parity)) {
            s_abort = 1;
            atomicExch(err, 1);
        }
        if (live) {
            const float *P = base + 3 * hb;  // core tiles
            const int c0 = (r + kZmHalo) * boxw + (xl + kZmHalo);
            const float *cy = c_list[(MODE == kBwd) ? rim_order(y, g.py, rec_w) : kPhyHalf];
            const float *cz = c_list[(MODE == kBwd) ? rim_order(z, g.pz, rec_w) : kPhyHalf];
            // x window of a field around the pair: e[j] = f[x - 4 + j], j = 0..9
            auto xwin2 = [&](const float *F, float *e) {
#pragma unroll
                for (int j = 0; j < 5; j++) {
                    const float2 v = *reinterpret_cast<const float2 *>(F + c0 - 4 + 2 * j);
                    e[2 * j] = v.x;
                    e[2 * j + 1] = v.y;
                }
            };
            auto ld2 = [&](const float *F, int off) { return *reinterpret_cast<const float2 *>(F + off); };
            float e[10];
            float Nx[2], Ny[2], Nz[2], Sxy[2], Sxz[2], Syz[2];
            // vx: Dm_x -> Nx, Dp_y -> Sxy, Dp_z -> Sxz
            xwin2(base, e);
#pragma unroll
            for (int c = 0; c < 2; c++) {
                float t = 0.f;
#pragma unroll
                for (int q = 0; q < 4; q++) t += cx[c][q] * (e[4 + c + q] - e[4 + c - q - 1]);
                Nx[c] = t * rdx;
            }
            {
                float2 t = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 a = ld2(base, c0 + (q + 1) * boxw), bb = ld2(base, c0 - q * boxw);
                    t.x += cy[q] * (a.x - bb.x);
                    t.y += cy[q] * (a.y - bb.y);
                }
                Sxy[0] = t.x * rdy;
                Sxy[1] = t.y * rdy;
                t = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    t.x += cz[q] * (rv[0][4 + q + 1].x - rv[0][4 - q].x);
                    t.y += cz[q] * (rv[0][4 + q + 1].y - rv[0][4 - q].y);
                }
                Sxz[0] = t.x * rdz;
                Sxz[1] = t.y * rdz;
            }
            // vy: Dp_x -> Sxy, Dm_y -> Ny, Dp_z -> Syz
            xwin2(base + hb, e);
#pragma unroll
            for (int c = 0; c < 2; c++) {
                float t = 0.f;
#pragma unroll
                for (int q = 0; q < 4; q++) t += cx[c][q] * (e[4 + c + q + 1] - e[4 + c - q]);
                Sxy[c] += t * rdx;
            }
            {
                float2 t = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 a = ld2(base + hb, c0 + q * boxw), bb = ld2(base + hb, c0 - (q + 1) * boxw);
                    t.x += cy[q] * (a.x - bb.x);
                    t.y += cy[q] * (a.y - bb.y);
                }
                Ny[0] = t.x * rdy;
                Ny[1] = t.y * rdy;
                t = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    t.x += cz[q] * (rv[1][4 + q + 1].x - rv[1][4 - q].x);
                    t.y += cz[q] * (rv[1][4 + q + 1].y - rv[1][4 - q].y);
                }
                Syz[0] = t.x * rdz;
                Syz[1] = t.y * rdz;
            }
            // vz: Dp_x -> Sxz, Dp_y -> Syz, Dm_z -> Nz
            xwin2(base + 2 * hb, e);
#pragma unroll
            for (int c = 0; c < 2; c++) {
                float t = 0.f;
#pragma unroll
                for (int q = 0; q < 4; q++) t += cx[c][q] * (e[4 + c + q + 1] - e[4 + c - q]);
                Sxz[c] += t * rdx;
            }
            {
                float2 t = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float2 a = ld2(base + 2 * hb, c0 + (q + 1) * boxw), bb = ld2(base + 2 * hb, c0 - q * boxw);
                    t.x += cy[q] * (a.x - bb.x);
                    t.y += cy[q] * (a.y - bb.y);
                }
                Syz[0] += t.x * rdy;
                Syz[1] += t.y * rdy;
                t = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    t.x += cz[q] * (rv[2][4 + q].x - rv[2][4 - q - 1].x);
                    t.y += cz[q] * (rv[2][4 + q].y - rv[2][4 - q - 1].y);
                }
                Nz[0] = t.x * rdz;
                Nz[1] = t.y * rdz;
            }
            const float2 l2 = ld2(P, 3 * cb + cc), m2 = ld2(P, 4 * cb + cc);
            const float l[2] = {l2.x, l2.y}, mm[2] = {m2.x, m2.y};
            float2 s0 = ld2(P, 5 * cb + cc), s1 = ld2(P, 6 * cb + cc), s2 = ld2(P, 7 * cb + cc);
            float sxx[2] = {s0.x, s0.y}, syy[2] = {s1.x, s1.y}, szz[2] = {s2.x, s2.y};
            if (MODE != kRev) {
                // explosive source, applied before the stress update of step it
                const long long d = st->src - (long long)i0;
                if (d >= 0 && d < nval) {
                    const float w0v = wavelet[st->it + it_off];
                    const float sv = (MODE == kBwd) ? -w0v : w0v;
                    sxx[d] += sv;
                    syy[d] += sv;
                    szz[d] += sv;
                }
            }
            float o[7][2];
            const float2 t8 = ld2(P, 8 * cb + cc), t9 = ld2(P, 9 * cb + cc), t10 = ld2(P, 10 * cb + cc);
            const float sxy0[2] = {t8.x, t8.y}, sxz0[2] = {t9.x, t9.y}, syz0[2] = {t10.x, t10.y};
            float sau0[2] = {0.f, 0.f};
            if (MODE != kFwd) {
                const float2 t11 = ld2(P, 11 * cb + cc);
                sau0[0] = t11.x;
                sau0[1] = t11.y;
            }
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const float l2m = l[c] + 2.0f * mm[c];
                o[0][c] = sxx[c] + dt * (l2m * Nx[c] + l[c] * Ny[c] + l[c] * Nz[c]);
                o[1][c] = syy[c] + dt * (l[c] * Nx[c] + l2m * Ny[c] + l[c] * Nz[c]);
                o[2][c] = szz[c] + dt * (l[c] * Nx[c] + l[c] * Ny[c] + l2m * Nz[c]);
                o[3][c] = sxy0[c] + dt * mm[c] * Sxy[c];
                o[4][c] = sxz0[c] + dt * mm[c] * Sxz[c];
                o[5][c] = syz0[c] + dt * mm[c] * Syz[c];
                o[6][c] = sau0[c] + dt * (l[c] + 2.0f * mm[c]) * (Nx[c] + Ny[c] + Nz[c]);
            }
            const int outf[7] = {SXX, SYY, SZZ, SXY, SXZ, SYZ, SAU};
            const int nout = (MODE != kFwd) ? 7 : 6;
#pragma unroll
            for (int j = 0; j < 7; j++) {
                if (j >= nout) break;
                float *dst = w.f[outf[j]] + i0;
                if (nval == 2) *reinterpret_cast<float2 *>(dst) = make_float2(o[j][0], o[j][1]);
                else dst[0] = o[j][0];
            }
            // advance the z windows: the plane five above came in with this item
#pragma unroll
            for (int f = 0; f < 3; f++) {
#pragma unroll
                for (int q = 0; q < 8; q++) rv[f][q] = rv[f][q + 1];
                rv[f][8] = ld2(P, f * cb + cc);
            }
        }
        __syncthreads();  // every thread is done with buffer b
        if (s_abort) {
            // stop issuing; give the copies still in flight (this item's and
            // the next one's) a bounded time to land before the CTA leaves
            if (tid == 0) {
                mbar_wait_bounded(b ? bar1 : bar0, parity);
                if (k + 1 < w1) {
                    const int k1 = k + 1 - w0;
                    mbar_wait_bounded((k1 & 1) ? bar1 : bar0, (uint32_t)((k1 >> 1) & 1));
                }
            }
            __syncthreads();
            return;
        }
        if (tid == 0 && k + 2 < w1) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(k + 2, b);
        }
    }
}

// ---------------------------------------------------------------- CPML

// Damping coefficients of one absorbing axis at one cell
// (FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_1_host_meat.hpp:147-620):
// d = temp (s/N)^2 with temp = log10(1/R) 7 vp / (2 N delta), alpha =
// pi fm (1 - s/N), b = exp(-(d+alpha) dt), a = d (b-1) / (d+alpha).  The
// axis table entry t holds the vp-independent factors of the integer and
// half node, {K, K_half, alpha, alpha_half} with d = vp K; K = 0 marks an
// index outside that axis' absorbing range (a = 0, b = 1 there).
__device__ __forceinline__ void cpml_coef(float vp, float4 t, float dt, float &A, float &B, float &Ah, float &Bh) {
    if (t.x > 0.f) {
        const float d = vp * t.x, dh = vp * t.y;
        B = expf(-(d + t.z) * dt);
        Bh = expf(-(dh + t.w) * dt);
        A = d * (B - 1.0f) / (d + t.z);
        Ah = dh * (Bh - 1.0f) / (dh + t.w);
    } else {
        A = 0.f; B = 1.f; Ah = 0.f; Bh = 1.f;
    }
}

// 4th-order y/z differences of the 4 cells of a group (stride s)
__device__ __forceinline__ void sdp2(const float *__restrict__ f, int i0, int s, float c0, float c1, float *out) {
    const float4 a = ld4(f, i0 + s), b = ld4(f, i0), c = ld4(f, i0 + 2 * s), d = ld4(f, i0 - s);
    out[0] = c0 * (a.x - b.x) + c1 * (c.x - d.x);
    out[1] = c0 * (a.y - b.y) + c1 * (c.y - d.y);
    out[2] = c0 * (a.z - b.z) + c1 * (c.z - d.z);
    out[3] = c0 * (a.w - b.w) + c1 * (c.w - d.w);
}
__device__ __forceinline__ void sdm2(const float *__restrict__ f, int i0, int s, float c0, float c1, float *out) {
    const float4 a = ld4(f, i0), b = ld4(f, i0 - s), c = ld4(f, i0 + s), d = ld4(f, i0 - 2 * s);
    out[0] = c0 * (a.x - b.x) + c1 * (c.x - d.x);
    out[1] = c0 * (a.y - b.y) + c1 * (c.y - d.y);
    out[2] = c0 * (a.z - b.z) + c1 * (c.z - d.z);
    out[3] = c0 * (a.w - b.w) + c1 * (c.w - d.w);
}
// 4th-order x differences of the 4 cells from the 12-value window
__device__ __forceinline__ void xdp2(const float *w, float c0, float c1, float *out) {
#pragma unroll
    for (int c = 0; c < 4; c++) out[c] = c0 * (w[5 + c] - w[4 + c]) + c1 * (w[6 + c] - w[3 + c]);
}
__device__ __forceinline__ void xdm2(const float *w, float c0, float c1, float *out) {
#pragma unroll
    for (int c = 0; c < 4; c++) out[c] = c0 * (w[4 + c] - w[3 + c]) + c1 * (w[5 + c] - w[2 + c]);
}

// b * psi + a * d for the 4 cells of a group (float4 memory variable)
__device__ __forceinline__ void psi4(float *p, const float *B, const float *A, float *d) {
    float4 v = *reinterpret_cast<float4 *>(p);
    v.x = B[0] * v.x + A[0] * d[0];
    v.y = B[1] * v.y + A[1] * d[1];
    v.z = B[2] * v.z + A[2] * d[2];
    v.w = B[3] * v.w + A[3] * d[3];
    *reinterpret_cast<float4 *>(p) = v;
    d[0] += v.x;
    d[1] += v.y;
    d[2] += v.z;
    d[3] += v.w;
}

__device__ __forceinline__ void st4m(float *f, int i0, const float *v, unsigned mask) {
    if (mask == 0xF) {
        *reinterpret_cast<float4 *>(f + i0) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (mask & (1u << c)) f[i0 + c] = v[c];
    }
}

// Thread -> one 4-cell x group of one row of one slab.  Returns false for
// threads past the slab's groups or rows.
struct PmlPos {
    int xs, y, z;        // first cell of the group
    unsigned mask;       // cells of the group inside the slab
    long long psi;       // arena offset of the group's first memory variable
    long long stride;    // floats between memory arrays of the slab
    int naxes;
    int z1;              // end plane of the slab
    int plane;           // memory-variable floats of one slab plane
};
__device__ __forceinline__ bool pml_pos(const CpmlDev &P, PmlPos &q) {
    const int b = blockIdx.x;
    PmlSlab S = P.s[0];
#pragma unroll
    for (int k = 1; k < 6; k++)
        if (k < P.nslab && b >= P.s[k].first_block) S = P.s[k];
    const int lb = b - S.first_block;
    const int bxi = lb % S.bx;
    const int t = lb / S.bx;
    const int byi = t % S.by;
    q.z = S.z0 + (t / S.by) * P.zp;
    const int tr = (int)threadIdx.x / S.gx;
    const int grp = bxi * S.gx + ((int)threadIdx.x - tr * S.gx);
    q.y = S.y0 + byi * S.gy + tr;
    if (tr >= S.gy || grp >= S.ngroups || q.y >= S.y1) return false;
    q.xs = S.gstart + 4 * grp;
    q.mask = 0;
#pragma unroll
    for (int c = 0; c < 4; c++)
        if (q.xs + c >= S.x0 && q.xs + c < S.x1) q.mask |= 1u << c;
    q.psi = S.psi_off + ((long long)(q.z - S.z0) * (S.y1 - S.y0) + (q.y - S.y0)) * S.pitch + 4 * grp;
    q.stride = S.stride;
    q.naxes = S.naxes;
    q.z1 = S.z1;
    q.plane = (S.y1 - S.y0) * S.pitch;
    return true;
}

__device__ __forceinline__ void xcoef4(const CpmlDev &P, const PmlPos &q, float vp4[4], float *A, float *B,
                                       float *Ah, float *Bh, bool &any) {
    any = false;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q.mask & (1u << c)) t = P.ax[0][q.xs + c];
        any |= t.x > 0.f;
        cpml_coef(vp4[c], t, P.dt, A[c], B[c], Ah[c], Bh[c]);
    }
}

// CPML velocity update of the six absorbing slabs: 4th order, memory
// variables on the absorbing axes (z-slabs x,y,z; y-slabs x,y; x-slabs x)
// (FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_2_kernel_device_{x,y,z}_meat.hpp)
__device__ __forceinline__ void vel_pml_group(const GridDev &g, const CpmlDev &P, const WaveDev &w,
                                              const float *__restrict__ bdt, const float *__restrict__ vpm,
                                              const PmlPos &q) {
    const int sy = (int)g.sy, sz = (int)g.sz;
    const int i0 = (int)g.xoff + q.xs + sy * q.y + sz * q.z;
    {
        // the group's DRAM-new lines (slab blocks run in plane order), as in
        // vel_prefetch4: pointwise arrays, fields read in their own plane, the
        // leading plane of each z difference, and the memory variables of the
        // axes on which the group absorbs
        pf_l2(bdt, i0);
        pf_l2(vpm, i0);
        pf_l2(w.f[VX], i0);
        pf_l2(w.f[VY], i0);
        pf_l2(w.f[VZ], i0);
        pf_l2(w.f[SXX], i0);
        pf_l2(w.f[SXY], i0);
        pf_l2(w.f[SYY], i0);
        pf_l2(w.f[SXZ], i0 + sz);
        pf_l2(w.f[SYZ], i0 + sz);
        pf_l2(w.f[SZZ], i0 + 2 * sz);
        const float *psi = P.psi + q.psi;
        const long long n = q.stride;
        bool anyx = false;
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (q.mask & (1u << c)) anyx |= P.ax[0][q.xs + c].x > 0.f;
        if (anyx)
#pragma unroll
            for (int a = 0; a < 3; a++) pf_l2(psi + a * n, 0);
        if (P.ax[1][q.y].x > 0.f)
#pragma unroll
            for (int a = 3; a < 6; a++) pf_l2(psi + a * n, 0);
        if (P.ax[2][q.z].x > 0.f)
#pragma unroll
            for (int a = 6; a < 9; a++) pf_l2(psi + a * n, 0);
    }
    const float c0 = c_dc2[0], c1 = c_dc2[1];
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    float win[12], sxx_x[4], syx_x[4], szx_x[4], sxy_y[4], syy_y[4], szy_y[4], sxz_z[4], syz_z[4], szz_z[4];
    xwin(w.f[SXX], i0, win);
    xdp2(win, c0, c1, sxx_x);
    xwin(w.f[SXY], i0, win);
    xdm2(win, c0, c1, syx_x);
    xwin(w.f[SXZ], i0, win);
    xdm2(win, c0, c1, szx_x);
    sdm2(w.f[SXY], i0, sy, c0, c1, sxy_y);
    sdp2(w.f[SYY], i0, sy, c0, c1, syy_y);
    sdm2(w.f[SYZ], i0, sy, c0, c1, szy_y);
    sdm2(w.f[SXZ], i0, sz, c0, c1, sxz_z);
    sdm2(w.f[SYZ], i0, sz, c0, c1, syz_z);
    sdp2(w.f[SZZ], i0, sz, c0, c1, szz_z);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        sxx_x[c] *= rdx; syx_x[c] *= rdx; szx_x[c] *= rdx;
        sxy_y[c] *= rdy; syy_y[c] *= rdy; szy_y[c] *= rdy;
        sxz_z[c] *= rdz; syz_z[c] *= rdz; szz_z[c] *= rdz;
    }
    float vp4[4];
    f4a(vp4, ld4(vpm, i0));
    float *psi = P.psi + q.psi;
    const long long n = q.stride;
    float A[4], B[4], Ah[4], Bh[4];
    bool any;
    xcoef4(P, q, vp4, A, B, Ah, Bh, any);
    if (any) {
        psi4(psi + 0 * n, Bh, Ah, sxx_x);
        psi4(psi + 1 * n, B, A, syx_x);
        psi4(psi + 2 * n, B, A, szx_x);
    }
    const float4 ty = P.ax[1][q.y], tz = P.ax[2][q.z];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ty.x > 0.f) {
#pragma unroll
        for (int c = 0; c < 4; c++) cpml_coef(vp4[c], (q.mask >> c) & 1u ? ty : z4, P.dt, A[c], B[c], Ah[c], Bh[c]);
        psi4(psi + 3 * n, B, A, sxy_y);
        psi4(psi + 4 * n, Bh, Ah, syy_y);
        psi4(psi + 5 * n, B, A, szy_y);
    }
    if (tz.x > 0.f) {
#pragma unroll
        for (int c = 0; c < 4; c++) cpml_coef(vp4[c], (q.mask >> c) & 1u ? tz : z4, P.dt, A[c], B[c], Ah[c], Bh[c]);
        psi4(psi + 6 * n, B, A, sxz_z);
        psi4(psi + 7 * n, B, A, syz_z);
        psi4(psi + 8 * n, Bh, Ah, szz_z);
    }
    float dtr[4], v[4];
    f4a(dtr, ld4(bdt, i0));  // P.dt > 0
    f4a(v, ldw4(w.f[VX], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] += dtr[c] * (sxx_x[c] + sxy_y[c] + sxz_z[c]);
    st4m(w.f[VX], i0, v, q.mask);
    f4a(v, ldw4(w.f[VY], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] += dtr[c] * (syx_x[c] + syy_y[c] + syz_z[c]);
    st4m(w.f[VY], i0, v, q.mask);
    f4a(v, ldw4(w.f[VZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] += dtr[c] * (szx_x[c] + szy_y[c] + szz_z[c]);
    st4m(w.f[VZ], i0, v, q.mask);
}

template <bool WITH_SAU>
__device__ __forceinline__ void stress_pml_group(const GridDev &g, const CpmlDev &P, const WaveDev &w,
                                                 const float *__restrict__ lam, const float *__restrict__ mu,
                                                 const float *__restrict__ vpm, const PmlPos &q) {
    const int sy = (int)g.sy, sz = (int)g.sz;
    const int i0 = (int)g.xoff + q.xs + sy * q.y + sz * q.z;
    const float c0 = c_dc2[0], c1 = c_dc2[1];
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    float win[12], vx_x[4], vy_x[4], vz_x[4], vx_y[4], vy_y[4], vz_y[4], vx_z[4], vy_z[4], vz_z[4];
    xwin(w.f[VX], i0, win);
    xdm2(win, c0, c1, vx_x);
    xwin(w.f[VY], i0, win);
    xdp2(win, c0, c1, vy_x);
    xwin(w.f[VZ], i0, win);
    xdp2(win, c0, c1, vz_x);
    sdp2(w.f[VX], i0, sy, c0, c1, vx_y);
    sdm2(w.f[VY], i0, sy, c0, c1, vy_y);
    sdp2(w.f[VZ], i0, sy, c0, c1, vz_y);
    sdp2(w.f[VX], i0, sz, c0, c1, vx_z);
    sdp2(w.f[VY], i0, sz, c0, c1, vy_z);
    sdm2(w.f[VZ], i0, sz, c0, c1, vz_z);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        vx_x[c] *= rdx; vy_x[c] *= rdx; vz_x[c] *= rdx;
        vx_y[c] *= rdy; vy_y[c] *= rdy; vz_y[c] *= rdy;
        vx_z[c] *= rdz; vy_z[c] *= rdz; vz_z[c] *= rdz;
    }
    float vp4[4];
    f4a(vp4, ld4(vpm, i0));
    float *psi = P.psi + q.psi + 3LL * q.naxes * q.stride;
    const long long n = q.stride;
    float A[4], B[4], Ah[4], Bh[4];
    bool any;
    xcoef4(P, q, vp4, A, B, Ah, Bh, any);
    if (any) {
        psi4(psi + 0 * n, B, A, vx_x);
        psi4(psi + 1 * n, Bh, Ah, vy_x);
        psi4(psi + 2 * n, Bh, Ah, vz_x);
    }
    const float4 ty = P.ax[1][q.y], tz = P.ax[2][q.z];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ty.x > 0.f) {
#pragma unroll
        for (int c = 0; c < 4; c++) cpml_coef(vp4[c], (q.mask >> c) & 1u ? ty : z4, P.dt, A[c], B[c], Ah[c], Bh[c]);
        psi4(psi + 3 * n, B, A, vy_y);
        psi4(psi + 4 * n, Bh, Ah, vx_y);
        psi4(psi + 5 * n, Bh, Ah, vz_y);
    }
    if (tz.x > 0.f) {
#pragma unroll
        for (int c = 0; c < 4; c++) cpml_coef(vp4[c], (q.mask >> c) & 1u ? tz : z4, P.dt, A[c], B[c], Ah[c], Bh[c]);
        psi4(psi + 6 * n, B, A, vz_z);
        psi4(psi + 7 * n, Bh, Ah, vx_z);
        psi4(psi + 8 * n, Bh, Ah, vy_z);
    }
    float l[4], m[4], a[4];
    f4a(l, ld4(lam, i0));
    f4a(m, ld4(mu, i0));
    const float dt = P.dt;
    f4a(a, ldw4(w.f[SXX], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * ((l[c] + 2.0f * m[c]) * vx_x[c] + l[c] * vy_y[c] + l[c] * vz_z[c]);
    st4m(w.f[SXX], i0, a, q.mask);
    f4a(a, ldw4(w.f[SYY], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * (l[c] * vx_x[c] + (l[c] + 2.0f * m[c]) * vy_y[c] + l[c] * vz_z[c]);
    st4m(w.f[SYY], i0, a, q.mask);
    f4a(a, ldw4(w.f[SZZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * (l[c] * vx_x[c] + l[c] * vy_y[c] + (l[c] + 2.0f * m[c]) * vz_z[c]);
    st4m(w.f[SZZ], i0, a, q.mask);
    if (WITH_SAU) {
        f4a(a, ldw4(w.f[SAU], i0));
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float l2m = l[c] + 2.0f * m[c];
            a[c] += dt * (l2m * vx_x[c] + l2m * vy_y[c] + l2m * vz_z[c]);
        }
        st4m(w.f[SAU], i0, a, q.mask);
    }
    f4a(a, ldw4(w.f[SXY], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * m[c] * (vy_x[c] + vx_y[c]);
    st4m(w.f[SXY], i0, a, q.mask);
    f4a(a, ldw4(w.f[SXZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * m[c] * (vz_x[c] + vx_z[c]);
    st4m(w.f[SXZ], i0, a, q.mask);
    f4a(a, ldw4(w.f[SYZ], i0));
#pragma unroll
    for (int c = 0; c < 4; c++) a[c] += dt * m[c] * (vz_y[c] + vy_z[c]);
    st4m(w.f[SYZ], i0, a, q.mask);
}

// Blocks of 256 threads over (slab, row block, plane block); a thread
// updates its group in P.zp consecutive planes of its slab.
template <int MINB, int ZP>
__global__ void __launch_bounds__(256, MINB) vel_pml(GridDev g, CpmlDev P, WaveDev w, const float *__restrict__ bdt,
                                                  const float *__restrict__ vpm) {
    PmlPos q;
    if (!pml_pos(P, q)) return;
#pragma unroll
    for (int zz = 0; zz < ZP; zz++) {
        if (q.z >= q.z1) break;
        vel_pml_group(g, P, w, bdt, vpm, q);
        q.z++;
        q.psi += q.plane;
    }
}

template <bool WITH_SAU, int MINB, int ZP>
__global__ void __launch_bounds__(256, MINB) stress_pml(GridDev g, CpmlDev P, WaveDev w,
                                                     const float *__restrict__ lam, const float *__restrict__ mu,
                                                     const float *__restrict__ vpm) {
    PmlPos q;
    if (!pml_pos(P, q)) return;
#pragma unroll
    for (int zz = 0; zz < ZP; zz++) {
        if (q.z >= q.z1) break;
        stress_pml_group<WITH_SAU>(g, P, w, lam, mu, vpm, q);
        q.z++;
        q.psi += q.plane;
    }
}

// ------------------------------------------------- full-gridext stress update
//
// Variant 4 of the stress update for the steps that carry absorbing
// layers (forward modelling, the RTM forward pass and the receiver
// wavefield): one persistent z-marching kernel over every updated cell of
// gridext, [2, n-2) on each axis.  It merges the 8th-order interior update
// (stress_zm3) and the 4th-order CPML update of the six slabs
// (stress_pml), so each velocity value is brought on chip once per step
// and the absorbing layers run behind the same TMA pipeline as the
// interior.  Items are (4-row tile, plane) with y in [2, ny-2) and z in
// [2, nz-2); a tile row is the whole updated x range.  Threads own x
// pairs: the first 4*hxi threads the physical x range [m, m+px), the rest
// the two absorbing x ranges [2, m) and [m+px, nx-2), so a warp takes one
// branch except at the single warp where the two groups meet and in tiles
// that straddle y = m or y = m+py.  Both m and px are even, which keeps
// every region boundary on a pair boundary.  A cell is interior when x, y
// and z are all in the physical range; it then takes the 8th-order update
// of stress_phy (FD/fdtd3d_0_base_module/fdtd3d_base_3_kernel_device_meat.hpp)
// and the explosive source.  Any other cell takes the CPML update of
// stress_pml_group (4th order, memory variables on its absorbing axes,
// FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_2_kernel_device_{x,y,z}_meat.hpp);
// its memory variables are the axis-major arrays of FzGeo, brought in by
// TMA with the fields and written back with plain stores.  The z windows hold
// planes z-4 .. z+4; planes outside gridext read as zero (their taps have
// zero weight wherever they are reached).

constexpr int kFzCore = kZmCore + 1;  // vx vy vz (window feed), lam, mu, vp, sxx syy szz sxy sxz syz, sau
constexpr int kFzStage = 3 * kZmHB + kFzCore * kZmCB;

struct FzMaps {
    CUtensorMap halo[3];
    CUtensorMap core[kFzCore];
    CUtensorMap psi[3];
};

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int x, int y, int z, int w,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(bar)
        : "memory");
}

// stage layout: halo planes, core tiles, then the three memory-variable
// boxes (3 arrays x 4 rows each), every region 128-byte aligned
__host__ __device__ constexpr int fz_round32(int n) { return (n + 31) / 32 * 32; }
__host__ __device__ inline int fz_stage(const FzGeo &g) {
    return kFzStage + fz_round32(12 * g.PX) + 2 * fz_round32(12 * g.PB);
}

// x tiles of the full-gridext kernels: the first cell of tile xt
__host__ __device__ inline int fz_xlo(const GridDev &g, const FzGeo &q, int xt) {
    return xt == 0 ? 2 : g.m + 2 * xt * q.TPP;
}
// ... and one past its last
__host__ __device__ inline int fz_xhi(const GridDev &g, const FzGeo &q, int xt) {
    return xt == q.NTX - 1 ? g.nx - 2 : g.m + 2 * (xt + 1) * q.TPP;
}

// The pair of a thread in an x tile.  FzLane holds the tile-invariant part
// (computed once per thread); fz_lane gives, for tile xt, the row r, the
// first cell x, whether it absorbs in x, and live = false when the thread
// has no pair there.  Threads [0, 4 TPP): physical pairs; up to tpad (a
// warp multiple where that still fits one CTA): none; from tpad:
// absorbing pairs -- then no warp mixes the two updates.
struct FzLane {
    int r, k;   // row; pair within the tile's physical pairs, or absorbing pair index
    bool phys;
};
__device__ __forceinline__ FzLane fz_lane0(const FzGeo &q, int tid) {
    FzLane L;
    L.phys = tid < q.tpad;
    if (L.phys) {
        L.r = tid / q.TPP;
        L.k = tid - L.r * q.TPP;
    } else {
        const int e = tid - q.tpad;
        L.r = e / q.hxe;
        L.k = e - L.r * q.hxe;
    }
    return L;
}
__device__ __forceinline__ void fz_lane(const GridDev &g, const FzGeo &q, const FzLane &L, int xt, int &r, int &x,
                                        bool &xabs, bool &live) {
    const int m = g.m;
    if (L.phys) {
        xabs = false;
        const int gp = xt * q.TPP + L.k;
        live = L.r < kZmRows && gp < q.hxi;
        r = live ? L.r : 0;
        x = m + 2 * (live ? gp : 0);
    } else {
        xabs = true;
        r = L.r;
        if (q.NTX == 1) {
            const int half = q.hxe / 2;
            x = L.k < half ? 2 + 2 * L.k : m + g.px + 2 * (L.k - half);
            live = true;
        } else {
            live = xt == 0 || xt == q.NTX - 1;
            x = xt == 0 ? 2 + 2 * L.k : m + g.px + 2 * L.k;
        }
    }
}

template <int MODE, bool XT>
__global__ void __launch_bounds__(kZmMaxThreads, 1)
    stress_fz(GridDev g, const __grid_constant__ FzMaps maps, WaveDev w, float dt, const float *__restrict__ wavelet,
              const StepState *__restrict__ st, int it_off, const __grid_constant__ FzGeo geo, int *err) {
    static_assert(MODE != kBwd, "the source reconstruction carries no absorbing layers");
    constexpr bool kSau = MODE != kFwd;
    constexpr int NCT = kSau ? kFzCore : kFzCore - 1;  // sau is neither read nor written in forward modelling
    extern __shared__ __align__(128) float sm[];
    constexpr int hb = kZmHB, cb = kZmCB, boxw = kZmPitch;
    const int stage = fz_stage(geo);
    const int pxr = fz_round32(12 * geo.PX), pyr = fz_round32(12 * geo.PB);
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_abort;
    // this CTA's runs: blockIdx.x, blockIdx.x + gridDim.x, ...; L items each
    const int nrun = (geo.R - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    const int w0 = 0, w1 = nrun * geo.L;
    if (nrun <= 0) return;
    // item -> (x tile, y tile, plane); planes past the last one are idle items
    const int ntile = geo.NTX * geo.ytiles;
    auto item_at = [&](int item, int &xt, int &yt, int &z) {
        const int j = item / geo.L, off = item - j * geo.L;
        const int rr = (int)blockIdx.x + j * (int)gridDim.x;
        const int q = rr / ntile, t = rr - q * ntile;
        if (!XT) {  // one x tile: every tile quantity is loop-invariant
            yt = t;
            xt = 0;
        } else {
            yt = t / geo.NTX;
            xt = t - yt * geo.NTX;
        }
        z = 2 + q * geo.L + off;
    };
    const int tid = threadIdx.x;
    const int m = g.m;
    const FzLane ln = fz_lane0(geo, tid);
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const uint32_t bytes_all = (uint32_t)(3 * hb + NCT * geo.corew * kZmRows) * 4u;
    const uint32_t bytes_feed = (uint32_t)(3 * geo.corew * kZmRows) * 4u;
    const uint32_t bytes_psx = (uint32_t)(12 * geo.PX) * 4u, bytes_psy = (uint32_t)(12 * geo.PB) * 4u;
    auto issue = [&](int item, int b) {
        int xt, yt, z;
        item_at(item, xt, yt, z);
        const uint32_t bar = b ? bar1 : bar0;
        if (z >= g.nz - 2) {
            mbar_expect(bar, 0);  // idle item: the phase completes with this arrival
            return;
        }
        const int Y = 2 + yt * kZmRows;
        float *base = sm + b * stage;
        const bool feed = z + 5 < g.nz;  // the window's next plane; none past gridext
        const bool zab = z < m || z >= m + g.pz;
        const bool ylo = Y < m, yhi = Y + kZmRows - 1 >= m + g.py;  // the tile holds absorbing rows
        const bool xab = !XT || xt == 0 || xt == geo.NTX - 1;      // ... or absorbing columns
        const int xlo = fz_xlo(g, geo, xt);
        const int XC = ((int)g.xoff + xlo) & ~3, XH = XC - kZmHalo, xb0 = (xlo - 2) & ~3;
        mbar_expect(bar, (feed ? bytes_all : bytes_all - bytes_feed) + (xab ? bytes_psx : 0u) +
                             (ylo || yhi ? bytes_psy : 0u) + (zab ? bytes_psy : 0u));
        for (int f = 0; f < 3; f++) tma_load_3d(smem_u32(base + f * hb), &maps.halo[f], XH, Y - kZmHalo, z, bar);
        if (feed)
            for (int f = 0; f < 3; f++)
                tma_load_3d(smem_u32(base + 3 * hb + f * cb), &maps.core[f], XC, Y, z + 5, bar);
        for (int f = 3; f < NCT; f++) tma_load_3d(smem_u32(base + 3 * hb + f * cb), &maps.core[f], XC, Y, z, bar);
        float *ps = base + kFzStage;
        if (xab) tma_load_4d(smem_u32(ps), &maps.psi[0], 0, Y - 2, z - 2, 0, bar);
        if (ylo || yhi)
            tma_load_4d(smem_u32(ps + pxr), &maps.psi[1], xb0, ylo ? Y - 2 : m - 2 + Y - (m + g.py), z - 2, 0, bar);
        if (zab)
            tma_load_4d(smem_u32(ps + pxr + pyr), &maps.psi[2], xb0, Y - 2, z < m ? z - 2 : m - 2 + z - (m + g.pz), 0,
                        bar);
    };
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        issue(w0, 0);
        if (w0 + 1 < w1) issue(w0 + 1, 1);
    }
    const int sy = (int)g.sy, sz = (int)g.sz;
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    float2 rv[3][9];                           // z windows: planes z-4 .. z+4 of vx, vy, vz
    const float *fv[3] = {w.f[VX], w.f[VY], w.f[VZ]};
    // with one x tile the pair and the boxes are the same for every item
    int r1, x1, XC1, xb1;
    bool xabs1, lane1;
    fz_lane(g, geo, ln, 0, r1, x1, xabs1, lane1);
    XC1 = ((int)g.xoff + 2) & ~3;
    xb1 = 0;
    int cur_t = -1, cur_z = -2;
    for (int k = w0; k < w1; k++) {
        int xt, yt, z;
        item_at(k, xt, yt, z);
        int r = r1, x = x1, XC = XC1, xb0 = xb1;
        bool xabs = xabs1, lane = lane1;
        if (XT) {
            fz_lane(g, geo, ln, xt, r, x, xabs, lane);
            const int xlo = fz_xlo(g, geo, xt);
            XC = ((int)g.xoff + xlo) & ~3;
            xb0 = (xlo - 2) & ~3;
        }
        const int hcol = (int)g.xoff + x - (XC - kZmHalo);  // the pair's first cell in a halo row (even)
        const int ccol = (int)g.xoff + x - XC;              // ... in a core row (even)
        const int y = 2 + yt * kZmRows + r;
        const bool live = lane && y < g.ny - 2 && z < g.nz - 2;
        const int i0 = (int)g.xoff + x + sy * y + sz * z;  // even: float2-aligned
        const int b = (k - w0) & 1;
        const uint32_t parity = (uint32_t)(((k - w0) >> 1) & 1);
        const float *base = sm + b * stage;
        const int cc = r * geo.corew + ccol;
        const int t = yt * geo.NTX + xt;
        if (t != cur_t || z != cur_z + 1) {
            // a new run of planes: fill the z windows from global memory
#pragma unroll
            for (int f = 0; f < 3; f++) {
#pragma unroll
                for (int q = 0; q < 9; q++) {
                    const int zq = z + q - 4;
                    rv[f][q] = (live && zq >= 0 && zq < g.nz)
                                   ? __ldg(reinterpret_cast<const float2 *>(fv[f] + i0 + (q - 4) * sz))
                                   : make_float2(0.f, 0.f);
                }
            }
        }
        cur_t = t;
        cur_z = z;
        if (!mbar_wait_bounded(b ? bar1 : bar0, parity)) {
            s_abort = 1;
            atomicExch(err, 1);
        }
        if (live) {
            const float *C = base + 3 * hb;  // core tiles
            const int c0 = (r + kZmHalo) * boxw + hcol;
            auto ld2 = [&](const float *F, int off) { return *reinterpret_cast<const float2 *>(F + off); };
            // x window of a field around the pair: e[j] = f[x - 4 + j], j = 0..9
            auto xwin2 = [&](const float *F, float *e) {
#pragma unroll
                for (int j = 0; j < 5; j++) {
                    const float2 v = ld2(F, c0 - 4 + 2 * j);
                    e[2 * j] = v.x;
                    e[2 * j + 1] = v.y;
                }
            };
            const bool zabs = z < m || z >= m + g.pz;
            const bool yabs = y < m || y >= m + g.py;
            const bool cpml = xabs || yabs || zabs;
            float Nx[2], Ny[2], Nz[2], Sxy[2], Sxz[2], Syz[2];
            float e[10];
            if (!cpml) {
                const float *cf = c_list[kPhyHalf];
                // vx: Dm_x -> Nx, Dp_y -> Sxy, Dp_z -> Sxz
                xwin2(base, e);
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    float t = 0.f;
#pragma unroll
                    for (int q = 0; q < 4; q++) t += cf[q] * (e[4 + c + q] - e[4 + c - q - 1]);
                    Nx[c] = t * rdx;
                }
                {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float2 a = ld2(base, c0 + (q + 1) * boxw), bb = ld2(base, c0 - q * boxw);
                        t.x += cf[q] * (a.x - bb.x);
                        t.y += cf[q] * (a.y - bb.y);
                    }
                    Sxy[0] = t.x * rdy;
                    Sxy[1] = t.y * rdy;
                    t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        t.x += cf[q] * (rv[0][4 + q + 1].x - rv[0][4 - q].x);
                        t.y += cf[q] * (rv[0][4 + q + 1].y - rv[0][4 - q].y);
                    }
                    Sxz[0] = t.x * rdz;
                    Sxz[1] = t.y * rdz;
                }
                // vy: Dp_x -> Sxy, Dm_y -> Ny, Dp_z -> Syz
                xwin2(base + hb, e);
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    float t = 0.f;
#pragma unroll
                    for (int q = 0; q < 4; q++) t += cf[q] * (e[4 + c + q + 1] - e[4 + c - q]);
                    Sxy[c] += t * rdx;
                }
                {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float2 a = ld2(base + hb, c0 + q * boxw), bb = ld2(base + hb, c0 - (q + 1) * boxw);
                        t.x += cf[q] * (a.x - bb.x);
                        t.y += cf[q] * (a.y - bb.y);
                    }
                    Ny[0] = t.x * rdy;
                    Ny[1] = t.y * rdy;
                    t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        t.x += cf[q] * (rv[1][4 + q + 1].x - rv[1][4 - q].x);
                        t.y += cf[q] * (rv[1][4 + q + 1].y - rv[1][4 - q].y);
                    }
                    Syz[0] = t.x * rdz;
                    Syz[1] = t.y * rdz;
                }
                // vz: Dp_x -> Sxz, Dp_y -> Syz, Dm_z -> Nz
                xwin2(base + 2 * hb, e);
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    float t = 0.f;
#pragma unroll
                    for (int q = 0; q < 4; q++) t += cf[q] * (e[4 + c + q + 1] - e[4 + c - q]);
                    Sxz[c] += t * rdx;
                }
                {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float2 a = ld2(base + 2 * hb, c0 + (q + 1) * boxw),
                                     bb = ld2(base + 2 * hb, c0 - q * boxw);
                        t.x += cf[q] * (a.x - bb.x);
                        t.y += cf[q] * (a.y - bb.y);
                    }
                    Syz[0] += t.x * rdy;
                    Syz[1] += t.y * rdy;
                    t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        t.x += cf[q] * (rv[2][4 + q].x - rv[2][4 - q - 1].x);
                        t.y += cf[q] * (rv[2][4 + q].y - rv[2][4 - q - 1].y);
                    }
                    Nz[0] = t.x * rdz;
                    Nz[1] = t.y * rdz;
                }
            } else {
                // 4th-order differences of the absorbing layers, then the
                // memory variables of the absorbing axes
                const float k0 = c_dc2[0], k1 = c_dc2[1];
                float d[9][2];  // vx_x vy_x vz_x | vy_y vx_y vz_y | vz_z vx_z vy_z
                xwin2(base, e);
#pragma unroll
                for (int c = 0; c < 2; c++) d[0][c] = (k0 * (e[4 + c] - e[3 + c]) + k1 * (e[5 + c] - e[2 + c])) * rdx;
                xwin2(base + hb, e);
#pragma unroll
                for (int c = 0; c < 2; c++) d[1][c] = (k0 * (e[5 + c] - e[4 + c]) + k1 * (e[6 + c] - e[3 + c])) * rdx;
                xwin2(base + 2 * hb, e);
#pragma unroll
                for (int c = 0; c < 2; c++) d[2][c] = (k0 * (e[5 + c] - e[4 + c]) + k1 * (e[6 + c] - e[3 + c])) * rdx;
                {
                    // Dm_y vy
                    const float *F = base + hb;
                    const float2 a = ld2(F, c0), bb = ld2(F, c0 - boxw), cq = ld2(F, c0 + boxw),
                                 dq = ld2(F, c0 - 2 * boxw);
                    d[3][0] = (k0 * (a.x - bb.x) + k1 * (cq.x - dq.x)) * rdy;
                    d[3][1] = (k0 * (a.y - bb.y) + k1 * (cq.y - dq.y)) * rdy;
                }
#pragma unroll
                for (int f = 0; f < 3; f += 2) {
                    // Dp_y vx -> d[4], Dp_y vz -> d[5]
                    const float *F = base + f * hb;
                    const float2 a = ld2(F, c0 + boxw), bb = ld2(F, c0), cq = ld2(F, c0 + 2 * boxw),
                                 dq = ld2(F, c0 - boxw);
                    d[4 + f / 2][0] = (k0 * (a.x - bb.x) + k1 * (cq.x - dq.x)) * rdy;
                    d[4 + f / 2][1] = (k0 * (a.y - bb.y) + k1 * (cq.y - dq.y)) * rdy;
                }
                // Dm_z vz -> d[6]; Dp_z vx -> d[7], vy -> d[8]
                d[6][0] = (k0 * (rv[2][4].x - rv[2][3].x) + k1 * (rv[2][5].x - rv[2][2].x)) * rdz;
                d[6][1] = (k0 * (rv[2][4].y - rv[2][3].y) + k1 * (rv[2][5].y - rv[2][2].y)) * rdz;
#pragma unroll
                for (int f = 0; f < 2; f++) {
                    d[7 + f][0] = (k0 * (rv[f][5].x - rv[f][4].x) + k1 * (rv[f][6].x - rv[f][3].x)) * rdz;
                    d[7 + f][1] = (k0 * (rv[f][5].y - rv[f][4].y) + k1 * (rv[f][6].y - rv[f][3].y)) * rdz;
                }
                // memory variables: this tile's boxes in shared memory, the
                // axis-major arrays in global memory
                const float *PS = base + kFzStage;
                const int zi = z - 2, yi = y - 2, xi = x - 2;
                const float2 vp2 = ld2(C, 5 * cb + cc);
                const float vpc[2] = {vp2.x, vp2.y};
                float A[2], B[2], Ah[2], Bh[2];
                auto upd = [&](const float *sp, float *gp, const float *BB, const float *AA, float *dd) {
                    float2 v = *reinterpret_cast<const float2 *>(sp);
                    v.x = BB[0] * v.x + AA[0] * dd[0];
                    v.y = BB[1] * v.y + AA[1] * dd[1];
                    *reinterpret_cast<float2 *>(gp) = v;
                    dd[0] += v.x;
                    dd[1] += v.y;
                };
                if (xabs) {
                    const int xc = x < m ? x - 2 : m - 2 + x - (m + g.px);
                    const long long a0 = ((long long)zi * (g.ny - 4) + yi) * geo.PX + xc;
                    const long long as = (long long)(g.nz - 4) * (g.ny - 4) * geo.PX;
                    const int s0 = r * geo.PX + xc, ss = 4 * geo.PX;
#pragma unroll
                    for (int c = 0; c < 2; c++) cpml_coef(vpc[c], __ldg(&geo.ax[0][x + c]), dt, A[c], B[c], Ah[c], Bh[c]);
                    upd(PS + s0, geo.psx + a0, B, A, d[0]);
                    upd(PS + s0 + ss, geo.psx + a0 + as, Bh, Ah, d[1]);
                    upd(PS + s0 + 2 * ss, geo.psx + a0 + 2 * as, Bh, Ah, d[2]);
                }
                if (yabs) {
                    const int yc = y < m ? y - 2 : m - 2 + y - (m + g.py);
                    const long long a0 = ((long long)zi * geo.W + yc) * geo.PY + xi;
                    const long long as = (long long)(g.nz - 4) * geo.W * geo.PY;
                    const int s0 = pxr + r * geo.PB + (xi - xb0), ss = 4 * geo.PB;
                    const float4 ty = __ldg(&geo.ax[1][y]);
#pragma unroll
                    for (int c = 0; c < 2; c++) cpml_coef(vpc[c], ty, dt, A[c], B[c], Ah[c], Bh[c]);
                    upd(PS + s0, geo.psy + a0, B, A, d[3]);
                    upd(PS + s0 + ss, geo.psy + a0 + as, Bh, Ah, d[4]);
                    upd(PS + s0 + 2 * ss, geo.psy + a0 + 2 * as, Bh, Ah, d[5]);
                }
                if (zabs) {
                    const int zc = z < m ? z - 2 : m - 2 + z - (m + g.pz);
                    const long long a0 = ((long long)zc * (g.ny - 4) + yi) * geo.PY + xi;
                    const long long as = (long long)geo.W * (g.ny - 4) * geo.PY;
                    const int s0 = pxr + pyr + r * geo.PB + (xi - xb0), ss = 4 * geo.PB;
                    const float4 tz = __ldg(&geo.ax[2][z]);
#pragma unroll
                    for (int c = 0; c < 2; c++) cpml_coef(vpc[c], tz, dt, A[c], B[c], Ah[c], Bh[c]);
                    upd(PS + s0, geo.psz + a0, B, A, d[6]);
                    upd(PS + s0 + ss, geo.psz + a0 + as, Bh, Ah, d[7]);
                    upd(PS + s0 + 2 * ss, geo.psz + a0 + 2 * as, Bh, Ah, d[8]);
                }
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    Nx[c] = d[0][c];
                    Ny[c] = d[3][c];
                    Nz[c] = d[6][c];
                    Sxy[c] = d[1][c] + d[4][c];
                    Sxz[c] = d[2][c] + d[7][c];
                    Syz[c] = d[5][c] + d[8][c];
                }
            }
            const float2 l2 = ld2(C, 3 * cb + cc), m2 = ld2(C, 4 * cb + cc);
            const float l[2] = {l2.x, l2.y}, mm[2] = {m2.x, m2.y};
            const float2 s0 = ld2(C, 6 * cb + cc), s1 = ld2(C, 7 * cb + cc), s2 = ld2(C, 8 * cb + cc);
            float sxx[2] = {s0.x, s0.y}, syy[2] = {s1.x, s1.y}, szz[2] = {s2.x, s2.y};
            if (MODE != kRev && !cpml) {
                // explosive source (physical cells), applied before the stress update of step it
                const long long dd = st->src - (long long)i0;
                if (dd >= 0 && dd < 2) {
                    const float sv = wavelet[st->it + it_off];
                    sxx[dd] += sv;
                    syy[dd] += sv;
                    szz[dd] += sv;
                }
            }
            const float2 t9 = ld2(C, 9 * cb + cc), t10 = ld2(C, 10 * cb + cc), t11 = ld2(C, 11 * cb + cc);
            const float sxy0[2] = {t9.x, t9.y}, sxz0[2] = {t10.x, t10.y}, syz0[2] = {t11.x, t11.y};
            float sau0[2] = {0.f, 0.f};
            if (kSau) {
                const float2 t12 = ld2(C, 12 * cb + cc);
                sau0[0] = t12.x;
                sau0[1] = t12.y;
            }
            float o[7][2];
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const float l2m = l[c] + 2.0f * mm[c];
                o[0][c] = sxx[c] + dt * (l2m * Nx[c] + l[c] * Ny[c] + l[c] * Nz[c]);
                o[1][c] = syy[c] + dt * (l[c] * Nx[c] + l2m * Ny[c] + l[c] * Nz[c]);
                o[2][c] = szz[c] + dt * (l[c] * Nx[c] + l[c] * Ny[c] + l2m * Nz[c]);
                o[3][c] = sxy0[c] + dt * mm[c] * Sxy[c];
                o[4][c] = sxz0[c] + dt * mm[c] * Sxz[c];
                o[5][c] = syz0[c] + dt * mm[c] * Syz[c];
                o[6][c] = sau0[c] + dt * l2m * (Nx[c] + Ny[c] + Nz[c]);
            }
            const int outf[7] = {SXX, SYY, SZZ, SXY, SXZ, SYZ, SAU};
#pragma unroll
            for (int j = 0; j < 7; j++) {
                if (j == 6 && !kSau) break;
                *reinterpret_cast<float2 *>(w.f[outf[j]] + i0) = make_float2(o[j][0], o[j][1]);
            }
            // advance the z windows: the plane five above came in with this item
            const bool fed = z + 5 < g.nz;
#pragma unroll
            for (int f = 0; f < 3; f++) {
#pragma unroll
                for (int q = 0; q < 8; q++) rv[f][q] = rv[f][q + 1];
                rv[f][8] = fed ? ld2(C, f * cb + cc) : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();  // every thread is done with buffer b
        if (s_abort) {
            if (tid == 0) {
                mbar_wait_bounded(b ? bar1 : bar0, parity);
                if (k + 1 < w1) {
                    const int k1 = k + 1 - w0;
                    mbar_wait_bounded((k1 & 1) ? bar1 : bar0, (uint32_t)((k1 >> 1) & 1));
                }
            }
            __syncthreads();
            return;
        }
        if (tid == 0 && k + 2 < w1) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(k + 2, b);
        }
    }
}

// --------------------------------------------- full-gridext velocity update
//
// Variant 4 of the velocity update for the steps that carry absorbing
// layers: vel_phy's 8th-order update of the physical cells
// (FD/fdtd3d_0_base_module/fdtd3d_base_3_kernel_device_meat.hpp) and
// vel_pml_group's 4th-order CPML update of the others in one persistent
// z-marching kernel, with the tiling, thread layout, run schedule and
// axis-major memory variables of stress_fz.  Per item TMA brings halo
// planes (12 rows) of sxy, syy, syz; 4-row bands with the x halo of sxx
// and sxz; the core tiles of dt/rho, vp, vx, vy, vz; the window feed of sxz,
// syz, szz five planes ahead; the memory-variable boxes.  The z windows
// hold sxz, syz, szz.  It serves the passes without P-wave velocities
// (forward modelling, the RTM forward pass) on grids of one x tile; the
// receiver wavefield and x-tiled grids keep vel_phy_v4 + vel_pml, which
// measured as fast or faster there.

constexpr int kFvStage = 3 * kZmHB + 10 * kZmCB;  // halo planes, 2 bands, 5 core tiles, 3 feed tiles

struct FvMaps {
    CUtensorMap halo[3];  // sxy syy syz
    CUtensorMap band[2];  // sxx sxz
    CUtensorMap core[5];  // dt/rho vp vx vy vz
    CUtensorMap feed[3];  // sxz syz szz (core boxes)
    CUtensorMap psi[3];
};

__host__ __device__ inline int fv_stage(const FzGeo &g) {
    return kFvStage + fz_round32(12 * g.PX) + 2 * fz_round32(12 * g.PB);
}

template <bool XT>
__global__ void __launch_bounds__(kZmMaxThreads, 1)
    vel_fz(GridDev g, const __grid_constant__ FvMaps maps, WaveDev w, float dt, const __grid_constant__ FzGeo geo,
           int *err) {
    extern __shared__ __align__(128) float sm[];
    constexpr int hb = kZmHB, cb = kZmCB, boxw = kZmPitch;
    const int stage = fv_stage(geo);
    const int pxr = fz_round32(12 * geo.PX), pyr = fz_round32(12 * geo.PB);
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ int s_abort;
    const int nrun = (geo.R - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    const int w0 = 0, w1 = nrun * geo.L;
    if (nrun <= 0) return;
    const int ntile = geo.NTX * geo.ytiles;
    auto item_at = [&](int item, int &xt, int &yt, int &z) {
        const int j = item / geo.L, off = item - j * geo.L;
        const int rr = (int)blockIdx.x + j * (int)gridDim.x;
        const int q = rr / ntile, t = rr - q * ntile;
        if (!XT) {  // one x tile: every tile quantity is loop-invariant
            yt = t;
            xt = 0;
        } else {
            yt = t / geo.NTX;
            xt = t - yt * geo.NTX;
        }
        z = 2 + q * geo.L + off;
    };
    const int tid = threadIdx.x;
    const int m = g.m;
    const FzLane ln = fz_lane0(geo, tid);
    const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const uint32_t bytes_feed = (uint32_t)(3 * geo.corew * kZmRows) * 4u;
    const uint32_t bytes_all = (uint32_t)(3 * hb + 2 * cb + 5 * geo.corew * kZmRows) * 4u + bytes_feed;
    const uint32_t bytes_psx = (uint32_t)(12 * geo.PX) * 4u, bytes_psy = (uint32_t)(12 * geo.PB) * 4u;
    auto issue = [&](int item, int b) {
        int xt, yt, z;
        item_at(item, xt, yt, z);
        const uint32_t bar = b ? bar1 : bar0;
        if (z >= g.nz - 2) {
            mbar_expect(bar, 0);
            return;
        }
        const int Y = 2 + yt * kZmRows;
        float *base = sm + b * stage;
        const bool feed = z + 5 < g.nz;
        const bool zab = z < m || z >= m + g.pz;
        const bool ylo = Y < m, yhi = Y + kZmRows - 1 >= m + g.py;
        const bool xab = !XT || xt == 0 || xt == geo.NTX - 1;
        const int xlo = fz_xlo(g, geo, xt);
        const int XC = ((int)g.xoff + xlo) & ~3, XH = XC - kZmHalo, xb0 = (xlo - 2) & ~3;
        mbar_expect(bar, (feed ? bytes_all : bytes_all - bytes_feed) + (xab ? bytes_psx : 0u) +
                             (ylo || yhi ? bytes_psy : 0u) + (zab ? bytes_psy : 0u));
        for (int f = 0; f < 3; f++) tma_load_3d(smem_u32(base + f * hb), &maps.halo[f], XH, Y - kZmHalo, z, bar);
        for (int f = 0; f < 2; f++) tma_load_3d(smem_u32(base + 3 * hb + f * cb), &maps.band[f], XH, Y, z, bar);
        for (int f = 0; f < 5; f++) tma_load_3d(smem_u32(base + 3 * hb + (2 + f) * cb), &maps.core[f], XC, Y, z, bar);
        if (feed)
            for (int f = 0; f < 3; f++)
                tma_load_3d(smem_u32(base + 3 * hb + (7 + f) * cb), &maps.feed[f], XC, Y, z + 5, bar);
        float *ps = base + kFvStage;
        if (xab) tma_load_4d(smem_u32(ps), &maps.psi[0], 0, Y - 2, z - 2, 0, bar);
        if (ylo || yhi)
            tma_load_4d(smem_u32(ps + pxr), &maps.psi[1], xb0, ylo ? Y - 2 : m - 2 + Y - (m + g.py), z - 2, 0, bar);
        if (zab)
            tma_load_4d(smem_u32(ps + pxr + pyr), &maps.psi[2], xb0, Y - 2, z < m ? z - 2 : m - 2 + z - (m + g.pz), 0,
                        bar);
    };
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        issue(w0, 0);
        if (w0 + 1 < w1) issue(w0 + 1, 1);
    }
    const int sy = (int)g.sy, sz = (int)g.sz;
    const float rdx = 1.0f / g.dx, rdy = 1.0f / g.dy, rdz = 1.0f / g.dz;
    float2 rv[3][9];  // z windows: planes z-4 .. z+4 of sxz, syz, szz
    const float *fv[3] = {w.f[SXZ], w.f[SYZ], w.f[SZZ]};
    // with one x tile the pair and the boxes are the same for every item
    int r1, x1, XC1, xb1;
    bool xabs1, lane1;
    fz_lane(g, geo, ln, 0, r1, x1, xabs1, lane1);
    XC1 = ((int)g.xoff + 2) & ~3;
    xb1 = 0;
    int cur_t = -1, cur_z = -2;
    for (int k = w0; k < w1; k++) {
        int xt, yt, z;
        item_at(k, xt, yt, z);
        int r = r1, x = x1, XC = XC1, xb0 = xb1;
        bool xabs = xabs1, lane = lane1;
        if (XT) {
            fz_lane(g, geo, ln, xt, r, x, xabs, lane);
            const int xlo = fz_xlo(g, geo, xt);
            XC = ((int)g.xoff + xlo) & ~3;
            xb0 = (xlo - 2) & ~3;
        }
        const int hcol = (int)g.xoff + x - (XC - kZmHalo);
        const int ccol = (int)g.xoff + x - XC;
        const int t = yt * geo.NTX + xt;
        const int y = 2 + yt * kZmRows + r;
        const bool live = lane && y < g.ny - 2 && z < g.nz - 2;
        const int i0 = (int)g.xoff + x + sy * y + sz * z;
        const int b = (k - w0) & 1;
        const uint32_t parity = (uint32_t)(((k - w0) >> 1) & 1);
        const float *base = sm + b * stage;
        const int cc = r * geo.corew + ccol;
        if (t != cur_t || z != cur_z + 1) {
#pragma unroll
            for (int f = 0; f < 3; f++) {
#pragma unroll
                for (int q = 0; q < 9; q++) {
                    const int zq = z + q - 4;
                    rv[f][q] = (live && zq >= 0 && zq < g.nz)
                                   ? __ldg(reinterpret_cast<const float2 *>(fv[f] + i0 + (q - 4) * sz))
                                   : make_float2(0.f, 0.f);
                }
            }
        }
        cur_t = t;
        cur_z = z;
        if (!mbar_wait_bounded(b ? bar1 : bar0, parity)) {
            s_abort = 1;
            atomicExch(err, 1);
        }
        if (live) {
            const float *H = base;                  // halo planes: sxy, syy, syz
            const float *BD = base + 3 * hb;         // bands: sxx, sxz
            const float *C = base + 3 * hb + 2 * cb; // core: dt/rho, vp, vx, vy, vz
            const float *FD = base + 3 * hb + 7 * cb;
            const int c0 = (r + kZmHalo) * boxw + hcol;  // a halo plane
            const int b0 = r * boxw + hcol;              // a band
            auto ld2 = [&](const float *F, int off) { return *reinterpret_cast<const float2 *>(F + off); };
            auto xwin2 = [&](const float *F, int at, float *e) {
#pragma unroll
                for (int j = 0; j < 5; j++) {
                    const float2 v = ld2(F, at - 4 + 2 * j);
                    e[2 * j] = v.x;
                    e[2 * j + 1] = v.y;
                }
            };
            const bool zabs = z < m || z >= m + g.pz;
            const bool yabs = y < m || y >= m + g.py;
            const bool cpml = xabs || yabs || zabs;
            float Dx[2], Dy[2], Dz[2];
            float e[10];
            if (!cpml) {
                const float *cf = c_list[kPhyHalf];
                // vx: Dp_x sxx + Dm_y sxy + Dm_z sxz
                xwin2(BD, b0, e);
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    float t = 0.f;
#pragma unroll
                    for (int q = 0; q < 4; q++) t += cf[q] * (e[4 + c + q + 1] - e[4 + c - q]);
                    Dx[c] = t * rdx;
                }
                {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float2 a = ld2(H, c0 + q * boxw), bb = ld2(H, c0 - (q + 1) * boxw);
                        t.x += cf[q] * (a.x - bb.x);
                        t.y += cf[q] * (a.y - bb.y);
                    }
                    Dx[0] += t.x * rdy;
                    Dx[1] += t.y * rdy;
                    t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        t.x += cf[q] * (rv[0][4 + q].x - rv[0][4 - q - 1].x);
                        t.y += cf[q] * (rv[0][4 + q].y - rv[0][4 - q - 1].y);
                    }
                    Dx[0] += t.x * rdz;
                    Dx[1] += t.y * rdz;
                }
                // vy: Dm_x sxy + Dp_y syy + Dm_z syz
                xwin2(H, c0, e);
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    float t = 0.f;
#pragma unroll
                    for (int q = 0; q < 4; q++) t += cf[q] * (e[4 + c + q] - e[4 + c - q - 1]);
                    Dy[c] = t * rdx;
                }
                {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float2 a = ld2(H + hb, c0 + (q + 1) * boxw), bb = ld2(H + hb, c0 - q * boxw);
                        t.x += cf[q] * (a.x - bb.x);
                        t.y += cf[q] * (a.y - bb.y);
                    }
                    Dy[0] += t.x * rdy;
                    Dy[1] += t.y * rdy;
                    t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        t.x += cf[q] * (rv[1][4 + q].x - rv[1][4 - q - 1].x);
                        t.y += cf[q] * (rv[1][4 + q].y - rv[1][4 - q - 1].y);
                    }
                    Dy[0] += t.x * rdz;
                    Dy[1] += t.y * rdz;
                }
                // vz: Dm_x sxz + Dm_y syz + Dp_z szz
                xwin2(BD + cb, b0, e);
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    float t = 0.f;
#pragma unroll
                    for (int q = 0; q < 4; q++) t += cf[q] * (e[4 + c + q] - e[4 + c - q - 1]);
                    Dz[c] = t * rdx;
                }
                {
                    float2 t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float2 a = ld2(H + 2 * hb, c0 + q * boxw), bb = ld2(H + 2 * hb, c0 - (q + 1) * boxw);
                        t.x += cf[q] * (a.x - bb.x);
                        t.y += cf[q] * (a.y - bb.y);
                    }
                    Dz[0] += t.x * rdy;
                    Dz[1] += t.y * rdy;
                    t = make_float2(0.f, 0.f);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        t.x += cf[q] * (rv[2][4 + q + 1].x - rv[2][4 - q].x);
                        t.y += cf[q] * (rv[2][4 + q + 1].y - rv[2][4 - q].y);
                    }
                    Dz[0] += t.x * rdz;
                    Dz[1] += t.y * rdz;
                }
            } else {
                const float k0 = c_dc2[0], k1 = c_dc2[1];
                // sxx_x syx_x szx_x | sxy_y syy_y szy_y | sxz_z syz_z szz_z
                float d[9][2];
                xwin2(BD, b0, e);  // sxx: Dp_x
#pragma unroll
                for (int c = 0; c < 2; c++) d[0][c] = (k0 * (e[5 + c] - e[4 + c]) + k1 * (e[6 + c] - e[3 + c])) * rdx;
                xwin2(H, c0, e);  // sxy: Dm_x
#pragma unroll
                for (int c = 0; c < 2; c++) d[1][c] = (k0 * (e[4 + c] - e[3 + c]) + k1 * (e[5 + c] - e[2 + c])) * rdx;
                xwin2(BD + cb, b0, e);  // sxz: Dm_x
#pragma unroll
                for (int c = 0; c < 2; c++) d[2][c] = (k0 * (e[4 + c] - e[3 + c]) + k1 * (e[5 + c] - e[2 + c])) * rdx;
#pragma unroll
                for (int f = 0; f < 3; f += 2) {
                    // Dm_y sxy -> d[3], Dm_y syz -> d[5]
                    const float *F = H + f * hb;
                    const float2 a = ld2(F, c0), bb = ld2(F, c0 - boxw), cq = ld2(F, c0 + boxw),
                                 dq = ld2(F, c0 - 2 * boxw);
                    d[3 + f][0] = (k0 * (a.x - bb.x) + k1 * (cq.x - dq.x)) * rdy;
                    d[3 + f][1] = (k0 * (a.y - bb.y) + k1 * (cq.y - dq.y)) * rdy;
                }
                {
                    // Dp_y syy -> d[4]
                    const float *F = H + hb;
                    const float2 a = ld2(F, c0 + boxw), bb = ld2(F, c0), cq = ld2(F, c0 + 2 * boxw),
                                 dq = ld2(F, c0 - boxw);
                    d[4][0] = (k0 * (a.x - bb.x) + k1 * (cq.x - dq.x)) * rdy;
                    d[4][1] = (k0 * (a.y - bb.y) + k1 * (cq.y - dq.y)) * rdy;
                }
                // Dm_z sxz -> d[6], syz -> d[7]; Dp_z szz -> d[8]
#pragma unroll
                for (int f = 0; f < 2; f++) {
                    d[6 + f][0] = (k0 * (rv[f][4].x - rv[f][3].x) + k1 * (rv[f][5].x - rv[f][2].x)) * rdz;
                    d[6 + f][1] = (k0 * (rv[f][4].y - rv[f][3].y) + k1 * (rv[f][5].y - rv[f][2].y)) * rdz;
                }
                d[8][0] = (k0 * (rv[2][5].x - rv[2][4].x) + k1 * (rv[2][6].x - rv[2][3].x)) * rdz;
                d[8][1] = (k0 * (rv[2][5].y - rv[2][4].y) + k1 * (rv[2][6].y - rv[2][3].y)) * rdz;
                const float *PS = base + kFvStage;
                const int zi = z - 2, yi = y - 2, xi = x - 2;
                const float2 vp2 = ld2(C, cb + cc);
                const float vpc[2] = {vp2.x, vp2.y};
                float A[2], B[2], Ah[2], Bh[2];
                auto upd = [&](const float *sp, float *gp, const float *BB, const float *AA, float *dd) {
                    float2 v = *reinterpret_cast<const float2 *>(sp);
                    v.x = BB[0] * v.x + AA[0] * dd[0];
                    v.y = BB[1] * v.y + AA[1] * dd[1];
                    *reinterpret_cast<float2 *>(gp) = v;
                    dd[0] += v.x;
                    dd[1] += v.y;
                };
                if (xabs) {
                    const int xc = x < m ? x - 2 : m - 2 + x - (m + g.px);
                    const long long a0 = ((long long)zi * (g.ny - 4) + yi) * geo.PX + xc;
                    const long long as = (long long)(g.nz - 4) * (g.ny - 4) * geo.PX;
                    const int s0 = r * geo.PX + xc, ss = 4 * geo.PX;
#pragma unroll
                    for (int c = 0; c < 2; c++) cpml_coef(vpc[c], __ldg(&geo.ax[0][x + c]), dt, A[c], B[c], Ah[c], Bh[c]);
                    upd(PS + s0, geo.psx + a0, Bh, Ah, d[0]);
                    upd(PS + s0 + ss, geo.psx + a0 + as, B, A, d[1]);
                    upd(PS + s0 + 2 * ss, geo.psx + a0 + 2 * as, B, A, d[2]);
                }
                if (yabs) {
                    const int yc = y < m ? y - 2 : m - 2 + y - (m + g.py);
                    const long long a0 = ((long long)zi * geo.W + yc) * geo.PY + xi;
                    const long long as = (long long)(g.nz - 4) * geo.W * geo.PY;
                    const int s0 = pxr + r * geo.PB + (xi - xb0), ss = 4 * geo.PB;
                    const float4 ty = __ldg(&geo.ax[1][y]);
#pragma unroll
                    for (int c = 0; c < 2; c++) cpml_coef(vpc[c], ty, dt, A[c], B[c], Ah[c], Bh[c]);
                    upd(PS + s0, geo.psy + a0, B, A, d[3]);
                    upd(PS + s0 + ss, geo.psy + a0 + as, Bh, Ah, d[4]);
                    upd(PS + s0 + 2 * ss, geo.psy + a0 + 2 * as, B, A, d[5]);
                }
                if (zabs) {
                    const int zc = z < m ? z - 2 : m - 2 + z - (m + g.pz);
                    const long long a0 = ((long long)zc * (g.ny - 4) + yi) * geo.PY + xi;
                    const long long as = (long long)geo.W * (g.ny - 4) * geo.PY;
                    const int s0 = pxr + pyr + r * geo.PB + (xi - xb0), ss = 4 * geo.PB;
                    const float4 tz = __ldg(&geo.ax[2][z]);
#pragma unroll
                    for (int c = 0; c < 2; c++) cpml_coef(vpc[c], tz, dt, A[c], B[c], Ah[c], Bh[c]);
                    upd(PS + s0, geo.psz + a0, B, A, d[6]);
                    upd(PS + s0 + ss, geo.psz + a0 + as, B, A, d[7]);
                    upd(PS + s0 + 2 * ss, geo.psz + a0 + 2 * as, Bh, Ah, d[8]);
                }
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    Dx[c] = d[0][c] + d[3][c] + d[6][c];
                    Dy[c] = d[1][c] + d[4][c] + d[7][c];
                    Dz[c] = d[2][c] + d[5][c] + d[8][c];
                }
            }
            const float2 rh = ld2(C, cc);
            const float dtr[2] = {signed_bdt(rh.x, dt), signed_bdt(rh.y, dt)};
            const float2 v0 = ld2(C, 2 * cb + cc), v1 = ld2(C, 3 * cb + cc), v2 = ld2(C, 4 * cb + cc);
            *reinterpret_cast<float2 *>(w.f[VX] + i0) = make_float2(v0.x + dtr[0] * Dx[0], v0.y + dtr[1] * Dx[1]);
            *reinterpret_cast<float2 *>(w.f[VY] + i0) = make_float2(v1.x + dtr[0] * Dy[0], v1.y + dtr[1] * Dy[1]);
            *reinterpret_cast<float2 *>(w.f[VZ] + i0) = make_float2(v2.x + dtr[0] * Dz[0], v2.y + dtr[1] * Dz[1]);
            const bool fed = z + 5 < g.nz;
#pragma unroll
            for (int f = 0; f < 3; f++) {
#pragma unroll
                for (int q = 0; q < 8; q++) rv[f][q] = rv[f][q + 1];
                rv[f][8] = fed ? ld2(FD, f * cb + cc) : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();
        if (s_abort) {
            if (tid == 0) {
                mbar_wait_bounded(b ? bar1 : bar0, parity);
                if (k + 1 < w1) {
                    const int k1 = k + 1 - w0;
                    mbar_wait_bounded((k1 & 1) ? bar1 : bar0, (uint32_t)((k1 >> 1) & 1));
                }
            }
            __syncthreads();
            return;
        }
        if (tid == 0 && k + 2 < w1) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(k + 2, b);
        }
    }
}


// ------------------------------------------------------------ receivers

__global__ void record(WaveDev w, const long long *__restrict__ rec, int nrec, int nt,
                       const StepState *__restrict__ st, int it_off) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    const int it = st->it + it_off;
    float *tx = st->tr[0], *ty = st->tr[1], *tz = st->tr[2];
    const long long i = rec[r];
    const long long o = (long long)r * nt + it;
    if (tx) tx[o] = w.f[VX][i];
    if (ty) ty[o] = w.f[VY][i];
    if (tz) tz[o] = w.f[VZ][i];
}

__global__ void inject_rec(WaveDev w, const long long *__restrict__ rec, int nrec, int nt,
                           const StepState *__restrict__ st, int it_off) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    const int it = st->it + it_off;
    const float *tx = st->obs[0], *ty = st->obs[1], *tz = st->obs[2];
    const long long i = rec[r];
    const long long o = (long long)r * nt + it;
    atomicAdd(w.f[VX] + i, tx[o]);
    atomicAdd(w.f[VY] + i, ty[o]);
    atomicAdd(w.f[VZ] + i, tz[o]);
}

// ---------------------------------------------------------------- VOWR

// The box of block b: the last box whose first block is not after b (a
// binary search over the table in the kernel parameters, block-uniform).
__device__ __forceinline__ int vowr_box(const VowrDev &v, int b) {
    int lo = 0, hi = v.nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((int)v.seg[mid].nblk_first <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// One block per 256 (x vw) elements of one face box.  pack: field ->
// store[slot]; else the reverse.  Blocks [b0, b0 + gridDim.x) of the face
// boxes (all of them, the velocity boxes or the stress boxes).
__global__ void __launch_bounds__(256) vowr(GridDev g, const __grid_constant__ WaveDev w,
                                            const __grid_constant__ VowrDev v, const StepState *__restrict__ st,
                                            int slot_shift, int pack, int b0) {
    const int slot = st->it + slot_shift;
    if (slot < 0 || slot >= v.nslot) return;
    const int b = b0 + (int)blockIdx.x;
    const SegDev &S = v.seg[vowr_box(v, b)];
    const int e = ((b - (int)S.nblk_first) * 256 + (int)threadIdx.x) * S.vw;
    const int cnt = S.nxb * S.nyb * S.nzb;
    if (e >= cnt) return;
    const int t = e / S.nxb;
    const int x = S.x0 + (e - t * S.nxb);
    const int z = t / S.nyb;
    const int y = S.y0 + (t - z * S.nyb);
    const int i = (int)g.xoff + x + (int)g.sy * y + (int)g.sz * (S.z0 + z);
    float *rec = v.store + (long long)slot * v.per_step + S.off + e;
    if (S.vw == 4) {  // 4 values of one row; record and field both 16-byte aligned (vowr_segments)
        float4 *f4 = reinterpret_cast<float4 *>(w.f[S.fld] + i), *r4 = reinterpret_cast<float4 *>(rec);
        if (pack) *r4 = *f4;
        else *f4 = *r4;
    } else if (pack) {
        *rec = w.f[S.fld][i];
    } else {
        w.f[S.fld][i] = *rec;
    }
}

// 16-bit boundary store.  Pass 1: each box's largest magnitude in this
// step (amax[parity][box], atomic max of the float bits, non-negative);
// the other parity's row, last read by the previous step's pass 2, is
// cleared for the next step.
__global__ void __launch_bounds__(256) vowr_amax(GridDev g, const __grid_constant__ WaveDev w,
                                                 const __grid_constant__ VowrDev v,
                                                 const StepState *__restrict__ st, int slot_shift) {
    const int slot = st->it + slot_shift;
    if (slot < 0 || slot >= v.nslot) return;
    unsigned *cur = v.amax + (slot & 1) * v.nseg, *nxt = v.amax + ((slot + 1) & 1) * v.nseg;
    if (blockIdx.x == 0)
        for (int q = threadIdx.x; q < v.nseg; q += blockDim.x) nxt[q] = 0u;
    const int b = (int)blockIdx.x;
    const int sg = vowr_box(v, b);
    const SegDev &S = v.seg[sg];
    const int e = (b - (int)S.nblk_first) * 256 + (int)threadIdx.x;
    float a = 0.f;
    if (e < S.nxb * S.nyb * S.nzb) {
        const int t = e / S.nxb;
        const int x = S.x0 + (e - t * S.nxb);
        const int z = t / S.nyb;
        const int y = S.y0 + (t - z * S.nyb);
        a = fabsf(w.f[S.fld][(int)g.xoff + x + (int)g.sy * y + (int)g.sz * (S.z0 + z)]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a = fmaxf(a, __shfl_xor_sync(0xffffffffu, a, o));
    if ((threadIdx.x & 31) == 0 && a > 0.f) atomicMax(cur + sg, __float_as_uint(a));
}

// Pass 2 (pack) and the unpack of a 16-bit store: value = q * scale.
template <int PREC>
__global__ void __launch_bounds__(256) vowr16(GridDev g, const __grid_constant__ WaveDev w,
                                              const __grid_constant__ VowrDev v, const StepState *__restrict__ st,
                                              int slot_shift, int pack, int b0) {
    const int slot = st->it + slot_shift;
    if (slot < 0 || slot >= v.nslot) return;
    const int b = b0 + (int)blockIdx.x;
    const int sg = vowr_box(v, b);
    const SegDev &S = v.seg[sg];
    const int e = (b - (int)S.nblk_first) * 256 + (int)threadIdx.x;
    if (e >= S.nxb * S.nyb * S.nzb) return;
    const int t = e / S.nxb;
    const int x = S.x0 + (e - t * S.nxb);
    const int z = t / S.nyb;
    const int y = S.y0 + (t - z * S.nyb);
    const int i = (int)g.xoff + x + (int)g.sy * y + (int)g.sz * (S.z0 + z);
    uint16_t *rec = v.store16 + (long long)slot * v.per_step + S.off + e;
    float *scale = v.scales + (long long)slot * v.nseg + sg;
    if (pack) {
        const float s = __uint_as_float(v.amax[(slot & 1) * v.nseg + sg]);
        if (e == 0) *scale = s;
        const float q = s > 0.f ? w.f[S.fld][i] / s : 0.f;
        if (PREC == kStoreBF16) *rec = __bfloat16_as_ushort(__float2bfloat16_rn(q));
        else *rec = __half_as_ushort(__float2half_rn(q));
    } else {
        const float q = PREC == kStoreBF16 ? __bfloat162float(__ushort_as_bfloat16(*rec))
                                        : __half2float(__ushort_as_half(*rec));
        w.f[S.fld][i] = q * *scale;
    }
}

__global__ void step_advance(StepState *st, int delta) { st->it += delta; }

__global__ void count_nonfinite_f(const float *p, size_t n, unsigned long long *out) {
    unsigned long long c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        c += !isfinite(p[i]);
    if (c) atomicAdd(out, c);
}
// FP64 energy (sum of squares) of the nine velocity and stress fields over
// gridphy, added into *out
__global__ void wave_energy(GridDev g, WaveDev w, double *out) {
    const long long n = (long long)g.px * g.py * g.pz;
    double e = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long t = c / g.px;
        const int x = (int)(c - t * g.px), y = (int)(t % g.py), z = (int)(t / g.py);
        const long long i = g.xoff + (x + g.m) + g.sy * (y + g.m) + g.sz * (z + g.m);
#pragma unroll
        for (int f = VX; f <= SYZ; f++) {
            const double v = w.f[f][i];
            e += v * v;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0 && e != 0.0) atomicAdd(out, e);
}

__global__ void count_nonfinite_d(const double *p, size_t n, unsigned long long *out) {
    unsigned long long c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        c += !isfinite(p[i]);
    if (c) atomicAdd(out, c);
}

// ---------------------------------------------------------- model prep

// gridext model: nearest-cell extension of gridphy (the 26 regions of
// FD/fdtd3d_0_base_module/fdtd3d_base_3_geomodel_meat.hpp:101-364) and
// lambda = rho (vp^2 - 2 vs^2), mu = rho vs^2 with the reference's
// float operation order (:454-460).  Density enters the velocity update
// only as dt / rho, so that quotient is stored (bdt, for dt > 0): the
// velocity kernels take it, negated for the backward update, in place of a
// division per cell and step.  IEEE division is sign-symmetric, so
// -(dt / rho) equals (-dt) / rho bit for bit.
__global__ void model_prep(GridDev g, const float *__restrict__ vp0, const float *__restrict__ vs0,
                           const float *__restrict__ rho0, float dt, float *vp, float *bdt, float *lam, float *mu) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx) return;
    const int px = min(max(x - g.m, 0), g.px - 1);
    const int py = min(max(y - g.m, 0), g.py - 1);
    const int pz = min(max(z - g.m, 0), g.pz - 1);
    const long long s = px + (long long)g.px * (py + (long long)g.py * pz);
    const long long i = g.xoff + x + g.sy * y + g.sz * z;
    const float a = vp0[s], b = vs0[s], r = rho0[s];
    vp[i] = a;
    bdt[i] = __fdiv_rn(dt, r);
    const float b2 = __fmul_rn(b, b);
    lam[i] = __fmul_rn(r, __fsub_rn(__fmul_rn(a, a), __fmul_rn(2.0f, b2)));
    mu[i] = __fmul_rn(r, b2);
}

__global__ void zero_range(float *p, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = 0.f;
}

// ------------------------------------------------------- image epilogue

// out: 8 float arrays of gridphy: compensated pp, ps, sp, ss, then the
// Laplacians of the uncompensated images (cells 2..n-3, zero elsewhere).
__global__ void image_stack(long long n, ImageDev shot, StackDev st) {
    const float *src[5] = {shot.ip, shot.pp, shot.ps, shot.sp, shot.ss};
    double *dst[5] = {st.ip, st.pp, st.ps, st.sp, st.ss};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 5; q++) dst[q][i] += (double)src[q][i];
    }
}

__global__ void image_finalize(GridDev g, StackDev img, float *out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= g.px) return;
    const long long sy = g.px, sz = (long long)g.px * g.py, n = sz * g.pz;
    const long long o = x + sy * y + sz * z;
    const double *src[4] = {img.pp, img.ps, img.sp, img.ss};
    const double ip = img.ip[o];
    const bool in = x >= 2 && x <= g.px - 3 && y >= 2 && y <= g.py - 3 && z >= 2 && z <= g.pz - 3;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double *f = src[q];
        const double v = f[o];
        out[q * n + o] = (float)(ip > 3.4e-38 ? v / ip : v);
        double l = 0.0;
        if (in) l = f[o + 1] + f[o - 1] + f[o + sy] + f[o - sy] + f[o + sz] + f[o - sz] - 6.0 * v;
        out[(4 + q) * n + o] = (float)l;
    }
}

inline int cerr() { return (int)cudaGetLastError(); }

}  // namespace

// --------------------------------------------------------------- hosts

int upload_coefficients(const float list[5][4], const float dc2[2]) {
    cudaError_t e = cudaMemcpyToSymbol(c_list, list, sizeof(float) * 20);
    if (e != cudaSuccess) return (int)e;
    return (int)cudaMemcpyToSymbol(c_dc2, dc2, sizeof(float) * 2);
}

int k_model_prep(const GridDev &g, const float *vp0, const float *vs0, const float *rho0, float dt, float *vp,
                 float *bdt, float *lam, float *mu, void *stream) {
    dim3 b(128), gr((g.nx + 127) / 128, g.ny, g.nz);
    model_prep<<<gr, b, 0, (cudaStream_t)stream>>>(g, vp0, vs0, rho0, dt, vp, bdt, lam, mu);
    return cerr();
}

int k_zero_range(float *p, size_t n, void *stream) {
    if (n == 0) return 0;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    zero_range<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(p, n);
    return cerr();
}

// Variant-2 launch shape: blocks of gx x-groups (4 cells each) by gy rows.
// By default a block spans a whole gridphy row when it has at most 64
// groups (256 cells), else the row is split evenly, so that no thread is
// idle beyond the last partial group (200 cells = 50 groups = one block
// row of 50 x 5); gy fills the block up to 256 threads.
static void v4_shape(const GridDev &g, const KCfg &kc, dim3 *b, dim3 *gr) {
    const int ngx = (g.px + 3) / 4;
    int gx = kc.gx;
    if (gx <= 0) {
        const int nb = (ngx + 63) / 64;
        gx = (ngx + nb - 1) / nb;
    }
    gx = std::min(std::max(gx, 1), 256);
    int gy = kc.gy > 0 ? kc.gy : std::max(1, 256 / gx);
    gy = std::min(std::max(gy, 1), 256 / gx);
    const int zp = kc.zp == 2 ? 2 : 1;
    *b = dim3(gx, gy);
    *gr = dim3((ngx + gx - 1) / gx, (g.py + gy - 1) / gy, (g.pz + zp - 1) / zp);
}

template <int MINB, int ZP>
static int launch_vel_v4(int mode, dim3 gr, dim3 b, cudaStream_t s, const GridDev &g, const WaveDev &w,
                         const float *bdt, float dt, int rec_w, const WaveDev *rev, const ImageDev *img,
                         const WaveDev &rv, const ImageDev &im) {
    switch (mode) {
    case kFwd: vel_phy_v4<kFwd, false, MINB, ZP><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im); break;
    case kRtmFwd: vel_phy_v4<kRtmFwd, false, MINB, ZP><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im); break;
    case kRev: vel_phy_v4<kRev, false, MINB, ZP><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im); break;
    case kBwd:
        if (img && rev) vel_phy_v4<kBwd, true, MINB, ZP><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im);
        else vel_phy_v4<kBwd, false, MINB, ZP><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im);
        break;
    default: return (int)cudaErrorInvalidValue;
    }
    return cerr();
}

template <int MINB, int ZP>
static int launch_stress_v4(int mode, dim3 gr, dim3 b, cudaStream_t s, const GridDev &g, const WaveDev &w,
                            const float *lam, const float *mu, float dt, int rec_w, const float *wavelet,
                            const StepState *st, int it_off) {
    switch (mode) {
    case kFwd: stress_phy_v4<kFwd, MINB, ZP><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    case kRtmFwd: stress_phy_v4<kRtmFwd, MINB, ZP><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    case kBwd: stress_phy_v4<kBwd, MINB, ZP><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    case kRev: stress_phy_v4<kRev, MINB, ZP><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    default: return (int)cudaErrorInvalidValue;
    }
    return cerr();
}

int k_vel_phy(int mode, const GridDev &g, const WaveDev &w, const float *bdt, float dt, int rec_w, const WaveDev *rev,
              const ImageDev *img, const KCfg &kc, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    WaveDev rv = rev ? *rev : WaveDev{};
    ImageDev im = img ? *img : ImageDev{};
    if (kc.variant >= 2) {
        dim3 b, gr;
        v4_shape(g, kc, &b, &gr);
        if (kc.zp == 2) {
            if (kc.minb == 4) return launch_vel_v4<4, 2>(mode, gr, b, s, g, w, bdt, dt, rec_w, rev, img, rv, im);
            return launch_vel_v4<3, 2>(mode, gr, b, s, g, w, bdt, dt, rec_w, rev, img, rv, im);
        }
        if (kc.minb == 4) return launch_vel_v4<4, 1>(mode, gr, b, s, g, w, bdt, dt, rec_w, rev, img, rv, im);
        return launch_vel_v4<3, 1>(mode, gr, b, s, g, w, bdt, dt, rec_w, rev, img, rv, im);
    }
    if (kc.variant == 1) {
        const int zc = kc.zchunk > 0 ? kc.zchunk : g.pz;
        dim3 b(kTX, kTY), gr((g.px + kTX - 1) / kTX, (g.py + kTY - 1) / kTY, (g.pz + zc - 1) / zc);
        switch (mode) {
        case kFwd: vel_phy_zm<kFwd, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im, zc); break;
        case kRtmFwd: vel_phy_zm<kRtmFwd, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im, zc); break;
        case kRev: vel_phy_zm<kRev, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im, zc); break;
        case kBwd:
            if (img && rev) vel_phy_zm<kBwd, true><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im, zc);
            else vel_phy_zm<kBwd, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im, zc);
            break;
        default: return (int)cudaErrorInvalidValue;
        }
        return cerr();
    }
    dim3 b(kTX, kTY), gr((g.px + kTX - 1) / kTX, (g.py + kTY - 1) / kTY, g.pz);
    switch (mode) {
    case kFwd: vel_phy<kFwd, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im); break;
    case kRtmFwd: vel_phy<kRtmFwd, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im); break;
    case kRev: vel_phy<kRev, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im); break;
    case kBwd:
        if (img && rev) vel_phy<kBwd, true><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im);
        else vel_phy<kBwd, false><<<gr, b, 0, s>>>(g, w, bdt, dt, rec_w, rv, im);
        break;
    default: return (int)cudaErrorInvalidValue;
    }
    return cerr();
}

// dynamic shared memory of stress_zm3: two stages of three halo planes and the core tiles
static size_t zm3_smem() { return (size_t)2 * kZmStage * sizeof(float); }

int k_make_wave_maps(const GridDev &g, const WaveDev &w, const float *lam, const float *mu, int *err_flag,
                     WaveMaps *maps) {
    maps->ok = false;
    const int boxw = kZmPitch, boxh = kZmBoxH;
    // x tiles: the whole row when its pairs fit one CTA and the row with its
    // halo one box; else the fewest tiles of an even number of pairs (so
    // that every tile's box origin stays 16-byte aligned) that fit both.
    // Tiles of fewer than 12 warps measured slower than the float4 kernel
    // (320 cells: two tiles of 320 threads, 665 against 633 us), so such
    // grids leave this kernel unused.
    const int hx = (g.px + 1) / 2;
    int ntx = 1, tpp = hx;
    auto fits = [&](int n) { return n * kZmRows <= kZmMaxThreads && (2 * n + 3) / 4 * 4 + 2 * kZmHalo <= kZmPitch; };
    if (!fits(tpp)) {
        for (ntx = 2; ntx <= 16; ntx++) {
            tpp = (hx + ntx - 1) / ntx;
            tpp += tpp & 1;
            if (fits(tpp)) break;
        }
        if (ntx > 16 || tpp * kZmRows < 384) return 0;
    }
    const int pxr = (2 * tpp + 3) / 4 * 4;  // the core box width
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return 0;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    static_assert(sizeof(CUtensorMap) == sizeof(FieldMap), "descriptor size");
    // the pitched gridext array as a 3-D tensor; box (bw, bh, 1)
    auto make = [&](const float *base, int bw, int bh, FieldMap *out) -> bool {
        CUtensorMap tm;
        const cuuint64_t dims[3] = {(cuuint64_t)g.sy, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
        const cuuint64_t strides[2] = {(cuuint64_t)g.sy * sizeof(float), (cuuint64_t)g.sz * sizeof(float)};
        const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        CUresult r = encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
        std::memcpy(out->bytes, &tm, sizeof(tm));
        return true;
    };
    const int vel[3] = {VX, VY, VZ};
    for (int f = 0; f < 3; f++)
        if (!make(w.f[vel[f]], boxw, boxh, &maps->halo[f]) || !make(w.f[vel[f]], pxr, kZmRows, &maps->core[f]))
            return 0;
    const float *pts[kZmCore - 3] = {lam, mu, w.f[SXX], w.f[SYY], w.f[SZZ], w.f[SXY], w.f[SXZ], w.f[SYZ], w.f[SAU]};
    for (int f = 0; f < kZmCore - 3; f++)
        if (!make(pts[f], pxr, kZmRows, &maps->core[3 + f])) return 0;
    const size_t smem = zm3_smem();
    cudaError_t e = cudaFuncSetAttribute(stress_zm3<kFwd>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stress_zm3<kRtmFwd>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stress_zm3<kBwd>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stress_zm3<kRev>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int)e;
    maps->rows = kZmRows;
    maps->boxw = boxw;
    maps->boxh = boxh;
    maps->corew = pxr;
    maps->ntx = ntx;
    maps->tpp = tpp;
    maps->nsm = nsm;
    maps->err = err_flag;
    maps->ok = true;
    return 0;
}

long long fz_psi_floats(const GridDev &g) {
    const int W = 2 * (g.m - 2), PX = (W + 3) / 4 * 4, PY = (g.nx - 4 + 3) / 4 * 4;
    const long long ny = g.ny - 4, nz = g.nz - 4;
    return 3LL * PX * ny * nz + 3LL * PY * W * nz + 3LL * PY * ny * W;
}

int k_make_full_maps(const GridDev &g, const WaveDev &w, const float *lam, const float *mu, const float *vp,
                     const float *bdt, float4 *const ax[3], float *psi, int *err_flag, int chunks,
                     FullMaps *maps) {
    maps->ok = false;
    const int m = g.m, xoff = (int)g.xoff;
    if ((m & 1) || (g.px & 1) || !psi) return 0;
    FzGeo geo{};
    geo.hxi = g.px / 2;
    geo.ytiles = (g.ny - 4 + kZmRows - 1) / kZmRows;
    geo.nzi = g.nz - 4;
    geo.W = 2 * (m - 2);
    geo.PX = (geo.W + 3) / 4 * 4;
    geo.PY = (g.nx - 4 + 3) / 4 * 4;
    // x tiles: the fewest for which a tile fits one CTA, each tile row with
    // its x halo fits the 256-float halo box, and the core and
    // memory-variable boxes are at most 256 wide
    int threads = 0;
    for (geo.NTX = 1; geo.NTX <= 64; geo.NTX++) {
        geo.TPP = (geo.hxi + geo.NTX - 1) / geo.NTX;
        geo.hxe = geo.NTX == 1 ? m - 2 : (m - 2) / 2;
        geo.tpad = (kZmRows * geo.TPP + 31) / 32 * 32;
        // the physical pairs end on a warp boundary unless that alone takes
        // the tile past one CTA; then one warp carries both updates (the
        // kernels have no warp-level collectives) rather than a tile more
        if (geo.tpad + kZmRows * geo.hxe > kZmMaxThreads) geo.tpad = kZmRows * geo.TPP;
        threads = geo.tpad + kZmRows * geo.hxe;
        bool fits = threads <= kZmMaxThreads && (geo.NTX - 1) * geo.TPP < geo.hxi;
        geo.corew = 0;
        geo.PB = 0;
        for (int t = 0; t < geo.NTX && fits; t++) {
            const int xlo = fz_xlo(g, geo, t), xhi = fz_xhi(g, geo, t);
            const int XC = (xoff + xlo) & ~3, XH = XC - kZmHalo, xb0 = (xlo - 2) & ~3;
            geo.corew = std::max(geo.corew, (xoff + xhi - XC + 3) / 4 * 4);
            geo.PB = std::max(geo.PB, (xhi - 2 - xb0 + 3) / 4 * 4);
            fits = xoff + xhi + 4 - XH <= kZmPitch;
        }
        if (fits && geo.corew <= kZmPitch && geo.PB <= kZmPitch) break;
        if (geo.TPP <= 16) return 0;
    }
    if (geo.NTX > 64) return 0;
    int dev = 0, nsm = 0, smem_max = 0;
    cudaGetDevice(&dev);
    cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return (int)e;
    const size_t smem = (size_t)2 * fz_stage(geo) * sizeof(float);
    if (smem + 1024 > (size_t)smem_max) return 0;
    const size_t vsmem = (size_t)2 * fv_stage(geo) * sizeof(float);
    if (vsmem + 1024 > (size_t)smem_max) return 0;
    // runs: the chunking with the shortest longest-CTA time (a run's first
    // plane costs about a window refill more); the three cheapest are kept
    // as the candidates of the measured choice
    long long qc[3] = {-1, -1, -1};
    int qn[3] = {0, 0, 0};
    for (int Q = 1; Q <= 64 && Q <= geo.nzi; Q++) {
        const int L = (geo.nzi + Q - 1) / Q, R = geo.NTX * geo.ytiles * Q;
        const int G = std::min(nsm, R);
        const long long cost = (long long)((R + G - 1) / G) * (L + 6);
        for (int k = 0; k < 3; k++) {
            if (qc[k] < 0 || cost < qc[k]) {
                for (int j = 2; j > k; j--) {
                    qc[j] = qc[j - 1];
                    qn[j] = qn[j - 1];
                }
                qc[k] = cost;
                qn[k] = Q;
                break;
            }
        }
    }
    const int Q = chunks >= 1 && chunks <= geo.nzi ? chunks : qn[0];
    geo.Q = Q;
    geo.L = (geo.nzi + Q - 1) / Q;
    geo.R = geo.NTX * geo.ytiles * Q;
    for (int a = 0; a < 3; a++) geo.ax[a] = ax[a];
    FzGeo vgeo = geo;
    // memory variables: the velocity set, then the stress set
    vgeo.psx = psi;
    vgeo.psy = vgeo.psx + 3LL * geo.PX * (g.ny - 4) * (g.nz - 4);
    vgeo.psz = vgeo.psy + 3LL * geo.PY * geo.W * (g.nz - 4);
    geo.psx = psi + fz_psi_floats(g);
    geo.psy = geo.psx + (vgeo.psy - vgeo.psx);
    geo.psz = geo.psx + (vgeo.psz - vgeo.psx);
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return 0;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    // a tensor of rank 3 or 4 over float32, packed except for its strides
    auto make = [&](const float *base, int rank, const cuuint64_t *dims, const cuuint32_t *box, FieldMap *out) {
        CUtensorMap tm;
        cuuint64_t strides[3];
        cuuint64_t acc = dims[0];
        for (int d = 1; d < rank; d++) {
            strides[d - 1] = acc * sizeof(float);
            acc *= dims[d];
        }
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        CUresult r = encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, (void *)base, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
        std::memcpy(out->bytes, &tm, sizeof(tm));
        return true;
    };
    // the pitched gridext arrays as 3-D tensors (sy, ny, nz)
    const cuuint64_t fd[3] = {(cuuint64_t)g.sy, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
    const cuuint32_t hbox[3] = {(cuuint32_t)kZmPitch, (cuuint32_t)kZmBoxH, 1};
    const cuuint32_t cbox[3] = {(cuuint32_t)geo.corew, (cuuint32_t)kZmRows, 1};
    const int vel[3] = {VX, VY, VZ};
    for (int f = 0; f < 3; f++)
        if (!make(w.f[vel[f]], 3, fd, hbox, &maps->halo[f]) || !make(w.f[vel[f]], 3, fd, cbox, &maps->core[f]))
            return 0;
    const float *pts[kFzCore - 3] = {lam, mu, vp, w.f[SXX], w.f[SYY], w.f[SZZ], w.f[SXY], w.f[SXZ], w.f[SYZ],
                                     w.f[SAU]};
    for (int f = 0; f < kFzCore - 3; f++)
        if (!make(pts[f], 3, fd, cbox, &maps->core[3 + f])) return 0;
    // the memory variables: 4-D (row, rows, planes, 3 arrays), boxes of 4 rows of one plane
    const cuuint64_t ny = (cuuint64_t)(g.ny - 4), nz = (cuuint64_t)(g.nz - 4), W = (cuuint64_t)geo.W;
    const cuuint64_t dx4[4] = {(cuuint64_t)geo.PX, ny, nz, 3}, dy4[4] = {(cuuint64_t)geo.PY, W, nz, 3},
                     dz4[4] = {(cuuint64_t)geo.PY, ny, W, 3};
    const cuuint32_t bx4[4] = {(cuuint32_t)geo.PX, (cuuint32_t)kZmRows, 1, 3},
                     by4[4] = {(cuuint32_t)geo.PB, (cuuint32_t)kZmRows, 1, 3};
    if (!make(geo.psx, 4, dx4, bx4, &maps->psi[0]) || !make(geo.psy, 4, dy4, by4, &maps->psi[1]) ||
        !make(geo.psz, 4, dz4, by4, &maps->psi[2]))
        return 0;
    if (!make(vgeo.psx, 4, dx4, bx4, &maps->vpsi[0]) || !make(vgeo.psy, 4, dy4, by4, &maps->vpsi[1]) ||
        !make(vgeo.psz, 4, dz4, by4, &maps->vpsi[2]))
        return 0;
    // the velocity kernel's field boxes
    const cuuint32_t bbox[3] = {(cuuint32_t)kZmPitch, (cuuint32_t)kZmRows, 1};
    const int vh[3] = {SXY, SYY, SYZ}, vb[2] = {SXX, SXZ}, vf[3] = {SXZ, SYZ, SZZ};
    const float *vc[5] = {bdt, vp, w.f[VX], w.f[VY], w.f[VZ]};
    for (int f = 0; f < 3; f++)
        if (!make(w.f[vh[f]], 3, fd, hbox, &maps->vhalo[f]) || !make(w.f[vf[f]], 3, fd, cbox, &maps->vfeed[f]))
            return 0;
    for (int f = 0; f < 2; f++)
        if (!make(w.f[vb[f]], 3, fd, bbox, &maps->vband[f])) return 0;
    for (int f = 0; f < 5; f++)
        if (!make(vc[f], 3, fd, cbox, &maps->vcore[f])) return 0;
    // The attribute belongs to the kernel, not to this context: contexts of
    // other grids launch the same kernel with other stage sizes, possibly
    // at the same time.  Every caller sets the same value, the device's
    // limit, and each launch asks for its own size below it.
    const int smem_attr = smem_max - 1024;
    const void *fns[8] = {(const void *)vel_fz<false>,          (const void *)vel_fz<true>,
                          (const void *)stress_fz<kFwd, false>,    (const void *)stress_fz<kFwd, true>,
                          (const void *)stress_fz<kRtmFwd, false>, (const void *)stress_fz<kRtmFwd, true>,
                          (const void *)stress_fz<kRev, false>,    (const void *)stress_fz<kRev, true>};
    e = cudaSuccess;
    for (int f = 0; f < 8 && e == cudaSuccess; f++)
        e = cudaFuncSetAttribute(fns[f], cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr);
    if (e != cudaSuccess) return (int)e;
    maps->geo = geo;
    maps->vgeo = vgeo;
    maps->threads = threads;
    maps->grid = std::min(nsm, geo.R);
    maps->smem = smem;
    maps->vsmem = vsmem;
    maps->err = err_flag;
    for (int k = 0; k < 3; k++) maps->qcand[k] = qn[k];
    maps->ok = true;
    return 0;
}

int k_vel_full(const GridDev &g, const WaveDev &w, float dt, const FullMaps &maps, void *stream) {
    if (!maps.ok) return (int)cudaErrorInvalidValue;
    FvMaps fm;
    static_assert(sizeof(FvMaps) == sizeof(maps.vhalo) + sizeof(maps.vband) + sizeof(maps.vcore) +
                                        sizeof(maps.vfeed) + sizeof(maps.vpsi),
                  "descriptor layout");
    std::memcpy(fm.halo, maps.vhalo, sizeof(maps.vhalo));
    std::memcpy(fm.band, maps.vband, sizeof(maps.vband));
    std::memcpy(fm.core, maps.vcore, sizeof(maps.vcore));
    std::memcpy(fm.feed, maps.vfeed, sizeof(maps.vfeed));
    std::memcpy(fm.psi, maps.vpsi, sizeof(maps.vpsi));
    if (maps.geo.NTX > 1) vel_fz<true><<<maps.grid, maps.threads, maps.vsmem, (cudaStream_t)stream>>>(g, fm, w, dt, maps.vgeo, maps.err);
    else vel_fz<false><<<maps.grid, maps.threads, maps.vsmem, (cudaStream_t)stream>>>(g, fm, w, dt, maps.vgeo, maps.err);
    return cerr();
}

int k_stress_full(int mode, const GridDev &g, const WaveDev &w, float dt, const float *wavelet, const StepState *st,
                  int it_off, const FullMaps &maps, void *stream) {
    if (!maps.ok) return (int)cudaErrorInvalidValue;
    FzMaps fm;
    static_assert(sizeof(FzMaps) == sizeof(maps.halo) + sizeof(maps.core) + sizeof(maps.psi), "descriptor layout");
    std::memcpy(fm.halo, maps.halo, sizeof(maps.halo));
    std::memcpy(fm.core, maps.core, sizeof(maps.core));
    std::memcpy(fm.psi, maps.psi, sizeof(maps.psi));
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid(maps.grid), block(maps.threads);
    const bool xt = maps.geo.NTX > 1;
#define JV_FZ(M)                                                                                                 \
    if (xt) stress_fz<M, true><<<grid, block, maps.smem, s>>>(g, fm, w, dt, wavelet, st, it_off, maps.geo, maps.err); \
    else stress_fz<M, false><<<grid, block, maps.smem, s>>>(g, fm, w, dt, wavelet, st, it_off, maps.geo, maps.err)
    switch (mode) {
    case kFwd: JV_FZ(kFwd); break;
    case kRtmFwd: JV_FZ(kRtmFwd); break;
    case kRev: JV_FZ(kRev); break;
    default: return (int)cudaErrorInvalidValue;
    }
#undef JV_FZ
    return cerr();
}

int k_stress_phy(int mode, const GridDev &g, const WaveDev &w, const float *lam, const float *mu, float dt, int rec_w,
                 const float *wavelet, const StepState *st, int it_off, const KCfg &kc, void *stream,
                 const WaveMaps *maps) {
    cudaStream_t s = (cudaStream_t)stream;
    if ((kc.variant == 3 || kc.variant == 4) && maps && maps->ok) {
        ZmMaps zm;
        static_assert(sizeof(ZmMaps) == sizeof(maps->halo) + sizeof(maps->core), "descriptor layout");
        std::memcpy(zm.halo, maps->halo, sizeof(maps->halo));
        std::memcpy(zm.core, maps->core, sizeof(maps->core));
        const int ytiles = (g.py + maps->rows - 1) / maps->rows;
        const long long items = (long long)ytiles * maps->ntx * g.pz;
        const int grid = (int)std::min<long long>(maps->nsm, items);
        const dim3 b(maps->tpp * maps->rows);
        const size_t smem = zm3_smem();
        switch (mode) {
#define JV_ZM3(M)                                                                                              \
    stress_zm3<M><<<grid, b, smem, s>>>(g, zm, w, dt, rec_w, wavelet, st, it_off, maps->corew, ytiles, maps->ntx, \
                                        maps->tpp, maps->err)
        case kFwd: JV_ZM3(kFwd); break;
        case kRtmFwd: JV_ZM3(kRtmFwd); break;
        case kBwd: JV_ZM3(kBwd); break;
        case kRev: JV_ZM3(kRev); break;
#undef JV_ZM3
        default: return (int)cudaErrorInvalidValue;
        }
        return cerr();
    }
    if (kc.variant >= 2) {
        dim3 b, gr;
        v4_shape(g, kc, &b, &gr);
        if (kc.zp == 2) {
            if (kc.minb == 4)
                return launch_stress_v4<4, 2>(mode, gr, b, s, g, w, lam, mu, dt, rec_w, wavelet, st, it_off);
            return launch_stress_v4<3, 2>(mode, gr, b, s, g, w, lam, mu, dt, rec_w, wavelet, st, it_off);
        }
        if (kc.minb == 4)
            return launch_stress_v4<4, 1>(mode, gr, b, s, g, w, lam, mu, dt, rec_w, wavelet, st, it_off);
        return launch_stress_v4<3, 1>(mode, gr, b, s, g, w, lam, mu, dt, rec_w, wavelet, st, it_off);
    }
    if (kc.variant == 1) {
        const int zc = kc.zchunk > 0 ? kc.zchunk : g.pz;
        dim3 b(kTX, kTY), gr((g.px + kTX - 1) / kTX, (g.py + kTY - 1) / kTY, (g.pz + zc - 1) / zc);
        switch (mode) {
        case kFwd: stress_phy_zm<kFwd><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, zc, it_off); break;
        case kRtmFwd: stress_phy_zm<kRtmFwd><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, zc, it_off); break;
        case kBwd: stress_phy_zm<kBwd><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, zc, it_off); break;
        case kRev: stress_phy_zm<kRev><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, zc, it_off); break;
        default: return (int)cudaErrorInvalidValue;
        }
        return cerr();
    }
    dim3 b(kTX, kTY), gr((g.px + kTX - 1) / kTX, (g.py + kTY - 1) / kTY, g.pz);
    switch (mode) {
    case kFwd: stress_phy<kFwd><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    case kRtmFwd: stress_phy<kRtmFwd><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    case kBwd: stress_phy<kBwd><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    case kRev: stress_phy<kRev><<<gr, b, 0, s>>>(g, w, lam, mu, dt, rec_w, wavelet, st, it_off); break;
    default: return (int)cudaErrorInvalidValue;
    }
    return cerr();
}

int k_vel_pml(const GridDev &g, const CpmlDev &c, const WaveDev &w, const float *bdt, const float *vp,
              const KCfg &kc, void *stream) {
    if (c.nblocks <= 0) return 0;
    const unsigned blocks = (unsigned)c.nblocks;
    cudaStream_t s = (cudaStream_t)stream;
    if (c.zp == 2) {
        if (kc.pml_minb == 4) vel_pml<4, 2><<<blocks, 256, 0, s>>>(g, c, w, bdt, vp);
        else vel_pml<3, 2><<<blocks, 256, 0, s>>>(g, c, w, bdt, vp);
    } else {
        if (kc.pml_minb == 4) vel_pml<4, 1><<<blocks, 256, 0, s>>>(g, c, w, bdt, vp);
        else vel_pml<3, 1><<<blocks, 256, 0, s>>>(g, c, w, bdt, vp);
    }
    return cerr();
}

int k_stress_pml(const GridDev &g, const CpmlDev &c, const WaveDev &w, const float *lam, const float *mu,
                 const float *vp, int with_sau, const KCfg &kc, void *stream) {
    if (c.nblocks <= 0) return 0;
    const unsigned blocks = (unsigned)c.nblocks;
    cudaStream_t s = (cudaStream_t)stream;
    const bool m4 = kc.pml_minb == 4;
    if (c.zp == 2) {
        if (with_sau) {
            if (m4) stress_pml<true, 4, 2><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
            else stress_pml<true, 3, 2><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
        } else {
            if (m4) stress_pml<false, 4, 2><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
            else stress_pml<false, 3, 2><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
        }
    } else {
        if (with_sau) {
            if (m4) stress_pml<true, 4, 1><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
            else stress_pml<true, 3, 1><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
        } else {
            if (m4) stress_pml<false, 4, 1><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
            else stress_pml<false, 3, 1><<<blocks, 256, 0, s>>>(g, c, w, lam, mu, vp);
        }
    }
    return cerr();
}

int k_record(const WaveDev &w, const long long *rec, int nrec, int nt, const StepState *st, int it_off,
             void *stream) {
    if (nrec <= 0) return 0;
    record<<<(nrec + 127) / 128, 128, 0, (cudaStream_t)stream>>>(w, rec, nrec, nt, st, it_off);
    return cerr();
}

int k_inject_rec(const WaveDev &w, const long long *rec, int nrec, int nt, const StepState *st, int it_off,
                 void *stream) {
    if (nrec <= 0) return 0;
    inject_rec<<<(nrec + 127) / 128, 128, 0, (cudaStream_t)stream>>>(w, rec, nrec, nt, st, it_off);
    return cerr();
}

int k_vowr(const GridDev &g, const WaveDev &w, const VowrDev &v, const StepState *st, int slot_shift, int pack,
           int which, void *stream) {
    const int b0 = which == 2 ? v.vel_blocks : 0;
    const int b1 = which == 1 ? v.vel_blocks : v.all_blocks;
    if (b1 <= b0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (v.prec == kStoreF32) {
        vowr<<<(unsigned)(b1 - b0), 256, 0, s>>>(g, w, v, st, slot_shift, pack, b0);
        return cerr();
    }
    if (pack) {
        if (b0 != 0 || b1 != v.all_blocks) return (int)cudaErrorInvalidValue;  // a step's boxes pack together
        vowr_amax<<<(unsigned)v.all_blocks, 256, 0, s>>>(g, w, v, st, slot_shift);
    }
    if (v.prec == kStoreBF16) vowr16<kStoreBF16><<<(unsigned)(b1 - b0), 256, 0, s>>>(g, w, v, st, slot_shift, pack, b0);
    else vowr16<kStoreFP16><<<(unsigned)(b1 - b0), 256, 0, s>>>(g, w, v, st, slot_shift, pack, b0);
    return cerr();
}

int k_step_advance(StepState *st, int delta, void *stream) {
    step_advance<<<1, 1, 0, (cudaStream_t)stream>>>(st, delta);
    return cerr();
}

int k_wave_energy(const GridDev &g, const WaveDev &w, double *out, void *stream) {
    wave_energy<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(g, w, out);
    return cerr();
}

int k_count_nonfinite(const void *p, size_t n, int is_double, unsigned long long *out, void *stream) {
    if (n == 0) return 0;
    if (is_double) count_nonfinite_d<<<148 * 4, 256, 0, (cudaStream_t)stream>>>((const double *)p, n, out);
    else count_nonfinite_f<<<148 * 4, 256, 0, (cudaStream_t)stream>>>((const float *)p, n, out);
    return cerr();
}

int k_image_stack(const GridDev &g, const ImageDev &shot, const StackDev &stack, void *stream) {
    const long long n = (long long)g.px * g.py * g.pz;
    image_stack<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(n, shot, stack);
    return cerr();
}

int k_image_finalize(const GridDev &g, const StackDev &img, float *out, void *stream) {
    dim3 b(128), gr((g.px + 127) / 128, g.py, g.pz);
    image_finalize<<<gr, b, 0, (cudaStream_t)stream>>>(g, img, out);
    return cerr();
}

}  // namespace jv
