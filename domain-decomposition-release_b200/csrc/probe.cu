// probe.cu -- attainable HBM bandwidth of a pointwise pass over many arrays.
//
// A stencil kernel of this library reads and writes many arrays per cell
// (the backward velocity update with imaging: 25 read, 11 written).  A
// plain copy streams two.  This diagnostic measures what a kernel with a
// given number of read and written arrays can move at best: one launch over
// n floats per array, one float4 of every array per thread (all loads
// independent and issued before any store), no stencil, no reuse.  Its rate
// bounds what a stencil kernel over the same arrays can reach, which a copy
// does not say.  No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "jv/jv.h"
#include "engine.hpp"

namespace {

constexpr int kProbeMaxArrays = 40;

struct ProbeArrays {
    float4 *p[kProbeMaxArrays];
};

// out_j = (j + 1) * sum of the read arrays: every load is needed, the
// stores are distinct
template <int NR, int NW>
__global__ void __launch_bounds__(256) stream_pass(const __grid_constant__ ProbeArrays a, long long n4) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n4) return;
    float4 v[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) v[r] = a.p[r][i];
    float4 s = v[0];
#pragma unroll
    for (int r = 1; r < NR; r++) {
        s.x += v[r].x;
        s.y += v[r].y;
        s.z += v[r].z;
        s.w += v[r].w;
    }
#pragma unroll
    for (int j = 0; j < NW; j++) {
        const float f = (float)(j + 1);
        a.p[NR + j][i] = make_float4(f * s.x, f * s.y, f * s.z, f * s.w);
    }
}

__global__ void probe_fill(float *p, long long n, float seed) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = seed + 1e-7f * (float)(i & 1023);
}

using Launch = void (*)(const ProbeArrays &, long long, int, cudaStream_t);
template <int NR, int NW>
void launch(const ProbeArrays &a, long long n4, int blocks, cudaStream_t s) {
    stream_pass<NR, NW><<<blocks, 256, 0, s>>>(a, n4);
}

// the footprints of this library's kernels (reads, writes per cell) and a copy
struct Shape {
    int nr, nw;
    Launch fn;
};
const Shape kShapes[] = {
    {1, 1, launch<1, 1>},     // copy
    {2, 1, launch<2, 1>},     // triad
    {10, 3, launch<10, 3>},   // velocity update, no P-wave velocities
    {12, 7, launch<12, 7>},   // stress update with sau
    {14, 6, launch<14, 6>},   // velocity update with P-wave velocities
    {25, 11, launch<25, 11>}, // backward velocity update with imaging
};

jv_status fail(jv_status c, const std::string &m) {
    jv::set_last_error(m);
    return c;
}

}  // namespace

extern "C" jv_status jv_stream_probe(int device, int n_read, int n_write, size_t n, int reps, double *gbs) {
    if (!gbs || reps < 1 || n < 4 || n % 4 || n > (1ull << 36)) return fail(JV_EINVAL, "jv_stream_probe: bad argument");
    const Shape *sh = nullptr;
    for (const Shape &s : kShapes)
        if (s.nr == n_read && s.nw == n_write) sh = &s;
    if (!sh)
        return fail(JV_EINVAL, "jv_stream_probe: (reads, writes) must be one of (1,1) (2,1) (10,3) (12,7) (14,6) (25,11)");
    if (cudaSetDevice(device) != cudaSuccess) return fail(JV_ECUDA, "jv_stream_probe: no such device");
    const int na = n_read + n_write;
    std::vector<float *> bufs(na, nullptr);
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<float> ms;
    cudaError_t err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    for (int q = 0; q < na && err == cudaSuccess; q++) err = cudaMalloc(&bufs[q], n * sizeof(float));
    if (err == cudaSuccess) {
        ProbeArrays a{};
        for (int q = 0; q < na; q++) {
            a.p[q] = reinterpret_cast<float4 *>(bufs[q]);
            probe_fill<<<1184, 256, 0, s>>>(bufs[q], (long long)n, 1.0f + q);
        }
        const long long n4 = (long long)(n / 4);
        const int blocks = (int)((n4 + 255) / 256);
        sh->fn(a, n4, blocks, s);  // warm-up
        for (int r = 0; r < reps && err == cudaSuccess; r++) {
            cudaEventRecord(e0, s);
            sh->fn(a, n4, blocks, s);
            cudaEventRecord(e1, s);
            err = cudaEventSynchronize(e1);
            float t = 0.f;
            if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
            ms.push_back(t);
        }
        if (err == cudaSuccess) err = cudaGetLastError();
    }
    if (s) cudaStreamSynchronize(s);
    for (float *b : bufs)
        if (b) cudaFree(b);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (err != cudaSuccess) return fail(err == cudaErrorMemoryAllocation ? JV_ENOMEM : JV_ECUDA, cudaGetErrorString(err));
    std::sort(ms.begin(), ms.end());
    const double t = ms[ms.size() / 2] * 1e-3;
    *gbs = (double)na * (double)n * sizeof(float) / t / 1e9;
    return JV_OK;
}
