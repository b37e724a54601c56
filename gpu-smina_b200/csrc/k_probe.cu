// Gather-bandwidth probe: the roofline the search kernel's gathers are
// measured against.  The search reads 32 B packed grid cells and 16 B pair
// table entries at data-dependent addresses from a working set (the maps of
// the ligand types and the table) that stays in L2, so its bound is the
// rate at which the memory system serves such gathers, not the HBM copy
// rate.  This kernel issues independent random gathers of the same size and
// alignment over a buffer of the same size, with every SM full, and reports
// the bytes served per second.
#include "engine.h"

namespace sg {

// 64-bit mix (SplitMix64 finaliser, Steele, Lea and Flood 2014)
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// units: buffer size in `vec`-float4 units (vec = 1: 16 B gathers, 2: 32 B);
// every thread makes `rounds` x 4 independent gathers
template <int VEC>
__global__ void __launch_bounds__(256) k_gather_probe(const float4* __restrict__ buf, unsigned long long units,
                                                      int rounds, unsigned long long salt, float* sink) {
    const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    float acc = 0.f;
    for (int r = 0; r < rounds; r++) {
        unsigned long long idx[4];
#pragma unroll
        for (int k = 0; k < 4; k++) idx[k] = mix64(salt ^ (tid * 4 + k) ^ ((unsigned long long)r << 40)) % units;
        float4 v[4][VEC];
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int j = 0; j < VEC; j++) v[k][j] = __ldg(buf + idx[k] * VEC + j);
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int j = 0; j < VEC; j++) acc += v[k][j].x + v[k][j].w;
    }
    if (acc == -1.2345678f) sink[0] = acc;  // keeps the loads; never true for the zero-filled buffer
}

cudaError_t gather_probe(size_t working_set, int bytes_per_lookup, int num_sms, double* gbs, cudaStream_t s) {
    const int vec = bytes_per_lookup / 16;
    const unsigned long long units = working_set / (16ull * vec);
    float4* buf = nullptr;
    float* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t rc = cudaMallocAsync((void**)&buf, units * 16ull * vec, s);
    if (rc == cudaSuccess) rc = cudaMallocAsync((void**)&sink, sizeof(float), s);
    if (rc == cudaSuccess) rc = cudaMemsetAsync(buf, 0, units * 16ull * vec, s);
    if (rc == cudaSuccess) rc = cudaEventCreate(&a);
    if (rc == cudaSuccess) rc = cudaEventCreate(&b);
    const int blocks = num_sms * 8, threads = 256, rounds = 64;
    float best_ms = 0;
    for (int rep = 0; rep < 4 && rc == cudaSuccess; rep++) {  // the first pass brings the buffer into L2
        cudaEventRecord(a, s);
        if (vec == 1) k_gather_probe<1><<<blocks, threads, 0, s>>>(buf, units, rounds, 0x9e3779b97f4a7c15ull * (rep + 1), sink);
        else k_gather_probe<2><<<blocks, threads, 0, s>>>(buf, units, rounds, 0x9e3779b97f4a7c15ull * (rep + 1), sink);
        cudaEventRecord(b, s);
        rc = cudaEventSynchronize(b);
        float ms = 0;
        if (rc == cudaSuccess) rc = cudaEventElapsedTime(&ms, a, b);
        if (rc == cudaSuccess && rep > 0 && (best_ms == 0 || ms < best_ms)) best_ms = ms;
    }
    if (rc == cudaSuccess) rc = cudaGetLastError();
    const double bytes = (double)blocks * threads * rounds * 4 * 16.0 * vec;
    *gbs = (rc == cudaSuccess && best_ms > 0) ? bytes / (best_ms * 1e-3) / 1e9 : 0.0;
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (buf) cudaFreeAsync(buf, s);
    if (sink) cudaFreeAsync(sink, s);
    return rc;
}

}  // namespace sg
