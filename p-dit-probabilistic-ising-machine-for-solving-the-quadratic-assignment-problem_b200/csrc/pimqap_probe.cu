// pimqap_probe.cu - shared-memory bandwidth probe.
//
// The resident sweep kernel is bounded by shared-memory read-modify-write bandwidth (the
// force update streams the CTA's rows of I through shared memory).  This kernel measures
// that ceiling on the current GPU with the same access pattern: 128-bit loads and stores of
// a shared buffer, two resident CTAs per SM, timed with CUDA events.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "pimqap.h"
#include "pimqap_weights.cuh"

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeBytes = 96 * 1024;   // per CTA; two CTAs fit one SM

__global__ void __launch_bounds__(kProbeThreads) smem_rmw_probe(int iters, int4 *sink) {
    extern __shared__ int4 buf[];
    const int nvec = kProbeBytes / 16;
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) buf[v] = make_int4(v, 1, 2, 3);
    __syncthreads();
    int4 acc = make_int4(0, 0, 0, 0);
    for (int it = 0; it < iters; ++it) {
        for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
            int4 x = buf[v];
            x.x += it; x.y += 3; x.z ^= it; x.w += x.x;
            buf[v] = x;
        }
    }
    __syncthreads();
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        acc.x += buf[v].x; acc.y += buf[v].y; acc.z += buf[v].z; acc.w += buf[v].w;
    }
    if (acc.x == 0x7fffffff) sink[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void weight_exp2_kernel(const float *x, float *y, long long count) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) y[k] = pimqap::exp2f_neg(x[k]);
}

}  // namespace

extern "C" pimqap_status pimqap_probe_weight_exp2(int32_t device, const float *x, float *y, int64_t count) {
    if (!x || !y || count < 0) return PIMQAP_ERR_ARG;
    if (count == 0) return PIMQAP_OK;
    if (cudaSetDevice(device) != cudaSuccess) return PIMQAP_ERR_CUDA;
    float *dx = nullptr, *dy = nullptr;
    const size_t bytes = (size_t)count * sizeof(float);
    if (cudaMalloc(&dx, bytes) != cudaSuccess) return PIMQAP_ERR_CUDA;
    if (cudaMalloc(&dy, bytes) != cudaSuccess) {
        cudaFree(dx);
        return PIMQAP_ERR_CUDA;
    }
    cudaError_t err = cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) {
        const long long blocks = (count + 255) / 256;
        weight_exp2_kernel<<<(unsigned)blocks, 256>>>(dx, dy, (long long)count);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpy(y, dy, bytes, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    return err == cudaSuccess ? PIMQAP_OK : PIMQAP_ERR_CUDA;
}

extern "C" pimqap_status pimqap_probe_smem_bandwidth(int32_t device, double *gbs) {
    if (!gbs) return PIMQAP_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return PIMQAP_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return PIMQAP_ERR_CUDA;
    if (cudaFuncSetAttribute(smem_rmw_probe, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kProbeBytes) != cudaSuccess)
        return PIMQAP_ERR_CUDA;
    const int blocks = 2 * sms, iters = 400;
    int4 *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(int4) * blocks * kProbeThreads) != cudaSuccess) return PIMQAP_ERR_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    smem_rmw_probe<<<blocks, kProbeThreads, kProbeBytes>>>(10, sink);   // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        smem_rmw_probe<<<blocks, kProbeThreads, kProbeBytes>>>(iters, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return PIMQAP_ERR_CUDA;
    const double bytes = 2.0 * (double)kProbeBytes * iters * blocks;   // read + write
    *gbs = bytes / (best * 1e-3) / 1e9;
    return PIMQAP_OK;
}
