// TEST INFRASTRUCTURE ONLY: stands in for GPU-CUPIM's random.cuh (perl-gpu/src/lib/random/
// random.cuh) when GPU-CUPIM's one-shot step is built by oracle/build_cupim.sh.  The original
// fills the step's uniforms with cuRANDDx Philox4 (mathdx, not vendored with the reference and
// not installed here); this generator instead copies the uniforms the oracle draws for the same
// (replica, location, step) from a device buffer the harness fills, so the reference's kernels
// and the oracle consume one stream.  Same two kernels, same signatures and launch shapes.
#ifndef PERL_RANDOM_CUH
#define PERL_RANDOM_CUH

#include <cuda_runtime.h>
#include <stdint.h>

// The uniforms of the coming step, replica-major ([replica][location], n floats padded to a
// multiple of 4); set by cupim_harness.cu before every step.
__device__ float4 *g_pin_uniforms;

// Fills buf_d[k] (k < ceil(n / 4)) from the harness's buffer; seed and offset are unused.
__global__ void generate_random_numbers(const uint32_t n, const uint64_t *seed, const uint64_t *offset,
                                        float4 *buf_d) {
    (void)seed;
    (void)offset;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (4u * k < n) buf_d[k] = g_pin_uniforms[k];
}

// Advances the step offset as the original does (the copy above ignores it).
__global__ void advance_rng(uint64_t *offset, const uint64_t stride) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *offset += stride;
}

#endif  // PERL_RANDOM_CUH
