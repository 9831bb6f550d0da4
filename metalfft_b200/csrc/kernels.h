// kernels.h -- internal registry of libmfft's kernels (host side).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mfft {

// adjoint = 0: the transform itself (forward unscaled, inverse scaled by 1/N);
// adjoint = 1: its adjoint (conjugate transpose) -- the inverse kernel unscaled
// (adjoint of the forward) or the forward kernel scaled by 1/N (adjoint of
// the inverse), the scaling fused into the store.
typedef cudaError_t (*batched_launch_fn)(const float2* in, float2* out, long long batch,
                                         const float2* tw, int* dev_err, cudaStream_t s, int adjoint);

// One instantiation of the batched in-shared-memory FFT.
struct BatchedKernel {
    int n;         // line length
    int e;         // elements per thread (= main radix)
    int fpb;       // lines per CTA
    int stages;    // 0: direct loads; >0: persistent, TMA bulk prefetch of `stages` groups
    int threads;   // threads per CTA
    int smem;      // dynamic shared memory per CTA (bytes)
    int tw_size;   // twiddle rows (float2) for this (n, e)
    batched_launch_fn fwd;
    batched_launch_fn inv;
    cudaError_t (*prepare)();  // opt in to > 48 KB dynamic shared memory
    void (*gen_twiddles)(float2* tw, cudaStream_t s);
};

const BatchedKernel* batched_kernels(int* count);
const BatchedKernel* find_batched(int n, int e, int fpb, int stages);
const BatchedKernel* default_batched(int n);

}  // namespace mfft
