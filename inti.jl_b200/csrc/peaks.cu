// Throughput probes for the roofline denominators of the pair kernels: FP64
// FMA, FP32 FMA and the MUFU reciprocal square root, each as many independent
// dependency chains per thread over a grid that fills every SM.  Timed with
// CUDA events on the context's stream at the clock the device runs at, so the
// peak and the kernel it normalises see the same conditions.
#include <cuda_runtime.h>

#include "common.h"

namespace inti {

constexpr int kChains = 8;

template <class T>
__global__ void fma_probe(int iters, T a, T b, T* out) {
  T v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = T(threadIdx.x + c) * T(1e-3);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = fma(v[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == T(12345.678)) out[0] = s;  // keeps the chains alive
}

__global__ void mufu_probe(int iters, float* out) {
  float v[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) v[c] = 1.5f + threadIdx.x * 1e-3f + c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = rsqrtf(v[c]);
  }
  float s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += v[c];
  if (s == 12345.678f) out[0] = s;
}

template <class F>
static double time_ms(inti_ctx* ctx, F&& launch) {
  cudaEvent_t e0, e1;
  INTI_CUDA(cudaEventCreate(&e0));
  INTI_CUDA(cudaEventCreate(&e1));
  launch();  // warm-up
  INTI_CUDA(cudaEventRecord(e0, ctx->stream));
  launch();
  INTI_CUDA(cudaEventRecord(e1, ctx->stream));
  INTI_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  INTI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

void measure_peaks(inti_ctx* ctx, double* fp64, double* fp32, double* mufu) {
  DevBuf sink;
  sink.ensure(64);
  const int tb = 256;
  const int blocks = ctx->num_sms * 8;
  const double threads = (double)tb * blocks;
  {
    const int iters = 4096;
    const double ms = time_ms(ctx, [&] {
      fma_probe<double><<<blocks, tb, 0, ctx->stream>>>(iters, 0.999999, 1e-7, sink.as<double>());
      ctx->launches++;
    });
    *fp64 = 2.0 * kChains * (double)iters * threads / (ms * 1e-3);
  }
  {
    const int iters = 8192;
    const double ms = time_ms(ctx, [&] {
      fma_probe<float><<<blocks, tb, 0, ctx->stream>>>(iters, 0.9999f, 1e-5f, sink.as<float>());
      ctx->launches++;
    });
    *fp32 = 2.0 * kChains * (double)iters * threads / (ms * 1e-3);
  }
  {
    const int iters = 2048;
    const double ms = time_ms(ctx, [&] {
      mufu_probe<<<blocks, tb, 0, ctx->stream>>>(iters, sink.as<float>());
      ctx->launches++;
    });
    *mufu = (double)kChains * (double)iters * threads / (ms * 1e-3);
  }
  INTI_CUDA(cudaGetLastError());
}

}  // namespace inti
