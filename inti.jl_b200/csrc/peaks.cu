// Throughput probes for the roofline denominators of the pair kernels: FP64
// FMA, FP32 FMA and the MUFU reciprocal square root, each as many independent
// dependency chains per thread over a grid that fills every SM.  Timed with
// CUDA events on the context's stream at the clock the device runs at, so the
// peak and the kernel it normalises see the same conditions.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "common.h"
#include "device_common.cuh"
#include "internal.h"

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

// Evaluates the pair loops' fast special functions on given inputs.
__global__ void math_probe(int n, const double* x, double* rs, double* rs3, double* rc, const double* u,
                           const double2* tab64, const float2* tab32, double2* e64, float2* e32) {
  __shared__ double2 t64[kExpiTable];
  __shared__ float2 t32[kExpiTable];
  for (int q = threadIdx.x; q < kExpiTable; q += blockDim.x) {
    t64[q] = tab64[q];
    t32[q] = tab32[q];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rs[i] = rsqrt_fast(x[i]);
  rs3[i] = rsqrt_cube_fast(x[i]);
  rc[i] = rcp_fast(x[i]);
  double c, s;
  expi_table_eval(u[i], 1.0, t64, 2 * kPi / kExpiTable, c, s);
  e64[i] = make_double2(c, s);
  float cf, sf;
  expi_table_eval((float)u[i], 1.0f, t32, (float)(2 * kPi / kExpiTable), cf, sf);
  e32[i] = make_float2(cf, sf);
}

// A bounded wait that runs out: one thread waits for the first phase of an
// mbarrier that nothing arrives at, with the pair kernels' own bounded wait,
// and records the timeout in the context's flag as they do.
__global__ void wait_timeout_probe(int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0)) atomicExch(err, kErrWaitTimeout);
}

void selftest_wait_timeout(inti_ctx* ctx) {
  ctx->flag_armed = true;
  wait_timeout_probe<<<1, 32, 0, ctx->stream>>>(ctx->err_flag.as<int>());
  ctx->launches++;
  INTI_CUDA(cudaGetLastError());
  sync_and_check(ctx);  // throws INTI_E_TIMEOUT and clears the flag
}

void selftest_math(inti_ctx* ctx, double* out) {
  const int n = 1 << 16;
  std::vector<double> x(n), u(n);
  uint64_t st = 88172645463325252ull;
  auto rnd = [&] {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int i = 0; i < n; ++i) {
    x[i] = std::pow(10.0, -27.0 + 54.0 * rnd());
    // phases: half up to 25 rad (k d of the workloads), half up to 1000 rad
    const double th = i < n / 2 ? 25.0 * rnd() : 1000.0 * rnd();
    u[i] = th * kExpiTable / (2 * kPi);
  }
  DevBuf dx, drs, drs3, drc, du, d64, d32;
  dx.ensure(8 * n);
  drs.ensure(8 * n);
  drs3.ensure(8 * n);
  drc.ensure(8 * n);
  du.ensure(8 * n);
  d64.ensure(16 * n);
  d32.ensure(8 * n);
  INTI_CUDA(cudaMemcpy(dx.p, x.data(), 8 * n, cudaMemcpyHostToDevice));
  INTI_CUDA(cudaMemcpy(du.p, u.data(), 8 * n, cudaMemcpyHostToDevice));
  math_probe<<<n / 256, 256, 0, ctx->stream>>>(n, dx.as<double>(), drs.as<double>(), drs3.as<double>(),
                                               drc.as<double>(), du.as<double>(),
                                               expi_table_f64(ctx), expi_table_f32(ctx),
                                               d64.as<double2>(), d32.as<float2>());
  ctx->launches++;
  INTI_CUDA(cudaGetLastError());
  INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  std::vector<double> rs(n), rs3(n), rc(n);
  std::vector<double2> e64(n);
  std::vector<float2> e32(n);
  INTI_CUDA(cudaMemcpy(rs.data(), drs.p, 8 * n, cudaMemcpyDeviceToHost));
  INTI_CUDA(cudaMemcpy(rs3.data(), drs3.p, 8 * n, cudaMemcpyDeviceToHost));
  INTI_CUDA(cudaMemcpy(rc.data(), drc.p, 8 * n, cudaMemcpyDeviceToHost));
  INTI_CUDA(cudaMemcpy(e64.data(), d64.p, 16 * n, cudaMemcpyDeviceToHost));
  INTI_CUDA(cudaMemcpy(e32.data(), d32.p, 8 * n, cudaMemcpyDeviceToHost));
  double m0 = 0, m1 = 0, m2 = 0, m3 = 0, m4 = 0, m5 = 0;
  const long double delta = (long double)(2 * kPi / kExpiTable);
  for (int i = 0; i < n; ++i) {
    const long double ref = 1.0L / sqrtl((long double)x[i]);
    m0 = std::max(m0, (double)fabsl(((long double)rs[i] - ref) / ref));
    const long double ref3 = ref * ref * ref;
    m4 = std::max(m4, (double)fabsl(((long double)rs3[i] - ref3) / ref3));
    const long double refr = 1.0L / (long double)x[i];
    m5 = std::max(m5, (double)fabsl(((long double)rc[i] - refr) / refr));
    const long double th = (long double)u[i] * delta;
    const double err64 = (double)std::max(fabsl(e64[i].x - cosl(th)), fabsl(e64[i].y - sinl(th)));
    const double err32 = (double)std::max(fabsl(e32[i].x - cosl(th)), fabsl(e32[i].y - sinl(th)));
    if (i < n / 2) {
      m1 = std::max(m1, err64);
      m3 = std::max(m3, err32);
    } else {
      m2 = std::max(m2, err64);
    }
  }
  out[0] = m0;
  out[1] = m1;
  out[2] = m2;
  out[3] = m3;
  out[4] = m4;
  out[5] = m5;
}

}  // namespace inti
