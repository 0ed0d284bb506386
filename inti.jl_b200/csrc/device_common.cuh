// Device-side helpers shared by the kernels: the Laplace / Helmholtz kernel
// values in FP64 (generic form, used off the hot loop), the bulk-copy (TMA)
// and mbarrier primitives with bounded waits, and warp reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace inti {

// ---------------------------------------------------------------------------
// Generic kernel values K(x, y) with the reference's constants
// (src/kernels.jl:137-204 Laplace, :347-413 Helmholtz 3D); zero when
// |x - y| <= 1e-14 (src/utils.jl:235).  Returned as (re, im).
// ---------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ double dotd(const double* a, const double* b) {
  double s = a[0] * b[0];
#pragma unroll
  for (int i = 1; i < DIM; ++i) s = fma(a[i], b[i], s);
  return s;
}

template <int PDE, int KIND, int DIM>
__device__ __forceinline__ double2 kernel_value(const double* x, const double* nx,
                                                const double* y, const double* ny, double k) {
  double r[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) r[i] = x[i] - y[i];
  const double d2 = dotd<DIM>(r, r);
  if (!(d2 > kSamePointTol2)) return make_double2(0.0, 0.0);
  const double d = sqrt(d2);
  if (PDE == LAPLACE) {
    if (KIND == SL) {
      if (DIM == 2) return make_double2(-log(d) / (2 * kPi), 0.0);
      return make_double2(1.0 / (4 * kPi) / d, 0.0);
    } else if (KIND == DL) {
      const double c = DIM == 2 ? 1.0 / (2 * kPi) / d2 : 1.0 / (4 * kPi) / (d2 * d);
      return make_double2(c * dotd<DIM>(r, ny), 0.0);
    } else if (KIND == ADL) {
      const double c = DIM == 2 ? -1.0 / (2 * kPi) / d2 : -1.0 / (4 * kPi) / (d2 * d);
      return make_double2(c * dotd<DIM>(r, nx), 0.0);
    } else {
      const double id2 = 1.0 / d2;
      const double nxdny = dotd<DIM>(nx, ny), rdnx = dotd<DIM>(r, nx), rdny = dotd<DIM>(r, ny);
      if (DIM == 2) return make_double2(id2 / (2 * kPi) * (nxdny - 2 * rdnx * rdny * id2), 0.0);
      return make_double2(id2 / (4 * kPi * d) * (nxdny - 3 * rdnx * rdny * id2), 0.0);
    }
  } else {
    double s, c;
    sincos(k * d, &s, &c);
    const double inv4pi = 1.0 / (4 * kPi);
    if (KIND == SL) {
      const double g = inv4pi / d;
      return make_double2(g * c, g * s);
    }
    // e^{ikd} (1/d - ik) = (c/d + k s) + i (s/d - k c)
    const double id = 1.0 / d;
    const double er = c * id + k * s, ei = s * id - k * c;
    if (KIND == DL || KIND == ADL) {
      const double rn = KIND == DL ? dotd<3>(r, ny) : -dotd<3>(r, nx);
      const double g = inv4pi / d2 * rn;
      return make_double2(g * er, g * ei);
    }
    // HS: a (r.nx)(r.ny) + b nx.ny
    const double rdnx = dotd<3>(r, nx), rdny = dotd<3>(r, ny), nxdny = dotd<3>(nx, ny);
    const double id2 = 1.0 / d2;
    // b = e^{ikd} id2/(4pi) (1/d - ik)
    const double br = er * id2 * inv4pi, bi = ei * id2 * inv4pi;
    // a = e^{ikd} id2^2/(4 pi d) (3(ikd - 1) + k^2 d^2)
    const double fr = -3.0 + k * k * d2, fi = 3.0 * k * d;
    const double sa = id2 * id2 * inv4pi * id;
    const double ar = sa * (c * fr - s * fi), ai = sa * (c * fi + s * fr);
    const double t = rdnx * rdny;
    return make_double2(ar * t + br * nxdny, ai * t + bi * nxdny);
  }
}

// ---------------------------------------------------------------------------
// Bulk asynchronous copies global -> shared (cp.async.bulk, the TMA engine)
// completed on an mbarrier, with waits bounded by an iteration limit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// dst (shared) and src (global) 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Upper bound on polls of one barrier phase.  Each poll that finds the phase
// incomplete may suspend the thread for a hardware-chosen interval (about
// 4 us on the B200: 2^22 polls took 16.6 s), so 2^18 polls give up after
// about a second, far beyond any healthy copy or MMA.
constexpr uint32_t kWaitLimit = 1u << 18;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < kWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Error codes written to the context's device flag.
constexpr int kErrWaitTimeout = 1;

// ---------------------------------------------------------------------------
// Fast special functions for the pair loops, from published methods:
//  * rsqrt: hardware approximation (MUFU) refined by one third-order Newton
//    step for 1/sqrt(x): with e = 1 - x*y^2, y' = y*(1 + e/2 + 3e^2/8)
//    (Householder's method of order 3); relative error ~(5/16)e^3.
//  * x^{-3/2} from the same seed: x^{-3/2} = y^3 (1 - e)^{-3/2}
//    = y^3 (1 + 3e/2 + 15e^2/8 + O(e^3)), the binomial series cut after the
//    quadratic term (relative error ~(35/16)e^3), one step instead of the
//    refined 1/sqrt(x) and two products.
//  * e^{i*theta} for theta = u*delta, u = d*kT, delta = 2*pi/kExpiTable:
//    split u = m + f (m = rint(u), |f| <= 1/2), take e^{i*m*delta} from a
//    table built on the host in extended precision, and e^{i*f*delta} from
//    its Taylor series (|f*delta| <= pi/1024: sin to r^5, cos to r^4 leave
//    truncation errors below 2e-18).  In FP64, m comes from adding and
//    subtracting 1.5*2^52 (for |u| < 2^51 the rounded sum's low word is m in
//    two's complement, the table index without a conversion instruction) and
//    delta's powers are folded into the series' coefficients.
// The FP32 pair loops take e^{i*theta} from the hardware sine and cosine of
// the phase reduced by whole turns (below).  The accuracy of all of them is
// measured on the device by inti_selftest_math.
// ---------------------------------------------------------------------------
constexpr int kExpiTable = 1024;

__device__ __forceinline__ double rsqrt_approx_f64(double x) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}
__device__ __forceinline__ float rsqrt_approx_f32(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// d^2 > (1e-14)^2 for d^2 >= +0 as a compare of the bit patterns (IEEE
// order of non-negative doubles), on the integer pipe.
__device__ __forceinline__ bool pair_keep(double d2) {
  return __double_as_longlong(d2) > __double_as_longlong(1.0e-28);
}

// 1/sqrt(x) to ~1 ulp for normal x > 0 (inf/NaN for x == 0, as 1/sqrt).
__device__ __forceinline__ double rsqrt_fast(double x) {
  const double y = rsqrt_approx_f64(x);
  const double t = x * y;
  const double e = fma(-t, y, 1.0);
  const double p = fma(e, 0.375, 0.5);
  return fma(y, e * p, y);
}
__device__ __forceinline__ float rsqrt_fast(float x) { return rsqrt_approx_f32(x); }

__device__ __forceinline__ double rcp_approx_f64(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}

// 1/x to ~1 ulp for normal x > 0 (NaN for x == 0): the hardware estimate y
// refined by one third-order Newton step for f(y) = 1/y - x,
// y' = y (1 + e + e^2) with e = 1 - x y, which cubes the relative error.
__device__ __forceinline__ double rcp_fast(double x) {
  const double y = rcp_approx_f64(x);
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

// x^{-3/2} to a few ulp for normal x > 0 (NaN for x == 0).
__device__ __forceinline__ double rsqrt_cube_fast(double x) {
  const double y = rsqrt_approx_f64(x);
  const double y2 = y * y;
  const double e = fma(-x, y2, 1.0);
  const double y3 = y2 * y;
  const double p = fma(e, 1.875, 1.5);
  return fma(y3, e * p, y3);
}
__device__ __forceinline__ float rsqrt_cube_fast(float x) {
  const float y = rsqrt_approx_f32(x);
  return y * y * y;
}

constexpr double kRoundShift = 6755399441055744.0;  // 1.5 * 2^52
constexpr double kExpiDelta = 2.0 * 3.14159265358979323846 / 1024.0;
// (c, s) = e^{i d kT delta}; delta = 2 pi / kExpiTable (FP32: passed in).
__device__ __forceinline__ void expi_table_eval(double d, double kT, const double2* __restrict__ tab,
                                                double /*delta*/, double& c, double& s) {
  constexpr double D = kExpiDelta;
  constexpr double C2 = -D * D / 2.0, C4 = D * D * D * D / 24.0;
  constexpr double S3 = -D * D * D / 6.0, S5 = D * D * D * D * D / 120.0;
  const double t = fma(d, kT, kRoundShift);
  const double m = t - kRoundShift;
  const double f = fma(d, kT, -m);
  const double f2 = f * f;
  const double cp = fma(f2, fma(f2, C4, C2), 1.0);
  const double sp = f * fma(f2, fma(f2, S5, S3), D);
  const double2 e = tab[__double2loint(t) & (kExpiTable - 1)];
  c = fma(cp, e.x, -sp * e.y);
  s = fma(sp, e.x, cp * e.y);
}

// FP32: the phase u = d*kT (in units of delta) is reduced by whole turns
// (multiples of kExpiTable, an exact subtraction: |u - m| <= kExpiTable/2 and
// m/2 <= u <= 2m), and the hardware sine and cosine (MUFU) take the reduced
// angle, |theta| <= pi.  The error is the rounding of u (relative 6e-8, i.e.
// 6e-8 * kd absolute) plus the approximations' 2^-21; the table is not used.
// Measured by inti_selftest_math: 1.05e-6 for kd <= 25 (the table form gave
// 7.5e-7 with about ten more instructions per evaluation).
__device__ __forceinline__ void expi_table_eval(float d, float kT, const float2* __restrict__ /*tab*/,
                                                float delta, float& c, float& s) {
  const float u = d * kT;
  const float m = rintf(u * (1.0f / kExpiTable)) * (float)kExpiTable;
  const float th = (u - m) * delta;
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(th));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(th));
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace inti
