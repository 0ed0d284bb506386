// Restarted GMRES on L = shift*I + sum_t coef_t*(A_t + C_t) with every vector
// resident in HBM.  Inti.jl itself has no solver; its examples call
// IterativeSolvers.gmres on a LinearMap sum (docs/src/examples/poisson.jl:
// 166-168, docs/src/examples/helmholtz_scattering.jl:485-495), one operator
// application per Krylov step.  This driver keeps that contract (restart,
// relative residual tolerance) and adds a precision form:
//
//  * FP64: Arnoldi on the FP64 operators.
//  * MIXED: iterative refinement.  The residual r = b - L x is formed with
//    the FP64 operators (pairs and correction SpMV in FP64); the correction
//    equation L e = r is solved by GMRES on FP32C twins of the operators (FP32
//    pairs with compensated sums, FP64 correction SpMV), x += e, repeat until
//    ||b - L x|| <= rtol ||b|| measured in FP64.
//
// Orthogonalisation is classical Gram-Schmidt applied twice (CGS2): two
// fused multi-dot / update kernel pairs per step, deterministic block
// reductions.  The small Hessenberg least-squares problem (Givens rotations)
// runs on the host from one device->host copy per step.  Small systems
// (n <= 8192 unknowns by default) take a whole step after the operator application in
// one single-CTA kernel (both CGS passes, the norm, the new basis vector and
// the Givens update on the device) and the host looks at the residuals once
// per kArnoldiBatch steps, so a step costs two or three launches and no
// round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <memory>
#include <vector>

#include "common.h"
#include "device_common.cuh"
#include "internal.h"

namespace inti {

using cplx = std::complex<double>;
constexpr int kDotBlock = 256;

template <bool C>
struct VT;
template <>
struct VT<false> { using T = double; };
template <>
struct VT<true> { using T = double2; };

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cjm(double2 a, double2 b) {  // conj(a)*b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// partial[blk][k] = sum over the block's rows of conj(V[k][i]) * w[i]
template <bool C>
__global__ void __launch_bounds__(kDotBlock) multi_dot(int64_t n, int kcount, const double* V,
                                                       int64_t ldv, const double* w,
                                                       double2* partial) {
  __shared__ double2 red[kDotBlock / 32];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int k = 0; k < kcount; ++k) {
    double sr = 0.0, si = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += kDotBlock) {
      if (C) {
        const double2 v = reinterpret_cast<const double2*>(V + 2 * (k * ldv))[i];
        const double2 x = reinterpret_cast<const double2*>(w)[i];
        const double2 p = cjm(v, x);
        sr += p.x;
        si += p.y;
      } else {
        sr = fma(V[k * ldv + i], w[i], sr);
      }
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = make_double2(sr, si);
    __syncthreads();
    if (threadIdx.x == 0) {
      double ar = 0.0, ai = 0.0;
      for (int q = 0; q < kDotBlock / 32; ++q) {
        ar += red[q].x;
        ai += red[q].y;
      }
      partial[(int64_t)blockIdx.x * kcount + k] = make_double2(ar, ai);
    }
    __syncthreads();
  }
}

// out[k] (+)= sum_blk partial[blk][k]
__global__ void dot_reduce(int nblk, int kcount, const double2* partial, double2* out, bool accumulate) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kcount) return;
  double sr = 0.0, si = 0.0;
  for (int b = 0; b < nblk; ++b) {
    sr += partial[(int64_t)b * kcount + k].x;
    si += partial[(int64_t)b * kcount + k].y;
  }
  if (accumulate) {
    out[k].x += sr;
    out[k].y += si;
  } else {
    out[k] = make_double2(sr, si);
  }
}

// w -= sum_k V[k] * h[k]   (or x += sum_k V[k] * h[k] when sign = +1)
template <bool C>
__global__ void multi_axpy(int64_t n, int kcount, const double* V, int64_t ldv, const double2* h,
                           double* w, double sign) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (C) {
    double2 acc = reinterpret_cast<double2*>(w)[i];
    for (int k = 0; k < kcount; ++k) {
      const double2 p = cm(reinterpret_cast<const double2*>(V + 2 * (k * ldv))[i], h[k]);
      acc.x += sign * p.x;
      acc.y += sign * p.y;
    }
    reinterpret_cast<double2*>(w)[i] = acc;
  } else {
    double acc = w[i];
    for (int k = 0; k < kcount; ++k) acc = fma(sign * h[k].x, V[k * ldv + i], acc);
    w[i] = acc;
  }
}

// y = a*x + b*y (complex a, b; real vectors use the real parts)
template <bool C>
__global__ void axpby(int64_t n, double ar, double ai, const double* x, double br, double bi,
                      double* y, bool bzero) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (C) {
    const double2 xv = reinterpret_cast<const double2*>(x)[i];
    double2 r = cm(make_double2(ar, ai), xv);
    if (!bzero) {
      const double2 yv = reinterpret_cast<const double2*>(y)[i];
      const double2 q = cm(make_double2(br, bi), yv);
      r.x += q.x;
      r.y += q.y;
    }
    reinterpret_cast<double2*>(y)[i] = r;
  } else {
    double r = ar * x[i];
    if (!bzero) r += br * y[i];
    y[i] = r;
  }
}

constexpr int kArnoldiThreads = 1024;
constexpr int kArnoldiBatch = 4;

// Device state of a small-system Arnoldi cycle: the rotated Hessenberg
// matrix R ((restart+1) x restart, column-major), the Givens rotations, the
// rotated right-hand side g, the residual estimate after each step and
// flags[0] = stop (converged or breakdown), flags[1] = steps done.
struct ArnoldiState {
  double2 *R, *cs, *sn, *g;
  double* res;
  int* flags;
};

__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }

template <bool C>
__device__ __forceinline__ double2 load_c(const double* v, int64_t i) {
  return C ? reinterpret_cast<const double2*>(v)[i] : make_double2(v[i], 0.0);
}

// Step j of a small-system cycle, after w = sum_t coef_t A_t v_j (the shift
// is added here, w += shift * v_j, saving a launch per step): w is orthogonalised
// against v_0..v_j twice (CGS2; sums in a fixed order), v_{j+1} = w/|w|,
// and thread 0 applies the earlier rotations to the new Hessenberg column,
// forms rotation j, and records |g[j+1]|.  A stopped cycle leaves later
// steps as no-ops.  Dynamic shared memory: 2 * (restart + 1) double2.
template <bool C>
__global__ void __launch_bounds__(kArnoldiThreads) arnoldi_small_step(int64_t n, int j, int restart, double* V,
                                                                      double* w, double2 shift, double tol_abs,
                                                                      ArnoldiState st) {
  extern __shared__ double2 hbuf[];
  __shared__ double2 red[kArnoldiThreads / 32][8];
  __shared__ double hn_s;
  if (st.flags[0]) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int comps = C ? 2 : 1;
  double2* hsum = hbuf;               // [restart + 1]
  double2* hp = hbuf + restart + 1;   // [restart + 1]
  for (int k = tid; k <= j; k += kArnoldiThreads) hsum[k] = make_double2(0.0, 0.0);
  if (shift.x != 0.0 || shift.y != 0.0) {  // each thread its own entries, as in the passes below
    const double* vj = V + (int64_t)comps * n * j;
    for (int64_t i = tid; i < n; i += kArnoldiThreads) {
      if (C) {
        const double2 a = reinterpret_cast<const double2*>(w)[i];
        const double2 p = cm(shift, reinterpret_cast<const double2*>(vj)[i]);
        reinterpret_cast<double2*>(w)[i] = make_double2(a.x + p.x, a.y + p.y);
      } else {
        w[i] += shift.x * vj[i];
      }
    }
  }
  for (int pass = 0; pass < 2; ++pass) {
    for (int k0 = 0; k0 <= j; k0 += 8) {
      double2 acc[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) acc[u] = make_double2(0.0, 0.0);
      for (int64_t i = tid; i < n; i += kArnoldiThreads) {
        const double2 wi = load_c<C>(w, i);
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (k0 + u <= j) acc[u] = c_add(acc[u], cjm(load_c<C>(V + (int64_t)comps * n * (k0 + u), i), wi));
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        acc[u].x = warp_sum(acc[u].x);
        acc[u].y = warp_sum(acc[u].y);
      }
      if (lane == 0)
#pragma unroll
        for (int u = 0; u < 8; ++u) red[warp][u] = acc[u];
      __syncthreads();
      if (tid < 8 && k0 + tid <= j) {
        double2 t = make_double2(0.0, 0.0);
        for (int q = 0; q < kArnoldiThreads / 32; ++q) t = c_add(t, red[q][tid]);
        hp[k0 + tid] = t;
      }
      __syncthreads();
    }
    // w -= V hp (each thread updates the entries it reads)
    for (int64_t i = tid; i < n; i += kArnoldiThreads) {
      double2 a = load_c<C>(w, i);
      for (int k = 0; k <= j; ++k) {
        const double2 p = cm(load_c<C>(V + (int64_t)comps * n * k, i), hp[k]);
        a.x -= p.x;
        a.y -= p.y;
      }
      if (C)
        reinterpret_cast<double2*>(w)[i] = a;
      else
        w[i] = a.x;
    }
    for (int k = tid; k <= j; k += kArnoldiThreads) hsum[k] = c_add(hsum[k], hp[k]);
    __syncthreads();
  }
  double s2 = 0.0;
  for (int64_t i = tid; i < n; i += kArnoldiThreads) {
    const double2 a = load_c<C>(w, i);
    s2 = fma(a.x, a.x, fma(a.y, a.y, s2));
  }
  s2 = warp_sum(s2);
  if (lane == 0) red[warp][0].x = s2;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int q = 0; q < kArnoldiThreads / 32; ++q) t += red[q][0].x;
    hn_s = sqrt(fmax(t, 0.0));
  }
  __syncthreads();
  const double hn = hn_s;
  if (hn > 0.0) {
    double* vn = V + (int64_t)comps * n * (j + 1);
    const double inv = 1.0 / hn;
    for (int64_t i = tid; i < n; i += kArnoldiThreads) {
      if (C) {
        const double2 a = reinterpret_cast<const double2*>(w)[i];
        reinterpret_cast<double2*>(vn)[i] = make_double2(a.x * inv, a.y * inv);
      } else {
        vn[i] = w[i] * inv;
      }
    }
  }
  if (tid == 0) {
    double2* col = hsum;  // column j of H, then rotated in place (row j + 1 = hn)
    col[j + 1] = make_double2(hn, 0.0);
    for (int i = 0; i < j; ++i) {
      const double2 a = col[i], b = col[i + 1], c = st.cs[i], sg = st.sn[i];
      col[i] = c_add(cm(c_conj(c), a), cm(c_conj(sg), b));
      const double2 t1 = cm(sg, a), t2 = cm(c, b);
      col[i + 1] = make_double2(t2.x - t1.x, t2.y - t1.y);
    }
    const double2 a = col[j], b = col[j + 1];
    const double den = sqrt(a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y);
    const double2 cj = den == 0.0 ? make_double2(1.0, 0.0) : make_double2(a.x / den, a.y / den);
    const double2 sj = den == 0.0 ? make_double2(0.0, 0.0) : make_double2(b.x / den, b.y / den);
    st.cs[j] = cj;
    st.sn[j] = sj;
    col[j] = make_double2(den, 0.0);
    const double2 gj = st.g[j];
    const double2 ng = cm(sj, gj);
    st.g[j + 1] = make_double2(-ng.x, -ng.y);
    st.g[j] = cm(c_conj(cj), gj);
    double2* Rj = st.R + (int64_t)(restart + 1) * j;
    for (int i = 0; i <= j; ++i) Rj[i] = col[i];
    const double2 gn = st.g[j + 1];
    const double res = sqrt(gn.x * gn.x + gn.y * gn.y);
    st.res[j] = res;
    st.flags[1] = j + 1;
    if (res <= tol_abs || hn == 0.0) st.flags[0] = 1;
  }
}

struct Solver {
  inti_ctx* ctx;
  int64_t n;
  bool C;  // complex arithmetic
  int comps;
  int nblk;
  std::vector<inti_op*> ops64, ops32;
  std::vector<cplx> coefs;
  cplx shift;
  int fp64_applies = 0, fp32_applies = 0;

  double* vec(DevBuf& b, int64_t count = 1) {
    b.ensure(sizeof(double) * comps * n * count);
    return b.as<double>();
  }
  void launch_axpby(cplx a, const double* x, cplx b, double* y) {
    const unsigned g = (unsigned)((n + 255) / 256);
    const bool bz = b == cplx(0, 0);
    if (C)
      axpby<true><<<g, 256, 0, ctx->stream>>>(n, a.real(), a.imag(), x, b.real(), b.imag(), y, bz);
    else
      axpby<false><<<g, 256, 0, ctx->stream>>>(n, a.real(), a.imag(), x, b.real(), b.imag(), y, bz);
    ctx->launches++;
  }
  // out = L v using the FP64 or FP32C operators
  void apply(bool fp32, const double* v, double* out) {
    launch_axpby(shift, v, cplx(0, 0), out);
    auto& ops = fp32 ? ops32 : ops64;
    for (size_t t = 0; t < ops.size(); ++t) {
      const double al[2] = {coefs[t].real(), coefs[t].imag()};
      const double be[2] = {1.0, 0.0};
      op_apply_device(ops[t], v, out, al, be);
    }
    (fp32 ? fp32_applies : fp64_applies)++;
  }
  // out = sum_t coef_t A_t v (no shift term; the small-system step adds it)
  void apply_unshifted(bool fp32, const double* v, double* out) {
    auto& ops = fp32 ? ops32 : ops64;
    for (size_t t = 0; t < ops.size(); ++t) {
      const double al[2] = {coefs[t].real(), coefs[t].imag()};
      const double be[2] = {t == 0 ? 0.0 : 1.0, 0.0};
      op_apply_device(ops[t], v, out, al, be);
    }
    (fp32 ? fp32_applies : fp64_applies)++;
  }
  // h[0:kcount] (=|+=) V^H w  (device)
  void dots(const double* V, int64_t ldv, int kcount, const double* w, double2* h, bool acc) {
    DevBuf& partial = ctx->krylov.partial;
    partial.ensure(sizeof(double2) * (size_t)nblk * std::max(kcount, 1));
    if (C)
      multi_dot<true><<<nblk, kDotBlock, 0, ctx->stream>>>(n, kcount, V, ldv, w, partial.as<double2>());
    else
      multi_dot<false><<<nblk, kDotBlock, 0, ctx->stream>>>(n, kcount, V, ldv, w, partial.as<double2>());
    dot_reduce<<<(kcount + 127) / 128, 128, 0, ctx->stream>>>(nblk, kcount, partial.as<double2>(), h, acc);
    ctx->launches += 2;
  }
  void maxpy(const double* V, int64_t ldv, int kcount, const double2* h, double* w, double sign) {
    const unsigned g = (unsigned)((n + 255) / 256);
    if (C)
      multi_axpy<true><<<g, 256, 0, ctx->stream>>>(n, kcount, V, ldv, h, w, sign);
    else
      multi_axpy<false><<<g, 256, 0, ctx->stream>>>(n, kcount, V, ldv, h, w, sign);
    ctx->launches++;
  }
  double norm(const double* w) {
    DevBuf& h = ctx->krylov.nrm;
    h.ensure(sizeof(double2));
    dots(w, 0, 1, w, h.as<double2>(), false);
    double2 v;
    INTI_CUDA(cudaMemcpyAsync(&v, h.p, sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    return std::sqrt(std::max(v.x, 0.0));
  }

  bool small_cycle(int restart) const { return n <= ctx->krylov_small && restart <= 1000; }

  // One Arnoldi cycle of a small system with v_0 = V[0] normalised and
  // g = (beta, 0, ...): steps of one operator application and one
  // arnoldi_small_step each, kArnoldiBatch at a time between host checks.
  // Fills H (rows 0..j-1 of the rotated Hessenberg matrix, row-major with
  // `restart` columns) and g[0..j], and returns the steps j kept; steps
  // enqueued after the cycle stopped are no-ops.
  int arnoldi_cycle_small(bool fp32, double* V, double* w, double beta, double tol_abs, int restart, int maxit,
                          int& it, double& res, bool& done, double* history, double bnorm_for_history,
                          int hist_offset, std::vector<cplx>& H, std::vector<cplx>& g) {
    const size_t nR = (size_t)(restart + 1) * restart;
    const size_t bytes = sizeof(double2) * (nR + 2 * (size_t)restart + (restart + 1)) + sizeof(double) * restart +
                         2 * sizeof(int);
    DevBuf& sb = ctx->krylov.small;
    sb.ensure(bytes);
    ArnoldiState st;
    st.R = sb.as<double2>();
    st.cs = st.R + nR;
    st.sn = st.cs + restart;
    st.g = st.sn + restart;
    st.res = reinterpret_cast<double*>(st.g + restart + 1);
    st.flags = reinterpret_cast<int*>(st.res + restart);
    INTI_CUDA(cudaMemsetAsync(st.g, 0, sizeof(double2) * (restart + 1), ctx->stream));
    INTI_CUDA(cudaMemsetAsync(st.flags, 0, 2 * sizeof(int), ctx->stream));
    const double2 g0 = make_double2(beta, 0.0);
    INTI_CUDA(cudaMemcpyAsync(st.g, &g0, sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    const size_t smem = sizeof(double2) * 2 * (restart + 1);
    std::vector<double> rh(restart);
    int flags[2] = {0, 0};
    int j = 0;
    while (j < restart && it < maxit && !done) {
      const int batch = std::min({kArnoldiBatch, restart - j, maxit - it});
      for (int b = 0; b < batch; ++b) {
        apply_unshifted(fp32, V + (size_t)comps * n * (j + b), w);
        const double2 sh = make_double2(shift.real(), shift.imag());
        if (C)
          arnoldi_small_step<true><<<1, kArnoldiThreads, smem, ctx->stream>>>(n, j + b, restart, V, w, sh, tol_abs,
                                                                               st);
        else
          arnoldi_small_step<false><<<1, kArnoldiThreads, smem, ctx->stream>>>(n, j + b, restart, V, w, sh,
                                                                                tol_abs, st);
        ctx->launches++;
      }
      INTI_CUDA(cudaMemcpyAsync(rh.data() + j, st.res + j, sizeof(double) * batch, cudaMemcpyDeviceToHost,
                                ctx->stream));
      INTI_CUDA(cudaMemcpyAsync(flags, st.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
      INTI_CUDA(cudaStreamSynchronize(ctx->stream));
      const int now = flags[1];  // steps done in this cycle
      for (; j < now; ++j) {
        ++it;
        res = rh[j];
        if (history) history[hist_offset + it] = res / bnorm_for_history;
      }
      if (flags[0]) done = true;
    }
    if (j > 0) {
      std::vector<double2> Rh((size_t)(restart + 1) * j), gh(j + 1);
      INTI_CUDA(cudaMemcpyAsync(Rh.data(), st.R, sizeof(double2) * Rh.size(), cudaMemcpyDeviceToHost, ctx->stream));
      INTI_CUDA(cudaMemcpyAsync(gh.data(), st.g, sizeof(double2) * (j + 1), cudaMemcpyDeviceToHost, ctx->stream));
      INTI_CUDA(cudaStreamSynchronize(ctx->stream));
      for (int c = 0; c < j; ++c)
        for (int r = 0; r <= c; ++r)
          H[(size_t)r * restart + c] = cplx(Rh[(size_t)(restart + 1) * c + r].x, Rh[(size_t)(restart + 1) * c + r].y);
      for (int r = 0; r <= j; ++r) g[r] = cplx(gh[r].x, gh[r].y);
    }
    return j;
  }

  // GMRES(restart) on L (fp32 selects the operators) for L e = rhs, e0 = x.
  // Stops at ||rhs - L x|| <= tol_abs (estimated by the Arnoldi recurrence)
  // or after maxit steps.  Returns the steps used; est receives the final
  // residual estimate.
  int gmres(bool fp32, const double* rhs, double* x, double tol_abs, int restart, int maxit,
            double bnorm_for_history, double* history, int hist_offset, double* est,
            bool x_is_zero, bool final_true_residual) {
    double* V = vec(ctx->krylov.V, restart + 1);
    double* w = vec(ctx->krylov.w);
    // the dot-product partials for the widest step, so no step reallocates
    ctx->krylov.partial.ensure(sizeof(double2) * (size_t)nblk * (restart + 2));
    DevBuf& hbuf = ctx->krylov.h;
    DevBuf& ybuf = ctx->krylov.y;
    hbuf.ensure(sizeof(double2) * (restart + 2) * 2);
    double2* h1 = hbuf.as<double2>();
    double2* h2 = h1 + (restart + 2);
    std::vector<double2> hh(restart + 2);
    int it = 0;
    double res = 0.0;
    bool zero = x_is_zero;
    while (true) {
      // r = rhs - L x into V[0]
      double* v0 = V;
      if (zero) {
        INTI_CUDA(cudaMemcpyAsync(v0, rhs, sizeof(double) * comps * n, cudaMemcpyDeviceToDevice, ctx->stream));
      } else {
        apply(fp32, x, w);
        launch_axpby(cplx(1, 0), rhs, cplx(0, 0), v0);
        launch_axpby(cplx(-1, 0), w, cplx(1, 0), v0);
      }
      const double beta = norm(v0);
      res = beta;
      if (beta <= tol_abs || it >= maxit || beta == 0.0) break;
      launch_axpby(cplx(1.0 / beta, 0), v0, cplx(0, 0), v0);
      std::vector<cplx> H((size_t)(restart + 1) * restart, cplx(0, 0)), cs(restart), sn(restart),
          g(restart + 1, cplx(0, 0));
      g[0] = beta;
      int j = 0;
      bool done = false;
      if (small_cycle(restart)) {
        j = arnoldi_cycle_small(fp32, V, w, beta, tol_abs, restart, maxit, it, res, done, history,
                                bnorm_for_history, hist_offset, H, g);
      }
      for (; !small_cycle(restart) && j < restart && it < maxit; ++j) {
        double* vj = V + (size_t)comps * n * j;
        apply(fp32, vj, w);
        // CGS2
        dots(V, n, j + 1, w, h1, false);
        maxpy(V, n, j + 1, h1, w, -1.0);
        dots(V, n, j + 1, w, h2, false);
        maxpy(V, n, j + 1, h2, w, -1.0);
        dots(w, 0, 1, w, h2 + j + 1, false);
        INTI_CUDA(cudaMemcpyAsync(hh.data(), h1, sizeof(double2) * (j + 1), cudaMemcpyDeviceToHost, ctx->stream));
        std::vector<double2> hh2(j + 2);
        INTI_CUDA(cudaMemcpyAsync(hh2.data(), h2, sizeof(double2) * (j + 2), cudaMemcpyDeviceToHost, ctx->stream));
        INTI_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int i = 0; i <= j; ++i) H[(size_t)i * restart + j] = cplx(hh[i].x + hh2[i].x, hh[i].y + hh2[i].y);
        const double hn = std::sqrt(std::max(hh2[j + 1].x, 0.0));
        H[(size_t)(j + 1) * restart + j] = hn;
        for (int i = 0; i < j; ++i) {
          const cplx a = H[(size_t)i * restart + j], b = H[(size_t)(i + 1) * restart + j];
          H[(size_t)i * restart + j] = std::conj(cs[i]) * a + std::conj(sn[i]) * b;
          H[(size_t)(i + 1) * restart + j] = -sn[i] * a + cs[i] * b;
        }
        const cplx a = H[(size_t)j * restart + j], b = H[(size_t)(j + 1) * restart + j];
        const double den = std::sqrt(std::norm(a) + std::norm(b));
        cs[j] = den == 0 ? cplx(1, 0) : a / den;
        sn[j] = den == 0 ? cplx(0, 0) : b / den;
        H[(size_t)j * restart + j] = den;
        H[(size_t)(j + 1) * restart + j] = 0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = std::conj(cs[j]) * g[j];
        ++it;
        res = std::abs(g[j + 1]);
        if (history) history[hist_offset + it] = res / bnorm_for_history;
        if (res <= tol_abs || hn == 0.0) {
          ++j;
          done = true;
          break;
        }
        launch_axpby(cplx(1.0 / hn, 0), w, cplx(0, 0), V + (size_t)comps * n * (j + 1));
      }
      // x += V y, R y = g
      std::vector<cplx> y(j);
      for (int i = j - 1; i >= 0; --i) {
        cplx s = g[i];
        for (int q = i + 1; q < j; ++q) s -= H[(size_t)i * restart + q] * y[q];
        y[i] = s / H[(size_t)i * restart + i];
      }
      std::vector<double2> yd(std::max(j, 1));
      for (int i = 0; i < j; ++i) yd[i] = make_double2(y[i].real(), y[i].imag());
      ybuf.ensure(sizeof(double2) * std::max(j, 1));
      INTI_CUDA(cudaMemcpyAsync(ybuf.p, yd.data(), sizeof(double2) * j, cudaMemcpyHostToDevice, ctx->stream));
      if (j > 0) {
        if (zero) {
          launch_axpby(cplx(0, 0), V, cplx(0, 0), x);  // x = 0 explicitly
          zero = false;
        }
        maxpy(V, n, j, ybuf.as<double2>(), x, +1.0);
      }
      if (done || it >= maxit) {
        if (!final_true_residual) break;
        apply(fp32, x, w);
        launch_axpby(cplx(1, 0), rhs, cplx(0, 0), v0);
        launch_axpby(cplx(-1, 0), w, cplx(1, 0), v0);
        res = norm(v0);
        break;
      }
    }
    if (zero) launch_axpby(cplx(0, 0), rhs, cplx(0, 0), x);
    *est = res;
    return it;
  }
};

void gmres_solve(inti_ctx* ctx, int32_t nterms, inti_op* const* ops, const double* coefs,
                 const double* shift, const double* b, double* x, double rtol, int32_t restart,
                 int32_t maxiter, int32_t mode, int on_device, double* history,
                 inti_gmres_stats* stats) {
  if (nterms < 1 || !ops) throw Error(INTI_E_ARG, "GMRES needs at least one operator");
  if (!b || !x) throw Error(INTI_E_ARG, "b/x NULL");
  if (!(rtol > 0)) throw Error(INTI_E_ARG, "rtol must be positive");
  if (restart < 1 || maxiter < 1) throw Error(INTI_E_ARG, "restart and maxiter must be >= 1");
  if (mode != INTI_GMRES_FP64 && mode != INTI_GMRES_MIXED) throw Error(INTI_E_ARG, "unknown GMRES mode");
  // the reported time covers the whole call, operator set-up included
  const auto t_enter = std::chrono::steady_clock::now();
  Solver S;
  S.ctx = ctx;
  const inti_quad* q = nullptr;
  bool cpx = false;
  for (int t = 0; t < nterms; ++t) {
    inti_op* op = ops[t];
    if (!op) throw Error(INTI_E_ARG, "operator is NULL");
    if (op->ctx != ctx) throw Error(INTI_E_STATE, "operator belongs to another context");
    if (op->precision != INTI_FP64) throw Error(INTI_E_ARG, "GMRES takes FP64 operators (MIXED builds its FP32C twins)");
    if (op->shard_n > 1) throw Error(INTI_E_STATE, "GMRES takes whole operators, not item shards");
    if (op->target->n != op->source->n) throw Error(INTI_E_SHAPE, "operators must be square");
    if (!q) q = op->source;
    if (op->source->n != q->n) throw Error(INTI_E_SHAPE, "operators differ in size");
    if (op->pde == INTI_HELMHOLTZ) cpx = true;
    S.ops64.push_back(op);
    const cplx c = coefs ? cplx(coefs[2 * t], coefs[2 * t + 1]) : cplx(1, 0);
    if (c.imag() != 0.0) cpx = true;
    S.coefs.push_back(c);
  }
  const auto t_fuse = std::chrono::steady_clock::now();
  // Fuse a double-layer and a single-layer term over the same nodes into one
  // combined-field operator: one pass over the pairs per Krylov step.  The
  // fused operator is kept on the double layer for later solves with the
  // same single layer and coefficients.
  for (size_t a = 0; a < S.ops64.size(); ++a) {
    if (S.ops64[a]->kind != INTI_DL || S.ops64[a]->dim != 3) continue;
    for (size_t b = 0; b < S.ops64.size(); ++b) {
      inti_op *D = S.ops64[a], *Sl = S.ops64[b];
      if (b == a || Sl->kind != INTI_SL || Sl->pde != D->pde || Sl->k != D->k || Sl->target != D->target ||
          Sl->source != D->source)
        continue;
      const double cd[2] = {S.coefs[a].real(), S.coefs[a].imag()};
      const double cs[2] = {S.coefs[b].real(), S.coefs[b].imag()};
      if (D->pde == INTI_LAPLACE && (cd[1] != 0.0 || cs[1] != 0.0)) continue;
      const double key[4] = {cd[0], cd[1], cs[0], cs[1]};
      if (!D->fused || D->fused_sl != Sl->id || !std::equal(key, key + 4, D->fused_c)) {
        D->fused.reset();
        D->fused.reset(op_create_combined(ctx, D->pde, D->k, 0.0, D->target, D->source, D->corr, Sl->corr,
                                          cd, cs, INTI_FP64));
        D->fused_sl = Sl->id;
        std::copy(key, key + 4, D->fused_c);
      }
      S.ops64[a] = D->fused.get();
      S.coefs[a] = cplx(1, 0);
      S.ops64.erase(S.ops64.begin() + b);
      S.coefs.erase(S.coefs.begin() + b);
      break;
    }
  }
  double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_fuse).count();
  S.shift = shift ? cplx(shift[0], shift[1]) : cplx(0, 0);
  if (S.shift.imag() != 0.0) cpx = true;
  for (auto* op : S.ops64)
    if (cpx && op->pde == INTI_LAPLACE)
      throw Error(INTI_E_UNSUPPORTED, "complex coefficients with real (Laplace) operators are not supported");
  S.C = cpx;
  S.comps = cpx ? 2 : 1;
  S.n = q->n;
  S.nblk = std::max(1, std::min<int>(ctx->num_sms * 2, (int)((S.n + kDotBlock - 1) / kDotBlock)));
  if (mode == INTI_GMRES_MIXED) {
    // FP32C twins, made once per operator.  A twin takes the launch shape
    // timed for an FP32C operator of the same kind and size, if one was
    // created on this context, else the heuristic one: timing the candidate
    // shapes here (a dozen launches) costs more than it saves in one solve.
    const auto t_twin = std::chrono::steady_clock::now();
    for (auto* op : S.ops64) {
      if (!op->twin32) op->twin32.reset(op_clone_precision(op, INTI_FP32C));
      S.ops32.push_back(op->twin32.get());
    }
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    setup_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t_twin).count();
  }
  const size_t bytes = sizeof(double) * S.comps * S.n;
  DevBuf& bd = ctx->krylov.b;
  DevBuf& xd = ctx->krylov.x;
  DevBuf& rd = ctx->krylov.r;
  DevBuf& ed = ctx->krylov.e;
  const double* bdev = b;
  double* xdev = x;
  if (!on_device) {
    bd.ensure(bytes);
    xd.ensure(bytes);
    INTI_CUDA(cudaMemcpyAsync(bd.p, b, bytes, cudaMemcpyHostToDevice, ctx->stream));
    INTI_CUDA(cudaMemcpyAsync(xd.p, x, bytes, cudaMemcpyHostToDevice, ctx->stream));
    bdev = bd.as<double>();
    xdev = xd.as<double>();
  }
  const double bn = S.norm(bdev);
  if (history) history[0] = 1.0;
  int iters = 0, outer = 0;
  double relres = 0.0;
  if (bn == 0.0) {
    S.launch_axpby(cplx(0, 0), bdev, cplx(0, 0), xdev);
    relres = 0.0;
  } else if (mode == INTI_GMRES_FP64) {
    double est = 0.0;
    const bool x0 = S.norm(xdev) == 0.0;
    iters = S.gmres(false, bdev, xdev, rtol * bn, restart, maxiter, bn, history, 0, &est, x0, true);
    relres = est / bn;
    outer = 1;
  } else {
    // refinement: r = b - L64 x, solve L32 e = r, x += e
    double* r = S.vec(rd);
    double* e = S.vec(ed);
    double* w = S.vec(ctx->krylov.w_outer);
    constexpr double kInnerRtol = 1.0e-5;  // FP32C operator resolves ~1e-6..1e-7
    const int max_outer = 20;
    if (S.norm(xdev) == 0.0) {
      S.launch_axpby(cplx(1, 0), bdev, cplx(0, 0), r);
    } else {
      S.apply(false, xdev, w);
      S.launch_axpby(cplx(1, 0), bdev, cplx(0, 0), r);
      S.launch_axpby(cplx(-1, 0), w, cplx(1, 0), r);
    }
    double rn = S.norm(r);
    relres = rn / bn;
    while (relres > rtol && iters < maxiter && outer < max_outer) {
      const double inner_tol = std::max(kInnerRtol * rn, 0.5 * rtol * bn);
      double est = 0.0;
      const int used = S.gmres(true, r, e, inner_tol, restart, maxiter - iters, bn, history, iters, &est, true, false);
      iters += used;
      S.launch_axpby(cplx(1, 0), e, cplx(1, 0), xdev);
      S.apply(false, xdev, w);
      S.launch_axpby(cplx(1, 0), bdev, cplx(0, 0), r);
      S.launch_axpby(cplx(-1, 0), w, cplx(1, 0), r);
      const double rn_new = S.norm(r);
      ++outer;
      if (history) history[iters] = rn_new / bn;
      if (used == 0 || rn_new >= rn) {  // stagnation: no further progress possible
        rn = rn_new;
        relres = rn / bn;
        break;
      }
      rn = rn_new;
      relres = rn / bn;
    }
  }
  if (!on_device) INTI_CUDA(cudaMemcpyAsync(x, xdev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  const double wall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_enter).count();
  if (stats) {
    stats->iterations = iters;
    stats->outer = outer;
    stats->fp64_applies = S.fp64_applies;
    stats->fp32_applies = S.fp32_applies;
    stats->converged = relres <= rtol ? 1 : 0;
    stats->reserved = 0;
    stats->relres = relres;
    stats->seconds = wall_s;
    stats->setup_seconds = setup_s;
  }
}

}  // namespace inti
