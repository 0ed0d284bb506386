// Hand-written adjoint of the Laplace layer-potential product
// u_i = sum_j K(x_i; y_j, n_j) w_j sigma_j (src/nystrom.jl:31-38, the
// IntegralPotential evaluation; the reference has no derivative of it).
//
// Given the cotangent g_i = dJ/du_i, one pass over all (target, source) pairs
// recomputes the kernel tiles (nothing m x n is stored) and accumulates, per
// source node j:
//   s_j  = sum_i g_i K_ij                       -> dJ/dsigma_j = w_j s_j,
//                                                  dJ/dw_j     = sigma_j s_j
//   a_j  = sum_i g_i dK_ij/dn_j                  -> dJ/dn_j = w_j sigma_j a_j
//   b_j  = sum_i g_i dK_ij/dy_j                  -> dJ/dy_j = w_j sigma_j b_j
// with, for r = x - y, d = |r|:
//   SL 3D: K = 1/(4 pi d)           dK/dy = r/(4 pi d^3)
//   DL 3D: K = (r.n)/(4 pi d^3)     dK/dn = r/(4 pi d^3),
//                                   dK/dy = (-n/d^3 + 3 (r.n) r/d^5)/(4 pi)
//   SL 2D: K = -log(d)/(2 pi)       dK/dy = r/(2 pi d^2)
//   DL 2D: K = (r.n)/(2 pi d^2)     dK/dn = r/(2 pi d^2),
//                                   dK/dy = (-n/d^2 + 2 (r.n) r/d^4)/(2 pi)
// Self pairs (|r| <= 1e-14) contribute nothing, as in the forward operator.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"
#include "device_common.cuh"
#include "internal.h"

namespace inti {

constexpr int kAdjBlock = 128;
constexpr int kAdjTile = 128;
constexpr int kAdjSpt = 2;  // sources per thread: each staged target serves two pairs

// partial layout per (split, source): [s, a_0..a_{D-1}, b_0..b_{D-1}, pad]
template <int KIND, int DIM, int SPT>
__global__ void __launch_bounds__(kAdjBlock) adjoint_sources(
    int64_t m, int64_t n, const double* __restrict__ tx, const double* __restrict__ g,
    const double* __restrict__ sx, const double* __restrict__ sn, int tiles_per_split,
    double* __restrict__ partial) {
  constexpr int W = 2 * DIM + 2;
  __shared__ double stx[kAdjTile * DIM], sg[kAdjTile];
  const int64_t j0 = blockIdx.x * (int64_t)(kAdjBlock * SPT) + threadIdx.x;
  double y[SPT][DIM], ny[SPT][DIM];
  // DL: the source's own normal factors out of two sums, accumulated as
  // scalars and applied at the end: s = n_y . a, and b = P*h - n_y*G with
  // h = sum g K' r (P = 3 in 3D, 2 in 2D) and G = sum g K'
  double s[SPT], G[SPT], a[SPT][DIM], b[SPT][DIM];
#pragma unroll
  for (int u = 0; u < SPT; ++u) {
    const int64_t jj = min(j0 + u * kAdjBlock, n - 1);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      y[u][c] = sx[DIM * jj + c];
      ny[u][c] = KIND == DL ? sn[DIM * jj + c] : 0.0;
      a[u][c] = b[u][c] = 0.0;
    }
    s[u] = G[u] = 0.0;
  }
  const int64_t ntile = (m + kAdjTile - 1) / kAdjTile;
  const int64_t t0 = (int64_t)blockIdx.y * tiles_per_split;
  const int64_t t1 = min(ntile, t0 + tiles_per_split);
  for (int64_t t = t0; t < t1; ++t) {
    __syncthreads();
    for (int q = threadIdx.x; q < kAdjTile; q += kAdjBlock) {
      const int64_t i = t * kAdjTile + q;
      const bool in = i < m;
#pragma unroll
      for (int c = 0; c < DIM; ++c) stx[q * DIM + c] = in ? tx[DIM * i + c] : 0.0;
      sg[q] = in ? g[i] : 0.0;
    }
    __syncthreads();
#pragma unroll 2
    for (int q = 0; q < kAdjTile; ++q) {
      double xt[DIM];
#pragma unroll
      for (int c = 0; c < DIM; ++c) xt[c] = stx[q * DIM + c];
      const double gi = sg[q];
#pragma unroll
      for (int u = 0; u < SPT; ++u) {
        double r[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) r[c] = xt[c] - y[u][c];
        double d2 = r[0] * r[0];
#pragma unroll
        for (int c = 1; c < DIM; ++c) d2 = fma(r[c], r[c], d2);
        const bool keep = pair_keep(d2);  // the self pair adds zero to every sum
        if (DIM == 3) {
          const double ri = keep ? rsqrt_fast(d2) : 0.0;
          const double ri3 = ri * ri * ri;
          if (KIND == SL) {
            s[u] = fma(gi, ri, s[u]);
#pragma unroll
            for (int c = 0; c < DIM; ++c) b[u][c] = fma(gi * ri3, r[c], b[u][c]);
          } else {
            double rn = r[0] * ny[u][0];
#pragma unroll
            for (int c = 1; c < DIM; ++c) rn = fma(r[c], ny[u][c], rn);
            const double gr3 = gi * ri3;
            G[u] += gr3;
            const double h = gr3 * rn * (ri * ri);
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
              a[u][c] = fma(gr3, r[c], a[u][c]);
              b[u][c] = fma(h, r[c], b[u][c]);
            }
          }
        } else {
          const double id2 = keep ? rcp_fast(d2) : 0.0;
          if (KIND == SL) {
            s[u] = fma(gi, keep ? log(d2) : 0.0, s[u]);  // scaled by -1/(4 pi) at the end
#pragma unroll
            for (int c = 0; c < DIM; ++c) b[u][c] = fma(gi * id2, r[c], b[u][c]);
          } else {
            double rn = r[0] * ny[u][0];
#pragma unroll
            for (int c = 1; c < DIM; ++c) rn = fma(r[c], ny[u][c], rn);
            const double gd = gi * id2;
            G[u] += gd;
            const double h = gd * rn * id2;
#pragma unroll
            for (int c = 0; c < DIM; ++c) {
              a[u][c] = fma(gd, r[c], a[u][c]);
              b[u][c] = fma(h, r[c], b[u][c]);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int u = 0; u < SPT; ++u) {
    if (KIND == DL) {
      constexpr double P = DIM == 3 ? 3.0 : 2.0;
      s[u] = a[u][0] * ny[u][0];
#pragma unroll
      for (int c = 1; c < DIM; ++c) s[u] = fma(a[u][c], ny[u][c], s[u]);
#pragma unroll
      for (int c = 0; c < DIM; ++c) b[u][c] = fma(P, b[u][c], -G[u] * ny[u][c]);
    }
    const int64_t j = j0 + u * kAdjBlock;
    if (j < n) {
      double* o = partial + ((int64_t)blockIdx.y * n + j) * W;
      o[0] = s[u];
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        o[1 + c] = a[u][c];
        o[1 + DIM + c] = b[u][c];
      }
    }
  }
}

template <int KIND, int DIM>
__global__ void adjoint_reduce(int64_t n, int split, const double* __restrict__ partial,
                               const double* __restrict__ w, const double* __restrict__ sigma,
                               double* dsigma, double* dcoords, double* dnormals, double* dweights) {
  constexpr int W = 2 * DIM + 2;
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double acc[W - 1];
#pragma unroll
  for (int c = 0; c < W - 1; ++c) acc[c] = 0.0;
  for (int s = 0; s < split; ++s) {
    const double* p = partial + ((int64_t)s * n + j) * W;
#pragma unroll
    for (int c = 0; c < W - 1; ++c) acc[c] += p[c];
  }
  const double c0 = DIM == 3 ? 1.0 / (4 * kPi) : 1.0 / (2 * kPi);
  // SL 2D value term is log(d^2) = 2 log(d): K = -log(d)/(2 pi) = -log(d^2)/(4 pi)
  const double cs = (DIM == 2 && KIND == SL) ? -1.0 / (4 * kPi) : c0;
  const double sv = cs * acc[0];
  const double wj = w[j], sj = sigma[j];
  if (dsigma) dsigma[j] = wj * sv;
  if (dweights) dweights[j] = sj * sv;
  const double ws = wj * sj * c0;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    if (dnormals) dnormals[DIM * j + c] = KIND == DL ? ws * acc[1 + c] : 0.0;
    if (dcoords) dcoords[DIM * j + c] = ws * acc[1 + DIM + c];
  }
}

void grad_sources(inti_op* op, const double* g, const double* sigma, double* dsigma,
                  double* dcoords, double* dnormals, double* dweights, int on_device) {
  inti_ctx* ctx = op->ctx;
  if (op->pde != INTI_LAPLACE || (op->kind != INTI_SL && op->kind != INTI_DL))
    throw Error(INTI_E_UNSUPPORTED, "source gradients are implemented for Laplace SL/DL");
  if (op->precision != INTI_FP64) throw Error(INTI_E_ARG, "source gradients need an FP64 operator");
  if (!g || !sigma) throw Error(INTI_E_ARG, "g/sigma NULL");
  const int64_t m = op->target->n, n = op->source->n;
  const int dim = op->dim;
  DevBuf gd, sd, o_s, o_c, o_n, o_w;
  const double* G = g;
  const double* SG = sigma;
  double *DS = dsigma, *DC = dcoords, *DN = dnormals, *DW = dweights;
  if (!on_device) {
    gd.ensure(sizeof(double) * m);
    sd.ensure(sizeof(double) * n);
    INTI_CUDA(cudaMemcpyAsync(gd.p, g, sizeof(double) * m, cudaMemcpyHostToDevice, ctx->stream));
    INTI_CUDA(cudaMemcpyAsync(sd.p, sigma, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    G = gd.as<double>();
    SG = sd.as<double>();
    if (dsigma) { o_s.ensure(sizeof(double) * n); DS = o_s.as<double>(); }
    if (dcoords) { o_c.ensure(sizeof(double) * dim * n); DC = o_c.as<double>(); }
    if (dnormals) { o_n.ensure(sizeof(double) * dim * n); DN = o_n.as<double>(); }
    if (dweights) { o_w.ensure(sizeof(double) * n); DW = o_w.as<double>(); }
  }
  const int64_t blocks = (n + kAdjBlock * kAdjSpt - 1) / (kAdjBlock * kAdjSpt);
  const int64_t ntile = (m + kAdjTile - 1) / kAdjTile;
  const int64_t want = (int64_t)ctx->num_sms * 8;
  int split = (int)std::max<int64_t>(1, std::min<int64_t>(ntile, (want + blocks - 1) / blocks));
  const int tps = (int)((ntile + split - 1) / split);
  split = (int)((ntile + tps - 1) / tps);
  const int W = 2 * dim + 2;
  op->gpartial.ensure(sizeof(double) * (size_t)split * n * W);
  double* part = op->gpartial.as<double>();
  const double* TX = op->target->coords.as<double>();
  const double* SX = op->source->coords.as<double>();
  const double* SN = op->source->has_normals ? op->source->normals.as<double>() : nullptr;
  const double* SW = op->source->weights.as<double>();
  auto go = [&](auto kind_c, auto dim_c) {
    constexpr int K = decltype(kind_c)::value;
    constexpr int D = decltype(dim_c)::value;
    {
      ProfScope pa(ctx, "adjoint");
      adjoint_sources<K, D, kAdjSpt><<<dim3((unsigned)blocks, (unsigned)split), kAdjBlock, 0, ctx->stream>>>(
          m, n, TX, G, SX, SN, tps, part);
    }
    adjoint_reduce<K, D><<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
        n, split, part, SW, SG, DS, DC, DN, DW);
    ctx->launches += 2;
  };
  if (dim == 3 && op->kind == INTI_SL) go(std::integral_constant<int, SL>(), std::integral_constant<int, 3>());
  else if (dim == 3) go(std::integral_constant<int, DL>(), std::integral_constant<int, 3>());
  else if (op->kind == INTI_SL) go(std::integral_constant<int, SL>(), std::integral_constant<int, 2>());
  else go(std::integral_constant<int, DL>(), std::integral_constant<int, 2>());
  INTI_CUDA(cudaGetLastError());
  if (!on_device) {
    if (dsigma) INTI_CUDA(cudaMemcpyAsync(dsigma, DS, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    if (dcoords) INTI_CUDA(cudaMemcpyAsync(dcoords, DC, sizeof(double) * dim * n, cudaMemcpyDeviceToHost, ctx->stream));
    if (dnormals) INTI_CUDA(cudaMemcpyAsync(dnormals, DN, sizeof(double) * dim * n, cudaMemcpyDeviceToHost, ctx->stream));
    if (dweights) INTI_CUDA(cudaMemcpyAsync(dweights, DW, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
  }
}

}  // namespace inti
