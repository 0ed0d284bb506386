// Sparse correction apply y = alpha*C*x + beta*y, the GPU replacement of
// SparseMatrixCSC * Vector inside LinearMap(Smat) + LinearMap(δS)
// (src/api.jl:179-184) and of axpy!(true, δS, Smat) (src/api.jl:171-173).
//
// HBM-bound: each row is owned by a group of G lanes (G a power of two chosen
// from the mean row length) that read the row's values and column indices
// with coalesced, vectorised loads and reduce with shuffles in a fixed order
// (deterministic).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"
#include "device_common.cuh"

namespace inti {

template <int G, bool CPLX>
__global__ void csr_kernel(int64_t m, const int64_t* __restrict__ rowptr,
                           const int32_t* __restrict__ col, const double* __restrict__ val,
                           const double* __restrict__ x, double* __restrict__ y, double ar,
                           double ai, double br, double bi, bool beta_zero) {
  const int64_t gtid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t row = gtid / G;
  const int lane = threadIdx.x % G;
  const bool active = row < m;
  double sr = 0.0, si = 0.0;
  if (active) {
    const int64_t p0 = rowptr[row], p1 = rowptr[row + 1];
    for (int64_t p = p0 + lane; p < p1; p += G) {
      const int32_t j = __ldg(col + p);
      if (CPLX) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(val) + p);
        const double2 xv = __ldg(reinterpret_cast<const double2*>(x) + j);
        sr = fma(v.x, xv.x, fma(-v.y, xv.y, sr));
        si = fma(v.x, xv.y, fma(v.y, xv.x, si));
      } else {
        sr = fma(__ldg(val + p), __ldg(x + j), sr);
      }
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, o, G);
    if (CPLX) si += __shfl_xor_sync(0xffffffffu, si, o, G);
  }
  if (!active || lane != 0) return;
  if (CPLX) {
    double yr = ar * sr - ai * si, yi = ar * si + ai * sr;
    if (!beta_zero) {
      const double2 yo = reinterpret_cast<const double2*>(y)[row];
      yr += br * yo.x - bi * yo.y;
      yi += br * yo.y + bi * yo.x;
    }
    reinterpret_cast<double2*>(y)[row] = make_double2(yr, yi);
  } else {
    double yr = ar * sr;
    if (!beta_zero) yr += br * y[row];
    y[row] = yr;
  }
}

template <int G>
static void csr_go(inti_ctx* ctx, const inti_csr* c, const double* x, double* y, double ar,
                   double ai, double br, double bi, bool bz) {
  const int tb = 256;
  const int64_t threads = c->m * G;
  const unsigned grid = (unsigned)((threads + tb - 1) / tb);
  if (c->dtype == INTI_C128)
    csr_kernel<G, true><<<grid, tb, 0, ctx->stream>>>(c->m, c->rowptr.as<int64_t>(),
                                                      c->col.as<int32_t>(), c->val.as<double>(),
                                                      x, y, ar, ai, br, bi, bz);
  else
    csr_kernel<G, false><<<grid, tb, 0, ctx->stream>>>(c->m, c->rowptr.as<int64_t>(),
                                                       c->col.as<int32_t>(), c->val.as<double>(),
                                                       x, y, ar, ai, br, bi, bz);
}

int csr_apply(inti_ctx* ctx, const inti_csr* c, const double* x, double* y, const double* alpha,
              const double* beta) {
  if (c->m == 0) return 0;
  const double ar = alpha ? alpha[0] : 1.0, ai = alpha ? alpha[1] : 0.0;
  const double br = beta ? beta[0] : 0.0, bi = beta ? beta[1] : 0.0;
  const bool bz = br == 0.0 && bi == 0.0;
  const double mean = (double)c->nnz / (double)c->m;
  ProfScope pc(ctx, "csr");
  if (mean <= 2)
    csr_go<2>(ctx, c, x, y, ar, ai, br, bi, bz);
  else if (mean <= 6)
    csr_go<4>(ctx, c, x, y, ar, ai, br, bi, bz);
  else if (mean <= 12)
    csr_go<8>(ctx, c, x, y, ar, ai, br, bi, bz);
  else if (mean <= 24)
    csr_go<16>(ctx, c, x, y, ar, ai, br, bi, bz);
  else
    csr_go<32>(ctx, c, x, y, ar, ai, br, bi, bz);
  INTI_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return 1;
}

}  // namespace inti
