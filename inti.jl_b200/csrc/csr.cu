// Sparse correction apply y = alpha*C*x + beta*y, the GPU replacement of
// SparseMatrixCSC * Vector inside LinearMap(Smat) + LinearMap(δS)
// (src/api.jl:179-184) and of axpy!(true, δS, Smat) (src/api.jl:171-173).
//
// HBM-bound.  Short rows (the DIM patterns: nq = 5..9 per row) use a
// row-block ("CSR-stream", Greathouse & Daga, SC'14) kernel: a CTA owns R
// consecutive rows, whose nonzeros are one contiguous range; all threads
// stream that range with coalesced loads, multiply by the gathered x and
// park the products in shared memory, then one thread per row sums its
// segment in order.  A block whose range overflows shared memory falls back
// to one warp per row.  Long rows use G lanes per row (G a power of two)
// with a shuffle reduction.  Every sum has a fixed order (deterministic).
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

constexpr int kStreamThreads = 256;
constexpr int kStreamBytes = 32768;  // products parked per CTA

template <bool CPLX>
__device__ __forceinline__ void csr_finish(int64_t row, double sr, double si, double* __restrict__ y,
                                           double ar, double ai, double br, double bi, bool beta_zero) {
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

template <bool CPLX>
__global__ void __launch_bounds__(kStreamThreads) csr_stream_kernel(
    int64_t m, int rows_per_block, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
    const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y, double ar,
    double ai, double br, double bi, bool beta_zero) {
  constexpr int CAP = kStreamBytes / (CPLX ? 16 : 8);
  __shared__ __align__(16) double prod[kStreamBytes / 8];
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = r0 + rows_per_block < m ? r0 + rows_per_block : m;
  const int64_t p0 = rowptr[r0], p1 = rowptr[r1];
  const int tid = threadIdx.x;
  if (p1 - p0 <= CAP) {
    for (int64_t p = p0 + tid; p < p1; p += kStreamThreads) {
      const int32_t j = __ldg(col + p);
      if (CPLX) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(val) + p);
        const double2 xv = __ldg(reinterpret_cast<const double2*>(x) + j);
        reinterpret_cast<double2*>(prod)[p - p0] =
            make_double2(fma(v.x, xv.x, -v.y * xv.y), fma(v.x, xv.y, v.y * xv.x));
      } else {
        prod[p - p0] = __ldg(val + p) * __ldg(x + j);
      }
    }
    __syncthreads();
    for (int64_t row = r0 + tid; row < r1; row += kStreamThreads) {
      const int a = (int)(rowptr[row] - p0), b = (int)(rowptr[row + 1] - p0);
      double sr = 0.0, si = 0.0;
      for (int q = a; q < b; ++q) {
        if (CPLX) {
          const double2 v = reinterpret_cast<const double2*>(prod)[q];
          sr += v.x;
          si += v.y;
        } else {
          sr += prod[q];
        }
      }
      csr_finish<CPLX>(row, sr, si, y, ar, ai, br, bi, beta_zero);
    }
    return;
  }
  // overflow: one warp per row, lanes striding the row, shuffle reduction
  const int warp = tid >> 5, lane = tid & 31;
  for (int64_t row = r0 + warp; row < r1; row += kStreamThreads / 32) {
    double sr = 0.0, si = 0.0;
    for (int64_t p = rowptr[row] + lane; p < rowptr[row + 1]; p += 32) {
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
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      if (CPLX) si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) csr_finish<CPLX>(row, sr, si, y, ar, ai, br, bi, beta_zero);
  }
}

// Bulk-staged row blocks, the form used for short rows: as csr_stream_kernel
// a CTA owns a block of rows whose nonzeros are one contiguous range
// [p0, p1), but the range's values and column indices are brought into
// shared memory by the bulk-copy (TMA) engine: one elected thread issues two
// cp.async.bulk copies of the 16-byte-aligned interiors, completing on one
// mbarrier, so the whole range is in flight at once instead of one load per
// thread.  The unaligned head and tail (< 16 bytes of each array) are plain
// loads.  Shared-memory slots are offset so that the interiors land 16-byte
// aligned: element p sits at vals[p - (p0 & ~(16/VB - 1))] and
// cols[p - (p0 & ~3)].  Then each thread forms products with the gathered x
// in place, and one thread per row sums its segment in order.  A range
// longer than the buffers takes the warp-per-row path.  The wait is bounded:
// on a timeout the CTA records the error, waits once more for its copies
// and leaves.
constexpr int kBulkThreads = 256;
// nonzeros staged per CTA (about 31 KB of shared memory either way, so that
// seven or eight CTAs fit on an SM)
template <bool CPLX>
constexpr int bulk_nnz() {
  return CPLX ? 1536 : 2560;
}

template <bool CPLX>
constexpr size_t csr_bulk_smem() {
  return (size_t)(bulk_nnz<CPLX>() + 2) * (CPLX ? 16 : 8) + (size_t)(bulk_nnz<CPLX>() + 4) * 4;
}

template <bool CPLX>
__global__ void __launch_bounds__(kBulkThreads) csr_bulk_kernel(
    int64_t m, int rows_per_block, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
    const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y, double ar,
    double ai, double br, double bi, bool beta_zero, int* err) {
  constexpr int VB = CPLX ? 16 : 8;   // bytes per value
  constexpr int VA = 16 / VB;          // values per 16 bytes
  constexpr int kBulkNnz = bulk_nnz<CPLX>();
  extern __shared__ __align__(16) unsigned char csm[];
  double* sval = reinterpret_cast<double*>(csm);
  int32_t* scol = reinterpret_cast<int32_t*>(csm + (size_t)(kBulkNnz + 2) * VB);
  __shared__ __align__(8) uint64_t bar;
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_block;
  const int64_t r1 = r0 + rows_per_block < m ? r0 + rows_per_block : m;
  const int64_t p0 = rowptr[r0], p1 = rowptr[r1];
  const int tid = threadIdx.x;
  if (p1 - p0 <= kBulkNnz) {
    // 32-bit offsets within the block: element p0 + q sits at vals[q + lv],
    // cols[q + lc]; the aligned interiors are q in [va, vb) and [ca, cb)
    const int cnt = (int)(p1 - p0);
    const int lv = (int)(p0 & (VA - 1)), lc = (int)(p0 & 3);
    const int va = (VA - lv) & (VA - 1), vb = cnt - (int)((p0 + cnt) & (VA - 1));
    const int ca = (4 - lc) & 3, cb = cnt - (int)((p0 + cnt) & 3);
    const uint32_t vbytes = vb > va ? (uint32_t)(vb - va) * VB : 0u;
    const uint32_t cbytes = cb > ca ? (uint32_t)(cb - ca) * 4u : 0u;
    const bool bulk = vbytes + cbytes > 0;
    if (tid == 0 && bulk) {
      mbar_init(&bar, 1);
      mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0 && bulk) {
      mbar_arrive_expect_tx(&bar, vbytes + cbytes);
      if (vbytes)
        bulk_copy_g2s(reinterpret_cast<unsigned char*>(sval) + (size_t)(va + lv) * VB,
                      reinterpret_cast<const unsigned char*>(val + (p0 + va) * (VB / 8)), vbytes, &bar);
      if (cbytes) bulk_copy_g2s(scol + ca + lc, col + p0 + ca, cbytes, &bar);
    }
    // heads and tails outside the aligned interiors (fewer than 16 bytes each)
    if (tid < 16) {
      const int q = tid < 8 ? tid : cnt - 16 + tid;  // the first and the last 8 elements
      if (q >= 0 && q < cnt && !(tid >= 8 && q < 8)) {
        if (q < va || q >= vb || vb <= va) {
          if (CPLX)
            reinterpret_cast<double2*>(sval)[q + lv] = reinterpret_cast<const double2*>(val)[p0 + q];
          else
            sval[q + lv] = val[p0 + q];
        }
        if (q < ca || q >= cb || cb <= ca) scol[q + lc] = col[p0 + q];
      }
    }
    if (bulk) {
      const bool ok = mbar_wait_bounded(&bar, 0);
      if (!__syncthreads_and(ok)) {
        if (tid == 0) {
          atomicExch(err, kErrWaitTimeout);
          mbar_wait_bounded(&bar, 0);
        }
        return;
      }
    } else {
      __syncthreads();
    }
    // products in place, in chunks: the thread's column indices first, then
    // their gathers of x (in flight together), then the products
    constexpr int PER = 5;
    for (int base = tid; base < cnt; base += PER * kBulkThreads) {
      int32_t js[PER];
#pragma unroll
      for (int u = 0; u < PER; ++u) {
        const int q = base + u * kBulkThreads;
        js[u] = q < cnt ? scol[q + lc] : 0;
      }
      if (CPLX) {
        double2 xs[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int q = base + u * kBulkThreads;
          xs[u] = q < cnt ? __ldg(reinterpret_cast<const double2*>(x) + js[u]) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int q = base + u * kBulkThreads;
          if (q < cnt) {
            double2* v = reinterpret_cast<double2*>(sval) + (q + lv);
            const double2 w = *v;
            *v = make_double2(fma(w.x, xs[u].x, -w.y * xs[u].y), fma(w.x, xs[u].y, w.y * xs[u].x));
          }
        }
      } else {
        double xs[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int q = base + u * kBulkThreads;
          xs[u] = q < cnt ? __ldg(x + js[u]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int q = base + u * kBulkThreads;
          if (q < cnt) sval[q + lv] *= xs[u];
        }
      }
    }
    __syncthreads();
    for (int64_t row = r0 + tid; row < r1; row += kBulkThreads) {
      const int qa = (int)(rowptr[row] - p0) + lv, qb = (int)(rowptr[row + 1] - p0) + lv;
      double sr = 0.0, si = 0.0;
      for (int q = qa; q < qb; ++q) {
        if (CPLX) {
          const double2 v = reinterpret_cast<const double2*>(sval)[q];
          sr += v.x;
          si += v.y;
        } else {
          sr += sval[q];
        }
      }
      csr_finish<CPLX>(row, sr, si, y, ar, ai, br, bi, beta_zero);
    }
    return;
  }
  // overflow: one warp per row, lanes striding the row, shuffle reduction
  const int warp = tid >> 5, lane = tid & 31;
  for (int64_t row = r0 + warp; row < r1; row += kBulkThreads / 32) {
    double sr = 0.0, si = 0.0;
    for (int64_t p = rowptr[row] + lane; p < rowptr[row + 1]; p += 32) {
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
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, o);
      if (CPLX) si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) csr_finish<CPLX>(row, sr, si, y, ar, ai, br, bi, beta_zero);
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
  const bool cplx = c->dtype == INTI_C128;
  if (mean <= 64) {
    // rows per CTA: fill ~90% of the staging buffers at the mean row length
    const int cap = cplx ? bulk_nnz<true>() : bulk_nnz<false>();
    const int rpb = (int)std::max<double>(1.0, std::min<double>(kBulkThreads, 0.9 * cap / std::max(mean, 1.0)));
    const unsigned grid = (unsigned)((c->m + rpb - 1) / rpb);
    int* err = ctx->err_flag.as<int>();
    ctx->flag_armed = true;
    if (cplx) {
      const size_t sm = csr_bulk_smem<true>();
      INTI_CUDA(cudaFuncSetAttribute(&csr_bulk_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      csr_bulk_kernel<true><<<grid, kBulkThreads, sm, ctx->stream>>>(
          c->m, rpb, c->rowptr.as<int64_t>(), c->col.as<int32_t>(), c->val.as<double>(), x, y, ar, ai, br, bi, bz,
          err);
    } else {
      const size_t sm = csr_bulk_smem<false>();
      INTI_CUDA(cudaFuncSetAttribute(&csr_bulk_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      csr_bulk_kernel<false><<<grid, kBulkThreads, sm, ctx->stream>>>(
          c->m, rpb, c->rowptr.as<int64_t>(), c->col.as<int32_t>(), c->val.as<double>(), x, y, ar, ai, br, bi, bz,
          err);
    }
  } else {
    csr_go<32>(ctx, c, x, y, ar, ai, br, bi, bz);
  }
  INTI_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return 1;
}

}  // namespace inti
