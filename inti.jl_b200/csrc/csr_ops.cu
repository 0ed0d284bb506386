// Sparse-correction set-up on the device.
//
// merge_corrections: C = ca*A + cb*B.  The correction of a combined-field
// operator c1*(D + δD) + c2*(S + δS) is c1*δD + c2*δS (src/api.jl:170-185
// keeps them as two LinearMaps; one fused operator needs their sum).  Both
// inputs have strictly increasing columns within a row (checked on upload;
// the DIM builder writes them so), so a row of C is the two-pointer union of
// the two rows.  One thread per row counts the union, a device scan turns
// the counts into row pointers, and a second pass writes the columns and the
// values (ca*a + cb*b where both have the column, in that order).
//
// csr_transpose: C^T for transposed applies.  The keys (column << 32 | row)
// of all nonzeros are radix-sorted with their positions, which orders C^T's
// rows by column and each row by the original row index: the layout a serial
// transpose that walks C row by row produces, so results do not depend on
// scheduling.  The row pointers come from a scan of the column counts.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>

#include "common.h"
#include "internal.h"

namespace inti {

struct MergeIn {
  const int64_t* rp;  // NULL: every row empty
  const int32_t* col;
  const double* val;  // real, or (re, im) pairs
};

__device__ __forceinline__ void merge_row_range(const MergeIn& a, int64_t i, int64_t& p, int64_t& e) {
  if (a.rp) {
    p = a.rp[i];
    e = a.rp[i + 1];
  } else {
    p = e = 0;
  }
}

__global__ void csr_merge_count(int64_t m, MergeIn a, MergeIn b, int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  int64_t pa, ea, pb, eb;
  merge_row_range(a, i, pa, ea);
  merge_row_range(b, i, pb, eb);
  int64_t c = 0;
  while (pa < ea || pb < eb) {
    const int32_t ja = pa < ea ? a.col[pa] : INT_MAX, jb = pb < eb ? b.col[pb] : INT_MAX;
    const int32_t j = ja < jb ? ja : jb;
    pa += ja == j;
    pb += jb == j;
    ++c;
  }
  cnt[i] = c;
}

template <bool CPLX>
__global__ void csr_merge_fill(int64_t m, MergeIn a, double2 ca, MergeIn b, double2 cb,
                               const int64_t* __restrict__ rp, int32_t* __restrict__ col, double* __restrict__ val) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  int64_t pa, ea, pb, eb;
  merge_row_range(a, i, pa, ea);
  merge_row_range(b, i, pb, eb);
  int64_t q = rp[i];
  while (pa < ea || pb < eb) {
    const int32_t ja = pa < ea ? a.col[pa] : INT_MAX, jb = pb < eb ? b.col[pb] : INT_MAX;
    const int32_t j = ja < jb ? ja : jb;
    double vr = 0.0, vi = 0.0;
    if (ja == j) {
      const double ar = CPLX ? a.val[2 * pa] : a.val[pa], ai = CPLX ? a.val[2 * pa + 1] : 0.0;
      vr += ca.x * ar - ca.y * ai;
      vi += ca.x * ai + ca.y * ar;
      ++pa;
    }
    if (jb == j) {
      const double br = CPLX ? b.val[2 * pb] : b.val[pb], bi = CPLX ? b.val[2 * pb + 1] : 0.0;
      vr += cb.x * br - cb.y * bi;
      vi += cb.x * bi + cb.y * br;
      ++pb;
    }
    col[q] = j;
    if (CPLX) {
      val[2 * q] = vr;
      val[2 * q + 1] = vi;
    } else {
      val[q] = vr;
    }
    ++q;
  }
}

std::unique_ptr<inti_csr> merge_corrections(inti_ctx* ctx, const inti_csr* a, const double* ca,
                                            const inti_csr* b, const double* cb, int64_t m, int64_t n,
                                            bool cplx) {
  const int comps = cplx ? 2 : 1;
  for (const inti_csr* c : {a, b})
    if (c) {
      if (c->m != m || c->n != n) throw Error(INTI_E_SHAPE, "correction shape differs from the operator's");
      if ((c->dtype == INTI_C128) != cplx) throw Error(INTI_E_ARG, "correction type differs from the operator's");
    }
  auto in = [](const inti_csr* c) {
    return c ? MergeIn{c->rowptr.as<int64_t>(), c->col.as<int32_t>(), c->val.as<double>()}
             : MergeIn{nullptr, nullptr, nullptr};
  };
  const MergeIn A = in(a), B = in(b);
  std::unique_ptr<inti_csr> out(new inti_csr());
  out->ctx = ctx;
  out->m = m;
  out->n = n;
  out->dtype = cplx ? INTI_C128 : INTI_F64;
  out->rowptr.ensure(sizeof(int64_t) * (m + 1));
  int64_t* rp = out->rowptr.as<int64_t>();
  INTI_CUDA(cudaMemsetAsync(rp, 0, sizeof(int64_t), ctx->stream));
  const unsigned grid = (unsigned)std::max<int64_t>(1, (m + 255) / 256);
  if (m > 0) {
    // counts in rp[1..m], then their inclusive scan in place
    csr_merge_count<<<grid, 256, 0, ctx->stream>>>(m, A, B, rp + 1);
    ctx->launches++;
    size_t tmp = 0;
    INTI_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, rp + 1, rp + 1, m, ctx->stream));
    ctx->scan_tmp.ensure(tmp);
    INTI_CUDA(cub::DeviceScan::InclusiveSum(ctx->scan_tmp.p, tmp, rp + 1, rp + 1, m, ctx->stream));
    ctx->launches++;
  }
  int64_t nnz = 0;
  INTI_CUDA(cudaMemcpyAsync(&nnz, rp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  out->nnz = nnz;
  out->col.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
  out->val.ensure(sizeof(double) * comps * std::max<int64_t>(nnz, 1));
  if (m > 0 && nnz > 0) {
    const double2 dca = make_double2(ca[0], ca[1]), dcb = make_double2(cb[0], cb[1]);
    if (cplx)
      csr_merge_fill<true><<<grid, 256, 0, ctx->stream>>>(m, A, dca, B, dcb, rp, out->col.as<int32_t>(),
                                                          out->val.as<double>());
    else
      csr_merge_fill<false><<<grid, 256, 0, ctx->stream>>>(m, A, dca, B, dcb, rp, out->col.as<int32_t>(),
                                                           out->val.as<double>());
    ctx->launches++;
  }
  INTI_CUDA(cudaGetLastError());
  return out;
}

__global__ void csr_transpose_keys(int64_t m, const int64_t* __restrict__ rp, const int32_t* __restrict__ col,
                                   uint64_t* __restrict__ keys, int64_t* __restrict__ pos,
                                   int* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
    const int32_t j = col[p];
    keys[p] = ((uint64_t)(uint32_t)j << 32) | (uint64_t)(uint32_t)i;
    pos[p] = p;
    atomicAdd(cnt + j, 1);  // counts only: their order does not matter
  }
}

template <bool CPLX>
__global__ void csr_transpose_fill(int64_t nnz, const uint64_t* __restrict__ keys, const int64_t* __restrict__ pos,
                                   const double* __restrict__ val, int32_t* __restrict__ tcol,
                                   double* __restrict__ tval) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= nnz) return;
  tcol[q] = (int32_t)(uint32_t)(keys[q] & 0xffffffffu);
  const int64_t p = pos[q];
  if (CPLX) {
    tval[2 * q] = val[2 * p];
    tval[2 * q + 1] = val[2 * p + 1];
  } else {
    tval[q] = val[p];
  }
}

__global__ void csr_counts_to_i64(int64_t n, const int* __restrict__ cnt, int64_t* __restrict__ out) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) out[j] = cnt[j];
}

std::unique_ptr<inti_csr> csr_transpose(inti_ctx* ctx, const inti_csr* c) {
  const bool cplx = c->dtype == INTI_C128;
  const int comps = cplx ? 2 : 1;
  const int64_t m = c->m, n = c->n, nnz = c->nnz;
  if (m >= ((int64_t)1 << 31) || n >= ((int64_t)1 << 31)) throw Error(INTI_E_ARG, "CSR too large to transpose");
  std::unique_ptr<inti_csr> t(new inti_csr());
  t->ctx = ctx;
  t->m = n;
  t->n = m;
  t->nnz = nnz;
  t->dtype = c->dtype;
  t->rowptr.ensure(sizeof(int64_t) * (n + 1));
  t->col.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
  t->val.ensure(sizeof(double) * comps * std::max<int64_t>(nnz, 1));
  int64_t* trp = t->rowptr.as<int64_t>();
  INTI_CUDA(cudaMemsetAsync(trp, 0, sizeof(int64_t) * (n + 1), ctx->stream));
  if (nnz == 0) {
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    return t;
  }
  // keys, positions (in and out), column counts; the sort's scratch after them
  DevBuf work;
  const size_t kb = sizeof(uint64_t) * nnz, pb = sizeof(int64_t) * nnz, cb = sizeof(int) * n;
  size_t sort_tmp = 0, scan_tmp = 0;
  INTI_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                            (const int64_t*)nullptr, (int64_t*)nullptr, nnz, 0, 64,
                                            ctx->stream));
  INTI_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_tmp, trp + 1, trp + 1, n, ctx->stream));
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  work.ensure(2 * up(kb) + 2 * up(pb) + up(cb) + up(std::max(sort_tmp, scan_tmp)));
  char* w = static_cast<char*>(work.p);
  uint64_t* k_in = reinterpret_cast<uint64_t*>(w);
  uint64_t* k_out = reinterpret_cast<uint64_t*>(w + up(kb));
  int64_t* p_in = reinterpret_cast<int64_t*>(w + 2 * up(kb));
  int64_t* p_out = reinterpret_cast<int64_t*>(w + 2 * up(kb) + up(pb));
  int* cnt = reinterpret_cast<int*>(w + 2 * up(kb) + 2 * up(pb));
  void* tmp = w + 2 * up(kb) + 2 * up(pb) + up(cb);
  INTI_CUDA(cudaMemsetAsync(cnt, 0, cb, ctx->stream));
  csr_transpose_keys<<<(unsigned)((m + 255) / 256), 256, 0, ctx->stream>>>(
      m, c->rowptr.as<int64_t>(), c->col.as<int32_t>(), k_in, p_in, cnt);
  INTI_CUDA(cub::DeviceRadixSort::SortPairs(tmp, sort_tmp, k_in, k_out, p_in, p_out, nnz, 0, 64, ctx->stream));
  csr_counts_to_i64<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, cnt, trp + 1);
  INTI_CUDA(cub::DeviceScan::InclusiveSum(tmp, scan_tmp, trp + 1, trp + 1, n, ctx->stream));
  const unsigned g = (unsigned)((nnz + 255) / 256);
  if (cplx)
    csr_transpose_fill<true><<<g, 256, 0, ctx->stream>>>(nnz, k_out, p_out, c->val.as<double>(),
                                                         t->col.as<int32_t>(), t->val.as<double>());
  else
    csr_transpose_fill<false><<<g, 256, 0, ctx->stream>>>(nnz, k_out, p_out, c->val.as<double>(),
                                                          t->col.as<int32_t>(), t->val.as<double>());
  ctx->launches += 5;
  INTI_CUDA(cudaGetLastError());
  INTI_CUDA(cudaStreamSynchronize(ctx->stream));  // before the work buffer is freed
  return t;
}

}  // namespace inti
