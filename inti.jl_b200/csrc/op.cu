// Operator handles: validation of the (pde, kernel, target, source,
// correction) combination that IntegralOperator/single_double_layer accept
// (src/nystrom.jl:79-89, src/api.jl:65-78) and sizing of the operator's
// scratch buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "common.h"
#include "device_common.cuh"
#include "internal.h"

namespace inti {

static void req(bool c, int code, const std::string& m) {
  if (!c) throw Error(code, m);
}

inti_op* op_create(inti_ctx* ctx, int pde, int kernel, double k_re, double k_im,
                   const inti_quad* target, const inti_quad* source, const inti_csr* correction,
                   int precision) {
  req(target && source, INTI_E_ARG, "target/source quadrature is NULL");
  req(target->ctx == ctx && source->ctx == ctx, INTI_E_STATE, "quadrature belongs to another context");
  req(pde == INTI_LAPLACE || pde == INTI_HELMHOLTZ, INTI_E_ARG, "unknown pde");
  req(kernel >= INTI_SL && kernel <= INTI_HS, INTI_E_ARG, "unknown kernel");
  req(precision == INTI_FP64 || precision == INTI_FP32C, INTI_E_ARG, "unknown precision");
  req(target->dim == source->dim, INTI_E_SHAPE, "target and source dimensions differ");
  const int dim = source->dim;
  if (pde == INTI_HELMHOLTZ) {
    req(dim == 3, INTI_E_UNSUPPORTED, "Helmholtz is implemented in 3D only");
    req(k_im == 0.0, INTI_E_UNSUPPORTED, "complex wavenumbers are not implemented");
    req(std::isfinite(k_re), INTI_E_NONFINITE, "wavenumber is not finite");
  }
  if (kernel == INTI_DL || kernel == INTI_HS)
    req(source->has_normals, INTI_E_ARG, "double-layer/hypersingular kernels need source normals");
  if (kernel == INTI_ADL || kernel == INTI_HS)
    req(target->has_normals, INTI_E_ARG, "adjoint-double-layer/hypersingular kernels need target normals");
  if (correction) {
    req(correction->ctx == ctx, INTI_E_STATE, "correction belongs to another context");
    req(correction->m == target->n && correction->n == source->n, INTI_E_SHAPE,
        "correction shape does not match (target, source)");
    req(correction->dtype == (pde == INTI_HELMHOLTZ ? INTI_C128 : INTI_F64), INTI_E_ARG,
        "correction dtype must be F64 for Laplace and C128 for Helmholtz");
  }
  std::unique_ptr<inti_op> op(new inti_op());
  op->ctx = ctx;
  op->pde = pde;
  op->kind = kernel;
  op->dim = dim;
  op->precision = precision;
  op->k = k_re;
  op->target = target;
  op->source = source;
  op->corr = correction;
  const int64_t tile = pair_tile(precision);
  op->n_tiles = std::max<int64_t>(1, (source->n + tile - 1) / tile);
  op->split = pair_plan_split(ctx, pde, kernel, dim, precision, target->n, source->n);
  op->packed.ensure((size_t)op->n_tiles * tile * pair_record_bytes(pde, kernel, dim, precision));
  op->partial.ensure((size_t)op->split * target->n * pair_partial_bytes(pde, precision));
  const int comps = pde == INTI_HELMHOLTZ ? 2 : 1;
  const int64_t big = std::max(target->n, source->n);
  op->xbuf.ensure(sizeof(double) * comps * big);
  op->ybuf.ensure(sizeof(double) * comps * big);
  return op.release();
}

void op_prepare_transpose(inti_op* op) {
  const int64_t ntile = (op->target->n + 63) / 64;
  const int64_t blocks = (op->source->n + 127) / 128;
  const int64_t want = (int64_t)op->ctx->num_sms * 8;
  op->tsplit = (int)std::max<int64_t>(1, std::min<int64_t>(ntile, (want + blocks - 1) / blocks));
  op->tpartial.ensure(sizeof(double2) * (size_t)op->tsplit * op->source->n);
  if (op->corr && !op->corrT) op->corrT = csr_transpose(op->ctx, op->corr);
}

__global__ void transpose_epilogue_kernel(int64_t n, int split, const double2* partial,
                                          const int64_t* rowptr, const int32_t* col,
                                          const double* val, const double* x, double* y,
                                          double ar, double ai, double br, double bi, bool bz,
                                          bool cplx) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double sr = 0.0, si = 0.0;
  for (int s = 0; s < split; ++s) {
    const double2 v = partial[(int64_t)s * n + j];
    sr += v.x;
    si += v.y;
  }
  if (rowptr) {
    for (int64_t p = rowptr[j]; p < rowptr[j + 1]; ++p) {
      const int32_t i = col[p];
      if (cplx) {
        const double vr = val[2 * p], vi = val[2 * p + 1];
        const double xr = x[2 * i], xi = x[2 * i + 1];
        sr = fma(vr, xr, fma(-vi, xi, sr));
        si = fma(vr, xi, fma(vi, xr, si));
      } else {
        sr = fma(val[p], x[i], sr);
      }
    }
  }
  if (cplx) {
    double yr = ar * sr - ai * si, yi = ar * si + ai * sr;
    if (!bz) {
      yr += br * y[2 * j] - bi * y[2 * j + 1];
      yi += br * y[2 * j + 1] + bi * y[2 * j];
    }
    y[2 * j] = yr;
    y[2 * j + 1] = yi;
  } else {
    double yr = ar * sr;
    if (!bz) yr += br * y[j];
    y[j] = yr;
  }
}

void transpose_epilogue(inti_ctx* ctx, int64_t n, int split, const void* partial,
                        const inti_csr* corrT, const double* x, double* y, const double* alpha,
                        const double* beta, bool cplx) {
  const double ar = alpha ? alpha[0] : 1.0, ai = alpha ? alpha[1] : 0.0;
  const double br = beta ? beta[0] : 0.0, bi = beta ? beta[1] : 0.0;
  const bool bz = br == 0.0 && bi == 0.0;
  transpose_epilogue_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(
      n, split, static_cast<const double2*>(partial), corrT ? corrT->rowptr.as<int64_t>() : nullptr,
      corrT ? corrT->col.as<int32_t>() : nullptr, corrT ? corrT->val.as<double>() : nullptr, x, y,
      ar, ai, br, bi, bz, cplx);
  INTI_CUDA(cudaGetLastError());
  ctx->launches += 1;
}

}  // namespace inti
