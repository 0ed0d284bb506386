// The C ABI of libinti_b200.so (declared in include/inti_b200.h): handle
// management, argument validation, host<->device staging and the order of
// launches.  No C++ exception crosses this boundary: every entry point
// returns a status and leaves a message for inti_last_error.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "batch.h"
#include "common.h"
#include "internal.h"

using inti::DevBuf;
using inti::Error;

static thread_local std::string g_thread_error;

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) {
      cudaError_t e = cudaSetDevice(dev);
      if (e != cudaSuccess) throw Error(INTI_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <class F>
int guarded(inti_ctx* ctx, F&& f) {
  try {
    if (ctx) {
      std::lock_guard<std::recursive_mutex> lk(ctx->mu);
      DeviceGuard dg(ctx->device);
      f();
      ctx->last_error.clear();
    } else {
      f();
    }
    return INTI_OK;
  } catch (const Error& e) {
    (ctx ? ctx->last_error : g_thread_error) = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    (ctx ? ctx->last_error : g_thread_error) = "host allocation failed";
    return INTI_E_NOMEM;
  } catch (const std::exception& e) {
    (ctx ? ctx->last_error : g_thread_error) = e.what();
    return INTI_E_ARG;
  }
}

void require(bool cond, int code, const std::string& msg) {
  if (!cond) throw Error(code, msg);
}

void check_finite(const double* p, size_t count, const char* what) {
  for (size_t i = 0; i < count; ++i)
    if (!std::isfinite(p[i])) throw Error(INTI_E_NONFINITE, std::string(what) + " contains NaN/Inf");
}

void h2d(inti_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes) INTI_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
}
void d2h(inti_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes) INTI_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
}

}  // namespace

namespace inti {

void noalloc_error_set(const char* msg) { g_thread_error = msg; }

void sync_and_check(inti_ctx* ctx) {
  if (!ctx->flag_armed) {  // nothing enqueued since the last check can have raised the flag
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    return;
  }
  // the flag comes back with the stream's other work: one round trip per call
  INTI_CUDA(cudaMemcpyAsync(ctx->err_host, ctx->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->flag_armed = false;
  const int flag = *ctx->err_host;
  if (flag) {
    *ctx->err_host = 0;
    INTI_CUDA(cudaMemsetAsync(ctx->err_flag.p, 0, sizeof(int), ctx->stream));
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    throw Error(INTI_E_TIMEOUT, "a device-side bounded wait ran out (code " + std::to_string(flag) + ")");
  }
}

// Fill a PairLaunch for op and density x (device pointer).
PairLaunch make_launch(inti_op* op, const double* xdev) {
  PairLaunch L;
  L.pde = op->pde;
  L.kind = op->kind;
  L.dim = op->dim;
  L.precision = op->precision;
  L.k = op->k;
  L.m = op->target->n;
  L.n = op->source->n;
  L.tcoords = op->target->coords.as<double>();
  L.tnormals = op->target->has_normals ? op->target->normals.as<double>() : nullptr;
  L.scoords = op->source->coords.as<double>();
  L.snormals = op->source->has_normals ? op->source->normals.as<double>() : nullptr;
  L.sweights = op->source->weights.as<double>();
  L.x = xdev;
  L.packed = op->packed.p;
  L.partial = op->partial.p;
  L.split = op->split;
  L.tpt = op->tpt;
  L.n_tiles = op->n_tiles;
  L.err_flag = op->ctx->err_flag.as<int>();
  L.c1[0] = op->c1[0];
  L.c1[1] = op->c1[1];
  L.c2[0] = op->c2[0];
  L.c2[1] = op->c2[1];
  if (op->symm) {
    L.symm = true;
    L.sym_nb = op->sym_nb;
    L.sym_nitems = op->sym_nitems;
    L.sym_items = op->sym_tab.as<int32_t>();
    L.sym_rowptr = L.sym_items + 3 * op->sym_nitems;
    L.sym_rowitems = L.sym_rowptr + op->sym_nb + 1;
    L.partial = op->ctx->sym_ypart.p;  // the context's shared symmetric scratch
    L.zpart = op->ctx->sym_zpart.p;
    L.sym_npanels = (int)op->sym_panels.size();
    if (L.sym_npanels > 1) {
      L.sym_panels = op->sym_panels.data();
      L.sym_table = op->sym_tab.as<int32_t>();
      L.sym_zld = op->sym_zld;
      L.sym_acc = op->ctx->sym_acc.p;
      const size_t pb = (size_t)pair_partial_bytes(op->pde, op->precision);
      L.sym_ypart_bytes = pb * op->sym_nitems * pair_symm_block(op->tpt);
      L.sym_zpart_bytes = pb * op->sym_nb * op->sym_zld;
    }
    if (op->shard_n > 1) {
      L.sym_launch_items = op->shard_items;
      L.sym_launch = op->shard_tab.as<int32_t>();
      L.sym_launch_ids = L.sym_launch + 3 * op->shard_items;
      L.sym_launch_panels = op->shard_panels.data();
    }
  }
  return L;
}

// Device-resident apply of one column: y = alpha*(A x + C x) + beta*y.
void op_apply_device(inti_op* op, const double* x, double* y, const double* alpha,
                     const double* beta) {
  PairLaunch L = make_launch(op, x);
  if (op->small && op->shard_n == 1) {
    pair_small(op->ctx, L, op->corr, x, y, alpha, beta);
    return;
  }
  if (op->shard_n > 1) {
    // this rank's items only: the partials of the others' items are zero, and
    // the correction and beta*y belong to rank 0 (the ranks' y are summed)
    // (with panels pair_launch clears them before each panel)
    if (L.sym_npanels <= 1) {
      const size_t pb = (size_t)pair_partial_bytes(op->pde, op->precision);
      INTI_CUDA(cudaMemsetAsync(L.partial, 0, pb * op->sym_nitems * pair_symm_block(op->tpt), op->ctx->stream));
      INTI_CUDA(cudaMemsetAsync(L.zpart, 0, pb * op->sym_nb * op->n_tiles * pair_tile(op->precision),
                                op->ctx->stream));
    }
    pair_launch(op->ctx, L);
    const double zero[2] = {0.0, 0.0};
    const bool lead = op->shard_rank == 0;
    pair_epilogue(op->ctx, L, lead ? op->corr : nullptr, x, y, alpha, lead ? beta : zero);
    return;
  }
  pair_launch(op->ctx, L);
  pair_epilogue(op->ctx, L, op->corr, x, y, alpha, beta);
}

void op_apply_transpose_device(inti_op* op, const double* x, double* y, const double* alpha,
                               const double* beta) {
  if (op->symm && op->small && op->shard_n == 1) {
    // small square operator: the transposed kernel with unit source weights
    // in the single-launch form, row j scaled by w_j, the transposed correction
    PairLaunch L = make_launch(op, x);
    L.kind = transposed_kind(op->kind);
    L.sweights = op->tones.as<double>();
    pair_small(op->ctx, L, op->corrT.get(), x, y, alpha, beta, op->source->weights.as<double>());
    return;
  }
  if (op->symm) {
    // square operator: the symmetric product of the transposed kernel with
    // unit weights on the same node blocks, work items and partial buffers
    PairLaunch L = make_launch(op, x);
    L.kind = transposed_kind(op->kind);
    L.sweights = op->tones.as<double>();
    L.packed = op->tpacked.p;
    {
      ProfScope pt(op->ctx, "transpose");
      pair_launch(op->ctx, L);
    }
    pair_epilogue(op->ctx, L, op->corrT.get(), x, y, alpha, beta, op->source->weights.as<double>());
    return;
  }
  // the forward pair product with targets and sources swapped (op_prepare_transpose)
  PairLaunch L = make_launch(op, x);
  L.kind = transposed_kind(op->kind);
  L.m = op->source->n;
  L.n = op->target->n;
  L.tcoords = op->source->coords.as<double>();
  L.tnormals = op->source->has_normals ? op->source->normals.as<double>() : nullptr;
  L.scoords = op->target->coords.as<double>();
  L.snormals = op->target->has_normals ? op->target->normals.as<double>() : nullptr;
  L.sweights = op->tones.as<double>();
  L.packed = op->tpacked.p;
  L.partial = op->tpartial.p;
  L.split = op->tsplit;
  L.tpt = op->ttpt;
  L.n_tiles = op->tn_tiles;
  {
    ProfScope pt(op->ctx, "transpose");
    pair_launch(op->ctx, L);
  }
  // y = alpha*(w_j * scale * sum partial + C^T x) + beta*y
  pair_epilogue(op->ctx, L, op->corrT.get(), x, y, alpha, beta, op->source->weights.as<double>());
}

}  // namespace inti

// ---------------------------------------------------------------- sparse
namespace {

inti_csr* csr_from_host(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz, const int64_t* rowptr,
                        const int32_t* col, const double* val, int dtype) {
  require(m >= 0 && n >= 0 && nnz >= 0, INTI_E_ARG, "negative CSR size");
  require(dtype == INTI_F64 || dtype == INTI_C128, INTI_E_ARG, "dtype must be F64 or C128");
  require(rowptr != nullptr, INTI_E_ARG, "rowptr is NULL");
  require(nnz == 0 || (col && val), INTI_E_ARG, "col/val are NULL");
  require(nnz < (int64_t)1 << 40, INTI_E_ARG, "nnz too large");
  require(rowptr[0] == 0 && rowptr[m] == nnz, INTI_E_SHAPE, "rowptr must start at 0 and end at nnz");
  for (int64_t i = 0; i < m; ++i) {
    require(rowptr[i + 1] >= rowptr[i], INTI_E_ARG, "rowptr is not non-decreasing");
    for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
      require(col[p] >= 0 && col[p] < n, INTI_E_ARG, "column index out of range");
      require(p == rowptr[i] || col[p] > col[p - 1], INTI_E_ARG,
              "columns must be strictly increasing within a row");
    }
  }
  const int comps = dtype == INTI_C128 ? 2 : 1;
  check_finite(val, (size_t)nnz * comps, "correction values");
  std::unique_ptr<inti_csr> c(new inti_csr());
  c->ctx = ctx;
  c->m = m;
  c->n = n;
  c->nnz = nnz;
  c->dtype = dtype;
  c->rowptr.ensure(sizeof(int64_t) * (m + 1));
  c->col.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
  c->val.ensure(sizeof(double) * comps * std::max<int64_t>(nnz, 1));
  h2d(ctx, c->rowptr.p, rowptr, sizeof(int64_t) * (m + 1));
  h2d(ctx, c->col.p, col, sizeof(int32_t) * nnz);
  h2d(ctx, c->val.p, val, sizeof(double) * comps * nnz);
  INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  return c.release();
}

}  // namespace

namespace inti {

inti_csr* csr_create_host(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz,
                          const int64_t* rowptr, const int32_t* col, const double* val,
                          int dtype) {
  return csr_from_host(ctx, m, n, nnz, rowptr, col, val, dtype);
}


}  // namespace inti


using namespace inti;

extern "C" {

int inti_version(void) { return INTI_B200_ABI_VERSION; }

int inti_ctx_create(int device, void* stream, inti_ctx** out) {
  if (!out) {
    g_thread_error = "out is NULL";
    return INTI_E_ARG;
  }
  *out = nullptr;
  return guarded(nullptr, [&] {
    int count = 0;
    INTI_CUDA(cudaGetDeviceCount(&count));
    require(device >= 0 && device < count, INTI_E_ARG, "device index out of range");
    DeviceGuard dg(device);
    std::unique_ptr<inti_ctx> c(new inti_ctx());
    c->device = device;
    if (stream) {
      c->stream = static_cast<cudaStream_t>(stream);
    } else {
      INTI_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    INTI_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
    dev_prepare(device);  // the memory pool and its reservation: set-up cost here, not in a first product
    c->err_flag.ensure(sizeof(int));
    INTI_CUDA(cudaMemset(c->err_flag.p, 0, sizeof(int)));
    INTI_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&c->err_host), sizeof(int), cudaHostAllocDefault));
    *c->err_host = 0;
    *out = c.release();
  });
}

int inti_ctx_destroy(inti_ctx* ctx) {
  if (!ctx) return INTI_OK;
  {
    DeviceGuard dg(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& s : ctx->spans) {
      cudaEventDestroy(s.a);
      cudaEventDestroy(s.b);
    }
    ctx->spans.clear();
    ctx->err_flag.release();
    ctx->scan_tmp.release();
    if (ctx->err_host) cudaFreeHost(ctx->err_host);
    ctx->err_host = nullptr;
    for (inti::DevBuf* d : {&ctx->krylov.V, &ctx->krylov.w, &ctx->krylov.r, &ctx->krylov.e, &ctx->krylov.w_outer,
                            &ctx->krylov.partial, &ctx->krylov.h, &ctx->krylov.y, &ctx->krylov.nrm, &ctx->krylov.b,
                            &ctx->krylov.x, &ctx->krylov.small, &ctx->expi64, &ctx->expi32, &ctx->dimwork.d_xs, &ctx->dimwork.g0,
                            &ctx->dimwork.g1, &ctx->dimwork.theta, &ctx->dimwork.part, &ctx->dimwork.mu})
      d->release();
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return INTI_OK;
}

const char* inti_last_error(const inti_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_thread_error.c_str();
}

int inti_ctx_synchronize(inti_ctx* ctx) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] { sync_and_check(ctx); });
}

void* inti_ctx_stream(inti_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int64_t inti_ctx_launch_count(const inti_ctx* ctx) { return ctx ? ctx->launches : -1; }

static void resolve_spans(inti_ctx* ctx) {
  if (ctx->spans.empty()) return;
  INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  for (auto& s : ctx->spans) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s.a, s.b) == cudaSuccess) {
      auto& t = ctx->prof_totals[s.name];
      t.first += ms;
      t.second += 1;
    }
    cudaEventDestroy(s.a);
    cudaEventDestroy(s.b);
  }
  ctx->spans.clear();
}

int inti_ctx_set_profiling(inti_ctx* ctx, int enable) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] {
    resolve_spans(ctx);
    ctx->prof_totals.clear();
    ctx->profiling = enable != 0;
  });
}

int inti_ctx_profile(inti_ctx* ctx, const char* kernel, double* total_ms, int64_t* launches) {
  if (!ctx || !kernel) return INTI_E_ARG;
  return guarded(ctx, [&] {
    resolve_spans(ctx);
    auto it = ctx->prof_totals.find(kernel);
    if (total_ms) *total_ms = it == ctx->prof_totals.end() ? 0.0 : it->second.first;
    if (launches) *launches = it == ctx->prof_totals.end() ? 0 : it->second.second;
  });
}

int inti_dev_alloc(inti_ctx* ctx, int64_t bytes, void** ptr) {
  if (!ctx || !ptr) return INTI_E_ARG;
  return guarded(ctx, [&] {
    require(bytes >= 0, INTI_E_ARG, "negative size");
    *ptr = nullptr;
    cudaError_t e = cudaMalloc(ptr, std::max<int64_t>(bytes, 16));
    if (e != cudaSuccess) throw Error(INTI_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  });
}

int inti_dev_free(inti_ctx* ctx, void* ptr) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] {
    if (ptr) INTI_CUDA(cudaFree(ptr));
  });
}

int inti_memcpy(inti_ctx* ctx, void* dst, const void* src, int64_t bytes, int direction) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] {
    require(bytes >= 0 && (bytes == 0 || (dst && src)), INTI_E_ARG, "bad copy arguments");
    cudaMemcpyKind k = direction == INTI_H2D   ? cudaMemcpyHostToDevice
                       : direction == INTI_D2H ? cudaMemcpyDeviceToHost
                       : direction == INTI_D2D ? cudaMemcpyDeviceToDevice
                                               : (throw Error(INTI_E_ARG, "bad direction"), cudaMemcpyDefault);
    if (bytes) INTI_CUDA(cudaMemcpyAsync(dst, src, (size_t)bytes, k, ctx->stream));
    if (direction != INTI_D2D) INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

// ---------------------------------------------------------------- quadrature
int inti_quad_create(inti_ctx* ctx, int dim, int64_t n, const double* coords,
                     const double* normals, const double* weights, int32_t nq, inti_quad** out) {
  if (!ctx || !out) return INTI_E_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    require(dim == 2 || dim == 3, INTI_E_ARG, "dim must be 2 or 3");
    require(n > 0, INTI_E_ARG, "a quadrature needs at least one node");
    require(n < (int64_t)1 << 31, INTI_E_ARG, "more than 2^31-1 nodes");
    require(coords != nullptr, INTI_E_ARG, "coords is NULL");
    require(nq >= 0, INTI_E_ARG, "nq must be >= 0");
    require(nq == 0 || n % nq == 0, INTI_E_SHAPE, "node count is not a multiple of nq");
    check_finite(coords, (size_t)dim * n, "coords");
    if (normals) check_finite(normals, (size_t)dim * n, "normals");
    if (weights) check_finite(weights, (size_t)n, "weights");
    std::unique_ptr<inti_quad> q(new inti_quad());
    q->ctx = ctx;
    q->dim = dim;
    q->n = n;
    q->nq = nq;
    q->has_normals = normals != nullptr;
    q->h_coords.assign(coords, coords + (size_t)dim * n);
    if (normals) q->h_normals.assign(normals, normals + (size_t)dim * n);
    if (weights)
      q->h_weights.assign(weights, weights + n);
    else
      q->h_weights.assign((size_t)n, 1.0);
    q->coords.ensure(sizeof(double) * dim * n);
    h2d(ctx, q->coords.p, q->h_coords.data(), sizeof(double) * dim * n);
    if (normals) {
      q->normals.ensure(sizeof(double) * dim * n);
      h2d(ctx, q->normals.p, q->h_normals.data(), sizeof(double) * dim * n);
    }
    q->weights.ensure(sizeof(double) * n);
    h2d(ctx, q->weights.p, q->h_weights.data(), sizeof(double) * n);
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = q.release();
  });
}

int inti_quad_destroy(inti_quad* q) {
  if (!q) return INTI_OK;
  inti_ctx* ctx = q->ctx;
  return guarded(ctx, [&] {
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    delete q;
  });
}

int64_t inti_quad_size(const inti_quad* q) { return q ? q->n : -1; }

int inti_csr_create(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz, const int64_t* rowptr,
                    const int32_t* col, const double* val, int dtype, inti_csr** out) {
  if (!ctx || !out) return INTI_E_ARG;
  *out = nullptr;
  return guarded(ctx, [&] { *out = csr_from_host(ctx, m, n, nnz, rowptr, col, val, dtype); });
}

int inti_csr_create_from_csc(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz,
                             const int64_t* colptr1, const int64_t* rowval1,
                             const double* nzval, int dtype, inti_csr** out) {
  if (!ctx || !out) return INTI_E_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    require(m >= 0 && n >= 0 && nnz >= 0, INTI_E_ARG, "negative size");
    require(colptr1 != nullptr, INTI_E_ARG, "colptr is NULL");
    require(colptr1[0] == 1 && colptr1[n] == nnz + 1, INTI_E_SHAPE,
            "colptr must start at 1 and end at nnz+1");
    require(m < ((int64_t)1 << 31), INTI_E_ARG, "too many rows for int32 columns");
    const int comps = dtype == INTI_C128 ? 2 : 1;
    std::vector<int64_t> rp(m + 1, 0);
    for (int64_t p = 0; p < nnz; ++p) {
      const int64_t r = rowval1[p] - 1;
      require(r >= 0 && r < m, INTI_E_ARG, "row index out of range");
      rp[r + 1]++;
    }
    for (int64_t i = 0; i < m; ++i) rp[i + 1] += rp[i];
    std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
    std::vector<int32_t> col(nnz);
    std::vector<double> val((size_t)nnz * comps);
    // columns visited in increasing order, so each CSR row comes out sorted
    for (int64_t j = 0; j < n; ++j)
      for (int64_t p = colptr1[j] - 1; p < colptr1[j + 1] - 1; ++p) {
        const int64_t q = fill[rowval1[p] - 1]++;
        col[q] = (int32_t)j;
        for (int k = 0; k < comps; ++k) val[q * comps + k] = nzval[p * comps + k];
      }
    *out = csr_from_host(ctx, m, n, nnz, rp.data(), col.data(), val.data(), dtype);
  });
}

int inti_csr_info(const inti_csr* c, int64_t* m, int64_t* n, int64_t* nnz, int* dtype) {
  if (!c) return INTI_E_ARG;
  if (m) *m = c->m;
  if (n) *n = c->n;
  if (nnz) *nnz = c->nnz;
  if (dtype) *dtype = c->dtype;
  return INTI_OK;
}

int inti_csr_download(const inti_csr* c, int64_t* rowptr, int32_t* col, double* val) {
  if (!c) return INTI_E_ARG;
  inti_ctx* ctx = c->ctx;
  return guarded(ctx, [&] {
    const int comps = c->dtype == INTI_C128 ? 2 : 1;
    if (rowptr) d2h(ctx, rowptr, c->rowptr.p, sizeof(int64_t) * (c->m + 1));
    if (col) d2h(ctx, col, c->col.p, sizeof(int32_t) * c->nnz);
    if (val) d2h(ctx, val, c->val.p, sizeof(double) * comps * c->nnz);
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int inti_csr_apply(inti_csr* c, const double* x, double* y, const double* alpha,
                   const double* beta, int on_device) {
  if (!c) return INTI_E_ARG;
  inti_ctx* ctx = c->ctx;
  return guarded(ctx, [&] {
    require(x && y, INTI_E_ARG, "x/y NULL");
    const int comps = c->dtype == INTI_C128 ? 2 : 1;
    if (on_device) {
      csr_apply(ctx, c, x, y, alpha, beta);
      return;
    }
    DevBuf xd, yd;
    xd.ensure(sizeof(double) * comps * std::max<int64_t>(c->n, 1));
    yd.ensure(sizeof(double) * comps * std::max<int64_t>(c->m, 1));
    h2d(ctx, xd.p, x, sizeof(double) * comps * c->n);
    const bool bz = !beta || (beta[0] == 0.0 && beta[1] == 0.0);
    if (!bz) h2d(ctx, yd.p, y, sizeof(double) * comps * c->m);
    csr_apply(ctx, c, xd.as<double>(), yd.as<double>(), alpha, beta);
    d2h(ctx, y, yd.p, sizeof(double) * comps * c->m);
    sync_and_check(ctx);
  });
}

int inti_csr_destroy(inti_csr* c) {
  if (!c) return INTI_OK;
  inti_ctx* ctx = c->ctx;
  return guarded(ctx, [&] {
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    delete c;
  });
}

// ---------------------------------------------------------------- operator
int inti_op_create(inti_ctx* ctx, int pde, int kernel, double k_re, double k_im,
                   const inti_quad* target, const inti_quad* source,
                   const inti_csr* correction, int precision, inti_op** out) {
  if (!ctx || !out) return INTI_E_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    std::unique_ptr<inti_op> op(op_create(ctx, pde, kernel, k_re, k_im, target, source, correction, precision));
    op_autotune(op.get(), true);
    *out = op.release();
  });
}

int inti_op_create_combined(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* target,
                            const inti_quad* source, const inti_csr* corr_dl, const inti_csr* corr_sl,
                            const double* c_dl, const double* c_sl, int precision, inti_op** out) {
  if (!ctx || !out) return INTI_E_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    std::unique_ptr<inti_op> op(op_create_combined(ctx, pde, k_re, k_im, target, source, corr_dl, corr_sl,
                                                   c_dl, c_sl, precision));
    op_autotune(op.get(), true);
    *out = op.release();
  });
}

int inti_op_tuning(const inti_op* op, int32_t* targets_per_thread, int32_t* split) {
  if (!op) return INTI_E_ARG;
  if (targets_per_thread) *targets_per_thread = op->tpt;
  if (split) *split = op->split;
  return INTI_OK;
}

int inti_ctx_set_autotune(inti_ctx* ctx, int enable) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] { ctx->autotune = enable != 0; });
}

int inti_ctx_set_symmetric(inti_ctx* ctx, int enable) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] { ctx->symmetric = enable != 0; });
}

int inti_op_set_shard(inti_op* op, int rank, int nranks) {
  if (!op) return INTI_E_ARG;
  inti_ctx* ctx = op->ctx;
  return guarded(ctx, [&] { op_set_shard(op, rank, nranks); });
}

int inti_op_symmetric(const inti_op* op) {
  if (!op) return -INTI_E_ARG;
  return op->symm ? 1 : 0;
}

int inti_ctx_set_gmres_small(inti_ctx* ctx, int64_t max_unknowns) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] {
    require(max_unknowns >= 0, INTI_E_ARG, "max_unknowns must be >= 0");
    ctx->krylov_small = max_unknowns;
  });
}

int inti_ctx_set_single_launch(inti_ctx* ctx, int enable) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] { ctx->single_launch = enable != 0; });
}

int inti_op_single_launch(const inti_op* op) {
  if (!op) return -INTI_E_ARG;
  return op->small ? 1 : 0;
}

int inti_ctx_set_partial_budget(inti_ctx* ctx, double bytes) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] {
    if (!(bytes >= 0.0) || !std::isfinite(bytes)) throw Error(INTI_E_ARG, "the partial budget must be >= 0 bytes");
    ctx->symm_budget = bytes > 0.0 ? bytes : 2.0e9;
  });
}

int inti_op_panels(const inti_op* op) {
  if (!op) return -INTI_E_ARG;
  return op->symm ? (int)op->sym_panels.size() : 0;
}

int inti_op_info(const inti_op* op, int64_t* m, int64_t* n, int* dtype) {
  if (!op) return INTI_E_ARG;
  if (m) *m = op->target->n;
  if (n) *n = op->source->n;
  if (dtype) *dtype = op->pde == INTI_HELMHOLTZ ? INTI_C128 : INTI_F64;
  return INTI_OK;
}

// Host-pointer applies of small vectors in page-locked host memory that the
// device can address (cudaHostAlloc, or cudaHostRegister on a system with
// unified addressing) skip the copy engines, whose round trip costs several
// microseconds per copy: one small kernel reads x into the device staging
// buffer, and the product writes y straight into the host buffer (each row
// once; read once when beta != 0).
constexpr size_t kZeroCopyMax = (size_t)64 << 10;

static void* device_view(const void* p, size_t bytes) {
  if (bytes > kZeroCopyMax) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

__global__ void copy_doubles(int64_t n, const double* __restrict__ src, double* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

static int apply_common(inti_op* op, const double* x, int64_t ldx, double* y, int64_t ldy,
                        int32_t nrhs, const double* alpha, const double* beta, int on_device,
                        bool transpose) {
  if (!op) return INTI_E_ARG;
  inti_ctx* ctx = op->ctx;
  return guarded(ctx, [&] {
    require(x && y, INTI_E_ARG, "x/y NULL");
    require(nrhs >= 1, INTI_E_ARG, "nrhs must be >= 1");
    const int comps = op->pde == INTI_HELMHOLTZ ? 2 : 1;
    const int64_t nin = transpose ? op->target->n : op->source->n;
    const int64_t nout = transpose ? op->source->n : op->target->n;
    require(ldx >= nin && ldy >= nout, INTI_E_SHAPE, "leading dimension smaller than the vector length");
    const bool bz = !beta || (beta[0] == 0.0 && beta[1] == 0.0);
    require(!(transpose && op->shard_n > 1), INTI_E_UNSUPPORTED, "transpose of an item-sharded operator");
    if (!transpose && nrhs >= kMrhsMinColumns && op_mrhs_supported(op) && op->shard_n == 1) {
      // all columns at once: each kernel value evaluated once per 64 columns
      const double* xd = x;
      double* yd = y;
      int64_t lx = ldx, ly = ldy;
      const size_t cx = sizeof(double) * comps * nin, cy = sizeof(double) * comps * nout;
      if (!on_device) {
        op->mx.ensure(cx * nrhs);
        op->my.ensure(cy * nrhs);
        INTI_CUDA(cudaMemcpy2DAsync(op->mx.p, cx, x, sizeof(double) * comps * ldx, cx, nrhs, cudaMemcpyHostToDevice,
                                    ctx->stream));
        if (!bz)
          INTI_CUDA(cudaMemcpy2DAsync(op->my.p, cy, y, sizeof(double) * comps * ldy, cy, nrhs,
                                      cudaMemcpyHostToDevice, ctx->stream));
        xd = op->mx.as<double>();
        yd = op->my.as<double>();
        lx = nin;
        ly = nout;
      }
      op_apply_mrhs(op, xd, lx, yd, ly, nrhs, alpha, beta);
      if (!on_device) {
        INTI_CUDA(cudaMemcpy2DAsync(y, sizeof(double) * comps * ldy, op->my.p, cy, cy, nrhs, cudaMemcpyDeviceToHost,
                                    ctx->stream));
        sync_and_check(ctx);
      }
      return;
    }
    if (transpose && !op->tpartial.p) op_prepare_transpose(op);
    for (int32_t r = 0; r < nrhs; ++r) {
      const double* xr = x + (size_t)r * ldx * comps;
      double* yr = y + (size_t)r * ldy * comps;
      const double* xd = xr;
      double* yd = yr;
      bool direct = false;  // y written in place in mapped host memory
      if (!on_device) {
        // host staging, made on the first host-pointer apply
        const size_t big = sizeof(double) * comps * std::max(op->target->n, op->source->n);
        op->xbuf.ensure(big);
        op->ybuf.ensure(big);
        const size_t bx = sizeof(double) * comps * nin, by = sizeof(double) * comps * nout;
        const void* xv = device_view(xr, bx);
        void* yv = xv ? device_view(yr, by) : nullptr;
        if (xv && yv) {
          const int64_t cnt = (int64_t)comps * nin;
          copy_doubles<<<(unsigned)std::min<int64_t>(64, (cnt + 255) / 256), 256, 0, ctx->stream>>>(
              cnt, static_cast<const double*>(xv), op->xbuf.as<double>());
          INTI_CUDA(cudaGetLastError());
          ctx->launches++;
          xd = op->xbuf.as<double>();
          yd = static_cast<double*>(yv);
          direct = true;
        } else {
          h2d(ctx, op->xbuf.p, xr, bx);
          if (!bz) h2d(ctx, op->ybuf.p, yr, by);
          xd = op->xbuf.as<double>();
          yd = op->ybuf.as<double>();
        }
      }
      if (transpose)
        op_apply_transpose_device(op, xd, yd, alpha, beta);
      else
        op_apply_device(op, xd, yd, alpha, beta);
      if (!on_device && !direct) d2h(ctx, yr, op->ybuf.p, sizeof(double) * comps * nout);
    }
    if (!on_device) sync_and_check(ctx);
  });
}

int inti_op_apply(inti_op* op, const double* x, int64_t ldx, double* y, int64_t ldy,
                  int32_t nrhs, const double* alpha, const double* beta, int on_device) {
  return apply_common(op, x, ldx, y, ldy, nrhs, alpha, beta, on_device, false);
}

int inti_op_apply_transpose(inti_op* op, const double* x, int64_t ldx, double* y, int64_t ldy,
                            int32_t nrhs, const double* alpha, const double* beta,
                            int on_device) {
  return apply_common(op, x, ldx, y, ldy, nrhs, alpha, beta, on_device, true);
}

int inti_op_assemble(inti_op* op, double* out, int on_device) {
  if (!op) return INTI_E_ARG;
  inti_ctx* ctx = op->ctx;
  return guarded(ctx, [&] {
    require(out != nullptr, INTI_E_ARG, "out is NULL");
    const int comps = op->pde == INTI_HELMHOLTZ ? 2 : 1;
    const size_t bytes = sizeof(double) * comps * (size_t)op->target->n * (size_t)op->source->n;
    PairLaunch L = make_launch(op, nullptr);
    if (on_device) {
      pair_assemble(ctx, L, out);
      return;
    }
    DevBuf d;
    d.ensure(bytes);
    pair_assemble(ctx, L, d.as<double>());
    d2h(ctx, out, d.p, bytes);
    sync_and_check(ctx);
  });
}

int inti_op_destroy(inti_op* op) {
  if (!op) return INTI_OK;
  inti_ctx* ctx = op->ctx;
  return guarded(ctx, [&] {
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    delete op;
  });
}

// ---------------------------------------------------------------- DIM
int inti_dim_correction(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* q,
                        int derivative, const double* green_multiplier, inti_csr** dS,
                        inti_csr** dD) {
  if (!ctx || !dS || !dD) return INTI_E_ARG;
  *dS = *dD = nullptr;
  return guarded(ctx, [&] {
    dim_correction(ctx, pde, k_re, k_im, q, derivative, green_multiplier, dS, dD);
  });
}

int inti_dim_correction_targets(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* target,
                                const inti_quad* source, int derivative, const double* green_multiplier,
                                double maxdist, inti_csr** dS, inti_csr** dD) {
  if (!ctx || !dS || !dD) return INTI_E_ARG;
  *dS = *dD = nullptr;
  return guarded(ctx, [&] {
    dim_correction_targets(ctx, pde, k_re, k_im, target, source, derivative, green_multiplier, maxdist, dS, dD);
  });
}

// ---------------------------------------------------------------- GMRES
int inti_gmres(inti_ctx* ctx, int32_t nterms, inti_op* const* ops, const double* coefs,
               const double* shift, const double* b, double* x, double rtol, int32_t restart,
               int32_t maxiter, int32_t mode, int on_device, double* history,
               inti_gmres_stats* stats) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] {
    gmres_solve(ctx, nterms, ops, coefs, shift, b, x, rtol, restart, maxiter, mode, on_device,
                history, stats);
  });
}

// ---------------------------------------------------------------- adjoint
int inti_op_grad_sources(inti_op* op, const double* g, const double* sigma, double* dsigma,
                         double* dcoords, double* dnormals, double* dweights, int on_device) {
  if (!op) return INTI_E_ARG;
  inti_ctx* ctx = op->ctx;
  return guarded(ctx, [&] {
    grad_sources(op, g, sigma, dsigma, dcoords, dnormals, dweights, on_device);
  });
}

int inti_batch_create(inti_ctx* ctx, int32_t nsurf, const inti_quad* const* quads, int pde, int kernel,
                      double k_re, double k_im, const double* c_dl, const double* c_sl,
                      const inti_csr* const* corr_dl, const inti_csr* const* corr_sl, inti_batch** out) {
  if (!ctx || !out) return INTI_E_ARG;
  *out = nullptr;
  return guarded(ctx, [&] {
    *out = batch_create(ctx, nsurf, quads, pde, kernel, k_re, k_im, c_dl, c_sl, corr_dl, corr_sl);
  });
}

int inti_batch_apply(inti_batch* b, int precision, const double* x, int64_t ldx, double* y, int64_t ldy,
                     int32_t nrhs, const double* alpha, const double* beta, int on_device) {
  if (!b) return INTI_E_ARG;
  inti_ctx* ctx = b->ctx;
  return guarded(ctx, [&] {
    require(x && y, INTI_E_ARG, "x/y NULL");
    require(nrhs >= 1, INTI_E_ARG, "nrhs must be >= 1");
    const int64_t n = b->off.back();
    require(ldx >= n && ldy >= n, INTI_E_SHAPE, "leading dimension smaller than the node count");
    const int comps = b->pde == INTI_HELMHOLTZ ? 2 : 1;
    if (on_device) {
      batch_apply_device(b, precision, x, ldx, y, ldy, nrhs, alpha, beta);
      return;
    }
    if (precision == INTI_TF32) {  // copies overlapped with the compute, surface group by group
      batch_apply_host_tf32(b, x, ldx, y, ldy, nrhs, alpha, beta);
      return;
    }
    // staging buffers are kept on the handle: no allocation per call once they fit
    DevBuf &xd = b->xstage, &yd = b->ystage;
    const size_t bx = sizeof(double) * comps * (size_t)ldx * nrhs, by = sizeof(double) * comps * (size_t)ldy * nrhs;
    xd.ensure(bx);
    yd.ensure(by);
    h2d(ctx, xd.p, x, bx);
    const bool bz = !beta || (beta[0] == 0.0 && beta[1] == 0.0);
    if (!bz) h2d(ctx, yd.p, y, by);
    batch_apply_device(b, precision, xd.as<double>(), ldx, yd.as<double>(), ldy, nrhs, alpha, beta);
    d2h(ctx, y, yd.p, by);
    sync_and_check(ctx);
  });
}

int inti_batch_gmres(inti_batch* b, const double* shift, const double* B, double* X, int64_t ld, int32_t nrhs,
                     double rtol, int32_t restart, int32_t maxiter, int32_t mode, int on_device, double* relres,
                     inti_gmres_stats* stats) {
  if (!b) return INTI_E_ARG;
  inti_ctx* ctx = b->ctx;
  return guarded(ctx, [&] {
    batch_gmres(b, shift, B, X, ld, nrhs, rtol, restart, maxiter, mode, on_device, relres, stats);
  });
}

int64_t inti_batch_size(const inti_batch* b) { return b ? b->off.back() : -1; }

int inti_batch_destroy(inti_batch* b) {
  if (!b) return INTI_OK;
  inti_ctx* ctx = b->ctx;
  return guarded(ctx, [&] {
    INTI_CUDA(cudaStreamSynchronize(ctx->stream));
    delete b;
  });
}

int inti_selftest_math(inti_ctx* ctx, double* out) {
  if (!ctx || !out) return INTI_E_ARG;
  return guarded(ctx, [&] { selftest_math(ctx, out); });
}

int inti_selftest_wait_timeout(inti_ctx* ctx) {
  if (!ctx) return INTI_E_ARG;
  return guarded(ctx, [&] { selftest_wait_timeout(ctx); });
}

int inti_measure_peaks(inti_ctx* ctx, double* fp64_flops, double* fp32_flops, double* mufu_ops) {
  if (!ctx || !fp64_flops || !fp32_flops || !mufu_ops) return INTI_E_ARG;
  return guarded(ctx, [&] { measure_peaks(ctx, fp64_flops, fp32_flops, mufu_ops); });
}

int inti_measure_peak_tf32(inti_ctx* ctx, double* tf32_flops) {
  if (!ctx || !tf32_flops) return INTI_E_ARG;
  return guarded(ctx, [&] { measure_peak_tf32(ctx, tf32_flops); });
}

}  // extern "C"
