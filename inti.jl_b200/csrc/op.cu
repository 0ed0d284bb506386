// Operator handles: validation of the (pde, kernel, target, source,
// correction) combination that IntegralOperator/single_double_layer accept
// (src/nystrom.jl:79-89, src/api.jl:65-78) and sizing of the operator's
// scratch buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "device_common.cuh"
#include "internal.h"

namespace inti {

static void req(bool c, int code, const std::string& m) {
  if (!c) throw Error(code, m);
}

// The checks of op_create, without creating anything.
static void op_validate(inti_ctx* ctx, int pde, int kernel, double k_re, double k_im, const inti_quad* target,
                        const inti_quad* source, const inti_csr* correction, int precision) {
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
}

inti_op* op_create(inti_ctx* ctx, int pde, int kernel, double k_re, double k_im,
                   const inti_quad* target, const inti_quad* source, const inti_csr* correction,
                   int precision) {
  op_validate(ctx, pde, kernel, k_re, k_im, target, source, correction, precision);
  const int dim = source->dim;
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
  op_symm_init(op.get());
  if (!op->symm) {
    // the one-sided records and partials (the symmetric form packs its own
    // records and keeps its partials in the context)
    op->packed.ensure((size_t)op->n_tiles * tile * pair_record_bytes(pde, kernel, dim, precision));
    op->partial.ensure((size_t)op->split * target->n * pair_partial_bytes(pde, precision));
  }
  op_autotune(op.get(), false);
  op->small = ctx->single_launch && pair_small_eligible(precision, target->n, source->n);
  return op.release();
}

// c1*C_dl + c2*C_sl with the union of the two patterns (merged on the device, once).
inti_op* op_create_combined(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* target,
                            const inti_quad* source, const inti_csr* corr_dl, const inti_csr* corr_sl,
                            const double* c_dl, const double* c_sl, int precision) {
  req(target && source, INTI_E_ARG, "target/source quadrature is NULL");
  req(source->dim == 3, INTI_E_UNSUPPORTED, "the combined-field operator is implemented in 3D");
  req(c_dl && c_sl, INTI_E_ARG, "coefficients are NULL");
  const bool cplx = pde == INTI_HELMHOLTZ;
  if (!cplx) req(c_dl[1] == 0.0 && c_sl[1] == 0.0, INTI_E_UNSUPPORTED,
                 "complex coefficients need a Helmholtz (complex) operator");
  // validate both halves like two ordinary operators
  op_validate(ctx, pde, INTI_DL, k_re, k_im, target, source, corr_dl, precision);
  op_validate(ctx, pde, INTI_SL, k_re, k_im, target, source, corr_sl, precision);
  std::unique_ptr<inti_op> op(new inti_op());
  op->ctx = ctx;
  op->pde = pde;
  op->kind = CF;
  op->dim = 3;
  op->precision = precision;
  op->k = k_re;
  op->target = target;
  op->source = source;
  op->c1[0] = c_dl[0];
  op->c1[1] = c_dl[1];
  op->c2[0] = c_sl[0];
  op->c2[1] = c_sl[1];
  if (corr_dl || corr_sl) {
    op->owned_corr = merge_corrections(ctx, corr_dl, c_dl, corr_sl, c_sl, target->n, source->n, cplx);
    op->corr = op->owned_corr.get();
  }
  const int64_t tile = pair_tile(precision);
  op->n_tiles = std::max<int64_t>(1, (source->n + tile - 1) / tile);
  op->split = pair_plan_split(ctx, pde, CF, 3, precision, target->n, source->n);
  op_symm_init(op.get());
  if (!op->symm) {
    op->packed.ensure((size_t)op->n_tiles * tile * pair_record_bytes(pde, CF, 3, precision));
    op->partial.ensure((size_t)op->split * target->n * pair_partial_bytes(pde, precision));
  }
  op_autotune(op.get(), false);
  op->small = ctx->single_launch && pair_small_eligible(precision, target->n, source->n);
  return op.release();
}

// The same operator (kernel, coefficients, correction) in another precision.
// The twin refers to op's correction: destroy it first.
inti_op* op_clone_precision(const inti_op* op, int precision) {
  std::unique_ptr<inti_op> t(new inti_op());
  t->ctx = op->ctx;
  t->pde = op->pde;
  t->kind = op->kind;
  t->dim = op->dim;
  t->precision = precision;
  t->k = op->k;
  t->target = op->target;
  t->source = op->source;
  t->corr = op->corr;
  for (int i = 0; i < 2; ++i) {
    t->c1[i] = op->c1[i];
    t->c2[i] = op->c2[i];
  }
  const int64_t tile = pair_tile(precision);
  t->n_tiles = std::max<int64_t>(1, (op->source->n + tile - 1) / tile);
  t->split = pair_plan_split(op->ctx, op->pde, op->kind, op->dim, precision, op->target->n, op->source->n);
  op_symm_init(t.get());
  if (!t->symm) {
    t->packed.ensure((size_t)t->n_tiles * tile * pair_record_bytes(op->pde, op->kind, op->dim, precision));
    t->partial.ensure((size_t)t->split * op->target->n * pair_partial_bytes(op->pde, precision));
  }
  op_autotune(t.get(), false);
  return t.release();
}

// The symmetric form keeps per work item a row partial (128*tpt values) and
// per row block a column partial of each later node (nb x n values, N^2/512
// at 4 targets per thread).  While both fit the partial budget (2 GB, and a
// quarter of the device memory free at creation; the budget is the
// context's, inti_ctx_set_partial_budget) the items run in one launch.  Beyond it the items are grouped into panels of source blocks: a
// panel's launch writes the column partials of its own nodes only
// (nb x panel width), a fold kernel adds them and the row partials into
// running sums, and the next panel reuses the buffers.  Memory stays
// O(N) + the budget; the pair evaluations are the same.
constexpr double kSymmMaxFreeShare = 0.25;

namespace {

// Partial bytes of a symmetric plan with panels of pcols source blocks.
double symm_partial_bytes(int64_t n, int tpt, int ch, int pcols, int pb) {
  const int64_t bt = pair_symm_block(tpt);
  const int64_t nb = std::max<int64_t>(1, (n + bt - 1) / bt);
  const int64_t pc = std::max<int64_t>(1, std::min<int64_t>(pcols, nb));
  const int64_t cw = std::max<int64_t>(1, std::min<int64_t>(ch, pc));
  const double items = (double)nb * (double)((pc + cw - 1) / cw);  // per panel, at most
  const double zl = pc >= nb ? (double)((n + 511) / 512 * 512) : (double)(pc * bt);
  return ((double)nb * zl + items * (double)bt) * pb;
}

}  // namespace

// Widest panel (in source blocks) whose partials fit `budget`; 0 if none does.
int symm_panel_width(int64_t n, int tpt, int ch, int pb, double budget) {
  const int64_t bt = pair_symm_block(tpt);
  const int nb = (int)std::max<int64_t>(1, (n + bt - 1) / bt);
  if (symm_partial_bytes(n, tpt, ch, nb, pb) <= budget) return nb;
  int lo = 0, hi = nb - 1;  // largest pcols in [1, nb) that fits
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (symm_partial_bytes(n, tpt, ch, mid, pb) <= budget) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Panel width and source blocks per item of a plan.  With several panels an
// item spans at most an eighth of a panel, so that each panel's launch has
// many items and a short tail.
void symm_layout(int64_t n, int tpt, int ch, int pb, double budget, int& pcols, int& ch_eff) {
  const int64_t bt = pair_symm_block(tpt);
  const int nb = (int)std::max<int64_t>(1, (n + bt - 1) / bt);
  ch_eff = std::max(1, ch);
  pcols = std::max(1, symm_panel_width(n, tpt, ch_eff, pb, budget));
  if (pcols >= nb) return;
  for (int it = 0; it < 4; ++it) {
    const int c = std::max(1, std::min(ch_eff, pcols / 8));
    if (c == ch_eff) break;
    ch_eff = c;
    pcols = std::max(1, symm_panel_width(n, tpt, ch_eff, pb, budget));
  }
}

double symm_budget(const inti_op* op) {
  size_t free_b = 0, total_b = 0;
  INTI_CUDA(cudaMemGetInfo(&free_b, &total_b));
  free_b += dev_cache_bytes(op->ctx->device);  // released memory the pool holds counts as free
  return std::min(op->ctx->symm_budget,
                  kSymmMaxFreeShare * (double)free_b + op->ctx->sym_ypart.bytes + op->ctx->sym_zpart.bytes);
}

void op_symm_configure(inti_op* op, int tpt, int ch) {
  std::vector<int32_t> tab;
  int nb = 0, nitems = 0;
  const int pb = pair_partial_bytes(op->pde, op->precision);
  int pcols = 1, ch_eff = 1;
  symm_layout(op->source->n, tpt, ch, pb, op->sym_budget, pcols, ch_eff);
  pair_symm_plan(op->source->n, tpt, ch_eff, pcols, tab, op->sym_panels, nb, nitems);
  INTI_CUDA(cudaStreamSynchronize(op->ctx->stream));  // no launch is reading the old table
  // half again as much room: a re-configuration (a tuned shape) then rarely reallocates
  if (op->sym_tab.bytes < sizeof(int32_t) * tab.size()) op->sym_tab.ensure(sizeof(int32_t) * tab.size() * 3 / 2);
  INTI_CUDA(cudaMemcpy(op->sym_tab.p, tab.data(), sizeof(int32_t) * tab.size(), cudaMemcpyHostToDevice));
  op->sym_nb = nb;
  op->sym_nitems = nitems;
  op->tpt = tpt;
  op->split = ch;
  const int64_t npad = op->n_tiles * pair_tile(op->precision);
  const bool panels = op->sym_panels.size() > 1;
  op->sym_zld = panels ? (int64_t)pcols * pair_symm_block(tpt) : npad;
  inti_ctx* ctx = op->ctx;
  const size_t yb = (size_t)pb * nitems * pair_symm_block(tpt);
  if (ctx->sym_ypart.bytes < yb) ctx->sym_ypart.ensure(yb + yb / 4);
  ctx->sym_zpart.ensure((size_t)pb * nb * op->sym_zld);
  if (panels) ctx->sym_acc.ensure(sizeof(double) * (op->pde == INTI_HELMHOLTZ ? 2 : 1) * op->source->n);
  if (op->shard_n > 1) op_set_shard(op, op->shard_rank, op->shard_n);  // the items changed
}

void op_set_shard(inti_op* op, int rank, int nranks) {
  if (nranks < 1 || rank < 0 || rank >= nranks) throw Error(INTI_E_ARG, "shard rank must be in [0, nranks)");
  if (nranks > 1 && !op->symm)
    throw Error(INTI_E_UNSUPPORTED, "item shards need the symmetric form (a square 3D operator); "
                                    "shard other operators by target rows");
  op->shard_rank = rank;
  op->shard_n = nranks;
  op->shard_items = 0;
  op->shard_panels.clear();
  if (nranks == 1) return;
  std::vector<int32_t> tab;
  std::vector<SymPanel> panels;
  int nb = 0, nitems = 0;
  const int pb = pair_partial_bytes(op->pde, op->precision);
  int pcols = 1, ch_eff = 1;
  symm_layout(op->source->n, op->tpt, op->split, pb, op->sym_budget, pcols, ch_eff);
  pair_symm_plan(op->source->n, op->tpt, ch_eff, pcols, tab, panels, nb, nitems);
  // round robin over the items of each panel (largest first); ids are the
  // panel-local item indices (the row-partial slots)
  std::vector<int32_t> items, ids;
  int global = 0;
  for (const SymPanel& P : panels) {
    op->shard_panels.push_back((int32_t)ids.size());
    int count = 0;
    for (int q = 0; q < P.nitems; ++q, ++global) {
      if (global % nranks != rank) continue;
      for (int c = 0; c < 3; ++c) items.push_back(tab[P.item_off + 3 * q + c]);
      ids.push_back(q);
      ++count;
    }
    op->shard_panels.push_back(count);
  }
  op->shard_items = (int)ids.size();
  items.insert(items.end(), ids.begin(), ids.end());
  INTI_CUDA(cudaStreamSynchronize(op->ctx->stream));
  op->shard_tab.ensure(sizeof(int32_t) * std::max<size_t>(items.size(), 1));
  if (!items.empty())
    INTI_CUDA(cudaMemcpy(op->shard_tab.p, items.data(), sizeof(int32_t) * items.size(), cudaMemcpyHostToDevice));
}

void op_symm_init(inti_op* op) {
  inti_ctx* ctx = op->ctx;
  op->symm = false;
  if (!ctx->symmetric || op->target != op->source) return;
  const int64_t n = op->source->n;
  const int tile = pair_tile(op->precision);
  const int64_t bmax = pair_symm_block(4);
  const int64_t npad = (n + bmax - 1) / bmax * bmax;  // whole blocks for both node-block sizes
  op->sym_budget = symm_budget(op);
  // the narrowest panel (one source block, 2 targets per thread) must fit
  if (symm_panel_width(n, 2, 1, pair_partial_bytes(op->pde, op->precision), op->sym_budget) < 1) return;
  op->symm = true;
  op->n_tiles = npad / tile;
  op->packed.ensure((size_t)npad * pair_symm_record_bytes(op->pde, op->kind, op->dim, op->precision));
  // untimed default shape: 4 targets per thread for FP32C (two target pairs
  // of the paired-FP32 kernel; timed picks at C3: 4 / 5 blocks per item),
  // 2 for FP64
  const int tpt = op->precision == INTI_FP32C ? 4 : 2;
  op_symm_configure(op, tpt, pair_symm_default_ch(ctx, op->pde, op->kind, op->dim, op->precision, n, tpt));
}

// Problems below this many pairs keep the heuristic shape (a timing pass
// would cost more than it could save).
constexpr double kTuneMinPairs = 67108864.0;

void op_autotune(inti_op* op, bool measure) {
  inti_ctx* ctx = op->ctx;
  const int64_t m = op->target->n, n = op->source->n;
  const std::string key = std::to_string(op->pde) + "/" + std::to_string(op->kind) + "/" +
                          std::to_string(op->dim) + "/" + std::to_string(op->precision) + "/" +
                          std::to_string(m) + "/" + std::to_string(n) + (op->symm ? "/symmetric" : "");
  if (op->symm) {
    // symmetric form: 4 or 2 targets per thread, each with the default number
    // of source blocks per item, half and twice it
    auto cached = ctx->tuned.find(key);
    if (cached != ctx->tuned.end()) {
      if (cached->second.first != op->tpt || cached->second.second != op->split)
        op_symm_configure(op, cached->second.first, cached->second.second);
      return;
    }
    if (!measure || !ctx->autotune || (double)m * (double)n < kTuneMinPairs) return;
    std::vector<std::pair<int, int>> cand;
    for (int tpt : {4, 2}) {
      const int c0 = pair_symm_default_ch(ctx, op->pde, op->kind, op->dim, op->precision, n, tpt);
      for (int ch : {c0, std::max(1, c0 / 2), 2 * c0})
        if (std::find(cand.begin(), cand.end(), std::make_pair(tpt, ch)) == cand.end()) cand.emplace_back(tpt, ch);
    }
    const int comps = op->pde == INTI_HELMHOLTZ ? 2 : 1;
    op->xbuf.ensure(sizeof(double) * comps * std::max(m, n));
    INTI_CUDA(cudaMemsetAsync(op->xbuf.p, 0, sizeof(double) * comps * n, ctx->stream));
    cudaEvent_t e0, e1;
    INTI_CUDA(cudaEventCreate(&e0));
    INTI_CUDA(cudaEventCreate(&e1));
    float best = -1.0f;
    std::pair<int, int> pick(op->tpt, op->split);
    int warmed = 0;
    for (auto& c : cand) {
      op_symm_configure(op, c.first, c.second);
      PairLaunch L = make_launch(op, op->xbuf.as<double>());
      if (c.first != warmed) {  // one warm-up per kernel (targets per thread); the others reuse it
        pair_launch(ctx, L);
        warmed = c.first;
      }
      INTI_CUDA(cudaEventRecord(e0, ctx->stream));
      pair_launch(ctx, L);
      INTI_CUDA(cudaEventRecord(e1, ctx->stream));
      INTI_CUDA(cudaEventSynchronize(e1));
      float ms = 0.0f;
      INTI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (best < 0.0f || ms < best) {
        best = ms;
        pick = c;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    sync_and_check(ctx);
    ctx->tuned[key] = pick;
    op_symm_configure(op, pick.first, pick.second);
    return;
  }
  const size_t pbytes = (size_t)pair_partial_bytes(op->pde, op->precision);
  auto set = [&](int tpt, int split) {
    op->tpt = tpt;
    op->split = split;
    op->partial.ensure((size_t)split * m * pbytes);
  };
  auto it = ctx->tuned.find(key);
  if (it != ctx->tuned.end()) {
    set(it->second.first, it->second.second);
    return;
  }
  if (!measure || !ctx->autotune || (double)m * (double)n < kTuneMinPairs) return;
  // candidates: 4 or 2 targets per thread, each with the heuristic split,
  // half of it and twice it (at most one chunk per source tile, kMaxSplit chunks)
  std::vector<std::pair<int, int>> cand;
  for (int tpt : {4, 2}) {
    const int s0 = pair_plan_split(ctx, op->pde, op->kind, op->dim, op->precision, m, n, tpt);
    const int hi = (int)std::min<int64_t>({(int64_t)2 * s0, op->n_tiles, (int64_t)kMaxSplit});
    for (int sp : {s0, std::max(1, s0 / 2), hi})
      if (std::find(cand.begin(), cand.end(), std::make_pair(tpt, sp)) == cand.end()) cand.emplace_back(tpt, sp);
  }
  int smax = 1;
  for (auto& c : cand) smax = std::max(smax, c.second);
  op->partial.ensure((size_t)smax * m * pbytes);
  // the pair kernel's cost does not depend on the density: time it on zeros
  const int comps = op->pde == INTI_HELMHOLTZ ? 2 : 1;
  op->xbuf.ensure(sizeof(double) * comps * std::max(m, n));
  INTI_CUDA(cudaMemsetAsync(op->xbuf.p, 0, sizeof(double) * comps * n, ctx->stream));
  PairLaunch L = make_launch(op, op->xbuf.as<double>());
  cudaEvent_t e0, e1;
  INTI_CUDA(cudaEventCreate(&e0));
  INTI_CUDA(cudaEventCreate(&e1));
  float best = -1.0f;
  std::pair<int, int> pick(op->tpt, op->split);
  int warmed = 0;
  for (auto& c : cand) {
    L.tpt = c.first;
    L.split = c.second;
    if (c.first != warmed) {  // one warm-up per kernel (targets per thread)
      pair_launch(ctx, L);
      warmed = c.first;
    }
    INTI_CUDA(cudaEventRecord(e0, ctx->stream));
    pair_launch(ctx, L);
    INTI_CUDA(cudaEventRecord(e1, ctx->stream));
    INTI_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    INTI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (best < 0.0f || ms < best) {
      best = ms;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  sync_and_check(ctx);
  ctx->tuned[key] = pick;
  set(pick.first, pick.second);
}

// A^T as a forward product with the roles swapped (square operators with the
// symmetric form: the symmetric product of the swapped kernel): (A^T g)_j =
// w_j sum_i K(x_i, y_j) g_i, and K(x_i, y_j) = K'(y_j, x_i) with K' the
// kernel of the swapped roles (the kernels of src/kernels.jl:137-204,
// 347-413 satisfy SL(x,y) = SL(y,x), DL(x,y) = ADL(y,x), ADL(x,y) = DL(y,x),
// HS(x,y) = HS(y,x), the normal travelling with its point).  So A^T runs on
// the pair kernel with targets = the source nodes (and their normals),
// sources = the target nodes with unit weights, density g, and w_j applied
// per row in the epilogue.
int transposed_kind(int kind) { return kind == DL ? ADL : kind == ADL ? DL : kind; }

void op_prepare_transpose(inti_op* op) {
  if (op->kind == CF) throw Error(INTI_E_UNSUPPORTED, "transpose of a combined-field operator");
  inti_ctx* ctx = op->ctx;
  const int kt = transposed_kind(op->kind);
  const int64_t m2 = op->source->n, n2 = op->target->n;
  const int tile = pair_tile(op->precision);
  op->tn_tiles = std::max<int64_t>(1, (n2 + tile - 1) / tile);
  // the context's timed shape for this problem when there is one, else the heuristic
  const std::string key = std::to_string(op->pde) + "/" + std::to_string(kt) + "/" + std::to_string(op->dim) +
                          "/" + std::to_string(op->precision) + "/" + std::to_string(m2) + "/" + std::to_string(n2);
  auto it = ctx->tuned.find(key);
  if (it != ctx->tuned.end()) {
    op->ttpt = it->second.first;
    op->tsplit = it->second.second;
  } else {
    op->ttpt = 4;
    op->tsplit = pair_plan_split(ctx, op->pde, kt, op->dim, op->precision, m2, n2, 4);
  }
  op->tpacked.ensure((size_t)op->tn_tiles * tile * pair_record_bytes(op->pde, kt, op->dim, op->precision));
  if (op->symm)  // the symmetric form packs all npad = n_tiles * tile nodes in its own records
    op->tpacked.ensure((size_t)op->n_tiles * tile * pair_symm_record_bytes(op->pde, kt, op->dim, op->precision));
  op->tpartial.ensure((size_t)op->tsplit * m2 * pair_partial_bytes(op->pde, op->precision));
  std::vector<double> ones((size_t)std::max<int64_t>(n2, 1), 1.0);
  op->tones.ensure(sizeof(double) * ones.size());
  INTI_CUDA(cudaMemcpy(op->tones.p, ones.data(), sizeof(double) * ones.size(), cudaMemcpyHostToDevice));
  if (op->corr && !op->corrT) op->corrT = csr_transpose(ctx, op->corr);
}

}  // namespace inti
