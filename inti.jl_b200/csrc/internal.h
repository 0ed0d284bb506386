// Operator handle and the functions the C ABI layer calls into.  Internal.
#pragma once

#include <atomic>
#include <memory>
#include <vector>

#include "common.h"

namespace inti {
// Identity of an operator handle, never reused within the process (a freed
// handle's address can be).
inline uint64_t next_op_id() {
  static std::atomic<uint64_t> counter{0};
  return ++counter;
}
}  // namespace inti

struct inti_op {
  const uint64_t id = inti::next_op_id();
  inti_ctx* ctx = nullptr;
  int pde = INTI_LAPLACE, kind = INTI_SL, dim = 3, precision = INTI_FP64;
  double k = 0.0;
  const inti_quad* target = nullptr;
  const inti_quad* source = nullptr;
  const inti_csr* corr = nullptr;
  std::unique_ptr<inti_csr> corrT;  // transposed correction, built on first A^T apply
  std::unique_ptr<inti_csr> owned_corr;  // CF: c1*C_dl + c2*C_sl merged
  double c1[2] = {1.0, 0.0}, c2[2] = {0.0, 0.0};  // CF coefficients
  // scratch owned by the operator
  inti::DevBuf packed;    // packed source records, n_tiles * tile
  inti::DevBuf partial;   // split x m accumulators
  inti::DevBuf xbuf, ybuf;  // staging for host-pointer applies
  inti::DevBuf tpartial, tpacked, tones;  // A^T: partials, packed target records, unit weights
  inti::DevBuf gpartial;  // source gradients: split x n x (2 dim + 2)
  inti::DevBuf mx, my;    // staging of host columns for multi-column applies
  int split = 1;
  int tpt = 4;  // targets per thread of the pair kernel (autotuned with split)
  int tsplit = 1, ttpt = 4;  // A^T launch shape
  // symmetric form (target set == source set, pair_symm): plan table and
  // column partials; split holds the source blocks per work item
  bool small = false;  // applies in the single-launch form (pair_small)
  bool symm = false;
  int sym_nb = 0, sym_nitems = 0;
  inti::DevBuf sym_tab;
  // panels of the work items (one unless the column partials of the whole
  // operator would pass the partial budget); the partials and running sums
  // themselves are the context's (sym_ypart, sym_zpart, sym_acc)
  std::vector<inti::SymPanel> sym_panels;
  int64_t sym_zld = 0;
  double sym_budget = 0.0;  // bytes of partials allowed, fixed at creation
  // item shard of this operator (inti_op_set_shard): rank, ranks, and the
  // rank's items (3 x n) followed by their ids; per panel (offset, count)
  int shard_rank = 0, shard_n = 1, shard_items = 0;
  inti::DevBuf shard_tab;
  std::vector<int32_t> shard_panels;
  int64_t n_tiles = 1, tn_tiles = 1;
  // Derived operators kept for repeated solves: the FP32C twin used by the
  // mixed-precision GMRES, and (on a double layer) the combined-field operator
  // fused with the single layer `fused_sl` under coefficients fused_c.
  std::unique_ptr<inti_op> twin32;
  std::unique_ptr<inti_op> fused;
  uint64_t fused_sl = 0;
  double fused_c[4] = {0.0, 0.0, 0.0, 0.0};
};

namespace inti {

// Applies of this many columns or more (FP64 3D operators, every kernel) take the
// multi-column MMA kernel instead of one pair product per column.
constexpr int kMrhsMinColumns = 8;

void sync_and_check(inti_ctx* ctx);
PairLaunch make_launch(inti_op* op, const double* xdev);
void op_apply_device(inti_op* op, const double* x, double* y, const double* alpha,
                     const double* beta);
void op_apply_transpose_device(inti_op* op, const double* x, double* y, const double* alpha,
                               const double* beta);
inti_op* op_create(inti_ctx* ctx, int pde, int kernel, double k_re, double k_im,
                   const inti_quad* target, const inti_quad* source, const inti_csr* correction,
                   int precision);
inti_op* op_create_combined(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* target,
                            const inti_quad* source, const inti_csr* corr_dl, const inti_csr* corr_sl,
                            const double* c_dl, const double* c_sl, int precision);
inti_op* op_clone_precision(const inti_op* op, int precision);
// Launch shape of the pair kernel: the context's cached choice for this
// problem, else (measure = true, autotuning on, problem large enough) the
// fastest candidate timed now, else the occupancy heuristic.
void op_autotune(inti_op* op, bool measure);
// Square operators (target === source, every kernel, 2D and 3D): switch to
// the symmetric form when the context allows it and its column partials fit.
void op_symm_init(inti_op* op);
void op_symm_configure(inti_op* op, int tpt, int ch);
// Restrict the symmetric form to the work items of rank `rank` of `nranks`
// (round robin over the items, largest first); nranks = 1 lifts it.
void op_set_shard(inti_op* op, int rank, int nranks);
std::unique_ptr<inti_csr> merge_corrections(inti_ctx* ctx, const inti_csr* a, const double* ca,
                                            const inti_csr* b, const double* cb, int64_t m, int64_t n,
                                            bool cplx);
void op_prepare_transpose(inti_op* op);
int transposed_kind(int kind);
inti_csr* csr_create_host(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz,
                          const int64_t* rowptr, const int32_t* col, const double* val,
                          int dtype);
std::unique_ptr<inti_csr> csr_transpose(inti_ctx* ctx, const inti_csr* c);

void dim_correction_targets(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* target,
                            const inti_quad* q, int derivative, const double* green_multiplier, double maxdist,
                            inti_csr** dS, inti_csr** dD);
void dim_correction(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* q,
                    int derivative, const double* green_multiplier, inti_csr** dS,
                    inti_csr** dD);
void gmres_solve(inti_ctx* ctx, int32_t nterms, inti_op* const* ops, const double* coefs,
                 const double* shift, const double* b, double* x, double rtol, int32_t restart,
                 int32_t maxiter, int32_t mode, int on_device, double* history,
                 inti_gmres_stats* stats);
void grad_sources(inti_op* op, const double* g, const double* sigma, double* dsigma,
                  double* dcoords, double* dnormals, double* dweights, int on_device);
void measure_peaks(inti_ctx* ctx, double* fp64, double* fp32, double* mufu);
void measure_peak_tf32(inti_ctx* ctx, double* tf32_flops);
void selftest_math(inti_ctx* ctx, double* out);
void selftest_wait_timeout(inti_ctx* ctx);

}  // namespace inti
