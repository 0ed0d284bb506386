// Batch handle and launch arguments shared by batch.cu (FP64 path, host)
// and mrhs_tc.cu (tensor-core path).  Internal.
#pragma once

#include <memory>
#include <vector>

#include "common.h"

struct inti_batch {
  inti_ctx* ctx = nullptr;
  int pde = INTI_HELMHOLTZ, kind = INTI_SL;
  double k = 0.0;
  double c1[2] = {1.0, 0.0}, c2[2] = {1.0, 0.0};
  std::vector<int64_t> off, h_off;  // node offsets of the surfaces (S+1)
  inti::DevBuf d_off, coords, normals, weights;
  inti::DevBuf item_surf, item_block;  // work items, largest surfaces first
  int nitems = 0;
  std::unique_ptr<inti_csr> corr;  // block-diagonal correction (global indices)
  const double2* expi = nullptr;
  // tensor-core path: packed density blocks and source records, tile
  // offsets, 256-target work items, work counter
  inti::DevBuf tc_b, tc_src, tc_counter, tc_toff, tc_items;
  inti::DevBuf xstage, ystage;  // staging for host-pointer applies
  // pipelined host-pointer TF32 apply: surface groups (contiguous surface
  // ranges grp_s[g] .. grp_s[g+1]-1), their items stored group after group
  // (largest surface first within a group) starting at grp_item[g], and the
  // copy streams and events
  std::vector<int> grp_s, grp_item;
  inti::DevBuf tc_items_grp;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  std::vector<cudaEvent_t> ev;
  ~inti_batch() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (s_in) cudaStreamDestroy(s_in);
    if (s_out) cudaStreamDestroy(s_out);
  }
  int64_t tc_ntiles = 0;
  int tc_nitems = 0;
};

namespace inti {

struct BatchArgs {
  const int64_t* off;
  const int32_t* item_surf;
  const int32_t* item_block;
  const double* coords;
  const double* normals;
  const double* weights;
  const double* x;
  int64_t ldx;
  double* y;
  int64_t ldy;
  int nrhs;
  double k;
  double c1r, c1i, c2r, c2i;
  double ar, ai, br, bi;
  bool beta_zero;
  const double2* expi;
  // single-operator form of the FP64 MMA kernel (tcoords != null): targets
  // tcoords[0, gm), sources coords/normals/weights[0, gn), work item b =
  // target block b; off, item_surf and item_block are unused
  const double* tcoords = nullptr;
  const double* tnormals = nullptr;  // adjoint double layer / hypersingular
  int64_t gm = 0, gn = 0;
};

void mrhs_tc_launch(inti_batch* b, const BatchArgs& a);
// Host-pointer TF32 apply with the copies overlapped: surface groups are
// copied in, computed and copied out on three streams.
void batch_apply_host_tf32(inti_batch* b, const double* x, int64_t ldx, double* y, int64_t ldy, int32_t nrhs,
                           const double* alpha, const double* beta);
void batch_correction_rows(inti_batch* b, const double* x, int64_t ldx, double* y, int64_t ldy, int32_t nrhs,
                           double ar, double ai, int64_t row0, int64_t row1);
inti_batch* batch_create(inti_ctx* ctx, int32_t nsurf, const inti_quad* const* quads, int pde, int kind,
                         double k_re, double k_im, const double* c_dl, const double* c_sl,
                         const inti_csr* const* corr_dl, const inti_csr* const* corr_sl);
void batch_gmres(inti_batch* b, const double* shift, const double* B, double* X, int64_t ldb, int32_t nrhs,
                 double rtol, int32_t restart, int32_t maxiter, int32_t mode, int on_device, double* relres_out,
                 inti_gmres_stats* stats);
void batch_apply_device(inti_batch* b, int precision, const double* x, int64_t ldx, double* y, int64_t ldy,
                        int32_t nrhs, const double* alpha, const double* beta);
// y = alpha*(A + C) x + beta*y for nrhs device columns of a 3D FP64 SL, DL or
// combined-field operator, each kernel value evaluated once for 64 columns
// (the batch FP64 MMA kernel in single-operator form).
bool op_mrhs_supported(const inti_op* op);
void op_apply_mrhs(inti_op* op, const double* x, int64_t ldx, double* y, int64_t ldy, int32_t nrhs,
                   const double* alpha, const double* beta);

}  // namespace inti
