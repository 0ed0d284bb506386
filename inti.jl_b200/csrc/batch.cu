// Batched multi-right-hand-side operators: many surfaces of uneven size and
// many densities per surface in one launch (the batching form of the
// workloads: plane-wave right-hand sides on a batch of star surfaces).
//
// A batch holds S quadratures concatenated in one node array (segment s =
// nodes off[s] .. off[s+1]-1) and one operator kind for all of them; the
// product is block diagonal: Y_s = A_s X_s (+ corrections), each A_s the
// on-the-fly Nystrom operator of surface s.  Densities are column-major
// (node, rhs) over the concatenated nodes.
//
// Two arithmetic forms of the pair product:
//  * FP64 (mrhs_mma): a CTA owns 64 targets and 64 right-hand sides; per
//    source tile the CUDA cores evaluate each kernel value once into shared
//    memory and the warps multiply that tile with the staged densities on
//    the FP64 MMA path (fp64_mma.cuh).
//  * TF32 on the tensor cores (mrhs_tc.cu): the kernel tile is generated by
//    CUDA cores into shared memory and multiplied with the staged density
//    block by tcgen05.mma into a TMEM accumulator.
// Work items are (surface, 128-target block) ordered by surface size,
// largest first, so the uneven surfaces balance across the SMs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <numeric>
#include <vector>

#include "batch.h"
#include "common.h"
#include "device_common.cuh"
#include "fp64_mma.cuh"
#include "internal.h"

namespace inti {

// Complex kernel value K(x, y) without the 1/(4 pi) factor, fast math
// (rsqrt_fast, table e^{ikd}); kind SL, DL or CF (= c1*DL + c2*SL with the
// coefficients applied by the caller through the returned pair).
struct KPair {
  double2 dl, sl;
};

__device__ __forceinline__ KPair helm_kernels(const double* x, const double* y, const double* ny, double k,
                                              double kT, double delta, const double2* tab, bool want_dl,
                                              bool want_sl) {
  const double r0 = x[0] - y[0], r1 = x[1] - y[1], r2 = x[2] - y[2];
  const double d2 = fma(r2, r2, fma(r1, r1, r0 * r0));
  const bool keep = pair_keep(d2);
  const double ri = keep ? rsqrt_fast(d2) : 0.0;
  const double d = d2 * ri;
  double cs, sn;
  expi_table_eval(d, kT, tab, delta, cs, sn);
  KPair o;
  o.sl = make_double2(0.0, 0.0);
  o.dl = make_double2(0.0, 0.0);
  if (want_sl) o.sl = make_double2(ri * cs, ri * sn);
  if (want_dl) {
    const double er = fma(cs, ri, k * sn), ei = fma(sn, ri, -k * cs);
    const double rn = fma(r2, ny[2], fma(r1, ny[1], r0 * ny[0]));
    const double f = rn * ri * ri;
    o.dl = make_double2(er * f, ei * f);
  }
  return o;
}

__device__ __forceinline__ double2 lap_kernels(const double* x, const double* y, const double* ny, double c1,
                                               double c2, int kind) {
  const double r0 = x[0] - y[0], r1 = x[1] - y[1], r2 = x[2] - y[2];
  const double d2 = fma(r2, r2, fma(r1, r1, r0 * r0));
  const bool keep = pair_keep(d2);
  const double ri = keep ? rsqrt_fast(d2) : 0.0;
  double v = 0.0;
  if (kind != SL) {
    const double rn = fma(r2, ny[2], fma(r1, ny[1], r0 * ny[0]));
    v = rn * ri * ri * ri * (kind == CF ? c1 : 1.0);
  }
  if (kind != DL) v = fma(ri, kind == CF ? c2 : 1.0, v);
  return make_double2(v, 0.0);
}

// Adjoint double layer (KIND ADL) or hypersingular (HS) value without the
// 1/(4 pi) factor, with the target normal nx: ADL = -e^{ikd}(1/d - ik)(r.n_x)/d^2
// (Laplace: -(r.n_x)/d^3); HS = e^{ikd} [(1/d - ik) p + (k^2 d^2 - 3 + 3ikd) s]
// with p = (n_x.n_y)/d^2, s = (r.n_x)(r.n_y)/d^5 (Laplace: (n_x.n_y - 3 (r.n_x)(r.n_y)/d^2)/d^3).
template <int PDE, int KIND>
__device__ __forceinline__ double2 normal_kernels(const double* x, const double* nx, const double* y,
                                                  const double* ny, double k, double kT, double delta,
                                                  const double2* tab) {
  const double r0 = x[0] - y[0], r1 = x[1] - y[1], r2 = x[2] - y[2];
  const double d2 = fma(r2, r2, fma(r1, r1, r0 * r0));
  const double ri = pair_keep(d2) ? rsqrt_fast(d2) : 0.0;
  const double id2 = ri * ri;
  const double rnx = fma(r2, nx[2], fma(r1, nx[1], r0 * nx[0]));
  if (PDE == LAPLACE) {
    if (KIND == ADL) return make_double2(-rnx * (id2 * ri), 0.0);
    const double rny = fma(r2, ny[2], fma(r1, ny[1], r0 * ny[0]));
    const double nn = fma(nx[2], ny[2], fma(nx[1], ny[1], nx[0] * ny[0]));
    return make_double2(fma(-3.0 * rnx * rny, id2, nn) * (id2 * ri), 0.0);
  }
  const double d = d2 * ri;
  double cs, sn;
  expi_table_eval(d, kT, tab, delta, cs, sn);
  if (KIND == ADL) {
    const double f = -rnx * id2;
    return make_double2(f * fma(cs, ri, k * sn), f * fma(sn, ri, -k * cs));
  }
  const double rny = fma(r2, ny[2], fma(r1, ny[1], r0 * ny[0]));
  const double nn = fma(nx[2], ny[2], fma(nx[1], ny[1], nx[0] * ny[0]));
  const double kd = k * d;
  const double fr = fma(kd, kd, -3.0), fi = 3.0 * kd;
  const double p = nn * id2;
  const double s5 = (rnx * rny) * (id2 * id2 * ri);
  const double wr = fma(ri, p, fr * s5), wi = fma(-k, p, fi * s5);
  return make_double2(fma(cs, wr, -sn * wi), fma(cs, wi, sn * wr));
}

constexpr int kMrhsBlock = 128;  // targets per work item

// FP64 form on the MMA path: one CTA = 64 targets x 64 right-hand sides;
// per tile of kMmaJ sources the CUDA cores evaluate K(x_i, y_j) w_j once per
// pair into A (complex: slots (Re, Im)), the density rows are staged as B
// (complex: row Re -> (Xr, Xi), row Im -> (-Xi, Xr) per column, so the
// accumulator pairs are (Re, Im) of Y), and the warps multiply A B with the
// FP64 MMA.  The next tile's densities and source records are loaded into
// registers while the MMA runs and stored to shared memory after it.
// Grid: x = 2 per 128-target work item, y = groups of RHS columns.  RHS =
// columns per CTA: 64, or 16 (complex) / 32 (real) for narrow applies.
constexpr int kMmaJ = 24;
constexpr int kMmaSrcVals = 7 * kMmaJ;  // x, n, w per source
static_assert(kMmaSrcVals <= kMmaThreads, "staging split");

template <bool CPLX, int RHS>
struct MrhsShape {
  static constexpr int NA = CPLX ? 2 : 1;
  using Sh = MmaShape<2, 4, RHS * NA / 32, kMmaJ * NA, CPLX ? 2 : 1>;
  static_assert(Sh::NCOL == RHS * NA, "columns");
  static constexpr int XPER = (kMmaJ * RHS + kMmaThreads - 1) / kMmaThreads;  // densities per thread
  static constexpr size_t smem_bytes() {
    return sizeof(double) * ((size_t)Sh::MT * Sh::LDA + (size_t)Sh::kK * Sh::LDB + kMmaSrcVals) +
           (CPLX ? sizeof(double2) * kExpiTable : 0);
  }
};

template <int PDE, int KIND, int RHS>
__global__ void __launch_bounds__(kMmaThreads, 2) mrhs_mma(BatchArgs a) {
  constexpr bool CPLX = PDE == HELMHOLTZ;
  using MS = MrhsShape<CPLX, RHS>;
  using Sh = typename MS::Sh;
  constexpr int NA = MS::NA;
  constexpr int XPER = MS::XPER;
  static_assert(Sh::MT == 64 && kMmaThreads % Sh::MT == 0 && kMmaJ % (kMmaThreads / Sh::MT) == 0, "shape");
  extern __shared__ __align__(16) double smem_d[];
  double* As = smem_d;
  double* Bs = As + Sh::MT * Sh::LDA;
  double* ssrc = Bs + Sh::kK * Sh::LDB;  // [x y z](J) [n](J) [w](J)
  double* sx = ssrc;
  double* sn = ssrc + 3 * kMmaJ;
  double* sw = ssrc + 6 * kMmaJ;
  double2* tab = reinterpret_cast<double2*>(ssrc + kMmaSrcVals);
  const int tid = threadIdx.x;
  const int item = blockIdx.x >> 1;
  // targets toff + [0, tn), sources off + [0, n) (one surface, or the operator)
  int64_t toff, tn, off, n, blk;
  const double* tc;
  if (a.tcoords) {
    toff = 0;
    tn = a.gm;
    off = 0;
    n = a.gn;
    blk = item;
    tc = a.tcoords;
  } else {
    const int s = a.item_surf[item];
    off = toff = a.off[s];
    n = tn = a.off[s + 1] - off;
    blk = a.item_block[item];
    tc = a.coords;
  }
  const int64_t base = blk * 128 + (blockIdx.x & 1) * Sh::MT;
  if (base >= tn) return;  // second half of a short last block (uniform per CTA)
  const int c0 = blockIdx.y * RHS;
  const int ncol = min(RHS, a.nrhs - c0);
  if (CPLX)
    for (int q = tid; q < kExpiTable; q += kMmaThreads) tab[q] = a.expi[q];
  // phase-1 role: target m, sources r0, r0 + R, ...
  constexpr int R = kMmaThreads / Sh::MT;
  const int m = tid % Sh::MT, r0 = tid / Sh::MT;
  const int64_t i = toff + min(base + m, tn - 1);
  const double xi[3] = {tc[3 * i], tc[3 * i + 1], tc[3 * i + 2]};
  constexpr bool TN = KIND == ADL || KIND == HS;  // kernels with the target normal
  double ni[3] = {0.0, 0.0, 0.0};
  if (TN) {
    const double* tnr = a.tcoords ? a.tnormals : a.normals;
    ni[0] = tnr[3 * i];
    ni[1] = tnr[3 * i + 1];
    ni[2] = tnr[3 * i + 2];
  }
  const double kT = a.k * kExpiTable / (2 * kPi), delta = 2 * kPi / kExpiTable;
  // staging roles: density element e = tid + r*256 -> (source e % J, column e / J)
  // (consecutive threads read consecutive nodes of one column); source value tid
  double2 xpre[XPER];
  double spre = 0.0;
  auto prefetch = [&](int64_t j0) {
#pragma unroll
    for (int r = 0; r < XPER; ++r) {
      const int e = tid + r * kMmaThreads, q = e % kMmaJ, c = e / kMmaJ;
      const int64_t j = j0 + q;
      double2 v = make_double2(0.0, 0.0);
      if (j < n && c < ncol) {  // c < ncol <= RHS also bounds e < J * RHS
        const int64_t idx = (int64_t)(c0 + c) * a.ldx + off + j;
        v = CPLX ? reinterpret_cast<const double2*>(a.x)[idx] : make_double2(a.x[idx], 0.0);
      }
      xpre[r] = v;
    }
    if (tid < kMmaSrcVals) {
      const int f = tid / kMmaJ, q = tid % kMmaJ;  // field 0..6 of source q
      const int64_t j = j0 + q;
      double v = 0.0;
      if (j < n) {
        if (f < 3) v = a.coords[3 * (off + j) + f];
        else if (f < 6) v = a.normals ? a.normals[3 * (off + j) + f - 3] : 0.0;
        else v = a.weights[off + j];
      }
      spre = v;
    }
  };
  auto store_staged = [&]() {
#pragma unroll
    for (int r = 0; r < XPER; ++r) {
      const int e = tid + r * kMmaThreads, q = e % kMmaJ, c = e / kMmaJ;
      if (c >= RHS) continue;  // (J * RHS not a multiple of the block)
      const double2 v = xpre[r];
      if (CPLX) {
        const int col = Sh::bcol(2 * q, 2 * c);
        *reinterpret_cast<double2*>(&Bs[(2 * q) * Sh::LDB + col]) = v;
        *reinterpret_cast<double2*>(&Bs[(2 * q + 1) * Sh::LDB + col]) = make_double2(-v.y, v.x);
      } else {
        Bs[q * Sh::LDB + Sh::bcol(q, c)] = v.x;
      }
    }
    if (tid < kMmaSrcVals) {
      const int f = tid / kMmaJ, q = tid % kMmaJ;
      if (f < 3) sx[3 * q + f] = spre;
      else if (f < 6) sn[3 * q + f - 3] = spre;
      else sw[q] = spre;
    }
  };
  double acc[4][Sh::kNT][2];
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < Sh::kNT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
  prefetch(0);
  for (int64_t j0 = 0; j0 < n; j0 += kMmaJ) {
    __syncthreads();  // the previous tile's A and B are consumed
    store_staged();
    __syncthreads();
    // phase 1: kernel values into A
#pragma unroll 2
    for (int q = r0; q < kMmaJ; q += R) {
      double2 kv;
      if (TN) {
        kv = normal_kernels<PDE, KIND>(xi, ni, &sx[3 * q], &sn[3 * q], a.k, kT, delta, tab);
      } else if (CPLX) {
        const KPair kp = helm_kernels(xi, &sx[3 * q], &sn[3 * q], a.k, kT, delta, tab, KIND != SL, KIND != DL);
        if (KIND == SL)
          kv = kp.sl;
        else if (KIND == DL)
          kv = kp.dl;
        else
          kv = make_double2(a.c1r * kp.dl.x - a.c1i * kp.dl.y + a.c2r * kp.sl.x - a.c2i * kp.sl.y,
                            a.c1r * kp.dl.y + a.c1i * kp.dl.x + a.c2r * kp.sl.y + a.c2i * kp.sl.x);
      } else {
        kv = lap_kernels(xi, &sx[3 * q], &sn[3 * q], a.c1r, a.c2r, KIND);
      }
      const double w = sw[q];
      if (CPLX) {
        *reinterpret_cast<double2*>(&As[m * Sh::LDA + NA * q]) = make_double2(kv.x * w, kv.y * w);
      } else {
        As[m * Sh::LDA + q] = kv.x * w;
      }
    }
    __syncthreads();
    if (j0 + kMmaJ < n) prefetch(j0 + kMmaJ);  // in flight during the MMA phase
    // phase 2: Y += A B on the FP64 MMA path
    mma_tile<Sh>(As, Bs, acc);
  }
  const double sc = 1.0 / (4 * kPi);
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int64_t il = base + mma_row<Sh>(mt);
    if (il >= tn) continue;
    const int64_t iy = toff + il;
#pragma unroll
    for (int nt = 0; nt < Sh::kNT; ++nt) {
      const int col = mma_col<Sh>(nt);
      if (CPLX) {
        const int c = col / 2;
        if (c >= ncol) continue;
        const int64_t idx = (int64_t)(c0 + c) * a.ldy + iy;
        const double yr = sc * acc[mt][nt][0], yi = sc * acc[mt][nt][1];
        double orr = a.ar * yr - a.ai * yi, oi = a.ar * yi + a.ai * yr;
        double2* Y = reinterpret_cast<double2*>(a.y);
        if (!a.beta_zero) {
          const double2 yo = Y[idx];
          orr += a.br * yo.x - a.bi * yo.y;
          oi += a.br * yo.y + a.bi * yo.x;
        }
        Y[idx] = make_double2(orr, oi);
      } else {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = col + e;
          if (c >= ncol) continue;
          const int64_t idx = (int64_t)(c0 + c) * a.ldy + iy;
          double o = a.ar * sc * acc[mt][nt][e];
          if (!a.beta_zero) o += a.br * a.y[idx];
          a.y[idx] = o;
        }
      }
    }
  }
}

// Multi-column CSR correction: Y[c][i] += alpha * sum_p val[p] X[c][col[p]]
template <bool CPLX>
__global__ void csr_mrhs(int64_t m, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                        const double* __restrict__ val, const double* __restrict__ x, int64_t ldx, double* y,
                        int64_t ldy, int nrhs, double ar, double ai) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (i >= m || c >= nrhs) return;
  double sr = 0.0, si = 0.0;
  for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) {
    const int64_t j = (int64_t)c * ldx + col[p];
    if (CPLX) {
      const double2 v = reinterpret_cast<const double2*>(val)[p];
      const double2 xv = reinterpret_cast<const double2*>(x)[j];
      sr = fma(v.x, xv.x, fma(-v.y, xv.y, sr));
      si = fma(v.x, xv.y, fma(v.y, xv.x, si));
    } else {
      sr = fma(val[p], x[j], sr);
    }
  }
  const int64_t o = (int64_t)c * ldy + i;
  if (CPLX) {
    double2* Y = reinterpret_cast<double2*>(y);
    double2 yo = Y[o];
    yo.x += ar * sr - ai * si;
    yo.y += ar * si + ai * sr;
    Y[o] = yo;
  } else {
    y[o] += ar * sr;
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
inti_batch* batch_create(inti_ctx* ctx, int32_t nsurf, const inti_quad* const* quads, int pde, int kind,
                         double k_re, double k_im, const double* c_dl, const double* c_sl,
                         const inti_csr* const* corr_dl, const inti_csr* const* corr_sl) {
  if (nsurf < 1 || !quads) throw Error(INTI_E_ARG, "a batch needs at least one surface");
  if (pde != INTI_LAPLACE && pde != INTI_HELMHOLTZ) throw Error(INTI_E_ARG, "unknown pde");
  if (kind != SL && kind != DL && kind != CF) throw Error(INTI_E_ARG, "batch kernels are SL, DL or the combined field");
  if (pde == INTI_HELMHOLTZ && k_im != 0.0) throw Error(INTI_E_UNSUPPORTED, "complex wavenumbers are not implemented");
  const bool cplx = pde == INTI_HELMHOLTZ;
  double c1[2] = {1.0, 0.0}, c2[2] = {1.0, 0.0};
  if (kind == CF) {
    if (!c_dl || !c_sl) throw Error(INTI_E_ARG, "combined-field coefficients are NULL");
    c1[0] = c_dl[0];
    c1[1] = c_dl[1];
    c2[0] = c_sl[0];
    c2[1] = c_sl[1];
    if (!cplx && (c1[1] != 0.0 || c2[1] != 0.0))
      throw Error(INTI_E_UNSUPPORTED, "complex coefficients need a Helmholtz operator");
  }
  std::unique_ptr<inti_batch> b(new inti_batch());
  b->ctx = ctx;
  b->pde = pde;
  b->kind = kind;
  b->k = k_re;
  for (int q = 0; q < 2; ++q) {
    b->c1[q] = c1[q];
    b->c2[q] = c2[q];
  }
  b->off.assign(nsurf + 1, 0);
  for (int s = 0; s < nsurf; ++s) {
    const inti_quad* q = quads[s];
    if (!q) throw Error(INTI_E_ARG, "quadrature is NULL");
    if (q->ctx != ctx) throw Error(INTI_E_STATE, "quadrature belongs to another context");
    if (q->dim != 3) throw Error(INTI_E_UNSUPPORTED, "batches are 3D");
    if (kind != SL && !q->has_normals) throw Error(INTI_E_ARG, "double-layer kernels need normals");
    b->off[s + 1] = b->off[s] + q->n;
  }
  const int64_t ntot = b->off[nsurf];
  std::vector<double> X(3 * ntot), N(3 * ntot, 0.0), W(ntot);
  for (int s = 0; s < nsurf; ++s) {
    const inti_quad* q = quads[s];
    std::copy(q->h_coords.begin(), q->h_coords.end(), X.begin() + 3 * b->off[s]);
    if (q->has_normals) std::copy(q->h_normals.begin(), q->h_normals.end(), N.begin() + 3 * b->off[s]);
    std::copy(q->h_weights.begin(), q->h_weights.end(), W.begin() + b->off[s]);
  }
  b->coords.ensure(sizeof(double) * 3 * ntot);
  b->normals.ensure(sizeof(double) * 3 * ntot);
  b->weights.ensure(sizeof(double) * ntot);
  INTI_CUDA(cudaMemcpy(b->coords.p, X.data(), sizeof(double) * 3 * ntot, cudaMemcpyHostToDevice));
  INTI_CUDA(cudaMemcpy(b->normals.p, N.data(), sizeof(double) * 3 * ntot, cudaMemcpyHostToDevice));
  INTI_CUDA(cudaMemcpy(b->weights.p, W.data(), sizeof(double) * ntot, cudaMemcpyHostToDevice));
  b->h_off = b->off;
  b->d_off.ensure(sizeof(int64_t) * (nsurf + 1));
  INTI_CUDA(cudaMemcpy(b->d_off.p, b->off.data(), sizeof(int64_t) * (nsurf + 1), cudaMemcpyHostToDevice));
  // work items: (surface, 128-target block), largest surfaces first
  std::vector<int> order(nsurf);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int c) { return quads[a]->n > quads[c]->n; });
  std::vector<int32_t> isurf, iblk;
  for (int s : order)
    for (int64_t t = 0; t * kMrhsBlock < quads[s]->n; ++t) {
      isurf.push_back(s);
      iblk.push_back((int32_t)t);
    }
  b->nitems = (int)isurf.size();
  b->item_surf.ensure(sizeof(int32_t) * b->nitems);
  b->item_block.ensure(sizeof(int32_t) * b->nitems);
  INTI_CUDA(cudaMemcpy(b->item_surf.p, isurf.data(), sizeof(int32_t) * b->nitems, cudaMemcpyHostToDevice));
  INTI_CUDA(cudaMemcpy(b->item_block.p, iblk.data(), sizeof(int32_t) * b->nitems, cudaMemcpyHostToDevice));
  // block-diagonal correction c1*C_dl + c2*C_sl (or the single kernel's)
  std::vector<int64_t> rp(ntot + 1, 0);
  std::vector<int32_t> col;
  std::vector<double> val;
  const int comps = cplx ? 2 : 1;
  bool any = false;
  for (int s = 0; s < nsurf; ++s) {
    const inti_csr* a = corr_dl ? corr_dl[s] : nullptr;
    const inti_csr* c = corr_sl ? corr_sl[s] : nullptr;
    if (kind == SL) a = nullptr;
    if (kind == DL) c = nullptr;
    const int64_t ns = quads[s]->n;
    for (const inti_csr* m : {a, c})
      if (m && (m->m != ns || m->n != ns || m->dtype != (cplx ? INTI_C128 : INTI_F64)))
        throw Error(INTI_E_SHAPE, "a correction does not match its surface (size or dtype)");
    std::unique_ptr<inti_csr> merged;
    const double one[2] = {1.0, 0.0};
    if (a || c) {
      merged = merge_corrections(ctx, a, kind == CF ? c1 : one, c, kind == CF ? c2 : one, ns, ns, cplx);
      any = true;
      std::vector<int64_t> mrp(ns + 1);
      std::vector<int32_t> mcol(merged->nnz);
      std::vector<double> mval((size_t)merged->nnz * comps);
      INTI_CUDA(cudaMemcpy(mrp.data(), merged->rowptr.p, sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost));
      INTI_CUDA(cudaMemcpy(mcol.data(), merged->col.p, sizeof(int32_t) * merged->nnz, cudaMemcpyDeviceToHost));
      INTI_CUDA(cudaMemcpy(mval.data(), merged->val.p, sizeof(double) * comps * merged->nnz, cudaMemcpyDeviceToHost));
      for (int64_t i = 0; i < ns; ++i) {
        for (int64_t p = mrp[i]; p < mrp[i + 1]; ++p) {
          col.push_back((int32_t)(mcol[p] + b->off[s]));
          for (int q = 0; q < comps; ++q) val.push_back(mval[p * comps + q]);
        }
        rp[b->off[s] + i + 1] = (int64_t)col.size();
      }
    } else {
      for (int64_t i = 0; i < ns; ++i) rp[b->off[s] + i + 1] = (int64_t)col.size();
    }
  }
  if (any)
    b->corr.reset(csr_create_host(ctx, ntot, ntot, (int64_t)col.size(), rp.data(), col.data(), val.data(),
                                  cplx ? INTI_C128 : INTI_F64));
  b->expi = expi_table_f64(ctx);
  return b.release();
}

// Launch of the FP64 MMA kernel for one (pde, kind); the dynamic shared
// memory attribute is set once per kernel, outside any stream capture.
// blocks = 128-target work items; the column width per CTA is 64, or the
// narrow one when all columns fit in it.
static void mrhs_mma_launch(inti_ctx* ctx, int pde, int kind, const BatchArgs& a, int64_t blocks) {
  auto go = [&](auto pc, auto kc) {
    constexpr int P = decltype(pc)::value, K = decltype(kc)::value;
    constexpr int narrow = P == HELMHOLTZ ? 16 : 32;
    auto launch = [&](auto rc) {
      constexpr int RHS = decltype(rc)::value;
      constexpr size_t smem = MrhsShape<P == HELMHOLTZ, RHS>::smem_bytes();
      auto* kern = &mrhs_mma<P, K, RHS>;
      static std::once_flag once;
      std::call_once(once, [kern] {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      });
      const dim3 grid((unsigned)(2 * blocks), (unsigned)((a.nrhs + RHS - 1) / RHS));
      kern<<<grid, kMmaThreads, smem, ctx->stream>>>(a);
    };
    if (a.nrhs <= narrow)
      launch(std::integral_constant<int, narrow>());
    else
      launch(std::integral_constant<int, 64>());
  };
  using H = std::integral_constant<int, HELMHOLTZ>;
  using Lp = std::integral_constant<int, LAPLACE>;
  auto by_kind = [&](auto pc) {
    switch (kind) {
      case SL: return go(pc, std::integral_constant<int, SL>());
      case DL: return go(pc, std::integral_constant<int, DL>());
      case ADL: return go(pc, std::integral_constant<int, ADL>());
      case HS: return go(pc, std::integral_constant<int, HS>());
      default: return go(pc, std::integral_constant<int, CF>());
    }
  };
  if (pde == INTI_HELMHOLTZ)
    by_kind(H());
  else
    by_kind(Lp());
  ctx->launches++;
  INTI_CUDA(cudaGetLastError());
}

void batch_apply_device(inti_batch* b, int precision, const double* x, int64_t ldx, double* y, int64_t ldy,
                        int32_t nrhs, const double* alpha, const double* beta) {
  inti_ctx* ctx = b->ctx;
  const bool cplx = b->pde == INTI_HELMHOLTZ;
  BatchArgs a;
  a.off = b->d_off.as<int64_t>();
  a.item_surf = b->item_surf.as<int32_t>();
  a.item_block = b->item_block.as<int32_t>();
  a.coords = b->coords.as<double>();
  a.normals = b->normals.as<double>();
  a.weights = b->weights.as<double>();
  a.x = x;
  a.ldx = ldx;
  a.y = y;
  a.ldy = ldy;
  a.nrhs = nrhs;
  a.k = b->k;
  a.c1r = b->c1[0];
  a.c1i = b->c1[1];
  a.c2r = b->c2[0];
  a.c2i = b->c2[1];
  a.ar = alpha ? alpha[0] : 1.0;
  a.ai = alpha ? alpha[1] : 0.0;
  a.br = beta ? beta[0] : 0.0;
  a.bi = beta ? beta[1] : 0.0;
  a.beta_zero = a.br == 0.0 && a.bi == 0.0;
  a.expi = b->expi;
  if (precision == INTI_TF32) {
    if (!cplx) throw Error(INTI_E_UNSUPPORTED, "the tensor-core form is implemented for Helmholtz");
    mrhs_tc_launch(b, a);
  } else if (precision == INTI_FP64) {
    ProfScope ps(ctx, "batch");
    mrhs_mma_launch(ctx, b->pde, b->kind, a, b->nitems);
  } else {
    throw Error(INTI_E_ARG, "batch precision must be FP64 or TF32");
  }
  INTI_CUDA(cudaGetLastError());
  if (b->corr) {
    const int64_t m = b->off.back();
    dim3 grid((unsigned)((m + 255) / 256), (unsigned)nrhs);
    if (cplx)
      csr_mrhs<true><<<grid, 256, 0, ctx->stream>>>(m, b->corr->rowptr.as<int64_t>(), b->corr->col.as<int32_t>(),
                                                    b->corr->val.as<double>(), x, ldx, y, ldy, nrhs, a.ar, a.ai);
    else
      csr_mrhs<false><<<grid, 256, 0, ctx->stream>>>(m, b->corr->rowptr.as<int64_t>(), b->corr->col.as<int32_t>(),
                                                     b->corr->val.as<double>(), x, ldx, y, ldy, nrhs, a.ar, a.ai);
    ctx->launches++;
    INTI_CUDA(cudaGetLastError());
  }
}

bool op_mrhs_supported(const inti_op* op) {
  const bool snormal = op->kind == DL || op->kind == CF || op->kind == HS;
  const bool tnormal = op->kind == ADL || op->kind == HS;
  return op->precision == INTI_FP64 && op->dim == 3 && (!snormal || op->source->has_normals) &&
         (!tnormal || op->target->has_normals);
}

void op_apply_mrhs(inti_op* op, const double* x, int64_t ldx, double* y, int64_t ldy, int32_t nrhs,
                   const double* alpha, const double* beta) {
  inti_ctx* ctx = op->ctx;
  const bool cplx = op->pde == INTI_HELMHOLTZ;
  BatchArgs a{};
  a.tcoords = op->target->coords.as<double>();
  a.tnormals = op->target->has_normals ? op->target->normals.as<double>() : nullptr;
  a.gm = op->target->n;
  a.gn = op->source->n;
  a.coords = op->source->coords.as<double>();
  a.normals = op->source->has_normals ? op->source->normals.as<double>() : nullptr;
  a.weights = op->source->weights.as<double>();
  a.x = x;
  a.ldx = ldx;
  a.y = y;
  a.ldy = ldy;
  a.nrhs = nrhs;
  a.k = op->k;
  // CF: c1*DL + c2*SL; single kernels ignore the coefficients
  a.c1r = op->c1[0];
  a.c1i = op->c1[1];
  a.c2r = op->c2[0];
  a.c2i = op->c2[1];
  a.ar = alpha ? alpha[0] : 1.0;
  a.ai = alpha ? alpha[1] : 0.0;
  a.br = beta ? beta[0] : 0.0;
  a.bi = beta ? beta[1] : 0.0;
  a.beta_zero = a.br == 0.0 && a.bi == 0.0;
  a.expi = cplx ? expi_table_f64(ctx) : nullptr;
  const int64_t blocks = (a.gm + kMrhsBlock - 1) / kMrhsBlock;
  {
    ProfScope ps(ctx, "mrhs");
    mrhs_mma_launch(ctx, op->pde, op->kind, a, blocks);
  }
  if (op->corr) {
    const inti_csr* c = op->corr;
    dim3 grid((unsigned)((a.gm + 255) / 256), (unsigned)nrhs);
    if (cplx)
      csr_mrhs<true><<<grid, 256, 0, ctx->stream>>>(a.gm, c->rowptr.as<int64_t>(), c->col.as<int32_t>(),
                                                    c->val.as<double>(), x, ldx, y, ldy, nrhs, a.ar, a.ai);
    else
      csr_mrhs<false><<<grid, 256, 0, ctx->stream>>>(a.gm, c->rowptr.as<int64_t>(), c->col.as<int32_t>(),
                                                     c->val.as<double>(), x, ldx, y, ldy, nrhs, a.ar, a.ai);
    ctx->launches++;
    INTI_CUDA(cudaGetLastError());
  }
}

// Rows [row0, row1) of Y += alpha*C*X for the block-diagonal correction (the
// rows of a group of surfaces in the pipelined host apply).
void batch_correction_rows(inti_batch* b, const double* x, int64_t ldx, double* y, int64_t ldy, int32_t nrhs,
                           double ar, double ai, int64_t row0, int64_t row1) {
  if (!b->corr || row1 <= row0) return;
  inti_ctx* ctx = b->ctx;
  const bool cplx = b->pde == INTI_HELMHOLTZ;
  const dim3 grid((unsigned)((row1 - row0 + 255) / 256), (unsigned)nrhs);
  const int64_t* rp = b->corr->rowptr.as<int64_t>() + row0;  // entries keep their global positions
  if (cplx)
    csr_mrhs<true><<<grid, 256, 0, ctx->stream>>>(row1 - row0, rp, b->corr->col.as<int32_t>(),
                                                  b->corr->val.as<double>(), x, ldx, y + 2 * row0, ldy, nrhs, ar, ai);
  else
    csr_mrhs<false><<<grid, 256, 0, ctx->stream>>>(row1 - row0, rp, b->corr->col.as<int32_t>(),
                                                   b->corr->val.as<double>(), x, ldx, y + row0, ldy, nrhs, ar, ai);
  ctx->launches++;
  INTI_CUDA(cudaGetLastError());
}

}  // namespace inti
