// On-the-fly Nyström pair product y = A x, A_ij = K(x_i, y_j) w_j
// (src/nystrom.jl:93-96 entries; src/nystrom.jl:117-124 is the CPU loop it
// replaces), for the Laplace (2D/3D) and Helmholtz (3D) single-layer,
// double-layer, adjoint-double-layer and hypersingular kernels
// (src/kernels.jl:137-204, 347-413).
//
// Design (B200, sm_100a):
//  * A pack kernel folds the density into per-source records
//    (coordinates + w*sigma, or the dipole w*sigma*n for DL/HS), padded to
//    whole tiles with zero charges.
//  * The pair kernel gives each thread TPT targets held in registers.  Source
//    tiles are streamed into shared memory by the TMA bulk-copy engine
//    (cp.async.bulk + mbarrier, two stages, one elected thread issues) and
//    read back as broadcasts.  Each CTA covers one target block and one chunk
//    of the source tiles (grid.y = split), so every SM stays busy even when
//    the target count is small; partial sums go to scratch and are reduced in
//    a fixed order by the epilogue (deterministic, no atomics).
//  * FP64 form: FP64 pairs and sums.  FP32C form: FP32 pairs, summed in FP32
//    over groups of 32 sources, groups folded into a (sum, compensation)
//    pair with Knuth's TwoSum (error-free), so the long sum over N sources
//    carries no O(N eps) growth.
//  * The epilogue applies the kernel constant, alpha/beta, and the CSR
//    correction row in the same pass (the fused near-field correction).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "common.h"
#include "device_common.cuh"

namespace inti {

constexpr int kBlock = 128;  // threads per CTA
constexpr int kTPT = 4;      // targets per thread
constexpr int kTile64 = 128; // sources per shared-memory stage (FP64)
constexpr int kTile32 = 256; // sources per shared-memory stage (FP32C)
constexpr int kGroup = 32;   // FP32C: sources summed before a compensated fold

// ---------------------------------------------------------------------------
// Source record layouts (elements of R per source):
//   Laplace  SL/ADL : x y [z] q            (q = w*sigma)
//   Laplace  DL/HS  : x y [z] p_x p_y [p_z] (p = w*sigma*n_y)
//   Helmholtz SL/ADL: x y z qr qi
//   Helmholtz DL/HS : x y z pr_x pr_y pr_z pi_x pi_y pi_z
// each padded so that a record is a multiple of 16 bytes.
// ---------------------------------------------------------------------------
//   combined field (CF): x y z | dipole c1*w*sigma*n_y | charge c2*w*sigma
template <int PDE, int KIND, int DIM, class R>
struct Rec {
  static constexpr bool dipole = (KIND == DL || KIND == HS || KIND == CF);
  static constexpr bool charge2 = (KIND == CF);
  static constexpr bool cplx = (PDE == HELMHOLTZ);
  static constexpr int used = DIM + (cplx ? 2 : 1) * ((dipole ? DIM : 1) + (charge2 ? 1 : 0));
  static constexpr int align = 16 / sizeof(R);
  static constexpr int n = (used + align - 1) / align * align;
  static constexpr bool tnormal = (KIND == ADL || KIND == HS);
};

// Record of source j (zero past n: a zero charge at the origin, which adds
// nothing to any target).
template <int PDE, int KIND, int DIM, class R>
__device__ __forceinline__ void build_record(int64_t j, int64_t n, const double* __restrict__ xs,
                                             const double* __restrict__ ns, const double* __restrict__ w,
                                             const double* __restrict__ sigma, double2 c1, double2 c2,
                                             R (&rec)[Rec<PDE, KIND, DIM, R>::n]) {
  using RC = Rec<PDE, KIND, DIM, R>;
#pragma unroll
  for (int c = 0; c < RC::n; ++c) rec[c] = R(0);
  if (j >= n) return;
#pragma unroll
  for (int c = 0; c < DIM; ++c) rec[c] = R(xs[DIM * j + c]);
  const double wj = w[j];
  double qr, qi = 0.0;
  if (RC::cplx) {
    qr = wj * sigma[2 * j];
    qi = wj * sigma[2 * j + 1];
  } else {
    qr = wj * sigma[j];
  }
  if (RC::charge2) {
    // monopole charge c2*q after the dipole block
    const double mr = c2.x * qr - c2.y * qi, mi = c2.x * qi + c2.y * qr;
    rec[DIM + (RC::cplx ? 2 : 1) * DIM] = R(mr);
    if (RC::cplx) rec[DIM + 2 * DIM + 1] = R(mi);
    const double dr = c1.x * qr - c1.y * qi, di = c1.x * qi + c1.y * qr;
    qr = dr;
    qi = di;
  }
  if (RC::dipole) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      rec[DIM + c] = R(qr * ns[DIM * j + c]);
      if (RC::cplx) rec[2 * DIM + c] = R(qi * ns[DIM * j + c]);
    }
  } else {
    rec[DIM] = R(qr);
    if (RC::cplx) rec[DIM + 1] = R(qi);
  }
}

template <int PDE, int KIND, int DIM, class R>
__global__ void pack_sources(int64_t n, int64_t npad, const double* __restrict__ xs,
                             const double* __restrict__ ns, const double* __restrict__ w,
                             const double* __restrict__ sigma, double2 c1, double2 c2,
                             R* __restrict__ out) {
  using RC = Rec<PDE, KIND, DIM, R>;
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= npad) return;
  R rec[RC::n];
  build_record<PDE, KIND, DIM, R>(j, n, xs, ns, w, sigma, c1, c2, rec);
  R* o = out + j * RC::n;
#pragma unroll
  for (int c = 0; c < RC::n; ++c) o[c] = rec[c];
}

// ---------------------------------------------------------------------------
// Per-pair accumulation.  Kernel constants (1/(4pi), signs) are applied once
// in the epilogue; the self pair (|r|^2 <= tol^2) contributes exactly zero.
// ---------------------------------------------------------------------------
template <class R>
struct MathOps;
template <>
struct MathOps<double> {
  using R2 = double2;
  static __device__ __forceinline__ double rsq(double v) { return rsqrt_fast(v); }
  static __device__ __forceinline__ double rsq3(double v) { return rsqrt_cube_fast(v); }
  static __device__ __forceinline__ double rcp(double v) { return rcp_fast(v); }
  static __device__ __forceinline__ double lg(double v) { return log(v); }
  static __device__ __forceinline__ bool keep(double d2) { return pair_keep(d2); }
};
template <>
struct MathOps<float> {
  using R2 = float2;
  static __device__ __forceinline__ float rsq(float v) { return rsqrt_fast(v); }
  static __device__ __forceinline__ float rsq3(float v) { return rsqrt_cube_fast(v); }
  static __device__ __forceinline__ float rcp(float v) { return 1.0f / v; }
  static __device__ __forceinline__ float lg(float v) { return __logf(v); }
  static __device__ __forceinline__ bool keep(float d2) { return d2 > 1.0e-28f; }
};

template <class R, int DIM, bool TN>
struct Target {
  R x[DIM];
  R n[TN ? DIM : 1];
};

// Helmholtz phase: e^{ikd} = expi(d * kT) with kT = k*kExpiTable/(2 pi)
// (table + Taylor, see expi_table_eval).
struct HelmConst {
  double kT, delta;
};

template <int PDE, int KIND, int DIM, class R>
__device__ __forceinline__ void pair_step(const Target<R, DIM, Rec<PDE, KIND, DIM, R>::tnormal>& t,
                                          const R* __restrict__ s, R kT, R delta, R k,
                                          const typename MathOps<R>::R2* __restrict__ tab, R& ar, R& ai) {
  using M = MathOps<R>;
  R r[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) r[c] = t.x[c] - s[c];
  R d2 = r[0] * r[0];
#pragma unroll
  for (int c = 1; c < DIM; ++c) d2 = fma(r[c], r[c], d2);
  const bool keep = M::keep(d2);
  if (PDE == LAPLACE) {
    if (KIND == SL) {
      if (DIM == 2) {
        // -log(d)/(2pi) = log(d^2) * (-1/(4pi)); constant in the epilogue
        const R l = M::lg(d2);
        ar += keep ? l * s[2] : R(0);
      } else {
        const R ri = keep ? M::rsq(d2) : R(0);
        ar = fma(ri, s[3], ar);
      }
    } else if (KIND == DL || KIND == CF) {
      R rp = r[0] * s[DIM];
#pragma unroll
      for (int c = 1; c < DIM; ++c) rp = fma(r[c], s[DIM + c], rp);
      if (DIM == 2) {
        const R ri = keep ? M::rcp(d2) : R(0);
        ar = fma(rp, ri, ar);
      } else if (KIND == CF) {
        const R ri = keep ? M::rsq(d2) : R(0);
        ar = fma(ri, s[2 * DIM], ar);
        ar = fma(rp, ri * ri * ri, ar);
      } else {
        ar = fma(rp, keep ? M::rsq3(d2) : R(0), ar);
      }
    } else if (KIND == ADL) {
      R rn = r[0] * t.n[0];
#pragma unroll
      for (int c = 1; c < DIM; ++c) rn = fma(r[c], t.n[c], rn);
      const R q = s[DIM];
      if (DIM == 2) {
        const R ri = keep ? M::rcp(d2) : R(0);
        ar = fma(rn * q, ri, ar);
      } else {
        ar = fma(rn * q, keep ? M::rsq3(d2) : R(0), ar);
      }
    } else {  // HS: (nx.p - DIM (r.nx)(r.p)/d^2) / d^DIM
      R rn = r[0] * t.n[0], rp = r[0] * s[DIM], np = t.n[0] * s[DIM];
#pragma unroll
      for (int c = 1; c < DIM; ++c) {
        rn = fma(r[c], t.n[c], rn);
        rp = fma(r[c], s[DIM + c], rp);
        np = fma(t.n[c], s[DIM + c], np);
      }
      if (DIM == 2) {
        const R id2 = keep ? M::rcp(d2) : R(0);
        ar = fma(id2, fma(R(-2) * rn * rp, id2, np), ar);
      } else {
        const R ri = keep ? M::rsq(d2) : R(0);
        const R id2 = ri * ri;
        ar = fma(id2 * ri, fma(R(-3) * rn * rp, id2, np), ar);
      }
    }
  } else {  // Helmholtz 3D
    const R ri = keep ? M::rsq(d2) : R(0);
    const R d = d2 * ri;  // 0 for the self pair
    R sn, cs;
    expi_table_eval(d, kT, tab, delta, cs, sn);
    if (KIND == SL || KIND == ADL) {
      R g_r, g_i;  // G (without 1/4pi) or the ADL factor
      if (KIND == SL) {
        g_r = ri * cs;
        g_i = ri * sn;
      } else {
        // e^{ikd}(1/d - ik) (r.nx) / d^2
        const R er = fma(cs, ri, k * sn), ei = fma(sn, ri, -k * cs);
        R rn = r[0] * t.n[0];
        rn = fma(r[1], t.n[1], rn);
        rn = fma(r[2], t.n[2], rn);
        const R f = rn * ri * ri;
        g_r = er * f;
        g_i = ei * f;
      }
      const R qr = s[3], qi = s[4];
      ar = fma(g_r, qr, fma(-g_i, qi, ar));
      ai = fma(g_r, qi, fma(g_i, qr, ai));
    } else if (KIND == DL || KIND == CF) {
      const R er = fma(cs, ri, k * sn), ei = fma(sn, ri, -k * cs);
      const R id2 = ri * ri;
      R A = r[0] * s[3], B = r[0] * s[6];
      A = fma(r[1], s[4], A);
      A = fma(r[2], s[5], A);
      B = fma(r[1], s[7], B);
      B = fma(r[2], s[8], B);
      const R gr = er * id2, gi = ei * id2;
      ar = fma(gr, A, fma(-gi, B, ar));
      ai = fma(gr, B, fma(gi, A, ai));
      if (KIND == CF) {  // + e^{ikd}/d * (c2 w sigma)
        const R hr = cs * ri, hi = sn * ri;
        const R qr = s[9], qi = s[10];
        ar = fma(hr, qr, fma(-hi, qi, ar));
        ai = fma(hr, qi, fma(hi, qr, ai));
      }
    } else {  // HS
      const R id2 = ri * ri;
      R rn = r[0] * t.n[0];
      rn = fma(r[1], t.n[1], rn);
      rn = fma(r[2], t.n[2], rn);
      R A = r[0] * s[3], B = r[0] * s[6], NA = t.n[0] * s[3], NB = t.n[0] * s[6];
#pragma unroll
      for (int c = 1; c < 3; ++c) {
        A = fma(r[c], s[3 + c], A);
        B = fma(r[c], s[6 + c], B);
        NA = fma(t.n[c], s[3 + c], NA);
        NB = fma(t.n[c], s[6 + c], NB);
      }
      // value = a (r.nx)(r.p) + b (nx.p) with b = e^{ikd}(1/d - ik)/d^2,
      // a = e^{ikd}(k^2 d^2 - 3 + 3ikd)/d^5 and the complex dipole sums
      // r.p = A + iB, nx.p = NA + iNB; formed as e^{ikd} W with
      // W = (k^2 d^2 - 3 + 3ikd) U + (1/d - ik) P, U = (r.nx)(A + iB)/d^5,
      // P = (NA + iNB)/d^2
      const R kd = k * d;
      const R fr = fma(kd, kd, R(-3)), fi = R(3) * kd;
      const R u = rn * (id2 * id2 * ri);
      const R ur = u * A, ui = u * B, pr = NA * id2, pi = NB * id2;
      const R wr = fma(fr, ur, fma(-fi, ui, fma(ri, pr, k * pi)));
      const R wi = fma(fr, ui, fma(fi, ur, fma(ri, pi, -k * pr)));
      ar = fma(cs, wr, fma(-sn, wi, ar));
      ai = fma(cs, wi, fma(sn, wr, ai));
    }
  }
}

// Accumulator: FP64 plain; FP32 with a per-group sum and a TwoSum-folded
// (hi, lo) pair.
template <class R, bool CPLX>
struct Acc;
template <bool CPLX>
struct Acc<double, CPLX> {
  double r = 0, i = 0;
  __device__ __forceinline__ double& gr() { return r; }
  __device__ __forceinline__ double& gi() { return i; }
  __device__ __forceinline__ void fold() {}
};
__device__ __forceinline__ void two_sum_fold(float& hi, float& lo, float& g) {
  const float t = hi + g;
  const float bp = t - hi;
  const float e = (hi - (t - bp)) + (g - bp);
  hi = t;
  lo += e;
  g = 0.f;
}
template <bool CPLX>
struct Acc<float, CPLX> {
  float gr_ = 0, gi_ = 0, hr = 0, lr = 0, hi = 0, li = 0;
  __device__ __forceinline__ float& gr() { return gr_; }
  __device__ __forceinline__ float& gi() { return gi_; }
  __device__ __forceinline__ void fold() {
    two_sum_fold(hr, lr, gr_);
    if (CPLX) two_sum_fold(hi, li, gi_);
  }
};

// Partial accumulator storage per (split, target).
template <class R, bool CPLX>
struct PartialT;
template <>
struct PartialT<double, false> { using T = double; };
template <>
struct PartialT<double, true> { using T = double2; };
template <>
struct PartialT<float, false> { using T = float2; };
template <>
struct PartialT<float, true> { using T = float4; };

__device__ __forceinline__ void store_partial(double* p, const Acc<double, false>& a) { *p = a.r; }
__device__ __forceinline__ void store_partial(double2* p, const Acc<double, true>& a) {
  *p = make_double2(a.r, a.i);
}
__device__ __forceinline__ void store_partial(float2* p, const Acc<float, false>& a) {
  *p = make_float2(a.hr, a.lr);
}
__device__ __forceinline__ void store_partial(float4* p, const Acc<float, true>& a) {
  *p = make_float4(a.hr, a.lr, a.hi, a.li);
}

struct FwdArgs {
  int64_t m;
  int64_t n_tiles;
  int tiles_per_split;
  const double* tcoords;
  const double* tnormals;
  const void* packed;
  void* partial;
  double k;
  double kT, delta;   // Helmholtz phase scaling (see HelmConst)
  const void* expi;   // kExpiTable (cos, sin) entries in R precision
  int* err;
};

template <int PDE, int KIND, int DIM, class R, int TILE, int TPT = kTPT>
__global__ void __launch_bounds__(kBlock) pair_forward(FwdArgs a) {
  using RC = Rec<PDE, KIND, DIM, R>;
  constexpr bool CPLX = RC::cplx;
  using P = typename PartialT<R, CPLX>::T;
  using R2 = typename MathOps<R>::R2;
  constexpr uint32_t kStageBytes = TILE * RC::n * sizeof(R);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* stage0 = reinterpret_cast<R*>(smem_raw);
  R* stage1 = reinterpret_cast<R*>(smem_raw + kStageBytes);
  R2* tab = reinterpret_cast<R2*>(smem_raw + 2 * kStageBytes);  // Helmholtz only
  __shared__ __align__(8) uint64_t full[2];

  const int tid = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * (kBlock * TPT);
  const int split = blockIdx.y;
  const int64_t t0 = (int64_t)split * a.tiles_per_split;
  const int64_t t1 = min(a.n_tiles, t0 + a.tiles_per_split);
  const R* src = static_cast<const R*>(a.packed);

  Target<R, DIM, RC::tnormal> tg[TPT];
  Acc<R, CPLX> acc[TPT];
#pragma unroll
  for (int u = 0; u < TPT; ++u) {
    const int64_t i = min(base + u * kBlock + tid, a.m - 1);
#pragma unroll
    for (int c = 0; c < DIM; ++c) tg[u].x[c] = R(a.tcoords[DIM * i + c]);
    if (RC::tnormal) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) tg[u].n[c] = R(a.tnormals[DIM * i + c]);
    }
  }
  const R k = R(a.k);
  const R kT = R(a.kT);
  const R delta = R(a.delta);
  if (RC::cplx) {
    const R2* g = static_cast<const R2*>(a.expi);
    for (int q = tid; q < kExpiTable; q += kBlock) tab[q] = g[q];
  }

  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int64_t issued = t0;  // next tile to issue (meaningful in thread 0)
  if (tid == 0) {
    for (int s = 0; s < 2 && issued < t1; ++s, ++issued) {
      mbar_arrive_expect_tx(&full[s], kStageBytes);
      bulk_copy_g2s(s ? stage1 : stage0, src + issued * TILE * RC::n, kStageBytes, &full[s]);
    }
  }

  for (int64_t t = t0; t < t1; ++t) {
    const int st = (int)((t - t0) & 1);
    const uint32_t parity = (uint32_t)(((t - t0) >> 1) & 1);
    const bool ok = mbar_wait_bounded(&full[st], parity);
    if (!__syncthreads_and(ok)) {
      // A bulk copy never completed: record it, drain what is still in
      // flight (bounded), and leave without touching the results.
      if (tid == 0) {
        atomicExch(a.err, kErrWaitTimeout);
        for (int64_t q = t + 1; q < issued; ++q)
          mbar_wait_bounded(&full[(q - t0) & 1], (uint32_t)(((q - t0) >> 1) & 1));
      }
      return;
    }
    const R* sp = st ? stage1 : stage0;
#pragma unroll 1
    for (int g = 0; g < TILE; g += kGroup) {
#pragma unroll 2
      for (int s = 0; s < kGroup; ++s) {
        const R* rec = sp + (g + s) * RC::n;
#pragma unroll
        for (int u = 0; u < TPT; ++u)
          pair_step<PDE, KIND, DIM, R>(tg[u], rec, kT, delta, k, tab, acc[u].gr(), acc[u].gi());
      }
#pragma unroll
      for (int u = 0; u < TPT; ++u) acc[u].fold();
    }
    __syncthreads();  // every thread is done reading this stage
    if (tid == 0 && issued < t1) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&full[st], kStageBytes);
      bulk_copy_g2s(st ? stage1 : stage0, src + issued * TILE * RC::n, kStageBytes, &full[st]);
      ++issued;
    }
  }
  P* out = static_cast<P*>(a.partial) + (int64_t)split * a.m;
#pragma unroll
  for (int u = 0; u < TPT; ++u) {
    const int64_t i = base + u * kBlock + tid;
    if (i < a.m) store_partial(out + i, acc[u]);
  }
}

// ---------------------------------------------------------------------------
// Epilogue: y_i = alpha*(scale*sum_s partial[s][i] + sum_p C_ip x_p) + beta*y_i
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 load_partial(const double* p) { return make_double2(*p, 0.0); }
__device__ __forceinline__ double2 load_partial(const double2* p) { return *p; }
__device__ __forceinline__ double2 load_partial(const float2* p) {
  const float2 v = *p;
  return make_double2((double)v.x + (double)v.y, 0.0);
}
__device__ __forceinline__ double2 load_partial(const float4* p) {
  const float4 v = *p;
  return make_double2((double)v.x + (double)v.y, (double)v.z + (double)v.w);
}

struct EpiArgs {
  int64_t m;
  int split;
  const void* partial;
  double scale;
  const int64_t* rowptr;  // null when no correction
  const int32_t* col;
  const double* val;
  const double* x;
  double* y;
  double ar, ai, br, bi;
  bool beta_zero;
  const double* rowscale = nullptr;  // per-row factor of the pair sum (A^T: the source weights)
  const int* err = nullptr;          // when set and nonzero (a pair kernel timed out): y gets NaN
};

// y[i] before the product (read only when beta != 0).
template <bool CPLX>
__device__ __forceinline__ double2 epilogue_y_old(const EpiArgs& e, int64_t i) {
  return CPLX ? reinterpret_cast<const double2*>(e.y)[i] : make_double2(e.y[i], 0.0);
}

// y[i] = alpha * (sr, si) + beta * yo, yo the old y[i].
template <bool CPLX>
__device__ __forceinline__ void epilogue_store(const EpiArgs& e, int64_t i, double sr, double si, double2 yo) {
  if (CPLX) {
    double yr = e.ar * sr - e.ai * si, yi = e.ar * si + e.ai * sr;
    if (!e.beta_zero) {
      yr += e.br * yo.x - e.bi * yo.y;
      yi += e.br * yo.y + e.bi * yo.x;
    }
    reinterpret_cast<double2*>(e.y)[i] = make_double2(yr, yi);
  } else {
    double yr = e.ar * sr;
    if (!e.beta_zero) yr += e.br * yo.x;
    e.y[i] = yr;
  }
}

// Kernel constant, correction row, alpha/beta and the store for row i, given
// the row's pair sum (sr, si).
template <bool CPLX>
__device__ __forceinline__ void epilogue_finish(const EpiArgs& e, int64_t i, double sr, double si) {
  const double sc = e.rowscale ? e.scale * e.rowscale[i] : e.scale;
  sr *= sc;
  si *= sc;
  if (e.rowptr) {
    const int64_t p0 = e.rowptr[i], p1 = e.rowptr[i + 1];
    for (int64_t p = p0; p < p1; ++p) {
      const int32_t j = e.col[p];
      if (CPLX) {
        const double2 v = reinterpret_cast<const double2*>(e.val)[p];
        const double2 xv = reinterpret_cast<const double2*>(e.x)[j];
        sr = fma(v.x, xv.x, fma(-v.y, xv.y, sr));
        si = fma(v.x, xv.y, fma(v.y, xv.x, si));
      } else {
        sr = fma(e.val[p], e.x[j], sr);
      }
    }
  }
  epilogue_store<CPLX>(e, i, sr, si, e.beta_zero ? make_double2(0.0, 0.0) : epilogue_y_old<CPLX>(e, i));
}

template <class P, bool CPLX>
__global__ void pair_epilogue_kernel(EpiArgs e) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= e.m) return;
  if (e.err && *e.err) {  // the partial sums are incomplete: make the failure visible in y
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (CPLX)
      reinterpret_cast<double2*>(e.y)[i] = make_double2(nan, nan);
    else
      e.y[i] = nan;
    return;
  }
  const P* part = static_cast<const P*>(e.partial);
  double sr = 0.0, si = 0.0;
  for (int s = 0; s < e.split; ++s) {
    const double2 v = load_partial(part + (int64_t)s * e.m + i);
    sr += v.x;
    si += v.y;
  }
  epilogue_finish<CPLX>(e, i, sr, si);
}

// ---------------------------------------------------------------------------
// Single-launch form for small FP64 operators (m*n up to kSmallPairs, e.g.
// the 1,000-node kite): one kernel per product, no pack.  The tiled kernels
// give such a problem a handful of CTAs whose threads each run a long chain
// of dependent global loads, so the launch is latency-bound.  Here a
// cluster of S CTAs takes 32 targets (one per lane); CTA s of the cluster
// takes the s-th slice of the sources, builds their records in shared memory
// from the raw nodes (build_record, kSmallTile at a time), and its warps
// split each staged tile.  S is chosen on the host so that the clusters
// fill the SMs.  The correction row of a target is split over the same
// S * kSmallWarps threads (entry p0 + s*kSmallWarps + warp, then strides of
// S*kSmallWarps); the first kSmallCorr entries of a thread are fetched before
// the pair loop so their latency hides behind it.  The warps' pair and
// correction sums are added in a fixed order, then the slices' sums, read
// by CTA 0 of the cluster from its peers' shared memory (distributed shared
// memory), in slice order; CTA 0 then applies the kernel constant to the
// pair sum, adds the correction sum and alpha/beta.  The step is
// pair_step's (the one-sided kernel's arithmetic).
// ---------------------------------------------------------------------------
constexpr int kSmallWarps = 8;
constexpr int kSmallTile = 32 * kSmallWarps;  // sources staged per pass, one per thread
constexpr int kSmallMaxSlices = 8;            // portable cluster size
constexpr int kSmallCorr = 2;                 // correction entries per thread fetched ahead

struct SmallSources {
  const double *xs, *ns, *w, *sigma;
  double2 c1, c2;
};

template <int PDE, int KIND, int DIM>
__global__ void __launch_bounds__(32 * kSmallWarps) pair_small_kernel(int64_t m, int64_t n, const double* tc,
                                                                      const double* tn, SmallSources src,
                                                                      double k, double kT, double delta,
                                                                      const double2* expi, EpiArgs e) {
  namespace cg = cooperative_groups;
  using RC = Rec<PDE, KIND, DIM, double>;
  constexpr bool CPLX = RC::cplx;
  // the staged records; after the last tile, the warps' sums (pair, correction)
  __shared__ __align__(16) double recs[kSmallTile * RC::n];
  __shared__ double4 slice_sum[32];
  __shared__ double2 tab[CPLX ? kExpiTable : 1];
  static_assert(kSmallTile * RC::n >= 4 * 32 * kSmallWarps, "the sums reuse the record buffer");
  cg::cluster_group cl = cg::this_cluster();
  const int64_t slices = cl.num_blocks(), slice = cl.block_rank();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = (blockIdx.x / slices) * 32 + lane;
  const bool lead = slice == 0 && warp == 0;
  if (CPLX)
    for (int q = threadIdx.x; q < kExpiTable; q += 32 * kSmallWarps) tab[q] = expi[q];
  Target<double, DIM, RC::tnormal> t;
  int64_t p = 0, p1 = 0;  // this thread's next correction entry, row end
  double2 yo = make_double2(0.0, 0.0);
  if (i < m) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) t.x[c] = tc[DIM * i + c];
    if constexpr (RC::tnormal) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) t.n[c] = tn[DIM * i + c];
    }
    if (e.rowptr) {
      p = e.rowptr[i] + slice * kSmallWarps + warp;
      p1 = e.rowptr[i + 1];
    }
    if (lead && !e.beta_zero) yo = epilogue_y_old<CPLX>(e, i);
  }
  const int64_t pstride = slices * kSmallWarps;
  const int64_t per = (n + slices - 1) / slices;
  const int64_t j0 = slice * per, j1 = j0 + per < n ? j0 + per : n;
  double ar = 0.0, ai = 0.0;
  int32_t cc[kSmallCorr];
  double2 cv[kSmallCorr];
  for (int64_t base = j0; base < j1; base += kSmallTile) {
    const int cnt = (int)(j1 - base < kSmallTile ? j1 - base : kSmallTile);
    __syncthreads();  // the previous tile is consumed
    if (threadIdx.x < cnt) {
      double rec[RC::n];
      build_record<PDE, KIND, DIM, double>(base + threadIdx.x, n, src.xs, src.ns, src.w, src.sigma, src.c1,
                                           src.c2, rec);
      double2* o = reinterpret_cast<double2*>(recs + threadIdx.x * RC::n);
#pragma unroll
      for (int c = 0; c < RC::n / 2; ++c) o[c] = make_double2(rec[2 * c], rec[2 * c + 1]);
    }
    if (base == j0) {
      // correction entries fetched ahead (their values are used after the pair loop)
#pragma unroll
      for (int u = 0; u < kSmallCorr; ++u) {
        const int64_t pu = p + u * pstride;
        cc[u] = pu < p1 ? e.col[pu] : -1;
        cv[u] = pu < p1 ? (CPLX ? reinterpret_cast<const double2*>(e.val)[pu] : make_double2(e.val[pu], 0.0))
                        : make_double2(0.0, 0.0);
      }
    }
    __syncthreads();
    if (i < m) {
      const int pw = (cnt + kSmallWarps - 1) / kSmallWarps;
      const int q0 = warp * pw, q1 = q0 + pw < cnt ? q0 + pw : cnt;
      for (int q = q0; q < q1; ++q) pair_step<PDE, KIND, DIM, double>(t, recs + q * RC::n, kT, delta, k, tab, ar, ai);
    }
  }
  if (j0 >= j1) {  // an empty slice still fetches its correction entries
#pragma unroll
    for (int u = 0; u < kSmallCorr; ++u) {
      const int64_t pu = p + u * pstride;
      cc[u] = pu < p1 ? e.col[pu] : -1;
      cv[u] = pu < p1 ? (CPLX ? reinterpret_cast<const double2*>(e.val)[pu] : make_double2(e.val[pu], 0.0))
                      : make_double2(0.0, 0.0);
    }
  }
  double cr = 0.0, ci = 0.0;
  auto corr_add = [&](int32_t j, double2 v) {
    if (CPLX) {
      const double2 xv = reinterpret_cast<const double2*>(e.x)[j];
      cr = fma(v.x, xv.x, fma(-v.y, xv.y, cr));
      ci = fma(v.x, xv.y, fma(v.y, xv.x, ci));
    } else {
      cr = fma(v.x, e.x[j], cr);
    }
  };
#pragma unroll
  for (int u = 0; u < kSmallCorr; ++u)
    if (cc[u] >= 0) corr_add(cc[u], cv[u]);
  for (int64_t pu = p + kSmallCorr * pstride; pu < p1; pu += pstride)
    corr_add(e.col[pu], CPLX ? reinterpret_cast<const double2*>(e.val)[pu] : make_double2(e.val[pu], 0.0));
  __syncthreads();  // every warp is done with the records: reuse them for the sums
  double4* part = reinterpret_cast<double4*>(recs);  // [warp][lane]
  part[warp * 32 + lane] = make_double4(ar, ai, cr, ci);
  __syncthreads();
  if (warp == 0) {
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
#pragma unroll
    for (int w = 0; w < kSmallWarps; ++w) {
      const double4 v = part[w * 32 + lane];
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
    slice_sum[lane] = acc;
  }
  cl.sync();  // every slice's sums are in its shared memory
  if (lead && i < m) {
    double4 acc = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int r = 0; r < (int)slices; ++r) {
      const double4 v = *cl.map_shared_rank(&slice_sum[lane], r);
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
    const double sc = e.rowscale ? e.scale * e.rowscale[i] : e.scale;
    epilogue_store<CPLX>(e, i, fma(acc.x, sc, acc.z), fma(acc.y, sc, acc.w), yo);
  }
  cl.sync();  // the peers' shared memory stays valid until CTA 0 has read it
}

// ---------------------------------------------------------------------------
// Symmetric form for square operators (the target set is the source set),// ---------------------------------------------------------------------------
// Symmetric form for square operators (the target set is the source set),
// every kernel: single layer, double layer, combined field (3D), adjoint
// double layer and hypersingular, in 3D and for the 2D Laplace kernels.
//
// Every kernel value of an unordered pair {a, b} serves both products:
//   SL: G(x_a, x_b) = G(x_b, x_a);
//   DL: K(x_a, x_b) p_b = d(r.p_b) and K(x_b, x_a) p_a = -d(r.p_a) with the
//       same radial factor d (r = x_a - x_b, p the packed dipoles w sigma n);
//   ADL and HS: see pair_sym_step;
// so the distance, the reciprocal square root and the phase are computed
// once per unordered pair.  Nodes are cut into blocks of BT = 128*TPT; a CTA
// takes one work item (row block I, source blocks J0 <= J < J1, J >= I):
// its threads hold the targets of block I (coordinates and their own packed
// charge/dipole), source tiles of the blocks J stream through shared memory
// as in pair_forward.  For J == I every ordered pair is evaluated (the
// forward step).  For J > I the row sums go to the target registers and the
// column sums of each source are reduced over the CTA (warp shuffles, then
// the four warps in a fixed order) and stored in zpart[I][j].  The epilogue
// adds, for node i of block B, the row partials of the items of row B and
// zpart[I][i] for I < B: a fixed order, so the result is deterministic.
// ---------------------------------------------------------------------------
struct SymArgs {
  int64_t npad;           // packed records: nb * BT (zero charges past n)
  const int32_t* items;   // (I, J0, J1) per CTA
  const int32_t* ids;     // row-partial slot of each CTA's item (NULL: the CTA index)
  const void* packed;
  void* ypart;            // [item][BT]
  void* zpart;            // [nb][zld]: node j of the panel's columns at j - zcol0
  int64_t zld, zcol0;     // one panel: npad and 0
  double k, kT, delta;
  const void* expi;
  int* err;
};

// Records of the symmetric form.  SL, DL and CF use the layouts of Rec.  The
// adjoint double layer and the hypersingular kernel take the normal of the
// target, so both ends of a pair need their normal and their charge:
//   x [DIM] | n [DIM] | q            (Laplace; 3D: 8 elements with one pad,
//                                     2D: 6 (FP64) or 8 (FP32))
//   x y z | n_x n_y n_z | qr qi      (Helmholtz: 8 elements)
// with q = w sigma; padded to a multiple of 16 bytes.
template <int PDE, int KIND, int DIM, class R>
struct SymRec {
  static constexpr bool normal = (KIND == ADL || KIND == HS);
  static constexpr bool cplx = (PDE == HELMHOLTZ);
  static constexpr int align = 16 / sizeof(R);
  static constexpr int nused = 2 * DIM + (cplx ? 2 : 1);
  static constexpr int used = normal ? nused : Rec<PDE, KIND, DIM, R>::used;
  static constexpr int n = normal ? (nused + align - 1) / align * align : Rec<PDE, KIND, DIM, R>::n;
};

template <int PDE, int DIM, class R>
__global__ void pack_sym_normal(int64_t n, int64_t npad, const double* __restrict__ xs,
                                const double* __restrict__ ns, const double* __restrict__ w,
                                const double* __restrict__ sigma, R* __restrict__ out) {
  constexpr int NR = SymRec<PDE, HS, DIM, R>::n;
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= npad) return;
  R rec[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) rec[c] = R(0);
  if (j < n) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      rec[c] = R(xs[DIM * j + c]);
      rec[DIM + c] = R(ns[DIM * j + c]);
    }
    const double wj = w[j];
    if (PDE == HELMHOLTZ) {
      rec[2 * DIM] = R(wj * sigma[2 * j]);
      rec[2 * DIM + 1] = R(wj * sigma[2 * j + 1]);
    } else {
      rec[2 * DIM] = R(wj * sigma[j]);
    }
  }
  R* o = out + j * NR;
#pragma unroll
  for (int c = 0; c < NR; ++c) o[c] = rec[c];
}

// Both products of one unordered pair: y_t += K(x_t, x_s) c_s and
// z_s += K(x_s, x_t) c_t, with c the packed charge/dipole records of the
// target t and the source s (layouts of SymRec), r = x_t - x_s.  With COL
// false only the row product is formed (the diagonal blocks of the
// adjoint double layer and hypersingular forms, which evaluate every ordered
// pair).
//   ADL: K(x_t, x_s) q_s = (r.n_t) f q_s and K(x_s, x_t) q_t = -(r.n_s) f q_t
//        with the same radial factor f (1/d^3; e^{ikd}(1/d - ik)/d^2);
//   HS : K(x_t, x_s) q_s = h q_s and K(x_s, x_t) q_t = h q_t with
//        h = a (r.n_t)(r.n_s) + b (n_t.n_s), a and b functions of d alone
//        (Laplace: a = -3/d^5, b = 1/d^3), so h is symmetric in the pair.
// 2D Laplace (kernel constants in the epilogue as in pair_step):
//   SL : log(d^2), symmetric;   DL : (r.p)/d^2, column -(r.p_t)/d^2;
//   ADL: (r.n_t) q/d^2, column -(r.n_s) q_t/d^2;
//   HS : h = (n_t.n_s - 2 (r.n_t)(r.n_s)/d^2)/d^2, symmetric.
template <int KIND, class R, bool COL>
__device__ __forceinline__ void pair_sym_step_2d(const R* __restrict__ t, const R* __restrict__ s, R& ar,
                                                 R& zr) {
  using M = MathOps<R>;
  const R r0 = t[0] - s[0], r1 = t[1] - s[1];
  const R d2 = fma(r1, r1, r0 * r0);
  const bool keep = M::keep(d2);
  if (KIND == SL) {
    const R l = keep ? M::lg(d2) : R(0);
    ar = fma(l, s[2], ar);
    if (COL) zr = fma(l, t[2], zr);
    return;
  }
  const R id2 = keep ? M::rcp(d2) : R(0);
  if (KIND == DL) {
    ar = fma(fma(r1, s[3], r0 * s[2]), id2, ar);
    if (COL) zr = fma(-fma(r1, t[3], r0 * t[2]), id2, zr);
  } else if (KIND == ADL) {
    ar = fma(fma(r1, t[3], r0 * t[2]) * id2, s[4], ar);
    if (COL) zr = fma(-fma(r1, s[3], r0 * s[2]) * id2, t[4], zr);
  } else if (KIND == HS) {
    const R rnt = fma(r1, t[3], r0 * t[2]), rns = fma(r1, s[3], r0 * s[2]);
    const R nn = fma(t[3], s[3], t[2] * s[2]);
    const R h = fma(R(-2) * rnt * rns, id2, nn) * id2;
    ar = fma(h, s[4], ar);
    if (COL) zr = fma(h, t[4], zr);
  }
}

template <int PDE, int KIND, int DIM, class R, bool COL = true>
__device__ __forceinline__ void pair_sym_step(const R* __restrict__ t, const R* __restrict__ s, R kT, R delta, R k,
                                              const typename MathOps<R>::R2* __restrict__ tab, R& ar, R& ai,
                                              R& zr, R& zi) {
  if constexpr (DIM == 2) {
    pair_sym_step_2d<KIND, R, COL>(t, s, ar, zr);
    return;
  }
  using M = MathOps<R>;
  const R r0 = t[0] - s[0], r1 = t[1] - s[1], r2 = t[2] - s[2];
  const R d2 = fma(r2, r2, fma(r1, r1, r0 * r0));
  const bool keep = M::keep(d2);
  if (KIND == ADL || KIND == HS) {
    const R rnt = fma(r2, t[5], fma(r1, t[4], r0 * t[3]));
    const R rns = COL || KIND == HS ? fma(r2, s[5], fma(r1, s[4], r0 * s[3])) : R(0);
    if (PDE == LAPLACE) {
      if (KIND == ADL) {
        const R ri3 = keep ? M::rsq3(d2) : R(0);
        ar = fma(rnt * ri3, s[6], ar);
        if (COL) zr = fma(-rns * ri3, t[6], zr);
      } else {
        const R nn = fma(t[5], s[5], fma(t[4], s[4], t[3] * s[3]));
        const R ri = keep ? M::rsq(d2) : R(0);
        const R id2 = ri * ri;
        const R h = fma(R(-3) * rnt * rns, id2, nn) * (id2 * ri);
        ar = fma(h, s[6], ar);
        if (COL) zr = fma(h, t[6], zr);
      }
    } else {
      const R ri = keep ? M::rsq(d2) : R(0);
      const R d = d2 * ri;
      R sn, cs;
      expi_table_eval(d, kT, tab, delta, cs, sn);
      const R id2 = ri * ri;
      R hr, hi, gr = R(0), gi = R(0);  // row factor h, column factor g
      if (KIND == ADL) {
        const R er = fma(cs, ri, k * sn), ei = fma(sn, ri, -k * cs);  // e^{ikd}(1/d - ik)
        const R br = er * id2, bi = ei * id2;
        hr = br * rnt;
        hi = bi * rnt;
        if (COL) {
          gr = -br * rns;
          gi = -bi * rns;
        }
      } else {
        // h = b (n_t.n_s) + a (r.n_t)(r.n_s) with b = e^{ikd}(1/d - ik)/d^2 and
        // a = e^{ikd}(k^2 d^2 - 3 + 3ikd)/d^5, i.e. h = e^{ikd} W with the
        // bracket W = (1/d - ik) p + (k^2 d^2 - 3 + 3ikd) s formed in real
        // arithmetic from p = (n_t.n_s)/d^2 and s = (r.n_t)(r.n_s)/d^5
        const R nn = fma(t[5], s[5], fma(t[4], s[4], t[3] * s[3]));
        const R kd = k * d;
        const R fr = fma(kd, kd, R(-3)), fi = R(3) * kd;
        const R p = nn * id2;
        const R s5 = (rnt * rns) * (id2 * id2 * ri);
        const R wr = fma(ri, p, fr * s5), wi = fma(-k, p, fi * s5);
        hr = fma(cs, wr, -sn * wi);
        hi = fma(cs, wi, sn * wr);
        gr = hr;
        gi = hi;
      }
      ar = fma(hr, s[6], fma(-hi, s[7], ar));
      ai = fma(hr, s[7], fma(hi, s[6], ai));
      if (COL) {
        zr = fma(gr, t[6], fma(-gi, t[7], zr));
        zi = fma(gr, t[7], fma(gi, t[6], zi));
      }
    }
    return;
  }
  if (PDE == LAPLACE) {
    if (KIND == SL) {
      const R ri = keep ? M::rsq(d2) : R(0);
      ar = fma(ri, s[3], ar);
      zr = fma(ri, t[3], zr);
    } else {
      const R rs = fma(r2, s[5], fma(r1, s[4], r0 * s[3]));
      const R rt = fma(r2, t[5], fma(r1, t[4], r0 * t[3]));
      if (KIND == DL) {
        const R ri3 = keep ? M::rsq3(d2) : R(0);
        ar = fma(rs, ri3, ar);
        zr = fma(-rt, ri3, zr);
      } else {  // CF: charge after the dipole
        const R ri = keep ? M::rsq(d2) : R(0);
        const R ri3 = ri * ri * ri;
        ar = fma(ri, s[6], fma(rs, ri3, ar));
        zr = fma(ri, t[6], fma(-rt, ri3, zr));
      }
    }
  } else {
    const R ri = keep ? M::rsq(d2) : R(0);
    R sn, cs;
    expi_table_eval(d2 * ri, kT, tab, delta, cs, sn);
    if (KIND == SL) {
      const R gr = ri * cs, gi = ri * sn;
      ar = fma(gr, s[3], fma(-gi, s[4], ar));
      ai = fma(gr, s[4], fma(gi, s[3], ai));
      zr = fma(gr, t[3], fma(-gi, t[4], zr));
      zi = fma(gr, t[4], fma(gi, t[3], zi));
    } else {  // dipole Re [3..5], Im [6..8]; CF: charge [9], [10]
      const R er = fma(cs, ri, k * sn), ei = fma(sn, ri, -k * cs);
      const R id2 = ri * ri;
      const R gr = er * id2, gi = ei * id2;
      const R A = fma(r2, s[5], fma(r1, s[4], r0 * s[3])), B = fma(r2, s[8], fma(r1, s[7], r0 * s[6]));
      const R At = fma(r2, t[5], fma(r1, t[4], r0 * t[3])), Bt = fma(r2, t[8], fma(r1, t[7], r0 * t[6]));
      ar = fma(gr, A, fma(-gi, B, ar));
      ai = fma(gr, B, fma(gi, A, ai));
      zr = fma(-gr, At, fma(gi, Bt, zr));
      zi = fma(-gr, Bt, fma(-gi, At, zi));
      if (KIND == CF) {
        const R hr = cs * ri, hi = sn * ri;
        ar = fma(hr, s[9], fma(-hi, s[10], ar));
        ai = fma(hr, s[10], fma(hi, s[9], ai));
        zr = fma(hr, t[9], fma(-hi, t[10], zr));
        zi = fma(hr, t[10], fma(hi, t[9], zi));
      }
    }
  }
}

// Warp sums of four values v[0..3] (one per source), reduce-scattered: lanes
// 0, 8, 16, 24 return the totals of v[0], v[1], v[2], v[3].  Levels 16 and 8
// exchange halves of the set instead of reducing every value over all five
// levels: 6 adds and 6 shuffles for four sums instead of 20 each.
template <class R>
__device__ __forceinline__ R warp_sum4(const R (&v)[4], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8;
  R k0 = b4 ? v[2] : v[0], k1 = b4 ? v[3] : v[1];
  k0 += __shfl_xor_sync(0xffffffffu, b4 ? v[0] : v[2], 16);
  k1 += __shfl_xor_sync(0xffffffffu, b4 ? v[1] : v[3], 16);
  R k = b3 ? k1 : k0;
  k += __shfl_xor_sync(0xffffffffu, b3 ? k0 : k1, 8);
  k += __shfl_xor_sync(0xffffffffu, k, 4);
  k += __shfl_xor_sync(0xffffffffu, k, 2);
  k += __shfl_xor_sync(0xffffffffu, k, 1);
  return k;
}

__device__ __forceinline__ void put_partial(double* p, double r, double) { *p = r; }
__device__ __forceinline__ void put_partial(double2* p, double r, double i) { *p = make_double2(r, i); }
__device__ __forceinline__ void put_partial(float2* p, float r, float) { *p = make_float2(r, 0.f); }
__device__ __forceinline__ void put_partial(float4* p, float r, float i) { *p = make_float4(r, 0.f, i, 0.f); }

template <int PDE, int KIND, int DIM, class R, int TILE, int TPT>
__global__ void __launch_bounds__(kBlock) pair_symm(SymArgs a) {
  using RC = SymRec<PDE, KIND, DIM, R>;
  constexpr bool CPLX = RC::cplx;
  using P = typename PartialT<R, CPLX>::T;
  using R2 = typename MathOps<R>::R2;
  constexpr int BT = kBlock * TPT;
  static_assert(BT % TILE == 0, "whole source tiles per node block");
  constexpr int TPB = BT / TILE;
  constexpr int NU = RC::used;
  constexpr int kWarps = kBlock / 32;
  constexpr uint32_t kStageBytes = TILE * RC::n * sizeof(R);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* stage0 = reinterpret_cast<R*>(smem_raw);
  R* stage1 = reinterpret_cast<R*>(smem_raw + kStageBytes);
  R2* tab = reinterpret_cast<R2*>(smem_raw + 2 * kStageBytes);  // Helmholtz only
  R* zsm = reinterpret_cast<R*>(smem_raw + 2 * kStageBytes + (CPLX ? kExpiTable * sizeof(R2) : 0));
  __shared__ __align__(8) uint64_t full[2];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int I = a.items[3 * blockIdx.x], J0 = a.items[3 * blockIdx.x + 1], J1 = a.items[3 * blockIdx.x + 2];
  const R* src = static_cast<const R*>(a.packed);
  R tg[TPT][NU];
  Acc<R, CPLX> acc[TPT];
#pragma unroll
  for (int u = 0; u < TPT; ++u) {
    const int64_t i = (int64_t)I * BT + u * kBlock + tid;
#pragma unroll
    for (int c = 0; c < NU; ++c) tg[u][c] = src[i * RC::n + c];
  }
  const R k = R(a.k), kT = R(a.kT), delta = R(a.delta);
  if (CPLX) {
    const R2* g = static_cast<const R2*>(a.expi);
    for (int q = tid; q < kExpiTable; q += kBlock) tab[q] = g[q];
  }
  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int64_t t0 = (int64_t)J0 * TPB, t1 = (int64_t)J1 * TPB;
  int64_t issued = t0;
  if (tid == 0) {
    for (int s = 0; s < 2 && issued < t1; ++s, ++issued) {
      mbar_arrive_expect_tx(&full[s], kStageBytes);
      bulk_copy_g2s(s ? stage1 : stage0, src + issued * TILE * RC::n, kStageBytes, &full[s]);
    }
  }
  for (int64_t t = t0; t < t1; ++t) {
    const int st = (int)((t - t0) & 1);
    const uint32_t parity = (uint32_t)(((t - t0) >> 1) & 1);
    const bool ok = mbar_wait_bounded(&full[st], parity);
    if (!__syncthreads_and(ok)) {
      if (tid == 0) {
        atomicExch(a.err, kErrWaitTimeout);
        for (int64_t q = t + 1; q < issued; ++q)
          mbar_wait_bounded(&full[(q - t0) & 1], (uint32_t)(((q - t0) >> 1) & 1));
      }
      return;
    }
    const R* sp = st ? stage1 : stage0;
    const bool diag = t / TPB == I;
    R* zb = zsm + st * (kWarps * TILE * 2);
    if (diag) {
#pragma unroll 1
      for (int g = 0; g < TILE; g += kGroup) {
#pragma unroll 2
        for (int s = 0; s < kGroup; ++s) {
          const R* rec = sp + (g + s) * RC::n;
#pragma unroll
          for (int u = 0; u < TPT; ++u) {
            if constexpr (RC::normal) {
              R unused_r = R(0), unused_i = R(0);  // the column half is not formed
              pair_sym_step<PDE, KIND, DIM, R, false>(tg[u], rec, kT, delta, k, tab, acc[u].gr(), acc[u].gi(),
                                                      unused_r, unused_i);
            } else {
              Target<R, DIM, false> tt;
#pragma unroll
              for (int c = 0; c < DIM; ++c) tt.x[c] = tg[u][c];
              pair_step<PDE, KIND, DIM, R>(tt, rec, kT, delta, k, tab, acc[u].gr(), acc[u].gi());
            }
          }
        }
#pragma unroll
        for (int u = 0; u < TPT; ++u) acc[u].fold();
      }
    } else {
#pragma unroll 1
      for (int g = 0; g < TILE; g += kGroup) {
#pragma unroll 1
        for (int s = 0; s < kGroup; s += 4) {
          R zr[4], zi[4];
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const R* rec = sp + (g + s + v) * RC::n;
            zr[v] = zi[v] = R(0);
#pragma unroll
            for (int u = 0; u < TPT; ++u)
              pair_sym_step<PDE, KIND, DIM, R>(tg[u], rec, kT, delta, k, tab, acc[u].gr(), acc[u].gi(), zr[v],
                                               zi[v]);
          }
          const R sr = warp_sum4(zr, lane);
          const R si = CPLX ? warp_sum4(zi, lane) : R(0);
          if ((lane & 7) == 0) {
            const int v = lane >> 3;
            zb[(warp * TILE + g + s + v) * 2] = sr;
            zb[(warp * TILE + g + s + v) * 2 + 1] = si;
          }
        }
#pragma unroll
        for (int u = 0; u < TPT; ++u) acc[u].fold();
      }
    }
    __syncthreads();  // the stage is read and this tile's column sums are in zb
    if (!diag) {
      P* zp = static_cast<P*>(a.zpart) + (int64_t)I * a.zld + (t * TILE - a.zcol0);
      for (int s = tid; s < TILE; s += kBlock) {
        R vr = zb[s * 2], vi = zb[s * 2 + 1];
#pragma unroll
        for (int w = 1; w < kWarps; ++w) {
          vr += zb[(w * TILE + s) * 2];
          vi += zb[(w * TILE + s) * 2 + 1];
        }
        put_partial(zp + s, vr, vi);
      }
    }
    if (tid == 0 && issued < t1) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&full[st], kStageBytes);
      bulk_copy_g2s(st ? stage1 : stage0, src + issued * TILE * RC::n, kStageBytes, &full[st]);
      ++issued;
    }
  }
  P* out = static_cast<P*>(a.ypart) + (int64_t)(a.ids ? a.ids[blockIdx.x] : (int)blockIdx.x) * BT;
#pragma unroll
  for (int u = 0; u < TPT; ++u) store_partial(out + u * kBlock + tid, acc[u]);
}

// ---------------------------------------------------------------------------
// Paired-FP32 form of the symmetric kernel for the FP32C Laplace single
// layer, double layer and combined field (3D).  The FP32 kernels are bound by
// instruction issue, not by the FP32 pipe; sm_100 issues two FP32 lanes per
// instruction (__fadd2_rn, __fmul2_rn, __ffma2_rn).  Each thread holds its
// targets in pairs (u, u + 1) as float2, and the records carry every value
// twice (x x y y z z | p_x p_x p_y p_y p_z p_z | q q), so one 16-byte shared
// load yields two ready operand pairs.  Per lane the arithmetic is that of
// pair_sym_step (the reciprocal square root and the self-pair test stay per
// lane); the column sum over the thread's targets is formed per lane and the
// two lanes added, so results differ from the scalar kernel by rounding only.
// ---------------------------------------------------------------------------
template <int KIND>
struct RecX2 {
  static constexpr int vals = (KIND == SL ? 4 : KIND == DL ? 6 : 7);  // x y z [p] [q]
  static constexpr int n = (2 * vals + 3) / 4 * 4;                      // floats per record
};

template <int KIND>
__global__ void pack_sources_x2(int64_t n, int64_t npad, const double* __restrict__ xs,
                                const double* __restrict__ ns, const double* __restrict__ w,
                                const double* __restrict__ sigma, double c1, double c2,
                                float* __restrict__ out) {
  constexpr int NR = RecX2<KIND>::n;
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= npad) return;
  float v[RecX2<KIND>::vals];
#pragma unroll
  for (int c = 0; c < RecX2<KIND>::vals; ++c) v[c] = 0.f;
  if (j < n) {
    v[0] = (float)xs[3 * j];
    v[1] = (float)xs[3 * j + 1];
    v[2] = (float)xs[3 * j + 2];
    const double q = w[j] * sigma[j];
    if (KIND == SL) {
      v[3] = (float)q;
    } else {
      const double qd = KIND == CF ? c1 * q : q;
#pragma unroll
      for (int c = 0; c < 3; ++c) v[3 + c] = (float)(qd * ns[3 * j + c]);
      if (KIND == CF) v[6] = (float)(c2 * q);
    }
  }
  float* o = out + j * NR;
#pragma unroll
  for (int c = 0; c < NR; ++c) o[c] = c / 2 < RecX2<KIND>::vals ? v[c / 2] : 0.f;
}

// One source against a pair of targets: the row products into (ar.x, ar.y);
// with COL the column terms into zq (ri q_t, CF) and zd (r.p_t ri^3).
template <int KIND, bool COL>
__device__ __forceinline__ void pair_x2_step(const float2 (&t)[RecX2<KIND>::vals], const float2* __restrict__ s,
                                             float2& ar, float2& zq, float2& zd) {
  const float2 m1 = make_float2(-1.f, -1.f);
  const float2 r0 = __ffma2_rn(s[0], m1, t[0]);  // t - s, one rounding per lane
  const float2 r1 = __ffma2_rn(s[1], m1, t[1]);
  const float2 r2 = __ffma2_rn(s[2], m1, t[2]);
  const float2 d2 = __ffma2_rn(r2, r2, __ffma2_rn(r1, r1, __fmul2_rn(r0, r0)));
  float2 ri;
  ri.x = d2.x > 1.0e-28f ? rsqrt_fast(d2.x) : 0.f;
  ri.y = d2.y > 1.0e-28f ? rsqrt_fast(d2.y) : 0.f;
  if (KIND == SL) {
    ar = __ffma2_rn(ri, s[3], ar);
    if (COL) zq = __ffma2_rn(ri, t[3], zq);
    return;
  }
  const float2 ri3 = __fmul2_rn(__fmul2_rn(ri, ri), ri);
  const float2 rs = __ffma2_rn(r2, s[5], __ffma2_rn(r1, s[4], __fmul2_rn(r0, s[3])));
  if (KIND == CF) {
    ar = __ffma2_rn(ri, s[6], __ffma2_rn(rs, ri3, ar));
  } else {
    ar = __ffma2_rn(rs, ri3, ar);
  }
  if (COL) {
    const float2 rt = __ffma2_rn(r2, t[5], __ffma2_rn(r1, t[4], __fmul2_rn(r0, t[3])));
    zd = __ffma2_rn(rt, ri3, zd);
    if (KIND == CF) zq = __ffma2_rn(ri, t[6], zq);
  }
}

template <int KIND, int TPT>
__global__ void __launch_bounds__(kBlock) pair_symm_x2(SymArgs a) {
  constexpr int TILE = kTile32;
  constexpr int NR = RecX2<KIND>::n, NV = RecX2<KIND>::vals;
  constexpr int BT = kBlock * TPT, NP = TPT / 2;
  static_assert(TPT % 2 == 0 && BT % TILE == 0, "target pairs, whole source tiles per node block");
  constexpr int TPB = BT / TILE;
  constexpr int kWarps = kBlock / 32;
  constexpr uint32_t kStageBytes = TILE * NR * sizeof(float);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* stage0 = reinterpret_cast<float*>(smem_raw);
  float* stage1 = reinterpret_cast<float*>(smem_raw + kStageBytes);
  float* zsm = reinterpret_cast<float*>(smem_raw + 2 * kStageBytes);
  __shared__ __align__(8) uint64_t full[2];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int I = a.items[3 * blockIdx.x], J0 = a.items[3 * blockIdx.x + 1], J1 = a.items[3 * blockIdx.x + 2];
  const float* src = static_cast<const float*>(a.packed);
  float2 tg[NP][NV];  // (target 2p, target 2p + 1), value c
  float2 g[NP];       // group sums per lane
  float hr[TPT], lr[TPT];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const int64_t i0 = (int64_t)I * BT + (2 * p) * kBlock + tid, i1 = i0 + kBlock;
#pragma unroll
    for (int c = 0; c < NV; ++c) tg[p][c] = make_float2(src[i0 * NR + 2 * c], src[i1 * NR + 2 * c]);
    g[p] = make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int u = 0; u < TPT; ++u) hr[u] = lr[u] = 0.f;
  auto fold = [&]() {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      two_sum_fold(hr[2 * p], lr[2 * p], g[p].x);
      two_sum_fold(hr[2 * p + 1], lr[2 * p + 1], g[p].y);
    }
  };
  if (tid == 0) {
    mbar_init(&full[0], 1);
    mbar_init(&full[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const int64_t t0 = (int64_t)J0 * TPB, t1 = (int64_t)J1 * TPB;
  int64_t issued = t0;
  if (tid == 0) {
    for (int s = 0; s < 2 && issued < t1; ++s, ++issued) {
      mbar_arrive_expect_tx(&full[s], kStageBytes);
      bulk_copy_g2s(s ? stage1 : stage0, src + issued * TILE * NR, kStageBytes, &full[s]);
    }
  }
  for (int64_t t = t0; t < t1; ++t) {
    const int st = (int)((t - t0) & 1);
    const uint32_t parity = (uint32_t)(((t - t0) >> 1) & 1);
    const bool ok = mbar_wait_bounded(&full[st], parity);
    if (!__syncthreads_and(ok)) {
      if (tid == 0) {
        atomicExch(a.err, kErrWaitTimeout);
        for (int64_t q = t + 1; q < issued; ++q)
          mbar_wait_bounded(&full[(q - t0) & 1], (uint32_t)(((q - t0) >> 1) & 1));
      }
      return;
    }
    const float* sp = st ? stage1 : stage0;
    const bool diag = t / TPB == I;
    float* zb = zsm + st * (kWarps * TILE * 2);
    if (diag) {
#pragma unroll 1
      for (int gq = 0; gq < TILE; gq += kGroup) {
#pragma unroll 2
        for (int s = 0; s < kGroup; ++s) {
          const float2* rec = reinterpret_cast<const float2*>(sp + (gq + s) * NR);
          float2 zq = make_float2(0.f, 0.f), zd = zq;  // the column half is not formed
#pragma unroll
          for (int p = 0; p < NP; ++p) pair_x2_step<KIND, false>(tg[p], rec, g[p], zq, zd);
        }
        fold();
      }
    } else {
#pragma unroll 1
      for (int gq = 0; gq < TILE; gq += kGroup) {
#pragma unroll 1
        for (int s = 0; s < kGroup; s += 4) {
          float zr[4];
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const float2* rec = reinterpret_cast<const float2*>(sp + (gq + s + v) * NR);
            float2 zq = make_float2(0.f, 0.f), zd = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < NP; ++p) pair_x2_step<KIND, true>(tg[p], rec, g[p], zq, zd);
            // K(x_s, x_t) c_t: SL and CF ri q_t, DL and CF -(r.p_t) ri^3
            zr[v] = KIND == DL ? -(zd.x + zd.y) : (KIND == SL ? zq.x + zq.y : (zq.x + zq.y) - (zd.x + zd.y));
          }
          const float sr = warp_sum4(zr, lane);
          if ((lane & 7) == 0) {
            const int v = lane >> 3;
            zb[(warp * TILE + gq + s + v) * 2] = sr;
            zb[(warp * TILE + gq + s + v) * 2 + 1] = 0.f;
          }
        }
        fold();
      }
    }
    __syncthreads();  // the stage is read and this tile's column sums are in zb
    if (!diag) {
      float2* zp = static_cast<float2*>(a.zpart) + (int64_t)I * a.zld + (t * TILE - a.zcol0);
      for (int s = tid; s < TILE; s += kBlock) {
        float vr = zb[s * 2];
#pragma unroll
        for (int w = 1; w < kWarps; ++w) vr += zb[(w * TILE + s) * 2];
        zp[s] = make_float2(vr, 0.f);
      }
    }
    if (tid == 0 && issued < t1) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&full[st], kStageBytes);
      bulk_copy_g2s(st ? stage1 : stage0, src + issued * TILE * NR, kStageBytes, &full[st]);
      ++issued;
    }
  }
  float2* out = static_cast<float2*>(a.ypart) + (int64_t)(a.ids ? a.ids[blockIdx.x] : (int)blockIdx.x) * BT;
#pragma unroll
  for (int u = 0; u < TPT; ++u) out[u * kBlock + tid] = make_float2(hr[u], lr[u]);
}

// Row sums of the symmetric form: the item partials of row block B and the
// column partials of the row blocks above.
// Running sums over panels: for node i of row block B (B < the panel's
// rows), acc[i] += the panel's row partials of B's items (in order), then,
// when B is one of the panel's source blocks, the column partials
// zpart[r][i - col0*bt] of the row blocks r < B.
struct SymFold {
  int64_t m;
  int bt;
  const int32_t* rowptr;
  const int32_t* rowitems;
  const void* ypart;
  const void* zpart;
  int64_t zld;
  int col0, ncols;
  void* acc;
};

// Four threads per node: slice s sums the column partials of the row blocks
// r = s, s + 4, ...; the slices are added in a fixed order (deterministic).
constexpr int kFoldNodes = 64, kFoldSlices = 4;

template <class P, bool CPLX>
__global__ void __launch_bounds__(kFoldNodes * kFoldSlices) pair_symm_fold_kernel(SymFold f) {
  __shared__ double2 part[kFoldSlices][kFoldNodes];
  const int tn = threadIdx.x % kFoldNodes, sl = threadIdx.x / kFoldNodes;
  const int64_t i = blockIdx.x * (int64_t)kFoldNodes + tn;
  const bool live = i < f.m;
  const int B = live ? (int)(i / f.bt) : 0, il = live ? (int)(i % f.bt) : 0;
  const P* yp = static_cast<const P*>(f.ypart);
  const P* zp = static_cast<const P*>(f.zpart);
  double2 c = make_double2(0.0, 0.0);
  if (live && B >= f.col0 && B < f.col0 + f.ncols) {
    const int64_t jl = i - (int64_t)f.col0 * f.bt;
    for (int r = sl; r < B; r += kFoldSlices) {
      const double2 v = load_partial(zp + (int64_t)r * f.zld + jl);
      c.x += v.x;
      c.y += v.y;
    }
  }
  part[sl][tn] = c;
  __syncthreads();
  if (sl != 0 || !live) return;
  double sr = 0.0, si = 0.0;
  if (CPLX) {
    const double2 v = static_cast<const double2*>(f.acc)[i];
    sr = v.x;
    si = v.y;
  } else {
    sr = static_cast<const double*>(f.acc)[i];
  }
  for (int q = f.rowptr[B]; q < f.rowptr[B + 1]; ++q) {
    const double2 v = load_partial(yp + (int64_t)f.rowitems[q] * f.bt + il);
    sr += v.x;
    si += v.y;
  }
  sr += (part[0][tn].x + part[1][tn].x) + (part[2][tn].x + part[3][tn].x);
  si += (part[0][tn].y + part[1][tn].y) + (part[2][tn].y + part[3][tn].y);
  if (CPLX)
    static_cast<double2*>(f.acc)[i] = make_double2(sr, si);
  else
    static_cast<double*>(f.acc)[i] = sr;
}

struct SymEpi {
  int64_t npad;
  int bt;
  const int32_t* rowptr;    // nb + 1
  const int32_t* rowitems;  // items of each row block
  const void* zpart;
};

template <class P, bool CPLX>
__global__ void pair_symm_epilogue_kernel(EpiArgs e, SymEpi s) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= e.m) return;
  const int B = (int)(i / s.bt), il = (int)(i % s.bt);
  const P* yp = static_cast<const P*>(e.partial);
  const P* zp = static_cast<const P*>(s.zpart);
  double sr = 0.0, si = 0.0;
  for (int q = s.rowptr[B]; q < s.rowptr[B + 1]; ++q) {
    const double2 v = load_partial(yp + (int64_t)s.rowitems[q] * s.bt + il);
    sr += v.x;
    si += v.y;
  }
  for (int r = 0; r < B; ++r) {
    const double2 v = load_partial(zp + (int64_t)r * s.npad + i);
    sr += v.x;
    si += v.y;
  }
  epilogue_finish<CPLX>(e, i, sr, si);
}

// ---------------------------------------------------------------------------
// Dense assembly out[i + m*j] = K(x_i, y_j) w_j (column-major).
// ---------------------------------------------------------------------------
template <int PDE, int KIND, int DIM>
__global__ void assemble_kernel(int64_t m, int64_t n, const double* tc, const double* tn,
                                const double* sc, const double* sn, const double* w, double k,
                                double* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t j = blockIdx.y;
  if (i >= m) return;
  const double2 v = kernel_value<PDE, KIND, DIM>(tc + DIM * i, tn ? tn + DIM * i : nullptr,
                                                 sc + DIM * j, sn ? sn + DIM * j : nullptr, k);
  const double wj = w[j];
  if (PDE == HELMHOLTZ) {
    reinterpret_cast<double2*>(out)[i + m * j] = make_double2(v.x * wj, v.y * wj);
  } else {
    out[i + m * j] = v.x * wj;
  }
}


// ---------------------------------------------------------------------------
// Host-side dispatch
// ---------------------------------------------------------------------------
int pair_tile(int precision) { return precision == INTI_FP32C ? kTile32 : kTile64; }

// e^{i m delta}, delta = fl(2 pi / kExpiTable), m = 0..kExpiTable-1, computed
// in x87 extended precision (m*delta is exact there) and rounded once.
static std::vector<long double> expi_host(bool sine) {
  const double delta = 2 * kPi / kExpiTable;
  std::vector<long double> v(kExpiTable);
  for (int m = 0; m < kExpiTable; ++m) {
    const long double a = (long double)m * (long double)delta;
    v[m] = sine ? sinl(a) : cosl(a);
  }
  return v;
}

const double2* expi_table_f64(inti_ctx* ctx) {
  if (!ctx->expi64.p) {
    const auto c = expi_host(false), s = expi_host(true);
    std::vector<double2> t(kExpiTable);
    for (int m = 0; m < kExpiTable; ++m) t[m] = make_double2((double)c[m], (double)s[m]);
    ctx->expi64.ensure(sizeof(double2) * kExpiTable);
    INTI_CUDA(cudaMemcpy(ctx->expi64.p, t.data(), sizeof(double2) * kExpiTable, cudaMemcpyHostToDevice));
  }
  return ctx->expi64.as<double2>();
}

const float2* expi_table_f32(inti_ctx* ctx) {
  if (!ctx->expi32.p) {
    const auto c = expi_host(false), s = expi_host(true);
    std::vector<float2> t(kExpiTable);
    for (int m = 0; m < kExpiTable; ++m) t[m] = make_float2((float)c[m], (float)s[m]);
    ctx->expi32.ensure(sizeof(float2) * kExpiTable);
    INTI_CUDA(cudaMemcpy(ctx->expi32.p, t.data(), sizeof(float2) * kExpiTable, cudaMemcpyHostToDevice));
  }
  return ctx->expi32.as<float2>();
}

template <class R>
static int rec_elems(int pde, int kind, int dim) {
  const bool dip = kind == DL || kind == HS || kind == CF;
  const bool cp = pde == HELMHOLTZ;
  const int used = dim + (cp ? 2 : 1) * ((dip ? dim : 1) + (kind == CF ? 1 : 0));
  const int al = 16 / (int)sizeof(R);
  return (used + al - 1) / al * al;
}

int pair_record_bytes(int pde, int kind, int dim, int precision) {
  return precision == INTI_FP32C ? rec_elems<float>(pde, kind, dim) * 4
                                 : rec_elems<double>(pde, kind, dim) * 8;
}

int pair_partial_bytes(int pde, int precision) {
  if (precision == INTI_FP32C) return pde == HELMHOLTZ ? 16 : 8;
  return pde == HELMHOLTZ ? 16 : 8;
}

// Kernel constant applied in the epilogue (see pair_step).
static double pair_scale(int pde, int kind, int dim) {
  const double c3 = 1.0 / (4 * kPi), c2 = 1.0 / (2 * kPi);
  if (kind == CF) return c3;  // 3D only: DL and SL share 1/(4 pi)
  if (pde == HELMHOLTZ) return kind == ADL ? -c3 : c3;
  if (dim == 2) {
    switch (kind) {
      case SL: return -1.0 / (4 * kPi);  // applied to log(d^2)
      case DL: return c2;
      case ADL: return -c2;
      default: return c2;
    }
  }
  return kind == ADL ? -c3 : c3;
}

template <class F>
static void dispatch(int pde, int kind, int dim, F&& f);

template <int PDE, int KIND, int DIM>
struct Tag {
  static constexpr int pde = PDE, kind = KIND, dim = DIM;
};

template <class F>
static void dispatch(int pde, int kind, int dim, F&& f) {
  if (pde == LAPLACE && dim == 3) {
    switch (kind) {
      case SL: return f(Tag<LAPLACE, SL, 3>());
      case DL: return f(Tag<LAPLACE, DL, 3>());
      case ADL: return f(Tag<LAPLACE, ADL, 3>());
      case HS: return f(Tag<LAPLACE, HS, 3>());
      case CF: return f(Tag<LAPLACE, CF, 3>());
    }
  } else if (pde == LAPLACE && dim == 2) {
    switch (kind) {
      case SL: return f(Tag<LAPLACE, SL, 2>());
      case DL: return f(Tag<LAPLACE, DL, 2>());
      case ADL: return f(Tag<LAPLACE, ADL, 2>());
      case HS: return f(Tag<LAPLACE, HS, 2>());
    }
  } else if (pde == HELMHOLTZ && dim == 3) {
    switch (kind) {
      case SL: return f(Tag<HELMHOLTZ, SL, 3>());
      case DL: return f(Tag<HELMHOLTZ, DL, 3>());
      case ADL: return f(Tag<HELMHOLTZ, ADL, 3>());
      case HS: return f(Tag<HELMHOLTZ, HS, 3>());
      case CF: return f(Tag<HELMHOLTZ, CF, 3>());
    }
  }
  throw Error(INTI_E_UNSUPPORTED, "unsupported operator: pde=" + std::to_string(pde) +
                                      " kernel=" + std::to_string(kind) +
                                      " dim=" + std::to_string(dim));
}

template <class T, class R, int TPT = kTPT>
static const void* fwd_kernel_ptr() {
  constexpr int TILE = std::is_same<R, float>::value ? kTile32 : kTile64;
  return reinterpret_cast<const void*>(&pair_forward<T::pde, T::kind, T::dim, R, TILE, TPT>);
}

template <class T, class R>
static size_t fwd_smem() {
  constexpr int TILE = std::is_same<R, float>::value ? kTile32 : kTile64;
  const size_t table = T::pde == HELMHOLTZ ? (size_t)kExpiTable * 2 * sizeof(R) : 0;
  return 2 * (size_t)TILE * Rec<T::pde, T::kind, T::dim, R>::n * sizeof(R) + table;
}

int pair_plan_split(const inti_ctx* ctx, int pde, int kind, int dim, int precision, int64_t m,
                    int64_t n, int tpt) {
  if (tpt != 2 && tpt != 4) throw Error(INTI_E_ARG, "targets per thread must be 2 or 4");
  int occ = 1;
  dispatch(pde, kind, dim, [&](auto tag) {
    using T = decltype(tag);
    const void* fn;
    size_t sm;
    if (precision == INTI_FP32C) {
      fn = tpt == 2 ? fwd_kernel_ptr<T, float, 2>() : fwd_kernel_ptr<T, float, 4>();
      sm = fwd_smem<T, float>();
    } else {
      fn = tpt == 2 ? fwd_kernel_ptr<T, double, 2>() : fwd_kernel_ptr<T, double, 4>();
      sm = fwd_smem<T, double>();
    }
    INTI_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    INTI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBlock, sm));
  });
  occ = std::max(occ, 1);
  const int64_t tile = pair_tile(precision);
  const int64_t n_tiles = std::max<int64_t>(1, (n + tile - 1) / tile);
  const int64_t blocks = (m + kBlock * tpt - 1) / (kBlock * tpt);
  const int64_t slots = (int64_t)ctx->num_sms * occ;
  // Smallest split whose last wave is >= 90% full (or that reaches 8
  // waves), never more chunks than source tiles.  Up to kMaxSplit chunks:
  // few target blocks (potentials at a few thousand points) need many.
  int best = 1;
  double best_eff = -1.0;
  for (int s = 1; s <= kMaxSplit && s <= n_tiles; ++s) {
    const int64_t tps = (n_tiles + s - 1) / s;
    const int64_t eff_s = (n_tiles + tps - 1) / tps;  // chunks actually used
    const double waves = (double)(blocks * eff_s) / (double)slots;
    const double eff = waves / std::ceil(waves);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = s;
    }
    if ((eff >= 0.9 && waves >= 1.0) || waves >= 8.0) {
      best = s;
      break;
    }
  }
  return best;
}

// Dynamic shared memory of the symmetric kernel: two source stages, the
// e^{i m delta} table, two buffers of per-warp column sums.
template <class T, class R>
static size_t symm_smem() {
  constexpr int TILE = std::is_same<R, float>::value ? kTile32 : kTile64;
  const size_t table = T::pde == HELMHOLTZ ? (size_t)kExpiTable * 2 * sizeof(R) : 0;
  return 2 * (size_t)TILE * SymRec<T::pde, T::kind, T::dim, R>::n * sizeof(R) + table +
         2 * (size_t)(kBlock / 32) * TILE * 2 * sizeof(R);
}

template <class T>
constexpr bool symm_kind() {
  return true;  // every kernel of the dispatch (3D, and 2D Laplace)
}

// FP32 Laplace SL/DL/CF in 3D run the paired-FP32 symmetric kernel.
template <class T, class R>
constexpr bool symm_x2() {
  return std::is_same<R, float>::value && T::pde == LAPLACE && T::dim == 3 &&
         (T::kind == SL || T::kind == DL || T::kind == CF);
}

template <class T>
static size_t symm_x2_smem() {
  return 2 * (size_t)kTile32 * RecX2<T::kind>::n * sizeof(float) + 2 * (size_t)(kBlock / 32) * kTile32 * 2 * sizeof(float);
}

int pair_symm_record_bytes(int pde, int kind, int dim, int precision) {
  int bytes = 0;
  dispatch(pde, kind, dim, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (symm_x2<T, float>())
      bytes = precision == INTI_FP32C ? RecX2<T::kind>::n * 4 : SymRec<T::pde, T::kind, T::dim, double>::n * 8;
    else
      bytes = precision == INTI_FP32C ? SymRec<T::pde, T::kind, T::dim, float>::n * 4
                                      : SymRec<T::pde, T::kind, T::dim, double>::n * 8;
  });
  return bytes;
}

int pair_symm_block(int tpt) { return kBlock * tpt; }

void pair_symm_plan(int64_t n, int tpt, int ch, int pcols, std::vector<int32_t>& table,
                    std::vector<SymPanel>& panels, int& nb, int& nitems) {
  const int bt = pair_symm_block(tpt);
  nb = (int)std::max<int64_t>(1, (n + bt - 1) / bt);
  ch = std::max(1, ch);
  pcols = std::max(1, std::min(pcols, nb));
  table.clear();
  panels.clear();
  nitems = 0;
  for (int c0 = 0; c0 < nb; c0 += pcols) {
    const int c1 = std::min(c0 + pcols, nb);
    std::vector<std::array<int32_t, 3>> it;
    for (int I = 0; I < c1; ++I)
      for (int J0 = std::max(I, c0); J0 < c1; J0 += ch) it.push_back({I, J0, std::min(J0 + ch, c1)});
    std::stable_sort(it.begin(), it.end(), [](const std::array<int32_t, 3>& a, const std::array<int32_t, 3>& b) {
      return a[2] - a[1] > b[2] - b[1];
    });
    SymPanel P;
    P.col0 = c0;
    P.ncols = c1 - c0;
    P.rows = c1;
    P.nitems = (int)it.size();
    P.item_off = (int)table.size();  // int32 offset of the items
    P.rowptr_off = P.item_off + 3 * P.nitems;
    P.rowitems_off = P.rowptr_off + P.rows + 1;
    table.resize((size_t)P.rowitems_off + P.nitems, 0);
    int32_t* items = table.data() + P.item_off;
    int32_t* rowptr = table.data() + P.rowptr_off;
    int32_t* rowitems = table.data() + P.rowitems_off;
    for (int q = 0; q < P.nitems; ++q) {
      items[3 * q] = it[q][0];
      items[3 * q + 1] = it[q][1];
      items[3 * q + 2] = it[q][2];
      ++rowptr[it[q][0] + 1];
    }
    for (int I = 0; I < P.rows; ++I) rowptr[I + 1] += rowptr[I];
    std::vector<int32_t> fill(rowptr, rowptr + P.rows);
    for (int q = 0; q < P.nitems; ++q) rowitems[fill[it[q][0]]++] = q;
    nitems = std::max(nitems, P.nitems);
    panels.push_back(P);
  }
}

int pair_symm_default_ch(const inti_ctx* ctx, int pde, int kind, int dim, int precision, int64_t n, int tpt) {
  int occ = 1;
  dispatch(pde, kind, dim, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (symm_kind<T>()) {
      const void* fn;
      size_t sm;
      if (precision == INTI_FP32C) {
        if constexpr (symm_x2<T, float>()) {
          fn = tpt == 2 ? (const void*)&pair_symm_x2<T::kind, 2> : (const void*)&pair_symm_x2<T::kind, 4>;
          sm = symm_x2_smem<T>();
        } else {
          fn = tpt == 2 ? (const void*)&pair_symm<T::pde, T::kind, T::dim, float, kTile32, 2>
                        : (const void*)&pair_symm<T::pde, T::kind, T::dim, float, kTile32, 4>;
          sm = symm_smem<T, float>();
        }
      } else {
        fn = tpt == 2 ? (const void*)&pair_symm<T::pde, T::kind, T::dim, double, kTile64, 2>
                      : (const void*)&pair_symm<T::pde, T::kind, T::dim, double, kTile64, 4>;
        sm = symm_smem<T, double>();
      }
      INTI_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      INTI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBlock, sm));
    }
  });
  occ = std::max(occ, 1);
  const int bt = pair_symm_block(tpt);
  const int64_t nb = std::max<int64_t>(1, (n + bt - 1) / bt);
  const int64_t pairs = nb * (nb + 1) / 2;         // block pairs J >= I
  const int64_t want = (int64_t)ctx->num_sms * occ * 8;  // about 8 waves of items
  return (int)std::max<int64_t>(1, std::min<int64_t>(nb, (pairs + want - 1) / want));
}

int pair_launch(inti_ctx* ctx, const PairLaunch& L) {
  const int tile = pair_tile(L.precision);
  const int64_t npad = L.n_tiles * tile;
  const int tps = (int)((L.n_tiles + L.split - 1) / L.split);
  int launches = 0;
  dispatch(L.pde, L.kind, L.dim, [&](auto tag) {
    using T = decltype(tag);
    auto go = [&](auto rtag) {
      using R = decltype(rtag);
      constexpr int TILE = std::is_same<R, float>::value ? kTile32 : kTile64;
      const int pb = 256;
      {
        ProfScope ps(ctx, "pack");
        const unsigned gp = (unsigned)((npad + pb - 1) / pb);
        bool done = false;
        if constexpr (symm_x2<T, R>()) {
          if (L.symm) {
            pack_sources_x2<T::kind><<<gp, pb, 0, ctx->stream>>>(L.n, npad, L.scoords, L.snormals, L.sweights, L.x,
                                                               L.c1[0], L.c2[0], static_cast<float*>(L.packed));
            done = true;
          }
        }
        if (done) {
        } else if (L.symm && (T::kind == ADL || T::kind == HS)) {
          pack_sym_normal<T::pde, T::dim, R><<<gp, pb, 0, ctx->stream>>>(L.n, npad, L.scoords, L.snormals,
                                                                         L.sweights, L.x,
                                                                         static_cast<R*>(L.packed));
        } else {
          pack_sources<T::pde, T::kind, T::dim, R><<<gp, pb, 0, ctx->stream>>>(
              L.n, npad, L.scoords, L.snormals, L.sweights, L.x, make_double2(L.c1[0], L.c1[1]),
              make_double2(L.c2[0], L.c2[1]), static_cast<R*>(L.packed));
        }
      }
      if constexpr (symm_kind<T>()) {
        if (L.symm) {
          SymArgs a;
          a.npad = npad;
          a.items = L.sym_launch ? L.sym_launch : L.sym_items;
          a.ids = L.sym_launch ? L.sym_launch_ids : nullptr;
          a.packed = L.packed;
          a.ypart = L.partial;
          a.zpart = L.zpart;
          a.k = L.k;
          a.kT = L.k * kExpiTable / (2 * kPi);
          a.delta = 2 * kPi / kExpiTable;
          a.expi = std::is_same<R, float>::value ? (const void*)expi_table_f32(ctx) : (const void*)expi_table_f64(ctx);
          a.err = L.err_flag;
          ctx->flag_armed = true;
          size_t sm;
          void (*fn)(SymArgs);
          if constexpr (symm_x2<T, R>()) {
            sm = symm_x2_smem<T>();
            fn = L.tpt == 2 ? &pair_symm_x2<T::kind, 2> : &pair_symm_x2<T::kind, 4>;
          } else {
            sm = symm_smem<T, R>();
            fn = L.tpt == 2 ? &pair_symm<T::pde, T::kind, T::dim, R, TILE, 2>
                            : &pair_symm<T::pde, T::kind, T::dim, R, TILE, 4>;
          }
          INTI_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
          a.zld = npad;
          a.zcol0 = 0;
          if (L.sym_npanels <= 1) {
            ProfScope pp(ctx, "pair");
            const int grid = L.sym_launch ? L.sym_launch_items : L.sym_nitems;
            if (grid > 0) fn<<<(unsigned)grid, kBlock, sm, ctx->stream>>>(a);
            launches = 2;
            return;
          }
          // panels one after another; after each, its partials are folded
          // into the running sums (fixed order: panels ascending)
          const int bt = pair_symm_block(L.tpt);
          const bool cplx = T::pde == HELMHOLTZ;
          INTI_CUDA(cudaMemsetAsync(L.sym_acc, 0, (size_t)L.m * (cplx ? 16 : 8), ctx->stream));
          a.zld = L.sym_zld;
          launches = 1;
          for (int p = 0; p < L.sym_npanels; ++p) {
            const SymPanel& P = L.sym_panels[p];
            int grid = P.nitems;
            a.items = L.sym_table + P.item_off;
            a.ids = nullptr;
            if (L.sym_launch) {
              grid = L.sym_launch_panels[2 * p + 1];
              a.items = L.sym_launch + 3 * L.sym_launch_panels[2 * p];
              a.ids = L.sym_launch_ids + L.sym_launch_panels[2 * p];
              INTI_CUDA(cudaMemsetAsync(L.partial, 0, L.sym_ypart_bytes, ctx->stream));
              INTI_CUDA(cudaMemsetAsync(L.zpart, 0, L.sym_zpart_bytes, ctx->stream));
            }
            a.zcol0 = (int64_t)P.col0 * bt;
            {
              ProfScope pp(ctx, "pair");
              if (grid > 0) fn<<<(unsigned)grid, kBlock, sm, ctx->stream>>>(a);
            }
            SymFold f;
            f.m = std::min<int64_t>(L.m, (int64_t)P.rows * bt);
            f.bt = bt;
            f.rowptr = L.sym_table + P.rowptr_off;
            f.rowitems = L.sym_table + P.rowitems_off;
            f.ypart = L.partial;
            f.zpart = L.zpart;
            f.zld = L.sym_zld;
            f.col0 = P.col0;
            f.ncols = P.ncols;
            f.acc = L.sym_acc;
            const unsigned gf = (unsigned)((f.m + kFoldNodes - 1) / kFoldNodes);
            const unsigned tf = kFoldNodes * kFoldSlices;
            ProfScope pf(ctx, "epilogue");
            if (std::is_same<R, float>::value) {
              if (cplx) pair_symm_fold_kernel<float4, true><<<gf, tf, 0, ctx->stream>>>(f);
              else pair_symm_fold_kernel<float2, false><<<gf, tf, 0, ctx->stream>>>(f);
            } else {
              if (cplx) pair_symm_fold_kernel<double2, true><<<gf, tf, 0, ctx->stream>>>(f);
              else pair_symm_fold_kernel<double, false><<<gf, tf, 0, ctx->stream>>>(f);
            }
            launches += 2;
          }
          return;
        }
      }
      if (L.symm) throw Error(INTI_E_UNSUPPORTED, "symmetric form of this kernel");
      FwdArgs a;
      a.m = L.m;
      a.n_tiles = L.n_tiles;
      a.tiles_per_split = tps;
      a.tcoords = L.tcoords;
      a.tnormals = L.tnormals;
      a.packed = L.packed;
      a.partial = L.partial;
      a.k = L.k;
      a.kT = L.k * kExpiTable / (2 * kPi);
      a.delta = 2 * kPi / kExpiTable;
      a.expi = std::is_same<R, float>::value ? (const void*)expi_table_f32(ctx) : (const void*)expi_table_f64(ctx);
      a.err = L.err_flag;
      ctx->flag_armed = true;
      const size_t sm = fwd_smem<T, R>();
      auto fn = L.tpt == 2 ? &pair_forward<T::pde, T::kind, T::dim, R, TILE, 2>
                           : &pair_forward<T::pde, T::kind, T::dim, R, TILE, 4>;
      INTI_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      dim3 grid((unsigned)((L.m + kBlock * L.tpt - 1) / (kBlock * L.tpt)), (unsigned)L.split);
      ProfScope pp(ctx, "pair");
      fn<<<grid, kBlock, sm, ctx->stream>>>(a);
      launches = 2;
    };
    if (L.precision == INTI_FP32C)
      go(float());
    else
      go(double());
  });
  INTI_CUDA(cudaGetLastError());
  ctx->launches += launches;
  return launches;
}

int pair_epilogue(inti_ctx* ctx, const PairLaunch& L, const inti_csr* corr, const double* x,
                  double* y, const double* alpha, const double* beta, const double* rowscale) {
  EpiArgs e;
  e.rowscale = rowscale;
  e.m = L.m;
  e.split = L.split;
  e.partial = L.partial;
  e.scale = pair_scale(L.pde, L.kind, L.dim);
  e.rowptr = corr ? corr->rowptr.as<int64_t>() : nullptr;
  e.col = corr ? corr->col.as<int32_t>() : nullptr;
  e.val = corr ? corr->val.as<double>() : nullptr;
  e.x = x;
  e.y = y;
  e.ar = alpha ? alpha[0] : 1.0;
  e.ai = alpha ? alpha[1] : 0.0;
  e.br = beta ? beta[0] : 0.0;
  e.bi = beta ? beta[1] : 0.0;
  e.beta_zero = (e.br == 0.0 && e.bi == 0.0);
  const int tb = 256;
  const unsigned gb = (unsigned)((L.m + tb - 1) / tb);
  const bool cplx = L.pde == HELMHOLTZ;
  ProfScope pe(ctx, "epilogue");
  if (L.symm && L.sym_npanels > 1) {
    // the panels' running sums hold the whole pair product
    e.partial = L.sym_acc;
    e.split = 1;
    if (cplx)
      pair_epilogue_kernel<double2, true><<<gb, tb, 0, ctx->stream>>>(e);
    else
      pair_epilogue_kernel<double, false><<<gb, tb, 0, ctx->stream>>>(e);
    INTI_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return 1;
  }
  if (L.symm) {
    SymEpi se;
    se.npad = L.n_tiles * pair_tile(L.precision);
    se.bt = pair_symm_block(L.tpt);
    se.rowptr = L.sym_rowptr;
    se.rowitems = L.sym_rowitems;
    se.zpart = L.zpart;
    if (L.precision == INTI_FP32C) {
      if (cplx)
        pair_symm_epilogue_kernel<float4, true><<<gb, tb, 0, ctx->stream>>>(e, se);
      else
        pair_symm_epilogue_kernel<float2, false><<<gb, tb, 0, ctx->stream>>>(e, se);
    } else {
      if (cplx)
        pair_symm_epilogue_kernel<double2, true><<<gb, tb, 0, ctx->stream>>>(e, se);
      else
        pair_symm_epilogue_kernel<double, false><<<gb, tb, 0, ctx->stream>>>(e, se);
    }
    INTI_CUDA(cudaGetLastError());
    ctx->launches += 1;
    return 1;
  }
  if (L.precision == INTI_FP32C) {
    if (cplx)
      pair_epilogue_kernel<float4, true><<<gb, tb, 0, ctx->stream>>>(e);
    else
      pair_epilogue_kernel<float2, false><<<gb, tb, 0, ctx->stream>>>(e);
  } else {
    if (cplx)
      pair_epilogue_kernel<double2, true><<<gb, tb, 0, ctx->stream>>>(e);
    else
      pair_epilogue_kernel<double, false><<<gb, tb, 0, ctx->stream>>>(e);
  }
  INTI_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return 1;
}

bool pair_small_eligible(int precision, int64_t m, int64_t n) {
  // sources capped so that a thread's chain (n / (8 slices * 8 warps)) stays short
  return precision == INTI_FP64 && (double)m * (double)n <= kSmallPairs && m > 0 && n > 0 && n <= 65536;
}

static int pair_small_slices(int num_sms, int64_t m, int64_t n) {
  const int64_t rows = (m + 31) / 32;
  int s = 1;
  while (s < kSmallMaxSlices && rows * 2 * s <= num_sms && n >= (int64_t)64 * 2 * s) s *= 2;
  return s;
}

int pair_small(inti_ctx* ctx, const PairLaunch& L, const inti_csr* corr, const double* x, double* y,
               const double* alpha, const double* beta, const double* rowscale) {
  EpiArgs e;
  e.rowscale = rowscale;
  e.m = L.m;
  e.split = 1;
  e.partial = nullptr;
  e.scale = pair_scale(L.pde, L.kind, L.dim);
  e.rowptr = corr ? corr->rowptr.as<int64_t>() : nullptr;
  e.col = corr ? corr->col.as<int32_t>() : nullptr;
  e.val = corr ? corr->val.as<double>() : nullptr;
  e.x = x;
  e.y = y;
  e.ar = alpha ? alpha[0] : 1.0;
  e.ai = alpha ? alpha[1] : 0.0;
  e.br = beta ? beta[0] : 0.0;
  e.bi = beta ? beta[1] : 0.0;
  e.beta_zero = (e.br == 0.0 && e.bi == 0.0);
  const SmallSources src{L.scoords, L.snormals, L.sweights, L.x, make_double2(L.c1[0], L.c1[1]),
                         make_double2(L.c2[0], L.c2[1])};
  const int slices = pair_small_slices(ctx->num_sms, L.m, L.n);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = slices;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)((L.m + 31) / 32 * slices));
  cfg.blockDim = dim3(32 * kSmallWarps);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const double2* expi = L.pde == HELMHOLTZ ? expi_table_f64(ctx) : nullptr;
  const double kT = L.k * kExpiTable / (2 * kPi), delta = 2 * kPi / kExpiTable;
  dispatch(L.pde, L.kind, L.dim, [&](auto tag) {
    using T = decltype(tag);
    ProfScope pp(ctx, "pair");
    INTI_CUDA(cudaLaunchKernelEx(&cfg, pair_small_kernel<T::pde, T::kind, T::dim>, (int64_t)L.m, (int64_t)L.n,
                                 L.tcoords, L.tnormals, src, (double)L.k, kT, delta, expi, e));
  });
  INTI_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return 1;
}

int pair_assemble(inti_ctx* ctx, const PairLaunch& L, double* out) {
  if (L.n > 65535 * 1024LL) throw Error(INTI_E_ARG, "assemble: too many source columns");
  if (L.kind == CF) throw Error(INTI_E_UNSUPPORTED, "assemble the DL and SL parts separately");
  dispatch(L.pde, L.kind, L.dim, [&](auto tag) {
    using T = decltype(tag);
    if constexpr (T::kind != CF) {
      dim3 grid((unsigned)((L.m + 255) / 256), (unsigned)L.n);
      assemble_kernel<T::pde, T::kind, T::dim><<<grid, 256, 0, ctx->stream>>>(
          L.m, L.n, L.tcoords, L.tnormals, L.scoords, L.snormals, L.sweights, L.k, out);
    }
  });
  INTI_CUDA(cudaGetLastError());
  ctx->launches += 1;
  return 1;
}

// Transpose: the roles of the two node sets swap; partial is split x n double2.
// ===========================================================================
// Allocation-free apply.
//
// Some callers cannot call cudaMalloc at the moment they need the operator:
// code running inside a framework whose caching allocator already owns nearly
// all device memory (so a fresh cudaMalloc fails or fragments it), and code
// that must not pay an allocation's latency or implicit synchronisation in a
// solver loop.  inti_apply_noalloc serves them:
// the caller passes every input and output as device pointers, and the
// scratch the pair product needs (packed source records and per-chunk partial
// sums) lives in one fixed array of kNoAllocScratchBytes declared below.  The
// module holds that array on every GPU that loads the library, until exit.
//
// The first call on a device resolves the array's device address with
// cudaGetSymbolAddress and uploads the e^{i m delta} tables into static
// device arrays; make that first call before any stream capture.  Every call
// on a device shares the array and leaves its contents behind: calls that
// overlap on the GPU (different streams, or different host threads) race
// on it.  Nothing in the array has to start at zero: the pack kernel writes
// every record (padding included) and the pair kernel writes every partial
// slot it owns; only the timeout flag is cleared at the start of each call.
// If a bounded wait of the pair kernel runs out, the epilogue writes NaN into
// every entry of y (with synchronize = 0 no status reports the timeout).
// ===========================================================================
constexpr size_t kNoAllocScratchBytes = 32u << 20;  // 32 MiB
constexpr size_t kNoAllocFlagBytes = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ __align__(16) double2 g_noalloc_expi64[kExpiTable];
static __device__ __align__(16) float2 g_noalloc_expi32[kExpiTable];

namespace {

struct NoAllocDevice {
  unsigned char* scratch = nullptr;
  const double2* expi64 = nullptr;
  const float2* expi32 = nullptr;
  int num_sms = 0;
};

std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc_dev[64];

// Once per device, with that device current: resolve the static arrays'
// device addresses (the host-side names are not device addresses) and fill
// the phase tables.
const NoAllocDevice& noalloc_setup(int dev) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 64) throw Error(INTI_E_ARG, "device index out of range for the static scratch");
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (d.scratch) return d;
  void* p = nullptr;
  INTI_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  void* t64 = nullptr;
  INTI_CUDA(cudaGetSymbolAddress(&t64, g_noalloc_expi64));
  void* t32 = nullptr;
  INTI_CUDA(cudaGetSymbolAddress(&t32, g_noalloc_expi32));
  const auto c = expi_host(false), s = expi_host(true);
  std::vector<double2> h64(kExpiTable);
  std::vector<float2> h32(kExpiTable);
  for (int m = 0; m < kExpiTable; ++m) {
    h64[m] = make_double2((double)c[m], (double)s[m]);
    h32[m] = make_float2((float)c[m], (float)s[m]);
  }
  INTI_CUDA(cudaMemcpyToSymbol(g_noalloc_expi64, h64.data(), sizeof(double2) * kExpiTable));
  INTI_CUDA(cudaMemcpyToSymbol(g_noalloc_expi32, h32.data(), sizeof(float2) * kExpiTable));
  INTI_CUDA(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev));
  d.expi64 = static_cast<const double2*>(t64);
  d.expi32 = static_cast<const float2*>(t32);
  d.scratch = static_cast<unsigned char*>(p);
  return d;
}

}  // namespace

int apply_noalloc(int pde, int kind, int dim, double k, int precision, int64_t m, const double* tc,
                  const double* tn, int64_t n, const double* sc, const double* sn, const double* sw,
                  const int64_t* rowptr, const int32_t* col, const double* val, const double* x, double* y,
                  const double* alpha, const double* beta, cudaStream_t stream, int synchronize) {
  if (pde != INTI_LAPLACE && pde != INTI_HELMHOLTZ) throw Error(INTI_E_ARG, "unknown pde");
  if (kind < INTI_SL || kind > INTI_HS) throw Error(INTI_E_ARG, "unknown kernel");
  if (precision != INTI_FP64 && precision != INTI_FP32C) throw Error(INTI_E_ARG, "unknown precision");
  if (dim != 2 && dim != 3) throw Error(INTI_E_ARG, "dim must be 2 or 3");
  if (pde == INTI_HELMHOLTZ && dim != 3) throw Error(INTI_E_UNSUPPORTED, "Helmholtz is implemented in 3D only");
  if (m <= 0 || n <= 0) throw Error(INTI_E_ARG, "m and n must be positive");
  if (!tc || !sc || !sw || !x || !y) throw Error(INTI_E_ARG, "a required device pointer is NULL");
  if ((kind == DL || kind == HS) && !sn) throw Error(INTI_E_ARG, "this kernel needs source normals");
  if ((kind == ADL || kind == HS) && !tn) throw Error(INTI_E_ARG, "this kernel needs target normals");
  if ((rowptr || col || val) && !(rowptr && col && val))
    throw Error(INTI_E_ARG, "the correction needs rowptr, col and val together");
  int dev = 0;
  INTI_CUDA(cudaGetDevice(&dev));
  const NoAllocDevice& D = noalloc_setup(dev);
  const int64_t tile = pair_tile(precision);
  const int64_t n_tiles = (n + tile - 1) / tile;
  const size_t rec_bytes = (size_t)n_tiles * tile * pair_record_bytes(pde, kind, dim, precision);
  const size_t packed_bytes = (rec_bytes + 255) / 256 * 256;
  const size_t pbytes = (size_t)m * pair_partial_bytes(pde, precision);
  const size_t room = kNoAllocScratchBytes - kNoAllocFlagBytes;
  if (packed_bytes + pbytes > room)
    throw Error(INTI_E_ARG, "problem too large for the fixed " + std::to_string(kNoAllocScratchBytes >> 20) +
                                " MiB scratch of inti_apply_noalloc: needs " +
                                std::to_string(packed_bytes + pbytes) + " bytes (use inti_op_apply)");
  // source chunks: enough CTAs for ~2 waves, bounded by the scratch and the tiles
  const int64_t blocks = (m + kBlock * kTPT - 1) / (kBlock * kTPT);
  int64_t split = std::max<int64_t>(1, (2LL * D.num_sms * 4 + blocks - 1) / blocks);
  split = std::min<int64_t>({split, n_tiles, 64, (int64_t)((room - packed_bytes) / pbytes)});
  const int64_t tps = (n_tiles + split - 1) / split;
  split = (n_tiles + tps - 1) / tps;
  int* flag = reinterpret_cast<int*>(D.scratch);
  void* packed = D.scratch + kNoAllocFlagBytes;
  void* partial = D.scratch + kNoAllocFlagBytes + packed_bytes;
  INTI_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), stream));
  dispatch(pde, kind, dim, [&](auto tag) {
    using T = decltype(tag);
    auto go = [&](auto rtag) {
      using R = decltype(rtag);
      constexpr int TILE = std::is_same<R, float>::value ? kTile32 : kTile64;
      const int64_t npad = n_tiles * TILE;
      pack_sources<T::pde, T::kind, T::dim, R><<<(unsigned)((npad + 255) / 256), 256, 0, stream>>>(
          n, npad, sc, sn, sw, x, make_double2(1.0, 0.0), make_double2(0.0, 0.0), static_cast<R*>(packed));
      FwdArgs a;
      a.m = m;
      a.n_tiles = n_tiles;
      a.tiles_per_split = (int)tps;
      a.tcoords = tc;
      a.tnormals = tn;
      a.packed = packed;
      a.partial = partial;
      a.k = k;
      a.kT = k * kExpiTable / (2 * kPi);
      a.delta = 2 * kPi / kExpiTable;
      a.expi = std::is_same<R, float>::value ? (const void*)D.expi32 : (const void*)D.expi64;
      a.err = flag;
      const size_t sm = fwd_smem<T, R>();
      auto fn = &pair_forward<T::pde, T::kind, T::dim, R, TILE>;
      INTI_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      fn<<<dim3((unsigned)blocks, (unsigned)split), kBlock, sm, stream>>>(a);
    };
    if (precision == INTI_FP32C)
      go(float());
    else
      go(double());
  });
  EpiArgs e;
  e.m = m;
  e.split = (int)split;
  e.partial = partial;
  e.scale = pair_scale(pde, kind, dim);
  e.rowptr = rowptr;
  e.col = col;
  e.val = val;
  e.x = x;
  e.y = y;
  e.ar = alpha ? alpha[0] : 1.0;
  e.ai = alpha ? alpha[1] : 0.0;
  e.br = beta ? beta[0] : 0.0;
  e.bi = beta ? beta[1] : 0.0;
  e.beta_zero = (e.br == 0.0 && e.bi == 0.0);
  e.err = flag;
  const unsigned gb = (unsigned)((m + 255) / 256);
  const bool cplx = pde == HELMHOLTZ;
  if (precision == INTI_FP32C) {
    if (cplx)
      pair_epilogue_kernel<float4, true><<<gb, 256, 0, stream>>>(e);
    else
      pair_epilogue_kernel<float2, false><<<gb, 256, 0, stream>>>(e);
  } else {
    if (cplx)
      pair_epilogue_kernel<double2, true><<<gb, 256, 0, stream>>>(e);
    else
      pair_epilogue_kernel<double, false><<<gb, 256, 0, stream>>>(e);
  }
  INTI_CUDA(cudaGetLastError());
  if (synchronize) {
    INTI_CUDA(cudaStreamSynchronize(stream));
    int f = 0;
    INTI_CUDA(cudaMemcpy(&f, flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (f) throw Error(INTI_E_TIMEOUT, "a device-side bounded wait ran out (code " + std::to_string(f) + ")");
  }
  return INTI_OK;
}

}  // namespace inti

extern "C" int inti_apply_noalloc(int pde, int kernel, int dim, double k, int precision, int64_t m,
                                  const double* tcoords, const double* tnormals, int64_t n,
                                  const double* scoords, const double* snormals, const double* sweights,
                                  const int64_t* rowptr, const int32_t* col, const double* val,
                                  const double* x, double* y, const double* alpha, const double* beta,
                                  void* stream, int synchronize) {
  try {
    return inti::apply_noalloc(pde, kernel, dim, k, precision, m, tcoords, tnormals, n, scoords, snormals,
                               sweights, rowptr, col, val, x, y, alpha, beta,
                               static_cast<cudaStream_t>(stream), synchronize);
  } catch (const inti::Error& e) {
    inti::noalloc_error_set(e.what());
    return e.code;
  } catch (const std::exception& e) {
    inti::noalloc_error_set(e.what());
    return INTI_E_ARG;
  }
}
