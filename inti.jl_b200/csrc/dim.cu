// Boundary density-interpolation (BDIM) correction built on the GPU, for
// target === source (src/bdim.jl:50-196 with the X === Y branch of
// etype_to_nearest_points, src/quadrature.jl:249-256):
//
//  1. ns = ceil(3*nq) monopole centres on a circle/sphere of radius
//     1.5*|bbox diagonal|/2 about the bounding-box centre (bdim.jl:79-92,
//     utils.jl:142-171) — host, O(n).
//  2. traces g0[j,k] = G(y_j, xs_k), g1[j,k] = ADL(y_j, xs_k) (bdim.jl:94-103).
//  3. Theta = mu*B(x) + S*g1 - D*g0 (bdim.jl:104-118): a multi-right-hand-side
//     pair product over all node pairs, S and D being the uncorrected Nystrom
//     operators (entries K*w), evaluated on the fly and never stored.
//  4. per element: Householder QR of M^T = [g0[el,:]; g1[el,:]]^T (ns x 2nq)
//     and least squares for each of the element's nq nodes (bdim.jl:154-185);
//     one warp per element, lane l owning row l.
//  5. values dS[i, e*nq+a] = -W[nq+a], dD[i, e*nq+a] = W[a] (bdim.jl:176-179)
//     written straight into CSR arrays with the element-block pattern.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "common.h"
#include "device_common.cuh"
#include "fp64_mma.cuh"
#include "internal.h"

namespace inti {

// Scalar abstraction: double (Laplace) or double2 (Helmholtz).
template <bool CPLX>
struct S;
template <>
struct S<false> {
  using T = double;
  static __device__ __forceinline__ T from(double2 v) { return v.x; }
  static __device__ __forceinline__ T zero() { return 0.0; }
  static __device__ __forceinline__ T one() { return 1.0; }
  static __device__ __forceinline__ T mul(T a, T b) { return a * b; }
  static __device__ __forceinline__ T cmul(T a, T b) { return a * b; }  // conj(a)*b
  static __device__ __forceinline__ T add(T a, T b) { return a + b; }
  static __device__ __forceinline__ T sub(T a, T b) { return a - b; }
  static __device__ __forceinline__ T scale(T a, double s) { return a * s; }
  static __device__ __forceinline__ double abs2(T a) { return a * a; }
  static __device__ __forceinline__ double re(T a) { return a; }
  static __device__ __forceinline__ double im(T) { return 0.0; }
  static __device__ __forceinline__ T conj(T a) { return a; }
  static __device__ __forceinline__ T div(T a, T b) { return a / b; }
  static __device__ __forceinline__ T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
  static __device__ __forceinline__ T wsum(T v) { return warp_sum(v); }
  static __device__ __forceinline__ T neg(T a) { return -a; }
  // acc + a*b and acc - a*b as fused multiply-adds
  static __device__ __forceinline__ T fmadd(T acc, T a, T b) { return fma(a, b, acc); }
  static __device__ __forceinline__ T fmsub(T acc, T a, T b) { return fma(-a, b, acc); }
};
template <>
struct S<true> {
  using T = double2;
  static __device__ __forceinline__ T from(double2 v) { return v; }
  static __device__ __forceinline__ T zero() { return make_double2(0.0, 0.0); }
  static __device__ __forceinline__ T one() { return make_double2(1.0, 0.0); }
  static __device__ __forceinline__ T mul(T a, T b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  static __device__ __forceinline__ T cmul(T a, T b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
  }
  static __device__ __forceinline__ T add(T a, T b) { return make_double2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ T sub(T a, T b) { return make_double2(a.x - b.x, a.y - b.y); }
  static __device__ __forceinline__ T scale(T a, double s) { return make_double2(a.x * s, a.y * s); }
  static __device__ __forceinline__ double abs2(T a) { return a.x * a.x + a.y * a.y; }
  static __device__ __forceinline__ double re(T a) { return a.x; }
  static __device__ __forceinline__ double im(T a) { return a.y; }
  static __device__ __forceinline__ T conj(T a) { return make_double2(a.x, -a.y); }
  static __device__ __forceinline__ T div(T a, T b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
  }
  static __device__ __forceinline__ T shfl(T v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
  }
  static __device__ __forceinline__ T wsum(T v) { return make_double2(warp_sum(v.x), warp_sum(v.y)); }
  static __device__ __forceinline__ T neg(T a) { return make_double2(-a.x, -a.y); }
  static __device__ __forceinline__ T fmadd(T acc, T a, T b) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
  }
  static __device__ __forceinline__ T fmsub(T acc, T a, T b) {
    return make_double2(fma(-a.x, b.x, fma(a.y, b.y, acc.x)), fma(-a.x, b.y, fma(-a.y, b.x, acc.y)));
  }
};

// S and D kernel values of one pair (without the weight), sharing r, 1/d and
// e^{ikd}: in 3D the single/double layer (DERIV false) or the adjoint double
// layer / hypersingular pair (DERIV true, target normal ni) from the refined
// hardware rsqrt and the tabulated e^{ikd} of the pair kernels (tab: the
// device table, read-only); 2D through kernel_value.
template <int PDE, int DIM, bool DERIV>
__device__ __forceinline__ void theta_sd(const double* xi, const double* ni, const double* yj,
                                         const double* nj, double k, double kT, double delta,
                                         const double2* __restrict__ tab, double2& sv, double2& dv) {
  if (DIM == 3 && !DERIV) {
    const double r0 = xi[0] - yj[0], r1 = xi[1] - yj[1], r2 = xi[2] - yj[2];
    const double d2 = fma(r2, r2, fma(r1, r1, r0 * r0));
    const double ri = pair_keep(d2) ? rsqrt_fast(d2) : 0.0;  // self pair: every value 0
    const double rn = fma(r2, nj[2], fma(r1, nj[1], r0 * nj[0]));
    constexpr double c4 = 1.0 / (4 * kPi);
    if (PDE == LAPLACE) {
      sv = make_double2(c4 * ri, 0.0);
      dv = make_double2(c4 * rn * (ri * ri * ri), 0.0);
    } else {
      double c, s;  // e^{ikd}
      expi_table_eval(d2 * ri, kT, tab, delta, c, s);
      const double g = c4 * ri;
      sv = make_double2(g * c, g * s);
      // e^{ikd} (1/d - ik) (r.n_y) / (4 pi d^2)
      const double h = c4 * rn * ri * ri;
      dv = make_double2(h * fma(c, ri, k * s), h * fma(s, ri, -k * c));
    }
  } else if (DIM == 3) {
    // derivative: (ADL, HS) with the target normal n_x = ni, source normal n_y
    const double r0 = xi[0] - yj[0], r1 = xi[1] - yj[1], r2 = xi[2] - yj[2];
    const double d2 = fma(r2, r2, fma(r1, r1, r0 * r0));
    const double ri = pair_keep(d2) ? rsqrt_fast(d2) : 0.0;
    const double rnx = fma(r2, ni[2], fma(r1, ni[1], r0 * ni[0]));
    const double rny = fma(r2, nj[2], fma(r1, nj[1], r0 * nj[0]));
    const double nn = fma(ni[2], nj[2], fma(ni[1], nj[1], ni[0] * nj[0]));
    constexpr double c4 = 1.0 / (4 * kPi);
    const double id2 = ri * ri;
    if (PDE == LAPLACE) {
      const double ri3 = id2 * ri;
      sv = make_double2(-c4 * rnx * ri3, 0.0);
      dv = make_double2(c4 * fma(-3.0 * rnx * rny, id2, nn) * ri3, 0.0);
    } else {
      const double d = d2 * ri;
      double c, s;  // e^{ikd}
      expi_table_eval(d, kT, tab, delta, c, s);
      // -e^{ikd} (1/d - ik) (r.n_x) / (4 pi d^2)
      const double f = -c4 * rnx * id2;
      sv = make_double2(f * fma(c, ri, k * s), f * fma(s, ri, -k * c));
      // e^{ikd} [(1/d - ik) p + (k^2 d^2 - 3 + 3ikd) s5] / (4 pi) with
      // p = (n_x.n_y)/d^2, s5 = (r.n_x)(r.n_y)/d^5
      const double kd = k * d;
      const double fr = fma(kd, kd, -3.0), fi = 3.0 * kd;
      const double p = nn * id2;
      const double s5 = (rnx * rny) * (id2 * id2 * ri);
      const double wr = c4 * fma(ri, p, fr * s5), wi = c4 * fma(-k, p, fi * s5);
      dv = make_double2(fma(c, wr, -s * wi), fma(c, wi, s * wr));
    }
  } else {
    constexpr int KS = DERIV ? ADL : SL;
    constexpr int KD = DERIV ? HS : DL;
    sv = kernel_value<PDE, KS, DIM>(xi, ni, yj, nj, k);
    dv = kernel_value<PDE, KD, DIM>(xi, ni, yj, nj, k);
  }
}

// ---------------------------------------------------------------------------
// 2. traces: g0/g1 are n x ns, row-major (ns contiguous per node).
// ---------------------------------------------------------------------------
template <int PDE, int DIM>
__global__ void dim_traces(int64_t n, int ns, const double* __restrict__ x,
                           const double* __restrict__ nrm, const double* __restrict__ xs, double k,
                           double2* __restrict__ g0, double2* __restrict__ g1) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n * ns) return;
  const int64_t j = t / ns;
  const int kk = (int)(t % ns);
  g0[t] = kernel_value<PDE, SL, DIM>(x + DIM * j, nrm + DIM * j, xs + DIM * kk, nullptr, k);
  g1[t] = kernel_value<PDE, ADL, DIM>(x + DIM * j, nrm + DIM * j, xs + DIM * kk, nullptr, k);
}

// ---------------------------------------------------------------------------
// 3. Theta partials: for targets i (one per thread) and a chunk of sources,
//    acc[k] = sum_j (K_S(x_i,y_j) w_j) g1[j,k] - (K_D(x_i,y_j) w_j) g0[j,k].
//    Source data and trace rows are staged in shared memory.
// ---------------------------------------------------------------------------
constexpr int kThetaBlock = 128;
constexpr int kThetaTile = 32;

template <int PDE, int DIM, bool DERIV, int NS>
__global__ void __launch_bounds__(kThetaBlock) dim_theta(
    int64_t m, int64_t n, int ns, const double* __restrict__ tx, const double* __restrict__ tn,
    const double* __restrict__ x, const double* __restrict__ nrm, const double* __restrict__ w,
    const double2* __restrict__ g0, const double2* __restrict__ g1, double k, double kT, double delta,
    const double2* __restrict__ tab, int tiles_per_split, double2* __restrict__ partial) {
  constexpr bool CPLX = PDE == HELMHOLTZ;
  using Sc = S<CPLX>;
  using T = typename Sc::T;
  __shared__ double sx[kThetaTile * DIM], sn[kThetaTile * DIM], sw[kThetaTile];
  __shared__ T s0[kThetaTile * NS], s1[kThetaTile * NS];
  const int64_t i = blockIdx.x * (int64_t)kThetaBlock + threadIdx.x;
  const int64_t ii = min(i, m - 1);
  double xi[DIM], ni[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    xi[c] = tx[DIM * ii + c];
    ni[c] = tn ? tn[DIM * ii + c] : 0.0;  // target normals enter ADL/HS only
  }
  T acc[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) acc[q] = Sc::zero();
  const int64_t ntile = (n + kThetaTile - 1) / kThetaTile;
  const int64_t t0 = (int64_t)blockIdx.y * tiles_per_split;
  const int64_t t1 = min(ntile, t0 + tiles_per_split);
  for (int64_t t = t0; t < t1; ++t) {
    __syncthreads();
    for (int q = threadIdx.x; q < kThetaTile; q += kThetaBlock) {
      const int64_t j = t * kThetaTile + q;
      const bool in = j < n;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        sx[q * DIM + c] = in ? x[DIM * j + c] : 0.0;
        sn[q * DIM + c] = in ? nrm[DIM * j + c] : 0.0;
      }
      sw[q] = in ? w[j] : 0.0;
    }
    for (int q = threadIdx.x; q < kThetaTile * NS; q += kThetaBlock) {
      const int a = q / NS, kk = q % NS;
      const int64_t j = t * kThetaTile + a;
      const bool in = j < n && kk < ns;
      s0[q] = in ? Sc::from(g0[j * ns + kk]) : Sc::zero();
      s1[q] = in ? Sc::from(g1[j * ns + kk]) : Sc::zero();
    }
    __syncthreads();
#pragma unroll 1
    for (int a = 0; a < kThetaTile; ++a) {
      const double wj = sw[a];
      double2 sv2, dv2;
      theta_sd<PDE, DIM, DERIV>(xi, ni, &sx[a * DIM], &sn[a * DIM], k, kT, delta, tab, sv2, dv2);
      const T sv = Sc::scale(Sc::from(sv2), wj);
      const T dv = Sc::scale(Sc::from(dv2), wj);
#pragma unroll
      for (int q = 0; q < NS; ++q) acc[q] = Sc::fmsub(Sc::fmadd(acc[q], sv, s1[a * NS + q]), dv, s0[a * NS + q]);
    }
  }
  if (i < m) {
    double2* out = partial + ((int64_t)blockIdx.y * m + i) * ns;
#pragma unroll
    for (int q = 0; q < NS; ++q)
      if (q < ns) out[q] = make_double2(Sc::re(acc[q]), Sc::im(acc[q]));
  }
}

// Theta partials on the FP64 MMA path (3D; DERIV: the (ADL, HS) pair of the
// derivative corrections in place of (S, D)): per tile of J
// sources the CUDA cores evaluate (S w, D w) once per pair into A (complex:
// slots Sr, Si, Dr, Di), the trace rows are staged as B (real: rows g1, -g0;
// complex, with (Re, Im) column pairs: (g1r, g1i), (-g1i, g1r), (-g0r, -g0i),
// (g0i, -g0r)), and the warps multiply A B with the FP64 MMA.  The next
// tile's traces and source records are loaded during the MMA phase.  Same
// partial layout as dim_theta.
template <int PDE, bool WIDE>
struct ThetaMma;
template <bool WIDE>
struct ThetaMma<LAPLACE, WIDE> {
  static constexpr int J = 16, NA = 2, kMaxNs = 32;
  using Sh = MmaShape<8, 1, 4, J * NA, 1>;  // 256 targets x 32 columns
};
template <bool WIDE>
struct ThetaMma<HELMHOLTZ, WIDE> {
  static constexpr int J = 8, NA = 4, kMaxNs = WIDE ? 32 : 24;
  using Sh = MmaShape<4, 2, WIDE ? 4 : 3, J * NA, 2>;  // 128 targets x 24 or 32 complex columns
};
template <int PDE, bool WIDE>
constexpr size_t theta_mma_smem() {
  using Sh = typename ThetaMma<PDE, WIDE>::Sh;
  return sizeof(double) * ((size_t)Sh::MT * Sh::LDA + (size_t)Sh::kK * Sh::LDB + 7 * ThetaMma<PDE, WIDE>::J) +
         (PDE == HELMHOLTZ ? sizeof(double2) * kExpiTable : 0);
}

template <int PDE, bool WIDE, bool DERIV>
__global__ void __launch_bounds__(kMmaThreads, 2) dim_theta_mma(
    int64_t m, int64_t n, int ns, const double* __restrict__ tx, const double* __restrict__ tn,
    const double* __restrict__ x,
    const double* __restrict__ nrm, const double* __restrict__ w, const double2* __restrict__ g0,
    const double2* __restrict__ g1, double k, double kT, double delta, const double2* __restrict__ tab_g,
    int tiles_per_split, double2* __restrict__ partial) {
  using TM = ThetaMma<PDE, WIDE>;
  using Sh = typename TM::Sh;
  constexpr bool CPLX = PDE == HELMHOLTZ;
  constexpr int J = TM::J, NA = TM::NA;
  constexpr int R = kMmaThreads / Sh::MT;                            // threads per target in phase 1
  constexpr int XPER = (J * TM::kMaxNs + kMmaThreads - 1) / kMmaThreads;  // trace values per thread
  static_assert(J % R == 0 && 7 * J <= kMmaThreads, "shape");
  extern __shared__ __align__(16) double smem_d[];
  double* As = smem_d;
  double* Bs = As + Sh::MT * Sh::LDA;
  double* sx = Bs + Sh::kK * Sh::LDB;
  double* sn = sx + 3 * J;
  double* sw = sx + 6 * J;
  double2* tab = reinterpret_cast<double2*>(sx + 7 * J);
  const int tid = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * Sh::MT;
  const int mloc = tid % Sh::MT, r0 = tid / Sh::MT;
  const int64_t ii = min(base + mloc, m - 1);
  const double xi[3] = {tx[3 * ii], tx[3 * ii + 1], tx[3 * ii + 2]};
  double ni[3] = {0.0, 0.0, 0.0};  // target normal: derivative corrections only
  if (DERIV) {
    ni[0] = tn[3 * ii];
    ni[1] = tn[3 * ii + 1];
    ni[2] = tn[3 * ii + 2];
  }
  for (int q = tid; q < Sh::kK * Sh::LDB; q += kMmaThreads) Bs[q] = 0.0;  // padding columns stay zero
  if (CPLX)
    for (int q = tid; q < kExpiTable; q += kMmaThreads) tab[q] = tab_g[q];
  const int64_t ntile = (n + J - 1) / J;
  const int64_t t0 = (int64_t)blockIdx.y * tiles_per_split;
  const int64_t t1 = min(ntile, t0 + tiles_per_split);
  const int tot = J * ns;  // trace values per tile and array
  double2 p0[XPER], p1[XPER];
  double spre = 0.0;
  auto prefetch = [&](int64_t t) {
    const int64_t j0 = t * J;
#pragma unroll
    for (int r = 0; r < XPER; ++r) {
      const int e = tid + r * kMmaThreads;
      const int64_t j = j0 + e / ns;
      const bool in = e < tot && j < n;
      const int64_t idx = j0 * ns + e;  // traces are node-major, ns per node
      p0[r] = in ? g0[idx] : make_double2(0.0, 0.0);
      p1[r] = in ? g1[idx] : make_double2(0.0, 0.0);
    }
    if (tid < 7 * J) {
      const int f = tid / J, q = tid % J;
      const int64_t j = j0 + q;
      double v = 0.0;
      if (j < n) v = f < 3 ? x[3 * j + f] : (f < 6 ? nrm[3 * j + f - 3] : w[j]);
      spre = v;
    }
  };
  auto store_staged = [&]() {
#pragma unroll
    for (int r = 0; r < XPER; ++r) {
      const int e = tid + r * kMmaThreads;
      if (e >= tot) continue;
      const int q = e / ns, kk = e % ns;
      const double2 a0 = p0[r], a1 = p1[r];
      if (CPLX) {
        const int k0 = NA * q;
        *reinterpret_cast<double2*>(&Bs[(k0 + 0) * Sh::LDB + Sh::bcol(k0 + 0, 2 * kk)]) = a1;
        *reinterpret_cast<double2*>(&Bs[(k0 + 1) * Sh::LDB + Sh::bcol(k0 + 1, 2 * kk)]) = make_double2(-a1.y, a1.x);
        *reinterpret_cast<double2*>(&Bs[(k0 + 2) * Sh::LDB + Sh::bcol(k0 + 2, 2 * kk)]) = make_double2(-a0.x, -a0.y);
        *reinterpret_cast<double2*>(&Bs[(k0 + 3) * Sh::LDB + Sh::bcol(k0 + 3, 2 * kk)]) = make_double2(a0.y, -a0.x);
      } else {
        Bs[(2 * q) * Sh::LDB + Sh::bcol(2 * q, kk)] = a1.x;
        Bs[(2 * q + 1) * Sh::LDB + Sh::bcol(2 * q + 1, kk)] = -a0.x;
      }
    }
    if (tid < 7 * J) {
      const int f = tid / J, q = tid % J;
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
  if (t0 < t1) prefetch(t0);
  for (int64_t t = t0; t < t1; ++t) {
    __syncthreads();  // previous tile consumed (and B zeroed, table loaded)
    store_staged();
    __syncthreads();
#pragma unroll 2
    for (int q = r0; q < J; q += R) {
      double2 sv, dv;
      theta_sd<PDE, 3, DERIV>(xi, ni, &sx[3 * q], &sn[3 * q], k, kT, delta, tab, sv, dv);
      const double wq = sw[q];
      if (CPLX) {
        double* a = &As[mloc * Sh::LDA + NA * q];
        *reinterpret_cast<double2*>(a) = make_double2(sv.x * wq, sv.y * wq);
        *reinterpret_cast<double2*>(a + 2) = make_double2(dv.x * wq, dv.y * wq);
      } else {
        *reinterpret_cast<double2*>(&As[mloc * Sh::LDA + NA * q]) = make_double2(sv.x * wq, dv.x * wq);
      }
    }
    __syncthreads();
    if (t + 1 < t1) prefetch(t + 1);
    mma_tile<Sh>(As, Bs, acc);
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
    const int64_t i = base + mma_row<Sh>(mt);
    if (i >= m) continue;
    double2* out = partial + ((int64_t)blockIdx.y * m + i) * ns;
#pragma unroll
    for (int nt = 0; nt < Sh::kNT; ++nt) {
      const int col = mma_col<Sh>(nt);
      if (CPLX) {
        if (col / 2 < ns) out[col / 2] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
      } else {
        if (col < ns) out[col] = make_double2(acc[mt][nt][0], 0.0);
        if (col + 1 < ns) out[col + 1] = make_double2(acc[mt][nt][1], 0.0);
      }
    }
  }
}

// theta[i,k] = mu_i * B(x_i, xs_k) + sum_s partial[s][i][k]
template <int PDE, int DIM, bool DERIV>
__global__ void dim_theta_reduce(int64_t m, int ns, int split, const double* __restrict__ tx,
                                 const double* __restrict__ tn, const double* __restrict__ xs,
                                 const double* __restrict__ mu, double k,
                                 const double2* __restrict__ partial, double2* __restrict__ theta) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= m * ns) return;
  const int64_t i = t / ns;
  const int kk = (int)(t % ns);
  // tn is only read by the ADL value kernel (derivative corrections)
  const double2 b = kernel_value<PDE, DERIV ? ADL : SL, DIM>(tx + DIM * i, tn ? tn + DIM * i : tx + DIM * i,
                                                             xs + DIM * kk, nullptr, k);
  const double mi = mu ? mu[i] : -0.5;
  double sr = mi * b.x, si = mi * b.y;
  for (int s = 0; s < split; ++s) {
    const double2 v = partial[(int64_t)s * m * ns + t];
    sr += v.x;
    si += v.y;
  }
  theta[t] = make_double2(sr, si);
}

// ---------------------------------------------------------------------------
// 4-5. per-element least squares.  Lane l owns row l of A = M^T (ns x 2NQ):
// A[l][a] = g0[e*nq+a][l], A[l][NQ+a] = g1[e*nq+a][l].  Householder vectors
// follow the LAPACK xLARFG convention (H = I - tau v v^H, v_k = 1, real beta).
// ---------------------------------------------------------------------------
template <bool CPLX, int NQ>
struct ElementLsq {
  using Sc = S<CPLX>;
  using T = typename Sc::T;
  static constexpr int NC = 2 * NQ;
  T A[NC];
  T tau[NC];
  int lane;
  bool row;

  __device__ __forceinline__ void factor(int64_t e, int ns, const double2* __restrict__ g0,
                                         const double2* __restrict__ g1) {
    lane = threadIdx.x & 31;
    row = lane < ns;
#pragma unroll
    for (int a = 0; a < NQ; ++a) {
      const int64_t j = e * NQ + a;
      A[a] = row ? Sc::from(g0[j * ns + lane]) : Sc::zero();
      A[NQ + a] = row ? Sc::from(g1[j * ns + lane]) : Sc::zero();
    }
#pragma unroll
    for (int kc = 0; kc < NC; ++kc) {
      // x = A[kc:, kc]; alpha = A[kc][kc]
      const T alpha = Sc::shfl(A[kc], kc);
      const double xn2 = warp_sum((row && lane > kc) ? Sc::abs2(A[kc]) : 0.0);
      if (xn2 == 0.0 && Sc::im(alpha) == 0.0) {
        tau[kc] = Sc::zero();
        continue;
      }
      const double nrm = sqrt(Sc::abs2(alpha) + xn2);
      const double beta = Sc::re(alpha) >= 0 ? -nrm : nrm;
      T tk;
      if (CPLX) {
        tk = Sc::from(make_double2((beta - Sc::re(alpha)) / beta, -Sc::im(alpha) / beta));
      } else {
        tk = Sc::from(make_double2((beta - Sc::re(alpha)) / beta, 0.0));
      }
      tau[kc] = tk;
      const T ab = Sc::sub(alpha, Sc::from(make_double2(beta, 0.0)));
      if (lane > kc) A[kc] = Sc::div(A[kc], ab);
      if (lane == kc) A[kc] = Sc::from(make_double2(beta, 0.0));
      // trailing columns: s = conj(tau) * (A[kc][j] + sum_{l>kc} conj(v_l) A[l][j])
#pragma unroll
      for (int j = kc + 1; j < NC; ++j) {
        T contrib = (row && lane > kc) ? Sc::cmul(A[kc], A[j]) : Sc::zero();
        if (lane == kc) contrib = A[j];
        const T s = Sc::cmul(tk, Sc::wsum(contrib));
        if (lane == kc) A[j] = Sc::sub(A[j], s);
        if (row && lane > kc) A[j] = Sc::sub(A[j], Sc::mul(s, A[kc]));
      }
    }
  }

  // Least-squares solution for one Theta row; W is the same in every lane.
  __device__ __forceinline__ void solve(const double2* __restrict__ theta_row, T* W) const {
    T b = row ? Sc::from(theta_row[lane]) : Sc::zero();
#pragma unroll
    for (int kc = 0; kc < NC; ++kc) {
      T contrib = (row && lane > kc) ? Sc::cmul(A[kc], b) : Sc::zero();
      if (lane == kc) contrib = b;
      const T s = Sc::cmul(tau[kc], Sc::wsum(contrib));
      if (lane == kc) b = Sc::sub(b, s);
      if (row && lane > kc) b = Sc::sub(b, Sc::mul(s, A[kc]));
    }
    // back substitution R W = (Q^H b)[0:NC]; lane c holds row c of R
#pragma unroll
    for (int c = NC - 1; c >= 0; --c) {
      T s = b;
#pragma unroll
      for (int j = c + 1; j < NC; ++j) s = Sc::sub(s, Sc::mul(A[j], W[j]));
      const T wc = Sc::div(s, A[c]);
      W[c] = Sc::shfl(wc, c);
    }
  }

  // dS = -W[NQ + a], dD = W[a] (bdim.jl:176-179) at CSR positions p0 + a
  __device__ __forceinline__ void store(const T* W, int64_t p0, double* __restrict__ dS,
                                        double* __restrict__ dD) const {
    if (lane >= NQ) return;
    T vS = Sc::zero(), vD = Sc::zero();
#pragma unroll
    for (int a = 0; a < NQ; ++a)
      if (a == lane) {
        vS = Sc::neg(W[NQ + a]);
        vD = W[a];
      }
    const int64_t p = p0 + lane;
    if (CPLX) {
      dS[2 * p] = Sc::re(vS);
      dS[2 * p + 1] = Sc::im(vS);
      dD[2 * p] = Sc::re(vD);
      dD[2 * p + 1] = Sc::im(vD);
    } else {
      dS[p] = Sc::re(vS);
      dD[p] = Sc::re(vD);
    }
  }
};

// target === source: each element solves for its own nq nodes; row i of the
// CSR holds columns e*NQ .. e*NQ+NQ-1 in order.
template <bool CPLX, int NQ>
__global__ void dim_lsq(int64_t nel, int ns, const double2* __restrict__ g0,
                        const double2* __restrict__ g1, const double2* __restrict__ theta,
                        double* __restrict__ dS, double* __restrict__ dD) {
  const int64_t e = blockIdx.x * (int64_t)(blockDim.x / 32) + threadIdx.x / 32;
  if (e >= nel) return;  // whole warp leaves together
  ElementLsq<CPLX, NQ> L;
  L.factor(e, ns, g0, g1);
  typename ElementLsq<CPLX, NQ>::T W[2 * NQ];
  for (int t = 0; t < NQ; ++t) {
    const int64_t i = e * NQ + t;
    L.solve(theta + i * ns, W);
    L.store(W, i * NQ, dS, dD);
  }
}

// target !== source: element e solves for its near targets etgt[etptr[e] ..
// etptr[e+1]) (rows of Theta), writing row tgt[j] of the CSR at rowptr.
template <bool CPLX, int NQ>
__global__ void dim_lsq_targets(int64_t nel, int ns, const double2* __restrict__ g0,
                                const double2* __restrict__ g1, const double2* __restrict__ theta,
                                const int64_t* __restrict__ etptr, const int64_t* __restrict__ etgt,
                                const int64_t* __restrict__ tgt, const int64_t* __restrict__ rowptr,
                                double* __restrict__ dS, double* __restrict__ dD) {
  const int64_t e = blockIdx.x * (int64_t)(blockDim.x / 32) + threadIdx.x / 32;
  if (e >= nel) return;
  const int64_t b0 = etptr[e], b1 = etptr[e + 1];
  if (b0 == b1) return;  // nothing near this element
  ElementLsq<CPLX, NQ> L;
  L.factor(e, ns, g0, g1);
  typename ElementLsq<CPLX, NQ>::T W[2 * NQ];
  for (int64_t b = b0; b < b1; ++b) {
    const int64_t j = etgt[b];
    L.solve(theta + j * ns, W);
    L.store(W, rowptr[tgt[j]], dS, dD);
  }
}

__global__ void block_pattern(int64_t n, int nq, int64_t* rowptr, int32_t* col) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > n) return;
  rowptr[i] = i * nq;
  if (i == n) return;
  const int64_t e = i / nq;
  for (int a = 0; a < nq; ++a) col[i * nq + a] = (int32_t)(e * nq + a);
}

// Nearest source node of each target (the KDTree nn of
// src/quadrature.jl:266-270, here exhaustive): squared distances are formed
// as ((dx*dx + dy*dy) + dz*dz) without contraction, ties go to the lowest
// index, so the choice is reproducible bit for bit on the host.
constexpr int kNearBlock = 256;
template <int DIM>
__global__ void __launch_bounds__(kNearBlock) nearest_node(int64_t m, const double* __restrict__ tx, int64_t n,
                                                          const double* __restrict__ x, int64_t* __restrict__ best_j,
                                                          double* __restrict__ best_d2) {
  __shared__ double sx[kNearBlock * DIM];
  const int64_t i = blockIdx.x * (int64_t)kNearBlock + threadIdx.x;
  const int64_t ii = min(i, m - 1);
  double xi[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) xi[c] = tx[DIM * ii + c];
  double bd = INFINITY;
  int64_t bj = -1;
  for (int64_t t0 = 0; t0 < n; t0 += kNearBlock) {
    __syncthreads();
    for (int q = threadIdx.x; q < kNearBlock * DIM; q += kNearBlock) {
      const int64_t j = t0 + q / DIM;
      sx[q] = j < n ? x[DIM * t0 + q] : 0.0;
    }
    __syncthreads();
    const int cnt = n - t0 < kNearBlock ? (int)(n - t0) : kNearBlock;
    for (int a = 0; a < cnt; ++a) {
      double d2 = 0.0;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const double dc = __dsub_rn(xi[c], sx[a * DIM + c]);
        d2 = c == 0 ? __dmul_rn(dc, dc) : __dadd_rn(d2, __dmul_rn(dc, dc));
      }
      if (d2 < bd) {
        bd = d2;
        bj = t0 + a;
      }
    }
  }
  if (i < m) {
    best_j[i] = bj;
    best_d2[i] = bd;
  }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
template <int NS, class F>
static bool ns_bucket(int ns, F&& f) {
  if (ns <= NS) {
    f(std::integral_constant<int, NS>());
    return true;
  }
  return false;
}

template <class F>
static void nq_dispatch(int nq, F&& f) {
  switch (nq) {
    case 1: return f(std::integral_constant<int, 1>());
    case 2: return f(std::integral_constant<int, 2>());
    case 3: return f(std::integral_constant<int, 3>());
    case 4: return f(std::integral_constant<int, 4>());
    case 5: return f(std::integral_constant<int, 5>());
    case 6: return f(std::integral_constant<int, 6>());
    case 7: return f(std::integral_constant<int, 7>());
    case 8: return f(std::integral_constant<int, 8>());
    case 9: return f(std::integral_constant<int, 9>());
    case 10: return f(std::integral_constant<int, 10>());
  }
  throw Error(INTI_E_UNSUPPORTED, "DIM correction supports 1..10 nodes per element");
}

// Steps 1-3 shared by both forms: monopole centres and traces on the source
// nodes, then Theta for m targets (coordinates tx, normals tn or NULL, green
// multipliers mu or NULL for -1/2, all on the device).
// Work arrays of one construction: the context's buffers, kept between
// constructions (hundreds of MB at N = 2e5, whose cudaMalloc/cudaFree per
// call would dominate the host time and synchronise the device).
struct DimWork {
  int ns = 0;
  DevBuf &d_xs, &g0, &g1, &theta, &part, &mu;
  explicit DimWork(inti_ctx* c)
      : d_xs(c->dimwork.d_xs), g0(c->dimwork.g0), g1(c->dimwork.g1), theta(c->dimwork.theta),
        part(c->dimwork.part), mu(c->dimwork.mu) {}
};

static void dim_source_setup(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* q,
                             DimWork& wk) {
  if (!q) throw Error(INTI_E_ARG, "quadrature is NULL");
  if (q->ctx != ctx) throw Error(INTI_E_STATE, "quadrature belongs to another context");
  if (!q->has_normals) throw Error(INTI_E_ARG, "DIM needs a source quadrature with normals");
  if (q->nq <= 0) throw Error(INTI_E_ARG, "DIM needs the element structure (nq > 0)");
  if (pde != INTI_LAPLACE && pde != INTI_HELMHOLTZ) throw Error(INTI_E_ARG, "unknown pde");
  if (pde == INTI_HELMHOLTZ && q->dim != 3) throw Error(INTI_E_UNSUPPORTED, "Helmholtz is 3D only");
  if (pde == INTI_HELMHOLTZ && k_im != 0.0) throw Error(INTI_E_UNSUPPORTED, "complex wavenumbers are not implemented");
  const int dim = q->dim;
  const int64_t n = q->n;
  const int nq = q->nq;
  wk.ns = (int)std::ceil(3.0 * nq);  // bdim.jl:79-80
  const int ns = wk.ns;
  if (ns > 32) throw Error(INTI_E_UNSUPPORTED, "ns > 32");
  // 1. monopole centres (bdim.jl:82-92; utils.jl:142-171)
  double lc[3] = {INFINITY, INFINITY, INFINITY}, hc[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t j = 0; j < n; ++j)
    for (int c = 0; c < dim; ++c) {
      lc[c] = std::min(lc[c], q->h_coords[dim * j + c]);
      hc[c] = std::max(hc[c], q->h_coords[dim * j + c]);
    }
  double xc[3] = {0, 0, 0}, diag2 = 0.0;
  for (int c = 0; c < dim; ++c) {
    xc[c] = (lc[c] + hc[c]) / 2;
    diag2 += (hc[c] - lc[c]) * (hc[c] - lc[c]);
  }
  const double R = 1.5 * std::sqrt(diag2) / 2;
  std::vector<double> xs((size_t)ns * dim);
  if (dim == 2) {
    for (int i = 0; i < ns; ++i) {
      xs[2 * i] = R * std::cos(2 * kPi * i / ns) + xc[0];
      xs[2 * i + 1] = R * std::sin(2 * kPi * i / ns) + xc[1];
    }
  } else {
    const double phi = kPi * (3 - std::sqrt(5.0));
    for (int i = 1; i <= ns; ++i) {
      const double ytmp = 1 - ((double)(i - 1) / (double)(ns - 1)) * 2;
      const double radius = std::sqrt(1 - ytmp * ytmp);
      const double theta = phi * i;
      xs[3 * (i - 1)] = std::cos(theta) * radius * R + xc[0];
      xs[3 * (i - 1) + 1] = ytmp * R + xc[1];
      xs[3 * (i - 1) + 2] = std::sin(theta) * radius * R + xc[2];
    }
  }
  wk.d_xs.ensure(sizeof(double) * xs.size());
  INTI_CUDA(cudaMemcpyAsync(wk.d_xs.p, xs.data(), sizeof(double) * xs.size(), cudaMemcpyHostToDevice, ctx->stream));
  // 2. traces (bdim.jl:94-103)
  wk.g0.ensure(sizeof(double2) * n * ns);
  wk.g1.ensure(sizeof(double2) * n * ns);
  const int64_t tot = n * ns;
  auto go = [&](auto pde_c, auto dim_c) {
    constexpr int P = decltype(pde_c)::value;
    constexpr int D = decltype(dim_c)::value;
    dim_traces<P, D><<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(
        n, ns, q->coords.as<double>(), q->normals.as<double>(), wk.d_xs.as<double>(), k_re, wk.g0.as<double2>(),
        wk.g1.as<double2>());
    ctx->launches++;
  };
  if (pde == INTI_LAPLACE && dim == 2)
    go(std::integral_constant<int, LAPLACE>(), std::integral_constant<int, 2>());
  else if (pde == INTI_LAPLACE)
    go(std::integral_constant<int, LAPLACE>(), std::integral_constant<int, 3>());
  else
    go(std::integral_constant<int, HELMHOLTZ>(), std::integral_constant<int, 3>());
  INTI_CUDA(cudaGetLastError());
}

// 3. Theta = mu*B(x) + S*g1 - D*g0 over all source nodes (bdim.jl:104-118)
static void dim_theta_run(inti_ctx* ctx, int pde, double k_re, const inti_quad* q, int derivative, int64_t m,
                          const double* tx, const double* tn, const double* mu, DimWork& wk) {
  const int dim = q->dim;
  const int64_t n = q->n;
  const int ns = wk.ns;
  wk.theta.ensure(sizeof(double2) * std::max<int64_t>(m, 1) * ns);
  if (m == 0) return;
  const double* X = q->coords.as<double>();
  const double* NR = q->normals.as<double>();
  const double* W = q->weights.as<double>();
  auto run = [&](auto pde_c, auto dim_c) {
    constexpr int P = decltype(pde_c)::value;
    constexpr int D = decltype(dim_c)::value;
    const int64_t tot = m * ns;
    if constexpr (D == 3) {
      // FP64 MMA form; split over sources for >= 8 waves of 2 CTAs per SM
      auto mma = [&](auto wide_c, auto deriv_c) {
        constexpr bool WIDE = decltype(wide_c)::value;
        constexpr bool DV = decltype(deriv_c)::value;
        using TM = ThetaMma<P, WIDE>;
        const int64_t blocks = (m + TM::Sh::MT - 1) / TM::Sh::MT;
        const int64_t ntile = (n + TM::J - 1) / TM::J;
        const int64_t want = (int64_t)ctx->num_sms * 16;
        int split = (int)std::max<int64_t>(1, std::min<int64_t>({ntile, (want + blocks - 1) / blocks, 64}));
        const int tps = (int)((ntile + split - 1) / split);
        split = (int)((ntile + tps - 1) / tps);
        wk.part.ensure(sizeof(double2) * (size_t)split * m * ns);
        constexpr size_t smem = theta_mma_smem<P, WIDE>();
        auto* kern = &dim_theta_mma<P, WIDE, DV>;
        static std::once_flag once;
        std::call_once(once, [kern] {
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        });
        ProfScope pd(ctx, "dim");
        kern<<<dim3((unsigned)blocks, (unsigned)split), kMmaThreads, smem, ctx->stream>>>(
            m, n, ns, tx, tn, X, NR, W, wk.g0.as<double2>(), wk.g1.as<double2>(), k_re,
            k_re * kExpiTable / (2 * kPi), 2 * kPi / kExpiTable, P == HELMHOLTZ ? expi_table_f64(ctx) : nullptr, tps,
            wk.part.as<double2>());
        ctx->launches++;
        dim_theta_reduce<P, D, DV><<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(
            m, ns, split, tx, tn, wk.d_xs.as<double>(), mu, k_re, wk.part.as<double2>(), wk.theta.as<double2>());
        ctx->launches++;
      };
      auto mma_d = [&](auto wide_c) {
        if (derivative)
          mma(wide_c, std::true_type());
        else
          mma(wide_c, std::false_type());
      };
      if (ns <= ThetaMma<P, false>::kMaxNs) {
        mma_d(std::false_type());
        return;
      }
      if constexpr (P == HELMHOLTZ) {
        if (ns <= ThetaMma<P, true>::kMaxNs) {
          mma_d(std::true_type());
          return;
        }
      }
    }
    // split over sources so the grid covers the device
    const int64_t blocks = (m + kThetaBlock - 1) / kThetaBlock;
    const int64_t ntile = (n + kThetaTile - 1) / kThetaTile;
    const int64_t want = (int64_t)ctx->num_sms * 6;
    int split = (int)std::max<int64_t>(1, std::min<int64_t>({ntile, (want + blocks - 1) / blocks, 64}));
    const int tps = (int)((ntile + split - 1) / split);
    split = (int)((ntile + tps - 1) / tps);
    wk.part.ensure(sizeof(double2) * (size_t)split * m * ns);
    auto theta_go = [&](auto nsb, auto deriv_c) {
      constexpr int NSB = decltype(nsb)::value;
      constexpr bool DV = decltype(deriv_c)::value;
      dim3 grid((unsigned)blocks, (unsigned)split);
      ProfScope pd(ctx, "dim");
      dim_theta<P, D, DV, NSB><<<grid, kThetaBlock, 0, ctx->stream>>>(
          m, n, ns, tx, tn, X, NR, W, wk.g0.as<double2>(), wk.g1.as<double2>(), k_re,
          k_re * kExpiTable / (2 * kPi), 2 * kPi / kExpiTable, P == HELMHOLTZ ? expi_table_f64(ctx) : nullptr, tps,
          wk.part.as<double2>());
      ctx->launches++;
      dim_theta_reduce<P, D, DV><<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(
          m, ns, split, tx, tn, wk.d_xs.as<double>(), mu, k_re, wk.part.as<double2>(), wk.theta.as<double2>());
      ctx->launches++;
    };
    auto by_ns = [&](auto deriv_c) {
      if (ns_bucket<8>(ns, [&](auto b) { theta_go(b, deriv_c); })) return;
      if (ns_bucket<16>(ns, [&](auto b) { theta_go(b, deriv_c); })) return;
      if (ns_bucket<24>(ns, [&](auto b) { theta_go(b, deriv_c); })) return;
      ns_bucket<32>(ns, [&](auto b) { theta_go(b, deriv_c); });
    };
    if (derivative)
      by_ns(std::true_type());
    else
      by_ns(std::false_type());
  };
  if (pde == INTI_LAPLACE && dim == 2)
    run(std::integral_constant<int, LAPLACE>(), std::integral_constant<int, 2>());
  else if (pde == INTI_LAPLACE)
    run(std::integral_constant<int, LAPLACE>(), std::integral_constant<int, 3>());
  else
    run(std::integral_constant<int, HELMHOLTZ>(), std::integral_constant<int, 3>());
  INTI_CUDA(cudaGetLastError());
}

static std::unique_ptr<inti_csr> new_csr(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz, bool cplx) {
  std::unique_ptr<inti_csr> c(new inti_csr());
  c->ctx = ctx;
  c->m = m;
  c->n = n;
  c->nnz = nnz;
  c->dtype = cplx ? INTI_C128 : INTI_F64;
  c->rowptr.ensure(sizeof(int64_t) * (m + 1));
  c->col.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1));
  c->val.ensure(sizeof(double) * (cplx ? 2 : 1) * std::max<int64_t>(nnz, 1));
  return c;
}

void dim_correction(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* q,
                    int derivative, const double* green_multiplier, inti_csr** dS,
                    inti_csr** dD) {
  DimWork wk(ctx);
  dim_source_setup(ctx, pde, k_re, k_im, q, wk);
  const int64_t n = q->n;
  const int nq = q->nq;
  const int64_t nel = n / nq;
  const int ns = wk.ns;
  const bool cplx = pde == INTI_HELMHOLTZ;
  DevBuf& d_mu = wk.mu;
  if (green_multiplier) {
    for (int64_t i = 0; i < n; ++i)
      if (!std::isfinite(green_multiplier[i])) throw Error(INTI_E_NONFINITE, "green_multiplier contains NaN/Inf");
    d_mu.ensure(sizeof(double) * n);
    INTI_CUDA(cudaMemcpyAsync(d_mu.p, green_multiplier, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  dim_theta_run(ctx, pde, k_re, q, derivative, n, q->coords.as<double>(), q->normals.as<double>(),
                green_multiplier ? d_mu.as<double>() : nullptr, wk);
  // output CSR handles with the element-block pattern
  const int64_t nnz = n * nq;
  auto cS = new_csr(ctx, n, n, nnz, cplx), cD = new_csr(ctx, n, n, nnz, cplx);
  block_pattern<<<(unsigned)((n + 1 + 255) / 256), 256, 0, ctx->stream>>>(n, nq, cS->rowptr.as<int64_t>(), cS->col.as<int32_t>());
  ctx->launches++;
  INTI_CUDA(cudaMemcpyAsync(cD->rowptr.p, cS->rowptr.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToDevice, ctx->stream));
  INTI_CUDA(cudaMemcpyAsync(cD->col.p, cS->col.p, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, ctx->stream));
  nq_dispatch(nq, [&](auto nqc) {
    constexpr int NQ = decltype(nqc)::value;
    const int warps = 4;
    const unsigned grid = (unsigned)((nel + warps - 1) / warps);
    if (cplx)
      dim_lsq<true, NQ><<<grid, 32 * warps, 0, ctx->stream>>>(nel, ns, wk.g0.as<double2>(), wk.g1.as<double2>(),
                                                              wk.theta.as<double2>(), cS->val.as<double>(), cD->val.as<double>());
    else
      dim_lsq<false, NQ><<<grid, 32 * warps, 0, ctx->stream>>>(nel, ns, wk.g0.as<double2>(), wk.g1.as<double2>(),
                                                               wk.theta.as<double2>(), cS->val.as<double>(), cD->val.as<double>());
    ctx->launches++;
  });
  INTI_CUDA(cudaGetLastError());
  sync_and_check(ctx);
  *dS = cS.release();
  *dD = cD.release();
}

void dim_correction_targets(inti_ctx* ctx, int pde, double k_re, double k_im, const inti_quad* target,
                            const inti_quad* q, int derivative, const double* green_multiplier, double maxdist,
                            inti_csr** dS, inti_csr** dD) {
  if (!target) throw Error(INTI_E_ARG, "target is NULL");
  if (target->ctx != ctx) throw Error(INTI_E_STATE, "target belongs to another context");
  if (!green_multiplier) throw Error(INTI_E_ARG, "off-surface targets need a green multiplier per target");
  if (std::isnan(maxdist) || maxdist < 0) throw Error(INTI_E_ARG, "maxdist must be >= 0");
  DimWork wk(ctx);
  dim_source_setup(ctx, pde, k_re, k_im, q, wk);
  if (target->dim != q->dim) throw Error(INTI_E_SHAPE, "target and source dimensions differ");
  if (derivative && !target->has_normals) throw Error(INTI_E_ARG, "derivative corrections need target normals");
  const int dim = q->dim;
  const int64_t m = target->n, n = q->n;
  const int nq = q->nq;
  const int64_t nel = n / nq;
  const int ns = wk.ns;
  const bool cplx = pde == INTI_HELMHOLTZ;
  for (int64_t i = 0; i < m; ++i)
    if (!std::isfinite(green_multiplier[i])) throw Error(INTI_E_NONFINITE, "green_multiplier contains NaN/Inf");

  // near lists (quadrature.jl:264-286): nearest source node of each target
  std::vector<int64_t> best(m);
  std::vector<double> bd2(m);
  if (m > 0) {
    DevBuf d_best, d_bd2;
    d_best.ensure(sizeof(int64_t) * m);
    d_bd2.ensure(sizeof(double) * m);
    auto go = [&](auto dim_c) {
      constexpr int D = decltype(dim_c)::value;
      nearest_node<D><<<(unsigned)((m + kNearBlock - 1) / kNearBlock), kNearBlock, 0, ctx->stream>>>(
          m, target->coords.as<double>(), n, q->coords.as<double>(), d_best.as<int64_t>(), d_bd2.as<double>());
    };
    if (dim == 2)
      go(std::integral_constant<int, 2>());
    else
      go(std::integral_constant<int, 3>());
    ctx->launches++;
    INTI_CUDA(cudaGetLastError());
    INTI_CUDA(cudaMemcpyAsync(best.data(), d_best.p, sizeof(int64_t) * m, cudaMemcpyDeviceToHost, ctx->stream));
    INTI_CUDA(cudaMemcpyAsync(bd2.data(), d_bd2.p, sizeof(double) * m, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
  }
  // near targets (compact order j), element lists, output row pointers
  std::vector<int64_t> tgt, elem_of, etptr(nel + 1, 0), rowptr(m + 1, 0);
  for (int64_t i = 0; i < m; ++i) {
    const bool near = best[i] >= 0 && !(std::sqrt(bd2[i]) > maxdist);
    rowptr[i + 1] = rowptr[i] + (near ? nq : 0);
    if (near) {
      tgt.push_back(i);
      elem_of.push_back(best[i] / nq);
      ++etptr[best[i] / nq + 1];
    }
  }
  const int64_t mn = (int64_t)tgt.size();
  for (int64_t e = 0; e < nel; ++e) etptr[e + 1] += etptr[e];
  std::vector<int64_t> etgt(std::max<int64_t>(mn, 1)), fill(etptr.begin(), etptr.end() - 1);
  for (int64_t j = 0; j < mn; ++j) etgt[fill[elem_of[j]]++] = j;
  // gathered near-target data for Theta
  std::vector<double> htx((size_t)std::max<int64_t>(mn, 1) * dim), htn, hmu(std::max<int64_t>(mn, 1));
  if (derivative) htn.resize(htx.size());
  for (int64_t j = 0; j < mn; ++j) {
    const int64_t i = tgt[j];
    for (int c = 0; c < dim; ++c) {
      htx[dim * j + c] = target->h_coords[dim * i + c];
      if (derivative) htn[dim * j + c] = target->h_normals[dim * i + c];
    }
    hmu[j] = green_multiplier[i];
  }
  DevBuf d_tx, d_tn, d_mu, d_etptr, d_etgt, d_tgt, d_rowptr;
  auto up = [&](DevBuf& b, const void* h, size_t bytes) {
    b.ensure(std::max<size_t>(bytes, 16));
    if (bytes) INTI_CUDA(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, ctx->stream));
  };
  up(d_tx, htx.data(), sizeof(double) * dim * mn);
  if (derivative) up(d_tn, htn.data(), sizeof(double) * dim * mn);
  up(d_mu, hmu.data(), sizeof(double) * mn);
  up(d_etptr, etptr.data(), sizeof(int64_t) * (nel + 1));
  up(d_etgt, etgt.data(), sizeof(int64_t) * mn);
  up(d_tgt, tgt.data(), sizeof(int64_t) * mn);
  dim_theta_run(ctx, pde, k_re, q, derivative, mn, d_tx.as<double>(), derivative ? d_tn.as<double>() : nullptr,
                d_mu.as<double>(), wk);
  // output CSR: row i holds the nq nodes of its element (sorted), or nothing
  const int64_t nnz = mn * nq;
  std::vector<int32_t> col((size_t)std::max<int64_t>(nnz, 1));
  for (int64_t j = 0; j < mn; ++j)
    for (int a = 0; a < nq; ++a) col[(size_t)j * nq + a] = (int32_t)(elem_of[j] * nq + a);
  auto cS = new_csr(ctx, m, n, nnz, cplx), cD = new_csr(ctx, m, n, nnz, cplx);
  for (auto* c : {cS.get(), cD.get()}) {
    INTI_CUDA(cudaMemcpyAsync(c->rowptr.p, rowptr.data(), sizeof(int64_t) * (m + 1), cudaMemcpyHostToDevice, ctx->stream));
    if (nnz) INTI_CUDA(cudaMemcpyAsync(c->col.p, col.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, ctx->stream));
  }
  if (mn > 0)
    nq_dispatch(nq, [&](auto nqc) {
      constexpr int NQ = decltype(nqc)::value;
      const int warps = 4;
      const unsigned grid = (unsigned)((nel + warps - 1) / warps);
      auto go = [&](auto cplx_c) {
        constexpr bool CP = decltype(cplx_c)::value;
        dim_lsq_targets<CP, NQ><<<grid, 32 * warps, 0, ctx->stream>>>(
            nel, ns, wk.g0.as<double2>(), wk.g1.as<double2>(), wk.theta.as<double2>(), d_etptr.as<int64_t>(),
            d_etgt.as<int64_t>(), d_tgt.as<int64_t>(), cS->rowptr.as<int64_t>(), cS->val.as<double>(),
            cD->val.as<double>());
      };
      if (cplx)
        go(std::true_type());
      else
        go(std::false_type());
      ctx->launches++;
    });
  INTI_CUDA(cudaGetLastError());
  sync_and_check(ctx);
  *dS = cS.release();
  *dD = cD.release();
}

}  // namespace inti
