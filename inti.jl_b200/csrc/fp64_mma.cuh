// FP64 matrix-multiply-accumulate on the tensor path for the multi-RHS pair
// products (batch FP64 apply, DIM Theta).
//
// The pair products Y(i, c) = sum_j K(x_i, y_j) X(j, c) for many columns c
// split into two phases per tile of J sources:
//   1. CUDA cores evaluate K(x_i, y_j) once per pair (the expensive,
//      transcendental part) into a shared-memory tile A (MT x K, K = J*NA
//      real slots per source: NA = 1 real, 2 for (Re, Im), ...);
//   2. each warp multiplies its 32 rows of A with the staged right-hand-side
//      rows B (K x NCOL) using mma.sync m8n8k4 FP64 into register
//      accumulators.
// tcgen05 has no FP64 kind, so the FP64 MMA is the warp-level mma.sync.  On
// the B200 it runs on the same FP64 datapath as DFMA (both ~36 TFLOP/s,
// together no more); what it removes is the per-FMA shared-memory operand
// load and instruction issue of a CUDA-core inner product, and the repeated
// kernel evaluation of column chunks.
//
// Fragment layouts of mma.m8n8k4 .f64 (PTX ISA): with g = lane >> 2 and
// t = lane & 3, A holds A[g][t], B holds B[t][g], and C/D hold C[g][2t] and
// C[g][2t + 1].
#pragma once

#include <cuda_runtime.h>

namespace inti {

constexpr int kMmaThreads = 256;  // 8 warps

__device__ __forceinline__ void dmma_884(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// WM x WN warps; each warp owns 32 rows x (8 * NT) columns.  Shared-memory
// layouts, chosen so that both the tile stores and the fragment loads run at
// the minimum number of wavefronts:
//  * A row pitch = 2 doubles mod 16: the fragment's 8 rows x 4 columns fall
//    on distinct bank pairs except pairs two slots apart (2 wavefronts), and
//    the phase-1 stores of 32 consecutive rows (one column, 8 or 16 bytes)
//    spread over 8 distinct 16-byte slots;
//  * B row pitch = 8 doubles mod 16 (rows t and t+1 of a fragment on opposite
//    halves of the banks), and column n of row k stored at
//    n ^ (SWZ * ((k >> 1) & 7)): the staging stores of consecutive sources
//    (rows 2q or q, one column) land on distinct slots instead of one, while
//    each fragment row still reads one permuted aligned 8-column block.
//    SWZ = 2 keeps (Re, Im) column pairs adjacent, SWZ = 1 for real columns.
template <int WM, int WN, int NT, int K, int SWZ>
struct MmaShape {
  static_assert(WM * WN == kMmaThreads / 32, "8 warps");
  static_assert(K % 4 == 0, "K is a multiple of the MMA depth");
  static_assert(SWZ == 1 || SWZ == 2, "swizzle step");
  static constexpr int kWM = WM, kWN = WN, kNT = NT, kK = K, kSWZ = SWZ;
  static constexpr int MT = 32 * WM;
  static constexpr int NCOL = 8 * NT * WN;
  static_assert(NCOL % 16 == 0, "the swizzle permutes within 16-column blocks");
  static constexpr int LDA = K + ((18 - K % 16) % 16);
  static constexpr int LDB = NCOL + ((24 - NCOL % 16) % 16);
  static __device__ __forceinline__ int bcol(int k, int n) { return n ^ (SWZ * ((k >> 1) & 7)); }
};

// acc[mt][nt] += A(rows of this warp, 0:K) * B(0:K, columns of this warp)
template <class Sh>
__device__ __forceinline__ void mma_tile(const double* __restrict__ As, const double* __restrict__ Bs,
                                         double (&acc)[4][Sh::kNT][2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp % Sh::kWM, wn = warp / Sh::kWM;
  const int t = lane & 3;
  const double* a = As + (wm * 32 + (lane >> 2)) * Sh::LDA + t;
  const double* b = Bs + t * Sh::LDB;
  const int n0 = wn * Sh::kNT * 8 + (lane >> 2);
#pragma unroll 2
  for (int ks = 0; ks < Sh::kK; ks += 4) {
    double af[4], bf[Sh::kNT];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) af[mt] = a[mt * 8 * Sh::LDA + ks];
#pragma unroll
    for (int nt = 0; nt < Sh::kNT; ++nt) bf[nt] = b[ks * Sh::LDB + Sh::bcol(ks + t, n0 + nt * 8)];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < Sh::kNT; ++nt) dmma_884(acc[mt][nt], af[mt], bf[nt]);
  }
}

// Row and first column of accumulator element acc[mt][nt][e] of this thread.
template <class Sh>
__device__ __forceinline__ int mma_row(int mt) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  return (warp % Sh::kWM) * 32 + mt * 8 + (lane >> 2);
}
template <class Sh>
__device__ __forceinline__ int mma_col(int nt) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  return ((warp / Sh::kWM) * Sh::kNT + nt) * 8 + 2 * (lane & 3);
}

}  // namespace inti
