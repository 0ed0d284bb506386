// Tensor-core (tcgen05, TF32 in / FP32 accumulate) form of the batched
// multi-right-hand-side Helmholtz product Y = K X over many surfaces.
//
// The complex product is a real GEMM: with A[i][2j] = Re K_ij,
// A[i][2j+1] = Im K_ij (targets x 2*sources) and, for right-hand side r,
// B[2j][r] = Re x_jr, B[2j+1][r] = -Im x_jr, B[2j][64+r] = Im x_jr,
// B[2j+1][64+r] = Re x_jr (x already multiplied by the weight w_j), the
// columns 0..63 of A*B are Re Y and 64..127 are Im Y.
//
// One persistent CTA per SM (18 warps) takes work items (surface, block of
// 256 targets) from an atomic counter, largest surfaces first.  Per stage of
// 32 sources:
//   * a producer warp copies the source records (FP32 coordinates/normals)
//     and the packed density block B of later stages into shared-memory
//     rings with the TMA bulk engine (cp.async.bulk) completing on mbarriers;
//   * 16 generator warps evaluate K for their target rows and the 32 sources
//     on the CUDA cores (FP32; e^{ikd} from the MUFU sine/cosine), round to
//     TF32 and store them with tcgen05.st straight into tensor memory, the A
//     operand of the MMAs (lanes = rows, one 32-bit column per K element);
//   * an MMA warp issues 2 x 8 tcgen05.mma (M = 128, N = 128, K = 8; A from
//     tensor memory, B from shared memory in the canonical K-major
//     no-swizzle layout: 8-row x 16-byte core matrices, LBO = 128 B between
//     K chunks, SBO = 2048 B between row groups) into two TMEM accumulators
//     (128 lanes x 128 FP32 columns each) and commits them to the mbarrier
//     that frees the A and B buffers.
// Generation of stage t+1 overlaps the MMAs of stage t; the roles meet only
// at mbarriers, with one CTA barrier per item.  At the end of an item each
// generator warp reads its lane quarter of the accumulators with tcgen05.ld
// and writes alpha*Y/(4 pi) + beta*Y in FP64.
//
// Every wait is bounded.  On a timeout the CTA records the error, drains its
// own copies and MMAs (bounded), frees its TMEM and leaves.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "batch.h"
#include "common.h"
#include "device_common.cuh"
#include "internal.h"

namespace inti {

constexpr int TC_GEN_WARPS = 16;                    // two generator threads per target row
constexpr int TC_THREADS = 32 * (TC_GEN_WARPS + 2);  // + MMA-issue and copy warps
constexpr int TC_ROWS = 256;             // targets per item (2 accumulators x 128)
constexpr int TC_R = 64;                 // complex right-hand sides per pass
constexpr int TC_N = 2 * TC_R;           // real accumulator columns
constexpr int TC_J = 32;                 // sources per stage
constexpr int TC_K = 2 * TC_J;           // K elements per stage
constexpr int TC_B_BYTES = TC_N * TC_K * 4;          // 32 KB
// every value twice (x x y y | z z nx nx | ny ny nz nz | pad): each 16-byte
// shared load gives the generator two ready operand pairs for its two rows
constexpr int TC_S_FLOATS = 16;
constexpr int TC_S_BYTES = TC_J * TC_S_FLOATS * 4;   // 2 KB
// dynamic shared memory layout (bytes)
// Ring depths: a bulk copy from L2 takes ~1500 cycles to land, longer than
// a stage's MMAs, so densities are fetched TC_NB - 1 stages and source
// records TC_NS - 1 stages ahead of use.
constexpr int TC_NB = 4;
constexpr int TC_NS = 8;
constexpr int TC_OFF_B = 0;                                   // TC_NB stages x 32 KB
constexpr int TC_OFF_S = TC_OFF_B + TC_NB * TC_B_BYTES;       // TC_NS stages x 1 KB
constexpr int TC_SMEM = TC_OFF_S + TC_NS * TC_S_BYTES;
// tensor memory (512 columns x 128 lanes x 32 bit): accumulators in columns
// 0..255 (128 each), then the A tiles, TC_K columns per accumulator and stage
constexpr uint32_t TC_TMEM_COLS = 512;
constexpr uint32_t TC_TMEM_A = 2 * TC_N;
__host__ __device__ constexpr uint32_t tc_a_col(uint32_t stage_buf, int acc) {
  return TC_TMEM_A + (2 * stage_buf + (uint32_t)acc) * TC_K;
}
static_assert(TC_TMEM_A + 4 * TC_K <= TC_TMEM_COLS, "A tiles exceed tensor memory");
// instruction descriptor: F32 accumulate, TF32 A and B, both K-major, N = 128, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                              ((uint32_t)(128 >> 4) << 24);

// K-major no-swizzle canonical offset of element (row, k) in a 128 x 64 shared-memory tile
__host__ __device__ constexpr uint32_t tc_kmajor_off(int row, int k) {
  return (uint32_t)((row >> 3) * 2048 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;    // leading byte offset: next K chunk
  d |= (uint64_t)((2048 >> 4) & 0x3FFF) << 32;   // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                        // descriptor version (sm_100)
  return d;                                      // base offset 0, no swizzle
}

__device__ __forceinline__ uint32_t to_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return r;
}

// Round-half-away to TF32 for the tensor core's own reads: adding half a TF32
// unit in the last place (bit 12) to the FP32 pattern makes the 19 bits the
// MMA reads the rounded value (one integer add; cvt.rna costs several
// instructions).  Finite inputs only.
__device__ __forceinline__ uint32_t tf32_bits(float v) { return __float_as_uint(v) + 0x1000u; }

// D (tensor memory) += A (tensor memory: lanes = rows, 8 columns = K) x B (shared memory descriptor)
__device__ __forceinline__ void tc_mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// The 8 MMAs (K = 8 each) of one accumulator and stage in one block: A
// columns advance by 8, the B descriptor's start address by 256 bytes (16 in
// its address field).  Only the first MMA of an item overwrites D.
__device__ __forceinline__ void tc_mma8_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t accumulate) {
#define TC_MMA_NEXT                                     \
  "add.u32 a, a, 8;\n\tadd.s64 b, b, 16;\n\t"          \
  "tcgen05.mma.cta_group::1.kind::tf32 [%0], [a], b, %3, q;\n\t"
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t.reg .b64 b;\n\t.reg .b32 a;\n\t"
      "setp.ne.b32 p, %4, 0;\n\tsetp.eq.b32 q, 0, 0;\n\t"
      "mov.b32 a, %1;\n\tmov.b64 b, %2;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [a], b, %3, p;\n\t" TC_MMA_NEXT TC_MMA_NEXT TC_MMA_NEXT TC_MMA_NEXT
          TC_MMA_NEXT TC_MMA_NEXT TC_MMA_NEXT "}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(TC_IDESC), "r"(accumulate));
#undef TC_MMA_NEXT
}
static_assert(TC_K == 64, "tc_mma8_ts issues exactly 8 K-steps of 8");

// True in exactly one lane of a converged warp.
__device__ __forceinline__ bool elect_one() {
  uint32_t e;
  asm volatile("{\n\t.reg .pred P;\n\telect.sync _|P, 0xffffffff;\n\tselp.b32 %0, 1, 0, P;\n\t}" : "=r"(e));
  return e != 0;
}

// 8 consecutive 32-bit columns of this thread's tensor-memory lane
__device__ __forceinline__ void tc_st8(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
               "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}
__device__ __forceinline__ void tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

struct TcArgs {
  const int64_t* off;        // surface node offsets
  const int64_t* toff;       // surface offsets in source tiles
  const int32_t* item_surf;  // items: surface, 256-target block
  const int32_t* item_block;
  int nitems;
  int ncolgroups;            // passes of 64 right-hand sides
  const float* src;          // packed source records, TC_J per tile
  const uint32_t* bpack;     // packed density blocks, per (column group, tile)
  int64_t ntiles;            // tiles per column group
  const double* coords;      // FP64 targets
  double* y;
  int64_t ldy;
  int nrhs;
  float k;
  float c1r, c1i, c2r, c2i;
  int kind;
  double ar, ai, br, bi;
  bool beta_zero;
  int* counter;
  int* err;
};

// Per-launch constants of the kernel values.
struct TcConst {
  float k, c1r, c1i, c2r, c2i, kc1r, kc1i;
};

// e^{i x} from the hardware sine/cosine approximations (MUFU).  Their
// absolute error (~1e-6 for the |k d| of a surface) is three orders below the
// TF32 rounding (2^-11) the values get next.
__device__ __forceinline__ void sincos_mufu(float x, float& s, float& c) {
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(x));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(x));
}

// Kernel variant of the combined field with c1 = 1 and c2 = i*eta (the
// Brakhage-Werner form D - i eta S), chosen on the host.
constexpr int CFI = 5;

// K(x, y) for the Helmholtz kernels (without 1/(4 pi)), FP32, with
// u = (r.n)/d, P = (r.n)/d^2 and Q = (r.n)/d^3:
//   SL:  e^{ikd}/d
//   DL:  e^{ikd} (1/d - ik) (r.n)/d^2          = e^{ikd} (Q - i k P)
//   CF:  e^{ikd} (c2/d + c1 (Q - i k P))
//   CFI: e^{ikd} (Q + i (eta - k u)/d)         (c1 = 1, c2 = i eta)
template <int KIND>
__device__ __forceinline__ float2 tc_kernel(const float* x, const float4 s0, const float2 s1, const TcConst& c) {
  const float r0 = x[0] - s0.x, r1 = x[1] - s0.y, r2 = x[2] - s0.z;
  const float d2 = fmaf(r2, r2, fmaf(r1, r1, r0 * r0));
  const float ri = d2 > 1.0e-28f ? rsqrt_approx_f32(d2) : 0.0f;
  float sn, cs;
  sincos_mufu(c.k * (d2 * ri), sn, cs);
  if (KIND == SL) return make_float2(cs * ri, sn * ri);
  const float rn = fmaf(r2, s1.y, fmaf(r1, s1.x, r0 * s0.w));
  const float u = rn * ri;
  float br, bi;
  if (KIND == CFI) {
    br = u * (ri * ri);
    bi = ri * fmaf(-c.k, u, c.c2i);
  } else {
    const float P = u * ri;
    const float Q = P * ri;
    if (KIND == DL) {
      br = Q;
      bi = -c.k * P;
    } else {
      br = fmaf(c.c2r, ri, fmaf(c.c1r, Q, c.kc1i * P));
      bi = fmaf(c.c2i, ri, fmaf(c.c1i, Q, -c.kc1r * P));
    }
  }
  return make_float2(fmaf(cs, br, -sn * bi), fmaf(cs, bi, sn * br));
}

// tc_kernel for the two target rows of a generator thread at once: the
// arithmetic runs on the paired FP32 instructions of sm_100 (two lanes per
// issue slot); the reciprocal square root, the sine and the cosine stay per
// lane.  Each lane performs tc_kernel's operations in the same order, so the
// values are the same bit for bit.
template <int KIND>
__device__ __forceinline__ void tc_kernel_x2(const float2 (&x)[3], const float4 sa, const float4 sb,
                                             const float4 sc, const TcConst& c, float2& k0, float2& k1) {
  // sa = (x x y y), sb = (z z nx nx), sc = (ny ny nz nz) of the source
  const float2 m1 = make_float2(-1.f, -1.f);
  const float2 r0 = __ffma2_rn(make_float2(sa.x, sa.y), m1, x[0]);  // x - s, one rounding
  const float2 r1 = __ffma2_rn(make_float2(sa.z, sa.w), m1, x[1]);
  const float2 r2 = __ffma2_rn(make_float2(sb.x, sb.y), m1, x[2]);
  const float2 d2 = __ffma2_rn(r2, r2, __ffma2_rn(r1, r1, __fmul2_rn(r0, r0)));
  float2 ri;
  ri.x = d2.x > 1.0e-28f ? rsqrt_approx_f32(d2.x) : 0.0f;
  ri.y = d2.y > 1.0e-28f ? rsqrt_approx_f32(d2.y) : 0.0f;
  const float2 kd = __fmul2_rn(make_float2(c.k, c.k), __fmul2_rn(d2, ri));
  float2 sn, cs;
  sincos_mufu(kd.x, sn.x, cs.x);
  sincos_mufu(kd.y, sn.y, cs.y);
  float2 br, bi;
  if (KIND == SL) {
    const float2 re = __fmul2_rn(cs, ri), im = __fmul2_rn(sn, ri);
    k0 = make_float2(re.x, im.x);
    k1 = make_float2(re.y, im.y);
    return;
  }
  const float2 rn = __ffma2_rn(r2, make_float2(sc.z, sc.w),
                               __ffma2_rn(r1, make_float2(sc.x, sc.y), __fmul2_rn(r0, make_float2(sb.z, sb.w))));
  const float2 u = __fmul2_rn(rn, ri);
  if (KIND == CFI) {
    br = __fmul2_rn(u, __fmul2_rn(ri, ri));
    bi = __fmul2_rn(ri, __ffma2_rn(make_float2(-c.k, -c.k), u, make_float2(c.c2i, c.c2i)));
  } else {
    const float2 P = __fmul2_rn(u, ri);
    const float2 Q = __fmul2_rn(P, ri);
    if (KIND == DL) {
      br = Q;
      bi = __fmul2_rn(make_float2(-c.k, -c.k), P);
    } else {
      br = __ffma2_rn(make_float2(c.c2r, c.c2r), ri,
                      __ffma2_rn(make_float2(c.c1r, c.c1r), Q, __fmul2_rn(make_float2(c.kc1i, c.kc1i), P)));
      bi = __ffma2_rn(make_float2(c.c2i, c.c2i), ri,
                      __ffma2_rn(make_float2(c.c1i, c.c1i), Q, __fmul2_rn(make_float2(-c.kc1r, -c.kc1r), P)));
    }
  }
  const float2 nsn = make_float2(-sn.x, -sn.y);
  const float2 re = __ffma2_rn(cs, br, __fmul2_rn(nsn, bi));
  const float2 im = __ffma2_rn(cs, bi, __fmul2_rn(sn, br));
  k0 = make_float2(re.x, im.x);
  k1 = make_float2(re.y, im.y);
}

// Roles (warp w, one elected lane for the first two):
//   w = 0       MMA issuer: waits for a stage's A tiles and density block,
//               issues its 16 MMAs and commits them;
//   w = 1       copy producer: refills the density and source-record rings
//               (TMA bulk copies) as soon as the MMAs of a stage have freed
//               its buffers;
//   w = 2..17   generators (each thread two target rows, one per
//               accumulator, and 8 sources of a stage) and the epilogue.
// Splitting issue and production keeps each lane's serial path short: the
// barrier and copy operations of one lane queue behind the generators' own
// shared/tensor-memory traffic, so a lane doing both fell behind.
// Hand-offs go through mbarriers:
//   fullS[NS]    source records of a stage landed    (copy engine)
//   fullB[NB]    density block of a stage landed     (copy engine)
//   aFull[2]     A tiles of a stage written          (16 generator warps)
//   mmaDone[NB]  MMA group of a stage complete       (tcgen05.commit)
// Stage g of the CTA (counted over all its items) uses fullS[g % NS],
// fullB[g % NB], mmaDone[g % NB] and A buffer g & 1.  Every wait names the
// phase of exactly one pending completion (the previous one on that barrier
// is known complete and the next cannot start before the waiter acts), so
// the parity test is exact.
// (Splitting aFull/mmaDone per K quarter, so that warp groups drift apart
// without waiting for one another, measured slower: four commits per stage
// cost more than the skew they hide.)
template <int KIND>
__global__ void __launch_bounds__(TC_THREADS, 1) mrhs_tc_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t fullS[TC_NS], fullB[TC_NB], aFull[2], mmaDone[TC_NB], drainBar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int item_sh;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gw = warp - 2;  // generator index 0..15
  const TcConst kc{a.k, a.c1r, a.c1i, a.c2r, a.c2i, a.k * a.c1r, a.k * a.c1i};
  if (tid == 0) {
    for (int q = 0; q < TC_NS; ++q) mbar_init(&fullS[q], 1);
    for (int q = 0; q < TC_NB; ++q) {
      mbar_init(&fullB[q], 1);
      mbar_init(&mmaDone[q], 1);
    }
    for (int q = 0; q < 2; ++q) mbar_init(&aFull[q], TC_GEN_WARPS);
    mbar_init(&drainBar, 1);
    mbar_fence_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const uint32_t sbase = smem_u32(sm);

  uint32_t g = 0;          // first stage of the current item (same in every thread)
  uint32_t nS = 0, nB = 0;  // producer lane: source and density copies issued
  uint32_t nC = 0;          // issuer lane: MMA groups committed
  bool ok = true;

  for (;;) {
    if (tid == 0) item_sh = atomicAdd(a.counter, 1);
    __syncthreads();
    const int it = item_sh;
    if (it >= a.nitems * a.ncolgroups) break;
    const int cg = it / a.nitems;
    const int item = it % a.nitems;
    const int s = a.item_surf[item];
    const int64_t off = a.off[s], n = a.off[s + 1] - off;
    const uint32_t T = (uint32_t)((n + TC_J - 1) / TC_J);
    const float* srcs = a.src + (size_t)a.toff[s] * TC_J * TC_S_FLOATS;
    const uint32_t* bp = a.bpack + ((size_t)cg * a.ntiles + a.toff[s]) * (TC_B_BYTES / 4);
    if (warp == 0) {
      // The whole warp runs the loop on warp-uniform operands and one elected
      // lane issues: measured ~2x faster MMA issue than a lone lane when the
      // generator warps compete for the scheduler.
      for (uint32_t t = 0; t < T; ++t) {
        const uint32_t gg = g + t, bb = gg & 1, nb = gg % TC_NB;
        ok = mbar_wait_bounded(&aFull[bb], (gg >> 1) & 1) && mbar_wait_bounded(&fullB[nb], (gg / TC_NB) & 1);
        if (!__all_sync(0xffffffffu, ok)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint64_t bdesc = tc_smem_desc(sbase + TC_OFF_B + nb * TC_B_BYTES);
        if (elect_one()) {
          tc_mma8_ts(tmem, tmem + tc_a_col(bb, 0), bdesc, t > 0 ? 1u : 0u);
          tc_mma8_ts(tmem + TC_N, tmem + tc_a_col(bb, 1), bdesc, t > 0 ? 1u : 0u);
          tc_commit(&mmaDone[nb]);
        }
        __syncwarp();
        ++nC;
      }
    } else if (warp == 1) {
      // Stage x's copies go to the buffers of stage x - NB (densities) and
      // x - NS (sources); both are free once MMA group x - NB, respectively
      // x - NS, is complete, which (MMAs completing in order) the wait for
      // the MMA group one stage earlier than x's first use guarantees.
      auto copyS = [&](uint32_t t) {
        const uint32_t b = (g + t) % TC_NS;
        if (elect_one()) {
          mbar_arrive_expect_tx(&fullS[b], TC_S_BYTES);
          bulk_copy_g2s(sm + TC_OFF_S + b * TC_S_BYTES, srcs + (size_t)t * TC_J * TC_S_FLOATS, TC_S_BYTES, &fullS[b]);
        }
        __syncwarp();
        ++nS;
      };
      auto copyB = [&](uint32_t t) {
        const uint32_t b = (g + t) % TC_NB;
        if (elect_one()) {
          mbar_arrive_expect_tx(&fullB[b], TC_B_BYTES);
          bulk_copy_g2s(sm + TC_OFF_B + b * TC_B_BYTES, bp + (size_t)t * (TC_B_BYTES / 4), TC_B_BYTES, &fullB[b]);
        }
        __syncwarp();
        ++nB;
      };
      // prologue: buffers released by the previous item
      for (uint32_t t = 0; t < TC_NS - 1 && t < T; ++t) copyS(t);
      for (uint32_t t = 0; t < TC_NB - 1 && t < T; ++t) copyB(t);
      for (uint32_t t = 0; t + TC_NB - 1 < T || t + TC_NS - 1 < T; ++t) {
        const uint32_t gg = g + t;
        // MMA group gg-1 read density buffer (gg-1)%NB and, through its A
        // tiles, the source records of stage gg-1
        if (gg >= 1) ok = mbar_wait_bounded(&mmaDone[(gg - 1) % TC_NB], ((gg - 1) / TC_NB) & 1);
        if (!__all_sync(0xffffffffu, ok)) {
          ok = false;
          break;
        }
        if (t + TC_NB - 1 < T) copyB(t + TC_NB - 1);
        if (t + TC_NS - 1 < T) copyS(t + TC_NS - 1);
      }
    } else {
      // generation: rows ra (accumulator 0) and ra + 128 (accumulator 1),
      // sources 8*(gw>>2) .. +7 of each stage; ra lies in the tensor-memory
      // lane quarter warp % 4 that this warp may access
      const int ra = 32 * (warp & 3) + lane;
      const int j0 = (gw >> 2) * (TC_J / 4);
      const int64_t blk0 = (int64_t)a.item_block[item] * TC_ROWS;
      float2 xt[3];  // (row ra, row ra + 128) coordinates
      {
        const int64_t t0i = off + min(blk0 + ra, n - 1), t1i = off + min(blk0 + ra + 128, n - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) xt[c] = make_float2((float)a.coords[3 * t0i + c], (float)a.coords[3 * t1i + c]);
      }
      const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
      for (uint32_t t = 0; t < T; ++t) {
        const uint32_t gg = g + t, sb = gg % TC_NS;
        bool w = mbar_wait_bounded(&fullS[sb], (gg / TC_NS) & 1);
        // A buffer gg&1 was last read by MMA group gg-2
        if (w && gg >= 2) w = mbar_wait_bounded(&mmaDone[(gg - 2) % TC_NB], ((gg - 2) / TC_NB) & 1);
        if (!__all_sync(0xffffffffu, w)) {
          ok = false;
          break;
        }
        tc_fence_after();
        // padded sources (past n) have zero density rows: their finite values add nothing
        const float* S = reinterpret_cast<const float*>(sm + TC_OFF_S + sb * TC_S_BYTES);
#pragma unroll
        for (int jq = 0; jq < TC_J / 4; jq += 4) {
          uint32_t v[2][8];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int j = j0 + jq + e;
            const float4 sa = *reinterpret_cast<const float4*>(S + j * TC_S_FLOATS);
            const float4 sb = *reinterpret_cast<const float4*>(S + j * TC_S_FLOATS + 4);
            const float4 sc = *reinterpret_cast<const float4*>(S + j * TC_S_FLOATS + 8);
            float2 k0, k1;
            tc_kernel_x2<KIND>(xt, sa, sb, sc, kc, k0, k1);
            v[0][2 * e] = tf32_bits(k0.x);
            v[0][2 * e + 1] = tf32_bits(k0.y);
            v[1][2 * e] = tf32_bits(k1.x);
            v[1][2 * e + 1] = tf32_bits(k1.y);
          }
#pragma unroll
          for (int h = 0; h < 2; ++h) tc_st8(lane_base + tc_a_col(gg & 1, h) + 2 * (j0 + jq), v[h]);
        }
        tc_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&aFull[gg & 1]);
      }
      if (ok) {
        const uint32_t gl = g + T - 1;
        ok = __all_sync(0xffffffffu, mbar_wait_bounded(&mmaDone[gl % TC_NB], (gl / TC_NB) & 1));
      }
      if (ok) {
        tc_fence_after();
        // generator gw: accumulator (gw>>2)&1, TMEM lane quarter warp&3, column half gw>>3
        const int acc = (gw >> 2) & 1, half = gw >> 3;
        const int64_t row_loc = blk0 + acc * 128 + ra;
        const bool active = row_loc < n;
        const uint32_t lane_addr = lane_base + acc * TC_N;
        const double sc = 1.0 / (4 * kPi);
        const int c0 = cg * TC_R;
        double2* Y = reinterpret_cast<double2*>(a.y);
        for (int m = half * (TC_R / 2); m < (half + 1) * (TC_R / 2); m += 16) {
          float re[16], im[16];
          tc_ld16(lane_addr + m, re);
          tc_ld16(lane_addr + TC_R + m, im);
          tc_wait_ld();
          if (active) {
#pragma unroll
            for (int c = 0; c < 16; ++c) {
              const int col = c0 + m + c;
              if (col >= a.nrhs) break;
              const int64_t o = (int64_t)col * a.ldy + off + row_loc;
              const double yr = sc * re[c], yi = sc * im[c];
              double orr = a.ar * yr - a.ai * yi, oi = a.ar * yi + a.ai * yr;
              if (!a.beta_zero) {
                const double2 yo = Y[o];
                orr += a.br * yo.x - a.bi * yo.y;
                oi += a.br * yo.y + a.bi * yo.x;
              }
              Y[o] = make_double2(orr, oi);
            }
          }
        }
      }
    }
    g += T;
    tc_fence_before();
    // accumulators read (or the item abandoned) before the next item's MMAs
    if (__syncthreads_or(!ok)) goto fail;
  }
  goto done;
fail:
  if (tid == 0) atomicExch(a.err, kErrWaitTimeout);
  // Everything this CTA put in flight must land before it leaves: at most the
  // last NS source copies and the last NB density copies are pending (each
  // alone on its barrier), and one more commit tracks every MMA issued.
  if (warp == 1 && lane == 0) {
    for (uint32_t q = nS > TC_NS ? nS - TC_NS : 0; q < nS; ++q) mbar_wait_bounded(&fullS[q % TC_NS], (q / TC_NS) & 1);
    for (uint32_t q = nB > TC_NB ? nB - TC_NB : 0; q < nB; ++q) mbar_wait_bounded(&fullB[q % TC_NB], (q / TC_NB) & 1);
  }
  if (warp == 0) {
    // the MMAs were issued by the elected lane: the same lane commits
    if (nC > 0 && elect_one()) {
      tc_commit(&drainBar);
      mbar_wait_bounded(&drainBar, 0);
    }
    __syncwarp();
  }
  __syncthreads();
done:
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
  }
}

// Source records (FP32) per source, every value twice: x x y y z z nx nx
// ny ny nz nz and four pad floats; tiles of TC_J per surface, zero-padded.
__global__ void tc_pack_sources(int nsurf, const int64_t* off, const int64_t* toff, const double* coords,
                                const double* normals, float* out) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // padded source slot
  // find the surface of slot g (tiles are few; linear scan over surfaces)
  int s = 0;
  while (s + 1 < nsurf && toff[s + 1] * TC_J <= g) ++s;
  if (g >= toff[nsurf] * TC_J) return;
  const int64_t j = g - toff[s] * TC_J;
  const int64_t n = off[s + 1] - off[s];
  float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (j < n) {
    const int64_t i = off[s] + j;
    for (int c = 0; c < 3; ++c) {
      v[c] = (float)coords[3 * i + c];
      v[3 + c] = normals ? (float)normals[3 * i + c] : 0.f;
    }
  }
  float4* o = reinterpret_cast<float4*>(out + g * TC_S_FLOATS);
  o[0] = make_float4(v[0], v[0], v[1], v[1]);
  o[1] = make_float4(v[2], v[2], v[3], v[3]);
  o[2] = make_float4(v[4], v[4], v[5], v[5]);
  o[3] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Density blocks: for column group cg and tile (surface s, local tile lt),
// B[n][k] in the canonical K-major layout (see the header), TF32.
__global__ void tc_pack_density(int nsurf, const int64_t* off, const int64_t* toff, int64_t tile0,
                                int64_t tile1, int64_t ntiles, const double* weights, const double* x,
                                int64_t ldx, int nrhs, int cg, uint32_t* out) {
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t tile = tile0 + gid / (TC_N * TC_K / 4);  // one thread per 16-byte chunk
  if (tile >= tile1) return;
  const int rem = (int)(gid % (TC_N * TC_K / 4));
  const int nn = rem / (TC_K / 4), kc = rem % (TC_K / 4);  // column n, K chunk
  int s = 0;
  while (s + 1 < nsurf && toff[s + 1] <= tile) ++s;
  const int64_t n = off[s + 1] - off[s];
  const int64_t lt = tile - toff[s];
  const int r = nn & (TC_R - 1);
  const bool imag_half = nn >= TC_R;
  const int col = cg * TC_R + r;
  uint32_t v[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const int k = 4 * kc + e;
    const int64_t j = lt * TC_J + (k >> 1);
    float val = 0.f;
    if (j < n && col < nrhs) {
      const int64_t node = off[s] + j;
      const double2 xv = reinterpret_cast<const double2*>(x)[(int64_t)col * ldx + node];
      const double w = weights[node];
      const double xr = w * xv.x, xi = w * xv.y;
      // rows 2j: (Re x, Im x) for the (Re, Im) halves; rows 2j+1: (-Im x, Re x)
      if ((k & 1) == 0)
        val = (float)(imag_half ? xi : xr);
      else
        val = (float)(imag_half ? xr : -xi);
    }
    v[e] = to_tf32(val);
  }
  uint32_t* o = out + (((size_t)cg * ntiles + tile) * (TC_B_BYTES / 4)) + tc_kmajor_off(nn, 4 * kc) / 4;
  *reinterpret_cast<uint4*>(o) = make_uint4(v[0], v[1], v[2], v[3]);
}

// Throughput of the tensor cores for the MMA shape the batch kernel issues
// (kind::tf32, M = N = 128, K = 8, A in tensor memory, B in shared memory):
// one CTA per SM issues `rounds` x 8 back-to-back MMAs on zeroed operands.
__global__ void __launch_bounds__(128, 1) tc_peak_probe(int rounds, int* err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base_sh;
  for (int i = threadIdx.x; i < TC_B_BYTES / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(sm)[i] = 0;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  if (threadIdx.x < 32) {
    const uint64_t bdesc = tc_smem_desc(smem_u32(sm));
    if (elect_one()) {
      for (int r = 0; r < rounds; ++r) tc_mma8_ts(tmem, tmem + TC_TMEM_A, bdesc, r > 0 ? 1u : 0u);
      tc_commit(&bar);
      if (!mbar_wait_bounded(&bar, 0)) atomicExch(err, kErrWaitTimeout);
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
  }
}

void measure_peak_tf32(inti_ctx* ctx, double* tf32_flops) {
  const int rounds = 8192;  // ~4 ms of MMAs: launch and TMEM allocation costs drop below 1%
  INTI_CUDA(cudaFuncSetAttribute(tc_peak_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_B_BYTES));
  cudaEvent_t e0, e1;
  INTI_CUDA(cudaEventCreate(&e0));
  INTI_CUDA(cudaEventCreate(&e1));
  ctx->flag_armed = true;
  tc_peak_probe<<<ctx->num_sms, 128, TC_B_BYTES, ctx->stream>>>(rounds, ctx->err_flag.as<int>());  // warm-up
  INTI_CUDA(cudaEventRecord(e0, ctx->stream));
  tc_peak_probe<<<ctx->num_sms, 128, TC_B_BYTES, ctx->stream>>>(rounds, ctx->err_flag.as<int>());
  INTI_CUDA(cudaEventRecord(e1, ctx->stream));
  ctx->launches += 2;
  INTI_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  INTI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  INTI_CUDA(cudaGetLastError());
  sync_and_check(ctx);
  *tf32_flops = 2.0 * 128 * TC_N * 8 * (TC_K / 8) * (double)rounds * ctx->num_sms / (ms * 1e-3);
}

// Tile offsets, 256-target items (largest surfaces first), packed source
// records and kernel attributes: built once per batch (an apply after the
// first only enqueues work, so it can be captured into a CUDA graph).
static void tc_setup(inti_batch* b) {
  if (b->tc_src.p) return;
  inti_ctx* ctx = b->ctx;
  const int nsurf = (int)b->off.size() - 1;
  std::vector<int64_t> toff(nsurf + 1, 0);
  for (int s = 0; s < nsurf; ++s) toff[s + 1] = toff[s] + (b->off[s + 1] - b->off[s] + TC_J - 1) / TC_J;
  std::vector<int> order(nsurf);
  for (int s = 0; s < nsurf; ++s) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
    return b->off[p + 1] - b->off[p] > b->off[q + 1] - b->off[q];
  });
  std::vector<int32_t> isurf, iblk;
  for (int s : order)
    for (int64_t t = 0; t * TC_ROWS < b->off[s + 1] - b->off[s]; ++t) {
      isurf.push_back(s);
      iblk.push_back((int32_t)t);
    }
  b->tc_ntiles = toff[nsurf];
  b->tc_nitems = (int)isurf.size();
  b->tc_toff.ensure(sizeof(int64_t) * (nsurf + 1));
  INTI_CUDA(cudaMemcpy(b->tc_toff.p, toff.data(), sizeof(int64_t) * (nsurf + 1), cudaMemcpyHostToDevice));
  b->tc_items.ensure(sizeof(int32_t) * 2 * b->tc_nitems);
  INTI_CUDA(cudaMemcpy(b->tc_items.p, isurf.data(), sizeof(int32_t) * b->tc_nitems, cudaMemcpyHostToDevice));
  INTI_CUDA(cudaMemcpy(b->tc_items.as<int32_t>() + b->tc_nitems, iblk.data(), sizeof(int32_t) * b->tc_nitems,
                       cudaMemcpyHostToDevice));
  // surface groups for the pipelined host apply: contiguous surface ranges of
  // about equal pair work, at most 8
  std::vector<double> work(nsurf);
  double total = 0.0;
  for (int s = 0; s < nsurf; ++s) {
    const double ns = (double)(b->off[s + 1] - b->off[s]);
    work[s] = ns * ns;
    total += work[s];
  }
  const int ngrp = std::min(nsurf, 8);
  b->grp_s.assign(1, 0);
  double acc = 0.0;
  for (int s = 0; s + 1 < nsurf; ++s) {
    acc += work[s];
    const int made = (int)b->grp_s.size();  // groups started so far
    if (made >= ngrp) break;
    // a new group at s + 1 once this one holds its share of the work, or when
    // every remaining surface has to start a group of its own
    if (acc >= total * made / ngrp || nsurf - (s + 1) == ngrp - made) b->grp_s.push_back(s + 1);
  }
  b->grp_s.push_back(nsurf);
  std::vector<int32_t> gs, gb;
  b->grp_item.assign(1, 0);
  for (size_t g = 0; g + 1 < b->grp_s.size(); ++g) {
    for (int s : order)
      if (s >= b->grp_s[g] && s < b->grp_s[g + 1])
        for (int64_t t = 0; t * TC_ROWS < b->off[s + 1] - b->off[s]; ++t) {
          gs.push_back(s);
          gb.push_back((int32_t)t);
        }
    b->grp_item.push_back((int)gs.size());
  }
  b->tc_items_grp.ensure(sizeof(int32_t) * 2 * gs.size());
  INTI_CUDA(cudaMemcpy(b->tc_items_grp.p, gs.data(), sizeof(int32_t) * gs.size(), cudaMemcpyHostToDevice));
  INTI_CUDA(cudaMemcpy(b->tc_items_grp.as<int32_t>() + gs.size(), gb.data(), sizeof(int32_t) * gb.size(),
                       cudaMemcpyHostToDevice));
  b->tc_src.ensure(sizeof(float) * TC_S_FLOATS * TC_J * b->tc_ntiles);
  const int64_t slots = b->tc_ntiles * TC_J;
  tc_pack_sources<<<(unsigned)((slots + 255) / 256), 256, 0, ctx->stream>>>(
      nsurf, b->d_off.as<int64_t>(), b->tc_toff.as<int64_t>(), b->coords.as<double>(),
      b->kind == SL ? nullptr : b->normals.as<double>(), b->tc_src.as<float>());
  ctx->launches++;
  b->tc_counter.ensure(sizeof(int));
  for (const void* kern : {(const void*)mrhs_tc_kernel<SL>, (const void*)mrhs_tc_kernel<DL>,
                           (const void*)mrhs_tc_kernel<CF>, (const void*)mrhs_tc_kernel<CFI>})
    INTI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
}

// Density blocks of tiles [tile0, tile1) for every 64-column group.
static void tc_pack(inti_batch* b, const double* x, int64_t ldx, int nrhs, int64_t tile0, int64_t tile1) {
  inti_ctx* ctx = b->ctx;
  const int nsurf = (int)b->off.size() - 1;
  const int ncg = (nrhs + TC_R - 1) / TC_R;
  b->tc_b.ensure((size_t)ncg * b->tc_ntiles * TC_B_BYTES);
  if (tile1 <= tile0) return;
  ProfScope pp(ctx, "batch_pack");
  for (int cg = 0; cg < ncg; ++cg) {
    const int64_t chunks = (tile1 - tile0) * (TC_N * TC_K / 4);
    tc_pack_density<<<(unsigned)((chunks + 255) / 256), 256, 0, ctx->stream>>>(
        nsurf, b->d_off.as<int64_t>(), b->tc_toff.as<int64_t>(), tile0, tile1, b->tc_ntiles,
        b->weights.as<double>(), x, ldx, nrhs, cg, b->tc_b.as<uint32_t>());
    ctx->launches++;
  }
}

// The tensor-core kernel over nitems work items (item_surf[i], item_block[i]).
static void tc_run(inti_batch* b, const BatchArgs& a, const int32_t* item_surf, const int32_t* item_block,
                   int nitems) {
  inti_ctx* ctx = b->ctx;
  TcArgs t;
  t.off = b->d_off.as<int64_t>();
  t.toff = b->tc_toff.as<int64_t>();
  t.item_surf = item_surf;
  t.item_block = item_block;
  t.nitems = nitems;
  t.ncolgroups = (a.nrhs + TC_R - 1) / TC_R;
  t.src = b->tc_src.as<float>();
  t.bpack = b->tc_b.as<uint32_t>();
  t.ntiles = b->tc_ntiles;
  t.coords = b->coords.as<double>();
  t.y = a.y;
  t.ldy = a.ldy;
  t.nrhs = a.nrhs;
  t.k = (float)b->k;
  t.c1r = (float)b->c1[0];
  t.c1i = (float)b->c1[1];
  t.c2r = (float)b->c2[0];
  t.c2i = (float)b->c2[1];
  t.kind = b->kind;
  t.ar = a.ar;
  t.ai = a.ai;
  t.br = a.br;
  t.bi = a.bi;
  t.beta_zero = a.beta_zero;
  t.counter = b->tc_counter.as<int>();
  t.err = ctx->err_flag.as<int>();
  ctx->flag_armed = true;
  INTI_CUDA(cudaMemsetAsync(b->tc_counter.p, 0, sizeof(int), ctx->stream));
  auto launch = [&](auto kern) {
    ProfScope pk(ctx, "batch_tc");
    kern<<<ctx->num_sms, TC_THREADS, TC_SMEM, ctx->stream>>>(t);
  };
  if (b->kind == SL)
    launch(mrhs_tc_kernel<SL>);
  else if (b->kind == DL)
    launch(mrhs_tc_kernel<DL>);
  else if (b->c1[0] == 1.0 && b->c1[1] == 0.0 && b->c2[0] == 0.0)
    launch(mrhs_tc_kernel<CFI>);
  else
    launch(mrhs_tc_kernel<CF>);
  ctx->launches++;
  INTI_CUDA(cudaGetLastError());
}

void mrhs_tc_launch(inti_batch* b, const BatchArgs& a) {
  tc_setup(b);
  tc_pack(b, a.x, a.ldx, a.nrhs, 0, b->tc_ntiles);
  tc_run(b, a, b->tc_items.as<int32_t>(), b->tc_items.as<int32_t>() + b->tc_nitems, b->tc_nitems);
}

void batch_apply_host_tf32(inti_batch* b, const double* x, int64_t ldx, double* y, int64_t ldy, int32_t nrhs,
                           const double* alpha, const double* beta) {
  inti_ctx* ctx = b->ctx;
  if (b->pde != INTI_HELMHOLTZ) throw Error(INTI_E_UNSUPPORTED, "the tensor-core form is implemented for Helmholtz");
  const size_t pitch_x = sizeof(double2) * ldx, pitch_y = sizeof(double2) * ldy;
  DevBuf &xd = b->xstage, &yd = b->ystage;
  xd.ensure(pitch_x * nrhs);
  yd.ensure(pitch_y * nrhs);
  tc_setup(b);
  const int ngrp = (int)b->grp_s.size() - 1;
  if (!b->s_in) {
    INTI_CUDA(cudaStreamCreateWithFlags(&b->s_in, cudaStreamNonBlocking));
    INTI_CUDA(cudaStreamCreateWithFlags(&b->s_out, cudaStreamNonBlocking));
  }
  while ((int)b->ev.size() < 2 * ngrp + 2) {
    cudaEvent_t e;
    INTI_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev.push_back(e);
  }
  BatchArgs a{};
  a.x = xd.as<double>();
  a.ldx = ldx;
  a.y = yd.as<double>();
  a.ldy = ldy;
  a.nrhs = nrhs;
  a.ar = alpha ? alpha[0] : 1.0;
  a.ai = alpha ? alpha[1] : 0.0;
  a.br = beta ? beta[0] : 0.0;
  a.bi = beta ? beta[1] : 0.0;
  a.beta_zero = a.br == 0.0 && a.bi == 0.0;
  std::vector<int64_t> toff(b->off.size());
  for (size_t s = 0; s + 1 < b->off.size(); ++s)
    toff[s + 1] = toff[s] + (b->off[s + 1] - b->off[s] + TC_J - 1) / TC_J;
  // the input stream starts after the work already queued on the context's stream
  INTI_CUDA(cudaEventRecord(b->ev[2 * ngrp], ctx->stream));
  INTI_CUDA(cudaStreamWaitEvent(b->s_in, b->ev[2 * ngrp], 0));
  INTI_CUDA(cudaStreamWaitEvent(b->s_out, b->ev[2 * ngrp], 0));
  const int32_t* gs = b->tc_items_grp.as<int32_t>();
  const int32_t* gb = gs + b->grp_item.back();
  for (int g = 0; g < ngrp; ++g) {
    const int s0 = b->grp_s[g], s1 = b->grp_s[g + 1];
    const int64_t r0 = b->off[s0], rows = b->off[s1] - r0;
    const size_t width = sizeof(double2) * rows;
    // in: X rows (and Y rows when beta != 0) of this group, all columns
    INTI_CUDA(cudaMemcpy2DAsync(xd.as<double2>() + r0, pitch_x, reinterpret_cast<const double2*>(x) + r0, pitch_x,
                                width, nrhs, cudaMemcpyHostToDevice, b->s_in));
    if (!a.beta_zero)
      INTI_CUDA(cudaMemcpy2DAsync(yd.as<double2>() + r0, pitch_y, reinterpret_cast<const double2*>(y) + r0,
                                  pitch_y, width, nrhs, cudaMemcpyHostToDevice, b->s_in));
    INTI_CUDA(cudaEventRecord(b->ev[2 * g], b->s_in));
    INTI_CUDA(cudaStreamWaitEvent(ctx->stream, b->ev[2 * g], 0));
    // compute: this group's density tiles, items and correction rows
    tc_pack(b, a.x, ldx, nrhs, toff[s0], toff[s1]);
    const int i0 = b->grp_item[g], i1 = b->grp_item[g + 1];
    tc_run(b, a, gs + i0, gb + i0, i1 - i0);
    batch_correction_rows(b, a.x, ldx, a.y, ldy, nrhs, a.ar, a.ai, r0, r0 + rows);
    INTI_CUDA(cudaEventRecord(b->ev[2 * g + 1], ctx->stream));
    // out: Y rows of this group
    INTI_CUDA(cudaStreamWaitEvent(b->s_out, b->ev[2 * g + 1], 0));
    INTI_CUDA(cudaMemcpy2DAsync(reinterpret_cast<double2*>(y) + r0, pitch_y, yd.as<double2>() + r0, pitch_y, width,
                                nrhs, cudaMemcpyDeviceToHost, b->s_out));
  }
  INTI_CUDA(cudaEventRecord(b->ev[2 * ngrp + 1], b->s_out));
  INTI_CUDA(cudaStreamWaitEvent(ctx->stream, b->ev[2 * ngrp + 1], 0));
  sync_and_check(ctx);
}

}  // namespace inti
