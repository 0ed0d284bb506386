// Internal declarations shared by the CUDA translation units of
// libinti_b200.so.  Nothing here is part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/inti_b200.h"

namespace inti {

// src/utils.jl:235 — pairs closer than this are the excluded self-pair.  The
// kernels compare the squared distance with its square.
constexpr double kSamePointTol = 1.0e-14;
constexpr double kSamePointTol2 = 1.0e-28;
constexpr double kPi = 3.14159265358979323846;

// An error carrying an ABI status code; caught at the C boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define INTI_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess)                                                           \
      throw ::inti::Error(INTI_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

// Device blocks are taken from, and given back to, a per-device CUDA memory
// pool that keeps released memory (devmem.cu): creating and destroying
// operators then rarely goes back to the driver, whose allocation latency on
// a busy host ranges from microseconds to tens of milliseconds.  Giving a
// block back waits for its device to be idle, as cudaFree does, so memory
// handed out again is never still in use.
void* dev_alloc(size_t nbytes, int* device, size_t* got);  // throws Error(INTI_E_NOMEM)
void dev_release(void* p, size_t bytes, int device);
size_t dev_cache_bytes(int device);  // bytes the pool holds free
void dev_prepare(int device);        // create the device's pool now (context creation)

// Device allocation owned by a handle.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int device = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) dev_release(p, bytes, device);
    p = nullptr;
    bytes = 0;
  }
  void ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return;
    release();
    if (nbytes == 0) nbytes = 16;
    p = dev_alloc(nbytes, &device, &bytes);
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

}  // namespace inti

struct inti_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  std::recursive_mutex mu;
  std::string last_error;
  int64_t launches = 0;
  inti::DevBuf err_flag;  // device int: nonzero when a bounded wait ran out
  int* err_host = nullptr;  // page-locked copy of err_flag, read after a stream sync
  // set when a kernel that can raise err_flag (one with bounded waits) is
  // enqueued; a synchronising call reads the flag back only then
  bool flag_armed = false;
  inti::DevBuf scan_tmp;    // device-scan scratch (correction merges), kept between calls
  inti::DevBuf expi64, expi32;  // e^{i m delta} tables of the Helmholtz pair loops
  // per-kernel-class event timing (inti_ctx_set_profiling)
  bool profiling = false;
  struct Span {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<Span> spans;
  std::map<std::string, std::pair<double, int64_t>> prof_totals;
  // pair-kernel launch shapes picked by measurement (inti_ctx_set_autotune):
  // key "pde/kind/dim/precision/m/n" -> (targets per thread, split)
  bool autotune = true;
  std::map<std::string, std::pair<int, int>> tuned;
  // square operators created while this is set use the symmetric pair
  // kernel (inti_ctx_set_symmetric)
  bool symmetric = true;
  // bytes of row and column partials a symmetric operator may hold before
  // its work is split into panels (inti_ctx_set_partial_budget)
  double symm_budget = 2.0e9;
  // FP64 operators of at most kSmallPairs pairs created while this is set
  // apply in the single-launch form (inti_ctx_set_single_launch)
  bool single_launch = true;
  // GMRES on systems of at most this many unknowns runs each Arnoldi step's
  // orthogonalisation and Givens update in one single-CTA kernel
  // (inti_ctx_set_gmres_small; 0 turns it off)
  int64_t krylov_small = 8192;
  // Row partials, column partials and panel running sums of the symmetric
  // form, shared by all of the context's symmetric operators: they are live
  // only from an apply's pair launch to its epilogue, and every launch of a
  // context goes to its one stream in call order (calls are serialised), so
  // no two applies use them at the same time.  Sized for the largest
  // operator (each within the partial budget).
  inti::DevBuf sym_ypart, sym_zpart, sym_acc;
  // GMRES workspace kept between solves: Krylov basis, work vectors, the
  // reduction scratch and the staged right-hand side / solution.
  struct {
    inti::DevBuf V, w, r, e, w_outer, partial, h, y, nrm, b, x, small;
  } krylov;
  // DIM construction workspace kept between constructions: source points,
  // traces, Theta, its partial sums, green multipliers.
  struct {
    inti::DevBuf d_xs, g0, g1, theta, part, mu;
  } dimwork;
};

struct inti_quad {
  inti_ctx* ctx = nullptr;
  int dim = 3;
  int64_t n = 0;
  int32_t nq = 0;
  bool has_normals = false;
  // device copies: coords/normals dim x n (AoS), weights n
  inti::DevBuf coords, normals, weights;
  std::vector<double> h_coords, h_normals, h_weights;  // host copies for setup work
};

struct inti_csr {
  inti_ctx* ctx = nullptr;
  int64_t m = 0, n = 0, nnz = 0;
  int dtype = INTI_F64;
  inti::DevBuf rowptr, col, val;
};

namespace inti {

// Records a CUDA event pair around the launches issued in its scope when the
// context is profiling.
struct ProfScope {
  inti_ctx* ctx;
  cudaEvent_t b = nullptr;
  const char* name;
  ProfScope(inti_ctx* c, const char* n) : ctx(c), name(n) {
    if (!ctx->profiling) return;
    cudaEvent_t a;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      b = nullptr;
      return;
    }
    cudaEventRecord(a, ctx->stream);
    ctx->spans.push_back({name, a, b});
  }
  ~ProfScope() {
    if (b) cudaEventRecord(b, ctx->stream);
  }
};

// Launch plumbing implemented in the .cu files.
enum Pde { LAPLACE = INTI_LAPLACE, HELMHOLTZ = INTI_HELMHOLTZ };
enum Kind { SL = INTI_SL, DL = INTI_DL, ADL = INTI_ADL, HS = INTI_HS, CF = 4 /* c1*DL + c2*SL */ };

// A panel of the symmetric form's work items: those whose source blocks lie
// in [col0, col0 + ncols).  Panels run one after another, so the column
// partials of one panel at a time are held (nb x ncols blocks).  Offsets are
// int32 indices into the plan table: items (3 x nitems), row pointers
// (rows + 1, panel-local item indices) and row items (nitems); rows = the
// row blocks with items in the panel (0 .. rows - 1).
struct SymPanel {
  int item_off = 0, nitems = 0;
  int rowptr_off = 0, rowitems_off = 0, rows = 0;
  int col0 = 0, ncols = 0;
};

// Per-apply description of the pair product A*x for one right-hand side.
struct PairLaunch {
  int pde, kind, dim, precision;
  double k;
  int64_t m, n;
  const double* tcoords;   // dim x m
  const double* tnormals;  // dim x m or null
  const double* scoords;   // dim x n
  const double* snormals;  // dim x n or null
  const double* sweights;  // n
  const double* x;         // density, n (x2 complex)
  void* packed;            // scratch: packed source records (n padded)
  void* partial;           // scratch: split x m accumulators
  double c1[2], c2[2];     // CF: dipole and charge coefficients (complex)
  int split;               // number of source chunks (computed by plan)
  int tpt = 4;             // targets per thread of the pair kernel (2 or 4)
  int64_t n_tiles;         // padded source tiles
  int* err_flag;
  // symmetric form (target set == source set; pair_symm): work items
  // (I, J0, J1), per row block the list of its items, column partials
  bool symm = false;
  int sym_nb = 0, sym_nitems = 0;
  const int32_t* sym_items = nullptr;     // 3 x nitems
  const int32_t* sym_rowptr = nullptr;    // nb + 1
  const int32_t* sym_rowitems = nullptr;  // nitems
  void* zpart = nullptr;                  // nb x (n_tiles * tile)
  // a shard of the items (inti_op_set_shard): launch these, with their ids
  int sym_launch_items = 0;
  const int32_t* sym_launch = nullptr;    // 3 x sym_launch_items
  const int32_t* sym_launch_ids = nullptr;
  // More than one panel: the panels (host array) index the plan table
  // sym_table; their column partials (rows of sym_zld nodes) are folded
  // into the running sums sym_acc (n x 8 B real, 16 B complex) after each
  // panel, and the epilogue reads sym_acc.  A shard launches, per panel p,
  // the sym_launch_panels[2p + 1] items at sym_launch_panels[2p] of its
  // table, clearing the sym_ypart_bytes / sym_zpart_bytes of partials first.
  int sym_npanels = 1;
  const SymPanel* sym_panels = nullptr;
  const int32_t* sym_table = nullptr;
  int64_t sym_zld = 0;
  void* sym_acc = nullptr;
  const int32_t* sym_launch_panels = nullptr;
  size_t sym_ypart_bytes = 0, sym_zpart_bytes = 0;
};

// Message for inti_last_error(NULL) from entry points that take no context.
void noalloc_error_set(const char* msg);
// e^{i m 2pi/1024} tables (device, owned by the context).
const double2* expi_table_f64(inti_ctx* ctx);
const float2* expi_table_f32(inti_ctx* ctx);
// Source records per tile (must match the kernel template parameter).
int pair_tile(int precision);
// Bytes of one packed source record.
// Most source chunks (partial sums per target) of one pair-kernel launch.
constexpr int kMaxSplit = 256;
int pair_record_bytes(int pde, int kind, int dim, int precision);
int pair_symm_record_bytes(int pde, int kind, int dim, int precision);  // packed record of the symmetric form
// Bytes of one partial accumulator per target per split.
int pair_partial_bytes(int pde, int precision);
// Symmetric form: node block of 128*tpt nodes; work items of row blocks
// against chunks of `ch` source blocks (the longest first), grouped into
// panels of `pcols` source blocks (pcols >= nb: one panel).  Per panel the
// table holds items (3 x nitems), row pointers (rows + 1) and row items
// (nitems); one panel gives the layout items, row pointers (nb + 1), row
// items.  nitems returns the largest panel's item count.
int pair_symm_block(int tpt);
void pair_symm_plan(int64_t n, int tpt, int ch, int pcols, std::vector<int32_t>& table,
                    std::vector<SymPanel>& panels, int& nb, int& nitems);
int pair_symm_default_ch(const inti_ctx* ctx, int pde, int kind, int dim, int precision, int64_t n, int tpt);
// Choose the split for a problem on this device.
int pair_plan_split(const inti_ctx* ctx, int pde, int kind, int dim, int precision, int64_t m,
                    int64_t n, int tpt = 4);
// Enqueue pack + pair kernels (results in L.partial); returns launches.
int pair_launch(inti_ctx* ctx, const PairLaunch& L);
// y = alpha*(scale*rowscale_i*sum_s partial + C x) + beta*y (rowscale NULL:
// 1); complex when cplx.
int pair_epilogue(inti_ctx* ctx, const PairLaunch& L, const inti_csr* corr, const double* x,
                  double* y, const double* alpha, const double* beta, const double* rowscale = nullptr);
// Dense assembly of A.
int pair_assemble(inti_ctx* ctx, const PairLaunch& L, double* out);
// Single-launch form of small FP64 products (one cluster kernel: source
// records, pair sums, correction rows, alpha/beta): operators of at most
// kSmallPairs pairs.  rowscale (nullable) scales row i's pair sum, as the
// epilogue does for transposed products (the source weights).
constexpr double kSmallPairs = 1048576.0;
bool pair_small_eligible(int precision, int64_t m, int64_t n);
int pair_small(inti_ctx* ctx, const PairLaunch& L, const inti_csr* corr, const double* x, double* y,
               const double* alpha, const double* beta, const double* rowscale = nullptr);

// CSR: y = alpha*C*x + beta*y (alpha/beta complex pairs); transpose via col scatter.
int csr_apply(inti_ctx* ctx, const inti_csr* c, const double* x, double* y, const double* alpha,
              const double* beta);

}  // namespace inti
