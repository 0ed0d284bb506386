// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// FP64 CPU restatement of the Inti.jl (v0.2.1) integral-operator path, used
// only as the checker by tests/, __graft_entry__.smoke() and the cpu_baseline
// leg of bench.py.  Nothing in the shipped library links or calls this file.
//
// Parity status: Inti.jl ships no golden vectors (its tests are tolerance
// checks against mathematical identities), and Julia is not available here,
// so the restatement is pinned against the reference's own known-answer
// identity tests re-run on it (tests/test_oracle_pins.py): Gauss-law D[1] =
// -1/2 on the surface, Green's identity with and without the DIM correction
// (test/green_identities_test.jl:93-105, test/normal_orientation_test.jl:
// 94-113), kernel normal derivatives versus finite differences
// (test/kernels_test.jl:41-67), and the quadrature identities of
// test/quadrature_test.jl:156-161 and test/meshgen_test.jl:16-26.
//
// Arithmetic mirrors the Julia source operation by operation (same grouping,
// no FMA contraction: build with -ffp-contract=off) so that results track the
// reference to rounding.  Every function cites the reference file:line it
// restates.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <atomic>
#include <thread>

using cd = std::complex<double>;
static const double PI = 3.14159265358979323846;

// src/utils.jl:235
static const double SAME_POINT_TOLERANCE = 1.0e-14;

enum { OR_LAPLACE = 0, OR_HELMHOLTZ = 1 };
enum { OR_SL = 0, OR_DL = 1, OR_ADL = 2, OR_HS = 3 };

// --------------------------------------------------------------------------
// Kernels: src/kernels.jl:137-204 (Laplace 2D/3D), :347-413 (Helmholtz 3D).
// r = x - y (target minus source); d = norm(r); zero when d <= 1e-14.
// --------------------------------------------------------------------------
template <int DIM>
static inline double dotv(const double* a, const double* b) {
  double s = a[0] * b[0];
  for (int i = 1; i < DIM; ++i) s = s + a[i] * b[i];
  return s;
}

template <int DIM>
static inline double laplace_kernel(int kind, const double* x, const double* nx,
                                    const double* y, const double* ny) {
  double r[DIM];
  for (int i = 0; i < DIM; ++i) r[i] = x[i] - y[i];
  const double d = std::sqrt(dotv<DIM>(r, r));
  if (d <= SAME_POINT_TOLERANCE) return 0.0;
  switch (kind) {
    case OR_SL:  // kernels.jl:137-151
      if (DIM == 2) return -1.0 / (2 * PI) * std::log(d);
      return 1.0 / (4 * PI) / d;
    case OR_DL:  // kernels.jl:153-168
      if (DIM == 2) return 1.0 / (2 * PI) / (d * d) * dotv<DIM>(r, ny);
      return 1.0 / (4 * PI) / (d * d * d) * dotv<DIM>(r, ny);
    case OR_ADL:  // kernels.jl:170-183
      if (DIM == 2) return -1.0 / (2 * PI) / (d * d) * dotv<DIM>(r, nx);
      return -1.0 / (4 * PI) / (d * d * d) * dotv<DIM>(r, nx);
    default: {  // OR_HS, kernels.jl:185-204
      const double id2 = 1.0 / (d * d);
      const double nxdny = dotv<DIM>(nx, ny);
      const double rdnx = dotv<DIM>(r, nx);
      const double rdny = dotv<DIM>(r, ny);
      if (DIM == 2) return id2 / (2 * PI) * (nxdny - 2 * rdnx * rdny * id2);
      return id2 / (4 * PI * d) * (nxdny - 3 * rdnx * rdny * id2);
    }
  }
}

// Helmholtz, 3D only (the 2D Hankel forms, kernels.jl:344-345, are not on
// this path).
static inline cd helmholtz3_kernel(int kind, double k, const double* x, const double* nx,
                                   const double* y, const double* ny) {
  double r[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
  const double d = std::sqrt(dotv<3>(r, r));
  if (d <= SAME_POINT_TOLERANCE) return cd(0.0, 0.0);
  const cd ik(0.0, k);
  const cd eikd = std::exp(ik * d);
  switch (kind) {
    case OR_SL:  // kernels.jl:347-358
      return 1.0 / (4 * PI) / d * eikd;
    case OR_DL:  // kernels.jl:362-373
      return (1.0 / (4 * PI * (d * d))) * eikd * (-ik + 1.0 / d) * dotv<3>(r, ny);
    case OR_ADL:  // kernels.jl:376-387
      return -(1.0 / (4 * PI * (d * d))) * eikd * (-ik + 1.0 / d) * dotv<3>(r, nx);
    default: {  // OR_HS, kernels.jl:390-413
      const double rdnx = dotv<3>(r, nx);
      const double rdny = dotv<3>(r, ny);
      const double nxdny = dotv<3>(nx, ny);
      const double id2 = 1.0 / (d * d);
      const cd b = eikd * id2 / (4 * PI) * (-ik + 1.0 / d);
      const cd a = eikd * id2 * id2 / (4 * PI * d) * (3.0 * (d * ik - 1.0) + d * d * k * k);
      return a * rdnx * rdny + b * nxdny;
    }
  }
}

static inline cd eval_kernel(int pde, int kind, int dim, double k, const double* x,
                             const double* nx, const double* y, const double* ny) {
  if (pde == OR_LAPLACE)
    return dim == 2 ? cd(laplace_kernel<2>(kind, x, nx, y, ny), 0.0)
                    : cd(laplace_kernel<3>(kind, x, nx, y, ny), 0.0);
  return helmholtz3_kernel(kind, k, x, nx, y, ny);
}

static int nthreads_or_default(int nt) {
  if (nt > 0) return nt;
  const unsigned hc = std::thread::hardware_concurrency();
  return hc ? (int)hc : 1;
}

// Dynamic-schedule parallel loop over [0, n) in chunks (std::thread; the
// oracle must not depend on an OpenMP runtime).
template <class F>
static void parallel_for(int64_t n, int nt, int64_t chunk, F&& body) {
  const int t = std::max(1, std::min<int>(nthreads_or_default(nt), (int)((n + chunk - 1) / std::max<int64_t>(chunk, 1))));
  if (t <= 1) {
    for (int64_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> pool;
  for (int q = 0; q < t; ++q)
    pool.emplace_back([&]() {
      for (;;) {
        const int64_t s = next.fetch_add(chunk);
        if (s >= n) break;
        const int64_t e = std::min(n, s + chunk);
        for (int64_t i = s; i < e; ++i) body(i);
      }
    });
  for (auto& th : pool) th.join();
}

// Real-valued Laplace rows: y_i = sum_j K(x_i, y_j) * w_j * sigma_j, summed in
// ascending j exactly like Base's generic AbstractMatrix*Vector over
// IntegralOperator entries (src/nystrom.jl:93-96: entry = K(x_i,y_j)*w_j).
template <int DIM>
static void laplace_rows(int kind, int64_t row0, int64_t nrows, const double* tx,
                         const double* tn, int64_t n, const double* sx, const double* sn,
                         const double* sw, const double* sigma, double* y, int nt) {
  parallel_for(nrows, nt, 16, [&](int64_t ii) {
    const int64_t i = row0 + ii;
    const double* x = tx + DIM * i;
    const double* nx = tn ? tn + DIM * i : nullptr;
    double acc = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      const double kij = laplace_kernel<DIM>(kind, x, nx, sx + DIM * j, sn ? sn + DIM * j : nullptr);
      acc = acc + (kij * sw[j]) * sigma[j];
    }
    y[ii] = acc;
  });
}

static void helmholtz_rows(int kind, double k, int64_t row0, int64_t nrows, const double* tx,
                           const double* tn, int64_t n, const double* sx, const double* sn,
                           const double* sw, const double* sigma, double* y, int nt) {
  const cd* s = reinterpret_cast<const cd*>(sigma);
  cd* out = reinterpret_cast<cd*>(y);
  parallel_for(nrows, nt, 16, [&](int64_t ii) {
    const int64_t i = row0 + ii;
    const double* x = tx + 3 * i;
    const double* nx = tn ? tn + 3 * i : nullptr;
    cd acc(0.0, 0.0);
    for (int64_t j = 0; j < n; ++j) {
      const cd kij = helmholtz3_kernel(kind, k, x, nx, sx + 3 * j, sn ? sn + 3 * j : nullptr);
      acc = acc + (kij * sw[j]) * s[j];
    }
    out[ii] = acc;
  });
}

extern "C" {

// Single kernel value K(x, y) as (re, im).  kernels.jl:137-204, 347-413.
int or_kernel(int pde, int kind, int dim, double k, const double* x, const double* nx,
              const double* y, const double* ny, double* out) {
  if (pde == OR_HELMHOLTZ && dim != 3) return 1;
  const cd v = eval_kernel(pde, kind, dim, k, x, nx, y, ny);
  out[0] = v.real();
  out[1] = v.imag();
  return 0;
}

// On-the-fly operator rows [row0, row0+nrows): y = (K .* w') * sigma.
// Laplace: sigma, y real.  Helmholtz: interleaved complex.  nystrom.jl:93-96.
int or_apply(int pde, int kind, int dim, double k, int64_t row0, int64_t nrows,
             const double* tx, const double* tn, int64_t n, const double* sx,
             const double* sn, const double* sw, const double* sigma, double* y,
             int nthreads) {
  if (pde == OR_LAPLACE) {
    if (dim == 2)
      laplace_rows<2>(kind, row0, nrows, tx, tn, n, sx, sn, sw, sigma, y, nthreads);
    else
      laplace_rows<3>(kind, row0, nrows, tx, tn, n, sx, sn, sw, sigma, y, nthreads);
    return 0;
  }
  if (dim != 3) return 1;
  helmholtz_rows(kind, k, row0, nrows, tx, tn, n, sx, sn, sw, sigma, y, nthreads);
  return 0;
}

// Dense column-major assembly out[i + m*j] = K(x_i, y_j) * w_j, threaded over
// source columns.  nystrom.jl:103-124 (_assemble_matrix!).
int or_assemble(int pde, int kind, int dim, double k, int64_t m, const double* tx,
                const double* tn, int64_t n, const double* sx, const double* sn,
                const double* sw, double* out, int nthreads) {
  if (pde == OR_HELMHOLTZ && dim != 3) return 1;
  const bool cplx = pde == OR_HELMHOLTZ;
  parallel_for(n, nthreads, 64, [&](int64_t j) {
    for (int64_t i = 0; i < m; ++i) {
      const cd v = eval_kernel(pde, kind, dim, k, tx + dim * i, tn ? tn + dim * i : nullptr,
                               sx + dim * j, sn ? sn + dim * j : nullptr) *
                   sw[j];
      if (cplx) {
        out[2 * (i + m * j)] = v.real();
        out[2 * (i + m * j) + 1] = v.imag();
      } else {
        out[i + m * j] = v.real();
      }
    }
  });
  return 0;
}

// y += A x for a 0-based CSR (rows sorted).  Restates SparseMatrixCSC*Vector
// as used by LinearMap(δS) (src/api.jl:179-184); the sum per row is taken in
// ascending column order.
void or_csr_apply(int64_t m, const int64_t* rowptr, const int32_t* col, const double* val,
                  int is_complex, const double* x, double* y) {
  for (int64_t i = 0; i < m; ++i) {
    if (is_complex) {
      cd acc(0.0, 0.0);
      for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p)
        acc += cd(val[2 * p], val[2 * p + 1]) * cd(x[2 * col[p]], x[2 * col[p] + 1]);
      y[2 * i] += acc.real();
      y[2 * i + 1] += acc.imag();
    } else {
      double acc = 0.0;
      for (int64_t p = rowptr[i]; p < rowptr[i + 1]; ++p) acc += val[p] * x[col[p]];
      y[i] += acc;
    }
  }
}

// COO -> CSR with duplicates summed and columns sorted within each row: the
// row-major view of SparseArrays.sparse(Is, Js, V, m, n) (src/bdim.jl:193-194),
// indices 0-based.  Returns nnz after merging; outputs sized for nnz_in.
int64_t or_coo_to_csr(int64_t m, int64_t nnz_in, const int64_t* I, const int64_t* J,
                      const double* V, int is_complex, int64_t* rowptr, int32_t* col,
                      double* val) {
  std::vector<int64_t> order(nnz_in);
  for (int64_t p = 0; p < nnz_in; ++p) order[p] = p;
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return I[a] != I[b] ? I[a] < I[b] : J[a] < J[b];
  });
  const int ncomp = is_complex ? 2 : 1;
  int64_t out = -1;
  std::vector<int64_t> cnt(m, 0);
  int64_t prevI = -1, prevJ = -1;
  for (int64_t q = 0; q < nnz_in; ++q) {
    const int64_t p = order[q];
    if (I[p] == prevI && J[p] == prevJ) {
      for (int c = 0; c < ncomp; ++c) val[ncomp * out + c] += V[ncomp * p + c];
    } else {
      ++out;
      col[out] = (int32_t)J[p];
      for (int c = 0; c < ncomp; ++c) val[ncomp * out + c] = V[ncomp * p + c];
      cnt[I[p]]++;
      prevI = I[p];
      prevJ = J[p];
    }
  }
  rowptr[0] = 0;
  for (int64_t i = 0; i < m; ++i) rowptr[i + 1] = rowptr[i] + cnt[i];
  return out + 1;
}

// DIM auxiliary source points: src/utils.jl:142-171 (uniform_points_circle,
// fibonnaci_points_sphere).
void or_dim_sources(int dim, int ns, double R, const double* c, double* xs) {
  if (dim == 2) {
    for (int i = 0; i < ns; ++i) {
      xs[2 * i] = R * std::cos(2 * PI * i / ns) + c[0];
      xs[2 * i + 1] = R * std::sin(2 * PI * i / ns) + c[1];
    }
    return;
  }
  const double phi = PI * (3 - std::sqrt(5.0));
  for (int i = 1; i <= ns; ++i) {
    const double ytmp = 1 - ((double)(i - 1) / (double)(ns - 1)) * 2;
    const double radius = std::sqrt(1 - ytmp * ytmp);
    const double theta = phi * i;
    xs[3 * (i - 1) + 0] = std::cos(theta) * radius * R + c[0];
    xs[3 * (i - 1) + 1] = ytmp * R + c[1];
    xs[3 * (i - 1) + 2] = std::sin(theta) * radius * R + c[2];
  }
}

}  // extern "C"

// --------------------------------------------------------------------------
// Householder QR least squares (no pivoting), real or complex, for the
// overdetermined ns x 2nq systems of src/bdim.jl:154-185 (qr!(transpose(M)),
// ldiv!).  Householder vectors follow the LAPACK xLARFG convention:
// H = I - tau v v^H with v(0) = 1 and a real beta on the diagonal.
// --------------------------------------------------------------------------
template <class T>
static inline double absv2(const T& v) { return std::norm(cd(v)); }
static inline double conjv(double v) { return v; }
static inline cd conjv(const cd& v) { return std::conj(v); }
static inline double realv(double v) { return v; }
static inline double realv(const cd& v) { return v.real(); }
static inline double imagv(double) { return 0.0; }
static inline double imagv(const cd& v) { return v.imag(); }

template <class T>
struct HouseholderQR {
  int rows, cols;       // rows >= cols
  std::vector<T> a;     // column-major rows x cols, R above diagonal, v below
  std::vector<T> tau;
  void factor() {
    tau.assign(cols, T(0));
    for (int k = 0; k < cols; ++k) {
      T* colk = &a[(size_t)k * rows];
      const T alpha = colk[k];
      double xnorm2 = 0.0;
      for (int i = k + 1; i < rows; ++i) xnorm2 += absv2(colk[i]);
      if (xnorm2 == 0.0 && imagv(alpha) == 0.0) {
        tau[k] = T(0);
        continue;
      }
      const double nrm = std::sqrt(absv2(alpha) + xnorm2);
      const double beta = realv(alpha) >= 0 ? -nrm : nrm;
      if constexpr (std::is_same<T, cd>::value)
        tau[k] = cd((beta - alpha.real()) / beta, -alpha.imag() / beta);
      else
        tau[k] = (beta - alpha) / beta;
      const T scal = T(1) / (alpha - T(beta));
      for (int i = k + 1; i < rows; ++i) colk[i] *= scal;
      colk[k] = T(beta);
      // apply H^H = I - conj(tau) v v^H to the trailing columns
      for (int j = k + 1; j < cols; ++j) {
        T* colj = &a[(size_t)j * rows];
        T s = colj[k];
        for (int i = k + 1; i < rows; ++i) s += conjv(colk[i]) * colj[i];
        s *= conjv(tau[k]);
        colj[k] -= s;
        for (int i = k + 1; i < rows; ++i) colj[i] -= s * colk[i];
      }
    }
  }
  // least-squares solution of A x = b (b has `rows` entries, overwritten)
  void solve(T* b, T* x) const {
    for (int k = 0; k < cols; ++k) {
      const T* colk = &a[(size_t)k * rows];
      T s = b[k];
      for (int i = k + 1; i < rows; ++i) s += conjv(colk[i]) * b[i];
      s *= conjv(tau[k]);
      b[k] -= s;
      for (int i = k + 1; i < rows; ++i) b[i] -= s * colk[i];
    }
    for (int k = cols - 1; k >= 0; --k) {
      T s = b[k];
      for (int j = k + 1; j < cols; ++j) s -= a[(size_t)j * rows + k] * x[j];
      x[k] = s / a[(size_t)k * rows + k];
    }
  }
};

// --------------------------------------------------------------------------
// BDIM correction, target === source (src/bdim.jl:50-196 with
// etype_to_nearest_points' X === Y branch, src/quadrature.jl:249-256).
// Elements are contiguous blocks of nq nodes (src/quadrature.jl:160).
// --------------------------------------------------------------------------
template <class T>
static T kval(int pde, int kind, int dim, double k, const double* x, const double* nx,
              const double* y, const double* ny);
template <>
double kval<double>(int pde, int kind, int dim, double k, const double* x, const double* nx,
                    const double* y, const double* ny) {
  (void)pde;
  (void)k;
  return dim == 2 ? laplace_kernel<2>(kind, x, nx, y, ny) : laplace_kernel<3>(kind, x, nx, y, ny);
}
template <>
cd kval<cd>(int pde, int kind, int dim, double k, const double* x, const double* nx,
            const double* y, const double* ny) {
  (void)pde;
  (void)dim;
  return helmholtz3_kernel(kind, k, x, nx, y, ny);
}

template <class T>
static int bdim_impl(int pde, int dim, double k, int64_t n, const double* x, const double* nrm,
                     const double* w, int nq, int derivative, const double* green_mult,
                     int64_t n_sel, const int64_t* sel, T* dS, T* dD, double* theta_out,
                     int nt) {
  const int64_t nel = n / nq;
  // bdim.jl:79-80: ns = ceil(3 * qmax)
  const int ns = (int)std::ceil(3.0 * nq);
  // bdim.jl:82-85: bounding box, centre, radius
  double lc[3] = {INFINITY, INFINITY, INFINITY}, hc[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t j = 0; j < n; ++j)
    for (int c = 0; c < dim; ++c) {
      lc[c] = std::min(lc[c], x[dim * j + c]);
      hc[c] = std::max(hc[c], x[dim * j + c]);
    }
  double xc[3], diag2 = 0.0;
  for (int c = 0; c < dim; ++c) {
    xc[c] = (lc[c] + hc[c]) / 2;
    diag2 += (hc[c] - lc[c]) * (hc[c] - lc[c]);
  }
  const double R = 1.5 * std::sqrt(diag2) / 2;
  std::vector<double> xs((size_t)ns * dim);
  or_dim_sources(dim, ns, R, xc, xs.data());
  // bdim.jl:94-103: traces of the monopoles on the source nodes
  const int kG = derivative ? OR_ADL : OR_SL;  // value kernel at targets
  const int kS = derivative ? OR_ADL : OR_SL;  // "S" operator kernel
  const int kD = derivative ? OR_HS : OR_DL;   // "D" operator kernel
  std::vector<T> g0((size_t)n * ns), g1((size_t)n * ns);
  parallel_for(n, nt, 64, [&](int64_t j) {
    for (int kk = 0; kk < ns; ++kk) {
      g0[(size_t)j * ns + kk] = kval<T>(pde, OR_SL, dim, k, x + dim * j, nrm + dim * j, &xs[dim * kk], nullptr);
      g1[(size_t)j * ns + kk] = kval<T>(pde, OR_ADL, dim, k, x + dim * j, nrm + dim * j, &xs[dim * kk], nullptr);
    }
  });
  // rows needed: every node of the selected elements
  std::vector<int64_t> elems;
  if (sel) elems.assign(sel, sel + n_sel);
  else {
    elems.resize(nel);
    for (int64_t e = 0; e < nel; ++e) elems[e] = e;
  }
  const int64_t nrow = (int64_t)elems.size() * nq;
  std::vector<T> theta((size_t)nrow * ns);
  // bdim.jl:104-118: Theta = mu*B(x) + S*g1 - D*g0, S/D uncorrected Nystrom
  // operators (entries K*w), summed over sources in ascending order.
  parallel_for(nrow, nt, 4, [&](int64_t r) {
    const int64_t i = elems[r / nq] * nq + (r % nq);
    const double* xi = x + dim * i;
    const double* ni = nrm + dim * i;
    const double mu = green_mult ? green_mult[i] : -0.5;
    std::vector<T> acc(ns);
    for (int kk = 0; kk < ns; ++kk) acc[kk] = mu * kval<T>(pde, kG, dim, k, xi, ni, &xs[dim * kk], nullptr);
    std::vector<T> accS(ns, T(0)), accD(ns, T(0));
    for (int64_t j = 0; j < n; ++j) {
      const T s = kval<T>(pde, kS, dim, k, xi, ni, x + dim * j, nrm + dim * j) * w[j];
      const T d = kval<T>(pde, kD, dim, k, xi, ni, x + dim * j, nrm + dim * j) * w[j];
      const T* g1j = &g1[(size_t)j * ns];
      const T* g0j = &g0[(size_t)j * ns];
      for (int kk = 0; kk < ns; ++kk) {
        accS[kk] += s * g1j[kk];
        accD[kk] += d * g0j[kk];
      }
    }
    for (int kk = 0; kk < ns; ++kk) theta[(size_t)r * ns + kk] = (acc[kk] + accS[kk]) - accD[kk];
  });
  if (theta_out) {
    for (size_t q = 0; q < theta.size(); ++q) {
      theta_out[2 * q] = realv(theta[q]);
      theta_out[2 * q + 1] = imagv(theta[q]);
    }
  }
  // bdim.jl:154-185: per element, QR of M^T (ns x 2nq), M = [g0[el,:]; g1[el,:]]
  // and least squares for each of the element's own nodes.
  parallel_for((int64_t)elems.size(), nt, 4, [&](int64_t q) {
    const int64_t e = elems[q];
    HouseholderQR<T> F;
    F.rows = ns;
    F.cols = 2 * nq;
    F.a.assign((size_t)ns * 2 * nq, T(0));
    for (int a = 0; a < nq; ++a) {
      const int64_t j = e * nq + a;
      for (int kk = 0; kk < ns; ++kk) {
        F.a[(size_t)a * ns + kk] = g0[(size_t)j * ns + kk];
        F.a[(size_t)(nq + a) * ns + kk] = g1[(size_t)j * ns + kk];
      }
    }
    F.factor();
    std::vector<T> b(ns), W(2 * nq);
    for (int t = 0; t < nq; ++t) {
      const int64_t r = q * nq + t;
      for (int kk = 0; kk < ns; ++kk) b[kk] = theta[(size_t)r * ns + kk];
      F.solve(b.data(), W.data());
      for (int a = 0; a < nq; ++a) {
        dS[(size_t)r * nq + a] = -W[nq + a];  // bdim.jl:178
        dD[(size_t)r * nq + a] = W[a];        // bdim.jl:179
      }
    }
  });
  return 0;
}

// --------------------------------------------------------------------------
// BDIM correction with targets other than the source nodes (src/api.jl:105-148
// with bdim.jl:50-196; the near list of etype_to_nearest_points,
// src/quadrature.jl:264-286).  Each target goes to the element of its nearest
// source node (KDTree nn in the reference; here an exhaustive search with
// squared distances ((dx*dx + dy*dy) + dz*dz), ties to the lowest index) when
// that distance is <= maxdist.  Theta uses the uncorrected operators from the
// near targets to all source nodes; each element with near targets is
// factored once and solved for every one of them.
// --------------------------------------------------------------------------
template <class T>
static int bdim_targets_impl(int pde, int dim, double k, int64_t m, const double* tx, const double* tn,
                             int64_t n, const double* x, const double* nrm, const double* w, int nq,
                             int derivative, const double* green_mult, double maxdist,
                             int64_t* near_elem, T* dS, T* dD, double* theta_out, int nt) {
  const int ns = (int)std::ceil(3.0 * nq);
  double lc[3] = {INFINITY, INFINITY, INFINITY}, hc[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t j = 0; j < n; ++j)
    for (int c = 0; c < dim; ++c) {
      lc[c] = std::min(lc[c], x[dim * j + c]);
      hc[c] = std::max(hc[c], x[dim * j + c]);
    }
  double xc[3], diag2 = 0.0;
  for (int c = 0; c < dim; ++c) {
    xc[c] = (lc[c] + hc[c]) / 2;
    diag2 += (hc[c] - lc[c]) * (hc[c] - lc[c]);
  }
  const double R = 1.5 * std::sqrt(diag2) / 2;
  std::vector<double> xs((size_t)ns * dim);
  or_dim_sources(dim, ns, R, xc, xs.data());
  const int kG = derivative ? OR_ADL : OR_SL;
  const int kS = derivative ? OR_ADL : OR_SL;
  const int kD = derivative ? OR_HS : OR_DL;
  std::vector<T> g0((size_t)n * ns), g1((size_t)n * ns);
  parallel_for(n, nt, 64, [&](int64_t j) {
    for (int kk = 0; kk < ns; ++kk) {
      g0[(size_t)j * ns + kk] = kval<T>(pde, OR_SL, dim, k, x + dim * j, nrm + dim * j, &xs[dim * kk], nullptr);
      g1[(size_t)j * ns + kk] = kval<T>(pde, OR_ADL, dim, k, x + dim * j, nrm + dim * j, &xs[dim * kk], nullptr);
    }
  });
  // near lists (quadrature.jl:264-286)
  parallel_for(m, nt, 16, [&](int64_t i) {
    double best = INFINITY;
    int64_t bj = -1;
    for (int64_t j = 0; j < n; ++j) {
      double d2 = 0.0;
      for (int c = 0; c < dim; ++c) {
        const double dc = tx[dim * i + c] - x[dim * j + c];
        d2 = c == 0 ? dc * dc : d2 + dc * dc;
      }
      if (d2 < best) {
        best = d2;
        bj = j;
      }
    }
    near_elem[i] = (bj >= 0 && !(std::sqrt(best) > maxdist)) ? bj / nq : -1;
  });
  std::vector<std::vector<int64_t>> elem_targets((size_t)(n / nq));
  for (int64_t i = 0; i < m; ++i)
    if (near_elem[i] >= 0) elem_targets[(size_t)near_elem[i]].push_back(i);
  // Theta rows of the near targets (bdim.jl:104-118)
  std::vector<T> theta((size_t)m * ns, T(0));
  parallel_for(m, nt, 2, [&](int64_t i) {
    if (near_elem[i] < 0) return;
    const double* xi = tx + dim * i;
    const double* ni = tn ? tn + dim * i : nullptr;
    const double mu = green_mult[i];
    std::vector<T> acc(ns), accS(ns, T(0)), accD(ns, T(0));
    for (int kk = 0; kk < ns; ++kk) acc[kk] = mu * kval<T>(pde, kG, dim, k, xi, ni, &xs[dim * kk], nullptr);
    for (int64_t j = 0; j < n; ++j) {
      const T sv = kval<T>(pde, kS, dim, k, xi, ni, x + dim * j, nrm + dim * j) * w[j];
      const T dv = kval<T>(pde, kD, dim, k, xi, ni, x + dim * j, nrm + dim * j) * w[j];
      const T* g1j = &g1[(size_t)j * ns];
      const T* g0j = &g0[(size_t)j * ns];
      for (int kk = 0; kk < ns; ++kk) {
        accS[kk] += sv * g1j[kk];
        accD[kk] += dv * g0j[kk];
      }
    }
    for (int kk = 0; kk < ns; ++kk) theta[(size_t)i * ns + kk] = (acc[kk] + accS[kk]) - accD[kk];
  });
  if (theta_out)
    for (size_t q = 0; q < theta.size(); ++q) {
      theta_out[2 * q] = realv(theta[q]);
      theta_out[2 * q + 1] = imagv(theta[q]);
    }
  // per element: factor once, solve for each near target (bdim.jl:154-185)
  parallel_for(n / nq, nt, 4, [&](int64_t e) {
    const auto& targets = elem_targets[(size_t)e];
    if (targets.empty()) return;
    HouseholderQR<T> F;
    F.rows = ns;
    F.cols = 2 * nq;
    F.a.assign((size_t)ns * 2 * nq, T(0));
    for (int a = 0; a < nq; ++a) {
      const int64_t j = e * nq + a;
      for (int kk = 0; kk < ns; ++kk) {
        F.a[(size_t)a * ns + kk] = g0[(size_t)j * ns + kk];
        F.a[(size_t)(nq + a) * ns + kk] = g1[(size_t)j * ns + kk];
      }
    }
    F.factor();
    std::vector<T> b(ns), W(2 * nq);
    for (int64_t i : targets) {
      for (int kk = 0; kk < ns; ++kk) b[kk] = theta[(size_t)i * ns + kk];
      F.solve(b.data(), W.data());
      for (int a = 0; a < nq; ++a) {
        dS[(size_t)i * nq + a] = -W[nq + a];
        dD[(size_t)i * nq + a] = W[a];
      }
    }
  });
  return 0;
}

extern "C" {

// Off-surface DIM: near_elem[i] = element of target i's nearest source node
// (-1 if beyond maxdist); row i of dS/dD (m x nq, interleaved complex for
// Helmholtz) holds the corrections to source nodes near_elem*nq + a.
// tn (target normals) is needed when derivative != 0.
int or_bdim_targets(int pde, int dim, double k, int64_t m, const double* tx, const double* tn, int64_t n,
                    const double* x, const double* nrm, const double* w, int nq, int derivative,
                    const double* green_mult, double maxdist, int64_t* near_elem, double* dS, double* dD,
                    double* theta_out, int nthreads) {
  if (n % nq) return 2;
  if (derivative && !tn) return 3;
  if (pde == OR_LAPLACE)
    return bdim_targets_impl<double>(pde, dim, k, m, tx, tn, n, x, nrm, w, nq, derivative, green_mult, maxdist,
                                     near_elem, dS, dD, theta_out, nthreads);
  if (dim != 3) return 1;
  return bdim_targets_impl<cd>(pde, dim, k, m, tx, tn, n, x, nrm, w, nq, derivative, green_mult, maxdist,
                               near_elem, reinterpret_cast<cd*>(dS), reinterpret_cast<cd*>(dD), theta_out,
                               nthreads);
}

}  // extern "C"

extern "C" {

// Block values of the DIM correction for the selected elements (all when
// sel == NULL).  For selected element e (position q in the selection) and its
// local target t, values for source node e*nq + a are at [(q*nq + t)*nq + a].
// Laplace: real; Helmholtz: interleaved complex.  theta_out (nullable) gets the
// Theta rows (complex interleaved, nrow x ns).
int or_bdim(int pde, int dim, double k, int64_t n, const double* x, const double* nrm,
            const double* w, int nq, int derivative, const double* green_mult, int64_t n_sel,
            const int64_t* sel, double* dS, double* dD, double* theta_out, int nthreads) {
  if (n % nq) return 2;
  if (pde == OR_LAPLACE)
    return bdim_impl<double>(pde, dim, k, n, x, nrm, w, nq, derivative, green_mult, n_sel, sel,
                             dS, dD, theta_out, nthreads);
  if (dim != 3) return 1;
  return bdim_impl<cd>(pde, dim, k, n, x, nrm, w, nq, derivative, green_mult, n_sel, sel,
                       reinterpret_cast<cd*>(dS), reinterpret_cast<cd*>(dD), theta_out, nthreads);
}

// Per-node monopole traces of the DIM construction (src/bdim.jl:94-103):
// g0[j, k] = G(y_j, xs_k), g1[j, k] = ADL(y_j, xs_k), interleaved complex,
// n x ns row-major; used by the tests to form each element's least-squares
// matrix and its condition number.
int or_dim_traces(int pde, int dim, double k, int64_t n, const double* x, const double* nrm,
                  int nq, double* g0, double* g1) {
  const int ns = (int)std::ceil(3.0 * nq);
  double lc[3] = {INFINITY, INFINITY, INFINITY}, hc[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t j = 0; j < n; ++j)
    for (int c = 0; c < dim; ++c) {
      lc[c] = std::min(lc[c], x[dim * j + c]);
      hc[c] = std::max(hc[c], x[dim * j + c]);
    }
  double xc[3], diag2 = 0.0;
  for (int c = 0; c < dim; ++c) {
    xc[c] = (lc[c] + hc[c]) / 2;
    diag2 += (hc[c] - lc[c]) * (hc[c] - lc[c]);
  }
  std::vector<double> xs((size_t)ns * dim);
  or_dim_sources(dim, ns, 1.5 * std::sqrt(diag2) / 2, xc, xs.data());
  for (int64_t j = 0; j < n; ++j)
    for (int kk = 0; kk < ns; ++kk) {
      const cd a = eval_kernel(pde, OR_SL, dim, k, x + dim * j, nrm + dim * j, &xs[dim * kk], nullptr);
      const cd b = eval_kernel(pde, OR_ADL, dim, k, x + dim * j, nrm + dim * j, &xs[dim * kk], nullptr);
      g0[2 * (j * ns + kk)] = a.real();
      g0[2 * (j * ns + kk) + 1] = a.imag();
      g1[2 * (j * ns + kk)] = b.real();
      g1[2 * (j * ns + kk) + 1] = b.imag();
    }
  return ns;
}

}  // extern "C"

// --------------------------------------------------------------------------
// Restarted GMRES(m) with modified Gram-Schmidt and Givens rotations
// (Saad & Schultz 1986), FP64, for L = shift*I + sum_t coef_t*(A_t + C_t)
// where A_t is the on-the-fly Nystrom operator and C_t an optional CSR
// correction.  Restates the external IterativeSolvers.gmres driver the
// reference docs call (docs/src/examples/poisson.jl:166-168,
// helmholtz_scattering.jl:494-495).  Stops when ||b - Lx|| <= rtol*||b||.
// --------------------------------------------------------------------------
struct OrTerm {
  int kind;
  double coef_re, coef_im;
  int64_t nnz;
  const int64_t* rowptr;
  const int32_t* col;
  const double* val;
};

static void apply_L(int pde, int dim, double k, int64_t n, const double* x, const double* nrm,
                    const double* w, double shift_re, double shift_im, int nterms,
                    const OrTerm* terms, const cd* v, cd* out, int nt) {
  const bool cplx = pde == OR_HELMHOLTZ;
  std::vector<double> vin(cplx ? 2 * n : n), tmp(cplx ? 2 * n : n);
  for (int64_t i = 0; i < n; ++i) {
    if (cplx) {
      vin[2 * i] = v[i].real();
      vin[2 * i + 1] = v[i].imag();
    } else {
      vin[i] = v[i].real();
    }
    out[i] = cd(shift_re, shift_im) * v[i];
  }
  for (int t = 0; t < nterms; ++t) {
    or_apply(pde, terms[t].kind, dim, k, 0, n, x, nrm, n, x, nrm, w, vin.data(), tmp.data(), nt);
    if (terms[t].rowptr) or_csr_apply(n, terms[t].rowptr, terms[t].col, terms[t].val, cplx, vin.data(), tmp.data());
    const cd c(terms[t].coef_re, terms[t].coef_im);
    for (int64_t i = 0; i < n; ++i) out[i] += c * (cplx ? cd(tmp[2 * i], tmp[2 * i + 1]) : cd(tmp[i], 0.0));
  }
}

static double nrm2(const std::vector<cd>& v) {
  double s = 0;
  for (auto& z : v) s += std::norm(z);
  return std::sqrt(s);
}

extern "C" {

// Real problems pass real b/x when pde == Laplace and all coefficients real;
// otherwise b/x are interleaved complex.  history (nullable, maxiter+1 long)
// receives relative residual estimates.  Returns iterations used, or -1.
int or_gmres(int pde, int dim, double k, int64_t n, const double* x, const double* nrm,
             const double* w, double shift_re, double shift_im, int nterms, const int* kinds,
             const double* coefs, const int64_t* const* rowptrs, const int32_t* const* cols,
             const double* const* vals, const double* b, double* sol, double rtol, int restart,
             int maxiter, int is_complex, double* history, double* final_relres, int nt) {
  std::vector<OrTerm> terms(nterms);
  for (int t = 0; t < nterms; ++t)
    terms[t] = {kinds[t], coefs[2 * t], coefs[2 * t + 1], 0, rowptrs ? rowptrs[t] : nullptr,
                cols ? cols[t] : nullptr, vals ? vals[t] : nullptr};
  std::vector<cd> bb(n), xx(n, cd(0, 0)), r(n), tmp(n);
  for (int64_t i = 0; i < n; ++i) bb[i] = is_complex ? cd(b[2 * i], b[2 * i + 1]) : cd(b[i], 0);
  const double bn = nrm2(bb);
  int it = 0;
  std::vector<std::vector<cd>> V;
  double rel = 1.0;
  if (history) history[0] = 1.0;
  while (it < maxiter) {
    apply_L(pde, dim, k, n, x, nrm, w, shift_re, shift_im, nterms, terms.data(), xx.data(), tmp.data(), nt);
    for (int64_t i = 0; i < n; ++i) r[i] = bb[i] - tmp[i];
    double beta = nrm2(r);
    rel = beta / bn;
    if (rel <= rtol) break;
    const int m = restart;
    V.assign(1, std::vector<cd>(n));
    for (int64_t i = 0; i < n; ++i) V[0][i] = r[i] / beta;
    std::vector<cd> H((size_t)(m + 1) * m, cd(0, 0)), cs(m), sn(m), g(m + 1, cd(0, 0));
    g[0] = beta;
    int j = 0;
    for (; j < m && it < maxiter; ++j) {
      std::vector<cd> wv(n);
      apply_L(pde, dim, k, n, x, nrm, w, shift_re, shift_im, nterms, terms.data(), V[j].data(), wv.data(), nt);
      for (int i = 0; i <= j; ++i) {
        cd h(0, 0);
        for (int64_t q = 0; q < n; ++q) h += std::conj(V[i][q]) * wv[q];
        H[(size_t)i * m + j] = h;
        for (int64_t q = 0; q < n; ++q) wv[q] -= h * V[i][q];
      }
      const double hn = nrm2(wv);
      H[(size_t)(j + 1) * m + j] = hn;
      for (int i = 0; i < j; ++i) {  // previous rotations
        const cd a = H[(size_t)i * m + j], bq = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = std::conj(cs[i]) * a + std::conj(sn[i]) * bq;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * bq;
      }
      const cd a = H[(size_t)j * m + j], bq = H[(size_t)(j + 1) * m + j];
      const double den = std::sqrt(std::norm(a) + std::norm(bq));
      cs[j] = den == 0 ? cd(1, 0) : a / den;
      sn[j] = den == 0 ? cd(0, 0) : bq / den;
      H[(size_t)j * m + j] = den;
      H[(size_t)(j + 1) * m + j] = 0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = std::conj(cs[j]) * g[j];
      ++it;
      rel = std::abs(g[j + 1]) / bn;
      if (history) history[it] = rel;
      if (rel <= rtol || hn == 0.0) {
        ++j;
        break;
      }
      V.emplace_back(n);
      for (int64_t q = 0; q < n; ++q) V[j + 1][q] = wv[q] / hn;
    }
    // back-substitution and update
    std::vector<cd> yv(j);
    for (int i = j - 1; i >= 0; --i) {
      cd s = g[i];
      for (int q = i + 1; q < j; ++q) s -= H[(size_t)i * m + q] * yv[q];
      yv[i] = s / H[(size_t)i * m + i];
    }
    for (int i = 0; i < j; ++i)
      for (int64_t q = 0; q < n; ++q) xx[q] += yv[i] * V[i][q];
  }
  apply_L(pde, dim, k, n, x, nrm, w, shift_re, shift_im, nterms, terms.data(), xx.data(), tmp.data(), nt);
  for (int64_t i = 0; i < n; ++i) r[i] = bb[i] - tmp[i];
  rel = nrm2(r) / bn;
  if (final_relres) *final_relres = rel;
  for (int64_t i = 0; i < n; ++i) {
    if (is_complex) {
      sol[2 * i] = xx[i].real();
      sol[2 * i + 1] = xx[i].imag();
    } else {
      sol[i] = xx[i].real();
    }
  }
  return it;
}

}  // extern "C"

// --------------------------------------------------------------------------
// Forward-mode (dual number) derivative of the Laplace 3D double-layer
// potential u_i = sum_j DL(x_i; y_j, n_j) w_j sigma_j (src/nystrom.jl:31-38)
// along a perturbation (dy, dn, dw, dsigma) of the source data: the method
// ForwardDiff applies (Project.toml:9, used at
// src/reference_interpolation.jl:36-38), restated with a two-component dual.
// --------------------------------------------------------------------------
struct Dual {
  double v, d;
};
static inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
static inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
static inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
static inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
static inline Dual dsqrt(Dual a) {
  const double s = std::sqrt(a.v);
  return {s, a.d / (2 * s)};
}

extern "C" {

void or_dl_potential_jvp(int64_t m, const double* tx, int64_t n, const double* sx,
                         const double* sn, const double* sw, const double* sigma,
                         const double* dsx, const double* dsn, const double* dsw,
                         const double* dsigma, double* u, double* du, int nt) {
  parallel_for(m, nt, 16, [&](int64_t i) {
    Dual acc{0, 0};
    for (int64_t j = 0; j < n; ++j) {
      Dual r[3], ny[3];
      for (int c = 0; c < 3; ++c) {
        r[c] = Dual{tx[3 * i + c], 0.0} - Dual{sx[3 * j + c], dsx ? dsx[3 * j + c] : 0.0};
        ny[c] = Dual{sn[3 * j + c], dsn ? dsn[3 * j + c] : 0.0};
      }
      const Dual d = dsqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      if (d.v <= SAME_POINT_TOLERANCE) continue;
      const Dual rn = r[0] * ny[0] + r[1] * ny[1] + r[2] * ny[2];
      const Dual kij = Dual{1.0 / (4 * PI), 0.0} / (d * d * d) * rn;
      acc = acc + kij * Dual{sw[j], dsw ? dsw[j] : 0.0} * Dual{sigma[j], dsigma ? dsigma[j] : 0.0};
    }
    u[i] = acc.v;
    du[i] = acc.d;
  });
}

}  // extern "C"
