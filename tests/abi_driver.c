/* Drives libinti_b200 through its C ABI the way a foreign-function caller
 * (Julia's ccall, a Fortran or C host) does: plain host arrays, a 1-based
 * CSC correction, interleaved complex doubles, status codes and
 * inti_last_error.  Checks the products against direct double loops here.
 *
 *   case 1: 2D Laplace double layer on a circle (src/kernels.jl:153-168)
 *           plus a correction given as 1-based CSC arrays, 3 columns with a
 *           padded leading dimension, alpha = 2, beta = 0.5;
 *   case 2: 3D Helmholtz single layer (k = 2) from points on a sphere to
 *           points off it (src/kernels.jl:347-356), complex alpha/beta;
 *   case 3: a mismatched leading dimension is refused with INTI_E_SHAPE and
 *           a message.
 *
 * Exit status: 0 pass, 77 no CUDA device (nothing else checked), 1 fail. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "inti_b200.h"

#define PI 3.14159265358979323846
#define CHECK(call)                                                                   \
  do {                                                                                \
    int st_ = (call);                                                                 \
    if (st_ != INTI_OK) {                                                             \
      fprintf(stderr, "%s failed: %d (%s)\n", #call, st_, inti_last_error(ctx));      \
      return 1;                                                                       \
    }                                                                                 \
  } while (0)

static double relerr(const double* a, const double* b, long n) {
  double num = 0.0, den = 0.0;
  for (long i = 0; i < n; ++i) {
    num += (a[i] - b[i]) * (a[i] - b[i]);
    den += b[i] * b[i];
  }
  return sqrt(num / (den > 0 ? den : 1.0));
}

static int laplace2d_case(inti_ctx* ctx) {
  const int n = 400, nrhs = 3, ldx = n + 2;
  double *X = malloc(sizeof(double) * 2 * n), *N = malloc(sizeof(double) * 2 * n), *W = malloc(sizeof(double) * n);
  for (int j = 0; j < n; ++j) {
    const double t = 2 * PI * j / n;
    X[2 * j] = cos(t) + 0.3 * cos(2 * t);
    X[2 * j + 1] = sin(t);
    const double tx = -sin(t) - 0.6 * sin(2 * t), ty = cos(t), s = sqrt(tx * tx + ty * ty);
    N[2 * j] = ty / s;
    N[2 * j + 1] = -tx / s;
    W[j] = s * 2 * PI / n;
  }
  /* correction C: C_jj = 0.5, C_{j+1,j} = 0.1 (column j), 1-based CSC */
  const long nnz = 2 * n - 1;
  int64_t* colptr = malloc(sizeof(int64_t) * (n + 1));
  int64_t* rowval = malloc(sizeof(int64_t) * nnz);
  double* nzval = malloc(sizeof(double) * nnz);
  long p = 0;
  for (int j = 0; j < n; ++j) {
    colptr[j] = p + 1;
    rowval[p] = j + 1;
    nzval[p++] = 0.5;
    if (j + 1 < n) {
      rowval[p] = j + 2;
      nzval[p++] = 0.1;
    }
  }
  colptr[n] = p + 1;
  inti_quad* q = NULL;
  inti_csr* c = NULL;
  inti_op* op = NULL;
  CHECK(inti_quad_create(ctx, 2, n, X, N, W, 0, &q));
  CHECK(inti_csr_create_from_csc(ctx, n, n, nnz, colptr, rowval, nzval, INTI_F64, &c));
  CHECK(inti_op_create(ctx, INTI_LAPLACE, INTI_DL, 0.0, 0.0, q, q, c, INTI_FP64, &op));
  double *x = malloc(sizeof(double) * ldx * nrhs), *y = malloc(sizeof(double) * ldx * nrhs),
         *ref = malloc(sizeof(double) * n * nrhs), *got = malloc(sizeof(double) * n * nrhs);
  for (int r = 0; r < nrhs; ++r)
    for (int j = 0; j < ldx; ++j) {
      x[r * ldx + j] = cos(0.37 * j + r) + 0.1 * r;
      y[r * ldx + j] = sin(0.11 * j - r);
    }
  const double alpha[2] = {2.0, 0.0}, beta[2] = {0.5, 0.0};
  for (int r = 0; r < nrhs; ++r)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = 0; j < n; ++j) {
        const double r0 = X[2 * i] - X[2 * j], r1 = X[2 * i + 1] - X[2 * j + 1], d2 = r0 * r0 + r1 * r1;
        if (sqrt(d2) <= 1e-14) continue;
        s += (r0 * N[2 * j] + r1 * N[2 * j + 1]) / (2 * PI * d2) * W[j] * x[r * ldx + j];
      }
      s += 0.5 * x[r * ldx + i] + (i > 0 ? 0.1 * x[r * ldx + i - 1] : 0.0);
      ref[r * n + i] = 2.0 * s + 0.5 * y[r * ldx + i];
    }
  CHECK(inti_op_apply(op, x, ldx, y, ldx, nrhs, alpha, beta, 0));
  for (int r = 0; r < nrhs; ++r) memcpy(got + r * n, y + r * ldx, sizeof(double) * n);
  const double e = relerr(got, ref, (long)n * nrhs);
  printf("laplace2d DL + CSC correction, 3 columns: relerr %.3e\n", e);
  int fail = !(e < 1e-12);
  for (int r = 0; r < nrhs; ++r) /* rows past n untouched */
    for (int j = n; j < ldx; ++j)
      if (y[r * ldx + j] != sin(0.11 * j - r)) fail = 1;
  /* case 3: leading dimension smaller than the vector length */
  const int st = inti_op_apply(op, x, n - 1, y, ldx, 1, alpha, beta, 0);
  const char* msg = inti_last_error(ctx);
  printf("ldx < n: status %d, message \"%s\"\n", st, msg ? msg : "");
  if (st != INTI_E_SHAPE || !msg || !msg[0]) fail = 1;
  CHECK(inti_op_destroy(op));
  CHECK(inti_csr_destroy(c));
  CHECK(inti_quad_destroy(q));
  free(X), free(N), free(W), free(colptr), free(rowval), free(nzval), free(x), free(y), free(ref), free(got);
  return fail;
}

static int helmholtz3d_case(inti_ctx* ctx) {
  const int n = 600, m = 300;
  const double k = 2.0, ga = PI * (3.0 - sqrt(5.0));
  double *Y = malloc(sizeof(double) * 3 * n), *W = malloc(sizeof(double) * n), *T = malloc(sizeof(double) * 3 * m);
  for (int j = 0; j < n; ++j) { /* Fibonacci points on the unit sphere */
    const double z = 1.0 - (2.0 * j + 1.0) / n, r = sqrt(1.0 - z * z), ph = ga * j;
    Y[3 * j] = r * cos(ph);
    Y[3 * j + 1] = r * sin(ph);
    Y[3 * j + 2] = z;
    W[j] = 4 * PI / n;
  }
  for (int i = 0; i < m; ++i) {
    const double z = 1.0 - (2.0 * i + 1.0) / m, r = sqrt(1.0 - z * z), ph = 0.7 + ga * i;
    T[3 * i] = 1.7 * r * cos(ph);
    T[3 * i + 1] = 1.7 * r * sin(ph);
    T[3 * i + 2] = 1.7 * z;
  }
  inti_quad *qs = NULL, *qt = NULL;
  inti_op* op = NULL;
  CHECK(inti_quad_create(ctx, 3, n, Y, NULL, W, 0, &qs));
  CHECK(inti_quad_create(ctx, 3, m, T, NULL, NULL, 0, &qt));
  CHECK(inti_op_create(ctx, INTI_HELMHOLTZ, INTI_SL, k, 0.0, qt, qs, NULL, INTI_FP64, &op));
  double *x = malloc(sizeof(double) * 2 * n), *y = malloc(sizeof(double) * 2 * m), *ref = malloc(sizeof(double) * 2 * m);
  for (int j = 0; j < n; ++j) {
    x[2 * j] = cos(0.2 * j);
    x[2 * j + 1] = sin(0.05 * j);
  }
  for (int i = 0; i < m; ++i) {
    y[2 * i] = 0.3 * i / m;
    y[2 * i + 1] = -0.1;
  }
  const double alpha[2] = {0.5, -1.0}, beta[2] = {0.0, 2.0};
  for (int i = 0; i < m; ++i) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < n; ++j) {
      const double r0 = T[3 * i] - Y[3 * j], r1 = T[3 * i + 1] - Y[3 * j + 1], r2 = T[3 * i + 2] - Y[3 * j + 2];
      const double d = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
      const double gr = cos(k * d) / (4 * PI * d) * W[j], gi = sin(k * d) / (4 * PI * d) * W[j];
      sr += gr * x[2 * j] - gi * x[2 * j + 1];
      si += gr * x[2 * j + 1] + gi * x[2 * j];
    }
    const double yr = y[2 * i], yi = y[2 * i + 1];
    ref[2 * i] = alpha[0] * sr - alpha[1] * si + beta[0] * yr - beta[1] * yi;
    ref[2 * i + 1] = alpha[0] * si + alpha[1] * sr + beta[0] * yi + beta[1] * yr;
  }
  CHECK(inti_op_apply(op, x, n, y, m, 1, alpha, beta, 0));
  const double e = relerr(y, ref, 2L * m);
  printf("helmholtz3d SL off-surface, complex alpha/beta: relerr %.3e\n", e);
  CHECK(inti_op_destroy(op));
  CHECK(inti_quad_destroy(qt));
  CHECK(inti_quad_destroy(qs));
  free(Y), free(W), free(T), free(x), free(y), free(ref);
  return !(e < 1e-12);
}

int main(void) {
  inti_ctx* ctx = NULL;
  printf("libinti_b200 ABI version %d\n", inti_version());
  const int st = inti_ctx_create(0, NULL, &ctx);
  if (st != INTI_OK) {
    const char* msg = inti_last_error(NULL);
    printf("no context (status %d): %s\n", st, msg ? msg : "");
    return st == INTI_E_CUDA ? 77 : 1;
  }
  int fail = laplace2d_case(ctx);
  fail |= helmholtz3d_case(ctx);
  if (inti_ctx_destroy(ctx) != INTI_OK) fail = 1;
  printf(fail ? "FAIL\n" : "PASS\n");
  return fail;
}
