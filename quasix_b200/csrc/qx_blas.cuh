// Generic FP64 helpers built on the DMMA mainloop (k_blas.cu).
#pragma once
#include "qx_internal.cuh"

namespace qx {

// C[b][m][n] = alpha * sum_k A[b][m][k] B[b][n][k] + beta * C[b][m][n]
// (row-major, K contiguous in A and B; leading dimensions and batch strides
// in elements, lda/ldb even, A/B 16-byte aligned).  splitk = 0 picks a split
// that fills the GPU.
struct GemmNT {
  int M, N, K;
  const double* A;
  int lda;
  size_t sA;
  const double* B;
  int ldb;
  size_t sB;
  double* C;
  int ldc;
  size_t sC;
  int batch;
  double alpha, beta;
  int splitk;
};
void gemm_nt_f64(qx_ctx* ctx, GemmNT g);

// out[r][k] = alpha * sum_i coef[i * ldc + r] V[i][k] + beta * out[r][k]
void combine_rows(qx_ctx* ctx, const double* V, int ldv, int nv, const double* coef, int ldc, int nr, int n,
                  double* out, int ldo, double alpha, double beta);

// Symmetric eigen-decomposition of A (n x n, lda), one CTA: eigenvalues
// ascending in w, eigenvectors as the columns of Z (ldz).  V is scratch
// (n x lda).  info[0] receives the number of sweeps.
void jacobi_eigh(qx_ctx* ctx, double* A, double* V, int n, int lda, double* w, double* Z, int ldz, int* info);

// Lowest k eigenpairs of the symmetric part of A (n x n, lda), one CTA:
// eigenvalues ascending in w[0..k), eigenvectors as the first k columns of Z
// (ldz).  work: eigh_lowest_work_doubles(n, k) doubles; iwork: k * n ints.
size_t eigh_lowest_work_doubles(int n, int k);
void eigh_lowest(qx_ctx* ctx, const double* A, int n, int lda, int k, double* w, double* Z, int ldz, double* work,
                 int* iwork);

// out[b][c][r] = in[b][r][c] (rows x cols per batch), through 32x32 smem tiles.
void transpose(qx_ctx* ctx, const double* in, int rows, int cols, int ldi, size_t si, double* out, int ldo, size_t so,
               int batch);

}  // namespace qx
