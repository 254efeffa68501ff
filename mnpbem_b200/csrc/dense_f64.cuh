// FP64 batched dense building blocks (see dense_f64.cu).
#pragma once
#include "common.cuh"

namespace mnpb {

int zgemm(cudaStream_t s, int m, int n, int k, int batch, cd alpha, const cd *A, int64_t lda,
          int64_t sA, const cd *B, int64_t ldb, int64_t sB, cd beta, cd *C, int64_t ldc,
          int64_t sC);
int trsm_llu(cudaStream_t s, int n, int m, int batch, const cd *L, int64_t ldl, int64_t sL,
             cd *B, int64_t ldb, int64_t sB);
int trsm_lun(cudaStream_t s, int n, int m, int batch, const cd *U, int64_t ldu, int64_t sU,
             cd *B, int64_t ldb, int64_t sB);
int trsm_run(cudaStream_t s, int n, int m, int batch, const cd *U, int64_t ldu, int64_t sU,
             cd *B, int64_t ldb, int64_t sB);
int trsm_rlu(cudaStream_t s, int n, int m, int batch, const cd *L, int64_t ldl, int64_t sL,
             cd *B, int64_t ldb, int64_t sB);
int laswp(cudaStream_t s, cd *A, int64_t lda, int64_t sA, int ncols, int jskip0, int jskip1,
          const int32_t *ipiv, int64_t sP, int c0, int c1, bool forward, int batch);
int getrf(cudaStream_t s, int n, int batch, cd *A, int64_t lda, int64_t sA, int32_t *ipiv,
          int64_t sP, int32_t *info);
int getrs(cudaStream_t s, int n, int nrhs, int batch, const cd *LU, int64_t lda, int64_t sA,
          const int32_t *ipiv, int64_t sP, cd *B, int64_t ldb, int64_t sB);
int right_solve(cudaStream_t s, int n, int m, int batch, const cd *LU, int64_t lda, int64_t sA,
                const int32_t *ipiv, int64_t sP, cd *B, int64_t ldb, int64_t sB);
int set_identity(cudaStream_t s, int n, int batch, cd *W, int64_t ldw, int64_t sW);

}  // namespace mnpb
