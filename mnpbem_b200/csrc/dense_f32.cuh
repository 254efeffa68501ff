// FP32 planar-complex batched dense building blocks (see dense_f32.cu).
#pragma once
#include "common.cuh"
#include "tc_gemm.cuh"

namespace mnpb {
namespace f32 {

// Launch context: stream, batch count and the tensor-core GEMM workspace.
struct Ctx {
    cudaStream_t s;
    int batch;
    float *work;
    int64_t work_bytes;
    Ctx(cudaStream_t s_, int batch_, float *work_, int64_t work_bytes_);
};

// round_out / a_tf32: see tc::cgemm_tf32 (store C as TF32; A holds TF32 values).
int gemm(Ctx &c, int m, int n, int k, float alpha, tc::CMatF A, tc::CMatF B, float beta,
         tc::CMatF C, bool round_out = false, bool a_tf32 = false);
int trsm_llu(Ctx &c, int n, int m, tc::CMatF L, tc::CMatF B);
int trsm_lun(Ctx &c, int n, int m, tc::CMatF U, tc::CMatF B);
int trsm_run(Ctx &c, int n, int m, tc::CMatF U, tc::CMatF B);
int trsm_rlu(Ctx &c, int n, int m, tc::CMatF L, tc::CMatF B);
int laswp(Ctx &c, tc::CMatF A, int j0, int j1, const int32_t *ipiv, int64_t sP, int c0, int c1,
          bool forward);
int getrf(Ctx &c, int n, tc::CMatF A, int32_t *ipiv, int64_t sP, int32_t *info);
int getrs(Ctx &c, int n, int nrhs, tc::CMatF LU, const int32_t *ipiv, int64_t sP, tc::CMatF B);
int right_solve(Ctx &c, int n, int m, tc::CMatF LU, const int32_t *ipiv, int64_t sP, tc::CMatF B);
int set_identity(Ctx &c, int n, tc::CMatF W);
// X <- A^-1 from the LU factorisation of A (getrf output and pivots), the
// forward solve exploiting the identity's zero upper part.
int lu_inverse(Ctx &c, int n, tc::CMatF LU, const int32_t *ipiv, int64_t sP, tc::CMatF X);

// Inverses of the 32 x 32 diagonal blocks of an LU factor (for getrs_few).
int64_t diag_inv_floats(int n, int batch);
int diag_inv(Ctx &c, int n, tc::CMatF LU, float *invL, float *invU);
// LU solve for m <= 16 right-hand sides: row swaps + one launch per triangle.
// state: device scratch of trsv_state_bytes(n, batch) bytes (per stream).
int64_t trsv_state_bytes(int n, int batch);
int getrs_few(Ctx &c, int n, int m, tc::CMatF LU, const int32_t *ipiv, int64_t sP,
              const float *invL, const float *invU, tc::CMatF B, int *state);
int trsv_error_read_and_clear(cudaStream_t s, int *code);
// One-thread kernel whose wait (kind 1: flag spin, kind 2: mbarrier) of the
// triangular solves can only time out after limit_ns; records code 9.
int trsv_wait_probe(cudaStream_t s, int kind, int *flag, uint64_t limit_ns);

}  // namespace f32
}  // namespace mnpb
