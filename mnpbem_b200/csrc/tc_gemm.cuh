// Tensor-core complex GEMM (tcgen05, TF32 inputs, FP32 accumulation).
#pragma once
#include "common.cuh"

namespace mnpb {
namespace tc {

// Planar complex FP32 matrix view: real plane at p, imaginary plane at
// p + plane, column-major with leading dimension ld, batch stride `stride`.
struct CMatF {
    float *p;
    int64_t ld, plane, stride;
    __host__ __device__ CMatF sub(int64_t r, int64_t c) const {
        return CMatF{p + c * ld + r, ld, plane, stride};
    }
};

int64_t cgemm_tf32_workspace(int M, int K, int batch);
// C = beta C + alpha A B (A: M x K, B: K x N, C: M x N), work >= cgemm_tf32_workspace.
// round_out: store C rounded to nearest TF32 (values that later GEMMs read as
// operands then reach the tensor cores unchanged).
// a_tf32: the caller guarantees every element of A is a TF32 value (low 13
// mantissa bits zero); A is then read in place by the tensor cores (MN-major
// TMA loads) instead of being packed, when it is 16-byte aligned.  Without
// that guarantee A is packed with round-to-nearest conversion.
int cgemm_tf32(cudaStream_t s, int M, int N, int K, int batch, float alpha, CMatF A, CMatF B,
               float beta, CMatF C, float *work, int64_t work_bytes, bool round_out = false,
               bool a_tf32 = false);
int tc_error_read_and_clear(cudaStream_t s, int *code);
// Counter bumped by every mnpb_gemm_config call (launch configuration epoch).
int64_t gemm_config_epoch();
// Launches a one-thread kernel whose mbarrier wait (the tensor-core kernels'
// bounded wait, limit `limit_ns`) can only time out; it records code 9.
int wait_probe(cudaStream_t s, uint64_t limit_ns);

// 3-D FP32 TMA descriptor (written into the 128-byte CUtensorMap storage at
// map): dims[0] contiguous, byte strides of dims 1 and 2, box, swizzle as
// CUtensorMapSwizzle.  Checks the 16-byte rules of base and strides.
int encode_map_f32(void *map, const float *base, const uint64_t dims[3],
                   const uint64_t stride_bytes[2], const uint32_t box[3], int swizzle);

}  // namespace tc
}  // namespace mnpb
