// Kernels of the warm-start network (a per-face MLP that predicts the BEM
// solution at the next wavelength; it has no counterpart in the reference).
//
// Layout: activations row-major [rows][features] FP32; layer weights W
// [out][in] in bf16 (the copy the products read) with an FP32 master copy
// for the optimiser; biases FP32.  Products accumulate in FP32.
//
//  * mnpb_mlp_gemm: C = op(A) op(B) for strided operands (one SIMT kernel,
//    64 x 64 tiles, 4 x 4 outputs per thread), with the forward epilogue
//    (bias, SiLU, pre-activation kept for the backward pass) or split-K
//    partial sums (weight gradients reduce over many rows).
//  * mnpb_mlp_silu_back, mnpb_mlp_colsum, mnpb_mlp_mse, mnpb_mlp_adam:
//    element-wise pieces of the backward pass and the Adam update.
#include "common.cuh"

#include <cuda_bf16.h>

#include <cmath>

namespace mnpb {
namespace mlp {

constexpr int TM = 64, TN = 64, TK = 16;

template <typename T> __device__ __forceinline__ float ld(const T *p);
template <> __device__ __forceinline__ float ld<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16 *p) {
    return __bfloat162float(*p);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// epilogue modes
enum { EP_STORE = 0, EP_FWD_SILU = 1, EP_FWD_LINEAR = 2 };

// C[m, n] = sum_k A[m*sam + k*sak] * B[k*sbk + n*sbn]; blockIdx.z = K split
// (rows kz*kchunk ... of K), partial results at C + z * csplit.
template <typename TB>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, const float *__restrict__ A,
                                                   int64_t sam, int64_t sak,
                                                   const TB *__restrict__ B, int64_t sbk,
                                                   int64_t sbn, float *__restrict__ C, int64_t scm,
                                                   int64_t scn, int64_t csplit, int kchunk,
                                                   const float *__restrict__ bias, int mode,
                                                   float *__restrict__ Z) {
    __shared__ float As[TK][TM + 1];
    __shared__ float Bs[TK][TN + 1];
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
    const int k0 = blockIdx.z * kchunk, k1 = min(K, k0 + kchunk);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[4][4] = {};
    for (int kb = k0; kb < k1; kb += TK) {
        for (int e = threadIdx.x; e < TK * TM; e += 256) {
            const int kk = e / TM, mm = e % TM;
            const int m = m0 + mm, k = kb + kk;
            As[kk][mm] = (m < M && k < k1) ? A[(int64_t)m * sam + (int64_t)k * sak] : 0.f;
        }
        for (int e = threadIdx.x; e < TK * TN; e += 256) {
            const int kk = e / TN, nn = e % TN;
            const int n = n0 + nn, k = kb + kk;
            Bs[kk][nn] = (n < N && k < k1) ? ld<TB>(B + (int64_t)k * sbk + (int64_t)n * sbn) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    float *Cz = C + (int64_t)blockIdx.z * csplit;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty + 16 * i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx + 16 * j;
            if (n >= N) continue;
            float v = acc[i][j];
            const int64_t o = (int64_t)m * scm + (int64_t)n * scn;
            if (mode == EP_STORE) {
                Cz[o] = v;
            } else {
                v += bias ? bias[n] : 0.f;
                if (Z) Z[o] = v;
                Cz[o] = mode == EP_FWD_SILU ? silu(v) : v;
            }
        }
    }
}

// C[e] = sum_z P[z * csplit + e]  (fixed order)
__global__ void split_reduce_kernel(int64_t len, int nz, int64_t csplit, const float *P, float *C) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= len) return;
    float t = 0.f;
    for (int z = 0; z < nz; ++z) t += P[(int64_t)z * csplit + e];
    C[e] = t;
}

// dZ = dY * silu'(Z)
__global__ void silu_back_kernel(int64_t len, const float *dY, const float *Z, float *dZ) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < len) dZ[e] = dY[e] * silu_grad(Z[e]);
}

// out[c] = sum_r X[r * ld + c]: one block per column chunk, two-stage over rows
__global__ void colsum_kernel(int rows, int cols, const float *X, int64_t ld, float *out) {
    __shared__ float sh[8][33];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int w = threadIdx.x >> 5;
    float t = 0.f;
    if (c < cols)
        for (int r = w; r < rows; r += 8) t += X[(int64_t)r * ld + c];
    sh[w][threadIdx.x & 31] = t;
    __syncthreads();
    if (w == 0 && c < cols) {
        float s = 0.f;
        for (int k = 0; k < 8; ++k) s += sh[k][threadIdx.x & 31];
        out[c] = s;
    }
}

// dY = 2 (Y - T) / len, partial sums of (Y - T)^2 per block
__global__ void mse_kernel(int64_t len, const float *Y, const float *T, float *dY, float *part) {
    __shared__ float sh[8];
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float d2 = 0.f;
    if (e < len) {
        const float d = Y[e] - T[e];
        dY[e] = 2.f * d / (float)len;
        d2 = d * d;
    }
    for (int o = 16; o > 0; o >>= 1) d2 += __shfl_xor_sync(0xffffffffu, d2, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = d2;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
        part[blockIdx.x] = s;
    }
}

// Adam on FP32 master weights; the bf16 copy is refreshed (bias-corrected
// step size lr_t = lr sqrt(1 - b2^t) / (1 - b1^t), Kingma & Ba 2015)
__global__ void adam_kernel(int64_t len, float *w, __nv_bfloat16 *wb, const float *g, float *m,
                            float *v, float lr_t, float b1, float b2, float eps) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= len) return;
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gg;
    const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    const float ww = w[e] - lr_t * mm / (sqrtf(vv) + eps);
    w[e] = ww;
    if (wb) wb[e] = __float2bfloat16_rn(ww);
}

__global__ void to_bf16_kernel(int64_t len, const float *w, __nv_bfloat16 *wb) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < len) wb[e] = __float2bfloat16_rn(w[e]);
}

}  // namespace mlp
}  // namespace mnpb

using namespace mnpb;

// C (M x N) = op(A) op(B) with element strides; b_bf16: B holds bf16.
// mode 0: C = product (nsplit > 1: the K range is split, partial sums in
// work (nsplit * M * N floats), reduced in fixed order into C); mode 1: C =
// SiLU(product + bias), Z = product + bias; mode 2: C = Z = product + bias.
extern "C" int mnpb_mlp_gemm(void *stream, int64_t M, int64_t N, int64_t K, const float *A,
                             int64_t sam, int64_t sak, const void *B, int64_t sbk, int64_t sbn,
                             int32_t b_bf16, float *C, int64_t scm, int64_t scn,
                             const float *bias, int32_t mode, float *Z, int64_t nsplit,
                             float *work) {
    clear_error();
    MNPB_REQUIRE(M > 0 && N > 0 && K > 0 && nsplit >= 1 && nsplit <= 1024 && mode >= 0 && mode <= 2,
                 "mlp_gemm: bad sizes");
    MNPB_REQUIRE(A && B && C, "mlp_gemm: null pointer");
    MNPB_REQUIRE(nsplit == 1 || (mode == 0 && work && scm == N && scn == 1),
                 "mlp_gemm: split-K needs mode 0, work and a row-major dense C");
    cudaStream_t s = as_stream(stream);
    const int kchunk = (int)(((K + nsplit - 1) / nsplit + mlp::TK - 1) / mlp::TK * mlp::TK);
    const int nz = (int)((K + kchunk - 1) / kchunk);
    dim3 g((unsigned)((M + mlp::TM - 1) / mlp::TM), (unsigned)((N + mlp::TN - 1) / mlp::TN),
           (unsigned)nz);
    float *out = nz > 1 ? work : C;
    const int64_t ocm = nz > 1 ? N : scm, ocn = nz > 1 ? 1 : scn;
    ProfScope ps(s, PC_MLP, 2.0 * (double)M * N * K);
    if (b_bf16)
        mlp::gemm_kernel<__nv_bfloat16><<<g, 256, 0, s>>>(
            (int)M, (int)N, (int)K, A, sam, sak, (const __nv_bfloat16 *)B, sbk, sbn, out, ocm, ocn,
            M * N, kchunk, bias, mode, Z);
    else
        mlp::gemm_kernel<float><<<g, 256, 0, s>>>((int)M, (int)N, (int)K, A, sam, sak,
                                                  (const float *)B, sbk, sbn, out, ocm, ocn, M * N,
                                                  kchunk, bias, mode, Z);
    MNPB_LAUNCH_CHECK("mlp gemm_kernel");
    if (nz > 1) {
        mlp::split_reduce_kernel<<<ceil_div(M * N, 256), 256, 0, s>>>(M * N, nz, M * N, work, C);
        MNPB_LAUNCH_CHECK("mlp split_reduce_kernel");
    }
    return MNPB_OK;
}

extern "C" int mnpb_mlp_silu_back(void *stream, int64_t len, const float *dY, const float *Z,
                                  float *dZ) {
    clear_error();
    MNPB_REQUIRE(len > 0 && dY && Z && dZ, "mlp_silu_back: bad arguments");
    cudaStream_t s = as_stream(stream);
    mlp::silu_back_kernel<<<ceil_div(len, 256), 256, 0, s>>>(len, dY, Z, dZ);
    MNPB_LAUNCH_CHECK("mlp silu_back_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_mlp_colsum(void *stream, int64_t rows, int64_t cols, const float *X,
                               int64_t ld, float *out) {
    clear_error();
    MNPB_REQUIRE(rows > 0 && cols > 0 && ld >= cols && X && out, "mlp_colsum: bad arguments");
    cudaStream_t s = as_stream(stream);
    mlp::colsum_kernel<<<ceil_div(cols, 32), 256, 0, s>>>((int)rows, (int)cols, X, ld, out);
    MNPB_LAUNCH_CHECK("mlp colsum_kernel");
    return MNPB_OK;
}

// part: ceil(len / 256) floats; loss = sum(part) / len
extern "C" int mnpb_mlp_mse(void *stream, int64_t len, const float *Y, const float *T, float *dY,
                            float *part) {
    clear_error();
    MNPB_REQUIRE(len > 0 && Y && T && dY && part, "mlp_mse: bad arguments");
    cudaStream_t s = as_stream(stream);
    mlp::mse_kernel<<<ceil_div(len, 256), 256, 0, s>>>(len, Y, T, dY, part);
    MNPB_LAUNCH_CHECK("mlp mse_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_mlp_adam(void *stream, int64_t len, float *w, void *wb, const float *g,
                             float *m, float *v, double lr, double b1, double b2, double eps,
                             int64_t step) {
    clear_error();
    MNPB_REQUIRE(len > 0 && w && g && m && v && step >= 1, "mlp_adam: bad arguments");
    cudaStream_t s = as_stream(stream);
    const double lr_t = lr * std::sqrt(1.0 - std::pow(b2, (double)step)) /
                        (1.0 - std::pow(b1, (double)step));
    mlp::adam_kernel<<<ceil_div(len, 256), 256, 0, s>>>(len, w, (__nv_bfloat16 *)wb, g, m, v,
                                                       (float)lr_t, (float)b1, (float)b2,
                                                       (float)eps);
    MNPB_LAUNCH_CHECK("mlp adam_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_mlp_to_bf16(void *stream, int64_t len, const float *w, void *wb) {
    clear_error();
    MNPB_REQUIRE(len > 0 && w && wb, "mlp_to_bf16: bad arguments");
    cudaStream_t s = as_stream(stream);
    mlp::to_bf16_kernel<<<ceil_div(len, 256), 256, 0, s>>>(len, w, (__nv_bfloat16 *)wb);
    MNPB_LAUNCH_CHECK("mlp to_bf16_kernel");
    return MNPB_OK;
}
