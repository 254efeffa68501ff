// Shared helpers for the mnpbem_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/mnpbem_b200.h"

namespace mnpb {

// ---------------------------------------------------------------------------
// error state and launch accounting
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
void clear_error();
extern std::atomic<int64_t> g_launches;

inline void count_launch(int64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// Checks the last launch; returns MNPB_ECUDA with a message on failure.
int check_launch(const char *what);

#define MNPB_REQUIRE(cond, ...)            \
    do {                                   \
        if (!(cond)) {                     \
            ::mnpb::set_error(__VA_ARGS__); \
            return MNPB_EINVAL;            \
        }                                  \
    } while (0)

#define MNPB_TRY(expr)                 \
    do {                               \
        int _rc = (expr);              \
        if (_rc != MNPB_OK) return _rc; \
    } while (0)

#define MNPB_LAUNCH_CHECK(what)                          \
    do {                                                 \
        ::mnpb::count_launch();                          \
        int _rc = ::mnpb::check_launch(what);            \
        if (_rc != MNPB_OK) return _rc;                  \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Current device ordinal (-1 if cudaGetDevice fails).
int current_device();
// Raise `fn`'s dynamic shared-memory limit to `bytes` on the current device
// (once per kernel and device; thread-safe).  MNPB_ECUDA with a message
// naming `what` on failure.
int smem_opt_in(const void *fn, int bytes, const char *what);
template <typename F> inline int smem_opt_in(F *fn, int bytes, const char *what) {
    return smem_opt_in((const void *)fn, bytes, what);
}
// Number of SMs of the current device (cached per device; 148 if unknown).
int device_sms();
// MNPB_EINVAL unless stream `s` belongs to the current device (the legacy
// and per-thread default streams always do).
int check_stream_device(cudaStream_t s, const char *what);

// ---------------------------------------------------------------------------
// optional per-kernel-class timing with CUDA events (mnpb_prof_begin/end)
// ---------------------------------------------------------------------------
enum ProfClass {
    PC_ASSEMBLE = 0,   // work = bytes written
    PC_REFINE = 1,
    PC_ZGEMM = 2,      // work = real flops
    PC_PANEL = 3,
    PC_TRSM = 4,
    PC_SWAP = 5,
    PC_ELEM = 6,
    PC_TCGEMM = 7,     // work = real flops (tensor cores)
    PC_FARFIELD = 8,
    PC_SGEMM = 9,
    PC_MATVEC = 10,    // work = bytes read
    PC_TRSV = 11,      // one-launch triangular solves, work = bytes of the triangle
    PC_PACK = 12,      // tensor-core operand packing
    PC_REFINE_EW = 13, // refinement element-wise kernels (residual, norms, conversions)
    PC_ACA = 14,       // ACA of low-rank blocks, dense-block gather
    PC_HMATVEC = 15,   // H-matrix times vectors
    PC_GMRES = 16,     // Arnoldi orthogonalisation (work = bytes of the basis read)
    PC_MLP = 17,       // warm-start network kernels
    PC_COUNT = 24
};
bool prof_on();
void prof_record(cudaStream_t s, int cls, double work, bool start);
void prof_tag(const char *fmt, ...);   // annotate the launch being recorded

struct ProfScope {
    cudaStream_t s;
    int cls;
    double work;
    bool on;
    ProfScope(cudaStream_t s_, int cls_, double work_) : s(s_), cls(cls_), work(work_), on(prof_on()) {
        if (on) prof_record(s, cls, work, true);
    }
    ~ProfScope() {
        if (on) prof_record(s, cls, work, false);
    }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Face normals of a batch of BEM systems: entry b's n x 3 table starts at
// p + b * stride (stride 0: one table shared by every entry, a wavelength
// sweep of one particle; stride n * 3: a batch of different particles with
// the same face count).
struct NvecView {
    const double *p;
    int64_t stride;
    __host__ __device__ NvecView shifted(int64_t b0) const { return NvecView{p + b0 * stride, stride}; }
    __host__ __device__ const double *at(int64_t b) const { return p + b * stride; }
};

// ---------------------------------------------------------------------------
// complex double helpers (interleaved re, im)
// ---------------------------------------------------------------------------
typedef double2 cd;

__host__ __device__ __forceinline__ cd cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cd cadd(cd a, cd b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cd csub(cd a, cd b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cd cmul(cd a, cd b) {
    return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cd cscale(cd a, double s) { return cmk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ cd cconj(cd a) { return cmk(a.x, -a.y); }
// c + a*b with fused multiply-adds
__device__ __forceinline__ cd cfma(cd a, cd b, cd c) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
    return c;
}
// c - a*b
__device__ __forceinline__ cd cfms(cd a, cd b, cd c) {
    c.x = fma(-a.x, b.x, c.x);
    c.x = fma(a.y, b.y, c.x);
    c.y = fma(-a.x, b.y, c.y);
    c.y = fma(-a.y, b.x, c.y);
    return c;
}
// 1 / b by Smith's scaling (robust for wide exponent ranges)
__host__ __device__ __forceinline__ cd crcp(cd b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return cmk(1.0 / d, -r / d);
    } else {
        double r = b.x / b.y, d = b.y + b.x * r;
        return cmk(r / d, -1.0 / d);
    }
}
__host__ __device__ __forceinline__ cd cdiv(cd a, cd b) { return cmul(a, crcp(b)); }
__host__ __device__ __forceinline__ double cabs1(cd a) { return fabs(a.x) + fabs(a.y); }

// exp(i k d) for complex k and real d
__device__ __forceinline__ cd cexpi(cd k, double d) {
    double s, c;
    sincos(k.x * d, &s, &c);
    double m = exp(-k.y * d);
    return cmk(m * c, m * s);
}

}  // namespace mnpb
