// Batched dense complex linear algebra in FP32 on planar storage (real plane,
// imaginary plane), column-major, for the mixed-precision solver.
//
// LU is recursive (split the columns in halves; factor the left half; update
// the right half with a triangular solve and a GEMM; factor the rest), so
// nearly all flops land in large GEMMs that run on the tensor cores
// (tc::cgemm_tf32); only the 32-column LU leaves, the 128 x 128 diagonal-block
// inverses and the 32-row leaves of small triangular solves run on CUDA cores.
#include "common.cuh"
#include "dense_f32.cuh"

#include <cuda.h>

namespace mnpb {
namespace f32 {

using tc::CMatF;

namespace {

constexpr int PANEL_THREADS = 512;
constexpr int TS = 32;

struct cf {
    float x, y;
};
__device__ __forceinline__ cf fmk(float r, float i) { return cf{r, i}; }
__device__ __forceinline__ cf fmul(cf a, cf b) { return cf{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cf ffms(cf a, cf b, cf c) {   // c - a*b
    c.x = fmaf(-a.x, b.x, c.x);
    c.x = fmaf(a.y, b.y, c.x);
    c.y = fmaf(-a.x, b.y, c.y);
    c.y = fmaf(-a.y, b.x, c.y);
    return c;
}
__device__ __forceinline__ cf frcp(cf b) {
    if (fabsf(b.x) >= fabsf(b.y)) {
        float r = b.y / b.x, d = b.x + b.y * r;
        return cf{1.f / d, -r / d};
    } else {
        float r = b.x / b.y, d = b.y + b.x * r;
        return cf{r / d, -1.f / d};
    }
}
// nearest TF32 (10-bit mantissa), ties away from zero
__device__ __forceinline__ float tf32_rna(float v) {
    uint32_t t;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(v));
    return __uint_as_float(t);
}
__device__ __forceinline__ cf rna(cf v) { return cf{tf32_rna(v.x), tf32_rna(v.y)}; }
__device__ __forceinline__ cf ld(const float *p, int64_t plane, int64_t o) {
    return cf{p[o], p[o + plane]};
}
__device__ __forceinline__ void st(float *p, int64_t plane, int64_t o, cf v) {
    p[o] = v.x;
    p[o + plane] = v.y;
}

// LU leaf: columns [k0, k0+kb) (kb <= 32) over rows [k0, n), one CTA per matrix.
__global__ void __launch_bounds__(PANEL_THREADS) panel_kernel(int n, int k0, int kb, float *A,
                                                              int64_t lda, int64_t plane,
                                                              int64_t sA, int32_t *ipiv,
                                                              int64_t sP, int32_t *info) {
    __shared__ float red_v[PANEL_THREADS / 32];
    __shared__ int red_i[PANEL_THREADS / 32];
    __shared__ cf prow[TS];
    __shared__ int s_piv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t b = blockIdx.x;
    A += b * sA;
    ipiv += b * sP;
    for (int jj = 0; jj < kb; ++jj) {
        const int c = k0 + jj;
        const int64_t co = (int64_t)c * lda;
        float best = -1.f;
        int bi = n;
        for (int r = c + tid; r < n; r += PANEL_THREADS) {
            float v = fabsf(A[co + r]) + fabsf(A[co + r + plane]);
            if (v > best) { best = v; bi = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            float ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { red_v[wid] = best; red_i[wid] = bi; }
        __syncthreads();
        if (wid == 0) {
            best = (lane < PANEL_THREADS / 32) ? red_v[lane] : -1.f;
            bi = (lane < PANEL_THREADS / 32) ? red_i[lane] : n;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                float ov = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) {
                int p = bi;
                if (!(best > 0.f)) {
                    p = c;
                    if (info && info[b] == 0) info[b] = c + 1;
                }
                s_piv = p;
                ipiv[c] = p;
            }
        }
        __syncthreads();
        const int p = s_piv;
        if (p != c) {
            for (int cc = tid; cc < kb; cc += PANEL_THREADS) {
                const int64_t o = (int64_t)(k0 + cc) * lda;
                cf t = ld(A, plane, o + c);
                st(A, plane, o + c, ld(A, plane, o + p));
                st(A, plane, o + p, t);
            }
        }
        __syncthreads();
        const int rest = kb - jj;
        for (int cc = tid; cc < rest; cc += PANEL_THREADS) {
            const int64_t o = (int64_t)(c + cc) * lda + c;
            const cf u = rna(ld(A, plane, o));
            prow[cc] = u;
            st(A, plane, o, u);
        }
        __syncthreads();
        const cf pv = prow[0];
        const bool nz = (pv.x != 0.f || pv.y != 0.f);
        const cf inv = nz ? frcp(pv) : fmk(0.f, 0.f);
        for (int r = c + 1 + tid; r < n; r += PANEL_THREADS) {
            cf l = ld(A, plane, co + r);
            if (nz) l = rna(fmul(l, inv));
            st(A, plane, co + r, l);
            for (int cc = 1; cc < rest; ++cc) {
                const int64_t o = (int64_t)(c + cc) * lda + r;
                st(A, plane, o, ffms(l, prow[cc], ld(A, plane, o)));
            }
        }
        __syncthreads();
    }
}

// LU leaf in shared memory: columns [k0, k0+kb) factored as kb/SW slabs of SW
// columns.  A slab (rows cs..n-1, SW columns, planar) is loaded into shared
// memory and factored there column by column (partial pivoting on |re|+|im|,
// as the global-memory leaf); row swaps are mirrored into the panel's other
// columns in global memory.  The 4-column slabs run two CTAs per SM (batches
// above the SM count), so that instantiation is held to 64 registers.  The panel's columns right of the slab then get
// one block update: U12 = L11^{-1} A12 on the slab's SW rows, A22 -= L21 U12
// below.  Compared with the global-memory leaf, each panel column is read and
// written once per slab instead of once per column.  Dynamic shared memory:
// SW * (n - k0) * 8 bytes.
constexpr int SLAB_THREADS = 512;
// D += A B for one m16n8k8 TF32 tile (A 16 x 8 row-major, B 8 x 8 column-major,
// FP32 accumulators in the mma.sync fragment layout)
__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4],
                                         const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
template <int SW>
__global__ void __launch_bounds__(SLAB_THREADS, SW == 4 ? 2 : 1) panel_slab_kernel(int n, int k0, int kb, float *A,
                                                                 int64_t lda, int64_t plane,
                                                                 int64_t sA, int32_t *ipiv,
                                                                 int64_t sP, int32_t *info) {
    extern __shared__ float slab_sm[];
    __shared__ float red_v[SLAB_THREADS / 32];
    __shared__ int red_i[SLAB_THREADS / 32];
    __shared__ cf u12[SW][TS];
    __shared__ int slab_piv[SW];   // local pivot row of each slab column
    __shared__ int sw_dst[2 * SW], sw_src[2 * SW], sw_n;   // the slab's composed interchanges
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t b = blockIdx.x;
    A += b * sA;
    ipiv += b * sP;
    const int mmax = n - k0;
    float *sre = slab_sm, *sim = slab_sm + (int64_t)SW * mmax;
    for (int cs = k0; cs < k0 + kb; cs += SW) {
        const int ms = n - cs;                         // slab rows cs .. n-1
        // every load of a thread's rows issued before its shared-memory stores
        // (SW columns x 2 rows x 2 planes in flight per thread).  Each step's
        // pivot search is carried along (cbest, cbi): over the first column
        // here, and over column jj + 1 in step jj's update, which touches the
        // same rows of this thread in the same order as a separate search
        float cbest = -1.f;
        int cbi = ms;
        {
            const float *src = A + (int64_t)cs * lda + cs;
            for (int i0 = tid; i0 < ms; i0 += 2 * SLAB_THREADS) {
                float vr[SW][2], vi[SW][2];
#pragma unroll
                for (int j = 0; j < SW; ++j)
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int i = i0 + u * SLAB_THREADS;
                        const int64_t o = (int64_t)j * lda + i;
                        vr[j][u] = i < ms ? __ldcg(src + o) : 0.f;
                        vi[j][u] = i < ms ? __ldcg(src + o + plane) : 0.f;
                    }
#pragma unroll
                for (int j = 0; j < SW; ++j)
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int i = i0 + u * SLAB_THREADS;
                        if (i < ms) {
                            sre[j * mmax + i] = vr[j][u];
                            sim[j * mmax + i] = vi[j][u];
                        }
                    }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = i0 + u * SLAB_THREADS;
                    if (i < ms) {
                        const float v = fabsf(vr[0][u]) + fabsf(vi[0][u]);
                        if (v > cbest) { cbest = v; cbi = i; }
                    }
                }
            }
        }
        __syncthreads();
        for (int jj = 0; jj < SW; ++jj) {
            const int c = cs + jj;
            float best = cbest;
            int bi = cbi;
            cbest = -1.f;
            cbi = ms;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float ov = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) { red_v[wid] = best; red_i[wid] = bi; }
            // two barriers per step: (A) the partial maxima are visible and
            // every row update of the previous step is done; warp 0 then
            // picks the pivot and, one lane per slab column, swaps the pivot
            // row into place and stores its U entries as TF32; (B) the pivot
            // row is ready for the update.  The update's end needs no barrier
            // of its own: the next step's (A) follows it
            __syncthreads();
            if (wid == 0) {
                best = (lane < SLAB_THREADS / 32) ? red_v[lane] : -1.f;
                bi = (lane < SLAB_THREADS / 32) ? red_i[lane] : ms;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const float ov = __shfl_xor_sync(0xffffffffu, best, o);
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
                }
                // every lane holds the same (best, bi) after the butterfly
                const int ip = (best > 0.f) ? bi : jj;
                if (lane == 0) {
                    if (!(best > 0.f) && info && info[b] == 0) info[b] = c + 1;
                    slab_piv[jj] = ip;
                    ipiv[c] = cs + ip;
                }
                if (lane < SW) {
                    const int j = lane;
                    if (ip != jj) {
                        float t = sre[j * mmax + jj];
                        sre[j * mmax + jj] = sre[j * mmax + ip];
                        sre[j * mmax + ip] = t;
                        t = sim[j * mmax + jj];
                        sim[j * mmax + jj] = sim[j * mmax + ip];
                        sim[j * mmax + ip] = t;
                    }
                    if (j >= jj) {
                        sre[j * mmax + jj] = tf32_rna(sre[j * mmax + jj]);
                        sim[j * mmax + jj] = tf32_rna(sim[j * mmax + jj]);
                    }
                }
            }
            __syncthreads();
            const cf pv = fmk(sre[jj * mmax + jj], sim[jj * mmax + jj]);
            const bool nz = (pv.x != 0.f || pv.y != 0.f);
            const cf inv = nz ? frcp(pv) : fmk(0.f, 0.f);
            for (int i = jj + 1 + tid; i < ms; i += SLAB_THREADS) {
                cf l = fmk(sre[jj * mmax + i], sim[jj * mmax + i]);
                if (nz) l = rna(fmul(l, inv));
                sre[jj * mmax + i] = l.x;
                sim[jj * mmax + i] = l.y;
                for (int j = jj + 1; j < SW; ++j) {
                    const cf u = fmk(sre[j * mmax + jj], sim[j * mmax + jj]);
                    cf a = fmk(sre[j * mmax + i], sim[j * mmax + i]);
                    a = ffms(l, u, a);
                    sre[j * mmax + i] = a.x;
                    sim[j * mmax + i] = a.y;
                    if (j == jj + 1) {
                        const float v = fabsf(a.x) + fabsf(a.y);
                        if (v > cbest) { cbest = v; cbi = i; }
                    }
                }
            }
        }
        __syncthreads();
        {
            float *dst = A + (int64_t)cs * lda + cs;
            for (int i = tid; i < ms; i += SLAB_THREADS)
#pragma unroll
                for (int j = 0; j < SW; ++j) {
                    dst[(int64_t)j * lda + i] = sre[j * mmax + i];
                    dst[(int64_t)j * lda + i + plane] = sim[j * mmax + i];
                }
        }
        // the slab's SW row interchanges, applied to the panel's other columns:
        // warp 0 composes them (lane t holds touched row P and the original row
        // V whose value ends there) into at most 2 SW (destination, source)
        // pairs, then every other column is one gather and one scatter
        if (wid == 0) {
            int P = -1, V = -1, np = 0;
            for (int jj = 0; jj < SW; ++jj) {
                const int r2 = slab_piv[jj];
                unsigned m = __ballot_sync(0xffffffffu, P == jj);
                const int ia = m ? __ffs(m) - 1 : np;
                if (!m) {
                    if (lane == np) P = V = jj;
                    ++np;
                }
                m = __ballot_sync(0xffffffffu, P == r2);
                const int ib = m ? __ffs(m) - 1 : np;
                if (!m) {
                    if (lane == np) P = V = r2;
                    ++np;
                }
                const int va = __shfl_sync(0xffffffffu, V, ia);
                const int vb = __shfl_sync(0xffffffffu, V, ib);
                if (lane == ia) V = vb;
                if (lane == ib) V = va;
            }
            const bool keep = lane < np && V != P;
            const unsigned mk = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int at = __popc(mk & ((1u << lane) - 1u));
                sw_dst[at] = P;
                sw_src[at] = V;
            }
            if (lane == 0) sw_n = __popc(mk);
        }
        __syncthreads();
        {
            const int m = sw_n;
            for (int cc = tid; cc < kb; cc += SLAB_THREADS) {
                const int col = k0 + cc;
                if (col >= cs && col < cs + SW) continue;
                const int64_t o = (int64_t)col * lda + cs;
                cf vals[2 * SW];
                for (int t = 0; t < m; ++t) vals[t] = ld(A, plane, o + sw_src[t]);
                for (int t = 0; t < m; ++t) st(A, plane, o + sw_dst[t], vals[t]);
            }
        }
        __syncthreads();
        const int c1 = cs + SW, R = k0 + kb - c1;
        if (R > 0) {
            // U12 = L11^{-1} A12 (unit lower SW x SW from the slab's top rows)
            for (int q = tid; q < R; q += SLAB_THREADS) {
                const int64_t o = (int64_t)(c1 + q) * lda + cs;
                cf x[SW];
#pragma unroll
                for (int r = 0; r < SW; ++r) x[r] = ld(A, plane, o + r);
#pragma unroll
                for (int r = 1; r < SW; ++r)
#pragma unroll
                    for (int t = 0; t < r; ++t)
                        x[r] = ffms(fmk(sre[t * mmax + r], sim[t * mmax + r]), x[t], x[r]);
#pragma unroll
                for (int r = 0; r < SW; ++r) {
                    x[r] = rna(x[r]);
                    st(A, plane, o + r, x[r]);
                    u12[r][q] = x[r];
                }
            }
            __syncthreads();
            // A22 -= L21 U12 on rows cs+SW .. n-1.  8-column slabs: TF32
            // tensor-core tiles (mma.sync m16n8k8, FP32 accumulation); L21 and
            // U12 hold TF32 values, so every product is exact as in the FMA
            // loop.  One warp per 16-row x 8-column tile; real and imaginary
            // parts as  Cr += Lr (-Ur) + Li Ui,  Ci += Lr (-Ui) + Li (-Ur).
            // Measured on LUs of 2884 x 2884 matrices: -15 % for this phase
            // with 8-column slabs, +34 % with 4-column ones (K = 4 padded to
            // 8), which keep the FMA loop.
            if constexpr (SW == 8) {
                const int g = lane >> 2, t4 = lane & 3;
                const int nrt = (ms - SW + 15) / 16, nqt = (R + 7) / 8;
                for (int tile = wid; tile < nrt * nqt; tile += SLAB_THREADS / 32) {
                    const int tr = tile / nqt, q0 = 8 * (tile - tr * nqt);
                    const int r0 = SW + 16 * tr + g, r1 = r0 + 8;
                    unsigned ar[4], ai[4], bur[2], bui[2], buin[2];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int r = (e & 1) ? r1 : r0, k = t4 + 4 * (e >> 1);
                        const bool ok = r < ms && k < SW;
                        ar[e] = ok ? __float_as_uint(sre[k * mmax + r]) : 0u;
                        ai[e] = ok ? __float_as_uint(sim[k * mmax + r]) : 0u;
                    }
                    const int qb = q0 + g;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int k = t4 + 4 * e;
                        const bool ok = k < SW && qb < R;
                        const cf u = ok ? u12[k][qb] : fmk(0.f, 0.f);
                        bur[e] = __float_as_uint(-u.x);
                        bui[e] = __float_as_uint(u.y);
                        buin[e] = __float_as_uint(-u.y);
                    }
                    float cr[4], ci[4];
                    float *pc[4];
                    bool okc[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int r = (e & 2) ? r1 : r0, q = q0 + 2 * t4 + (e & 1);
                        okc[e] = r < ms && q < R;
                        pc[e] = A + (int64_t)(c1 + q) * lda + cs + r;
                        cr[e] = okc[e] ? pc[e][0] : 0.f;
                        ci[e] = okc[e] ? pc[e][plane] : 0.f;
                    }
                    mma_tf32(cr, ar, bur);
                    mma_tf32(cr, ai, bui);
                    mma_tf32(ci, ar, buin);
                    mma_tf32(ci, ai, bur);
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (okc[e]) {
                            pc[e][0] = cr[e];
                            pc[e][plane] = ci[e];
                        }
                }
            } else {
            // A22 -= L21 U12 on rows cs+SW .. n-1
            // all of a row's loads issued before its stores (one memory
            // round trip per row instead of one per column)
            for (int i = SW + tid; i < ms; i += SLAB_THREADS) {
                cf l[SW];
#pragma unroll
                for (int t = 0; t < SW; ++t) l[t] = fmk(sre[t * mmax + i], sim[t * mmax + i]);
                float *col = A + (int64_t)c1 * lda + cs + i;
                for (int q0 = 0; q0 < R; q0 += 8) {
                    cf a[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        if (q0 + q < R)
                            a[q] = fmk(col[(int64_t)(q0 + q) * lda],
                                       col[(int64_t)(q0 + q) * lda + plane]);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (q0 + q < R) {
#pragma unroll
                            for (int t = 0; t < SW; ++t) a[q] = ffms(l[t], u12[t][q0 + q], a[q]);
                            col[(int64_t)(q0 + q) * lda] = a[q].x;
                            col[(int64_t)(q0 + q) * lda + plane] = a[q].y;
                        }
                    }
                }
            }
            }
        }
        __syncthreads();
    }
}

// Row / column interchanges of a pivot range.  Pivoting on these matrices
// rarely moves a row, so each CTA first compacts the range's non-trivial
// interchanges (pivot p != c) into shared memory, in order, 1024 pivots at a
// time (warp 0, ballot + popc), and its threads then apply only those to
// their own column (laswp) or row (colswp).
constexpr int SWP_CHUNK = 1024;

__device__ int compact_swaps(const int32_t *pv, int lo, int hi, int2 *list) {
    // warp 0 fills list[0..count) with (c, pv[c]) for pv[c] != c, c in [lo, hi)
    __shared__ int s_count;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int count = 0;
        for (int c0 = lo; c0 < hi; c0 += 32) {
            const int c = c0 + lane;
            const int p = c < hi ? pv[c] : c;
            const bool f = p != c;
            const unsigned m = __ballot_sync(0xffffffffu, f);
            if (f) list[count + __popc(m & ((1u << lane) - 1u))] = make_int2(c, p);
            count += __popc(m);
        }
        if (lane == 0) s_count = count;
    }
    __syncthreads();
    const int n = s_count;
    __syncthreads();
    return n;
}

// Column segments of one interchange launch: columns [brk[i], brk[i+1])
// take the interchanges [cs[i], end) (cs[i] == end: none).
constexpr int SWP_MAXSEG = 24;
struct SwpSegs {
    int n, end;
    int brk[SWP_MAXSEG + 1];
    int cs[SWP_MAXSEG];
};

// segs != nullptr: column j takes only the interchanges of its segment's
// range (the recursive LU's fused forward + deferred backward interchanges)
__global__ void laswp_kernel(float *A, int64_t lda, int64_t plane, int64_t sA, int j0, int j1,
                             const int32_t *ipiv, int64_t sP, int c0, int c1, int forward,
                             const SwpSegs segs, int use_segs) {
    __shared__ int2 list[SWP_CHUNK];
    const int64_t b = blockIdx.y;
    const int j = j0 + blockIdx.x * blockDim.x + threadIdx.x;
    float *col = A + b * sA + (int64_t)j * lda;
    const int32_t *pv = ipiv + b * sP;
    const int nch = (c1 - c0 + SWP_CHUNK - 1) / SWP_CHUNK;
    for (int q = 0; q < nch; ++q) {
        const int ch = forward ? q : nch - 1 - q;
        const int lo = c0 + ch * SWP_CHUNK, hi = min(c1, lo + SWP_CHUNK);
        const int cnt = compact_swaps(pv, lo, hi, list);
        if (j < j1) {
            int cmin = c0;
            if (use_segs) {
                cmin = segs.end;
                for (int q = 0; q < segs.n; ++q)
                    if (j >= segs.brk[q] && j < segs.brk[q + 1]) cmin = segs.cs[q];
            }
            for (int t = 0; t < cnt; ++t) {
                const int2 e = list[forward ? t : cnt - 1 - t];
                if (e.x < cmin) continue;
                const cf x = ld(col, plane, e.x);
                st(col, plane, e.x, ld(col, plane, e.y));
                st(col, plane, e.y, x);
            }
        }
        __syncthreads();
    }
}

__global__ void colswp_kernel(float *X, int64_t ldx, int64_t plane, int64_t sX, int m,
                              const int32_t *ipiv, int64_t sP, int n) {
    __shared__ int2 list[SWP_CHUNK];
    const int64_t b = blockIdx.y;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float *x = X + b * sX + r;
    const int32_t *pv = ipiv + b * sP;
    const int nch = (n + SWP_CHUNK - 1) / SWP_CHUNK;
    for (int q = nch - 1; q >= 0; --q) {
        const int lo = q * SWP_CHUNK, hi = min(n, lo + SWP_CHUNK);
        const int cnt = compact_swaps(pv, lo, hi, list);
        if (r < m) {
            for (int t = cnt - 1; t >= 0; --t) {
                const int2 e = list[t];
                const cf v = ld(x, plane, (int64_t)e.x * ldx);
                st(x, plane, (int64_t)e.x * ldx, ld(x, plane, (int64_t)e.y * ldx));
                st(x, plane, (int64_t)e.y * ldx, v);
            }
        }
        __syncthreads();
    }
}

// Small triangular solves (kb <= 32), same modes as the FP64 version:
// 0 left lower unit, 1 left upper non-unit, 2 right upper non-unit,
// 3 right lower unit.
__global__ void __launch_bounds__(128) trsm_small_kernel(int mode, int kb, const float *T,
                                                         int64_t ldt, int64_t planeT, int64_t sT,
                                                         float *B, int64_t ldb, int64_t planeB,
                                                         int64_t sB, int nvec) {
    __shared__ cf Ts[TS][TS + 1];
    const int64_t b = blockIdx.y;
    T += b * sT;
    B += b * sB;
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
        const int r = e % TS, c = e / TS;
        Ts[r][c] = (r < kb && c < kb) ? ld(T, planeT, (int64_t)c * ldt + r)
                                      : fmk(r == c ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
    // non-unit modes: keep 1 / diagonal on the diagonal, so that no thread's
    // substitution chain contains a division
    if ((mode == 1 || mode == 2) && threadIdx.x < TS) Ts[threadIdx.x][threadIdx.x] = frcp(Ts[threadIdx.x][threadIdx.x]);
    __syncthreads();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvec) return;
    cf x[TS];
    const bool left = mode < 2;
#pragma unroll
    for (int e = 0; e < TS; ++e)
        x[e] = (e < kb) ? ld(B, planeB, left ? (int64_t)v * ldb + e : (int64_t)e * ldb + v)
                        : fmk(0.f, 0.f);
    if (mode == 0) {
#pragma unroll
        for (int r = 1; r < TS; ++r)
#pragma unroll
            for (int c = 0; c < r; ++c) x[r] = ffms(Ts[r][c], x[c], x[r]);
    } else if (mode == 1) {
#pragma unroll
        for (int r = TS - 1; r >= 0; --r) {
#pragma unroll
            for (int c = r + 1; c < TS; ++c) x[r] = ffms(Ts[r][c], x[c], x[r]);
            x[r] = fmul(x[r], Ts[r][r]);
        }
    } else if (mode == 2) {
#pragma unroll
        for (int c = 0; c < TS; ++c) {
#pragma unroll
            for (int r = 0; r < c; ++r) x[c] = ffms(x[r], Ts[r][c], x[c]);
            x[c] = fmul(x[c], Ts[c][c]);
        }
    } else {
#pragma unroll
        for (int c = TS - 1; c >= 0; --c)
#pragma unroll
            for (int r = c + 1; r < TS; ++r) x[c] = ffms(x[r], Ts[r][c], x[c]);
    }
#pragma unroll
    for (int e = 0; e < TS; ++e)
        if (e < kb) st(B, planeB, left ? (int64_t)v * ldb + e : (int64_t)e * ldb + v, rna(x[e]));
}

// Inverses of the 128 x 128 diagonal blocks of a unit-lower (lower = 1) or
// non-unit upper (lower = 0) triangle, one CTA per (block, matrix); the last
// block may be short (kb < 128) and is padded with the identity.  The block
// sits in shared memory column-major (k-th column contiguous), one warp
// builds one column j of the inverse by column-oriented substitution
// (T x = e_j): rows 32r + lane live in the lane's registers x[r], the newly
// final entry x_k is broadcast by a shuffle and subtracted, times column k
// of T, from the rows it feeds.  Output: out[b][blk][2][128][128] (planar,
// column-major, leading dimension 128).
constexpr int TL = 128;
constexpr int TINV_THREADS = 512;
constexpr int TINV_CPW = 4;      // columns a warp inverts together


__global__ void __launch_bounds__(TINV_THREADS) tri_inv_kernel(int n, int lower, const float *A,
                                                               int64_t lda, int64_t plane,
                                                               int64_t sA, float *out, int nb) {
    extern __shared__ __align__(16) unsigned char tinv_smem[];
    cf *Tc = reinterpret_cast<cf *>(tinv_smem);   // Tc[k * TL + i] = T(i, k)
    __shared__ cf dinv[TL];
    const int blk = blockIdx.x;
    const int64_t b = blockIdx.y;
    const int o = blk * TL, kb = min(TL, n - o);
    A += b * sA;
    for (int e = threadIdx.x; e < TL * TL; e += TINV_THREADS) {
        const int i = e % TL, k = e / TL;
        cf v = fmk(0.f, 0.f);
        if (i < kb && k < kb) {
            if (lower ? (i > k) : (i <= k)) v = ld(A, plane, (int64_t)(o + k) * lda + o + i);
        } else if (i == k) {
            v = fmk(1.f, 0.f);
        }
        Tc[e] = v;
    }
    __syncthreads();
    if (!lower && threadIdx.x < TL) {
        const cf d = Tc[threadIdx.x * TL + threadIdx.x];
        dinv[threadIdx.x] = (d.x != 0.f || d.y != 0.f) ? frcp(d) : fmk(0.f, 0.f);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *ob = out + ((b * nb + blk) * 2) * TL * TL;
    // Each warp solves two groups of TINV_CPW consecutive columns, group g
    // paired with group (TL / TINV_CPW - 1 - g) so every warp carries the same
    // substitution length.  The columns of a group share every step's
    // triangle loads and run as independent chains; a column whose index is
    // past the step carries zeros there (x_k = 0 above / below its unit
    // entry), so running the group's common step range is exact.
    static_assert(TL / TINV_CPW == 2 * (TINV_THREADS / 32), "two column groups per warp");
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
        const int grp = half == 0 ? w : TL / TINV_CPW - 1 - w;
        const int j0 = grp * TINV_CPW;
        cf x[TINV_CPW][4];
#pragma unroll
        for (int c = 0; c < TINV_CPW; ++c)
#pragma unroll
            for (int r = 0; r < 4; ++r) x[c][r] = fmk(32 * r + lane == j0 + c ? 1.f : 0.f, 0.f);
        if (lower) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (32 * r + 31 < j0) continue;
                for (int kk = (32 * r < j0 ? j0 - 32 * r : 0); kk < 32; ++kk) {
                    const int k = 32 * r + kk;
                    cf t[4];
#pragma unroll
                    for (int r2 = 0; r2 < 4; ++r2) t[r2] = r2 >= r ? Tc[k * TL + 32 * r2 + lane] : fmk(0.f, 0.f);
#pragma unroll
                    for (int c = 0; c < TINV_CPW; ++c) {
                        const cf xk = fmk(__shfl_sync(0xffffffffu, x[c][r].x, kk),
                                          __shfl_sync(0xffffffffu, x[c][r].y, kk));
#pragma unroll
                        for (int r2 = r; r2 < 4; ++r2)
                            if (r2 > r || lane > kk) x[c][r2] = ffms(t[r2], xk, x[c][r2]);
                    }
                }
            }
        } else {
            const int jt = j0 + TINV_CPW - 1;      // largest column of the group
#pragma unroll
            for (int r = 3; r >= 0; --r) {
                if (32 * r > jt) continue;
                for (int kk = min(31, jt - 32 * r); kk >= 0; --kk) {
                    const int k = 32 * r + kk;
                    cf t[4];
#pragma unroll
                    for (int r2 = 0; r2 < 4; ++r2) t[r2] = r2 <= r ? Tc[k * TL + 32 * r2 + lane] : fmk(0.f, 0.f);
                    const cf dk = dinv[k];
#pragma unroll
                    for (int c = 0; c < TINV_CPW; ++c) {
                        const cf xk = fmul(fmk(__shfl_sync(0xffffffffu, x[c][r].x, kk),
                                               __shfl_sync(0xffffffffu, x[c][r].y, kk)),
                                           dk);
                        if (lane == kk) x[c][r] = xk;
#pragma unroll
                        for (int r2 = 0; r2 <= r; ++r2)
                            if (r2 < r || lane < kk) x[c][r2] = ffms(t[r2], xk, x[c][r2]);
                    }
                }
            }
        }
        // stored rounded to nearest TF32, the precision the leaf GEMM reads
#pragma unroll
        for (int c = 0; c < TINV_CPW; ++c)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                ob[(j0 + c) * TL + 32 * r + lane] = tf32_rna(x[c][r].x);
                ob[TL * TL + (j0 + c) * TL + 32 * r + lane] = tf32_rna(x[c][r].y);
            }
    }
}

// Round rows [0, rows) of every column of a planar block to nearest TF32 in
// place: the right-hand sides of a left leaf, read by the tensor cores as the
// B operand (which would otherwise drop the low mantissa bits, a bias towards
// zero) and overwritten by the leaf's result right after.
// One CTA rounds RT_COLS columns of `rows` (<= 128) entries, both planes.
constexpr int RT_COLS = 8;
__global__ void __launch_bounds__(128) round_tf32_kernel(float *B, int64_t ldb, int64_t plane,
                                                         int64_t sB, int rows, int cols) {
    const int i = threadIdx.x;
    if (i >= rows) return;
    const int c0 = blockIdx.x * RT_COLS, c1 = min(cols, c0 + RT_COLS);
    float *base = B + blockIdx.y * sB + i;
#pragma unroll
    for (int c = c0; c < c1; ++c) {
        float *p = base + (int64_t)c * ldb;
        p[0] = tf32_rna(p[0]);
        p[plane] = tf32_rna(p[plane]);
    }
}

// Skinny GEMM C = alpha A B + beta C for at most NC (<= 16) columns (matrix
// times a few vectors): one thread per row, A streamed once with coalesced
// column reads, B broadcast from shared memory.  Real alpha, beta.
constexpr int SK_N = 16, SK_KT = 64;

template <int NC>
__global__ void __launch_bounds__(128) skinny_kernel(int m, int n, int k, float alpha,
                                                     const float *__restrict__ A, int64_t lda,
                                                     int64_t planeA, int64_t sA,
                                                     const float *__restrict__ B, int64_t ldb,
                                                     int64_t planeB, int64_t sB, float beta,
                                                     float *__restrict__ C, int64_t ldc,
                                                     int64_t planeC, int64_t sC, int rnd) {
    __shared__ cf Bs[SK_KT][NC];
    const int64_t b = blockIdx.y;
    A += b * sA;
    B += b * sB;
    C += b * sC;
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    cf acc[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) acc[j] = fmk(0.f, 0.f);
    for (int k0 = 0; k0 < k; k0 += SK_KT) {
        __syncthreads();
        for (int e = threadIdx.x; e < SK_KT * NC; e += blockDim.x) {
            const int kk = e % SK_KT, j = e / SK_KT;
            Bs[kk][j] = (k0 + kk < k && j < n) ? ld(B, planeB, (int64_t)j * ldb + k0 + kk)
                                               : fmk(0.f, 0.f);
        }
        __syncthreads();
        if (row < m) {
            const int kend = min(SK_KT, k - k0);
            const float *ar = A + (int64_t)k0 * lda + row;
#pragma unroll 4
            for (int kk = 0; kk < kend; ++kk) {
                const cf a = fmk(__ldg(ar + (int64_t)kk * lda), __ldg(ar + (int64_t)kk * lda + planeA));
#pragma unroll
                for (int j = 0; j < NC; ++j) {
                    acc[j].x = fmaf(a.x, Bs[kk][j].x, acc[j].x);
                    acc[j].x = fmaf(-a.y, Bs[kk][j].y, acc[j].x);
                    acc[j].y = fmaf(a.x, Bs[kk][j].y, acc[j].y);
                    acc[j].y = fmaf(a.y, Bs[kk][j].x, acc[j].y);
                }
            }
        }
    }
    if (row >= m) return;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        if (j < n) {
            const int64_t o = (int64_t)j * ldc + row;
            cf c = beta != 0.f ? ld(C, planeC, o) : fmk(0.f, 0.f);
            cf v = fmk(alpha * acc[j].x + beta * c.x, alpha * acc[j].y + beta * c.y);
            if (rnd) v = fmk(tf32_rna(v.x), tf32_rna(v.y));
            st(C, planeC, o, v);
        }
    }
}


// ---------------------------------------------------------------------------
// Few-RHS triangular solves in one launch per triangle.
//
// Block rows of 32: block j needs the solution of every earlier block (in
// solve order).  A CTA takes a ticket from an atomic counter and handles the
// (block, matrix) pair of that ticket, tickets ordered block-major, so every
// block it waits for has a lower ticket and has started: the smallest
// unfinished ticket can always proceed.  Blocks publish their solution with a
// release (fence + atomic flag = epoch); waiters use acquire loads, bounded
// by a 1 s wall-clock limit after which an error word is set and the kernel
// continues (the solve is then invalid and reported, but nothing hangs).
// The 32 x 32 diagonal blocks are applied through precomputed inverses.
// ---------------------------------------------------------------------------
constexpr int TB = 32;
constexpr uint64_t TRSV_WAIT_NS = 1000000000ull;

__device__ int g_trsv_error;

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Spins (acquire loads) until *p == want, for at most `limit` ns of wall
// time; false if it gave up.
__device__ __forceinline__ bool wait_flag(const int *p, int want, uint64_t limit) {
    const uint64_t t0 = gtimer();
    while (ld_acquire(p) != want)
        if (gtimer() - t0 > limit) return false;
    return true;
}

// Inverse of each 32 x 32 diagonal block of the unit-lower (lower = 1) or
// upper (lower = 0) factor; out[b][blk][2][32][32] (planar, column-major).
__global__ void __launch_bounds__(TB) diag_inv_kernel(int n, int lower, const float *A,
                                                      int64_t lda, int64_t plane, int64_t sA,
                                                      float *out, int nb) {
    __shared__ cf T[TB][TB + 1];
    const int blk = blockIdx.x;
    const int64_t b = blockIdx.y;
    const int r0 = blk * TB, kb = min(TB, n - r0);
    A += b * sA;
    for (int c = 0; c < TB; ++c) {
        const int r = threadIdx.x;
        cf v = fmk(r == c ? 1.f : 0.f, 0.f);
        if (r < kb && c < kb) {
            const bool in = lower ? (r > c) : (r <= c);
            if (in) v = ld(A, plane, (int64_t)(r0 + c) * lda + r0 + r);
            else v = (lower && r == c) ? fmk(1.f, 0.f) : fmk(0.f, 0.f);
        }
        T[r][c] = v;
    }
    __syncthreads();
    // column t of the inverse: solve T x = e_t
    const int t = threadIdx.x;
    cf x[TB];
#pragma unroll
    for (int e = 0; e < TB; ++e) x[e] = fmk(e == t ? 1.f : 0.f, 0.f);
    if (lower) {
#pragma unroll
        for (int r = 1; r < TB; ++r)
#pragma unroll
            for (int c = 0; c < r; ++c) x[r] = ffms(T[r][c], x[c], x[r]);
    } else {
#pragma unroll
        for (int r = TB - 1; r >= 0; --r) {
#pragma unroll
            for (int c = r + 1; c < TB; ++c) x[r] = ffms(T[r][c], x[c], x[r]);
            x[r] = fmul(x[r], frcp(T[r][r]));
        }
    }
    float *o = out + ((b * nb + blk) * 2) * TB * TB;
#pragma unroll
    for (int e = 0; e < TB; ++e) {
        o[t * TB + e] = x[e].x;
        o[TB * TB + t * TB + e] = x[e].y;
    }
}

template <int NC>
__global__ void __launch_bounds__(256) trsv_kernel(int n, int m, int lower, const float *A,
                                                   int64_t lda, int64_t plane, int64_t sA,
                                                   const float *__restrict__ Dinv, float *X,
                                                   int64_t ldx, int64_t planeX, int64_t sX,
                                                   int *flags, unsigned *ticket, int epoch,
                                                   int nb, int batch) {
    __shared__ int s_ticket;
    __shared__ cf red[8][TB][NC];
    __shared__ cf rhs[TB][NC];
    __shared__ cf dinv_s[TB][TB + 1];
    const int tid = threadIdx.x, r = tid & 31, q = tid >> 5;
    if (tid == 0) s_ticket = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int tk = s_ticket;
    const int jj = tk / batch;
    const int64_t b = tk % batch;
    const int j = lower ? jj : nb - 1 - jj;
    const int r0 = j * TB, rows = min(TB, n - r0);
    A += b * sA;
    X += b * sX;
    int *fl = flags + b * nb;
    // stage the inverse of the diagonal block (independent of other blocks)
    const float *Di = Dinv + (b * nb + j) * 2 * TB * TB;
    for (int e = tid; e < TB * TB; e += 256) {
        const int rr = e % TB, k = e / TB;
        dinv_s[rr][k] = fmk(__ldg(Di + k * TB + rr), __ldg(Di + TB * TB + k * TB + rr));
    }
    cf acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = fmk(0.f, 0.f);
    // blocks finish in chain order, so once the last dependency is published
    // every earlier one is too
    int known = -1;
    if (jj > 0 && r == 0) {
        const int last = lower ? jj - 1 : nb - jj;
        if (ld_acquire(fl + last) == epoch) known = jj - 1;
    }
    known = __shfl_sync(0xffffffffu, known, 0);
    __syncwarp();   // orders the lanes' later reads after lane 0's acquire
    for (int ii = 0; ii < jj; ++ii) {
        const int i = lower ? ii : nb - 1 - ii;
        // factor entries first: they do not depend on other blocks
        cf a[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int col = i * TB + q + 8 * t;
            a[t] = fmk(0.f, 0.f);
            if (col < n && r < rows) {
                const int64_t o = (int64_t)col * lda + r0 + r;
                a[t] = fmk(A[o], A[o + plane]);
            }
        }
        if (ii > known) {
            // lane 0 of each warp waits (acquire); __syncwarp orders the lanes' reads
            if (r == 0 && !wait_flag(fl + i, epoch, TRSV_WAIT_NS)) atomicCAS(&g_trsv_error, 0, 1);
            __syncwarp();
            known = ii;
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int col = i * TB + q + 8 * t;
            if (col < n && r < rows) {
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    if (c < m) {
                        const int64_t xo = (int64_t)c * ldx + col;
                        const cf xv = fmk(__ldcg(X + xo), __ldcg(X + xo + planeX));
                        acc[c].x = fmaf(a[t].x, xv.x, acc[c].x);
                        acc[c].x = fmaf(-a[t].y, xv.y, acc[c].x);
                        acc[c].y = fmaf(a[t].x, xv.y, acc[c].y);
                        acc[c].y = fmaf(a[t].y, xv.x, acc[c].y);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) red[q][r][c] = acc[c];
    __syncthreads();
    for (int e = tid; e < TB * NC; e += 256) {
        const int rr = e % TB, c = e / TB;
        cf v = fmk(0.f, 0.f);
        if (rr < rows && c < m) {
            const int64_t xo = (int64_t)c * ldx + r0 + rr;
            v = fmk(__ldcg(X + xo), __ldcg(X + xo + planeX));
#pragma unroll
            for (int qq = 0; qq < 8; ++qq) {
                v.x -= red[qq][rr][c].x;
                v.y -= red[qq][rr][c].y;
            }
        }
        rhs[rr][c] = v;
    }
    __syncthreads();
    for (int e = tid; e < TB * NC; e += 256) {
        const int rr = e % TB, c = e / TB;
        if (rr < rows && c < m) {
            cf y = fmk(0.f, 0.f);
#pragma unroll 8
            for (int k = 0; k < TB; ++k) {
                const cf d = dinv_s[rr][k];
                y.x = fmaf(d.x, rhs[k][c].x, y.x);
                y.x = fmaf(-d.y, rhs[k][c].y, y.x);
                y.y = fmaf(d.x, rhs[k][c].y, y.y);
                y.y = fmaf(d.y, rhs[k][c].x, y.y);
            }
            const int64_t xo = (int64_t)c * ldx + r0 + rr;
            X[xo] = y.x;
            X[xo + planeX] = y.y;
        }
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        atomicExch(fl + j, epoch);
    }
}

// Few-RHS triangular solve, one CTA per matrix, right-looking: the whole
// right-hand side lives in shared memory (r[i][c], n x NC), each 32-row block
// is solved through its precomputed diagonal inverse, then every row the
// block feeds (below it for L, above it for U) subtracts T[i, block] x_block,
// streaming that column block of the triangle once.  Two rows per thread with
// 8-byte loads, 16 columns in flight; the next block's diagonal inverse is
// staged while the current block's update runs.  No inter-CTA waits.
constexpr int RL_THREADS = 512;
template <int NC>
__global__ void __launch_bounds__(RL_THREADS) trsv_rl_kernel(int n, int m, int lower,
                                                             const float *__restrict__ A,
                                                             int64_t lda, int64_t plane,
                                                             int64_t sA,
                                                             const float *__restrict__ Dinv,
                                                             float *X, int64_t ldx,
                                                             int64_t planeX, int64_t sX, int nb) {
    extern __shared__ __align__(16) unsigned char rl_smem[];
    cf *r = reinterpret_cast<cf *>(rl_smem);   // r[i * NC + c]
    __shared__ cf dsm[2][TB][TB + 1];
    __shared__ cf xj[TB][NC];
    const int tid = threadIdx.x;
    const int64_t b = blockIdx.x;
    A += b * sA;
    X += b * sX;
    const float *Db = Dinv + b * nb * 2 * TB * TB;
    for (int e = tid; e < n * NC; e += RL_THREADS) {
        const int i = e % n, c = e / n;
        r[i * NC + c] = c < m ? ld(X, planeX, (int64_t)c * ldx + i) : fmk(0.f, 0.f);
    }
    {
        const int j = lower ? 0 : nb - 1;
        const float *Di = Db + (int64_t)j * 2 * TB * TB;
        for (int e = tid; e < TB * TB; e += RL_THREADS) {
            const int rr = e % TB, k = e / TB;
            dsm[0][rr][k] = fmk(__ldg(Di + k * TB + rr), __ldg(Di + TB * TB + k * TB + rr));
        }
    }
    __syncthreads();
    for (int jj = 0; jj < nb; ++jj) {
        const int j = lower ? jj : nb - 1 - jj, r0 = j * TB, rows = min(TB, n - r0);
        const int buf = jj & 1;
        // diagonal block: x_j = D_j^{-1} r_j
        if (tid < TB * NC) {
            const int rr = tid % TB, c = tid / TB;
            cf y = fmk(0.f, 0.f);
            if (rr < rows && c < m) {
#pragma unroll 8
                for (int k = 0; k < TB; ++k) {
                    if (k < rows) {
                        const cf d = dsm[buf][rr][k], v = r[(r0 + k) * NC + c];
                        y.x = fmaf(d.x, v.x, y.x);
                        y.x = fmaf(-d.y, v.y, y.x);
                        y.y = fmaf(d.x, v.y, y.y);
                        y.y = fmaf(d.y, v.x, y.y);
                    }
                }
                st(X, planeX, (int64_t)c * ldx + r0 + rr, y);
            }
            xj[rr][c] = y;
        }
        __syncthreads();
        // stage the next block's inverse while this block's update runs
        if (jj + 1 < nb) {
            const int jn = lower ? j + 1 : j - 1;
            const float *Di = Db + (int64_t)jn * 2 * TB * TB;
            for (int e = tid; e < TB * TB; e += RL_THREADS) {
                const int rr = e % TB, k = e / TB;
                dsm[buf ^ 1][rr][k] =
                    fmk(__ldg(Di + k * TB + rr), __ldg(Di + TB * TB + k * TB + rr));
            }
        }
        const int lo = lower ? r0 + rows : 0, hi = lower ? n : r0;
        const float *Ac = A + (int64_t)r0 * lda;
        for (int i = lo + 2 * tid; i < hi; i += 2 * RL_THREADS) {
            const bool two = i + 1 < hi;
            cf a0[NC], a1[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) a0[c] = a1[c] = fmk(0.f, 0.f);
            for (int k0 = 0; k0 < rows; k0 += 16) {
                float2 vr[16], vi[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    vr[k] = vi[k] = make_float2(0.f, 0.f);
                    if (k0 + k < rows) {
                        const float *p = Ac + (int64_t)(k0 + k) * lda + i;
                        if (two) {
                            vr[k] = __ldg(reinterpret_cast<const float2 *>(p));
                            vi[k] = __ldg(reinterpret_cast<const float2 *>(p + plane));
                        } else {
                            vr[k].x = __ldg(p);
                            vi[k].x = __ldg(p + plane);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < 16; ++k) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const cf x = xj[(k0 + k) & (TB - 1)][c];
                        a0[c].x = fmaf(vr[k].x, x.x, a0[c].x);
                        a0[c].x = fmaf(-vi[k].x, x.y, a0[c].x);
                        a0[c].y = fmaf(vr[k].x, x.y, a0[c].y);
                        a0[c].y = fmaf(vi[k].x, x.x, a0[c].y);
                        a1[c].x = fmaf(vr[k].y, x.x, a1[c].x);
                        a1[c].x = fmaf(-vi[k].y, x.y, a1[c].x);
                        a1[c].y = fmaf(vr[k].y, x.y, a1[c].y);
                        a1[c].y = fmaf(vi[k].y, x.x, a1[c].y);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                cf &u = r[i * NC + c];
                u.x -= a0[c].x;
                u.y -= a0[c].y;
                if (two) {
                    cf &w = r[(i + 1) * NC + c];
                    w.x -= a1[c].x;
                    w.y -= a1[c].y;
                }
            }
        }
        __syncthreads();
    }
}

// ---- few-RHS triangular solve with the triangle streamed by TMA ------------
//
// One CTA per matrix; the right-hand sides r (n x NC) stay in shared memory.
// Warp 9 (one lane) streams the triangle block column by block column in the
// order the solve consumes it: for 32-column block j, the inverse of its
// diagonal block (8 KB, bulk copy) and then every 128-row tile the block
// updates (below it for L, above it, bottom tile first, for U), through a
// ring of S stages; it runs ahead of the arithmetic, bounded only by the
// ring.  Warp 8 solves the diagonal blocks (x_j = D_j^{-1} r_j) into a double
// buffer as soon as the first tile of the previous block has updated block
// j's rows; warps 0-7 update r with each tile: thread t takes row t % 128 and
// half of the tile's 32 columns (t / 128); the second half's partial sums
// meet the first half's through a double buffer in shared memory.  Every
// mbarrier wait is bounded; on a timeout the kernel records an error in
// g_trsv_error and stops.
constexpr int STR_ROWS = 128;                                  // rows per tile
constexpr int STR_TILE_BYTES = 2 * TB * STR_ROWS * 4;          // re + im planes
constexpr int STR_CONS = 256;                                  // consumer threads
constexpr int STR_THREADS = STR_CONS + 64;
constexpr uint64_t STR_WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t s_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void sbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void sbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void sbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool sbar_wait(uint32_t bar, uint32_t parity,
                                          uint64_t limit = STR_WAIT_NS) {
    const uint64_t t0 = gtimer();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (gtimer() - t0 > limit) return false;
    }
}
__device__ __forceinline__ void s_tma3(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0,
                                       int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}
__device__ __forceinline__ void s_bulk(uint32_t dst, const void *src, uint32_t bytes,
                                       uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(dst),
        "l"((uint64_t)src), "r"(bytes), "r"(bar)
        : "memory");
}

template <int NC>
__global__ void __launch_bounds__(STR_THREADS, 1)
    trsv_stream_kernel(const __grid_constant__ CUtensorMap tmRe,
                       const __grid_constant__ CUtensorMap tmIm, int n, int m, int lower,
                       const float *__restrict__ Dinv, float *X, int64_t ldx, int64_t planeX,
                       int64_t sX, int nb, int S) {
    extern __shared__ __align__(1024) unsigned char str_raw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)str_raw + 1023) & ~(uintptr_t)1023);
    float *ring = (float *)sm;                                        // S tiles
    float *dsm = (float *)(sm + (size_t)S * STR_TILE_BYTES);          // 2 x [2][32][32]
    cf *xb = (cf *)(dsm + 2 * 2 * TB * TB);                           // 2 x [32][NC]
    cf *red = xb + 2 * TB * NC;                                       // 2 x [128][NC]
    cf *r = red + 2 * STR_ROWS * NC;                                  // [n][NC]
    uint64_t *bars = (uint64_t *)(r + (size_t)n * NC);
    // bars: full[S], empty[S], dfull[2], dempty[2], rows_ready, xready[2],
    // red_full[2], red_empty[2]
    uint64_t *full = bars, *empty = bars + S, *dfull = bars + 2 * S, *dempty = dfull + 2;
    uint64_t *rows_ready = dempty + 2, *xready = rows_ready + 1;
    uint64_t *red_full = xready + 2, *red_empty = red_full + 2;
    volatile int *abort_flag = (volatile int *)(red_empty + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t b = blockIdx.x;
    X += b * sX;
    const float *Db = Dinv + b * nb * 2 * TB * TB;

    for (int e = tid; e < n * NC; e += STR_THREADS) {
        const int i = e % n, c = e / n;
        r[i * NC + c] = c < m ? ld(X, planeX, (int64_t)c * ldx + i) : fmk(0.f, 0.f);
    }
    if (tid == 0) {
        for (int q = 0; q < S; ++q) {
            sbar_init(s_u32(&full[q]), 1);
            sbar_init(s_u32(&empty[q]), STR_CONS);
        }
        for (int q = 0; q < 2; ++q) {
            sbar_init(s_u32(&dfull[q]), 1);
            sbar_init(s_u32(&dempty[q]), 1);
            sbar_init(s_u32(&xready[q]), 1);
            sbar_init(s_u32(&red_full[q]), STR_CONS / 2);
            sbar_init(s_u32(&red_empty[q]), STR_CONS / 2);
        }
        sbar_init(s_u32(rows_ready), STR_ROWS);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // tile t of block j: first row and row range [lo, hi) that the block updates
    auto range = [&](int j, int &lo, int &hi) {
        if (lower) {
            lo = (j + 1) * TB;
            hi = n;
        } else {
            lo = 0;
            hi = j * TB;
        }
        if (lo > hi) lo = hi;
    };
    auto tile_row = [&](int lo, int hi, int t) {
        return lower ? lo + t * STR_ROWS : hi - (t + 1) * STR_ROWS;
    };
    auto fail = [&](int code) {
        atomicCAS(&g_trsv_error, 0, code);
        *abort_flag = 1;
    };

    if (warp == 9) {
        if (lane == 0) {
            uint32_t g = 0;
            // the inverse of block jj's diagonal block; block jj + 1's is
            // requested right after the first tile of block jj, so that the
            // diagonal solve never waits for it
            auto load_dinv = [&](int jj) -> bool {
                const int j = lower ? jj : nb - 1 - jj, buf = jj & 1;
                if (jj >= 2 && !sbar_wait(s_u32(&dempty[buf]), ((jj - 2) >> 1) & 1)) {
                    fail(11);
                    return false;
                }
                sbar_expect(s_u32(&dfull[buf]), 2 * TB * TB * 4);
                s_bulk(s_u32(dsm + buf * 2 * TB * TB), Db + (int64_t)j * 2 * TB * TB,
                       2 * TB * TB * 4, s_u32(&dfull[buf]));
                return true;
            };
            bool ok = load_dinv(0);
            for (int jj = 0; jj < nb && ok && !*abort_flag; ++jj) {
                const int j = lower ? jj : nb - 1 - jj;
                int lo, hi;
                range(j, lo, hi);
                const int nt = (hi - lo + STR_ROWS - 1) / STR_ROWS;
                for (int t = 0; t < nt; ++t, ++g) {
                    const int q = g % S;
                    if (g >= (uint32_t)S && !sbar_wait(s_u32(&empty[q]), ((g / S) - 1) & 1)) {
                        fail(12);
                        ok = false;
                        break;
                    }
                    const uint32_t dst = s_u32(ring) + q * STR_TILE_BYTES;
                    sbar_expect(s_u32(&full[q]), STR_TILE_BYTES);
                    s_tma3(dst, &tmRe, s_u32(&full[q]), tile_row(lo, hi, t), j * TB, (int)b);
                    s_tma3(dst + STR_TILE_BYTES / 2, &tmIm, s_u32(&full[q]), tile_row(lo, hi, t),
                           j * TB, (int)b);
                    if (t == 0 && jj + 1 < nb && !load_dinv(jj + 1)) {
                        ++g;
                        ok = false;
                        break;
                    }
                }
            }
            // copies still in flight (only after an abort): wait for them, bounded
            if (*abort_flag) {
                const uint32_t first = g > (uint32_t)S ? g - S : 0;
                for (uint32_t h = first; h < g; ++h)
                    sbar_wait(s_u32(&full[h % S]), (h / S) & 1);
                for (int q = 0; q < 2 && q < nb; ++q) {
                    // last use of each inverse buffer: jl = largest block index with jl % 2 == q
                    const int jl = ((nb - 1 - q) / 2) * 2 + q;
                    sbar_wait(s_u32(&dfull[q]), (jl >> 1) & 1);
                }
            }
        }
    } else if (warp == 8) {
        for (int jj = 0; jj < nb && !*abort_flag; ++jj) {
            const int j = lower ? jj : nb - 1 - jj, buf = jj & 1;
            const int r0 = j * TB, rows = min(TB, n - r0);
            if (jj >= 1 && !sbar_wait(s_u32(rows_ready), (jj - 1) & 1)) {
                if (lane == 0) fail(13);
                break;
            }
            if (!sbar_wait(s_u32(&dfull[buf]), (jj >> 1) & 1)) {
                if (lane == 0) fail(14);
                break;
            }
            const float *Dr = dsm + buf * 2 * TB * TB, *Di = Dr + TB * TB;
            cf *xo = xb + buf * TB * NC;
            cf y[NC];
#pragma unroll
            for (int c = 0; c < NC; ++c) y[c] = fmk(0.f, 0.f);
            if (lane < rows) {
#pragma unroll 4
                for (int k = 0; k < rows; ++k) {
                    const cf d = fmk(Dr[k * TB + lane], Di[k * TB + lane]);
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        const cf v = r[(r0 + k) * NC + c];
                        y[c].x = fmaf(d.x, v.x, y[c].x);
                        y[c].x = fmaf(-d.y, v.y, y[c].x);
                        y[c].y = fmaf(d.x, v.y, y[c].y);
                        y[c].y = fmaf(d.y, v.x, y[c].y);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                if (c >= m) y[c] = fmk(0.f, 0.f);
                if (lane < rows && c < m) st(X, planeX, (int64_t)c * ldx + r0 + lane, y[c]);
                xo[lane * NC + c] = y[c];
            }
            __syncwarp();
            if (lane == 0) {
                sbar_arrive(s_u32(&xready[buf]));
                sbar_arrive(s_u32(&dempty[buf]));
            }
        }
    } else {
        // warps 0-7: row tid % 128 of each tile, columns [16 h, 16 h + 16), h = tid / 128
        const int row = tid & (STR_ROWS - 1), h = tid >> 7;
        uint32_t g = 0;
        for (int jj = 0; jj < nb && !*abort_flag; ++jj) {
            const int j = lower ? jj : nb - 1 - jj, buf = jj & 1;
            if (!sbar_wait(s_u32(&xready[buf]), (jj >> 1) & 1)) {
                fail(15);
                break;
            }
            const cf *xj = xb + buf * TB * NC;
            int lo, hi;
            range(j, lo, hi);
            const int nt = (hi - lo + STR_ROWS - 1) / STR_ROWS;
            bool ok = true;
            for (int t = 0; t < nt; ++t, ++g) {
                const int q = g % S;
                if (!sbar_wait(s_u32(&full[q]), (g / S) & 1)) {
                    fail(16);
                    ok = false;
                    break;
                }
                const float *tr = ring + (size_t)q * (STR_TILE_BYTES / 4), *ti = tr + TB * STR_ROWS;
                cf acc[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) acc[c] = fmk(0.f, 0.f);
#pragma unroll
                for (int kk = 0; kk < TB / 2; ++kk) {
                    const int k = 16 * h + kk;
                    const float ar = tr[k * STR_ROWS + row], ai = ti[k * STR_ROWS + row];
                    cf x[NC];
                    if (NC % 2 == 0) {
#pragma unroll
                        for (int c = 0; c < NC; c += 2) {
                            const float4 v = *reinterpret_cast<const float4 *>(xj + k * NC + c);
                            x[c] = fmk(v.x, v.y);
                            x[c + 1] = fmk(v.z, v.w);
                        }
                    } else {
#pragma unroll
                        for (int c = 0; c < NC; ++c) x[c] = xj[k * NC + c];
                    }
#pragma unroll
                    for (int c = 0; c < NC; ++c) {
                        acc[c].x = fmaf(ar, x[c].x, acc[c].x);
                        acc[c].x = fmaf(-ai, x[c].y, acc[c].x);
                        acc[c].y = fmaf(ar, x[c].y, acc[c].y);
                        acc[c].y = fmaf(ai, x[c].x, acc[c].y);
                    }
                }
                sbar_arrive(s_u32(&empty[q]));   // this thread's reads of the tile are done
                // second half -> first half through a double buffer (bounded waits)
                const int rbuf = g & 1;
                cf *rb = red + rbuf * STR_ROWS * NC;
                if (h == 1) {
                    if (g >= 2 && !sbar_wait(s_u32(&red_empty[rbuf]), ((g >> 1) - 1) & 1)) {
                        fail(17);
                        ok = false;
                        break;
                    }
#pragma unroll
                    for (int c = 0; c < NC; ++c) rb[row * NC + c] = acc[c];
                    sbar_arrive(s_u32(&red_full[rbuf]));
                } else {
                    if (!sbar_wait(s_u32(&red_full[rbuf]), (g >> 1) & 1)) {
                        fail(18);
                        ok = false;
                        break;
                    }
                    const int i = tile_row(lo, hi, t) + row;
                    cf o[NC];
#pragma unroll
                    for (int c = 0; c < NC; ++c) o[c] = rb[row * NC + c];
                    sbar_arrive(s_u32(&red_empty[rbuf]));
                    if (i >= lo && i < hi) {
#pragma unroll
                        for (int c = 0; c < NC; ++c) {
                            cf &u = r[i * NC + c];
                            u.x -= acc[c].x + o[c].x;
                            u.y -= acc[c].y + o[c].y;
                        }
                    }
                    if (t == 0 && jj < nb - 1) sbar_arrive(s_u32(rows_ready));
                }
            }
            if (!ok) break;
        }
    }
}

__global__ void set_identity_kernel(float *W, int64_t ldw, int64_t plane, int64_t sW, int n) {
    const int64_t b = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    float *w = W + b * sW + (int64_t)j * ldw + i;
    w[0] = (i == j) ? 1.f : 0.f;
    w[plane] = 0.f;
}

}  // namespace

// Same product with four rows per thread and 16-byte loads (A's leading
// dimension, planes and batch stride multiples of 4 floats, A 16-byte
// aligned, m a multiple of 4): one vector load per plane brings four rows,
// so a thread keeps more of the matrix stream in flight per instruction.
template <int NC>
__global__ void __launch_bounds__(128) skinny4_kernel(int m, int n, int k, float alpha,
                                                      const float *__restrict__ A, int64_t lda,
                                                      int64_t planeA, int64_t sA,
                                                      const float *__restrict__ B, int64_t ldb,
                                                      int64_t planeB, int64_t sB, float beta,
                                                      float *__restrict__ C, int64_t ldc,
                                                      int64_t planeC, int64_t sC, int rnd) {
    __shared__ cf Bs[SK_KT][NC];
    const int64_t b = blockIdx.y;
    A += b * sA;
    B += b * sB;
    C += b * sC;
    const int row = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    cf acc[4][NC];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int j = 0; j < NC; ++j) acc[r][j] = fmk(0.f, 0.f);
    for (int k0 = 0; k0 < k; k0 += SK_KT) {
        __syncthreads();
        for (int e = threadIdx.x; e < SK_KT * NC; e += blockDim.x) {
            const int kk = e % SK_KT, j = e / SK_KT;
            Bs[kk][j] = (k0 + kk < k && j < n) ? ld(B, planeB, (int64_t)j * ldb + k0 + kk)
                                               : fmk(0.f, 0.f);
        }
        __syncthreads();
        if (row < m) {
            const int kend = min(SK_KT, k - k0);
            const float *ar = A + (int64_t)k0 * lda + row;
#pragma unroll 4
            for (int kk = 0; kk < kend; ++kk) {
                const float4 re = __ldg(reinterpret_cast<const float4 *>(ar + (int64_t)kk * lda));
                const float4 im =
                    __ldg(reinterpret_cast<const float4 *>(ar + (int64_t)kk * lda + planeA));
                const float ar4[4] = {re.x, re.y, re.z, re.w}, ai4[4] = {im.x, im.y, im.z, im.w};
#pragma unroll
                for (int j = 0; j < NC; ++j) {
                    const cf bv = Bs[kk][j];
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        acc[r][j].x = fmaf(ar4[r], bv.x, acc[r][j].x);
                        acc[r][j].x = fmaf(-ai4[r], bv.y, acc[r][j].x);
                        acc[r][j].y = fmaf(ar4[r], bv.y, acc[r][j].y);
                        acc[r][j].y = fmaf(ai4[r], bv.x, acc[r][j].y);
                    }
                }
            }
        }
    }
    if (row >= m) return;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        if (j < n) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int64_t o = (int64_t)j * ldc + row + r;
                cf c = beta != 0.f ? ld(C, planeC, o) : fmk(0.f, 0.f);
                cf v = fmk(alpha * acc[r][j].x + beta * c.x, alpha * acc[r][j].y + beta * c.y);
                if (rnd) v = fmk(tf32_rna(v.x), tf32_rna(v.y));
                st(C, planeC, o, v);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
Ctx::Ctx(cudaStream_t s_, int batch_, float *work_, int64_t work_bytes_)
    : s(s_), batch(batch_), work(work_), work_bytes(work_bytes_) {}

int gemm(Ctx &c, int m, int n, int k, float alpha, CMatF A, CMatF B, float beta, CMatF C,
         bool round_out, bool a_tf32) {
    if (m <= 0 || n <= 0) return MNPB_OK;
    if (k <= 0) {
        if (beta == 1.f) return MNPB_OK;
        set_error("f32 gemm: k = 0 with beta != 1 is not supported");
        return MNPB_EINVAL;
    }
    // four rows per thread only where that still leaves enough threads to
    // keep the GPU's memory pipes full (small batches of small matrices keep
    // one row per thread)
    const bool vec4 = n <= 4 && m % 4 == 0 && A.ld % 4 == 0 && A.plane % 4 == 0 &&
                      A.stride % 4 == 0 && ((uintptr_t)A.p & 15) == 0 &&
                      (int64_t)c.batch * (m / 4) >= (int64_t)device_sms() * 256;
    if (vec4) {
        dim3 grid(ceil_div(m, 512), c.batch);
        ProfScope ps(c.s, PC_SGEMM, 8.0 * (double)m * k * c.batch);   // bytes of A streamed
        prof_tag("M=%d N=%d K=%d B=%d v4", m, n, k, c.batch);
#define MNPB_SKINNY4(NC)                                                                        \
    skinny4_kernel<NC><<<grid, 128, 0, c.s>>>(m, n, k, alpha, A.p, A.ld, A.plane, A.stride,   \
                                              B.p, B.ld, B.plane, B.stride, beta, C.p, C.ld,  \
                                              C.plane, C.stride, round_out ? 1 : 0)
        if (n <= 1) MNPB_SKINNY4(1);
        else if (n <= 2) MNPB_SKINNY4(2);
        else MNPB_SKINNY4(4);
#undef MNPB_SKINNY4
        MNPB_LAUNCH_CHECK("skinny4_kernel");
        return MNPB_OK;
    }
    if (n <= SK_N) {
        dim3 grid(ceil_div(m, 128), c.batch);
        ProfScope ps(c.s, PC_SGEMM, 8.0 * (double)m * k * c.batch);   // bytes of A streamed
        prof_tag("M=%d N=%d K=%d B=%d", m, n, k, c.batch);
#define MNPB_SKINNY(NC)                                                                        \
    skinny_kernel<NC><<<grid, 128, 0, c.s>>>(m, n, k, alpha, A.p, A.ld, A.plane, A.stride, B.p, \
                                             B.ld, B.plane, B.stride, beta, C.p, C.ld, C.plane, \
                                             C.stride, round_out ? 1 : 0)
        if (n <= 1) MNPB_SKINNY(1);
        else if (n <= 2) MNPB_SKINNY(2);
        else if (n <= 4) MNPB_SKINNY(4);
        else if (n <= 8) MNPB_SKINNY(8);
        else MNPB_SKINNY(16);
#undef MNPB_SKINNY
        MNPB_LAUNCH_CHECK("skinny_kernel");
        return MNPB_OK;
    }
    return tc::cgemm_tf32(c.s, m, n, k, c.batch, alpha, A, B, beta, C, c.work, c.work_bytes,
                          round_out, a_tf32);
}

static int trsm_small(Ctx &c, int mode, int kb, CMatF T, CMatF B, int nvec) {
    if (nvec <= 0 || kb <= 0) return MNPB_OK;
    dim3 grid(ceil_div(nvec, 128), c.batch);
    ProfScope ps(c.s, PC_TRSM, 4.0 * kb * kb * (double)nvec * c.batch);
    prof_tag("mode=%d kb=%d nvec=%d B=%d", mode, kb, nvec, c.batch);
    trsm_small_kernel<<<grid, 128, 0, c.s>>>(mode, kb, T.p, T.ld, T.plane, T.stride, B.p, B.ld,
                                             B.plane, B.stride, nvec);
    MNPB_LAUNCH_CHECK("trsm_small_kernel(f32)");
    return MNPB_OK;
}

static int dev_sms() { return device_sms(); }

static int split_point(int n) {
    int h = n / 2;
    h = (h / TS) * TS;
    return h < TS ? TS : h;
}

// Triangular solves with many right-hand sides, recursive: split the
// triangle, solve one half, update the other half's right-hand sides with a
// tensor-core GEMM, solve the other half.  Two leaf kinds:
//  * 32-row leaves on CUDA cores (trsm_small) with splits at multiples of 32;
//  * when there are at least TL right-hand sides and the workspace holds
//    the inverses of the triangle's 128 x 128 diagonal blocks, 128-row
//    leaves applied as one tensor-core GEMM with the block's inverse (splits
//    at multiples of 128).  The leaf GEMM overwrites its own right-hand
//    sides: for a left solve (inverse as A, the RHS rows as B, C = B) each
//    output tile is a single 128-row tile whose columns no other tile reads,
//    and its epilogue runs after all of its loads; for a right solve the RHS
//    block is A and is copied into the packed operand before the GEMM.
//  mode 0 left lower unit, 1 left upper non-unit, 2 right upper non-unit,
//  3 right lower unit.
struct InvSet {
    const float *p;   // tri_inv_kernel output of the whole triangle
    int nb;           // 128-blocks of that triangle
};

static CMatF inv_block(const InvSet &iv, int blk) {
    return CMatF{(float *)iv.p + (int64_t)blk * 2 * TL * TL, TL, (int64_t)TL * TL,
                 (int64_t)iv.nb * 2 * TL * TL};
}

static int split_tl(int n) {
    int h = n / 2;
    h = (h / TL) * TL;
    return h < TL ? TL : h;
}

// `fresh`: B still holds the caller's right-hand side (not TF32); otherwise
// every update that wrote it stored its output rounded to nearest TF32, so a
// leaf reads it as an exact tensor-core operand without a rounding pass.
static int trsm_rec(Ctx &c, int mode, int n, int m, CMatF T, CMatF B, const InvSet *iv,
                    int blk0, bool fresh = true) {
    if (!iv && n <= TS) return trsm_small(c, mode, n, T, B, m);
    if (iv && n <= TL) {
        const CMatF I = inv_block(*iv, blk0);
        if (mode >= 2) {
            // right leaf: A is the right-hand-side block; packed with rounding
            // while fresh, read in place once the updates have rounded it
            if (fresh) return gemm(c, m, n, n, 1.f, B, I, 0.f, B, true);
            return gemm(c, m, n, n, 1.f, B, I, 0.f, B, true, true);
        }
        if (fresh) {
            ProfScope ps(c.s, PC_PACK, 16.0 * (double)n * m * c.batch);   // bytes read + written
            prof_tag("round n=%d m=%d B=%d", n, m, c.batch);
            round_tf32_kernel<<<dim3(ceil_div(m, RT_COLS), c.batch), TL, 0, c.s>>>(
                B.p, B.ld, B.plane, B.stride, n, m);
            MNPB_LAUNCH_CHECK("round_tf32_kernel");
        }
        return gemm(c, n, m, n, 1.f, I, B, 0.f, B, true, true);
    }
    const int n1 = iv ? split_tl(n) : split_point(n);
    const int blk1 = blk0 + n1 / TL;
    // the A operand of every update is TF32 already: a factor block (stored
    // rounded by the LU) or right-hand-side rows a leaf has finished (stored
    // rounded), so the tensor cores read it in place.  With the block
    // inverses (iv) the updates store their output rounded to TF32 as well,
    // for the leaves that read it next.
    const bool rnd = iv != nullptr;
    switch (mode) {
    case 0:
        MNPB_TRY(trsm_rec(c, 0, n1, m, T, B, iv, blk0, fresh));
        MNPB_TRY(gemm(c, n - n1, m, n1, -1.f, T.sub(n1, 0), B, 1.f, B.sub(n1, 0), rnd, true));
        return trsm_rec(c, 0, n - n1, m, T.sub(n1, n1), B.sub(n1, 0), iv, blk1, fresh && !rnd);
    case 1:
        MNPB_TRY(trsm_rec(c, 1, n - n1, m, T.sub(n1, n1), B.sub(n1, 0), iv, blk1, fresh));
        MNPB_TRY(gemm(c, n1, m, n - n1, -1.f, T.sub(0, n1), B.sub(n1, 0), 1.f, B, rnd, true));
        return trsm_rec(c, 1, n1, m, T, B, iv, blk0, fresh && !rnd);
    case 2:
        MNPB_TRY(trsm_rec(c, 2, n1, m, T, B, iv, blk0, fresh));
        MNPB_TRY(gemm(c, m, n - n1, n1, -1.f, B, T.sub(0, n1), 1.f, B.sub(0, n1), rnd, true));
        return trsm_rec(c, 2, n - n1, m, T.sub(n1, n1), B.sub(0, n1), iv, blk1, fresh && !rnd);
    default:
        MNPB_TRY(trsm_rec(c, 3, n - n1, m, T.sub(n1, n1), B.sub(0, n1), iv, blk1, fresh));
        MNPB_TRY(gemm(c, m, n1, n - n1, -1.f, B.sub(0, n1), T.sub(n1, 0), 1.f, B, rnd, true));
        return trsm_rec(c, 3, n1, m, T, B, iv, blk0, fresh && !rnd);
    }
}

// Packed-operand bytes of the largest GEMM trsm_rec issues with 128-leaves.
static int64_t trsm_pack_bytes(int mode, int n, int m, int batch) {
    const int big = n - split_tl(n) > TL ? n - split_tl(n) : TL;
    return mode < 2 ? tc::cgemm_tf32_workspace(big, big, batch)
                    : tc::cgemm_tf32_workspace(m, big, batch);
}

static int trsm(Ctx &c, int mode, int n, int m, CMatF T, CMatF B) {
    if (n <= 0 || m <= 0) return MNPB_OK;
    const int nb = ceil_div(n, TL);
    const int64_t inv_bytes = ((int64_t)c.batch * nb * 2 * TL * TL * 4 + 255) / 256 * 256;
    const int64_t keep = (c.work_bytes - inv_bytes) / 256 * 256;
    if (n <= TS || m < TL || keep < trsm_pack_bytes(mode, n, m, c.batch))
        return trsm_rec(c, mode, n, m, T, B, nullptr, 0);
    MNPB_TRY(smem_opt_in(tri_inv_kernel, TL * TL * (int)sizeof(cf), "tri_inv_kernel"));
    float *inv = (float *)((char *)c.work + keep);
    {
        dim3 grid(nb, c.batch);
        ProfScope ps(c.s, PC_TRSM, 8.0 * TL * TL * TL / 3.0 * nb * c.batch);
        prof_tag("tri_inv n=%d B=%d %s", n, c.batch, (mode == 0 || mode == 3) ? "L" : "U");
        tri_inv_kernel<<<grid, TINV_THREADS, TL * TL * sizeof(cf), c.s>>>(
            n, (mode == 0 || mode == 3) ? 1 : 0, T.p, T.ld, T.plane, T.stride, inv, nb);
        MNPB_LAUNCH_CHECK("tri_inv_kernel");
    }
    Ctx c2(c.s, c.batch, c.work, keep);
    const InvSet iv{inv, nb};
    return trsm_rec(c2, mode, n, m, T, B, &iv, 0);
}

// ---- inverse of an LU factorisation: A^-1 = U^-1 L^-1 P^T ---------------------
// Copy of each matrix's n x n diagonal-block inverse (planar, ld TL) into X.
__global__ void copy_inv_block_kernel(int n, const float *__restrict__ inv, int64_t sinv,
                                      float *X, int64_t ldx, int64_t plane, int64_t sX) {
    const int64_t b = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= n) return;
    const float *src = inv + b * sinv + (int64_t)j * TL + i;
    float *dst = X + b * sX + (int64_t)j * ldx + i;
    dst[0] = src[0];
    dst[plane] = src[(int64_t)TL * TL];
}

// X <- L^-1 for the unit lower factor in T, with X holding the identity on
// entry: the rows of an identity column above its diagonal stay zero, so
// X11 = L11^-1 (recursively), X21 = -L22^-1 (L21 X11) (one product and one
// general solve with n1 right-hand sides), X22 = L22^-1 (recursively), and a
// leaf is the stored inverse of its diagonal block -- a quarter fewer flops
// than solving against the full identity.
static int trsm_llu_eye_rec(Ctx &c, int n, CMatF T, CMatF X, const InvSet &iv, int blk0) {
    if (n <= TL) {
        const CMatF I = inv_block(iv, blk0);
        dim3 grid(ceil_div(n, 128), n, c.batch);
        copy_inv_block_kernel<<<grid, 128, 0, c.s>>>(n, I.p, I.stride, X.p, X.ld, X.plane,
                                                     X.stride);
        MNPB_LAUNCH_CHECK("copy_inv_block_kernel");
        return MNPB_OK;
    }
    const int n1 = split_tl(n);
    const int blk1 = blk0 + n1 / TL;
    MNPB_TRY(trsm_llu_eye_rec(c, n1, T, X, iv, blk0));
    MNPB_TRY(gemm(c, n - n1, n1, n1, -1.f, T.sub(n1, 0), X, 0.f, X.sub(n1, 0), true, true));
    MNPB_TRY(trsm_rec(c, 0, n - n1, n1, T.sub(n1, n1), X.sub(n1, 0), &iv, blk1, false));
    return trsm_llu_eye_rec(c, n - n1, T.sub(n1, n1), X.sub(n1, n1), iv, blk1);
}

int lu_inverse(Ctx &c, int n, CMatF LU, const int32_t *ipiv, int64_t sP, CMatF X) {
    MNPB_TRY(set_identity(c, n, X));
    const int nb = ceil_div(n, TL);
    const int64_t inv_bytes = ((int64_t)c.batch * nb * 2 * TL * TL * 4 + 255) / 256 * 256;
    const int64_t keep = (c.work_bytes - inv_bytes) / 256 * 256;
    if (n <= TL || keep < trsm_pack_bytes(0, n, n, c.batch)) {
        // no room for the block inverses: the plain getrs on the permuted identity
        MNPB_TRY(laswp(c, X, 0, n, ipiv, sP, 0, n, true));
        MNPB_TRY(trsm_llu(c, n, n, LU, X));
        return trsm_lun(c, n, n, LU, X);
    }
    MNPB_TRY(smem_opt_in(tri_inv_kernel, TL * TL * (int)sizeof(cf), "tri_inv_kernel"));
    float *inv = (float *)((char *)c.work + keep);
    {
        dim3 grid(nb, c.batch);
        ProfScope ps(c.s, PC_TRSM, 8.0 * TL * TL * TL / 3.0 * nb * c.batch);
        prof_tag("tri_inv n=%d B=%d L", n, c.batch);
        tri_inv_kernel<<<grid, TINV_THREADS, TL * TL * sizeof(cf), c.s>>>(
            n, 1, LU.p, LU.ld, LU.plane, LU.stride, inv, nb);
        MNPB_LAUNCH_CHECK("tri_inv_kernel");
    }
    Ctx c2(c.s, c.batch, c.work, keep);
    MNPB_TRY(trsm_llu_eye_rec(c2, n, LU, X, InvSet{inv, nb}, 0));
    MNPB_TRY(trsm_lun(c, n, n, LU, X));
    // X <- X P^T: the row interchanges of the factorisation, as column
    // interchanges in reverse order
    dim3 grid(ceil_div(n, 128), c.batch);
    ProfScope ps(c.s, PC_SWAP, 0.0);
    colswp_kernel<<<grid, 128, 0, c.s>>>(X.p, X.ld, X.plane, X.stride, n, ipiv, sP, n);
    MNPB_LAUNCH_CHECK("colswp_kernel(f32)");
    return MNPB_OK;
}

int trsm_llu(Ctx &c, int n, int m, CMatF L, CMatF B) { return trsm(c, 0, n, m, L, B); }
int trsm_lun(Ctx &c, int n, int m, CMatF U, CMatF B) { return trsm(c, 1, n, m, U, B); }
int trsm_run(Ctx &c, int n, int m, CMatF U, CMatF B) { return trsm(c, 2, n, m, U, B); }
int trsm_rlu(Ctx &c, int n, int m, CMatF L, CMatF B) { return trsm(c, 3, n, m, L, B); }

int laswp(Ctx &c, CMatF A, int j0, int j1, const int32_t *ipiv, int64_t sP, int c0, int c1,
          bool forward) {
    if (j1 <= j0 || c1 <= c0) return MNPB_OK;
    dim3 grid(ceil_div(j1 - j0, 128), c.batch);
    ProfScope ps(c.s, PC_SWAP, 0.0);
    SwpSegs none{};
    laswp_kernel<<<grid, 128, 0, c.s>>>(A.p, A.ld, A.plane, A.stride, j0, j1, ipiv, sP, c0, c1,
                                        forward ? 1 : 0, none, 0);
    MNPB_LAUNCH_CHECK("laswp_kernel(f32)");
    return MNPB_OK;
}

// One launch of the segment table t (forward order): columns [t.brk[0],
// t.brk[t.n]), interchanges from the smallest segment start to t.end.
static int laswp_segs(Ctx &c, CMatF A, const int32_t *ipiv, int64_t sP, const SwpSegs &t) {
    if (t.n == 0) return MNPB_OK;
    int c0 = t.end;
    for (int q = 0; q < t.n; ++q) c0 = min(c0, t.cs[q]);
    const int j0 = t.brk[0], j1 = t.brk[t.n];
    if (j1 <= j0 || t.end <= c0) return MNPB_OK;
    dim3 grid(ceil_div(j1 - j0, 128), c.batch);
    ProfScope ps(c.s, PC_SWAP, 0.0);
    laswp_kernel<<<grid, 128, 0, c.s>>>(A.p, A.ld, A.plane, A.stride, j0, j1, ipiv, sP, c0,
                                        t.end, 1, t, 1);
    MNPB_LAUNCH_CHECK("laswp_kernel(f32, segments)");
    return MNPB_OK;
}

// append segment [j0, j1) -> interchanges [cs, t.end) to table t
static int seg_push(SwpSegs &t, int j0, int j1, int cs) {
    if (j1 <= j0) return MNPB_OK;
    if (t.n >= SWP_MAXSEG) {
        set_error("getrf: interchange segment table full");
        return MNPB_EINVAL;
    }
    if (t.n == 0) t.brk[0] = j0;
    if (t.brk[t.n] != j0) {               // gap: nothing owed there
        t.cs[t.n] = t.end;
        t.brk[++t.n] = j0;
        if (t.n >= SWP_MAXSEG) {
            set_error("getrf: interchange segment table full");
            return MNPB_EINVAL;
        }
    }
    t.cs[t.n] = cs;
    t.brk[++t.n] = j1;
    return MNPB_OK;
}

// Factor columns [off, off+w) over rows [off, n) of the full matrix A;
// pivots are absolute row indices.  The backward interchanges this node's
// columns still owe (its right half's pivots on its left half, and what its
// right half owes) are returned in `owed` (pivots up to off + w) instead of
// applied: the caller applies them in its next interchange launch, together
// with its own forward interchanges, before anything reads these columns.
static int rgetrf(Ctx &c, int n, int off, int w, CMatF A, int32_t *ipiv, int64_t sP,
                  int32_t *info, SwpSegs &owed) {
    owed.n = 0;
    owed.end = off + w;
    if (w <= TS) {
        ProfScope ps(c.s, PC_PANEL, 8.0 * w * w * (double)(n - off) * c.batch / 2);
        prof_tag("off=%d w=%d B=%d", off, w, c.batch);
        MNPB_TRY(smem_opt_in(panel_slab_kernel<8>, 200 * 1024, "panel_slab_kernel<8>"));
        MNPB_TRY(smem_opt_in(panel_slab_kernel<4>, 200 * 1024, "panel_slab_kernel<4>"));
        // more matrices than SMs: 4-column slabs, half the shared memory, so
        // that two CTAs share an SM and the batch runs in one wave
        const int64_t slab8 = (int64_t)8 * (n - off) * 8, slab4 = slab8 / 2;
        if (c.batch > dev_sms() && w % 4 == 0 && w <= TS && slab4 <= 100 * 1024) {
            panel_slab_kernel<4><<<c.batch, SLAB_THREADS, (size_t)slab4, c.s>>>(
                n, off, w, A.p, A.ld, A.plane, A.stride, ipiv, sP, info);
            MNPB_LAUNCH_CHECK("panel_slab_kernel<4>(f32)");
            return MNPB_OK;
        }
        if (w % 8 == 0 && w <= TS && slab8 <= 200 * 1024) {
            panel_slab_kernel<8><<<c.batch, SLAB_THREADS, (size_t)slab8, c.s>>>(
                n, off, w, A.p, A.ld, A.plane, A.stride, ipiv, sP, info);
            MNPB_LAUNCH_CHECK("panel_slab_kernel(f32)");
            return MNPB_OK;
        }
        panel_kernel<<<c.batch, PANEL_THREADS, 0, c.s>>>(n, off, w, A.p, A.ld, A.plane, A.stride,
                                                         ipiv, sP, info);
        MNPB_LAUNCH_CHECK("panel_kernel(f32)");
        return MNPB_OK;
    }
    const int w1 = split_point(w);
    SwpSegs pl;
    MNPB_TRY(rgetrf(c, n, off, w1, A, ipiv, sP, info, pl));
    // one launch: what the left half owes (pivots up to off + w1) and the
    // left half's pivots on the right half's columns
    SwpSegs t = pl;
    MNPB_TRY(seg_push(t, off + w1, off + w, off));
    MNPB_TRY(laswp_segs(c, A, ipiv, sP, t));
    MNPB_TRY(trsm_llu(c, w1, w - w1, A.sub(off, off), A.sub(off, off + w1)));
    // L21 is stored rounded to TF32 by the panels: read in place
    MNPB_TRY(gemm(c, n - off - w1, w - w1, w1, -1.f, A.sub(off + w1, off),
                  A.sub(off, off + w1), 1.f, A.sub(off + w1, off + w1), false, true));
    SwpSegs pr;
    MNPB_TRY(rgetrf(c, n, off + w1, w - w1, A, ipiv, sP, info, pr));
    // owed: the right half's pivots on the left half's columns, and what the
    // right half owes (both up to off + w)
    MNPB_TRY(seg_push(owed, off, off + w1, off + w1));
    for (int q = 0; q < pr.n; ++q) MNPB_TRY(seg_push(owed, pr.brk[q], pr.brk[q + 1], pr.cs[q]));
    return MNPB_OK;
}

int getrf(Ctx &c, int n, CMatF A, int32_t *ipiv, int64_t sP, int32_t *info) {
    SwpSegs owed;
    MNPB_TRY(rgetrf(c, n, 0, n, A, ipiv, sP, info, owed));
    return laswp_segs(c, A, ipiv, sP, owed);
}

int getrs(Ctx &c, int n, int nrhs, CMatF LU, const int32_t *ipiv, int64_t sP, CMatF B) {
    MNPB_TRY(laswp(c, B, 0, nrhs, ipiv, sP, 0, n, true));
    MNPB_TRY(trsm_llu(c, n, nrhs, LU, B));
    return trsm_lun(c, n, nrhs, LU, B);
}

int right_solve(Ctx &c, int n, int m, CMatF LU, const int32_t *ipiv, int64_t sP, CMatF B) {
    MNPB_TRY(trsm_run(c, n, m, LU, B));
    MNPB_TRY(trsm_rlu(c, n, m, LU, B));
    dim3 grid(ceil_div(m, 128), c.batch);
    ProfScope ps(c.s, PC_SWAP, 0.0);
    colswp_kernel<<<grid, 128, 0, c.s>>>(B.p, B.ld, B.plane, B.stride, m, ipiv, sP, n);
    MNPB_LAUNCH_CHECK("colswp_kernel(f32)");
    return MNPB_OK;
}

// ---- few-RHS solves ---------------------------------------------------------
int64_t trsv_state_bytes(int n, int batch) {
    return ((int64_t)ceil_div(n, TB) * batch + 64) * sizeof(int);
}

int64_t diag_inv_floats(int n, int batch) { return (int64_t)batch * ceil_div(n, TB) * 2 * TB * TB; }

int diag_inv(Ctx &c, int n, CMatF LU, float *invL, float *invU) {
    const int nb = ceil_div(n, TB);
    dim3 grid(nb, c.batch);
    ProfScope ps(c.s, PC_TRSM, 0.0);
    diag_inv_kernel<<<grid, TB, 0, c.s>>>(n, 1, LU.p, LU.ld, LU.plane, LU.stride, invL, nb);
    MNPB_LAUNCH_CHECK("diag_inv_kernel(L)");
    diag_inv_kernel<<<grid, TB, 0, c.s>>>(n, 0, LU.p, LU.ld, LU.plane, LU.stride, invU, nb);
    MNPB_LAUNCH_CHECK("diag_inv_kernel(U)");
    return MNPB_OK;
}

// state: caller-provided device scratch of trsv_state_bytes(n, batch) bytes
// (flags per block and the ticket counter), cleared before each launch.
template <int NC>
static int trsv_rl(Ctx &c, bool lower, int n, int m, CMatF T, const float *inv, CMatF X) {
    const int nb = ceil_div(n, TB);
    const int dyn = n * NC * (int)sizeof(cf);
    if (dyn > 48 * 1024) MNPB_TRY(smem_opt_in(trsv_rl_kernel<NC>, dyn, "trsv_rl_kernel"));
    ProfScope ps(c.s, PC_TRSV, 4.0 * (double)n * n * c.batch);   // bytes of the triangle
    prof_tag("n=%d m=%d B=%d %s", n, m, c.batch, lower ? "L" : "U");
    trsv_rl_kernel<NC><<<c.batch, RL_THREADS, dyn, c.s>>>(n, m, lower ? 1 : 0, T.p, T.ld, T.plane,
                                                         T.stride, inv, X.p, X.ld, X.plane,
                                                         X.stride, nb);
    MNPB_LAUNCH_CHECK("trsv_rl_kernel");
    return MNPB_OK;
}

// Shared memory of trsv_stream_kernel<NC> with S ring stages (0 if too large).
static int stream_smem(int n, int nc, int S) {
    const int64_t b = 1024 + (int64_t)S * STR_TILE_BYTES + 2 * 2 * TB * TB * 4 +
                      2 * TB * nc * (int64_t)sizeof(cf) + 2 * STR_ROWS * nc * (int64_t)sizeof(cf) +
                      (int64_t)n * nc * sizeof(cf) + (2 * S + 11) * 8 + 16;
    return b <= 220 * 1024 ? (int)b : 0;
}

template <int NC>
static int trsv_stream(Ctx &c, bool lower, int n, int m, CMatF T, const float *inv, CMatF X,
                       int S) {
    const int nb = ceil_div(n, TB);
    const int smem = stream_smem(n, NC, S);
    MNPB_TRY(smem_opt_in(trsv_stream_kernel<NC>, smem, "trsv_stream_kernel"));
    CUtensorMap mr, mi;
    const uint64_t dims[3] = {(uint64_t)n, (uint64_t)n, (uint64_t)c.batch};
    const uint64_t strides[2] = {(uint64_t)T.ld * 4, (uint64_t)T.stride * 4};
    const uint32_t box[3] = {STR_ROWS, TB, 1};
    MNPB_TRY(tc::encode_map_f32(&mr, T.p, dims, strides, box, 0));
    MNPB_TRY(tc::encode_map_f32(&mi, T.p + T.plane, dims, strides, box, 0));
    ProfScope ps(c.s, PC_TRSV, 4.0 * (double)n * n * c.batch);   // bytes of the triangle
    prof_tag("n=%d m=%d B=%d %s stream", n, m, c.batch, lower ? "L" : "U");
    trsv_stream_kernel<NC><<<c.batch, STR_THREADS, smem, c.s>>>(
        mr, mi, n, m, lower ? 1 : 0, inv, X.p, X.ld, X.plane, X.stride, nb, S);
    MNPB_LAUNCH_CHECK("trsv_stream_kernel");
    return MNPB_OK;
}

static int trsv(Ctx &c, bool lower, int n, int m, CMatF T, const float *inv, CMatF X,
                int *state) {
    // triangle streamed by TMA when it is 16-byte aligned and the ring fits
    // beside the right-hand sides in shared memory
    const bool a16 = ((uintptr_t)T.p & 15) == 0 && T.ld % 4 == 0 && T.plane % 4 == 0 &&
                     T.stride % 4 == 0 && ((uintptr_t)inv & 15) == 0;
    if (a16 && m <= 4) {
        const int nc = m <= 1 ? 1 : 4;
        int S = 6;
        while (S >= 2 && stream_smem(n, nc, S) == 0) --S;
        if (S >= 2)
            return nc == 1 ? trsv_stream<1>(c, lower, n, m, T, inv, X, S)
                           : trsv_stream<4>(c, lower, n, m, T, inv, X, S);
    }
    // one CTA per matrix when the right-hand sides fit in shared memory and
    // the triangle allows 8-byte row-pair loads
    const bool even = ((uintptr_t)T.p & 7) == 0 && T.ld % 2 == 0 && T.plane % 2 == 0 &&
                      T.stride % 2 == 0;
    if (even && m <= 8) {
        const int nc = m <= 1 ? 1 : m <= 4 ? 4 : 8;
        if ((int64_t)n * nc * (int64_t)sizeof(cf) <= 200 * 1024) {
            if (nc == 1) return trsv_rl<1>(c, lower, n, m, T, inv, X);
            if (nc == 4) return trsv_rl<4>(c, lower, n, m, T, inv, X);
            return trsv_rl<8>(c, lower, n, m, T, inv, X);
        }
    }
    const int nb = ceil_div(n, TB);
    int *flags = state;
    unsigned *ticket = (unsigned *)(state + (int64_t)nb * c.batch);
    if (cudaMemsetAsync(state, 0, trsv_state_bytes(n, c.batch), c.s) != cudaSuccess) {
        set_error("trsv: memset failed");
        return MNPB_ECUDA;
    }
    const int grid = nb * c.batch;
    ProfScope ps(c.s, PC_TRSV, 4.0 * (double)n * n * c.batch);   // bytes of the triangle
    prof_tag("n=%d m=%d B=%d %s", n, m, c.batch, lower ? "L" : "U");
#define MNPB_TRSV(NC)                                                                          \
    trsv_kernel<NC><<<grid, 256, 0, c.s>>>(n, m, lower ? 1 : 0, T.p, T.ld, T.plane, T.stride,   \
                                           inv, X.p, X.ld, X.plane, X.stride, flags, ticket, 1, \
                                           nb, c.batch)
    if (m <= 4) MNPB_TRSV(4);
    else if (m <= 8) MNPB_TRSV(8);
    else MNPB_TRSV(16);
#undef MNPB_TRSV
    MNPB_LAUNCH_CHECK("trsv_kernel");
    return MNPB_OK;
}

int getrs_few(Ctx &c, int n, int m, CMatF LU, const int32_t *ipiv, int64_t sP,
              const float *invL, const float *invU, CMatF B, int *state) {
    if (m > 16) return getrs(c, n, m, LU, ipiv, sP, B);
    MNPB_TRY(laswp(c, B, 0, m, ipiv, sP, 0, n, true));
    MNPB_TRY(trsv(c, true, n, m, LU, invL, B, state));
    return trsv(c, false, n, m, LU, invU, B, state);
}

// Failure-path probe of the triangular solves' two wait helpers: kind 1
// spins with wait_flag on a zeroed flag for the value 1 (which nothing
// writes), kind 2 waits with sbar_wait on an mbarrier that expects one
// arrival and never gets it.  Each gives up after `limit_ns`, records code 9
// in the error word as a solve would, and returns.
__global__ void trsv_wait_probe_kernel(int kind, const int *flag, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    bool ok;
    if (kind == 1) {
        ok = wait_flag(flag, 1, limit_ns);
    } else {
        const uint32_t b = s_u32(&bar);
        sbar_init(b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        ok = sbar_wait(b, 0, limit_ns);
    }
    if (!ok) atomicCAS(&g_trsv_error, 0, 9);
}

int trsv_wait_probe(cudaStream_t s, int kind, int *flag, uint64_t limit_ns) {
    if (cudaMemsetAsync(flag, 0, sizeof(int), s) != cudaSuccess) {
        set_error("trsv_wait_probe: cannot clear the flag");
        return MNPB_ECUDA;
    }
    trsv_wait_probe_kernel<<<1, 1, 0, s>>>(kind, flag, limit_ns);
    MNPB_LAUNCH_CHECK("trsv_wait_probe_kernel");
    return MNPB_OK;
}

int trsv_error_read_and_clear(cudaStream_t s, int *code) {
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbolAsync(&v, g_trsv_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyToSymbolAsync(g_trsv_error, &z, sizeof(int), 0, cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("trsv: cannot read the error word");
        return MNPB_ECUDA;
    }
    *code = v;
    return MNPB_OK;
}

int set_identity(Ctx &c, int n, CMatF W) {
    dim3 grid(ceil_div(n, 128), n, c.batch);
    set_identity_kernel<<<grid, 128, 0, c.s>>>(W.p, W.ld, W.plane, W.stride, n);
    MNPB_LAUNCH_CHECK("set_identity_kernel(f32)");
    return MNPB_OK;
}

}  // namespace f32
}  // namespace mnpb

using namespace mnpb;

extern "C" int64_t mnpb_f32_workspace(int64_t n, int64_t batch) {
    // packed-A buffer of the largest tensor-core GEMM the recursions issue
    return tc::cgemm_tf32_workspace((int)n, (int)n, (int)batch);
}

extern "C" int mnpb_getrf_c32p(void *stream, int64_t n, int64_t batch, float *A, int64_t ld,
                               int64_t plane, int64_t stride, int32_t *piv, int64_t pstride,
                               int32_t *info, void *work, int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && batch < 65536 && ld >= n, "getrf_c32p: bad sizes");
    MNPB_REQUIRE(A && piv && work, "getrf_c32p: null pointer");
    MNPB_REQUIRE(ld % 4 == 0 && plane % 4 == 0 && stride % 4 == 0 && ((uintptr_t)A & 15) == 0,
                 "getrf_c32p: ld, plane and stride must be multiples of 4 floats and A 16-byte "
                 "aligned");
    f32::Ctx c(as_stream(stream), (int)batch, (float *)work, work_bytes);
    return f32::getrf(c, (int)n, tc::CMatF{A, ld, plane, stride}, piv, pstride, info);
}

extern "C" int mnpb_getri_c32p(void *stream, int64_t n, int64_t batch, const float *LU,
                               int64_t ld, int64_t plane, int64_t stride, const int32_t *piv,
                               int64_t pstride, float *X, int64_t ldx, int64_t planeX,
                               int64_t xstride, void *work, int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && ld >= n && ldx >= n, "getri_c32p: bad sizes");
    MNPB_REQUIRE(ld % 4 == 0 && plane % 4 == 0 && stride % 4 == 0 && ldx % 4 == 0 &&
                     planeX % 4 == 0 && xstride % 4 == 0 && ((uintptr_t)LU & 15) == 0 &&
                     ((uintptr_t)X & 15) == 0,
                 "getri_c32p: leading dimensions, planes and strides must be multiples of 4 "
                 "floats and base pointers 16-byte aligned");
    MNPB_REQUIRE(LU && piv && X && work, "getri_c32p: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_f32_workspace(n, batch), "getri_c32p: workspace too small");
    f32::Ctx c(as_stream(stream), (int)batch, (float *)work, work_bytes);
    return f32::lu_inverse(c, (int)n, tc::CMatF{(float *)LU, ld, plane, stride}, piv, pstride,
                           tc::CMatF{X, ldx, planeX, xstride});
}

extern "C" int mnpb_getrs_c32p(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                               const float *LU, int64_t ld, int64_t plane, int64_t stride,
                               const int32_t *piv, int64_t pstride, float *B, int64_t ldb,
                               int64_t planeB, int64_t bstride, void *work, int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && nrhs > 0 && ld >= n && ldb >= n, "getrs_c32p: bad sizes");
    MNPB_REQUIRE(ld % 4 == 0 && plane % 4 == 0 && stride % 4 == 0 && ldb % 4 == 0 &&
                     planeB % 4 == 0 && bstride % 4 == 0 && ((uintptr_t)LU & 15) == 0 &&
                     ((uintptr_t)B & 15) == 0,
                 "getrs_c32p: leading dimensions, planes and strides must be multiples of 4 "
                 "floats and base pointers 16-byte aligned");
    MNPB_REQUIRE(LU && piv && B && work, "getrs_c32p: null pointer");
    f32::Ctx c(as_stream(stream), (int)batch, (float *)work, work_bytes);
    return f32::getrs(c, (int)n, (int)nrhs, tc::CMatF{(float *)LU, ld, plane, stride}, piv,
                      pstride, tc::CMatF{B, ldb, planeB, bstride});
}

// ---------------------------------------------------------------------------
// Failure-path probe of the bounded device waits (see the header).
// ---------------------------------------------------------------------------
#include "tc_gemm.cuh"

extern "C" int mnpb_wait_probe(void *stream, int32_t kind, int64_t limit_ns, int32_t *flag) {
    using namespace mnpb;
    clear_error();
    MNPB_REQUIRE(kind >= 0 && kind <= 2, "wait_probe: kind must be 0, 1 or 2");
    MNPB_REQUIRE(limit_ns > 0 && limit_ns <= 2000000000ll, "wait_probe: limit_ns in (0, 2e9]");
    MNPB_REQUIRE(kind != 1 || flag, "wait_probe: kind 1 needs a device int");
    cudaStream_t s = as_stream(stream);
    int code = 0;
    if (kind == 0) {
        MNPB_TRY(tc::wait_probe(s, (uint64_t)limit_ns));
        MNPB_TRY(tc::tc_error_read_and_clear(s, &code));
    } else {
        MNPB_TRY(f32::trsv_wait_probe(s, kind, (int *)flag, (uint64_t)limit_ns));
        MNPB_TRY(f32::trsv_error_read_and_clear(s, &code));
    }
    if (code) {
        set_error("wait_probe: the %s wait gave up after %lld ns (error word %d)",
                  kind == 0 ? "tensor-core mbarrier" : kind == 1 ? "triangular-solve flag"
                                                                 : "triangular-solve mbarrier",
                  (long long)limit_ns, code);
        return MNPB_ETIMEOUT;
    }
    return MNPB_OK;
}
