// H-matrix kernels of the iterative retarded solver:
//
//  * partially-pivoted ACA of every low-rank block, one CTA per block, in FP64
//    from the dense FP64 matrix (the reference samples its dense matrix the
//    same way, mnpbem/greenfun/aca_compgreen_ret.py:196-208 and
//    mnpbem/greenfun/hmatrix.py:195-336);
//  * gather of the dense (leaf x leaf) blocks and compaction of the ACA
//    factors into complex64 storage;
//  * H-matrix times a few vectors (hmatrix.py:450-541) in two bandwidth-bound
//    launches: t_b = V_b^T x for every low-rank block, then one CTA per leaf
//    cluster sums the dense and U_b t_b contributions of its rows.  Each row
//    has exactly one writer, so the result is deterministic (no atomics);
//    factors are read as complex64 and accumulated in FP64;
//  * the packed 8N BEM operator on top of the four products
//    (mnpb_bem_afun, mnpbem/bem/bem_ret_iter.py:1362-1501, scalar eps).
//
// Matrices are column-major complex128 (A[i + j * lda]) in face order; block
// coordinates are cluster positions, mapped to faces by c2p.
#include "common.cuh"

namespace mnpb {
namespace hm {

constexpr int ACA_T = 256;
constexpr int ACA_MAXK = 128;   // largest supported kmax

// complex arithmetic without contraction (same rounding as NumPy's complex
// multiply a*b = (ar br - ai bi, ar bi + ai br))
__device__ __forceinline__ cd mul_nf(cd a, cd b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ cd sub_nf(cd a, cd b) {
    return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
// Smith's complex division (R. L. Smith, CACM 5, 435 (1962)), the algorithm
// NumPy's complex divide uses; b != 0 here.
__device__ __forceinline__ cd div_smith(cd a, cd b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double rat = __ddiv_rn(b.y, b.x);
        const double scl = __ddiv_rn(1.0, __dadd_rn(b.x, __dmul_rn(b.y, rat)));
        return make_double2(__dmul_rn(__dadd_rn(a.x, __dmul_rn(a.y, rat)), scl),
                            __dmul_rn(__dsub_rn(a.y, __dmul_rn(a.x, rat)), scl));
    }
    const double rat = __ddiv_rn(b.x, b.y);
    const double scl = __ddiv_rn(1.0, __dadd_rn(b.y, __dmul_rn(b.x, rat)));
    return make_double2(__dmul_rn(__dadd_rn(__dmul_rn(a.x, rat), a.y), scl),
                        __dmul_rn(__dsub_rn(__dmul_rn(a.y, rat), a.x), scl));
}
__device__ __forceinline__ cd cconj_mul(cd a, cd b) {   // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

struct ArgMax {
    double v;
    int i;
};
// larger value wins; on equal values the smaller index (np.argmax's first hit)
__device__ __forceinline__ ArgMax amax(ArgMax a, ArgMax b) {
    if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
    return a;
}
__device__ ArgMax block_argmax(ArgMax a, ArgMax *sh) {
    for (int o = 16; o > 0; o >>= 1) {
        ArgMax b{__shfl_xor_sync(0xffffffffu, a.v, o), __shfl_xor_sync(0xffffffffu, a.i, o)};
        a = amax(a, b);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        ArgMax r = sh[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = amax(r, sh[k]);
        sh[0] = r;
    }
    __syncthreads();
    return sh[0];
}
__device__ double block_sum(double a, double *sh) {
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
        sh[0] = r;
    }
    __syncthreads();
    return sh[0];
}

// One CTA per low-rank block.  U (m x cap) and V (n x cap) are column-major
// FP64 scratch at UV + offU[b] / offV[b]; the block is ~ U V^T with the rank
// written to rank_out[b].  Dynamic shared memory: m + n used-flags.
__global__ void __launch_bounds__(ACA_T) aca_kernel(const cd *__restrict__ A, int64_t lda,
                                                    const int *__restrict__ c2p,
                                                    const int4 *__restrict__ blk,
                                                    const int64_t *__restrict__ offU,
                                                    const int64_t *__restrict__ offV, int kmax,
                                                    double htol, cd *UV, int *rank_out) {
    extern __shared__ unsigned char used[];
    __shared__ cd sk[ACA_MAXK];
    __shared__ ArgMax sa[32];
    __shared__ double sd[32];
    __shared__ double cross[ACA_MAXK];
    __shared__ int s_stop;
    const int4 bk = blk[blockIdx.x];
    const int r0 = bk.x, m = bk.y, c0 = bk.z, n = bk.w;
    const int cap = min(min(m, n), kmax);
    cd *U = UV + offU[blockIdx.x];
    cd *V = UV + offV[blockIdx.x];
    for (int e = threadIdx.x; e < m + n; e += blockDim.x) used[e] = 0;
    int rank = 0, prow = 0;
    double fro = 0.0;
    __syncthreads();
    for (int it = 0; it < cap; ++it) {
        // residual row prow: A(prow, :) - sum_r U[prow, r] V[:, r]
        for (int r = threadIdx.x; r < rank; r += blockDim.x) sk[r] = U[prow + (int64_t)r * m];
        __syncthreads();
        const int64_t grow = c2p[r0 + prow];
        ArgMax best{-1.0, 0x7fffffff};
        double vsq = 0.0;
        cd *vrow = V + (int64_t)rank * n;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            cd v = A[grow + (int64_t)c2p[c0 + j] * lda];
            for (int r = 0; r < rank; ++r) v = sub_nf(v, mul_nf(sk[r], V[j + (int64_t)r * n]));
            vrow[j] = v;
            vsq += v.x * v.x + v.y * v.y;
            const double a = used[m + j] ? 0.0 : hypot(v.x, v.y);
            best = amax(best, ArgMax{a, j});
        }
        best = block_argmax(best, sa);
        const int pcol = best.i;
        vsq = block_sum(vsq, sd);
        const cd piv = vrow[pcol];
        if (hypot(piv.x, piv.y) < 1e-15) break;
        // residual column pcol, divided by the pivot
        for (int r = threadIdx.x; r < rank; r += blockDim.x) sk[r] = V[pcol + (int64_t)r * n];
        __syncthreads();
        const int64_t gcol = (int64_t)c2p[c0 + pcol] * lda;
        cd *ucol = U + (int64_t)rank * m;
        ArgMax nextr{-1.0, 0x7fffffff};
        double usq = 0.0;
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            cd c = A[c2p[r0 + i] + gcol];
            for (int r = 0; r < rank; ++r) c = sub_nf(c, mul_nf(sk[r], U[i + (int64_t)r * m]));
            const cd u = div_smith(c, piv);
            ucol[i] = u;
            usq += u.x * u.x + u.y * u.y;
            const double a = (used[i] || i == prow) ? 0.0 : hypot(u.x, u.y);
            nextr = amax(nextr, ArgMax{a, i});
        }
        nextr = block_argmax(nextr, sa);
        usq = block_sum(usq, sd);
        ++rank;
        // cross terms 2 Re(<U_j, u><V_j, v>) for the earlier columns, one warp per j
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        for (int j = w; j < rank - 1; j += (int)(blockDim.x >> 5)) {
            cd du = cmk(0, 0), dv = cmk(0, 0);
            for (int i = l; i < m; i += 32) du = cadd(du, cconj_mul(U[i + (int64_t)j * m], ucol[i]));
            for (int i = l; i < n; i += 32) dv = cadd(dv, cconj_mul(V[i + (int64_t)j * n], vrow[i]));
            for (int o = 16; o > 0; o >>= 1) {
                du.x += __shfl_xor_sync(0xffffffffu, du.x, o);
                du.y += __shfl_xor_sync(0xffffffffu, du.y, o);
                dv.x += __shfl_xor_sync(0xffffffffu, dv.x, o);
                dv.y += __shfl_xor_sync(0xffffffffu, dv.y, o);
            }
            if (l == 0) cross[j] = 2.0 * (du.x * dv.x - du.y * dv.y);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            used[prow] = 1;
            used[m + pcol] = 1;
            const double nw = usq * vsq;
            double cr = 0.0;
            for (int j = 0; j < rank - 1; ++j) cr += cross[j];
            fro += nw + cr;
            s_stop = (fro > 0.0 && sqrt(nw) < htol * sqrt(fabs(fro))) ? 1 : 0;
        }
        __syncthreads();
        if (s_stop) break;
        prow = nextr.i;
    }
    if (threadIdx.x == 0) rank_out[blockIdx.x] = rank;
}

// Dense blocks: out[offD[b] + i + j*m] = A(c2p[r0+i], c2p[c0+j]) as complex64.
__global__ void gather_dense_kernel(const cd *__restrict__ A, int64_t lda,
                                    const int *__restrict__ c2p, const int4 *__restrict__ blk,
                                    const int64_t *__restrict__ offD, float2 *__restrict__ out) {
    const int4 bk = blk[blockIdx.x];
    float2 *o = out + offD[blockIdx.x];
    const int64_t tot = (int64_t)bk.y * bk.w;
    for (int64_t e = threadIdx.x; e < tot; e += blockDim.x) {
        const int i = (int)(e % bk.y), j = (int)(e / bk.y);
        const cd v = A[c2p[bk.x + i] + (int64_t)c2p[bk.z + j] * lda];
        o[e] = make_float2((float)v.x, (float)v.y);
    }
}

// ACA factors (FP64 scratch, capacity columns) -> complex64 at their final
// offsets, rank columns each.
__global__ void compact_kernel(const int4 *__restrict__ blk, const int *__restrict__ rank,
                               const int64_t *__restrict__ offU, const int64_t *__restrict__ offV,
                               const cd *__restrict__ UV, const int64_t *__restrict__ outU,
                               const int64_t *__restrict__ outV, float2 *__restrict__ fU,
                               float2 *__restrict__ fV) {
    const int b = blockIdx.x;
    const int4 bk = blk[b];
    const int r = rank[b];
    const int64_t nu = (int64_t)bk.y * r, nv = (int64_t)bk.w * r;
    for (int64_t e = threadIdx.x; e < nu; e += blockDim.x) {
        const cd v = UV[offU[b] + e];
        fU[outU[b] + e] = make_float2((float)v.x, (float)v.y);
    }
    // V transposed: (j, q) -> q + j * r
    for (int64_t e = threadIdx.x; e < nv; e += blockDim.x) {
        const int64_t j = e % bk.w, q = e / bk.w;
        const cd v = UV[offV[b] + e];
        fV[outV[b] + q + j * r] = make_float2((float)v.x, (float)v.y);
    }
}

// ---------------------------------------------------------------------------
// H-matrix times vectors
// ---------------------------------------------------------------------------
// Work records, built on the host once the ranks are known (one array per
// matrix, since the low-rank offsets depend on the ranks):
//
// RowEnt, one per entry of a leaf's contribution list: the leaf's rows of a
// dense block (kind 0, columns = the block's columns, x = X in cluster order
// from column xo) or of a low-rank factor U (kind 1, columns = rank, x = the
// block's t = V^T x at T + xo * NC).  a: float2 offset, in D or U, of the
// entry (first row of the leaf, column 0); column stride lda.
struct RowEnt {
    long long a, xo;
    int lda, cnt, kind, pad;
};
// VtxEnt, one per V^T x work item (a segment of <= 64 columns of one
// low-rank block): V(j, q) of the segment at V + v + (j - j0) * r + q; its
// x columns start at xo (cluster order); the item's partial t goes to
// TP + out * 4 (r rows of 4 right-hand sides).
struct VtxEnt {
    long long v, out;
    int xo, cnt, r, pad;
};

// Per matrix (up to 4 in one launch, blockIdx.y):
struct HMat {
    const float2 *D;      // dense blocks, column-major
    const float2 *U, *V;  // low-rank factors (U column-major, V transposed)
    const int *rank;      // per low-rank block
    const int64_t *offT;  // t_b at T + offT[b] * nc
    const cd *X;          // n x nc input (face order), column stride n
    cd *Y;                // n x nc output (face order)
    cd *T;                // scratch V^T x
    cd *Xc;               // scratch: X in cluster order (n x nc)
    const int64_t *offTP; // per low-rank block: start of its segment partials (entries / 4)
    cd *TP;               // scratch: segment partials of V^T x
    const RowEnt *rent;   // row-sum records (one per contribution-list entry)
    const VtxEnt *vent;   // V^T x records (one per item)
};
struct HMats {
    HMat h[4];
};

// Warps per block of the product kernels (one work item per warp) and the
// launch-bound block count per SM.  Measured on the four matrices of the
// 25,152-face rod (4 right-hand sides): 4 warps x >= 6 blocks 0.971 ms per
// product, 4 x 4 1.05 ms, 8 x 3 1.06 ms, 8 x 4 (64 registers, spills)
// 1.24 ms, 4 x 6 with 2 columns in flight 1.18 ms.
#ifndef HM_WPB
#define HM_WPB 4
#endif
#ifndef HM_MINB
#define HM_MINB 6
#endif
// Matrix columns in flight per lane in the row sums (software pipeline depth).
#ifndef HM_RUN
#define HM_RUN 4
#endif
constexpr int HM_VSEG = 64;      // columns per V^T x item (the host cuts segments this long)
constexpr int HM_XS = 32;        // x columns per shared-memory stage of the row sums

// 16-byte asynchronous copies global -> shared (completion per thread via
// commit / wait groups; a __syncwarp after the wait publishes the warp's copies)
__device__ __forceinline__ void cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ float2 ld_stream(const float2 *p) { return __ldcs(p); }

// t_b = V_b^T x in two steps.  One warp per VtxEnt item: the item's x
// columns (<= 64, all right-hand sides) are staged in shared memory with
// asynchronous copies while the first factor loads are in flight; lane =
// factor column q (V is stored transposed, so the lanes of one j read
// consecutive words) and the x values are shared-memory broadcasts.  Blocks
// of rank <= 16 put 2 or 4 columns in flight per warp (groups of 16 or 8
// lanes, summed in a fixed order at the end).  hm_vtx_reduce_kernel adds a
// block's segments in order (deterministic).
template <int NC>
__global__ void __launch_bounds__(32 * HM_WPB, HM_MINB) hm_vtx_kernel(HMats P, int n, int nc,
                                                                       int nvitem) {
    __shared__ __align__(16) cd xsm[HM_WPB][HM_VSEG * NC];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int it = blockIdx.x * HM_WPB + w;
    if (it >= nvitem) return;
    const HMat &H = P.h[blockIdx.y];
    const VtxEnt ve = H.vent[it];
    const int r = ve.r, cnt = ve.cnt;
    if (r == 0 || cnt == 0) return;
    cd *xb = xsm[w];
    for (int j = l; j < cnt; j += 32)
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if (c < nc) cp16(xb + j * NC + c, H.Xc + ve.xo + j + (int64_t)c * n);
    cp_commit();
    const float2 *V = H.V + ve.v;
    cd *out = H.TP + ve.out * 4;
    if (r <= 16) {
        const int Pl = r <= 8 ? 8 : 16, G = 32 / Pl;
        const int g = l / Pl, q = l - g * Pl;
        const bool live = q < r;
        constexpr int U4 = 4;
        cd acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = cmk(0, 0);
        float2 v[U4];
#pragma unroll
        for (int u = 0; u < U4; ++u) {
            const int j = g + u * G;
            v[u] = (live && j < cnt) ? ld_stream(V + (int64_t)j * r + q) : make_float2(0.f, 0.f);
        }
        cp_wait<0>();
        __syncwarp();
        for (int j = g; j < cnt; j += U4 * G) {
            float2 nx[U4];
#pragma unroll
            for (int u = 0; u < U4; ++u) {
                const int jj = j + (U4 + u) * G;
                nx[u] = (live && jj < cnt) ? ld_stream(V + (int64_t)jj * r + q)
                                           : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < U4; ++u) {
                const int jj = j + u * G;
                if (jj < cnt) {
                    const cd vv = cmk(v[u].x, v[u].y);
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        if (c < nc) acc[c] = cfma(vv, xb[jj * NC + c], acc[c]);
                }
            }
#pragma unroll
            for (int u = 0; u < U4; ++u) v[u] = nx[u];
        }
        for (int o = Pl; o < 32; o <<= 1)
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
                acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
            }
        if (g == 0 && live)
#pragma unroll
            for (int c = 0; c < NC; ++c) out[(int64_t)q * 4 + c] = acc[c];
        return;
    }
    cp_wait<0>();
    __syncwarp();
    constexpr int UN = 8;
    for (int q0 = 0; q0 < r; q0 += 32) {
        const int q = q0 + l;
        const bool live = q < r;
        cd acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = cmk(0, 0);
        float2 v[UN];
#pragma unroll
        for (int u = 0; u < UN; ++u)
            v[u] = (live && u < cnt) ? ld_stream(V + (int64_t)u * r + q) : make_float2(0.f, 0.f);
        for (int j = 0; j < cnt; j += UN) {
            float2 nx[UN];
#pragma unroll
            for (int u = 0; u < UN; ++u) {
                const int jj = j + UN + u;
                nx[u] = (live && jj < cnt) ? ld_stream(V + (int64_t)jj * r + q)
                                           : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < UN; ++u)
                if (j + u < cnt) {
                    const cd vv = cmk(v[u].x, v[u].y);
#pragma unroll
                    for (int c = 0; c < NC; ++c)
                        if (c < nc) acc[c] = cfma(vv, xb[(j + u) * NC + c], acc[c]);
                }
#pragma unroll
            for (int u = 0; u < UN; ++u) v[u] = nx[u];
        }
        if (live)
#pragma unroll
            for (int c = 0; c < NC; ++c) out[(int64_t)q * 4 + c] = acc[c];
    }
}

// T[offT[b] * nc + q * nc + c] = sum over the block's segments (in order);
// one warp per low-rank block, lane = q; vptr: items of block b are
// vptr[b] .. vptr[b+1]-1 (segments 0, 1, ...).
template <int NC>
__global__ void __launch_bounds__(256) hm_vtx_reduce_kernel(HMats P, int nc, int nblk,
                                                            const int *__restrict__ vptr) {
    const int b = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (b >= nblk) return;
    const HMat &H = P.h[blockIdx.y];
    const int l = threadIdx.x & 31;
    const int r = H.rank[b];
    const int nseg = vptr[b + 1] - vptr[b];
    const cd *in = H.TP + H.offTP[b] * NC;
    cd *T = H.T + H.offT[b] * nc;
    for (int q = l; q < r; q += 32) {
        cd acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = cmk(0, 0);
        for (int sg = 0; sg < nseg; ++sg)
#pragma unroll
            for (int c = 0; c < NC; ++c) acc[c] = cadd(acc[c], in[((int64_t)sg * r + q) * NC + c]);
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if (c < nc) T[(int64_t)q * nc + c] = acc[c];
    }
}

// Row sums in two steps.  Work items (shared by the matrices): (chunk,
// first entry, end entry, first row within the leaf << 6 | live rows) -- a
// 32-row piece of a leaf and a segment of at most a few entries of the
// leaf's contribution list.  One warp per item, lane = row.  The entries'
// columns are walked in stages of HM_XS: the x values of the next stage
// (X in cluster order for a dense block, t for a low-rank one) are copied
// to shared memory asynchronously while the current stage is multiplied, so
// the only long-latency loads in the inner loop are the streamed matrix
// columns (prefetched UN at a time).  The warp writes a 32 x NC partial;
// hm_reduce_kernel adds the partials of each chunk in item order (so the
// result is deterministic) and scatters the rows to face order.
template <int NC>
__global__ void __launch_bounds__(32 * HM_WPB, HM_MINB) hm_rows_kernel(
    HMats P, int n, int nitem, const int4 *__restrict__ items, cd *__restrict__ partial) {
    __shared__ __align__(16) cd xsm[HM_WPB][2][HM_XS * NC];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int it = blockIdx.x * HM_WPB + w;
    if (it >= nitem) return;
    const HMat &H = P.h[blockIdx.y];
    const int4 item = items[it];
    const int ne = item.z - item.y;           // <= 32 (host cuts the lists)
    const int r0 = item.w >> 6;
    const bool live = l < (item.w & 63);
    // lane q holds the record of entry item.y + q
    RowEnt mine;
    mine.a = 0; mine.xo = 0; mine.lda = 0; mine.cnt = 0; mine.kind = 0; mine.pad = 0;
    if (l < ne) mine = H.rent[item.y + l];
    const unsigned FULL = 0xffffffffu;
    // (e, j0): current stage = columns j0 .. j0 + HM_XS of entry e
    auto advance = [&](int &e, int &j0, int &cnt) -> bool {
        j0 += HM_XS;
        if (j0 < cnt) return true;
        j0 = 0;
        do {
            if (++e >= ne) return false;
            cnt = __shfl_sync(FULL, mine.cnt, e);
        } while (cnt == 0);
        return true;
    };
    auto stage_x = [&](int e, int j0, int cnt, cd *buf) {
        const long long xo = __shfl_sync(FULL, mine.xo, e);
        const int kind = __shfl_sync(FULL, mine.kind, e);
        const int ncol = min(HM_XS, cnt - j0);
        if (l < ncol) {
            if (kind == 0) {
                const cd *src = H.Xc + xo + j0 + l;
#pragma unroll
                for (int c = 0; c < NC; ++c) cp16(buf + l * NC + c, src + (int64_t)c * n);
            } else {
                const cd *src = H.T + (xo + j0 + l) * NC;
#pragma unroll
                for (int c = 0; c < NC; ++c) cp16(buf + l * NC + c, src + c);
            }
        }
        cp_commit();
    };
    cd acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = cmk(0, 0);
    int e = -1, j0 = 0, cnt = 0, buf = 0;
    bool have = advance(e, j0, cnt);
    if (have) stage_x(e, j0, cnt, xsm[w][0]);
    constexpr int UN = HM_RUN;
    while (have) {
        int en = e, jn = j0, cn = cnt;
        const bool more = advance(en, jn, cn);
        if (more) stage_x(en, jn, cn, xsm[w][buf ^ 1]);
        else cp_commit();                       // an empty group keeps the count uniform
        const long long ao = __shfl_sync(FULL, mine.a, e);
        const int lda = __shfl_sync(FULL, mine.lda, e);
        const int kind = __shfl_sync(FULL, mine.kind, e);
        const int ncol = min(HM_XS, cnt - j0);
        const float2 *A = (kind == 0 ? H.D : H.U) + ao + r0 + l + (int64_t)j0 * lda;
        float2 a[UN];
#pragma unroll
        for (int u = 0; u < UN; ++u)
            a[u] = (live && u < ncol) ? ld_stream(A + (int64_t)u * lda) : make_float2(0.f, 0.f);
        cp_wait<1>();
        __syncwarp();
        const cd *xb = xsm[w][buf];
        for (int j = 0; j < ncol; j += UN) {
            float2 nx[UN];
#pragma unroll
            for (int u = 0; u < UN; ++u) {
                const int jj = j + UN + u;
                nx[u] = (live && jj < ncol) ? ld_stream(A + (int64_t)jj * lda)
                                            : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < UN; ++u)
                if (j + u < ncol) {
                    const cd av = cmk(a[u].x, a[u].y);
#pragma unroll
                    for (int c = 0; c < NC; ++c) acc[c] = cfma(av, xb[(j + u) * NC + c], acc[c]);
                }
#pragma unroll
            for (int u = 0; u < UN; ++u) a[u] = nx[u];
        }
        __syncwarp();                           // stage buffer free for the copy after next
        buf ^= 1;
        e = en;
        j0 = jn;
        cnt = cn;
        have = more;
    }
    cd *out = partial + ((int64_t)blockIdx.y * nitem + it) * 32 * 4;
#pragma unroll
    for (int c = 0; c < NC; ++c) out[c * 32 + l] = acc[c];
}

// y rows of chunk k = sum of the partials of items cptr[k] .. cptr[k+1]-1
template <int NC>
__global__ void __launch_bounds__(256) hm_reduce_kernel(HMats P, int n, int nc, int nchunk,
                                                        int nitem, const int *__restrict__ cptr,
                                                        const int2 *__restrict__ chunks,
                                                        const int2 *__restrict__ leaf_rows,
                                                        const int *__restrict__ c2p,
                                                        const cd *__restrict__ partial) {
    const int k = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (k >= nchunk) return;
    const HMat &H = P.h[blockIdx.y];
    const int l = threadIdx.x & 31;
    const int2 ch = chunks[k];
    const int2 lf = leaf_rows[ch.x];
    if (ch.y + l >= lf.y) return;
    cd acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = cmk(0, 0);
    const cd *base = partial + (int64_t)blockIdx.y * nitem * 32 * 4;
    for (int i = cptr[k]; i < cptr[k + 1]; ++i)
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = cadd(acc[c], base[((int64_t)i * 4 + c) * 32 + l]);
    const int64_t yr = c2p[lf.x + ch.y + l];
#pragma unroll
    for (int c = 0; c < NC; ++c)
        if (c < nc) H.Y[yr + (int64_t)c * n] = acc[c];
}

// Xc[c + col*n] = X[c2p[c] + col*n] for every matrix of the launch (blockIdx.y)
__global__ void permute_kernel(HMats P, int n, int nc, const int *__restrict__ c2p) {
    const HMat &H = P.h[blockIdx.y];
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * nc) return;
    const int c = (int)(e % n), col = (int)(e / n);
    H.Xc[e] = H.X[c2p[c] + (int64_t)col * n];
}

// y = A x for the packed operator.  P1 = G1 [sig1|h1], P2 = G2 [sig2|h2],
// Q1 = H1 [sig1|h1], Q2 = H2 [sig2|h2], each n x 4K (columns sig then h x,y,z,
// K each); y uses the excitation layout [phi | a (3) | De | alpha (3)].
__global__ void afun_kernel(int n, int K, const cd *P1, const cd *P2, const cd *Q1,
                            const cd *Q2, cd *y, cd e1, cd e2, double k,
                            const double *__restrict__ nvec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cd ik = cmk(0.0, k);
    const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
    auto at = [&](const cd *p, int col) { return p[(int64_t)col * n + i]; };
    for (int q = 0; q < K; ++q) {
        const cd gs1 = at(P1, q), gs2 = at(P2, q), hs1 = at(Q1, q), hs2 = at(Q2, q);
        const cd egs = csub(cmul(e1, gs1), cmul(e2, gs2));
        cd negh = cmk(0, 0);
        y[(int64_t)q * n + i] = csub(gs1, gs2);
        for (int c = 0; c < 3; ++c) {
            const int col = K + c * K + q;
            const cd gh1 = at(P1, col), gh2 = at(P2, col), hh1 = at(Q1, col), hh2 = at(Q2, col);
            y[(int64_t)(K + c * K + q) * n + i] = csub(gh1, gh2);
            y[(int64_t)(5 * K + c * K + q) * n + i] =
                csub(csub(hh1, hh2), cmul(ik, cscale(egs, nv[c])));
            negh = cadd(negh, cscale(csub(cmul(e1, gh1), cmul(e2, gh2)), nv[c]));
        }
        y[(int64_t)(4 * K + q) * n + i] =
            csub(csub(cmul(e1, hs1), cmul(e2, hs2)), cmul(ik, negh));
    }
}

}  // namespace hm
}  // namespace mnpb

using namespace mnpb;

extern "C" int mnpb_hmat_aca(void *stream, int64_t n, const double *A, int64_t lda,
                             const int32_t *c2p, int64_t nblk, const int32_t *blocks,
                             const int64_t *offU, const int64_t *offV, int64_t max_mn,
                             int64_t kmax, double htol, double *UV, int32_t *rank) {
    clear_error();
    MNPB_REQUIRE(n > 0 && lda >= n && nblk >= 0 && kmax > 0 && kmax <= hm::ACA_MAXK && htol > 0,
                 "hmat_aca: bad sizes (kmax <= %d)", hm::ACA_MAXK);
    if (nblk == 0) return MNPB_OK;
    MNPB_REQUIRE(A && c2p && blocks && offU && offV && UV && rank, "hmat_aca: null pointer");
    MNPB_REQUIRE(max_mn > 0 && max_mn <= 200 * 1024, "hmat_aca: block too large (m + n = %lld)",
                 (long long)max_mn);
    cudaStream_t s = as_stream(stream);
    const int smem = (int)max_mn;
    if (smem > 48 * 1024) MNPB_TRY(smem_opt_in(hm::aca_kernel, smem, "hmat_aca"));
    ProfScope ps(s, PC_ACA, 0.0);
    hm::aca_kernel<<<(unsigned)nblk, hm::ACA_T, smem, s>>>(
        (const cd *)A, lda, c2p, (const int4 *)blocks, offU, offV, (int)kmax, htol, (cd *)UV, rank);
    MNPB_LAUNCH_CHECK("aca_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_hmat_gather_dense(void *stream, const double *A, int64_t lda,
                                      const int32_t *c2p, int64_t nblk, const int32_t *blocks,
                                      const int64_t *offD, float *out) {
    clear_error();
    if (nblk == 0) return MNPB_OK;
    MNPB_REQUIRE(A && c2p && blocks && offD && out && lda > 0, "hmat_gather_dense: bad arguments");
    cudaStream_t s = as_stream(stream);
    ProfScope ps(s, PC_ACA, 0.0);
    hm::gather_dense_kernel<<<(unsigned)nblk, 256, 0, s>>>((const cd *)A, lda, c2p,
                                                          (const int4 *)blocks, offD, (float2 *)out);
    MNPB_LAUNCH_CHECK("gather_dense_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_hmat_compact(void *stream, int64_t nblk, const int32_t *blocks,
                                 const int32_t *rank, const int64_t *offU, const int64_t *offV,
                                 const double *UV, const int64_t *outU, const int64_t *outV,
                                 float *U, float *V) {
    clear_error();
    if (nblk == 0) return MNPB_OK;
    MNPB_REQUIRE(blocks && rank && offU && offV && UV && outU && outV && U && V,
                 "hmat_compact: null pointer");
    cudaStream_t s = as_stream(stream);
    hm::compact_kernel<<<(unsigned)nblk, 256, 0, s>>>((const int4 *)blocks, rank, offU, offV,
                                                     (const cd *)UV, outU, outV, (float2 *)U,
                                                     (float2 *)V);
    MNPB_LAUNCH_CHECK("compact_kernel");
    return MNPB_OK;
}

// One matrix of an H-matrix product, as passed through the C ABI.
struct mnpb_hmat_desc {
    const float *D, *U, *V;
    const int32_t *rank;
    const int64_t *offT;
    const double *X;
    double *Y, *T, *Xc;
    const int64_t *offTP;
    double *TP;
    const void *rent, *vent;
};

extern "C" int mnpb_hmat_matvec(void *stream, int64_t n, int64_t nc, int64_t nmat,
                                const void *descs, const int32_t *c2p, int64_t nlr,
                                int64_t nchunk, const int32_t *chunks, const int32_t *leaf_rows,
                                int64_t nitem, const int32_t *items, const int32_t *cptr,
                                double *partial, int64_t nvitem, const int32_t *vptr) {
    clear_error();
    MNPB_REQUIRE(n > 0 && nc > 0 && nc <= 64 && nmat >= 1 && nmat <= 4 && nchunk > 0 &&
                     nitem > 0,
                 "hmat_matvec: bad sizes (nc <= 64, nmat <= 4)");
    MNPB_REQUIRE(descs && c2p && leaf_rows && chunks && items && cptr && partial &&
                     (nlr == 0 || (vptr && nvitem > 0)),
                 "hmat_matvec: null pointer");
    cudaStream_t s = as_stream(stream);
    const mnpb_hmat_desc *d = (const mnpb_hmat_desc *)descs;
    hm::HMats P;
    for (int q = 0; q < 4; ++q) {
        const mnpb_hmat_desc &e = d[q < nmat ? q : 0];
        MNPB_REQUIRE(e.rent && (nlr == 0 || e.vent), "hmat_matvec: missing work records");
        P.h[q] = hm::HMat{(const float2 *)e.D, (const float2 *)e.U, (const float2 *)e.V, e.rank,
                          e.offT, (const cd *)e.X, (cd *)e.Y, (cd *)e.T, (cd *)e.Xc, e.offTP,
                          (cd *)e.TP, (const hm::RowEnt *)e.rent, (const hm::VtxEnt *)e.vent};
    }
    ProfScope ps(s, PC_HMATVEC, 0.0);
    // columns in chunks of at most 4 (register bound of the kernels); T
    // holds sum(rank) x 4 entries and is reused by every chunk
    for (int64_t c0 = 0; c0 < nc; c0 += 4) {
        const int ncc = (int)(nc - c0 < 4 ? nc - c0 : 4);
        hm::HMats Q = P;
        for (int q = 0; q < 4; ++q) {
            Q.h[q].X = P.h[q].X + c0 * n;
            Q.h[q].Y = P.h[q].Y + c0 * n;
        }
        hm::permute_kernel<<<dim3((unsigned)ceil_div(n * ncc, 256), (unsigned)nmat), 256, 0, s>>>(
            Q, (int)n, ncc, c2p);
        MNPB_LAUNCH_CHECK("hm permute_kernel");
        if (nlr > 0) {
            dim3 g((unsigned)ceil_div(nvitem, HM_WPB), (unsigned)nmat);
            hm::hm_vtx_kernel<4><<<g, 32 * HM_WPB, 0, s>>>(Q, (int)n, ncc, (int)nvitem);
            MNPB_LAUNCH_CHECK("hm_vtx_kernel");
            dim3 gr((unsigned)ceil_div(nlr, 8), (unsigned)nmat);
            hm::hm_vtx_reduce_kernel<4><<<gr, 256, 0, s>>>(Q, ncc, (int)nlr, vptr);
            MNPB_LAUNCH_CHECK("hm_vtx_reduce_kernel");
        }
        dim3 g((unsigned)ceil_div(nitem, HM_WPB), (unsigned)nmat);
        dim3 gr((unsigned)ceil_div(nchunk, 8), (unsigned)nmat);
#define MNPB_HM_ROWS(NCV)                                                                       \
    hm::hm_rows_kernel<NCV><<<g, 32 * HM_WPB, 0, s>>>(Q, (int)n, (int)nitem,                     \
                                                     (const int4 *)items, (cd *)partial);        \
    hm::hm_reduce_kernel<NCV><<<gr, 256, 0, s>>>(Q, (int)n, NCV, (int)nchunk, (int)nitem, cptr,  \
                                                 (const int2 *)chunks, (const int2 *)leaf_rows,  \
                                                 c2p, (const cd *)partial)
        switch (ncc) {
        case 1: MNPB_HM_ROWS(1); break;
        case 2: MNPB_HM_ROWS(2); break;
        case 3: MNPB_HM_ROWS(3); break;
        default: MNPB_HM_ROWS(4); break;
        }
#undef MNPB_HM_ROWS
        MNPB_LAUNCH_CHECK("hm_rows_kernel");
    }
    return MNPB_OK;
}

extern "C" int mnpb_bem_afun(void *stream, int64_t n, int64_t nrhs, const double *P1,
                             const double *P2, const double *Q1, const double *Q2, double *y,
                             double e1_re, double e1_im, double e2_re, double e2_im, double k,
                             const double *nvec) {
    clear_error();
    MNPB_REQUIRE(n > 0 && nrhs > 0, "bem_afun: bad sizes");
    MNPB_REQUIRE(P1 && P2 && Q1 && Q2 && y && nvec, "bem_afun: null pointer");
    cudaStream_t s = as_stream(stream);
    hm::afun_kernel<<<ceil_div(n, 128), 128, 0, s>>>((int)n, (int)nrhs, (const cd *)P1,
                                                     (const cd *)P2, (const cd *)Q1, (const cd *)Q2,
                                                     (cd *)y, cmk(e1_re, e1_im), cmk(e2_re, e2_im),
                                                     k, nvec);
    MNPB_LAUNCH_CHECK("afun_kernel");
    return MNPB_OK;
}
