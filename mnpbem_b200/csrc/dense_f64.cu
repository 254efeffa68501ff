// Batched dense complex linear algebra in FP64 (interleaved complex128,
// column-major): GEMM, LU with partial pivoting, triangular solves.
//
// Every routine works on `batch` independent matrices `stride` elements
// apart, so a whole spectrum of wavelengths goes through each launch
// together: per-matrix latency (the column-by-column panel) is hidden by the
// other matrices in the batch.
#include "common.cuh"
#include "dense_f64.cuh"

namespace mnpb {

// ---------------------------------------------------------------------------
// GEMM: C = alpha A B + beta C, all no-transpose.  64x64 tile per CTA,
// 128 threads, each thread 8 rows x 4 columns (columns interleaved by 16 so
// that the shared-memory reads of B are conflict free).
// ---------------------------------------------------------------------------
namespace {
constexpr int GBM = 64, GBN = 64, GBK = 8;

__global__ void __launch_bounds__(128, 2) zgemm_kernel(int m, int n, int k, cd alpha,
                                                       const cd *__restrict__ A, int64_t lda,
                                                       int64_t sA, const cd *__restrict__ B,
                                                       int64_t ldb, int64_t sB, cd beta,
                                                       cd *__restrict__ C, int64_t ldc,
                                                       int64_t sC) {
    // B rows padded by one element: the loader's 8 consecutive threads store
    // 8 different rows, which must not share shared-memory banks
    __shared__ cd As[GBK][GBM];
    __shared__ cd Bs[GBK][GBN + 1];
    const int tid = threadIdx.x;
    const int tn = tid & 15, tm = tid >> 4;
    const int m0 = blockIdx.x * GBM, n0 = blockIdx.y * GBN;
    const int64_t b = blockIdx.z;
    A += b * sA;
    B += b * sB;
    C += b * sC;
    cd acc[8][4];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = cmk(0.0, 0.0);

    const int ar = tid & 63, ak = tid >> 6;   // A loader: row, first k
    const int bk = tid & 7, bc = tid >> 3;    // B loader: k, first column
    cd pa[4], pb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int gr = m0 + ar, gk = k0 + ak + 2 * q;
            pa[q] = (gr < m && gk < k) ? A[(int64_t)gk * lda + gr] : cmk(0.0, 0.0);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int gc = n0 + bc + 16 * q, gk = k0 + bk;
            pb[q] = (gc < n && gk < k) ? B[(int64_t)gc * ldb + gk] : cmk(0.0, 0.0);
        }
    };
    if (k > 0) load(0);
    for (int k0 = 0; k0 < k; k0 += GBK) {
#pragma unroll
        for (int q = 0; q < 4; ++q) As[ak + 2 * q][ar] = pa[q];
#pragma unroll
        for (int q = 0; q < 4; ++q) Bs[bk][bc + 16 * q] = pb[q];
        __syncthreads();
        if (k0 + GBK < k) load(k0 + GBK);   // next tile in flight during the math
#pragma unroll
        for (int kk = 0; kk < GBK; ++kk) {
            cd bv[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) bv[c] = Bs[kk][tn + 16 * c];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const cd a = As[kk][tm * 8 + r];
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = cfma(a, bv[c], acc[r][c]);
            }
        }
        __syncthreads();
    }
    const bool beta0 = (beta.x == 0.0 && beta.y == 0.0);
    // two halves of the C fragment: all loads of a half in flight, then stores
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        cd cv[8][2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int gc = n0 + tn + 16 * (2 * h + c);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int gr = m0 + tm * 8 + r;
                cv[r][c] = (!beta0 && gc < n && gr < m) ? __ldg(C + (int64_t)gc * ldc + gr)
                                                        : cmk(0.0, 0.0);
            }
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int gc = n0 + tn + 16 * (2 * h + c);
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int gr = m0 + tm * 8 + r;
                if (gc < n && gr < m)
                    C[(int64_t)gc * ldc + gr] = cfma(beta, cv[r][c], cmul(alpha, acc[r][2 * h + c]));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// LU panel: columns [k0, k0+kb) over rows [k0, n), one CTA per matrix.
// Pivot = first row of maximal |re|+|im| (LAPACK izamax rule).
// ---------------------------------------------------------------------------
constexpr int PANEL_THREADS = 512;

__global__ void __launch_bounds__(PANEL_THREADS) panel_kernel(int n, int k0, int kb, cd *A,
                                                              int64_t lda, int64_t sA,
                                                              int32_t *ipiv, int64_t sP,
                                                              int32_t *info) {
    __shared__ double red_v[PANEL_THREADS / 32];
    __shared__ int red_i[PANEL_THREADS / 32];
    __shared__ cd prow[64];
    __shared__ int s_piv;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int64_t b = blockIdx.x;
    A += b * sA;
    ipiv += b * sP;
    for (int jj = 0; jj < kb; ++jj) {
        const int c = k0 + jj;
        cd *col = A + (int64_t)c * lda;
        double best = -1.0;
        int bi = n;
        for (int r = c + tid; r < n; r += PANEL_THREADS) {
            double v = cabs1(col[r]);
            if (v > best) { best = v; bi = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { red_v[wid] = best; red_i[wid] = bi; }
        __syncthreads();
        if (wid == 0) {
            best = (lane < PANEL_THREADS / 32) ? red_v[lane] : -1.0;
            bi = (lane < PANEL_THREADS / 32) ? red_i[lane] : n;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) {
                int p = bi;
                if (!(best > 0.0)) {       // zero column: no interchange, record singularity
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
                cd *cp = A + (int64_t)(k0 + cc) * lda;
                cd t = cp[c];
                cp[c] = cp[p];
                cp[p] = t;
            }
        }
        __syncthreads();
        const int rest = kb - jj;
        for (int cc = tid; cc < rest; cc += PANEL_THREADS) prow[cc] = A[(int64_t)(c + cc) * lda + c];
        __syncthreads();
        const cd piv = prow[0];
        const bool nz = (piv.x != 0.0 || piv.y != 0.0);
        const cd inv = nz ? crcp(piv) : cmk(0.0, 0.0);
        for (int r = c + 1 + tid; r < n; r += PANEL_THREADS) {
            cd l = col[r];
            if (nz) l = cmul(l, inv);
            col[r] = l;
            for (int cc = 1; cc < rest; ++cc) {
                cd *q = A + (int64_t)(c + cc) * lda + r;
                *q = cfms(l, prow[cc], *q);
            }
        }
        __syncthreads();
    }
}

// Row interchanges piv[c0..c1) applied to columns [j0, j1) (forward or
// backward order), one thread per column.
__global__ void laswp_kernel(cd *A, int64_t lda, int64_t sA, int j0, int j1, int jskip0,
                             int jskip1, const int32_t *ipiv, int64_t sP, int c0, int c1,
                             int forward) {
    const int64_t b = blockIdx.y;
    int j = j0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= j1) return;
    if (j >= jskip0 && j < jskip1) return;
    cd *col = A + b * sA + (int64_t)j * lda;
    const int32_t *pv = ipiv + b * sP;
    if (forward) {
        for (int c = c0; c < c1; ++c) {
            int p = pv[c];
            if (p != c) { cd t = col[c]; col[c] = col[p]; col[p] = t; }
        }
    } else {
        for (int c = c1 - 1; c >= c0; --c) {
            int p = pv[c];
            if (p != c) { cd t = col[c]; col[c] = col[p]; col[p] = t; }
        }
    }
}

// Column interchanges of X (rows [0, m)), c from n-1 down to 0: X <- X P.
__global__ void colswp_kernel(cd *X, int64_t ldx, int64_t sX, int m, const int32_t *ipiv,
                              int64_t sP, int n) {
    const int64_t b = blockIdx.y;
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    cd *x = X + b * sX + r;
    const int32_t *pv = ipiv + b * sP;
    for (int c = n - 1; c >= 0; --c) {
        int p = pv[c];
        if (p != c) {
            cd t = x[(int64_t)c * ldx];
            x[(int64_t)c * ldx] = x[(int64_t)p * ldx];
            x[(int64_t)p * ldx] = t;
        }
    }
}

// Small triangular solves on a kb x kb diagonal block (kb <= 32).
// mode 0: left lower unit     L x = b   (one thread per column of B)
// mode 1: left upper non-unit U x = b   (one thread per column of B)
// mode 2: right upper non-unit x U = b  (one thread per row of B)
// mode 3: right lower unit     x L = b  (one thread per row of B)
constexpr int TS = 32;

__global__ void __launch_bounds__(128) trsm_small_kernel(int mode, int kb, const cd *T,
                                                         int64_t ldt, int64_t sT, cd *B,
                                                         int64_t ldb, int64_t sB, int nvec) {
    __shared__ cd Ts[TS][TS + 1];
    const int64_t b = blockIdx.y;
    T += b * sT;
    B += b * sB;
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
        int r = e % TS, c = e / TS;
        Ts[r][c] = (r < kb && c < kb) ? T[(int64_t)c * ldt + r] : cmk(r == c ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvec) return;
    cd x[TS];
    const bool left = (mode < 2);
    // element e of the vector: left -> B(e, v); right -> B(v, e)
#pragma unroll
    for (int e = 0; e < TS; ++e)
        x[e] = (e < kb) ? (left ? B[(int64_t)v * ldb + e] : B[(int64_t)e * ldb + v]) : cmk(0, 0);
    if (mode == 0) {
#pragma unroll
        for (int r = 1; r < TS; ++r)
#pragma unroll
            for (int c = 0; c < r; ++c) x[r] = cfms(Ts[r][c], x[c], x[r]);
    } else if (mode == 1) {
#pragma unroll
        for (int r = TS - 1; r >= 0; --r) {
#pragma unroll
            for (int c = r + 1; c < TS; ++c) x[r] = cfms(Ts[r][c], x[c], x[r]);
            x[r] = cdiv(x[r], Ts[r][r]);
        }
    } else if (mode == 2) {
#pragma unroll
        for (int c = 0; c < TS; ++c) {
#pragma unroll
            for (int r = 0; r < c; ++r) x[c] = cfms(x[r], Ts[r][c], x[c]);
            x[c] = cdiv(x[c], Ts[c][c]);
        }
    } else {
#pragma unroll
        for (int c = TS - 1; c >= 0; --c)
#pragma unroll
            for (int r = c + 1; r < TS; ++r) x[c] = cfms(x[r], Ts[r][c], x[c]);
    }
#pragma unroll
    for (int e = 0; e < TS; ++e)
        if (e < kb) {
            if (left) B[(int64_t)v * ldb + e] = x[e];
            else B[(int64_t)e * ldb + v] = x[e];
        }
}

__global__ void set_identity_kernel(cd *W, int64_t ldw, int64_t sW, int n) {
    const int64_t b = blockIdx.z;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= n) return;
    W[b * sW + (int64_t)j * ldw + i] = cmk(i == j ? 1.0 : 0.0, 0.0);
}

}  // namespace

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
int zgemm(cudaStream_t s, int m, int n, int k, int batch, cd alpha, const cd *A, int64_t lda,
          int64_t sA, const cd *B, int64_t ldb, int64_t sB, cd beta, cd *C, int64_t ldc,
          int64_t sC) {
    if (m <= 0 || n <= 0 || batch <= 0) return MNPB_OK;
    dim3 grid(ceil_div(m, GBM), ceil_div(n, GBN), batch);
    ProfScope ps(s, PC_ZGEMM, 8.0 * m * n * (double)(k > 0 ? k : 0) * batch);
    if (k <= 0) {
        // C = beta C
        zgemm_kernel<<<grid, 128, 0, s>>>(m, n, 0, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
    } else {
        zgemm_kernel<<<grid, 128, 0, s>>>(m, n, k, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
    }
    MNPB_LAUNCH_CHECK("zgemm_kernel");
    return MNPB_OK;
}

static int trsm_small(cudaStream_t s, int mode, int kb, const cd *T, int64_t ldt, int64_t sT,
                      cd *B, int64_t ldb, int64_t sB, int nvec, int batch) {
    if (nvec <= 0 || kb <= 0) return MNPB_OK;
    dim3 grid(ceil_div(nvec, 128), batch);
    ProfScope ps(s, PC_TRSM, 4.0 * kb * kb * (double)nvec * batch);
    trsm_small_kernel<<<grid, 128, 0, s>>>(mode, kb, T, ldt, sT, B, ldb, sB, nvec);
    MNPB_LAUNCH_CHECK("trsm_small_kernel");
    return MNPB_OK;
}

static int split_point(int n) {
    int h = n / 2;
    h = (h / TS) * TS;
    return h < TS ? TS : h;
}

// L X = B, L unit lower n x n; B n x m.
int trsm_llu(cudaStream_t s, int n, int m, int batch, const cd *L, int64_t ldl, int64_t sL,
             cd *B, int64_t ldb, int64_t sB) {
    if (n <= TS) return trsm_small(s, 0, n, L, ldl, sL, B, ldb, sB, m, batch);
    int n1 = split_point(n);
    MNPB_TRY(trsm_llu(s, n1, m, batch, L, ldl, sL, B, ldb, sB));
    MNPB_TRY(zgemm(s, n - n1, m, n1, batch, cmk(-1, 0), L + n1, ldl, sL, B, ldb, sB, cmk(1, 0),
                   B + n1, ldb, sB));
    return trsm_llu(s, n - n1, m, batch, L + n1 + (int64_t)n1 * ldl, ldl, sL, B + n1, ldb, sB);
}

// U X = B, U upper non-unit.
int trsm_lun(cudaStream_t s, int n, int m, int batch, const cd *U, int64_t ldu, int64_t sU,
             cd *B, int64_t ldb, int64_t sB) {
    if (n <= TS) return trsm_small(s, 1, n, U, ldu, sU, B, ldb, sB, m, batch);
    int n1 = split_point(n);
    MNPB_TRY(trsm_lun(s, n - n1, m, batch, U + n1 + (int64_t)n1 * ldu, ldu, sU, B + n1, ldb, sB));
    MNPB_TRY(zgemm(s, n1, m, n - n1, batch, cmk(-1, 0), U + (int64_t)n1 * ldu, ldu, sU, B + n1,
                   ldb, sB, cmk(1, 0), B, ldb, sB));
    return trsm_lun(s, n1, m, batch, U, ldu, sU, B, ldb, sB);
}

// X U = B, U upper non-unit n x n; X, B m x n.
int trsm_run(cudaStream_t s, int n, int m, int batch, const cd *U, int64_t ldu, int64_t sU,
             cd *B, int64_t ldb, int64_t sB) {
    if (n <= TS) return trsm_small(s, 2, n, U, ldu, sU, B, ldb, sB, m, batch);
    int n1 = split_point(n);
    MNPB_TRY(trsm_run(s, n1, m, batch, U, ldu, sU, B, ldb, sB));
    MNPB_TRY(zgemm(s, m, n - n1, n1, batch, cmk(-1, 0), B, ldb, sB, U + (int64_t)n1 * ldu, ldu,
                   sU, cmk(1, 0), B + (int64_t)n1 * ldb, ldb, sB));
    return trsm_run(s, n - n1, m, batch, U + n1 + (int64_t)n1 * ldu, ldu, sU,
                    B + (int64_t)n1 * ldb, ldb, sB);
}

// X L = B, L unit lower n x n; X, B m x n.
int trsm_rlu(cudaStream_t s, int n, int m, int batch, const cd *L, int64_t ldl, int64_t sL,
             cd *B, int64_t ldb, int64_t sB) {
    if (n <= TS) return trsm_small(s, 3, n, L, ldl, sL, B, ldb, sB, m, batch);
    int n1 = split_point(n);
    MNPB_TRY(trsm_rlu(s, n - n1, m, batch, L + n1 + (int64_t)n1 * ldl, ldl, sL,
                      B + (int64_t)n1 * ldb, ldb, sB));
    MNPB_TRY(zgemm(s, m, n1, n - n1, batch, cmk(-1, 0), B + (int64_t)n1 * ldb, ldb, sB, L + n1,
                   ldl, sL, cmk(1, 0), B, ldb, sB));
    return trsm_rlu(s, n1, m, batch, L, ldl, sL, B, ldb, sB);
}

int laswp(cudaStream_t s, cd *A, int64_t lda, int64_t sA, int ncols, int jskip0, int jskip1,
          const int32_t *ipiv, int64_t sP, int c0, int c1, bool forward, int batch) {
    if (ncols <= 0 || c1 <= c0) return MNPB_OK;
    dim3 grid(ceil_div(ncols, 128), batch);
    ProfScope ps(s, PC_SWAP, 0.0);
    laswp_kernel<<<grid, 128, 0, s>>>(A, lda, sA, 0, ncols, jskip0, jskip1, ipiv, sP, c0, c1,
                                      forward ? 1 : 0);
    MNPB_LAUNCH_CHECK("laswp_kernel");
    return MNPB_OK;
}

// Row interchanges piv[c0..c1) applied to the columns [j0, j1) only.
static int laswp_range(cudaStream_t s, cd *A, int64_t lda, int64_t sA, int j0, int j1,
                       const int32_t *ipiv, int64_t sP, int c0, int c1, int batch) {
    if (j1 <= j0 || c1 <= c0) return MNPB_OK;
    dim3 grid(ceil_div(j1 - j0, 128), batch);
    ProfScope ps(s, PC_SWAP, 0.0);
    laswp_kernel<<<grid, 128, 0, s>>>(A, lda, sA, j0, j1, 0, 0, ipiv, sP, c0, c1, 1);
    MNPB_LAUNCH_CHECK("laswp_kernel");
    return MNPB_OK;
}

// Recursive LU: factor columns [off, off+w) over rows [off, n); absolute pivots.
static int rgetrf(cudaStream_t s, int n, int off, int w, int batch, cd *A, int64_t lda,
                  int64_t sA, int32_t *ipiv, int64_t sP, int32_t *info) {
    if (w <= TS) {
        ProfScope ps(s, PC_PANEL, 8.0 * w * w * (double)(n - off) * batch / 2);
        panel_kernel<<<batch, PANEL_THREADS, 0, s>>>(n, off, w, A, lda, sA, ipiv, sP, info);
        MNPB_LAUNCH_CHECK("panel_kernel");
        return MNPB_OK;
    }
    const int w1 = split_point(w);
    MNPB_TRY(rgetrf(s, n, off, w1, batch, A, lda, sA, ipiv, sP, info));
    MNPB_TRY(laswp_range(s, A, lda, sA, off + w1, off + w, ipiv, sP, off, off + w1, batch));
    cd *A11 = A + off + (int64_t)off * lda;
    cd *A12 = A + off + (int64_t)(off + w1) * lda;
    MNPB_TRY(trsm_llu(s, w1, w - w1, batch, A11, lda, sA, A12, lda, sA));
    MNPB_TRY(zgemm(s, n - off - w1, w - w1, w1, batch, cmk(-1, 0), A11 + w1, lda, sA, A12, lda,
                   sA, cmk(1, 0), A12 + w1, lda, sA));
    MNPB_TRY(rgetrf(s, n, off + w1, w - w1, batch, A, lda, sA, ipiv, sP, info));
    return laswp_range(s, A, lda, sA, off, off + w1, ipiv, sP, off + w1, off + w, batch);
}

int getrf(cudaStream_t s, int n, int batch, cd *A, int64_t lda, int64_t sA, int32_t *ipiv,
          int64_t sP, int32_t *info) {
    return rgetrf(s, n, 0, n, batch, A, lda, sA, ipiv, sP, info);
}

int getrs(cudaStream_t s, int n, int nrhs, int batch, const cd *LU, int64_t lda, int64_t sA,
          const int32_t *ipiv, int64_t sP, cd *B, int64_t ldb, int64_t sB) {
    MNPB_TRY(laswp(s, B, ldb, sB, nrhs, 0, 0, ipiv, sP, 0, n, true, batch));
    MNPB_TRY(trsm_llu(s, n, nrhs, batch, LU, lda, sA, B, ldb, sB));
    return trsm_lun(s, n, nrhs, batch, LU, lda, sA, B, ldb, sB);
}

// X A = B in place on B (m x n), A = P^T L U from getrf.
int right_solve(cudaStream_t s, int n, int m, int batch, const cd *LU, int64_t lda, int64_t sA,
                const int32_t *ipiv, int64_t sP, cd *B, int64_t ldb, int64_t sB) {
    MNPB_TRY(trsm_run(s, n, m, batch, LU, lda, sA, B, ldb, sB));
    MNPB_TRY(trsm_rlu(s, n, m, batch, LU, lda, sA, B, ldb, sB));
    dim3 grid(ceil_div(m, 128), batch);
    ProfScope ps(s, PC_SWAP, 0.0);
    colswp_kernel<<<grid, 128, 0, s>>>(B, ldb, sB, m, ipiv, sP, n);
    MNPB_LAUNCH_CHECK("colswp_kernel");
    return MNPB_OK;
}

int set_identity(cudaStream_t s, int n, int batch, cd *W, int64_t ldw, int64_t sW) {
    dim3 grid(ceil_div(n, 128), n, batch);
    set_identity_kernel<<<grid, 128, 0, s>>>(W, ldw, sW, n);
    MNPB_LAUNCH_CHECK("set_identity_kernel");
    return MNPB_OK;
}

}  // namespace mnpb

using namespace mnpb;

extern "C" int mnpb_zgemm(void *stream, int64_t m, int64_t n, int64_t k, int64_t batch,
                          double alpha_re, double alpha_im, const double *A, int64_t lda,
                          int64_t sA, const double *B, int64_t ldb, int64_t sB, double beta_re,
                          double beta_im, double *C, int64_t ldc, int64_t sC) {
    clear_error();
    MNPB_REQUIRE(m >= 0 && n >= 0 && k >= 0 && batch >= 0 && batch < 65536,
                 "zgemm: bad sizes");
    MNPB_REQUIRE(C && (k == 0 || (A && B)), "zgemm: null pointer");
    return zgemm(as_stream(stream), (int)m, (int)n, (int)k, (int)batch, cmk(alpha_re, alpha_im),
                 (const cd *)A, lda, sA, (const cd *)B, ldb, sB, cmk(beta_re, beta_im), (cd *)C,
                 ldc, sC);
}

extern "C" int mnpb_getrf_f64(void *stream, int64_t n, int64_t batch, double *A, int64_t ld,
                              int64_t stride, int32_t *piv, int64_t pstride, int32_t *info) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && ld >= n && batch < 65536, "getrf: bad sizes");
    MNPB_REQUIRE(A && piv, "getrf: null pointer");
    return getrf(as_stream(stream), (int)n, (int)batch, (cd *)A, ld, stride, piv, pstride, info);
}

extern "C" int mnpb_getrs_f64(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                              const double *LU, int64_t ld, int64_t stride, const int32_t *piv,
                              int64_t pstride, double *B, int64_t ldb, int64_t bstride) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && nrhs > 0 && ld >= n && ldb >= n, "getrs: bad sizes");
    MNPB_REQUIRE(LU && piv && B, "getrs: null pointer");
    return getrs(as_stream(stream), (int)n, (int)nrhs, (int)batch, (const cd *)LU, ld, stride,
                 piv, pstride, (cd *)B, ldb, bstride);
}
