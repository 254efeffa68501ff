// FP64 GMRES building blocks (the Krylov solver of the iterative retarded
// solver; the reference calls scipy.sparse.linalg.gmres with restart =
// min(n, maxit), mnpbem/bem/bem_iter.py:79-89).
//
//  * mnpb_gmres_arnoldi: one Arnoldi step with classical Gram-Schmidt run
//    twice (CGS2, as stable as modified Gram-Schmidt, but each pass is two
//    bandwidth-bound launches instead of j dependent dot products):
//    h = V^H w, w -= V h (twice), h_{j+1} = |w|, v_{j+1} = w / h_{j+1}.
//  * mnpb_gmres_givens: applies the previous Givens rotations to Hessenberg
//    column j, forms rotation j, updates g and reports |g_{j+1}| (the
//    residual norm of the least-squares problem), on the device.
//  * mnpb_gmres_update: back substitution R y = g, then x += V y.
//
// Vectors are complex128 of length L; the basis V is column-major with
// column stride ldv; H is column-major (ldh >= m + 1).  All arithmetic FP64.
#include "common.cuh"

namespace mnpb {
namespace gm {

constexpr int CH = 2048;   // elements per partial-dot chunk

// partial[q * nch + c] = sum over chunk c of conj(V[:, q]) w
__global__ void dots_kernel(int64_t L, int nq, const cd *__restrict__ V, int64_t ldv,
                            const cd *__restrict__ w, cd *__restrict__ partial, int nch) {
    __shared__ cd sh[32];
    const int c = blockIdx.x, q = blockIdx.y;
    const int64_t e0 = (int64_t)c * CH, e1 = min(L, e0 + CH);
    const cd *v = V + (int64_t)q * ldv;
    cd a = cmk(0, 0);
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const cd x = v[e], y = w[e];
        a.x += x.x * y.x + x.y * y.y;
        a.y += x.x * y.y - x.y * y.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
        a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        cd t = cmk(0, 0);
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t = cadd(t, sh[k]);
        partial[(int64_t)q * nch + c] = t;
    }
}

// h[q] (+)= sum_c partial[q][c]  (fixed order: deterministic)
__global__ void reduce_dots_kernel(int nq, int nch, const cd *__restrict__ partial, cd *h,
                                   int accumulate) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    cd t = cmk(0, 0);
    for (int c = 0; c < nch; ++c) t = cadd(t, partial[(int64_t)q * nch + c]);
    h[q] = accumulate ? cadd(h[q], t) : t;
}

// w -= V[:, 0:nq] hq  (hq = the dots of this pass)
__global__ void project_kernel(int64_t L, int nq, const cd *__restrict__ V, int64_t ldv,
                               const cd *__restrict__ hq, cd *__restrict__ w) {
    extern __shared__ cd sh_h[];
    for (int q = threadIdx.x; q < nq; q += blockDim.x) sh_h[q] = hq[q];
    __syncthreads();
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L) return;
    cd acc = w[e];
    for (int q = 0; q < nq; ++q) acc = csub(acc, cmul(V[(int64_t)q * ldv + e], sh_h[q]));
    w[e] = acc;
}

// partial squared norms of w
__global__ void norm_kernel(int64_t L, const cd *__restrict__ w, double *__restrict__ partial) {
    __shared__ double sh[32];
    const int64_t e0 = (int64_t)blockIdx.x * CH, e1 = min(L, e0 + CH);
    double a = 0.0;
    for (int64_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) a += w[e].x * w[e].x + w[e].y * w[e].y;
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
        partial[blockIdx.x] = t;
    }
}

// out[v] = sqrt(sum_c partial[v * nch + c])
__global__ void norm_finish_kernel(int nvec, int nch, const double *__restrict__ partial,
                                   double *out) {
    for (int v = threadIdx.x; v < nvec; v += blockDim.x) {
        double t = 0.0;
        for (int c = 0; c < nch; ++c) t += partial[(int64_t)v * nch + c];
        out[v] = sqrt(t);
    }
}

// Hcol[q] = h1[q] + h2[q] for q <= j; Hcol[j+1] = |w|; nrm_out = |w|
__global__ void finish_col_kernel(int j, int nch, const double *__restrict__ partial,
                                  const cd *__restrict__ h1, const cd *__restrict__ h2, cd *Hcol,
                                  double *nrm_out) {
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int c = 0; c < nch; ++c) t += partial[c];
        const double nrm = sqrt(t);
        Hcol[j + 1] = cmk(nrm, 0.0);
        *nrm_out = nrm;
    }
    for (int q = threadIdx.x; q <= j; q += blockDim.x) Hcol[q] = cadd(h1[q], h2[q]);
}

// v_out = w / nrm (zero if nrm == 0: an exact breakdown)
__global__ void scale_kernel(int64_t L, const cd *__restrict__ w, const double *nrm,
                             cd *__restrict__ v) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L) return;
    const double s = *nrm;
    v[e] = s > 0.0 ? cscale(w[e], 1.0 / s) : cmk(0, 0);
}

// Givens step j on column j of H (complex rotations, LAPACK zlartg-style
// with real cosine): apply rotations 0..j-1, form rotation j zeroing
// H[j+1, j], rotate g; out[0] = |g[j+1]|.
__global__ void givens_kernel(int j, cd *H, int64_t ldh, double *cs, cd *sn, cd *g,
                              double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    cd *h = H + (int64_t)j * ldh;
    for (int i = 0; i < j; ++i) {
        const cd a = h[i], b = h[i + 1];
        // [c  s; -conj(s) c] [a; b]
        h[i] = cadd(cscale(a, cs[i]), cmul(sn[i], b));
        h[i + 1] = csub(cscale(b, cs[i]), cmul(cmk(sn[i].x, -sn[i].y), a));
    }
    const cd a = h[j], b = h[j + 1];
    const double na = hypot(a.x, a.y), nb = hypot(b.x, b.y);
    double c;
    cd s, r;
    if (nb == 0.0) {
        c = 1.0;
        s = cmk(0, 0);
        r = a;
    } else if (na == 0.0) {
        c = 0.0;
        s = cmk(b.x / nb, -b.y / nb);          // conj(b) / |b|
        r = cmk(nb, 0.0);
    } else {
        const double nrm = hypot(na, nb);
        c = na / nrm;
        const cd ph = cmk(a.x / na, a.y / na);   // a / |a|
        s = cmul(ph, cmk(b.x / nrm, -b.y / nrm));   // (a/|a|) conj(b) / nrm
        r = cscale(ph, nrm);
    }
    cs[j] = c;
    sn[j] = s;
    h[j] = r;
    h[j + 1] = cmk(0, 0);
    const cd gj = g[j];
    g[j] = cscale(gj, c);
    g[j + 1] = cmul(cmk(-s.x, s.y), gj);         // -conj(s) g_j
    out[0] = hypot(g[j + 1].x, g[j + 1].y);
}

// y = R^{-1} g (R = upper triangle of H, m x m), one thread
__global__ void backsub_kernel(int m, const cd *H, int64_t ldh, const cd *g, cd *y) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = m - 1; i >= 0; --i) {
        cd t = g[i];
        for (int k = i + 1; k < m; ++k) t = csub(t, cmul(H[(int64_t)k * ldh + i], y[k]));
        const cd d = H[(int64_t)i * ldh + i];
        y[i] = (d.x == 0.0 && d.y == 0.0) ? cmk(0, 0) : cmul(t, crcp(d));
    }
}

// x += V[:, 0:m] y
__global__ void update_kernel(int64_t L, int m, const cd *__restrict__ V, int64_t ldv,
                              const cd *__restrict__ y, cd *__restrict__ x) {
    extern __shared__ cd sh_y[];
    for (int q = threadIdx.x; q < m; q += blockDim.x) sh_y[q] = y[q];
    __syncthreads();
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L) return;
    cd acc = x[e];
    for (int q = 0; q < m; ++q) acc = cadd(acc, cmul(V[(int64_t)q * ldv + e], sh_y[q]));
    x[e] = acc;
}

}  // namespace gm
}  // namespace mnpb

using namespace mnpb;

static int64_t gm_chunks(int64_t L) { return (L + gm::CH - 1) / gm::CH; }

// Scratch (bytes) for mnpb_gmres_arnoldi with basis index up to jmax.
extern "C" int64_t mnpb_gmres_workspace(int64_t L, int64_t jmax) {
    const int64_t nch = gm_chunks(L);
    return (jmax + 1) * nch * 16 + 2 * (jmax + 1) * 16 + nch * 8 + 8 + 1024;
}

extern "C" int mnpb_gmres_arnoldi(void *stream, int64_t L, int64_t j, double *V, int64_t ldv,
                                  double *w, double *Hcol, double *nrm, void *work,
                                  int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(L > 0 && j >= 0 && ldv >= L && j < 4096, "gmres_arnoldi: bad sizes");
    MNPB_REQUIRE(V && w && Hcol && nrm && work, "gmres_arnoldi: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_gmres_workspace(L, j), "gmres_arnoldi: workspace too small");
    cudaStream_t s = as_stream(stream);
    const int nq = (int)j + 1;
    const int nch = (int)gm_chunks(L);
    char *wp = (char *)work;
    cd *partial = (cd *)wp;
    wp += (int64_t)nq * nch * 16;
    cd *h1 = (cd *)wp;
    cd *h2 = h1 + nq;
    double *np_ = (double *)(h2 + nq);
    ProfScope ps(s, PC_GMRES, 4.0 * 16.0 * (double)L * nq);
    const unsigned gl = (unsigned)((L + 255) / 256);
    const size_t shq = (size_t)nq * 16;
    if (shq > 48 * 1024) {
        set_error("gmres_arnoldi: basis too large (%d vectors)", nq);
        return MNPB_EINVAL;
    }
    cd *hs[2] = {h1, h2};
    for (int pass = 0; pass < 2; ++pass) {
        gm::dots_kernel<<<dim3(nch, nq), 256, 0, s>>>(L, nq, (const cd *)V, ldv, (const cd *)w,
                                                     partial, nch);
        gm::reduce_dots_kernel<<<(nq + 127) / 128, 128, 0, s>>>(nq, nch, partial, hs[pass], 0);
        gm::project_kernel<<<gl, 256, shq, s>>>(L, nq, (const cd *)V, ldv, hs[pass], (cd *)w);
    }
    gm::norm_kernel<<<nch, 256, 0, s>>>(L, (const cd *)w, np_);
    gm::finish_col_kernel<<<1, 256, 0, s>>>((int)j, nch, np_, h1, h2, (cd *)Hcol, nrm);
    gm::scale_kernel<<<gl, 256, 0, s>>>(L, (const cd *)w, nrm, (cd *)V + (int64_t)(j + 1) * ldv);
    count_launch(8);
    MNPB_LAUNCH_CHECK("gmres arnoldi kernels");
    return MNPB_OK;
}

extern "C" int mnpb_gmres_givens(void *stream, int64_t j, double *H, int64_t ldh, double *cs,
                                 double *sn, double *g, double *out) {
    clear_error();
    MNPB_REQUIRE(j >= 0 && ldh >= j + 2, "gmres_givens: bad sizes");
    MNPB_REQUIRE(H && cs && sn && g && out, "gmres_givens: null pointer");
    cudaStream_t s = as_stream(stream);
    gm::givens_kernel<<<1, 32, 0, s>>>((int)j, (cd *)H, ldh, cs, (cd *)sn, (cd *)g, out);
    MNPB_LAUNCH_CHECK("givens_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_gmres_update(void *stream, int64_t L, int64_t m, const double *H,
                                 int64_t ldh, const double *g, const double *V, int64_t ldv,
                                 double *y, double *x) {
    clear_error();
    MNPB_REQUIRE(L > 0 && m >= 0 && ldh >= m && ldv >= L && m < 3000, "gmres_update: bad sizes");
    if (m == 0) return MNPB_OK;
    MNPB_REQUIRE(H && g && V && y && x, "gmres_update: null pointer");
    cudaStream_t s = as_stream(stream);
    gm::backsub_kernel<<<1, 32, 0, s>>>((int)m, (const cd *)H, ldh, (const cd *)g, (cd *)y);
    gm::update_kernel<<<(unsigned)((L + 255) / 256), 256, (size_t)m * 16, s>>>(
        L, (int)m, (const cd *)V, ldv, (const cd *)y, (cd *)x);
    count_launch(1);
    MNPB_LAUNCH_CHECK("gmres update kernels");
    return MNPB_OK;
}

// Euclidean norms of nvec vectors of L complex entries (stride ldx):
// out[v] = |x_v|, deterministic two-stage sums.  partial: nvec * ceil(L/2048)
// doubles of scratch.
extern "C" int mnpb_vec_norms(void *stream, int64_t L, int64_t nvec, const double *x,
                              int64_t ldx, double *partial, double *out) {
    clear_error();
    MNPB_REQUIRE(L > 0 && nvec > 0 && ldx >= L && x && partial && out, "vec_norms: bad arguments");
    cudaStream_t s = as_stream(stream);
    const int nch = (int)gm_chunks(L);
    for (int64_t v = 0; v < nvec; ++v)
        gm::norm_kernel<<<nch, 256, 0, s>>>(L, (const cd *)x + v * ldx, partial + v * nch);
    gm::norm_finish_kernel<<<1, 128, 0, s>>>((int)nvec, nch, partial, out);
    MNPB_LAUNCH_CHECK("vec_norms kernels");
    return MNPB_OK;
}
