// Retarded BEM solver (BEMRet) in FP64 on the GPU, batched over wavelengths.
//
// init (mnpbem/bem/bem_ret.py:437-523), Garcia de Abajo & Howie PRB 65,
// 115418 (2002) Eqs. (19-22), for scalar (per-wavelength) eps1, eps2:
//   LU(G1), LU(G2); Sigma1 = H1 G1^-1, Sigma2 = H2 G2^-1 (right solves);
//   Delta = Sigma1 - Sigma2; Delta^-1 from LU(Delta);
//   Sigma = eps1 Sigma1 - eps2 Sigma2 + k^2 (eps1-eps2)^2 (Delta^-1 o n n^T);
//   LU(Sigma).
// solve (bem_ret.py:1690-1810):
//   alpha' = alpha - Sigma1 a + ik n (eps1 phi)
//   De'    = De - Sigma1 (eps1 phi) + ik n.(eps1 a)
//   sig2   = Sigma^-1 (De' + ik n.((eps1-eps2) Delta^-1 alpha'))
//   h2     = Delta^-1 (ik n (eps1-eps2) sig2 + alpha')
//   sig1 = G1^-1 (sig2 + phi), h1 = G1^-1 (h2 + a), sig2 = G2^-1 sig2, h2 = G2^-1 h2
#include "common.cuh"
#include "dense_f64.cuh"

namespace mnpb {
namespace {

struct EpsK {
    cd e1, e2;
    double k;
};

__device__ __forceinline__ EpsK load_epsk(const double *eps, const double *kvac, int64_t b) {
    EpsK r;
    r.e1 = cmk(eps[4 * b], eps[4 * b + 1]);
    r.e2 = cmk(eps[4 * b + 2], eps[4 * b + 3]);
    r.k = kvac[b];
    return r;
}

// D = S1 - S2 ; S2 <- eps1 S1 - eps2 S2
__global__ void form_delta_kernel(int n, const cd *S1, cd *S2, cd *D, int64_t ld, int64_t st,
                                  const double *eps, const double *kvac) {
    const int64_t b = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const int64_t o = b * st + (int64_t)j * ld + i;
    const cd s1 = S1[o], s2 = S2[o];
    D[o] = csub(s1, s2);
    S2[o] = csub(cmul(ek.e1, s1), cmul(ek.e2, s2));
}

// S <- S + k^2 (eps1-eps2)^2 (W o n n^T) ; D <- W
__global__ void form_sigma_kernel(int n, cd *S, const cd *W, int64_t ldw, int64_t sw, cd *D,
                                  int64_t ld, int64_t st, const double *eps, const double *kvac,
                                  const double *nvec) {
    const int64_t b = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd L = csub(ek.e1, ek.e2);
    const cd c = cscale(cmul(L, L), ek.k * ek.k);
    const double nn = nvec[3 * i] * nvec[3 * j] + nvec[3 * i + 1] * nvec[3 * j + 1] +
                      nvec[3 * i + 2] * nvec[3 * j + 2];
    const int64_t o = b * st + (int64_t)j * ld + i;
    const cd w = W[b * sw + (int64_t)j * ldw + i];
    S[o] = cadd(S[o], cmul(c, cscale(w, nn)));
    D[o] = w;
}

// x_in columns: phi[0,K) a[K,4K) De[4K,5K) alpha[5K,8K) (component-major)
// T = [a | eps1 phi]
__global__ void solve_prep_kernel(int n, int K, const cd *xin, int64_t sx, cd *T, int64_t sT,
                                  const double *eps, const double *kvac) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd *x = xin + b * sx;
    cd *t = T + b * sT;
    for (int c = 0; c < 3 * K; ++c) t[(int64_t)c * n + i] = x[(int64_t)(K + c) * n + i];
    for (int r = 0; r < K; ++r) t[(int64_t)(3 * K + r) * n + i] = cmul(ek.e1, x[(int64_t)r * n + i]);
}

// U = Sigma1 T.  AP = alpha' (n x 3K), R = De' (n x K)
__global__ void solve_alpha_kernel(int n, int K, const cd *xin, int64_t sx, const cd *U,
                                   int64_t sU, cd *AP, int64_t sAP, cd *R, int64_t sR,
                                   const double *eps, const double *kvac, const double *nvec) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd *x = xin + b * sx;
    const cd *u = U + b * sU;
    cd *ap = AP + b * sAP;
    cd *rr = R + b * sR;
    const cd ik = cmk(0.0, ek.k);
    const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
    for (int r = 0; r < K; ++r) {
        const cd e1phi = cmul(ek.e1, x[(int64_t)r * n + i]);
        cd nea = cmk(0, 0);
        for (int c = 0; c < 3; ++c) {
            const int col = c * K + r;
            const cd alpha = x[(int64_t)(5 * K + col) * n + i];
            const cd s1a = u[(int64_t)col * n + i];
            ap[(int64_t)col * n + i] = cadd(csub(alpha, s1a), cmul(ik, cscale(e1phi, nv[c])));
            nea = cadd(nea, cscale(cmul(ek.e1, x[(int64_t)(K + col) * n + i]), nv[c]));
        }
        const cd de = x[(int64_t)(4 * K + r) * n + i];
        const cd s1phi = u[(int64_t)(3 * K + r) * n + i];
        rr[(int64_t)r * n + i] = cadd(csub(de, s1phi), cmul(ik, nea));
    }
}

// R += ik n.((eps1-eps2) V)   with V = Delta^-1 alpha' (n x 3K)
__global__ void solve_rhs_kernel(int n, int K, const cd *V, int64_t sV, cd *R, int64_t sR,
                                 const double *eps, const double *kvac, const double *nvec) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd L = csub(ek.e1, ek.e2);
    const cd ikL = cmul(cmk(0.0, ek.k), L);
    const cd *v = V + b * sV;
    cd *rr = R + b * sR;
    for (int r = 0; r < K; ++r) {
        cd s = cmk(0, 0);
        for (int c = 0; c < 3; ++c) s = cadd(s, cscale(v[(int64_t)(c * K + r) * n + i], nvec[3 * i + c]));
        rr[(int64_t)r * n + i] = cadd(rr[(int64_t)r * n + i], cmul(ikL, s));
    }
}

// AP <- ik n (eps1-eps2) sig2 + AP     (sig2 in R)
__global__ void solve_h2pre_kernel(int n, int K, cd *AP, int64_t sAP, const cd *R, int64_t sR,
                                   const double *eps, const double *kvac, const double *nvec) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd ikL = cmul(cmk(0.0, ek.k), csub(ek.e1, ek.e2));
    cd *ap = AP + b * sAP;
    const cd *rr = R + b * sR;
    for (int r = 0; r < K; ++r) {
        const cd t = cmul(ikL, rr[(int64_t)r * n + i]);
        for (int c = 0; c < 3; ++c) {
            const int64_t o = (int64_t)(c * K + r) * n + i;
            ap[o] = cadd(ap[o], cscale(t, nvec[3 * i + c]));
        }
    }
}

// out = [sig2 + phi | h2 + a | sig2 | h2]
__global__ void solve_out_kernel(int n, int K, const cd *xin, int64_t sx, const cd *R,
                                 int64_t sR, const cd *H, int64_t sH, cd *out, int64_t so) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cd *x = xin + b * sx;
    const cd *rr = R + b * sR;
    const cd *h = H + b * sH;
    cd *o = out + b * so;
    for (int r = 0; r < K; ++r) {
        const cd s2 = rr[(int64_t)r * n + i];
        o[(int64_t)r * n + i] = cadd(s2, x[(int64_t)r * n + i]);
        o[(int64_t)(4 * K + r) * n + i] = s2;
    }
    for (int c = 0; c < 3 * K; ++c) {
        const cd hv = h[(int64_t)c * n + i];
        o[(int64_t)(K + c) * n + i] = cadd(hv, x[(int64_t)(K + c) * n + i]);
        o[(int64_t)(5 * K + c) * n + i] = hv;
    }
}


// Excitation variables (mnpbem/bem/bem_ret.py:1360-1429):
//   phi = phi2 - phi1, a = a2 - a1,
//   alpha = a2' - a1' - ik (n phi2 eps2 - n phi1 eps1),
//   De = eps2 phi2' - eps1 phi1' - ik (n.a2 eps2 - n.a1 eps1).
// pots columns (component-major, K each): phi1, phi1', a1 (3), a1' (3),
// phi2, phi2', a2 (3), a2' (3).
__global__ void excitation_kernel(int n, int K, const cd *pots, cd *xin, const double *eps,
                                  const double *kvac, const double *nvec) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd ik = cmk(0.0, ek.k);
    const cd *q = pots + b * (int64_t)n * 16 * K;
    cd *x = xin + b * (int64_t)n * 8 * K;
    auto P = [&](int comp, int r) { return q[(int64_t)(comp * K + r) * n + i]; };
    const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
    for (int r = 0; r < K; ++r) {
        const cd phi1 = P(0, r), phi1p = P(1, r), phi2 = P(8, r), phi2p = P(9, r);
        x[(int64_t)r * n + i] = csub(phi2, phi1);
        cd na1 = cmk(0, 0), na2 = cmk(0, 0);
        for (int c = 0; c < 3; ++c) {
            const cd a1 = P(2 + c, r), a1p = P(5 + c, r), a2 = P(10 + c, r), a2p = P(13 + c, r);
            x[(int64_t)(K + c * K + r) * n + i] = csub(a2, a1);
            const cd t = csub(cscale(cmul(phi2, ek.e2), nv[c]), cscale(cmul(phi1, ek.e1), nv[c]));
            x[(int64_t)(5 * K + c * K + r) * n + i] = csub(csub(a2p, a1p), cmul(ik, t));
            na1 = cadd(na1, cscale(a1, nv[c]));
            na2 = cadd(na2, cscale(a2, nv[c]));
        }
        const cd de = csub(cmul(ek.e2, phi2p), cmul(ek.e1, phi1p));
        x[(int64_t)(4 * K + r) * n + i] =
            csub(de, cmul(ik, csub(cmul(na2, ek.e2), cmul(na1, ek.e1))));
    }
}

}  // namespace
}  // namespace mnpb

using namespace mnpb;

static int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

extern "C" int64_t mnpb_bemret_workspace_f64(int64_t n, int64_t batch) {
    // W: batch x n x n complex; pivD: batch x n int32
    return align_up(batch * n * n * 16, 256) + align_up(batch * n * 4, 256);
}

extern "C" int mnpb_bemret_init_f64(void *stream, int64_t n, int64_t batch, double *G1,
                                    double *G2, double *H1, double *H2, double *D, int64_t ld,
                                    int64_t stride, const double *eps, const double *kvac,
                                    const double *nvec, int32_t *piv, int32_t *info, void *work,
                                    int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && batch < 65536 && n < 65536 && ld >= n &&
                     stride >= ld * n,
                 "bemret_init: bad sizes");
    MNPB_REQUIRE(G1 && G2 && H1 && H2 && D && eps && kvac && nvec && piv && info && work,
                 "bemret_init: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_bemret_workspace_f64(n, batch),
                 "bemret_init: workspace %lld < %lld bytes", (long long)work_bytes,
                 (long long)mnpb_bemret_workspace_f64(n, batch));
    cudaStream_t s = as_stream(stream);
    const int N = (int)n, B = (int)batch;
    cd *g1 = (cd *)G1, *g2 = (cd *)G2, *h1 = (cd *)H1, *h2 = (cd *)H2, *d = (cd *)D;
    cd *W = (cd *)work;
    const int64_t sw = n * n;
    int32_t *pivD = (int32_t *)((char *)work + align_up(batch * n * n * 16, 256));
    const int64_t ps = 3 * n;
    if (cudaMemsetAsync(info, 0, sizeof(int32_t) * batch, s) != cudaSuccess) {
        set_error("bemret_init: memset failed");
        return MNPB_ECUDA;
    }
    MNPB_TRY(getrf(s, N, B, g1, ld, stride, piv, ps, info));
    MNPB_TRY(getrf(s, N, B, g2, ld, stride, piv + n, ps, info));
    MNPB_TRY(right_solve(s, N, N, B, g1, ld, stride, piv, ps, h1, ld, stride));
    MNPB_TRY(right_solve(s, N, N, B, g2, ld, stride, piv + n, ps, h2, ld, stride));
    dim3 grid(ceil_div(n, 128), N, B);
    form_delta_kernel<<<grid, 128, 0, s>>>(N, h1, h2, d, ld, stride, eps, kvac);
    MNPB_LAUNCH_CHECK("form_delta_kernel");
    MNPB_TRY(getrf(s, N, B, d, ld, stride, pivD, n, info));
    MNPB_TRY(set_identity(s, N, B, W, n, sw));
    MNPB_TRY(getrs(s, N, N, B, d, ld, stride, pivD, n, W, n, sw));
    form_sigma_kernel<<<grid, 128, 0, s>>>(N, h2, W, n, sw, d, ld, stride, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("form_sigma_kernel");
    MNPB_TRY(getrf(s, N, B, h2, ld, stride, piv + 2 * n, ps, info));
    return MNPB_OK;
}

extern "C" int mnpb_bemret_solve_f64(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                                     const double *G1, const double *G2, const double *S1,
                                     const double *S, const double *D, int64_t ld,
                                     int64_t stride, const int32_t *piv, const double *eps,
                                     const double *kvac, const double *nvec, const double *x_in,
                                     double *x_out, void *work, int64_t work_bytes) {
    clear_error();
    const int64_t K = nrhs;
    MNPB_REQUIRE(n > 0 && batch > 0 && K > 0 && K <= 64 && ld >= n, "bemret_solve: bad sizes");
    MNPB_REQUIRE(G1 && G2 && S1 && S && D && piv && eps && kvac && nvec && x_in && x_out && work,
                 "bemret_solve: null pointer");
    const int64_t per = n * (4 * K + 4 * K + 3 * K + 3 * K + K);
    MNPB_REQUIRE(work_bytes >= batch * per * 16, "bemret_solve: workspace %lld < %lld bytes",
                 (long long)work_bytes, (long long)(batch * per * 16));
    cudaStream_t s = as_stream(stream);
    const int N = (int)n, B = (int)batch, k = (int)K;
    cd *T = (cd *)work;
    cd *U = T + batch * n * 4 * K;
    cd *AP = U + batch * n * 4 * K;
    cd *V = AP + batch * n * 3 * K;
    cd *R = V + batch * n * 3 * K;
    const int64_t sT = n * 4 * K, sAP = n * 3 * K, sR = n * K, sx = n * 8 * K;
    const cd *xin = (const cd *)x_in;
    cd *xout = (cd *)x_out;
    const int64_t ps = 3 * n;
    dim3 g(ceil_div(n, 128), B);
    solve_prep_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, T, sT, eps, kvac);
    MNPB_LAUNCH_CHECK("solve_prep_kernel");
    MNPB_TRY(zgemm(s, N, 4 * k, N, B, cmk(1, 0), (const cd *)S1, ld, stride, T, n, sT, cmk(0, 0),
                   U, n, sT));
    solve_alpha_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, U, sT, AP, sAP, R, sR, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("solve_alpha_kernel");
    MNPB_TRY(zgemm(s, N, 3 * k, N, B, cmk(1, 0), (const cd *)D, ld, stride, AP, n, sAP,
                   cmk(0, 0), V, n, sAP));
    solve_rhs_kernel<<<g, 128, 0, s>>>(N, k, V, sAP, R, sR, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("solve_rhs_kernel");
    MNPB_TRY(getrs(s, N, k, B, (const cd *)S, ld, stride, piv + 2 * n, ps, R, n, sR));
    solve_h2pre_kernel<<<g, 128, 0, s>>>(N, k, AP, sAP, R, sR, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("solve_h2pre_kernel");
    MNPB_TRY(zgemm(s, N, 3 * k, N, B, cmk(1, 0), (const cd *)D, ld, stride, AP, n, sAP,
                   cmk(0, 0), V, n, sAP));
    solve_out_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, R, sR, V, sAP, xout, sx);
    MNPB_LAUNCH_CHECK("solve_out_kernel");
    MNPB_TRY(getrs(s, N, 4 * k, B, (const cd *)G1, ld, stride, piv, ps, xout, n, sx));
    MNPB_TRY(getrs(s, N, 4 * k, B, (const cd *)G2, ld, stride, piv + n, ps, xout + 4 * K * n, n,
                   sx));
    return MNPB_OK;
}

extern "C" int mnpb_bemret_excitation(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                                      const double *pots, const double *eps, const double *kvac,
                                      const double *nvec, double *x_in) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && nrhs > 0 && batch < 65536, "bemret_excitation: bad sizes");
    MNPB_REQUIRE(pots && eps && kvac && nvec && x_in, "bemret_excitation: null pointer");
    dim3 g(ceil_div(n, 128), (unsigned)batch);
    excitation_kernel<<<g, 128, 0, as_stream(stream)>>>((int)n, (int)nrhs, (const cd *)pots,
                                                        (cd *)x_in, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("excitation_kernel");
    return MNPB_OK;
}
