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
#include "bemret_kernels.cuh"

using namespace mnpb::bemk;

using namespace mnpb;

static int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

extern "C" int64_t mnpb_bemret_workspace_f64(int64_t n, int64_t batch) {
    // W: batch x n x n complex; pivD: batch x n int32
    return align_up(batch * n * n * 16, 256) + align_up(batch * n * 4, 256);
}

extern "C" int mnpb_bemret_init_f64(void *stream, int64_t n, int64_t batch, double *G1,
                                    double *G2, double *H1, double *H2, double *D, int64_t ld,
                                    int64_t stride, const double *eps, const double *kvac,
                                    const double *nvec, int64_t nvec_stride, int32_t *piv,
                                    int32_t *info, void *work, int64_t work_bytes) {
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
    // pivots [3][batch][n]: G1, G2, Sigma; info [2][batch]
    const int64_t ps = n;
    int32_t *piv1 = piv, *piv2 = piv + batch * n, *pivS = piv + 2 * batch * n;
    if (cudaMemsetAsync(info, 0, sizeof(int32_t) * 2 * batch, s) != cudaSuccess) {
        set_error("bemret_init: memset failed");
        return MNPB_ECUDA;
    }
    // G1 and G2 (and H1, H2) stored back to back go through every launch together
    const bool pair = (g2 == g1 + batch * stride) && (h2 == h1 + batch * stride);
    if (pair) {
        MNPB_TRY(getrf(s, N, 2 * B, g1, ld, stride, piv1, ps, info));
        MNPB_TRY(right_solve(s, N, N, 2 * B, g1, ld, stride, piv1, ps, h1, ld, stride));
    } else {
        MNPB_TRY(getrf(s, N, B, g1, ld, stride, piv1, ps, info));
        MNPB_TRY(getrf(s, N, B, g2, ld, stride, piv2, ps, info + batch));
        MNPB_TRY(right_solve(s, N, N, B, g1, ld, stride, piv1, ps, h1, ld, stride));
        MNPB_TRY(right_solve(s, N, N, B, g2, ld, stride, piv2, ps, h2, ld, stride));
    }
    dim3 grid(ceil_div(n, 128), N, B);
    form_delta_kernel<<<grid, 128, 0, s>>>(N, h1, h2, d, ld, stride, eps, kvac);
    MNPB_LAUNCH_CHECK("form_delta_kernel");
    MNPB_TRY(getrf(s, N, B, d, ld, stride, pivD, n, info));
    MNPB_TRY(set_identity(s, N, B, W, n, sw));
    MNPB_TRY(getrs(s, N, N, B, d, ld, stride, pivD, n, W, n, sw));
    form_sigma_kernel<<<grid, 128, 0, s>>>(N, h2, W, n, sw, d, ld, stride, eps, kvac,
                                           NvecView{nvec, nvec_stride});
    MNPB_LAUNCH_CHECK("form_sigma_kernel");
    MNPB_TRY(getrf(s, N, B, h2, ld, stride, pivS, ps, info));
    return MNPB_OK;
}

extern "C" int mnpb_bemret_solve_f64(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                                     const double *G1, const double *G2, const double *S1,
                                     const double *S, const double *D, int64_t ld,
                                     int64_t stride, const int32_t *piv, const double *eps,
                                     const double *kvac, const double *nvec, int64_t nvec_stride,
                                     const double *x_in, double *x_out, void *work,
                                     int64_t work_bytes) {
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
    const int64_t ps = n;
    const int32_t *piv1 = piv, *piv2 = piv + batch * n, *pivS = piv + 2 * batch * n;
    const NvecView nv{nvec, nvec_stride};
    dim3 g(ceil_div(n, 128), B);
    solve_prep_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, T, sT, eps, kvac);
    MNPB_LAUNCH_CHECK("solve_prep_kernel");
    MNPB_TRY(zgemm(s, N, 4 * k, N, B, cmk(1, 0), (const cd *)S1, ld, stride, T, n, sT, cmk(0, 0),
                   U, n, sT));
    solve_alpha_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, U, sT, AP, sAP, R, sR, eps, kvac, nv);
    MNPB_LAUNCH_CHECK("solve_alpha_kernel");
    MNPB_TRY(zgemm(s, N, 3 * k, N, B, cmk(1, 0), (const cd *)D, ld, stride, AP, n, sAP,
                   cmk(0, 0), V, n, sAP));
    solve_rhs_kernel<<<g, 128, 0, s>>>(N, k, V, sAP, R, sR, eps, kvac, nv);
    MNPB_LAUNCH_CHECK("solve_rhs_kernel");
    MNPB_TRY(getrs(s, N, k, B, (const cd *)S, ld, stride, pivS, ps, R, n, sR));
    solve_h2pre_kernel<<<g, 128, 0, s>>>(N, k, AP, sAP, R, sR, eps, kvac, nv);
    MNPB_LAUNCH_CHECK("solve_h2pre_kernel");
    MNPB_TRY(zgemm(s, N, 3 * k, N, B, cmk(1, 0), (const cd *)D, ld, stride, AP, n, sAP,
                   cmk(0, 0), V, n, sAP));
    solve_out_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, R, sR, V, sAP, xout, sx);
    MNPB_LAUNCH_CHECK("solve_out_kernel");
    MNPB_TRY(getrs(s, N, 4 * k, B, (const cd *)G1, ld, stride, piv1, ps, xout, n, sx));
    MNPB_TRY(getrs(s, N, 4 * k, B, (const cd *)G2, ld, stride, piv2, ps, xout + 4 * K * n, n,
                   sx));
    return MNPB_OK;
}

extern "C" int mnpb_bemret_excitation(void *stream, int64_t n, int64_t batch, int64_t nrhs,
                                      const double *pots, const double *eps, const double *kvac,
                                      const double *nvec, int64_t nvec_stride, double *x_in) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && nrhs > 0 && batch < 65536, "bemret_excitation: bad sizes");
    MNPB_REQUIRE(pots && eps && kvac && nvec && x_in, "bemret_excitation: null pointer");
    dim3 g(ceil_div(n, 128), (unsigned)batch);
    excitation_kernel<<<g, 128, 0, as_stream(stream)>>>((int)n, (int)nrhs, (const cd *)pots,
                                                        (cd *)x_in, eps, kvac,
                                                        NvecView{nvec, nvec_stride});
    MNPB_LAUNCH_CHECK("excitation_kernel");
    return MNPB_OK;
}

// ---------------------------------------------------------------------------
// Entries of different face counts in one batch: entry e holds its particle's
// n_e x n_e matrices in the top-left corner of npad x npad buffers.  The rest
// becomes block-diagonal identity padding -- G1 = G2 = H1 = I, H2 = 0 on the
// pad block, zero coupling -- so Sigma1 = I, Sigma2 = 0, Delta = I and
// Sigma = eps1 I there, every factorisation stays exact for the particle's
// block, and a zero right-hand side on the pad gives a zero solution there.
// ---------------------------------------------------------------------------
namespace {
__global__ void pad_entries_kernel(int npad, const int32_t *__restrict__ n_of, cd *G1, cd *G2,
                                   cd *H1, cd *H2, int64_t ld, int64_t st, float *G1p, float *G2p,
                                   float *H1p, float *H2p, int64_t ldp, int64_t planep,
                                   int64_t stp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int64_t e = blockIdx.z;
    const int ne = n_of[e];
    if (i >= npad || (i < ne && j < ne)) return;
    const double d = i == j ? 1.0 : 0.0;
    const int64_t o = e * st + (int64_t)j * ld + i;
    G1[o] = G2[o] = H1[o] = cmk(d, 0.0);
    H2[o] = cmk(0.0, 0.0);
    const int64_t op = e * stp + (int64_t)j * ldp + i;
    G1p[op] = G2p[op] = H1p[op] = (float)d;
    G1p[op + planep] = G2p[op + planep] = H1p[op + planep] = 0.f;
    H2p[op] = H2p[op + planep] = 0.f;
}
}  // namespace

extern "C" int mnpb_pad_entries(void *stream, int64_t npad, int64_t batch,
                                const int32_t *n_of_entry, double *G1, double *G2, double *H1,
                                double *H2, int64_t ld, int64_t stride, float *G1p, float *G2p,
                                float *H1p, float *H2p, int64_t ldp, int64_t planep,
                                int64_t stridep) {
    clear_error();
    MNPB_REQUIRE(npad > 0 && npad < 65536 && batch > 0 && batch < 65536 && ld >= npad &&
                     stride >= ld * npad && ldp >= npad && planep >= ldp * npad &&
                     stridep >= 2 * planep,
                 "pad_entries: bad sizes");
    MNPB_REQUIRE(n_of_entry && G1 && G2 && H1 && H2 && G1p && G2p && H1p && H2p,
                 "pad_entries: null pointer");
    dim3 grid(ceil_div(npad, 128), (unsigned)npad, (unsigned)batch);
    pad_entries_kernel<<<grid, 128, 0, as_stream(stream)>>>(
        (int)npad, n_of_entry, (cd *)G1, (cd *)G2, (cd *)H1, (cd *)H2, ld, stride, G1p, G2p, H1p,
        H2p, ldp, planep, stridep);
    MNPB_LAUNCH_CHECK("pad_entries_kernel");
    return MNPB_OK;
}
