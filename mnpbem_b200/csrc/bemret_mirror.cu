// Retarded BEM solver for particles with mirror symmetry (BEMRetMirror), FP64,
// batched over wavelengths.
//
// The particle is given by its irreducible part (n faces); the full particle
// repeats it in nk = 2 (sym 'x' or 'y') or 4 ('xy') mirror images.  For each
// symmetry value s (a row of the symmetry table tab, nsym = nk rows) the
// Green functions contract to n x n matrices
//   G_s(i, j) = sum_k tab[s][k] G_full(i, j + k n)          (i, j < n)
// (mnpbem/greenfun/compgreen_ret_mirror.py:36-95).  Per wavelength and
// symmetry value (an "entry", e = b * nsym + s):
//   LU(G1_s), LU(G2_s), Sigma1_s = H1_s G1_s^-1, Sigma2_s = H2_s G2_s^-1,
//   Delta_s^-1 = (Sigma1_s - Sigma2_s)^-1
// (mnpbem/bem/bem_ret_mirror.py:182-328).  An excitation whose x, y, z
// components carry symmetry values with table rows (x, y, z) needs
//   Sigma_xyz = eps1 Sigma1_z - eps2 Sigma2_z
//             + k^2 (eps1 - eps2)^2 sum_d n_d n_d^T o Delta_{idx_d}^-1
// (bem_ret_mirror.py:568-619, Garcia de Abajo & Howie PRB 65, 115418, Eqs.
// 21-22) and is solved as BEMRet with the matrices of component d taken at
// idx_d (bem_ret_mirror.py:654-760).  Scalar (per-wavelength) eps1, eps2.
#include "common.cuh"
#include "dense_f64.cuh"
#include "bemret_kernels.cuh"

using namespace mnpb::bemk;
using namespace mnpb;

namespace {

constexpr int MAX_NK = 4;

struct Tab {
    double t[MAX_NK * MAX_NK];
};

// out(b, s)[i, j] = sum_k tab[s][k] full(b)[i, j + k n]
__global__ void mirror_contract_kernel(int n, int nk, int nsym, const cd *__restrict__ full,
                                       int64_t ldf, int64_t sf, Tab tab, cd *__restrict__ out,
                                       int64_t ld, int64_t so) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (i >= n) return;
    cd v[MAX_NK];
    const cd *f = full + b * sf + i;
    for (int k = 0; k < nk; ++k) v[k] = f[(int64_t)(j + k * n) * ldf];
    for (int s = 0; s < nsym; ++s) {
        cd acc = cmk(0.0, 0.0);
        for (int k = 0; k < nk; ++k) acc = cadd(acc, cscale(v[k], tab.t[s * nk + k]));
        out[(b * nsym + s) * so + (int64_t)j * ld + i] = acc;
    }
}

// D = S1 - S2 (entry-wise)
__global__ void mirror_delta_kernel(int n, const cd *S1, const cd *S2, cd *D, int64_t ld,
                                    int64_t st, int64_t ldd, int64_t sd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int64_t e = blockIdx.z;
    if (i >= n) return;
    const int64_t o = e * st + (int64_t)j * ld + i;
    D[e * sd + (int64_t)j * ldd + i] = csub(S1[o], S2[o]);
}

// S(b) = eps1 Sigma1_z - eps2 Sigma2_z + k^2 (eps1-eps2)^2 sum_d n_d n_d^T o Dinv_{idx_d}
__global__ void mirror_sigma_kernel(int n, int nsym, const cd *S1, const cd *S2, const cd *Dinv,
                                    int64_t ld, int64_t st, int ix, int iy, int iz,
                                    const double *eps, const double *kvac, const double *nvec,
                                    cd *S, int64_t sS) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd L = csub(ek.e1, ek.e2);
    const cd c = cscale(cmul(L, L), ek.k * ek.k);
    const int64_t oj = (int64_t)j * ld + i;
    const int64_t ez = (b * nsym + iz) * st;
    cd acc = csub(cmul(ek.e1, S1[ez + oj]), cmul(ek.e2, S2[ez + oj]));
    const int idx[3] = {ix, iy, iz};
    cd w = cmk(0.0, 0.0);
    for (int d = 0; d < 3; ++d) {
        const double nn = nvec[3 * i + d] * nvec[3 * j + d];
        w = cadd(w, cscale(Dinv[(b * nsym + idx[d]) * st + oj], nn));
    }
    S[b * sS + oj] = cadd(acc, cmul(c, w));
}

}  // namespace

static int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

extern "C" int mnpb_mirror_contract(void *stream, int64_t n, int64_t nk, int64_t nsym,
                                    int64_t batch, const double *full, int64_t ldf, int64_t sf,
                                    const double *tab, double *out, int64_t ld, int64_t stride) {
    clear_error();
    MNPB_REQUIRE(n > 0 && n < 65536 && batch > 0 && batch < 65536, "mirror_contract: bad sizes");
    MNPB_REQUIRE((nk == 2 || nk == 4) && nsym >= 1 && nsym <= nk,
                 "mirror_contract: nk must be 2 or 4 and 1 <= nsym <= nk");
    MNPB_REQUIRE(ldf >= nk * n && ld >= n && stride >= ld * n && sf >= ldf * nk * n,
                 "mirror_contract: bad leading dimensions or strides");
    MNPB_REQUIRE(full && tab && out, "mirror_contract: null pointer");
    Tab t{};
    for (int64_t a = 0; a < nsym * nk; ++a) t.t[a] = tab[a];
    dim3 grid(ceil_div(n, 128), (unsigned)n, (unsigned)batch);
    mirror_contract_kernel<<<grid, 128, 0, as_stream(stream)>>>(
        (int)n, (int)nk, (int)nsym, (const cd *)full, ldf, sf, t, (cd *)out, ld, stride);
    MNPB_LAUNCH_CHECK("mirror_contract_kernel");
    return MNPB_OK;
}

extern "C" int64_t mnpb_bemret_mirror_workspace(int64_t n, int64_t entries) {
    return align_up(entries * n * n * 16, 256);   // LU(Delta) of every entry
}

extern "C" int mnpb_bemret_init_mirror_f64(void *stream, int64_t n, int64_t entries, double *G1,
                                           double *G2, double *H1, double *H2, int64_t ld,
                                           int64_t stride, double *Dinv, int32_t *piv,
                                           int32_t *info, void *work, int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(n > 0 && n < 65536 && entries > 0 && entries < 65536 && ld >= n &&
                     stride >= ld * n,
                 "bemret_init_mirror: bad sizes");
    MNPB_REQUIRE(G1 && G2 && H1 && H2 && Dinv && piv && info && work,
                 "bemret_init_mirror: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_bemret_mirror_workspace(n, entries),
                 "bemret_init_mirror: workspace %lld < %lld bytes", (long long)work_bytes,
                 (long long)mnpb_bemret_mirror_workspace(n, entries));
    cudaStream_t s = as_stream(stream);
    const int N = (int)n, E = (int)entries;
    cd *g1 = (cd *)G1, *g2 = (cd *)G2, *h1 = (cd *)H1, *h2 = (cd *)H2, *di = (cd *)Dinv;
    cd *D = (cd *)work;
    const int64_t sd = n * n, ps = n;
    int32_t *piv1 = piv, *piv2 = piv + entries * n, *pivD = piv + 2 * entries * n;
    if (cudaMemsetAsync(info, 0, sizeof(int32_t) * 3 * entries, s) != cudaSuccess) {
        set_error("bemret_init_mirror: memset failed");
        return MNPB_ECUDA;
    }
    if (g2 == g1 + entries * stride && h2 == h1 + entries * stride) {
        MNPB_TRY(getrf(s, N, 2 * E, g1, ld, stride, piv1, ps, info));
        MNPB_TRY(right_solve(s, N, N, 2 * E, g1, ld, stride, piv1, ps, h1, ld, stride));
    } else {
        MNPB_TRY(getrf(s, N, E, g1, ld, stride, piv1, ps, info));
        MNPB_TRY(getrf(s, N, E, g2, ld, stride, piv2, ps, info + entries));
        MNPB_TRY(right_solve(s, N, N, E, g1, ld, stride, piv1, ps, h1, ld, stride));
        MNPB_TRY(right_solve(s, N, N, E, g2, ld, stride, piv2, ps, h2, ld, stride));
    }
    dim3 grid(ceil_div(n, 128), N, E);
    mirror_delta_kernel<<<grid, 128, 0, s>>>(N, h1, h2, D, ld, stride, n, sd);
    MNPB_LAUNCH_CHECK("mirror_delta_kernel");
    MNPB_TRY(getrf(s, N, E, D, n, sd, pivD, ps, info + 2 * entries));
    MNPB_TRY(set_identity(s, N, E, di, ld, stride));
    MNPB_TRY(getrs(s, N, N, E, D, n, sd, pivD, ps, di, ld, stride));
    return MNPB_OK;
}

extern "C" int mnpb_bemret_sigma_mirror_f64(void *stream, int64_t n, int64_t nsym, int64_t batch,
                                            const double *H1, const double *H2,
                                            const double *Dinv, int64_t ld, int64_t stride,
                                            const double *eps, const double *kvac,
                                            const double *nvec, int32_t ix, int32_t iy,
                                            int32_t iz, double *S, int64_t sS, int32_t *pivS,
                                            int32_t *info) {
    clear_error();
    MNPB_REQUIRE(n > 0 && n < 65536 && batch > 0 && batch < 65536 && ld >= n &&
                     stride >= ld * n && sS >= ld * n,
                 "bemret_sigma_mirror: bad sizes");
    MNPB_REQUIRE(nsym >= 1 && nsym <= MAX_NK && ix >= 0 && ix < nsym && iy >= 0 && iy < nsym &&
                     iz >= 0 && iz < nsym,
                 "bemret_sigma_mirror: symmetry indices outside [0, %lld)", (long long)nsym);
    MNPB_REQUIRE(H1 && H2 && Dinv && eps && kvac && nvec && S && pivS && info,
                 "bemret_sigma_mirror: null pointer");
    cudaStream_t s = as_stream(stream);
    const int N = (int)n, B = (int)batch;
    if (cudaMemsetAsync(info, 0, sizeof(int32_t) * batch, s) != cudaSuccess) {
        set_error("bemret_sigma_mirror: memset failed");
        return MNPB_ECUDA;
    }
    dim3 grid(ceil_div(n, 128), N, B);
    mirror_sigma_kernel<<<grid, 128, 0, s>>>(N, (int)nsym, (const cd *)H1, (const cd *)H2,
                                             (const cd *)Dinv, ld, stride, ix, iy, iz, eps, kvac,
                                             nvec, (cd *)S, sS);
    MNPB_LAUNCH_CHECK("mirror_sigma_kernel");
    return getrf(s, N, B, (cd *)S, ld, sS, pivS, n, info);
}

extern "C" int64_t mnpb_bemret_solve_mirror_workspace(int64_t n, int64_t batch, int64_t nrhs) {
    return batch * n * (4 * nrhs + 4 * nrhs + 3 * nrhs + 3 * nrhs + nrhs) * 16;
}

extern "C" int mnpb_bemret_solve_mirror_f64(
    void *stream, int64_t n, int64_t nsym, int64_t batch, int64_t nrhs, const double *G1,
    const double *G2, const double *H1, const double *Dinv, int64_t ld, int64_t stride,
    const int32_t *piv, const double *S, int64_t sS, const int32_t *pivS, int32_t ix,
    int32_t iy, int32_t iz, const double *eps, const double *kvac, const double *nvec,
    const double *x_in, double *x_out, void *work, int64_t work_bytes) {
    clear_error();
    const int64_t K = nrhs;
    MNPB_REQUIRE(n > 0 && n < 65536 && batch > 0 && batch < 65536 && K > 0 && K <= 64 &&
                     ld >= n && stride >= ld * n && sS >= ld * n,
                 "bemret_solve_mirror: bad sizes");
    MNPB_REQUIRE(nsym >= 1 && nsym <= MAX_NK && ix >= 0 && ix < nsym && iy >= 0 && iy < nsym &&
                     iz >= 0 && iz < nsym,
                 "bemret_solve_mirror: symmetry indices outside [0, %lld)", (long long)nsym);
    MNPB_REQUIRE(G1 && G2 && H1 && Dinv && piv && S && pivS && eps && kvac && nvec && x_in &&
                     x_out && work,
                 "bemret_solve_mirror: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_bemret_solve_mirror_workspace(n, batch, K),
                 "bemret_solve_mirror: workspace too small");
    cudaStream_t s = as_stream(stream);
    const int N = (int)n, B = (int)batch, k = (int)K;
    const int64_t entries = batch * nsym;
    const int64_t me = nsym * stride;                 // stride between wavelengths
    auto M = [&](const double *base, int idx) { return (const cd *)base + idx * stride; };
    const int32_t *piv1 = piv, *piv2 = piv + entries * n;
    cd *T = (cd *)work;
    cd *U = T + batch * n * 4 * K;
    cd *AP = U + batch * n * 4 * K;
    cd *V = AP + batch * n * 3 * K;
    cd *R = V + batch * n * 3 * K;
    const int64_t sT = n * 4 * K, sAP = n * 3 * K, sR = n * K, sx = n * 8 * K;
    const cd *xin = (const cd *)x_in;
    cd *xout = (cd *)x_out;
    const NvecView nv{nvec, 0};
    const int idx[3] = {ix, iy, iz};
    const cd one = cmk(1, 0), zero = cmk(0, 0);
    dim3 g(ceil_div(n, 128), B);
    // T = [a (3K) | eps1 phi (K)];  U = Sigma1 T, component d with Sigma1_{idx_d},
    // eps1 phi with Sigma1_z
    solve_prep_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, T, sT, eps, kvac);
    MNPB_LAUNCH_CHECK("solve_prep_kernel");
    for (int d = 0; d < 4; ++d) {
        const int id = d < 3 ? idx[d] : iz;
        MNPB_TRY(zgemm(s, N, k, N, B, one, M(H1, id), ld, me, T + (int64_t)d * K * n, n, sT,
                       zero, U + (int64_t)d * K * n, n, sT));
    }
    solve_alpha_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, U, sT, AP, sAP, R, sR, eps, kvac, nv);
    MNPB_LAUNCH_CHECK("solve_alpha_kernel");
    for (int d = 0; d < 3; ++d)
        MNPB_TRY(zgemm(s, N, k, N, B, one, M(Dinv, idx[d]), ld, me, AP + (int64_t)d * K * n, n,
                       sAP, zero, V + (int64_t)d * K * n, n, sAP));
    solve_rhs_kernel<<<g, 128, 0, s>>>(N, k, V, sAP, R, sR, eps, kvac, nv);
    MNPB_LAUNCH_CHECK("solve_rhs_kernel");
    MNPB_TRY(getrs(s, N, k, B, (const cd *)S, ld, sS, pivS, n, R, n, sR));
    solve_h2pre_kernel<<<g, 128, 0, s>>>(N, k, AP, sAP, R, sR, eps, kvac, nv);
    MNPB_LAUNCH_CHECK("solve_h2pre_kernel");
    for (int d = 0; d < 3; ++d)
        MNPB_TRY(zgemm(s, N, k, N, B, one, M(Dinv, idx[d]), ld, me, AP + (int64_t)d * K * n, n,
                       sAP, zero, V + (int64_t)d * K * n, n, sAP));
    solve_out_kernel<<<g, 128, 0, s>>>(N, k, xin, sx, R, sR, V, sAP, xout, sx);
    MNPB_LAUNCH_CHECK("solve_out_kernel");
    // sig1 = G1_z^-1 (sig2 + phi), h1_d = G1_{idx_d}^-1 (h2_d + a_d); the same with G2
    for (int side = 0; side < 2; ++side) {
        const double *G = side == 0 ? G1 : G2;
        const int32_t *pv = side == 0 ? piv1 : piv2;
        cd *x0 = xout + (int64_t)side * 4 * K * n;
        for (int d = 0; d < 4; ++d) {
            const int id = d == 0 ? iz : idx[d - 1];
            MNPB_TRY(getrs(s, N, k, B, M(G, id), ld, me, pv + (int64_t)id * n, nsym * n,
                           x0 + (int64_t)d * K * n, n, sx));
        }
    }
    return MNPB_OK;
}
