// Far fields of the surface charges/currents and the quasistatic BEM matrix.
#include "common.cuh"

namespace mnpb {
namespace {

constexpr int FF_THREADS = 256;

__device__ __forceinline__ cd block_sum(cd v, cd *sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    cd r = cmk(0, 0);
    if (threadIdx.x == 0)
        for (int w = 0; w < FF_THREADS / 32; ++w) r = cadd(r, sh[w]);
    return r;
}

// One CTA per (direction, polarisation, wavelength).
// e = i k0 sum ph h - i k dir sum ph sig,  h = i k dir x sum ph h,
// ph_j = exp(-i k dir.pos_j) area_j over faces whose inside (sig1, h1) or
// outside (sig2, h2) medium is the embedding medium
// (mnpbem/spectrum/spectrum_ret.py:331-376).
__global__ void __launch_bounds__(FF_THREADS) farfield_kernel(
    int n, int npol, int ndir, const double *__restrict__ pos, const double *__restrict__ area,
    const int8_t *__restrict__ side_in, const int8_t *__restrict__ side_out,
    const double *__restrict__ dirs, const double *__restrict__ kmed,
    const double *__restrict__ k0v, const cd *__restrict__ sol, cd *__restrict__ e_out,
    cd *__restrict__ h_out) {
    __shared__ cd sh[FF_THREADS / 32];
    const int dir = blockIdx.x, pol = blockIdx.y;
    const int64_t b = blockIdx.z;
    const cd k = cmk(kmed[2 * b], kmed[2 * b + 1]);
    const double k0 = k0v[b];
    const double dx = dirs[3 * dir], dy = dirs[3 * dir + 1], dz = dirs[3 * dir + 2];
    const int K = npol;
    const cd *x = sol + b * (int64_t)n * 8 * K;
    cd sh_[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    cd ss = cmk(0, 0);
    for (int j = threadIdx.x; j < n; j += FF_THREADS) {
        const double sp = dx * pos[3 * j] + dy * pos[3 * j + 1] + dz * pos[3 * j + 2];
        // exp(-i k s) = exp(k.y s) (cos(k.x s) - i sin(k.x s))
        double sn, cs;
        sincos(k.x * sp, &sn, &cs);
        const double m = exp(k.y * sp) * area[j];
        const cd ph = cmk(m * cs, -m * sn);
        if (side_in[j]) {
            ss = cfma(ph, x[(int64_t)pol * n + j], ss);
            for (int c = 0; c < 3; ++c) sh_[c] = cfma(ph, x[(int64_t)(K + c * K + pol) * n + j], sh_[c]);
        }
        if (side_out[j]) {
            ss = cfma(ph, x[(int64_t)(4 * K + pol) * n + j], ss);
            for (int c = 0; c < 3; ++c)
                sh_[c] = cfma(ph, x[(int64_t)(5 * K + c * K + pol) * n + j], sh_[c]);
        }
    }
    ss = block_sum(ss, sh);
    for (int c = 0; c < 3; ++c) sh_[c] = block_sum(sh_[c], sh);
    if (threadIdx.x == 0) {
        const cd ik0 = cmk(0.0, k0);
        const cd ik = cmk(-k.y, k.x);
        const double d[3] = {dx, dy, dz};
        cd *e = e_out + ((b * npol + pol) * (int64_t)ndir + dir) * 3;
        cd *h = h_out + ((b * npol + pol) * (int64_t)ndir + dir) * 3;
        for (int c = 0; c < 3; ++c) e[c] = csub(cmul(ik0, sh_[c]), cmul(ik, cscale(ss, d[c])));
        // dir x P
        cd cr[3];
        cr[0] = csub(cscale(sh_[2], dy), cscale(sh_[1], dz));
        cr[1] = csub(cscale(sh_[0], dz), cscale(sh_[2], dx));
        cr[2] = csub(cscale(sh_[1], dx), cscale(sh_[0], dy));
        for (int c = 0; c < 3; ++c) h[c] = cmul(ik, cr[c]);
    }
}

// M_b = -(diag(lambda_b) + F), lambda = 2 pi (eps1 + eps2) / (eps1 - eps2)
__global__ void stat_matrix_kernel(int n, const double *__restrict__ F, int64_t ldf,
                                   const double *__restrict__ eps12, cd *__restrict__ M,
                                   int64_t ld, int64_t st) {
    const int64_t b = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    cd v = cmk(-F[(int64_t)j * ldf + i], 0.0);
    if (i == j) {
        const double *e = eps12 + (b * n + i) * 4;
        const cd e1 = cmk(e[0], e[1]), e2 = cmk(e[2], e[3]);
        const cd lam = cscale(cdiv(cadd(e1, e2), csub(e1, e2)), 6.283185307179586);
        v = csub(v, lam);
    }
    M[b * st + (int64_t)j * ld + i] = v;
}


// Plane-wave potentials a = e^{i k r.dir}/(i k0) pol and a' = i k (n.dir) a on
// faces whose inside (a1, a1') / outside (a2, a2') medium is the embedding
// medium (mnpbem/simulation/planewave_ret.py:257-361).  pots layout
// [b][16][K][n]: phi1, phi1', a1 (3), a1' (3), phi2, phi2', a2 (3), a2' (3).
__global__ void planewave_pot_kernel(int n, int K, const double *__restrict__ pos,
                                     const double *__restrict__ nvec,
                                     const int8_t *__restrict__ side_in,
                                     const int8_t *__restrict__ side_out,
                                     const double *__restrict__ pol,
                                     const double *__restrict__ dirs,
                                     const double *__restrict__ kmed,
                                     const double *__restrict__ k0v, cd *__restrict__ pots) {
    const int64_t b = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cd k = cmk(kmed[2 * b], kmed[2 * b + 1]);
    const double k0 = k0v[b];
    cd *q = pots + b * (int64_t)n * 16 * K;
    auto Q = [&](int comp, int r) -> cd & { return q[(int64_t)(comp * K + r) * n + i]; };
    for (int r = 0; r < K; ++r) {
        const double *d = dirs + 3 * r, *pl = pol + 3 * r;
        const double s = pos[3 * i] * d[0] + pos[3 * i + 1] * d[1] + pos[3 * i + 2] * d[2];
        const double nd = nvec[3 * i] * d[0] + nvec[3 * i + 1] * d[1] + nvec[3 * i + 2] * d[2];
        // e^{i k s} / (i k0)
        const cd e = cexpi(k, s);
        const cd ph = cmk(e.y / k0, -e.x / k0);
        const cd ikn = cmk(-k.y * nd, k.x * nd);
        const cd php = cmul(ikn, ph);
        Q(0, r) = Q(1, r) = Q(8, r) = Q(9, r) = cmk(0, 0);
        for (int c = 0; c < 3; ++c) {
            const bool in = side_in[i] != 0, out = side_out[i] != 0;
            Q(2 + c, r) = in ? cscale(ph, pl[c]) : cmk(0, 0);
            Q(5 + c, r) = in ? cscale(php, pl[c]) : cmk(0, 0);
            Q(10 + c, r) = out ? cscale(ph, pl[c]) : cmk(0, 0);
            Q(13 + c, r) = out ? cscale(php, pl[c]) : cmk(0, 0);
        }
    }
}

}  // namespace
}  // namespace mnpb

using namespace mnpb;

extern "C" int mnpb_farfield(void *stream, int64_t n, int64_t batch, int64_t npol, int64_t ndir,
                             const double *pos, const double *area, const int8_t *side_in,
                             const int8_t *side_out, const double *dirs, const double *kmed,
                             const double *k0, const double *sol, double *e_out,
                             double *h_out) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && npol > 0 && ndir > 0 && batch < 65536 && npol < 65536,
                 "farfield: bad sizes");
    MNPB_REQUIRE(pos && area && side_in && side_out && dirs && kmed && k0 && sol && e_out &&
                     h_out,
                 "farfield: null pointer");
    dim3 grid((unsigned)ndir, (unsigned)npol, (unsigned)batch);
    ProfScope ps(as_stream(stream), PC_FARFIELD, 0.0);
    farfield_kernel<<<grid, FF_THREADS, 0, as_stream(stream)>>>(
        (int)n, (int)npol, (int)ndir, pos, area, side_in, side_out, dirs, kmed, k0,
        (const cd *)sol, (cd *)e_out, (cd *)h_out);
    MNPB_LAUNCH_CHECK("farfield_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_stat_matrix(void *stream, int64_t n, int64_t batch, const double *F,
                                int64_t ldf, const double *eps12, double *M, int64_t ld,
                                int64_t stride) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && n < 65536 && batch < 65536 && ld >= n && ldf >= n,
                 "stat_matrix: bad sizes");
    MNPB_REQUIRE(F && eps12 && M, "stat_matrix: null pointer");
    dim3 grid(ceil_div(n, 128), (unsigned)n, (unsigned)batch);
    stat_matrix_kernel<<<grid, 128, 0, as_stream(stream)>>>((int)n, F, ldf, eps12, (cd *)M, ld,
                                                           stride);
    MNPB_LAUNCH_CHECK("stat_matrix_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_planewave_potential(void *stream, int64_t n, int64_t batch, int64_t npol,
                                        const double *pos, const double *nvec,
                                        const int8_t *side_in, const int8_t *side_out,
                                        const double *pol, const double *dirs,
                                        const double *kmed, const double *k0, double *pots) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && npol > 0 && batch < 65536, "planewave_potential: bad sizes");
    MNPB_REQUIRE(pos && nvec && side_in && side_out && pol && dirs && kmed && k0 && pots,
                 "planewave_potential: null pointer");
    dim3 g(ceil_div(n, 128), (unsigned)batch);
    planewave_pot_kernel<<<g, 128, 0, as_stream(stream)>>>((int)n, (int)npol, pos, nvec, side_in,
                                                           side_out, pol, dirs, kmed, k0,
                                                           (cd *)pots);
    MNPB_LAUNCH_CHECK("planewave_pot_kernel");
    return MNPB_OK;
}
