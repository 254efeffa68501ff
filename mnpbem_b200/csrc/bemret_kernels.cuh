// Element-wise kernels of the BEMRet solve (shared by the FP64 and the
// mixed-precision solvers).  All vectors are interleaved complex double,
// component-major blocks of n (see mnpb_bemret_solve_f64 in the C ABI).
#pragma once
#include "common.cuh"

namespace mnpb {
namespace bemk {

struct EpsK {
    cd e1, e2;
    double k;
};

static __device__ __forceinline__ EpsK load_epsk(const double *eps, const double *kvac, int64_t b) {
    EpsK r;
    r.e1 = cmk(eps[4 * b], eps[4 * b + 1]);
    r.e2 = cmk(eps[4 * b + 2], eps[4 * b + 3]);
    r.k = kvac[b];
    return r;
}

// D = S1 - S2 ; S2 <- eps1 S1 - eps2 S2
static __global__ void form_delta_kernel(int n, const cd *S1, cd *S2, cd *D, int64_t ld, int64_t st,
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
static __global__ void form_sigma_kernel(int n, cd *S, const cd *W, int64_t ldw, int64_t sw, cd *D,
                                  int64_t ld, int64_t st, const double *eps, const double *kvac,
                                  NvecView nvv) {
    const int64_t b = blockIdx.z;
    const double *nvec = nvv.at(b);
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
static __global__ void solve_prep_kernel(int n, int K, const cd *xin, int64_t sx, cd *T, int64_t sT,
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
static __global__ void solve_alpha_kernel(int n, int K, const cd *xin, int64_t sx, const cd *U,
                                   int64_t sU, cd *AP, int64_t sAP, cd *R, int64_t sR,
                                   const double *eps, const double *kvac, NvecView nvv) {
    const int64_t b = blockIdx.y;
    const double *nvec = nvv.at(b);
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
static __global__ void solve_rhs_kernel(int n, int K, const cd *V, int64_t sV, cd *R, int64_t sR,
                                 const double *eps, const double *kvac, NvecView nvv) {
    const int64_t b = blockIdx.y;
    const double *nvec = nvv.at(b);
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
static __global__ void solve_h2pre_kernel(int n, int K, cd *AP, int64_t sAP, const cd *R, int64_t sR,
                                   const double *eps, const double *kvac, NvecView nvv) {
    const int64_t b = blockIdx.y;
    const double *nvec = nvv.at(b);
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
static __global__ void solve_out_kernel(int n, int K, const cd *xin, int64_t sx, const cd *R,
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
static __global__ void excitation_kernel(int n, int K, const cd *pots, cd *xin, const double *eps,
                                  const double *kvac, NvecView nvv) {
    const int64_t b = blockIdx.y;
    const double *nvec = nvv.at(b);
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


}  // namespace bemk
}  // namespace mnpb
