// Mixed-precision retarded BEM solver: the Sigma/Delta algebra and all four
// LU factorisations run in FP32 storage with TF32 tensor-core GEMMs; the
// solution is then refined in FP64 against the exact FP64 operator (the
// packed 8N system of mnpbem/bem/bem_ret_iter.py:1362-1501, Eqs. 10, 11, 14,
// 17 of Garcia de Abajo & Howie), with the mixed BEMRet solve as the
// correction operator -- the structure the reference itself uses for its
// preconditioned iterative solver (bem_ret_iter.py:1503-1634).
#include "common.cuh"

#include <mutex>
#include <vector>
#include "bemret_kernels.cuh"
#include "dense_f32.cuh"

#include <cmath>
#include <vector>

namespace mnpb {
namespace mixed {

using tc::CMatF;
using namespace mnpb::bemk;

namespace {

struct cfl {
    float x, y;
};

// D = S1 - S2 ; S2 <- eps1 S1 - eps2 S2   (planar FP32)
__global__ void form_delta_p(int n, const float *S1, float *S2, float *D, int64_t ld,
                             int64_t plane, int64_t st, const double *eps, const double *kvac) {
    const int64_t b = blockIdx.z;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const int64_t o = b * st + (int64_t)j * ld + i;
    const cd s1 = cmk(S1[o], S1[o + plane]), s2 = cmk(S2[o], S2[o + plane]);
    const cd d = csub(s1, s2);
    const cd s0 = csub(cmul(ek.e1, s1), cmul(ek.e2, s2));
    D[o] = (float)d.x;
    D[o + plane] = (float)d.y;
    S2[o] = (float)s0.x;
    S2[o + plane] = (float)s0.y;
}

// S <- S + k^2 (eps1-eps2)^2 (W o n n^T) ; D <- W   (planar FP32)
__global__ void form_sigma_p(int n, float *S, const float *W, float *D, int64_t ld, int64_t plane,
                             int64_t st, const double *eps, const double *kvac,
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
    const cd w = cmk(W[o], W[o + plane]);
    const cd v = cadd(cmk(S[o], S[o + plane]), cmul(c, cscale(w, nn)));
    S[o] = (float)v.x;
    S[o + plane] = (float)v.y;
    D[o] = (float)w.x;
    D[o + plane] = (float)w.y;
}

// c128 block (n x m, leading dimension n) <-> planar FP32 block
__global__ void to_f32p(int n, int m, const cd *X, int64_t sx, float *Y, int64_t sy) {
    const int64_t b = blockIdx.y;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * m) return;
    const cd v = X[b * sx + e];
    float *y = Y + b * sy;
    y[e] = (float)v.x;
    y[e + (int64_t)n * m] = (float)v.y;
}
__global__ void from_f32p(int n, int m, const float *Y, int64_t sy, cd *X, int64_t sx) {
    const int64_t b = blockIdx.y;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * m) return;
    const float *y = Y + b * sy;
    X[b * sx + e] = cmk((double)y[e], (double)y[e + (int64_t)n * m]);
}

// FP64 matrix times a few vectors: Y = A X, A n x n (c128, column-major),
// X n x m (m <= NC <= 16).  A CTA covers 64 rows with 4 K-lanes (warp w reads
// 32 consecutive rows of every 4th column, 512 B per load), so each matrix
// element is read once and many loads are in flight; the lanes' partial sums
// are reduced in shared memory.
constexpr int ZS_KT = 32, ZS_ROWS = 64, ZS_KL = 4;
template <int NC>
__global__ void __launch_bounds__(256) zskinny_kernel(int n, int m, const cd *__restrict__ A,
                                                      int64_t lda, int64_t sA,
                                                      const cd *__restrict__ X, int64_t sX,
                                                      cd *__restrict__ Y, int64_t sY) {
    __shared__ cd Xs[ZS_KT][NC];
    __shared__ cd part[ZS_KL][ZS_ROWS][NC];
    const int64_t b = blockIdx.y;
    A += b * sA;
    X += b * sX;
    Y += b * sY;
    const int rl = threadIdx.x % ZS_ROWS, kl = threadIdx.x / ZS_ROWS;
    const int row = blockIdx.x * ZS_ROWS + rl;
    cd acc[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) acc[j] = cmk(0, 0);
    for (int k0 = 0; k0 < n; k0 += ZS_KT) {
        __syncthreads();
        for (int e = threadIdx.x; e < ZS_KT * NC; e += blockDim.x) {
            const int kk = e % ZS_KT, j = e / ZS_KT;
            Xs[kk][j] = (k0 + kk < n && j < m) ? X[(int64_t)j * n + k0 + kk] : cmk(0, 0);
        }
        __syncthreads();
        if (row < n) {
            const int kend = min(ZS_KT, n - k0);
#pragma unroll 4
            for (int kk = kl; kk < kend; kk += ZS_KL) {
                const cd a = __ldg(A + (int64_t)(k0 + kk) * lda + row);
#pragma unroll
                for (int j = 0; j < NC; ++j) acc[j] = cfma(a, Xs[kk][j], acc[j]);
            }
        }
    }
#pragma unroll
    for (int j = 0; j < NC; ++j) part[kl][rl][j] = acc[j];
    __syncthreads();
    for (int e = threadIdx.x; e < ZS_ROWS * NC; e += blockDim.x) {
        const int r = e % ZS_ROWS, j = e / ZS_ROWS;
        const int gr = blockIdx.x * ZS_ROWS + r;
        if (gr < n && j < m) {
            cd v = part[0][r][j];
#pragma unroll
            for (int q = 1; q < ZS_KL; ++q) v = cadd(v, part[q][r][j]);
            Y[(int64_t)j * n + gr] = v;
        }
    }
}

// r = b - A x for the packed operator.  P1 = G1 [sig1|h1], P2 = G2 [sig2|h2],
// Q1 = H1 [sig1|h1], Q2 = H2 [sig2|h2] (each n x 4K, columns sig then h x,y,z).
// b and r use the excitation layout [phi | a (3) | De | alpha (3)].
__global__ void residual_kernel(int n, int K, const cd *P1, const cd *P2, const cd *Q1,
                                const cd *Q2, int64_t sP, const cd *bvec, cd *r, int64_t sx,
                                const double *eps, const double *kvac, NvecView nvv) {
    const int64_t b = blockIdx.y;
    const double *nvec = nvv.at(b);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const EpsK ek = load_epsk(eps, kvac, b);
    const cd ik = cmk(0.0, ek.k);
    const cd *p1 = P1 + b * sP, *p2 = P2 + b * sP, *q1 = Q1 + b * sP, *q2 = Q2 + b * sP;
    const cd *bb = bvec + b * sx;
    cd *rr = r + b * sx;
    const double nv[3] = {nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]};
    auto at = [&](const cd *p, int col) { return p[(int64_t)col * n + i]; };
    for (int q = 0; q < K; ++q) {
        const cd gs1 = at(p1, q), gs2 = at(p2, q), hs1 = at(q1, q), hs2 = at(q2, q);
        const cd egs = csub(cmul(ek.e1, gs1), cmul(ek.e2, gs2));
        cd negh = cmk(0, 0);
        const int64_t o_phi = (int64_t)q * n + i;
        rr[o_phi] = csub(bb[o_phi], csub(gs1, gs2));
        for (int c = 0; c < 3; ++c) {
            const int col = K + c * K + q;
            const cd gh1 = at(p1, col), gh2 = at(p2, col), hh1 = at(q1, col), hh2 = at(q2, col);
            const int64_t o_a = (int64_t)(K + c * K + q) * n + i;
            rr[o_a] = csub(bb[o_a], csub(gh1, gh2));
            const cd alpha = csub(csub(hh1, hh2), cmul(ik, cscale(egs, nv[c])));
            const int64_t o_al = (int64_t)(5 * K + c * K + q) * n + i;
            rr[o_al] = csub(bb[o_al], alpha);
            negh = cadd(negh, cscale(csub(cmul(ek.e1, gh1), cmul(ek.e2, gh2)), nv[c]));
        }
        const cd de = csub(csub(cmul(ek.e1, hs1), cmul(ek.e2, hs2)), cmul(ik, negh));
        const int64_t o_de = (int64_t)(4 * K + q) * n + i;
        rr[o_de] = csub(bb[o_de], de);
    }
}

// per batch entry: sum |r|^2 and sum |b|^2 over len entries
__global__ void norms_kernel(int64_t len, const cd *r, const cd *bvec, int64_t sx, double *out) {
    __shared__ double s1[32], s2[32];
    const int64_t b = blockIdx.x;
    double a1 = 0.0, a2 = 0.0;
    for (int64_t e = threadIdx.x; e < len; e += blockDim.x) {
        const cd x = r[b * sx + e], y = bvec[b * sx + e];
        a1 += x.x * x.x + x.y * x.y;
        a2 += y.x * y.x + y.y * y.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s1[threadIdx.x >> 5] = a1;
        s2[threadIdx.x >> 5] = a2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t1 = 0.0, t2 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t1 += s1[w];
            t2 += s2[w];
        }
        out[2 * b] = t1;
        out[2 * b + 1] = t2;
    }
}

__global__ void axpy_kernel(int64_t len, const cd *d, cd *x) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < len) x[e] = cadd(x[e], d[e]);
}

}  // namespace

// Device buffers of the mixed factorisation (planar FP32, ld = leading dim,
// plane = ld*n, stride = 2*plane).
struct Factors {
    float *G1, *G2, *S1, *S, *D;
    int64_t ld, plane, stride;
    const int32_t *pivG1, *pivG2, *pivS;            // n per batch entry
    const float *iG1L, *iG1U, *iG2L, *iG2U, *iSL, *iSU;   // diagonal-block inverses
    int64_t n, dinv_per;                            // dinv_per: floats per entry
    int *trsv_state;      // flags + ticket of the one-launch triangular solves
    // the same factors for batch entries b0, b0 + 1, ...
    Factors at(int b0) const {
        Factors f = *this;
        const int64_t o = (int64_t)b0 * stride, op = (int64_t)b0 * n, oi = (int64_t)b0 * dinv_per;
        f.G1 += o;
        f.G2 += o;
        f.S1 += o;
        f.S += o;
        f.D += o;
        f.pivG1 += op;
        f.pivG2 += op;
        f.pivS += op;
        f.iG1L += oi;
        f.iG1U += oi;
        f.iG2L += oi;
        f.iG2U += oi;
        f.iSL += oi;
        f.iSU += oi;
        return f;
    }
};

// Offsets (floats) into the diagonal-block-inverse buffer: G1/G2 unit-lower
// blocks (2 x batch entries), G1/G2 upper, then Sigma lower, Sigma upper.
struct DinvOff {
    int64_t S;   // floats per matrix
    int64_t gL(int which, int64_t B) const { return which * B * S; }
    int64_t gU(int which, int64_t B) const { return 2 * B * S + which * B * S; }
    int64_t sL(int64_t B) const { return 4 * B * S; }
    int64_t sU(int64_t B) const { return 5 * B * S; }
};

static int convert_in(cudaStream_t s, int n, int m, int batch, const cd *X, int64_t sx, float *Y) {
    dim3 g(ceil_div((int64_t)n * m, 256), batch);
    ProfScope ps(s, PC_REFINE_EW, 0.0);
    to_f32p<<<g, 256, 0, s>>>(n, m, X, sx, Y, 2 * (int64_t)n * m);
    MNPB_LAUNCH_CHECK("to_f32p");
    return MNPB_OK;
}
static int convert_out(cudaStream_t s, int n, int m, int batch, const float *Y, cd *X, int64_t sx) {
    dim3 g(ceil_div((int64_t)n * m, 256), batch);
    ProfScope ps(s, PC_REFINE_EW, 0.0);
    from_f32p<<<g, 256, 0, s>>>(n, m, Y, 2 * (int64_t)n * m, X, sx);
    MNPB_LAUNCH_CHECK("from_f32p");
    return MNPB_OK;
}

// y (c128 n x m) = A_f32 x (c128 n x m), through a planar FP32 scratch.
static int mgemm(f32::Ctx &c, int n, int m, const float *A, const Factors &F, const cd *x,
                 int64_t sx, cd *y, int64_t sy, float *t1, float *t2) {
    MNPB_TRY(convert_in(c.s, n, m, c.batch, x, sx, t1));
    const int64_t pl = (int64_t)n * m;
    MNPB_TRY(f32::gemm(c, n, m, n, 1.f, CMatF{(float *)A, F.ld, F.plane, F.stride},
                       CMatF{t1, n, pl, 2 * pl}, 0.f, CMatF{t2, n, pl, 2 * pl}));
    return convert_out(c.s, n, m, c.batch, t2, y, sy);
}

// x (c128 n x m, in place) <- LU^-1 x
static int mgetrs(f32::Ctx &c, int n, int m, const float *LU, const Factors &F,
                  const int32_t *piv, const float *invL, const float *invU, cd *x, int64_t sx,
                  float *t1) {
    MNPB_TRY(convert_in(c.s, n, m, c.batch, x, sx, t1));
    const int64_t pl = (int64_t)n * m;
    MNPB_TRY(f32::getrs_few(c, n, m, CMatF{(float *)LU, F.ld, F.plane, F.stride}, piv,
                            (int64_t)n, invL, invU, CMatF{t1, n, pl, 2 * pl}, F.trsv_state));
    return convert_out(c.s, n, m, c.batch, t1, x, sx);
}

// Mixed BEMRet solve x_out = M^-1 x_in (same steps as mnpb_bemret_solve_f64).
// Scratch: per batch entry 15 K n complex double + 2 x 8 K n planar float.
static int msolve(f32::Ctx &c, int n, int K, const Factors &F, const double *eps,
                  const double *kvac, NvecView nvec, const cd *xin, cd *xout, cd *scr,
                  float *fscr) {
    cudaStream_t s = c.s;
    const int B = c.batch;
    const int64_t nn = n;
    cd *T = scr;
    cd *U = T + (int64_t)B * nn * 4 * K;
    cd *AP = U + (int64_t)B * nn * 4 * K;
    cd *V = AP + (int64_t)B * nn * 3 * K;
    cd *R = V + (int64_t)B * nn * 3 * K;
    float *t1 = fscr, *t2 = fscr + (int64_t)B * nn * 16 * K;
    const int64_t sT = nn * 4 * K, sAP = nn * 3 * K, sR = nn * K, sx = nn * 8 * K;
    dim3 g(ceil_div(n, 128), B);
    solve_prep_kernel<<<g, 128, 0, s>>>(n, K, xin, sx, T, sT, eps, kvac);
    MNPB_LAUNCH_CHECK("solve_prep_kernel");
    MNPB_TRY(mgemm(c, n, 4 * K, F.S1, F, T, sT, U, sT, t1, t2));
    solve_alpha_kernel<<<g, 128, 0, s>>>(n, K, xin, sx, U, sT, AP, sAP, R, sR, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("solve_alpha_kernel");
    MNPB_TRY(mgemm(c, n, 3 * K, F.D, F, AP, sAP, V, sAP, t1, t2));
    solve_rhs_kernel<<<g, 128, 0, s>>>(n, K, V, sAP, R, sR, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("solve_rhs_kernel");
    MNPB_TRY(mgetrs(c, n, K, F.S, F, F.pivS, F.iSL, F.iSU, R, sR, t1));
    solve_h2pre_kernel<<<g, 128, 0, s>>>(n, K, AP, sAP, R, sR, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("solve_h2pre_kernel");
    MNPB_TRY(mgemm(c, n, 3 * K, F.D, F, AP, sAP, V, sAP, t1, t2));
    solve_out_kernel<<<g, 128, 0, s>>>(n, K, xin, sx, R, sR, V, sAP, xout, sx);
    MNPB_LAUNCH_CHECK("solve_out_kernel");
    MNPB_TRY(mgetrs(c, n, 4 * K, F.G1, F, F.pivG1, F.iG1L, F.iG1U, xout, sx, t1));
    return mgetrs(c, n, 4 * K, F.G2, F, F.pivG2, F.iG2L, F.iG2U, xout + 4 * K * nn, sx, t1);
}

}  // namespace mixed
}  // namespace mnpb

using namespace mnpb;
using namespace mnpb::mixed;

static int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

extern "C" int64_t mnpb_bemret_workspace_mixed(int64_t n, int64_t batch) {
    const int64_t ld = (n + 3) / 4 * 4;
    // tensor-core packing buffer + W (planar, for Delta^-1) + pivots of Delta
    return align_up(tc::cgemm_tf32_workspace((int)n, (int)n, 2 * (int)batch), 256) +
           align_up(batch * 2 * ld * n * 4, 256) + align_up(batch * n * 4, 256);
}

extern "C" int64_t mnpb_bemret_dinv_floats(int64_t n, int64_t batch) {
    return 6 * f32::diag_inv_floats((int)n, (int)batch);
}

static int init_mixed_body(cudaStream_t s, int64_t n, int64_t batch, float *G1, float *G2,
                           float *H1, float *H2, float *D, int64_t ld, const double *eps,
                           const double *kvac, NvecView nvec, int32_t *piv, int32_t *info,
                           float *dinv, void *work, int64_t work_bytes) {
    const int N = (int)n, B = (int)batch;
    const int64_t plane = ld * n, stride = 2 * plane;
    const int64_t tcw = align_up(tc::cgemm_tf32_workspace(N, N, 2 * B), 256);
    float *W = (float *)((char *)work + tcw);
    int32_t *pivD = (int32_t *)((char *)W + align_up(batch * 2 * ld * n * 4, 256));
    f32::Ctx c(s, B, (float *)work, tcw);
    CMatF g1{G1, ld, plane, stride}, g2{G2, ld, plane, stride}, h1{H1, ld, plane, stride},
        h2{H2, ld, plane, stride}, d{D, ld, plane, stride}, w{W, ld, plane, stride};
    // pivots [3][batch][n]: G1, G2, Sigma; info [2][batch]
    const int64_t ps = n;
    int32_t *piv1 = piv, *piv2 = piv + batch * n, *pivS = piv + 2 * batch * n;
    if (cudaMemsetAsync(info, 0, sizeof(int32_t) * 2 * batch, s) != cudaSuccess) {
        set_error("bemret_init_mixed: memset failed");
        return MNPB_ECUDA;
    }
    // G1/G2 (and H1/H2) stored back to back: one launch sequence over 2 x batch matrices
    if (G2 == G1 + batch * stride && H2 == H1 + batch * stride) {
        f32::Ctx c2(s, 2 * B, (float *)work, tcw);
        MNPB_TRY(f32::getrf(c2, N, g1, piv1, ps, info));
        MNPB_TRY(f32::right_solve(c2, N, N, g1, piv1, ps, h1));
    } else {
        MNPB_TRY(f32::getrf(c, N, g1, piv1, ps, info));
        MNPB_TRY(f32::getrf(c, N, g2, piv2, ps, info + batch));
        MNPB_TRY(f32::right_solve(c, N, N, g1, piv1, ps, h1));
        MNPB_TRY(f32::right_solve(c, N, N, g2, piv2, ps, h2));
    }
    dim3 grid(ceil_div(n, 128), N, B);
    form_delta_p<<<grid, 128, 0, s>>>(N, H1, H2, D, ld, plane, stride, eps, kvac);
    MNPB_LAUNCH_CHECK("form_delta_p");
    MNPB_TRY(f32::getrf(c, N, d, pivD, n, info));
    MNPB_TRY(f32::lu_inverse(c, N, d, pivD, n, w));
    form_sigma_p<<<grid, 128, 0, s>>>(N, H2, W, D, ld, plane, stride, eps, kvac, nvec);
    MNPB_LAUNCH_CHECK("form_sigma_p");
    MNPB_TRY(f32::getrf(c, N, h2, pivS, ps, info));
    // inverses of the 32 x 32 diagonal blocks for the few-RHS solves
    const DinvOff dv{f32::diag_inv_floats(N, 1)};
    MNPB_TRY(f32::diag_inv(c, N, g1, dinv + dv.gL(0, B), dinv + dv.gU(0, B)));
    MNPB_TRY(f32::diag_inv(c, N, g2, dinv + dv.gL(1, B), dinv + dv.gU(1, B)));
    return f32::diag_inv(c, N, h2, dinv + dv.sL(B), dinv + dv.sU(B));
}

// The factorisation is ~2,000 launches whose arguments depend only on the
// sizes and the buffer addresses, so it is replayed as a CUDA graph: the
// first call with a given (sizes, addresses, device) runs normally, the
// second is captured (thread-local capture mode, on a stream of the
// library's own), instantiated and launched on the caller's stream, later
// ones launch the instantiated graph.  Calls made while the caller's stream
// is itself being captured take the plain launch sequence.  Up to kGraphs such graphs are
// kept (least recently used replaced).  Not used while the event profiler
// records (its per-launch records come from the host-side launch sequence).
namespace {
struct InitKey {
    const void *p[12];
    int64_t n, batch, ld, work_bytes, nvec_stride, cfg_epoch;
    int dev;
    bool operator==(const InitKey &o) const {
        for (int i = 0; i < 12; ++i)
            if (p[i] != o.p[i]) return false;
        return n == o.n && batch == o.batch && ld == o.ld && work_bytes == o.work_bytes &&
               nvec_stride == o.nvec_stride && cfg_epoch == o.cfg_epoch && dev == o.dev;
    }
};
struct InitGraph {
    InitKey key;
    cudaGraphExec_t exec;   // null until captured
    int64_t launches;       // kernels in the graph (for the launch counter)
    uint64_t used;
};
constexpr int kGraphs = 4;
constexpr int kMaxDev = 64;
// one non-blocking stream per device for the captures (created once)
cudaStream_t capture_stream(int dev) {
    static cudaStream_t st[kMaxDev] = {};
    if (!st[dev] && cudaStreamCreateWithFlags(&st[dev], cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        st[dev] = nullptr;
    }
    return st[dev];
}
std::mutex g_graph_mu;
std::vector<InitGraph> g_graphs;
uint64_t g_graph_clock = 0;
}  // namespace

extern "C" int mnpb_bemret_init_mixed(void *stream, int64_t n, int64_t batch, float *G1,
                                      float *G2, float *H1, float *H2, float *D, int64_t ld,
                                      const double *eps, const double *kvac, const double *nvec,
                                      int64_t nvec_stride, int32_t *piv, int32_t *info,
                                      float *dinv, void *work, int64_t work_bytes) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && batch < 65536 && n < 65536 && ld >= n && ld % 4 == 0,
                 "bemret_init_mixed: bad sizes");
    MNPB_REQUIRE(G1 && G2 && H1 && H2 && D && eps && kvac && nvec && piv && info && dinv && work,
                 "bemret_init_mixed: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_bemret_workspace_mixed(n, batch),
                 "bemret_init_mixed: workspace too small");
    cudaStream_t s = as_stream(stream);
    auto body = [&](cudaStream_t st) {
        return init_mixed_body(st, n, batch, G1, G2, H1, H2, D, ld, eps, kvac,
                               NvecView{nvec, nvec_stride}, piv, info,
                               dinv, work, work_bytes);
    };
    if (prof_on()) return body(s);
    // a caller that is capturing its own graph gets the plain launch sequence
    cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cst) != cudaSuccess || cst != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return body(s);
    }
    InitKey key{{G1, G2, H1, H2, D, eps, kvac, nvec, piv, info, dinv, work},
                n, batch, ld, work_bytes, nvec_stride, tc::gemm_config_epoch(), 0};
    if (cudaGetDevice(&key.dev) != cudaSuccess || key.dev < 0 || key.dev >= kMaxDev) {
        cudaGetLastError();
        return body(s);
    }
    std::lock_guard<std::mutex> lk(g_graph_mu);
    InitGraph *hit = nullptr;
    for (auto &g : g_graphs)
        if (g.key == key) hit = &g;
    if (!hit) {
        // first sighting: remember the key, run normally
        if ((int)g_graphs.size() >= kGraphs) {
            auto lru = g_graphs.begin();
            for (auto it = g_graphs.begin(); it != g_graphs.end(); ++it)
                if (it->used < lru->used) lru = it;
            if (lru->exec) cudaGraphExecDestroy(lru->exec);
            g_graphs.erase(lru);
        }
        g_graphs.push_back(InitGraph{key, nullptr, 0, ++g_graph_clock});
        return body(s);
    }
    hit->used = ++g_graph_clock;
    if (!hit->exec) {
        // captured on a stream of the library's own (the caller's may be the
        // legacy default stream, which cannot be captured); capturing runs
        // nothing, the instantiated graph is then launched on the caller's
        const cudaStream_t cs = capture_stream(key.dev);
        if (!cs || cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return body(s);
        }
        const int64_t l0 = g_launches.load();
        const int rc = body(cs);
        cudaGraph_t graph = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(cs, &graph);
        hit->launches = g_launches.load() - l0;
        g_launches.fetch_sub(hit->launches);   // counted again when the graph runs
        if (rc != MNPB_OK || ec != cudaSuccess || !graph) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return rc != MNPB_OK ? rc : body(s);
        }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            cudaGetLastError();
            return body(s);
        }
        hit->exec = exec;
    }
    if (cudaGraphLaunch(hit->exec, s) != cudaSuccess) {
        set_error("bemret_init_mixed: graph launch failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
        return MNPB_ECUDA;
    }
    count_launch(hit->launches);
    return MNPB_OK;
}

extern "C" int64_t mnpb_bemret_refine_workspace(int64_t n, int64_t batch, int64_t nrhs) {
    const int64_t K = nrhs;
    // msolve scratch (15 K n c128 + 2 x 16 K n float... per entry) + r, d, P1..Q2 + norms
    return batch * n * K * (15 * 16 + 2 * 16 * 8 + 2 * 8 * 16 + 4 * 4 * 16) + 8 * 256 +
           align_up(f32::trsv_state_bytes((int)n, (int)batch), 256) +
           align_up(tc::cgemm_tf32_workspace((int)n, 64, (int)batch), 256);
}

// Solve with the mixed factorisation and refine in FP64:
//   x = M^-1 b;  repeat { r = b - A x (FP64); stop if |r|/|b| < tol; x += M^-1 r }
// b, x: [batch][8][nrhs][n] (b in the excitation layout phi,a,De,alpha; x in
// sig1,h1,sig2,h2).  iters (host int32, batch) and relres (host double,
// batch) receive the iterations used and the final relative residuals.
extern "C" int mnpb_bemret_solve_refine(
    void *stream, int64_t n, int64_t batch, int64_t nrhs, const float *G1p, const float *G2p,
    const float *S1p, const float *Sp, const float *Dp, int64_t ld, const int32_t *piv,
    const float *dinv, const double *G1, const double *G2, const double *H1, const double *H2,
    const double *eps,
    const double *kvac, const double *nvec, int64_t nvec_stride, const double *bvec, double *x,
    int max_iter,
    double tol, int32_t *iters, double *relres, void *work, int64_t work_bytes) {
    clear_error();
    const int64_t K = nrhs;
    MNPB_REQUIRE(n > 0 && batch > 0 && K > 0 && K <= 4 && ld >= n && ld % 4 == 0,
                 "bemret_solve_refine: bad sizes (nrhs <= 4)");
    MNPB_REQUIRE(G1p && G2p && S1p && Sp && Dp && piv && dinv && G1 && G2 && H1 && H2 && eps && kvac &&
                     nvec && bvec && x && iters && relres && work,
                 "bemret_solve_refine: null pointer");
    MNPB_REQUIRE(work_bytes >= mnpb_bemret_refine_workspace(n, batch, nrhs),
                 "bemret_solve_refine: workspace too small");
    cudaStream_t s = as_stream(stream);
    const int N = (int)n, B = (int)batch, k = (int)K;
    const int64_t plane = ld * n;
    const DinvOff dv{f32::diag_inv_floats(n, 1)};
    const int64_t Bn = batch * n;
    Factors F{(float *)G1p, (float *)G2p, (float *)S1p, (float *)Sp, (float *)Dp, ld, plane,
              2 * plane, piv, piv + Bn, piv + 2 * Bn, dinv + dv.gL(0, batch),
              dinv + dv.gU(0, batch), dinv + dv.gL(1, batch), dinv + dv.gU(1, batch),
              dinv + dv.sL(batch), dinv + dv.sU(batch), n, dv.S, nullptr};
    const int64_t per = n * K;
    char *wp = (char *)work;
    auto take = [&](int64_t bytes) {
        char *p = wp;
        wp += align_up(bytes, 256);
        return p;
    };
    cd *scr = (cd *)take(batch * per * 15 * 16);
    float *fscr = (float *)take(batch * per * 2 * 16 * 8);
    cd *r = (cd *)take(batch * per * 8 * 16);
    cd *dx = (cd *)take(batch * per * 8 * 16);
    cd *P = (cd *)take(batch * per * 4 * 4 * 16);
    double *nrm = (double *)take(batch * 4 * 8);
    F.trsv_state = (int *)take(f32::trsv_state_bytes(N, B));
    const int64_t tcw = (int64_t)((char *)work + work_bytes - wp);
    f32::Ctx c(s, B, (float *)wp, tcw);
    const int64_t sx = per * 8, sP4 = per * 4;
    cd *P1 = P, *P2 = P + batch * sP4, *Q1 = P + 2 * batch * sP4, *Q2 = P + 3 * batch * sP4;
    const cd *bb = (const cd *)bvec;
    cd *xx = (cd *)x;

    const NvecView nv{nvec, nvec_stride};
    MNPB_TRY(msolve(c, N, k, F, eps, kvac, nv, bb, xx, scr, fscr));
    std::vector<double> hn(4 * batch);
    std::vector<int> done(batch, 0);
    for (int b = 0; b < B; ++b) {
        iters[b] = 0;
        relres[b] = 0.0;
    }
    const int64_t sG = ld * n;   // c128 matrices use the same leading dimension
    // r = b - A x on entries [e0, B) (residual vectors at r + e0 * sx)
    auto residual = [&](int e0) -> int {
        const int Bp = B - e0;
        dim3 gz(ceil_div(n, 128), Bp);
        dim3 gzs(ceil_div(n, ZS_ROWS), Bp);
        const cd *xa = xx + (int64_t)e0 * sx;
        ProfScope ps(s, PC_MATVEC, 4.0 * 16.0 * (double)n * n * Bp);   // bytes of A read
        const int64_t om = (int64_t)e0 * sG;
        const cd *mats[4] = {(const cd *)G1 + om, (const cd *)G2 + om, (const cd *)H1 + om,
                             (const cd *)H2 + om};
        const cd *xs[4] = {xa, xa + 4 * per, xa, xa + 4 * per};
        cd *ys[4] = {P1, P2, Q1, Q2};
        for (int q = 0; q < 4; ++q) {
            // at most 8 columns per launch (shared-memory bound of the lane reduction)
            for (int c0 = 0; c0 < 4 * k; c0 += 8) {
                const int mc = min(8, 4 * k - c0);
                const cd *xq = xs[q] + (int64_t)c0 * N;
                cd *yq = ys[q] + (int64_t)c0 * N;
                if (mc <= 4)
                    zskinny_kernel<4><<<gzs, 256, 0, s>>>(N, mc, mats[q], ld, sG, xq, sx, yq, sP4);
                else
                    zskinny_kernel<8><<<gzs, 256, 0, s>>>(N, mc, mats[q], ld, sG, xq, sx, yq, sP4);
            }
        }
        count_launch(3);
        MNPB_LAUNCH_CHECK("zskinny_kernel");
        residual_kernel<<<gz, 128, 0, s>>>(N, k, P1, P2, Q1, Q2, sP4, bb + (int64_t)e0 * sx,
                                           r + (int64_t)e0 * sx, sx, eps + 4 * (int64_t)e0,
                                           kvac + e0, nv.shifted(e0));
        MNPB_LAUNCH_CHECK("residual_kernel");
        return MNPB_OK;
    };
    // per entry of [e0, B): |dx|^2, |x|^2 (hn[2 i], hn[2 i + 1]) and |r|^2, |b|^2
    // (hn[2 Bp + 2 i], hn[2 Bp + 2 i + 1]) to the host
    auto norms = [&](int e0) -> int {
        const int Bp = B - e0;
        norms_kernel<<<Bp, 256, 0, s>>>(sx, dx + (int64_t)e0 * sx, xx + (int64_t)e0 * sx, sx, nrm);
        norms_kernel<<<Bp, 256, 0, s>>>(sx, r + (int64_t)e0 * sx, bb + (int64_t)e0 * sx, sx,
                                        nrm + 2 * Bp);
        MNPB_LAUNCH_CHECK("norms_kernel");
        if (cudaMemcpyAsync(hn.data(), nrm, sizeof(double) * 4 * Bp, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            set_error("bemret_solve_refine: norm copy failed");
            return MNPB_ECUDA;
        }
        return MNPB_OK;
    };
    // Classical iterative refinement: r = b - A x (FP64), dx = M^-1 r (mixed),
    // x += dx; an entry is finished when its last correction is below tol
    // relative to the solution (a forward-error test: the residual alone
    // under-states the error of ill-conditioned entries).  Entries finish at
    // different rates; each pass works on [b0, B), b0 = the first entry not
    // finished (the batch is a wavelength sweep whose slow entries gather at
    // one end), through offset pointers.
    int b0 = 0;
    bool all = false;
    for (int it = 0; it < max_iter && !all; ++it) {
        const int Bp = B - b0;
        MNPB_TRY(residual(b0));
        f32::Ctx ca(s, Bp, (float *)wp, tcw);
        MNPB_TRY(msolve(ca, N, k, F.at(b0), eps + 4 * (int64_t)b0, kvac + b0, nv.shifted(b0),
                        r + (int64_t)b0 * sx, dx + (int64_t)b0 * sx, scr, fscr));
        axpy_kernel<<<ceil_div((int64_t)Bp * sx, 256), 256, 0, s>>>((int64_t)Bp * sx,
                                                                    dx + (int64_t)b0 * sx,
                                                                    xx + (int64_t)b0 * sx);
        MNPB_LAUNCH_CHECK("axpy_kernel");
        MNPB_TRY(norms(b0));
        all = true;
        for (int i = 0; i < Bp; ++i) {
            const int b = b0 + i;
            if (done[b]) continue;
            iters[b] = it + 1;
            relres[b] = hn[2 * Bp + 2 * i + 1] > 0
                            ? std::sqrt(hn[2 * Bp + 2 * i] / hn[2 * Bp + 2 * i + 1])
                            : 0.0;
            const double rel = hn[2 * i + 1] > 0 ? std::sqrt(hn[2 * i] / hn[2 * i + 1]) : 0.0;
            if (rel < tol) done[b] = 1;
            if (!done[b]) all = false;
        }
        while (b0 < B && done[b0]) ++b0;
    }
    // relres holds each entry's relative residual before its last correction
    // (no extra pass over the FP64 operator just to report the final one)
    int terr = 0, gerr = 0;
    MNPB_TRY(f32::trsv_error_read_and_clear(s, &terr));
    MNPB_TRY(tc::tc_error_read_and_clear(s, &gerr));
    if (terr || gerr) {
        set_error("bemret_solve_refine: a bounded device wait timed out (%s)",
                  terr ? "triangular solve" : "tensor-core GEMM of the factorisation");
        return MNPB_ETIMEOUT;
    }
    for (int b = 0; b < B; ++b)
        if (!done[b]) {
            set_error("bemret_solve_refine: batch entry %d: the last of %d corrections was "
                      "still above the tolerance %.1e (relative residual %.3e)",
                      b, max_iter, tol, relres[b]);
            return MNPB_ENOCONV;
        }
    return MNPB_OK;
}
