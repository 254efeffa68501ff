// Green-function kernels: refined Taylor coefficients (FP64 singular and
// near-singular quadrature), closed-surface sums, the quasistatic matrix and
// the batched retarded assembly of G1, H1, G2, H2.
#include "common.cuh"

namespace mnpb {

static constexpr double kEps = 2.220446049250313e-16;   // numpy finfo(float).eps
static constexpr int kOrder = 5;                          // Taylor order of the refinement
static constexpr int kMaxParts = 16;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// Refined coefficients, one warp per refined pair.
// Self pairs  (mnpbem/greenfun/greenret_refined.py:166-248): polar points of
//   the face, g_n = sum w r^(n-1)/n!, f = nvec f1 + tvec1 f2 + tvec2 f3 with
//   f1_n = sum w (n-1) n.r r^(n-3)/n!, f2_n = sum w (n-1) t1.r r^n/rr^3/n!,
//   rr = max(r, 1e-4 max r).
// Near pairs  (greenret_refined.py:336-442): face points of the column face,
//   delta = r - r0, g_n = sum w delta^n/(r n!), f_0 = -sum w x/r^3,
//   f_n = sum w x (-delta^n/(r^3 n!) + delta^(n-1)/(r^2 (n-1)!)).
// Static values (compgreen_stat.py:340-416): gstat = sum w/r,
//   fstat = -sum w n.x/r^3.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) refine_kernel(
    const double *__restrict__ pos, const double *__restrict__ nvec,
    const double *__restrict__ tv1, const double *__restrict__ tv2, int64_t nref,
    const int32_t *__restrict__ rows, const int32_t *__restrict__ cols,
    const int8_t *__restrict__ kinds, const double *__restrict__ qpos,
    const double *__restrict__ qw, const int64_t *__restrict__ qoff,
    const double *__restrict__ ppos, const double *__restrict__ pw,
    const int64_t *__restrict__ poff, double *__restrict__ g, double *__restrict__ f,
    double *__restrict__ gstat, double *__restrict__ fstat) {
    const int64_t pair = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (pair >= nref) return;
    const int i = rows[pair], j = cols[pair];
    const int kind = kinds[pair];
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double nx = nvec[3 * i], ny = nvec[3 * i + 1], nz = nvec[3 * i + 2];
    const double inv_fact[kOrder + 1] = {1.0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0};

    double ag[kOrder + 1], a1[kOrder + 1], a2[kOrder + 1], a3[kOrder + 1];
#pragma unroll
    for (int m = 0; m <= kOrder; ++m) ag[m] = a1[m] = a2[m] = a3[m] = 0.0;
    double sg = 0.0, sf = 0.0;

    if (kind == 2) {
        const double ax = tv1[3 * i], ay = tv1[3 * i + 1], az = tv1[3 * i + 2];
        const double bx = tv2[3 * i], by = tv2[3 * i + 1], bz = tv2[3 * i + 2];
        const int64_t lo = poff[j], hi = poff[j + 1];
        double rmax = 0.0;
        for (int64_t p = lo + lane; p < hi; p += 32) {
            double vx = px - ppos[3 * p], vy = py - ppos[3 * p + 1], vz = pz - ppos[3 * p + 2];
            double r = fmax(sqrt(vx * vx + vy * vy + vz * vz), kEps);
            rmax = fmax(rmax, r);
        }
        rmax = warp_max(rmax);
        for (int64_t p = lo + lane; p < hi; p += 32) {
            double vx = px - ppos[3 * p], vy = py - ppos[3 * p + 1], vz = pz - ppos[3 * p + 2];
            double w = pw[p];
            double r = fmax(sqrt(vx * vx + vy * vy + vz * vz), kEps);
            double ndr = nx * vx + ny * vy + nz * vz;
            double in1 = ax * vx + ay * vy + az * vz;
            double in2 = bx * vx + by * vy + bz * vz;
            double rr = fmax(r, 1e-4 * rmax);
            double irr3 = 1.0 / (rr * rr * rr);
            double ir = 1.0 / r;
            double rp1 = ir;                 // r^(n-1)
            double rp3 = ir * ir * ir;       // r^(n-3)
            double rpn = 1.0;                // r^n
            sg += w * ir;
            sf -= w * ndr * ir * ir * ir;
#pragma unroll
            for (int m = 0; m <= kOrder; ++m) {
                double wm = w * (double)(m - 1);
                ag[m] += w * rp1;
                a1[m] += wm * ndr * rp3;
                a2[m] += wm * in1 * rpn * irr3;
                a3[m] += wm * in2 * rpn * irr3;
                rp1 *= r;
                rp3 *= r;
                rpn *= r;
            }
        }
#pragma unroll
        for (int m = 0; m <= kOrder; ++m) {
            ag[m] = warp_sum(ag[m]) * inv_fact[m];
            a1[m] = warp_sum(a1[m]) * inv_fact[m];
            a2[m] = warp_sum(a2[m]) * inv_fact[m];
            a3[m] = warp_sum(a3[m]) * inv_fact[m];
        }
        sg = warp_sum(sg);
        sf = warp_sum(sf);
        if (lane == 0) {
            for (int m = 0; m <= kOrder; ++m) {
                g[6 * pair + m] = ag[m];
                f[18 * pair + 0 * 6 + m] = nx * a1[m] + ax * a2[m] + bx * a3[m];
                f[18 * pair + 1 * 6 + m] = ny * a1[m] + ay * a2[m] + by * a3[m];
                f[18 * pair + 2 * 6 + m] = nz * a1[m] + az * a2[m] + bz * a3[m];
            }
            gstat[pair] = sg;
            fstat[pair] = sf;
        }
    } else {
        const double cx = pos[3 * j] - px, cy = pos[3 * j + 1] - py, cz = pos[3 * j + 2] - pz;
        const double r0 = sqrt(cx * cx + cy * cy + cz * cz);
        const int64_t lo = qoff[j], hi = qoff[j + 1];
        // a1/a2/a3 hold the x/y/z components of f
        for (int64_t p = lo + lane; p < hi; p += 32) {
            double x = px - qpos[3 * p], y = py - qpos[3 * p + 1], z = pz - qpos[3 * p + 2];
            double w = qw[p];
            double r = fmax(sqrt(x * x + y * y + z * z), kEps);
            double ir = 1.0 / r, ir2 = ir * ir, ir3 = ir2 * ir;
            double dl = r - r0;
            sg += w * ir;
            sf -= w * (nx * x + ny * y + nz * z) * ir3;
            double dpn = 1.0;
#pragma unroll
            for (int m = 0; m <= kOrder; ++m) {
                ag[m] += dpn * ir * inv_fact[m] * w;
                dpn *= dl;
            }
            double fs = -ir3 * w;
            a1[0] += x * fs;
            a2[0] += y * fs;
            a3[0] += z * fs;
            double dpm = 1.0;
            dpn = dl;
#pragma unroll
            for (int m = 1; m <= kOrder; ++m) {
                double s = (-dpn * ir3 * inv_fact[m] + dpm * ir2 * inv_fact[m - 1]) * w;
                a1[m] += x * s;
                a2[m] += y * s;
                a3[m] += z * s;
                dpm = dpn;
                dpn *= dl;
            }
        }
#pragma unroll
        for (int m = 0; m <= kOrder; ++m) {
            ag[m] = warp_sum(ag[m]);
            a1[m] = warp_sum(a1[m]);
            a2[m] = warp_sum(a2[m]);
            a3[m] = warp_sum(a3[m]);
        }
        sg = warp_sum(sg);
        sf = warp_sum(sf);
        if (lane == 0) {
            for (int m = 0; m <= kOrder; ++m) {
                g[6 * pair + m] = ag[m];
                f[18 * pair + 0 * 6 + m] = a1[m];
                f[18 * pair + 1 * 6 + m] = a2[m];
                f[18 * pair + 2 * 6 + m] = a3[m];
            }
            gstat[pair] = sg;
            fstat[pair] = sf;
        }
    }
}


// Closure correction on the self pairs (mnpbem/greenfun/compgreen_ret.py:376-400:
// f[self, :, 0] += corr_i nvec_i) and the normal projection fn = n_row . f used
// by the F assembly.
__device__ __forceinline__ double closure_corr(const double *cdir, const double *fsum, int i) {
    // -2 pi dir - f on faces of a closed surface (dir = +-1), 0 elsewhere
    return cdir[i] != 0.0 ? -6.283185307179586 * cdir[i] - fsum[i] : 0.0;
}

__global__ void refine_finalize_kernel(int64_t nref, const int32_t *__restrict__ rows,
                                       const int32_t *__restrict__ cols,
                                       const double *__restrict__ nvec,
                                       const double *__restrict__ cdir,
                                       const double *__restrict__ fsum, double *__restrict__ f,
                                       double *__restrict__ fn) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nref) return;
    const int i = rows[p];
    const double n0 = nvec[3 * i], n1 = nvec[3 * i + 1], n2 = nvec[3 * i + 2];
    double *fp = f + 18 * p;
    if (cdir && i == cols[p]) {
        const double c = closure_corr(cdir, fsum, i);
        fp[0] += c * n0;
        fp[6] += c * n1;
        fp[12] += c * n2;
    }
    for (int m = 0; m <= kOrder; ++m) fn[6 * p + m] = n0 * fp[m] + n1 * fp[6 + m] + n2 * fp[12 + m];
}

__device__ __forceinline__ double static_far_F(const double *pos, const double *nvec,
                                               const double *area, int i, int j) {
    double rx = pos[3 * i] - pos[3 * j];
    double ry = pos[3 * i + 1] - pos[3 * j + 1];
    double rz = pos[3 * i + 2] - pos[3 * j + 2];
    double d = fmax(sqrt(rx * rx + ry * ry + rz * rz), kEps);
    double ndr = nvec[3 * i] * rx + nvec[3 * i + 1] * ry + nvec[3 * i + 2] * rz;
    return -ndr * area[j] / (d * d * d);
}

// Closed-surface sums, one warp per column j.  Refined rows of column j are
// sorted (CSC); membership is found by binary search.
__global__ void closure_kernel(int64_t n, const double *__restrict__ pos,
                               const double *__restrict__ nvec, const double *__restrict__ area,
                               const int64_t *__restrict__ grp_lo,
                               const int64_t *__restrict__ grp_hi,
                               const int64_t *__restrict__ cptr,
                               const int32_t *__restrict__ crows,
                               const double *__restrict__ cfstat, double *__restrict__ fsum) {
    const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= n) return;
    const int64_t c0 = cptr[j], c1 = cptr[j + 1];
    const double aj = area[j];
    double acc = 0.0;
    for (int64_t i = grp_lo[j] + lane; i < grp_hi[j]; i += 32) {
        int64_t lo = c0, hi = c1;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (crows[mid] < i) lo = mid + 1; else hi = mid;
        }
        double F;
        if (lo < c1 && crows[lo] == i) F = cfstat[lo];
        else F = static_far_F(pos, nvec, area, (int)i, (int)j);
        acc += area[i] * F / aj;
    }
    acc = warp_sum(acc);
    if (lane == 0) fsum[j] = acc;
}

__global__ void static_far_kernel(int64_t n, const double *__restrict__ pos,
                                  const double *__restrict__ nvec,
                                  const double *__restrict__ area, double *__restrict__ F,
                                  int64_t ld) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = blockIdx.y;
    if (i >= n) return;
    F[j * ld + i] = (i == j) ? 0.0 : static_far_F(pos, nvec, area, (int)i, (int)j);
}

__global__ void static_overlay_kernel(int64_t n, const int64_t *__restrict__ rptr,
                                      const int32_t *__restrict__ rcols,
                                      const double *__restrict__ rfstat,
                                      const double *__restrict__ cdir,
                                      const double *__restrict__ fsum, double *__restrict__ F,
                                      int64_t ld) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int64_t p = rptr[i]; p < rptr[i + 1]; ++p) {
        int64_t j = rcols[p];
        double v = rfstat[p];
        if (j == i && cdir) v += closure_corr(cdir, fsum, (int)i);
        F[j * ld + i] = v;
    }
}

// ---------------------------------------------------------------------------
// Retarded assembly.
// ---------------------------------------------------------------------------
struct PartTable {
    int nparts;
    int64_t off[kMaxParts + 1];
};

__device__ __forceinline__ int part_of(const PartTable &t, int64_t i) {
    int p = 0;
    while (p + 1 < t.nparts && i >= t.off[p + 1]) ++p;
    return p;
}

struct StoreC128 {
    cd *G1, *H1, *G2, *H2;
    int64_t ld, stride;
    __device__ __forceinline__ void put(int64_t b, int64_t i, int64_t j, cd g1, cd h1, cd g2,
                                        cd h2) const {
        int64_t o = b * stride + j * ld + i;
        G1[o] = g1;
        H1[o] = h1;
        G2[o] = g2;
        H2[o] = h2;
    }
};

struct StoreC32P {
    float *G1, *H1, *G2, *H2;
    int64_t ld, stride, plane;
    __device__ __forceinline__ void put(int64_t b, int64_t i, int64_t j, cd g1, cd h1, cd g2,
                                        cd h2) const {
        int64_t o = b * stride + j * ld + i;
        G1[o] = (float)g1.x;
        G1[o + plane] = (float)g1.y;
        H1[o] = (float)h1.x;
        H1[o + plane] = (float)h1.y;
        G2[o] = (float)g2.x;
        G2[o + plane] = (float)g2.y;
        H2[o] = (float)h2.x;
        H2[o + plane] = (float)h2.y;
    }
};

struct StoreBoth {
    StoreC128 a;
    StoreC32P b;
    __device__ __forceinline__ void put(int64_t bb, int64_t i, int64_t j, cd g1, cd h1, cd g2,
                                        cd h2) const {
        a.put(bb, i, j, g1, h1, g2, h2);
        b.put(bb, i, j, g1, h1, g2, h2);
    }
};

// Far-field formula for one entry and one wavenumber (greenret_refined.py:738,
// 764-767, 745): G = a/d e^{ikd}, F = (nx faux x + ny faux y + nz faux z) a e^{ikd}
// with faux = (ik - 1/d)/d^2.
__device__ __forceinline__ void far_entry(cd k, double d, double inv_d, double x, double y,
                                          double z, double nx, double ny, double nz, double a,
                                          cd &G, cd &F) {
    cd ph = cexpi(k, d);
    double inv_d2 = inv_d * inv_d;
    cd faux = cmk((-k.y - inv_d) * inv_d2, k.x * inv_d2);
    cd t = cadd(cadd(cscale(faux, nx * x), cscale(faux, ny * y)), cscale(faux, nz * z));
    G = cscale(ph, a * inv_d);
    F = cmul(cscale(t, a), ph);
}

template <class Store>
__global__ void __launch_bounds__(128) assemble_far_kernel(
    int64_t n, PartTable parts, const double *__restrict__ pos,
    const double *__restrict__ nvec, const double *__restrict__ area,
    const double *__restrict__ kblk, const double *__restrict__ sblk, Store st) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (i >= n) return;
    const int pi = part_of(parts, i), pj = part_of(parts, j);
    const int np = parts.nparts;
    const int64_t t1 = ((b * 2 + 0) * np + pi) * np + pj;
    const int64_t t2 = ((b * 2 + 1) * np + pi) * np + pj;
    const double s1 = sblk[t1], s2 = sblk[t2];
    const cd k1 = cmk(kblk[2 * t1], kblk[2 * t1 + 1]);
    const cd k2 = cmk(kblk[2 * t2], kblk[2 * t2 + 1]);
    double x = pos[3 * i] - pos[3 * j];
    double y = pos[3 * i + 1] - pos[3 * j + 1];
    double z = pos[3 * i + 2] - pos[3 * j + 2];
    double d = sqrt(x * x + y * y + z * z);
    if (d < kEps || (i == j)) d = kEps;
    const double inv_d = 1.0 / d;
    const double nx = nvec[3 * i], ny = nvec[3 * i + 1], nz = nvec[3 * i + 2];
    const double a = area[j];
    cd G1 = cmk(0, 0), F1 = cmk(0, 0), G2 = cmk(0, 0), F2 = cmk(0, 0);
    if (s1 != 0.0) {
        far_entry(k1, d, inv_d, x, y, z, nx, ny, nz, a, G1, F1);
        G1 = cscale(G1, s1);
        F1 = cscale(F1, s1);
    }
    if (s2 != 0.0) {
        far_entry(k2, d, inv_d, x, y, z, nx, ny, nz, a, G2, F2);
        G2 = cscale(G2, s2);
        F2 = cscale(F2, s2);
    }
    const double two_pi = 6.283185307179586;
    if (i == j) {
        F1.x += two_pi;
        F2.x -= two_pi;
    }
    st.put(b, i, j, G1, F1, G2, F2);
}

// Refined overlay: one thread per (refined pair, wavelength).  Replaces the
// far value by sum_n c_n (ik)^n times the same phase (greenret_refined.py:740-745,
// 769-776).
template <class Store>
__global__ void assemble_refined_kernel(int64_t nref, int64_t batch, PartTable parts,
                                        const double *__restrict__ pos,
                                        const double *__restrict__ kblk,
                                        const double *__restrict__ sblk,
                                        const int32_t *__restrict__ rows,
                                        const int32_t *__restrict__ cols,
                                        const double *__restrict__ g,
                                        const double *__restrict__ fn, Store st) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nref * batch) return;
    const int64_t p = t % nref, b = t / nref;
    const int i = rows[p], j = cols[p];
    const int pi = part_of(parts, i), pj = part_of(parts, j);
    const int np = parts.nparts;
    double x = pos[3 * i] - pos[3 * j];
    double y = pos[3 * i + 1] - pos[3 * j + 1];
    double z = pos[3 * i + 2] - pos[3 * j + 2];
    double d = sqrt(x * x + y * y + z * z);
    if (d < kEps || i == j) d = kEps;
    cd out[4];
    for (int s = 0; s < 2; ++s) {
        const int64_t tt = ((b * 2 + s) * np + pi) * np + pj;
        const double sg = sblk[tt];
        const cd k = cmk(kblk[2 * tt], kblk[2 * tt + 1]);
        cd Gs = cmk(0, 0), Fs = cmk(0, 0);
        if (sg != 0.0) {
            const cd ik = cmk(-k.y, k.x);
            cd pw = cmk(1.0, 0.0);
            for (int m = 0; m <= kOrder; ++m) {
                Gs = cadd(Gs, cscale(pw, g[6 * p + m]));
                Fs = cadd(Fs, cscale(pw, fn[6 * p + m]));
                pw = cmul(pw, ik);
            }
            const cd ph = cexpi(k, d);
            Gs = cscale(cmul(Gs, ph), sg);
            Fs = cscale(cmul(Fs, ph), sg);
        }
        out[2 * s] = Gs;
        out[2 * s + 1] = Fs;
    }
    if (i == j) {
        out[1].x += 6.283185307179586;
        out[3].x -= 6.283185307179586;
    }
    st.put(b, i, j, out[0], out[1], out[2], out[3]);
}

// ---------------------------------------------------------------------------
// Region-pair Green functions entry by entry and their products with surface
// charges and currents.
//
// CompGreenRet.eval / eval_block / eval(ind) (mnpbem/greenfun/compgreen_ret.py:
// 507-738, 859-908) assemble, for region pair (i, j), every particle block
// whose connectivity is non-zero at that block's wavenumber; the entries are
// those of GreenRetRefined.eval (greenret_refined.py:654-867): the far formula
// with the phase, the refined Taylor sum on near/self pairs, H1/H2 = F +- 2 pi
// and H1p/H2p = Gp +- 2 pi nvec on the diagonal.  Gp is the Cartesian
// derivative (faux r a e^{ikd}, refined sum_n f[:, c, n] (ik)^n).  With k = 0
// the same entries are the quasistatic ones of CompGreenStat (compgreen_stat.py:
// 219-464, 859-990): e^0 = 1 and (ik)^n = 0 for n > 0 leave the order-0
// coefficients, which equal the static refined values.
// ---------------------------------------------------------------------------
enum GreenKey { GK_G = 0, GK_F = 1, GK_H1 = 2, GK_H2 = 3, GK_GP = 4, GK_H1P = 5, GK_H2P = 6 };

struct EvalTables {
    int64_t n;
    PartTable parts;
    const double *pos, *nvec, *area;
    const double *kblk;    // nparts x nparts complex wavenumbers (re, im)
    const double *sblk;    // nparts x nparts factors (0: block not connected)
    const int64_t *rptr;   // refined pairs, CSR by row, columns ascending
    const int32_t *cols;
    const double *g, *fn, *f;   // (nref, 6), (nref, 6), (nref, 3, 6)
};

__device__ __forceinline__ int64_t find_refined(const EvalTables &t, int64_t i, int64_t j) {
    int64_t lo = t.rptr[i], hi = t.rptr[i + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int64_t c = t.cols[mid];
        if (c < j)
            lo = mid + 1;
        else if (c > j)
            hi = mid;
        else
            return mid;
    }
    return -1;
}

// Entry (i, j) for `key`: v[0] for scalar keys, v[0..2] for Gp/H1p/H2p.
__device__ void green_entry(const EvalTables &t, int key, int64_t i, int64_t j, cd v[3]) {
    v[0] = v[1] = v[2] = cmk(0.0, 0.0);
    const int np = t.parts.nparts;
    const int64_t blk = (int64_t)part_of(t.parts, i) * np + part_of(t.parts, j);
    const double sg = t.sblk[blk];
    if (sg == 0.0) return;
    const cd k = cmk(t.kblk[2 * blk], t.kblk[2 * blk + 1]);
    const double x = t.pos[3 * i] - t.pos[3 * j];
    const double y = t.pos[3 * i + 1] - t.pos[3 * j + 1];
    const double z = t.pos[3 * i + 2] - t.pos[3 * j + 2];
    double d = sqrt(x * x + y * y + z * z);
    if (d < kEps || i == j) d = kEps;
    const bool vec = key >= GK_GP;
    const cd ph = cexpi(k, d);
    const int64_t p = find_refined(t, i, j);
    if (p >= 0) {
        const cd ik = cmk(-k.y, k.x);
        cd pw = cmk(1.0, 0.0), s0 = cmk(0.0, 0.0), s1 = s0, s2 = s0;
        for (int m = 0; m <= kOrder; ++m) {
            if (!vec) {
                s0 = cadd(s0, cscale(pw, key == GK_G ? t.g[6 * p + m] : t.fn[6 * p + m]));
            } else {
                s0 = cadd(s0, cscale(pw, t.f[18 * p + m]));
                s1 = cadd(s1, cscale(pw, t.f[18 * p + 6 + m]));
                s2 = cadd(s2, cscale(pw, t.f[18 * p + 12 + m]));
            }
            pw = cmul(pw, ik);
        }
        v[0] = cmul(s0, ph);
        if (vec) {
            v[1] = cmul(s1, ph);
            v[2] = cmul(s2, ph);
        }
    } else {
        const double a = t.area[j];
        const double inv_d = 1.0 / d;
        if (key == GK_G) {
            v[0] = cscale(ph, a * inv_d);
        } else {
            const double inv_d2 = inv_d * inv_d;
            const cd faux = cmk((-k.y - inv_d) * inv_d2, k.x * inv_d2);
            if (!vec) {
                const double nx = t.nvec[3 * i], ny = t.nvec[3 * i + 1], nz = t.nvec[3 * i + 2];
                const cd tt = cadd(cadd(cscale(faux, nx * x), cscale(faux, ny * y)),
                                   cscale(faux, nz * z));
                v[0] = cmul(cscale(tt, a), ph);
            } else {
                v[0] = cmul(cscale(cscale(faux, x), a), ph);
                v[1] = cmul(cscale(cscale(faux, y), a), ph);
                v[2] = cmul(cscale(cscale(faux, z), a), ph);
            }
        }
    }
    if (sg != 1.0)
        for (int c = 0; c < 3; ++c) v[c] = cscale(v[c], sg);
    if (i == j) {
        const double two_pi = 6.283185307179586;
        if (key == GK_H1) v[0].x += two_pi;
        if (key == GK_H2) v[0].x -= two_pi;
        if (key == GK_H1P || key == GK_H2P) {
            const double sgn = key == GK_H1P ? two_pi : -two_pi;
            for (int c = 0; c < 3; ++c) v[c].x += sgn * t.nvec[3 * i + c];
        }
    }
}

// Dense column range [c0, c0 + ncol) (ind == NULL; out row-major (n, ncol) or
// (n, 3, ncol)), or the entries at row-major linear indices ind[0..nind)
// (out (nind) or (nind, 3)).
__global__ void __launch_bounds__(256) green_eval_kernel(EvalTables t, int key, int64_t c0,
                                                         int64_t ncol, const int64_t *ind,
                                                         int64_t nind, cd *out) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool vec = key >= GK_GP;
    cd v[3];
    if (ind) {
        if (tid >= nind) return;
        const int64_t l = ind[tid];
        green_entry(t, key, l / t.n, l % t.n, v);
        if (vec)
            for (int c = 0; c < 3; ++c) out[3 * tid + c] = v[c];
        else
            out[tid] = v[0];
        return;
    }
    if (tid >= t.n * ncol) return;
    const int64_t i = tid / ncol, jj = tid - i * ncol;
    green_entry(t, key, i, c0 + jj, v);
    if (vec)
        for (int c = 0; c < 3; ++c) out[(i * 3 + c) * ncol + jj] = v[c];
    else
        out[tid] = v[0];
}

// Products with the region-pair matrix, one CTA per row i, entries computed
// on the fly (no n x n storage):
//   mode 0 (scalar key): y(i, c)    = sum_j M_ij x(j, c),             c < m
//   mode 1 (vector key): y(i, q, c) = sum_j Gp_ij[q] x(j, c),         c < m
//   mode 2 (vector key): y(i, :, c) = sum_j Gp_ij x x(j, :, c)  (cross product)
// x, y row-major complex; m <= APPLY_MAXM columns (m <= APPLY_MAXM / 3 for
// modes 1 and 2).
constexpr int APPLY_MAXM = 12;
constexpr int APPLY_T = 128;

__global__ void __launch_bounds__(APPLY_T) green_apply_kernel(EvalTables t, int key, int mode,
                                                              int m, const cd *__restrict__ x,
                                                              cd *__restrict__ y) {
    const int64_t i = blockIdx.x;
    const int nout = mode == 0 ? m : 3 * m;
    double acc[2 * APPLY_MAXM];
#pragma unroll
    for (int q = 0; q < 2 * APPLY_MAXM; ++q) acc[q] = 0.0;
    for (int64_t j = threadIdx.x; j < t.n; j += APPLY_T) {
        cd v[3];
        green_entry(t, key, i, j, v);
        if (mode == 0) {
#pragma unroll
            for (int c = 0; c < APPLY_MAXM; ++c)
                if (c < m) {
                    const cd r = cmul(v[0], x[j * m + c]);
                    acc[2 * c] += r.x;
                    acc[2 * c + 1] += r.y;
                }
        } else if (mode == 1) {
#pragma unroll
            for (int c = 0; c < APPLY_MAXM / 3; ++c)
                if (c < m) {
                    const cd xv = x[j * m + c];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const cd r = cmul(v[q], xv);
                        acc[2 * (q * m + c)] += r.x;
                        acc[2 * (q * m + c) + 1] += r.y;
                    }
                }
        } else {
#pragma unroll
            for (int c = 0; c < APPLY_MAXM / 3; ++c)
                if (c < m) {
                    const cd hx = x[(j * 3 + 0) * m + c], hy = x[(j * 3 + 1) * m + c],
                             hz = x[(j * 3 + 2) * m + c];
                    const cd r0 = csub(cmul(v[1], hz), cmul(v[2], hy));
                    const cd r1 = csub(cmul(v[2], hx), cmul(v[0], hz));
                    const cd r2 = csub(cmul(v[0], hy), cmul(v[1], hx));
                    acc[2 * (0 * m + c)] += r0.x;
                    acc[2 * (0 * m + c) + 1] += r0.y;
                    acc[2 * (1 * m + c)] += r1.x;
                    acc[2 * (1 * m + c) + 1] += r1.y;
                    acc[2 * (2 * m + c)] += r2.x;
                    acc[2 * (2 * m + c) + 1] += r2.y;
                }
        }
    }
    __shared__ double red[APPLY_T / 32][2 * APPLY_MAXM];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 2 * APPLY_MAXM; ++q) {
        const double w = warp_sum(acc[q]);
        if (lane == 0) red[warp][q] = w;
    }
    __syncthreads();
    if (threadIdx.x < 2 * nout) {
        double sum = 0.0;
        for (int w = 0; w < APPLY_T / 32; ++w) sum += red[w][threadIdx.x];
        reinterpret_cast<double *>(y + i * nout)[threadIdx.x] = sum;
    }
}

}  // namespace mnpb

using namespace mnpb;

static int eval_tables(EvalTables &t, int64_t n, const double *pos, const double *nvec,
                       const double *area, int nparts, const int64_t *poff, const double *kblk,
                       const double *sblk, const int64_t *rptr, const int32_t *cols,
                       const double *g, const double *fn, const double *f, const char *what) {
    MNPB_REQUIRE(n > 0 && n < (int64_t(1) << 31), "%s: bad n", what);
    MNPB_REQUIRE(nparts >= 1 && nparts <= kMaxParts, "%s: nparts must be 1..%d", what,
                 kMaxParts);
    MNPB_REQUIRE(pos && nvec && area && poff && kblk && sblk && rptr && cols && g && fn && f,
                 "%s: null pointer", what);
    t.n = n;
    t.parts.nparts = nparts;
    for (int p = 0; p <= nparts; ++p) t.parts.off[p] = poff[p];
    MNPB_REQUIRE(t.parts.off[0] == 0 && t.parts.off[nparts] == n, "%s: bad offsets", what);
    t.pos = pos;
    t.nvec = nvec;
    t.area = area;
    t.kblk = kblk;
    t.sblk = sblk;
    t.rptr = rptr;
    t.cols = cols;
    t.g = g;
    t.fn = fn;
    t.f = f;
    return MNPB_OK;
}

extern "C" int mnpb_green_eval(void *stream, int64_t n, const double *pos, const double *nvec,
                               const double *area, int nparts, const int64_t *poff,
                               const double *kblk, const double *sblk, const int64_t *rptr,
                               const int32_t *cols, const double *g, const double *fn,
                               const double *f, int key, int64_t col_start, int64_t ncol,
                               const int64_t *ind, int64_t nind, double *out) {
    clear_error();
    EvalTables t;
    MNPB_TRY(eval_tables(t, n, pos, nvec, area, nparts, poff, kblk, sblk, rptr, cols, g, fn, f,
                         "green_eval"));
    MNPB_REQUIRE(key >= GK_G && key <= GK_H2P, "green_eval: key must be 0..6");
    MNPB_REQUIRE(out, "green_eval: null output");
    const int64_t tot = ind ? nind : n * ncol;
    if (!ind)
        MNPB_REQUIRE(col_start >= 0 && ncol >= 0 && col_start + ncol <= n,
                     "green_eval: column range [%lld, %lld) outside [0, %lld)",
                     (long long)col_start, (long long)(col_start + ncol), (long long)n);
    else
        MNPB_REQUIRE(nind >= 0, "green_eval: nind < 0");
    if (tot == 0) return MNPB_OK;
    cudaStream_t s = as_stream(stream);
    green_eval_kernel<<<ceil_div(tot, 256), 256, 0, s>>>(t, key, col_start, ncol, ind, nind,
                                                        (cd *)out);
    MNPB_LAUNCH_CHECK("green_eval_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_green_apply(void *stream, int64_t n, const double *pos, const double *nvec,
                                const double *area, int nparts, const int64_t *poff,
                                const double *kblk, const double *sblk, const int64_t *rptr,
                                const int32_t *cols, const double *g, const double *fn,
                                const double *f, int key, int mode, int64_t m, const double *x,
                                double *y) {
    clear_error();
    EvalTables t;
    MNPB_TRY(eval_tables(t, n, pos, nvec, area, nparts, poff, kblk, sblk, rptr, cols, g, fn, f,
                         "green_apply"));
    MNPB_REQUIRE(key >= GK_G && key <= GK_H2P, "green_apply: key must be 0..6");
    MNPB_REQUIRE(mode >= 0 && mode <= 2 && (mode == 0) == (key < GK_GP),
                 "green_apply: mode 0 takes a scalar key, modes 1 and 2 a vector key");
    MNPB_REQUIRE(m >= 1 && m <= (mode == 0 ? APPLY_MAXM : APPLY_MAXM / 3),
                 "green_apply: m = %lld columns out of range", (long long)m);
    MNPB_REQUIRE(x && y, "green_apply: null pointer");
    green_apply_kernel<<<(unsigned)n, APPLY_T, 0, as_stream(stream)>>>(t, key, mode, (int)m,
                                                                       (const cd *)x, (cd *)y);
    MNPB_LAUNCH_CHECK("green_apply_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_refine_coefficients(void *stream, int64_t n, const double *pos,
                                        const double *nvec, const double *tvec1,
                                        const double *tvec2, int64_t nref, const int32_t *rows,
                                        const int32_t *cols, const int8_t *kinds,
                                        const double *qpos, const double *qw,
                                        const int64_t *qoff, const double *ppos,
                                        const double *pw, const int64_t *poff, double *g,
                                        double *f, double *gstat, double *fstat) {
    clear_error();
    MNPB_REQUIRE(n > 0 && nref >= 0, "refine_coefficients: bad sizes");
    MNPB_REQUIRE(pos && nvec && tvec1 && tvec2 && qoff && poff && g && f && gstat && fstat,
                 "refine_coefficients: null pointer");
    if (nref == 0) return MNPB_OK;
    const int threads = 256;
    const int64_t blocks = (nref * 32 + threads - 1) / threads;
    ProfScope ps(as_stream(stream), PC_REFINE, 0.0);
    refine_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(
        pos, nvec, tvec1, tvec2, nref, rows, cols, kinds, qpos, qw, qoff, ppos, pw, poff, g, f,
        gstat, fstat);
    MNPB_LAUNCH_CHECK("refine_kernel");
    return MNPB_OK;
}


extern "C" int mnpb_refine_finalize(void *stream, int64_t n, int64_t nref, const int32_t *rows,
                                    const int32_t *cols, const double *nvec, const double *cdir,
                                    const double *fsum, double *f, double *fn) {
    clear_error();
    MNPB_REQUIRE(n > 0 && nref >= 0, "refine_finalize: bad sizes");
    MNPB_REQUIRE(rows && cols && nvec && f && fn && (!cdir || fsum),
                 "refine_finalize: null pointer");
    if (nref == 0) return MNPB_OK;
    refine_finalize_kernel<<<ceil_div(nref, 256), 256, 0, as_stream(stream)>>>(
        nref, rows, cols, nvec, cdir, fsum, f, fn);
    MNPB_LAUNCH_CHECK("refine_finalize_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_closure_sums(void *stream, int64_t n, const double *pos, const double *nvec,
                                 const double *area, const int64_t *grp_lo,
                                 const int64_t *grp_hi, const int64_t *cptr,
                                 const int32_t *crows, const double *cfstat, double *fsum) {
    clear_error();
    MNPB_REQUIRE(n > 0, "closure_sums: bad size");
    MNPB_REQUIRE(pos && nvec && area && grp_lo && grp_hi && cptr && fsum,
                 "closure_sums: null pointer");
    const int threads = 256;
    closure_kernel<<<ceil_div(n * 32, threads), threads, 0, as_stream(stream)>>>(
        n, pos, nvec, area, grp_lo, grp_hi, cptr, crows, cfstat, fsum);
    MNPB_LAUNCH_CHECK("closure_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_static_matrix(void *stream, int64_t n, const double *pos, const double *nvec,
                                  const double *area, const int64_t *rptr, const int32_t *rcols,
                                  const double *rfstat, const double *cdir, const double *fsum,
                                  double *F, int64_t ld) {
    clear_error();
    MNPB_REQUIRE(n > 0 && ld >= n && n < 65536, "static_matrix: bad sizes");
    MNPB_REQUIRE(pos && nvec && area && rptr && F, "static_matrix: null pointer");
    dim3 grid(ceil_div(n, 128), (unsigned)n);
    static_far_kernel<<<grid, 128, 0, as_stream(stream)>>>(n, pos, nvec, area, F, ld);
    MNPB_LAUNCH_CHECK("static_far_kernel");
    static_overlay_kernel<<<ceil_div(n, 128), 128, 0, as_stream(stream)>>>(
        n, rptr, rcols, rfstat, cdir, fsum, F, ld);
    MNPB_LAUNCH_CHECK("static_overlay_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_assemble_ret(void *stream, int64_t n, int64_t batch, const double *pos,
                                 const double *nvec, const double *area, int nparts,
                                 const int64_t *poff, const double *kblk, const double *sblk,
                                 int64_t nref, const int32_t *rows, const int32_t *cols,
                                 const double *g, const double *fn, int out_mode, void *G1,
                                 void *H1, void *G2, void *H2, int64_t ld, int64_t stride,
                                 int64_t plane) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && ld >= n && n < 65536 && batch < 65536,
                 "assemble_ret: bad sizes n=%lld batch=%lld ld=%lld", (long long)n,
                 (long long)batch, (long long)ld);
    MNPB_REQUIRE(nparts >= 1 && nparts <= kMaxParts, "assemble_ret: nparts must be 1..%d",
                 kMaxParts);
    MNPB_REQUIRE(pos && nvec && area && poff && kblk && sblk && G1 && H1 && G2 && H2,
                 "assemble_ret: null pointer");
    MNPB_REQUIRE(stride >= ld * n, "assemble_ret: stride too small");
    PartTable parts;
    parts.nparts = nparts;
    for (int p = 0; p <= nparts; ++p) parts.off[p] = poff[p];
    MNPB_REQUIRE(parts.off[0] == 0 && parts.off[nparts] == n, "assemble_ret: bad offsets");
    cudaStream_t s = as_stream(stream);
    dim3 grid(ceil_div(n, 128), (unsigned)n, (unsigned)batch);
    const int64_t tot = nref * batch;
    ProfScope ps(s, PC_ASSEMBLE, (out_mode == 0 ? 64.0 : 32.0) * (double)n * n * batch +
                                     96.0 * (double)nref);
    if (out_mode == 0) {
        StoreC128 st{(cd *)G1, (cd *)H1, (cd *)G2, (cd *)H2, ld, stride};
        assemble_far_kernel<StoreC128><<<grid, 128, 0, s>>>(n, parts, pos, nvec, area, kblk,
                                                            sblk, st);
        MNPB_LAUNCH_CHECK("assemble_far_kernel<c128>");
        if (tot > 0) {
            assemble_refined_kernel<StoreC128><<<ceil_div(tot, 128), 128, 0, s>>>(
                nref, batch, parts, pos, kblk, sblk, rows, cols, g, fn, st);
            MNPB_LAUNCH_CHECK("assemble_refined_kernel<c128>");
        }
    } else if (out_mode == 1) {
        MNPB_REQUIRE(plane >= ld * n, "assemble_ret: plane offset too small");
        StoreC32P st{(float *)G1, (float *)H1, (float *)G2, (float *)H2, ld, stride, plane};
        assemble_far_kernel<StoreC32P><<<grid, 128, 0, s>>>(n, parts, pos, nvec, area, kblk,
                                                            sblk, st);
        MNPB_LAUNCH_CHECK("assemble_far_kernel<c32p>");
        if (tot > 0) {
            assemble_refined_kernel<StoreC32P><<<ceil_div(tot, 128), 128, 0, s>>>(
                nref, batch, parts, pos, kblk, sblk, rows, cols, g, fn, st);
            MNPB_LAUNCH_CHECK("assemble_refined_kernel<c32p>");
        }
    } else {
        set_error("assemble_ret: unknown out_mode %d", out_mode);
        return MNPB_EINVAL;
    }
    return MNPB_OK;
}

extern "C" int mnpb_assemble_ret2(void *stream, int64_t n, int64_t batch, const double *pos,
                                  const double *nvec, const double *area, int nparts,
                                  const int64_t *poff, const double *kblk, const double *sblk,
                                  int64_t nref, const int32_t *rows, const int32_t *cols,
                                  const double *g, const double *fn, double *G1, double *H1,
                                  double *G2, double *H2, int64_t ld, int64_t stride, float *G1p,
                                  float *H1p, float *G2p, float *H2p, int64_t ldp,
                                  int64_t stridep, int64_t planep) {
    clear_error();
    MNPB_REQUIRE(n > 0 && batch > 0 && ld >= n && ldp >= n && n < 65536 && batch < 65536,
                 "assemble_ret2: bad sizes");
    MNPB_REQUIRE(nparts >= 1 && nparts <= kMaxParts, "assemble_ret2: nparts must be 1..%d",
                 kMaxParts);
    MNPB_REQUIRE(pos && nvec && area && poff && kblk && sblk && G1 && H1 && G2 && H2 && G1p &&
                     H1p && G2p && H2p,
                 "assemble_ret2: null pointer");
    MNPB_REQUIRE(stride >= ld * n && planep >= ldp * n && stridep >= 2 * planep,
                 "assemble_ret2: strides too small");
    PartTable parts;
    parts.nparts = nparts;
    for (int p = 0; p <= nparts; ++p) parts.off[p] = poff[p];
    MNPB_REQUIRE(parts.off[0] == 0 && parts.off[nparts] == n, "assemble_ret2: bad offsets");
    cudaStream_t s = as_stream(stream);
    StoreBoth st{StoreC128{(cd *)G1, (cd *)H1, (cd *)G2, (cd *)H2, ld, stride},
                 StoreC32P{G1p, H1p, G2p, H2p, ldp, stridep, planep}};
    dim3 grid(ceil_div(n, 128), (unsigned)n, (unsigned)batch);
    ProfScope ps(s, PC_ASSEMBLE, 96.0 * (double)n * n * batch + 96.0 * (double)nref);
    assemble_far_kernel<StoreBoth><<<grid, 128, 0, s>>>(n, parts, pos, nvec, area, kblk, sblk, st);
    MNPB_LAUNCH_CHECK("assemble_far_kernel<both>");
    const int64_t tot = nref * batch;
    if (tot > 0) {
        assemble_refined_kernel<StoreBoth><<<ceil_div(tot, 128), 128, 0, s>>>(
            nref, batch, parts, pos, kblk, sblk, rows, cols, g, fn, st);
        MNPB_LAUNCH_CHECK("assemble_refined_kernel<both>");
    }
    return MNPB_OK;
}
