// Points off the particle surface: dipole excitations and Green functions
// between observation points and the faces.
//
//  * dipole_pot_kernel     potentials of oscillating dipoles at the faces
//                          (mnpbem/simulation/dipole_ret.py:319-515)
//  * dipole_field_kernel   the dipoles' own fields at observation positions
//                          (dipole_ret.py:163-317, Jackson 9.18)
//  * dipole_farfield_kernel far fields of the dipoles, added onto the far
//                          fields of the surface charges (dipole_ret.py:602-672)
//  * refine_points_kernel  refined Taylor coefficients of point-face pairs
//                          (greenfun/greenret_refined.py:287-442, the point as
//                          source, Cartesian derivative)
//  * point_green_kernel    fields / potentials at the points from surface
//                          charges and currents (greenfun/compgreen_ret.py:
//                          912-1036 with a point set as p1)
//  * point_eval_kernel     entries G / Gp of a point-face region pair
//  * dipole_stat_kernel    quasistatic dipole fields at observation positions
//                          and their normal projections (simulation/
//                          dipole_stat.py:149-289)
#include "common.cuh"

namespace mnpb {
namespace {

constexpr double kEpsP = 2.220446049250313e-16;   // numpy finfo(float).eps
constexpr int kOrd = 5;                           // Taylor order of the refinement

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// Dipole potentials.  Face i, side s (0 inside, 1 outside) and point q are
// connected when the medium on side s of the face is the point's medium m;
// with eps, k of that medium, x = (pos_i - pt_q) / r, dipole d:
//   G = e^{ikr}/r, F = (ik - 1/r) G, en = n.x, ep = x.d, nd = n.d
//   phi  = -ep F / eps
//   phi' = (nd - 3 en ep)/r^2 (1 - ikr) G/eps + k^2 ep en G/eps
//   a    = -i k0 d G,  a' = -i k0 d en F,  k0 = 2 pi / lambda
// pots [b][16][K][n], column K index = q * ndip + idip.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) dipole_pot_kernel(
    int n, int npt, int ndip, const double *__restrict__ pos, const double *__restrict__ nvec,
    const int32_t *__restrict__ face_med, const double *__restrict__ ptpos,
    const int32_t *__restrict__ pt_med, const double *__restrict__ dip, int nmed,
    const double *__restrict__ eps_t, const double *__restrict__ k_t,
    const double *__restrict__ k0v, cd *__restrict__ pots) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (i >= n) return;
    const int K = npt * ndip;
    cd *out = pots + b * (int64_t)16 * K * n;
    auto P = [&](int comp, int col) -> cd & { return out[(int64_t)(comp * K + col) * n + i]; };
    const int m = pt_med[q];
    const double k0 = k0v[b];
    const double x0 = pos[3 * i] - ptpos[3 * q], y0 = pos[3 * i + 1] - ptpos[3 * q + 1],
                 z0 = pos[3 * i + 2] - ptpos[3 * q + 2];
    const double r = sqrt(x0 * x0 + y0 * y0 + z0 * z0);
    const double ux = x0 / r, uy = y0 / r, uz = z0 / r;
    const double nx = nvec[3 * i], ny = nvec[3 * i + 1], nz = nvec[3 * i + 2];
    const double en = nx * ux + ny * uy + nz * uz;
    for (int s = 0; s < 2; ++s) {
        const int base = 8 * s;
        const bool con = m > 0 && m <= nmed && face_med[2 * i + s] == m;
        cd ieps = cmk(0, 0), k = cmk(0, 0), G = cmk(0, 0), F = cmk(0, 0), fac = cmk(0, 0),
           k2 = cmk(0, 0);
        if (con) {
            const int64_t e = b * nmed + (m - 1);
            ieps = crcp(cmk(eps_t[2 * e], eps_t[2 * e + 1]));
            k = cmk(k_t[2 * e], k_t[2 * e + 1]);
            G = cscale(cexpi(k, r), 1.0 / r);
            F = cmul(cmk(-1.0 / r, 0.0), G);
            F = cadd(F, cmul(cmk(-k.y, k.x), G));                  // (ik - 1/r) G
            // (1 - ikr) G / (eps r^2)
            fac = cscale(cmul(cmul(cmk(1.0 + k.y * r, -k.x * r), G), ieps), 1.0 / (r * r));
            k2 = cmul(cmul(cmul(k, k), G), ieps);                  // k^2 G / eps
        }
        for (int id = 0; id < ndip; ++id) {
            const int col = q * ndip + id;
            if (!con) {
                P(base + 0, col) = P(base + 1, col) = cmk(0, 0);
                for (int c = 0; c < 3; ++c) P(base + 2 + c, col) = P(base + 5 + c, col) = cmk(0, 0);
                continue;
            }
            const double dx = dip[(3 * q + 0) * ndip + id], dy = dip[(3 * q + 1) * ndip + id],
                         dz = dip[(3 * q + 2) * ndip + id];
            const double ep = ux * dx + uy * dy + uz * dz;
            const double nd = nx * dx + ny * dy + nz * dz;
            P(base + 0, col) = cscale(cmul(F, ieps), -ep);
            P(base + 1, col) = cadd(cscale(fac, nd - 3.0 * en * ep), cscale(k2, ep * en));
            const cd ag = cmul(cmk(0.0, -k0), G);                  // -i k0 G
            const cd af = cscale(cmul(cmk(0.0, -k0), F), en);      // -i k0 en F
            const double dd[3] = {dx, dy, dz};
            for (int c = 0; c < 3; ++c) {
                P(base + 2 + c, col) = cscale(ag, dd[c]);
                P(base + 5 + c, col) = cscale(af, dd[c]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Fields of the dipoles at observation positions obs_i in medium med_i
// (Jackson 9.18), connected points only (medium equal):
//   h = k^2 G (1 - 1/(ikr)) / sqrt(eps) (x × d)
//   e = k^2 G/eps (d - (x.d) x) + G (1/r^2 - ik/r)/eps (3 (x.d) x - d)
// out e, h [b][nobs][3][K].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) dipole_field_kernel(
    int nobs, int npt, int ndip, const double *__restrict__ obs, const int32_t *__restrict__ med,
    const double *__restrict__ ptpos, const int32_t *__restrict__ pt_med,
    const double *__restrict__ dip, int nmed, const double *__restrict__ eps_t,
    const double *__restrict__ k_t, const double *__restrict__ nb_t, cd *__restrict__ e_out,
    cd *__restrict__ h_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (i >= nobs) return;
    const int K = npt * ndip;
    cd *eo = e_out + b * (int64_t)nobs * 3 * K + (int64_t)i * 3 * K;
    cd *ho = h_out + b * (int64_t)nobs * 3 * K + (int64_t)i * 3 * K;
    const int m = pt_med[q];
    if (m <= 0 || m > nmed || med[i] != m) {
        for (int id = 0; id < ndip; ++id)
            for (int c = 0; c < 3; ++c)
                eo[c * K + q * ndip + id] = ho[c * K + q * ndip + id] = cmk(0, 0);
        return;
    }
    const int64_t e = b * nmed + (m - 1);
    const cd ieps = crcp(cmk(eps_t[2 * e], eps_t[2 * e + 1]));
    const cd inb = crcp(cmk(nb_t[2 * e], nb_t[2 * e + 1]));
    const cd k = cmk(k_t[2 * e], k_t[2 * e + 1]);
    const double x0 = obs[3 * i] - ptpos[3 * q], y0 = obs[3 * i + 1] - ptpos[3 * q + 1],
                 z0 = obs[3 * i + 2] - ptpos[3 * q + 2];
    const double r = sqrt(x0 * x0 + y0 * y0 + z0 * z0);
    const double u[3] = {x0 / r, y0 / r, z0 / r};
    const cd G = cscale(cexpi(k, r), 1.0 / r);
    const cd k2G = cmul(cmul(k, k), G);
    // 1 - 1/(ikr)
    const cd t = csub(cmk(1.0, 0.0), crcp(cmk(-k.y * r, k.x * r)));
    const cd fh = cmul(cmul(k2G, t), inb);
    const cd f1 = cmul(k2G, ieps);
    // G (1/r^2 - ik/r) / eps
    const cd f2 = cmul(cmul(G, cmk(1.0 / (r * r) + k.y / r, -k.x / r)), ieps);
    for (int id = 0; id < ndip; ++id) {
        const double d[3] = {dip[(3 * q + 0) * ndip + id], dip[(3 * q + 1) * ndip + id],
                             dip[(3 * q + 2) * ndip + id]};
        const double in = u[0] * d[0] + u[1] * d[1] + u[2] * d[2];
        const double cr[3] = {u[1] * d[2] - u[2] * d[1], u[2] * d[0] - u[0] * d[2],
                              u[0] * d[1] - u[1] * d[0]};
        const int col = q * ndip + id;
        for (int c = 0; c < 3; ++c) {
            ho[c * K + col] = cscale(fh, cr[c]);
            eo[c * K + col] = cadd(cscale(f1, d[c] - in * u[c]), cscale(f2, 3.0 * in * u[c] - d[c]));
        }
    }
}

// ---------------------------------------------------------------------------
// Quasistatic dipole fields (Jackson 4.13), screened by the dielectric
// function eps_q of the medium of dipole q; every observation position sees
// every dipole:
//   e = (3 x (x.d) - d) / (eps_q r^3),   x = (obs_i - pt_q) / r.
// Without normals out = e [nobs][3][npt][ndip]; with normals n_i out =
// phi' = -n_i.e [nobs][npt][ndip].  One thread per (observation, dipole
// position).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) dipole_stat_kernel(
    int nobs, int npt, int ndip, const double *__restrict__ obs,
    const double *__restrict__ nvec, const double *__restrict__ ptpos,
    const double *__restrict__ dip, const double *__restrict__ eps_pt, cd *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if (i >= nobs) return;
    double x[3];
    for (int c = 0; c < 3; ++c) x[c] = obs[3 * i + c] - ptpos[3 * q + c];
    const double r = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    for (int c = 0; c < 3; ++c) x[c] /= r;
    const cd ie = crcp(cmk(eps_pt[2 * q], eps_pt[2 * q + 1]));
    const double ir3 = 1.0 / (r * r * r);
    for (int a = 0; a < ndip; ++a) {
        const double *d = dip + ((int64_t)q * 3) * ndip + a;       // d[c * ndip]
        const double in = x[0] * d[0] + x[1] * d[ndip] + x[2] * d[2 * ndip];
        double e[3];
        for (int c = 0; c < 3; ++c) e[c] = (3.0 * x[c] * in - d[c * ndip]) * ir3;
        if (nvec) {
            const double *nv = nvec + 3 * i;
            const double en = nv[0] * e[0] + nv[1] * e[1] + nv[2] * e[2];
            out[((int64_t)i * npt + q) * ndip + a] = cscale(ie, -en);
        } else {
            for (int c = 0; c < 3; ++c)
                out[(((int64_t)i * 3 + c) * npt + q) * ndip + a] = cscale(ie, e[c]);
        }
    }
}

// ---------------------------------------------------------------------------
// Far fields of the dipoles in the embedding medium, added onto e, h
// [b][K][ndir][3]: with g = exp(-i k dir.pt),
//   h += k^2 / nb (dir × d) g,   e += k^2 / eps ((dir × d) g) × dir.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) dipole_farfield_kernel(
    int ndir, int npt, int ndip, const double *__restrict__ ptpos,
    const int8_t *__restrict__ pt_on, const double *__restrict__ dip,
    const double *__restrict__ dirs, const double *__restrict__ emb, cd *__restrict__ e,
    cd *__restrict__ h) {
    const int di = blockIdx.x * blockDim.x + threadIdx.x;
    const int col = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (di >= ndir) return;
    const int q = col / ndip, id = col - q * ndip;
    if (!pt_on[q]) return;
    const int K = npt * ndip;
    const cd eps = cmk(emb[6 * b], emb[6 * b + 1]);
    const cd k = cmk(emb[6 * b + 2], emb[6 * b + 3]);
    const cd nb = cmk(emb[6 * b + 4], emb[6 * b + 5]);
    const double *u = dirs + 3 * di;
    const double s = u[0] * ptpos[3 * q] + u[1] * ptpos[3 * q + 1] + u[2] * ptpos[3 * q + 2];
    const cd g = cexpi(cmk(-k.x, -k.y), s);                 // exp(-i k s)
    const cd k2 = cmul(k, k);
    const cd fe = cmul(cmul(k2, crcp(eps)), g);
    const cd fh = cmul(cmul(k2, crcp(nb)), g);
    const double d[3] = {dip[(3 * q + 0) * ndip + id], dip[(3 * q + 1) * ndip + id],
                         dip[(3 * q + 2) * ndip + id]};
    const double c[3] = {u[1] * d[2] - u[2] * d[1], u[2] * d[0] - u[0] * d[2],
                         u[0] * d[1] - u[1] * d[0]};
    const double ce[3] = {c[1] * u[2] - c[2] * u[1], c[2] * u[0] - c[0] * u[2],
                          c[0] * u[1] - c[1] * u[0]};
    const int64_t o = ((b * K + col) * (int64_t)ndir + di) * 3;
    for (int a = 0; a < 3; ++a) {
        h[o + a] = cadd(h[o + a], cscale(fh, c[a]));
        e[o + a] = cadd(e[o + a], cscale(fe, ce[a]));
    }
}

// ---------------------------------------------------------------------------
// Refined coefficients of point-face pairs, one warp per pair: the near-pair
// expansion of the face-face case with the point as source (no normal):
//   delta = r - r0, g_n = sum w delta^n / (r n!), f_0 = -sum w x / r^3,
//   f_n = sum w x (-delta^n / (r^3 n!) + delta^(n-1) / (r^2 (n-1)!)).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) refine_points_kernel(
    const double *__restrict__ ptpos, const double *__restrict__ pos, int64_t nref,
    const int32_t *__restrict__ rows, const int32_t *__restrict__ cols,
    const double *__restrict__ qpos, const double *__restrict__ qw,
    const int64_t *__restrict__ qoff, double *__restrict__ g, double *__restrict__ f) {
    const int64_t pair = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (pair >= nref) return;
    const int i = rows[pair], j = cols[pair];
    const double inv_fact[kOrd + 1] = {1.0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0};
    const double px = ptpos[3 * i], py = ptpos[3 * i + 1], pz = ptpos[3 * i + 2];
    const double cx = pos[3 * j] - px, cy = pos[3 * j + 1] - py, cz = pos[3 * j + 2] - pz;
    const double r0 = sqrt(cx * cx + cy * cy + cz * cz);
    double ag[kOrd + 1], a1[kOrd + 1], a2[kOrd + 1], a3[kOrd + 1];
#pragma unroll
    for (int m = 0; m <= kOrd; ++m) ag[m] = a1[m] = a2[m] = a3[m] = 0.0;
    for (int64_t p = qoff[j] + lane; p < qoff[j + 1]; p += 32) {
        const double x = px - qpos[3 * p], y = py - qpos[3 * p + 1], z = pz - qpos[3 * p + 2];
        const double w = qw[p];
        const double r = fmax(sqrt(x * x + y * y + z * z), kEpsP);
        const double ir = 1.0 / r, ir2 = ir * ir, ir3 = ir2 * ir;
        const double dl = r - r0;
        double dpn = 1.0;
#pragma unroll
        for (int m = 0; m <= kOrd; ++m) {
            ag[m] += dpn * ir * inv_fact[m] * w;
            dpn *= dl;
        }
        const double fs = -ir3 * w;
        a1[0] += x * fs;
        a2[0] += y * fs;
        a3[0] += z * fs;
        double dpm = 1.0;
        dpn = dl;
#pragma unroll
        for (int m = 1; m <= kOrd; ++m) {
            const double s = (-dpn * ir3 * inv_fact[m] + dpm * ir2 * inv_fact[m - 1]) * w;
            a1[m] += x * s;
            a2[m] += y * s;
            a3[m] += z * s;
            dpm = dpn;
            dpn *= dl;
        }
    }
#pragma unroll
    for (int m = 0; m <= kOrd; ++m) {
        ag[m] = wsum(ag[m]);
        a1[m] = wsum(a1[m]);
        a2[m] = wsum(a2[m]);
        a3[m] = wsum(a3[m]);
    }
    if (lane == 0)
        for (int m = 0; m <= kOrd; ++m) {
            g[6 * pair + m] = ag[m];
            f[18 * pair + m] = a1[m];
            f[18 * pair + 6 + m] = a2[m];
            f[18 * pair + 12 + m] = a3[m];
        }
}

// ---------------------------------------------------------------------------
// Point-face Green function entries.
// ---------------------------------------------------------------------------
struct PointTables {
    int64_t npt, n;
    int nmed;
    const double *ptpos, *pos, *area;
    const int32_t *pt_med, *face_med;   // (npt), (n, 2)
    const double *k_t;                  // (batch, nmed) complex wavenumbers
    const int64_t *rptr;                // refined point-face pairs, CSR by point
    const int32_t *cols;                //   columns ascending
    const double *g, *f;                // (nref, 6), (nref, 3, 6)
};

__device__ __forceinline__ int64_t find_pair(const PointTables &t, int64_t i, int64_t j) {
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

// G and Gp = dG/d(point) of point i and face j with wavenumber k: the far
// formula G = e^{ikd}/d a_j, Gp = (ik - 1/d)/d^2 (pt_i - pos_j) a_j e^{ikd},
// or for refined pairs sum_n (ik)^n g_n e^{ikd} and the same with f_n
// (greenret_refined.py:727-845).
__device__ __forceinline__ void point_entry(const PointTables &t, cd k, int64_t i, int64_t j,
                                            cd &G, cd Gp[3]) {
    const double x = t.ptpos[3 * i] - t.pos[3 * j];
    const double y = t.ptpos[3 * i + 1] - t.pos[3 * j + 1];
    const double z = t.ptpos[3 * i + 2] - t.pos[3 * j + 2];
    double d = sqrt(x * x + y * y + z * z);
    if (d < kEpsP) d = kEpsP;
    const cd ph = cexpi(k, d);
    const int64_t p = find_pair(t, i, j);
    if (p >= 0) {
        const cd ik = cmk(-k.y, k.x);
        cd pw = cmk(1.0, 0.0), s0 = cmk(0, 0), s1 = s0, s2 = s0, s3 = s0;
        for (int m = 0; m <= kOrd; ++m) {
            s0 = cadd(s0, cscale(pw, t.g[6 * p + m]));
            s1 = cadd(s1, cscale(pw, t.f[18 * p + m]));
            s2 = cadd(s2, cscale(pw, t.f[18 * p + 6 + m]));
            s3 = cadd(s3, cscale(pw, t.f[18 * p + 12 + m]));
            pw = cmul(pw, ik);
        }
        G = cmul(s0, ph);
        Gp[0] = cmul(s1, ph);
        Gp[1] = cmul(s2, ph);
        Gp[2] = cmul(s3, ph);
        return;
    }
    const double a = t.area[j];
    const double inv_d = 1.0 / d, inv_d2 = inv_d * inv_d;
    G = cscale(ph, a * inv_d);
    const cd faux = cmk((-k.y - inv_d) * inv_d2, k.x * inv_d2);
    Gp[0] = cmul(cscale(cscale(faux, x), a), ph);
    Gp[1] = cmul(cscale(cscale(faux, y), a), ph);
    Gp[2] = cmul(cscale(cscale(faux, z), a), ph);
}

// Fields (mode 0) or potentials (mode 1) at the points, one CTA per (point,
// column chunk, wavelength); faces whose side s borders the point's medium
// contribute with the charges / currents of side s:
//   mode 0: e = i k0 sum G h_s - sum Gp sig_s,   h = sum Gp × h_s
//   mode 1: phi = sum G sig_s,                   a = sum G h_s
// sol [b][8][K][n] (sig1, h1 xyz, sig2, h2 xyz); out o1, o2 [b][npt][3][KC]
// (mode 1: o1 = phi [b][npt][KC], o2 = a [b][npt][3][KC]).  With diag > 0
// point i reads only columns [i diag, (i + 1) diag) and KC = diag, else
// KC = K.
constexpr int PG_T = 128;
constexpr int PG_CH = 4;

__global__ void __launch_bounds__(PG_T) point_green_kernel(PointTables t, int mode, int K,
                                                           int diag,
                                                           const double *__restrict__ k0v,
                                                           const cd *__restrict__ sol,
                                                           cd *__restrict__ o1,
                                                           cd *__restrict__ o2) {
    const int64_t i = blockIdx.x;
    const int64_t b = blockIdx.z;
    const int KC = diag > 0 ? diag : K;
    const int c_lo = blockIdx.y * PG_CH;                 // within the point's KC columns
    const int nc = min(PG_CH, KC - c_lo);
    const int col0 = (diag > 0 ? (int)i * diag : 0) + c_lo;
    const int mpt = t.pt_med[i] <= t.nmed ? t.pt_med[i] : 0;
    const cd k = mpt > 0 ? cmk(t.k_t[2 * (b * t.nmed + mpt - 1)], t.k_t[2 * (b * t.nmed + mpt - 1) + 1])
                         : cmk(0, 0);
    const double k0 = k0v[b];
    const int64_t n = t.n;
    const cd *x = sol + b * (int64_t)8 * K * n;
    double acc[PG_CH * 12];
#pragma unroll
    for (int q = 0; q < PG_CH * 12; ++q) acc[q] = 0.0;
    if (mpt > 0 && nc > 0) {
        for (int64_t j = threadIdx.x; j < n; j += PG_T) {
            const int s0 = t.face_med[2 * j] == mpt, s1 = t.face_med[2 * j + 1] == mpt;
            if (!s0 && !s1) continue;
            cd G, Gp[3];
            point_entry(t, k, i, j, G, Gp);
            for (int s = 0; s < 2; ++s) {
                if (!(s == 0 ? s0 : s1)) continue;
                const int base = 4 * s;
#pragma unroll
                for (int c = 0; c < PG_CH; ++c) {
                    if (c >= nc) break;
                    const int col = col0 + c;
                    const cd sg = x[(int64_t)(base * K + col) * n + j];
                    const cd hx = x[(int64_t)((base + 1) * K + col) * n + j];
                    const cd hy = x[(int64_t)((base + 2) * K + col) * n + j];
                    const cd hz = x[(int64_t)((base + 3) * K + col) * n + j];
                    double *A = acc + 12 * c;
                    cd v[6];
                    if (mode == 0) {
                        const cd ikG = cscale(cmk(-G.y, G.x), k0);   // i k0 G
                        v[0] = csub(cmul(ikG, hx), cmul(Gp[0], sg));
                        v[1] = csub(cmul(ikG, hy), cmul(Gp[1], sg));
                        v[2] = csub(cmul(ikG, hz), cmul(Gp[2], sg));
                        v[3] = csub(cmul(Gp[1], hz), cmul(Gp[2], hy));
                        v[4] = csub(cmul(Gp[2], hx), cmul(Gp[0], hz));
                        v[5] = csub(cmul(Gp[0], hy), cmul(Gp[1], hx));
                    } else {
                        v[0] = cmul(G, sg);
                        v[1] = cmul(G, hx);
                        v[2] = cmul(G, hy);
                        v[3] = cmul(G, hz);
                        v[4] = v[5] = cmk(0, 0);
                    }
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        A[2 * q] += v[q].x;
                        A[2 * q + 1] += v[q].y;
                    }
                }
            }
        }
    }
    __shared__ double red[PG_T / 32][PG_CH * 12];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < PG_CH * 12; ++q) {
        const double w = wsum(acc[q]);
        if (lane == 0) red[warp][q] = w;
    }
    __syncthreads();
    if (threadIdx.x < 12 * nc) {
        double s = 0.0;
        for (int w = 0; w < PG_T / 32; ++w) s += red[w][threadIdx.x];
        const int c = threadIdx.x / 12, q = (threadIdx.x % 12) >> 1, re = threadIdx.x & 1;
        const int cc = c_lo + c;                      // column within KC
        double *dst;
        if (mode == 0) {
            cd *base = q < 3 ? o1 : o2;
            const int comp = q < 3 ? q : q - 3;
            dst = reinterpret_cast<double *>(base + ((b * t.npt + i) * 3 + comp) * KC + cc);
        } else {
            if (q >= 4) return;
            dst = q == 0 ? reinterpret_cast<double *>(o1 + (b * t.npt + i) * KC + cc)
                         : reinterpret_cast<double *>(o2 + ((b * t.npt + i) * 3 + q - 1) * KC + cc);
        }
        dst[re] = s;
    }
}

// Entries of the point-face region pair (points, side `side` of the faces):
// G (out [npt][ncol]) or Gp (out [npt][3][ncol]) for face columns
// [c0, c0 + ncol); 0 where the face's side does not border the point's medium.
__global__ void __launch_bounds__(256) point_eval_kernel(PointTables t, int side, int vec,
                                                         int64_t c0, int64_t ncol,
                                                         cd *__restrict__ out) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= t.npt * ncol) return;
    const int64_t i = tid / ncol, jj = tid - i * ncol, j = c0 + jj;
    const int mpt = t.pt_med[i] <= t.nmed ? t.pt_med[i] : 0;
    cd G = cmk(0, 0), Gp[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    if (mpt > 0 && t.face_med[2 * j + side] == mpt) {
        const cd k = cmk(t.k_t[2 * (mpt - 1)], t.k_t[2 * (mpt - 1) + 1]);
        point_entry(t, k, i, j, G, Gp);
    }
    if (vec)
        for (int c = 0; c < 3; ++c) out[(i * 3 + c) * ncol + jj] = Gp[c];
    else
        out[tid] = G;
}

}  // namespace
}  // namespace mnpb

using namespace mnpb;

static int point_tables(PointTables &t, int64_t npt, const double *ptpos, const int32_t *pt_med,
                        int64_t n, const double *pos, const double *area,
                        const int32_t *face_med, int nmed, const double *k_t,
                        const int64_t *rptr, const int32_t *cols, const double *g,
                        const double *f, const char *what) {
    MNPB_REQUIRE(npt > 0 && npt < 65536 && n > 0 && n < (int64_t(1) << 31),
                 "%s: bad sizes npt = %lld, n = %lld", what, (long long)npt, (long long)n);
    MNPB_REQUIRE(nmed >= 1 && nmed <= 64, "%s: nmed must be 1..64", what);
    MNPB_REQUIRE(ptpos && pt_med && pos && area && face_med && k_t && rptr && cols && g && f,
                 "%s: null pointer", what);
    t.npt = npt;
    t.n = n;
    t.nmed = nmed;
    t.ptpos = ptpos;
    t.pos = pos;
    t.area = area;
    t.pt_med = pt_med;
    t.face_med = face_med;
    t.k_t = k_t;
    t.rptr = rptr;
    t.cols = cols;
    t.g = g;
    t.f = f;
    return MNPB_OK;
}

extern "C" int mnpb_dipole_potential(void *stream, int64_t n, int64_t batch, int64_t npt,
                                     int64_t ndip, const double *pos, const double *nvec,
                                     const int32_t *face_med, const double *ptpos,
                                     const int32_t *pt_med, const double *dip, int nmed,
                                     const double *eps, const double *k, const double *k0,
                                     double *pots) {
    clear_error();
    MNPB_REQUIRE(n > 0 && n < (int64_t(1) << 31) && batch > 0 && batch < 65536 && npt > 0 &&
                     npt < 65536 && ndip > 0 && npt * ndip < (int64_t(1) << 31),
                 "dipole_potential: bad sizes");
    MNPB_REQUIRE(nmed >= 1 && nmed <= 64, "dipole_potential: nmed must be 1..64");
    MNPB_REQUIRE(pos && nvec && face_med && ptpos && pt_med && dip && eps && k && k0 && pots,
                 "dipole_potential: null pointer");
    dim3 grid(ceil_div(n, 128), (unsigned)npt, (unsigned)batch);
    dipole_pot_kernel<<<grid, 128, 0, as_stream(stream)>>>(
        (int)n, (int)npt, (int)ndip, pos, nvec, face_med, ptpos, pt_med, dip, nmed, eps, k, k0,
        (cd *)pots);
    MNPB_LAUNCH_CHECK("dipole_pot_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_dipole_field(void *stream, int64_t nobs, int64_t batch, int64_t npt,
                                 int64_t ndip, const double *obs, const int32_t *obs_med,
                                 const double *ptpos, const int32_t *pt_med, const double *dip,
                                 int nmed, const double *eps, const double *k, const double *nb,
                                 double *e, double *h) {
    clear_error();
    MNPB_REQUIRE(nobs > 0 && nobs < (int64_t(1) << 31) && batch > 0 && batch < 65536 &&
                     npt > 0 && npt < 65536 && ndip > 0,
                 "dipole_field: bad sizes");
    MNPB_REQUIRE(nmed >= 1 && nmed <= 64, "dipole_field: nmed must be 1..64");
    MNPB_REQUIRE(obs && obs_med && ptpos && pt_med && dip && eps && k && nb && e && h,
                 "dipole_field: null pointer");
    dim3 grid(ceil_div(nobs, 128), (unsigned)npt, (unsigned)batch);
    dipole_field_kernel<<<grid, 128, 0, as_stream(stream)>>>(
        (int)nobs, (int)npt, (int)ndip, obs, obs_med, ptpos, pt_med, dip, nmed, eps, k, nb,
        (cd *)e, (cd *)h);
    MNPB_LAUNCH_CHECK("dipole_field_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_dipole_stat_field(void *stream, int64_t nobs, int64_t npt, int64_t ndip,
                                      const double *obs, const double *nvec,
                                      const double *ptpos, const double *dip,
                                      const double *eps_pt, double *out) {
    clear_error();
    MNPB_REQUIRE(nobs > 0 && nobs < (int64_t(1) << 31) && npt > 0 && npt < 65536 && ndip > 0 &&
                     ndip < 4096,
                 "dipole_stat_field: bad sizes");
    MNPB_REQUIRE(obs && ptpos && dip && eps_pt && out, "dipole_stat_field: null pointer");
    dim3 grid(ceil_div(nobs, 128), (unsigned)npt);
    dipole_stat_kernel<<<grid, 128, 0, as_stream(stream)>>>((int)nobs, (int)npt, (int)ndip, obs,
                                                            nvec, ptpos, dip, eps_pt, (cd *)out);
    MNPB_LAUNCH_CHECK("dipole_stat_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_dipole_farfield(void *stream, int64_t ndir, int64_t batch, int64_t npt,
                                    int64_t ndip, const double *ptpos, const int8_t *pt_on,
                                    const double *dip, const double *dirs, const double *emb,
                                    double *e, double *h) {
    clear_error();
    MNPB_REQUIRE(ndir > 0 && batch > 0 && batch < 65536 && npt > 0 && ndip > 0 &&
                     npt * ndip < 65536,
                 "dipole_farfield: bad sizes");
    MNPB_REQUIRE(ptpos && pt_on && dip && dirs && emb && e && h, "dipole_farfield: null pointer");
    dim3 grid(ceil_div(ndir, 128), (unsigned)(npt * ndip), (unsigned)batch);
    dipole_farfield_kernel<<<grid, 128, 0, as_stream(stream)>>>(
        (int)ndir, (int)npt, (int)ndip, ptpos, pt_on, dip, dirs, emb, (cd *)e, (cd *)h);
    MNPB_LAUNCH_CHECK("dipole_farfield_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_refine_points(void *stream, int64_t npt, const double *ptpos, int64_t n,
                                  const double *pos, int64_t nref, const int32_t *rows,
                                  const int32_t *cols, const double *qpos, const double *qw,
                                  const int64_t *qoff, double *g, double *f) {
    clear_error();
    MNPB_REQUIRE(npt > 0 && n > 0 && nref >= 0, "refine_points: bad sizes");
    if (nref == 0) return MNPB_OK;
    MNPB_REQUIRE(ptpos && pos && rows && cols && qpos && qw && qoff && g && f,
                 "refine_points: null pointer");
    const int64_t blocks = (nref * 32 + 255) / 256;
    MNPB_REQUIRE(blocks < (int64_t(1) << 31), "refine_points: too many pairs");
    refine_points_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
        ptpos, pos, nref, rows, cols, qpos, qw, qoff, g, f);
    MNPB_LAUNCH_CHECK("refine_points_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_point_green(void *stream, int64_t npt, const double *ptpos,
                                const int32_t *pt_med, int64_t n, const double *pos,
                                const double *area, const int32_t *face_med, int nmed,
                                const double *k, const int64_t *rptr, const int32_t *cols,
                                const double *g, const double *f, int mode, int64_t batch,
                                int64_t K, int64_t diag, const double *k0, const double *sol,
                                double *o1, double *o2) {
    clear_error();
    PointTables t;
    MNPB_TRY(point_tables(t, npt, ptpos, pt_med, n, pos, area, face_med, nmed, k, rptr, cols, g,
                          f, "point_green"));
    MNPB_REQUIRE(mode == 0 || mode == 1, "point_green: mode must be 0 (field) or 1 (potential)");
    MNPB_REQUIRE(batch > 0 && batch < 65536 && K > 0 && K < (int64_t(1) << 24),
                 "point_green: bad batch / K");
    MNPB_REQUIRE(diag >= 0 && (diag == 0 || npt * diag <= K),
                 "point_green: diag = %lld needs npt * diag <= K", (long long)diag);
    MNPB_REQUIRE(k0 && sol && o1 && o2, "point_green: null pointer");
    const int64_t KC = diag > 0 ? diag : K;
    dim3 grid((unsigned)npt, ceil_div(KC, PG_CH), (unsigned)batch);
    MNPB_REQUIRE(grid.y < 65536, "point_green: too many columns");
    point_green_kernel<<<grid, PG_T, 0, as_stream(stream)>>>(t, mode, (int)K, (int)diag, k0,
                                                            (const cd *)sol, (cd *)o1, (cd *)o2);
    MNPB_LAUNCH_CHECK("point_green_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_point_green_eval(void *stream, int64_t npt, const double *ptpos,
                                     const int32_t *pt_med, int64_t n, const double *pos,
                                     const double *area, const int32_t *face_med, int nmed,
                                     const double *k, const int64_t *rptr, const int32_t *cols,
                                     const double *g, const double *f, int side, int vec,
                                     int64_t col_start, int64_t ncol, double *out) {
    clear_error();
    PointTables t;
    MNPB_TRY(point_tables(t, npt, ptpos, pt_med, n, pos, area, face_med, nmed, k, rptr, cols, g,
                          f, "point_green_eval"));
    MNPB_REQUIRE(side == 0 || side == 1, "point_green_eval: side must be 0 or 1");
    MNPB_REQUIRE(col_start >= 0 && ncol >= 0 && col_start + ncol <= n,
                 "point_green_eval: column range outside the faces");
    MNPB_REQUIRE(out, "point_green_eval: null output");
    const int64_t tot = npt * ncol;
    if (tot == 0) return MNPB_OK;
    point_eval_kernel<<<ceil_div(tot, 256), 256, 0, as_stream(stream)>>>(t, side, vec ? 1 : 0,
                                                                         col_start, ncol,
                                                                         (cd *)out);
    MNPB_LAUNCH_CHECK("point_eval_kernel");
    return MNPB_OK;
}
