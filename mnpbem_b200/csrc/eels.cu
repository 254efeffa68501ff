// Electron-beam (EELS) excitation on the GPU: potentials of infinite beams at
// the faces, potentials of beam segments inside particles (charged wires),
// and the beams' own fields (mnpbem/simulation/eels_ret.py,
// mnpbem/simulation/eels_base.py).
//
// Units and conventions follow the reference: beams run along z through the
// impact parameters b_j = (x, y), velocity vel in units of c, beam width w
// regularises the distance (rr = sqrt(x^2 + y^2 + w^2)).
#include "common.cuh"

namespace mnpb {
namespace {

constexpr int LGL_N = 11;      // Legendre-Gauss-Lobatto nodes of the wire integral

struct LGL {
    double x[LGL_N], w[LGL_N];
};

// Modified Bessel functions K0(z), K1(z) for complex z with Re z > 0.
// Method: the integral representation K_nu(z) = int_0^inf exp(-z cosh t)
// cosh(nu t) dt (Abramowitz & Stegun 9.6.24) evaluated by the trapezoidal
// rule, which converges geometrically for integrands analytic in a strip
// (Trefethen & Weideman, SIAM Review 56, 2014).  The integrand is analytic
// for |Im t| < pi/2 - |arg z| and, written as e^{-z} exp(-z (cosh t - 1)),
// bounded there by exp(Re z y^2 / 2); the step
//   h = min(0.1, 0.4 / sqrt|z|, 2 pi (pi/2 - |arg z|) / 48)
// keeps the discretisation error below ~1e-15 relative for |arg z| <= 1 and
// ~1e-12 at |arg z| = 1.2 (checked against AMOS through scipy.special.kv over
// 1e-5 <= |z| <= 300).  cosh t - 1 = 2 sinh^2(t/2) avoids cancellation; the
// sum stops once Re z (cosh t - 1) > 40 (terms below e^-40 of the first).
__device__ void bessel_k01(cd z, cd &k0, cd &k1) {
    const double az = sqrt(z.x * z.x + z.y * z.y);
    if (!(z.x > 0.0) || !(az > 0.0)) {
        k0 = k1 = cmk(nan(""), nan(""));
        return;
    }
    const double d = fmax(1.5707963267948966 - fabs(atan2(z.y, z.x)), 0.2);
    const double h = fmin(fmin(0.1, 0.4 / sqrt(az)), 6.283185307179586 * d / 48.0);
    double s0r = 0.5, s0i = 0.0, s1r = 0.5, s1i = 0.0;
    for (int m = 1; m < 8192; ++m) {
        const double sh = sinh(0.5 * m * h);
        const double c1 = 2.0 * sh * sh;             // cosh t - 1
        if (z.x * c1 > 40.0) break;
        double sn, cs;
        sincos(-z.y * c1, &sn, &cs);
        const double mag = exp(-z.x * c1);
        const double er = mag * cs, ei = mag * sn;    // exp(-z c1)
        s0r += er;
        s0i += ei;
        s1r += er * (1.0 + c1);
        s1i += ei * (1.0 + c1);
    }
    double sn, cs;
    sincos(-z.y, &sn, &cs);
    const cd ez = cscale(cmk(cs, sn), exp(-z.x) * h);   // h e^{-z}
    k0 = cmul(ez, cmk(s0r, s0i));
    k1 = cmul(ez, cmk(s1r, s1i));
}

// phi, phip of the infinite beam through b at face point r with normal nv
// (eels_base.py:315-416, potinfty):
//   phi  = -2/vel e^{iqz} K0(q rr / gamma)
//   phip = -2/vel e^{iqz} q (i K0 n_z - K1 / gamma (x n_x + y n_y) / rr)
__device__ __forceinline__ void beam_pot(const double *r, const double *nv, double bx,
                                         double by, double width, double vel, double q,
                                         cd igam, cd &phi, cd &phip) {
    const double x = r[0] - bx, y = r[1] - by, z = r[2];
    const double rp = sqrt(x * x + y * y);
    const double rr = sqrt(rp * rp + width * width);
    cd K0, K1;
    bessel_k01(cscale(igam, q * rr), K0, K1);
    double sn, cs;
    sincos(q * z, &sn, &cs);
    const cd e = cscale(cmk(cs, sn), -2.0 / vel);
    phi = cmul(e, K0);
    const cd t = csub(cmk(-K0.y * nv[2], K0.x * nv[2]),
                      cscale(cmul(K1, igam), (x * nv[0] + y * nv[1]) / rr));
    phip = cmul(cscale(e, q), t);
}

// Potential of a charged wire from z0 to z1 along the beam through b at
// distance rr and height z (eels_base.py:713-783, potwire): with
// u = sinh-type substitution v = log(s + sqrt(rr^2 + s^2)),
//   I  = (v1 - v0)/2 e^{iqz} sum_g w_g f_g,  f_g = exp(i (q u_g + k R_g)),
//   Ir = (v1 - v0)/2 e^{iqz} sum_g w_g rr (ik/R_g - 1/R_g^2) f_g,
//   Iz = -(v1 - v0)/2 e^{iqz} sum_g w_g u_g (ik/R_g - 1/R_g^2) f_g,
// R_g = sqrt(rr^2 + u_g^2).  The derivatives are formed only with DERIV.
template <bool DERIV>
__device__ __forceinline__ void wire_pot(double rr, double z, double q, cd k, double z0,
                                         double z1, const LGL &g, cd &I, cd &Ir, cd &Iz) {
    const double s0 = z0 - z, s1 = z1 - z;
    const double v0 = log(s0 + sqrt(rr * rr + s0 * s0));
    const double v1 = log(s1 + sqrt(rr * rr + s1 * s1));
    cd acc = cmk(0.0, 0.0), accr = acc, accz = acc;
    for (int a = 0; a < LGL_N; ++a) {
        const double v = 0.5 * ((1.0 - g.x[a]) * v0 + (1.0 + g.x[a]) * v1);
        const double u = 0.5 * (exp(v) - rr * rr * exp(-v));
        const double R = sqrt(rr * rr + u * u);
        // exp(i (q u + k R)) with complex k
        const double ph = q * u + k.x * R;
        double sn, cs;
        sincos(ph, &sn, &cs);
        const double m = exp(-k.y * R) * g.w[a];
        const cd f = cmk(m * cs, m * sn);
        acc = cadd(acc, f);
        if (DERIV) {
            const double iR = 1.0 / R;
            const cd d = cmul(cmk(-k.y * iR - iR * iR, k.x * iR), f);   // (ik/R - 1/R^2) f
            accr = cadd(accr, cscale(d, rr));
            accz = csub(accz, cscale(d, u));
        }
    }
    double sn, cs;
    sincos(q * z, &sn, &cs);
    const cd pre = cscale(cmk(cs, sn), 0.5 * (v1 - v0));
    I = cmul(acc, pre);
    if (DERIV) {
        Ir = cmul(accr, pre);
        Iz = cmul(accz, pre);
    }
}

struct BeamFaces {
    int n, nimp;
    const double *pos, *nvec, *area;
    const double *impact;            // (nimp, 2)
    const int8_t *indquad;           // (n, nimp): integrate over the face
    const double *qpos, *qw;         // face quadrature points, sorted by face
    const int64_t *qoff;             // (n + 1)
    double width, vel;
};

// potinfty at face i for impact j: centroid value, or the face-quadrature
// average (weights / area) where indquad is set.
__device__ void beam_pot_face(const BeamFaces &t, int i, int j, double q, cd igam, cd &phi,
                              cd &phip) {
    const double bx = t.impact[2 * j], by = t.impact[2 * j + 1];
    const double *nv = t.nvec + 3 * i;
    if (!t.indquad[(int64_t)i * t.nimp + j]) {
        beam_pot(t.pos + 3 * i, nv, bx, by, t.width, t.vel, q, igam, phi, phip);
        return;
    }
    phi = phip = cmk(0.0, 0.0);
    const double ia = 1.0 / t.area[i];
    for (int64_t p = t.qoff[i]; p < t.qoff[i + 1]; ++p) {
        cd a, b;
        beam_pot(t.qpos + 3 * p, nv, bx, by, t.width, t.vel, q, igam, a, b);
        const double w = t.qw[p] * ia;
        phi = cadd(phi, cscale(a, w));
        phip = cadd(phip, cscale(b, w));
    }
}

// Excitation of the BEM solver (eels_ret.py:149-294): face i, side s with
// medium m gets the infinite-beam potential in medium m (gamma_m) of every
// impact j with beam_in[m][j] set, provided med_on[m]:
//   phi_s = phi / eps_m, phi'_s = phip / eps_m, a_s = vel z^ phi, a'_s = vel z^ phip.
// pots [b][16][nimp][n].
__global__ void __launch_bounds__(128) eels_potential_kernel(
    BeamFaces t, const int32_t *__restrict__ face_med, int nmed,
    const int8_t *__restrict__ med_on, const int8_t *__restrict__ beam_in,
    const double *__restrict__ qv, const double *__restrict__ eps_t,
    const double *__restrict__ igam_t, cd *__restrict__ pots) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int64_t b = blockIdx.z;
    if (i >= t.n) return;
    const int K = t.nimp, n = t.n;
    cd *out = pots + b * (int64_t)16 * K * n;
    auto P = [&](int comp) -> cd & { return out[(int64_t)(comp * K + j) * n + i]; };
    for (int s = 0; s < 2; ++s) {
        const int base = 8 * s;
        const int m = face_med[2 * i + s];
        for (int c = 0; c < 8; ++c) P(base + c) = cmk(0.0, 0.0);
        if (m < 1 || m > nmed || !med_on[m - 1] || !beam_in[(int64_t)(m - 1) * K + j]) continue;
        const int64_t e = b * nmed + (m - 1);
        const cd ieps = crcp(cmk(eps_t[2 * e], eps_t[2 * e + 1]));
        const cd igam = cmk(igam_t[2 * e], igam_t[2 * e + 1]);
        cd phi, phip;
        beam_pot_face(t, i, j, qv[b], igam, phi, phip);
        P(base + 0) = cmul(phi, ieps);
        P(base + 1) = cmul(phip, ieps);
        P(base + 4) = cscale(phi, t.vel);        // a_z
        P(base + 7) = cscale(phip, t.vel);       // a'_z
    }
}

// Raw infinite-beam potentials phi, phip (nimp, n) of one wavelength and one
// medium for faces with face_on set (0 elsewhere).
__global__ void __launch_bounds__(128) eels_infty_kernel(BeamFaces t,
                                                         const int8_t *__restrict__ face_on,
                                                         double q, cd igam,
                                                         cd *__restrict__ phi,
                                                         cd *__restrict__ phip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= t.n) return;
    cd a = cmk(0.0, 0.0), b = a;
    if (face_on[i]) beam_pot_face(t, i, j, q, igam, a, b);
    phi[(int64_t)j * t.n + i] = a;
    phip[(int64_t)j * t.n + i] = b;
}

// Wire potentials of beam segments inside particles (eels_base.py:418-523,
// potinside): segment c of impact imp[c] from z0 to z1,
//   phi  = -1/vel I(rr, z),
//   phip = -1/vel (Iz n_z + Ir (x n_x + y n_y) / rr)      (DERIV only),
// face-quadrature averages where indquad[i, imp[c]]; out (nseg, n), 0 for
// faces without face_on.
template <bool DERIV>
__global__ void __launch_bounds__(128) eels_wire_kernel(BeamFaces t,
                                                        const int8_t *__restrict__ face_on,
                                                        int nseg, const double *__restrict__ seg,
                                                        const int32_t *__restrict__ seg_imp,
                                                        double q, cd k, LGL g,
                                                        cd *__restrict__ phi,
                                                        cd *__restrict__ phip) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (i >= t.n) return;
    cd acc = cmk(0.0, 0.0), accp = acc;
    if (face_on[i]) {
        const int j = seg_imp[c];
        const double bx = t.impact[2 * j], by = t.impact[2 * j + 1];
        const double z0 = seg[2 * c], z1 = seg[2 * c + 1];
        const double *nv = t.nvec + 3 * i;
        auto one = [&](const double *r, double w) {
            const double x = r[0] - bx, y = r[1] - by;
            const double rp = sqrt(x * x + y * y);
            const double rr = sqrt(rp * rp + t.width * t.width);
            cd I, Ir, Iz;
            wire_pot<DERIV>(rr, r[2], q, k, z0, z1, g, I, Ir, Iz);
            acc = cadd(acc, cscale(I, w));
            if (DERIV)
                accp = cadd(accp, cscale(cadd(cscale(Iz, nv[2]),
                                              cscale(Ir, (x * nv[0] + y * nv[1]) / rr)), w));
        };
        if (!t.indquad[(int64_t)i * t.nimp + j]) {
            one(t.pos + 3 * i, 1.0);
        } else {
            const double ia = 1.0 / t.area[i];
            for (int64_t p = t.qoff[i]; p < t.qoff[i + 1]; ++p)
                one(t.qpos + 3 * p, t.qw[p] * ia);
        }
        acc = cscale(acc, -1.0 / t.vel);
        accp = cscale(accp, -1.0 / t.vel);
    }
    phi[(int64_t)c * t.n + i] = acc;
    if (DERIV) phip[(int64_t)c * t.n + i] = accp;
}

// Fields of the beams at observation points in medium med_i (eels_ret.py:
// 506-637, Garcia de Abajo RMP 82, 209, Eqs. 5-6), beams of impact j in medium
// m where beam_in[m][j]:
//   q = k / (vel sqrt(eps)), gamma, K0/K1 of q r / gamma, fac = 2 q/(vel gamma) e^{iqz}
//   e = (-fac/eps K1 x^, -fac/eps K1 y^, i fac/eps K0 / gamma),
//   h = (vel fac K1 y^, -vel fac K1 x^, 0);  out e, h (nobs, 3, nimp).
__global__ void __launch_bounds__(128) eels_field_kernel(
    int nobs, int nimp, const double *__restrict__ obs, const int32_t *__restrict__ med,
    int nmed, const int8_t *__restrict__ beam_in, const double *__restrict__ impact,
    double width, double vel, const double *__restrict__ mtab, cd *__restrict__ e_out,
    cd *__restrict__ h_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= nobs) return;
    cd e[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)}, h[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    const int m = med[i];
    if (m >= 1 && m <= nmed && beam_in[(int64_t)(m - 1) * nimp + j]) {
        // mtab per medium: eps, q, 1/gamma (complex)
        const double *mt = mtab + 6 * (m - 1);
        const cd eps = cmk(mt[0], mt[1]), q = cmk(mt[2], mt[3]), igam = cmk(mt[4], mt[5]);
        const double x = obs[3 * i] - impact[2 * j], y = obs[3 * i + 1] - impact[2 * j + 1];
        const double z = obs[3 * i + 2];
        const double r = sqrt(x * x + y * y + width * width);
        const double xh = x / r, yh = y / r;
        cd K0, K1;
        bessel_k01(cscale(cmul(q, igam), r), K0, K1);
        // 2 q / (vel gamma) exp(i q z)
        const cd fac = cmul(cscale(cmul(q, igam), 2.0 / vel), cexpi(q, z));
        const cd fe = cmul(fac, crcp(eps));
        e[0] = cscale(cmul(fe, K1), -xh);
        e[1] = cscale(cmul(fe, K1), -yh);
        const cd t = cmul(cmul(fe, K0), igam);
        e[2] = cmk(-t.y, t.x);                        // i t
        h[0] = cscale(cmul(fac, K1), vel * yh);
        h[1] = cscale(cmul(fac, K1), -vel * xh);
    }
    for (int c = 0; c < 3; ++c) {
        e_out[((int64_t)i * 3 + c) * nimp + j] = e[c];
        h_out[((int64_t)i * 3 + c) * nimp + j] = h[c];
    }
}

}  // namespace
}  // namespace mnpb

using namespace mnpb;

static int beam_faces(BeamFaces &t, int64_t n, int64_t nimp, const double *pos,
                      const double *nvec, const double *area, const double *impact,
                      const int8_t *indquad, const double *qpos, const double *qw,
                      const int64_t *qoff, double width, double vel, const char *what) {
    MNPB_REQUIRE(n > 0 && n < (int64_t(1) << 31) && nimp > 0 && nimp < 65536,
                 "%s: bad sizes n = %lld, nimp = %lld", what, (long long)n, (long long)nimp);
    MNPB_REQUIRE(pos && nvec && area && impact && indquad && qpos && qw && qoff,
                 "%s: null pointer", what);
    MNPB_REQUIRE(width > 0.0 && vel > 0.0 && vel < 1.0, "%s: need width > 0 and 0 < vel < 1",
                 what);
    t.n = (int)n;
    t.nimp = (int)nimp;
    t.pos = pos;
    t.nvec = nvec;
    t.area = area;
    t.impact = impact;
    t.indquad = indquad;
    t.qpos = qpos;
    t.qw = qw;
    t.qoff = qoff;
    t.width = width;
    t.vel = vel;
    return MNPB_OK;
}

extern "C" int mnpb_eels_potential(void *stream, int64_t n, int64_t batch, int64_t nimp,
                                   const double *pos, const double *nvec, const double *area,
                                   const int32_t *face_med, int nmed, const int8_t *med_on,
                                   const int8_t *beam_in, const double *impact,
                                   const int8_t *indquad, const double *qpos, const double *qw,
                                   const int64_t *qoff, double width, double vel,
                                   const double *q, const double *eps, const double *igam,
                                   double *pots) {
    clear_error();
    BeamFaces t;
    MNPB_TRY(beam_faces(t, n, nimp, pos, nvec, area, impact, indquad, qpos, qw, qoff, width, vel,
                        "eels_potential"));
    MNPB_REQUIRE(batch > 0 && batch < 65536, "eels_potential: bad batch");
    MNPB_REQUIRE(nmed >= 1 && nmed <= 64, "eels_potential: nmed must be 1..64");
    MNPB_REQUIRE(face_med && med_on && beam_in && q && eps && igam && pots,
                 "eels_potential: null pointer");
    dim3 grid(ceil_div(n, 128), (unsigned)nimp, (unsigned)batch);
    eels_potential_kernel<<<grid, 128, 0, as_stream(stream)>>>(t, face_med, nmed, med_on,
                                                               beam_in, q, eps, igam,
                                                               (cd *)pots);
    MNPB_LAUNCH_CHECK("eels_potential_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_eels_infty(void *stream, int64_t n, int64_t nimp, const double *pos,
                               const double *nvec, const double *area, const int8_t *face_on,
                               const double *impact, const int8_t *indquad, const double *qpos,
                               const double *qw, const int64_t *qoff, double width, double vel,
                               double q, double igam_re, double igam_im, double *phi,
                               double *phip) {
    clear_error();
    BeamFaces t;
    MNPB_TRY(beam_faces(t, n, nimp, pos, nvec, area, impact, indquad, qpos, qw, qoff, width, vel,
                        "eels_infty"));
    MNPB_REQUIRE(face_on && phi && phip, "eels_infty: null pointer");
    dim3 grid(ceil_div(n, 128), (unsigned)nimp);
    eels_infty_kernel<<<grid, 128, 0, as_stream(stream)>>>(t, face_on, q, cmk(igam_re, igam_im),
                                                           (cd *)phi, (cd *)phip);
    MNPB_LAUNCH_CHECK("eels_infty_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_eels_wire(void *stream, int64_t n, int64_t nimp, const double *pos,
                              const double *nvec, const double *area, const int8_t *face_on,
                              const double *impact, const int8_t *indquad, const double *qpos,
                              const double *qw, const int64_t *qoff, double width, double vel,
                              int64_t nseg, const double *seg, const int32_t *seg_imp, double q,
                              double k_re, double k_im, const double *lgl_x,
                              const double *lgl_w, double *phi, double *phip) {
    clear_error();
    BeamFaces t;
    MNPB_TRY(beam_faces(t, n, nimp, pos, nvec, area, impact, indquad, qpos, qw, qoff, width, vel,
                        "eels_wire"));
    MNPB_REQUIRE(nseg > 0 && nseg < 65536, "eels_wire: bad nseg");
    MNPB_REQUIRE(face_on && seg && seg_imp && lgl_x && lgl_w && phi, "eels_wire: null pointer");
    LGL g;
    for (int a = 0; a < LGL_N; ++a) {
        g.x[a] = lgl_x[a];
        g.w[a] = lgl_w[a];
    }
    dim3 grid(ceil_div(n, 128), (unsigned)nseg);
    if (phip)
        eels_wire_kernel<true><<<grid, 128, 0, as_stream(stream)>>>(
            t, face_on, (int)nseg, seg, seg_imp, q, cmk(k_re, k_im), g, (cd *)phi, (cd *)phip);
    else
        eels_wire_kernel<false><<<grid, 128, 0, as_stream(stream)>>>(
            t, face_on, (int)nseg, seg, seg_imp, q, cmk(k_re, k_im), g, (cd *)phi, nullptr);
    MNPB_LAUNCH_CHECK("eels_wire_kernel");
    return MNPB_OK;
}

extern "C" int mnpb_eels_field(void *stream, int64_t nobs, int64_t nimp, const double *obs,
                               const int32_t *obs_med, int nmed, const int8_t *beam_in,
                               const double *impact, double width, double vel,
                               const double *mtab, double *e, double *h) {
    clear_error();
    MNPB_REQUIRE(nobs > 0 && nobs < (int64_t(1) << 31) && nimp > 0 && nimp < 65536,
                 "eels_field: bad sizes");
    MNPB_REQUIRE(nmed >= 1 && nmed <= 64, "eels_field: nmed must be 1..64");
    MNPB_REQUIRE(width > 0.0 && vel > 0.0 && vel < 1.0,
                 "eels_field: need width > 0 and 0 < vel < 1");
    MNPB_REQUIRE(obs && obs_med && beam_in && impact && mtab && e && h,
                 "eels_field: null pointer");
    dim3 grid(ceil_div(nobs, 128), (unsigned)nimp);
    eels_field_kernel<<<grid, 128, 0, as_stream(stream)>>>((int)nobs, (int)nimp, obs, obs_med,
                                                           nmed, beam_in, impact, width, vel,
                                                           mtab, (cd *)e, (cd *)h);
    MNPB_LAUNCH_CHECK("eels_field_kernel");
    return MNPB_OK;
}
