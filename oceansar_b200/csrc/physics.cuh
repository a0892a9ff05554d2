// Scattering physics evaluated per facet on the device, templated on the arithmetic type
// (double for the drop-in form, float for the mixed form).
//
// * romeiser_facet: the Romeiser & Alpers (1997) composite Bragg RCS of both Bragg lines,
//   oceansar/nrcs/romeiser97.py:252-322 (_rcs_numba) + :324-393 (rcs_numba): tilted local
//   incidence, complex Bragg coefficients, folded directional spectrum (linear
//   interpolation of the omni-directional spectrum on k = 1, 1.1, ... < 2 k0, fill 1
//   outside, times the spreading function) and the bad_ones mask.
// * kodis_facet: the Kodis (1966) stationary-phase specular field, oceansar/nrcs/kodis.py:38-73.
// * ka_facet: the monostatic Kirchhoff-approximation field of a facet, oceansar/nrcs/ka.py:110-284
//   (facet approach and stationary-phase approximation).
#pragma once
#include "common.cuh"

namespace ocs {

enum { POL_VV = 0, POL_HH = 1, POL_DP = 2 };
enum { SPREAD_ELFOUHAILY = 0, SPREAD_COS2S = 1 };

template <typename T> OCS_D T tsqrt(T x);
template <> OCS_D double tsqrt(double x) { return sqrt(x); }
template <> OCS_D float tsqrt(float x) { return sqrtf(x); }
template <typename T> OCS_D T tatan(T x);
template <> OCS_D double tatan(double x) { return atan(x); }
template <> OCS_D float tatan(float x) { return atanf(x); }
template <typename T> OCS_D T tsin(T x);
template <> OCS_D double tsin(double x) { return sin(x); }
template <> OCS_D float tsin(float x) { return sinf(x); }
template <typename T> OCS_D T tcos(T x);
template <> OCS_D double tcos(double x) { return cos(x); }
template <> OCS_D float tcos(float x) { return cosf(x); }
template <typename T> OCS_D T ttanh(T x);
template <> OCS_D double ttanh(double x) { return tanh(x); }
template <> OCS_D float ttanh(float x) { return tanhf(x); }
template <typename T> OCS_D T tpow(T x, T y);
template <> OCS_D double tpow(double x, double y) { return pow(x, y); }
template <> OCS_D float tpow(float x, float y) { return powf(x, y); }
template <typename T> OCS_D T tatan2(T y, T x);
template <> OCS_D double tatan2(double y, double x) { return atan2(y, x); }
template <> OCS_D float tatan2(float y, float x) { return atan2f(y, x); }

template <typename T> OCS_D cplx<T> cdiv(cplx<T> a, cplx<T> b) {
    // Smith's algorithm (the scaling numpy's complex division uses)
    if (fabs(b.re) >= fabs(b.im)) {
        T r = b.im / b.re, den = b.re + b.im * r;
        return {(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    }
    T r = b.re / b.im, den = b.re * r + b.im;
    return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}

// np.angle(np.exp(1j*x)): wrap to (-pi, pi].
template <typename T> OCS_D T wrap_angle(T x) { return tatan2(tsin(x), tcos(x)); }

struct RomeiserParams {
    double k0, d, dx, dy, wind_dir, wind_U;
    int pol;
    int spread;
    // Elfouhaily spreading: Delta(k) = tanh(a0 + ap (cK/cKp)^2.5 + am (cKm/cK)^2.5)
    double ck_p, ck_m, a0, ap, am;
    // omni-directional spectrum table (interp1d, bounds_error=False, fill_value=1)
    const double *tab_k;
    const double *tab_s;
    int tab_n;
    // sea-water permittivity (constants.py:50): eps, sqrt(eps), eps^2
    double eps_re, eps_im, seps_re, seps_im, eps2_re, eps2_im;
};

// scipy interp1d(kind='linear') at x: searchsorted(left), clip to [1, n-1], slope form.
template <typename T> OCS_D T spec_interp(const RomeiserParams &p, T x) {
    const int n = p.tab_n;
    const double xd = (double)x;
    if (!(xd >= p.tab_k[0]) || !(xd <= p.tab_k[n - 1])) {
        if (xd != xd) return (T)xd;                // NaN propagates
        return (T)1;
    }
    int g = (int)((xd - p.tab_k[0]) * 10.0);
    g = g < 0 ? 0 : (g > n - 1 ? n - 1 : g);
    for (int it = 0; it < 4 && g > 0 && p.tab_k[g - 1] >= xd; ++it) --g;
    for (int it = 0; it < 4 && g < n && p.tab_k[g] < xd; ++it) ++g;
    g = g < 1 ? 1 : (g > n - 1 ? n - 1 : g);
    const T x_lo = (T)p.tab_k[g - 1], x_hi = (T)p.tab_k[g];
    const T y_lo = (T)p.tab_s[g - 1], y_hi = (T)p.tab_s[g];
    const T slope = (y_hi - y_lo) / (x_hi - x_lo);
    return slope * (x - x_lo) + y_lo;
}

template <typename T> OCS_D T spread_fn(const RomeiserParams &p, T k, T theta) {
    const T half_pi = (T)1.5707963267948966;
    if (p.spread == SPREAD_COS2S) {
        if (theta < -half_pi || theta > half_pi) return (T)0;
        T c = tcos(theta);
        return c * c / (T)3.141592653589793;
    }
    if (!(theta > -half_pi && theta < half_pi)) return (T)0;
    const T g = (T)9.80665, s_rho = (T)(0.072 / 1000.);
    T ck = tsqrt(g / k + s_rho * k);
    T delta = ttanh((T)p.a0 + (T)p.ap * tpow(ck / (T)p.ck_p, (T)2.5) + (T)p.am * tpow((T)p.ck_m / ck, (T)2.5));
    return ((T)1 + delta * tcos((T)2 * theta)) / (T)3.141592653589793;
}

// RCS of both Bragg lines for the requested polarisations at one facet.
// inc: local nominal incidence; cos_az/sin_az of the ground-projected azimuth angle.
template <typename T>
OCS_D void romeiser_facet(const RomeiserParams &p, T inc, T az, T cos_az, T sin_az, T diffx, T diffy,
                          T rcs_hh[2], T rcs_vv[2]) {
    const T s_p = tatan(cos_az * diffx + sin_az * diffy);
    const T s_t = tatan(-sin_az * diffx + cos_az * diffy);
    const T cos_s_t = tcos(s_t);
    const T cos_s_t_2 = cos_s_t * cos_s_t;
    const T sin_s_t_2 = (T)1 - cos_s_t_2;
    const T sin_ip = tsin(inc - s_p);
    const T cos_ip = tcos(inc - s_p);
    const T cos_ip_2 = cos_ip * cos_ip;
    const T sin_ip_2 = sin_ip * sin_ip;
    const T cos_th = cos_ip * cos_s_t;
    const T sin_th_2 = (T)1 - cos_th * cos_th;
    const cplx<T> eps = {(T)p.eps_re, (T)p.eps_im};
    const cplx<T> seps = {(T)p.seps_re, (T)p.seps_im};
    const cplx<T> eps2 = {(T)p.eps2_re, (T)p.eps2_im};
    cplx<T> q = {cos_th + seps.re, seps.im};
    const cplx<T> b_hh = cdiv(eps, cmul(q, q));
    cplx<T> r = {eps.re * cos_th + seps.re, eps.im * cos_th + seps.im};
    const cplx<T> b_vv = cdiv(cscale(eps2, (T)1 + sin_th_2), cmul(r, r));
    const T w = cos_ip / (tcos(inc) * tcos(s_p));
    const T a = sin_s_t_2 / sin_th_2;
    const T b = sin_ip_2 * cos_s_t_2 / sin_th_2;
    const T kc = (T)p.k0 * cos_th;
    const T kc2 = kc * kc;
    const T F0 = (T)(8 * 3.141592653589793) * (kc2 * kc2);
    const cplx<T> v1 = {b * b_vv.re + a * b_hh.re, b * b_vv.im + a * b_hh.im};
    const cplx<T> h1 = {b * b_hh.re + a * b_vv.re, b * b_hh.im + a * b_vv.im};
    const T T_vv = w * (F0 * (v1.re * v1.re + v1.im * v1.im));
    const T T_hh = w * (F0 * (h1.re * h1.re + h1.im * h1.im));
    T k_b = (T)2 * (T)p.k0 * tsqrt(sin_ip_2 + cos_ip_2 * sin_s_t_2);
    if (k_b > (T)2 * (T)p.k0) k_b = (T)0;
    const T phi_b = az + tatan((cos_ip * tsin(-s_t)) / tsin(inc - s_p));
    const T th0 = wrap_angle(phi_b - (T)p.wind_dir);
    const T th1 = wrap_angle(phi_b + (T)3.141592653589793 - (T)p.wind_dir);
    const T s1 = spec_interp<T>(p, k_b);
    const T sp0 = s1 / k_b * spread_fn<T>(p, k_b, th0);
    const T sp1 = s1 / k_b * spread_fn<T>(p, k_b, th1);
    const T dxv = (T)p.dx, dyv = (T)p.dy;
    const bool bad = (T)4 * sin_ip_2 < (T)(p.d * p.d);
    rcs_vv[0] = bad ? (T)0 : T_vv * sp0 * dxv * dyv;
    rcs_vv[1] = bad ? (T)0 : T_vv * sp1 * dxv * dyv;
    // in DP mode the reference leaves line 0 of hh unmasked (romeiser97.py:391-392)
    rcs_hh[0] = (bad && p.pol == POL_HH) ? (T)0 : T_hh * sp0 * dxv * dyv;
    rcs_hh[1] = bad ? (T)0 : T_hh * sp1 * dxv * dyv;
}

struct KodisParams {
    double k0;
    double R_re, R_im;       // (eps - sqrt eps) / (eps + sqrt eps)
    double hdx, hdy;         // facet half sizes dx/2, dy/2
};

// Specular field E (without the sqrt(4 pi) of sar_raw_nompi.py:394) at one facet.
template <typename T>
OCS_D cplx<T> kodis_facet(const KodisParams &kp, double sr, double sin_inc, double cos_inc, double tan_inc,
                          double cos_az, double sin_az, float diffx, float diffy, float diffxx,
                          float diffyy, float diffxy) {
    // J and its magnitude are float32 products in the reference (the fields are float32)
    float J = __fsub_rn(__fmul_rn(diffxx, diffyy), __fmul_rn(diffxy, diffxy));
    if (J == 0.f) return {(T)0, (T)0};                  // J -> NaN: never stationary
    const float J_abs = fabsf(J);
    double delta_x, delta_y;
    if (sizeof(T) == 8) {
        const double inv_j = (double)(1.f / J_abs);
        const double ty = (double)diffy - tan_inc * sin_az;
        const double tx = (double)diffx - tan_inc * cos_az;
        delta_x = inv_j * ((double)diffxy * ty - (double)diffyy * tx);
        delta_y = inv_j * ((double)diffxy * tx - (double)diffxx * ty);
    } else {
        // mixed form: the stationary-point offsets in float32 (only the facet-window test
        // and the small range offset depend on them)
        const float inv_j = __fdividef(1.0f, J_abs);
        const float ty = diffy - (float)(tan_inc * sin_az);
        const float tx = diffx - (float)(tan_inc * cos_az);
        delta_x = (double)(inv_j * (diffxy * ty - diffyy * tx));
        delta_y = (double)(inv_j * (diffxy * tx - diffxx * ty));
    }
    const double hdx = kp.hdx, hdy = kp.hdy;
    if (!((-hdx < delta_x) && (delta_x < hdx) && (-hdy < delta_y) && (delta_y < hdy)))
        return {(T)0, (T)0};
    const double delta_z = delta_x * diffx + delta_y * diffy;
    const double sr_p2 = sr + (sin_inc * cos_az * delta_x + sin_inc * sin_az * delta_y - cos_inc * delta_z);
    cplx<T> eps;
    if (J > 0.f) eps = {(T)((diffxx > 0.f) - (diffxx < 0.f)), (T)0};
    else eps = {(T)0, (T)1};
    const cplx<T> halfR = {(T)(0.5 * kp.R_re), (T)(0.5 * kp.R_im)};
    const float fac = __fadd_rn(__fadd_rn(__fmul_rn(diffx, diffx), __fmul_rn(diffy, diffy)), 1.f);
    const T sq = (T)sqrtf(J_abs);
    cplx<T> v = cscale(cmul(halfR, eps), (T)fac);
    double ph = (-2.0 * kp.k0) * sr_p2;
    cplx<T> e;
    if (sizeof(T) == 8) {
        double s, c;
        sincos(ph, &s, &c);
        e = {(T)c, (T)s};
    } else {
        float s, c;
        __sincosf((float)reduce_2pi(ph), &s, &c);
        e = {(T)c, (T)s};
    }
    v = cmul(v, e);
    return {v.re / sq, v.im / sq};
}

// Principal square root of a complex number: t = sqrt((|z| + |re|) / 2) on the larger side.
OCS_D c128 csqrt128(c128 z) {
    const double r = hypot(z.re, z.im);
    if (z.re >= 0.0) {
        const double t = sqrt(0.5 * (r + z.re));
        return {t, t == 0.0 ? 0.0 : z.im / (2.0 * t)};
    }
    const double t = sqrt(0.5 * (r - z.re));
    return {fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

OCS_D c128 cmulr(c128 a, double s) { return {dmul(a.re, s), dmul(a.im, s)}; }
OCS_D c128 cmul128(c128 a, c128 b) {
    return {dsub(dmul(a.re, b.re), dmul(a.im, b.im)), dadd(dmul(a.re, b.im), dmul(a.im, b.re))};
}

struct KaParams {
    double k0, dx, dy;
    double K_re, K_im;        // -1j k0 exp(-1j k0 (R_i + R_s)) / ((4 pi)^2 R_i R_s)
    int mode;                 // 0: facet approach, 1: stationary phase
};

// Monostatic Kirchhoff field of one facet (RCSKA.field, ka.py:110-284) for the incident /
// scattered polarisations pol_i, pol_s (0 = h, 1 = v).  st, ct, tt: sin / cos / tan of the
// incidence; sp, cp: sin / cos of the azimuth; (x, y) the facet position.  The float32
// surface derivatives enter as the reference combines them: the normal's norm and
// components, the curvature determinant and its inverse are float32 quantities.
OCS_D c128 ka_facet(const KaParams &kp, int pol_i, int pol_s, double x, double y, double st, double ct,
                    double tt, double sp, double cp, float Dz, float Dx, float Dy, float Dxx, float Dyy,
                    float Dxy) {
    const double hv[2][3] = {{-sp, cp, 0.0}, {-(ct * cp), -(ct * sp), -st}};
    const double *ai = hv[pol_i], *as = hv[pol_s];
    const float nn = sqrtf(fadd(fadd(fmul(Dx, Dx), fmul(Dy, Dy)), 1.f));
    const double n[3] = {(double)__fdiv_rn(-Dx, nn), (double)__fdiv_rn(-Dy, nn), (double)__fdiv_rn(1.f, nn)};
    const double ni[3] = {st * cp, st * sp, -ct};
    const double ns[3] = {-(st * cp), -(st * sp), ct};
    const double q[3] = {kp.k0 * (ns[0] - ni[0]), kp.k0 * (ns[1] - ni[1]), kp.k0 * (ns[2] - ni[2])};
    double t[3] = {ni[1] * n[2] - ni[2] * n[1], ni[2] * n[0] - ni[0] * n[2], ni[0] * n[1] - ni[1] * n[0]};
    const double tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    t[0] /= tn; t[1] /= tn; t[2] /= tn;
    const double d[3] = {ni[1] * t[2] - ni[2] * t[1], ni[2] * t[0] - ni[0] * t[2], ni[0] * t[1] - ni[1] * t[0]};
    const double cos_l = -(n[0] * ni[0] + n[1] * ni[1] + n[2] * ni[2]);
    // Fresnel coefficients, eps = 73 + 18j
    const c128 root = csqrt128({73.0 + cos_l * cos_l - 1.0, 18.0});
    const c128 ec = {73.0 * cos_l, 18.0 * cos_l};
    const c128 r_v = cdiv<double>({ec.re - root.re, ec.im - root.im}, {ec.re + root.re, ec.im + root.im});
    const c128 r_h = cdiv<double>({cos_l - root.re, -root.im}, {cos_l + root.re, root.im});
    const double a_t = ai[0] * t[0] + ai[1] * t[1] + ai[2] * t[2];
    const double a_d = ai[0] * d[0] + ai[1] * d[1] + ai[2] * d[2];
    const double n_ni = -cos_l;
    const double nxt[3] = {n[1] * t[2] - n[2] * t[1], n[2] * t[0] - n[0] * t[2], n[0] * t[1] - n[1] * t[0]};
    const c128 c1 = cmulr({1.0 + r_h.re, r_h.im}, a_t);
    const c128 c2 = cmulr(cmulr({1.0 - r_v.re, -r_v.im}, n_ni), a_d);
    const c128 c3 = cmulr(cmulr({1.0 - r_h.re, -r_h.im}, n_ni), a_t);
    const c128 c4 = cmulr({1.0 + r_v.re, r_v.im}, a_d);
    c128 es[3], hs[3];
    for (int k = 0; k < 3; ++k) {
        es[k] = {c1.re * nxt[k] - c2.re * t[k], c1.im * nxt[k] - c2.im * t[k]};
        hs[k] = {-(c3.re * t[k] + c4.re * nxt[k]), -(c3.im * t[k] + c4.im * nxt[k])};
    }
    // p = a_s . (n_s x (n x E_s - n_s x eta n x H_s))
    c128 u[3];
    for (int k = 0; k < 3; ++k) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        const c128 w = {ns[k1] * hs[k2].re - ns[k2] * hs[k1].re, ns[k1] * hs[k2].im - ns[k2] * hs[k1].im};
        u[k] = {es[k].re - w.re, es[k].im - w.im};
    }
    c128 p = {0.0, 0.0};
    for (int k = 0; k < 3; ++k) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        const c128 z = {ns[k1] * u[k2].re - ns[k2] * u[k1].re, ns[k1] * u[k2].im - ns[k2] * u[k1].im};
        p = {p.re + as[k] * z.re, p.im + as[k] * z.im};
    }
    const c128 K = {kp.K_re, kp.K_im};
    if (kp.mode == 1) {
        const float J = fsub(fmul(Dxx, Dyy), fmul(Dxy, Dxy));
        if (J == 0.f) return {0.0, 0.0};                      // J -> NaN: never stationary
        const float J_abs = fabsf(J);
        const double inv_j = (double)__fdiv_rn(1.f, J_abs);
        const double tsp = dmul(tt, sp), tcp = dmul(tt, cp);
        const double dxv = dmul(inv_j, dsub(dmul((double)Dxy, dsub((double)Dy, tsp)), dmul((double)Dyy, dsub((double)Dx, tcp))));
        const double dyv = dmul(inv_j, dsub(dmul((double)Dxy, dsub((double)Dx, tcp)), dmul((double)Dxx, dsub((double)Dy, tsp))));
        const double hx = 0.5 * kp.dx, hy = 0.5 * kp.dy;
        if (!((-hx < dxv) && (dxv < hx) && (-hy < dyv) && (dyv < hy))) return {0.0, 0.0};
        const double dzv = dadd(dmul(dxv, (double)Dx), dmul(dyv, (double)Dy));
        const c128 eps = (J > 0.f) ? c128{(double)((Dxx > 0.f) - (Dxx < 0.f)), 0.0} : c128{0.0, 1.0};
        c128 e = cmul128(cmul128(eps, p), K);
        e = cmul128(e, cexpi(dadd(dadd(dmul(q[0], dxv), dmul(q[1], dyv)), dmul(q[2], dzv))));
        e = cmulr(cmulr(e, 2.0), 3.141592653589793);
        e = {ddiv(e.re, q[2]), ddiv(e.im, q[2])};
        e = cmulr(e, (double)nn);
        const double sj = (double)sqrtf(J_abs);
        return {ddiv(e.re, sj), ddiv(e.im, sj)};
    }
    // facet approach: I = exp(-i q.r) |n| dx dy sinc((q_x + q_z Diffx) dx/2) sinc((q_y + q_z Diffy) dy/2)
    const double qr = dadd(dadd(dmul(q[0], x), dmul(q[1], y)), dmul(q[2], (double)Dz));
    c128 I = cexpi(-qr);
    I = cmulr(cmulr(cmulr(I, (double)nn), kp.dx), kp.dy);
    I = cmulr(I, np_sinc(ddiv(dmul(dadd(q[0], dmul(q[2], (double)Dx)), kp.dx), 2.0)));
    I = cmulr(I, np_sinc(ddiv(dmul(dadd(q[1], dmul(q[2], (double)Dy)), kp.dy), 2.0)));
    return cmul128(cmul128(K, I), p);
}

}  // namespace ocs
