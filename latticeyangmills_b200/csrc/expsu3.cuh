// e^{iQ} for a Hermitian traceless 3x3 Q by the Cayley-Hamilton theorem
// (Morningstar & Peardon, Phys. Rev. D 69 (2004) 054501, eqs. 23-34) — the
// method of the reference's exp(const SU3&) (src/Math/su3.cpp:96-183):
//
//   c0 = det Q = tr(Q^3)/3,  c1 = tr(Q^2)/2,  c0max = 2 (c1/3)^{3/2}
//   theta = acos(c0/c0max),  u = sqrt(c1/3) cos(theta/3),  w = sqrt(c1) sin(theta/3)
//   h0 = (u^2 - w^2) e^{2iu} + e^{-iu} [8u^2 cos w + 2iu (3u^2 + w^2) xi(w)]
//   h1 = 2u e^{2iu} - e^{-iu} [2u cos w - i (3u^2 - w^2) xi(w)]
//   h2 = e^{2iu} - e^{-iu} [cos w + 3iu xi(w)]
//   f_j = h_j / (9u^2 - w^2),   e^{iQ} = f0 + f1 Q + f2 Q^2
//
// with c0 < 0 handled by f_j(-c0) = (-1)^j conj(f_j(c0)) and xi(w) = sin(w)/w
// replaced by its series for |w| < 0.05, both as the reference does.
//
// Deliberate differences from the reference, all where it returns NaN:
//   * c0/c0max is clamped to 1 (rounding can push it above 1 for a doubly
//     degenerate spectrum, where the reference's acos gives NaN);
//   * c1 below a tiny threshold (Q = 0, e.g. a cold field) uses the series
//     1 + iQ - Q^2/2, where the reference computes 0/0.
// tr(Q^3)/3 is evaluated as det Q (equal for traceless Q) and Q^2 from its six
// independent entries; both agree with the reference to rounding.
//
// For small Q (c1 <= YM_SERIES_C1, which holds for every link of a flow at
// eps <= 0.02) the coefficients f_j come instead from the truncated power
// series of e^{iQ} reduced by the same Cayley-Hamilton identity (ch_series):
// exact to the working precision, with no acos / sincos / sqrt / division.
// The result equals the closed form to rounding; the closed form remains for
// larger Q.
#pragma once
#include "su3.cuh"

namespace ym {

// e^{iQ} = (1 + f0m1) + f1 Q + f2 Q^2.  The constant coefficient is kept as
// f0 - 1, so that e^{iQ} - 1 (small for small Q) is formed without rounding a
// 1 into it: an FP32 link update U + (e^{iQ} - 1) U then carries only the
// rounding of the stored link, not that of e^{iQ}'s entries near 1, which
// otherwise drifts the FP32 flow systematically (t^2 E about 1e-6 off at t = 2
// with reunitarisation every 10 steps).
template <class S>
struct ChCoef {
    Cx<S> f0m1, f1, f2;
};

template <class S>
__device__ __forceinline__ S ch_small_c1();
template <>
__device__ __forceinline__ double ch_small_c1<double>() { return 1e-60; }
template <>
__device__ __forceinline__ float ch_small_c1<float>() { return 1e-20f; }

// The same coefficients from the power series of e^{iQ}, for small Q.  By the
// Cayley-Hamilton theorem Q^3 = c1 Q + c0, so every power reduces to
// Q^n = A_n + B_n Q + C_n Q^2 with the real recursion
//   A_{n+1} = c0 C_n,   B_{n+1} = A_n + c1 C_n,   C_{n+1} = B_n,
// and f_j = sum_n i^n {A,B,C}_n / n!.  Truncating after Q^N is truncating
// the series of e^{iQ} itself: the error is below rho^{N+1}/(N+1)! e^rho with
// rho the largest |eigenvalue| of Q, rho^2 <= 4 c1 / 3.  No transcendental
// function, no division and no cancellation: every term is a small correction
// to (1, i, -1/2), and f0 - 1 is the sum of the terms alone.
template <class S, int N>
__device__ __forceinline__ ChCoef<S> ch_series(S c0, S c1) {
    ChCoef<S> f;
    f.f0m1 = cx(S(0), S(0));
    f.f1 = cx(S(0), S(1));
    f.f2 = cx(S(-0.5), S(0));
    S a = S(0), b = S(0), c = S(0.5);  // A_2/2!, B_2/2!, C_2/2!
#pragma unroll
    for (int n = 3; n <= N; n++) {
        const S inv = S(1.0 / n);
        const S na = c0 * c * inv;
        const S nb = fma(c1, c, a) * inv;
        const S nc = b * inv;
        a = na;
        b = nb;
        c = nc;
        switch (n & 3) {  // i^n
            case 0: f.f0m1.re += a; f.f1.re += b; f.f2.re += c; break;
            case 1: f.f0m1.im += a; f.f1.im += b; f.f2.im += c; break;
            case 2: f.f0m1.re -= a; f.f1.re -= b; f.f2.re -= c; break;
            default: f.f0m1.im -= a; f.f1.im -= b; f.f2.im -= c; break;
        }
    }
    return f;
}

// Where the series replaces the closed form: c1 <= YM_SERIES_C1, i.e. every
// eigenvalue of Q within rho <= sqrt(4 YM_SERIES_C1 / 3) = 0.163 of zero.  The
// flow stays far inside it (eps Z at eps = 0.02 has c1 <= 0.011 on the
// benchmark fields, Haar-mixed included).  Terms: FP64 up to Q^11 (truncation
// below 0.163^12/12! = 7e-19), FP32 up to Q^6 (below 0.163^7/7! = 2e-9).
#define YM_SERIES_C1 0.02
template <class S>
struct SeriesTerms;
template <>
struct SeriesTerms<double> {
    static constexpr int value = 11;
};
template <>
struct SeriesTerms<float> {
    static constexpr int value = 6;
};

// Cayley-Hamilton coefficients from c0 = det Q and c1 = tr(Q^2)/2, in type S.
template <class S>
__device__ __forceinline__ ChCoef<S> ch_coefficients(S c0, S c1) {
    ChCoef<S> f;
    if (!(c1 > ch_small_c1<S>())) {  // also catches NaN c1: falls to the series
        f.f0m1 = cx(S(0), S(0));
        f.f1 = cx(S(0), S(1));
        f.f2 = cx(S(-0.5), S(0));
        return f;
    }
    const bool neg = c0 < S(0);
    if (neg) c0 = -c0;
    const S inv_sqrt3 = S(0.57735026918962576451);
    const S c1sqrt = sqrt(c1);
    const S c0max = c1 * c1sqrt * inv_sqrt3 * S(2.0 / 3.0);
    S x = c0 / c0max;
    x = x > S(1) ? S(1) : x;
    const S theta = acos(x);
    S st, ct;
    sincos(theta * S(1.0 / 3.0), &st, &ct);
    const S w = c1sqrt * st;
    const S u = c1sqrt * inv_sqrt3 * ct;
    const S u2 = u * u, w2 = w * w;
    S sw, cw;
    sincos(w, &sw, &cw);
    const S xi = fabs(w) < S(0.05) ? S(1) - w2 / S(6) * (S(1) - w2 / S(20) * (S(1) - w2 / S(42))) : sw / w;
    S su, cu;
    sincos(u, &su, &cu);
    const S cmu = cu, smu = -su;  // e^{-iu}
    const S c2u = cmu * cmu - smu * smu, s2u = S(-2) * cmu * smu;  // e^{2iu}
    const S cwcmu = cw * cmu, cwsmu = cw * smu, xicmu = xi * cmu, xismu = xi * smu;
    S h0r = (u2 - w2) * c2u + S(8) * u2 * cwcmu - S(2) * u * (S(3) * u2 + w2) * xismu;
    S h0i = (u2 - w2) * s2u + S(8) * u2 * cwsmu + S(2) * u * (S(3) * u2 + w2) * xicmu;
    S h1r = S(2) * u * c2u - S(2) * u * cwcmu - (S(3) * u2 - w2) * xismu;
    S h1i = S(2) * u * s2u - S(2) * u * cwsmu + (S(3) * u2 - w2) * xicmu;
    S h2r = c2u - cwcmu + S(3) * u * xismu;
    S h2i = s2u - cwsmu - S(3) * u * xicmu;
    if (neg) {
        h0i = -h0i;
        h1r = -h1r;
        h2i = -h2i;
    }
    const S norm = S(1) / (S(9) * u2 - w2);
    f.f0m1 = cx(h0r * norm - S(1), h0i * norm);
    f.f1 = cx(h1r * norm, h1i * norm);
    f.f2 = cx(h2r * norm, h2i * norm);
    return f;
}

template <class R>
struct QSquared {  // Q^2, Hermitian: real diagonal and the upper triangle
    R a00, a11, a22;
    Cx<R> a01, a02, a12;
};

template <class R>
__device__ __forceinline__ QSquared<R> q_squared(const Herm8<R>& q, R q22) {
    QSquared<R> s;
    const R n01 = q.z01.re * q.z01.re + q.z01.im * q.z01.im;
    const R n02 = q.z02.re * q.z02.re + q.z02.im * q.z02.im;
    const R n12 = q.z12.re * q.z12.re + q.z12.im * q.z12.im;
    s.a00 = q.d0 * q.d0 + n01 + n02;
    s.a11 = q.d1 * q.d1 + n01 + n12;
    s.a22 = q22 * q22 + n02 + n12;
    // (Q^2)_01 = q00 q01 + q01 q11 + q02 conj(q12)
    s.a01 = cx((q.d0 + q.d1) * q.z01.re + q.z02.re * q.z12.re + q.z02.im * q.z12.im,
               (q.d0 + q.d1) * q.z01.im + q.z02.im * q.z12.re - q.z02.re * q.z12.im);
    // (Q^2)_02 = q00 q02 + q01 q12 + q02 q22
    s.a02 = cx((q.d0 + q22) * q.z02.re + q.z01.re * q.z12.re - q.z01.im * q.z12.im,
               (q.d0 + q22) * q.z02.im + q.z01.re * q.z12.im + q.z01.im * q.z12.re);
    // (Q^2)_12 = conj(q01) q02 + q11 q12 + q12 q22
    s.a12 = cx((q.d1 + q22) * q.z12.re + q.z01.re * q.z02.re + q.z01.im * q.z02.im,
               (q.d1 + q22) * q.z12.im + q.z01.re * q.z02.im - q.z01.im * q.z02.re);
    return s;
}

// det Q for Hermitian Q: q00 q11 q22 + 2 Re(q01 q12 conj(q02)) - q00|q12|^2 - q11|q02|^2 - q22|q01|^2
template <class S, class R>
__device__ __forceinline__ S herm_det(const Herm8<R>& q, R q22r) {
    const S a = S(q.d0), b = S(q.d1), c = S(q22r);
    const S xr = S(q.z01.re), xi = S(q.z01.im), yr = S(q.z02.re), yi = S(q.z02.im);
    const S zr = S(q.z12.re), zi = S(q.z12.im);
    const S pr = xr * zr - xi * zi, pi = xr * zi + xi * zr;  // q01 q12
    const S re3 = pr * yr + pi * yi;                          // Re(q01 q12 conj(q02))
    return a * b * c + S(2) * re3 - a * (zr * zr + zi * zi) - b * (yr * yr + yi * yi) - c * (xr * xr + xi * xi);
}

template <class S, class R>
__device__ __forceinline__ S herm_c1(const Herm8<R>& q, R q22r) {
    const S a = S(q.d0), b = S(q.d1), c = S(q22r);
    const S n = S(q.z01.re) * S(q.z01.re) + S(q.z01.im) * S(q.z01.im) + S(q.z02.re) * S(q.z02.re) +
                S(q.z02.im) * S(q.z02.im) + S(q.z12.re) * S(q.z12.re) + S(q.z12.im) * S(q.z12.im);
    return S(0.5) * (a * a + b * b + c * c) + n;
}

// Threshold on c0/c0max above which the mixed path evaluates the coefficients in
// FP64: near a doubly degenerate spectrum acos loses about half the significand.
#define YM_DEGENERATE_X 0.98

template <class R>
__device__ __forceinline__ ChCoef<R> exp_coefficients(const Herm8<R>& q, R q22);

template <>
__device__ __forceinline__ ChCoef<double> exp_coefficients<double>(const Herm8<double>& q, double q22) {
    const double c0 = herm_det<double>(q, q22), c1 = herm_c1<double>(q, q22);
    if (c1 <= YM_SERIES_C1) return ch_series<double, SeriesTerms<double>::value>(c0, c1);
    return ch_coefficients<double>(c0, c1);
}

// Mixed path: the FP32 series for small Q; otherwise the FP32 closed form
// unless the spectrum is nearly degenerate (or tiny), then the closed form in
// FP64 from the FP32 entries.
template <>
__device__ __forceinline__ ChCoef<float> exp_coefficients<float>(const Herm8<float>& q, float q22) {
    const float c0 = herm_det<float>(q, q22);
    const float c1 = herm_c1<float>(q, q22);
    if (c1 <= float(YM_SERIES_C1)) return ch_series<float, SeriesTerms<float>::value>(c0, c1);
    const float c1s = sqrtf(c1);
    const float c0max = c1 * c1s * 0.38490017945975050f;  // 2/(3 sqrt 3)
    const float x = fabsf(c0) / c0max;
    if (x < float(YM_DEGENERATE_X) && c1 > 1e-12f) return ch_coefficients<float>(c0, c1);
    ChCoef<double> d = ch_coefficients<double>(herm_det<double>(q, q22), herm_c1<double>(q, q22));
    ChCoef<float> f;
    f.f0m1 = cx(float(d.f0m1.re), float(d.f0m1.im));
    f.f1 = cx(float(d.f1.re), float(d.f1.im));
    f.f2 = cx(float(d.f2.re), float(d.f2.im));
    return f;
}

// E = e^{iQ} = f0 + f1 Q + f2 Q^2 as a full matrix.
template <class R>
__device__ __forceinline__ void exp_iq(const Herm8<R>& q, M3<R>& e) {
    const R q22 = -(q.d0 + q.d1);
    const ChCoef<R> f = exp_coefficients<R>(q, q22);
    const QSquared<R> s = q_squared(q, q22);
    // diagonal: 1 + f0m1 + f1 q_ii + f2 (Q^2)_ii  (q_ii and (Q^2)_ii real)
    e.e[0][0] = cx(R(1) + (f.f0m1.re + f.f1.re * q.d0 + f.f2.re * s.a00), f.f0m1.im + f.f1.im * q.d0 + f.f2.im * s.a00);
    e.e[1][1] = cx(R(1) + (f.f0m1.re + f.f1.re * q.d1 + f.f2.re * s.a11), f.f0m1.im + f.f1.im * q.d1 + f.f2.im * s.a11);
    e.e[2][2] = cx(R(1) + (f.f0m1.re + f.f1.re * q22 + f.f2.re * s.a22), f.f0m1.im + f.f1.im * q22 + f.f2.im * s.a22);
    // off-diagonal: f1 q_ij + f2 (Q^2)_ij; lower entries use the conjugates of q and Q^2
#define YM_OFFD(I, J, QV, SV)                                                                     \
    e.e[I][J] = cx(f.f1.re * QV.re - f.f1.im * QV.im + f.f2.re * SV.re - f.f2.im * SV.im,         \
                   f.f1.re * QV.im + f.f1.im * QV.re + f.f2.re * SV.im + f.f2.im * SV.re);        \
    e.e[J][I] = cx(f.f1.re * QV.re + f.f1.im * QV.im + f.f2.re * SV.re + f.f2.im * SV.im,         \
                   -f.f1.re * QV.im + f.f1.im * QV.re - f.f2.re * SV.im + f.f2.im * SV.re);
    YM_OFFD(0, 1, q.z01, s.a01)
    YM_OFFD(0, 2, q.z02, s.a02)
    YM_OFFD(1, 2, q.z12, s.a12)
#undef YM_OFFD
}

// Rows 0 and 1 of e^{iQ} - 1 (enough to update an SU(3) link through its
// first two rows as U + (e^{iQ} - 1) U).
template <class R>
__device__ __forceinline__ void expm1_iq_rows2(const Herm8<R>& q, Rows2<R>& e) {
    const R q22 = -(q.d0 + q.d1);
    const ChCoef<R> f = exp_coefficients<R>(q, q22);
    const QSquared<R> s = q_squared(q, q22);
    e.e[0][0] = cx(f.f0m1.re + f.f1.re * q.d0 + f.f2.re * s.a00, f.f0m1.im + f.f1.im * q.d0 + f.f2.im * s.a00);
    e.e[1][1] = cx(f.f0m1.re + f.f1.re * q.d1 + f.f2.re * s.a11, f.f0m1.im + f.f1.im * q.d1 + f.f2.im * s.a11);
    // upper entries f1 q_ij + f2 (Q^2)_ij; e10 from the conjugates of q01 and (Q^2)_01
    e.e[0][1] = cx(f.f1.re * q.z01.re - f.f1.im * q.z01.im + f.f2.re * s.a01.re - f.f2.im * s.a01.im,
                   f.f1.re * q.z01.im + f.f1.im * q.z01.re + f.f2.re * s.a01.im + f.f2.im * s.a01.re);
    e.e[0][2] = cx(f.f1.re * q.z02.re - f.f1.im * q.z02.im + f.f2.re * s.a02.re - f.f2.im * s.a02.im,
                   f.f1.re * q.z02.im + f.f1.im * q.z02.re + f.f2.re * s.a02.im + f.f2.im * s.a02.re);
    e.e[1][2] = cx(f.f1.re * q.z12.re - f.f1.im * q.z12.im + f.f2.re * s.a12.re - f.f2.im * s.a12.im,
                   f.f1.re * q.z12.im + f.f1.im * q.z12.re + f.f2.re * s.a12.im + f.f2.im * s.a12.re);
    e.e[1][0] = cx(f.f1.re * q.z01.re + f.f1.im * q.z01.im + f.f2.re * s.a01.re + f.f2.im * s.a01.im,
                   -f.f1.re * q.z01.im + f.f1.im * q.z01.re - f.f2.re * s.a01.im + f.f2.im * s.a01.re);
}

}  // namespace ym
