// SU(3) algebra on the device, templated on the arithmetic type (double for the
// FP64 path, float for the mixed path).
//
// A link is a 3x3 complex matrix, row-major, the same element order as the
// reference's SU3 (include/Math/su3.h:63: 18 doubles, (re, im) interleaved).
// Products are written out with fused multiply-adds; the reference evaluates
// the same sums without FMA (su3.h:143-183), so the two agree to rounding.
#pragma once
#include <cuda_runtime.h>

namespace ym {

template <class R>
struct Cx {
    R re, im;
};

template <class R>
struct M3 {
    Cx<R> e[3][3];
};

// Hermitian traceless generator stored as 8 reals:
//   d0 = Z00, d1 = Z11 (Z22 = -d0 - d1, real diagonal),
//   z01, z02, z12 the upper off-diagonal entries (lower = conjugate).
template <class R>
struct Herm8 {
    R d0, d1;
    Cx<R> z01, z02, z12;
};

template <class R>
__device__ __forceinline__ Cx<R> cx(R re, R im) {
    Cx<R> c;
    c.re = re;
    c.im = im;
    return c;
}

// c = op(a) * op(b) with op = identity or dagger (DA / DB).
template <bool DA, bool DB, class R>
__device__ __forceinline__ void mmul(const M3<R>& a, const M3<R>& b, M3<R>& c) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            R re = R(0), im = R(0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const R xr = DA ? a.e[k][i].re : a.e[i][k].re;
                const R xi = DA ? -a.e[k][i].im : a.e[i][k].im;
                const R yr = DB ? b.e[j][k].re : b.e[k][j].re;
                const R yi = DB ? -b.e[j][k].im : b.e[k][j].im;
                re = fma(xr, yr, re);
                re = fma(-xi, yi, re);
                im = fma(xr, yi, im);
                im = fma(xi, yr, im);
            }
            c.e[i][j] = cx(re, im);
        }
    }
}

// c += op(a) * op(b)
template <bool DA, bool DB, class R>
__device__ __forceinline__ void mmul_acc(const M3<R>& a, const M3<R>& b, M3<R>& c) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            R re = c.e[i][j].re, im = c.e[i][j].im;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const R xr = DA ? a.e[k][i].re : a.e[i][k].re;
                const R xi = DA ? -a.e[k][i].im : a.e[i][k].im;
                const R yr = DB ? b.e[j][k].re : b.e[k][j].re;
                const R yi = DB ? -b.e[j][k].im : b.e[k][j].im;
                re = fma(xr, yr, re);
                re = fma(-xi, yi, re);
                im = fma(xr, yi, im);
                im = fma(xi, yr, im);
            }
            c.e[i][j] = cx(re, im);
        }
    }
}

template <class R>
__device__ __forceinline__ void mzero(M3<R>& a) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) a.e[i][j] = cx(R(0), R(0));
}

template <class R>
__device__ __forceinline__ void madd(M3<R>& a, const M3<R>& b) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            a.e[i][j].re += b.e[i][j].re;
            a.e[i][j].im += b.e[i][j].im;
        }
}

template <class R>
__device__ __forceinline__ R re_trace(const M3<R>& a) {
    return a.e[0][0].re + a.e[1][1].re + a.e[2][2].re;
}

// Re tr(a * b) and Re tr(a * b^+) without forming the product.
template <class R>
__device__ __forceinline__ R re_trace_mul(const M3<R>& a, const M3<R>& b) {
    R s = R(0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s = fma(a.e[i][k].re, b.e[k][i].re, s);
            s = fma(-a.e[i][k].im, b.e[k][i].im, s);
        }
    return s;
}

// Row 2 of an SU(3) matrix from rows 0 and 1: r2 = conj(r0 x r1).
template <class R>
__device__ __forceinline__ void reconstruct_row2(M3<R>& a) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int i = (k + 1) % 3, j = (k + 2) % 3;
        const Cx<R> p = a.e[0][i], q = a.e[1][j], r = a.e[0][j], s = a.e[1][i];
        R re = p.re * q.re - p.im * q.im - (r.re * s.re - r.im * s.im);
        R im = p.re * q.im + p.im * q.re - (r.re * s.im + r.im * s.re);
        a.e[2][k] = cx(re, -im);
    }
}

// ---------------------------------------------------------------------------
// Products of SU(3) matrices through their first two rows.  For A, B in SU(3)
// the product is in SU(3), so rows 0 and 1 of op(A) op(B) (18 complex
// multiply-adds) determine row 2 = conj(row0 x row1) (6 complex products):
// 24 instead of 27 complex multiply-adds, and a chain of products needs only
// the first two rows of its running left factor.
// ---------------------------------------------------------------------------
template <class R>
struct Rows2 {
    Cx<R> e[2][3];
};

// c(rows 0,1) = op(a) * op(b).  DA: a is read through its columns (dagger), so all
// of a's rows are needed; otherwise only a's rows 0 and 1 are read.
template <bool DA, bool DB, class R, class MA>
__device__ __forceinline__ void mmul_rows2(const MA& a, const M3<R>& b, Rows2<R>& c) {
#pragma unroll
    for (int i = 0; i < 2; i++) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            R re = R(0), im = R(0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const R xr = DA ? a.e[k][i].re : a.e[i][k].re;
                const R xi = DA ? -a.e[k][i].im : a.e[i][k].im;
                const R yr = DB ? b.e[j][k].re : b.e[k][j].re;
                const R yi = DB ? -b.e[j][k].im : b.e[k][j].im;
                re = fma(xr, yr, re);
                re = fma(-xi, yi, re);
                im = fma(xr, yi, im);
                im = fma(xi, yr, im);
            }
            c.e[i][j] = cx(re, im);
        }
    }
}

// row 2 of an SU(3) matrix given by its first two rows: conj(r0 x r1), entry k
template <class R>
__device__ __forceinline__ Cx<R> row2_entry(const Rows2<R>& a, int k) {
    const int i = (k + 1) % 3, j = (k + 2) % 3;
    const Cx<R> p = a.e[0][i], q = a.e[1][j], r = a.e[0][j], s = a.e[1][i];
    const R re = fma(p.re, q.re, fma(-p.im, q.im, -fma(r.re, s.re, -r.im * s.im)));
    const R im = fma(p.re, q.im, fma(p.im, q.re, -fma(r.re, s.im, r.im * s.re)));
    return cx(re, -im);
}

// acc += the SU(3) matrix whose first two rows are a
template <class R>
__device__ __forceinline__ void madd_su3_rows2(M3<R>& acc, const Rows2<R>& a) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            acc.e[i][j].re += a.e[i][j].re;
            acc.e[i][j].im += a.e[i][j].im;
        }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const Cx<R> r = row2_entry(a, k);
        acc.e[2][k].re += r.re;
        acc.e[2][k].im += r.im;
    }
}

template <class R>
__device__ __forceinline__ void full_from_rows2(const Rows2<R>& a, M3<R>& m) {
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) m.e[i][j] = a.e[i][j];
#pragma unroll
    for (int k = 0; k < 3; k++) m.e[2][k] = row2_entry(a, k);
}

// Products of SU(3) links through their first two rows (third row rebuilt as conj(r0 x r1))
// save 22% of the staple multiply-adds but rebuild a row from rounded rows.
// In FP64 that costs nothing measurable; in FP32 the rebuilt rows of the fused
// kernel's staples carried a systematic bias that grew linearly with flow time
// (t^2<E> at t = 4 on 32^4 drifted 4e-6 from FP64 against 5e-7 with full
// products, measured before the link update took its e^{iQ} - 1 form), so the
// fused kernel's FP32 staples form all three rows.  The plaquette field and
// the observables form their products through two rows in every precision
// (t = 4 error against FP64 1.0e-7 either way).
template <class R>
struct kTwoRowStaples {
    static constexpr bool value = sizeof(R) == 8;
};

// Entry (i,j) of u * w (full matrices).
template <class R>
__device__ __forceinline__ Cx<R> mul_entry(const M3<R>& u, const M3<R>& w, int i, int j) {
    R re = R(0), im = R(0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        re = fma(u.e[i][k].re, w.e[k][j].re, re);
        re = fma(-u.e[i][k].im, w.e[k][j].im, re);
        im = fma(u.e[i][k].re, w.e[k][j].im, im);
        im = fma(u.e[i][k].im, w.e[k][j].re, im);
    }
    return cx(re, im);
}

// Im of entry (i,i) of u * w.
template <class R>
__device__ __forceinline__ R mul_diag_im(const M3<R>& u, const M3<R>& w, int i) {
    R im = R(0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        im = fma(u.e[i][k].re, w.e[k][i].im, im);
        im = fma(u.e[i][k].im, w.e[k][i].re, im);
    }
    return im;
}

// Flow generator from X = U * Omega (Omega the staple sum):
//   Z = (i/2) [X - X^+]_traceless   (Hermitian, traceless),
// the quantity the reference returns from PureGauge::computeDerivative
// (src/Actions/puregauge.cpp:62-79, where X is formed as (Omega^+ U^+)^+).
template <class R>
__device__ __forceinline__ Herm8<R> force_from_x(const M3<R>& x) {
    Herm8<R> z;
    const R i0 = x.e[0][0].im, i1 = x.e[1][1].im, i2 = x.e[2][2].im;
    const R mean = (i0 + i1 + i2) * R(1.0 / 3.0);
    z.d0 = mean - i0;
    z.d1 = mean - i1;
    // (i/2)(a + ib) = (-b/2, a/2) with a + ib = X_ij - conj(X_ji)
    z.z01 = cx(R(-0.5) * (x.e[0][1].im + x.e[1][0].im), R(0.5) * (x.e[0][1].re - x.e[1][0].re));
    z.z02 = cx(R(-0.5) * (x.e[0][2].im + x.e[2][0].im), R(0.5) * (x.e[0][2].re - x.e[2][0].re));
    z.z12 = cx(R(-0.5) * (x.e[1][2].im + x.e[2][1].im), R(0.5) * (x.e[1][2].re - x.e[2][1].re));
    return z;
}

// The same generator from U and Omega without forming X: only the six
// off-diagonal entries and the imaginary diagonal of U * Omega are computed.
template <class R>
__device__ __forceinline__ Herm8<R> force_from_u_omega(const M3<R>& u, const M3<R>& w) {
    Herm8<R> z;
    const R i0 = mul_diag_im(u, w, 0), i1 = mul_diag_im(u, w, 1), i2 = mul_diag_im(u, w, 2);
    const R mean = (i0 + i1 + i2) * R(1.0 / 3.0);
    z.d0 = mean - i0;
    z.d1 = mean - i1;
    const Cx<R> x01 = mul_entry(u, w, 0, 1), x10 = mul_entry(u, w, 1, 0);
    const Cx<R> x02 = mul_entry(u, w, 0, 2), x20 = mul_entry(u, w, 2, 0);
    const Cx<R> x12 = mul_entry(u, w, 1, 2), x21 = mul_entry(u, w, 2, 1);
    z.z01 = cx(R(-0.5) * (x01.im + x10.im), R(0.5) * (x01.re - x10.re));
    z.z02 = cx(R(-0.5) * (x02.im + x20.im), R(0.5) * (x02.re - x20.re));
    z.z12 = cx(R(-0.5) * (x12.im + x21.im), R(0.5) * (x12.re - x21.re));
    return z;
}

// The generator (i/2)[X - X^+]_traceless of X = B C^+ without forming X: the
// six off-diagonal entries and the imaginary diagonal of B C^+.
template <class R>
__device__ __forceinline__ Herm8<R> force_from_b_cdag(const M3<R>& b, const M3<R>& c) {
    auto entry = [&](int i, int j) {  // (B C^+)_ij = sum_k b_ik conj(c_jk)
        R re = R(0), im = R(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re = fma(b.e[i][k].re, c.e[j][k].re, re);
            re = fma(b.e[i][k].im, c.e[j][k].im, re);
            im = fma(b.e[i][k].im, c.e[j][k].re, im);
            im = fma(-b.e[i][k].re, c.e[j][k].im, im);
        }
        return cx(re, im);
    };
    auto diag_im = [&](int i) {
        R im = R(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            im = fma(b.e[i][k].im, c.e[i][k].re, im);
            im = fma(-b.e[i][k].re, c.e[i][k].im, im);
        }
        return im;
    };
    Herm8<R> z;
    const R i0 = diag_im(0), i1 = diag_im(1), i2 = diag_im(2);
    const R mean = (i0 + i1 + i2) * R(1.0 / 3.0);
    z.d0 = mean - i0;
    z.d1 = mean - i1;
    const Cx<R> x01 = entry(0, 1), x10 = entry(1, 0);
    const Cx<R> x02 = entry(0, 2), x20 = entry(2, 0);
    const Cx<R> x12 = entry(1, 2), x21 = entry(2, 1);
    z.z01 = cx(R(-0.5) * (x01.im + x10.im), R(0.5) * (x01.re - x10.re));
    z.z02 = cx(R(-0.5) * (x02.im + x20.im), R(0.5) * (x02.re - x20.re));
    z.z12 = cx(R(-0.5) * (x12.im + x21.im), R(0.5) * (x12.re - x21.re));
    return z;
}

// The same generator of X = B C^+ for X in SU(3), from B's first two rows:
// rows 0 and 1 of X (six entries), then of row 2 = conj(row0 x row1) only
// X_20, X_21 and Im X_22.  92 multiply-adds, against 90 plus the 27 that
// rebuild B's row 2 for the full form.
template <class R>
__device__ __forceinline__ Herm8<R> force_from_b2_cdag(const Rows2<R>& b, const M3<R>& c) {
    Cx<R> x[2][3];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {  // (B C^+)_ij = sum_k b_ik conj(c_jk)
            R re = R(0), im = R(0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                re = fma(b.e[i][k].re, c.e[j][k].re, re);
                re = fma(b.e[i][k].im, c.e[j][k].im, re);
                im = fma(b.e[i][k].im, c.e[j][k].re, im);
                im = fma(-b.e[i][k].re, c.e[j][k].im, im);
            }
            x[i][j] = cx(re, im);
        }
    // row 2 = conj(row0 x row1): X_2k = conj(X_0i X_1j - X_0j X_1i), (i, j) = (k+1, k+2) mod 3
    auto cross = [&](int i, int j) {
        const Cx<R> p = x[0][i], q = x[1][j], r = x[0][j], s = x[1][i];
        const R re = fma(p.re, q.re, fma(-p.im, q.im, -fma(r.re, s.re, -r.im * s.im)));
        const R im = fma(p.re, q.im, fma(p.im, q.re, -fma(r.re, s.im, r.im * s.re)));
        return cx(re, -im);
    };
    const Cx<R> x20 = cross(1, 2), x21 = cross(2, 0);
    const R i2 = -fma(x[0][0].re, x[1][1].im, fma(x[0][0].im, x[1][1].re, -fma(x[0][1].re, x[1][0].im, x[0][1].im * x[1][0].re)));
    Herm8<R> z;
    const R i0 = x[0][0].im, i1 = x[1][1].im;
    const R mean = (i0 + i1 + i2) * R(1.0 / 3.0);
    z.d0 = mean - i0;
    z.d1 = mean - i1;
    z.z01 = cx(R(-0.5) * (x[0][1].im + x[1][0].im), R(0.5) * (x[0][1].re - x[1][0].re));
    z.z02 = cx(R(-0.5) * (x[0][2].im + x20.im), R(0.5) * (x[0][2].re - x20.re));
    z.z12 = cx(R(-0.5) * (x[1][2].im + x21.im), R(0.5) * (x[1][2].re - x21.re));
    return z;
}

// v^+ h v for a Hermitian traceless h: Hermitian and traceless again, so only
// its diagonal d0, d1 and upper triangle are formed.  W = h v uses h's real
// diagonal (h22 = -d0 - d1) and conjugate lower triangle.
template <class R>
__device__ __forceinline__ Herm8<R> herm_conj_by(const M3<R>& v, const Herm8<R>& h) {
    const R d2 = -(h.d0 + h.d1);
    M3<R> w;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const Cx<R> a = v.e[0][j], b = v.e[1][j], c = v.e[2][j];
        // row 0: d0 a + z01 b + z02 c
        w.e[0][j].re = fma(h.d0, a.re, fma(h.z01.re, b.re, fma(-h.z01.im, b.im, fma(h.z02.re, c.re, -h.z02.im * c.im))));
        w.e[0][j].im = fma(h.d0, a.im, fma(h.z01.re, b.im, fma(h.z01.im, b.re, fma(h.z02.re, c.im, h.z02.im * c.re))));
        // row 1: conj(z01) a + d1 b + z12 c
        w.e[1][j].re = fma(h.z01.re, a.re, fma(h.z01.im, a.im, fma(h.d1, b.re, fma(h.z12.re, c.re, -h.z12.im * c.im))));
        w.e[1][j].im = fma(h.z01.re, a.im, fma(-h.z01.im, a.re, fma(h.d1, b.im, fma(h.z12.re, c.im, h.z12.im * c.re))));
        // row 2: conj(z02) a + conj(z12) b + d2 c
        w.e[2][j].re = fma(h.z02.re, a.re, fma(h.z02.im, a.im, fma(h.z12.re, b.re, fma(h.z12.im, b.im, d2 * c.re))));
        w.e[2][j].im = fma(h.z02.re, a.im, fma(-h.z02.im, a.re, fma(h.z12.re, b.im, fma(-h.z12.im, b.re, d2 * c.im))));
    }
    auto entry = [&](int i, int j) {  // (v^+ w)_ij = sum_k conj(v_ki) w_kj
        R re = R(0), im = R(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re = fma(v.e[k][i].re, w.e[k][j].re, re);
            re = fma(v.e[k][i].im, w.e[k][j].im, re);
            im = fma(v.e[k][i].re, w.e[k][j].im, im);
            im = fma(-v.e[k][i].im, w.e[k][j].re, im);
        }
        return cx(re, im);
    };
    auto diag_re = [&](int i) {
        R re = R(0);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            re = fma(v.e[k][i].re, w.e[k][i].re, re);
            re = fma(v.e[k][i].im, w.e[k][i].im, re);
        }
        return re;
    };
    Herm8<R> r;
    r.d0 = diag_re(0);
    r.d1 = diag_re(1);
    r.z01 = entry(0, 1);
    r.z02 = entry(0, 2);
    r.z12 = entry(1, 2);
    return r;
}

template <class R>
__device__ __forceinline__ Herm8<R> h8_axpby(R a, const Herm8<R>& x, R b, const Herm8<R>& y) {
    Herm8<R> r;
    r.d0 = a * x.d0 - b * y.d0;
    r.d1 = a * x.d1 - b * y.d1;
    r.z01 = cx(a * x.z01.re - b * y.z01.re, a * x.z01.im - b * y.z01.im);
    r.z02 = cx(a * x.z02.re - b * y.z02.re, a * x.z02.im - b * y.z02.im);
    r.z12 = cx(a * x.z12.re - b * y.z12.re, a * x.z12.im - b * y.z12.im);
    return r;
}

template <class R>
__device__ __forceinline__ Herm8<R> h8_scale(R a, const Herm8<R>& x) {
    Herm8<R> r;
    r.d0 = a * x.d0;
    r.d1 = a * x.d1;
    r.z01 = cx(a * x.z01.re, a * x.z01.im);
    r.z02 = cx(a * x.z02.re, a * x.z02.im);
    r.z12 = cx(a * x.z12.re, a * x.z12.im);
    return r;
}

}  // namespace ym
