/*
 * ymoracle.c — CPU restatement (plain C, FP64) of the reference's Wilson-flow
 * hot path.  TEST INFRASTRUCTURE ONLY (parity checker and "port" CPU
 * baseline); the product never links or calls it.
 *
 * Every arithmetic routine below follows the reference's operation order
 * term by term so that, compiled without FMA contraction (-ffp-contract=off),
 * it reproduces the reference binary bit for bit.  The golden tables under
 * tests/golden were produced by the reference itself (oracle/_ref/ref_flow)
 * and pin this file.
 *
 * Per-site work is split over OpenMP threads; every global sum is taken
 * sequentially in site order, as the reference's Lattice sum() does
 * (include/Math/lattice.h:264-296), so results do not depend on the thread
 * count.
 */
#include "ymoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

int yo_version(void) { return 1; }

/* ---------------------------------------------------------------------------
 * 3x3 complex algebra
 * ------------------------------------------------------------------------- */

/* c = a*b.  Entry (i,j): sum over k = 0,1,2 of re/im products, evaluated left to
 * right in the order of include/Math/su3.h:146-166 (real: ar*br - ai*bi per k;
 * imag: ar*bi + ai*br per k).  c may alias neither a nor b. */
void yo_mul(const double* a, const double* b, double* c) {
    for (int i = 0; i < 3; i++) {
        const double* ar = a + 6 * i;
        for (int j = 0; j < 3; j++) {
            const double* b0 = b + 2 * j;
            const double* b1 = b + 6 + 2 * j;
            const double* b2 = b + 12 + 2 * j;
            double re = ar[0] * b0[0] - ar[1] * b0[1] + ar[2] * b1[0] - ar[3] * b1[1] + ar[4] * b2[0] -
                        ar[5] * b2[1];
            double im = ar[0] * b0[1] + ar[1] * b0[0] + ar[2] * b1[1] + ar[3] * b1[0] + ar[4] * b2[1] +
                        ar[5] * b2[0];
            c[6 * i + 2 * j] = re;
            c[6 * i + 2 * j + 1] = im;
        }
    }
}

/* c = a^dagger (src/Math/su3.cpp:28-37). */
void yo_dag(const double* a, double* c) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            c[2 * (3 * i + j)] = a[2 * (3 * j + i)];
            c[2 * (3 * i + j) + 1] = -a[2 * (3 * j + i) + 1];
        }
}

static inline double re_trace(const double* a) { return a[0] + a[8] + a[16]; }  /* su3.cpp:75-77 */
static inline double im_trace(const double* a) { return a[1] + a[9] + a[17]; }  /* su3.cpp:79-81 */

/* c = a * b^dagger, with the dagger materialised first as the reference's adj() does. */
static inline void mul_nd(const double* a, const double* b, double* c) {
    double bd[18];
    yo_dag(b, bd);
    yo_mul(a, bd, c);
}
static inline void mul_dn(const double* a, const double* b, double* c) {
    double ad[18];
    yo_dag(a, ad);
    yo_mul(ad, b, c);
}
static inline void mul_dd(const double* a, const double* b, double* c) {
    double ad[18], bd[18];
    yo_dag(a, ad);
    yo_dag(b, bd);
    yo_mul(ad, bd, c);
}

/* e^{iQ}, Cayley-Hamilton after Morningstar & Peardon, statement for statement as
 * src/Math/su3.cpp:96-183 (including its NaN for Q = 0, where acos sees 0/0). */
void yo_exp(const double* q, double* r) {
    double q2[18], q3[18];
    yo_mul(q, q, q2);
    yo_mul(q2, q, q3);
    double c0 = re_trace(q3) / 3.0;
    double c1 = re_trace(q2) / 2.0;
    int c0neg = 0;
    if (c0 < 0) {
        c0neg = 1;
        c0 = -c0;
    }
    double c1sqrt = sqrt(c1);
    double inv_sqrt3 = 1.0 / sqrt(3.0);
    double c0max = c1 * c1sqrt * inv_sqrt3 * 2.0 / 3.0;
    double theta = acos(c0 / c0max);
    double w = c1sqrt * sin(theta / 3.0);
    double u = c1sqrt * inv_sqrt3 * cos(theta / 3.0);
    double u2 = u * u, w2 = w * w;
    double xi;
    if (fabs(w) < 0.05)
        xi = 1.0 - w2 / 6.0 * (1 - w2 / 20.0 * (1 - w2 / 42.0));
    else
        xi = sin(w) / w;
    double cmu = cos(-u), smu = sin(-u);
    double c2u = cmu * cmu - smu * smu;
    double s2u = -2.0 * cmu * smu;
    double cw = cos(w);
    double cwcmu = cw * cmu, cwsmu = cw * smu, xicmu = xi * cmu, xismu = xi * smu;
    double h0r = (u2 - w2) * c2u + 8.0 * u2 * cwcmu - 2.0 * u * (3.0 * u2 + w2) * xismu;
    double h0i = (u2 - w2) * s2u + 8.0 * u2 * cwsmu + 2.0 * u * (3.0 * u2 + w2) * xicmu;
    double h1r = 2 * u * c2u - 2 * u * cwcmu - (3.0 * u2 - w2) * xismu;
    double h1i = 2 * u * s2u - 2 * u * cwsmu + (3.0 * u2 - w2) * xicmu;
    double h2r = c2u - cwcmu + 3 * u * xismu;
    double h2i = s2u - cwsmu - 3 * u * xicmu;
    if (c0neg) {
        h0i *= -1;
        h1r *= -1;
        h2i *= -1;
    }
    double norm = 1.0 / (9.0 * u2 - w2);
    h0r *= norm;
    h0i *= norm;
    h1r *= norm;
    h1i *= norm;
    h2r *= norm;
    h2i *= norm;
    for (int i = 0; i < 18; i += 2) {
        double re = h1r * q[i] - h1i * q[i + 1];
        re += h2r * q2[i] - h2i * q2[i + 1];
        if (i % 8 == 0) re += h0r;
        double im = h1r * q[i + 1] + h1i * q[i];
        im += h2r * q2[i + 1] + h2i * q2[i];
        if (i % 8 == 0) im += h0i;
        r[i] = re;
        r[i + 1] = im;
    }
}

void yo_exp_many(const double* q, double* r, long n) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) yo_exp(q + 18 * i, r + 18 * i);
}

/* ---------------------------------------------------------------------------
 * Lattice indexing (include/Math/lattice.h:87-89; periodic shift :360-594)
 * ------------------------------------------------------------------------- */

static inline long site_of(const int n[4], const int c[4]) {
    return c[0] + (long)n[0] * (c[1] + (long)n[1] * (c[2] + (long)n[2] * c[3]));
}
static inline void coords_of(const int n[4], long s, int c[4]) {
    c[0] = (int)(s % n[0]);
    s /= n[0];
    c[1] = (int)(s % n[1]);
    s /= n[1];
    c[2] = (int)(s % n[2]);
    c[3] = (int)(s / n[2]);
}
/* site of c + d1*e_dir1 + d2*e_dir2 (periodic); pass d2 = 0 for one step. */
static inline long hop(const int n[4], const int c[4], int dir1, int d1, int dir2, int d2) {
    int m[4] = {c[0], c[1], c[2], c[3]};
    m[dir1] = (m[dir1] + d1 + n[dir1]) % n[dir1];
    if (d2) m[dir2] = (m[dir2] + d2 + n[dir2]) % n[dir2];
    return site_of(n, m);
}
static inline const double* link(const double* U, long s, int mu) { return U + (s * 4 + mu) * 18; }
static inline long volume(const int n[4]) { return (long)n[0] * n[1] * n[2] * n[3]; }

/* ---------------------------------------------------------------------------
 * Force (src/Actions/puregauge.cpp:36-79)
 * ------------------------------------------------------------------------- */

/* Z_mu(x) for one site.  Staples: for nu != mu ascending, the upper staple
 * U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ then the lower staple taken at y = x-nu,
 * U_nu(y+mu)^+ U_mu(y)^+ U_nu(y) (puregauge.cpp:41-51).  Then
 * M = Omega^+ U_mu^+ (:64), A = M^+ - M (:65), the imaginary-diagonal trace
 * removed (:67-70) and Z = (i/2) A as (re, im) -> (-im/2, re/2) (:72-76). */
static void derivative_site(const double* U, const int n[4], long s, int mu, double* z) {
    int c[4];
    coords_of(n, s, c);
    double omega[18];
    memset(omega, 0, sizeof(omega));
    double t1[18], t2[18];
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        long xpm = hop(n, c, mu, 1, 0, 0);
        long xpn = hop(n, c, nu, 1, 0, 0);
        mul_nd(link(U, xpm, nu), link(U, xpn, mu), t1);
        mul_nd(t1, link(U, s, nu), t2);
        for (int k = 0; k < 18; k++) omega[k] += t2[k];

        long y = hop(n, c, nu, -1, 0, 0);
        long ypm = hop(n, c, nu, -1, mu, 1);
        mul_dd(link(U, ypm, nu), link(U, y, mu), t1);
        yo_mul(t1, link(U, y, nu), t2);
        for (int k = 0; k < 18; k++) omega[k] += t2[k];
    }
    double m[18], a[18];
    mul_dd(omega, link(U, s, mu), m);
    yo_dag(m, a);
    for (int k = 0; k < 18; k++) a[k] = a[k] - m[k];
    double tr = im_trace(a) / 3.0;
    for (int i = 1; i < 18; i += 8) a[i] -= tr;
    for (int i = 0; i < 18; i += 2) {
        double re = a[i];
        z[i] = -a[i + 1] * 0.5;
        z[i + 1] = re * 0.5;
    }
}

void yo_derivative(const double* U, const int n[4], int mu, double* Zmu) {
    long V = volume(n);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; s++) derivative_site(U, n, s, mu, Zmu + 18 * s);
}

/* ---------------------------------------------------------------------------
 * RK3 step (src/Apps/wilsonflow.cpp:141-172)
 * ------------------------------------------------------------------------- */

/* U <- exp(Q) U for Q = (Z * s1) * s2 elementwise (s2 = 1 skips the second scale
 * exactly as multiplying by 1.0 would). */
static void update_links(double* U, const double* Z, long V, double s1, double s2, int two_scales) {
#pragma omp parallel for schedule(static)
    for (long l = 0; l < 4 * V; l++) {
        double q[18], e[18], u[18];
        for (int k = 0; k < 18; k++) {
            q[k] = Z[18 * l + k] * s1;
            if (two_scales) q[k] = q[k] * s2;
        }
        yo_exp(q, e);
        memcpy(u, U + 18 * l, sizeof(u));
        yo_mul(e, u, U + 18 * l);
    }
}

/* Z <- D(U) * cd - Z * cz for every link (cz = 0 and first = 1: Z <- D(U)). */
static void combine_force(const double* U, double* Z, const int n[4], double cd, double cz, int first) {
    long V = volume(n);
#pragma omp parallel for schedule(static)
    for (long s = 0; s < V; s++) {
        for (int mu = 0; mu < 4; mu++) {
            double d[18];
            derivative_site(U, n, s, mu, d);
            double* z = Z + (s * 4 + mu) * 18;
            for (int k = 0; k < 18; k++) z[k] = first ? d[k] : d[k] * cd - z[k] * cz;
        }
    }
}

void yo_flow_step(double* U, double* Z, const int n[4], double eps) {
    long V = volume(n);
    combine_force(U, Z, n, 0.0, 0.0, 1);                    /* Z0 (:143-144) */
    update_links(U, Z, V, eps, 1.0 / 4.0, 1);               /* W1 (:147-149) */
    combine_force(U, Z, n, 8.0 / 9.0, 17.0 / 36.0, 0);      /* Z1 (:152-154) */
    update_links(U, Z, V, eps, 1.0, 0);                     /* W2 (:158-160) */
    combine_force(U, Z, n, 3.0 / 4.0, 1.0, 0);              /* Z2 (:163-165), "- Z" */
    update_links(U, Z, V, eps, 1.0, 0);                     /* W3 (:169-171) */
}

/* One of the three stages of yo_flow_step alone (stage 0, 1, 2): the pieces of
 * src/Apps/wilsonflow.cpp:143-149, :152-160 and :163-171.  Lets a caller run
 * a decomposed lattice stage by stage with its halos exchanged in between. */
void yo_flow_stage(double* U, double* Z, const int n[4], double eps, int stage) {
    long V = volume(n);
    if (stage == 0) {
        combine_force(U, Z, n, 0.0, 0.0, 1);
        update_links(U, Z, V, eps, 1.0 / 4.0, 1);
    } else if (stage == 1) {
        combine_force(U, Z, n, 8.0 / 9.0, 17.0 / 36.0, 0);
        update_links(U, Z, V, eps, 1.0, 0);
    } else {
        combine_force(U, Z, n, 3.0 / 4.0, 1.0, 0);
        update_links(U, Z, V, eps, 1.0, 0);
    }
}

/* ---------------------------------------------------------------------------
 * Observables (src/Observables/superobs.cpp:31-128)
 * ------------------------------------------------------------------------- */

/* The four 4-link loops of plane (mu,nu) at site s, each multiplied left to right
 * as at superobs.cpp:47-68.  shiftmu = U_nu(x+mu), shiftnu = U_mu(x+nu). */
static void loops_site(const double* U, const int n[4], long s, int mu, int nu, double* leaf, double* tmm,
                       double* tmp, double* tpm) {
    int c[4];
    coords_of(n, s, c);
    const double* umu = link(U, s, mu);
    const double* unu = link(U, s, nu);
    const double* smu = link(U, hop(n, c, mu, 1, 0, 0), nu);
    const double* snu = link(U, hop(n, c, nu, 1, 0, 0), mu);
    double a[18], b[18];
    if (leaf) {
        yo_mul(umu, smu, a);
        mul_nd(a, snu, b);
        mul_nd(b, unu, leaf);
    }
    if (tmm) {
        mul_dd(snu, unu, a);
        yo_mul(a, umu, b);
        yo_mul(b, smu, tmm);
    }
    if (tmp) {
        mul_nd(snu, smu, a);
        mul_nd(a, umu, b);
        yo_mul(b, unu, tmp);
    }
    if (tpm) {
        mul_dn(umu, unu, a);
        yo_mul(a, snu, b);
        mul_nd(b, smu, tpm);
    }
}

void yo_superobs(const double* U, const int n[4], double out[3]) {
    long V = volume(n);
    double* leaf = (double*)malloc(sizeof(double) * 18 * V);
    double* G = (double*)malloc(sizeof(double) * 18 * V * 6);
    double* per = (double*)malloc(sizeof(double) * V);
    double plaq_sum[18];
    memset(plaq_sum, 0, sizeof(plaq_sum));
    double energy = 0.0, topc = 0.0;
    int plane = 0;
    int plane_of[4][4];
    for (int mu = 0; mu < 4; mu++) {
        for (int nu = mu + 1; nu < 4; nu++, plane++) {
            plane_of[mu][nu] = plane;
            double* g = G + (long)plane * 18 * V;
#pragma omp parallel for schedule(static)
            for (long s = 0; s < V; s++) {
                int c[4];
                coords_of(n, s, c);
                double cl[18], t[18], cd[18];
                loops_site(U, n, s, mu, nu, leaf + 18 * s, NULL, NULL, NULL);
                memcpy(cl, leaf + 18 * s, sizeof(cl));
                /* clover += shift(shift(tempmm,mu,-1),nu,-1): tempmm at x-mu-nu (:72) */
                loops_site(U, n, hop(n, c, mu, -1, nu, -1), mu, nu, NULL, t, NULL, NULL);
                for (int k = 0; k < 18; k++) cl[k] += t[k];
                /* clover -= shift(tempmp,nu,-1): tempmp at x-nu (:73) */
                loops_site(U, n, hop(n, c, nu, -1, 0, 0), mu, nu, NULL, NULL, t, NULL);
                for (int k = 0; k < 18; k++) cl[k] -= t[k];
                /* clover -= shift(temppm,mu,-1): temppm at x-mu (:74) */
                loops_site(U, n, hop(n, c, mu, -1, 0, 0), mu, nu, NULL, NULL, NULL, t);
                for (int k = 0; k < 18; k++) cl[k] -= t[k];
                /* G = C - C^+, imaginary-diagonal trace removed (:101-106) */
                yo_dag(cl, cd);
                double* gs = g + 18 * s;
                for (int k = 0; k < 18; k++) gs[k] = cl[k] - cd[k];
                double tr = im_trace(gs) / 3.0;
                for (int i = 1; i < 18; i += 8) gs[i] -= tr;
                double gg[18];
                yo_mul(gs, gs, gg);
                per[s] = re_trace(gg);
            }
            /* plaqSum += sum(clovers) before the other leaves are added (:71) */
            double lsum[18];
            memset(lsum, 0, sizeof(lsum));
            for (long s = 0; s < V; s++)
                for (int k = 0; k < 18; k++) lsum[k] += leaf[18 * s + k];
            for (int k = 0; k < 18; k++) plaq_sum[k] += lsum[k];
            double esum = 0.0;
            for (long s = 0; s < V; s++) esum += per[s];
            energy += esum; /* (:109) */
        }
    }
    /* topc -= sum(ReTr(G_{0nu} G_{rho sig})) with G_{31} formed as adj(G_{13}) (:114-124) */
    for (int nu = 1; nu < 4; nu++) {
        int rho = nu % 3 + 1;
        int sig = rho % 3 + 1;
        const double* ga = G + (long)plane_of[0][nu] * 18 * V;
        int swap = !(rho < sig);
        const double* gb = swap ? G + (long)plane_of[sig][rho] * 18 * V : G + (long)plane_of[rho][sig] * 18 * V;
#pragma omp parallel for schedule(static)
        for (long s = 0; s < V; s++) {
            double p[18];
            if (swap)
                mul_nd(ga + 18 * s, gb + 18 * s, p);
            else
                yo_mul(ga + 18 * s, gb + 18 * s, p);
            per[s] = re_trace(p);
        }
        double tsum = 0.0;
        for (long s = 0; s < V; s++) tsum += per[s];
        topc -= tsum;
    }
    double plaq = re_trace(plaq_sum) / 18.0 / (double)n[0] / (double)n[1] / (double)n[2] / (double)n[3] / 1.0;
    topc /= (16 * 16 * M_PI * M_PI);
    out[0] = plaq;
    out[1] = topc;
    out[2] = energy;
    free(leaf);
    free(G);
    free(per);
}

int yo_flow(double* U, const int n[4], double eps, int nsteps, int every, double* table) {
    long V = volume(n);
    double* Z = (double*)malloc(sizeof(double) * 18 * 4 * V);
    int rows = 0;
    double t = 0.0, o[3];
    yo_superobs(U, n, o);
    double* r = table;
    r[0] = 0; r[1] = t; r[2] = o[0]; r[3] = o[1]; r[4] = o[2];
    rows = 1;
    for (int s = 1; s <= nsteps; s++) {
        yo_flow_step(U, Z, n, eps);
        t += eps;
        if (every > 0 && (s % every == 0 || s == nsteps)) {
            yo_superobs(U, n, o);
            r = table + 5 * rows;
            r[0] = s; r[1] = t; r[2] = o[0]; r[3] = o[1]; r[4] = o[2];
            rows++;
        }
    }
    free(Z);
    return rows;
}

/* ---------------------------------------------------------------------------
 * Seeded synthetic fields
 * ------------------------------------------------------------------------- */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the
 * multiply-xor bijection with the published multipliers and Weyl key steps. */
void yo_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Streams of the field recipes (counter word 3 = stream << 16 | block). */
enum { STREAM_H = 0, STREAM_HAAR = 1, STREAM_PICK = 2, STREAM_MC = 3 };

static inline double u53(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* Two standard normals from block `block` of (link, stream): Box-Muller on one
 * Philox output (two 53-bit uniforms). */
static void gauss2(uint64_t seed, uint32_t config, uint64_t lidx, uint32_t stream, uint32_t block, double g[2]) {
    uint32_t ctr[4] = {(uint32_t)lidx, (uint32_t)(lidx >> 32), config, (stream << 16) | block};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    yo_philox4x32(ctr, key, o);
    double u1 = 1.0 - u53(o[0], o[1]); /* (0, 1] */
    double u2 = u53(o[2], o[3]);
    double r = sqrt(-2.0 * log(u1));
    double ph = 6.283185307179586 * u2;
    g[0] = r * cos(ph);
    g[1] = r * sin(ph);
}

/* U = e^{i a H}: H traceless Hermitian with 9 iid N(0,1) reals (3 diagonal, 3 Re and
 * 3 Im of the upper triangle; lower = conjugate), diagonal trace/3 removed. */
static void expiah_link(uint64_t seed, uint32_t config, uint64_t lidx, double a, double* u) {
    double g[10];
    for (uint32_t b = 0; b < 5; b++) gauss2(seed, config, lidx, STREAM_H, b, g + 2 * b);
    double h[18];
    double tr = (g[0] + g[1] + g[2]) / 3.0;
    h[0] = g[0] - tr; h[1] = 0;
    h[8] = g[1] - tr; h[9] = 0;
    h[16] = g[2] - tr; h[17] = 0;
    h[2] = g[3]; h[3] = g[4];     /* (0,1) */
    h[4] = g[5]; h[5] = g[6];     /* (0,2) */
    h[10] = g[7]; h[11] = g[8];   /* (1,2) */
    h[6] = g[3]; h[7] = -g[4];    /* (1,0) */
    h[12] = g[5]; h[13] = -g[6];  /* (2,0) */
    h[14] = g[7]; h[15] = -g[8];  /* (2,1) */
    double q[18];
    for (int k = 0; k < 18; k++) q[k] = a * h[k];
    yo_exp(q, u);
}

void yo_gen_expiah(double* U, const int n[4], double a, uint64_t seed, uint32_t config) {
    long L = 4 * volume(n);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < L; l++) expiah_link(seed, config, (uint64_t)l, a, U + 18 * l);
}

/* Haar-random SU(3): rows of a complex Gaussian 3x3 orthonormalised by
 * Gram-Schmidt (= QR with positive real R diagonal, Mezzadri 2007), then
 * divided by the principal cube root of the determinant. */
static void haar_link(uint64_t seed, uint32_t config, uint64_t lidx, double* u) {
    double g[18];
    for (uint32_t b = 0; b < 9; b++) gauss2(seed, config, lidx, STREAM_HAAR, b, g + 2 * b);
    memcpy(u, g, sizeof(g));
    yo_reunitarize(u, 1); /* orthonormal rows 0,1 and row 2 = conj(row0 x row1): det = 1 */
    /* reunitarize replaces row 2 by the cross product, which keeps Haar measure on the
     * first two rows and fixes det = 1 exactly. */
}

void yo_gen_haar_mix(double* U, const int n[4], double frac, uint64_t seed, uint32_t config) {
    long L = 4 * volume(n);
#pragma omp parallel for schedule(static)
    for (long l = 0; l < L; l++) {
        uint32_t ctr[4] = {(uint32_t)l, (uint32_t)((uint64_t)l >> 32), config, (uint32_t)STREAM_PICK << 16};
        uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        uint32_t o[4];
        yo_philox4x32(ctr, key, o);
        if (u53(o[0], o[1]) < frac) haar_link(seed, config, (uint64_t)l, U + 18 * l);
    }
}

void yo_gen_cold(double* U, const int n[4]) {
    long L = 4 * volume(n);
    for (long l = 0; l < L; l++) {
        double* u = U + 18 * l;
        memset(u, 0, 18 * sizeof(double));
        u[0] = u[8] = u[16] = 1.0;
    }
}

/* Sequential Philox stream for the Metropolis generator. */
typedef struct {
    uint32_t key[2];
    uint64_t n;
    uint32_t buf[4];
    int pos;
} stream_t;

static uint32_t next_u32(stream_t* st) {
    if (st->pos == 4) {
        uint32_t ctr[4] = {(uint32_t)st->n, (uint32_t)(st->n >> 32), 0u, (uint32_t)STREAM_MC << 16};
        yo_philox4x32(ctr, st->key, st->buf);
        st->n++;
        st->pos = 0;
    }
    return st->buf[st->pos++];
}
static double next_uniform(stream_t* st) {
    uint32_t a = next_u32(st);
    uint32_t b = next_u32(st);
    return u53(a, b);
}

/* Near-identity SU(3) proposal: product of three SU(2) elements embedded in the
 * (0,1), (0,2) and (1,2) blocks, each x0 = +-sqrt(1-eps^2) and a uniformly
 * oriented 3-vector of length eps (after src/Math/random.cpp:71-156). */
static void su2_embed(stream_t* st, double eps, int p, int q, double* m) {
    double x[4], norm = 0.0;
    x[0] = next_uniform(st) - 0.5;
    for (int i = 1; i < 4; i++) {
        x[i] = next_uniform(st) - 0.5;
        norm += x[i] * x[i];
    }
    norm = sqrt(norm);
    x[0] = (x[0] < 0 ? -1.0 : 1.0) * sqrt(1 - eps * eps);
    for (int i = 1; i < 4; i++) x[i] = x[i] * eps / norm;
    memset(m, 0, 18 * sizeof(double));
    m[0] = m[8] = m[16] = 1.0;
    /* [[x0 + i x3, x2 + i x1], [-x2 + i x1, x0 - i x3]] on rows/cols (p, q) */
    m[2 * (3 * p + p)] = x[0]; m[2 * (3 * p + p) + 1] = x[3];
    m[2 * (3 * q + q)] = x[0]; m[2 * (3 * q + q) + 1] = -x[3];
    m[2 * (3 * p + q)] = x[2]; m[2 * (3 * p + q) + 1] = x[1];
    m[2 * (3 * q + p)] = -x[2]; m[2 * (3 * q + p) + 1] = x[1];
}

static void proposal(stream_t* st, double eps, double* x) {
    double r[18], s[18], t[18], rs[18];
    su2_embed(st, eps, 0, 1, r);
    su2_embed(st, eps, 0, 2, s);
    su2_embed(st, eps, 1, 2, t);
    yo_mul(r, s, rs);
    yo_mul(rs, t, x);
}

/* Staple sum Omega_mu(x) of one link, same products as derivative_site. */
static void staple_site(const double* U, const int n[4], long s, int mu, double* omega) {
    int c[4];
    coords_of(n, s, c);
    memset(omega, 0, 18 * sizeof(double));
    double t1[18], t2[18];
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        mul_nd(link(U, hop(n, c, mu, 1, 0, 0), nu), link(U, hop(n, c, nu, 1, 0, 0), mu), t1);
        mul_nd(t1, link(U, s, nu), t2);
        for (int k = 0; k < 18; k++) omega[k] += t2[k];
        long y = hop(n, c, nu, -1, 0, 0);
        mul_dd(link(U, hop(n, c, nu, -1, mu, 1), nu), link(U, y, mu), t1);
        yo_mul(t1, link(U, y, nu), t2);
        for (int k = 0; k < 18; k++) omega[k] += t2[k];
    }
}

/* Metropolis sweeps in the loop order of src/Apps/gaugefieldfactory.cpp:192-220
 * (x outermost, then y, z, t, mu; `hits` proposals X*U per link against a staple
 * sum computed once per link) with dS = -(beta/3) Re tr[(U' - U) A]
 * (the action written in the comment at src/Actions/puregauge.cpp:28).
 * Starts from whatever U holds (cold start: call yo_gen_cold first). */
double yo_gen_metropolis(double* U, const int n[4], double beta, double su3eps, int sweeps, int hits,
                         uint64_t seed) {
    stream_t st;
    st.key[0] = (uint32_t)seed;
    st.key[1] = (uint32_t)(seed >> 32);
    st.n = 0;
    st.pos = 4;
    long acc = 0, tries = 0;
    for (int sw = 0; sw < sweeps; sw++) {
        for (int x = 0; x < n[0]; x++)
            for (int y = 0; y < n[1]; y++)
                for (int z = 0; z < n[2]; z++)
                    for (int t = 0; t < n[3]; t++)
                        for (int mu = 0; mu < 4; mu++) {
                            int c[4] = {x, y, z, t};
                            long s = site_of(n, c);
                            double A[18];
                            staple_site(U, n, s, mu, A);
                            double* u = U + (s * 4 + mu) * 18;
                            for (int h = 0; h < hits; h++) {
                                double X[18], un[18], d[18], p[18];
                                proposal(&st, su3eps, X);
                                yo_mul(X, u, un);
                                for (int k = 0; k < 18; k++) d[k] = un[k] - u[k];
                                yo_mul(d, A, p);
                                double dS = -beta / 3.0 * re_trace(p);
                                if (exp(-dS) > next_uniform(&st)) {
                                    memcpy(u, un, sizeof(un));
                                    acc++;
                                }
                                tries++;
                            }
                        }
    }
    return tries ? (double)acc / (double)tries : 0.0;
}

/* The device generator's chain (test infrastructure for the checkerboard
 * Metropolis kernel): the same update as yo_gen_metropolis, visited as a
 * checkerboard -- sweep, then mu, then site parity, every link of that parity
 * (their staples hold no link of the same direction and parity, so the order
 * inside a parity class is immaterial) -- with the random numbers of
 * (link l = 4 s + mu, sweep, hit) drawn counter-based: Philox4x32-10 with key
 * (seed_lo, seed_hi ^ 0x4D455452) and counter (l_lo, l_hi ^ call << 24,
 * sweep, hit) for call = 0..3; uniforms (w + 1/2) 2^-32; words 0-11 build the
 * three SU(2) factors X = R S T, word 13 < 1/2 proposes X^+ U instead of X U
 * (X and X^+ equally likely, so the proposal is symmetric and the chain keeps
 * detailed balance, which R S T alone -- distributed unlike its inverse
 * T^+ S^+ R^+ -- does not), word 12 is the accept draw.  dS is formed as
 * -(beta/3) (Re tr U'A - Re tr UA).  Sweeps are numbered from sweep0. */
static inline double unit32(uint32_t w) { return ((double)w + 0.5) * 2.3283064365386963e-10; }

static void su2_from(const double r[4], double eps, int p, int q, double* m) {
    double v1 = r[1] - 0.5, v2 = r[2] - 0.5, v3 = r[3] - 0.5;
    const double norm = sqrt(v1 * v1 + v2 * v2 + v3 * v3);
    const double x0 = (r[0] - 0.5 < 0.0 ? -1.0 : 1.0) * sqrt(1.0 - eps * eps);
    v1 = v1 * eps / norm;
    v2 = v2 * eps / norm;
    v3 = v3 * eps / norm;
    memset(m, 0, 18 * sizeof(double));
    m[0] = m[8] = m[16] = 1.0;
    m[2 * (3 * p + p)] = x0; m[2 * (3 * p + p) + 1] = v3;
    m[2 * (3 * q + q)] = x0; m[2 * (3 * q + q) + 1] = -v3;
    m[2 * (3 * p + q)] = v2; m[2 * (3 * p + q) + 1] = v1;
    m[2 * (3 * q + p)] = -v2; m[2 * (3 * q + p) + 1] = v1;
}

static double re_trace_prod(const double* a, const double* b) {
    double t = 0.0;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
            const double* x = a + 2 * (3 * i + k);
            const double* y = b + 2 * (3 * k + i);
            t += x[0] * y[0] - x[1] * y[1];
        }
    return t;
}

long yo_gen_metropolis_cb(double* U, const int n[4], double beta, double su3eps, int sweeps, int hits,
                          uint64_t seed, uint32_t sweep0) {
    const long V = volume(n);
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x4D455452u};
    long acc = 0;
    for (int sw = 0; sw < sweeps; sw++)
        for (int mu = 0; mu < 4; mu++)
            for (int parity = 0; parity < 2; parity++)
                for (long s = 0; s < V; s++) {
                    int c[4];
                    coords_of(n, s, c);
                    if (((c[0] + c[1] + c[2] + c[3]) & 1) != parity) continue;
                    double A[18];
                    staple_site(U, n, s, mu, A);
                    double* u = U + (s * 4 + mu) * 18;
                    const uint64_t l = (uint64_t)s * 4 + (uint64_t)mu;
                    for (int h = 0; h < hits; h++) {
                        double r[16];
                        for (uint32_t call = 0; call < 4; call++) {
                            const uint32_t ctr[4] = {(uint32_t)l, (uint32_t)(l >> 32) ^ (call << 24),
                                                     sweep0 + (uint32_t)sw, (uint32_t)h};
                            uint32_t o[4];
                            yo_philox4x32(ctr, key, o);
                            for (int k = 0; k < 4; k++) r[4 * call + k] = unit32(o[k]);
                        }
                        double a[18], b[18], ab[18], X[18], un[18];
                        su2_from(r + 0, su3eps, 0, 1, a);
                        su2_from(r + 4, su3eps, 0, 2, b);
                        yo_mul(a, b, ab);
                        su2_from(r + 8, su3eps, 1, 2, a);
                        yo_mul(ab, a, X);
                        if (r[13] < 0.5) {
                            double Xd[18];
                            yo_dag(X, Xd);
                            yo_mul(Xd, u, un);
                        } else {
                            yo_mul(X, u, un);
                        }
                        const double dS = -beta / 3.0 * (re_trace_prod(un, A) - re_trace_prod(u, A));
                        if (exp(-dS) > r[12]) {
                            memcpy(u, un, sizeof(un));
                            acc++;
                        }
                    }
                }
    return acc;
}

/* Rows 0 and 1 normalised by Gram-Schmidt; row 2 = conj(row0 x row1). */
void yo_reunitarize(double* U, long nlinks) {
#pragma omp parallel for schedule(static)
    for (long l = 0; l < nlinks; l++) {
        double* u = U + 18 * l;
        double n0 = 0.0;
        for (int k = 0; k < 6; k++) n0 += u[k] * u[k];
        n0 = 1.0 / sqrt(n0);
        for (int k = 0; k < 6; k++) u[k] *= n0;
        /* p = <row0, row1> = sum conj(r0_k) r1_k */
        double pr = 0.0, pi = 0.0;
        for (int k = 0; k < 3; k++) {
            double ar = u[2 * k], ai = u[2 * k + 1], br = u[6 + 2 * k], bi = u[6 + 2 * k + 1];
            pr += ar * br + ai * bi;
            pi += ar * bi - ai * br;
        }
        for (int k = 0; k < 3; k++) {
            double ar = u[2 * k], ai = u[2 * k + 1];
            u[6 + 2 * k] -= pr * ar - pi * ai;
            u[6 + 2 * k + 1] -= pr * ai + pi * ar;
        }
        double n1 = 0.0;
        for (int k = 6; k < 12; k++) n1 += u[k] * u[k];
        n1 = 1.0 / sqrt(n1);
        for (int k = 6; k < 12; k++) u[k] *= n1;
        /* row2_k = conj(r0_i r1_j - r0_j r1_i), (i,j,k) cyclic */
        for (int k = 0; k < 3; k++) {
            int i = (k + 1) % 3, j = (k + 2) % 3;
            double ar = u[2 * i], ai = u[2 * i + 1], br = u[6 + 2 * j], bi = u[6 + 2 * j + 1];
            double cr = u[2 * j], ci = u[2 * j + 1], dr = u[6 + 2 * i], di = u[6 + 2 * i + 1];
            double re = (ar * br - ai * bi) - (cr * dr - ci * di);
            double im = (ar * bi + ai * br) - (cr * di + ci * dr);
            u[12 + 2 * k] = re;
            u[12 + 2 * k + 1] = -im;
        }
    }
}

void yo_unitarity(const double* U, long nlinks, double out[2]) {
    double worst = 0.0, worst_det = 0.0;
    for (long l = 0; l < nlinks; l++) {
        const double* u = U + 18 * l;
        double p[18];
        mul_nd(u, u, p);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double re = p[2 * (3 * i + j)] - (i == j ? 1.0 : 0.0);
                double im = p[2 * (3 * i + j) + 1];
                double e = sqrt(re * re + im * im);
                if (e > worst) worst = e;
            }
        /* det = row0 . (row1 x row2) */
        double dr = 0.0, di = 0.0;
        for (int k = 0; k < 3; k++) {
            int i = (k + 1) % 3, j = (k + 2) % 3;
            double ar = u[6 + 2 * i], ai = u[6 + 2 * i + 1], br = u[12 + 2 * j], bi = u[12 + 2 * j + 1];
            double cr = u[6 + 2 * j], ci = u[6 + 2 * j + 1], er = u[12 + 2 * i], ei = u[12 + 2 * i + 1];
            double xr = (ar * br - ai * bi) - (cr * er - ci * ei);
            double xi = (ar * bi + ai * br) - (cr * ei + ci * er);
            dr += u[2 * k] * xr - u[2 * k + 1] * xi;
            di += u[2 * k] * xi + u[2 * k + 1] * xr;
        }
        double e = sqrt((dr - 1.0) * (dr - 1.0) + di * di);
        if (e > worst_det) worst_det = e;
    }
    out[0] = worst;
    out[1] = worst_det;
}
