// Device code of the fused RK3 stage, shared by the single-configuration
// kernel (flow.cu) and the ensemble kernel (ensemble.cu).
//
// Per link (x, mu):
//   Omega = sum over nu != mu of the upper staple U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
//           and the lower staple U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
//           (src/Actions/puregauge.cpp:36-54, same nu order: upper then lower)
//   D     = (i/2) [U Omega - (U Omega)^+]_traceless     (puregauge.cpp:62-79)
//   Z     = D                       stage 0   (src/Apps/wilsonflow.cpp:143-144)
//         = 8/9 D - 17/36 Z_prev    stage 1   (:152-154)
//         = 3/4 D - Z_prev          stage 2   (:163-165)
//   U'    = exp(i eps_s Z) U,  eps_s = eps/4, eps, eps   (:147-149, :158-160, :169-171)
//
// Stages are Jacobi updates: every Z of a stage is computed from the same
// field, so links are read from `in` and written to `out` (ping-pong).  Z is
// written by stages 0 and 1 and read by stages 1 and 2.
#pragma once
#include "expsu3.cuh"
#include "field.cuh"

namespace ym {

// Resident 128-thread blocks per SM the stage kernel is compiled for (caps its
// registers), swept at 32^4 on B200: FP64 is fastest at 4 blocks (128
// registers), the FP32 18-real form at 6 (80 registers, 24 warps; 1.21 against
// 1.24-1.37 ms per step at 5) and the 12-real form at 5 (96 registers; its row
// rebuild spills heavily at 80).
template <class F>
struct StageMinBlocks {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 4 : (F::kElems == 9 ? 6 : 5);
};

// D_mu(x) = (i/2)[U Omega - (U Omega)^+]_traceless for one link; also returns U_mu(x).
// Each staple is a product of three SU(3) links; of U Omega only the entries
// the traceless anti-Hermitian part needs are computed.  mu is warp-uniform and the nu loop is kept rolled: one copy of
// the staple code serves every direction, which keeps the kernel inside the
// instruction cache.
template <class F>
__device__ __forceinline__ Herm8<typename F::Real> link_force(const F& in, const Geo& g, int s, const int c[4],
                                                              int mu, M3<typename F::Real>& u) {
    using R = typename F::Real;
    M3<R> omega;
    mzero(omega);
    const int cmu = g.coord(c, mu);
    const int s_pm = g.hop_rt(s, cmu, mu, +1);
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const int cnu = g.coord(c, nu);
        const int s_pn = g.hop_rt(s, cnu, nu, +1);
        const int s_mn = g.hop_rt(s, cnu, nu, -1);
        const int s_pm_mn = g.hop_rt(s_mn, cmu, mu, +1);
        if (kTwoRowStaples<R>::value) {
            {  // upper staple U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
                Rows2<R> t, st;
                {
                    const Rows2<R> a = in.load_rows2(nu, s_pm);
                    const M3<R> b = in.load(mu, s_pn);
                    mmul_rows2<false, true>(a, b, t);
                }
                const M3<R> d = in.load(nu, s);
                mmul_rows2<false, true>(t, d, st);
                madd_su3_rows2(omega, st);
            }
            {  // lower staple U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
                Rows2<R> t, st;
                {
                    const M3<R> a = in.load(nu, s_pm_mn);
                    const M3<R> b = in.load(mu, s_mn);
                    mmul_rows2<true, true>(a, b, t);
                }
                const M3<R> d = in.load(nu, s_mn);
                mmul_rows2<false, false>(t, d, st);
                madd_su3_rows2(omega, st);
            }
        } else {
            {  // upper staple, all three rows
                M3<R> t;
                {
                    const M3<R> a = in.load(nu, s_pm);
                    const M3<R> b = in.load(mu, s_pn);
                    mmul<false, true>(a, b, t);
                }
                const M3<R> d = in.load(nu, s);
                mmul_acc<false, true>(t, d, omega);
            }
            {  // lower staple, all three rows
                M3<R> t;
                {
                    const M3<R> a = in.load(nu, s_pm_mn);
                    const M3<R> b = in.load(mu, s_mn);
                    mmul<true, true>(a, b, t);
                }
                const M3<R> d = in.load(nu, s_mn);
                mmul_acc<false, false>(t, d, omega);
            }
        }
    }
    u = in.load(mu, s);
    return force_from_u_omega(u, omega);
}

// One link through one RK3 stage: generator, RK combination with the stored
// generator, e^{i eps_s Z} and the update of the link from `in` into `out`.
// Where a slab's new boundary links also go, for a time slab of a decomposed
// configuration: the neighbouring slabs' output buffers of the same stage
// (peer pointers when they sit on other GPUs).  Local slice 1 is the lower
// slab's upper halo (its slice lower_t = its nt + 1), local slice nt the upper
// slab's lower halo (its slice 0).  A slab's own kernel never writes its
// halo slices, so these stores race with nothing.
template <class F>
struct HaloTargets {
    F lower, upper;
    int slice_sites;  // sites per time slice (a multiple of 32)
    int nt;           // this slab's interior slices
    int lower_t;
};

// The rest of a link's stage once its generator dz = D_mu(x) is known: the RK
// combination with the stored generator, e^{i eps_s Z} and the new link
// e^{i eps_s Z} U stored into `out` (returned for the halo stores).
template <class F, int STAGE>
__device__ __forceinline__ Rows2<typename F::Real> rk_finish(const F& out, const ForceField<typename F::Real>& zf,
                                                            typename F::Real eps, int s, int mu,
                                                            const Herm8<typename F::Real>& dz,
                                                            const M3<typename F::Real>& u) {
    using R = typename F::Real;
    Herm8<R> z;
    if (STAGE == 0) {
        z = dz;
        zf.store(mu, s, z);
    } else if (STAGE == 1) {
        z = h8_axpby(R(8.0 / 9.0), dz, R(17.0 / 36.0), zf.load(mu, s));
        zf.store(mu, s, z);
    } else {
        z = h8_axpby(R(3.0 / 4.0), dz, R(1.0), zf.load(mu, s));
    }
    const Herm8<R> q = h8_scale(eps, z);
    Rows2<R> d, un;
    expm1_iq_rows2(q, d);
    mmul_rows2<false, false>(d, u, un);  // e^{iQ} U = U + (e^{iQ} - 1) U is in SU(3): two rows suffice
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            un.e[i][j].re += u.e[i][j].re;
            un.e[i][j].im += u.e[i][j].im;
        }
    out.store_rows2(mu, s, un);
    return un;
}

template <class F, int STAGE, bool HALO>
__device__ __forceinline__ void rk_link_update_to(const F& in, const F& out, const ForceField<typename F::Real>& zf,
                                                  const Geo& g, typename F::Real eps, int s, int mu,
                                                  const HaloTargets<F>& h) {
    using R = typename F::Real;
    int c[4];
    g.coords(s, c);
    M3<R> u;
    const Herm8<R> dz = link_force(in, g, s, c, mu, u);
    const Rows2<R> un = rk_finish<F, STAGE>(out, zf, eps, s, mu, dz, u);
    if constexpr (HALO) {
        if (c[3] == 1) h.lower.store_rows2(mu, h.lower_t * h.slice_sites + (s - h.slice_sites), un);
        if (c[3] == h.nt) h.upper.store_rows2(mu, s - h.nt * h.slice_sites, un);
    }
}

template <class F, int STAGE>
__device__ __forceinline__ void rk_link_update(const F& in, const F& out, const ForceField<typename F::Real>& zf,
                                               const Geo& g, typename F::Real eps, int s, int mu) {
    rk_link_update_to<F, STAGE, false>(in, out, zf, g, eps, s, mu, HaloTargets<F>{});
}

// ---------------------------------------------------------------------------
// The two-kernel stage (derivation in flow_split.cu): a field of the six plane
// generators H_p(x) = (i/2)[P_p(x) - P_p(x)^+]_TL per site, then each link's
//   D_mu(x) = sum_{nu != mu} s_{mu nu} [ H_p(x) - U_nu(y)^+ H_p(y) U_nu(y) ],  y = x - nu.
// ---------------------------------------------------------------------------

// plane index of directions a < b: (0,1) (0,2) (0,3) (1,2) (1,3) (2,3) -> 0..5
__device__ __forceinline__ int plane_index(int a, int b) { return a * (5 - a) / 2 + b - 1; }

// directions a < b of plane p
__device__ __forceinline__ int plane_a(int p) { return p < 3 ? 0 : (p < 5 ? 1 : 2); }
__device__ __forceinline__ int plane_b(int p) { return p < 3 ? p + 1 : (p < 5 ? p - 1 : 3); }

// H_ab(x) = (i/2)[P_ab(x) - P_ab(x)^+]_TL at site s with coordinates c.
template <class F>
__device__ __forceinline__ Herm8<typename F::Real> plane_generator(const F& u, const Geo& g, int s, const int c[4],
                                                                   int a, int b) {
    using R = typename F::Real;
    const int s_pa = g.hop_rt(s, g.coord(c, a), a, +1);
    const int s_pb = g.hop_rt(s, g.coord(c, b), b, +1);
    // lo = U_a(x) U_b(x+a) and up = U_b(x) U_a(x+b) (P = lo up^+), each
    // through its first two rows: rows 0 and 1 of the left link times the
    // right link; up's row 2 = conj(row0 x row1), and of P only rows 0 and 1
    // are multiplied out (its row 2 from their cross product), so lo's row 2
    // and the left links' rows 2 are never formed.  Against full-row
    // products: 36 of 162 multiply-adds per product fewer, and 25 per plane
    // in P; the FP32-12 plaquette-field kernel at 32^4 on B200 0.150 -> 0.126
    // ms (two-row products, both planes of a pair formed before either is
    // stored) -> 0.118 ms (P from its rows 0 and 1), |d(t^2 E)|/t^2 E
    // against FP64 at t = 4 unchanged (1.0e-7).
    Rows2<R> lo;
    M3<R> up;
    {
        const Rows2<R> x = u.load_rows2(a, s);
        const M3<R> y = u.load(b, s_pa);
        mmul_rows2<false, false>(x, y, lo);
    }
    {
        Rows2<R> t;
        const Rows2<R> x = u.load_rows2(b, s);
        const M3<R> y = u.load(a, s_pb);
        mmul_rows2<false, false>(x, y, t);
        full_from_rows2(t, up);
    }
    return force_from_b2_cdag(lo, up);
}

// H_p(x) of plane p at site s into hf.
template <class F>
__device__ __forceinline__ void plaq_plane(const F& u, const ForceField<typename F::Real>& hf, const Geo& g, int s,
                                           int p) {
    int c[4];
    g.coords(s, c);
    hf.store(p, s, plane_generator(u, g, s, c, plane_a(p), plane_b(p)));
}

// One link through one stage with its generator built from the plane field hf
// (which holds the plane generators of `in`); HALO: a slab's boundary links
// also go into its neighbours' halos, as in rk_link_update_to.
template <class F, int STAGE, bool HALO>
__device__ __forceinline__ void split_link_update_to(const F& in, const F& out,
                                                     const ForceField<typename F::Real>& zf,
                                                     const ForceField<typename F::Real>& hf, const Geo& g,
                                                     typename F::Real eps, int s, int mu, const HaloTargets<F>& h) {
    using R = typename F::Real;
    int c[4];
    g.coords(s, c);
    Herm8<R> d;
    d.d0 = d.d1 = R(0);
    d.z01 = d.z02 = d.z12 = cx(R(0), R(0));
    // The three directions nu != mu in ascending order, unrolled so that the
    // next direction's link and plane-generator loads issue during this one's
    // conjugation: 6.7 % off the FP32-12 stage kernel at 32^4 on B200 (0.183 ->
    // 0.171 ms per launch) at the same 64 registers; the staple form's loop
    // stays rolled (three copies of its code miss the instruction cache).
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int nu = k + (k >= mu ? 1 : 0);
        const int p = mu < nu ? plane_index(mu, nu) : plane_index(nu, mu);
        const R sg = mu < nu ? R(1) : R(-1);
        const int y = g.hop_rt(s, g.coord(c, nu), nu, -1);
        const M3<R> v = in.load(nu, y);
        const Herm8<R> lower = herm_conj_by(v, hf.load_ro(p, y));
        const Herm8<R> upper = hf.load_ro(p, s);
        d.d0 = fma(sg, upper.d0 - lower.d0, d.d0);
        d.d1 = fma(sg, upper.d1 - lower.d1, d.d1);
        d.z01 = cx(fma(sg, upper.z01.re - lower.z01.re, d.z01.re), fma(sg, upper.z01.im - lower.z01.im, d.z01.im));
        d.z02 = cx(fma(sg, upper.z02.re - lower.z02.re, d.z02.re), fma(sg, upper.z02.im - lower.z02.im, d.z02.im));
        d.z12 = cx(fma(sg, upper.z12.re - lower.z12.re, d.z12.re), fma(sg, upper.z12.im - lower.z12.im, d.z12.im));
    }
    const M3<R> uu = in.load(mu, s);
    const Rows2<R> un = rk_finish<F, STAGE>(out, zf, eps, s, mu, d, uu);
    if constexpr (HALO) {
        if (c[3] == 1) h.lower.store_rows2(mu, h.lower_t * h.slice_sites + (s - h.slice_sites), un);
        if (c[3] == h.nt) h.upper.store_rows2(mu, s - h.nt * h.slice_sites, un);
    }
}

template <class F, int STAGE>
__device__ __forceinline__ void split_link_update(const F& in, const F& out, const ForceField<typename F::Real>& zf,
                                                  const ForceField<typename F::Real>& hf, const Geo& g,
                                                  typename F::Real eps, int s, int mu) {
    split_link_update_to<F, STAGE, false>(in, out, zf, hf, g, eps, s, mu, HaloTargets<F>{});
}

// Resident blocks of the two-kernel stage kernel: FP32 forms at 8 (64
// registers, 32 warps per SM): 0.98 ms per RK3 step for the 12-real form at
// 32^4 on B200 against 1.05 at the 76 registers of 6 blocks; FP64 at 4 (its
// fused kernel's budget).
// Resident 192-thread blocks per SM the plaquette-field kernels are compiled
// for: FP32 at 5 (64 registers, 30 warps per SM).  At 6 (56 registers, 8
// bytes spilled) the FP32-12 step at 32^4 on B200 ran 3 % faster in short
// bursts at full clock (0.787 -> 0.764 ms) but 1.5 % slower in the
// power-capped steady state of a long flow (0.855 -> 0.868 ms, 2000-step
// runs alternated on one GPU).  FP64 at 4 (80 registers, one plane per
// thread: 0.274 -> 0.266 ms per launch at 32^4 against the 146 registers the
// compiler takes unbounded; at 5 or 6 blocks it spills and the step goes
// 1.73 -> 1.85 / 2.13 ms).
template <class F>
struct PlaqMinBlocks {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 4 : 5;
};

template <class F>
struct SplitMinBlocks {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 4 : 8;
};

}  // namespace ym
