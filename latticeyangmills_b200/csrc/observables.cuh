// Device code of the observables (plaquette, clover energy, clover charge):
// per-site values, FP64 block partials and the fixed-order fold.  Shared by
// observables.cu and any kernel that needs the same reduction.
#pragma once
#include "field.cuh"
#include "su3.cuh"

namespace ym {

// anti-Hermitian traceless G as its imaginary diagonal and upper triangle
template <class R>
struct AH {
    R g0, g1, g2;
    Cx<R> g01, g02, g12;
};

template <class R>
__device__ __forceinline__ R ah_re_trace_mul(const AH<R>& a, const AH<R>& b) {
    // Re tr(A B) for anti-Hermitian A, B: -sum_i a_ii b_ii - 2 sum_{i<j} Re(A_ij conj(B_ij))
    R d = a.g0 * b.g0 + a.g1 * b.g1 + a.g2 * b.g2;
    R o = a.g01.re * b.g01.re + a.g01.im * b.g01.im + a.g02.re * b.g02.re + a.g02.im * b.g02.im +
          a.g12.re * b.g12.re + a.g12.im * b.g12.im;
    return -d - R(2) * o;
}

template <class R>
__device__ __forceinline__ AH<R> ah_of_clover(const M3<R>& cl) {
    AH<R> G;
    const R i0 = R(2) * cl.e[0][0].im, i1 = R(2) * cl.e[1][1].im, i2 = R(2) * cl.e[2][2].im;
    const R m = (i0 + i1 + i2) * R(1.0 / 3.0);
    G.g0 = i0 - m;
    G.g1 = i1 - m;
    G.g2 = i2 - m;
    G.g01 = cx(cl.e[0][1].re - cl.e[1][0].re, cl.e[0][1].im + cl.e[1][0].im);
    G.g02 = cx(cl.e[0][2].re - cl.e[2][0].re, cl.e[0][2].im + cl.e[2][0].im);
    G.g12 = cx(cl.e[1][2].re - cl.e[2][1].re, cl.e[1][2].im + cl.e[2][1].im);
    return G;
}

// G_{mu nu}(x) and Re tr Q1.  Each leaf (a product of four SU(3) links) is
// formed through its first two rows with the third rebuilt, in every
// precision: exact to the working precision's rounding for a measurement
// (unlike the flow's staples, nothing accumulates it over steps), 10 % off an
// FP32 evaluation at 32^4 on B200 (0.53 -> 0.48 ms) with the FP32 accuracy
// against FP64 unchanged, and within the FP64 kernel's registers.
template <class F>
__device__ __forceinline__ AH<typename F::Real> clover(const F& u, const Geo& g, int s, const int c[4], int MU, int NU,
                                                       typename F::Real& plaq) {
    using R = typename F::Real;
    const int cmu = g.coord(c, MU), cnu = g.coord(c, NU);
    const int s_pm = g.hop_rt(s, cmu, MU, +1), s_pn = g.hop_rt(s, cnu, NU, +1);
    const int s_mm = g.hop_rt(s, cmu, MU, -1), s_mn = g.hop_rt(s, cnu, NU, -1);
    const int s_mm_pn = g.hop_rt(s_mm, cnu, NU, +1), s_mm_mn = g.hop_rt(s_mm, cnu, NU, -1);
    const int s_pm_mn = g.hop_rt(s_pm, cnu, NU, -1);
    M3<R> cl;
    Rows2<R> t, w, l;
    {  // Q1
        mmul_rows2<false, false>(u.load_rows2(MU, s), u.load(NU, s_pm), t);
        mmul_rows2<false, true>(t, u.load(MU, s_pn), w);
        mmul_rows2<false, true>(w, u.load(NU, s), l);
        full_from_rows2(l, cl);
        plaq = re_trace(cl);
    }
    {  // Q2
        mmul_rows2<false, true>(u.load_rows2(NU, s), u.load(MU, s_mm_pn), t);
        mmul_rows2<false, true>(t, u.load(NU, s_mm), w);
        mmul_rows2<false, false>(w, u.load(MU, s_mm), l);
        madd_su3_rows2(cl, l);
    }
    {  // Q3
        mmul_rows2<true, true>(u.load(MU, s_mm), u.load(NU, s_mm_mn), t);
        mmul_rows2<false, false>(t, u.load(MU, s_mm_mn), w);
        mmul_rows2<false, false>(w, u.load(NU, s_mn), l);
        madd_su3_rows2(cl, l);
    }
    {  // Q4
        mmul_rows2<true, false>(u.load(NU, s_mn), u.load(MU, s_mn), t);
        mmul_rows2<false, false>(t, u.load(NU, s_pm_mn), w);
        mmul_rows2<false, true>(w, u.load(MU, s), l);
        madd_su3_rows2(cl, l);
    }
    return ah_of_clover(cl);
}

// The planes in the pairs (01,23), (02,13), (03,12); the pair loop is kept
// rolled so one copy of the clover code serves all six planes.
template <class F>
__device__ __forceinline__ void site_observables(const F& u, const Geo& g, int s, double& plaq, double& energy,
                                                 double& topc) {
    using R = typename F::Real;
    int c[4];
    g.coords(s, c);
    double q = 0.0;
#pragma unroll 1
    for (int k = 0; k < 3; k++) {
        const int mu_b = k == 0 ? 2 : 1;
        const int nu_a = k + 1, nu_b = k == 0 ? 3 : (k == 1 ? 3 : 2);
        R p;
        const AH<R> a = clover(u, g, s, c, 0, nu_a, p);
        plaq += double(p);
        energy += double(ah_re_trace_mul(a, a));
        const AH<R> b = clover(u, g, s, c, mu_b, nu_b, p);
        plaq += double(p);
        energy += double(ah_re_trace_mul(b, b));
        // Re tr(G01 G23), Re tr(G02 G13^+) = -Re tr(G02 G13), Re tr(G03 G12)
        const double t = double(ah_re_trace_mul(a, b));
        q += k == 1 ? -t : t;
    }
    topc -= q;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sums three values over the block; thread 0 gets the totals.
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c) {
    __shared__ double sh[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
        sh[2][wid] = c;
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (wid == 0) {
        a = lane < nw ? sh[0][lane] : 0.0;
        b = lane < nw ? sh[1][lane] : 0.0;
        c = lane < nw ? sh[2][lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
    }
}

// One thread per site, the three plane pairs in a loop; block partials, one
// per block of sites (the allocation-free entry point's form, whose scratch
// is sized by it).
template <class F>
__global__ void __launch_bounds__(256) observables_site_kernel(F u, Geo g, double* partials) {
    const int s = g.site0 + int(blockIdx.x) * blockDim.x + threadIdx.x;
    double plaq = 0.0, energy = 0.0, topc = 0.0;
    if (s < g.site1) site_observables(u, g, s, plaq, energy, topc);
    block_sum3(plaq, energy, topc);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x + 0] = plaq;
        partials[3 * blockIdx.x + 1] = energy;
        partials[3 * blockIdx.x + 2] = topc;
    }
}

// One thread per (site, plane): six warps per 32 sites, warp p building the
// clover of plane p = (01, 02, 03, 12, 13, 23) for its 32 sites, so one
// clover is live per thread.  Holding a plane pair per thread (the site form
// above) needs 188 registers in FP64: 8 warps per SM.  Planes 12, 13, 23 leave
// their G in shared memory for the charge pairs (03,12), (02,13), (01,23).
// The grid is at most kObsMaxBlocks blocks that stride over the 32-site
// groups, so the partials do not grow with the volume; the sums are
// deterministic for a given grid.
constexpr int kObsSites = 32;
constexpr int kObsThreads = 6 * kObsSites;
constexpr int kObsMaxBlocks = 148 * 8;

// Two resident blocks (12 warps) per SM: FP64 168 registers, FP32 143-165, no
// spills to speak of.  Measured per evaluation against the site-per-thread
// form: FP64 32^4 0.91 -> 0.78 ms, 16^3x32 0.145 -> 0.114 ms; FP32-18 32^4
// 0.44 -> 0.46 ms; 8^4 0.036-0.045 -> 0.032 ms (three blocks spill in FP32).
constexpr int kObsMinBlocks = 2;

template <class F>
__global__ void __launch_bounds__(kObsThreads, kObsMinBlocks)
    observables_kernel(F u, Geo g, double* partials) {
    using R = typename F::Real;
    __shared__ R gb[3][9][32];
    const int p = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int MU = p < 3 ? 0 : (p < 5 ? 1 : 2);
    const int NU = p < 3 ? p + 1 : (p == 3 ? 2 : 3);
    const int groups = (g.site1 - g.site0 + kObsSites - 1) / kObsSites;
    double plaq = 0.0, energy = 0.0, topc = 0.0;
    for (int grp = blockIdx.x; grp < groups; grp += gridDim.x) {  // block-uniform trip count
        int s = g.site0 + grp * kObsSites + lane;
        bool active = s < g.site1;
        if (!active) s = g.site0;  // computed but not counted: every thread reaches the barriers
        int c[4];
        g.coords(s, c);
        active = active && g.interior(c);  // a block's halo sites are its neighbours'
        R pl;
        const AH<R> G = clover(u, g, s, c, MU, NU, pl);
        if (active) {
            plaq += double(pl);
            energy += double(ah_re_trace_mul(G, G));
        }
        if (p >= 3) {
            R* d = &gb[p - 3][0][lane];
            d[0] = G.g0;
            d[32] = G.g1;
            d[64] = G.g2;
            d[96] = G.g01.re;
            d[128] = G.g01.im;
            d[160] = G.g02.re;
            d[192] = G.g02.im;
            d[224] = G.g12.re;
            d[256] = G.g12.im;
        }
        __syncthreads();
        if (p < 3 && active) {
            // topc = -(Re tr(G01 G23) - Re tr(G02 G13) + Re tr(G03 G12)): plane p meets slot 2 - p
            const R* d = &gb[2 - p][0][lane];
            AH<R> B;
            B.g0 = d[0];
            B.g1 = d[32];
            B.g2 = d[64];
            B.g01 = cx(d[96], d[128]);
            B.g02 = cx(d[160], d[192]);
            B.g12 = cx(d[224], d[256]);
            const double t = double(ah_re_trace_mul(G, B));
            topc += p == 1 ? t : -t;
        }
        __syncthreads();  // the slots are rewritten by the next group
    }
    block_sum3(plaq, energy, topc);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x + 0] = plaq;
        partials[3 * blockIdx.x + 1] = energy;
        partials[3 * blockIdx.x + 2] = topc;
    }
}

}  // namespace ym
