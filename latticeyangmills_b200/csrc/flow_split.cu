// K1 as two kernels: the RK3 stage of one configuration with its force built
// from a stored plaquette field.
//
// Each link's generator D_mu(x) = (i/2)[U Omega - (U Omega)^+]_TL
// (src/Actions/puregauge.cpp:36-79) is a sum over the six plaquettes through
// the link, each read from the link's own corner.  With
//   P_ab(x) = U_a(x) U_b(x+a) U_a(x+b)^+ U_b(x)^+,   a < b, six planes per site,
//   H_ab(x) = (i/2)[P_ab(x) - P_ab(x)^+]_TL          (Hermitian traceless, 8 reals),
// the upper loop of link (mu, x) in plane (mu, nu) is P_{mu nu}(x) and the lower
// loop is U_nu(y)^+ P_{mu nu}(y)^+ U_nu(y) with y = x - nu; P_{nu mu} = P_{mu nu}^+,
// and (i/2)[.]_TL commutes with the conjugation by a unitary matrix, so
//   D_mu(x) = sum_{nu != mu} s_{mu nu} [ H_p(x) - U_nu(y)^+ H_p(y) U_nu(y) ],
// with p the plane {mu, nu} and s_{mu nu} = +1 for mu < nu, -1 otherwise.
//
// plaq_field_kernel forms the six H_p(x) of every site (three SU(3) products
// each, 8 reals stored); rk_split_stage_kernel then builds D from three
// conjugations v^+ H v per link and finishes the stage as the fused kernel does.
// Per link that is 6 x 3 / 4 + 3 x (1 + 1/2) products' worth of multiply-adds
// in place of 13, for 2 x 6 x 8 reals of plaquette field per site written and
// read.
#include "flow_device.cuh"
#include "kernels.h"

namespace ym {

// plane index of directions a < b: (0,1) (0,2) (0,3) (1,2) (1,3) (2,3) -> 0..5
__device__ __forceinline__ int plane_index(int a, int b) { return a * (5 - a) / 2 + b - 1; }

// One thread per (site, plane): six warps cover 32 sites, warp w plane w.
template <class F>
__global__ void __launch_bounds__(192) plaq_field_kernel(F u, ForceField<typename F::Real> hf, Geo g) {
    using R = typename F::Real;
    const int p = int(threadIdx.x >> 5);
    const int s = g.site0 + int(blockIdx.x) * 32 + int(threadIdx.x & 31);
    if (s >= g.site1) return;
    const int a = p < 3 ? 0 : (p < 5 ? 1 : 2);
    const int b = p < 3 ? p + 1 : (p < 5 ? p - 1 : 3);
    int c[4];
    g.coords(s, c);
    const int s_pa = g.hop_rt(s, g.coord(c, a), a, +1);
    const int s_pb = g.hop_rt(s, g.coord(c, b), b, +1);
    M3<R> lo, up;  // U_a(x) U_b(x+a) and U_b(x) U_a(x+b): P = lo up^+
    {
        const M3<R> x = u.load(a, s);
        const M3<R> y = u.load(b, s_pa);
        mmul<false, false>(x, y, lo);
    }
    {
        const M3<R> x = u.load(b, s);
        const M3<R> y = u.load(a, s_pb);
        mmul<false, false>(x, y, up);
    }
    hf.store(p, s, force_from_b_cdag(lo, up));
}

// FP32 forms at 8 resident blocks (64 registers, 32 warps per SM): 0.98 ms per
// RK3 step for the 12-real form at 32^4 on B200 against 1.05 at the 76
// registers of 6 blocks; FP64 at 4 (its fused kernel's budget).
template <class F>
struct SplitMinBlocks {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 4 : 8;
};

template <class F, int STAGE>
__global__ void __launch_bounds__(128, SplitMinBlocks<F>::value)
    rk_split_stage_kernel(F in, F out, ForceField<typename F::Real> zf, ForceField<typename F::Real> hf, Geo g,
                          typename F::Real eps) {
    using R = typename F::Real;
    const int mu = int(threadIdx.x >> 5) & 3;
    const int s = g.site0 + int(blockIdx.x) * 32 + int(threadIdx.x & 31);
    if (s >= g.site1) return;
    int c[4];
    g.coords(s, c);
    Herm8<R> d;
    d.d0 = d.d1 = R(0);
    d.z01 = d.z02 = d.z12 = cx(R(0), R(0));
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
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
    rk_finish<F, STAGE>(out, zf, eps, s, mu, d, uu);
}

template <class F>
static cudaError_t launch_plaq_typed(const void* u, void* h, const Geo& g, cudaStream_t st) {
    F in{const_cast<void*>(u), g.V};
    ForceField<typename F::Real> hf{h, g.V};
    plaq_field_kernel<F><<<unsigned((g.site1 - g.site0 + 31) / 32), 192, 0, st>>>(in, hf, g);
    return cudaGetLastError();
}

template <class F>
static cudaError_t launch_split_typed(int stage, const void* uin, void* uout, void* z, const void* h, const Geo& g,
                                      double eps, cudaStream_t st) {
    using R = typename F::Real;
    F in{const_cast<void*>(uin), g.V}, out{uout, g.V};
    ForceField<R> zf{z, g.V}, hf{const_cast<void*>(h), g.V};
    const dim3 grid(unsigned((g.site1 - g.site0 + 31) / 32));
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    switch (stage) {
        case 0: rk_split_stage_kernel<F, 0><<<grid, 128, 0, st>>>(in, out, zf, hf, g, e); break;
        case 1: rk_split_stage_kernel<F, 1><<<grid, 128, 0, st>>>(in, out, zf, hf, g, e); break;
        default: rk_split_stage_kernel<F, 2><<<grid, 128, 0, st>>>(in, out, zf, hf, g, e); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_plaq_field(int prec, const void* u, void* h, const Geo& g, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_plaq_typed<FieldD18>(u, h, g, st);
        case kFP32_18: return launch_plaq_typed<FieldF18>(u, h, g, st);
        case kFP32_12: return launch_plaq_typed<FieldF12>(u, h, g, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_rk_split_stage(int prec, int stage, const void* uin, void* uout, void* z, const void* h,
                                  const Geo& g, double eps, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_split_typed<FieldD18>(stage, uin, uout, z, h, g, eps, st);
        case kFP32_18: return launch_split_typed<FieldF18>(stage, uin, uout, z, h, g, eps, st);
        case kFP32_12: return launch_split_typed<FieldF12>(stage, uin, uout, z, h, g, eps, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ym
