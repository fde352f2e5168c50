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
// conjugations v^+ H v per link and finishes the stage as the fused kernel does
// (device code in flow_device.cuh, shared with the ensemble kernels).
// Per link that is 6 x 3 / 4 + 3 x (1 + 1/2) products' worth of multiply-adds
// in place of 13, for 2 x 6 x 8 reals of plaquette field per site written and
// read.
#include "flow_device.cuh"
#include "kernels.h"

namespace ym {

// Planes per thread of the plaquette-field kernel (below): two for the FP32
// forms; one in FP64, where a pair needs 132 registers (2 blocks of 6 warps
// per SM) and a single plane 80: at 32^4 on B200 the FP64 field kernel runs
// 0.294 -> 0.270 ms per launch, the two-kernel FP64 step 1.80 -> 1.73 ms.
template <class F>
struct PlaqPlanesPerThread {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 1 : 2;
};

// One thread per (site, pair of planes): six warps cover 64 sites, warps
// 3k .. 3k + 2 the planes {(0,1), (0,2)}, {(0,3), (1,3)}, {(1,2), (2,3)} of
// site group k (the two planes of a pair share one of the site's links,
// loaded once).  The second plane's loads issue during the first plane's
// products: against one plane per thread, the FP32-18 kernel ran 16 % faster
// at 32^4 on B200 (0.180 -> 0.151 ms), the 12-real one 1.6 % (0.148 -> 0.146).
// With one plane per thread (PlaqPlanesPerThread 1) six warps cover 32 sites,
// warp w plane w.

template <class F>
__global__ void __launch_bounds__(192, PlaqMinBlocks<F>::value) plaq_field_kernel(F u, ForceField<typename F::Real> hf, Geo g) {
    const int w = int(threadIdx.x >> 5);
    // FP32: blocks walk the lattice from its end, so the stage kernel that
    // follows starts at site 0, whose links and plane generators this launch
    // touched last and are still in L2: 1 % off the FP32-12 step at 32^4 on
    // B200, in bursts (0.7535 -> 0.747 ms) and in the power-capped steady
    // state (0.886 -> 0.878); in FP64 the field kernel itself runs 9 % slower
    // that way (0.274 -> 0.298 ms), so FP64 keeps the ascending order
    const int blk = sizeof(typename F::Real) == 4 ? int(gridDim.x - 1 - blockIdx.x) : int(blockIdx.x);
    int c[4];
    if (PlaqPlanesPerThread<F>::value == 1) {
        const int s = g.site0 + blk * 32 + int(threadIdx.x & 31);
        if (s >= g.site1) return;
        g.coords(s, c);
        hf.store(w, s, plane_generator(u, g, s, c, plane_a(w), plane_b(w)));
        return;
    }
    const int s = g.site0 + (blk * 2 + w / 3) * 32 + int(threadIdx.x & 31);
    if (s >= g.site1) return;
    const int pr = w % 3;
    const int p0 = pr == 0 ? 0 : (pr == 1 ? 2 : 3);
    const int p1 = pr == 0 ? 1 : (pr == 1 ? 4 : 5);
    g.coords(s, c);
    // both planes before either store: the link the two share is loaded once
    const auto h0 = plane_generator(u, g, s, c, plane_a(p0), plane_b(p0));
    const auto h1 = plane_generator(u, g, s, c, plane_a(p1), plane_b(p1));
    hf.store(p0, s, h0);
    hf.store(p1, s, h1);
}

// One thread per link: four warps (directions) per 32 sites.
template <class F, int STAGE>
__global__ void __launch_bounds__(128, SplitMinBlocks<F>::value)
    rk_split_stage_kernel(F in, F out, ForceField<typename F::Real> zf, ForceField<typename F::Real> hf, Geo g,
                          typename F::Real eps) {
    const int mu = int(threadIdx.x >> 5) & 3;
    const int s = g.site0 + int(blockIdx.x) * 32 + int(threadIdx.x & 31);
    if (s >= g.site1) return;
    split_link_update<F, STAGE>(in, out, zf, hf, g, eps, s, mu);
}

// The same for a time slab, storing its boundary links into its neighbours'
// halos (the two-kernel form of rk_stage_halo_kernel).
template <class F, int STAGE>
__global__ void __launch_bounds__(128, SplitMinBlocks<F>::value)
    rk_split_stage_halo_kernel(F in, F out, ForceField<typename F::Real> zf, ForceField<typename F::Real> hf, Geo g,
                               typename F::Real eps, HaloTargets<F> h) {
    const int mu = int(threadIdx.x >> 5) & 3;
    const int s = g.site0 + int(blockIdx.x) * 32 + int(threadIdx.x & 31);
    if (s >= g.site1) return;
    split_link_update_to<F, STAGE, true>(in, out, zf, hf, g, eps, s, mu, h);
}

template <class F>
static cudaError_t launch_split_halo_typed(int stage, const void* uin, void* uout, void* z, const void* hp,
                                           const Geo& g, double eps, void* lower_out, int lower_v, int lower_t,
                                           void* upper_out, int upper_v, cudaStream_t st) {
    using R = typename F::Real;
    F in{const_cast<void*>(uin), g.V}, out{uout, g.V};
    ForceField<R> zf{z, g.V}, hf{const_cast<void*>(hp), g.V};
    HaloTargets<F> h{F{lower_out, lower_v}, F{upper_out, upper_v}, g.site0, (g.site1 - g.site0) / g.site0, lower_t};
    const dim3 grid(unsigned((g.site1 - g.site0 + 31) / 32));
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    switch (stage) {
        case 0: rk_split_stage_halo_kernel<F, 0><<<grid, 128, 0, st>>>(in, out, zf, hf, g, e, h); break;
        case 1: rk_split_stage_halo_kernel<F, 1><<<grid, 128, 0, st>>>(in, out, zf, hf, g, e, h); break;
        default: rk_split_stage_halo_kernel<F, 2><<<grid, 128, 0, st>>>(in, out, zf, hf, g, e, h); break;
    }
    return cudaGetLastError();
}

template <class F>
static cudaError_t launch_plaq_typed(const void* u, void* h, const Geo& g, cudaStream_t st) {
    F in{const_cast<void*>(u), g.V};
    ForceField<typename F::Real> hf{h, g.V};
    const unsigned groups = unsigned((g.site1 - g.site0 + 31) / 32);
    plaq_field_kernel<F><<<PlaqPlanesPerThread<F>::value == 1 ? groups : (groups + 1) / 2, 192, 0, st>>>(in, hf, g);
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

cudaError_t launch_rk_split_stage_halo(int prec, int stage, const void* uin, void* uout, void* z, const void* h,
                                       const Geo& g, double eps, void* lower_out, int lower_v, int lower_t,
                                       void* upper_out, int upper_v, cudaStream_t st) {
    if (g.site0 <= 0 || g.site0 % 32 || (g.site1 - g.site0) % g.site0) return cudaErrorInvalidValue;
    switch (prec) {
        case kFP64:
            return launch_split_halo_typed<FieldD18>(stage, uin, uout, z, h, g, eps, lower_out, lower_v, lower_t,
                                                     upper_out, upper_v, st);
        case kFP32_18:
            return launch_split_halo_typed<FieldF18>(stage, uin, uout, z, h, g, eps, lower_out, lower_v, lower_t,
                                                     upper_out, upper_v, st);
        case kFP32_12:
            return launch_split_halo_typed<FieldF12>(stage, uin, uout, z, h, g, eps, lower_out, lower_v, lower_t,
                                                     upper_out, upper_v, st);
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
