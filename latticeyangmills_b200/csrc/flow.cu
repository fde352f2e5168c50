// K1: one fused kernel per RK3 stage of the Wilson flow over one configuration
// (the link body is in flow_device.cuh), plus the force and exponential
// kernels behind ymflow_derivative and ymflow_su3_exp.
#include "flow_device.cuh"
#include "kernels.h"

namespace ym {

// Thread layout: a block covers blockDim/4 sites; warp w works on direction
// mu = w & 3 for 32 consecutive sites, so the four directions of a site range
// run side by side and share their neighbour links through L1/L2 (a grid that
// sweeps all sites once per direction streams the field through L2 four times).
// TILED: the block order of Geo::block_group (FP64 stage kernels); otherwise
// blocks take consecutive groups.
template <bool TILED>
__device__ __forceinline__ void link_of_thread(const Geo& g, int& s, int& mu) {
    const int w = threadIdx.x >> 5;
    mu = w & 3;
    const int b = TILED ? g.block_group(int(blockIdx.x)) : int(blockIdx.x);
    s = g.site0 + b * 32 + (threadIdx.x & 31);  // 128 threads: one 32-site group per block
}

template <class F, int STAGE>
__global__ void __launch_bounds__(128, StageMinBlocks<F>::value)
    rk_stage_kernel(F in, F out, ForceField<typename F::Real> zf, Geo g, typename F::Real eps) {
    int s;
    int mu;
    link_of_thread<sizeof(typename F::Real) == 8>(g, s, mu);
    if (s >= g.site1) return;
    rk_link_update<F, STAGE>(in, out, zf, g, eps, s, mu);
}

// The same stage for a slab whose boundary links also go straight into its
// neighbours' halos: the halo exchange fused into the stage.
template <class F, int STAGE>
__global__ void __launch_bounds__(128, StageMinBlocks<F>::value)
    rk_stage_halo_kernel(F in, F out, ForceField<typename F::Real> zf, Geo g, typename F::Real eps,
                         HaloTargets<F> h) {
    int s;
    int mu;
    link_of_thread<false>(g, s, mu);  // slabs: plain order
    if (s >= g.site1) return;
    rk_link_update_to<F, STAGE, true>(in, out, zf, g, eps, s, mu, h);
}

template <class F>
static cudaError_t launch_halo_typed(int stage, const void* uin, void* uout, void* z, const Geo& g, double eps,
                                     void* lower_out, int lower_v, int lower_t, void* upper_out, int upper_v,
                                     cudaStream_t st) {
    using R = typename F::Real;
    F in{const_cast<void*>(uin), g.V}, out{uout, g.V};
    ForceField<R> zf{z, g.V};
    HaloTargets<F> h{F{lower_out, lower_v}, F{upper_out, upper_v}, g.site0, (g.site1 - g.site0) / g.site0, lower_t};
    dim3 grid(unsigned((g.site1 - g.site0 + 31) / 32));
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    switch (stage) {
        case 0: rk_stage_halo_kernel<F, 0><<<grid, 128, 0, st>>>(in, out, zf, g, e, h); break;
        case 1: rk_stage_halo_kernel<F, 1><<<grid, 128, 0, st>>>(in, out, zf, g, e, h); break;
        default: rk_stage_halo_kernel<F, 2><<<grid, 128, 0, st>>>(in, out, zf, g, e, h); break;
    }
    return cudaGetLastError();
}

template <class F>
static cudaError_t launch_typed(int stage, const void* uin, void* uout, void* z, const Geo& g, double eps, int block,
                                cudaStream_t st) {
    using R = typename F::Real;
    F in{const_cast<void*>(uin), g.V}, out{uout, g.V};
    ForceField<R> zf{z, g.V};
    const int sites_per_block = block / 4;
    dim3 grid(unsigned((g.site1 - g.site0 + sites_per_block - 1) / sites_per_block));
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    switch (stage) {
        case 0: rk_stage_kernel<F, 0><<<grid, block, 0, st>>>(in, out, zf, g, e); break;
        case 1: rk_stage_kernel<F, 1><<<grid, block, 0, st>>>(in, out, zf, g, e); break;
        default: rk_stage_kernel<F, 2><<<grid, block, 0, st>>>(in, out, zf, g, e); break;
    }
    return cudaGetLastError();
}

// D_mu of every site as full 3x3 matrices (18 doubles per site, site order):
// PureGauge::computeDerivative(mu) (src/Actions/puregauge.cpp:62-79).
template <class F>
__global__ void __launch_bounds__(128) force_kernel(F in, Geo g, int mu, double* out) {
    using R = typename F::Real;
    const int s = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    g.coords(s, c);
    M3<R> u;
    const Herm8<R> z = link_force(in, g, s, c, mu, u);
    double* o = out + 18 * int64_t(s);
    const double d0 = double(z.d0), d1 = double(z.d1), d2 = -(d0 + d1);
    o[0] = d0; o[1] = 0.0; o[8] = d1; o[9] = 0.0; o[16] = d2; o[17] = 0.0;
    o[2] = double(z.z01.re); o[3] = double(z.z01.im); o[6] = double(z.z01.re); o[7] = -double(z.z01.im);
    o[4] = double(z.z02.re); o[5] = double(z.z02.im); o[12] = double(z.z02.re); o[13] = -double(z.z02.im);
    o[10] = double(z.z12.re); o[11] = double(z.z12.im); o[14] = double(z.z12.re); o[15] = -double(z.z12.im);
}

template <class F>
static cudaError_t launch_force_typed(int mu, const void* u, const Geo& g, double* out, cudaStream_t st) {
    F in{const_cast<void*>(u), g.V};
    const int b = 128;
    const unsigned nb = unsigned((g.V + b - 1) / b);
    force_kernel<F><<<nb, b, 0, st>>>(in, g, mu, out);
    return cudaGetLastError();
}

cudaError_t launch_force(int prec, int mu, const void* u, const Geo& g, double* out, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_force_typed<FieldD18>(mu, u, g, out, st);
        case kFP32_18: return launch_force_typed<FieldF18>(mu, u, g, out, st);
        case kFP32_12: return launch_force_typed<FieldF12>(mu, u, g, out, st);
        default: return cudaErrorInvalidValue;
    }
}

// e^{iQ} of n Hermitian traceless matrices given as 18 doubles each (only the
// diagonal d0, d1 and the upper triangle are read; q22 = -(d0 + d1)).
__global__ void exp_kernel(const double* q, double* r, int64_t n) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = q + 18 * i;
    Herm8<double> h;
    h.d0 = a[0];
    h.d1 = a[8];
    h.z01 = cx(a[2], a[3]);
    h.z02 = cx(a[4], a[5]);
    h.z12 = cx(a[10], a[11]);
    M3<double> e;
    exp_iq(h, e);
    double* o = r + 18 * i;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        o[2 * k] = e.e[k / 3][k % 3].re;
        o[2 * k + 1] = e.e[k / 3][k % 3].im;
    }
}

cudaError_t launch_exp(const double* q, double* r, int64_t n, cudaStream_t st) {
    const int b = 128;
    exp_kernel<<<unsigned((n + b - 1) / b), b, 0, st>>>(q, r, n);
    return cudaGetLastError();
}

cudaError_t launch_rk_stage_halo(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g, double eps,
                                 void* lower_out, int lower_v, int lower_t, void* upper_out, int upper_v,
                                 cudaStream_t st) {
    if (g.site0 <= 0 || g.site0 % 32 || (g.site1 - g.site0) % g.site0) return cudaErrorInvalidValue;
    switch (prec) {
        case kFP64:
            return launch_halo_typed<FieldD18>(stage, uin, uout, z, g, eps, lower_out, lower_v, lower_t, upper_out,
                                               upper_v, st);
        case kFP32_18:
            return launch_halo_typed<FieldF18>(stage, uin, uout, z, g, eps, lower_out, lower_v, lower_t, upper_out,
                                               upper_v, st);
        case kFP32_12:
            return launch_halo_typed<FieldF12>(stage, uin, uout, z, g, eps, lower_out, lower_v, lower_t, upper_out,
                                               upper_v, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_rk_stage(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g, double eps,
                            int block, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_typed<FieldD18>(stage, uin, uout, z, g, eps, block, st);
        case kFP32_18: return launch_typed<FieldF18>(stage, uin, uout, z, g, eps, block, st);
        case kFP32_12: return launch_typed<FieldF12>(stage, uin, uout, z, g, eps, block, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ym
