// K1: one fused kernel per RK3 stage of the Wilson flow.
//
// Per link (x, mu), one thread:
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
// field, so links are read from `uin` and written to `uout` (ping-pong).  Z is
// written by stages 0 and 1 and read by stages 1 and 2.  The direction mu is
// the grid's y index, uniform per block, and is a template parameter of the
// link body so every neighbour offset is resolved at compile time.
#include "expsu3.cuh"
#include "kernels.h"

namespace ym {

// D_mu(x) = (i/2)[U Omega - (U Omega)^+]_traceless for one link; also returns U_mu(x).
template <class F, int MU>
__device__ __forceinline__ Herm8<typename F::Real> link_force(const F& in, const Geo& g, int64_t s, const int c[4],
                                                              M3<typename F::Real>& u) {
    using R = typename F::Real;
    M3<R> omega;
    mzero(omega);
#pragma unroll
    for (int nu = 0; nu < 4; nu++) {
        if (nu == MU) continue;
        const int64_t s_pm = g.hop(s, c, MU, +1);
        const int64_t s_pn = g.hop(s, c, nu, +1);
        const int64_t s_mn = g.hop(s, c, nu, -1);
        const int64_t s_pm_mn = g.hop(s_mn, c, MU, +1);
        {
            M3<R> t;
            {
                const M3<R> a = in.load(nu, s_pm);
                const M3<R> b = in.load(MU, s_pn);
                mmul<false, true>(a, b, t);
            }
            const M3<R> d = in.load(nu, s);
            mmul_acc<false, true>(t, d, omega);
        }
        {
            M3<R> t;
            {
                const M3<R> a = in.load(nu, s_pm_mn);
                const M3<R> b = in.load(MU, s_mn);
                mmul<true, true>(a, b, t);
            }
            const M3<R> d = in.load(nu, s_mn);
            mmul_acc<false, false>(t, d, omega);
        }
    }
    u = in.load(MU, s);
    M3<R> x;
    mmul<false, false>(u, omega, x);
    return force_from_x(x);
}

template <class F, int STAGE, int MU>
__device__ __forceinline__ void rk_link(const F& in, const F& out, const ForceField<typename F::Real>& zf,
                                        const Geo& g, typename F::Real eps, int64_t s) {
    using R = typename F::Real;
    int c[4];
    g.coords(s, c);
    M3<R> u;
    const Herm8<R> dz = link_force<F, MU>(in, g, s, c, u);
    Herm8<R> z;
    if (STAGE == 0) {
        z = dz;
        zf.store(MU, s, z);
    } else if (STAGE == 1) {
        z = h8_axpby(R(8.0 / 9.0), dz, R(17.0 / 36.0), zf.load(MU, s));
        zf.store(MU, s, z);
    } else {
        z = h8_axpby(R(3.0 / 4.0), dz, R(1.0), zf.load(MU, s));
    }
    const Herm8<R> q = h8_scale(eps, z);
    M3<R> e;
    exp_iq(q, e);
    M3<R> un;
    mmul<false, false>(e, u, un);
    out.store(MU, s, un);
}

template <class F, int STAGE>
__global__ void __launch_bounds__(256) rk_stage_kernel(F in, F out, ForceField<typename F::Real> zf, Geo g,
                                                        typename F::Real eps) {
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    switch (blockIdx.y) {
        case 0: rk_link<F, STAGE, 0>(in, out, zf, g, eps, s); break;
        case 1: rk_link<F, STAGE, 1>(in, out, zf, g, eps, s); break;
        case 2: rk_link<F, STAGE, 2>(in, out, zf, g, eps, s); break;
        default: rk_link<F, STAGE, 3>(in, out, zf, g, eps, s); break;
    }
}

template <class F>
static cudaError_t launch_typed(int stage, const void* uin, void* uout, void* z, const Geo& g, double eps, int block,
                                cudaStream_t st) {
    using R = typename F::Real;
    F in{(typename F::V2*)uin, g.V}, out{(typename F::V2*)uout, g.V};
    ForceField<R> zf{(R*)z, g.V};
    dim3 grid(unsigned((g.V + block - 1) / block), 4);
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
template <class F, int MU>
__global__ void __launch_bounds__(128) force_kernel(F in, Geo g, double* out) {
    using R = typename F::Real;
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    int c[4];
    g.coords(s, c);
    M3<R> u;
    const Herm8<R> z = link_force<F, MU>(in, g, s, c, u);
    double* o = out + 18 * s;
    const double d0 = double(z.d0), d1 = double(z.d1), d2 = -(d0 + d1);
    o[0] = d0; o[1] = 0.0; o[8] = d1; o[9] = 0.0; o[16] = d2; o[17] = 0.0;
    o[2] = double(z.z01.re); o[3] = double(z.z01.im); o[6] = double(z.z01.re); o[7] = -double(z.z01.im);
    o[4] = double(z.z02.re); o[5] = double(z.z02.im); o[12] = double(z.z02.re); o[13] = -double(z.z02.im);
    o[10] = double(z.z12.re); o[11] = double(z.z12.im); o[14] = double(z.z12.re); o[15] = -double(z.z12.im);
}

template <class F>
static cudaError_t launch_force_typed(int mu, const void* u, const Geo& g, double* out, cudaStream_t st) {
    F in{(typename F::V2*)u, g.V};
    const int b = 128;
    const unsigned nb = unsigned((g.V + b - 1) / b);
    switch (mu) {
        case 0: force_kernel<F, 0><<<nb, b, 0, st>>>(in, g, out); break;
        case 1: force_kernel<F, 1><<<nb, b, 0, st>>>(in, g, out); break;
        case 2: force_kernel<F, 2><<<nb, b, 0, st>>>(in, g, out); break;
        default: force_kernel<F, 3><<<nb, b, 0, st>>>(in, g, out); break;
    }
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
