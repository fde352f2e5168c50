// Gauge-field generation on the device: Metropolis updates of the Wilson
// action, the step before the flow.  The reference's generator app
// (src/Apps/gaugefieldfactory.cpp:192-220) does not compile and draws from an
// unseedable generator; this restates its intended update with a seeded,
// counter-based random stream:
//
//   per link, `hits` proposals U' = X U with X a product R S T of three SU(2)
//   elements embedded in the (0,1), (0,2), (1,2) blocks, each with
//   x0 = +-sqrt(1 - eps^2) (sign of a uniform draw) and an eps-long vector of
//   uniform direction (src/Math/random.cpp:71-156), or X^+ U with equal
//   probability: R S T is not distributed like its inverse T^+ S^+ R^+, and
//   without the X^+ choice the proposal is not symmetric and the chain misses
//   detailed balance;
//   accept when exp(-dS) > r,  dS = -(beta/3) Re tr[(U' - U) A],
//   A the staple sum of the link (the action written at
//   src/Actions/puregauge.cpp:28, staples as puregauge.cpp:36-54).
//
// The sweep is a checkerboard: for each direction mu and site parity, every
// link U_mu(x) of that parity is updated in parallel (its staples involve no
// link of the same direction and parity), in place.  The random numbers of a
// (link, sweep, hit) come from Philox4x32-10 keyed by the seed with counter
// (link index, sweep, hit, call), so the chain does not depend on the launch
// shape; oracle/ymoracle.c runs the same chain on the CPU.
#include "field.cuh"
#include "kernels.h"

namespace ym {

namespace {

__device__ __forceinline__ uint4 philox_g(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ double unit(uint32_t w) { return (double(w) + 0.5) * 2.3283064365386963e-10; }

// one embedded SU(2) element from four uniforms, on rows/columns (p, q)
template <class R>
__device__ __forceinline__ void su2_in(const double x[4], double eps, int p, int q, M3<R>& m) {
    double v1 = x[1] - 0.5, v2 = x[2] - 0.5, v3 = x[3] - 0.5;
    const double norm = sqrt(v1 * v1 + v2 * v2 + v3 * v3);
    const double x0 = (x[0] - 0.5 < 0.0 ? -1.0 : 1.0) * sqrt(1.0 - eps * eps);
    v1 = v1 * eps / norm;
    v2 = v2 * eps / norm;
    v3 = v3 * eps / norm;
    mzero(m);
    m.e[0][0].re = m.e[1][1].re = m.e[2][2].re = R(1);
    m.e[p][p] = cx(R(x0), R(v3));
    m.e[q][q] = cx(R(x0), R(-v3));
    m.e[p][q] = cx(R(v2), R(v1));
    m.e[q][p] = cx(R(-v2), R(v1));
}

template <class F>
__device__ __forceinline__ M3<typename F::Real> staple_sum(const F& u, const Geo& g, int s, const int c[4], int mu) {
    using R = typename F::Real;
    M3<R> omega;
    mzero(omega);
    const int cmu = g.coord(c, mu);
    const int s_pm = g.hop_rt(s, cmu, mu, +1);
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const int cnu = g.coord(c, nu);
        const int s_pn = g.hop_rt(s, cnu, nu, +1);
        const int s_mn = g.hop_rt(s, cnu, nu, -1);
        const int s_pm_mn = g.hop_rt(s_mn, cmu, mu, +1);
        M3<R> t;
        mmul<false, true>(u.load(nu, s_pm), u.load(mu, s_pn), t);
        mmul_acc<false, true>(t, u.load(nu, s), omega);
        mmul<true, true>(u.load(nu, s_pm_mn), u.load(mu, s_mn), t);
        mmul_acc<false, false>(t, u.load(nu, s_mn), omega);
    }
    return omega;
}

template <class F>
__global__ void __launch_bounds__(128) metropolis_kernel(F u, Geo g, int mu, int parity, double beta, double eps,
                                                         int hits, uint64_t seed, uint32_t sweep,
                                                         unsigned long long* accepted) {
    using R = typename F::Real;
    const int s = int(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned acc = 0;
    if (s < g.V) {
        int c[4];
        g.coords(s, c);
        if (((c[0] + c[1] + c[2] + c[3]) & 1) == parity) {
            const M3<R> A = staple_sum(u, g, s, c, mu);
            M3<R> U = u.load(mu, s);
            const uint64_t l = uint64_t(s) * 4 + uint64_t(mu);
            const uint2 key = make_uint2(uint32_t(seed), uint32_t(seed >> 32) ^ 0x4D455452u);
            for (int h = 0; h < hits; h++) {
                double r[16];
#pragma unroll
                for (uint32_t call = 0; call < 4; call++) {
                    const uint4 o = philox_g(make_uint4(uint32_t(l), uint32_t(l >> 32) ^ (call << 24), sweep, uint32_t(h)), key);
                    r[4 * call + 0] = unit(o.x);
                    r[4 * call + 1] = unit(o.y);
                    r[4 * call + 2] = unit(o.z);
                    r[4 * call + 3] = unit(o.w);
                }
                M3<R> a, b, ab, X, Un;
                su2_in(r + 0, eps, 0, 1, a);
                su2_in(r + 4, eps, 0, 2, b);
                mmul<false, false>(a, b, ab);
                su2_in(r + 8, eps, 1, 2, a);
                mmul<false, false>(ab, a, X);
                if (r[13] < 0.5)
                    mmul<true, false>(X, U, Un);
                else
                    mmul<false, false>(X, U, Un);
                // dS = -(beta/3) Re tr[(U' - U) A]
                const R dtr = re_trace_mul(Un, A) - re_trace_mul(U, A);
                const double dS = -beta / 3.0 * double(dtr);
                if (exp(-dS) > r[12]) {
                    U = Un;
                    acc++;
                }
            }
            u.store(mu, s, U);
        }
    }
    // warp sum, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(accepted, (unsigned long long)acc);
}

template <class F>
cudaError_t launch_metro_typed(void* u, const Geo& g, int mu, int parity, double beta, double eps, int hits,
                               uint64_t seed, uint32_t sweep, unsigned long long* accepted, cudaStream_t st) {
    const int b = 128;
    metropolis_kernel<F><<<unsigned((g.V + b - 1) / b), b, 0, st>>>(F{u, g.V}, g, mu, parity, beta, eps, hits, seed,
                                                                     sweep, accepted);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_metropolis(int prec, void* u, const Geo& g, int mu, int parity, double beta, double eps, int hits,
                              uint64_t seed, uint32_t sweep, unsigned long long* accepted, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_metro_typed<FieldD18>(u, g, mu, parity, beta, eps, hits, seed, sweep, accepted, st);
        case kFP32_18: return launch_metro_typed<FieldF18>(u, g, mu, parity, beta, eps, hits, seed, sweep, accepted, st);
        case kFP32_12: return launch_metro_typed<FieldF12>(u, g, mu, parity, beta, eps, hits, seed, sweep, accepted, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ym
