// K3-K5: layout conversion, seeded field generation and FP64 reunitarisation.
#include "expsu3.cuh"
#include "kernels.h"

namespace ym {

// ---------------------------------------------------------------------------
// K4: the reference's .bin layout (site-major, mu = 0..3, 18 doubles; see
// src/InputOutput/inputconf.cpp:114-155) <-> the device SoA layout.
// One thread per link; the AoS side is read/written 16 bytes at a time.
// ---------------------------------------------------------------------------
// A .bin double with its bytes reversed (the big-endian "Chroma" files that
// inputconf.cpp:135-143 reads with ReverseDouble).
__device__ __forceinline__ double reverse_bytes(double x) {
    const unsigned long long v = (unsigned long long)__double_as_longlong(x);
    const uint32_t lo = __byte_perm(uint32_t(v >> 32), 0u, 0x0123);
    const uint32_t hi = __byte_perm(uint32_t(v), 0u, 0x0123);
    return __longlong_as_double((long long)((uint64_t(hi) << 32) | lo));
}

// Sites [first, first + n) of a .bin-layout block (aos points at site `first`).
template <class F>
__global__ void pack_kernel(const double* __restrict__ aos, F u, Geo g, int first, int n, bool swap) {
    const int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= 4 * int64_t(n)) return;
    const int s = g.own_site(first + int(l >> 2));
    const int mu = int(l & 3);
    const double2* src = reinterpret_cast<const double2*>(aos + l * 18);
    M3<typename F::Real> a;
#pragma unroll
    for (int e = 0; e < 9; e++) {
        double2 v = src[e];
        if (swap) v = make_double2(reverse_bytes(v.x), reverse_bytes(v.y));
        a.e[e / 3][e % 3] = cx(typename F::Real(v.x), typename F::Real(v.y));
    }
    u.store(mu, s, a);
}

template <class F>
__global__ void unpack_kernel(F u, Geo g, double* __restrict__ aos, int first, int n, bool swap) {
    const int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (l >= 4 * int64_t(n)) return;
    const int s = g.own_site(first + int(l >> 2));
    const int mu = int(l & 3);
    const M3<typename F::Real> a = u.load(mu, s);
    double2* dst = reinterpret_cast<double2*>(aos + l * 18);
#pragma unroll
    for (int e = 0; e < 9; e++) {
        double2 v = make_double2(double(a.e[e / 3][e % 3].re), double(a.e[e / 3][e % 3].im));
        if (swap) v = make_double2(reverse_bytes(v.x), reverse_bytes(v.y));
        dst[e] = v;
    }
}

cudaError_t launch_pack_range(int prec, const double* aos, void* u, const Geo& g, int first, int n, bool swap,
                              cudaStream_t st) {
    if (first < 0 || n < 0 || int64_t(first) + n > g.V) return cudaErrorInvalidValue;  // (own sites <= V)
    if (n == 0) return cudaSuccess;
    const int b = 256;
    const unsigned nb = unsigned((4 * int64_t(n) + b - 1) / b);
    void* v = const_cast<void*>((const void*)u);
    switch (prec) {
        case kFP64: pack_kernel<<<nb, b, 0, st>>>(aos, FieldD18{v, g.V}, g, first, n, swap); break;
        case kFP32_18: pack_kernel<<<nb, b, 0, st>>>(aos, FieldF18{v, g.V}, g, first, n, swap); break;
        case kFP32_12: pack_kernel<<<nb, b, 0, st>>>(aos, FieldF12{v, g.V}, g, first, n, swap); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_unpack_range(int prec, const void* u, double* aos, const Geo& g, int first, int n, bool swap,
                                cudaStream_t st) {
    if (first < 0 || n < 0 || int64_t(first) + n > g.V) return cudaErrorInvalidValue;  // (own sites <= V)
    if (n == 0) return cudaSuccess;
    const int b = 256;
    const unsigned nb = unsigned((4 * int64_t(n) + b - 1) / b);
    void* v = const_cast<void*>(u);
    switch (prec) {
        case kFP64: unpack_kernel<<<nb, b, 0, st>>>(FieldD18{v, g.V}, g, aos, first, n, swap); break;
        case kFP32_18: unpack_kernel<<<nb, b, 0, st>>>(FieldF18{v, g.V}, g, aos, first, n, swap); break;
        case kFP32_12: unpack_kernel<<<nb, b, 0, st>>>(FieldF12{v, g.V}, g, aos, first, n, swap); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_pack(int prec, const double* aos, void* u, const Geo& g, cudaStream_t st) {
    return launch_pack_range(prec, aos, u, g, 0, g.V, false, st);
}

cudaError_t launch_unpack(int prec, const void* u, double* aos, const Geo& g, cudaStream_t st) {
    return launch_unpack_range(prec, u, aos, g, 0, g.V, false, st);
}

// ---------------------------------------------------------------------------
// K5: seeded fields.  Philox4x32-10 (Salmon et al., SC'11) keyed by the 64-bit
// seed, counter = (global link index in .bin order, config id, stream<<16 | block);
// two 53-bit uniforms per output, Box-Muller for normals.  The CPU generator of
// the test fixtures follows the same recipe; the two agree to the last few ulp
// (libm vs CUDA transcendental rounding).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32(uint4 c, uint2 k) {
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

__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    return (double(a >> 5) * 67108864.0 + double(b >> 6)) * (1.0 / 9007199254740992.0);
}

enum { kStreamH = 0, kStreamHaar = 1, kStreamPick = 2 };

__device__ __forceinline__ double2 gauss2(uint64_t seed, uint32_t config, uint64_t lidx, uint32_t stream,
                                          uint32_t block) {
    const uint4 o = philox4x32(make_uint4(uint32_t(lidx), uint32_t(lidx >> 32), config, (stream << 16) | block),
                               make_uint2(uint32_t(seed), uint32_t(seed >> 32)));
    const double u1 = 1.0 - u53(o.x, o.y);
    const double u2 = u53(o.z, o.w);
    const double r = sqrt(-2.0 * log(u1));
    double sp, cp;
    sincos(6.283185307179586 * u2, &sp, &cp);
    return make_double2(r * cp, r * sp);
}

// Links of the sites [g.site0, g.site1); the random numbers of a link are drawn
// by its configuration-wide index (l below), so a slab of a decomposed
// configuration holds the same links as the whole-lattice field.
template <class F>
__global__ void init_kernel(F u, Geo g, int kind, double a, uint64_t seed, uint32_t config) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= 4 * int64_t(g.site1 - g.site0)) return;
    const int s = g.site0 + int(k >> 2);
    const int mu = int(k & 3);
    const int64_t l = 4 * g.global0 + k;
    using R = typename F::Real;
    M3<double> m;
    if (kind == kCold) {
        mzero(m);
        m.e[0][0].re = m.e[1][1].re = m.e[2][2].re = 1.0;
    } else {
        double g[10];
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const double2 v = gauss2(seed, config, uint64_t(l), kStreamH, b);
            g[2 * b] = v.x;
            g[2 * b + 1] = v.y;
        }
        const double tr = (g[0] + g[1] + g[2]) / 3.0;
        Herm8<double> q;
        q.d0 = a * (g[0] - tr);
        q.d1 = a * (g[1] - tr);
        q.z01 = cx(a * g[3], a * g[4]);
        q.z02 = cx(a * g[5], a * g[6]);
        q.z12 = cx(a * g[7], a * g[8]);
        exp_iq(q, m);
    }
    M3<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.e[i][j] = cx(R(m.e[i][j].re), R(m.e[i][j].im));
    u.store(mu, s, r);
}

// Rows 0 and 1 orthonormalised (Gram-Schmidt, FP64), row 2 = conj(row0 x row1).
__device__ __forceinline__ void gram_schmidt(M3<double>& m) {
    double n0 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) n0 += m.e[0][k].re * m.e[0][k].re + m.e[0][k].im * m.e[0][k].im;
    n0 = rsqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        m.e[0][k].re *= n0;
        m.e[0][k].im *= n0;
    }
    double pr = 0.0, pi = 0.0;  // <row0, row1>
#pragma unroll
    for (int k = 0; k < 3; k++) {
        pr += m.e[0][k].re * m.e[1][k].re + m.e[0][k].im * m.e[1][k].im;
        pi += m.e[0][k].re * m.e[1][k].im - m.e[0][k].im * m.e[1][k].re;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        m.e[1][k].re -= pr * m.e[0][k].re - pi * m.e[0][k].im;
        m.e[1][k].im -= pr * m.e[0][k].im + pi * m.e[0][k].re;
    }
    double n1 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) n1 += m.e[1][k].re * m.e[1][k].re + m.e[1][k].im * m.e[1][k].im;
    n1 = rsqrt(n1);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        m.e[1][k].re *= n1;
        m.e[1][k].im *= n1;
    }
    reconstruct_row2(m);
}

template <class F>
__global__ void haar_kernel(F u, Geo g, double frac, uint64_t seed, uint32_t config) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= 4 * int64_t(g.site1 - g.site0)) return;
    const int64_t l = 4 * g.global0 + k;
    const uint4 o = philox4x32(make_uint4(uint32_t(l), uint32_t(uint64_t(l) >> 32), config, uint32_t(kStreamPick) << 16),
                               make_uint2(uint32_t(seed), uint32_t(seed >> 32)));
    if (!(u53(o.x, o.y) < frac)) return;
    M3<double> m;
#pragma unroll
    for (int b = 0; b < 9; b++) {
        const double2 v = gauss2(seed, config, uint64_t(l), kStreamHaar, b);
        m.e[b / 3][b % 3] = cx(v.x, v.y);
    }
    gram_schmidt(m);
    using R = typename F::Real;
    M3<R> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.e[i][j] = cx(R(m.e[i][j].re), R(m.e[i][j].im));
    u.store(int(k & 3), g.site0 + int(k >> 2), r);
}

cudaError_t launch_init_links(int prec, void* u, const Geo& g, int kind, double a, uint64_t seed, uint32_t config,
                              cudaStream_t st) {
    const int b = 128;
    const unsigned nb = unsigned((4 * int64_t(g.site1 - g.site0) + b - 1) / b);
    if (nb == 0) return cudaSuccess;
    switch (prec) {
        case kFP64: init_kernel<<<nb, b, 0, st>>>(FieldD18{const_cast<void*>((const void*)u), g.V}, g, kind, a, seed, config); break;
        case kFP32_18: init_kernel<<<nb, b, 0, st>>>(FieldF18{const_cast<void*>((const void*)u), g.V}, g, kind, a, seed, config); break;
        case kFP32_12: init_kernel<<<nb, b, 0, st>>>(FieldF12{const_cast<void*>((const void*)u), g.V}, g, kind, a, seed, config); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_haar_mix(int prec, void* u, const Geo& g, double frac, uint64_t seed, uint32_t config,
                            cudaStream_t st) {
    const int b = 128;
    const unsigned nb = unsigned((4 * int64_t(g.site1 - g.site0) + b - 1) / b);
    if (nb == 0) return cudaSuccess;
    switch (prec) {
        case kFP64: haar_kernel<<<nb, b, 0, st>>>(FieldD18{const_cast<void*>((const void*)u), g.V}, g, frac, seed, config); break;
        case kFP32_18: haar_kernel<<<nb, b, 0, st>>>(FieldF18{const_cast<void*>((const void*)u), g.V}, g, frac, seed, config); break;
        case kFP32_12: haar_kernel<<<nb, b, 0, st>>>(FieldF12{const_cast<void*>((const void*)u), g.V}, g, frac, seed, config); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K3: FP64 reunitarisation (mixed path only; the FP64 path never reunitarises,
// as the reference never does).
// ---------------------------------------------------------------------------
// One thread per link, four warps (directions) per 32-site group, so each
// load and store instruction of a warp moves 512 contiguous bytes of the
// warp-group layout; rows 0 and 1 are read (row 2 comes from the FP64
// Gram-Schmidt).  At 32^4 on B200 the FP32-12 launch takes 0.111 ms, against
// 0.138 with one thread per link in (site, mu) order and the row rebuilt on
// load; the results are bit-identical.
template <class F>
__global__ void __launch_bounds__(128) reunit_kernel(F u, int V, unsigned long long* deviation) {
    const int mu = int(threadIdx.x >> 5);
    const int s = int(blockIdx.x) * 32 + int(threadIdx.x & 31);
    double dev = 0.0;
    if (s < V) {
        const Rows2<typename F::Real> a = u.load_rows2(mu, s);
        M3<double> m;
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) m.e[i][j] = cx(double(a.e[i][j].re), double(a.e[i][j].im));
#pragma unroll
        for (int i = 0; i < 2; i++) {
            double n = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) n += m.e[i][k].re * m.e[i][k].re + m.e[i][k].im * m.e[i][k].im;
            dev = fmax(dev, fabs(n - 1.0));
        }
        gram_schmidt(m);
        using R = typename F::Real;
        M3<R> r;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) r.e[i][j] = cx(R(m.e[i][j].re), R(m.e[i][j].im));
        u.store(mu, s, r);
    }
    // Warp max, then block max, then one atomic per block, and only where the
    // block's max exceeds the value already recorded: a few hundred atomics on
    // one address per launch instead of one per warp (131,072 at 32^4), which
    // serialised in L2 and made the launch several times its memory time.
    // Non-negative doubles order like their bit patterns.
    __shared__ double warp_max[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dev = fmax(dev, __shfl_down_sync(0xffffffffu, dev, o));
    if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = dev;
    __syncthreads();
    if (threadIdx.x == 0 && deviation) {
        for (int w = 1; w < int(blockDim.x >> 5); w++) dev = fmax(dev, warp_max[w]);
        const unsigned long long bits = (unsigned long long)__double_as_longlong(dev);
        if (bits > *reinterpret_cast<volatile unsigned long long*>(deviation)) atomicMax(deviation, bits);
    }
}

cudaError_t launch_reunitarize(int prec, void* u, const Geo& g, unsigned long long* deviation, cudaStream_t st) {
    const int b = 128;
    const unsigned nb = unsigned((g.V + 31) / 32);
    switch (prec) {
        case kFP64: reunit_kernel<<<nb, b, 0, st>>>(FieldD18{const_cast<void*>((const void*)u), g.V}, g.V, deviation); break;
        case kFP32_18: reunit_kernel<<<nb, b, 0, st>>>(FieldF18{const_cast<void*>((const void*)u), g.V}, g.V, deviation); break;
        case kFP32_12: reunit_kernel<<<nb, b, 0, st>>>(FieldF12{const_cast<void*>((const void*)u), g.V}, g.V, deviation); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ym
