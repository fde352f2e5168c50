// K1t: one RK3 stage of one configuration in a single kernel, the plaquette
// field of a tile of sites held in shared memory.
//
// The force is the plaquette-field form of flow_split.cu,
//   D_mu(x) = sum_{nu != mu} s_{mu nu} [ H_p(x) - U_nu(y)^+ H_p(y) U_nu(y) ],  y = x - nu,
// (the generator of src/Actions/puregauge.cpp:36-79), but the six H_p of a site
// never reach HBM: a block computes them for a tile of sites into shared memory
// and finishes the tile's links from there.
//
// Tiling.  A tile is Lx x Ty x Tz sites of one time slice (whole x lines, a
// Ty x Tz patch of (y, z)): one thread per site.  A block owns a run of
// consecutive work units, a unit being one tile column (yb, zb) at one time t,
// t fastest, and streams through them along t:
//   * the generators of the three planes (a, t) of slice t stay in shared
//     memory for slice t + 1, whose links (mu, x) need H_{mu t}(x - t); only
//     the first slice of a run (and a column's t = 0) recomputes them;
//   * the lower faces of the tile, sites x - y and x - z outside it, are
//     recomputed for the three planes through y (resp. z) each slice, unless
//     the tile spans the whole extent, when the periodic neighbour is inside;
//   * x - x is always inside (whole lines, periodic).
// A unit's work: the plane generators of the tile (and faces, and the
// previous slice's time planes where needed) into shared memory, a barrier,
// then each thread advances its site's four links (rk_finish, shared with the
// other stage kernels), a barrier.  Links go from `in` to `out` (ping-pong), so
// blocks never wait on one another.
//
// Against the two-kernel stage this removes the plaquette field's HBM round
// trip (6 s_Z per site written and read) and its second launch; the cost is
// the recomputed faces, 3 (Ty [Tz < Lz] + Tz [Ty < Ly]) / (6 Ty Tz) of the
// plane work (25 % at 4 x 4).  The accumulation order of D is the two-kernel
// form's (nu ascending), with the same per-plane and conjugation code.
#include <algorithm>

#include "flow_device.cuh"
#include "kernels.h"

namespace ym {

// A plane generator as 16-byte vectors in shared memory: float4 x 2 (FP32) or
// double2 x 4 (FP64).  Layout [slot][vector][entry]: consecutive threads touch
// consecutive 16-byte words (no bank conflicts).
template <class R>
struct HVec;
template <>
struct HVec<float> {
    using V = float4;
    static constexpr int KU = 2;
    __device__ __forceinline__ static void put(V* q, int n, const Herm8<float>& h) {
        q[0] = make_float4(h.d0, h.d1, h.z01.re, h.z01.im);
        q[n] = make_float4(h.z02.re, h.z02.im, h.z12.re, h.z12.im);
    }
    __device__ __forceinline__ static Herm8<float> get(const V* q, int n) {
        const float4 a = q[0], b = q[n];
        Herm8<float> h;
        h.d0 = a.x;
        h.d1 = a.y;
        h.z01 = cx(a.z, a.w);
        h.z02 = cx(b.x, b.y);
        h.z12 = cx(b.z, b.w);
        return h;
    }
};
template <>
struct HVec<double> {
    using V = double2;
    static constexpr int KU = 4;
    __device__ __forceinline__ static void put(V* q, int n, const Herm8<double>& h) {
        q[0] = make_double2(h.d0, h.d1);
        q[n] = make_double2(h.z01.re, h.z01.im);
        q[2 * n] = make_double2(h.z02.re, h.z02.im);
        q[3 * n] = make_double2(h.z12.re, h.z12.im);
    }
    __device__ __forceinline__ static Herm8<double> get(const V* q, int n) {
        const double2 a = q[0], b = q[n], c = q[2 * n], d = q[3 * n];
        Herm8<double> h;
        h.d0 = a.x;
        h.d1 = a.y;
        h.z01 = cx(b.x, b.y);
        h.z02 = cx(c.x, c.y);
        h.z12 = cx(d.x, d.y);
        return h;
    }
};

// Buffers of the block's shared memory, in entries (ns = sites of a tile):
//   S      the spatial planes (0,1) (0,2) (1,2) of slice t      3 x ns
//   T[2]   the time planes (0,3) (1,3) (2,3), slices t and t-1   2 x 3 x ns
//   FY     planes (0,1) (1,2) (1,3) of the face y0 - 1          3 x Lx Tz
//   FZ     planes (0,2) (1,2) (2,3) of the face z0 - 1          3 x Lx Ty
__device__ __forceinline__ int spatial_slot(int p) { return p == 3 ? 2 : p; }                // p in {0, 1, 3}
__device__ __forceinline__ int time_slot(int p) { return p == 2 ? 0 : p - 3; }                // p in {2, 4, 5}
__device__ __forceinline__ int yface_slot(int p) { return p == 0 ? 0 : p - 2; }               // p in {0, 3, 4}
__device__ __forceinline__ int zface_slot(int p) { return p == 1 ? 0 : (p == 3 ? 1 : 2); }    // p in {1, 3, 5}

template <class F, int STAGE>
__global__ void __launch_bounds__(512, 1)
    rk_tile_stage_kernel(F in, F out, ForceField<typename F::Real> zf, Geo g, TileShape tp, typename F::Real eps) {
    using R = typename F::Real;
    using HV = HVec<R>;
    using V = typename HV::V;
    constexpr int KU = HV::KU;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    V* const sm = reinterpret_cast<V*>(tile_smem);
    const int ns = tp.ns, Lx = g.n[0], Lt = g.n[3];
    V* const S = sm;
    V* const T0 = sm + 3 * KU * ns;
    V* const T1 = sm + 6 * KU * ns;
    V* const FY = sm + 9 * KU * ns;
    V* const FZ = FY + 3 * KU * tp.nfy;

    const int tid = int(threadIdx.x);
    const int x = tid % Lx;
    const int jyz = tid / Lx;
    const int jy = jyz % tp.ty, jz = jyz / tp.ty;
    const int u0 = int((long long)blockIdx.x * tp.units / gridDim.x);
    const int u1 = int((long long)(blockIdx.x + 1) * tp.units / gridDim.x);
    const int nface = 3 * (tp.nfy + tp.nfz);
    int cur = 0;

    for (int u = u0; u < u1; u++) {
        const int col = u / Lt, t = u - col * Lt;
        const int zb = col / tp.nyt, yb = col - zb * tp.nyt;
        const int y0 = yb * tp.ty, z0 = zb * tp.tz;
        const int c[4] = {x, y0 + jy, z0 + jz, t};
        const int s = x + g.stride[1] * c[1] + g.stride[2] * c[2] + g.stride[3] * t;
        V* const Tc = cur ? T1 : T0;
        V* const Tp = cur ? T0 : T1;

        // Plane generators: [0, 3 ns) the time planes of slice t - 1 (first
        // unit of a run or of a column only), [3 ns, 9 ns) the six planes of
        // slice t, then the faces.  One copy of the plane code for all.
        const bool prologue = u == u0 || t == 0;
        for (int i = (prologue ? 0 : 3 * ns) + tid; i < 9 * ns + nface; i += ns) {
            int cs[4], p, n, idx;
            V* dst;
            if (i < 9 * ns) {
                cs[0] = c[0];
                cs[1] = c[1];
                cs[2] = c[2];
                idx = tid;
                n = ns;
                if (i < 3 * ns) {
                    const int k = i / ns;
                    p = k == 0 ? 2 : k + 3;
                    cs[3] = t == 0 ? Lt - 1 : t - 1;
                    dst = Tp + k * KU * ns;
                } else {
                    p = i / ns - 3;
                    cs[3] = t;
                    dst = plane_b(p) == 3 ? Tc + time_slot(p) * KU * ns : S + spatial_slot(p) * KU * ns;
                }
            } else if (i < 9 * ns + 3 * tp.nfy) {
                const int r = i - 9 * ns;
                const int k = r / tp.nfy;
                idx = r - k * tp.nfy;
                p = k == 0 ? 0 : k + 2;
                cs[0] = idx % Lx;
                cs[1] = y0 == 0 ? g.n[1] - 1 : y0 - 1;
                cs[2] = z0 + idx / Lx;
                cs[3] = t;
                n = tp.nfy;
                dst = FY + k * KU * n;
            } else {
                const int r = i - 9 * ns - 3 * tp.nfy;
                const int k = r / tp.nfz;
                idx = r - k * tp.nfz;
                p = 2 * k + 1;
                cs[0] = idx % Lx;
                cs[1] = y0 + idx / Lx;
                cs[2] = z0 == 0 ? g.n[2] - 1 : z0 - 1;
                cs[3] = t;
                n = tp.nfz;
                dst = FZ + k * KU * n;
            }
            const int ss = cs[0] + g.stride[1] * cs[1] + g.stride[2] * cs[2] + g.stride[3] * cs[3];
            HV::put(dst + idx, n, plane_generator(in, g, ss, cs, plane_a(p), plane_b(p)));
        }
        __syncthreads();

        // The four links of the site, each from the tile's plane generators.
#pragma unroll 1
        for (int mu = 0; mu < 4; mu++) {
            Herm8<R> d;
            d.d0 = d.d1 = R(0);
            d.z01 = d.z02 = d.z12 = cx(R(0), R(0));
#pragma unroll 1
            for (int nu = 0; nu < 4; nu++) {
                if (nu == mu) continue;
                const int p = mu < nu ? plane_index(mu, nu) : plane_index(nu, mu);
                const R sg = mu < nu ? R(1) : R(-1);
                V* const own = plane_b(p) == 3 ? Tc + time_slot(p) * KU * ns : S + spatial_slot(p) * KU * ns;
                const Herm8<R> upper = HV::get(own + tid, ns);
                // H_p(x - nu): inside the tile, on a recomputed face, or slice t - 1
                const V* lb = own;
                int ln = ns, li;
                if (nu == 0) {
                    li = x == 0 ? tid + Lx - 1 : tid - 1;
                } else if (nu == 1) {
                    if (jy > 0 || tp.nfy == 0) {
                        li = jy > 0 ? tid - Lx : tid + Lx * (tp.ty - 1);
                    } else {
                        lb = FY + yface_slot(p) * KU * tp.nfy;
                        ln = tp.nfy;
                        li = x + Lx * jz;
                    }
                } else if (nu == 2) {
                    if (jz > 0 || tp.nfz == 0) {
                        li = jz > 0 ? tid - Lx * tp.ty : tid + Lx * tp.ty * (tp.tz - 1);
                    } else {
                        lb = FZ + zface_slot(p) * KU * tp.nfz;
                        ln = tp.nfz;
                        li = x + Lx * jy;
                    }
                } else {
                    lb = Tp + time_slot(p) * KU * ns;
                    li = tid;
                }
                const int y = g.hop_rt(s, g.coord(c, nu), nu, -1);
                const M3<R> v = in.load(nu, y);
                const Herm8<R> lower = herm_conj_by(v, HV::get(lb + li, ln));
                d.d0 = fma(sg, upper.d0 - lower.d0, d.d0);
                d.d1 = fma(sg, upper.d1 - lower.d1, d.d1);
                d.z01 = cx(fma(sg, upper.z01.re - lower.z01.re, d.z01.re), fma(sg, upper.z01.im - lower.z01.im, d.z01.im));
                d.z02 = cx(fma(sg, upper.z02.re - lower.z02.re, d.z02.re), fma(sg, upper.z02.im - lower.z02.im, d.z02.im));
                d.z12 = cx(fma(sg, upper.z12.re - lower.z12.re, d.z12.re), fma(sg, upper.z12.im - lower.z12.im, d.z12.im));
            }
            const M3<R> uu = in.load(mu, s);
            rk_finish<F, STAGE>(out, zf, eps, s, mu, d, uu);
        }
        __syncthreads();
        cur ^= 1;
    }
}

template <class F>
static void* tile_kernel_ptr(int stage) {
    switch (stage) {
        case 0: return (void*)rk_tile_stage_kernel<F, 0>;
        case 1: return (void*)rk_tile_stage_kernel<F, 1>;
        default: return (void*)rk_tile_stage_kernel<F, 2>;
    }
}

static void* tile_kernel(int prec, int stage) {
    switch (prec) {
        case kFP64: return tile_kernel_ptr<FieldD18>(stage);
        case kFP32_18: return tile_kernel_ptr<FieldF18>(stage);
        default: return tile_kernel_ptr<FieldF12>(stage);
    }
}

size_t tile_smem_bytes(int prec, const TileShape& tp) {
    const size_t entry = prec == kFP64 ? 64 : 32;
    return entry * size_t(9 * tp.ns + 3 * (tp.nfy + tp.nfz));
}

bool make_tile_shape(int prec, const Geo& g, int ty, int tz, TileShape* out) {
    const int Lx = g.n[0], Ly = g.n[1], Lz = g.n[2];
    if (ty < 1 || tz < 1 || ty > Ly || tz > Lz || Ly % ty || Lz % tz) return false;
    if (g.site0 != 0 || g.site1 != g.V) return false;  // whole-lattice contexts
    const long long ns = (long long)Lx * ty * tz;
    // whole warps of consecutive sites: every warp inside one (x, y) run
    if (ns > 512 || ns < 64 || (Lx * ty) % 32) return false;
    TileShape tp;
    tp.ty = ty;
    tp.tz = tz;
    tp.ns = int(ns);
    tp.nyt = Ly / ty;
    tp.nzt = Lz / tz;
    tp.nfy = ty < Ly ? Lx * tz : 0;
    tp.nfz = tz < Lz ? Lx * ty : 0;
    tp.units = tp.nyt * tp.nzt * g.n[3];
    tp.grid = 0;
    if (tile_smem_bytes(prec, tp) > size_t(227 * 1024)) return false;
    *out = tp;
    return true;
}

cudaError_t prepare_tile_kernels(int prec) {
    for (int s = 0; s < 3; s++) {
        cudaError_t e = cudaFuncSetAttribute(tile_kernel(prec, s), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             227 * 1024);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t tile_grid(int prec, int device, TileShape* tp) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_kernel(prec, 1), tp->ns,
                                                      tile_smem_bytes(prec, *tp));
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    tp->grid = std::min(tp->units, sms * per_sm);
    return cudaSuccess;
}

template <class F>
static cudaError_t launch_tile_typed(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g,
                                     const TileShape& tp, double eps, cudaStream_t st) {
    using R = typename F::Real;
    F in{const_cast<void*>(uin), g.V}, out{uout, g.V};
    ForceField<R> zf{z, g.V};
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    const size_t sm = tile_smem_bytes(prec, tp);
    switch (stage) {
        case 0: rk_tile_stage_kernel<F, 0><<<tp.grid, tp.ns, sm, st>>>(in, out, zf, g, tp, e); break;
        case 1: rk_tile_stage_kernel<F, 1><<<tp.grid, tp.ns, sm, st>>>(in, out, zf, g, tp, e); break;
        default: rk_tile_stage_kernel<F, 2><<<tp.grid, tp.ns, sm, st>>>(in, out, zf, g, tp, e); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_rk_tile_stage(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g,
                                 const TileShape& tp, double eps, cudaStream_t st) {
    if (tp.grid < 1 || tp.ns < 1 || tp.ns > 512) return cudaErrorInvalidValue;
    switch (prec) {
        case kFP64: return launch_tile_typed<FieldD18>(prec, stage, uin, uout, z, g, tp, eps, st);
        case kFP32_18: return launch_tile_typed<FieldF18>(prec, stage, uin, uout, z, g, tp, eps, st);
        case kFP32_12: return launch_tile_typed<FieldF12>(prec, stage, uin, uout, z, g, tp, eps, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ym
