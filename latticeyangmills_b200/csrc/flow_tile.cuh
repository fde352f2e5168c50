// Device code of the one-kernel RK3 stage with a tile's plaquette field in
// shared memory, shared by the single-configuration kernel (flow_tile.cu) and
// the batched-ensemble kernel (ensemble.cu).
//
// The force is the plaquette-field form of flow_split.cu,
//   D_mu(x) = sum_{nu != mu} s_{mu nu} [ H_p(x) - U_nu(y)^+ H_p(y) U_nu(y) ],  y = x - nu,
// (the generator of src/Actions/puregauge.cpp:36-79), but the six H_p of a site
// never reach HBM: a block computes them for a tile of sites into shared memory
// and finishes the tile's links from there.
//
// Tiling.  A tile is Lx x Ty x Tz sites of one time slice (whole x lines, a
// Ty x Tz patch of (y, z)); a thread advances 1, 2 or 4 of a site's links
// (lpt), so a block has 4 ns / lpt threads.  A work unit is one tile
// column (yb, zb) at one time t; a block owns a run of consecutive units, t
// fastest, and streams through them along t:
//   * the generators of the three planes (a, t) of slice t stay in shared
//     memory for slice t + 1, whose links (mu, x) need H_{mu t}(x - t); only
//     the first slice of a run (and a column's t = 0) recomputes them;
//   * the lower faces of the tile, sites x - y and x - z outside it, are
//     recomputed for the three planes through y (resp. z) each slice, unless
//     the tile spans the whole extent, when the periodic neighbour is inside;
//   * x - x is always inside (whole lines, periodic).
// A unit's work: the plane generators of the tile (and faces, and the
// previous slice's time planes where needed) into shared memory, a barrier,
// then each thread advances its links (rk_finish, shared with the other stage
// kernels), a barrier.  Links go from `in` to `out` (ping-pong), so
// blocks never wait on one another.
//
// Against the two-kernel stage this removes the plaquette field's HBM round
// trip (6 s_Z per site written and read) and its second launch; the cost is
// the recomputed faces, 3 (Ty [Tz < Lz] + Tz [Ty < Ly]) / (6 Ty Tz) of the
// plane work (25 % at 4 x 4).  The accumulation order of D is the two-kernel
// form's (nu ascending), with the same per-plane and conjugation code.
#pragma once
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
__device__ __forceinline__ int spatial_slot(int p) { return p == 3 ? 2 : p; }              // p in {0, 1, 3}
__device__ __forceinline__ int time_slot(int p) { return p == 2 ? 0 : p - 3; }              // p in {2, 4, 5}
__device__ __forceinline__ int yface_slot(int p) { return p == 0 ? 0 : p - 2; }             // p in {0, 3, 4}
__device__ __forceinline__ int zface_slot(int p) { return p == 1 ? 0 : (p == 3 ? 1 : 2); }  // p in {1, 3, 5}

// One work unit: tile column `col` of g at time t.  Every thread of the block
// takes part in the plane work and the barriers; threads [0, ns 4 / lpt) then
// advance lpt links each: thread i the links (i / ns) lpt ... + lpt - 1 of
// tile site i % ns (warp-uniform directions when ns is a multiple of 32).
// `prologue`: the time planes of slice t - 1 are not in shared memory yet
// (first unit of a run or of a column).  `cur` selects which T buffer is slice
// t's.
template <class F, int STAGE>
__device__ __forceinline__ void tile_unit(const F& in, const F& out, const ForceField<typename F::Real>& zf,
                                          const Geo& g, const TileShape& tp, typename F::Real eps,
                                          typename HVec<typename F::Real>::V* sm, int tid, int nthreads, int col,
                                          int t, bool prologue, int cur) {
    using R = typename F::Real;
    using HV = HVec<R>;
    using V = typename HV::V;
    constexpr int KU = HV::KU;
    const int ns = tp.ns, Lx = g.n[0], Lt = g.n[3];
    V* const S = sm;
    V* const Tc = sm + (cur ? 6 : 3) * KU * ns;
    V* const Tp = sm + (cur ? 3 : 6) * KU * ns;
    V* const FY = sm + 9 * KU * ns;
    V* const FZ = FY + 3 * KU * tp.nfy;
    const int zb = col / tp.nyt, yb = col - zb * tp.nyt;
    const int y0 = yb * tp.ty, z0 = zb * tp.tz;

    // Plane generators: [0, 3 ns) the time planes of slice t - 1 (prologue
    // only), [3 ns, 9 ns) the six planes of slice t, then the faces.  Each item
    // is decoded from its index alone; one copy of the plane code for all.
    const int nface = 3 * (tp.nfy + tp.nfz);
    for (int i = (prologue ? 0 : 3 * ns) + tid; i < 9 * ns + nface; i += nthreads) {
        int cs[4], p, n, idx;
        V* dst;
        if (i < 9 * ns) {
            const int k = i / ns;
            idx = i - k * ns;
            const int j = idx / Lx;
            cs[0] = idx - j * Lx;
            cs[1] = y0 + j % tp.ty;
            cs[2] = z0 + j / tp.ty;
            n = ns;
            if (k < 3) {
                p = k == 0 ? 2 : k + 3;
                cs[3] = t == 0 ? Lt - 1 : t - 1;
                dst = Tp + k * KU * ns;
            } else {
                p = k - 3;
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

    // The thread's links, each from the tile's plane generators.
    if (tid < ns * (4 / tp.lpt)) {
        const int grp = tid / ns;
        const int st = tid - grp * ns;  // the site within the tile
        const int x = st % Lx;
        const int jyz = st / Lx;
        const int jy = jyz % tp.ty, jz = jyz / tp.ty;
        const int c[4] = {x, y0 + jy, z0 + jz, t};
        const int s = x + g.stride[1] * c[1] + g.stride[2] * c[2] + g.stride[3] * t;
#pragma unroll 1
        for (int mu = grp * tp.lpt; mu < (grp + 1) * tp.lpt; mu++) {
            Herm8<R> d;
            d.d0 = d.d1 = R(0);
            d.z01 = d.z02 = d.z12 = cx(R(0), R(0));
#pragma unroll 1
            for (int nu = 0; nu < 4; nu++) {
                if (nu == mu) continue;
                const int p = mu < nu ? plane_index(mu, nu) : plane_index(nu, mu);
                const R sg = mu < nu ? R(1) : R(-1);
                V* const own = plane_b(p) == 3 ? Tc + time_slot(p) * KU * ns : S + spatial_slot(p) * KU * ns;
                const Herm8<R> upper = HV::get(own + st, ns);
                // H_p(x - nu): inside the tile, on a recomputed face, or slice t - 1
                const V* lb = own;
                int ln = ns, li;
                if (nu == 0) {
                    li = x == 0 ? st + Lx - 1 : st - 1;
                } else if (nu == 1) {
                    if (jy > 0 || tp.nfy == 0) {
                        li = jy > 0 ? st - Lx : st + Lx * (tp.ty - 1);
                    } else {
                        lb = FY + yface_slot(p) * KU * tp.nfy;
                        ln = tp.nfy;
                        li = x + Lx * jz;
                    }
                } else if (nu == 2) {
                    if (jz > 0 || tp.nfz == 0) {
                        li = jz > 0 ? st - Lx * tp.ty : st + Lx * tp.ty * (tp.tz - 1);
                    } else {
                        lb = FZ + zface_slot(p) * KU * tp.nfz;
                        ln = tp.nfz;
                        li = x + Lx * jy;
                    }
                } else {
                    lb = Tp + time_slot(p) * KU * ns;
                    li = st;
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
    }
    __syncthreads();
}

}  // namespace ym
