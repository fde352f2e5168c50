// Device storage of gauge fields and flow generators, and the lattice geometry.
//
// HBM layout: sites in groups of 32 (one warp's sites), structure of arrays
// inside a group.  For each (mu, group) the link components are consecutive
// 512-byte blocks, each holding one 16-byte vector for the 32 sites:
//
//   FP64 links   9 double2 blocks: element e of the 32 sites
//   FP32 links   float4 blocks of element pairs (0,1) (2,3) (4,5) for the
//                two-row 12-real form; the 18-real form adds (6,7) and a
//                256-byte float2 block for element 8
//   generator    the Hermitian traceless Z as 8 reals (Herm8: Z00, Z11, Re/Im Z01,
//                Z02, Z12): 4 double2 or 2 float4 blocks
//
// A warp's 32 consecutive sites read 512 contiguous bytes per load
// instruction, and the blocks of one link are at fixed offsets from one
// address, so a link costs one address computation whatever its number of
// vectors.  Groups run over [mu][group]; the volume is padded to a multiple of
// 32 sites (padding lanes are never read).  Offsets are 32-bit counts of
// 16-byte units (the context checks 4 x padded V x link bytes / 16 < 2^32).
//
// Elements are row-major, (re, im); the two-row form stores rows 0 and 1 and
// rebuilds row 2 = conj(row0 x row1) on load.  Site order is the reference's
// lexicographic order, x fastest (include/Math/lattice.h:87-89), so the .bin
// byte order maps one-to-one.  Site indices are 32-bit (V < 2^31).
#pragma once
#include <cstdint>

#include "su3.cuh"

namespace ym {

// Division of a site index (< 2^31) by a lattice extent d <= 4096 with one
// multiply: q = (x * m) >> (32 + l), m = floor(2^(32+l)/d) + 1, l = ceil(log2 d)
// (Granlund & Montgomery, PLDI 1994, Thm 4.2 with N = 32; x * m < 2^64 here).
struct FastDiv {
    uint64_t m;
    int l;
};

inline FastDiv make_fastdiv(int d) {
    int l = 0;
    while ((1 << l) < d) l++;
    FastDiv f;
    f.m = ((uint64_t(1) << (32 + l)) / uint64_t(d)) + 1;
    f.l = l;
    return f;
}

// Periodic 4-D lattice in lexicographic order.  Coordinates are recovered once
// per thread; neighbours are index offsets with wrap-around, replacing the
// reference's whole-field shift() with its MPI self-exchange
// (include/Math/lattice.h:360-594).
struct Geo {
    int n[4];
    int stride[4];  // 1, nx, nx*ny, nx*ny*nz
    int V;
    FastDiv div[3];  // by n[0], n[1], n[2]
    // Sites this context updates and measures, [site0, site1): the whole
    // lattice, or the interior time slices of a slab of a decomposed
    // configuration (whose first and last slices are halos).  global0 is the
    // configuration-wide site index of site0 (seeded fields use global link
    // indices), vglobal the configuration's volume (normalisations).
    int site0, site1;
    long long global0, vglobal;
    // Block order of the stage kernel (one 32-site group per block): 0 = plain;
    // otherwise the time coordinate advances every tile_groups blocks, so a
    // link read as a time neighbour is read again a few hundred blocks later,
    // still in L2 (tile_groups divides slice_groups, the groups per time slice).
    int slice_groups, tile_groups;
    // A block of a configuration decomposed in several directions
    // (ymflow_create_block): bit d of halo_mask set where the local lattice
    // carries one halo layer on each side in direction d; bext[] the block's
    // own extents (the local extents less the halos).  0 / unused otherwise.
    int halo_mask;
    int bext[4];

    // whether site coordinates c are the block's own (not a halo)
    __device__ __forceinline__ bool interior(const int c[4]) const {
        if (!halo_mask) return true;
#pragma unroll
        for (int d = 0; d < 4; d++)
            if (((halo_mask >> d) & 1) && (c[d] == 0 || c[d] == n[d] - 1)) return false;
        return true;
    }
    // local site of the block's k-th own site (own sites in lexicographic order, x fastest)
    __device__ __forceinline__ int own_site(int k) const {
        if (!halo_mask) return k;
        int s = 0;
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int q = k / bext[d];
            const int cd = k - q * bext[d] + ((halo_mask >> d) & 1);
            k = q;
            s += cd * stride[d];
        }
        return s;
    }

    __device__ __forceinline__ int block_group(int b) const {
        if (tile_groups == 0) return b;
        const int per_tile = tile_groups * n[3];
        const int ti = b / per_tile;
        const int r = b - ti * per_tile;
        const int t = r / tile_groups;
        return t * slice_groups + ti * tile_groups + (r - t * tile_groups);
    }

    __device__ __forceinline__ static int fdiv(int x, const FastDiv& f) {
        return int((uint64_t(uint32_t(x)) * f.m) >> (32 + f.l));
    }
    __device__ __forceinline__ void coords(int s, int c[4]) const {
        const int q0 = fdiv(s, div[0]);
        c[0] = s - q0 * n[0];
        const int q1 = fdiv(q0, div[1]);
        c[1] = q0 - q1 * n[1];
        const int q2 = fdiv(q1, div[2]);
        c[2] = q1 - q2 * n[2];
        c[3] = q2;
    }
    // index of the site one step from (s, c) along d (dir = +1 or -1)
    __device__ __forceinline__ int hop(int s, const int c[4], int d, int dir) const {
        if (dir > 0) return c[d] == n[d] - 1 ? s - (n[d] - 1) * stride[d] : s + stride[d];
        return c[d] == 0 ? s + (n[d] - 1) * stride[d] : s - stride[d];
    }
    // the same with a direction known only at run time (warp-uniform): the
    // coordinate, extent and stride are picked by selects (no dynamic register
    // or parameter indexing, which would go through local memory)
    __device__ __forceinline__ int coord(const int c[4], int d) const {
        return d == 0 ? c[0] : (d == 1 ? c[1] : (d == 2 ? c[2] : c[3]));
    }
    __device__ __forceinline__ int ext(int d) const {
        return d == 0 ? n[0] : (d == 1 ? n[1] : (d == 2 ? n[2] : n[3]));
    }
    __device__ __forceinline__ int str(int d) const {
        return d == 0 ? stride[0] : (d == 1 ? stride[1] : (d == 2 ? stride[2] : stride[3]));
    }
    __device__ __forceinline__ int hop_rt(int s, int cd, int d, int dir) const {
        const int nd = ext(d);
        const int sd = str(d);
        if (dir > 0) return cd == nd - 1 ? s - (nd - 1) * sd : s + sd;
        return cd == 0 ? s + (nd - 1) * sd : s - sd;
    }
};

inline Geo make_geo(const int dims[4]) {
    Geo g;
    for (int i = 0; i < 4; i++) g.n[i] = dims[i];
    g.stride[0] = 1;
    g.stride[1] = dims[0];
    g.stride[2] = dims[0] * dims[1];
    g.stride[3] = dims[0] * dims[1] * dims[2];
    g.V = dims[0] * dims[1] * dims[2] * dims[3];
    for (int i = 0; i < 3; i++) g.div[i] = make_fastdiv(dims[i]);
    g.site0 = 0;
    g.site1 = g.V;
    g.global0 = 0;
    g.vglobal = g.V;
    const int vs = dims[0] * dims[1] * dims[2];
    g.slice_groups = vs % 32 == 0 ? vs / 32 : 0;
    g.tile_groups = 0;
    g.halo_mask = 0;
    for (int i = 0; i < 4; i++) g.bext[i] = dims[i];
    return g;
}

// The tiled block order with tiles of about `target` groups (a divisor of the
// groups per time slice), where the slices hold more than `target` groups.
inline void set_tiled_order(Geo& g, int target) {
    g.tile_groups = 0;
    if (g.slice_groups <= target || g.site0 != 0 || g.site1 != g.V) return;
    for (int t = target; t >= target / 4; t--)
        if (g.slice_groups % t == 0) {
            g.tile_groups = t;
            return;
        }
}

inline int64_t padded_sites(int64_t V) { return (V + 31) & ~int64_t(31); }

// First 16-byte unit of the (mu, group of s) block run, plus the lane of s;
// `units` = 16-byte units per group (32 x bytes per link / 16).
__device__ __forceinline__ uint32_t group_lane_unit(int mu, int s, int V, int units) {
    const int groups = (V + 31) >> 5;
    return uint32_t(mu * groups + (s >> 5)) * uint32_t(units) + uint32_t(s & 31);
}

template <class R>
__device__ __forceinline__ void set_elem(M3<R>& a, int e, R re, R im) {
    a.e[e / 3][e % 3] = cx(re, im);
}

// Link field of NE stored complex elements per link (9: full, 6: two rows).
template <class R, int NE>
struct LinkField;

template <int NE>
struct LinkField<double, NE> {
    using Real = double;
    static constexpr int kElems = NE;
    static constexpr int kUnits = NE * 32;  // 16-byte units per group
    void* p;
    int V;

    // element 0 of link (mu, s); element e is 32 units further per e
    __device__ __forceinline__ const double2* link(int mu, int s) const {
        return reinterpret_cast<const double2*>(p) + group_lane_unit(mu, s, V, kUnits);
    }
    __device__ __forceinline__ Rows2<double> load_rows2(int mu, int s) const {
        const double2* b = link(mu, s);
        Rows2<double> a;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            const double2 v = __ldg(b + 32 * e);
            a.e[e / 3][e % 3] = cx(v.x, v.y);
        }
        return a;
    }
    __device__ __forceinline__ M3<double> load(int mu, int s) const {
        const double2* b = link(mu, s);
        M3<double> a;
#pragma unroll
        for (int e = 0; e < NE; e++) {
            const double2 v = __ldg(b + 32 * e);
            set_elem(a, e, v.x, v.y);
        }
        if (NE == 6) reconstruct_row2(a);
        return a;
    }
    __device__ __forceinline__ void put(int mu, int e, int s, Cx<double> v) const {
        double2* q = const_cast<double2*>(link(mu, s)) + 32 * e;
        *q = make_double2(v.re, v.im);
    }
    __device__ __forceinline__ void store(int mu, int s, const M3<double>& a) const {
        double2* q = const_cast<double2*>(link(mu, s));
#pragma unroll
        for (int e = 0; e < NE; e++) q[32 * e] = make_double2(a.e[e / 3][e % 3].re, a.e[e / 3][e % 3].im);
    }
    __device__ __forceinline__ void store_rows2(int mu, int s, const Rows2<double>& a) const {
        double2* q = const_cast<double2*>(link(mu, s));
#pragma unroll
        for (int e = 0; e < 6; e++) q[32 * e] = make_double2(a.e[e / 3][e % 3].re, a.e[e / 3][e % 3].im);
        if (NE == 9) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const Cx<double> r = row2_entry(a, k);
                q[32 * (6 + k)] = make_double2(r.re, r.im);
            }
        }
    }
};

template <int NE>
struct LinkField<float, NE> {
    using Real = float;
    static constexpr int kElems = NE;
    static constexpr int kPairs = NE / 2;                        // float4 blocks: 3 (12-real) or 4 (18-real)
    static constexpr int kUnits = kPairs * 32 + (NE == 9 ? 16 : 0);  // + the float2 block of element 8
    void* p;
    int V;

    // pair 0 of link (mu, s); pair k is 32 units further per k
    __device__ __forceinline__ const float4* link(int mu, int s) const {
        return reinterpret_cast<const float4*>(p) + group_lane_unit(mu, s, V, kUnits);
    }
    // element 8 of the 18-real form: the float2 block after the float4 blocks
    __device__ __forceinline__ const float2* tail(const float4* l, int s) const {
        return reinterpret_cast<const float2*>(l - (s & 31) + 32 * kPairs) + (s & 31);
    }
    __device__ __forceinline__ Rows2<float> load_rows2(int mu, int s) const {
        const float4* b = link(mu, s);
        Rows2<float> a;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float4 v = __ldg(b + 32 * k);
            a.e[(2 * k) / 3][(2 * k) % 3] = cx(v.x, v.y);
            a.e[(2 * k + 1) / 3][(2 * k + 1) % 3] = cx(v.z, v.w);
        }
        return a;
    }
    __device__ __forceinline__ M3<float> load(int mu, int s) const {
        const float4* b = link(mu, s);
        M3<float> a;
#pragma unroll
        for (int k = 0; k < kPairs; k++) {
            const float4 v = __ldg(b + 32 * k);
            set_elem(a, 2 * k, v.x, v.y);
            set_elem(a, 2 * k + 1, v.z, v.w);
        }
        if (NE == 9) {
            const float2 v = __ldg(tail(b, s));
            set_elem(a, 8, v.x, v.y);
        } else {
            reconstruct_row2(a);
        }
        return a;
    }
    __device__ __forceinline__ void store(int mu, int s, const M3<float>& a) const {
        float4* q = const_cast<float4*>(link(mu, s));
#pragma unroll
        for (int k = 0; k < kPairs; k++) {
            const Cx<float> x = a.e[(2 * k) / 3][(2 * k) % 3], y = a.e[(2 * k + 1) / 3][(2 * k + 1) % 3];
            q[32 * k] = make_float4(x.re, x.im, y.re, y.im);
        }
        if (NE == 9) *const_cast<float2*>(tail(q, s)) = make_float2(a.e[2][2].re, a.e[2][2].im);
    }
    __device__ __forceinline__ void store_rows2(int mu, int s, const Rows2<float>& a) const {
        float4* q = const_cast<float4*>(link(mu, s));
        q[0] = make_float4(a.e[0][0].re, a.e[0][0].im, a.e[0][1].re, a.e[0][1].im);
        q[32] = make_float4(a.e[0][2].re, a.e[0][2].im, a.e[1][0].re, a.e[1][0].im);
        q[64] = make_float4(a.e[1][1].re, a.e[1][1].im, a.e[1][2].re, a.e[1][2].im);
        if (NE == 9) {
            const Cx<float> r0 = row2_entry(a, 0), r1 = row2_entry(a, 1), r2 = row2_entry(a, 2);
            q[96] = make_float4(r0.re, r0.im, r1.re, r1.im);
            *const_cast<float2*>(tail(q, s)) = make_float2(r2.re, r2.im);
        }
    }
};

using FieldD18 = LinkField<double, 9>;
using FieldF18 = LinkField<float, 9>;
using FieldF12 = LinkField<float, 6>;

template <class R>
struct ForceField;

template <>
struct ForceField<double> {
    void* p;  // 4 double2 blocks per (mu, group)
    int V;
    __device__ __forceinline__ double2* link(int mu, int s) const {
        return reinterpret_cast<double2*>(p) + group_lane_unit(mu, s, V, 4 * 32);
    }
    __device__ __forceinline__ Herm8<double> load(int mu, int s) const {
        const double2* q = link(mu, s);
        const double2 a = q[0], b = q[32], c = q[64], d = q[96];
        return unpack(a, b, c, d);
    }
    // the same through the read-only data path (fields no thread of the kernel writes)
    __device__ __forceinline__ Herm8<double> load_ro(int mu, int s) const {
        const double2* q = link(mu, s);
        return unpack(__ldg(q), __ldg(q + 32), __ldg(q + 64), __ldg(q + 96));
    }
    __device__ __forceinline__ static Herm8<double> unpack(double2 a, double2 b, double2 c, double2 d) {
        Herm8<double> z;
        z.d0 = a.x;
        z.d1 = a.y;
        z.z01 = cx(b.x, b.y);
        z.z02 = cx(c.x, c.y);
        z.z12 = cx(d.x, d.y);
        return z;
    }
    __device__ __forceinline__ void store(int mu, int s, const Herm8<double>& z) const {
        double2* q = link(mu, s);
        q[0] = make_double2(z.d0, z.d1);
        q[32] = make_double2(z.z01.re, z.z01.im);
        q[64] = make_double2(z.z02.re, z.z02.im);
        q[96] = make_double2(z.z12.re, z.z12.im);
    }
};

template <>
struct ForceField<float> {
    void* p;  // 2 float4 blocks per (mu, group)
    int V;
    __device__ __forceinline__ float4* link(int mu, int s) const {
        return reinterpret_cast<float4*>(p) + group_lane_unit(mu, s, V, 2 * 32);
    }
    __device__ __forceinline__ Herm8<float> load(int mu, int s) const {
        const float4* q = link(mu, s);
        const float4 a = q[0], b = q[32];
        return unpack(a, b);
    }
    // the same through the read-only data path (fields no thread of the kernel writes)
    __device__ __forceinline__ Herm8<float> load_ro(int mu, int s) const {
        const float4* q = link(mu, s);
        return unpack(__ldg(q), __ldg(q + 32));
    }
    __device__ __forceinline__ static Herm8<float> unpack(float4 a, float4 b) {
        Herm8<float> z;
        z.d0 = a.x;
        z.d1 = a.y;
        z.z01 = cx(a.z, a.w);
        z.z02 = cx(b.x, b.y);
        z.z12 = cx(b.z, b.w);
        return z;
    }
    __device__ __forceinline__ void store(int mu, int s, const Herm8<float>& z) const {
        float4* q = link(mu, s);
        q[0] = make_float4(z.d0, z.d1, z.z01.re, z.z01.im);
        q[32] = make_float4(z.z02.re, z.z02.im, z.z12.re, z.z12.im);
    }
};

}  // namespace ym
