// Device storage of gauge fields and flow generators, and the lattice geometry.
//
// HBM layout (structure of arrays, one plane per link direction and matrix
// element so that a warp's 32 consecutive sites load 32 consecutive vectors):
//
//   links  U[mu][e][site]   e = complex element, row-major (9 stored, or 6 for the
//                           two-row "12-real" form whose third row is rebuilt);
//                           each entry a double2 (FP64) or float2 (FP32) (re, im)
//   force  Z[mu][k][site]   the Hermitian traceless generator as 8 reals
//                           (Herm8: Z00, Z11, Re/Im Z01, Re/Im Z02, Re/Im Z12)
//
// Site order is the reference's lexicographic order, x fastest
// (include/Math/lattice.h:87-89), so the .bin byte order maps one-to-one.
#pragma once
#include <cstdint>

#include "su3.cuh"

namespace ym {

template <class R>
struct Vec2;
template <>
struct Vec2<double> {
    using T = double2;
};
template <>
struct Vec2<float> {
    using T = float2;
};

// Periodic 4-D lattice in lexicographic order.  Coordinates are recovered by
// division once per thread; neighbours are index offsets with wrap-around,
// replacing the reference's whole-field shift() with its MPI self-exchange
// (include/Math/lattice.h:360-594).
struct Geo {
    int n[4];
    int64_t stride[4];  // 1, nx, nx*ny, nx*ny*nz
    int64_t V;

    __device__ __forceinline__ void coords(int64_t s, int c[4]) const {
        int64_t r = s;
        c[0] = int(r % n[0]);
        r /= n[0];
        c[1] = int(r % n[1]);
        r /= n[1];
        c[2] = int(r % n[2]);
        c[3] = int(r / n[2]);
    }
    // index of the site one step from (s, c) along d (dir = +1 or -1)
    __device__ __forceinline__ int64_t hop(int64_t s, const int c[4], int d, int dir) const {
        if (dir > 0) return c[d] == n[d] - 1 ? s - int64_t(n[d] - 1) * stride[d] : s + stride[d];
        return c[d] == 0 ? s + int64_t(n[d] - 1) * stride[d] : s - stride[d];
    }
    // c[d] after one step along d
    __device__ __forceinline__ int step_coord(int cd, int d, int dir) const {
        if (dir > 0) return cd == n[d] - 1 ? 0 : cd + 1;
        return cd == 0 ? n[d] - 1 : cd - 1;
    }
    // index after a step along d1 then a step along d2 (d1 != d2)
    __device__ __forceinline__ int64_t hop2(int64_t s, const int c[4], int d1, int dir1, int d2, int dir2) const {
        const int64_t s1 = hop(s, c, d1, dir1);
        return hop(s1, c, d2, dir2);  // c[d2] unchanged by the first step
    }
};

// Link field of NE stored complex elements per link (9: full, 6: two rows).
template <class R, int NE>
struct LinkField {
    using Real = R;
    using V2 = typename Vec2<R>::T;
    static constexpr int kElems = NE;
    V2* p;
    int64_t V;

    __device__ __forceinline__ M3<R> load(int mu, int64_t s) const {
        M3<R> a;
        const V2* b = p + int64_t(mu) * NE * V + s;
#pragma unroll
        for (int e = 0; e < NE; e++) {
            const V2 v = __ldg(b + int64_t(e) * V);
            a.e[e / 3][e % 3] = cx(R(v.x), R(v.y));
        }
        if (NE == 6) reconstruct_row2(a);
        return a;
    }
    __device__ __forceinline__ void store(int mu, int64_t s, const M3<R>& a) const {
        V2* b = p + int64_t(mu) * NE * V + s;
#pragma unroll
        for (int e = 0; e < NE; e++) {
            V2 v;
            v.x = a.e[e / 3][e % 3].re;
            v.y = a.e[e / 3][e % 3].im;
            b[int64_t(e) * V] = v;
        }
    }
};

using FieldD18 = LinkField<double, 9>;
using FieldF18 = LinkField<float, 9>;
using FieldF12 = LinkField<float, 6>;

template <class R>
struct ForceField {
    R* p;  // [4][8][V]
    int64_t V;
    __device__ __forceinline__ Herm8<R> load(int mu, int64_t s) const {
        const R* b = p + int64_t(mu) * 8 * V + s;
        Herm8<R> z;
        z.d0 = b[0];
        z.d1 = b[V];
        z.z01 = cx(b[2 * V], b[3 * V]);
        z.z02 = cx(b[4 * V], b[5 * V]);
        z.z12 = cx(b[6 * V], b[7 * V]);
        return z;
    }
    __device__ __forceinline__ void store(int mu, int64_t s, const Herm8<R>& z) const {
        R* b = p + int64_t(mu) * 8 * V + s;
        b[0] = z.d0;
        b[V] = z.d1;
        b[2 * V] = z.z01.re;
        b[3 * V] = z.z01.im;
        b[4 * V] = z.z02.re;
        b[5 * V] = z.z02.im;
        b[6 * V] = z.z12.re;
        b[7 * V] = z.z12.im;
    }
};

}  // namespace ym
