// K6: batched ensemble.  Many configurations of uneven lattice sizes advance
// through each RK3 stage together: in one launch per kernel over a work list
// of every (configuration, block of sites) pair, each item looking its
// configuration up in a prefix table (the per-link kernel over a persistent
// grid-stride loop or one block per item, the two-kernel stage, the tile
// kernel), or in two launches per run of equal-extent configurations, the
// runs as concurrent branches (stage form 3).  The launches of a step are
// replayed as a captured CUDA graph; the project's autotuner picks the form.
// The reference flows its configurations one after another
// (src/Apps/wilsonflow.cpp:96-109); small lattices cannot fill a B200 that way.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "api_util.h"
#include "flow_tile.cuh"
#include "ymflow.h"

namespace ym {

struct EnsConf {
    Geo g;
    int64_t uoff;  // start of this configuration in the link pool (bytes, 16-aligned)
    int64_t zoff;  // start in the generator pool (bytes, 16-aligned)
    int64_t hoff;  // start in the plane-generator pool of the two-kernel stage (bytes, 16-aligned)
    int blk0;      // first work item
    int nblk;      // work items (blocks of sites)
    TileShape tp;  // the tile kernel's tiling of this configuration
    int unit0;     // its first tile unit in the ensemble's unit list
};

__device__ __forceinline__ int find_conf(const EnsConf* confs, int nconf, int item) {
    int lo = 0, hi = nconf - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&confs[mid].blk0) <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class F>
struct EnsMinBlocks {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 4 : 5;  // the persistent loop spills at 80 registers
};

template <class F, int STAGE>
__global__ void __launch_bounds__(128, EnsMinBlocks<F>::value) ens_stage_kernel(char* uin, char* uout, char* z,
                                                         const EnsConf* __restrict__ confs, int nconf, int nitems,
                                                         typename F::Real eps) {
    using R = typename F::Real;
    const int spb = blockDim.x >> 2;  // sites per block: four warps (directions) per 32 sites
    const int w = threadIdx.x >> 5;
    const int mu = w & 3;
    const int lane_site = ((w >> 2) << 5) + (threadIdx.x & 31);
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const EnsConf& C = confs[find_conf(confs, nconf, item)];
        const Geo& g = C.g;
        const int s = (item - C.blk0) * spb + lane_site;
        if (s < g.V) {
            const F in{uin + C.uoff, g.V}, out{uout + C.uoff, g.V};
            const ForceField<R> zf{z + C.zoff, g.V};
            rk_link_update<F, STAGE>(in, out, zf, g, eps, s, mu);
        }
    }
}

// One block per work item (the grid the autotuner picks when every item gets
// its own block): no item loop, so the kernel keeps the single-configuration
// kernel's register budget (80 in the FP32 18-real form; the looping kernel
// spills there).
template <class F>
struct EnsFlatMinBlocks {
    static constexpr int value = sizeof(typename F::Real) == 8 ? 4 : (F::kElems == 9 ? 6 : 5);
};

template <class F, int STAGE>
__global__ void __launch_bounds__(128, EnsFlatMinBlocks<F>::value)
    ens_flat_kernel(char* uin, char* uout, char* z, const EnsConf* __restrict__ confs, int nconf,
                    typename F::Real eps) {
    using R = typename F::Real;
    const int w = threadIdx.x >> 5;
    const int mu = w & 3;
    const int item = blockIdx.x;
    const EnsConf& C = confs[find_conf(confs, nconf, item)];
    const Geo& g = C.g;  // read where used (L1), not held in registers
    const int s = (item - C.blk0) * (blockDim.x >> 2) + ((w >> 2) << 5) + (threadIdx.x & 31);
    if (s >= g.V) return;
    const F in{uin + C.uoff, g.V}, out{uout + C.uoff, g.V};
    const ForceField<R> zf{z + C.zoff, g.V};
    rk_link_update<F, STAGE>(in, out, zf, g, eps, s, mu);
}

template <class F>
static cudaError_t launch_ens_typed(int stage, void* uin, void* uout, void* z, const EnsConf* confs, int nconf,
                                    int nitems, int grid, int block, double eps, cudaStream_t st) {
    using R = typename F::Real;
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    char *a = (char*)uin, *b = (char*)uout, *zz = (char*)z;
    if (grid >= nitems) {
        switch (stage) {
            case 0: ens_flat_kernel<F, 0><<<nitems, block, 0, st>>>(a, b, zz, confs, nconf, e); break;
            case 1: ens_flat_kernel<F, 1><<<nitems, block, 0, st>>>(a, b, zz, confs, nconf, e); break;
            default: ens_flat_kernel<F, 2><<<nitems, block, 0, st>>>(a, b, zz, confs, nconf, e); break;
        }
        return cudaGetLastError();
    }
    switch (stage) {
        case 0: ens_stage_kernel<F, 0><<<grid, block, 0, st>>>(a, b, zz, confs, nconf, nitems, e); break;
        case 1: ens_stage_kernel<F, 1><<<grid, block, 0, st>>>(a, b, zz, confs, nconf, nitems, e); break;
        default: ens_stage_kernel<F, 2><<<grid, block, 0, st>>>(a, b, zz, confs, nconf, nitems, e); break;
    }
    return cudaGetLastError();
}

// The two-kernel stage over the work list (FP32 ensembles): one 192-thread block
// per 32-site item forms that item's six plane generators, then one 128-thread
// block per item runs the stage from them.  One block per item, as the flat kernel.
template <class F>
__global__ void __launch_bounds__(192) ens_plaq_kernel(char* u, char* h, const EnsConf* __restrict__ confs, int nconf) {
    const int item = blockIdx.x;
    const EnsConf& C = confs[find_conf(confs, nconf, item)];
    const Geo& g = C.g;
    const int s = (item - C.blk0) * 32 + int(threadIdx.x & 31);
    if (s >= g.V) return;
    const F uf{u + C.uoff, g.V};
    const ForceField<typename F::Real> hf{h + C.hoff, g.V};
    plaq_plane(uf, hf, g, s, int(threadIdx.x >> 5));
}

template <class F, int STAGE>
__global__ void __launch_bounds__(128, SplitMinBlocks<F>::value)
    ens_split_kernel(char* uin, char* uout, char* z, char* h, const EnsConf* __restrict__ confs, int nconf,
                     typename F::Real eps) {
    using R = typename F::Real;
    const int mu = int(threadIdx.x >> 5) & 3;
    const int item = blockIdx.x;
    const EnsConf& C = confs[find_conf(confs, nconf, item)];
    const Geo& g = C.g;
    const int s = (item - C.blk0) * 32 + int(threadIdx.x & 31);
    if (s >= g.V) return;
    const F in{uin + C.uoff, g.V}, out{uout + C.uoff, g.V};
    const ForceField<R> zf{z + C.zoff, g.V}, hf{h + C.hoff, g.V};
    split_link_update<F, STAGE>(in, out, zf, hf, g, eps, s, mu);
}

// The same two kernels with the work list as a launch parameter (up to
// kParamConfs configurations): the binary search and every geometry read of
// the link code come from the constant bank instead of global memory, as a
// single configuration's Geo does.  The plaquette-field kernel takes two
// planes per thread (64 sites per block), as the single-configuration one.
constexpr int kParamConfs = 128;
struct EnsTable {
    EnsConf c[kParamConfs];
    int n;
};

__device__ __forceinline__ int find_conf_param(const EnsTable& t, int item) {
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.c[mid].blk0 <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class F>
__global__ void __launch_bounds__(192, PlaqMinBlocks<F>::value) ens_plaq_param_kernel(char* u, char* h, const __grid_constant__ EnsTable tab) {
    const int w = int(threadIdx.x >> 5);
    const int item = int(blockIdx.x) * 2 + w / 3;
    if (item >= tab.c[tab.n - 1].blk0 + tab.c[tab.n - 1].nblk) return;
    const EnsConf& C = tab.c[find_conf_param(tab, item)];
    const Geo& g = C.g;
    const int s = (item - C.blk0) * 32 + int(threadIdx.x & 31);
    if (s >= g.V) return;
    const F uf{u + C.uoff, g.V};
    const ForceField<typename F::Real> hf{h + C.hoff, g.V};
    const int pr = w % 3;
    const int p0 = pr == 0 ? 0 : (pr == 1 ? 2 : 3);
    const int p1 = pr == 0 ? 1 : (pr == 1 ? 4 : 5);
    int c[4];
    g.coords(s, c);
    // both planes before either store: the link the two share is loaded once
    const auto h0 = plane_generator(uf, g, s, c, plane_a(p0), plane_b(p0));
    const auto h1 = plane_generator(uf, g, s, c, plane_a(p1), plane_b(p1));
    hf.store(p0, s, h0);
    hf.store(p1, s, h1);
}

template <class F, int STAGE>
__global__ void __launch_bounds__(128, SplitMinBlocks<F>::value)
    ens_split_param_kernel(char* uin, char* uout, char* z, char* h, const __grid_constant__ EnsTable tab,
                           typename F::Real eps) {
    using R = typename F::Real;
    const int mu = int(threadIdx.x >> 5) & 3;
    const int item = blockIdx.x;
    const EnsConf& C = tab.c[find_conf_param(tab, item)];
    const Geo& g = C.g;
    const int s = (item - C.blk0) * 32 + int(threadIdx.x & 31);
    if (s >= g.V) return;
    const F in{uin + C.uoff, g.V}, out{uout + C.uoff, g.V};
    const ForceField<R> zf{z + C.zoff, g.V}, hf{h + C.hoff, g.V};
    split_link_update<F, STAGE>(in, out, zf, hf, g, eps, s, mu);
}

template <class F>
static cudaError_t launch_ens_split_typed(int stage, void* uin, void* uout, void* z, void* h, const EnsConf* confs,
                                          int nconf, int nitems, double eps, cudaStream_t st,
                                          const EnsConf* host_confs) {
    using R = typename F::Real;
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    char *a = (char*)uin, *b = (char*)uout, *zz = (char*)z, *hh = (char*)h;
    if (host_confs && nconf <= kParamConfs) {
        EnsTable tab;
        std::memcpy(tab.c, host_confs, sizeof(EnsConf) * size_t(nconf));
        tab.n = nconf;
        ens_plaq_param_kernel<F><<<(nitems + 1) / 2, 192, 0, st>>>(a, hh, tab);
        switch (stage) {
            case 0: ens_split_param_kernel<F, 0><<<nitems, 128, 0, st>>>(a, b, zz, hh, tab, e); break;
            case 1: ens_split_param_kernel<F, 1><<<nitems, 128, 0, st>>>(a, b, zz, hh, tab, e); break;
            default: ens_split_param_kernel<F, 2><<<nitems, 128, 0, st>>>(a, b, zz, hh, tab, e); break;
        }
        return cudaGetLastError();
    }
    ens_plaq_kernel<F><<<nitems, 192, 0, st>>>(a, hh, confs, nconf);
    switch (stage) {
        case 0: ens_split_kernel<F, 0><<<nitems, 128, 0, st>>>(a, b, zz, hh, confs, nconf, e); break;
        case 1: ens_split_kernel<F, 1><<<nitems, 128, 0, st>>>(a, b, zz, hh, confs, nconf, e); break;
        default: ens_split_kernel<F, 2><<<nitems, 128, 0, st>>>(a, b, zz, hh, confs, nconf, e); break;
    }
    return cudaGetLastError();
}

// The same two kernels per run of consecutive configurations of one geometry
// (EnsRun): the run's work items are its (configuration, 32-site group) pairs,
// configuration-major, and the geometry is a launch parameter read at fixed
// constant-bank offsets, exactly as the single-configuration kernels read
// their Geo; a block finds its configuration by one division.  A stage is
// one plaquette-field launch and one stage launch per run.
struct EnsRun {
    Geo g;
    int nconf;                          // configurations in the run
    int nblk;                           // 32-site groups per configuration
    int64_t ustride, zstride, hstride;  // bytes from one configuration to the next in each pool
};

template <class F>
__global__ void __launch_bounds__(192, PlaqMinBlocks<F>::value) ens_run_plaq_kernel(char* u, char* h, const __grid_constant__ EnsRun r) {
    const int w = int(threadIdx.x >> 5);
    if constexpr (sizeof(typename F::Real) == 8) {  // FP64: one plane per thread, warp w plane w of one item
        const int item = int(blockIdx.x);
        const int conf = item / r.nblk;
        if (conf >= r.nconf) return;
        const Geo& g = r.g;
        const int s = (item - conf * r.nblk) * 32 + int(threadIdx.x & 31);
        if (s >= g.V) return;
        const F uf{u + conf * r.ustride, g.V};
        const ForceField<typename F::Real> hf{h + conf * r.hstride, g.V};
        int c[4];
        g.coords(s, c);
        hf.store(w, s, plane_generator(uf, g, s, c, plane_a(w), plane_b(w)));
        return;
    }
    // FP32: from the run's end, as plaq_field_kernel (its stage kernel starts
    // on the L2-resident items)
    const int blk = int(gridDim.x - 1 - blockIdx.x);
    const int item = blk * 2 + w / 3;
    const int conf = item / r.nblk;
    if (conf >= r.nconf) return;
    const Geo& g = r.g;
    const int s = (item - conf * r.nblk) * 32 + int(threadIdx.x & 31);
    if (s >= g.V) return;
    const F uf{u + conf * r.ustride, g.V};
    const ForceField<typename F::Real> hf{h + conf * r.hstride, g.V};
    const int pr = w % 3;
    const int p0 = pr == 0 ? 0 : (pr == 1 ? 2 : 3);
    const int p1 = pr == 0 ? 1 : (pr == 1 ? 4 : 5);
    int c[4];
    g.coords(s, c);
    // both planes before either store: the link the two share is loaded once
    const auto h0 = plane_generator(uf, g, s, c, plane_a(p0), plane_b(p0));
    const auto h1 = plane_generator(uf, g, s, c, plane_a(p1), plane_b(p1));
    hf.store(p0, s, h0);
    hf.store(p1, s, h1);
}

template <class F, int STAGE>
__global__ void __launch_bounds__(128, SplitMinBlocks<F>::value)
    ens_run_split_kernel(char* uin, char* uout, char* z, char* h, const __grid_constant__ EnsRun r,
                         typename F::Real eps) {
    using R = typename F::Real;
    const int mu = int(threadIdx.x >> 5) & 3;
    const int item = int(blockIdx.x);
    const int conf = item / r.nblk;
    const Geo& g = r.g;
    const int s = (item - conf * r.nblk) * 32 + int(threadIdx.x & 31);
    if (s >= g.V) return;
    const F in{uin + conf * r.ustride, g.V}, out{uout + conf * r.ustride, g.V};
    const ForceField<R> zf{z + conf * r.zstride, g.V}, hf{h + conf * r.hstride, g.V};
    split_link_update<F, STAGE>(in, out, zf, hf, g, eps, s, mu);
}

// A run and where its first configuration starts in each pool.
struct EnsRunLaunch {
    EnsRun r;
    int64_t uoff, zoff, hoff;
};

// One stage of one run: its plaquette-field launch, then its stage launch.
template <class F>
static cudaError_t launch_ens_run_typed(int stage, void* uin, void* uout, void* z, void* h, const EnsRunLaunch& L,
                                        double eps, cudaStream_t st) {
    using R = typename F::Real;
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    const int items = L.r.nconf * L.r.nblk;
    char *a = (char*)uin + L.uoff, *b = (char*)uout + L.uoff, *zz = (char*)z + L.zoff, *hh = (char*)h + L.hoff;
    ens_run_plaq_kernel<F><<<sizeof(R) == 8 ? items : (items + 1) / 2, 192, 0, st>>>(a, hh, L.r);
    switch (stage) {
        case 0: ens_run_split_kernel<F, 0><<<items, 128, 0, st>>>(a, b, zz, hh, L.r, e); break;
        case 1: ens_run_split_kernel<F, 1><<<items, 128, 0, st>>>(a, b, zz, hh, L.r, e); break;
        default: ens_run_split_kernel<F, 2><<<items, 128, 0, st>>>(a, b, zz, hh, L.r, e); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_ens_run_stage(int prec, int stage, void* uin, void* uout, void* z, void* h, const EnsRunLaunch& L,
                                 double eps, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_ens_run_typed<FieldD18>(stage, uin, uout, z, h, L, eps, st);
        case kFP32_18: return launch_ens_run_typed<FieldF18>(stage, uin, uout, z, h, L, eps, st);
        case kFP32_12: return launch_ens_run_typed<FieldF12>(stage, uin, uout, z, h, L, eps, st);
        default: return cudaErrorInvalidValue;
    }
}

// The one-kernel stage with a tile's plaquette field in shared memory
// (flow_tile.cuh) over every configuration at once: the unit lists of all
// configurations, concatenated, are split into contiguous runs, one per
// persistent block; a block streams through its run along t, crossing from
// one tile column or configuration to the next.  Every configuration's tile
// has at most blockDim.x sites (threads beyond a tile's sites only help with
// its plane generators).
__device__ __forceinline__ int find_unit_conf(const EnsConf* confs, int nconf, int unit) {
    int lo = 0, hi = nconf - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&confs[mid].unit0) <= unit) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <class F, int STAGE>
__global__ void __launch_bounds__(512, 1)
    ens_tile_kernel(char* uin, char* uout, char* z, const EnsConf* __restrict__ confs, int nconf, int nunits,
                    typename F::Real eps) {
    using R = typename F::Real;
    using V = typename HVec<R>::V;
    extern __shared__ __align__(16) unsigned char ens_tile_smem[];
    V* const sm = reinterpret_cast<V*>(ens_tile_smem);
    const int u0 = int((long long)blockIdx.x * nunits / gridDim.x);
    const int u1 = int((long long)(blockIdx.x + 1) * nunits / gridDim.x);
    int cur = 0;
    for (int u = u0; u < u1; u++) {
        const EnsConf& C = confs[find_unit_conf(confs, nconf, u)];
        const int Lt = C.g.n[3];
        const int local = u - C.unit0;
        const int col = local / Lt, t = local - col * Lt;
        const F in{uin + C.uoff, C.g.V}, out{uout + C.uoff, C.g.V};
        const ForceField<R> zf{z + C.zoff, C.g.V};
        tile_unit<F, STAGE>(in, out, zf, C.g, C.tp, eps, sm, int(threadIdx.x), int(blockDim.x), col, t,
                            u == u0 || t == 0, cur);
        cur ^= 1;
    }
}

template <class F>
static void* ens_tile_ptr(int stage) {
    switch (stage) {
        case 0: return (void*)ens_tile_kernel<F, 0>;
        case 1: return (void*)ens_tile_kernel<F, 1>;
        default: return (void*)ens_tile_kernel<F, 2>;
    }
}

static void* ens_tile_fn(int prec, int stage) {
    switch (prec) {
        case kFP64: return ens_tile_ptr<FieldD18>(stage);
        case kFP32_18: return ens_tile_ptr<FieldF18>(stage);
        default: return ens_tile_ptr<FieldF12>(stage);
    }
}

cudaError_t prepare_ens_tile(int prec) {
    for (int s = 0; s < 3; s++) {
        const cudaError_t e =
            cudaFuncSetAttribute(ens_tile_fn(prec, s), cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int ens_tile_resident(int prec, int threads, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_tile_fn(prec, 1), threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

template <class F>
static cudaError_t launch_ens_tile_typed(int stage, void* uin, void* uout, void* z, const EnsConf* confs, int nconf,
                                         int nunits, int grid, int threads, size_t smem, double eps, cudaStream_t st) {
    using R = typename F::Real;
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    char *a = (char*)uin, *b = (char*)uout, *zz = (char*)z;
    switch (stage) {
        case 0: ens_tile_kernel<F, 0><<<grid, threads, smem, st>>>(a, b, zz, confs, nconf, nunits, e); break;
        case 1: ens_tile_kernel<F, 1><<<grid, threads, smem, st>>>(a, b, zz, confs, nconf, nunits, e); break;
        default: ens_tile_kernel<F, 2><<<grid, threads, smem, st>>>(a, b, zz, confs, nconf, nunits, e); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_ens_tile_stage(int prec, int stage, void* uin, void* uout, void* z, const EnsConf* confs,
                                  int nconf, int nunits, int grid, int threads, size_t smem, double eps,
                                  cudaStream_t st) {
    if (grid < 1 || threads < 32 || threads > 512) return cudaErrorInvalidValue;
    switch (prec) {
        case kFP64:
            return launch_ens_tile_typed<FieldD18>(stage, uin, uout, z, confs, nconf, nunits, grid, threads, smem,
                                                   eps, st);
        case kFP32_18:
            return launch_ens_tile_typed<FieldF18>(stage, uin, uout, z, confs, nconf, nunits, grid, threads, smem,
                                                   eps, st);
        case kFP32_12:
            return launch_ens_tile_typed<FieldF12>(stage, uin, uout, z, confs, nconf, nunits, grid, threads, smem,
                                                   eps, st);
        default: return cudaErrorInvalidValue;
    }
}

// Work items must be 32-site groups (block 128).
cudaError_t launch_ens_split_stage(int prec, int stage, void* uin, void* uout, void* z, void* h, const EnsConf* confs,
                                   int nconf, int nitems, double eps, cudaStream_t st,
                                   const EnsConf* host_confs = nullptr) {
    switch (prec) {
        case kFP64: return launch_ens_split_typed<FieldD18>(stage, uin, uout, z, h, confs, nconf, nitems, eps, st, host_confs);
        case kFP32_18: return launch_ens_split_typed<FieldF18>(stage, uin, uout, z, h, confs, nconf, nitems, eps, st, host_confs);
        case kFP32_12: return launch_ens_split_typed<FieldF12>(stage, uin, uout, z, h, confs, nconf, nitems, eps, st, host_confs);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_ens_stage(int prec, int stage, void* uin, void* uout, void* z, const EnsConf* confs, int nconf,
                             int nitems, int grid, int block, double eps, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_ens_typed<FieldD18>(stage, uin, uout, z, confs, nconf, nitems, grid, block, eps, st);
        case kFP32_18: return launch_ens_typed<FieldF18>(stage, uin, uout, z, confs, nconf, nitems, grid, block, eps, st);
        case kFP32_12: return launch_ens_typed<FieldF12>(stage, uin, uout, z, confs, nconf, nitems, grid, block, eps, st);
        default: return cudaErrorInvalidValue;
    }
}

int ens_max_resident(int prec, int block) {
    int n = 0;
    cudaError_t e = cudaSuccess;
    switch (prec) {
        case kFP64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_stage_kernel<FieldD18, 1>, block, 0); break;
        case kFP32_18: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_stage_kernel<FieldF18, 1>, block, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_stage_kernel<FieldF12, 1>, block, 0); break;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return std::max(n, 1);
}

// Tuning results shared by every ensemble with the same signature in this process.
struct EnsTuning {
    int form, block, grid;
};
std::mutex g_tune_mu;
std::map<std::string, EnsTuning> g_tune_cache;

}  // namespace ym

using namespace ym;

struct ymflow_ens {
    int nconf = 0;
    int prec = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<EnsConf> confs;  // host copy
    EnsConf* confs_dev = nullptr;
    void* u[2] = {nullptr, nullptr};
    int cur = 0;
    void* z = nullptr;
    void* h = nullptr;       // plane generators of the two-kernel stage (FP32 ensembles)
    bool split = false;      // FP32: the two-kernel stage, one block per work item
    bool by_runs = false;    // ... launched per run of equal-geometry configurations
    std::vector<EnsRunLaunch> runs;
    // the runs' launch streams (run i on side[i % side.size()]): each run's
    // stages depend only on its own earlier stages, so the runs flow
    // concurrently, as parallel branches of the step graph
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> side_done;
    cudaEvent_t fork = nullptr;
    bool tile = false;       // the one-kernel stage with tiles in shared memory (over split / fused)
    int tile_threads = 0;    // its block size: every configuration's tile has at most this many sites
    int tile_grid = 0;       // its persistent blocks
    size_t tile_smem = 0;    // its shared memory per block (the largest configuration's)
    int nunits = 0;          // tile units of all configurations
    int64_t pool_links = 0;  // bytes per link pool
    int64_t pool_force = 0;  // bytes of the generator pool
    double* staging = nullptr;  // .bin-layout buffer sized for the largest configuration
    int64_t max_v = 0;
    double* partials = nullptr;
    int partial_cap = 0;
    double* meas = nullptr;
    int meas_cap = 0;
    double* meas_host = nullptr;
    unsigned long long* deviation = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_eps[2] = {0.0, 0.0};
    int graph_cfg[2][2] = {{0, 0}, {0, 0}};
    int block = 128;
    int grid = 0;  // persistent CTAs (0: one per work item)
    bool use_graph = true;
    bool tuned = false;
    std::vector<char> loaded;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t step = 0;
    double t = 0.0;
    std::string err;
    std::string signature;
};

namespace {

thread_local std::string g_ens_create_error;

int efail(ymflow_ens* e, int code, const std::string& m) {
    if (e) e->err = m;
    return code;
}
int ecuda(ymflow_ens* e, cudaError_t c, const char* what) { return efail(e, status_of(c), cuda_message(c, what)); }

#define YE_CK(ens, call, what)                                     \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return ecuda(ens, e_, what);        \
    } while (0)

// Rebuild the work-list prefix table for a block size and upload it.
int set_block(ymflow_ens* e, int block) {
    const int spb = block / 4;
    int blk = 0;
    for (EnsConf& c : e->confs) {
        c.blk0 = blk;
        c.nblk = (c.g.V + spb - 1) / spb;
        blk += c.nblk;
    }
    YE_CK(e, cudaMemcpyAsync(e->confs_dev, e->confs.data(), sizeof(EnsConf) * e->confs.size(),
                             cudaMemcpyHostToDevice, e->stream),
          "work list upload");
    YE_CK(e, cudaStreamSynchronize(e->stream), "work list upload");
    e->block = block;
    return YMFLOW_OK;
}

// Tiles for every configuration with at most `threads` sites each: per
// configuration the tile with the least estimated time per site (threads
// idle beyond the tile's sites, recomputed faces), then the unit list and
// the persistent grid.  false if a configuration has no such tile or the
// largest shared memory does not fit.
bool set_tiles(ymflow_ens* e, int threads) {
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    std::vector<TileShape> tps(e->nconf);
    size_t smem = 0;
    for (int c = 0; c < e->nconf; c++) {
        const Geo& g = e->confs[c].g;
        bool found = false;
        double best = 0.0;
        for (int ty = 1; ty <= g.n[1]; ty++)
            for (int tz = 1; tz <= g.n[2]; tz++) {
                TileShape tp;
                if (!make_tile_shape(e->prec, g, ty, tz, &tp, false) || tp.ns > threads) continue;
                const double cost = double(threads) / tp.ns * (12.0 + 3.0 * (tp.nfy + tp.nfz) / tp.ns);
                if (!found || cost < best) {
                    tps[c] = tp;
                    best = cost;
                    found = true;
                }
            }
        if (!found) return false;
        smem = std::max(smem, tile_smem_bytes(e->prec, tps[c]));
    }
    const int resident = ens_tile_resident(e->prec, threads, smem);
    if (resident < 1) return false;
    int unit = 0;
    for (int c = 0; c < e->nconf; c++) {
        e->confs[c].tp = tps[c];
        e->confs[c].unit0 = unit;
        unit += tps[c].units;
    }
    if (cudaMemcpyAsync(e->confs_dev, e->confs.data(), sizeof(EnsConf) * e->confs.size(), cudaMemcpyHostToDevice,
                        e->stream) != cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    e->nunits = unit;
    e->tile_threads = threads;
    e->tile_smem = smem;
    e->tile_grid = std::min(unit, resident * sms);
    return true;
}

int nitems(const ymflow_ens* e) {
    return e->confs.empty() ? 0 : e->confs.back().blk0 + e->confs.back().nblk;
}

// Puts the ensemble into a tuning's form; a tiling that no longer fits falls
// back to one 128-thread block per work item.
int apply_tuning(ymflow_ens* e, const EnsTuning& tn) {
    e->by_runs = tn.form == 3;
    if (tn.form == 0) e->split = false;
    if (tn.form == 1 || tn.form == 3) e->split = true;
    if (tn.form == 2 && set_tiles(e, tn.block)) {
        e->tile = true;
        return YMFLOW_OK;
    }
    e->tile = false;
    e->grid = tn.form == 2 ? 0 : tn.grid;
    return set_block(e, tn.form == 2 ? 128 : tn.block);
}

// Stages [0, nst) of every run, in[s] -> out[s]: forked from the ensemble's
// stream onto the side streams and joined back (parallel branches when
// captured into the step graph).  With one side stream, everything stays on
// the ensemble's stream.
cudaError_t enqueue_runs(ymflow_ens* e, int nst, void* const* in, void* const* out, double eps) {
    const int ns = int(e->side.size());
    if (ns == 0) {
        for (int s = 0; s < nst; s++)
            for (const EnsRunLaunch& L : e->runs) {
                const cudaError_t r = launch_ens_run_stage(e->prec, s, in[s], out[s], e->z, e->h, L, eps, e->stream);
                if (r != cudaSuccess) return r;
            }
        return cudaSuccess;
    }
    cudaError_t r = cudaEventRecord(e->fork, e->stream);
    for (int k = 0; k < ns && r == cudaSuccess; k++) r = cudaStreamWaitEvent(e->side[k], e->fork, 0);
    for (int s = 0; s < nst && r == cudaSuccess; s++)
        for (size_t i = 0; i < e->runs.size() && r == cudaSuccess; i++)
            r = launch_ens_run_stage(e->prec, s, in[s], out[s], e->z, e->h, e->runs[i], eps, e->side[i % ns]);
    for (int k = 0; k < ns; k++) {  // join every branch, also after a failed launch
        const cudaError_t j = cudaEventRecord(e->side_done[k], e->side[k]);
        const cudaError_t w = j == cudaSuccess ? cudaStreamWaitEvent(e->stream, e->side_done[k], 0) : j;
        if (r == cudaSuccess) r = w;
    }
    return r;
}

cudaError_t enqueue_ens_step(ymflow_ens* e, int from, double eps) {
    void* a = e->u[from];
    void* b = e->u[1 - from];
    void* in[3] = {a, b, a};
    void* out[3] = {b, a, b};
    const int ni = nitems(e);
    const int grid = e->grid > 0 ? std::min(e->grid, ni) : ni;
    if (!e->tile && e->split && e->by_runs) return enqueue_runs(e, 3, in, out, eps);
    for (int s = 0; s < 3; s++) {
        cudaError_t r = e->tile ? launch_ens_tile_stage(e->prec, s, in[s], out[s], e->z, e->confs_dev, e->nconf,
                                                        e->nunits, e->tile_grid, e->tile_threads, e->tile_smem, eps,
                                                        e->stream)
                        : e->split ? launch_ens_split_stage(e->prec, s, in[s], out[s], e->z, e->h, e->confs_dev,
                                                            e->nconf, ni, eps, e->stream, e->confs.data())
                                   : launch_ens_stage(e->prec, s, in[s], out[s], e->z, e->confs_dev, e->nconf, ni,
                                                      grid, e->block, eps, e->stream);
        if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
}

void drop_graphs(ymflow_ens* e) {
    for (int i = 0; i < 2; i++) {
        if (e->graph[i]) cudaGraphExecDestroy(e->graph[i]);
        e->graph[i] = nullptr;
    }
}

int run_ens_step(ymflow_ens* e, double eps) {
    const int from = e->cur;
    if (e->use_graph) {
        if (!e->graph[from] || e->graph_eps[from] != eps || e->graph_cfg[from][0] != e->block ||
            e->graph_cfg[from][1] != e->grid) {
            if (e->graph[from]) cudaGraphExecDestroy(e->graph[from]);
            e->graph[from] = nullptr;
            cudaGraph_t g = nullptr;
            YE_CK(e, cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            cudaError_t le = enqueue_ens_step(e, from, eps);
            cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
            if (le != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return ecuda(e, le, "stage launch during capture");
            }
            YE_CK(e, ce, "end capture");
            cudaError_t ie = cudaGraphInstantiate(&e->graph[from], g, 0);
            cudaGraphDestroy(g);
            YE_CK(e, ie, "instantiate step graph");
            e->graph_eps[from] = eps;
            e->graph_cfg[from][0] = e->block;
            e->graph_cfg[from][1] = e->grid;
        }
        YE_CK(e, cudaGraphLaunch(e->graph[from], e->stream), "launch step graph");
    } else {
        YE_CK(e, enqueue_ens_step(e, from, eps), "stage launch");
    }
    e->cur = 1 - from;
    return YMFLOW_OK;
}

int ens_alloc(ymflow_ens* e, void** p, size_t bytes, const char* what) {
    cudaError_t c = cudaMalloc(p, bytes);
    if (c != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return ecuda(e, c, what);
    }
    return YMFLOW_OK;
}

int ensure_ens_meas(ymflow_ens* e, int rows) {
    const int need = rows * e->nconf;
    if (need <= e->meas_cap) return YMFLOW_OK;
    if (e->meas) cudaFree(e->meas);
    if (e->meas_host) cudaFreeHost(e->meas_host);
    e->meas = nullptr;
    e->meas_host = nullptr;
    e->meas_cap = 0;
    int r = ens_alloc(e, (void**)&e->meas, size_t(need) * 4 * sizeof(double), "measurement rows");
    if (r != YMFLOW_OK) return r;
    YE_CK(e, cudaMallocHost((void**)&e->meas_host, size_t(need) * 4 * sizeof(double)), "pinned rows");
    e->meas_cap = need;
    return YMFLOW_OK;
}

// Observables of every configuration into rows [row*nconf, row*nconf + nconf).
int enqueue_ens_measure(ymflow_ens* e, int row) {
    for (int c = 0; c < e->nconf; c++) {
        const EnsConf& C = e->confs[c];
        const void* u = (const char*)e->u[e->cur] + C.uoff;
        YE_CK(e, launch_observables(e->prec, u, C.g, e->partials, e->stream), "observables launch");
        YE_CK(e, launch_obs_finalize(e->partials, obs_blocks(C.g), C.g,
                                     e->meas + 4 * (size_t(row) * e->nconf + c), e->stream),
              "observables fold");
    }
    return YMFLOW_OK;
}

void* conf_links(const ymflow_ens* e, int c) { return (char*)e->u[e->cur] + e->confs[c].uoff; }

float time_stage0(ymflow_ens* e, double eps, int reps) {
    // stage 0 reads u[cur] and writes only u[1-cur] and z, which the next step
    // overwrites anyway, so tuning does not disturb the flow state
    const int ni = nitems(e);
    const int grid = e->grid > 0 ? std::min(e->grid, ni) : ni;
    void* a = e->u[e->cur];
    void* b = e->u[1 - e->cur];
    auto launch = [&]() {
        if (e->tile)
            return launch_ens_tile_stage(e->prec, 0, a, b, e->z, e->confs_dev, e->nconf, e->nunits, e->tile_grid,
                                         e->tile_threads, e->tile_smem, eps, e->stream);
        if (e->split && e->by_runs) return enqueue_runs(e, 1, &a, &b, eps);
        if (e->split)
            return launch_ens_split_stage(e->prec, 0, a, b, e->z, e->h, e->confs_dev, e->nconf, ni, eps, e->stream,
                                          e->confs.data());
        return launch_ens_stage(e->prec, 0, a, b, e->z, e->confs_dev, e->nconf, ni, grid, e->block, eps, e->stream);
    };
    if (launch() != cudaSuccess) return -1.f;
    cudaEventRecord(e->ev0, e->stream);
    for (int i = 0; i < reps; i++)
        if (launch() != cudaSuccess) return -1.f;
    cudaEventRecord(e->ev1, e->stream);
    if (cudaEventSynchronize(e->ev1) != cudaSuccess) return -1.f;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    return ms / float(reps);
}

}  // namespace

extern "C" {

ymflow_ens* ymflow_ensemble_create(int nconf, const int* dims, int precision, int device, int* status) {
    auto set = [&](int s, const std::string& m) {
        if (status) *status = s;
        g_ens_create_error = m;
    };
    if (nconf < 1 || !dims) {
        set(YMFLOW_ERR_ARG, "need at least one configuration and its dims");
        return nullptr;
    }
    if (precision < YMFLOW_FP64 || precision > YMFLOW_FP32_12) {
        set(YMFLOW_ERR_ARG, "unknown precision");
        return nullptr;
    }
    std::string why;
    if (!device_usable(device, &why)) {
        set(YMFLOW_ERR_NODEVICE, why);
        return nullptr;
    }
    ymflow_ens* e = new (std::nothrow) ymflow_ens();
    if (!e) {
        set(YMFLOW_ERR_OOM, "host allocation failed");
        return nullptr;
    }
    DeviceGuard guard(device);
    e->nconf = nconf;
    e->prec = precision;
    e->device = device;
    e->confs.resize(nconf);
    e->loaded.assign(nconf, 0);
    int64_t uo = 0, zo = 0, ho = 0;
    for (int c = 0; c < nconf; c++) {
        const int* d = dims + 4 * c;
        int64_t V = 1;
        for (int i = 0; i < 4; i++) {
            if (d[i] < 1 || d[i] > 4096) {
                set(YMFLOW_ERR_ARG, "configuration " + std::to_string(c) + ": extents must be in 1..4096");
                delete e;
                return nullptr;
            }
            V *= d[i];
        }
        if (V >= (int64_t(1) << 31) || !volume_addressable(precision, V)) {
            set(YMFLOW_ERR_ARG, "configuration " + std::to_string(c) + ": volume too large");
            delete e;
            return nullptr;
        }
        EnsConf& C = e->confs[c];
        C.g = make_geo(d);
        C.uoff = uo;
        C.zoff = zo;
        C.hoff = ho;
        uo += int64_t(link_field_bytes(e->prec, V));
        zo += int64_t(force_field_bytes(e->prec, V));
        ho += int64_t(plane_field_bytes(e->prec, V));
        e->max_v = std::max(e->max_v, V);
        e->signature += std::to_string(d[0]) + "x" + std::to_string(d[1]) + "x" + std::to_string(d[2]) + "x" +
                        std::to_string(d[3]) + ";";
    }
    e->signature += "p" + std::to_string(precision);
    e->pool_links = uo;
    e->pool_force = zo;
    int r = YMFLOW_OK;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) r = YMFLOW_ERR_CUDA;
    if (r == YMFLOW_OK) r = ens_alloc(e, &e->u[0], size_t(uo), "link pool 0");
    if (r == YMFLOW_OK) r = ens_alloc(e, &e->u[1], size_t(uo), "link pool 1");
    if (r == YMFLOW_OK) r = ens_alloc(e, &e->z, size_t(zo), "generator pool");
    // FP32 ensembles flow with the two-kernel stage, as FP32 single contexts do
    // FP32 ensembles flow with the two-kernel stage, FP64 ones with the fused
    // kernel until the autotuner or ymflow_ensemble_set_tuning picks the
    // per-run two-kernel form; an FP64 ensemble without room for the plane
    // generators keeps the fused kernel only
    e->split = precision != YMFLOW_FP64;
    if (r == YMFLOW_OK) {
        r = ens_alloc(e, &e->h, size_t(ho), "plane-generator pool");
        if (r == YMFLOW_ERR_OOM && !e->split) {
            r = YMFLOW_OK;
            e->err.clear();
        }
    }
    for (int c = 0; c < nconf; c++) {  // runs of consecutive configurations with equal extents
        const EnsConf& C = e->confs[c];
        if (c > 0 && std::equal(C.g.n, C.g.n + 4, e->confs[c - 1].g.n)) {
            e->runs.back().r.nconf++;
            continue;
        }
        EnsRunLaunch L;
        L.r.g = C.g;
        L.r.nconf = 1;
        L.r.nblk = (C.g.V + 31) / 32;
        L.r.ustride = int64_t(link_field_bytes(e->prec, C.g.V));
        L.r.zstride = int64_t(force_field_bytes(e->prec, C.g.V));
        L.r.hstride = int64_t(plane_field_bytes(e->prec, C.g.V));
        L.uoff = C.uoff;
        L.zoff = C.zoff;
        L.hoff = C.hoff;
        e->runs.push_back(L);
    }
    if (r == YMFLOW_OK && e->h && e->runs.size() > 1) {  // up to four concurrent branches
        const size_t ns = std::min<size_t>(e->runs.size(), 4);
        if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) r = YMFLOW_ERR_CUDA;
        for (size_t k = 0; k < ns && r == YMFLOW_OK; k++) {
            cudaStream_t st = nullptr;
            cudaEvent_t ev = nullptr;
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
                r = YMFLOW_ERR_CUDA;
                break;
            }
            e->side.push_back(st);
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
                r = YMFLOW_ERR_CUDA;
                break;
            }
            e->side_done.push_back(ev);
        }
        if (r == YMFLOW_OK && e->side_done.size() != e->side.size()) r = YMFLOW_ERR_CUDA;
    }
    if (r == YMFLOW_OK) r = ens_alloc(e, (void**)&e->confs_dev, sizeof(EnsConf) * nconf, "work list");
    if (r == YMFLOW_OK) r = ens_alloc(e, (void**)&e->deviation, sizeof(unsigned long long), "drift flag");
    if (r == YMFLOW_OK) {
        // most observable blocks of any configuration (the kernel's grid is capped)
        int cap = 1;
        for (const EnsConf& C : e->confs) cap = std::max(cap, obs_blocks(C.g));
        e->partial_cap = cap;
        r = ens_alloc(e, (void**)&e->partials, size_t(e->partial_cap) * 3 * sizeof(double), "partials");
    }
    if (r == YMFLOW_OK && (cudaEventCreate(&e->ev0) != cudaSuccess || cudaEventCreate(&e->ev1) != cudaSuccess))
        r = YMFLOW_ERR_CUDA;
    if (r == YMFLOW_OK) r = set_block(e, 128);
    if (r == YMFLOW_OK && prepare_ens_tile(e->prec) != cudaSuccess) {
        const cudaError_t ce = cudaGetLastError();
        r = ecuda(e, ce == cudaSuccess ? cudaErrorInvalidValue : ce, "tile kernel set-up");
    }
    if (r == YMFLOW_OK) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(e->signature);
        if (it != g_tune_cache.end()) {
            r = apply_tuning(e, it->second);
            e->tuned = true;
        }
    }
    if (r != YMFLOW_OK) {
        set(r, e->err.empty() ? "ensemble setup failed" : e->err);
        ymflow_ensemble_destroy(e);
        return nullptr;
    }
    if (status) *status = YMFLOW_OK;
    return e;
}

void ymflow_ensemble_destroy(ymflow_ens* e) {
    if (!e) return;
    DeviceGuard guard(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    drop_graphs(e);
    for (void* p : {e->u[0], e->u[1], e->z, e->h, (void*)e->confs_dev, (void*)e->staging, (void*)e->partials,
                    (void*)e->meas, (void*)e->deviation})
        if (p) cudaFree(p);
    if (e->meas_host) cudaFreeHost(e->meas_host);
    for (cudaStream_t st : e->side) cudaStreamDestroy(st);
    for (cudaEvent_t ev : e->side_done) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

const char* ymflow_ensemble_last_error(const ymflow_ens* e) { return e ? e->err.c_str() : g_ens_create_error.c_str(); }

int ymflow_ensemble_upload(ymflow_ens* e, int conf, const double* links) {
    if (!e || !links || conf < 0 || conf >= e->nconf) return efail(e, YMFLOW_ERR_ARG, "bad argument to upload");
    DeviceGuard guard(e->device);
    if (!e->staging) {
        int r = ens_alloc(e, (void**)&e->staging, size_t(e->max_v) * 4 * 18 * sizeof(double), "staging buffer");
        if (r != YMFLOW_OK) return r;
    }
    const EnsConf& C = e->confs[conf];
    YE_CK(e, cudaMemcpyAsync(e->staging, links, size_t(C.g.V) * 72 * sizeof(double), cudaMemcpyHostToDevice,
                             e->stream),
          "upload copy");
    YE_CK(e, launch_pack(e->prec, e->staging, conf_links(e, conf), C.g, e->stream), "pack");
    YE_CK(e, cudaStreamSynchronize(e->stream), "upload");
    e->loaded[conf] = 1;
    return YMFLOW_OK;
}

int ymflow_ensemble_download(ymflow_ens* e, int conf, double* links) {
    if (!e || !links || conf < 0 || conf >= e->nconf) return efail(e, YMFLOW_ERR_ARG, "bad argument to download");
    if (!e->loaded[conf]) return efail(e, YMFLOW_ERR_STATE, "configuration not loaded");
    DeviceGuard guard(e->device);
    if (!e->staging) {
        int r = ens_alloc(e, (void**)&e->staging, size_t(e->max_v) * 4 * 18 * sizeof(double), "staging buffer");
        if (r != YMFLOW_OK) return r;
    }
    const EnsConf& C = e->confs[conf];
    YE_CK(e, launch_unpack(e->prec, conf_links(e, conf), e->staging, C.g, e->stream), "unpack");
    YE_CK(e, cudaMemcpyAsync(links, e->staging, size_t(C.g.V) * 72 * sizeof(double), cudaMemcpyDeviceToHost,
                             e->stream),
          "download copy");
    YE_CK(e, cudaStreamSynchronize(e->stream), "download");
    return YMFLOW_OK;
}

int ymflow_ensemble_init_links(ymflow_ens* e, int conf, int kind, double a, uint64_t seed, uint32_t config,
                               double haar_frac) {
    if (!e || conf < 0 || conf >= e->nconf) return efail(e, YMFLOW_ERR_ARG, "bad configuration index");
    if (kind != YMFLOW_FIELD_COLD && kind != YMFLOW_FIELD_EXPIAH) return efail(e, YMFLOW_ERR_ARG, "unknown kind");
    DeviceGuard guard(e->device);
    const EnsConf& C = e->confs[conf];
    YE_CK(e, launch_init_links(e->prec, conf_links(e, conf), C.g, kind == YMFLOW_FIELD_COLD ? kCold : kExpIAH, a,
                               seed, config, e->stream),
          "init");
    if (haar_frac > 0.0)
        YE_CK(e, launch_haar_mix(e->prec, conf_links(e, conf), C.g, haar_frac, seed, config, e->stream), "haar");
    YE_CK(e, cudaStreamSynchronize(e->stream), "init links");
    e->loaded[conf] = 1;
    return YMFLOW_OK;
}

int ymflow_ensemble_flow(ymflow_ens* e, double eps, int nsteps, int measure_every, int reunit_every,
                         ymflow_obs* out, int rows_cap, int* n_rows) {
    NvtxRange range("ymflow_ensemble_flow");
    if (!e) return YMFLOW_ERR_ARG;
    if (n_rows) *n_rows = 0;
    if (nsteps < 0) return efail(e, YMFLOW_ERR_ARG, "nsteps < 0");
    for (int c = 0; c < e->nconf; c++)
        if (!e->loaded[c]) return efail(e, YMFLOW_ERR_STATE, "configuration " + std::to_string(c) + " not loaded");
    int rows = 1;
    for (int s = 1; s <= nsteps; s++)
        if ((measure_every > 0 && s % measure_every == 0) || s == nsteps) rows++;
    if (out && rows_cap < rows) return efail(e, YMFLOW_ERR_CAPACITY, "output holds too few rows");
    DeviceGuard guard(e->device);
    int r = ensure_ens_meas(e, rows);
    if (r != YMFLOW_OK) return r;
    std::vector<int64_t> rs(rows);
    std::vector<double> rt(rows);
    const bool reunit = e->prec != YMFLOW_FP64 && reunit_every > 0;
    if (reunit) YE_CK(e, cudaMemsetAsync(e->deviation, 0, sizeof(unsigned long long), e->stream), "reset drift");
    int row = 0;
    if ((r = enqueue_ens_measure(e, row)) != YMFLOW_OK) return r;
    rs[row] = e->step;
    rt[row] = e->t;
    row++;
    for (int s = 1; s <= nsteps; s++) {
        if ((r = run_ens_step(e, eps)) != YMFLOW_OK) return r;
        e->step++;
        e->t += eps;
        if (reunit && s % reunit_every == 0)
            for (int c = 0; c < e->nconf; c++)
                YE_CK(e, launch_reunitarize(e->prec, conf_links(e, c), e->confs[c].g, e->deviation, e->stream),
                      "reunitarise");
        if ((measure_every > 0 && s % measure_every == 0) || s == nsteps) {
            if ((r = enqueue_ens_measure(e, row)) != YMFLOW_OK) return r;
            rs[row] = e->step;
            rt[row] = e->t;
            row++;
        }
    }
    YE_CK(e, cudaMemcpyAsync(e->meas_host, e->meas, size_t(rows) * e->nconf * 4 * sizeof(double),
                             cudaMemcpyDeviceToHost, e->stream),
          "rows copy");
    unsigned long long bits = 0;
    if (reunit)
        YE_CK(e, cudaMemcpyAsync(&bits, e->deviation, sizeof(bits), cudaMemcpyDeviceToHost, e->stream), "drift copy");
    YE_CK(e, cudaStreamSynchronize(e->stream), "ensemble flow");
    bool nonfinite = false;
    for (int i = 0; i < rows; i++)
        for (int c = 0; c < e->nconf; c++) {
            const double* m = e->meas_host + 4 * (size_t(i) * e->nconf + c);
            if (out) {
                ymflow_obs& o = out[size_t(i) * e->nconf + c];
                o.step = int32_t(rs[i]);
                o.pad = 0;
                o.t = rt[i];
                o.plaq = m[0];
                o.topc = m[1];
                o.energy = m[2];
                o.t2E = -rt[i] * rt[i] * m[2] / (64.0 * double(e->confs[c].g.V));
            }
            if (m[3] != 0.0) nonfinite = true;
        }
    if (n_rows) *n_rows = rows;
    if (nonfinite) return efail(e, YMFLOW_ERR_NONFINITE, "non-finite observable during the ensemble flow");
    if (reunit) {
        double d;
        std::memcpy(&d, &bits, sizeof(d));
        if (d > 1e-3) return efail(e, YMFLOW_ERR_UNITARITY, "links drifted from SU(3)");
    }
    return YMFLOW_OK;
}

int ymflow_ensemble_time_steps(ymflow_ens* e, double eps, int nsteps, float* elapsed_ms) {
    NvtxRange range("ymflow_ensemble_time_steps");
    if (!e || !elapsed_ms || nsteps < 1) return efail(e, YMFLOW_ERR_ARG, "bad argument to time_steps");
    for (int c = 0; c < e->nconf; c++)
        if (!e->loaded[c]) return efail(e, YMFLOW_ERR_STATE, "configuration not loaded");
    DeviceGuard guard(e->device);
    YE_CK(e, cudaEventRecord(e->ev0, e->stream), "event");
    for (int s = 0; s < nsteps; s++) {
        int r = run_ens_step(e, eps);
        if (r != YMFLOW_OK) return r;
        e->step++;
        e->t += eps;
    }
    YE_CK(e, cudaEventRecord(e->ev1, e->stream), "event");
    YE_CK(e, cudaEventSynchronize(e->ev1), "timed steps");
    YE_CK(e, cudaEventElapsedTime(elapsed_ms, e->ev0, e->ev1), "elapsed");
    return YMFLOW_OK;
}

int ymflow_ensemble_autotune(ymflow_ens* e, double eps, int* block_out, int* grid_out) {
    if (!e) return YMFLOW_ERR_ARG;
    for (int c = 0; c < e->nconf; c++)
        if (!e->loaded[c]) return efail(e, YMFLOW_ERR_STATE, "configuration not loaded");
    DeviceGuard guard(e->device);
    auto report = [&]() {
        if (block_out) *block_out = e->tile ? e->tile_threads : e->block;
        if (grid_out) *grid_out = e->tile ? e->tile_grid : e->grid;
    };
    bool cached = false;
    EnsTuning tn{};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(e->signature);
        if (it != g_tune_cache.end()) {
            cached = true;
            tn = it->second;
        }
    }
    if (cached) {  // an ensemble of the same sizes and precision was tuned in this process
        const int r = apply_tuning(e, tn);
        if (r != YMFLOW_OK) return r;
        drop_graphs(e);
        e->tuned = true;
        report();
        return YMFLOW_OK;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    // candidates: the per-link kernel over {one block per item, 1x and 2x the
    // resident blocks} (FP64) or the two-kernel stage (FP32), and the tile
    // kernel with 128 / 256 / 384 / 512 threads (tiles of at most that many sites)
    std::vector<EnsTuning> cands;
    if (e->prec != YMFLOW_FP64) {
        cands.push_back({1, 128, 0});
        cands.push_back({3, 128, 0});
    } else {
        const int resident = ens_max_resident(e->prec, 128);
        for (int grid : {0, resident * sms, 2 * resident * sms}) cands.push_back({0, 128, grid});
        if (e->h) cands.push_back({3, 128, 0});
    }
    for (int threads : {128, 256, 384, 512}) cands.push_back({2, threads, 0});
    const bool was_split = e->split;
    float best = 1e30f;
    EnsTuning pick = cands.front();
    for (const EnsTuning& ch : cands) {
        e->tile = false;
        e->by_runs = ch.form == 3;
        e->split = ch.form == 1 || ch.form == 3;
        if (ch.form == 2) {
            if (!set_tiles(e, ch.block)) continue;
            e->tile = true;
        } else {
            e->grid = ch.grid;
            int r = set_block(e, ch.block);
            if (r != YMFLOW_OK) return r;
        }
        const float ms = time_stage0(e, eps, 3);
        if (ms < 0.f) return ecuda(e, cudaGetLastError(), "tuning launch");
        if (ms < best) {
            best = ms;
            pick = ch;
        }
    }
    e->split = was_split;  // a tile pick flows over the form the ensemble had
    const int r = apply_tuning(e, pick);
    if (r != YMFLOW_OK) return r;
    drop_graphs(e);
    e->tuned = true;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[e->signature] = pick;
    }
    report();
    return YMFLOW_OK;
}

int ymflow_ensemble_set_tuning(ymflow_ens* e, int stage_form, int block, int grid) {
    if (!e) return YMFLOW_ERR_ARG;
    DeviceGuard guard(e->device);
    if (stage_form == 2) {
        if (block < 32 || block > 512 || !set_tiles(e, block))
            return efail(e, YMFLOW_ERR_ARG, "no tiling of every configuration within " + std::to_string(block) +
                                                " threads and 227 KB of shared memory");
        e->tile = true;
        e->by_runs = false;
    } else if (stage_form == 0 || ((stage_form == 1 || stage_form == 3) && e->h)) {
        if (stage_form != 0 && block != 128) return efail(e, YMFLOW_ERR_ARG, "the two-kernel stage runs 128 threads");
        if (block != 128) return efail(e, YMFLOW_ERR_ARG, "the per-link kernel runs 128 threads");
        if (grid < 0) return efail(e, YMFLOW_ERR_ARG, "grid < 0");
        e->tile = false;
        e->split = stage_form == 1 || stage_form == 3;
        e->by_runs = stage_form == 3;
        e->grid = stage_form == 0 ? grid : 0;
        const int r = set_block(e, 128);
        if (r != YMFLOW_OK) return r;
    } else {
        return efail(e, YMFLOW_ERR_ARG, "stage form is 0, 1, 2 or 3 (1 and 3 need the plane-generator pool)");
    }
    YE_CK(e, cudaStreamSynchronize(e->stream), "set tuning");
    drop_graphs(e);
    return YMFLOW_OK;
}

int ymflow_ensemble_tuning(const ymflow_ens* e, int* stage_form, int* block, int* grid) {
    if (!e) return YMFLOW_ERR_ARG;
    if (stage_form) *stage_form = e->tile ? 2 : (e->split ? (e->by_runs ? 3 : 1) : 0);
    if (block) *block = e->tile ? e->tile_threads : e->block;
    if (grid) *grid = e->tile ? e->tile_grid : e->grid;
    return YMFLOW_OK;
}

int ymflow_ensemble_reset_time(ymflow_ens* e) {
    if (!e) return YMFLOW_ERR_ARG;
    e->step = 0;
    e->t = 0.0;
    return YMFLOW_OK;
}

}  // extern "C"
