// K1t: one RK3 stage of one configuration in a single kernel, the plaquette
// field of a tile of sites held in shared memory (design and device code in
// flow_tile.cuh), and its host side: tile shapes, shared-memory opt-in and the
// persistent grid.
#include <algorithm>

#include "flow_tile.cuh"

namespace ym {

// One block per run of units, streaming along t (device code in flow_tile.cuh).
// LEAN: compiled for 64 registers (1024-thread blocks, or two 512-thread
// blocks per SM) instead of 128 (up to 512 threads, one block per SM).
template <class F, int STAGE, int LEAN>
__global__ void __launch_bounds__(LEAN ? 1024 : 512, 1)
    rk_tile_stage_kernel(F in, F out, ForceField<typename F::Real> zf, Geo g, TileShape tp, typename F::Real eps) {
    using V = typename HVec<typename F::Real>::V;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    V* const sm = reinterpret_cast<V*>(tile_smem);
    const int Lt = g.n[3];
    const int u0 = int((long long)blockIdx.x * tp.units / gridDim.x);
    const int u1 = int((long long)(blockIdx.x + 1) * tp.units / gridDim.x);
    int cur = 0;
    for (int u = u0; u < u1; u++) {
        const int col = u / Lt, t = u - col * Lt;
        tile_unit<F, STAGE>(in, out, zf, g, tp, eps, sm, int(threadIdx.x), int(blockDim.x), col, t,
                            u == u0 || t == 0, cur);
        cur ^= 1;
    }
}

template <class F, int LEAN>
static void* tile_kernel_ptr(int stage) {
    switch (stage) {
        case 0: return (void*)rk_tile_stage_kernel<F, 0, LEAN>;
        case 1: return (void*)rk_tile_stage_kernel<F, 1, LEAN>;
        default: return (void*)rk_tile_stage_kernel<F, 2, LEAN>;
    }
}

static void* tile_kernel(int prec, int stage, int lean) {
    switch (prec) {
        case kFP64: return lean ? tile_kernel_ptr<FieldD18, 1>(stage) : tile_kernel_ptr<FieldD18, 0>(stage);
        case kFP32_18: return lean ? tile_kernel_ptr<FieldF18, 1>(stage) : tile_kernel_ptr<FieldF18, 0>(stage);
        default: return lean ? tile_kernel_ptr<FieldF12, 1>(stage) : tile_kernel_ptr<FieldF12, 0>(stage);
    }
}

size_t tile_smem_bytes(int prec, const TileShape& tp) {
    const size_t entry = prec == kFP64 ? 64 : 32;
    return entry * size_t(9 * tp.ns + 3 * (tp.nfy + tp.nfz));
}

bool make_tile_shape(int prec, const Geo& g, int ty, int tz, TileShape* out, bool whole_warps, int lpt, int lean) {
    const int Lx = g.n[0], Ly = g.n[1], Lz = g.n[2];
    if (ty < 1 || tz < 1 || ty > Ly || tz > Lz || Ly % ty || Lz % tz) return false;
    if (g.site0 != 0 || g.site1 != g.V) return false;  // whole-lattice contexts
    if (lpt != 1 && lpt != 2 && lpt != 4) return false;
    const long long ns = (long long)Lx * ty * tz;
    const long long threads = ns * (4 / lpt);
    // whole warps of consecutive sites: every warp inside one (x, y) run
    if (ns > 512 || ns < (whole_warps ? 64 : 32) || (whole_warps && (Lx * ty) % 32)) return false;
    if (threads > (lean ? 1024 : 512)) return false;
    TileShape tp;
    tp.ty = ty;
    tp.tz = tz;
    tp.ns = int(ns);
    tp.lpt = lpt;
    tp.threads = int(threads);
    tp.lean = lean ? 1 : 0;
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
    for (int lean = 0; lean < 2; lean++)
        for (int s = 0; s < 3; s++) {
            cudaError_t e = cudaFuncSetAttribute(tile_kernel(prec, s, lean),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

cudaError_t tile_grid(int prec, int device, TileShape* tp) {
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_kernel(prec, 1, tp->lean), tp->threads,
                                                      tile_smem_bytes(prec, *tp));
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    tp->grid = std::min(tp->units, sms * per_sm);
    return cudaSuccess;
}

template <class F, int LEAN>
static cudaError_t launch_tile_typed(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g,
                                     const TileShape& tp, double eps, cudaStream_t st) {
    using R = typename F::Real;
    F in{const_cast<void*>(uin), g.V}, out{uout, g.V};
    ForceField<R> zf{z, g.V};
    const R e = R(stage == 0 ? eps * 0.25 : eps);
    const size_t sm = tile_smem_bytes(prec, tp);
    switch (stage) {
        case 0: rk_tile_stage_kernel<F, 0, LEAN><<<tp.grid, tp.threads, sm, st>>>(in, out, zf, g, tp, e); break;
        case 1: rk_tile_stage_kernel<F, 1, LEAN><<<tp.grid, tp.threads, sm, st>>>(in, out, zf, g, tp, e); break;
        default: rk_tile_stage_kernel<F, 2, LEAN><<<tp.grid, tp.threads, sm, st>>>(in, out, zf, g, tp, e); break;
    }
    return cudaGetLastError();
}

template <class F>
static cudaError_t launch_tile_form(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g,
                                    const TileShape& tp, double eps, cudaStream_t st) {
    return tp.lean ? launch_tile_typed<F, 1>(prec, stage, uin, uout, z, g, tp, eps, st)
                   : launch_tile_typed<F, 0>(prec, stage, uin, uout, z, g, tp, eps, st);
}

cudaError_t launch_rk_tile_stage(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g,
                                 const TileShape& tp, double eps, cudaStream_t st) {
    if (tp.grid < 1 || tp.ns < 1 || tp.threads != tp.ns * (4 / tp.lpt) || tp.threads > (tp.lean ? 1024 : 512))
        return cudaErrorInvalidValue;
    switch (prec) {
        case kFP64: return launch_tile_form<FieldD18>(prec, stage, uin, uout, z, g, tp, eps, st);
        case kFP32_18: return launch_tile_form<FieldF18>(prec, stage, uin, uout, z, g, tp, eps, st);
        case kFP32_12: return launch_tile_form<FieldF12>(prec, stage, uin, uout, z, g, tp, eps, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ym
