// Host-side launchers of the device kernels (one translation unit per kernel
// family).  All take a CUDA stream and return the launch's cudaError_t.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "field.cuh"

namespace ym {

enum Precision { kFP64 = 0, kFP32_18 = 1, kFP32_12 = 2 };

// bytes of one stored link / one stored generator for a precision
inline int link_elems(int prec) { return prec == kFP32_12 ? 6 : 9; }
inline size_t link_bytes(int prec) { return prec == kFP64 ? 9 * 16 : size_t(link_elems(prec)) * 8; }
inline size_t force_bytes(int prec) { return prec == kFP64 ? 64 : 32; }
// device bytes of a link field / a generator field (volume padded to whole warp groups)
inline size_t link_field_bytes(int prec, int64_t V) { return size_t(4 * padded_sites(V)) * link_bytes(prec); }
inline size_t force_field_bytes(int prec, int64_t V) { return size_t(4 * padded_sites(V)) * force_bytes(prec); }
// device bytes of a plaquette field: the six H_p of every site, generator-sized
inline size_t plane_field_bytes(int prec, int64_t V) { return size_t(6 * padded_sites(V)) * force_bytes(prec); }
// whether field.cuh's 32-bit offsets (16-byte units) reach every link of V sites
inline bool volume_addressable(int prec, int64_t V) { return link_field_bytes(prec, V) / 16 < (size_t(1) << 32); }

// One RK3 stage (0, 1, 2) over every link: staples, generator, RK combination
// with the stored generator, e^{i eps_stage Z} and the link update uin -> uout.
cudaError_t launch_rk_stage(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g, double eps,
                            int block, cudaStream_t st);

// The same stage as two kernels (flow_split.cu): the six plaquettes' generators
// of every site of u into h (plane_field_bytes), then the stage with each
// link's force built from h (h must hold uin's plaquette field).
cudaError_t launch_plaq_field(int prec, const void* u, void* h, const Geo& g, cudaStream_t st);
cudaError_t launch_rk_split_stage(int prec, int stage, const void* uin, void* uout, void* z, const void* h,
                                  const Geo& g, double eps, cudaStream_t st);
// Its slab form with the halo stores of launch_rk_stage_halo (h must hold the
// plane generators of local slices 0..nt, see plaq_range).
cudaError_t launch_rk_split_stage_halo(int prec, int stage, const void* uin, void* uout, void* z, const void* h,
                                       const Geo& g, double eps, void* lower_out, int lower_v, int lower_t,
                                       void* upper_out, int upper_v, cudaStream_t st);
// The same stage in one kernel with the plane generators of a tile of sites in
// shared memory (flow_tile.cu): tiles of whole x lines x ty x tz (y, z) of one
// time slice, one thread per site, each block streaming along t through a run
// of (tile column, t) units.
struct TileShape {
    int ty, tz;      // tile extent in y and z
    int ns;          // sites per tile (Lx ty tz)
    int lpt;         // links a thread advances: 1, 2 or 4
    int threads;     // threads per block: ns 4 / lpt (at most 1024)
    int lean;        // 1: the kernel compiled for 64 registers (1024 threads, or two 512-thread blocks per SM)
    int nyt, nzt;    // tiles along y and z
    int nfy, nfz;    // sites of the recomputed lower y / z faces (0: the tile spans the extent)
    int units;       // tile columns x time slices
    int grid;        // blocks (persistent: min(units, SMs x resident blocks))
};
// Whether (ty, tz) tiles the whole-lattice geometry g (whole warps per x-y run,
// 64..512 threads, shared memory within 227 KB); fills *out (grid left 0).
// whole_warps = false drops the warp rule (x-y runs of any length, 32..512
// threads): correct, with warps straddling rows (the ensemble's 12^4).
bool make_tile_shape(int prec, const Geo& g, int ty, int tz, TileShape* out, bool whole_warps = true, int lpt = 4,
                     int lean = 0);
size_t tile_smem_bytes(int prec, const TileShape& tp);
// Opt the tile kernels of a precision into their shared memory (per device).
cudaError_t prepare_tile_kernels(int prec);
// tp->grid for `device` from the kernel's occupancy.
cudaError_t tile_grid(int prec, int device, TileShape* tp);
cudaError_t launch_rk_tile_stage(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g,
                                 const TileShape& tp, double eps, cudaStream_t st);

// The sites whose plane generators a stage reads: a slab's links of slice 1
// read those of halo slice 0, so its range starts there (g.site0 = one slice).
inline Geo plaq_range(const Geo& g, bool slab) {
    Geo p = g;
    if (slab) p.site0 = 0;
    return p;
}

// The same stage for a time slab (g.site0 = sites per slice, interior slices
// [1, nt]): each new link of local slice 1 is also stored into the lower slab's
// buffer lower_out (lower_v sites) at its slice lower_t, and each of slice nt
// into upper_out's slice 0: the halo exchange inside the stage kernel.
cudaError_t launch_rk_stage_halo(int prec, int stage, const void* uin, void* uout, void* z, const Geo& g, double eps,
                                 void* lower_out, int lower_v, int lower_t, void* upper_out, int upper_v,
                                 cudaStream_t st);

// D_mu (18 doubles per site, site order) for one direction: the reference's
// PureGauge::computeDerivative(mu).
cudaError_t launch_force(int prec, int mu, const void* u, const Geo& g, double* out, cudaStream_t st);
// e^{iQ} for n Hermitian traceless matrices (18 doubles each).
cudaError_t launch_exp(const double* q, double* r, int64_t n, cudaStream_t st);

// Observables of the sites [g.site0, g.site1): per-block FP64 partial sums (plaq, energy,
// topc) into partials[3 * obs_blocks(g)], then one block folds them in a fixed order into
// out[3] = (plaq, topc, energy) with the reference's normalisations, out[3] = 1.0 when any
// value is not finite.
int obs_blocks(const Geo& g);
cudaError_t launch_observables(int prec, const void* u, const Geo& g, double* partials, cudaStream_t st);
cudaError_t launch_obs_finalize(const double* partials, int nblocks, const Geo& g, double* out, cudaStream_t st);

// .bin layout (site-major, mu, 18 doubles) <-> device layout
// Sites [first, first + n) between a .bin-layout block (aos points at site
// `first`) and the device links; swap = each double byte-reversed.
cudaError_t launch_pack_range(int prec, const double* aos, void* u, const Geo& g, int first, int n, bool swap,
                              cudaStream_t st);
cudaError_t launch_unpack_range(int prec, const void* u, double* aos, const Geo& g, int first, int n, bool swap,
                                cudaStream_t st);
cudaError_t launch_pack(int prec, const double* aos, void* u, const Geo& g, cudaStream_t st);
cudaError_t launch_unpack(int prec, const void* u, double* aos, const Geo& g, cudaStream_t st);

// Seeded fields written straight into the device layout.
enum FieldKind { kCold = 0, kExpIAH = 1 };
cudaError_t launch_init_links(int prec, void* u, const Geo& g, int kind, double a, uint64_t seed, uint32_t config,
                              cudaStream_t st);
cudaError_t launch_haar_mix(int prec, void* u, const Geo& g, double frac, uint64_t seed, uint32_t config,
                            cudaStream_t st);

// One checkerboard sub-sweep of Metropolis updates (generate.cu): every link
// U_mu(x) with site parity `parity`, `hits` proposals each; accepted counts add
// into *accepted.
cudaError_t launch_metropolis(int prec, void* u, const Geo& g, int mu, int parity, double beta, double eps, int hits,
                              uint64_t seed, uint32_t sweep, unsigned long long* accepted, cudaStream_t st);

// FP64 Gram-Schmidt reunitarisation of every link; deviation[0] receives the
// largest |row norm - 1| seen before the fix (as an ordered-int atomic max).
cudaError_t launch_reunitarize(int prec, void* u, const Geo& g, unsigned long long* deviation, cudaStream_t st);

}  // namespace ym
