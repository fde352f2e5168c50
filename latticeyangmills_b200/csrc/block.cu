// Decomposition of one configuration in any set of directions: the
// reference's domain decomposition (src/ParallelTools/parallel.cpp:57-100, a
// Cartesian grid of sub-lattices of extents SubLatticeSize, and the
// second-neighbour ranks of the clover, :117-140) for one process holding the
// blocks on one or several GPUs.
//
// A block context (ymflow_create_block) holds its own sites [origin, origin +
// extent) of the configuration in a local periodic lattice that adds one halo
// layer on each side in every direction the decomposition splits.  Its stage
// kernels are the whole-lattice ones over every local site: the halo sites come
// out wrong (their neighbours wrap inside the local lattice) and are refreshed
// before anything reads them.  The observables count the own sites only
// (Geo::interior).
//
// Halo exchange after every stage (block_exchange), one direction at a time,
// the split directions in order x, y, z, t: each block pulls, with a copy
// kernel on its own stream, its two faces in direction d from its neighbours'
// buffers (own sites next to the face, plus the halo layers of the directions
// exchanged before d).  Carrying the earlier directions' halos fills the
// edges: the sites x + a - b outside the block in two directions at once, which
// the staples (x + mu - nu) and the clover leaves read and which the reference
// fetches from its second-neighbour ranks.  Each block waits for its two
// neighbours in d to finish the previous direction (or the stage) before it
// pulls; a block only ever writes its own halos, so no copy races with another.
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"

namespace ym {
namespace {

// Pull the face (c_d = dst_c) of dst's local lattice from src's (c_d = src_c),
// every other coordinate over the full local extents (the two lattices agree
// in every direction but d).  One thread per link of the face; src may sit on
// another GPU (plain peer loads).
template <class F>
__global__ void halo_pull_kernel(F dst, Geo gd, F src, Geo gs, int d, int dst_c, int src_c) {
    const int64_t l = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int face = gd.V / gd.n[d];
    if (l >= 4 * int64_t(face)) return;
    const int mu = int(l & 3);
    int k = int(l >> 2);
    int sd = 0, ss = 0;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        int ce;
        if (e == d) {
            sd += dst_c * gd.stride[e];
            ss += src_c * gs.stride[e];
            continue;
        }
        const int q = k / gd.n[e];
        ce = k - q * gd.n[e];
        k = q;
        sd += ce * gd.stride[e];
        ss += ce * gs.stride[e];
    }
    dst.store(mu, sd, src.load(mu, ss));
}

template <class F>
cudaError_t launch_pull_typed(void* dst, const Geo& gd, const void* src, const Geo& gs, int d, int dst_c, int src_c,
                              cudaStream_t st) {
    const int64_t links = 4 * int64_t(gd.V / gd.n[d]);
    const int b = 256;
    halo_pull_kernel<F><<<unsigned((links + b - 1) / b), b, 0, st>>>(F{dst, gd.V}, gd, F{const_cast<void*>(src), gs.V},
                                                                      gs, d, dst_c, src_c);
    return cudaGetLastError();
}

cudaError_t launch_pull(int prec, void* dst, const Geo& gd, const void* src, const Geo& gs, int d, int dst_c,
                        int src_c, cudaStream_t st) {
    switch (prec) {
        case kFP64: return launch_pull_typed<FieldD18>(dst, gd, src, gs, d, dst_c, src_c, st);
        case kFP32_18: return launch_pull_typed<FieldF18>(dst, gd, src, gs, d, dst_c, src_c, st);
        case kFP32_12: return launch_pull_typed<FieldF12>(dst, gd, src, gs, d, dst_c, src_c, st);
        default: return cudaErrorInvalidValue;
    }
}

// Whether kernels on `from` can read `to`'s memory (enabling peer access once).
bool block_peer_reachable(int from, int to) {
    if (from == to) return true;
    int ok = 0;
    if (cudaDeviceCanAccessPeer(&ok, from, to) != cudaSuccess || !ok) {
        cudaGetLastError();
        return false;
    }
    DeviceGuard g(from);
    const cudaError_t e = cudaDeviceEnablePeerAccess(to, 0);
    if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) {
        cudaGetLastError();
        return false;
    }
    cudaGetLastError();
    return true;
}

struct BlockEvents {
    std::vector<cudaEvent_t> ev;
    ~BlockEvents() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

// The group's grid: block i sits at grid coordinates (i % g0, i / g0 % g1, ...).
struct BlockGrid {
    int g[4];
    int coord(int i, int d) const {
        for (int e = 0; e < d; e++) i /= g[e];
        return i % g[d];
    }
    int neighbour(int i, int d, int dir) const {
        int stride = 1;
        for (int e = 0; e < d; e++) stride *= g[e];
        const int c = coord(i, d);
        const int cn = (c + dir + g[d]) % g[d];
        return i + (cn - c) * stride;
    }
};

// Refresh every block's halos of its current buffer, direction by direction.
int block_exchange(ymflow_ctx* const* cs, int n, const BlockGrid& G, std::vector<cudaEvent_t>& ev) {
    for (int d = 0; d < 4; d++) {
        if (G.g[d] < 2) continue;
        for (int i = 0; i < n; i++) {
            DeviceGuard g(cs[i]->device);
            YM_CK(cs[i], cudaEventRecord(ev[i], cs[i]->stream), "event record");
        }
        for (int i = 0; i < n; i++) {
            ymflow_ctx* c = cs[i];
            const ymflow_ctx* lo = cs[G.neighbour(i, d, -1)];
            const ymflow_ctx* hi = cs[G.neighbour(i, d, +1)];
            DeviceGuard g(c->device);
            YM_CK(c, cudaStreamWaitEvent(c->stream, ev[G.neighbour(i, d, -1)], 0), "wait lower block");
            YM_CK(c, cudaStreamWaitEvent(c->stream, ev[G.neighbour(i, d, +1)], 0), "wait upper block");
            const int nd = c->geo.n[d];
            // lower halo <- the lower block's last own layer; upper halo <- the upper block's first
            YM_CK(c, launch_pull(c->prec, c->u[c->cur], c->geo, lo->u[lo->cur], lo->geo, d, 0, lo->geo.n[d] - 2,
                                 c->stream),
                  "lower halo pull");
            YM_CK(c, launch_pull(c->prec, c->u[c->cur], c->geo, hi->u[hi->cur], hi->geo, d, nd - 1, 1, c->stream),
                  "upper halo pull");
        }
    }
    return YMFLOW_OK;
}

}  // namespace
}  // namespace ym

using namespace ym;

extern "C" {

ymflow_ctx* ymflow_create_block(const int global_dims[4], const int origin[4], const int extent[4], int precision,
                                int device, int* status) {
    auto bad = [&](const char* m) -> ymflow_ctx* {
        if (status) *status = YMFLOW_ERR_ARG;
        set_create_error(m);
        return nullptr;
    };
    if (!global_dims || !origin || !extent) return bad("global_dims, origin or extent is NULL");
    int local[4];
    int64_t vglobal = 1;
    for (int d = 0; d < 4; d++) {
        if (global_dims[d] < 1 || global_dims[d] > 4096 || extent[d] < 1 || extent[d] > global_dims[d] ||
            origin[d] < 0 || origin[d] >= global_dims[d] || int64_t(origin[d]) + extent[d] > global_dims[d])
            return bad("block [origin, origin + extent) outside the lattice");
        local[d] = extent[d] < global_dims[d] ? extent[d] + 2 : extent[d];
        vglobal *= global_dims[d];
    }
    if (vglobal >= (int64_t(1) << 31)) return bad("lattice volume must be below 2^31 sites");
    ymflow_ctx* c = ymflow_create(local, precision, device, status);
    if (!c) return nullptr;
    c->is_block = true;
    c->tile_ok = false;  // the shared-memory stage is for whole lattices; blocks keep form 0 / 1
    c->use_graph = false;
    c->geo.halo_mask = 0;
    for (int d = 0; d < 4; d++) {
        c->gdims[d] = global_dims[d];
        c->borigin[d] = origin[d];
        c->geo.bext[d] = extent[d];
        if (extent[d] < global_dims[d]) c->geo.halo_mask |= 1 << d;
    }
    c->geo.vglobal = vglobal;
    c->geo.tile_groups = 0;
    return c;
}

int ymflow_block_group_flow(ymflow_ctx* const* ctxs, int n, const int grid[4], double eps, int nsteps,
                            int measure_every, int reunit_every, ymflow_obs* out, int out_cap, int* n_out) {
    NvtxRange range("ymflow_block_group_flow");
    if (n_out) *n_out = 0;
    if (!ctxs || n < 1 || !grid) return YMFLOW_ERR_ARG;
    for (int i = 0; i < n; i++)
        if (!ctxs[i]) return YMFLOW_ERR_ARG;
    ymflow_ctx* c0 = ctxs[0];
    if (nsteps < 0 || !std::isfinite(eps)) return fail(c0, YMFLOW_ERR_ARG, "nsteps < 0 or eps not finite");
    BlockGrid G;
    int64_t cells = 1;
    for (int d = 0; d < 4; d++) {
        if (grid[d] < 1) return fail(c0, YMFLOW_ERR_ARG, "grid extents must be >= 1");
        G.g[d] = grid[d];
        cells *= grid[d];
    }
    if (cells != n) return fail(c0, YMFLOW_ERR_ARG, "the grid does not hold n blocks");
    // the blocks must tile the configuration as a Cartesian grid, block i at
    // grid coordinates (i % g0, i / g0 % g1, ...), origins increasing along each direction
    for (int i = 0; i < n; i++) {
        const ymflow_ctx* c = ctxs[i];
        if (!c->is_block) return fail(c0, YMFLOW_ERR_ARG, "every context must be a block (ymflow_create_block)");
        if (c->prec != c0->prec || std::memcmp(c->gdims, c0->gdims, sizeof(c->gdims)) != 0)
            return fail(c0, YMFLOW_ERR_ARG, "blocks of different configurations or precisions");
        if (c->stage_form != c0->stage_form) return fail(c0, YMFLOW_ERR_ARG, "blocks with different stage forms");
        if (!c->loaded) return fail(c0, YMFLOW_ERR_STATE, "block " + std::to_string(i) + " has no links");
        for (int d = 0; d < 4; d++) {
            const bool split = (c->geo.halo_mask >> d) & 1;
            if (split != (G.g[d] > 1)) return fail(c0, YMFLOW_ERR_ARG, "halos do not match the grid");
            const int cd = G.coord(i, d);
            if (cd == 0 && c->borigin[d] != 0) return fail(c0, YMFLOW_ERR_ARG, "blocks do not start at the origin");
            if (cd > 0) {
                const ymflow_ctx* prev = ctxs[G.neighbour(i, d, -1)];
                if (prev->borigin[d] + prev->geo.bext[d] != c->borigin[d])
                    return fail(c0, YMFLOW_ERR_ARG, "blocks do not tile the lattice in grid order");
            }
            if (cd == G.g[d] - 1 && c->borigin[d] + c->geo.bext[d] != c->gdims[d])
                return fail(c0, YMFLOW_ERR_ARG, "blocks do not cover the lattice");
            for (int e = 0; e < 4; e++)  // neighbours along d share every other direction
                if (e != d && G.g[d] > 1) {
                    const ymflow_ctx* nb = ctxs[G.neighbour(i, d, +1)];
                    if (nb->borigin[e] != c->borigin[e] || nb->geo.bext[e] != c->geo.bext[e])
                        return fail(c0, YMFLOW_ERR_ARG, "blocks are not a Cartesian grid");
                }
        }
        for (int d = 0; d < 4; d++)
            if (G.g[d] > 1)
                for (int dir : {-1, 1})
                    if (!block_peer_reachable(c->device, ctxs[G.neighbour(i, d, dir)]->device))
                        return fail(c0, YMFLOW_ERR_ARG, "neighbouring blocks on GPUs that cannot reach each other");
    }
    int rows = 1;
    for (int s = 1; s <= nsteps; s++)
        if ((measure_every > 0 && s % measure_every == 0) || s == nsteps) rows++;
    if (out && out_cap < rows)
        return fail(c0, YMFLOW_ERR_CAPACITY,
                    "output holds " + std::to_string(out_cap) + " rows, flow needs " + std::to_string(rows));
    BlockEvents evs;
    evs.ev.assign(size_t(n), nullptr);
    for (int i = 0; i < n; i++) {
        DeviceGuard g(ctxs[i]->device);
        int r = ensure_meas(ctxs[i], rows);
        if (r != YMFLOW_OK) return r;
        YM_CK(ctxs[i], cudaEventCreateWithFlags(&evs.ev[i], cudaEventDisableTiming), "event create");
    }
    const bool reunit = c0->prec != YMFLOW_FP64 && reunit_every > 0;
    for (int i = 0; i < n; i++)
        if (reunit) {
            DeviceGuard g(ctxs[i]->device);
            YM_CK(ctxs[i], cudaMemsetAsync(ctxs[i]->deviation, 0, sizeof(unsigned long long), ctxs[i]->stream),
                  "reset drift");
        }
    auto measure = [&](int row) {
        for (int i = 0; i < n; i++) {
            DeviceGuard g(ctxs[i]->device);
            const int r = enqueue_measure(ctxs[i], row);
            if (r != YMFLOW_OK) return r;
        }
        return int(YMFLOW_OK);
    };
    std::vector<int64_t> row_step(rows);
    std::vector<double> row_t(rows);
    int r = block_exchange(ctxs, n, G, evs.ev);
    if (r == YMFLOW_OK) r = measure(0);
    if (r != YMFLOW_OK) return r;
    row_step[0] = c0->step;
    row_t[0] = c0->t;
    int row = 1;
    for (int s = 1; s <= nsteps; s++) {
        for (int stage = 0; stage < 3; stage++) {
            for (int i = 0; i < n; i++) {
                ymflow_ctx* c = ctxs[i];
                DeviceGuard g(c->device);
                YM_CK(c, enqueue_stage(c, stage, c->u[c->cur], c->u[1 - c->cur], eps), "stage launch");
                c->cur = 1 - c->cur;
                // The reunitarisation goes before the step's last exchange:
                // the neighbours then pull the reunitarised links into their
                // halos.  After the exchange it would rewrite links that a
                // neighbour's pull may still be reading.
                if (stage == 2 && reunit && s % reunit_every == 0)
                    YM_CK(c, launch_reunitarize(c->prec, c->u[c->cur], c->geo, c->deviation, c->stream),
                          "reunitarise");
            }
            if ((r = block_exchange(ctxs, n, G, evs.ev)) != YMFLOW_OK) return r;
        }
        for (int i = 0; i < n; i++) {
            ctxs[i]->step++;
            ctxs[i]->t += eps;
        }
        if ((measure_every > 0 && s % measure_every == 0) || s == nsteps) {
            if ((r = measure(row)) != YMFLOW_OK) return r;
            row_step[row] = c0->step;
            row_t[row] = c0->t;
            row++;
        }
    }
    std::vector<double> sum(size_t(rows) * 4, 0.0);
    double drift = 0.0;
    for (int i = 0; i < n; i++) {
        ymflow_ctx* c = ctxs[i];
        DeviceGuard g(c->device);
        unsigned long long bits = 0;
        YM_CK(c, cudaMemcpyAsync(c->meas_host, c->meas, size_t(rows) * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream),
              "measurement copy");
        if (reunit)
            YM_CK(c, cudaMemcpyAsync(&bits, c->deviation, sizeof(bits), cudaMemcpyDeviceToHost, c->stream),
                  "drift copy");
        YM_CK(c, cudaStreamSynchronize(c->stream), "block group flow");
        for (int k = 0; k < rows * 4; k++) sum[k] += c->meas_host[k];
        double dv;
        std::memcpy(&dv, &bits, sizeof(dv));
        drift = std::fmax(drift, dv);
    }
    bool nonfinite = false;
    for (int k = 0; k < rows; k++) {
        if (out) fill_obs(c0, sum.data() + 4 * k, row_step[k], row_t[k], out + k);
        if (sum[4 * k + 3] != 0.0) nonfinite = true;
    }
    if (n_out) *n_out = rows;
    if (nonfinite) return fail(c0, YMFLOW_ERR_NONFINITE, "non-finite observable during the flow");
    if (reunit && drift > 1e-3)
        return fail(c0, YMFLOW_ERR_UNITARITY, "links drifted from SU(3): |row norm - 1| = " + std::to_string(drift));
    return YMFLOW_OK;
}

}  // extern "C"
