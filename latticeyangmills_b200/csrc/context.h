// Internal to libymflow: the flow context and the helpers the ABI files share.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "api_util.h"
#include "kernels.h"
#include "ymflow.h"

using ym::Geo;

struct ymflow_ctx {
    int dims[4] = {0, 0, 0, 0};
    int prec = 0;
    int device = 0;
    Geo geo{};
    cudaStream_t stream = nullptr;
    void* u[2] = {nullptr, nullptr};  // ping-pong link buffers
    int cur = 0;                      // which of u[] holds the current field
    void* z = nullptr;                // RK generator, 8 reals per link
    void* hfield = nullptr;           // plaquette field of the two-kernel stage (stage_form 1)
    int stage_form = 0;               // 0: fused stage kernel, 1: plaquette field + stage kernel,
                                      // 2: one kernel with the tile's plaquette field in shared memory
    ym::TileShape tile{};             // stage form 2's tiling (valid when tile_ok)
    bool tile_ok = false;
    int timed_reunit = 0;             // time_steps / time_kernels: reunitarise every n-th step (0: never)
    double* staging = nullptr;        // .bin-layout device buffer for upload/download
    size_t staging_bytes = 0;
    double* partials = nullptr;       // observables: 3 doubles per block
    int partial_cap = 0;
    double* meas = nullptr;           // measurement rows on the device, 4 doubles each
    int meas_cap = 0;
    double* meas_host = nullptr;      // pinned copy of the rows
    unsigned long long* deviation = nullptr;  // reunitarisation drift (ordered bits)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    double graph_eps[2] = {0.0, 0.0};
    int graph_block[2] = {0, 0};
    std::vector<cudaEvent_t> events;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int block = 128;
    bool use_graph = true;
    bool loaded = false;
    int64_t step = 0;
    double t = 0.0;
    uint32_t gen_sweep = 0;           // Metropolis sweeps since the last cold/hot start
    // One time slab of a configuration decomposed along t (ymflow_create_slab):
    // global slices [t0, t0 + nt) in local slices 1..nt, halos in 0 and nt + 1.
    bool slab = false;
    int t0 = 0, nt = 0;
    int gdims[4] = {0, 0, 0, 0};
    // One block of a configuration decomposed in several directions
    // (ymflow_create_block): its own sites [origin, origin + extent) of the
    // configuration, held in a local lattice with one halo layer on each side
    // in every direction the decomposition splits (geo.halo_mask).
    bool is_block = false;
    int borigin[4] = {0, 0, 0, 0};
    void* comm = nullptr;             // NCCL communicator (ymflow_slab_connect)
    int rank = 0, nranks = 0, lower = -1, upper = -1;
    int64_t bytes = 0;
    std::string err;
};

namespace ym {

int fail(ymflow_ctx* c, int code, const std::string& msg);
// The text ymflow_last_error(NULL) returns after a failed constructor.
void set_create_error(const std::string& msg);
int cuda_fail(ymflow_ctx* c, cudaError_t e, const char* what);

#define YM_CK(ctx, call, what)                                      \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return ::ym::cuda_fail(ctx, e_, what); \
    } while (0)

int ensure_meas(ymflow_ctx* c, int rows);
// One RK3 stage (0, 1, 2) of the context's stage form from link buffer `in`
// into `out` over all of the context's sites.
cudaError_t enqueue_stage(ymflow_ctx* c, int stage, const void* in, void* out, double eps);
// Observables of the current field (the context's sites) into measurement row `row` on the device.
int enqueue_measure(ymflow_ctx* c, int row);
void fill_obs(const ymflow_ctx* c, const double* m, int64_t step, double t, ymflow_obs* o);

// Slab transport (slab.cu): halo exchange of link buffer u[buf] and the sum of a
// measurement row over the ranks, both on the context's stream.
int slab_exchange(ymflow_ctx* c, int buf);
int slab_reduce_row(ymflow_ctx* c, double* row_device);
void slab_release(ymflow_ctx* c);

}  // namespace ym
