// Decomposition of one configuration along t into slabs (the reference's
// domain decomposition, src/ParallelTools/parallel.cpp:57-100, restricted to
// the time direction).  A slab context (ymflow_create_slab) holds its nt time
// slices in local slices 1..nt and one halo slice on each side (0 and nt + 1),
// which every stage reads for the staples and the observables read for the
// clover leaves: a one-slice halo covers both, since no path of either leaves
// the slab by more than one step in t.  The stage and observables kernels run
// on the interior sites only; after each stage the new interior boundary
// slices are copied into the neighbours' halos.
//
// Two transports:
//  * NCCL between processes (one per GPU): ymflow_slab_connect joins a
//    communicator; ymflow_flow / ymflow_observables then exchange halos with
//    grouped ncclSend/ncclRecv on the context's stream and sum each
//    measurement row with ncclAllReduce.  NCCL is loaded at run time
//    (YMFLOW_NCCL_LIB, else the libnccl.so.2 already in the process, else the
//    loader's), so the library needs it only when this is used.
//  * Inside one process: ymflow_slab_group_flow flows the slab contexts of one
//    configuration (on one or several GPUs) stage by stage.  Each slab's stage
//    kernel also stores its new boundary links straight into its neighbours'
//    halo slices (peer stores over NVLink when they sit on other GPUs): the
//    exchange is part of the stage.  Before the next stage every slab's stream
//    waits for both neighbours' stage events; no kernel waits on another.
//    Where two GPUs cannot reach each other's memory (or with
//    YMFLOW_SLAB_COPY_EXCHANGE set) the halos are cudaMemcpyPeerAsync copies
//    after the stage instead.
//
// In the warp-group layout a time slice of one direction is one contiguous run
// of the link buffer (the slab's spatial volume is a multiple of 32 sites), so
// a halo is four runs, one per direction, sent and received in place.
#include <dlfcn.h>
#include <nccl.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "context.h"

namespace ym {
namespace {

// --- NCCL, resolved at run time ------------------------------------------------
struct NcclApi {
    bool loaded = false;
    std::string why;
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*group_start)() = nullptr;
    ncclResult_t (*group_end)() = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};

const NcclApi& nccl() {
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        // Which NCCL: YMFLOW_NCCL_LIB (a path) first, then one the process has
        // already loaded (a framework's), then the loader's libnccl.so.2.  A
        // process must hold one NCCL: a framework imported later binds to the
        // libnccl.so.2 loaded here, which must then be the one it was built for.
        void* h = nullptr;
        if (const char* path = std::getenv("YMFLOW_NCCL_LIB")) h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL | RTLD_NOLOAD);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            api.why = "libnccl.so.2 not found";
            return;
        }
        auto sym = [&](const char* n) { return dlsym(h, n); };
        api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(sym("ncclGetUniqueId"));
        api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(sym("ncclCommInitRank"));
        api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(sym("ncclCommDestroy"));
        api.send = reinterpret_cast<decltype(api.send)>(sym("ncclSend"));
        api.recv = reinterpret_cast<decltype(api.recv)>(sym("ncclRecv"));
        api.group_start = reinterpret_cast<decltype(api.group_start)>(sym("ncclGroupStart"));
        api.group_end = reinterpret_cast<decltype(api.group_end)>(sym("ncclGroupEnd"));
        api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(sym("ncclAllReduce"));
        api.error_string = reinterpret_cast<decltype(api.error_string)>(sym("ncclGetErrorString"));
        api.loaded = api.get_unique_id && api.comm_init_rank && api.comm_destroy && api.send && api.recv &&
                     api.group_start && api.group_end && api.all_reduce && api.error_string;
        if (!api.loaded) api.why = "libnccl.so.2 lacks a needed symbol";
    });
    return api;
}

int nccl_fail(ymflow_ctx* c, ncclResult_t r, const char* what) {
    return fail(c, YMFLOW_ERR_CUDA, std::string(what) + ": " + nccl().error_string(r));
}

#define YM_NCCL(ctx, call, what)                                        \
    do {                                                                \
        ncclResult_t r_ = (call);                                       \
        if (r_ != ncclSuccess) return nccl_fail(ctx, r_, what);         \
    } while (0)

// --- geometry of the halo runs ------------------------------------------------
size_t slice_bytes(const ymflow_ctx* c) { return size_t(c->geo.site0) * link_bytes(c->prec); }

// Byte offset of local time slice t of direction mu in a link buffer.
size_t slice_offset(const ymflow_ctx* c, int mu, int t) {
    const int64_t groups = padded_sites(c->geo.V) / 32;
    const int64_t slice_groups = c->geo.site0 / 32;
    return size_t(mu * groups + int64_t(t) * slice_groups) * 32 * link_bytes(c->prec);
}

char* slice_ptr(const ymflow_ctx* c, int buf, int mu, int t) {
    return static_cast<char*>(c->u[buf]) + slice_offset(c, mu, t);
}

}  // namespace

int slab_exchange(ymflow_ctx* c, int buf) {
    if (!c->slab || !c->comm) return YMFLOW_OK;
    const NcclApi& n = nccl();
    ncclComm_t comm = static_cast<ncclComm_t>(c->comm);
    const size_t bytes = slice_bytes(c);
    // Posting order fixes the matching between a pair of ranks (NCCL matches
    // the sends and receives of one pair in order): first every rank's lowest
    // interior slice goes down into its lower neighbour's upper halo, then its
    // highest interior slice goes up into its upper neighbour's lower halo.
    YM_NCCL(c, n.group_start(), "ncclGroupStart");
    for (int mu = 0; mu < 4; mu++) {
        YM_NCCL(c, n.send(slice_ptr(c, buf, mu, 1), bytes, ncclChar, c->lower, comm, c->stream), "ncclSend");
        YM_NCCL(c, n.recv(slice_ptr(c, buf, mu, c->nt + 1), bytes, ncclChar, c->upper, comm, c->stream), "ncclRecv");
    }
    for (int mu = 0; mu < 4; mu++) {
        YM_NCCL(c, n.send(slice_ptr(c, buf, mu, c->nt), bytes, ncclChar, c->upper, comm, c->stream), "ncclSend");
        YM_NCCL(c, n.recv(slice_ptr(c, buf, mu, 0), bytes, ncclChar, c->lower, comm, c->stream), "ncclRecv");
    }
    YM_NCCL(c, n.group_end(), "ncclGroupEnd");
    return YMFLOW_OK;
}

int slab_reduce_row(ymflow_ctx* c, double* row) {
    // plaq (already divided by 18 x the configuration's volume), topc, raw
    // energy and the non-finite flag are sums over sites: add them over ranks
    YM_NCCL(c, nccl().all_reduce(row, row, 4, ncclDouble, ncclSum, static_cast<ncclComm_t>(c->comm), c->stream),
            "ncclAllReduce");
    return YMFLOW_OK;
}

void slab_release(ymflow_ctx* c) {
    if (c->comm) nccl().comm_destroy(static_cast<ncclComm_t>(c->comm));
    c->comm = nullptr;
}

namespace {

// --- in-process group --------------------------------------------------------
struct GroupEvents {
    std::vector<cudaEvent_t> ev;
    ~GroupEvents() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

// Every slab's halos of buffer u[buf] from its neighbours' interior boundary
// slices: record each slab's stream, make each stream wait for its two
// neighbours, then copy on the receiving slab's stream.
int group_exchange(ymflow_ctx* const* cs, int n, const int* buf, std::vector<cudaEvent_t>& ev) {
    for (int i = 0; i < n; i++) {
        DeviceGuard g(cs[i]->device);
        YM_CK(cs[i], cudaEventRecord(ev[i], cs[i]->stream), "event record");
    }
    for (int i = 0; i < n; i++) {
        ymflow_ctx* c = cs[i];
        const ymflow_ctx* lo = cs[(i + n - 1) % n];
        const ymflow_ctx* hi = cs[(i + 1) % n];
        const int blo = buf[(i + n - 1) % n], bhi = buf[(i + 1) % n];
        DeviceGuard g(c->device);
        YM_CK(c, cudaStreamWaitEvent(c->stream, ev[(i + n - 1) % n], 0), "wait lower slab");
        YM_CK(c, cudaStreamWaitEvent(c->stream, ev[(i + 1) % n], 0), "wait upper slab");
        const size_t bytes = slice_bytes(c);
        for (int mu = 0; mu < 4; mu++) {
            YM_CK(c, cudaMemcpyPeerAsync(slice_ptr(c, buf[i], mu, 0), c->device, slice_ptr(lo, blo, mu, lo->nt),
                                         lo->device, bytes, c->stream),
                  "lower halo copy");
            YM_CK(c, cudaMemcpyPeerAsync(slice_ptr(c, buf[i], mu, c->nt + 1), c->device, slice_ptr(hi, bhi, mu, 1),
                                         hi->device, bytes, c->stream),
                  "upper halo copy");
        }
    }
    return YMFLOW_OK;
}

// After every slab's fused stage: each slab's next work waits for both
// neighbours' stages, which wrote its halos.
int group_order(ymflow_ctx* const* cs, int n, std::vector<cudaEvent_t>& ev) {
    for (int i = 0; i < n; i++) {
        DeviceGuard g(cs[i]->device);
        YM_CK(cs[i], cudaEventRecord(ev[i], cs[i]->stream), "event record");
    }
    for (int i = 0; i < n; i++) {
        DeviceGuard g(cs[i]->device);
        YM_CK(cs[i], cudaStreamWaitEvent(cs[i]->stream, ev[(i + n - 1) % n], 0), "wait lower slab");
        YM_CK(cs[i], cudaStreamWaitEvent(cs[i]->stream, ev[(i + 1) % n], 0), "wait upper slab");
    }
    return YMFLOW_OK;
}

// Whether kernels on `from` can store into `to`'s memory (enabling peer access once).
bool peer_reachable(int from, int to) {
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

}  // namespace
}  // namespace ym

using namespace ym;

extern "C" {

int ymflow_nccl_unique_id(void* id) {
    if (!id) return YMFLOW_ERR_ARG;
    const NcclApi& n = nccl();
    if (!n.loaded) return YMFLOW_ERR_NODEVICE;
    ncclUniqueId u;
    if (n.get_unique_id(&u) != ncclSuccess) return YMFLOW_ERR_CUDA;
    static_assert(sizeof(ncclUniqueId) == YMFLOW_NCCL_ID_BYTES, "NCCL unique id size");
    std::memcpy(id, &u, sizeof(u));
    return YMFLOW_OK;
}

int ymflow_slab_connect(ymflow_ctx* c, const void* id, int rank, int nranks, int lower_rank, int upper_rank) {
    if (!c || !id) return YMFLOW_ERR_ARG;
    if (!c->slab) return fail(c, YMFLOW_ERR_STATE, "not a slab context (ymflow_create_slab)");
    if (c->comm) return fail(c, YMFLOW_ERR_STATE, "slab already connected");
    if (nranks < 1 || rank < 0 || rank >= nranks || lower_rank < 0 || lower_rank >= nranks || upper_rank < 0 ||
        upper_rank >= nranks)
        return fail(c, YMFLOW_ERR_ARG, "ranks outside [0, nranks)");
    const NcclApi& n = nccl();
    if (!n.loaded) return fail(c, YMFLOW_ERR_NODEVICE, n.why);
    DeviceGuard guard(c->device);
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    ncclComm_t comm = nullptr;
    YM_NCCL(c, n.comm_init_rank(&comm, nranks, u, rank), "ncclCommInitRank");
    c->comm = comm;
    c->rank = rank;
    c->nranks = nranks;
    c->lower = lower_rank;
    c->upper = upper_rank;
    return YMFLOW_OK;
}

int ymflow_slab_group_flow(ymflow_ctx* const* ctxs, int n, double eps, int nsteps, int measure_every,
                           int reunit_every, ymflow_obs* out, int out_cap, int* n_out) {
    NvtxRange range("ymflow_slab_group_flow");
    if (n_out) *n_out = 0;
    if (!ctxs || n < 1) return YMFLOW_ERR_ARG;
    for (int i = 0; i < n; i++)
        if (!ctxs[i]) return YMFLOW_ERR_ARG;
    ymflow_ctx* c0 = ctxs[0];
    if (nsteps < 0 || !std::isfinite(eps)) return fail(c0, YMFLOW_ERR_ARG, "nsteps < 0 or eps not finite");
    int t = 0;
    for (int i = 0; i < n; i++) {
        const ymflow_ctx* c = ctxs[i];
        if (!c->slab || c->comm) return fail(c0, YMFLOW_ERR_ARG, "every context must be an unconnected slab");
        if (c->stage_form != c0->stage_form) return fail(c0, YMFLOW_ERR_ARG, "slabs with different stage forms");
        if (c->prec != c0->prec || std::memcmp(c->gdims, c0->gdims, sizeof(c->gdims)) != 0)
            return fail(c0, YMFLOW_ERR_ARG, "slabs of different configurations or precisions");
        if (c->t0 != t) return fail(c0, YMFLOW_ERR_ARG, "slabs must tile the time extent in order");
        if (!c->loaded) return fail(c0, YMFLOW_ERR_STATE, "slab " + std::to_string(i) + " has no links");
        t += c->nt;
    }
    if (t != c0->gdims[3]) return fail(c0, YMFLOW_ERR_ARG, "slabs do not cover the time extent");
    int rows = 1;
    for (int s = 1; s <= nsteps; s++)
        if ((measure_every > 0 && s % measure_every == 0) || s == nsteps) rows++;
    if (out && out_cap < rows)
        return fail(c0, YMFLOW_ERR_CAPACITY,
                    "output holds " + std::to_string(out_cap) + " rows, flow needs " + std::to_string(rows));
    GroupEvents evs;
    evs.ev.assign(size_t(n), nullptr);
    for (int i = 0; i < n; i++) {
        DeviceGuard g(ctxs[i]->device);
        int r = ensure_meas(ctxs[i], rows);
        if (r != YMFLOW_OK) return r;
        YM_CK(ctxs[i], cudaEventCreateWithFlags(&evs.ev[i], cudaEventDisableTiming), "event create");
    }
    const bool reunit = c0->prec != YMFLOW_FP64 && reunit_every > 0;
    // the fused exchange needs every slab's GPU to reach its neighbours' memory
    bool fused = std::getenv("YMFLOW_SLAB_COPY_EXCHANGE") == nullptr;
    for (int i = 0; i < n && fused; i++)
        for (int j : {(i + n - 1) % n, (i + 1) % n})
            if (fused && !peer_reachable(ctxs[i]->device, ctxs[j]->device)) fused = false;
    std::vector<int> buf(static_cast<size_t>(n));
    auto exchange_current = [&]() {
        for (int i = 0; i < n; i++) buf[i] = ctxs[i]->cur;
        return group_exchange(ctxs, n, buf.data(), evs.ev);
    };
    auto measure = [&](int row) {
        for (int i = 0; i < n; i++) {
            DeviceGuard g(ctxs[i]->device);
            const int r = enqueue_measure(ctxs[i], row);
            if (r != YMFLOW_OK) return r;
        }
        return int(YMFLOW_OK);
    };
    for (int i = 0; i < n; i++)
        if (reunit) {
            DeviceGuard g(ctxs[i]->device);
            YM_CK(ctxs[i], cudaMemsetAsync(ctxs[i]->deviation, 0, sizeof(unsigned long long), ctxs[i]->stream),
                  "reset drift");
        }
    std::vector<int64_t> row_step(rows);
    std::vector<double> row_t(rows);
    int r = exchange_current();
    if (r == YMFLOW_OK) r = measure(0);
    if (r != YMFLOW_OK) return r;
    row_step[0] = c0->step;
    row_t[0] = c0->t;
    int row = 1;
    for (int s = 1; s <= nsteps; s++) {
        for (int stage = 0; stage < 3; stage++) {
            if (fused) {
                // each slab's stage stores its boundary links into its neighbours' halos itself
                for (int i = 0; i < n; i++) {
                    ymflow_ctx* c = ctxs[i];
                    ymflow_ctx* lo = ctxs[(i + n - 1) % n];
                    ymflow_ctx* hi = ctxs[(i + 1) % n];
                    DeviceGuard g(c->device);
                    if (c->stage_form == 1) {
                        YM_CK(c, launch_plaq_field(c->prec, c->u[c->cur], c->hfield, plaq_range(c->geo, true),
                                                   c->stream),
                              "plaquette-field launch");
                        YM_CK(c, launch_rk_split_stage_halo(c->prec, stage, c->u[c->cur], c->u[1 - c->cur], c->z,
                                                            c->hfield, c->geo, eps, lo->u[1 - lo->cur], lo->geo.V,
                                                            lo->nt + 1, hi->u[1 - hi->cur], hi->geo.V, c->stream),
                              "stage launch");
                    } else {
                        YM_CK(c, launch_rk_stage_halo(c->prec, stage, c->u[c->cur], c->u[1 - c->cur], c->z, c->geo,
                                                      eps, lo->u[1 - lo->cur], lo->geo.V, lo->nt + 1,
                                                      hi->u[1 - hi->cur], hi->geo.V, c->stream),
                              "stage launch");
                    }
                }
                for (int i = 0; i < n; i++) ctxs[i]->cur = 1 - ctxs[i]->cur;
                if ((r = group_order(ctxs, n, evs.ev)) != YMFLOW_OK) return r;
            } else {
                for (int i = 0; i < n; i++) {
                    ymflow_ctx* c = ctxs[i];
                    DeviceGuard g(c->device);
                    if (c->stage_form == 1) {
                        YM_CK(c, launch_plaq_field(c->prec, c->u[c->cur], c->hfield, plaq_range(c->geo, true),
                                                   c->stream),
                              "plaquette-field launch");
                        YM_CK(c, launch_rk_split_stage(c->prec, stage, c->u[c->cur], c->u[1 - c->cur], c->z,
                                                       c->hfield, c->geo, eps, c->stream),
                              "stage launch");
                    } else {
                        YM_CK(c, launch_rk_stage(c->prec, stage, c->u[c->cur], c->u[1 - c->cur], c->z, c->geo, eps,
                                                 c->block, c->stream),
                              "stage launch");
                    }
                    c->cur = 1 - c->cur;
                    // before the step's last exchange, whose copies then carry
                    // the reunitarised links (after it, the reunitarisation
                    // would rewrite links a neighbour's copy may still read)
                    if (stage == 2 && reunit && s % reunit_every == 0)
                        YM_CK(c, launch_reunitarize(c->prec, c->u[c->cur], c->geo, c->deviation, c->stream),
                              "reunitarise");
                }
                if ((r = exchange_current()) != YMFLOW_OK) return r;
            }
        }
        for (int i = 0; i < n; i++) {
            ymflow_ctx* c = ctxs[i];
            // three stages flipped the buffer three times; the step's result is the third stage's
            c->step++;
            c->t += eps;
            if (fused && reunit && s % reunit_every == 0) {
                // every local site, halos included (the neighbours' stages stored
                // them before group_order): the same links as their owners'
                DeviceGuard g(c->device);
                YM_CK(c, launch_reunitarize(c->prec, c->u[c->cur], c->geo, c->deviation, c->stream), "reunitarise");
            }
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
        YM_CK(c, cudaStreamSynchronize(c->stream), "group flow");
        for (int k = 0; k < rows * 4; k++) sum[k] += c->meas_host[k];
        double d;
        std::memcpy(&d, &bits, sizeof(d));
        drift = std::fmax(drift, d);
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
