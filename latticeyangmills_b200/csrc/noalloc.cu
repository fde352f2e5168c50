// ymflow_observables_noalloc: plaquette, clover energy and clover charge of a
// configuration that the caller already holds in device memory, computed
// without allocating anything.
//
// Who needs this: callers that cannot call cudaMalloc at the point where they
// want the observables.  A host application that reserved the whole device
// for its own memory pool at start-up has no free memory left for a library
// allocation, and a caller measuring inside a latency-critical loop cannot
// afford the implicit device synchronisation that cudaMalloc and cudaFree may
// perform.  Such callers keep their links in device memory and pass them in.
//
// Scratch: the per-block partial sums live in the file-scope device array
// below, sized for kNoAllocMaxBlocks blocks of 128 sites, so the largest
// lattice accepted is YMFLOW_NOALLOC_MAX_SITES sites (8,388,608, e.g. 48^4 or
// 32^3 x 256).  The array is part of the loaded library: every GPU that loads
// it holds these 1.5 MB until the process exits.  Host code cannot pass the
// array's name to a kernel (in host code it names a host-side stand-in), so
// on the first call on each device, with that device current, the device
// address is fetched once with cudaGetSymbolAddress and cached.  Make that
// first call before any stream capture.  The cache lives as long as the
// process's CUDA context: after a cudaDeviceReset the library must be
// reloaded before this entry point is used again.
//
// The links are read as 16-byte vectors and the results written as doubles,
// so the links must start on a 16-byte boundary and the output on an 8-byte
// one; a caller passing an offset into its own pool (one link is 144 bytes,
// a site 576) gets YMFLOW_ERR_ARG for an unaligned pointer before anything is
// launched, instead of a misaligned-address fault that would end its context.
//
// Every call shares the array.  Each block writes (never accumulates) its own
// partial and the fold reads only the partials written by the same call, so
// nothing has to be cleared between calls; the array keeps the last call's
// partials afterwards.  Calls whose kernels overlap on the GPU (different
// streams, or different host threads, on one device) race on the array and
// must be ordered by the caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "kernels.h"
#include "observables.cuh"
#include "ymflow.h"

namespace ym {

constexpr int kNoAllocBlock = 128;
constexpr int kNoAllocMaxBlocks = YMFLOW_NOALLOC_MAX_SITES / kNoAllocBlock;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[3 * kNoAllocMaxBlocks];

// Links in the reference's .bin layout, read in place from device memory:
// site-major, then mu, then 18 doubles (row-major 3x3, re/im interleaved).
struct AosField {
    using Real = double;
    const double* p;
    int V;
    __device__ __forceinline__ const double2* link(int mu, int s) const {
        return reinterpret_cast<const double2*>(p + (int64_t(s) * 4 + mu) * 18);
    }
    __device__ __forceinline__ M3<double> load(int mu, int s) const {
        const double2* b = link(mu, s);
        M3<double> a;
#pragma unroll
        for (int e = 0; e < 9; e++) {
            const double2 v = __ldg(b + e);
            set_elem(a, e, v.x, v.y);
        }
        return a;
    }
    __device__ __forceinline__ Rows2<double> load_rows2(int mu, int s) const {
        const double2* b = link(mu, s);
        Rows2<double> a;
#pragma unroll
        for (int e = 0; e < 6; e++) {
            const double2 v = __ldg(b + e);
            a.e[e / 3][e % 3] = cx(v.x, v.y);
        }
        return a;
    }
};

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device (set up once per device).
cudaError_t noalloc_scratch(int device, double** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[device] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

}  // namespace ym

using namespace ym;

extern "C" int ymflow_observables_noalloc(const double* links_aos_device, const int dims[4], double* out_device,
                                          void* stream) {
    if (!links_aos_device || !dims || !out_device) return YMFLOW_ERR_ARG;
    int64_t v = 1;
    for (int i = 0; i < 4; i++) {
        if (dims[i] < 1) return YMFLOW_ERR_ARG;
        v *= dims[i];
        if (v > YMFLOW_NOALLOC_MAX_SITES) return YMFLOW_ERR_CAPACITY;
    }
    if (reinterpret_cast<uintptr_t>(links_aos_device) % 16 != 0 || reinterpret_cast<uintptr_t>(out_device) % 8 != 0)
        return YMFLOW_ERR_ARG;
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kNoAllocMaxDevices) {
        cudaGetLastError();
        return YMFLOW_ERR_NODEVICE;
    }
    double* partials = nullptr;
    if (noalloc_scratch(device, &partials) != cudaSuccess) {
        cudaGetLastError();
        return YMFLOW_ERR_CUDA;
    }
    const Geo g = make_geo(dims);
    const int nb = int((g.V + kNoAllocBlock - 1) / kNoAllocBlock);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    observables_site_kernel<<<nb, kNoAllocBlock, 0, st>>>(AosField{links_aos_device, g.V}, g, partials);
    if (cudaGetLastError() != cudaSuccess) return YMFLOW_ERR_CUDA;
    if (launch_obs_finalize(partials, nb, g, out_device, st) != cudaSuccess) return YMFLOW_ERR_CUDA;
    return YMFLOW_OK;
}
