// Host helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <string>

#include "ymflow.h"

namespace ym {

// An NVTX range over an ABI call, named after it, so that profiler timelines
// show the library's work (header-only NVTX v3; free when no tool listens).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Makes `d` current for the scope of a call and restores the caller's device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

inline int status_of(cudaError_t e) { return e == cudaErrorMemoryAllocation ? YMFLOW_ERR_OOM : YMFLOW_ERR_CUDA; }

inline std::string cuda_message(cudaError_t e, const char* what) {
    return std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
}

// true when `device` exists and is an sm_100 part; otherwise *why says why
inline bool device_usable(int device, std::string* why) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        *why = "no CUDA device with that index";
        return false;
    }
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
    if (major != 10 || minor != 0) {
        *why = "libymflow is built for sm_100a (B200); device has sm_" + std::to_string(major) + std::to_string(minor);
        return false;
    }
    return true;
}

}  // namespace ym
