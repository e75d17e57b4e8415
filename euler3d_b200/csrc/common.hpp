// Shared host-side helpers of the euler3d_b200 library: error reporting across the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>

#include "euler3d_b200.h"

namespace e3d {

// An error that carries the C-ABI status to return.
struct Error : std::runtime_error {
    e3d_status status;
    Error(e3d_status s, const std::string &msg) : std::runtime_error(msg), status(s) {}
};

void set_last_error(const std::string &msg);

inline void cuda_check(cudaError_t err, const char *what) {
    if (err == cudaSuccess) return;
    if (err == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        throw Error(E3D_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(err));
    }
    throw Error(E3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

#define E3D_CUDA(call) ::e3d::cuda_check((call), #call)

// Raise a kernel's dynamic shared-memory limit on the current device to at least `bytes`.  Never
// lowers it: solvers of different meshes, driven from several host threads, share the kernels.
inline void raise_smem_limit(const void *func, size_t bytes) {
    static std::mutex m;
    static std::map<std::pair<const void *, int>, size_t> limit;
    int dev = 0;
    E3D_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> g(m);
    size_t &cur = limit[{func, dev}];
    if (bytes <= cur) return;
    E3D_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    cur = bytes;
}

// Runs fn and converts exceptions into an e3d_status plus the thread's last-error message.
template <typename F>
e3d_status guarded(F &&fn) {
    try {
        fn();
        return E3D_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return E3D_ERR_OOM;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return E3D_ERR_MESH;
    } catch (...) {
        set_last_error("unknown error");
        return E3D_ERR_CUDA;
    }
}

}  // namespace e3d
