// Shared host-side helpers of the euler3d_b200 library: error reporting across the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

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
