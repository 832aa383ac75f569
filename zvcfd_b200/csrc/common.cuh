// Shared helpers of the zvfv B200 library: status codes, the last-error string, launch checks.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "topology_tables.h"

namespace zvfv {

// Status codes returned by every C-ABI entry point (0 = success).
enum Status : int {
    OK = 0,
    BAD_ARGUMENT = 1,
    CUDA_FAILURE = 2,
    OUT_OF_MEMORY = 3,
    NOT_CONVERGED = 4,
    TIMED_OUT = 5,
    NON_FINITE = 6,
    UNSUPPORTED = 7,
};

void set_error(const char *fmt, ...);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// The status of the launches just made; records the CUDA error text on failure.
inline int launch_status(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? OUT_OF_MEMORY : CUDA_FAILURE;
}

inline int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? OUT_OF_MEMORY : CUDA_FAILURE;
}

#define ZV_TRY(...)                          \
    do {                                     \
        int _rc = (__VA_ARGS__);             \
        if (_rc != ::zvfv::OK) return _rc;   \
    } while (0)

inline unsigned grid_for(long long work, int per_block) {
    long long g = (work + per_block - 1) / per_block;
    return (unsigned)(g > 0 ? g : 1);
}

// Every kernel launch of the library counts itself here (zvfv_launch_count reads the total).
void count_launch();
// A replayed CUDA graph counts its kernels (recorded while it was captured, when nothing ran).
void count_launches(long long k);
long long launches_so_far();

// Number of SMs of the current device (cached per process; one device per process).
int sm_count();

}  // namespace zvfv
