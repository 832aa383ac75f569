// Device memory owned by a solver handle: stream-ordered allocations, released together.
#pragma once

#include <vector>

#include "common.cuh"

namespace zvfv {

class Arena {
   public:
    explicit Arena(cudaStream_t s = 0) : st_(s) {}
    ~Arena() { release(); }
    Arena(const Arena &) = delete;
    Arena &operator=(const Arena &) = delete;

    void set_stream(cudaStream_t s) { st_ = s; }

    template <typename T>
    int get(T **p, size_t n) {
        void *q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, (n ? n : 1) * sizeof(T), st_);
        if (e != cudaSuccess) {
            *p = nullptr;
            return cuda_status(e, "device allocation");
        }
        blocks_.push_back(q);
        *p = static_cast<T *>(q);
        return OK;
    }

    void release() {
        for (void *q : blocks_) cudaFreeAsync(q, st_);
        blocks_.clear();
    }

   private:
    cudaStream_t st_;
    std::vector<void *> blocks_;
};

}  // namespace zvfv
