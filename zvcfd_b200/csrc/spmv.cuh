// Block-CSR SpMV of 4x4 blocks, y = A x or r = b - A x, in FP64 or FP32.
//
// Layout (the reference's BlockMatrix, zvcfd/fv/linear.py:75-135): indptr int64 (N+1),
// sorted int32 column indices, blocks of 16 values row-major, x and y (N, 4).
//
// A group of G lanes works on one block row; its lanes form G/4 "slots" of 4 lanes, each
// slot one block per step: lane r of the slot loads row r of the block (32 B in FP64 as two
// 128-bit loads, 16 B in FP32 as one) and the column's 4-vector of x, and accumulates the
// dot product for output component r. A step of the group therefore reads G/4 consecutive
// blocks, one contiguous span; the slots' partial sums meet in an xor-shuffle reduction.
// Blocks and indices are streamed with evict-first loads so that x stays resident in L2.
#pragma once

#include "common.cuh"

namespace zvfv {

template <typename V>
struct Vec4;
template <>
struct Vec4<double> {
    double v[4];
    __device__ static Vec4 load_stream(const double *p) {
        Vec4 r;
        const double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
        const double2 b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y;
        return r;
    }
    __device__ static Vec4 load(const double *p) {
        Vec4 r;
        const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
        const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = b.x; r.v[3] = b.y;
        return r;
    }
};
template <>
struct Vec4<float> {
    float v[4];
    __device__ static Vec4 load_stream(const float *p) {
        Vec4 r;
        const float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
        return r;
    }
    __device__ static Vec4 load(const float *p) {
        Vec4 r;
        const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
        r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
        return r;
    }
};

// RESID: y = b - A x instead of A x
template <int G, bool RESID, typename V, typename XT>
__global__ void __launch_bounds__(256)
k_bsr_spmv(long long n, const long long *__restrict__ indptr, const int *__restrict__ indices,
           const V *__restrict__ data, const XT *__restrict__ x, const XT *__restrict__ bvec,
           XT *__restrict__ y) {
    static_assert(G == 4 || G == 8 || G == 16 || G == 32, "lanes per row");
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    XT acc = 0;
    if (row < n) {
        const long long p1 = indptr[row + 1];
        long long p = indptr[row] + slot;
        for (; p + S < p1; p += 2 * S) {           // two blocks per slot in flight
            const int j0 = __ldcs(indices + p), j1 = __ldcs(indices + p + S);
            const Vec4<V> a0 = Vec4<V>::load_stream(data + p * 16 + r * 4);
            const Vec4<V> a1 = Vec4<V>::load_stream(data + (p + S) * 16 + r * 4);
            const Vec4<XT> x0 = Vec4<XT>::load(x + (long long)j0 * 4);
            const Vec4<XT> x1 = Vec4<XT>::load(x + (long long)j1 * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (XT)a0.v[c] * x0.v[c];
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (XT)a1.v[c] * x1.v[c];
        }
        if (p < p1) {
            const int j0 = __ldcs(indices + p);
            const Vec4<V> a0 = Vec4<V>::load_stream(data + p * 16 + r * 4);
            const Vec4<XT> x0 = Vec4<XT>::load(x + (long long)j0 * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (XT)a0.v[c] * x0.v[c];
        }
    }
#pragma unroll
    for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    if (row < n && slot == 0) y[row * 4 + r] = RESID ? bvec[row * 4 + r] - acc : acc;
}

template <bool RESID, typename V, typename XT>
inline int bsr_spmv_launch(int lanes, long long n, const long long *indptr, const int *indices,
                           const V *data, const XT *x, const XT *b, XT *y, cudaStream_t st) {
    if (n <= 0) return OK;
    switch (lanes) {
        case 4:
            k_bsr_spmv<4, RESID, V, XT><<<grid_for(n * 4, 256), 256, 0, st>>>(n, indptr, indices, data, x, b, y); count_launch();
            break;
        case 8:
            k_bsr_spmv<8, RESID, V, XT><<<grid_for(n * 8, 256), 256, 0, st>>>(n, indptr, indices, data, x, b, y); count_launch();
            break;
        case 16:
            k_bsr_spmv<16, RESID, V, XT><<<grid_for(n * 16, 256), 256, 0, st>>>(n, indptr, indices, data, x, b, y); count_launch();
            break;
        case 32:
            k_bsr_spmv<32, RESID, V, XT><<<grid_for(n * 32, 256), 256, 0, st>>>(n, indptr, indices, data, x, b, y); count_launch();
            break;
        default:
            set_error("bsr_spmv: lanes per row %d (4, 8, 16 or 32)", lanes);
            return BAD_ARGUMENT;
    }
    return launch_status("bsr_spmv");
}

// y = A^T x (RESID: b - A^T x) through the transpose's structure: for block row j of A^T,
// tptr[j]..tptr[j+1] list the blocks p = tperm[q] of column j of A with their rows trow[q]
// (rows ascending). Lane r of a slot forms column r of the block: the four lanes of a slot
// still read the block's 128 contiguous bytes, in four 32-byte rounds.
template <int G, bool RESID, typename V, typename XT>
__global__ void __launch_bounds__(256)
k_bsr_spmv_t(long long n, const long long *__restrict__ tptr, const int *__restrict__ trow,
             const long long *__restrict__ tperm, const V *__restrict__ data,
             const XT *__restrict__ x, const XT *__restrict__ bvec, XT *__restrict__ y) {
    constexpr int S = G / 4;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = gid / G;
    const int lane = threadIdx.x % G;
    const int slot = lane / 4, r = lane % 4;
    XT acc = 0;
    if (row < n) {
        const long long q1 = tptr[row + 1];
        for (long long q = tptr[row] + slot; q < q1; q += S) {
            const int i = trow[q];
            const V *blk = data + tperm[q] * 16;
            const Vec4<XT> xv = Vec4<XT>::load(x + (long long)i * 4);
#pragma unroll
            for (int c = 0; c < 4; ++c) acc += (XT)__ldg(blk + c * 4 + r) * xv.v[c];
        }
    }
#pragma unroll
    for (int off = 4; off < G; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off, G);
    if (row < n && slot == 0) y[row * 4 + r] = RESID ? bvec[row * 4 + r] - acc : acc;
}

template <bool RESID, typename V, typename XT>
inline int bsr_spmv_t_launch(int lanes, long long n, const long long *tptr, const int *trow,
                             const long long *tperm, const V *data, const XT *x, const XT *b,
                             XT *y, cudaStream_t st) {
    if (n <= 0) return OK;
    switch (lanes) {
        case 8:
            k_bsr_spmv_t<8, RESID, V, XT><<<grid_for(n * 8, 256), 256, 0, st>>>(n, tptr, trow, tperm, data, x, b, y); count_launch();
            break;
        case 16:
            k_bsr_spmv_t<16, RESID, V, XT><<<grid_for(n * 16, 256), 256, 0, st>>>(n, tptr, trow, tperm, data, x, b, y); count_launch();
            break;
        case 32:
            k_bsr_spmv_t<32, RESID, V, XT><<<grid_for(n * 32, 256), 256, 0, st>>>(n, tptr, trow, tperm, data, x, b, y); count_launch();
            break;
        default:
            set_error("bsr_spmv_t: lanes per row %d (8, 16 or 32)", lanes);
            return BAD_ARGUMENT;
    }
    return launch_status("bsr_spmv_t");
}

}  // namespace zvfv
