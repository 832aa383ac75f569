// Once-per-mesh device setup: the block pattern, the element colouring and slot order, and
// small permutation helpers. Temporary memory comes from the stream-ordered allocator
// (cudaMallocAsync) and is returned before each entry point returns.
#include <cub/cub.cuh>

#include "common.cuh"

namespace zvfv {
namespace {

template <typename T>
struct DevBuf {
    T *p = nullptr;
    cudaStream_t st = 0;
    int alloc(size_t n, cudaStream_t s) {
        st = s;
        return cuda_status(cudaMallocAsync((void **)&p, (n ? n : 1) * sizeof(T), s), "alloc");
    }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, st);
    }
};

// ------------------------------------------------------------------------ block pattern

// key = row * N + col of every (row node, column node) pair of every element
__global__ void k_pair_keys(const int *__restrict__ conn, long long E, int n, long long N,
                            unsigned long long *__restrict__ keys) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nn = (long long)n * n;
    if (i >= E * nn) return;
    const long long e = i / nn;
    const int t = (int)(i % nn), a = t / n, c = t % n;
    keys[i] = (unsigned long long)conn[e * n + a] * (unsigned long long)N +
              (unsigned long long)conn[e * n + c];
}

// indptr[i] = first unique key of row i (lower bound of i * N), indptr[N] = nnzb
__global__ void k_row_starts(const unsigned long long *__restrict__ keys, long long nnz,
                             long long N, long long *__restrict__ indptr) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > N) return;
    if (i == N) { indptr[N] = nnz; return; }
    const unsigned long long target = (unsigned long long)i * (unsigned long long)N;
    long long lo = 0, hi = nnz;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < target) lo = mid + 1; else hi = mid;
    }
    indptr[i] = lo;
}

__global__ void k_cols(const unsigned long long *__restrict__ keys, long long nnz, long long N,
                       int *__restrict__ indices) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nnz) indices[i] = (int)(keys[i] % (unsigned long long)N);
}

int bits_for(unsigned long long v) {
    int b = 1;
    while (b < 64 && (v >> b)) ++b;
    return b;
}

// ------------------------------------------------------------------------ colouring

// A hash of the element index in the high 32 bits, the index in the low 32
// (zvcfd/fv/fast.py:84-92): distinct keys in a pseudo-random order. The hash is the
// SplitMix64 output function (Steele, Lea and Flood, OOPSLA 2014; these are its published
// constants), which the colouring must share with the reference to come out the same.
__global__ void k_colour_keys(long long E, unsigned long long *__restrict__ key) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    unsigned long long z = (unsigned long long)e + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    key[e] = (z & 0xFFFFFFFF00000000ull) | (unsigned long long)e;
}

// Round, part 1: each node keeps the smallest key of its uncoloured elements.
__global__ void k_colour_claim(const int *__restrict__ conn, int n, long long E,
                               const unsigned long long *__restrict__ key,
                               const int *__restrict__ colour, unsigned long long *__restrict__ best) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || colour[e] >= 0) return;
    const unsigned long long k = key[e];
    for (int a = 0; a < n; ++a) atomicMin(&best[conn[e * n + a]], k);
}

// Round, part 2: an element holding the smallest key at all of its nodes takes the lowest
// colour that none of its nodes has used. Winners share no node, so their reads and writes
// of the node masks never meet; the result is independent of thread order.
// ctr[0]: elements left uncoloured; ctr[1]: winners that found no free colour in W words.
__global__ void k_colour_pick(const int *__restrict__ conn, int n, long long E,
                              const unsigned long long *__restrict__ key, int *__restrict__ colour,
                              const unsigned long long *__restrict__ best,
                              unsigned long long *__restrict__ used, int W,
                              unsigned long long *__restrict__ ctr) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E || colour[e] >= 0) return;
    const unsigned long long k = key[e];
    for (int a = 0; a < n; ++a)
        if (best[conn[e * n + a]] != k) {
            atomicAdd(&ctr[0], 1ull);
            return;
        }
    int c = -1;
    for (int w = 0; w < W && c < 0; ++w) {
        unsigned long long m = 0ull;
        for (int a = 0; a < n; ++a) m |= used[(long long)conn[e * n + a] * W + w];
        const unsigned long long free_bits = ~m;
        if (free_bits) c = w * 64 + (__ffsll((long long)free_bits) - 1);
    }
    if (c < 0) {
        atomicAdd(&ctr[1], 1ull);
        return;
    }
    colour[e] = c;
    const unsigned long long bit = 1ull << (c % 64);
    for (int a = 0; a < n; ++a) used[(long long)conn[e * n + a] * W + c / 64] |= bit;
}

__global__ void k_fill_u64(unsigned long long *p, long long n, unsigned long long v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_fill_i32(int *p, long long n, int v) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_iota(int *p, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (int)i;
}

// offsets[c] = first position of colour c in the sorted colours, offsets[C] = E
__global__ void k_colour_offsets(const int *__restrict__ sorted, long long E, int C,
                                 long long *__restrict__ offsets) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > C) return;
    long long lo = 0, hi = E;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (sorted[mid] < c) lo = mid + 1; else hi = mid;
    }
    offsets[c] = lo;
}

__global__ void k_widen(const int *__restrict__ src, long long n, long long *__restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

__global__ void k_gather_rows(const unsigned char *__restrict__ src, const long long *__restrict__ idx,
                              long long rows, long long width, unsigned char *__restrict__ dst,
                              int scatter) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * width) return;
    const long long r = i / width, b = i % width;
    if (scatter) dst[idx[r] * width + b] = src[r * width + b];
    else dst[r * width + b] = src[idx[r] * width + b];
}

__global__ void k_row_of_block(long long n, const long long *__restrict__ indptr,
                               long long *__restrict__ row) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (long long p = indptr[i]; p < indptr[i + 1]; ++p) row[p] = i;
}

__global__ void k_transpose_fill(long long nnz, const long long *__restrict__ perm,
                                 const long long *__restrict__ row, int *__restrict__ trow) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nnz) trow[q] = (int)row[perm[q]];
}

__global__ void k_col_starts(const int *__restrict__ sorted, long long nnz, long long n,
                             long long *__restrict__ tptr) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j > n) return;
    long long lo = 0, hi = nnz;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (sorted[mid] < j) lo = mid + 1; else hi = mid;
    }
    tptr[j] = lo;
}

__global__ void k_iota64s(long long *p, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = i;
}

}  // namespace

struct Pattern {
    long long n_nodes = 0, nnz = 0;
    unsigned long long *keys = nullptr;
};

}  // namespace zvfv

using namespace zvfv;

extern "C" {

// Sorted unique (row, col) node pairs of all elements (zvcfd/fv/pattern.py:18-33): builds the
// pattern's keys in a handle and reports its number of blocks. The stream is synchronised.
int zvfv_pattern_create(void **handle, int64_t n_nodes, int n_kinds, const int32_t *const *conn,
                        const int64_t *n_elems, const int32_t *nodes_per, int64_t *nnzb,
                        void *stream) {
    if (!handle || !nnzb || n_nodes <= 0 || n_kinds <= 0) {
        set_error("pattern_create: bad arguments");
        return BAD_ARGUMENT;
    }
    cudaStream_t st = as_stream(stream);
    long long total = 0;
    for (int k = 0; k < n_kinds; ++k) total += n_elems[k] * (long long)nodes_per[k] * nodes_per[k];
    DevBuf<unsigned long long> keys, sorted, uniq;
    DevBuf<long long> nsel;
    ZV_TRY(keys.alloc(total, st));
    ZV_TRY(sorted.alloc(total, st));
    ZV_TRY(nsel.alloc(1, st));
    long long off = 0;
    for (int k = 0; k < n_kinds; ++k) {
        const long long m = n_elems[k] * (long long)nodes_per[k] * nodes_per[k];
        if (m)
            k_pair_keys<<<grid_for(m, 256), 256, 0, st>>>(conn[k], n_elems[k], nodes_per[k],
                                                          n_nodes, keys.p + off); count_launch();
        off += m;
    }
    ZV_TRY(launch_status("pattern keys"));
    const int end_bit = bits_for((unsigned long long)n_nodes * (unsigned long long)n_nodes);
    size_t tmp_sort = 0, tmp_uniq = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, keys.p, sorted.p, (int64_t)total, 0, end_bit, st);
    cub::DeviceSelect::Unique(nullptr, tmp_uniq, sorted.p, keys.p, nsel.p, (int64_t)total, st);
    DevBuf<unsigned char> tmp;
    ZV_TRY(tmp.alloc(tmp_sort > tmp_uniq ? tmp_sort : tmp_uniq, st));
    ZV_TRY(cuda_status(cub::DeviceRadixSort::SortKeys(tmp.p, tmp_sort, keys.p, sorted.p,
                                                      (int64_t)total, 0, end_bit, st), "sort"));
    ZV_TRY(cuda_status(cub::DeviceSelect::Unique(tmp.p, tmp_uniq, sorted.p, keys.p, nsel.p,
                                                 (int64_t)total, st), "unique"));
    long long nnz = 0;
    ZV_TRY(cuda_status(cudaMemcpyAsync(&nnz, nsel.p, sizeof(long long), cudaMemcpyDeviceToHost, st),
                       "copy"));
    ZV_TRY(cuda_status(cudaStreamSynchronize(st), "sync"));
    Pattern *h = new Pattern;
    h->n_nodes = n_nodes;
    h->nnz = nnz;
    if (cudaMalloc((void **)&h->keys, (nnz ? nnz : 1) * sizeof(unsigned long long)) != cudaSuccess) {
        delete h;
        set_error("pattern_create: out of memory");
        return OUT_OF_MEMORY;
    }
    cudaMemcpyAsync(h->keys, keys.p, nnz * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st);
    *handle = h;
    *nnzb = nnz;
    return launch_status("pattern");
}

// indptr int64 (N+1) and indices int32 (nnzb) of the pattern, into caller memory
int zvfv_pattern_fill(void *handle, int64_t *indptr, int32_t *indices, void *stream) {
    Pattern *h = static_cast<Pattern *>(handle);
    if (!h) return BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    k_row_starts<<<grid_for(h->n_nodes + 1, 256), 256, 0, st>>>(h->keys, h->nnz, h->n_nodes,
                                                                (long long *)indptr); count_launch();
    if (h->nnz)
        k_cols<<<grid_for(h->nnz, 256), 256, 0, st>>>(h->keys, h->nnz, h->n_nodes, indices); count_launch();
    return launch_status("pattern fill");
}

int zvfv_pattern_destroy(void *handle) {
    Pattern *h = static_cast<Pattern *>(handle);
    if (!h) return OK;
    cudaFree(h->keys);
    delete h;
    return OK;
}

// Element colours (zvcfd/fv/fast.py:94-130): rounds of claim and pick until every element is
// coloured; node masks of `words` 64-bit words, doubled (and the colouring restarted) when
// an element finds no free colour. The stream is synchronised once per round.
int zvfv_colour(const int32_t *conn, int n, int64_t E, int64_t n_nodes, int words,
                int32_t *colour, int32_t *n_colours, int64_t max_rounds, void *stream) {
    if (E < 0 || n <= 0 || n_nodes <= 0 || words <= 0) {
        set_error("colour: bad arguments");
        return BAD_ARGUMENT;
    }
    cudaStream_t st = as_stream(stream);
    if (E == 0) {
        *n_colours = 0;
        return OK;
    }
    DevBuf<unsigned long long> key, best, ctr;
    ZV_TRY(key.alloc(E, st));
    ZV_TRY(best.alloc(n_nodes, st));
    ZV_TRY(ctr.alloc(2, st));
    k_colour_keys<<<grid_for(E, 256), 256, 0, st>>>(E, key.p); count_launch();
    const unsigned grid = grid_for(E, 256);
    unsigned long long host[2];
    for (int attempt = 0; attempt < 16; ++attempt, words *= 2) {
        DevBuf<unsigned long long> used;
        ZV_TRY(used.alloc((size_t)n_nodes * words, st));
        ZV_TRY(cuda_status(cudaMemsetAsync(used.p, 0, (size_t)n_nodes * words * 8, st), "memset"));
        k_fill_i32<<<grid, 256, 0, st>>>(colour, E, -1); count_launch();
        bool full = false, done = false;
        for (long long round = 0; round < max_rounds; ++round) {
            k_fill_u64<<<grid_for(n_nodes, 256), 256, 0, st>>>(best.p, n_nodes, ~0ull); count_launch();
            ZV_TRY(cuda_status(cudaMemsetAsync(ctr.p, 0, 16, st), "memset"));
            k_colour_claim<<<grid, 256, 0, st>>>(conn, n, E, key.p, colour, best.p); count_launch();
            k_colour_pick<<<grid, 256, 0, st>>>(conn, n, E, key.p, colour, best.p, used.p, words,
                                                ctr.p); count_launch();
            ZV_TRY(cuda_status(cudaMemcpyAsync(host, ctr.p, 16, cudaMemcpyDeviceToHost, st), "copy"));
            ZV_TRY(cuda_status(cudaStreamSynchronize(st), "colour round"));
            if (host[1]) { full = true; break; }
            if (host[0] == 0) { done = true; break; }
        }
        if (done) {
            // the number of colours: max + 1, by a reduction of the colours
            DevBuf<int> mx;
            ZV_TRY(mx.alloc(1, st));
            size_t tmp_bytes = 0;
            cub::DeviceReduce::Max(nullptr, tmp_bytes, colour, mx.p, (int64_t)E, st);
            DevBuf<unsigned char> tmp;
            ZV_TRY(tmp.alloc(tmp_bytes, st));
            cub::DeviceReduce::Max(tmp.p, tmp_bytes, colour, mx.p, (int64_t)E, st);
            int cmax = 0;
            ZV_TRY(cuda_status(cudaMemcpyAsync(&cmax, mx.p, 4, cudaMemcpyDeviceToHost, st), "copy"));
            ZV_TRY(cuda_status(cudaStreamSynchronize(st), "sync"));
            *n_colours = cmax + 1;
            return OK;
        }
        if (!full) {
            set_error("colour: not finished in %lld rounds", (long long)max_rounds);
            return NOT_CONVERGED;
        }
    }
    set_error("colour: more than 2^20 colours");
    return UNSUPPORTED;
}

// Slot order: elements sorted stably by colour (argsort(colour * E + e), zvcfd/fv/fast.py:200),
// and the first slot of each colour (offsets, C + 1 entries).
int zvfv_slot_order(const int32_t *colour, int64_t E, int32_t n_colours, int64_t *order,
                    int64_t *offsets, void *stream) {
    cudaStream_t st = as_stream(stream);
    if (E <= 0 || n_colours <= 0) {
        set_error("slot_order: no elements or colours");
        return BAD_ARGUMENT;
    }
    DevBuf<int> idx, sorted_c, sorted_i;
    ZV_TRY(idx.alloc(E, st));
    ZV_TRY(sorted_c.alloc(E, st));
    ZV_TRY(sorted_i.alloc(E, st));
    k_iota<<<grid_for(E, 256), 256, 0, st>>>(idx.p, E); count_launch();
    const int end_bit = bits_for((unsigned long long)n_colours);
    size_t tmp_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, colour, sorted_c.p, idx.p, sorted_i.p,
                                    (int64_t)E, 0, end_bit, st);
    DevBuf<unsigned char> tmp;
    ZV_TRY(tmp.alloc(tmp_bytes, st));
    ZV_TRY(cuda_status(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, colour, sorted_c.p, idx.p,
                                                       sorted_i.p, (int64_t)E, 0, end_bit, st),
                       "sort"));
    k_widen<<<grid_for(E, 256), 256, 0, st>>>(sorted_i.p, E, (long long *)order); count_launch();
    k_colour_offsets<<<grid_for(n_colours + 1, 256), 256, 0, st>>>(sorted_c.p, E, n_colours,
                                                                   (long long *)offsets); count_launch();
    return launch_status("slot order");
}

// The structure of A^T for a block-CSR pattern: tptr int64 (n+1), and per entry q of
// column j the row trow[q] (int32, ascending) and the block index tperm[q] (int64) of A.
int zvfv_bsr_transpose(int64_t n, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                       int64_t *tptr, int32_t *trow, int64_t *tperm, void *stream) {
    cudaStream_t st = as_stream(stream);
    if (n <= 0 || nnz <= 0) {
        set_error("bsr_transpose: empty pattern");
        return BAD_ARGUMENT;
    }
    DevBuf<long long> idx, row;
    DevBuf<int> cols;
    ZV_TRY(idx.alloc(nnz, st));
    ZV_TRY(row.alloc(nnz, st));
    ZV_TRY(cols.alloc(nnz, st));
    k_iota64s<<<grid_for(nnz, 256), 256, 0, st>>>(idx.p, nnz); count_launch();
    k_row_of_block<<<grid_for(n, 256), 256, 0, st>>>(n, (const long long *)indptr, row.p); count_launch();
    const int end_bit = bits_for((unsigned long long)n);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, indices, cols.p, idx.p, (long long *)tperm,
                                    (int64_t)nnz, 0, end_bit, st);
    DevBuf<unsigned char> tmp;
    ZV_TRY(tmp.alloc(tb, st));
    ZV_TRY(cuda_status(cub::DeviceRadixSort::SortPairs(tmp.p, tb, indices, cols.p, idx.p,
                                                       (long long *)tperm, (int64_t)nnz, 0,
                                                       end_bit, st), "sort"));
    k_col_starts<<<grid_for(n + 1, 256), 256, 0, st>>>(cols.p, nnz, n, (long long *)tptr); count_launch();
    k_transpose_fill<<<grid_for(nnz, 256), 256, 0, st>>>(nnz, (const long long *)tperm, row.p, trow); count_launch();
    return launch_status("bsr transpose");
}

// dst[r] = src[idx[r]] (gather) or dst[idx[r]] = src[r] (scatter), rows of `width` bytes
int zvfv_permute_rows(const void *src, const int64_t *idx, int64_t rows, int64_t width,
                      void *dst, int scatter, void *stream) {
    if (rows <= 0 || width <= 0) return OK;
    k_gather_rows<<<grid_for(rows * width, 256), 256, 0, as_stream(stream)>>>(
        (const unsigned char *)src, (const long long *)idx, rows, width, (unsigned char *)dst,
        scatter); count_launch();
    return launch_status("permute rows");
}

}  // extern "C"
