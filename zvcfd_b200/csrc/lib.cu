// Library-wide state: the last error message, device properties, version, and the C-ABI
// wrappers of the block-CSR SpMV.
#include <atomic>
#include <cstdarg>
#include <cstring>

#include "spmv.cuh"

namespace zvfv {

static thread_local char g_error[512] = "";
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void count_launches(long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

int sm_count() {
    static int cached = 0;
    if (!cached) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
        if (cached <= 0) cached = 148;
    }
    return cached;
}

}  // namespace zvfv

using namespace zvfv;

extern "C" {

const char *zvfv_last_error(void) { return g_error; }

int zvfv_version(void) { return 1; }

// kernels launched by this library since the process started
int64_t zvfv_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int zvfv_bsr_spmv(int64_t n, const int64_t *indptr, const int32_t *indices, const double *data,
                  const double *x, double *y, int lanes, void *stream) {
    return bsr_spmv_launch<false, double, double>(lanes, n, (const long long *)indptr, indices,
                                                  data, x, nullptr, y, as_stream(stream));
}

int zvfv_bsr_residual(int64_t n, const int64_t *indptr, const int32_t *indices,
                      const double *data, const double *x, const double *b, double *r, int lanes,
                      void *stream) {
    return bsr_spmv_launch<true, double, double>(lanes, n, (const long long *)indptr, indices,
                                                 data, x, b, r, as_stream(stream));
}

int zvfv_bsr_spmv_f32(int64_t n, const int64_t *indptr, const int32_t *indices,
                      const float *data, const float *x, float *y, int lanes, void *stream) {
    return bsr_spmv_launch<false, float, float>(lanes, n, (const long long *)indptr, indices, data,
                                                x, nullptr, y, as_stream(stream));
}

// y = A^T x through the transpose structure of zvfv_bsr_transpose (the adjoint's product)
int zvfv_bsr_spmv_t(int64_t n, const int64_t *tptr, const int32_t *trow, const int64_t *tperm,
                    const double *data, const double *x, double *y, int lanes, void *stream) {
    return bsr_spmv_t_launch<false, double, double>(lanes, n, (const long long *)tptr, trow,
                                                    (const long long *)tperm, data, x, nullptr, y,
                                                    as_stream(stream));
}

}  // extern "C"
