// y = A x and x.y for a 6x6 block-sparse matrix, with no device allocation.
//
// The solver handles of this library allocate their workspaces with
// cudaMalloc once, at create time. Some callers cannot do that: a host
// application whose device memory is owned by another allocator (a framework's
// caching pool that has reserved the GPU), or a real-time capture loop that
// forbids allocation after start-up because cudaMalloc may synchronise the
// device. For them this file offers the PCG operator step — the block SpMV with
// its fused FP64 dot product, the same computation pcg_spmv_kernel performs on
// the solver's own matrix — over a matrix and vectors the caller already holds.
//
// The only global memory the kernel needs beyond its inputs and outputs is the
// per-CTA partial sums of x.y, a completion ticket and an error flag. They live
// in the file-scope array g_noalloc_scratch below, which every GPU that loads
// the library holds until the process exits. Host code cannot use that name as
// a device address, so the entry point looks the address up with
// cudaGetSymbolAddress on the current device and passes it to the kernel.
#include "kernels_common.cuh"

#include <mutex>
#include <string>

namespace mvdr {

int record_failure(int code, const std::string& msg);

namespace {

constexpr uint32_t kRowsPerCta = 32;   // block rows per CTA (6 threads each)
constexpr uint32_t kThreads = 6 * kRowsPerCta;
constexpr uint32_t kMaxCtas = MVDR_NOALLOC_MAX_BLOCK_ROWS / kRowsPerCta;
static_assert(kMaxCtas * kRowsPerCta == MVDR_NOALLOC_MAX_BLOCK_ROWS, "row limit must be a multiple of the CTA rows");

// [0, kMaxCtas): per-CTA partial sums of x.y; [kMaxCtas]: completion ticket;
// [kMaxCtas + 1]: error flag (a column index outside the matrix). The last two
// are read as 64-bit integers and cleared by the host before every launch.
constexpr uint32_t kTicketSlot = kMaxCtas;
constexpr uint32_t kFlagSlot = kMaxCtas + 1;
static __device__ __align__(256) double g_noalloc_scratch[kMaxCtas + 2];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// The device address of g_noalloc_scratch on the current device. A call on a
// stream that is not being captured looks the address up again (a
// cudaDeviceReset since the last call reloads the module, and the old address
// would belong to the destroyed context) and keeps it for the device; a call
// on a capturing stream uses the kept address, because the lookup may load
// the module, which a capture does not allow.
cudaError_t scratch_for_current_device(cudaStream_t st, double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    } else if (!g_scratch_ptr[dev]) {
        return cudaErrorStreamCaptureUnsupported;  // no call on this device before the capture
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

// Six threads per block row, one per scalar row; row-major blocks,
// blocks[36 s + 6 r + k] = A(r, k) of stored block s. Rows accumulate in
// double; x.y uses the stored (rounded) y and is summed in double, the CTA
// partials in index order by the last CTA to finish.
__global__ void __launch_bounds__(kThreads) noalloc_spmv_dot_kernel(uint32_t num_rows, uint32_t num_blocks,
                                                                     const int32_t* __restrict__ rowptr,
                                                                     const int32_t* __restrict__ colidx,
                                                                     const float* __restrict__ blocks,
                                                                     const float* __restrict__ x, float* __restrict__ y,
                                                                     double* __restrict__ x_dot_y, double* scratch) {
    const uint32_t br = blockIdx.x * kRowsPerCta + threadIdx.x / 6;
    const uint32_t r = threadIdx.x % 6;
    double part = 0.0;
    bool bad = false;
    if (br < num_rows) {
        // clamp the row's range to the stored blocks so that a malformed
        // rowptr cannot read past them
        int64_t s0 = rowptr[br], s1 = rowptr[br + 1];
        s0 = s0 < 0 ? 0 : (s0 > (int64_t)num_blocks ? (int64_t)num_blocks : s0);
        s1 = s1 < s0 ? s0 : (s1 > (int64_t)num_blocks ? (int64_t)num_blocks : s1);
        double acc = 0.0;
        for (int64_t s = s0; s < s1; ++s) {
            const int32_t col = colidx[s];
            if (col < 0 || (uint32_t)col >= num_rows) {
                bad = true;
                continue;
            }
            const float* a = blocks + 36 * s + 6 * r;
            const float* xv = x + 6 * (size_t)col;
#pragma unroll
            for (int k = 0; k < 6; ++k) acc += (double)a[k] * (double)xv[k];
        }
        const float yv = (float)acc;
        y[6 * (size_t)br + r] = yv;
        part = (double)x[6 * (size_t)br + r] * (double)yv;
    }
    if (__any_sync(0xffffffffu, bad) && lane_id() == 0)
        atomicOr(reinterpret_cast<unsigned long long*>(scratch + kFlagSlot), 1ull);

    __shared__ double ws[kThreads / 32];
    __shared__ bool last;
    part = warp_sum(part);
    if (lane_id() == 0) ws[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (uint32_t w = 0; w < kThreads / 32; ++w) s += ws[w];
        scratch[blockIdx.x] = s;
        __threadfence();
        const unsigned long long prev =
            atomicAdd(reinterpret_cast<unsigned long long*>(scratch + kTicketSlot), 1ull);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    const volatile double* pp = scratch;
    double total = 0.0;
    for (uint32_t c = 0; c < gridDim.x; ++c) total += pp[c];
    const volatile unsigned long long* flag = reinterpret_cast<const volatile unsigned long long*>(scratch + kFlagSlot);
    *x_dot_y = *flag ? __longlong_as_double(0x7ff8000000000000ll) : total;
}

}  // namespace
}  // namespace mvdr

extern "C" MVDR_API int mvdr_bsr6_spmv_dot_noalloc(uint32_t num_block_rows, uint32_t num_blocks,
                                                   const int32_t* rowptr, const int32_t* colidx, const float* blocks,
                                                   const float* x, float* y, double* x_dot_y, void* stream) {
    using namespace mvdr;
    if (!rowptr || !x || !y || !x_dot_y || (num_blocks && (!colidx || !blocks)))
        return record_failure(MVDR_EINVAL, "mvdr_bsr6_spmv_dot_noalloc: null argument");
    if (num_block_rows > MVDR_NOALLOC_MAX_BLOCK_ROWS)
        return record_failure(MVDR_ECAPACITY, "mvdr_bsr6_spmv_dot_noalloc: " + std::to_string(num_block_rows) +
                                                  " block rows exceed the maximum of " +
                                                  std::to_string(MVDR_NOALLOC_MAX_BLOCK_ROWS));
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* scratch = nullptr;
    cudaError_t e = scratch_for_current_device(st, &scratch);
    if (e != cudaSuccess)
        return record_failure(MVDR_ECUDA, std::string("mvdr_bsr6_spmv_dot_noalloc: scratch address lookup: ") +
                                              cudaGetErrorString(e));
    if (num_block_rows == 0) {
        e = cudaMemsetAsync(x_dot_y, 0, sizeof(double), st);
    } else {
        // the ticket and the error flag must start at zero; the partial sums
        // are overwritten by their CTAs
        e = cudaMemsetAsync(scratch + kTicketSlot, 0, 2 * sizeof(double), st);
        if (e == cudaSuccess) {
            const uint32_t ctas = (num_block_rows + kRowsPerCta - 1) / kRowsPerCta;
            MVDR_LAUNCH(noalloc_spmv_dot_kernel, dim3(ctas), kThreads, 0, st, num_block_rows, num_blocks, rowptr,
                        colidx, blocks, x, y, x_dot_y, scratch);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess)
        return record_failure(MVDR_ECUDA, std::string("mvdr_bsr6_spmv_dot_noalloc: ") + cudaGetErrorString(e));
    return MVDR_OK;
}
