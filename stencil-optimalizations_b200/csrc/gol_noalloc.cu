// gol_rows_run_noalloc: a multi-generation run that allocates nothing.
//
// Some callers cannot call cudaMalloc: code running where allocation is not
// allowed or not wanted, such as a framework that owns all device memory
// through its own pool, a real-time loop that cannot take the device-wide
// synchronisation a cudaMalloc/cudaFree may cause, or a plugin host that
// forbids foreign allocations. They hand in the input and output grids; the
// ping-pong partner grid the passes need comes from a fixed array compiled
// into this library instead of from the allocator.
//
// The scratch is a file-scope __device__ array of kNoAllocMaxBytes (32 MiB,
// room for a 16384 x 16384 grid). Every GPU that loads the library holds it
// until the process exits. In host code its name is only a host-side
// stand-in, not a device address, so the address is looked up once per
// device with cudaGetSymbolAddress (with that device current) and cached.
// The cached address belongs to the device's current context: after a
// cudaDeviceReset it is stale, and calls on that device must not be made
// again in this process.
#include <mutex>

#include "gol_b200.h"
#include "gol_internal.h"

namespace {

constexpr size_t kNoAllocMaxBytes = (size_t)32 << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxBytes / sizeof(uint32_t)];

std::mutex g_noalloc_mu;
uint32_t* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device (looked up on
// the first call for that device).
int noalloc_scratch(int dev, uint32_t** out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return GOL_E_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return GOL_E_CUDA;
        g_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return GOL_OK;
}

} // namespace

extern "C" int gol_rows_run_noalloc(const void* d_in, void* d_out, uint64_t x, uint64_t y,
                                    uint64_t n, uint32_t k, void* stream) {
    if (!d_in || !d_out || d_in == d_out || x % 32 || x == 0 || y == 0) return GOL_E_INVALID;
    if (((uintptr_t)d_in | (uintptr_t)d_out) & 15u) return GOL_E_INVALID;
    if (k == 0) k = 4;
    if (k > (uint32_t)golb200::kMaxTemporalSteps) return GOL_E_INVALID;
    // The same limits as every other entry point (x / 32 and y fit the
    // kernels' int indices), before any size arithmetic can wrap.
    if (x / 32 > (1ull << 30) || y > (1ull << 30)) return GOL_E_INVALID;
    const uint64_t bytes = x / 8 * y;
    if (bytes > kNoAllocMaxBytes) return GOL_E_UNSUPPORTED;   // grid larger than the scratch
    const int W = (int)(x / 32), Y = (int)y;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        return cudaMemcpyAsync(d_out, d_in, bytes, cudaMemcpyDeviceToDevice, s) == cudaSuccess
                   ? GOL_OK
                   : GOL_E_CUDA;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GOL_E_CUDA;
    uint32_t* scratch = nullptr;
    int rc = noalloc_scratch(dev, &scratch);
    if (rc != GOL_OK) return rc;

    // Passes of k generations (the last one shorter when k does not divide
    // n). Launch i writes d_out when (passes - 1 - i) is even, otherwise the
    // scratch, so the chain ends in d_out and no pass writes what it reads.
    // Each pass writes every word of its destination before anything reads
    // it, so the scratch needs no clearing between calls.
    const uint64_t full = n / k;
    const int rem = (int)(n % k);
    const uint64_t passes = full + (rem ? 1 : 0);
    const int sms = golb200::device_sm_count(dev);
    const uint32_t* src = static_cast<const uint32_t*>(d_in);
    for (uint64_t i = 0; i < passes; ++i) {
        const int kk = (i < full) ? (int)k : rem;
        uint32_t* dst = ((passes - 1 - i) % 2 == 0) ? static_cast<uint32_t*>(d_out) : scratch;
        golb200::RowsPlan p;
        if (!golb200::plan_rows(W, Y, kk, 0, 0, sms, &p)) return GOL_E_UNSUPPORTED;
        if (golb200::launch_rows_pass(src, dst, W, Y, kk, p, s) != cudaSuccess) return GOL_E_CUDA;
        src = dst;
    }
    return GOL_OK;
}
