// Kernel instantiations and launch dispatch for the row-band temporal
// kernel, plus device-side pack/unpack between uint8 cells and row words.
#include <algorithm>

#include "gol_b200.h"
#include "gol_internal.h"
#include "gol_rows_resident.cuh"
#include "gol_rows_stream.cuh"
#include "gol_rows_temporal.cuh"
#include "gol_word_ops.cuh"

#ifndef GOL_STREAM_THREADS
#define GOL_STREAM_THREADS 128   // CTA size of the one-generation streaming kernel
#endif
#ifndef GOL_STREAM_CTAS_PER_SM
// Default band of the streaming kernel: about this many CTAs per SM per pass
// (at 32768^2: 9-row bands; 8-, 12- and 16-row bands ran at 5.40, 5.31 and
// 5.15 TB/s algorithmic).
#define GOL_STREAM_CTAS_PER_SM 48
#endif

namespace golb200 {

namespace {

// Launched as a programmatic dependent of the previous kernel in the
// stream: its CTAs may be scheduled while that kernel drains and wait in
// griddepcontrol.wait (full completion and memory flush of the previous
// grid) before touching global memory, which hides the launch gap between
// consecutive passes.
template <int WPL, int K>
cudaError_t launch_one(const RowsLaunch& a, const RowsPlan& p, cudaStream_t stream) {
    // Deep passes need more than the default 48 KB of dynamic shared memory
    // (the edge table grows with K): opt in once per instantiation.
    static const cudaError_t attr_ok = cudaFuncSetAttribute(
        rows_temporal_kernel<WPL, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)temporal_smem_bytes(K, kTemporalMaxThreads, WPL));
    if (attr_ok != cudaSuccess) return attr_ok;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.nbands, p.nslices);
    cfg.blockDim = dim3(p.threads);
    cfg.dynamicSmemBytes = temporal_smem_bytes(K, p.threads, WPL);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, rows_temporal_kernel<WPL, K>, a);
}

// The one-generation streaming kernel, also a programmatic dependent.
template <int WPL>
cudaError_t launch_stream(const RowsLaunch& a, const RowsPlan& p, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    const long long ctas = (long long)p.nslices * p.nbands;
    if (ctas > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(p.threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, rows_stream_kernel<WPL>, a);
}

template <int WPL, int K>
cudaError_t dispatch_k(int k, const RowsLaunch& a, const RowsPlan& p, cudaStream_t stream) {
    if constexpr (K > kMaxKForWpl(WPL)) {
        return cudaErrorInvalidValue;
    } else {
        if (k == K) return launch_one<WPL, K>(a, p, stream);
        return dispatch_k<WPL, K + 1>(k, a, p, stream);
    }
}

} // namespace

int device_sm_count(int device) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) n = 148;
    return n > 0 ? n : 148;
}

bool plan_rows(int W, int Y, int k, int band_rows, int wpl, int num_sms, RowsPlan* plan,
               bool allow_stream) {
    if (k < 1 || k > kMaxTemporalSteps || W <= 0) return false;
    if (wpl != 0) {
        if ((wpl != 1 && wpl != 2 && wpl != 4) || W % wpl || k > kMaxKForWpl(wpl)) return false;
    } else {
        // Widest lane access whose register rings fit this depth.
        for (int cand : {4, 2, 1}) {
            if (W % cand == 0 && k <= kMaxKForWpl(cand)) {
                wpl = cand;
                break;
            }
        }
        if (wpl == 0) return false;
    }
    plan->wpl = wpl;
    const int lanes = W / wpl;
    plan->stream = k == 1 && allow_stream;
    if (plan->stream) {
        // One generation: lanes of wpl words across the row in CTAs of up to
        // GOL_STREAM_THREADS threads, each thread walking `band` rows. The
        // default band gives about GOL_STREAM_CTAS_PER_SM CTAs per SM (many
        // waves of short-lived CTAs), never below 8 rows (each band re-reads
        // one halo row above and one below, from L2) nor above 64.
        plan->threads = std::min(GOL_STREAM_THREADS, (lanes + 31) / 32 * 32);
        plan->nslices = (lanes + plan->threads - 1) / plan->threads;
        plan->slice = plan->threads * wpl;
        plan->halo = 0;
        int band = band_rows;
        if (band <= 0) {
            const long long ctas = (long long)GOL_STREAM_CTAS_PER_SM * num_sms;
            band = (int)std::min<long long>(64, std::max<long long>(8, ((long long)Y * plan->nslices + ctas - 1) / ctas));
        }
        band = std::min(band, std::max(Y, 1));
        plan->band = band;
        plan->nbands = (Y + band - 1) / band;
        return true;
    }
    if (lanes <= kTemporalMaxThreads) {
        plan->slice = W;
        plan->nslices = 1;
        plan->halo = 0;
        plan->threads = std::max(32, (lanes + 31) / 32 * 32);
    } else {
        const int per = kTemporalMaxThreads - 2;               // one halo lane each side
        const int ns = (lanes + per - 1) / per;
        const int slice_lanes = (lanes + ns - 1) / ns;
        plan->slice = slice_lanes * wpl;
        plan->nslices = (W + plan->slice - 1) / plan->slice;
        plan->halo = wpl;
        plan->threads = (slice_lanes + 2 + 31) / 32 * 32;
    }
    int band = band_rows;
    if (band <= 0) {
        // About two CTAs per SM, or more when a CTA has fewer than four
        // warps (narrow grids: at 8192^2, k = 4, 2-warp CTAs with 16-row
        // bands ran at 18.9 T cell-updates/s against 16.0 T with 28-row
        // ones); never thinner than a few times the depth, whose y-halo
        // costs ~k extra rows per stage per band.
        const int warps = plan->threads / 32;
        const int per_sm = warps >= 4 ? 2 : 2 * ((4 + warps - 1) / warps);
        const int target = std::max(1, per_sm * num_sms / plan->nslices);
        band = (Y + target - 1) / target;
        band = std::max(band, std::max(8, 4 * k));
    }
    band = std::min(band, std::max(Y, 1));
    plan->band = band;
    plan->nbands = (Y + band - 1) / band;
    return true;
}

#ifndef GOL_RESIDENT_K
#define GOL_RESIDENT_K 8   // generations per epoch of the resident run
#endif
#ifndef GOL_RESIDENT_WPL
#define GOL_RESIDENT_WPL 2
#endif
#ifndef GOL_RESIDENT_THREADS
#define GOL_RESIDENT_THREADS 512   // threads per CTA (lanes across a row x row groups)
#endif

bool plan_resident(int W, int Y, int k_epoch, int device, ResidentPlan* p) {
    const int K = k_epoch > 0 ? k_epoch : GOL_RESIDENT_K;
    if (K < 1 || K > 64 || W <= 0 || Y <= 0) return false;
    int wpl = GOL_RESIDENT_WPL;
    while (wpl > 1 && W % wpl) wpl /= 2;
    const int lanes = ((W + wpl - 1) / wpl + 31) / 32 * 32;
    if (lanes > kResidentMaxThreads) return false;
    const int groups = std::max(1, std::min(GOL_RESIDENT_THREADS, kResidentMaxThreads) / lanes);
    int sms = 0, smem_max = 0, coop = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop)
        return false;
    // Every band at least K rows (a band's halo comes from its neighbours
    // only), at most one CTA per SM; the largest band's two buffers must fit.
    // A grid of fewer than K rows is one band with no neighbours.
    const int nbands = std::max(1, std::min(sms, Y / K));
    const int band = (Y + nbands - 1) / nbands;
    const size_t smem = resident_smem_bytes(band, K, lanes, wpl);
    if (smem + 1024 > (size_t)smem_max) return false;
    p->wpl = wpl;
    p->lanes = lanes;
    p->groups = groups;
    p->K = K;
    p->band = band;
    p->nbands = nbands;
    p->smem = smem;
    p->pub_words = (size_t)nbands * 4 * K * W;
    return true;
}

template <int WPL, int LANES>
static cudaError_t launch_resident_lanes(const ResidentLaunch& a, const ResidentPlan& p,
                                         cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(rows_resident_kernel<WPL, LANES>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    if (e != cudaSuccess) return e;
    ResidentLaunch arg = a;
    void* args[] = {&arg};
    return cudaLaunchCooperativeKernel((const void*)rows_resident_kernel<WPL, LANES>,
                                       dim3(p.nbands), dim3(p.lanes * p.groups), args, p.smem,
                                       stream);
}

// Row widths of 64, 128 and 256 lanes (4096-, 8192- and 16384-cell rows at
// two words per lane) get a compile-time row stride; others a runtime one.
template <int WPL>
static cudaError_t launch_resident_wpl(const ResidentLaunch& a, const ResidentPlan& p,
                                       cudaStream_t stream) {
    switch (p.lanes) {
        case 64: return launch_resident_lanes<WPL, 64>(a, p, stream);
        case 128: return launch_resident_lanes<WPL, 128>(a, p, stream);
        case 256: return launch_resident_lanes<WPL, 256>(a, p, stream);
        default: return launch_resident_lanes<WPL, 0>(a, p, stream);
    }
}

cudaError_t launch_resident(const uint32_t* src, uint32_t* dst, int W, int Y, long long gens,
                            const ResidentPlan& p, uint32_t* pub, int* epoch_done, int* status,
                            cudaStream_t stream, long long spin_limit) {
    cudaError_t e = cudaMemsetAsync(epoch_done, 0, (size_t)p.nbands * sizeof(int), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    ResidentLaunch a{src, dst, pub, epoch_done, status, W, Y, p.K, p.lanes, p.groups, gens,
                     spin_limit > 0 ? spin_limit : (1ll << 24)};
    switch (p.wpl) {
        case 4: return launch_resident_wpl<4>(a, p, stream);
        case 2: return launch_resident_wpl<2>(a, p, stream);
        case 1: return launch_resident_wpl<1>(a, p, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_rows_pass(const uint32_t* src, uint32_t* dst, int W, int Y, int k,
                             const RowsPlan& p, cudaStream_t stream, int pitch) {
    if (Y <= 0 || W <= 0) return cudaSuccess;
    RowsLaunch a{src, dst, W, Y, p.band, p.slice, p.halo, pitch ? pitch : W};
    if (p.stream) {
        if (k != 1) return cudaErrorInvalidValue;
        switch (p.wpl) {
            case 4: return launch_stream<4>(a, p, stream);
            case 2: return launch_stream<2>(a, p, stream);
            case 1: return launch_stream<1>(a, p, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (p.wpl) {
        case 4: return dispatch_k<4, 1>(k, a, p, stream);
        case 2: return dispatch_k<2, 1>(k, a, p, stream);
        case 1: return dispatch_k<1, 1>(k, a, p, stream);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Device pack / unpack (uint8 cell grid <-> row words), the device-side form
// of GeneralBitGrid::fill_grid / to_grid (general_bit_grid.hpp:171-246).
// ---------------------------------------------------------------------------

namespace {

// 8 cells (one byte each, nonzero = alive) -> 8 bits, cell i at bit i.
__device__ __forceinline__ uint32_t pack8(unsigned long long v) {
    v |= v >> 4;
    v |= v >> 2;
    v |= v >> 1;
    v &= 0x0101010101010101ull;
    return (uint32_t)((v * 0x0102040810204080ull) >> 56);
}

// 8 bits -> 8 cells of 0/1, bit i to byte i.
__device__ __forceinline__ unsigned long long unpack8(uint32_t b) {
    unsigned long long v = (unsigned long long)(b & 0xffu) * 0x0101010101010101ull;
    v &= 0x8040201008040201ull;
    return ((v + 0x7f7f7f7f7f7f7f7full) >> 7) & 0x0101010101010101ull;
}

__global__ void pack_cells_kernel(const uint8_t* __restrict__ cells, uint32_t* __restrict__ words,
                                  size_t nwords) {
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < nwords;
         w += (size_t)gridDim.x * blockDim.x) {
        const ulonglong2* p = reinterpret_cast<const ulonglong2*>(cells + w * 32);
        const ulonglong2 a = p[0];
        const ulonglong2 b = p[1];
        words[w] = pack8(a.x) | (pack8(a.y) << 8) | (pack8(b.x) << 16) | (pack8(b.y) << 24);
    }
}

__global__ void unpack_cells_kernel(const uint32_t* __restrict__ words, uint8_t* __restrict__ cells,
                                    size_t nwords) {
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < nwords;
         w += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = words[w];
        ulonglong2* p = reinterpret_cast<ulonglong2*>(cells + w * 32);
        p[0] = make_ulonglong2(unpack8(v), unpack8(v >> 8));
        p[1] = make_ulonglong2(unpack8(v >> 16), unpack8(v >> 24));
    }
}

// Counter-based Bernoulli cells: cell i (raster order) of a grid with seed s
// is alive iff (mix64(s + (i + 1) * 0x9E3779B97F4A7C15) >> 11) * 2^-53 <
// density, mix64 the SplitMix64 finaliser. Each thread writes one word.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void hash_bernoulli_kernel(uint32_t* __restrict__ words, size_t nwords,
                                      unsigned long long seed, unsigned long long threshold) {
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < nwords;
         w += (size_t)gridDim.x * blockDim.x) {
        uint32_t v = 0;
        const unsigned long long base = (unsigned long long)w * 32ull;
#pragma unroll 8
        for (int b = 0; b < 32; ++b) {
            const unsigned long long h = mix64(seed + (base + b + 1ull) * 0x9E3779B97F4A7C15ull);
            v |= (uint32_t)((h >> 11) < threshold) << b;
        }
        words[w] = v;
    }
}

int grid_for(size_t n, int threads) {
    size_t blocks = (n + threads - 1) / threads;
    return (int)std::min<size_t>(std::max<size_t>(blocks, 1), 148 * 16);
}

} // namespace

cudaError_t launch_pack_cells(const uint8_t* cells, uint32_t* words, size_t x, size_t y,
                              cudaStream_t stream) {
    const size_t n = x / 32 * y;
    if (n == 0) return cudaSuccess;
    pack_cells_kernel<<<grid_for(n, 256), 256, 0, stream>>>(cells, words, n);
    return cudaPeekAtLastError();
}

unsigned long long bernoulli_threshold(double density) {
    if (!(density > 0)) return 0ull;
    if (density >= 1) return 1ull << 53;
    return (unsigned long long)(density * 9007199254740992.0);   // density * 2^53
}

cudaError_t launch_hash_bernoulli(uint32_t* words, size_t x, size_t y, uint64_t seed,
                                  double density, cudaStream_t stream) {
    const size_t n = x / 32 * y;
    if (n == 0) return cudaSuccess;
    hash_bernoulli_kernel<<<grid_for(n, 256), 256, 0, stream>>>(words, n, seed,
                                                                  bernoulli_threshold(density));
    return cudaPeekAtLastError();
}

void host_hash_bernoulli(uint8_t* cells, size_t n, uint64_t seed, double density) {
    const unsigned long long t = bernoulli_threshold(density);
    for (size_t i = 0; i < n; ++i)
        cells[i] = (mix64(seed + (i + 1ull) * 0x9E3779B97F4A7C15ull) >> 11) < t ? 1 : 0;
}

cudaError_t launch_unpack_cells(const uint32_t* words, uint8_t* cells, size_t x, size_t y,
                                cudaStream_t stream) {
    const size_t n = x / 32 * y;
    if (n == 0) return cudaSuccess;
    unpack_cells_kernel<<<grid_for(n, 256), 256, 0, stream>>>(words, cells, n);
    return cudaPeekAtLastError();
}

// ---------------------------------------------------------------------------
// Integer-pipe peak probe: independent LOP3 chains (8 per thread) with no
// memory traffic, to measure the lane-ops/s ceiling the temporal kernel's
// bit-sliced arithmetic is bounded by.
// ---------------------------------------------------------------------------

namespace {

__global__ void lop3_rate_kernel(uint32_t* sink, int iters, uint32_t seed) {
    uint32_t v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = (threadIdx.x + 1u) * (2u * j + 3u) ^ seed;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
                v[j] = lop3<LUT_XOR3>(v[j], v[(j + 1) & 7], v[(j + 3) & 7]);
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc ^= v[j];
    if (acc == 0x9e3779b9u) sink[blockIdx.x] = acc;   // keeps the chains live
}

} // namespace

cudaError_t probe_lop3_rate(int device, cudaStream_t stream, double* lane_ops_per_s) {
    const int sms = device_sm_count(device);
    const int blocks = sms * 8, threads = 256, iters = 4096;
    uint32_t* sink = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(uint32_t) * blocks);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    if (e == cudaSuccess) {
        lop3_rate_kernel<<<blocks, threads, 0, stream>>>(sink, iters / 8, 1u);   // warm-up
        cudaEventRecord(a, stream);
        lop3_rate_kernel<<<blocks, threads, 0, stream>>>(sink, iters, 2u);
        cudaEventRecord(b, stream);
        e = cudaEventSynchronize(b);
    }
    if (e == cudaSuccess) {
        float ms = 0.f;
        e = cudaEventElapsedTime(&ms, a, b);
        const double ops = (double)blocks * threads * iters * 16.0 * 8.0;
        *lane_ops_per_s = ops / (ms * 1e-3);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (sink) cudaFree(sink);
    return e;
}

} // namespace golb200
