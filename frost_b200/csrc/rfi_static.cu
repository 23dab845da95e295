// Allocation-free normalisation: frost_rfi_normalize_static.
//
// Some callers cannot call cudaMalloc while they process data: a real-time
// ring-buffer consumer that pre-allocates everything at start-up and must
// not touch the device allocator (which can block, synchronise the device or
// fail under memory pressure) once observing begins, or a host program whose
// device memory is owned by another framework's pool. For them this entry
// point cleans and normalises one block with the quiet configuration (no
// automatic excision: per-window bandpass from the sampled remedian with
// clipped refinement, dead channels masked, (x - loc) / scale in
// [channel][time] order, low frequency first) using only the caller's input
// and output buffers plus a fixed scratch array compiled into this file.
//
// The scratch is a file-scope static __device__ array of kScratchFloats
// floats (32 MiB + 256 KiB): every GPU that loads this module holds it until
// the process exits. Its device address is looked up once per device, on the
// first call made with that device current; under lazy module loading that
// lookup is also when the driver loads this module onto the device and sets
// the array up, so callers make that first call at start-up, before any
// stream capture. Every call shares the one array, so calls whose
// work overlaps on the GPU (different streams, or other threads) race and
// must be serialised by the caller; the array keeps the last call's contents
// and the call clears what must start at zero. No cudaMalloc, cudaFree or
// allocating library routine is called.

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <mutex>
#include <string>

#include "common.hpp"
#include "rfi_cleaner.hpp"
#include "rfi_kernels.hpp"

namespace fb::rfi {

namespace {

constexpr size_t kSampleFloats  = size_t{8} * 1024 * 1024; // sampled spectra
constexpr size_t kTableFloats   = size_t{64} * 1024;       // per-window tables, flags
constexpr size_t kScratchFloats = kSampleFloats + kTableFloats;

static __device__ __align__(256) float g_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
std::array<float*, kMaxDevices> g_scratch_ptr{};
std::array<std::once_flag, kMaxDevices> g_scratch_once;

float* scratch_for(int device) {
    if (device < 0 || device >= kMaxDevices)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "normalize_static: device index out of range");
    cudaError_t err = cudaSuccess;
    std::call_once(g_scratch_once[device], [&] {
        void* p = nullptr;
        err     = cudaGetSymbolAddress(&p, g_scratch);
        if (err == cudaSuccess)
            g_scratch_ptr[device] = static_cast<float*>(p);
    });
    if (err != cudaSuccess)
        throw Error(FROST_ERR_DEVICE, std::string("normalize_static: cudaGetSymbolAddress failed: ") +
                                          cudaGetErrorString(err));
    if (g_scratch_ptr[device] == nullptr)
        throw Error(FROST_ERR_DEVICE, "normalize_static: scratch set-up failed on an earlier call");
    return g_scratch_ptr[device];
}

template <int D> __device__ __forceinline__ float decode(const uint8_t* __restrict__ row, uint64_t c) {
    if constexpr (D == FROST_UINT8) {
        return static_cast<float>(row[c]);
    } else if constexpr (D == FROST_UINT16) {
        return static_cast<float>(reinterpret_cast<const uint16_t*>(row)[c]);
    } else if constexpr (D == FROST_UINT32) {
        return static_cast<float>(reinterpret_cast<const uint32_t*>(row)[c]);
    } else if constexpr (D == FROST_FLOAT32) {
        return reinterpret_cast<const float*>(row)[c];
    } else {
        constexpr unsigned kBits = D == FROST_UINT1 ? 1U : D == FROST_UINT2 ? 2U : 4U;
        const uint64_t bit       = c * kBits;
        return static_cast<float>((row[bit >> 3U] >> (bit & 7U)) & ((1U << kBits) - 1U));
    }
}

// Channels with no variance in the bandpass sample of every window are dead
// when constant over the block (lib/cpu/rfi_cpu.cpp:350-366).
template <int D>
__global__ void k_dead(Dims d, const uint8_t* __restrict__ raw, const uint32_t* __restrict__ unmeasured,
                       uint32_t* __restrict__ dead) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= d.nchans)
        return;
    uint32_t is_dead = 0;
    if (unmeasured[c] >= d.nwin) {
        float lo = FLT_MAX, hi = -FLT_MAX;
        for (uint64_t t = 0; t < d.nsamps; ++t) {
            const float x = decode<D>(raw + t * d.row_bytes, c);
            lo            = (x < lo) ? x : lo;
            hi            = (hi < x) ? x : hi;
        }
        is_dead = (hi > lo) ? 0U : 1U;
    }
    dead[c] = is_dead;
}

constexpr int kTile = 32;

template <int D>
__global__ void k_normalize_raw(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                                const float* __restrict__ scale, const uint32_t* __restrict__ dead,
                                int flip, uint64_t capacity, float* __restrict__ out) {
    __shared__ float tile[kTile][kTile + 1];
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kTile;
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.y) * kTile;
    const uint64_t n  = d.nchans;
    for (int k = threadIdx.y; k < kTile; k += blockDim.y) {
        const uint64_t t = t0 + k, c = c0 + threadIdx.x;
        float v          = 0.0F;
        if (t < d.nsamps && c < n && dead[c] == 0) {
            uint64_t w = t / d.window;
            w          = w < d.nwin - 1 ? w : d.nwin - 1;
            const uint64_t i = w * n + c;
            const float s    = scale[i] > 0.0F ? 1.0F / scale[i] : 1.0F;
            v                = (decode<D>(raw + t * d.row_bytes, c) - loc[i]) * s;
        }
        tile[k][threadIdx.x] = v;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < kTile; k += blockDim.y) {
        const uint64_t c = c0 + k, t = t0 + threadIdx.x;
        if (c < n && t < capacity) {
            const uint64_t dst      = flip ? n - 1 - c : c;
            out[dst * capacity + t] = tile[threadIdx.x][k];
        }
    }
}

__global__ void k_find_nonfinite(const uint32_t* __restrict__ w, uint64_t n,
                                 unsigned long long* first_bad) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
        if ((w[i] & 0x7F800000U) == 0x7F800000U)
            atomicMin(first_bad, static_cast<unsigned long long>(i));
}

#define FB_STATIC_DISPATCH(dtype, ...)                                                            \
    switch (dtype) {                                                                              \
    case FROST_UINT1: { constexpr int D = FROST_UINT1; __VA_ARGS__; } break;                      \
    case FROST_UINT2: { constexpr int D = FROST_UINT2; __VA_ARGS__; } break;                      \
    case FROST_UINT4: { constexpr int D = FROST_UINT4; __VA_ARGS__; } break;                      \
    case FROST_UINT8: { constexpr int D = FROST_UINT8; __VA_ARGS__; } break;                      \
    case FROST_UINT16: { constexpr int D = FROST_UINT16; __VA_ARGS__; } break;                    \
    case FROST_UINT32: { constexpr int D = FROST_UINT32; __VA_ARGS__; } break;                    \
    case FROST_FLOAT32: { constexpr int D = FROST_FLOAT32; __VA_ARGS__; } break;                  \
    default: throw Error(FROST_ERR_INVALID_ARGUMENT, "normalize_static: unsupported dtype");      \
    }

} // namespace

void normalize_static(const frost_block_layout& layout, float baseline_length, const uint8_t* block,
                      size_t block_bytes, size_t nsamps, float* out, size_t out_count,
                      cudaStream_t stream) {
    validate_layout(layout, baseline_length);
    const uint64_t n         = layout.nchans;
    const uint64_t row_bytes = n * static_cast<uint64_t>(bits_of(layout.dtype)) / 8;
    if (block == nullptr || out == nullptr)
        invalid("normalize_static: null block or output");
    // samples wider than a byte and the float output are read and written
    // as whole words: a misaligned pointer would fault the kernels
    const uintptr_t word = bits_of(layout.dtype) > 8 ? static_cast<uintptr_t>(bits_of(layout.dtype) / 8) : 1;
    if (reinterpret_cast<uintptr_t>(block) % word != 0 || reinterpret_cast<uintptr_t>(out) % 4 != 0)
        invalid("normalize_static: block and output must be aligned to their element size");
    if (block_bytes % row_bytes != 0 || block_bytes / row_bytes > layout.max_nsamps)
        invalid("normalize_static: invalid block size");
    const uint64_t capacity = block_bytes / row_bytes;
    const uint64_t valid    = nsamps == 0 ? capacity : nsamps;
    if (valid > capacity)
        invalid("normalize_static: nsamps exceeds block");
    if (valid < static_cast<uint64_t>(kMinBlockSamps))
        invalid("normalize_static: needs at least 64 samples (short tails need a retained "
                "calibration; use frost_rfi_execute_normalized)");
    if (out_count < capacity * n)
        invalid("normalize_static: output holds fewer than nchans * capacity floats");

    const double window_samples = static_cast<double>(baseline_length) / layout.tsamp;
    Dims d{};
    d.dtype     = layout.dtype;
    d.nchans    = n;
    d.row_bytes = row_bytes;
    d.nsamps    = valid;
    d.window    = std::max(static_cast<uint64_t>(window_samples), uint64_t{kMinWindow});
    d.nwin      = std::max<uint64_t>(valid / d.window, 1);
    d.nchunks   = 1;
    d.chunk     = valid;

    // Scratch layout (floats): samples [nwin][3125][n] | loc | scale | inv
    // [nwin][n] each | unmeasured [n] | dead [n] | first_bad (2 words).
    const uint64_t sample_need = d.nwin * kMaxBandpassRows * n;
    const uint64_t table_need  = 3 * d.nwin * n + 2 * n + 4;
    if (sample_need > kSampleFloats || table_need > kTableFloats)
        invalid("normalize_static: block needs " + std::to_string(sample_need) + " sample and " +
                std::to_string(table_need) + " table scratch floats; the static scratch holds " +
                std::to_string(kSampleFloats) + " and " + std::to_string(kTableFloats) +
                " (windows x channels <= " + std::to_string(kSampleFloats / kMaxBandpassRows) + ")");

    int device = 0;
    FB_CUDA(cudaGetDevice(&device));
    float* base          = scratch_for(device);
    float* samples       = base;
    float* loc           = base + kSampleFloats;
    float* scale         = loc + d.nwin * n;
    float* inv           = scale + d.nwin * n;
    uint32_t* unmeasured = reinterpret_cast<uint32_t*>(inv + d.nwin * n);
    uint32_t* dead       = unmeasured + n;
    auto* first_bad      = reinterpret_cast<unsigned long long*>(
        base + kSampleFloats + ((3 * d.nwin * n + 2 * n + 1) & ~uint64_t{1}));

    if (layout.dtype == FROST_FLOAT32) {
        const uint64_t words     = valid * n;
        unsigned long long first = words;
        FB_CUDA(cudaMemcpyAsync(first_bad, &first, sizeof(first), cudaMemcpyHostToDevice, stream));
        const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((words + 255) / 256, 148 * 16));
        k_find_nonfinite<<<blocks, 256, 0, stream>>>(reinterpret_cast<const uint32_t*>(block), words,
                                                     first_bad);
        FB_LAUNCH_CHECK();
        FB_CUDA(cudaMemcpyAsync(&first, first_bad, sizeof(first), cudaMemcpyDeviceToHost, stream));
        FB_CUDA(cudaStreamSynchronize(stream));
        if (first != words)
            invalid("RFI: non-finite float32 input at sample " + std::to_string(first / n) +
                    ", channel " + std::to_string(first % n));
    }
    FB_CUDA(cudaMemsetAsync(unmeasured, 0, n * sizeof(uint32_t), stream));
    launch_sample_rows(d, block, samples, stream);
    launch_bandpass(d, samples, loc, scale, inv, unmeasured, stream);
    FB_STATIC_DISPATCH(d.dtype, {
        k_dead<D><<<static_cast<unsigned>((n + 127) / 128), 128, 0, stream>>>(d, block, unmeasured, dead);
        FB_LAUNCH_CHECK();
        const dim3 grid(static_cast<unsigned>((capacity + kTile - 1) / kTile),
                        static_cast<unsigned>((n + kTile - 1) / kTile));
        k_normalize_raw<D><<<grid, dim3(kTile, 8), 0, stream>>>(d, block, loc, scale, dead,
                                                                layout.df < 0.0 ? 1 : 0, capacity, out);
        FB_LAUNCH_CHECK();
    });
    FB_CUDA(cudaStreamSynchronize(stream));
}

} // namespace fb::rfi
