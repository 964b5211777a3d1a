/*
 * tg_noalloc.cu -- tracking without any device allocation by the library.
 *
 * Some callers cannot let a library call cudaMalloc: a host application
 * that owns the GPU's memory budget and hands plugins fixed buffers at start
 * up, or a latency-bound loop in which cudaMalloc/cudaFree (which may
 * synchronise the device) are not acceptable.  For them this file provides
 * tg_tractogram_noalloc(): the persistent lane-refill tracker writing the
 * reference's dense output into caller buffers, whose only scratch memory
 * (a work-item counter and the per-batch RNG seeds) lives
 * in the file-scope __device__ array below.
 *
 * Properties of that array, which every caller shares:
 *   - It is 256 B of counters plus room for kNoAllocMaxBatches batch seeds
 *     (64 KiB + 256 B); it exists on every GPU that loads the library and is
 *     held until the process exits.
 *   - Host code only sees a host-side stand-in for its name.  Its device
 *     address is obtained once per device with cudaGetSymbolAddress, with
 *     that device current, on the first call made on that device; make that
 *     first call before any stream capture.
 *   - Each call clears the counter and overwrites the seeds it uses; the
 *     array otherwise keeps the last call's contents.  The seeds are copied
 *     from the caller's host array on the call's stream: from pageable
 *     memory the call returns once they are copied; from page-locked memory
 *     it may return first, and the host array must then stay unchanged until
 *     the stream has run the copy.  Calls that overlap on
 *     the GPU (different streams, or host threads on one device) race on it:
 *     serialise them.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "tg_step.cuh"
#include "tractography_b200.h"

namespace tg {

// Defined in tg_capi.cu (which owns the tg_domain / tg_field layouts).
int track_params_from_handles(const tg_algorithm* a, const tg_domain* d, const tg_field* f, float save_at,
                              uint32_t n_steps, TrackParams* out, int* model, int* lmax);
int set_last_error(int code, const std::string& msg);

namespace {

constexpr uint32_t kNoAllocHeaderWords = 64;       // 256 B: counters
constexpr uint32_t kNoAllocMaxBatches = TG_NOALLOC_MAX_BATCHES;
constexpr uint32_t kNoAllocWords = kNoAllocHeaderWords + kNoAllocMaxBatches;

// words [0, 2): work-item counter (u64); [2, 64): unused;
// [64, 64 + n_batches): per-batch RNG seeds.
static __device__ __align__(256) uint32_t tg_noalloc_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
uint32_t* g_scratch_addr[kMaxDevices] = {};

template <int MODEL, int LMAX, int ALGO>
__global__ void __launch_bounds__(128) track_persistent_dense_kernel(TrackParams p, const float4* __restrict__ seeds,
                                                                     uint32_t n_seeds, uint32_t batch_size,
                                                                     uint64_t seed_offset, uint32_t* scratch,
                                                                     float4* __restrict__ out,
                                                                     uint32_t* __restrict__ lengths)
{
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    unsigned long long* item_counter = reinterpret_cast<unsigned long long*>(scratch);
    const uint32_t* batch_seeds = scratch + kNoAllocHeaderWords;
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;
    while (true) {
        const unsigned long long it = atomicAdd(item_counter, 1ull);
        if (it >= n_seeds) break;
        const uint32_t item = (uint32_t)it;
        const uint32_t batch = item / batch_size;
        const uint32_t local = item - batch * batch_size;
        const float4 a = seeds[2 * (size_t)item];
        const float4 b = seeds[2 * (size_t)item + 1];
        Lane s;
        lane_init(s, a, b, batch_seeds[batch], local, seed_offset + item);
        float4* line = out + (size_t)item * p.n_steps;
        line[0] = a;
        while (s.n < p.n_steps && s.steps < p.max_steps) {
            float qx, qy, qz;
            const int r = track_step<MODEL, LMAX, ALGO, CPAD>(p, s, c, qx, qy, qz);
            if (r == 0) break;
            if (r == 2) {
                line[s.n] = make_float4(qx, qy, qz, 1.0f);
                s.n++;
            }
        }
        lengths[item] = s.n;
    }
}

template <int M, int L, int A>
cudaError_t launch_variant(const TrackParams& p, const float4* seeds, uint32_t n, uint32_t batch_size,
                           uint64_t seed_offset, uint32_t* scratch, float4* out, uint32_t* lengths,
                           cudaStream_t stream)
{
    int dev = 0, sms = 0, blocks = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, track_persistent_dense_kernel<M, L, A>, 128, 0);
    if (e != cudaSuccess) return e;
    const int grid = (sms > 0 ? sms : 1) * (blocks > 0 ? blocks : 1);
    track_persistent_dense_kernel<M, L, A><<<grid, 128, 0, stream>>>(p, seeds, n, batch_size, seed_offset, scratch,
                                                                      out, lengths);
    return cudaGetLastError();
}

cudaError_t launch(int model, int lmax, int algo, const TrackParams& p, const float4* seeds, uint32_t n,
                   uint32_t batch_size, uint64_t seed_offset, uint32_t* scratch, float4* out, uint32_t* lengths,
                   cudaStream_t s)
{
#define TG_NA_CASE(M, L, A)                                                                      \
    if (model == M && (M == kModelDTI || lmax == L) && algo == A)                                \
        return launch_variant<M, L, A>(p, seeds, n, batch_size, seed_offset, scratch, out, lengths, s);
    TG_NA_CASE(kModelSH, 0, kTransport) TG_NA_CASE(kModelSH, 0, kDiffusion)
    TG_NA_CASE(kModelSH, 2, kTransport) TG_NA_CASE(kModelSH, 2, kDiffusion)
    TG_NA_CASE(kModelSH, 4, kTransport) TG_NA_CASE(kModelSH, 4, kDiffusion)
    TG_NA_CASE(kModelSH, 6, kTransport) TG_NA_CASE(kModelSH, 6, kDiffusion)
    TG_NA_CASE(kModelSH, 8, kTransport) TG_NA_CASE(kModelSH, 8, kDiffusion)
    TG_NA_CASE(kModelDTI, 0, kTransport) TG_NA_CASE(kModelDTI, 0, kDiffusion)
#undef TG_NA_CASE
    return cudaErrorInvalidValue;
}

int fail(int code, const std::string& msg) { return set_last_error(code, msg); }

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int scratch_address(uint32_t** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(TG_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        uint32_t* ptr = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), tg_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            return fail(TG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = ptr;
    }
    *out = g_scratch_addr[dev];
    return TG_OK;
}

}  // namespace
}  // namespace tg

extern "C" int tg_tractogram_noalloc(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                                     const float* seeds, uint32_t n_seeds, uint32_t batch_size,
                                     const uint32_t* batch_rng_seeds, float save_at, uint32_t n_steps,
                                     float* streamlines, uint32_t* lengths, void* stream)
{
    using namespace tg;
    TrackParams p;
    int model = 0, lmax = 0;
    int st = track_params_from_handles(algorithm, domain, field, save_at, n_steps, &p, &model, &lmax);
    if (st != TG_OK) return st;
    if (p.domain_kind != kDomainImage) return fail(TG_ERR_UNSUPPORTED, "tg_tractogram_noalloc takes image domains");
    if (n_seeds == 0) return TG_OK;
    if (n_steps == 0) return fail(TG_ERR_INVALID_ARGUMENT, "n_steps must be positive");
    if (batch_size == 0) return fail(TG_ERR_INVALID_ARGUMENT, "batch_size must be positive");
    if (seeds == nullptr || streamlines == nullptr || lengths == nullptr || batch_rng_seeds == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null buffer");
    const uint64_t n_batches = ((uint64_t)n_seeds + batch_size - 1) / batch_size;
    if (n_batches > kNoAllocMaxBatches)
        return fail(TG_ERR_INVALID_ARGUMENT,
                    "tg_tractogram_noalloc: " + std::to_string(n_batches) + " batches exceed the maximum of " +
                        std::to_string(kNoAllocMaxBatches) + " (raise batch_size or split the call)");
    uint32_t* scratch = nullptr;
    st = scratch_address(&scratch);
    if (st != TG_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(scratch, 0, kNoAllocHeaderWords * sizeof(uint32_t), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scratch + kNoAllocHeaderWords, batch_rng_seeds, n_batches * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch(model, lmax, algorithm->algorithm, p, reinterpret_cast<const float4*>(seeds), n_seeds, batch_size,
                   algorithm->seed_offset, scratch, reinterpret_cast<float4*>(streamlines), lengths, s);
    if (e != cudaSuccess) return fail(TG_ERR_CUDA, std::string("tg_tractogram_noalloc: ") + cudaGetErrorString(e));
    return TG_OK;
}
