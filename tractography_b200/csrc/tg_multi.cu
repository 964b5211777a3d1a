/*
 * tg_multi.cu -- many tracking jobs in one persistent launch.
 *
 * A job is one reference `tracking.tractogram` call (its own field, domain,
 * algorithm parameters, seeds and RNG seeds).  All jobs of a request mix are
 * queued at once: each class of jobs with the same compiled code path
 * (model, lmax, algorithm) has a device queue of seeds drained by its own
 * persistent launch, all classes launched together on concurrent streams;
 * lanes pull seeds from their class queue and refill as their streamlines
 * terminate.  Lanes of a warp never diverge across code paths, small
 * jobs share the GPU with large ones, and no job waits for another job's
 * longest streamline.  Per-lane job parameters are read from the job table
 * when a lane takes a new seed.  Output goes to the tracker's chunk pool
 * exactly as the single-job persistent kernel's does.
 */
#include <cuda_runtime.h>

#include "tg_step.cuh"

namespace tg {

int class_kind(int model, int lmax, int algorithm)
{
    if (model == kModelDTI) return algorithm == kTransport ? kDTIT : kDTID;
    const int base = (lmax / 2) * 2;   // kSH0T, kSH2T, ... are consecutive pairs
    return base + (algorithm == kTransport ? 0 : 1);
}

namespace {

__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t* a, uint32_t n, uint32_t v)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool m_chunk_alloc(const MultiParams& mp, int32_t& chunk)
{
    const unsigned int nc = atomicAdd(mp.chunk_counter, 1u);
    if (nc >= mp.n_chunks) return false;
    mp.chunk_next[nc] = -1;
    chunk = (int32_t)nc;
    return true;
}

__device__ __forceinline__ bool m_emit(const MultiParams& mp, int32_t& chunk, uint32_t& fill, float x, float y,
                                       float z)
{
    if (fill == (uint32_t)kChunkPoints) {
        int32_t nc;
        if (!m_chunk_alloc(mp, nc)) return false;
        mp.chunk_next[chunk] = nc;
        chunk = nc;
        fill = 0;
    }
    float* q = mp.pool + ((size_t)chunk * kChunkPoints + fill) * 3;
    q[0] = x;
    q[1] = y;
    q[2] = z;
    fill++;
    return true;
}

// Drain one class: lanes take seeds from the class queue until it is empty.
// Tracking parameters of the first kSharedJobs jobs of a class are staged in
// shared memory at kernel start: every step reads ~25 of them (affine rows,
// step and noise scales, limits), and lanes of one warp usually follow
// several jobs, which in the job table in global memory costs one L1
// wavefront per distinct job per load.
constexpr int kSharedJobs = 48;

template <int MODEL, int LMAX, int ALGO>
__device__ __forceinline__ unsigned long long drain_class(const MultiParams& mp, const ClassDev& cls,
                                                          const TrackParams* shared_t, uint32_t n_shared)
{
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;
    unsigned long long steps_total = 0;
    const JobDev* J = nullptr;
    const TrackParams* P = nullptr;
    Lane s;
    int32_t chunk = -1;
    uint32_t fill = 0;
    uint32_t g = 0;

    const unsigned long long n_items = mp.carry_in != nullptr ? *mp.carry_in_count : cls.n_items;

    auto fetch = [&]() -> bool {
        while (true) {
            const unsigned long long k = atomicAdd(cls.counter, 1ull);
            if (k >= n_items) return false;
            if (mp.carry_in != nullptr) {
                lane_restore<ALGO != kTransport>(s, mp.carry_in[k], g, chunk, fill);
                J = mp.jobs + (upper_bound_u32(mp.job_base, mp.n_jobs + 1, g) - 1);
                P = &J->t;
                return true;
            }
            uint32_t job, i;
            if (cls.item_ids != nullptr) {
                g = cls.item_ids[k];
                job = upper_bound_u32(mp.job_base, mp.n_jobs + 1, g) - 1;
                i = g - mp.job_base[job];
                J = mp.jobs + job;
                P = &J->t;
            } else {
                const uint32_t q = upper_bound_u32(cls.prefix, cls.n_jobs + 1, (uint32_t)k) - 1;
                job = cls.jobs[q];
                i = (uint32_t)k - cls.prefix[q];
                g = mp.job_base[job] + i;
                J = mp.jobs + job;
                P = q < n_shared ? shared_t + q : &J->t;
            }
            const float4 a = J->seeds[2 * (size_t)i];
            const float4 b = J->seeds[2 * (size_t)i + 1];
            const uint32_t batch = i / J->batch_size;
            lane_init(s, a, b, mp.batch_rng_seeds[J->rng_base + batch], i - batch * J->batch_size,
                      J->seed_offset + i);
            if (!m_chunk_alloc(mp, chunk)) {
                mp.first_chunk[g] = -1;
                mp.lengths[g] = kOverflowBit;
                continue;
            }
            mp.first_chunk[g] = chunk;
            fill = 0;
            m_emit(mp, chunk, fill, a.x, a.y, a.z);
            return true;
        }
    };

    bool live = fetch();
    while (true) {
        const unsigned active = __ballot_sync(0xffffffffu, live);
        if (active == 0u) break;
        if (mp.carry_out != nullptr && warp_should_compact(active, mp.compact_lanes)) {
            if (live)
                lane_save<ALGO != kTransport>(mp.carry_out + atomicAdd(mp.carry_out_count, 1u), s, g, chunk, fill);
            break;
        }
        if (!live) continue;
        bool done = s.n >= P->n_steps || s.steps >= P->max_steps;
        bool overflow = false;
        if (!done) {
            float qx, qy, qz;
            const int r = track_step<MODEL, LMAX, ALGO, CPAD>(*P, s, c, qx, qy, qz);
            if (r == 0) {
                done = true;
            } else if (r == 2) {
                if (m_emit(mp, chunk, fill, qx, qy, qz)) {
                    s.n++;
                } else {
                    done = true;
                    overflow = true;
                }
            }
        }
        if (done) {
            mp.lengths[g] = overflow ? (s.n | kOverflowBit) : s.n;
            if (!overflow) steps_total += s.steps;
            live = fetch();
        }
    }
    return steps_total;
}

template <int MODEL, int LMAX, int ALGO>
__global__ void __launch_bounds__(128, 5) track_class_kernel(const MultiParams mp, const ClassDev cls)
{
    extern __shared__ uint4 shared_raw[];
    TrackParams* table = reinterpret_cast<TrackParams*>(shared_raw);
    const uint32_t n_shared = cls.n_jobs < (uint32_t)kSharedJobs ? cls.n_jobs : (uint32_t)kSharedJobs;
    constexpr uint32_t kWords = sizeof(TrackParams) / sizeof(uint32_t);
    static_assert(sizeof(TrackParams) % sizeof(uint32_t) == 0, "TrackParams is copied as words");
    for (uint32_t w = threadIdx.x; w < n_shared * kWords; w += blockDim.x) {
        const uint32_t q = w / kWords, o = w - q * kWords;
        reinterpret_cast<uint32_t*>(table + q)[o] =
            reinterpret_cast<const uint32_t*>(&mp.jobs[cls.jobs[q]].t)[o];
    }
    __syncthreads();
    const unsigned long long steps = drain_class<MODEL, LMAX, ALGO>(mp, cls, table, n_shared);
    if (steps != 0) atomicAdd(mp.steps_done, steps);
}

size_t class_shared_bytes(uint32_t n_jobs)
{
    const uint32_t n = n_jobs < (uint32_t)kSharedJobs ? n_jobs : (uint32_t)kSharedJobs;
    return (size_t)n * sizeof(TrackParams);
}

template <int M, int L, int A>
struct ClassLaunch {
    static cudaError_t run(const MultiParams& mp, const ClassDev& cls, int grid, cudaStream_t stream)
    {
        track_class_kernel<M, L, A><<<grid, 128, class_shared_bytes(cls.n_jobs), stream>>>(mp, cls);
        return cudaGetLastError();
    }
};

template <int M, int L, int A>
struct ClassOccupancy {
    static cudaError_t run(int* blocks)
    {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, track_class_kernel<M, L, A>, 128,
                                                             class_shared_bytes(kSharedJobs));
    }
};

template <template <int, int, int> class Fn, typename... Args>
cudaError_t class_dispatch(int kind, Args&&... args)
{
    switch (kind) {
    case kSH0T: return Fn<kModelSH, 0, kTransport>::run(args...);
    case kSH0D: return Fn<kModelSH, 0, kDiffusion>::run(args...);
    case kSH2T: return Fn<kModelSH, 2, kTransport>::run(args...);
    case kSH2D: return Fn<kModelSH, 2, kDiffusion>::run(args...);
    case kSH4T: return Fn<kModelSH, 4, kTransport>::run(args...);
    case kSH4D: return Fn<kModelSH, 4, kDiffusion>::run(args...);
    case kSH6T: return Fn<kModelSH, 6, kTransport>::run(args...);
    case kSH6D: return Fn<kModelSH, 6, kDiffusion>::run(args...);
    case kSH8T: return Fn<kModelSH, 8, kTransport>::run(args...);
    case kSH8D: return Fn<kModelSH, 8, kDiffusion>::run(args...);
    case kDTIT: return Fn<kModelDTI, 0, kTransport>::run(args...);
    case kDTID: return Fn<kModelDTI, 0, kDiffusion>::run(args...);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int class_blocks_per_sm(int kind)
{
    int blocks = 0;
    if (class_dispatch<ClassOccupancy>(kind, &blocks) != cudaSuccess || blocks < 1) blocks = 1;
    return blocks;
}

cudaError_t launch_track_class(const MultiParams& mp, const ClassDev& cls, int grid, cudaStream_t s)
{
    if (cls.n_items == 0) return cudaSuccess;
    return class_dispatch<ClassLaunch>(cls.kind, mp, cls, grid, s);
}

}  // namespace tg
