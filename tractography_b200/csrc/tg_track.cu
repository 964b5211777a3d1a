/*
 * tg_track.cu -- streamline tracking kernels for sm_100a.
 *
 * Two forms of the reference's `tractogram` kernel (tracking.py:93-149):
 *
 *   track_dense_kernel       one thread per seed, dense (n, n_steps, float4)
 *                            output exactly as the reference lays it out.
 *                            This is the plain one-launch-per-batch form.
 *
 *   track_persistent_kernel  a grid sized to the GPU (blocks-per-SM x 148)
 *                            whose lanes pull seeds from a device counter and
 *                            refill as soon as their streamline terminates,
 *                            so a warp never idles behind its longest
 *                            streamline.  Points go to a pool of 32-point
 *                            chunks linked per streamline; gather_kernel
 *                            packs them into one (total_points, 3) array.
 *                            Memory scales with the points produced, not with
 *                            n_seeds x n_steps.
 *
 * Both run the identical per-step arithmetic of tg_device.cuh.  Field
 * coefficients of the current voxel stay in registers and are reloaded only
 * when the nearest voxel changes (every ~10 steps at a 0.1-voxel step,
 * every ~1250 steps at 0.001 mm in 1.25 mm voxels).
 */
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include "tg_internal.h"
#include "tg_step.cuh"

namespace tg {

// ------------------------------------------------------------------ dense

template <int MODEL, int LMAX, int ALGO, int DOM>
__global__ void __launch_bounds__(128) track_dense_kernel(TrackParams p, const float4* __restrict__ seeds,
                                                          uint32_t n_seeds, uint32_t rng_seed,
                                                          uint64_t seed_offset, float4* __restrict__ out,
                                                          uint32_t* __restrict__ lengths)
{
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n_seeds) return;
    Lane s;
    const float4 a = seeds[2 * (size_t)gid];
    const float4 b = seeds[2 * (size_t)gid + 1];
    lane_init(s, a, b, rng_seed, gid, seed_offset + gid);
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;
    float4* line = out + (size_t)gid * p.n_steps;
    line[0] = a;
    while (s.n < p.n_steps && s.steps < p.max_steps) {
        float qx, qy, qz;
        const int r = track_step<MODEL, LMAX, ALGO, CPAD, DOM>(p, s, c, qx, qy, qz);
        if (r == 0) break;
        if (r == 2) {
            line[s.n] = make_float4(qx, qy, qz, 1.0f);
            s.n++;
        }
    }
    lengths[gid] = s.n;
}

// ------------------------------------------------------------- persistent

__device__ __forceinline__ bool chunk_alloc(const PersistentParams& pp, int32_t& chunk)
{
    const unsigned int nc = atomicAdd(pp.chunk_counter, 1u);
    if (nc >= pp.n_chunks) return false;
    pp.chunk_next[nc] = -1;
    chunk = (int32_t)nc;
    return true;
}

__device__ __forceinline__ bool emit_point(const PersistentParams& pp, int32_t& chunk, uint32_t& fill,
                                           float x, float y, float z)
{
    if (fill == (uint32_t)kChunkPoints) {
        int32_t nc;
        if (!chunk_alloc(pp, nc)) return false;
        pp.chunk_next[chunk] = nc;
        chunk = nc;
        fill = 0;
    }
    float* q = pp.pool + ((size_t)chunk * kChunkPoints + fill) * 3;
    q[0] = x;
    q[1] = y;
    q[2] = z;
    fill++;
    return true;
}

// ------------------------------------------------------------ time slicing

constexpr uint32_t kRingWaitLimit = 1u << 22;   // polls of a slot (64 ns apart) before a wait gives up
constexpr uint32_t kRingClaimLimit = 1u << 20;  // lost claim races before a claim gives up
constexpr uint32_t kRingTicketLimit = 0xF0000000u;

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Polls *p until it equals want, 64 ns apart, at most kRingWaitLimit times;
// false (and the ring's fault word set) when the limit is reached.
__device__ __forceinline__ bool ring_wait(const TrackRing& R, const uint32_t* p, uint32_t want)
{
    for (uint32_t k = 0; k < kRingWaitLimit; ++k) {
        if (ld_acquire(p) == want) return true;
        __nanosleep(64);
    }
    atomicOr(R.ctl + 2, 1u);
    return false;
}

// Other work waiting: seeds left in the launch's queue, or saved
// streamlines in the ring (tickets reserved and not yet claimed).
__device__ __forceinline__ bool work_waiting(const PersistentParams& pp, unsigned long long n_items)
{
    const unsigned long long next = *reinterpret_cast<volatile const unsigned long long*>(pp.item_counter);
    if (next < n_items) return true;
    const uint32_t head = ld_relaxed(pp.ring.ctl);
    const uint32_t tail = ld_relaxed(pp.ring.ctl + 1);
    return head < tail && tail < kRingTicketLimit;
}

// Saves the lane's streamline at the ring's tail.  The slot's previous
// ticket was claimed capacity tickets ago; the wait is for its reader to
// have finished.
template <bool RNG>
__device__ __forceinline__ void ring_push(const TrackRing& R, const Lane& s, uint32_t item, int32_t chunk,
                                          uint32_t fill)
{
    const uint32_t t = atomicAdd(R.ctl + 1, 1u);
    const uint32_t slot = t % R.capacity;
    if (t >= R.capacity && !ring_wait(R, R.released + slot, t - R.capacity + 1u)) return;
    LaneCarry c;
    lane_save<RNG>(&c, s, item, chunk, fill);
    const uint4* src = reinterpret_cast<const uint4*>(&c);
    uint4* dst = reinterpret_cast<uint4*>(R.items + slot);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(LaneCarry) / 16); ++k) __stcg(dst + k, src[k]);
    st_release(R.seq + slot, t + 1u);
}

// Claims the ring's oldest saved streamline into the lane; false when the
// ring holds none.  A ticket is claimed only below the tail, so its writer
// has reserved it and is at most a few stores from publishing it.  With at
// least `lanes` tickets between head and tail a plain increment of the head
// cannot pass the tail (each lane has at most one claim in flight); with
// fewer, the claim is a compare-and-swap that fails when another lane got
// the ticket first.  (Compare-and-swap alone serialises the claims of
// thousands of lanes, one success per round trip.)
template <bool RNG>
__device__ __forceinline__ bool ring_take(const TrackRing& R, Lane& s, uint32_t& item, int32_t& chunk,
                                          uint32_t& fill)
{
    uint32_t h = 0;
    bool claimed = false;
    for (uint32_t k = 0; k < kRingClaimLimit && !claimed; ++k) {
        h = ld_relaxed(R.ctl);
        const uint32_t tail = ld_relaxed(R.ctl + 1);
        if (h >= tail) return false;
        if (tail - h >= R.lanes) {
            h = atomicAdd(R.ctl, 1u);
            claimed = true;
        } else {
            claimed = atomicCAS(R.ctl, h, h + 1u) == h;
        }
    }
    if (!claimed) {
        atomicOr(R.ctl + 2, 2u);
        return false;
    }
    const uint32_t slot = h % R.capacity;
    if (!ring_wait(R, R.seq + slot, h + 1u)) return false;
    LaneCarry c;
    const uint4* src = reinterpret_cast<const uint4*>(R.items + slot);
    uint4* dst = reinterpret_cast<uint4*>(&c);
#pragma unroll
    for (int k = 0; k < (int)(sizeof(LaneCarry) / 16); ++k) dst[k] = __ldcg(src + k);
    st_release(R.released + slot, h + 1u);
    lane_restore<RNG>(s, c, item, chunk, fill);
    return true;
}

// SLICE: compiled with time slicing (pp.ring set) or without, so that the
// plain form keeps its registers.
template <int MODEL, int LMAX, int ALGO, int DOM, bool SLICE>
__global__ void __launch_bounds__(128, (persistent_min_blocks<MODEL, LMAX, DOM>())) track_persistent_kernel(
    const PersistentParams pp)
{
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    const TrackParams& p = pp.t;
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;

    Lane s;
    int32_t chunk = -1;
    uint32_t fill = 0;
    uint32_t item = 0;
    bool live = false;
    unsigned long long steps_total = 0;

    const unsigned long long n_items = pp.carry_in != nullptr ? *pp.carry_in_count : pp.n_items;

    // Pull the next seed (or carried streamline); false when the queue is drained.
    auto fetch = [&]() -> bool {
        while (true) {
            if (SLICE &&
                *reinterpret_cast<volatile const unsigned long long*>(pp.item_counter) >= n_items)
                return ring_take<ALGO != kTransport>(pp.ring, s, item, chunk, fill);
            const unsigned long long it = atomicAdd(pp.item_counter, 1ull);
            if (it >= n_items) return SLICE && ring_take<ALGO != kTransport>(pp.ring, s, item, chunk, fill);
            if (pp.carry_in != nullptr) {
                lane_restore<ALGO != kTransport>(s, pp.carry_in[it], item, chunk, fill);
                return true;
            }
            item = pp.item_ids != nullptr ? pp.item_ids[it] : (uint32_t)it;
            const float4 a = pp.seeds[2 * (size_t)item];
            const float4 b = pp.seeds[2 * (size_t)item + 1];
            const uint32_t batch = item / pp.batch_size;
            const uint32_t local = item - batch * pp.batch_size;
            lane_init(s, a, b, pp.batch_rng_seeds[batch], local, pp.seed_offset + item);
            if (DOM == kDomainMesh && pp.seed_inside != nullptr) s.seed_state = pp.seed_inside[item] ? 1u : 2u;
            if (!chunk_alloc(pp, chunk)) {
                pp.first_chunk[item] = -1;
                pp.lengths[item] = kOverflowBit;
                continue;
            }
            pp.first_chunk[item] = chunk;
            fill = 0;
            emit_point(pp, chunk, fill, a.x, a.y, a.z);
            return true;
        }
    };

    live = fetch();
    while (true) {
        const unsigned active = __ballot_sync(0xffffffffu, live);
        if (active == 0u) break;
        if (pp.carry_out != nullptr && warp_should_compact(active, pp.compact_lanes)) {
            if (live)
                lane_save<ALGO != kTransport>(pp.carry_out + atomicAdd(pp.carry_out_count, 1u), s, item, chunk,
                                              fill);
            break;
        }
        // Closed surface: the segment tests of this iteration, done here while
        // the warp is together, so that leaf-list tests are shared out over
        // all its lanes (warp_leaves_hit); same answers as a test per lane.
        int surface = -1;
        if constexpr (DOM == kDomainMesh) {
            const bool testing = live && s.n < p.n_steps && s.steps < p.max_steps && s.steps > 0u;
            uint32_t list = 0;
            int route = 0;
            Segment g;
            g.sx = g.sy = g.sz = g.dx = g.dy = g.dz = g.ix = g.iy = g.iz = 0.0f;
            g.px = g.py = g.pz = false;
            if (testing) {
                route = mesh_route(p.mesh, s.lx, s.ly, s.lz, s.px, s.py, s.pz, list);
                if (route == 1) g = make_segment(s.lx, s.ly, s.lz, s.px, s.py, s.pz);
            }
            bool hit = false;
            if (__any_sync(0xffffffffu, route == 1)) hit = warp_leaves_hit(p.mesh, route == 1, g, list);
            if (testing) surface = route == 0 ? 0 : (route == 1 ? (hit ? 1 : 0) : -1);
        }
        bool refill = false;
        bool slice_end = false;
        if (live) {
            bool done = s.n >= p.n_steps || s.steps >= p.max_steps;
            bool overflow = false;
            if (!done) {
                float qx, qy, qz;
                const int r = track_step<MODEL, LMAX, ALGO, CPAD, DOM>(p, s, c, qx, qy, qz, surface);
                if (r == 0) {
                    done = true;
                } else if (r == 2) {
                    if (emit_point(pp, chunk, fill, qx, qy, qz)) {
                        s.n++;
                        // a slice ends on a saved point: no test on the other steps
                        if (SLICE && (s.n & pp.slice_mask) == 0u) slice_end = true;
                    } else {
                        done = true;
                        overflow = true;
                    }
                }
            }
            if (done) {
                pp.lengths[item] = overflow ? (s.n | kOverflowBit) : s.n;
                if (!overflow) steps_total += s.steps;
                refill = true;
            } else if (SLICE && slice_end && work_waiting(pp, n_items)) {
                ring_push<ALGO != kTransport>(pp.ring, s, item, chunk, fill);
                refill = true;
            }
        }
        // Time slicing: the warp's saved streamlines are all published
        // before any of its lanes waits for a claimed one, so a lane never
        // waits on a lane of its own warp.
        if (SLICE) __syncwarp();
        if (refill) live = fetch();
    }
    if (pp.steps_done != nullptr && steps_total != 0) atomicAdd(pp.steps_done, steps_total);
}

// ----------------------------------------------------------------- gather

__global__ void __launch_bounds__(256) gather_kernel(const float* __restrict__ pool,
                                                     const int32_t* __restrict__ chunk_next,
                                                     const int32_t* __restrict__ first_chunk,
                                                     const uint32_t* __restrict__ lengths,
                                                     const uint64_t* __restrict__ offsets,
                                                     const uint32_t* __restrict__ seed_ids, uint32_t n_ids,
                                                     float* __restrict__ out)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k = warp; k < n_ids; k += n_warps) {
        const uint32_t seed = seed_ids != nullptr ? seed_ids[k] : k;
        int32_t chunk = first_chunk[seed];
        const uint32_t len = lengths[seed];
        const uint64_t off = offsets[seed];
        for (uint32_t base = 0; base < len && chunk >= 0; base += kChunkPoints) {
            const uint32_t j = base + lane;
            if (j < len) {
                const float* src = pool + ((size_t)chunk * kChunkPoints + lane) * 3;
                float* dst = out + (off + j) * 3;
                dst[0] = src[0];
                dst[1] = src[1];
                dst[2] = src[2];
            }
            chunk = chunk_next[chunk];
        }
    }
}

// --------------------------------------------------------------- dispatch

template <template <int, int, int, int> class Fn, typename... Args>
cudaError_t dispatch(int model, int lmax, int algo, int dom, Args&&... args)
{
#define TG_CASE(M, L, A)                                                                     \
    if (model == M && (M == kModelDTI || lmax == L) && algo == A)                            \
        return dom == kDomainMesh ? Fn<M, L, A, kDomainMesh>::run(args...)                   \
                                  : Fn<M, L, A, kDomainImage>::run(args...);
    TG_CASE(kModelSH, 0, kTransport) TG_CASE(kModelSH, 0, kDiffusion)
    TG_CASE(kModelSH, 2, kTransport) TG_CASE(kModelSH, 2, kDiffusion)
    TG_CASE(kModelSH, 4, kTransport) TG_CASE(kModelSH, 4, kDiffusion)
    TG_CASE(kModelSH, 6, kTransport) TG_CASE(kModelSH, 6, kDiffusion)
    TG_CASE(kModelSH, 8, kTransport) TG_CASE(kModelSH, 8, kDiffusion)
    TG_CASE(kModelDTI, 0, kTransport) TG_CASE(kModelDTI, 0, kDiffusion)
#undef TG_CASE
    return cudaErrorInvalidValue;
}

template <int M, int L, int A, int D>
struct DenseLaunch {
    static cudaError_t run(const TrackParams& p, const float4* seeds, uint32_t n, uint32_t rng_seed,
                           uint64_t seed_offset, float4* out, uint32_t* lengths, cudaStream_t stream)
    {
        const int block = 128;
        const int grid = (int)((n + block - 1) / block);
        track_dense_kernel<M, L, A, D><<<grid, block, 0, stream>>>(p, seeds, n, rng_seed, seed_offset, out, lengths);
        return cudaGetLastError();
    }
};

template <int M, int L, int A, int D>
struct PersistentLaunch {
    static cudaError_t run(const PersistentParams& p, int grid, int block, cudaStream_t stream)
    {
        if (p.ring.items != nullptr)
            track_persistent_kernel<M, L, A, D, true><<<grid, block, 0, stream>>>(p);
        else
            track_persistent_kernel<M, L, A, D, false><<<grid, block, 0, stream>>>(p);
        return cudaGetLastError();
    }
};

template <int M, int L, int A, int D>
struct PersistentOccupancy {
    static cudaError_t run(int* blocks)
    {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, track_persistent_kernel<M, L, A, D, true>,
                                                             persistent_block_size(), 0);
    }
};

int lmax_for(uint32_t n_params)
{
    int l = 0;
    while ((uint32_t)n_coef_full(l) < n_params) l += 2;
    return l;
}

int persistent_block_size() { return 128; }

int persistent_blocks_per_sm(const FieldDev& f, int algorithm, int domain_kind)
{
    int blocks = 0;
    if (dispatch<PersistentOccupancy>(f.model, f.lmax, algorithm, domain_kind, &blocks) != cudaSuccess ||
        blocks < 1)
        blocks = 1;
    return blocks;
}

cudaError_t launch_track_dense(const FieldDev& f, const TrackParams& p, const float4* seeds,
                               uint32_t n_seeds, uint32_t rng_seed, uint64_t seed_offset, float4* out,
                               uint32_t* lengths, cudaStream_t stream)
{
    if (n_seeds == 0) return cudaSuccess;
    return dispatch<DenseLaunch>(f.model, f.lmax, p.algorithm, p.domain_kind, p, seeds, n_seeds, rng_seed,
                                 seed_offset,
                                 out, lengths, stream);
}

cudaError_t launch_track_persistent(const FieldDev& f, const PersistentParams& p, int grid, int block,
                                    cudaStream_t stream)
{
    if (p.n_items == 0) return cudaSuccess;
    return dispatch<PersistentLaunch>(f.model, f.lmax, p.t.algorithm, p.t.domain_kind, p, grid, block, stream);
}

cudaError_t launch_gather(const float* pool, const int32_t* chunk_next, const int32_t* first_chunk,
                          const uint32_t* lengths, const uint64_t* offsets, const uint32_t* seed_ids,
                          uint32_t n_ids, float* out_points, cudaStream_t stream)
{
    if (n_ids == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int block = 256;
    const uint64_t threads = (uint64_t)n_ids * 32u;
    uint64_t grid = (threads + block - 1) / block;
    if (grid > (uint64_t)sms * 16) grid = (uint64_t)sms * 16;
    gather_kernel<<<(int)grid, block, 0, stream>>>(pool, chunk_next, first_chunk, lengths, offsets, seed_ids,
                                                   n_ids, out_points);
    return cudaGetLastError();
}

// Lengths of streamlines that overflowed the pool count as 0; the count
// of such streamlines goes to totals[1].
__global__ void masked_lengths_kernel(const uint32_t* __restrict__ lengths, uint32_t n, uint64_t* __restrict__ out,
                                      unsigned long long* __restrict__ totals)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool over = i < n && (lengths[i] & kOverflowBit) != 0u;
    if (i < n) out[i] = over ? 0ull : (uint64_t)lengths[i];
    const unsigned b = __ballot_sync(0xffffffffu, over);
    if ((threadIdx.x & 31u) == 0u && b != 0u) atomicAdd(totals + 1, (unsigned long long)__popc(b));
}

__global__ void offsets_total_kernel(const uint64_t* __restrict__ masked, const uint64_t* __restrict__ offsets,
                                     uint32_t n, unsigned long long* __restrict__ totals)
{
    totals[0] = offsets[n - 1] + masked[n - 1];
}

cudaError_t launch_offsets(const uint32_t* lengths, uint32_t n, uint64_t* masked, uint64_t* offsets,
                           unsigned long long* totals, void* temp, size_t* temp_bytes, cudaStream_t stream)
{
    if (temp == nullptr) return cub::DeviceScan::ExclusiveSum(nullptr, *temp_bytes, masked, offsets, (int)n, stream);
    cudaError_t e = cudaMemsetAsync(totals, 0, 2 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess || n == 0) return e;
    masked_lengths_kernel<<<(n + 255) / 256, 256, 0, stream>>>(lengths, n, masked, totals);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(temp, *temp_bytes, masked, offsets, (int)n, stream);
    if (e != cudaSuccess) return e;
    offsets_total_kernel<<<1, 1, 0, stream>>>(masked, offsets, n, totals);
    return cudaGetLastError();
}

}  // namespace tg
