/*
 * tg_serve.cu -- continuous-batching tracking server (tg_server_*).
 *
 * No reference counterpart: the reference runs one tg.tractogram call at a
 * time.  The server keeps fields, domains and surfaces resident (they are
 * ordinary tg_field / tg_domain handles) and runs admitted requests in
 * epochs:
 *
 *   - every request is one reference tg.tractogram job (tg_job); its seeds
 *     join the FIFO queue of its code path (model, lmax, algorithm, domain
 *     kind);
 *   - an epoch launches one persistent kernel per code path with work, on
 *     concurrent streams.  Lanes first resume the streamlines carried over
 *     from the previous epoch, then take new seeds from the queue; every lane
 *     executes at most `epoch_steps` loop iterations and, when an epoch time
 *     is set, stops at the epoch's deadline on the device clock (so code
 *     paths with costlier steps, e.g. closed-surface domains, end with the
 *     rest instead of holding the GPU), after which a live streamline is
 *     saved (position, orientation, RNG state, output cursor) and resumed in
 *     the next epoch.  Requests that arrive while others run
 *     enter at the next epoch, so a small request never waits for the tail
 *     of a large one, and lanes freed by finished streamlines are refilled
 *     from any request of the same code path;
 *   - output points go to a chunk pool shared by all requests; chunks come
 *     from a free list.  After every epoch the streamlines that finished in
 *     it are harvested: their points move to their request's result buffer
 *     and their chunks return to the free list, so the pool only ever holds
 *     streamlines in flight;
 *   - a request is admitted when a job slot is free and its buffers fit in
 *     the HBM budget next to the resident objects and the pool; the rest
 *     wait on the host in arrival order;
 *   - a streamline starts only after reserving its worst-case number of
 *     chunks (ceil(n_steps / 32)) against the pool; a seed that finds no room
 *     is carried, unstarted, to the next epoch, and unused reservations and
 *     freed chunks are given back, so an allocation never fails and every
 *     streamline that starts finishes (the overflow re-queue path remains as
 *     a safety net).
 *
 * A streamline's arithmetic depends only on its seed, its batch's RNG seed
 * and its index in the batch, so every request's result is identical to the
 * same job tracked alone (tg_tracker_run), whatever else is in the mix.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <string>
#include <unordered_map>
#include <vector>

#include <cub/cub.cuh>

#include "tg_internal.h"
#include "tg_step.cuh"
#include "tractography_b200.h"

namespace tg {

int set_last_error(int code, const std::string& msg);
int track_params_from_handles(const tg_algorithm* a, const tg_domain* d, const tg_field* f, float save_at,
                              uint32_t n_steps, TrackParams* out, int* model, int* lmax);

namespace {

constexpr int kServeKinds = 2 * kClassKinds;     // code path x domain kind

struct ServeJob {
    TrackParams t;
    const float4* seeds;
    uint32_t n_seeds;
    uint32_t batch_size;
    const uint32_t* batch_rng_seeds;
    uint64_t seed_offset;
    uint32_t* lengths;
    int32_t* first_chunk;
    const uint8_t* seed_inside; // closed surface: the seeds' inside tests, done at admission; nullable
    unsigned int* counts;       // [0] streamlines in flight, [1] overflowed
    uint32_t chunks_needed;     // worst case per streamline: ceil(n_steps / 32)
    unsigned long long* finished_points;   // points of streamlines finished this epoch
    float* result;              // current result segment: (capacity, 3) harvested points
    uint64_t result_first;      // request-wide index of the segment's first point
    uint64_t* result_offset;    // per seed: request-wide index of its first point
    unsigned long long* cursor; // points harvested so far
};

struct Finished {
    uint32_t slot;
    uint32_t item;
};

struct ServePool {
    float* pool;
    int32_t* chunk_next;
    int32_t* free_list;
    unsigned int* alloc;        // [0] free chunks at the list's head, [1] taken this epoch
    // chunks held or reserved: a streamline starts only after reserving its
    // worst case, so an allocation never fails; freed chunks and unused
    // reservations are given back
    unsigned long long* committed;
    uint32_t n_chunks;
};

struct ServeParams {
    const ServeJob* jobs;
    ServePool P;
    const LaneCarry* carry_in;
    uint32_t n_carry;
    LaneCarry* carry_out;
    unsigned int* carry_out_count;
    const uint32_t* seg_slot;
    const uint32_t* seg_start;
    const uint32_t* seg_prefix;  // n_seg + 1
    uint32_t n_seg;
    uint32_t n_new;
    unsigned long long* counter;
    uint32_t step_budget;
    const unsigned long long* deadline;   // epoch end on the device clock (ns); null: steps only
    unsigned long long* steps_done;
    Finished* finished;          // streamlines that finished this epoch
    unsigned int* n_finished;
};

__device__ __forceinline__ unsigned long long device_clock_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The epoch's deadline: now + budget on the device clock.
__global__ void epoch_deadline_kernel(unsigned long long* deadline, unsigned long long budget_ns)
{
    *deadline = device_clock_ns() + budget_ns;
}

__device__ __forceinline__ uint32_t seg_upper_bound(const uint32_t* a, uint32_t n, uint32_t v)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool s_alloc(const ServePool& P, uint32_t avail, int32_t& chunk)
{
    const unsigned int k = atomicAdd(P.alloc + 1, 1u);
    if (k >= avail) return false;
    const int32_t c = P.free_list[avail - 1u - k];
    P.chunk_next[c] = -1;
    chunk = c;
    return true;
}

__device__ __forceinline__ bool s_emit(const ServePool& P, uint32_t avail, int32_t& chunk, uint32_t& fill, float x,
                                       float y, float z)
{
    if (fill == (uint32_t)kChunkPoints) {
        int32_t nc;
        if (!s_alloc(P, avail, nc)) return false;
        P.chunk_next[chunk] = nc;
        chunk = nc;
        fill = 0;
    }
    float* q = P.pool + ((size_t)chunk * kChunkPoints + fill) * 3;
    q[0] = x;
    q[1] = y;
    q[2] = z;
    fill++;
    return true;
}

template <int MODEL, int LMAX, int ALGO, int DOM>
__global__ void __launch_bounds__(128, (persistent_min_blocks<MODEL, LMAX, DOM>())) serve_kernel(const ServeParams sp)
{
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;
    const uint32_t avail = sp.P.alloc[0];
    Lane s;
    s.px = s.py = s.pz = 0.0f;
    const ServeJob* J = nullptr;
    uint32_t slot = 0, item = 0, fill = 0;
    int32_t chunk = -1;
    uint32_t budget = sp.step_budget;
    const unsigned long long deadline = sp.deadline != nullptr ? *sp.deadline : ~0ull;
    unsigned long long steps_total = 0;

    // Reserve the streamline's worst-case chunks, take its first chunk and
    // write the seed point; false when the pool cannot hold it now.
    auto start = [&]() -> bool {
        const unsigned long long W = J->chunks_needed;
        if (atomicAdd(sp.P.committed, W) + W > (unsigned long long)sp.P.n_chunks) {
            atomicAdd(sp.P.committed, (unsigned long long)(-(long long)W));
            return false;
        }
        if (!s_alloc(sp.P, avail, chunk)) {             // cannot happen while reservations hold
            atomicAdd(sp.P.committed, (unsigned long long)(-(long long)W));
            return false;
        }
        J->first_chunk[item] = chunk;
        fill = 0;
        s_emit(sp.P, avail, chunk, fill, s.px, s.py, s.pz);
        return true;
    };

    auto fetch = [&]() -> bool {
        if (budget == 0u) return false;
        const unsigned long long k = atomicAdd(sp.counter, 1ull);
        if (k < sp.n_carry) {
            const LaneCarry& cc = sp.carry_in[k];
            lane_restore<ALGO != kTransport>(s, cc, item, chunk, fill);
            slot = cc.job;
            J = sp.jobs + slot;
        } else {
            const unsigned long long q0 = k - sp.n_carry;
            if (q0 >= sp.n_new) return false;
            const uint32_t q = seg_upper_bound(sp.seg_prefix, sp.n_seg + 1, (uint32_t)q0) - 1;
            slot = sp.seg_slot[q];
            item = sp.seg_start[q] + ((uint32_t)q0 - sp.seg_prefix[q]);
            J = sp.jobs + slot;
            const float4 a = J->seeds[2 * (size_t)item];
            const float4 b = J->seeds[2 * (size_t)item + 1];
            const uint32_t batch = item / J->batch_size;
            lane_init(s, a, b, J->batch_rng_seeds[batch], item - batch * J->batch_size, J->seed_offset + item);
            if (DOM == kDomainMesh && J->seed_inside != nullptr) s.seed_state = J->seed_inside[item] ? 1u : 2u;
            atomicAdd(J->counts, 1u);
            chunk = -1;
        }
        if (chunk < 0 && !start()) {
            // no room in the pool now: hand the unstarted seed to the next epoch
            lane_save<ALGO != kTransport>(sp.carry_out + atomicAdd(sp.carry_out_count, 1u), s, item, -1, 0u, slot);
            return false;
        }
        return true;
    };

    bool live = fetch();
    while (true) {
        const unsigned active = __ballot_sync(0xffffffffu, live);
        if (active == 0u) break;
        // the epoch ends after step_budget iterations or at the deadline,
        // read by lane 0 every 8 iterations (the whole warp stops together);
        // every warp runs at least 8 iterations, so every epoch makes progress
        const uint32_t used = sp.step_budget - budget;
        if (budget != 0u && used != 0u && (used & 7u) == 0u && deadline != ~0ull) {
            unsigned long long now = 0;
            if ((threadIdx.x & 31u) == 0u) now = device_clock_ns();
            if (__shfl_sync(0xffffffffu, now, 0) > deadline) budget = 0u;
        }
        if (budget == 0u) {
            if (live)
                lane_save<ALGO != kTransport>(sp.carry_out + atomicAdd(sp.carry_out_count, 1u), s, item, chunk, fill,
                                              slot);
            break;
        }
        budget -= 1u;
        if (!live) continue;
        bool done = s.n >= J->t.n_steps || s.steps >= J->t.max_steps;
        bool overflow = false;
        if (!done) {
            float qx, qy, qz;
            const int r = track_step<MODEL, LMAX, ALGO, CPAD, DOM>(J->t, s, c, qx, qy, qz);
            if (r == 0) {
                done = true;
            } else if (r == 2) {
                if (s_emit(sp.P, avail, chunk, fill, qx, qy, qz)) {
                    s.n++;
                } else {
                    done = true;
                    overflow = true;
                }
            }
        }
        if (done) {
            J->lengths[item] = overflow ? (s.n | kOverflowBit) : s.n;
            // give back the reservation this streamline will not use (its
            // chunks are given back when they are freed)
            const unsigned long long held = ((unsigned long long)s.n + kChunkPoints - 1) / kChunkPoints;
            const unsigned long long W = J->chunks_needed;
            atomicAdd(sp.P.committed, (unsigned long long)(-(long long)(W > held ? W - held : 0ull)));
            if (overflow) {
                atomicAdd(J->counts + 1, 1u);
            } else {
                steps_total += s.steps;
                sp.finished[atomicAdd(sp.n_finished, 1u)] = Finished{slot, item};
                atomicAdd(J->finished_points, (unsigned long long)s.n);
            }
            atomicSub(J->counts, 1u);
            live = fetch();
        }
    }
    if (steps_total != 0) atomicAdd(sp.steps_done, steps_total);
}

template <int M, int L, int A, int D>
struct ServeLaunch {
    static cudaError_t run(const ServeParams& sp, int grid, cudaStream_t s)
    {
        serve_kernel<M, L, A, D><<<grid, 128, 0, s>>>(sp);
        return cudaGetLastError();
    }
};

template <int M, int L, int A, int D>
struct ServeOccupancy {
    static cudaError_t run(int* blocks)
    {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, serve_kernel<M, L, A, D>, 128, 0);
    }
};

template <template <int, int, int, int> class Fn, typename... Args>
cudaError_t serve_dispatch(int kind, Args&&... args)
{
    const int cls = kind >> 1;
    const bool mesh = (kind & 1) != 0;
#define TG_SERVE(K, M, L, A)                                                                          \
    case K:                                                                                          \
        return mesh ? Fn<M, L, A, kDomainMesh>::run(args...) : Fn<M, L, A, kDomainImage>::run(args...);
    switch (cls) {
        TG_SERVE(kSH0T, kModelSH, 0, kTransport)
        TG_SERVE(kSH0D, kModelSH, 0, kDiffusion)
        TG_SERVE(kSH2T, kModelSH, 2, kTransport)
        TG_SERVE(kSH2D, kModelSH, 2, kDiffusion)
        TG_SERVE(kSH4T, kModelSH, 4, kTransport)
        TG_SERVE(kSH4D, kModelSH, 4, kDiffusion)
        TG_SERVE(kSH6T, kModelSH, 6, kTransport)
        TG_SERVE(kSH6D, kModelSH, 6, kDiffusion)
        TG_SERVE(kSH8T, kModelSH, 8, kTransport)
        TG_SERVE(kSH8D, kModelSH, 8, kDiffusion)
        TG_SERVE(kDTIT, kModelDTI, 0, kTransport)
        TG_SERVE(kDTID, kModelDTI, 0, kDiffusion)
    default:
        return cudaErrorInvalidValue;
    }
#undef TG_SERVE
}

__global__ void pool_init_kernel(int32_t* free_list, uint32_t n, unsigned int* alloc)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) free_list[i] = (int32_t)i;
    if (i == 0) {
        alloc[0] = n;
        alloc[1] = 0u;
    }
}

// After an epoch: chunks handed out are no longer free.
__global__ void pool_settle_kernel(unsigned int* alloc)
{
    const unsigned int taken = alloc[1] < alloc[0] ? alloc[1] : alloc[0];
    alloc[0] -= taken;
    alloc[1] = 0u;
}

// Harvest the streamlines that finished in an epoch (one warp each): copy
// their points to their request's result buffer and return their chunks to
// the free list.
__global__ void __launch_bounds__(256) harvest_kernel(const ServeJob* __restrict__ jobs,
                                                      const Finished* __restrict__ finished, uint32_t n,
                                                      const float* __restrict__ pool, const int32_t* chunk_next,
                                                      int32_t* free_list, unsigned int* alloc,
                                                      unsigned long long* committed)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k = warp; k < n; k += n_warps) {
        const Finished f = finished[k];
        const ServeJob& J = jobs[f.slot];
        const uint32_t len = J.lengths[f.item];
        int32_t chunk = J.first_chunk[f.item];
        unsigned long long off = 0;
        if (lane == 0) {
            off = atomicAdd(J.cursor, (unsigned long long)len);
            J.result_offset[f.item] = off;
        }
        off = __shfl_sync(0xffffffffu, off, 0);
        // lane q holds the q-th chunk of the current group of up to 32;
        // each group goes back to the free list with one atomic
        int32_t held = -1;
        uint32_t n_held = 0, n_freed = 0;
        auto give_back = [&]() {
            unsigned int at = 0;
            if (lane == 0) at = atomicAdd(alloc, n_held);
            at = __shfl_sync(0xffffffffu, at, 0);
            if (lane < n_held) free_list[at + lane] = held;
            n_freed += n_held;
            n_held = 0;
        };
        for (uint32_t base = 0; base < len && chunk >= 0; base += kChunkPoints) {
            const uint32_t j = base + lane;
            if (j < len) {
                const float* src = pool + ((size_t)chunk * kChunkPoints + lane) * 3;
                float* dst = J.result + (off - J.result_first + j) * 3;
                dst[0] = src[0];
                dst[1] = src[1];
                dst[2] = src[2];
            }
            if (lane == n_held) held = chunk;
            n_held += 1;
            chunk = chunk_next[chunk];
            if (n_held == 32u) give_back();
        }
        if (n_held > 0u) give_back();
        if (lane == 0 && n_freed > 0u) atomicAdd(committed, (unsigned long long)(-(long long)n_freed));
    }
}

// Release the chunks of the listed (overflowed) streamlines and reset them.
__global__ void release_kernel(const int32_t* chunk_next, int32_t* first_chunk, uint32_t* lengths,
                               const uint32_t* ids, uint32_t n, int32_t* free_list, unsigned int* alloc,
                               unsigned long long* committed)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = ids[k];
    int32_t chunk = first_chunk[i];
    while (chunk >= 0) {
        const int32_t next = chunk_next[chunk];
        free_list[atomicAdd(alloc, 1u)] = chunk;
        atomicAdd(committed, (unsigned long long)-1ll);
        chunk = next;
    }
    first_chunk[i] = -1;
    lengths[i] = 0u;
}

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace tg

using namespace tg;

struct ResultSegment {
    float* ptr = nullptr;
    uint64_t first = 0;         // request-wide index of its first point
    uint64_t cap = 0;           // points
};

struct ServeRequest {
    uint64_t id = 0;
    int kind = 0;
    tg_job job{};
    TrackParams tp{};
    const float* host_seeds = nullptr;        // caller's, valid until the request finishes
    const uint32_t* host_rng = nullptr;
    uint32_t n_batches = 0;
    uint64_t reserve = 0;       // bytes counted against the budget while admitted
    // device (admitted)
    float4* d_seeds = nullptr;
    uint8_t* d_inside = nullptr;
    uint32_t* d_rng = nullptr;
    uint32_t* d_lengths = nullptr;
    int32_t* d_first = nullptr;
    uint64_t* d_offset = nullptr;
    // Harvested points live in segments: when an epoch's points do not fit
    // the current one, a new segment starts at the next point (no copy).
    std::vector<ResultSegment> segments;
    uint64_t harvested = 0;     // points
    std::deque<std::pair<uint32_t, uint32_t>> queue;   // (first seed, count) not yet taken
    double t_submit = 0.0;
};

struct ServeResult {
    uint32_t n_seeds = 0;
    uint64_t n_points = 0;
    uint32_t* d_lengths = nullptr;
    uint64_t* d_offset = nullptr;
    std::vector<ResultSegment> segments;
    uint64_t bytes = 0;
    double t_submit = 0.0, t_done = 0.0;
};

struct tg_server {
    uint64_t budget = 0;
    uint64_t fixed = 0;
    uint64_t reserved = 0;
    uint32_t epoch_steps = 1024;
    uint32_t max_slots = 256;
    uint64_t points_estimate = 160;  // result points per seed assumed at admission
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t kstream[kServeKinds] = {};
    cudaEvent_t kdone[kServeKinds] = {};
    cudaEvent_t ev_fork = nullptr;
    ServeJob* d_jobs = nullptr;
    std::vector<ServeJob> h_jobs;
    unsigned int* d_counts = nullptr;                // 2 per slot
    unsigned long long* d_slot_points = nullptr;     // 2 per slot: finished this epoch, cursor
    ServePool P{};
    uint32_t n_chunks = 0;
    LaneCarry* carry[kServeKinds][2] = {};
    size_t carry_cap[kServeKinds] = {};
    int carry_cur[kServeKinds] = {};
    uint32_t carry_n[kServeKinds] = {};
    unsigned int* d_carry_count = nullptr;      // kServeKinds
    unsigned long long* d_counter = nullptr;    // kServeKinds
    unsigned long long* d_steps = nullptr;
    uint32_t* d_segs = nullptr;
    size_t cap_segs = 0;
    Finished* d_finished = nullptr;
    size_t cap_finished = 0;
    unsigned int* d_n_finished = nullptr;
    int blocks_per_sm[kServeKinds] = {};
    // host
    std::vector<ServeRequest*> slots;           // max_slots, null when free
    std::deque<ServeRequest*> pending;
    std::unordered_map<uint64_t, ServeResult> results;
    std::vector<uint64_t> finished;
    uint64_t next_id = 1;
    uint64_t steps_total = 0;
    uint64_t epochs = 0;
    double busy_s = 0.0;
    // device-clock epoch budget (0: epoch_steps only) and device timing
    uint64_t epoch_ns = 0;
    unsigned long long* d_deadline = nullptr;
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr, ev_t2 = nullptr, ev_t3 = nullptr;
    double kernel_s = 0.0, harvest_s = 0.0, between_s = 0.0;
    // request buffers come from the server's own pool, which keeps freed
    // memory (up to the budget) for the next requests instead of returning
    // it to the driver at every synchronisation
    cudaMemPool_t mempool = nullptr;
    // pinned host block for the per-epoch read-back of counters
    unsigned char* h_readback = nullptr;
};

namespace {

int sfail(int code, const std::string& msg) { return tg::set_last_error(code, msg); }

int sfail_cuda(cudaError_t e, const char* what)
{
    return sfail(e == cudaErrorMemoryAllocation ? TG_ERR_OUT_OF_MEMORY : TG_ERR_CUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

#define TG_STRY(call)                                        \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return sfail_cuda(e_, #call); \
    } while (0)

void free_request_buffers(tg_server* S, ServeRequest* r)
{
    void* bufs[] = {r->d_seeds, r->d_inside, r->d_rng, r->d_first, r->d_lengths, r->d_offset};
    for (void* b : bufs)
        if (b) cudaFreeAsync(b, S->stream);
    for (ResultSegment& g : r->segments)
        if (g.ptr) cudaFreeAsync(g.ptr, S->stream);
    r->segments.clear();
    r->d_seeds = nullptr;
    r->d_inside = nullptr;
    r->d_rng = nullptr;
    r->d_first = nullptr;
    r->d_lengths = nullptr;
    r->d_offset = nullptr;
}

int write_slot(tg_server* S, int slot)
{
    TG_STRY(cudaMemcpyAsync(S->d_jobs + slot, &S->h_jobs[slot], sizeof(ServeJob), cudaMemcpyHostToDevice,
                            S->stream));
    return TG_OK;
}

// Admit pending requests in arrival order while slots and budget allow.
int admit(tg_server* S)
{
    while (!S->pending.empty()) {
        ServeRequest* r = S->pending.front();
        int slot = -1;
        for (uint32_t k = 0; k < S->max_slots; ++k)
            if (S->slots[k] == nullptr) {
                slot = (int)k;
                break;
            }
        if (slot < 0 || S->fixed + S->reserved + r->reserve > S->budget) return TG_OK;
        const uint32_t n = r->job.n_seeds;
        ResultSegment seg;
        seg.cap = std::max<uint64_t>(1024, (uint64_t)n * std::min<uint64_t>(r->job.n_steps, S->points_estimate));
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_seeds), (size_t)n * 32, S->mempool, S->stream));
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_rng), (size_t)r->n_batches * 4, S->mempool, S->stream));
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_lengths), (size_t)n * 4, S->mempool, S->stream));
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_first), (size_t)n * 4, S->mempool, S->stream));
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_offset), (size_t)n * 8, S->mempool, S->stream));
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&seg.ptr), seg.cap * 12, S->mempool, S->stream));
        r->segments.assign(1, seg);
        // pageable copies are staged before cudaMemcpyAsync returns
        TG_STRY(cudaMemcpyAsync(r->d_seeds, r->host_seeds, (size_t)n * 32, cudaMemcpyHostToDevice, S->stream));
        TG_STRY(cudaMemcpyAsync(r->d_rng, r->host_rng, (size_t)r->n_batches * 4, cudaMemcpyHostToDevice, S->stream));
        if (r->tp.domain_kind == kDomainMesh) {
            // the seeds' inside tests (three ray walks each), done here for the
            // whole request instead of by single lanes holding their warps
            TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->d_inside), n, S->mempool, S->stream));
            TG_STRY(launch_mesh_contains(r->tp.mesh, r->d_seeds, n, r->d_inside, S->stream, 2u));
        }
        ServeJob& J = S->h_jobs[slot];
        std::memset(&J, 0, sizeof J);
        J.t = r->tp;
        J.seeds = r->d_seeds;
        J.n_seeds = n;
        J.batch_size = r->job.batch_size;
        J.batch_rng_seeds = r->d_rng;
        J.seed_offset = r->job.algorithm.seed_offset;
        J.lengths = r->d_lengths;
        J.first_chunk = r->d_first;
        J.seed_inside = r->d_inside;
        J.counts = S->d_counts + 2 * slot;
        J.finished_points = S->d_slot_points + 2 * slot;
        J.cursor = S->d_slot_points + 2 * slot + 1;
        J.result = seg.ptr;
        J.result_first = 0;
        J.result_offset = r->d_offset;
        J.chunks_needed = (r->job.n_steps + kChunkPoints - 1) / kChunkPoints;
        int st = write_slot(S, slot);
        if (st != TG_OK) return st;
        TG_STRY(cudaMemsetAsync(S->d_counts + 2 * slot, 0, 2 * sizeof(unsigned int), S->stream));
        TG_STRY(cudaMemsetAsync(S->d_slot_points + 2 * slot, 0, 2 * sizeof(unsigned long long), S->stream));
        r->queue.emplace_back(0u, n);
        r->harvested = 0;
        S->slots[slot] = r;
        S->reserved += r->reserve;
        S->pending.pop_front();
    }
    return TG_OK;
}

int ensure_carry(tg_server* S, int kind, size_t lanes)
{
    if (S->carry_cap[kind] >= lanes && S->carry[kind][0] != nullptr) return TG_OK;
    // carried streamlines of this kind, if any, move to the new buffers
    LaneCarry* fresh[2] = {nullptr, nullptr};
    TG_STRY(cudaMalloc(reinterpret_cast<void**>(&fresh[0]), lanes * sizeof(LaneCarry)));
    TG_STRY(cudaMalloc(reinterpret_cast<void**>(&fresh[1]), lanes * sizeof(LaneCarry)));
    const int cur = S->carry_cur[kind];
    if (S->carry_n[kind] > 0)
        TG_STRY(cudaMemcpyAsync(fresh[cur], S->carry[kind][cur], S->carry_n[kind] * sizeof(LaneCarry),
                                cudaMemcpyDeviceToDevice, S->stream));
    TG_STRY(cudaStreamSynchronize(S->stream));
    cudaFree(S->carry[kind][0]);
    cudaFree(S->carry[kind][1]);
    S->carry[kind][0] = fresh[0];
    S->carry[kind][1] = fresh[1];
    S->carry_cap[kind] = lanes;
    return TG_OK;
}

int kind_blocks(tg_server* S, int kind)
{
    if (S->blocks_per_sm[kind] == 0) {
        int b = 0;
        if (serve_dispatch<ServeOccupancy>(kind, &b) != cudaSuccess || b < 1) b = 1;
        S->blocks_per_sm[kind] = b;
    }
    return S->blocks_per_sm[kind];
}

// A request whose seeds were all taken and whose streamlines all finished:
// its result is the harvested points with per-seed offsets and lengths.
void complete(tg_server* S, int slot)
{
    ServeRequest* r = S->slots[slot];
    ServeResult res;
    res.n_seeds = r->job.n_seeds;
    res.n_points = r->harvested;
    res.t_submit = r->t_submit;
    res.t_done = now_s();
    res.d_lengths = r->d_lengths;
    res.d_offset = r->d_offset;
    res.segments.swap(r->segments);
    res.bytes = (uint64_t)res.n_seeds * 12;
    for (const ResultSegment& g : res.segments) res.bytes += g.cap * 12;
    r->d_lengths = nullptr;
    r->d_offset = nullptr;
    free_request_buffers(S, r);
    S->reserved -= r->reserve;
    S->reserved += res.bytes;
    S->results[r->id] = res;
    S->finished.push_back(r->id);
    S->slots[slot] = nullptr;
    delete r;
}

// Re-queue the overflowed streamlines of a request from their seeds.
int requeue_overflow(tg_server* S, int slot)
{
    ServeRequest* r = S->slots[slot];
    const uint32_t n = r->job.n_seeds;
    std::vector<uint32_t> len(n);
    TG_STRY(cudaMemcpyAsync(len.data(), r->d_lengths, (size_t)n * 4, cudaMemcpyDeviceToHost, S->stream));
    TG_STRY(cudaStreamSynchronize(S->stream));
    std::vector<uint32_t> ids;
    for (uint32_t i = 0; i < n; ++i)
        if (len[i] & kOverflowBit) ids.push_back(i);
    if (!ids.empty()) {
        uint32_t* d_ids = nullptr;
        TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&d_ids), ids.size() * 4, S->mempool, S->stream));
        TG_STRY(cudaMemcpyAsync(d_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, S->stream));
        release_kernel<<<((uint32_t)ids.size() + 127) / 128, 128, 0, S->stream>>>(
            S->P.chunk_next, r->d_first, r->d_lengths, d_ids, (uint32_t)ids.size(), S->P.free_list, S->P.alloc,
            S->P.committed);
        TG_STRY(cudaGetLastError());
        TG_STRY(cudaFreeAsync(d_ids, S->stream));
        size_t a = 0;                            // contiguous runs become queue segments
        while (a < ids.size()) {
            size_t b = a + 1;
            while (b < ids.size() && ids[b] == ids[b - 1] + 1) ++b;
            r->queue.emplace_back(ids[a], (uint32_t)(b - a));
            a = b;
        }
    }
    TG_STRY(cudaMemsetAsync(S->d_counts + 2 * slot + 1, 0, sizeof(unsigned int), S->stream));
    return TG_OK;
}

// Start a new result segment at the request's next point, large enough for
// `add` more points (at least twice the last segment); nothing is copied.
int new_result_segment(tg_server* S, int slot, uint64_t add)
{
    ServeRequest* r = S->slots[slot];
    ResultSegment seg;
    seg.first = r->harvested;
    seg.cap = std::max<uint64_t>(add, r->segments.empty() ? 1024 : 2 * r->segments.back().cap);
    TG_STRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&seg.ptr), seg.cap * 12, S->mempool, S->stream));
    S->reserved += seg.cap * 12;
    r->reserve += seg.cap * 12;
    r->segments.push_back(seg);
    S->h_jobs[slot].result = seg.ptr;
    S->h_jobs[slot].result_first = seg.first;
    return write_slot(S, slot);
}

}  // namespace

extern "C" {

int tg_server_create(uint64_t hbm_budget_bytes, uint64_t pool_points, uint32_t epoch_steps, uint32_t max_requests,
                     tg_server** out)
{
    if (out == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (epoch_steps == 0) return sfail(TG_ERR_INVALID_ARGUMENT, "epoch_steps must be positive");
    if (max_requests == 0 || max_requests > 4096) return sfail(TG_ERR_INVALID_ARGUMENT, "max_requests must be 1..4096");
    tg_server* S = new tg_server();
    S->budget = hbm_budget_bytes;
    S->epoch_steps = epoch_steps;
    S->max_slots = max_requests;
    S->slots.assign(max_requests, nullptr);
    S->h_jobs.assign(max_requests, ServeJob{});
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&S->sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t chunks = (pool_points + kChunkPoints - 1) / kChunkPoints;
    if (chunks == 0) chunks = 1u << 20;
    if (chunks > 0x7fffffffull) chunks = 0x7fffffffull;
    S->n_chunks = (uint32_t)chunks;
    cudaError_t e = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev_t0);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev_t1);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev_t2);
    if (e == cudaSuccess) e = cudaEventCreate(&S->ev_t3);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_deadline), sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMallocHost(reinterpret_cast<void**>(&S->h_readback),
                           kServeKinds * (sizeof(unsigned long long) + sizeof(unsigned int)) +
                               (size_t)max_requests * 2 * (sizeof(unsigned int) + sizeof(unsigned long long)) + 64);
    if (e == cudaSuccess) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        e = cudaMemPoolCreate(&S->mempool, &props);
        if (e == cudaSuccess) {
            uint64_t keep = hbm_budget_bytes;
            e = cudaMemPoolSetAttribute(S->mempool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_jobs), max_requests * sizeof(ServeJob));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_counts), 2 * max_requests * sizeof(unsigned int));
    if (e == cudaSuccess)
        e = cudaMalloc(reinterpret_cast<void**>(&S->d_slot_points), 2 * max_requests * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->P.pool), chunks * kChunkPoints * 3 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->P.chunk_next), chunks * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->P.free_list), chunks * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->P.alloc), 2 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->P.committed), sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(S->P.committed, 0, sizeof(unsigned long long), S->stream);
    S->P.n_chunks = (uint32_t)chunks;
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_carry_count), kServeKinds * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_counter), kServeKinds * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_steps), sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&S->d_n_finished), sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(S->d_steps, 0, sizeof(unsigned long long), S->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->d_n_finished, 0, sizeof(unsigned int), S->stream);
    if (e == cudaSuccess) {
        pool_init_kernel<<<(unsigned)((chunks + 255) / 256), 256, 0, S->stream>>>(S->P.free_list, (uint32_t)chunks,
                                                                                  S->P.alloc);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->stream);
    if (e != cudaSuccess) {
        tg_server_destroy(S);
        return sfail_cuda(e, "tg_server_create");
    }
    S->fixed = chunks * kChunkPoints * 12 + chunks * 8 + max_requests * (sizeof(ServeJob) + 24);
    if (S->fixed > S->budget) {
        tg_server_destroy(S);
        return sfail(TG_ERR_OUT_OF_MEMORY, "the point pool alone exceeds the HBM budget");
    }
    *out = S;
    return TG_OK;
}

int tg_server_destroy(tg_server* S)
{
    if (S == nullptr) return TG_OK;
    if (S->stream) cudaStreamSynchronize(S->stream);
    for (ServeRequest* r : S->slots)
        if (r) {
            free_request_buffers(S, r);
            delete r;
        }
    for (ServeRequest* r : S->pending) delete r;
    for (auto& kv : S->results) {
        void* bufs[] = {kv.second.d_lengths, kv.second.d_offset};
        for (void* b : bufs)
            if (b) cudaFreeAsync(b, S->stream);
        for (const ResultSegment& g : kv.second.segments)
            if (g.ptr) cudaFreeAsync(g.ptr, S->stream);
    }
    if (S->stream) cudaStreamSynchronize(S->stream);
    for (int k = 0; k < kServeKinds; ++k) {
        cudaFree(S->carry[k][0]);
        cudaFree(S->carry[k][1]);
        if (S->kstream[k]) cudaStreamDestroy(S->kstream[k]);
        if (S->kdone[k]) cudaEventDestroy(S->kdone[k]);
    }
    void* bufs[] = {S->d_jobs, S->d_counts, S->d_slot_points, S->P.pool, S->P.chunk_next, S->P.free_list,
                    S->P.alloc, S->P.committed, S->d_carry_count, S->d_counter, S->d_steps, S->d_segs, S->d_finished,
                    S->d_n_finished, S->d_deadline};
    for (void* b : bufs) cudaFree(b);
    if (S->mempool) cudaMemPoolDestroy(S->mempool);
    if (S->h_readback) cudaFreeHost(S->h_readback);
    cudaEvent_t evs[] = {S->ev_fork, S->ev_t0, S->ev_t1, S->ev_t2, S->ev_t3};
    for (cudaEvent_t ev : evs)
        if (ev) cudaEventDestroy(ev);
    if (S->stream) cudaStreamDestroy(S->stream);
    delete S;
    return TG_OK;
}

int tg_server_submit(tg_server* S, const tg_job* job, uint64_t* request_id)
{
    if (S == nullptr || job == nullptr || request_id == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "null argument");
    TrackParams tp;
    int model = 0, lmax = 0;
    int st = track_params_from_handles(&job->algorithm, job->domain, job->field, job->save_at, job->n_steps, &tp,
                                       &model, &lmax);
    if (st != TG_OK) return st;
    if (job->n_steps == 0) return sfail(TG_ERR_INVALID_ARGUMENT, "n_steps must be positive");
    if (job->n_seeds > 0 && (job->seeds == nullptr || job->batch_rng_seeds == nullptr || job->batch_size == 0))
        return sfail(TG_ERR_INVALID_ARGUMENT, "missing seeds or batch seeds");
    if ((job->n_steps + kChunkPoints - 1) / kChunkPoints > S->n_chunks)
        return sfail(TG_ERR_POOL_EXHAUSTED, "the server's point pool cannot hold one streamline of this request");
    ServeRequest* r = new ServeRequest();
    r->id = S->next_id++;
    r->kind = 2 * class_kind(model, lmax, job->algorithm.algorithm) + (tp.domain_kind == kDomainMesh ? 1 : 0);
    r->job = *job;
    r->tp = tp;
    const uint32_t n = job->n_seeds;
    r->n_batches = n ? (n + job->batch_size - 1) / job->batch_size : 0;
    r->host_seeds = job->seeds;
    r->host_rng = job->batch_rng_seeds;
    r->reserve = (uint64_t)n * 49 + (uint64_t)r->n_batches * 4 +
                 std::max<uint64_t>(1024, (uint64_t)n * std::min<uint64_t>(job->n_steps, S->points_estimate)) * 12;
    r->t_submit = now_s();
    *request_id = r->id;
    if (n == 0) {
        ServeResult res;
        res.t_submit = res.t_done = r->t_submit;
        S->results[r->id] = res;
        S->finished.push_back(r->id);
        delete r;
        return TG_OK;
    }
    if (S->fixed + r->reserve > S->budget) {
        delete r;
        return sfail(TG_ERR_OUT_OF_MEMORY, "request larger than the server's HBM budget");
    }
    S->pending.push_back(r);
    return TG_OK;
}

int tg_server_poll(tg_server* S, uint64_t* finished_ids, uint32_t capacity, uint32_t* n_finished,
                   uint32_t* n_active, uint32_t* n_pending)
{
    if (S == nullptr || n_finished == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "null argument");
    *n_finished = 0;
    int st = admit(S);
    if (st != TG_OK) return st;

    // per kind: the queue segments offered this epoch, requests in arrival order
    std::vector<uint32_t> seg_slot[kServeKinds], seg_start[kServeKinds], seg_prefix[kServeKinds];
    uint64_t n_new[kServeKinds] = {};
    std::vector<uint32_t> order;
    for (uint32_t slot = 0; slot < S->max_slots; ++slot)
        if (S->slots[slot] != nullptr) order.push_back(slot);
    std::sort(order.begin(), order.end(), [S](uint32_t a, uint32_t b) { return S->slots[a]->id < S->slots[b]->id; });
    for (uint32_t slot : order) {
        ServeRequest* r = S->slots[slot];
        const int k = r->kind;
        // an epoch cannot take more seeds than its lanes can start: at most
        // one per lane per loop iteration
        const uint64_t cap = std::min<uint64_t>(0x7fffffffull, (uint64_t)S->sms * kind_blocks(S, k) * 128 *
                                                                   S->epoch_steps);
        for (auto& seg : r->queue) {
            if (n_new[k] >= cap) break;                          // offered next epoch
            if (seg_prefix[k].empty()) seg_prefix[k].push_back(0);
            seg_slot[k].push_back(slot);
            seg_start[k].push_back(seg.first);
            n_new[k] += seg.second;
            seg_prefix[k].push_back((uint32_t)n_new[k]);
        }
    }
    bool any = false;
    uint64_t offered = 0;
    for (int k = 0; k < kServeKinds; ++k) {
        any = any || n_new[k] > 0 || S->carry_n[k] > 0;
        offered += n_new[k] + S->carry_n[k];
    }

    if (any) {
        const double t0 = now_s();
        int grid[kServeKinds] = {};
        for (int k = 0; k < kServeKinds; ++k) {
            if (n_new[k] == 0 && S->carry_n[k] == 0) continue;
            // every kind is launched with as many blocks as its work fills,
            // up to a full GPU, on its own stream: the block scheduler gives
            // SMs freed by a kind whose queue drained to the others (a fixed
            // split would leave them idle until the deadline).  At least one
            // lane per carried streamline (it resumes in the lane's first fetch).
            const int full = S->sms * kind_blocks(S, k);
            const int need = (int)((S->carry_n[k] + 127) / 128);
            const int work = (int)std::min<uint64_t>((uint64_t)full, (n_new[k] + S->carry_n[k] + 127) / 128);
            grid[k] = std::max(1, std::max(need, work));
            st = ensure_carry(S, k, (size_t)full * 128);
            if (st != TG_OK) return st;
            if (S->kstream[k] == nullptr) {
                TG_STRY(cudaStreamCreateWithFlags(&S->kstream[k], cudaStreamNonBlocking));
                TG_STRY(cudaEventCreateWithFlags(&S->kdone[k], cudaEventDisableTiming));
            }
        }
        if (S->cap_finished < offered) {
            cudaFree(S->d_finished);
            S->d_finished = nullptr;
            S->cap_finished = 0;
            const size_t cap = std::max<size_t>(offered, (size_t)1 << 20);
            TG_STRY(cudaMalloc(reinterpret_cast<void**>(&S->d_finished), cap * sizeof(Finished)));
            S->cap_finished = cap;
        }
        // one upload of all segment tables
        std::vector<uint32_t> segs;
        size_t at[kServeKinds][3] = {};
        for (int k = 0; k < kServeKinds; ++k) {
            at[k][0] = segs.size();
            segs.insert(segs.end(), seg_slot[k].begin(), seg_slot[k].end());
            at[k][1] = segs.size();
            segs.insert(segs.end(), seg_start[k].begin(), seg_start[k].end());
            at[k][2] = segs.size();
            segs.insert(segs.end(), seg_prefix[k].begin(), seg_prefix[k].end());
        }
        if (S->cap_segs < segs.size() + 1) {
            cudaFree(S->d_segs);
            S->d_segs = nullptr;
            S->cap_segs = 0;
            TG_STRY(cudaMalloc(reinterpret_cast<void**>(&S->d_segs), (segs.size() + 1) * 2 * sizeof(uint32_t)));
            S->cap_segs = (segs.size() + 1) * 2;
        }
        if (!segs.empty())
            TG_STRY(cudaMemcpyAsync(S->d_segs, segs.data(), segs.size() * 4, cudaMemcpyHostToDevice, S->stream));
        TG_STRY(cudaMemsetAsync(S->d_counter, 0, kServeKinds * sizeof(unsigned long long), S->stream));
        TG_STRY(cudaMemsetAsync(S->d_carry_count, 0, kServeKinds * sizeof(unsigned int), S->stream));
        TG_STRY(cudaMemsetAsync(S->d_n_finished, 0, sizeof(unsigned int), S->stream));
        TG_STRY(cudaEventRecord(S->ev_t0, S->stream));
        if (S->epoch_ns > 0) {
            epoch_deadline_kernel<<<1, 1, 0, S->stream>>>(S->d_deadline, (unsigned long long)S->epoch_ns);
            TG_STRY(cudaGetLastError());
        }
        TG_STRY(cudaEventRecord(S->ev_fork, S->stream));
        for (int k = 0; k < kServeKinds; ++k) {
            if (grid[k] == 0) continue;
            ServeParams sp;
            std::memset(&sp, 0, sizeof sp);
            sp.jobs = S->d_jobs;
            sp.P = S->P;
            sp.carry_in = S->carry[k][S->carry_cur[k]];
            sp.n_carry = S->carry_n[k];
            sp.carry_out = S->carry[k][S->carry_cur[k] ^ 1];
            sp.carry_out_count = S->d_carry_count + k;
            sp.seg_slot = S->d_segs + at[k][0];
            sp.seg_start = S->d_segs + at[k][1];
            sp.seg_prefix = S->d_segs + at[k][2];
            sp.n_seg = (uint32_t)seg_slot[k].size();
            sp.n_new = (uint32_t)n_new[k];
            sp.counter = S->d_counter + k;
            sp.step_budget = S->epoch_steps;
            sp.deadline = S->epoch_ns > 0 ? S->d_deadline : nullptr;
            sp.steps_done = S->d_steps;
            sp.finished = S->d_finished;
            sp.n_finished = S->d_n_finished;
            TG_STRY(cudaStreamWaitEvent(S->kstream[k], S->ev_fork, 0));
            TG_STRY(serve_dispatch<ServeLaunch>(k, sp, grid[k], S->kstream[k]));
            TG_STRY(cudaEventRecord(S->kdone[k], S->kstream[k]));
            TG_STRY(cudaStreamWaitEvent(S->stream, S->kdone[k], 0));
        }
        TG_STRY(cudaEventRecord(S->ev_t1, S->stream));
        pool_settle_kernel<<<1, 1, 0, S->stream>>>(S->P.alloc);
        TG_STRY(cudaGetLastError());
        // read-back into one pinned block (asynchronous copies, one synchronisation)
        unsigned long long* const slot_points = reinterpret_cast<unsigned long long*>(S->h_readback);
        unsigned long long* const counter = slot_points + 2 * (size_t)S->max_slots;
        unsigned long long* const steps_p = counter + kServeKinds;
        unsigned int* const counts = reinterpret_cast<unsigned int*>(steps_p + 1);
        unsigned int* const carry_count = counts + 2 * (size_t)S->max_slots;
        unsigned int* const n_fin_p = carry_count + kServeKinds;
        TG_STRY(cudaMemcpyAsync(counter, S->d_counter, kServeKinds * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, S->stream));
        TG_STRY(cudaMemcpyAsync(carry_count, S->d_carry_count, kServeKinds * sizeof(unsigned int),
                                cudaMemcpyDeviceToHost, S->stream));
        TG_STRY(cudaMemcpyAsync(counts, S->d_counts, 2 * (size_t)S->max_slots * sizeof(unsigned int),
                                cudaMemcpyDeviceToHost, S->stream));
        TG_STRY(cudaMemcpyAsync(slot_points, S->d_slot_points, 2 * (size_t)S->max_slots * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, S->stream));
        TG_STRY(cudaMemcpyAsync(n_fin_p, S->d_n_finished, sizeof(unsigned int), cudaMemcpyDeviceToHost, S->stream));
        TG_STRY(cudaMemcpyAsync(steps_p, S->d_steps, sizeof(unsigned long long), cudaMemcpyDeviceToHost, S->stream));
        TG_STRY(cudaStreamSynchronize(S->stream));
        const unsigned int n_fin = *n_fin_p;
        const unsigned long long steps = *steps_p;
        S->steps_total = steps;
        S->epochs += 1;
        // result buffers large enough for this epoch's finished streamlines,
        // then the harvest (points to results, chunks back to the free list)
        for (uint32_t slot : order) {
            ServeRequest* r = S->slots[slot];
            const uint64_t add = slot_points[2 * slot];
            if (add == 0) continue;
            const ResultSegment& cur = r->segments.back();
            if (r->harvested + add > cur.first + cur.cap) {
                st = new_result_segment(S, (int)slot, add);
                if (st != TG_OK) return st;
            }
            r->harvested += add;
        }
        TG_STRY(cudaEventRecord(S->ev_t3, S->stream));
        if (n_fin > 0) {
            uint64_t g = ((uint64_t)n_fin * 32 + 255) / 256;
            if (g > (uint64_t)S->sms * 16) g = (uint64_t)S->sms * 16;
            harvest_kernel<<<(int)g, 256, 0, S->stream>>>(S->d_jobs, S->d_finished, n_fin, S->P.pool,
                                                          S->P.chunk_next, S->P.free_list, S->P.alloc,
                                                          S->P.committed);
            TG_STRY(cudaGetLastError());
        }
        TG_STRY(cudaEventRecord(S->ev_t2, S->stream));
        for (uint32_t slot : order) {
            if (slot_points[2 * slot] != 0)
                TG_STRY(cudaMemsetAsync(S->d_slot_points + 2 * slot, 0, sizeof(unsigned long long), S->stream));
        }
        // advance the queues by the seeds each kind took, in offer order
        for (int k = 0; k < kServeKinds; ++k) {
            if (grid[k] == 0) continue;
            const unsigned long long c = counter[k];
            uint64_t taken = c > S->carry_n[k] ? c - S->carry_n[k] : 0;
            if (taken > n_new[k]) taken = n_new[k];
            for (size_t q = 0; q < seg_slot[k].size() && taken > 0; ++q) {
                ServeRequest* r = S->slots[seg_slot[k][q]];
                auto& seg = r->queue.front();
                const uint32_t use = (uint32_t)std::min<uint64_t>(taken, seg.second);
                seg.first += use;
                seg.second -= use;
                taken -= use;
                if (seg.second == 0) r->queue.pop_front();
            }
            S->carry_n[k] = carry_count[k];
            S->carry_cur[k] ^= 1;
        }
        // finished requests; overflowed streamlines go back to their queue
        for (uint32_t slot : order) {
            ServeRequest* r = S->slots[slot];
            if (!r->queue.empty() || counts[2 * slot] != 0) continue;
            if (counts[2 * slot + 1] != 0) {
                st = requeue_overflow(S, (int)slot);
                if (st != TG_OK) return st;
                continue;
            }
            complete(S, (int)slot);
        }
        TG_STRY(cudaStreamSynchronize(S->stream));
        S->busy_s += now_s() - t0;
        float k_ms = 0.0f, b_ms = 0.0f, h_ms = 0.0f;
        if (cudaEventElapsedTime(&k_ms, S->ev_t0, S->ev_t1) == cudaSuccess) S->kernel_s += 1e-3 * k_ms;
        if (cudaEventElapsedTime(&b_ms, S->ev_t1, S->ev_t3) == cudaSuccess) S->between_s += 1e-3 * b_ms;
        if (cudaEventElapsedTime(&h_ms, S->ev_t3, S->ev_t2) == cudaSuccess) S->harvest_s += 1e-3 * h_ms;
        st = admit(S);
        if (st != TG_OK) return st;
    }
    const uint32_t n = (uint32_t)std::min<size_t>(capacity, S->finished.size());
    for (uint32_t i = 0; i < n; ++i) finished_ids[i] = S->finished[i];
    S->finished.erase(S->finished.begin(), S->finished.begin() + n);
    *n_finished = n;
    if (n_active) {
        uint32_t a = 0;
        for (ServeRequest* r : S->slots) a += r != nullptr;
        *n_active = a;
    }
    if (n_pending) *n_pending = (uint32_t)S->pending.size();
    return TG_OK;
}

int tg_server_result_size(tg_server* S, uint64_t request_id, uint32_t* n_seeds, uint64_t* n_points,
                          double* seconds)
{
    if (S == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "server is null");
    auto it = S->results.find(request_id);
    if (it == S->results.end()) return sfail(TG_ERR_INVALID_ARGUMENT, "no finished request with this id");
    if (n_seeds) *n_seeds = it->second.n_seeds;
    if (n_points) *n_points = it->second.n_points;
    if (seconds) *seconds = it->second.t_done - it->second.t_submit;
    return TG_OK;
}

int tg_server_take(tg_server* S, uint64_t request_id, uint32_t* lengths, uint64_t* offsets, float* points)
{
    if (S == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "server is null");
    auto it = S->results.find(request_id);
    if (it == S->results.end()) return sfail(TG_ERR_INVALID_ARGUMENT, "no finished request with this id");
    ServeResult& res = it->second;
    if (res.n_seeds > 0 && lengths)
        TG_STRY(cudaMemcpyAsync(lengths, res.d_lengths, (size_t)res.n_seeds * 4, cudaMemcpyDeviceToHost, S->stream));
    if (res.n_seeds > 0 && offsets)
        TG_STRY(cudaMemcpyAsync(offsets, res.d_offset, (size_t)res.n_seeds * 8, cudaMemcpyDeviceToHost, S->stream));
    for (size_t k = 0; k < res.segments.size(); ++k) {
        const ResultSegment& g = res.segments[k];
        const uint64_t end = k + 1 < res.segments.size() ? res.segments[k + 1].first : res.n_points;
        if (points && end > g.first)
            TG_STRY(cudaMemcpyAsync(points + g.first * 3, g.ptr, (end - g.first) * 12, cudaMemcpyDeviceToHost,
                                    S->stream));
    }
    void* bufs[] = {res.d_lengths, res.d_offset};
    for (void* b : bufs)
        if (b) TG_STRY(cudaFreeAsync(b, S->stream));
    for (const ResultSegment& g : res.segments)
        if (g.ptr) TG_STRY(cudaFreeAsync(g.ptr, S->stream));
    TG_STRY(cudaStreamSynchronize(S->stream));
    S->reserved -= std::min(S->reserved, res.bytes);
    S->results.erase(it);
    return admit(S);
}

int tg_server_reserve(tg_server* S, uint64_t bytes)
{
    if (S == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "server is null");
    if (bytes == 0) return TG_OK;
    // allocate and free once: the pool keeps the memory (its release
    // threshold is the budget), so later request buffers are carved from it
    // instead of mapping new memory while requests wait
    void* p = nullptr;
    const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, S->mempool, S->stream);
    if (e != cudaSuccess) {
        // A reservation that does not fit only costs time later (the pool
        // then maps memory as requests need it), so it must not leave its
        // error as the thread's last CUDA error, where the next launch check
        // of an epoch would report it.  Drain the stream first, then clear.
        cudaStreamSynchronize(S->stream);
        cudaGetLastError();
        return sfail_cuda(e, "cudaMallocFromPoolAsync (reservation)");
    }
    TG_STRY(cudaFreeAsync(p, S->stream));
    TG_STRY(cudaStreamSynchronize(S->stream));
    return TG_OK;
}

int tg_server_set_epoch_time(tg_server* S, double seconds)
{
    if (S == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "server is null");
    if (!(seconds >= 0.0) || seconds > 60.0) return sfail(TG_ERR_INVALID_ARGUMENT, "epoch time must be 0..60 s");
    S->epoch_ns = (uint64_t)(seconds * 1e9);
    return TG_OK;
}

int tg_server_timing(const tg_server* S, double* kernel_seconds, double* between_seconds, double* harvest_seconds)
{
    if (S == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "server is null");
    if (kernel_seconds) *kernel_seconds = S->kernel_s;
    if (between_seconds) *between_seconds = S->between_s;
    if (harvest_seconds) *harvest_seconds = S->harvest_s;
    return TG_OK;
}

int tg_server_stats(const tg_server* S, uint64_t* steps, uint64_t* epochs, double* busy_seconds,
                    uint64_t* reserved_bytes)
{
    if (S == nullptr) return sfail(TG_ERR_INVALID_ARGUMENT, "server is null");
    if (steps) *steps = S->steps_total;
    if (epochs) *epochs = S->epochs;
    if (busy_seconds) *busy_seconds = S->busy_s;
    if (reserved_bytes) *reserved_bytes = S->fixed + S->reserved;
    return TG_OK;
}

}  // extern "C"
