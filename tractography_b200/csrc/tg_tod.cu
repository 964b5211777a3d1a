/*
 * tg_tod.cu -- track orientation distribution (tracking.py:181-385).
 *
 * Every boundary seed is one track, as in the reference's `tod` kernel (one
 * work-item per seed): the seed is drawn on the domain boundary from
 * rng_init(rng_seed, index) (the same state then drives the Diffusion noise),
 * the streamline is integrated for at most
 * floor(maximum_streamline_length / step_size) iterations, and at every
 * iteration the real symmetric SH basis (lmax 8, 45 terms) of the current
 * orientation is added to the output voxel nearest the point.  Consecutive
 * iterations in the same voxel are summed in the thread's accumulator
 * (shared memory, 45 floats per thread) and flushed with one atomicAdd per
 * coefficient when the voxel changes or the track ends -- the reference does
 * the same with a compare-and-swap loop (core.cl:80-99).  Float additions
 * from different threads land in arbitrary order, so results agree with a
 * sequential sum to float tolerance, not bit for bit.  Lanes of an
 * occupancy-sized grid take seed indices from a device counter and start the
 * next track as soon as theirs ends.
 */
#include <cuda_runtime.h>

#include <algorithm>

#include "tg_internal.h"
#include "tg_step.cuh"

namespace tg {

namespace {

constexpr int kTodCoefficients = 45;
constexpr int kTodThreads = 128;

__device__ __forceinline__ void tod_flush(float* __restrict__ out, const float* acc, int tid, int ix, int iy, int iz,
                                          const TodParams& q)
{
    const size_t base = (((size_t)ix * q.ny + iy) * q.nz + iz) * kTodCoefficients;
#pragma unroll 5
    for (int k = 0; k < kTodCoefficients; ++k) atomicAdd(out + base + k, acc[k * kTodThreads + tid]);
}

template <int MODEL, int LMAX, int ALGO, int DOM>
__global__ void __launch_bounds__(kTodThreads) tod_kernel(const TodParams q)
{
    __shared__ float acc[kTodCoefficients * kTodThreads];
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    const int tid = threadIdx.x;
    const TrackParams& p = q.t;
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;
    Lane s;
    int prev_x = -1, prev_y = -1, prev_z = -1;
    uint32_t step = 0;
    unsigned long long steps_total = 0;

    // Next track: seed index from the counter, drawn on the boundary from
    // rng_init(rng_seed, index); false when every seed is taken.
    auto start = [&]() -> bool {
        const unsigned long long k = atomicAdd(q.counter, 1ull);
        if (k >= q.n_seeds) return false;
        const uint32_t gid = (uint32_t)k;
        Mwc st = rng_init(q.rng_seed, gid);
        float px, py, pz, ox, oy, oz;
        sample_boundary(q.vertices, q.triangles, q.cumulative, q.n_triangles, st, px, py, pz, ox, oy, oz);
        lane_init(s, make_float4(px, py, pz, 1.0f), make_float4(ox, oy, oz, 0.0f), 0u, 0u, q.seed_offset + gid);
        s.rng.mwc = st;
        prev_x = prev_y = prev_z = -1;
        step = 0;
        return true;
    };

    // One loop iteration per step of every live lane; a lane whose track
    // ended flushes it and starts the next in the same iteration, so lanes
    // stay busy while the queue lasts (a loop per track would hold finished
    // lanes until the warp's longest track ends).
    bool live = start();
    while (__any_sync(0xffffffffu, live)) {
        if (!live) continue;
        bool go = step < q.n_steps && locate<MODEL, LMAX, CPAD, DOM>(p, s, c);
        if (go) {
            // output voxel nearest the point, floor(A^-1 p + 0.5) (tracking.py:294-300)
            const float vx = floorf(dot4(q.out_row0, s.px, s.py, s.pz, 1.0f) + 0.5f);
            const float vy = floorf(dot4(q.out_row1, s.px, s.py, s.pz, 1.0f) + 0.5f);
            const float vz = floorf(dot4(q.out_row2, s.px, s.py, s.pz, 1.0f) + 0.5f);
            if (vx >= 0.0f && vx < (float)q.nx && vy >= 0.0f && vy < (float)q.ny && vz >= 0.0f &&
                vz < (float)q.nz) {
                const int ix = (int)vx, iy = (int)vy, iz = (int)vz;
                float Y[kTodCoefficients];
                const Frame f = frame_of(s.ox, s.oy, s.oz);
                sh_basis<8>(f.ct, f.st, f.cp, f.sp, Y);
                if (ix == prev_x && iy == prev_y && iz == prev_z) {
#pragma unroll
                    for (int k = 0; k < kTodCoefficients; ++k) acc[k * kTodThreads + tid] += Y[k];
                } else {
                    if (prev_x >= 0) tod_flush(q.coefficients, acc, tid, prev_x, prev_y, prev_z, q);
#pragma unroll
                    for (int k = 0; k < kTodCoefficients; ++k) acc[k * kTodThreads + tid] = Y[k];
                    prev_x = ix;
                    prev_y = iy;
                    prev_z = iz;
                }
            } else if (prev_x >= 0) {
                tod_flush(q.coefficients, acc, tid, prev_x, prev_y, prev_z, q);
                prev_x = prev_y = prev_z = -1;
            }
            update_orientation<MODEL, LMAX, ALGO>(p.algo, c, s.ox, s.oy, s.oz, s.rng);
            s.steps += 1u;
            // tracking.py:343: stop on a non-finite or degenerate orientation
            const float len = sqrtf(s.ox * s.ox + s.oy * s.oy + s.oz * s.oz);
            if (!(isfinite(s.ox) && isfinite(s.oy) && isfinite(s.oz)) || len < 0.5f) {
                go = false;
            } else {
                const float h = p.algo.step_size;
                s.px = fmaf(h, s.ox, s.px);
                s.py = fmaf(h, s.oy, s.py);
                s.pz = fmaf(h, s.oz, s.pz);
                step += 1u;
            }
        }
        if (!go) {
            if (prev_x >= 0) tod_flush(q.coefficients, acc, tid, prev_x, prev_y, prev_z, q);
            steps_total += s.steps;
            live = start();
        }
    }
    add_steps64(q.steps, steps_total);
}

template <int M, int L, int A, int D>
cudaError_t run_tod(const TodParams& q, cudaStream_t stream)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tod_kernel<M, L, A, D>, kTodThreads, 0) !=
            cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint64_t want = ((uint64_t)q.n_seeds + kTodThreads - 1) / kTodThreads;
    const int grid = (int)std::min<uint64_t>(want, (uint64_t)sms * per_sm);
    tod_kernel<M, L, A, D><<<grid, kTodThreads, 0, stream>>>(q);
    return cudaGetLastError();
}

template <int M, int L, int A>
cudaError_t run_tod_domain(const TodParams& q, cudaStream_t stream)
{
    return q.t.domain_kind == kDomainMesh ? run_tod<M, L, A, kDomainMesh>(q, stream)
                                          : run_tod<M, L, A, kDomainImage>(q, stream);
}

}  // namespace

cudaError_t launch_tod(int model, int lmax, const TodParams& q, cudaStream_t stream)
{
    if (q.n_seeds == 0 || q.n_steps == 0) return cudaSuccess;
    const int a = q.t.algorithm;
#define TG_TOD(M, L)                                                                                    \
    if (model == M && (M == kModelDTI || lmax == L))                                                    \
        return a == kTransport ? run_tod_domain<M, L, kTransport>(q, stream)                            \
                               : run_tod_domain<M, L, kDiffusion>(q, stream);
    TG_TOD(kModelSH, 0)
    TG_TOD(kModelSH, 2)
    TG_TOD(kModelSH, 4)
    TG_TOD(kModelSH, 6)
    TG_TOD(kModelSH, 8)
    TG_TOD(kModelDTI, 0)
#undef TG_TOD
    return cudaErrorInvalidValue;
}

}  // namespace tg
