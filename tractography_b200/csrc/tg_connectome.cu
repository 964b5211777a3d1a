/*
 * tg_connectome.cu -- boundary connectome (tracking.py:388-602).
 *
 * Every boundary seed is one track, as in the reference's `connectome`
 * kernel (one work-item per seed): the seed is drawn on the domain boundary
 * (its triangle and barycentric coordinates kept), the track is integrated for at most
 * floor(maximum_streamline_length / step_size) iterations, and when it stops
 * for any reason its final segment is tested against the boundary BVH
 * (closest hit, bvh.cl:83-131).  A track that moved at least the minimum
 * length and hit the boundary writes the nine products of its start and end
 * barycentric weights at (start vertex, end vertex) pairs; the host sums them
 * into a sparse matrix.  Lanes of an occupancy-sized grid take seed indices
 * from a device counter and start the next track as soon as theirs ends;
 * each track's output slots depend on its index only, so results are
 * deterministic.
 */
#include <cuda_runtime.h>

#include <algorithm>

#include "tg_internal.h"
#include "tg_step.cuh"

namespace tg {

namespace {

template <int MODEL, int LMAX, int ALGO, int DOM>
__global__ void __launch_bounds__(128) connectome_kernel(const ConnectomeParams q)
{
    constexpr int CPAD = ModelShape<MODEL, LMAX>::CPAD;
    const TrackParams& p = q.t;
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = 0.0f;
    Lane s;
    uint32_t gid = 0, step = 0, tracked = 0, start_tri = 0;
    float start_w[3] = {0.0f, 0.0f, 0.0f};
    float qx = 0.0f, qy = 0.0f, qz = 0.0f;          // previous point
    unsigned long long steps_total = 0;

    // Next track: seed index from the counter; false when every seed is taken.
    auto start = [&]() -> bool {
        const unsigned long long k = atomicAdd(q.counter, 1ull);
        if (k >= q.n_seeds) return false;
        gid = (uint32_t)k;
        const size_t base = 9 * (size_t)gid;
#pragma unroll
        for (int m = 0; m < 9; ++m) q.rows[base + m] = -1;
        Mwc st = rng_init(q.rng_seed, gid);
        float px, py, pz, ox, oy, oz;
        sample_boundary(q.vertices, q.triangles, q.cumulative, q.n_triangles, st, px, py, pz, ox, oy, oz, &start_tri,
                        start_w);
        lane_init(s, make_float4(px, py, pz, 1.0f), make_float4(ox, oy, oz, 0.0f), 0u, 0u, q.seed_offset + gid);
        s.rng.mwc = st;
        qx = px;
        qy = py;
        qz = pz;
        step = 0;
        tracked = 0;
        return true;
    };

    // The end of a track: a track that moved at least the minimum length
    // and whose final segment hits the boundary writes its nine products.
    auto finish = [&]() {
        steps_total += s.steps;
        if ((float)tracked * p.algo.step_size < q.minimum_length) return;
        const Segment g = make_segment(qx, qy, qz, s.px, s.py, s.pz);
        float t, u = 0.0f, v = 0.0f;
        uint32_t hit_tri = 0;
        if (mesh_walk<0>(q.bvh, g, t, hit_tri, u, v) == 0u) return;
        const float end_w[3] = {1.0f - u - v, u, v};
        const uint4 a = q.triangles[start_tri], b = q.triangles[hit_tri];
        const uint32_t sv[3] = {a.x, a.y, a.z}, ev[3] = {b.x, b.y, b.z};
        const size_t base = 9 * (size_t)gid;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                q.rows[base + 3 * i + j] = (int32_t)sv[i];
                q.columns[base + 3 * i + j] = (int32_t)ev[j];
                q.weights[base + 3 * i + j] = start_w[i] * end_w[j];
            }
    };

    // One loop iteration per step of every live lane; a lane whose track
    // ended finishes it and starts the next in the same iteration.
    bool live = start();
    while (__any_sync(0xffffffffu, live)) {
        if (!live) continue;
        bool go = step < q.n_steps && locate<MODEL, LMAX, CPAD, DOM>(p, s, c);
        if (go) {
            update_orientation<MODEL, LMAX, ALGO>(p.algo, c, s.ox, s.oy, s.oz, s.rng);
            s.steps += 1u;
            const float len = sqrtf(s.ox * s.ox + s.oy * s.oy + s.oz * s.oz);
            if (!(isfinite(s.ox) && isfinite(s.oy) && isfinite(s.oz)) || len < 0.5f) {
                go = false;
            } else {
                qx = s.px;
                qy = s.py;
                qz = s.pz;
                const float h = p.algo.step_size;
                s.px = fmaf(h, s.ox, s.px);
                s.py = fmaf(h, s.oy, s.py);
                s.pz = fmaf(h, s.oz, s.pz);
                tracked += 1u;
                step += 1u;
            }
        }
        if (!go) {
            finish();
            live = start();
        }
    }
    add_steps64(q.steps, steps_total);
}

template <int M, int L, int A, int D>
cudaError_t run(const ConnectomeParams& q, cudaStream_t stream)
{
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, connectome_kernel<M, L, A, D>, 128, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const uint64_t want = ((uint64_t)q.n_seeds + 127) / 128;
    const int grid = (int)std::min<uint64_t>(want, (uint64_t)sms * per_sm);
    connectome_kernel<M, L, A, D><<<grid, 128, 0, stream>>>(q);
    return cudaGetLastError();
}

template <int M, int L, int A>
cudaError_t run_domain(const ConnectomeParams& q, cudaStream_t stream)
{
    return q.t.domain_kind == kDomainMesh ? run<M, L, A, kDomainMesh>(q, stream) : run<M, L, A, kDomainImage>(q, stream);
}

}  // namespace

cudaError_t launch_connectome(int model, int lmax, const ConnectomeParams& q, cudaStream_t stream)
{
    if (q.n_seeds == 0) return cudaSuccess;
    const int a = q.t.algorithm;
#define TG_CONN(M, L)                                                                                   \
    if (model == M && (M == kModelDTI || lmax == L))                                                    \
        return a == kTransport ? run_domain<M, L, kTransport>(q, stream) : run_domain<M, L, kDiffusion>(q, stream);
    TG_CONN(kModelSH, 0)
    TG_CONN(kModelSH, 2)
    TG_CONN(kModelSH, 4)
    TG_CONN(kModelSH, 6)
    TG_CONN(kModelSH, 8)
    TG_CONN(kModelDTI, 0)
#undef TG_CONN
    return cudaErrorInvalidValue;
}

}  // namespace tg
