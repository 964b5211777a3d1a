/*
 * tg_step.cuh -- one iteration of the tracking loop (tracking.py:121-147)
 * and the per-lane state, shared by the tracking kernels.
 */
#ifndef TG_STEP_CUH
#define TG_STEP_CUH

#include "tg_internal.h"

namespace tg {

template <int MODEL, int LMAX>
struct ModelShape {
    static constexpr int CP = (MODEL == kModelDTI) ? 6 : n_coef_full(LMAX);
    static constexpr int CPAD = (CP + 3) / 4 * 4;
};

struct Lane {
    float px, py, pz;
    float ox, oy, oz;
    float time;
    uint32_t n;
    RngState rng;
    // rounded voxel coordinates of the last domain test and field gather;
    // while they are unchanged the mask bit (inside) and the coefficients in
    // registers are still valid, so the bounds tests, index arithmetic and
    // loads are skipped.  NaN forces the first evaluation.
    float dvx, dvy, dvz;
    float fvx, fvy, fvz;
    uint32_t steps;
};

// One iteration of tracking.py:121-147 after the n < N_STEPS test.
// Returns 0 when the streamline stops (domain or field check failed),
// 1 after a step without a saved point, 2 after a step that saved point q.
template <int MODEL, int LMAX, int ALGO, int CPAD>
__device__ __forceinline__ int track_step(const TrackParams& p, Lane& s, float (&c)[CPAD],
                                          float& qx, float& qy, float& qz)
{
    // domain.py:358-382 and field.py:88-114 share the voxel-space point when
    // both images have the same grid (the default of tg.tractogram).
    const float ax = dot4(p.dgrid.row0, s.px, s.py, s.pz, 1.0f);
    const float ay = dot4(p.dgrid.row1, s.px, s.py, s.pz, 1.0f);
    const float az = dot4(p.dgrid.row2, s.px, s.py, s.pz, 1.0f);
    const float vx = floorf(ax + 0.5f), vy = floorf(ay + 0.5f), vz = floorf(az + 0.5f);
    if (vx != s.dvx || vy != s.dvy || vz != s.dvz) {
        if (!(vx >= 0.0f && vx < (float)p.dgrid.nx && vy >= 0.0f && vy < (float)p.dgrid.ny &&
              vz >= 0.0f && vz < (float)p.dgrid.nz))
            return 0;
        const int64_t k = ((int64_t)(int32_t)vx * p.dgrid.ny + (int32_t)vy) * p.dgrid.nz + (int32_t)vz;
        if (__ldg(p.mask + k) == 0) return 0;
        s.dvx = vx;
        s.dvy = vy;
        s.dvz = vz;
    }
    float bx = ax, by = ay, bz = az;
    if (!p.same_grid) {
        bx = dot4(p.fgrid.row0, s.px, s.py, s.pz, 1.0f);
        by = dot4(p.fgrid.row1, s.px, s.py, s.pz, 1.0f);
        bz = dot4(p.fgrid.row2, s.px, s.py, s.pz, 1.0f);
    }
    const float fx = rintf(bx), fy = rintf(by), fz = rintf(bz);
    if (fx != s.fvx || fy != s.fvy || fz != s.fvz) {
        if (!(fx >= 0.0f && fx < (float)p.fgrid.nx && fy >= 0.0f && fy < (float)p.fgrid.ny &&
              fz >= 0.0f && fz < (float)p.fgrid.nz))
            return 0;
        const int64_t fv = ((int64_t)(int32_t)fx * p.fgrid.ny + (int32_t)fy) * p.fgrid.nz + (int32_t)fz;
        const float4* src = reinterpret_cast<const float4*>(p.field) + fv * (CPAD / 4);
#pragma unroll
        for (int k = 0; k < CPAD / 4; ++k) {
            const float4 v = __ldg(src + k);
            c[4 * k] = v.x;
            c[4 * k + 1] = v.y;
            c[4 * k + 2] = v.z;
            c[4 * k + 3] = v.w;
        }
        s.fvx = fx;
        s.fvy = fy;
        s.fvz = fz;
    }

    update_orientation<MODEL, LMAX, ALGO>(p.algo, c, s.ox, s.oy, s.oz, s.rng);
    s.steps += 1u;

    const float step = p.algo.step_size;
    s.px = fmaf(step, s.ox, s.px);
    s.py = fmaf(step, s.oy, s.py);
    s.pz = fmaf(step, s.oz, s.pz);
    s.time = s.time + step;
    if (s.time >= p.save_at) {
        s.time = s.time - p.save_at;
        qx = fmaf(-s.time, s.ox, s.px);
        qy = fmaf(-s.time, s.oy, s.py);
        qz = fmaf(-s.time, s.oz, s.pz);
        return 2;
    }
    return 1;
}

__device__ __forceinline__ void lane_init(Lane& s, float4 a, float4 b, uint32_t rng_seed,
                                          uint32_t stream_id, uint64_t index)
{
    s.px = a.x; s.py = a.y; s.pz = a.z;
    s.ox = b.x; s.oy = b.y; s.oz = b.z;
    s.time = 0.0f;
    s.n = 1;
    s.rng.mwc = rng_init(rng_seed, stream_id);
    s.rng.index = index;
    s.rng.step = 0u;
    s.dvx = s.dvy = s.dvz = __int_as_float(0x7fc00000);
    s.fvx = s.fvy = s.fvz = __int_as_float(0x7fc00000);
    s.steps = 0u;
}

}  // namespace tg

#endif  // TG_STEP_CUH
