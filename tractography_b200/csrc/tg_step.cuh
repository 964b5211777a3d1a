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

// Resident blocks of 128 lanes per SM that the persistent kernels are
// compiled for: 5 (at most 102 registers), except the closed-surface
// variants of the larger SH bands, whose coefficients plus surface-test
// state do not fit 102 registers without spilling (4 blocks, 128), and the
// closed-surface tensor variant, whose few coefficients leave room for 6 (85).
template <int MODEL, int LMAX, int DOM>
constexpr int persistent_min_blocks()
{
    return DOM == kDomainMesh ? (MODEL == kModelDTI ? 6 : (LMAX >= 6 ? 4 : 5)) : 5;
}

struct Lane {
    float px, py, pz;
    float ox, oy, oz;
    float time;
    uint32_t n;
    RngState rng;
    // Voxel cache of the last domain test and field gather; while it holds,
    // the mask bit (inside) and the coefficients in registers are still
    // valid, so the voxel rounding, bounds tests, index arithmetic and loads
    // are skipped.  Domain and field on one grid: the open interval
    // (dv, fv) per axis in which both voxels are unchanged.  Otherwise (and
    // for closed surfaces, fv only): the rounded voxel coordinates of the
    // domain test (dv) and the field gather (fv).  NaN forces an evaluation.
    float dvx, dvy, dvz;
    float fvx, fvy, fvz;
    uint32_t steps;
    // closed-surface domain: the point of the last passed domain test, and
    // the seed's inside test when a pre-pass computed it (0: not known, test
    // here; 1: inside; 2: outside)
    float lx, ly, lz;
    uint32_t seed_state;
};

// One iteration of tracking.py:121-147 after the n < N_STEPS test.
// Returns 0 when the streamline stops (domain or field check failed),
// 1 after a step without a saved point, 2 after a step that saved point q.
//
// DOM selects the domain test: the image mask (domain.py:358-382), or a
// closed surface, where the seed must be inside and every later point must
// be reached by a segment from the previous one that does not hit the
// surface (the found flag of bvh.cl:83-131).
// The domain test and the field gather of one iteration (tracking.py:123-
// 133): false when the streamline stops; otherwise c holds the coefficients
// of the nearest field voxel.
// `surface` (closed surface, after the first step): the segment test's
// answer when the caller computed it for the whole warp (0 clear, 1
// blocked), -1 to compute it here.
template <int MODEL, int LMAX, int CPAD, int DOM>
__device__ __forceinline__ bool locate(const TrackParams& p, Lane& s, float (&c)[CPAD], int surface = -1)
{
    float ax, ay, az;
    if constexpr (DOM == kDomainMesh) {
        if (s.steps == 0u) {
            const bool inside = s.seed_state == 0u ? mesh_contains(p.mesh, s.px, s.py, s.pz) : s.seed_state == 1u;
            if (!inside) return false;
        } else if (surface >= 0 ? surface != 0 : mesh_segment_blocked(p.mesh, s.lx, s.ly, s.lz, s.px, s.py, s.pz)) {
            return false;
        }
        s.lx = s.px;
        s.ly = s.py;
        s.lz = s.pz;
        ax = dot4(p.fgrid.row0, s.px, s.py, s.pz, 1.0f);
        ay = dot4(p.fgrid.row1, s.px, s.py, s.pz, 1.0f);
        az = dot4(p.fgrid.row2, s.px, s.py, s.pz, 1.0f);
    } else {
        // domain.py:358-382 and field.py:88-114 share the voxel-space point
        // when both images have the same grid (the default of tg.tractogram).
        ax = dot4(p.dgrid.row0, s.px, s.py, s.pz, 1.0f);
        ay = dot4(p.dgrid.row1, s.px, s.py, s.pz, 1.0f);
        az = dot4(p.dgrid.row2, s.px, s.py, s.pz, 1.0f);
        if (p.same_grid) {
            // For a voxel f and f - 0.5 < a < f + 0.5 (open), rint(a) = f and
            // floor(fl(a + 0.5)) = f: the sum lies in [f, f + 1) after rounding
            // (f is representable and a + 0.5 < f + 1 rounds to at most a
            // value below f + 1 for |a| < 2^22).  So six comparisons with the
            // cached interval certify both voxels unchanged.
            if (ax > s.dvx && ax < s.fvx && ay > s.dvy && ay < s.fvy && az > s.dvz && az < s.fvz) return true;
            const float vx = floorf(ax + 0.5f), vy = floorf(ay + 0.5f), vz = floorf(az + 0.5f);
            const float fx = rintf(ax), fy = rintf(ay), fz = rintf(az);
            if (!(vx >= 0.0f && vx < (float)p.dgrid.nx && vy >= 0.0f && vy < (float)p.dgrid.ny && vz >= 0.0f &&
                  vz < (float)p.dgrid.nz))
                return false;
            if (!(fx >= 0.0f && fx < (float)p.fgrid.nx && fy >= 0.0f && fy < (float)p.fgrid.ny && fz >= 0.0f &&
                  fz < (float)p.fgrid.nz))
                return false;
            const int64_t k = ((int64_t)(int32_t)vx * p.dgrid.ny + (int32_t)vy) * p.dgrid.nz + (int32_t)vz;
            const uint8_t inside = __ldg(p.mask + k);
            const int64_t fv = ((int64_t)(int32_t)fx * p.fgrid.ny + (int32_t)fy) * p.fgrid.nz + (int32_t)fz;
            const float4* src = reinterpret_cast<const float4*>(p.field) + fv * (CPAD / 4);
#pragma unroll
            for (int k4 = 0; k4 < CPAD / 4; ++k4) {
                const float4 v = __ldg(src + k4);
                c[4 * k4] = v.x;
                c[4 * k4 + 1] = v.y;
                c[4 * k4 + 2] = v.z;
                c[4 * k4 + 3] = v.w;
            }
            if (inside == 0) return false;
            // a point on a voxel face (a = f + 0.5 exactly) has different
            // domain and field voxels: leave the cache invalid
            const bool tie = vx != fx || vy != fy || vz != fz;
            const float nan = __int_as_float(0x7fc00000);
            s.dvx = tie ? nan : fx - 0.5f;
            s.dvy = tie ? nan : fy - 0.5f;
            s.dvz = tie ? nan : fz - 0.5f;
            s.fvx = tie ? nan : fx + 0.5f;
            s.fvy = tie ? nan : fy + 0.5f;
            s.fvz = tie ? nan : fz + 0.5f;
            return true;
        }
        const float vx = floorf(ax + 0.5f), vy = floorf(ay + 0.5f), vz = floorf(az + 0.5f);
        const float bx = dot4(p.fgrid.row0, s.px, s.py, s.pz, 1.0f);
        const float by = dot4(p.fgrid.row1, s.px, s.py, s.pz, 1.0f);
        const float bz = dot4(p.fgrid.row2, s.px, s.py, s.pz, 1.0f);
        const float fx = rintf(bx), fy = rintf(by), fz = rintf(bz);
        const bool dchange = vx != s.dvx || vy != s.dvy || vz != s.dvz;
        const bool fchange = fx != s.fvx || fy != s.fvy || fz != s.fvz;
        // Every failed test stops the streamline the same way, so both bounds
        // tests come first and the mask byte and the coefficients are then
        // fetched together: one memory round trip per voxel change, not two.
        // (A streamline stopped by its mask leaves c overwritten; nothing
        // reads c after a stop.)
        if (dchange && !(vx >= 0.0f && vx < (float)p.dgrid.nx && vy >= 0.0f && vy < (float)p.dgrid.ny &&
                         vz >= 0.0f && vz < (float)p.dgrid.nz))
            return false;
        if (fchange && !(fx >= 0.0f && fx < (float)p.fgrid.nx && fy >= 0.0f && fy < (float)p.fgrid.ny &&
                         fz >= 0.0f && fz < (float)p.fgrid.nz))
            return false;
        uint8_t inside = 1;
        if (dchange) {
            const int64_t k = ((int64_t)(int32_t)vx * p.dgrid.ny + (int32_t)vy) * p.dgrid.nz + (int32_t)vz;
            inside = __ldg(p.mask + k);
        }
        if (fchange) {
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
        }
        if (inside == 0) return false;
        if (dchange) {
            s.dvx = vx;
            s.dvy = vy;
            s.dvz = vz;
        }
        if (fchange) {
            s.fvx = fx;
            s.fvy = fy;
            s.fvz = fz;
        }
        return true;
    }
    // closed surface: the field gather of the point (ax, ay, az are field-voxel coordinates)
    const float fx = rintf(ax), fy = rintf(ay), fz = rintf(az);
    if (fx != s.fvx || fy != s.fvy || fz != s.fvz) {
        if (!(fx >= 0.0f && fx < (float)p.fgrid.nx && fy >= 0.0f && fy < (float)p.fgrid.ny &&
              fz >= 0.0f && fz < (float)p.fgrid.nz))
            return false;
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
    return true;
}

template <int MODEL, int LMAX, int ALGO, int CPAD, int DOM = kDomainImage>
__device__ __forceinline__ int track_step(const TrackParams& p, Lane& s, float (&c)[CPAD],
                                          float& qx, float& qy, float& qz, int surface = -1)
{
    if (!locate<MODEL, LMAX, CPAD, DOM>(p, s, c, surface)) return 0;
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

// domain.py:95-120 domain_sample_boundary: a point uniform over the
// boundary's area (triangle by the normalised cumulative areas), its inward
// normal, the point moved 1e-4 inward; three draws from st.  Vector
// operations in the reference's order (normalize = v / length(v)).
__device__ __forceinline__ void sample_boundary(const float4* __restrict__ vertices,
                                               const uint4* __restrict__ triangles,
                                               const float* __restrict__ cumulative, uint32_t n_triangles,
                                               Mwc& st, float& px, float& py, float& pz, float& ox, float& oy,
                                               float& oz, uint32_t* triangle = nullptr, float* bary = nullptr)
{
    const float target = randu(st);
    uint32_t lo = 0, hi = n_triangles;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (cumulative[mid] <= target) lo = mid + 1;
        else hi = mid;
    }
    const uint32_t tri = lo < n_triangles - 1 ? lo : n_triangles - 1;
    const uint4 ix = triangles[tri];
    const float4 a = vertices[ix.x], b = vertices[ix.y], c = vertices[ix.z];
    const float root_u = sqrtf(randu(st));
    const float v = randu(st);
    const float wa = 1.0f - root_u, wb = root_u * (1.0f - v), wc = root_u * v;
    if (triangle != nullptr) {
        *triangle = tri;
        bary[0] = wa;
        bary[1] = wb;
        bary[2] = wc;
    }
    const float sx = (wa * a.x + wb * b.x) + wc * c.x;
    const float sy = (wa * a.y + wb * b.y) + wc * c.y;
    const float sz = (wa * a.z + wb * b.z) + wc * c.z;
    const float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
    const float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
    const float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);
    ox = -(nx / len);
    oy = -(ny / len);
    oz = -(nz / len);
    px = sx + 1e-4f * ox;
    py = sy + 1e-4f * oy;
    pz = sz + 1e-4f * oz;
}

// A live streamline handed from one round of a persistent launch to the
// next (tail compaction): everything the step reads, plus its output
// cursor.  The voxel caches are not carried; the next step reloads them,
// which gives the same values.
struct __align__(16) LaneCarry {
    float px, py, pz, time;
    float ox, oy, oz, lx;
    float ly, lz;
    uint32_t n, steps;
    uint32_t mwc_x, mwc_c, rng_step, item;
    uint64_t rng_index;
    int32_t chunk;
    uint32_t fill;
    uint32_t job;            // job slot (multi-request serving); 0 otherwise
};

// RNG: the streamline draws random numbers (Diffusion); Transport draws
// none, so its RNG state is neither carried nor kept in registers.
template <bool RNG = true>
__device__ __forceinline__ void lane_save(LaneCarry* dst, const Lane& s, uint32_t item, int32_t chunk,
                                          uint32_t fill, uint32_t job = 0u)
{
    LaneCarry c;
    c.job = job;
    c.px = s.px; c.py = s.py; c.pz = s.pz; c.time = s.time;
    c.ox = s.ox; c.oy = s.oy; c.oz = s.oz; c.lx = s.lx;
    c.ly = s.ly; c.lz = s.lz; c.n = s.n; c.steps = s.steps;
    c.item = item;
    if (RNG) {
        c.mwc_x = s.rng.mwc.x; c.mwc_c = s.rng.mwc.c; c.rng_step = s.rng.step;
        c.rng_index = s.rng.index;
    } else {
        c.mwc_x = 0u; c.mwc_c = 0u; c.rng_step = 0u;
        c.rng_index = 0ull;
    }
    c.chunk = chunk;
    c.fill = fill;
    *dst = c;
}

template <bool RNG = true>
__device__ __forceinline__ void lane_restore(Lane& s, const LaneCarry& c, uint32_t& item, int32_t& chunk,
                                             uint32_t& fill)
{
    s.px = c.px; s.py = c.py; s.pz = c.pz; s.time = c.time;
    s.ox = c.ox; s.oy = c.oy; s.oz = c.oz; s.lx = c.lx;
    s.ly = c.ly; s.lz = c.lz; s.n = c.n; s.steps = c.steps;
    item = c.item;
    if (RNG) {
        s.rng.mwc.x = c.mwc_x; s.rng.mwc.c = c.mwc_c; s.rng.step = c.rng_step;
        s.rng.index = c.rng_index;
    }
    s.dvx = s.dvy = s.dvz = __int_as_float(0x7fc00000);
    s.fvx = s.fvy = s.fvz = __int_as_float(0x7fc00000);
    s.seed_state = 0u;
    chunk = c.chunk;
    fill = c.fill;
}

// Adds the steps of the warp's lanes to *total, one atomic per warp; called
// by all 32 lanes together.
__device__ __forceinline__ void add_steps64(unsigned long long* total, unsigned long long steps)
{
    if (total == nullptr) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) steps += __shfl_xor_sync(0xffffffffu, steps, o);
    if ((threadIdx.x & 31u) == 0u) atomicAdd(total, steps);
}

// Tail compaction rule, evaluated by whole warps: once a lane of the warp
// has found its queue empty (so the warp is not full), a warp with at most
// `compact_lanes` live lanes hands them to the next round and exits.
__device__ __forceinline__ bool warp_should_compact(unsigned active, uint32_t compact_lanes)
{
    return active != 0xffffffffu && (uint32_t)__popc(active) <= compact_lanes;
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
    s.lx = a.x;
    s.ly = a.y;
    s.lz = a.z;
    s.seed_state = 0u;
}

}  // namespace tg

#endif  // TG_STEP_CUH
