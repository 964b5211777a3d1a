/*
 * tg_device.cuh -- per-step device arithmetic of the streamline tracker.
 *
 * Implements, for sm_100a, the reference tracking kernel's per-step work
 * (tractography/tracking.py:121-147): image-domain test (domain.py:358-382),
 * nearest-voxel field gather (field.py:88-114), local models
 * (local.py:91-120 spherical harmonics, local.py:212-230 tensor),
 * orientation updates (algorithm.py:83-112 Transport, 198-228 Diffusion),
 * the spherical exponential map (core.cl:101-109) and the random streams
 * (core.cl:180-245 MWC64X, plus a counter-based Philox4x32-10 mode).
 *
 * Every floating-point operation is an IEEE binary32 operation in a fixed
 * order with explicit fmaf; the translation unit is compiled with
 * -fmad=false so nothing is contracted behind our back.  This is the same
 * sequence the CPU oracle performs, which makes GPU and CPU results equal
 * bit for bit (the Transport update amplifies last-bit differences into
 * whole voxels, so tolerance-level agreement would not be reproducible).
 */
#ifndef TG_DEVICE_CUH
#define TG_DEVICE_CUH

#include <cstdint>

#include "tg_fmath.h"

namespace tg {

constexpr float kSoftmaxScale = 100.0f;   // local.py:17
constexpr float kSoftmaxInvScale = 0x1.47ae14p-7f;   // 1/100 rounded

template <int LMAX>
__device__ __forceinline__ void sh_eval(const float* c, float ct, float st, float cp, float sp,
                                        float* val, float* dth, float* dph);
template <int LMAX>
__device__ __forceinline__ void sh_basis(float ct, float st, float cp, float sp, float* Y);
template <int LMAX>
__device__ __forceinline__ void sh_eval_folded(const float* a, float ct, float st, float cp, float sp,
                                               float* val, float* dth, float* dph);

}  // namespace tg

#include "tg_sh_eval.cuh"
#include "tg_sh_fold.h"
#include "tg_sh_folded.cuh"

namespace tg {

enum { kModelSH = 0, kModelDTI = 1 };
enum { kTransport = 0, kDiffusion = 1 };
enum { kRngMWC64X = 0, kRngPhilox = 1 };

__host__ __device__ constexpr int n_coef_full(int lmax) { return (lmax + 1) * (lmax + 2) / 2; }

// OpenCL float max(): y if x < y else x.
__device__ __forceinline__ float cl_max(float x, float y) { return (x < y) ? y : x; }

// ---------------------------------------------------------------- RNG

struct Mwc {
    uint32_t x, c;
};

__device__ __forceinline__ uint32_t mwc64x(Mwc& s)
{
    constexpr uint32_t A = 4294883355u;
    const uint32_t res = s.x ^ s.c;
    const uint32_t hi = __umulhi(s.x, A);
    const uint32_t x = s.x * A + s.c;
    s.c = hi + (x < s.c ? 1u : 0u);
    s.x = x;
    return res;
}

__device__ __forceinline__ uint32_t rng_mix32(uint32_t v)
{
    v ^= v >> 16;
    v *= 0x7feb352du;
    v ^= v >> 15;
    v *= 0x846ca68bu;
    v ^= v >> 16;
    return v;
}

__device__ __forceinline__ Mwc rng_init(uint32_t seed, uint32_t id)
{
    Mwc s;
    uint32_t x = rng_mix32(seed ^ (id + 0x9e3779b9u));
    s.x = x < 1u ? 1u : x;
    s.c = rng_mix32(seed + id * 0x85ebca6bu) % 4294883355u;
    return s;
}

__device__ __forceinline__ float randu(Mwc& s)
{
    return (float)(mwc64x(s) >> 8) * 0x1p-24f;
}

__device__ __forceinline__ uint32_t randi(Mwc& s, uint32_t max)
{
    return (uint32_t)(randu(s) * (float)max);
}

__device__ __forceinline__ float randn(Mwc& s)
{
    float n = randu(s);
    while (n <= 0.0f) n = randu(s);   // terminates: 2^-24 resolution, MWC64X period ~2^63
    const float radius = sqrtf(-2.0f * tgm_log_pos(n));
    // cos(2 pi randu): the same draw, as its 24-bit integer
    return radius * tgm_cos2pi_u24(mwc64x(s) >> 8);
}

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ void philox_normal2(uint64_t key, uint64_t index, uint32_t step,
                                               float* n1, float* n2)
{
    const uint4 w = philox4x32_10(make_uint4((uint32_t)index, (uint32_t)(index >> 32), step, 0x5eedu),
                                  make_uint2((uint32_t)key, (uint32_t)(key >> 32)));
    const float u1 = (float)((w.x >> 8) + 1u) * 0x1p-24f;
    const float u2 = (float)(w.y >> 8) * 0x1p-24f;
    const float radius = sqrtf(-2.0f * tgm_log_pos(u1));
    float s, c;
    tgm_sincosf(TGM_TWO_PI * u2, &s, &c);
    *n1 = radius * c;
    *n2 = radius * s;
}

// ----------------------------------------------------------- geometry

struct Frame {
    float ct, st, cp, sp;
};

// cart2sph (core.cl:142-153) as direction cosines of colatitude/azimuth:
// ct = z/r, st = rho/r, cp = x/rho, sp = y/rho.  Orientations leave the
// exponential map with |o|^2 = 1 within a few ulp; for |r^2 - 1| < 2^-14,
// 1/r = 1.5 - r^2/2 to within 1.4e-9 relative (its expansion about 1), far
// inside binary32 rounding, and 1/rho comes from tgm_rsqrt_pos (rho^2 at
// least 2^-100; nearer the axis from a square root and a division).
// Otherwise both reciprocals come from one division, 1/r = rho q and
// 1/rho = r q with q = 1/(r rho); on the axis (r rho rounds to 0) phi is
// taken as 0.
__device__ __forceinline__ Frame frame_of(float x, float y, float z)
{
    Frame f;
    const float rho2 = fmaf(y, y, x * x);
    const float r2 = fmaf(z, z, rho2);
    if (fabsf(r2 - 1.0f) < 0x1p-14f) {
        const float ir = fmaf(-0.5f, r2, 1.5f);
        f.ct = fminf(fmaxf(z * ir, -1.0f), 1.0f);
        if (rho2 >= 0x1p-100f) {
            // 1/rho without a square root or a division; rho = rho2 / rho
            const float irho = tgm_rsqrt_pos(rho2);
            f.st = fminf((rho2 * irho) * ir, 1.0f);
            f.cp = x * irho;
            f.sp = y * irho;
            return f;
        }
        const float rho = sqrtf(rho2);
        f.st = fminf(rho * ir, 1.0f);
        if (rho > 0.0f) {
            const float irho = 1.0f / rho;
            f.cp = x * irho;
            f.sp = y * irho;
        } else {
            f.cp = 1.0f;
            f.sp = 0.0f;
        }
        return f;
    }
    const float r = sqrtf(r2);
    if (r <= 0.0f) {
        f.ct = 1.0f; f.st = 0.0f; f.cp = 1.0f; f.sp = 0.0f;
        return f;
    }
    const float rho = sqrtf(rho2);
    const float rr = r * rho;
    if (rr > 0.0f) {
        const float q = 1.0f / rr;
        const float ir = rho * q, irho = r * q;
        f.ct = fminf(fmaxf(z * ir, -1.0f), 1.0f);
        f.st = fminf(rho * ir, 1.0f);
        f.cp = x * irho;
        f.sp = y * irho;
    } else {
        f.ct = fminf(fmaxf(z / r, -1.0f), 1.0f);
        f.st = 0.0f;
        f.cp = 1.0f;
        f.sp = 0.0f;
    }
    return f;
}

__device__ __forceinline__ float dot4(float4 a, float x, float y, float z, float w)
{
    return fmaf(a.w, w, fmaf(a.z, z, fmaf(a.y, y, a.x * x)));
}

// ------------------------------------------------------------- models

struct ModelValue {
    float value, dtheta, dphi;
    float inv;   // 1 / max(value, 1e-6), the drift's divisor (algorithm.py:98, :216)
};

// core.cl:111-115 (the seeding kernel's model value; tracking uses tgm_softplus)
__device__ __forceinline__ float softmax(float x, float k)
{
    if (x * k < 30.0f) return tgm_logf(1.0f + tgm_expf(k * x)) / k;
    return x;
}

// local.py:91-120 from folded coefficients (tgsh_fold): the field the
// trackers read is folded once per voxel when it is created.
template <int LMAX>
__device__ __forceinline__ ModelValue sh_model(const float* folded, const Frame& f)
{
    ModelValue r;
    float raw, d;
    sh_eval_folded<LMAX>(folded, f.ct, f.st, f.cp, f.sp, &raw, &r.dtheta, &r.dphi);
    // local.py:106-118: softplus of the value, derivatives times its slope
    tgm_softplus(raw, kSoftmaxScale, kSoftmaxInvScale, &r.value, &d, &r.inv);
    r.dtheta = r.dtheta * d;
    r.dphi = r.dphi * d;
    return r;
}

__device__ __forceinline__ ModelValue dti_model(const float* m, float x, float y, float z, const Frame& f)
{
    const float dux = fmaf(m[4], z, fmaf(m[3], y, m[0] * x));
    const float duy = fmaf(m[5], z, fmaf(m[1], y, m[3] * x));
    const float duz = fmaf(m[2], z, fmaf(m[5], y, m[4] * x));
    ModelValue r;
    r.value = fmaf(z, duz, fmaf(y, duy, x * dux));
    const float etx = f.ct * f.cp, ety = f.ct * f.sp, etz = -f.st;
    r.dtheta = 2.0f * fmaf(duz, etz, fmaf(duy, ety, dux * etx));
    r.dphi = 2.0f * fmaf(duy, f.cp, dux * (-f.sp));
    r.inv = 1.0f / cl_max(r.value, 1e-6f);
    return r;
}

template <int MODEL, int LMAX>
__device__ __forceinline__ ModelValue model_eval(const float* c, float x, float y, float z, const Frame& f)
{
    if constexpr (MODEL == kModelDTI) {
        return dti_model(c, x, y, z, f);
    } else {
        return sh_model<LMAX>(c, f);
    }
}

// --------------------------------------------------------- algorithms

struct AlgoParams {
    float step_size;
    float gamma;
    float noise_variance;
    float scale_drift;   // gamma * step_size
    float scale_noise;   // sqrt(noise_variance * gamma * step_size)
    int32_t rng_mode;
    uint64_t philox_key;
};

struct RngState {
    Mwc mwc;
    uint64_t index;
    uint32_t step;
};

__device__ __forceinline__ void exps2(float& ox, float& oy, float& oz, float tx, float ty, float tz)
{
    const float n2 = fmaf(tz, tz, fmaf(ty, ty, tx * tx));
    if (n2 <= 0.0f) return;
    float c, k;
    tgm_exps2_factors(n2, &c, &k);
    ox = fmaf(tx, k, c * ox);
    oy = fmaf(ty, k, c * oy);
    oz = fmaf(tz, k, c * oz);
}

template <int MODEL, int LMAX, int ALGO>
__device__ __forceinline__ void update_orientation(const AlgoParams& a, const float* c,
                                                   float& ox, float& oy, float& oz, RngState& rng)
{
    const Frame f = frame_of(ox, oy, oz);
    const ModelValue mv = model_eval<MODEL, LMAX>(c, ox, oy, oz, f);
    const float etx = f.ct * f.cp, ety = f.ct * f.sp, etz = -f.st;
    const float epx = -f.sp, epy = f.cp;
    const float inv = mv.inv;
    const float gx = fmaf(mv.dphi, epx, mv.dtheta * etx);
    const float gy = fmaf(mv.dphi, epy, mv.dtheta * ety);
    const float gz = mv.dtheta * etz;
    const float dx = gx * inv, dy = gy * inv, dz = gz * inv;
    float tx, ty, tz;
    if constexpr (ALGO == kTransport) {
        tx = a.scale_drift * dx;
        ty = a.scale_drift * dy;
        tz = a.scale_drift * dz;
    } else {
        float nx = 0.0f, ny = 0.0f, nz = 0.0f;
        if (a.noise_variance > 0.0f) {
            float n1, n2;
            if (a.rng_mode == kRngMWC64X) {
                n1 = randn(rng.mwc);
                n2 = randn(rng.mwc);
            } else {
                philox_normal2(a.philox_key, rng.index, rng.step, &n1, &n2);
            }
            nx = fmaf(n2, epx, n1 * etx);
            ny = fmaf(n2, epy, n1 * ety);
            nz = n1 * etz;
        }
        tx = fmaf(a.scale_noise, nx, a.scale_drift * dx);
        ty = fmaf(a.scale_noise, ny, a.scale_drift * dy);
        tz = fmaf(a.scale_noise, nz, a.scale_drift * dz);
    }
    exps2(ox, oy, oz, tx, ty, tz);
    if constexpr (ALGO != kTransport) rng.step += 1u;
}

// ----------------------------------------------------- domain / field

struct Grid {
    float4 row0, row1, row2;   // inverse affine rows 0..2
    uint32_t nx, ny, nz;
};

// domain.py:358-382: voxel = floor(v + 0.5), half-open cells; -1 outside.
__device__ __forceinline__ int64_t voxel_floor_half(const Grid& g, float x, float y, float z)
{
    const float vx = floorf(dot4(g.row0, x, y, z, 1.0f) + 0.5f);
    const float vy = floorf(dot4(g.row1, x, y, z, 1.0f) + 0.5f);
    const float vz = floorf(dot4(g.row2, x, y, z, 1.0f) + 0.5f);
    if (!(vx >= 0.0f && vx < (float)g.nx && vy >= 0.0f && vy < (float)g.ny && vz >= 0.0f && vz < (float)g.nz))
        return -1;
    return ((int64_t)(int32_t)vx * g.ny + (int32_t)vy) * g.nz + (int32_t)vz;
}

// field.py:88-114: voxel = rint(v) (ties to even); -1 outside.
__device__ __forceinline__ int64_t voxel_rint(const Grid& g, float x, float y, float z)
{
    const float vx = rintf(dot4(g.row0, x, y, z, 1.0f));
    const float vy = rintf(dot4(g.row1, x, y, z, 1.0f));
    const float vz = rintf(dot4(g.row2, x, y, z, 1.0f));
    if (!(vx >= 0.0f && vx < (float)g.nx && vy >= 0.0f && vy < (float)g.ny && vz >= 0.0f && vz < (float)g.nz))
        return -1;
    return ((int64_t)(int32_t)vx * g.ny + (int32_t)vy) * g.nz + (int32_t)vz;
}

}  // namespace tg

#endif  // TG_DEVICE_CUH
