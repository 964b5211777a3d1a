/*
 * tg_oracle.c -- CPU oracle (test infrastructure only; see tg_oracle.h).
 *
 * Restates, in plain C, the reference's tracking kernel
 * (tractography/tracking.py:93-149) with its plugins: image domain
 * (domain.py:358-382), image field (field.py:88-114), spherical-harmonic and
 * tensor local models (local.py:91-120, 212-230; spharm.cl:216-413;
 * core.cl:111-120, 142-153), Transport and Diffusion updates
 * (algorithm.py:83-112, 198-228; core.cl:101-109), the MWC64X stream
 * (core.cl:180-245) and FOD seeding (seeds.cl:12-118, seeds.py:174-216).
 *
 * Build: gcc -O2 -std=c99 -ffp-contract=off -fopenmp (see oracle/Makefile).
 */
#include "tg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "tg_fmath.h"
#include "tg_sh_table.h"
#include "tg_sh_fold.h"

#define N_DIRECTIONS 1000
#define SOFTMAX_SCALE 100.0f
#define SOFTMAX_INV_SCALE 0x1.47ae14p-7f   /* 1/100 rounded */

/* OpenCL max()/min() on floats (x < y ? y : x), core to the reference's
 * max(value, 1e-6f) and max(value, 0.0f). */
static float cl_maxf(float x, float y) { return (x < y) ? y : x; }

/* ------------------------------------------------------------------ */
/* RNG: core.cl:180-245                                                */
/* ------------------------------------------------------------------ */

static uint32_t mwc64x(uint32_t s[2])
{
    const uint32_t A = 4294883355u;                 /* core.cl:182 */
    uint32_t x = s[0], c = s[1];
    const uint32_t res = x ^ c;
    const uint32_t hi = (uint32_t)(((uint64_t)x * A) >> 32);
    x = x * A + c;
    c = hi + (x < c);
    s[0] = x;
    s[1] = c;
    return res;
}

static uint32_t rng_mix32(uint32_t v)               /* core.cl:193-201 */
{
    v ^= v >> 16;
    v *= 0x7feb352du;
    v ^= v >> 15;
    v *= 0x846ca68bu;
    v ^= v >> 16;
    return v;
}

void tgo_rng_init(uint32_t seed, uint32_t id, uint32_t s[2])   /* core.cl:203-208 */
{
    uint32_t x = rng_mix32(seed ^ (id + 0x9e3779b9u));
    if (x < 1u) x = 1u;
    s[0] = x;
    s[1] = rng_mix32(seed + id * 0x85ebca6bu) % 4294883355u;
}

static float randu(uint32_t s[2])                    /* core.cl:212-214 */
{
    return (float)(mwc64x(s) >> 8) * 0x1p-24f;
}

static uint32_t randi(uint32_t s[2], uint32_t max)   /* core.cl:227-229 */
{
    return (uint32_t)(randu(s) * (float)max);
}

static float randn(uint32_t s[2])                    /* core.cl:240-245 */
{
    float n = randu(s);
    while (n <= 0.0f) n = randu(s);
    const float radius = sqrtf(-2.0f * tgm_log_pos(n));
    /* cos(2 pi randu): the same draw, as its 24-bit integer */
    return radius * tgm_cos2pi_u24(mwc64x(s) >> 8);
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter-based stream
 * keyed by (seed index, step), used by the optional keyed mode. */
void tgo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Two standard normals for (seed index, step) under a key: Box-Muller on
 * u1 = ((w0 >> 8) + 1) 2^-24 in (0, 1] and u2 = (w1 >> 8) 2^-24. */
static void philox_normal2(uint64_t key, uint64_t index, uint32_t step, float* n1, float* n2)
{
    const uint32_t ctr[4] = {(uint32_t)index, (uint32_t)(index >> 32), step, 0x5eedu};
    const uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
    uint32_t w[4];
    tgo_philox(ctr, k, w);
    const float u1 = (float)((w[0] >> 8) + 1u) * 0x1p-24f;
    const float u2 = (float)(w[1] >> 8) * 0x1p-24f;
    const float radius = sqrtf(-2.0f * tgm_log_pos(u1));
    float s, c;
    tgm_sincosf(TGM_TWO_PI * u2, &s, &c);
    *n1 = radius * c;
    *n2 = radius * s;
}

/* ------------------------------------------------------------------ */
/* Geometry: core.cl:142-153 (cart2sph) expressed as the frame        */
/* cos/sin of colatitude and azimuth.                                 */
/* ------------------------------------------------------------------ */

typedef struct { float ct, st, cp, sp; } frame_t;

static frame_t frame_of(float x, float y, float z)
{
    frame_t f;
    const float rho2 = fmaf(y, y, x * x);
    const float r2 = fmaf(z, z, rho2);
    if (fabsf(r2 - 1.0f) < 0x1p-14f) {               /* near unit: 1/r = 1.5 - r^2/2 */
        const float ir = fmaf(-0.5f, r2, 1.5f);
        f.ct = fminf(fmaxf(z * ir, -1.0f), 1.0f);
        if (rho2 >= 0x1p-100f) {                     /* 1/rho by tgm_rsqrt_pos */
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
    if (r <= 0.0f) {                                 /* core.cl:144-146 */
        f.ct = 1.0f; f.st = 0.0f; f.cp = 1.0f; f.sp = 0.0f;
        return f;
    }
    /* off the axis, 1/r = rho q and 1/rho = r q with q = 1/(r rho) */
    const float rho = sqrtf(rho2);
    const float rr = r * rho;
    if (rr > 0.0f) {
        const float q = 1.0f / rr;
        const float ir = rho * q, irho = r * q;
        f.ct = fminf(fmaxf(z * ir, -1.0f), 1.0f);    /* core.cl:151 clamp */
        f.st = fminf(rho * ir, 1.0f);
        f.cp = x * irho;
        f.sp = y * irho;
    } else {                                         /* atan2(0, 0) = 0 */
        f.ct = fminf(fmaxf(z / r, -1.0f), 1.0f);
        f.st = 0.0f;
        f.cp = 1.0f;
        f.sp = 0.0f;
    }
    return f;
}

/* x.row of a row-major 4x4 matrix (used for both the inverse affines of
 * domain.py:362-366 / field.py:92-96 and apply_affine of core.cl:164-170). */
static float dot4(const float* a, float x, float y, float z, float w)
{
    return fmaf(a[3], w, fmaf(a[2], z, fmaf(a[1], y, a[0] * x)));
}

/* ------------------------------------------------------------------ */
/* Local models                                                        */
/* ------------------------------------------------------------------ */

/* value, d/dtheta, (d/dphi)/sin(theta), and 1 / max(value, 1e-6) (the
 * drift's divisor, algorithm.py:98, :216) */
typedef struct { float value, dtheta, dphi, inv; } model_value_t;

static int lmax_for(uint32_t n_params)
{
    int l = 0;
    while ((uint32_t)((l + 1) * (l + 2) / 2) < n_params) l += 2;
    return l;
}

static float horner_u(const float* a, int n, float u)
{
    float h = a[n - 1];
    for (int j = n - 2; j >= 0; --j) h = fmaf(h, u, a[j]);
    return h;
}

/* core.cl:111-120 */
static float softmax(float x, float k)
{
    if (x * k < 30.0f) return tgm_logf(1.0f + tgm_expf(k * x)) / k;
    return x;
}


/* The folded evaluation: tgsh_fold turned the coefficients of each order m
 * and part (cos: index +m, sin: index -m) into one polynomial S(u) in
 * u = cos^2(theta), highest power first, so that the part's sum over l is
 * x^p S(u) with p = m & 1 and x = cos(theta).  Per block, S and S' by one
 * Horner pass, A = x^p S and dA/dx; then the same combination into value,
 * d/dtheta and (d/dphi)/sin(theta).  The tracking kernels run
 * this operation sequence straight-line (tg_sh_folded.cuh). */
static model_value_t sh_folded(const float* a, int lmax, frame_t f)
{
    const float ct = f.ct, st = f.st, cp = f.cp, sp = f.sp;
    const float u = ct * ct;
    const float x2 = ct + ct;
    const float u2 = u + u;
    const float tc = cp + cp;
    float cm[TG_SH_LMAX + 1], sm[TG_SH_LMAX + 1], stp[TG_SH_LMAX + 2];
    cm[0] = 1.0f; sm[0] = 0.0f;
    cm[1] = cp; sm[1] = sp;
    for (int m = 2; m <= lmax; ++m) {
        cm[m] = fmaf(tc, cm[m - 1], -cm[m - 2]);
        sm[m] = fmaf(tc, sm[m - 1], -sm[m - 2]);
    }
    stp[0] = 1.0f;
    for (int k = 1; k <= lmax + 1; ++k) stp[k] = stp[k - 1] * st;

    model_value_t r = {0.0f, 0.0f, 0.0f, 0.0f};
    int off = 0;
    for (int m = 0; m <= lmax; ++m) {
        const int parity = m & 1;
        const int K = (lmax - m - parity) / 2 + 1;     /* even l in [m, lmax] */
        float X[2] = {0.0f, 0.0f}, Xp[2] = {0.0f, 0.0f};
        int deriv = 0;
        for (int part = 0; part < (m == 0 ? 1 : 2); ++part) {
            const float* blk = a + off;
            off += K;
            float S, D = 0.0f;
            if (K == 1) {
                S = blk[0];
            } else {
                D = blk[0];
                S = fmaf(blk[0], u, blk[1]);
                for (int t = 2; t < K; ++t) {
                    D = fmaf(D, u, S);
                    S = fmaf(S, u, blk[t]);
                }
            }
            if (parity) {
                X[part] = S * ct;
                Xp[part] = K == 1 ? S : fmaf(u2, D, S);
                deriv = 1;
            } else {
                X[part] = S;
                if (K > 1) {
                    Xp[part] = x2 * D;
                    deriv = 1;
                }
            }
        }
        const float A = X[0], Ap = Xp[0], B = X[1], Bp = Xp[1];
        if (m == 0) {
            r.value = r.value + A;
            if (deriv) r.dtheta = fmaf(-stp[1], Ap, r.dtheta);
        } else {
            const float F = fmaf(B, sm[m], A * cm[m]);
            const float G = fmaf(-A, sm[m], B * cm[m]);
            r.value = fmaf(stp[m], F, r.value);
            const float mw = (float)m * stp[m - 1];
            const float wct = mw * ct;
            r.dtheta = fmaf(wct, F, r.dtheta);
            if (deriv) {
                const float Fp = fmaf(Bp, sm[m], Ap * cm[m]);
                r.dtheta = fmaf(-stp[m + 1], Fp, r.dtheta);
            }
            r.dphi = fmaf(mw, G, r.dphi);
        }
    }
    return r;
}

/* The coefficients the tracking loop evaluates (tg_field_create does the same
 * per voxel on the device): SH coefficients zero-padded to the full band of
 * lmax_for(n_params) and folded (tgsh_fold), tensor coefficients as given. */
static void model_coefficients(int32_t model, const float* params, uint32_t n_params, float* out)
{
    if (model == TGO_MODEL_DTI) {
        for (int i = 0; i < 6; ++i) out[i] = params[i];
        return;
    }
    float c[48];
    const int lmax = lmax_for(n_params);
    const int full = (lmax + 1) * (lmax + 2) / 2;
    for (int i = 0; i < full; ++i) c[i] = (uint32_t)i < n_params ? params[i] : 0.0f;
    tgsh_fold(lmax, c, out);
}

/* local.py:91-120 from folded coefficients */
static model_value_t sh_model(const float* folded, uint32_t n_params, frame_t f)
{
    model_value_t r = sh_folded(folded, lmax_for(n_params), f);
    /* core.cl:111-120 softmax and dsoftmax from one exponential */
    float d;
    tgm_softplus(r.value, SOFTMAX_SCALE, SOFTMAX_INV_SCALE, &r.value, &d, &r.inv);
    r.dtheta = r.dtheta * d;
    r.dphi = r.dphi * d;
    return r;
}

/* local.py:212-230 (orientation used as given, angles from its direction). */
static model_value_t dti_model(const float* m, float x, float y, float z, frame_t f)
{
    const float dux = fmaf(m[4], z, fmaf(m[3], y, m[0] * x));
    const float duy = fmaf(m[5], z, fmaf(m[1], y, m[3] * x));
    const float duz = fmaf(m[2], z, fmaf(m[5], y, m[4] * x));
    model_value_t r;
    r.value = fmaf(z, duz, fmaf(y, duy, x * dux));
    const float etx = f.ct * f.cp, ety = f.ct * f.sp, etz = -f.st;
    r.dtheta = 2.0f * fmaf(duz, etz, fmaf(duy, ety, dux * etx));
    r.dphi = 2.0f * fmaf(duy, f.cp, dux * (-f.sp));
    r.inv = 1.0f / cl_maxf(r.value, 1e-6f);
    return r;
}

/* params: model coefficients (model_coefficients) */
static model_value_t model_eval(int32_t model, const float* params, uint32_t n_params,
                                float x, float y, float z, frame_t f)
{
    if (model == TGO_MODEL_DTI) return dti_model(params, x, y, z, f);
    return sh_model(params, n_params, f);
}

/* ------------------------------------------------------------------ */
/* Algorithms: algorithm.py:83-112 (Transport), 198-228 (Diffusion)   */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t mwc[2];
    uint64_t index;
    uint32_t step;
} rng_t;

static void exps2(float o[3], const float t[3])      /* core.cl:101-109 */
{
    const float n2 = fmaf(t[2], t[2], fmaf(t[1], t[1], t[0] * t[0]));
    if (n2 <= 0.0f) return;
    float c, k;
    tgm_exps2_factors(n2, &c, &k);
    o[0] = fmaf(t[0], k, c * o[0]);
    o[1] = fmaf(t[1], k, c * o[1]);
    o[2] = fmaf(t[2], k, c * o[2]);
}

/* The folded coefficients of the field voxel a tracking loop evaluated last
 * (folded again only when the voxel changes). */
typedef struct {
    const float* src;
    float a[48];
} voxel_fold_t;

static const float* fold_voxel(const tgo_problem* p, voxel_fold_t* cache, const float* c, uint32_t C)
{
    if (cache->src != c) {
        model_coefficients(p->model, c, C, cache->a);
        cache->src = c;
    }
    return cache->a;
}

/* params: model coefficients (model_coefficients) */
static void update_orientation(const tgo_problem* p, const float* params, uint32_t n_params,
                               float o[3], rng_t* rng)
{
    const frame_t f = frame_of(o[0], o[1], o[2]);
    const model_value_t mv = model_eval(p->model, params, n_params, o[0], o[1], o[2], f);
    const float etx = f.ct * f.cp, ety = f.ct * f.sp, etz = -f.st;
    const float epx = -f.sp, epy = f.cp;
    const float inv = mv.inv;
    const float gx = fmaf(mv.dphi, epx, mv.dtheta * etx);
    const float gy = fmaf(mv.dphi, epy, mv.dtheta * ety);
    const float gz = mv.dtheta * etz;
    const float dx = gx * inv, dy = gy * inv, dz = gz * inv;
    const float scale_drift = p->gamma * p->step_size;
    float t[3];
    if (p->algorithm == TGO_ALGO_TRANSPORT) {
        t[0] = scale_drift * dx;
        t[1] = scale_drift * dy;
        t[2] = scale_drift * dz;
    } else {
        float nx = 0.0f, ny = 0.0f, nz = 0.0f;
        if (p->noise_variance > 0.0f) {
            float n1, n2;
            if (p->rng_mode == TGO_RNG_MWC64X) {
                n1 = randn(rng->mwc);                 /* first draw scales e_theta */
                n2 = randn(rng->mwc);
            } else {
                philox_normal2(p->philox_key, rng->index, rng->step, &n1, &n2);
            }
            nx = fmaf(n2, epx, n1 * etx);
            ny = fmaf(n2, epy, n1 * ety);
            nz = n1 * etz;
        }
        const float scale_noise = sqrtf(p->noise_variance * p->gamma * p->step_size);
        t[0] = fmaf(scale_noise, nx, scale_drift * dx);
        t[1] = fmaf(scale_noise, ny, scale_drift * dy);
        t[2] = fmaf(scale_noise, nz, scale_drift * dz);
    }
    exps2(o, t);
    rng->step += 1u;
}

/* ------------------------------------------------------------------ */
/* Domain and field                                                    */
/* ------------------------------------------------------------------ */

/* domain.py:358-382: nearest voxel by floor(v + 0.5), half-open cells. */
static int domain_contains(const tgo_problem* p, float x, float y, float z)
{
    int32_t idx[3];
    for (int i = 0; i < 3; ++i) {
        const float v = floorf(dot4(p->mask_inv_affine + 4 * i, x, y, z, 1.0f) + 0.5f);
        if (!(v >= 0.0f && v < (float)p->mask_dims[i])) return 0;
        idx[i] = (int32_t)v;
    }
    const size_t k = ((size_t)idx[0] * p->mask_dims[1] + (size_t)idx[1]) * p->mask_dims[2] + (size_t)idx[2];
    return p->mask[k] != 0;
}

/* field.py:88-114: nearest voxel by rint (ties to even); 0 when outside. */
static const float* field_voxel(const tgo_problem* p, float x, float y, float z)
{
    int32_t idx[3];
    for (int i = 0; i < 3; ++i) {
        const float v = rintf(dot4(p->field_inv_affine + 4 * i, x, y, z, 1.0f));
        if (!(v >= 0.0f && v < (float)p->field_dims[i])) return NULL;
        idx[i] = (int32_t)v;
    }
    const size_t k = ((size_t)idx[0] * p->field_dims[1] + (size_t)idx[1]) * p->field_dims[2] + (size_t)idx[2];
    return p->field + k * p->field_dims[3];
}

/* ------------------------------------------------------------------ */
/* Boundary BVH: bvh.cl:16-131                                          */
/* ------------------------------------------------------------------ */

static float cl_minf(float x, float y) { return (y < x) ? y : x; }

static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static void cross3(const float* a, const float* b, float* r)
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

/* bvh.cl:16-45: slab test of the segment start + t * direction, t in [0, max_t]. */
static int bounds_hit(const tgo_bvh* b, uint32_t node, const float* start, const float* dir, float max_t)
{
    float t_lo = 0.0f, t_hi = max_t;
    const float* lo = b->bounds_min + 4 * (size_t)node;
    const float* hi = b->bounds_max + 4 * (size_t)node;
    for (int a = 0; a < 3; ++a) {
        if (fabsf(dir[a]) < 1e-12f) {
            if (start[a] < lo[a] || start[a] > hi[a]) return 0;
            continue;
        }
        const float inv = 1.0f / dir[a];
        float t0 = (lo[a] - start[a]) * inv;
        float t1 = (hi[a] - start[a]) * inv;
        if (t0 > t1) {
            const float tmp = t0;
            t0 = t1;
            t1 = tmp;
        }
        t_lo = cl_maxf(t_lo, t0);
        t_hi = cl_minf(t_hi, t1);
        if (t_lo > t_hi) return 0;
    }
    return 1;
}

/* bvh.cl:47-80: Moller-Trumbore with the reference's tolerances. */
static int triangle_hit(const tgo_bvh* b, uint32_t tri, const float* start, const float* dir, float max_t,
                        float* t_out, float* bary)
{
    const uint32_t* ix = b->triangles + 4 * (size_t)tri;
    const float* A = b->vertices + 4 * (size_t)ix[0];
    const float* B = b->vertices + 4 * (size_t)ix[1];
    const float* Cv = b->vertices + 4 * (size_t)ix[2];
    const float e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
    const float e2[3] = {Cv[0] - A[0], Cv[1] - A[1], Cv[2] - A[2]};
    float pv[3], qv[3];
    cross3(dir, e2, pv);
    const float det = dot3(e1, pv);
    if (fabsf(det) < 1e-10f) return 0;
    const float inv_det = 1.0f / det;
    const float off[3] = {start[0] - A[0], start[1] - A[1], start[2] - A[2]};
    const float u = dot3(off, pv) * inv_det;
    if (u < -1e-6f || u > 1.0f + 1e-6f) return 0;
    cross3(off, e1, qv);
    const float v = dot3(dir, qv) * inv_det;
    if (v < -1e-6f || u + v > 1.0f + 1e-6f) return 0;
    const float t = dot3(e2, qv) * inv_det;
    if (t <= 1e-6f || t > max_t) return 0;
    *t_out = t;
    bary[0] = 1.0f - u - v;
    bary[1] = u;
    bary[2] = v;
    return 1;
}

/* bvh.cl:83-131: depth-first with an explicit 64-entry stack, left child
 * popped first, closest hit kept (a later hit at equal t replaces it). */
int tgo_bvh_segment_hit(const tgo_bvh* b, const float start[3], const float end[3], uint32_t* triangle,
                        float barycentric[3], float* t)
{
    const float dir[3] = {end[0] - start[0], end[1] - start[1], end[2] - start[2]};
    int32_t stack[64];
    uint32_t depth = 1;
    stack[0] = 0;
    *t = 1.0f;
    *triangle = 0;
    int found = 0;
    while (depth > 0) {
        const uint32_t node = (uint32_t)stack[--depth];
        if (!bounds_hit(b, node, start, dir, *t)) continue;
        const int32_t* nd = b->nodes + 4 * (size_t)node;
        if (nd[3] > 0) {
            for (int32_t i = 0; i < nd[3]; ++i) {
                const uint32_t tri = b->ordered_triangles[nd[2] + i];
                float tt, bc[3];
                if (triangle_hit(b, tri, start, dir, *t, &tt, bc)) {
                    *t = tt;
                    *triangle = tri;
                    barycentric[0] = bc[0];
                    barycentric[1] = bc[1];
                    barycentric[2] = bc[2];
                    found = 1;
                }
            }
        } else {
            if (depth + 2 > 64) return found;
            stack[depth++] = nd[1];
            stack[depth++] = nd[0];
        }
    }
    return found;
}

uint32_t tgo_bvh_count_hits(const tgo_bvh* b, const float start[3], const float end[3])
{
    const float dir[3] = {end[0] - start[0], end[1] - start[1], end[2] - start[2]};
    int32_t stack[64];
    uint32_t depth = 1, hits = 0;
    stack[0] = 0;
    while (depth > 0) {
        const uint32_t node = (uint32_t)stack[--depth];
        if (!bounds_hit(b, node, start, dir, 1.0f)) continue;
        const int32_t* nd = b->nodes + 4 * (size_t)node;
        if (nd[3] > 0) {
            for (int32_t i = 0; i < nd[3]; ++i) {
                float tt, bc[3];
                hits += (uint32_t)triangle_hit(b, b->ordered_triangles[nd[2] + i], start, dir, 1.0f, &tt, bc);
            }
        } else {
            if (depth + 2 > 64) return hits;
            stack[depth++] = nd[1];
            stack[depth++] = nd[0];
        }
    }
    return hits;
}

/* Three fixed ray directions of the closed-surface inside test (unit
 * length to float precision, chosen off every coordinate plane and
 * diagonal so that rays rarely meet mesh edges). */
static const float kMeshRays[3][3] = {
    {0.53896236f, 0.77412713f, 0.33221170f},
    {-0.68169260f, 0.22392839f, 0.69653570f},
    {0.17420970f, -0.54785200f, 0.81824590f},
};

int tgo_mesh_contains(const tgo_bvh* b, float x, float y, float z)
{
    const float p[3] = {x, y, z};
    const float* lo = b->bounds_min;
    const float* hi = b->bounds_max;
    for (int a = 0; a < 3; ++a)
        if (!(p[a] >= lo[a] && p[a] <= hi[a])) return 0;
    const float reach = (((hi[0] - lo[0]) + (hi[1] - lo[1])) + (hi[2] - lo[2])) + 1.0f;
    int odd = 0;
    for (int r = 0; r < 3; ++r) {
        const float e[3] = {p[0] + reach * kMeshRays[r][0], p[1] + reach * kMeshRays[r][1],
                            p[2] + reach * kMeshRays[r][2]};
        odd += (int)(tgo_bvh_count_hits(b, p, e) & 1u);
    }
    return odd >= 2;
}

void tgo_segment_hits(const tgo_bvh* b, const float* starts, const float* ends, uint32_t n, uint8_t* found,
                      uint32_t* triangle, float* hit, int n_threads)
{
    long i;
#pragma omp parallel for schedule(dynamic, 64) num_threads(n_threads > 0 ? n_threads : 1)
    for (i = 0; i < (long)n; ++i) {
        float t = 1.0f, bc[3] = {0.0f, 0.0f, 0.0f};
        uint32_t tri = 0;
        found[i] = (uint8_t)tgo_bvh_segment_hit(b, starts + 4 * i, ends + 4 * i, &tri, bc, &t);
        triangle[i] = tri;
        hit[4 * i] = bc[0];
        hit[4 * i + 1] = bc[1];
        hit[4 * i + 2] = bc[2];
        hit[4 * i + 3] = t;
    }
}

/* domain.py:95-120 domain_sample_boundary, once per seed (:520-545). */
static void sample_boundary_full(const float* vertices, const uint32_t* triangles, const float* cumulative,
                                 uint32_t n_triangles, uint32_t st[2], float* out, uint32_t* tri_out,
                                 float* bary_out);

static void sample_boundary(const float* vertices, const uint32_t* triangles, const float* cumulative,
                            uint32_t n_triangles, uint32_t st[2], float* out)
{
    uint32_t tri;
    float bary[3];
    sample_boundary_full(vertices, triangles, cumulative, n_triangles, st, out, &tri, bary);
}

static void sample_boundary_full(const float* vertices, const uint32_t* triangles, const float* cumulative,
                                 uint32_t n_triangles, uint32_t st[2], float* out, uint32_t* tri_out,
                                 float* bary_out)
{
    {
        const float target = randu(st);
        uint32_t lower = 0, upper = n_triangles;
        while (lower < upper) {
            const uint32_t middle = lower + (upper - lower) / 2;
            if (cumulative[middle] <= target) lower = middle + 1;
            else upper = middle;
        }
        const uint32_t tri = lower < n_triangles - 1 ? lower : n_triangles - 1;
        const float* a = vertices + 4 * (size_t)triangles[4 * (size_t)tri];
        const float* b = vertices + 4 * (size_t)triangles[4 * (size_t)tri + 1];
        const float* c = vertices + 4 * (size_t)triangles[4 * (size_t)tri + 2];
        const float root_u = sqrtf(randu(st));
        const float v = randu(st);
        *tri_out = tri;
        bary_out[0] = 1.0f - root_u;
        bary_out[1] = root_u * (1.0f - v);
        bary_out[2] = root_u * v;
        float p[3], e1[3], e2[3], nrm[3];
        for (int k = 0; k < 3; ++k) {
            p[k] = ((1.0f - root_u) * a[k] + (root_u * (1.0f - v)) * b[k]) + (root_u * v) * c[k];
            e1[k] = b[k] - a[k];
            e2[k] = c[k] - a[k];
        }
        cross3(e1, e2, nrm);
        const float len = sqrtf(dot3(nrm, nrm));
        for (int k = 0; k < 3; ++k) {
            const float o = -(nrm[k] / len);
            out[k] = p[k] + 1e-4f * o;
            out[4 + k] = o;
        }
        out[3] = 1.0f;
        out[7] = 0.0f;
    }
}

void tgo_boundary_seeds(const float* vertices, const uint32_t* triangles, const float* cumulative,
                        uint32_t n_triangles, uint32_t rng_seed, uint32_t n, float* seeds)
{
    for (uint32_t gid = 0; gid < n; ++gid) {
        uint32_t st[2];
        tgo_rng_init(rng_seed, gid, st);
        sample_boundary(vertices, triangles, cumulative, n_triangles, st, seeds + 8 * (size_t)gid);
    }
}

/* ------------------------------------------------------------------ */
/* Tracking loop: tracking.py:105-148                                  */
/* ------------------------------------------------------------------ */

static uint32_t track_one(const tgo_problem* p, const float* seed, uint32_t gid, float* out,
                          uint64_t* steps)
{
    const uint32_t n_steps = p->n_steps;
    const uint32_t C = p->field_dims[3];
    float pos[3] = {seed[0], seed[1], seed[2]};
    float o[3] = {seed[4], seed[5], seed[6]};
    rng_t rng;
    tgo_rng_init(p->rng_seed, gid, rng.mwc);
    rng.index = p->seed_offset + gid;
    rng.step = 0u;
    out[0] = seed[0]; out[1] = seed[1]; out[2] = seed[2]; out[3] = seed[3];
    uint32_t n = 1;
    float time = 0.0f;
    float last[3] = {pos[0], pos[1], pos[2]};
    int first = 1;
    voxel_fold_t fold = {NULL, {0.0f}};
    while (n < n_steps) {
        if (p->mesh) {
            /* closed surface: the seed must be inside, each later point is
             * reached by a segment that does not hit the surface */
            if (first) {
                if (!tgo_mesh_contains(p->mesh, pos[0], pos[1], pos[2])) break;
            } else {
                uint32_t tri;
                float bc[3], t;
                if (tgo_bvh_segment_hit(p->mesh, last, pos, &tri, bc, &t)) break;
            }
            first = 0;
            last[0] = pos[0];
            last[1] = pos[1];
            last[2] = pos[2];
        } else if (!domain_contains(p, pos[0], pos[1], pos[2])) {
            break;
        }
        const float* c = field_voxel(p, pos[0], pos[1], pos[2]);
        if (!c) break;
        update_orientation(p, fold_voxel(p, &fold, c, C), C, o, &rng);
        *steps += 1;
        pos[0] = fmaf(p->step_size, o[0], pos[0]);
        pos[1] = fmaf(p->step_size, o[1], pos[1]);
        pos[2] = fmaf(p->step_size, o[2], pos[2]);
        time = time + p->step_size;
        if (time >= p->save_at) {
            time = time - p->save_at;
            float* q = out + 4 * (size_t)n;
            q[0] = fmaf(-time, o[0], pos[0]);
            q[1] = fmaf(-time, o[1], pos[1]);
            q[2] = fmaf(-time, o[2], pos[2]);
            q[3] = 1.0f;
            n++;
        }
    }
    return n;
}

static void sh_basis(int lmax, frame_t f, float* Y);

static void tod_flush(float* coefficients, const float* acc, const int32_t* idx, const uint32_t* dims)
{
    const size_t base = (((size_t)idx[0] * dims[1] + (size_t)idx[1]) * dims[2] + (size_t)idx[2]) * 45;
    for (int k = 0; k < 45; ++k) coefficients[base + k] += acc[k];
}

void tgo_tod(const tgo_problem* p, const float* vertices, const uint32_t* triangles, const float* cumulative,
             uint32_t n_triangles, uint32_t n_seeds, uint32_t n_steps, const uint32_t out_dims[3],
             const float out_inverse_affine[16], float* coefficients)
{
    const uint32_t C = p->field_dims[3];
    for (uint32_t gid = 0; gid < n_seeds; ++gid) {
        rng_t rng;
        float seed[8];
        tgo_rng_init(p->rng_seed, gid, rng.mwc);
        sample_boundary(vertices, triangles, cumulative, n_triangles, rng.mwc, seed);
        rng.index = p->seed_offset + gid;
        rng.step = 0u;
        float pos[3] = {seed[0], seed[1], seed[2]};
        float o[3] = {seed[4], seed[5], seed[6]};
        float last[3] = {pos[0], pos[1], pos[2]};
        int first = 1;
    voxel_fold_t fold = {NULL, {0.0f}};
        float acc[45];
        int32_t prev[3] = {-1, -1, -1};
        for (uint32_t step = 0; step < n_steps; ++step) {
            if (p->mesh) {
                if (first) {
                    if (!tgo_mesh_contains(p->mesh, pos[0], pos[1], pos[2])) break;
                } else {
                    uint32_t tri;
                    float bc[3], t;
                    if (tgo_bvh_segment_hit(p->mesh, last, pos, &tri, bc, &t)) break;
                }
                first = 0;
                last[0] = pos[0];
                last[1] = pos[1];
                last[2] = pos[2];
            } else if (!domain_contains(p, pos[0], pos[1], pos[2])) {
                break;
            }
            const float* c = field_voxel(p, pos[0], pos[1], pos[2]);
            if (!c) break;
            int32_t idx[3];
            int inside = 1;
            for (int i = 0; i < 3; ++i) {
                const float v = floorf(dot4(out_inverse_affine + 4 * i, pos[0], pos[1], pos[2], 1.0f) + 0.5f);
                if (!(v >= 0.0f && v < (float)out_dims[i])) inside = 0;
                idx[i] = inside ? (int32_t)v : 0;
            }
            if (inside) {
                float Y[45];
                sh_basis(8, frame_of(o[0], o[1], o[2]), Y);
                if (idx[0] == prev[0] && idx[1] == prev[1] && idx[2] == prev[2]) {
                    for (int k = 0; k < 45; ++k) acc[k] += Y[k];
                } else {
                    if (prev[0] >= 0) tod_flush(coefficients, acc, prev, out_dims);
                    for (int k = 0; k < 45; ++k) acc[k] = Y[k];
                    prev[0] = idx[0];
                    prev[1] = idx[1];
                    prev[2] = idx[2];
                }
            } else if (prev[0] >= 0) {
                tod_flush(coefficients, acc, prev, out_dims);
                prev[0] = prev[1] = prev[2] = -1;
            }
            update_orientation(p, fold_voxel(p, &fold, c, C), C, o, &rng);
            const float len = sqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
            if (!(isfinite(o[0]) && isfinite(o[1]) && isfinite(o[2])) || len < 0.5f) break;
            pos[0] = fmaf(p->step_size, o[0], pos[0]);
            pos[1] = fmaf(p->step_size, o[1], pos[1]);
            pos[2] = fmaf(p->step_size, o[2], pos[2]);
        }
        if (prev[0] >= 0) tod_flush(coefficients, acc, prev, out_dims);
    }
}

void tgo_connectome(const tgo_problem* p, const tgo_bvh* boundary, const float* vertices, const uint32_t* triangles,
                    const float* cumulative, uint32_t n_triangles, uint32_t n_seeds, uint32_t n_steps,
                    float minimum_length, int32_t* rows, int32_t* columns, float* weights)
{
    const uint32_t C = p->field_dims[3];
    long g;
#pragma omp parallel for schedule(dynamic, 16)
    for (g = 0; g < (long)n_seeds; ++g) {
        const uint32_t gid = (uint32_t)g;
        const size_t base = 9 * (size_t)gid;
        for (int k = 0; k < 9; ++k) rows[base + k] = -1;
        rng_t rng;
        float seed[8], start_w[3];
        uint32_t start_tri;
        tgo_rng_init(p->rng_seed, gid, rng.mwc);
        sample_boundary_full(vertices, triangles, cumulative, n_triangles, rng.mwc, seed, &start_tri, start_w);
        rng.index = p->seed_offset + gid;
        rng.step = 0u;
        float pos[3] = {seed[0], seed[1], seed[2]};
        float o[3] = {seed[4], seed[5], seed[6]};
        float prev[3] = {pos[0], pos[1], pos[2]};
        float last[3] = {pos[0], pos[1], pos[2]};
        int first = 1;
    voxel_fold_t fold = {NULL, {0.0f}};
        uint32_t tracked = 0;
        for (uint32_t step = 0; step < n_steps; ++step) {
            if (p->mesh) {
                if (first) {
                    if (!tgo_mesh_contains(p->mesh, pos[0], pos[1], pos[2])) break;
                } else {
                    uint32_t tri;
                    float bc[3], t;
                    if (tgo_bvh_segment_hit(p->mesh, last, pos, &tri, bc, &t)) break;
                }
                first = 0;
                last[0] = pos[0];
                last[1] = pos[1];
                last[2] = pos[2];
            } else if (!domain_contains(p, pos[0], pos[1], pos[2])) {
                break;
            }
            const float* c = field_voxel(p, pos[0], pos[1], pos[2]);
            if (!c) break;
            update_orientation(p, fold_voxel(p, &fold, c, C), C, o, &rng);
            const float len = sqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
            if (!(isfinite(o[0]) && isfinite(o[1]) && isfinite(o[2])) || len < 0.5f) break;
            prev[0] = pos[0];
            prev[1] = pos[1];
            prev[2] = pos[2];
            pos[0] = fmaf(p->step_size, o[0], pos[0]);
            pos[1] = fmaf(p->step_size, o[1], pos[1]);
            pos[2] = fmaf(p->step_size, o[2], pos[2]);
            tracked++;
        }
        if ((float)tracked * p->step_size < minimum_length) continue;
        uint32_t hit_tri;
        float end_w[3], t;
        if (!tgo_bvh_segment_hit(boundary, prev, pos, &hit_tri, end_w, &t)) continue;
        const uint32_t* sv = triangles + 4 * (size_t)start_tri;
        const uint32_t* ev = triangles + 4 * (size_t)hit_tri;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                rows[base + 3 * i + j] = (int32_t)sv[i];
                columns[base + 3 * i + j] = (int32_t)ev[j];
                weights[base + 3 * i + j] = start_w[i] * end_w[j];
            }
    }
}

uint64_t tgo_tractogram(const tgo_problem* p, const float* seeds, uint32_t n_seeds,
                        float* streamlines, uint32_t* lengths, int n_threads)
{
    if (p->n_steps == 0) {
        for (uint32_t i = 0; i < n_seeds; ++i) lengths[i] = 0;
        return 0;
    }
    uint64_t total = 0;
    long i;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total) num_threads(n_threads > 0 ? n_threads : 1)
    for (i = 0; i < (long)n_seeds; ++i) {
        float* out = streamlines + (size_t)i * p->n_steps * 4;
        uint64_t steps = 0;
        lengths[i] = track_one(p, seeds + 8 * (size_t)i, (uint32_t)i, out, &steps);
        total += steps;
    }
    return total;
}

uint64_t tgo_tractogram_ids(const tgo_problem* p, const float* seeds, const uint32_t* ids, uint32_t n_seeds,
                            float* streamlines, uint32_t* lengths, int n_threads)
{
    if (p->n_steps == 0) {
        for (uint32_t i = 0; i < n_seeds; ++i) lengths[i] = 0;
        return 0;
    }
    uint64_t total = 0;
    long i;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) num_threads(n_threads > 0 ? n_threads : 1)
    for (i = 0; i < (long)n_seeds; ++i) {
        float* out = streamlines + (size_t)i * p->n_steps * 4;
        uint64_t steps = 0;
        lengths[i] = track_one(p, seeds + 8 * (size_t)i, ids[i], out, &steps);
        total += steps;
    }
    return total;
}

void tgo_contains(const tgo_problem* p, const float* points, uint32_t n, uint8_t* out)
{
    for (uint32_t i = 0; i < n; ++i)
        out[i] = (uint8_t)(p->mesh ? tgo_mesh_contains(p->mesh, points[4 * i], points[4 * i + 1], points[4 * i + 2])
                                   : domain_contains(p, points[4 * i], points[4 * i + 1], points[4 * i + 2]));
}

void tgo_field_evaluate(const tgo_problem* p, const float* points, uint32_t n, float* out)
{
    const uint32_t C = p->field_dims[3];
    for (uint32_t i = 0; i < n; ++i) {
        const float* c = field_voxel(p, points[4 * i], points[4 * i + 1], points[4 * i + 2]);
        for (uint32_t j = 0; j < C; ++j) out[(size_t)i * C + j] = c ? c[j] : 0.0f;
    }
}

void tgo_local_evaluate(int32_t model, uint32_t n_params, const float* params,
                        const float* orientations, uint32_t n, float* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        const float* o = orientations + 4 * (size_t)i;
        const frame_t f = frame_of(o[0], o[1], o[2]);
        float coeffs[48];
        model_coefficients(model, params + (size_t)i * n_params, n_params, coeffs);
        const model_value_t r = model_eval(model, coeffs, n_params, o[0], o[1], o[2], f);
        out[3 * i] = r.value;
        out[3 * i + 1] = r.dtheta;
        out[3 * i + 2] = r.dphi;
    }
}

void tgo_update_orientation(const tgo_problem* p, uint32_t n_params, const float* params,
                            const float* orientations, uint32_t n, float* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        rng_t rng;
        tgo_rng_init(p->rng_seed, i, rng.mwc);
        rng.index = p->seed_offset + i;
        rng.step = 0u;
        float o[3] = {orientations[4 * i], orientations[4 * i + 1], orientations[4 * i + 2]};
        float coeffs[48];
        model_coefficients(p->model, params + (size_t)i * n_params, n_params, coeffs);
        update_orientation(p, coeffs, n_params, o, &rng);
        out[4 * i] = o[0]; out[4 * i + 1] = o[1]; out[4 * i + 2] = o[2]; out[4 * i + 3] = 0.0f;
    }
}

/* ------------------------------------------------------------------ */
/* FOD seeding: seeds.cl:12-118                                        */
/* ------------------------------------------------------------------ */

/* seeds.cl:12-25: n-th of n_points Fibonacci-lattice directions. */
static void fibonacci(uint32_t n, uint32_t n_points, float d[3])
{
    const float phi = (sqrtf(5.0f) + 1.0f) * 0.5f;
    const float golden_angle = TGM_TWO_PI / phi;
    const float theta = (float)n * golden_angle;
    const float z = 1.0f - (2.0f * (float)n / (float)(n_points - 1));
    const float radius = sqrtf(fmaf(-z, z, 1.0f));
    float s, c;
    tgm_sincosf(theta, &s, &c);
    d[0] = radius * c;
    d[1] = radius * s;
    d[2] = z;
}

/* Real SH basis Y_i (i < (lmax+1)(lmax+2)/2) at one direction, the
 * value-only basis: Y = R * st^m * trig(m phi). */
static void sh_basis(int lmax, frame_t f, float* Y)
{
    const float ct = f.ct, st = f.st, cp = f.cp, sp = f.sp;
    const float u = ct * ct;
    const float tc = cp + cp;
    float cm[TG_SH_LMAX + 1], sm[TG_SH_LMAX + 1], stp[TG_SH_LMAX + 1];
    cm[0] = 1.0f; sm[0] = 0.0f; cm[1] = cp; sm[1] = sp;
    for (int m = 2; m <= lmax; ++m) {
        cm[m] = fmaf(tc, cm[m - 1], -cm[m - 2]);
        sm[m] = fmaf(tc, sm[m - 1], -sm[m - 2]);
    }
    stp[0] = 1.0f;
    for (int k = 1; k <= lmax; ++k) stp[k] = stp[k - 1] * st;
    for (int k = 0; k < TG_SH_NPAIRS; ++k) {
        const int* e = TG_SH_PAIRS[k];
        const int l = e[0], m = e[1];
        if (l > lmax) continue;
        float R = horner_u(TG_SH_COEF + e[3], e[4], u);
        if (e[2]) R = R * ct;
        const int ip = l * (l + 1) / 2 + m;
        if (m == 0) {
            Y[ip] = R;
        } else {
            const float P = R * stp[m];
            Y[ip] = P * cm[m];
            Y[l * (l + 1) / 2 - m] = P * sm[m];
        }
    }
}

typedef struct {
    float dir[N_DIRECTIONS][3];
    float Y[N_DIRECTIONS][48];
} fib_table_t;

static float fod_value(int32_t model, const float* c, uint32_t C, const fib_table_t* t, int i)
{
    if (model == TGO_MODEL_DTI) {
        const float* d = t->dir[i];
        const frame_t f = frame_of(d[0], d[1], d[2]);
        return dti_model(c, d[0], d[1], d[2], f).value;
    }
    float raw = 0.0f;
    for (uint32_t j = 0; j < C; ++j) raw = fmaf(c[j], t->Y[i][j], raw);
    return softmax(raw, SOFTMAX_SCALE);
}

void tgo_seeds_from_fod(int32_t model, uint32_t C, const float* fod,
                        const float* voxels, uint32_t nnz, const float affine[16],
                        const uint32_t* states, uint32_t n_seeds, float* seeds,
                        int n_threads)
{
    fib_table_t* t = (fib_table_t*)malloc(sizeof(fib_table_t));
    const int lmax = lmax_for(C);
    for (int i = 0; i < N_DIRECTIONS; ++i) {
        fibonacci((uint32_t)i, N_DIRECTIONS, t->dir[i]);
        if (model == TGO_MODEL_SH) {
            const frame_t f = frame_of(t->dir[i][0], t->dir[i][1], t->dir[i][2]);
            sh_basis(lmax, f, t->Y[i]);
        }
    }
    long g;
#pragma omp parallel for schedule(static) num_threads(n_threads > 0 ? n_threads : 1)
    for (g = 0; g < (long)n_seeds; ++g) {
        uint32_t s[2] = {states[2 * g], states[2 * g + 1]};
        uint32_t vi = randi(s, nnz);                  /* seeds.cl:89 */
        if (vi >= nnz) vi = nnz - 1;
        const float* v = voxels + 4 * (size_t)vi;
        float vx = v[0], vy = v[1], vz = v[2], vw = v[3];
        vx = vx + (randu(s) - 0.5f);                 /* seeds.cl:94, x then y then z */
        vy = vy + (randu(s) - 0.5f);
        vz = vz + (randu(s) - 0.5f);
        const float* c = fod + (size_t)vi * C;
        float sum = 0.0f;                            /* seeds.cl:29-35 */
        for (int i = 0; i < N_DIRECTIONS; ++i) sum = sum + cl_maxf(fod_value(model, c, C, t, i), 0.0f);
        const float threshold = randu(s) * sum;      /* seeds.cl:38 */
        float cs = 0.0f;
        int selected = N_DIRECTIONS;
        for (int i = 0; i < N_DIRECTIONS; ++i) {
            cs = cs + cl_maxf(fod_value(model, c, C, t, i), 0.0f);
            if (selected == N_DIRECTIONS && cs > threshold) selected = i;
        }
        float* out = seeds + 8 * (size_t)g;
        out[0] = dot4(affine + 0, vx, vy, vz, vw);   /* seeds.cl:105, apply_affine */
        out[1] = dot4(affine + 4, vx, vy, vz, vw);
        out[2] = dot4(affine + 8, vx, vy, vz, vw);
        out[3] = dot4(affine + 12, vx, vy, vz, vw);
        if (selected < N_DIRECTIONS) {
            out[4] = t->dir[selected][0]; out[5] = t->dir[selected][1]; out[6] = t->dir[selected][2];
        } else {
            out[4] = 0.0f; out[5] = 0.0f; out[6] = 1.0f;
        }
        out[7] = 0.0f;
    }
    free(t);
}

/* ------------------------------------------------------------------ */
/* Streams for tests (core.cl:218-238)                                 */
/* ------------------------------------------------------------------ */

void tgo_randu_stream(uint32_t s0, uint32_t s1, uint32_t n, float* out)
{
    uint32_t s[2] = {s0, s1};
    for (uint32_t i = 0; i < n; ++i) out[i] = randu(s);
}

void tgo_randn_stream(uint32_t s0, uint32_t s1, uint32_t n, float* out)
{
    uint32_t s[2] = {s0, s1};
    for (uint32_t i = 0; i < n; ++i) out[i] = randn(s);
}

void tgo_randi_stream(uint32_t s0, uint32_t s1, uint32_t n, uint32_t max, uint32_t* out)
{
    uint32_t s[2] = {s0, s1};
    for (uint32_t i = 0; i < n; ++i) out[i] = randi(s, max);
}

void tgo_math(int which, const float* x, uint32_t n, float* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        switch (which) {
        case 0: out[i] = tgm_sinf(x[i]); break;
        case 1: out[i] = tgm_cosf(x[i]); break;
        case 2: out[i] = tgm_expf(x[i]); break;
        case 3: out[i] = tgm_logf(x[i]); break;
        case 4: { float c, k; tgm_exps2_factors(x[i], &c, &k); out[i] = c; } break;
        case 5: { float c, k; tgm_exps2_factors(x[i], &c, &k); out[i] = k; } break;
        case 6: { float v, d, q; tgm_softplus(x[i], SOFTMAX_SCALE, SOFTMAX_INV_SCALE, &v, &d, &q); out[i] = v; } break;
        case 7: { float v, d, q; tgm_softplus(x[i], SOFTMAX_SCALE, SOFTMAX_INV_SCALE, &v, &d, &q); out[i] = d; } break;
        case 8: { float v, d, q; tgm_softplus(x[i], SOFTMAX_SCALE, SOFTMAX_INV_SCALE, &v, &d, &q); out[i] = q; } break;
        case 9: out[i] = tgm_cos2pi_u24((uint32_t)x[i]); break;
        case 10: out[i] = tgm_log_pos(x[i]); break;
        case 11: out[i] = tgm_exp_upto30(x[i]); break;
        case 12: out[i] = tgm_rsqrt_pos(x[i]); break;
        default: out[i] = x[i]; break;
        }
    }
}
