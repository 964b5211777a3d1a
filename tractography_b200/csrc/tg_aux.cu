/*
 * tg_aux.cu -- FOD seeding and the per-element kernels behind the
 * reference's standalone entry points:
 *
 *   seeds_from_fod_kernel    seeds.cl:99-118 (tg.seeds.from_fod, OpenCL path)
 *   contains_kernel          domain.py:456-469 (tg.domain.contains)
 *   field_evaluate_kernel    field.py:158-175 (tg.field.evaluate)
 *   local_evaluate_kernel    local.py:316-335 (tg.local.evaluate)
 *   update_orientation_kernel algorithm.py:738-759 (tg.algorithm.update_orientation)
 *   rng_stream_kernel        core.cl:218-238 (randus / randis test streams)
 */
#include <cuda_runtime.h>

#include "tg_internal.h"
#include "tg_step.cuh"

namespace tg {

constexpr int kDirections = 1000;   // seeds.cl:10

// ------------------------------------------------------------ seeding

// seeds.cl:12-25: n-th of n_points Fibonacci-lattice directions.
__device__ __forceinline__ float3 fibonacci(uint32_t n, uint32_t n_points)
{
    const float phi = (sqrtf(5.0f) + 1.0f) * 0.5f;
    const float golden_angle = TGM_TWO_PI / phi;
    const float theta = (float)n * golden_angle;
    const float z = 1.0f - (2.0f * (float)n / (float)(n_points - 1));
    const float radius = sqrtf(fmaf(-z, z, 1.0f));
    float s, c;
    tgm_sincosf(theta, &s, &c);
    return make_float3(radius * c, radius * s, z);
}

// Table of the 1000 directions (float4, w = 0) and, for SH, the basis
// values Y_i at each direction, rows of `cpad` floats.
template <int LMAX>
__global__ void fod_table_kernel(float4* dirs, float* Y, int cpad, int is_sh)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kDirections) return;
    const float3 d = fibonacci((uint32_t)i, kDirections);
    dirs[i] = make_float4(d.x, d.y, d.z, 0.0f);
    if (is_sh) {
        float row[n_coef_full(LMAX)];
        const Frame f = frame_of(d.x, d.y, d.z);
        sh_basis<LMAX>(f.ct, f.st, f.cp, f.sp, row);
        for (int j = 0; j < cpad; ++j) Y[(size_t)i * cpad + j] = j < n_coef_full(LMAX) ? row[j] : 0.0f;
    }
}

template <int MODEL, int CPAD>
__device__ __forceinline__ float fod_value(const float (&c)[CPAD], uint32_t C, const float4* dirs,
                                           const float* Y, int i)
{
    if constexpr (MODEL == kModelDTI) {
        const float4 d = __ldg(dirs + i);
        const Frame f = frame_of(d.x, d.y, d.z);
        return dti_model(c, d.x, d.y, d.z, f).value;
    } else {
        const float4* row = reinterpret_cast<const float4*>(Y + (size_t)i * CPAD);
        float raw = 0.0f;
#pragma unroll
        for (int k = 0; k < CPAD / 4; ++k) {
            const float4 y = __ldg(row + k);
            if (4 * k + 0 < (int)C) raw = fmaf(c[4 * k + 0], y.x, raw);
            if (4 * k + 1 < (int)C) raw = fmaf(c[4 * k + 1], y.y, raw);
            if (4 * k + 2 < (int)C) raw = fmaf(c[4 * k + 2], y.z, raw);
            if (4 * k + 3 < (int)C) raw = fmaf(c[4 * k + 3], y.w, raw);
        }
        return softmax(raw, kSoftmaxScale);
    }
}

template <int MODEL, int CPAD>
__global__ void __launch_bounds__(128) seeds_from_fod_kernel(const float* __restrict__ fod, uint32_t C,
                                                             const float4* __restrict__ voxels, uint32_t nnz,
                                                             const float* __restrict__ affine,
                                                             const uint2* __restrict__ states, uint32_t n_seeds,
                                                             const float4* __restrict__ dirs,
                                                             const float* __restrict__ Y,
                                                             float4* __restrict__ seeds)
{
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n_seeds) return;
    const uint2 st = states[gid];
    Mwc s;
    s.x = st.x;
    s.c = st.y;
    uint32_t vi = randi(s, nnz);                          // seeds.cl:89
    if (vi >= nnz) vi = nnz - 1;
    const float4 v = voxels[vi];
    float vx = v.x, vy = v.y, vz = v.z;
    vx = vx + (randu(s) - 0.5f);                          // seeds.cl:94 (x, y, z order)
    vy = vy + (randu(s) - 0.5f);
    vz = vz + (randu(s) - 0.5f);
    float c[CPAD];
#pragma unroll
    for (int k = 0; k < CPAD; ++k) c[k] = (uint32_t)k < C ? fod[(size_t)vi * C + k] : 0.0f;

    float sum = 0.0f;                                     // seeds.cl:29-35
    for (int i = 0; i < kDirections; ++i) sum = sum + cl_max(fod_value<MODEL, CPAD>(c, C, dirs, Y, i), 0.0f);
    const float threshold = randu(s) * sum;               // seeds.cl:38
    float cs = 0.0f;
    int selected = kDirections;
    for (int i = 0; i < kDirections; ++i) {
        cs = cs + cl_max(fod_value<MODEL, CPAD>(c, C, dirs, Y, i), 0.0f);
        if (selected == kDirections && cs > threshold) selected = i;
    }
    float4 loc;
    const float4 r0 = make_float4(affine[0], affine[1], affine[2], affine[3]);
    const float4 r1 = make_float4(affine[4], affine[5], affine[6], affine[7]);
    const float4 r2 = make_float4(affine[8], affine[9], affine[10], affine[11]);
    const float4 r3 = make_float4(affine[12], affine[13], affine[14], affine[15]);
    loc.x = dot4(r0, vx, vy, vz, v.w);
    loc.y = dot4(r1, vx, vy, vz, v.w);
    loc.z = dot4(r2, vx, vy, vz, v.w);
    loc.w = dot4(r3, vx, vy, vz, v.w);
    seeds[2 * (size_t)gid] = loc;
    seeds[2 * (size_t)gid + 1] = selected < kDirections ? dirs[selected] : make_float4(0.0f, 0.0f, 1.0f, 0.0f);
}

cudaError_t launch_seeds_from_fod(int model, uint32_t C, const float* fod, const float4* voxels, uint32_t nnz,
                                  const float* affine, const uint2* states, uint32_t n_seeds, float4* seeds,
                                  cudaStream_t stream)
{
    if (n_seeds == 0) return cudaSuccess;
    const int lmax = lmax_for(C);
    const int cpad = model == kModelDTI ? 8 : (n_coef_full(lmax) + 3) / 4 * 4;
    float4* dirs = nullptr;
    float* Y = nullptr;
    cudaError_t e = cudaMallocAsync(&dirs, kDirections * sizeof(float4), stream);
    if (e != cudaSuccess) return e;
    e = cudaMallocAsync(&Y, (size_t)kDirections * cpad * sizeof(float), stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(dirs, stream);
        return e;
    }
    const int is_sh = model == kModelSH;
    const int tb = 128, tg_ = (kDirections + tb - 1) / tb;
    switch (is_sh ? lmax : 0) {
    case 0: fod_table_kernel<0><<<tg_, tb, 0, stream>>>(dirs, Y, cpad, is_sh); break;
    case 2: fod_table_kernel<2><<<tg_, tb, 0, stream>>>(dirs, Y, cpad, is_sh); break;
    case 4: fod_table_kernel<4><<<tg_, tb, 0, stream>>>(dirs, Y, cpad, is_sh); break;
    case 6: fod_table_kernel<6><<<tg_, tb, 0, stream>>>(dirs, Y, cpad, is_sh); break;
    default: fod_table_kernel<8><<<tg_, tb, 0, stream>>>(dirs, Y, cpad, is_sh); break;
    }
    const int block = 128;
    const int grid = (int)((n_seeds + block - 1) / block);
    if (model == kModelDTI) {
        seeds_from_fod_kernel<kModelDTI, 8><<<grid, block, 0, stream>>>(fod, C, voxels, nnz, affine, states,
                                                                        n_seeds, dirs, Y, seeds);
    } else {
        switch (cpad) {
        case 4: seeds_from_fod_kernel<kModelSH, 4><<<grid, block, 0, stream>>>(fod, C, voxels, nnz, affine, states, n_seeds, dirs, Y, seeds); break;
        case 8: seeds_from_fod_kernel<kModelSH, 8><<<grid, block, 0, stream>>>(fod, C, voxels, nnz, affine, states, n_seeds, dirs, Y, seeds); break;
        case 16: seeds_from_fod_kernel<kModelSH, 16><<<grid, block, 0, stream>>>(fod, C, voxels, nnz, affine, states, n_seeds, dirs, Y, seeds); break;
        case 28: seeds_from_fod_kernel<kModelSH, 28><<<grid, block, 0, stream>>>(fod, C, voxels, nnz, affine, states, n_seeds, dirs, Y, seeds); break;
        default: seeds_from_fod_kernel<kModelSH, 48><<<grid, block, 0, stream>>>(fod, C, voxels, nnz, affine, states, n_seeds, dirs, Y, seeds); break;
        }
    }
    e = cudaGetLastError();
    cudaFreeAsync(Y, stream);
    cudaFreeAsync(dirs, stream);
    return e;
}

// ------------------------------------------------------------ unit hooks

__global__ void contains_kernel(Grid g, const uint8_t* __restrict__ mask, const float4* __restrict__ pts,
                                uint32_t n, uint8_t* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pts[i];
    const int64_t k = voxel_floor_half(g, p.x, p.y, p.z);
    out[i] = (k >= 0 && mask[k] != 0) ? 1 : 0;
}

__global__ void field_evaluate_kernel(Grid g, const float* __restrict__ field, uint32_t C, uint32_t cpad,
                                      const float4* __restrict__ pts, uint32_t n, float* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pts[i];
    const int64_t k = voxel_rint(g, p.x, p.y, p.z);
    for (uint32_t j = 0; j < C; ++j) out[(size_t)i * C + j] = k >= 0 ? field[k * cpad + j] : 0.0f;
}

// The coefficients model_eval takes: SH coefficients folded (tgsh_fold),
// tensor coefficients as they are.
template <int MODEL, int LMAX, int CP>
__device__ __forceinline__ void model_coefficients(const float (&raw)[CP], float (&c)[CP])
{
    if constexpr (MODEL == kModelDTI) {
#pragma unroll
        for (int k = 0; k < CP; ++k) c[k] = raw[k];
    } else {
        tgsh_fold(LMAX, raw, c);
    }
}

// Folds a field's SH coefficients per voxel (cpad floats each, zero beyond
// the band) for the tracking kernels.
__global__ void fold_field_kernel(const float* __restrict__ raw, float* __restrict__ folded, uint64_t n_voxels,
                                  uint32_t cpad, int lmax)
{
    const int n = (lmax + 1) * (lmax + 2) / 2;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n_voxels;
         v += (uint64_t)gridDim.x * blockDim.x) {
        float c[48], a[48];
        for (uint32_t k = 0; k < cpad; ++k) c[k] = raw[v * cpad + k];
        tgsh_fold(lmax, c, a);
        for (uint32_t k = 0; k < cpad; ++k) folded[v * cpad + k] = (int)k < n ? a[k] : 0.0f;
    }
}

cudaError_t launch_fold_field(const float* raw, float* folded, uint64_t n_voxels, uint32_t cpad, int lmax,
                              cudaStream_t stream)
{
    if (n_voxels == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int block = 128;
    uint64_t grid = (n_voxels + block - 1) / block;
    if (grid > (uint64_t)sms * 32) grid = (uint64_t)sms * 32;
    fold_field_kernel<<<(int)grid, block, 0, stream>>>(raw, folded, n_voxels, cpad, lmax);
    return cudaGetLastError();
}

template <int MODEL, int LMAX>
__global__ void local_evaluate_kernel(const float* __restrict__ params, uint32_t n_params,
                                      const float4* __restrict__ o, uint32_t n, float* __restrict__ out)
{
    constexpr int CP = MODEL == kModelDTI ? 6 : n_coef_full(LMAX);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float raw[CP], c[CP];
#pragma unroll
    for (int k = 0; k < CP; ++k) raw[k] = (uint32_t)k < n_params ? params[(size_t)i * n_params + k] : 0.0f;
    model_coefficients<MODEL, LMAX, CP>(raw, c);
    const float4 v = o[i];
    const Frame f = frame_of(v.x, v.y, v.z);
    const ModelValue r = model_eval<MODEL, LMAX>(c, v.x, v.y, v.z, f);
    out[3 * (size_t)i] = r.value;
    out[3 * (size_t)i + 1] = r.dtheta;
    out[3 * (size_t)i + 2] = r.dphi;
}

template <int MODEL, int LMAX, int ALGO>
__global__ void update_orientation_kernel(AlgoParams a, uint32_t rng_seed, uint64_t seed_offset,
                                          const float* __restrict__ params, uint32_t n_params,
                                          const float4* __restrict__ o, uint32_t n, float4* __restrict__ out)
{
    constexpr int CP = MODEL == kModelDTI ? 6 : n_coef_full(LMAX);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float raw[CP], c[CP];
#pragma unroll
    for (int k = 0; k < CP; ++k) raw[k] = (uint32_t)k < n_params ? params[(size_t)i * n_params + k] : 0.0f;
    model_coefficients<MODEL, LMAX, CP>(raw, c);
    RngState rng;
    rng.mwc = rng_init(rng_seed, i);
    rng.index = seed_offset + i;
    rng.step = 0u;
    float4 v = o[i];
    update_orientation<MODEL, LMAX, ALGO>(a, c, v.x, v.y, v.z, rng);
    out[i] = make_float4(v.x, v.y, v.z, 0.0f);
}

__global__ void rng_stream_kernel(int which, uint32_t s0, uint32_t s1, uint32_t n, uint32_t max, void* out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    Mwc s;
    s.x = s0;
    s.c = s1;
    for (uint32_t i = 0; i < n; ++i) {
        if (which == 0) reinterpret_cast<float*>(out)[i] = randu(s);
        else if (which == 1) reinterpret_cast<float*>(out)[i] = randn(s);
        else reinterpret_cast<uint32_t*>(out)[i] = randi(s, max);
    }
}

static Grid grid_of(const float* inv, uint32_t nx, uint32_t ny, uint32_t nz)
{
    Grid g;
    g.row0 = make_float4(inv[0], inv[1], inv[2], inv[3]);
    g.row1 = make_float4(inv[4], inv[5], inv[6], inv[7]);
    g.row2 = make_float4(inv[8], inv[9], inv[10], inv[11]);
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    return g;
}

cudaError_t launch_contains(const DomainDev& d, const float4* points, uint32_t n, uint8_t* out, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    const int block = 256;
    contains_kernel<<<(n + block - 1) / block, block, 0, stream>>>(grid_of(d.inv_affine, d.nx, d.ny, d.nz), d.mask,
                                                                   points, n, out);
    return cudaGetLastError();
}

cudaError_t launch_field_evaluate(const FieldDev& f, const float4* points, uint32_t n, float* out,
                                  cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    const int block = 256;
    field_evaluate_kernel<<<(n + block - 1) / block, block, 0, stream>>>(grid_of(f.inv_affine, f.nx, f.ny, f.nz),
                                                                         f.data, f.n_params, f.cpad, points, n, out);
    return cudaGetLastError();
}

cudaError_t launch_local_evaluate(int model, uint32_t n_params, const float* params, const float4* o, uint32_t n,
                                  float* out, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    const int block = 128, grid = (int)((n + block - 1) / block);
    if (model == kModelDTI) {
        local_evaluate_kernel<kModelDTI, 0><<<grid, block, 0, stream>>>(params, n_params, o, n, out);
    } else {
        switch (lmax_for(n_params)) {
        case 0: local_evaluate_kernel<kModelSH, 0><<<grid, block, 0, stream>>>(params, n_params, o, n, out); break;
        case 2: local_evaluate_kernel<kModelSH, 2><<<grid, block, 0, stream>>>(params, n_params, o, n, out); break;
        case 4: local_evaluate_kernel<kModelSH, 4><<<grid, block, 0, stream>>>(params, n_params, o, n, out); break;
        case 6: local_evaluate_kernel<kModelSH, 6><<<grid, block, 0, stream>>>(params, n_params, o, n, out); break;
        case 8: local_evaluate_kernel<kModelSH, 8><<<grid, block, 0, stream>>>(params, n_params, o, n, out); break;
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

template <int M, int L>
static void launch_uo(int algorithm, int grid, int block, cudaStream_t stream, const AlgoParams& a, uint32_t rng_seed,
                      uint64_t seed_offset, const float* params, uint32_t n_params, const float4* o, uint32_t n,
                      float4* out)
{
    if (algorithm == kTransport)
        update_orientation_kernel<M, L, kTransport><<<grid, block, 0, stream>>>(a, rng_seed, seed_offset, params,
                                                                                n_params, o, n, out);
    else
        update_orientation_kernel<M, L, kDiffusion><<<grid, block, 0, stream>>>(a, rng_seed, seed_offset, params,
                                                                                n_params, o, n, out);
}

cudaError_t launch_update_orientation(int model, uint32_t n_params, int algorithm, const AlgoParams& a,
                                      uint32_t rng_seed, uint64_t seed_offset, const float* params, const float4* o,
                                      uint32_t n, float4* out, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    const int block = 128, grid = (int)((n + block - 1) / block);
    if (model == kModelDTI) {
        launch_uo<kModelDTI, 0>(algorithm, grid, block, stream, a, rng_seed, seed_offset, params, n_params, o, n, out);
    } else {
        switch (lmax_for(n_params)) {
        case 0: launch_uo<kModelSH, 0>(algorithm, grid, block, stream, a, rng_seed, seed_offset, params, n_params, o, n, out); break;
        case 2: launch_uo<kModelSH, 2>(algorithm, grid, block, stream, a, rng_seed, seed_offset, params, n_params, o, n, out); break;
        case 4: launch_uo<kModelSH, 4>(algorithm, grid, block, stream, a, rng_seed, seed_offset, params, n_params, o, n, out); break;
        case 6: launch_uo<kModelSH, 6>(algorithm, grid, block, stream, a, rng_seed, seed_offset, params, n_params, o, n, out); break;
        case 8: launch_uo<kModelSH, 8>(algorithm, grid, block, stream, a, rng_seed, seed_offset, params, n_params, o, n, out); break;
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

// domain.py:95-120 domain_sample_boundary + :520-545 per seed: triangle by
// the normalised cumulative areas, uniform point in it, inward normal, point
// moved 1e-4 inward.  Vector operations in the reference's order (OpenCL
// float3 arithmetic component by component, normalize = v / length(v)).
__global__ void __launch_bounds__(128) boundary_seeds_kernel(const float4* __restrict__ vertices,
                                                             const uint4* __restrict__ triangles,
                                                             const float* __restrict__ cumulative,
                                                             uint32_t n_triangles, uint32_t rng_seed, uint32_t n,
                                                             float4* __restrict__ out)
{
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n) return;
    Mwc st = rng_init(rng_seed, gid);
    float px, py, pz, ox, oy, oz;
    sample_boundary(vertices, triangles, cumulative, n_triangles, st, px, py, pz, ox, oy, oz);
    out[2 * (size_t)gid] = make_float4(px, py, pz, 1.0f);
    out[2 * (size_t)gid + 1] = make_float4(ox, oy, oz, 0.0f);
}

cudaError_t launch_boundary_seeds(const float4* vertices, const uint4* triangles, const float* cumulative,
                                  uint32_t n_triangles, uint32_t rng_seed, uint32_t n, float4* out,
                                  cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    boundary_seeds_kernel<<<(n + 127) / 128, 128, 0, stream>>>(vertices, triangles, cumulative, n_triangles,
                                                              rng_seed, n, out);
    return cudaGetLastError();
}

cudaError_t launch_rng_streams(int which, uint32_t s0, uint32_t s1, uint32_t n, uint32_t max, void* out,
                               cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    rng_stream_kernel<<<1, 1, 0, stream>>>(which, s0, s1, n, max, out);
    return cudaGetLastError();
}

}  // namespace tg
