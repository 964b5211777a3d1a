/*
 * step_costs.cu -- instruction cost of the tracking step's device functions.
 *
 * A measurement program, not part of the library: one kernel per function
 * of the per-step arithmetic (tg_fmath.h, tg_device.cuh, the folded SH
 * evaluation), each thread calling it REPS times in a dependent chain, plus
 * a kernel with the same loop and a trivial body.  Run under ncu with
 *     --metrics smsp__inst_executed.sum,smsp__thread_inst_executed.sum
 * thread instructions / (threads x REPS), minus the trivial kernel's, is the
 * cost of one call with the warp converged.  Every index stays below n and
 * every loop is bounded.
 */
#include <cuda_runtime.h>

#include <cstdio>

#include "tg_step.cuh"

using namespace tg;

namespace {

constexpr int REPS = 64;

__global__ void cost_loop(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i];
    for (int r = 0; r < REPS; ++r) x = x * 1.0001f + 0.5f;
    out[i] = x;
}

__global__ void cost_log(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i];
    for (int r = 0; r < REPS; ++r) x = tgm_logf(x * 1.0001f + 0.5f) + 1.0f;
    out[i] = x;
}

__global__ void cost_log_pos(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i];
    for (int r = 0; r < REPS; ++r) x = tgm_log_pos(x * 1.0001f + 0.5f) + 1.0f;
    out[i] = x;
}

__global__ void cost_exp(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i];
    for (int r = 0; r < REPS; ++r) x = tgm_expf(x * 1.0001f + 0.5f) * 1e-3f;
    out[i] = x;
}

__global__ void cost_div(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i];
    for (int r = 0; r < REPS; ++r) x = 1.0f / (x * 1.0001f + 0.5f);
    out[i] = x;
}

__global__ void cost_sqrt(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i];
    for (int r = 0; r < REPS; ++r) x = sqrtf(x * 1.0001f + 0.5f);
    out[i] = x;
}

__global__ void cost_cos2pi(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = __float_as_uint(in[i]);
    float acc = 0.0f;
    for (int r = 0; r < REPS; ++r) {
        acc += tgm_cos2pi_u24(k & 0xffffffu);
        k = k * 1664525u + 1013904223u;
    }
    out[i] = acc;
}

__global__ void cost_randn(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Mwc s = rng_init(__float_as_uint(in[i]), (uint32_t)i);
    float acc = 0.0f;
    for (int r = 0; r < REPS; ++r) acc += randn(s);
    out[i] = acc;
}

__global__ void cost_frame(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i], y = 0.3f, z = 0.5f;
    for (int r = 0; r < REPS; ++r) {
        const Frame f = frame_of(x, y, z);
        x = f.ct + 0.1f;
        y = f.sp;
        z = f.cp;
    }
    out[i] = x + y + z;
}

__global__ void cost_sh8(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c[48];
    for (int k = 0; k < 48; ++k) c[k] = in[(i + k) % n];
    float ct = 0.3f, cp = 0.6f, acc = 0.0f;
    for (int r = 0; r < REPS; ++r) {
        float v, dt, dp;
        sh_eval_folded<8>(c, ct, 0.9f, cp, 0.8f, &v, &dt, &dp);
        acc += v;
        ct = fminf(dt, 0.9f);
        cp = fminf(dp, 0.9f);
    }
    out[i] = acc;
}

__global__ void cost_softplus(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[i] * 0.01f - 0.2f, acc = 0.0f;
    for (int r = 0; r < REPS; ++r) {
        float v, d, q;
        tgm_softplus(x, kSoftmaxScale, kSoftmaxInvScale, &v, &d, &q);
        acc += d + q;
        x = v - 0.25f;
    }
    out[i] = acc;
}

__global__ void cost_exps2(const float* in, float* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float ox = 0.0f, oy = 0.6f, oz = 0.8f;
    const float t = in[i] * 1e-3f;
    for (int r = 0; r < REPS; ++r) exps2(ox, oy, oz, t, -t, 0.5f * t);
    out[i] = ox + oy + oz;
}

template <int ALGO>
__global__ void cost_update(const float* in, float* out, int n, AlgoParams a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float raw[45], c[45];
    for (int k = 0; k < 45; ++k) raw[k] = in[(i * 7 + k) % n] * 0.05f;
    raw[0] = 0.3f;
    tgsh_fold(8, raw, c);
    RngState rng;
    rng.mwc = rng_init(7u, (uint32_t)i);
    rng.index = (uint64_t)i;
    rng.step = 0u;
    float ox = 0.0f, oy = 0.6f, oz = 0.8f;
    for (int r = 0; r < REPS; ++r) update_orientation<kModelSH, 8, ALGO>(a, c, ox, oy, oz, rng);
    out[i] = ox + oy + oz;
}

}  // namespace

int main()
{
    const int n = 148 * 1024;
    const int block = 128, grid = n / block;
    float *in = nullptr, *out = nullptr;
    if (cudaMalloc(&in, n * sizeof(float)) != cudaSuccess || cudaMalloc(&out, n * sizeof(float)) != cudaSuccess) {
        std::fprintf(stderr, "step_costs: device allocation failed\n");
        return 1;
    }
    float* host = new float[n];
    for (int i = 0; i < n; ++i) host[i] = 0.25f + (float)(((uint32_t)i * 2654435761u) >> 8) * 0x1p-24f;
    cudaMemcpy(in, host, n * sizeof(float), cudaMemcpyHostToDevice);
    delete[] host;
    AlgoParams a{};
    a.step_size = 0.001f;
    a.gamma = 1.0f;
    a.noise_variance = 0.1f;
    a.scale_drift = 0.001f;
    a.scale_noise = sqrtf(0.1f * 0.001f);
    a.rng_mode = kRngMWC64X;
    cost_loop<<<grid, block>>>(in, out, n);
    cost_log<<<grid, block>>>(in, out, n);
    cost_log_pos<<<grid, block>>>(in, out, n);
    cost_exp<<<grid, block>>>(in, out, n);
    cost_div<<<grid, block>>>(in, out, n);
    cost_sqrt<<<grid, block>>>(in, out, n);
    cost_cos2pi<<<grid, block>>>(in, out, n);
    cost_randn<<<grid, block>>>(in, out, n);
    cost_frame<<<grid, block>>>(in, out, n);
    cost_sh8<<<grid, block>>>(in, out, n);
    cost_softplus<<<grid, block>>>(in, out, n);
    cost_exps2<<<grid, block>>>(in, out, n);
    cost_update<kTransport><<<grid, block>>>(in, out, n, a);
    cost_update<kDiffusion><<<grid, block>>>(in, out, n, a);
    const cudaError_t e = cudaDeviceSynchronize();
    std::printf("step_costs: %s (%d threads, %d calls each)\n", cudaGetErrorString(e), n, REPS);
    cudaFree(in);
    cudaFree(out);
    return e == cudaSuccess ? 0 : 1;
}
