/*
 * tg_capi.cu -- the C ABI declared in include/tractography_b200.h.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "tg_internal.h"
#include "tg_step.cuh"
#include "tractography_b200.h"

using namespace tg;

struct tg_field {
    FieldDev d;
};

struct tg_domain {
    DomainDev d;
};

struct tg_tracker {
    uint64_t pool_points_request = 0;
    // chunk pool
    float* pool = nullptr;
    int32_t* chunk_next = nullptr;
    uint32_t n_chunks = 0;
    // counters: [0] items, [1] steps; chunk counter separately
    unsigned long long* counters = nullptr;
    unsigned int* chunk_counter = nullptr;
    // per-seed buffers
    int32_t* first_chunk = nullptr;
    uint32_t* lengths = nullptr;
    uint64_t* offsets = nullptr;
    uint32_t* ids = nullptr;
    uint32_t* done_ids = nullptr;
    size_t cap_seeds = 0;
    // closed-surface domain: the seeds' inside tests, done before tracking
    uint8_t* seed_inside = nullptr;
    size_t cap_seed_inside = 0;
    // device offsets of a run whose streamlines all fit the pool
    uint64_t* masked = nullptr;
    size_t cap_masked = 0;
    uint8_t* scan_temp = nullptr;
    size_t cap_scan_temp = 0;
    unsigned long long* d_totals = nullptr;
    size_t cap_totals = 0;
    float4* seeds = nullptr;
    size_t cap_seed_copy = 0;
    uint32_t* batch_seeds = nullptr;
    size_t cap_batches = 0;
    // packed output
    float* points = nullptr;
    uint64_t cap_points = 0;
    uint64_t total_points = 0;
    // host staging
    std::vector<uint32_t> h_len;
    std::vector<uint32_t> h_done;
    std::vector<uint32_t> h_retry;
    // multi-job runs: one stream per code path, job and class tables
    cudaStream_t class_stream[kClassKinds] = {};
    cudaEvent_t class_done[kClassKinds] = {};
    cudaEvent_t ev_fork = nullptr;
    JobDev* d_jobs = nullptr;
    size_t cap_jobs = 0;
    uint32_t* d_job_base = nullptr;
    size_t cap_job_base = 0;
    uint32_t* d_class_lists = nullptr;   // job lists and prefixes of all classes
    size_t cap_class_lists = 0;
    unsigned long long* d_class_counters = nullptr;
    // launch shape and tail compaction (tg_tracker_set_tuning); slot
    // kClassKinds holds the single-job tracker's carry buffers
    uint32_t blocks_per_sm = 0;        // 0: the occupancy maximum
    uint32_t compact_lanes = 0;        // 0: no compaction (measured faster by default)
    uint32_t compact_rounds = 4;
    // time slicing of tg_tracker_run (tg_tracker_set_slicing): the ring of
    // saved streamlines, its seq and released words and its control words
    uint32_t slice_steps = kDefaultSliceSteps;
    LaneCarry* ring_items = nullptr;
    size_t cap_ring = 0;
    uint32_t* ring_flags = nullptr;    // seq then released, cap_ring each
    size_t cap_ring_flags = 0;
    unsigned int* ring_ctl = nullptr;  // head, tail, fault, spare
    size_t cap_ring_ctl = 0;
    LaneCarry* carry[kClassKinds + 1][2] = {};
    size_t carry_cap[kClassKinds + 1] = {};
    unsigned int* carry_count = nullptr;   // 2 per slot
    // statistics of the last run
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    float kernel_ms = 0.0f;
    uint32_t waves = 0;
    uint32_t launches = 0;
};

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg)
{
    g_error = msg;
    return code;
}

int fail_cuda(cudaError_t e, const char* what)
{
    const int code = (e == cudaErrorMemoryAllocation) ? TG_ERR_OUT_OF_MEMORY : TG_ERR_CUDA;
    return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define TG_TRY(call)                                     \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call); \
    } while (0)

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

Grid grid_of(const float* inv, uint32_t nx, uint32_t ny, uint32_t nz)
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

int check_algorithm(const tg_algorithm* a)
{
    if (a == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "algorithm is null");
    if (a->algorithm != TG_ALGO_TRANSPORT && a->algorithm != TG_ALGO_DIFFUSION)
        return fail(TG_ERR_UNSUPPORTED, "unsupported algorithm id");
    if (!std::isfinite(a->step_size) || a->step_size <= 0.0f)
        return fail(TG_ERR_INVALID_ARGUMENT, "step_size must be finite and positive");
    if (!std::isfinite(a->gamma)) return fail(TG_ERR_INVALID_ARGUMENT, "gamma must be finite");
    if (a->algorithm == TG_ALGO_DIFFUSION && (!std::isfinite(a->noise_variance) || a->noise_variance < 0.0f))
        return fail(TG_ERR_INVALID_ARGUMENT, "noise_variance must be finite and non-negative");
    if (a->rng_mode != TG_RNG_MWC64X && a->rng_mode != TG_RNG_PHILOX)
        return fail(TG_ERR_UNSUPPORTED, "unsupported rng_mode");
    return TG_OK;
}

AlgoParams algo_params(const tg_algorithm* a)
{
    AlgoParams p;
    p.step_size = a->step_size;
    p.gamma = a->gamma;
    p.noise_variance = a->algorithm == TG_ALGO_DIFFUSION ? a->noise_variance : 0.0f;
    // algorithm.py:106 and 222-225, evaluated in binary32 as the kernel would.
    p.scale_drift = a->gamma * a->step_size;
    p.scale_noise = sqrtf(p.noise_variance * a->gamma * a->step_size);
    p.rng_mode = a->rng_mode;
    p.philox_key = a->philox_key;
    return p;
}

}  // namespace

namespace tg {

// The most iterations of tracking.py:121-147 that can separate two saved
// points, or 0 when some streamline would never save another one.
//
// The loop adds step to time in binary32 until time >= save_at.  Rounding
// is monotonic, so a time that starts higher never falls behind one that
// starts at 0: the count from time = 0 is the worst case.  In the binade
// [2^(e-1), 2^e) (spacing u = 2^(e-24)) an iteration whose sum stays in the
// binade advances time by at least inc = step rounded down to a multiple of
// u (up to one when the remainder exceeds u/2), and one more iteration
// leaves the binade.  Where inc is 0 -- step at most half the spacing of
// the largest float below save_at -- time + step == time for some time and
// the streamline never ends.  The sum over binades bounds the count.
uint64_t steps_per_point_bound(float step, float save_at)
{
    if (!(step > 0.0f) || !(save_at > 0.0f) || !std::isfinite(step) || !std::isfinite(save_at)) return 0;
    if (step >= save_at) return 1;   // every iteration saves a point
    const double s = step;
    uint64_t count = 1;              // the first iteration: time 0 -> step, exact
    int e = 0;
    std::frexp(step, &e);            // step in [2^(e-1), 2^e)
    double lo = s;
    while (lo < (double)save_at) {
        const double hi = std::min(std::ldexp(1.0, e), (double)save_at);
        // spacing of binary32 values in [2^(e-1), 2^e); subnormal spacing below
        const double u = std::ldexp(1.0, std::max(e - 24, -149));
        const double q = std::floor(s / u);
        const double r = s - q * u;
        const double inc = (r > 0.5 * u) ? (q + 1.0) * u : q * u;
        if (inc <= 0.0) return 0;
        const double n = std::floor((hi - lo) / inc) + 1.0;
        if (n > 1e18) return 0;
        count += (uint64_t)n;
        lo = hi;
        ++e;
    }
    return count;
}

}  // namespace tg

namespace {

int step_bound(float step, float save_at, uint32_t n_steps, uint64_t* out)
{
    const uint64_t per_point = steps_per_point_bound(step, save_at);
    if (per_point == 0)
        return fail(TG_ERR_INVALID_ARGUMENT,
                    "step_size is too small for save_at: in float32, time + step_size no longer "
                    "reaches save_at, so streamlines would never end");
    const uint64_t bound = (uint64_t)std::max<uint32_t>(n_steps, 1u) * per_point;
    if (per_point > 0xffffffffull || bound > 0xffffffffull)
        return fail(TG_ERR_INVALID_ARGUMENT,
                    "step_size is too small for save_at and the maximum streamline length: a "
                    "streamline could take more than 2^32 - 1 steps");
    *out = bound;
    return TG_OK;
}

// make_track_params checks save_at against step_size (the reference's
// tractogram loop) unless the caller's loop counts steps instead of time
// (TOD, connectome: tracking.py:181-385, 388-602).
int make_track_params(const tg_algorithm* a, const tg_domain* d, const tg_field* f, float save_at,
                      uint32_t n_steps, TrackParams* out, bool time_loop = true)
{
    int st = check_algorithm(a);
    if (st != TG_OK) return st;
    if (!std::isfinite(save_at) || save_at <= 0.0f)
        return fail(TG_ERR_INVALID_ARGUMENT, "save_at must be finite and positive");
    uint32_t max_steps = 0xffffffffu;
    if (time_loop) {
        uint64_t bound = 0;
        st = step_bound(a->step_size, save_at, n_steps, &bound);
        if (st != TG_OK) return st;
        max_steps = (uint32_t)bound;
    }
    if (d == nullptr || f == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "domain and field are required");
    TrackParams p;
    std::memset(&p, 0, sizeof p);
    p.domain_kind = d->d.kind;
    p.fgrid = grid_of(f->d.inv_affine, f->d.nx, f->d.ny, f->d.nz);
    p.field = f->d.folded;
    p.cpad = f->d.cpad;
    if (d->d.kind == kDomainMesh) {
        p.mesh = d->d.mesh;
        p.same_grid = 0;
    } else {
        p.dgrid = grid_of(d->d.inv_affine, d->d.nx, d->d.ny, d->d.nz);
        p.mask = d->d.mask;
        // one voxel test serves both images (tg_step.cuh locate) for axes
        // below 2^22 voxels, where voxel index +- 0.5 is exact in binary32
        p.same_grid = d->d.nx == f->d.nx && d->d.ny == f->d.ny && d->d.nz == f->d.nz &&
                      std::memcmp(d->d.inv_affine, f->d.inv_affine, 12 * sizeof(float)) == 0 &&
                      f->d.nx < (1u << 22) && f->d.ny < (1u << 22) && f->d.nz < (1u << 22);
    }
    p.algorithm = a->algorithm;
    p.algo = algo_params(a);
    p.save_at = save_at;
    p.n_steps = n_steps;
    p.max_steps = max_steps;
    *out = p;
    return TG_OK;
}

template <typename T>
cudaError_t ensure(T** ptr, size_t* cap, size_t n)
{
    if (*cap >= n && *ptr != nullptr) return cudaSuccess;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    const size_t want = std::max<size_t>(n, 1);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(ptr), want * sizeof(T));
    if (e == cudaSuccess) *cap = want;
    return e;
}

int sm_count()
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

}  // namespace

namespace tg {

// Used by tg_noalloc.cu, which cannot see the handle layouts.
int track_params_from_handles(const tg_algorithm* a, const tg_domain* d, const tg_field* f, float save_at,
                              uint32_t n_steps, TrackParams* out, int* model, int* lmax)
{
    const int st = make_track_params(a, d, f, save_at, n_steps, out);
    if (st != TG_OK) return st;
    *model = f->d.model;
    *lmax = f->d.lmax;
    return TG_OK;
}

int set_last_error(int code, const std::string& msg) { return fail(code, msg); }

}  // namespace tg

extern "C" {

int tg_abi_version(void) { return TG_ABI_VERSION; }

const char* tg_status_string(int status)
{
    switch (status) {
    case TG_OK: return "ok";
    case TG_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TG_ERR_CUDA: return "CUDA error";
    case TG_ERR_OUT_OF_MEMORY: return "out of device memory";
    case TG_ERR_UNSUPPORTED: return "unsupported";
    case TG_ERR_POOL_EXHAUSTED: return "point pool exhausted";
    default: return "unknown status";
    }
}

const char* tg_last_error(void) { return g_error.c_str(); }

int tg_field_create(int32_t model, const float* values, uint32_t nx, uint32_t ny, uint32_t nz,
                    uint32_t n_parameters, const float inverse_affine[16], void* stream, tg_field** out)
{
    if (out == nullptr || values == nullptr || inverse_affine == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (nx == 0 || ny == 0 || nz == 0 || n_parameters == 0)
        return fail(TG_ERR_INVALID_ARGUMENT, "field dimensions must be positive");
    if (model == TG_MODEL_SH && n_parameters > 45)
        return fail(TG_ERR_UNSUPPORTED, "spherical-harmonic fields support at most 45 coefficients (lmax 8)");
    if (model == TG_MODEL_DTI && n_parameters != 6)
        return fail(TG_ERR_INVALID_ARGUMENT, "tensor fields have 6 coefficients");
    if (model != TG_MODEL_SH && model != TG_MODEL_DTI) return fail(TG_ERR_UNSUPPORTED, "unknown model");
    tg_field* f = new tg_field();
    f->d.nx = nx;
    f->d.ny = ny;
    f->d.nz = nz;
    f->d.n_params = n_parameters;
    f->d.model = model;
    f->d.lmax = model == TG_MODEL_SH ? lmax_for(n_parameters) : 0;
    f->d.cpad = model == TG_MODEL_SH ? (uint32_t)((n_coef_full(f->d.lmax) + 3) / 4 * 4) : 8u;
    std::memcpy(f->d.inv_affine, inverse_affine, sizeof f->d.inv_affine);
    const size_t nvox = (size_t)nx * ny * nz;
    f->d.bytes = nvox * f->d.cpad * sizeof(float);
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&f->d.data), f->d.bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(f->d.data, 0, f->d.bytes, s);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(f->d.data, f->d.cpad * sizeof(float), values, n_parameters * sizeof(float),
                              n_parameters * sizeof(float), nvox, cudaMemcpyHostToDevice, s);
    // the trackers' copy: SH coefficients folded per voxel, tensors as given
    if (e == cudaSuccess && model == TG_MODEL_SH) {
        e = cudaMalloc(reinterpret_cast<void**>(&f->d.folded), f->d.bytes);
        if (e == cudaSuccess) e = launch_fold_field(f->d.data, f->d.folded, nvox, f->d.cpad, f->d.lmax, s);
    } else if (e == cudaSuccess) {
        f->d.folded = f->d.data;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        if (f->d.folded && f->d.folded != f->d.data) cudaFree(f->d.folded);
        if (f->d.data) cudaFree(f->d.data);
        delete f;
        return fail_cuda(e, "tg_field_create");
    }
    *out = f;
    return TG_OK;
}

int tg_field_destroy(tg_field* field)
{
    if (field == nullptr) return TG_OK;
    if (field->d.folded && field->d.folded != field->d.data) cudaFree(field->d.folded);
    if (field->d.data) cudaFree(field->d.data);
    delete field;
    return TG_OK;
}

int tg_domain_create(const uint8_t* mask, uint32_t nx, uint32_t ny, uint32_t nz, const float inverse_affine[16],
                     void* stream, tg_domain** out)
{
    if (out == nullptr || mask == nullptr || inverse_affine == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (nx == 0 || ny == 0 || nz == 0) return fail(TG_ERR_INVALID_ARGUMENT, "domain dimensions must be positive");
    tg_domain* d = new tg_domain();
    d->d.nx = nx;
    d->d.ny = ny;
    d->d.nz = nz;
    std::memcpy(d->d.inv_affine, inverse_affine, sizeof d->d.inv_affine);
    d->d.bytes = (size_t)nx * ny * nz;
    cudaStream_t s = as_stream(stream);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&d->d.mask), d->d.bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d->d.mask, mask, d->d.bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        if (d->d.mask) cudaFree(d->d.mask);
        delete d;
        return fail_cuda(e, "tg_domain_create");
    }
    *out = d;
    return TG_OK;
}

int tg_domain_destroy(tg_domain* domain)
{
    if (domain == nullptr) return TG_OK;
    if (domain->d.mask) cudaFree(domain->d.mask);
    if (domain->d.nodes) cudaFree(domain->d.nodes);
    if (domain->d.tris) cudaFree(domain->d.tris);
    if (domain->d.cells) cudaFree(domain->d.cells);
    if (domain->d.lists) cudaFree(domain->d.lists);
    delete domain;
    return TG_OK;
}

int tg_domain_create_mesh(const double* vertices, uint32_t n_vertices, const uint32_t* faces, uint32_t n_faces,
                          void* stream, tg_domain** out)
{
    if (out == nullptr || vertices == nullptr || faces == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    BoundaryBvhHost b;
    std::string err;
    if (build_boundary_bvh(vertices, n_vertices, faces, n_faces, &b, &err) != 0)
        return fail(TG_ERR_INVALID_ARGUMENT, err);
    tg_domain* d = new tg_domain();
    const cudaError_t e = upload_mesh(b, &d->d, as_stream(stream));
    if (e != cudaSuccess) {
        tg_domain_destroy(d);
        return fail_cuda(e, "tg_domain_create_mesh");
    }
    *out = d;
    return TG_OK;
}

int tg_bvh_build_host(const double* vertices, uint32_t n_vertices, const uint32_t* faces, uint32_t n_faces,
                      uint32_t* n_triangles, uint32_t* n_nodes, float* vertices4, uint32_t* triangles4,
                      float* bounds_min, float* bounds_max, int32_t* nodes, uint32_t* ordered_triangles)
{
    if (vertices == nullptr || faces == nullptr || n_triangles == nullptr || n_nodes == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    BoundaryBvhHost b;
    std::string err;
    if (build_boundary_bvh(vertices, n_vertices, faces, n_faces, &b, &err) != 0)
        return fail(TG_ERR_INVALID_ARGUMENT, err);
    *n_triangles = b.n_triangles;
    *n_nodes = b.n_nodes;
    if (vertices4 == nullptr || triangles4 == nullptr || bounds_min == nullptr || bounds_max == nullptr ||
        nodes == nullptr || ordered_triangles == nullptr)
        return TG_OK;
    std::memcpy(vertices4, b.vertices4.data(), b.vertices4.size() * sizeof(float));
    std::memcpy(triangles4, b.triangles4.data(), b.triangles4.size() * sizeof(uint32_t));
    std::memcpy(bounds_min, b.bounds_min.data(), b.bounds_min.size() * sizeof(float));
    std::memcpy(bounds_max, b.bounds_max.data(), b.bounds_max.size() * sizeof(float));
    std::memcpy(nodes, b.nodes.data(), b.nodes.size() * sizeof(int32_t));
    std::memcpy(ordered_triangles, b.ordered.data(), b.ordered.size() * sizeof(uint32_t));
    return TG_OK;
}

int tg_mesh_info(const tg_domain* domain, uint32_t* n_triangles, uint32_t* n_nodes, uint32_t grid[3],
                 uint64_t* device_bytes)
{
    if (domain == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "domain is null");
    if (domain->d.kind != kDomainMesh) return fail(TG_ERR_INVALID_ARGUMENT, "not a mesh domain");
    if (n_triangles) *n_triangles = domain->d.n_triangles;
    if (n_nodes) *n_nodes = domain->d.mesh.n_nodes;
    if (grid) {
        grid[0] = domain->d.nx;
        grid[1] = domain->d.ny;
        grid[2] = domain->d.nz;
    }
    if (device_bytes) *device_bytes = domain->d.bytes;
    return TG_OK;
}

int tg_mesh_segment_hits(const tg_domain* domain, const float* starts, const float* ends, uint32_t n,
                         uint8_t* found, uint32_t* triangle, float* hit, void* stream)
{
    if (domain == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "domain is null");
    if (domain->d.kind != kDomainMesh) return fail(TG_ERR_INVALID_ARGUMENT, "not a mesh domain");
    if (n == 0) return TG_OK;
    TG_TRY(launch_mesh_segment_hits(domain->d.mesh, reinterpret_cast<const float4*>(starts),
                                    reinterpret_cast<const float4*>(ends), n, found, triangle,
                                    reinterpret_cast<float4*>(hit), as_stream(stream)));
    return TG_OK;
}

int tg_mesh_segments_blocked(const tg_domain* domain, const float* starts, const float* ends, uint32_t n,
                             uint8_t* blocked, void* stream)
{
    if (domain == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "domain is null");
    if (domain->d.kind != kDomainMesh) return fail(TG_ERR_INVALID_ARGUMENT, "not a mesh domain");
    if (n == 0) return TG_OK;
    TG_TRY(launch_mesh_segments_blocked(domain->d.mesh, reinterpret_cast<const float4*>(starts),
                                        reinterpret_cast<const float4*>(ends), n, blocked, as_stream(stream)));
    return TG_OK;
}

int tg_tractogram(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field, const float* seeds,
                  uint32_t n_seeds, float save_at, uint32_t n_steps, float* streamlines, uint32_t* lengths,
                  void* stream)
{
    TrackParams p;
    int st = make_track_params(algorithm, domain, field, save_at, n_steps, &p);
    if (st != TG_OK) return st;
    if (n_seeds == 0) return TG_OK;
    if (n_steps == 0) return fail(TG_ERR_INVALID_ARGUMENT, "n_steps must be positive");
    if (seeds == nullptr || streamlines == nullptr || lengths == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null buffer");
    TG_TRY(launch_track_dense(field->d, p, reinterpret_cast<const float4*>(seeds), n_seeds, algorithm->rng_seed,
                              algorithm->seed_offset, reinterpret_cast<float4*>(streamlines), lengths,
                              as_stream(stream)));
    return TG_OK;
}

int tg_tractogram_host(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                       const float* seeds, uint32_t n_seeds, float save_at, uint32_t n_steps, float* streamlines,
                       uint32_t* lengths, void* stream)
{
    TrackParams p;
    int st = make_track_params(algorithm, domain, field, save_at, n_steps, &p);
    if (st != TG_OK) return st;
    if (n_seeds == 0) return TG_OK;
    if (n_steps == 0) return fail(TG_ERR_INVALID_ARGUMENT, "n_steps must be positive");
    cudaStream_t s = as_stream(stream);
    float* d_seeds = nullptr;
    float* d_out = nullptr;
    uint32_t* d_len = nullptr;
    const size_t out_bytes = (size_t)n_seeds * n_steps * 4 * sizeof(float);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&d_seeds), (size_t)n_seeds * 8 * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d_out), out_bytes);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d_len), (size_t)n_seeds * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_seeds, seeds, (size_t)n_seeds * 8 * sizeof(float), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_track_dense(field->d, p, reinterpret_cast<const float4*>(d_seeds), n_seeds, algorithm->rng_seed,
                               algorithm->seed_offset, reinterpret_cast<float4*>(d_out), d_len, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(streamlines, d_out, out_bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(lengths, d_len, (size_t)n_seeds * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d_seeds);
    cudaFree(d_out);
    cudaFree(d_len);
    if (e != cudaSuccess) return fail_cuda(e, "tg_tractogram_host");
    return TG_OK;
}

int tg_tracker_create(uint64_t pool_points, tg_tracker** out)
{
    if (out == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    tg_tracker* t = new tg_tracker();
    t->pool_points_request = pool_points;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&t->counters), 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&t->chunk_counter), sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaEventCreate(&t->ev_start);
    if (e == cudaSuccess) e = cudaEventCreate(&t->ev_stop);
    if (e != cudaSuccess) {
        tg_tracker_destroy(t);
        return fail_cuda(e, "tg_tracker_create");
    }
    *out = t;
    return TG_OK;
}

int tg_tracker_destroy(tg_tracker* t)
{
    if (t == nullptr) return TG_OK;
    cudaFree(t->pool);
    cudaFree(t->chunk_next);
    cudaFree(t->counters);
    cudaFree(t->chunk_counter);
    cudaFree(t->first_chunk);
    cudaFree(t->lengths);
    cudaFree(t->offsets);
    cudaFree(t->ids);
    cudaFree(t->done_ids);
    cudaFree(t->masked);
    cudaFree(t->seed_inside);
    cudaFree(t->scan_temp);
    cudaFree(t->d_totals);
    cudaFree(t->seeds);
    cudaFree(t->batch_seeds);
    cudaFree(t->points);
    cudaFree(t->ring_items);
    cudaFree(t->ring_flags);
    cudaFree(t->ring_ctl);
    if (t->ev_start) cudaEventDestroy(t->ev_start);
    if (t->ev_stop) cudaEventDestroy(t->ev_stop);
    for (int k = 0; k < kClassKinds; ++k) {
        if (t->class_stream[k]) cudaStreamDestroy(t->class_stream[k]);
        if (t->class_done[k]) cudaEventDestroy(t->class_done[k]);
    }
    if (t->ev_fork) cudaEventDestroy(t->ev_fork);
    cudaFree(t->d_jobs);
    cudaFree(t->d_job_base);
    cudaFree(t->d_class_lists);
    cudaFree(t->d_class_counters);
    for (int k = 0; k <= kClassKinds; ++k) {
        cudaFree(t->carry[k][0]);
        cudaFree(t->carry[k][1]);
    }
    cudaFree(t->carry_count);
    delete t;
    return TG_OK;
}

int tg_tracker_set_tuning(tg_tracker* t, uint32_t blocks_per_sm, uint32_t compact_lanes, uint32_t compact_rounds)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    if (compact_lanes > 31) return fail(TG_ERR_INVALID_ARGUMENT, "compact_lanes must be at most 31");
    if (compact_rounds > 16) return fail(TG_ERR_INVALID_ARGUMENT, "compact_rounds must be at most 16");
    if (blocks_per_sm > 32) return fail(TG_ERR_INVALID_ARGUMENT, "blocks_per_sm must be at most 32");
    t->blocks_per_sm = blocks_per_sm;
    t->compact_lanes = compact_lanes;
    t->compact_rounds = compact_rounds;
    return TG_OK;
}

int tg_tracker_set_slicing(tg_tracker* t, uint32_t slice_steps)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    if (slice_steps > (1u << 30) || (slice_steps & (slice_steps - 1u)) != 0u)
        return fail(TG_ERR_INVALID_ARGUMENT, "slice_steps must be 0 or a power of two up to 2^30");
    t->slice_steps = slice_steps;
    return TG_OK;
}

int tg_tracker_get_slicing(const tg_tracker* t, uint32_t* slice_steps)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    if (slice_steps) *slice_steps = t->slice_steps;
    return TG_OK;
}

int tg_tracker_get_tuning(const tg_tracker* t, uint32_t* blocks_per_sm, uint32_t* compact_lanes,
                          uint32_t* compact_rounds)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    if (blocks_per_sm) *blocks_per_sm = t->blocks_per_sm;
    if (compact_lanes) *compact_lanes = t->compact_lanes;
    if (compact_rounds) *compact_rounds = t->compact_rounds;
    return TG_OK;
}

int tg_tracker_stats(const tg_tracker* t, float* kernel_ms, uint32_t* waves, uint32_t* launches)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    if (kernel_ms) *kernel_ms = t->kernel_ms;
    if (waves) *waves = t->waves;
    if (launches) *launches = t->launches;
    return TG_OK;
}

// Carry buffers of one slot for a grid of `lanes` threads (each lane hands
// over at most one streamline per round).
static int tracker_carry(tg_tracker* t, int slot, size_t lanes)
{
    if (t->carry_count == nullptr) {
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->carry_count), 2 * (kClassKinds + 1) * sizeof(unsigned int)));
    }
    if (t->carry_cap[slot] >= lanes && t->carry[slot][0] != nullptr) return TG_OK;
    cudaFree(t->carry[slot][0]);
    cudaFree(t->carry[slot][1]);
    t->carry[slot][0] = t->carry[slot][1] = nullptr;
    t->carry_cap[slot] = 0;
    TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->carry[slot][0]), lanes * sizeof(LaneCarry)));
    TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->carry[slot][1]), lanes * sizeof(LaneCarry)));
    t->carry_cap[slot] = lanes;
    return TG_OK;
}

static int tracker_pool(tg_tracker* t, uint64_t want_points)
{
    uint64_t chunks = (want_points + kChunkPoints - 1) / kChunkPoints;
    if (chunks < 1) chunks = 1;
    if (chunks > 0x7fffffffull) chunks = 0x7fffffffull;
    if (t->pool != nullptr && t->n_chunks >= chunks) return TG_OK;
    cudaFree(t->pool);
    cudaFree(t->chunk_next);
    t->pool = nullptr;
    t->chunk_next = nullptr;
    t->n_chunks = 0;
    TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->pool), (size_t)chunks * kChunkPoints * 3 * sizeof(float)));
    TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->chunk_next), (size_t)chunks * sizeof(int32_t)));
    t->n_chunks = (uint32_t)chunks;
    return TG_OK;
}

static int tracker_points(tg_tracker* t, uint64_t need, cudaStream_t s)
{
    if (t->cap_points >= need && t->points != nullptr) return TG_OK;
    uint64_t cap = std::max<uint64_t>(need, t->cap_points + t->cap_points / 2);
    cap = std::max<uint64_t>(cap, 1);
    float* np = nullptr;
    TG_TRY(cudaMalloc(reinterpret_cast<void**>(&np), (size_t)cap * 3 * sizeof(float)));
    if (t->points != nullptr && t->total_points > 0) {
        cudaError_t e = cudaMemcpyAsync(np, t->points, (size_t)t->total_points * 3 * sizeof(float),
                                        cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaFree(np);
            return fail_cuda(e, "grow point buffer");
        }
    }
    cudaFree(t->points);
    t->points = np;
    t->cap_points = cap;
    return TG_OK;
}

int tg_tracker_run(tg_tracker* t, const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                   const float* seeds, int seeds_on_host, uint32_t n_seeds, uint32_t batch_size,
                   const uint32_t* batch_rng_seeds, float save_at, uint32_t n_steps, uint32_t* h_lengths,
                   uint64_t* h_offsets, uint64_t* total_points, uint64_t* total_steps, void* stream)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    TrackParams tp;
    int st = make_track_params(algorithm, domain, field, save_at, n_steps, &tp);
    if (st != TG_OK) return st;
    t->total_points = 0;
    t->kernel_ms = 0.0f;
    t->waves = 0;
    t->launches = 0;
    if (total_points) *total_points = 0;
    if (total_steps) *total_steps = 0;
    if (n_seeds == 0) return TG_OK;
    if (n_steps == 0) return fail(TG_ERR_INVALID_ARGUMENT, "n_steps must be positive");
    if (batch_size == 0) return fail(TG_ERR_INVALID_ARGUMENT, "batch_size must be positive");
    if (seeds == nullptr || batch_rng_seeds == nullptr || h_lengths == nullptr || h_offsets == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null buffer");
    cudaStream_t s = as_stream(stream);
    const uint32_t n_batches = (n_seeds + batch_size - 1) / batch_size;

    TG_TRY(ensure(&t->batch_seeds, &t->cap_batches, n_batches));
    TG_TRY(cudaMemcpyAsync(t->batch_seeds, batch_rng_seeds, n_batches * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    const float4* d_seeds = reinterpret_cast<const float4*>(seeds);
    if (seeds_on_host) {
        TG_TRY(ensure(&t->seeds, &t->cap_seed_copy, (size_t)n_seeds * 2));
        TG_TRY(cudaMemcpyAsync(t->seeds, seeds, (size_t)n_seeds * 8 * sizeof(float), cudaMemcpyHostToDevice, s));
        d_seeds = t->seeds;
    }
    if (t->cap_seeds < n_seeds) {
        cudaFree(t->first_chunk);
        cudaFree(t->lengths);
        cudaFree(t->offsets);
        cudaFree(t->ids);
        cudaFree(t->done_ids);
        t->first_chunk = nullptr;
        t->lengths = nullptr;
        t->offsets = nullptr;
        t->ids = nullptr;
        t->done_ids = nullptr;
        t->cap_seeds = 0;
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->first_chunk), (size_t)n_seeds * sizeof(int32_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->lengths), (size_t)n_seeds * sizeof(uint32_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->offsets), (size_t)n_seeds * sizeof(uint64_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->ids), (size_t)n_seeds * sizeof(uint32_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->done_ids), (size_t)n_seeds * sizeof(uint32_t)));
        t->cap_seeds = n_seeds;
    }

    // Pool: the worst case (every streamline fills n_steps points, rounded
    // up to whole chunks) when it fits a third of free memory; otherwise
    // the pool is smaller and streamlines that run out are re-tracked in a
    // later wave (results depend only on the seed and its RNG stream).
    const uint64_t per_seed = ((uint64_t)n_steps + kChunkPoints - 1) / kChunkPoints * kChunkPoints;
    uint64_t want = t->pool_points_request;
    if (want == 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const uint64_t budget = (uint64_t)(free_b / 3) / (3 * sizeof(float) + 1);
        want = std::min<uint64_t>(per_seed * n_seeds, std::max<uint64_t>(budget, per_seed * 64));
    }
    st = tracker_pool(t, want);
    if (st != TG_OK) return st;

    PersistentParams pp;
    std::memset(&pp, 0, sizeof pp);
    pp.t = tp;
    pp.seeds = d_seeds;
    pp.n_seeds = n_seeds;
    pp.batch_size = batch_size;
    pp.batch_rng_seeds = t->batch_seeds;
    pp.seed_offset = algorithm->seed_offset;
    pp.item_counter = t->counters;
    pp.steps_done = t->counters + 1;
    pp.chunk_counter = t->chunk_counter;
    pp.first_chunk = t->first_chunk;
    pp.lengths = t->lengths;
    if (tp.domain_kind == kDomainMesh) {
        // The inside test of a seed walks three long rays through the BVH.
        // Inside the tracking kernel the lane that starts a streamline would
        // hold its whole warp for those walks; a pre-pass (in the timed
        // region) does them for every seed, with the same arithmetic.
        TG_TRY(ensure(&t->seed_inside, &t->cap_seed_inside, n_seeds));
        pp.seed_inside = t->seed_inside;
    }

    const int block = persistent_block_size();
    int per_sm = persistent_blocks_per_sm(field->d, algorithm->algorithm, domain->d.kind);
    if (t->blocks_per_sm > 0 && (int)t->blocks_per_sm < per_sm) per_sm = (int)t->blocks_per_sm;
    const int grid = sm_count() * per_sm;
    const uint32_t rounds = t->compact_lanes > 0 ? t->compact_rounds : 0u;
    if (rounds > 0) {
        st = tracker_carry(t, kClassKinds, (size_t)grid * block);
        if (st != TG_OK) return st;
    }
    // slicing only where a streamline can outlast a slice
    if (t->slice_steps > 0 && tp.max_steps > t->slice_steps) {
        // every streamline live in a launch is in a lane or once in the ring
        const size_t cap = (size_t)n_seeds + (size_t)grid * block + 1;
        if (cap > 0xFFFFFFFFull) return fail(TG_ERR_INVALID_ARGUMENT, "too many seeds for time slicing");
        TG_TRY(ensure(&t->ring_items, &t->cap_ring, cap));
        TG_TRY(ensure(&t->ring_flags, &t->cap_ring_flags, 2 * cap));
        TG_TRY(ensure(&t->ring_ctl, &t->cap_ring_ctl, 4));
        TG_TRY(cudaMemsetAsync(t->ring_ctl, 0, 4 * sizeof(unsigned int), s));
        pp.ring.items = t->ring_items;
        pp.ring.seq = t->ring_flags;
        pp.ring.released = t->ring_flags + cap;
        pp.ring.ctl = t->ring_ctl;
        pp.ring.capacity = (uint32_t)cap;
        pp.ring.lanes = (uint32_t)grid * (uint32_t)block;
        // the slice in saved points: the largest power of two whose points
        // take at most slice_steps steps (steps_per_point_bound each)
        const uint64_t per_point = std::max<uint64_t>(1, steps_per_point_bound(algorithm->step_size, save_at));
        const uint64_t points = std::max<uint64_t>(1, t->slice_steps / per_point);
        uint32_t slice_points = 1;
        while ((uint64_t)slice_points * 2 <= points && slice_points < (1u << 30)) slice_points *= 2;
        pp.slice_mask = slice_points - 1u;
    }
    unsigned int* ccount = t->carry_count + 2 * kClassKinds;

    t->h_len.resize(n_seeds);
    TG_TRY(cudaMemsetAsync(t->counters + 1, 0, sizeof(unsigned long long), s));
    uint64_t total = 0;
    bool first_wave = true;
    int stalls = 0;
    std::vector<uint32_t> wave_items;
    while (first_wave || !wave_items.empty()) {
        const uint32_t n_items = first_wave ? n_seeds : (uint32_t)wave_items.size();
        if (!first_wave)
            TG_TRY(cudaMemcpyAsync(t->ids, wave_items.data(), n_items * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        pp.item_ids = first_wave ? nullptr : t->ids;
        pp.n_items = n_items;
        pp.pool = t->pool;
        pp.chunk_next = t->chunk_next;
        pp.n_chunks = t->n_chunks;
        TG_TRY(cudaMemsetAsync(t->chunk_counter, 0, sizeof(unsigned int), s));
        TG_TRY(cudaEventRecord(t->ev_start, s));
        if (first_wave && pp.seed_inside != nullptr) {
            TG_TRY(launch_mesh_contains(tp.mesh, d_seeds, n_seeds, t->seed_inside, s, 2u));
            t->launches += 1;
        }
        // round 0 pulls seeds; rounds 1..R resume the streamlines handed over
        // by sparse warps of the previous round; the last round compacts no more
        for (uint32_t r = 0; r <= rounds; ++r) {
            TG_TRY(cudaMemsetAsync(t->counters, 0, sizeof(unsigned long long), s));
            pp.carry_in = r == 0 ? nullptr : t->carry[kClassKinds][(r - 1) & 1];
            pp.carry_in_count = r == 0 ? nullptr : ccount + ((r - 1) & 1);
            pp.carry_out = r < rounds ? t->carry[kClassKinds][r & 1] : nullptr;
            pp.carry_out_count = ccount + (r & 1);
            pp.compact_lanes = t->compact_lanes;
            if (r < rounds) TG_TRY(cudaMemsetAsync(ccount + (r & 1), 0, sizeof(unsigned int), s));
            if (pp.ring.items != nullptr) {
                // an empty ring for each launch; the fault word spans the run
                TG_TRY(cudaMemsetAsync(pp.ring.seq, 0, 2 * (size_t)pp.ring.capacity * sizeof(uint32_t), s));
                TG_TRY(cudaMemsetAsync(pp.ring.ctl, 0, 2 * sizeof(unsigned int), s));
            }
            TG_TRY(launch_track_persistent(field->d, pp, grid, block, s));
            t->launches += 1;
        }
        TG_TRY(cudaEventRecord(t->ev_stop, s));
        if (first_wave) {
            // Common case: every streamline fit the pool; offsets by a device
            // scan (tg_tracker_run_jobs does the same).
            size_t temp_bytes = 0;
            TG_TRY(launch_offsets(t->lengths, n_seeds, nullptr, nullptr, nullptr, nullptr, &temp_bytes, s));
            TG_TRY(ensure(&t->masked, &t->cap_masked, n_seeds));
            TG_TRY(ensure(&t->scan_temp, &t->cap_scan_temp, temp_bytes));
            TG_TRY(ensure(&t->d_totals, &t->cap_totals, 2));
            TG_TRY(launch_offsets(t->lengths, n_seeds, t->masked, t->offsets, t->d_totals, t->scan_temp, &temp_bytes,
                                  s));
            t->launches += 2;   // masked_lengths_kernel, offsets_total_kernel (the scan between is cub's)
            unsigned long long totals[2] = {0ull, 0ull};
            TG_TRY(cudaMemcpyAsync(totals, t->d_totals, sizeof totals, cudaMemcpyDeviceToHost, s));
            TG_TRY(cudaStreamSynchronize(s));
            if (totals[1] == 0ull) {
                float wave_ms = 0.0f;
                TG_TRY(cudaEventElapsedTime(&wave_ms, t->ev_start, t->ev_stop));
                t->kernel_ms += wave_ms;
                t->waves += 1;
                total = totals[0];
                st = tracker_points(t, total, s);
                if (st != TG_OK) return st;
                TG_TRY(launch_gather(t->pool, t->chunk_next, t->first_chunk, t->lengths, t->offsets, nullptr, n_seeds,
                                     t->points, s));
                t->launches += 1;
                t->total_points = total;
                TG_TRY(cudaMemcpyAsync(h_lengths, t->lengths, (size_t)n_seeds * sizeof(uint32_t),
                                       cudaMemcpyDeviceToHost, s));
                TG_TRY(cudaMemcpyAsync(h_offsets, t->offsets, (size_t)n_seeds * sizeof(uint64_t),
                                       cudaMemcpyDeviceToHost, s));
                break;
            }
        }
        TG_TRY(cudaMemcpyAsync(t->h_len.data(), t->lengths, (size_t)n_seeds * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, s));
        TG_TRY(cudaStreamSynchronize(s));
        float wave_ms = 0.0f;
        TG_TRY(cudaEventElapsedTime(&wave_ms, t->ev_start, t->ev_stop));
        t->kernel_ms += wave_ms;
        t->waves += 1;

        t->h_done.clear();
        t->h_retry.clear();
        for (uint32_t k = 0; k < n_items; ++k) {
            const uint32_t i = first_wave ? k : wave_items[k];
            const uint32_t L = t->h_len[i];
            if (L & kOverflowBit) {
                t->h_retry.push_back(i);
            } else {
                t->h_done.push_back(i);
                h_offsets[i] = total;
                h_lengths[i] = L;
                total += L;
            }
        }
        if (t->h_done.empty()) {
            // No streamline fit: grow the pool and repeat the wave.
            if (++stalls > 4) return fail(TG_ERR_POOL_EXHAUSTED, "point pool too small for one streamline");
            st = tracker_pool(t, (uint64_t)t->n_chunks * kChunkPoints * 4);
            if (st != TG_OK) return st;
            wave_items.assign(t->h_retry.begin(), t->h_retry.end());
            first_wave = false;
            continue;
        }
        st = tracker_points(t, total, s);
        if (st != TG_OK) return st;
        TG_TRY(cudaMemcpyAsync(t->offsets, h_offsets, (size_t)n_seeds * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        TG_TRY(cudaMemcpyAsync(t->done_ids, t->h_done.data(), t->h_done.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, s));
        TG_TRY(launch_gather(t->pool, t->chunk_next, t->first_chunk, t->lengths, t->offsets, t->done_ids,
                             (uint32_t)t->h_done.size(), t->points, s));
        t->launches += 1;
        t->total_points = total;
        wave_items.assign(t->h_retry.begin(), t->h_retry.end());
        first_wave = false;
    }
    unsigned long long steps = 0;
    unsigned int ring_fault = 0;
    TG_TRY(cudaMemcpyAsync(&steps, t->counters + 1, sizeof steps, cudaMemcpyDeviceToHost, s));
    if (pp.ring.items != nullptr)
        TG_TRY(cudaMemcpyAsync(&ring_fault, pp.ring.ctl + 2, sizeof ring_fault, cudaMemcpyDeviceToHost, s));
    TG_TRY(cudaStreamSynchronize(s));
    if (ring_fault != 0u)
        return fail(TG_ERR_CUDA, std::string("time slicing: a bounded wait on the queue of saved streamlines ran "
                                             "out (") + ((ring_fault & 1u) ? "slot" : "") +
                                     ((ring_fault & 2u) ? " claim" : "") + ")");
    t->total_points = total;
    if (total_points) *total_points = total;
    if (total_steps) *total_steps = steps;
    return TG_OK;
}

int tg_tracker_run_jobs(tg_tracker* t, const tg_job* jobs, uint32_t n_jobs, int seeds_on_host, uint32_t* h_lengths,
                        uint64_t* h_offsets, uint64_t* total_points, uint64_t* total_steps, void* stream)
{
    if (t == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "tracker is null");
    t->total_points = 0;
    t->kernel_ms = 0.0f;
    t->waves = 0;
    t->launches = 0;
    if (total_points) *total_points = 0;
    if (total_steps) *total_steps = 0;
    if (n_jobs == 0) return TG_OK;
    if (jobs == nullptr || h_lengths == nullptr || h_offsets == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null buffer");
    cudaStream_t s = as_stream(stream);

    // Validate the jobs and lay them out in one global seed index space.
    std::vector<JobDev> table(n_jobs);
    std::vector<uint32_t> job_base(n_jobs + 1, 0);
    std::vector<uint32_t> rng_base(n_jobs, 0);
    std::vector<int> kind(n_jobs, 0);
    uint64_t n_total = 0, n_batches_total = 0, worst = 0;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const tg_job& J = jobs[j];
        TrackParams tp;
        int st = make_track_params(&J.algorithm, J.domain, J.field, J.save_at, J.n_steps, &tp);
        if (st != TG_OK) return fail(st, "job " + std::to_string(j) + ": " + g_error);
        if (tp.domain_kind != kDomainImage)
            return fail(TG_ERR_UNSUPPORTED, "job " + std::to_string(j) + ": mesh domains run through tg_tracker_run");
        if (J.n_steps == 0) return fail(TG_ERR_INVALID_ARGUMENT, "job " + std::to_string(j) + ": n_steps must be positive");
        if (J.n_seeds > 0 && (J.seeds == nullptr || J.batch_rng_seeds == nullptr || J.batch_size == 0))
            return fail(TG_ERR_INVALID_ARGUMENT, "job " + std::to_string(j) + ": missing seeds or batch seeds");
        std::memset(&table[j], 0, sizeof(JobDev));
        table[j].t = tp;
        table[j].n_seeds = J.n_seeds;
        table[j].batch_size = J.batch_size > 0 ? J.batch_size : 1;
        table[j].seed_offset = J.algorithm.seed_offset;
        kind[j] = class_kind(J.field->d.model, J.field->d.lmax, J.algorithm.algorithm);
        job_base[j] = (uint32_t)n_total;
        rng_base[j] = (uint32_t)n_batches_total;
        n_total += J.n_seeds;
        n_batches_total += (J.n_seeds + table[j].batch_size - 1) / table[j].batch_size;
        worst += (uint64_t)J.n_seeds * (((uint64_t)J.n_steps + kChunkPoints - 1) / kChunkPoints * kChunkPoints);
        if (n_total >= 0x80000000ull) return fail(TG_ERR_INVALID_ARGUMENT, "too many seeds in one run");
    }
    job_base[n_jobs] = (uint32_t)n_total;
    if (n_total == 0) return TG_OK;

    // Device copies: seeds (when given on the host), batch seeds, tables.
    TG_TRY(ensure(&t->batch_seeds, &t->cap_batches, n_batches_total));
    TG_TRY(ensure(&t->seeds, &t->cap_seed_copy, seeds_on_host ? (size_t)n_total * 2 : 1));
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const tg_job& J = jobs[j];
        if (J.n_seeds == 0) continue;
        const uint64_t nb = (J.n_seeds + table[j].batch_size - 1) / table[j].batch_size;
        TG_TRY(cudaMemcpyAsync(t->batch_seeds + rng_base[j], J.batch_rng_seeds, nb * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, s));
        if (seeds_on_host) {
            TG_TRY(cudaMemcpyAsync(t->seeds + 2 * (size_t)job_base[j], J.seeds, (size_t)J.n_seeds * 8 * sizeof(float),
                                   cudaMemcpyHostToDevice, s));
            table[j].seeds = t->seeds + 2 * (size_t)job_base[j];
        } else {
            table[j].seeds = reinterpret_cast<const float4*>(J.seeds);
        }
        table[j].rng_base = rng_base[j];
    }
    TG_TRY(ensure(&t->d_jobs, &t->cap_jobs, n_jobs));
    TG_TRY(ensure(&t->d_job_base, &t->cap_job_base, n_jobs + 1));
    TG_TRY(cudaMemcpyAsync(t->d_jobs, table.data(), n_jobs * sizeof(JobDev), cudaMemcpyHostToDevice, s));
    TG_TRY(cudaMemcpyAsync(t->d_job_base, job_base.data(), (n_jobs + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s));

    // Classes: jobs grouped by code path, longest point budget first.
    std::vector<std::vector<uint32_t>> members(kClassKinds);
    for (uint32_t j = 0; j < n_jobs; ++j)
        if (jobs[j].n_seeds > 0) members[kind[j]].push_back(j);
    std::vector<uint32_t> lists;            // per class: jobs then prefix (n + 1)
    std::vector<size_t> list_at(kClassKinds, 0);
    for (int k = 0; k < kClassKinds; ++k) {
        auto& m = members[k];
        std::stable_sort(m.begin(), m.end(), [&](uint32_t a, uint32_t b) { return jobs[a].n_steps > jobs[b].n_steps; });
        list_at[k] = lists.size();
        lists.insert(lists.end(), m.begin(), m.end());
        uint32_t acc = 0;
        lists.push_back(0);
        for (uint32_t j : m) {
            acc += jobs[j].n_seeds;
            lists.push_back(acc);
        }
    }
    TG_TRY(ensure(&t->d_class_lists, &t->cap_class_lists, lists.size()));
    TG_TRY(cudaMemcpyAsync(t->d_class_lists, lists.data(), lists.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    if (t->d_class_counters == nullptr)
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->d_class_counters), kClassKinds * sizeof(unsigned long long)));
    if (t->ev_fork == nullptr) TG_TRY(cudaEventCreateWithFlags(&t->ev_fork, cudaEventDisableTiming));
    for (int k = 0; k < kClassKinds; ++k) {
        if (members[k].empty() || t->class_stream[k] != nullptr) continue;
        TG_TRY(cudaStreamCreateWithFlags(&t->class_stream[k], cudaStreamNonBlocking));
        TG_TRY(cudaEventCreateWithFlags(&t->class_done[k], cudaEventDisableTiming));
    }

    // Per-seed buffers and the point pool.
    if (t->cap_seeds < n_total) {
        cudaFree(t->first_chunk);
        cudaFree(t->lengths);
        cudaFree(t->offsets);
        cudaFree(t->ids);
        cudaFree(t->done_ids);
        t->first_chunk = nullptr;
        t->lengths = nullptr;
        t->offsets = nullptr;
        t->ids = nullptr;
        t->done_ids = nullptr;
        t->cap_seeds = 0;
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->first_chunk), n_total * sizeof(int32_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->lengths), n_total * sizeof(uint32_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->offsets), n_total * sizeof(uint64_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->ids), n_total * sizeof(uint32_t)));
        TG_TRY(cudaMalloc(reinterpret_cast<void**>(&t->done_ids), n_total * sizeof(uint32_t)));
        t->cap_seeds = n_total;
    }
    uint64_t want = t->pool_points_request;
    if (want == 0) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const uint64_t budget = (uint64_t)(free_b / 3) / (3 * sizeof(float) + 1);
        want = std::min<uint64_t>(worst, std::max<uint64_t>(budget, (uint64_t)1 << 20));
    }
    int st = tracker_pool(t, want);
    if (st != TG_OK) return st;

    MultiParams mp;
    std::memset(&mp, 0, sizeof mp);
    mp.jobs = t->d_jobs;
    mp.job_base = t->d_job_base;
    mp.n_jobs = n_jobs;
    mp.batch_rng_seeds = t->batch_seeds;
    mp.chunk_counter = t->chunk_counter;
    mp.first_chunk = t->first_chunk;
    mp.lengths = t->lengths;
    mp.steps_done = t->counters + 1;
    const int sms = sm_count();

    t->h_len.resize(n_total);
    TG_TRY(cudaMemsetAsync(t->counters + 1, 0, sizeof(unsigned long long), s));
    uint64_t total = 0;
    bool first_wave = true;
    int stalls = 0;
    std::vector<std::vector<uint32_t>> retry(kClassKinds);
    std::vector<uint32_t> wave_ids;
    while (true) {
        // per class: its item source for this wave
        std::vector<size_t> retry_at(kClassKinds, 0);
        uint64_t wave_items = 0;
        wave_ids.clear();
        for (int k = 0; k < kClassKinds; ++k) {
            retry_at[k] = wave_ids.size();
            if (!first_wave) wave_ids.insert(wave_ids.end(), retry[k].begin(), retry[k].end());
        }
        if (!first_wave) {
            if (wave_ids.empty()) break;
            TG_TRY(cudaMemcpyAsync(t->ids, wave_ids.data(), wave_ids.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        }
        mp.pool = t->pool;
        mp.chunk_next = t->chunk_next;
        mp.n_chunks = t->n_chunks;
        TG_TRY(cudaMemsetAsync(t->d_class_counters, 0, kClassKinds * sizeof(unsigned long long), s));
        TG_TRY(cudaMemsetAsync(t->chunk_counter, 0, sizeof(unsigned int), s));
        TG_TRY(cudaEventRecord(t->ev_start, s));
        TG_TRY(cudaEventRecord(t->ev_fork, s));
        std::vector<int> launched;
        // classes with the most point budget first
        std::vector<int> order;
        for (int k = 0; k < kClassKinds; ++k) order.push_back(k);
        std::vector<uint64_t> budget(kClassKinds, 0);
        for (int k = 0; k < kClassKinds; ++k)
            for (uint32_t j : members[k]) budget[k] += (uint64_t)jobs[j].n_seeds * jobs[j].n_steps;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return budget[a] > budget[b]; });
        // launch shapes and carry buffers first: no allocation while kernels run
        const uint32_t rounds = t->compact_lanes > 0 ? t->compact_rounds : 0u;
        std::vector<int> kgrid(kClassKinds, 0);
        for (int k : order) {
            if (members[k].empty()) continue;
            int per_sm = class_blocks_per_sm(k);
            if (t->blocks_per_sm > 0 && (int)t->blocks_per_sm < per_sm) per_sm = (int)t->blocks_per_sm;
            kgrid[k] = sms * per_sm;
            if (rounds > 0) {
                st = tracker_carry(t, k, (size_t)kgrid[k] * 128);
                if (st != TG_OK) return st;
            }
        }
        for (int k : order) {
            ClassDev cls;
            std::memset(&cls, 0, sizeof cls);
            cls.kind = k;
            cls.n_jobs = (uint32_t)members[k].size();
            cls.jobs = t->d_class_lists + list_at[k];
            cls.prefix = t->d_class_lists + list_at[k] + members[k].size();
            cls.counter = t->d_class_counters + k;
            if (first_wave) {
                cls.n_items = members[k].empty() ? 0 : lists[list_at[k] + 2 * members[k].size()];
            } else {
                cls.item_ids = t->ids + retry_at[k];
                cls.n_items = (uint32_t)retry[k].size();
            }
            if (cls.n_items == 0) continue;
            wave_items += cls.n_items;
            cudaStream_t ks = t->class_stream[k];
            TG_TRY(cudaStreamWaitEvent(ks, t->ev_fork, 0));
            unsigned int* ccount = t->carry_count + 2 * k;
            for (uint32_t r = 0; r <= rounds; ++r) {
                MultiParams mk = mp;
                mk.carry_in = r == 0 ? nullptr : t->carry[k][(r - 1) & 1];
                mk.carry_in_count = r == 0 ? nullptr : ccount + ((r - 1) & 1);
                mk.carry_out = r < rounds ? t->carry[k][r & 1] : nullptr;
                mk.carry_out_count = ccount + (r & 1);
                mk.compact_lanes = t->compact_lanes;
                if (r > 0) TG_TRY(cudaMemsetAsync(cls.counter, 0, sizeof(unsigned long long), ks));
                if (r < rounds) TG_TRY(cudaMemsetAsync(ccount + (r & 1), 0, sizeof(unsigned int), ks));
                TG_TRY(launch_track_class(mk, cls, kgrid[k], ks));
                t->launches += 1;
            }
            TG_TRY(cudaEventRecord(t->class_done[k], ks));
            TG_TRY(cudaStreamWaitEvent(s, t->class_done[k], 0));
            launched.push_back(k);
        }
        TG_TRY(cudaEventRecord(t->ev_stop, s));
        if (first_wave) {
            // Common case: every streamline fit the pool.  Offsets come from a
            // device scan of the lengths (streamlines packed in seed order) and
            // the host reads two totals instead of visiting every seed.
            size_t temp_bytes = 0;
            TG_TRY(launch_offsets(t->lengths, (uint32_t)n_total, nullptr, nullptr, nullptr, nullptr, &temp_bytes, s));
            TG_TRY(ensure(&t->masked, &t->cap_masked, n_total));
            TG_TRY(ensure(&t->scan_temp, &t->cap_scan_temp, temp_bytes));
            TG_TRY(ensure(&t->d_totals, &t->cap_totals, 2));
            TG_TRY(launch_offsets(t->lengths, (uint32_t)n_total, t->masked, t->offsets, t->d_totals, t->scan_temp,
                                  &temp_bytes, s));
            t->launches += 2;   // masked_lengths_kernel, offsets_total_kernel
            unsigned long long totals[2] = {0ull, 0ull};
            TG_TRY(cudaMemcpyAsync(totals, t->d_totals, sizeof totals, cudaMemcpyDeviceToHost, s));
            TG_TRY(cudaStreamSynchronize(s));
            if (totals[1] == 0ull) {
                float wave_ms = 0.0f;
                TG_TRY(cudaEventElapsedTime(&wave_ms, t->ev_start, t->ev_stop));
                t->kernel_ms += wave_ms;
                t->waves += 1;
                total = totals[0];
                st = tracker_points(t, total, s);
                if (st != TG_OK) return st;
                TG_TRY(launch_gather(t->pool, t->chunk_next, t->first_chunk, t->lengths, t->offsets, nullptr,
                                     (uint32_t)n_total, t->points, s));
                t->launches += 1;
                t->total_points = total;
                TG_TRY(cudaMemcpyAsync(h_lengths, t->lengths, n_total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                TG_TRY(cudaMemcpyAsync(h_offsets, t->offsets, n_total * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
                break;
            }
        }
        TG_TRY(cudaMemcpyAsync(t->h_len.data(), t->lengths, n_total * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        TG_TRY(cudaStreamSynchronize(s));
        float wave_ms = 0.0f;
        TG_TRY(cudaEventElapsedTime(&wave_ms, t->ev_start, t->ev_stop));
        t->kernel_ms += wave_ms;
        t->waves += 1;

        // collect finished streamlines, queue the others for the next wave
        t->h_done.clear();
        std::vector<std::vector<uint32_t>> next(kClassKinds);
        auto visit = [&](uint32_t g, int k) {
            const uint32_t L = t->h_len[g];
            if (L & kOverflowBit) {
                next[k].push_back(g);
            } else {
                t->h_done.push_back(g);
                h_offsets[g] = total;
                h_lengths[g] = L;
                total += L;
            }
        };
        for (int k : launched) {
            if (first_wave) {
                for (uint32_t j : members[k])
                    for (uint32_t i = 0; i < jobs[j].n_seeds; ++i) visit(job_base[j] + i, k);
            } else {
                for (uint32_t g : retry[k]) visit(g, k);
            }
        }
        (void)wave_items;
        if (t->h_done.empty()) {
            if (++stalls > 4) return fail(TG_ERR_POOL_EXHAUSTED, "point pool too small for one streamline");
            st = tracker_pool(t, (uint64_t)t->n_chunks * kChunkPoints * 4);
            if (st != TG_OK) return st;
        } else {
            st = tracker_points(t, total, s);
            if (st != TG_OK) return st;
            TG_TRY(cudaMemcpyAsync(t->offsets, h_offsets, n_total * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
            TG_TRY(cudaMemcpyAsync(t->done_ids, t->h_done.data(), t->h_done.size() * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, s));
            TG_TRY(launch_gather(t->pool, t->chunk_next, t->first_chunk, t->lengths, t->offsets, t->done_ids,
                                 (uint32_t)t->h_done.size(), t->points, s));
            t->launches += 1;
            t->total_points = total;
        }
        retry.swap(next);
        first_wave = false;
    }
    unsigned long long steps = 0;
    TG_TRY(cudaMemcpyAsync(&steps, t->counters + 1, sizeof steps, cudaMemcpyDeviceToHost, s));
    TG_TRY(cudaStreamSynchronize(s));
    t->total_points = total;
    if (total_points) *total_points = total;
    if (total_steps) *total_steps = steps;
    return TG_OK;
}

int tg_tracker_copy_points(tg_tracker* t, float* dst, uint64_t first, uint64_t count, int dst_on_host, void* stream)
{
    if (t == nullptr || (dst == nullptr && count > 0)) return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (first + count > t->total_points) return fail(TG_ERR_INVALID_ARGUMENT, "point range out of bounds");
    if (count == 0) return TG_OK;
    cudaStream_t s = as_stream(stream);
    TG_TRY(cudaMemcpyAsync(dst, t->points + first * 3, (size_t)count * 3 * sizeof(float),
                           dst_on_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    if (dst_on_host) TG_TRY(cudaStreamSynchronize(s));
    return TG_OK;
}

int tg_seeds_from_fod(int32_t model, uint32_t n_coefficients, const float* fod, const float* voxels, uint32_t nnz,
                      const float* affine, const uint32_t* states, uint32_t n_seeds, float* seeds, void* stream)
{
    if (n_seeds == 0) return TG_OK;
    if (fod == nullptr || voxels == nullptr || affine == nullptr || states == nullptr || seeds == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null buffer");
    if (nnz == 0) return fail(TG_ERR_INVALID_ARGUMENT, "the FOD has no nonzero voxel");
    if (model == TG_MODEL_SH && (n_coefficients == 0 || n_coefficients > 45))
        return fail(TG_ERR_UNSUPPORTED, "spherical-harmonic FODs support 1..45 coefficients");
    if (model == TG_MODEL_DTI && n_coefficients != 6) return fail(TG_ERR_INVALID_ARGUMENT, "tensors have 6 coefficients");
    TG_TRY(launch_seeds_from_fod(model, n_coefficients, fod, reinterpret_cast<const float4*>(voxels), nnz, affine,
                                 reinterpret_cast<const uint2*>(states), n_seeds, reinterpret_cast<float4*>(seeds),
                                 as_stream(stream)));
    return TG_OK;
}

int tg_domain_contains(const tg_domain* domain, const float* points, uint32_t n, uint8_t* out, void* stream)
{
    if (domain == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "domain is null");
    if (n == 0) return TG_OK;
    if (domain->d.kind == kDomainMesh) {
        TG_TRY(launch_mesh_contains(domain->d.mesh, reinterpret_cast<const float4*>(points), n, out,
                                    as_stream(stream)));
        return TG_OK;
    }
    TG_TRY(launch_contains(domain->d, reinterpret_cast<const float4*>(points), n, out, as_stream(stream)));
    return TG_OK;
}

int tg_boundary_seeds(const float* vertices, uint32_t n_vertices, const uint32_t* triangles,
                      const float* cumulative_areas, uint32_t n_triangles, uint32_t rng_seed, uint32_t n_seeds,
                      float* seeds, void* stream)
{
    if (n_seeds == 0) return TG_OK;
    if (vertices == nullptr || triangles == nullptr || cumulative_areas == nullptr || seeds == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (n_triangles == 0 || n_vertices == 0)
        return fail(TG_ERR_INVALID_ARGUMENT, "The boundary mesh must contain at least one triangle.");
    TG_TRY(launch_boundary_seeds(reinterpret_cast<const float4*>(vertices), reinterpret_cast<const uint4*>(triangles),
                                 cumulative_areas, n_triangles, rng_seed, n_seeds, reinterpret_cast<float4*>(seeds),
                                 as_stream(stream)));
    return TG_OK;
}

int tg_tod(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field, const float* vertices,
           uint32_t n_vertices, const uint32_t* triangles, const float* cumulative_areas, uint32_t n_triangles,
           uint32_t n_seeds, uint32_t n_steps, const uint32_t out_dims[3], const float out_inverse_affine[16],
           float* coefficients, uint64_t* steps, void* stream)
{
    TodParams q;
    std::memset(&q, 0, sizeof q);
    int st = make_track_params(algorithm, domain, field, 1.0f, 1u, &q.t, false);
    if (st != TG_OK) return st;
    if (n_seeds == 0 || n_steps == 0) return TG_OK;
    if (vertices == nullptr || triangles == nullptr || cumulative_areas == nullptr || coefficients == nullptr ||
        out_dims == nullptr || out_inverse_affine == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (n_triangles == 0 || n_vertices == 0)
        return fail(TG_ERR_INVALID_ARGUMENT, "The boundary mesh must contain at least one triangle.");
    q.vertices = reinterpret_cast<const float4*>(vertices);
    q.triangles = reinterpret_cast<const uint4*>(triangles);
    q.cumulative = cumulative_areas;
    q.n_triangles = n_triangles;
    q.rng_seed = algorithm->rng_seed;
    q.seed_offset = algorithm->seed_offset;
    q.n_seeds = n_seeds;
    q.n_steps = n_steps;
    const Grid g = grid_of(out_inverse_affine, out_dims[0], out_dims[1], out_dims[2]);
    q.out_row0 = g.row0;
    q.out_row1 = g.row1;
    q.out_row2 = g.row2;
    q.nx = out_dims[0];
    q.ny = out_dims[1];
    q.nz = out_dims[2];
    q.coefficients = coefficients;
    q.steps = reinterpret_cast<unsigned long long*>(steps);
    // the lanes' seed counter: stream-ordered, freed after the launch
    cudaStream_t s = as_stream(stream);
    TG_TRY(cudaMallocAsync(reinterpret_cast<void**>(&q.counter), sizeof(unsigned long long), s));
    cudaError_t e = cudaMemsetAsync(q.counter, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = launch_tod(field->d.model, field->d.lmax, q, s);
    cudaFreeAsync(q.counter, s);
    TG_TRY(e);
    return TG_OK;
}

int tg_connectome(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                  const tg_domain* boundary, const float* vertices, uint32_t n_vertices, const uint32_t* triangles,
                  const float* cumulative_areas, uint32_t n_triangles, uint32_t n_seeds, uint32_t n_steps,
                  float minimum_length, int32_t* rows, int32_t* columns, float* weights, uint64_t* steps,
                  void* stream)
{
    ConnectomeParams q;
    std::memset(&q, 0, sizeof q);
    int st = make_track_params(algorithm, domain, field, 1.0f, 1u, &q.t, false);
    if (st != TG_OK) return st;
    if (n_seeds == 0) return TG_OK;
    if (boundary == nullptr || boundary->d.kind != kDomainMesh)
        return fail(TG_ERR_INVALID_ARGUMENT, "boundary must be a mesh domain of the boundary surface");
    if (vertices == nullptr || triangles == nullptr || cumulative_areas == nullptr || rows == nullptr ||
        columns == nullptr || weights == nullptr)
        return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (n_triangles == 0 || n_vertices == 0)
        return fail(TG_ERR_INVALID_ARGUMENT, "The boundary mesh must contain at least one triangle.");
    if (boundary->d.n_triangles != n_triangles)
        return fail(TG_ERR_INVALID_ARGUMENT, "boundary BVH and sampler arrays describe different triangles");
    q.vertices = reinterpret_cast<const float4*>(vertices);
    q.triangles = reinterpret_cast<const uint4*>(triangles);
    q.cumulative = cumulative_areas;
    q.n_triangles = n_triangles;
    q.bvh = boundary->d.mesh;
    q.rng_seed = algorithm->rng_seed;
    q.seed_offset = algorithm->seed_offset;
    q.n_seeds = n_seeds;
    q.n_steps = n_steps;
    q.minimum_length = minimum_length;
    q.rows = rows;
    q.columns = columns;
    q.weights = weights;
    q.steps = reinterpret_cast<unsigned long long*>(steps);
    cudaStream_t s = as_stream(stream);
    TG_TRY(cudaMallocAsync(reinterpret_cast<void**>(&q.counter), sizeof(unsigned long long), s));
    cudaError_t e = cudaMemsetAsync(q.counter, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = launch_connectome(field->d.model, field->d.lmax, q, s);
    cudaFreeAsync(q.counter, s);
    TG_TRY(e);
    return TG_OK;
}

int tg_field_evaluate(const tg_field* field, const float* points, uint32_t n, float* out, void* stream)
{
    if (field == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "field is null");
    if (n == 0) return TG_OK;
    TG_TRY(launch_field_evaluate(field->d, reinterpret_cast<const float4*>(points), n, out, as_stream(stream)));
    return TG_OK;
}

int tg_local_evaluate(int32_t model, uint32_t n_parameters, const float* parameters, const float* orientations,
                      uint32_t n, float* out, void* stream)
{
    if (model == TG_MODEL_SH && (n_parameters == 0 || n_parameters > 45))
        return fail(TG_ERR_UNSUPPORTED, "spherical-harmonic models support 1..45 coefficients");
    if (model == TG_MODEL_DTI && n_parameters != 6) return fail(TG_ERR_INVALID_ARGUMENT, "tensors have 6 coefficients");
    if (model != TG_MODEL_SH && model != TG_MODEL_DTI) return fail(TG_ERR_UNSUPPORTED, "unknown model");
    if (n == 0) return TG_OK;
    TG_TRY(launch_local_evaluate(model, n_parameters, parameters, reinterpret_cast<const float4*>(orientations), n,
                                 out, as_stream(stream)));
    return TG_OK;
}

int tg_update_orientation(int32_t model, uint32_t n_parameters, const tg_algorithm* algorithm,
                          const float* parameters, const float* orientations, uint32_t n, float* out, void* stream)
{
    int st = check_algorithm(algorithm);
    if (st != TG_OK) return st;
    if (model == TG_MODEL_SH && (n_parameters == 0 || n_parameters > 45))
        return fail(TG_ERR_UNSUPPORTED, "spherical-harmonic models support 1..45 coefficients");
    if (model == TG_MODEL_DTI && n_parameters != 6) return fail(TG_ERR_INVALID_ARGUMENT, "tensors have 6 coefficients");
    if (model != TG_MODEL_SH && model != TG_MODEL_DTI) return fail(TG_ERR_UNSUPPORTED, "unknown model");
    if (n == 0) return TG_OK;
    TG_TRY(launch_update_orientation(model, n_parameters, algorithm->algorithm, algo_params(algorithm),
                                     algorithm->rng_seed, algorithm->seed_offset, parameters,
                                     reinterpret_cast<const float4*>(orientations), n,
                                     reinterpret_cast<float4*>(out), as_stream(stream)));
    return TG_OK;
}

int tg_step_bound(float step_size, float save_at, uint32_t n_steps, uint64_t* max_steps)
{
    if (max_steps == nullptr) return fail(TG_ERR_INVALID_ARGUMENT, "null argument");
    if (!std::isfinite(step_size) || step_size <= 0.0f)
        return fail(TG_ERR_INVALID_ARGUMENT, "step_size must be finite and positive");
    if (!std::isfinite(save_at) || save_at <= 0.0f)
        return fail(TG_ERR_INVALID_ARGUMENT, "save_at must be finite and positive");
    return step_bound(step_size, save_at, n_steps, max_steps);
}

int tg_rng_stream(int32_t which, uint32_t s0, uint32_t s1, uint32_t n, uint32_t max, void* out, void* stream)
{
    if (which < 0 || which > 2) return fail(TG_ERR_INVALID_ARGUMENT, "which must be 0, 1 or 2");
    if (n == 0) return TG_OK;
    TG_TRY(launch_rng_streams(which, s0, s1, n, max, out, as_stream(stream)));
    return TG_OK;
}

}  // extern "C"
