/*
 * tractography_b200.h -- C ABI of the B200 streamline-tracking library
 * (libtg_b200.so).
 *
 * The reference (cronos-inria/tractography) assembles OpenCL C from its
 * plugin objects and launches one `tractogram` kernel per batch through
 * PyOpenCL (tractography/tracking.py:22-178, tractography/opencl.py).  This
 * library replaces that backend: the same kernel contract as compiled
 * sm_100a code, with device-resident fields and domains, a persistent
 * batched tracker and the standalone per-element kernels the reference
 * exposes.  Plain C types only: pointers, sizes and POD structs.
 *
 * Conventions
 *   - Every function returns a tg status code (TG_OK == 0).  On failure
 *     tg_last_error() returns a message for the calling thread.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *   - Arrays are C-contiguous float32/uint32 in the layouts the reference
 *     uses: seeds (n, 8) = (x, y, z, 1, dx, dy, dz, 0); points float4.
 *   - Objects (tg_field, tg_domain, tg_tracker) are owned by the library
 *     and released by their *_destroy function; per-call inputs and outputs
 *     are owned by the caller.
 *   - Threading: calls on different objects may run concurrently; calls on
 *     one tg_tracker must be serialised by the caller.
 */
#ifndef TRACTOGRAPHY_B200_H
#define TRACTOGRAPHY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TG_ABI_VERSION 1

/* Status codes. */
#define TG_OK 0
#define TG_ERR_INVALID_ARGUMENT 1
#define TG_ERR_CUDA 2
#define TG_ERR_OUT_OF_MEMORY 3
#define TG_ERR_UNSUPPORTED 4
#define TG_ERR_POOL_EXHAUSTED 5

/* Local models (tractography/local.py:74-262). */
#define TG_MODEL_SH 0   /* RealSymmetricSphericalHarmonics, C <= 45 coefficients */
#define TG_MODEL_DTI 1  /* DiffusionTensorImaging, 6 coefficients */

/* Algorithms (tractography/algorithm.py:56-269). */
#define TG_ALGO_TRANSPORT 0
#define TG_ALGO_DIFFUSION 1

/* Random streams. */
#define TG_RNG_MWC64X 0  /* reference stream: rng_init(rng_seed, index in call), core.cl:180-245 */
#define TG_RNG_PHILOX 1  /* counter-based Philox4x32-10 keyed by (philox_key, seed index, step) */

typedef struct tg_field tg_field;
typedef struct tg_domain tg_domain;
typedef struct tg_tracker tg_tracker;

/* Orientation-update parameters: the ALGORITHM_ARGS of algorithm.py:75,189
 * plus the per-call rng_seed of tracking.py:164. */
typedef struct {
    int32_t algorithm;     /* TG_ALGO_* */
    float step_size;       /* algorithm.step_size */
    float gamma;           /* algorithm.gamma */
    float noise_variance;  /* Diffusion only (algorithm.py:176) */
    int32_t rng_mode;      /* TG_RNG_* */
    uint32_t rng_seed;     /* MWC64X: seed of this call (Diffusion.get_rng_seed, algorithm.py:239-241) */
    uint64_t philox_key;   /* Philox: stream key */
    uint64_t seed_offset;  /* Philox: global index of seed 0 of this call */
} tg_algorithm;

/* Library information. */
int tg_abi_version(void);
const char* tg_status_string(int status);
const char* tg_last_error(void);

/* Device-resident image field.  Replaces field.Image.__init__ + get_args
 * (tractography/field.py:54-69, 117-122), which re-uploaded the whole volume
 * on every batch.  `values` is a host (nx, ny, nz, n_parameters) float32
 * C-order array; `inverse_affine` is the row-major 4x4 world-to-voxel
 * matrix in float32.  model = TG_MODEL_SH (any C <= 45) or TG_MODEL_DTI
 * (C == 6). */
int tg_field_create(int32_t model, const float* values, uint32_t nx, uint32_t ny, uint32_t nz,
                    uint32_t n_parameters, const float inverse_affine[16], void* stream,
                    tg_field** out);
int tg_field_destroy(tg_field* field);

/* Device-resident image domain.  Replaces domain.Image.__init__ + get_args
 * (tractography/domain.py:275-311, 385-398).  `mask` is a host
 * (nx, ny, nz) uint8 C-order array, nonzero = inside. */
int tg_domain_create(const uint8_t* mask, uint32_t nx, uint32_t ny, uint32_t nz,
                     const float inverse_affine[16], void* stream, tg_domain** out);
int tg_domain_destroy(tg_domain* domain);

/* Closed triangle surface as a tracking domain.  The reference builds a
 * boundary mesh and its BVH for every domain (BaseDomain._set_boundary_data,
 * domain.py:44-116) and traverses it with bvh_segment_hit (utils/bvh.cl:
 * 83-131); this entry point makes such a surface the domain itself: a seed
 * is inside by a three-ray crossing-parity vote and a streamline stops at
 * the first step whose segment from the previous point hits the surface.
 * `vertices` (n_vertices, 3) float64 and `faces` (n_faces, 3) are host
 * arrays; faces wound outward.  The BVH is built on the host (median split
 * of domain.py:72-116) and stays resident with a distance grid that lets
 * steps far from the surface skip the traversal without changing a result.
 * Mesh domains are accepted by tg_tractogram, tg_tractogram_host,
 * tg_tracker_run and tg_domain_contains (not by tg_tracker_run_jobs or
 * tg_tractogram_noalloc, which return TG_ERR_UNSUPPORTED). */
int tg_domain_create_mesh(const double* vertices, uint32_t n_vertices, const uint32_t* faces,
                          uint32_t n_faces, void* stream, tg_domain** out);

/* The boundary BVH of domain.py:72-116 built on the host only, in the
 * reference's array layout (no device needed).  Call with null arrays to
 * get n_triangles (non-degenerate faces kept) and n_nodes; then with
 * arrays of (n_vertices, 4) float, (n_triangles, 4) uint32, (n_nodes, 4)
 * float bounds_min / bounds_max, (n_nodes, 4) int32 nodes and
 * (n_triangles,) ordered triangle ids. */
int tg_bvh_build_host(const double* vertices, uint32_t n_vertices, const uint32_t* faces,
                      uint32_t n_faces, uint32_t* n_triangles, uint32_t* n_nodes, float* vertices4,
                      uint32_t* triangles4, float* bounds_min, float* bounds_max, int32_t* nodes,
                      uint32_t* ordered_triangles);

/* Size of a mesh domain: triangles, BVH nodes, distance-grid cells per axis
 * and device bytes held. */
int tg_mesh_info(const tg_domain* domain, uint32_t* n_triangles, uint32_t* n_nodes, uint32_t grid[3],
                 uint64_t* device_bytes);

/* bvh_segment_hit (utils/bvh.cl:83-131) per segment: device arrays
 * starts/ends (n, 4) float32; writes found (n) uint8, triangle (n) uint32
 * (index among the kept faces) and hit (n, 4) = barycentric (1-u-v, u, v)
 * and the segment parameter t. */
int tg_mesh_segment_hits(const tg_domain* domain, const float* starts, const float* ends, uint32_t n,
                         uint8_t* found, uint32_t* triangle, float* hit, void* stream);

/* The closed-surface domain test of tracking, per segment: blocked[i] = 1
 * when the segment starts[i] -> ends[i] hits the surface (the found flag of
 * bvh_segment_hit, utils/bvh.cl:83-131), computed as the tracking kernels
 * compute it (distance grid, per-cell leaf lists, walk).  Device arrays:
 * starts/ends (n, 4) float32, blocked (n) uint8. */
int tg_mesh_segments_blocked(const tg_domain* domain, const float* starts, const float* ends, uint32_t n,
                             uint8_t* blocked, void* stream);

/* The reference kernel contract (tracking.py:93-176): one launch over
 * n_seeds device seeds; writes the dense (n_seeds, n_steps, 4) float32
 * points and uint32 lengths to device memory exactly as the reference's
 * `tractogram` kernel does.  Stream-ordered, does not synchronise. */
int tg_tractogram(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                  const float* seeds, uint32_t n_seeds, float save_at, uint32_t n_steps,
                  float* streamlines, uint32_t* lengths, void* stream);

/* tg_tractogram with host buffers (tracking.py:152-176 including the
 * uploads and read-backs); synchronises the stream. */
int tg_tractogram_host(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                       const float* seeds, uint32_t n_seeds, float save_at, uint32_t n_steps,
                       float* streamlines, uint32_t* lengths, void* stream);

/* Persistent batched tracker (the tg.tractogram batch loop of
 * tractography/__init__.py:524-539 as one device-scheduled launch).
 * Seeds are split into batches of `batch_size`; batch b uses
 * batch_rng_seeds[b] and stream ids 0..batch_size-1, which reproduces the
 * per-batch MWC64X streams of the reference.  Points are packed, not dense.
 * pool_points bounds the device point pool (0 = size on first use). */
int tg_tracker_create(uint64_t pool_points, tg_tracker** out);
int tg_tracker_destroy(tg_tracker* tracker);

/* Track `n_seeds` seeds (device pointer, or host pointer when seeds_on_host
 * != 0).  On return (the stream is synchronised) h_lengths[i] holds the
 * point count of streamline i, h_offsets[i] the index of its first point in
 * the tracker's packed point buffer, *total_points the buffer's size and
 * *total_steps the number of accepted steps (loop iterations of
 * tracking.py:121-147 that passed both checks).  batch_rng_seeds is a host
 * array of ceil(n_seeds / batch_size) seeds. */
int tg_tracker_run(tg_tracker* tracker, const tg_algorithm* algorithm, const tg_domain* domain,
                   const tg_field* field, const float* seeds, int seeds_on_host, uint32_t n_seeds,
                   uint32_t batch_size, const uint32_t* batch_rng_seeds, float save_at,
                   uint32_t n_steps, uint32_t* h_lengths, uint64_t* h_offsets,
                   uint64_t* total_points, uint64_t* total_steps, void* stream);

/* One tracking job: the arguments of one reference tg.tractogram call
 * (tractography/__init__.py:369-540) after its host-side preparation. */
typedef struct {
    const tg_domain* domain;
    const tg_field* field;
    tg_algorithm algorithm;          /* rng_seed unused: see batch_rng_seeds */
    const float* seeds;              /* (n_seeds, 8); host or device, see seeds_on_host */
    uint32_t n_seeds;
    uint32_t batch_size;
    const uint32_t* batch_rng_seeds; /* host, ceil(n_seeds / batch_size) seeds */
    float save_at;
    uint32_t n_steps;
} tg_job;

/* Track many jobs of uneven size, model, algorithm and length at once: every
 * job's seeds go to a device queue of its code path (model, lmax,
 * algorithm); one persistent launch per code path, all on concurrent
 * streams, drains the queues with lanes refilling as streamlines terminate.
 * Outputs are over the concatenation of the jobs' seeds in the order given:
 * h_lengths and h_offsets have sum(n_seeds) entries; points are read with
 * tg_tracker_copy_points.  Results equal those of one tg_tracker_run per
 * job.  No reference counterpart: the reference runs jobs one after another. */
int tg_tracker_run_jobs(tg_tracker* tracker, const tg_job* jobs, uint32_t n_jobs, int seeds_on_host,
                        uint32_t* h_lengths, uint64_t* h_offsets, uint64_t* total_points,
                        uint64_t* total_steps, void* stream);

/* Statistics of the last tg_tracker_run: device time of the tracking
 * kernel launches (CUDA events on the run's stream), number of waves (more
 * than one only when the point pool ran out) and number of kernel launches.
 * No reference counterpart: instrumentation for the benchmark. */
int tg_tracker_stats(const tg_tracker* tracker, float* kernel_ms, uint32_t* waves, uint32_t* launches);

/* Launch shape and tail compaction of the tracker's persistent launches.
 * blocks_per_sm: resident blocks of 128 lanes per SM (0 = the occupancy
 * maximum; larger values are capped to it).  Tail compaction: once a launch's
 * queue is empty, a warp with at most compact_lanes live streamlines hands
 * them to the next round and exits; compact_rounds further rounds run those
 * streamlines in full warps, the last round to completion (compact_lanes 0:
 * one launch, no compaction).  Results do not depend on these settings.
 * Defaults: 0, 0, 4 (compaction off: a carried streamline waits for the
 * previous round's tail, which costs more than the sparse warps it saves on
 * the workloads measured).  No reference counterpart: the autotuner's knobs. */
int tg_tracker_set_tuning(tg_tracker* tracker, uint32_t blocks_per_sm, uint32_t compact_lanes,
                          uint32_t compact_rounds);
int tg_tracker_get_tuning(const tg_tracker* tracker, uint32_t* blocks_per_sm, uint32_t* compact_lanes,
                          uint32_t* compact_rounds);

/* Time slicing of tg_tracker_run's persistent launch.  slice_steps 0: every
 * lane tracks a streamline to its end before taking the next seed.  A power
 * of two: the slice is K saved points, K the largest power of two whose
 * points take at most slice_steps steps (by the most steps that can separate
 * two saved points); a streamline whose point count reaches a multiple of K
 * while other work waits (seeds not yet started, or streamlines already
 * saved) is saved to a device queue and its lane takes the next work, seeds
 * first, then the saved streamlines in the order they were saved.  Every
 * seed then starts early and the long streamlines share the lanes
 * round-robin, so the launch no longer ends with a long streamline that
 * started last running on an otherwise idle GPU.  Runs whose step bound
 * (tg_step_bound) does not exceed slice_steps are not sliced.  Results do
 * not depend on this setting (a saved streamline carries its position,
 * orientation, RNG state and output cursor).  The queue takes about 104
 * bytes per seed of a sliced run.  Default 65536.  Returns
 * TG_ERR_INVALID_ARGUMENT for other values.  No reference counterpart:
 * scheduling only. */
int tg_tracker_set_slicing(tg_tracker* tracker, uint32_t slice_steps);
int tg_tracker_get_slicing(const tg_tracker* tracker, uint32_t* slice_steps);

/* Continuous-batching server.  No reference counterpart (the reference
 * tracks one tg.tractogram call at a time).  Fields, domains and surfaces
 * stay resident as ordinary handles; requests (tg_job with HOST seeds and
 * batch seeds, which the caller keeps valid until the request is reported
 * finished; they are copied to the device at admission) are admitted in
 * arrival order while a
 * request slot is free and the server's memory -- the shared point pool,
 * per-request buffers and unclaimed results -- fits in hbm_budget_bytes.
 * Each tg_server_poll runs one epoch: one persistent launch per code path
 * on concurrent streams, every lane executing at most epoch_steps loop
 * iterations; live streamlines carry over to the next epoch and new
 * arrivals enter the queues between epochs.  After each epoch the
 * streamlines that finished move from the shared pool to their request's
 * result buffer.  Finished requests are reported by id; their results equal
 * the same job run alone.
 * pool_points sizes the shared point pool (0 = 32M points). */
typedef struct tg_server tg_server;
int tg_server_create(uint64_t hbm_budget_bytes, uint64_t pool_points, uint32_t epoch_steps,
                     uint32_t max_requests, tg_server** out);
int tg_server_destroy(tg_server* server);
int tg_server_submit(tg_server* server, const tg_job* job, uint64_t* request_id);
/* One epoch; writes up to `capacity` finished request ids.  n_active and
 * n_pending (nullable) report admitted and waiting requests afterwards. */
int tg_server_poll(tg_server* server, uint64_t* finished_ids, uint32_t capacity, uint32_t* n_finished,
                   uint32_t* n_active, uint32_t* n_pending);
/* Size of a finished request's result and seconds from submission to completion. */
int tg_server_result_size(tg_server* server, uint64_t request_id, uint32_t* n_seeds, uint64_t* n_points,
                          double* seconds);
/* Copy the result to host arrays and release it: lengths (n_seeds uint32),
 * offsets (n_seeds uint64: first point of each streamline in `points`) and
 * points ((n_points, 3) float32, streamlines in the order they finished).
 * Any pointer may be null to skip that array. */
int tg_server_take(tg_server* server, uint64_t request_id, uint32_t* lengths, uint64_t* offsets,
                   float* points);
int tg_server_stats(const tg_server* server, uint64_t* steps, uint64_t* epochs, double* busy_seconds,
                    uint64_t* reserved_bytes);
/* Map `bytes` of device memory into the server's memory pool now (they stay
 * reserved for request buffers and results, up to the budget), so that
 * admissions and growing results do not map memory between epochs. */
int tg_server_reserve(tg_server* server, uint64_t bytes);
/* Device-clock budget of an epoch in seconds (0, the default: epoch_steps
 * alone ends an epoch).  With a budget, every code path's lanes stop at the
 * same deadline, whatever their step cost; results do not change. */
int tg_server_set_epoch_time(tg_server* server, double seconds);
/* Device-timeline seconds, summed over epochs: the tracking launches; from
 * their end to the harvest's start (counter read-back and host bookkeeping);
 * the harvest. */
int tg_server_timing(const tg_server* server, double* kernel_seconds, double* between_seconds,
                     double* harvest_seconds);

/* Copy points [first, first + count) of the packed (total_points, 3)
 * float32 buffer of the last run to `dst` (host when dst_on_host != 0). */
int tg_tracker_copy_points(tg_tracker* tracker, float* dst, uint64_t first, uint64_t count,
                           int dst_on_host, void* stream);

/* Largest number of batches one tg_tractogram_noalloc call accepts. */
#define TG_NOALLOC_MAX_BATCHES 16384

/* Tracking for callers that cannot allow the library to allocate device
 * memory (for example a host application that owns the GPU memory budget and
 * hands fixed buffers to plugins, or a loop where cudaMalloc's possible device
 * synchronisation is unacceptable).  No counterpart in the reference: it is
 * tg_tractogram's dense contract run by the persistent lane-refill tracker
 * over batches (as tg_tracker_run numbers them: batch b = seeds
 * [b * batch_size, (b + 1) * batch_size) with seed batch_rng_seeds[b], a host
 * array), writing into the caller's device buffers `streamlines`
 * (n_seeds, n_steps, 4) and `lengths` (n_seeds).  It calls no cudaMalloc,
 * cudaFree or allocating library routine; its only scratch is a library-wide
 * static device array of 64 KiB + 256 B per GPU (held until process exit)
 * that holds at most TG_NOALLOC_MAX_BATCHES batch seeds -- more batches are
 * rejected with TG_ERR_INVALID_ARGUMENT.  The first call on a device looks
 * up that array's address (cudaGetSymbolAddress) and should come before any
 * stream capture.  batch_rng_seeds is copied into the array on `stream`:
 * from pageable host memory the call returns after the copy; from
 * page-locked memory it may return before, and the caller must leave the
 * array unchanged until the stream has run the copy.  Every call shares the
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller. */
int tg_tractogram_noalloc(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                          const float* seeds, uint32_t n_seeds, uint32_t batch_size,
                          const uint32_t* batch_rng_seeds, float save_at, uint32_t n_steps, float* streamlines,
                          uint32_t* lengths, void* stream);

/* FOD seeding: seeds.cl:99-118 as launched by seeds.py:174-216.  `fod` is
 * the device sparse (nnz, n_coefficients) array, `voxels` the device
 * (nnz, 4) voxel indices with w = 1, `affine` the device voxel-to-world
 * row-major 4x4, `states` the device (n_seeds, 2) MWC64X states drawn on the
 * host.  Writes device (n_seeds, 8) seeds. */
int tg_seeds_from_fod(int32_t model, uint32_t n_coefficients, const float* fod, const float* voxels,
                      uint32_t nnz, const float* affine, const uint32_t* states, uint32_t n_seeds,
                      float* seeds, void* stream);

/* Per-element kernels of the reference's standalone entry points (device
 * pointers; points/orientations are (n, 4) float32). */
/* domain.contains, domain.py:433-491 */
int tg_domain_contains(const tg_domain* domain, const float* points, uint32_t n, uint8_t* out,
                       void* stream);
/* field.evaluate, field.py:144-197: out (n, C) */
int tg_field_evaluate(const tg_field* field, const float* points, uint32_t n, float* out, void* stream);
/* tracking.tod (tracking.py:181-385): n_seeds boundary seeds (sampler
 * arrays as for tg_boundary_seeds, rng_init(algorithm->rng_seed, i) then the
 * Diffusion noise of the same stream) integrated for at most n_steps
 * iterations; the lmax-8 real SH basis of the orientation at every iteration
 * is added into `coefficients`, a device (out_dims[0], out_dims[1],
 * out_dims[2], 45) float32 array (not cleared; the caller zeroes it), at the
 * voxel floor(A^-1 p + 0.5) of the output grid (out_inverse_affine,
 * row-major 4x4).  Additions from different threads are unordered.
 * steps (nullable, device uint64): the iterations that passed the domain and
 * field tests are added to it. */
int tg_tod(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field, const float* vertices,
           uint32_t n_vertices, const uint32_t* triangles, const float* cumulative_areas, uint32_t n_triangles,
           uint32_t n_seeds, uint32_t n_steps, const uint32_t out_dims[3], const float out_inverse_affine[16],
           float* coefficients, uint64_t* steps, void* stream);
/* tracking.connectome (tracking.py:388-602): n_seeds boundary seeds
 * (sampler arrays as for tg_boundary_seeds) tracked for at most n_steps
 * iterations; a track that moved at least minimum_length and whose final
 * segment hits the boundary (closest hit in `boundary`, a mesh domain made
 * from the same vertices and faces) writes the 9 products of its start and
 * end barycentric weights at (start vertex, end vertex) pairs into rows,
 * columns and weights (device, 9 per seed; rows = -1 where nothing was
 * written).  Deterministic.  steps (nullable, device uint64) as for
 * tg_tod. */
int tg_connectome(const tg_algorithm* algorithm, const tg_domain* domain, const tg_field* field,
                  const tg_domain* boundary, const float* vertices, uint32_t n_vertices, const uint32_t* triangles,
                  const float* cumulative_areas, uint32_t n_triangles, uint32_t n_seeds, uint32_t n_steps,
                  float minimum_length, int32_t* rows, int32_t* columns, float* weights, uint64_t* steps,
                  void* stream);
/* domain.seed, domain.py:494-575 with domain_sample_boundary (:95-120):
 * n_seeds seeds uniform over a boundary surface's area, pointing inward,
 * seed i drawing from rng_init(rng_seed, i).  Device arrays: vertices
 * (n_vertices, 4) float32, triangles (n_triangles, 4) uint32, normalised
 * cumulative areas (n_triangles) float32 (last = 1); seeds (n_seeds, 8). */
int tg_boundary_seeds(const float* vertices, uint32_t n_vertices, const uint32_t* triangles,
                      const float* cumulative_areas, uint32_t n_triangles, uint32_t rng_seed, uint32_t n_seeds,
                      float* seeds, void* stream);
/* local.evaluate, local.py:285-363: out (n, 3) = value, d/dtheta, (d/dphi)/sin(theta) */
int tg_local_evaluate(int32_t model, uint32_t n_parameters, const float* parameters,
                      const float* orientations, uint32_t n, float* out, void* stream);
/* algorithm.update_orientation, algorithm.py:701-790: out (n, 4) */
int tg_update_orientation(int32_t model, uint32_t n_parameters, const tg_algorithm* algorithm,
                          const float* parameters, const float* orientations, uint32_t n, float* out,
                          void* stream);
/* randus / randis test streams, core.cl:218-238 (which: 0 randu, 1 randn,
 * 2 randi below `max`), from the raw MWC64X state (s0, s1). */
int tg_rng_stream(int32_t which, uint32_t s0, uint32_t s1, uint32_t n, uint32_t max, void* out,
                  void* stream);

/* The step limit every tracking entry point applies to a streamline of the
 * tractogram loop (tracking.py:121-147), which saves a point each time the
 * binary32 sum time += step_size reaches save_at.  *max_steps receives
 * n_steps times the most loop iterations that can separate two saved points
 * (a bound that never ends a streamline the reference would continue).
 * Returns TG_ERR_INVALID_ARGUMENT when time + step_size == time for some
 * time below save_at (the reference's loop would then run for ever on a
 * streamline that stays in the domain) or when the limit exceeds 2^32 - 1;
 * every tracking entry point rejects the same parameters.  Host only. */
int tg_step_bound(float step_size, float save_at, uint32_t n_steps, uint64_t* max_steps);

#ifdef __cplusplus
}
#endif

#endif /* TRACTOGRAPHY_B200_H */
