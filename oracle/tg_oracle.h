/*
 * tg_oracle.h -- CPU oracle for the streamline-tracking path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference's OpenCL tracking kernel and its plugins, used by the tests, by
 * the smoke check and by the benchmark's CPU-baseline leg to check the CUDA
 * path.  Nothing in the product links or calls it.
 *
 * Arithmetic contract: every float operation below is an IEEE-754 binary32
 * operation in a fixed order (explicit fmaf, no contraction, transcendentals
 * from tg_fmath.h), the same contract the CUDA kernels follow, so the two
 * agree bit for bit.  Against the reference itself (whose transcendentals
 * come from the OpenCL platform) agreement is to float tolerance.
 */
#ifndef TG_ORACLE_H
#define TG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { TGO_MODEL_SH = 0, TGO_MODEL_DTI = 1 };
enum { TGO_ALGO_TRANSPORT = 0, TGO_ALGO_DIFFUSION = 1 };
enum { TGO_RNG_MWC64X = 0, TGO_RNG_PHILOX = 1 };

/* Boundary BVH in the reference's layout (domain.py:72-116, bvh.cl:6-14):
 * preorder nodes, leaves with left = right = -1 and (first, count) into
 * ordered_triangles, float32 node bounds, float4 vertices, uint4 triangles. */
typedef struct {
    const float* vertices;              /* (V, 4) */
    const uint32_t* triangles;          /* (T, 4), 4th unused */
    const float* bounds_min;            /* (N, 4) */
    const float* bounds_max;            /* (N, 4) */
    const int32_t* nodes;               /* (N, 4): left, right, first, count */
    const uint32_t* ordered_triangles;  /* leaf slots -> triangle ids */
    uint32_t n_nodes;
} tgo_bvh;

typedef struct {
    /* domain (domain.py:350-356): int32 mask, dims, inverse affine rows */
    const int32_t* mask;
    uint32_t mask_dims[3];
    float mask_inv_affine[16];
    /* field (field.py:82-86): float32 (X, Y, Z, C), dims, inverse affine */
    const float* field;
    uint32_t field_dims[4];
    float field_inv_affine[16];
    /* local model and algorithm (local.py:74-230, algorithm.py:56-228) */
    int32_t model;
    int32_t algorithm;
    float step_size;
    float gamma;
    float noise_variance;
    /* random stream: MWC64X seeded by rng_init(rng_seed, index within the
     * call) as the reference does, or Philox4x32-10 keyed by philox_key and
     * counted by (seed_offset + index, step). */
    int32_t rng_mode;
    uint32_t rng_seed;
    uint64_t philox_key;
    uint64_t seed_offset;
    /* output */
    float save_at;
    uint32_t n_steps;
    /* closed-surface domain; when set, the mask above is not used.  A seed is
     * inside by tgo_mesh_contains; a streamline stops at the first step whose
     * segment from the previous point hits the surface (bvh.cl:83-131). */
    const tgo_bvh* mesh;
} tgo_problem;

/* tracking.py:93-149: dense (n_seeds, n_steps, 4) points and lengths.
 * Returns the number of accepted steps (loop iterations that passed both the
 * domain and the field check). */
uint64_t tgo_tractogram(const tgo_problem* p, const float* seeds, uint32_t n_seeds,
                        float* streamlines, uint32_t* lengths, int n_threads);

/* tgo_tractogram for seeds taken out of a larger call: seed i is work item
 * ids[i] of that call (tracking.py:103 get_global_id, which keys its
 * rng_init stream and its Philox counter). */
uint64_t tgo_tractogram_ids(const tgo_problem* p, const float* seeds, const uint32_t* ids, uint32_t n_seeds,
                            float* streamlines, uint32_t* lengths, int n_threads);

/* domain.py:358-382 for n points (x, y, z, w) -> 0/1. */
void tgo_contains(const tgo_problem* p, const float* points, uint32_t n, uint8_t* out);

/* field.py:88-114 for n points -> (n, C) coefficients, zero outside. */
void tgo_field_evaluate(const tgo_problem* p, const float* points, uint32_t n, float* out);

/* local.py:91-120, 212-230: (n, 3) value, d/dtheta, (d/dphi)/sin(theta). */
void tgo_local_evaluate(int32_t model, uint32_t n_params, const float* params,
                        const float* orientations, uint32_t n, float* out);

/* algorithm.py:738-759: one orientation update per row, RNG stream per row. */
void tgo_update_orientation(const tgo_problem* p, uint32_t n_params, const float* params,
                            const float* orientations, uint32_t n, float* out);

/* seeds.cl:68-118 + seeds.py:174-216: seeds (n, 8) from a sparse FOD. */
void tgo_seeds_from_fod(int32_t model, uint32_t n_coefficients, const float* fod,
                        const float* voxels, uint32_t nnz, const float affine[16],
                        const uint32_t* states, uint32_t n_seeds, float* seeds,
                        int n_threads);

/* bvh.cl:83-131: closest hit of the segment start-end; returns found and
 * writes the triangle id, barycentric (1-u-v, u, v) and the segment
 * parameter t in (1e-6, 1]. */
int tgo_bvh_segment_hit(const tgo_bvh* b, const float start[3], const float end[3], uint32_t* triangle,
                        float barycentric[3], float* t);

/* Number of triangles the segment crosses (bvh.cl:16-80 tests, max_t = 1). */
uint32_t tgo_bvh_count_hits(const tgo_bvh* b, const float start[3], const float end[3]);

/* Inside test of a closed surface: majority over three fixed rays of the
 * parity of surface crossings; 0 outside the root bounds. */
int tgo_mesh_contains(const tgo_bvh* b, float x, float y, float z);

/* Batched segment hits: starts/ends (n, 4); found (n); triangle (n);
 * hit (n, 4) = barycentric xyz and t. */
void tgo_segment_hits(const tgo_bvh* b, const float* starts, const float* ends, uint32_t n, uint8_t* found,
                      uint32_t* triangle, float* hit, int n_threads);

/* domain.py:494-575 + domain_sample_boundary (:95-120): seeds (n, 8)
 * uniform over a boundary surface's area, seed i from rng_init(rng_seed, i). */
void tgo_boundary_seeds(const float* vertices, const uint32_t* triangles, const float* cumulative,
                        uint32_t n_triangles, uint32_t rng_seed, uint32_t n, float* seeds);

/* tracking.py:181-385 (tod): boundary seeds integrated for at most n_steps
 * iterations, the lmax-8 SH basis of the orientation added at the output
 * voxel of every iteration, seeds processed in order; coefficients
 * (nx, ny, nz, 45) accumulate (not cleared). */
void tgo_tod(const tgo_problem* p, const float* vertices, const uint32_t* triangles, const float* cumulative,
             uint32_t n_triangles, uint32_t n_seeds, uint32_t n_steps, const uint32_t out_dims[3],
             const float out_inverse_affine[16], float* coefficients);

/* tracking.py:388-602 (connectome): per seed, 9 (row, column, weight)
 * contributions (rows -1 when none) from the start barycentric weights and
 * the closest boundary hit of the final segment in `boundary`. */
void tgo_connectome(const tgo_problem* p, const tgo_bvh* boundary, const float* vertices, const uint32_t* triangles,
                    const float* cumulative, uint32_t n_triangles, uint32_t n_seeds, uint32_t n_steps,
                    float minimum_length, int32_t* rows, int32_t* columns, float* weights);

/* core.cl:180-245 primitives. */
void tgo_rng_init(uint32_t seed, uint32_t stream_id, uint32_t state[2]);
void tgo_randu_stream(uint32_t s0, uint32_t s1, uint32_t n, float* out);
void tgo_randn_stream(uint32_t s0, uint32_t s1, uint32_t n, float* out);
void tgo_randi_stream(uint32_t s0, uint32_t s1, uint32_t n, uint32_t max, uint32_t* out);
void tgo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Shared math layer, exposed so tests can measure its accuracy. */
void tgo_math(int which, const float* x, uint32_t n, float* out);

#ifdef __cplusplus
}
#endif

#endif
