/*
 * tg_internal.h -- structures shared by the CUDA launchers and the C-ABI.
 */
#ifndef TG_INTERNAL_H
#define TG_INTERNAL_H

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "tg_bvh.cuh"
#include "tg_device.cuh"

namespace tg {

struct LaneCarry;   // tg_step.cuh

// Default time slice of tg_tracker_run (tg_tracker_set_slicing), in steps.
constexpr uint32_t kDefaultSliceSteps = 65536;

// A FIFO of saved streamlines shared by one launch's lanes.  Ticket t
// (taken from ctl[1]) is written to slot t % capacity, published by
// seq[slot] = t + 1; a lane claims the oldest ticket (ctl[0]) only while it
// is below ctl[1], and marks the slot free again by released[slot] = t + 1.
// ctl[2]: nonzero when a bounded wait ran out (1: a slot's wait, 2: a
// claim's retries; the run then fails).  seq,
// released and ctl are zero at the launch.  capacity exceeds the number of
// streamlines that can be live at once, so a ticket's slot was claimed long
// before the ticket capacity later reuses it.
struct TrackRing {
    LaneCarry* items;
    uint32_t* seq;
    uint32_t* released;
    unsigned int* ctl;
    uint32_t capacity;
    uint32_t lanes;      // lanes of the launch: claims in flight at most
};

constexpr int kChunkPoints = 32;   // points per output chunk (chunk = 32 x 12 B)

// Device-resident image field (field.py:52-122): float32 coefficients,
// voxel-major (x, y, z) C order, each voxel padded to cpad floats
// (cpad = round_up(full band, 4)) so a voxel loads as float4s.
struct FieldDev {
    float* data = nullptr;
    // what the trackers read: SH coefficients folded per voxel (tgsh_fold,
    // same layout and padding); the raw coefficients for tensors
    float* folded = nullptr;
    uint32_t nx = 0, ny = 0, nz = 0;
    uint32_t n_params = 0;     // C as given by the caller
    uint32_t cpad = 0;
    int model = kModelSH;      // SH unless created as a tensor field
    int lmax = 0;
    float inv_affine[16];
    size_t bytes = 0;
};

// Device-resident domain.  Image (domain.py:267-398): uint8 mask, same voxel
// order as the reference's int32 mask.  Mesh: a closed triangle surface with
// its boundary BVH (domain.py:44-116) and distance grid (tg_bvh.cuh).
struct DomainDev {
    int kind = kDomainImage;
    uint8_t* mask = nullptr;
    uint32_t nx = 0, ny = 0, nz = 0;
    float inv_affine[16];
    size_t bytes = 0;
    // mesh
    float4* nodes = nullptr;
    float4* tris = nullptr;
    uint32_t* cells = nullptr;    // distance | leaf list offset << 8
    uint32_t* lists = nullptr;
    uint32_t n_triangles = 0;
    MeshDev mesh{};
};

// Everything one tracking launch needs, by value.
struct TrackParams {
    int domain_kind;         // kDomainImage (mask) or kDomainMesh
    MeshDev mesh;
    Grid dgrid;
    const uint8_t* mask;
    Grid fgrid;
    const float* field;
    uint32_t cpad;
    int same_grid;           // domain and field inverse affines/dims identical
    int algorithm;           // kTransport or kDiffusion
    AlgoParams algo;
    float save_at;
    uint32_t n_steps;
    // Upper bound on the steps of one streamline (step_bound in tg_capi.cu):
    // n_steps saved points times the most loop iterations binary32 time
    // accumulation can take between two of them.  It never binds for the
    // inputs the host accepts; it only guarantees that every lane ends.
    uint32_t max_steps;
};

// Batched persistent launch over work items 0..n_items-1; item k tracks
// seed item_ids[k] (or k when item_ids is null).  Seed i belongs to batch
// i / batch_size with stream id i % batch_size (tracking.py:105,115,
// __init__.py:525), which keeps the reference's per-batch MWC64X streams.
constexpr uint32_t kOverflowBit = 0x80000000u;   // in lengths[]: pool ran out

struct PersistentParams {
    TrackParams t;
    const float4* seeds;          // (n_seeds, 2) float4
    uint32_t n_seeds;
    const uint32_t* item_ids;     // nullable
    uint32_t n_items;
    uint32_t batch_size;
    const uint32_t* batch_rng_seeds;
    uint64_t seed_offset;         // Philox index base
    const uint8_t* seed_inside;   // closed surface: per seed, the inside test done by a pre-pass; nullable
    unsigned long long* item_counter;
    // output: chunk pool
    float* pool;                  // n_chunks * kChunkPoints * 3 floats
    int32_t* chunk_next;          // n_chunks
    uint32_t n_chunks;
    unsigned int* chunk_counter;
    int32_t* first_chunk;         // n_seeds
    uint32_t* lengths;            // n_seeds; kOverflowBit set when retried
    unsigned long long* steps_done;   // total accepted steps
    // Tail compaction.  A round pulls seeds (carry_in null) or resumes the
    // streamlines carry_in[0 .. *carry_in_count) left by the previous round;
    // with carry_out set, a warp whose queue is empty and whose live lanes
    // number at most compact_lanes writes them to carry_out and exits, so
    // the next round runs them in full warps.
    const LaneCarry* carry_in;
    const unsigned int* carry_in_count;
    LaneCarry* carry_out;
    unsigned int* carry_out_count;
    uint32_t compact_lanes;
    // Time slicing (tg_tracker_set_slicing): with ring.items set, a
    // streamline whose point count reaches a multiple of slice_mask + 1
    // while other work waits (seeds left in the queue, or streamlines in the
    // ring) is saved at the ring's tail and its lane takes the next work;
    // lanes take seeds first, then the ring in order.  Every seed thus starts
    // early and the long streamlines share the lanes round-robin, instead of
    // a long streamline started last setting the end of the launch.
    TrackRing ring;
    uint32_t slice_mask;
};

// Many jobs queued at once (tg_multi.cu).  Job j covers global seed indices
// [job_base[j], job_base[j + 1]); its seeds, field, domain and parameters
// are in jobs[j].  Jobs are grouped in classes of identical code path
// (model, lmax, algorithm), each drained by one persistent launch whose
// lanes refill from the class's queue as their streamlines terminate.
struct JobDev {
    TrackParams t;
    const float4* seeds;
    uint32_t n_seeds;
    uint32_t batch_size;
    uint32_t rng_base;          // index of this job's batch 0 in batch_rng_seeds
    uint32_t pad;
    uint64_t seed_offset;       // Philox index base
};

enum ClassKind : int {
    kSH0T, kSH0D, kSH2T, kSH2D, kSH4T, kSH4D, kSH6T, kSH6D, kSH8T, kSH8D, kDTIT, kDTID, kClassKinds
};

struct ClassDev {
    int kind;
    uint32_t n_jobs;
    const uint32_t* jobs;       // job indices of this class, in queue order
    const uint32_t* prefix;     // n_jobs + 1 prefix sums of their seed counts
    const uint32_t* item_ids;   // nullable: global seed indices to retry
    uint32_t n_items;
    unsigned long long* counter;
};

struct MultiParams {
    // tail compaction, per class round as in PersistentParams
    const LaneCarry* carry_in;
    const unsigned int* carry_in_count;
    LaneCarry* carry_out;
    unsigned int* carry_out_count;
    uint32_t compact_lanes;
    const JobDev* jobs;
    const uint32_t* job_base;   // n_jobs + 1
    uint32_t n_jobs;
    const uint32_t* batch_rng_seeds;
    float* pool;
    int32_t* chunk_next;
    uint32_t n_chunks;
    unsigned int* chunk_counter;
    int32_t* first_chunk;       // per global seed
    uint32_t* lengths;          // per global seed; kOverflowBit when retried
    unsigned long long* steps_done;
};

// One persistent launch per class (code path); classes run concurrently on
// separate streams and share the point pool.
cudaError_t launch_track_class(const MultiParams& mp, const ClassDev& cls, int grid, cudaStream_t stream);
int class_blocks_per_sm(int kind);
int class_kind(int model, int lmax, int algorithm);

// Track orientation distribution (tg_tod.cu, tracking.py:181-385).
struct TodParams {
    TrackParams t;                 // domain, field, algorithm
    const float4* vertices;        // boundary sampler arrays (device)
    const uint4* triangles;
    const float* cumulative;
    uint32_t n_triangles;
    uint32_t rng_seed;
    uint64_t seed_offset;          // Philox index base
    uint32_t n_seeds;
    uint32_t n_steps;              // floor(maximum_streamline_length / step_size)
    float4 out_row0, out_row1, out_row2;   // output grid inverse affine rows
    uint32_t nx, ny, nz;
    float* coefficients;           // (nx, ny, nz, 45) float32, accumulated
    unsigned long long* steps;     // nullable: loop iterations that passed the domain and field tests
    unsigned long long* counter;   // next seed index (zeroed by the launcher)
};
cudaError_t launch_tod(int model, int lmax, const TodParams& q, cudaStream_t stream);

// Boundary connectome (tg_connectome.cu, tracking.py:388-602).
struct ConnectomeParams {
    TrackParams t;                 // domain, field, algorithm
    const float4* vertices;        // boundary sampler arrays (device)
    const uint4* triangles;
    const float* cumulative;
    uint32_t n_triangles;
    MeshDev bvh;                   // BVH of the same boundary triangles
    uint32_t rng_seed;
    uint64_t seed_offset;
    uint32_t n_seeds;
    uint32_t n_steps;
    float minimum_length;
    int32_t* rows;                 // 9 per seed, -1 when the track contributes nothing
    int32_t* columns;
    float* weights;
    unsigned long long* steps;     // nullable: loop iterations that passed the domain and field tests
    unsigned long long* counter;   // next seed index (zeroed by the launcher)
};
cudaError_t launch_connectome(int model, int lmax, const ConnectomeParams& q, cudaStream_t stream);

// Boundary seeding (tg_aux.cu).
cudaError_t launch_boundary_seeds(const float4* vertices, const uint4* triangles, const float* cumulative,
                                  uint32_t n_triangles, uint32_t rng_seed, uint32_t n, float4* out,
                                  cudaStream_t stream);

// Closed-surface domain (tg_mesh.cu).  The boundary BVH in the reference's
// array layout (domain.py:100-116), built on the host.
struct BoundaryBvhHost {
    std::vector<float> vertices4;      // (V, 4), w = 1
    std::vector<uint32_t> triangles4;  // (T, 4), kept (non-degenerate) faces
    std::vector<float> bounds_min;     // (N, 4)
    std::vector<float> bounds_max;     // (N, 4)
    std::vector<int32_t> nodes;        // (N, 4): left, right, first, count
    std::vector<uint32_t> ordered;     // (T,)
    uint32_t n_nodes = 0;
    uint32_t n_triangles = 0;
};
int build_boundary_bvh(const double* vertices, uint32_t n_vertices, const uint32_t* faces, uint32_t n_faces,
                       BoundaryBvhHost* out, std::string* error);
cudaError_t upload_mesh(const BoundaryBvhHost& b, DomainDev* d, cudaStream_t stream);
cudaError_t launch_mesh_segments_blocked(const MeshDev& m, const float4* starts, const float4* ends, uint32_t n,
                                         uint8_t* blocked, cudaStream_t stream);
cudaError_t launch_mesh_segment_hits(const MeshDev& m, const float4* starts, const float4* ends, uint32_t n,
                                     uint8_t* found, uint32_t* triangle, float4* hit, cudaStream_t stream);
// Inside test of points[i * stride] (stride 2 for (n, 2) float4 seeds).
cudaError_t launch_mesh_contains(const MeshDev& m, const float4* points, uint32_t n, uint8_t* out,
                                 cudaStream_t stream, uint32_t stride = 1);

// Launchers (tg_track.cu).
cudaError_t launch_track_dense(const FieldDev& f, const TrackParams& p, const float4* seeds,
                               uint32_t n_seeds, uint32_t rng_seed, uint64_t seed_offset,
                               float4* out, uint32_t* lengths, cudaStream_t stream);
cudaError_t launch_track_persistent(const FieldDev& f, const PersistentParams& p, int grid,
                                    int block, cudaStream_t stream);
// offsets[i] = exclusive prefix sum of the lengths, overflowed streamlines
// counted as 0; totals[0] = points, totals[1] = overflowed streamlines.
// With temp == nullptr, only sets *temp_bytes (scan scratch size).
cudaError_t launch_offsets(const uint32_t* lengths, uint32_t n, uint64_t* masked, uint64_t* offsets,
                           unsigned long long* totals, void* temp, size_t* temp_bytes, cudaStream_t stream);
// seed_ids == nullptr: seeds 0..n_ids-1.
cudaError_t launch_gather(const float* pool, const int32_t* chunk_next, const int32_t* first_chunk,
                          const uint32_t* lengths, const uint64_t* offsets, const uint32_t* seed_ids,
                          uint32_t n_ids, float* out_points, cudaStream_t stream);

// Unit hooks (tg_aux.cu).
cudaError_t launch_contains(const DomainDev& d, const float4* points, uint32_t n, uint8_t* out,
                            cudaStream_t stream);
// SH fields: the folded copy the trackers read (tgsh_fold per voxel).
cudaError_t launch_fold_field(const float* raw, float* folded, uint64_t n_voxels, uint32_t cpad, int lmax,
                              cudaStream_t stream);
cudaError_t launch_field_evaluate(const FieldDev& f, const float4* points, uint32_t n, float* out,
                                  cudaStream_t stream);
cudaError_t launch_local_evaluate(int model, uint32_t n_params, const float* params,
                                  const float4* orientations, uint32_t n, float* out,
                                  cudaStream_t stream);
cudaError_t launch_update_orientation(int model, uint32_t n_params, int algorithm,
                                      const AlgoParams& a, uint32_t rng_seed, uint64_t seed_offset,
                                      const float* params, const float4* orientations, uint32_t n,
                                      float4* out, cudaStream_t stream);
cudaError_t launch_seeds_from_fod(int model, uint32_t n_coefficients, const float* fod,
                                  const float4* voxels, uint32_t nnz, const float* affine,
                                  const uint2* states, uint32_t n_seeds, float4* seeds,
                                  cudaStream_t stream);
cudaError_t launch_rng_streams(int which, uint32_t s0, uint32_t s1, uint32_t n, uint32_t max,
                               void* out, cudaStream_t stream);

int lmax_for(uint32_t n_params);
int persistent_block_size();
int persistent_blocks_per_sm(const FieldDev& f, int algorithm, int domain_kind);

}  // namespace tg

#endif
