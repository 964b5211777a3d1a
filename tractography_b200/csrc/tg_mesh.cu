/*
 * tg_mesh.cu -- closed-surface domain: the boundary BVH build (host), its
 * device layout and distance grid, and the segment-hit and inside-test
 * kernels.
 *
 * The build follows BaseDomain._set_boundary_data (domain.py:44-116):
 * triangles of zero or non-finite area are dropped; triangle bounds and
 * centroids are float64; a node holding more than 4 triangles sorts them by
 * centroid along the longest axis of its bounds (the first such axis on
 * ties) and gives the first half (n / 2) to its left child and the rest to
 * its right child; nodes are numbered in preorder and bounds stored as
 * float32.  The sort is stable, where NumPy's default argsort in the
 * reference is not: the two agree whenever no two centroids of a node are
 * equal along its split axis.  Subtree sizes depend only on triangle
 * counts, so node numbers and leaf slots are known before a subtree is
 * built and the upper levels build in parallel threads.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "tg_internal.h"

namespace tg {

namespace {

constexpr uint32_t kLeafSize = 4;      // domain.py:85
constexpr int kMaxDepth = 60;          // bvh.cl:124 stack of 64 entries
constexpr int kParallelLevels = 4;     // up to 16 build threads
constexpr uint32_t kParallelMin = 16384;

uint32_t subtree_nodes(uint32_t n)
{
    return n <= kLeafSize ? 1u : 1u + subtree_nodes(n / 2) + subtree_nodes(n - n / 2);
}

int subtree_depth(uint32_t n) { return n <= kLeafSize ? 1 : 1 + subtree_depth(n - n / 2); }

struct Builder {
    const double* tmin;
    const double* tmax;
    const double* centroid;
    BoundaryBvhHost* out;

    void build(uint32_t* ids, uint32_t n, uint32_t node, uint32_t slot, int level) const
    {
        double lo[3] = {INFINITY, INFINITY, INFINITY};
        double hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t id = ids[k];
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], tmin[3 * (size_t)id + a]);
                hi[a] = std::max(hi[a], tmax[3 * (size_t)id + a]);
            }
        }
        for (int a = 0; a < 3; ++a) {
            out->bounds_min[4 * (size_t)node + a] = (float)lo[a];
            out->bounds_max[4 * (size_t)node + a] = (float)hi[a];
        }
        int32_t* nd = out->nodes.data() + 4 * (size_t)node;
        if (n <= kLeafSize) {
            nd[0] = -1;
            nd[1] = -1;
            nd[2] = (int32_t)slot;
            nd[3] = (int32_t)n;
            std::copy(ids, ids + n, out->ordered.begin() + slot);
            return;
        }
        int axis = 0;                                  // np.argmax: first maximum
        const double ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
        if (ext[1] > ext[axis]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        const double* key = centroid;
        std::stable_sort(ids, ids + n, [key, axis](uint32_t x, uint32_t y) {
            return key[3 * (size_t)x + axis] < key[3 * (size_t)y + axis];
        });
        const uint32_t half = n / 2;
        const uint32_t left = node + 1;
        const uint32_t right = node + 1 + subtree_nodes(half);
        nd[0] = (int32_t)left;
        nd[1] = (int32_t)right;
        nd[2] = 0;
        nd[3] = 0;
        if (level < kParallelLevels && n >= kParallelMin) {
            std::thread worker([&] { build(ids, half, left, slot, level + 1); });
            build(ids + half, n - half, right, slot + half, level + 1);
            worker.join();
        } else {
            build(ids, half, left, slot, level + 1);
            build(ids + half, n - half, right, slot + half, level + 1);
        }
    }
};

}  // namespace

int build_boundary_bvh(const double* vertices, uint32_t n_vertices, const uint32_t* faces, uint32_t n_faces,
                       BoundaryBvhHost* out, std::string* error)
{
    if (n_faces == 0) {
        *error = "The boundary mesh must contain at least one triangle.";
        return 1;
    }
    for (size_t k = 0; k < 3 * (size_t)n_faces; ++k) {
        if (faces[k] >= n_vertices) {
            *error = "face vertex index out of range";
            return 1;
        }
    }
    // domain.py:49-57: keep triangles of finite, positive area
    std::vector<uint32_t> kept;
    kept.reserve(n_faces);
    for (uint32_t f = 0; f < n_faces; ++f) {
        const double* A = vertices + 3 * (size_t)faces[3 * f];
        const double* B = vertices + 3 * (size_t)faces[3 * f + 1];
        const double* C = vertices + 3 * (size_t)faces[3 * f + 2];
        const double u[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
        const double v[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
        const double c[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
        const double area = 0.5 * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        if (std::isfinite(area) && area > 0.0) kept.push_back(f);
    }
    if (kept.empty()) {
        *error = "The boundary mesh must contain a non-degenerate triangle.";
        return 1;
    }
    const uint32_t T = (uint32_t)kept.size();
    if (T >= (1u << 28)) {
        *error = "boundary meshes are limited to 2^28 triangles";
        return 1;
    }
    if (subtree_depth(T) > kMaxDepth) {
        *error = "boundary BVH deeper than the traversal allows";
        return 1;
    }
    out->vertices4.assign(4 * (size_t)n_vertices, 1.0f);
    for (uint32_t i = 0; i < n_vertices; ++i)
        for (int a = 0; a < 3; ++a) out->vertices4[4 * (size_t)i + a] = (float)vertices[3 * (size_t)i + a];
    out->triangles4.assign(4 * (size_t)T, 0u);
    std::vector<double> tmin(3 * (size_t)T), tmax(3 * (size_t)T), centroid(3 * (size_t)T);
    for (uint32_t k = 0; k < T; ++k) {
        const uint32_t f = kept[k];
        for (int j = 0; j < 3; ++j) out->triangles4[4 * (size_t)k + j] = faces[3 * (size_t)f + j];
        for (int a = 0; a < 3; ++a) {
            const double x = vertices[3 * (size_t)faces[3 * f] + a];
            const double y = vertices[3 * (size_t)faces[3 * f + 1] + a];
            const double z = vertices[3 * (size_t)faces[3 * f + 2] + a];
            tmin[3 * (size_t)k + a] = std::min(std::min(x, y), z);
            tmax[3 * (size_t)k + a] = std::max(std::max(x, y), z);
            centroid[3 * (size_t)k + a] = (tmin[3 * (size_t)k + a] + tmax[3 * (size_t)k + a]) * 0.5;
        }
    }
    const uint32_t N = subtree_nodes(T);
    out->bounds_min.assign(4 * (size_t)N, 0.0f);
    out->bounds_max.assign(4 * (size_t)N, 0.0f);
    out->nodes.assign(4 * (size_t)N, 0);
    out->ordered.assign(T, 0u);
    out->n_nodes = N;
    out->n_triangles = T;
    std::vector<uint32_t> ids(T);
    for (uint32_t k = 0; k < T; ++k) ids[k] = k;
    const Builder b{tmin.data(), tmax.data(), centroid.data(), out};
    b.build(ids.data(), T, 0u, 0u, 0);
    return 0;
}

namespace {

// Distance grid over the root bounds: Chebyshev distance in cells to the
// nearest cell touched by a leaf box grown by a margin well above the
// rounding of the cell computation and of the slab test, capped at 255.
// Beside it, per cell A, the leaves whose grown box meets A's half-cell
// neighbourhood [A - 0.5, A + 1.5) (cell units, per axis): a segment inside
// that neighbourhood can pass the box test of no other leaf.  Cell word =
// distance | (list offset in 16-byte units << 8); a list is its leaf count
// followed by the leaf node indices (preorder) and zero padding up to
// 4 * (ceil(count / 4) + 1) words, all that the device's reads of four ids
// at a time reach; offset 0 is the empty list.  When the offsets would not
// fit in 24 bits every cell holds kNoLeafList and segments take the walk.
struct DistanceGrid {
    std::vector<uint8_t> d;
    std::vector<uint32_t> words;
    std::vector<uint32_t> lists;
    uint32_t g[3];
    float origin[3];
    float inv_cell;
};

DistanceGrid distance_grid(const BoundaryBvhHost& b)
{
    DistanceGrid G;
    double lo[3], hi[3], ext[3];
    double emax = 0.0;
    for (int a = 0; a < 3; ++a) {
        lo[a] = b.bounds_min[a];
        hi[a] = b.bounds_max[a];
        ext[a] = hi[a] - lo[a];
        emax = std::max(emax, ext[a]);
    }
    const double want = std::ceil(0.5 * std::sqrt((double)b.n_triangles));
    const int longest = (int)std::min(256.0, std::max(8.0, want));
    const float cell = (float)(emax / (double)(longest - 4));
    G.inv_cell = 1.0f / cell;
    for (int a = 0; a < 3; ++a) {
        G.origin[a] = (float)(lo[a] - 2.0 * (double)cell);
        G.g[a] = (uint32_t)std::ceil(ext[a] / (double)cell) + 4u;
    }
    const size_t gx = G.g[0], gy = G.g[1], gz = G.g[2];
    const double margin = 1e-5 * (emax + 4.0 * (double)cell) + 1e-3 * (double)cell;
    std::vector<uint8_t> occ(gx * gy * gz, 0);
    auto cell_of = [&](double x, int a) {
        const double c = std::floor((x - (double)G.origin[a]) * (double)G.inv_cell);
        return (long)std::min(std::max(c, 0.0), (double)(G.g[a] - 1));
    };
    for (uint32_t i = 0; i < b.n_nodes; ++i) {
        if (b.nodes[4 * (size_t)i + 3] <= 0) continue;          // internal node
        long c0[3], c1[3];
        for (int a = 0; a < 3; ++a) {
            c0[a] = cell_of((double)b.bounds_min[4 * (size_t)i + a] - margin, a);
            c1[a] = cell_of((double)b.bounds_max[4 * (size_t)i + a] + margin, a);
        }
        for (long x = c0[0]; x <= c1[0]; ++x)
            for (long y = c0[1]; y <= c1[1]; ++y)
                for (long z = c0[2]; z <= c1[2]; ++z) occ[((size_t)x * gy + y) * gz + z] = 1;
    }
    // two raster passes of the 26-neighbour chamfer: exact chessboard distance
    G.d.assign(gx * gy * gz, 255);
    for (size_t k = 0; k < occ.size(); ++k)
        if (occ[k]) G.d[k] = 0;
    auto pass = [&](int sign) {
        const long X = (long)gx, Y = (long)gy, Z = (long)gz;
        for (long xi = 0; xi < X; ++xi) {
            const long x = sign > 0 ? xi : X - 1 - xi;
            for (long yi = 0; yi < Y; ++yi) {
                const long y = sign > 0 ? yi : Y - 1 - yi;
                for (long zi = 0; zi < Z; ++zi) {
                    const long z = sign > 0 ? zi : Z - 1 - zi;
                    uint8_t& here = G.d[((size_t)x * gy + y) * gz + z];
                    if (here == 0) continue;
                    int best = here;
                    for (int dx = -1; dx <= 1; ++dx)
                        for (int dy = -1; dy <= 1; ++dy)
                            for (int dz = -1; dz <= 1; ++dz) {
                                // neighbours already visited in this pass
                                const int lex = dx != 0 ? dx : (dy != 0 ? dy : dz);
                                if (lex != -sign) continue;
                                const long nx = x + dx, ny = y + dy, nz = z + dz;
                                if (nx < 0 || ny < 0 || nz < 0 || nx >= X || ny >= Y || nz >= Z) continue;
                                best = std::min(best, (int)G.d[((size_t)nx * gy + ny) * gz + nz] + 1);
                            }
                    here = (uint8_t)std::min(best, 255);
                }
            }
        }
    };
    pass(+1);
    pass(-1);

    // leaf lists: start cells A with A - 0.5 <= hi and A + 1.5 >= lo (grown box, cell units)
    std::vector<uint32_t> count(gx * gy * gz, 0u);
    auto start_range = [&](uint32_t i, long a0[3], long a1[3]) {
        for (int a = 0; a < 3; ++a) {
            const double l = ((double)b.bounds_min[4 * (size_t)i + a] - margin - (double)G.origin[a]) *
                             (double)G.inv_cell;
            const double h = ((double)b.bounds_max[4 * (size_t)i + a] + margin - (double)G.origin[a]) *
                             (double)G.inv_cell;
            a0[a] = (long)std::max(0.0, std::ceil(l - 1.5));
            a1[a] = (long)std::min((double)(G.g[a] - 1), std::floor(h + 0.5));
            if (a0[a] > a1[a]) return false;
        }
        return true;
    };
    for (uint32_t i = 0; i < b.n_nodes; ++i) {
        if (b.nodes[4 * (size_t)i + 3] <= 0) continue;
        long a0[3], a1[3];
        if (!start_range(i, a0, a1)) continue;
        for (long x = a0[0]; x <= a1[0]; ++x)
            for (long y = a0[1]; y <= a1[1]; ++y)
                for (long z = a0[2]; z <= a1[2]; ++z) count[((size_t)x * gy + y) * gz + z] += 1u;
    }
    std::vector<uint32_t> offset(count.size(), 0u);
    size_t total = 1;                                        // unit 0: the empty list
    for (size_t k = 0; k < count.size(); ++k)
        if (count[k] > 0) {
            offset[k] = (uint32_t)std::min<size_t>(total, 0xFFFFFFFFu);
            // count word + ids in 16-byte units, plus the padding that the
            // device's reads of four ids at a time reach: ceil(count/4) + 1
            total += (count[k] + 3u) / 4u + 1u;
        }
    G.words.assign(count.size(), 0u);
    if (total <= (size_t)kNoLeafList) {
        G.lists.assign(4 * (total + 1), 0u);
        std::vector<uint32_t> fill(count.size(), 0u);
        for (uint32_t i = 0; i < b.n_nodes; ++i) {
            if (b.nodes[4 * (size_t)i + 3] <= 0) continue;
            long a0[3], a1[3];
            if (!start_range(i, a0, a1)) continue;
            for (long x = a0[0]; x <= a1[0]; ++x)
                for (long y = a0[1]; y <= a1[1]; ++y)
                    for (long z = a0[2]; z <= a1[2]; ++z) {
                        const size_t k = ((size_t)x * gy + y) * gz + z;
                        G.lists[4 * (size_t)offset[k] + 1 + fill[k]++] = i;
                    }
        }
        for (size_t k = 0; k < count.size(); ++k) {
            if (count[k] > 0) G.lists[4 * (size_t)offset[k]] = count[k];
            G.words[k] = (uint32_t)G.d[k] | (offset[k] << 8);
        }
    } else {
        G.lists.assign(4, 0u);
        for (size_t k = 0; k < count.size(); ++k) G.words[k] = (uint32_t)G.d[k] | ((uint32_t)kNoLeafList << 8);
    }
    return G;
}

inline float bits_f(uint32_t u)
{
    float f;
    std::memcpy(&f, &u, sizeof f);
    return f;
}

}  // namespace

cudaError_t upload_mesh(const BoundaryBvhHost& b, DomainDev* d, cudaStream_t stream)
{
    const uint32_t N = b.n_nodes, T = b.n_triangles;
    // skip index = node + size of its subtree (children follow their parent)
    std::vector<uint32_t> size(N, 1u);
    for (uint32_t i = N; i-- > 0;) {
        const int32_t* nd = b.nodes.data() + 4 * (size_t)i;
        if (nd[3] <= 0) size[i] = 1u + size[nd[0]] + size[nd[1]];
    }
    std::vector<float4> nodes(2 * (size_t)N), tris(3 * (size_t)T);
    for (uint32_t i = 0; i < N; ++i) {
        const int32_t* nd = b.nodes.data() + 4 * (size_t)i;
        const float* lo = b.bounds_min.data() + 4 * (size_t)i;
        const float* hi = b.bounds_max.data() + 4 * (size_t)i;
        const int32_t code = nd[3] > 0 ? (int32_t)(((uint32_t)nd[2] << 3) | (uint32_t)nd[3]) : -1;
        nodes[2 * (size_t)i] = make_float4(lo[0], lo[1], lo[2], bits_f(i + size[i]));
        nodes[2 * (size_t)i + 1] = make_float4(hi[0], hi[1], hi[2], bits_f((uint32_t)code));
    }
    for (uint32_t k = 0; k < T; ++k) {
        const uint32_t id = b.ordered[k];
        const uint32_t* ix = b.triangles4.data() + 4 * (size_t)id;
        const float* A = b.vertices4.data() + 4 * (size_t)ix[0];
        const float* B = b.vertices4.data() + 4 * (size_t)ix[1];
        const float* C = b.vertices4.data() + 4 * (size_t)ix[2];
        tris[3 * (size_t)k] = make_float4(A[0], A[1], A[2], bits_f(id));
        tris[3 * (size_t)k + 1] = make_float4(B[0] - A[0], B[1] - A[1], B[2] - A[2], 0.0f);
        tris[3 * (size_t)k + 2] = make_float4(C[0] - A[0], C[1] - A[1], C[2] - A[2], 0.0f);
    }
    const DistanceGrid G = distance_grid(b);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&d->nodes), nodes.size() * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d->tris), tris.size() * sizeof(float4));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d->cells), G.words.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&d->lists), G.lists.size() * sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d->nodes, nodes.data(), nodes.size() * sizeof(float4), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d->tris, tris.data(), tris.size() * sizeof(float4), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d->cells, G.words.data(), G.words.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d->lists, G.lists.data(), G.lists.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    d->kind = kDomainMesh;
    d->n_triangles = T;
    d->bytes = nodes.size() * sizeof(float4) + tris.size() * sizeof(float4) +
               (G.words.size() + G.lists.size()) * sizeof(uint32_t);
    MeshDev& m = d->mesh;
    m.nodes = d->nodes;
    m.tris = d->tris;
    m.cells = d->cells;
    m.lists = reinterpret_cast<const uint4*>(d->lists);
    m.n_nodes = N;
    m.gx = (float)G.g[0];
    m.gy = (float)G.g[1];
    m.gz = (float)G.g[2];
    m.ox = G.origin[0];
    m.oy = G.origin[1];
    m.oz = G.origin[2];
    m.inv_cell = G.inv_cell;
    d->nx = G.g[0];
    d->ny = G.g[1];
    d->nz = G.g[2];
    return cudaSuccess;
}

// ------------------------------------------------------------------ kernels

__global__ void __launch_bounds__(128) mesh_segment_hits_kernel(MeshDev m, const float4* __restrict__ starts,
                                                                const float4* __restrict__ ends, uint32_t n,
                                                                uint8_t* __restrict__ found,
                                                                uint32_t* __restrict__ triangle,
                                                                float4* __restrict__ hit)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 s = starts[i], e = ends[i];
    const Segment g = make_segment(s.x, s.y, s.z, e.x, e.y, e.z);
    float t, u = 0.0f, v = 0.0f;
    uint32_t tri;
    const bool h = mesh_walk<0>(m, g, t, tri, u, v) != 0u;
    found[i] = h ? 1 : 0;
    triangle[i] = tri;
    hit[i] = h ? make_float4(1.0f - u - v, u, v, t) : make_float4(0.0f, 0.0f, 0.0f, t);
}

__global__ void __launch_bounds__(128) mesh_contains_kernel(MeshDev m, const float4* __restrict__ points,
                                                            uint32_t n, uint32_t stride, uint8_t* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = points[(size_t)i * stride];
    out[i] = mesh_contains(m, p.x, p.y, p.z) ? 1 : 0;
}

__global__ void __launch_bounds__(128) mesh_segments_blocked_kernel(MeshDev m, const float4* __restrict__ starts,
                                                                    const float4* __restrict__ ends, uint32_t n,
                                                                    uint8_t* __restrict__ blocked)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 s = starts[i], e = ends[i];
    blocked[i] = mesh_segment_blocked(m, s.x, s.y, s.z, e.x, e.y, e.z) ? 1 : 0;
}

cudaError_t launch_mesh_segments_blocked(const MeshDev& m, const float4* starts, const float4* ends, uint32_t n,
                                         uint8_t* blocked, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    mesh_segments_blocked_kernel<<<(n + 127) / 128, 128, 0, stream>>>(m, starts, ends, n, blocked);
    return cudaGetLastError();
}

cudaError_t launch_mesh_segment_hits(const MeshDev& m, const float4* starts, const float4* ends, uint32_t n,
                                     uint8_t* found, uint32_t* triangle, float4* hit, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    mesh_segment_hits_kernel<<<(n + 127) / 128, 128, 0, stream>>>(m, starts, ends, n, found, triangle, hit);
    return cudaGetLastError();
}

cudaError_t launch_mesh_contains(const MeshDev& m, const float4* points, uint32_t n, uint8_t* out,
                                 cudaStream_t stream, uint32_t stride)
{
    if (n == 0) return cudaSuccess;
    mesh_contains_kernel<<<(n + 127) / 128, 128, 0, stream>>>(m, points, n, stride, out);
    return cudaGetLastError();
}

}  // namespace tg
