/*
 * tg_bvh.cuh -- closed-surface domain: BVH segment queries on the device.
 *
 * The BVH is the reference's boundary BVH (domain.py:72-116: median split
 * on the longest axis, leaves of at most 4 triangles, nodes in preorder)
 * and the per-node and per-triangle tests are those of utils/bvh.cl:16-80
 * in the same binary32 operations.  Two things differ in form, not in
 * result:
 *
 *   - no stack.  bvh.cl:83-131 walks the tree depth first with a 64-entry
 *     stack, left child first.  Because nodes are numbered in preorder, the
 *     left child of node i is i + 1 and the node visited after i's subtree
 *     is i + size(subtree(i)), stored per node as its "skip" index.  The walk
 *     below (descend to i + 1 on a box hit, else jump to skip) visits the
 *     same nodes in the same order with the same running closest t, so the
 *     hit, its triangle and barycentric coordinates are identical, with no
 *     per-lane stack in local memory.  (The reference's stack only overflows
 *     past depth 62; the host build rejects such trees.)
 *
 *   - a distance grid in front of the walk for tracking.  Each cell holds
 *     the Chebyshev distance, in cells, to the nearest cell that a leaf box
 *     (grown by a rounding margin) touches.  When both ends of a segment lie
 *     in cells closer to each other than that distance, the segment lies in
 *     an axis-aligned box of empty cells that is separated from every leaf
 *     box along some axis by more than the rounding of the slab test, so
 *     every leaf slab test fails and the walk would find nothing: the walk is
 *     skipped.  Near the surface each cell also lists the leaves whose grown
 *     box meets its half-cell neighbourhood; a short segment starting in the
 *     cell tests those leaves (independent loads) instead of walking ~2 x
 *     depth dependent nodes.  The result is the walk's result in every case
 *     (mesh_segment_blocked gives the argument).
 *
 * Layout (built on the host, tg_mesh.cu):
 *   nodes  2 float4 per node: (min.xyz, skip as uint bits), (max.xyz, leaf
 *          code as int bits: -1 internal, else first << 3 | count)
 *   tris   3 float4 per leaf slot: (a.xyz, triangle id bits), (b - a, 0),
 *          (c - a, 0), the edge vectors rounded exactly as bvh.cl:59-60
 *          rounds them
 */
#ifndef TG_BVH_CUH
#define TG_BVH_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "tg_device.cuh"

namespace tg {

constexpr int kDomainImage = 0;
constexpr int kDomainMesh = 1;

// Cell word: distance (low 8 bits) | leaf list offset in 16-byte units.
constexpr uint32_t kNoLeafList = 0xFFFFFFu;

struct MeshDev {
    const float4* nodes;
    const float4* tris;
    const uint32_t* cells;   // per grid cell: distance | leaf list offset << 8
    const uint4* lists;      // leaf lists: count, then leaf node indices
    uint32_t n_nodes;
    float gx, gy, gz;        // grid cells per axis
    float ox, oy, oz;        // grid origin
    float inv_cell;          // 1 / cell edge
};

// Three fixed directions of the inside test (unit length to float
// precision, off every coordinate plane and diagonal).
__host__ __device__ __forceinline__ void mesh_ray(int r, float& x, float& y, float& z)
{
    x = r == 0 ? 0.53896236f : (r == 1 ? -0.68169260f : 0.17420970f);
    y = r == 0 ? 0.77412713f : (r == 1 ? 0.22392839f : -0.54785200f);
    z = r == 0 ? 0.33221170f : (r == 1 ? 0.69653570f : 0.81824590f);
}

// One segment start + t * d, t in [0, 1], with the per-axis reciprocals
// bvh.cl:32 recomputes per node (same IEEE division, same value).
struct Segment {
    float sx, sy, sz;
    float dx, dy, dz;
    float ix, iy, iz;
    bool px, py, pz;         // |d| < 1e-12 on that axis (bvh.cl:29)
};

__device__ __forceinline__ Segment make_segment(float sx, float sy, float sz, float ex, float ey, float ez)
{
    Segment g;
    g.sx = sx; g.sy = sy; g.sz = sz;
    g.dx = ex - sx; g.dy = ey - sy; g.dz = ez - sz;
    g.px = fabsf(g.dx) < 1e-12f;
    g.py = fabsf(g.dy) < 1e-12f;
    g.pz = fabsf(g.dz) < 1e-12f;
    g.ix = 1.0f / g.dx;
    g.iy = 1.0f / g.dy;
    g.iz = 1.0f / g.dz;
    return g;
}

// OpenCL float min(): y if y < x else x (cl_max is in tg_device.cuh).
__device__ __forceinline__ float cl_min(float x, float y) { return (y < x) ? y : x; }

// bvh.cl:16-45 for one axis; false when the slab interval empties.
__device__ __forceinline__ bool slab(bool parallel, float s, float inv, float lo, float hi, float& t0, float& t1)
{
    if (parallel) return !(s < lo || s > hi);
    float a = (lo - s) * inv;
    float b = (hi - s) * inv;
    if (a > b) {
        const float c = a;
        a = b;
        b = c;
    }
    t0 = cl_max(t0, a);
    t1 = cl_min(t1, b);
    return !(t0 > t1);
}

__device__ __forceinline__ bool box_hit(const Segment& g, float4 lo, float4 hi, float max_t)
{
    float t0 = 0.0f, t1 = max_t;
    if (!slab(g.px, g.sx, g.ix, lo.x, hi.x, t0, t1)) return false;
    if (!slab(g.py, g.sy, g.iy, lo.y, hi.y, t0, t1)) return false;
    return slab(g.pz, g.sz, g.iz, lo.z, hi.z, t0, t1);
}

// bvh.cl:47-80 (Moller-Trumbore, the reference's tolerances).
__device__ __forceinline__ bool triangle_hit(const Segment& g, const float4* tri, float max_t, float& t_out,
                                             float& u_out, float& v_out)
{
    const float4 a = __ldg(tri);
    const float4 e1 = __ldg(tri + 1);
    const float4 e2 = __ldg(tri + 2);
    // p = cross(direction, edge2)
    const float px = g.dy * e2.z - g.dz * e2.y;
    const float py = g.dz * e2.x - g.dx * e2.z;
    const float pz = g.dx * e2.y - g.dy * e2.x;
    const float det = e1.x * px + e1.y * py + e1.z * pz;
    if (fabsf(det) < 1e-10f) return false;
    const float inv_det = 1.0f / det;
    const float ox = g.sx - a.x, oy = g.sy - a.y, oz = g.sz - a.z;
    const float u = (ox * px + oy * py + oz * pz) * inv_det;
    if (u < -1e-6f || u > 1.0f + 1e-6f) return false;
    // q = cross(offset, edge1)
    const float qx = oy * e1.z - oz * e1.y;
    const float qy = oz * e1.x - ox * e1.z;
    const float qz = ox * e1.y - oy * e1.x;
    const float v = (g.dx * qx + g.dy * qy + g.dz * qz) * inv_det;
    if (v < -1e-6f || u + v > 1.0f + 1e-6f) return false;
    const float t = (e2.x * qx + e2.y * qy + e2.z * qz) * inv_det;
    if (t <= 1e-6f || t > max_t) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    return true;
}

// MODE 0: closest hit (bvh.cl:83-131); 1: any hit, stop at the first;
// 2: count every hit with max_t fixed at 1.
template <int MODE>
__device__ __forceinline__ uint32_t mesh_walk(const MeshDev& m, const Segment& g, float& t, uint32_t& tri,
                                              float& u, float& v)
{
    t = 1.0f;
    tri = 0u;
    uint32_t hits = 0u;
    uint32_t i = 0u;
    while (i < m.n_nodes) {
        const float4 lo = __ldg(m.nodes + 2 * (size_t)i);
        const float4 hi = __ldg(m.nodes + 2 * (size_t)i + 1);
        const uint32_t skip = __float_as_uint(lo.w);
        if (!box_hit(g, lo, hi, MODE == 2 ? 1.0f : t)) {
            i = skip;
            continue;
        }
        const int code = __float_as_int(hi.w);
        if (code < 0) {
            i = i + 1u;
            continue;
        }
        const uint32_t first = (uint32_t)code >> 3;
        const uint32_t count = (uint32_t)code & 7u;
        for (uint32_t k = 0; k < count; ++k) {
            const float4* tp = m.tris + 3 * (size_t)(first + k);
            float tt, uu, vv;
            if (triangle_hit(g, tp, MODE == 2 ? 1.0f : t, tt, uu, vv)) {
                hits += 1u;
                if (MODE == 0) {
                    t = tt;
                    u = uu;
                    v = vv;
                    tri = __float_as_uint(__ldg(tp).w);
                } else if (MODE == 1) {
                    return 1u;
                }
            }
        }
        i = skip;
    }
    return hits;
}

// Inside test: majority over three rays of the parity of crossings; points
// outside the root bounds are outside.
__device__ __forceinline__ bool mesh_contains(const MeshDev& m, float x, float y, float z)
{
    const float4 lo = __ldg(m.nodes);
    const float4 hi = __ldg(m.nodes + 1);
    if (!(x >= lo.x && x <= hi.x && y >= lo.y && y <= hi.y && z >= lo.z && z <= hi.z)) return false;
    const float reach = (((hi.x - lo.x) + (hi.y - lo.y)) + (hi.z - lo.z)) + 1.0f;
    int odd = 0;
#pragma unroll 1
    for (int r = 0; r < 3; ++r) {
        float rx, ry, rz;
        mesh_ray(r, rx, ry, rz);
        const Segment g = make_segment(x, y, z, x + reach * rx, y + reach * ry, z + reach * rz);
        float t, u, v;
        uint32_t tri;
        odd += (int)(mesh_walk<2>(m, g, t, tri, u, v) & 1u);
    }
    return odd >= 2;
}

// Any hit among the leaves of one cell's list (count, then leaf node
// indices), with max_t = 1 as in the walk's any-hit mode.  The boxes of
// kLeafBatch leaves are fetched before they are tested (more in flight
// costs registers that the tracking kernels do not have).
constexpr int kLeafBatch = 2;

__device__ __forceinline__ bool mesh_leaves_hit(const MeshDev& m, const Segment& g, const uint4* list)
{
    const uint32_t* ids = reinterpret_cast<const uint32_t*>(list);
    const uint32_t count = __ldg(ids);
#pragma unroll 1
    for (uint32_t k = 1; k <= count; k += kLeafBatch) {
        float4 lo[kLeafBatch], hi[kLeafBatch];
#pragma unroll
        for (int q = 0; q < kLeafBatch; ++q) {
            // ids past the count are the list's zero padding (node 0, not tested)
            const uint32_t leaf = __ldg(ids + k + q);
            lo[q] = __ldg(m.nodes + 2 * (size_t)leaf);
            hi[q] = __ldg(m.nodes + 2 * (size_t)leaf + 1);
        }
#pragma unroll
        for (int q = 0; q < kLeafBatch; ++q) {
            if (k + (uint32_t)q > count || !box_hit(g, lo[q], hi[q], 1.0f)) continue;
            const int code = __float_as_int(hi[q].w);
            const uint32_t first = (uint32_t)code >> 3;
            const uint32_t n = (uint32_t)code & 7u;
            for (uint32_t j = 0; j < n; ++j) {
                float tt, uu, vv;
                if (triangle_hit(g, m.tris + 3 * (size_t)(first + j), 1.0f, tt, uu, vv)) return true;
            }
        }
    }
    return false;
}

// True when the segment from the last point to the current one hits the
// surface (the found flag of bvh.cl:83-131).  Three routes, one result:
//   - both ends in cells nearer each other than the start cell's distance:
//     no leaf box test can pass, nothing is hit;
//   - both ends inside the start cell's half-cell neighbourhood (with a
//     0.01-cell allowance for the rounding of the cell coordinates): the
//     cell's leaf list holds every leaf whose box test can pass.  Rounding
//     is monotonic, so an ancestor's slab interval contains its leaf's and
//     an ancestor passes whenever one of its leaves does; the walk therefore
//     reaches a leaf exactly when the leaf's own box test passes, and the
//     any-hit over the list equals the walk's;
//   - otherwise the any-hit walk from the root.
// Which route decides a segment: 0 the distance grid (nothing can be hit),
// 1 the start cell's leaf list (its offset in `list`), 2 the walk.
__device__ __forceinline__ int mesh_route(const MeshDev& m, float sx, float sy, float sz, float ex, float ey,
                                          float ez, uint32_t& list)
{
    const float usx = (sx - m.ox) * m.inv_cell, usy = (sy - m.oy) * m.inv_cell, usz = (sz - m.oz) * m.inv_cell;
    const float uex = (ex - m.ox) * m.inv_cell, uey = (ey - m.oy) * m.inv_cell, uez = (ez - m.oz) * m.inv_cell;
    const float ax = floorf(usx), ay = floorf(usy), az = floorf(usz);
    const float bx = floorf(uex), by = floorf(uey), bz = floorf(uez);
    if (ax >= 0.0f && ax < m.gx && ay >= 0.0f && ay < m.gy && az >= 0.0f && az < m.gz && bx >= 0.0f &&
        bx < m.gx && by >= 0.0f && by < m.gy && bz >= 0.0f && bz < m.gz) {
        const size_t cell = ((size_t)ax * (size_t)m.gy + (size_t)ay) * (size_t)m.gz + (size_t)az;
        const uint32_t word = __ldg(m.cells + cell);
        const float reach = (float)(word & 255u);
        const float cheb = fmaxf(fmaxf(fabsf(bx - ax), fabsf(by - ay)), fabsf(bz - az));
        if (cheb < reach) return 0;
        list = word >> 8;
        const float lo = -0.49f, hi = 1.49f;
        if (list != kNoLeafList && uex - ax >= lo && uex - ax <= hi && uey - ay >= lo && uey - ay <= hi &&
            uez - az >= lo && uez - az <= hi)
            return 1;
    }
    return 2;
}

__device__ __forceinline__ bool mesh_segment_blocked(const MeshDev& m, float sx, float sy, float sz, float ex,
                                                     float ey, float ez)
{
    uint32_t list = 0;
    const int route = mesh_route(m, sx, sy, sz, ex, ey, ez, list);
    if (route == 0) return false;
    const Segment g = make_segment(sx, sy, sz, ex, ey, ez);
    if (route == 1) return mesh_leaves_hit(m, g, m.lists + list);
    float t, u, v;
    uint32_t tri;
    return mesh_walk<1>(m, g, t, tri, u, v) != 0u;
}

// The leaf-list route for a whole warp at once.  Called by all 32 lanes
// together; lanes with `need` set have a segment g and a leaf list.  The
// warp's (lane, leaf) pairs are dealt to its lanes, one pair per lane per
// round -- the owner's segment comes by shuffle -- so a few lanes near the
// surface no longer run their lists one after the other while the rest of
// the warp waits.  Any-hit is independent of the order of the tests, so
// each lane's answer is the one mesh_leaves_hit gives.
__device__ __forceinline__ bool warp_leaves_hit(const MeshDev& m, bool need, const Segment& g, uint32_t list)
{
    constexpr unsigned kFull = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t count = need ? __ldg(reinterpret_cast<const uint32_t*>(m.lists + list)) : 0u;
    uint32_t incl = count;
#pragma unroll
    for (uint32_t o = 1; o < 32u; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    const uint32_t flags = (g.px ? 1u : 0u) | (g.py ? 2u : 0u) | (g.pz ? 4u : 0u);
    unsigned hits = 0u;
    for (uint32_t base = 0; base < total; base += 32u) {
        const uint32_t w = base + lane;
        // owner: the first lane whose inclusive count exceeds w
        uint32_t owner = 0;
#pragma unroll
        for (uint32_t step = 16; step > 0u; step >>= 1) {
            const uint32_t v = __shfl_sync(kFull, incl, owner + step - 1u);
            if (v <= w) owner += step;
        }
        const uint32_t first = __shfl_sync(kFull, incl, owner) - __shfl_sync(kFull, count, owner);
        Segment o;
        o.sx = __shfl_sync(kFull, g.sx, owner);
        o.sy = __shfl_sync(kFull, g.sy, owner);
        o.sz = __shfl_sync(kFull, g.sz, owner);
        o.dx = __shfl_sync(kFull, g.dx, owner);
        o.dy = __shfl_sync(kFull, g.dy, owner);
        o.dz = __shfl_sync(kFull, g.dz, owner);
        o.ix = __shfl_sync(kFull, g.ix, owner);
        o.iy = __shfl_sync(kFull, g.iy, owner);
        o.iz = __shfl_sync(kFull, g.iz, owner);
        const uint32_t of = __shfl_sync(kFull, flags, owner);
        o.px = (of & 1u) != 0u;
        o.py = (of & 2u) != 0u;
        o.pz = (of & 4u) != 0u;
        const uint32_t olist = __shfl_sync(kFull, list, owner);
        bool h = false;
        if (w < total) {
            const uint32_t leaf = __ldg(reinterpret_cast<const uint32_t*>(m.lists + olist) + 1u + (w - first));
            const float4 lo = __ldg(m.nodes + 2 * (size_t)leaf);
            const float4 hi = __ldg(m.nodes + 2 * (size_t)leaf + 1);
            if (box_hit(o, lo, hi, 1.0f)) {
                const int code = __float_as_int(hi.w);
                const uint32_t tfirst = (uint32_t)code >> 3;
                const uint32_t tn = (uint32_t)code & 7u;
                for (uint32_t j = 0; j < tn && !h; ++j) {
                    float tt, uu, vv;
                    h = triangle_hit(o, m.tris + 3 * (size_t)(tfirst + j), 1.0f, tt, uu, vv);
                }
            }
        }
        hits |= __reduce_or_sync(kFull, h ? (1u << owner) : 0u);
    }
    return need && ((hits >> lane) & 1u) != 0u;
}

}  // namespace tg

#endif  // TG_BVH_CUH
