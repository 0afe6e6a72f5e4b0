// bvh_build.cu - on-GPU BVH construction for the hdcx tracer.
//
// Replaces the closed driver build behind vkCmdBuildAccelerationStructuresKHR
// (src/gpu/vulkan_path_tracer.cpp:3032-3127: one BLAS over all flattened
// triangles, one identity TLAS). Steps, all on the device:
//   1. triangle boxes and the scene box;
//   2. 63-bit Morton codes of the box centres, sorted with their triangle ids;
//   3. a binary tree by PLOC agglomerative clustering in Morton order, with
//      node boxes and triangle counts, and, round by round, the SAH costs of
//      its optimal collapse into 8-wide nodes (collapseCostKernel);
//   4. a top-down collapse into 8-wide nodes along those costs: each wide
//      node takes the children (subtrees or leaves of up to three triangles)
//      of its lowest-cost distribution over eight slots; children take the
//      octant slot their centre points to, so traversal visits them nearest
//      first; child boxes are quantised to 8 bits per plane against a
//      power-of-two step, padded by one step on every side; leaf triangles are
//      copied in leaf order.
#include "bvh_build.h"
#include "device_memory.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

namespace hdcx {
namespace {

constexpr int kMaxLeafTriangles = 3;
constexpr int kMaxDepth = 64;
constexpr int kBlock = 256;

#define CUDA_OK(expr)                                                                               \
    do {                                                                                            \
        cudaError_t err__ = (expr);                                                                 \
        if (err__ != cudaSuccess) throw std::runtime_error(std::string("BVH build: ") + #expr + ": " + \
                                                           cudaGetErrorString(err__));              \
    } while (0)

struct Box {
    float3 lo;
    float3 hi;
};

__device__ __forceinline__ uint32_t floatToOrdered(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedToFloat(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void triangleBoxesKernel(const float4* vertices, const uint32_t* indices, uint32_t n, float4* boxLo,
                                    float4* boxHi, uint32_t* sceneBounds)
{
    __shared__ uint32_t sb[6];
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const float4 a = vertices[indices[3 * i + 0]];
        const float4 b = vertices[indices[3 * i + 1]];
        const float4 c = vertices[indices[3 * i + 2]];
        const float3 lo = make_float3(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)));
        const float3 hi = make_float3(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)));
        boxLo[i] = make_float4(lo.x, lo.y, lo.z, 0.0f);
        boxHi[i] = make_float4(hi.x, hi.y, hi.z, 0.0f);
        // Scene bounds of the box centres (for the Morton grid).
        const float cx = 0.5f * (lo.x + hi.x), cy = 0.5f * (lo.y + hi.y), cz = 0.5f * (lo.z + hi.z);
        atomicMin(&sb[0], floatToOrdered(cx));
        atomicMin(&sb[1], floatToOrdered(cy));
        atomicMin(&sb[2], floatToOrdered(cz));
        atomicMax(&sb[3], floatToOrdered(cx));
        atomicMax(&sb[4], floatToOrdered(cy));
        atomicMax(&sb[5], floatToOrdered(cz));
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&sceneBounds[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&sceneBounds[threadIdx.x], sb[threadIdx.x]);
}

__device__ __forceinline__ uint64_t spreadBits21(uint64_t v)
{
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void mortonKernel(const float4* boxLo, const float4* boxHi, uint32_t n, const uint32_t* sceneBounds,
                             uint64_t* keys, uint32_t* ids)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 lo = make_float3(orderedToFloat(sceneBounds[0]), orderedToFloat(sceneBounds[1]), orderedToFloat(sceneBounds[2]));
    const float3 hi = make_float3(orderedToFloat(sceneBounds[3]), orderedToFloat(sceneBounds[4]), orderedToFloat(sceneBounds[5]));
    const float4 a = boxLo[i], b = boxHi[i];
    const float c[3] = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)};
    const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) {
        const float extent = h[k] - l[k];
        float u = extent > 0.0f ? (c[k] - l[k]) / extent : 0.5f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        q[k] = static_cast<uint64_t>(fminf(u * 2097152.0f, 2097151.0f));
    }
    keys[i] = (spreadBits21(q[0]) << 2) | (spreadBits21(q[1]) << 1) | spreadBits21(q[2]);
    ids[i] = i;
}

// ---------------------------------------------------------------------------
// Binary tree: PLOC (Meister and Bittner, "Parallel Locally-Ordered Clustering
// for Bounding Volume Hierarchy Construction", IEEE TVCG 2018). Clusters stay
// in Morton order; each pass every cluster finds the neighbour within
// +-kSearchRadius positions whose merged box has the smallest surface area,
// mutual nearest neighbours merge into a new internal node, and the cluster
// list is compacted, until one cluster (the root) is left. Candidates of equal
// area are ordered by their index pair, so the globally best pair is always
// mutual and every pass makes progress.
// Binary node ids: internal 0..n-2 (in merge order), leaf k -> (n-1)+k.
// nodeLo.w holds the subtree's triangle count.
// ---------------------------------------------------------------------------
// 16 measured against 32 and 64: the wider searches changed the heavy scene
// by +1% and -2% and cost the spectral-stress scene 4-5% (more nodes and
// triangles per ray after the collapse).
#ifndef HDCX_PLOC_RADIUS
#define HDCX_PLOC_RADIUS 16
#endif
constexpr int kSearchRadius = HDCX_PLOC_RADIUS;

__global__ void initLeavesKernel(int n, const uint32_t* sortedIds, const float4* triLo, const float4* triHi,
                                 float4* nodeLo, float4* nodeHi, int* clusters)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t prim = sortedIds[k];
    float4 lo = triLo[prim];
    lo.w = 1.0f;
    nodeLo[(n - 1) + k] = lo;
    nodeHi[(n - 1) + k] = triHi[prim];
    clusters[k] = (n - 1) + k;
}

__device__ __forceinline__ float mergedArea(float4 la, float4 ha, float4 lb, float4 hb)
{
    const float dx = fmaxf(ha.x, hb.x) - fminf(la.x, lb.x);
    const float dy = fmaxf(ha.y, hb.y) - fminf(la.y, lb.y);
    const float dz = fmaxf(ha.z, hb.z) - fminf(la.z, lb.z);
    return dx * dy + dy * dz + dz * dx;
}

__global__ void nearestNeighbourKernel(const int* clusters, int m, const float4* nodeLo, const float4* nodeHi, int* nn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int ci = clusters[i];
    const float4 li = nodeLo[ci], hi = nodeHi[ci];
    float best = 3.4e38f;
    int bestJ = -1;
    const int j0 = max(0, i - kSearchRadius), j1 = min(m - 1, i + kSearchRadius);
    for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const int cj = clusters[j];
        const float a = mergedArea(li, hi, nodeLo[cj], nodeHi[cj]);
        // Candidates are visited in increasing j, so the first of equal areas
        // is the one with the smallest (min(i,j), max(i,j)) pair.
        if (a < best || bestJ < 0) {
            best = a;
            bestJ = j;
        }
    }
    nn[i] = bestJ;
}

__global__ void mergeKernel(const int* clusters, int m, const int* nn, int* left, int* right, float4* nodeLo,
                            float4* nodeHi, uint32_t* nodeCounter, int* merged, int* keep)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    if (mutual && i > j) {
        keep[i] = 0;  // merged by its partner
        return;
    }
    keep[i] = 1;
    if (!mutual) {
        merged[i] = clusters[i];
        return;
    }
    const int a = clusters[i], b = clusters[j];
    const int k = static_cast<int>(atomicAdd(nodeCounter, 1u));
    const float4 la = nodeLo[a], lb = nodeLo[b], ha = nodeHi[a], hb = nodeHi[b];
    left[k] = a;
    right[k] = b;
    nodeLo[k] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), la.w + lb.w);
    nodeHi[k] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.0f);
    merged[i] = k;
}

struct CollapseItem {
    int binaryNode;
    uint32_t wideIndex;
    uint32_t depth;
    uint32_t pad;
};

__device__ __forceinline__ float surfaceArea(float4 lo, float4 hi)
{
    const float dx = fmaxf(hi.x - lo.x, 0.0f), dy = fmaxf(hi.y - lo.y, 0.0f), dz = fmaxf(hi.z - lo.z, 0.0f);
    return dx * dy + dy * dz + dz * dx;
}

// ---------------------------------------------------------------------------
// Optimal collapse of the binary tree into 8-wide nodes (Ylitie, Karras and
// Laine, HPG 2017, sec. 3.1). For every binary node n and i = 1..7, C(n, i)
// is the lowest SAH cost of representing n's subtree as at most i children
// of a wide node:
//   C(n, 1) = min(leaf: A(n) * p(n) * cPrim if p(n) <= 3 triangles,
//                 internal: A(n) * cNode + D(n, 8))
//   C(n, i) = min(C(n, i - 1), D(n, i))                       for i > 1
//   D(n, j) = min over 0 < k < j of C(left, k) + C(right, j - k)
// with A the box's surface area and p the triangle count; a binary leaf is
// one triangle, A * cPrim for every i. The costs are filled bottom up (the
// internal nodes of a clustering round only have children from earlier
// rounds) and read top down by collapseKernel, which gives each wide node
// the children D(n, 8) chose. cPrim = cNode was measured best among 0.3, 0.6
// and 1.0 on the heavy and stress scenes (a wide-node test is some 200
// instructions and a triangle test 80, but a triangle also costs three
// 16-byte loads, the closest-hit bookkeeping and, for cutouts, an opacity
// lookup).
// decision[8 n + i - 1] for i = 1..7: C(n, 1): 0 leaf, 1 internal; i > 1:
// 0 take C(n, i - 1), else the k of D(n, i); decision[8 n + 7]: the k of D(n, 8).
// ---------------------------------------------------------------------------
#ifndef HDCX_COLLAPSE_PRIM_COST
#define HDCX_COLLAPSE_PRIM_COST 1.0f
#endif
constexpr float kCollapseNodeCost = 1.0f;
constexpr float kCollapsePrimCost = HDCX_COLLAPSE_PRIM_COST;

__global__ void collapseCostKernel(int n, const int* left, const int* right, const float4* nodeLo, const float4* nodeHi,
                                   uint32_t first, uint32_t last, float* cost, uint8_t* decision)
{
    const uint32_t node = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= last) return;
    const int leafBase = n - 1;
    float cl[8], cr[8];  // C(child, i) at index i = 1..7
    auto load = [&](int b, float* c) {
        if (b >= leafBase) {
            const float v = kCollapsePrimCost * surfaceArea(nodeLo[b], nodeHi[b]);
            for (int i = 1; i < 8; ++i) c[i] = v;
        } else {
            for (int i = 1; i < 8; ++i) c[i] = cost[7 * static_cast<size_t>(b) + (i - 1)];
        }
    };
    load(left[node], cl);
    load(right[node], cr);
    float dist[9];
    uint8_t split[9];
    for (int j = 2; j <= 8; ++j) {
        dist[j] = INFINITY;
        split[j] = 1;
        for (int k = 1; k < j; ++k) {
            const float v = cl[k] + cr[j - k];
            if (v < dist[j]) {
                dist[j] = v;
                split[j] = static_cast<uint8_t>(k);
            }
        }
    }
    const float area = surfaceArea(nodeLo[node], nodeHi[node]);
    const int count = static_cast<int>(nodeLo[node].w);
    const float internal = kCollapseNodeCost * area + dist[8];
    const float leaf = count <= kMaxLeafTriangles ? kCollapsePrimCost * area * static_cast<float>(count) : INFINITY;
    float* c = cost + 7 * static_cast<size_t>(node);
    uint8_t* d = decision + 8 * static_cast<size_t>(node);
    float previous = fminf(leaf, internal);
    c[0] = previous;
    d[0] = leaf <= internal ? 0u : 1u;
    for (int i = 2; i <= 7; ++i) {
        if (previous <= dist[i]) {
            d[i - 1] = 0u;
        } else {
            previous = dist[i];
            d[i - 1] = split[i];
        }
        c[i - 1] = previous;
    }
    d[7] = split[8];
}

__device__ __forceinline__ int ceilLog2Double(double x)
{
    int e;
    const double m = frexp(x, &e);  // x = m * 2^e, m in [0.5, 1)
    return m == 0.5 ? e - 1 : e;
}

// Quantisation frame of a wide node whose children span [lo, hi]: per axis a
// power-of-two step (at least the box extent / 252 and the floor
// max(|coordinate|, sceneScale) / 65536) and an origin one step below lo,
// rounded down. Shared by the build and the refit, so both quantise alike.
__device__ void nodeFrame(float4 lo, float4 hi, float sceneScale, float origin[3], double step[3], uint8_t biased[3])
{
    const float l3[3] = {lo.x, lo.y, lo.z}, h3[3] = {hi.x, hi.y, hi.z};
    for (int k = 0; k < 3; ++k) {
        const double extent = static_cast<double>(h3[k]) - static_cast<double>(l3[k]);
        const double floorStep = fmax(fmax(fabs(static_cast<double>(l3[k])), fabs(static_cast<double>(h3[k]))),
                                      static_cast<double>(sceneScale)) * (1.0 / 65536.0);
        double q = fmax(fmax(extent / 252.0, floorStep), 1e-30);
        int e = ceilLog2Double(q);
        e = max(-126, min(127, e));
        step[k] = ldexp(1.0, e);
        biased[k] = static_cast<uint8_t>(e + 127);
        origin[k] = __double2float_rd(static_cast<double>(l3[k]) - step[k]);
    }
}

// A child box [cl, ch] on the node's grid, padded by one step on every side.
__device__ void quantizeChild(float4 cl, float4 ch, const float origin[3], const double step[3], uint8_t ql[3],
                              uint8_t qh[3])
{
    const float cl3[3] = {cl.x, cl.y, cl.z}, ch3[3] = {ch.x, ch.y, ch.z};
    for (int k = 0; k < 3; ++k) {
        const double lo_q = floor((static_cast<double>(cl3[k]) - origin[k]) / step[k]) - 1.0;
        const double hi_q = ceil((static_cast<double>(ch3[k]) - origin[k]) / step[k]) + 1.0;
        ql[k] = static_cast<uint8_t>(fmin(fmax(lo_q, 0.0), 255.0));
        qh[k] = static_cast<uint8_t>(fmin(fmax(hi_q, 0.0), 255.0));
    }
}

struct CollapseArgs {
    int n;
    const int* left;
    const int* right;
    const float4* nodeLo;
    const float4* nodeHi;
    const uint32_t* sortedIds;
    const uint32_t* primIds;  // null: a triangle's id is its position in the input list
    const float* opacityHint;  // null: -1 (no hint) in every leaf copy
    const float4* vertices;
    const uint32_t* indices;
    float sceneScale;  // max |coordinate| and scene extent, for the padding floor
    const uint8_t* decision;  // collapseCostKernel's choices, 8 per internal binary node
    WideNode* wide;
    float4* triVerts;
    uint32_t* wideCounter;
    uint32_t* triCounter;
    uint32_t* errorFlag;
};

__global__ void collapseKernel(CollapseArgs a, const CollapseItem* items, uint32_t itemCount, CollapseItem* nextItems,
                               uint32_t* nextCount)
{
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= itemCount) return;
    const CollapseItem item = items[w];
    const int leafBase = a.n - 1;
    auto isLeaf = [&](int b) { return b >= leafBase; };
    auto count = [&](int b) { return static_cast<int>(a.nodeLo[b].w); };

    // A binary node becomes an internal child (a wide node of its own) when
    // its optimal single-slot form is internal, else a leaf of <= 3 triangles.
    auto isInternal = [&](int b) { return !isLeaf(b) && a.decision[8 * static_cast<size_t>(b)] != 0u; };

    // The children of this wide node: D(node, 8) unfolded, each binary node
    // given j slots taking C(node, j)'s choice (fewer slots, or a split).
    int entries[8];
    int m = 0;
    if (isLeaf(item.binaryNode)) {
        entries[m++] = item.binaryNode;
    } else {
        int pendingNode[16], pendingSlots[16];
        int sp = 0;
        const int k8 = a.decision[8 * static_cast<size_t>(item.binaryNode) + 7];
        pendingNode[sp] = a.right[item.binaryNode];
        pendingSlots[sp++] = 8 - k8;
        pendingNode[sp] = a.left[item.binaryNode];
        pendingSlots[sp++] = k8;
        while (sp > 0 && m < 8) {
            --sp;
            const int b = pendingNode[sp];
            int j = pendingSlots[sp];
            if (isLeaf(b)) {
                entries[m++] = b;
                continue;
            }
            const uint8_t* d = a.decision + 8 * static_cast<size_t>(b);
            while (j > 1 && d[j - 1] == 0u) --j;
            if (j <= 1) {
                entries[m++] = b;
                continue;
            }
            const int k = d[j - 1];
            pendingNode[sp] = a.right[b];
            pendingSlots[sp++] = j - k;
            pendingNode[sp] = a.left[b];
            pendingSlots[sp++] = k;
        }
    }

    // Node box and octant slot assignment.
    float4 lo = a.nodeLo[entries[0]], hi = a.nodeHi[entries[0]];
    for (int i = 1; i < m; ++i) {
        const float4 l = a.nodeLo[entries[i]], h = a.nodeHi[entries[i]];
        lo = make_float4(fminf(lo.x, l.x), fminf(lo.y, l.y), fminf(lo.z, l.z), 0.0f);
        hi = make_float4(fmaxf(hi.x, h.x), fmaxf(hi.y, h.y), fmaxf(hi.z, h.z), 0.0f);
    }
    const float cx = 0.5f * (lo.x + hi.x), cy = 0.5f * (lo.y + hi.y), cz = 0.5f * (lo.z + hi.z);
    int slotOf[8];
    int entryOfSlot[8];
    for (int i = 0; i < 8; ++i) { slotOf[i] = -1; entryOfSlot[i] = -1; }
    for (int round = 0; round < m; ++round) {
        float bestScore = -3.4e38f;
        int be = -1, bs = -1;
        for (int i = 0; i < m; ++i) {
            if (slotOf[i] >= 0) continue;
            const float4 l = a.nodeLo[entries[i]], h = a.nodeHi[entries[i]];
            const float vx = 0.5f * (l.x + h.x) - cx, vy = 0.5f * (l.y + h.y) - cy, vz = 0.5f * (l.z + h.z) - cz;
            for (int s = 0; s < 8; ++s) {
                if (entryOfSlot[s] >= 0) continue;
                const float score = ((s & 1) ? vx : -vx) + ((s & 2) ? vy : -vy) + ((s & 4) ? vz : -vz);
                if (score > bestScore) { bestScore = score; be = i; bs = s; }
            }
        }
        if (be < 0) {  // non-finite boxes: first free entry into the first free slot
            for (int i = 0; i < m && be < 0; ++i) if (slotOf[i] < 0) be = i;
            for (int q = 0; q < 8 && bs < 0; ++q) if (entryOfSlot[q] < 0) bs = q;
        }
        slotOf[be] = bs;
        entryOfSlot[bs] = be;
    }

    // Quantisation grid per axis.
    float origin[3];
    double step[3];
    uint8_t biased[3];
    nodeFrame(lo, hi, a.sceneScale, origin, step, biased);

    // Allocate internal children and leaf triangles.
    int internalCount = 0, triangleCount = 0;
    for (int s = 0; s < 8; ++s) {
        const int i = entryOfSlot[s];
        if (i < 0) continue;
        const int b = entries[i];
        if (isInternal(b)) internalCount++;
        else triangleCount += isLeaf(b) ? 1 : count(b);
    }
    const uint32_t childBase = internalCount ? atomicAdd(a.wideCounter, static_cast<uint32_t>(internalCount)) : 0u;
    const uint32_t triBase = triangleCount ? atomicAdd(a.triCounter, static_cast<uint32_t>(triangleCount)) : 0u;
    if (item.depth + 1 >= kMaxDepth && internalCount) atomicOr(a.errorFlag, 1u);

    WideNode node;
    node.px = origin[0];
    node.py = origin[1];
    node.pz = origin[2];
    node.ex = biased[0];
    node.ey = biased[1];
    node.ez = biased[2];
    node.imask = 0;
    node.childBase = childBase;
    node.triBase = triBase;
    int internalRank = 0, triOffset = 0;
    for (int s = 0; s < 8; ++s) {
        const int i = entryOfSlot[s];
        node.meta[s] = 0;
        node.qlox[s] = node.qloy[s] = node.qloz[s] = 0;
        node.qhix[s] = node.qhiy[s] = node.qhiz[s] = 0;
        if (i < 0) continue;
        const int b = entries[i];
        uint8_t ql[3], qh[3];
        quantizeChild(a.nodeLo[b], a.nodeHi[b], origin, step, ql, qh);
        node.qlox[s] = ql[0]; node.qloy[s] = ql[1]; node.qloz[s] = ql[2];
        node.qhix[s] = qh[0]; node.qhiy[s] = qh[1]; node.qhiz[s] = qh[2];
        if (isInternal(b)) {
            node.imask |= static_cast<uint8_t>(1u << s);
            node.meta[s] = 0;  // internal children carry no triangle bits
            const uint32_t slot = atomicAdd(nextCount, 1u);
            nextItems[slot] = CollapseItem{b, childBase + static_cast<uint32_t>(internalRank), item.depth + 1u, 0u};
            internalRank++;
        } else {
            // Leaf slot: its triangles in subtree order.
            int stack[8];
            int sp = 0;
            stack[sp++] = b;
            int written = 0;
            while (sp > 0) {
                const int x = stack[--sp];
                if (isLeaf(x)) {
                    const uint32_t prim = a.sortedIds[x - leafBase];
                    const uint32_t dst = triBase + static_cast<uint32_t>(triOffset + written);
                    const float4 v0 = a.vertices[a.indices[3 * prim + 0]];
                    const float4 v1 = a.vertices[a.indices[3 * prim + 1]];
                    const float4 v2 = a.vertices[a.indices[3 * prim + 2]];
                    const uint32_t id = a.primIds ? a.primIds[prim] : prim;
                    a.triVerts[3 * dst + 0] = make_float4(v0.x, v0.y, v0.z, __uint_as_float(id));
                    a.triVerts[3 * dst + 1] = make_float4(v1.x, v1.y, v1.z, a.opacityHint ? a.opacityHint[prim] : -1.0f);
                    a.triVerts[3 * dst + 2] = make_float4(v2.x, v2.y, v2.z, 0.0f);
                    written++;
                } else if (sp + 2 <= 8) {
                    stack[sp++] = a.right[x];
                    stack[sp++] = a.left[x];
                }
            }
            const uint32_t unary = written >= 3 ? 7u : (written == 2 ? 3u : 1u);
            node.meta[s] = static_cast<uint8_t>((unary << 5) | static_cast<uint32_t>(triOffset));
            triOffset += written;
        }
    }
    a.wide[item.wideIndex] = node;
}

template <typename T>
T* deviceAlloc(size_t count)
{
    return static_cast<T*>(deviceMalloc(std::max<size_t>(count, 1) * sizeof(T)));
}

}  // namespace

namespace {

// Leaf triangle copies from the current vertices (a refit keeps the leaf
// order; the id in .w is the triangle's position in the input list).
__global__ void refitTrianglesKernel(const float4* vertices, const uint32_t* indices, float4* triVerts, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = __float_as_uint(triVerts[3 * i].w);
    for (int k = 0; k < 3; ++k) {
        const float4 v = vertices[indices[3 * id + k]];
        triVerts[3 * i + k] = make_float4(v.x, v.y, v.z, triVerts[3 * i + k].w);  // id and opacity hint stay
    }
}

// One level of a refit: each node's children get their boxes from the level
// below (internal children) or from their triangles (leaf children), and the
// node is quantised again exactly as the build quantises it.
__global__ void refitLevelKernel(WideNode* nodes, const float4* triVerts, float4* boxes, uint32_t begin, uint32_t end,
                                 float sceneScale)
{
    const uint32_t n = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= end) return;
    WideNode node = nodes[n];
    float4 cl[8], ch[8];
    uint32_t present = 0u;
    float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.0f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
    for (int s = 0; s < 8; ++s) {
        const uint32_t meta = node.meta[s];
        if ((node.imask >> s) & 1u) {
            const uint32_t child = node.childBase + __popc(node.imask & ((1u << s) - 1u));
            cl[s] = boxes[2 * child];
            ch[s] = boxes[2 * child + 1];
        } else if (meta != 0u) {
            const uint32_t first = node.triBase + (meta & 31u), count = __popc(meta >> 5);
            cl[s] = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
            ch[s] = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
            for (uint32_t t = first; t < first + count; ++t) {
                for (int k = 0; k < 3; ++k) {
                    const float4 v = triVerts[3 * t + k];
                    cl[s] = make_float4(fminf(cl[s].x, v.x), fminf(cl[s].y, v.y), fminf(cl[s].z, v.z), 0.0f);
                    ch[s] = make_float4(fmaxf(ch[s].x, v.x), fmaxf(ch[s].y, v.y), fmaxf(ch[s].z, v.z), 0.0f);
                }
            }
        } else {
            continue;
        }
        present |= 1u << s;
        lo = make_float4(fminf(lo.x, cl[s].x), fminf(lo.y, cl[s].y), fminf(lo.z, cl[s].z), 0.0f);
        hi = make_float4(fmaxf(hi.x, ch[s].x), fmaxf(hi.y, ch[s].y), fmaxf(hi.z, ch[s].z), 0.0f);
    }
    float origin[3];
    double step[3];
    uint8_t biased[3];
    nodeFrame(lo, hi, sceneScale, origin, step, biased);
    node.px = origin[0];
    node.py = origin[1];
    node.pz = origin[2];
    node.ex = biased[0];
    node.ey = biased[1];
    node.ez = biased[2];
    for (int s = 0; s < 8; ++s) {
        uint8_t ql[3] = {0, 0, 0}, qh[3] = {0, 0, 0};
        if ((present >> s) & 1u) quantizeChild(cl[s], ch[s], origin, step, ql, qh);
        node.qlox[s] = ql[0];
        node.qloy[s] = ql[1];
        node.qloz[s] = ql[2];
        node.qhix[s] = qh[0];
        node.qhiy[s] = qh[1];
        node.qhiz[s] = qh[2];
    }
    nodes[n] = node;
    boxes[2 * n] = lo;
    boxes[2 * n + 1] = hi;
}

}  // namespace

void refitWideBvh(WideBvh& bvh, const float4* vertices, const uint32_t* indices, float sceneScale, cudaStream_t stream)
{
    if (bvh.nodeCount == 0 || bvh.levelStart.size() < 2) return;
    if (!bvh.nodeBoxes) bvh.nodeBoxes = deviceAlloc<float4>(2 * size_t(bvh.nodeCount));
    refitTrianglesKernel<<<(bvh.triangleCount + kBlock - 1) / kBlock, kBlock, 0, stream>>>(vertices, indices, bvh.triVerts,
                                                                                          bvh.triangleCount);
    CUDA_OK(cudaGetLastError());
    for (size_t d = bvh.levelStart.size() - 1; d-- > 0;) {
        const uint32_t begin = bvh.levelStart[d], end = bvh.levelStart[d + 1];
        if (end <= begin) continue;
        refitLevelKernel<<<(end - begin + kBlock - 1) / kBlock, kBlock, 0, stream>>>(bvh.nodes, bvh.triVerts,
                                                                                    bvh.nodeBoxes, begin, end, sceneScale);
        CUDA_OK(cudaGetLastError());
    }
    bvh.sceneScale = sceneScale;
    CUDA_OK(cudaStreamSynchronize(stream));
}

WideBvh buildWideBvh(const float4* vertices, const uint32_t* indices, uint32_t triangleCount, float sceneScale,
                     cudaStream_t stream, const uint32_t* primIds, const float* opacityHint)
{
    WideBvh out;
    if (triangleCount == 0) return out;
    const int n = static_cast<int>(triangleCount);
    const int blocks = (n + kBlock - 1) / kBlock;
    std::vector<void*> temps;
    auto tmp = [&](size_t bytes) {
        void* p = deviceMalloc(std::max<size_t>(bytes, 16));
        temps.push_back(p);
        return p;
    };
    try {
        float4* triLo = static_cast<float4*>(tmp(sizeof(float4) * n));
        float4* triHi = static_cast<float4*>(tmp(sizeof(float4) * n));
        uint32_t* bounds = static_cast<uint32_t*>(tmp(sizeof(uint32_t) * 6));
        const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        CUDA_OK(cudaMemcpyAsync(bounds, init, sizeof init, cudaMemcpyHostToDevice, stream));
        triangleBoxesKernel<<<blocks, kBlock, 0, stream>>>(vertices, indices, triangleCount, triLo, triHi, bounds);
        uint64_t* keys = static_cast<uint64_t*>(tmp(sizeof(uint64_t) * n));
        uint64_t* keysSorted = static_cast<uint64_t*>(tmp(sizeof(uint64_t) * n));
        uint32_t* ids = static_cast<uint32_t*>(tmp(sizeof(uint32_t) * n));
        uint32_t* idsSorted = static_cast<uint32_t*>(tmp(sizeof(uint32_t) * n));
        mortonKernel<<<blocks, kBlock, 0, stream>>>(triLo, triHi, triangleCount, bounds, keys, ids);
        size_t sortBytes = 0;
        CUDA_OK(cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, keys, keysSorted, ids, idsSorted, n, 0, 63, stream));
        void* sortTemp = tmp(sortBytes);
        CUDA_OK(cub::DeviceRadixSort::SortPairs(sortTemp, sortBytes, keys, keysSorted, ids, idsSorted, n, 0, 63, stream));

        const int nodes = 2 * n - 1;
        int* left = static_cast<int*>(tmp(sizeof(int) * std::max(n - 1, 1)));
        int* right = static_cast<int*>(tmp(sizeof(int) * std::max(n - 1, 1)));
        float4* nodeLo = static_cast<float4*>(tmp(sizeof(float4) * nodes));
        float4* nodeHi = static_cast<float4*>(tmp(sizeof(float4) * nodes));
        int* clustersA = static_cast<int*>(tmp(sizeof(int) * n));
        int* clustersB = static_cast<int*>(tmp(sizeof(int) * n));
        int* nn = static_cast<int*>(tmp(sizeof(int) * n));
        int* keep = static_cast<int*>(tmp(sizeof(int) * n));
        uint32_t* plocCounters = static_cast<uint32_t*>(tmp(sizeof(uint32_t) * 2));  // internal nodes, clusters
        CUDA_OK(cudaMemsetAsync(plocCounters, 0, sizeof(uint32_t) * 2, stream));
        initLeavesKernel<<<blocks, kBlock, 0, stream>>>(n, idsSorted, triLo, triHi, nodeLo, nodeHi, clustersA);
        size_t selectBytes = 0;
        CUDA_OK(cub::DeviceSelect::Flagged(nullptr, selectBytes, clustersB, keep, clustersA, plocCounters + 1, n, stream));
        void* selectTemp = tmp(selectBytes);
        float* collapseCost = static_cast<float*>(tmp(sizeof(float) * 7 * static_cast<size_t>(std::max(n - 1, 1))));
        uint8_t* collapseDecision = static_cast<uint8_t*>(tmp(8 * static_cast<size_t>(std::max(n - 1, 1))));
        uint32_t internalDone = 0;  // internal nodes whose collapse costs are filled
        int m = n;
        while (m > 1) {
            const int mb = (m + kBlock - 1) / kBlock;
            nearestNeighbourKernel<<<mb, kBlock, 0, stream>>>(clustersA, m, nodeLo, nodeHi, nn);
            mergeKernel<<<mb, kBlock, 0, stream>>>(clustersA, m, nn, left, right, nodeLo, nodeHi, plocCounters, clustersB,
                                                   keep);
            CUDA_OK(cub::DeviceSelect::Flagged(selectTemp, selectBytes, clustersB, keep, clustersA, plocCounters + 1, m,
                                               stream));
            uint32_t progress[2] = {0u, 0u};  // internal nodes, clusters
            CUDA_OK(cudaMemcpyAsync(progress, plocCounters, sizeof progress, cudaMemcpyDeviceToHost, stream));
            CUDA_OK(cudaStreamSynchronize(stream));
            const uint32_t next = progress[1];
            if (static_cast<int>(next) >= m) throw std::runtime_error("BVH build: clustering made no progress");
            m = static_cast<int>(next);
            // This round's nodes have children from earlier rounds (or leaves) only.
            if (progress[0] > internalDone) {
                const uint32_t count = progress[0] - internalDone;
                collapseCostKernel<<<(count + kBlock - 1) / kBlock, kBlock, 0, stream>>>(
                    n, left, right, nodeLo, nodeHi, internalDone, progress[0], collapseCost, collapseDecision);
                CUDA_OK(cudaGetLastError());
                internalDone = progress[0];
            }
        }
        int rootNode = 0;
        CUDA_OK(cudaMemcpyAsync(&rootNode, clustersA, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CUDA_OK(cudaStreamSynchronize(stream));

        out.nodes = deviceAlloc<WideNode>(n);
        out.triVerts = deviceAlloc<float4>(3 * static_cast<size_t>(n));
        uint32_t* counters = static_cast<uint32_t*>(tmp(sizeof(uint32_t) * 4));
        const uint32_t initCounters[4] = {1u, 0u, 0u, 0u};  // wide nodes (root allocated), triangles, error, next
        CUDA_OK(cudaMemcpyAsync(counters, initCounters, sizeof initCounters, cudaMemcpyHostToDevice, stream));
        CollapseItem* itemsA = static_cast<CollapseItem*>(tmp(sizeof(CollapseItem) * n));
        CollapseItem* itemsB = static_cast<CollapseItem*>(tmp(sizeof(CollapseItem) * n));
        const CollapseItem root{rootNode, 0u, 0u, 0u};
        CUDA_OK(cudaMemcpyAsync(itemsA, &root, sizeof root, cudaMemcpyHostToDevice, stream));
        CollapseArgs args{n,          left,       right,         nodeLo,       nodeHi,       idsSorted,
                          primIds,    opacityHint, vertices,     indices,      sceneScale,   collapseDecision,
                          out.nodes,  out.triVerts, counters + 0, counters + 1, counters + 2};
        uint32_t itemCount = 1;
        uint32_t depth = 0;
        // Nodes are allocated level by level: level d is [levelStart[d], levelStart[d+1]).
        out.levelStart = {0u, 1u};
        while (itemCount > 0) {
            CUDA_OK(cudaMemsetAsync(counters + 3, 0, sizeof(uint32_t), stream));
            collapseKernel<<<(itemCount + kBlock - 1) / kBlock, kBlock, 0, stream>>>(args, itemsA, itemCount, itemsB, counters + 3);
            CUDA_OK(cudaGetLastError());
            uint32_t progress[4];
            CUDA_OK(cudaMemcpyAsync(progress, counters, sizeof progress, cudaMemcpyDeviceToHost, stream));
            CUDA_OK(cudaStreamSynchronize(stream));
            itemCount = progress[3];
            if (itemCount > 0) out.levelStart.push_back(progress[0]);
            std::swap(itemsA, itemsB);
            ++depth;
        }
        out.sceneScale = sceneScale;
        uint32_t finalCounters[4];
        CUDA_OK(cudaMemcpyAsync(finalCounters, counters, sizeof finalCounters, cudaMemcpyDeviceToHost, stream));
        CUDA_OK(cudaStreamSynchronize(stream));
        if (finalCounters[2] != 0u) throw std::runtime_error("BVH build: tree deeper than the traversal stack");
        if (finalCounters[1] != triangleCount) throw std::runtime_error("BVH build: leaf triangle count mismatch");
        out.nodeCount = finalCounters[0];
        out.depth = depth;
        out.triangleCount = triangleCount;
    } catch (...) {
        for (void* p : temps) deviceFree(p);
        deviceFree(out.nodes);
        deviceFree(out.triVerts);
        throw;
    }
    for (void* p : temps) deviceFree(p);
    return out;
}

void freeWideBvh(WideBvh& bvh)
{
    deviceFree(bvh.nodes);
    deviceFree(bvh.triVerts);
    deviceFree(bvh.nodeBoxes);
    bvh = WideBvh{};
}

}  // namespace hdcx
