// oracle_trace.cpp - CPU ray queries for the oracle: a binned-SAH binary BVH,
// the watertight ray/triangle test and the confirmation rules that stand in
// for the Vulkan ray-query candidate loop. TEST INFRASTRUCTURE ONLY.
//
// The reference traverses with VK_KHR_ray_query (vulkan_path_tracer.cpp:
// 1228-1243 closest hit with stochastic opacity, :855-912 shadow rays with a
// 0.5 opacity threshold, :1130-1151 opaque boundary rays). Its BVH and
// triangle test live in the closed Vulkan driver, so the hit/miss decision is
// defined here as the watertight test of Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2(1), 2013, in binary32 without fused
// multiply-add, with a binary64 recomputation of degenerate edge functions.
// The closest hit is the confirmed candidate with the smallest t; equal t goes
// to the smaller flattened primitive index. Any BVH that visits every
// candidate gives the same answer, which is what makes the GPU and CPU
// results comparable bit for bit.
#include "oracle_internal.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace oracle {

uint32_t hashState(uint32_t value)
{
    // lowbias32 integer hash (vulkan_path_tracer.cpp:100-107)
    value ^= value >> 16;
    value *= 0x7feb352du;
    value ^= value >> 15;
    value *= 0x846ca68bu;
    return value ^ (value >> 16);
}

// Order-independent stand-in for the reference's per-candidate
// `randomFloat(rng) <= surfaceOpacity(...)` (vulkan_path_tracer.cpp:1239),
// whose draw order depends on the driver's traversal order. The threshold of
// a candidate is a hash of the path's RNG state when the ray starts and the
// primitive index, mapped to [0, 1] like randomFloat; the RNG state itself is
// not advanced by candidates.
float anyHitThreshold(uint32_t rayRng, uint32_t primitive)
{
    const uint32_t h = hashState(rayRng ^ hashState(primitive ^ 0x27d4eb2fu));
    return uintToFloat(h) * (1.0f / 4294967296.0f);
}

namespace {

struct RayPre {
    vec3 o;
    int kx, ky, kz;
    float sx, sy, sz;
};

float Comp(vec3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

RayPre Precompute(vec3 o, vec3 d)
{
    RayPre r;
    r.o = o;
    const float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) { kz = 2; }
    int kx = kz + 1;
    if (kx == 3) kx = 0;
    int ky = kx + 1;
    if (ky == 3) ky = 0;
    if (Comp(d, kz) < 0.0f) std::swap(kx, ky);
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    const float dz = Comp(d, kz);
    r.sx = Comp(d, kx) / dz;
    r.sy = Comp(d, ky) / dz;
    r.sz = 1.0f / dz;
    return r;
}

// Returns true with t and the weights of vertex 1 and vertex 2.
bool IntersectTriangle(const RayPre& r, vec3 v0, vec3 v1, vec3 v2, float tmin, float tmax,
                       float* tOut, vec2* bary)
{
    const vec3 a = v0 - r.o;
    const vec3 b = v1 - r.o;
    const vec3 c = v2 - r.o;
    const float az = Comp(a, r.kz), bz = Comp(b, r.kz), cz = Comp(c, r.kz);
    const float ax = Comp(a, r.kx) - r.sx * az;
    const float ay = Comp(a, r.ky) - r.sy * az;
    const float bx = Comp(b, r.kx) - r.sx * bz;
    const float by = Comp(b, r.ky) - r.sy * bz;
    const float cx = Comp(c, r.kx) - r.sx * cz;
    const float cy = Comp(c, r.ky) - r.sy * cz;
    float u = cx * by - cy * bx;
    float v = ax * cy - ay * cx;
    float w = bx * ay - by * ax;
    if (u == 0.0f || v == 0.0f || w == 0.0f) {
        u = static_cast<float>(static_cast<double>(cx) * by - static_cast<double>(cy) * bx);
        v = static_cast<float>(static_cast<double>(ax) * cy - static_cast<double>(ay) * cx);
        w = static_cast<float>(static_cast<double>(bx) * ay - static_cast<double>(by) * ax);
    }
    if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f)) return false;
    const float det = u + v + w;
    if (det == 0.0f) return false;
    const float saz = r.sz * az, sbz = r.sz * bz, scz = r.sz * cz;
    const float tScaled = u * saz + v * sbz + w * scz;
    const float t = tScaled / det;
    if (!(t >= tmin && t <= tmax)) return false;
    *tOut = t;
    *bary = V2(v / det, w / det);
    return true;
}

vec3 Vertex(const PackedScene& s, uint32_t prim, uint32_t corner)
{
    return xyz(s.vertices[s.indices[prim * 3u + corner]]);
}

struct BuildItem {
    float lo[3], hi[3], c[3];
    uint32_t prim;
};

uint32_t BuildRecursive(Bvh& bvh, std::vector<BuildItem>& items, size_t begin, size_t end)
{
    const uint32_t nodeIndex = static_cast<uint32_t>(bvh.nodes.size());
    bvh.nodes.push_back({});
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (size_t i = begin; i < end; ++i) {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], items[i].lo[k]);
            hi[k] = std::max(hi[k], items[i].hi[k]);
            clo[k] = std::min(clo[k], items[i].c[k]);
            chi[k] = std::max(chi[k], items[i].c[k]);
        }
    }
    const size_t count = end - begin;
    auto makeLeaf = [&]() {
        BvhNode& node = bvh.nodes[nodeIndex];
        std::memcpy(node.lo, lo, sizeof lo);
        std::memcpy(node.hi, hi, sizeof hi);
        node.left = static_cast<uint32_t>(bvh.primitives.size());
        node.count = static_cast<uint32_t>(count);
        node.right = 0;
        for (size_t i = begin; i < end; ++i) bvh.primitives.push_back(items[i].prim);
        return nodeIndex;
    };
    if (count <= 4) return makeLeaf();
    // Binned SAH over the centroid bounds, 16 bins per axis.
    constexpr int kBins = 16;
    int bestAxis = -1;
    int bestSplit = 0;
    double bestCost = 1e300;
    auto area = [](const float* l, const float* h) {
        const double dx = std::max(0.0f, h[0] - l[0]), dy = std::max(0.0f, h[1] - l[1]),
                     dz = std::max(0.0f, h[2] - l[2]);
        return dx * dy + dy * dz + dz * dx;
    };
    for (int axis = 0; axis < 3; ++axis) {
        const float extent = chi[axis] - clo[axis];
        if (!(extent > 0.0f)) continue;
        struct Bin {
            float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            size_t n = 0;
        } bins[kBins];
        for (size_t i = begin; i < end; ++i) {
            int b = static_cast<int>((items[i].c[axis] - clo[axis]) / extent * kBins);
            b = std::clamp(b, 0, kBins - 1);
            bins[b].n++;
            for (int k = 0; k < 3; ++k) {
                bins[b].lo[k] = std::min(bins[b].lo[k], items[i].lo[k]);
                bins[b].hi[k] = std::max(bins[b].hi[k], items[i].hi[k]);
            }
        }
        double rightArea[kBins];
        size_t rightCount[kBins];
        float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        size_t rn = 0;
        for (int b = kBins - 1; b > 0; --b) {
            rn += bins[b].n;
            for (int k = 0; k < 3; ++k) {
                rlo[k] = std::min(rlo[k], bins[b].lo[k]);
                rhi[k] = std::max(rhi[k], bins[b].hi[k]);
            }
            rightArea[b] = rn ? area(rlo, rhi) : 0.0;
            rightCount[b] = rn;
        }
        float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        size_t ln = 0;
        for (int b = 0; b < kBins - 1; ++b) {
            ln += bins[b].n;
            for (int k = 0; k < 3; ++k) {
                llo[k] = std::min(llo[k], bins[b].lo[k]);
                lhi[k] = std::max(lhi[k], bins[b].hi[k]);
            }
            if (ln == 0 || rightCount[b + 1] == 0) continue;
            const double cost = ln * area(llo, lhi) + rightCount[b + 1] * rightArea[b + 1];
            if (cost < bestCost) {
                bestCost = cost;
                bestAxis = axis;
                bestSplit = b;
            }
        }
    }
    size_t mid;
    if (bestAxis < 0) {
        mid = begin + count / 2;  // all centroids coincide: split by index
    } else {
        const float extent = chi[bestAxis] - clo[bestAxis];
        auto it = std::partition(items.begin() + begin, items.begin() + end, [&](const BuildItem& item) {
            int b = static_cast<int>((item.c[bestAxis] - clo[bestAxis]) / extent * kBins);
            b = std::clamp(b, 0, kBins - 1);
            return b <= bestSplit;
        });
        mid = static_cast<size_t>(it - items.begin());
        if (mid == begin || mid == end) mid = begin + count / 2;
    }
    const uint32_t left = BuildRecursive(bvh, items, begin, mid);
    const uint32_t right = BuildRecursive(bvh, items, mid, end);
    BvhNode& node = bvh.nodes[nodeIndex];
    std::memcpy(node.lo, lo, sizeof lo);
    std::memcpy(node.hi, hi, sizeof hi);
    node.left = left;
    node.right = right;
    node.count = 0;
    return nodeIndex;
}

// Conservative slab test in binary64 with a relative pad, so that no box that
// holds a candidate the triangle test accepts is rejected.
bool BoxHit(const BvhNode& n, const double o[3], const double inv[3], double tmin, double tmax,
            double* tNear)
{
    double t0 = tmin, t1 = tmax;
    for (int k = 0; k < 3; ++k) {
        const double pad = 1e-5 * (std::fabs(static_cast<double>(n.hi[k]) - n.lo[k]) +
                                   std::fabs(static_cast<double>(n.lo[k])) +
                                   std::fabs(static_cast<double>(n.hi[k]))) + 1e-7;
        double a = (n.lo[k] - pad - o[k]) * inv[k];
        double b = (n.hi[k] + pad - o[k]) * inv[k];
        if (a > b) std::swap(a, b);
        if (std::isnan(a) || std::isnan(b)) {
            // Direction component is zero and the origin sits on a padded slab
            // boundary: inside the slab, keep the interval.
            if (o[k] < n.lo[k] - pad || o[k] > n.hi[k] + pad) return false;
            continue;
        }
        t0 = std::max(t0, a);
        t1 = std::min(t1, b);
        if (t0 > t1) return false;
    }
    *tNear = t0;
    return true;
}

template <bool kAny>
bool Traverse(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction, float tmin,
              float tmax, AcceptMode mode, uint32_t rayRng, Hit* hit)
{
    if (bvh.nodes.empty()) return false;
    const RayPre pre = Precompute(origin, direction);
    const double o[3] = {origin.x, origin.y, origin.z};
    const double inv[3] = {1.0 / static_cast<double>(direction.x), 1.0 / static_cast<double>(direction.y),
                           1.0 / static_cast<double>(direction.z)};
    float bestT = tmax;
    uint32_t bestPrim = 0xffffffffu;
    vec2 bestBary{0.0f, 0.0f};
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const BvhNode& node = bvh.nodes[stack[--sp]];
        double tNear;
        const double limit = static_cast<double>(bestT) * (1.0 + 1e-5) + 1e-6;
        if (!BoxHit(node, o, inv, static_cast<double>(tmin) * (1.0 - 1e-5) - 1e-6, limit, &tNear)) continue;
        if (node.count == 0) {
            if (sp + 2 > 128) continue;
            stack[sp++] = node.right;
            stack[sp++] = node.left;
            continue;
        }
        for (uint32_t i = 0; i < node.count; ++i) {
            const uint32_t prim = bvh.primitives[node.left + i];
            float t;
            vec2 bary;
            if (!IntersectTriangle(pre, Vertex(scene, prim, 0), Vertex(scene, prim, 1),
                                   Vertex(scene, prim, 2), tmin, tmax, &t, &bary)) {
                continue;
            }
            if (!kAny) {
                if (t > bestT) continue;
                if (t == bestT && prim > bestPrim) continue;
            }
            bool confirmed = true;
            if (mode == AcceptMode::Stochastic) {
                confirmed = anyHitThreshold(rayRng, prim) <= surfaceOpacity(scene, prim, bary);
            } else if (mode == AcceptMode::Threshold) {
                confirmed = surfaceOpacity(scene, prim, bary) >= 0.5f;
            }
            if (!confirmed) continue;
            if (kAny) return true;
            bestT = t;
            bestPrim = prim;
            bestBary = bary;
        }
    }
    if (kAny || bestPrim == 0xffffffffu) return false;
    hit->primitive = bestPrim;
    hit->t = bestT;
    hit->barycentrics = bestBary;
    return true;
}

}  // namespace

Bvh BuildBvh(const PackedScene& scene)
{
    Bvh bvh;
    const uint32_t n = scene.primitiveCount;
    if (n == 0) return bvh;
    std::vector<BuildItem> items(n);
    for (uint32_t p = 0; p < n; ++p) {
        const vec3 v[3] = {Vertex(scene, p, 0), Vertex(scene, p, 1), Vertex(scene, p, 2)};
        BuildItem& it = items[p];
        it.prim = p;
        const float* c0 = &v[0].x;
        const float* c1 = &v[1].x;
        const float* c2 = &v[2].x;
        for (int k = 0; k < 3; ++k) {
            it.lo[k] = std::min(c0[k], std::min(c1[k], c2[k]));
            it.hi[k] = std::max(c0[k], std::max(c1[k], c2[k]));
            it.c[k] = 0.5f * (it.lo[k] + it.hi[k]);
        }
    }
    bvh.nodes.reserve(2 * n);
    BuildRecursive(bvh, items, 0, n);
    return bvh;
}

bool TraceClosest(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction, float tmin,
                  float tmax, AcceptMode mode, uint32_t rayRng, Hit* hit)
{
    return Traverse<false>(scene, bvh, origin, direction, tmin, tmax, mode, rayRng, hit);
}

void TraceAll(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction, float tmin, float tmax,
              std::vector<Hit>* hits)
{
    hits->clear();
    if (bvh.nodes.empty()) return;
    const RayPre pre = Precompute(origin, direction);
    const double o[3] = {origin.x, origin.y, origin.z};
    const double inv[3] = {1.0 / static_cast<double>(direction.x), 1.0 / static_cast<double>(direction.y),
                           1.0 / static_cast<double>(direction.z)};
    const double limit = static_cast<double>(tmax) * (1.0 + 1e-5) + 1e-6;
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const BvhNode& node = bvh.nodes[stack[--sp]];
        double tNear;
        if (!BoxHit(node, o, inv, static_cast<double>(tmin) * (1.0 - 1e-5) - 1e-6, limit, &tNear)) continue;
        if (node.count == 0) {
            if (sp + 2 > 128) continue;
            stack[sp++] = node.right;
            stack[sp++] = node.left;
            continue;
        }
        for (uint32_t i = 0; i < node.count; ++i) {
            const uint32_t prim = bvh.primitives[node.left + i];
            float t;
            vec2 bary;
            if (IntersectTriangle(pre, Vertex(scene, prim, 0), Vertex(scene, prim, 1), Vertex(scene, prim, 2), tmin,
                                  tmax, &t, &bary)) {
                hits->push_back(Hit{prim, t, bary});
            }
        }
    }
}

bool TraceAny(const PackedScene& scene, const Bvh& bvh, vec3 origin, vec3 direction, float tmin,
              float tmax, AcceptMode mode)
{
    return Traverse<true>(scene, bvh, origin, direction, tmin, tmax, mode, 0u, nullptr);
}

}  // namespace oracle
