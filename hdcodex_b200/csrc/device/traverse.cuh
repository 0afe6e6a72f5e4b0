// traverse.cuh - ray queries on the 8-wide compressed BVH.
//
// Replaces the reference's VK_KHR_ray_query loops (vulkan_path_tracer.cpp:
// 1228-1243 closest hit with stochastic opacity, :855-912 shadow any-hit with
// a 0.5 opacity threshold, :1130-1151 opaque boundary rays).
//
// * Triangle test: watertight test of Woop, Benthin and Wald (JCGT 2013) in
//   binary32 with no fused multiply-add, degenerate edge functions recomputed
//   in binary64, t = T / det, accepted when tmin <= t <= tmax. The CPU oracle
//   states the same test, so hit/miss and (t, barycentrics) agree bit for bit.
// * Closest hit: smallest t among confirmed candidates; equal t goes to the
//   smaller flattened primitive index. The result does not depend on the
//   order in which the traversal meets candidates.
// * Traversal: one thread per ray over 80-byte nodes (Ylitie, Karras and
//   Laine, HPG 2017): the eight quantised child boxes are tested per node
//   with one fused multiply-add per plane; internal hits are visited nearest
//   octant first, leaf triangles of the node are tested before descending,
//   and pending node groups go on a per-thread stack. Child boxes are padded
//   by one quantisation step on every side at build time, which keeps the
//   binary32 slab test conservative. The 48 plane distances of a node are
//   evaluated two children at a time with the packed fused multiply-add of
//   sm_100 (__ffma2_rn), the slab intervals with its three-input min/max.
// * Faults: a node group that finds the stack full, or a traversal that
//   visits more nodes than the BVH holds (a malformed node array), sets a
//   bit in the traversal's fault word; the kernels OR it into the render's
//   counters once per thread, outside their loops, and the host reports it
//   as an error of the render.
#pragma once

#include "common.cuh"
#include "shading.cuh"

namespace hdcx {

constexpr int kTraversalStack = 64;


enum class Accept : int {
    Opaque = 0,      // every candidate is confirmed
    Stochastic = 1,  // confirmed iff anyHitThreshold(rayRng, prim) <= opacity
    Threshold = 2,   // confirmed iff opacity >= 0.5
};

struct HitRecord {
    float t;
    uint32_t primitive;
    float b1;
    float b2;
};

struct RayPre {
    float3 o;
    int kx, ky, kz;
    float sx, sy, sz;
};

HDCX_D float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

HDCX_D RayPre precomputeRay(float3 o, float3 d)
{
    RayPre r;
    r.o = o;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) { kz = 1; m = ay; }
    if (az > m) kz = 2;
    int kx = kz + 1;
    if (kx == 3) kx = 0;
    int ky = kx + 1;
    if (ky == 3) ky = 0;
    const float dz = comp(d, kz);
    if (dz < 0.0f) {
        const int tmp = kx;
        kx = ky;
        ky = tmp;
    }
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.sx = __fdiv_rn(comp(d, kx), dz);
    r.sy = __fdiv_rn(comp(d, ky), dz);
    r.sz = __fdiv_rn(1.0f, dz);
    return r;
}

HDCX_D bool intersectTriangle(const RayPre& r, float3 v0, float3 v1, float3 v2, float tmin, float tmax, float& tOut,
                              float& b1, float& b2)
{
    const float3 a = v0 - r.o;
    const float3 b = v1 - r.o;
    const float3 c = v2 - r.o;
    const float az = comp(a, r.kz), bz = comp(b, r.kz), cz = comp(c, r.kz);
    const float ax = __fsub_rn(comp(a, r.kx), __fmul_rn(r.sx, az));
    const float ay = __fsub_rn(comp(a, r.ky), __fmul_rn(r.sy, az));
    const float bx = __fsub_rn(comp(b, r.kx), __fmul_rn(r.sx, bz));
    const float by = __fsub_rn(comp(b, r.ky), __fmul_rn(r.sy, bz));
    const float cx = __fsub_rn(comp(c, r.kx), __fmul_rn(r.sx, cz));
    const float cy = __fsub_rn(comp(c, r.ky), __fmul_rn(r.sy, cz));
    float u = __fsub_rn(__fmul_rn(cx, by), __fmul_rn(cy, bx));
    float v = __fsub_rn(__fmul_rn(ax, cy), __fmul_rn(ay, cx));
    float w = __fsub_rn(__fmul_rn(bx, ay), __fmul_rn(by, ax));
    if (u == 0.0f || v == 0.0f || w == 0.0f) {
        u = __double2float_rn(__dsub_rn(__dmul_rn(cx, by), __dmul_rn(cy, bx)));
        v = __double2float_rn(__dsub_rn(__dmul_rn(ax, cy), __dmul_rn(ay, cx)));
        w = __double2float_rn(__dsub_rn(__dmul_rn(bx, ay), __dmul_rn(by, ax)));
    }
    if ((u < 0.0f || v < 0.0f || w < 0.0f) && (u > 0.0f || v > 0.0f || w > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(u, v), w);
    if (det == 0.0f) return false;
    const float saz = __fmul_rn(r.sz, az), sbz = __fmul_rn(r.sz, bz), scz = __fmul_rn(r.sz, cz);
    const float tScaled = __fadd_rn(__fadd_rn(__fmul_rn(u, saz), __fmul_rn(v, sbz)), __fmul_rn(w, scz));
    const float t = __fdiv_rn(tScaled, det);
    if (!(t >= tmin && t <= tmax)) return false;
    tOut = t;
    b1 = __fdiv_rn(v, det);
    b2 = __fdiv_rn(w, det);
    return true;
}

// Byte `index` of `word` as the float 2^23 + byte: the byte is placed in the
// low mantissa bits of 2^23 (bit pattern 0x4B0000bb), exactly. A byte permute
// runs on a full-rate pipe, where an integer-to-float conversion would queue
// on the quarter-rate conversion pipe (eight children x six planes per node).
HDCX_D float biasedByte(uint32_t word, int index)
{
    return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7440u + static_cast<uint32_t>(index)));
}

// Quantised planes of children 2j and 2j+1 (bytes k and k+1 of `word`, k
// even) as distances t = (2^23 + q) * a + c, with c = b - 2^23 * a, two lanes
// per packed fused multiply-add.
HDCX_D float2 planePair(uint32_t word, int k, float2 a, float2 c)
{
    return __ffma2_rn(make_float2(biasedByte(word, k), biasedByte(word, k + 1)), a, c);
}

// Three-input minimum and maximum of sm_100 (PTX min/max with three f32
// operands): one instruction where two-input forms take two.
HDCX_D float max3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
HDCX_D float min3(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Moves bit i of an 8-bit mask to bit i ^ x (x in 0..7): three conditional
// swaps, of neighbouring bits, bit pairs and nibbles.
HDCX_D uint32_t permuteSlots(uint32_t m, uint32_t x)
{
    if (x & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (x & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (x & 4u) m = ((m & 0x0fu) << 4) | ((m >> 4) & 0x0fu);
    return m;
}

// Opacity of a candidate from its leaf copy: the second vertex's .w holds the
// constant opacity of a material without an opacity texture (the value
// surfaceOpacity returns for it), else -1; only then are the material and
// the texture read.
HDCX_D float leafOpacity(float hint, const DeviceScene& s, uint32_t prim, float b1, float b2)
{
    return hint >= 0.0f ? hint : surfaceOpacity(s, prim, b1, b2);
}

// State of one ray's traversal: the ray, the closest confirmed hit so far,
// the current node group and triangle group; pending node groups live on a
// per-thread stack of kTraversalStack entries held by the caller.
struct Traversal {
    RayPre pre;
    float idx, idy, idz;
    uint32_t octInv;
    float tmin;
    float bestT;
    uint32_t bestPrim;
    float bestB1, bestB2;
    uint2 nodeGroup;  // x: base index of the internal children; y: hit bits in 24..31 (by visiting order) | imask
    uint2 triGroup;   // x: first triangle slot; y: bits of the triangles left to test
    int sp;
    uint32_t budget;  // every node is entered at most once; guards against a malformed node array
    uint32_t rayRng;
    uint32_t fault;   // kTraversalOverflow | kTraversalBudget
};

enum : int { kStepContinue = 0, kStepDone = 1, kStepAnyHit = 2 };

HDCX_D void beginTraversal(Traversal& st, const DeviceScene& s, float3 o, float3 d, float tmin, float tmax,
                           uint32_t rayRng)
{
    st.pre = precomputeRay(o, d);
    const float tiny = 8.271806e-25f;  // 2^-80: direction components below it are treated as 2^-80
    st.idx = 1.0f / (fabsf(d.x) > tiny ? d.x : copysignf(tiny, d.x));
    st.idy = 1.0f / (fabsf(d.y) > tiny ? d.y : copysignf(tiny, d.y));
    st.idz = 1.0f / (fabsf(d.z) > tiny ? d.z : copysignf(tiny, d.z));
    st.octInv = ((d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u)) ^ 7u;
    st.tmin = tmin;
    st.bestT = tmax;
    st.bestPrim = kInvalidPrimitive;
    st.bestB1 = 0.0f;
    st.bestB2 = 0.0f;
    // The root is child slot 0 of a virtual parent whose children start at node 0.
    st.nodeGroup = s.nodeCount == 0u ? make_uint2(0u, 0u) : make_uint2(0u, (1u << (24u + (0u ^ st.octInv))) | 1u);
    st.triGroup = make_uint2(0u, 0u);
    st.sp = 0;
    st.budget = s.nodeCount + 1u;
    st.rayRng = rayRng;
    st.fault = 0u;
}

// Tests the eight children of node `nodeIndex` against a ray (origin o,
// inverse direction id, octant mask octInv) up to bestT: hit internal
// children become nodeGroup (hit bits in 24..31 by visiting order | imask),
// hit leaf triangles triGroup (first slot, bits).
//
// A plane at quantised coordinate q lies at t = q * a + b along the ray, with
// a = scale * id and b = (p - o) * id. The byte arrives as the float 2^23 + q
// (biasedByte), so the offset is folded once per node: c = b - 2^23 * a,
// rounded once, an error of at most half of |a|, half a quantisation step.
// The build pads every child box by one step on each side, which covers it:
// the test stays conservative, and only which nodes are entered depends on
// it, never a hit. The folded offset is finite for nodes narrower than about
// 2^32 scene units (|a| * 2^23 below the binary32 range with |id| <= 2^80).
template <bool kMargin>
HDCX_D void testNode(const WideNode* nodes, uint32_t nodeIndex, float3 o, float idx, float idy, float idz,
                     uint32_t octInv, float bestT, float mx, float my, float mz, uint2& nodeGroup, uint2& triGroup)
{
    const uint4* np = reinterpret_cast<const uint4*>(nodes + nodeIndex);
    const uint4 n0 = __ldg(np + 0), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
    const float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    const uint32_t e = n0.w;
    const float scx = __uint_as_float((e & 0xffu) << 23);
    const float scy = __uint_as_float(((e >> 8) & 0xffu) << 23);
    const float scz = __uint_as_float(((e >> 16) & 0xffu) << 23);
    const uint32_t imask = e >> 24;
    const float ax = scx * idx, ay = scy * idy, az = scz * idz;
    const float bx = (px - o.x) * idx, by = (py - o.y) * idy, bz = (pz - o.z) * idz;
    constexpr float kBias = -8388608.0f;  // -2^23
    // With kMargin every box is widened by (mx, my, mz) in t per axis: the
    // near plane's distance drops by the margin, the far plane's grows.
    const float cxn = fmaf(kBias, ax, kMargin ? bx - mx : bx), cxf = kMargin ? fmaf(kBias, ax, bx + mx) : cxn;
    const float cyn = fmaf(kBias, ay, kMargin ? by - my : by), cyf = kMargin ? fmaf(kBias, ay, by + my) : cyn;
    const float czn = fmaf(kBias, az, kMargin ? bz - mz : bz), czf = kMargin ? fmaf(kBias, az, bz + mz) : czn;
    const float2 ax2 = make_float2(ax, ax), ay2 = make_float2(ay, ay), az2 = make_float2(az, az);
    const float2 cxn2 = make_float2(cxn, cxn), cyn2 = make_float2(cyn, cyn), czn2 = make_float2(czn, czn);
    const float2 cxf2 = make_float2(cxf, cxf), cyf2 = make_float2(cyf, cyf), czf2 = make_float2(czf, czf);
    const uint32_t loX0 = n2.x, loX1 = n2.y, loY0 = n2.z, loY1 = n2.w, loZ0 = n3.x, loZ1 = n3.y;
    const uint32_t hiX0 = n3.z, hiX1 = n3.w, hiY0 = n4.x, hiY1 = n4.y, hiZ0 = n4.z, hiZ1 = n4.w;
    const bool sx = idx >= 0.0f, sy = idy >= 0.0f, sz = idz >= 0.0f;
    const uint32_t nearX0 = sx ? loX0 : hiX0, nearX1 = sx ? loX1 : hiX1, farX0 = sx ? hiX0 : loX0, farX1 = sx ? hiX1 : loX1;
    const uint32_t nearY0 = sy ? loY0 : hiY0, nearY1 = sy ? loY1 : hiY1, farY0 = sy ? hiY0 : loY0, farY1 = sy ? hiY1 : loY1;
    const uint32_t nearZ0 = sz ? loZ0 : hiZ0, nearZ1 = sz ? loZ1 : hiZ1, farZ0 = sz ? hiZ0 : loZ0, farZ1 = sz ? hiZ1 : loZ1;
    const uint32_t meta0 = n1.z, meta1 = n1.w;
    uint32_t hits = 0u, triHits = 0u;
    // Children 2j and 2j+1 share a word per plane (bytes k and k+1). The meta
    // byte of a leaf child is its unary triangle count << 5 | first triangle;
    // internal and empty children have meta 0 and add no triangle bits.
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int k = (2 * j) & 3;
        const bool low = j < 2;
        const float2 tnx = planePair(low ? nearX0 : nearX1, k, ax2, cxn2);
        const float2 tny = planePair(low ? nearY0 : nearY1, k, ay2, cyn2);
        const float2 tnz = planePair(low ? nearZ0 : nearZ1, k, az2, czn2);
        const float2 tfx = planePair(low ? farX0 : farX1, k, ax2, cxf2);
        const float2 tfy = planePair(low ? farY0 : farY1, k, ay2, cyf2);
        const float2 tfz = planePair(low ? farZ0 : farZ1, k, az2, czf2);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * j + h;
            const uint32_t metaShift = (low ? meta0 : meta1) >> (8 * (k + h));  // low 5 bits: first triangle
            const uint32_t tris = __funnelshift_l(0u, (metaShift >> 5) & 7u, metaShift);
            const float tNear = max3(h ? tnx.y : tnx.x, h ? tny.y : tny.x, fmaxf(h ? tnz.y : tnz.x, 0.0f));
            const float tFar = min3(h ? tfx.y : tfx.x, h ? tfy.y : tfy.x, fminf(h ? tfz.y : tfz.x, bestT));
            if (tNear <= tFar) {
                hits |= 1u << i;
                triHits |= tris;
            }
        }
    }
    // Internal children in visiting order: bit i goes to i ^ octInv.
    nodeGroup = make_uint2(n1.x, (permuteSlots(hits & imask, octInv) << 24) | imask);
    triGroup = make_uint2(n1.y, triHits);
}

// One traversal step: the triangles of the current triangle group, then one
// node (its eight children are tested; hit internal children become the new
// node group, hit leaf triangles the new triangle group). Returns
// kStepContinue, kStepDone (closest hit, if any, in st.best*) or, for kAny,
// kStepAnyHit at the first confirmed candidate.
template <Accept kMode, bool kAny, bool kCount = false>
HDCX_D int traversalStep(Traversal& st, uint2* stack, const DeviceScene& s, uint2* work)
{
    while (st.triGroup.y != 0u) {
        const int bit = __ffs(st.triGroup.y) - 1;
        st.triGroup.y &= st.triGroup.y - 1u;
        const uint32_t slot = st.triGroup.x + static_cast<uint32_t>(bit);
        const float4 w0 = __ldg(s.triVerts + slot * 3u + 0u);
        const float4 w1 = __ldg(s.triVerts + slot * 3u + 1u);
        const float4 w2 = __ldg(s.triVerts + slot * 3u + 2u);
        if (kCount) work->y++;
        float t, b1, b2;
        if (!intersectTriangle(st.pre, xyz(w0), xyz(w1), xyz(w2), st.tmin, st.bestT, t, b1, b2)) continue;
        const uint32_t prim = __float_as_uint(w0.w);
        if (!kAny) {
            if (t > st.bestT) continue;
            if (t == st.bestT && prim > st.bestPrim) continue;
        }
        if (kMode == Accept::Stochastic) {
            // The threshold lies in [0, 1]: an opacity of 1 always confirms.
            const float opacity = leafOpacity(w1.w, s, prim, b1, b2);
            if (opacity < 1.0f && !(anyHitThreshold(st.rayRng, prim) <= opacity)) continue;
        } else if (kMode == Accept::Threshold) {
            if (!(leafOpacity(w1.w, s, prim, b1, b2) >= 0.5f)) continue;
        }
        if (kAny) return kStepAnyHit;
        st.bestT = t;
        st.bestPrim = prim;
        st.bestB1 = b1;
        st.bestB2 = b2;
    }
    if ((st.nodeGroup.y & 0xff000000u) == 0u) {
        if (st.sp == 0) return kStepDone;
        st.nodeGroup = stack[--st.sp];
    }
    if (st.budget-- == 0u) {
        st.fault |= kTraversalBudget;
        return kStepDone;
    }
    // Next child of the current group, nearest octant first.
    const uint32_t hitBits = st.nodeGroup.y >> 24;
    const uint32_t pos = 31u - __clz(hitBits);
    st.nodeGroup.y &= ~(1u << (24u + pos));
    const uint32_t childSlot = pos ^ st.octInv;
    const uint32_t parentMask = st.nodeGroup.y & 0xffu;
    const uint32_t nodeIndex = st.nodeGroup.x + __popc(parentMask & ((1u << childSlot) - 1u));
    if ((st.nodeGroup.y & 0xff000000u) != 0u) {
        if (st.sp < kTraversalStack) stack[st.sp++] = st.nodeGroup;
        else st.fault |= kTraversalOverflow;
    }

    if (kCount) work->x++;
    testNode<false>(s.nodes, nodeIndex, st.pre.o, st.idx, st.idy, st.idz, st.octInv, st.bestT, 0.0f, 0.0f, 0.0f,
                    st.nodeGroup, st.triGroup);
    return kStepContinue;
}

// ---------------------------------------------------------------------------
// Two-level scenes. The top-level BVH's leaves are instances; for each hit
// instance its BLAS is traversed with the ray in object space (the BLAS of
// the scene's non-instanced triangles is in world space), sharing the
// closest hit. Node tests of an instanced BLAS use the object-space ray with
// boxes widened by a margin that covers the rounding of the transformed ray
// and of the world vertices; triangle tests always use the world ray and the
// world-space (flattened) vertices, so hits, distances, barycentrics and the
// tie rule are those of the flattened scene bit for bit.
// ---------------------------------------------------------------------------
constexpr int kTopStack = 32;

struct ClosestHit {
    float t;
    uint32_t prim;
    float b1, b2;
};

// Same acceptance as the single-level traversal (closest, ties to the
// smaller id; any-hit opacity rules).
template <Accept kMode, bool kAny>
HDCX_D bool confirmCandidate(const DeviceScene& s, uint32_t rayRng, uint32_t prim, float t, float b1, float b2,
                             const ClosestHit& best)
{
    if (!kAny) {
        if (t > best.t) return false;
        if (t == best.t && prim > best.prim) return false;
    }
    if (kMode == Accept::Stochastic) {
        const float opacity = surfaceOpacity(s, prim, b1, b2);
        if (opacity < 1.0f && !(anyHitThreshold(rayRng, prim) <= opacity)) return false;
    } else if (kMode == Accept::Threshold) {
        if (!(surfaceOpacity(s, prim, b1, b2) >= 0.5f)) return false;
    }
    return true;
}

HDCX_D float3 inverseDirection(float3 d)
{
    const float tiny = 8.271806e-25f;  // 2^-80, as beginTraversal
    return make_float3(1.0f / (fabsf(d.x) > tiny ? d.x : copysignf(tiny, d.x)),
                       1.0f / (fabsf(d.y) > tiny ? d.y : copysignf(tiny, d.y)),
                       1.0f / (fabsf(d.z) > tiny ? d.z : copysignf(tiny, d.z)));
}

HDCX_D uint32_t octantMask(float3 d)
{
    return ((d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u)) ^ 7u;
}

HDCX_D float maxAbs3(float3 v) { return fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fabsf(v.z)); }

// Pops the next child node of `group` (nearest octant first), pushing the
// rest of the group. Returns false when the group and the stack are empty.
HDCX_D bool nextNode(uint2& group, uint2* stack, int& sp, int capacity, uint32_t octInv, uint32_t& nodeIndex,
                     uint32_t& fault)
{
    if ((group.y & 0xff000000u) == 0u) {
        if (sp == 0) return false;
        group = stack[--sp];
    }
    const uint32_t hitBits = group.y >> 24;
    const uint32_t pos = 31u - __clz(hitBits);
    group.y &= ~(1u << (24u + pos));
    const uint32_t childSlot = pos ^ octInv;
    nodeIndex = group.x + __popc((group.y & 0xffu) & ((1u << childSlot) - 1u));
    if ((group.y & 0xff000000u) != 0u) {
        if (sp < capacity) stack[sp++] = group;
        else fault |= kTraversalOverflow;
    }
    return true;
}

// The BLAS of instance `inst`; returns true for kAny at the first confirmed
// candidate, else updates `best`.
template <Accept kMode, bool kAny, bool kCount>
HDCX_D bool traceInstance(const DeviceScene& s, const RayPre& pre, float3 o, float3 d, float tmin, uint32_t rayRng,
                          uint32_t inst, ClosestHit& best, uint2* stack, uint2* work, uint32_t& fault)
{
    const InstanceDesc I = s.instances[inst];
    const BlasDesc B = s.blases[I.blas];
    float3 ro = o, rd = d;
    float margin = 0.0f;
    if (!I.identity) {
        const float ox = o.x - I.inv0.w, oy = o.y - I.inv1.w, oz = o.z - I.inv2.w;
        ro = make_float3((ox * I.inv0.x + oy * I.inv1.x) + oz * I.inv2.x, (ox * I.inv0.y + oy * I.inv1.y) + oz * I.inv2.y,
                         (ox * I.inv0.z + oy * I.inv1.z) + oz * I.inv2.z);
        rd = make_float3((d.x * I.inv0.x + d.y * I.inv1.x) + d.z * I.inv2.x, (d.x * I.inv0.y + d.y * I.inv1.y) + d.z * I.inv2.y,
                         (d.x * I.inv0.z + d.y * I.inv1.z) + d.z * I.inv2.z);
        // Rounding of the transformed ray: a few ulps of the magnitudes that
        // enter it, along the whole segment up to the current closest hit.
        margin = I.margin + 9.5367432e-7f * (maxAbs3(ro) + I.invNorm * maxAbs3(o) + fminf(best.t, 3.0e38f) * maxAbs3(rd));
    }
    const float3 id = inverseDirection(rd);
    const uint32_t octInv = octantMask(rd);
    const float mx = margin * fabsf(id.x), my = margin * fabsf(id.y), mz = margin * fabsf(id.z);
    uint2 group = B.nodeCount == 0u ? make_uint2(0u, 0u) : make_uint2(0u, (1u << (24u + octInv)) | 1u);
    uint2 tris = make_uint2(0u, 0u);
    int sp = 0;
    uint32_t budget = B.nodeCount + 1u;
    for (;;) {
        while (tris.y != 0u) {
            const int bit = __ffs(tris.y) - 1;
            tris.y &= tris.y - 1u;
            const uint32_t slot = tris.x + static_cast<uint32_t>(bit);
            const float4 w0 = __ldg(B.triVerts + slot * 3u + 0u);
            float3 v0, v1, v2;
            uint32_t prim;
            if (I.identity) {
                prim = __float_as_uint(w0.w);
                v0 = xyz(w0);
                v1 = xyz(__ldg(B.triVerts + slot * 3u + 1u));
                v2 = xyz(__ldg(B.triVerts + slot * 3u + 2u));
            } else {
                // The instance's flattened triangle: world-space vertices.
                prim = I.triBase + __float_as_uint(w0.w);
                v0 = xyz(__ldg(s.vertices + __ldg(s.indices + prim * 3u + 0u)));
                v1 = xyz(__ldg(s.vertices + __ldg(s.indices + prim * 3u + 1u)));
                v2 = xyz(__ldg(s.vertices + __ldg(s.indices + prim * 3u + 2u)));
            }
            if (kCount) work->y++;
            float t, b1, b2;
            if (!intersectTriangle(pre, v0, v1, v2, tmin, best.t, t, b1, b2)) continue;
            if (!confirmCandidate<kMode, kAny>(s, rayRng, prim, t, b1, b2, best)) continue;
            if (kAny) return true;
            best = ClosestHit{t, prim, b1, b2};
        }
        uint32_t nodeIndex;
        if (!nextNode(group, stack, sp, kTraversalStack, octInv, nodeIndex, fault)) return false;
        if (budget-- == 0u) {
            fault |= kTraversalBudget;
            return false;
        }
        if (kCount) work->x++;
        if (I.identity) {
            testNode<false>(B.nodes, nodeIndex, ro, id.x, id.y, id.z, octInv, best.t, 0.0f, 0.0f, 0.0f, group, tris);
        } else {
            testNode<true>(B.nodes, nodeIndex, ro, id.x, id.y, id.z, octInv, best.t, mx, my, mz, group, tris);
        }
    }
}

template <Accept kMode, bool kAny, bool kCount>
HDCX_D bool traceInstanced(const DeviceScene& s, float3 o, float3 d, float tmin, float tmax, uint32_t rayRng,
                           HitRecord& hit, uint2* work, uint32_t& fault)
{
    const RayPre pre = precomputeRay(o, d);
    const float3 id = inverseDirection(d);
    const uint32_t octInv = octantMask(d);
    ClosestHit best{tmax, kInvalidPrimitive, 0.0f, 0.0f};
    uint2 topStack[kTopStack];
    uint2 stack[kTraversalStack];
    uint2 group = make_uint2(0u, (1u << (24u + octInv)) | 1u);
    uint2 leaves = make_uint2(0u, 0u);
    int sp = 0;
    uint32_t budget = s.nodeCount + 1u;
    for (;;) {
        while (leaves.y != 0u) {
            const int bit = __ffs(leaves.y) - 1;
            leaves.y &= leaves.y - 1u;
            const uint32_t slot = leaves.x + static_cast<uint32_t>(bit);
            const uint32_t inst = __float_as_uint(__ldg(&s.triVerts[slot * 3u].w));
            if (traceInstance<kMode, kAny, kCount>(s, pre, o, d, tmin, rayRng, inst, best, stack, work, fault)) return true;
        }
        uint32_t nodeIndex;
        if (!nextNode(group, topStack, sp, kTopStack, octInv, nodeIndex, fault)) break;
        if (budget-- == 0u) {
            fault |= kTraversalBudget;
            break;
        }
        if (kCount) work->x++;
        testNode<false>(s.nodes, nodeIndex, o, id.x, id.y, id.z, octInv, best.t, 0.0f, 0.0f, 0.0f, group, leaves);
    }
    if (kAny || best.prim == kInvalidPrimitive) return false;
    hit.t = best.t;
    hit.primitive = best.prim;
    hit.b1 = best.b1;
    hit.b2 = best.b2;
    return true;
}

// Traverses the scene. kAny: stop at the first confirmed candidate.
// Returns true on a (confirmed) hit; for closest queries fills `hit`.
// kCount adds the wide nodes loaded to work.x and the triangle tests to work.y.
// kInst: 0 single-level scenes only, 1 two-level scenes only, -1 either
// (decided per call by DeviceScene::instances). Traversal faults are ORed
// into *fault.
template <Accept kMode, bool kAny, bool kCount = false, int kInst = -1>
HDCX_D bool traceRay(const DeviceScene& s, float3 o, float3 d, float tmin, float tmax, uint32_t rayRng, HitRecord& hit,
                     uint32_t& fault, uint2* work = nullptr)
{
    if (s.nodeCount == 0u) return false;
    if (kInst == 1 || (kInst == -1 && s.instances != nullptr))
        return traceInstanced<kMode, kAny, kCount>(s, o, d, tmin, tmax, rayRng, hit, work, fault);
    Traversal st;
    beginTraversal(st, s, o, d, tmin, tmax, rayRng);
    uint2 stack[kTraversalStack];
    int r;
    while ((r = traversalStep<kMode, kAny, kCount>(st, stack, s, work)) == kStepContinue) {
    }
    fault |= st.fault;
    if (kAny) return r == kStepAnyHit;
    if (st.bestPrim == kInvalidPrimitive) return false;
    hit.t = st.bestT;
    hit.primitive = st.bestPrim;
    hit.b1 = st.bestB1;
    hit.b2 = st.bestB2;
    return true;
}

}  // namespace hdcx
