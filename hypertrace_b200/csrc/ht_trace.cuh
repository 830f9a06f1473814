// ht_trace.cuh -- scene access and the per-hop path logic for the two scene recipes.
//
// Device-side restatement of render/scene.inl:16-44 (hop loop), object/vector.inl:24-74
// (nearest-hit scan), object/mapped.inl:24-51, object/covered.inl:23-56, the shapes in
// shape/hy/{plane,horosphere}.cc and shape/eu/{plane,sphere}.cc, the mixture material
// (material/mixture/impl.inl:16-27 with colored.inl, lambertian.cc, specular.cc,
// emissive.inl, absorbing.cc), the point camera (view/point/impl.inl:18-25,
// view/mapped.inl:20-26) and the constant background (background/constant.inl:18-21).
//
// Scheduling differs from the reference, results do not:
//  * the object scan keeps only (distance, index) per candidate and recomputes the
//    winner's local hit afterwards -- the same inputs through the same operations give the
//    same bits, so this equals keeping every candidate's light/cache copy;
//  * only the winner is mapped back to world space (the reference maps every candidate
//    back, mapped.inl:34, but only the kept copy is observable);
//  * inverse maps are computed once per launch and staged in shared memory.
#pragma once
#include "ht_math.cuh"
#include "ht_bound.cuh"

namespace ht {

constexpr int RECIPE_HY = 1;
constexpr int RECIPE_EU = 2;
constexpr float EPSF = 1e-6f;   // EPS for real = float (kernel/ocl/algebra/real.hh:19-25)
constexpr uint32_t HASH_NEVER = 0xFFFFFFFFu;  // hash_never (kernel/ocl/hash.cc:22-24)
constexpr uint32_t OBJ_STRIDE = 128;
constexpr uint32_t FLAG_JITTER_YX = 1u;

// Serialized scene byte offsets (see hypertrace_b200/scene.py for the derivation).
template <int R> struct Layout;
template <> struct Layout<RECIPE_HY> {
    static constexpr uint32_t FOV = 32, BG = 64, COUNT = 96, OBJECTS = 128;
};
template <> struct Layout<RECIPE_EU> {
    static constexpr uint32_t FOV = 32, BG = 48, COUNT = 64, OBJECTS = 80;
};
// Object record offsets (Mapped<Covered<Choice, Mixture>, Map>).
constexpr uint32_t O_DIFFUSE_COLOR = 32, O_DIFFUSE = 48, O_SPECULAR = 64, O_EMISSION = 80,
                   O_LUMINOUS = 96, O_SHAPE = 112;

struct Material {
    Col diffuse_color;
    float diffuse, specular, luminous;
    Col emission;
};

HT_D float ldf(const uint8_t *base, uint32_t off) { return __ldg(reinterpret_cast<const float *>(base + off)); }
HT_D float4 ldf4(const uint8_t *base, uint32_t off) { return __ldg(reinterpret_cast<const float4 *>(base + off)); }
HT_D uint32_t ldu(const uint8_t *base, uint32_t off) { return __ldg(reinterpret_cast<const uint32_t *>(base + off)); }

HT_D Material load_material(const uint8_t *obj) {
    Material m;
    float4 dc = ldf4(obj, O_DIFFUSE_COLOR);
    m.diffuse_color.x = dc.x; m.diffuse_color.y = dc.y; m.diffuse_color.z = dc.z;
    m.diffuse = ldf(obj, O_DIFFUSE);
    m.specular = ldf(obj, O_SPECULAR);
    float4 em = ldf4(obj, O_EMISSION);
    m.emission.x = em.x; m.emission.y = em.y; m.emission.z = em.z;
    m.luminous = ldf(obj, O_LUMINOUS);
    return m;
}

HT_D Mo load_mo(const uint8_t *p) {
    float4 a = ldf4(p, 0), b = ldf4(p, 16);
    Mo m;
    m.a.x = a.x; m.a.y = a.y; m.b.x = a.z; m.b.y = a.w;
    m.c.x = b.x; m.c.y = b.y; m.d.x = b.z; m.d.y = b.w;
    return m;
}
HT_D Hom load_hom(const uint8_t *p) {
    float4 a = ldf4(p, 0), b = ldf4(p, 16);
    Hom h;
    h.shift = v3(a.x, a.y, a.z);
    h.rot = q4(b.x, b.y, b.z, b.w);
    return h;
}
HT_D Mo mo_from(float4 a, float4 b) {
    Mo m;
    m.a.x = a.x; m.a.y = a.y; m.b.x = a.z; m.b.y = a.w;
    m.c.x = b.x; m.c.y = b.y; m.d.x = b.z; m.d.y = b.w;
    return m;
}
HT_D Hom hom_from(float4 a, float4 b) {
    Hom h;
    h.shift = v3(a.x, a.y, a.z);
    h.rot = q4(b.x, b.y, b.z, b.w);
    return h;
}

// Mixture interact: one uniform draw picks the component; returns false when the path ends
// (Emissive<Absorbing>, or the draw falls past every portion).
HT_D bool mixture_interact(const Material &m, uint32_t &rng, V3 normal, V3 &dir, Col &intensity,
                           Col &emission) {
    float alpha = rng_uniform(rng);
    alpha -= m.diffuse;
    if (alpha < 0.0f) {
        intensity.x *= m.diffuse_color.x;
        intensity.y *= m.diffuse_color.y;
        intensity.z *= m.diffuse_color.z;
        if (dot3(dir, normal) > 0.0f) normal = v3(-normal.x, -normal.y, -normal.z);
        V3 rnd = hemisphere_cosine(rng);
        Q4 rot = rot3_look_at(v3(-normal.x, -normal.y, -normal.z));
        dir = rot3_apply(rot, rnd);
        return true;
    }
    alpha -= m.specular;
    if (alpha < 0.0f) {
        float k = 2.0f * dot3(dir, normal);
        dir = v3(dir.x - k * normal.x, dir.y - k * normal.y, dir.z - k * normal.z);
        return true;
    }
    alpha -= m.luminous;
    if (alpha < 0.0f) {
        emission.x += intensity.x * m.emission.x;
        emission.y += intensity.y * m.emission.y;
        emission.z += intensity.z * m.emission.z;
        return false;
    }
    return false;
}

// Staged scene, per slot in shared memory (hyperbolic scenes: planes first, then
// horospheres, each in scene order; Euclidean scenes: slot = scene index).
struct StagedScene {
    const float4 *inv;       // shared, 2 per slot
    const uint32_t *shape;   // shared
    const float4 *bound;     // shared, 1 per slot: world-space form for distance bounds
    const float4 *pa, *pb;   // shared, per pair of slots: {x0, x1, y0, y1}, {z0, z1, w0, w1} of bound
    const float2 *pmag;      // shared, per pair of slots: {mag0, mag1}
    const float *mag;        // shared, 1 per slot: BOUND_EPS * max |bound component|
    const uint32_t *orig;    // shared, 1 per slot: the object's index in the scene
    float4 *win;             // shared, this thread's 2 float4: the scan winner's local ray
    const uint8_t *objects;  // global, OBJ_STRIDE per object (forward maps, materials), by scene index
    uint32_t n;              // objects
    uint32_t ns;             // slots: n, plus the dummy slot of a hyperbolic scene with an odd plane count
    uint32_t n_planes;       // hyperbolic: slots [0, n_planes) are planes, horospheres from the next even slot
    uint32_t dummy;          // the dummy slot, or 0xFFFFFFFF
    float fov;
    Col background;
    float4 cam0, cam1;       // camera map (Moebius or Homogenous3) as stored
};

// -------------------------------------------------------------------------- hyperbolic
struct HyPath { Q4 p, v; };

// Plane test up to the hit point (shape/hy/plane.cc:4-37 without the direction update);
// returns x of the hit distance (see hy_x), or -1 on a miss.
HT_D float plane_hy_x(Q4 p, Q4 d) {
    float pd = dot4(p, d);
    if (fabsf(pd) < EPSF) return -1.0f;
    float s = 1.0f - dot4(p, p);
    float t = s / (2.0f * pd);
    if (t < -EPSF) return -1.0f;
    float hx = p.x + d.x * t, hy = p.y + d.y * t;
    float pxy2 = dot2(hx, hy, hx, hy);
    if (pxy2 > 1.0f) return -1.0f;
    Q4 h = q4(hx, hy, sqrtf(1.0f - pxy2), 0.0f);
    return hy_x(p, h);
}
// Horosphere test up to the hit point (shape/hy/horosphere.cc:4-34); x or -1.
HT_D float horosphere_x(Q4 p, Q4 d, bool repeat) {
    float dxy = sqrtf(dot2(d.x, d.y, d.x, d.y));
    if (p.z < dxy) return -1.0f;
    float dt = sqrtf(p.z * p.z - dxy * dxy);
    float t = p.z * d.z - dt;
    float w = repeat ? EPSF : -EPSF;   // EPS * (2*repeat - 1)
    if (t < w) {
        t += 2.0f * dt;
        if (t < w) return -1.0f;
    }
    t /= dxy * dxy;
    Q4 h = q4(p.x + d.x * t, p.y + d.y * t, 1.0f, 0.0f);
    return hy_x(p, h);
}
// Full tests for the winning object: hit point, transported direction, local normal.
HT_D void plane_hy_hit(Q4 p, Q4 d, HyPath &hit, Q4 &normal) {
    float pd = dot4(p, d);
    float s = 1.0f - dot4(p, p);
    float t = s / (2.0f * pd);
    float hx = p.x + d.x * t, hy = p.y + d.y * t;
    float pxy2 = dot2(hx, hy, hx, hy);
    Q4 h = q4(hx, hy, sqrtf(1.0f - pxy2), 0.0f);
    hit.p = h;
    hit.v = hy_dir_at(p, d, h);
    normal = q4(-h.x, -h.y, -h.z, -h.w);
}
HT_D void horosphere_hit(Q4 p, Q4 d, bool repeat, HyPath &hit, Q4 &normal) {
    float dxy = sqrtf(dot2(d.x, d.y, d.x, d.y));
    float dt = sqrtf(p.z * p.z - dxy * dxy);
    float t = p.z * d.z - dt;
    float w = repeat ? EPSF : -EPSF;
    if (t < w) t += 2.0f * dt;
    t /= dxy * dxy;
    Q4 h = q4(p.x + d.x * t, p.y + d.y * t, 1.0f, 0.0f);
    hit.p = h;
    hit.v = hy_dir_at(p, d, h);
    normal = q4(0.0f, 0.0f, -1.0f, 0.0f);
}

// Camera ray: view/point/impl.inl:18-25 (hy_origin = j, hyperbolic.cc:4-6) then the
// camera Moebius map (view/mapped.inl:20-26).
// Out of line: once per sample, and keeping its code out of the hop kernel's instruction
// stream measured 3 % faster at 1920x1080 / 200 objects.
static __device__ __noinline__ HyPath camera_hy(const StagedScene &s, float px, float py, float size, uint32_t &rng,
                                                uint32_t flags) {
    float u0 = rng_uniform(rng);
    float u1 = rng_uniform(rng);
    float jx = (flags & FLAG_JITTER_YX) ? u1 : u0;
    float jy = (flags & FLAG_JITTER_YX) ? u0 : u1;
    float sx = px + size * (jx - 0.5f);
    float sy = py + size * (jy - 0.5f);
    V3 ld = normalize3(v3(sx, sy, -1.0f / s.fov));
    HyRay r = view_hy_map(mo_from(s.cam0, s.cam1), q4(0.0f, 0.0f, 1.0f, 0.0f), q4(ld.x, ld.y, ld.z, 0.0f));
    HyPath o; o.p = r.p; o.v = r.v;
    return o;
}

// One hop (one iteration of render/scene.inl:25-41). Returns true while the path goes on.
// `hit` reports whether the scan found an object (for the hop statistics).
// ---------------------------------------------------------------- the scan's packed point bound
// Objects the upper estimate looks at (the first ones in index order).
#ifndef HT_EST_OBJECTS
#define HT_EST_OBJECTS 24u   // 12 planes + 12 horospheres: 492.6 Msamples/s at 1080p, 16: 480.4, 32: 485.8, 40: 470.3
#endif
struct PairRay { float2 r2, x, y, K; };   // the bound ray's constants, each in both halves
HT_D PairRay pair_ray(const BoundRay &r) {
    PairRay p;
    p.r2 = make_float2(r.r2, r.r2);
    p.x = make_float2(r.x, r.x);
    p.y = make_float2(r.y, r.y);
    p.K = make_float2(r.K, r.K);
    return p;
}
HT_D uint32_t survivors2(float4 a, float4 b, float2 mag, const PairRay &r, const PointCut &k) {
    // F = rec.x r2 + (rec.y x + (rec.z y + rec.w)), as culled_point evaluates it
    float2 F = __ffma2_rn(make_float2(b.x, b.y), r.y, make_float2(b.z, b.w));
    F = __ffma2_rn(make_float2(a.z, a.w), r.x, F);
    F = __ffma2_rn(make_float2(a.x, a.y), r.r2, F);
    const float2 e = __fmul2_rn(mag, r.K);                      // eF, once for both sides
    const float2 up = __fadd2_rn(F, e);                          // F + eF
    const float2 dn = __fadd2_rn(F, make_float2(-e.x, -e.y));   // F - eF
    const bool c0 = up.x < k.lo.x || dn.x > k.hi.x;
    const bool c1 = up.y < k.lo.y || dn.y > k.hi.y;
    return (c0 ? 0u : 1u) | (c1 ? 0u : 2u);
}
HT_D bool culled_slot(const StagedScene &s, uint32_t q, const BoundRay &r, const PointCut &kp, const PointCut &kh) {
    return culled_point(s.bound[q], s.mag[q], r, s.shape[q] == 0 ? kp : kh);
}

// Upper estimate of the nearest hit that the reference surely reports (the least
// sure_crossing_e2) among the first HT_EST_OBJECTS / 2 planes and the first HT_EST_OBJECTS / 2
// horospheres of the staged slots, +inf when none qualifies. A threshold derived from it
// (cull_from_dist) then culls before the first exact test.
HT_D float est_range(const StagedScene &s, uint32_t q0, uint32_t q1, const BoundRay &r, uint32_t prev_hash, float best) {
    for (uint32_t q = q0; q < q1; ++q)   // warp-uniform: broadcast loads
        best = fminf(best, sure_crossing_e2(bound_fw(s.bound[q], s.mag[q], r), s.shape[q], s.orig[q] == prev_hash, r.t));
    return best;
}
HT_D float upper_estimate(const StagedScene &s, const BoundRay &r, uint32_t prev_hash) {
    const uint32_t half = HT_EST_OBJECTS / 2, h0 = (s.n_planes + 1) & ~1u;
    float best = est_range(s, 0, min(half, s.n_planes), r, prev_hash, __int_as_float(0x7f800000));
    best = est_range(s, h0, min(h0 + half, s.ns), r, prev_hash, best);
    return best < __int_as_float(0x7f800000) ? dist_from_e2(best) : best;
}

// Warp pre-cull (wavefront kernels, full warps whose lanes can all cull): each lane tests
// one slot of a 32-slot chunk against the whole warp at once — F over the box of the lanes'
// (|p|^2, x, y), the largest error allowance and the loosest thresholds of the warp — and a
// slot the warp test culls is culled by every lane's own point test, so the lanes run that
// test only on the pairs the warp keeps and reach the same candidate masks bit for bit. The
// warp test adds a slack of 2^-16 of the magnitudes involved, far above the rounding of
// either evaluation (a few units of 2^-24 each), so float rounding cannot break that
// implication. After the coherence sort a warp's rays start in one cell, the box is small,
// and most slots go in one test per warp instead of one per lane.
struct WarpBox { float r2lo, r2hi, xlo, xhi, ylo, yhi, K; };
HT_D uint32_t ord_bits(float f) {   // order-preserving map of floats (no NaN) to unsigned
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
HT_D float ord_float(uint32_t o) { return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o); }
HT_D float warp_min(float f) { return ord_float(__reduce_min_sync(0xffffffffu, ord_bits(f))); }
HT_D float warp_max(float f) { return ord_float(__reduce_max_sync(0xffffffffu, ord_bits(f))); }
HT_D WarpBox warp_box(const BoundRay &r) {
    WarpBox b;
    b.r2lo = warp_min(r.r2); b.r2hi = warp_max(r.r2);
    b.xlo = warp_min(r.x);   b.xhi = warp_max(r.x);
    b.ylo = warp_min(r.y);   b.yhi = warp_max(r.y);
    b.K = warp_max(r.K);
    return b;
}
// interval of a * u over u in [lo, hi], and a bound of |a u| there
HT_D void box_term(float a, float lo, float hi, float &flo, float &fhi, float &mag) {
    const float p = a * lo, q = a * hi;
    flo += fminf(p, q);
    fhi += fmaxf(p, q);
    mag += fmaxf(fabsf(p), fabsf(q));
}
// Slots of chunk [c0, c0 + cn) that some lane of the warp may keep (every lane calls this).
HT_D uint32_t warp_survivors(const StagedScene &s, uint32_t c0, uint32_t valid, const WarpBox &b,
                             const PointCut &kp, const PointCut &kh) {
    const uint32_t lane = threadIdx.x & 31;
    const float hp = warp_max(kp.hi.x);   // planes: lo = -hi
    const float lh = warp_min(kh.lo.x), hh = warp_max(kh.hi.x);
    bool keep = false;
    if (valid >> lane & 1u) {
        const uint32_t q = c0 + lane;
        const float4 rec = s.bound[q];
        const float e = s.mag[q] * b.K;
        float flo = rec.w, fhi = rec.w, mag = fabsf(rec.w);
        box_term(rec.x, b.r2lo, b.r2hi, flo, fhi, mag);
        box_term(rec.y, b.xlo, b.xhi, flo, fhi, mag);
        box_term(rec.z, b.ylo, b.yhi, flo, fhi, mag);
        const float slack = 0x1p-16f * (mag + e);
        float lo = lh, hi = hh;
        if (s.shape[q] == 0) {
            lo = -hp;
            hi = hp;
        }
        keep = !((fhi + e) + slack < lo || (flo - e) - slack > hi);   // NaN: kept
    }
    return __ballot_sync(0xffffffffu, keep);
}

// WARP: the warp pre-cull is compiled in; `full_warp` (all 32 lanes of the warp are in this
// call together, uniform across the warp) turns it on.
template <bool OOL, bool WARP = false>
HT_D bool hop_hy(const StagedScene &s, HyPath &ray, uint32_t &rng, uint32_t &prev_hash,
                 Col &intensity, Col &emission, bool &hit, uint32_t &n_exact, bool full_warp = false) {
    // Nearest hit with ties to the lowest scene index (object/vector.inl:37-50): candidates
    // are compared on (distance, index), so the order of the slots does not matter; x =
    // cosh(distance) is compared first and the logarithm taken only when x can win; objects
    // whose distance bound rules them out are not tested.
    float min_dist = -1.0f;
    float min_x = __int_as_float(0x7f800000);   // +inf
    uint32_t kmin = 0, kmin_orig = 0xFFFFFFFFu;
    const Q4 p = ray.p, v = ray.v;
    const bool can_cull = cull_point_ok(p);
    const BoundRay br = bound_ray(p, v);
    const PairRay pr = pair_ray(br);
    Cull cull = cull_none();
    if (can_cull) {   // a threshold before the first exact test, from the first slots' crossings
        const float u = upper_estimate(s, br, prev_hash);
        if (u < __int_as_float(0x7f800000)) cull = cull_from_dist(u);
    }
    PointCut kp = point_cut(0, br.t, cull), kh = point_cut(1, br.t, cull);
    bool warp_pre = false;
    WarpBox wb;
    if constexpr (WARP) {
        if (full_warp) {
            __syncwarp();
            warp_pre = __all_sync(0xffffffffu, can_cull);
            if (warp_pre) wb = warp_box(br);
        }
    }
    for (uint32_t c0 = 0; c0 < s.ns; c0 += 32) {
        const uint32_t cn = min(32u, s.ns - c0);
        uint32_t valid = cn == 32 ? 0xFFFFFFFFu : (1u << cn) - 1u;
        if (s.dummy - c0 < 32u) valid &= ~(1u << (s.dummy - c0));
        uint32_t mask = valid;
        if (can_cull) {
            mask = 0;
            if constexpr (WARP) {
                // one copy of the pair loop for both cases (instruction fetch): over the pairs
                // with a slot the warp keeps, or over every valid pair without the warp test
                uint32_t keep = valid;
                if (warp_pre) {   // uniform: every lane can cull
                    __syncwarp();
                    keep = warp_survivors(s, c0, valid, wb, kp, kh);
                }
                uint32_t pm = (keep | (keep >> 1)) & 0x55555555u;
                while (pm) {   // this lane's point test
                    const uint32_t j = __ffs(pm) - 1;
                    pm &= pm - 1;
                    const uint32_t pq = (c0 + j) >> 1;
                    const PointCut &k = c0 + j >= s.n_planes ? kh : kp;
                    mask |= survivors2(s.pa[pq], s.pb[pq], s.pmag[pq], pr, k) << j;
                }
                mask &= keep;
            } else {
                // kept rolled: the kernel is bound by instruction fetch as much as by issue
#pragma unroll 1
                for (uint32_t j = 0; j < cn; j += 2) {   // warp-uniform: broadcast loads, two slots at once
                    const uint32_t pq = (c0 + j) >> 1;
                    const PointCut &k = c0 + j >= s.n_planes ? kh : kp;
                    mask |= survivors2(s.pa[pq], s.pb[pq], s.pmag[pq], pr, k) << j;
                }
            }
            mask &= valid;
            // per lane: the ray-aware bound on the survivors only
            uint32_t m = mask;
            while (m) {
                const uint32_t j = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t q = c0 + j;
                if (culled<OOL>(s.bound[q], s.mag[q], s.shape[q], br, cull)) mask &= ~(1u << j);
            }
        }
        while (mask) {   // this lane's candidates, in slot order
            const uint32_t q = c0 + (__ffs(mask) - 1);
            mask &= mask - 1;
            const uint32_t shape = s.shape[q];
            if (can_cull && culled_slot(s, q, br, kp, kh)) continue;
            const uint32_t k = s.orig[q];
            const bool repeat = (k == prev_hash);
            if (shape == 0 && repeat) continue;   // a geodesic plane is never hit twice in a row
            ++n_exact;
            // the out-of-line copy of the map, shared with the hit path: one copy of its code
            // (the kernel is bound by instruction fetch as much as by issue)
            HyRay l = ray_hy_map_call(mo_from(s.inv[2 * q], s.inv[2 * q + 1]), p, v);
            const float x = shape == 0 ? plane_hy_x(l.p, l.v) : horosphere_x(l.p, l.v, repeat);
            // x above the best's gives a distance no smaller (hy_dist_from_x is non-decreasing),
            // which can only win a tie, and only from a lower scene index
            if (x >= 1.0f && (x <= min_x || k < kmin_orig)) {
                const float dist = hy_dist_from_x(x);
                if (dist > -EPSF && (min_dist <= -EPSF || dist < min_dist || (dist == min_dist && k < kmin_orig))) {
                    min_dist = dist;
                    min_x = x;
                    kmin = q;
                    kmin_orig = k;
                    cull = cull_from_dist(dist);
                    kp = point_cut(0, br.t, cull);
                    kh = point_cut(1, br.t, cull);
                    s.win[0] = make_float4(l.p.x, l.p.y, l.p.z, l.p.w);   // kept for the hit
                    s.win[1] = make_float4(l.v.x, l.v.y, l.v.z, l.v.w);
                }
            }
        }
    }
    if (!(min_dist > -EPSF)) {
        hit = false;
        emission.x += s.background.x * intensity.x;
        emission.y += s.background.y * intensity.y;
        emission.z += s.background.z * intensity.z;
        return false;
    }
    hit = true;
    const Mo inv = mo_from(s.inv[2 * kmin], s.inv[2 * kmin + 1]);
    const uint8_t *obj = s.objects + (size_t)kmin_orig * OBJ_STRIDE;
    const Mo fwd = load_mo(obj);
    const bool repeat = (kmin_orig == prev_hash);
    HyRay l;   // the winner's local ray, as the scan computed it (the same map, the same bits)
    {
        const float4 a = s.win[0], b = s.win[1];
        l.p = q4(a.x, a.y, a.z, a.w);
        l.v = q4(b.x, b.y, b.z, b.w);
    }
    HyPath lh;
    Q4 normal;
    if (s.shape[kmin] == 0) plane_hy_hit(l.p, l.v, lh, normal);
    else horosphere_hit(l.p, l.v, repeat, lh, normal);
    HyRay w = ray_hy_map_call(fwd, lh.p, lh.v);          // detect: map back (mapped.inl:34)
    HyRay loc = ray_hy_map_call(inv, w.p, w.v);          // interact: to local (mapped.inl:46-47)
    Material m = load_material(obj);
    V3 dir = v3(loc.v.x, loc.v.y, loc.v.z);          // light_hy_to_local (light/hy.cc:3-8)
    bool ret = mixture_interact(m, rng, v3(normal.x, normal.y, normal.z), dir, intensity, emission);
    HyRay out = ray_hy_map_call(fwd, loc.p, q4(dir.x, dir.y, dir.z, 0.0f));  // mapped.inl:49
    ray.p = out.p;
    ray.v = out.v;
    if (!ret) return false;
    prev_hash = kmin_orig;   // the hasher state after hash_usize(0, index) is the index
    return true;
}

// -------------------------------------------------------------------------- euclidean
struct EuPath { V3 p, v; };

HT_D float sphere_eu_dist(V3 pos, V3 dir, bool repeat) {   // shape/eu/sphere.cc:3-29
    float b = -dot3(dir, pos);
    V3 g = v3(pos.x + dir.x * b, pos.y + dir.y * b, pos.z + dir.z * b);
    float d = 1.0f - dot3(g, g);
    if (d < 0.0f) return -1.0f;
    d = sqrtf(d);
    float e = b - d;
    float w = repeat ? EPSF : -EPSF;
    if (e < w) {
        e = b + d;
        if (e < w) return -1.0f;
    }
    return e;
}
HT_D float plane_eu_dist(V3 pos, V3 dir) {   // shape/eu/plane.cc:3-21 (repeat handled by caller)
    if (pos.z * dir.z > 0.0f) return -1.0f;
    return -pos.z / dir.z;
}

HT_D EuPath camera_eu(const StagedScene &s, float px, float py, float size, uint32_t &rng, uint32_t flags) {
    float u0 = rng_uniform(rng);
    float u1 = rng_uniform(rng);
    float jx = (flags & FLAG_JITTER_YX) ? u1 : u0;
    float jy = (flags & FLAG_JITTER_YX) ? u0 : u1;
    float sx = px + size * (jx - 0.5f);
    float sy = py + size * (jy - 0.5f);
    V3 ld = normalize3(v3(sx, sy, -1.0f / s.fov));
    Hom cam = hom_from(s.cam0, s.cam1);
    EuPath o;
    o.v = rot3_apply(cam.rot, ld);                       // hom3_apply_dir: not normalized
    o.p = hom3_apply_pos(cam, v3(0.0f, 0.0f, 0.0f));
    return o;
}

HT_D bool hop_eu(const StagedScene &s, EuPath &ray, uint32_t &rng, uint32_t &prev_hash,
                 Col &intensity, Col &emission, bool &hit, uint32_t &n_exact) {
    n_exact += s.n;
    float min_dist = -1.0f;
    uint32_t kmin = 0;
    const V3 p = ray.p, v = ray.v;
    for (uint32_t k = 0; k < s.n; ++k) {
        const uint32_t shape = s.shape[k];
        const bool repeat = (k == prev_hash);
        float dist = -1.0f;
        if (shape == 0) {
            if (!repeat) {
                EuRay l = ray_eu_map(hom_from(s.inv[2 * k], s.inv[2 * k + 1]), p, v);
                dist = plane_eu_dist(l.p, l.v);
            }
        } else {
            EuRay l = ray_eu_map(hom_from(s.inv[2 * k], s.inv[2 * k + 1]), p, v);
            dist = sphere_eu_dist(l.p, l.v, repeat);
        }
        if (dist > -EPSF && (min_dist <= -EPSF || dist < min_dist)) {
            min_dist = dist;
            kmin = k;
        }
    }
    if (!(min_dist > -EPSF)) {
        hit = false;
        emission.x += s.background.x * intensity.x;
        emission.y += s.background.y * intensity.y;
        emission.z += s.background.z * intensity.z;
        return false;
    }
    hit = true;
    const Hom inv = hom_from(s.inv[2 * kmin], s.inv[2 * kmin + 1]);
    const uint8_t *obj = s.objects + (size_t)kmin * OBJ_STRIDE;
    const Hom fwd = load_hom(obj);
    EuRay l = ray_eu_map(inv, p, v);
    EuPath lh;
    V3 normal;
    lh.v = l.v;
    if (s.shape[kmin] == 0) {
        float t = -l.p.z / l.v.z;
        lh.p = v3(l.p.x + l.v.x * t, l.p.y + l.v.y * t, 0.0f);
        normal = v3(0.0f, 0.0f, -1.0f);
    } else {
        float e = sphere_eu_dist(l.p, l.v, kmin == prev_hash);
        V3 h = normalize3(v3(l.p.x + l.v.x * e, l.p.y + l.v.y * e, l.p.z + l.v.z * e));
        lh.p = h;
        normal = h;
    }
    EuRay w = ray_eu_map(fwd, lh.p, lh.v);
    EuRay loc = ray_eu_map(inv, w.p, w.v);
    Material m = load_material(obj);
    V3 dir = loc.v;
    bool ret = mixture_interact(m, rng, normal, dir, intensity, emission);
    EuRay out = ray_eu_map(fwd, loc.p, dir);
    ray.p = out.p;
    ray.v = out.v;
    if (!ret) return false;
    prev_hash = kmin;
    return true;
}

}  // namespace ht
