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
// ---------------------------------------------------------------- distance bounds
// The object scan only needs the exact (reference) test for objects that can be hit nearer
// than the best hit found so far. Whether and where the geodesic ray from (p, v) meets an
// object has a closed form in world space, evaluated here with explicit error terms and wide
// margins; objects it rules out are not tested. This changes which objects are evaluated,
// never the result. Per object one float4 `rec`, staged once per launch (stage_bound):
//   geodesic plane  rec = (A, 2Re B, 2Im B, C): the world plane's normalised Hermitian form,
//                   |B|^2 - A C = 1. F = rec . (|p|^2, x, y, 1) = Q and sinh(signed distance
//                   to the plane) = Q / (2t); along the unit-speed geodesic it is exactly
//                   a cosh s + b sinh s with a = F / 2t, b = W / 2t, so the ray meets the plane
//                   at s* = atanh(-a/b) when 0 <= -a/b < 1.
//   horosphere      rec = (|n21|^2, 2 Re w, -2 Im w, |n22|^2), w = conj(n22) n21, N = M^-1
//                   normalised to det 1: F = rec . (|p|^2, x, y, 1) = t / t' (t' = local
//                   height; inside the horoball when t' > 1). Along the geodesic
//                   1/t' = P cosh s + V sinh s with P = F / t, V = W / t; it crosses 1 at
//                   e^s = (P - V) / (1 + r) (entry) and (1 + r) / (P + V) (exit), r^2 = 1 - P^2 + V^2.
//   both            W = t (2 rec.x (p.v) + rec.y v.x + rec.z v.y) - F v.z
// with p = (x, y, t) the ray start, v its unit direction (v.z along the height).
// The threshold is thr = best (1 + CULL_REL) + CULL_ABS; objects with large map entries get
// NaN records (never culled) and ray starts outside a well-conditioned box disable culling.
constexpr float CULL_REL = 1e-2f, CULL_ABS = 1e-2f;

constexpr float BOUND_EPS = 1e-5f;   // relative error allowance of F and W (>> f32 rounding)
constexpr float HORO_M = 1e-3f;      // relative margin of the horosphere root bounds
// Objects the upper estimate looks at (the first ones in index order).
#ifndef HT_EST_OBJECTS
#define HT_EST_OBJECTS 32u
#endif

// Hardware approximations (PTX rcp / sqrt / lg2 / ex2 .approx, relative error near 2^-22) for
// the bound arithmetic only: every quantity they produce carries a margin of at least 1e-6
// relative (the threshold itself 1e-2), so they never decide a culling the exact values
// would not allow. The path's own arithmetic (ray maps, shape tests) never uses them.
HT_D float rcp_approx(float x) { float r; asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
HT_D float sqrt_approx(float x) { float r; asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
HT_D float lg2_approx(float x) { float r; asm("lg2.approx.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
HT_D float ex2_approx(float x) { float r; asm("ex2.approx.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
constexpr float LN2F = 0.693147180559945f, LOG2EF = 1.442695040888963f;

// Error allowance of F for one object: BOUND_EPS * max |rec component|, so that
// eF = mag * (|p|^2 + |x| + |y| + 1) >= BOUND_EPS * sum of |terms| of F (one multiply per object).
HT_D float bound_mag(float4 rec) {
    return BOUND_EPS * fmaxf(fmaxf(fabsf(rec.x), fabsf(rec.y)), fmaxf(fabsf(rec.z), fabsf(rec.w)));
}

struct Cull { float S, E, T; };   // sinh, exp, tanh of the threshold; S = E = inf, T = 1: none

// World-space bound record of one object from its f32 map M, in FP64 (once per launch).
// N = adj(M) maps world to local (c22_inverse_n, matrix_complex.cc:60-65).
HT_D float4 stage_bound(const Mo &m, uint32_t shape) {
    const double ar = m.a.x, ai = m.a.y, br = m.b.x, bi = m.b.y;
    const double cr = m.c.x, ci = m.c.y, dr = m.d.x, di = m.d.y;
    const double det_r = (ar * dr - ai * di) - (br * cr - bi * ci);
    const double det_i = (ar * di + ai * dr) - (br * ci + bi * cr);
    const double adet = sqrt(det_r * det_r + det_i * det_i);
    const double maxe = fmax(fmax(fabs(ar) + fabs(ai), fabs(br) + fabs(bi)), fmax(fabs(cr) + fabs(ci), fabs(dr) + fabs(di)));
    const float nan = __int_as_float(0x7fc00000);
    if (!(maxe <= 32.0 && adet >= 0.5 && adet <= 2.0)) return make_float4(nan, nan, nan, nan);
    // N = [[n11, n12], [n21, n22]] = [[d, -b], [-c, a]]
    const double n11r = dr, n11i = di, n12r = -br, n12i = -bi, n21r = -cr, n21i = -ci, n22r = ar, n22i = ai;
    if (shape == 0) {
        const double A = (n11r * n11r + n11i * n11i) - (n21r * n21r + n21i * n21i);
        // B = conj(n11) n12 - conj(n21) n22
        const double Br = (n11r * n12r + n11i * n12i) - (n21r * n22r + n21i * n22i);
        const double Bi = (n11r * n12i - n11i * n12r) - (n21r * n22i - n21i * n22r);
        const double C = (n12r * n12r + n12i * n12i) - (n22r * n22r + n22i * n22i);
        return make_float4((float)(A / adet), (float)(2.0 * Br / adet), (float)(2.0 * Bi / adet), (float)(C / adet));
    }
    // horosphere: scale N by 1 / sqrt|det| so the height formula holds
    const double k2 = 1.0 / adet;
    const double c2 = (n21r * n21r + n21i * n21i) * k2;
    const double wr = (n22r * n21r + n22i * n21i) * k2;   // w = conj(n22) n21
    const double wi = (n22r * n21i - n22i * n21r) * k2;
    const double n22sq = (n22r * n22r + n22i * n22i) * k2;
    return make_float4((float)c2, (float)(2.0 * wr), (float)(-2.0 * wi), (float)n22sq);
}

// Per-hop constants of the bound evaluation.
struct BoundRay {
    float x, y, t, r2, pv, vx, vy, vz, ax, ay;
    float K;    // |p|^2 + |x| + |y| + 1: eF = mag * K
    float Kw;   // t (2 |p.v| + |vx| + |vy|): the part of eW that scales with mag
};
HT_D bool cull_point_ok(Q4 p) {
    return p.z >= 0x1p-20f && p.z <= 0x1p20f && fabsf(p.x) + fabsf(p.y) <= 0x1p10f * p.z &&
           fabsf(p.w) <= 1e-3f * p.z;
}
HT_D BoundRay bound_ray(Q4 p, Q4 v) {
    BoundRay b;
    b.x = p.x; b.y = p.y; b.t = p.z;
    b.r2 = fmaf(p.x, p.x, fmaf(p.y, p.y, p.z * p.z));
    b.pv = fmaf(p.x, v.x, fmaf(p.y, v.y, p.z * v.z));
    b.vx = v.x; b.vy = v.y; b.vz = v.z;
    b.ax = fabsf(p.x); b.ay = fabsf(p.y);
    b.K = b.r2 + b.ax + b.ay + 1.0f;
    b.Kw = b.t * (2.0f * fabsf(b.pv) + fabsf(b.vx) + fabsf(b.vy));
    return b;
}
// eF and eW of one object (the bounds of the float error of F and W)
HT_D float bound_eF(float mag, const BoundRay &r) { return mag * r.K; }
HT_D float bound_eW(float mag, float eF, float W, const BoundRay &r) {
    return fmaf(mag, r.Kw, fmaf(eF, fabsf(r.vz), BOUND_EPS * fabsf(W)));
}
// S, E, T are upper bounds of sinh, exp, tanh of the threshold: E from ex2.approx raised by
// 1e-5 relative (more than its error plus the rounding of thr * log2(e) for thr < 89, above
// which it is +inf), S and T increasing functions of it.
HT_D Cull cull_from_dist(float d) {
    const float thr = fmaf(d, 1.0f + CULL_REL, CULL_ABS);
    Cull c;
    c.E = ex2_approx(thr * LOG2EF) * (1.0f + 1e-5f);
    c.S = 0.5f * (c.E - rcp_approx(c.E));
    c.T = 1.0f - 2.0f * rcp_approx(fmaf(c.E, c.E, 1.0f));
    return c;
}
HT_D Cull cull_none() {
    Cull c;
    c.S = c.E = __int_as_float(0x7f800000);
    c.T = 1.0f;
    return c;
}
// Cheap bound: the distance from the ray start to the object alone (any hit lies on it),
// F = rec . (|p|^2, x, y, 1) with its error allowance eF:
//   geodesic plane  culled when |F| - eF > 2 t S (sinh of the distance to the plane);
//   horosphere      culled when t > E (F + eF) or t E < F - eF (the local height t' = t / F
//                   outside [e^-thr, e^thr] even with F's error).
// The point bound of two slots of one shape at once (packed FP32: each component rounds as the
// scalar operation does). An object is culled when F + eF < lo or F - eF > hi:
//   geodesic plane  lo = -2 t S, hi = 2 t S: the same decision as |F| - eF > 2 t S, op for
//                   op (|F| - eF = -(F + eF) exactly when F < 0);
//   horosphere      lo = t / E (E an upper bound of e^thr raised by 1e-5, so this stays below
//                   t e^-thr after its rounding and the rcp approximation), hi = t E: the
//                   test t > E (F + eF) or t E < F - eF with the division moved to the threshold.
// A NaN record (ill-conditioned map) is never culled. Returns the survivors as bits 0 and 1.
struct PointCut { float2 lo, hi; };
HT_D PointCut point_cut(uint32_t shape, float t, const Cull &c) {
    PointCut k;
    if (shape == 0) {
        const float h = 2.0f * t * c.S;
        k.lo = make_float2(-h, -h);
        k.hi = make_float2(h, h);
    } else {
        const float l = t * rcp_approx(c.E), h = t * c.E;
        k.lo = make_float2(l, l);
        k.hi = make_float2(h, h);
    }
    return k;
}
struct PairRay { float2 r2, x, y, K, nK; };   // the bound ray's constants, each in both halves
HT_D PairRay pair_ray(const BoundRay &r) {
    PairRay p;
    p.r2 = make_float2(r.r2, r.r2);
    p.x = make_float2(r.x, r.x);
    p.y = make_float2(r.y, r.y);
    p.K = make_float2(r.K, r.K);
    p.nK = make_float2(-r.K, -r.K);
    return p;
}
HT_D uint32_t survivors2(float4 a, float4 b, float2 mag, const PairRay &r, const PointCut &k) {
    // F = rec.x r2 + (rec.y x + (rec.z y + rec.w)), as culled_point evaluates it
    float2 F = __ffma2_rn(make_float2(b.x, b.y), r.y, make_float2(b.z, b.w));
    F = __ffma2_rn(make_float2(a.z, a.w), r.x, F);
    F = __ffma2_rn(make_float2(a.x, a.y), r.r2, F);
    const float2 up = __fadd2_rn(F, __fmul2_rn(mag, r.K));     // F + eF
    const float2 dn = __fadd2_rn(F, __fmul2_rn(mag, r.nK));    // F - eF (m (-K) = -(m K) exactly)
    const bool c0 = up.x < k.lo.x || dn.x > k.hi.x;
    const bool c1 = up.y < k.lo.y || dn.y > k.hi.y;
    return (c0 ? 0u : 1u) | (c1 ? 0u : 2u);
}
HT_D bool culled_slot(const StagedScene &s, uint32_t q, const BoundRay &r, const PointCut &kp, const PointCut &kh) {
    const float4 rec = s.bound[q];
    const float F = fmaf(rec.x, r.r2, fmaf(rec.y, r.x, fmaf(rec.z, r.y, rec.w)));
    const float eF = s.mag[q] * r.K;
    const PointCut &k = s.shape[q] == 0 ? kp : kh;
    return F + eF < k.lo.x || F - eF > k.hi.x;
}

// true when object `rec` provably cannot be hit nearer than the current threshold
// F, W of one object along the ray and the bounds of their float error
struct BoundFW { float F, eF, W, eW; };
HT_D BoundFW bound_fw(float4 rec, float mag, const BoundRay &r) {
    BoundFW b;
    b.F = fmaf(rec.x, r.r2, fmaf(rec.y, r.x, fmaf(rec.z, r.y, rec.w)));
    b.eF = bound_eF(mag, r);
    const float G = fmaf(2.0f * rec.x, r.pv, fmaf(rec.y, r.vx, rec.z * r.vy));
    b.W = fmaf(r.t, G, -b.F * r.vz);
    b.eW = bound_eW(mag, b.eF, b.W, r);
    return b;
}
HT_D bool culled_fw(const BoundFW &b, uint32_t shape, float t, const Cull &c) {
    const float F = b.F, eF = b.eF, W = b.W, eW = b.eW;
    if (shape == 0) {
        const float Fa = fabsf(F) - eF;       // lower bound of |2 t a|
        const float Wlo = fabsf(W) - eW, Whi = fabsf(W) + eW;
        // starts off the plane and moves away from it: |a| > 0.01, |b| > 0.001, same signs
        const bool away = (F > 0.0f) == (W > 0.0f) && Fa > 0.02f * t && Wlo > 0.002f * t;
        // |a| > 1.01 T |b| + 0.01: no root (T = 1) or the root lies beyond the threshold
        const bool far = Fa > fmaf(1.01f * c.T, Whi, 0.02f * t);
        // the start point itself is farther than the threshold
        const bool point = Fa > 2.0f * t * c.S;
        return away || far || point;
    } else {
        // In the object's frame the reference's horosphere test (shape/hy/horosphere.cc:4-34)
        // looks at two roots; with P = F/t (1 / local height), V = W/t (its derivative along
        // the ray), r^2 = 1 - P^2 + V^2 their parameters are t1 = -(V + rP)/P^2 and
        // t2 = (rP - V)/P^2, and a root is reported only when its parameter is >= -EPS (it
        // accepts roots up to EPS behind the start, before dividing by |d.xy|^2). The roots
        // are the crossings at e^s = (P - V)/(1 + r) and (1 + r)/(P + V). The object is
        // culled when every root that can be reported lies farther than the threshold.
        const float Flo = F - eF, Fhi = F + eF, Wlo = W - eW, Whi = W + eW;
        const float aWlo = fmaxf(fabsf(W) - eW, 0.0f), aWhi = fabsf(W) + eW;
        if (t > c.E * Fhi || t * c.E < Flo) return true;   // every point farther than the threshold
        if (!(Flo > 0.0f)) return false;
        const float R2lo = t * t - Fhi * Fhi + aWlo * aWlo, R2hi = t * t - Flo * Flo + aWhi * aWhi;
        if (R2hi < -HORO_M * t * t) return true;        // no crossing
        if (R2lo < HORO_M * t * t) return false;        // nearly tangent: test exactly
        const float Rlo = sqrt_approx(R2lo) * (1.0f - 1e-6f), Rhi = sqrt_approx(R2hi) * (1.0f + 1e-6f);   // r t
        // margin of the reference's own root test: 2 EPS plus its float error
        const float tol = 2e-6f * Fhi * Fhi + 1e-5f * (aWhi * t + Rhi * Fhi);
        const bool r1 = !(Wlo * t + Rlo * Flo > tol);   // root 1 may be reported
        const bool r2 = !(Wlo * t - Rhi * Fhi > tol);   // root 2 may be reported
        const float E1 = c.E * (1.0f + HORO_M);
        const bool r1_far = (Flo - Whi) > E1 * (t + Rhi) || (Fhi - Wlo) * E1 < (t + Rlo);
        const bool r2_far = (Flo + Wlo) > 0.0f && ((t + Rlo) > E1 * (Fhi + Whi) || (t + Rhi) * E1 < (Flo + Wlo));
        return (!r1 || r1_far) && (!r2 || r2_far);
    }
}
static __device__ __noinline__ bool culled_fw_call(const BoundFW b, uint32_t shape, float t, const Cull c) {
    return culled_fw(b, shape, t, c);
}
// OOL: the root tests out of line (one copy of their code, called per survivor). Measured at
// 1920x1080 / 200 objects: the single-view wavefront kernel 5.95 -> 5.55 ms per pass out of
// line, the batched kernels (both recipes per module) 954 -> 938 Msamples/s: each kernel takes
// the faster form.
template <bool OOL>
HT_D bool culled(float4 rec, float mag, uint32_t shape, const BoundRay &r, const Cull &c) {
    const BoundFW b = bound_fw(rec, mag, r);
    return OOL ? culled_fw_call(b, shape, r.t, c) : culled_fw(b, shape, r.t, c);
}

// Upper bound of e^(2 s) at the nearest crossing of one object that the reference surely
// reports (s = distance along the ray): geodesic planes crossed ahead (tanh s = |F| / |W|,
// not the plane the ray just left), horospheres entered ahead from outside or left ahead
// from inside (e^s of the crossing), with margins far above the float error of either side.
// +inf when the object has no such crossing.
HT_D float sure_crossing_e2(const BoundFW &b, uint32_t shape, bool plane_repeat, float t) {
    const float inf = __int_as_float(0x7f800000);
    const float F = b.F, eF = b.eF, W = b.W, eW = b.eW;
    if (shape == 0) {
        if (plane_repeat) return inf;   // a plane is never hit twice in a row
        const float Fa = fabsf(F) - eF, Wlo = fabsf(W) - eW;
        if (!((F > 0.0f) != (W > 0.0f) && Fa > 0.02f * t && Wlo > 0.0f)) return inf;
        const float rr = (fabsf(F) + eF) * rcp_approx(Wlo);   // >= tanh s
        if (!(rr < 0.99f)) return inf;
        return (1.0f + rr) * rcp_approx(1.0f - rr);
    }
    const float Flo = F - eF, Fhi = F + eF, Wlo = W - eW, Whi = W + eW;
    float e = inf;
    if (Fhi < 0.999f * t && Flo > 0.0f && (Flo + Wlo) > 0.0f) {   // inside: exit ahead
        const float aWlo = fmaxf(fabsf(W) - eW, 0.0f), aWhi = fabsf(W) + eW;
        const float R2lo = t * t - Fhi * Fhi + aWlo * aWlo, R2hi = t * t - Flo * Flo + aWhi * aWhi;
        if (R2lo > 1e-3f * t * t) {
            const float Rlo = sqrt_approx(R2lo) * (1.0f - 1e-6f), Rhi = sqrt_approx(R2hi) * (1.0f + 1e-6f);
            const float tol = 2e-6f * Fhi * Fhi + 1e-5f * (aWhi * t + Rhi * Fhi);
            const bool r1 = !(Wlo * t + Rlo * Flo > tol);
            const bool r2_sure = (Wlo * t - Rhi * Fhi) < -tol - 1e-3f * t * t;
            if (!r1 && r2_sure) e = (t + Rhi) * rcp_approx(Flo + Wlo) * 1.001f;
        }
    } else if (Flo > 1.01f * t && Whi < -0.01f * t) {   // outside, approaching: entry ahead
        const float it = rcp_approx(t);
        const float aVlo = -Whi * it, P = Fhi * it;
        const float D = 1.0f - P * P + aVlo * aVlo;
        if (D > 0.02f) e = (Fhi - Wlo) * it * rcp_approx(1.0f + sqrt_approx(D));
    }
    return e * e;
}
// Distance of a crossing from its e^(2 s) bound (the threshold built from it adds 1e-2 margins).
HT_D float dist_from_e2(float x) { return 0.5f * LN2F * lg2_approx(x); }

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

template <bool OOL>
HT_D bool hop_hy(const StagedScene &s, HyPath &ray, uint32_t &rng, uint32_t &prev_hash,
                 Col &intensity, Col &emission, bool &hit, uint32_t &n_exact) {
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
    for (uint32_t c0 = 0; c0 < s.ns; c0 += 32) {
        const uint32_t cn = min(32u, s.ns - c0);
        uint32_t valid = cn == 32 ? 0xFFFFFFFFu : (1u << cn) - 1u;
        if (s.dummy - c0 < 32u) valid &= ~(1u << (s.dummy - c0));
        uint32_t mask = valid;
        if (can_cull) {
            mask = 0;
            // kept rolled: the kernel is bound by instruction fetch as much as by issue
#pragma unroll 1
            for (uint32_t j = 0; j < cn; j += 2) {   // warp-uniform: broadcast loads, two slots at once
                const uint32_t pq = (c0 + j) >> 1;
                const PointCut &k = c0 + j >= s.n_planes ? kh : kp;
                mask |= survivors2(s.pa[pq], s.pb[pq], s.pmag[pq], pr, k) << j;
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
