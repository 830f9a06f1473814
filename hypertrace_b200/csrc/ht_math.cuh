// ht_math.cuh -- device float math for the render path, in the reference's evaluation order.
//
// Every helper keeps the operation order and rounding points of the reference's kernel
// library (kernel/ocl/algebra/*.cc, transform/*.cc) so that, compiled with FMA
// contraction off (-fmad=false) and IEEE division / square root, each result is
// bit-identical to the reference compiled for the host. Transcendentals are the
// exception: logf is CUDA's, cos and sin are evaluated in FP64 and rounded once (see below);
// the host libm's float versions return other values on a small fraction of arguments.
#pragma once
#ifdef __CUDACC_RTC__
// Runtime compilation (NVRTC) has no C++ standard headers; these are the only ones used.
typedef unsigned char uint8_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
typedef int int32_t;
typedef unsigned long long uintptr_t;
#else
#include <cstdint>
#endif

namespace ht {

struct C2 { float x, y; };
struct Q4 { float x, y, z, w; };   // x = real part; (y, z, w) = (i, j, k)
struct V3 { float x, y, z; };
struct Col { float x, y, z; };
struct Mo { C2 a, b, c, d; };      // (a p + b)(c p + d)^-1
struct Hom { V3 shift; Q4 rot; };  // Chain<Shift3, Rotation3>: p -> rot(p) + shift

#define HT_D __device__ __forceinline__

HT_D Q4 q4(float x, float y, float z, float w) { Q4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
HT_D V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }

// ------------------------------------------------------------------- RNG
// kernel/ocl/random.cc:8-14
HT_D uint32_t rng_next(uint32_t &s) { s = 1103515245u * s + 12345u; return s; }
HT_D float rng_uniform(uint32_t &s) {
    return __uint2float_rn(rng_next(s)) / 4294967296.0f;
}

// ------------------------------------------------------------------- vectors
// dot = (((0 + a0 b0) + a1 b1) + ...): kernel/ocl/algebra/vector_math.hpp:8-15
HT_D float dot2(float ax, float ay, float bx, float by) {
    float c = 0.0f; c += ax * bx; c += ay * by; return c;
}
HT_D float dot3(V3 a, V3 b) { float c = 0.0f; c += a.x * b.x; c += a.y * b.y; c += a.z * b.z; return c; }
HT_D float dot4(Q4 a, Q4 b) {
    float c = 0.0f; c += a.x * b.x; c += a.y * b.y; c += a.z * b.z; c += a.w * b.w; return c;
}
HT_D V3 normalize3(V3 a) { float l = sqrtf(dot3(a, a)); return v3(a.x / l, a.y / l, a.z / l); }
HT_D Q4 normalize4(Q4 a) { float l = sqrtf(dot4(a, a)); return q4(a.x / l, a.y / l, a.z / l, a.w / l); }
HT_D V3 cross3(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// ------------------------------------------------------------------- quaternions
// kernel/ocl/algebra/quaternion.cc:4-56
HT_D Q4 q_conj(Q4 a) { return q4(a.x, -a.y, -a.z, -a.w); }
HT_D Q4 q_mul(Q4 a, Q4 b) {
    return q4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
              a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
              a.x * b.z + a.z * b.x - a.y * b.w + a.w * b.y,
              a.x * b.w + a.w * b.x + a.y * b.z - a.z * b.y);
}
HT_D Q4 cq_mul(C2 a, Q4 b) {
    return q4(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x, a.x * b.z - a.y * b.w, a.x * b.w + a.y * b.z);
}
HT_D Q4 q_add(Q4 a, Q4 b) { return q4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
HT_D Q4 q_sub(Q4 a, Q4 b) { return q4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
HT_D Q4 q_addc(Q4 a, C2 b) { return q4(a.x + b.x, a.y + b.y, a.z + 0.0f, a.w + 0.0f); }  // + q_new(c, C0)

// ------------------------------------------------------------------- division
// Correctly rounded quotients that share one reciprocal (Markstein's correction step):
//   y = RN(1/b),  q0 = RN(a*y),  r = a - b*q0 (exact with an FMA),  q = RN(q0 + r*y) = RN(a/b)
// (P. Markstein, "IA-64 and Elementary Functions", 2000; Muller et al., "Handbook of
// Floating-Point Arithmetic", 2nd ed., section 4.7, Markstein's theorem). The identity
// needs every intermediate to be a normal number, so each quotient checks that |q0| lies in
// [2^-60, 2^60] (or a == 0, where q0 already carries the IEEE sign of zero) and each divisor
// that |b| does; a group with any value outside redoes its divisions with IEEE division.
// tests/test_gpu_math.py compares qdiv with IEEE division on billions of inputs.
struct Rcp { float b, y; };
HT_D bool in_safe_range(float x) {
    const float ax = fabsf(x);
    return ax >= 0x1p-60f && ax <= 0x1p60f;
}
HT_D Rcp rcp_of(float b, bool &bad) {
    bad |= !in_safe_range(b);
    Rcp r;
    r.b = b;
    r.y = __frcp_rn(b);
    return r;
}
HT_D float qdiv(float a, const Rcp &r, bool &bad) {
    const float q0 = a * r.y;
    const float e = fmaf(-r.b, q0, a);
    const float q = fmaf(e, r.y, q0);
    bad |= (a != 0.0f) & !in_safe_range(q0);
    return q0 == 0.0f ? q0 : q;
}
HT_D Q4 qdiv4(Q4 a, const Rcp &r, bool &bad) {
    return q4(qdiv(a.x, r, bad), qdiv(a.y, r, bad), qdiv(a.z, r, bad), qdiv(a.w, r, bad));
}
// normalize4 through one correctly rounded reciprocal of the length.
HT_D Q4 normalize4_fast(Q4 a, bool &bad) {
    float l = sqrtf(dot4(a, a));
    Rcp r = rcp_of(l, bad);
    return qdiv4(a, r, bad);
}

// ------------------------------------------------------------------- Moebius
// mo_apply_q and mo_deriv_q (kernel/ocl/transform/moebius.cc:20-42) share the numerator u,
// the denominator d, |d|^2 and q_inverse(d) = conj(d) / |d|^2.
struct HyRay { Q4 p, v; };

// Reference evaluation with IEEE division everywhere (the fallback of ray_hy_map).
static __device__ __noinline__ HyRay ray_hy_map_ieee(const Mo m, const Q4 p, const Q4 v) {
    Q4 u = q_addc(cq_mul(m.a, p), m.b);
    Q4 d = q_addc(cq_mul(m.c, p), m.d);
    float d2 = dot4(d, d);
    Q4 di = q4(d.x / d2, (-d.y) / d2, (-d.z) / d2, (-d.w) / d2);   // q_inverse(d)
    HyRay o;
    o.p = q_mul(u, di);                                             // mo_apply_q
    Q4 g1 = q_mul(cq_mul(m.a, v), di);                              // q_div(cq_mul(a, v), d)
    Q4 cv = cq_mul(m.c, v);
    Q4 g21 = q_conj(cv);
    float k = (2.0f * dot4(d, cv)) / d2;
    Q4 dc = q_conj(d);
    Q4 g22 = q4(k * dc.x, k * dc.y, k * dc.z, k * dc.w);
    Q4 t = q_sub(g21, g22);
    Q4 g2 = q_mul(u, q4(t.x / d2, t.y / d2, t.z / d2, t.w / d2));
    Q4 deriv = q_add(g1, g2);
    o.v = normalize4(normalize4(deriv));   // mo_apply_dir normalizes, ray_map.inl:19 again
    return o;
}

// ray_<hy>_map (geometry/ray_map.inl:15-21): the nine divisions by |d|^2 share one
// reciprocal, each normalize shares one; results are bit-identical to ray_hy_map_ieee.
HT_D HyRay ray_hy_map(const Mo &m, Q4 p, Q4 v) {
    bool bad = false;
    Q4 u = q_addc(cq_mul(m.a, p), m.b);
    Q4 d = q_addc(cq_mul(m.c, p), m.d);
    float d2 = dot4(d, d);
    Rcp rd = rcp_of(d2, bad);
    Q4 di = qdiv4(q4(d.x, -d.y, -d.z, -d.w), rd, bad);
    HyRay o;
    o.p = q_mul(u, di);
    Q4 g1 = q_mul(cq_mul(m.a, v), di);
    Q4 cv = cq_mul(m.c, v);
    Q4 g21 = q_conj(cv);
    float k = qdiv(2.0f * dot4(d, cv), rd, bad);
    Q4 dc = q_conj(d);
    Q4 g22 = q4(k * dc.x, k * dc.y, k * dc.z, k * dc.w);
    Q4 g2 = q_mul(u, qdiv4(q_sub(g21, g22), rd, bad));
    Q4 deriv = q_add(g1, g2);
    o.v = normalize4_fast(normalize4_fast(deriv, bad), bad);
    if (bad) return ray_hy_map_ieee(m, p, v);
    return o;
}
// The same map, out of line: the object scan and the hit path share this one copy of its
// code (instruction-cache footprint; an inlined copy in the scan measured slower).
static __device__ __noinline__ HyRay ray_hy_map_call(const Mo m, const Q4 p, const Q4 v) { return ray_hy_map(m, p, v); }

// Camera map (view/mapped.inl:20-26): direction = mo_apply_dir (one normalize), then start.
// Once per sample, so plain IEEE division.
HT_D HyRay view_hy_map(const Mo &m, Q4 p, Q4 v) {
    Q4 u = q_addc(cq_mul(m.a, p), m.b);
    Q4 d = q_addc(cq_mul(m.c, p), m.d);
    float d2 = dot4(d, d);
    Q4 di = q4(d.x / d2, (-d.y) / d2, (-d.z) / d2, (-d.w) / d2);
    HyRay o;
    o.p = q_mul(u, di);
    Q4 g1 = q_mul(cq_mul(m.a, v), di);
    Q4 cv = cq_mul(m.c, v);
    Q4 g21 = q_conj(cv);
    float k = (2.0f * dot4(d, cv)) / d2;
    Q4 dc = q_conj(d);
    Q4 g22 = q4(k * dc.x, k * dc.y, k * dc.z, k * dc.w);
    Q4 t = q_sub(g21, g22);
    Q4 g2 = q_mul(u, q4(t.x / d2, t.y / d2, t.z / d2, t.w / d2));
    o.v = normalize4(q_add(g1, g2));
    return o;
}
// c22_inverse_n (kernel/ocl/algebra/matrix_complex.cc:60-65): adjugate, det = 1 assumed.
HT_D Mo mo_inverse(const Mo &m) {
    Mo r;
    r.a = m.d;
    r.b.x = -m.b.x; r.b.y = -m.b.y;
    r.c.x = -m.c.x; r.c.y = -m.c.y;
    r.d = m.a;
    return r;
}

// ------------------------------------------------------------------- Euclidean maps
// rot3_apply_pos = (q (0, p) q*).yzw (transform/rotation.cc); chain.inl:36-73; shift.cc
struct EuRay { V3 p, v; };
HT_D V3 rot3_apply(Q4 q, V3 p) {
    Q4 r = q_mul(q_mul(q, q4(0.0f, p.x, p.y, p.z)), q_conj(q));
    return v3(r.y, r.z, r.w);
}
HT_D V3 hom3_apply_pos(const Hom &m, V3 p) {
    V3 r = rot3_apply(m.rot, p);
    return v3(r.x + m.shift.x, r.y + m.shift.y, r.z + m.shift.z);
}
HT_D EuRay ray_eu_map(const Hom &m, V3 p, V3 v) {
    EuRay o;
    o.p = hom3_apply_pos(m, p);
    o.v = normalize3(rot3_apply(m.rot, v));
    return o;
}
HT_D Hom hom3_inverse(const Hom &m) {
    Hom s;
    s.shift = v3(-m.shift.x, -m.shift.y, -m.shift.z);
    s.rot = q_conj(m.rot);
    s.shift = rot3_apply(s.rot, s.shift);
    return s;
}

// ------------------------------------------------------------------- hyperbolic geometry
// kernel/ocl/geometry/hyperbolic.cc:20-33, split in two: hy_distance(a, b) =
// hy_dist_from_x(hy_x(a, b)). The object scan compares x and evaluates the logarithm only
// for a candidate that can be nearer than the current one; that equals comparing the
// distances because hy_dist_from_x, as compiled here, is non-decreasing on [1, inf]
// (checked exhaustively over every float in tests/test_gpu_math.py).
HT_D float hy_x(Q4 a, Q4 b) {
    Q4 d = q_sub(a, b);
    return 1.0f + dot4(d, d) / (2.0f * a.z * b.z);
}
// CUDA's single-precision logf. Evaluating it in FP64 and rounding once (what the host libm's
// logf returns) was measured: the share of pixels that differ from the reference over 16
// passes of the 1080p frame stayed 0.365 % (the flips come from cos / sin, below), and the
// headline kernel lost 4.5 % (the generic kernel 30 %).
HT_D float hy_dist_from_x(float x) {
    return logf(x + sqrtf(x * x - 1.0f));
}
HT_D float hy_distance(Q4 a, Q4 b) { return hy_dist_from_x(hy_x(a, b)); }
HT_D Q4 hy_dir_at(Q4 p, Q4 d, Q4 h) {
    float lpxy = sqrtf(dot2(p.x - h.x, p.y - h.y, p.x - h.x, p.y - h.y));
    float ldxy = sqrtf(dot2(d.x, d.y, d.x, d.y));
    float k = h.z / p.z;
    return q4(k * d.x, k * d.y, d.z - lpxy / p.z * ldxy, 0.0f);
}

// ------------------------------------------------------------------- samplers / rotations
// random_hemisphere_cosine (kernel/ocl/random.cc:37-39,53-59). cos/sin are evaluated in
// FP64 and rounded once: this lands on the correctly rounded float, which the host libm
// the reference is built against matches far more often than a float kernel does.
HT_D V3 hemisphere_cosine(uint32_t &s) {
    float phi = 2.0f * 3.14159265358979323846f * rng_uniform(s);
    float sqr_cos_theta = rng_uniform(s);
    float cos_theta = sqrtf(sqr_cos_theta);
    float sin_theta = sqrtf(1.0f - sqr_cos_theta);
    double sd, cd;
    sincos((double)phi, &sd, &cd);
    return v3((float)cd * sin_theta, (float)sd * sin_theta, cos_theta);
}
// rot3_look_at_cont / rot3_look_at / rot3_from_axis (kernel/ocl/transform/rotation.cc)
HT_D Q4 rot3_look_at_cont(V3 d) {
    V3 z = v3(0.0f, 0.0f, -1.0f);
    float c2 = dot3(d, z);
    float c = sqrtf((1.0f + c2) / 2.0f);
    float sm = 1.0f / (2.0f * c);
    V3 x = cross3(z, d);
    return q4(c, sm * x.x, sm * x.y, sm * x.z);
}
HT_D Q4 rot3_look_at(V3 d) {
    if (d.z < 0.0f) return rot3_look_at_cont(d);
    Q4 a = rot3_look_at_cont(v3(-d.x, -d.y, -d.z));
    const float half = 3.14159265358979323846f / 2.0f;
    double sh, ch;
    sincos((double)half, &sh, &ch);
    float s = (float)sh;
    Q4 b = q4((float)ch, s * 1.0f, s * 0.0f, s * 0.0f);
    return q_mul(a, b);
}

}  // namespace ht
