// ht_bound.cuh -- distance bounds of the hyperbolic object scans: world-space records of
// geodesic planes and horospheres and the culling tests on them. Shared by the hand-written
// scene kernels (ht_trace.cuh) and the generic template kernels (ht_generic.cuh, also
// compiled at run time by NVRTC). They decide only which objects are tested exactly, never a
// result: tests/cull_check/cull_check.c restates them on the CPU and checks every hop's
// winner against the full scan of the reference.
#pragma once
#include "ht_math.cuh"

namespace ht {

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
// The same test on one object (the scalar form of the packed loop).
HT_D bool culled_point(float4 rec, float mag, const BoundRay &r, const PointCut &k) {
    const float F = fmaf(rec.x, r.r2, fmaf(rec.y, r.x, fmaf(rec.z, r.y, rec.w)));
    const float eF = mag * r.K;
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


}  // namespace ht
