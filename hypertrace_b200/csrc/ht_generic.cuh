// ht_generic.cuh -- the reference's scene type system as CUDA C++ templates.
//
// The reference builds one OpenCL program per Rust scene type: every entity (view, map,
// object, shape, material, background, container) contributes a struct and a source
// template, instantiated by text substitution (types/src/source.rs:102-168,
// type-macros/src/source.rs:94-204, objects/src/scene.rs:44-67). Here every entity is a
// C++ class template with
//   - `lay<W>()`: its serialized size and alignment for a usize of W bytes, computed by the
//     reference's layout rules (type-macros/src/entity.rs:7-200: fields in order, each
//     aligned to its own alignment, alignment = lcm of the fields', size rounded up to it;
//     enums = usize index + payload at the enum's alignment; Vec = usize count + elements),
//   - device functions with the reference's semantics and operation order, reading the
//     serialized bytes in place (no host-side parsing),
// so a scene type is a C++ type expression, compiled by nvcc for the built-in recipes and
// by NVRTC at run time for any other type (include/htcuda.h: htc_program_build).
//
// Entities (reference files):
//   maps        Moebius (transform/moebius.cc), Shift3 (shift.cc), Rotation3 (rotation.cc),
//               Linear3 (linear.cc), Chain<A, B> of Shift3 with Rotation3 or Linear3 in either
//               order (chain.inl; Homogenous3 = Chain<Shift3, Rotation3>)
//   views       PointView<G> (view/point/impl.inl), MappedView<G, V, M> (view/mapped.inl)
//   shapes      PlaneHy, Horosphere (shape/hy/*.cc), PlaneEu, Sphere, Cube (shape/eu/*.cc),
//               ShapeVec<G, S> (shape/vector.inl), MappedShape<G, S, M> (shape/mapped.inl),
//               ShapeChoice<G, S...> (shape/choice/impl.inl)
//   objects     Covered<G, S, M> (object/covered.inl), MappedObject<G, O, M>
//               (object/mapped.inl), ObjectVec<G, O> (object/vector.inl), ObjectChoice<G, O...>
//               (object/choice/impl.inl), TiledPlane<M, K, N> (object/hy/tiled_plane/impl.inl),
//               TiledHorosphere<M, K, N> (object/hy/tiled_horosphere/impl.inl)
//   materials   Lambertian, Specular, Absorbing, Transparent, Refractive (material/*.cc),
//               Colored<M>, Emissive<M> (colored.inl, emissive.inl), Mixture<Component<M>...>
//               (material/mixture/impl.inl)
//   backgrounds ConstBg (background/constant.inl), GradBg (background/gradient.cc)
//   scene       SceneImpl<G, V, O, B> (render/scene.inl; the hop count H is a launch argument)
#pragma once
#include "ht_math.cuh"
#include "ht_bound.cuh"

namespace htg {
using namespace ht;

typedef unsigned int u32;
constexpr float EPSF = 1e-6f;          // EPS for real = float (kernel/ocl/algebra/real.hh:19-25)
constexpr float PIF = 3.14159265358979323846f;
constexpr u32 HASH_NEVER = 0xFFFFFFFFu;
constexpr u32 FLAG_JITTER_YX = 1u;
constexpr u32 ERR_SCENE = 1u;

// ============================================================================ layout
struct Lay { u32 size, align; };
__host__ __device__ constexpr u32 upm(u32 x, u32 a) { return (x + a - 1u) / a * a; }
__host__ __device__ constexpr u32 gcdc(u32 a, u32 b) { return b ? gcdc(b, a % b) : a; }
__host__ __device__ constexpr u32 lcmc(u32 a, u32 b) { return a / gcdc(a, b) * b; }

// Struct of fields F... (type-macros/src/entity.rs:7-12 align, :31-63 size, :277-315 store).
template <int W, class... F> struct Rec {
    static constexpr u32 N = sizeof...(F);
    __host__ __device__ static constexpr Lay at(u32 i) {
        const Lay l[] = {Lay{0u, 1u}, F::template lay<W>()...};
        return l[i + 1];
    }
    __host__ __device__ static constexpr u32 align() {
        u32 a = 1;
        for (u32 k = 0; k < N; ++k) a = lcmc(a, at(k).align);
        return a;
    }
    __host__ __device__ static constexpr u32 off(u32 i) {
        u32 o = 0;
        for (u32 k = 0; k < i; ++k) o = upm(o, at(k).align) + at(k).size;
        return upm(o, at(i).align);
    }
    __host__ __device__ static constexpr Lay lay() {
        u32 o = 0;
        for (u32 k = 0; k < N; ++k) o = upm(o, at(k).align) + at(k).size;
        return Lay{upm(o, align()), align()};
    }
};

// Enum of single-field variants V...: usize index, then the payload at the enum's alignment
// (type-macros/src/entity.rs:14-27 align, :160-181 size, :319-344 store).
template <int W, class... V> struct Enum {
    static constexpr u32 N = sizeof...(V);
    __host__ __device__ static constexpr Lay at(u32 i) {
        const Lay l[] = {Lay{0u, 1u}, V::template lay<W>()...};
        return l[i + 1];
    }
    __host__ __device__ static constexpr u32 align() {
        u32 a = (u32)W;
        for (u32 k = 0; k < N; ++k) a = lcmc(a, at(k).align);
        return a;
    }
    __host__ __device__ static constexpr u32 payload() { return upm((u32)W, align()); }
    __host__ __device__ static constexpr Lay lay() {
        u32 s = 0;
        for (u32 k = 0; k < N; ++k) {
            const u32 v = upm((u32)W, at(k).align) + at(k).size;
            s = v > s ? v : s;
        }
        return Lay{upm(s, align()), align()};
    }
};

// ============================================================================ loads
typedef const uint8_t *Ptr;
HT_D float ldf(Ptr p) { return __ldg(reinterpret_cast<const float *>(p)); }
HT_D u32 ldu(Ptr p) { return __ldg(reinterpret_cast<const u32 *>(p)); }
HT_D V3 ldv3(Ptr p) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    return v3(v.x, v.y, v.z);
}
HT_D Col ldc3(Ptr p) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    Col c; c.x = v.x; c.y = v.y; c.z = v.z;
    return c;
}
HT_D Q4 ldq(Ptr p) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    return q4(v.x, v.y, v.z, v.w);
}
// usize of W bytes: the low word (little endian); an index above 2^32 reads as out of range.
template <int W> HT_D u32 ldusize(Ptr p) {
    if (W == 8 && ldu(p + 4) != 0u) return 0xFFFFFFFFu;
    return ldu(p);
}

// Primitive entities.
struct Zst { template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; } };   // unit / PhantomData
struct F32 { template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{4u, 4u}; } };   // f32, and f64 as real
struct R3 { template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{16u, 16u}; } };  // Vector<_, 3>
template <int N> struct Arr {   // [T; N] (types/src/containers/array.rs)
    template <class T, int W> __host__ __device__ static constexpr Lay lay() { return Lay{T::template lay<W>().size * N, T::template lay<W>().align}; }
};

// ============================================================================ context
struct Ctx {
    u32 rng;        // Rng state (kernel/ocl/random.cc:3-14)
    u32 hasher;     // sdbm state (kernel/ocl/hash.cc:5-24)
    u32 prev;       // previous hop's hash (render/context.cc:3-13)
    u32 flags;
    u32 tests;      // leaf object tests (statistics)
    Ptr end;        // one past the scene bytes: dynamic containers are clamped to it
    u32 *err;
    // distance bounds of the scene's top-level object vector, staged in shared memory by the
    // kernel (render_generic): bvec is that vector's address (NULL: no culling), culled counts
    // the element tests the bounds skipped (statistics)
    Ptr bvec;
    const float4 *brec;
    const float *bmag;
    const u32 *bkind;
    u32 culled;
};
HT_D bool is_repeat(const Ctx &c) { return c.hasher == c.prev; }
HT_D void hash_usize(Ctx &c, u32 x) { const u32 h = c.hasher; c.hasher = x + (h << 6) + (h << 16) - h; }
HT_D void random2(Ctx &c, float &x, float &y) {   // random_uniform2 (random.cc:15-20)
    const float u0 = rng_uniform(c.rng);
    const float u1 = rng_uniform(c.rng);
    x = (c.flags & FLAG_JITTER_YX) ? u1 : u0;
    y = (c.flags & FLAG_JITTER_YX) ? u0 : u1;
}

// ============================================================================ geometries
struct Hy {
    typedef Q4 Pos;
    typedef Q4 Dir;
    HT_D static Pos origin() { return q4(0.0f, 0.0f, 1.0f, 0.0f); }               // hyperbolic.cc:4-6
    HT_D static Dir from_local(Pos, V3 d) { return q4(d.x, d.y, d.z, 0.0f); }    // hyperbolic.cc:13-15
    HT_D static V3 to_local(Pos, Dir d) { return v3(d.x, d.y, d.z); }            // hyperbolic.cc:9-11
};
struct Eu {
    typedef V3 Pos;
    typedef V3 Dir;
    HT_D static Pos origin() { return v3(0.0f, 0.0f, 0.0f); }                    // euclidean.cc:4-6
    HT_D static Dir from_local(Pos, V3 d) { return d; }
    HT_D static V3 to_local(Pos, Dir d) { return d; }
};
// LightBase{intensity} + Ray{start, direction} (render/light/base.hh:5-13, light/{hy,eu}.hh)
template <class G> struct Light { Col k; typename G::Pos p; typename G::Dir v; };
struct LightLocal { Col k; V3 v; };   // render/light/base.hh LightLocal

HT_D Q4 normalize_q(Q4 a) { return normalize4(a); }
HT_D V3 normalize_q(V3 a) { return normalize3(a); }

// ============================================================================ maps
// Each map: V (the value), lay, load, inverse, pos, dir (apply_dir), normal (apply_normal),
// ray (ray_<geo>_map: start = pos, direction = normalize(dir), geometry/ray_map.inl:15-21)
// and view (view/mapped.inl:20-26: direction = dir, then start = pos).
HT_D Q4 mo_apply_pos(const Mo &m, Q4 p) {   // mo_apply_q (transform/moebius.cc:20-25)
    Q4 u = q_addc(cq_mul(m.a, p), m.b);
    Q4 d = q_addc(cq_mul(m.c, p), m.d);
    float d2 = dot4(d, d);
    Q4 di = q4(d.x / d2, (-d.y) / d2, (-d.z) / d2, (-d.w) / d2);
    return q_mul(u, di);
}
struct Moebius {
    typedef Mo V;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{32u, 32u}; }   // comp2x2 (matrix.rs:174-209)
    HT_D static V load(Ptr p) {
        const Q4 a = ldq(p), b = ldq(p + 16);
        Mo m;
        m.a.x = a.x; m.a.y = a.y; m.b.x = a.z; m.b.y = a.w;
        m.c.x = b.x; m.c.y = b.y; m.d.x = b.z; m.d.y = b.w;
        return m;
    }
    HT_D static V inverse(const V &m) { return mo_inverse(m); }
    HT_D static Q4 pos(const V &m, Q4 p) { return mo_apply_pos(m, p); }
    HT_D static Q4 normal(const V &m, Q4 p, Q4 v) { HyRay r = view_hy_map(m, p, v); return r.v; }
    HT_D static void ray(const V &m, Q4 &p, Q4 &v) { HyRay r = ray_hy_map(m, p, v); p = r.p; v = r.v; }
    HT_D static void view(const V &m, Q4 &p, Q4 &v) { HyRay r = view_hy_map(m, p, v); p = r.p; v = r.v; }
};
struct Shift3 {
    typedef V3 V;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{16u, 16u}; }
    HT_D static V load(Ptr p) { return ldv3(p); }
    HT_D static V inverse(const V &m) { return v3(-m.x, -m.y, -m.z); }
    HT_D static V3 pos(const V &m, V3 p) { return v3(p.x + m.x, p.y + m.y, p.z + m.z); }
    HT_D static V3 dir(const V &, V3, V3 d) { return d; }
    HT_D static V3 normal(const V &, V3, V3 d) { return d; }
};
struct Rotation3 {
    typedef Q4 V;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{16u, 16u}; }
    HT_D static V load(Ptr p) { return ldq(p); }
    HT_D static V inverse(const V &m) { return q_conj(m); }
    HT_D static V3 pos(const V &m, V3 p) { return rot3_apply(m, p); }
    HT_D static V3 dir(const V &m, V3, V3 d) { return rot3_apply(m, d); }
    HT_D static V3 normal(const V &m, V3, V3 d) { return rot3_apply(m, d); }
};
// Linear3: a 3x3 matrix stored as a 4x4 real16, rows (m0 m1 m2 0), (m4 m5 m6 0),
// (m8 m9 m10 0), (0 0 0 1) (types/src/primitive/matrix.rs:117-165; transform/linear.cc,
// algebra/matrix_real.cc).
struct M33 { float m[16]; };
HT_D V3 r33_dot_mv(const M33 &a, V3 b) {   // r44_dot_mv(a, (b, 0)).xyz: dot of 4-vectors from 0
    V3 r;
    float c;
    c = 0.0f; c += a.m[0] * b.x; c += a.m[1] * b.y; c += a.m[2] * b.z; c += a.m[3] * 0.0f; r.x = c;
    c = 0.0f; c += a.m[4] * b.x; c += a.m[5] * b.y; c += a.m[6] * b.z; c += a.m[7] * 0.0f; r.y = c;
    c = 0.0f; c += a.m[8] * b.x; c += a.m[9] * b.y; c += a.m[10] * b.z; c += a.m[11] * 0.0f; r.z = c;
    return r;
}
HT_D M33 r33_transpose(const M33 &a) {
    M33 t;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) t.m[4 * i + j] = a.m[4 * j + i];
    return t;
}
HT_D M33 r33_inverse(const M33 &a) {   // matrix_real.cc:106-120: adjugate / det, then s_f = 1
    const float *m = a.m;
    const float det = m[0] * m[5] * m[10] + m[1] * m[6] * m[8] + m[2] * m[4] * m[9]
                    - m[0] * m[6] * m[9] - m[1] * m[4] * m[10] - m[2] * m[5] * m[8];
    const float adj[16] = {m[5] * m[10] - m[6] * m[9], m[2] * m[9] - m[1] * m[10], m[1] * m[6] - m[2] * m[5], 0.0f,
                           m[6] * m[8] - m[4] * m[10], m[0] * m[10] - m[2] * m[8], m[2] * m[4] - m[0] * m[6], 0.0f,
                           m[4] * m[9] - m[5] * m[8], m[1] * m[8] - m[0] * m[9], m[0] * m[5] - m[1] * m[4], 0.0f,
                           0.0f, 0.0f, 0.0f, 0.0f};
    M33 r;
    for (int i = 0; i < 16; ++i) r.m[i] = adj[i] / det;
    r.m[15] = 1.0f;
    return r;
}
struct Linear3 {
    typedef M33 V;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{64u, 64u}; }
    HT_D static V load(Ptr p) {
        M33 m;
        for (int i = 0; i < 4; ++i) {
            const float4 r = __ldg(reinterpret_cast<const float4 *>(p + 16 * i));
            m.m[4 * i] = r.x; m.m[4 * i + 1] = r.y; m.m[4 * i + 2] = r.z; m.m[4 * i + 3] = r.w;
        }
        return m;
    }
    HT_D static V inverse(const V &m) { return r33_inverse(m); }
    HT_D static V3 pos(const V &m, V3 p) { return r33_dot_mv(m, p); }
    HT_D static V3 dir(const V &m, V3, V3 d) { return normalize3(r33_dot_mv(m, d)); }
    HT_D static V3 normal(const V &m, V3, V3 d) { return normalize3(r33_dot_mv(r33_transpose(r33_inverse(m)), d)); }
};

// <inner>_<outer>_reorder (rotation.cc: rot3_shf3_reorder, shf3_rot3_reorder;
// linear.cc: lin3_shf3_reorder, shf3_lin3_reorder)
template <class Inner, class Outer> struct Reorder;
template <> struct Reorder<Rotation3, Shift3> {
    HT_D static void apply(Q4 &inner, V3 &outer) { outer = rot3_apply(inner, outer); }
};
template <> struct Reorder<Shift3, Rotation3> {
    HT_D static void apply(V3 &inner, Q4 &outer) { inner = rot3_apply(q_conj(outer), inner); }
};
template <> struct Reorder<Linear3, Shift3> {
    HT_D static void apply(M33 &inner, V3 &outer) { outer = r33_dot_mv(inner, outer); }
};
template <> struct Reorder<Shift3, Linear3> {
    HT_D static void apply(V3 &inner, M33 &outer) { inner = r33_dot_mv(r33_inverse(outer), inner); }
};
template <class A, class B> struct Chain {   // outer A after inner B (transform/chain.inl)
    struct V { typename A::V a; typename B::V b; };
    template <int W> __host__ __device__ static constexpr Lay lay() {   // types/src/map.rs:190-235
        return Lay{upm(upm(A::template lay<W>().size, B::template lay<W>().align) + B::template lay<W>().size,
                       lcmc(A::template lay<W>().align, B::template lay<W>().align)),
                   lcmc(A::template lay<W>().align, B::template lay<W>().align)};
    }
    HT_D static V load(Ptr p) {
        V m;
        m.a = A::load(p);
        m.b = B::load(p + upm(A::template lay<4>().size, B::template lay<4>().align));
        return m;
    }
    HT_D static V inverse(const V &m) {
        V s;
        s.a = A::inverse(m.a);
        s.b = B::inverse(m.b);
        Reorder<B, A>::apply(s.b, s.a);
        return s;
    }
    HT_D static V3 pos(const V &m, V3 p) { return A::pos(m.a, B::pos(m.b, p)); }
    HT_D static V3 dir(const V &m, V3 p, V3 d) { return A::dir(m.a, B::pos(m.b, p), B::dir(m.b, p, d)); }
    HT_D static V3 normal(const V &m, V3 p, V3 d) { return A::normal(m.a, B::pos(m.b, p), B::normal(m.b, p, d)); }
};
typedef Chain<Shift3, Rotation3> Homogenous3;

// Euclidean maps: ray / view from pos and dir.
template <class M> struct EuMapOps {
    HT_D static void ray(const typename M::V &m, V3 &p, V3 &v) {
        const V3 np = M::pos(m, p);
        v = normalize3(M::dir(m, p, v));
        p = np;
    }
    HT_D static void view(const typename M::V &m, V3 &p, V3 &v) {
        v = M::dir(m, p, v);
        p = M::pos(m, p);
    }
    HT_D static void ray_cold(const typename M::V &m, V3 &p, V3 &v) { ray(m, p, v); }
};
template <class M> struct MapOps : EuMapOps<M> {};
template <> struct MapOps<Moebius> {
    HT_D static void ray(const Mo &m, Q4 &p, Q4 &v) { Moebius::ray(m, p, v); }
    HT_D static void view(const Mo &m, Q4 &p, Q4 &v) { Moebius::view(m, p, v); }
    // The same map through one out-of-line copy, for the once-per-hop paths (the winner's
    // full detection, the interaction): only the distance scan keeps an inlined copy.
    HT_D static void ray_cold(const Mo &m, Q4 &p, Q4 &v) { HyRay r = ray_hy_map_call(m, p, v); p = r.p; v = r.v; }
};

// ============================================================================ views
template <class G> struct PointView {   // {fov, phantom} (objects/src/view/point.rs:11-14)
    typedef Rec<4, F32, Zst> R4;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, F32, Zst>::lay(); }
    template <int W>
    HT_D static Light<G> sample(Ptr self, Ctx &c, float px, float py, float size) {   // view/point/impl.inl:18-25
        const float fov = ldf(self);
        float ux, uy;
        random2(c, ux, uy);
        const float sx = px + size * (ux - 0.5f);
        const float sy = py + size * (uy - 0.5f);
        Light<G> l;
        l.p = G::origin();
        l.v = G::from_local(l.p, normalize3(v3(sx, sy, -1.0f / fov)));
        return l;
    }
};
template <class G, class V, class M> struct MappedView {   // Mapped{phantom, map, inner}
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, Zst, M, V>::lay(); }
    template <int W>
    HT_D static Light<G> sample(Ptr self, Ctx &c, float px, float py, float size) {
        Light<G> l = V::template sample<W>(self + Rec<W, Zst, M, V>::off(2), c, px, py, size);
        const typename M::V m = M::load(self + Rec<W, Zst, M, V>::off(1));
        MapOps<M>::view(m, l.p, l.v);
        return l;
    }
};

// ============================================================================ shapes
// detect(self, ctx, normal, light) -> distance (> -EPS on a hit); on a hit the light's ray
// starts at the hit point.
struct PlaneHy {   // shape/hy/plane.cc:4-37
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, Q4 &normal, Light<Hy> &l) {
        if (is_repeat(c)) return -1.0f;
        const Q4 p = l.p, d = l.v;
        const float pd = dot4(p, d);
        if (fabsf(pd) < EPSF) return -1.0f;
        const float s = 1.0f - dot4(p, p);
        const float t = s / (2.0f * pd);
        if (t < -EPSF) return -1.0f;
        const float hx = p.x + d.x * t, hy = p.y + d.y * t;
        const float pxy2 = dot2(hx, hy, hx, hy);
        if (pxy2 > 1.0f) return -1.0f;
        const Q4 h = q4(hx, hy, sqrtf(1.0f - pxy2), 0.0f);
        if (F) {
            l.p = h;
            l.v = hy_dir_at(p, d, h);
            normal = q4(-h.x, -h.y, -h.z, -h.w);
        }
        return hy_distance(p, h);
    }
};
struct Horosphere {   // shape/hy/horosphere.cc:4-34
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, Q4 &normal, Light<Hy> &l) {
        const bool repeat = is_repeat(c);
        const Q4 p = l.p, d = l.v;
        const float dxy = sqrtf(dot2(d.x, d.y, d.x, d.y));
        if (p.z < dxy) return -1.0f;
        const float dt = sqrtf(p.z * p.z - dxy * dxy);
        float t = p.z * d.z - dt;
        const float w = repeat ? EPSF : -EPSF;
        if (t < w) {
            t += 2.0f * dt;
            if (t < w) return -1.0f;
        }
        t /= dxy * dxy;
        const Q4 h = q4(p.x + d.x * t, p.y + d.y * t, 1.0f, 0.0f);
        if (F) {
            l.p = h;
            l.v = hy_dir_at(p, d, h);
            normal = q4(0.0f, 0.0f, -1.0f, 0.0f);
        }
        return hy_distance(p, h);
    }
};
struct PlaneEu {   // shape/eu/plane.cc:3-21
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, V3 &normal, Light<Eu> &l) {
        if (is_repeat(c)) return -1.0f;
        const V3 pos = l.p, dir = l.v;
        if (pos.z * dir.z > 0.0f) return -1.0f;
        const float t = -pos.z / dir.z;
        l.p = v3(pos.x + dir.x * t, pos.y + dir.y * t, 0.0f);
        normal = v3(0.0f, 0.0f, -1.0f);
        return t;
    }
};
struct Sphere {   // shape/eu/sphere.cc:3-29
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, V3 &normal, Light<Eu> &l) {
        const bool repeat = is_repeat(c);
        const V3 pos = l.p, dir = l.v;
        const float b = -dot3(dir, pos);
        const V3 g = v3(pos.x + dir.x * b, pos.y + dir.y * b, pos.z + dir.z * b);
        float d = 1.0f - dot3(g, g);
        if (d < 0.0f) return -1.0f;
        d = sqrtf(d);
        float e = b - d;
        const float w = repeat ? EPSF : -EPSF;
        if (e < w) {
            e = b + d;
            if (e < w) return -1.0f;
        }
        if (F) {
            const V3 h = normalize3(v3(pos.x + dir.x * e, pos.y + dir.y * e, pos.z + dir.z * e));
            normal = h;
            l.p = h;
        }
        return e;
    }
};
HT_D float signf(float a) { return (float)((0.0f < a) - (a < 0.0f)); }   // math.hh sign
struct Cube {   // shape/eu/cube.cc:3-65
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    HT_D static float nearest(V3 near, V3 &n) {   // cube_eu_detect_nearest
        const bool xy = near.x > near.y, yz = near.y > near.z, xz = near.x > near.z;
        if (xy && xz) { n.x = 1.0f; return near.x; }
        if (yz) { n.y = 1.0f; return near.y; }
        n.z = 1.0f;
        return near.z;
    }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, V3 &normal, Light<Eu> &l) {
        const bool repeat = is_repeat(c);
        const V3 s = l.p, d = l.v;
        const V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
        const V3 vmin = v3((-1.0f - s.x) * inv.x, (-1.0f - s.y) * inv.y, (-1.0f - s.z) * inv.z);
        const V3 vmax = v3((1.0f - s.x) * inv.x, (1.0f - s.y) * inv.y, (1.0f - s.z) * inv.z);
        const V3 near = v3(fminf(vmin.x, vmax.x), fminf(vmin.y, vmax.y), fminf(vmin.z, vmax.z));
        const V3 far = v3(fmaxf(vmin.x, vmax.x), fmaxf(vmin.y, vmax.y), fmaxf(vmin.z, vmax.z));
        const V3 sg = v3(signf(d.x), signf(d.y), signf(d.z));
        V3 nin = v3(0.0f, 0.0f, 0.0f);
        const float din = nearest(near, nin);
        nin = v3(nin.x * -sg.x, nin.y * -sg.y, nin.z * -sg.z);
        V3 nout = v3(0.0f, 0.0f, 0.0f);
        const float dout = -nearest(v3(-far.x, -far.y, -far.z), nout);
        nout = v3(nout.x * sg.x, nout.y * sg.y, nout.z * sg.z);
        if (din > dout) return -1.0f;
        float dist = din;
        V3 n = nin;
        const float w = 2.0f * EPSF * (repeat ? 1.0f : -1.0f);
        if (dist < w) {
            dist = dout;
            n = nout;
            if (dist < w) return -1.0f;
        }
        l.p = v3(s.x + dist * d.x, s.y + dist * d.y, s.z + dist * d.z);
        normal = n;
        return dist;
    }
};
template <class G, class S> struct ShapeVec {   // shape/vector.inl
    template <int W> __host__ __device__ static constexpr Lay lay() {
        return Lay{upm((u32)W, S::template lay<W>().align), lcmc((u32)W, S::template lay<W>().align)};
    }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, typename G::Dir &normal, Light<G> &l) {
        constexpr u32 stride = S::template lay<W>().size;
        constexpr u32 head = upm((u32)W, S::template lay<W>().align);
        u32 n = ldusize<W>(self);
        if (stride > 0 && (c.end < self + head || n > (u32)((c.end - self - head) / stride))) { atomicOr(c.err, ERR_SCENE); n = 0; }
        // Distances first, then the winner's full detection again (same operations, same
        // bits) instead of keeping every candidate's light and normal (shape/vector.inl).
        const u32 orig = c.hasher;
        float min_dist = -1.0f;
        u32 min_index = 0, min_hasher = orig;
        for (u32 i = 0; i < n; ++i) {
            Light<G> cur = l;
            typename G::Dir cn;
            hash_usize(c, i);
            const float dist = S::template detect<W, false>(self + head + i * stride, c, cn, cur);
            if (dist > -EPSF && (min_dist <= -EPSF || dist < min_dist)) {
                min_dist = dist; min_index = i; min_hasher = c.hasher;
            }
            c.hasher = orig;
        }
        if (!(min_dist > -EPSF)) return -1.0f;
        if (F) {
            const u32 tests = c.tests;
            hash_usize(c, min_index);
            S::template detect<W, true>(self + head + min_index * stride, c, normal, l);
            c.tests = tests;
        }
        c.hasher = min_hasher;
        return min_dist;
    }
};
template <class G, class S, class M> struct MappedShape {   // shape/mapped.inl
    typedef Rec<4, Zst, M, S> R4;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, Zst, M, S>::lay(); }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, typename G::Dir &normal, Light<G> &l) {
        const typename M::V m = M::load(self + Rec<W, Zst, M, S>::off(1));
        if (F) MapOps<M>::ray_cold(M::inverse(m), l.p, l.v);
        else MapOps<M>::ray(M::inverse(m), l.p, l.v);
        const float dist = S::template detect<W, F>(self + Rec<W, Zst, M, S>::off(2), c, normal, l);
        if (F) {
            normal = M::normal(m, l.p, normal);
            MapOps<M>::ray_cold(m, l.p, l.v);
        }
        return dist;
    }
};
template <class G, class... S> struct ShapeChoice;   // shape/choice/impl.inl
template <class G> struct ShapeChoice<G> {
    template <int W, bool F> HT_D static float dispatch(u32, Ptr, Ctx &, typename G::Dir &, Light<G> &) { return -1.0f; }
};
template <class G, class S0, class... S> struct ShapeChoice<G, S0, S...> {
    template <int W> __host__ __device__ static constexpr Lay lay() { return Enum<W, S0, S...>::lay(); }
    template <int W, bool F> HT_D static float dispatch(u32 i, Ptr pay, Ctx &c, typename G::Dir &n, Light<G> &l) {
        if (i == 0) return S0::template detect<W, F>(pay, c, n, l);
        return ShapeChoice<G, S...>::template dispatch<W, F>(i - 1, pay, c, n, l);
    }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, typename G::Dir &n, Light<G> &l) {
        return dispatch<W, F>(ldusize<W>(self), self + Enum<W, S0, S...>::payload(), c, n, l);
    }
};

// ============================================================================ materials
// interact(self, ctx, normal (local), light (local), emission) -> false when the path ends.
struct Lambertian {   // material/lambertian.cc:6-14
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W> HT_D static bool interact(Ptr, Ctx &c, V3 n, LightLocal &l, Col &) {
        if (dot3(l.v, n) > 0.0f) n = v3(-n.x, -n.y, -n.z);
        const V3 rnd = hemisphere_cosine(c.rng);
        const Q4 rot = rot3_look_at(v3(-n.x, -n.y, -n.z));
        l.v = rot3_apply(rot, rnd);
        return true;
    }
};
struct Specular {   // material/specular.cc:4-7
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W> HT_D static bool interact(Ptr, Ctx &, V3 n, LightLocal &l, Col &) {
        const float k = 2.0f * dot3(l.v, n);
        l.v = v3(l.v.x - k * n.x, l.v.y - k * n.y, l.v.z - k * n.z);
        return true;
    }
};
struct Absorbing {   // material/absorbing.cc:4-6
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W> HT_D static bool interact(Ptr, Ctx &, V3, LightLocal &, Col &) { return false; }
};
struct Transparent {   // material/transparent.cc:4-6
    template <int W> __host__ __device__ static constexpr Lay lay() { return Lay{0u, 1u}; }
    template <int W> HT_D static bool interact(Ptr, Ctx &, V3, LightLocal &, Col &) { return true; }
};
struct Refractive {   // {index} (objects/src/material/refractive.rs), material/refractive.cc:4-22
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, F32>::lay(); }
    template <int W> HT_D static bool interact(Ptr self, Ctx &, V3 n, LightLocal &l, Col &) {
        V3 d = l.v;
        float k = ldf(self);
        const float a = dot3(d, n);
        if (a < -EPSF) k = 1.0f / k;
        const float x = (a * a - 1.0f) * (k * k) + 1.0f;
        if (x > EPSF) {
            const float b = signf(a) * sqrtf(x);
            const float m = b - a * k;
            d = v3(d.x * k + m * n.x, d.y * k + m * n.y, d.z * k + m * n.z);
        } else {
            const float m = 2.0f * a;
            d = v3(d.x - m * n.x, d.y - m * n.y, d.z - m * n.z);
        }
        l.v = d;
        return true;
    }
};
template <class M> struct Colored {   // {color, inner} (material/modifier.rs), colored.inl
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, R3, M>::lay(); }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, V3 n, LightLocal &l, Col &e) {
        const Col col = ldc3(self);
        l.k.x *= col.x; l.k.y *= col.y; l.k.z *= col.z;
        return M::template interact<W>(self + Rec<W, R3, M>::off(1), c, n, l, e);
    }
};
template <class M> struct Emissive {   // {emission, inner}, emissive.inl
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, R3, M>::lay(); }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, V3 n, LightLocal &l, Col &e) {
        const Col em = ldc3(self);
        e.x += l.k.x * em.x; e.y += l.k.y * em.y; e.z += l.k.z * em.z;
        return M::template interact<W>(self + Rec<W, R3, M>::off(1), c, n, l, e);
    }
};
template <class M> struct Component {   // {material, portion} (material/mixture.rs:4-9)
    typedef M Material;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, M, F32>::lay(); }
    template <int W> __host__ __device__ static constexpr u32 portion_off() { return Rec<W, M, F32>::off(1); }
};
template <class... C> struct Mixture {   // material/mixture/impl.inl + macros.hh
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, C...>::lay(); }
    template <int W, u32 I> HT_D static bool step(Ptr, Ctx &, V3, LightLocal &, Col &, float) { return false; }
    template <int W, u32 I, class C0, class... CR>
    HT_D static bool step(Ptr self, Ctx &c, V3 n, LightLocal &l, Col &e, float alpha) {
        const Ptr comp = self + Rec<W, C...>::off(I);
        alpha -= ldf(comp + C0::template portion_off<W>());
        if (alpha < 0.0f) return C0::Material::template interact<W>(comp, c, n, l, e);
        return step<W, I + 1, CR...>(self, c, n, l, e, alpha);
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, V3 n, LightLocal &l, Col &e) {
        const float alpha = rng_uniform(c.rng);
        return step<W, 0, C...>(self, c, n, l, e, alpha);
    }
};

// ============================================================================ backgrounds
struct ConstBg {   // background/constant.inl:18-21
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, R3>::lay(); }
    template <int W, class G> HT_D static void interact(Ptr self, Ctx &, const Light<G> &l, Col &e) {
        const Col col = ldc3(self);
        e.x += col.x * l.k.x; e.y += col.y * l.k.y; e.z += col.z * l.k.z;
    }
};
// pow(x, y) for x in [0, 1]: FP64 rounded once, like the gamma filter.
HT_D float powf_rounded(float x, float y) { return (float)pow((double)x, (double)y); }
struct GradBg {   // {direction, colors[2], power} (background/basic.rs:54-58), gradient.cc:3-13
    typedef Rec<4, R3, R3, R3, F32> R4;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, R3, R3, R3, F32>::lay(); }
    template <int W> HT_D static void interact(Ptr self, Ctx &, const Light<Eu> &l, Col &e) {
        const V3 dir = ldv3(self);
        const Col c0 = ldc3(self + 16), c1 = ldc3(self + 32);
        const float power = ldf(self + 48);
        float f = 0.5f * (dot3(l.v, dir) + 1.0f);
        f = (f < 0.0f) ? 0.0f : f;   // clamp = min(max(f, 0), 1) with std::max / std::min (math.hh)
        f = (1.0f < f) ? 1.0f : f;
        f = powf_rounded(f, power);
        const float g = 1.0f - f;
        e.x += (f * c0.x + g * c1.x) * l.k.x;
        e.y += (f * c0.y + g * c1.y) * l.k.y;
        e.z += (f * c0.z + g * c1.z) * l.k.z;
    }
};

// ============================================================================ objects
// detect(self, ctx, cache, light) -> distance; interact(self, ctx, cache, light, emission).
template <class G> struct NormalCache { typename G::Dir normal; };

// A material's interaction out of line: one copy per material type however many variants of
// an object choice share it (the tiled objects call it; each would otherwise inline it).
// Measured on the hy.rs example type: +9 %; a plain covered object keeps it inline (one copy
// anyway, and the call costs the eu.rs type 8 %).
template <class M, int W>
__device__ __noinline__ bool material_interact_shared(Ptr m, Ctx &c, V3 n, LightLocal &l, Col &e) {
    return M::template interact<W>(m, c, n, l, e);
}

template <class G, class S, class M> struct Covered {   // {material, shape} (object/covered.rs:12-18)
    typedef NormalCache<G> Cache;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, Zst, M, S>::lay(); }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, Cache &cache, Light<G> &l) {
        ++c.tests;
        return S::template detect<W, F>(self + Rec<W, Zst, M, S>::off(2), c, cache.normal, l);
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, Cache &cache, Light<G> &l, Col &e) {
        LightLocal ll;   // light_<geo>_to_local
        ll.k = l.k;
        ll.v = G::to_local(l.p, l.v);
        const bool ret = M::template interact<W>(self + Rec<W, Zst, M, S>::off(1), c, G::to_local(l.p, cache.normal), ll, e);
        l.v = G::from_local(l.p, ll.v);   // light_<geo>_update_local
        l.k = ll.k;
        return ret;
    }
};
template <class G, class O, class M> struct MappedObject {   // object/mapped.inl
    typedef typename O::Cache Cache;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Rec<W, Zst, M, O>::lay(); }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, Cache &cache, Light<G> &l) {
        const typename M::V m = M::load(self + Rec<W, Zst, M, O>::off(1));
        if (F) MapOps<M>::ray_cold(M::inverse(m), l.p, l.v);
        else MapOps<M>::ray(M::inverse(m), l.p, l.v);
        const float dist = O::template detect<W, F>(self + Rec<W, Zst, M, O>::off(2), c, cache, l);
        if (F) MapOps<M>::ray_cold(m, l.p, l.v);
        return dist;
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, Cache &cache, Light<G> &l, Col &e) {
        const typename M::V m = M::load(self + Rec<W, Zst, M, O>::off(1));
        MapOps<M>::ray_cold(M::inverse(m), l.p, l.v);
        const bool ret = O::template interact<W>(self + Rec<W, Zst, M, O>::off(2), c, cache, l, e);
        MapOps<M>::ray_cold(m, l.p, l.v);
        return ret;
    }
};
template <class G, class O> struct ObjectVec {   // object/vector.inl
    struct Cache { typename O::Cache inner; u32 index; };
    template <int W> __host__ __device__ static constexpr Lay lay() {
        return Lay{upm((u32)W, O::template lay<W>().align), lcmc((u32)W, O::template lay<W>().align)};
    }
    template <int W> HT_D static u32 count(Ptr self, Ctx &c) {
        constexpr u32 stride = O::template lay<W>().size;
        constexpr u32 head = upm((u32)W, O::template lay<W>().align);
        u32 n = ldusize<W>(self);
        if (stride > 0 && (c.end < self + head || n > (u32)((c.end - self - head) / stride))) { atomicOr(c.err, ERR_SCENE); n = 0; }
        return n;
    }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, Cache &cache, Light<G> &l);
    template <int W, bool F> HT_D static float detect_culled(Ptr self, Ctx &c, Cache &cache, Light<G> &l);
    template <int W, bool F = true> HT_D static float detect_all(Ptr self, Ctx &c, Cache &cache, Light<G> &l) {
        constexpr u32 stride = O::template lay<W>().size;
        constexpr u32 head = upm((u32)W, O::template lay<W>().align);
        // Distances first (no map back, no hit direction), then the winner's full detection
        // again: the same operations give the same bits as keeping every candidate's light
        // and cache (object/vector.inl:24-62), for one map back per hop instead of one per
        // candidate.
        const u32 n = count<W>(self, c);
        const u32 orig = c.hasher;
        float min_dist = -1.0f;
        u32 min_index = 0, min_hasher = orig;
        for (u32 i = 0; i < n; ++i) {
            Light<G> cur = l;
            typename O::Cache cc;
            hash_usize(c, i);
            const float dist = O::template detect<W, false>(self + head + i * stride, c, cc, cur);
            if (dist > -EPSF && (min_dist <= -EPSF || dist < min_dist)) {
                min_dist = dist; min_index = i; min_hasher = c.hasher;
            }
            c.hasher = orig;
        }
        if (!(min_dist > -EPSF)) return -1.0f;
        if (F) {
            const u32 tests = c.tests;
            hash_usize(c, min_index);
            O::template detect<W, true>(self + head + min_index * stride, c, cache.inner, l);
            c.tests = tests;
            cache.index = min_index;
        }
        c.hasher = min_hasher;
        return min_dist;
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, Cache &cache, Light<G> &l, Col &e) {
        constexpr u32 stride = O::template lay<W>().size;
        constexpr u32 head = upm((u32)W, O::template lay<W>().align);
        return O::template interact<W>(self + head + cache.index * stride, c, cache.inner, l, e);
    }
};

// ObjectChoice: one cache per variant (objects/src/object/choice.rs: ChoiceCache).
template <class... O> struct CacheTuple;
template <> struct CacheTuple<> {};
template <class O0, class... O> struct CacheTuple<O0, O...> { typename O0::Cache head; CacheTuple<O...> tail; };
template <class G, class... O> struct ObjectChoiceImpl;
template <class G> struct ObjectChoiceImpl<G> {
    template <int W, bool F = true> HT_D static float detect(u32, Ptr, Ctx &, CacheTuple<> &, Light<G> &) { return -1.0f; }
    template <int W> HT_D static bool interact(u32, Ptr, Ctx &, CacheTuple<> &, Light<G> &, Col &) { return false; }
};
template <class G, class O0, class... O> struct ObjectChoiceImpl<G, O0, O...> {
    template <int W, bool F = true> HT_D static float detect(u32 i, Ptr pay, Ctx &c, CacheTuple<O0, O...> &cache, Light<G> &l) {
        if (i == 0) return O0::template detect<W, F>(pay, c, cache.head, l);
        return ObjectChoiceImpl<G, O...>::template detect<W, F>(i - 1, pay, c, cache.tail, l);
    }
    template <int W> HT_D static bool interact(u32 i, Ptr pay, Ctx &c, CacheTuple<O0, O...> &cache, Light<G> &l, Col &e) {
        if (i == 0) return O0::template interact<W>(pay, c, cache.head, l, e);
        return ObjectChoiceImpl<G, O...>::template interact<W>(i - 1, pay, c, cache.tail, l, e);
    }
};
template <class G, class... O> struct ObjectChoice {   // object/choice/impl.inl
    typedef CacheTuple<O...> Cache;
    template <int W> __host__ __device__ static constexpr Lay lay() { return Enum<W, O...>::lay(); }
    template <int W, bool F = true> HT_D static float detect(Ptr self, Ctx &c, Cache &cache, Light<G> &l) {
        return ObjectChoiceImpl<G, O...>::template detect<W, F>(ldusize<W>(self), self + Enum<W, O...>::payload(), c, cache, l);
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, Cache &cache, Light<G> &l, Col &e) {
        return ObjectChoiceImpl<G, O...>::template interact<W>(ldusize<W>(self), self + Enum<W, O...>::payload(), c, cache, l, e);
    }
};

// ---------------------------------------------------------------- tiled hyperbolic objects
// Tilings (objects/src/object/tiling.rs) and their constants. The pentagonal tilings use
// fixed Moebius maps and directions that the reference recomputes in float on every call
// (object/hy/tiled_plane/impl.inl:50-110); here they are computed once per module by
// tiling_init with the same float operations (transcendentals in FP64, rounded once) and
// read from global memory.
struct TilingUniform {};
struct TilingSquare {};
struct TilingHexagonal {};
struct TilingPentagonal {};
struct TilingPentastar {};

struct PentaTables {
    float Q, S, L, K;
    Mo m0;          // hy_chain(hy_xshift(-Q), hy_zrotate(-PI/4))
    Mo m2[3];       // hy_chain(hy_zrotate(-PI/5), hy_chain(hy_xshift(-2S), hy_zrotate(-o))), o = 2PI(i-1)/5
    Mo m1[2];       // hy_chain(hy_xshift(-2Q), hy_zrotate(-o)), o = PI(2i-1)/5
    float d3x[3], d3y[3];   // (cos, sin) of 2PI(i-1)/5
    float d5x[5], d5y[5];   // (cos, sin) of 2PI i/5
    u32 ready;
};
__device__ PentaTables g_penta;

HT_D float cosr(float x) { return (float)cos((double)x); }
HT_D float sinr(float x) { return (float)sin((double)x); }
HT_D float coshr(float x) { return (float)cosh((double)x); }
HT_D float sinhr(float x) { return (float)sinh((double)x); }
HT_D float logr(float x) { return (float)log((double)x); }
HT_D C2 c2(float x, float y) { C2 r; r.x = x; r.y = y; return r; }
HT_D C2 c_mul(C2 a, C2 b) { return c2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
HT_D C2 c_add(C2 a, C2 b) { return c2(a.x + b.x, a.y + b.y); }
HT_D Mo mo4(C2 a, C2 b, C2 c, C2 d) { Mo m; m.a = a; m.b = b; m.c = c; m.d = d; return m; }
HT_D Mo mo_chain(const Mo &a, const Mo &b) {   // c22_dot (algebra/matrix_complex.cc:38-45)
    return mo4(c_add(c_mul(a.a, b.a), c_mul(a.b, b.c)), c_add(c_mul(a.a, b.b), c_mul(a.b, b.d)),
               c_add(c_mul(a.c, b.a), c_mul(a.d, b.c)), c_add(c_mul(a.c, b.b), c_mul(a.d, b.d)));
}
HT_D Mo hy_xshift(float l) {   // geometry/hyperbolic.cc:40-44
    const float l2 = l / 2.0f;
    const float c = coshr(l2), s = sinhr(l2);
    return mo4(c2(c * 1.0f, c * 0.0f), c2(s * 1.0f, s * 0.0f), c2(s * 1.0f, s * 0.0f), c2(c * 1.0f, c * 0.0f));
}
HT_D Mo hy_zrotate(float phi) {   // geometry/hyperbolic.cc:51-54
    const float c = cosr(phi / 2.0f), s = sinr(phi / 2.0f);
    return mo4(c2(c, s), c2(0.0f, 0.0f), c2(0.0f, 0.0f), c2(c, -s));
}
// One thread fills g_penta (object/hy/tiled_plane/impl.inl:51-60 and the loop's maps).
extern "C" __global__ void htg_tiling_init() {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    PentaTables &t = g_penta;
    const float a = PIF / 4.0f + PIF / 5.0f, b = PIF / 4.0f - PIF / 5.0f;
    float Q = sqrtf(cosr(a) / cosr(b));
    const float T = sqrtf(cosr(a) * cosr(b));
    float S = (cosr(PIF / 4.0f) - sinr(PIF / 5.0f)) / T;
    const float L = T / cosr(PIF / 4.0f);
    const float K = L * (2.0f * cosr(PIF / 5.0f) - 1.0f / cosr(PIF / 5.0f));
    Q = logr((1.0f + Q) / (1.0f - Q));
    S = logr((1.0f + S) / (1.0f - S));
    t.Q = Q; t.S = S; t.L = L; t.K = K;
    t.m0 = mo_chain(hy_xshift(-Q), hy_zrotate(-PIF / 4.0f));
    for (int i = 0; i < 3; ++i) {
        const float o = 2.0f * PIF * (float)(i - 1) / 5.0f;
        t.d3x[i] = cosr(o);
        t.d3y[i] = sinr(o);
        t.m2[i] = mo_chain(hy_zrotate(-PIF / 5.0f), mo_chain(hy_xshift(-2.0f * S), hy_zrotate(-o)));
    }
    for (int i = 0; i < 2; ++i) {
        const float o = PIF * (float)(2 * i - 1) / 5.0f;
        t.m1[i] = mo_chain(hy_xshift(-2.0f * Q), hy_zrotate(-o));
    }
    for (int i = 0; i < 5; ++i) {
        const float o = 2.0f * PIF * (float)i / 5.0f;
        t.d5x[i] = cosr(o);
        t.d5y[i] = sinr(o);
    }
    t.ready = 1u;
}

template <class M, class K, int N> struct TiledFields {   // {tiling, materials, border_material, cell_size, border_width}
    struct Mats { template <int W> __host__ __device__ static constexpr Lay lay() { return Arr<N>::template lay<M, W>(); } };
    template <int W> using R = Rec<W, Zst, Mats, M, F32, F32>;
};
// Interaction of a tiled object: material chosen from the local hit point, then the
// covered-object interaction (light to local, material, update).
template <int W, class M>
HT_D bool tiled_interact(Ptr material, Ctx &c, const Q4 &normal, Light<Hy> &l, Col &e) {
    LightLocal ll;
    ll.k = l.k;
    ll.v = Hy::to_local(l.p, l.v);
    const bool ret = material_interact_shared<M, W>(material, c, Hy::to_local(l.p, normal), ll, e);
    l.v = Hy::from_local(l.p, ll.v);
    l.k = ll.k;
    return ret;
}
// The cell of a pentagonal / pentastar tiling (object/hy/tiled_plane/impl.inl:48-137): 0 / 1
// the cell's material, 2 the border; `one` when the object has a single material. One
// out-of-line copy for both tilings, its reflection loop kept rolled (instruction-cache
// footprint: +4 % on the hy.rs example type).
__device__ __noinline__ u32 penta_cell(float br, Q4 p, bool star, bool one) {
    const PentaTables &t = g_penta;
    bool w = false;
    if (p.x < 0.0f) { p.x = -p.x; w = !w; }
    if (p.y < 0.0f) { p.y = -p.y; w = !w; }
    p = mo_apply_pos(t.m0, p);
    bool e = false;
#pragma unroll 1
    for (int j = 0; j < 5; ++j) {
        bool a[3] = {false, false, false};
        for (int i = 0; i < 3 - (int)e; ++i) a[i] = dot2(t.d3x[i], t.d3y[i], p.x, p.y) < t.L;
        a[2] = a[2] || e;
        const int s = (int)a[0] + (int)a[1] + (int)a[2];
        if (s == 3) break;
        if (s == 2) {
            const int i = (int)(!a[1]) + 2 * (int)(!a[2]);
            p = mo_apply_pos(t.m2[i], p);
            e = true;
            w = !w;
        } else {
            const int i = (int)a[0];
            p = mo_apply_pos(t.m1[i], p);
            e = false;
        }
    }
    bool bh = false;
    for (int i = 0; i < 5; ++i) {
        const float dp = dot2(t.d5x[i], t.d5y[i], p.x, p.y);
        bh = bh || (dp > (t.L - br * p.z));
        if (star) {
            const float ps = t.K + dp;
            w = w ^ (ps < 0.0f);
            bh = bh || (fabsf(ps) < br * p.z);
        }
    }
    if (bh) return 2u;
    return (w || one) ? 0u : 1u;
}

template <class M, class K, int N> struct TiledPlane {   // object/hy/tiled_plane/impl.inl
    typedef NormalCache<Hy> Cache;
    template <int W> using R = typename TiledFields<M, K, N>::template R<W>;
    template <int W> __host__ __device__ static constexpr Lay lay() { return R<W>::lay(); }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, Cache &cache, Light<Hy> &l) {
        ++c.tests;
        return PlaneHy::detect<W, F>(nullptr, c, cache.normal, l);
    }
    template <int W> HT_D static u32 cell(Ptr self, Q4 p) {   // 0 / 1: materials, 2: border
        return penta_cell(ldf(self + R<W>::off(4)), p, K::star, N < 2);
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, Cache &cache, Light<Hy> &l, Col &e) {
        constexpr u32 msz = M::template lay<W>().size;
        Ptr mat = self + R<W>::off(1);
        if (K::penta) {
            const u32 k = cell<W>(self, l.p);
            mat = k == 2u ? self + R<W>::off(2) : self + R<W>::off(1) + k * msz;
        }
        return tiled_interact<W, M>(mat, c, cache.normal, l, e);
    }
};
struct PlaneUniform { static constexpr bool penta = false, star = false; };
struct PlanePentagonal { static constexpr bool penta = true, star = false; };
struct PlanePentastar { static constexpr bool penta = true, star = true; };

// (int)x of a float as the reference's host build converts it (x86 cvttss2si: out of range
// and NaN give INT_MIN); in range it truncates like C.
HT_D int f2i(float x) {
    if (!(x >= -2147483648.0f && x < 2147483648.0f)) return (int)0x80000000u;
    return __float2int_rz(x);
}
HT_D int remi(int a, int b) { return ((a % b) + b) % b; }   // math.hh rem

struct HoroUniform { static constexpr int kind = 0; };
struct HoroSquare { static constexpr int kind = 1; };
struct HoroHexagonal { static constexpr int kind = 2; };
template <class M, class K, int N> struct TiledHorosphere {   // object/hy/tiled_horosphere/impl.inl
    typedef NormalCache<Hy> Cache;
    template <int W> using R = typename TiledFields<M, K, N>::template R<W>;
    template <int W> __host__ __device__ static constexpr Lay lay() { return R<W>::lay(); }
    template <int W, bool F = true> HT_D static float detect(Ptr, Ctx &c, Cache &cache, Light<Hy> &l) {
        ++c.tests;
        return Horosphere::detect<W, F>(nullptr, c, cache.normal, l);
    }
    template <int W> HT_D static bool interact(Ptr self, Ctx &c, Cache &cache, Light<Hy> &l, Col &e) {
        int material_no = 0;
        bool border = false;
        const float cell_size = ldf(self + R<W>::off(3));
        const float br = ldf(self + R<W>::off(4)) / cell_size;
        const float gx = l.p.x, gy = l.p.y;
        if (K::kind == 1) {
            const float vx = gx / cell_size, vy = gy / cell_size;
            const float kx = floorf(vx), ky = floorf(vy);
            const float fx = vx - kx, fy = vy - ky;
            if (fx < br || fx > 1.0f - br || fy < br || fy > 1.0f - br) {
                border = true;
            } else {
                const int hx = remi(f2i(kx), 2), hy = remi(f2i(ky), 2);
                material_no = 3 * hy - 2 * hx * hy + hx;
            }
        } else if (K::kind == 2) {
            const float r3 = sqrtf(3.0f);
            const float bxx = 2.0f / r3, bxy = 0.0f;
            const float byx = -1.0f / r3, byy = 1.0f;
            const float s = cell_size * r3 / 2.0f;
            float hxf = dot2(bxx, bxy, gx, gy) / s;
            float hyf = dot2(byx, byy, gx, gy) / s;
            const int hx = f2i(floorf((floorf(hxf) - floorf(hyf)) / 3.0f));
            const int hy = f2i(floorf((floorf(hxf + hyf) - (float)hx) / 2.0f));
            const float ox = (float)hx * 2.0f + (float)hy * 1.0f;
            const float oy = (float)hx * -1.0f + (float)hy * 1.0f;
            hxf = hxf - ox;
            hyf = hyf - oy;
            if (fabsf(hxf - 1.0f) > 1.0f - br || fabsf(hyf) > 1.0f - br || fabsf(hxf + hyf - 1.0f) > 1.0f - br) {
                border = true;
            } else {
                material_no = 2 * hx + hy;
            }
        }
        constexpr u32 msz = M::template lay<W>().size;
        const Ptr mat = border ? self + R<W>::off(2) : self + R<W>::off(1) + (u32)remi(material_no, N) * msz;
        return tiled_interact<W, M>(mat, c, cache.normal, l, e);
    }
};

// ============================================================================ distance bounds
// Which hyperbolic shape an object is, for the world-space distance bounds of ht_bound.cuh:
// kind 0 = geodesic plane, 1 = horosphere, 2 = read from the object's bytes (a choice whose
// variants are all plane- or horosphere-shaped), -1 = none (the object is never culled).
// of<W>(self) gives the shape of one object (2 for kind -1: no bound record).
template <class O> struct BoundKind {
    static constexpr int kind = -1;
    template <int W> HT_D static u32 of(Ptr) { return 2u; }
};
template <int K> struct BoundKindFixed {
    static constexpr int kind = K;
    template <int W> HT_D static u32 of(Ptr) { return (u32)K; }
};
template <> struct BoundKind<PlaneHy> : BoundKindFixed<0> {};
template <> struct BoundKind<Horosphere> : BoundKindFixed<1> {};
template <class M, class K, int N> struct BoundKind<TiledPlane<M, K, N>> : BoundKindFixed<0> {};
template <class M, class K, int N> struct BoundKind<TiledHorosphere<M, K, N>> : BoundKindFixed<1> {};
template <class S, class M> struct BoundKind<Covered<Hy, S, M>> {
    static constexpr int kind = BoundKind<S>::kind;
    template <int W> HT_D static u32 of(Ptr self) { return BoundKind<S>::template of<W>(self + Rec<W, Zst, M, S>::off(2)); }
};
// A choice: the shape of the variant its index names (all variants of a fixed kind).
template <class... V> struct VariantKind;
template <> struct VariantKind<> {
    static constexpr bool fixed = true;
    HT_D static u32 of(u32) { return 2u; }
};
template <class V0, class... V> struct VariantKind<V0, V...> {
    static constexpr bool fixed = (BoundKind<V0>::kind == 0 || BoundKind<V0>::kind == 1) && VariantKind<V...>::fixed;
    HT_D static u32 of(u32 i) { return i == 0 ? (u32)BoundKind<V0>::kind : VariantKind<V...>::of(i - 1); }
};
template <class... S> struct BoundKind<ShapeChoice<Hy, S...>> {
    static constexpr int kind = VariantKind<S...>::fixed ? 2 : -1;
    template <int W> HT_D static u32 of(Ptr self) { return kind == 2 ? VariantKind<S...>::of(ldusize<W>(self)) : 2u; }
};
template <class... O> struct BoundKind<ObjectChoice<Hy, O...>> {
    static constexpr int kind = VariantKind<O...>::fixed ? 2 : -1;
    template <int W> HT_D static u32 of(Ptr self) { return kind == 2 ? VariantKind<O...>::of(ldusize<W>(self)) : 2u; }
};

// A vector of Moebius-mapped objects of a known shape gets distance bounds: one world-space
// record per element (stage_bound of the element's map) in shared memory, staged once per
// block by render_generic when the vector is the scene's top-level object and holds between
// HTG_BOUND_MIN and HTG_BOUND_CAP elements (below 32 the bound arithmetic costs more than the
// exact tests it saves: the hy.rs example's 4 objects ran 625 Msamples/s with it, 644 without).
#ifndef HTG_BOUND_CAP
#define HTG_BOUND_CAP 256u
#endif
#ifndef HTG_BOUND_MIN
#define HTG_BOUND_MIN 32u
#endif
template <class G, class O> struct VecBounds { static constexpr bool ok = false; };
template <class X> struct VecBounds<Hy, MappedObject<Hy, X, Moebius>> {
    static constexpr bool ok = BoundKind<X>::kind >= 0;
    template <int W> HT_D static u32 kind_of(Ptr elem) {
        return BoundKind<X>::template of<W>(elem + Rec<W, Zst, Moebius, X>::off(2));
    }
    template <int W> HT_D static Mo map_of(Ptr elem) { return Moebius::load(elem + Rec<W, Zst, Moebius, X>::off(1)); }
};
// Stages the records of the vector at `self` (all threads of the block; returns the element
// count staged, or 0xFFFFFFFF when the vector is too small or too large for the bounds or its
// count does not fit the bytes).
template <class G, class O, int W>
HT_D u32 stage_vec_bounds(Ptr self, Ptr end, float4 *rec, float *mag, u32 *kind) {
    typedef VecBounds<G, O> B;
    constexpr u32 stride = O::template lay<W>().size;
    constexpr u32 head = upm((u32)W, O::template lay<W>().align);
    const u32 n = ldusize<W>(self);
    if (stride == 0 || end < self + head || n > (u32)((end - self - head) / stride) || n > HTG_BOUND_CAP ||
        n < HTG_BOUND_MIN)
        return 0xFFFFFFFFu;
    const float nan = __int_as_float(0x7fc00000);
    for (u32 i = threadIdx.x; i < n; i += blockDim.x) {
        const Ptr elem = self + head + i * stride;
        const u32 k = B::template kind_of<W>(elem);
        const float4 r = k <= 1u ? stage_bound(B::template map_of<W>(elem), k) : make_float4(nan, nan, nan, nan);
        rec[i] = r;
        mag[i] = bound_mag(r);
        kind[i] = k;
    }
    return n;
}

template <class G, class O> template <int W, bool F>
HT_D float ObjectVec<G, O>::detect(Ptr self, Ctx &c, Cache &cache, Light<G> &l) {
    if constexpr (VecBounds<G, O>::ok) {
        if (c.bvec == self) return detect_culled<W, F>(self, c, cache, l);
    }
    return detect_all<W, F>(self, c, cache, l);
}

// The scan of ObjectVec::detect_all with the distance bounds of the hand-written hyperbolic
// kernel (ht_trace.cuh hop_hy): an upper estimate of the nearest sure crossing among the first
// 32 elements sets a threshold before the first exact test, each chunk of 32 elements is
// culled by the point bound (warp-uniform) and the ray-aware bound (per lane), and the
// survivors are tested in index order with the threshold tightening on every nearer hit. The
// elements are visited in index order, so the reference's comparison (object/vector.inl:37-50)
// is unchanged; culling only skips elements that cannot be nearer than the threshold.
template <class G, class O> template <int W, bool F>
HT_D float ObjectVec<G, O>::detect_culled(Ptr self, Ctx &c, Cache &cache, Light<G> &l) {
    constexpr u32 stride = O::template lay<W>().size;
    constexpr u32 head = upm((u32)W, O::template lay<W>().align);
    const u32 n = count<W>(self, c);
    const u32 orig = c.hasher;
    const Q4 p = l.p, v = l.v;
    const bool can = cull_point_ok(p);
    const BoundRay br = bound_ray(p, v);
    Cull cull = cull_none();
    if (can) {
        float best = __int_as_float(0x7f800000);
        const u32 ne = n < 32u ? n : 32u;
        for (u32 i = 0; i < ne; ++i) {   // warp-uniform: broadcast loads
            const u32 h = i + (orig << 6) + (orig << 16) - orig;   // the element's hash (hash_usize)
            best = fminf(best, sure_crossing_e2(bound_fw(c.brec[i], c.bmag[i], br), c.bkind[i], h == c.prev, br.t));
        }
        if (best < __int_as_float(0x7f800000)) cull = cull_from_dist(dist_from_e2(best));
    }
    PointCut kp = point_cut(0, br.t, cull), kh = point_cut(1, br.t, cull);
    float min_dist = -1.0f;
    u32 min_index = 0, min_hasher = orig, tested = 0;
    for (u32 c0 = 0; c0 < n; c0 += 32) {
        const u32 cn = n - c0 < 32u ? n - c0 : 32u;
        u32 mask = cn == 32u ? 0xFFFFFFFFu : (1u << cn) - 1u;
        if (can) {
            u32 m = 0;
#pragma unroll 1
            for (u32 j = 0; j < cn; ++j) {   // warp-uniform: broadcast loads
                const u32 k = c0 + j;
                if (!culled_point(c.brec[k], c.bmag[k], br, c.bkind[k] == 0u ? kp : kh)) m |= 1u << j;
            }
            mask = m;
            while (m) {   // per lane: the ray-aware bound on the survivors
                const u32 j = __ffs(m) - 1;
                m &= m - 1;
                const u32 k = c0 + j;
                if (culled<true>(c.brec[k], c.bmag[k], c.bkind[k], br, cull)) mask &= ~(1u << j);
            }
        }
        while (mask) {   // this lane's candidates, in index order
            const u32 i = c0 + (__ffs(mask) - 1);
            mask &= mask - 1;
            if (can && culled_point(c.brec[i], c.bmag[i], br, c.bkind[i] == 0u ? kp : kh)) continue;
            ++tested;
            Light<G> cur = l;
            typename O::Cache cc;
            hash_usize(c, i);
            const float dist = O::template detect<W, false>(self + head + i * stride, c, cc, cur);
            if (dist > -EPSF && (min_dist <= -EPSF || dist < min_dist)) {
                min_dist = dist; min_index = i; min_hasher = c.hasher;
                cull = cull_from_dist(dist);
                kp = point_cut(0, br.t, cull);
                kh = point_cut(1, br.t, cull);
            }
            c.hasher = orig;
        }
    }
    c.culled += n - tested;
    if (!(min_dist > -EPSF)) return -1.0f;
    if (F) {
        const u32 tests = c.tests;
        hash_usize(c, min_index);
        O::template detect<W, true>(self + head + min_index * stride, c, cache.inner, l);
        c.tests = tests;
        cache.index = min_index;
    }
    c.hasher = min_hasher;
    return min_dist;
}

// ============================================================================ scene
template <class G, class V, class O, class B> struct SceneImpl {   // {phantom, view, background, object}
    template <int W> using R = Rec<W, Zst, V, B, O>;
    typedef O Object;
    typedef G Geometry;
    template <int W> __host__ __device__ static constexpr u32 static_size() { return R<W>::off(3) + O::template lay<W>().size; }
    // render/scene.inl:16-44 with H = hops; returns the path's emission.
    template <int W>
    HT_D static Col sample(Ptr self, Ctx &c, float px, float py, float size, u32 hops, u32 &hops_done, u32 &hits) {
        Light<G> l = V::template sample<W>(self + R<W>::off(1), c, px, py, size);
        l.k.x = 1.0f; l.k.y = 1.0f; l.k.z = 1.0f;
        Col e; e.x = 0.0f; e.y = 0.0f; e.z = 0.0f;
        c.prev = HASH_NEVER;
        for (u32 i = 0; i < hops; ++i) {
            c.hasher = 0u;
            typename O::Cache cache;
            ++hops_done;
            const float dist = O::template detect<W, true>(self + R<W>::off(3), c, cache, l);
            if (dist > -0.5f) {
                ++hits;
                const bool ret = O::template interact<W>(self + R<W>::off(3), c, cache, l, e);
                if (!ret) break;
                c.prev = c.hasher;
            } else {
                B::template interact<W>(self + R<W>::off(2), c, l, e);
                break;
            }
        }
        return e;
    }
};

// The element type of a top-level object vector.
template <class O> struct VecElem { static constexpr bool is_vec = false; typedef Zst T; };
template <class G, class O> struct VecElem<ObjectVec<G, O>> { static constexpr bool is_vec = true; typedef O T; };

// ============================================================================ kernel
// One thread per pixel (render/render.cl:6-27); `passes` samples of the pixel in order, the
// same float additions as `passes` launches of one pass.
// Resident 128-thread blocks per SM requested from ptxas (register cap 64): the scan is a
// chain of dependent FP32 operations, so more resident warps beat the few spilled values
// (8 blocks measured fastest against 1, 5, 6, 7 on the example scene types).
#ifndef HTG_MIN_BLOCKS
#define HTG_MIN_BLOCKS 8
#endif
template <class Scene, int W>
__global__ void __launch_bounds__(128, HTG_MIN_BLOCKS) render_generic(Ptr scene, uint64_t scene_size, u32 width, u32 height,
                                                     u32 hops, u32 passes, u32 flags, float4 *canvas, u32 *seeds,
                                                     unsigned long long *stats, u32 *err) {
    const u32 idx = blockIdx.x * 128u + threadIdx.x;
    u32 samples = 0, hops_done = 0, hits = 0, tests = 0, culled = 0;
    typedef typename Scene::Object Obj;
    typedef typename Scene::Geometry Geo;
    Ptr bvec = nullptr;
    const float4 *brec = nullptr;
    const float *bmag = nullptr;
    const u32 *bkind = nullptr;
    if constexpr (VecBounds<Geo, typename VecElem<Obj>::T>::ok && VecElem<Obj>::is_vec) {
        // the top-level object vector's distance bounds, staged once per block
        __shared__ float4 s_rec[HTG_BOUND_CAP];
        __shared__ float s_mag[HTG_BOUND_CAP];
        __shared__ u32 s_kind[HTG_BOUND_CAP];
        const Ptr vec = scene + Scene::template R<W>::off(3);
        const u32 nb = stage_vec_bounds<Geo, typename VecElem<Obj>::T, W>(vec, scene + scene_size, s_rec, s_mag, s_kind);
        __syncthreads();
        if (nb != 0xFFFFFFFFu) {
            bvec = vec;
            brec = s_rec;
            bmag = s_mag;
            bkind = s_kind;
        }
    }
    if (idx < width * height) {
        const u32 x = idx % width, y = idx / width;
        const float px = (__uint2float_rn(2u * x + 1u) - __uint2float_rn(width)) / __uint2float_rn(height);
        const float py = (__uint2float_rn(height) - __uint2float_rn(2u * y + 1u)) / __uint2float_rn(height);
        const float size = 2.0f / __uint2float_rn(height);
        Ctx c;
        c.rng = seeds[idx];
        c.hasher = 0u;
        c.prev = HASH_NEVER;
        c.flags = flags;
        c.tests = 0;
        c.end = scene + scene_size;
        c.err = err;
        c.bvec = bvec;
        c.brec = brec;
        c.bmag = bmag;
        c.bkind = bkind;
        c.culled = 0;
        float4 acc = canvas[idx];
        for (u32 k = 0; k < passes; ++k) {
            const Col col = Scene::template sample<W>(scene, c, px, py, size, hops, hops_done, hits);
            acc.x += col.x; acc.y += col.y; acc.z += col.z; acc.w += 1.0f;
            ++samples;
        }
        canvas[idx] = acc;
        seeds[idx] = c.rng;
        tests = c.tests;
        culled = c.culled;
    }
    if (stats) {   // samples, hops, object tests the reference makes, hits, tests evaluated
        unsigned long long v[5] = {samples, hops_done, (unsigned long long)tests + culled, hits, tests};
        for (int k = 0; k < 5; ++k) {
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xFFFFFFFFu, v[k], o);
        }
        if ((threadIdx.x & 31u) == 0) {
            for (int k = 0; k < 5; ++k) atomicAdd(stats + k, v[k]);
        }
    }
}

}  // namespace htg
