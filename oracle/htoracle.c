/*
 * htoracle.c -- CPU restatement of hypertrace's per-pixel path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle the CUDA path is checked against; it is
 * never linked into, called by, or used as a fallback for the product. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity is pinned two ways (tests/test_oracle_pin.py):
 *   - against oracle/_ref, the reference's own kernel sources compiled as host C++
 *     (bit-exact RNG state and radiance for the same scene bytes and seeds);
 *   - against the committed fixtures in tests/golden/ generated from oracle/_ref.
 *
 * Built twice: REAL=float (the f32 path the GPU mirrors) and -DHT_REAL_DOUBLE (the FP64
 * accuracy oracle, like the reference's DOUBLE_PRECISION build,
 * kernel/CMakeLists.txt:90-96). Colors stay float in both, as in the reference
 * (kernel/ocl/algebra/color.hh:6-7).
 *
 * Every arithmetic expression keeps the reference's evaluation order and its rounding
 * points (compile with -ffp-contract=off); each function cites the file:line it restates
 * (paths relative to the reference project).
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>

#ifdef HT_REAL_DOUBLE
typedef double R;
#define EPS 1e-12
#define PI_R 3.141592653589793238462643383279502884
#define RSQRT(x) sqrt(x)
#define RLOG(x) log(x)
#define RCOS(x) cos(x)
#define RSIN(x) sin(x)
#define RFABS(x) fabs(x)
#define HTO(name) hto64_##name
#else
typedef float R;
#define EPS 1e-6f
#define PI_R 3.141592653589793238462643383279502884f
#define RSQRT(x) sqrtf(x)
#define RLOG(x) logf(x)
#define RCOS(x) cosf(x)
#define RSIN(x) sinf(x)
#define RFABS(x) fabsf(x)
#define HTO(name) hto32_##name
#endif

typedef struct { R x, y; } comp;
typedef struct { R x, y, z, w; } quat;   /* x = real part; (y, z, w) = i, j, k */
typedef struct { R x, y, z; } vec3;
typedef struct { float x, y, z; } col3;
typedef struct { comp a, b, c, d; } moebius;   /* (a p + b)(c p + d)^-1 */
typedef struct { vec3 shift; quat rot; } hom3;  /* Chain<Shift3, Rotation3> */

/* Flags. */
#define HTO_JITTER_YX 1u  /* first jitter draw -> y (g++ host order of random_uniform2) */

enum { RECIPE_HY = 1, RECIPE_EU = 2 };
enum { OBJ_STRIDE = 128 };

/* ------------------------------------------------------------------ RNG
 * kernel/ocl/random.cc:8-14: LCG, u = (real)s / (real)2^32. */
static inline uint32_t rng_next(uint32_t *s) { *s = 1103515245u * *s + 12345u; return *s; }
static inline R rng_uniform(uint32_t *s) {
    return (R)rng_next(s) / (R)4294967296.0;
}

/* ------------------------------------------------------------------ vectors
 * dot: kernel/ocl/algebra/vector_math.hpp:8-15 (c = 0; c += a[i]*b[i]). */
static inline R dot2(R ax, R ay, R bx, R by) { R c = 0; c += ax * bx; c += ay * by; return c; }
static inline R dot3(vec3 a, vec3 b) { R c = 0; c += a.x * b.x; c += a.y * b.y; c += a.z * b.z; return c; }
static inline R dot4(quat a, quat b) {
    R c = 0; c += a.x * b.x; c += a.y * b.y; c += a.z * b.z; c += a.w * b.w; return c;
}
static inline vec3 v3(R x, R y, R z) { vec3 r = {x, y, z}; return r; }
static inline quat q4(R x, R y, R z, R w) { quat r = {x, y, z, w}; return r; }
/* normalize = a / length(a): vector_math.hpp:29-42 */
static inline vec3 normalize3(vec3 a) { R l = RSQRT(dot3(a, a)); return v3(a.x / l, a.y / l, a.z / l); }
static inline quat normalize4(quat a) { R l = RSQRT(dot4(a, a)); return q4(a.x / l, a.y / l, a.z / l, a.w / l); }
static inline vec3 cross3(vec3 a, vec3 b) {  /* vector_math.hpp:16-23 */
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

/* ------------------------------------------------------------------ quaternions
 * kernel/ocl/algebra/quaternion.cc:4-56 */
static inline quat q_conj(quat a) { return q4(a.x, -a.y, -a.z, -a.w); }
static inline quat q_mul(quat a, quat b) {
    return q4(
        a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
        a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
        a.x * b.z + a.z * b.x - a.y * b.w + a.w * b.y,
        a.x * b.w + a.w * b.x + a.y * b.z - a.z * b.y);
}
static inline quat cq_mul(comp a, quat b) {
    return q4(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x, a.x * b.z - a.y * b.w, a.x * b.w + a.y * b.z);
}
static inline quat q_inverse(quat a) {
    quat c = q_conj(a); R n = dot4(a, a);
    return q4(c.x / n, c.y / n, c.z / n, c.w / n);
}
static inline quat q_div(quat a, quat b) { return q_mul(a, q_inverse(b)); }
static inline quat q_add(quat a, quat b) { return q4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline quat q_sub(quat a, quat b) { return q4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
static inline quat q_scale(R k, quat a) { return q4(k * a.x, k * a.y, k * a.z, k * a.w); }
static inline quat q_divs(quat a, R k) { return q4(a.x / k, a.y / k, a.z / k, a.w / k); }
static inline quat q_from_c(comp c) { return q4(c.x, c.y, (R)0, (R)0); }  /* q_new(c, C0) */

/* ------------------------------------------------------------------ Moebius
 * kernel/ocl/transform/moebius.cc:20-56 */
static inline quat mo_apply_q(moebius m, quat p) {
    return q_div(q_add(cq_mul(m.a, p), q_from_c(m.b)), q_add(cq_mul(m.c, p), q_from_c(m.d)));
}
static inline quat mo_deriv_q(moebius m, quat p, quat v) {
    quat u = q_add(cq_mul(m.a, p), q_from_c(m.b));
    quat d = q_add(cq_mul(m.c, p), q_from_c(m.d));
    R d2 = dot4(d, d);
    quat g1 = q_div(cq_mul(m.a, v), d);
    quat cv = cq_mul(m.c, v);
    quat g21 = q_conj(cv);
    quat g22 = q_scale(((R)2 * dot4(d, cv)) / d2, q_conj(d));
    quat g2 = q_mul(u, q_divs(q_sub(g21, g22), d2));
    return q_add(g1, g2);
}
/* mo_inverse = c22_inverse_n (adjugate, det = 1 assumed): matrix_complex.cc:60-65 */
static inline moebius mo_inverse(moebius m) {
    moebius r;
    r.a = m.d;
    r.b.x = -m.b.x; r.b.y = -m.b.y;
    r.c.x = -m.c.x; r.c.y = -m.c.y;
    r.d = m.a;
    return r;
}

typedef struct { quat start, dir; } ray_hy;
typedef struct { vec3 start, dir; } ray_eu;

/* ray_<geo>_map: geometry/ray_map.inl:15-21 (apply_pos, normalize(apply_dir));
 * mo_apply_dir already normalizes once (moebius.cc:47-49). */
static inline ray_hy ray_hy_map(ray_hy r, moebius m) {
    ray_hy o;
    o.start = mo_apply_q(m, r.start);
    o.dir = normalize4(normalize4(mo_deriv_q(m, r.start, r.dir)));
    return o;
}

/* ------------------------------------------------------------------ Euclidean maps
 * rotation.cc: rot3_apply_pos = (q (0,p) q*).yzw ; chain.inl:36-73 ; shift.cc:44-59 */
static inline vec3 rot3_apply(quat q, vec3 p) {
    quat r = q_mul(q_mul(q, q4((R)0, p.x, p.y, p.z)), q_conj(q));
    return v3(r.y, r.z, r.w);
}
static inline vec3 hom3_apply_pos(hom3 m, vec3 p) {
    vec3 r = rot3_apply(m.rot, p);
    return v3(r.x + m.shift.x, r.y + m.shift.y, r.z + m.shift.z);
}
static inline vec3 hom3_apply_dir(hom3 m, vec3 d) { return rot3_apply(m.rot, d); }
static inline hom3 hom3_inverse(hom3 m) {  /* chain.inl:65-73 */
    hom3 s;
    s.shift = v3(-m.shift.x, -m.shift.y, -m.shift.z);
    s.rot = q_conj(m.rot);
    s.shift = rot3_apply(s.rot, s.shift);  /* rot3_shf3_reorder */
    return s;
}
static inline ray_eu ray_eu_map(ray_eu r, hom3 m) {
    ray_eu o;
    o.start = hom3_apply_pos(m, r.start);
    o.dir = normalize3(hom3_apply_dir(m, r.dir));
    return o;
}

/* ------------------------------------------------------------------ hyperbolic geometry
 * geometry/hyperbolic.cc:20-33 */
static inline R hy_distance(quat a, quat b) {
    quat d = q_sub(a, b);
    R x = (R)1 + dot4(d, d) / ((R)2 * a.z * b.z);
    return RLOG(x + RSQRT(x * x - (R)1));
}
static inline quat hy_dir_at(quat p, quat d, quat h) {
    R lpxy = RSQRT(dot2(p.x - h.x, p.y - h.y, p.x - h.x, p.y - h.y));
    R ldxy = RSQRT(dot2(d.x, d.y, d.x, d.y));
    return q4(h.z / p.z * d.x, h.z / p.z * d.y, d.z - lpxy / p.z * ldxy, (R)0);
}

/* ------------------------------------------------------------------ shapes
 * Each returns the hit distance or -1, and on a hit rewrites the ray start/direction
 * and the local normal. */
static inline R plane_hy_detect(int repeat, quat *normal, ray_hy *ray) {  /* shape/hy/plane.cc:4-37 */
    if (repeat) return (R)-1;
    quat p = ray->start, d = ray->dir;
    R pd = dot4(p, d);
    if (RFABS(pd) < EPS) return (R)-1;
    R s = (R)1 - dot4(p, p);
    R t = s / ((R)2 * pd);
    if (t < -EPS) return (R)-1;
    quat h = q4(p.x + d.x * t, p.y + d.y * t, (R)0, (R)0);
    R pxy2 = dot2(h.x, h.y, h.x, h.y);
    if (pxy2 > (R)1) return (R)-1;
    h.z = RSQRT((R)1 - pxy2);
    ray->start = h;
    ray->dir = hy_dir_at(p, d, h);
    *normal = q4(-h.x, -h.y, -h.z, -h.w);
    return hy_distance(p, h);
}
static inline R horosphere_detect(int repeat, quat *normal, ray_hy *ray) {  /* shape/hy/horosphere.cc:4-34 */
    quat p = ray->start, d = ray->dir;
    R dxy = RSQRT(dot2(d.x, d.y, d.x, d.y));
    if (p.z < dxy) return (R)-1;
    R dt = RSQRT(p.z * p.z - dxy * dxy);
    R t = p.z * d.z - dt;
    R w = EPS * (R)(2 * repeat - 1);
    if (t < w) {
        t += (R)2 * dt;
        if (t < w) return (R)-1;
    }
    t /= dxy * dxy;
    quat h = q4(p.x + d.x * t, p.y + d.y * t, (R)1, (R)0);
    ray->start = h;
    ray->dir = hy_dir_at(p, d, h);
    *normal = q4((R)0, (R)0, (R)-1, (R)0);
    return hy_distance(p, h);
}
static inline R sphere_eu_detect(int repeat, vec3 *normal, ray_eu *ray) {  /* shape/eu/sphere.cc:3-29 */
    vec3 pos = ray->start, dir = ray->dir;
    R b = -dot3(dir, pos);
    vec3 g = v3(pos.x + dir.x * b, pos.y + dir.y * b, pos.z + dir.z * b);
    R d = (R)1 - dot3(g, g);
    if (d < (R)0) return (R)-1;
    d = RSQRT(d);
    R e = b - d;
    R w = EPS * (R)(2 * repeat - 1);
    if (e < w) {
        e = b + d;
        if (e < w) return (R)-1;
    }
    vec3 h = normalize3(v3(pos.x + dir.x * e, pos.y + dir.y * e, pos.z + dir.z * e));
    *normal = h;
    ray->start = h;
    return e;
}
static inline R plane_eu_detect(int repeat, vec3 *normal, ray_eu *ray) {  /* shape/eu/plane.cc:3-21 */
    if (repeat) return (R)-1;
    vec3 pos = ray->start, dir = ray->dir;
    if (pos.z * dir.z > (R)0) return (R)-1;
    R t = -pos.z / dir.z;
    ray->start = v3(pos.x + dir.x * t, pos.y + dir.y * t, (R)0);
    *normal = v3((R)0, (R)0, (R)-1);
    return t;
}

/* ------------------------------------------------------------------ materials */
/* random_hemisphere_cosine: random.cc:37-39,53-59 */
static inline vec3 hemisphere_cosine(uint32_t *s) {
    R phi = (R)2 * PI_R * rng_uniform(s);
    R sqr_cos_theta = rng_uniform(s);
    R cos_theta = RSQRT(sqr_cos_theta);
    R sin_theta = RSQRT((R)1 - sqr_cos_theta);
    return v3(RCOS(phi) * sin_theta, RSIN(phi) * sin_theta, cos_theta);
}
/* rot3_look_at_cont / rot3_look_at / rot3_from_axis: transform/rotation.cc */
static inline quat rot3_look_at_cont(vec3 d) {
    vec3 z = v3((R)0, (R)0, (R)-1);
    R c2 = dot3(d, z);
    R c = RSQRT(((R)1 + c2) / (R)2);
    R sm = (R)1 / ((R)2 * c);
    vec3 x = cross3(z, d);
    return q4(c, sm * x.x, sm * x.y, sm * x.z);
}
static inline quat rot3_look_at(vec3 d) {
    if (d.z < (R)0) return rot3_look_at_cont(d);
    quat a = rot3_look_at_cont(v3(-d.x, -d.y, -d.z));
    R half = PI_R / (R)2;
    R sh = RSIN(half);
    quat b = q4(RCOS(half), sh * (R)1, sh * (R)0, sh * (R)0);
    return q_mul(a, b);
}

typedef struct {
    col3 diffuse_color; R diffuse_portion;
    R specular_portion;
    col3 emission; R luminous_portion;
    uint32_t shape;
} material_rec;

/* Mixture interact (material/mixture/impl.inl:16-27 + macros.hh:3-13) with the three
 * components: Colored<Lambertian> (colored.inl:15-23, lambertian.cc:6-14),
 * Specular (specular.cc:4-7), Emissive<Absorbing> (emissive.inl:15-23, absorbing.cc:4-6).
 * Returns false when the path ends. */
static inline int mixture_interact(const material_rec *m, uint32_t *rng, vec3 normal,
                                   vec3 *dir, col3 *intensity, col3 *emission) {
    R alpha = rng_uniform(rng);
    alpha -= m->diffuse_portion;
    if (alpha < (R)0) {
        intensity->x *= m->diffuse_color.x;
        intensity->y *= m->diffuse_color.y;
        intensity->z *= m->diffuse_color.z;
        if (dot3(*dir, normal) > (R)0) normal = v3(-normal.x, -normal.y, -normal.z);
        vec3 rnd = hemisphere_cosine(rng);
        quat rot = rot3_look_at(v3(-normal.x, -normal.y, -normal.z));
        *dir = rot3_apply(rot, rnd);
        return 1;
    }
    alpha -= m->specular_portion;
    if (alpha < (R)0) {
        R k = (R)2 * dot3(*dir, normal);
        *dir = v3(dir->x - k * normal.x, dir->y - k * normal.y, dir->z - k * normal.z);
        return 1;
    }
    alpha -= m->luminous_portion;
    if (alpha < (R)0) {
        emission->x += intensity->x * m->emission.x;
        emission->y += intensity->y * m->emission.y;
        emission->z += intensity->z * m->emission.z;
        return 0;
    }
    return 0;  /* "unreachable" fall-through of the mixture: the path ends */
}

/* ------------------------------------------------------------------ scene */
typedef struct {
    int recipe;
    uint32_t n;
    R fov;
    col3 background;
    moebius cam_mo;
    hom3 cam_hom;
    moebius *mo;      /* per object map (hyperbolic) */
    moebius *mo_inv;
    hom3 *hom;        /* per object map (euclidean) */
    hom3 *hom_inv;
    material_rec *mat;
} scene_t;

static float rd_f(const uint8_t *b, size_t off) { float v; memcpy(&v, b + off, 4); return v; }
static uint32_t rd_u(const uint8_t *b, size_t off) { uint32_t v; memcpy(&v, b + off, 4); return v; }

static moebius rd_mo(const uint8_t *b) {
    moebius m;
    m.a.x = rd_f(b, 0);  m.a.y = rd_f(b, 4);
    m.b.x = rd_f(b, 8);  m.b.y = rd_f(b, 12);
    m.c.x = rd_f(b, 16); m.c.y = rd_f(b, 20);
    m.d.x = rd_f(b, 24); m.d.y = rd_f(b, 28);
    return m;
}
static hom3 rd_hom(const uint8_t *b) {
    hom3 m;
    m.shift = v3(rd_f(b, 0), rd_f(b, 4), rd_f(b, 8));
    m.rot = q4(rd_f(b, 16), rd_f(b, 20), rd_f(b, 24), rd_f(b, 28));
    return m;
}

static void scene_free(scene_t *s) {
    free(s->mo); free(s->mo_inv); free(s->hom); free(s->hom_inv); free(s->mat);
    memset(s, 0, sizeof(*s));
}

/* Scene byte ABI: see hypertrace_b200/scene.py (serializer) and include/htcuda.h. */
static int scene_parse(int recipe, const uint8_t *b, size_t len, int address_width, scene_t *s) {
    memset(s, 0, sizeof(*s));
    if (address_width != 32 && address_width != 64) return -4;
    size_t hdr, objs;
    if (recipe == RECIPE_HY) { hdr = 96; objs = 128; }
    else if (recipe == RECIPE_EU) { hdr = 64; objs = 80; }
    else return -2;
    if (len < objs) return -1;
    s->recipe = recipe;
    s->n = rd_u(b, hdr);
    if (address_width == 64 && rd_u(b, hdr + 4) != 0) return -1;
    if ((len - objs) / OBJ_STRIDE < s->n) return -1;
    s->fov = rd_f(b, 32);
    size_t bg = recipe == RECIPE_HY ? 64 : 48;
    s->background.x = rd_f(b, bg); s->background.y = rd_f(b, bg + 4); s->background.z = rd_f(b, bg + 8);
    uint32_t n = s->n ? s->n : 1;
    s->mat = (material_rec *)calloc(n, sizeof(material_rec));
    if (recipe == RECIPE_HY) {
        s->cam_mo = rd_mo(b);
        s->mo = (moebius *)calloc(n, sizeof(moebius));
        s->mo_inv = (moebius *)calloc(n, sizeof(moebius));
    } else {
        s->cam_hom = rd_hom(b);
        s->hom = (hom3 *)calloc(n, sizeof(hom3));
        s->hom_inv = (hom3 *)calloc(n, sizeof(hom3));
    }
    for (uint32_t i = 0; i < s->n; ++i) {
        const uint8_t *o = b + objs + (size_t)i * OBJ_STRIDE;
        material_rec *m = &s->mat[i];
        m->diffuse_color.x = rd_f(o, 32); m->diffuse_color.y = rd_f(o, 36); m->diffuse_color.z = rd_f(o, 40);
        m->diffuse_portion = rd_f(o, 48);
        m->specular_portion = rd_f(o, 64);
        m->emission.x = rd_f(o, 80); m->emission.y = rd_f(o, 84); m->emission.z = rd_f(o, 88);
        m->luminous_portion = rd_f(o, 96);
        m->shape = rd_u(o, 112);
        if (address_width == 64 && rd_u(o, 116) != 0) { scene_free(s); return -1; }
        if (m->shape > 1) { scene_free(s); return -5; }
        if (recipe == RECIPE_HY) {
            s->mo[i] = rd_mo(o);
            s->mo_inv[i] = mo_inverse(s->mo[i]);
        } else {
            s->hom[i] = rd_hom(o);
            s->hom_inv[i] = hom3_inverse(s->hom[i]);
        }
    }
    return 0;
}

typedef struct { uint64_t samples, hops, object_tests, hits; } stats_t;

/* <scene>_sample: render/scene.inl:16-44, with the object vector detect of
 * object/vector.inl:24-62 (nearest hit, ties to the lowest index, hash = index since the
 * hasher restarts from 0 every hop: hash.cc:11-14, context.cc:11-13) and the mapped
 * object detect/interact of object/mapped.inl:24-51. */
static col3 sample_hy(const scene_t *sc, uint32_t hops, uint32_t *rng, R px, R py, R size,
                      uint32_t flags, stats_t *st) {
    /* view: view/point/impl.inl:18-25 then view/mapped.inl:20-26 */
    R u0 = rng_uniform(rng);
    R u1 = rng_uniform(rng);
    R jx = (flags & HTO_JITTER_YX) ? u1 : u0;
    R jy = (flags & HTO_JITTER_YX) ? u0 : u1;
    R sx = px + size * (jx - (R)0.5f);
    R sy = py + size * (jy - (R)0.5f);
    vec3 ld = normalize3(v3(sx, sy, (R)-1 / sc->fov));
    quat start = q4((R)0, (R)0, (R)1, (R)0);
    quat dir = q4(ld.x, ld.y, ld.z, (R)0);
    ray_hy ray;
    ray.dir = normalize4(mo_deriv_q(sc->cam_mo, start, dir));
    ray.start = mo_apply_q(sc->cam_mo, start);

    col3 intensity = {1.0f, 1.0f, 1.0f};
    col3 emission = {0.0f, 0.0f, 0.0f};
    uint32_t prev_hash = 0xFFFFFFFFu;
    st->samples += 1;
    for (uint32_t i = 0; i < hops; ++i) {
        st->hops += 1;
        st->object_tests += sc->n;
        R min_dist = (R)-1;
        uint32_t min_index = 0;
        ray_hy min_local = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        quat min_normal = {0, 0, 0, 0};
        for (uint32_t k = 0; k < sc->n; ++k) {
            int repeat = (k == prev_hash);
            ray_hy local = ray_hy_map(ray, sc->mo_inv[k]);
            quat normal;
            R dist = sc->mat[k].shape == 0 ? plane_hy_detect(repeat, &normal, &local)
                                           : horosphere_detect(repeat, &normal, &local);
            /* the reference maps every candidate back (mapped.inl:34); only the kept one
             * is observable, so it is mapped back once below */
            if (dist > -EPS && (min_dist <= -EPS || dist < min_dist)) {
                min_dist = dist; min_index = k; min_local = local; min_normal = normal;
            }
        }
        if (min_dist > -EPS) {
            st->hits += 1;
            ray_hy hit = ray_hy_map(min_local, sc->mo[min_index]);
            /* interact: mapped.inl:39-51 -> covered.inl:38-56 -> light/hy.cc */
            ray_hy loc = ray_hy_map(hit, sc->mo_inv[min_index]);
            vec3 d3 = v3(loc.dir.x, loc.dir.y, loc.dir.z);
            vec3 n3 = v3(min_normal.x, min_normal.y, min_normal.z);
            int ret = mixture_interact(&sc->mat[min_index], rng, n3, &d3, &intensity, &emission);
            loc.dir = q4(d3.x, d3.y, d3.z, (R)0);
            ray = ray_hy_map(loc, sc->mo[min_index]);
            if (!ret) break;
            prev_hash = min_index;
        } else {
            /* background/constant.inl:18-21 */
            emission.x += sc->background.x * intensity.x;
            emission.y += sc->background.y * intensity.y;
            emission.z += sc->background.z * intensity.z;
            break;
        }
    }
    return emission;
}

static col3 sample_eu(const scene_t *sc, uint32_t hops, uint32_t *rng, R px, R py, R size,
                      uint32_t flags, stats_t *st) {
    R u0 = rng_uniform(rng);
    R u1 = rng_uniform(rng);
    R jx = (flags & HTO_JITTER_YX) ? u1 : u0;
    R jy = (flags & HTO_JITTER_YX) ? u0 : u1;
    R sx = px + size * (jx - (R)0.5f);
    R sy = py + size * (jy - (R)0.5f);
    vec3 ld = normalize3(v3(sx, sy, (R)-1 / sc->fov));
    ray_eu ray;
    ray.dir = hom3_apply_dir(sc->cam_hom, ld);
    ray.start = hom3_apply_pos(sc->cam_hom, v3((R)0, (R)0, (R)0));

    col3 intensity = {1.0f, 1.0f, 1.0f};
    col3 emission = {0.0f, 0.0f, 0.0f};
    uint32_t prev_hash = 0xFFFFFFFFu;
    st->samples += 1;
    for (uint32_t i = 0; i < hops; ++i) {
        st->hops += 1;
        st->object_tests += sc->n;
        R min_dist = (R)-1;
        uint32_t min_index = 0;
        ray_eu min_local = {{0, 0, 0}, {0, 0, 0}};
        vec3 min_normal = {0, 0, 0};
        for (uint32_t k = 0; k < sc->n; ++k) {
            int repeat = (k == prev_hash);
            ray_eu local = ray_eu_map(ray, sc->hom_inv[k]);
            vec3 normal;
            R dist = sc->mat[k].shape == 0 ? plane_eu_detect(repeat, &normal, &local)
                                           : sphere_eu_detect(repeat, &normal, &local);
            if (dist > -EPS && (min_dist <= -EPS || dist < min_dist)) {
                min_dist = dist; min_index = k; min_local = local; min_normal = normal;
            }
        }
        if (min_dist > -EPS) {
            st->hits += 1;
            ray_eu hit = ray_eu_map(min_local, sc->hom[min_index]);
            ray_eu loc = ray_eu_map(hit, sc->hom_inv[min_index]);
            int ret = mixture_interact(&sc->mat[min_index], rng, min_normal, &loc.dir, &intensity, &emission);
            ray = ray_eu_map(loc, sc->hom[min_index]);
            if (!ret) break;
            prev_hash = min_index;
        } else {
            emission.x += sc->background.x * intensity.x;
            emission.y += sc->background.y * intensity.y;
            emission.z += sc->background.z * intensity.z;
            break;
        }
    }
    return emission;
}

/* render: render/render.cl:6-27 for one pixel index. */
static void render_pixel(const scene_t *sc, uint32_t hops, uint32_t W, uint32_t H, uint32_t px,
                         float *canvas4, uint32_t *seed, uint32_t flags, stats_t *st) {
    uint32_t x = px % W, y = px / W;
    R pxr = ((R)(2u * x + 1u) - (R)W) / (R)H;
    R pyr = ((R)H - (R)(2u * y + 1u)) / (R)H;
    R size = (R)2 / (R)H;
    uint32_t rng = *seed;
    col3 c = sc->recipe == RECIPE_HY ? sample_hy(sc, hops, &rng, pxr, pyr, size, flags, st)
                                     : sample_eu(sc, hops, &rng, pxr, pyr, size, flags, st);
    canvas4[0] += c.x;
    canvas4[1] += c.y;
    canvas4[2] += c.z;
    canvas4[3] += 1.0f;
    *seed = rng;
}

typedef struct {
    const scene_t *sc;
    uint32_t hops, W, H, passes, flags;
    const uint32_t *pixels;
    size_t n;
    float *canvas;
    uint32_t *seeds;
    size_t next;
    pthread_mutex_t lock;
} job_t;

typedef struct { job_t *job; stats_t st; } worker_t;

static void *worker_main(void *arg) {
    worker_t *w = (worker_t *)arg;
    job_t *j = w->job;
    const size_t CHUNK = 64;
    for (;;) {
        pthread_mutex_lock(&j->lock);
        size_t start = j->next;
        j->next += CHUNK;
        pthread_mutex_unlock(&j->lock);
        if (start >= j->n) break;
        size_t end = start + CHUNK < j->n ? start + CHUNK : j->n;
        for (size_t i = start; i < end; ++i)
            for (uint32_t p = 0; p < j->passes; ++p)
                render_pixel(j->sc, j->hops, j->W, j->H, j->pixels[i], j->canvas + 4 * i,
                             j->seeds + i, j->flags, &w->st);
    }
    return NULL;
}

/* Renders `passes` passes over the listed pixels; same contract as htref_render.
 * Returns 0, or a negative error (-1 short/bad scene, -2 unknown recipe, -3 bad hops,
 * -4 bad address width, -5 bad shape index). */
static int render_ext(int recipe, uint32_t hops, const uint8_t *scene, size_t scene_len, int address_width,
                      uint32_t W, uint32_t H, const uint32_t *pixels, size_t n_pixels, uint32_t passes,
                      float *canvas, uint32_t *seeds, uint32_t flags, int threads, uint64_t *stats);

int HTO(render)(int recipe, uint32_t hops, const uint8_t *scene, size_t scene_len, int address_width,
                uint32_t W, uint32_t H, const uint32_t *pixels, size_t n_pixels, uint32_t passes,
                float *canvas, uint32_t *seeds, uint32_t flags, int threads, uint64_t *stats) {
    if (recipe == 3 || recipe == 4 || recipe == 5)
        return render_ext(recipe, hops, scene, scene_len, address_width, W, H, pixels, n_pixels, passes, canvas,
                          seeds, flags, threads, stats);
    if (hops == 0) return -3;
    if (W == 0 || H == 0) return -1;
    scene_t sc;
    int rc = scene_parse(recipe, scene, scene_len, address_width, &sc);
    if (rc != 0) return rc;
    if (threads < 1) threads = 1;
    job_t job;
    job.sc = &sc; job.hops = hops; job.W = W; job.H = H; job.passes = passes; job.flags = flags;
    job.pixels = pixels; job.n = n_pixels; job.canvas = canvas; job.seeds = seeds; job.next = 0;
    pthread_mutex_init(&job.lock, NULL);
    worker_t *ws = (worker_t *)calloc((size_t)threads, sizeof(worker_t));
    pthread_t *ts = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) ws[t].job = &job;
    for (int t = 1; t < threads; ++t) pthread_create(&ts[t], NULL, worker_main, &ws[t]);
    worker_main(&ws[0]);
    for (int t = 1; t < threads; ++t) pthread_join(ts[t], NULL);
    if (stats) {
        stats_t s = {0, 0, 0, 0};
        for (int t = 0; t < threads; ++t) {
            s.samples += ws[t].st.samples; s.hops += ws[t].st.hops;
            s.object_tests += ws[t].st.object_tests; s.hits += ws[t].st.hits;
        }
        stats[0] = s.samples; stats[1] = s.hops; stats[2] = s.object_tests; stats[3] = s.hits;
    }
    free(ws); free(ts);
    pthread_mutex_destroy(&job.lock);
    scene_free(&sc);
    return 0;
}

/* Post chain: extract (canvas.rs:126-135), gamma (filter/gamma.rs:10-19),
 * pack (canvas.rs:176-186; OpenCL convert_uchar4 rounds toward zero). */
void HTO(extract_gamma_pack)(uint32_t n_pixels, uint32_t passes, float gamma, const float *canvas,
                             float *image, uint8_t *packed) {
    for (uint32_t i = 0; i < 4u * n_pixels; ++i) {
        float v = canvas[i] / (float)passes;
        float m = v > 0.0f ? v : 0.0f;   /* max(x, 0) */
        float g = powf(m, gamma);
        if (image) image[i] = g;
        float c = g < 0.0f ? 0.0f : (g > 1.0f ? 1.0f : g);
        if (packed) packed[i] = (uint8_t)(255.0f * c);
    }
}

/* Pack alone (canvas.rs:176-186): u8 = convert_uchar4(0xFF * clamp(x, 0, 1)). OpenCL's
 * clamp is fmin(fmax(x, 0), 1), so NaN gives 0; the default conversion rounds toward zero. */
void HTO(pack)(uint32_t n_pixels, const float *image, uint8_t *packed) {
    for (uint32_t i = 0; i < 4u * n_pixels; ++i) {
        float c = fminf(fmaxf(image[i], 0.0f), 1.0f);
        packed[i] = (uint8_t)(255.0f * c);
    }
}

int HTO(real_size)(void) { return (int)sizeof(R); }

void HTO(rng_uniforms)(uint32_t seed, uint32_t n, double *out, uint32_t *state_out) {
    uint32_t s = seed;
    for (uint32_t i = 0; i < n; ++i) out[i] = (double)rng_uniform(&s);
    if (state_out) *state_out = s;
}

/* ======================================================================================
 * The scene types of the reference's hy and eu examples (recipes 3 and 4).
 *
 *   3: SceneImpl<Hyperbolic3, Mapped<PointView, Moebius>, Vec<Mapped<Choice{
 *        TiledPlane<M, Pentastar, 2>, TiledPlane<M, Pentagonal, 2>,
 *        TiledHorosphere<M, Hexagonal, 3>, TiledHorosphere<M, Square, 4>}, Moebius>>, ConstBg, H>
 *      M = Emissive<Mixture{Colored<Lambertian>, Specular, Transparent}>  (main/examples/hy.rs)
 *   4: SceneImpl<Euclidean3, Mapped<PointView, Homogenous3>, Vec<Mapped<Covered<
 *        Choice{Plane, Sphere, Cube}, Mixture{Colored<Lambertian>, Specular,
 *        Colored<Refractive>}>, Shift3>>, GradBg, H>                      (main/examples/eu.rs)
 *
 * Byte offsets (from the layout rules of type-macros/src/entity.rs, as written by
 * hypertrace_b200/types.py; identical for address width 32 and 64):
 *   3: view map @0, fov @32, background @64, count @96, objects @128 + 384 i;
 *      object: map @0, variant index @32, payload @48 = N materials of 64 bytes, border
 *      material, cell_size, border_width; material: emission @0, diffuse color @16,
 *      diffuse portion @32, specular portion @48, transparent portion @52.
 *   4: view Homogenous3 @0, fov @32, GradBg{direction @48, colors @64 @80, power @96},
 *      count @112, objects @128 + 128 i; object: shift @0, diffuse color @16, diffuse
 *      portion @32, specular portion @48, refractive color @64, index @80, portion @96,
 *      shape index @112.
 * ====================================================================================== */

typedef struct {
    col3 emission;
    col3 diffuse_color; R diffuse, specular, transparent;
} tl_material;

typedef struct {
    moebius map, inv;
    uint32_t variant;
    tl_material mats[4];
    tl_material border;
    R cell_size, border_width;
} tl_object;

typedef struct {
    col3 diffuse_color; R diffuse, specular;
    col3 refr_color; R refr_index, refr;
    vec3 shift, shift_inv;
    uint32_t shape;
} gr_object;

/* Linear3 (transform/linear.cc, algebra/matrix_real.cc): 16 reals, rows padded. */
typedef struct { R m[16]; } m33;
/* Recipe 5: one object (map Chain<Linear3, Shift3>) whose shape is a vector of mapped shapes
 * (maps Chain<Shift3, Linear3>); the material of recipe 4's objects. */
typedef struct { vec3 shift; m33 lin; vec3 shift_inv; m33 lin_inv; uint32_t shape; } cp_shape;

typedef struct {
    int recipe;
    uint32_t n;
    R fov;
    moebius cam_mo;
    hom3 cam_hom;
    col3 background;
    vec3 grad_dir; col3 grad_c0, grad_c1; float grad_power;
    tl_object *tl;
    gr_object *gr;
    /* recipe 5 */
    m33 obj_lin, obj_lin_inv;
    vec3 obj_shift, obj_shift_inv;
    gr_object cp_mat;
    cp_shape *cp;
} ext_scene_t;

static inline vec3 r33_mv(const m33 *a, vec3 b) {   /* r44_dot_mv(a, (b, 0)).xyz */
    const R *m = a->m;
    R x = 0; x += m[0] * b.x; x += m[1] * b.y; x += m[2] * b.z; x += m[3] * (R)0;
    R y = 0; y += m[4] * b.x; y += m[5] * b.y; y += m[6] * b.z; y += m[7] * (R)0;
    R z = 0; z += m[8] * b.x; z += m[9] * b.y; z += m[10] * b.z; z += m[11] * (R)0;
    return v3(x, y, z);
}
static inline m33 r33_tr(const m33 *a) {
    m33 t;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) t.m[4 * i + j] = a->m[4 * j + i];
    return t;
}
static inline m33 r33_inv(const m33 *a) {   /* matrix_real.cc:106-120 */
    const R *m = a->m;
    R det = m[0] * m[5] * m[10] + m[1] * m[6] * m[8] + m[2] * m[4] * m[9]
          - m[0] * m[6] * m[9] - m[1] * m[4] * m[10] - m[2] * m[5] * m[8];
    R adj[16] = {m[5] * m[10] - m[6] * m[9], m[2] * m[9] - m[1] * m[10], m[1] * m[6] - m[2] * m[5], 0,
                 m[6] * m[8] - m[4] * m[10], m[0] * m[10] - m[2] * m[8], m[2] * m[4] - m[0] * m[6], 0,
                 m[4] * m[9] - m[5] * m[8], m[1] * m[8] - m[0] * m[9], m[0] * m[5] - m[1] * m[4], 0,
                 0, 0, 0, 0};
    m33 r;
    for (int i = 0; i < 16; ++i) r.m[i] = adj[i] / det;
    r.m[15] = (R)1;
    return r;
}
static inline vec3 lin_normal(const m33 *l, vec3 d) {   /* lin3_apply_normal */
    m33 inv = r33_inv(l);
    m33 it = r33_tr(&inv);
    return normalize3(r33_mv(&it, d));
}
/* Chain<Linear3, Shift3> (outer linear after inner shift, chain.inl:36-73): ray map */
static inline ray_eu ray_ls(ray_eu r, const m33 *l, vec3 s) {
    ray_eu o;
    o.start = r33_mv(l, v3(r.start.x + s.x, r.start.y + s.y, r.start.z + s.z));
    o.dir = normalize3(normalize3(r33_mv(l, r.dir)));
    return o;
}
/* Chain<Shift3, Linear3> (outer shift after inner linear): ray map */
static inline ray_eu ray_sl(ray_eu r, vec3 s, const m33 *l) {
    ray_eu o;
    vec3 p = r33_mv(l, r.start);
    o.start = v3(p.x + s.x, p.y + s.y, p.z + s.z);
    o.dir = normalize3(normalize3(r33_mv(l, r.dir)));
    return o;
}
static m33 rd_lin(const uint8_t *b) {
    m33 m;
    for (int i = 0; i < 16; ++i) m.m[i] = rd_f(b, 4 * i);
    return m;
}

static col3 rd_col(const uint8_t *b, size_t off) { col3 c = {rd_f(b, off), rd_f(b, off + 4), rd_f(b, off + 8)}; return c; }

static tl_material rd_tl_material(const uint8_t *b) {
    tl_material m;
    m.emission = rd_col(b, 0);
    m.diffuse_color = rd_col(b, 16);
    m.diffuse = rd_f(b, 32);
    m.specular = rd_f(b, 48);
    m.transparent = rd_f(b, 52);
    return m;
}

static int ext_parse(int recipe, const uint8_t *b, size_t len, int aw, ext_scene_t *s) {
    memset(s, 0, sizeof(*s));
    if (aw != 32 && aw != 64) return -4;
    s->recipe = recipe;
    if (len < 128) return -1;
    s->fov = rd_f(b, 32);
    if (recipe == 3) {
        static const uint32_t counts[4] = {2, 2, 3, 4};
        s->cam_mo = rd_mo(b);
        s->background = rd_col(b, 64);
        s->n = rd_u(b, 96);
        if (aw == 64 && rd_u(b, 100) != 0) return -1;
        if ((len - 128) / 384 < s->n) return -1;
        s->tl = (tl_object *)calloc(s->n ? s->n : 1, sizeof(tl_object));
        for (uint32_t i = 0; i < s->n; ++i) {
            const uint8_t *o = b + 128 + (size_t)i * 384;
            tl_object *t = &s->tl[i];
            t->map = rd_mo(o);
            t->inv = mo_inverse(t->map);
            t->variant = rd_u(o, 32);
            if ((aw == 64 && rd_u(o, 36) != 0) || t->variant > 3) { free(s->tl); return -5; }
            const uint32_t nm = counts[t->variant];
            for (uint32_t k = 0; k < nm; ++k) t->mats[k] = rd_tl_material(o + 48 + 64 * k);
            t->border = rd_tl_material(o + 48 + 64 * nm);
            t->cell_size = rd_f(o, 48 + 64 * nm + 64);
            t->border_width = rd_f(o, 48 + 64 * nm + 68);
        }
        return 0;
    }
    s->cam_hom = rd_hom(b);
    s->grad_dir = v3(rd_f(b, 48), rd_f(b, 52), rd_f(b, 56));
    s->grad_c0 = rd_col(b, 64);
    s->grad_c1 = rd_col(b, 80);
    s->grad_power = rd_f(b, 96);
    if (recipe == 5) {
        /* object map Chain<Linear3, Shift3> @128 (linear @128, shift @192); material @256;
         * shape vector: count @384, elements @448 + 192 i (shift @0, linear @64, choice @128) */
        if (len < 448) return -1;
        s->obj_lin = rd_lin(b + 128);
        s->obj_shift = v3(rd_f(b, 192), rd_f(b, 196), rd_f(b, 200));
        /* chain inverse: outer^-1, inner^-1, then shf3_lin3_reorder (linear.cc) */
        s->obj_lin_inv = r33_inv(&s->obj_lin);
        {
            m33 back = r33_inv(&s->obj_lin_inv);
            s->obj_shift_inv = r33_mv(&back, v3(-s->obj_shift.x, -s->obj_shift.y, -s->obj_shift.z));
        }
        gr_object *g = &s->cp_mat;
        g->diffuse_color = rd_col(b, 256);
        g->diffuse = rd_f(b, 272);
        g->specular = rd_f(b, 288);
        g->refr_color = rd_col(b, 304);
        g->refr_index = rd_f(b, 320);
        g->refr = rd_f(b, 336);
        s->n = rd_u(b, 384);
        if (aw == 64 && rd_u(b, 388) != 0) return -1;
        if ((len - 448) / 192 < s->n) return -1;
        s->cp = (cp_shape *)calloc(s->n ? s->n : 1, sizeof(cp_shape));
        for (uint32_t i = 0; i < s->n; ++i) {
            const uint8_t *o = b + 448 + (size_t)i * 192;
            cp_shape *c = &s->cp[i];
            c->shift = v3(rd_f(o, 0), rd_f(o, 4), rd_f(o, 8));
            c->lin = rd_lin(o + 64);
            c->shape = rd_u(o, 128);
            if ((aw == 64 && rd_u(o, 132) != 0) || c->shape > 2) { free(s->cp); return -5; }
            /* Chain<Shift3, Linear3> inverse: -shift, lin^-1, then lin3_shf3_reorder */
            c->lin_inv = r33_inv(&c->lin);
            c->shift_inv = r33_mv(&c->lin_inv, v3(-c->shift.x, -c->shift.y, -c->shift.z));
        }
        return 0;
    }
    s->n = rd_u(b, 112);
    if (aw == 64 && rd_u(b, 116) != 0) return -1;
    if ((len - 128) / 128 < s->n) return -1;
    s->gr = (gr_object *)calloc(s->n ? s->n : 1, sizeof(gr_object));
    for (uint32_t i = 0; i < s->n; ++i) {
        const uint8_t *o = b + 128 + (size_t)i * 128;
        gr_object *g = &s->gr[i];
        g->shift = v3(rd_f(o, 0), rd_f(o, 4), rd_f(o, 8));
        g->shift_inv = v3(-g->shift.x, -g->shift.y, -g->shift.z);   /* shf3_inverse (shift.cc) */
        g->diffuse_color = rd_col(o, 16);
        g->diffuse = rd_f(o, 32);
        g->specular = rd_f(o, 48);
        g->refr_color = rd_col(o, 64);
        g->refr_index = rd_f(o, 80);
        g->refr = rd_f(o, 96);
        g->shape = rd_u(o, 112);
        if ((aw == 64 && rd_u(o, 116) != 0) || g->shape > 2) { free(s->gr); return -5; }
    }
    return 0;
}

/* ------------------------------------------------------------------ materials (shared) */
static inline void lambertian(uint32_t *rng, vec3 normal, vec3 *dir) {   /* lambertian.cc:6-14 */
    if (dot3(*dir, normal) > (R)0) normal = v3(-normal.x, -normal.y, -normal.z);
    vec3 rnd = hemisphere_cosine(rng);
    quat rot = rot3_look_at(v3(-normal.x, -normal.y, -normal.z));
    *dir = rot3_apply(rot, rnd);
}
static inline void specular(vec3 normal, vec3 *dir) {   /* specular.cc:4-7 */
    R k = (R)2 * dot3(*dir, normal);
    *dir = v3(dir->x - k * normal.x, dir->y - k * normal.y, dir->z - k * normal.z);
}
static inline R signr(R a) { return (R)(((R)0 < a) - (a < (R)0)); }   /* math.hh sign */
static inline void refractive(R index, vec3 normal, vec3 *dir) {   /* refractive.cc:4-22 */
    vec3 d = *dir;
    R k = index;
    R a = dot3(d, normal);
    if (a < -EPS) k = (R)1 / k;
    R x = (a * a - (R)1) * (k * k) + (R)1;
    if (x > EPS) {
        R b = signr(a) * RSQRT(x);
        R m = b - a * k;
        d = v3(d.x * k + m * normal.x, d.y * k + m * normal.y, d.z * k + m * normal.z);
    } else {
        R m = (R)2 * a;
        d = v3(d.x - m * normal.x, d.y - m * normal.y, d.z - m * normal.z);
    }
    *dir = d;
}

/* Emissive<Mixture{Colored<Lambertian>, Specular, Transparent}> (emissive.inl:15-23,
 * mixture/impl.inl:16-27, colored.inl:15-23, transparent.cc:4-6). */
static int tl_material_interact(const tl_material *m, uint32_t *rng, vec3 normal, vec3 *dir, col3 *k, col3 *e) {
    e->x += k->x * m->emission.x;
    e->y += k->y * m->emission.y;
    e->z += k->z * m->emission.z;
    R alpha = rng_uniform(rng);
    alpha -= m->diffuse;
    if (alpha < (R)0) {
        k->x *= m->diffuse_color.x; k->y *= m->diffuse_color.y; k->z *= m->diffuse_color.z;
        lambertian(rng, normal, dir);
        return 1;
    }
    alpha -= m->specular;
    if (alpha < (R)0) { specular(normal, dir); return 1; }
    alpha -= m->transparent;
    if (alpha < (R)0) return 1;
    return 0;
}

/* ------------------------------------------------------------------ hyperbolic maps
 * geometry/hyperbolic.cc:40-54 (hy_xshift, hy_zrotate), matrix_complex.cc:38-45 (c22_dot) */
static inline comp cmake(R x, R y) { comp c = {x, y}; return c; }
static inline comp c_mul(comp a, comp b) { return cmake(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
static inline comp c_add(comp a, comp b) { return cmake(a.x + b.x, a.y + b.y); }
static inline moebius mo_chain(moebius a, moebius b) {
    moebius r;
    r.a = c_add(c_mul(a.a, b.a), c_mul(a.b, b.c));
    r.b = c_add(c_mul(a.a, b.b), c_mul(a.b, b.d));
    r.c = c_add(c_mul(a.c, b.a), c_mul(a.d, b.c));
    r.d = c_add(c_mul(a.c, b.b), c_mul(a.d, b.d));
    return r;
}
#ifdef HT_REAL_DOUBLE
#define RCOSH(x) cosh(x)
#define RSINH(x) sinh(x)
#define RFLOOR(x) floor(x)
#else
#define RCOSH(x) coshf(x)
#define RSINH(x) sinhf(x)
#define RFLOOR(x) floorf(x)
#endif
static inline moebius hy_xshift(R l) {
    R l2 = l / (R)2;
    R c = RCOSH(l2), s = RSINH(l2);
    moebius m;
    m.a = cmake(c * (R)1, c * (R)0); m.b = cmake(s * (R)1, s * (R)0);
    m.c = cmake(s * (R)1, s * (R)0); m.d = cmake(c * (R)1, c * (R)0);
    return m;
}
static inline moebius hy_zrotate(R phi) {
    R c = RCOS(phi / (R)2), s = RSIN(phi / (R)2);
    moebius m;
    m.a = cmake(c, s); m.b = cmake((R)0, (R)0); m.c = cmake((R)0, (R)0); m.d = cmake(c, -s);
    return m;
}

/* TiledPlane material choice (object/hy/tiled_plane/impl.inl:48-137): 0 / 1 the cell's
 * material, 2 the border. */
static int tiled_plane_cell(const tl_object *t, quat p, int star) {
    int w = 0;
    R Q = RSQRT(RCOS(PI_R / 4 + PI_R / 5) / RCOS(PI_R / 4 - PI_R / 5));
    R T = RSQRT(RCOS(PI_R / 4 + PI_R / 5) * RCOS(PI_R / 4 - PI_R / 5));
    R S = (RCOS(PI_R / 4) - RSIN(PI_R / 5)) / T;
    R L = T / RCOS(PI_R / 4);
    R K = L * (2 * RCOS(PI_R / 5) - 1 / RCOS(PI_R / 5));
    Q = RLOG((1 + Q) / (1 - Q));
    S = RLOG((1 + S) / (1 - S));
    if (p.x < (R)0) { p.x = -p.x; w = !w; }
    if (p.y < (R)0) { p.y = -p.y; w = !w; }
    p = mo_apply_q(mo_chain(hy_xshift(-Q), hy_zrotate(-PI_R / 4)), p);
    int e = 0;
    for (int j = 0; j < 5; ++j) {
        int a[3] = {0, 0, 0};
        for (int i = 0; i < 3 - e; ++i) {
            R o = 2 * PI_R * (i - 1) / 5;
            a[i] = dot2(RCOS(o), RSIN(o), p.x, p.y) < L;
        }
        a[2] = a[2] || e;
        int s = a[0] + a[1] + a[2];
        if (s == 3) {
            break;
        } else if (s == 2) {
            int i = (!a[1]) + 2 * (!a[2]);
            R o = 2 * PI_R * (i - 1) / 5;
            p = mo_apply_q(mo_chain(hy_zrotate(-PI_R / 5), mo_chain(hy_xshift(-2 * S), hy_zrotate(-o))), p);
            e = 1;
            w = !w;
        } else {
            int i = a[0];
            R o = PI_R * (2 * i - 1) / 5;
            p = mo_apply_q(mo_chain(hy_xshift(-2 * Q), hy_zrotate(-o)), p);
            e = 0;
        }
    }
    const R br = t->border_width;
    int bh = 0;
    for (int i = 0; i < 5; ++i) {
        R o = 2 * PI_R * i / 5;
        R dp = dot2(RCOS(o), RSIN(o), p.x, p.y);
        bh = bh || (dp > (L - br * p.z));
        if (star) {
            R ps = K + dp;
            w = w ^ (ps < (R)0);
            bh = bh || (RFABS(ps) < br * p.z);
        }
    }
    if (bh) return 2;
    return w ? 0 : 1;
}

#define REM(a, b) ((((a) % (b)) + (b)) % (b))   /* math.hh rem */

/* TiledHorosphere material choice (object/hy/tiled_horosphere/impl.inl:44-95). */
static const tl_material *tiled_horosphere_material(const tl_object *t, quat p, int hexagonal, int n) {
    int material_no = 0;
    int border = 0;
    R br = t->border_width / t->cell_size;
    R gx = p.x, gy = p.y;
    if (!hexagonal) {
        R vx = gx / t->cell_size, vy = gy / t->cell_size;
        R kx = RFLOOR(vx), ky = RFLOOR(vy);
        R fx = vx - kx, fy = vy - ky;
        if (fx < br || fx > 1 - br || fy < br || fy > 1 - br) {
            border = 1;
        } else {
            int hx = REM((int)kx, 2);
            int hy = REM((int)ky, 2);
            material_no = 3 * hy - 2 * hx * hy + hx;
        }
    } else {
        R r3 = RSQRT((R)3);
        R bxx = 2 / r3, bxy = 0;
        R byx = -1 / r3, byy = 1;
        R s = t->cell_size * r3 / 2;
        R hxf = dot2(bxx, bxy, gx, gy) / s;
        R hyf = dot2(byx, byy, gx, gy) / s;
        int hx = (int)RFLOOR((RFLOOR(hxf) - RFLOOR(hyf)) / 3);
        int hy = (int)RFLOOR((RFLOOR(hxf + hyf) - hx) / 2);
        R ox = (R)hx * 2 + (R)hy * 1;
        R oy = (R)hx * -1 + (R)hy * 1;
        hxf -= ox;
        hyf -= oy;
        if (RFABS(hxf - 1) > 1 - br || RFABS(hyf) > 1 - br || RFABS(hxf + hyf - 1) > 1 - br) {
            border = 1;
        } else {
            material_no = 2 * hx + hy;
        }
    }
    if (border) return &t->border;
    return &t->mats[REM(material_no, n)];
}

static col3 sample_tl(const ext_scene_t *sc, uint32_t hops, uint32_t *rng, R px, R py, R size, uint32_t flags,
                      stats_t *st) {
    R u0 = rng_uniform(rng);
    R u1 = rng_uniform(rng);
    R jx = (flags & HTO_JITTER_YX) ? u1 : u0;
    R jy = (flags & HTO_JITTER_YX) ? u0 : u1;
    R sx = px + size * (jx - (R)0.5f);
    R sy = py + size * (jy - (R)0.5f);
    vec3 ld = normalize3(v3(sx, sy, (R)-1 / sc->fov));
    quat start = q4((R)0, (R)0, (R)1, (R)0);
    ray_hy ray;
    ray.dir = normalize4(mo_deriv_q(sc->cam_mo, start, q4(ld.x, ld.y, ld.z, (R)0)));
    ray.start = mo_apply_q(sc->cam_mo, start);
    col3 intensity = {1.0f, 1.0f, 1.0f};
    col3 emission = {0.0f, 0.0f, 0.0f};
    uint32_t prev_hash = 0xFFFFFFFFu;
    st->samples += 1;
    for (uint32_t i = 0; i < hops; ++i) {
        st->hops += 1;
        st->object_tests += sc->n;
        R min_dist = (R)-1;
        uint32_t min_index = 0;
        ray_hy min_local = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        quat min_normal = {0, 0, 0, 0};
        for (uint32_t k = 0; k < sc->n; ++k) {
            int repeat = (k == prev_hash);
            ray_hy local = ray_hy_map(ray, sc->tl[k].inv);
            quat normal;
            R dist = sc->tl[k].variant < 2 ? plane_hy_detect(repeat, &normal, &local)
                                           : horosphere_detect(repeat, &normal, &local);
            if (dist > -EPS && (min_dist <= -EPS || dist < min_dist)) {
                min_dist = dist; min_index = k; min_local = local; min_normal = normal;
            }
        }
        if (min_dist > -EPS) {
            st->hits += 1;
            const tl_object *t = &sc->tl[min_index];
            ray_hy hit = ray_hy_map(min_local, t->map);
            ray_hy loc = ray_hy_map(hit, t->inv);
            const tl_material *m;
            if (t->variant < 2) {
                int c = tiled_plane_cell(t, loc.start, t->variant == 0);
                m = c == 2 ? &t->border : &t->mats[c];
            } else {
                m = tiled_horosphere_material(t, loc.start, t->variant == 2, t->variant == 2 ? 3 : 4);
            }
            vec3 d3 = v3(loc.dir.x, loc.dir.y, loc.dir.z);
            vec3 n3 = v3(min_normal.x, min_normal.y, min_normal.z);
            int ret = tl_material_interact(m, rng, n3, &d3, &intensity, &emission);
            loc.dir = q4(d3.x, d3.y, d3.z, (R)0);
            ray = ray_hy_map(loc, t->map);
            if (!ret) break;
            prev_hash = min_index;
        } else {
            emission.x += sc->background.x * intensity.x;
            emission.y += sc->background.y * intensity.y;
            emission.z += sc->background.z * intensity.z;
            break;
        }
    }
    return emission;
}

/* ------------------------------------------------------------------ euclidean extras */
/* cube_eu_detect (shape/eu/cube.cc:3-65); the reference keeps dist_in / dist_out in float. */
static inline R cube_nearest(vec3 near, vec3 *n) {
    int xy = near.x > near.y, yz = near.y > near.z, xz = near.x > near.z;
    if (xy && xz) { n->x = (R)1; return near.x; }
    if (yz) { n->y = (R)1; return near.y; }
    n->z = (R)1;
    return near.z;
}
#ifdef HT_REAL_DOUBLE
#define RFMIN(a, b) fmin(a, b)
#define RFMAX(a, b) fmax(a, b)
#else
#define RFMIN(a, b) fminf(a, b)
#define RFMAX(a, b) fmaxf(a, b)
#endif
static inline R cube_eu_detect(int repeat, vec3 *normal, ray_eu *ray) {
    vec3 s = ray->start, d = ray->dir;
    vec3 inv = v3((R)1 / d.x, (R)1 / d.y, (R)1 / d.z);
    vec3 vmin = v3(((R)-1 - s.x) * inv.x, ((R)-1 - s.y) * inv.y, ((R)-1 - s.z) * inv.z);
    vec3 vmax = v3(((R)1 - s.x) * inv.x, ((R)1 - s.y) * inv.y, ((R)1 - s.z) * inv.z);
    vec3 near = v3(RFMIN(vmin.x, vmax.x), RFMIN(vmin.y, vmax.y), RFMIN(vmin.z, vmax.z));
    vec3 far = v3(RFMAX(vmin.x, vmax.x), RFMAX(vmin.y, vmax.y), RFMAX(vmin.z, vmax.z));
    vec3 sg = v3(signr(d.x), signr(d.y), signr(d.z));
    vec3 nin = v3(0, 0, 0);
    float din = (float)cube_nearest(near, &nin);
    nin = v3(nin.x * -sg.x, nin.y * -sg.y, nin.z * -sg.z);
    vec3 nout = v3(0, 0, 0);
    float dout = -(float)cube_nearest(v3(-far.x, -far.y, -far.z), &nout);
    nout = v3(nout.x * sg.x, nout.y * sg.y, nout.z * sg.z);
    if (din > dout) return (R)-1;
    R dist = din;
    vec3 n = nin;
    R w = 2 * EPS * (R)(2 * repeat - 1);
    if (dist < w) {
        dist = dout;
        n = nout;
        if (dist < w) return (R)-1;
    }
    ray->start = v3(s.x + dist * d.x, s.y + dist * d.y, s.z + dist * d.z);
    *normal = n;
    return dist;
}

/* ray_eu_map with Shift3 (ray_map.inl:15-21, shift.cc:44-59): start + v, normalize(dir). */
static inline ray_eu ray_shift(ray_eu r, vec3 v) {
    ray_eu o;
    o.start = v3(r.start.x + v.x, r.start.y + v.y, r.start.z + v.z);
    o.dir = normalize3(r.dir);
    return o;
}

/* Mixture{Colored<Lambertian>, Specular, Colored<Refractive>} */
static int gr_material_interact(const gr_object *g, uint32_t *rng, vec3 normal, vec3 *dir, col3 *k) {
    R alpha = rng_uniform(rng);
    alpha -= g->diffuse;
    if (alpha < (R)0) {
        k->x *= g->diffuse_color.x; k->y *= g->diffuse_color.y; k->z *= g->diffuse_color.z;
        lambertian(rng, normal, dir);
        return 1;
    }
    alpha -= g->specular;
    if (alpha < (R)0) { specular(normal, dir); return 1; }
    alpha -= g->refr;
    if (alpha < (R)0) {
        k->x *= g->refr_color.x; k->y *= g->refr_color.y; k->z *= g->refr_color.z;
        refractive(g->refr_index, normal, dir);
        return 1;
    }
    return 0;
}

static col3 sample_gr(const ext_scene_t *sc, uint32_t hops, uint32_t *rng, R px, R py, R size, uint32_t flags,
                      stats_t *st) {
    R u0 = rng_uniform(rng);
    R u1 = rng_uniform(rng);
    R jx = (flags & HTO_JITTER_YX) ? u1 : u0;
    R jy = (flags & HTO_JITTER_YX) ? u0 : u1;
    R sx = px + size * (jx - (R)0.5f);
    R sy = py + size * (jy - (R)0.5f);
    vec3 ld = normalize3(v3(sx, sy, (R)-1 / sc->fov));
    ray_eu ray;
    ray.dir = hom3_apply_dir(sc->cam_hom, ld);
    ray.start = hom3_apply_pos(sc->cam_hom, v3((R)0, (R)0, (R)0));
    col3 intensity = {1.0f, 1.0f, 1.0f};
    col3 emission = {0.0f, 0.0f, 0.0f};
    uint32_t prev_hash = 0xFFFFFFFFu;
    st->samples += 1;
    for (uint32_t i = 0; i < hops; ++i) {
        st->hops += 1;
        st->object_tests += sc->n;
        R min_dist = (R)-1;
        uint32_t min_index = 0;
        ray_eu min_local = {{0, 0, 0}, {0, 0, 0}};
        vec3 min_normal = {0, 0, 0};
        for (uint32_t k = 0; k < sc->n; ++k) {
            int repeat = (k == prev_hash);
            ray_eu local = ray_shift(ray, sc->gr[k].shift_inv);
            vec3 normal;
            uint32_t sh = sc->gr[k].shape;
            R dist = sh == 0 ? plane_eu_detect(repeat, &normal, &local)
                   : sh == 1 ? sphere_eu_detect(repeat, &normal, &local)
                             : cube_eu_detect(repeat, &normal, &local);
            if (dist > -EPS && (min_dist <= -EPS || dist < min_dist)) {
                min_dist = dist; min_index = k; min_local = local; min_normal = normal;
            }
        }
        if (min_dist > -EPS) {
            st->hits += 1;
            const gr_object *g = &sc->gr[min_index];
            ray_eu hit = ray_shift(min_local, g->shift);
            ray_eu loc = ray_shift(hit, g->shift_inv);
            int ret = gr_material_interact(g, rng, min_normal, &loc.dir, &intensity);
            ray = ray_shift(loc, g->shift);
            if (!ret) break;
            prev_hash = min_index;
        } else {
            /* GradBg (background/gradient.cc:3-13): all in float */
            float f = 0.5f * ((float)dot3(ray.dir, sc->grad_dir) + 1.0f);
            f = f < 0.0f ? 0.0f : f;
            f = 1.0f < f ? 1.0f : f;
            f = powf(f, sc->grad_power);
            float g = 1.0f - f;
            emission.x += (f * sc->grad_c0.x + g * sc->grad_c1.x) * intensity.x;
            emission.y += (f * sc->grad_c0.y + g * sc->grad_c1.y) * intensity.y;
            emission.z += (f * sc->grad_c0.z + g * sc->grad_c1.z) * intensity.z;
            break;
        }
    }
    return emission;
}

/* Recipe 5 hop loop: the object (object/mapped.inl) -> covered (object/covered.inl) ->
 * shape vector (shape/vector.inl: nearest hit, ties to the lowest index, hash = index) ->
 * mapped shapes (shape/mapped.inl: local hit, normal through apply_normal, ray mapped back). */
static col3 sample_cp(const ext_scene_t *sc, uint32_t hops, uint32_t *rng, R px, R py, R size, uint32_t flags,
                      stats_t *st) {
    R u0 = rng_uniform(rng);
    R u1 = rng_uniform(rng);
    R jx = (flags & HTO_JITTER_YX) ? u1 : u0;
    R jy = (flags & HTO_JITTER_YX) ? u0 : u1;
    R sx = px + size * (jx - (R)0.5f);
    R sy = py + size * (jy - (R)0.5f);
    vec3 ld = normalize3(v3(sx, sy, (R)-1 / sc->fov));
    ray_eu ray;
    ray.dir = hom3_apply_dir(sc->cam_hom, ld);
    ray.start = hom3_apply_pos(sc->cam_hom, v3((R)0, (R)0, (R)0));
    col3 intensity = {1.0f, 1.0f, 1.0f};
    col3 emission = {0.0f, 0.0f, 0.0f};
    uint32_t prev_hash = 0xFFFFFFFFu;
    st->samples += 1;
    for (uint32_t i = 0; i < hops; ++i) {
        st->hops += 1;
        st->object_tests += 1;
        ray_eu local = ray_ls(ray, &sc->obj_lin_inv, sc->obj_shift_inv);
        R min_dist = (R)-1;
        uint32_t min_index = 0;
        ray_eu min_hit = {{0, 0, 0}, {0, 0, 0}};
        vec3 min_normal = {0, 0, 0};
        for (uint32_t k = 0; k < sc->n; ++k) {
            int repeat = (k == prev_hash);
            const cp_shape *c = &sc->cp[k];
            ray_eu sl = ray_sl(local, c->shift_inv, &c->lin_inv);
            vec3 n;
            R dist = c->shape == 0 ? plane_eu_detect(repeat, &n, &sl)
                   : c->shape == 1 ? sphere_eu_detect(repeat, &n, &sl)
                                   : cube_eu_detect(repeat, &n, &sl);
            if (dist > -EPS && (min_dist <= -EPS || dist < min_dist)) {
                min_dist = dist; min_index = k; min_hit = sl; min_normal = n;
            }
        }
        if (min_dist > -EPS) {
            st->hits += 1;
            const cp_shape *c = &sc->cp[min_index];
            vec3 normal = lin_normal(&c->lin, min_normal);            /* shf3 normal = identity */
            ray_eu hit_obj = ray_sl(min_hit, c->shift, &c->lin);       /* shape map back */
            ray_eu world = ray_ls(hit_obj, &sc->obj_lin, sc->obj_shift);   /* object map back */
            ray_eu loc = ray_ls(world, &sc->obj_lin_inv, sc->obj_shift_inv);
            int ret = gr_material_interact(&sc->cp_mat, rng, normal, &loc.dir, &intensity);
            ray = ray_ls(loc, &sc->obj_lin, sc->obj_shift);
            if (!ret) break;
            prev_hash = min_index;
        } else {
            /* object/mapped.inl:33-35 maps the ray back even when nothing was hit: the
             * background sees the round-tripped direction */
            ray = ray_ls(local, &sc->obj_lin, sc->obj_shift);
            float f = 0.5f * ((float)dot3(ray.dir, sc->grad_dir) + 1.0f);
            f = f < 0.0f ? 0.0f : f;
            f = 1.0f < f ? 1.0f : f;
            f = powf(f, sc->grad_power);
            float g = 1.0f - f;
            emission.x += (f * sc->grad_c0.x + g * sc->grad_c1.x) * intensity.x;
            emission.y += (f * sc->grad_c0.y + g * sc->grad_c1.y) * intensity.y;
            emission.z += (f * sc->grad_c0.z + g * sc->grad_c1.z) * intensity.z;
            break;
        }
    }
    return emission;
}

typedef struct {
    const ext_scene_t *sc;
    uint32_t hops, W, H, passes, flags;
    const uint32_t *pixels;
    size_t n;
    float *canvas;
    uint32_t *seeds;
    size_t next;
    pthread_mutex_t lock;
} ext_job_t;

typedef struct { ext_job_t *job; stats_t st; } ext_worker_t;

static void *ext_worker_main(void *arg) {
    ext_worker_t *w = (ext_worker_t *)arg;
    ext_job_t *j = w->job;
    for (;;) {
        pthread_mutex_lock(&j->lock);
        size_t start = j->next;
        j->next += 64;
        pthread_mutex_unlock(&j->lock);
        if (start >= j->n) break;
        size_t end = start + 64 < j->n ? start + 64 : j->n;
        for (size_t i = start; i < end; ++i) {
            const uint32_t px = j->pixels[i];
            const uint32_t x = px % j->W, y = px / j->W;
            const R pxr = ((R)(2u * x + 1u) - (R)j->W) / (R)j->H;
            const R pyr = ((R)j->H - (R)(2u * y + 1u)) / (R)j->H;
            const R size = (R)2 / (R)j->H;
            for (uint32_t p = 0; p < j->passes; ++p) {
                uint32_t rng = j->seeds[i];
                col3 c = j->sc->recipe == 3 ? sample_tl(j->sc, j->hops, &rng, pxr, pyr, size, j->flags, &w->st)
                       : j->sc->recipe == 4 ? sample_gr(j->sc, j->hops, &rng, pxr, pyr, size, j->flags, &w->st)
                                            : sample_cp(j->sc, j->hops, &rng, pxr, pyr, size, j->flags, &w->st);
                float *cv = j->canvas + 4 * i;
                cv[0] += c.x; cv[1] += c.y; cv[2] += c.z; cv[3] += 1.0f;
                j->seeds[i] = rng;
            }
        }
    }
    return NULL;
}

static int render_ext(int recipe, uint32_t hops, const uint8_t *scene, size_t scene_len, int address_width,
                      uint32_t W, uint32_t H, const uint32_t *pixels, size_t n_pixels, uint32_t passes,
                      float *canvas, uint32_t *seeds, uint32_t flags, int threads, uint64_t *stats) {
    if (hops == 0) return -3;
    if (W == 0 || H == 0) return -1;
    ext_scene_t sc;
    int rc = ext_parse(recipe, scene, scene_len, address_width, &sc);
    if (rc != 0) return rc;
    if (threads < 1) threads = 1;
    ext_job_t job;
    job.sc = &sc; job.hops = hops; job.W = W; job.H = H; job.passes = passes; job.flags = flags;
    job.pixels = pixels; job.n = n_pixels; job.canvas = canvas; job.seeds = seeds; job.next = 0;
    pthread_mutex_init(&job.lock, NULL);
    ext_worker_t *ws = (ext_worker_t *)calloc((size_t)threads, sizeof(ext_worker_t));
    pthread_t *ts = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) ws[t].job = &job;
    for (int t = 1; t < threads; ++t) pthread_create(&ts[t], NULL, ext_worker_main, &ws[t]);
    ext_worker_main(&ws[0]);
    for (int t = 1; t < threads; ++t) pthread_join(ts[t], NULL);
    if (stats) {
        stats_t s = {0, 0, 0, 0};
        for (int t = 0; t < threads; ++t) {
            s.samples += ws[t].st.samples; s.hops += ws[t].st.hops;
            s.object_tests += ws[t].st.object_tests; s.hits += ws[t].st.hits;
        }
        stats[0] = s.samples; stats[1] = s.hops; stats[2] = s.object_tests; stats[3] = s.hits;
    }
    free(ws); free(ts);
    pthread_mutex_destroy(&job.lock);
    free(sc.tl); free(sc.gr); free(sc.cp);
    return 0;
}
