/* cull_check.c -- test infrastructure: a CPU restatement of the distance-bound culling of the
 * hyperbolic object scan (hypertrace_b200/csrc/ht_trace.cuh: stage_bound, bound_ray,
 * point_cut / survivors2 / culled_slot, culled_fw, sure_crossing_e2, upper_estimate,
 * cull_from_dist and the chunked scan of hop_hy over the staged slots: planes first, then
 * horospheres, each in scene order, hits compared on (distance, scene index)), run against
 * the full scan on every hop of sampled paths.
 *
 * The culling may only skip objects that cannot win, so on every hop the culled scan must pick
 * the object the full scan picks (the nearest reported hit, ties to the lowest index) at the
 * same distance. Shape tests and ray maps come from the oracle's restatement of the
 * reference (oracle/htoracle.c), the float arithmetic of the bounds follows the kernel
 * operation by operation (build with -ffp-contract=off), and where the kernel uses the PTX
 * approximations (rcp / sqrt / lg2 / ex2 .approx) this program can push each result 2^-21
 * relative the way that culls more (adversarial mode), beyond their documented error.
 *
 * usage: cull_check <scene bytes> <width> <height> <hops> <pixels> <global seed> <adversarial 0|1>
 * prints: hops <n> exact_per_hop <x> wrong <k>
 */
#include "../../oracle/htoracle.c"
#include <stdio.h>

static int ADV = 0;
#define ADV_EPS 4.76837158203125e-7f   /* 2^-21 */
/* x pushed by 2^-21 relative in direction dir (+1 up, -1 down) in adversarial mode */
static float adv(float x, int dir) { return ADV ? x * (1.0f + (float)dir * ADV_EPS) : x; }

#define CULL_REL 1e-2f
#define CULL_ABS 1e-2f
#define BOUND_EPS 1e-5f
#define HORO_M 1e-3f
#define EST_OBJECTS 24u
#define LN2F 0.693147180559945f
#define LOG2EF 1.442695040888963f

typedef struct { float x, y, z, w; } f4;
typedef struct { float S, E, T; } cull_t;
typedef struct { float x, y, t, r2, pv, vx, vy, vz, ax, ay, K, Kw; } bray_t;
typedef struct { float F, eF, W, eW; } fw_t;

static f4 stage_bound(moebius m, uint32_t shape) {
    double ar = m.a.x, ai = m.a.y, br = m.b.x, bi = m.b.y, cr = m.c.x, ci = m.c.y, dr = m.d.x, di = m.d.y;
    double det_r = (ar * dr - ai * di) - (br * cr - bi * ci);
    double det_i = (ar * di + ai * dr) - (br * ci + bi * cr);
    double adet = sqrt(det_r * det_r + det_i * det_i);
    double maxe = fmax(fmax(fabs(ar) + fabs(ai), fabs(br) + fabs(bi)), fmax(fabs(cr) + fabs(ci), fabs(dr) + fabs(di)));
    f4 nanr = {NAN, NAN, NAN, NAN};
    if (!(maxe <= 32.0 && adet >= 0.5 && adet <= 2.0)) return nanr;
    double n11r = dr, n11i = di, n12r = -br, n12i = -bi, n21r = -cr, n21i = -ci, n22r = ar, n22i = ai;
    if (shape == 0) {
        double A = (n11r * n11r + n11i * n11i) - (n21r * n21r + n21i * n21i);
        double Br = (n11r * n12r + n11i * n12i) - (n21r * n22r + n21i * n22i);
        double Bi = (n11r * n12i - n11i * n12r) - (n21r * n22i - n21i * n22r);
        double C = (n12r * n12r + n12i * n12i) - (n22r * n22r + n22i * n22i);
        f4 r = {(float)(A / adet), (float)(2.0 * Br / adet), (float)(2.0 * Bi / adet), (float)(C / adet)};
        return r;
    }
    double k2 = 1.0 / adet;
    double c2 = (n21r * n21r + n21i * n21i) * k2;
    double wr = (n22r * n21r + n22i * n21i) * k2;
    double wi = (n22r * n21i - n22i * n21r) * k2;
    double n22sq = (n22r * n22r + n22i * n22i) * k2;
    f4 r = {(float)c2, (float)(2.0 * wr), (float)(-2.0 * wi), (float)n22sq};
    return r;
}
static float bound_mag(f4 rec) {
    return BOUND_EPS * fmaxf(fmaxf(fabsf(rec.x), fabsf(rec.y)), fmaxf(fabsf(rec.z), fabsf(rec.w)));
}
static int cull_point_ok(quat p) {
    return p.z >= 0x1p-20f && p.z <= 0x1p20f && fabsf(p.x) + fabsf(p.y) <= 0x1p10f * p.z &&
           fabsf(p.w) <= 1e-3f * p.z;
}
static bray_t bound_ray(quat p, quat v) {
    bray_t b;
    b.x = p.x; b.y = p.y; b.t = p.z;
    b.r2 = fmaf(p.x, p.x, fmaf(p.y, p.y, p.z * p.z));
    b.pv = fmaf(p.x, v.x, fmaf(p.y, v.y, p.z * v.z));
    b.vx = v.x; b.vy = v.y; b.vz = v.z;
    b.ax = fabsf(p.x); b.ay = fabsf(p.y);
    b.K = b.r2 + b.ax + b.ay + 1.0f;
    b.Kw = b.t * (2.0f * fabsf(b.pv) + fabsf(b.vx) + fabsf(b.vy));
    return b;
}
/* upper bounds of sinh, exp, tanh of the threshold; adversarial mode lowers each */
static cull_t cull_from_dist(float d) {
    float thr = fmaf(d, 1.0f + CULL_REL, CULL_ABS);
    cull_t c;
    c.E = adv((float)exp2((double)(thr * LOG2EF)), -1) * (1.0f + 1e-5f);
    c.S = 0.5f * (c.E - adv(1.0f / c.E, +1));
    c.T = 1.0f - 2.0f * adv(1.0f / fmaf(c.E, c.E, 1.0f), +1);
    return c;
}
static cull_t cull_none(void) { cull_t c = {INFINITY, INFINITY, 1.0f}; return c; }
/* point bound of one slot: culled when F + eF < lo or F - eF > hi (point_cut / survivors2) */
static int culled_point(f4 rec, float mag, uint32_t shape, const bray_t *r, cull_t c) {
    float t = r->t;
    float F = fmaf(rec.x, r->r2, fmaf(rec.y, r->x, fmaf(rec.z, r->y, rec.w)));
    float eF = mag * r->K;
    float lo, hi;
    if (shape == 0) { hi = 2.0f * t * c.S; lo = -hi; }
    else { lo = t * adv(1.0f / c.E, +1); hi = t * c.E; }
    return (F + eF < lo) || (F + (mag * -r->K) > hi);
}
static fw_t bound_fw(f4 rec, float mag, const bray_t *r) {
    fw_t b;
    b.F = fmaf(rec.x, r->r2, fmaf(rec.y, r->x, fmaf(rec.z, r->y, rec.w)));
    b.eF = mag * r->K;
    float G = fmaf(2.0f * rec.x, r->pv, fmaf(rec.y, r->vx, rec.z * r->vy));
    b.W = fmaf(r->t, G, -b.F * r->vz);
    b.eW = fmaf(mag, r->Kw, fmaf(b.eF, fabsf(r->vz), BOUND_EPS * fabsf(b.W)));
    return b;
}
static int culled_fw(fw_t b, uint32_t shape, float t, cull_t c) {
    float F = b.F, eF = b.eF, W = b.W, eW = b.eW;
    if (shape == 0) {
        float Fa = fabsf(F) - eF, Wlo = fabsf(W) - eW, Whi = fabsf(W) + eW;
        int away = (F > 0.0f) == (W > 0.0f) && Fa > 0.02f * t && Wlo > 0.002f * t;
        int far = Fa > fmaf(1.01f * c.T, Whi, 0.02f * t);
        int point = Fa > 2.0f * t * c.S;
        return away || far || point;
    }
    float Flo = F - eF, Fhi = F + eF, Wlo = W - eW, Whi = W + eW;
    float aWlo = fmaxf(fabsf(W) - eW, 0.0f), aWhi = fabsf(W) + eW;
    if (t > c.E * Fhi || t * c.E < Flo) return 1;
    if (!(Flo > 0.0f)) return 0;
    float R2lo = t * t - Fhi * Fhi + aWlo * aWlo, R2hi = t * t - Flo * Flo + aWhi * aWhi;
    if (R2hi < -HORO_M * t * t) return 1;
    if (R2lo < HORO_M * t * t) return 0;
    float Rlo = adv(sqrtf(R2lo), +1) * (1.0f - 1e-6f), Rhi = adv(sqrtf(R2hi), -1) * (1.0f + 1e-6f);
    float tol = 2e-6f * Fhi * Fhi + 1e-5f * (aWhi * t + Rhi * Fhi);
    int r1 = !(Wlo * t + Rlo * Flo > tol);
    int r2 = !(Wlo * t - Rhi * Fhi > tol);
    float E1 = c.E * (1.0f + HORO_M);
    int r1_far = (Flo - Whi) > E1 * (t + Rhi) || (Fhi - Wlo) * E1 < (t + Rlo);
    int r2_far = (Flo + Wlo) > 0.0f && ((t + Rlo) > E1 * (Fhi + Whi) || (t + Rhi) * E1 < (Flo + Wlo));
    return (!r1 || r1_far) && (!r2 || r2_far);
}
/* upper bound of e^(2 s) of a sure crossing; adversarial mode lowers every approximated value */
static float sure_crossing_e2(fw_t b, uint32_t shape, int plane_repeat, float t) {
    float F = b.F, eF = b.eF, W = b.W, eW = b.eW;
    if (shape == 0) {
        if (plane_repeat) return INFINITY;
        float Fa = fabsf(F) - eF, Wlo = fabsf(W) - eW;
        if (!((F > 0.0f) != (W > 0.0f) && Fa > 0.02f * t && Wlo > 0.0f)) return INFINITY;
        float rr = (fabsf(F) + eF) * adv(1.0f / Wlo, -1);
        if (!(rr < 0.99f)) return INFINITY;
        return (1.0f + rr) * adv(1.0f / (1.0f - rr), -1);
    }
    float Flo = F - eF, Fhi = F + eF, Wlo = W - eW, Whi = W + eW;
    float e = INFINITY;
    if (Fhi < 0.999f * t && Flo > 0.0f && (Flo + Wlo) > 0.0f) {
        float aWlo = fmaxf(fabsf(W) - eW, 0.0f), aWhi = fabsf(W) + eW;
        float R2lo = t * t - Fhi * Fhi + aWlo * aWlo, R2hi = t * t - Flo * Flo + aWhi * aWhi;
        if (R2lo > 1e-3f * t * t) {
            float Rlo = adv(sqrtf(R2lo), +1) * (1.0f - 1e-6f), Rhi = adv(sqrtf(R2hi), -1) * (1.0f + 1e-6f);
            float tol = 2e-6f * Fhi * Fhi + 1e-5f * (aWhi * t + Rhi * Fhi);
            int r1 = !(Wlo * t + Rlo * Flo > tol);
            int r2_sure = (Wlo * t - Rhi * Fhi) < -tol - 1e-3f * t * t;
            if (!r1 && r2_sure) e = (t + Rhi) * adv(1.0f / (Flo + Wlo), -1) * 1.001f;
        }
    } else if (Flo > 1.01f * t && Whi < -0.01f * t) {
        float it = adv(1.0f / t, -1);
        float aVlo = -Whi * it, P = Fhi * it;
        float D = 1.0f - P * P + aVlo * aVlo;
        if (D > 0.02f) e = (Fhi - Wlo) * it * adv(1.0f / (1.0f + adv(sqrtf(D), +1)), -1);
    }
    return e * e;
}
static float dist_from_e2(float x) { return 0.5f * LN2F * (float)log2((double)x) - (ADV ? 1e-6f : 0.0f); }

typedef struct { f4 *bound; float *mag; uint32_t *shape; } staged_t;

/* over the first EST_OBJECTS / 2 planes and the first EST_OBJECTS / 2 horospheres */
static float upper_estimate(const staged_t *st, const uint32_t *slot_obj, uint32_t n, uint32_t np, const bray_t *r,
                            uint32_t prev) {
    float best = INFINITY;
    const uint32_t half = EST_OBJECTS / 2;
    for (uint32_t q = 0; q < n; ++q) {
        if (!(q < np ? q < half : q - np < half)) continue;
        best = fminf(best, sure_crossing_e2(bound_fw(st->bound[q], st->mag[q], r), st->shape[q], slot_obj[q] == prev, r->t));
    }
    return best < INFINITY ? dist_from_e2(best) : best;
}

static uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16; return h;
}

#ifndef CULL_CHECK_NO_MAIN
int main(int argc, char **argv) {
    if (argc < 8) { fprintf(stderr, "usage\n"); return 2; }
    FILE *f = fopen(argv[1], "rb");
    if (!f) { fprintf(stderr, "scene file\n"); return 2; }
    static uint8_t buf[1 << 24];
    size_t len = fread(buf, 1, sizeof buf, f);
    fclose(f);
    uint32_t W = (uint32_t)atoi(argv[2]), H = (uint32_t)atoi(argv[3]), hops = (uint32_t)atoi(argv[4]);
    uint32_t npix = (uint32_t)atoi(argv[5]), gseed = (uint32_t)strtoul(argv[6], NULL, 10);
    ADV = atoi(argv[7]);
    scene_t sc;
    if (scene_parse(1, buf, len, 32, &sc)) { fprintf(stderr, "scene parse\n"); return 2; }
    staged_t st;
    st.bound = malloc(sizeof(f4) * (sc.n + 1));
    st.mag = malloc(sizeof(float) * (sc.n + 1));
    st.shape = malloc(sizeof(uint32_t) * (sc.n + 1));
    for (uint32_t k = 0; k < sc.n; ++k) {
        st.shape[k] = sc.mat[k].shape;
        st.bound[k] = stage_bound(sc.mo[k], st.shape[k]);
        st.mag[k] = bound_mag(st.bound[k]);
    }
    long long n_hops = 0, n_exact = 0, wrong = 0;
    /* scan order of the staged slots: planes, then horospheres, each in scene order (the
     * kernel's dummy slot after an odd number of planes is never a candidate: left out) */
    uint32_t *slot_obj = malloc(sizeof(uint32_t) * (sc.n + 1));
    uint32_t ns = 0, np = 0;
    for (uint32_t k = 0; k < sc.n; ++k) np += st.shape[k] == 0;
    for (uint32_t want = 0; want < 2; ++want)
        for (uint32_t k = 0; k < sc.n; ++k)
            if (st.shape[k] == want) slot_obj[ns++] = k;
    staged_t ss;
    ss.bound = malloc(sizeof(f4) * (sc.n + 1));
    ss.mag = malloc(sizeof(float) * (sc.n + 1));
    ss.shape = malloc(sizeof(uint32_t) * (sc.n + 1));
    for (uint32_t q = 0; q < sc.n; ++q) {
        ss.bound[q] = st.bound[slot_obj[q]];
        ss.mag[q] = st.mag[slot_obj[q]];
        ss.shape[q] = st.shape[slot_obj[q]];
    }
    for (uint32_t pi = 0; pi < npix; ++pi) {
        uint32_t px = (uint32_t)(((uint64_t)pi * 2654435761u) % ((uint64_t)W * H));
        uint32_t rng = fmix32(gseed ^ fmix32(px));
        uint32_t x = px % W, y = px / W;
        R pxr = ((R)(2u * x + 1u) - (R)W) / (R)H, pyr = ((R)H - (R)(2u * y + 1u)) / (R)H, size = (R)2 / (R)H;
        R u0 = rng_uniform(&rng), u1 = rng_uniform(&rng);
        R sx = pxr + size * (u0 - (R)0.5f), sy = pyr + size * (u1 - (R)0.5f);
        vec3 ld = normalize3(v3(sx, sy, (R)-1 / sc.fov));
        quat start = q4(0, 0, 1, 0);
        ray_hy ray;
        ray.dir = normalize4(mo_deriv_q(sc.cam_mo, start, q4(ld.x, ld.y, ld.z, 0)));
        ray.start = mo_apply_q(sc.cam_mo, start);
        col3 inten = {1, 1, 1}, em = {0, 0, 0};
        uint32_t prev = 0xFFFFFFFFu;
        for (uint32_t h = 0; h < hops; ++h) {
            ++n_hops;
            /* the full scan, in the reference's order */
            R min_dist = -1; uint32_t min_index = 0; ray_hy min_local = ray; quat min_normal = q4(0, 0, 0, 0);
            for (uint32_t k = 0; k < sc.n; ++k) {
                int rep = (k == prev);
                ray_hy local = ray_hy_map(ray, sc.mo_inv[k]);
                quat nrm;
                R d = st.shape[k] == 0 ? plane_hy_detect(rep, &nrm, &local) : horosphere_detect(rep, &nrm, &local);
                if (d > -EPS && (min_dist <= -EPS || d < min_dist)) { min_dist = d; min_index = k; min_local = local; min_normal = nrm; }
            }
            /* the culled scan, as hop_hy runs it */
            bray_t br = bound_ray(ray.start, ray.dir);
            int can = cull_point_ok(ray.start);
            cull_t cull = cull_none();
            if (can) {
                float u = upper_estimate(&ss, slot_obj, sc.n, np, &br, prev);
                if (u < INFINITY) cull = cull_from_dist(u);
            }
            R cd = -1; uint32_t ck = 0;
            for (uint32_t c0 = 0; c0 < sc.n; c0 += 32) {
                uint32_t cn = sc.n - c0 < 32 ? sc.n - c0 : 32, mask = 0;
                for (uint32_t j = 0; j < cn; ++j)
                    if (!can || !culled_point(ss.bound[c0 + j], ss.mag[c0 + j], ss.shape[c0 + j], &br, cull)) mask |= 1u << j;
                if (can)
                    for (uint32_t j = 0; j < cn; ++j)
                        if ((mask >> j & 1) && culled_fw(bound_fw(ss.bound[c0 + j], ss.mag[c0 + j], &br), ss.shape[c0 + j], br.t, cull))
                            mask &= ~(1u << j);
                for (uint32_t j = 0; j < cn; ++j) {
                    if (!(mask >> j & 1)) continue;
                    uint32_t q = c0 + j, k = slot_obj[q];
                    if (can && culled_point(ss.bound[q], ss.mag[q], ss.shape[q], &br, cull)) continue;
                    int rep = (k == prev);
                    if (ss.shape[q] == 0 && rep) continue;
                    ++n_exact;
                    ray_hy local = ray_hy_map(ray, sc.mo_inv[k]);
                    quat nrm;
                    R d = ss.shape[q] == 0 ? plane_hy_detect(rep, &nrm, &local) : horosphere_detect(rep, &nrm, &local);
                    /* (distance, scene index): the slots are not in scene order */
                    if (d > -EPS && (cd <= -EPS || d < cd || (d == cd && k < ck))) { cd = d; ck = k; cull = cull_from_dist((float)d); }
                }
            }
            if ((cd > -EPS) != (min_dist > -EPS) || (cd > -EPS && (cd != min_dist || ck != min_index))) ++wrong;
            /* the path goes on as the reference's does (covered.inl, mapped.inl) */
            if (!(min_dist > -EPS)) break;
            ray_hy hit = ray_hy_map(min_local, sc.mo[min_index]);
            ray_hy loc = ray_hy_map(hit, sc.mo_inv[min_index]);
            vec3 d3 = v3(loc.dir.x, loc.dir.y, loc.dir.z), n3 = v3(min_normal.x, min_normal.y, min_normal.z);
            int ret = mixture_interact(&sc.mat[min_index], &rng, n3, &d3, &inten, &em);
            loc.dir = q4(d3.x, d3.y, d3.z, 0);
            ray = ray_hy_map(loc, sc.mo[min_index]);
            if (!ret) break;
            prev = min_index;
        }
    }
    printf("hops %lld exact_per_hop %.3f wrong %lld\n", n_hops, n_hops ? (double)n_exact / n_hops : 0.0, wrong);
    scene_free(&sc);
    return 0;
}
#endif  /* CULL_CHECK_NO_MAIN */
