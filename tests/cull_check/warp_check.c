/* warp_check.c -- test infrastructure: the warp pre-cull of the wavefront scan
 * (hypertrace_b200/csrc/ht_trace.cuh: warp_box / warp_survivors) restated on the CPU and
 * checked against the lanes' own point test on real and on adversarially tight warps.
 *
 * The kernel culls a slot for a whole warp when F over the box of the lanes' (|p|^2, x, y),
 * widened by the warp's largest error allowance and a slack of 2^-16 of the magnitudes, lies
 * outside the loosest thresholds of the warp; each lane then runs its own packed point test
 * (F + eF < lo or F - eF > hi) only on the slots the warp keeps. That is exact only if a slot
 * the warp test culls is culled by every lane's own test in float arithmetic. This program
 * evaluates both tests operation by operation as the kernel does (build with
 * -ffp-contract=off) and counts the violations, on:
 *   - the hop depths of sampled paths of a scene, each depth's rays sorted by the kernel's
 *     16-bit key (direction cell, start cell) and cut into warps of 32, as the coherence sort
 *     arranges them;
 *   - "tight" warps: each sampled ray with 31 copies whose starts and thresholds differ by a
 *     few units in the last place, where the warp test is as close to each lane's test as a
 *     warp can make it and a slack too small for the rounding would show.
 *
 * usage: warp_check <scene bytes> <width> <height> <hops> <pixels> <global seed>
 * prints: warps <n> slots <n> culled <n> violations <n> tight_warps <n> tight_culled <n> tight_violations <n>
 */
#define CULL_CHECK_NO_MAIN
#include "cull_check.c"
#include <string.h>

typedef struct {
    bray_t br;
    float hp, lh, hh;   /* the lane's thresholds: planes -hp / hp, horospheres lh / hh */
    int can;
    float vx, vy, vz;
    uint32_t key;
} lane_t;

/* warp_box + warp_survivors for one slot: 1 when the warp test culls it */
static void box_term(float a, float lo, float hi, float *flo, float *fhi, float *mag) {
    float p = a * lo, q = a * hi;
    *flo += fminf(p, q);
    *fhi += fmaxf(p, q);
    *mag += fmaxf(fabsf(p), fabsf(q));
}
static int warp_culls(f4 rec, float mag, uint32_t shape, const lane_t *w) {
    float r2lo = INFINITY, r2hi = -INFINITY, xlo = INFINITY, xhi = -INFINITY, ylo = INFINITY, yhi = -INFINITY;
    float K = -INFINITY, hp = -INFINITY, lh = INFINITY, hh = -INFINITY;
    for (int l = 0; l < 32; ++l) {
        r2lo = fminf(r2lo, w[l].br.r2); r2hi = fmaxf(r2hi, w[l].br.r2);
        xlo = fminf(xlo, w[l].br.x);    xhi = fmaxf(xhi, w[l].br.x);
        ylo = fminf(ylo, w[l].br.y);    yhi = fmaxf(yhi, w[l].br.y);
        K = fmaxf(K, w[l].br.K);
        hp = fmaxf(hp, w[l].hp); lh = fminf(lh, w[l].lh); hh = fmaxf(hh, w[l].hh);
    }
    float e = mag * K;
    float flo = rec.w, fhi = rec.w, m = fabsf(rec.w);
    box_term(rec.x, r2lo, r2hi, &flo, &fhi, &m);
    box_term(rec.y, xlo, xhi, &flo, &fhi, &m);
    box_term(rec.z, ylo, yhi, &flo, &fhi, &m);
    float slack = 0x1p-16f * (m + e);
    float lo = lh, hi = hh;
    if (shape == 0) { lo = -hp; hi = hp; }
    return ((fhi + e) + slack < lo) || ((flo - e) - slack > hi);
}
/* the lane's own point test (survivors2: eF once, F + eF and F - eF) */
static int lane_culls(f4 rec, float mag, uint32_t shape, const lane_t *l) {
    float F = fmaf(rec.x, l->br.r2, fmaf(rec.y, l->br.x, fmaf(rec.z, l->br.y, rec.w)));
    float e = mag * l->br.K;
    float lo = l->lh, hi = l->hh;
    if (shape == 0) { lo = -l->hp; hi = l->hp; }
    return (F + e < lo) || (F + (-e) > hi);
}
static void lane_thresholds(lane_t *l, cull_t c) {
    float t = l->br.t;
    l->hp = 2.0f * t * c.S;
    l->lh = t * (1.0f / c.E);
    l->hh = t * c.E;
}

/* the kernel's sort key (sort_dir_cell, sort_axis_cell, spread3) */
static uint32_t axis_cell(float u, float lo, float scale) {
    float v = fminf(fmaxf((u - lo) * scale, 0.0f), 7.0f);
    return (uint32_t)v;
}
static uint32_t spread3(uint32_t c) { return (c & 1u) | ((c & 2u) << 2) | ((c & 4u) << 4); }
static uint32_t dir_cell(float vx, float vy, float vz) {
    float ax = fabsf(vx), ay = fabsf(vy), az = fabsf(vz), m, a, b;
    uint32_t face;
    if (ax >= ay && ax >= az) { face = vx > 0.0f ? 1u : 0u; m = ax; a = vy; b = vz; }
    else if (ay >= az)        { face = vy > 0.0f ? 3u : 2u; m = ay; a = vz; b = vx; }
    else                      { face = vz > 0.0f ? 5u : 4u; m = az; a = vx; b = vy; }
    float r = m > 0.0f ? 1.0f / m : 0.0f;
    uint32_t ia = (uint32_t)fminf(fmaxf((a * r + 1.0f) * 2.0f, 0.0f), 3.0f);
    uint32_t ib = (uint32_t)fminf(fmaxf((b * r + 1.0f) * 2.0f, 0.0f), 3.0f);
    return face * 16u + ia * 4u + ib;
}
static int by_key(const void *a, const void *b) {
    const lane_t *x = (const lane_t *)a, *y = (const lane_t *)b;
    return x->key < y->key ? -1 : x->key > y->key;
}

/* every slot of the scene against one warp: adds to the counts */
static void check_warp(const lane_t *w, const staged_t *ss, uint32_t n, long long *slots, long long *culled,
                       long long *violations) {
    for (int l = 0; l < 32; ++l)
        if (!w[l].can) return;   /* the kernel runs the warp test only when every lane can cull */
    for (uint32_t q = 0; q < n; ++q) {
        ++*slots;
        if (!warp_culls(ss->bound[q], ss->mag[q], ss->shape[q], w)) continue;
        ++*culled;
        for (int l = 0; l < 32; ++l)
            if (!lane_culls(ss->bound[q], ss->mag[q], ss->shape[q], &w[l])) {
                if (*violations < 5)
                    fprintf(stderr, "violation: slot %u lane %d\n", q, l);
                ++*violations;
            }
    }
}

static lane_t make_lane(quat p, quat v, uint32_t prev, const staged_t *ss, const uint32_t *slot_obj, uint32_t n,
                        uint32_t np) {
    lane_t l;
    memset(&l, 0, sizeof l);
    l.br = bound_ray(p, v);
    l.can = cull_point_ok(p);
    cull_t c = cull_none();
    if (l.can) {
        float u = upper_estimate(ss, slot_obj, n, np, &l.br, prev);
        if (u < INFINITY) c = cull_from_dist(u);
    }
    lane_thresholds(&l, c);
    l.vx = v.x; l.vy = v.y; l.vz = v.z;
    return l;
}

int main(int argc, char **argv) {
    if (argc < 7) { fprintf(stderr, "usage\n"); return 2; }
    FILE *f = fopen(argv[1], "rb");
    if (!f) { fprintf(stderr, "scene file\n"); return 2; }
    static uint8_t buf[1 << 24];
    size_t len = fread(buf, 1, sizeof buf, f);
    fclose(f);
    uint32_t W = (uint32_t)atoi(argv[2]), H = (uint32_t)atoi(argv[3]), hops = (uint32_t)atoi(argv[4]);
    uint32_t npix = (uint32_t)atoi(argv[5]), gseed = (uint32_t)strtoul(argv[6], NULL, 10);
    scene_t sc;
    if (scene_parse(1, buf, len, 32, &sc)) { fprintf(stderr, "scene parse\n"); return 2; }
    /* slots in the kernel's scan order: planes, then horospheres, each in scene order */
    uint32_t n = sc.n, np = 0, ns = 0;
    uint32_t *slot_obj = malloc(sizeof(uint32_t) * n);
    staged_t ss;
    ss.bound = malloc(sizeof(f4) * n);
    ss.mag = malloc(sizeof(float) * n);
    ss.shape = malloc(sizeof(uint32_t) * n);
    for (uint32_t k = 0; k < n; ++k) np += sc.mat[k].shape == 0;
    for (uint32_t want = 0; want < 2; ++want)
        for (uint32_t k = 0; k < n; ++k)
            if (sc.mat[k].shape == want) slot_obj[ns++] = k;
    for (uint32_t q = 0; q < n; ++q) {
        uint32_t k = slot_obj[q];
        ss.shape[q] = sc.mat[k].shape;
        ss.bound[q] = stage_bound(sc.mo[k], ss.shape[q]);
        ss.mag[q] = bound_mag(ss.bound[q]);
    }
    /* rays of every hop depth of the sampled paths, as the kernel's queues hold them */
    lane_t **depth = malloc(sizeof(lane_t *) * hops);
    quat **dp = malloc(sizeof(quat *) * hops), **dv = malloc(sizeof(quat *) * hops);
    uint32_t **dprev = malloc(sizeof(uint32_t *) * hops);
    uint32_t *cnt = calloc(hops, sizeof(uint32_t));
    for (uint32_t h = 0; h < hops; ++h) {
        depth[h] = malloc(sizeof(lane_t) * npix);
        dp[h] = malloc(sizeof(quat) * npix); dv[h] = malloc(sizeof(quat) * npix);
        dprev[h] = malloc(sizeof(uint32_t) * npix);
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
            uint32_t i = cnt[h]++;
            depth[h][i] = make_lane(ray.start, ray.dir, prev, &ss, slot_obj, n, np);
            dp[h][i] = ray.start; dv[h][i] = ray.dir; dprev[h][i] = prev;
            /* the path goes on as the reference's does: nearest hit of the full scan */
            R min_dist = -1; uint32_t min_index = 0; ray_hy min_local = ray; quat min_normal = q4(0, 0, 0, 0);
            for (uint32_t k = 0; k < n; ++k) {
                int rep = (k == prev);
                ray_hy local = ray_hy_map(ray, sc.mo_inv[k]);
                quat nrm;
                R d = sc.mat[k].shape == 0 ? plane_hy_detect(rep, &nrm, &local) : horosphere_detect(rep, &nrm, &local);
                if (d > -EPS && (min_dist <= -EPS || d < min_dist)) { min_dist = d; min_index = k; min_local = local; min_normal = nrm; }
            }
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
    long long warps = 0, slots = 0, culled = 0, viol = 0, twarps = 0, tslots = 0, tculled = 0, tviol = 0;
    for (uint32_t h = 0; h < hops; ++h) {
        lane_t *a = depth[h];
        uint32_t m = cnt[h];
        if (m < 32) continue;
        /* the sort key: cells over mean +- 2 sigma of this depth's starts */
        double s[6] = {0, 0, 0, 0, 0, 0};
        for (uint32_t i = 0; i < m; ++i) {
            double lz = a[i].br.t > 0.0f ? log((double)a[i].br.t) : 0.0;
            s[0] += a[i].br.x; s[1] += (double)a[i].br.x * a[i].br.x;
            s[2] += a[i].br.y; s[3] += (double)a[i].br.y * a[i].br.y;
            s[4] += lz; s[5] += lz * lz;
        }
        float lo[3], sc3[3];
        for (int ax = 0; ax < 3; ++ax) {
            double mean = s[2 * ax] / m, sd = sqrt(fmax(s[2 * ax + 1] / m - mean * mean, 0.0));
            lo[ax] = (float)(mean - 2.0 * sd);
            sc3[ax] = sd > 0.0 ? (float)(2.0 / sd) : 0.0f;
        }
        for (uint32_t i = 0; i < m; ++i) {
            float lz = a[i].br.t > 0.0f ? logf(a[i].br.t) : 0.0f;
            uint32_t cx = axis_cell(a[i].br.x, lo[0], sc3[0]), cy = axis_cell(a[i].br.y, lo[1], sc3[1]);
            uint32_t cz = axis_cell(lz, lo[2], sc3[2]);
            a[i].key = dir_cell(a[i].vx, a[i].vy, a[i].vz) * 512u + (spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2));
        }
        /* tight warps first (they read the queue order), then the sorted warps */
        for (uint32_t i = 0; i < m; i += 7) {
            lane_t w[32];
            for (int l = 0; l < 32; ++l) {
                quat p = dp[h][i];
                int kx = l % 5 - 2, ky = (l / 5) % 5 - 2, kz = (l / 25) % 3 - 1;
                for (int k = 0; k < abs(kx); ++k) p.x = nextafterf(p.x, kx > 0 ? INFINITY : -INFINITY);
                for (int k = 0; k < abs(ky); ++k) p.y = nextafterf(p.y, ky > 0 ? INFINITY : -INFINITY);
                for (int k = 0; k < abs(kz); ++k) p.z = nextafterf(p.z, kz > 0 ? INFINITY : -INFINITY);
                w[l] = make_lane(p, dv[h][i], dprev[h][i], &ss, slot_obj, n, np);
            }
            ++twarps;
            check_warp(w, &ss, n, &tslots, &tculled, &tviol);
        }
        qsort(a, m, sizeof(lane_t), by_key);
        for (uint32_t i = 0; i + 32 <= m; i += 32) {
            ++warps;
            check_warp(a + i, &ss, n, &slots, &culled, &viol);
        }
    }
    printf("warps %lld slots %lld culled %lld violations %lld tight_warps %lld tight_culled %lld tight_violations %lld\n",
           warps, slots, culled, viol, twarps, tculled, tviol);
    (void)tslots;
    scene_free(&sc);
    return 0;
}
