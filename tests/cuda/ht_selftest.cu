// Test-only CUDA library (tests/cuda/libht_selftest.so): device unit tests of the render
// path's float helpers. It checks that the shared-reciprocal division (qdiv) and the fast
// Moebius ray map are bit-identical to their IEEE-division forms, and evaluates the device
// primitives (Moebius maps, distances, shape tests, samplers, materials) on given inputs for
// the property tests of tests/test_gpu_properties.py. Not part of the product.
#include <cuda_runtime.h>
#include <cstdint>

#include "../../hypertrace_b200/csrc/ht_math.cuh"
#include "../../hypertrace_b200/csrc/ht_generic.cuh"

using namespace ht;

__device__ __forceinline__ uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ float bits_float(uint32_t sign, uint32_t exp, uint32_t mant) {
    return __uint_as_float((sign << 31) | (exp << 23) | (mant & 0x7FFFFFu));
}

// mode 0: random signs/mantissas, exponents in [127-75, 127+75] (some outside the safe range)
// mode 1: every divisor mantissa in turn (i mod 2^23), random numerator
// mode 2: every numerator mantissa in turn, random divisor
// mode 3: numerators with tiny/zero/huge values around the range limits
__global__ void k_div(uint64_t n, uint64_t seed, int mode, unsigned long long *out) {
    unsigned long long fast = 0, mism = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h1 = splitmix(seed ^ (i * 2 + 0)), h2 = splitmix(seed ^ (i * 2 + 1));
        uint32_t ea = 52 + (uint32_t)(h1 % 151), eb = 52 + (uint32_t)(h2 % 151);
        uint32_t ma = (uint32_t)(h1 >> 20), mb = (uint32_t)(h2 >> 20);
        if (mode == 1) mb = (uint32_t)(i & 0x7FFFFF);
        if (mode == 2) ma = (uint32_t)(i & 0x7FFFFF);
        if (mode == 3) ea = (uint32_t)(h1 >> 40) % 3 == 0 ? 0 : 40 + (uint32_t)(h1 % 175);
        float a = bits_float((uint32_t)(h1 >> 63), ea, ma);
        float b = bits_float((uint32_t)(h2 >> 63), eb, mb);
        bool bad = false;
        Rcp r = rcp_of(b, bad);
        float q = qdiv(a, r, bad);
        if (!bad) {
            ++fast;
            if (__float_as_uint(q) != __float_as_uint(__fdiv_rn(a, b))) ++mism;
        }
    }
    atomicAdd(&out[0], fast);
    atomicAdd(&out[1], mism);
}

// Random Moebius maps (det not normalised: the map only has to be well defined), points
// in the upper half-space and unit directions: fast vs IEEE ray map, all 8 outputs.
__global__ void k_raymap(uint64_t n, uint64_t seed, unsigned long long *out) {
    unsigned long long cnt = 0, mism = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float f[16];
        for (int k = 0; k < 16; ++k) {
            uint64_t h = splitmix(seed ^ (i * 16 + k));
            f[k] = ((float)(h >> 40) / 16777216.0f) * 4.0f - 2.0f;
        }
        Mo m;
        m.a.x = f[0]; m.a.y = f[1]; m.b.x = f[2]; m.b.y = f[3];
        m.c.x = f[4]; m.c.y = f[5]; m.d.x = f[6]; m.d.y = f[7];
        Q4 p = q4(f[8], f[9], fabsf(f[10]) + 0.01f, 0.0f);
        Q4 v = normalize4(q4(f[11], f[12], f[13], 0.0f));
        HyRay a = ray_hy_map(m, p, v);
        HyRay b = ray_hy_map_ieee(m, p, v);
        ++cnt;
        bool same = __float_as_uint(a.p.x) == __float_as_uint(b.p.x) && __float_as_uint(a.p.y) == __float_as_uint(b.p.y) &&
                    __float_as_uint(a.p.z) == __float_as_uint(b.p.z) && __float_as_uint(a.p.w) == __float_as_uint(b.p.w) &&
                    __float_as_uint(a.v.x) == __float_as_uint(b.v.x) && __float_as_uint(a.v.y) == __float_as_uint(b.v.y) &&
                    __float_as_uint(a.v.z) == __float_as_uint(b.v.z) && __float_as_uint(a.v.w) == __float_as_uint(b.v.w);
        // NaN outputs compare by bit pattern too; count only real differences
        if (!same) ++mism;
    }
    atomicAdd(&out[0], cnt);
    atomicAdd(&out[1], mism);
}

// Exhaustive: hy_dist_from_x(x) <= hy_dist_from_x(next float after x) for every float x in
// [1, +inf). Counts violations (a NaN result counts as one).
__global__ void k_monotone(unsigned long long *out) {
    unsigned long long checked = 0, viol = 0;
    const uint32_t lo = 0x3f800000u, hi = 0x7f800000u;
    for (uint32_t b = lo + blockIdx.x * blockDim.x + threadIdx.x; b < hi; b += gridDim.x * blockDim.x) {
        const float f0 = hy_dist_from_x(__uint_as_float(b));
        const float f1 = hy_dist_from_x(__uint_as_float(b + 1));
        ++checked;
        if (!(f0 <= f1)) ++viol;
    }
    atomicAdd(&out[0], checked);
    atomicAdd(&out[1], viol);
}

static int run(void (*launch)(unsigned long long *), unsigned long long *host) {
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess) return -2;
    cudaMemset(d, 0, 2 * sizeof(unsigned long long));
    launch(d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(host, d, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -2;
}

static uint64_t g_n, g_seed;
static int g_mode;

extern "C" int ht_selftest_div(uint64_t n, uint64_t seed, int mode, unsigned long long *host_out) {
    g_n = n; g_seed = seed; g_mode = mode;
    return run([](unsigned long long *d) { k_div<<<148 * 16, 256>>>(g_n, g_seed, g_mode, d); }, host_out);
}
extern "C" int ht_selftest_raymap(uint64_t n, uint64_t seed, unsigned long long *host_out) {
    g_n = n; g_seed = seed;
    return run([](unsigned long long *d) { k_raymap<<<148 * 8, 256>>>(g_n, g_seed, d); }, host_out);
}
extern "C" int ht_selftest_monotone(unsigned long long *host_out) {
    return run([](unsigned long long *d) { k_monotone<<<148 * 16, 256>>>(d); }, host_out);
}

// ------------------------------------------------------------------ primitive evaluation
// Each item reads IN floats from `in` (stride `is`) and writes OUT floats (stride `os`);
// `seeds` carries an RNG state per item for the samplers and materials.
enum {
    EV_MO_APPLY = 0,      // m[8] p[4] -> mo_apply_pos(m, p)[4]
    EV_MO_CHAIN = 1,      // a[8] b[8] p[4] -> apply(chain(a, b), p)[4], apply(a, apply(b, p))[4]
    EV_RAY_MAP = 2,       // m[8] p[4] v[4] -> ray_hy_map(m, p, v): p'[4] v'[4]
    EV_HY_DIST = 3,       // a[4] b[4] m[8] -> d(a, b), d(m a, m b)
    EV_PLANE_HY = 4,      // p[4] d[4] repeat -> dist, start[4], dir[4], normal[4]
    EV_HOROSPHERE = 5,    // same
    EV_HEMI = 6,          // (seed) -> v[3]
    EV_LAMBERT = 7,       // n[3] d[3] (seed) -> d'[3], ret
    EV_SPECULAR = 8,      // n[3] d[3] -> d'[3], ret
    EV_REFRACTIVE = 9,    // n[3] d[3] index -> d'[3], ret
    EV_SPHERE = 10,       // p[3] d[3] repeat -> dist, start[3], normal[3]
    EV_CUBE = 11,         // same
    EV_PLANE_EU = 12,     // same
    EV_RNG = 13,          // (seed) -> four successive uniforms
};
__device__ Mo ld_mo(const float *a) {
    Mo m;
    m.a.x = a[0]; m.a.y = a[1]; m.b.x = a[2]; m.b.y = a[3];
    m.c.x = a[4]; m.c.y = a[5]; m.d.x = a[6]; m.d.y = a[7];
    return m;
}
__device__ Q4 ld_q(const float *a) { return q4(a[0], a[1], a[2], a[3]); }
__device__ V3 ld_v(const float *a) { return v3(a[0], a[1], a[2]); }
__device__ void st_q(float *o, Q4 q) { o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w; }
__device__ void st_v(float *o, V3 v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

__global__ void k_eval(int kind, uint32_t n, const float *in, int is, float *out, int os, uint32_t *seeds) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *a = in + (size_t)i * is;
    float *o = out + (size_t)i * os;
    htg::Ctx c;
    c.rng = seeds ? seeds[i] : 0u;
    c.hasher = 0u;
    c.prev = 0xFFFFFFFFu;
    c.flags = 0u;
    c.tests = 0u;
    c.end = nullptr;
    c.err = nullptr;
    switch (kind) {
    case EV_MO_APPLY: st_q(o, htg::mo_apply_pos(ld_mo(a), ld_q(a + 8))); break;
    case EV_MO_CHAIN: {
        const Mo x = ld_mo(a), y = ld_mo(a + 8);
        const Q4 p = ld_q(a + 16);
        st_q(o, htg::mo_apply_pos(htg::mo_chain(x, y), p));
        st_q(o + 4, htg::mo_apply_pos(x, htg::mo_apply_pos(y, p)));
        break;
    }
    case EV_RAY_MAP: {
        const HyRay r = ray_hy_map(ld_mo(a), ld_q(a + 8), ld_q(a + 12));
        st_q(o, r.p);
        st_q(o + 4, r.v);
        break;
    }
    case EV_HY_DIST: {
        const Q4 x = ld_q(a), y = ld_q(a + 4);
        const Mo m = ld_mo(a + 8);
        o[0] = hy_distance(x, y);
        o[1] = hy_distance(htg::mo_apply_pos(m, x), htg::mo_apply_pos(m, y));
        break;
    }
    case EV_PLANE_HY:
    case EV_HOROSPHERE: {
        htg::Light<htg::Hy> l;
        l.p = ld_q(a);
        l.v = ld_q(a + 4);
        if (a[8] != 0.0f) c.prev = c.hasher;   // repeat
        Q4 nrm = q4(0.0f, 0.0f, 0.0f, 0.0f);
        o[0] = kind == EV_PLANE_HY ? htg::PlaneHy::detect<4, true>(nullptr, c, nrm, l)
                                   : htg::Horosphere::detect<4, true>(nullptr, c, nrm, l);
        st_q(o + 1, l.p);
        st_q(o + 5, l.v);
        st_q(o + 9, nrm);
        break;
    }
    case EV_HEMI: st_v(o, hemisphere_cosine(c.rng)); break;
    case EV_LAMBERT:
    case EV_SPECULAR:
    case EV_REFRACTIVE: {
        htg::LightLocal l;
        l.k.x = l.k.y = l.k.z = 1.0f;
        l.v = ld_v(a + 3);
        Col e; e.x = e.y = e.z = 0.0f;
        bool ret;
        if (kind == EV_LAMBERT) ret = htg::Lambertian::interact<4>(nullptr, c, ld_v(a), l, e);
        else if (kind == EV_SPECULAR) ret = htg::Specular::interact<4>(nullptr, c, ld_v(a), l, e);
        else ret = htg::Refractive::interact<4>(reinterpret_cast<const uint8_t *>(a + 6), c, ld_v(a), l, e);
        st_v(o, l.v);
        o[3] = ret ? 1.0f : 0.0f;
        break;
    }
    case EV_SPHERE:
    case EV_CUBE:
    case EV_PLANE_EU: {
        htg::Light<htg::Eu> l;
        l.p = ld_v(a);
        l.v = ld_v(a + 3);
        if (a[6] != 0.0f) c.prev = c.hasher;
        V3 nrm = v3(0.0f, 0.0f, 0.0f);
        o[0] = kind == EV_SPHERE ? htg::Sphere::detect<4, true>(nullptr, c, nrm, l)
             : kind == EV_CUBE ? htg::Cube::detect<4, true>(nullptr, c, nrm, l)
                               : htg::PlaneEu::detect<4, true>(nullptr, c, nrm, l);
        st_v(o + 1, l.p);
        st_v(o + 4, nrm);
        break;
    }
    case EV_RNG:
        for (int k = 0; k < 4; ++k) o[k] = rng_uniform(c.rng);
        break;
    }
    if (seeds) seeds[i] = c.rng;
}

extern "C" int ht_selftest_eval(int kind, uint32_t n, const float *h_in, int is, float *h_out, int os,
                                uint32_t *h_seeds) {
    float *d_in = nullptr, *d_out = nullptr;
    uint32_t *d_seeds = nullptr;
    cudaError_t e = cudaMalloc(&d_in, sizeof(float) * (size_t)n * is + 16);
    if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(float) * (size_t)n * os + 16);
    if (e == cudaSuccess && h_seeds) e = cudaMalloc(&d_seeds, sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = cudaMemcpy(d_in, h_in, sizeof(float) * (size_t)n * is, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h_seeds) e = cudaMemcpy(d_seeds, h_seeds, sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_eval<<<(n + 127) / 128, 128>>>(kind, n, d_in, is, d_out, os, d_seeds);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h_out, d_out, sizeof(float) * (size_t)n * os, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && h_seeds) e = cudaMemcpy(h_seeds, d_seeds, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_seeds);
    return e == cudaSuccess ? 0 : -1;
}
