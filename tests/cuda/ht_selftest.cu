// Test-only CUDA library (tests/cuda/libht_selftest.so): device unit tests of the render
// path's float helpers. It checks that the shared-reciprocal division (qdiv) and the fast
// Moebius ray map are bit-identical to their IEEE-division forms. Not part of the product.
#include <cuda_runtime.h>
#include <cstdint>

#include "../../hypertrace_b200/csrc/ht_math.cuh"

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
