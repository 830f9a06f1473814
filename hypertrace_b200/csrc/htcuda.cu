// htcuda.cu -- kernels and the C ABI of libhtcuda.so (declared in include/htcuda.h).
//
// Kernels:
//   render_plain<R>      one thread per pixel, one pass: the reference's `render` kernel
//                        (kernel/ocl/render/render.cl:6-27) launched over a (W,H) grid.
//   render_wave<R, FH>   one launch per hop depth of a pass (FH: hop 0 from the pixels, or a
//                        later hop from a queue of ray states); survivors are appended to
//                        the other queue with warp-aggregated atomics, so warps scan with
//                        full lanes. The form htc_render_passes uses.
//   render_batch_wave<RF, FH>  the same over many views at once, one launch per pass index,
//                        hop depth and recipe, tiles of the views' queues cut on the device.
//   render_persistent<R> one launch for P passes: warps pull pixels from a queue, each lane
//                        runs its pixel's P samples in order and regenerates a finished path
//                        in place (the allocation-free entry point uses it).
//   post kernels         extract / gamma / pack (processing/src/canvas.rs:126-135,176-186,
//                        processing/src/filter/gamma.rs:10-19) and their fused form.
// Every render kernel stages the scene's inverse object maps, distance-bound records and
// shape indices in shared memory once per block (per view change in the batched kernels);
// the object scan reads them as warp-uniform broadcasts. Each pixel's samples take the same
// float operations in the same order in every form, so all forms give the same bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/htcuda.h"
#include "ht_trace.cuh"
#include "ht_host.hpp"

using namespace ht;

// ============================================================================ errors
thread_local std::string g_last_error;

// Minimum resident blocks per SM requested from ptxas for the render kernels (register cap).
// The scan is latency-bound on dependent FP32 chains, so resident warps matter, but the
// packed point-bound loop and the slot bookkeeping hold more values than the earlier scan.
// Measured on the current code at 1080p / 200 objects (Msamples/s): 7 -> 6 -> 5 blocks (72 ->
// 80 -> 96 registers) took the wavefront kernel 368.6 -> 373.2 -> 377.4 and the batched mix
// (spp / 16) 994 -> 1012 -> 1019; the one-pass kernel 288.6 -> 296.5 -> 295.6. The earlier
// scan had measured 7 best (239.5 against 232 for 6). With the coherence sort and the warp
// pre-cull, 6 -> 5 -> 4 blocks gave the single-view wavefront kernel 489.5 -> 493.0 -> 508.1
// and the batched kernels (mix at spp / 16) 1170.8 -> 1210.2 -> 1172.2, so the two now have
// caps of their own; 3 blocks for the later hops measured 462.2, 6 for hop 0 508.6 (510.3).
#ifndef HT_PERSIST_MINB
#define HT_PERSIST_MINB 6
#endif
#ifndef HT_PLAIN_MINB
#define HT_PLAIN_MINB 6
#endif
#ifndef HT_WAVE_MINB    // render_wave, hop depths after the first
#define HT_WAVE_MINB 4
#endif
#ifndef HT_WAVE0_MINB   // render_wave, hop depth 0 (camera rays: 0.764 ms per launch at 5, 0.792 at 4)
#define HT_WAVE0_MINB 5
#endif
#ifndef HT_BATCH_MINB   // render_batch_wave (one recipe per kernel)
#define HT_BATCH_MINB 5
#endif
// htc_render_passes: 2 = wavefronts (one launch per hop depth), 1 = the persistent kernel,
// 0 = one launch of the one-pass kernel per pass. All three give the same bits. Measured at
// 1920x1080 / 200 objects / H = 8 (Msamples/s): wavefronts 286.9, one-pass kernel 239.3,
// persistent kernel 208.6.
#ifndef HT_PASSES_MODE
#define HT_PASSES_MODE 2
#endif
#ifndef HT_BATCH_SORT   // coherence sort of the batch's hyperbolic views (with HT_BATCH_SPLIT)
#define HT_BATCH_SORT 1
#endif
// Batched wavefronts: 1 = one launch per recipe for each (pass, hop depth), 0 = one launch for both.
#ifndef HT_BATCH_SPLIT
#define HT_BATCH_SPLIT 1
#endif

// Device error word bits.
constexpr uint32_t ERR_SCENE = 1u;
constexpr uint32_t ERR_SMEM = 2u;

struct htc_program {
    int recipe;
    uint32_t hops;
    int address_width;
    uint32_t flags;
    uint32_t *d_err;     // device error word
    uint32_t *d_queue;   // [0] next pixel, [1] finished blocks (persistent kernel)
    int num_sms;
    int max_smem;
    GenericProgram *generic;   // scene types served by render_generic (htgeneric.cu), else NULL
    void *wave_buf;            // two wavefront queues (WAVE_SLOT_BYTES per slot each), grown on demand
    size_t wave_slots;         // slots per queue
    uint32_t *d_wave_ctr;      // 2 counters per hop depth
    void *sort_buf;            // coherence sort of the hyperbolic queues (SortBuf), grown with them
    size_t sort_slots;
    int double_support;        // scene bytes in the double_support layout, narrowed before rendering
    uint8_t *narrow_buf;       // the narrowed (f32 layout) scene, grown on demand
    size_t narrow_bytes;
};

// ============================================================================ staging
// Loads the scene header and the per-object data the scan reads into shared memory. Returns
// false (uniformly across the block) when the scene bytes fail validation.
//
// Hyperbolic scenes are staged in scan order, geodesic planes first (in index order), then
// horospheres (in index order); when the plane count is odd a dummy slot follows the planes,
// so that every pair of slots (2p, 2p + 1) holds one shape and the point-bound loop can test
// two objects per packed FP32 instruction. `orig[slot]` is the object's index in the scene:
// the scan compares hits on (distance, index), the reference's nearest-hit rule
// (object/vector.inl:37-50), so the order of the slots never changes the winner. Euclidean
// scenes are staged in index order (slot = index).
//
// Shared-memory layout for up to n objects (n + 1 slots, smem_bytes(n) bytes): inverse maps
// (2 float4 per slot), bound records (float4), the bound records again as pairs of slots
// ({x0, x1, y0, y1}, {z0, z1, w0, w1} per pair) and their magnitudes ({m0, m1}), then shape,
// bound magnitude and scene index per slot (u32 / f32 / u32), then 2 float4 per thread of a
// 128-thread block (the scan's winner, local frame).
constexpr uint32_t BLOCK_THREADS = 128;
struct SceneSmem {
    float4 *inv, *bound, *pa, *pb;
    float2 *pmag;
    uint32_t *shape, *orig;
    float *mag;
    float4 *win;
    float4 *end;   // first float4 past the layout
};
__host__ __device__ constexpr uint32_t scene_slots(uint32_t n) { return n + 1; }
__host__ __device__ constexpr size_t scene_win_offset(uint32_t n) {
    return ((size_t)scene_slots(n) * 60u + (size_t)((scene_slots(n) + 1) / 2) * 40u + 15u) & ~(size_t)15u;
}
__device__ __forceinline__ SceneSmem carve_scene(float4 *smem, uint32_t n) {
    const uint32_t ns = scene_slots(n), np = (ns + 1) / 2;
    SceneSmem c;
    c.inv = smem;
    c.bound = c.inv + 2 * ns;
    c.pa = c.bound + ns;
    c.pb = c.pa + np;
    c.pmag = reinterpret_cast<float2 *>(c.pb + np);
    c.shape = reinterpret_cast<uint32_t *>(c.pmag + np);
    c.mag = reinterpret_cast<float *>(c.shape + ns);
    c.orig = reinterpret_cast<uint32_t *>(c.mag + ns);
    c.win = smem + scene_win_offset(n) / 16;
    c.end = c.win + 2 * BLOCK_THREADS;
    return c;
}

// Stages object k (shape `shape`) into slot q.
template <int R>
__device__ __forceinline__ void stage_object(const uint8_t *obj, uint32_t shape, uint32_t k, uint32_t q,
                                             const SceneSmem &sm) {
    sm.shape[q] = shape;
    sm.orig[q] = k;
    float4 rec = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float mag = 0.0f;
    if (R == RECIPE_HY) {
        const Mo fwd = load_mo(obj);
        Mo inv = mo_inverse(fwd);
        sm.inv[2 * q] = make_float4(inv.a.x, inv.a.y, inv.b.x, inv.b.y);
        sm.inv[2 * q + 1] = make_float4(inv.c.x, inv.c.y, inv.d.x, inv.d.y);
        rec = stage_bound(fwd, shape);
        mag = bound_mag(rec);
    } else {
        Hom inv = hom3_inverse(load_hom(obj));
        sm.inv[2 * q] = make_float4(inv.shift.x, inv.shift.y, inv.shift.z, 0.0f);
        sm.inv[2 * q + 1] = make_float4(inv.rot.x, inv.rot.y, inv.rot.z, inv.rot.w);
    }
    sm.bound[q] = rec;
    sm.mag[q] = mag;
    float *pa = reinterpret_cast<float *>(&sm.pa[q >> 1]), *pb = reinterpret_cast<float *>(&sm.pb[q >> 1]);
    const uint32_t o = q & 1u;
    pa[o] = rec.x; pa[2 + o] = rec.y; pb[o] = rec.z; pb[2 + o] = rec.w;
    reinterpret_cast<float *>(&sm.pmag[q >> 1])[o] = mag;
}

template <int R>
__device__ bool stage_scene(const uint8_t *scene, size_t scene_size, uint32_t max_objects,
                            int address_width, uint32_t *err, StagedScene &s, const SceneSmem &sm,
                            uint32_t *s_hdr) {
    using L = Layout<R>;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        uint32_t ok = 1;
        uint32_t n = 0;
        if (scene_size < L::OBJECTS) ok = 0;
        if (ok) {
            n = ldu(scene, L::COUNT);
            if (address_width == 64 && ldu(scene, L::COUNT + 4) != 0) ok = 0;
            if ((scene_size - L::OBJECTS) / OBJ_STRIDE < n) ok = 0;
            if (n > max_objects) ok = 0;
        }
        s_hdr[0] = ok;
        s_hdr[1] = n;
    }
    __syncthreads();
    const uint32_t n = s_hdr[1];
    const bool header_ok = s_hdr[0] != 0;
    __syncthreads();
    if (!header_ok) {
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicOr(err, ERR_SCENE);
        return false;
    }
    const uint32_t tid = threadIdx.x + blockDim.x * threadIdx.y;
    const uint32_t nthreads = blockDim.x * blockDim.y;
    const uint8_t *objects = scene + L::OBJECTS;
    bool bad = false;
    uint32_t n_planes = 0, dummy = 0xFFFFFFFFu;
    if (R == RECIPE_HY) {
        // pass 1: the number of planes
        for (uint32_t r0 = 0; r0 < n; r0 += nthreads) {
            const uint32_t k = r0 + tid;
            const bool plane = k < n && ldu(objects + (size_t)k * OBJ_STRIDE, O_SHAPE) == 0;
            n_planes += (uint32_t)__syncthreads_count(plane ? 1 : 0);
        }
        // pass 2: slot = rank among the planes, or n_planes (rounded up to even) + rank among
        // the horospheres; ranks from a ballot per warp and the warps' counts in s_hdr[2..]
        const uint32_t h0 = (n_planes + 1) & ~1u;
        const uint32_t lane = tid & 31u, warp = tid >> 5, nwarps = (nthreads + 31) >> 5;
        uint32_t before = 0;   // planes among the objects before this block-wide step
        for (uint32_t r0 = 0; r0 < n; r0 += nthreads) {
            const uint32_t k = r0 + tid;
            const bool in = k < n;
            const uint8_t *obj = objects + (size_t)k * OBJ_STRIDE;
            const uint32_t shape = in ? ldu(obj, O_SHAPE) : 1u;
            const uint32_t ballot = __ballot_sync(0xffffffffu, in && shape == 0);
            if (lane == 0) s_hdr[2 + warp] = (uint32_t)__popc(ballot);
            __syncthreads();
            uint32_t rank = before + (uint32_t)__popc(ballot & ((1u << lane) - 1u)), total = 0;
            for (uint32_t w = 0; w < nwarps; ++w) {
                const uint32_t c = s_hdr[2 + w];
                if (w < warp) rank += c;
                total += c;
            }
            __syncthreads();
            before += total;
            if (in) {
                if (address_width == 64 && ldu(obj, O_SHAPE + 4) != 0) bad = true;
                if (shape > 1) bad = true;
                stage_object<R>(obj, shape > 1 ? 1u : shape, k, shape == 0 ? rank : h0 + (k - rank), sm);
            }
        }
        if (n_planes & 1u) {   // the dummy slot: never a candidate (masked), NaN bound record
            dummy = n_planes;
            if (tid == 0) {
                const float nan = __int_as_float(0x7fc00000);
                sm.shape[dummy] = 0;
                sm.orig[dummy] = 0xFFFFFFFFu;
                sm.bound[dummy] = make_float4(nan, nan, nan, nan);
                sm.mag[dummy] = 0.0f;
                float *pa = reinterpret_cast<float *>(&sm.pa[dummy >> 1]), *pb = reinterpret_cast<float *>(&sm.pb[dummy >> 1]);
                pa[1] = 0.0f; pa[3] = 0.0f; pb[1] = 0.0f; pb[3] = 0.0f;   // the odd half of its pair
                reinterpret_cast<float *>(&sm.pmag[dummy >> 1])[1] = 0.0f;
            }
        }
    } else {
        for (uint32_t k = tid; k < n; k += nthreads) {
            const uint8_t *obj = objects + (size_t)k * OBJ_STRIDE;
            const uint32_t shape = ldu(obj, O_SHAPE);
            if (address_width == 64 && ldu(obj, O_SHAPE + 4) != 0) bad = true;
            if (shape > 1) bad = true;
            stage_object<R>(obj, shape > 1 ? 1u : shape, k, k, sm);
        }
    }
    const int any_bad = __syncthreads_or(bad ? 1 : 0);
    if (any_bad) {
        if (tid == 0) atomicOr(err, ERR_SCENE);
        return false;
    }
    s.inv = sm.inv;
    s.bound = sm.bound;
    s.pa = sm.pa;
    s.pb = sm.pb;
    s.pmag = sm.pmag;
    s.shape = sm.shape;
    s.mag = sm.mag;
    s.orig = sm.orig;
    s.win = sm.win + 2 * tid;
    s.objects = objects;
    s.n = n;
    s.ns = n + (dummy != 0xFFFFFFFFu ? 1u : 0u);
    s.n_planes = R == RECIPE_HY ? n_planes : 0u;
    s.dummy = dummy;
    s.fov = ldf(scene, L::FOV);
    float4 bg = ldf4(scene, L::BG);
    s.background.x = bg.x; s.background.y = bg.y; s.background.z = bg.z;
    s.cam0 = ldf4(scene, 0);
    s.cam1 = ldf4(scene, 16);
    return true;
}

template <int R> struct PathOf;
template <> struct PathOf<RECIPE_HY> { using T = HyPath; };
template <> struct PathOf<RECIPE_EU> { using T = EuPath; };

template <int R>
__device__ __forceinline__ typename PathOf<R>::T camera(const StagedScene &s, float px, float py,
                                                        float size, uint32_t &rng, uint32_t flags) {
    if constexpr (R == RECIPE_HY) return camera_hy(s, px, py, size, rng, flags);
    else return camera_eu(s, px, py, size, rng, flags);
}
// WARP / full_warp: the hyperbolic scan's warp pre-cull (hop_hy), for callers whose warps
// enter together.
template <int R, bool OOL = true, bool WARP = false>
__device__ __forceinline__ bool hop(const StagedScene &s, typename PathOf<R>::T &ray, uint32_t &rng,
                                    uint32_t &prev_hash, Col &intensity, Col &emission, bool &hit,
                                    uint32_t &n_exact, bool full_warp = false) {
    if constexpr (R == RECIPE_HY)
        return hop_hy<OOL, WARP>(s, ray, rng, prev_hash, intensity, emission, hit, n_exact, full_warp);
    else return hop_eu(s, ray, rng, prev_hash, intensity, emission, hit, n_exact);
}

// Pixel centre and size (render.cl:12-18).
__device__ __forceinline__ void pixel_pos(uint32_t x, uint32_t y, uint32_t W, uint32_t H, float &px,
                                          float &py, float &size) {
    px = (__uint2float_rn(2u * x + 1u) - __uint2float_rn(W)) / __uint2float_rn(H);
    py = (__uint2float_rn(H) - __uint2float_rn(2u * y + 1u)) / __uint2float_rn(H);
    size = 2.0f / __uint2float_rn(H);
}

__device__ __forceinline__ void flush_stats(uint64_t *stats, uint32_t samples32, uint32_t hops32,
                                            uint32_t hits32, uint32_t exact32, uint32_t n_objects) {
    if (!stats) return;
    uint64_t samples = samples32, hops = hops32, hits = hits32, exact = exact32;
    for (int off = 16; off > 0; off >>= 1) {
        samples += __shfl_down_sync(0xffffffffu, samples, off);
        hops += __shfl_down_sync(0xffffffffu, hops, off);
        hits += __shfl_down_sync(0xffffffffu, hits, off);
        exact += __shfl_down_sync(0xffffffffu, exact, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd((unsigned long long *)&stats[HTC_STAT_SAMPLES], (unsigned long long)samples);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_HOPS], (unsigned long long)hops);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_OBJECT_TESTS], (unsigned long long)(hops * n_objects));
        atomicAdd((unsigned long long *)&stats[HTC_STAT_HITS], (unsigned long long)hits);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_EXACT_TESTS], (unsigned long long)exact);
    }
}

// ============================================================================ plain
template <int R>
__global__ void __launch_bounds__(128, HT_PLAIN_MINB) render_plain(
    const uint8_t *__restrict__ scene, size_t scene_size, uint32_t max_objects, int address_width,
    uint32_t W, uint32_t H, uint32_t hops, uint32_t flags, float4 *__restrict__ canvas,
    uint32_t *__restrict__ seeds, uint64_t *stats, uint32_t *err) {
    extern __shared__ float4 smem[];
    __shared__ uint32_t s_hdr[2 + BLOCK_THREADS / 32];
    const SceneSmem sm = carve_scene(smem, max_objects);
    StagedScene s;
    if (!stage_scene<R>(scene, scene_size, max_objects, address_width, err, s, sm, s_hdr)) return;

    // 128 threads = 32 x 4 pixels: each warp covers 32 consecutive pixels of a row.
    const uint32_t x = blockIdx.x * 32 + (threadIdx.x & 31);
    const uint32_t y = blockIdx.y * 4 + (threadIdx.x >> 5);
    const bool inside = x < W && y < H;
    uint32_t n_samples = 0, n_hops = 0, n_hits = 0, n_exact = 0;
    if (inside) {
        const uint32_t idx = x + W * y;
        float px, py, size;
        pixel_pos(x, y, W, H, px, py, size);
        uint32_t rng = seeds[idx];
        auto ray = camera<R>(s, px, py, size, rng, flags);
        Col intensity = {1.0f, 1.0f, 1.0f};
        Col emission = {0.0f, 0.0f, 0.0f};
        uint32_t prev_hash = HASH_NEVER;
        for (uint32_t i = 0; i < hops; ++i) {
            bool hit;
            n_hops += 1;
            // root tests inline: faster for this kernel (per view on the mixed workload's
            // views, 2138 vs 2177 ms), unlike the wavefront kernel
            bool go = hop<R, false>(s, ray, rng, prev_hash, intensity, emission, hit, n_exact);
            n_hits += hit ? 1 : 0;
            if (!go) break;
        }
        n_samples = 1;
        float4 c = canvas[idx];
        c.x += emission.x; c.y += emission.y; c.z += emission.z; c.w += 1.0f;
        canvas[idx] = c;
        seeds[idx] = rng;
    }
    flush_stats(stats, n_samples, n_hops, n_hits, n_exact, s.n);
}

// ============================================================================ persistent
constexpr uint32_t NO_PIXEL = 0xFFFFFFFFu;

// Counters of one thread, flushed once per launch.
struct LaneStats {
    uint32_t samples = 0, hops = 0, hits = 0, exact = 0;
    uint64_t tests = 0;   // object tests the reference makes (hops x objects)
};

__device__ __forceinline__ void flush_lane_stats(uint64_t *stats, const LaneStats &st) {
    if (!stats) return;
    uint64_t samples = st.samples, hops = st.hops, hits = st.hits, exact = st.exact, tests = st.tests;
    for (int off = 16; off > 0; off >>= 1) {
        samples += __shfl_down_sync(0xffffffffu, samples, off);
        hops += __shfl_down_sync(0xffffffffu, hops, off);
        hits += __shfl_down_sync(0xffffffffu, hits, off);
        exact += __shfl_down_sync(0xffffffffu, exact, off);
        tests += __shfl_down_sync(0xffffffffu, tests, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd((unsigned long long *)&stats[HTC_STAT_SAMPLES], (unsigned long long)samples);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_HOPS], (unsigned long long)hops);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_OBJECT_TESTS], (unsigned long long)tests);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_HITS], (unsigned long long)hits);
        atomicAdd((unsigned long long *)&stats[HTC_STAT_EXACT_TESTS], (unsigned long long)exact);
    }
}

// The persistent lane loop of render_persistent: warps take pixel
// indices [first, first + count) from `*counter` (global or shared memory) with one atomic
// per warp; each lane renders its pixel's `passes` samples in order and regenerates a camera
// ray as soon as a path ends. Returns when the warp has no pixel left.
template <int R>
__device__ __forceinline__ void trace_pixels(const StagedScene &s, uint32_t *counter, uint32_t first,
                                             uint32_t count, uint32_t W, uint32_t H, uint32_t hops,
                                             uint32_t passes, uint32_t flags, float4 *__restrict__ canvas,
                                             uint32_t *__restrict__ seeds, LaneStats &st) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t pixel = NO_PIXEL;
    bool done = passes == 0;
    uint32_t pass = 0, rng = 0, prev_hash = HASH_NEVER, hop_i = 0;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    float px = 0.f, py = 0.f, size = 0.f;
    typename PathOf<R>::T ray;
    Col intensity = {1.0f, 1.0f, 1.0f};
    Col emission = {0.0f, 0.0f, 0.0f};
    bool in_path = false;

    for (;;) {
        // Lanes without a pixel take the next ones from the counter: one atomic per warp.
        const bool need = !done && pixel == NO_PIXEL;
        const uint32_t mask = __ballot_sync(0xffffffffu, need);
        if (mask) {
            uint32_t base = 0;
            const int leader = __ffs(mask) - 1;
            if (lane == (uint32_t)leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const uint32_t mine = base + __popc(mask & ((1u << lane) - 1u));
                if (mine < count) {
                    pixel = first + mine;
                    const uint32_t x = pixel % W, y = pixel / W;
                    pixel_pos(x, y, W, H, px, py, size);
                    rng = seeds[pixel];
                    acc = canvas[pixel];
                    pass = 0;
                    in_path = false;
                } else {
                    done = true;
                }
            }
        }
        if (__all_sync(0xffffffffu, done)) break;
        if (pixel != NO_PIXEL && !in_path) {
            ray = camera<R>(s, px, py, size, rng, flags);
            intensity.x = intensity.y = intensity.z = 1.0f;
            emission.x = emission.y = emission.z = 0.0f;
            prev_hash = HASH_NEVER;
            hop_i = 0;
            in_path = true;
        }
        if (in_path) {
            bool hit;
            st.hops += 1;
            bool go = hop<R>(s, ray, rng, prev_hash, intensity, emission, hit, st.exact);
            st.hits += hit ? 1 : 0;
            hop_i += 1;
            if (!go || hop_i >= hops) {
                acc.x += emission.x; acc.y += emission.y; acc.z += emission.z; acc.w += 1.0f;
                st.samples += 1;
                in_path = false;
                pass += 1;
                if (pass >= passes) {
                    canvas[pixel] = acc;
                    seeds[pixel] = rng;
                    pixel = NO_PIXEL;
                }
            }
        }
    }
}

// The last block to finish rewinds the launch's queue words for the next launch.
__device__ __forceinline__ void rewind_queue(uint32_t *queue) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t finished = atomicAdd(&queue[1], 1u);
        if (finished == gridDim.x - 1) {
            queue[0] = 0;
            queue[1] = 0;
            __threadfence();
        }
    }
}

template <int R>
__global__ void __launch_bounds__(128, HT_PERSIST_MINB) render_persistent(
    const uint8_t *__restrict__ scene, size_t scene_size, uint32_t max_objects, int address_width,
    uint32_t W, uint32_t H, uint32_t hops, uint32_t passes, uint32_t flags,
    float4 *__restrict__ canvas, uint32_t *__restrict__ seeds, uint64_t *stats, uint32_t *err,
    uint32_t *queue) {
    extern __shared__ float4 smem[];
    __shared__ uint32_t s_hdr[2 + BLOCK_THREADS / 32];
    const SceneSmem sm = carve_scene(smem, max_objects);
    StagedScene s;
    const bool staged = stage_scene<R>(scene, scene_size, max_objects, address_width, err, s, sm, s_hdr);
    LaneStats st;
    if (staged) trace_pixels<R>(s, &queue[0], 0, W * H, W, H, hops, passes, flags, canvas, seeds, st);
    flush_stats(stats, st.samples, st.hops, st.hits, st.exact, staged ? s.n : 0);
    rewind_queue(queue);
}

// ============================================================================ wavefront
// One launch per hop depth. Launch h takes the paths that are still going after h hops
// from a queue, runs one hop on each and appends the survivors to the other queue; paths
// that end add their sample to the canvas right there. Hop 0 starts from the pixels
// (camera ray, no queue read). Warps take 32 queue slots at a time from a counter and
// append survivors with one atomic per warp, order kept within the warp, so a warp's
// lanes stay paths that started at neighbouring pixels and ran the same number of hops:
// no lane idles on a finished path while its warp scans, which is where the one-pass
// kernel loses a third of its lanes. The hop itself is `hop<R>` unchanged, so the result
// is bit-identical to render_plain.
struct WaveQueue {      // ray state, structure of arrays (one float4 load / store each)
    float4 *p;          // ray start
    float4 *v;          // ray direction
    float4 *t;          // intensity xyz, RNG state (bits) in w
    float4 *e;          // emission xyz, pixel index (bits) in w
    uint32_t *h;        // previous hit hash
    const uint32_t *o;  // read order: lane i of a hop takes slot o[i] (NULL: slot i)
};
constexpr size_t WAVE_SLOT_BYTES = 4 * sizeof(float4) + sizeof(uint32_t);

template <int R> __device__ __forceinline__ void path_store(float4 *p, float4 *v, const typename PathOf<R>::T &r) {
    if constexpr (R == RECIPE_HY) {
        *p = make_float4(r.p.x, r.p.y, r.p.z, r.p.w);
        *v = make_float4(r.v.x, r.v.y, r.v.z, r.v.w);
    } else {
        *p = make_float4(r.p.x, r.p.y, r.p.z, 0.0f);
        *v = make_float4(r.v.x, r.v.y, r.v.z, 0.0f);
    }
}
template <int R> __device__ __forceinline__ typename PathOf<R>::T path_load(float4 p, float4 v) {
    typename PathOf<R>::T r;
    if constexpr (R == RECIPE_HY) {
        r.p = q4(p.x, p.y, p.z, p.w);
        r.v = q4(v.x, v.y, v.z, v.w);
    } else {
        r.p = v3(p.x, p.y, p.z);
        r.v = v3(v.x, v.y, v.z);
    }
    return r;
}

__host__ __device__ inline WaveQueue wave_at(const WaveQueue &q, uint64_t off) {
    WaveQueue r;
    r.p = q.p ? q.p + off : nullptr;
    r.v = q.v ? q.v + off : nullptr;
    r.t = q.t ? q.t + off : nullptr;
    r.e = q.e ? q.e + off : nullptr;
    r.h = q.h ? q.h + off : nullptr;
    r.o = q.o ? q.o + off : nullptr;
    return r;
}

// One hop for the 32 queue slots [base, base + 32) of a warp (slots >= n idle): on hop 0 a
// slot is a pixel (camera ray from its seed), later a path read from `in`. Paths that go on
// are appended to `out` with one atomic on `out_count` per warp; paths that end add their
// sample to the canvas (render.cl:20-26). Every lane of the warp calls this together.
// FH: 1 = hop 0 (pixels), 2 = a later hop (queue), known at compile time so that each
// kernel carries only its own half (the kernel is bound by instruction fetch as much as by
// issue); 0 = decided by `first_hop` at run time.
template <int R, int FH, bool OOL = true>
__device__ __forceinline__ void wave_chunk(const StagedScene &s, uint32_t base, uint32_t n, bool first_hop,
                                           bool last_hop, uint32_t W, uint32_t H, uint32_t flags,
                                           float4 *__restrict__ canvas, uint32_t *__restrict__ seeds,
                                           const WaveQueue &in, const WaveQueue &out, uint32_t *out_count,
                                           LaneStats &st) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t i = base + lane;
    bool cont = false;
    typename PathOf<R>::T ray;
    uint32_t rng = 0, prev_hash = HASH_NEVER, pixel = 0;
    Col intensity = {1.0f, 1.0f, 1.0f};
    Col emission = {0.0f, 0.0f, 0.0f};
    const bool first = FH == 1 || (FH == 0 && first_hop);
    const bool full_warp = __ballot_sync(0xffffffffu, i < n) == 0xffffffffu;   // every lane has a path
    if (i < n) {
        if (first) {
            pixel = i;
            float px, py, size;
            pixel_pos(i % W, i / W, W, H, px, py, size);
            rng = seeds[i];
            ray = camera<R>(s, px, py, size, rng, flags);
        } else {
            const uint32_t k = in.o ? in.o[i] : i;
            ray = path_load<R>(in.p[k], in.v[k]);
            const float4 t = in.t[k], e = in.e[k];
            intensity.x = t.x; intensity.y = t.y; intensity.z = t.z;
            rng = __float_as_uint(t.w);
            emission.x = e.x; emission.y = e.y; emission.z = e.z;
            pixel = __float_as_uint(e.w);
            prev_hash = in.h[k];
        }
        bool hit;
        st.hops += 1;
        st.tests += s.n;
        const bool go = hop<R, OOL, true>(s, ray, rng, prev_hash, intensity, emission, hit, st.exact, full_warp);
        st.hits += hit ? 1 : 0;
        cont = go && !last_hop;
        if (!cont) {
            st.samples += 1;
            float4 c = canvas[pixel];
            c.x += emission.x; c.y += emission.y; c.z += emission.z; c.w += 1.0f;
            canvas[pixel] = c;
            seeds[pixel] = rng;
        }
    }
    const uint32_t want = __ballot_sync(0xffffffffu, cont);
    if (want) {
        const int leader = __ffs(want) - 1;
        uint32_t obase = 0;
        if (lane == (uint32_t)leader) obase = atomicAdd(out_count, (uint32_t)__popc(want));
        obase = __shfl_sync(0xffffffffu, obase, leader);
        if (cont) {
            const uint32_t j = obase + __popc(want & ((1u << lane) - 1u));
            path_store<R>(&out.p[j], &out.v[j], ray);
            out.t[j] = make_float4(intensity.x, intensity.y, intensity.z, __uint_as_float(rng));
            out.e[j] = make_float4(emission.x, emission.y, emission.z, __uint_as_float(pixel));
            out.h[j] = prev_hash;
        }
    }
}

// ctr[0]: slots taken by warps of this launch; ctr[1]: paths appended to `out`.
// in_count: paths in `in` (NULL for hop 0, which covers the W*H pixels).
template <int R, int FH>
__global__ void __launch_bounds__(128, FH == 1 ? HT_WAVE0_MINB : HT_WAVE_MINB) render_wave(
    const uint8_t *__restrict__ scene, size_t scene_size, uint32_t max_objects, int address_width,
    uint32_t W, uint32_t H, uint32_t hops, uint32_t hop_index, uint32_t flags, float4 *__restrict__ canvas,
    uint32_t *__restrict__ seeds, uint64_t *stats, uint32_t *err, WaveQueue in, const uint32_t *in_count,
    WaveQueue out, uint32_t *ctr) {
    extern __shared__ float4 smem[];
    __shared__ uint32_t s_hdr[2 + BLOCK_THREADS / 32];
    const uint32_t n = FH == 1 ? W * H : *reinterpret_cast<const volatile uint32_t *>(in_count);
    if (n == 0 || blockIdx.x * 128u >= n) return;   // nothing for this block: skip the staging
    const SceneSmem sm = carve_scene(smem, max_objects);
    StagedScene s;
    if (!stage_scene<R>(scene, scene_size, max_objects, address_width, err, s, sm, s_hdr)) return;

    const uint32_t lane = threadIdx.x & 31;
    const bool last = hop_index + 1 >= hops;
    LaneStats st;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&ctr[0], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        wave_chunk<R, FH>(s, base, n, FH == 1, last, W, H, flags, canvas, seeds, in, out, &ctr[1], st);
    }
    flush_lane_stats(stats, st);
}

// ============================================================================ coherence sort
// Between two hop depths of a hyperbolic pass the new queue gets a read order in which
// neighbouring slots hold rays that leave in similar directions from nearby points: from
// hop depth 2 on, rays start all over the scene, and the lanes of a warp otherwise carry
// unrelated candidate lists through the per-lane loops of the scan (ray-aware bound, exact
// tests), which then run with about 18 of 32 lanes active. Each path keeps its own state,
// so the order changes no result, only which paths share a warp.
//
// The order is a counting sort on a 16-bit key: direction cell (the cube face the
// direction points at, 4 x 4 cells per face: 96 cells) in the high bits, then a 3-bit
// cell per axis of the ray start (x, y, log z) over mean +- 2 sigma of that hop depth's
// queue in the previous pass, interleaved (Morton order); until a depth has been seen once,
// its cells are all zero and the sort goes by direction alone. Four launches per hop depth,
// sized for the largest queue and reading its length on the device: keys, their histogram
// and the position sums (k_sort_keys); the histogram's block totals (k_sort_scan_blocks);
// the exclusive scan into cursors, which also clears the histogram and turns the sums into
// the depth's next cells (k_sort_scan); the scatter of slot indices to their sorted
// positions (k_sort_scatter). Ties within a key land in atomic order. The work stays out of
// the hop kernel: that kernel is bound by instruction fetch as much as by issue, and the
// same steps inlined at its append site made every hop launch slower than these launches.
constexpr uint32_t SORT_BINS = 1u << 16;
constexpr uint32_t SORT_THREADS = 256;
constexpr uint32_t SORT_SCAN_BLOCKS = SORT_BINS / (4 * SORT_THREADS);   // 64: one uint4 of bins per thread
constexpr uint32_t SORT_DEPTH_WORDS = 8;   // per hop depth: 6 sums (double) / 6 cell bounds (float)
struct SortBuf {
    double *acc;        // per hop depth: sum and sum of squares of x, y, log z
    float *cut;         // per hop depth: lower bound of x, y, log z, then cells per unit
    uint32_t *hist;     // SORT_BINS counts
    uint32_t *bsum;     // SORT_SCAN_BLOCKS block totals of the histogram
    uint32_t *cursor;   // SORT_BINS next positions
    uint16_t *key;      // per slot
    uint32_t *perm;     // per sorted position: the slot
};
constexpr size_t sort_head_bytes(uint32_t hops) {   // acc, cut, hist: cleared at allocation
    return (size_t)hops * SORT_DEPTH_WORDS * (sizeof(double) + sizeof(float)) + sizeof(uint32_t) * SORT_BINS;
}
constexpr size_t sort_bytes(size_t slots, uint32_t hops) {
    return sort_head_bytes(hops) + sizeof(uint32_t) * (SORT_SCAN_BLOCKS + SORT_BINS) +
           ((sizeof(uint16_t) * slots + 15) & ~(size_t)15) + sizeof(uint32_t) * slots;
}
static SortBuf sort_buf_at(void *base, size_t slots, uint32_t hops) {
    SortBuf b;
    b.acc = reinterpret_cast<double *>(base);
    b.cut = reinterpret_cast<float *>(b.acc + (size_t)hops * SORT_DEPTH_WORDS);
    b.hist = reinterpret_cast<uint32_t *>(b.cut + (size_t)hops * SORT_DEPTH_WORDS);
    b.bsum = b.hist + SORT_BINS;
    b.cursor = b.bsum + SORT_SCAN_BLOCKS;
    b.key = reinterpret_cast<uint16_t *>(b.cursor + SORT_BINS);
    b.perm = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(b.key) +
                                          ((sizeof(uint16_t) * slots + 15) & ~(size_t)15));
    return b;
}

__device__ __forceinline__ float sort_logz(float z) { return z > 0.0f ? __logf(z) : 0.0f; }
__device__ __forceinline__ uint32_t sort_axis_cell(float u, float lo, float scale) {
    return (uint32_t)fminf(fmaxf((u - lo) * scale, 0.0f), 7.0f);   // NaN -> 0
}
__device__ __forceinline__ uint32_t spread3(uint32_t c) {   // bits b2 b1 b0 -> b2 0 0 b1 0 0 b0
    return (c & 1u) | ((c & 2u) << 2) | ((c & 4u) << 4);
}
__device__ __forceinline__ uint32_t sort_dir_cell(float4 v) {
    const float ax = fabsf(v.x), ay = fabsf(v.y), az = fabsf(v.z);
    uint32_t face;
    float m, a, b;
    if (ax >= ay && ax >= az) { face = v.x > 0.0f ? 1u : 0u; m = ax; a = v.y; b = v.z; }
    else if (ay >= az)        { face = v.y > 0.0f ? 3u : 2u; m = ay; a = v.z; b = v.x; }
    else                      { face = v.z > 0.0f ? 5u : 4u; m = az; a = v.x; b = v.y; }
    const float r = m > 0.0f ? __frcp_rn(m) : 0.0f;
    const uint32_t ia = (uint32_t)fminf(fmaxf((a * r + 1.0f) * 2.0f, 0.0f), 3.0f);
    const uint32_t ib = (uint32_t)fminf(fmaxf((b * r + 1.0f) * 2.0f, 0.0f), 3.0f);
    return face * 16u + ia * 4u + ib;   // < 96
}

// Keys (< 96 * 512 = 49152) of the `count` queued paths with the depth's cells `cut`, their
// histogram (lanes of a warp with equal keys add once) and the position sums into `acc`.
__global__ void __launch_bounds__(SORT_THREADS) k_sort_keys(const float4 *__restrict__ p, const float4 *__restrict__ v,
                                                           const uint32_t *count, const float *cut, double *acc,
                                                           uint16_t *__restrict__ key, uint32_t *hist) {
    const uint32_t n = *count;
    if (n == 0) return;
    const float lo0 = cut[0], lo1 = cut[1], lo2 = cut[2], sc0 = cut[3], sc1 = cut[4], sc2 = cut[5];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (SORT_THREADS / 32);
    float s[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t base = (blockIdx.x * (SORT_THREADS / 32) + (threadIdx.x >> 5)) * 32u; base < n; base += warps * 32u) {
        const uint32_t i = base + lane;
        const bool valid = i < n;
        uint32_t k = 0x10000u + lane;   // lanes past the end group alone
        if (valid) {
            const float4 q = p[i];
            const float l = sort_logz(q.z);
            s[0] += q.x; s[1] += q.x * q.x;
            s[2] += q.y; s[3] += q.y * q.y;
            s[4] += l;   s[5] += l * l;
            const uint32_t cx = sort_axis_cell(q.x, lo0, sc0);
            const uint32_t cy = sort_axis_cell(q.y, lo1, sc1);
            const uint32_t cz = sort_axis_cell(l, lo2, sc2);
            k = sort_dir_cell(v[i]) * 512u + (spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2));
            key[i] = (uint16_t)k;
        }
        const uint32_t grp = __match_any_sync(0xffffffffu, k);
        if (valid && lane == (uint32_t)(__ffs(grp) - 1)) atomicAdd(&hist[k], (uint32_t)__popc(grp));
    }
    __shared__ double part[SORT_THREADS / 32][6];
    const uint32_t warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double d = s[q];
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) part[warp][q] = d;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double d = 0.0;
        for (uint32_t w = 0; w < SORT_THREADS / 32; ++w) d += part[w][threadIdx.x];
        if (d != 0.0) atomicAdd(&acc[threadIdx.x], d);
    }
}

// Block totals of the histogram: block b sums bins [1024 b, 1024 b + 1024), one coalesced
// 16-byte load per thread.
__global__ void __launch_bounds__(SORT_THREADS) k_sort_scan_blocks(const uint32_t *hist, uint32_t *bsum) {
    const uint4 a = reinterpret_cast<const uint4 *>(hist)[(size_t)blockIdx.x * SORT_THREADS + threadIdx.x];
    uint32_t s = (a.x + a.y) + (a.z + a.w);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ uint32_t w[SORT_THREADS / 32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) w[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (uint32_t k = 0; k < SORT_THREADS / 32; ++k) t += w[k];
        bsum[blockIdx.x] = t;
    }
}

// Exclusive scan of the histogram into the cursors (block b: bins [1024 b, 1024 b + 1024),
// offset by the totals of the blocks before it), clearing the histogram. With `seg_base`,
// the histogram is cut into segments of `seg_bins` bins (a multiple of 1024), one per
// view, and the cursor value at each segment's first bin is recorded there, so that
// positions within a view's queue are cursor - seg_base. With `acc`, block 0 also turns the
// depth's position sums over its `count` paths into the cells the next pass keys it with
// (mean - 2 sigma, 8 cells over 4 sigma per axis) and clears the sums.
__global__ void __launch_bounds__(SORT_THREADS) k_sort_scan(uint32_t *hist, const uint32_t *bsum, uint32_t *cursor,
                                                           uint32_t seg_bins, uint32_t *seg_base, double *acc,
                                                           float *cut, const uint32_t *count) {
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    __shared__ uint32_t w[SORT_THREADS / 32];
    __shared__ uint32_t base_w[SORT_THREADS / 32];
    uint32_t before = 0;   // the totals of the blocks before this one
    for (uint32_t k = t; k < blockIdx.x; k += SORT_THREADS) before += bsum[k];
    for (int o = 16; o; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
    if (lane == 0) base_w[warp] = before;
    uint4 *h4 = reinterpret_cast<uint4 *>(hist) + (size_t)blockIdx.x * SORT_THREADS + t;
    const uint4 a = *h4;
    const uint32_t s4 = (a.x + a.y) + (a.z + a.w);
    uint32_t x = s4;   // inclusive scan within the warp
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) w[warp] = x;
    __syncthreads();
    uint32_t run = x - s4;
    for (uint32_t k = 0; k < SORT_THREADS / 32; ++k) run += base_w[k] + (k < warp ? w[k] : 0u);
    uint4 r;
    r.x = run;
    r.y = r.x + a.x;
    r.z = r.y + a.y;
    r.w = r.z + a.z;
    const size_t bin = ((size_t)blockIdx.x * SORT_THREADS + t) * 4;
    reinterpret_cast<uint4 *>(cursor)[(size_t)blockIdx.x * SORT_THREADS + t] = r;
    *h4 = make_uint4(0u, 0u, 0u, 0u);
    if (seg_base && bin % seg_bins == 0) seg_base[bin / seg_bins] = r.x;
    if (acc && blockIdx.x == 0 && t < 3) {
        const uint32_t n = *count;
        if (n) {
            const double mean = acc[2 * t] / (double)n;
            const double sd = sqrt(fmax(acc[2 * t + 1] / (double)n - mean * mean, 0.0));
            cut[t] = (float)(mean - 2.0 * sd);
            cut[3 + t] = sd > 0.0 ? (float)(2.0 / sd) : 0.0f;   // 8 cells over 4 sigma
        }
        acc[2 * t] = 0.0;
        acc[2 * t + 1] = 0.0;
    }
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_scatter(const uint16_t *__restrict__ key, const uint32_t *count,
                                                              uint32_t *cursor, uint32_t *__restrict__ perm) {
    const uint32_t n = *count;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (SORT_THREADS / 32);
    for (uint32_t base = (blockIdx.x * (SORT_THREADS / 32) + (threadIdx.x >> 5)) * 32u; base < n; base += warps * 32u) {
        const uint32_t i = base + lane;
        const bool valid = i < n;
        const uint32_t k = valid ? (uint32_t)key[i] : 0x10000u + lane;
        const uint32_t grp = __match_any_sync(0xffffffffu, k);
        const int leader = __ffs(grp) - 1;
        uint32_t at = 0;
        if (valid && lane == (uint32_t)leader) at = atomicAdd(&cursor[k], (uint32_t)__popc(grp));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (valid) perm[at + __popc(grp & ((1u << lane) - 1u))] = i;
    }
}

// ============================================================================ batch
struct BatchView {          // device copy of htc_view plus host-derived fields
    const uint8_t *scene;
    uint64_t scene_size;
    float4 *canvas;
    uint32_t *seeds;
    uint32_t width, height;
    int32_t recipe;
    uint32_t hops, flags;
    int32_t address_width;
    uint32_t passes;
    uint32_t max_objects;   // objects the scene buffer can hold
    uint64_t qoff;          // first slot of the view's region in the wavefront queues
};

// Wavefront form of the batch: one launch per (pass, hop depth) over every view. Each view
// has its own region of the two queues and its own append counter; the launch cuts the
// views' current paths into tiles of `tile_slots` (a block-wide prefix sum over the views'
// counts, expensive views first), blocks take tiles from a counter and stage a view's scene
// only when it changes, and warps take 32 slots of the tile at a time (wave_chunk). A
// view's paths therefore run exactly as in render_wave, and every view's canvas and seeds
// are bit-identical to rendering it alone.
//   cnt[h * n_views + v]: paths of view v appended by hop h of this pass;
//   grab: tiles taken by the blocks of one launch (a word of its own per launch of a pass).
__device__ __forceinline__ uint32_t batch_wave_count(const BatchView &v, uint32_t vi, uint32_t pass, uint32_t h,
                                                     const uint32_t *cnt, uint32_t n_views) {
    if (pass >= v.passes || h >= v.hops) return 0;
    if (h == 0) return v.width * v.height;
    return *reinterpret_cast<const volatile uint32_t *>(&cnt[(h - 1) * n_views + vi]);
}

// RF = 0 serves views of either recipe (a runtime branch per tile); RF = RECIPE_HY or
// RECIPE_EU compiles one recipe only (its views alone in `order`), with fewer registers.
template <int RF, int FH>
__global__ void __launch_bounds__(128, RF ? HT_BATCH_MINB : HT_PERSIST_MINB) render_batch_wave(
    const BatchView *__restrict__ views, const uint32_t *__restrict__ order, uint32_t n_order, uint32_t n_views,
    uint32_t pass, uint32_t h, uint32_t tile_slots, uint32_t smem_objects, WaveQueue in, WaveQueue out,
    uint32_t *cnt, uint32_t *grab, uint64_t *stats, uint32_t *err, uint32_t n_sorted) {
    extern __shared__ float4 smem[];
    __shared__ uint32_t s_hdr[2 + BLOCK_THREADS / 32];
    __shared__ uint32_t s_tile, s_next, s_total, s_tsize;
    __shared__ int s_staged_view, s_staged_ok;
    const SceneSmem sm = carve_scene(smem, smem_objects);
    uint32_t *s_pref = reinterpret_cast<uint32_t *>(sm.end);   // n_order + 1 tile offsets
    const uint32_t tid = threadIdx.x, lane = tid & 31;

    // tiles of every view at this hop, in `order`, as a prefix sum. The tile size adapts to
    // the launch: about 16 tiles per block when the paths are few (a multiple of 128 slots,
    // so the four warps of a block take equal shares; at least one chunk per warp),
    // `tile_slots` when they are many, so a launch ends with short tiles.
    for (uint32_t i = tid; i < n_order; i += blockDim.x) {
        const uint32_t vi = order[i];
        s_pref[i + 1] = batch_wave_count(views[vi], vi, pass, h, cnt, n_views);
    }
    if (tid == 0) {
        s_pref[0] = 0;
        s_staged_view = -1;
    }
    __syncthreads();
    if (tid < 32) {
        uint64_t paths = 0;
        for (uint32_t i = lane; i < n_order; i += 32) paths += s_pref[i + 1];
        for (int off = 16; off > 0; off >>= 1) paths += __shfl_xor_sync(0xffffffffu, paths, off);
        uint64_t per = (paths / (16ull * gridDim.x) + 127) & ~127ull;
        if (per < 128) per = 128;
        if (per > tile_slots) per = tile_slots;
        if (lane == 0) s_tsize = (uint32_t)per;
    }
    __syncthreads();
    const uint32_t tile = s_tsize;
    for (uint32_t i = tid; i < n_order; i += blockDim.x) s_pref[i + 1] = (s_pref[i + 1] + tile - 1) / tile;
    __syncthreads();
    if (tid < 32) {
        uint32_t carry = 0;
        for (uint32_t b0 = 0; b0 < n_order; b0 += 32) {
            const uint32_t i = b0 + lane;
            uint32_t x = i < n_order ? s_pref[i + 1] : 0;
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
                if (lane >= (uint32_t)off) x += y;
            }
            if (i < n_order) s_pref[i + 1] = x + carry;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) s_total = carry;
    }
    __syncthreads();
    const uint32_t total = s_total;
    StagedScene s;
    s.n = 0;
    LaneStats st;
    for (;;) {
        __syncthreads();
        if (tid == 0) {
            s_tile = total ? atomicAdd(grab, 1u) : 0u;
            s_next = 0;
        }
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= total) break;
        uint32_t lo = 0, hi = n_order - 1;   // the last view whose first tile is <= t
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (s_pref[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const uint32_t vi = order[lo];
        const BatchView &v = views[vi];
        const uint32_t n = batch_wave_count(v, vi, pass, h, cnt, n_views);
        const uint32_t first = (t - s_pref[lo]) * tile;
        const uint32_t count = min(tile, n - first);
        const int32_t recipe = RF ? RF : v.recipe;
        if ((int)vi != s_staged_view) {
            bool ok;
            if (recipe == RECIPE_HY)
                ok = stage_scene<RECIPE_HY>(v.scene, v.scene_size, min(v.max_objects, smem_objects), v.address_width,
                                            err, s, sm, s_hdr);
            else
                ok = stage_scene<RECIPE_EU>(v.scene, v.scene_size, min(v.max_objects, smem_objects), v.address_width,
                                            err, s, sm, s_hdr);
            __syncthreads();
            if (tid == 0) {
                s_staged_view = (int)vi;
                s_staged_ok = ok ? 1 : 0;
            }
            __syncthreads();
        }
        if (!s_staged_ok) continue;
        // the first n_sorted views of `order` read a tile's paths through their sorted order
        // (view-relative slots), the others in queue order
        const bool sorted = in.o != nullptr && lo < n_sorted;
        WaveQueue vin = wave_at(in, sorted ? v.qoff : v.qoff + first);
        vin.o = sorted ? in.o + v.qoff + first : nullptr;
        const WaveQueue vout = wave_at(out, v.qoff);
        const bool first_hop = FH == 1, last_hop = h + 1 >= v.hops;
        uint32_t *out_count = &cnt[h * n_views + vi];
        float4 *canvas = v.canvas;
        uint32_t *seeds = v.seeds;
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&s_next, 32u);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= count) break;
            // slots are pixel numbers on hop 0, tile-relative queue slots later
            const uint32_t b0 = first_hop ? first + base : base, n0 = first_hop ? first + count : count;
            if (recipe == RECIPE_HY)
                wave_chunk<RECIPE_HY, FH, false>(s, b0, n0, first_hop, last_hop, v.width, v.height, v.flags, canvas, seeds, vin,
                                      vout, out_count, st);
            else
                wave_chunk<RECIPE_EU, FH, false>(s, b0, n0, first_hop, last_hop, v.width, v.height, v.flags, canvas, seeds, vin,
                                      vout, out_count, st);
        }
    }
    flush_lane_stats(stats, st);
}

// ============================================================================ batch: coherence sort
// The coherence sort of the single-view wavefronts, per view: the first `n_seg` hyperbolic
// views of the launch order (the most expensive ones; at most BATCH_SORT_VIEWS) each get a
// segment of SORT_BINS_VIEW bins of one histogram, and their queued paths a read order
// within their own queue region. Position cells are kept per view and hop depth.
constexpr uint32_t BATCH_SORT_VIEWS = 128;
constexpr uint32_t SORT_BINS_VIEW = 96u * 512u;   // 48 blocks of the scan per view
struct BatchSortBuf {
    double *acc;        // per view and hop depth: 6 position sums
    float *cut;         // per view and hop depth: 6 cell bounds
    uint32_t *hist;     // BATCH_SORT_VIEWS x SORT_BINS_VIEW
    uint32_t *bsum;     // scan block totals
    uint32_t *cursor;   // as hist
    uint32_t *seg_base; // per segment: cursor value at its first bin
    uint16_t *key;      // per queue slot
    uint32_t *perm;     // per queue slot: view-relative slot in sorted order
};
constexpr size_t batch_sort_head_bytes(uint32_t max_views, uint32_t hops) {   // acc, cut, hist
    return (size_t)max_views * hops * SORT_DEPTH_WORDS * (sizeof(double) + sizeof(float)) +
           sizeof(uint32_t) * (size_t)BATCH_SORT_VIEWS * SORT_BINS_VIEW;
}
constexpr size_t batch_sort_bytes(uint32_t max_views, uint32_t hops, uint64_t slots) {
    return batch_sort_head_bytes(max_views, hops) +
           sizeof(uint32_t) * ((size_t)BATCH_SORT_VIEWS * SORT_BINS_VIEW / 1024 + (size_t)BATCH_SORT_VIEWS * SORT_BINS_VIEW +
                               BATCH_SORT_VIEWS) +
           ((sizeof(uint16_t) * slots + 15) & ~(size_t)15) + sizeof(uint32_t) * slots;
}
static BatchSortBuf batch_sort_at(void *base, uint32_t max_views, uint32_t hops, uint64_t slots) {
    BatchSortBuf b;
    b.acc = reinterpret_cast<double *>(base);
    b.cut = reinterpret_cast<float *>(b.acc + (size_t)max_views * hops * SORT_DEPTH_WORDS);
    b.hist = reinterpret_cast<uint32_t *>(b.cut + (size_t)max_views * hops * SORT_DEPTH_WORDS);
    b.bsum = b.hist + (size_t)BATCH_SORT_VIEWS * SORT_BINS_VIEW;
    b.cursor = b.bsum + (size_t)BATCH_SORT_VIEWS * SORT_BINS_VIEW / 1024;
    b.seg_base = b.cursor + (size_t)BATCH_SORT_VIEWS * SORT_BINS_VIEW;
    b.key = reinterpret_cast<uint16_t *>(b.seg_base + BATCH_SORT_VIEWS);
    b.perm = reinterpret_cast<uint32_t *>(reinterpret_cast<uint8_t *>(b.key) + ((sizeof(uint16_t) * slots + 15) & ~(size_t)15));
    return b;
}

// The views' path counts at queue depth h, as an exclusive prefix over the first n_seg
// entries of `order` (s_pref: n_seg + 1 words), and the segment of the path numbered g.
__device__ __forceinline__ void bsort_prefix(const BatchView *views, const uint32_t *order, uint32_t n_seg,
                                             uint32_t n_views, uint32_t pass, uint32_t h, const uint32_t *cnt,
                                             uint32_t *s_pref) {
    for (uint32_t i = threadIdx.x; i < n_seg; i += blockDim.x) {
        const uint32_t vi = order[i];
        s_pref[i + 1] = batch_wave_count(views[vi], vi, pass, h, cnt, n_views);
    }
    if (threadIdx.x == 0) s_pref[0] = 0;
    __syncthreads();
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        uint32_t carry = 0;
        for (uint32_t b0 = 0; b0 < n_seg; b0 += 32) {
            const uint32_t i = b0 + lane;
            uint32_t x = i < n_seg ? s_pref[i + 1] : 0;
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
                if (lane >= (uint32_t)off) x += y;
            }
            if (i < n_seg) s_pref[i + 1] = x + carry;
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
    }
    __syncthreads();
}
__device__ __forceinline__ uint32_t bsort_segment(const uint32_t *s_pref, uint32_t n_seg, uint32_t g) {
    uint32_t lo = 0, hi = n_seg - 1;   // the last segment whose first path is <= g
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (s_pref[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Keys, histogram and position sums of the sorted views' paths at queue depth h. Block b
// takes a contiguous range of the paths numbered over the views in order, so its position
// sums (shared memory, n_seg x 6 floats) touch few views.
__global__ void __launch_bounds__(SORT_THREADS) k_bsort_keys(const BatchView *__restrict__ views,
                                                            const uint32_t *__restrict__ order, uint32_t n_seg,
                                                            uint32_t n_views, uint32_t pass, uint32_t h,
                                                            const uint32_t *cnt, uint32_t hops_max,
                                                            const float4 *__restrict__ qp, const float4 *__restrict__ qv,
                                                            const float *cut, double *acc, uint16_t *__restrict__ key,
                                                            uint32_t *hist) {
    extern __shared__ uint32_t s_pref[];                                  // n_seg + 1
    float *s_acc = reinterpret_cast<float *>(s_pref + n_seg + 1);         // n_seg x 6
    for (uint32_t i = threadIdx.x; i < 6 * n_seg; i += blockDim.x) s_acc[i] = 0.0f;
    bsort_prefix(views, order, n_seg, n_views, pass, h, cnt, s_pref);
    const uint32_t total = s_pref[n_seg];
    const uint32_t per = ((total + gridDim.x - 1) / gridDim.x + 31) & ~31u;
    const uint32_t g0 = blockIdx.x * per, g1 = min(total, g0 + per);
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t base = g0 + (threadIdx.x >> 5) * 32u; base < g1; base += SORT_THREADS) {
        const uint32_t g = base + lane;
        const bool valid = g < g1;
        uint32_t bin = 0x80000000u + lane;   // lanes past the end group alone
        uint32_t sg = 0;
        float m[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (valid) {
            sg = bsort_segment(s_pref, n_seg, g);
            const uint32_t vi = order[sg];
            const uint64_t slot = views[vi].qoff + (g - s_pref[sg]);
            const float *c = cut + ((size_t)vi * hops_max + h) * SORT_DEPTH_WORDS;
            const float4 q = qp[slot];
            const float l = sort_logz(q.z);
            m[0] = q.x; m[1] = q.x * q.x;
            m[2] = q.y; m[3] = q.y * q.y;
            m[4] = l;   m[5] = l * l;
            const uint32_t cx = sort_axis_cell(q.x, c[0], c[3]);
            const uint32_t cy = sort_axis_cell(q.y, c[1], c[4]);
            const uint32_t cz = sort_axis_cell(l, c[2], c[5]);
            const uint32_t k = sort_dir_cell(qv[slot]) * 512u + (spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2));
            key[slot] = (uint16_t)k;
            bin = sg * SORT_BINS_VIEW + k;
        }
        const uint32_t grp = __match_any_sync(0xffffffffu, bin);
        if (valid && lane == (uint32_t)(__ffs(grp) - 1)) atomicAdd(&hist[bin], (uint32_t)__popc(grp));
        // position sums: one add per value when the warp's paths are one view's (lane 0 is
        // always a path here), else one per lane
        const uint32_t sg0 = __shfl_sync(0xffffffffu, sg, 0);
        if (__all_sync(0xffffffffu, !valid || sg == sg0)) {
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                for (int o = 16; o; o >>= 1) m[q] += __shfl_xor_sync(0xffffffffu, m[q], o);
                if (lane == 0) atomicAdd(&s_acc[6 * sg0 + q], m[q]);
            }
        } else if (valid) {
#pragma unroll
            for (int q = 0; q < 6; ++q) atomicAdd(&s_acc[6 * sg + q], m[q]);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 6 * n_seg; i += blockDim.x)
        if (s_acc[i] != 0.0f)
            atomicAdd(&acc[((size_t)order[i / 6] * hops_max + h) * SORT_DEPTH_WORDS + i % 6], (double)s_acc[i]);
}

// Sorted positions of the sorted views' paths at queue depth h: perm[qoff + position] =
// view-relative slot. Block 0 first turns each view's position sums into its cells for the
// next pass (the keys of this pass are already made) and clears the sums.
__global__ void __launch_bounds__(SORT_THREADS) k_bsort_scatter(const BatchView *__restrict__ views,
                                                               const uint32_t *__restrict__ order, uint32_t n_seg,
                                                               uint32_t n_views, uint32_t pass, uint32_t h,
                                                               const uint32_t *cnt, uint32_t hops_max,
                                                               const uint16_t *__restrict__ key, uint32_t *cursor,
                                                               const uint32_t *seg_base, double *acc, float *cut,
                                                               uint32_t *__restrict__ perm) {
    extern __shared__ uint32_t s_pref[];   // n_seg + 1
    bsort_prefix(views, order, n_seg, n_views, pass, h, cnt, s_pref);
    if (blockIdx.x == 0)
        for (uint32_t i = threadIdx.x; i < 3 * n_seg; i += blockDim.x) {
            const uint32_t sg = i / 3, ax = i % 3;
            const size_t d = ((size_t)order[sg] * hops_max + h) * SORT_DEPTH_WORDS;
            const uint32_t n = s_pref[sg + 1] - s_pref[sg];
            if (n) {
                const double mean = acc[d + 2 * ax] / (double)n;
                const double sd = sqrt(fmax(acc[d + 2 * ax + 1] / (double)n - mean * mean, 0.0));
                cut[d + ax] = (float)(mean - 2.0 * sd);
                cut[d + 3 + ax] = sd > 0.0 ? (float)(2.0 / sd) : 0.0f;
            }
            acc[d + 2 * ax] = 0.0;
            acc[d + 2 * ax + 1] = 0.0;
        }
    const uint32_t total = s_pref[n_seg];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (SORT_THREADS / 32);
    for (uint32_t base = (blockIdx.x * (SORT_THREADS / 32) + (threadIdx.x >> 5)) * 32u; base < total; base += warps * 32u) {
        const uint32_t g = base + lane;
        const bool valid = g < total;
        uint32_t bin = 0x80000000u + lane, sg = 0, j = 0;
        uint64_t qoff = 0;
        if (valid) {
            sg = bsort_segment(s_pref, n_seg, g);
            j = g - s_pref[sg];
            qoff = views[order[sg]].qoff;
            bin = sg * SORT_BINS_VIEW + key[qoff + j];
        }
        const uint32_t grp = __match_any_sync(0xffffffffu, bin);
        const int leader = __ffs(grp) - 1;
        uint32_t at = 0;
        if (valid && lane == (uint32_t)leader) at = atomicAdd(&cursor[bin], (uint32_t)__popc(grp)) - seg_base[sg];
        at = __shfl_sync(0xffffffffu, at, leader);
        if (valid) perm[qoff + at + __popc(grp & ((1u << lane) - 1u))] = j;
    }
}

// ============================================================================ double_support
// A scene serialized with double_support (types/src/config.rs:38-43) stores every f64 field
// in 8 bytes, and a primitive vector or matrix of f64 is aligned to its own size
// (types/src/primitive/scalar.rs:186-215, types/src/primitive/matrix.rs:171-209); colors stay
// f32. The reference then builds its kernel with real = double (processing/src/render.rs:50).
// This path narrows such a scene once per render call into the f32 layout the kernels read,
// rounding each f64 to the nearest f32 -- the value the reference's own serializer writes for
// the same scene without double_support (`*self as f32`, scalar.rs:198-207) -- and then
// transports in FP32 as for any other scene: a double_support scene renders bit for bit as
// its f32 serialization does. The field tables follow the layouts hypertrace_b200/types.py
// derives (Moebius 8 reals, Shift3 3 + 1, Rotation3 4, fov and portions 1).
struct NarrowField { uint16_t src, dst; uint8_t kind, n; };   // kind: 0 = n f64 -> f32, 1 = n words, 2 = usize
struct NarrowLayout {
    uint32_t src_objects, src_stride, dst_objects, dst_stride, src_count, dst_count;
    uint32_t n_header, n_object;
    NarrowField header[5], object[8];
};
__constant__ NarrowLayout c_narrow[2] = {
    // HTC_RECIPE_HY: view map, fov, background | map, diffuse color / portion, specular portion,
    // emission, luminous portion, shape index
    {256, 192, 128, 128, 192, 96, 3, 7,
     {{0, 0, 0, 8}, {64, 32, 0, 1}, {128, 64, 1, 3}},
     {{0, 0, 0, 8}, {64, 32, 1, 3}, {80, 48, 0, 1}, {96, 64, 0, 1}, {112, 80, 1, 3}, {128, 96, 0, 1}, {144, 112, 2, 1}}},
    // HTC_RECIPE_EU: view shift, rotation, fov, background | shift, rotation, diffuse color /
    // portion, specular portion, emission, luminous portion, shape index
    {160, 160, 80, 128, 128, 64, 4, 8,
     {{0, 0, 0, 3}, {32, 16, 0, 4}, {64, 32, 0, 1}, {96, 48, 1, 3}},
     {{0, 0, 0, 3}, {32, 16, 0, 4}, {64, 32, 1, 3}, {80, 48, 0, 1}, {96, 64, 0, 1}, {112, 80, 1, 3}, {128, 96, 0, 1},
      {144, 112, 2, 1}}},
};
constexpr uint32_t NARROW_SRC_OBJECTS[2] = {256, 160}, NARROW_SRC_STRIDE[2] = {192, 160};

__device__ __forceinline__ void narrow_fields(const uint8_t *src, uint8_t *dst, const NarrowField *f, uint32_t nf,
                                              int usize_bytes) {
    for (uint32_t i = 0; i < nf; ++i) {
        const NarrowField fd = f[i];
        if (fd.kind == 0) {
            const double *a = reinterpret_cast<const double *>(src + fd.src);
            float *b = reinterpret_cast<float *>(dst + fd.dst);
            for (uint32_t j = 0; j < fd.n; ++j) b[j] = __double2float_rn(a[j]);
        } else {
            const uint32_t words = fd.kind == 1 ? fd.n : (uint32_t)usize_bytes / 4u;
            const uint32_t *a = reinterpret_cast<const uint32_t *>(src + fd.src);
            uint32_t *b = reinterpret_cast<uint32_t *>(dst + fd.dst);
            for (uint32_t j = 0; j < words; ++j) b[j] = a[j];
        }
    }
}
// One thread per record (record 0 = the header, record 1 + i = object i). An object count the
// source buffer cannot hold (or the destination was not sized for) is written as all ones,
// which the render's own staging rejects as a scene error.
__global__ void k_narrow_scene(int li, const uint8_t *__restrict__ src, uint64_t src_size, uint8_t *__restrict__ dst,
                               uint32_t dst_capacity, int usize_bytes) {
    const NarrowLayout &L = c_narrow[li];
    const uint32_t count_lo = *reinterpret_cast<const uint32_t *>(src + L.src_count);
    const uint32_t count_hi = usize_bytes == 8 ? *reinterpret_cast<const uint32_t *>(src + L.src_count + 4) : 0u;
    const uint64_t holds = src_size >= L.src_objects ? (src_size - L.src_objects) / L.src_stride : 0u;
    const bool ok = count_hi == 0 && count_lo <= holds && count_lo <= dst_capacity;
    const uint32_t n = ok ? count_lo : 0u;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += gridDim.x * blockDim.x) {
        if (r == 0) {
            narrow_fields(src, dst, L.header, L.n_header, usize_bytes);
            uint32_t *c = reinterpret_cast<uint32_t *>(dst + L.dst_count);
            c[0] = ok ? count_lo : 0xFFFFFFFFu;
            if (usize_bytes == 8) c[1] = ok ? 0u : 0xFFFFFFFFu;
        } else {
            narrow_fields(src + L.src_objects + (size_t)(r - 1) * L.src_stride,
                          dst + L.dst_objects + (size_t)(r - 1) * L.dst_stride, L.object, L.n_object, usize_bytes);
        }
    }
}

// ============================================================================ post
// pow(max(x, 0), gamma) is evaluated in FP64 and rounded once (the host libm's powf is
// within a fraction of an ulp of that).
__device__ __forceinline__ float gamma1(float x, float g) {
    float m = fmaxf(x, 0.0f);
    return (float)pow((double)m, (double)g);
}
__device__ __forceinline__ uint8_t pack1(float x) {
    float c = fminf(fmaxf(x, 0.0f), 1.0f);
    return (uint8_t)__float2uint_rz(255.0f * c);
}

__global__ void k_extract(uint32_t n, float passes, const float4 *__restrict__ canvas, float4 *__restrict__ image) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = canvas[i];
        image[i] = make_float4(c.x / passes, c.y / passes, c.z / passes, c.w / passes);
    }
}
__global__ void k_gamma(uint32_t n, float g, const float4 *__restrict__ in, float4 *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = in[i];
        out[i] = make_float4(gamma1(c.x, g), gamma1(c.y, g), gamma1(c.z, g), gamma1(c.w, g));
    }
}
__global__ void k_pack(uint32_t n, const float4 *__restrict__ in, uchar4 *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = in[i];
        out[i] = make_uchar4(pack1(c.x), pack1(c.y), pack1(c.z), pack1(c.w));
    }
}
// Per-pixel initial RNG states: seed_i = fmix32(global_seed ^ fmix32(i + offset)), MurmurHash3's
// 32-bit finaliser (the harness seeds; the reference fills the buffer from a host SmallRng,
// processing/src/canvas.rs:193-195, and its kernel only consumes it).
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
__global__ void k_fill_seeds(uint32_t n, uint32_t global_seed, uint32_t offset, uint32_t *__restrict__ seeds) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        seeds[i] = fmix32(global_seed ^ fmix32(i + offset));
}

__global__ void k_extract_gamma_pack(uint32_t n, float passes, float g, const float4 *__restrict__ canvas,
                                     uchar4 *__restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = canvas[i];
        out[i] = make_uchar4(pack1(gamma1(c.x / passes, g)), pack1(gamma1(c.y / passes, g)),
                             pack1(gamma1(c.z / passes, g)), pack1(gamma1(c.w / passes, g)));
    }
}

// ============================================================================ calibration
// FP32 FMA throughput probe: independent FMA chains per thread, enough warps to fill every
// scheduler. 2 flops per FMA; the result is written so nothing is dead code.
__global__ void __launch_bounds__(256) k_fma_probe(float *out, int iters) {
    float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
    float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
            a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

// ============================================================================ C ABI
static int check_program(const htc_program *p) {
    if (!p) return fail(HTC_ERR_INVALID, "program is NULL");
    return HTC_OK;
}
static size_t smem_bytes(uint32_t max_objects) {   // carve_scene's layout
    return scene_win_offset(max_objects) + 2u * 16u * BLOCK_THREADS;
}
static uint32_t objects_capacity(int recipe, size_t scene_size) {
    const size_t hdr = recipe == HTC_RECIPE_HY ? Layout<RECIPE_HY>::OBJECTS : Layout<RECIPE_EU>::OBJECTS;
    if (scene_size < hdr) return 0;
    size_t n = (scene_size - hdr) / OBJ_STRIDE;
    return n > 0xFFFFFFu ? 0xFFFFFFu : (uint32_t)n;
}

template <int R>
static int set_smem_attr(size_t smem) {
    HTC_CUDA(cudaFuncSetAttribute(render_plain<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HTC_CUDA(cudaFuncSetAttribute(render_persistent<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HTC_CUDA(cudaFuncSetAttribute(render_wave<R, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    HTC_CUDA(cudaFuncSetAttribute(render_wave<R, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return HTC_OK;
}

static int validate_render_args(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                                const float *canvas, const uint32_t *seeds, uint32_t *max_objects, size_t *smem) {
    int rc = check_program(p);
    if (rc) return rc;
    if (W == 0 || H == 0) return fail(HTC_ERR_INVALID, "canvas width and height must be positive");
    if ((uint64_t)W * (uint64_t)H >= 0xFFFFFFFFull) return fail(HTC_ERR_INVALID, "canvas too large (W*H must fit in 32 bits)");
    if (!scene || !canvas || !seeds) return fail(HTC_ERR_INVALID, "scene, canvas and seeds must be device pointers");
    if ((reinterpret_cast<uintptr_t>(scene) & 15u) != 0 || (reinterpret_cast<uintptr_t>(canvas) & 15u) != 0)
        return fail(HTC_ERR_INVALID, "scene and canvas must be 16-byte aligned");
    *max_objects = objects_capacity(p->recipe, scene_size);
    if (scene_size < (p->recipe == HTC_RECIPE_HY ? 128u : 80u))
        return fail(HTC_ERR_SCENE, "scene buffer is smaller than the scene header");
    *smem = smem_bytes(*max_objects);
    if (*smem > (size_t)p->max_smem)
        return fail(HTC_ERR_UNSUPPORTED, "scene has more objects than shared memory can stage");
    return HTC_OK;
}

// A program around a generic scene kernel: error word only (no staging, no queue).
static int wrap_generic(GenericProgram *g, int recipe, uint32_t light_hops, int address_width, uint32_t flags,
                        htc_program **out) {
    htc_program *p = new htc_program();
    p->recipe = recipe;
    p->hops = light_hops;
    p->address_width = address_width;
    p->flags = flags;
    p->generic = g;
    cudaError_t e = cudaMalloc(&p->d_err, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(p->d_err, 0, sizeof(uint32_t));
    if (e != cudaSuccess) {
        if (p->d_err) cudaFree(p->d_err);
        generic_program_destroy(g);
        delete p;
        return cuda_fail(e, "htc_program_create");
    }
    *out = p;
    return HTC_OK;
}

extern "C" {

const char *htc_last_error(void) { return g_last_error.c_str(); }
int htc_version(void) { return 10000; }

int htc_device_count(int *count) {
    if (!count) return fail(HTC_ERR_INVALID, "count is NULL");
    HTC_CUDA(cudaGetDeviceCount(count));
    return HTC_OK;
}
int htc_set_device(int device) {
    HTC_CUDA(cudaSetDevice(device));
    return HTC_OK;
}

int htc_program_create(int recipe, uint32_t light_hops, int address_width, int double_support,
                       uint32_t flags, htc_program **out) {
    if (!out) return fail(HTC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (recipe != HTC_RECIPE_HY && recipe != HTC_RECIPE_EU && recipe != HTC_RECIPE_HY_TILED &&
        recipe != HTC_RECIPE_EU_GRADIENT)
        return fail(HTC_ERR_UNSUPPORTED, "unknown scene recipe");
    if (light_hops == 0) return fail(HTC_ERR_INVALID, "light_hops must be positive");
    if (address_width != 32 && address_width != 64) return fail(HTC_ERR_INVALID, "address_width must be 32 or 64");
    if (flags & ~(HTC_FLAG_JITTER_YX | HTC_FLAG_NO_SORT)) return fail(HTC_ERR_INVALID, "unknown program flags");
    if (double_support && recipe != HTC_RECIPE_HY && recipe != HTC_RECIPE_EU)
        return fail(HTC_ERR_UNSUPPORTED, "double_support scenes are served for HTC_RECIPE_HY and HTC_RECIPE_EU only");
    if (recipe == HTC_RECIPE_HY_TILED || recipe == HTC_RECIPE_EU_GRADIENT) {
        GenericProgram *g = nullptr;
        int rc = generic_program_create(recipe, address_width, &g);
        if (rc) return rc;
        return wrap_generic(g, recipe, light_hops, address_width, flags, out);
    }
    int dev = 0;
    HTC_CUDA(cudaGetDevice(&dev));
    htc_program *p = new htc_program();
    p->recipe = recipe;
    p->hops = light_hops;
    p->address_width = address_width;
    p->flags = flags;
    p->double_support = double_support ? 1 : 0;
    cudaError_t e = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_err, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_queue, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(p->d_err, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(p->d_queue, 0, 2 * sizeof(uint32_t));
    if (e != cudaSuccess) {
        if (p->d_err) cudaFree(p->d_err);
        if (p->d_queue) cudaFree(p->d_queue);
        delete p;
        return cuda_fail(e, "htc_program_create");
    }
    p->max_smem -= 1024;   // static shared memory of the kernels
    int rc = recipe == HTC_RECIPE_HY ? set_smem_attr<RECIPE_HY>(p->max_smem) : set_smem_attr<RECIPE_EU>(p->max_smem);
    if (rc) {
        cudaFree(p->d_err);
        cudaFree(p->d_queue);
        delete p;
        return rc;
    }
    *out = p;
    return HTC_OK;
}

void htc_program_destroy(htc_program *p) {
    if (!p) return;
    cudaFree(p->d_err);
    if (p->d_queue) cudaFree(p->d_queue);
    if (p->wave_buf) cudaFree(p->wave_buf);
    if (p->d_wave_ctr) cudaFree(p->d_wave_ctr);
    if (p->sort_buf) cudaFree(p->sort_buf);
    if (p->narrow_buf) cudaFree(p->narrow_buf);
    if (p->generic) generic_program_destroy(p->generic);
    delete p;
}

int htc_program_build(const char *scene_type, uint32_t light_hops, int address_width, uint32_t flags, char *log,
                      size_t log_len, htc_program **out) {
    if (!out) return fail(HTC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!scene_type || !scene_type[0]) return fail(HTC_ERR_INVALID, "scene_type is empty");
    if (light_hops == 0) return fail(HTC_ERR_INVALID, "light_hops must be positive");
    if (address_width != 32 && address_width != 64) return fail(HTC_ERR_INVALID, "address_width must be 32 or 64");
    if (flags & ~HTC_FLAG_JITTER_YX) return fail(HTC_ERR_INVALID, "unknown program flags");
    GenericProgram *g = nullptr;
    int rc = generic_program_build(scene_type, address_width, log, log_len, &g);
    if (rc) return rc;
    return wrap_generic(g, HTC_RECIPE_CUSTOM, light_hops, address_width, flags, out);
}

int htc_program_static_size(const htc_program *p, uint64_t *bytes) {
    int rc = check_program(p);
    if (rc) return rc;
    if (!bytes) return fail(HTC_ERR_INVALID, "bytes is NULL");
    if (p->generic) *bytes = generic_min_size(p->generic);
    else if (p->double_support) *bytes = NARROW_SRC_OBJECTS[p->recipe == HTC_RECIPE_HY ? 0 : 1];
    else *bytes = p->recipe == HTC_RECIPE_HY ? Layout<RECIPE_HY>::OBJECTS : Layout<RECIPE_EU>::OBJECTS;
    return HTC_OK;
}

int htc_program_check(htc_program *p, void *stream) {
    int rc = check_program(p);
    if (rc) return rc;
    uint32_t err = 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    HTC_CUDA(cudaMemcpyAsync(&err, p->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    HTC_CUDA(cudaStreamSynchronize(st));
    if (err) {
        HTC_CUDA(cudaMemsetAsync(p->d_err, 0, sizeof(uint32_t), st));
        HTC_CUDA(cudaStreamSynchronize(st));
        if (err & ERR_SCENE) return fail(HTC_ERR_SCENE, "scene bytes failed validation (object count or shape index out of range)");
        return fail(HTC_ERR_SCENE, "device error word set");
    }
    return HTC_OK;
}

int htc_malloc(void **dptr, size_t bytes) {
    if (!dptr) return fail(HTC_ERR_INVALID, "dptr is NULL");
    HTC_CUDA(cudaMalloc(dptr, bytes ? bytes : 1));
    return HTC_OK;
}
int htc_free(void *dptr) {
    HTC_CUDA(cudaFree(dptr));
    return HTC_OK;
}
int htc_memcpy_htod(void *dst, const void *src, size_t bytes, void *stream) {
    HTC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, reinterpret_cast<cudaStream_t>(stream)));
    return HTC_OK;
}
int htc_memcpy_dtoh(void *dst, const void *src, size_t bytes, void *stream) {
    HTC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, reinterpret_cast<cudaStream_t>(stream)));
    return HTC_OK;
}
int htc_memset(void *dst, int value, size_t bytes, void *stream) {
    HTC_CUDA(cudaMemsetAsync(dst, value, bytes, reinterpret_cast<cudaStream_t>(stream)));
    return HTC_OK;
}
int htc_stream_sync(void *stream) {
    HTC_CUDA(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
    return HTC_OK;
}

// Argument checks and launch of a generic scene program (passes samples per pixel).
static int render_generic_program(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                                  float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats, void *stream) {
    if (W == 0 || H == 0) return fail(HTC_ERR_INVALID, "canvas width and height must be positive");
    if ((uint64_t)W * (uint64_t)H >= 0xFFFFFFFFull) return fail(HTC_ERR_INVALID, "canvas too large (W*H must fit in 32 bits)");
    if (!scene || !canvas || !seeds) return fail(HTC_ERR_INVALID, "scene, canvas and seeds must be device pointers");
    if ((reinterpret_cast<uintptr_t>(scene) & 31u) != 0 || (reinterpret_cast<uintptr_t>(canvas) & 15u) != 0)
        return fail(HTC_ERR_INVALID, "scene must be 32-byte and canvas 16-byte aligned");
    if (passes == 0) return HTC_OK;
    return generic_render(p->generic, W, H, p->hops, p->flags, scene, scene_size, canvas, seeds, passes, stats,
                          p->d_err, stream);
}

}  // extern "C"

// A double_support program's scene, narrowed on `stream` into the program's f32-layout buffer
// (k_narrow_scene); *scene / *scene_size then name that buffer. Other programs: unchanged.
static int narrow_scene(htc_program *p, const void **scene, size_t *scene_size, void *stream) {
    if (!p || !p->double_support) return HTC_OK;
    const int li = p->recipe == HTC_RECIPE_HY ? 0 : 1;
    if (!*scene) return fail(HTC_ERR_INVALID, "scene must be a device pointer");
    if ((reinterpret_cast<uintptr_t>(*scene) & 15u) != 0) return fail(HTC_ERR_INVALID, "scene must be 16-byte aligned");
    if (*scene_size < NARROW_SRC_OBJECTS[li])
        return fail(HTC_ERR_SCENE, "scene buffer is smaller than the scene header (double_support layout)");
    uint64_t cap = (*scene_size - NARROW_SRC_OBJECTS[li]) / NARROW_SRC_STRIDE[li];
    if (cap > 0xFFFFFFull) cap = 0xFFFFFFull;
    const size_t dst_objects = li == 0 ? Layout<RECIPE_HY>::OBJECTS : Layout<RECIPE_EU>::OBJECTS;
    const size_t bytes = dst_objects + (size_t)cap * OBJ_STRIDE;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (p->narrow_bytes < bytes) {
        if (p->narrow_buf) HTC_CUDA(cudaFree(p->narrow_buf));
        p->narrow_buf = nullptr;
        p->narrow_bytes = 0;
        HTC_CUDA(cudaMalloc(&p->narrow_buf, bytes));
        HTC_CUDA(cudaMemsetAsync(p->narrow_buf, 0, bytes, st));   // the layout's padding
        p->narrow_bytes = bytes;
    }
    const uint32_t records = (uint32_t)cap + 1u;
    const unsigned blocks = std::min<unsigned>((records + 127u) / 128u, 148u * 8u);
    k_narrow_scene<<<blocks, 128, 0, st>>>(li, reinterpret_cast<const uint8_t *>(*scene), *scene_size, p->narrow_buf,
                                           (uint32_t)cap, p->address_width / 8);
    HTC_CUDA(cudaGetLastError());
    *scene = p->narrow_buf;
    *scene_size = bytes;
    return HTC_OK;
}

static int render_ex_impl(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                          float *canvas, uint32_t *seeds, uint64_t *stats, void *stream) {
    if (p && p->generic) return render_generic_program(p, W, H, scene, scene_size, canvas, seeds, 1, stats, stream);
    uint32_t max_objects = 0;
    size_t smem = 0;
    int rc = validate_render_args(p, W, H, scene, scene_size, canvas, seeds, &max_objects, &smem);
    if (rc) return rc;
    dim3 grid((W + 31) / 32, (H + 3) / 4);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint8_t *sc = reinterpret_cast<const uint8_t *>(scene);
    float4 *cv = reinterpret_cast<float4 *>(canvas);
    if (p->recipe == HTC_RECIPE_HY)
        render_plain<RECIPE_HY><<<grid, 128, smem, st>>>(sc, scene_size, max_objects, p->address_width, W, H,
                                                         p->hops, p->flags, cv, seeds, stats, p->d_err);
    else
        render_plain<RECIPE_EU><<<grid, 128, smem, st>>>(sc, scene_size, max_objects, p->address_width, W, H,
                                                         p->hops, p->flags, cv, seeds, stats, p->d_err);
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}

extern "C" {

int htc_render_ex(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                  float *canvas, uint32_t *seeds, uint64_t *stats, void *stream) {
    if (p && canvas && seeds && W && H) {   // argument errors are reported by the render checks
        int rc = narrow_scene(p, &scene, &scene_size, stream);
        if (rc) return rc;
    }
    return render_ex_impl(p, W, H, scene, scene_size, canvas, seeds, stats, stream);
}

int htc_render(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size, float *canvas,
               uint32_t *seeds, void *stream) {
    return htc_render_ex(p, W, H, scene, scene_size, canvas, seeds, nullptr, stream);
}

}  // extern "C"

// Queues of W*H slots each (a hop never has more paths than pixels) and the hop counters;
// allocated on the first call that needs more and kept with the program.
static int wave_reserve(htc_program *p, size_t slots) {
    if (!p->d_wave_ctr) {
        // hop counts are 32-bit; 2 words per hop depth
        HTC_CUDA(cudaMalloc(&p->d_wave_ctr, 2 * sizeof(uint32_t) * (size_t)p->hops));
    }
    slots = (slots + 63) & ~(size_t)63;   // keeps the second queue and every array 16-byte aligned
    if (p->recipe == HTC_RECIPE_HY && !(p->flags & HTC_FLAG_NO_SORT) && p->sort_slots < slots) {
        if (p->sort_buf) {
            HTC_CUDA(cudaFree(p->sort_buf));
            p->sort_buf = nullptr;
            p->sort_slots = 0;
        }
        HTC_CUDA(cudaMalloc(&p->sort_buf, sort_bytes(slots, p->hops)));
        // sums, cells and histogram start cleared; k_sort_scan clears sums and histogram after each use
        HTC_CUDA(cudaMemset(p->sort_buf, 0, sort_head_bytes(p->hops)));
        p->sort_slots = slots;
    }
    if (p->wave_slots >= slots) return HTC_OK;
    if (p->wave_buf) {
        HTC_CUDA(cudaFree(p->wave_buf));
        p->wave_buf = nullptr;
        p->wave_slots = 0;
    }
    HTC_CUDA(cudaMalloc(&p->wave_buf, 2 * WAVE_SLOT_BYTES * slots));
    p->wave_slots = slots;
    return HTC_OK;
}
static WaveQueue wave_queue(htc_program *p, int which) {
    const size_t n = p->wave_slots;
    uint8_t *b = reinterpret_cast<uint8_t *>(p->wave_buf) + (size_t)which * WAVE_SLOT_BYTES * n;
    WaveQueue q;
    q.p = reinterpret_cast<float4 *>(b);
    q.v = q.p + n;
    q.t = q.v + n;
    q.e = q.t + n;
    q.h = reinterpret_cast<uint32_t *>(q.e + n);
    q.o = nullptr;
    return q;
}
template <int R>
static int launch_wave(htc_program *p, uint32_t W, uint32_t H, const uint8_t *sc, size_t scene_size,
                       uint32_t max_objects, size_t smem, float4 *cv, uint32_t *seeds, uint32_t passes,
                       uint64_t *stats, cudaStream_t st) {
    int per_sm = 0;
    // a grid per kernel: the hop-0 and later-hop kernels have register caps of their own
    int per_sm0 = 0;
    HTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_wave<R, 2>, 128, smem));
    HTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm0, render_wave<R, 1>, 128, smem));
    if (per_sm < 1) per_sm = 1;
    if (per_sm0 < 1) per_sm0 = 1;
    const uint64_t needed = ((uint64_t)W * H + 127) / 128;
    const uint64_t blocks = std::min<uint64_t>((uint64_t)per_sm * (uint64_t)p->num_sms, needed);
    const uint64_t blocks0 = std::min<uint64_t>((uint64_t)per_sm0 * (uint64_t)p->num_sms, needed);
    const WaveQueue q[2] = {wave_queue(p, 0), wave_queue(p, 1)};
    const WaveQueue none = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    const bool sorted = R == RECIPE_HY && p->sort_buf != nullptr && !(p->flags & HTC_FLAG_NO_SORT);
    const SortBuf sb = sorted ? sort_buf_at(p->sort_buf, p->sort_slots, p->hops) : SortBuf{};
    const unsigned sort_blocks = (unsigned)std::min<uint64_t>((uint64_t)p->num_sms * 8u,
                                                             ((uint64_t)W * H + SORT_THREADS - 1) / SORT_THREADS);
    for (uint32_t pass = 0; pass < passes; ++pass) {
        HTC_CUDA(cudaMemsetAsync(p->d_wave_ctr, 0, 2 * sizeof(uint32_t) * (size_t)p->hops, st));
        for (uint32_t h = 0; h < p->hops; ++h) {
            WaveQueue in = h == 0 ? none : q[(h - 1) & 1];
            const uint32_t *in_count = h == 0 ? nullptr : p->d_wave_ctr + 2 * (h - 1) + 1;
            if (sorted && h > 0) {
                double *acc = sb.acc + (size_t)h * SORT_DEPTH_WORDS;
                float *cut = sb.cut + (size_t)h * SORT_DEPTH_WORDS;
                k_sort_keys<<<sort_blocks, SORT_THREADS, 0, st>>>(in.p, in.v, in_count, cut, acc, sb.key, sb.hist);
                k_sort_scan_blocks<<<SORT_SCAN_BLOCKS, SORT_THREADS, 0, st>>>(sb.hist, sb.bsum);
                k_sort_scan<<<SORT_SCAN_BLOCKS, SORT_THREADS, 0, st>>>(sb.hist, sb.bsum, sb.cursor, SORT_BINS, nullptr,
                                                                      acc, cut, in_count);
                k_sort_scatter<<<sort_blocks, SORT_THREADS, 0, st>>>(sb.key, in_count, sb.cursor, sb.perm);
                in.o = sb.perm;
            }
            (h == 0 ? render_wave<R, 1> : render_wave<R, 2>)<<<(unsigned)(h == 0 ? blocks0 : blocks), 128, smem, st>>>(sc, scene_size, max_objects, p->address_width, W, H,
                                                               p->hops, h, p->flags, cv, seeds, stats, p->d_err, in,
                                                               in_count, q[h & 1], p->d_wave_ctr + 2 * h);
        }
        HTC_CUDA(cudaGetLastError());
    }
    return HTC_OK;
}

extern "C" {

}  // extern "C"

static int render_wavefront_impl(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                                 float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats, void *stream) {
    if (p && p->generic) return fail(HTC_ERR_UNSUPPORTED, "the wavefront form serves the built-in recipes only");
    uint32_t max_objects = 0;
    size_t smem = 0;
    int rc = validate_render_args(p, W, H, scene, scene_size, canvas, seeds, &max_objects, &smem);
    if (rc) return rc;
    if (passes == 0) return HTC_OK;
    rc = wave_reserve(p, (size_t)W * H);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint8_t *sc = reinterpret_cast<const uint8_t *>(scene);
    float4 *cv = reinterpret_cast<float4 *>(canvas);
    if (p->recipe == HTC_RECIPE_HY)
        return launch_wave<RECIPE_HY>(p, W, H, sc, scene_size, max_objects, smem, cv, seeds, passes, stats, st);
    return launch_wave<RECIPE_EU>(p, W, H, sc, scene_size, max_objects, smem, cv, seeds, passes, stats, st);
}

extern "C" {

int htc_render_wavefront(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                         float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats, void *stream) {
    if (p && canvas && seeds && W && H && passes) {
        int rc = narrow_scene(p, &scene, &scene_size, stream);
        if (rc) return rc;
    }
    return render_wavefront_impl(p, W, H, scene, scene_size, canvas, seeds, passes, stats, stream);
}

int htc_render_passes(htc_program *p, uint32_t W, uint32_t H, const void *scene, size_t scene_size,
                      float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats, void *stream) {
    if (p && p->generic) return render_generic_program(p, W, H, scene, scene_size, canvas, seeds, passes, stats, stream);
    if (p && canvas && seeds && W && H && passes) {
        int rc = narrow_scene(p, &scene, &scene_size, stream);
        if (rc) return rc;
    }
    uint32_t max_objects = 0;
    size_t smem = 0;
    int rc = validate_render_args(p, W, H, scene, scene_size, canvas, seeds, &max_objects, &smem);
    if (rc) return rc;
    if (passes == 0) return HTC_OK;
    // Small canvases of cheap scenes run the one-pass kernel: their deeper hop launches would
    // leave most of the GPU idle (measured per view, 256x256 and 640x480: Euclidean 26.9 vs
    // 34.6 ms, hyperbolic with fewer than 100 objects 122.7 vs 131.5 ms, one-pass vs
    // wavefronts). Either way the result is the same bits.
    const bool cheap = (uint64_t)W * H < (1u << 19) && (p->recipe == HTC_RECIPE_EU || max_objects < 100);
    if (HT_PASSES_MODE == 2 && !cheap)
        return render_wavefront_impl(p, W, H, scene, scene_size, canvas, seeds, passes, stats, stream);
    if (HT_PASSES_MODE == 0 || HT_PASSES_MODE == 2) {
        for (uint32_t k = 0; k < passes; ++k) {
            int rc2 = render_ex_impl(p, W, H, scene, scene_size, canvas, seeds, stats, stream);
            if (rc2) return rc2;
        }
        return HTC_OK;
    }
    int per_sm = 0;
    cudaError_t e;
    if (p->recipe == HTC_RECIPE_HY)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_persistent<RECIPE_HY>, 128, smem);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_persistent<RECIPE_EU>, 128, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)per_sm * (uint64_t)p->num_sms;
    const uint64_t needed = ((uint64_t)W * H + 127) / 128;
    if (blocks > needed) blocks = needed;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint8_t *sc = reinterpret_cast<const uint8_t *>(scene);
    float4 *cv = reinterpret_cast<float4 *>(canvas);
    if (p->recipe == HTC_RECIPE_HY)
        render_persistent<RECIPE_HY><<<(unsigned)blocks, 128, smem, st>>>(sc, scene_size, max_objects, p->address_width, W, H,
                                                                          p->hops, passes, p->flags, cv, seeds, stats,
                                                                          p->d_err, p->d_queue);
    else
        render_persistent<RECIPE_EU><<<(unsigned)blocks, 128, smem, st>>>(sc, scene_size, max_objects, p->address_width, W, H,
                                                                          p->hops, passes, p->flags, cv, seeds, stats,
                                                                          p->d_err, p->d_queue);
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}

static unsigned post_blocks(uint32_t n) {
    uint32_t b = (n + 255) / 256;
    return b > 148u * 16u ? 148u * 16u : (b ? b : 1u);
}

int htc_extract(uint32_t W, uint32_t H, uint32_t passes, const float *canvas, float *image, void *stream) {
    if (!canvas || !image || passes == 0) return fail(HTC_ERR_INVALID, "bad extract arguments");
    uint32_t n = W * H;
    k_extract<<<post_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        n, (float)passes, reinterpret_cast<const float4 *>(canvas), reinterpret_cast<float4 *>(image));
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}
int htc_gamma(uint32_t W, uint32_t H, float gamma, const float *input, float *output, void *stream) {
    if (!input || !output) return fail(HTC_ERR_INVALID, "bad gamma arguments");
    uint32_t n = W * H;
    k_gamma<<<post_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        n, gamma, reinterpret_cast<const float4 *>(input), reinterpret_cast<float4 *>(output));
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}
int htc_pack(uint32_t W, uint32_t H, const float *image, uint8_t *packed, void *stream) {
    if (!image || !packed) return fail(HTC_ERR_INVALID, "bad pack arguments");
    uint32_t n = W * H;
    k_pack<<<post_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        n, reinterpret_cast<const float4 *>(image), reinterpret_cast<uchar4 *>(packed));
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}
int htc_extract_gamma_pack(uint32_t W, uint32_t H, uint32_t passes, float gamma, const float *canvas,
                           uint8_t *packed, void *stream) {
    if (!canvas || !packed || passes == 0) return fail(HTC_ERR_INVALID, "bad extract_gamma_pack arguments");
    uint32_t n = W * H;
    k_extract_gamma_pack<<<post_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        n, (float)passes, gamma, reinterpret_cast<const float4 *>(canvas), reinterpret_cast<uchar4 *>(packed));
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}

int htc_fill_seeds(uint32_t *seeds, uint32_t n, uint32_t global_seed, uint32_t offset, void *stream) {
    if (!seeds && n) return fail(HTC_ERR_INVALID, "seeds is NULL");
    if (n == 0) return HTC_OK;
    k_fill_seeds<<<post_blocks(n), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, global_seed, offset, seeds);
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}

// ---------------------------------------------------------------- batches
}  // extern "C"

struct htc_batch {
    uint32_t max_views;
    BatchView *d_views;
    uint32_t *d_err;
    uint32_t smem_objects;
    uint32_t blocks_per_sm;
    uint32_t tile_pixels;
    int num_sms, max_smem;
    cudaGraph_t graph;
    cudaGraphExec_t graph_exec;
    uint64_t *graph_stats;   // the stats buffer the graph's launches write
    std::vector<BatchView> h_views;
    // Two pinned staging slots for the asynchronous descriptor upload; slot i may be
    // rewritten once its last copy (event staged[i]) has run.
    BatchView *p_views[2];
    cudaEvent_t staged[2];
    int slot;
    // wavefront form: view order (expensive first), queues, counters
    uint32_t *d_order;
    uint32_t *p_order[2];
    uint32_t n_views, n_order, n_hy, n_eu, hops_max, passes_max;
    void *wave_buf;
    uint64_t wave_slots;     // slots per queue
    uint32_t *d_wcnt;
    size_t wcnt_words;
    void *sort_buf;          // coherence sort of the hyperbolic views (BatchSortBuf)
    uint64_t sort_slots;     // = wave_slots when allocated
    uint32_t sort_hops;
};

static void batch_free(htc_batch *b) {
    if (!b) return;
    for (int i = 0; i < 2; ++i) {
        if (b->staged[i]) {
            cudaEventSynchronize(b->staged[i]);
            cudaEventDestroy(b->staged[i]);
        }
        if (b->p_views[i]) cudaFreeHost(b->p_views[i]);
        if (b->p_order[i]) cudaFreeHost(b->p_order[i]);
    }
    if (b->d_order) cudaFree(b->d_order);
    if (b->wave_buf) cudaFree(b->wave_buf);
    if (b->d_wcnt) cudaFree(b->d_wcnt);
    if (b->sort_buf) cudaFree(b->sort_buf);
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_views);
    cudaFree(b->d_err);
    delete b;
}

template <int RF>
static cudaError_t batch_wave_smem_attr(int smem) {
    cudaError_t e = cudaFuncSetAttribute(render_batch_wave<RF, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(render_batch_wave<RF, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    return e;
}

template <int RF>
static int batch_wave_blocks(htc_batch *b, size_t smem, unsigned *blocks) {
    int per_sm = 0;
    HTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_batch_wave<RF, 2>, 128, smem));
    if (b->blocks_per_sm && (int)b->blocks_per_sm < per_sm) per_sm = (int)b->blocks_per_sm;
    if (per_sm < 1) per_sm = 1;
    *blocks = (unsigned)per_sm * (unsigned)b->num_sms;
    return HTC_OK;
}

static int batch_launch_wave(htc_batch *b, uint64_t *stats, cudaStream_t st) {
    if (b->n_order == 0) return HTC_OK;
    const size_t smem = smem_bytes(b->smem_objects) + sizeof(uint32_t) * ((size_t)b->n_views + 1);
    WaveQueue q[2];
    for (int k = 0; k < 2; ++k) {
        uint8_t *base = reinterpret_cast<uint8_t *>(b->wave_buf) + (size_t)k * WAVE_SLOT_BYTES * b->wave_slots;
        const uint64_t n = b->wave_slots;
        q[k].p = reinterpret_cast<float4 *>(base);
        q[k].v = q[k].p + n;
        q[k].t = q[k].v + n;
        q[k].e = q[k].t + n;
        q[k].h = reinterpret_cast<uint32_t *>(q[k].e + n);
        q[k].o = nullptr;
    }
    unsigned blocks_any = 0, blocks_hy = 0, blocks_eu = 0;
    int rc = HT_BATCH_SPLIT ? batch_wave_blocks<RECIPE_HY>(b, smem, &blocks_hy) : batch_wave_blocks<0>(b, smem, &blocks_any);
    if (!rc && HT_BATCH_SPLIT) rc = batch_wave_blocks<RECIPE_EU>(b, smem, &blocks_eu);
    if (rc) return rc;
    const size_t words = (size_t)(b->n_views + 3) * b->hops_max;
    uint32_t *grab = b->d_wcnt + (size_t)b->n_views * b->hops_max;   // 3 words per hop depth
    const uint32_t *order_hy = b->d_order + b->n_order, *order_eu = order_hy + b->n_hy;
    // coherence sort of the first n_seg hyperbolic views in launch order (the expensive ones)
    const uint32_t n_seg = HT_BATCH_SORT && HT_BATCH_SPLIT && b->sort_buf ? std::min(b->n_hy, BATCH_SORT_VIEWS) : 0u;
    const BatchSortBuf sb = n_seg ? batch_sort_at(b->sort_buf, b->max_views, b->sort_hops, b->sort_slots) : BatchSortBuf{};
    const unsigned sort_blocks = (unsigned)b->num_sms * 8u;
    const size_t keys_smem = sizeof(uint32_t) * (n_seg + 1) + sizeof(float) * 6 * n_seg;
    for (uint32_t pass = 0; pass < b->passes_max; ++pass) {
        HTC_CUDA(cudaMemsetAsync(b->d_wcnt, 0, sizeof(uint32_t) * words, st));
        for (uint32_t h = 0; h < b->hops_max; ++h) {
            const WaveQueue &in = q[(h + 1) & 1], &out = q[h & 1];
            if (!HT_BATCH_SPLIT) {
                (h == 0 ? render_batch_wave<0, 1> : render_batch_wave<0, 2>)<<<blocks_any, 128, smem, st>>>(b->d_views, b->d_order, b->n_order, b->n_views, pass,
                                                                   h, b->tile_pixels, b->smem_objects, in, out,
                                                                   b->d_wcnt, grab + 3 * h, stats, b->d_err, 0u);
                continue;
            }
            WaveQueue in_hy = in;
            if (n_seg && h > 0) {
                k_bsort_keys<<<sort_blocks, SORT_THREADS, keys_smem, st>>>(b->d_views, order_hy, n_seg, b->n_views, pass, h,
                                                                          b->d_wcnt, b->hops_max, in.p, in.v, sb.cut,
                                                                          sb.acc, sb.key, sb.hist);
                k_sort_scan_blocks<<<n_seg * (SORT_BINS_VIEW / 1024), SORT_THREADS, 0, st>>>(sb.hist, sb.bsum);
                k_sort_scan<<<n_seg * (SORT_BINS_VIEW / 1024), SORT_THREADS, 0, st>>>(sb.hist, sb.bsum, sb.cursor,
                                                                                     SORT_BINS_VIEW, sb.seg_base, nullptr,
                                                                                     nullptr, nullptr);
                k_bsort_scatter<<<sort_blocks, SORT_THREADS, sizeof(uint32_t) * (n_seg + 1), st>>>(
                    b->d_views, order_hy, n_seg, b->n_views, pass, h, b->d_wcnt, b->hops_max, sb.key, sb.cursor,
                    sb.seg_base, sb.acc, sb.cut, sb.perm);
                in_hy.o = sb.perm;
            }
            if (b->n_hy)
                (h == 0 ? render_batch_wave<RECIPE_HY, 1> : render_batch_wave<RECIPE_HY, 2>)<<<blocks_hy, 128, smem, st>>>(b->d_views, order_hy, b->n_hy, b->n_views,
                                                                           pass, h, b->tile_pixels, b->smem_objects, in_hy,
                                                                           out, b->d_wcnt, grab + 3 * h + 1, stats,
                                                                           b->d_err, n_seg);
            if (b->n_eu)
                (h == 0 ? render_batch_wave<RECIPE_EU, 1> : render_batch_wave<RECIPE_EU, 2>)<<<blocks_eu, 128, smem, st>>>(b->d_views, order_eu, b->n_eu, b->n_views,
                                                                           pass, h, b->tile_pixels, b->smem_objects, in,
                                                                           out, b->d_wcnt, grab + 3 * h + 2, stats,
                                                                           b->d_err, 0u);
        }
        HTC_CUDA(cudaGetLastError());
    }
    return HTC_OK;
}

extern "C" {

int htc_batch_create(uint32_t max_views, htc_batch **out) {
    if (!out) return fail(HTC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (max_views == 0) return fail(HTC_ERR_INVALID, "max_views must be positive");
    int dev = 0;
    HTC_CUDA(cudaGetDevice(&dev));
    htc_batch *b = new htc_batch();
    b->max_views = max_views;
    cudaError_t e = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_views, sizeof(BatchView) * max_views);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_order, 2 * sizeof(uint32_t) * max_views);   // all, then by recipe
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(uint32_t));
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaHostAlloc(reinterpret_cast<void **>(&b->p_views[i]), sizeof(BatchView) * max_views, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&b->p_order[i]), 2 * sizeof(uint32_t) * max_views, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->staged[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) {
        b->max_smem -= 1024;
        e = batch_wave_smem_attr<0>(b->max_smem);
        if (e == cudaSuccess) e = batch_wave_smem_attr<RECIPE_HY>(b->max_smem);
        if (e == cudaSuccess) e = batch_wave_smem_attr<RECIPE_EU>(b->max_smem);
    }
    if (e != cudaSuccess) {
        batch_free(b);
        return cuda_fail(e, "htc_batch_create");
    }
    *out = b;
    return HTC_OK;
}

void htc_batch_destroy(htc_batch *b) { batch_free(b); }

}  // extern "C"

// Grows the wavefront queues (slots per queue) and counters (words) when a view set needs
// more; launches already enqueued on `st` may still use the old ones, so they finish first.
static int batch_grow(htc_batch *b, uint64_t slots, size_t words, uint32_t hops, cudaStream_t st) {
    if (slots <= b->wave_slots && words <= b->wcnt_words && (!HT_BATCH_SORT || (b->sort_slots >= b->wave_slots &&
                                                                              hops <= b->sort_hops)))
        return HTC_OK;
    HTC_CUDA(cudaStreamSynchronize(st));
    // a captured graph holds the old buffers' addresses: the next graph launch captures anew
    if (b->graph_exec) { cudaGraphExecDestroy(b->graph_exec); b->graph_exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    if (slots > b->wave_slots) {
        if (b->wave_buf) HTC_CUDA(cudaFree(b->wave_buf));
        b->wave_buf = nullptr;
        b->wave_slots = 0;
        const uint64_t cap = (slots + slots / 4 + 63) & ~(uint64_t)63;
        HTC_CUDA(cudaMalloc(&b->wave_buf, 2 * WAVE_SLOT_BYTES * cap));
        b->wave_slots = cap;
    }
    if (words > b->wcnt_words) {
        if (b->d_wcnt) HTC_CUDA(cudaFree(b->d_wcnt));
        b->d_wcnt = nullptr;
        b->wcnt_words = 0;
        HTC_CUDA(cudaMalloc(&b->d_wcnt, sizeof(uint32_t) * words));
        b->wcnt_words = words;
    }
    if (HT_BATCH_SORT && (b->sort_slots < b->wave_slots || hops > b->sort_hops)) {
        if (b->sort_buf) HTC_CUDA(cudaFree(b->sort_buf));
        b->sort_buf = nullptr;
        b->sort_slots = 0;
        const uint32_t sh = std::max(hops, b->sort_hops);
        HTC_CUDA(cudaMalloc(&b->sort_buf, batch_sort_bytes(b->max_views, sh, b->wave_slots)));
        // sums, cells and histogram start cleared; the sort launches clear sums and histogram after each use
        HTC_CUDA(cudaMemset(b->sort_buf, 0, batch_sort_head_bytes(b->max_views, sh)));
        b->sort_slots = b->wave_slots;
        b->sort_hops = sh;
    }
    return HTC_OK;
}

extern "C" {

int htc_batch_reserve(htc_batch *b, uint64_t pixels, uint32_t max_hops, void *stream) {
    if (!b) return fail(HTC_ERR_INVALID, "batch is NULL");
    if (max_hops == 0) return fail(HTC_ERR_INVALID, "max_hops must be positive");
    // each view's region is rounded up to 64 slots
    return batch_grow(b, pixels + 64ull * b->max_views, (size_t)(b->max_views + 3) * max_hops, max_hops,
                      reinterpret_cast<cudaStream_t>(stream));
}

int htc_batch_set_views(htc_batch *b, const htc_view *views, uint32_t n_views, uint32_t tile_pixels,
                        uint32_t blocks_per_sm, void *stream) {
    if (!b) return fail(HTC_ERR_INVALID, "batch is NULL");
    if (n_views > b->max_views) return fail(HTC_ERR_INVALID, "more views than the batch was created for");
    if (n_views && !views) return fail(HTC_ERR_INVALID, "views is NULL");
    if (tile_pixels == 0) return fail(HTC_ERR_INVALID, "tile_pixels must be positive");
    b->h_views.assign(n_views, BatchView());
    uint32_t smem_objects = 0;
    std::vector<std::pair<double, uint32_t>> order;
    for (uint32_t i = 0; i < n_views; ++i) {
        const htc_view &v = views[i];
        if (v.recipe != HTC_RECIPE_HY && v.recipe != HTC_RECIPE_EU) return fail(HTC_ERR_UNSUPPORTED, "unknown scene recipe in a view");
        if (v.light_hops == 0) return fail(HTC_ERR_INVALID, "light_hops must be positive");
        if (v.address_width != 32 && v.address_width != 64) return fail(HTC_ERR_INVALID, "address_width must be 32 or 64");
        if (v.flags & ~HTC_FLAG_JITTER_YX) return fail(HTC_ERR_INVALID, "unknown view flags");
        if (v.width == 0 || v.height == 0 || (uint64_t)v.width * v.height >= 0xFFFFFFFFull)
            return fail(HTC_ERR_INVALID, "view size must be positive and fit 32 bits");
        if (!v.scene || !v.canvas || !v.seeds) return fail(HTC_ERR_INVALID, "view buffers must be device pointers");
        if ((reinterpret_cast<uintptr_t>(v.scene) & 15u) || (reinterpret_cast<uintptr_t>(v.canvas) & 15u))
            return fail(HTC_ERR_INVALID, "scene and canvas must be 16-byte aligned");
        if (v.scene_size < (v.recipe == HTC_RECIPE_HY ? 128u : 80u)) return fail(HTC_ERR_SCENE, "view scene smaller than its header");
        BatchView &d = b->h_views[i];
        d.scene = reinterpret_cast<const uint8_t *>(v.scene);
        d.scene_size = v.scene_size;
        d.canvas = reinterpret_cast<float4 *>(v.canvas);
        d.seeds = v.seeds;
        d.width = v.width;
        d.height = v.height;
        d.recipe = v.recipe;
        d.hops = v.light_hops;
        d.flags = v.flags;
        d.address_width = v.address_width;
        d.passes = v.passes;
        d.max_objects = objects_capacity(v.recipe, v.scene_size);
        if (v.passes == 0) continue;
        if (d.max_objects > smem_objects) smem_objects = d.max_objects;
        // cost per pixel ~ passes x hops x objects: expensive views first (longest-first order
        // shortens the tail of the persistent launch)
        order.push_back({(double)v.passes * v.light_hops * (1.0 + d.max_objects), i});
    }
    if (smem_bytes(smem_objects) + sizeof(uint32_t) * ((size_t)n_views + 1) > (size_t)b->max_smem)
        return fail(HTC_ERR_UNSUPPORTED, "a view has more objects than shared memory can stage");
    std::stable_sort(order.begin(), order.end(), [](const std::pair<double, uint32_t> &a, const std::pair<double, uint32_t> &c) { return a.first > c.first; });
    // wavefront queues: one region of W*H slots (rounded to 64: 16-byte aligned arrays) per view
    uint64_t slots = 0;
    uint32_t hops_max = 0, passes_max = 0;
    for (const auto &o : order) {
        BatchView &d = b->h_views[o.second];
        d.qoff = slots;
        slots += ((uint64_t)d.width * d.height + 63) & ~(uint64_t)63;
        hops_max = std::max(hops_max, d.hops);
        passes_max = std::max(passes_max, d.passes);
    }
    b->smem_objects = smem_objects;
    b->blocks_per_sm = blocks_per_sm;
    b->tile_pixels = tile_pixels;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    {
        int rc = batch_grow(b, slots, (size_t)(n_views + 3) * hops_max, hops_max, st);
        if (rc) return rc;
    }
    b->n_views = n_views;
    b->n_order = (uint32_t)order.size();
    b->hops_max = hops_max;
    b->passes_max = passes_max;
    // Asynchronous upload through the next pinned slot: wait only for that slot's previous
    // copy, then copy on `stream` (ordered after any launch still reading the device arrays).
    const int k = b->slot;
    b->slot ^= 1;
    HTC_CUDA(cudaEventSynchronize(b->staged[k]));
    if (n_views) std::memcpy(b->p_views[k], b->h_views.data(), sizeof(BatchView) * n_views);
    // the cost order of every view, then the same order split by recipe
    uint32_t *po = b->p_order[k];
    b->n_hy = b->n_eu = 0;
    for (uint32_t i = 0; i < b->n_order; ++i) po[i] = order[i].second;
    for (uint32_t i = 0; i < b->n_order; ++i)
        if (b->h_views[order[i].second].recipe == RECIPE_HY) po[b->n_order + b->n_hy++] = order[i].second;
    for (uint32_t i = 0; i < b->n_order; ++i)
        if (b->h_views[order[i].second].recipe != RECIPE_HY) po[b->n_order + b->n_hy + b->n_eu++] = order[i].second;
    if (b->n_order) HTC_CUDA(cudaMemcpyAsync(b->d_order, po, 2 * sizeof(uint32_t) * b->n_order, cudaMemcpyHostToDevice, st));
    if (n_views) HTC_CUDA(cudaMemcpyAsync(b->d_views, b->p_views[k], sizeof(BatchView) * n_views, cudaMemcpyHostToDevice, st));
    HTC_CUDA(cudaEventRecord(b->staged[k], st));
    if (b->graph_exec) { cudaGraphExecDestroy(b->graph_exec); b->graph_exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    return HTC_OK;
}

int htc_batch_render(htc_batch *b, uint64_t *stats, void *stream) {
    if (!b) return fail(HTC_ERR_INVALID, "batch is NULL");
    return batch_launch_wave(b, stats, reinterpret_cast<cudaStream_t>(stream));
}

int htc_batch_graph_launch(htc_batch *b, uint64_t *stats, void *stream) {
    if (!b) return fail(HTC_ERR_INVALID, "batch is NULL");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (b->graph_exec && b->graph_stats != stats) {   // the graph's kernels hold the stats pointer
        cudaGraphExecDestroy(b->graph_exec);
        b->graph_exec = nullptr;
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    if (!b->graph_exec) {
        cudaStream_t cap;
        HTC_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        int rc = HTC_OK;
        if (e == cudaSuccess) rc = batch_launch_wave(b, stats, cap);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e2 != cudaSuccess) return cuda_fail(e2, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->graph_exec, g, 0);
        if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(e, "cudaGraphInstantiate"); }
        b->graph = g;
        b->graph_stats = stats;
    }
    HTC_CUDA(cudaGraphLaunch(b->graph_exec, st));
    return HTC_OK;
}

int htc_batch_check(htc_batch *b, void *stream) {
    if (!b) return fail(HTC_ERR_INVALID, "batch is NULL");
    uint32_t err = 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    HTC_CUDA(cudaMemcpyAsync(&err, b->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    HTC_CUDA(cudaStreamSynchronize(st));
    if (err) {
        HTC_CUDA(cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), st));
        HTC_CUDA(cudaStreamSynchronize(st));
        return fail(HTC_ERR_SCENE, "a view's scene bytes failed validation");
    }
    return HTC_OK;
}


// ---------------------------------------------------------------- allocation-free entry
// Scratch of htc_render_passes_noalloc: the persistent kernel's work-queue words
// ([0] next pixel, [1] finished blocks) and the error word the kernel writes when the caller
// passes no `status` ([2]; nothing reads it, so such a caller gets no error report, as the
// header says). A file-scope device array, so the entry point never allocates; it lives on
// every device that loads this library until the process exits. In host code
// `g_noalloc_scratch` is only a stand-in for the symbol: its device address comes from
// cudaGetSymbolAddress.
constexpr uint32_t NOALLOC_SCRATCH_WORDS = 64;   // 256 bytes
constexpr uint64_t NOALLOC_MAX_PIXELS = 1ull << 31;   // the queue word counts pixels
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
uint32_t *g_noalloc_ptr[NOALLOC_MAX_DEVICES];
int g_noalloc_sms[NOALLOC_MAX_DEVICES];
int g_noalloc_smem[NOALLOC_MAX_DEVICES];

// Once per device, with that device current: resolve the scratch address and the launch
// limits. Allocates nothing. The cached address and kernel attributes outlive a device reset,
// which the header therefore excludes after the first call.
int noalloc_setup(int dev, uint32_t **scratch, int *num_sms, int *max_smem) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(HTC_ERR_UNSUPPORTED, "device index beyond the supported range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        uint32_t *ptr = nullptr;
        HTC_CUDA(cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_noalloc_scratch));
        int sms = 0, smem = 0;
        HTC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        HTC_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        smem -= 1024;
        int rc = set_smem_attr<RECIPE_HY>(smem);
        if (rc) return rc;
        rc = set_smem_attr<RECIPE_EU>(smem);
        if (rc) return rc;
        g_noalloc_sms[dev] = sms;
        g_noalloc_smem[dev] = smem;
        g_noalloc_ptr[dev] = ptr;
    }
    *scratch = g_noalloc_ptr[dev];
    *num_sms = g_noalloc_sms[dev];
    *max_smem = g_noalloc_smem[dev];
    return HTC_OK;
}
}  // namespace

int htc_render_passes_noalloc(int recipe, uint32_t light_hops, int address_width, uint32_t flags, uint32_t W,
                              uint32_t H, const void *scene, size_t scene_size, float *canvas, uint32_t *seeds,
                              uint32_t passes, uint64_t *stats, uint32_t *status, void *stream) {
    if (recipe != HTC_RECIPE_HY && recipe != HTC_RECIPE_EU) return fail(HTC_ERR_UNSUPPORTED, "unknown scene recipe");
    if (light_hops == 0) return fail(HTC_ERR_INVALID, "light_hops must be positive");
    if (address_width != 32 && address_width != 64) return fail(HTC_ERR_INVALID, "address_width must be 32 or 64");
    if (flags & ~HTC_FLAG_JITTER_YX) return fail(HTC_ERR_INVALID, "unknown program flags");
    if (W == 0 || H == 0) return fail(HTC_ERR_INVALID, "canvas width and height must be positive");
    if ((uint64_t)W * (uint64_t)H > NOALLOC_MAX_PIXELS)
        return fail(HTC_ERR_UNSUPPORTED, "htc_render_passes_noalloc serves at most 2^31 pixels per call (width*height)");
    if (!scene || !canvas || !seeds) return fail(HTC_ERR_INVALID, "scene, canvas and seeds must be device pointers");
    if ((reinterpret_cast<uintptr_t>(scene) & 15u) != 0 || (reinterpret_cast<uintptr_t>(canvas) & 15u) != 0)
        return fail(HTC_ERR_INVALID, "scene and canvas must be 16-byte aligned");
    if (scene_size < (recipe == HTC_RECIPE_HY ? 128u : 80u))
        return fail(HTC_ERR_SCENE, "scene buffer is smaller than the scene header");
    int dev = 0;
    HTC_CUDA(cudaGetDevice(&dev));
    uint32_t *scratch = nullptr;
    int num_sms = 0, max_smem = 0;
    int rc = noalloc_setup(dev, &scratch, &num_sms, &max_smem);
    if (rc) return rc;
    const uint32_t max_objects = objects_capacity(recipe, scene_size);
    const size_t smem = smem_bytes(max_objects);
    if (smem > (size_t)max_smem) return fail(HTC_ERR_UNSUPPORTED, "scene has more objects than shared memory can stage");
    if (passes == 0) return HTC_OK;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // The queue words must start at zero; the array keeps whatever the last call left.
    HTC_CUDA(cudaMemsetAsync(scratch, 0, 3 * sizeof(uint32_t), st));
    int per_sm = 0;
    cudaError_t e = recipe == HTC_RECIPE_HY
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_persistent<RECIPE_HY>, 128, smem)
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_persistent<RECIPE_EU>, 128, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = (uint64_t)per_sm * (uint64_t)num_sms;
    const uint64_t needed = ((uint64_t)W * H + 127) / 128;
    if (blocks > needed) blocks = needed;
    uint32_t *err = status ? status : scratch + 2;
    const uint8_t *sc = reinterpret_cast<const uint8_t *>(scene);
    float4 *cv = reinterpret_cast<float4 *>(canvas);
    if (recipe == HTC_RECIPE_HY)
        render_persistent<RECIPE_HY><<<(unsigned)blocks, 128, smem, st>>>(sc, scene_size, max_objects, address_width, W, H,
                                                                          light_hops, passes, flags, cv, seeds, stats, err,
                                                                          scratch);
    else
        render_persistent<RECIPE_EU><<<(unsigned)blocks, 128, smem, st>>>(sc, scene_size, max_objects, address_width, W, H,
                                                                          light_hops, passes, flags, cv, seeds, stats, err,
                                                                          scratch);
    HTC_CUDA(cudaGetLastError());
    return HTC_OK;
}

int htc_fp32_probe(float *scratch, uint32_t blocks, int iters, double *flops, void *stream) {
    if (!scratch || !flops || blocks == 0 || iters <= 0) return fail(HTC_ERR_INVALID, "bad probe arguments");
    k_fma_probe<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(scratch, iters);
    HTC_CUDA(cudaGetLastError());
    *flops = 2.0 * 8.0 * 16.0 * (double)iters * 256.0 * (double)blocks;
    return HTC_OK;
}

}  // extern "C"
