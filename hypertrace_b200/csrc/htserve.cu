// htserve.cu -- the continuous-batching render server of libhtcuda.so (htc_server_*, declared
// in include/htcuda.h). No counterpart in the reference, whose examples render one view per
// frame in a time-budgeted loop (main/examples/hearth.rs:116-135).
//
// Requests (a scene, a canvas size, a pass count) are submitted from the host at any time.
// Each htc_server_step call
//   1. retires finished steps (events), and waits for the older one when `depth` steps are
//      in flight;
//   2. admits waiting requests -- interactive ones first -- while their device memory fits the
//      HBM budget: scene, canvas, seeds and RGBA8 image come from a stream-ordered memory pool
//      (cudaMallocAsync), so admission never synchronises the device, and a request larger
//      than the whole budget is refused at submission (HTC_ERR_BUDGET);
//   3. plans the step (htc_serve_plan: interactive frames whole, in arrival order, then batch
//      jobs by quantum, within the step's sample budget);
//   4. renders the planned passes of every admitted request in one batched launch sequence
//      (htc_batch_set_views + htc_batch_render: one launch per pass index, hop depth and
//      recipe over all views);
//   5. for each request that the step completes, enqueues the post chain
//      (htc_extract_gamma_pack), the copies of the image (and, when asked, canvas and seeds)
//      to the request's host buffers and the release of its device memory (cudaFreeAsync), all
//      ordered after the step on the stream, then records the step's event.
// htc_server_poll returns the requests whose host buffers are complete. Each request's pixels
// keep their own RNG streams and sample order, so its result is bit-identical to rendering it
// alone (tests/test_gpu_serve.py).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/htcuda.h"
#include "ht_host.hpp"

namespace {

struct ServeReq {
    htc_request r;                 // as submitted (host pointers stay the caller's)
    std::vector<uint8_t> scene;    // host copy of the scene bytes
    uint64_t id = 0;
    uint32_t done = 0;             // passes rendered (or enqueued)
    uint64_t bytes = 0;            // device bytes charged to the budget while admitted
    void *d_scene = nullptr;
    float *d_canvas = nullptr;
    uint32_t *d_seeds = nullptr;
    uint8_t *d_packed = nullptr;
};

struct ServeStep {
    cudaEvent_t ev = nullptr;
    std::vector<uint64_t> finishing;
};

// Device bytes of one admitted request: scene, canvas (16 B per pixel), seeds (4 B), RGBA8
// image (4 B), and its share of the batch's two wavefront queues (2 x 68 B per pixel).
uint64_t request_bytes(const htc_request &r) {
    const uint64_t px = (uint64_t)r.width * r.height;
    return ((r.scene_size + 255) & ~255ull) + px * (16 + 4 + 4 + 136);
}

}  // namespace

struct htc_server {
    uint64_t budget = 0, used = 0, step_samples = 0;
    uint32_t depth = 2, tile_pixels = 512, admit_per_step = 8;
    htc_batch *batch = nullptr;
    cudaMemPool_t pool = nullptr;
    uint64_t next_id = 1;
    std::unordered_map<uint64_t, ServeReq> reqs;
    std::deque<uint64_t> waiting_i, waiting_b;   // arrival order per class
    std::vector<uint64_t> active;                // admitted, arrival order
    std::deque<ServeStep> inflight;
    std::vector<uint64_t> done;                  // finished, not yet polled
    std::vector<cudaEvent_t> spare_events;
    uint64_t steps = 0;
    // scratch of a step
    std::vector<htc_plan_item> items;
    std::vector<uint32_t> passes;
    std::vector<htc_view> views;
};

static int retire_front(htc_server *s, bool wait) {
    ServeStep &st = s->inflight.front();
    if (wait) {
        HTC_CUDA(cudaEventSynchronize(st.ev));
    } else {
        const cudaError_t q = cudaEventQuery(st.ev);
        if (q == cudaErrorNotReady) return 1;
        if (q != cudaSuccess) return cuda_fail(q, "cudaEventQuery");
    }
    for (uint64_t id : st.finishing) s->done.push_back(id);
    s->spare_events.push_back(st.ev);
    s->inflight.pop_front();
    return HTC_OK;
}

static int retire(htc_server *s) {
    while (!s->inflight.empty()) {
        const int rc = retire_front(s, false);
        if (rc == 1) break;
        if (rc) return rc;
    }
    return HTC_OK;
}

static void free_request_memory(ServeReq &q, cudaStream_t st) {
    if (q.d_scene) cudaFreeAsync(q.d_scene, st);
    if (q.d_canvas) cudaFreeAsync(q.d_canvas, st);
    if (q.d_seeds) cudaFreeAsync(q.d_seeds, st);
    if (q.d_packed) cudaFreeAsync(q.d_packed, st);
    q.d_scene = q.d_canvas = nullptr;
    q.d_seeds = nullptr;
    q.d_packed = nullptr;
}

static int admit(htc_server *s, ServeReq &q, cudaStream_t st) {
    const uint64_t px = (uint64_t)q.r.width * q.r.height;
    cudaError_t e = cudaMallocFromPoolAsync(&q.d_scene, (q.r.scene_size + 15) & ~15ull, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&q.d_canvas), 16 * px, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&q.d_seeds), 4 * px, s->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&q.d_packed), 4 * px, s->pool, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.d_scene, q.scene.data(), q.r.scene_size, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(q.d_canvas, 0, 16 * px, st);
    if (e != cudaSuccess) {
        free_request_memory(q, st);
        return cuda_fail(e, "htc_server_step: admission");
    }
    int rc = htc_fill_seeds(q.d_seeds, (uint32_t)px, q.r.global_seed, 0, st);
    if (rc) {
        free_request_memory(q, st);
        return rc;
    }
    s->used += q.bytes;
    s->active.push_back(q.id);
    return HTC_OK;
}

extern "C" {

int htc_serve_plan(const htc_plan_item *items, uint32_t n, uint64_t step_samples, uint32_t *passes) {
    if (n && (!items || !passes)) return fail(HTC_ERR_INVALID, "items and passes must not be NULL");
    uint64_t left = step_samples;
    bool any = false;
    for (uint32_t i = 0; i < n; ++i) passes[i] = 0;
    // interactive frames first, whole, in the given (arrival) order; a frame that does not fit
    // waits for the next step unless nothing is planned yet
    for (uint32_t i = 0; i < n; ++i) {
        const htc_plan_item &it = items[i];
        if (it.priority != HTC_PRIORITY_INTERACTIVE || it.remaining == 0) continue;
        const uint64_t cost = it.pixels * it.remaining;
        if (cost <= left || !any) {
            passes[i] = it.remaining;
            left = cost <= left ? left - cost : 0;
            any = true;
        }
    }
    // then batch jobs in order, each up to its quantum, with what is left (at least one pass
    // of one job when nothing else runs)
    for (uint32_t i = 0; i < n; ++i) {
        const htc_plan_item &it = items[i];
        if (it.priority == HTC_PRIORITY_INTERACTIVE || it.remaining == 0) continue;
        uint64_t p = std::min<uint64_t>(std::max<uint32_t>(it.quantum, 1u), it.remaining);
        if (it.pixels) p = std::min<uint64_t>(p, left / it.pixels);
        if (p == 0 && !any) p = 1;
        if (p > 0) {
            passes[i] = (uint32_t)p;
            const uint64_t cost = it.pixels * p;
            left = cost <= left ? left - cost : 0;
            any = true;
        }
    }
    return HTC_OK;
}

int htc_server_create(uint64_t hbm_budget, uint64_t step_samples, uint32_t max_views, htc_server **out) {
    if (!out) return fail(HTC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (hbm_budget == 0 || step_samples == 0 || max_views == 0)
        return fail(HTC_ERR_INVALID, "hbm_budget, step_samples and max_views must be positive");
    int dev = 0;
    HTC_CUDA(cudaGetDevice(&dev));
    htc_server *s = new htc_server();
    s->budget = hbm_budget;
    s->step_samples = step_samples;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        // keep freed blocks in the pool: admission reuses them without going to the driver
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        if (s->pool) cudaMemPoolDestroy(s->pool);
        delete s;
        return cuda_fail(e, "htc_server_create");
    }
    int rc = htc_batch_create(max_views, &s->batch);
    if (rc) {
        cudaMemPoolDestroy(s->pool);
        delete s;
        return rc;
    }
    *out = s;
    return HTC_OK;
}

void htc_server_destroy(htc_server *s) {
    if (!s) return;
    cudaDeviceSynchronize();
    for (auto &kv : s->reqs) free_request_memory(kv.second, nullptr);
    cudaDeviceSynchronize();
    for (auto &st : s->inflight) cudaEventDestroy(st.ev);
    for (cudaEvent_t ev : s->spare_events) cudaEventDestroy(ev);
    htc_batch_destroy(s->batch);
    cudaMemPoolDestroy(s->pool);
    delete s;
}

int htc_server_configure(htc_server *s, uint32_t depth, uint32_t tile_pixels, uint32_t admit_per_step,
                         uint64_t reserve_pixels, void *stream) {
    if (!s) return fail(HTC_ERR_INVALID, "server is NULL");
    if (depth == 0 || tile_pixels == 0 || admit_per_step == 0)
        return fail(HTC_ERR_INVALID, "depth, tile_pixels and admit_per_step must be positive");
    s->depth = depth;
    s->tile_pixels = tile_pixels;
    s->admit_per_step = admit_per_step;
    if (reserve_pixels) return htc_batch_reserve(s->batch, reserve_pixels, 8, stream);
    return HTC_OK;
}

int htc_server_submit(htc_server *s, const htc_request *r, uint64_t *id) {
    if (!s || !r || !id) return fail(HTC_ERR_INVALID, "server, request and id must not be NULL");
    *id = 0;
    if (!r->scene || r->scene_size == 0) return fail(HTC_ERR_INVALID, "request scene is empty");
    if (r->recipe != HTC_RECIPE_HY && r->recipe != HTC_RECIPE_EU) return fail(HTC_ERR_UNSUPPORTED, "unknown scene recipe in a request");
    if (r->width == 0 || r->height == 0 || (uint64_t)r->width * r->height >= 0xFFFFFFFFull)
        return fail(HTC_ERR_INVALID, "request size must be positive and fit 32 bits");
    if (r->light_hops == 0 || r->passes == 0) return fail(HTC_ERR_INVALID, "light_hops and passes must be positive");
    if (r->address_width != 32 && r->address_width != 64) return fail(HTC_ERR_INVALID, "address_width must be 32 or 64");
    if (r->flags & ~HTC_FLAG_JITTER_YX) return fail(HTC_ERR_INVALID, "unknown request flags");
    if (r->priority != HTC_PRIORITY_INTERACTIVE && r->priority != HTC_PRIORITY_BATCH)
        return fail(HTC_ERR_INVALID, "unknown request priority");
    if (!r->out_rgba8) return fail(HTC_ERR_INVALID, "out_rgba8 must be a host buffer of width*height*4 bytes");
    const uint64_t bytes = request_bytes(*r);
    if (bytes > s->budget) return fail(HTC_ERR_BUDGET, "request needs more device memory than the whole HBM budget");
    ServeReq q;
    q.r = *r;
    q.scene.assign(reinterpret_cast<const uint8_t *>(r->scene), reinterpret_cast<const uint8_t *>(r->scene) + r->scene_size);
    q.r.scene = nullptr;   // the host copy above is what admission uploads
    q.id = s->next_id++;
    q.bytes = bytes;
    (r->priority == HTC_PRIORITY_INTERACTIVE ? s->waiting_i : s->waiting_b).push_back(q.id);
    *id = q.id;
    s->reqs.emplace(q.id, std::move(q));
    return HTC_OK;
}

int htc_server_step(htc_server *s, void *stream, uint32_t *rendered_views) {
    if (!s) return fail(HTC_ERR_INVALID, "server is NULL");
    if (rendered_views) *rendered_views = 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int rc = retire(s);
    if (rc) return rc;
    while (s->inflight.size() >= s->depth) {
        rc = retire_front(s, true);
        if (rc) return rc;
    }
    // admission: interactive first, then batch jobs, while the budget allows
    uint32_t admits = 0;
    for (std::deque<uint64_t> *w : {&s->waiting_i, &s->waiting_b}) {
        while (!w->empty() && admits < s->admit_per_step) {
            ServeReq &q = s->reqs.at(w->front());
            if (s->used + q.bytes > s->budget) break;
            rc = admit(s, q, st);
            if (rc) return rc;
            w->pop_front();
            ++admits;
        }
    }
    if (s->active.empty()) return HTC_OK;
    // plan: the active requests in arrival order (ids grow with submission)
    const uint32_t n = (uint32_t)s->active.size();
    s->items.resize(n);
    s->passes.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        const ServeReq &q = s->reqs.at(s->active[i]);
        htc_plan_item &it = s->items[i];
        it.pixels = (uint64_t)q.r.width * q.r.height;
        it.remaining = q.r.passes - q.done;
        it.quantum = q.r.quantum;
        it.priority = q.r.priority;
    }
    rc = htc_serve_plan(s->items.data(), n, s->step_samples, s->passes.data());
    if (rc) return rc;
    s->views.clear();
    for (uint32_t i = 0; i < n; ++i) {
        if (!s->passes[i]) continue;
        const ServeReq &q = s->reqs.at(s->active[i]);
        htc_view v;
        v.scene = q.d_scene;
        v.scene_size = q.r.scene_size;
        v.canvas = q.d_canvas;
        v.seeds = q.d_seeds;
        v.width = q.r.width;
        v.height = q.r.height;
        v.recipe = q.r.recipe;
        v.light_hops = q.r.light_hops;
        v.flags = q.r.flags;
        v.address_width = q.r.address_width;
        v.passes = s->passes[i];
        v.reserved = 0;
        s->views.push_back(v);
    }
    rc = htc_batch_set_views(s->batch, s->views.data(), (uint32_t)s->views.size(), s->tile_pixels, 0, stream);
    if (rc) return rc;
    rc = htc_batch_render(s->batch, nullptr, stream);
    if (rc) return rc;
    if (rendered_views) *rendered_views = (uint32_t)s->views.size();
    // requests this step completes: post chain, read-back and release, ordered after the step
    ServeStep step;
    std::vector<uint64_t> still;
    still.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        ServeReq &q = s->reqs.at(s->active[i]);
        q.done += s->passes[i];
        if (q.done < q.r.passes) {
            still.push_back(q.id);
            continue;
        }
        const uint64_t px = (uint64_t)q.r.width * q.r.height;
        rc = htc_extract_gamma_pack(q.r.width, q.r.height, q.r.passes, q.r.gamma, q.d_canvas, q.d_packed, stream);
        if (rc) return rc;
        HTC_CUDA(cudaMemcpyAsync(q.r.out_rgba8, q.d_packed, 4 * px, cudaMemcpyDeviceToHost, st));
        if (q.r.out_canvas) HTC_CUDA(cudaMemcpyAsync(q.r.out_canvas, q.d_canvas, 16 * px, cudaMemcpyDeviceToHost, st));
        if (q.r.out_seeds) HTC_CUDA(cudaMemcpyAsync(q.r.out_seeds, q.d_seeds, 4 * px, cudaMemcpyDeviceToHost, st));
        free_request_memory(q, st);
        s->used -= q.bytes;
        step.finishing.push_back(q.id);
    }
    s->active.swap(still);
    if (s->spare_events.empty()) {
        cudaEvent_t ev;
        HTC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        s->spare_events.push_back(ev);
    }
    step.ev = s->spare_events.back();
    s->spare_events.pop_back();
    HTC_CUDA(cudaEventRecord(step.ev, st));
    s->inflight.push_back(std::move(step));
    s->steps += 1;
    return HTC_OK;
}

int htc_server_poll(htc_server *s, uint64_t *ids, uint32_t max_ids, uint32_t *n, int wait_all) {
    if (!s || !n) return fail(HTC_ERR_INVALID, "server and n must not be NULL");
    if (max_ids && !ids) return fail(HTC_ERR_INVALID, "ids is NULL");
    *n = 0;
    if (wait_all) {
        while (!s->inflight.empty()) {
            int rc = retire_front(s, true);
            if (rc) return rc;
        }
    } else {
        int rc = retire(s);
        if (rc) return rc;
    }
    const uint32_t k = (uint32_t)std::min<size_t>(max_ids, s->done.size());
    for (uint32_t i = 0; i < k; ++i) {
        ids[i] = s->done[i];
        s->reqs.erase(s->done[i]);
    }
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return HTC_OK;
}

int htc_server_stats(const htc_server *s, htc_server_info *info) {
    if (!s || !info) return fail(HTC_ERR_INVALID, "server and info must not be NULL");
    info->waiting = (uint32_t)(s->waiting_i.size() + s->waiting_b.size());
    info->active = (uint32_t)s->active.size();
    info->in_flight = (uint32_t)s->inflight.size();
    info->finished = (uint32_t)s->done.size();
    info->used_bytes = s->used;
    info->budget_bytes = s->budget;
    info->steps = s->steps;
    return HTC_OK;
}

}  // extern "C"
