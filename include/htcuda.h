/*
 * htcuda.h -- C ABI of the B200-native hypertrace render path (libhtcuda.so).
 *
 * This is the drop-in boundary for the reference's OpenCL dispatch layer: a
 * `backend_cuda` feature of the `processing` crate binds these symbols where
 * `backend_ocl` drives the `ocl` crate today (processing/src/context.rs:3-16).
 * Every entry point returns an int status (HTC_OK = 0, negative on error) and sets a
 * thread-local message readable with htc_last_error(). No C++ exception crosses the ABI.
 * Streams are `cudaStream_t` values passed as `void *` (NULL = legacy default stream);
 * device pointers are plain `cudaMalloc`'d (or torch-owned) addresses.
 */
#ifndef HTCUDA_H
#define HTCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define HTC_OK 0
#define HTC_ERR_INVALID (-1)      /* bad argument */
#define HTC_ERR_CUDA (-2)         /* a CUDA runtime call failed */
#define HTC_ERR_SCENE (-3)        /* scene bytes failed validation (device-side check) */
#define HTC_ERR_UNSUPPORTED (-4)  /* configuration this build does not serve */
#define HTC_ERR_BUDGET (-5)       /* a request needs more device memory than the server's whole budget */

/* ---------------------------------------------------------------- scene recipes
 * The scene types the hand-written kernels serve (the Rust types that the reference's
 * codegen turns into OpenCL C, objects/src/scene.rs:44-67):
 *   HTC_RECIPE_HY  SceneImpl<Hyperbolic3, Mapped<PointView, Moebius>,
 *                    Vec<Mapped<Covered<Choice{Plane, Horosphere},
 *                      Mixture{Colored<Lambertian>, Specular, Emissive<Absorbing>}>, Moebius>>,
 *                    ConstBg, H>                          (main/examples/hearth.rs:27-41)
 *   HTC_RECIPE_EU  the same over Euclidean3 with Homogenous3 maps and
 *                  Choice{Plane, Sphere}                  (main/examples/eu.rs:30-44)
 */
#define HTC_RECIPE_HY 1
#define HTC_RECIPE_EU 2
/* Scene types served by the generic template kernels (compiled into the library):
 *   HTC_RECIPE_HY_TILED     SceneImpl<Hyperbolic3, Mapped<PointView, Moebius>,
 *                             Vec<Mapped<Choice{TiledPlane<M, Pentastar, 2>,
 *                               TiledPlane<M, Pentagonal, 2>, TiledHorosphere<M, Hexagonal, 3>,
 *                               TiledHorosphere<M, Square, 4>}, Moebius>>, ConstBg, H>,
 *                           M = Emissive<Mixture{Colored<Lambertian>, Specular, Transparent}>
 *                                                        (main/examples/hy.rs:35-75)
 *   HTC_RECIPE_EU_GRADIENT  SceneImpl<Euclidean3, Mapped<PointView, Homogenous3>,
 *                             Vec<Mapped<Covered<Choice{Plane, Sphere, Cube},
 *                               Mixture{Colored<Lambertian>, Specular, Colored<Refractive>}>,
 *                               Shift3>>, GradBg, H>   (main/examples/eu.rs:30-44)
 * HTC_RECIPE_CUSTOM is the recipe of a program made by htc_program_build. */
#define HTC_RECIPE_HY_TILED 3
#define HTC_RECIPE_EU_GRADIENT 4
#define HTC_RECIPE_CUSTOM 100

/* Program flags. */
#define HTC_FLAG_JITTER_YX 1u  /* first pixel-jitter draw goes to y: the order in which g++
                                  evaluates random_uniform2's arguments in the reference's
                                  host build (kernel/ocl/random.cc:15-20); the default is
                                  the OpenCL order (first draw -> x). */
#define HTC_FLAG_NO_SORT 2u    /* hyperbolic wavefronts (htc_render_wavefront / _passes) take
                                  each hop depth's paths in queue order instead of sorting them
                                  by direction and start cell first; the results are the same
                                  bits either way (htc_program_create only). */

/* Render statistics written by the entry points that take a `stats` pointer (device
 * buffer of HTC_STAT_COUNT x uint64, accumulated with atomics; zero it before the launch). */
#define HTC_STAT_SAMPLES 0       /* completed paths (scene_sample calls) */
#define HTC_STAT_HOPS 1          /* executed hop iterations (ray bounces) */
#define HTC_STAT_OBJECT_TESTS 2  /* object detect calls the reference makes (hops x objects) */
#define HTC_STAT_HITS 3          /* hops that hit an object */
#define HTC_STAT_EXACT_TESTS 4   /* object tests actually evaluated (after distance culling) */
#define HTC_STAT_COUNT 8

typedef struct htc_program htc_program;

/* ---------------------------------------------------------------- runtime */
const char *htc_last_error(void);
int htc_version(void);
int htc_device_count(int *count);
int htc_set_device(int device);

/* Replaces Render::new (processing/src/render.rs:72-100): selects the compiled kernel
 * family for a scene recipe and light-hop count H (objects/src/scene.rs:21,64).
 * address_width: 32 or 64 (types/src/config.rs:18-31). double_support (types/src/config.rs:
 * 38-43) != 0 is served for HTC_RECIPE_HY and HTC_RECIPE_EU: the scene bytes are in the
 * double_support layout (8-byte f64 fields, f64 vectors and maps aligned to their size), and
 * every render call narrows them on the device to the f32 layout (each f64 rounded to the
 * nearest f32, the value the reference serializes without double_support) into a buffer the
 * program keeps, then transports in FP32 -- the result is bit for bit that of the f32
 * serialization; an object count the buffer cannot hold is reported by htc_program_check. */
int htc_program_create(int recipe, uint32_t light_hops, int address_width, int double_support,
                       uint32_t flags, htc_program **out);
void htc_program_destroy(htc_program *program);
/* Replaces the source generation and ocl::Program::build of Render::new
 * (processing/src/render.rs:14-100, types/src/source.rs:102-168) for any scene type:
 * `scene_type` is the C++ type expression of the scene over the templates of
 * hypertrace_b200/csrc/ht_generic.cuh (e.g. "SceneImpl<Eu, MappedView<Eu, PointView<Eu>,
 * Homogenous3>, ObjectVec<Eu, ...>, ConstBg>", as hypertrace_b200/types.py writes it),
 * compiled at run time with NVRTC for sm_100a. The compiler log goes to `log` (may be
 * NULL). The program renders with htc_render / htc_render_ex / htc_render_passes. */
int htc_program_build(const char *scene_type, uint32_t light_hops, int address_width, uint32_t flags,
                      char *log, size_t log_len, htc_program **out);
/* Serialized size of the program's scene type without its dynamic part (for a Vec of
 * objects: the bytes up to the first element); a smaller scene buffer is rejected. */
int htc_program_static_size(const htc_program *program, uint64_t *bytes);
/* Reads and clears the device-side error word of the program's last launches
 * (synchronises `stream`). Returns HTC_OK or HTC_ERR_SCENE. */
int htc_program_check(htc_program *program, void *stream);

/* ---------------------------------------------------------------- buffers */
int htc_malloc(void **dptr, size_t bytes);
int htc_free(void *dptr);
int htc_memcpy_htod(void *dst, const void *src, size_t bytes, void *stream);
int htc_memcpy_dtoh(void *dst, const void *src, size_t bytes, void *stream);
int htc_memset(void *dst, int value, size_t bytes, void *stream);
int htc_stream_sync(void *stream);

/* ---------------------------------------------------------------- render
 * One pass over a width x height canvas: the `render` kernel of
 * kernel/ocl/render/render.cl:6-27 as enqueued by Render::render
 * (processing/src/render.rs:102-118): canvas[idx] += (radiance, 1), seeds[idx] advanced.
 *   scene       device pointer to the serialized scene bytes (EntityBuffer, buffer.rs:14-29)
 *   scene_size  its size in bytes (bounds every device read of the scene)
 *   canvas      device float4[width*height];  seeds: device uint32[width*height]
 * Asynchronous on `stream`; scene validity is reported by htc_program_check. */
int htc_render(htc_program *program, uint32_t width, uint32_t height, const void *scene,
               size_t scene_size, float *canvas, uint32_t *seeds, void *stream);

/* `passes` successive passes; bit-identical to `passes` htc_render calls (each pixel's
 * samples run in order and keep its RNG stream). For the built-in recipes this is
 * htc_render_wavefront, so the program keeps the queues that form allocates -- except for
 * canvases under 2^19 pixels whose scene is Euclidean or holds fewer than 100 objects, which
 * run the one-pass kernel once per pass (faster there; the same bits either way). stats (optional, device uint64[HTC_STAT_COUNT])
 * accumulates the HTC_STAT_* counters. */
int htc_render_passes(htc_program *program, uint32_t width, uint32_t height, const void *scene,
                      size_t scene_size, float *canvas, uint32_t *seeds, uint32_t passes,
                      uint64_t *stats, void *stream);

/* `passes` successive passes as wavefronts: per pass, one launch per hop depth runs one hop
 * of every path still going, from a queue of ray states, and appends the survivors to the
 * next queue (warp-aggregated, order kept within a warp). Bit-identical to htc_render_passes.
 * The program keeps two queues of width*height slots (68 bytes each), allocated by the first
 * call that needs them. No counterpart in the reference (its Render enqueues one kernel per
 * pass, processing/src/render.rs:102-118). stats as in htc_render_passes. */
int htc_render_wavefront(htc_program *program, uint32_t width, uint32_t height, const void *scene,
                         size_t scene_size, float *canvas, uint32_t *seeds, uint32_t passes,
                         uint64_t *stats, void *stream);

/* Allocation-free form of htc_render_passes, for callers that cannot call cudaMalloc --
 * e.g. hosts that hand the renderer a fixed memory budget, or custom allocators that own
 * all device memory -- and so cannot create an htc_program (which allocates its queue and
 * error words). No counterpart in the reference. The recipe, hop count, address width and
 * flags are passed directly; the work-queue words live in a 256-byte file-scope device array
 * that every device loading the library holds until exit. The first call on a device
 * resolves that array's address (cudaGetSymbolAddress) and the launch limits, so make the
 * first call on each device before any stream capture; they are kept for the rest of the
 * process, so resetting the device (cudaDeviceReset) after that first call is not supported.
 * Calls share the array and zero its queue words on entry: calls that overlap on the GPU
 * race and must not be issued concurrently.
 * Limit: width*height <= 2^31 pixels (HTC_ERR_UNSUPPORTED beyond). `status` (device uint32,
 * zeroed by the caller) receives the scene-validation error bits that htc_program_check
 * would report (non-zero = HTC_ERR_SCENE); a scene that fails validation is not rendered
 * (canvas and seeds keep their contents). `status` may be NULL, but then such a failure is
 * reported nowhere: pass it wherever the scene bytes are not known to be valid. */
int htc_render_passes_noalloc(int recipe, uint32_t light_hops, int address_width, uint32_t flags,
                              uint32_t width, uint32_t height, const void *scene, size_t scene_size,
                              float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats,
                              uint32_t *status, void *stream);

/* htc_render with statistics (the plain one-pass kernel). */
int htc_render_ex(htc_program *program, uint32_t width, uint32_t height, const void *scene,
                  size_t scene_size, float *canvas, uint32_t *seeds, uint64_t *stats,
                  void *stream);

/* ---------------------------------------------------------------- batches
 * Many views -- scenes of either recipe, resolutions, hop counts and pass counts -- rendered
 * together: one launch per pass index, hop depth and recipe covers every view's queue of ray
 * states (no counterpart in the reference, whose Pipeline renders one view per enqueue).
 * Each view's result is bit-identical to rendering it alone with htc_render_passes: pixels
 * keep their own RNG streams and sample order. */
typedef struct htc_view {
    const void *scene;       /* device pointer to the serialized scene bytes */
    uint64_t scene_size;
    float *canvas;           /* device float4[width*height], accumulated */
    uint32_t *seeds;         /* device uint32[width*height], advanced in place */
    uint32_t width, height;
    int32_t recipe;          /* HTC_RECIPE_* */
    uint32_t light_hops;
    uint32_t flags;          /* HTC_FLAG_* */
    int32_t address_width;   /* 32 or 64 */
    uint32_t passes;         /* passes of this view each htc_batch_render renders (0 = skip) */
    uint32_t reserved;
} htc_view;

typedef struct htc_batch htc_batch;
int htc_batch_create(uint32_t max_views, htc_batch **out);
void htc_batch_destroy(htc_batch *batch);
/* Uploads the views (most expensive first, each given a region of the batch's queues);
 * `tile_pixels` caps the queue slots a block takes at a time (each launch cuts its tiles on
 * the device, shorter when its paths are few); blocks_per_sm caps residency (0 = as many as
 * fit). Asynchronous on `stream`
 * (double-buffered pinned staging): the next launch on `stream` sees the new views, launches
 * already enqueued keep theirs. Blocks only while the staging slot it reuses is still being
 * copied (two calls back). */
int htc_batch_set_views(htc_batch *batch, const htc_view *views, uint32_t n_views,
                        uint32_t tile_pixels, uint32_t blocks_per_sm, void *stream);
/* Sizes the batch's wavefront queues (2 x 68 bytes per pixel) for view sets of up to `pixels`
 * pixels in total and up to `max_hops` light hops, so that htc_batch_set_views need not grow
 * them (growing waits for the launches already enqueued on `stream`). */
int htc_batch_reserve(htc_batch *batch, uint64_t pixels, uint32_t max_hops, void *stream);
/* Renders every view's `passes`: one launch per pass index, hop depth and recipe over all the
 * views (wavefronts). stats as in htc_render_passes. */
int htc_batch_render(htc_batch *batch, uint64_t *stats, void *stream);
/* The same launch through a CUDA graph captured on first use and re-captured after
 * htc_batch_set_views, after an htc_batch_reserve that grows the queues, and when `stats`
 * differs from the pointer of the last capture (the graph's kernels hold it). */
int htc_batch_graph_launch(htc_batch *batch, uint64_t *stats, void *stream);
/* Reads and clears the batch's device error word (synchronises `stream`). */
int htc_batch_check(htc_batch *batch, void *stream);

/* ---------------------------------------------------------------- serving
 * A continuous-batching render server (no counterpart in the reference, whose examples render
 * one view per frame in a time-budgeted loop, main/examples/hearth.rs:116-135). Requests are
 * submitted at any time; every htc_server_step admits waiting requests while their device
 * memory fits the HBM budget (interactive ones first; memory from a stream-ordered pool, so
 * admission never synchronises the device), plans the step (htc_serve_plan) and renders the
 * planned passes of all admitted requests together (the batch launches above). Requests that
 * a step completes get the post chain and their read-back enqueued after it, and their device
 * memory released; htc_server_poll reports them once their host buffers are written. Each
 * request's result is bit-identical to rendering it alone. One server serves one stream and
 * one host thread at a time. */
#define HTC_PRIORITY_INTERACTIVE 0   /* all remaining passes in the next step, planned first */
#define HTC_PRIORITY_BATCH 1         /* up to `quantum` passes per step, with what is left */

typedef struct htc_request {
    const void *scene;       /* host pointer to the serialized scene bytes (copied at submission) */
    uint64_t scene_size;
    uint32_t width, height;
    int32_t recipe;          /* HTC_RECIPE_HY or HTC_RECIPE_EU */
    uint32_t light_hops;
    uint32_t flags;          /* HTC_FLAG_* */
    int32_t address_width;   /* 32 or 64 */
    uint32_t passes;         /* samples per pixel to render */
    uint32_t global_seed;    /* per-pixel seeds as htc_fill_seeds(seeds, w*h, global_seed, 0) */
    uint32_t priority;       /* HTC_PRIORITY_* */
    uint32_t quantum;        /* batch jobs: passes per step */
    float gamma;             /* post chain exponent (1/2.2 in the reference's pipeline) */
    uint32_t reserved;
    void *out_rgba8;         /* host, width*height*4 bytes: the packed image (pinned keeps the copy async) */
    void *out_canvas;        /* host, width*height*16 bytes, or NULL: the float4 accumulation */
    void *out_seeds;         /* host, width*height*4 bytes, or NULL: the final RNG states */
} htc_request;

/* One request as the planner sees it. */
typedef struct htc_plan_item {
    uint64_t pixels;
    uint32_t remaining;      /* passes still to render */
    uint32_t quantum;
    uint32_t priority;
    uint32_t reserved;
} htc_plan_item;

typedef struct htc_server_info {
    uint32_t waiting, active, in_flight, finished;
    uint64_t used_bytes, budget_bytes, steps;
} htc_server_info;

typedef struct htc_server htc_server;
/* The step planner alone (host only, no device): passes[i] for items in arrival order --
 * interactive items whole while they fit `step_samples` samples (the first one always), then
 * batch items up to their quantum with what is left (at least one pass when nothing else runs). */
int htc_serve_plan(const htc_plan_item *items, uint32_t n, uint64_t step_samples, uint32_t *passes);
/* A server for the current device: `hbm_budget` bytes of request memory (scene, canvas, seeds,
 * image and a 136-byte-per-pixel share of the wavefront queues), steps of at most
 * `step_samples` samples (bounds how long a new arrival waits), up to `max_views` requests in
 * one step. */
int htc_server_create(uint64_t hbm_budget, uint64_t step_samples, uint32_t max_views, htc_server **out);
void htc_server_destroy(htc_server *server);
/* Steps in flight (default 2), the batch tile size (default 512), admissions per step
 * (default 8), and queue slots to reserve up front (0 = none). */
int htc_server_configure(htc_server *server, uint32_t depth, uint32_t tile_pixels, uint32_t admit_per_step,
                         uint64_t reserve_pixels, void *stream);
/* Queues a request (copies its scene bytes); *id identifies it in htc_server_poll.
 * HTC_ERR_BUDGET when it alone needs more than the whole budget. */
int htc_server_submit(htc_server *server, const htc_request *request, uint64_t *id);
/* One step on `stream` (see above); *rendered_views (may be NULL) = requests it renders
 * (0 when nothing is admitted). Blocks only while `depth` steps are still in flight. */
int htc_server_step(htc_server *server, void *stream, uint32_t *rendered_views);
/* Ids of finished requests (host buffers written), up to max_ids; wait_all != 0 first waits
 * for every step in flight. */
int htc_server_poll(htc_server *server, uint64_t *ids, uint32_t max_ids, uint32_t *n, int wait_all);
int htc_server_stats(const htc_server *server, htc_server_info *info);

/* ---------------------------------------------------------------- post chain
 * Extractor (processing/src/canvas.rs:126-135): image = canvas / passes.
 * GammaFilter (processing/src/filter/gamma.rs:10-19): out = pow(max(in, 0), gamma).
 * Packer (processing/src/canvas.rs:176-186): u8 = (uchar)(255 * clamp(x, 0, 1)), toward 0. */
int htc_extract(uint32_t width, uint32_t height, uint32_t passes, const float *canvas,
                float *image, void *stream);
int htc_gamma(uint32_t width, uint32_t height, float gamma, const float *input, float *output,
              void *stream);
int htc_pack(uint32_t width, uint32_t height, const float *image, uint8_t *packed, void *stream);
/* The three stages fused in one pass over the canvas (what Pipeline::get_image computes,
 * processing/src/pipeline.rs:53-62). */
int htc_extract_gamma_pack(uint32_t width, uint32_t height, uint32_t passes, float gamma,
                           const float *canvas, uint8_t *packed, void *stream);

/* Initial per-pixel RNG states seeds[i] = fmix32(global_seed ^ fmix32(i + offset)) (MurmurHash3's
 * 32-bit finaliser), written on the device. The reference fills its seed buffer from a host
 * SmallRng stream (processing/src/canvas.rs:193-195) and its kernel only reads it; these are
 * the seeds every test and benchmark of this library uses (hypertrace_b200.scene.pixel_seeds
 * computes the same values on the host). */
int htc_fill_seeds(uint32_t *seeds, uint32_t n, uint32_t global_seed, uint32_t offset, void *stream);

/* ---------------------------------------------------------------- calibration
 * FP32 FMA throughput probe used as the roofline denominator of the render kernels
 * (they are FP32-issue bound). Launches `blocks` x 256 threads of independent FMA chains;
 * `scratch` is a device float[blocks*256]; *flops receives the flop count of the launch
 * (2 per FMA). Time it with events on `stream`. No counterpart in the reference. */
int htc_fp32_probe(float *scratch, uint32_t blocks, int iters, double *flops, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HTCUDA_H */
