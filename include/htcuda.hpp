// htcuda.hpp -- C++ mirror of the reference's `processing` crate over the C ABI.
//
// Header-only RAII wrappers with the names and meaning of processing/src/*.rs:
// Context, EntityBuffer (buffer.rs:13-29), Canvas (canvas.rs:130-237), Render
// (render.rs:8-119), Pipeline (pipeline.rs:8-67). Errors become htc::Error exceptions
// on the C++ side of the boundary (no exception crosses the C ABI itself).
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "htcuda.h"

namespace htc {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error("htcuda error " + std::to_string(c) + ": " + m), code(c) {}
};

inline void check(int rc) {
    if (rc != HTC_OK) throw Error(rc, htc_last_error());
}

// Owning device allocation.
class DeviceBuffer {
  public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t bytes) : bytes_(bytes) { check(htc_malloc(&ptr_, bytes)); }
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    DeviceBuffer(DeviceBuffer &&o) noexcept : ptr_(std::exchange(o.ptr_, nullptr)), bytes_(o.bytes_) {}
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
        std::swap(ptr_, o.ptr_);
        std::swap(bytes_, o.bytes_);
        return *this;
    }
    ~DeviceBuffer() {
        if (ptr_) htc_free(ptr_);
    }
    void *get() const { return ptr_; }
    size_t size() const { return bytes_; }
    void upload(const void *src, size_t n, void *stream = nullptr) { check(htc_memcpy_htod(ptr_, src, n, stream)); }
    void download(void *dst, size_t n, void *stream = nullptr) const { check(htc_memcpy_dtoh(dst, ptr_, n, stream)); }
    void zero(void *stream = nullptr) { check(htc_memset(ptr_, 0, bytes_, stream)); }

  private:
    void *ptr_ = nullptr;
    size_t bytes_ = 0;
};

// types::Config + processing::Context: the device and the serialization config.
struct Config {
    int address_width = 32;
    bool double_support = false;
};
class Context {
  public:
    explicit Context(int device = 0, Config config = {}) : device_(device), config_(config) { check(htc_set_device(device)); }
    const Config &config() const { return config_; }
    int device() const { return device_; }
    void *stream() const { return stream_; }

  private:
    int device_;
    Config config_;
    void *stream_ = nullptr;   // legacy default stream, like the reference's single queue
};

// Serialized scene bytes on the device (EntityBuffer::new uploads what types::io wrote).
class EntityBuffer {
  public:
    EntityBuffer(const Context &ctx, const std::vector<uint8_t> &bytes) : buf_(bytes.size() ? bytes.size() : 1) {
        buf_.upload(bytes.data(), bytes.size(), ctx.stream());
        size_ = bytes.size();
    }
    const void *raw() const { return buf_.get(); }
    size_t size() const { return size_; }

  private:
    DeviceBuffer buf_;
    size_t size_ = 0;
};

// float4 accumulation + per-pixel RNG states; seeds persist across clean() (canvas.rs:102-106).
class Canvas {
  public:
    Canvas(const Context &ctx, uint32_t width, uint32_t height, const std::vector<uint32_t> &seeds)
        : w_(width), h_(height), image_(16ull * width * height), seeds_(4ull * width * height), ctx_(&ctx) {
        if (seeds.size() != (size_t)width * height) throw Error(HTC_ERR_INVALID, "one seed per pixel");
        image_.zero(ctx.stream());
        seeds_.upload(seeds.data(), 4ull * width * height, ctx.stream());
    }
    uint32_t width() const { return w_; }
    uint32_t height() const { return h_; }
    uint32_t passes() const { return passes_; }
    void add_pass(uint32_t n = 1) { passes_ += n; }
    void clean() {
        image_.zero(ctx_->stream());
        passes_ = 0;
    }
    float *image() const { return static_cast<float *>(image_.get()); }
    uint32_t *seeds() const { return static_cast<uint32_t *>(seeds_.get()); }

  private:
    uint32_t w_, h_, passes_ = 0;
    DeviceBuffer image_, seeds_;
    const Context *ctx_;
};

// The render kernel of one scene recipe and hop count (Render::new / Render::render).
class Render {
  public:
    Render(const Context &ctx, int recipe, uint32_t light_hops, uint32_t flags = 0) : ctx_(&ctx) {
        check(htc_program_create(recipe, light_hops, ctx.config().address_width, ctx.config().double_support ? 1 : 0,
                                 flags, &prog_));
    }
    Render(const Render &) = delete;
    Render &operator=(const Render &) = delete;
    ~Render() { htc_program_destroy(prog_); }
    // One pass, blocking like the reference (enqueue, finish, add_pass).
    void render(const EntityBuffer &scene, Canvas &canvas) {
        check(htc_render(prog_, canvas.width(), canvas.height(), scene.raw(), scene.size(), canvas.image(),
                         canvas.seeds(), ctx_->stream()));
        check(htc_program_check(prog_, ctx_->stream()));
        canvas.add_pass();
    }
    // `passes` passes in one persistent launch (bit-identical to `passes` render calls).
    void render_passes(const EntityBuffer &scene, Canvas &canvas, uint32_t passes) {
        check(htc_render_passes(prog_, canvas.width(), canvas.height(), scene.raw(), scene.size(), canvas.image(),
                                canvas.seeds(), passes, nullptr, ctx_->stream()));
        check(htc_program_check(prog_, ctx_->stream()));
        canvas.add_pass(passes);
    }

  private:
    const Context *ctx_;
    htc_program *prog_ = nullptr;
};

// processing::Pipeline: scene buffer, render, canvas and the post chain to RGBA8.
class Pipeline {
  public:
    Pipeline(const Context &ctx, uint32_t width, uint32_t height, int recipe, uint32_t light_hops,
             const std::vector<uint8_t> &scene, const std::vector<uint32_t> &seeds, float gamma = 1.0f / 2.2f,
             uint32_t flags = 0)
        : ctx_(&ctx), scene_(ctx, scene), render_(ctx, recipe, light_hops, flags), canvas_(ctx, width, height, seeds),
          packed_(4ull * width * height), gamma_(gamma) {}
    void set_scene(const std::vector<uint8_t> &scene) { scene_ = EntityBuffer(*ctx_, scene); }
    void render(uint32_t passes = 1) {
        if (passes == 1) render_.render(scene_, canvas_);
        else render_.render_passes(scene_, canvas_, passes);
    }
    // extract + gamma + pack, then a blocking read-back (pipeline.rs:53-62)
    std::vector<uint8_t> get_image() {
        const uint32_t w = canvas_.width(), h = canvas_.height();
        check(htc_extract_gamma_pack(w, h, canvas_.passes() ? canvas_.passes() : 1, gamma_, canvas_.image(),
                                     static_cast<uint8_t *>(packed_.get()), ctx_->stream()));
        std::vector<uint8_t> out(4ull * w * h);
        packed_.download(out.data(), out.size(), ctx_->stream());
        check(htc_stream_sync(ctx_->stream()));
        return out;
    }
    void clean() { canvas_.clean(); }
    Canvas &canvas() { return canvas_; }

  private:
    const Context *ctx_;
    EntityBuffer scene_;
    Render render_;
    Canvas canvas_;
    DeviceBuffer packed_;
    float gamma_;
};

}  // namespace htc
