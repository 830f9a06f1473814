// htgeneric.cu -- generic scene programs: built-in instantiations of ht_generic.cuh and the
// NVRTC path for any scene type (the counterpart of the reference's per-scene-type OpenCL
// codegen and `ocl::Program::build`, processing/src/render.rs:14-100).
//
// A generic program holds one kernel `htg::render_generic<Scene, W>`:
//   - recipes HTC_RECIPE_HY_TILED and HTC_RECIPE_EU_GRADIENT are compiled into this library;
//   - htc_program_build compiles `render_generic<type, W>` for a C++ type expression at run
//     time with NVRTC for sm_100a (same flags as the library: no FMA contraction, IEEE
//     division and square root), loads the cubin with the driver API and keeps the module.
// NVRTC and the driver API are reached at run time (dlopen of libnvrtc, and
// cudaGetDriverEntryPoint), so the library loads on hosts without either.
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/htcuda.h"
#include "ht_generic.cuh"
#include "ht_host.hpp"

using namespace htg;

// ============================================================================ built-in types
namespace htg {
// main/examples/hy.rs:35-75: Emissive<Mixture{Colored<Lambertian>, Specular, Transparent}>,
// Choice{PlaneStar, PlanePenta, HoroHexa, HoroSquare} of tiled objects, H = 3 in the example.
typedef Emissive<Mixture<Component<Colored<Lambertian>>, Component<Specular>, Component<Transparent>>> HyTiledMaterial;
typedef ObjectChoice<Hy, TiledPlane<HyTiledMaterial, PlanePentastar, 2>, TiledPlane<HyTiledMaterial, PlanePentagonal, 2>,
                     TiledHorosphere<HyTiledMaterial, HoroHexagonal, 3>, TiledHorosphere<HyTiledMaterial, HoroSquare, 4>>
    HyTiledChoice;
typedef SceneImpl<Hy, MappedView<Hy, PointView<Hy>, Moebius>, ObjectVec<Hy, MappedObject<Hy, HyTiledChoice, Moebius>>,
                  ConstBg>
    SceneHyTiled;
// main/examples/eu.rs:30-44,71-122: Choice{Plane, Sphere, Cube},
// Mixture{Colored<Lambertian>, Specular, Colored<Refractive>}, Shift3 object maps,
// Homogenous3 camera, gradient background, H = 4 in the example.
typedef Mixture<Component<Colored<Lambertian>>, Component<Specular>, Component<Colored<Refractive>>> EuGradMaterial;
typedef SceneImpl<Eu, MappedView<Eu, PointView<Eu>, Homogenous3>,
                  ObjectVec<Eu, MappedObject<Eu, Covered<Eu, ShapeChoice<Eu, PlaneEu, Sphere, Cube>, EuGradMaterial>, Shift3>>,
                  GradBg>
    SceneEuGradient;
}  // namespace htg

// ============================================================================ NVRTC / driver
namespace {

// Header texts for NVRTC (generated from ht_math.cuh, ht_bound.cuh and ht_generic.cuh at build time).
#include "generated/nvrtc_headers.inc"

typedef int (*nvrtcCreateProgram_t)(void **, const char *, const char *, int, const char *const *, const char *const *);
typedef int (*nvrtcAddNameExpression_t)(void *, const char *);
typedef int (*nvrtcCompileProgram_t)(void *, int, const char *const *);
typedef int (*nvrtcGetProgramLogSize_t)(void *, size_t *);
typedef int (*nvrtcGetProgramLog_t)(void *, char *);
typedef int (*nvrtcGetCUBINSize_t)(void *, size_t *);
typedef int (*nvrtcGetCUBIN_t)(void *, char *);
typedef int (*nvrtcGetLoweredName_t)(void *, const char *, const char **);
typedef int (*nvrtcDestroyProgram_t)(void **);

struct Nvrtc {
    bool ok = false;
    std::string error;
    nvrtcCreateProgram_t create = nullptr;
    nvrtcAddNameExpression_t add_name = nullptr;
    nvrtcCompileProgram_t compile = nullptr;
    nvrtcGetProgramLogSize_t log_size = nullptr;
    nvrtcGetProgramLog_t log = nullptr;
    nvrtcGetCUBINSize_t cubin_size = nullptr;
    nvrtcGetCUBIN_t cubin = nullptr;
    nvrtcGetLoweredName_t lowered = nullptr;
    nvrtcDestroyProgram_t destroy = nullptr;
};

Nvrtc &nvrtc() {
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void *h = nullptr;
        for (const char *nm : names) {
            h = dlopen(nm, RTLD_NOW | RTLD_LOCAL);
            if (h) break;
        }
        if (!h) {
            n.error = "libnvrtc not found (dlopen libnvrtc.so.12)";
            return;
        }
        n.create = (nvrtcCreateProgram_t)dlsym(h, "nvrtcCreateProgram");
        n.add_name = (nvrtcAddNameExpression_t)dlsym(h, "nvrtcAddNameExpression");
        n.compile = (nvrtcCompileProgram_t)dlsym(h, "nvrtcCompileProgram");
        n.log_size = (nvrtcGetProgramLogSize_t)dlsym(h, "nvrtcGetProgramLogSize");
        n.log = (nvrtcGetProgramLog_t)dlsym(h, "nvrtcGetProgramLog");
        n.cubin_size = (nvrtcGetCUBINSize_t)dlsym(h, "nvrtcGetCUBINSize");
        n.cubin = (nvrtcGetCUBIN_t)dlsym(h, "nvrtcGetCUBIN");
        n.lowered = (nvrtcGetLoweredName_t)dlsym(h, "nvrtcGetLoweredName");
        n.destroy = (nvrtcDestroyProgram_t)dlsym(h, "nvrtcDestroyProgram");
        n.ok = n.create && n.add_name && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.lowered &&
               n.destroy;
        if (!n.ok) n.error = "libnvrtc lacks an expected symbol";
    });
    return n;
}

typedef CUresult (*cuModuleLoadData_t)(CUmodule *, const void *);
typedef CUresult (*cuModuleGetFunction_t)(CUfunction *, CUmodule, const char *);
typedef CUresult (*cuModuleUnload_t)(CUmodule);
typedef CUresult (*cuModuleGetGlobal_t)(CUdeviceptr *, size_t *, CUmodule, const char *);
typedef CUresult (*cuLaunchKernel_t)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                                     CUstream, void **, void **);

struct Driver {
    bool ok = false;
    cuModuleLoadData_t load = nullptr;
    cuModuleGetFunction_t get = nullptr;
    cuModuleUnload_t unload = nullptr;
    cuLaunchKernel_t launch = nullptr;
    cuModuleGetGlobal_t global = nullptr;
};

Driver &driver() {
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuModuleLoadData", &p, cudaEnableDefault, &q) == cudaSuccess) d.load = (cuModuleLoadData_t)p;
        if (cudaGetDriverEntryPoint("cuModuleGetFunction", &p, cudaEnableDefault, &q) == cudaSuccess) d.get = (cuModuleGetFunction_t)p;
        if (cudaGetDriverEntryPoint("cuModuleUnload", &p, cudaEnableDefault, &q) == cudaSuccess) d.unload = (cuModuleUnload_t)p;
        if (cudaGetDriverEntryPoint("cuLaunchKernel", &p, cudaEnableDefault, &q) == cudaSuccess) d.launch = (cuLaunchKernel_t)p;
        if (cudaGetDriverEntryPoint("cuModuleGetGlobal", &p, cudaEnableDefault, &q) == cudaSuccess) d.global = (cuModuleGetGlobal_t)p;
        d.ok = d.load && d.get && d.unload && d.launch && d.global;
    });
    return d;
}

}  // namespace

// ============================================================================ programs
struct GenericProgram {
    const void *static_kernel = nullptr;   // built-in: render_generic<Scene, W>
    CUmodule module = nullptr;              // NVRTC: the loaded cubin
    CUfunction kernel = nullptr;
    uint64_t min_size = 0;                  // serialized size of the scene without its dynamic part
    std::string type_expr;
};

int generic_program_create(int recipe, int address_width, GenericProgram **out) {
    GenericProgram *g = new GenericProgram();
    if (recipe == HTC_RECIPE_HY_TILED) {
        g->static_kernel = address_width == 64 ? (const void *)render_generic<SceneHyTiled, 8>
                                               : (const void *)render_generic<SceneHyTiled, 4>;
        g->min_size = address_width == 64 ? SceneHyTiled::static_size<8>() : SceneHyTiled::static_size<4>();
    } else {
        g->static_kernel = address_width == 64 ? (const void *)render_generic<SceneEuGradient, 8>
                                               : (const void *)render_generic<SceneEuGradient, 4>;
        g->min_size = address_width == 64 ? SceneEuGradient::static_size<8>() : SceneEuGradient::static_size<4>();
    }
    htg_tiling_init<<<1, 1>>>();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(e, "htg_tiling_init");
    }
    *out = g;
    return HTC_OK;
}

// Compiles render_generic<type_expr, W> (plus the static size of the scene type) with NVRTC.
int generic_program_build(const char *type_expr, int address_width, char *log, size_t log_len, GenericProgram **out) {
    if (log && log_len) log[0] = 0;
    Nvrtc &n = nvrtc();
    if (!n.ok) return fail(HTC_ERR_UNSUPPORTED, n.error);
    Driver &d = driver();
    if (!d.ok) return fail(HTC_ERR_UNSUPPORTED, "CUDA driver entry points unavailable");
    const int W = address_width == 64 ? 8 : 4;
    std::string src = "#include \"ht_generic.cuh\"\nnamespace htg {\ntypedef " + std::string(type_expr) +
                      " UserScene;\n}\nextern \"C\" __device__ unsigned long long htg_static_size = htg::UserScene::static_size<" +
                      std::to_string(W) + ">();\n";
    const std::string kname = "&htg::render_generic<htg::UserScene, " + std::to_string(W) + ">";
    void *prog = nullptr;
    const char *hdr_src[] = {k_header_ht_math, k_header_ht_bound, k_header_ht_generic};
    const char *hdr_name[] = {"ht_math.cuh", "ht_bound.cuh", "ht_generic.cuh"};
    if (n.create(&prog, src.c_str(), "user_scene.cu", 3, hdr_src, hdr_name) != 0) return fail(HTC_ERR_CUDA, "nvrtcCreateProgram failed");
    n.add_name(prog, kname.c_str());
    const char *opts[] = {"-arch=sm_100a", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
                          "-ftz=false", "-lineinfo", "-default-device"};
    const int rc = n.compile(prog, (int)(sizeof(opts) / sizeof(opts[0])), opts);
    size_t ls = 0;
    n.log_size(prog, &ls);
    std::string text(ls, '\0');
    if (ls) n.log(prog, &text[0]);
    if (log && log_len) {
        const size_t k = text.size() < log_len - 1 ? text.size() : log_len - 1;
        std::memcpy(log, text.data(), k);
        log[k] = 0;
    }
    if (rc != 0) {
        n.destroy(&prog);
        return fail(HTC_ERR_INVALID, "scene type failed to compile: " + text.substr(0, 2000));
    }
    const char *lowered = nullptr;
    n.lowered(prog, kname.c_str(), &lowered);
    const std::string kernel_name = lowered ? lowered : "";
    size_t cs = 0;
    n.cubin_size(prog, &cs);
    std::vector<char> cubin(cs);
    if (cs) n.cubin(prog, cubin.data());
    n.destroy(&prog);
    if (!cs || kernel_name.empty()) return fail(HTC_ERR_CUDA, "NVRTC produced no cubin");

    GenericProgram *g = new GenericProgram();
    g->type_expr = type_expr;
    cudaFree(nullptr);   // the runtime's primary context becomes current on this thread
    CUresult r = d.load(&g->module, cubin.data());
    if (r == CUDA_SUCCESS) r = d.get(&g->kernel, g->module, kernel_name.c_str());
    CUfunction init = nullptr;
    if (r == CUDA_SUCCESS) r = d.get(&init, g->module, "htg_tiling_init");
    if (r == CUDA_SUCCESS) r = d.launch(init, 1, 1, 1, 1, 1, 1, 0, nullptr, nullptr, nullptr);
    if (r != CUDA_SUCCESS) {
        if (g->module) d.unload(g->module);
        delete g;
        return fail(HTC_ERR_CUDA, "loading the compiled scene program failed (CUresult " + std::to_string((int)r) + ")");
    }
    // The static size of the scene type is a __device__ constant of the module.
    CUdeviceptr gp = 0;
    size_t gbytes = 0;
    if (d.global(&gp, &gbytes, g->module, "htg_static_size") != CUDA_SUCCESS || gbytes != sizeof(uint64_t)) {
        d.unload(g->module);
        delete g;
        return fail(HTC_ERR_CUDA, "compiled scene program lacks htg_static_size");
    }
    cudaError_t e = cudaMemcpy(&g->min_size, reinterpret_cast<const void *>(gp), sizeof(uint64_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        d.unload(g->module);
        delete g;
        return cuda_fail(e, "htg_tiling_init");
    }
    *out = g;
    return HTC_OK;
}

void generic_program_destroy(GenericProgram *g) {
    if (!g) return;
    if (g->module) driver().unload(g->module);
    delete g;
}

int generic_render(GenericProgram *g, uint32_t W, uint32_t H, uint32_t hops, uint32_t flags, const void *scene,
                   size_t scene_size, float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats, uint32_t *d_err,
                   void *stream) {
    if (scene_size < g->min_size) return fail(HTC_ERR_SCENE, "scene buffer is smaller than the scene type's fixed part");
    const uint64_t pixels = (uint64_t)W * H;
    const unsigned blocks = (unsigned)((pixels + 127) / 128);
    const uint8_t *sc = reinterpret_cast<const uint8_t *>(scene);
    uint64_t ss = scene_size;
    float4 *cv = reinterpret_cast<float4 *>(canvas);
    unsigned long long *st = reinterpret_cast<unsigned long long *>(stats);
    void *args[] = {(void *)&sc, (void *)&ss, (void *)&W, (void *)&H, (void *)&hops, (void *)&passes,
                    (void *)&flags, (void *)&cv, (void *)&seeds, (void *)&st, (void *)&d_err};
    if (g->static_kernel) {
        HTC_CUDA(cudaLaunchKernel(g->static_kernel, dim3(blocks), dim3(128), args, 0, reinterpret_cast<cudaStream_t>(stream)));
        return HTC_OK;
    }
    CUresult r = driver().launch(g->kernel, blocks, 1, 1, 128, 1, 1, 0, reinterpret_cast<CUstream>(stream), args, nullptr);
    if (r != CUDA_SUCCESS) return fail(HTC_ERR_CUDA, "cuLaunchKernel failed (CUresult " + std::to_string((int)r) + ")");
    return HTC_OK;
}

uint64_t generic_min_size(const GenericProgram *g) { return g->min_size; }
