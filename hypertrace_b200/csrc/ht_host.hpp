// ht_host.hpp -- host-side helpers shared by the translation units of libhtcuda.so:
// the thread-local last-error message and the status helpers of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

extern thread_local std::string g_last_error;

inline int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
inline int cuda_fail(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return HTC_ERR_CUDA;
}
#define HTC_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// Generic scene programs (htgeneric.cu).
struct GenericProgram;
int generic_program_create(int recipe, int address_width, GenericProgram **out);
int generic_program_build(const char *type_expr, int address_width, char *log, size_t log_len, GenericProgram **out);
void generic_program_destroy(GenericProgram *g);
int generic_render(GenericProgram *g, uint32_t W, uint32_t H, uint32_t hops, uint32_t flags, const void *scene,
                   size_t scene_size, float *canvas, uint32_t *seeds, uint32_t passes, uint64_t *stats, uint32_t *d_err,
                   void *stream);
uint64_t generic_min_size(const GenericProgram *g);
