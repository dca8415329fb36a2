// cud_mttkrp_noalloc: the MTTKRP entry point for callers that cannot allocate
// device memory -- code running where cudaMalloc is forbidden or unsafe, such
// as inside a custom allocator's own hooks (a cudaMalloc there re-enters the
// allocator), or a process whose device memory is entirely owned and
// pre-carved by its host framework.  The call launches kernels on the
// caller's stream, so it is not for stream callbacks (cudaLaunchHostFunc),
// where CUDA forbids API calls.  The regular cud_mttkrp draws its split-contraction workspace
// from a growing per-device arena (cudaMalloc on first use or growth); this
// variant runs the same kernels with the workspace taken from a fixed
// file-scope __device__ array instead, and calls no allocating routine.
//
// Limits and sharing:
//  * the array holds kNoAllocScratchBytes (32 MiB); a call whose workspace
//    (split partials: splits x R x I_mode floats, plus 256 bytes of flags)
//    would not fit is rejected with CUD_ERR_INVALID_ARGUMENT and a message
//    from cud_last_error_detail();
//  * every GPU that loads this module holds the array until process exit;
//    under lazy module loading (CUDA_MODULE_LOADING=LAZY, the CUDA 12.2+
//    default) the module -- and with it the 32 MiB -- is loaded by the first
//    call on a device, so that call belongs at start-up, while the memory is
//    free;
//  * all calls on a device share the one array, which keeps the last call's
//    contents -- each call rewrites everything it reads (the kernels
//    overwrite every partial and clear their error flag), but calls whose
//    execution overlaps on the GPU (different streams, no ordering between
//    them) race on it and must be serialised by the caller;
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress, with that device current); make that first call
//    before any stream capture.
#include <mutex>
#include <stdio.h>

#include "kernels.cuh"

namespace cud {

constexpr size_t kNoAllocScratchBytes = 32u << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {nullptr};

// Device address of g_noalloc_scratch on the current device (resolved once
// per device; in host code the symbol's name is only a host-side handle).
int noalloc_scratch(void **out) {
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUD_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cud_mttkrp_noalloc cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return CUD_OK;
}

}  // namespace

}  // namespace cud

using namespace cud;

extern "C" int cud_mttkrp_noalloc(const float *X, int order, const long *dims,
                                  const float *const *U, int mode, long R, float *out,
                                  int precision, void *stream) {
    if (order < 2 || order > kMaxOrder || !dims || mode < 0 || mode >= order || R <= 0 || !X ||
        !U || !out || precision < 0 || precision > CUD_PREC_DEFAULT)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
        if (m != mode && !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
    }
    size_t need = mttkrp_ws_bytes(order, dims, mode, R, precision);
    if (need > kNoAllocScratchBytes) {
        char msg[160];
        snprintf(msg, sizeof(msg),
                 "cud_mttkrp_noalloc: workspace of %zu bytes exceeds the static %zu-byte scratch",
                 need, kNoAllocScratchBytes);
        return set_status_msg(CUD_ERR_INVALID_ARGUMENT, msg);
    }
    void *ws = nullptr;
    int st = noalloc_scratch(&ws);
    if (st) return set_status(st);
    return set_status(mttkrp_run(X, order, dims, U, mode, R, out, precision, ws, as_stream(stream)));
}
