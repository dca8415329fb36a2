// Shared plumbing for the B200 dense CP/Tucker library: status codes, the
// thread-local last-error side channel of the legacy void entry points, launch
// helpers and the per-device scratch arena.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <stddef.h>
#include <algorithm>

#include "../../include/cudecompose_c.h"

namespace cud {

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

// Records `st` as this thread's last status (read by cud_get_last_error) and
// returns it unchanged, so entry points can `return set_status(...)`.
int set_status(int st);

// Records `st` with a detail message (read by cud_last_error_detail).
int set_status_msg(int st, const char *msg);

// Maps a CUDA runtime error to a library status, recording the CUDA message.
int cuda_status(cudaError_t e, const char *where);

#define CUD_CHECK(call)                                              \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return ::cud::cuda_status(e_, #call); \
    } while (0)

#define CUD_CHECK_LAUNCH(where)                                      \
    do {                                                             \
        cudaError_t e_ = cudaGetLastError();                         \
        if (e_ != cudaSuccess) return ::cud::cuda_status(e_, where); \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

inline unsigned blocks_for(long n, int threads, long cap = 148L * 16) {
    long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

// Scratch arena: one growing device buffer per (device, slot), kept until
// process exit.  Growth frees the old buffer, which synchronises the device,
// so callers size their workspace before any stream capture.
void *scratch(int slot, size_t bytes, int *status);

enum ScratchSlot {
    kSlotReduce = 0,    // reduction partials (rse, norms)
    kSlotMttkrp = 1,    // split-K MTTKRP partials
    kSlotTmp0 = 2,      // general temporaries
    kSlotTmp1 = 3,
    kSlotTmp2 = 4,
    kSlotEig = 5,       // eigensolver work
    kSlotGram = 6,      // factor Gram partials
    kNumSlots = 8
};

// Pinned host scalar buffer (for device->host reads of norms and fits).
double *pinned_scalars();

// Measurement hooks (runtime.cu): a CUDA event pair around a main kernel
// when timing is enabled (cud_prof_enable); prof_begin returns -1 when off.
int prof_begin(cudaStream_t s);
void prof_end(int k, cudaStream_t s);

// A launch configuration with programmatic stream serialization: the kernel
// may start while the previous kernel on the stream finishes; it must call
// griddepcontrol.wait before it reads that kernel's output.
struct PdlLaunch {
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg;
    PdlLaunch(unsigned grid, unsigned block, size_t smem, cudaStream_t s) {
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg = cudaLaunchConfig_t{};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

}  // namespace cud
