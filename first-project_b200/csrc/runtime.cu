// Status side channel, scratch arena and pinned host scalars.
#include <atomic>
#include <mutex>
#include <stdio.h>
#include <string.h>

#include "common.cuh"

namespace cud {

static thread_local int t_last_status = CUD_OK;
static thread_local char t_last_detail[256] = {0};

int set_status(int st) {
    t_last_status = st;
    if (st == CUD_OK) t_last_detail[0] = 0;
    return st;
}

int set_status_msg(int st, const char *msg) {
    t_last_status = st;
    snprintf(t_last_detail, sizeof(t_last_detail), "%s", msg ? msg : "");
    return st;
}

int cuda_status(cudaError_t e, const char *where) {
    snprintf(t_last_detail, sizeof(t_last_detail), "%s: %s", where, cudaGetErrorString(e));
    int st = (e == cudaErrorMemoryAllocation) ? CUD_ERR_NO_MEMORY : CUD_ERR_CUDA;
    t_last_status = st;
    return st;
}

struct Arena {
    void *ptr[kNumSlots] = {nullptr};
    size_t size[kNumSlots] = {0};
};

static std::mutex g_arena_mu;
static Arena g_arena[64];

void *scratch(int slot, size_t bytes, int *status) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || slot < 0 ||
        slot >= kNumSlots) {
        if (status) *status = CUD_ERR_CUDA;
        return nullptr;
    }
    if (bytes == 0) bytes = 256;
    std::lock_guard<std::mutex> lk(g_arena_mu);
    Arena &a = g_arena[dev];
    if (a.size[slot] < bytes) {
        if (a.ptr[slot]) cudaFree(a.ptr[slot]);
        a.ptr[slot] = nullptr;
        a.size[slot] = 0;
        size_t want = bytes + bytes / 4;
        want = (want + 4095) & ~size_t(4095);
        cudaError_t e = cudaMalloc(&a.ptr[slot], want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            if (status) *status = cuda_status(e, "scratch cudaMalloc");
            return nullptr;
        }
        a.size[slot] = want;
    }
    if (status) *status = CUD_OK;
    return a.ptr[slot];
}

double *pinned_scalars() {
    static thread_local double *p = nullptr;
    if (!p) {
        if (cudaMallocHost(&p, 64 * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
    }
    return p;
}

// Kernel timing for measurement (off unless cud_prof_enable turned it on):
// the MTTKRP entry points bracket their main kernel with a pair of CUDA
// events recorded on the call's stream (not while the stream is being
// captured into a graph).  Up to kProfPairs pairs are kept until read.
constexpr int kProfPairs = 256;
static std::mutex g_prof_mu;
static std::atomic<bool> g_prof_on{false};  // read by every MTTKRP call without the lock
static int g_prof_n = 0;
static cudaEvent_t g_prof_ev[2 * kProfPairs];
static bool g_prof_made = false;

int prof_begin(cudaStream_t s) {
    if (!g_prof_on) return -1;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return -1;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof_made || g_prof_n >= kProfPairs) return -1;
    const int k = g_prof_n++;
    if (cudaEventRecord(g_prof_ev[2 * k], s) != cudaSuccess) return -1;
    return k;
}

void prof_end(int k, cudaStream_t s) {
    if (k >= 0) cudaEventRecord(g_prof_ev[2 * k + 1], s);
}

}  // namespace cud

extern "C" int cud_prof_enable(int on) {
    using namespace cud;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (on && !g_prof_made) {
        for (int i = 0; i < 2 * kProfPairs; i++)
            if (cudaEventCreate(&g_prof_ev[i]) != cudaSuccess) return set_status(CUD_ERR_CUDA);
        g_prof_made = true;
    }
    g_prof_on = on != 0;
    g_prof_n = 0;
    return set_status(CUD_OK);
}

extern "C" int cud_prof_kernel_times(float *ms, int max_n, int *count) {
    using namespace cud;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    int n = 0;
    for (int k = 0; k < g_prof_n; k++) {
        if (cudaEventSynchronize(g_prof_ev[2 * k + 1]) != cudaSuccess) return set_status(CUD_ERR_CUDA);
        float t = 0.f;
        if (cudaEventElapsedTime(&t, g_prof_ev[2 * k], g_prof_ev[2 * k + 1]) != cudaSuccess)
            return set_status(CUD_ERR_CUDA);
        if (ms && n < max_n) ms[n] = t;
        n++;
    }
    g_prof_n = 0;
    if (count) *count = n;
    return set_status(CUD_OK);
}

extern "C" int cud_get_last_error(void) { return cud::t_last_status; }

extern "C" const char *cud_last_error_detail(void) { return cud::t_last_detail; }

extern "C" const char *cud_status_string(int status) {
    switch (status) {
        case CUD_OK: return "ok";
        case CUD_ERR_INVALID_ARGUMENT: return "invalid argument";
        case CUD_ERR_CUDA: return "CUDA runtime error";
        case CUD_ERR_NO_MEMORY: return "out of device memory";
        case CUD_ERR_NOT_CONVERGED: return "iteration limit reached";
        case CUD_ERR_UNSUPPORTED: return "unsupported shape or precision";
        case CUD_ERR_SINGULAR: return "singular normal equations (pseudo-inverse used)";
        case CUD_ERR_DEVICE_TIMEOUT: return "bounded device wait expired";
        default: return "unknown status";
    }
}
