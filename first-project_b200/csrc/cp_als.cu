// CP-ALS driver: a reusable plan (workspace + captured per-sweep CUDA graph)
// and the one-shot cud_cp_als built on it.
//
// One sweep = for each mode n: MTTKRP_n (native layout) -> V^-1 from the
// Hadamard product of the other factors' FP64 Grams (Gauss-Jordan inverse
// with SPD pivots, Jacobi pseudo-inverse fallback) -> U_n = M V^-1 -> Gram of U_n; then the fit from the identity
// ||X - Xhat||^2 = ||X||^2 - 2 <M_N, U_N> + sum prod_m G_m.  The sweep is
// captured once into a CUDA graph and replayed; the plan owns every buffer
// the graph touches.  Mirrors the update order and equations of
// src/cp_als.cu:44-119 and src/cp4_als.cu:64-164, without their per-sweep
// allocations and device synchronisations.
#include <mutex>
#include <vector>
#include <curand.h>

#include "kernels.cuh"
#include "solve.cuh"

using namespace cud;

struct cud_cp_plan_s {
    int order = 0;
    long dims[kMaxOrder] = {0};
    long R = 0;
    const float *X = nullptr;
    float *U[kMaxOrder] = {nullptr};
    cud_cp_options opt;
    int device = 0;
    double normx2 = 0.0;
    // device memory owned by the plan
    char *mem = nullptr;
    float *M = nullptr;
    float *Mraw = nullptr;  // fused layout: where a CUDA-core MTTKRP writes (the update writes M)
    double *G = nullptr, *Vinv = nullptr, *work = nullptr, *fit = nullptr;
    int *fallbacks = nullptr;
    unsigned *counter = nullptr;  // ticket of the fused update's last-CTA reduction
    double *gpart = nullptr;      // its per-CTA partial Grams
    void *ws = nullptr;
    double *hbuf = nullptr;  // pinned
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // fused layout: kMultiSweeps sweeps in one graph, so each sweep's last
    // Gram and fit (side stream) run beside the next sweep's first MTTKRP
    cudaGraph_t graph_multi = nullptr;
    cudaGraphExec_t exec_multi = nullptr;
    // the Delta-fit loop on the device: a graph whose WHILE node replays one
    // sweep and k_loop_cond until the sweep limit or the tolerance stops it
    cudaGraph_t graph_loop = nullptr;
    cudaGraphExec_t exec_loop = nullptr;
    struct LoopState *loop = nullptr;  // device
    // the R x R inverse of mode n depends only on the other modes' Grams, so
    // it runs on a second stream beside the mode-n MTTKRP
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int kernels_per_sweep = -1;
    size_t reset_bytes = 0;  // fit scalars, fallback count and update ticket (zeroed by a refresh)
    bool fused = false;      // sweep layout (fused_sweep_pays)
};

// State of the device-side sweep loop (plan memory, set before each launch).
struct LoopState {
    int done;         // sweeps run by this launch
    int max_sweeps;
    int check_every;  // the tolerance is judged after every check_every-th sweep
    int pad;
    double tol;
};

namespace {

// After each sweep of the loop graph: count it and decide whether the WHILE
// node runs another -- the host loop's rule (stop at the sweep limit, or
// when |fit - fit_prev| < tol at a checked sweep from the second on).
__global__ void k_loop_cond(cudaGraphConditionalHandle h, LoopState *st, const double *fit) {
    if (threadIdx.x != 0) return;
    const int d = st->done + 1;
    st->done = d;
    bool more = d < st->max_sweeps;
    if (more && st->tol > 0.0 && d >= 2 && d % st->check_every == 0 && fabs(fit[0] - fit[1]) < st->tol)
        more = false;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

bool valid_dims(int order, const long *dims) {
    if (order < 1 || order > kMaxOrder || !dims) return false;
    for (int m = 0; m < order; m++)
        if (dims[m] <= 0) return false;
    return true;
}

int count_kernel_nodes(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return -1;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return -1;
    int k = 0;
    for (size_t i = 0; i < n; i++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

NormalArgs normal_args(const cud_cp_plan_s *p, int mode) {
    NormalArgs na;
    for (int m = 0; m < p->order; m++) na.G[m] = p->G + (size_t)m * p->R * p->R;
    na.nG = p->order;
    na.mode = mode;
    na.R = (int)p->R;
    na.Vinv = p->Vinv;
    na.work = p->work;
    na.fallbacks = p->fallbacks;
    return na;
}

constexpr int kMultiSweeps = 4;

// The fused sweep (R <= FU_RMAX).  Per mode n, on the main stream: MTTKRP_n
// (split partials left unsummed), then one kernel that sums them and forms
// U_n = M V_n^-1.  On the side stream, beside the next MTTKRP: the Gram of
// U_n, then V_{n+1}^-1 (it needs G_n); after the last mode, its Gram and the
// fit instead, joined at the end of the sweep.  V_0^-1 runs beside MTTKRP_0.
// The main stream waits for the side stream only before each update, and,
// with join_end, at the end of the sweep (a sweep followed by another in the
// same graph leaves the last Gram and fit running beside the next MTTKRP:
// the next update waits for them through the side stream's order).
int enqueue_sweep_fused(cud_cp_plan_s *p, cudaStream_t s, bool join_end) {
    int st;
    const long R = p->R;
    const int N = p->order;
    CUD_CHECK(cudaEventRecord(p->ev_fork, s));
    CUD_CHECK(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    if ((st = normal_inverse(normal_args(p, 0), p->side))) return st;
    CUD_CHECK(cudaEventRecord(p->ev_join, p->side));
    for (int n = 0; n < N; n++) {
        MttkrpParts parts;
        st = mttkrp_run_parts(p->X, N, p->dims, (const float *const *)p->U, n, R, p->Mraw, p->opt.precision, p->ws,
                              s, &parts);
        if (st) return st;
        CUD_CHECK(cudaStreamWaitEvent(s, p->ev_join, 0));
        if ((st = update_from_parts(parts, p->Vinv, p->dims[n], (int)R, p->M, p->U[n], s))) return st;
        CUD_CHECK(cudaEventRecord(p->ev_fork, s));
        CUD_CHECK(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
        UpdateArgs ua;
        ua.M = p->U[n];  // Gram of U_n
        ua.I = p->dims[n];
        ua.R = (int)R;
        // beside the next MTTKRP, whose grid leaves four CTA slots free
        ua.max_blocks = (n + 1 < N) ? 4 : 0;
        ua.G_out = p->G + (size_t)n * R * R;
        ua.gpart = p->gpart;
        ua.counter = p->counter;
        if (n == N - 1) {
            for (int m = 0; m < N; m++) ua.Gall[m] = p->G + (size_t)m * R * R;
            ua.nG = N;
            ua.mode = n;
            ua.normx2 = p->normx2;
            ua.fit_out = p->fit;
            ua.Mfit = p->M;
        }
        if ((st = factor_update(ua, p->side))) return st;
        if (n + 1 < N && (st = normal_inverse(normal_args(p, n + 1), p->side))) return st;
        CUD_CHECK(cudaEventRecord(p->ev_join, p->side));
    }
    if (join_end) CUD_CHECK(cudaStreamWaitEvent(s, p->ev_join, 0));
    return CUD_OK;
}

// The fused sweep lengthens the side stream (the Gram of U_n, then
// V_{n+1}^-1) to take the split reduce and the Gram off the main one.  On
// B200 (BF16x3, ms a sweep, layout 1 / layout 2) it paid from 64 MiB of X
// up: 256^3 R16 0.107 / 0.098, 64^4 R32 0.182 / 0.175, 384^3 R64 0.243 /
// 0.236, 96^4 R16 0.390 / 0.366, 512^3 R64 0.406 / 0.349; below, the side
// stream outlasts the MTTKRP: 128^3 R16 0.076 / 0.083, 192^3 R32 0.129 /
// 0.135.  (Between, the two stay within 5 %: 128^3 R64 0.219 / 0.207,
// 256^3 R64 0.204 / 0.211.)
bool fused_sweep_pays(const cud_cp_plan_s *p) {
    if (p->R > FU_RMAX) return false;
    double xbytes = 4.0;
    for (int m = 0; m < p->order; m++) xbytes *= (double)p->dims[m];
    return xbytes >= 64.0 * 1024 * 1024;
}

int enqueue_sweep(cud_cp_plan_s *p, cudaStream_t s) {
    int st;
    const long R = p->R;
    if (p->fused) return enqueue_sweep_fused(p, s, true);
    for (int n = 0; n < p->order; n++) {
        // fork: V^-1 of mode n on the side stream, concurrent with the MTTKRP
        CUD_CHECK(cudaEventRecord(p->ev_fork, s));
        CUD_CHECK(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
        NormalArgs na;
        for (int m = 0; m < p->order; m++) na.G[m] = p->G + (size_t)m * R * R;
        na.nG = p->order;
        na.mode = n;
        na.R = (int)R;
        na.Vinv = p->Vinv;
        na.work = p->work;
        na.fallbacks = p->fallbacks;
        if ((st = normal_inverse(na, p->side))) return st;
        CUD_CHECK(cudaEventRecord(p->ev_join, p->side));
        st = mttkrp_run(p->X, p->order, p->dims, (const float *const *)p->U, n, R, p->M,
                        p->opt.precision, p->ws, s);
        if (st) return st;
        CUD_CHECK(cudaStreamWaitEvent(s, p->ev_join, 0));
        // join: U_n = M V^-1, its Gram, and after the last mode the fit
        UpdateArgs ua;
        ua.M = p->M;
        ua.Vinv = p->Vinv;
        ua.U = p->U[n];
        ua.I = p->dims[n];
        ua.R = (int)R;
        ua.G_out = p->G + (size_t)n * R * R;
        ua.gpart = p->gpart;
        ua.counter = p->counter;
        if (n == p->order - 1) {
            for (int m = 0; m < p->order; m++) ua.Gall[m] = p->G + (size_t)m * R * R;
            ua.nG = p->order;
            ua.mode = n;
            ua.normx2 = p->normx2;
            ua.fit_out = p->fit;
        }
        if ((st = factor_update(ua, s))) return st;
    }
    return CUD_OK;
}

// Capture needs a stream other than the legacy default one.
struct SideStream {
    cudaStream_t s = nullptr;
    cudaStream_t user = nullptr;
    bool own = false;
    int open(cudaStream_t u) {
        user = u;
        if (u != nullptr && u != cudaStreamLegacy && u != cudaStreamPerThread) {
            s = u;
            return CUD_OK;
        }
        CUD_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        own = true;
        cudaEvent_t ev;
        CUD_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CUD_CHECK(cudaEventRecord(ev, u));
        CUD_CHECK(cudaStreamWaitEvent(s, ev, 0));
        cudaEventDestroy(ev);
        return CUD_OK;
    }
    int close() {
        if (!own || !s) return CUD_OK;
        // later work on the caller's stream orders after ours
        cudaEvent_t ev;
        CUD_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CUD_CHECK(cudaEventRecord(ev, s));
        CUD_CHECK(cudaStreamWaitEvent(user, ev, 0));
        cudaEventDestroy(ev);
        cudaStreamDestroy(s);
        s = nullptr;
        return CUD_OK;
    }
};

}  // namespace

extern "C" void cud_cp_default_options(cud_cp_options *opt) {
    if (!opt) return;
    opt->max_sweeps = 500;
    opt->tol = 0.0;
    opt->precision = CUD_PREC_DEFAULT;
    opt->use_graph = 1;
    opt->check_every = 1;
    opt->target_fit = 0.0;
    opt->sweep_layout = 0;
}

extern "C" int cud_cp_init_curand(int order, const long *dims, long R, float *const *U,
                                  unsigned long long seed, void *stream) {
    if (!valid_dims(order, dims) || R <= 0 || !U) return set_status(CUD_ERR_INVALID_ARGUMENT);
    curandGenerator_t gen;
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS)
        return set_status(CUD_ERR_CUDA);
    int st = CUD_OK;
    if (curandSetStream(gen, as_stream(stream)) != CURAND_STATUS_SUCCESS ||
        curandSetPseudoRandomGeneratorSeed(gen, seed) != CURAND_STATUS_SUCCESS)
        st = CUD_ERR_CUDA;
    for (int m = 1; m < order && st == CUD_OK; m++) {
        if (!U[m]) { st = CUD_ERR_INVALID_ARGUMENT; break; }
        if (curandGenerateUniform(gen, U[m], (size_t)(dims[m] * R)) != CURAND_STATUS_SUCCESS)
            st = CUD_ERR_CUDA;
    }
    curandDestroyGenerator(gen);
    return set_status(st);
}

extern "C" int cud_factor_gram(const float *U, long I, long R, double *G, void *stream) {
    if (I <= 0 || R <= 0 || !U || !G) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(factor_gram(U, I, R, G, as_stream(stream)));
}

extern "C" int cud_cp_solve(const float *M, long I, long R, int order, const double *const *G,
                            int mode, float *U, double *work, void *stream) {
    if (I <= 0 || R <= 0 || R > 160 || order < 2 || order > kMaxOrder || mode < 0 || mode >= order ||
        !M || !G || !U || !work)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    NormalArgs na;
    for (int m = 0; m < order; m++) {
        if (m != mode && !G[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
        na.G[m] = (m == mode) ? G[(mode + 1) % order] : G[m];
    }
    na.nG = order;
    na.mode = mode;
    na.R = (int)R;
    na.Vinv = work;
    na.work = work + R * R;
    na.fallbacks = reinterpret_cast<int *>(work + 3 * R * R);
    int st = normal_inverse(na, s);
    if (st == CUD_OK) st = apply_inverse(M, na.Vinv, I, R, U, s);
    return set_status(st);
}

extern "C" int cud_cp_normal_inverse(long R, int order, const double *const *G, int mode, double *work,
                                     void *stream) {
    if (R <= 0 || R > 160 || order < 2 || order > kMaxOrder || mode < 0 || mode >= order || !G || !work)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    NormalArgs na;
    for (int m = 0; m < order; m++) {
        if (m != mode && !G[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
        na.G[m] = (m == mode) ? G[(mode + 1) % order] : G[m];
    }
    na.nG = order;
    na.mode = mode;
    na.R = (int)R;
    na.Vinv = work;
    na.work = work + R * R;
    na.fallbacks = reinterpret_cast<int *>(work + 3 * R * R);
    return set_status(normal_inverse(na, as_stream(stream)));
}

extern "C" int cud_cp_apply_inverse(const float *M, long I, long R, const double *work, float *U, void *stream) {
    if (I <= 0 || R <= 0 || R > 160 || !M || !work || !U) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(apply_inverse(M, work, I, R, U, as_stream(stream)));
}

extern "C" int cud_cp_fit_terms(const float *M, const float *U, long IR, int order,
                                const double *const *G, long R, double *inner, double *norm_hat2,
                                void *stream) {
    if (!M || !U || IR <= 0 || order < 1 || order > kMaxOrder || !G || R <= 0 || !inner || !norm_hat2)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    int st;
    double *d = (double *)scratch(kSlotReduce, 8 * sizeof(double), &st);
    if (!d) return set_status(st);
    FitArgs fa;
    fa.M = M;
    fa.U = U;
    fa.IR = IR;
    for (int m = 0; m < order; m++) fa.G[m] = G[m];
    fa.nG = order;
    fa.R = (int)R;
    fa.normx2 = 1.0;
    fa.out = d;
    if ((st = fit_eval(fa, s))) return set_status(st);
    double h[4];
    CUD_CHECK(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    *inner = h[2];
    *norm_hat2 = h[3];
    return set_status(CUD_OK);
}

extern "C" int cud_cp_plan_destroy(cud_cp_plan p) {
    if (!p) return set_status(CUD_OK);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->exec_multi) cudaGraphExecDestroy(p->exec_multi);
    if (p->graph_multi) cudaGraphDestroy(p->graph_multi);
    if (p->exec_loop) cudaGraphExecDestroy(p->exec_loop);
    if (p->graph_loop) cudaGraphDestroy(p->graph_loop);
    if (p->side) {
        cudaStreamSynchronize(p->side);
        cudaStreamDestroy(p->side);
    }
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_join) cudaEventDestroy(p->ev_join);
    if (p->mem) cudaFree(p->mem);
    if (p->hbuf) cudaFreeHost(p->hbuf);
    if (prev >= 0) cudaSetDevice(prev);
    delete p;
    return set_status(CUD_OK);
}

// The data-dependent state of a plan, from X and the current factors:
// ||X||^2, the factor Grams, and zeroed fit scalars, fallback count and
// update ticket.  Synchronises the stream (the norm is read on the host).
static int plan_refresh(cud_cp_plan_s *p, cudaStream_t s) {
    long total = 1;
    for (int m = 0; m < p->order; m++) total *= p->dims[m];
    double o[2];
    int st = residual_norms(p->X, nullptr, total, 0, o, s);
    if (st) return st;
    p->normx2 = o[1];
    if (cudaMemsetAsync(p->fit, 0, p->reset_bytes, s) != cudaSuccess) return CUD_ERR_CUDA;
    for (int m = 0; m < p->order && st == CUD_OK; m++)
        st = factor_gram(p->U[m], p->dims[m], p->R, p->G + (size_t)m * p->R * p->R, s);
    return st;
}

// The device-side loop graph (optional: the host loop is kept when the
// driver refuses any step).  Its WHILE node's body is one sweep, as
// enqueue_sweep captures it, then k_loop_cond; the condition is 1 at each
// launch, so the body runs at least once (the caller launches it only for a
// sweep limit >= 1).
void build_loop_graph(cud_cp_plan_s *p, cudaStream_t s) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
    cudaGraphConditionalHandle h = 0;
    cudaGraph_t body = nullptr;
    if (ok) ok = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        ok = cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess;
        if (ok) body = np.conditional.phGraph_out[0];
    }
    if (ok) ok = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                 cudaSuccess;
    if (ok) {
        int cst = enqueue_sweep(p, s);
        if (cst == CUD_OK) {
            k_loop_cond<<<1, 32, 0, s>>>(h, p->loop, p->fit);
            if (cudaGetLastError() != cudaSuccess) cst = CUD_ERR_CUDA;
        }
        cudaGraph_t captured = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &captured);
        ok = cst == CUD_OK && e == cudaSuccess;
    }
    if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    (void)cudaGetLastError();  // a refused step leaves the host loop in place
    if (ok) {
        p->graph_loop = g;
        p->exec_loop = ex;
    } else {
        if (ex) cudaGraphExecDestroy(ex);
        if (g) cudaGraphDestroy(g);
    }
}

extern "C" int cud_cp_plan_create(const float *X, int order, const long *dims, long R,
                                  float *const *U, const cud_cp_options *opt_in, void *stream,
                                  cud_cp_plan *out) {
    if (!out) return set_status(CUD_ERR_INVALID_ARGUMENT);
    *out = nullptr;
    if (!valid_dims(order, dims) || order < 2 || R <= 0 || !X || !U) return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++)
        if (!U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (R > 160) return set_status(CUD_ERR_UNSUPPORTED);
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    if (opt_in) opt = *opt_in;
    if (opt.max_sweeps < 0 || opt.check_every < 0 || opt.precision < 0 || opt.precision > CUD_PREC_DEFAULT ||
        opt.sweep_layout < 0 || opt.sweep_layout > 2)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (opt.check_every == 0) opt.check_every = 1;

    cud_cp_plan_s *p = new cud_cp_plan_s();
    p->order = order;
    p->R = R;
    p->X = X;
    p->opt = opt;
    cudaGetDevice(&p->device);
    long maxd = 0, total = 1;
    size_t wsb = 0;
    for (int m = 0; m < order; m++) {
        p->dims[m] = dims[m];
        p->U[m] = U[m];
        maxd = std::max(maxd, dims[m]);
        total *= dims[m];
    }
    for (int m = 0; m < order; m++) wsb = std::max(wsb, mttkrp_ws_bytes(order, dims, m, R, opt.precision));
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t off_M = 0;
    size_t off_Mr = off_M + up(sizeof(float) * maxd * R);
    size_t off_G = off_Mr + up(sizeof(float) * maxd * R);
    size_t off_V = off_G + up(sizeof(double) * order * R * R);
    size_t off_W = off_V + up(sizeof(double) * R * R);
    size_t off_F = off_W + up(sizeof(double) * 2 * R * R);
    size_t off_C = off_F + up(sizeof(double) * 4);  // fallbacks (int) + counter
    size_t off_L = off_C + 256;                      // loop state
    size_t off_P = off_L + up(sizeof(LoopState));
    size_t off_S = off_P + up(sizeof(double) * update_ws_doubles(maxd, R));
    size_t bytes = off_S + up(wsb);
    cudaError_t e = cudaMalloc((void **)&p->mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cud_cp_plan_destroy(p);
        return set_status(cuda_status(e, "cud_cp_plan_create cudaMalloc"));
    }
    if (cudaMallocHost((void **)&p->hbuf, 8 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        cud_cp_plan_destroy(p);
        return set_status(CUD_ERR_NO_MEMORY);
    }
    p->M = (float *)(p->mem + off_M);
    p->Mraw = (float *)(p->mem + off_Mr);
    p->G = (double *)(p->mem + off_G);
    p->Vinv = (double *)(p->mem + off_V);
    p->work = (double *)(p->mem + off_W);
    p->fit = (double *)(p->mem + off_F);
    p->fallbacks = (int *)(p->mem + off_C);
    p->counter = (unsigned *)(p->mem + off_C + 64);
    p->loop = (LoopState *)(p->mem + off_L);
    p->gpart = (double *)(p->mem + off_P);
    p->ws = p->mem + off_S;
    if (cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        cud_cp_plan_destroy(p);
        return set_status(CUD_ERR_CUDA);
    }

    SideStream ss;
    int st = ss.open(as_stream(stream));
    p->reset_bytes = off_P - off_F;
    p->fused = (opt.sweep_layout == 2 && R <= FU_RMAX) || (opt.sweep_layout == 0 && fused_sweep_pays(p));
    if (st == CUD_OK) st = plan_refresh(p, ss.s);
    if (st == CUD_OK) st = normal_inverse_prepare();
    if (st == CUD_OK && opt.use_graph) {
        if (cudaStreamBeginCapture(ss.s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            st = CUD_ERR_CUDA;
        } else {
            int cst = enqueue_sweep(p, ss.s);
            e = cudaStreamEndCapture(ss.s, &p->graph);
            if (cst) st = cst;
            else if (e != cudaSuccess) st = cuda_status(e, "cp plan capture");
            else {
                e = cudaGraphInstantiate(&p->exec, p->graph, 0);
                if (e != cudaSuccess) st = cuda_status(e, "cp plan instantiate");
                else p->kernels_per_sweep = count_kernel_nodes(p->graph);
            }
        }
        if (st == CUD_OK && p->fused) {
            if (cudaStreamBeginCapture(ss.s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                st = CUD_ERR_CUDA;
            } else {
                int cst = CUD_OK;
                for (int k = 0; k < kMultiSweeps && cst == CUD_OK; k++)
                    cst = enqueue_sweep_fused(p, ss.s, k == kMultiSweeps - 1);
                e = cudaStreamEndCapture(ss.s, &p->graph_multi);
                if (cst) st = cst;
                else if (e != cudaSuccess) st = cuda_status(e, "cp plan capture (multi)");
                else if ((e = cudaGraphInstantiate(&p->exec_multi, p->graph_multi, 0)) != cudaSuccess)
                    st = cuda_status(e, "cp plan instantiate (multi)");
            }
        }
        if (st == CUD_OK) build_loop_graph(p, ss.s);
    }
    if (st == CUD_OK && cudaStreamSynchronize(ss.s) != cudaSuccess) st = CUD_ERR_CUDA;
    ss.close();
    if (st != CUD_OK) {
        cud_cp_plan_destroy(p);
        return set_status(st);
    }
    *out = p;
    return set_status(CUD_OK);
}

extern "C" int cud_cp_plan_run(cud_cp_plan p, int sweeps, void *stream) {
    if (!p || sweeps < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    for (int i = 0; i < sweeps;) {
        if (p->exec_multi && sweeps - i >= kMultiSweeps) {
            CUD_CHECK(cudaGraphLaunch(p->exec_multi, s));
            i += kMultiSweeps;
        } else if (p->exec) {
            CUD_CHECK(cudaGraphLaunch(p->exec, s));
            i++;
        } else {
            int st = enqueue_sweep(p, s);
            if (st) return set_status(st);
            i++;
        }
    }
    return set_status(CUD_OK);
}

extern "C" int cud_cp_plan_fit(cud_cp_plan p, double *fit, double *fit_prev, void *stream) {
    if (!p) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    CUD_CHECK(cudaMemcpyAsync(p->hbuf, p->fit, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaMemcpyAsync(p->hbuf + 2, p->fallbacks, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    if (fit) *fit = p->hbuf[0];
    if (fit_prev) *fit_prev = p->hbuf[1];
    return set_status(CUD_OK);
}

extern "C" int cud_cp_plan_true_fit(cud_cp_plan p, double *fit, void *stream) {
    if (!p) return set_status(CUD_ERR_INVALID_ARGUMENT);
    // ||X||^2 is the plan's (FP64, from its refresh): the residual pass
    // only sums (x - xh)^2
    double res2 = 0.0;
    int st = cp_residual_host(p->X, p->order, p->dims, const_cast<const float *const *>(p->U), p->R, false, &res2,
                              nullptr, as_stream(stream));
    if (st) return set_status(st);
    const double x2 = p->normx2;
    if (fit) *fit = 1.0 - sqrt(res2) / sqrt(x2 > 0.0 ? x2 : 1.0);
    return set_status(CUD_OK);
}

extern "C" int cud_cp_plan_info(cud_cp_plan p, int *kernels_per_sweep, int *fallbacks) {
    if (!p) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (kernels_per_sweep) *kernels_per_sweep = p->kernels_per_sweep;
    if (fallbacks) {
        int v = 0;
        CUD_CHECK(cudaMemcpy(&v, p->fallbacks, sizeof(int), cudaMemcpyDeviceToHost));
        *fallbacks = v;
    }
    return set_status(CUD_OK);
}

// The one-shot cud_cp_als keeps its last plan for the next call with the
// same device, tensor and factor pointers, shape, rank, precision and graph
// setting: the buffers and the captured sweep graph carry over (the graph
// holds pointers, not data), and plan_refresh recomputes ||X||^2 and the
// Grams from the data.  One plan is kept (its memory stays allocated until
// a call with other arguments replaces it, or cud_cp_als_release frees it);
// concurrent calls each take or build their own.
namespace {
std::mutex g_cache_mu;
cud_cp_plan g_cache = nullptr;

bool plan_matches(const cud_cp_plan_s *p, const float *X, int order, const long *dims, long R, float *const *U,
                  const cud_cp_options &opt) {
    int dev = -1;
    cudaGetDevice(&dev);
    if (!p || p->device != dev || p->X != X || p->order != order || p->R != R ||
        p->opt.precision != opt.precision || (p->opt.use_graph != 0) != (opt.use_graph != 0) ||
        p->opt.sweep_layout != opt.sweep_layout)
        return false;
    for (int m = 0; m < order; m++)
        if (p->dims[m] != dims[m] || p->U[m] != U[m]) return false;
    return true;
}
}  // namespace

extern "C" int cud_cp_als_release(void) {
    cud_cp_plan old = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        old = g_cache;
        g_cache = nullptr;
    }
    return cud_cp_plan_destroy(old);
}

extern "C" int cud_cp_als(const float *X, int order, const long *dims, long R, float *const *U,
                          const cud_cp_options *opt_in, cud_cp_result *res, void *stream) {
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    if (opt_in) opt = *opt_in;
    cud_cp_plan p = nullptr;
    int st = CUD_OK;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        if (plan_matches(g_cache, X, order, dims, R, U, opt)) {
            p = g_cache;
            g_cache = nullptr;
        }
    }
    if (p) {
        p->opt = opt;
        SideStream rs;
        st = rs.open(as_stream(stream));
        if (st == CUD_OK) st = plan_refresh(p, rs.s);
        rs.close();
        if (st) {
            cud_cp_plan_destroy(p);
            return set_status(st);
        }
    } else {
        st = cud_cp_plan_create(X, order, dims, R, U, &opt, stream, &p);
        if (st) return set_status(st);
    }
    SideStream ss;
    st = ss.open(as_stream(stream));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    int sweeps = 0;
    double fit = 0.0, fit_prev = 0.0, true_fit = 0.0;
    if (st == CUD_OK) {
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, ss.s);
        int chunk = (opt.tol > 0 || opt.target_fit > 0) ? opt.check_every : opt.max_sweeps;
        if (chunk <= 0) chunk = 1;
        if (p->exec_loop && opt.tol > 0 && opt.target_fit <= 0 && opt.max_sweeps > 0) {
            // the Delta-fit loop runs on the device: no host round trip per check
            LoopState ls = {0, opt.max_sweeps, opt.check_every, 0, opt.tol};
            if (cudaMemcpyAsync(p->loop, &ls, sizeof(ls), cudaMemcpyHostToDevice, ss.s) != cudaSuccess ||
                cudaGraphLaunch(p->exec_loop, ss.s) != cudaSuccess ||
                cudaMemcpyAsync(&ls, p->loop, sizeof(ls), cudaMemcpyDeviceToHost, ss.s) != cudaSuccess ||
                cudaStreamSynchronize(ss.s) != cudaSuccess)
                st = cuda_status(cudaGetLastError(), "cp loop graph");
            sweeps = ls.done;
        }
        while (sweeps < opt.max_sweeps && st == CUD_OK && !(p->exec_loop && opt.tol > 0 && opt.target_fit <= 0)) {
            int n = std::min(chunk, opt.max_sweeps - sweeps);
            st = cud_cp_plan_run(p, n, ss.s);
            sweeps += n;
            if (st == CUD_OK && (opt.tol > 0 || opt.target_fit > 0)) {
                st = cud_cp_plan_fit(p, &fit, &fit_prev, ss.s);
                if (st == CUD_OK && opt.tol > 0 && sweeps >= 2 && fabs(fit - fit_prev) < opt.tol) break;
                // the target is judged on the exact fit: the estimate's
                // cancellation error can exceed the distance to the target
                if (st == CUD_OK && opt.target_fit > 0) {
                    st = cud_cp_plan_true_fit(p, &true_fit, ss.s);
                    if (st == CUD_OK && true_fit >= opt.target_fit) break;
                }
            }
        }
        cudaEventRecord(t1, ss.s);
        if (st == CUD_OK) st = cud_cp_plan_fit(p, &fit, &fit_prev, ss.s);
        if (st == CUD_OK) st = cud_cp_plan_true_fit(p, &true_fit, ss.s);
    }
    if (st == CUD_OK && res) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        res->sweeps = sweeps;
        res->fit = true_fit;
        res->fit_estimate = fit;
        res->fit_prev = fit_prev;
        res->seconds = ms * 1e-3;
        cud_cp_plan_info(p, &res->kernels_per_sweep, &res->fallbacks);
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    ss.close();
    if (st == CUD_OK) {
        // keep this plan for the next call; release the one it replaces
        cud_cp_plan old = nullptr;
        {
            std::lock_guard<std::mutex> lk(g_cache_mu);
            old = g_cache;
            g_cache = p;
        }
        cud_cp_plan_destroy(old);
    } else {
        cud_cp_plan_destroy(p);
    }
    if (st == CUD_OK) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_status(e, "cud_cp_als");
    }
    return set_status(st);
}
