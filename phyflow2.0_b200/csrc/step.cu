// step.cu -- one step of a resident blob set in a single call: the induced
// velocity at the blobs (FMM on a known tree box, or the direct sum) and the
// M4' remesh with the window found on the device, with no host
// synchronisation.  A serving loop makes one call per request instead of a
// dozen small ones.  pf_step_graph_* capture that call once into a CUDA graph
// and replay it with one graph launch per step (no launch gaps between the
// step's ~35 kernels and memsets).
#include <cmath>
#include <new>

#include "fmm_api.cuh"

extern "C" pf_status pf_blob_step(pf_ctx *ctx, const pf_step *s, void *stream) {
    PF_RANGE("pf_blob_step");
    pf::clear_error();
    PF_CHECK_ARG(ctx != nullptr, "pf_blob_step: NULL context");
    PF_CHECK_ARG(s != nullptr, "pf_blob_step: NULL step");
    PF_CHECK_ARG(s->method == PF_FMM_METHOD || s->method == PF_DIRECT_METHOD,
                 "pf_blob_step: method must be PF_FMM_METHOD or PF_DIRECT_METHOD");
    PF_CHECK_ARG(s->leaf_level == 0 ||
                     (s->leaf_level >= 2 && s->leaf_level <= pf::fmmx::MAX_LEVEL),
                 "pf_blob_step: leaf level must be 0 (auto) or in [2, %d]", pf::fmmx::MAX_LEVEL);
    PF_CHECK_ARG(s->n >= 0 && s->n < ((int64_t)1 << 31), "pf_blob_step: bad n");
    if (s->method == PF_DIRECT_METHOD) {
        PF_TRY(pf_velocity_direct(ctx, s->n, s->x, s->y, s->g, s->n, s->x, s->y, s->ksigmasqr,
                                  s->vx, s->vy, stream));
    } else {
        int L0, np0, kb0;
        pf::fmmx::tuning_get(&L0, &np0, &kb0);
        pf::fmmx::tuning_set(s->leaf_level, 0, 1);
        const pf_status st = pf_velocity_fmm_box(ctx, s->n, s->x, s->y, s->g, s->n, s->x, s->y,
                                                 s->ksigmasqr, s->xopt, s->cutoff, s->tol, 35,
                                                 s->box, s->vx, s->vy, stream);
        pf::fmmx::tuning_set(L0, np0, kb0);
        PF_TRY(st);
    }
    return pf_remesh_async(ctx, s->n, s->x, s->y, s->g, s->h, s->xb0, s->yb0, s->c,
                           s->max_base_cells, s->capacity, s->x_out, s->y_out, s->g_out, nullptr,
                           nullptr, s->n_out_dev, s->status_dev, nullptr, s->moments_dev,
                           stream);
}

// ---------------------------------------------------------------------------
// A resident set's step as one CUDA graph.  The graph owns a private context:
// its scratch arena and its hold on the FMM plan stay fixed for the graph's
// life, so the captured addresses stay valid whatever other calls do.
struct pf_step_graph {
    pf_ctx *ctx = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
};

static void step_graph_free(pf_step_graph *g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->cap) cudaStreamDestroy(g->cap);
    if (g->ctx) pf_destroy(g->ctx);
    delete g;
}

extern "C" pf_status pf_step_graph_create(pf_ctx *ctx, const pf_step *s, pf_step_graph **out) {
    PF_RANGE("pf_step_graph_create");
    pf::clear_error();
    PF_CHECK_ARG(out != nullptr, "pf_step_graph_create: out is NULL");
    *out = nullptr;
    PF_CHECK_ARG(ctx != nullptr, "pf_step_graph_create: NULL context");
    PF_CHECK_ARG(s != nullptr, "pf_step_graph_create: NULL step");
    pf::DeviceGuard dg(ctx->device);
    pf_step_graph *g = new (std::nothrow) pf_step_graph();
    if (!g) {
        pf::set_error("pf_step_graph_create: host allocation failed");
        return PF_ERR_OOM;
    }
    pf_status st = pf_create(ctx->device, &g->ctx);
    cudaError_t e = cudaSuccess;
    if (st == PF_OK) e = cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking);
    // the inputs may have been written by work queued anywhere on the device
    if (st == PF_OK && e == cudaSuccess) e = cudaDeviceSynchronize();
    // one uncaptured step sizes the arena, builds or finds the FMM plan and
    // checks the arguments; then the same call is captured
    if (st == PF_OK && e == cudaSuccess) st = pf_blob_step(g->ctx, s, g->cap);
    if (st == PF_OK && e == cudaSuccess) e = cudaStreamSynchronize(g->cap);
    if (st == PF_OK && e == cudaSuccess)
        e = cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeThreadLocal);
    if (st == PF_OK && e == cudaSuccess) {
        st = pf_blob_step(g->ctx, s, g->cap);
        cudaGraph_t gr = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(g->cap, &gr);
        g->graph = gr;
        if (st == PF_OK) e = e2;
    }
    if (st == PF_OK && e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    if (st == PF_OK && e == cudaSuccess) e = pf::graph_kernel_nodes(g->graph, &g->kernels);
    if (st != PF_OK || e != cudaSuccess) {
        if (st == PF_OK) {
            pf::set_error("pf_step_graph_create: %s", cudaGetErrorString(e));
            st = PF_ERR_CUDA;
        }
        cudaGetLastError();
        step_graph_free(g);
        return st;
    }
    *out = g;
    return PF_OK;
}

extern "C" pf_status pf_step_graph_launch(pf_step_graph *g, void *stream) {
    PF_RANGE("pf_step_graph_launch");
    pf::clear_error();
    PF_CHECK_ARG(g != nullptr, "pf_step_graph_launch: NULL graph");
    pf::DeviceGuard dg(g->ctx->device);
    PF_CUDA_TRY(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
    pf::count_launches((uint64_t)g->kernels);
    return PF_OK;
}

extern "C" pf_status pf_step_graph_kernels(const pf_step_graph *g, int64_t *kernels) {
    pf::clear_error();
    PF_CHECK_ARG(g != nullptr && kernels != nullptr, "pf_step_graph_kernels: NULL argument");
    *kernels = g->kernels;
    return PF_OK;
}

extern "C" pf_status pf_step_graph_destroy(pf_step_graph *g) {
    pf::clear_error();
    if (!g) return PF_OK;
    pf::DeviceGuard dg(g->ctx->device);
    // pf_destroy of the private context waits for the device first
    step_graph_free(g);
    return PF_OK;
}
