// batch.cu -- many independent blob simulations per launch.
//
// pf_batch_create plans every instance on the host (FMM tree and operators,
// remesh lattice window, method), allocates every buffer, and captures the
// whole step -- velocity of every instance plus its remesh -- into one CUDA
// graph:
//   * instances using the direct sum are evaluated together by ONE persistent
//     kernel that takes (instance, target tile) items from a device counter,
//     largest first (k_direct_batch);
//   * FMM instances and all remesh jobs are spread over library streams
//     (longest-processing-time-first by estimated cost), fork/joined inside
//     the capture, so independent instances overlap on the GPU;
//   * nothing in the graph synchronises with the host or allocates.
// pf_batch_run replays the graph with a single launch.  The reference has no
// counterpart (one simulation per call, src/python/blobs/__blobsClass.py:546-628).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "direct_api.cuh"
#include "fmm_api.cuh"
#include "remesh.cuh"

namespace {

__global__ void k_batch_collect(int32_t *__restrict__ totals, int32_t *__restrict__ bads, int n,
                                int64_t *__restrict__ n_out, int32_t *__restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    n_out[i] = totals[i];
    status[i] = bads[i];
}

struct Job {
    int inst;
    int kind;  // 0 = FMM velocity, 1 = remesh
    double cost;
    size_t scratch;
};

// host copy of the remesh window-left index (same operation order as the device)
int64_t left_index_host(double x, double b0, double h) {
    const double h2 = 2.0 * h, h05 = 0.5 * h;
    volatile double t = ((x - b0) - h2);
    t = t + h05;
    volatile double q = t / h;
    // far outside any admissible window (the caller rejects it); keeps the
    // conversion defined
    if (!(std::fabs(q) < 1e15)) return q > 0 ? ((int64_t)1 << 52) : -((int64_t)1 << 52);
    return (int64_t)std::ceil(q) - 1;
}

}  // namespace

struct pf_batch {
    pf_ctx *ctx = nullptr;
    int n = 0;
    std::vector<pf_batch_instance> inst;
    std::vector<pf::fmmx::Plan *> plans;
    std::vector<int> method;  // resolved
    std::vector<int64_t> ixmin, iymin, nbx, nby;
    int nstreams = 0;
    std::vector<cudaStream_t> streams;
    cudaStream_t direct_stream = nullptr, cap_stream = nullptr;
    std::vector<cudaEvent_t> events;
    std::vector<std::vector<Job>> slot_jobs;
    std::vector<char *> slot_scratch;
    std::vector<size_t> slot_bytes;
    unsigned long long *d_ctr = nullptr;  // FMM_COUNTERS per slot
    pf::DirectInstance *d_dinst = nullptr;
    int2 *d_items = nullptr;
    int n_items = 0;
    int2 *d_red_items = nullptr;  // (instance, tile) reductions of split instances
    int n_red = 0;
    float4 *d_part = nullptr;     // partial sums of all split instances
    int *d_counter = nullptr;
    int direct_grid = 0;
    int32_t *d_totals = nullptr, *d_bads = nullptr, *d_status = nullptr;
    int64_t *d_nout = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t last_stream = nullptr;
    int64_t n_direct = 0, n_fmm = 0;
};

static void batch_free(pf_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto *p : b->plans) pf::fmmx::plan_free(p);
    for (auto s : b->streams) cudaStreamDestroy(s);
    if (b->direct_stream) cudaStreamDestroy(b->direct_stream);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    for (auto e : b->events) cudaEventDestroy(e);
    for (auto p : b->slot_scratch) cudaFree(p);
    cudaFree(b->d_ctr);
    cudaFree(b->d_dinst);
    cudaFree(b->d_items);
    cudaFree(b->d_red_items);
    cudaFree(b->d_part);
    cudaFree(b->d_counter);
    cudaFree(b->d_totals);
    cudaFree(b->d_bads);
    cudaFree(b->d_status);
    cudaFree(b->d_nout);
    delete b;
}

static pf_status batch_build(pf_batch *b, double tol) {
    pf_ctx *ctx = b->ctx;
    const int n = b->n;
    b->plans.assign(n, nullptr);
    b->method.assign(n, PF_DIRECT_METHOD);
    b->ixmin.assign(n, 0);
    b->iymin.assign(n, 0);
    b->nbx.assign(n, 0);
    b->nby.assign(n, 0);
    std::vector<Job> jobs;
    std::vector<std::pair<double, int2>> items;  // cost, (inst, tile * splits + segment)
    std::vector<int2> red_items;                  // (inst, tile) of split instances
    std::vector<std::pair<int, size_t>> part_off; // (inst, offset in float4) of split instances
    size_t part_total = 0;
    std::vector<pf::DirectInstance> dinst(n);
    const int tile = pf::direct_tile_targets();
    for (int i = 0; i < n; ++i) {
        const pf_batch_instance &d = b->inst[i];
        int m = d.method;
        if (d.n == 0) m = PF_DIRECT_METHOD;
        if (m == PF_FMM_METHOD && tol > 0.0) {
            int L = d.leaf_level ? d.leaf_level : pf::fmmx::auto_level(d.n, 35);
            const int np = d.expansion_terms ? d.expansion_terms : pf::fmmx::np_for_tol(tol);
            double w0 = std::max(d.box[1] - d.box[0], d.box[3] - d.box[2]);
            if (!(w0 > 0.0)) w0 = 1.0;
            w0 *= 1.0 + 1e-9;
            pf::fmmx::Plan *p = nullptr;
            while (L >= 3) {
                if (!p) p = pf::fmmx::plan_new();
                bool ok = false;
                PF_TRY(pf::fmmx::plan_build(p, L, 1, np, d.box[0], d.box[2], w0, d.cutoff, &ok));
                if (ok) break;
                --L;
            }
            if (L >= 3) {
                b->plans[i] = p;
                m = PF_FMM_METHOD;
                jobs.push_back({i, 0, (double)d.n * (np * np / 256.0 + 30.0),
                                pf::fmmx::plan_scratch(p, d.n, d.n, true)});
                ++b->n_fmm;
            } else {
                pf::fmmx::plan_free(p);
                m = PF_DIRECT_METHOD;
            }
        } else {
            m = PF_DIRECT_METHOD;
        }
        b->method[i] = m;
        if (m == PF_DIRECT_METHOD && d.n > 0) {
            const pf::DirectSplit sp = pf::direct_split(d.n, d.n);
            dinst[i] = {d.x, d.y, d.g, d.n, d.x, d.y, d.n, pfd::make_gauss_params(d.ksigmasqr),
                        d.vx, d.vy, sp.splits, sp.seg, nullptr};
            const int64_t tiles = pf::ceil_div(d.n, tile);
            for (int64_t t = 0; t < tiles; ++t) {
                const double tn = (double)std::min<int64_t>(tile, d.n - t * tile);
                for (int k = 0; k < sp.splits; ++k) {
                    const double sn = (double)std::min<int64_t>(sp.seg, d.n - k * sp.seg);
                    items.push_back({sn * tn, make_int2(i, (int)(t * sp.splits + k))});
                }
                if (sp.splits > 1) red_items.push_back(make_int2(i, (int)t));
            }
            if (sp.splits > 1) {
                part_off.push_back({i, part_total});
                part_total += (size_t)sp.splits * (size_t)d.n;
            }
            ++b->n_direct;
        } else {
            dinst[i] = {nullptr, nullptr, nullptr, 0, nullptr, nullptr, 0,
                        pfd::make_gauss_params(1.0), nullptr, nullptr, 1, 1, nullptr};
        }
        if (d.remesh && d.n > 0) {
            b->ixmin[i] = left_index_host(d.box[0], d.xb0, d.h);
            b->iymin[i] = left_index_host(d.box[2], d.yb0, d.h);
            b->nbx[i] = left_index_host(d.box[1], d.xb0, d.h) - b->ixmin[i] + 1;
            b->nby[i] = left_index_host(d.box[3], d.yb0, d.h) - b->iymin[i] + 1;
            const int64_t lim = (int64_t)1 << 30;
            if (b->nbx[i] <= 0 || b->nby[i] <= 0 || b->nbx[i] >= lim || b->nby[i] >= lim ||
                b->ixmin[i] <= -lim || b->iymin[i] <= -lim || b->ixmin[i] + b->nbx[i] >= lim ||
                b->iymin[i] + b->nby[i] >= lim ||
                (b->nbx[i] + 3) * (b->nby[i] + 3) >= ((int64_t)1 << 31)) {
                pf::set_error("pf_batch_create: instance %d remesh window invalid", i);
                return PF_ERR_INVALID_ARG;
            }
            jobs.push_back({i, 1, 0.05 * (double)d.n,
                            pf::remesh_scratch_bytes(d.n, b->nbx[i] * b->nby[i],
                                                     (b->nbx[i] + 3) * (b->nby[i] + 3), false) +
                                1024});
        }
    }
    // direct work items, largest first
    std::stable_sort(items.begin(), items.end(),
                     [](const std::pair<double, int2> &a, const std::pair<double, int2> &c) {
                         return a.first > c.first;
                     });
    b->n_items = (int)items.size();
    {
        std::vector<int2> it(items.size());
        for (size_t k = 0; k < items.size(); ++k) it[k] = items[k].second;
        PF_CUDA_TRY(cudaMalloc(&b->d_items, sizeof(int2) * std::max<size_t>(1, it.size())));
        if (!it.empty())
            PF_CUDA_TRY(cudaMemcpy(b->d_items, it.data(), sizeof(int2) * it.size(),
                                   cudaMemcpyHostToDevice));
        if (part_total > 0) {
            PF_CUDA_TRY(cudaMalloc(&b->d_part, sizeof(float4) * part_total));
            for (const auto &po : part_off) dinst[po.first].part = b->d_part + po.second;
        }
        b->n_red = (int)red_items.size();
        PF_CUDA_TRY(cudaMalloc(&b->d_red_items, sizeof(int2) * std::max<size_t>(1, red_items.size())));
        if (!red_items.empty())
            PF_CUDA_TRY(cudaMemcpy(b->d_red_items, red_items.data(), sizeof(int2) * red_items.size(),
                                   cudaMemcpyHostToDevice));
        PF_CUDA_TRY(cudaMalloc(&b->d_dinst, sizeof(pf::DirectInstance) * std::max(1, n)));
        PF_CUDA_TRY(cudaMemcpy(b->d_dinst, dinst.data(), sizeof(pf::DirectInstance) * n,
                               cudaMemcpyHostToDevice));
        PF_CUDA_TRY(cudaMalloc(&b->d_counter, 16));
        b->direct_grid = pf::direct_batch_grid(ctx->num_sms);
    }
    // longest processing time first onto the streams
    std::stable_sort(jobs.begin(), jobs.end(),
                     [](const Job &a, const Job &c) { return a.cost > c.cost; });
    const int S = b->nstreams;
    b->slot_jobs.assign(S, {});
    std::vector<double> load(S, 0.0);
    for (const Job &j : jobs) {
        const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[s] += j.cost;
        b->slot_jobs[s].push_back(j);
    }
    b->slot_scratch.assign(S, nullptr);
    b->slot_bytes.assign(S, 0);
    for (int s = 0; s < S; ++s) {
        size_t mx = 4096;
        for (const Job &j : b->slot_jobs[s]) mx = std::max(mx, j.scratch);
        b->slot_bytes[s] = mx;
        cudaError_t e = cudaMalloc(&b->slot_scratch[s], mx);
        if (e != cudaSuccess) {
            cudaGetLastError();
            pf::set_error("pf_batch_create: scratch allocation of %zu bytes failed", mx);
            return PF_ERR_OOM;
        }
    }
    PF_CUDA_TRY(cudaMalloc(&b->d_ctr, sizeof(unsigned long long) * pf::fmmx::FMM_COUNTERS * std::max(1, S)));
    PF_CUDA_TRY(cudaMalloc(&b->d_totals, sizeof(int32_t) * std::max(1, n)));
    PF_CUDA_TRY(cudaMalloc(&b->d_bads, sizeof(int32_t) * std::max(1, n)));
    PF_CUDA_TRY(cudaMalloc(&b->d_status, sizeof(int32_t) * std::max(1, n)));
    PF_CUDA_TRY(cudaMalloc(&b->d_nout, sizeof(int64_t) * std::max(1, n)));
    PF_CUDA_TRY(cudaMemset(b->d_totals, 0, sizeof(int32_t) * std::max(1, n)));
    PF_CUDA_TRY(cudaMemset(b->d_nout, 0, sizeof(int64_t) * std::max(1, n)));
    return PF_OK;
}

static pf_status batch_enqueue(pf_batch *b) {
    const int S = b->nstreams;
    cudaStream_t cap = b->cap_stream;
    cudaEvent_t fork = b->events[0];
    PF_CUDA_TRY(cudaEventRecord(fork, cap));
    PF_CUDA_TRY(cudaStreamWaitEvent(b->direct_stream, fork, 0));
    for (int s = 0; s < S; ++s) PF_CUDA_TRY(cudaStreamWaitEvent(b->streams[s], fork, 0));
    PF_CUDA_TRY(cudaMemsetAsync(b->d_bads, 0, sizeof(int32_t) * std::max(1, b->n), cap));
    PF_CUDA_TRY(cudaEventRecord(b->events[1], cap));
    for (int s = 0; s < S; ++s) PF_CUDA_TRY(cudaStreamWaitEvent(b->streams[s], b->events[1], 0));
    // the persistent direct kernel
    PF_TRY(pf::launch_direct_batch(b->d_dinst, b->d_items, b->n_items, b->d_red_items, b->n_red,
                                   b->d_counter, b->direct_grid, b->direct_stream));
    for (int s = 0; s < S; ++s) {
        cudaStream_t st = b->streams[s];
        for (const Job &j : b->slot_jobs[s]) {
            const pf_batch_instance &d = b->inst[j.inst];
            pf::Bump sc{b->slot_scratch[s], b->slot_bytes[s], 0};
            if (j.kind == 0) {
                PF_TRY(pf::fmmx::plan_exec(b->plans[j.inst], sc, d.n, d.x, d.y, d.g, d.n, d.x, d.y,
                                           d.ksigmasqr, d.vx, d.vy, b->d_ctr + pf::fmmx::FMM_COUNTERS * s, nullptr, st));
            } else {
                const int64_t nbx = b->nbx[j.inst], nby = b->nby[j.inst];
                const pf::RmWindow win{false, (int32_t)b->ixmin[j.inst], (int32_t)b->iymin[j.inst],
                                       nbx, nby, nbx * nby, (nbx + 3) * (nby + 3), 0};
                PF_TRY(pf::remesh_core(sc, d.n, d.x, d.y, d.g, d.h, d.xb0, d.yb0, d.c, win,
                                       d.capacity, d.x_out, d.y_out, d.g_out, nullptr, nullptr,
                                       b->d_totals + j.inst, b->d_bads + j.inst, st,
                                       b->ctx->num_sms));
            }
        }
        PF_CUDA_TRY(cudaEventRecord(b->events[2 + s], st));
    }
    PF_CUDA_TRY(cudaEventRecord(b->events[2 + S], b->direct_stream));
    for (int s = 0; s <= S; ++s) PF_CUDA_TRY(cudaStreamWaitEvent(cap, b->events[2 + s], 0));
    k_batch_collect<<<(unsigned)pf::ceil_div(std::max(1, b->n), 256), 256, 0, cap>>>(
        b->d_totals, b->d_bads, b->n, b->d_nout, b->d_status);
    return pf::launch_status("k_batch_collect");
}

extern "C" pf_status pf_batch_create(pf_ctx *ctx, int32_t n, const pf_batch_instance *inst,
                                     double tol, int32_t n_streams, pf_batch **out) {
    PF_RANGE("pf_batch_create");
    pf::clear_error();
    PF_CHECK_ARG(ctx && out, "pf_batch_create: NULL argument");
    *out = nullptr;
    PF_CHECK_ARG(n >= 0 && (n == 0 || inst), "pf_batch_create: bad instance array");
    PF_CHECK_ARG(n_streams >= 1 && n_streams <= 64, "pf_batch_create: n_streams in [1, 64]");
    PF_CHECK_ARG(tol >= 0.0 && tol < 1.0, "pf_batch_create: tol must be in [0, 1)");
    for (int i = 0; i < n; ++i) {
        const pf_batch_instance &d = inst[i];
        PF_CHECK_ARG(d.n >= 0 && d.n < ((int64_t)1 << 31), "instance %d: bad n", i);
        PF_CHECK_ARG(d.n == 0 || (d.x && d.y && d.g && d.vx && d.vy), "instance %d: NULL array", i);
        PF_CHECK_ARG(d.ksigmasqr > 0.0 && std::isfinite(d.ksigmasqr), "instance %d: bad ksigmasqr", i);
        PF_CHECK_ARG(d.cutoff >= 0.0 && std::isfinite(d.cutoff), "instance %d: bad cutoff", i);
        PF_CHECK_ARG(d.expansion_terms == 0 || d.expansion_terms == 16 || d.expansion_terms == 20 ||
                         d.expansion_terms == 24 || d.expansion_terms == 28 ||
                         d.expansion_terms == 32,
                     "instance %d: expansion terms must be 0 (from tol) or one of 16,20,24,28,32", i);
        PF_CHECK_ARG(std::isfinite(d.box[0]) && std::isfinite(d.box[1]) && std::isfinite(d.box[2]) &&
                         std::isfinite(d.box[3]) && d.box[1] >= d.box[0] && d.box[3] >= d.box[2],
                     "instance %d: bad box", i);
        PF_CHECK_ARG(d.method == PF_FMM_METHOD || d.method == PF_DIRECT_METHOD,
                     "instance %d: method must be PF_FMM_METHOD or PF_DIRECT_METHOD", i);
        PF_CHECK_ARG(d.leaf_level == 0 || (d.leaf_level >= 3 && d.leaf_level <= pf::fmmx::MAX_LEVEL),
                     "instance %d: leaf level", i);
        PF_CHECK_ARG(!d.remesh || (d.h > 0.0 && std::isfinite(d.h) && std::isfinite(d.xb0) &&
                                   std::isfinite(d.yb0) && std::isfinite(d.c) && d.capacity >= 0 &&
                                   (d.capacity == 0 || (d.x_out && d.y_out && d.g_out))),
                     "instance %d: bad remesh arguments", i);
    }
    pf::DeviceGuard dg(ctx->device);
    pf_batch *b = new (std::nothrow) pf_batch();
    if (!b) {
        pf::set_error("pf_batch_create: host allocation failed");
        return PF_ERR_OOM;
    }
    b->ctx = ctx;
    b->n = n;
    b->inst.assign(inst, inst + n);
    b->nstreams = n_streams;
    pf_status s = batch_build(b, tol);
    if (s == PF_OK) {
        b->streams.resize(n_streams);
        for (int k = 0; k < n_streams && s == PF_OK; ++k)
            if (cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking) != cudaSuccess)
                s = PF_ERR_CUDA;
        if (s == PF_OK &&
            (cudaStreamCreateWithFlags(&b->direct_stream, cudaStreamNonBlocking) != cudaSuccess ||
             cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess))
            s = PF_ERR_CUDA;
        b->events.resize(n_streams + 3);
        for (auto &e : b->events)
            if (s == PF_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                s = PF_ERR_CUDA;
        if (s == PF_ERR_CUDA) pf::set_error("pf_batch_create: stream/event creation failed");
    }
    if (s == PF_OK) {
        cudaError_t e = cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) {
            pf::set_error("cudaStreamBeginCapture failed: %s", cudaGetErrorString(e));
            s = PF_ERR_CUDA;
        } else {
            pf_status se = batch_enqueue(b);
            e = cudaStreamEndCapture(b->cap_stream, &b->graph);
            if (se != PF_OK) s = se;
            else if (e != cudaSuccess) {
                pf::set_error("cudaStreamEndCapture failed: %s", cudaGetErrorString(e));
                s = PF_ERR_CUDA;
            }
        }
    }
    if (s == PF_OK) {
        cudaError_t e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) {
            pf::set_error("cudaGraphInstantiate failed: %s", cudaGetErrorString(e));
            s = PF_ERR_CUDA;
        }
    }
    if (s != PF_OK) {
        cudaGetLastError();
        batch_free(b);
        return s;
    }
    *out = b;
    return PF_OK;
}

extern "C" pf_status pf_batch_run(pf_batch *b, void *stream) {
    PF_RANGE("pf_batch_run");
    pf::clear_error();
    PF_CHECK_ARG(b != nullptr, "pf_batch_run: NULL batch");
    pf::DeviceGuard dg(b->ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PF_CUDA_TRY(cudaGraphLaunch(b->exec, st));
    b->last_stream = st;
    return PF_OK;
}

extern "C" pf_status pf_batch_results(pf_batch *b, int64_t *n_out, int32_t *status) {
    pf::clear_error();
    PF_CHECK_ARG(b != nullptr, "pf_batch_results: NULL batch");
    pf::DeviceGuard dg(b->ctx->device);
    PF_CUDA_TRY(cudaStreamSynchronize(b->last_stream));
    if (n_out && b->n)
        PF_CUDA_TRY(cudaMemcpy(n_out, b->d_nout, sizeof(int64_t) * b->n, cudaMemcpyDeviceToHost));
    if (status && b->n)
        PF_CUDA_TRY(cudaMemcpy(status, b->d_status, sizeof(int32_t) * b->n, cudaMemcpyDeviceToHost));
    return PF_OK;
}

extern "C" pf_status pf_batch_info(const pf_batch *b, int32_t *methods, int32_t *leaf_levels,
                                   int64_t *kernel_nodes) {
    pf::clear_error();
    PF_CHECK_ARG(b != nullptr, "pf_batch_info: NULL batch");
    for (int i = 0; i < b->n; ++i) {
        if (methods) methods[i] = b->method[i];
        if (leaf_levels) leaf_levels[i] = b->plans[i] ? pf::fmmx::plan_level(b->plans[i]) : 0;
    }
    if (kernel_nodes) {
        size_t nn = 0;
        PF_CUDA_TRY(cudaGraphGetNodes(b->graph, nullptr, &nn));
        std::vector<cudaGraphNode_t> nodes(nn);
        PF_CUDA_TRY(cudaGraphGetNodes(b->graph, nodes.data(), &nn));
        int64_t k = 0;
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            PF_CUDA_TRY(cudaGraphNodeGetType(nd, &t));
            if (t == cudaGraphNodeTypeKernel) ++k;
        }
        *kernel_nodes = k;
    }
    return PF_OK;
}

extern "C" pf_status pf_batch_destroy(pf_batch *b) {
    pf::clear_error();
    if (!b) return PF_OK;
    pf::DeviceGuard dg(b->ctx->device);
    cudaDeviceSynchronize();
    batch_free(b);
    return PF_OK;
}
