// wf_batch.cu - batched time step of several independent cases.
//
// Cases of uneven size (wind directions, inflow speeds, building layouts)
// are independent: nothing couples them inside a step.  Stepping them one
// after another leaves small grids unable to fill the 148 SMs (a 96 x 48 x
// 96 case has a few hundred blocks per kernel, the wavefront kernels only
// dozens), and each of the ~200 kernels of a step pays its launch gap.  The
// batch instead composes every case's captured step graph as an independent
// branch of one parent graph: one graph launch advances all cases by one
// step, and kernels of different cases fill each other's idle SMs and gaps.
// No block of one case waits on another, so there are no spin barriers.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "wf_solver.cuh"

struct wf_batch {
    std::vector<wf_solver*> s;
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float last_ms = 0.f;
    long long launches = 0;  // kernels launched by batched steps
    int width = 0;           // concurrent chains of cases (0: every case its own)
    std::string err;
    struct Entry {
        cudaGraphExec_t exec = nullptr;
        std::vector<wf_solver::RoleKey> after;
        long long kernels = 0;
    };
    std::map<std::vector<wf_solver::RoleKey>, Entry> graphs;
};

namespace {

int fail(wf_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

void destroy_graphs(wf_batch* b) {
    for (auto& kv : b->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    b->graphs.clear();
}

// Parent graph with one child-graph branch per case for the cases' current
// buffer roles.
int ensure_batch_graph(wf_batch* b, const wf_batch::Entry** out) {
    std::vector<wf_solver::RoleKey> key;
    key.reserve(b->s.size());
    for (wf_solver* h : b->s) key.push_back({h->iT, h->iF, h->iI, h->iPC, h->iPCL});
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        cudaGraph_t parent = nullptr;
        if (cudaGraphCreate(&parent, 0) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaGraphCreate failed");
        wf_batch::Entry ent;
        // Cases are dealt round-robin onto `width` chains; the chains run
        // concurrently, the cases of one chain one after another.
        const int width = b->width > 0 ? std::min<int>(b->width, (int)b->s.size()) : (int)b->s.size();
        std::vector<cudaGraphNode_t> tail(width, nullptr);
        for (size_t i = 0; i < b->s.size(); ++i) {
            wf_solver* h = b->s[i];
            const wf_solver::GraphEntry* ge = nullptr;
            const int st = wf::ensure_step_graph(h, &ge);
            if (st != WF_OK) {
                cudaGraphDestroy(parent);
                return fail(b, st, "capturing a case's step failed: " + h->err);
            }
            cudaGraphNode_t node;
            cudaGraphNode_t& prev = tail[i % width];
            if (cudaGraphAddChildGraphNode(&node, parent, prev ? &prev : nullptr, prev ? 1 : 0, ge->graph) !=
                cudaSuccess) {
                cudaGraphDestroy(parent);
                return fail(b, WF_ERR_CUDA, "cudaGraphAddChildGraphNode failed");
            }
            prev = node;
            ent.after.push_back(ge->after);
            ent.kernels += ge->kernels;
        }
        const cudaError_t e = cudaGraphInstantiate(&ent.exec, parent, 0);
        cudaGraphDestroy(parent);
        if (e != cudaSuccess) return fail(b, WF_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        it = b->graphs.emplace(key, std::move(ent)).first;
    }
    *out = &it->second;
    return WF_OK;
}

}  // namespace

extern "C" {

int wf_batch_create(wf_solver* const* solvers, int n, wf_batch** out) {
    if (!out || !solvers || n <= 0) return WF_ERR_INVALID_ARG;
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        if (!solvers[i]) return WF_ERR_INVALID_ARG;
        if (solvers[i]->device != solvers[0]->device) return WF_ERR_INVALID_ARG;
        if (solvers[i]->nonuniform) return WF_ERR_UNSUPPORTED;  // uniform-grid cases only
        for (int j = 0; j < i; ++j)
            if (solvers[j] == solvers[i]) return WF_ERR_INVALID_ARG;
    }
    auto* b = new (std::nothrow) wf_batch;
    if (!b) return WF_ERR_OOM;
    b->s.assign(solvers, solvers + n);
    b->device = solvers[0]->device;
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
        if (b->st) cudaStreamDestroy(b->st);
        delete b;
        return WF_ERR_CUDA;
    }
    *out = b;
    return WF_OK;
}

int wf_batch_destroy(wf_batch* b) {
    if (!b) return WF_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->st);
    destroy_graphs(b);
    cudaEventDestroy(b->e0);
    cudaEventDestroy(b->e1);
    cudaStreamDestroy(b->st);
    delete b;
    return WF_OK;
}

int wf_batch_step(wf_batch* b, int n_steps) {
    if (!b) return WF_ERR_INVALID_ARG;
    if (n_steps < 0) return fail(b, WF_ERR_INVALID_ARG, "n_steps must be >= 0");
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaSetDevice failed");
    // Work still queued on a case's own stream (an inflow-plane upload, an
    // asynchronous step) finishes before the batch touches the case.
    for (wf_solver* h : b->s)
        if (cudaStreamSynchronize(h->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "case stream failed");
    // Cases not yet in the graph-replay state (first step after an init or
    // a field write) take one eager step on their own stream first.
    bool any_eager = false;
    for (wf_solver* h : b->s) {
        if (!h->cfg.use_graph || h->cfg.calc_residual)
            return fail(b, WF_ERR_UNSUPPORTED, "batched cases need use_graph and no residual checks");
        if (!wf::step_graphable(h) && n_steps > 0) {
            const int st = wf::run_step_eager(h);
            if (st != WF_OK) return fail(b, st, "eager step failed: " + h->err);
            any_eager = true;
        }
    }
    if (any_eager) {
        for (wf_solver* h : b->s)
            if (cudaStreamSynchronize(h->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "case stream failed");
        --n_steps;
    }
    if (cudaEventRecord(b->e0, b->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaEventRecord failed");
    for (int k = 0; k < n_steps; ++k) {
        const wf_batch::Entry* ent = nullptr;
        const int st = ensure_batch_graph(b, &ent);
        if (st != WF_OK) return st;
        if (cudaGraphLaunch(ent->exec, b->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaGraphLaunch failed");
        for (size_t i = 0; i < b->s.size(); ++i) {
            wf_solver::GraphEntry ge;
            ge.after = ent->after[i];
            ge.kernels = 0;
            wf::commit_graph_step(b->s[i], ge);
        }
        b->launches += ent->kernels;
    }
    if (cudaEventRecord(b->e1, b->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaEventRecord failed");
    const cudaError_t e = cudaStreamSynchronize(b->st);
    if (e != cudaSuccess) return fail(b, WF_ERR_CUDA, std::string("batch step: ") + cudaGetErrorString(e));
    cudaEventElapsedTime(&b->last_ms, b->e0, b->e1);
    return WF_OK;
}

int wf_batch_last_step_ms(const wf_batch* b, float* ms) {
    if (!b || !ms) return WF_ERR_INVALID_ARG;
    *ms = b->last_ms;
    return WF_OK;
}

const char* wf_batch_last_error(const wf_batch* b) { return b ? b->err.c_str() : "null batch"; }

int wf_batch_set_width(wf_batch* b, int width) {
    if (!b) return WF_ERR_INVALID_ARG;
    if (width < 0) return fail(b, WF_ERR_INVALID_ARG, "width must be >= 0");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->st);
    destroy_graphs(b);
    b->width = width;
    return WF_OK;
}

int wf_batch_prepare_graphs(wf_batch* b) {
    if (!b) return WF_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaSetDevice failed");
    for (wf_solver* h : b->s)
        if (!wf::step_graphable(h)) return WF_OK;  // not in the replay state yet
    auto current = [&]() {
        std::vector<wf_solver::RoleKey> k;
        for (wf_solver* h : b->s) k.push_back({h->iT, h->iF, h->iI, h->iPC, h->iPCL});
        return k;
    };
    auto apply = [&](const std::vector<wf_solver::RoleKey>& k) {
        for (size_t i = 0; i < b->s.size(); ++i) {
            wf_solver* h = b->s[i];
            h->iT = std::get<0>(k[i]);
            h->iF = std::get<1>(k[i]);
            h->iI = std::get<2>(k[i]);
            h->iPC = std::get<3>(k[i]);
            h->iPCL = std::get<4>(k[i]);
        }
    };
    const std::vector<wf_solver::RoleKey> start = current();
    int st = WF_OK;
    for (int i = 0; i < 64 && st == WF_OK; ++i) {
        const wf_batch::Entry* ent = nullptr;
        st = ensure_batch_graph(b, &ent);
        if (st != WF_OK) break;
        apply(ent->after);
        if (current() == start) break;
    }
    apply(start);
    return st;
}

int wf_batch_kernel_launches(const wf_batch* b, int64_t* total) {
    if (!b || !total) return WF_ERR_INVALID_ARG;
    *total = b->launches;
    return WF_OK;
}

int wf_set_blocking(wf_solver* h, int pres_k, int vel_k) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (pres_k < 1 || pres_k > 4 || vel_k < 1 || vel_k > 2) {
        h->err = "pres_k must be 1..4 and vel_k 1..2";
        return WF_ERR_INVALID_ARG;
    }
    if (cudaSetDevice(h->device) != cudaSuccess) return WF_ERR_CUDA;
    cudaStreamSynchronize(h->st);
    wf::drop_graphs(h);  // captured steps encode the old depths
    h->pres_k = pres_k;
    h->vel_k = vel_k;
    return WF_OK;
}

int wf_get_blocking(const wf_solver* h, int* pres_k, int* vel_k) {
    if (!h || !pres_k || !vel_k) return WF_ERR_INVALID_ARG;
    *pres_k = h->pres_k;
    *vel_k = h->vel_k;
    return WF_OK;
}

}  // extern "C"
