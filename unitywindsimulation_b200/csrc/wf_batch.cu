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
//
// The persistent mode (WF_BATCH_PERSISTENT) instead records each case's step
// as captured segments of its once-per-step kernels around its four Jacobi
// loops, and runs each loop of all cases as one cooperative launch whose
// blocks walk a (case, tile) work queue with a bounded grid barrier between
// sweeps: 4 loop launches per batched step instead of about 80 per case.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "wf_solver.cuh"
#include "wf_sweeps.cuh"

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

    // ---- persistent mode ----
    int mode = WF_BATCH_GRAPHS;
    double barrier_timeout_ms = 2000.0;
    wf::GridBar* bar = nullptr;  // device
    int sms = 148;
    // one case's step for one buffer-role state: segment graphs and the
    // recorded loops between them
    struct CaseSteps {
        std::vector<cudaGraph_t> graphs;  // segment graphs (children of the step graph)
        std::vector<cudaGraphExec_t> seg;
        std::vector<int> kinds;
        std::vector<wf::VelLoopRec> vel;
        std::vector<wf::PresLoopRec> pres;
        wf_solver::RoleKey after{};
        long long kernels = 0;
    };
    std::vector<std::map<wf_solver::RoleKey, CaseSteps>> case_steps;
    // the loop launches of all cases for one combination of role states
    struct LoopLaunch {
        int kind = 0;
        void* table = nullptr;  // device tables (FusedVelCase... / FusedPresCase...)
        int ncases = 0, nitems = 0, nsweeps = 0, nrounds = 0, blocks = 0;
        const void* cases = nullptr;
        const void* passes = nullptr;
        const int* round_items = nullptr;
    };
    struct FusedEntry {
        cudaGraphExec_t exec = nullptr;  // whole step: segments and loop launches
        std::vector<const CaseSteps*> cases;
        std::vector<LoopLaunch> loops;
        std::vector<wf_solver::RoleKey> after;
        long long kernels = 0;
    };
    std::map<std::vector<wf_solver::RoleKey>, FusedEntry> fused;
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
    for (auto& kv : b->fused) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        for (auto& l : kv.second.loops)
            if (l.table) cudaFree(l.table);
    }
    b->fused.clear();
    for (auto& m : b->case_steps)
        for (auto& kv : m) {
            for (cudaGraphExec_t e : kv.second.seg)
                if (e) cudaGraphExecDestroy(e);
            for (cudaGraph_t g : kv.second.graphs)
                if (g) cudaGraphDestroy(g);
        }
    b->case_steps.assign(b->s.size(), {});
}

std::vector<wf_solver::RoleKey> role_keys(const wf_batch* b) {
    std::vector<wf_solver::RoleKey> key;
    key.reserve(b->s.size());
    for (wf_solver* h : b->s) key.push_back({h->iT, h->iF, h->iI, h->iPC, h->iPCL});
    return key;
}

// Segments and loop plans of case i's step from its current roles.
int ensure_case_steps(wf_batch* b, size_t i, const wf_batch::CaseSteps** out) {
    wf_solver* h = b->s[i];
    const wf_solver::RoleKey key{h->iT, h->iF, h->iI, h->iPC, h->iPCL};
    auto& m = b->case_steps[i];
    auto it = m.find(key);
    if (it == m.end()) {
        wf::LoopRecorder rec;
        wf_batch::CaseSteps cs;
        const int st = wf::capture_step_segments(h, &rec, &cs.after, &cs.kernels);
        int res = st == WF_OK ? WF_OK : fail(b, st, "recording a case's step failed: " + h->err);
        for (cudaGraph_t g : rec.segments) {
            cudaGraphExec_t e = nullptr;
            if (res == WF_OK && cudaGraphInstantiate(&e, g, 0) != cudaSuccess)
                res = fail(b, WF_ERR_CUDA, "cudaGraphInstantiate of a step segment failed");
            if (e) cs.seg.push_back(e);
            cs.graphs.push_back(g);
        }
        if (res == WF_OK && cs.seg.size() != rec.kinds.size() + 1)
            res = fail(b, WF_ERR_CUDA, "segment count does not match the recorded loops");
        if (res != WF_OK) {
            for (cudaGraphExec_t e : cs.seg) cudaGraphExecDestroy(e);
            for (cudaGraph_t g : cs.graphs) cudaGraphDestroy(g);
            return res;
        }
        cs.kinds = std::move(rec.kinds);
        cs.vel = std::move(rec.vel);
        cs.pres = std::move(rec.pres);
        it = m.emplace(key, std::move(cs)).first;
    }
    *out = &it->second;
    return WF_OK;
}

// Packs host structs and pointer arrays into one device allocation.
struct Packer {
    std::vector<char> host;
    template <typename T>
    size_t add(const T* v, size_t n) {
        size_t off = (host.size() + 255) & ~size_t(255);
        host.resize(off + n * sizeof(T));
        std::memcpy(host.data() + off, v, n * sizeof(T));
        return off;
    }
};

int upload(wf_batch* b, Packer& pk, void** dev) {
    if (cudaMalloc(dev, pk.host.size()) != cudaSuccess) return fail(b, WF_ERR_OOM, "loop tables: cudaMalloc failed");
    if (cudaMemcpy(*dev, pk.host.data(), pk.host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(*dev);
        *dev = nullptr;
        return fail(b, WF_ERR_CUDA, "loop tables: copy failed");
    }
    return WF_OK;
}

// The persistent launch of momentum loop `vi` of every case.
int build_vel_loop(wf_batch* b, const std::vector<const wf_batch::CaseSteps*>& cs, int vi, wf_batch::LoopLaunch* L) {
    const size_t n = cs.size();
    const int nsweeps = (int)cs[0]->vel[vi].src.size();
    Packer pk;
    std::vector<wf::FusedVelCase> tab(n);
    pk.add(tab.data(), n);  // placeholder, rewritten below with device offsets
    std::vector<size_t> src_off(n), dst_off(n);
    int items = 0;
    for (size_t c = 0; c < n; ++c) {
        const wf::VelLoopRec& v = cs[c]->vel[vi];
        if ((int)v.src.size() != nsweeps) return fail(b, WF_ERR_UNSUPPORTED, "cases differ in momentum sweeps");
        src_off[c] = pk.add(v.src.data(), v.src.size());
        dst_off[c] = pk.add(v.dst.data(), v.dst.size());
        const wf::Params& P = b->s[c]->P;
        wf::FusedVelCase& q = tab[c];
        q.P = P;
        q.A = v.A;
        q.iD = v.iD;
        q.bv = v.bv;
        q.vec4 = v.vec4 ? 1 : 0;
        const int xt = v.vec4 ? P.nx / 4 : P.nx;
        q.gx = (xt + 31) / 32;
        q.gy = (P.ny + 3) / 4;
        q.gz = (P.nz + 1) / 2;
        q.item0 = items;
        items += q.gx * q.gy * q.gz;
    }
    void* dev = nullptr;
    for (size_t c = 0; c < n; ++c) {
        tab[c].src = nullptr;
        tab[c].dst = nullptr;
    }
    // device addresses of the pointer arrays are known only after the
    // allocation: allocate, patch, copy
    if (cudaMalloc(&dev, pk.host.size()) != cudaSuccess) return fail(b, WF_ERR_OOM, "loop tables: cudaMalloc failed");
    for (size_t c = 0; c < n; ++c) {
        tab[c].src = reinterpret_cast<const float* const*>(static_cast<char*>(dev) + src_off[c]);
        tab[c].dst = reinterpret_cast<float* const*>(static_cast<char*>(dev) + dst_off[c]);
    }
    std::memcpy(pk.host.data(), tab.data(), n * sizeof(wf::FusedVelCase));
    if (cudaMemcpy(dev, pk.host.data(), pk.host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(dev);
        return fail(b, WF_ERR_CUDA, "loop tables: copy failed");
    }
    int per_sm = 0;
    if (wf::fused_vel_blocks_per_sm(&per_sm) != WF_OK || per_sm < 1) {
        cudaFree(dev);
        return fail(b, WF_ERR_CUDA, "occupancy of the persistent momentum loop");
    }
    L->kind = 0;
    L->table = dev;
    L->cases = dev;
    L->ncases = (int)n;
    L->nitems = items;
    L->nsweeps = nsweeps;
    L->blocks = std::max(1, std::min(items, per_sm * b->sms));
    return WF_OK;
}

// The persistent launch of pressure loop `pi` of every case.
int build_pres_loop(wf_batch* b, const std::vector<const wf_batch::CaseSteps*>& cs, int pi, wf_batch::LoopLaunch* L) {
    const size_t n = cs.size();
    int nrounds = 0;
    for (const auto* c : cs) nrounds = std::max(nrounds, (int)c->pres[pi].passes.size());
    std::vector<wf::FusedPresCase> tab(n);
    std::vector<wf::FusedPresPass> passes(n * std::max(nrounds, 1));
    std::vector<int> round_items(std::max(nrounds, 1), 0);
    for (size_t c = 0; c < n; ++c) {
        const wf::PresLoopRec& pr = cs[c]->pres[pi];
        tab[c].P = b->s[c]->P;
        tab[c].c3 = pr.c3;
        tab[c].ainv = pr.ainv;
        tab[c].rhs = pr.rhs;
    }
    for (int r = 0; r < nrounds; ++r) {
        int items = 0;
        for (size_t c = 0; c < n; ++c) {
            wf::FusedPresPass& ps = passes[c * nrounds + r];
            ps = {};
            ps.item0 = items;
            const wf::PresLoopRec& pr = cs[c]->pres[pi];
            if (r >= (int)pr.passes.size()) continue;
            ps.k = pr.passes[r].k;
            ps.in = pr.passes[r].in;
            ps.out = pr.passes[r].out;
            wf::fused_pres_geometry(b->s[c]->P, ps.k, &ps.gx, &ps.gy, &ps.nchunk, &ps.zchunk);
            items += ps.gx * ps.gy * ps.nchunk;
        }
        round_items[r] = items;
    }
    Packer pk;
    const size_t o_cases = pk.add(tab.data(), n);
    const size_t o_passes = pk.add(passes.data(), passes.size());
    const size_t o_items = pk.add(round_items.data(), round_items.size());
    void* dev = nullptr;
    const int st = upload(b, pk, &dev);
    if (st != WF_OK) return st;
    int per_sm = 0;
    if (wf::fused_pres_blocks_per_sm(&per_sm) != WF_OK || per_sm < 1) {
        cudaFree(dev);
        return fail(b, WF_ERR_CUDA, "occupancy of the persistent pressure loop");
    }
    L->kind = 1;
    L->table = dev;
    L->cases = static_cast<char*>(dev) + o_cases;
    L->passes = static_cast<char*>(dev) + o_passes;
    L->round_items = reinterpret_cast<const int*>(static_cast<char*>(dev) + o_items);
    L->ncases = (int)n;
    L->nrounds = nrounds;
    L->blocks = per_sm * b->sms;
    return WF_OK;
}

// The whole persistent-mode step as one graph: segment i of every case as
// parallel child graphs, then a reset of the barrier and loop i as a
// cooperative kernel node that waits for all of them.  Returns false (and
// leaves exec null) when the graph cannot be built; the step then launches
// the same work one launch at a time.
bool build_fused_graph(wf_batch* b, wf_batch::FusedEntry* ent) {
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
    const unsigned long long timeout_ns = (unsigned long long)(b->barrier_timeout_ms * 1e6);
    bool ok = true;
    cudaGraphNode_t join = nullptr;
    const size_t nseg = ent->loops.size() + 1;
    for (size_t i = 0; i < nseg && ok; ++i) {
        std::vector<cudaGraphNode_t> segs;
        for (const auto* cs : ent->cases) {
            cudaGraphNode_t n = nullptr;
            ok = ok && cudaGraphAddChildGraphNode(&n, g, join ? &join : nullptr, join ? 1 : 0, cs->graphs[i]) ==
                           cudaSuccess;
            segs.push_back(n);
        }
        if (!ok || i + 1 == nseg) break;
        cudaMemsetParams mp = {};
        mp.dst = b->bar;
        mp.value = 0;
        mp.elementSize = sizeof(unsigned);
        mp.width = 2;  // arrival count and generation; the error word stays
        mp.height = 1;
        cudaGraphNode_t reset = nullptr;
        ok = cudaGraphAddMemsetNode(&reset, g, segs.data(), segs.size(), &mp) == cudaSuccess;
        if (!ok) break;
        const wf_batch::LoopLaunch& L = ent->loops[i];
        cudaKernelNodeParams kp = {};
        const void* cases = L.cases;
        const void* passes = L.passes;
        const int* items = L.round_items;
        int ncases = L.ncases, nitems = L.nitems, nsweeps = L.nsweeps, nrounds = L.nrounds;
        wf::GridBar* bar = b->bar;
        unsigned long long tns = timeout_ns;
        void* vargs[] = {(void*)&cases, (void*)&ncases, (void*)&nitems, (void*)&nsweeps, (void*)&bar, (void*)&tns};
        void* pargs[] = {(void*)&cases, (void*)&ncases, (void*)&passes, (void*)&items, (void*)&nrounds,
                         (void*)&bar, (void*)&tns};
        kp.gridDim = dim3(L.blocks);
        if (L.kind == 0) {
            kp.func = const_cast<void*>(wf::fused_vel_kernel());
            kp.blockDim = dim3(32, 4, 2);
            kp.sharedMemBytes = 0;
            kp.kernelParams = vargs;
        } else {
            kp.func = const_cast<void*>(wf::fused_pres_kernel());
            kp.blockDim = dim3(32, 32);
            kp.sharedMemBytes = (unsigned)wf::fused_pres_smem();
            kp.kernelParams = pargs;
        }
        cudaGraphNode_t kn = nullptr;
        ok = cudaGraphAddKernelNode(&kn, g, &reset, 1, &kp) == cudaSuccess;
        if (!ok) break;
        cudaKernelNodeAttrValue av = {};
        av.cooperative = 1;
        ok = cudaGraphKernelNodeSetAttribute(kn, cudaLaunchAttributeCooperative, &av) == cudaSuccess;
        join = kn;
    }
    if (ok) ok = cudaGraphInstantiate(&ent->exec, g, 0) == cudaSuccess;
    cudaGraphDestroy(g);
    if (!ok) {
        ent->exec = nullptr;
        cudaGetLastError();  // the failed graph calls leave no sticky error; clear the last one
    }
    return ok;
}

int ensure_fused(wf_batch* b, const wf_batch::FusedEntry** out) {
    const auto key = role_keys(b);
    auto it = b->fused.find(key);
    if (it == b->fused.end()) {
        wf_batch::FusedEntry ent;
        for (size_t i = 0; i < b->s.size(); ++i) {
            const wf_batch::CaseSteps* cs = nullptr;
            const int st = ensure_case_steps(b, i, &cs);
            if (st != WF_OK) return st;
            if (cs->kinds != (ent.cases.empty() ? cs->kinds : ent.cases[0]->kinds))
                return fail(b, WF_ERR_UNSUPPORTED, "persistent batches need cases with the same step structure");
            ent.cases.push_back(cs);
            ent.after.push_back(cs->after);
            ent.kernels += cs->kernels;
        }
        const std::vector<int>& kinds = ent.cases[0]->kinds;
        int vi = 0, pi = 0;
        for (int kind : kinds) {
            wf_batch::LoopLaunch L;
            const int st = kind == 0 ? build_vel_loop(b, ent.cases, vi++, &L) : build_pres_loop(b, ent.cases, pi++, &L);
            if (st != WF_OK) {
                for (auto& l : ent.loops) cudaFree(l.table);
                return st;
            }
            ent.loops.push_back(L);
            ent.kernels += 1;
        }
        build_fused_graph(b, &ent);
        it = b->fused.emplace(key, std::move(ent)).first;
    }
    *out = &it->second;
    return WF_OK;
}

// One batched step in the persistent mode: segment i of every case, then
// loop i of all cases as one cooperative launch.
int fused_step(wf_batch* b) {
    const wf_batch::FusedEntry* ent = nullptr;
    const int st = ensure_fused(b, &ent);
    if (st != WF_OK) return st;
    const unsigned long long timeout_ns = (unsigned long long)(b->barrier_timeout_ms * 1e6);
    const size_t nseg = ent->exec ? 0 : ent->loops.size() + 1;
    if (ent->exec && cudaGraphLaunch(ent->exec, b->st) != cudaSuccess)
        return fail(b, WF_ERR_CUDA, "persistent step graph launch failed");
    for (size_t i = 0; i < nseg; ++i) {
        for (const auto* cs : ent->cases)
            if (cudaGraphLaunch(cs->seg[i], b->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "segment launch failed");
        if (i + 1 == nseg) break;
        const wf_batch::LoopLaunch& L = ent->loops[i];
        // fresh arrival count and generation (the error word stays sticky)
        if (cudaMemsetAsync(b->bar, 0, 2 * sizeof(unsigned), b->st) != cudaSuccess)
            return fail(b, WF_ERR_CUDA, "barrier reset failed");
        cudaError_t e;
        if (L.kind == 0)
            e = wf::launch_fused_vel_loop(b->st, L.blocks, static_cast<const wf::FusedVelCase*>(L.cases), L.ncases,
                                          L.nitems, L.nsweeps, b->bar, timeout_ns);
        else
            e = wf::launch_fused_pres_loop(b->st, L.blocks, static_cast<const wf::FusedPresCase*>(L.cases), L.ncases,
                                           static_cast<const wf::FusedPresPass*>(L.passes), L.round_items, L.nrounds,
                                           b->bar, timeout_ns);
        if (e != cudaSuccess) return fail(b, WF_ERR_CUDA, std::string("persistent loop launch: ") + cudaGetErrorString(e));
    }
    for (size_t i = 0; i < b->s.size(); ++i) {
        wf_solver::GraphEntry ge;
        ge.after = ent->after[i];
        ge.kernels = 0;
        wf::commit_graph_step(b->s[i], ge);
    }
    b->launches += ent->kernels;
    return WF_OK;
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
    b->case_steps.assign(b->s.size(), {});
    b->sms = solvers[0]->num_sms;
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess ||
        cudaMalloc(&b->bar, sizeof(wf::GridBar)) != cudaSuccess ||
        cudaMemset(b->bar, 0, sizeof(wf::GridBar)) != cudaSuccess) {
        if (b->bar) cudaFree(b->bar);
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
    cudaFree(b->bar);
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
    const bool persistent = b->mode == WF_BATCH_PERSISTENT;
    if (persistent && cudaMemsetAsync(b->bar, 0, sizeof(wf::GridBar), b->st) != cudaSuccess)
        return fail(b, WF_ERR_CUDA, "barrier reset failed");
    if (cudaEventRecord(b->e0, b->st) != cudaSuccess) return fail(b, WF_ERR_CUDA, "cudaEventRecord failed");
    for (int k = 0; k < n_steps && persistent; ++k) {
        const int st = fused_step(b);
        if (st != WF_OK) return st;
    }
    for (int k = 0; k < n_steps && !persistent; ++k) {
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
    bool waits_ran_out = false;
    for (wf_solver* h : b->s)
        if (h->hstat && *(volatile int*)h->hstat) {
            *(volatile int*)h->hstat = 0;
            waits_ran_out = true;
        }
    if (waits_ran_out)
        return fail(b, WF_ERR_TIMEOUT, "a bounded wait of a TMA-staged pressure pass ran out; the cases' fields are "
                                       "not valid");
    if (persistent) {
        wf::GridBar hb{};
        if (cudaMemcpy(&hb, b->bar, sizeof(hb), cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(b, WF_ERR_CUDA, "barrier read failed");
        if (hb.err)
            return fail(b, WF_ERR_TIMEOUT, "a grid barrier of a persistent loop waited longer than the barrier "
                                           "timeout; the cases' fields are not valid");
    }
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
        std::vector<wf_solver::RoleKey> after;
        if (b->mode == WF_BATCH_PERSISTENT) {
            const wf_batch::FusedEntry* ent = nullptr;
            st = ensure_fused(b, &ent);
            if (st == WF_OK) after = ent->after;
        } else {
            const wf_batch::Entry* ent = nullptr;
            st = ensure_batch_graph(b, &ent);
            if (st == WF_OK) after = ent->after;
        }
        if (st != WF_OK) break;
        apply(after);
        if (current() == start) break;
    }
    apply(start);
    return st;
}

int wf_batch_set_mode(wf_batch* b, int mode) {
    if (!b) return WF_ERR_INVALID_ARG;
    if (mode != WF_BATCH_GRAPHS && mode != WF_BATCH_PERSISTENT) return fail(b, WF_ERR_INVALID_ARG, "unknown batch mode");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->st);
    destroy_graphs(b);
    b->mode = mode;
    return WF_OK;
}

int wf_batch_get_mode(const wf_batch* b, int* mode) {
    if (!b || !mode) return WF_ERR_INVALID_ARG;
    *mode = b->mode;
    return WF_OK;
}

int wf_batch_set_barrier_timeout(wf_batch* b, double ms) {
    if (!b) return WF_ERR_INVALID_ARG;
    if (!(ms > 0.0) || ms > 600000.0) return fail(b, WF_ERR_INVALID_ARG, "timeout must be in (0, 600000] ms");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->st);
    destroy_graphs(b);  // the persistent step graphs hold the limit as a kernel argument
    b->barrier_timeout_ms = ms;
    return WF_OK;
}

int wf_grid_barrier_selftest(int device, int blocks, int extra, double timeout_ms, int* status) {
    if (!status || blocks < 1 || extra < 0 || !(timeout_ms > 0.0) || timeout_ms > 60000.0) return WF_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return WF_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return WF_ERR_CUDA;
    if (blocks > sms) return WF_ERR_INVALID_ARG;  // one block per SM is always resident
    wf::GridBar* bar = nullptr;
    if (cudaMalloc(&bar, sizeof(wf::GridBar)) != cudaSuccess) return WF_ERR_OOM;
    cudaStream_t st = nullptr;
    int res = WF_OK;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) res = WF_ERR_CUDA;
    if (res == WF_OK && cudaMemsetAsync(bar, 0, sizeof(wf::GridBar), st) != cudaSuccess) res = WF_ERR_CUDA;
    if (res == WF_OK &&
        wf::launch_barrier_selftest(st, blocks, extra, bar, (unsigned long long)(timeout_ms * 1e6)) != cudaSuccess)
        res = WF_ERR_CUDA;
    wf::GridBar hb{};
    if (res == WF_OK && cudaMemcpyAsync(&hb, bar, sizeof(hb), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        res = WF_ERR_CUDA;
    if (st && cudaStreamSynchronize(st) != cudaSuccess) res = WF_ERR_CUDA;
    if (st) cudaStreamDestroy(st);
    cudaFree(bar);
    if (res != WF_OK) return res;
    *status = hb.err ? WF_ERR_TIMEOUT : WF_OK;
    return WF_OK;
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

int wf_set_tiles(wf_solver* h, int pres_rows, int vel_bx, int vel_by, int vel_bz) {
    if (!h) return WF_ERR_INVALID_ARG;
    if ((pres_rows != 32 && pres_rows != 16) || vel_bx < 1 || vel_by < 1 || vel_bz < 1 ||
        vel_bx * vel_by * vel_bz != 256) {
        h->err = "pres_rows must be 32 or 16 and vel_bx * vel_by * vel_bz 256";
        return WF_ERR_INVALID_ARG;
    }
    if (cudaSetDevice(h->device) != cudaSuccess) return WF_ERR_CUDA;
    cudaStreamSynchronize(h->st);
    wf::drop_graphs(h);  // captured steps encode the old tiles
    h->pres_ty = pres_rows;
    h->vel_blk[0] = vel_bx;
    h->vel_blk[1] = vel_by;
    h->vel_blk[2] = vel_bz;
    return WF_OK;
}

int wf_get_tiles(const wf_solver* h, int* pres_rows, int* vel_bx, int* vel_by, int* vel_bz) {
    if (!h || !pres_rows || !vel_bx || !vel_by || !vel_bz) return WF_ERR_INVALID_ARG;
    *pres_rows = h->pres_ty;
    *vel_bx = h->vel_blk[0];
    *vel_by = h->vel_blk[1];
    *vel_bz = h->vel_blk[2];
    return WF_OK;
}

int wf_get_blocking(const wf_solver* h, int* pres_k, int* vel_k) {
    if (!h || !pres_k || !vel_k) return WF_ERR_INVALID_ARG;
    *pres_k = h->pres_k;
    *vel_k = h->vel_k;
    return WF_OK;
}

}  // extern "C"
