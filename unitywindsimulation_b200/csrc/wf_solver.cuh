// wf_solver.cuh - the solver handle behind the C ABI (private).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>

#include "wf_common.cuh"

namespace wf {
struct LoopRecorder;
}

struct wf_solver {
    wf_config cfg{};
    wf::Params P{};
    wf::Bnd B{};
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    // ---- device fields (see wf_common.cuh for the layout) ----
    uint8_t* fl = nullptr;
    uint8_t* nbm = nullptr;   // neighbour masks (Params::nbm)
    // Three velocity buffers rotated by role like the reference's
    // velField / velFieldLastTime / velFieldLastIter textures.  When
    // iter_alias is set, velFieldLastIter is logically equal to
    // velFieldLastTime and buffer vb[iI] holds no meaningful fluid values
    // (this replaces the end-of-step copy, FvmSolverGpu.cs:1106).
    // A fourth, spare buffer lets the multi-sweep kernels write iterates n
    // and n-1 while velFieldLastTime and the pass input stay intact.  Solid
    // cells hold the same values in all four (no kernel writes them).
    float* vb[4] = {nullptr, nullptr, nullptr, nullptr};
    int iT = 0, iF = 1, iI = 2;
    bool iter_alias = false;
    float *uc = nullptr, *Dv = nullptr, *bv = nullptr, *aodu = nullptr, *face = nullptr;
    float* pr = nullptr;
    // presCorrectField / presCorrectFieldLastIter.  When pc_zero is set both
    // are logically all-zero (replaces SetPresCorrectFieldtoZero,
    // FvmSolverGpu.cs:1545-1554; the first sweep then reads no input).
    // Three physical buffers: the multi-sweep kernels need a third one to
    // materialise iterate n-1 next to iterate n.
    float* pcb[3] = {nullptr, nullptr, nullptr};
    int iPC = 0, iPCL = 1;
    bool pc_zero = true;
    float *Dp = nullptr, *bp = nullptr, *eddy = nullptr;
    float* drag = nullptr;    // Brinkman drag per cell (allocated when first set)
    // non-uniform collocated grid (wf_nonuniform.cu): face positions
    // fx[nx+1], fy[ny+1], fz[nz+1] back to back, and the face-flux texture
    // (three planes of (nx+1)(ny+1)(nz+1)); nonuniform selects its kernels
    float* fpos = nullptr;
    float* flux = nullptr;
    float* nucoef = nullptr;  // the pressure sweeps' per-step coefficient planes (wf::kNuCoefPlanes)
    bool nonuniform = false;
    float* bnd[6] = {};
    // sweep coefficient caches of the fast path (wf_sweeps.cu)
    float* pcoef = nullptr;   // pressure: c_E, c_N, c_U, 1/Dp, PISO rhs (5 planes)
    float* vcoef = nullptr;   // momentum: A_E..A_D, 1/D (9 planes)
    float* grad = nullptr;    // cell-centre velocity gradient tensors (9 planes)
    // generation of DField (bumped by every write) and the generation the
    // cached pressure face coefficients c_E, c_N, c_U were built from: the
    // three pressure solves of a step share D, so they share the coefficients
    long long d_gen = 1, c3_gen = 0;
    long long id_gen = 0;     // generation of D the cached 1/D (vcoef + 6N) belongs to
    // the momentum pre-compute of the step in progress wrote vcoef (A and
    // 1/D) for the current D; the step's sweeps take them as they are
    bool vcoef_step = false;
    // scratch
    double* part = nullptr;
    double* dsum = nullptr;   // 4 doubles
    float* dref = nullptr;
    int* dbad = nullptr;
    void* stage = nullptr;    // 4N floats of device staging for host I/O
    // inflow-plane upload: page-locked staging (3 * ny * nz floats) and the
    // event after which the staging may be rewritten
    float* in_stage = nullptr;
    cudaEvent_t ev_in = nullptr;
    // asynchronous readback: snapshot (4N + N floats), copy stream, events
    float* snap = nullptr;
    cudaStream_t cst = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_done = nullptr;
    bool rb_pending = false;
    double* hsum = nullptr;   // pinned

    float wind = 0.f;
    int64_t step = 0;
    float res_vel = -1.f, res_pres = -1.f;
    float last_ms = 0.f;
    int fast = 1;             // use the fast Jacobi kernels (wf_sweeps.cu)
    int pres_k = 4;           // pressure sweeps per multi-sweep pass (1..4)
    int vel_k = 1;            // momentum sweeps per multi-sweep pass (1..2)
    int pres_ty = 32;         // tile rows of the pressure multi-sweep kernel (32 or 16)
    int pres_tma = 1;         // four-sweep passes with TMA-staged tiles where they apply
                              // (WF_TMA=0: the per-thread-staged kernel; same iterates)
    // sticky status of the bounded waits in the TMA-staged kernel: page-locked
    // host word (hstat) and its device alias (dstat); nonzero = a wait ran out
    int* hstat = nullptr;
    int* dstat = nullptr;
    int vel_blk[3] = {32, 4, 2};  // block of the four-cell momentum sweep (256 threads)
    int num_sms = 148;        // multiprocessors of the device
    int pdl = 1;              // programmatic dependent launch in the non-uniform grid's sweep chains
                              // (WF_PDL=0: plain stream order)
    int vec4 = 1;             // 4-cell vector momentum sweep when nx % 4 == 0 and the
                              // planes are 16-byte aligned (WF_VEC4=0: one cell per thread)
    bool in_step = false;     // inside wf_step: skip iterates no later kernel reads
    wf::LoopRecorder* rec = nullptr;  // set while a batch records the step in segments
    long long launches = 0;   // kernels launched by wf_step
    std::string err;

    // CUDA-graph cache of one step, keyed by the buffer roles before the step.
    using RoleKey = std::tuple<int, int, int, int, int>;
    struct GraphEntry {
        cudaGraph_t graph = nullptr;  // kept for composition into batch graphs
        cudaGraphExec_t exec = nullptr;
        RoleKey after{};
        long long kernels = 0;
    };
    std::map<RoleKey, GraphEntry> graphs;
};

namespace wf {
// Step-graph plumbing shared by the single-handle and the batched step.
bool step_graphable(const wf_solver* h);
// Captures (once per buffer-role assignment) the graph of one step from the
// handle's current state without running it.
int ensure_step_graph(wf_solver* h, const wf_solver::GraphEntry** out);
// Applies the role rotation and counters of one replayed step.
void commit_graph_step(wf_solver* h, const wf_solver::GraphEntry& e);
// One step launched kernel by kernel on the handle's stream.
int run_step_eager(wf_solver* h);
// Captures one step from the handle's current state as segments around its
// Jacobi loops (rec), without running it; *after receives the roles after
// the step and *kernels the kernels in the segments.
int capture_step_segments(wf_solver* h, LoopRecorder* rec, wf_solver::RoleKey* after, long long* kernels);
void drop_graphs(wf_solver* h);
}  // namespace wf
