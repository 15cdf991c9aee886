// wf_sweeps.cuh - fast Jacobi loops of the momentum predictor and of the
// pressure(-correction) equations.
#pragma once
#include <vector>

#include "wf_solver.cuh"

namespace wf {

// Per-device kernel attributes of the sweep kernels; call once per device
// before the first launch.
int sweeps_setup();

// n sweeps of CSVelPredict with the VelPredict buffer rotation
// (FvmSolverGpu.cs:1244-1279): on return vb[iF] holds iterate n and vb[iI]
// iterate n-1, exactly as after the reference loop.
int vel_sweeps_fast(wf_solver* h, int n);

// n sweeps of CSPresCorrectRhieChow (piso = false, FvmSolverGpu.cs:1372-1415)
// or CSPisoPresCorrection (piso = true, :1493-1514) with the same rotation.
int pres_sweeps_fast(wf_solver* h, int n, bool piso);

// Explicit-pointer launchers of the fast Jacobi building blocks: momentum
// coefficients A (6 planes) and 1/D (3), one momentum sweep, pressure face
// coefficients c_E/c_N/c_U, 1/Dp, PISO diagonal and right-hand side.  The
// momentum sweep writes every cell (non-fluid cells copy the input iterate),
// so each output buffer holds a complete iterate.
void launch_vel_coef_ptr(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uT, const float* eddy,
                         const float* face, const float* Dv, float* A, float* iD);
void launch_vel_sweep1_ptr(const Params& P, cudaStream_t st, const float* A, const float* iD, const float* bv,
                           const float* ui, float* uo);
void launch_pres_coef_ptr(const Params& P, cudaStream_t st, const uint8_t* fl, const float* Dv, const float* iD,
                          float* c3);
void launch_inv_ptr(const Params& P, cudaStream_t st, const uint8_t* fl, const float* Dp, float* ainv);
void launch_piso_pre_ptr(const Params& P, cudaStream_t st, const uint8_t* fl, const float* Dv, const float* iD,
                         const float* aodu, float* ainv, float* rhs);

// n pressure-type sweeps po = ainv (rhs - C pi) (rhs == nullptr: 0) by the
// multi-sweep kernel, every iterate kept: slot k of `stack` (stride N floats)
// receives iterate k for k = 1..n on every cell (0 on non-fluid cells).  The
// first pass reads slot 0, or the all-zero iterate when from_zero is set.
// Four-sweep passes take the TMA-staged kernel where it applies and
// `status` is given (the handle's wait status), else k_pres_msweep<4, 32>.
void launch_pres_stack(const Params& P, cudaStream_t st, int sms, const float* c3, const float* ainv,
                       const float* rhs, float* stack, int n, bool from_zero, int* status = nullptr);

// ---- loop recording and persistent multi-case loops (wf_batch.cu) ----
//
// While a handle's `rec` is set (inside a stream capture of its step), the
// Jacobi loops are not launched: each loop ends the current capture segment
// (LoopRecorder::cut), its sweeps are recorded as a plan of buffer pointers,
// and the buffer roles rotate exactly as if the sweeps had run.  The batch
// then runs every case's segments and, for each loop, one persistent
// cooperative launch over all cases.

// One recorded momentum loop: sweep k reads src[k] and writes dst[k].
struct VelLoopRec {
    const float* A = nullptr;
    const float* iD = nullptr;
    const float* bv = nullptr;
    bool vec4 = false;
    std::vector<const float*> src;
    std::vector<float*> dst;
};
// One pass of a recorded pressure loop: k sweeps from `in` (nullptr: the
// all-zero iterate) to `out`.
struct PresPassRec {
    int k;
    const float* in;
    float* out;
};
struct PresLoopRec {
    const float* c3 = nullptr;
    const float* ainv = nullptr;
    const float* rhs = nullptr;
    std::vector<PresPassRec> passes;
};
struct LoopRecorder {
    cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    std::vector<cudaGraph_t> segments;   // captured once-per-step kernels between the loops
    std::vector<int> kinds;              // per loop: 0 momentum, 1 pressure
    std::vector<VelLoopRec> vel;
    std::vector<PresLoopRec> pres;
    // Ends the current capture segment on h's stream and begins the next.
    int cut(wf_solver* h);
};

// Grid-wide barrier of the persistent loops: arrival count, generation, and
// a sticky error word (set when a wait runs out; every later wait returns at
// once).
struct GridBar {
    unsigned int count;
    unsigned int gen;
    int err;
    int pad;
};

// Device-side tables of a persistent momentum loop (one entry per case).
struct FusedVelCase {
    Params P;
    const float* A;
    const float* iD;
    const float* bv;
    const float* const* src;   // [nsweeps], device array
    float* const* dst;         // [nsweeps], device array
    int vec4;                  // four-cell form
    int gx, gy, gz;            // blocks of the case's sweep grid (block 32 x 4 x 2)
    int item0;                 // first work item of the case
};
// Device-side tables of a persistent pressure loop: passes[c * nrounds + r]
// is round r of case c (k == 0: the case has no pass in that round).
struct FusedPresPass {
    int k;
    int gx, gy, nchunk, zchunk;
    int item0;                 // first work item of the case in this round
    const float* in;
    float* out;
};
struct FusedPresCase {
    Params P;
    const float* c3;
    const float* ainv;
    const float* rhs;
};

// The persistent loop kernels (for graph kernel nodes): momentum blocks are
// 32 x 4 x 2 threads, pressure blocks 32 x 32 with fused_pres_smem() bytes
// of dynamic shared memory.  Argument order as in launch_fused_*_loop.
const void* fused_vel_kernel();
const void* fused_pres_kernel();
size_t fused_pres_smem();
// Resident blocks per SM of the persistent momentum / pressure kernels.
int fused_vel_blocks_per_sm(int* out);
int fused_pres_blocks_per_sm(int* out);
// z chunk of a case's tiles in a persistent pressure pass.
void fused_pres_geometry(const Params& P, int k, int* gx, int* gy, int* nchunk, int* zchunk);
cudaError_t launch_fused_vel_loop(cudaStream_t st, int blocks, const FusedVelCase* cases, int ncases, int nitems,
                                  int nsweeps, GridBar* bar, unsigned long long timeout_ns);
cudaError_t launch_fused_pres_loop(cudaStream_t st, int blocks, const FusedPresCase* cases, int ncases,
                                   const FusedPresPass* passes, const int* round_items, int nrounds, GridBar* bar,
                                   unsigned long long timeout_ns);
// One cooperative launch of `blocks` blocks that meet at a barrier expecting
// blocks + extra arrivals (extra > 0: a barrier nothing releases).
cudaError_t launch_barrier_selftest(cudaStream_t st, int blocks, int extra, GridBar* bar,
                                    unsigned long long timeout_ns);

// Four pressure sweeps per pass with TMA-staged tiles (wf_pres_tma.cu):
// the same iterates (and, with `stack`, the same per-level slots) as
// k_pres_msweep<4, 32>, bit for bit.  Applies where pres_tma_ok (nx % 4 ==
// 0, 16-byte aligned planes, the driver's tensor-map encoder present).  c3
// holds c_E, c_N, c_U as consecutive N-float planes.  A bounded wait that
// runs out (wait_ms per wait; <= 0: 1 s) sets *status (device-visible) to
// 1.  short_stage (self-test only): each block's first loaded stage expects
// 16 bytes more than its loads deliver, so its wait runs out.
size_t pres_tma_smem();
const void* pres_tma_kernel();
bool pres_tma_ok(const Params& P, const float* c3, const float* ainv, const float* rhs, const float* in);
cudaError_t launch_pres_tma4(const Params& P, cudaStream_t st, int sms, const float* c3, const float* ainv,
                             const float* rhs, const float* in, float* out, float* prev, float* stack, int* status,
                             double wait_ms = 0.0, bool short_stage = false);

// Two momentum sweeps per pass with TMA-staged tiles (wf_vel_tma.cu): the
// same iterates n and n-1 as two k_vel_sweep4 sweeps, bit for bit.  A holds
// A_E..A_D and iD the three components of 1/D, each as consecutive N-float
// planes.  Applies where vel_tma_ok (nx % 4 == 0, 16-byte aligned planes,
// the driver's tensor-map encoder present).  A bounded wait that runs out
// sets *status to 1.
size_t vel_tma_smem();
const void* vel_tma_kernel();
bool vel_tma_ok(const Params& P, const float* A, const float* iD, const float* bv, const float* in);
cudaError_t launch_vel_tma2(const Params& P, cudaStream_t st, int sms, const float* A, const float* iD,
                            const float* bv, const float* in, float* out, float* prev, int* status,
                            double wait_ms = 0.0);

// Event-timed launches of one hot kernel (WF_KERNEL_*), see wf_time_kernel.
int time_kernel(wf_solver* h, int which, int reps, bool flush, float* ms, double* bytes, int* sweeps);

}  // namespace wf
