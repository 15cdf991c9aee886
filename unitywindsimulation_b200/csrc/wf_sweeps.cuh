// wf_sweeps.cuh - fast Jacobi loops of the momentum predictor and of the
// pressure(-correction) equations.
#pragma once
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
void launch_pres_stack(const Params& P, cudaStream_t st, int sms, const float* c3, const float* ainv,
                       const float* rhs, float* stack, int n, bool from_zero);

// Event-timed launches of one hot kernel (WF_KERNEL_*), see wf_time_kernel.
int time_kernel(wf_solver* h, int which, int reps, bool flush, float* ms, double* bytes, int* sweeps);

}  // namespace wf
