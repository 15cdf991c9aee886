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

// Event-timed launches of one hot kernel (WF_KERNEL_*), see wf_time_kernel.
int time_kernel(wf_solver* h, int which, int reps, bool flush, float* ms, double* bytes, int* sweeps);

}  // namespace wf
