/*
 * windfvm_oracle.h - C ABI of the CPU oracle (test infrastructure only).
 *
 * The oracle is a plain C++17 restatement of the reference's HLSL kernels for
 * the collocated SIMPLE/PISO LES step of puppy2333/UnityWindSimulation, run in
 * FP32 or FP64 with OpenMP over z.  It is the checker for the CUDA library
 * (include/windfvm.h): only the tests, the smoke check and the CPU-baseline
 * leg of the benchmark load it.  The product path never calls it.
 *
 * Parity status: pinned on the reference's own kernels.  The reference ships
 * no tests or golden vectors for this path and its host (C# under Unity, D3D
 * dispatch) cannot run here, but its compute shaders compile as C++ through
 * oracle/hlsl_shim.h (oracle/ref_kernels.py, oracle/ref_driver.cpp).  The FP32
 * instance of this oracle is bit-identical to them on every field of every
 * step tested (tests/test_ref_pin.py, tests/golden/ref_kernels.npz).  It is
 * also checked by known-answer tests (quiescent box, free-stream
 * preservation, closed-form wall function, linear-shear Smagorinsky,
 * adjoint-stencil symmetry) and by the agreement of its FP32 and FP64
 * instances.
 *
 * Every wfo_* entry mirrors the wf_* entry of the same name in windfvm.h and
 * uses the same wf_config, field ids and layouts.
 */
#ifndef WINDFVM_ORACLE_H
#define WINDFVM_ORACLE_H

#include "../include/windfvm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct wfo_solver wfo_solver;

/* precision: 32 -> float, 64 -> double.  threads <= 0: OpenMP default. */
int wfo_create(const wf_config* cfg, int precision, int threads, wfo_solver** out);
int wfo_destroy(wfo_solver* h);
int wfo_init_flags(wfo_solver* h, const int32_t* flags, size_t n);
int wfo_init_vel_pres_fields(wfo_solver* h);
int wfo_set_fixed_value_vel_bnd_cond(wfo_solver* h, float wind_speed);
int wfo_set_inflow_plane(wfo_solver* h, const float* x0_plane_xyz);
int wfo_init_from_background(wfo_solver* h, const wfo_solver* bg, const float pos[3], const float pos_bg[3],
                             float rot_deg);
int wfo_step(wfo_solver* h, int n_steps);
int wfo_set_face_positions(wfo_solver* h, const float* fx, const float* fy, const float* fz);
int wfo_get_face_flux(wfo_solver* h, double* out);

/* Field transfer in FP64 (so the FP64 instance loses nothing); vectors SoA. */
int wfo_field_size(const wfo_solver* h, int field, size_t* points, int* comps);
int wfo_get_field(wfo_solver* h, int field, double* out);
int wfo_set_field(wfo_solver* h, int field, const double* in);
int wfo_get_flags(wfo_solver* h, int32_t* out);

int wfo_op_wallfunc(wfo_solver* h);
int wfo_op_eddy_vis(wfo_solver* h);
int wfo_op_les_term(wfo_solver* h);
int wfo_op_vel_precompute(wfo_solver* h);
int wfo_op_vel_sweeps(wfo_solver* h, int n);
int wfo_op_pres_precompute(wfo_solver* h);
int wfo_op_pres_sweeps(wfo_solver* h, int n);
int wfo_op_apply_pres(wfo_solver* h);
int wfo_op_normalize(wfo_solver* h);
int wfo_op_apply_vel(wfo_solver* h);
int wfo_op_zero_pres_correct(wfo_solver* h);
int wfo_op_piso(wfo_solver* h, int n);
int wfo_op_end_step(wfo_solver* h);
int wfo_op_vel_residual(wfo_solver* h, double* out);
int wfo_op_pres_residual(wfo_solver* h, double* out);
int wfo_residuals(wfo_solver* h, double* vel, double* pres);
int wfo_mass_imbalance(wfo_solver* h, double* out);

/* Stand-alone log-law wall function (WallFunc.compute:77-123) for unit tests. */
double wfo_log_law_wall_func(double uP, double dx, double nu, double den, int precision);

#ifdef __cplusplus
}
#endif
#endif
