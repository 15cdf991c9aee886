// wf_kernels.cuh - launchers of the per-operation kernels (wf_kernels.cu) and
// of the multi-sweep kernels (wf_sweeps.cu).
#pragma once
#include <cuda_runtime.h>

#include "wf_common.cuh"

namespace wf {

int cell_grid_blocks(const Params& P);

void launch_wallfunc(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uT, float* face);
// grad (nullable): 9 planes receiving / holding the cell-centre velocity
// gradient tensors.
// face (nullable): the wall function's face viscosities (k_wallfunc's
// values) from the same pass.
void launch_eddy_vis(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT, float* eddy,
                     float* grad, float* face = nullptr);
void launch_cell_grad(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT,
                      float* grad);
void launch_les_term(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT,
                     const float* eddy, const float* face, const float* grad, float* bles);
// drag (nullable): Brinkman drag coefficient per cell, added to D as dv*drag.
void launch_vel_precompute(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT,
                           const float* pr, const float* eddy, const float* face, const float* bles,
                           const float* drag, float* Dv, float* bv, float* A = nullptr, float* iD = nullptr);
void launch_vel_sweep(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uI, const float* uT,
                      const float* eddy, const float* face, const float* Dv, const float* bv, float* uo);
// iD (nullable): cached 1/D of the same D (bit-identical to dividing).
void launch_pres_precompute(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* u,
                            const float* pr, const float* Dv, const float* iD, float* Dp, float* bp,
                            float* c3 = nullptr);
void launch_pres_sweep(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pin, const float* Dv,
                       const float* Dp, const float* bp, float* pout);
void launch_apply_pres(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pc, float* pr);
void launch_normalize(const Params& P, cudaStream_t st, const uint8_t* fl, float* pr, float* ref);
void launch_apply_vel(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pc, const float* Dv,
                      const float* iD, float* uc, float* u, float* pr = nullptr);
void launch_piso_aodu(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uc, const float* uT,
                      const float* eddy, const float* face, float* aodu);
void launch_piso_pres_sweep(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pin, const float* Dv,
                            const float* aodu, float* pout);
void launch_piso_vel(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pc, const float* Dv,
                     const float* iD, const float* aodu, float* uc, float* u, float* pr = nullptr);
// Neighbour masks (Params::nbm) from the flags; run after every flag change.
void launch_nbmask(const Params& P, cudaStream_t st, const uint8_t* fl, uint8_t* nbm);
void launch_vel_residual(const Params& P, cudaStream_t st, const float* Dv, const float* u, const float* uI,
                         double* part, double* out);
void launch_pres_residual(const Params& P, cudaStream_t st, const float* Dp, const float* pc, const float* pcL,
                          double* part, double* out);
void launch_mass_imbalance(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* u,
                           double* part, double* out);
void launch_check_finite(cudaStream_t st, const float* a, long long n, int* bad);
void launch_init_fields(const Params& P, cudaStream_t st, int logp, float wind, float fric, float kappa, float z0,
                        int centre, float* u0, float* u1, float* u2, float* uc, float* pr);
void launch_init_flags(const Params& P, cudaStream_t st, const int32_t* src, uint8_t* fl, float* u0, float* u1,
                       float* u2);
void launch_set_log_inlet(const Params& P, cudaStream_t st, float fric, float kappa, float z0, float* x0);
void launch_fill3(cudaStream_t st, float* a, int n, float v0, float v1, float v2);
void launch_soa_to_interleaved(cudaStream_t st, const float* s, int n, float* d, int w4);
void launch_flags_to_i32(cudaStream_t st, const uint8_t* f, int n, int32_t* o);

}  // namespace wf

// Non-uniform collocated grid (wf_nonuniform.cu); the launchers take the
// handle (mesh, face-flux texture and stream live there).
struct wf_solver;
namespace wf {
constexpr int kNuCoefPlanes = 7;  // per-step pressure-sweep coefficients of the non-uniform grid (N floats each)
size_t nu_flux_texels(const Params& P);
void launch_nu_vel_precompute(const wf_solver* h);
void launch_nu_pres_precompute(wf_solver* h, const float* u);
void launch_nu_pres_sweep(const wf_solver* h, const float* pin, float* pout, bool pre);
void launch_nu_apply_vel(wf_solver* h, const float* pc, float* u);
void launch_nu_init_log(wf_solver* h, float fric, float kappa, float z0);
void launch_nu_log_inlet(wf_solver* h, float fric, float kappa, float z0);
}  // namespace wf
