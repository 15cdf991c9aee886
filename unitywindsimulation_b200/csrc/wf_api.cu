// wf_api.cu - host implementation of the windfvm C ABI (include/windfvm.h).
//
// Sequencing follows FvmSolverGpu (Assets/Code/FvmSolver/FvmSolverGpu.cs of
// puppy2333/UnityWindSimulation): constructor :173-222, Step :1050-1121,
// VelPredict :1238-1282, PresCorrect :1367-1439, ApplyVelCorrection
// :1441-1452, PisoCorrection :1482-1533.  Buffer roles are rotated exactly
// where the C# driver swaps its textures; the two copies it makes per step
// (end-of-step velocity copy and zeroing the pressure correction) are
// replaced by role flags (iter_alias, pc_zero) that the kernels honour.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "wf_kernels.cuh"
#include "wf_solver.cuh"
#include "wf_sweeps.cuh"

using wf::Params;

namespace {

#define WF_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                \
            return e_ == cudaErrorMemoryAllocation ? WF_ERR_OOM : WF_ERR_CUDA;          \
        }                                                                               \
    } while (0)

#define WF_CHECK_LAUNCH()                                                               \
    do {                                                                                \
        cudaError_t e_ = cudaGetLastError();                                            \
        if (e_ != cudaSuccess) {                                                        \
            h->err = std::string("kernel launch: ") + cudaGetErrorString(e_);           \
            return WF_ERR_CUDA;                                                         \
        }                                                                               \
    } while (0)

#define WF_TRY(expr)                \
    do {                            \
        int s_ = (expr);            \
        if (s_ != WF_OK) return s_; \
    } while (0)

int set_err(wf_solver* h, int code, const char* msg) {
    if (h) h->err = msg;
    return code;
}

bool any_fixed_pres(const wf_config& c) {
    for (int f = 0; f < 6; ++f)
        if (c.pres_bc[f] == WF_BND_FIXED_VALUE) return true;
    return false;
}

const char* validate(const wf_config* c) {
    if (!c) return "config is NULL";
    if (c->struct_size != sizeof(wf_config)) return "config struct_size does not match this library";
    if (c->nx < 3 || c->ny < 3 || c->nz < 3) return "grid must be at least 3 cells on every axis";
    const double n = double(c->nx) * c->ny * c->nz;
    if (n * 4.0 >= 2147483647.0) return "grid too large (4*nx*ny*nz must fit in int32)";
    if (!(c->dx > 0.f) || !std::isfinite(c->dx)) return "dx must be > 0";
    if (!(c->dt > 0.f) || !std::isfinite(c->dt)) return "dt must be > 0";
    if (!(c->den > 0.f)) return "den must be > 0";
    if (!(c->mu >= 0.f)) return "mu must be >= 0";
    for (int f = 0; f < 6; ++f) {
        if (c->vel_bc[f] < 0 || c->vel_bc[f] > 2) return "vel_bc out of range";
        if (c->pres_bc[f] < 0 || c->pres_bc[f] > 2) return "pres_bc out of range";
    }
    if (c->solver_type != WF_SOLVER_SIMPLE && c->solver_type != WF_SOLVER_PISO) return "solver_type out of range";
    if (c->turbulence != WF_TURB_NONE && c->turbulence != WF_TURB_SMAGORINSKY) return "turbulence out of range";
    if (c->inflow_type != WF_INFLOW_CONSTANT && c->inflow_type != WF_INFLOW_LOG) return "inflow_type out of range";
    if (c->vel_iters < 0 || c->pres_iters < 0 || c->piso_correctors < 0) return "iteration counts must be >= 0";
    if (c->inflow_type == WF_INFLOW_LOG) {
        if (!(c->inflow_z0 > 0.f) || !(c->inflow_kappa > 0.f)) return "log inflow needs z0 > 0 and kappa > 0";
        if (!(c->inflow_ustar > 0.f) && !(c->inflow_href > 0.f)) return "log inflow needs ustar > 0 or href > 0";
    }
    if (c->calc_residual && (c->vel_res_interval <= 0 || c->pres_res_interval <= 0))
        return "residual intervals must be > 0 when calc_residual is set";
    if (c->compat_flags & ~(WF_COMPAT_RFLOAT_FACE_EDDY_VIS | WF_COMPAT_INIT_PROFILE_CELL_CENTRE |
                            WF_COMPAT_PISO_CONSISTENT))
        return "unknown compat flag";
    return nullptr;
}

float fric_vel(const wf_solver* h) {
    const wf_config& c = h->cfg;
    if (c.inflow_ustar > 0.f) return c.inflow_ustar;
    return c.inflow_kappa * h->wind / logf((c.inflow_href + c.inflow_z0) / c.inflow_z0);
}

int alloc(wf_solver* h, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
        return WF_ERR_OOM;
    }
    e = cudaMemsetAsync(*p, 0, bytes, h->st);
    if (e != cudaSuccess) {
        h->err = std::string("cudaMemset: ") + cudaGetErrorString(e);
        return WF_ERR_CUDA;
    }
    return WF_OK;
}

void free_all(wf_solver* h) {
    wf::drop_graphs(h);
    void* ptrs[] = {h->fl, h->vb[0], h->vb[1], h->vb[2], h->vb[3], h->uc, h->Dv, h->bv, h->aodu, h->face, h->pr,
                    h->pcb[0], h->pcb[1], h->pcb[2], h->Dp, h->bp, h->eddy, h->pcoef, h->vcoef, h->grad, h->part, h->dsum, h->dref,
                    h->dbad, h->stage, h->bnd[0], h->drag, h->nbm, h->fpos, h->flux, h->nucoef};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->hsum) cudaFreeHost(h->hsum);
    if (h->hstat) cudaFreeHost(h->hstat);
    if (h->cst) {
        cudaStreamSynchronize(h->cst);
        cudaStreamDestroy(h->cst);
    }
    if (h->ev_in) {
        cudaEventSynchronize(h->ev_in);
        cudaEventDestroy(h->ev_in);
    }
    if (h->in_stage) cudaFreeHost(h->in_stage);
    if (h->ev_snap) cudaEventDestroy(h->ev_snap);
    if (h->ev_done) cudaEventDestroy(h->ev_done);
    if (h->snap) cudaFree(h->snap);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->st) cudaStreamDestroy(h->st);
}

int sync(wf_solver* h) {
    WF_CUDA(cudaStreamSynchronize(h->st));
    if (h->hstat && *(volatile int*)h->hstat) {
        *(volatile int*)h->hstat = 0;
        return set_err(h, WF_ERR_TIMEOUT,
                       "a bounded wait of the TMA-staged pressure sweep ran out; the pressure fields are not valid");
    }
    return WF_OK;
}

// Makes velFieldLastIter a real buffer again (copy of velFieldLastTime).
int materialize_iter(wf_solver* h) {
    if (!h->iter_alias) return WF_OK;
    WF_CUDA(cudaMemcpyAsync(h->vb[h->iI], h->vb[h->iT], 3 * sizeof(float) * h->P.N, cudaMemcpyDeviceToDevice, h->st));
    h->iter_alias = false;
    return WF_OK;
}
// Makes both pressure-correction buffers real zeros again.
int materialize_pc(wf_solver* h) {
    if (!h->pc_zero) return WF_OK;
    WF_CUDA(cudaMemsetAsync(h->pcb[h->iPC], 0, sizeof(float) * h->P.N, h->st));
    WF_CUDA(cudaMemsetAsync(h->pcb[h->iPCL], 0, sizeof(float) * h->P.N, h->st));
    h->pc_zero = false;
    return WF_OK;
}

// ---------------------------------------------------------- stage bodies
// Each function enqueues work on h->st only (no host sync) unless residuals
// are requested, so a whole step can be captured into a CUDA graph.

int do_les(wf_solver* h) {
    const Params& P = h->P;
    const float* uT = h->vb[h->iT];
    // CalWallFunc and CSCalEddyVis in one pass over velFieldLastTime
    wf::launch_eddy_vis(P, h->B, h->st, h->fl, uT, h->eddy, h->grad, h->face);
    wf::launch_les_term(P, h->B, h->st, h->fl, uT, h->eddy, h->face, h->grad, h->bv);
    WF_CHECK_LAUNCH();
    return WF_OK;
}

// 1/D cached by the fast momentum path for the current D, or null.
const float* cur_inv_d(const wf_solver* h) { return h->id_gen == h->d_gen ? h->vcoef + 6 * (size_t)h->P.N : nullptr; }

int do_vel_precompute(wf_solver* h) {
    ++h->d_gen;
    if (h->nonuniform) {
        wf::launch_nu_vel_precompute(h);
        WF_CHECK_LAUNCH();
        return WF_OK;
    }
    // inside a step the fast momentum sweeps' coefficients (A, 1/D) come out
    // of the same pass; nothing between here and the sweeps changes their
    // inputs (velFieldLastTime, the eddy viscosity, D)
    const bool coef = h->in_step && h->fast;
    float* A = coef ? h->vcoef : nullptr;
    float* iD = coef ? h->vcoef + 6 * (size_t)h->P.N : nullptr;
    wf::launch_vel_precompute(h->P, h->B, h->st, h->fl, h->vb[h->iT], h->pr, h->eddy, h->face,
                              h->P.les ? h->bv : nullptr, h->drag, h->Dv, h->bv, A, iD);
    WF_CHECK_LAUNCH();
    h->vcoef_step = coef;
    return WF_OK;
}

int read_residual(wf_solver* h, double* out) {
    WF_CUDA(cudaMemcpyAsync(h->hsum, h->dsum, sizeof(double), cudaMemcpyDeviceToHost, h->st));
    WF_TRY(sync(h));
    *out = h->hsum[0];
    return WF_OK;
}

// VelPredict loop (FvmSolverGpu.cs:1244-1279) with n sweeps.
int do_vel_sweeps(wf_solver* h, int n, bool allow_fast) {
    const Params& P = h->P;
    const bool resid = h->cfg.calc_residual != 0;
    const bool from_alias = h->iter_alias;
    int k = 0;
    if (allow_fast && h->fast && !resid && n > 0) {
        // Multi-sweep path: same buffer roles, several sweeps per launch.
        // On the non-uniform grid too: its pre-compute stored A and 1/D.
        WF_TRY(wf::vel_sweeps_fast(h, n));
        return WF_OK;
    }
    for (; k < n; ++k) {
        const float* src = h->iter_alias ? h->vb[h->iT] : h->vb[h->iI];
        if (h->nonuniform)  // the pre-compute's A and 1/D (vcoef)
            wf::launch_vel_sweep1_ptr(P, h->st, h->vcoef, h->vcoef + 6 * (size_t)P.N, h->bv, src, h->vb[h->iF]);
        else
            wf::launch_vel_sweep(P, h->st, h->fl, src, h->vb[h->iT], h->eddy, h->face, h->Dv, h->bv, h->vb[h->iF]);
        WF_CHECK_LAUNCH();
        if (resid && k % h->cfg.vel_res_interval == 0) {
            wf::launch_vel_residual(P, h->st, h->Dv, h->vb[h->iF], src, h->part, h->dsum);
            double s = 0.0;
            WF_TRY(read_residual(h, &s));
            h->res_vel = (float)std::sqrt(s / (3.0 * P.N));
            if (h->res_vel < h->cfg.vel_tol) break;
        }
        std::swap(h->iI, h->iF);
        h->iter_alias = false;
    }
    std::swap(h->iI, h->iF);
    // one complete sweep from the aliased state: iterate 0 (velFieldLastIter
    // after the loop) is velFieldLastTime itself
    if (k == 1 && n == 1 && from_alias) h->iter_alias = true;
    return WF_OK;
}

int do_pres_precompute(wf_solver* h) {
    if (h->nonuniform) {
        wf::launch_nu_pres_precompute(h, h->vb[h->iF]);
        WF_CHECK_LAUNCH();
        return WF_OK;
    }
    // the fast path's pressure face coefficients come out of the same pass
    // (they depend on D only, like the cache generation they are keyed by)
    float* c3 = h->fast ? h->pcoef : nullptr;
    wf::launch_pres_precompute(h->P, h->B, h->st, h->fl, h->vb[h->iF], h->pr, h->Dv, cur_inv_d(h), h->Dp, h->bp, c3);
    WF_CHECK_LAUNCH();
    if (c3) h->c3_gen = h->d_gen;
    return WF_OK;
}

// PresCorrect loop (FvmSolverGpu.cs:1372-1415) with n sweeps.
int do_pres_sweeps(wf_solver* h, int n, bool allow_fast) {
    const Params& P = h->P;
    const bool resid = h->cfg.calc_residual != 0;
    if (allow_fast && h->fast && !resid && n > 0 && !h->nonuniform) {
        WF_TRY(wf::pres_sweeps_fast(h, n, /*piso=*/false));
        return WF_OK;
    }
    for (int k = 0; k < n; ++k) {
        const float* src = h->pc_zero ? nullptr : h->pcb[h->iPCL];
        if (h->nonuniform)
            wf::launch_nu_pres_sweep(h, src, h->pcb[h->iPC], k > 0);
        else
            wf::launch_pres_sweep(P, h->st, h->fl, src, h->Dv, h->Dp, h->bp, h->pcb[h->iPC]);
        WF_CHECK_LAUNCH();
        h->pc_zero = false;
        if (resid && k % h->cfg.pres_res_interval == 0) {
            wf::launch_pres_residual(P, h->st, h->Dp, h->pcb[h->iPC], src, h->part, h->dsum);
            double s = 0.0;
            WF_TRY(read_residual(h, &s));
            h->res_pres = (float)std::sqrt(s / double(P.N));
            if (h->res_pres < h->cfg.pres_tol) break;
        }
        std::swap(h->iPCL, h->iPC);
    }
    std::swap(h->iPCL, h->iPC);
    return WF_OK;
}

const float* pc_cur(const wf_solver* h) { return h->pc_zero ? nullptr : h->pcb[h->iPC]; }

int do_apply_pres(wf_solver* h) {
    wf::launch_apply_pres(h->P, h->st, h->fl, pc_cur(h), h->pr);
    WF_CHECK_LAUNCH();
    return WF_OK;
}
int do_normalize(wf_solver* h) {
    wf::launch_normalize(h->P, h->st, h->fl, h->pr, h->dref);
    WF_CHECK_LAUNCH();
    return WF_OK;
}
int do_apply_vel(wf_solver* h) {
    if (h->nonuniform) {
        wf::launch_nu_apply_vel(h, pc_cur(h), h->vb[h->iF]);
        WF_CHECK_LAUNCH();
        return WF_OK;
    }
    wf::launch_apply_vel(h->P, h->st, h->fl, pc_cur(h), h->Dv, cur_inv_d(h), h->uc, h->vb[h->iF]);
    WF_CHECK_LAUNCH();
    return WF_OK;
}
// ApplyVelCorrection together with ApplyPresCorrection (p += p'), one pass;
// the velocity correction does not read p, so the two commute.
int do_apply_vel_pres(wf_solver* h) {
    wf::launch_apply_vel(h->P, h->st, h->fl, pc_cur(h), h->Dv, cur_inv_d(h), h->uc, h->vb[h->iF], h->pr);
    WF_CHECK_LAUNCH();
    return WF_OK;
}

// PisoCorrection (FvmSolverGpu.cs:1482-1533) with n pressure sweeps; p'
// starts from the zero state.
int do_piso(wf_solver* h, int n, bool allow_fast) {
    const Params& P = h->P;
    if (h->nonuniform) return set_err(h, WF_ERR_UNSUPPORTED, "PISO runs on the uniform grid only");
    wf::launch_piso_aodu(P, h->st, h->fl, h->uc, h->vb[h->iT], h->eddy, h->face, h->aodu);
    WF_CHECK_LAUNCH();
    if (allow_fast && h->fast && n > 0) {
        WF_TRY(wf::pres_sweeps_fast(h, n, /*piso=*/true));
    } else {
        for (int k = 0; k < n; ++k) {
            const float* src = h->pc_zero ? nullptr : h->pcb[h->iPCL];
            wf::launch_piso_pres_sweep(P, h->st, h->fl, src, h->Dv, h->aodu, h->pcb[h->iPC]);
            WF_CHECK_LAUNCH();
            h->pc_zero = false;
            std::swap(h->iPCL, h->iPC);
        }
        std::swap(h->iPCL, h->iPC);
    }
    // PisoApplyPresCorrection (p += p'') in the same pass as the velocity
    // correction, which does not read p
    const float* pc = pc_cur(h);
    if (pc) {
        wf::launch_piso_vel(P, h->st, h->fl, pc, h->Dv, cur_inv_d(h), h->aodu, h->uc, h->vb[h->iF], h->pr);
    } else {
        // p'' == 0: PisoVelCorrection with a zero field still applies -D^-1 AodU
        WF_TRY(materialize_pc(h));
        wf::launch_piso_vel(P, h->st, h->fl, h->pcb[h->iPC], h->Dv, cur_inv_d(h), h->aodu, h->uc, h->vb[h->iF],
                            h->pr);
    }
    WF_CHECK_LAUNCH();
    h->pc_zero = true;  // SetPresCorrectFieldtoZero (:1532)
    return WF_OK;
}

int do_end_step(wf_solver* h) {
    std::swap(h->iT, h->iF);
    h->iter_alias = true;  // CopyVelField(velFieldLastIter <- velFieldLastTime)
    h->step += 1;
    return WF_OK;
}

// One complete Step() (FvmSolverGpu.cs:1050-1121) with fixed counts.
int enqueue_step_body(wf_solver* h);

int enqueue_step(wf_solver* h) {
    h->in_step = true;
    const int s = enqueue_step_body(h);
    h->in_step = false;
    h->vcoef_step = false;
    return s;
}

int enqueue_step_body(wf_solver* h) {
    const wf_config& c = h->cfg;
    if (h->P.les) WF_TRY(do_les(h));
    WF_TRY(do_vel_precompute(h));
    WF_TRY(do_vel_sweeps(h, c.vel_iters, true));
    WF_TRY(do_pres_precompute(h));
    WF_TRY(do_pres_sweeps(h, c.pres_iters, true));
    if (h->nonuniform) {
        WF_TRY(do_apply_pres(h));
        if (!any_fixed_pres(c)) WF_TRY(do_normalize(h));
        WF_TRY(do_apply_vel(h));
    } else {
        // p += p' in the velocity-correction pass; the normalisation reads
        // the corrected p and the velocity correction does not read p
        WF_TRY(do_apply_vel_pres(h));
        if (!any_fixed_pres(c)) WF_TRY(do_normalize(h));
    }
    h->pc_zero = true;  // SetPresCorrectFieldtoZero (:1088)
    if (c.solver_type == WF_SOLVER_PISO)
        for (int n = 0; n < c.piso_correctors; ++n) WF_TRY(do_piso(h, c.pres_iters, true));
    return do_end_step(h);
}

wf_solver::RoleKey role_key(const wf_solver* h) { return {h->iT, h->iF, h->iI, h->iPC, h->iPCL}; }
void set_roles(wf_solver* h, const wf_solver::RoleKey& k) {
    h->iT = std::get<0>(k);
    h->iF = std::get<1>(k);
    h->iI = std::get<2>(k);
    h->iPC = std::get<3>(k);
    h->iPCL = std::get<4>(k);
}

// Runs one step, replaying a cached CUDA graph when the handle is in its
// steady state (iter_alias and pc_zero set, no residual reads).
int run_step(wf_solver* h) {
    if (!wf::step_graphable(h)) return wf::run_step_eager(h);
    const wf_solver::GraphEntry* ent = nullptr;
    WF_TRY(wf::ensure_step_graph(h, &ent));
    WF_CUDA(cudaGraphLaunch(ent->exec, h->st));
    wf::commit_graph_step(h, *ent);
    return WF_OK;
}

int check_finite(wf_solver* h) {
    WF_CUDA(cudaMemsetAsync(h->dbad, 0, sizeof(int), h->st));
    wf::launch_check_finite(h->st, h->vb[h->iT], 3LL * h->P.N, h->dbad);
    wf::launch_check_finite(h->st, h->pr, h->P.N, h->dbad);
    WF_CHECK_LAUNCH();
    int bad = 0;
    WF_CUDA(cudaMemcpyAsync(&bad, h->dbad, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    WF_TRY(sync(h));
    if (bad) return set_err(h, WF_ERR_NONFINITE, "non-finite value in velocity or pressure");
    return WF_OK;
}

// Resolves a field id to its device pointer and size.
float* field_ptr(wf_solver* h, int field, size_t* points, int* comps) {
    const Params& P = h->P;
    *points = (size_t)P.N;
    *comps = 3;
    switch (field) {
        case WF_FIELD_VEL: return h->vb[h->iF];
        case WF_FIELD_VEL_LAST_TIME: return h->vb[h->iT];
        case WF_FIELD_VEL_LAST_ITER: return h->iter_alias ? h->vb[h->iT] : h->vb[h->iI];
        case WF_FIELD_VEL_CORRECT: return h->uc;
        case WF_FIELD_D: return h->Dv;
        case WF_FIELD_B: return h->bv;
        case WF_FIELD_AODU: return h->aodu;
        case WF_FIELD_FACE_EDDY_VIS: return h->face;
        default: break;
    }
    *comps = 1;
    switch (field) {
        case WF_FIELD_PRES: return h->pr;
        case WF_FIELD_PRES_CORRECT: return h->pcb[h->iPC];
        case WF_FIELD_PRES_CORRECT_LAST_ITER: return h->pcb[h->iPCL];
        case WF_FIELD_DP: return h->Dp;
        case WF_FIELD_BP: return h->bp;
        case WF_FIELD_EDDY_VIS: return h->eddy;
        case WF_FIELD_DRAG: return h->drag;
        default: break;
    }
    if (field >= WF_FIELD_BND_X0 && field <= WF_FIELD_BND_ZN) {
        const int f = field - WF_FIELD_BND_X0;
        *points = (size_t)P.plane[f];
        *comps = 3;
        return h->bnd[f];
    }
    return nullptr;
}

}  // namespace

namespace wf {

bool step_graphable(const wf_solver* h) {
    return h->cfg.use_graph && !h->cfg.calc_residual && h->iter_alias && h->pc_zero;
}

int run_step_eager(wf_solver* h) {
    const long long l0 = g_launches;
    const int s = enqueue_step(h);
    h->launches += g_launches - l0;
    return s;
}

int ensure_step_graph(wf_solver* h, const wf_solver::GraphEntry** out) {
    const auto key = role_key(h);
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
        cudaGraph_t g = nullptr;
        WF_CUDA(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
        const int64_t step0 = h->step;
        const long long l0 = g_launches;
        const int s = enqueue_step(h);
        const long long nk = g_launches - l0;
        cudaError_t e = cudaStreamEndCapture(h->st, &g);
        const auto after = role_key(h);
        // capture only recorded the work: restore the roles it rotated
        set_roles(h, key);
        h->iter_alias = true;
        h->pc_zero = true;
        h->step = step0;
        g_launches = l0;
        if (s != WF_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        if (e != cudaSuccess) {
            h->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
            return WF_ERR_CUDA;
        }
        wf_solver::GraphEntry ent;
        ent.graph = g;
        ent.kernels = nk;
        ent.after = after;
        e = cudaGraphInstantiate(&ent.exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            h->err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
            return WF_ERR_CUDA;
        }
        it = h->graphs.emplace(key, ent).first;
    }
    *out = &it->second;
    return WF_OK;
}

int LoopRecorder::cut(wf_solver* h) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->st, &g);
    if (e != cudaSuccess) {
        h->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
        return WF_ERR_CUDA;
    }
    segments.push_back(g);
    e = cudaStreamBeginCapture(h->st, mode);
    if (e != cudaSuccess) {
        h->err = std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e);
        return WF_ERR_CUDA;
    }
    return WF_OK;
}

int capture_step_segments(wf_solver* h, LoopRecorder* rec, wf_solver::RoleKey* after, long long* kernels) {
    const auto key = role_key(h);
    const int64_t step0 = h->step;
    const long long l0 = g_launches;
    WF_CUDA(cudaStreamBeginCapture(h->st, rec->mode));
    h->rec = rec;
    const int s = enqueue_step(h);
    h->rec = nullptr;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->st, &g);
    if (g) rec->segments.push_back(g);
    *kernels = g_launches - l0;
    *after = role_key(h);
    // the capture only recorded the work: restore the roles it rotated
    set_roles(h, key);
    h->iter_alias = true;
    h->pc_zero = true;
    h->step = step0;
    g_launches = l0;
    if (s != WF_OK) return s;
    if (e != cudaSuccess) {
        h->err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e);
        return WF_ERR_CUDA;
    }
    return WF_OK;
}

void commit_graph_step(wf_solver* h, const wf_solver::GraphEntry& e) {
    set_roles(h, e.after);
    h->iter_alias = true;
    h->pc_zero = true;
    h->step += 1;
    h->launches += e.kernels;
}

void drop_graphs(wf_solver* h) {
    for (auto& kv : h->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    h->graphs.clear();
}

}  // namespace wf

// =====================================================================
extern "C" {

void wf_config_default(wf_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->struct_size = sizeof(wf_config);
    // FluidSimConfig.cs:113-178 defaults
    c->nx = 100; c->ny = 50; c->nz = 100;   // physDomainSize (10,5,10), gridResX 100
    c->dx = 0.1f;
    c->dt = 0.1f;
    c->mu = 0.005f;
    c->den = 1.0f;
    // canonical urban boundary set (Assets/Code/Config/AijBuilding0.asset)
    c->vel_bc[WF_FACE_X0] = WF_BND_FIXED_VALUE;
    c->vel_bc[WF_FACE_XN] = WF_BND_ZERO_GRAD;
    c->vel_bc[WF_FACE_Y0] = WF_BND_FIXED_VALUE;
    c->vel_bc[WF_FACE_YN] = WF_BND_SYMMETRY;
    c->vel_bc[WF_FACE_Z0] = WF_BND_SYMMETRY;
    c->vel_bc[WF_FACE_ZN] = WF_BND_SYMMETRY;
    c->pres_bc[WF_FACE_X0] = WF_BND_ZERO_GRAD;
    c->pres_bc[WF_FACE_XN] = WF_BND_FIXED_VALUE;
    c->pres_bc[WF_FACE_Y0] = WF_BND_ZERO_GRAD;
    c->pres_bc[WF_FACE_YN] = WF_BND_SYMMETRY;
    c->pres_bc[WF_FACE_Z0] = WF_BND_SYMMETRY;
    c->pres_bc[WF_FACE_ZN] = WF_BND_SYMMETRY;
    c->solver_type = WF_SOLVER_SIMPLE;
    c->piso_correctors = 2;
    c->turbulence = WF_TURB_NONE;
    c->cs = 0.15f;
    c->vel_iters = 50;
    c->pres_iters = 400;
    c->inflow_type = WF_INFLOW_CONSTANT;
    c->wind_speed = 10.0f;   // RuntimeConfig.windSpeed default
    c->inflow_ustar = 0.f;
    c->inflow_z0 = 1.0f;     // FvmSolverGpu.cs:818
    c->inflow_kappa = 0.4f;  // :817
    c->inflow_href = 10.0f;  // :819
    c->calc_residual = 0;
    c->vel_res_interval = 10;
    c->pres_res_interval = 20;
    c->vel_tol = 1e-15f;
    c->pres_tol = 1e-3f;
    c->compat_flags = 0;
    c->check_finite = 0;
    c->use_graph = 1;
}

int wf_create(const wf_config* cfg, int device, wf_solver** out) {
    if (!out) return WF_ERR_INVALID_ARG;
    *out = nullptr;
    if (const char* why = validate(cfg)) {
        (void)why;
        return WF_ERR_INVALID_ARG;
    }
    // Host-side fault injection for failure-path tests: no GPU work is done.
    if (const char* fi = std::getenv("WF_FAULT_INJECT")) {
        if (std::strcmp(fi, "oom") == 0) return WF_ERR_OOM;
        if (std::strcmp(fi, "cuda") == 0) return WF_ERR_CUDA;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return WF_ERR_CUDA;
    if (device < 0 || device >= ndev) return WF_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return WF_ERR_CUDA;

    auto* h = new (std::nothrow) wf_solver;
    if (!h) return WF_ERR_OOM;
    h->cfg = *cfg;
    h->device = device;
    h->wind = cfg->wind_speed;
    if (const char* fe = std::getenv("WF_FAST")) h->fast = std::atoi(fe);
    if (const char* pk = std::getenv("WF_PRES_K")) h->pres_k = std::min(std::max(std::atoi(pk), 1), 4);
    if (const char* vk = std::getenv("WF_VEL_K")) h->vel_k = std::min(std::max(std::atoi(vk), 1), 2);
    if (const char* v4 = std::getenv("WF_VEC4")) h->vec4 = std::atoi(v4);
    if (const char* pd = std::getenv("WF_PDL")) h->pdl = std::atoi(pd);
    if (const char* tm = std::getenv("WF_TMA")) h->pres_tma = std::atoi(tm);

    Params& P = h->P;
    P.nx = cfg->nx; P.ny = cfg->ny; P.nz = cfg->nz;
    P.N = cfg->nx * cfg->ny * cfg->nz;
    P.plane[WF_FACE_X0] = P.plane[WF_FACE_XN] = P.ny * P.nz;
    P.plane[WF_FACE_Y0] = P.plane[WF_FACE_YN] = P.nx * P.nz;
    P.plane[WF_FACE_Z0] = P.plane[WF_FACE_ZN] = P.nx * P.ny;
    P.dx = cfg->dx;
    P.ds = cfg->dx * cfg->dx;             // FluidSimConfig.cs:326
    P.dv = cfg->dx * cfg->dx * cfg->dx;   // :327
    P.dt = cfg->dt;
    P.nu = cfg->mu / cfg->den;            // :339
    P.den = cfg->den;
    P.rdx = 1.0f / P.dx;
    P.rdx2 = 1.0f / (2.f * P.dx);
    P.rden = 1.0f / P.den;
    P.dvden = P.dv / P.den;
    P.cs = cfg->cs;
    for (int i = 0; i < 3; ++i) P.force[i] = cfg->ext_force[i];
    for (int f = 0; f < 6; ++f) { P.vbc[f] = cfg->vel_bc[f]; P.pbc[f] = cfg->pres_bc[f]; }
    P.les = cfg->turbulence == WF_TURB_SMAGORINSKY;
    P.compat = cfg->compat_flags;
    P.vec4 = h->vec4;

    int s = WF_OK;
    auto fail = [&](int code) {
        free_all(h);
        delete h;
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) return fail(WF_ERR_CUDA);
    if (wf::sweeps_setup() != WF_OK) return fail(WF_ERR_CUDA);
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) return fail(WF_ERR_CUDA);
    const size_t N = P.N, v = 3 * sizeof(float) * N, sc = sizeof(float) * N;
    size_t planes = 0;
    for (int f = 0; f < 6; ++f) planes += 3 * (size_t)P.plane[f];
    const int nblk = wf::cell_grid_blocks(P);
    if ((s = alloc(h, (void**)&h->fl, N)) ||
        (s = alloc(h, (void**)&h->vb[0], v)) || (s = alloc(h, (void**)&h->vb[1], v)) ||
        (s = alloc(h, (void**)&h->vb[2], v)) || (s = alloc(h, (void**)&h->vb[3], v)) ||
        (s = alloc(h, (void**)&h->uc, v)) ||
        (s = alloc(h, (void**)&h->Dv, v)) || (s = alloc(h, (void**)&h->bv, v)) ||
        (s = alloc(h, (void**)&h->aodu, v)) || (s = alloc(h, (void**)&h->face, v)) ||
        (s = alloc(h, (void**)&h->pr, sc)) || (s = alloc(h, (void**)&h->pcb[0], sc)) ||
        (s = alloc(h, (void**)&h->pcb[1], sc)) || (s = alloc(h, (void**)&h->pcb[2], sc)) ||
        (s = alloc(h, (void**)&h->Dp, sc)) ||
        (s = alloc(h, (void**)&h->bp, sc)) || (s = alloc(h, (void**)&h->eddy, sc)) ||
        (s = alloc(h, (void**)&h->pcoef, 5 * sc)) || (s = alloc(h, (void**)&h->vcoef, 9 * sc)) ||
        (s = alloc(h, (void**)&h->grad, 9 * sc)) ||
        (s = alloc(h, (void**)&h->part, sizeof(double) * (size_t)std::max(nblk, 1))) ||
        (s = alloc(h, (void**)&h->dsum, 4 * sizeof(double))) || (s = alloc(h, (void**)&h->dref, sizeof(float) * 4)) ||
        (s = alloc(h, (void**)&h->dbad, sizeof(int) * 4)) || (s = alloc(h, (void**)&h->bnd[0], sizeof(float) * planes)))
        return fail(s);
    if ((s = alloc(h, (void**)&h->nbm, N))) return fail(s);
    P.nbm = h->nbm;
    wf::launch_nbmask(P, h->st, h->fl, h->nbm);  // all fluid until wf_init_flags
    for (int f = 1; f < 6; ++f) h->bnd[f] = h->bnd[f - 1] + 3 * (size_t)P.plane[f - 1];
    for (int f = 0; f < 6; ++f) h->B.p[f] = h->bnd[f];
    if (cudaMallocHost((void**)&h->hsum, 4 * sizeof(double)) != cudaSuccess) return fail(WF_ERR_OOM);
    if (cudaHostAlloc((void**)&h->hstat, sizeof(int), cudaHostAllocMapped) != cudaSuccess) return fail(WF_ERR_OOM);
    *h->hstat = 0;
    if (cudaHostGetDevicePointer((void**)&h->dstat, h->hstat, 0) != cudaSuccess) return fail(WF_ERR_CUDA);

    // Constructor sequence, FvmSolverGpu.cs:207-221.  Flags start all fluid
    // (zeroed allocation = CELL_FLUID); faceEddyVis starts at 0 because
    // InitFaceEddyVisField dispatches kernel 0 (:941-945).
    if ((s = wf_init_vel_pres_fields(h)) != WF_OK) return fail(s);
    if ((s = wf_set_fixed_value_vel_bnd_cond(h, h->wind)) != WF_OK) return fail(s);
    if ((s = sync(h)) != WF_OK) return fail(s);
    *out = h;
    return WF_OK;
}

int wf_destroy(wf_solver* h) {
    if (!h) return WF_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->st);
    free_all(h);
    delete h;
    return WF_OK;
}

int wf_init_flags(wf_solver* h, const int32_t* flags, size_t n) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!flags || n != (size_t)h->P.N) return set_err(h, WF_ERR_INVALID_ARG, "flags must hold nx*ny*nz int32");
    WF_CUDA(cudaSetDevice(h->device));
    if (!h->stage) WF_TRY(alloc(h, &h->stage, 4 * sizeof(float) * (size_t)h->P.N));
    WF_CUDA(cudaMemcpyAsync(h->stage, flags, n * sizeof(int32_t), cudaMemcpyHostToDevice, h->st));
    wf::launch_init_flags(h->P, h->st, (const int32_t*)h->stage, h->fl, h->vb[0], h->vb[1], h->vb[2]);
    wf::launch_init_flags(h->P, h->st, (const int32_t*)h->stage, h->fl, h->vb[3], nullptr, nullptr);
    wf::launch_nbmask(h->P, h->st, h->fl, h->nbm);
    WF_CHECK_LAUNCH();
    return sync(h);
}

int wf_init_vel_pres_fields(wf_solver* h) {
    if (!h) return WF_ERR_INVALID_ARG;
    WF_CUDA(cudaSetDevice(h->device));
    const wf_config& c = h->cfg;
    const int logp = c.inflow_type == WF_INFLOW_LOG;
    const float fric = logp ? fric_vel(h) : 0.f;
    const int centre = (c.compat_flags & WF_COMPAT_INIT_PROFILE_CELL_CENTRE) != 0;
    if (logp && h->nonuniform)
        wf::launch_nu_init_log(h, fric, c.inflow_kappa, c.inflow_z0);
    else
        wf::launch_init_fields(h->P, h->st, logp, h->wind, fric, c.inflow_kappa, c.inflow_z0, centre, h->vb[0],
                               h->vb[1], h->vb[2], h->uc, h->pr);
    WF_CHECK_LAUNCH();
    WF_CUDA(cudaMemcpyAsync(h->vb[3], h->vb[0], 3 * sizeof(float) * h->P.N, cudaMemcpyDeviceToDevice, h->st));
    for (int b = 0; b < 3; ++b) WF_CUDA(cudaMemsetAsync(h->pcb[b], 0, sizeof(float) * h->P.N, h->st));
    h->iter_alias = false;
    h->pc_zero = true;
    return sync(h);
}

int wf_set_fixed_value_vel_bnd_cond(wf_solver* h, float wind_speed) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!std::isfinite(wind_speed)) return set_err(h, WF_ERR_INVALID_ARG, "wind speed must be finite");
    WF_CUDA(cudaSetDevice(h->device));
    h->wind = wind_speed;
    const wf_config& c = h->cfg;
    if (c.inflow_type == WF_INFLOW_LOG && h->nonuniform) {
        wf::launch_nu_log_inlet(h, fric_vel(h), c.inflow_kappa, c.inflow_z0);
    } else if (c.inflow_type == WF_INFLOW_LOG) {
        wf::launch_set_log_inlet(h->P, h->st, fric_vel(h), c.inflow_kappa, c.inflow_z0, h->bnd[WF_FACE_X0]);
    } else {
        wf::launch_fill3(h->st, h->bnd[WF_FACE_X0], h->P.plane[WF_FACE_X0], wind_speed, 0.f, 0.f);
        wf::launch_fill3(h->st, h->bnd[WF_FACE_ZN], h->P.plane[WF_FACE_ZN], c.vel_zn[0], c.vel_zn[1], c.vel_zn[2]);
    }
    WF_CHECK_LAUNCH();
    return sync(h);
}

int wf_change_phys_field_pos(wf_solver* h) { return wf_init_vel_pres_fields(h); }

int wf_set_face_positions(wf_solver* h, const float* fx, const float* fy, const float* fz) {
    if (!h) return WF_ERR_INVALID_ARG;
    WF_CUDA(cudaSetDevice(h->device));
    const Params& P = h->P;
    if (!fx && !fy && !fz) {
        h->nonuniform = false;
        wf::drop_graphs(h);
        return WF_OK;
    }
    if (!fx || !fy || !fz) return set_err(h, WF_ERR_INVALID_ARG, "face positions: all three axes or none");
    // the reference has no PISO shader for this grid (FvmSolverGpu.cs:493-496)
    if (h->cfg.solver_type != WF_SOLVER_SIMPLE)
        return set_err(h, WF_ERR_UNSUPPORTED, "the non-uniform grid runs SIMPLE (the reference has no PISO for it)");
    const int n[3] = {P.nx, P.ny, P.nz};
    const float* f[3] = {fx, fy, fz};
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i < n[a]; ++i)
            if (!(std::isfinite(f[a][i]) && std::isfinite(f[a][i + 1]) && f[a][i + 1] > f[a][i]))
                return set_err(h, WF_ERR_INVALID_ARG, "face positions must be finite and strictly increasing");
    const size_t nf = (size_t)(P.nx + 1) + (P.ny + 1) + (P.nz + 1);
    if (!h->fpos) WF_TRY(alloc(h, (void**)&h->fpos, nf * sizeof(float)));
    if (!h->flux) WF_TRY(alloc(h, (void**)&h->flux, 3 * wf::nu_flux_texels(P) * sizeof(float)));
    if (!h->nucoef) WF_TRY(alloc(h, (void**)&h->nucoef, (size_t)wf::kNuCoefPlanes * P.N * sizeof(float)));
    WF_CUDA(cudaMemcpyAsync(h->fpos, fx, (P.nx + 1) * sizeof(float), cudaMemcpyHostToDevice, h->st));
    WF_CUDA(cudaMemcpyAsync(h->fpos + P.nx + 1, fy, (P.ny + 1) * sizeof(float), cudaMemcpyHostToDevice, h->st));
    WF_CUDA(cudaMemcpyAsync(h->fpos + P.nx + 1 + P.ny + 1, fz, (P.nz + 1) * sizeof(float), cudaMemcpyHostToDevice,
                            h->st));
    WF_CUDA(cudaMemsetAsync(h->flux, 0, 3 * wf::nu_flux_texels(P) * sizeof(float), h->st));
    h->nonuniform = true;
    wf::drop_graphs(h);
    return sync(h);
}

int wf_set_face_flux(wf_solver* h, const float* in) {
    if (!h || !in) return WF_ERR_INVALID_ARG;
    if (!h->nonuniform) return set_err(h, WF_ERR_INVALID_ARG, "no non-uniform grid set");
    WF_CUDA(cudaSetDevice(h->device));
    WF_CUDA(cudaMemcpyAsync(h->flux, in, 3 * wf::nu_flux_texels(h->P) * sizeof(float), cudaMemcpyHostToDevice,
                            h->st));
    return sync(h);
}

int wf_get_face_flux(wf_solver* h, float* out) {
    if (!h || !out) return WF_ERR_INVALID_ARG;
    if (!h->nonuniform) return set_err(h, WF_ERR_INVALID_ARG, "no non-uniform grid set");
    WF_CUDA(cudaSetDevice(h->device));
    WF_CUDA(cudaMemcpyAsync(out, h->flux, 3 * wf::nu_flux_texels(h->P) * sizeof(float), cudaMemcpyDeviceToHost,
                            h->st));
    return sync(h);
}

int wf_set_inflow_plane(wf_solver* h, const float* pl) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!pl) return set_err(h, WF_ERR_INVALID_ARG, "plane is NULL");
    WF_CUDA(cudaSetDevice(h->device));
    const size_t n = (size_t)h->P.plane[WF_FACE_X0];
    // The plane is transposed into a page-locked staging buffer owned by the
    // handle and copied on the solver stream, ordered before the next step,
    // without waiting for the GPU: the caller may reuse `pl` at once.  The
    // staging is rewritten only after the previous upload has left it.
    if (!h->in_stage) {
        if (cudaMallocHost((void**)&h->in_stage, 3 * n * sizeof(float)) != cudaSuccess) {
            h->in_stage = nullptr;
            cudaGetLastError();
            return set_err(h, WF_ERR_OOM, "page-locked staging for the inflow plane");
        }
        WF_CUDA(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
    } else {
        WF_CUDA(cudaEventSynchronize(h->ev_in));
    }
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) h->in_stage[(size_t)c * n + i] = pl[3 * i + c];
    WF_CUDA(cudaMemcpyAsync(h->bnd[WF_FACE_X0], h->in_stage, 3 * n * sizeof(float), cudaMemcpyHostToDevice, h->st));
    WF_CUDA(cudaEventRecord(h->ev_in, h->st));
    return WF_OK;
}

int wf_prepare_graphs(wf_solver* h) {
    if (!h) return WF_ERR_INVALID_ARG;
    WF_CUDA(cudaSetDevice(h->device));
    if (!wf::step_graphable(h)) return WF_OK;  // not in the replay state yet
    const auto start = role_key(h);
    for (int i = 0; i < 64; ++i) {
        const wf_solver::GraphEntry* e = nullptr;
        const int st = wf::ensure_step_graph(h, &e);
        if (st != WF_OK) {
            set_roles(h, start);
            return st;
        }
        set_roles(h, e->after);
        if (role_key(h) == start) break;
    }
    set_roles(h, start);
    return WF_OK;
}

namespace {
// Host NVTX range, closed when the scope ends.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace

int wf_step(wf_solver* h, int n_steps, int* ready) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (n_steps < 0) return set_err(h, WF_ERR_INVALID_ARG, "n_steps must be >= 0");
    NvtxRange range("wf_step");
    WF_CUDA(cudaSetDevice(h->device));
    WF_CUDA(cudaEventRecord(h->ev0, h->st));
    for (int i = 0; i < n_steps; ++i) WF_TRY(run_step(h));
    WF_CUDA(cudaEventRecord(h->ev1, h->st));
    WF_TRY(sync(h));
    WF_CUDA(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
    if (h->cfg.check_finite) WF_TRY(check_finite(h));
    if (ready) *ready = 1;
    return WF_OK;
}

int wf_step_async(wf_solver* h, int n_steps) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (n_steps < 0) return set_err(h, WF_ERR_INVALID_ARG, "n_steps must be >= 0");
    NvtxRange range("wf_step_async");
    WF_CUDA(cudaSetDevice(h->device));
    for (int i = 0; i < n_steps; ++i) WF_TRY(run_step(h));
    return WF_OK;
}

int wf_sync(wf_solver* h) {
    if (!h) return WF_ERR_INVALID_ARG;
    WF_CUDA(cudaSetDevice(h->device));
    return sync(h);
}

int wf_step_phases(wf_solver* h, float* phase_ms) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!phase_ms) return set_err(h, WF_ERR_INVALID_ARG, "phase_ms is NULL");
    NvtxRange range("wf_step_phases");
    WF_CUDA(cudaSetDevice(h->device));
    for (int p = 0; p < WF_PHASE_COUNT; ++p) phase_ms[p] = 0.f;
    struct Events {
        cudaEvent_t e[WF_PHASE_COUNT + 1] = {};
        ~Events() {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } E;
    for (cudaEvent_t& e : E.e) WF_CUDA(cudaEventCreate(&e));
    const wf_config& c = h->cfg;
    const long long l0 = wf::g_launches;
    int phase = -1;
    // closes the previous phase at the current point of the stream
    auto mark = [&](int next) -> int {
        if (phase >= 0) nvtxRangePop();
        WF_CUDA(cudaEventRecord(E.e[next], h->st));
        phase = next;
        if (next < WF_PHASE_COUNT) {
            static const char* names[WF_PHASE_COUNT] = {"les", "vel_pre", "vel_sweeps", "pres_pre",
                                                        "pres_sweeps", "correct", "piso", "end"};
            nvtxRangePushA(names[next]);
        }
        return WF_OK;
    };
    h->in_step = true;
    int st = WF_OK;
    do {
        if ((st = mark(WF_PHASE_LES)) != WF_OK) break;
        if (h->P.les && (st = do_les(h)) != WF_OK) break;
        if ((st = mark(WF_PHASE_VEL_PRE)) != WF_OK) break;
        if ((st = do_vel_precompute(h)) != WF_OK) break;
        if ((st = mark(WF_PHASE_VEL_SWEEPS)) != WF_OK) break;
        if ((st = do_vel_sweeps(h, c.vel_iters, true)) != WF_OK) break;
        if ((st = mark(WF_PHASE_PRES_PRE)) != WF_OK) break;
        if ((st = do_pres_precompute(h)) != WF_OK) break;
        if ((st = mark(WF_PHASE_PRES_SWEEPS)) != WF_OK) break;
        if ((st = do_pres_sweeps(h, c.pres_iters, true)) != WF_OK) break;
        if ((st = mark(WF_PHASE_CORRECT)) != WF_OK) break;
        if (h->nonuniform) {
            if ((st = do_apply_pres(h)) != WF_OK) break;
            if (!any_fixed_pres(c) && (st = do_normalize(h)) != WF_OK) break;
            if ((st = do_apply_vel(h)) != WF_OK) break;
        } else {
            if ((st = do_apply_vel_pres(h)) != WF_OK) break;
            if (!any_fixed_pres(c) && (st = do_normalize(h)) != WF_OK) break;
        }
        h->pc_zero = true;  // SetPresCorrectFieldtoZero (:1088)
        if ((st = mark(WF_PHASE_PISO)) != WF_OK) break;
        if (c.solver_type == WF_SOLVER_PISO)
            for (int n = 0; n < c.piso_correctors && st == WF_OK; ++n) st = do_piso(h, c.pres_iters, true);
        if (st != WF_OK) break;
        if ((st = mark(WF_PHASE_END)) != WF_OK) break;
        if ((st = do_end_step(h)) != WF_OK) break;
        st = mark(WF_PHASE_COUNT);
    } while (false);
    h->in_step = false;
    h->vcoef_step = false;
    if (phase >= 0 && phase < WF_PHASE_COUNT) nvtxRangePop();
    h->launches += wf::g_launches - l0;
    if (st != WF_OK) return st;
    WF_TRY(sync(h));
    for (int p = 0; p < WF_PHASE_COUNT; ++p) WF_CUDA(cudaEventElapsedTime(&phase_ms[p], E.e[p], E.e[p + 1]));
    if (h->cfg.check_finite) WF_TRY(check_finite(h));
    return WF_OK;
}

int wf_get_vel(wf_solver* h, float* out, int layout) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!out || layout < 0 || layout > 2) return set_err(h, WF_ERR_INVALID_ARG, "bad output or layout");
    WF_CUDA(cudaSetDevice(h->device));
    const size_t N = h->P.N;
    const float* src = h->vb[h->iT];
    if (layout == WF_LAYOUT_SOA) {
        WF_CUDA(cudaMemcpyAsync(out, src, 3 * N * sizeof(float), cudaMemcpyDeviceToHost, h->st));
        return sync(h);
    }
    if (!h->stage) WF_TRY(alloc(h, &h->stage, 4 * sizeof(float) * N));
    wf::launch_soa_to_interleaved(h->st, src, (int)N, (float*)h->stage, layout == WF_LAYOUT_XYZW);
    WF_CHECK_LAUNCH();
    const size_t per = layout == WF_LAYOUT_XYZW ? 4 : 3;
    WF_CUDA(cudaMemcpyAsync(out, h->stage, per * N * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    return sync(h);
}

int wf_readback_wait(wf_solver* h) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!h->rb_pending) return WF_OK;
    WF_CUDA(cudaSetDevice(h->device));
    h->rb_pending = false;
    WF_CUDA(cudaEventSynchronize(h->ev_done));
    return WF_OK;
}

int wf_readback_begin(wf_solver* h, float* vel, float* pres, int layout) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!vel || !pres || layout < 0 || layout > 2) return set_err(h, WF_ERR_INVALID_ARG, "bad output or layout");
    WF_CUDA(cudaSetDevice(h->device));
    WF_TRY(wf_readback_wait(h));
    const size_t N = h->P.N;
    if (!h->snap) {
        WF_TRY(alloc(h, (void**)&h->snap, 5 * sizeof(float) * N));
        WF_CUDA(cudaStreamCreateWithFlags(&h->cst, cudaStreamNonBlocking));
        WF_CUDA(cudaEventCreateWithFlags(&h->ev_snap, cudaEventDisableTiming));
        WF_CUDA(cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming));
    }
    // snapshot on the solver stream (ordered after the last step, before the
    // next one), then the copies to the host on the copy stream
    const size_t per = layout == WF_LAYOUT_XYZW ? 4 : 3;
    if (layout == WF_LAYOUT_SOA) {
        WF_CUDA(cudaMemcpyAsync(h->snap, h->vb[h->iT], 3 * sizeof(float) * N, cudaMemcpyDeviceToDevice, h->st));
    } else {
        wf::launch_soa_to_interleaved(h->st, h->vb[h->iT], (int)N, h->snap, layout == WF_LAYOUT_XYZW);
        WF_CHECK_LAUNCH();
    }
    float* psnap = h->snap + 4 * N;
    WF_CUDA(cudaMemcpyAsync(psnap, h->pr, sizeof(float) * N, cudaMemcpyDeviceToDevice, h->st));
    WF_CUDA(cudaEventRecord(h->ev_snap, h->st));
    WF_CUDA(cudaStreamWaitEvent(h->cst, h->ev_snap, 0));
    WF_CUDA(cudaMemcpyAsync(vel, h->snap, per * sizeof(float) * N, cudaMemcpyDeviceToHost, h->cst));
    WF_CUDA(cudaMemcpyAsync(pres, psnap, sizeof(float) * N, cudaMemcpyDeviceToHost, h->cst));
    WF_CUDA(cudaEventRecord(h->ev_done, h->cst));
    h->rb_pending = true;
    return WF_OK;
}

int wf_get_pres(wf_solver* h, float* out) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    WF_CUDA(cudaSetDevice(h->device));
    WF_CUDA(cudaMemcpyAsync(out, h->pr, h->P.N * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    return sync(h);
}

int wf_get_flags(wf_solver* h, int32_t* out) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    WF_CUDA(cudaSetDevice(h->device));
    if (!h->stage) WF_TRY(alloc(h, &h->stage, 4 * sizeof(float) * (size_t)h->P.N));
    wf::launch_flags_to_i32(h->st, h->fl, h->P.N, (int32_t*)h->stage);
    WF_CHECK_LAUNCH();
    WF_CUDA(cudaMemcpyAsync(out, h->stage, h->P.N * sizeof(int32_t), cudaMemcpyDeviceToHost, h->st));
    return sync(h);
}

int wf_get_state(wf_solver* h, float* vel, float* pres, int64_t* step) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (vel) WF_TRY(wf_get_vel(h, vel, WF_LAYOUT_SOA));
    if (pres) WF_TRY(wf_get_pres(h, pres));
    if (step) *step = h->step;
    return WF_OK;
}

int wf_set_state(wf_solver* h, const float* vel, const float* pres, int64_t step) {
    if (!h) return WF_ERR_INVALID_ARG;
    WF_CUDA(cudaSetDevice(h->device));
    const size_t N = h->P.N;
    if (vel) {
        // velFieldLastTime and velFieldLastIter both take the state, as after
        // a completed step (FvmSolverGpu.cs:1105-1106).
        WF_CUDA(cudaMemcpyAsync(h->vb[h->iT], vel, 3 * N * sizeof(float), cudaMemcpyHostToDevice, h->st));
        h->iter_alias = true;
    }
    if (pres) WF_CUDA(cudaMemcpyAsync(h->pr, pres, N * sizeof(float), cudaMemcpyHostToDevice, h->st));
    h->pc_zero = true;
    for (int b = 0; b < 3; ++b) WF_CUDA(cudaMemsetAsync(h->pcb[b], 0, sizeof(float) * N, h->st));
    h->step = step;
    return sync(h);
}

int wf_field_size(const wf_solver* hc, int field, size_t* points, int* comps) {
    wf_solver* h = const_cast<wf_solver*>(hc);
    if (!h || !points || !comps) return WF_ERR_INVALID_ARG;
    if (field == WF_FIELD_DRAG) {  // stored only once set
        *points = (size_t)h->P.N;
        *comps = 1;
        return WF_OK;
    }
    if (!field_ptr(h, field, points, comps)) return WF_ERR_INVALID_ARG;
    return WF_OK;
}

int wf_get_field(wf_solver* h, int field, float* out) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    WF_CUDA(cudaSetDevice(h->device));
    if ((field == WF_FIELD_PRES_CORRECT || field == WF_FIELD_PRES_CORRECT_LAST_ITER) && h->pc_zero)
        WF_TRY(materialize_pc(h));
    if (field == WF_FIELD_DRAG && !h->drag) {
        for (int i = 0; i < h->P.N; ++i) out[i] = 0.f;
        return WF_OK;
    }
    size_t n = 0;
    int comps = 0;
    float* p = field_ptr(h, field, &n, &comps);
    if (!p) return set_err(h, WF_ERR_INVALID_ARG, "unknown field id");
    WF_CUDA(cudaMemcpyAsync(out, p, n * comps * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    return sync(h);
}

int wf_set_field(wf_solver* h, int field, const float* in) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!in) return set_err(h, WF_ERR_INVALID_ARG, "in is NULL");
    WF_CUDA(cudaSetDevice(h->device));
    if (field == WF_FIELD_VEL_LAST_TIME || field == WF_FIELD_VEL_LAST_ITER) WF_TRY(materialize_iter(h));
    if (field == WF_FIELD_PRES_CORRECT || field == WF_FIELD_PRES_CORRECT_LAST_ITER) WF_TRY(materialize_pc(h));
    if (field == WF_FIELD_D) ++h->d_gen;
    if (field == WF_FIELD_DRAG && !h->drag) {
        // first use: the captured step graphs hold the old (null) pointer
        WF_TRY(sync(h));
        wf::drop_graphs(h);
        WF_TRY(alloc(h, (void**)&h->drag, sizeof(float) * h->P.N));
    }
    size_t n = 0;
    int comps = 0;
    float* p = field_ptr(h, field, &n, &comps);
    if (!p) return set_err(h, WF_ERR_INVALID_ARG, "unknown field id");
    WF_CUDA(cudaMemcpyAsync(p, in, n * comps * sizeof(float), cudaMemcpyHostToDevice, h->st));
    return sync(h);
}

int wf_get_device_fields(wf_solver* h, wf_device_fields* out) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    const size_t N = h->P.N;
    for (int c = 0; c < 3; ++c) out->vel[c] = h->vb[h->iT] + c * N;
    out->pres = h->pr;
    out->flags = h->fl;
    out->n_cells = (int64_t)N;
    out->stream = (void*)h->st;
    return WF_OK;
}

int wf_residuals(wf_solver* h, float* vel, float* pres, float* mass) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (vel) *vel = h->res_vel;
    if (pres) *pres = h->res_pres;
    if (mass) {
        if (!h->cfg.calc_residual) {
            *mass = -1.f;
        } else {
            double m = 0.0;
            WF_TRY(wf_mass_imbalance(h, &m));
            *mass = (float)m;
        }
    }
    return WF_OK;
}

int wf_mass_imbalance(wf_solver* h, double* out) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    WF_CUDA(cudaSetDevice(h->device));
    wf::launch_mass_imbalance(h->P, h->B, h->st, h->fl, h->vb[h->iT], h->part, h->dsum);
    WF_CHECK_LAUNCH();
    return read_residual(h, out);
}

int wf_check_finite(wf_solver* h) {
    if (!h) return WF_ERR_INVALID_ARG;
    WF_CUDA(cudaSetDevice(h->device));
    return check_finite(h);
}

// ------------------------------------------------------------- per-kernel ops
#define WF_OP_BEGIN()                       \
    if (!h) return WF_ERR_INVALID_ARG;      \
    WF_CUDA(cudaSetDevice(h->device))

int wf_op_wallfunc(wf_solver* h) {
    WF_OP_BEGIN();
    wf::launch_wallfunc(h->P, h->st, h->fl, h->vb[h->iT], h->face);
    WF_CHECK_LAUNCH();
    return sync(h);
}
int wf_op_eddy_vis(wf_solver* h) {
    WF_OP_BEGIN();
    wf::launch_eddy_vis(h->P, h->B, h->st, h->fl, h->vb[h->iT], h->eddy, nullptr);
    WF_CHECK_LAUNCH();
    return sync(h);
}
int wf_op_les_term(wf_solver* h) {
    WF_OP_BEGIN();
    // the gradient tensors are rebuilt from velFieldLastTime (the eddy
    // viscosity may have been set independently)
    wf::launch_cell_grad(h->P, h->B, h->st, h->fl, h->vb[h->iT], h->grad);
    wf::launch_les_term(h->P, h->B, h->st, h->fl, h->vb[h->iT], h->eddy, h->face, h->grad, h->bv);
    WF_CHECK_LAUNCH();
    return sync(h);
}
int wf_op_vel_precompute(wf_solver* h) {
    WF_OP_BEGIN();
    WF_TRY(do_vel_precompute(h));
    return sync(h);
}
int wf_op_vel_sweeps(wf_solver* h, int n) {
    WF_OP_BEGIN();
    if (n < 0) return set_err(h, WF_ERR_INVALID_ARG, "n must be >= 0");
    WF_TRY(do_vel_sweeps(h, n, true));
    return sync(h);
}
int wf_op_pres_precompute(wf_solver* h) {
    WF_OP_BEGIN();
    WF_TRY(do_pres_precompute(h));
    return sync(h);
}
int wf_op_pres_sweeps(wf_solver* h, int n) {
    WF_OP_BEGIN();
    if (n < 0) return set_err(h, WF_ERR_INVALID_ARG, "n must be >= 0");
    WF_TRY(do_pres_sweeps(h, n, true));
    return sync(h);
}
int wf_op_apply_pres(wf_solver* h) {
    WF_OP_BEGIN();
    WF_TRY(do_apply_pres(h));
    return sync(h);
}
int wf_op_normalize(wf_solver* h) {
    WF_OP_BEGIN();
    WF_TRY(do_normalize(h));
    return sync(h);
}
int wf_op_apply_vel(wf_solver* h) {
    WF_OP_BEGIN();
    WF_TRY(do_apply_vel(h));
    return sync(h);
}
int wf_op_zero_pres_correct(wf_solver* h) {
    WF_OP_BEGIN();
    h->pc_zero = true;
    WF_TRY(materialize_pc(h));
    h->pc_zero = true;
    return sync(h);
}
int wf_op_piso(wf_solver* h, int n) {
    WF_OP_BEGIN();
    if (n < 0) return set_err(h, WF_ERR_INVALID_ARG, "n must be >= 0");
    WF_TRY(do_piso(h, n, true));
    return sync(h);
}
int wf_op_end_step(wf_solver* h) {
    WF_OP_BEGIN();
    WF_TRY(do_end_step(h));
    return sync(h);
}
int wf_op_vel_residual(wf_solver* h, float* out) {
    WF_OP_BEGIN();
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    const float* uI = h->iter_alias ? h->vb[h->iT] : h->vb[h->iI];
    wf::launch_vel_residual(h->P, h->st, h->Dv, h->vb[h->iF], uI, h->part, h->dsum);
    WF_CHECK_LAUNCH();
    double s = 0.0;
    WF_TRY(read_residual(h, &s));
    *out = (float)std::sqrt(s / (3.0 * h->P.N));
    return WF_OK;
}
int wf_op_pres_residual(wf_solver* h, float* out) {
    WF_OP_BEGIN();
    if (!out) return set_err(h, WF_ERR_INVALID_ARG, "out is NULL");
    wf::launch_pres_residual(h->P, h->st, h->Dp, pc_cur(h), h->pc_zero ? nullptr : h->pcb[h->iPCL], h->part,
                             h->dsum);
    WF_CHECK_LAUNCH();
    double s = 0.0;
    WF_TRY(read_residual(h, &s));
    *out = (float)std::sqrt(s / double(h->P.N));
    return WF_OK;
}

const char* wf_last_error(const wf_solver* h) { return h ? h->err.c_str() : "null handle"; }

const char* wf_strerror(int s) {
    switch (s) {
        case WF_OK: return "ok";
        case WF_ERR_INVALID_ARG: return "invalid argument";
        case WF_ERR_CUDA: return "CUDA runtime error";
        case WF_ERR_OOM: return "out of device memory";
        case WF_ERR_NONFINITE: return "non-finite value in the solution";
        case WF_ERR_TIMEOUT: return "bounded device wait timed out";
        case WF_ERR_UNSUPPORTED: return "unsupported option";
        case WF_NOT_FINISHED: return "step not finished";
        case WF_ERR_STATE: return "invalid handle state";
        case WF_ERR_IO: return "file error";
        default: return "unknown status";
    }
}

int wf_version(void) { return WF_ABI_VERSION; }

int wf_last_step_ms(const wf_solver* h, float* ms) {
    if (!h || !ms) return WF_ERR_INVALID_ARG;
    *ms = h->last_ms;
    return WF_OK;
}

int wf_kernel_launches(const wf_solver* h, int64_t* total) {
    if (!h || !total) return WF_ERR_INVALID_ARG;
    *total = h->launches;
    return WF_OK;
}

int wf_stage_wait_selftest(wf_solver* h, int short_stage, double timeout_ms, int* status) {
    if (!h || !status || !(timeout_ms > 0)) return WF_ERR_INVALID_ARG;
    if (h->nonuniform) return set_err(h, WF_ERR_UNSUPPORTED, "the TMA pass runs on the uniform grid only");
    WF_CUDA(cudaSetDevice(h->device));
    const size_t N = h->P.N;
    if (!h->stage) WF_TRY(alloc(h, &h->stage, 4 * N * sizeof(float)));
    float* out = static_cast<float*>(h->stage);
    if (!wf::pres_tma_ok(h->P, h->pcoef, h->pcoef + 3 * N, h->bp, nullptr))
        return set_err(h, WF_ERR_UNSUPPORTED, "the TMA pass needs nx % 4 == 0");
    WF_TRY(sync(h));
    WF_CUDA(wf::launch_pres_tma4(h->P, h->st, h->num_sms, h->pcoef, h->pcoef + 3 * N, h->bp, nullptr, out, nullptr,
                                 nullptr, h->dstat, timeout_ms, short_stage != 0));
    WF_CUDA(cudaStreamSynchronize(h->st));
    *status = *(volatile int*)h->hstat ? WF_ERR_TIMEOUT : WF_OK;
    *(volatile int*)h->hstat = 0;
    return WF_OK;
}

int wf_time_kernel(wf_solver* h, int kernel, int reps, int flush_l2, float* ms_per_launch,
                   double* alg_bytes_per_launch, int* sweeps_per_launch) {
    if (!h) return WF_ERR_INVALID_ARG;
    if (h->nonuniform) return set_err(h, WF_ERR_UNSUPPORTED, "times the uniform-grid Jacobi kernels");
    if (!ms_per_launch || !alg_bytes_per_launch || !sweeps_per_launch || reps <= 0 ||
        (kernel != WF_KERNEL_PRES_SWEEP && kernel != WF_KERNEL_VEL_SWEEP))
        return set_err(h, WF_ERR_INVALID_ARG, "bad kernel id, reps or output pointer");
    WF_CUDA(cudaSetDevice(h->device));
    const int s = wf::time_kernel(h, kernel, reps, flush_l2 != 0, ms_per_launch, alg_bytes_per_launch,
                                  sweeps_per_launch);
    if (s != WF_OK) return set_err(h, s, "kernel timing failed");
    return WF_OK;
}

}  // extern "C"
