// wf_sweeps.cu - fast Jacobi loops.
//
// The Jacobi operators of the reference (CSVelPredict, FvmColl.compute:
// 1863-2069; CSPresCorrectRhieChow, :2790-2848; CSPisoPresCorrection,
// PisoColl.compute:181-256) rebuild their off-diagonal coefficients from
// velFieldLastTime, the eddy viscosities, the flags and DField on every
// sweep, although none of these change inside the loop.  Here the
// coefficients are formed once per loop and each sweep reads only the
// coefficients, the right-hand side and the previous iterate:
//
//   momentum:  u_P = (1/D_P) (sum_f A_f u_f + b_P), A_f = nu_f ds/dx -/+ F_f/4
//              per cell: 6 A_f + 3 (1/D) + 3 b + 3 u  (float, SoA)
//   pressure:  p_P = (1/Dp_P) (rhs_P - sum_f c_f p_f), c_f shared by the two
//              cells of a face: per cell c_E, c_N, c_U, 1/Dp, rhs, p.
//
// A coefficient is 0 on faces that are not fluid-fluid, which reproduces the
// reference's InRegionAndIsFluid tests; 1/D (1/Dp) is 0 on non-fluid cells,
// which are skipped as in the reference.
#include <cuda_runtime.h>

#include <utility>

#include "wf_kernels.cuh"
#include "wf_sweeps.cuh"

namespace wf {

namespace {

__device__ __forceinline__ float ld(const float* p, size_t i) { return __ldg(p + i); }
__device__ __forceinline__ bool fluid_at(const uint8_t* fl, int i) { return __ldg(fl + i) == WF_CELL_FLUID; }

__device__ __forceinline__ float face_read(const Params& P, const float* face, int i, int axis) {
    if ((P.compat & WF_COMPAT_RFLOAT_FACE_EDDY_VIS) && axis != 0) return 0.f;
    return ld(face, (size_t)axis * P.N + i);
}
// Same face viscosity as the reference sweep (FvmColl.compute:1962-2001).
__device__ __forceinline__ float vis_face(const Params& P, const uint8_t* fl, const float* eddy, const float* face,
                                          int x, int y, int z, int i, int f) {
    if (!P.les) return P.nu;
    const int X = x + face_ox(f), Y = y + face_oy(f), Z = z + face_oz(f);
    const float eP = ld(eddy, i);
    float v = P.nu + eP;
    if (in_region(P, X, Y, Z)) {
        const int q = cidx(P, X, Y, Z);
        if (fluid_at(fl, q)) v = P.nu + 0.5f * (eP + ld(eddy, q));
        else v = P.nu + face_read(P, face, face_sign(f) > 0 ? q : i, face_axis(f));
    } else if (f == 3 && P.vbc[WF_FACE_Y0] == WF_BND_FIXED_VALUE) {
        v = P.nu + face_read(P, face, i, 1);
    }
    return v;
}

// Momentum coefficients.  A: 6 planes (faces E,W,N,S,U,D), iD: 3 planes.
__global__ void k_vel_coef(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                           const float* __restrict__ uT, const float* __restrict__ eddy,
                           const float* __restrict__ face, const float* __restrict__ Dv,
                           float* __restrict__ A, float* __restrict__ iD) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    if (!fluid_at(fl, i)) {
#pragma unroll
        for (int f = 0; f < 6; ++f) A[f * N + i] = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) iD[k * N + i] = 0.f;
        return;
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const int X = x + face_ox(f), Y = y + face_oy(f), Z = z + face_oz(f);
        float c = 0.f;
        if (in_region(P, X, Y, Z)) {
            const int q = cidx(P, X, Y, Z);
            if (fluid_at(fl, q)) {
                const float conv = P.ds * 0.25f * (ld(uT, a * N + i) + ld(uT, a * N + q));
                const float vis = vis_face(P, fl, eddy, face, x, y, z, i, f);
                const float dif = vis * P.ds / P.dx;
                c = face_sign(f) > 0 ? dif - conv : dif + conv;
            }
        }
        A[f * N + i] = c;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) iD[k * N + i] = 1.0f / ld(Dv, k * N + i);
}

// One momentum sweep: uo_P = iD_P (sum_f A_f ui_f + b_P) on fluid cells.
__global__ void __launch_bounds__(256) k_vel_sweep1(const __grid_constant__ Params P, const float* __restrict__ A,
                                                    const float* __restrict__ iD, const float* __restrict__ bv,
                                                    const float* __restrict__ ui, float* __restrict__ uo) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    const float d0 = ld(iD, i);
    if (d0 == 0.f) return;  // non-fluid cell
    const float a0 = ld(A, i), a1 = ld(A, N + i), a2 = ld(A, 2 * N + i);
    const float a3 = ld(A, 3 * N + i), a4 = ld(A, 4 * N + i), a5 = ld(A, 5 * N + i);
    const int sx = P.nx, sz = P.nx * P.ny;
    const int iE = x + 1 < P.nx ? i + 1 : i, iW = x > 0 ? i - 1 : i;
    const int iN = y + 1 < P.ny ? i + sx : i, iS = y > 0 ? i - sx : i;
    const int iU = z + 1 < P.nz ? i + sz : i, iDn = z > 0 ? i - sz : i;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float* u = ui + k * N;
        float s = a0 * ld(u, iE);
        s += a1 * ld(u, iW);
        s += a2 * ld(u, iN);
        s += a3 * ld(u, iS);
        s += a4 * ld(u, iU);
        s += a5 * ld(u, iDn);
        const float dk = k == 0 ? d0 : ld(iD, k * N + i);
        uo[k * N + i] = dk * (s + ld(bv, k * N + i));
    }
}

// Pressure face coefficients c_E, c_N, c_U (FvmColl.compute:2813-2814 form
// ((dv/den) * DInv) / dx) for fluid-fluid faces, else 0.
__global__ void k_pres_coef(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                            const float* __restrict__ Dv, float* __restrict__ c3) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    const bool me = fluid_at(fl, i);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int f = 2 * a;  // E, N, U
        const int X = x + face_ox(f), Y = y + face_oy(f), Z = z + face_oz(f);
        float c = 0.f;
        if (me && in_region(P, X, Y, Z)) {
            const int q = cidx(P, X, Y, Z);
            if (fluid_at(fl, q)) {
                const float DInv = 0.5f * (1.f / ld(Dv, a * N + i) + 1.f / ld(Dv, a * N + q));
                c = (P.dv / P.den) * DInv / P.dx;
            }
        }
        c3[a * N + i] = c;
    }
}

// 1/Dp for the SIMPLE pressure equation (0 on non-fluid cells).
__global__ void k_inv(const __grid_constant__ Params P, const uint8_t* __restrict__ fl, const float* __restrict__ Dp,
                      float* __restrict__ ainv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.N) return;
    ainv[i] = fluid_at(fl, i) ? 1.f / ld(Dp, i) : 0.f;
}

// PISO diagonal and right-hand side (PisoColl.compute:196-255, the parts of
// the sweep that do not involve p''): ainv = 1/presCoeff, rhs = velTerm.
__global__ void k_piso_pre(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                           const float* __restrict__ Dv, const float* __restrict__ aodu,
                           float* __restrict__ ainv, float* __restrict__ rhs) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    if (!fluid_at(fl, i)) {
        ainv[i] = 0.f;
        rhs[i] = 0.f;
        return;
    }
    const bool consistent = (P.compat & WF_COMPAT_PISO_CONSISTENT) != 0;
    float coeff = 0.f, vt = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const int X = x + face_ox(f), Y = y + face_oy(f), Z = z + face_oz(f);
        if (!in_region(P, X, Y, Z)) {
            if (consistent && P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE) {
                const float DInv = 1.f / ld(Dv, a * N + i);
                coeff -= 2.f * (P.dv / P.den) * DInv / P.dx;
            }
            continue;
        }
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float AdInv = 0.5f * (1.f / ld(Dv, a * N + i) + 1.f / ld(Dv, a * N + q));
        const float Aod = 0.5f * (ld(aodu, a * N + i) + ld(aodu, a * N + q));
        if (a == 0) coeff -= (P.dv / P.den) * (AdInv / P.dx);
        else coeff -= (P.dv / P.den) * AdInv / P.dx;
        vt = face_sign(f) > 0 ? vt - AdInv * Aod : vt + AdInv * Aod;
    }
    ainv[i] = 1.f / coeff;
    rhs[i] = vt;
}

// One pressure sweep: po_P = ainv_P (rhs_P - sum_f c_f pi_f) on fluid cells;
// pi == nullptr is the all-zero iterate.
__global__ void __launch_bounds__(256) k_pres_sweep1(const __grid_constant__ Params P, const float* __restrict__ c3,
                                                     const float* __restrict__ ainv, const float* __restrict__ rhs,
                                                     const float* __restrict__ pi, float* __restrict__ po) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    const float ai = ld(ainv, i);
    if (ai == 0.f) return;
    float t = 0.f;
    if (pi) {
        const int sx = P.nx, sz = P.nx * P.ny;
        const float* cE = c3;
        const float* cN = c3 + N;
        const float* cU = c3 + 2 * N;
        if (x + 1 < P.nx) t -= ld(cE, i) * ld(pi, i + 1);
        if (x > 0) t -= ld(cE, i - 1) * ld(pi, i - 1);
        if (y + 1 < P.ny) t -= ld(cN, i) * ld(pi, i + sx);
        if (y > 0) t -= ld(cN, i - sx) * ld(pi, i - sx);
        if (z + 1 < P.nz) t -= ld(cU, i) * ld(pi, i + sz);
        if (z > 0) t -= ld(cU, i - sz) * ld(pi, i - sz);
    }
    po[i] = ai * (t + ld(rhs, i));
}

dim3 blk() { return dim3(32, 4, 2); }
dim3 grd(const Params& P) {
    dim3 b = blk();
    return dim3((P.nx + b.x - 1) / b.x, (P.ny + b.y - 1) / b.y, (P.nz + b.z - 1) / b.z);
}

void vel_coef(wf_solver* h) {
    const Params& P = h->P;
    const size_t N = P.N;
    WF_COUNT_LAUNCH();
    k_vel_coef<<<grd(P), blk(), 0, h->st>>>(P, h->fl, h->vb[h->iT], h->eddy, h->face, h->Dv, h->vcoef,
                                            h->vcoef + 6 * N);
}

void launch_vel_sweep_fast(wf_solver* h, const float* src, float* dst) {
    const Params& P = h->P;
    const size_t N = P.N;
    WF_COUNT_LAUNCH();
    k_vel_sweep1<<<grd(P), blk(), 0, h->st>>>(P, h->vcoef, h->vcoef + 6 * N, h->bv, src, dst);
}

// Pressure coefficients of the SIMPLE (piso = false) or PISO equation;
// returns the right-hand side plane.
const float* pres_coef(wf_solver* h, bool piso) {
    const Params& P = h->P;
    const size_t N = P.N;
    float* c3 = h->pcoef;
    float* ainv = h->pcoef + 3 * N;
    float* rhs = piso ? h->pcoef + 4 * N : h->bp;
    WF_COUNT_LAUNCH();
    k_pres_coef<<<grd(P), blk(), 0, h->st>>>(P, h->fl, h->Dv, c3);
    WF_COUNT_LAUNCH();
    if (piso) {
        k_piso_pre<<<grd(P), blk(), 0, h->st>>>(P, h->fl, h->Dv, h->aodu, ainv, rhs);
    } else {
        k_inv<<<(P.N + 255) / 256, 256, 0, h->st>>>(P, h->fl, h->Dp, ainv);
    }
    return rhs;
}

void launch_pres_sweep_fast(wf_solver* h, const float* rhs, const float* src, float* dst) {
    const Params& P = h->P;
    const size_t N = P.N;
    WF_COUNT_LAUNCH();
    k_pres_sweep1<<<grd(P), blk(), 0, h->st>>>(P, h->pcoef, h->pcoef + 3 * N, rhs, src, dst);
}

}  // namespace

int vel_sweeps_fast(wf_solver* h, int n) {
    vel_coef(h);
    for (int k = 0; k < n; ++k) {
        const float* src = h->iter_alias ? h->vb[h->iT] : h->vb[h->iI];
        launch_vel_sweep_fast(h, src, h->vb[h->iF]);
        std::swap(h->iI, h->iF);
        h->iter_alias = false;
    }
    std::swap(h->iI, h->iF);
    return cudaGetLastError() == cudaSuccess ? WF_OK : WF_ERR_CUDA;
}

int pres_sweeps_fast(wf_solver* h, int n, bool piso) {
    const float* rhs = pres_coef(h, piso);
    for (int k = 0; k < n; ++k) {
        const float* src = h->pc_zero ? nullptr : h->pcb[h->iPCL];
        launch_pres_sweep_fast(h, rhs, src, h->pcb[h->iPC]);
        h->pc_zero = false;
        std::swap(h->iPCL, h->iPC);
    }
    std::swap(h->iPCL, h->iPC);
    return cudaGetLastError() == cudaSuccess ? WF_OK : WF_ERR_CUDA;
}

// Times the step's hot kernels on scratch copies of the iterate; the solver
// fields are not modified (coefficient caches are rebuilt from the current
// fields, as the next step would).
int time_kernel(wf_solver* h, int which, int reps, bool flush, float* ms, double* bytes, int* sweeps) {
    const Params& P = h->P;
    const size_t N = P.N;
    if (reps <= 0) return WF_ERR_INVALID_ARG;
    const size_t flush_bytes = size_t(256) << 20;
    void* fbuf = nullptr;
    float* scratch = nullptr;
    const size_t per = which == WF_KERNEL_VEL_SWEEP ? 3 : 1;
    if (cudaMalloc(&scratch, 2 * per * N * sizeof(float)) != cudaSuccess) return WF_ERR_OOM;
    if (flush && cudaMalloc(&fbuf, flush_bytes) != cudaSuccess) {
        cudaFree(scratch);
        return WF_ERR_OOM;
    }
    float* a = scratch;
    float* b = scratch + per * N;
    const long long saved = g_launches;
    const float* rhs = nullptr;
    if (which == WF_KERNEL_VEL_SWEEP) {
        vel_coef(h);
        cudaMemcpyAsync(a, h->vb[h->iT], 3 * N * sizeof(float), cudaMemcpyDeviceToDevice, h->st);
    } else {
        rhs = pres_coef(h, false);
        cudaMemsetAsync(a, 0, N * sizeof(float), h->st);
    }
    cudaMemcpyAsync(b, a, per * N * sizeof(float), cudaMemcpyDeviceToDevice, h->st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float total = 0.f;
    for (int r = 0; r < reps; ++r) {
        if (flush) cudaMemsetAsync(fbuf, r & 0xff, flush_bytes, h->st);
        cudaEventRecord(e0, h->st);
        if (which == WF_KERNEL_VEL_SWEEP) launch_vel_sweep_fast(h, a, b);
        else launch_pres_sweep_fast(h, rhs, a, b);
        cudaEventRecord(e1, h->st);
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        total += t;
        std::swap(a, b);
    }
    g_launches = saved;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t err = cudaGetLastError();
    cudaStreamSynchronize(h->st);
    cudaFree(scratch);
    if (fbuf) cudaFree(fbuf);
    if (err != cudaSuccess) return WF_ERR_CUDA;
    *ms = total / reps;
    *sweeps = 1;
    // compulsory bytes of the reference kernels per cell and sweep:
    // CSPresCorrectRhieChow 29 B, CSVelPredict 77 B
    *bytes = double(which == WF_KERNEL_VEL_SWEEP ? 77 : 29) * double(N);
    return WF_OK;
}

}  // namespace wf
