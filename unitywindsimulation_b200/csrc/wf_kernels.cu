// wf_kernels.cu - per-operation CUDA kernels of the collocated SIMPLE/PISO LES
// step (one thread per cell).  Each kernel restates one HLSL kernel of
// puppy2333/UnityWindSimulation (file:line given on each) with the same face
// order and operand order, on the SoA device layout of wf_common.cuh.
//
// These are the building blocks of the step and of the per-kernel parity
// entry points (wf_op_*).  The hot Jacobi loops have faster multi-sweep
// kernels in wf_sweeps.cu; these single-sweep kernels remain the reference
// form they are checked against.
#include <cuda_runtime.h>

#include "wf_common.cuh"
#include "wf_kernels.cuh"

namespace wf {

namespace {

__device__ __forceinline__ float ld(const float* p, size_t i) { return __ldg(p + i); }
__device__ __forceinline__ bool fluid_at(const uint8_t* fl, int i) { return __ldg(fl + i) == WF_CELL_FLUID; }

struct Cell {
    int x, y, z, i;
};
__device__ __forceinline__ bool cell_of_thread(const Params& P, Cell& c) {
    c.x = blockIdx.x * blockDim.x + threadIdx.x;
    c.y = blockIdx.y * blockDim.y + threadIdx.y;
    c.z = blockIdx.z * blockDim.z + threadIdx.z;
    if (c.x >= P.nx || c.y >= P.ny || c.z >= P.nz) return false;
    c.i = cidx(P, c.x, c.y, c.z);
    return true;
}

// faceEddyVisField read; single channel under WF_COMPAT_RFLOAT_FACE_EDDY_VIS
// (FvmSolverGpu.cs:304 allocates it RFloat).
__device__ __forceinline__ float face_read(const Params& P, const float* face, int i, int axis) {
    if ((P.compat & WF_COMPAT_RFLOAT_FACE_EDDY_VIS) && axis != 0) return 0.f;
    return ld(face, (size_t)axis * P.N + i);
}

// Face viscosity nu + nu_t, FvmColl.compute:1596-1635 (also :1962-2001 and
// LES.compute:643-679).
__device__ __forceinline__ float vis_face(const Params& P, const uint8_t* fl, const float* eddy,
                                          const float* face, const Cell& c, int f) {
    if (!P.les) return P.nu;
    const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
    const float eP = ld(eddy, c.i);
    float v = P.nu + eP;
    if (in_region(P, X, Y, Z)) {
        const int q = cidx(P, X, Y, Z);
        if (fluid_at(fl, q)) {
            v = P.nu + 0.5f * (eP + ld(eddy, q));
        } else {
            v = P.nu + face_read(P, face, face_sign(f) > 0 ? q : c.i, face_axis(f));
        }
    } else if (f == 3 && P.vbc[WF_FACE_Y0] == WF_BND_FIXED_VALUE) {
        v = P.nu + face_read(P, face, c.i, 1);
    }
    return v;
}

// vis_face from the neighbour mask (same values).
__device__ __forceinline__ float vis_face_m(const Params& P, unsigned m, const float* eddy, const float* face,
                                            const Cell& c, int f) {
    if (!P.les) return P.nu;
    const float eP = ld(eddy, c.i);
    float v = P.nu + eP;
    if (face_in(P, c.x, c.y, c.z, f)) {
        const int q = c.i + face_off(P, f);
        if (nb_fluid(m, f)) {
            v = P.nu + 0.5f * (eP + ld(eddy, q));
        } else {
            v = P.nu + face_read(P, face, face_sign(f) > 0 ? q : c.i, face_axis(f));
        }
    } else if (f == 3 && P.vbc[WF_FACE_Y0] == WF_BND_FIXED_VALUE) {
        v = P.nu + face_read(P, face, c.i, 1);
    }
    return v;
}
// vis_face_m with the eddy viscosities of the cell (eP) and of the neighbour
// across f (eQ) already loaded.  Same values.
__device__ __forceinline__ float vis_face_v(const Params& P, unsigned m, const float* face, const Cell& c, int f,
                                            float eP, float eQ) {
    if (!P.les) return P.nu;
    float v = P.nu + eP;
    if (face_in(P, c.x, c.y, c.z, f)) {
        if (nb_fluid(m, f)) {
            v = P.nu + 0.5f * (eP + eQ);
        } else {
            v = P.nu + face_read(P, face, face_sign(f) > 0 ? c.i + face_off(P, f) : c.i, face_axis(f));
        }
    } else if (f == 3 && P.vbc[WF_FACE_Y0] == WF_BND_FIXED_VALUE) {
        v = P.nu + face_read(P, face, c.i, 1);
    }
    return v;
}
// 1/D of component a at cell i: from the cached reciprocals when given
// (computed with the same division), else divided here.
__device__ __forceinline__ float inv_d(const float* iD, const float* Dv, size_t N, int a, int i) {
    return iD ? ld(iD, a * N + i) : 1.f / ld(Dv, a * N + i);
}

// LogLawWallFunc, WallFunc.compute:77-123
__device__ float log_law(float uP, float dx, float nu, float den) {
    const float E = 9.8f, k = 0.41f;
    const float C = E * (dx / 2.0f) / nu;
    float eddyVis = 0.f;
    float uTau = 1.0f;
    uP = fabsf(uP);
    if (uP < 1e-5f) {
        uTau = 0.f;
    } else {
        for (int it = 0; it < 10; ++it) {
            const float lg = logf(C * uTau);
            const float f = __fsub_rn(__fmul_rn(uTau, lg), __fmul_rn(k, uP));
            const float df = lg + 1.0f;
            if (fabsf(df) < 1e-6f) break;
            uTau = uTau - f / df;
            if (uTau < 1e-5f) uTau = 1e-5f;
        }
        const float tauWall = uTau * uTau * den;
        const float strainRate = uP / (dx / 2.0f);
        eddyVis = tauWall / (strainRate * den) - nu;
        if (eddyVis < 0.f) eddyVis = 0.f;
    }
    return eddyVis;
}

__device__ __forceinline__ float hypot2(float a, float b) { return sqrtf(__fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b))); }

// Get{E,W,N,S,U,D}FaceVelLastTime, LES.compute:104-258
__device__ __forceinline__ void face_vel(const Params& P, const Bnd& B, const uint8_t* fl, const float* uT,
                                         int x, int y, int z, int f, float r[3]) {
    const int X = x + face_ox(f), Y = y + face_oy(f), Z = z + face_oz(f);
    const int i = cidx(P, x, y, z);
    r[0] = r[1] = r[2] = 0.f;
    if (in_region(P, X, Y, Z)) {
        const int q = cidx(P, X, Y, Z);
        if (fluid_at(fl, q)) {
#pragma unroll
            for (int k = 0; k < 3; ++k) r[k] = 0.5f * (ld(uT, (size_t)k * P.N + i) + ld(uT, (size_t)k * P.N + q));
        }
    } else {
        const int bc = face_bc(f), bt = P.vbc[bc];
        if (bt == WF_BND_FIXED_VALUE) {
#pragma unroll
            for (int k = 0; k < 3; ++k) r[k] = bnd_comp(P, B, bc, x, y, z, k);
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) r[k] = ld(uT, (size_t)k * P.N + i);
            if (bt == WF_BND_SYMMETRY) r[face_axis(f)] = 0.f;
        }
    }
}
// g[i][j] = d u_i / d x_j at a cell centre, LES.compute:296-306
__device__ __forceinline__ void cell_grad(const Params& P, const Bnd& B, const uint8_t* fl, const float* uT,
                                          int x, int y, int z, float g[3][3]) {
    float fv[6][3];
#pragma unroll
    for (int f = 0; f < 6; ++f) face_vel(P, B, fl, uT, x, y, z, f, fv[f]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) g[i][j] = (fv[2 * j][i] - fv[2 * j + 1][i]) * P.rdx;
}

// cell_grad from the neighbour mask and loaded values: uP = own velocity,
// uq[f] = velocity of the (clamped) neighbour across face f.  Same values.
__device__ __forceinline__ void cell_grad_v(const Params& P, const Bnd& B, unsigned m, const Cell& c,
                                            const float uP[3], const float uq[6][3], float g[3][3]) {
    float fv[6][3];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        fv[f][0] = fv[f][1] = fv[f][2] = 0.f;
        if (face_in(P, c.x, c.y, c.z, f)) {
            if (nb_fluid(m, f)) {
#pragma unroll
                for (int k = 0; k < 3; ++k) fv[f][k] = 0.5f * (uP[k] + uq[f][k]);
            }
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            if (bt == WF_BND_FIXED_VALUE) {
#pragma unroll
                for (int k = 0; k < 3; ++k) fv[f][k] = bnd_comp(P, B, bc, c.x, c.y, c.z, k);
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k) fv[f][k] = uP[k];
                if (bt == WF_BND_SYMMETRY) fv[f][face_axis(f)] = 0.f;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) g[i][j] = (fv[2 * j][i] - fv[2 * j + 1][i]) * P.rdx;
}

// ------------------------------------------------------------ wall function
// CSCalLogLawWallFunc, WallFunc.compute:128-190.  Writes the W/S/D face
// slots of every cell.
__global__ void k_wallfunc(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                           const float* __restrict__ uT, float* __restrict__ face) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    float fe0 = 0.f, fe1 = 0.f, fe2 = 0.f;
    const size_t N = P.N;
    auto u = [&](int i, int k) { return ld(uT, (size_t)k * N + i); };
    const bool me_fluid = fluid_at(fl, c.i);
    const bool w_in = c.x > 0, s_in = c.y > 0, d_in = c.z > 0;
    const int iw = c.i - 1, is = c.i - P.nx, id = c.i - P.nx * P.ny;
    if (me_fluid) {
        if (w_in && !fluid_at(fl, iw)) fe0 += log_law(hypot2(u(c.i, 1), u(c.i, 2)), P.dx, P.nu, P.den);
        if ((s_in && !fluid_at(fl, is)) || (!s_in && P.vbc[WF_FACE_Y0] == WF_BND_FIXED_VALUE))
            fe1 += log_law(hypot2(u(c.i, 0), u(c.i, 2)), P.dx, P.nu, P.den);
        if (d_in && !fluid_at(fl, id)) fe2 += log_law(hypot2(u(c.i, 0), u(c.i, 1)), P.dx, P.nu, P.den);
    } else {
        if (w_in && fluid_at(fl, iw)) fe0 += log_law(hypot2(u(iw, 1), u(iw, 2)), P.dx, P.nu, P.den);
        if (s_in && fluid_at(fl, is)) fe1 += log_law(hypot2(u(is, 0), u(is, 2)), P.dx, P.nu, P.den);
        if (d_in && fluid_at(fl, id)) fe2 += log_law(hypot2(u(id, 0), u(id, 1)), P.dx, P.nu, P.den);
    }
    face[c.i] = fe0;
    face[N + c.i] = fe1;
    face[2 * N + c.i] = fe2;
}

// ------------------------------------------------------------------- LES
// CSCalEddyVis, LES.compute:268-324
// When `grad` is given, the cell-centre gradient tensor is also stored (9
// planes, g[i][j] at plane 3i+j) for the LES term, which needs it at the cell
// and its six neighbours.
// `face` (nullable): also runs the wall function first (CSCalLogLawWallFunc,
// WallFunc.compute:128-190, the same values as k_wallfunc) from the
// velocities this kernel loads anyway: a fluid cell's own, a solid cell's
// W/S/D neighbours'.
__global__ void k_eddy_vis(const __grid_constant__ Params P, const Bnd B, const uint8_t* __restrict__ fl,
                           const float* __restrict__ uT, float* __restrict__ eddy, float* __restrict__ grad,
                           float* __restrict__ face) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    (void)fl;
    // Every load of the interior path before the fluid test.
    const unsigned m = __ldg(P.nbm + c.i);
    float uP[3], uq[6][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) uP[k] = ld(uT, (size_t)k * P.N + c.i);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int q = nb_idx(P, c.x, c.y, c.z, c.i, f);
#pragma unroll
        for (int k = 0; k < 3; ++k) uq[f][k] = ld(uT, (size_t)k * P.N + q);
    }
    if (face) {
        // faces W (1), S (3), D (5); a neighbour outside the domain counts as
        // not fluid only for the ground of a fixed-value Y0 (fluid cells)
        float fe0 = 0.f, fe1 = 0.f, fe2 = 0.f;
        const bool w_in = c.x > 0, s_in = c.y > 0, d_in = c.z > 0;
        if (m & 64u) {
            if (w_in && !nb_fluid(m, 1)) fe0 += log_law(hypot2(uP[1], uP[2]), P.dx, P.nu, P.den);
            if ((s_in && !nb_fluid(m, 3)) || (!s_in && P.vbc[WF_FACE_Y0] == WF_BND_FIXED_VALUE))
                fe1 += log_law(hypot2(uP[0], uP[2]), P.dx, P.nu, P.den);
            if (d_in && !nb_fluid(m, 5)) fe2 += log_law(hypot2(uP[0], uP[1]), P.dx, P.nu, P.den);
        } else {
            if (nb_fluid(m, 1)) fe0 += log_law(hypot2(uq[1][1], uq[1][2]), P.dx, P.nu, P.den);
            if (nb_fluid(m, 3)) fe1 += log_law(hypot2(uq[3][0], uq[3][2]), P.dx, P.nu, P.den);
            if (nb_fluid(m, 5)) fe2 += log_law(hypot2(uq[5][0], uq[5][1]), P.dx, P.nu, P.den);
        }
        face[c.i] = fe0;
        face[P.N + c.i] = fe1;
        face[2 * (size_t)P.N + c.i] = fe2;
    }
    if (!(m & 64u)) return;
    float g[3][3];
    cell_grad_v(P, B, m, c, uP, uq, g);
    if (grad) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) grad[(size_t)(3 * i + j) * P.N + c.i] = g[i][j];
    }
    const float Sxx = g[0][0], Syy = g[1][1], Szz = g[2][2];
    const float Sxy = 0.5f * (g[0][1] + g[1][0]);
    const float Syz = 0.5f * (g[1][2] + g[2][1]);
    const float Szx = 0.5f * (g[2][0] + g[0][2]);
    const float Sabs = sqrtf(2.0f * (Sxx * Sxx + Syy * Syy + Szz * Szz + 2.0f * Sxy * Sxy + 2.0f * Syz * Syz +
                                     2.0f * Szx * Szx));
    eddy[c.i] = (P.cs * P.cs) * (P.dx * P.dx) * Sabs;
}

// CSCalLesDeferCorrectTerm, LES.compute:327-687.  Output: the explicit LES
// term per momentum component (bField on the reference).
// Gradient tensor only (for the LES term when the eddy viscosity comes from
// elsewhere).
__global__ void k_cell_grad(const __grid_constant__ Params P, const Bnd B, const uint8_t* __restrict__ fl,
                            const float* __restrict__ uT, float* __restrict__ grad) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    if (!fluid_at(fl, c.i)) return;
    float g[3][3];
    cell_grad(P, B, fl, uT, c.x, c.y, c.z, g);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) grad[(size_t)(3 * i + j) * P.N + c.i] = g[i][j];
}

// `grad` (nullable) holds the stored gradient tensors of every fluid cell;
// without it they are recomputed (the reference recomputes them in place,
// LES.compute:381-616).
__global__ void k_les_term(const __grid_constant__ Params P, const Bnd B, const uint8_t* __restrict__ fl,
                           const float* __restrict__ uT, const float* __restrict__ eddy,
                           const float* __restrict__ face, const float* __restrict__ grad,
                           float* __restrict__ bles) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    const size_t N = P.N;
    // Every load of the interior path before the fluid test: the stored
    // gradient tensor of the cell, row a of each (clamped) neighbour's tensor
    // across an a-normal face, the velocity and the eddy viscosities.
    const unsigned m = __ldg(P.nbm + c.i);
    float g[3][3], gq[6][3], uP[3], eq[6];
    if (grad) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) g[i][j] = ld(grad, (size_t)(3 * i + j) * N + c.i);
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int q = nb_idx(P, c.x, c.y, c.z, c.i, f);
        const int a = face_axis(f);
#pragma unroll
        for (int j = 0; j < 3; ++j) gq[f][j] = grad ? ld(grad, (size_t)(3 * a + j) * N + q) : 0.f;
        eq[f] = P.les ? ld(eddy, q) : 0.f;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) uP[k] = ld(uT, (size_t)k * N + c.i);
    const float eP = P.les ? ld(eddy, c.i) : 0.f;
    if (!(m & 64u)) return;
    if (!grad) cell_grad(P, B, fl, uT, c.x, c.y, c.z, g);
    float fg[6][3];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        fg[f][0] = fg[f][1] = fg[f][2] = 0.f;
        const int a = face_axis(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (face_in(P, c.x, c.y, c.z, f)) {
            if (nb_fluid(m, f)) {
                if (grad) {
#pragma unroll
                    for (int j = 0; j < 3; ++j) fg[f][j] = 0.5f * (g[a][j] + gq[f][j]);
                } else {
                    float gn[3][3];
                    cell_grad(P, B, fl, uT, X, Y, Z, gn);
#pragma unroll
                    for (int j = 0; j < 3; ++j) fg[f][j] = 0.5f * (g[a][j] + gn[a][j]);
                }
            } else {
                const float v = uP[a] * (2.f * P.rdx);
                fg[f][a] = face_sign(f) > 0 ? -v : v;
            }
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            if (bt == WF_BND_FIXED_VALUE) {
                const float b = bnd_comp(P, B, bc, c.x, c.y, c.z, a);
                const float u = uP[a];
                fg[f][a] = face_sign(f) > 0 ? (b - u) * (2.f * P.rdx) : (u - b) * (2.f * P.rdx);
            } else {
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    if (j != a) fg[f][j] = g[a][j];
            }
        }
    }
    float vis[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) vis[f] = vis_face_v(P, m, face, c, f, eP, eq[f]);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const float t = vis[0] * fg[0][j] - vis[1] * fg[1][j] + vis[2] * fg[2][j] - vis[3] * fg[3][j] +
                        vis[4] * fg[4][j] - vis[5] * fg[5][j];
        bles[(size_t)j * N + c.i] = P.ds * t;
    }
}

// ------------------------------------------------------- momentum predictor
// CSVelPredictPreCompute, FvmColl.compute:1292-1859.  bles (may be null when
// LES is off) holds the LES term; D and b are written.  bles may alias b.
// A, iD (nullable): also stores the fast momentum sweeps' coefficients of
// this D, the values k_vel_coef computes: A_f = nu_f ds/dx -/+ ds (u_P +
// u_f)/4 on fluid-fluid faces (6 planes) and 1/D (3 planes), 0 on non-fluid
// cells; the expressions are k_vel_coef's.
__global__ void k_vel_precompute(const __grid_constant__ Params P, const Bnd B, const uint8_t* __restrict__ fl,
                                 const float* __restrict__ uT, const float* __restrict__ pr,
                                 const float* __restrict__ eddy, const float* __restrict__ face,
                                 const float* bles, const float* __restrict__ drag, float* __restrict__ Dv,
                                 float* bv, float* __restrict__ A, float* __restrict__ iD) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    (void)fl;
    const size_t N = P.N;
    // Every load of the interior path before the fluid test (boundary planes
    // and wall-face viscosities stay where they are used).
    const unsigned m = __ldg(P.nbm + c.i);
    float uP[3], uq[6], pq[6], eq[6], bl[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) uP[k] = ld(uT, k * N + c.i);
    const float pP = ld(pr, c.i);
    const float eP = P.les ? ld(eddy, c.i) : 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int q = nb_idx(P, c.x, c.y, c.z, c.i, f);
        uq[f] = ld(uT, face_axis(f) * N + q);
        pq[f] = ld(pr, q);
        eq[f] = P.les ? ld(eddy, q) : 0.f;
    }
    const bool add_les = P.les && bles;
#pragma unroll
    for (int k = 0; k < 3; ++k) bl[k] = add_les ? bles[k * N + c.i] : 0.f;
    const float dr = drag ? ld(drag, c.i) : 0.f;
    if (!(m & 64u)) {
        if (A) {
#pragma unroll
            for (int f = 0; f < 6; ++f) A[f * N + c.i] = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) iD[k * N + c.i] = 0.f;
        }
        return;
    }
    const float dvdt = P.dv / P.dt;
    float D[3] = {dvdt, dvdt, dvdt};
    float b[3] = {0.f, 0.f, 0.f};
    // advection, :1314-1482
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        if (face_in(P, c.x, c.y, c.z, f)) {
            if (nb_fluid(m, f)) {
                const float t = P.ds * 0.25f * (uP[a] + uq[f]);
#pragma unroll
                for (int k = 0; k < 3; ++k) D[k] = face_sign(f) > 0 ? D[k] + t : D[k] - t;
            }
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            if (bt == WF_BND_FIXED_VALUE) {
                const float ba = bnd_comp(P, B, bc, c.x, c.y, c.z, a);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float t = P.ds * bnd_comp(P, B, bc, c.x, c.y, c.z, k) * ba;
                    b[k] = face_sign(f) > 0 ? b[k] - t : b[k] + t;
                }
            } else if (bt == WF_BND_ZERO_GRAD) {
                const float t = P.ds * uP[a];
#pragma unroll
                for (int k = 0; k < 3; ++k) D[k] = face_sign(f) > 0 ? D[k] + t : D[k] - t;
            }
        }
    }
    // pressure, :1484-1591
    float pf[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (face_in(P, c.x, c.y, c.z, f)) {
            pf[f] = nb_fluid(m, f) ? 0.5f * (pP + pq[f]) : pP;
        } else {
            pf[f] = P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE ? 0.f : pP;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) b[a] += -P.rden * P.ds * (pf[2 * a] - pf[2 * a + 1]);
    // diffusion, :1593-1836
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const float vis = vis_face_v(P, m, face, c, f, eP, eq[f]);
        if (face_in(P, c.x, c.y, c.z, f)) {
            const float t = nb_fluid(m, f) ? vis * P.ds * P.rdx : 2.f * vis * P.ds * P.rdx;
#pragma unroll
            for (int k = 0; k < 3; ++k) D[k] += t;
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            const float t = 2.f * vis * P.ds * P.rdx;
            if (bt == WF_BND_FIXED_VALUE) {
#pragma unroll
                for (int k = 0; k < 3; ++k) b[k] += t * bnd_comp(P, B, bc, c.x, c.y, c.z, k);
#pragma unroll
                for (int k = 0; k < 3; ++k) D[k] += t;
            } else if (bt == WF_BND_SYMMETRY) {
                D[face_axis(f)] += t;
            }
        }
    }
    // time, force, LES, :1838-1854
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] += dvdt * uP[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] += P.dv * P.force[k];
    if (add_les) {
#pragma unroll
        for (int k = 0; k < 3; ++k) b[k] += bl[k];
    }
    // Brinkman drag of a soft obstacle mask (no reference counterpart)
    if (drag) {
        const float t = P.dv * dr;
#pragma unroll
        for (int k = 0; k < 3; ++k) D[k] += t;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Dv[k * N + c.i] = D[k];
        bv[k * N + c.i] = b[k];
    }
    if (A) {
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            float cf = 0.f;
            if (nb_fluid(m, f)) {
                const float conv = P.ds * 0.25f * (uP[face_axis(f)] + uq[f]);
                const float vis = P.les ? P.nu + 0.5f * (eP + eq[f]) : P.nu;
                const float dif = vis * P.ds * P.rdx;
                cf = face_sign(f) > 0 ? dif - conv : dif + conv;
            }
            A[f * N + c.i] = cf;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) iD[k * N + c.i] = 1.0f / D[k];
    }
}

// CSVelPredict, FvmColl.compute:1863-2069.  uI == nullptr is not allowed
// here (the sweep always reads a previous iterate).
__global__ void k_vel_sweep(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                            const float* __restrict__ uI, const float* __restrict__ uT,
                            const float* __restrict__ eddy, const float* __restrict__ face,
                            const float* __restrict__ Dv, const float* __restrict__ bv, float* __restrict__ uo) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    if (!fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    float adv[3] = {0.f, 0.f, 0.f}, dif[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (!in_region(P, X, Y, Z)) continue;
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float sum = ld(uT, a * N + c.i) + ld(uT, a * N + q);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float t = P.ds * 0.25f * ld(uI, k * N + q) * sum;
            adv[k] = face_sign(f) > 0 ? adv[k] - t : adv[k] + t;
        }
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (!in_region(P, X, Y, Z)) continue;
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float vis = vis_face(P, fl, eddy, face, c, f);
#pragma unroll
        for (int k = 0; k < 3; ++k) dif[k] += vis * P.ds * P.rdx * ld(uI, k * N + q);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) uo[k * N + c.i] = 1.0f / ld(Dv, k * N + c.i) * (adv[k] + dif[k] + ld(bv, k * N + c.i));
}

// ----------------------------------------------------- pressure correction
// CSPresCorrectRhieChowPreCompute, FvmColl.compute:2481-2787.  iD
// (nullable): cached 1/D of the same D.
// c3 (nullable): also stores the pressure sweeps' face coefficients c_E,
// c_N, c_U (three planes; (dv/den) DInv / dx on fluid-fluid faces, else 0),
// the values k_pres_coef computes from the same D, as the same products.
__global__ void k_pres_precompute(const __grid_constant__ Params P, const Bnd B, const uint8_t* __restrict__ fl,
                                  const float* __restrict__ u, const float* __restrict__ pr,
                                  const float* __restrict__ Dv, const float* __restrict__ iD,
                                  float* __restrict__ Dp, float* __restrict__ bp, float* __restrict__ c3) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    (void)fl;
    const size_t N = P.N;
    // Every load of the interior path before the fluid test: per face the
    // neighbour's mask, 1/D and velocity, and the pressures at distance 1 and
    // 2 along each axis (indices clamped in-domain; a clamped value is never
    // used, since the mask bits that select it are then 0).
    const unsigned m = __ldg(P.nbm + c.i);
    const float pP = ld(pr, c.i);
    float uP[3], dP[3], uq[6], dq[6], pq[6], pq2[6];
    unsigned mq[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        uP[a] = ld(u, a * N + c.i);
        dP[a] = inv_d(iD, Dv, N, a, c.i);
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const int q = nb_idx(P, c.x, c.y, c.z, c.i, f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        const int q2 = in_region(P, X, Y, Z) ? nb_idx(P, X, Y, Z, q, f) : q;
        mq[f] = __ldg(P.nbm + q);
        dq[f] = inv_d(iD, Dv, N, a, q);
        uq[f] = ld(u, a * N + q);
        pq[f] = ld(pr, q);
        pq2[f] = ld(pr, q2);
    }
    if (!(m & 64u)) {
        if (c3) {
#pragma unroll
            for (int a = 0; a < 3; ++a) c3[a * N + c.i] = 0.f;
        }
        return;
    }
    float DP = 0.f, bP = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f), s = face_sign(f);
        if (face_in(P, c.x, c.y, c.z, f)) {
            if (!nb_fluid(m, f)) {
                if (c3 && s > 0) c3[a * N + c.i] = 0.f;
                continue;
            }
            const float DInv = 0.5f * (dP[a] + dq[f]);
            DP -= P.dvden * DInv * P.rdx;
            if (c3 && s > 0) c3[a * N + c.i] = __fmul_rn(__fmul_rn(P.dvden, DInv), P.rdx);
            const float fl_ = 0.5f * (uP[a] + uq[f]);
            bP = s > 0 ? bP + fl_ : bP - fl_;
            // Rhie-Chow over the face between low cell L and high cell H: the
            // cell beyond Q (q + off(f)) and the cell behind P (i - off(f))
            const bool beyondQ = nb_fluid(mq[f], f), behindP = nb_fluid(m, f ^ 1);
            const bool hh = s > 0 ? beyondQ : behindP;
            const bool ll = s > 0 ? behindP : beyondQ;
            const float pL = s > 0 ? pP : pq[f], pH = s > 0 ? pq[f] : pP;
            const float pHH = s > 0 ? pq2[f] : pq[f ^ 1], pLL = s > 0 ? pq[f ^ 1] : pq2[f];
            const float presGrad = (pH - pL) * P.rdx;
            float ave = presGrad;
            if (hh || ll) {
                const float gH = hh ? (pHH - pL) * P.rdx2 : (pH - pL) * P.rdx2;
                const float gL = ll ? (pH - pLL) * P.rdx2 : (pH - pL) * P.rdx2;
                ave = 0.5f * (gH + gL);
            }
            const float vct = -(P.dv * DInv) * P.rden * (presGrad - ave);
            bP = s > 0 ? bP + vct : bP - vct;
        } else {
            if (c3 && s > 0) c3[a * N + c.i] = 0.f;
            const int bc = face_bc(f), vb = P.vbc[bc];
            if (vb == WF_BND_FIXED_VALUE) {
                const float t = bnd_comp(P, B, bc, c.x, c.y, c.z, a);
                bP = s > 0 ? bP + t : bP - t;
            } else if (vb == WF_BND_ZERO_GRAD) {
                const float t = uP[a];
                bP = s > 0 ? bP + t : bP - t;
            }
            if (P.pbc[bc] == WF_BND_FIXED_VALUE) DP -= 2.f * P.dvden * dP[a] * P.rdx;
        }
    }
    Dp[c.i] = DP;
    bp[c.i] = bP;
}

// CSPresCorrectRhieChow, FvmColl.compute:2790-2848.  pin == nullptr reads as
// an all-zero previous iterate.
__global__ void k_pres_sweep(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                             const float* __restrict__ pin, const float* __restrict__ Dv,
                             const float* __restrict__ Dp, const float* __restrict__ bp, float* __restrict__ pout) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    if (!fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    float t = 0.f;
    if (pin) {
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const int a = face_axis(f);
            const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
            if (!in_region(P, X, Y, Z)) continue;
            const int q = cidx(P, X, Y, Z);
            if (!fluid_at(fl, q)) continue;
            const float DInv = 0.5f * (1.f / ld(Dv, a * N + c.i) + 1.f / ld(Dv, a * N + q));
            t -= P.dvden * DInv * P.rdx * ld(pin, q);
        }
    }
    pout[c.i] = (1.f / ld(Dp, c.i)) * (t + ld(bp, c.i));
}

// CSApplyPresCorrection, FvmColl.compute:2851-2862 (non-solid cells) and
// CSPisoApplyPresCorrection, PisoColl.compute:259-267 (fluid cells).  With
// flags restricted to {fluid, solid} both select the fluid cells.
__global__ void k_apply_pres(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                             const float* __restrict__ pc, float* __restrict__ pr) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    if (__ldg(fl + c.i) == WF_CELL_SOLID) return;
    pr[c.i] += pc ? ld(pc, c.i) : 0.f;
}

// k_apply_pres on four consecutive cells per thread, every load issued before
// the solid test; solid cells are stored back unchanged.  n4 = N / 4.
__global__ void k_apply_pres4(int n4, const uint8_t* __restrict__ fl, const float* __restrict__ pc,
                              float* __restrict__ pr) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n4) return;
    const uchar4 f = __ldg(reinterpret_cast<const uchar4*>(fl) + q);
    const float4 c = pc ? __ldg(reinterpret_cast<const float4*>(pc) + q) : make_float4(0.f, 0.f, 0.f, 0.f);
    float4 p = reinterpret_cast<const float4*>(pr)[q];
    if (f.x != WF_CELL_SOLID) p.x += c.x;
    if (f.y != WF_CELL_SOLID) p.y += c.y;
    if (f.z != WF_CELL_SOLID) p.z += c.z;
    if (f.w != WF_CELL_SOLID) p.w += c.w;
    reinterpret_cast<float4*>(pr)[q] = p;
}

// CSPresNormalization, FvmColl.compute:2865-2880, split in two launches so
// the reference value is read before any cell is updated.
__global__ void k_norm_read(const __grid_constant__ Params P, const float* __restrict__ pr, float* __restrict__ ref) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *ref = pr[cidx(P, 2, P.ny / 2, 2)];
}
__global__ void k_norm_apply(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                             const float* __restrict__ ref, float* __restrict__ pr) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    if (__ldg(fl + c.i) == WF_CELL_SOLID) return;
    pr[c.i] -= __ldg(ref);
}

// CSApplyVelCorrectionDivergenceTheorem, FvmColl.compute:2951-3121.
// pc == nullptr reads as zero; iD (nullable): cached 1/D of the same D.
// pr (nullable): also applies the pressure correction p += p' on the fluid
// cells (CSApplyPresCorrection, :2851-2862, the same addition), so the step
// needs no separate pass over p.
__global__ void k_apply_vel(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                            const float* __restrict__ pc, const float* __restrict__ Dv,
                            const float* __restrict__ iD, float* __restrict__ uc, float* __restrict__ u,
                            float* __restrict__ pr) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    (void)fl;
    const size_t N = P.N;
    // Every load before the fluid test (one wait on memory per thread).
    const unsigned m = __ldg(P.nbm + c.i);
    const float pP = pc ? ld(pc, c.i) : 0.f;
    float pn[6], di[3], uo[3];
#pragma unroll
    for (int f = 0; f < 6; ++f) pn[f] = pc ? ld(pc, nb_idx(P, c.x, c.y, c.z, c.i, f)) : 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        di[a] = inv_d(iD, Dv, N, a, c.i);
        uo[a] = ld(u, a * N + c.i);
    }
    if (!(m & 64u)) return;
    if (pr) pr[c.i] += pP;
    float pf[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (face_in(P, c.x, c.y, c.z, f)) {
            pf[f] = nb_fluid(m, f) ? 0.5f * (pP + pn[f]) : pP;
        } else {
            pf[f] = P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE ? 0.f : pP;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float corr = -P.dvden * di[a] * (pf[2 * a] - pf[2 * a + 1]) * P.rdx;
        uc[a * N + c.i] = corr;
        u[a * N + c.i] = uo[a] + corr;
    }
}

// ------------------------------------------------------------------ PISO
// CSPisoCalAodUCorrect, PisoColl.compute:71-178.  The advection and
// diffusion sums run over the faces in the reference's order, in one loop
// (each with its own accumulator, so the values are those of two loops).
__global__ void k_piso_aodu(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                            const float* __restrict__ uc, const float* __restrict__ uT,
                            const float* __restrict__ eddy, const float* __restrict__ face,
                            float* __restrict__ aodu) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    (void)fl;
    const size_t N = P.N;
    // Every load of the ordinary path before the fluid test.
    const unsigned m = __ldg(P.nbm + c.i);
    float uTP[3], uTq[6], ucq[6][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) uTP[a] = ld(uT, a * N + c.i);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int q = nb_idx(P, c.x, c.y, c.z, c.i, f);
        uTq[f] = ld(uT, face_axis(f) * N + q);
#pragma unroll
        for (int k = 0; k < 3; ++k) ucq[f][k] = ld(uc, k * N + q);
    }
    if (!(m & 64u)) return;
    const bool consistent = (P.compat & WF_COMPAT_PISO_CONSISTENT) != 0;
    float adv[3] = {0.f, 0.f, 0.f}, dif[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!nb_fluid(m, f)) continue;
        const float sum = uTP[face_axis(f)] + uTq[f];
        const float vis = consistent ? vis_face_m(P, m, eddy, face, c, f) : P.nu;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float uq = ucq[f][k];
            const float t = P.ds * 0.25f * uq * sum;
            adv[k] = face_sign(f) > 0 ? adv[k] + t : adv[k] - t;
            dif[k] -= vis * P.ds * P.rdx * uq;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) aodu[k * N + c.i] = adv[k] + dif[k];
}

// CSPisoPresCorrection, PisoColl.compute:181-256.  pin == nullptr reads as 0.
__global__ void k_piso_pres_sweep(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                                  const float* __restrict__ pin, const float* __restrict__ Dv,
                                  const float* __restrict__ aodu, float* __restrict__ pout) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    if (!fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const bool consistent = (P.compat & WF_COMPAT_PISO_CONSISTENT) != 0;
    float coeff = 0.f, pt = 0.f, vt = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (!in_region(P, X, Y, Z)) {
            if (consistent && P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE) {
                const float DInv = 1.f / ld(Dv, a * N + c.i);
                coeff -= 2.f * P.dvden * DInv * P.rdx;
            }
            continue;
        }
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float AdInv = 0.5f * (1.f / ld(Dv, a * N + c.i) + 1.f / ld(Dv, a * N + q));
        const float Aod = 0.5f * (ld(aodu, a * N + c.i) + ld(aodu, a * N + q));
        const float pq = pin ? ld(pin, q) : 0.f;
        if (a == 0) {
            coeff -= P.dvden * (AdInv * P.rdx);
            pt -= P.dvden * (AdInv * P.rdx) * pq;
        } else {
            coeff -= P.dvden * AdInv * P.rdx;
            pt -= P.dvden * AdInv * P.rdx * pq;
        }
        vt = face_sign(f) > 0 ? vt - AdInv * Aod : vt + AdInv * Aod;
    }
    pout[c.i] = (1.f / coeff) * (pt + vt);
}

// CSPisoVelCorrection, PisoColl.compute:270-337.  iD (nullable): cached
// 1/D of the same D.
// pr (nullable): also applies p += p'' on the fluid cells
// (CSPisoApplyPresCorrection, PisoColl.compute:259-267, the same addition).
__global__ void k_piso_vel(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                           const float* __restrict__ pc, const float* __restrict__ Dv,
                           const float* __restrict__ iD, const float* __restrict__ aodu, float* __restrict__ uc,
                           float* __restrict__ u, float* __restrict__ pr) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    (void)fl;
    const size_t N = P.N;
    // Every load before the fluid test.
    const unsigned m = __ldg(P.nbm + c.i);
    const float pP = ld(pc, c.i);
    float pn[6], di[3], ao[3], uo[3];
#pragma unroll
    for (int f = 0; f < 6; ++f) pn[f] = ld(pc, nb_idx(P, c.x, c.y, c.z, c.i, f));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        di[a] = inv_d(iD, Dv, N, a, c.i);
        ao[a] = ld(aodu, a * N + c.i);
        uo[a] = ld(u, a * N + c.i);
    }
    if (!(m & 64u)) return;
    if (pr) pr[c.i] += pP;
    float pf[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) pf[f] = nb_fluid(m, f) ? 0.5f * (pP + pn[f]) : pP;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float grad = (pf[2 * a] - pf[2 * a + 1]) * P.rdx;
        const float corr = -di[a] * (ao[a] + P.dvden * grad);
        uc[a * N + c.i] = corr;
        u[a * N + c.i] = uo[a] + corr;
    }
}

// --------------------------------------------------------------- residuals
// Block partial sums of squared residuals (FvmColl.compute:3124-3199): warp
// shuffles, then one value per block; a second pass adds the partials in
// block order, so the result is deterministic.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int lane = tid & 31, warp = tid >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    double r = 0.0;
    if (warp == 0) {
        r = lane < nw ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}
__device__ __forceinline__ int block_linear() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ bool block_leader() { return threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0; }

__global__ void k_vel_residual(const __grid_constant__ Params P, const float* __restrict__ Dv,
                               const float* __restrict__ u, const float* __restrict__ uI, double* __restrict__ part) {
    Cell c;
    double s = 0.0;
    if (cell_of_thread(P, c)) {
        const size_t N = P.N;
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float l = ld(Dv, k * N + c.i) * (ld(u, k * N + c.i) - ld(uI, k * N + c.i));
            acc += l * l;
        }
        s = acc;
    }
    s = block_sum(s);
    if (block_leader()) part[block_linear()] = s;
}
__global__ void k_pres_residual(const __grid_constant__ Params P, const float* __restrict__ Dp,
                                const float* __restrict__ pc, const float* __restrict__ pcL,
                                double* __restrict__ part) {
    Cell c;
    double s = 0.0;
    if (cell_of_thread(P, c)) {
        const float a = pc ? ld(pc, c.i) : 0.f, b = pcL ? ld(pcL, c.i) : 0.f;
        const float l = ld(Dp, c.i) * (a - b);
        s = l * l;
    }
    s = block_sum(s);
    if (block_leader()) part[block_linear()] = s;
}
__global__ void k_sum_partials(const double* __restrict__ part, int n, double* __restrict__ out) {
    __shared__ double sh[1024];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// Sum over fluid cells of |net face flux| of u (BC-aware, no Rhie-Chow).
__global__ void k_mass_imbalance(const __grid_constant__ Params P, const Bnd B, const uint8_t* __restrict__ fl,
                                 const float* __restrict__ u, double* __restrict__ part) {
    Cell c;
    double s = 0.0;
    if (cell_of_thread(P, c) && fluid_at(fl, c.i)) {
        const size_t N = P.N;
        double div = 0.0;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const int a = face_axis(f);
            const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
            double uf = 0.0;
            if (in_region(P, X, Y, Z)) {
                const int q = cidx(P, X, Y, Z);
                if (fluid_at(fl, q)) uf = 0.5 * ((double)ld(u, a * N + c.i) + (double)ld(u, a * N + q));
            } else {
                const int bc = face_bc(f), vb = P.vbc[bc];
                if (vb == WF_BND_FIXED_VALUE) uf = bnd_comp(P, B, bc, c.x, c.y, c.z, a);
                else if (vb == WF_BND_ZERO_GRAD) uf = ld(u, a * N + c.i);
            }
            div += face_sign(f) * uf;
        }
        s = fabs(div) * (double)P.ds;
    }
    s = block_sum(s);
    if (block_leader()) part[block_linear()] = s;
}

// Non-finite scan: sets *bad = 1 when any value is NaN/Inf.
__global__ void k_check_finite(const float* __restrict__ a, long long n, int* __restrict__ bad) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int b = 0;
    for (; i < n; i += stride) b |= !isfinite(__ldg(a + i));
    if (__syncthreads_or(b) && threadIdx.x == 0) atomicOr(bad, 1);
}

// ------------------------------------------------------------------ set-up
// CSInitVelPresFields / CSInitLogVelPresFields, InitShaderColl.compute:95-132:
// every cell of the three velocity buffers gets the profile, velCorrect and
// pressures are zeroed.  fric_vel <= 0 selects the constant profile.
__global__ void k_init_fields(const __grid_constant__ Params P, int logp, float wind, float fric, float kappa,
                              float z0, int centre, float* u0, float* u1, float* u2, float* uc, float* pr) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    const size_t N = P.N;
    float vx = wind;
    if (logp) {
        const float yPhys = centre ? ((float)c.y + 0.5f) * P.dx : (float)c.y * P.dx;
        vx = fric / kappa * logf((yPhys + z0) / z0);
    }
    float* bufs[3] = {u0, u1, u2};
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        if (!bufs[b]) continue;
        bufs[b][c.i] = vx;
        bufs[b][N + c.i] = 0.f;
        bufs[b][2 * N + c.i] = 0.f;
    }
    uc[c.i] = 0.f;
    uc[N + c.i] = 0.f;
    uc[2 * N + c.i] = 0.f;
    pr[c.i] = 0.f;
}

// CSInitModelFlag, InitShaderColl.compute:346-364
__global__ void k_init_flags(const __grid_constant__ Params P, const int32_t* __restrict__ src,
                             uint8_t* __restrict__ fl, float* u0, float* u1, float* u2) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    const size_t N = P.N;
    if ((double)src[c.i] > 0.5) {
        fl[c.i] = WF_CELL_SOLID;
        float* bufs[3] = {u0, u1, u2};
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            if (!bufs[b]) continue;
            bufs[b][c.i] = 0.f;
            bufs[b][N + c.i] = 0.f;
            bufs[b][2 * N + c.i] = 0.f;
        }
    } else {
        fl[c.i] = WF_CELL_FLUID;
    }
}

// CSSetLogVelBndCond, InitShaderColl.compute:273-285 (X0 plane, ny*nz points)
__global__ void k_set_log_inlet(int ny, int nz, float dx, float fric, float kappa, float z0, float* x0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = ny * nz;
    if (i >= n) return;
    const int y = i % ny;
    const float yPhys = ((float)y + 0.5f) * dx;
    x0[i] = fric / kappa * logf((yPhys + z0) / z0);
    x0[n + i] = 0.f;
    x0[2 * n + i] = 0.f;
}
__global__ void k_fill3(float* a, int n, float v0, float v1, float v2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = v0;
    a[n + i] = v1;
    a[2 * n + i] = v2;
}

// Layout conversion for host I/O.
__global__ void k_soa_to_xyzw(const float* __restrict__ s, int n, float* __restrict__ d, int w4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (w4) {
        reinterpret_cast<float4*>(d)[i] = make_float4(s[i], s[n + i], s[2 * (size_t)n + i], 0.f);
    } else {
        d[3 * (size_t)i] = s[i];
        d[3 * (size_t)i + 1] = s[n + i];
        d[3 * (size_t)i + 2] = s[2 * (size_t)n + i];
    }
}
__global__ void k_flags_to_i32(const uint8_t* __restrict__ f, int n, int32_t* __restrict__ o) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = f[i];
}
// Neighbour mask (Params::nbm) of every cell from the flags.
__global__ void k_nbmask(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                         uint8_t* __restrict__ nbm) {
    Cell c;
    if (!cell_of_thread(P, c)) return;
    unsigned m = fluid_at(fl, c.i) ? 64u : 0u;
#pragma unroll
    for (int f = 0; f < 6; ++f)
        if (face_in(P, c.x, c.y, c.z, f) && fluid_at(fl, c.i + face_off(P, f))) m |= 1u << f;
    nbm[c.i] = (uint8_t)m;
}

}  // namespace

// ----------------------------------------------------------------- launchers
thread_local long long g_launches = 0;

static dim3 cell_block() { return dim3(32, 4, 2); }
static dim3 cell_grid(const Params& P) {
    dim3 b = cell_block();
    return dim3((P.nx + b.x - 1) / b.x, (P.ny + b.y - 1) / b.y, (P.nz + b.z - 1) / b.z);
}
int cell_grid_blocks(const Params& P) {
    dim3 g = cell_grid(P);
    return (int)(g.x * g.y * g.z);
}

#define WF_LAUNCH(kernel, ...) \
    (WF_COUNT_LAUNCH(), kernel<<<cell_grid(P), cell_block(), 0, st>>>(P, __VA_ARGS__))

void launch_wallfunc(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uT, float* face) {
    WF_LAUNCH(k_wallfunc, fl, uT, face);
}
void launch_eddy_vis(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT, float* eddy,
                     float* grad, float* face) {
    WF_LAUNCH(k_eddy_vis, B, fl, uT, eddy, grad, face);
}
void launch_cell_grad(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT,
                      float* grad) {
    WF_LAUNCH(k_cell_grad, B, fl, uT, grad);
}
void launch_les_term(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT,
                     const float* eddy, const float* face, const float* grad, float* bles) {
    WF_LAUNCH(k_les_term, B, fl, uT, eddy, face, grad, bles);
}
void launch_vel_precompute(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* uT,
                           const float* pr, const float* eddy, const float* face, const float* bles,
                           const float* drag, float* Dv, float* bv, float* A, float* iD) {
    WF_LAUNCH(k_vel_precompute, B, fl, uT, pr, eddy, face, bles, drag, Dv, bv, A, iD);
}
void launch_vel_sweep(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uI, const float* uT,
                      const float* eddy, const float* face, const float* Dv, const float* bv, float* uo) {
    WF_LAUNCH(k_vel_sweep, fl, uI, uT, eddy, face, Dv, bv, uo);
}
void launch_pres_precompute(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* u,
                            const float* pr, const float* Dv, const float* iD, float* Dp, float* bp, float* c3) {
    WF_LAUNCH(k_pres_precompute, B, fl, u, pr, Dv, iD, Dp, bp, c3);
}
void launch_pres_sweep(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pin, const float* Dv,
                       const float* Dp, const float* bp, float* pout) {
    WF_LAUNCH(k_pres_sweep, fl, pin, Dv, Dp, bp, pout);
}
void launch_apply_pres(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pc, float* pr) {
    if (quad_ok(P, {fl, pc, pr})) {
        WF_COUNT_LAUNCH();
        const int n4 = P.N / 4;
        k_apply_pres4<<<(n4 + 255) / 256, 256, 0, st>>>(n4, fl, pc, pr);
        return;
    }
    WF_LAUNCH(k_apply_pres, fl, pc, pr);
}
void launch_normalize(const Params& P, cudaStream_t st, const uint8_t* fl, float* pr, float* ref) {
    WF_COUNT_LAUNCH();
    k_norm_read<<<1, 32, 0, st>>>(P, pr, ref);
    WF_LAUNCH(k_norm_apply, fl, ref, pr);
}
void launch_apply_vel(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pc, const float* Dv,
                      const float* iD, float* uc, float* u, float* pr) {
    WF_LAUNCH(k_apply_vel, fl, pc, Dv, iD, uc, u, pr);
}
void launch_piso_aodu(const Params& P, cudaStream_t st, const uint8_t* fl, const float* uc, const float* uT,
                      const float* eddy, const float* face, float* aodu) {
    WF_LAUNCH(k_piso_aodu, fl, uc, uT, eddy, face, aodu);
}
void launch_piso_pres_sweep(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pin, const float* Dv,
                            const float* aodu, float* pout) {
    WF_LAUNCH(k_piso_pres_sweep, fl, pin, Dv, aodu, pout);
}
void launch_piso_vel(const Params& P, cudaStream_t st, const uint8_t* fl, const float* pc, const float* Dv,
                     const float* iD, const float* aodu, float* uc, float* u, float* pr) {
    WF_LAUNCH(k_piso_vel, fl, pc, Dv, iD, aodu, uc, u, pr);
}
void launch_nbmask(const Params& P, cudaStream_t st, const uint8_t* fl, uint8_t* nbm) {
    WF_LAUNCH(k_nbmask, fl, nbm);
}
void launch_vel_residual(const Params& P, cudaStream_t st, const float* Dv, const float* u, const float* uI,
                         double* part, double* out) {
    WF_LAUNCH(k_vel_residual, Dv, u, uI, part);
    WF_COUNT_LAUNCH();
    k_sum_partials<<<1, 1024, 0, st>>>(part, cell_grid_blocks(P), out);
}
void launch_pres_residual(const Params& P, cudaStream_t st, const float* Dp, const float* pc, const float* pcL,
                          double* part, double* out) {
    WF_LAUNCH(k_pres_residual, Dp, pc, pcL, part);
    WF_COUNT_LAUNCH();
    k_sum_partials<<<1, 1024, 0, st>>>(part, cell_grid_blocks(P), out);
}
void launch_mass_imbalance(const Params& P, const Bnd& B, cudaStream_t st, const uint8_t* fl, const float* u,
                           double* part, double* out) {
    WF_LAUNCH(k_mass_imbalance, B, fl, u, part);
    WF_COUNT_LAUNCH();
    k_sum_partials<<<1, 1024, 0, st>>>(part, cell_grid_blocks(P), out);
}
void launch_check_finite(cudaStream_t st, const float* a, long long n, int* bad) {
    int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    if (blocks < 1) blocks = 1;
    k_check_finite<<<blocks, 256, 0, st>>>(a, n, bad);
}
void launch_init_fields(const Params& P, cudaStream_t st, int logp, float wind, float fric, float kappa, float z0,
                        int centre, float* u0, float* u1, float* u2, float* uc, float* pr) {
    WF_LAUNCH(k_init_fields, logp, wind, fric, kappa, z0, centre, u0, u1, u2, uc, pr);
}
void launch_init_flags(const Params& P, cudaStream_t st, const int32_t* src, uint8_t* fl, float* u0, float* u1,
                       float* u2) {
    WF_LAUNCH(k_init_flags, src, fl, u0, u1, u2);
}
void launch_set_log_inlet(const Params& P, cudaStream_t st, float fric, float kappa, float z0, float* x0) {
    const int n = P.ny * P.nz;
    k_set_log_inlet<<<(n + 255) / 256, 256, 0, st>>>(P.ny, P.nz, P.dx, fric, kappa, z0, x0);
}
void launch_fill3(cudaStream_t st, float* a, int n, float v0, float v1, float v2) {
    k_fill3<<<(n + 255) / 256, 256, 0, st>>>(a, n, v0, v1, v2);
}
void launch_soa_to_interleaved(cudaStream_t st, const float* s, int n, float* d, int w4) {
    k_soa_to_xyzw<<<(n + 255) / 256, 256, 0, st>>>(s, n, d, w4);
}
void launch_flags_to_i32(cudaStream_t st, const uint8_t* f, int n, int32_t* o) {
    k_flags_to_i32<<<(n + 255) / 256, 256, 0, st>>>(f, n, o);
}

}  // namespace wf
