// wf_adjoint.cu - discrete adjoint of the fixed-iteration SIMPLE/PISO step.
//
// No counterpart in the reference (it has no derivatives).  The forward step
// (wf_api.cu sequencing of FvmSolverGpu.Step, LES off) is a fixed
// composition of maps; its vector-Jacobian product is the same composition
// reversed:
//
//   (D, b)   = PRE(u0, p0, g)           momentum diagonal / right-hand side
//   (A, 1/D) = VCOEF(u0, D)             Picard coefficients of the sweep
//   u^{k+1}  = 1/D (A u^k + b)          nV sweeps, u^0 = u0        -> u*
//   (Dp, bp) = PPRE(u*, p0, D, g)       Rhie-Chow face-flux assembly
//   c, 1/Dp  = PCOEF(D), 1/Dp           face coefficients
//   q^{k+1}  = 1/Dp (bp - C q^k)        nP sweeps, q^0 = 0         -> q
//   p1 = p0 + q,  c1 = CORR(q, D),  u1 = u* + c1
//   per PISO corrector m: a = AOD(c_m, u0); (1/coef, r) = PISOPRE(D, a);
//   s^{k+1} = 1/coef (r - C s^k), nP sweeps; p += s; c_{m+1} = PVEL(s, D, a);
//   u += c_{m+1}
//
// Linear sweeps reverse as transposed gathers (each cell collects from its
// neighbours, no atomics); the once-per-step maps scatter their local
// derivatives with atomicAdd.  The forward step is re-run from its input
// state with every Jacobi iterate kept (the "tape"), using the one-sweep
// kernels of wf_sweeps.cu.
//
// Supported: turbulence off, binary obstacle mask, any boundary set,
// SIMPLE or PISO, no compat flags that change the PISO corrector.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>
#include <vector>

#include "wf_kernels.cuh"
#include "wf_solver.cuh"
#include "wf_sweeps.cuh"

struct wf_adjoint;

namespace {
// Wait status of the TMA-staged pressure passes, or nullptr where the
// handle runs the per-thread-staged kernel (WF_TMA=0).
int* tma_status(const wf_solver* h) { return h->pres_tma ? h->dstat : nullptr; }
}  // namespace

namespace wf {
namespace {

__device__ __forceinline__ float ld(const float* p, size_t i) { return __ldg(p + i); }
__device__ __forceinline__ bool fluid_at(const uint8_t* fl, int i) { return __ldg(fl + i) == WF_CELL_FLUID; }
__device__ __forceinline__ void aadd(float* p, float v) {
    if (v != 0.f) atomicAdd(p, v);
}

struct Cell {
    int x, y, z, i;
};
__device__ __forceinline__ bool thread_cell(const Params& P, Cell& c) {
    c.x = blockIdx.x * blockDim.x + threadIdx.x;
    c.y = blockIdx.y * blockDim.y + threadIdx.y;
    c.z = blockIdx.z * blockDim.z + threadIdx.z;
    if (c.x >= P.nx || c.y >= P.ny || c.z >= P.nz) return false;
    c.i = cidx(P, c.x, c.y, c.z);
    return true;
}

// Mutable boundary planes for the adjoint of the boundary values.
struct BndBar {
    float* p[6];
};
__device__ __forceinline__ float* bnd_bar(const Params& P, const BndBar& G, int bc, int x, int y, int z, int c) {
    return G.p[bc] + (size_t)c * P.plane[bc] + plane_idx(P, bc, x, y, z);
}

// ---------------------------------------------------------------- PISO
// VJP of PVEL: c[a] = -(1/D_a) (aod[a] + dv/den * (pf+ - pf-)/dx), face values
// of s averaged with fluid neighbours, else the cell's own (PisoColl.compute:
// 294-336).
__global__ void k_adj_pvel(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                           const float* __restrict__ cbar, const float* __restrict__ ss,
                           const float* __restrict__ Dv, const float* __restrict__ aod, float* __restrict__ abar,
                           float* __restrict__ ssbar, float* __restrict__ Dbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float pP = ld(ss, c.i);
    float pf[6];
    int qn[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        qn[f] = -1;
        pf[f] = pP;
        if (in_region(P, X, Y, Z)) {
            const int q = cidx(P, X, Y, Z);
            if (fluid_at(fl, q)) {
                qn[f] = q;
                pf[f] = 0.5f * (pP + ld(ss, q));
            }
        }
    }
    float pfb[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float k = P.dv / P.den;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float w = ld(cbar, a * N + c.i);
        if (w == 0.f) continue;
        const float Da = ld(Dv, a * N + c.i);
        const float grad = (pf[2 * a] - pf[2 * a + 1]) / P.dx;
        const float K = ld(aod, a * N + c.i) + k * grad;
        aadd(Dbar + a * N + c.i, w * K / (Da * Da));
        aadd(abar + a * N + c.i, -w / Da);
        const float gb = -w / Da * k / P.dx;
        pfb[2 * a] += gb;
        pfb[2 * a + 1] -= gb;
    }
    float own = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (qn[f] >= 0) {
            own += 0.5f * pfb[f];
            aadd(ssbar + qn[f], 0.5f * pfb[f]);
        } else {
            own += pfb[f];
        }
    }
    aadd(ssbar + c.i, own);
}

// Reversed pressure-type Jacobi loop s^{k+1} = ai (r - C s^k), s^0 = 0,
// k = 0..n-1, in the variable W^k = ai * sbar^k (sbar^k: adjoint of s^k):
//   W^n = ai * sbar^n,   W^k = ai * (-C W^{k+1})
// (C is symmetric, so the transposed sweep is the forward sweep with a zero
// right-hand side, run by the multi-sweep kernel with every level kept),
// then one pass over the stored iterates gives the adjoints of the loop's
// inputs:  rbar = sum_k W^k,  coefbar = -sum_k W^k s^k (adjoint of 1/ai),
// cbar_f(P) = -sum_k (W^k_P s^{k-1}_Q + W^k_Q s^{k-1}_P).
__global__ void k_adj_pinit(int n, const float* __restrict__ ai, const float* __restrict__ sbar,
                            float* __restrict__ W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) W[i] = ai[i] * sbar[i];
}
// W: stack with W^k in slot n-k (k = 1..n), s: stack of s^0..s^n.
__global__ void __launch_bounds__(256) k_adj_pacc(const __grid_constant__ Params P, int n,
                                                  const float* __restrict__ ai, const float* __restrict__ W,
                                                  const float* __restrict__ s, float* __restrict__ rbar,
                                                  float* __restrict__ coefbar, float* __restrict__ c3bar) {
    Cell c;
    if (!thread_cell(P, c)) return;
    const size_t N = P.N;
    if (ld(ai, c.i) == 0.f) {
        rbar[c.i] = 0.f;
        coefbar[c.i] = 0.f;
        return;
    }
    const int sx = P.nx, sz = P.nx * P.ny;
    const bool hE = c.x + 1 < P.nx, hN = c.y + 1 < P.ny, hU = c.z + 1 < P.nz;
    float r = 0.f, d = 0.f, cE = 0.f, cN = 0.f, cU = 0.f;
    for (int k = 1; k <= n; ++k) {
        const float* Wk = W + (size_t)(n - k) * N;
        const float* sk = s + (size_t)k * N;
        const float* sm = s + (size_t)(k - 1) * N;
        const float w = ld(Wk, c.i);
        r += w;
        d -= w * ld(sk, c.i);
        if (k > 1) {
            const float sP = ld(sm, c.i);
            if (hE) cE -= w * ld(sm, c.i + 1) + ld(Wk, c.i + 1) * sP;
            if (hN) cN -= w * ld(sm, c.i + sx) + ld(Wk, c.i + sx) * sP;
            if (hU) cU -= w * ld(sm, c.i + sz) + ld(Wk, c.i + sz) * sP;
        }
    }
    rbar[c.i] = r;
    coefbar[c.i] = d;
    c3bar[c.i] += cE;
    c3bar[N + c.i] += cN;
    c3bar[2 * N + c.i] += cU;
}

// k_adj_pacc with four x-consecutive cells per thread (nx % 4 == 0, aligned
// planes): 128-bit loads, the same per-cell sums (bit-identical).
__device__ __forceinline__ float4 ld4p(const float* p, size_t i) {
    return __ldg(reinterpret_cast<const float4*>(p + i));
}
__device__ __forceinline__ float f4p(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }
__global__ void __launch_bounds__(256) k_adj_pacc4(const __grid_constant__ Params P, int n,
                                                   const float* __restrict__ ai, const float* __restrict__ W,
                                                   const float* __restrict__ s, float* __restrict__ rbar,
                                                   float* __restrict__ coefbar, float* __restrict__ c3bar) {
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x0 >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x0, y, z);
    const size_t N = P.N;
    const int sx = P.nx, sz = P.nx * P.ny;
    const bool hE3 = x0 + 4 < P.nx, hN = y + 1 < P.ny, hU = z + 1 < P.nz;
    const int iE = hE3 ? i + 4 : i + 3, iN = hN ? i + sx : i, iU = hU ? i + sz : i;
    const float4 a4 = ld4p(ai, i);
    float r[4] = {0.f, 0.f, 0.f, 0.f}, d[4] = {0.f, 0.f, 0.f, 0.f};
    float cE[4] = {0.f, 0.f, 0.f, 0.f}, cN[4] = {0.f, 0.f, 0.f, 0.f}, cU[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
    for (int k = 1; k <= n; ++k) {
        const float* Wk = W + (size_t)(n - k) * N;
        const float* sk = s + (size_t)k * N;
        const float* sm = s + (size_t)(k - 1) * N;
        const float4 w = ld4p(Wk, i), sv = ld4p(sk, i);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            r[j] += f4p(w, j);
            d[j] -= f4p(w, j) * f4p(sv, j);
        }
        if (k > 1) {
            const float4 sp = ld4p(sm, i), sn = ld4p(sm, iN), su = ld4p(sm, iU);
            const float4 wn = ld4p(Wk, iN), wu = ld4p(Wk, iU);
            const float se3 = __ldg(sm + iE), we3 = __ldg(Wk + iE);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float wj = f4p(w, j), sP = f4p(sp, j);
                if (j < 3 || hE3) {
                    const float sE = j < 3 ? f4p(sp, j + 1) : se3;
                    const float wE = j < 3 ? f4p(w, j + 1) : we3;
                    cE[j] -= wj * sE + wE * sP;
                }
                if (hN) cN[j] -= wj * f4p(sn, j) + f4p(wn, j) * sP;
                if (hU) cU[j] -= wj * f4p(su, j) + f4p(wu, j) * sP;
            }
        }
    }
    float ro[4], co[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const bool fl = f4p(a4, j) != 0.f;
        ro[j] = fl ? r[j] : 0.f;
        co[j] = fl ? d[j] : 0.f;
        if (fl) {
            c3bar[i + j] += cE[j];
            c3bar[N + i + j] += cN[j];
            c3bar[2 * N + i + j] += cU[j];
        }
    }
    *reinterpret_cast<float4*>(rbar + i) = make_float4(ro[0], ro[1], ro[2], ro[3]);
    *reinterpret_cast<float4*>(coefbar + i) = make_float4(co[0], co[1], co[2], co[3]);
}

// VJP of PISOPRE: coef = -sum_f (dv/den) AdInv_f / dx, ai = 1/coef,
// r = -sum_f s_f AdInv_f Aod_f (PisoColl.compute:196-255); coefbar is the
// adjoint of coef.
__global__ void k_adj_pisopre(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                              const float* __restrict__ coefbar, const float* __restrict__ rbar,
                              const float* __restrict__ Dv, const float* __restrict__ aod, float* __restrict__ abar,
                              float* __restrict__ Dbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float coefb = ld(coefbar, c.i);
    const float rb = ld(rbar, c.i);
    const float k = P.dv / P.den / P.dx;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f), s = face_sign(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (!in_region(P, X, Y, Z)) continue;
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float DP = ld(Dv, a * N + c.i), DQ = ld(Dv, a * N + q);
        const float AdInv = 0.5f * (1.f / DP + 1.f / DQ);
        const float Aod = 0.5f * (ld(aod, a * N + c.i) + ld(aod, a * N + q));
        const float adinvb = -k * coefb - s * Aod * rb;
        const float aodb = -s * AdInv * rb;
        aadd(abar + a * N + c.i, 0.5f * aodb);
        aadd(abar + a * N + q, 0.5f * aodb);
        aadd(Dbar + a * N + c.i, -0.5f * adinvb / (DP * DP));
        aadd(Dbar + a * N + q, -0.5f * adinvb / (DQ * DQ));
    }
}

// VJP of the face coefficients c_f = (dv/den) 0.5 (1/D_P + 1/D_Q) / dx
// (owner cell P holds its E/N/U faces).
__global__ void k_adj_c3(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                         const float* __restrict__ c3bar, const float* __restrict__ Dv, float* __restrict__ Dbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float k = P.dv / P.den / P.dx;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float cb = ld(c3bar, a * N + c.i);
        if (cb == 0.f) continue;
        const int f = 2 * a;
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (!in_region(P, X, Y, Z)) continue;
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float DP = ld(Dv, a * N + c.i), DQ = ld(Dv, a * N + q);
        aadd(Dbar + a * N + c.i, -0.5f * k * cb / (DP * DP));
        aadd(Dbar + a * N + q, -0.5f * k * cb / (DQ * DQ));
    }
}

// VJP of AOD: a_P[c] = sum_fluid f (s_f ds/4 (uT_P[a] + uT_Q[a]) - nu ds/dx) cm_Q[c]
// (PisoColl.compute:90-177, reference nu-only diffusion).
__global__ void k_adj_aod(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                          const float* __restrict__ abar, const float* __restrict__ cm,
                          const float* __restrict__ uT, float* __restrict__ cmbar, float* __restrict__ uTbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float ab[3] = {ld(abar, c.i), ld(abar, N + c.i), ld(abar, 2 * N + c.i)};
    if (ab[0] == 0.f && ab[1] == 0.f && ab[2] == 0.f) return;
    const float dif = P.nu * P.ds / P.dx;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f), s = face_sign(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (!in_region(P, X, Y, Z)) continue;
        const int q = cidx(P, X, Y, Z);
        if (!fluid_at(fl, q)) continue;
        const float sum = ld(uT, a * N + c.i) + ld(uT, a * N + q);
        const float coef = s * (P.ds * 0.25f * sum) - dif;
        float t = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            aadd(cmbar + k * N + q, coef * ab[k]);
            t += ld(cm, k * N + q) * ab[k];
        }
        t *= s * P.ds * 0.25f;
        aadd(uTbar + a * N + c.i, t);
        aadd(uTbar + a * N + q, t);
    }
}

// Face value of a pressure-type field with the SIMPLE boundary rules
// (FvmColl.compute:2975-3113): fluid neighbour -> average, solid neighbour ->
// own value, domain face -> 0 for fixed pressure else own value.  Returns the
// neighbour index that shares the face (-1 if none) and whether the face is a
// fixed-pressure domain face.
__device__ __forceinline__ void face_rule(const Params& P, const uint8_t* fl, const Cell& c, int f, int& q,
                                          bool& fixed0) {
    const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
    q = -1;
    fixed0 = false;
    if (in_region(P, X, Y, Z)) {
        const int n = cidx(P, X, Y, Z);
        if (fluid_at(fl, n)) q = n;
    } else {
        fixed0 = P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE;
    }
}

// VJP of CORR (CSApplyVelCorrectionDivergenceTheorem):
// c[a] = -(dv/den) (1/D_a) (pf+ - pf-) / dx.
__global__ void k_adj_corr(const __grid_constant__ Params P, const uint8_t* __restrict__ fl,
                           const float* __restrict__ cbar, const float* __restrict__ qf,
                           const float* __restrict__ Dv, float* __restrict__ qbar, float* __restrict__ Dbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float pP = ld(qf, c.i);
    float pf[6];
    int qn[6];
    bool fx[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        face_rule(P, fl, c, f, qn[f], fx[f]);
        pf[f] = qn[f] >= 0 ? 0.5f * (pP + ld(qf, qn[f])) : (fx[f] ? 0.f : pP);
    }
    float pfb[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float k = P.dv / P.den;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float w = ld(cbar, a * N + c.i);
        if (w == 0.f) continue;
        const float Da = ld(Dv, a * N + c.i);
        const float K = k * (pf[2 * a] - pf[2 * a + 1]) / P.dx;
        aadd(Dbar + a * N + c.i, w * K / (Da * Da));
        const float g = -w * k / (Da * P.dx);
        pfb[2 * a] += g;
        pfb[2 * a + 1] -= g;
    }
    float own = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (qn[f] >= 0) {
            own += 0.5f * pfb[f];
            aadd(qbar + qn[f], 0.5f * pfb[f]);
        } else if (!fx[f]) {
            own += pfb[f];
        }
    }
    aadd(qbar + c.i, own);
}

// VJP of PPRE (CSPresCorrectRhieChowPreCompute, FvmColl.compute:2481-2787).
__global__ void k_adj_ppre(const __grid_constant__ Params P, const BndBar G,
                           const uint8_t* __restrict__ fl, const float* __restrict__ Dpbar,
                           const float* __restrict__ bpbar, const float* __restrict__ pr,
                           const float* __restrict__ Dv, float* __restrict__ ubar, float* __restrict__ pbar,
                           float* __restrict__ Dbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float dpb = ld(Dpbar, c.i), bpb = ld(bpbar, c.i);
    if (dpb == 0.f && bpb == 0.f) return;
    const float dx2 = 2.f * P.dx;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f), s = face_sign(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (in_region(P, X, Y, Z)) {
            const int q = cidx(P, X, Y, Z);
            if (!fluid_at(fl, q)) continue;
            const float DP = ld(Dv, a * N + c.i), DQ = ld(Dv, a * N + q);
            const float DInv = 0.5f * (1.f / DP + 1.f / DQ);
            float dinvb = -(P.dv / P.den) / P.dx * dpb;
            // face flux 0.5 (u_P + u_Q)
            aadd(ubar + a * N + c.i, 0.5f * s * bpb);
            aadd(ubar + a * N + q, 0.5f * s * bpb);
            // Rhie-Chow: vct = -(dv DInv / den) (presGrad - ave), linear in p
            const int L = s > 0 ? c.i : q, H = s > 0 ? q : c.i;
            const int lx = s > 0 ? c.x : X, ly = s > 0 ? c.y : Y, lz = s > 0 ? c.z : Z;
            const int hx = s > 0 ? X : c.x, hy = s > 0 ? Y : c.y, hz = s > 0 ? Z : c.z;
            const int ex = (a == 0), ey = (a == 1), ez = (a == 2);
            const bool hhin = in_region(P, hx + ex, hy + ey, hz + ez);
            const bool llin = in_region(P, lx - ex, ly - ey, lz - ez);
            const int HH = hhin ? cidx(P, hx + ex, hy + ey, hz + ez) : -1;
            const int LL = llin ? cidx(P, lx - ex, ly - ey, lz - ez) : -1;
            const bool hh = hhin && fluid_at(fl, HH);
            const bool ll = llin && fluid_at(fl, LL);
            if (hh || ll) {
                float wL = -1.f / P.dx, wH = 1.f / P.dx, wLL = 0.f, wHH = 0.f;
                // subtract ave = 0.5 (gH + gL)
                if (hh) { wHH -= 0.5f / dx2; wL += 0.5f / dx2; }
                else { wH -= 0.5f / dx2; wL += 0.5f / dx2; }
                if (ll) { wH -= 0.5f / dx2; wLL += 0.5f / dx2; }
                else { wH -= 0.5f / dx2; wL += 0.5f / dx2; }
                const float pL = ld(pr, L), pH = ld(pr, H);
                float diff = wL * pL + wH * pH;
                if (hh) diff += wHH * ld(pr, HH);
                if (ll) diff += wLL * ld(pr, LL);
                const float vctb = s * bpb;
                dinvb += -(P.dv / P.den) * diff * vctb;
                const float diffb = -(P.dv * DInv) / P.den * vctb;
                aadd(pbar + L, wL * diffb);
                aadd(pbar + H, wH * diffb);
                if (hh) aadd(pbar + HH, wHH * diffb);
                if (ll) aadd(pbar + LL, wLL * diffb);
            }
            aadd(Dbar + a * N + c.i, -0.5f * dinvb / (DP * DP));
            aadd(Dbar + a * N + q, -0.5f * dinvb / (DQ * DQ));
        } else {
            const int bc = face_bc(f), vb = P.vbc[bc];
            if (vb == WF_BND_FIXED_VALUE) {
                aadd(bnd_bar(P, G, bc, c.x, c.y, c.z, a), s * bpb);
            } else if (vb == WF_BND_ZERO_GRAD) {
                aadd(ubar + a * N + c.i, s * bpb);
            }
            if (P.pbc[bc] == WF_BND_FIXED_VALUE) {
                const float DP = ld(Dv, a * N + c.i);
                aadd(Dbar + a * N + c.i, dpb * 2.f * (P.dv / P.den) / (P.dx * DP * DP));
            }
        }
    }
}

// Reversed momentum Jacobi loop u^{k+1} = iD (A u^k + b), u^0 = uT, in the
// variable W^k = iD * ubar^k (fluid cells):
//   W^n = iD * ubar^n,  W^k = iD * (A^T W^{k+1}),  ubar^0 = A^T W^1
// (non-fluid cells keep their value through the loop, so their ubar^0 is
// ubar^n).  A^T is stored per receiving cell: AT_f(Q) = A_{f^1}(nb_f(Q)),
// the coefficient with which neighbour nb_f(Q) reads Q; it is 0 unless both
// cells are fluid.
__global__ void k_adj_vtrans(const __grid_constant__ Params P, const float* __restrict__ A, float* __restrict__ AT) {
    Cell c;
    if (!thread_cell(P, c)) return;
    const size_t N = P.N;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        AT[f * N + c.i] = in_region(P, X, Y, Z) ? ld(A, (size_t)(f ^ 1) * N + cidx(P, X, Y, Z)) : 0.f;
    }
}
__global__ void k_adj_vinit(long long n3, const float* __restrict__ iD, const float* __restrict__ ubar,
                            float* __restrict__ W) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n3) W[i] = iD[i] * ubar[i];
}
// kLast: out += ubar^0 (ubarN on non-fluid cells); else out = W^k.
template <bool kLast>
__global__ void __launch_bounds__(256) k_adj_vsweepT(const __grid_constant__ Params P, const float* __restrict__ AT,
                                                     const float* __restrict__ iD, const float* __restrict__ Wi,
                                                     const float* __restrict__ ubarN, float* __restrict__ out) {
    Cell c;
    if (!thread_cell(P, c)) return;
    const size_t N = P.N;
    if (kLast && ld(iD, c.i) == 0.f) {
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k * N + c.i] += ld(ubarN, k * N + c.i);
        return;
    }
    // non-fluid cells: AT = 0 and iD = 0, so W^k = 0 there without a test
    const int sx = P.nx, sz = P.nx * P.ny;
    const int iE = c.x + 1 < P.nx ? c.i + 1 : c.i, iW = c.x > 0 ? c.i - 1 : c.i;
    const int iN = c.y + 1 < P.ny ? c.i + sx : c.i, iS = c.y > 0 ? c.i - sx : c.i;
    const int iU = c.z + 1 < P.nz ? c.i + sz : c.i, iDn = c.z > 0 ? c.i - sz : c.i;
    const float t0 = ld(AT, c.i), t1 = ld(AT, N + c.i), t2 = ld(AT, 2 * N + c.i);
    const float t3 = ld(AT, 3 * N + c.i), t4 = ld(AT, 4 * N + c.i), t5 = ld(AT, 5 * N + c.i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float* w = Wi + k * N;
        float s = t0 * ld(w, iE);
        s += t1 * ld(w, iW);
        s += t2 * ld(w, iN);
        s += t3 * ld(w, iS);
        s += t4 * ld(w, iU);
        s += t5 * ld(w, iDn);
        if (kLast) out[k * N + c.i] += s;
        else out[k * N + c.i] = ld(iD, k * N + c.i) * s;
    }
}
// k_adj_vsweepT<false> with four x-consecutive cells per thread (nx % 4 == 0,
// 16-byte aligned planes): 128-bit loads, every load issued first, the same
// arithmetic per cell (the forward sweep's four-cell form, transposed).
__device__ __forceinline__ float4 ld4a(const float* p, size_t i) {
    return __ldg(reinterpret_cast<const float4*>(p + i));
}
__device__ __forceinline__ float f4a(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }
__global__ void __launch_bounds__(256) k_adj_vsweepT4(const __grid_constant__ Params P, const float* __restrict__ AT,
                                                      const float* __restrict__ iD, const float* __restrict__ Wi,
                                                      float* __restrict__ out) {
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x0 >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x0, y, z);
    const size_t N = P.N;
    const int sx = P.nx, sz = P.nx * P.ny;
    const int iN = y + 1 < P.ny ? i + sx : i, iS = y > 0 ? i - sx : i;
    const int iU = z + 1 < P.nz ? i + sz : i, iDn = z > 0 ? i - sz : i;
    const int iE = x0 + 4 < P.nx ? i + 4 : i + 3, iW = x0 > 0 ? i - 1 : i;
    const float4 t0 = ld4a(AT, i), t1 = ld4a(AT, N + i), t2 = ld4a(AT, 2 * N + i);
    const float4 t3 = ld4a(AT, 3 * N + i), t4 = ld4a(AT, 4 * N + i), t5 = ld4a(AT, 5 * N + i);
    float4 c[3], n[3], so[3], up[3], dn[3], dd[3];
    float e3[3], w0[3];
    // 1/D: the first component stands for all three outside d_split cells,
    // read there from one address (an L1 hit) so no load waits on a branch
    const size_t o1 = d_split(P, x0, x0 + 3, y, z) ? N : 0;
    dd[0] = ld4a(iD, i);
    dd[1] = ld4a(iD, o1 + i);
    dd[2] = ld4a(iD, 2 * o1 + i);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float* w = Wi + k * N;
        c[k] = ld4a(w, i);
        n[k] = ld4a(w, iN);
        so[k] = ld4a(w, iS);
        up[k] = ld4a(w, iU);
        dn[k] = ld4a(w, iDn);
        e3[k] = __ldg(w + iE);
        w0[k] = __ldg(w + iW);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float we = j < 3 ? f4a(c[k], j + 1) : e3[k];
            const float ww = j > 0 ? f4a(c[k], j - 1) : w0[k];
            float s = f4a(t0, j) * we;
            s += f4a(t1, j) * ww;
            s += f4a(t2, j) * f4a(n[k], j);
            s += f4a(t3, j) * f4a(so[k], j);
            s += f4a(t4, j) * f4a(up[k], j);
            s += f4a(t5, j) * f4a(dn[k], j);
            v[j] = f4a(dd[k], j) * s;
        }
        *reinterpret_cast<float4*>(out + k * N + i) = make_float4(v[0], v[1], v[2], v[3]);
    }
}

// One pass over the loop's iterates (u: stack u^0..u^n, W: stack W^1..W^n,
// slot k at k*3N): bbar = sum_k W^k, Dbar -= sum_k W^k u^k (adjoint of 1/D
// folded in), Abar_f = sum_k W^k . u^{k-1}_nb, and the adjoint of
// A_f = nu ds/dx - s_f ds/4 (uT_P[a] + uT_Q[a]) scattered to uTbar.
__global__ void __launch_bounds__(256) k_adj_vacc(const __grid_constant__ Params P, int n,
                                                  const uint8_t* __restrict__ fl, const float* __restrict__ W,
                                                  const float* __restrict__ u, float* __restrict__ bbar,
                                                  float* __restrict__ Dbar, float* __restrict__ uTbar) {
    Cell c;
    if (!thread_cell(P, c)) return;
    const size_t N = P.N, N3 = 3 * N;
    if (!fluid_at(fl, c.i)) return;
    int nb[6];
    bool has[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        has[f] = in_region(P, X, Y, Z) && fluid_at(fl, cidx(P, X, Y, Z));
        nb[f] = has[f] ? cidx(P, X, Y, Z) : c.i;
    }
    float Ab[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float bb[3] = {0.f, 0.f, 0.f}, db[3] = {0.f, 0.f, 0.f};
#pragma unroll 2
    for (int k = 1; k <= n; ++k) {
        const float* Wk = W + k * N3;
        const float* uk = u + k * N3;
        const float* um = u + (k - 1) * N3;
        float w[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            w[j] = ld(Wk, j * N + c.i);
            bb[j] += w[j];
            db[j] -= w[j] * ld(uk, j * N + c.i);
        }
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (!has[f]) continue;
            Ab[f] += w[0] * ld(um, nb[f]) + w[1] * ld(um, N + nb[f]) + w[2] * ld(um, 2 * N + nb[f]);
        }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        bbar[j * N + c.i] = bb[j];
        aadd(Dbar + j * N + c.i, db[j]);
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!has[f]) continue;
        const int a = face_axis(f), s = face_sign(f);
        const float t = -s * P.ds * 0.25f * Ab[f];
        aadd(uTbar + a * N + c.i, t);
        aadd(uTbar + a * N + nb[f], t);
    }
}

// k_adj_vacc with four x-consecutive cells per thread (nx % 4 == 0, aligned
// planes): every iterate plane is read with 128-bit loads (the x neighbours
// beyond the four cells with scalar loads), a quarter of the load
// instructions of one cell per thread; the per-cell sums are the same
// (bbar and the own-cell parts bit-identical, the scattered parts to the
// order of the float atomics).  Fluid cells and fluid-fluid faces come from
// the neighbour mask.
__global__ void __launch_bounds__(128) k_adj_vacc4(const __grid_constant__ Params P, int n,
                                                   const float* __restrict__ W, const float* __restrict__ u,
                                                   float* __restrict__ bbar, float* __restrict__ Dbar,
                                                   float* __restrict__ uTbar) {
    const int x0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x0 >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x0, y, z);
    const size_t N = P.N, N3 = 3 * N;
    const uchar4 m4 = __ldg(reinterpret_cast<const uchar4*>(P.nbm + i));
    const unsigned mm[4] = {m4.x, m4.y, m4.z, m4.w};
    const int sx = P.nx, sz = P.nx * P.ny;
    const int iN = y + 1 < P.ny ? i + sx : i, iS = y > 0 ? i - sx : i;
    const int iU = z + 1 < P.nz ? i + sz : i, iDn = z > 0 ? i - sz : i;
    const int iE = x0 + 4 < P.nx ? i + 4 : i + 3, iW = x0 > 0 ? i - 1 : i;
    float Ab[4][6], bb[4][3], db[4][3];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int f = 0; f < 6; ++f) Ab[j][f] = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) bb[j][c] = db[j][c] = 0.f;
    }
#pragma unroll 1
    for (int k = 1; k <= n; ++k) {
        const float* Wk = W + k * N3;
        const float* uk = u + k * N3;
        const float* um = u + (k - 1) * N3;
        float4 w[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            w[c] = ld4a(Wk, c * N + i);
            const float4 uu = ld4a(uk, c * N + i);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                bb[j][c] += f4a(w[c], j);
                db[j][c] -= f4a(w[c], j) * f4a(uu, j);
            }
        }
        float nv[3][4][6];  // u^{k-1} at the neighbour across f of cell j
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float* p = um + c * N;
            const float4 cc = ld4a(p, i), nn = ld4a(p, iN), ss = ld4a(p, iS), uu = ld4a(p, iU), dd = ld4a(p, iDn);
            const float e3 = __ldg(p + iE), w0 = __ldg(p + iW);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                nv[c][j][0] = j < 3 ? f4a(cc, j + 1) : e3;
                nv[c][j][1] = j > 0 ? f4a(cc, j - 1) : w0;
                nv[c][j][2] = f4a(nn, j);
                nv[c][j][3] = f4a(ss, j);
                nv[c][j][4] = f4a(uu, j);
                nv[c][j][5] = f4a(dd, j);
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                if (!nb_fluid(mm[j], f)) continue;
                Ab[j][f] += f4a(w[0], j) * nv[0][j][f] + f4a(w[1], j) * nv[1][j][f] + f4a(w[2], j) * nv[2][j][f];
            }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!(mm[j] & 64u)) continue;
        const int ij = i + j;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            bbar[c * N + ij] = bb[j][c];
            aadd(Dbar + c * N + ij, db[j][c]);
        }
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (!nb_fluid(mm[j], f)) continue;
            const int a = face_axis(f), s = face_sign(f);
            const float t = -s * P.ds * 0.25f * Ab[j][f];
            aadd(uTbar + a * N + ij, t);
            aadd(uTbar + a * N + ij + face_off(P, f), t);
        }
    }
}

// VJP of PRE (CSVelPredictPreCompute with LES off, FvmColl.compute:1292-1859).
__global__ void k_adj_pre(const __grid_constant__ Params P, const Bnd B, const BndBar G,
                          const uint8_t* __restrict__ fl, const float* __restrict__ Dbar,
                          const float* __restrict__ bbar, float* __restrict__ uTbar, float* __restrict__ pbar,
                          float* __restrict__ dragbar) {
    Cell c;
    if (!thread_cell(P, c) || !fluid_at(fl, c.i)) return;
    const size_t N = P.N;
    const float db[3] = {ld(Dbar, c.i), ld(Dbar, N + c.i), ld(Dbar, 2 * N + c.i)};
    const float bb[3] = {ld(bbar, c.i), ld(bbar, N + c.i), ld(bbar, 2 * N + c.i)};
    const float sD = db[0] + db[1] + db[2];
    // Brinkman drag: D[k] += dv * drag for every k
    dragbar[c.i] += P.dv * sD;
    // advection
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f), s = face_sign(f);
        const int X = c.x + face_ox(f), Y = c.y + face_oy(f), Z = c.z + face_oz(f);
        if (in_region(P, X, Y, Z)) {
            const int q = cidx(P, X, Y, Z);
            if (fluid_at(fl, q)) {
                const float t = s * P.ds * 0.25f * sD;
                aadd(uTbar + a * N + c.i, t);
                aadd(uTbar + a * N + q, t);
            }
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            if (bt == WF_BND_FIXED_VALUE) {
                float g[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) g[k] = bnd_comp(P, B, bc, c.x, c.y, c.z, k);
                float tsum = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    aadd(bnd_bar(P, G, bc, c.x, c.y, c.z, k), -s * P.ds * g[a] * bb[k]);
                    tsum += g[k] * bb[k];
                }
                aadd(bnd_bar(P, G, bc, c.x, c.y, c.z, a), -s * P.ds * tsum);
                // diffusion of the fixed value: b[k] += 2 nu ds/dx g[k]
                const float t = 2.f * P.nu * P.ds / P.dx;
#pragma unroll
                for (int k = 0; k < 3; ++k) aadd(bnd_bar(P, G, bc, c.x, c.y, c.z, k), t * bb[k]);
            } else if (bt == WF_BND_ZERO_GRAD) {
                aadd(uTbar + a * N + c.i, s * P.ds * sD);
            }
        }
    }
    // pressure: b[a] += -(1/den) ds (pf[2a] - pf[2a+1])
    float own = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const float pfb = (f & 1) ? (P.ds / P.den) * bb[a] : -(P.ds / P.den) * bb[a];
        int q;
        bool fx;
        face_rule(P, fl, c, f, q, fx);
        if (q >= 0) {
            own += 0.5f * pfb;
            aadd(pbar + q, 0.5f * pfb);
        } else if (!fx) {
            own += pfb;
        }
    }
    aadd(pbar + c.i, own);
    // time term
    const float dvdt = P.dv / P.dt;
#pragma unroll
    for (int k = 0; k < 3; ++k) aadd(uTbar + k * N + c.i, dvdt * bb[k]);
}

__global__ void k_axpy(long long n, float a, const float* __restrict__ x, float* __restrict__ y) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}
// y[i] += x[i] on cells of the mask (solid_ok: every non-solid cell; else fluid)
__global__ void k_add_masked(int n, const uint8_t* __restrict__ fl, const float* __restrict__ x,
                             float* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && fl[i] == WF_CELL_FLUID) y[i] += x[i];
}

// Objective: J += w * sum of |u|^2 over the fluid cells of the patch, and
// ubar += 2 w u there.
__global__ void k_objective(const __grid_constant__ Params P, const uint8_t* __restrict__ fl, int x0, int x1, int y,
                            int z0, int z1, float w, const float* __restrict__ u, float* __restrict__ ubar,
                            double* __restrict__ Jacc) {
    const int x = x0 + blockIdx.x * blockDim.x + threadIdx.x;
    const int z = z0 + blockIdx.y * blockDim.y + threadIdx.y;
    double s = 0.0;
    if (x < x1 && z < z1 && fl[cidx(P, x, y, z)] == WF_CELL_FLUID) {
        const int i = cidx(P, x, y, z);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float v = u[(size_t)k * P.N + i];
            s += (double)v * v;
            if (ubar) ubar[(size_t)k * P.N + i] += 2.f * w * v;
        }
    }
    if (Jacc) {
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(Jacc, s * (double)w);
    }
}

dim3 cblk() { return dim3(32, 4, 2); }
dim3 cgrd(const Params& P) {
    dim3 b = cblk();
    return dim3((P.nx + b.x - 1) / b.x, (P.ny + b.y - 1) / b.y, (P.nz + b.z - 1) / b.z);
}
int lin_blocks(long long n) { return (int)((n + 255) / 256); }

}  // namespace
}  // namespace wf

// =====================================================================
namespace {
// Everything one forward step leaves behind for its adjoint.
struct Tape {
    float *uT = nullptr, *p0 = nullptr;         // step input
    float *D = nullptr, *b = nullptr;           // momentum diagonal, rhs (3N each)
    float *A = nullptr, *iD = nullptr;          // sweep coefficients (6N, 3N)
    float* uit = nullptr;                       // u^0..u^nV ((nV+1) x 3N)
    float *Dp = nullptr, *bp = nullptr, *c3 = nullptr, *ainv = nullptr;
    float* qit = nullptr;                       // q^0..q^nP ((nP+1) x N)
    float* cbuf = nullptr;                      // corrections c_0..c_nC ((nC+1) x 3N)
    float *aod = nullptr, *pai = nullptr, *prhs = nullptr;  // per PISO corrector
    float* sit = nullptr;                       // s^0..s^nP per corrector
    float *uout = nullptr, *pout = nullptr;     // step output
};
}  // namespace

struct wf_adjoint {
    wf_solver* h = nullptr;
    cudaStream_t st = nullptr;
    int nV = 0, nP = 0, nC = 0;
    size_t N = 0;
    std::vector<Tape> tapes;                    // tapes[0] always allocated
    int max_tapes = 0;                          // cap on the tapes a gradient uses (0: as many as fit)
    bool shorten = true;                        // segments no longer than the tapes that fit
    std::vector<void*> blocks;                  // allocations behind the tapes
    // adjoint work
    float *ub = nullptr, *uTb = nullptr, *pb = nullptr, *pb_in = nullptr;
    float *Db = nullptr, *bb = nullptr, *AT = nullptr, *Wv = nullptr, *Wp = nullptr, *c3b = nullptr;
    float *cb = nullptr, *cb2 = nullptr, *ab = nullptr, *sb = nullptr;
    float *rb = nullptr, *dgb = nullptr;
    float* gb = nullptr;     // adjoint of the 6 boundary planes (same layout)
    float* dragb = nullptr;  // adjoint of the drag field (N)
    double* dJ = nullptr;    // device accumulator of the objective
    std::vector<float*> ck;  // stored states (4N each: u then p)
    std::string err;
};

namespace {

using wf::Params;

int adj_fail(wf_adjoint* a, int code, const char* msg) {
    a->err = msg;
    return code;
}

#define WFA_CUDA(call)                                                         \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            a->err = std::string(#call) + ": " + cudaGetErrorString(e_);       \
            return e_ == cudaErrorMemoryAllocation ? WF_ERR_OOM : WF_ERR_CUDA; \
        }                                                                      \
    } while (0)

// WF_ERR_TIMEOUT when a bounded wait of the TMA-staged pressure passes ran
// out since the last check (the solver's sticky wait status).
int adj_check_waits(wf_adjoint* a) {
    volatile int* st = a->h->hstat;
    if (!st || !*st) return WF_OK;
    *st = 0;
    return adj_fail(a, WF_ERR_TIMEOUT, "a bounded wait of the TMA-staged pressure pass ran out; results are not valid");
}

float* V(const wf_adjoint* a, float* base, int k) { return base + (size_t)k * 3 * a->N; }
float* S(const wf_adjoint* a, float* base, int k) { return base + (size_t)k * a->N; }
float* SIT(const wf_adjoint* a, const Tape& t, int m, int k) {
    return t.sit + ((size_t)m * (a->nP + 1) + k) * a->N;
}

wf::BndBar bnd_bar(const wf_adjoint* a) {
    wf::BndBar G;
    const Params& P = a->h->P;
    float* p = a->gb;
    for (int f = 0; f < 6; ++f) {
        G.p[f] = p;
        p += 3 * (size_t)P.plane[f];
    }
    return G;
}
size_t plane_floats(const Params& P) {
    size_t n = 0;
    for (int f = 0; f < 6; ++f) n += 3 * (size_t)P.plane[f];
    return n;
}

// Floats of one tape, carved from one allocation.
size_t tape_floats(const wf_adjoint* a) {
    const size_t N = a->N, nC1 = a->nC > 0 ? a->nC : 1;
    return N * (3 + 1 + 3 + 3 + 6 + 3 + 3 * (a->nV + 1) + 4 + 3 + (a->nP + 1) + 3 * (a->nC + 1) + nC1 * (3 + 1 + 1) +
                nC1 * (a->nP + 1) + 3 + 1);
}
void carve(const wf_adjoint* a, float* base, Tape& t) {
    const size_t N = a->N, nC1 = a->nC > 0 ? a->nC : 1;
    float* p = base;
    auto take = [&](float** dst, size_t n) {
        *dst = p;
        p += n;
    };
    take(&t.uT, 3 * N); take(&t.p0, N); take(&t.D, 3 * N); take(&t.b, 3 * N); take(&t.A, 6 * N);
    take(&t.iD, 3 * N); take(&t.uit, 3 * N * (a->nV + 1)); take(&t.Dp, N); take(&t.bp, N); take(&t.c3, 3 * N);
    take(&t.ainv, N); take(&t.qit, N * (a->nP + 1)); take(&t.cbuf, 3 * N * (a->nC + 1)); take(&t.aod, 3 * N * nC1);
    take(&t.pai, N * nC1); take(&t.prhs, N * nC1); take(&t.sit, N * nC1 * (a->nP + 1)); take(&t.uout, 3 * N);
    take(&t.pout, N);
}
int ensure_tapes(wf_adjoint* a, int n) {
    if ((int)a->tapes.size() >= n) return WF_OK;
    const size_t bytes = tape_floats(a) * sizeof(float);
    while ((int)a->tapes.size() < n) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return adj_fail(a, WF_ERR_OOM, "no device memory for the step tapes: lower checkpoint_every");
        }
        a->blocks.push_back(p);
        Tape t;
        carve(a, (float*)p, t);
        a->tapes.push_back(t);
    }
    return WF_OK;
}

// Forward step from (u_in, p_in) into tape t with every intermediate kept.
// phases: 1 = stop after the momentum predictor, 2 = after the SIMPLE
// correction, 3 = the whole step.  Output state in t.uout / t.pout.
int record_step(wf_adjoint* a, Tape& t, const float* u_in, const float* p_in, int phases) {
    wf_solver* h = a->h;
    const Params& P = h->P;
    cudaStream_t st = a->st;
    const size_t N = a->N;
    const size_t v = 3 * N * sizeof(float), s = N * sizeof(float);
    WFA_CUDA(cudaMemcpyAsync(t.uT, u_in, v, cudaMemcpyDeviceToDevice, st));
    WFA_CUDA(cudaMemcpyAsync(t.p0, p_in, s, cudaMemcpyDeviceToDevice, st));
    wf::launch_vel_precompute(P, h->B, st, h->fl, t.uT, t.p0, h->eddy, h->face, nullptr, h->drag, t.D, t.b);
    wf::launch_vel_coef_ptr(P, st, h->fl, t.uT, h->eddy, h->face, t.D, t.A, t.iD);
    WFA_CUDA(cudaMemcpyAsync(V(a, t.uit, 0), t.uT, v, cudaMemcpyDeviceToDevice, st));
    for (int k = 0; k < a->nV; ++k)
        wf::launch_vel_sweep1_ptr(P, st, t.A, t.iD, t.b, V(a, t.uit, k), V(a, t.uit, k + 1));
    const float* ustar = V(a, t.uit, a->nV);
    WFA_CUDA(cudaMemcpyAsync(t.uout, ustar, v, cudaMemcpyDeviceToDevice, st));
    WFA_CUDA(cudaMemcpyAsync(t.pout, t.p0, s, cudaMemcpyDeviceToDevice, st));
    if (phases >= 2) {
        wf::launch_pres_precompute(P, h->B, st, h->fl, ustar, t.p0, t.D, t.iD, t.Dp, t.bp);
        wf::launch_pres_coef_ptr(P, st, h->fl, t.D, t.iD, t.c3);
        wf::launch_inv_ptr(P, st, h->fl, t.Dp, t.ainv);
        WFA_CUDA(cudaMemsetAsync(t.qit, 0, s, st));
        wf::launch_pres_stack(P, st, h->num_sms, t.c3, t.ainv, t.bp, t.qit, a->nP, true, tma_status(h));
        const float* q = S(a, t.qit, a->nP);
        WFA_CUDA(cudaMemsetAsync(t.cbuf, 0, v, st));
        wf::launch_apply_vel(P, st, h->fl, q, t.D, t.iD, V(a, t.cbuf, 0), t.uout);
        wf::launch_apply_pres(P, st, h->fl, q, t.pout);
    }
    if (phases >= 3) {
        for (int m = 0; m < a->nC; ++m) {
            WFA_CUDA(cudaMemsetAsync(V(a, t.aod, m), 0, v, st));
            WFA_CUDA(cudaMemsetAsync(V(a, t.cbuf, m + 1), 0, v, st));
            WFA_CUDA(cudaMemsetAsync(SIT(a, t, m, 0), 0, s, st));
            wf::launch_piso_aodu(P, st, h->fl, V(a, t.cbuf, m), t.uT, h->eddy, h->face, V(a, t.aod, m));
            wf::launch_piso_pre_ptr(P, st, h->fl, t.D, t.iD, V(a, t.aod, m), S(a, t.pai, m), S(a, t.prhs, m));
            wf::launch_pres_stack(P, st, h->num_sms, t.c3, S(a, t.pai, m), S(a, t.prhs, m), SIT(a, t, m, 0),
                                  a->nP, true, tma_status(h));
            const float* ss = SIT(a, t, m, a->nP);
            wf::launch_apply_pres(P, st, h->fl, ss, t.pout);
            wf::launch_piso_vel(P, st, h->fl, ss, t.D, t.iD, V(a, t.aod, m), V(a, t.cbuf, m + 1), t.uout);
        }
    }
    WFA_CUDA(cudaGetLastError());
    return WF_OK;
}

// Reversed pressure-type loop: on entry a->sb holds the adjoint of the final
// iterate; on exit a->rb holds the adjoint of the right-hand side, a->dgb the
// adjoint of the diagonal coefficient (1/ai), and a->c3b has the face
// coefficient adjoints added.  sstack: the loop's iterates s^0..s^n.
void reverse_pres_loop(wf_adjoint* a, const float* ai, const float* c3, const float* sstack) {
    const Params& P = a->h->P;
    cudaStream_t st = a->st;
    const dim3 g = wf::cgrd(P), bk = wf::cblk();
    const int n = a->nP;
    if (n == 0) {
        cudaMemsetAsync(a->rb, 0, a->N * sizeof(float), st);
        cudaMemsetAsync(a->dgb, 0, a->N * sizeof(float), st);
        return;
    }
    // slot j of a->Wp holds W^{n-j}
    wf::k_adj_pinit<<<wf::lin_blocks(a->N), 256, 0, st>>>((int)a->N, ai, a->sb, a->Wp);
    if (n > 1) wf::launch_pres_stack(P, st, a->h->num_sms, c3, ai, nullptr, a->Wp, n - 1, false, tma_status(a->h));
    if (wf::quad_ok(P, {ai, a->Wp, sstack, a->rb, a->dgb, a->c3b})) {
        const dim3 b4 = wf::cblk(), g4q((P.nx / 4 + b4.x - 1) / b4.x, (P.ny + b4.y - 1) / b4.y, (P.nz + b4.z - 1) / b4.z);
        wf::k_adj_pacc4<<<g4q, b4, 0, st>>>(P, n, ai, a->Wp, sstack, a->rb, a->dgb, a->c3b);
    } else {
        wf::k_adj_pacc<<<g, bk, 0, st>>>(P, n, ai, a->Wp, sstack, a->rb, a->dgb, a->c3b);
    }
}

// Reverse of record_step: on entry a->ub / a->pb hold the adjoints of
// (uout, pout); on exit they hold the adjoints of (uT, p0), and a->gb /
// a->dragb have the boundary-plane and drag adjoints added.
int adjoint_step(wf_adjoint* a, const Tape& t, int phases) {
    wf_solver* h = a->h;
    const Params& P = h->P;
    cudaStream_t st = a->st;
    const size_t N = a->N;
    const size_t v = 3 * N * sizeof(float), s = N * sizeof(float);
    const dim3 g = wf::cgrd(P), bk = wf::cblk();
    const wf::BndBar G = bnd_bar(a);
    WFA_CUDA(cudaMemsetAsync(a->uTb, 0, v, st));
    WFA_CUDA(cudaMemsetAsync(a->Db, 0, v, st));
    WFA_CUDA(cudaMemsetAsync(a->c3b, 0, v, st));
    WFA_CUDA(cudaMemcpyAsync(a->pb_in, a->pb, s, cudaMemcpyDeviceToDevice, st));
    if (phases >= 2) WFA_CUDA(cudaMemcpyAsync(a->cb, a->ub, v, cudaMemcpyDeviceToDevice, st));
    if (phases >= 3) {
        // a->cb: adjoint of the newest correction
        for (int m = a->nC - 1; m >= 0; --m) {
            WFA_CUDA(cudaMemsetAsync(a->ab, 0, v, st));
            WFA_CUDA(cudaMemsetAsync(a->sb, 0, s, st));
            const float* ss = SIT(a, t, m, a->nP);
            wf::k_adj_pvel<<<g, bk, 0, st>>>(P, h->fl, a->cb, ss, t.D, V(a, t.aod, m), a->ab, a->sb, a->Db);
            wf::k_add_masked<<<wf::lin_blocks(N), 256, 0, st>>>((int)N, h->fl, a->pb, a->sb);
            reverse_pres_loop(a, S(a, t.pai, m), t.c3, SIT(a, t, m, 0));
            wf::k_adj_pisopre<<<g, bk, 0, st>>>(P, h->fl, a->dgb, a->rb, t.D, V(a, t.aod, m), a->ab, a->Db);
            // adjoint of c_m: the velocity adjoint (u gains c_m) plus its use in AOD
            WFA_CUDA(cudaMemcpyAsync(a->cb2, a->ub, v, cudaMemcpyDeviceToDevice, st));
            wf::k_adj_aod<<<g, bk, 0, st>>>(P, h->fl, a->ab, V(a, t.cbuf, m), t.uT, a->cb2, a->uTb);
            std::swap(a->cb, a->cb2);
        }
    }
    if (phases >= 2) {
        const float* q = S(a, t.qit, a->nP);
        WFA_CUDA(cudaMemsetAsync(a->sb, 0, s, st));
        wf::k_adj_corr<<<g, bk, 0, st>>>(P, h->fl, a->cb, q, t.D, a->sb, a->Db);
        wf::k_add_masked<<<wf::lin_blocks(N), 256, 0, st>>>((int)N, h->fl, a->pb, a->sb);
        reverse_pres_loop(a, t.ainv, t.c3, t.qit);
        // a->rb: adjoint of bp; a->dgb: adjoint of Dp
        wf::k_adj_c3<<<g, bk, 0, st>>>(P, h->fl, a->c3b, t.D, a->Db);
        wf::k_adj_ppre<<<g, bk, 0, st>>>(P, G, h->fl, a->dgb, a->rb, t.p0, t.D, a->ub, a->pb_in, a->Db);
    }
    // momentum loop in reverse; a->ub is the adjoint of u*
    if (a->nV > 0) {
        const int n = a->nV;
        wf::k_adj_vtrans<<<g, bk, 0, st>>>(P, t.A, a->AT);
        wf::k_adj_vinit<<<wf::lin_blocks(3 * (long long)N), 256, 0, st>>>(3 * (long long)N, t.iD, a->ub,
                                                                           V(a, a->Wv, n));
        const bool v4 = n > 1 && wf::quad_ok(P, {a->AT, t.iD, V(a, a->Wv, n), V(a, a->Wv, n - 1)});
        const dim3 g4((P.nx / 4 + bk.x - 1) / bk.x, (P.ny + bk.y - 1) / bk.y, (P.nz + bk.z - 1) / bk.z);
        for (int k = n - 1; k >= 1; --k) {
            if (v4)
                wf::k_adj_vsweepT4<<<g4, bk, 0, st>>>(P, a->AT, t.iD, V(a, a->Wv, k + 1), V(a, a->Wv, k));
            else
                wf::k_adj_vsweepT<false><<<g, bk, 0, st>>>(P, a->AT, t.iD, V(a, a->Wv, k + 1), nullptr,
                                                          V(a, a->Wv, k));
        }
        wf::k_adj_vsweepT<true><<<g, bk, 0, st>>>(P, a->AT, t.iD, V(a, a->Wv, 1), a->ub, a->uTb);
        if (wf::quad_ok(P, {a->Wv, t.uit, a->bb, a->Db, a->uTb})) {
            const dim3 b4(32, 4, 1), g4q((P.nx / 4 + 31) / 32, (P.ny + 3) / 4, P.nz);
            wf::k_adj_vacc4<<<g4q, b4, 0, st>>>(P, n, a->Wv, t.uit, a->bb, a->Db, a->uTb);
        } else {
            wf::k_adj_vacc<<<g, bk, 0, st>>>(P, n, h->fl, a->Wv, t.uit, a->bb, a->Db, a->uTb);
        }
    } else {
        wf::k_axpy<<<wf::lin_blocks(3 * (long long)N), 256, 0, st>>>(3 * (long long)N, 1.f, a->ub, a->uTb);
        WFA_CUDA(cudaMemsetAsync(a->bb, 0, v, st));
    }
    wf::k_adj_pre<<<g, bk, 0, st>>>(P, h->B, G, h->fl, a->Db, a->bb, a->uTb, a->pb_in, a->dragb);
    WFA_CUDA(cudaMemcpyAsync(a->ub, a->uTb, v, cudaMemcpyDeviceToDevice, st));
    WFA_CUDA(cudaMemcpyAsync(a->pb, a->pb_in, s, cudaMemcpyDeviceToDevice, st));
    WFA_CUDA(cudaGetLastError());
    return WF_OK;
}

void free_adj(wf_adjoint* a) {
    float* ptrs[] = {a->ub, a->uTb, a->pb, a->pb_in, a->Db, a->bb, a->AT, a->Wv, a->Wp, a->c3b, a->cb, a->cb2,
                     a->ab, a->sb, a->rb, a->dgb, a->gb, a->dragb};
    for (float* p : ptrs)
        if (p) cudaFree(p);
    for (void* p : a->blocks) cudaFree(p);
    a->blocks.clear();
    a->tapes.clear();
    if (a->dJ) cudaFree(a->dJ);
    for (float* p : a->ck)
        if (p) cudaFree(p);
    a->ck.clear();
    if (a->st) cudaStreamDestroy(a->st);
}

}  // namespace

extern "C" {

int wf_adj_create(wf_solver* h, wf_adjoint** out) {
    if (!h || !out) return WF_ERR_INVALID_ARG;
    *out = nullptr;
    if (h->P.les) return WF_ERR_UNSUPPORTED;
    if (h->nonuniform) return WF_ERR_UNSUPPORTED;  // the uniform-grid step is differentiated
    if (h->cfg.calc_residual) return WF_ERR_UNSUPPORTED;  // early exits change the iteration counts
    if (h->cfg.compat_flags & WF_COMPAT_PISO_CONSISTENT) return WF_ERR_UNSUPPORTED;
    bool fixed_p = false;
    for (int f = 0; f < 6; ++f) fixed_p |= h->cfg.pres_bc[f] == WF_BND_FIXED_VALUE;
    if (!fixed_p) return WF_ERR_UNSUPPORTED;  // pressure normalisation not differentiated
    if (cudaSetDevice(h->device) != cudaSuccess) return WF_ERR_CUDA;
    auto* a = new (std::nothrow) wf_adjoint;
    if (!a) return WF_ERR_OOM;
    a->h = h;
    a->N = h->P.N;
    a->nV = h->cfg.vel_iters;
    a->nP = h->cfg.pres_iters;
    a->nC = h->cfg.solver_type == WF_SOLVER_PISO ? h->cfg.piso_correctors : 0;
    const size_t N = a->N, v = 3 * N * sizeof(float), s = N * sizeof(float);
    bool ok = cudaStreamCreateWithFlags(&a->st, cudaStreamNonBlocking) == cudaSuccess;
    auto al = [&](float** p, size_t bytes) {
        if (!ok) return;
        ok = cudaMalloc((void**)p, bytes) == cudaSuccess && cudaMemsetAsync(*p, 0, bytes, a->st) == cudaSuccess;
    };
    al(&a->ub, v); al(&a->uTb, v); al(&a->pb, s); al(&a->pb_in, s); al(&a->Db, v); al(&a->bb, v);
    al(&a->AT, 2 * v); al(&a->Wv, (size_t)(a->nV + 1) * v); al(&a->Wp, (size_t)(a->nP + 1) * s);
    al(&a->c3b, v); al(&a->cb, v); al(&a->cb2, v); al(&a->ab, v); al(&a->sb, s); al(&a->rb, s); al(&a->dgb, s);
    al(&a->gb, plane_floats(h->P) * sizeof(float));
    al(&a->dragb, s);
    if (ok) ok = cudaMalloc((void**)&a->dJ, sizeof(double)) == cudaSuccess;
    if (ok) ok = ensure_tapes(a, 1) == WF_OK;
    if (ok) ok = cudaStreamSynchronize(a->st) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        free_adj(a);
        delete a;
        return WF_ERR_OOM;
    }
    *out = a;
    return WF_OK;
}

int wf_adj_destroy(wf_adjoint* a) {
    if (!a) return WF_ERR_INVALID_ARG;
    cudaSetDevice(a->h->device);
    cudaStreamSynchronize(a->st);
    free_adj(a);
    delete a;
    return WF_OK;
}

const char* wf_adj_last_error(const wf_adjoint* a) { return a ? a->err.c_str() : "null adjoint"; }

int wf_adj_set_segment_policy(wf_adjoint* a, int shorten) {
    if (!a || (shorten != 0 && shorten != 1)) return WF_ERR_INVALID_ARG;
    a->shorten = shorten != 0;
    return WF_OK;
}

int wf_adj_set_max_tapes(wf_adjoint* a, int max_tapes) {
    if (!a || max_tapes < 0) return WF_ERR_INVALID_ARG;
    a->max_tapes = max_tapes;
    return WF_OK;
}

int wf_adj_step_vjp(wf_adjoint* a, int phases, const float* ubar_out, const float* pbar_out, float* ubar_in,
                    float* pbar_in, float* gbar_planes, float* dragbar) {
    if (!a || phases < 1 || phases > 3 || !ubar_out || !pbar_out || !ubar_in || !pbar_in)
        return WF_ERR_INVALID_ARG;
    wf_solver* h = a->h;
    WFA_CUDA(cudaSetDevice(h->device));
    WFA_CUDA(cudaStreamSynchronize(h->st));
    const size_t N = a->N, v = 3 * N * sizeof(float), s = N * sizeof(float);
    Tape& t = a->tapes[0];
    // the solver's current state is the step input
    int st = record_step(a, t, h->vb[h->iT], h->pr, phases);
    if (st != WF_OK) return st;
    WFA_CUDA(cudaMemcpyAsync(a->ub, ubar_out, v, cudaMemcpyHostToDevice, a->st));
    WFA_CUDA(cudaMemcpyAsync(a->pb, pbar_out, s, cudaMemcpyHostToDevice, a->st));
    WFA_CUDA(cudaMemsetAsync(a->gb, 0, plane_floats(h->P) * sizeof(float), a->st));
    WFA_CUDA(cudaMemsetAsync(a->dragb, 0, s, a->st));
    st = adjoint_step(a, t, phases);
    if (st != WF_OK) return st;
    WFA_CUDA(cudaMemcpyAsync(ubar_in, a->ub, v, cudaMemcpyDeviceToHost, a->st));
    WFA_CUDA(cudaMemcpyAsync(pbar_in, a->pb, s, cudaMemcpyDeviceToHost, a->st));
    if (gbar_planes)
        WFA_CUDA(cudaMemcpyAsync(gbar_planes, a->gb, plane_floats(h->P) * sizeof(float), cudaMemcpyDeviceToHost,
                                 a->st));
    if (dragbar) WFA_CUDA(cudaMemcpyAsync(dragbar, a->dragb, s, cudaMemcpyDeviceToHost, a->st));
    WFA_CUDA(cudaStreamSynchronize(a->st));
    return adj_check_waits(a);
}

int wf_adj_step_forward(wf_adjoint* a, int phases, float* u_out, float* p_out) {
    if (!a || phases < 1 || phases > 3 || !u_out || !p_out) return WF_ERR_INVALID_ARG;
    wf_solver* h = a->h;
    WFA_CUDA(cudaSetDevice(h->device));
    WFA_CUDA(cudaStreamSynchronize(h->st));
    Tape& t = a->tapes[0];
    const int st = record_step(a, t, h->vb[h->iT], h->pr, phases);
    if (st != WF_OK) return st;
    WFA_CUDA(cudaMemcpyAsync(u_out, t.uout, 3 * a->N * sizeof(float), cudaMemcpyDeviceToHost, a->st));
    WFA_CUDA(cudaMemcpyAsync(p_out, t.pout, a->N * sizeof(float), cudaMemcpyDeviceToHost, a->st));
    WFA_CUDA(cudaStreamSynchronize(a->st));
    return adj_check_waits(a);
}

int wf_adj_gradient(wf_adjoint* a, const wf_objective* obj, int n_steps, int checkpoint_every, int include_init,
                    double* J, double* dJ_dustar, double* dJ_dz0, float* dJ_ddrag, float* ms_forward,
                    float* ms_total) {
    if (!a || !obj || n_steps < 1 || checkpoint_every < 1) return WF_ERR_INVALID_ARG;
    wf_solver* h = a->h;
    const Params& P = h->P;
    const wf_config& c = h->cfg;
    if (obj->x0 < 0 || obj->x1 > P.nx || obj->x0 >= obj->x1 || obj->z0 < 0 || obj->z1 > P.nz || obj->z0 >= obj->z1 ||
        obj->y < 0 || obj->y >= P.ny || obj->window < 1 || obj->window > n_steps)
        return adj_fail(a, WF_ERR_INVALID_ARG, "objective region or window out of range");
    if (c.inflow_type != WF_INFLOW_LOG || !(c.inflow_ustar > 0.f))
        return adj_fail(a, WF_ERR_UNSUPPORTED, "inflow gradients need the log inflow with inflow_ustar > 0");
    WFA_CUDA(cudaSetDevice(h->device));
    WFA_CUDA(cudaStreamSynchronize(h->st));
    const size_t N = a->N, v = 3 * N * sizeof(float), s = N * sizeof(float);
    const int area = (obj->x1 - obj->x0) * (obj->z1 - obj->z0);
    const float w = 1.f / (float)(obj->window * area);
    const dim3 og((obj->x1 - obj->x0 + 31) / 32, (obj->z1 - obj->z0 + 7) / 8), ob(32, 8);
    // Step tapes are kept for as many steps as device memory holds (up to
    // max_tapes, and never more than the window).  The last R steps of the
    // window are taped during the forward pass itself and reversed without
    // recomputation; the first nf = n_steps - R steps run as the solver's own
    // step with checkpoints every C steps (state n for n % C == 0, n < nf),
    // and each of their segments is recomputed into tapes and reversed: all
    // at once when the segment's tapes fit, else its states are stored and
    // it is reversed in sub-blocks of as many tapes as fit (one more
    // recomputation per step).
    int C = std::min(checkpoint_every, n_steps);
    struct Scratch {
        cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
        float* states = nullptr;  // C states of 4N floats (sub-block mode)
        ~Scratch() {
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
            if (states) cudaFree(states);
        }
    } E;
    for (float* p : a->ck) cudaFree(p);
    a->ck.clear();
    const int cap = a->max_tapes > 0 ? std::min(n_steps, a->max_tapes) : n_steps;
    int T = std::min((int)a->tapes.size(), cap);
    if (T < cap) {
        // as many tapes as fit, keeping room for the checkpoints and the
        // segment states of the sub-block mode
        const size_t tape_bytes = tape_floats(a) * sizeof(float);
        const int nck_max = (n_steps + C - 1) / C;
        const size_t reserve = (size_t)(C + nck_max) * (v + s) + (size_t(1) << 30);
        while (T < cap) {
            size_t fr = 0, tot = 0;
            if (cudaMemGetInfo(&fr, &tot) != cudaSuccess || fr < tape_bytes + reserve) break;
            if (ensure_tapes(a, T + 1) != WF_OK) break;
            T = (int)a->tapes.size();
        }
        cudaGetLastError();
        if (T < 1) return adj_fail(a, WF_ERR_OOM, "no device memory for one step tape");
    }
    T = std::min(T, cap);
    const int R = T, nf = n_steps - R;
    // When a segment's tapes do not all fit, shorter segments (one more
    // checkpoint per T steps) recompute each step once; the sub-block mode
    // recomputes it twice.  Fall back to the sub-block mode when the extra
    // checkpoints do not fit.
    int nck = nf > 0 ? (nf + C - 1) / C : 0;
    if (a->shorten && nf > 0 && T < C) {
        const int nck_short = (nf + T - 1) / T;
        std::vector<float*> ck(nck_short, nullptr);
        bool ok = true;
        for (int i = 0; i < nck_short && ok; ++i) ok = cudaMalloc((void**)&ck[i], v + s) == cudaSuccess;
        if (ok) {
            C = T;
            nck = nck_short;
            a->ck = ck;
        } else {
            cudaGetLastError();
            for (float* p : ck) cudaFree(p);
        }
    }
    if (a->ck.empty()) {
        a->ck.assign(nck, nullptr);
        for (int i = 0; i < nck; ++i)
            if (cudaMalloc((void**)&a->ck[i], v + s) != cudaSuccess) {
                cudaGetLastError();
                return adj_fail(a, WF_ERR_OOM, "checkpoint memory");
            }
    }
    if (nf > 0 && T < C && cudaMalloc((void**)&E.states, (size_t)C * (v + s)) != cudaSuccess) {
        cudaGetLastError();
        return adj_fail(a, WF_ERR_OOM, "no device memory for the segment states: lower checkpoint_every");
    }
    for (cudaEvent_t& e : E.ev) WFA_CUDA(cudaEventCreate(&e));
    WFA_CUDA(cudaMemsetAsync(a->dJ, 0, sizeof(double), h->st));
    WFA_CUDA(cudaEventRecord(E.ev[0], h->st));
    // ---- forward: the solver's own (fast) step with checkpoints, then the
    // taped tail; the objective on the way
    for (int n = 0; n < nf; ++n) {
        if (n % C == 0) {
            WFA_CUDA(cudaMemcpyAsync(a->ck[n / C], h->vb[h->iT], v, cudaMemcpyDeviceToDevice, h->st));
            WFA_CUDA(cudaMemcpyAsync(a->ck[n / C] + 3 * N, h->pr, s, cudaMemcpyDeviceToDevice, h->st));
        }
        const int st = wf_step(h, 1, nullptr);
        if (st != WF_OK) return adj_fail(a, st, "forward step failed");
        if (n + 1 > n_steps - obj->window)
            wf::k_objective<<<og, ob, 0, h->st>>>(P, h->fl, obj->x0, obj->x1, obj->y, obj->z0, obj->z1, w,
                                                  h->vb[h->iT], nullptr, a->dJ);
    }
    WFA_CUDA(cudaStreamSynchronize(h->st));
    int rs = WF_OK;
    for (int j = 0; j < R; ++j) {
        const float* ui = j == 0 ? h->vb[h->iT] : a->tapes[j - 1].uout;
        const float* pi = j == 0 ? h->pr : a->tapes[j - 1].pout;
        rs = record_step(a, a->tapes[j], ui, pi, 3);
        if (rs != WF_OK) return rs;
        if (nf + j + 1 > n_steps - obj->window)
            wf::k_objective<<<og, ob, 0, a->st>>>(P, h->fl, obj->x0, obj->x1, obj->y, obj->z0, obj->z1, w,
                                                  a->tapes[j].uout, nullptr, a->dJ);
    }
    WFA_CUDA(cudaEventRecord(E.ev[1], a->st));
    if (R > 0) {
        // the solver ends at the window's last state, as after R more steps
        // (velFieldLastTime and velFieldLastIter take it; the pressure
        // corrections restart from zero)
        WFA_CUDA(cudaMemcpyAsync(h->vb[h->iT], a->tapes[R - 1].uout, v, cudaMemcpyDeviceToDevice, a->st));
        WFA_CUDA(cudaMemcpyAsync(h->pr, a->tapes[R - 1].pout, s, cudaMemcpyDeviceToDevice, a->st));
        for (int b = 0; b < 3; ++b) WFA_CUDA(cudaMemsetAsync(h->pcb[b], 0, s, a->st));
        h->iter_alias = true;
        h->pc_zero = true;
        h->step += R;
    }
    WFA_CUDA(cudaStreamSynchronize(a->st));
    // ---- reverse: the taped tail, then one segment at a time
    WFA_CUDA(cudaMemsetAsync(a->ub, 0, v, a->st));
    WFA_CUDA(cudaMemsetAsync(a->pb, 0, s, a->st));
    WFA_CUDA(cudaMemsetAsync(a->gb, 0, plane_floats(P) * sizeof(float), a->st));
    WFA_CUDA(cudaMemsetAsync(a->dragb, 0, s, a->st));
    for (int j = R - 1; j >= 0; --j) {
        const Tape& t = a->tapes[j];
        if (nf + j + 1 > n_steps - obj->window)
            wf::k_objective<<<og, ob, 0, a->st>>>(P, h->fl, obj->x0, obj->x1, obj->y, obj->z0, obj->z1, w, t.uout,
                                                  a->ub, nullptr);
        rs = adjoint_step(a, t, 3);
        if (rs != WF_OK) return rs;
    }
    for (int sgi = nck - 1; sgi >= 0; --sgi) {
        const int n0 = sgi * C, n1 = std::min(nf, n0 + C), L = n1 - n0;
        // state j of the segment (state n0 + j): from the checkpoint, or
        // from the stored segment states in sub-block mode
        auto state = [&](int j) -> float* { return j == 0 ? a->ck[sgi] : E.states + (size_t)j * 4 * N; };
        if (L > T) {
            for (int j = 1; j < L; ++j) {
                rs = record_step(a, a->tapes[0], state(j - 1), state(j - 1) + 3 * N, 3);
                if (rs != WF_OK) return rs;
                WFA_CUDA(cudaMemcpyAsync(state(j), a->tapes[0].uout, v, cudaMemcpyDeviceToDevice, a->st));
                WFA_CUDA(cudaMemcpyAsync(state(j) + 3 * N, a->tapes[0].pout, s, cudaMemcpyDeviceToDevice, a->st));
            }
        }
        for (int hi = L; hi > 0;) {
            const int lo = std::max(0, hi - T);
            for (int j = lo; j < hi; ++j) {
                Tape& t = a->tapes[j - lo];
                const float* ui = j == lo ? state(lo) : a->tapes[j - lo - 1].uout;
                const float* pi = j == lo ? state(lo) + 3 * N : a->tapes[j - lo - 1].pout;
                rs = record_step(a, t, ui, pi, 3);
                if (rs != WF_OK) return rs;
            }
            for (int j = hi - 1; j >= lo; --j) {
                // step n0 + j maps state n0 + j to state n0 + j + 1
                const Tape& t = a->tapes[j - lo];
                if (n0 + j + 1 > n_steps - obj->window)
                    wf::k_objective<<<og, ob, 0, a->st>>>(P, h->fl, obj->x0, obj->x1, obj->y, obj->z0, obj->z1, w,
                                                          t.uout, a->ub, nullptr);
                rs = adjoint_step(a, t, 3);
                if (rs != WF_OK) return rs;
            }
            hi = lo;
        }
    }
    WFA_CUDA(cudaEventRecord(E.ev[2], a->st));
    WFA_CUDA(cudaStreamSynchronize(a->st));
    if (const int w = adj_check_waits(a)) return w;
    // ---- chain to the inflow parameters: X0 plane g_x(y) = u*/k ln((y_c+z0)/z0)
    const int np = P.plane[WF_FACE_X0];
    std::vector<float> gx(np);
    WFA_CUDA(cudaMemcpy(gx.data(), a->gb, np * sizeof(float), cudaMemcpyDeviceToHost));  // x component of X0
    const double us = c.inflow_ustar, z0 = c.inflow_z0, kap = c.inflow_kappa, dx = c.dx;
    double gu = 0.0, gz = 0.0;
    for (int z = 0; z < P.nz; ++z)
        for (int y = 0; y < P.ny; ++y) {
            const double yc = (y + 0.5) * dx;
            const double gb = gx[(size_t)z * P.ny + y];
            gu += gb * std::log((yc + z0) / z0) / kap;
            gz += gb * us / kap * (1.0 / (yc + z0) - 1.0 / z0);
        }
    if (include_init) {
        // initial interior profile u_x(y) = u*/k ln((y_p + z0)/z0) on fluid cells
        std::vector<float> ubar(3 * N);
        std::vector<uint8_t> flg(N);
        WFA_CUDA(cudaMemcpy(ubar.data(), a->ub, 3 * N * sizeof(float), cudaMemcpyDeviceToHost));
        WFA_CUDA(cudaMemcpy(flg.data(), h->fl, N, cudaMemcpyDeviceToHost));
        const bool centre = (c.compat_flags & WF_COMPAT_INIT_PROFILE_CELL_CENTRE) != 0;
        for (int z = 0; z < P.nz; ++z)
            for (int y = 0; y < P.ny; ++y) {
                const double yp = centre ? (y + 0.5) * dx : y * dx;
                const double du = std::log((yp + z0) / z0) / kap;
                const double dz = us / kap * (1.0 / (yp + z0) - 1.0 / z0);
                for (int x = 0; x < P.nx; ++x) {
                    const size_t i = ((size_t)z * P.ny + y) * P.nx + x;
                    if (flg[i] != WF_CELL_FLUID) continue;
                    gu += ubar[i] * du;
                    gz += ubar[i] * dz;
                }
            }
    }
    if (dJ_ddrag) WFA_CUDA(cudaMemcpy(dJ_ddrag, a->dragb, s, cudaMemcpyDeviceToHost));
    double Jh = 0.0;
    WFA_CUDA(cudaMemcpy(&Jh, a->dJ, sizeof(double), cudaMemcpyDeviceToHost));
    if (J) *J = Jh;
    if (dJ_dustar) *dJ_dustar = gu;
    if (dJ_dz0) *dJ_dz0 = gz;
    float tf = 0.f, tt = 0.f;
    WFA_CUDA(cudaEventElapsedTime(&tf, E.ev[0], E.ev[1]));
    WFA_CUDA(cudaEventElapsedTime(&tt, E.ev[0], E.ev[2]));
    if (ms_forward) *ms_forward = tf;
    if (ms_total) *ms_total = tt;
    return WF_OK;
}

}  // extern "C"
