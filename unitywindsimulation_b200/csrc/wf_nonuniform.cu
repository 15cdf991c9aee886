// wf_nonuniform.cu - the non-uniform collocated grid (the reference's gridType
// CollNonUniform): FvmCollNonUniform.compute's SIMPLE kernels and the two
// mesh-aware set-up kernels of InitShaderColl.compute, one thread per cell;
// the momentum sweeps are the uniform grid's (wf_sweeps.cu) over the
// coefficient planes the non-uniform pre-compute stores.
//
// The mesh is given by face positions along each axis (facePosX/Y/Z,
// FvmSolverGpu.cs:682-788): cell x spans fx[x]..fx[x+1].  Every kernel
// derives its spacings, interpolation weights and face areas from them with
// the reference's own expressions and operand order.  The face fluxes the
// pressure pre-compute writes (velFaceFluxField, (nx+1)(ny+1)(nz+1) texels,
// three SoA planes here) feed the next momentum pre-compute and sweeps: the
// reference leaves that texture unbound for those two kernels
// (FvmSolverGpu.cs:1160,1196 are commented out); this library binds it, the
// intended data flow.  SIMPLE runs on this grid, with or without the
// Smagorinsky model: as in the reference, the wall function and the LES
// kernels run with the constant dx (Les and WallFunc have no non-uniform
// form) and the momentum kernels interpolate the eddy viscosity to the faces
// with the mesh weights (useLES).  The reference has no PISO shader for this
// grid (FvmSolverGpu.cs:493-496 throws), so PISO is refused here too.
#include <cuda_runtime.h>

#include <cmath>

#include "wf_common.cuh"
#include "wf_kernels.cuh"
#include "wf_solver.cuh"

namespace wf {

namespace {

__device__ __forceinline__ float ldn(const float* p, size_t i) { return __ldg(p + i); }

// Pressure coefficient planes (N floats each) the pressure pre-compute
// stores for the sweeps: face coefficients ((dv / den) DInv) / h, zero at
// faces without a fluid neighbour, and 1/Dp.
constexpr int kCoefP = 0, kCoefInvDp = 6;
static_assert(kCoefInvDp + 1 == kNuCoefPlanes, "plane count");

// Spacing of cell i along one axis and of its neighbours; a neighbour
// outside the domain takes the cell's own spacing (FvmCollNonUniform.compute:
// 130-142, 954-977 for the second neighbours).
struct Axis {
    float d, dp, dm, dpp, dmm;
};
__device__ __forceinline__ Axis axis_of(const float* f, int i, int n) {
    Axis a;
    a.d = ldn(f, i + 1) - ldn(f, i);
    a.dp = i + 1 < n ? ldn(f, i + 2) - ldn(f, i + 1) : a.d;
    a.dm = i > 0 ? ldn(f, i) - ldn(f, i - 1) : a.d;
    a.dpp = i + 2 < n ? ldn(f, i + 3) - ldn(f, i + 2) : a.d;
    a.dmm = i > 1 ? ldn(f, i - 1) - ldn(f, i - 2) : a.d;
    return a;
}

struct Geo {
    Axis a[3];
    float ds[3];  // dsx = dy dz, dsy = dx dz, dsz = dx dy
    float dv;
};
__device__ __forceinline__ Geo geo_of(const Params& P, const float* fx, const float* fy, const float* fz, int x,
                                      int y, int z) {
    Geo g;
    g.a[0] = axis_of(fx, x, P.nx);
    g.a[1] = axis_of(fy, y, P.ny);
    g.a[2] = axis_of(fz, z, P.nz);
    const float dx = g.a[0].d, dy = g.a[1].d, dz = g.a[2].d;
    g.ds[0] = dy * dz;
    g.ds[1] = dx * dz;
    g.ds[2] = dx * dy;
    g.dv = dx * dy * dz;
    return g;
}
// Interpolation weight of the cell itself at face f (wPe = dxE / (dx + dxE)
// and the like, :146-168).
__device__ __forceinline__ float w_self(const Geo& g, int f) {
    const Axis& a = g.a[face_axis(f)];
    const float dq = face_sign(f) > 0 ? a.dp : a.dm;
    return dq / (a.d + dq);
}
// Centre distance across face f (0.5 d + 0.5 d_neighbour).
__device__ __forceinline__ float h_face(const Geo& g, int f) {
    const Axis& a = g.a[face_axis(f)];
    return 0.5f * a.d + 0.5f * (face_sign(f) > 0 ? a.dp : a.dm);
}

struct Flux {
    const float* p;
    int sx, sy, sxy;  // texels per row (nx + 1), rows per plane (ny + 1), per plane
    size_t n;         // texels per component plane, (nx + 1)(ny + 1)(nz + 1)
};
__device__ __forceinline__ Flux flux_of(const Params& P, const float* p) {
    Flux F;
    F.p = p;
    F.sx = P.nx + 1;
    F.sy = P.ny + 1;
    F.sxy = F.sx * F.sy;
    F.n = (size_t)F.sxy * (P.nz + 1);
    return F;
}
__device__ __forceinline__ int tex(const Flux& F, int x, int y, int z) { return (z * F.sy + y) * F.sx + x; }
// Face flux of face f of cell (x, y, z): the texel of the cell itself for
// the W/S/D faces, of the neighbour for the E/N/U faces.
__device__ __forceinline__ float face_flux(const Flux& F, int x, int y, int z, int f) {
    const int a = face_axis(f);
    const int t = face_sign(f) > 0 ? tex(F, x + face_ox(f), y + face_oy(f), z + face_oz(f)) : tex(F, x, y, z);
    return ldn(F.p, (size_t)a * F.n + t);
}

__device__ __forceinline__ bool fluid_cell(const uint8_t* fl, int i) { return __ldg(fl + i) == WF_CELL_FLUID; }
// Fluid cell two cells away across face f, inside the domain
// (InRegionAndIsFluid(EE) and the like, :1011-1018).
__device__ __forceinline__ bool fluid_far(const Params& P, const uint8_t* fl, int x, int y, int z, int f) {
    const int X = x + 2 * face_ox(f), Y = y + 2 * face_oy(f), Z = z + 2 * face_oz(f);
    return in_region(P, X, Y, Z) && fluid_cell(fl, cidx(P, X, Y, Z));
}

// Face viscosities of the non-uniform momentum kernels (FvmCollNonUniform.
// compute:483-505 and 846-868): nu without LES (eddy == nullptr); with LES
// nu + nu_t,P, and across a face to a fluid neighbour nu + wP nu_t,P + wQ
// nu_t,Q with the mesh's interpolation weights (wQ = 1 - wP).
__device__ __forceinline__ void nu_face_vis(const Params& P, const Geo& g, unsigned m, const float* eddy, int i,
                                            float vis[6]) {
    if (!eddy) {
#pragma unroll
        for (int f = 0; f < 6; ++f) vis[f] = P.nu;
        return;
    }
    const float eP = ldn(eddy, i);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        vis[f] = P.nu + eP;
        if (nb_fluid(m, f)) {
            const float wP = w_self(g, f), wQ = 1.0f - wP;
            vis[f] = P.nu + wP * eP + wQ * ldn(eddy, i + face_off(P, f));
        }
    }
}

// CSVelPredictPreCompute, FvmCollNonUniform.compute:111-721.
// Besides D and b it stores the sweep's coefficients for the step: per
// fluid-neighbour face A_f = (nu ds) / h -+ (ds w_neighbour) F_f (the
// diffusion and advection factors CSVelPredict multiplies u_neighbour by,
// :797-907) and 1/D, in the layout of the uniform grid's momentum sweep
// (A: 6 planes, 1/D: 3 planes; zero on non-fluid cells), so the same
// four-cells-per-thread sweep runs on both grids.  Summing A_f u rather
// than the advection and diffusion sums apart reorders the additions: the
// fields agree with the reference's kernels within FP32 rounding.
__global__ void k_nu_vel_precompute(const __grid_constant__ Params P, const Bnd B, const float* __restrict__ fx,
                                    const float* __restrict__ fy, const float* __restrict__ fz,
                                    const uint8_t* __restrict__ fl, const float* __restrict__ uT,
                                    const float* __restrict__ pr, const float* __restrict__ flux,
                                    const float* __restrict__ eddy, float* __restrict__ Dv,
                                    float* __restrict__ bv, float* __restrict__ A, float* __restrict__ iD) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    if (!fluid_cell(fl, i)) {
#pragma unroll
        for (int f = 0; f < 6; ++f) A[f * N + i] = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) iD[k * N + i] = 0.f;
        return;
    }
    const unsigned m = __ldg(P.nbm + i);
    const Geo g = geo_of(P, fx, fy, fz, x, y, z);
    const Flux F = flux_of(P, flux);
    const float dvdt = g.dv / P.dt;
    float D[3] = {dvdt, dvdt, dvdt};
    float b[3] = {0.f, 0.f, 0.f};
    // advection with the last face fluxes, :200-335
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const bool pos = face_sign(f) > 0;
        if (nb_fluid(m, f)) {
            const float t = g.ds[a] * w_self(g, f) * face_flux(F, x, y, z, f);
#pragma unroll
            for (int k = 0; k < 3; ++k) D[k] = pos ? D[k] + t : D[k] - t;
        } else if (!face_in(P, x, y, z, f)) {
            const int bc = face_bc(f), bt = P.vbc[bc];
            const float Fv = face_flux(F, x, y, z, f);
            if (bt == WF_BND_FIXED_VALUE) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float t = g.ds[a] * bnd_comp(P, B, bc, x, y, z, k) * Fv;
                    b[k] = pos ? b[k] - t : b[k] + t;
                }
            } else if (bt == WF_BND_ZERO_GRAD) {
                const float t = g.ds[a] * Fv;
#pragma unroll
                for (int k = 0; k < 3; ++k) D[k] = pos ? D[k] + t : D[k] - t;
            }
        }
    }
    // pressure, :337-466
    const float pP = ldn(pr, i);
    float pf[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (face_in(P, x, y, z, f)) {
            if (nb_fluid(m, f)) {
                const float wP = w_self(g, f), wQ = 1.0f - wP;
                pf[f] = wP * pP + wQ * ldn(pr, i + face_off(P, f));
            } else {
                pf[f] = pP;
            }
        } else {
            pf[f] = P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE ? 0.f : pP;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) b[a] += -(1.0f / P.den) * g.ds[a] * (pf[2 * a] - pf[2 * a + 1]);
    // diffusion with the face viscosities, :468-697
    float visf[6];
    nu_face_vis(P, g, m, eddy, i, visf);
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const float vis = visf[f];
        if (face_in(P, x, y, z, f)) {
            const float t = nb_fluid(m, f) ? vis * g.ds[a] / h_face(g, f) : vis * g.ds[a] / (0.5f * g.a[a].d);
#pragma unroll
            for (int k = 0; k < 3; ++k) D[k] += t;
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            const float t = vis * g.ds[a] / (0.5f * g.a[a].d);
            if (bt == WF_BND_FIXED_VALUE) {
#pragma unroll
                for (int k = 0; k < 3; ++k) b[k] += t * bnd_comp(P, B, bc, x, y, z, k);
#pragma unroll
                for (int k = 0; k < 3; ++k) D[k] += t;
            } else if (bt == WF_BND_SYMMETRY) {
                D[a] += t;
            }
        }
    }
    // time and force, :699-710
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] += g.dv / P.dt * ldn(uT, k * N + i);
#pragma unroll
    for (int k = 0; k < 3; ++k) b[k] += g.dv * P.force[k];
    // LES deferred-correction term the LES kernel left in bField, :712-717
    if (eddy) {
#pragma unroll
        for (int k = 0; k < 3; ++k) b[k] += ldn(bv, k * N + i);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Dv[k * N + i] = D[k];
        bv[k * N + i] = b[k];
    }
    // sweep coefficients (FvmCollNonUniform.compute:797-842 and 844-907
    // evaluate them inline in every sweep)
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        float c = 0.f;
        if (nb_fluid(m, f)) {
            const int a = face_axis(f);
            const float adv = g.ds[a] * (1.0f - w_self(g, f)) * face_flux(F, x, y, z, f);
            const float dif = visf[f] * g.ds[a] / h_face(g, f);
            c = face_sign(f) > 0 ? dif - adv : dif + adv;
        }
        A[f * N + i] = c;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) iD[k * N + i] = 1.0f / D[k];
}

// One thread per cell over a 1-D grid (no idle threads at the x edge of a
// non-multiple-of-32 grid); every load leaves before the fluid test.
__device__ __forceinline__ bool linear_cell(const Params& P, int& x, int& y, int& z, int& i) {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.N) return false;
    x = i % P.nx;
    const int r = i / P.nx;
    y = r % P.ny;
    z = r / P.ny;
    return true;
}

// Rhie-Chow average of the pressure gradient at face f
// (FvmCollNonUniform.compute:1011-1020 for E and the like for the others).
__device__ __forceinline__ float grad_ave(const Params& P, const uint8_t* fl, const float* pr, const Geo& g, int x,
                                          int y, int z, int i, unsigned m, int f, float pP, float pQ, float grad) {
    const Axis& a = g.a[face_axis(f)];
    const int o = face_off(P, f);
    const int fr = f ^ 1;  // the opposite face
    const bool fqq = fluid_far(P, fl, x, y, z, f), frr = nb_fluid(m, fr);
    if (face_sign(f) > 0) {  // E, N, U: Q = +1, QQ = +2, R = -1
        const float h = a.d, hQ = a.dp, hQQ = a.dpp, hR = a.dm;
        if (fqq && frr) {
            const float pQQ = ldn(pr, i + 2 * o), pR = ldn(pr, i - o);
            return 0.5f * ((pQQ - pP) / (0.5f * hQQ + hQ + 0.5f * h) + (pQ - pR) / (0.5f * hQ + h + 0.5f * hR));
        }
        if (fqq) {
            const float pQQ = ldn(pr, i + 2 * o);
            return 0.5f * ((pQQ - pP) / (0.5f * hQQ + hQ + 0.5f * h) + (pQ - pP) / (0.5f * hQ + 1.5f * h));
        }
        if (frr) {
            const float pR = ldn(pr, i - o);
            return 0.5f * ((pQ - pP) / (1.5f * hQ + 0.5f * h) + (pQ - pR) / (0.5f * hQ + h + 0.5f * hR));
        }
        return grad;
    }
    // W, S, D: Q = -1, QQ = -2, R = +1
    const float h = a.d, hQ = a.dm, hQQ = a.dmm, hR = a.dp;
    if (fqq && frr) {
        const float pQQ = ldn(pr, i + 2 * o), pR = ldn(pr, i - o);
        return 0.5f * ((pR - pQ) / (0.5f * hR + h + 0.5f * hQ) + (pP - pQQ) / (0.5f * h + hQ + 0.5f * hQQ));
    }
    if (fqq) {
        const float pQQ = ldn(pr, i + 2 * o);
        return 0.5f * ((pP - pQ) / (1.5f * h + 0.5f * hQ) + (pP - pQQ) / (0.5f * h + hQ + 0.5f * hQQ));
    }
    if (frr) {
        const float pR = ldn(pr, i - o);
        return 0.5f * ((pR - pQ) / (0.5f * hR + h + 0.5f * hQ) + (pP - pQ) / (0.5f * h + 1.5f * hQ));
    }
    return grad;
}

// CSPresCorrectRhieChowPreCompute, FvmCollNonUniform.compute:920-1344:
// Dp, bp and the face fluxes (written to the W/S/D texels of the cell, and
// to the E/N/U texels beyond the domain).
__global__ void k_nu_pres_precompute(const __grid_constant__ Params P, const Bnd B, const float* __restrict__ fx,
                                     const float* __restrict__ fy, const float* __restrict__ fz,
                                     const uint8_t* __restrict__ fl, const float* __restrict__ u,
                                     const float* __restrict__ pr, const float* __restrict__ Dv,
                                     float* __restrict__ flux, float* __restrict__ Dp, float* __restrict__ bp,
                                     float* __restrict__ coef) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    if (!fluid_cell(fl, i)) return;
    const size_t N = P.N;
    const unsigned m = __ldg(P.nbm + i);
    const Geo g = geo_of(P, fx, fy, fz, x, y, z);
    const float pP = ldn(pr, i);
    float dp = 0.f, b = 0.f;
    float uf[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float cf[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int a = face_axis(f);
        const bool pos = face_sign(f) > 0;
        if (face_in(P, x, y, z, f)) {
            if (!nb_fluid(m, f)) continue;  // solid neighbour: no flux
            const int q = i + face_off(P, f);
            const float wP = w_self(g, f), wQ = 1.0f - wP;
            const float DInv = wP * (1.0f / ldn(Dv, a * N + i)) + wQ * (1.0f / ldn(Dv, a * N + q));
            const float h2 = h_face(g, f);
            // the sweeps' face coefficient (CSPresCorrectRhieChow evaluates
            // the same expression, FvmCollNonUniform.compute:1398-1449)
            cf[f] = (g.dv / P.den) * DInv / h2;
            dp -= cf[f];
            float v = wP * ldn(u, a * N + i) + wQ * ldn(u, a * N + q);
            const float pQ = ldn(pr, q);
            const float grad = pos ? (pQ - pP) / h2 : (pP - pQ) / h2;
            const float ave = grad_ave(P, fl, pr, g, x, y, z, i, m, f, pP, pQ, grad);
            v -= (g.dv * DInv) / P.den * (grad - ave);
            uf[f] = v;
            b = pos ? b + v : b - v;
        } else {
            const int bc = face_bc(f), bt = P.vbc[bc];
            if (bt == WF_BND_FIXED_VALUE) {
                const float v = bnd_comp(P, B, bc, x, y, z, a);
                uf[f] = v;
                b = pos ? b + v : b - v;
            } else if (bt == WF_BND_ZERO_GRAD) {
                const float v = ldn(u, a * N + i);
                uf[f] = v;
                b = pos ? b + v : b - v;
            }
            if (P.pbc[bc] == WF_BND_FIXED_VALUE) {
                const float DInv = 1.0f / ldn(Dv, a * N + i);
                dp -= (g.dv / P.den) * DInv / (0.5f * g.a[a].d);
            }
        }
    }
    const Flux F = flux_of(P, flux);
    float* fo = flux;
    const int t = tex(F, x, y, z);
    fo[t] = uf[1];
    fo[F.n + t] = uf[3];
    fo[2 * F.n + t] = uf[5];
    if (x + 1 == P.nx) {
        const int te = tex(F, x + 1, y, z);
        fo[te] = uf[0];
        fo[F.n + te] = 0.f;
        fo[2 * F.n + te] = 0.f;
    }
    if (y + 1 == P.ny) {
        const int tn = tex(F, x, y + 1, z);
        fo[tn] = 0.f;
        fo[F.n + tn] = uf[2];
        fo[2 * F.n + tn] = 0.f;
    }
    if (z + 1 == P.nz) {
        const int tu = tex(F, x, y, z + 1);
        fo[tu] = 0.f;
        fo[F.n + tu] = 0.f;
        fo[2 * F.n + tu] = uf[4];
    }
    Dp[i] = dp;
    bp[i] = b;
#pragma unroll
    for (int f = 0; f < 6; ++f) coef[(kCoefP + f) * N + i] = cf[f];
    coef[kCoefInvDp * N + i] = 1.0f / dp;
}

// CSPresCorrectRhieChow, FvmCollNonUniform.compute:1346-1452, with the
// step's face coefficients: p' = (1/Dp) (-sum_f c_f p'_Q + bp).  pin null:
// the previous iterate is zero.
__global__ void __launch_bounds__(256) k_nu_pres_sweep(const __grid_constant__ Params P,
                                                       const float* __restrict__ pin,
                                                       const float* __restrict__ coef,
                                                       const float* __restrict__ bp, float* __restrict__ pout) {
    chain_wait();
    chain_release();
    int x, y, z, i;
    if (!linear_cell(P, x, y, z, i)) return;
    const size_t N = P.N;
    const unsigned m = __ldg(P.nbm + i);
    float pq[6], c[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        pq[f] = pin ? ldn(pin, nb_idx(P, x, y, z, i, f)) : 0.f;
        c[f] = ldn(coef, (kCoefP + f) * N + i);
    }
    const float inv = ldn(coef, kCoefInvDp * N + i), b = ldn(bp, i);
    if (!(m & 64u)) return;
    float term = 0.f;
#pragma unroll
    for (int f = 0; f < 6; ++f)
        if (nb_fluid(m, f)) term -= c[f] * pq[f];
    pout[i] = inv * (term + b);
}

// k_nu_pres_sweep with four x-consecutive cells per thread (nx % 4 == 0,
// 16-byte aligned planes): 128-bit loads of the coefficient planes, the
// iterate and its y/z neighbours, two scalar loads for the x neighbours
// beyond the four cells; the same arithmetic per cell.
__device__ __forceinline__ float4 ld4n(const float* p, size_t i) {
    return __ldg(reinterpret_cast<const float4*>(p + i));
}
__device__ __forceinline__ float c4(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }

// The per-step inputs of four cells' pressure updates: neighbour masks,
// face coefficients, 1/Dp and bp.
struct NuPresCoef {
    uchar4 mq;
    float4 c[6], inv, b;
};
__device__ __forceinline__ NuPresCoef nu_pres_coef(const Params& P, const float* coef, const float* bp, int i) {
    const size_t N = P.N;
    NuPresCoef k;
    k.mq = __ldg(reinterpret_cast<const uchar4*>(P.nbm + i));
#pragma unroll
    for (int f = 0; f < 6; ++f) k.c[f] = ld4n(coef, (kCoefP + f) * N + i);
    k.inv = ld4n(coef, kCoefInvDp * N + i);
    k.b = ld4n(bp, i);
    return k;
}

__global__ void __launch_bounds__(256) k_nu_pres_sweep4(const __grid_constant__ Params P,
                                                        const float* __restrict__ pin,
                                                        const float* __restrict__ coef,
                                                        const float* __restrict__ bp, float* __restrict__ pout,
                                                        int pre) {
    // pre: the coefficient planes, bp and the masks were written before the
    // previous grid of the chain (every sweep after the first): they load
    // before chain_wait.
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = q < P.N / 4;
    const int i = in ? 4 * q : 0;
    NuPresCoef k{};
    if (pre && in) k = nu_pres_coef(P, coef, bp, i);
    chain_wait();
    chain_release();
    if (!in) return;
    if (!pre) k = nu_pres_coef(P, coef, bp, i);
    const uchar4 mq = k.mq;
    const float4* c = k.c;
    const float4 inv = k.inv, b = k.b;
    const int x0 = i % P.nx, r = i / P.nx, y = r % P.ny, z = r / P.ny;
    const int sx = P.nx, sz = P.nx * P.ny;
    const int iN = y + 1 < P.ny ? i + sx : i, iS = y > 0 ? i - sx : i;
    const int iU = z + 1 < P.nz ? i + sz : i, iDn = z > 0 ? i - sz : i;
    const int iE = x0 + 4 < P.nx ? i + 4 : i + 3, iW = x0 > 0 ? i - 1 : i;
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 pc = pin ? ld4n(pin, i) : z4, pn = pin ? ld4n(pin, iN) : z4, ps = pin ? ld4n(pin, iS) : z4;
    const float4 pu = pin ? ld4n(pin, iU) : z4, pd = pin ? ld4n(pin, iDn) : z4;
    const float pe3 = pin ? __ldg(pin + iE) : 0.f, pw0 = pin ? __ldg(pin + iW) : 0.f;
    const unsigned ms[4] = {mq.x, mq.y, mq.z, mq.w};
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const unsigned m = ms[j];
        const float pq[6] = {j < 3 ? c4(pc, j + 1) : pe3, j > 0 ? c4(pc, j - 1) : pw0, c4(pn, j), c4(ps, j),
                             c4(pu, j), c4(pd, j)};
        float term = 0.f;
#pragma unroll
        for (int f = 0; f < 6; ++f)
            if (nb_fluid(m, f)) term -= c4(c[f], j) * pq[f];
        v[j] = c4(inv, j) * (term + c4(b, j));
    }
    const bool all = (ms[0] & ms[1] & ms[2] & ms[3] & 64u) != 0;
    if (all) {
        *reinterpret_cast<float4*>(pout + i) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (ms[j] & 64u) pout[i + j] = v[j];
    }
}

// CSApplyVelCorrectionDivergenceTheorem, FvmCollNonUniform.compute:1487-1731.
// pc null: the correction field is zero.
__global__ void k_nu_apply_vel(const __grid_constant__ Params P, const float* __restrict__ fx,
                               const float* __restrict__ fy, const float* __restrict__ fz,
                               const uint8_t* __restrict__ fl, const float* __restrict__ pc,
                               const float* __restrict__ Dv, float* __restrict__ uc, float* __restrict__ u) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    if (!fluid_cell(fl, i)) return;
    const size_t N = P.N;
    const unsigned m = __ldg(P.nbm + i);
    const Geo g = geo_of(P, fx, fy, fz, x, y, z);
    const float cP = pc ? ldn(pc, i) : 0.f;
    float pf[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (face_in(P, x, y, z, f)) {
            if (nb_fluid(m, f)) {
                const float wP = w_self(g, f), wQ = 1.0f - wP;
                const float cQ = pc ? ldn(pc, i + face_off(P, f)) : 0.f;
                pf[f] = wP * cP + wQ * cQ;
            } else {
                pf[f] = cP;
            }
        } else {
            pf[f] = P.pbc[face_bc(f)] == WF_BND_FIXED_VALUE ? 0.f : cP;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float D = ldn(Dv, a * N + i);
        const float c = -(g.dv / P.den) * (1.0f / D) * (pf[2 * a] - pf[2 * a + 1]) / g.a[a].d;
        uc[a * N + i] = c;
        u[a * N + i] += c;
    }
}

// CSInitLogVelPresFieldsNonUniform, InitShaderColl.compute:134-154: the log
// profile at the cell-centre height 0.5 (fy[y] + fy[y+1]).
__global__ void k_nu_init_log(const __grid_constant__ Params P, const float* __restrict__ fy, float fric,
                              float kappa, float z0, float* u0, float* u1, float* u2, float* uc, float* pr) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const int i = cidx(P, x, y, z);
    const size_t N = P.N;
    const float yPhys = 0.5f * (ldn(fy, y) + ldn(fy, y + 1));
    const float vx = fric / kappa * logf((yPhys + z0) / z0);
    float* bufs[3] = {u0, u1, u2};
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        bufs[b][i] = vx;
        bufs[b][N + i] = 0.f;
        bufs[b][2 * N + i] = 0.f;
    }
    uc[i] = 0.f;
    uc[N + i] = 0.f;
    uc[2 * N + i] = 0.f;
    pr[i] = 0.f;
}

// CSSetLogVelBndCondNonUniform, InitShaderColl.compute:287-300.
__global__ void k_nu_log_inlet(int ny, int nz, const float* __restrict__ fy, float fric, float kappa, float z0,
                               float* x0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = ny * nz;
    if (i >= n) return;
    const int y = i % ny;
    const float yPhys = 0.5f * (ldn(fy, y) + ldn(fy, y + 1));
    x0[i] = fric / kappa * logf((yPhys + z0) / z0);
    x0[n + i] = 0.f;
    x0[2 * n + i] = 0.f;
}

dim3 nu_block() { return dim3(32, 4, 2); }
dim3 nu_grid(const Params& P) {
    const dim3 b = nu_block();
    return dim3((P.nx + b.x - 1) / b.x, (P.ny + b.y - 1) / b.y, (P.nz + b.z - 1) / b.z);
}

}  // namespace

size_t nu_flux_texels(const Params& P) { return (size_t)(P.nx + 1) * (P.ny + 1) * (P.nz + 1); }

void launch_nu_vel_precompute(const wf_solver* h) {
    const Params& P = h->P;
    const float* fx = h->fpos;
    const float* fy = fx + P.nx + 1;
    const float* fz = fy + P.ny + 1;
    WF_COUNT_LAUNCH();
    k_nu_vel_precompute<<<nu_grid(P), nu_block(), 0, h->st>>>(P, h->B, fx, fy, fz, h->fl, h->vb[h->iT], h->pr,
                                                               h->flux, P.les ? h->eddy : nullptr, h->Dv, h->bv,
                                                               h->vcoef, h->vcoef + 6 * (size_t)P.N);
}

void launch_nu_pres_precompute(wf_solver* h, const float* u) {
    const Params& P = h->P;
    const float* fx = h->fpos;
    const float* fy = fx + P.nx + 1;
    const float* fz = fy + P.ny + 1;
    WF_COUNT_LAUNCH();
    k_nu_pres_precompute<<<nu_grid(P), nu_block(), 0, h->st>>>(P, h->B, fx, fy, fz, h->fl, u, h->pr, h->Dv,
                                                                h->flux, h->Dp, h->bp, h->nucoef);
}

void launch_nu_pres_sweep(const wf_solver* h, const float* pin, float* pout, bool pre) {
    const Params& P = h->P;
    WF_COUNT_LAUNCH();
    const float* c = h->nucoef;
    const float* b = h->bp;
    if (quad_ok(P, {pin, h->nucoef, h->bp, pout, P.nbm})) {
        const int nq = P.N / 4;
        launch_chained(k_nu_pres_sweep4, dim3((nq + 255) / 256), dim3(256), h->st, h->pdl != 0, P, pin, c, b, pout,
                       (h->pdl != 0 && pre) ? 1 : 0);
    } else {
        launch_chained(k_nu_pres_sweep, dim3((P.N + 255) / 256), dim3(256), h->st, h->pdl != 0, P, pin, c, b, pout);
    }
}

void launch_nu_apply_vel(wf_solver* h, const float* pc, float* u) {
    const Params& P = h->P;
    const float* fx = h->fpos;
    const float* fy = fx + P.nx + 1;
    const float* fz = fy + P.ny + 1;
    WF_COUNT_LAUNCH();
    k_nu_apply_vel<<<nu_grid(P), nu_block(), 0, h->st>>>(P, fx, fy, fz, h->fl, pc, h->Dv, h->uc, u);
}

void launch_nu_init_log(wf_solver* h, float fric, float kappa, float z0) {
    const Params& P = h->P;
    k_nu_init_log<<<nu_grid(P), nu_block(), 0, h->st>>>(P, h->fpos + P.nx + 1, fric, kappa, z0, h->vb[0], h->vb[1],
                                                         h->vb[2], h->uc, h->pr);
}

void launch_nu_log_inlet(wf_solver* h, float fric, float kappa, float z0) {
    const Params& P = h->P;
    const int n = P.ny * P.nz;
    k_nu_log_inlet<<<(n + 255) / 256, 256, 0, h->st>>>(P.ny, P.nz, h->fpos + P.nx + 1, fric, kappa, z0,
                                                      h->bnd[WF_FACE_X0]);
}

}  // namespace wf
