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

// ------------------------------------------------------------------------
// K pressure sweeps per pass (temporal blocking, 2.5D wavefront).
//
// A block owns a 32 x 32 column tile of the x-y plane, K cells wider than
// its output tile on every side, and streams a chunk of z planes.  Level 0
// is the input iterate; level s (1..K) is sweep s.  At pipeline step t the
// block pushes input plane zs + t and level s computes plane zs + t - s from
// level s-1's planes zs+t-s-1 .. zs+t-s+1: the own column's three planes sit
// in registers, the x/y neighbours in a double-buffered shared plane per
// level.  Coefficients are read from DRAM once per pass: the own column's
// c_U, 1/Dp and rhs ride in register queues, c_E and c_N (needed by the x/y
// neighbours) in a shared ring of K+1 planes.  Every load of step t+1 is
// issued at the top of step t, so its latency hides behind step t's
// arithmetic; one __syncthreads per step.  The valid region shrinks by one
// cell per level on every side, so level K is exact on the output tile and
// z chunk.  Cells outside the domain carry zero values and coefficients,
// which reproduces the reference's InRegion tests without branches, and
// non-fluid cells have 1/Dp = 0, so they stay 0 inside the pass and are
// never written.
//
// DRAM traffic per pass and cell: coefficients (c_E, c_N, c_U, 1/Dp, rhs:
// 20 B) and the input iterate (4 B) once, the output iterate (4 B) once,
// against 28 B per sweep for one sweep per launch.
constexpr int MS_TX = 32, MS_TY = 32;
constexpr size_t pres_msweep_smem(int K) { return sizeof(float) * MS_TX * MS_TY * (2 * K + 2 * (K + 1)); }

template <int K>
__global__ void __launch_bounds__(MS_TX* MS_TY, 1)
    k_pres_msweep(const __grid_constant__ Params P, const float* __restrict__ c3, const float* __restrict__ ainv,
                  const float* __restrict__ rhs, const float* __restrict__ pin, float* __restrict__ pout,
                  float* __restrict__ pprev, int zchunk) {
    // dynamic shared memory (above the 48 KB static limit for K >= 3):
    // V[K][2][TY][TX] level planes, CE/CN[K+1][TY][TX] coefficient rings
    extern __shared__ float msm[];
    float(*V)[2][MS_TY][MS_TX] = reinterpret_cast<float(*)[2][MS_TY][MS_TX]>(msm);
    float(*CE)[MS_TY][MS_TX] = reinterpret_cast<float(*)[MS_TY][MS_TX]>(msm + K * 2 * MS_TY * MS_TX);
    float(*CN)[MS_TY][MS_TX] = CE + (K + 1);
    const int tx = threadIdx.x, ty = threadIdx.y;
    constexpr int OX = MS_TX - 2 * K, OY = MS_TY - 2 * K;
    const int x = blockIdx.x * OX - K + tx;
    const int y = blockIdx.y * OY - K + ty;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(z0 + zchunk, P.nz);
    const bool inxy = x >= 0 && x < P.nx && y >= 0 && y < P.ny;
    const bool out_col = inxy && tx >= K && tx < MS_TX - K && ty >= K && ty < MS_TY - K;
    const size_t N = P.N;
    const int sxy = P.nx * P.ny;
    const int col = inxy ? y * P.nx + x : 0;
    const float* cEg = c3;
    const float* cNg = c3 + N;
    const float* cUg = c3 + 2 * N;
    const int xe = min(tx + 1, MS_TX - 1), xw = max(tx - 1, 0);
    const int yn = min(ty + 1, MS_TY - 1), ys = max(ty - 1, 0);

#pragma unroll
    for (int s = 0; s < K; ++s) V[s][0][ty][tx] = V[s][1][ty][tx] = 0.f;
#pragma unroll
    for (int s = 0; s <= K; ++s) CE[s][ty][tx] = CN[s][ty][tx] = 0.f;
    float h[K + 1][3];
    float qa[K + 1], qr[K + 1], qu[K + 2];
#pragma unroll
    for (int s = 0; s <= K; ++s) h[s][0] = h[s][1] = h[s][2] = qa[s] = qr[s] = 0.f;
#pragma unroll
    for (int s = 0; s < K + 2; ++s) qu[s] = 0.f;

    const int zs = z0 - K;
    const int T = (z1 - z0) + 2 * K;
    float pv = 0.f, pe = 0.f, pn = 0.f, pu = 0.f, pa = 0.f, pr = 0.f;
    {
        const int p = zs;
        if (inxy && p >= 0 && p < P.nz) {
            const int i = p * sxy + col;
            pv = pin ? __ldg(pin + i) : 0.f;
            pe = __ldg(cEg + i); pn = __ldg(cNg + i); pu = __ldg(cUg + i);
            pa = __ldg(ainv + i); pr = __ldg(rhs + i);
        }
    }
    __syncthreads();
    for (int t = 0; t < T; ++t) {
        const int cur = t & 1, prv = cur ^ 1;
        // prefetch step t+1
        float nv = 0.f, ne = 0.f, nn = 0.f, nu = 0.f, na = 0.f, nr = 0.f;
        {
            const int p = zs + t + 1;
            if (inxy && p >= 0 && p < P.nz && t + 1 < T) {
                const int i = p * sxy + col;
                nv = pin ? __ldg(pin + i) : 0.f;
                ne = __ldg(cEg + i); nn = __ldg(cNg + i); nu = __ldg(cUg + i);
                na = __ldg(ainv + i); nr = __ldg(rhs + i);
            }
        }
        // level 0 and the coefficients of plane zs + t
        h[0][0] = h[0][1]; h[0][1] = h[0][2]; h[0][2] = pv;
        V[0][cur][ty][tx] = pv;
        const int cw = t % (K + 1);
        CE[cw][ty][tx] = pe;
        CN[cw][ty][tx] = pn;
#pragma unroll
        for (int s = K; s > 0; --s) { qa[s] = qa[s - 1]; qr[s] = qr[s - 1]; }
        qa[0] = pa; qr[0] = pr;
#pragma unroll
        for (int s = K + 1; s > 0; --s) qu[s] = qu[s - 1];
        qu[0] = pu;
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            const int rs = (t - s + K + 1) % (K + 1);
            const float(*L)[MS_TX] = V[s - 1][prv];
            float acc = -(CE[rs][ty][tx] * L[ty][xe]);
            acc -= CE[rs][ty][xw] * L[ty][xw];
            acc -= CN[rs][ty][tx] * L[yn][tx];
            acc -= CN[rs][ys][tx] * L[ys][tx];
            acc -= qu[s] * h[s - 1][2];
            acc -= qu[s + 1] * h[s - 1][0];
            const float v = qa[s] * (acc + qr[s]);
            if (s == K) {
                const int p = zs + t - K;
                if (out_col && p >= z0 && p < z1 && qa[K] != 0.f) {
                    const int i = p * sxy + col;
                    pout[i] = v;
                    if (pprev) pprev[i] = h[K - 1][1];
                }
            }
            h[s][0] = h[s][1]; h[s][1] = h[s][2]; h[s][2] = v;
            if (s < K) V[s][cur][ty][tx] = v;
        }
        __syncthreads();
        pv = nv; pe = ne; pn = nn; pu = nu; pa = na; pr = nr;
    }
}

// K momentum sweeps per pass: the same wavefront for the three velocity
// components on a 32 x 16 tile (three components need three times the
// registers per level).  All 12 coefficient planes (A_E..A_D, 1/D, b) are
// the own column's, so they ride in register queues.  Per pass and cell the
// coefficients (48 B) and the input iterate (12 B) are read once and the
// output iterate (12 B) written once.
constexpr int MV_TX = 32, MV_TY = 16;

template <int K>
__global__ void __launch_bounds__(MV_TX* MV_TY, 1)
    k_vel_msweep(const __grid_constant__ Params P, const float* __restrict__ A, const float* __restrict__ iD,
                 const float* __restrict__ bv, const float* __restrict__ uin, float* __restrict__ uout,
                 float* __restrict__ uprev, int zchunk) {
    __shared__ float V[K][2][3][MV_TY][MV_TX];
    const int tx = threadIdx.x, ty = threadIdx.y;
    constexpr int OX = MV_TX - 2 * K, OY = MV_TY - 2 * K;
    const int x = blockIdx.x * OX - K + tx;
    const int y = blockIdx.y * OY - K + ty;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(z0 + zchunk, P.nz);
    const bool inxy = x >= 0 && x < P.nx && y >= 0 && y < P.ny;
    const bool out_col = inxy && tx >= K && tx < MV_TX - K && ty >= K && ty < MV_TY - K;
    const size_t N = P.N;
    const int sxy = P.nx * P.ny;
    const int col = inxy ? y * P.nx + x : 0;
    const int xe = min(tx + 1, MV_TX - 1), xw = max(tx - 1, 0);
    const int yn = min(ty + 1, MV_TY - 1), ys = max(ty - 1, 0);

#pragma unroll
    for (int s = 0; s < K; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) V[s][0][c][ty][tx] = V[s][1][c][ty][tx] = 0.f;
    float h[K + 1][3][3];
    float qc[K + 1][12];  // A_E..A_D, 1/D x3, b x3 of planes zs+t, zs+t-1, ...
#pragma unroll
    for (int s = 0; s <= K; ++s) {
#pragma unroll
        for (int c = 0; c < 3; ++c) h[s][c][0] = h[s][c][1] = h[s][c][2] = 0.f;
#pragma unroll
        for (int j = 0; j < 12; ++j) qc[s][j] = 0.f;
    }
    const int zs = z0 - K;
    const int T = (z1 - z0) + 2 * K;
    float pv[3], pc[12];
    auto load = [&](int p, bool ok, float v[3], float c[12]) {
        if (ok && inxy && p >= 0 && p < P.nz) {
            const int i = p * sxy + col;
#pragma unroll
            for (int k = 0; k < 3; ++k) v[k] = __ldg(uin + k * N + i);
#pragma unroll
            for (int f = 0; f < 6; ++f) c[f] = __ldg(A + f * N + i);
#pragma unroll
            for (int k = 0; k < 3; ++k) c[6 + k] = __ldg(iD + k * N + i);
#pragma unroll
            for (int k = 0; k < 3; ++k) c[9 + k] = __ldg(bv + k * N + i);
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) v[k] = 0.f;
#pragma unroll
            for (int j = 0; j < 12; ++j) c[j] = 0.f;
        }
    };
    load(zs, true, pv, pc);
    __syncthreads();
    for (int t = 0; t < T; ++t) {
        const int cur = t & 1, prv = cur ^ 1;
        float nv[3], nc[12];
        load(zs + t + 1, t + 1 < T, nv, nc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            h[0][c][0] = h[0][c][1]; h[0][c][1] = h[0][c][2]; h[0][c][2] = pv[c];
            V[0][cur][c][ty][tx] = pv[c];
        }
#pragma unroll
        for (int s = K; s > 0; --s)
#pragma unroll
            for (int j = 0; j < 12; ++j) qc[s][j] = qc[s - 1][j];
#pragma unroll
        for (int j = 0; j < 12; ++j) qc[0][j] = pc[j];
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            float v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float(*L)[MV_TX] = V[s - 1][prv][c];
                float acc = qc[s][0] * L[ty][xe];
                acc += qc[s][1] * L[ty][xw];
                acc += qc[s][2] * L[yn][tx];
                acc += qc[s][3] * L[ys][tx];
                acc += qc[s][4] * h[s - 1][c][2];
                acc += qc[s][5] * h[s - 1][c][0];
                v[c] = qc[s][6 + c] * (acc + qc[s][9 + c]);
            }
            if (s == K) {
                const int p = zs + t - K;
                if (out_col && p >= z0 && p < z1 && qc[K][6] != 0.f) {
                    const int i = p * sxy + col;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        uout[c * N + i] = v[c];
                        if (uprev) uprev[c * N + i] = h[K - 1][c][1];
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                h[s][c][0] = h[s][c][1]; h[s][c][1] = h[s][c][2]; h[s][c][2] = v[c];
                if (s < K) V[s][cur][c][ty][tx] = v[c];
            }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 3; ++c) pv[c] = nv[c];
#pragma unroll
        for (int j = 0; j < 12; ++j) pc[j] = nc[j];
    }
}

// Reads a buffer larger than L2 so the next launch starts cold.  Reading
// (not writing) leaves no dirty lines whose write-back would be billed to
// the timed kernel.
__global__ void k_flush_read(const float4* __restrict__ buf, size_t n, float* __restrict__ sink) {
    float acc = 0.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float4 v = __ldcs(buf + i);
        acc += v.x + v.y + v.z + v.w;
    }
    if (acc == 1.2345f) sink[0] = acc;  // keeps the loads alive
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

namespace {

// z chunking of the wavefront kernels (one resident block per SM): as many
// chunks as fit one wave of blocks on the device's SMs, so no SM runs a
// second, partly empty wave; each chunk re-reads 2K halo planes.
void wave_chunks(const wf_solver* h, int blocks_xy, int K, int& zchunk, int& nchunk) {
    const int sms = h->num_sms > 0 ? h->num_sms : 148;
    nchunk = std::max(1, sms / std::max(blocks_xy, 1));
    zchunk = std::max(2 * K + 2, (h->P.nz + nchunk - 1) / nchunk);
    nchunk = (h->P.nz + zchunk - 1) / zchunk;
}

template <int K>
void launch_vmsweep_k(wf_solver* h, const float* in, float* out, float* prev) {
    const Params& P = h->P;
    const size_t N = P.N;
    constexpr int OX = MV_TX - 2 * K, OY = MV_TY - 2 * K;
    const int gx = (P.nx + OX - 1) / OX, gy = (P.ny + OY - 1) / OY;
    int zchunk = 0, nchunk = 0;
    wave_chunks(h, gx * gy, K, zchunk, nchunk);
    WF_COUNT_LAUNCH();
    k_vel_msweep<K><<<dim3(gx, gy, nchunk), dim3(MV_TX, MV_TY), 0, h->st>>>(P, h->vcoef, h->vcoef + 6 * N, h->bv,
                                                                          in, out, prev, zchunk);
}

void launch_vmsweep(wf_solver* h, int k, const float* in, float* out, float* prev) {
    switch (k) {
        case 1: launch_vmsweep_k<1>(h, in, out, prev); break;
        case 2: launch_vmsweep_k<2>(h, in, out, prev); break;
        default: launch_vmsweep_k<3>(h, in, out, prev); break;
    }
}

}  // namespace

int sweeps_setup() {
    // dynamic shared memory above 48 KB needs the opt-in, per device
    cudaError_t e = cudaSuccess;
    e = cudaFuncSetAttribute(k_pres_msweep<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pres_msweep_smem(1));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_pres_msweep<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pres_msweep_smem(2));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_pres_msweep<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pres_msweep_smem(3));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_pres_msweep<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pres_msweep_smem(4));
    return e == cudaSuccess ? WF_OK : WF_ERR_CUDA;
}

int vel_sweeps_fast(wf_solver* h, int n) {
    vel_coef(h);
    const int kmax = std::min(std::max(h->vel_k, 1), 3);
    if (kmax > 1) {
        // Passes of up to kmax sweeps over buffers other than velFieldLastTime;
        // the last pass also writes iterate n-1 (the reference's
        // velFieldLastIter after the loop) unless inside a full step.
        int in_idx = h->iter_alias ? h->iT : h->iI;
        int out_idx = -1, prev_idx = -1;
        bool prev_is_time = false;
        int remaining = n;
        auto pick = [&](int a, int b, int c) {
            for (int i = 0; i < 4; ++i)
                if (i != a && i != b && i != c) return i;
            return -1;
        };
        while (remaining > 0) {
            const int k = std::min(kmax, remaining);
            const bool last = remaining == k;
            out_idx = pick(h->iT, in_idx, -1);
            float* prev = nullptr;
            if (last && k >= 2) {
                prev_idx = pick(h->iT, in_idx, out_idx);
                if (!h->in_step) prev = h->vb[prev_idx];
            } else if (last) {
                prev_idx = in_idx;
                prev_is_time = in_idx == h->iT;
            }
            launch_vmsweep(h, k, h->vb[in_idx], h->vb[out_idx], prev);
            remaining -= k;
            if (!last) in_idx = out_idx;
        }
        h->iF = out_idx;
        if (prev_is_time) {
            // iterate n-1 is velFieldLastTime itself (n == 1 from the alias)
            h->iI = pick(h->iT, h->iF, -1);
            h->iter_alias = true;
        } else {
            h->iI = prev_idx;
            h->iter_alias = false;
        }
        return cudaGetLastError() == cudaSuccess ? WF_OK : WF_ERR_CUDA;
    }
    for (int k = 0; k < n; ++k) {
        const float* src = h->iter_alias ? h->vb[h->iT] : h->vb[h->iI];
        launch_vel_sweep_fast(h, src, h->vb[h->iF]);
        std::swap(h->iI, h->iF);
        h->iter_alias = false;
    }
    std::swap(h->iI, h->iF);
    return cudaGetLastError() == cudaSuccess ? WF_OK : WF_ERR_CUDA;
}

namespace {

template <int K>
void launch_msweep_k(wf_solver* h, const float* rhs, const float* in, float* out, float* prev) {
    const Params& P = h->P;
    const size_t N = P.N;
    constexpr int OX = MS_TX - 2 * K, OY = MS_TY - 2 * K;
    const int gx = (P.nx + OX - 1) / OX, gy = (P.ny + OY - 1) / OY;
    int zchunk = 0, nchunk = 0;
    wave_chunks(h, gx * gy, K, zchunk, nchunk);
    const size_t smem = pres_msweep_smem(K);
    WF_COUNT_LAUNCH();
    k_pres_msweep<K><<<dim3(gx, gy, nchunk), dim3(MS_TX, MS_TY), smem, h->st>>>(P, h->pcoef, h->pcoef + 3 * N, rhs,
                                                                              in, out, prev, zchunk);
}

void launch_msweep(wf_solver* h, int k, const float* rhs, const float* in, float* out, float* prev) {
    switch (k) {
        case 1: launch_msweep_k<1>(h, rhs, in, out, prev); break;
        case 2: launch_msweep_k<2>(h, rhs, in, out, prev); break;
        case 3: launch_msweep_k<3>(h, rhs, in, out, prev); break;
        default: launch_msweep_k<4>(h, rhs, in, out, prev); break;
    }
}

}  // namespace

int pres_sweeps_fast(wf_solver* h, int n, bool piso) {
    const float* rhs = pres_coef(h, piso);
    const int kmax = std::min(std::max(h->pres_k, 1), 4);
    if (kmax == 1) {
        for (int k = 0; k < n; ++k) {
            const float* src = h->pc_zero ? nullptr : h->pcb[h->iPCL];
            launch_pres_sweep_fast(h, rhs, src, h->pcb[h->iPC]);
            h->pc_zero = false;
            std::swap(h->iPCL, h->iPC);
        }
        std::swap(h->iPCL, h->iPC);
        return cudaGetLastError() == cudaSuccess ? WF_OK : WF_ERR_CUDA;
    }
    // Passes of up to kmax sweeps ping-pong between two of the three buffers;
    // the last pass also writes iterate n-1 to the third one (skipped inside
    // a full step, where nothing reads presCorrectFieldLastIter afterwards).
    int in_idx = h->pc_zero ? -1 : h->iPCL;  // -1: the all-zero start
    int out_idx = -1, prev_idx = -1;
    int remaining = n;
    while (remaining > 0) {
        const int k = std::min(kmax, remaining);
        const bool last = remaining == k;
        out_idx = in_idx == 0 ? 1 : 0;
        float* prev = nullptr;
        if (last && k >= 2) {
            prev_idx = in_idx < 0 ? (out_idx == 0 ? 1 : 0) : 3 - in_idx - out_idx;
            if (!h->in_step) prev = h->pcb[prev_idx];
        } else if (last) {
            prev_idx = in_idx;  // iterate n-1 is this pass's input
        }
        launch_msweep(h, k, rhs, in_idx < 0 ? nullptr : h->pcb[in_idx], h->pcb[out_idx], prev);
        remaining -= k;
        if (!last) in_idx = out_idx;
    }
    h->pc_zero = false;
    h->iPC = out_idx;
    if (prev_idx < 0) {
        // n == 1 from the zero start: iterate 0 is all zeros
        prev_idx = out_idx == 0 ? 1 : 0;
        if (!h->in_step) cudaMemsetAsync(h->pcb[prev_idx], 0, sizeof(float) * h->P.N, h->st);
    }
    h->iPCL = prev_idx;
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
    if (flush) cudaMemsetAsync(fbuf, 0, flush_bytes, h->st);
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
    const int kv = std::min(std::max(h->vel_k, 1), 3), kp = std::min(std::max(h->pres_k, 1), 4);
    for (int r = 0; r < reps; ++r) {
        if (flush) k_flush_read<<<148 * 4, 512, 0, h->st>>>((const float4*)fbuf, flush_bytes / 16, (float*)fbuf);
        cudaEventRecord(e0, h->st);
        if (which == WF_KERNEL_VEL_SWEEP) {
            if (kv > 1) launch_vmsweep(h, kv, a, b, nullptr);
            else launch_vel_sweep_fast(h, a, b);
        } else {
            if (kp > 1) launch_msweep(h, kp, rhs, a, b, nullptr);
            else launch_pres_sweep_fast(h, rhs, a, b);
        }
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
    *sweeps = which == WF_KERNEL_VEL_SWEEP ? kv : kp;
    // compulsory bytes of the reference kernels per cell and sweep:
    // CSPresCorrectRhieChow 29 B, CSVelPredict 77 B
    *bytes = double(which == WF_KERNEL_VEL_SWEEP ? 77 : 29) * double(N) * double(*sweeps);
    return WF_OK;
}

}  // namespace wf
