// wf_vel_tma.cu - two momentum Jacobi sweeps per pass with TMA-staged halo
// tiles (CSVelPredict, FvmColl.compute:1863-2069, temporal blocking).
//
// A block owns a 32 x 32 column tile of the x-y plane (a 28 x 28 output tile
// with a 2-cell halo on every side) and streams a chunk of z planes; level 1
// computes plane zs + t - 1 and level 2 plane zs + t - 2 at step t.  Each z
// plane of the tile arrives as 14 planes of 36 x 32 FP32 values: the six
// off-diagonal coefficients A_E..A_D, the first two components of 1/D, the
// three components of b and of the input iterate.  The boxes start at x = 28 bx - 4
// (16-byte aligned) and are 36 wide, so the thread of column tx reads column
// tx + 2 and its x neighbours are always inside the box.  One thread issues
// the loads (four cp.async.bulk.tensor per plane, one mbarrier) one plane
// ahead into a ring of three slots.  The tensor maps' bounds give zeros
// outside the domain; there the coefficients are zero, as the reference's
// boundary faces carry no off-diagonal term.
//
// Threads: 32 x 16, each owning two adjacent tile rows; per level a row reads
// its x neighbours and one y neighbour from shared memory and the other y
// neighbour from the thread's own registers.  Level 1 reads plane t-1's
// coefficients from its ring slot and keeps them in registers for level 2 at
// the next step (two register sets, alternating with the step's parity).
// The three components of 1/D are bit-identical outside the cells with a
// symmetry domain face (d_split), and each differs from the others only by
// the term of faces normal to its own axis: the third component is taken
// from the first two, and read from global memory only on z-symmetry planes
// and x-y symmetry edges.  Non-fluid cells (1/D = 0) carry their input value
// through both levels and are never written.  The arithmetic, its order and
// every stored value are those of k_vel_sweep4, so two sweeps of either give
// bit-identical iterates.
//
// Every mbarrier wait is bounded as in the TMA pressure pass (wf_pres_tma.cu)
// and a wait that runs out sets the handle's sticky wait status.
//
// Selected by a momentum blocking depth of 2 (wf_set_blocking).  Not the
// default: on the 256 x 96 x 192 urban block it takes 47.7 us per sweep
// against 50.2 us for one k_vel_sweep4 launch per sweep in isolation, but
// the graph-replayed step gains only 0.6 % (back to back, the one-sweep
// launches find part of their input in L2); the autotuner picks either per
// grid.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>

#include "wf_sweeps.cuh"
#include "wf_tma.cuh"

namespace wf {
namespace {

using namespace tma;

constexpr int VK = 2;              // sweeps per pass
constexpr int VT = 32;             // tile edge in threads (x) and rows (y)
constexpr int VO = VT - 2 * VK;    // output tile edge (28)
constexpr int VW = VT + 4;         // box width: 2 extra columns on each side
constexpr int VPL = VW * VT;       // floats per staged plane
constexpr int VR = 2;              // tile rows per thread
constexpr int VTHR = VT * VT / VR; // threads per block
constexpr int VD = 1;              // planes loaded ahead of the consumed one
constexpr int VC = VD + 2;         // ring slots (a plane is read at steps p and p + 1)
constexpr int VU = 6;              // unrolled steps per trip: lcm of 3 (slots, rings) and 2 (sets)
// staged planes of one slot: A_E..A_D, 1/D (first two components), b, u
enum { S_A = 0, S_ID = 6, S_ID1 = 7, S_B = 8, S_U = 11, VQ = 14 };
constexpr int kVSlot = VQ * VPL;
constexpr size_t kVSmemFloats = (size_t)VC * kVSlot + (size_t)2 * 3 * VPL;
constexpr size_t kVSmemBytes = kVSmemFloats * sizeof(float) + VC * sizeof(unsigned long long) + 1024;
constexpr unsigned long long kVWaitNs = 1000000000ull;

static_assert(VO % 4 == 0, "box origins x = 28 bx - 4 must be 16-byte aligned");
static_assert(kVSmemBytes <= 232448, "ring exceeds the shared memory of one block");
static_assert(VU % VC == 0 && (VU / VC) % 2 == 0 && VU % 2 == 0, "trip must cover the ring an even number of times");

struct VelMaps {
    CUtensorMap A;    // 4-D {nx, ny, nz, 6}, box 36 x 32 x 1 x 6
    CUtensorMap iD;   // 4-D {nx, ny, nz, 2}, box of the first two components
    CUtensorMap b;    // 4-D {nx, ny, nz, 3}, box of three planes
    CUtensorMap u;    // 4-D {nx, ny, nz, 3}, box of three planes
};

struct VelWaveT {
    float* ring;              // VC slots of kVSlot floats
    float* V1;                // level-1 planes [2][3][VT][VW]
    unsigned bar0;
    const VelMaps* maps;
    const float* __restrict__ iDg;  // 1/D in global memory (all three components)
    float* __restrict__ uout;
    float* __restrict__ uprev;
    size_t N;
    int me;                   // row 0's own offset in a staged plane (column tx + 2)
    int r0, zs, z0, z1, T, sxy, x0, y0, tfail;
    int col[VR];
    bool out_col[VR], in_xy[VR], split_x[VR], split_y[VR];  // the cell has a symmetry x / y domain face
    bool edge_xy[VR];         // inside the domain with both an x and a y symmetry face
    bool split_z0, split_zn;  // symmetry faces at z = 0 / z = nz - 1
    bool bad, lead;
    int nz;
    unsigned long long wait_ns;
    // level values of the own cells: [row][plane ring of 3][component]
    float h0[VR][3][3], h1[VR][3][3];
    // coefficient sets [parity][row]: A_E..A_D, 1/D (three components), b
    float cA[2][VR][6], cI[2][VR][3], cB[2][VR][3];

    __device__ __forceinline__ void issue(int t, int slot) const {
        const unsigned bar = bar0 + slot * 8;
        const int p = zs + t;
        const unsigned dst = smem_addr(ring + slot * kVSlot);
        mbar_expect(bar, (unsigned)(sizeof(float) * VPL * VQ));
        tma_4d(dst + sizeof(float) * VPL * S_A, &maps->A, x0, y0, p, 0, bar);
        tma_4d(dst + sizeof(float) * VPL * S_ID, &maps->iD, x0, y0, p, 0, bar);
        tma_4d(dst + sizeof(float) * VPL * S_B, &maps->b, x0, y0, p, 0, bar);
        tma_4d(dst + sizeof(float) * VPL * S_U, &maps->u, x0, y0, p, 0, bar);
    }

    __device__ __forceinline__ const float* plane(int slot, int q) const { return ring + slot * kVSlot + q * VPL; }
    __device__ __forceinline__ float* v1(int buf, int c) const { return V1 + (buf * 3 + c) * VPL; }

    // The momentum stencil of one cell and component, in the order of
    // k_vel_sweep4: r = (1/D) (A_E u_E + A_W u_W + A_N u_N + A_S u_S + A_U u_U
    // + A_D u_D + b).
    static __device__ __forceinline__ float stencil(const float* a, float id, float bb, float ue, float uw, float un,
                                                    float us, float uu, float ud) {
        float acc = a[0] * ue;
        acc += a[1] * uw;
        acc += a[2] * un;
        acc += a[3] * us;
        acc += a[4] * uu;
        acc += a[5] * ud;
        return id * (acc + bb);
    }

    // Step t = trip base + PH: plane zs + t arrives, level 1 computes plane
    // zs + t - 1, level 2 plane zs + t - 2.
    template <int PH>
    __device__ __forceinline__ void step(int t) {
        if (t >= T) return;  // uniform over the block
        constexpr int cur = PH & 1, prv = cur ^ 1;
        constexpr int sN = PH % VC, sP = (PH + 2) % VC;        // slots of planes t and t - 1
        constexpr int q0 = PH % 3, q1 = (PH + 2) % 3, q2 = (PH + 1) % 3;  // rings: planes t, t-1, t-2 (t-3 = t)
        constexpr int c1 = PH % 2, c2 = (PH + 1) % 2;           // coefficient sets of levels 1 and 2
        constexpr unsigned parity = (PH / VC) & 1;
        if (!bad) bad = !mbar_wait(bar0 + sN * 8, parity, wait_ns);
        const int ys0 = r0 == 0 ? 0 : -VW;           // south of row 0 (clamped at the tile edge)
        const int yn1 = r0 + 1 == VT - 1 ? 0 : VW;   // north of row 1
        // plane t enters level 0
#pragma unroll
        for (int k = 0; k < VR; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) h0[k][q0][c] = plane(sN, S_U + c)[me + k * VW];
        // ---- level 1 on plane t - 1 (every row; rows 0 and 31 feed nothing)
        {
            const int p = zs + t - 1;
            const bool pin = p >= 0 && p < nz;
            const bool zface = (p == 0 && split_z0) || (p == nz - 1 && split_zn);  // implies pin
            bool fl[VR];
#pragma unroll
            for (int k = 0; k < VR; ++k) {
                const int o = me + k * VW;
#pragma unroll
                for (int f = 0; f < 6; ++f) cA[c1][k][f] = plane(sP, S_A + f)[o];
                const float id0 = plane(sP, S_ID)[o], id1 = plane(sP, S_ID1)[o];
                // component c of 1/D is the base value plus the symmetry term of
                // faces normal to axis c: the third equals the first outside
                // x-symmetry cells and the second outside y-symmetry cells; only
                // z-symmetry planes and x-y symmetry edges read it from memory
                cI[c1][k][0] = id0;
                cI[c1][k][1] = id1;
                cI[c1][k][2] = split_x[k] ? id1 : id0;
#pragma unroll
                for (int c = 0; c < 3; ++c) cB[c1][k][c] = plane(sP, S_B + c)[o];
                if ((pin && edge_xy[k]) || (zface && in_xy[k]))
                    cI[c1][k][2] = __ldg(iDg + 2 * N + (size_t)p * sxy + col[k]);
                fl[k] = id0 != 0.f;  // 1/D is 0 on non-fluid cells
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float* U = plane(sP, S_U + c);
                float* W = v1(cur, c);
#pragma unroll
                for (int k = 0; k < VR; ++k) {
                    const int o = me + k * VW;
                    const float un = k + 1 < VR ? h0[k + 1][q1][c] : U[o + yn1];
                    const float us = k > 0 ? h0[k - 1][q1][c] : U[o + ys0];
                    const float r = stencil(cA[c1][k], cI[c1][k][c], cB[c1][k][c], U[o + 1], U[o - 1], un, us,
                                            h0[k][q0][c], h0[k][q2][c]);
                    const float v = fl[k] ? r : h0[k][q1][c];
                    h1[k][q1][c] = v;
                    W[o] = v;
                }
            }
        }
        // ---- level 2 on plane t - 2 (rows 2..29)
        if (r0 >= VK && r0 + VR - 1 < VT - VK) {
            const int q = zs + t - 2;
            const bool emit = uout && q >= z0 && q < z1;
            float r2[VR][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float* U = v1(prv, c);
#pragma unroll
                for (int k = 0; k < VR; ++k) {
                    const int o = me + k * VW;
                    const float un = k + 1 < VR ? h1[k + 1][q2][c] : U[o + VW];
                    const float us = k > 0 ? h1[k - 1][q2][c] : U[o - VW];
                    r2[k][c] = stencil(cA[c2][k], cI[c2][k][c], cB[c2][k][c], U[o + 1], U[o - 1], un, us,
                                       h1[k][q1][c], h1[k][q0][c]);
                }
            }
            if (emit) {
#pragma unroll
                for (int k = 0; k < VR; ++k) {
                    if (!out_col[k] || cI[c2][k][0] == 0.f) continue;
                    float* o = uout + (size_t)q * sxy + col[k];
                    o[0] = r2[k][0];
                    o[N] = r2[k][1];
                    o[2 * N] = r2[k][2];
                    if (uprev) {
                        float* w = uprev + (size_t)q * sxy + col[k];
                        w[0] = h1[k][q2][0];
                        w[N] = h1[k][q2][1];
                        w[2 * N] = h1[k][q2][2];
                    }
                }
            }
        }
        if (__syncthreads_or(bad)) {
            bad = true;
            tfail = t;
            return;
        }
        // slot of plane t - 1 (last read by level 1 above) takes plane t + 2
        if (lead && t + 1 + VD < T) issue(t + 1 + VD, sP);
    }
};

template <int PH>
__device__ __forceinline__ bool vtrip(VelWaveT& w, int t0) {
    if constexpr (PH < VU) {
        w.step<PH>(t0 + PH);
        if (w.bad) return false;
        return vtrip<PH + 1>(w, t0);
    } else {
        return true;
    }
}

__global__ void __launch_bounds__(VTHR, 1)
    k_vel_tma2(const __grid_constant__ VelMaps maps, const __grid_constant__ Params P, const float* __restrict__ iDg,
               float* __restrict__ uout, float* __restrict__ uprev, int zchunk, int* __restrict__ status,
               unsigned long long wait_ns) {
    extern __shared__ __align__(1024) unsigned char vsm_raw[];
    const unsigned pad = (1024u - (smem_addr(vsm_raw) & 1023u)) & 1023u;
    float* base = reinterpret_cast<float*>(vsm_raw + pad);
    VelWaveT w;
    w.ring = base;
    w.V1 = base + VC * kVSlot;
    w.bar0 = smem_addr(base + kVSmemFloats);
    w.maps = &maps;
    w.iDg = iDg;
    w.uout = uout;
    w.uprev = uprev;
    w.N = (size_t)P.N;
    w.nz = P.nz;
    const int tx = threadIdx.x;
    const int tid = threadIdx.y * VT + tx;
    w.lead = tid == 0;
    w.r0 = threadIdx.y * VR;
    w.me = w.r0 * VW + tx + 2;
    w.x0 = blockIdx.x * VO - 4;
    w.y0 = blockIdx.y * VO - VK;
    const int x = blockIdx.x * VO - VK + tx;
    w.z0 = blockIdx.z * zchunk;
    w.z1 = min(w.z0 + zchunk, P.nz);
    w.sxy = P.nx * P.ny;
    w.split_z0 = P.vbc[WF_FACE_Z0] == WF_BND_SYMMETRY;
    w.split_zn = P.vbc[WF_FACE_ZN] == WF_BND_SYMMETRY;
#pragma unroll
    for (int k = 0; k < VR; ++k) {
        const int r = w.r0 + k, y = w.y0 + r;
        const bool inxy = x >= 0 && x < P.nx && y >= 0 && y < P.ny;
        w.in_xy[k] = inxy;
        w.out_col[k] = inxy && tx >= VK && tx < VT - VK && r >= VK && r < VT - VK;
        w.col[k] = inxy ? y * P.nx + x : 0;
        w.split_x[k] = inxy && ((x == 0 && P.vbc[WF_FACE_X0] == WF_BND_SYMMETRY) ||
                                (x == P.nx - 1 && P.vbc[WF_FACE_XN] == WF_BND_SYMMETRY));
        w.split_y[k] = inxy && ((y == 0 && P.vbc[WF_FACE_Y0] == WF_BND_SYMMETRY) ||
                                (y == P.ny - 1 && P.vbc[WF_FACE_YN] == WF_BND_SYMMETRY));
        w.edge_xy[k] = w.split_x[k] && w.split_y[k];
    }
    w.bad = false;
    w.tfail = 0;
    w.wait_ns = wait_ns;
    static_assert(kVSmemFloats % 4 == 0, "the ring is cleared with 16-byte stores");
    for (int i = tid; i < (int)(kVSmemFloats / 4); i += VTHR)
        reinterpret_cast<float4*>(base)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < VR; ++k) {
#pragma unroll
        for (int q = 0; q < 3; ++q)
#pragma unroll
            for (int c = 0; c < 3; ++c) w.h0[k][q][c] = w.h1[k][q][c] = 0.f;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
#pragma unroll
            for (int f = 0; f < 6; ++f) w.cA[s][k][f] = 0.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) w.cI[s][k][c] = w.cB[s][k][c] = 0.f;
        }
    }
    w.zs = w.z0 - VK;
    w.T = (w.z1 - w.z0) + 2 * VK;
    if (w.lead) {
        for (int c = 0; c < VC; ++c) mbar_init(w.bar0 + c * 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (w.lead)
        for (int t = 0; t <= VD && t < w.T; ++t) w.issue(t, t % VC);
    for (int t0 = 0; t0 < w.T; t0 += VU)
        if (!vtrip<0>(w, t0)) break;
    if (w.bad && w.lead) {
        if (status) atomicExch(status, 1);
        for (int t = w.tfail; t <= w.tfail + VD && t < w.T; ++t)
            mbar_wait(w.bar0 + (t % VC) * 8, (unsigned)((t / VC) & 1), wait_ns);
    }
}

bool aligned16v(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

size_t vel_tma_smem() { return kVSmemBytes; }
const void* vel_tma_kernel() { return reinterpret_cast<const void*>(k_vel_tma2); }

bool vel_tma_ok(const Params& P, const float* A, const float* iD, const float* bv, const float* in) {
    return P.nx % 4 == 0 && A && iD && bv && in && aligned16v(A) && aligned16v(iD) && aligned16v(bv) &&
           aligned16v(in) && tma_available();
}

cudaError_t launch_vel_tma2(const Params& P, cudaStream_t st, int sms, const float* A, const float* iD,
                            const float* bv, const float* in, float* out, float* prev, int* status, double wait_ms) {
    VelMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    if (!tma_encode(&maps.A, P, A, 6, VW, VT, 6) || !tma_encode(&maps.iD, P, iD, 2, VW, VT, 2) ||
        !tma_encode(&maps.b, P, bv, 3, VW, VT, 3) || !tma_encode(&maps.u, P, in, 3, VW, VT, 3))
        return cudaErrorInvalidValue;
    const int gx = (P.nx + VO - 1) / VO, gy = (P.ny + VO - 1) / VO;
    sms = sms > 0 ? sms : 148;
    int nchunk = std::max(1, sms / std::max(gx * gy, 1));
    const int zchunk = std::max(2 * VK + 2, (P.nz + nchunk - 1) / nchunk);
    nchunk = (P.nz + zchunk - 1) / zchunk;
    WF_COUNT_LAUNCH();
    const unsigned long long wait_ns = wait_ms > 0 ? (unsigned long long)(wait_ms * 1e6) : kVWaitNs;
    k_vel_tma2<<<dim3(gx, gy, nchunk), dim3(VT, VT / VR), kVSmemBytes, st>>>(maps, P, iD, out, prev, zchunk, status,
                                                                            wait_ns);
    return cudaGetLastError();
}

}  // namespace wf
