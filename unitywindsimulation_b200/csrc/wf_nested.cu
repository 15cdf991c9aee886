// wf_nested.cu - initialisation of a domain from a running background
// domain (nested set-up of FvmSolverController.cs:143-151, :690): every cell
// of this domain samples the background's velocity and pressure at its
// position, with the domain rotated about the vertical axis.
//
// Restates CSInitVelPresFieldsFromBGFlowRotate (InitShaderColl.compute:185-
// 226) and its host side (FvmSolverGpu.cs:898-929):
//   loc  = (cell index - res/2) * dx             (integer res/2, index not centre)
//   glo  = pos + R(theta) loc,  R rotates x-z:   (x c + z s, y, z c - x s)
//   locB = R(-theta) (glo - posB)
//   uvw  = locB / (resB * dxB) + 0.5,  sampled trilinearly with clamped
//          addressing (texel centres at (i + 0.5) / resB)
// The sampled velocity vector is copied as is (not rotated), as in the
// reference.  theta = degrees * (float)(3.1415926 / 180) as on the host side.
#include <cuda_runtime.h>

#include <cmath>

#include "wf_kernels.cuh"
#include "wf_solver.cuh"

namespace wf {
namespace {

struct Frame {
    float pos[3], posb[3];
    float dx, dxb;
    int nbx, nby, nbz;
    float s1, c1, s2, c2;  // sin/cos of theta and of -theta
};

// Texture-style trilinear sample of one SoA plane in normalised coordinates
// with clamp-to-edge addressing.
__device__ __forceinline__ float sample(const float* __restrict__ f, const Frame& F, float u, float v, float w) {
    const float tx = u * (float)F.nbx - 0.5f, ty = v * (float)F.nby - 0.5f, tz = w * (float)F.nbz - 0.5f;
    const float bx = floorf(tx), by = floorf(ty), bz = floorf(tz);
    const float ax = tx - bx, ay = ty - by, az = tz - bz;
    const int x0 = min(max((int)bx, 0), F.nbx - 1), x1 = min(max((int)bx + 1, 0), F.nbx - 1);
    const int y0 = min(max((int)by, 0), F.nby - 1), y1 = min(max((int)by + 1, 0), F.nby - 1);
    const int z0 = min(max((int)bz, 0), F.nbz - 1), z1 = min(max((int)bz + 1, 0), F.nbz - 1);
    auto at = [&](int x, int y, int z) { return __ldg(f + ((size_t)z * F.nby + y) * F.nbx + x); };
    const float c00 = at(x0, y0, z0) * (1.f - ax) + at(x1, y0, z0) * ax;
    const float c10 = at(x0, y1, z0) * (1.f - ax) + at(x1, y1, z0) * ax;
    const float c01 = at(x0, y0, z1) * (1.f - ax) + at(x1, y0, z1) * ax;
    const float c11 = at(x0, y1, z1) * (1.f - ax) + at(x1, y1, z1) * ax;
    const float c0 = c00 * (1.f - ay) + c10 * ay;
    const float c1 = c01 * (1.f - ay) + c11 * ay;
    return c0 * (1.f - az) + c1 * az;
}

__global__ void k_init_from_bg(const __grid_constant__ Params P, const Frame F, const float* __restrict__ vbg,
                               const float* __restrict__ pbg, float* u0, float* u1, float* u2, float* u3,
                               float* __restrict__ uc, float* __restrict__ pr) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= P.nx || y >= P.ny || z >= P.nz) return;
    const float lx = (float)(x - P.nx / 2) * F.dx;
    const float ly = (float)(y - P.ny / 2) * F.dx;
    const float lz = (float)(z - P.nz / 2) * F.dx;
    const float gx = F.pos[0] + (lx * F.c1 + lz * F.s1);
    const float gy = F.pos[1] + ly;
    const float gz = F.pos[2] + (lz * F.c1 - lx * F.s1);
    const float rx = gx - F.posb[0], ry = gy - F.posb[1], rz = gz - F.posb[2];
    const float bx = rx * F.c2 + rz * F.s2, by = ry, bz = rz * F.c2 - rx * F.s2;
    const float u = bx / ((float)F.nbx * F.dxb) + 0.5f;
    const float v = by / ((float)F.nby * F.dxb) + 0.5f;
    const float w = bz / ((float)F.nbz * F.dxb) + 0.5f;
    const size_t Nb = (size_t)F.nbx * F.nby * F.nbz, N = P.N;
    const int i = cidx(P, x, y, z);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float val = sample(vbg + k * Nb, F, u, v, w);
        u0[k * N + i] = val;
        u1[k * N + i] = val;
        u2[k * N + i] = val;
        u3[k * N + i] = val;
        uc[k * N + i] = 0.f;
    }
    pr[i] = sample(pbg, F, u, v, w);
}

}  // namespace
}  // namespace wf

extern "C" int wf_init_from_background(wf_solver* h, const wf_solver* bg, const float pos[3], const float pos_bg[3],
                                       float rot_deg) {
    if (!h || !bg || !pos || !pos_bg) return WF_ERR_INVALID_ARG;
    if (h == bg || h->device != bg->device) {
        h->err = "background must be another handle on the same device";
        return WF_ERR_INVALID_ARG;
    }
    if (!std::isfinite(rot_deg)) {
        h->err = "rotation must be finite";
        return WF_ERR_INVALID_ARG;
    }
    if (cudaSetDevice(h->device) != cudaSuccess) return WF_ERR_CUDA;
    // the background's current state must be complete before it is read
    if (cudaStreamSynchronize(bg->st) != cudaSuccess) return WF_ERR_CUDA;
    wf::Frame F;
    for (int k = 0; k < 3; ++k) {
        F.pos[k] = pos[k];
        F.posb[k] = pos_bg[k];
    }
    F.dx = h->cfg.dx;
    F.dxb = bg->cfg.dx;
    F.nbx = bg->P.nx;
    F.nby = bg->P.ny;
    F.nbz = bg->P.nz;
    const float th = rot_deg * (float)(3.1415926 / 180);
    F.s1 = std::sin(th);
    F.c1 = std::cos(th);
    F.s2 = std::sin(-th);
    F.c2 = std::cos(-th);
    const dim3 b(32, 4, 2), g((h->P.nx + 31) / 32, (h->P.ny + 3) / 4, (h->P.nz + 1) / 2);
    WF_COUNT_LAUNCH();
    wf::k_init_from_bg<<<g, b, 0, h->st>>>(h->P, F, bg->vb[bg->iT], bg->pr, h->vb[0], h->vb[1], h->vb[2], h->vb[3],
                                           h->uc, h->pr);
    cudaError_t e = cudaGetLastError();
    for (int k = 0; k < 3 && e == cudaSuccess; ++k)
        e = cudaMemsetAsync(h->pcb[k], 0, sizeof(float) * h->P.N, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) {
        h->err = std::string("init from background: ") + cudaGetErrorString(e);
        return WF_ERR_CUDA;
    }
    h->iter_alias = false;
    h->pc_zero = true;
    return WF_OK;
}
