// wf_raster.cu - building footprints rasterised into the flag array on the
// GPU (the case generator's step; the reference voxelises Unity meshes by
// ray casting, BuildingVoxelizer.cs:355-413, and hands the same int32 flag
// layout to InitFlags).  Boxes (x0, x1, z0, z1, h) in cells are rotated by
// an angle about the domain centre in the x-z plane and tested at cell
// centres; cells within `margin` of the x/z boundaries stay fluid.  The
// rotation and the tests run in double precision with every rounding
// explicit, so the flags match the double-precision NumPy generator
// (cases.rasterise_boxes) bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/windfvm.h"

namespace {

// One thread per (x, z) column: the column is solid up to the tallest box
// that contains its centre (min(h, ny - 1) cells; h rounded half to even).
__global__ void k_raster(int nx, int ny, int nz, const double* __restrict__ boxes, int n, double c, double s,
                         int margin, int32_t* __restrict__ flags) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= nx || z >= nz) return;
    const double X = x + 0.5, Z = z + 0.5;
    const double cx = nx / 2.0, cz = nz / 2.0;
    const double dX = __dsub_rn(X, cx), dZ = __dsub_rn(Z, cz);
    // Xr = cx + (X - cx) c + (Z - cz) s ;  Zr = cz - (X - cx) s + (Z - cz) c
    const double Xr = __dadd_rn(__dadd_rn(cx, __dmul_rn(dX, c)), __dmul_rn(dZ, s));
    const double Zr = __dadd_rn(__dsub_rn(cz, __dmul_rn(dX, s)), __dmul_rn(dZ, c));
    const bool inside = X > margin && X < nx - margin && Z > margin && Z < nz - margin;
    int hmax = 0;
    if (inside) {
        for (int b = 0; b < n; ++b) {
            const double* q = boxes + 5 * b;
            const int h = (int)rint(q[4]);
            if (h <= 0) continue;
            if (Xr >= q[0] && Xr < q[1] && Zr >= q[2] && Zr < q[3]) hmax = max(hmax, min(h, ny - 1));
        }
    }
    for (int y = 0; y < ny; ++y) flags[((size_t)z * ny + y) * nx + x] = y < hmax ? WF_CELL_SOLID : WF_CELL_FLUID;
}

}  // namespace

extern "C" int wf_rasterise_boxes(int nx, int ny, int nz, const double* boxes, int n_boxes, double angle_deg,
                                  int margin, int device, int32_t* flags) {
    if (nx < 1 || ny < 1 || nz < 1 || n_boxes < 0 || (n_boxes > 0 && !boxes) || !flags || margin < 0)
        return WF_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return WF_ERR_CUDA;
    const size_t n = (size_t)nx * ny * nz;
    // the angle's sine and cosine on the host, as the generator computes them
    const double th = angle_deg * (M_PI / 180.0);
    const double c = std::cos(th), s = std::sin(th);
    double* db = nullptr;
    int32_t* df = nullptr;
    int st = WF_OK;
    if (cudaMalloc((void**)&df, n * sizeof(int32_t)) != cudaSuccess) st = WF_ERR_OOM;
    if (st == WF_OK && n_boxes > 0 && cudaMalloc((void**)&db, 5 * (size_t)n_boxes * sizeof(double)) != cudaSuccess)
        st = WF_ERR_OOM;
    if (st == WF_OK && n_boxes > 0 &&
        cudaMemcpy(db, boxes, 5 * (size_t)n_boxes * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        st = WF_ERR_CUDA;
    if (st == WF_OK) {
        const dim3 b(32, 8), g((nx + 31) / 32, (nz + 7) / 8);
        k_raster<<<g, b>>>(nx, ny, nz, db, n_boxes, c, s, margin, df);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpy(flags, df, n * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
            st = WF_ERR_CUDA;
    }
    if (db) cudaFree(db);
    if (df) cudaFree(df);
    if (st != WF_OK) cudaGetLastError();
    return st;
}
