// wf_common.cuh - shared device definitions of the windfvm CUDA library.
//
// Device layout (private to the library): every scalar field is one plane of
// N = nx*ny*nz FP32 values, x fastest (index (z*ny + y)*nx + x, the reference's
// host layout, InitShaderColl.compute:353).  A vector field is three such
// planes back to back (SoA: component c at base + c*N).  Flags are one byte
// per cell (0 fluid, 1 solid).  Boundary planes are SoA too: X planes ny*nz
// (index z*ny+y), Y planes nx*nz (z*nx+x), Z planes nx*ny (y*nx+x), matching
// the reference's Texture2D addressing bndFieldX0[int2(y, z)] etc.
#pragma once
#include <cstddef>
#include <cstdint>
#include <initializer_list>

#include "../../include/windfvm.h"

namespace wf {

// Kernels launched by this thread through the library (counted by every
// launch site; wf_step reports the per-step total).
extern thread_local long long g_launches;
#define WF_COUNT_LAUNCH() (++::wf::g_launches)

// Scalars and switches of one solver, passed by value to every kernel.
struct Params {
    int nx, ny, nz;
    int N;          // nx*ny*nz (checked < 2^31 / 4 at create)
    int plane[6];   // point count of each boundary plane
    float dx, ds, dv, dt, nu, den, cs;
    // Reciprocals computed once on the host: x * rdx in place of x / dx (and
    // the like) saves an IEEE division per use.  Exact where dx and den are
    // powers of two (every benchmarked workload: dx = 0.5, den = 1); within one
    // rounding of the quotient otherwise.  dvden = dv / den is the quotient
    // itself.
    float rdx, rdx2, rden, dvden;
    float force[3];
    int vbc[6], pbc[6];
    int les;
    unsigned compat;
    int vec4;       // != 0: four-cells-per-thread kernels where nx % 4 == 0
    // per-cell neighbour mask (see nb_fluid): bit f (0..5) = the neighbour
    // across face f is inside the domain and fluid, bit 6 = the cell is fluid
    const uint8_t* nbm;
};

// Boundary planes: base pointer of each plane (3 SoA components of
// plane[f] points each).
struct Bnd {
    const float* p[6];
};

// Face f in {E, W, N, S, U, D} = {0..5}: the order every reference kernel
// accumulates its face terms in.
__host__ __device__ __forceinline__ constexpr int face_ox(int f) { return f == 0 ? 1 : (f == 1 ? -1 : 0); }
__host__ __device__ __forceinline__ constexpr int face_oy(int f) { return f == 2 ? 1 : (f == 3 ? -1 : 0); }
__host__ __device__ __forceinline__ constexpr int face_oz(int f) { return f == 4 ? 1 : (f == 5 ? -1 : 0); }
__host__ __device__ __forceinline__ constexpr int face_axis(int f) { return f >> 1; }
__host__ __device__ __forceinline__ constexpr int face_sign(int f) { return (f & 1) ? -1 : 1; }
// Domain face crossed by face f of a boundary cell.
__host__ __device__ __forceinline__ constexpr int face_bc(int f) {
    return f == 0 ? WF_FACE_XN : f == 1 ? WF_FACE_X0 : f == 2 ? WF_FACE_YN
         : f == 3 ? WF_FACE_Y0 : f == 4 ? WF_FACE_ZN : WF_FACE_Z0;
}

__device__ __forceinline__ bool in_region(const Params& P, int x, int y, int z) {
    return (unsigned)x < (unsigned)P.nx && (unsigned)y < (unsigned)P.ny && (unsigned)z < (unsigned)P.nz;
}
__device__ __forceinline__ int cidx(const Params& P, int x, int y, int z) {
    return (z * P.ny + y) * P.nx + x;
}
// Index offset of the neighbour across face f.
__device__ __forceinline__ int face_off(const Params& P, int f) {
    return f == 0 ? 1 : f == 1 ? -1 : f == 2 ? P.nx : f == 3 ? -P.nx : f == 4 ? P.nx * P.ny : -(P.nx * P.ny);
}
// The neighbour across face f of cell (x, y, z) is inside the domain.
__device__ __forceinline__ bool face_in(const Params& P, int x, int y, int z, int f) {
    return f == 0 ? x + 1 < P.nx : f == 1 ? x > 0 : f == 2 ? y + 1 < P.ny : f == 3 ? y > 0 : f == 4 ? z + 1 < P.nz : z > 0;
}
__device__ __forceinline__ bool nb_fluid(unsigned mask, int f) { return (mask >> f) & 1u; }
// Index of the neighbour across face f, or of the cell itself where that
// neighbour is outside the domain: always a valid index, so a kernel can load
// from every face before it knows which faces count.
__device__ __forceinline__ int nb_idx(const Params& P, int x, int y, int z, int i, int f) {
    return face_in(P, x, y, z, f) ? i + face_off(P, f) : i;
}
__device__ __forceinline__ int plane_idx(const Params& P, int bc, int x, int y, int z) {
    return bc <= WF_FACE_XN ? z * P.ny + y : (bc <= WF_FACE_YN ? z * P.nx + x : y * P.nx + x);
}
__device__ __forceinline__ float bnd_comp(const Params& P, const Bnd& B, int bc, int x, int y, int z, int c) {
    return __ldg(B.p[bc] + (size_t)c * P.plane[bc] + plane_idx(P, bc, x, y, z));
}

// The three components of the momentum diagonal D (and of 1/D) are bit-
// identical in every cell but those with a domain-boundary face under a
// symmetry velocity condition: there the diffusion term adds to the normal
// component only (FvmColl.compute:1666,1699,1732,1765,1798,1831); every other
// term of D adds one value to all three.  True when any of the cells x0..x1
// of row (y, z) is such a cell, i.e. where a sweep must read all three
// components of 1/D rather than the first one alone.
__device__ __forceinline__ bool d_split(const Params& P, int x0, int x1, int y, int z) {
    return (x0 == 0 && P.vbc[WF_FACE_X0] == WF_BND_SYMMETRY) ||
           (x1 == P.nx - 1 && P.vbc[WF_FACE_XN] == WF_BND_SYMMETRY) ||
           (y == 0 && P.vbc[WF_FACE_Y0] == WF_BND_SYMMETRY) ||
           (y == P.ny - 1 && P.vbc[WF_FACE_YN] == WF_BND_SYMMETRY) ||
           (z == 0 && P.vbc[WF_FACE_Z0] == WF_BND_SYMMETRY) ||
           (z == P.nz - 1 && P.vbc[WF_FACE_ZN] == WF_BND_SYMMETRY);
}

// Programmatic dependent launch inside a chain of Jacobi sweeps.
// chain_wait: wait until the previous grid in the stream has completed and
// its writes are visible.  chain_release (after chain_wait): let the next
// launch of the chain be scheduled; it then starts once every block of
// this grid has passed this point, i.e. after the grid before this one has
// completed, so data written before that grid (the step's coefficient
// planes) may be read before the next grid's own chain_wait.  Without the
// launch attribute both calls return at once.
__device__ __forceinline__ void chain_wait() { cudaGridDependencySynchronize(); }
__device__ __forceinline__ void chain_release() { cudaTriggerProgrammaticLaunchCompletion(); }

// Launches kernel<<<grid, block, 0, st>>>(args...), as a programmatic
// dependent launch when `chained` (the kernel calls chain_wait before it
// reads the previous grid's output, then chain_release).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_chained(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, bool chained,
                                  Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = chained ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Where a four-cells-per-thread kernel applies: the switch (Params::vec4),
// nx % 4 == 0 and 16-byte aligned planes.
inline bool quad_ok(const Params& P, std::initializer_list<const void*> ptrs) {
    if (!P.vec4 || P.nx % 4 != 0) return false;
    for (const void* p : ptrs)
        if (p && (reinterpret_cast<uintptr_t>(p) & 15u) != 0) return false;
    return true;
}

}  // namespace wf
