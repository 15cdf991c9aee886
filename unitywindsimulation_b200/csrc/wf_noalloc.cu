// wf_noalloc.cu - pressure-correction residual that allocates no device memory.
//
// Some hosts cannot call cudaMalloc from the code that wants this number: a
// plugin inside a game engine or visualiser whose device memory is owned and
// budgeted by the engine, a real-time loop where cudaMalloc's implicit device
// synchronisation would stall a frame, or a process whose allocator is
// locked down.  They keep their fields in memory someone else allocated and
// only need the reduction.  This entry point does the reduction with a
// fixed scratch array that lives in the library image instead of on the
// heap: the block partial sums go to g_noalloc_scratch, a file-scope
// __device__ array of WF_NOALLOC_BLOCKS + 1 doubles (32 KiB + 8 B) that
// every GPU loading the library holds until the process exits.
#include <cuda_runtime.h>

#include <cmath>

#include "wf_common.cuh"

namespace {

constexpr int kThreads = 256;

// Block partial sums [0, WF_NOALLOC_BLOCKS) and the final sum at
// [WF_NOALLOC_BLOCKS].  Shared by every call on a device.
static __device__ __align__(256) double g_noalloc_scratch[WF_NOALLOC_BLOCKS + 1];

__global__ void k_noalloc_partials(const float* __restrict__ dp, const float* __restrict__ pc,
                                   const float* __restrict__ pcl, long long n, double* __restrict__ part) {
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)kThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kThreads) {
        const float a = __ldg(pc + i);
        const float b = pcl ? __ldg(pcl + i) : 0.f;
        const float l = __ldg(dp + i) * (a - b);
        s += (double)(l * l);
    }
    __shared__ double sh[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double r = threadIdx.x < kThreads / 32 ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        if (threadIdx.x == 0) part[blockIdx.x] = r;  // every slot < gridDim.x is written
    }
}

__global__ void k_noalloc_total(double* __restrict__ scratch, int nblocks) {
    __shared__ double sh[kThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += kThreads) s += scratch[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int st = kThreads / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) scratch[WF_NOALLOC_BLOCKS] = sh[0];
}

// The device address of the scratch array in the CUDA context current on
// the calling thread.  Looked up on every call rather than cached: an address
// belongs to one context, and a host may call from a context it created
// itself, or after cudaDeviceReset replaced the primary context.  The lookup
// allocates nothing; the first one in a context loads the library's device
// code into it.  Host code must never pass g_noalloc_scratch itself to a
// kernel: on the host the name is a stand-in, not device memory.
int scratch_for_current_context(double** out) {
    double* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) return WF_ERR_CUDA;
    *out = p;
    return WF_OK;
}

// Launches kernel<<<grid, block, 0, st>>>(args...) and returns that launch's
// own status (not an error left behind by some earlier, unrelated call).
template <typename... KArgs, typename... Args>
cudaError_t launch(void (*kernel)(KArgs...), int grid, int block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace

extern "C" int wf_pres_residual_noalloc(const float* d_dp, const float* d_pc, const float* d_pc_last,
                                        int64_t n_cells, void* stream, float* out) {
    if (!d_dp || !d_pc || !out) return WF_ERR_INVALID_ARG;
    if (n_cells < 1 || n_cells > (int64_t)WF_NOALLOC_MAX_CELLS) return WF_ERR_INVALID_ARG;
    double* scratch = nullptr;
    const int s = scratch_for_current_context(&scratch);
    if (s != WF_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    long long want = (n_cells + kThreads - 1) / kThreads;
    const int nblocks = (int)(want < WF_NOALLOC_BLOCKS ? want : WF_NOALLOC_BLOCKS);
    if (launch(k_noalloc_partials, nblocks, kThreads, st, d_dp, d_pc, d_pc_last, (long long)n_cells, scratch) !=
        cudaSuccess)
        return WF_ERR_CUDA;
    if (launch(k_noalloc_total, 1, kThreads, st, scratch, nblocks) != cudaSuccess) return WF_ERR_CUDA;
    double total = 0.0;
    if (cudaMemcpyAsync(&total, scratch + WF_NOALLOC_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
        return WF_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return WF_ERR_CUDA;
    *out = (float)std::sqrt(total / (double)n_cells);
    return WF_OK;
}
