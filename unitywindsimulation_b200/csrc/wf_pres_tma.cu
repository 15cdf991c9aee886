// wf_pres_tma.cu - four pressure Jacobi sweeps per pass with TMA-staged
// halo tiles (CSPresCorrectRhieChow, FvmColl.compute:2790-2848, and
// CSPisoPresCorrection, PisoColl.compute:181-256).
//
// Same 2.5D wavefront as k_pres_msweep<4, 32> (wf_sweeps.cu): a block owns a
// 32 x 32 column tile of the x-y plane (a 24 x 24 output tile with a 4-cell
// halo on every side) and streams a chunk of z planes; level s (1..4) is
// sweep s and computes plane zs + t - s at step t.  The block has 32 x 16
// threads, each owning two adjacent tile rows (TR), so one of each row's two
// y neighbours and one south face coefficient come from the thread's own
// registers; 16 warps per SM with two independent cells each.
// What differs is how a plane reaches shared memory.  Each z plane of the
// tile arrives as six 32 x 32 FP32 planes (24 KB): c_E and c_N (one 4-D
// tensor-map box of two consecutive planes of the coefficient cache), c_U,
// 1/Dp, the right-hand side and the input iterate (3-D boxes), written by up
// to five cp.async.bulk.tensor loads that complete on one mbarrier.  With a
// `stack` the pass also writes every level of every cell (the adjoint's
// taped and reversed loops).  One thread
// issues them TD planes ahead of the plane the block consumes, into two
// rings (below) that hold every plane a level still reads.  So no thread
// issues a global load or a staging store: per step a thread reads its own
// column's new values (input, c_E, c_N, c_U, 1/Dp, rhs) into register rings
// and, per level, the four neighbour values and the west and south face
// coefficients from shared memory, at offsets the unrolled z loop fixes at
// compile time.
//
// Out-of-domain cells: the tensor maps' bounds give zeros outside the domain
// (a box may start at x = -4, y = -4 or a plane below 0, and run past the
// far edges), which is the reference's InRegion test without branches.
// Non-fluid cells have 1/Dp = 0 and are never written.
// The arithmetic, its order and every stored value are those of
// k_pres_msweep<4, 32>, so the two kernels give bit-identical iterates.
//
// Every wait on a stage's mbarrier is bounded (kWaitNs of %globaltimer).  A
// wait that runs out sets *status, the block agrees on the failure at its
// next barrier, the issuing thread waits (bounded again) for the loads it
// still has in flight, and every thread returns; the host reports
// WF_ERR_TIMEOUT.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "wf_sweeps.cuh"
#include "wf_tma.cuh"

namespace wf {
namespace {

using namespace tma;

constexpr int TK = 4;              // sweeps per pass
constexpr int TT = 32;             // tile edge (threads per row, rows)
constexpr int TO = TT - 2 * TK;    // output tile edge
#ifndef WF_TMA_AHEAD
#define WF_TMA_AHEAD 3
#endif
constexpr int TD = WF_TMA_AHEAD;   // planes loaded ahead of the consumed one
constexpr int TPL = TT * TT;       // floats per tile plane
// Two rings.  The face ring holds c_E, c_N of a plane (the x/y neighbours of
// every level read them, level K four steps after the plane arrived); the
// column ring holds c_U, 1/Dp, rhs and the input iterate (read into the own
// column's registers when the plane arrives, the input also as level 1's
// neighbours one step later).  The z loop is unrolled by TU steps, a
// multiple of both ring lengths and of every register-ring period, so every
// slot, mbarrier and parity below is a compile-time constant.
constexpr int TU = 12;             // unrolled z steps per loop trip
constexpr int TF = 12;             // face-ring slots (plane t in slot t % TF)
constexpr int TC = 6;              // column-ring slots, one mbarrier each
enum { F_CE = 0, F_CN = 1, TFQ = 2 };
enum { C_CU = 0, C_AI = 1, C_RHS = 2, C_PIN = 3, TCQ = 4 };
constexpr int kFace = TFQ * TPL;   // floats per face-ring slot
constexpr int kCol = TCQ * TPL;    // floats per column-ring slot
constexpr int kR = 6;              // register-ring period (c_U, 1/Dp, rhs)
// shared memory: the two rings, level planes 1..K-1 (double-buffered), TC
// mbarriers; plus slack to align the base to 1 KB.
constexpr size_t kSmemFloats = (size_t)TF * kFace + (size_t)TC * kCol + (size_t)(TK - 1) * 2 * TPL;
constexpr size_t kSmemBytes = kSmemFloats * sizeof(float) + TC * sizeof(unsigned long long) + 1024;
constexpr unsigned long long kWaitNs = 1000000000ull;  // default limit of one wait: 1 s

static_assert(TO % 4 == 0 && TK % 4 == 0, "tile origins x = bx*TO - TK must be 16-byte aligned");
static_assert(kSmemBytes <= 232448, "rings exceed the shared memory of one block");
static_assert(TU % TF == 0 && TU % TC == 0 && TU % kR == 0 && TU % 3 == 0 && TU % 2 == 0,
              "the unrolled trip must be a multiple of every ring period");
// Slot reuse: the column slot of plane t is refilled (at the end of step
// t - 1 - TD + TC) after its last reader, level 1 at step t + 1; the face
// slot after level K's read at step t + K.
static_assert(TD + 2 <= TC && TK + 1 + TD <= TF, "rings too short for the prefetch distance");

struct TmaMaps {
    CUtensorMap face;  // 4-D {nx, ny, nz, 2} (c_E, c_N), box of both planes
    CUtensorMap cu;    // 3-D {nx, ny, nz}: c_U
    CUtensorMap ai;    // 3-D {nx, ny, nz}: 1/Dp
    CUtensorMap rhs;   // 3-D {nx, ny, nz}
    CUtensorMap pin;   // 3-D {nx, ny, nz}
};

// One block of TT x (TT / R) threads; thread (tx, j) owns the R adjacent
// tile rows R*j .. R*j + R - 1 of column tx.  With R = 2 a thread's second
// row takes its south neighbour values and south face coefficient, and its
// first row its north neighbour values, from the thread's own registers.
template <int R>
struct TmaWave {
    float* face;            // TF slots of kFace floats
    float* colr;            // TC slots of kCol floats
    float (*V)[2][TT][TT];  // V[s - 1]: level s = 1..K-1
    unsigned bar0;          // shared address of mbarrier 0 (column slot c: bar0 + 8c)
    const TmaMaps* maps;
    float* __restrict__ pout;
    float* __restrict__ pprev;
    float* __restrict__ stack;  // optional: level s of every cell to stack + s*N
    size_t N;
    int me, xe, xw, yn, ys;  // row 0: own, east, west offsets; north of the last row, south of row 0
    int r0, zs, z0, z1, T, sxy, x0, y0, tfail;
    int col[R];             // grid index (x, y) of each row's column
    unsigned long long wait_ns;
    unsigned extra_tx;      // self-test: bytes the block's first stage expects beyond its loads
    unsigned tx_bytes;      // bytes the loads of one plane deliver
    bool out_col[R];
    bool has_rhs, has_pin, bad, lead;
    float h[R][TK + 1][3];            // level values, ring of the last 3 planes
    float qa[R][kR], qr[R][kR], qu[R][kR];  // own column's 1/Dp, rhs, c_U of the last kR planes
    float qe[R][kR], qn[R][kR];       // own column's c_E, c_N of the last kR planes

    // Issued by thread 0: the loads of plane zs + t (t = trip base + PH)
    // into face slot PH % TF and column slot PH % TC, completing on the
    // column slot's mbarrier.  Planes outside [0, nz) read as zeros.
    template <int PH>
    __device__ __forceinline__ void issue(int t) const {
        constexpr int fs = PH % TF, cs = PH % TC;
        const unsigned bar = bar0 + cs * 8;
        const int p = zs + t;
        const unsigned fdst = smem_addr(face + fs * kFace);
        const unsigned cdst = smem_addr(colr + cs * kCol);
        mbar_expect(bar, tx_bytes + (t == 0 ? extra_tx : 0u));
        tma_4d(fdst, &maps->face, x0, y0, p, 0, bar);  // c_E, c_N
        tma_3d(cdst + sizeof(float) * TPL * C_CU, &maps->cu, x0, y0, p, bar);
        tma_3d(cdst + sizeof(float) * TPL * C_AI, &maps->ai, x0, y0, p, bar);
        if (has_rhs) tma_3d(cdst + sizeof(float) * TPL * C_RHS, &maps->rhs, x0, y0, p, bar);
        if (has_pin) tma_3d(cdst + sizeof(float) * TPL * C_PIN, &maps->pin, x0, y0, p, bar);
    }

    // Step t = trip base + PH: plane zs + t enters level 0, level s computes
    // plane zs + t - s.  Planes before zs (t < s) feed only values outside
    // the pass's dependency cone; their slots hold zeros.
    template <int PH>
    __device__ __forceinline__ void step(int t) {
        if (t >= T) return;  // uniform over the block
        constexpr int cur = PH & 1, prv = cur ^ 1;
        constexpr int h0 = PH % 3, hm1 = (PH + 2) % 3, hm2 = (PH + 1) % 3;
        constexpr int cs = PH % TC;
        constexpr unsigned parity = (PH / TC) & 1;  // use t / TC of the slot; TU / TC is even
        if (!bad) bad = !mbar_wait(bar0 + cs * 8, parity, wait_ns);
        // plane zs + t enters level 0 and the own-column rings
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const float* cn = colr + cs * kCol + me + k * TT;
            h[k][0][h0] = cn[C_PIN * TPL];
            qu[k][PH % kR] = cn[C_CU * TPL];
            qa[k][PH % kR] = cn[C_AI * TPL];
            qr[k][PH % kR] = cn[C_RHS * TPL];
            qe[k][PH % kR] = face[(PH % TF) * kFace + F_CE * TPL + me + k * TT];
            qn[k][PH % kR] = face[(PH % TF) * kFace + F_CN * TPL + me + k * TT];
        }
#pragma unroll
        for (int s = 1; s <= TK; ++s) {
            // rows this level must produce: [s, TT - s); a thread computes all
            // its rows when any of them is in that range (the others give values
            // no later level reads)
            if (r0 + R - 1 >= s && r0 < TT - s) {
                const int rs = (PH - s + 2 * kR) % kR;
                const int rd = (PH - s - 1 + 2 * kR) % kR;
                const float* fq = face + ((PH - s + TF) % TF) * kFace;
                // level s-1 on plane zs+t-s: the input iterate (column ring) or a level plane
                const float* L = s == 1 ? colr + ((PH - 1 + TC) % TC) * kCol + C_PIN * TPL : &V[s - 2][prv][0][0];
                float v[R];
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    // level s-1 on plane zs+t-s in the rows above and below,
                    // and the south face coefficient
                    const float ln = k + 1 < R ? h[k + 1][s - 1][hm1] : L[yn];
                    const float ls = k > 0 ? h[k - 1][s - 1][hm1] : L[ys];
                    const float cs_ = k > 0 ? qn[k - 1][rs] : fq[F_CN * TPL + ys];
                    float acc = -(qe[k][rs] * L[xe + k * TT]);
                    acc -= fq[F_CE * TPL + xw + k * TT] * L[xw + k * TT];
                    acc -= qn[k][rs] * ln;
                    acc -= cs_ * ls;
                    acc -= qu[k][rs] * h[k][s - 1][h0];
                    acc -= qu[k][rd] * h[k][s - 1][hm2];
                    v[k] = qa[k][rs] * (acc + qr[k][rs]);
                }
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    if (stack) {  // every level, non-fluid cells included (v = 0 there)
                        const int q = zs + t - s;
                        if (out_col[k] && q >= z0 && q < z1) stack[(size_t)s * N + q * sxy + col[k]] = v[k];
                    }
                    if (s == TK && pout) {
                        const int q = zs + t - TK;
                        if (out_col[k] && q >= z0 && q < z1 && qa[k][rs] != 0.f) {
                            const int i = q * sxy + col[k];
                            pout[i] = v[k];
                            if (pprev) pprev[i] = h[k][TK - 1][hm1];
                        }
                    }
                    h[k][s][h0] = v[k];
                    if (s < TK) (&V[s - 1][cur][0][0])[me + k * TT] = v[k];
                }
            }
        }
        // every read of step t is done: the slots of plane zs + t + 1 + TD
        // (last read by level 1 at step t + TD + 2 - TC and by level K at
        // step t + TD + 1 + K - TF) may be refilled
        if (__syncthreads_or(bad)) {
            bad = true;
            tfail = t;
            return;
        }
        if (lead && t + 1 + TD < T) issue<(PH + 1 + TD) % TU>(t + 1 + TD);
    }
};

// Prologue: thread 0 issues planes 0..TD.
template <int P, int R>
__device__ __forceinline__ void issue_first(const TmaWave<R>& w) {
    if constexpr (P <= TD) {
        if (P < w.T) w.template issue<P>(P);
        issue_first<P + 1>(w);
    }
}

// Steps t0 + PH .. t0 + TU - 1 of one unrolled trip; false once a wait ran out.
template <int PH, int R>
__device__ __forceinline__ bool trip(TmaWave<R>& w, int t0) {
    if constexpr (PH < TU) {
        w.template step<PH>(t0 + PH);
        if (w.bad) return false;
        return trip<PH + 1>(w, t0);
    } else {
        return true;
    }
}

static_assert((TU / TC) % 2 == 0, "a trip must advance every column slot by an even number of uses");

#ifndef WF_TMA_ROWS
#define WF_TMA_ROWS 2
#endif
// Tile rows per thread.  Measured on the 256 x 96 x 192 urban block, four
// sweeps per pass, on two machines: 68.3 / 87.1 us with one row (1024
// threads), 65.7 / 73.0 us with two (512 threads), 78.9 us (first machine)
// with four (256 threads); bit-identical iterates.
constexpr int TR = WF_TMA_ROWS;
static_assert(TT % TR == 0, "rows per thread must divide the tile");

__global__ void __launch_bounds__(TT* TT / TR, 1)
    k_pres_tma4(const __grid_constant__ TmaMaps maps, int nx, int ny, int nz, int has_rhs, int has_pin,
                float* __restrict__ pout, float* __restrict__ pprev, int zchunk, float* __restrict__ stack,
                int* __restrict__ status, unsigned long long wait_ns, unsigned extra_tx) {
    extern __shared__ __align__(1024) unsigned char tsm_raw[];
    // offset (not an integer round trip) keeps every pointer in the shared
    // window, so the compiler emits shared-memory loads
    const unsigned pad = (1024u - (smem_addr(tsm_raw) & 1023u)) & 1023u;
    float* base = reinterpret_cast<float*>(tsm_raw + pad);
    TmaWave<TR> w;
    w.face = base;
    w.colr = base + TF * kFace;
    w.V = reinterpret_cast<float(*)[2][TT][TT]>(w.colr + TC * kCol);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(w.colr + TC * kCol + (TK - 1) * 2 * TPL);
    w.bar0 = smem_addr(bars);
    w.maps = &maps;
    const int tx = threadIdx.x;
    const int tid = threadIdx.y * TT + tx;
    w.lead = tid == 0;
    w.r0 = threadIdx.y * TR;
    w.me = w.r0 * TT + tx;
    w.xe = w.r0 * TT + min(tx + 1, TT - 1);
    w.xw = w.r0 * TT + max(tx - 1, 0);
    w.yn = min(w.r0 + TR, TT - 1) * TT + tx;  // north of the last row
    w.ys = max(w.r0 - 1, 0) * TT + tx;        // south of the first row
    w.x0 = blockIdx.x * TO - TK;
    w.y0 = blockIdx.y * TO - TK;
    const int x = w.x0 + tx;
    w.z0 = blockIdx.z * zchunk;
    w.z1 = min(w.z0 + zchunk, nz);
#pragma unroll
    for (int k = 0; k < TR; ++k) {
        const int r = w.r0 + k, y = w.y0 + r;
        const bool inxy = x >= 0 && x < nx && y >= 0 && y < ny;
        w.out_col[k] = inxy && tx >= TK && tx < TT - TK && r >= TK && r < TT - TK;
        w.col[k] = inxy ? y * nx + x : 0;
    }
    w.sxy = nx * ny;
    w.pout = pout;
    w.pprev = pprev;
    w.stack = stack;
    w.N = (size_t)nx * ny * nz;
    w.has_rhs = has_rhs != 0;
    w.has_pin = has_pin != 0;
    w.tx_bytes = (unsigned)(sizeof(float) * TPL * (4 + (has_rhs ? 1 : 0) + (has_pin ? 1 : 0)));
    w.bad = false;
    w.tfail = 0;
    w.wait_ns = wait_ns;
    w.extra_tx = extra_tx;
    // The rings and the level planes start at zero (the rhs and input planes
    // stay zero when absent: no load writes them).
    static_assert(kSmemFloats % 4 == 0, "the rings are cleared with 16-byte stores");
    for (int i = tid; i < (int)(kSmemFloats / 4); i += TT * TT / TR)
        reinterpret_cast<float4*>(base)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < TR; ++k) {
#pragma unroll
        for (int r = 0; r < kR; ++r) w.qa[k][r] = w.qr[k][r] = w.qu[k][r] = w.qe[k][r] = w.qn[k][r] = 0.f;
#pragma unroll
        for (int s = 0; s <= TK; ++s) w.h[k][s][0] = w.h[k][s][1] = w.h[k][s][2] = 0.f;
    }
    w.zs = w.z0 - TK;
    w.T = (w.z1 - w.z0) + 2 * TK;
    if (w.lead) {
        for (int c = 0; c < TC; ++c) mbar_init(w.bar0 + c * 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // generic-proxy zeroing above before any async-proxy write to the rings
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (w.lead) issue_first<0>(w);
    for (int t0 = 0; t0 < w.T; t0 += TU)
        if (!trip<0>(w, t0)) break;
    if (w.bad && w.lead) {
        if (status) atomicExch(status, 1);
        // Loads still in flight: the plane of the failed step and the TD
        // planes issued ahead of it.  Wait for them (bounded) before the
        // block's shared memory is released.
        for (int t = w.tfail; t <= w.tfail + TD && t < w.T; ++t)
            mbar_wait(w.bar0 + (t % TC) * 8, (unsigned)((t / TC) & 1), wait_ns);
    }
}
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder() {
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}

#ifndef WF_TMA_L2P
#define WF_TMA_L2P CU_TENSOR_MAP_L2_PROMOTION_L2_256B
#endif
constexpr CUtensorMapL2promotion kL2Promotion = WF_TMA_L2P;

}  // namespace

bool tma_available() { return encoder() != nullptr; }

bool tma_encode(CUtensorMap* m, const Params& P, const float* base, int planes, int box_w, int box_h,
                int box_planes) {
    EncodeFn fn = encoder();
    if (!fn || !base) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)P.nx, (cuuint64_t)P.ny, (cuuint64_t)P.nz, (cuuint64_t)planes};
    const cuuint64_t strides[3] = {sizeof(float) * (cuuint64_t)P.nx, sizeof(float) * (cuuint64_t)P.nx * P.ny,
                                   sizeof(float) * (cuuint64_t)P.N};
    const cuuint32_t box[4] = {(cuuint32_t)box_w, (cuuint32_t)box_h, 1, (cuuint32_t)box_planes};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, planes > 1 ? 4 : 3, const_cast<float*>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, kL2Promotion,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

namespace {

// Map of this pass's 32 x 32 tiles.
bool encode(CUtensorMap* m, const Params& P, const float* base, int planes, int box_planes) {
    return tma_encode(m, P, base, planes, TT, TT, box_planes);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

size_t pres_tma_smem() { return kSmemBytes; }
const void* pres_tma_kernel() { return reinterpret_cast<const void*>(k_pres_tma4); }

bool pres_tma_ok(const Params& P, const float* c3, const float* ainv, const float* rhs, const float* in) {
    return P.nx % 4 == 0 && c3 && ainv && aligned16(c3) && aligned16(ainv) && aligned16(rhs) && aligned16(in) &&
           tma_available();
}

cudaError_t launch_pres_tma4(const Params& P, cudaStream_t st, int sms, const float* c3, const float* ainv,
                             const float* rhs, const float* in, float* out, float* prev, float* stack, int* status,
                             double wait_ms, bool short_stage) {
    TmaMaps maps;
    std::memset(&maps, 0, sizeof(maps));
    if (!encode(&maps.face, P, c3, 2, 2) || !encode(&maps.cu, P, c3 + 2 * (size_t)P.N, 1, 1) ||
        !encode(&maps.ai, P, ainv, 1, 1))
        return cudaErrorInvalidValue;
    if (rhs && !encode(&maps.rhs, P, rhs, 1, 1)) return cudaErrorInvalidValue;
    if (in && !encode(&maps.pin, P, in, 1, 1)) return cudaErrorInvalidValue;
    const int gx = (P.nx + TO - 1) / TO, gy = (P.ny + TO - 1) / TO;
    sms = sms > 0 ? sms : 148;
    int nchunk = std::max(1, sms / std::max(gx * gy, 1));
    const int zchunk = std::max(2 * TK + 2, (P.nz + nchunk - 1) / nchunk);
    nchunk = (P.nz + zchunk - 1) / zchunk;
    WF_COUNT_LAUNCH();
    const unsigned long long wait_ns = wait_ms > 0 ? (unsigned long long)(wait_ms * 1e6) : kWaitNs;
    k_pres_tma4<<<dim3(gx, gy, nchunk), dim3(TT, TT / TR), kSmemBytes, st>>>(
        maps, P.nx, P.ny, P.nz, rhs ? 1 : 0, in ? 1 : 0, out, prev, zchunk, stack, status, wait_ns,
        short_stage ? 16u : 0u);
    return cudaGetLastError();
}

}  // namespace wf
