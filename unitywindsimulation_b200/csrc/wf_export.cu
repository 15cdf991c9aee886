// wf_export.cu - field export while the solver runs.
//
// Counterpart of NcFlowFieldExporter (NcFlowFieldExporter.cs:197-393): the
// same file layout (netCDF dimensions time/velX/velY/velZ/velVec/presX/
// presY/presZ, coordinate variables at cell centres, global attributes
// gridLayoutType and dt, record variables velField[time][z][y][x][4] and
// presField[time][z][y][x]) written without libnetcdf: the file is netCDF
// classic with 64-bit offsets (CDF-2), laid out here directly.
//
// Pipeline per frame: a kernel on the solver's stream turns the SoA fields
// into the file's record (x fastest, four velocity channels, big-endian) in
// a device staging buffer, one asynchronous copy moves it into a pinned
// host slot, and a writer thread waits for the copy's event and writes the
// record at its offset.  A ring of pinned slots bounds the frames in flight;
// wf_export_frame blocks only when every slot is still being written.  The
// reference's equivalent is AsyncGPUReadback into NativeArrays plus a
// ConcurrentQueue drained by a writer thread (:300-393).
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "wf_kernels.cuh"
#include "wf_solver.cuh"

namespace wf {
namespace {

__device__ __forceinline__ unsigned be32(float v) { return __byte_perm(__float_as_uint(v), 0, 0x0123); }

// Record of one frame: [time][velField (4 channels, w = 0)][presField],
// big-endian.  velrec / presrec: the two field parts (either may be null).
__global__ void k_pack_record(long long n, const float* __restrict__ vel, const float* __restrict__ pr,
                              unsigned* __restrict__ velrec, unsigned* __restrict__ presrec) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (velrec) {
        uint4 q;
        q.x = be32(__ldg(vel + i));
        q.y = be32(__ldg(vel + n + i));
        q.z = be32(__ldg(vel + 2 * n + i));
        q.w = 0u;
        reinterpret_cast<uint4*>(velrec)[i] = q;
    }
    if (presrec) presrec[i] = be32(__ldg(pr + i));
}

// ---- netCDF classic (CDF-2) header writer ----
struct Bytes {
    std::vector<unsigned char> b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void f32(float f) {
        uint32_t v;
        std::memcpy(&v, &f, 4);
        u32(v);
    }
    void name(const std::string& s) {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        while (b.size() % 4) b.push_back(0);
    }
};
enum : uint32_t { NC_DIMENSION = 0x0A, NC_VARIABLE = 0x0B, NC_ATTRIBUTE = 0x0C, NC_CHAR = 2, NC_FLOAT = 5 };

struct Var {
    std::string name;
    std::vector<int> dims;  // dimension ids
    bool record;
    uint64_t vsize;         // bytes of one record slice (or of the whole variable)
    uint64_t begin = 0;
};

}  // namespace
}  // namespace wf

struct wf_exporter {
    wf_solver* h = nullptr;
    FILE* f = nullptr;
    std::string path, err;
    bool vel = true, pres = true;
    size_t N = 0;
    uint64_t rec_begin = 0, recsize = 0, vel_off = 0, pres_off = 0;  // offsets inside a record
    unsigned char* dstage = nullptr;               // device record staging (record at dstage + 12,
                                                   // so the velocity part is 16-byte aligned)
    std::vector<unsigned char*> slots;             // pinned host records
    std::vector<cudaEvent_t> ev;
    std::vector<int> busy;                         // slot in flight
    std::deque<std::pair<int, int64_t>> queue;     // (slot, record index)
    int64_t next_record = 0, written = 0;
    bool stop = false, failed = false;
    std::mutex m;
    std::condition_variable cv;
    std::thread writer;
};

namespace {

using wf::Bytes;
using wf::Var;

// Lays out the header and the non-record variables; returns the header
// bytes and sets every variable's begin offset.
std::vector<unsigned char> build_header(wf_exporter* e, std::vector<Var>& vars, std::vector<std::vector<float>>& data) {
    const wf_solver* h = e->h;
    const int nx = h->P.nx, ny = h->P.ny, nz = h->P.nz;
    const float dx = h->cfg.dx;
    // dimensions: 0 time (record), 1 velX, 2 velY, 3 velZ, 4 velVec, 5 presX, 6 presY, 7 presZ
    const char* dn[8] = {"time", "velX", "velY", "velZ", "velVec", "presX", "presY", "presZ"};
    const uint32_t dl[8] = {0, (uint32_t)nx, (uint32_t)ny, (uint32_t)nz, 4, (uint32_t)nx, (uint32_t)ny, (uint32_t)nz};
    vars.clear();
    data.clear();
    auto coord = [&](const char* name, int dim, int n, float scale, float shift) {
        Var v{name, {dim}, false, 4ull * n};
        vars.push_back(v);
        std::vector<float> d(n);
        for (int i = 0; i < n; ++i) d[i] = (i + shift) * scale;
        data.push_back(d);
    };
    vars.push_back(Var{"time", {0}, true, 4});
    data.push_back({});
    coord("velX", 1, nx, dx, 0.5f);
    coord("velY", 2, ny, dx, 0.5f);
    coord("velZ", 3, nz, dx, 0.5f);
    coord("velVec", 4, 4, 1.f, 0.f);
    coord("presX", 5, nx, dx, 0.5f);
    coord("presY", 6, ny, dx, 0.5f);
    coord("presZ", 7, nz, dx, 0.5f);
    const uint64_t cells = (uint64_t)nx * ny * nz;
    if (e->vel) {
        vars.push_back(Var{"velField", {0, 3, 2, 1, 4}, true, 16ull * cells});
        data.push_back({});
    }
    if (e->pres) {
        vars.push_back(Var{"presField", {0, 7, 6, 5}, true, 4ull * cells});
        data.push_back({});
    }
    auto encode = [&](uint64_t numrecs) {
        Bytes H;
        H.b = {'C', 'D', 'F', 2};
        H.u32((uint32_t)numrecs);
        H.u32(wf::NC_DIMENSION);
        H.u32(8);
        for (int d = 0; d < 8; ++d) {
            H.name(dn[d]);
            H.u32(dl[d]);
        }
        // global attributes gridLayoutType = "Collocated", dt
        H.u32(wf::NC_ATTRIBUTE);
        H.u32(2);
        H.name("gridLayoutType");
        H.u32(wf::NC_CHAR);
        const std::string gl = "Collocated";
        H.u32((uint32_t)gl.size());
        H.b.insert(H.b.end(), gl.begin(), gl.end());
        while (H.b.size() % 4) H.b.push_back(0);
        H.name("dt");
        H.u32(wf::NC_FLOAT);
        H.u32(1);
        H.f32(h->cfg.dt);
        H.u32(wf::NC_VARIABLE);
        H.u32((uint32_t)vars.size());
        for (const Var& v : vars) {
            H.name(v.name);
            H.u32((uint32_t)v.dims.size());
            for (int d : v.dims) H.u32((uint32_t)d);
            H.u32(0);  // no variable attributes (ABSENT)
            H.u32(0);
            H.u32(wf::NC_FLOAT);
            H.u32((uint32_t)std::min<uint64_t>(v.vsize, 0xFFFFFFFFull));
            H.u64(v.begin);
        }
        return H.b;
    };
    // first pass for the header size, then the offsets
    const size_t hsize = encode(0).size();
    uint64_t off = hsize;
    for (Var& v : vars)
        if (!v.record) {
            v.begin = off;
            off += v.vsize;
        }
    e->rec_begin = off;
    uint64_t roff = 0;
    for (Var& v : vars)
        if (v.record) {
            v.begin = off + roff;
            if (v.name == "velField") e->vel_off = roff;
            if (v.name == "presField") e->pres_off = roff;
            roff += v.vsize;
        }
    e->recsize = roff;
    return encode(0);
}

void writer_loop(wf_exporter* e) {
    cudaSetDevice(e->h->device);
    for (;;) {
        std::pair<int, int64_t> job;
        {
            std::unique_lock<std::mutex> lk(e->m);
            e->cv.wait(lk, [&] { return e->stop || !e->queue.empty(); });
            if (e->queue.empty()) return;  // stop requested and drained
            job = e->queue.front();
            e->queue.pop_front();
        }
        const int s = job.first;
        bool ok = cudaEventSynchronize(e->ev[s]) == cudaSuccess;
        const uint64_t off = e->rec_begin + (uint64_t)job.second * e->recsize;
        if (ok) ok = fseeko(e->f, (off_t)off, SEEK_SET) == 0 && fwrite(e->slots[s], 1, e->recsize, e->f) == e->recsize;
        {
            std::lock_guard<std::mutex> lk(e->m);
            e->busy[s] = 0;
            if (ok) {
                e->written = std::max<int64_t>(e->written, job.second + 1);
            } else if (!e->failed) {
                e->failed = true;
                e->err = "writing record " + std::to_string(job.second) + " of " + e->path + " failed";
            }
        }
        e->cv.notify_all();
    }
}

void free_exporter(wf_exporter* e) {
    if (e->f) fclose(e->f);
    for (unsigned char* p : e->slots)
        if (p) cudaFreeHost(p);
    for (cudaEvent_t v : e->ev)
        if (v) cudaEventDestroy(v);
    if (e->dstage) cudaFree(e->dstage);
}

}  // namespace

extern "C" {

int wf_export_open(wf_solver* h, const char* path, int save_vel, int save_pres, int ring, wf_exporter** out) {
    if (!h || !path || !out || (!save_vel && !save_pres) || ring < 1 || ring > 16) return WF_ERR_INVALID_ARG;
    *out = nullptr;
    if (cudaSetDevice(h->device) != cudaSuccess) return WF_ERR_CUDA;
    auto* e = new (std::nothrow) wf_exporter;
    if (!e) return WF_ERR_OOM;
    e->h = h;
    e->path = path;
    e->vel = save_vel != 0;
    e->pres = save_pres != 0;
    e->N = h->P.N;
    std::vector<Var> vars;
    std::vector<std::vector<float>> data;
    const std::vector<unsigned char> hdr = build_header(e, vars, data);
    e->f = fopen(path, "w+b");
    if (!e->f) {
        delete e;
        h->err = std::string("cannot create ") + path;
        return WF_ERR_IO;
    }
    bool ok = fwrite(hdr.data(), 1, hdr.size(), e->f) == hdr.size();
    for (size_t i = 0; ok && i < vars.size(); ++i) {
        if (vars[i].record) continue;
        Bytes B;
        for (float v : data[i]) B.f32(v);
        ok = fseeko(e->f, (off_t)vars[i].begin, SEEK_SET) == 0 && fwrite(B.b.data(), 1, B.b.size(), e->f) == B.b.size();
    }
    if (ok) ok = fflush(e->f) == 0;
    if (!ok) {
        free_exporter(e);
        delete e;
        h->err = std::string("cannot write the header of ") + path;
        return WF_ERR_IO;
    }
    bool cu = cudaMalloc((void**)&e->dstage, e->recsize + 16) == cudaSuccess;
    e->slots.assign(ring, nullptr);
    e->ev.assign(ring, nullptr);
    e->busy.assign(ring, 0);
    for (int s = 0; cu && s < ring; ++s)
        cu = cudaMallocHost((void**)&e->slots[s], e->recsize) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->ev[s], cudaEventDisableTiming) == cudaSuccess;
    if (!cu) {
        cudaGetLastError();
        free_exporter(e);
        delete e;
        h->err = "no memory for the export buffers";
        return WF_ERR_OOM;
    }
    e->writer = std::thread(writer_loop, e);
    *out = e;
    return WF_OK;
}

int wf_export_frame(wf_exporter* e, float phys_time) {
    if (!e) return WF_ERR_INVALID_ARG;
    wf_solver* h = e->h;
    if (cudaSetDevice(h->device) != cudaSuccess) return WF_ERR_CUDA;
    int s = -1;
    {
        std::unique_lock<std::mutex> lk(e->m);
        if (e->failed) return WF_ERR_IO;
        e->cv.wait(lk, [&] {
            for (int i = 0; i < (int)e->busy.size(); ++i)
                if (!e->busy[i]) return true;
            return e->failed;
        });
        if (e->failed) return WF_ERR_IO;
        for (int i = 0; i < (int)e->busy.size(); ++i)
            if (!e->busy[i]) {
                s = i;
                break;
            }
        e->busy[s] = 1;
    }
    // time value (big-endian) at the start of the record
    uint32_t tv;
    std::memcpy(&tv, &phys_time, 4);
    const uint32_t tbe = ((tv >> 24) & 0xFF) | ((tv >> 8) & 0xFF00) | ((tv << 8) & 0xFF0000) | (tv << 24);
    std::memcpy(e->slots[s], &tbe, 4);
    const long long n = (long long)e->N;
    // record = [time][velField][presField]: the time value (offset 0) is
    // written by the host; velField starts at offset 4, which sits at
    // dstage + 16 (16-byte aligned for the kernel's 128-bit stores)
    unsigned char* rec = e->dstage + 12;
    unsigned* velrec = e->vel ? reinterpret_cast<unsigned*>(rec + e->vel_off) : nullptr;
    unsigned* presrec = e->pres ? reinterpret_cast<unsigned*>(rec + e->pres_off) : nullptr;
    WF_COUNT_LAUNCH();
    wf::k_pack_record<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>(n, h->vb[h->iT], h->pr, velrec, presrec);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(e->slots[s] + 4, rec + 4, e->recsize - 4, cudaMemcpyDeviceToHost, h->st);
    if (err == cudaSuccess) err = cudaEventRecord(e->ev[s], h->st);
    {
        std::lock_guard<std::mutex> lk(e->m);
        if (err != cudaSuccess) {
            e->busy[s] = 0;
            h->err = std::string("export frame: ") + cudaGetErrorString(err);
            return WF_ERR_CUDA;
        }
        e->queue.emplace_back(s, e->next_record++);
    }
    e->cv.notify_all();
    return WF_OK;
}

int wf_export_frames_written(wf_exporter* e, int64_t* n) {
    if (!e || !n) return WF_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(e->m);
    *n = e->written;
    return WF_OK;
}

const char* wf_export_last_error(const wf_exporter* e) { return e ? e->err.c_str() : "null exporter"; }

int wf_export_close(wf_exporter* e) {
    if (!e) return WF_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(e->m);
        e->stop = true;
    }
    e->cv.notify_all();
    if (e->writer.joinable()) e->writer.join();
    int st = e->failed ? WF_ERR_IO : WF_OK;
    // numrecs (bytes 4..7 of the header)
    if (st == WF_OK) {
        const uint32_t nr = (uint32_t)e->written;
        const unsigned char b[4] = {(unsigned char)(nr >> 24), (unsigned char)(nr >> 16), (unsigned char)(nr >> 8),
                                    (unsigned char)nr};
        if (fseeko(e->f, 4, SEEK_SET) != 0 || fwrite(b, 1, 4, e->f) != 4 || fflush(e->f) != 0) st = WF_ERR_IO;
    }
    free_exporter(e);
    delete e;
    return st;
}

}  // extern "C"
