// hlsl_shim.h - the small subset of HLSL that the reference's compute
// shaders use on the hot path and in its set-up, as C++ (test infrastructure
// only).
//
// With it, oracle/ref_kernels.py turns the reference's own kernel sources
// into C++ translation units (written to oracle/_ref/), so the CPU oracle can
// be checked against the reference's kernels themselves rather than only
// against a restatement.  Semantics follow D3D11 compute shaders:
//   - float literals are single precision (the generator adds the suffix),
//     arithmetic is FP32 without contraction (built with -ffp-contract=off);
//   - texture reads outside the resource return 0, writes outside are
//     dropped;
//   - pow(x, 2) is evaluated as x * x, the form HLSL compilers emit for a
//     literal exponent of 2;
//   - group-shared memory and barriers exist only so the residual kernels
//     compile; the driver never dispatches those kernels.
#pragma once
#include <cmath>
#include <cstdint>

namespace hlsl {

struct uint3;
struct int2 {
    int x, y;
    constexpr int2(int a = 0, int b = 0) : x(a), y(b) {}
};
struct int3 {
    int x, y, z;
    constexpr int3(int a = 0, int b = 0, int c = 0) : x(a), y(b), z(c) {}
    inline int3(const uint3& u);
};
struct uint3 {
    unsigned x, y, z;
    constexpr uint3(unsigned a = 0, unsigned b = 0, unsigned c = 0) : x(a), y(b), z(c) {}
};
inline int3::int3(const uint3& u) : x((int)u.x), y((int)u.y), z((int)u.z) {}
inline int3 operator+(int3 a, int3 b) { return int3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline int3 operator-(int3 a, int3 b) { return int3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline int3 operator/(int3 a, int b) { return int3(a.x / b, a.y / b, a.z / b); }
inline int3 operator*(int3 a, int b) { return int3(a.x * b, a.y * b, a.z * b); }
struct float3;
inline float3 operator*(int3 a, float s);

struct float3 {
    float x, y, z;
    float3() : x(0), y(0), z(0) {}
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
    float3(float s) : x(s), y(s), z(s) {}  // scalar splat (HLSL converts implicitly)
};
inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float3 b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator*(float s, float3 a) { return float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator*(float3 a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator/(float3 a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator-(float3 a) { return float3(-a.x, -a.y, -a.z); }
inline float3& operator+=(float3& a, float3 b) { return a = a + b; }
inline float3& operator-=(float3& a, float3 b) { return a = a - b; }
// int3 * float is a float3 in HLSL (each component converted first).
inline float3 operator*(int3 a, float s) { return float3((float)a.x * s, (float)a.y * s, (float)a.z * s); }

struct float4 {
    float x, y, z, w;
    float4() : x(0), y(0), z(0), w(0) {}
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float4(float3 v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
    float3 xyz() const { return float3(x, y, z); }
};
inline float4 operator+(float4 a, float4 b) { return float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline float4 operator-(float4 a, float4 b) { return float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline float4 operator*(float s, float4 a) { return float4(s * a.x, s * a.y, s * a.z, s * a.w); }
inline float4 operator*(float4 a, float s) { return float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4& operator+=(float4& a, float4 b) { return a = a + b; }

// The sampler object of Texture3D::SampleLevel; only linear filtering with
// clamped addressing (sampler_linear_clamp) is used by the kernels.
struct SamplerState {};

// Out-of-range access: a per-thread element reset to zero on every use, so a
// read gives 0 and a write lands nowhere that is read back.
template <class T>
inline T& oob() {
    static thread_local T s;
    s = T{};
    return s;
}

// 3D and 2D textures over caller-owned storage (x fastest), read and write
// through operator[]; out-of-range reads give 0, writes are dropped.
template <class T>
struct Tex3 {
    T* p = nullptr;
    int nx = 0, ny = 0, nz = 0;
    void bind(T* ptr, int a, int b, int c) {
        p = ptr;
        nx = a;
        ny = b;
        nz = c;
    }
    T& at(int x, int y, int z) const {
        if (!p || x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return oob<T>();
        return p[((size_t)z * ny + y) * nx + x];
    }
    T& operator[](int3 i) const { return at(i.x, i.y, i.z); }
    T& operator[](uint3 i) const { return at((int)i.x, (int)i.y, (int)i.z); }
    // Trilinear filtering with clamped addressing at normalised coordinates
    // uvw (texel centres at (i + 0.5) / n), with exact FP32 weights.  Texture
    // units weigh with a few fractional bits only, so GPU results differ
    // from this in the last bits.
    T SampleLevel(SamplerState, float3 uvw, int) const;
};
template <class T>
struct Tex2 {
    T* p = nullptr;
    int nx = 0, ny = 0;
    void bind(T* ptr, int a, int b) {
        p = ptr;
        nx = a;
        ny = b;
    }
    T& operator[](int2 i) const {
        if (!p || i.x < 0 || i.y < 0 || i.x >= nx || i.y >= ny) return oob<T>();
        return p[(size_t)i.y * nx + i.x];
    }
};
template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    T& operator[](unsigned i) const { return (!p || i >= n) ? oob<T>() : p[i]; }
};

template <class T>
T Tex3<T>::SampleLevel(SamplerState, float3 uvw, int) const {
    const float tx = uvw.x * (float)nx - 0.5f, ty = uvw.y * (float)ny - 0.5f, tz = uvw.z * (float)nz - 0.5f;
    const float fx = std::floor(tx), fy = std::floor(ty), fz = std::floor(tz);
    const float ax = tx - fx, ay = ty - fy, az = tz - fz;
    auto cl = [](int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); };
    const int x0 = cl((int)fx, nx), x1 = cl((int)fx + 1, nx);
    const int y0 = cl((int)fy, ny), y1 = cl((int)fy + 1, ny);
    const int z0 = cl((int)fz, nz), z1 = cl((int)fz + 1, nz);
    const T c00 = at(x0, y0, z0) * (1.0f - ax) + at(x1, y0, z0) * ax;
    const T c10 = at(x0, y1, z0) * (1.0f - ax) + at(x1, y1, z0) * ax;
    const T c01 = at(x0, y0, z1) * (1.0f - ax) + at(x1, y0, z1) * ax;
    const T c11 = at(x0, y1, z1) * (1.0f - ax) + at(x1, y1, z1) * ax;
    const T c0 = c00 * (1.0f - ay) + c10 * ay;
    const T c1 = c01 * (1.0f - ay) + c11 * ay;
    return c0 * (1.0f - az) + c1 * az;
}

inline void sincos(float a, float& s, float& c) {
    s = std::sin(a);
    c = std::cos(a);
}
inline float pow(float x, float y) { return y == 2.0f ? x * x : std::pow(x, y); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float log(float x) { return std::log(x); }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float max(float a, float b) { return a > b ? a : b; }
inline float min(float a, float b) { return a < b ? a : b; }
inline void GroupMemoryBarrierWithGroupSync() {}

}  // namespace hlsl

// HLSL resource types named as in the shaders.
#define RWTexture3D hlsl::Tex3
#define Texture3D hlsl::Tex3
#define Texture2D hlsl::Tex2
#define RWTexture2D hlsl::Tex2
#define RWStructuredBuffer hlsl::Buf
#define StructuredBuffer hlsl::Buf
#define groupshared static
