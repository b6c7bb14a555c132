// Shared definitions of libbaemm_cuda.so: error handling, device buffers,
// complex helpers and the per-context operator parameters.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/baemm.h"

namespace baemm
{

struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define BAEMM_CUDA(call)                                                                    \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            throw ::baemm::Error(BAEMM_ERR_CUDA, std::string(#call) + " failed: " +         \
                                                     cudaGetErrorString(e_));               \
    } while (0)

// Process-wide count of kernel launches (reported by baemm_kernel_launch_count).
extern std::atomic<long long> g_kernel_launches;
// Bumped by every device-buffer (re)allocation of the library: a captured CUDA
// graph holds raw pointers and is valid only while this stays unchanged.
extern std::atomic<long long> g_devbuf_epoch;
#define BAEMM_LAUNCH_CHECK()                                                                \
    do {                                                                                    \
        BAEMM_CUDA(cudaGetLastError());                                                     \
        ::baemm::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                 \
    } while (0)

#define BAEMM_REQUIRE(cond, code, msg)                                                      \
    do {                                                                                    \
        if (!(cond)) throw ::baemm::Error((code), (msg));                                   \
    } while (0)

// Largest mesh (triangles, vertices) a context takes.  The host topology and
// the device sparse operators index with int32: AvOp^T holds 3 nt entries and
// the mass matrix at most nv + 6 nt, both below 2^31 at this size.
constexpr int64_t kMaxMeshSize = (int64_t)1 << 28;

// Makes a device current for one entry-point call and restores the caller's
// device afterwards, so contexts on different GPUs can be driven from one
// thread (allocations, streams and launches all belong to the context's
// device) and a host framework's device selection is left as it was.
struct DeviceScope
{
    int prev = -1;
    explicit DeviceScope(int dev)   // dev < 0: only restore the caller's device at the end
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
        {
            (void)cudaGetLastError();
            prev = -1;
        }
        if (dev >= 0 && prev != dev) BAEMM_CUDA(cudaSetDevice(dev));
    }
    ~DeviceScope()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) (void)cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope &) = delete;
    DeviceScope &operator=(const DeviceScope &) = delete;
};

// Grow-only device buffer.
template <class T>
struct DevBuf
{
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    T *reserve(size_t count)
    {
        if (count > n)
        {
            release();
            if (count)
            {
                cudaError_t e = cudaMalloc(&p, count * sizeof(T));
                if (e != cudaSuccess)
                {
                    p = nullptr;
                    (void)cudaGetLastError();
                    throw Error(BAEMM_ERR_ALLOC, "cudaMalloc of " + std::to_string(count * sizeof(T)) +
                                                     " bytes failed: " + cudaGetErrorString(e));
                }
            }
            n = count;
            g_devbuf_epoch.fetch_add(1, std::memory_order_relaxed);
        }
        return p;
    }
    operator T *() const { return p; }
};

// ---- complex helpers (float2 / double2 as complex) -------------------------
template <class R> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <class R> using cplx = typename cplx_t<R>::type;

template <class R> __host__ __device__ __forceinline__ cplx<R> mk(R x, R y) { cplx<R> c; c.x = x; c.y = y; return c; }
template <class C> __host__ __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <class C> __host__ __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <class C> __host__ __device__ __forceinline__ C cmul(C a, C b)
{
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <class C, class R> __host__ __device__ __forceinline__ C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }
template <class C> __host__ __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// acc += a * b
template <class C> __host__ __device__ __forceinline__ void cfma(C &acc, C a, C b)
{
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
__host__ __device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__host__ __device__ __forceinline__ double2 to_d(double2 a) { return a; }
__host__ __device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
__host__ __device__ __forceinline__ float2 to_f(float2 a) { return a; }
template <class C> __host__ __device__ __forceinline__ C from_d(double2 a);
template <> __host__ __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }
template <> __host__ __device__ __forceinline__ float2 from_d<float2>(double2 a) { return to_f(a); }

// ---- operator parameters -----------------------------------------------------
// One entry per wave chunk: the wavenumber and the four coefficients (mass, SL,
// DL, adjoint DL), c1..c3 scaled by factor/(4 pi) as LoadParameters.hpp:65-79.
constexpr int kMaxWaveCount = 1024;
constexpr int kMaxChunks = 1024;

struct ChunkParamsF { float kappa; float pad; float2 c[4]; };     // 40 bytes
struct ChunkParamsD { double kappa; double pad; double2 c[4]; };  // 80 bytes

struct OpFlags
{
    bool re_mass = false, im_mass = false, re_sl = false, im_sl = false;
    bool re_dl = false, im_dl = false, re_adl = false, im_adl = false;
    bool mass() const { return re_mass || im_mass; }
    bool sl() const { return re_sl || im_sl; }
    bool dl() const { return re_dl || im_dl; }
    bool adl() const { return re_adl || im_adl; }
    bool any_layer() const { return sl() || dl() || adl(); }
};

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

} // namespace baemm
