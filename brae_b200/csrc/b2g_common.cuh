// b2g_common.cuh -- shared internals of the B200 GAMG-PCG library: error handling, RAII device
// buffers, launch helpers and the exact-rounding arithmetic the parity kernels use.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/brae_gamg.h"

namespace b2g {

// An error that maps to a b2g_status at the C ABI.
struct Error : std::runtime_error
{
    b2g_status code;
    Error(b2g_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(b2g_status c, const std::string& m) { throw Error(c, m); }

inline void cudaCheck(cudaError_t e, const char* what, const char* file, int line)
{
    if (e != cudaSuccess)
    {
        const b2g_status st = (e == cudaErrorMemoryAllocation) ? B2G_ERR_NO_MEMORY : B2G_ERR_CUDA;
        fail(st, std::string("b2g: CUDA error in ") + what + " (" + file + ":" + std::to_string(line) +
                     "): " + cudaGetErrorString(e));
    }
}
#define B2G_CUDA(x) ::b2g::cudaCheck((x), #x, __FILE__, __LINE__)
#define B2G_LAUNCH_CHECK() ::b2g::cudaCheck(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// The library's own stream-ordered memory pool on the current device. It keeps the memory freed
// into it (release threshold: never), so the work arrays of one solve are reused by the next
// instead of being unmapped at every synchronisation and mapped again; the process's default pool
// is left as it is.
cudaMemPool_t libraryPool();

// A device array. Allocation is stream-ordered (cudaMallocFromPoolAsync from libraryPool()).
template <class T>
struct DBuf
{
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;

    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept
    {
        if (this != &o)
        {
            release();
            p = o.p; n = o.n; s = o.s;
            o.p = nullptr; o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }

    void alloc(size_t count, cudaStream_t stream)
    {
        release();
        s = stream;
        n = count;
        if (count)
        {
            B2G_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), libraryPool(), stream));
        }
    }
    // alloc unless the array already holds exactly `count` elements: a rebuild with new values keeps
    // the address, so launches captured in a CUDA graph stay valid
    void ensure(size_t count, cudaStream_t stream)
    {
        if (p && n == count) return;
        alloc(count, stream);
    }
    void zero(cudaStream_t stream)
    {
        if (n) B2G_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), stream));
    }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    void upload(const T* h, size_t count, cudaStream_t stream)
    {
        alloc(count, stream);
        if (count) B2G_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, stream));
    }
    std::vector<T> download(cudaStream_t stream) const
    {
        std::vector<T> h(n);
        if (n) B2G_CUDA(cudaMemcpyAsync(h.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, stream));
        B2G_CUDA(cudaStreamSynchronize(stream));
        return h;
    }
    T* get() const { return p; }
    size_t bytes() const { return n * sizeof(T); }
};

inline int ceilDiv(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

// Device properties of the current device, cached.
struct DeviceInfo
{
    int device = 0;
    int numSMs = 148;
    int maxSmemPerBlockOptin = 227 * 1024;
    static const DeviceInfo& get();
};

// Exact-rounding FP64 helpers: every parity kernel composes these so no multiply-add is ever
// contracted into an FMA (the reference's host path rounds the product and the sum separately).
__device__ __forceinline__ double mulRn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double addRn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double subRn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double divRn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float mulRn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float addRn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float subRn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float divRn(float a, float b) { return __fdiv_rn(a, b); }

// L2-coherent loads for data other CTAs may have written during the same kernel.
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ float ldcg(const float* p) { return __ldcg(p); }

// Release/acquire on a 32-bit progress word at GPU scope.
__device__ __forceinline__ unsigned ldAcquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ldRelaxedGpu(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fenceAcqRelGpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void stRelease(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Profiling switch (b2g_set_profiling) and the last-error slot.
extern bool g_profiling;

}  // namespace b2g
