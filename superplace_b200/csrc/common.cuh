// Shared helpers of the sm_100a GP engine: error handling, launch accounting, and the
// bit-exact float footprint arithmetic of the density operators.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>

#include "spgpu.h"

namespace spg {

// A CUDA failure or a bad argument inside the library; converted to an SPG_E_* status at
// the C ABI boundary.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Diagnostics: with SPG_SLOW_CALLS=<ms> set, every checked CUDA call that takes longer than
// that on the host is reported on stderr (time, source line, start time in microseconds,
// thread, expression), so calls that stall behind other threads can be told apart.
inline double slow_call_ms() {
    static const double ms = [] {
        const char* e = std::getenv("SPG_SLOW_CALLS");
        return e ? std::atof(e) : 0.0;
    }();
    return ms;
}
struct CallClock {
    const char* what;
    int line;
    std::chrono::steady_clock::time_point t0;
    CallClock(const char* w, int l) : what(w), line(l) {
        if (slow_call_ms() > 0.0) t0 = std::chrono::steady_clock::now();
    }
    ~CallClock() {
        const double lim = slow_call_ms();
        if (lim <= 0.0) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > lim)
            std::fprintf(stderr, "[spg slow call] %.2f ms line %d t0 %lld tid %zu: %s\n", ms, line,
                         static_cast<long long>(std::chrono::duration_cast<std::chrono::microseconds>(
                                                    t0.time_since_epoch()).count()),
                         std::hash<std::thread::id>{}(std::this_thread::get_id()) % 100000, what);
    }
};

#define SPG_CUDA(call)                                                                   \
    do {                                                                                 \
        const ::spg::CallClock clk_(#call, __LINE__);                                    \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            throw ::spg::Error(SPG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define SPG_CHECK_LAUNCH() SPG_CUDA(cudaGetLastError())

#define SPG_REQUIRE(cond, code, msg)                  \
    do {                                              \
        if (!(cond)) throw ::spg::Error((code), (msg)); \
    } while (0)

// Count of kernels this library launched (process-wide), reported by the benchmark.
extern std::atomic<int64_t> g_launches;
inline void count_launch(int n = 1) { g_launches += n; }

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

// ---------------------------------------------------------------------------------------
// Device memory. Buffers come from a library-owned stream-ordered pool per device: they are
// allocated on the stream of the context (or Poisson plan) being set up and freed in order on
// that same stream, so creating or destroying one context never waits for the work of
// another (a plain cudaFree would synchronize the device). Entry points that (re)allocate
// open an AllocScope with their stream; outside any scope the calls fall back to
// cudaMalloc / cudaFree.
extern thread_local cudaStream_t t_alloc_stream;
struct AllocScope {
    cudaStream_t prev;
    explicit AllocScope(cudaStream_t s) : prev(t_alloc_stream) { t_alloc_stream = s; }
    ~AllocScope() { t_alloc_stream = prev; }
    AllocScope(const AllocScope&) = delete;
    AllocScope& operator=(const AllocScope&) = delete;
};
// `bytes` of device memory, usable on every stream when this returns; *owner receives the
// stream its free must be ordered on (nullptr: plain cudaMalloc).
void* dev_alloc(size_t bytes, cudaStream_t* owner);
void dev_free(void* p, cudaStream_t owner);
// Host -> device copy queued on `s` (through the current context's pinned staging memory
// when `s` is its stream); the source may be reused on return.
void upload_bytes(void* dst, const void* src, size_t bytes, cudaStream_t s);
// Device -> host copy, complete on return.
void download_bytes(void* dst, const void* src, size_t bytes, cudaStream_t s);
// Two device -> host copies of `bytes` each, complete on return, with one wait.
void download_pair(void* dst0, const void* src0, void* dst1, const void* src1, size_t bytes, cudaStream_t s);
// Host wait for the work queued on `s`, sleeping rather than spinning.
cudaError_t host_wait(cudaStream_t s);

// ---------------------------------------------------------------------------------------
// Programmatic dependent launch. A kernel launched by launch_pdl may begin while the kernel
// before it on the stream is still finishing: its blocks get scheduled (and may run a
// prologue that touches no global data) as soon as every block of the earlier kernel has
// called pdl_trigger() or exited. pdl_wait() then blocks until the earlier kernel has
// completed and its memory is visible, so every kernel calls it before its first global
// access. In a kernel launched without the attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// False when SPG_PDL=0 (every launch then waits for the previous kernel as usual).
bool pdl_enabled();

// Scheduling priority of a launch (a kernel-node attribute, kept by graph capture): the
// latency-bound chain of an iteration runs at the device's greatest priority, the WA pass
// beside it at the least, so blocks of the chain get SMs first as blocks retire.
int launch_priority(bool high);

template <typename... KArgs, typename... Args>
inline void launch_prio(bool high, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                        Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    attr[1].id = cudaLaunchAttributePriority;
    attr[1].val.priority = launch_priority(high);
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    SPG_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
    count_launch();
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
    launch_prio(true, kernel, grid, block, smem, s, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------------------------------
// Float arithmetic with explicit round-to-nearest intrinsics: no FMA contraction, so every
// value equals the reference's un-contracted float expression (src/gp/bin_grid.cpp:22-54,
// src/db/geometry.h:35-39).

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// std::min / std::max on non-NaN floats
__device__ __forceinline__ float fmin_(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmax_(float a, float b) { return (a < b) ? b : a; }

// Geometry of the bin grid, passed by value to every density kernel.
struct GridGeom {
    int dim;
    float step_x, step_y, origin_x, origin_y;
    float target_density;
    int shift;            // fixed-point scale 2^shift
    double scale;         // 2^shift
    double inv_scale;     // 2^-shift
    double inv_step_x;    // 1 / step_x and 1 / step_y, rounded to double (bin_index)
    double inv_step_y;
    float scale_f;        // 2^shift as a float when shift >= 0, else 0 (to_fixed)
};

// Per density node data fixed for a stage: half extents after local smoothing and the
// charge weight (footprintOf + chargeWeight, bin_grid.cpp:22-62).
struct Footprint {
    int bx0, bx1, by0, by1;
    float lx, ly, hx, hy;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// The bin index int(a / step) of bin_grid.cpp:49-52, with a / step the float quotient,
// formed as the double product a * (1/step) rounded once to float. This is the float quotient
// bit for bit: the double product is within 2^-52 (relative) of the exact quotient a/step,
// and the exact quotient of two floats with 24-bit significands is either a float or at least
// 2^-49 (relative) away from every midpoint between consecutive floats (a = mid * step would
// need an odd 25-bit significand times a 24-bit one to fit in 24 bits), so both round to the
// same float; the truncation to int follows as before. Checked against the float division
// over bin-boundary neighbourhoods and random operands (tests/test_gpu_parity.py).
__device__ __forceinline__ int bin_index(float a, double inv_step) {
    return static_cast<int>(__double2float_rn(__dmul_rn(static_cast<double>(a), inv_step)));
}

// Bin range and smoothed rectangle of a node at centre (x, y). hw/hh are the half extents
// 0.5f*max(w, step) exactly as footprintOf forms lx = x - 0.5f*W.
__device__ __forceinline__ Footprint footprint(const GridGeom& g, float x, float y, float hw,
                                               float hh) {
    Footprint f;
    f.lx = fsub(x, hw);
    f.hx = fadd(x, hw);
    f.ly = fsub(y, hh);
    f.hy = fadd(y, hh);
    const int d = g.dim - 1;
    f.bx0 = clampi(bin_index(fsub(f.lx, g.origin_x), g.inv_step_x), 0, d);
    f.bx1 = clampi(bin_index(fsub(f.hx, g.origin_x), g.inv_step_x), 0, d);
    f.by0 = clampi(bin_index(fsub(f.ly, g.origin_y), g.inv_step_y), 0, d);
    f.by1 = clampi(bin_index(fsub(f.hy, g.origin_y), g.inv_step_y), 0, d);
    return f;
}

// overlapArea(bin(bx,by), rect) * w (bin_grid.cpp:228-233).
__device__ __forceinline__ float bin_contribution(const GridGeom& g, int bx, int by,
                                                  const Footprint& f, float w) {
    const float blx = fadd(g.origin_x, fmul(static_cast<float>(bx), g.step_x));
    const float bly = fadd(g.origin_y, fmul(static_cast<float>(by), g.step_y));
    const float bhx = fadd(blx, g.step_x);
    const float bhy = fadd(bly, g.step_y);
    const float dx = fsub(fmin_(bhx, f.hx), fmax_(blx, f.lx));
    const float dy = fsub(fmin_(bhy, f.hy), fmax_(bly, f.ly));
    const float a = (dx > 0.f && dy > 0.f) ? fmul(dx, dy) : 0.f;
    return fmul(a, w);
}

// Fixed-point image of one contribution: round-to-nearest-even of c * 2^shift. The product
// is exact in double, and in float too when shift >= 0 (a power-of-two scale of a float that
// stays below the float range), so the float form is the same single rounding.
__device__ __forceinline__ unsigned long long to_fixed(float c, const GridGeom& g) {
    if (g.scale_f > 0.f) return static_cast<unsigned long long>(__float2ll_rn(fmul(c, g.scale_f)));
    return static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(c) * g.scale));
}

}  // namespace spg
