// A Poisson solve that allocates nothing, for callers that cannot call cudaMalloc.
//
// Some hosts of this library own all device memory themselves: they reserve it up front
// in their own pool or arena and forbid any later driver allocation (for instance a
// placement service that admits work against a fixed HBM budget, or an embedding program
// that runs this solve from a code path where an allocation would stall or fail). Such a
// caller cannot create a spg_poisson plan, because a plan allocates its basis tables and
// work buffers with cudaMalloc.
//
// spg_poisson_solve_static() is the plain-FP32 cosine-contraction solve of a plan (poisson.cu;
// the same kernels run through the same poisson_solve()), but its bases and work buffers live
// in one file-scope device array, g_static_scratch, whose size is fixed when the library is
// loaded: every GPU that loads the library holds those kStaticScratchFloats floats (11 MB)
// until the process exits. The caller passes the input and output grids. Its basis tables
// are computed on the device (cospi / sinpi in FP64, rounded once to float) where a plan
// computes them on the host, so a table entry may differ from the plan's by one float ulp:
// the results agree with a plan's solve to 1e-5 of max|result|, not bit for bit.
//
// Limits and sharing:
//   * nx, ny in [2, 512]; anything larger is rejected with SPG_E_CAPACITY.
//   * All calls on a device share the one array and it keeps the last call's contents.
//     Each call rewrites every region it reads (the bases are regenerated from nx, ny and
//     the steps on every call, and every work region is fully overwritten), so nothing has
//     to start at zero. Calls whose work overlaps on the GPU (on different streams, or
//     from different host threads) race on the array and corrupt each other's results;
//     serialise them.
//   * Every call made outside a stream capture looks up the array's device address with
//     cudaGetSymbolAddress (so a device reset cannot leave a stale address); a call on a
//     stream being captured reuses the address of the last uncaptured call on its device.
//     Make the first call on a device before any stream capture on that device.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "common.cuh"
#include "poisson.h"

namespace spg {

int record_error(const std::exception& e);  // engine.cu: sets spg_last_error()

namespace {

constexpr int kStaticMaxDim = 512;
constexpr int64_t kRegionAlign = 64;  // floats: 256-byte aligned regions
// bases 3*ny^2 + 3*nx^2 + nx*ny, work 4*nx*ny + 4*max(nx, ny), plus region padding
constexpr int64_t kStaticScratchFloats =
    11LL * kStaticMaxDim * kStaticMaxDim + 4LL * kStaticMaxDim + 9 * kRegionAlign;

__device__ __align__(256) float g_static_scratch[kStaticScratchFloats];

constexpr int kMaxDevices = 64;
float* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Device address of g_static_scratch for the current device. It is looked up again on every
// call made outside a stream capture, so a device reset (which reloads the module and may move
// the array) never leaves a stale address behind; a call made while `s` is being captured
// uses the address of the last uncaptured call on that device, and fails when there was none.
float* scratch_for_current_device(cudaStream_t s) {
    int dev = 0;
    SPG_CUDA(cudaGetDevice(&dev));
    SPG_REQUIRE(dev >= 0 && dev < kMaxDevices, SPG_E_INVALID, "device ordinal out of range");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    SPG_CUDA(cudaStreamIsCapturing(s, &cap));
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess)
            throw Error(SPG_E_CUDA, std::string("cudaGetSymbolAddress(g_static_scratch): ") +
                                        cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<float*>(p);
    }
    SPG_REQUIRE(g_scratch_ptr[dev], SPG_E_STATE,
                "spg_poisson_solve_static: the first call on a device must come before any stream capture");
    return g_scratch_ptr[dev];
}

int64_t round_up(int64_t v) { return (v + kRegionAlign - 1) / kRegionAlign * kRegionAlign; }

// The plan's basis tables (poisson.cu, poisson_plan_create) generated on the device in FP64
// and rounded once to float: Cy, Cx, [Ay; Sy], [Ax; Sx] and the spectral scale.
__global__ void static_bases_kernel(int nx, int ny, double sx, double sy, float* cy, float* cx,
                                    float* bcat, float* acat, float* scale) {
    const int64_t X = nx, Y = ny;
    const int64_t total = Y * Y + X * X + X * Y;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (i < Y * Y) {
            const int64_t k = i / Y, y = i % Y;
            const int64_t r = (k * (2 * y + 1)) % (4 * Y);
            const double t = static_cast<double>(r) / static_cast<double>(2 * Y);
            const double c = cospi(t), s = sinpi(t);
            const double v = M_PI * static_cast<double>(k) / (static_cast<double>(ny) * sy);
            cy[k * Y + y] = static_cast<float>(c);
            bcat[y * Y + k] = static_cast<float>((k == 0 ? 1.0 : 2.0) * c);
            bcat[(Y + y) * Y + k] = static_cast<float>(2.0 * v * s);
        } else if (i < Y * Y + X * X) {
            const int64_t q = i - Y * Y;
            const int64_t j = q / X, x = q % X;
            const int64_t r = (j * (2 * x + 1)) % (4 * X);
            const double t = static_cast<double>(r) / static_cast<double>(2 * X);
            const double c = cospi(t), s = sinpi(t);
            const double u = M_PI * static_cast<double>(j) / (static_cast<double>(nx) * sx);
            cx[j * X + x] = static_cast<float>(c);
            acat[x * X + j] = static_cast<float>((j == 0 ? 1.0 : 2.0) * c);
            acat[(X + x) * X + j] = static_cast<float>(2.0 * u * s);
        } else {
            const int64_t q = i - Y * Y - X * X;
            const int64_t j = q / Y, k = q % Y;
            const double u = M_PI * static_cast<double>(j) / (static_cast<double>(nx) * sx);
            const double v = M_PI * static_cast<double>(k) / (static_cast<double>(ny) * sy);
            const double den = u * u + v * v;
            scale[j * Y + k] = den > 0.0 ? static_cast<float>(1.0 / (static_cast<double>(nx) * ny * den)) : 0.f;
        }
    }
}

}  // namespace

}  // namespace spg

extern "C" int spg_poisson_solve_static(int nx, int ny, float step_x, float step_y,
                                        const float* d_rho, float* d_phi, float* d_field_x,
                                        float* d_field_y, void* stream) {
    try {
        using namespace spg;
        SPG_REQUIRE(nx >= 2 && ny >= 2, SPG_E_INVALID, "Poisson: grid must be at least 2x2");
        SPG_REQUIRE(nx <= kStaticMaxDim && ny <= kStaticMaxDim, SPG_E_CAPACITY,
                    "spg_poisson_solve_static: nx and ny must be at most 512 (the static "
                    "scratch array is sized for 512x512)");
        SPG_REQUIRE(step_x > 0.f && step_y > 0.f, SPG_E_INVALID, "Poisson: bin step must be positive");
        SPG_REQUIRE(d_rho && d_phi && d_field_x && d_field_y, SPG_E_INVALID, "null argument");
        const int64_t X = nx, Y = ny;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        float* base = scratch_for_current_device(s);
        int64_t off = 0;
        auto take = [&](int64_t n) {
            float* p = base + off;
            off += round_up(n);
            return p;
        };
        PoissonPlan pl;
        pl.nx = nx;
        pl.ny = ny;
        pl.step_x = step_x;
        pl.step_y = step_y;
        pl.precision = SPG_POISSON_FP32;
        pl.batch_cap = 1;
        pl.cy = take(Y * Y);
        pl.cx = take(X * X);
        pl.bcat = take(2 * Y * Y);
        pl.acat = take(2 * X * X);
        pl.scale = take(X * Y);
        pl.t0t = take(X * Y);
        pl.p = take(X * Y);
        pl.t12t = take(2 * X * Y);
        pl.dc = take(4 * std::max(X, Y));
        SPG_REQUIRE(off <= kStaticScratchFloats, SPG_E_CAPACITY,
                    "spg_poisson_solve_static: layout exceeds the static scratch array");
        const int64_t work = Y * Y + X * X + X * Y;
        const int blocks = static_cast<int>(std::min<int64_t>((work + 255) / 256, 4096));
        static_bases_kernel<<<blocks, 256, 0, s>>>(nx, ny, step_x, step_y, pl.cy, pl.cx, pl.bcat,
                                                    pl.acat, pl.scale);
        count_launch();
        SPG_CHECK_LAUNCH();
        poisson_solve(pl, 1, d_rho, d_phi, d_field_x, d_field_y, s);
        pl.cy = pl.cx = pl.bcat = pl.acat = pl.scale = pl.t0t = pl.p = pl.t12t = pl.dc = nullptr;
        return SPG_OK;
    } catch (const std::exception& e) {
        return spg::record_error(e);
    }
}
