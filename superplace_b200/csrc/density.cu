// Density operators of the GP iteration on sm_100a:
//   * fixed-point charge scatter   (BinGrid::accumulate, src/gp/bin_grid.cpp:191-251)
//   * rho assembly + overflow tau  (BinGrid::solveField/overflow, bin_grid.cpp:253-285)
//   * field gather q*xi            (BinGrid::gatherForce, bin_grid.cpp:287-318)
//
// Scatter: every contribution overlap(bin, rect) * w is formed with the reference's float
// operations (no contraction), rounded once to a 64-bit fixed-point integer and added with
// an integer atomic. Integer addition is associative, so the maps are bit-identical run to
// run and independent of launch shape; the reference gets the same property from fixed
// 8-chunk local grids (bin_grid.cpp:196-251). The maps (16 B per bin for node + filler)
// stay in L2 for every grid size the engine accepts (1024^2 -> 16 MB of the 126 MB L2).
//
// Roofline: these kernels are HBM/L2 bound. Algorithmic bytes per evaluation:
//   scatter 17 B/node + 16 B/bin, rho+tau 28 B/bin, gather 25 B/node.
#include <cuda_bf16.h>

#include "engine.h"

namespace spg {

namespace {

constexpr int kThreads = 256;

// The small density nodes of `list` (count entries), or, with no list, every node i < count
// whose kind marks it a small density node. The fixed-point sums do not depend on the order.
__global__ void __launch_bounds__(kThreads) acc_small_kernel(DevPtrs p, const int* list, int count) {
    pdl_wait();
    pdl_trigger();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int i = list ? list[t] : t;
    const uint8_t k = p.kind[i];
    if (!list && (k & (K_DENSITY | K_LARGE)) != K_DENSITY) return;
    rasterize(p, p.x[i], p.y[i], p.hw[i], p.hh[i], p.wgt[i], (k & K_FILLER) != 0);
}

// One block per large node (macros): the block's threads split its footprint's bins.
__global__ void __launch_bounds__(kThreads) acc_large_kernel(DevPtrs p, const int* list) {
    pdl_wait();
    pdl_trigger();
    const int i = list[blockIdx.x];
    const GridGeom& g = p.geom;
    const Footprint f = footprint(g, p.x[i], p.y[i], p.hw[i], p.hh[i]);
    const float w = p.wgt[i];
    unsigned long long* map = (p.kind[i] & K_FILLER) ? p.filler_fix : p.node_fix;
    const int ny = f.by1 - f.by0 + 1;
    const int nb = (f.bx1 - f.bx0 + 1) * ny;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const int bx = f.bx0 + j / ny, by = f.by0 + j % ny;
        const float c = bin_contribution(g, bx, by, f, w);
        if (c <= 0.f) continue;
        atomicAdd(map + static_cast<size_t>(bx) * g.dim + by, to_fixed(c, g));
    }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-order block sum (warp trees, then warp 0 over the warp sums); result in thread 0.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    double r = 0.0;
    if (wid == 0) {
        r = lane < nw ? ws[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// rho = (node + filler + terminal + base) * (1/binArea) as float (bin_grid.cpp:253-259) and
// the tau partial sums sum max(rho' - target, 0) * binArea over rho' without fillers
// (bin_grid.cpp:265-285). Reads the fixed-point maps and clears them for the next
// evaluation when `zero` is set.
__global__ void __launch_bounds__(RED_THREADS) rho_overflow_kernel(DevPtrs p, int write_maps,
                                                                   int zero) {
    pdl_wait();
    pdl_trigger();
    const GridGeom& g = p.geom;
    const size_t n = static_cast<size_t>(g.dim) * g.dim;
    const float bin_area_f = fmul(g.step_x, g.step_y);
    const float inv_area = fdiv(1.0f, bin_area_f);
    const double area = static_cast<double>(bin_area_f);
    const double target = static_cast<double>(g.target_density);
    double over = 0.0;
    for (size_t b = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; b < n;
         b += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const long long nfix = static_cast<long long>(p.node_fix[b]);
        const long long ffix = static_cast<long long>(p.filler_fix[b]);
        const float nd = static_cast<float>(static_cast<double>(nfix) * g.inv_scale);
        const float fd = static_cast<float>(static_cast<double>(ffix) * g.inv_scale);
        const float t = p.terminal[b], bs = p.base[b];
        p.rho[b] = fmul(fadd(fadd(fadd(nd, fd), t), bs), inv_area);
        const double r = __dadd_rn(__dadd_rn(static_cast<double>(nd), static_cast<double>(t)),
                                   static_cast<double>(bs)) / area;
        const double d = r - target;
        over += d > 0.0 ? __dmul_rn(d, area) : 0.0;
        if (write_maps) {
            p.node_map[b] = nd;
            p.filler_map[b] = fd;
        }
        if (zero) {
            p.node_fix[b] = 0ull;
            p.filler_fix[b] = 0ull;
        }
    }
    over = block_sum(over);
    put_partial(p, SLOT_OVERFLOW, over);
}

// hi/lo BF16 split of v (v = hi + lo to about 16 bits), as the tensor-core solve splits its
// operands
__device__ __forceinline__ void split_bf16_pair(float v, uint16_t& hi, uint16_t& lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

// rho and the tau partials (as rho_overflow_kernel, clearing the fixed maps) fused with the
// first operand split of a one-grid tensor-core Poisson solve (prep_split_kernel with
// centring): one block per bin row bx. Each thread keeps its bins' rho in registers; the
// row's FP64 sum is the split kernel's fixed-order block reduction (thread partials in bin
// order, warp trees, then the warp sums in order), so the mean, the split planes of
// rho - mean and the exact row sum equal the solve's own split bit for bit.
constexpr int kRhoPrepThreads = 256;
constexpr int kRhoPrepPer = 4;  // bins per thread: rows up to 1024 bins
__global__ void __launch_bounds__(kRhoPrepThreads) rho_prep_kernel(DevPtrs p, uint16_t* planes,
                                                                   int64_t plane_stride, int64_t ld,
                                                                   float* sums) {
    pdl_wait();
    pdl_trigger();
    __shared__ double wsum[kRhoPrepThreads / 32];
    __shared__ double row_total;
    const GridGeom& g = p.geom;
    const int dim = g.dim;
    const int row = blockIdx.x, tid = threadIdx.x;
    const float bin_area_f = fmul(g.step_x, g.step_y);
    const float inv_area = fdiv(1.0f, bin_area_f);
    const double area = static_cast<double>(bin_area_f);
    const double target = static_cast<double>(g.target_density);
    const size_t base = static_cast<size_t>(row) * dim;
    double over = 0.0, v = 0.0;
    float rho[kRhoPrepPer];
#pragma unroll
    for (int j = 0; j < kRhoPrepPer; ++j) {
        const int i = tid + j * kRhoPrepThreads;
        rho[j] = 0.f;
        if (i >= dim) continue;
        const size_t b = base + i;
        const long long nfix = static_cast<long long>(p.node_fix[b]);
        const long long ffix = static_cast<long long>(p.filler_fix[b]);
        const float nd = static_cast<float>(static_cast<double>(nfix) * g.inv_scale);
        const float fd = static_cast<float>(static_cast<double>(ffix) * g.inv_scale);
        const float t = p.terminal[b], bs = p.base[b];
        rho[j] = fmul(fadd(fadd(fadd(nd, fd), t), bs), inv_area);
        p.rho[b] = rho[j];
        const double r = __dadd_rn(__dadd_rn(static_cast<double>(nd), static_cast<double>(t)),
                                   static_cast<double>(bs)) / area;
        const double d = r - target;
        over += d > 0.0 ? __dmul_rn(d, area) : 0.0;
        p.node_fix[b] = 0ull;
        p.filler_fix[b] = 0ull;
        v += static_cast<double>(rho[j]);
    }
    // the row sum: warp trees, then the warp sums in warp order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) wsum[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < kRhoPrepThreads / 32; ++w) s += wsum[w];
        row_total = s;
        sums[row] = static_cast<float>(s);
    }
    __syncthreads();
    const float mean = static_cast<float>(row_total / dim);
    uint16_t* hi = planes + row * ld;
    uint16_t* lo = hi + plane_stride;
#pragma unroll
    for (int j = 0; j < kRhoPrepPer; ++j) {
        const int i = tid + j * kRhoPrepThreads;
        if (i >= dim) continue;
        uint16_t h, l;
        split_bf16_pair(rho[j] - mean, h, l);
        hi[i] = h;
        lo[i] = l;
    }
    over = block_sum(over);
    put_partial(p, SLOT_OVERFLOW, over);
}

// force = sum over the footprint of q * xi, bx outer, by inner, as gatherForce sums it.
__device__ __forceinline__ void gather_node(const DevPtrs& p, int i, float& fx, float& fy) {
    const GridGeom& g = p.geom;
    const Footprint f = footprint(g, p.x[i], p.y[i], p.hw[i], p.hh[i]);
    const float w = p.wgt[i];
    fx = 0.f;
    fy = 0.f;
    for (int bx = f.bx0; bx <= f.bx1; ++bx) {
        const size_t row = static_cast<size_t>(bx) * g.dim;
        for (int by = f.by0; by <= f.by1; ++by) {
            const float q = bin_contribution(g, bx, by, f, w);
            if (q <= 0.f) continue;
            fx = fadd(fx, fmul(q, __ldg(p.ex + row + by)));
            fy = fadd(fy, fmul(q, __ldg(p.ey + row + by)));
        }
    }
}

// Large nodes: the block splits the footprint; per-thread partial sums are combined in a
// fixed tree (deterministic, but not the reference's sequential order).
__device__ __forceinline__ void gather_large(const DevPtrs& p, int i, float& fx, float& fy) {
    const GridGeom& g = p.geom;
    const Footprint f = footprint(g, p.x[i], p.y[i], p.hw[i], p.hh[i]);
    const float w = p.wgt[i];
    const int ny = f.by1 - f.by0 + 1;
    const int nb = (f.bx1 - f.bx0 + 1) * ny;
    float ax = 0.f, ay = 0.f;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const int bx = f.bx0 + j / ny, by = f.by0 + j % ny;
        const float q = bin_contribution(g, bx, by, f, w);
        if (q <= 0.f) continue;
        const size_t idx = static_cast<size_t>(bx) * g.dim + by;
        ax = fadd(ax, fmul(q, p.ex[idx]));
        ay = fadd(ay, fmul(q, p.ey[idx]));
    }
    __shared__ float sx[32], sy[32];
    ax = warp_sum(ax);
    ay = warp_sum(ay);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sx[wid] = ax;
        sy[wid] = ay;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        ax = lane < nw ? sx[lane] : 0.f;
        ay = lane < nw ? sy[lane] : 0.f;
        ax = warp_sum(ax);
        ay = warp_sum(ay);
    }
    fx = ax;
    fy = ay;
}

__global__ void __launch_bounds__(kThreads) gather_opt_large_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const int k = p.opt_large[blockIdx.x];
    float fx, fy;
    gather_large(p, p.opt_idx[k], fx, fy);
    if (threadIdx.x == 0) {
        p.force[k] = fx;
        p.force[p.n_opt + k] = fy;
    }
}

__global__ void __launch_bounds__(kThreads) gather_all_small_kernel(DevPtrs p, float* out) {
    pdl_wait();
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.total || (p.kind[i] & (K_DENSITY | K_LARGE)) != K_DENSITY) return;  // small density nodes
    float fx, fy;
    gather_node(p, i, fx, fy);
    out[i] = fx;
    out[p.total + i] = fy;
}

__global__ void __launch_bounds__(kThreads) gather_all_large_kernel(DevPtrs p, float* out) {
    pdl_wait();
    pdl_trigger();
    const int i = p.dens_large[blockIdx.x];
    float fx, fy;
    gather_large(p, i, fx, fy);
    if (threadIdx.x == 0) {
        out[i] = fx;
        out[p.total + i] = fy;
    }
}

}  // namespace

void launch_density_accumulate(const DevPtrs& p, cudaStream_t s) {
    if (p.n_dens_small > 0) {
        launch_pdl(acc_small_kernel, dim3(ceil_div(p.total, kThreads)), dim3(kThreads), 0, s, p,
                   static_cast<const int*>(nullptr), p.total);
    }
    if (p.n_dens_large > 0) {
        launch_pdl(acc_large_kernel, dim3(p.n_dens_large), dim3(kThreads), 0, s, p, p.dens_large);
    }
}

void launch_density_rest(const DevPtrs& p, cudaStream_t s) {
    if (p.n_rest_small > 0) {
        launch_pdl(acc_small_kernel, dim3(ceil_div(p.n_rest_small, kThreads)), dim3(kThreads), 0, s, p,
                   p.rest_small, p.n_rest_small);
    }
    if (p.n_rest_large > 0) {
        launch_pdl(acc_large_kernel, dim3(p.n_rest_large), dim3(kThreads), 0, s, p, p.rest_large);
    }
}

void launch_rho_overflow(const DevPtrs& p, int write_maps, int zero, cudaStream_t s) {
    const int grid = work_grid(reinterpret_cast<const void*>(rho_overflow_kernel),
                               static_cast<int64_t>(p.geom.dim) * p.geom.dim, RED_THREADS);
    launch_pdl(rho_overflow_kernel, dim3(grid), dim3(RED_THREADS), 0, s, p, write_maps, zero);
}

void launch_rho_prep(const DevPtrs& p, uint16_t* planes, int64_t plane_stride, int64_t ld, float* sums,
                     cudaStream_t s) {
    SPG_REQUIRE(p.geom.dim <= kRhoPrepThreads * kRhoPrepPer && p.geom.dim <= RED_CAP, SPG_E_INVALID,
                "rho_prep: grid too large");
    launch_pdl(rho_prep_kernel, dim3(p.geom.dim), dim3(kRhoPrepThreads), 0, s, p, planes, plane_stride, ld, sums);
}

void launch_gather_opt_large(const DevPtrs& p, cudaStream_t s) {
    if (p.n_opt_large > 0) {
        launch_pdl(gather_opt_large_kernel, dim3(p.n_opt_large), dim3(kThreads), 0, s, p);
    }
}

// Self-check of bin_index: the truncated float quotient a / step and bin_index's product form.
__global__ void bin_index_check_kernel(const float* a, int n, float step, double inv, int* q_div, int* q_mul) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    q_div[i] = static_cast<int>(fdiv(a[i], step));
    q_mul[i] = bin_index(a[i], inv);
}

void launch_bin_index_check(const float* a, int n, float step, double inv, int* q_div, int* q_mul, cudaStream_t s) {
    if (n > 0)
        bin_index_check_kernel<<<ceil_div(n, kThreads), kThreads, 0, s>>>(a, n, step, inv, q_div, q_mul);
}

void launch_gather_all(const DevPtrs& p, float* out, cudaStream_t s) {
    if (p.n_dens_small > 0) {
        launch_pdl(gather_all_small_kernel, dim3(ceil_div(p.total, kThreads)), dim3(kThreads), 0, s, p, out);
    }
    if (p.n_dens_large > 0) {
        launch_pdl(gather_all_large_kernel, dim3(p.n_dens_large), dim3(kThreads), 0, s, p, out);
    }
}

}  // namespace spg
