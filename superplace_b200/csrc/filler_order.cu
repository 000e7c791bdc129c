// Spatial order of the fillers in the optimisation set.
//
// Fillers are most of the opt set (908k of 1.12M nodes at 211k cells) and start scattered
// uniformly at random (scatterFillers, src/gp/filler.cpp:33-45), so consecutive fillers land
// in unrelated bins: every charge the loop's step kernel adds is a separate 64-bit global
// atomic, and the assembly's field gathers of neighbouring threads touch unrelated lines.
// Fillers settle within the first few iterations (their median move is ~23 bins in the first
// 10 iterations of the 211k-cell mGP and ~26 bins over all 143), so the stage loop pauses once,
// at iteration 8 by default, and reorders the filler segment [filler_k0, n_opt) of the opt set by
// 4x4-bin tile in Z order of the tiles (fillers of one tile by their previous index). Then the
// fillers of one warp sit in a few neighbouring bins, and the assembly's field gathers
// (gather_at in optimizer.cu) hit the same cache lines. (Staging a block's fixed-point charge in
// shared memory on top of this order was slower than the direct atomics: the step kernel's
// atomics are fire-and-forget reductions, and the staging's block barriers cost more than the
// L2 atomic traffic they saved.)
//
// The reorder is a permutation of the filler segment of every optimizer vector the loop still
// reads (its live roles and the snapshots, x and y halves), of the fillers' node ids (opt_idx),
// and of the filler id table
// that maps the permuted slots back to the fillers. It changes no value, only the order of the
// FP64 sums over the opt set, and it is deterministic: tile counts are order-free, and each
// tile's fillers are ranked by their previous index.
//
// Kernels (one pass each over the fillers, on the context's stream):
//   key    tile key of each filler at its current u, and the tile counts
//   scan   exclusive scan of the counts (one block); a tile above kSegCap fillers marks the
//          reorder as skipped (the order then stays as it is)
//   place  each filler into its tile's segment (any order within the segment)
//   rank   each segment sorted by previous index (one warp per tile, rank by comparison)
//   apply  gather those vectors' filler segments into a scratch copy; commit copies them
//          back and rewrites opt_idx
#include <algorithm>

#include "engine.h"

namespace spg {

namespace {

constexpr int kTileBins = 4;
constexpr int kSegCap = 1024;  // fillers one tile's segment sort holds
constexpr int kScanThreads = 1024;

__device__ __forceinline__ uint32_t spread8(uint32_t v) {
    v &= 0xFFu;
    v = (v | (v << 4)) & 0x0F0Fu;
    v = (v | (v << 2)) & 0x3333u;
    v = (v | (v << 1)) & 0x5555u;
    return v;
}

__global__ void fsort_key_kernel(DevPtrs p, int* key_of, int* count) {
    pdl_wait();
    pdl_trigger();
    const float* u = role_ptr(p, R_U);
    const int n = p.n_opt, k0 = p.filler_k0, nf = n - k0;
    const GridGeom& g = p.geom;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nf; j += gridDim.x * blockDim.x) {
        const float x = u[k0 + j], y = u[n + k0 + j];
        const int bx = clampi(static_cast<int>(floorf((x - g.origin_x) / g.step_x)), 0, g.dim - 1);
        const int by = clampi(static_cast<int>(floorf((y - g.origin_y) / g.step_y)), 0, g.dim - 1);
        const int key = static_cast<int>(spread8(static_cast<uint32_t>(bx / kTileBins)) |
                                         (spread8(static_cast<uint32_t>(by / kTileBins)) << 1));
        key_of[j] = key;
        atomicAdd(count + key, 1);
    }
}

// One block: offset = exclusive scan of count, cursor = 0, *skip = (a tile above kSegCap).
__global__ void __launch_bounds__(kScanThreads) fsort_scan_kernel(const int* count, int* offset, int* cursor,
                                                                  int n_keys, int* skip) {
    pdl_wait();
    pdl_trigger();
    __shared__ int warp_sum[kScanThreads / 32];
    __shared__ int any_big;
    if (threadIdx.x == 0) any_big = 0;
    const int per = (n_keys + kScanThreads - 1) / kScanThreads;
    const int a = threadIdx.x * per, b = min(a + per, n_keys);
    int local = 0, big = 0;
    for (int i = a; i < b; ++i) {
        local += count[i];
        big |= count[i] > kSegCap;
    }
    // inclusive scan of the per-thread sums across the block (warp shuffles, then warp totals)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int v = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_sum[wid] = v;
    __syncthreads();
    if (big) atomicOr(&any_big, 1);
    if (wid == 0) {
        int w = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        warp_sum[lane] = w;  // inclusive totals of warps 0..lane
    }
    __syncthreads();
    int run = v - local + (wid > 0 ? warp_sum[wid - 1] : 0);  // exclusive start of this thread
    for (int i = a; i < b; ++i) {
        offset[i] = run;
        cursor[i] = 0;
        run += count[i];
    }
    if (threadIdx.x == 0) *skip = any_big;
}

__global__ void fsort_place_kernel(const int* key_of, const int* offset, int* cursor, int* tmp, int nf) {
    pdl_wait();
    pdl_trigger();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nf; j += gridDim.x * blockDim.x) {
        const int key = key_of[j];
        tmp[offset[key] + atomicAdd(cursor + key, 1)] = j;
    }
}

// One warp per tile: the segment's entries (distinct previous indices) ranked by comparison.
constexpr int kRankWarps = 8;
__global__ void __launch_bounds__(32 * kRankWarps) fsort_rank_kernel(const int* count, const int* offset,
                                                                     const int* tmp, int* perm, int n_keys,
                                                                     const int* skip) {
    pdl_wait();
    pdl_trigger();
    __shared__ int seg[kRankWarps][kSegCap];
    if (*skip) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int key = blockIdx.x * kRankWarps + wid; key < n_keys; key += gridDim.x * kRankWarps) {
        const int c = count[key], o = offset[key];
        for (int i = lane; i < c; i += 32) seg[wid][i] = tmp[o + i];
        __syncwarp();
        for (int i = lane; i < c; i += 32) {
            const int e = seg[wid][i];
            int r = 0;
            for (int t = 0; t < c; ++t) r += seg[wid][t] < e;
            perm[o + r] = e;
        }
        __syncwarp();
    }
}

// The pool vectors whose filler segments the reorder permutes: the six roles the loop reads
// before it writes them (u, v, uPrev, vPrev, g, gPrevTmp) and every snapshot slot. The other
// roles are written whole before they are next read (u', v' by the step kernel, the delivered
// positions by the deliver kernel) or serve only the stage's set-up (probe, gA, gB).
constexpr int kOrderVectors = 6 + SNAP_MAX;

__device__ __forceinline__ int order_slot(const DevPtrs& p, int v) {
    switch (v) {
        case 0: return p.st->role[R_U];
        case 1: return p.st->role[R_V];
        case 2: return p.st->role[R_UPREV];
        case 3: return p.st->role[R_VPREV];
        case 4: return p.st->role[R_G];
        case 5: return p.st->role[R_GPREVTMP];
        default: return NUM_ROLES + (v - 6);
    }
}

// scratch[(v * 2 + h) * nf + j] = pool vector v, half h, filler perm[j]; fid_new[j] = fid[perm[j]]
__global__ void fsort_apply_kernel(DevPtrs p, const int* perm, const int* fid, int* fid_new, float* scratch,
                                   const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (*skip) return;
    const int n = p.n_opt, k0 = p.filler_k0, nf = n - k0;
    const int v = blockIdx.y;
    const float* src = p.pool + static_cast<size_t>(order_slot(p, v)) * p.vec_stride;
    float* dst = scratch + static_cast<size_t>(v) * 2 * nf;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nf; j += gridDim.x * blockDim.x) {
        const int q = perm[j];
        dst[j] = src[k0 + q];
        dst[nf + j] = src[n + k0 + q];
        if (v == 0) fid_new[j] = fid[q];
    }
}

__global__ void fsort_commit_kernel(DevPtrs p, const float* scratch, const int* fid_new, int* fid, int* opt_idx,
                                    const int* skip) {
    pdl_wait();
    pdl_trigger();
    if (*skip) return;
    const int n = p.n_opt, k0 = p.filler_k0, nf = n - k0;
    const int v = blockIdx.y;
    float* dst = p.pool + static_cast<size_t>(order_slot(p, v)) * p.vec_stride;
    const float* src = scratch + static_cast<size_t>(v) * 2 * nf;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nf; j += gridDim.x * blockDim.x) {
        dst[k0 + j] = src[j];
        dst[n + k0 + j] = src[nf + j];
        if (v == 0) {
            const int f = fid_new[j];
            fid[j] = f;
            opt_idx[k0 + j] = p.filler_node0 + k0 + f;  // node num_nodes + f
        }
    }
}

}  // namespace

int filler_order_vectors() { return kOrderVectors; }

int filler_order_keys(int dim) {
    int t = (dim + kTileBins - 1) / kTileBins, side = 1;
    while (side < t) side <<= 1;
    return side * side;
}

void launch_filler_order(const DevPtrs& p, const FillerOrderBufs& b, cudaStream_t s) {
    const int nf = p.n_opt - p.filler_k0;
    if (nf <= 0) return;
    const int n_keys = filler_order_keys(p.geom.dim);
    const int n_vec = kOrderVectors;
    SPG_CUDA(cudaMemsetAsync(b.count, 0, static_cast<size_t>(n_keys) * sizeof(int), s));
    const int blocks = std::min(ceil_div(nf, 256), 148 * 8);
    launch_pdl(fsort_key_kernel, dim3(blocks), dim3(256), 0, s, p, b.key_of, b.count);
    launch_pdl(fsort_scan_kernel, dim3(1), dim3(kScanThreads), 0, s, static_cast<const int*>(b.count), b.offset,
               b.cursor, n_keys, b.skip);
    launch_pdl(fsort_place_kernel, dim3(blocks), dim3(256), 0, s, static_cast<const int*>(b.key_of),
               static_cast<const int*>(b.offset), b.cursor, b.tmp, nf);
    launch_pdl(fsort_rank_kernel, dim3(std::min(ceil_div(n_keys, kRankWarps), 148 * 4)), dim3(32 * kRankWarps), 0, s,
               static_cast<const int*>(b.count), static_cast<const int*>(b.offset), static_cast<const int*>(b.tmp),
               b.perm, n_keys, static_cast<const int*>(b.skip));
    const dim3 g2(std::min(ceil_div(nf, 256), 148 * 2), n_vec);
    launch_pdl(fsort_apply_kernel, g2, dim3(256), 0, s, p, static_cast<const int*>(b.perm),
               static_cast<const int*>(b.fid), b.fid_tmp, b.scratch, static_cast<const int*>(b.skip));
    launch_pdl(fsort_commit_kernel, g2, dim3(256), 0, s, p, static_cast<const float*>(b.scratch),
               static_cast<const int*>(b.fid_tmp), b.fid, b.opt_idx, static_cast<const int*>(b.skip));
}

}  // namespace spg
