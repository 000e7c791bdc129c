// Split-BF16 tensor-core Poisson path for sm_100a (tcgen05 + TMA + TMEM).
//
// Every contraction of poisson.h's chain, C[m][n] = sum_k A[m][k] B[n][k], runs as a
// split-BF16 product: each FP32 operand x is stored as two BF16 planes hi = bf16(x),
// lo = bf16(x - hi), and C = A_hi.B_hi + A_hi.B_lo + A_lo.B_hi accumulated in FP32 in
// tensor memory (the lo.lo term, ~2^-16 relative, is dropped). The three products are one
// accumulation: each K slab's four planes arrive in one ring stage and the MMA thread issues
// hi.hi, hi.lo and lo.hi for every 16-wide K step.
//
// Kernel (one 128 x BN output tile per cluster of S split-K CTAs, 128 threads each):
//   warp 0 lane 0   TMA producer: 128x64 A hi/lo and BNx64 B hi/lo bf16 tiles (128-byte
//                   swizzle) into a STAGES-deep shared-memory ring (full/empty mbarriers)
//   warp 1 lane 0   MMA issuer: 12 x tcgen05.mma.kind::f16 (M=128, N=BN, K=16) per slab,
//                   tcgen05.commit frees the slab, a final commit publishes the accumulator
//   warps 0-3       epilogue: tcgen05.ld of the TMEM partial into shared memory, a
//                   cluster-wide reduction of the S partials over DSMEM (rank order), the
//                   optional spectral scale and DC-row override, and either an FP32 store
//                   or a split store of the next contraction's BF16 hi/lo planes
// Every mbarrier wait is bounded (2 s of %globaltimer); on timeout the kernel records
// SPG_E_CUDA in the plan's error word, stops issuing, frees its TMEM and returns.
//
// DC split (poisson.h): the forward contractions subtract each B row's mean before the
// split (prep_split_kernel, one block per row segment; for the engine's one-grid solves the
// density's split comes from its rho kernel, rho_prep_kernel, with the same reduction order)
// and restore the DC row exactly in the epilogue. G4 computes phi, xi_x and xi_y in one launch
// (xi_y as an alternate M region reading its own A and B rows).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "poisson.h"

namespace spg {

namespace {

constexpr int TC_BM = 128;
constexpr int TC_BK = 64;  // bf16 elements per K slab = one 128-byte swizzle row
constexpr int TC_THREADS = 128;
constexpr unsigned long long kWaitNs = 2000000000ull;  // bounded mbarrier waits: 2 s

enum TcMode : int { TC_F32 = 0, TC_SPLIT = 1 };

struct TcArgs {
    int M, N, K;            // tile-multiple problem dims (K per split pass)
    int a_row0, a_lo;       // A: first row, rows between hi and lo planes
    int b_row0, b_lo;       // B: first row, rows between hi and lo planes
    int b_col_z;            // B column offset per blockIdx.z (batched over grids)
    int mode;               // TcMode
    float* out;             // F32: rows < split -> out, else out2 ; SPLIT: hi plane
    float* out2;
    int split;
    int64_t ldc;            // output row pitch (elements)
    int64_t out_z;          // output offset per blockIdx.z (elements)
    uint16_t* planes;       // SPLIT: hi plane base (lo plane at + plane_stride)
    int64_t plane_stride;
    int64_t plane_z;        // SPLIT: offset per blockIdx.z (elements)
    const float* scale;     // optional S[m][n] (ld = N of one grid), multiplies the result
    int64_t lds;
    const float* row0;      // optional: output row 0 := row0[z*row0_z + n] (* scale[n])
    int64_t row0_z;
    int* err;
    // optional alternate region (m_alt > 0): output rows m >= m_alt read A from row
    // a_alt_row0 + (m - m_alt) and B from row b_alt_row0 + n, and go to out3 row m - m_alt
    // (F32 mode), so two products sharing A's layout run as one launch
    int m_alt, a_alt_row0, b_alt_row0;
    float* out3;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete; false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = gtime();
    while (!mbar_try(bar, parity))
        if (gtime() - t0 > kWaitNs) return false;
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr & 0x3FFFFu) >> 4);  // start address
    d |= static_cast<uint64_t>(1) << 16;                  // leading byte offset (unused here)
    d |= static_cast<uint64_t>(1024 >> 4) << 32;          // stride byte offset
    d |= static_cast<uint64_t>(1) << 46;                  // descriptor version (sm_100)
    d |= static_cast<uint64_t>(2) << 61;                  // SWIZZLE_128B
    return d;
}

// Instruction descriptor of tcgen05.mma.kind::f16: BF16 A and B (K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4)                              // D format: F32
           | (1u << 7)                            // A format: BF16
           | (1u << 10)                           // B format: BF16
           | (static_cast<uint32_t>(n >> 3) << 17)  // N / 8
           | (static_cast<uint32_t>(m >> 4) << 24);  // M / 16
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void split_bf16(float v, uint16_t& hi, uint16_t& lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t map_rank(uint32_t local_addr, uint32_t rank) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local_addr), "r"(rank));
    return remote;
}

// 16-byte store into another CTA's shared memory (a shared::cluster address from mapa).
__device__ __forceinline__ void st_dsmem4(uint32_t addr, float a, float b, float c, float d) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.aligned;" ::: "memory"); }

// 16-byte load from another CTA's shared memory (volatile keeps it after the cluster barrier).
__device__ __forceinline__ float4 ld_dsmem4(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr));
    return v;
}

// The epilogue's factors for the outputs at (m, n..n+3) of grid z: the spectral scale, and on
// row 0 with row0 set the exact DC row times it (ones when the CTA does not run).
__device__ __forceinline__ float4 epi_scale(const TcArgs& g, int m, int n, int z, bool run) {
    float4 sc = make_float4(1.f, 1.f, 1.f, 1.f);
    if (run && g.scale) sc = __ldg(reinterpret_cast<const float4*>(g.scale + m * g.lds + n));
    if (run && m == 0 && g.row0) {
        const float4 r0 = __ldg(reinterpret_cast<const float4*>(g.row0 + z * g.row0_z + n));
        sc = make_float4(r0.x * sc.x, r0.y * sc.y, r0.z * sc.z, r0.w * sc.w);
    }
    return sc;
}

// The epilogue of four reduced outputs at (m, n..n+3) of grid z: the spectral scale (sc) or,
// on row 0 with row0 set, the exact DC row held in sc; then an FP32 store or the split store of
// the next contraction's BF16 hi/lo planes.
__device__ __forceinline__ void tile_store(const TcArgs& g, int m, int n, int z, float4 sc, float* v) {
    if (m == 0 && g.row0) {  // the DC row: the exact sums (times the scale), in sc
        v[0] = sc.x;
        v[1] = sc.y;
        v[2] = sc.z;
        v[3] = sc.w;
    } else if (g.scale) {
        v[0] *= sc.x;
        v[1] *= sc.y;
        v[2] *= sc.z;
        v[3] *= sc.w;
    }
    if (g.mode == TC_F32) {
        float* dst = (g.m_alt > 0 && m >= g.m_alt) ? g.out3 + z * g.out_z + (m - g.m_alt) * g.ldc
                     : (m < g.split) ? g.out + z * g.out_z + m * g.ldc
                                     : g.out2 + z * g.out_z + (m - g.split) * g.ldc;
        *reinterpret_cast<float4*>(dst + n) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        uint16_t h[4], l[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) split_bf16(v[i], h[i], l[i]);
        uint16_t* hi = g.planes + z * g.plane_z + m * g.ldc + n;
        *reinterpret_cast<uint2*>(hi) = *reinterpret_cast<const uint2*>(h);
        *reinterpret_cast<uint2*>(hi + g.plane_stride) = *reinterpret_cast<const uint2*>(l);
    }
}

// Per-CTA pipeline state, carried across the tiles one CTA computes: a standalone GEMM launch
// computes one tile per CTA, the fused solve several (tc_fused_kernel).
struct TileState {
    uint8_t* base;             // the 1024-aligned stage ring
    uint32_t full0, empty0, accb;
    uint32_t tmem;
    uint32_t it;               // ring slabs this CTA has streamed so far
    uint32_t acc_n;            // accumulator phases completed
};

template <int BN, int STAGES>
__device__ __forceinline__ void tile_setup(uint8_t* smem_raw, TileState& t) {
    constexpr uint32_t STAGE_BYTES = 2 * TC_BM * TC_BK * 2 + 2 * BN * TC_BK * 2;
    t.base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bars = reinterpret_cast<uint64_t*>(t.base + STAGES * STAGE_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 1);
    t.full0 = smem_u32(bars);
    t.empty0 = smem_u32(bars + STAGES);
    t.accb = smem_u32(bars + 2 * STAGES);
    t.it = 0;
    t.acc_n = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < STAGES; ++i) {
            mbar_init(t.full0 + 8 * i, 1);
            mbar_init(t.empty0 + 8 * i, 1);
        }
        mbar_init(t.accb, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if ((threadIdx.x >> 5) == 0) {  // TMEM accumulator: BN fp32 columns x 128 lanes
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(static_cast<uint32_t>(BN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    t.tmem = *tmem_slot;
}

template <int BN>
__device__ __forceinline__ void tile_teardown(const TileState& t) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(t.tmem), "r"(static_cast<uint32_t>(BN)));
}

// One 128 x BN output tile (rows m0.., columns n0.., grid z) of the contraction g, of which
// this CTA computes K slabs [rank*nk/S, (rank+1)*nk/S): the tile's S CTAs are cluster ranks
// group0 .. group0+S-1. A ring stage holds one K slab of all four operand planes (A hi, A lo,
// B hi, B lo), from which the MMA thread issues the three products, so every plane crosses L2
// once per slab. Each CTA accumulates its slice in TMEM and stages it in shared memory (over
// the ring, which is idle by then); then CTA r reduces rows [r*128/S, (r+1)*128/S) over the S
// partials through distributed shared memory, in rank order (deterministic), with all of its
// remote loads in flight at once, and runs the epilogue for those rows with consecutive
// threads on consecutive columns (coalesced stores). All threads of the CTA call it. With
// active = false (a CTA without a tile in this round) or after an earlier failure (*g.err set)
// the CTA streams and writes nothing but still takes the tile's cluster barriers.
//
// PUSH (a CTA that computes one tile in its launch, S > 1): instead of staging its partial in
// its own ring for the others to pull, each CTA stores the rows that CTA r reduces straight
// into r's receive area (past the ring and its barriers, so a store cannot land on a ring the
// MMAs still read), slot = the sender's rank; one cluster barrier makes them visible and each
// CTA sums its S slots locally in rank order: the same sums as the pull form, with one cluster
// barrier fewer and local instead of remote loads. The caller has arrived on the cluster barrier
// once after tile_setup (cluster_arrive_relaxed), so every CTA of the cluster is running before
// the first remote store.
template <int BN, int STAGES, int S, bool PUSH = false>
__device__ __forceinline__ void gemm_tile(const CUtensorMap& tmA, const CUtensorMap& tmB, const TcArgs& g, int m0,
                                          int n0, int z, int rank, int group0, bool active, TileState& t) {
    constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2;  // one plane
    constexpr uint32_t B_BYTES = BN * TC_BK * 2;
    constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    constexpr int RED_LD = BN + 4;  // staged partial tile row pitch (floats, 16-byte rows)
    constexpr int R = TC_BM / S;    // output rows this CTA reduces
    constexpr int GPT = R * (BN / 4) / TC_THREADS;  // float4 groups per thread
    static_assert(GPT >= 1 && R * (BN / 4) % TC_THREADS == 0, "reduction must split evenly");
    static_assert(TC_BM * RED_LD * 4 <= STAGES * STAGE_BYTES, "partial tile must fit the ring");
    float* red = reinterpret_cast<float*>(t.base);  // reuses the ring after the main loop
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __shared__ int run_s;
    if (threadIdx.x == 0) run_s = active && __ldcg(g.err) == 0;
    __syncthreads();
    const bool run = run_s != 0;

    const int nk = g.K / TC_BK;
    const int s0 = rank * nk / S, s1 = (rank + 1) * nk / S;
    if (run && warp == 0 && lane == 0) {
        // producer: one stage = K slab kk of A hi, A lo, B hi, B lo
        for (int s = s0; s < s1; ++s) {
            const uint32_t i = t.it + static_cast<uint32_t>(s - s0), st = i % STAGES;
            const uint32_t ph = (i / STAGES) & 1;
            if (!mbar_wait(t.empty0 + 8 * st, ph ^ 1)) break;
            const int kk = s * TC_BK;
            const uint32_t sa = smem_u32(t.base + st * STAGE_BYTES);
            const bool alt = g.m_alt > 0 && m0 >= g.m_alt;
            const int arow = alt ? g.a_alt_row0 + (m0 - g.m_alt) : g.a_row0 + m0;
            const int brow = (alt ? g.b_alt_row0 : g.b_row0) + n0, bcol = kk + z * g.b_col_z;
            mbar_expect_tx(t.full0 + 8 * st, STAGE_BYTES);
            tma_load_2d(sa, &tmA, kk, arow, t.full0 + 8 * st);
            tma_load_2d(sa + A_BYTES, &tmA, kk, arow + g.a_lo, t.full0 + 8 * st);
            tma_load_2d(sa + 2 * A_BYTES, &tmB, bcol, brow, t.full0 + 8 * st);
            tma_load_2d(sa + 2 * A_BYTES + B_BYTES, &tmB, bcol, brow + g.b_lo, t.full0 + 8 * st);
        }
    } else if (run && warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(TC_BM, BN);
        bool ok = true;
        for (int s = s0; s < s1; ++s) {
            const uint32_t i = t.it + static_cast<uint32_t>(s - s0), st = i % STAGES;
            const uint32_t ph = (i / STAGES) & 1;
            if (!mbar_wait(t.full0 + 8 * st, ph)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ahi = smem_u32(t.base + st * STAGE_BYTES), alo = ahi + A_BYTES;
            const uint32_t bhi = ahi + 2 * A_BYTES, blo = bhi + B_BYTES;
            const bool first = s == s0;
#pragma unroll
            for (int k = 0; k < TC_BK / 16; ++k) {  // 16 bf16 = 32 bytes per MMA along K
                const uint32_t o = 32 * k;
                umma_bf16(t.tmem, sw128_desc(ahi + o), sw128_desc(bhi + o), idesc, (!first || k > 0) ? 1u : 0u);
                umma_bf16(t.tmem, sw128_desc(ahi + o), sw128_desc(blo + o), idesc, 1u);
                umma_bf16(t.tmem, sw128_desc(alo + o), sw128_desc(bhi + o), idesc, 1u);
            }
            umma_commit(t.empty0 + 8 * st);
        }
        if (ok) umma_commit(t.accb);
    }
    __syncwarp();

    // epilogue inputs that do not depend on the partials, fetched while the MMAs run: this
    // thread's output groups (row, 4 columns), the spectral scale and the exact DC row. A
    // 128 x 128 tile reduced by one CTA (BIG: 32 groups per thread) forms them group by group
    // in its epilogue instead, to stay within its registers.
    constexpr bool BIG = GPT > 16;
    static_assert(!BIG || (S == 1 && !PUSH), "a 128-wide tile is reduced by its own CTA");
    int grow[BIG ? 1 : GPT], gcol[BIG ? 1 : GPT];
    float4 sc[BIG ? 1 : GPT];
    if constexpr (!BIG) {
#pragma unroll
        for (int j = 0; j < GPT; ++j) {
            const int e = threadIdx.x + j * TC_THREADS;
            grow[j] = rank * R + e / (BN / 4);
            gcol[j] = (e % (BN / 4)) * 4;
            sc[j] = epi_scale(g, m0 + grow[j], n0 + gcol[j], z, run);
        }
    }

    static_assert(!PUSH || S > 1, "the push form reduces over S > 1 partials");
    // the receive area of the push form: S slots of R rows at RED_LD floats
    float* recv = reinterpret_cast<float*>(t.base + STAGES * STAGE_BYTES + 256);
    if (PUSH) {
        bool acc_ok = false;
        if (run) {
            acc_ok = __all_sync(0xffffffffu, mbar_wait(t.accb, t.acc_n & 1) ? 1 : 0) != 0;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        cluster_wait();  // every CTA of the cluster has started (arrived after its set-up)
        if (run && acc_ok) {
            const int r = 32 * warp + lane;  // this thread's tile row
            const int dst = r / R, rr = r % R;
            const uint32_t remote = map_rank(smem_u32(recv + (rank * R + rr) * RED_LD), static_cast<uint32_t>(group0 + dst));
#pragma unroll 1
            for (int c = 0; c < BN; c += 32) {
                float v[32];
                tmem_ld32(t.tmem + (static_cast<uint32_t>(32 * warp) << 16) + c, v);
#pragma unroll
                for (int i = 0; i < 32; i += 4) st_dsmem4(remote + 4u * static_cast<uint32_t>(c + i), v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        } else if (run && threadIdx.x == 0) {
            atomicCAS(g.err, 0, SPG_E_CUDA);
        }
        const int ok_cta = __syncthreads_and(!run || acc_ok ? 1 : 0);
        cluster_sync_all();  // every CTA's rows are in their reducers' slots
        if (run && ok_cta) {
#pragma unroll
            for (int j = 0; j < GPT; ++j) {
                const int rr = grow[j] - rank * R;
                float v[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    const float4 a = *reinterpret_cast<const float4*>(recv + (q * R + rr) * RED_LD + gcol[j]);
                    v[0] += a.x;
                    v[1] += a.y;
                    v[2] += a.z;
                    v[3] += a.w;
                }
                tile_store(g, m0 + grow[j], n0 + gcol[j], z, sc[j], v);
            }
        }
        if (run) {
            t.it += static_cast<uint32_t>(s1 - s0);
            t.acc_n += 1;
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        return;
    }

    // stage this CTA's partial tile (TMEM lane = tile row; warp w owns rows 32w..32w+31)
    bool acc_ok = false;
    if (run) {
        acc_ok = __all_sync(0xffffffffu, mbar_wait(t.accb, t.acc_n & 1) ? 1 : 0) != 0;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (acc_ok) {
            const int r = 32 * warp + lane;
#pragma unroll 1
            for (int c = 0; c < BN; c += 32) {
                float v[32];
                tmem_ld32(t.tmem + (static_cast<uint32_t>(32 * warp) << 16) + c, v);
#pragma unroll
                for (int i = 0; i < 32; i += 4)
                    *reinterpret_cast<float4*>(red + r * RED_LD + c + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        } else if (threadIdx.x == 0) {
            atomicCAS(g.err, 0, SPG_E_CUDA);
        }
    }
    const int ok_cta = __syncthreads_and(acc_ok ? 1 : 0);
    if (S > 1) cluster_sync_all();  // every CTA of the cluster has staged its partial
    if constexpr (BIG) {
        if (ok_cta) {
#pragma unroll 4
            for (int j = 0; j < GPT; ++j) {
                const int e = threadIdx.x + j * TC_THREADS;
                const int row = e / (BN / 4), col = (e % (BN / 4)) * 4;
                const float4 a = *reinterpret_cast<const float4*>(red + row * RED_LD + col);
                float v[4] = {0.f, 0.f, 0.f, 0.f};  // the sum of the one partial, as below
                v[0] += a.x;
                v[1] += a.y;
                v[2] += a.z;
                v[3] += a.w;
                tile_store(g, m0 + row, n0 + col, z, epi_scale(g, m0 + row, n0 + col, z, run), v);
            }
        }
    } else if (ok_cta) {
        const uint32_t red_addr = smem_u32(red);
        float4 parts[GPT][S];
#pragma unroll
        for (int j = 0; j < GPT; ++j) {
            const uint32_t off = 4u * static_cast<uint32_t>(grow[j] * RED_LD + gcol[j]);
#pragma unroll
            for (int q = 0; q < S; ++q)
                parts[j][q] = S > 1 ? ld_dsmem4(map_rank(red_addr, static_cast<uint32_t>(group0 + q)) + off)
                                    : *reinterpret_cast<const float4*>(red + grow[j] * RED_LD + gcol[j]);
        }
#pragma unroll
        for (int j = 0; j < GPT; ++j) {
            float v[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int q = 0; q < S; ++q) {
                v[0] += parts[j][q].x;
                v[1] += parts[j][q].y;
                v[2] += parts[j][q].z;
                v[3] += parts[j][q].w;
            }
            tile_store(g, m0 + grow[j], n0 + gcol[j], z, sc[j], v);
        }
    }
    if (S > 1) cluster_sync_all();  // no CTA reuses its ring while another may still read it
    if (run) {
        t.it += static_cast<uint32_t>(s1 - s0);
        t.acc_n += 1;
    }
    // the TMEM reads above are done before the next tile's MMAs overwrite the accumulator
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
}

// Grid (S, N/BN, (M/128) * batch), cluster (S, 1, 1): the S CTAs of a cluster share one
// 128 x BN output tile and split its K/64 K slabs evenly (split-K), one tile per CTA.
// PUSH: the partials are reduced in the push form (gemm_tile).
template <int BN, int STAGES, int S, bool PUSH = false>
__global__ void __launch_bounds__(TC_THREADS, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const TcArgs g) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    TileState t;
    tile_setup<BN, STAGES>(smem_raw, t);
    if (PUSH) cluster_arrive_relaxed();  // waited for before the first store into a peer
    // everything above touched only this CTA's shared memory and TMEM: wait for the kernel
    // that produced the operands only now
    pdl_wait();
    pdl_trigger();
    const int tiles_m = g.M / TC_BM;
    gemm_tile<BN, STAGES, S, PUSH>(tmA, tmB, g, (blockIdx.z % tiles_m) * TC_BM, blockIdx.y * BN,
                                   blockIdx.z / tiles_m, blockIdx.x, 0, true, t);
    tile_teardown<BN>(t);
}

// ------------------------------------------------------------------ the fused one-grid solve
// tc_fused_kernel runs a one-grid solve's chain in one launch: G1, the split of G1's output
// (its rows minus their means into BF16 planes, with the exact row sums), G2, G3 and G4, with a
// grid-wide barrier between phases. Every phase computes what the separate launches compute,
// with the same tiles, the same split-K factors and the same reduction orders, so the results
// are the same bits; what goes away is four launches and their drains. The grid is kFusedClusters
// clusters of kFusedCluster CTAs, one CTA per SM, all resident at once (the host checks the
// cluster occupancy first); a phase's tiles go round-robin over the clusters, S CTAs per tile.
// The barrier is a counter in global memory: each CTA arrives once per phase and waits until all
// have, at most kWaitNs, then records SPG_E_CUDA and goes on without waiting (later phases skip
// their work once the flag is set). The last CTA to finish zeroes the counter for the next launch. Writes made by one phase reach the next phase's TMA loads
// through release / acquire at GPU scope and async-proxy fences on both sides.
constexpr int kFusedCluster = 4;
constexpr int kFusedClusters = 32;
constexpr int kPrepThreads = 256;  // prep_split_kernel's block (its reduction order is the split's)

struct FusedMaps {
    CUtensorMap a[4], b[4];  // G1..G4: A (bases) and B (data planes)
};

struct FusedArgs {
    TcArgs g[4];
    int split[4];               // split-K factor of each contraction (pick_splits)
    const float* t0t32;         // G1's FP32 output, rows of `len` at stride ld
    int rows, len;
    int64_t ld;
    uint16_t* t0t_s;            // its split planes (lo plane at + plane_stride), row r at r * ld
    int64_t plane_stride;
    float* sum_t;               // exact row sums
    unsigned int* bar;          // [0] arrivals, [1] exits: zero at launch, zeroed again by the last CTA
    int* err;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All CTAs of the grid: arrive on *bar and wait until `target` arrivals (bounded).
__device__ void grid_sync(unsigned int* bar, unsigned int target, int* err) {
    asm volatile("fence.proxy.async.global;" ::: "memory");  // this thread's stores, for the async proxy
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned long long t0 = gtime();
        while (ld_acquire_u32(bar) < target) {
            if (__ldcg(err) != 0) break;
            if (gtime() - t0 > kWaitNs) {
                atomicCAS(err, 0, SPG_E_CUDA);
                break;
            }
        }
        __threadfence();
        asm volatile("fence.proxy.async.global;" ::: "memory");  // before this thread's next TMA loads
    }
    __syncthreads();
}

// The split of G1's output, one warp per row, with exactly the arithmetic of prep_split_kernel
// (center = 1, one segment per row): its 256 threads' partial sums (elements t, t+256, ... in
// order), the warp trees of lane 0, and the eight warp sums in order.
__device__ void fused_split(const FusedArgs& a) {
    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (TC_THREADS / 32) + (threadIdx.x >> 5), nw = gridDim.x * (TC_THREADS / 32);
    for (int r = gw; r < a.rows; r += nw) {
        const float* p = a.t0t32 + r * a.ld;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kPrepThreads / 32; ++w) {
            const int t = 32 * w + lane;  // the prep kernel's thread t
            double v = 0.0;
            for (int i = t; i < a.len; i += kPrepThreads) v += static_cast<double>(p[i]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            s += __shfl_sync(0xffffffffu, v, 0);
        }
        const float mean = static_cast<float>(s / a.len);
        if (lane == 0) a.sum_t[r] = static_cast<float>(s);
        uint16_t* hi = a.t0t_s + r * a.ld;
        uint16_t* lo = hi + a.plane_stride;
        for (int i = lane; i < a.len; i += 32) {
            uint16_t h, l;
            split_bf16(p[i] - mean, h, l);
            hi[i] = h;
            lo[i] = l;
        }
    }
}

// One contraction of the fused solve: its tiles round-robin over the clusters, 4/S tiles per
// cluster and round; every CTA of a cluster takes the same number of rounds.
template <int BN, int STAGES, int S>
__device__ void fused_gemm(const CUtensorMap& tmA, const CUtensorMap& tmB, const TcArgs& g, TileState& t) {
    const int tiles_m = g.M / TC_BM, tiles = tiles_m * (g.N / BN);
    const int crank = static_cast<int>(blockIdx.x % kFusedCluster), cid = static_cast<int>(blockIdx.x / kFusedCluster);
    const int per = kFusedCluster / S, ncl = static_cast<int>(gridDim.x) / kFusedCluster;
    const int group = crank / S, rank = crank % S;
    const int rounds = (tiles + ncl * per - 1) / (ncl * per);
    for (int rd = 0; rd < rounds; ++rd) {
        const int tile = (rd * ncl + cid) * per + group;
        const bool active = tile < tiles;
        const int tt = active ? tile : 0;
        gemm_tile<BN, STAGES, S>(tmA, tmB, g, (tt % tiles_m) * TC_BM, (tt / tiles_m) * BN, 0, rank, group * S, active,
                                 t);
    }
}

template <int BN, int STAGES, int S>
__device__ __forceinline__ void fused_phase(const FusedMaps& mp, const FusedArgs& a, int k, TileState& t) {
    fused_gemm<BN, STAGES, S>(mp.a[k], mp.b[k], a.g[k], t);
}

template <int BN, int STAGES>
__device__ void fused_phase_any(const FusedMaps& mp, const FusedArgs& a, int k, TileState& t) {
    switch (a.split[k]) {  // uniform over the grid
        case 4: fused_phase<BN, STAGES, 4>(mp, a, k, t); break;
        case 2: fused_phase<BN, STAGES, 2>(mp, a, k, t); break;
        default: fused_phase<BN, STAGES, 1>(mp, a, k, t); break;
    }
}

template <int BN, int STAGES>
__global__ void __launch_bounds__(TC_THREADS, 1)
    tc_fused_kernel(const __grid_constant__ FusedMaps mp, const __grid_constant__ FusedArgs a) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    TileState t;
    tile_setup<BN, STAGES>(smem_raw, t);
    pdl_wait();
    pdl_trigger();
    const unsigned int n = gridDim.x;
    fused_phase_any<BN, STAGES>(mp, a, 0, t);  // G1
    grid_sync(a.bar, n, a.err);
    if (__ldcg(a.err) == 0) fused_split(a);
    grid_sync(a.bar, 2 * n, a.err);
    fused_phase_any<BN, STAGES>(mp, a, 1, t);  // G2
    grid_sync(a.bar, 3 * n, a.err);
    fused_phase_any<BN, STAGES>(mp, a, 2, t);  // G3
    grid_sync(a.bar, 4 * n, a.err);
    fused_phase_any<BN, STAGES>(mp, a, 3, t);  // G4
    // the last CTA out (every CTA has left its last barrier by then) zeroes the counters for
    // the next launch
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(a.bar + 1, 1u) == n - 1) {
        atomicExch(a.bar, 0u);
        atomicExch(a.bar + 1, 0u);
    }
    tile_teardown<BN>(t);
}

// Row means (FP64) of `seg`-long row segments; writes the split BF16 planes of
// (value - mean) when `center`, else of the value, and the exact segment sums.
// One block per (row, segment); outputs planes[row][col] with lo plane at + plane_stride.
// The segment sum is a fixed-order block reduction (each thread's elements in order, warp
// trees, then the warp sums in order).
__global__ void __launch_bounds__(kPrepThreads) prep_split_kernel(const float* src, int rows, int nseg, int64_t ld,
                                                                  int seg, int center, uint16_t* planes,
                                                                  int64_t plane_stride, float* sums) {
    pdl_wait();
    pdl_trigger();
    __shared__ double wsum[kPrepThreads / 32];
    __shared__ float mean_s;
    const int w = blockIdx.x, tid = threadIdx.x;
    const int r = w % rows, sg = w / rows;
    const float* p = src + r * ld + static_cast<int64_t>(sg) * seg;
    float mean = 0.f;
    if (center) {
        double v = 0.0;
        for (int i = tid; i < seg; i += kPrepThreads) v += static_cast<double>(p[i]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) wsum[tid >> 5] = v;
        __syncthreads();
        if (tid == 0) {
            double s = 0.0;
            for (int k = 0; k < kPrepThreads / 32; ++k) s += wsum[k];
            mean_s = static_cast<float>(s / seg);
            if (sums) sums[w] = static_cast<float>(s);
        }
        __syncthreads();
        mean = mean_s;
    }
    uint16_t* hi = planes + r * ld + static_cast<int64_t>(sg) * seg;
    uint16_t* lo = hi + plane_stride;
    for (int i = tid; i < seg; i += kPrepThreads) {
        uint16_t h, l;
        split_bf16(p[i] - mean, h, l);
        hi[i] = h;
        lo[i] = l;
    }
}

// ------------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        SPG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        SPG_REQUIRE(q == cudaDriverEntryPointSuccess && p, SPG_E_CUDA, "cuTensorMapEncodeTiled unavailable");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// 2-D bf16 tensor map over a [rows][cols] plane stack, box 64 (K) x box_rows.
CUtensorMap make_map(const uint16_t* ptr, int64_t rows, int64_t cols, int box_rows) {
    CUtensorMap m;
    cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
    cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols * 2)};
    cuuint32_t box[2] = {static_cast<cuuint32_t>(TC_BK), static_cast<cuuint32_t>(box_rows)};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<uint16_t*>(ptr), dims,
                                   strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    SPG_REQUIRE(r == CUDA_SUCCESS, SPG_E_CUDA, "cuTensorMapEncodeTiled failed");
    return m;
}

constexpr int TC_BN = 64;
constexpr int TC_STAGES = 4;
constexpr size_t tc_smem_bytes() {
    // 1024-byte alignment slack + stage ring (four planes per stage) + mbarriers + TMEM slot
    return 1024 + TC_STAGES * 2 * (TC_BM * TC_BK * 2 + TC_BN * TC_BK * 2) + (2 * TC_STAGES + 1) * 8 + 128;
}
static_assert(tc_smem_bytes() <= 227 * 1024, "ring exceeds the shared memory of one CTA");
// The push form's launches (S > 1): each CTA streams at most K/64/2 slabs, so a 3-deep ring,
// then 256 bytes of barriers and the receive area of S slots x (128/S) rows x (TC_BN + 4) floats.
constexpr int TC_PUSH_STAGES = 3;
constexpr size_t tc_push_smem_bytes() {
    return 1024 + TC_PUSH_STAGES * 2 * (TC_BM * TC_BK * 2 + TC_BN * TC_BK * 2) + 256 + TC_BM * (TC_BN + 4) * 4;
}
static_assert(tc_push_smem_bytes() <= 227 * 1024, "push form exceeds the shared memory of one CTA");

// Wide launches: 128 x 128 tiles, one CTA each (no split-K), for contractions whose one grid
// has at least a full wave of them (2048^2 grids, and G4 from 1024^2): each K slab then brings
// 64 KB for twice the MMAs of a 128 x 64 tile's 48 KB, where the L2 -> shared-memory fill
// bounds the large grids. Chosen from one grid's problem, so a grid's result does not depend
// on the batch it is solved in. SPG_TC_WIDE=0 keeps 64-wide tiles everywhere.
constexpr int TC_WIDE_BN = 128;
constexpr int TC_WIDE_STAGES = 3;
constexpr size_t tc_wide_smem_bytes() {
    return 1024 + TC_WIDE_STAGES * 2 * (TC_BM * TC_BK * 2 + TC_WIDE_BN * TC_BK * 2) + (2 * TC_WIDE_STAGES + 1) * 8 + 128;
}
static_assert(tc_wide_smem_bytes() <= 227 * 1024, "wide ring exceeds the shared memory of one CTA");
bool tc_wide() {
    static const bool on = [] {
        const char* e = std::getenv("SPG_TC_WIDE");
        return !(e && e[0] == '0');
    }();
    return on;
}

// SPG_TC_PUSH=0: the pull form for every launch (the receive area unused).
bool tc_push() {
    static const bool on = [] {
        const char* e = std::getenv("SPG_TC_PUSH");
        return !(e && e[0] == '0');
    }();
    return on;
}

struct TcState {
    // tensor maps: bases (A operands) and data planes (B operands)
    CUtensorMap cy, cx, bcat, acat;         // A: box rows 128
    CUtensorMap rho_b, t0t_b, p_b, t12t_b;  // B: box rows TC_BN
    CUtensorMap rho_w, t0t_w, p_w, t12t_w;  // B: box rows TC_WIDE_BN (the wide launches)
    float* t0t32 = nullptr;                 // FP32 T0t (G1 output, before its DC split)
    float* sums = nullptr;                  // DC row sums (rho rows, T0t rows per grid)
    int* err = nullptr;
    unsigned int* bar = nullptr;            // the fused solve's grid barrier counter
    int8_t wide[4] = {-1, -1, -1, -1};      // G1..G4 as wide tiles (tc_tune); -1 not chosen yet
};

// Split-K factor: the largest S in {8, 4, 2} (S divides the 128 tile rows, which the
// reduction splits into S bands) dividing the slab count, with one grid's tiles * S CTAs
// in one wave over the 148 SMs (1 CTA per SM), else 1. It depends on one grid's problem
// only, so a grid's result does not depend on the batch it is solved in.
int pick_splits(int tiles, int slabs) {
    for (int s : {8, 4, 2})
        if (slabs % s == 0 && tiles * s <= 148) return s;
    return 1;
}

// Whether contraction g may run as wide tiles, and whether its one grid (grid_tiles 64-wide
// tiles) has the full wave of them that makes the wide form the default.
bool wide_valid(const TcArgs& g) { return tc_wide() && g.N % TC_WIDE_BN == 0 && g.M % TC_BM == 0; }
bool wide_default(const TcArgs& g, int grid_tiles) { return wide_valid(g) && grid_tiles / 2 >= 148; }

void launch_tc(const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap& b_wide, const TcArgs& g, int batch,
               int grid_tiles, bool wide, cudaStream_t s) {
    SPG_REQUIRE(g.M % TC_BM == 0 && g.N % TC_BN == 0 && g.K % TC_BK == 0, SPG_E_INVALID,
                "tensor-core GEMM dims must be tile multiples");
    if (wide && wide_valid(g)) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(1, g.N / TC_WIDE_BN, (g.M / TC_BM) * batch);
        cfg.blockDim = dim3(TC_THREADS);
        cfg.dynamicSmemBytes = tc_wide_smem_bytes();
        cfg.stream = s;
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
        attr[1].id = cudaLaunchAttributePriority;
        attr[1].val.priority = launch_priority(true);
        cfg.attrs = attr;
        cfg.numAttrs = 2;
        SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_WIDE_BN, TC_WIDE_STAGES, 1>, a, b_wide, g));
        count_launch();
        return;
    }
    const int S = pick_splits(grid_tiles, g.K / TC_BK);
    cudaLaunchConfig_t cfg = {};
    const bool push = S > 1 && tc_push();
    cfg.gridDim = dim3(S, g.N / TC_BN, (g.M / TC_BM) * batch);
    cfg.blockDim = dim3(TC_THREADS);
    cfg.dynamicSmemBytes = push ? tc_push_smem_bytes() : tc_smem_bytes();
    cfg.stream = s;
    cudaLaunchAttribute attr[3];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = S;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    attr[2].id = cudaLaunchAttributePriority;
    attr[2].val.priority = launch_priority(true);
    cfg.attrs = attr;
    cfg.numAttrs = 3;
    switch (S) {
        case 8:
            if (push) SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_PUSH_STAGES, 8, true>, a, b, g));
            else SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_STAGES, 8>, a, b, g));
            break;
        case 4:
            if (push) SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_PUSH_STAGES, 4, true>, a, b, g));
            else SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_STAGES, 4>, a, b, g));
            break;
        case 2:
            if (push) SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_PUSH_STAGES, 2, true>, a, b, g));
            else SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_STAGES, 2>, a, b, g));
            break;
        default: SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<TC_BN, TC_STAGES, 1>, a, b, g)); break;
    }
    count_launch();
}

// Whether kFusedClusters clusters of the fused kernel fit on the device at once (checked once
// per device); SPG_POISSON_FUSED=0 turns the fused solve off.
bool fused_resident() {
    const char* off = std::getenv("SPG_POISSON_FUSED");
    if (off && off[0] == '0') return false;
    static std::mutex mu;
    static std::vector<std::pair<int, bool>> seen;
    int dev = 0;
    SPG_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& e : seen)
        if (e.first == dev) return e.second;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kFusedCluster * kFusedClusters);
    cfg.blockDim = dim3(TC_THREADS);
    cfg.dynamicSmemBytes = tc_smem_bytes();
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kFusedCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    const bool ok = cudaOccupancyMaxActiveClusters(&clusters, tc_fused_kernel<TC_BN, TC_STAGES>, &cfg) == cudaSuccess &&
                    clusters >= kFusedClusters;
    cudaGetLastError();
    seen.emplace_back(dev, ok);
    return ok;
}

void launch_fused(const FusedMaps& mp, const FusedArgs& a, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kFusedCluster * kFusedClusters);
    cfg.blockDim = dim3(TC_THREADS);
    cfg.dynamicSmemBytes = tc_smem_bytes();
    cfg.stream = s;
    cudaLaunchAttribute attr[3];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kFusedCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    attr[2].id = cudaLaunchAttributePriority;
    attr[2].val.priority = launch_priority(true);
    cfg.attrs = attr;
    cfg.numAttrs = 3;
    SPG_CUDA(cudaLaunchKernelEx(&cfg, tc_fused_kernel<TC_BN, TC_STAGES>, mp, a));
    count_launch();
}

void prep_split(const float* src, int rows, int cols, int64_t ld, int seg, int center, uint16_t* planes,
                int64_t plane_stride, float* sums, cudaStream_t s) {
    launch_pdl(prep_split_kernel, dim3(rows * (cols / seg)), dim3(kPrepThreads), 0, s, src, rows, cols / seg, ld,
               seg, center, planes, plane_stride, sums);
}

void split_host(const std::vector<float>& v, std::vector<uint16_t>& out) {
    const size_t n = v.size();
    out.resize(2 * n);
    for (size_t i = 0; i < n; ++i) {
        const __nv_bfloat16 h = __float2bfloat16_rn(v[i]);
        const __nv_bfloat16 l = __float2bfloat16_rn(v[i] - __bfloat162float(h));
        out[i] = __bfloat16_as_ushort(h);
        out[n + i] = __bfloat16_as_ushort(l);
    }
}

}  // namespace

bool tc_supported(int nx, int ny) { return nx >= 128 && ny >= 128 && nx % 128 == 0 && ny % 128 == 0; }

void tc_plan_create(PoissonPlan& pl, const std::vector<float>& cy, const std::vector<float>& cx,
                    const std::vector<float>& bcat, const std::vector<float>& acat) {
    const int64_t X = pl.nx, Y = pl.ny, B = pl.batch_cap;
    auto up = [&](uint16_t*& dst, const std::vector<uint16_t>& h) {
        dst = static_cast<uint16_t*>(dev_alloc(h.size() * 2, &pl.stream));
        pl.bytes += h.size() * 2;
        upload_bytes(dst, h.data(), h.size() * 2, pl.stream);
    };
    std::vector<uint16_t> sp;
    split_host(cy, sp);
    up(pl.cy_s, sp);
    split_host(cx, sp);
    up(pl.cx_s, sp);
    split_host(bcat, sp);
    up(pl.bcat_s, sp);
    split_host(acat, sp);
    up(pl.acat_s, sp);
    auto al16 = [&](uint16_t*& p, size_t n) {
        p = static_cast<uint16_t*>(dev_alloc(n * 2, &pl.stream));
        pl.bytes += n * 2;
    };
    al16(pl.rho_s, 2 * B * X * Y);
    al16(pl.t0t_s, 2 * B * X * Y);
    al16(pl.p_s, 2 * B * X * Y);
    al16(pl.t12t_s, 4 * B * X * Y);
    auto* st = new TcState;
    pl.tc = st;
    st->t0t32 = static_cast<float*>(dev_alloc(B * X * Y * 4, &pl.stream));
    st->sums = static_cast<float*>(dev_alloc(2 * B * std::max(X, Y) * 4, &pl.stream));
    st->err = static_cast<int*>(dev_alloc(4, &pl.stream));
    SPG_CUDA(cudaMemsetAsync(st->err, 0, 4, pl.stream));
    st->bar = static_cast<unsigned int*>(dev_alloc(16, &pl.stream));
    SPG_CUDA(cudaMemsetAsync(st->bar, 0, 16, pl.stream));
    pl.bytes += B * X * Y * 4 + 2 * B * std::max(X, Y) * 4 + 4;
    st->cy = make_map(pl.cy_s, 2 * Y, Y, TC_BM);
    st->cx = make_map(pl.cx_s, 2 * X, X, TC_BM);
    st->bcat = make_map(pl.bcat_s, 4 * Y, Y, TC_BM);
    st->acat = make_map(pl.acat_s, 4 * X, X, TC_BM);
    st->rho_b = make_map(pl.rho_s, 2 * B * X, Y, TC_BN);
    st->t0t_b = make_map(pl.t0t_s, 2 * Y, B * X, TC_BN);
    st->p_b = make_map(pl.p_s, 2 * B * X, Y, TC_BN);
    st->t12t_b = make_map(pl.t12t_s, 4 * Y, B * X, TC_BN);
    st->rho_w = make_map(pl.rho_s, 2 * B * X, Y, TC_WIDE_BN);
    st->t0t_w = make_map(pl.t0t_s, 2 * Y, B * X, TC_WIDE_BN);
    st->p_w = make_map(pl.p_s, 2 * B * X, Y, TC_WIDE_BN);
    st->t12t_w = make_map(pl.t12t_s, 4 * Y, B * X, TC_WIDE_BN);
    // per device (the attribute is a property of the kernel on the current device)
    const int bytes = static_cast<int>(tc_smem_bytes());
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_STAGES, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_STAGES, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_STAGES, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_STAGES, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_fused_kernel<TC_BN, TC_STAGES>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_WIDE_BN, TC_WIDE_STAGES, 1>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(tc_wide_smem_bytes())));
    const int push_bytes = static_cast<int>(tc_push_smem_bytes());
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_PUSH_STAGES, 2, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, push_bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_PUSH_STAGES, 4, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, push_bytes));
    SPG_CUDA(cudaFuncSetAttribute(tc_gemm_kernel<TC_BN, TC_PUSH_STAGES, 8, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, push_bytes));
}

void tc_plan_refill_sines(PoissonPlan& pl, const std::vector<float>& sy_rows, const std::vector<float>& sx_rows) {
    // plane stacks are [hi | lo] of the whole [A; S] matrix: the S rows start half-way into
    // each plane
    const size_t X = pl.nx, Y = pl.ny;
    std::vector<uint16_t> sp;
    split_host(sy_rows, sp);  // sp = [hi(Y*Y) | lo(Y*Y)]
    upload_bytes(pl.bcat_s + Y * Y, sp.data(), Y * Y * 2, pl.stream);
    upload_bytes(pl.bcat_s + 2 * Y * Y + Y * Y, sp.data() + Y * Y, Y * Y * 2, pl.stream);
    split_host(sx_rows, sp);
    upload_bytes(pl.acat_s + X * X, sp.data(), X * X * 2, pl.stream);
    upload_bytes(pl.acat_s + 2 * X * X + X * X, sp.data() + X * X, X * X * 2, pl.stream);
}

void tc_plan_destroy(PoissonPlan& pl) {
    for (uint16_t* q : {pl.cy_s, pl.cx_s, pl.bcat_s, pl.acat_s, pl.rho_s, pl.t0t_s, pl.p_s, pl.t12t_s})
        dev_free(q, pl.stream);
    pl.cy_s = pl.cx_s = pl.bcat_s = pl.acat_s = pl.rho_s = pl.t0t_s = pl.p_s = pl.t12t_s = nullptr;
    if (auto* st = static_cast<TcState*>(pl.tc)) {
        dev_free(st->t0t32, pl.stream);
        dev_free(st->sums, pl.stream);
        dev_free(st->err, pl.stream);
        dev_free(st->bar, pl.stream);
        delete st;
        pl.tc = nullptr;
    }
}

const int* tc_error_flag(const PoissonPlan& pl) {
    const auto* st = static_cast<const TcState*>(pl.tc);
    return st ? st->err : nullptr;
}

bool tc_rho_operand(const PoissonPlan& pl, RhoOperand* out) {
    if (!pl.tc) return false;
    const auto* st = static_cast<const TcState*>(pl.tc);
    out->planes = pl.rho_s;
    out->plane_stride = static_cast<int64_t>(pl.batch_cap) * pl.nx * pl.ny;
    out->ld = pl.ny;
    out->sums = st->sums;
    return true;
}

// The tile-shape tuner. For each contraction whose tiles may be either 128 x 64 or 128 x 128,
// both with one CTA per tile (pick_splits gives no split-K), it times both on the plan's buffers
// (3 launches each after one warm-up, CUDA events on the solve's stream) and keeps the faster;
// the choices are kept per device, grid and batch size for the process, so later plans of the
// same shape skip the measurement. Both forms add the same products in the same order for every
// output, so the choice changes the time of a solve, never its bits. A solve enqueued while its
// stream is being captured (a CUDA graph) takes the default choice (wide_default) instead, and
// so does every solve with SPG_TC_TUNE=0.
void tc_tune(TcState* st, const CUtensorMap* const maps[4][3], const TcArgs* const gs[4], const int batches[4],
             const int tiles[4], cudaStream_t s) {
    int dev = 0;
    SPG_CUDA(cudaGetDevice(&dev));
    const std::array<int64_t, 6> key = {dev, gs[0]->M, gs[1]->M, gs[0]->N, gs[1]->N, batches[1]};
    static std::mutex mu;
    static std::vector<std::pair<std::array<int64_t, 6>, std::array<int8_t, 4>>> known;
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& k : known)
        if (k.first == key) {
            for (int i = 0; i < 4; ++i) st->wide[i] = k.second[i];
            return;
        }
    for (int i = 0; i < 4; ++i) st->wide[i] = wide_default(*gs[i], tiles[i]) ? 1 : 0;
    const char* e = std::getenv("SPG_TC_TUNE");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    SPG_CUDA(cudaStreamIsCapturing(s, &cap));
    if ((e && e[0] == '0') || cap != cudaStreamCaptureStatusNone) return;  // defaults, not kept
    cudaEvent_t e0, e1;
    SPG_CUDA(cudaEventCreate(&e0));
    SPG_CUDA(cudaEventCreate(&e1));
    std::array<int8_t, 4> pick{};
    for (int i = 0; i < 4; ++i) {
        pick[i] = st->wide[i];
        // only where the 64-wide form splits no K either, so both add the same products in order
        if (!wide_valid(*gs[i]) || pick_splits(tiles[i], gs[i]->K / TC_BK) != 1) continue;
        float ms[2] = {0.f, 0.f};
        for (int w = 0; w < 2; ++w) {
            launch_tc(*maps[i][0], *maps[i][1], *maps[i][2], *gs[i], batches[i], tiles[i], w != 0, s);
            SPG_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < 3; ++r)
                launch_tc(*maps[i][0], *maps[i][1], *maps[i][2], *gs[i], batches[i], tiles[i], w != 0, s);
            SPG_CUDA(cudaEventRecord(e1, s));
            SPG_CUDA(cudaEventSynchronize(e1));
            SPG_CUDA(cudaEventElapsedTime(&ms[w], e0, e1));
        }
        pick[i] = ms[1] < ms[0] ? 1 : 0;
        st->wide[i] = pick[i];
        if (const char* log = std::getenv("SPG_TC_TUNE_LOG"); log && log[0] == '1')
            std::fprintf(stderr, "[spg tc tune] G%d %dx%dx%d batch %d: 64-wide %.1f us, 128-wide %.1f us -> %s\n", i + 1,
                         gs[i]->M, gs[i]->N, gs[i]->K, batches[i], 1e3 * ms[0] / 3, 1e3 * ms[1] / 3,
                         pick[i] ? "128-wide" : "64-wide");
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    known.emplace_back(key, pick);
}

void tc_solve(PoissonPlan& pl, int batch, const float* rho, float* phi, float* ex, float* ey,
              cudaStream_t s, bool rho_split_ready) {
    auto* st = static_cast<TcState*>(pl.tc);
    const int X = pl.nx, Y = pl.ny;
    const int64_t Bc = pl.batch_cap, BX = static_cast<int64_t>(batch) * X, XY = static_cast<int64_t>(X) * Y;
    const int64_t BXc = Bc * X;  // plane row/column extents are sized for the plan's capacity
    float* sum_r = st->sums;
    float* sum_t = st->sums + Bc * std::max(X, Y);
    // rho rows minus their means -> split planes (B operand of G1), exact row sums
    if (!rho_split_ready) prep_split(rho, static_cast<int>(BX), Y, Y, Y, 1, pl.rho_s, BXc * Y, sum_r, s);
    // G1: T0t (Y x BX) = Cy . rho'^T in FP32, DC row from the row sums
    TcArgs g1{};
    g1.M = Y; g1.N = static_cast<int>(BX); g1.K = Y;
    g1.a_row0 = 0; g1.a_lo = Y; g1.b_row0 = 0; g1.b_lo = static_cast<int>(BXc); g1.b_col_z = 0;
    g1.mode = TC_F32; g1.out = st->t0t32; g1.out2 = st->t0t32; g1.split = Y; g1.ldc = BXc; g1.out_z = 0;
    g1.row0 = sum_r; g1.row0_z = 0; g1.err = st->err;
    // T0t rows minus their per-grid means -> split planes (B operand of G2), segment sums
    // G2: P_z (X x Y) = Cx . T0t'[:, z]^T, times the spectral scale, DC row from the sums
    TcArgs g2{};
    g2.M = X; g2.N = Y; g2.K = X;
    g2.a_row0 = 0; g2.a_lo = X; g2.b_row0 = 0; g2.b_lo = Y; g2.b_col_z = X;
    g2.mode = TC_SPLIT; g2.planes = pl.p_s; g2.plane_stride = BXc * Y; g2.plane_z = XY; g2.ldc = Y;
    g2.scale = pl.scale; g2.lds = Y; g2.row0 = sum_t; g2.row0_z = Y; g2.err = st->err;
    // G3: T12t (2Y x BX) = [Ay; Sy] . P^T  -> split planes
    TcArgs g3{};
    g3.M = 2 * Y; g3.N = static_cast<int>(BX); g3.K = Y;
    g3.a_row0 = 0; g3.a_lo = 2 * Y; g3.b_row0 = 0; g3.b_lo = static_cast<int>(BXc); g3.b_col_z = 0;
    g3.mode = TC_SPLIT; g3.planes = pl.t12t_s; g3.plane_stride = 2 * static_cast<int64_t>(Y) * BXc;
    g3.plane_z = 0; g3.ldc = BXc; g3.err = st->err;
    // G4 in one launch of 3X rows: [phi; xi_x]_z = [Ax; Sx] . T1t[:, z]^T (rows < 2X) and
    // xi_y_z = Ax . T2t[:, z]^T (the alternate region, rows >= 2X)
    TcArgs g4{};
    g4.M = 3 * X; g4.N = Y; g4.K = X;
    g4.a_row0 = 0; g4.a_lo = 2 * X; g4.b_row0 = 0; g4.b_lo = 2 * Y; g4.b_col_z = X;
    g4.mode = TC_F32; g4.out = phi; g4.out2 = ex; g4.split = X; g4.ldc = Y; g4.out_z = XY; g4.err = st->err;
    g4.m_alt = 2 * X; g4.a_alt_row0 = 0; g4.b_alt_row0 = Y; g4.out3 = ey;
    const int tiles[4] = {(X / TC_BN) * (Y / TC_BM), (Y / TC_BN) * (X / TC_BM), (X / TC_BN) * (2 * Y / TC_BM),
                          (Y / TC_BN) * (3 * X / TC_BM)};
    const int slabs[4] = {Y / TC_BK, X / TC_BK, Y / TC_BK, X / TC_BK};
    int split[4];
    bool fusable = batch == 1;
    for (int k = 0; k < 4; ++k) {
        split[k] = pick_splits(tiles[k], slabs[k]);
        fusable = fusable && split[k] <= kFusedCluster;
    }
    if (fusable && pl.single_launch && fused_resident()) {
        // one launch: G1, the split of T0t, G2, G3, G4 (same tiles, splits and orders as below)
        FusedMaps mp;
        mp.a[0] = st->cy;
        mp.b[0] = st->rho_b;
        mp.a[1] = st->cx;
        mp.b[1] = st->t0t_b;
        mp.a[2] = st->bcat;
        mp.b[2] = st->p_b;
        mp.a[3] = st->acat;
        mp.b[3] = st->t12t_b;
        FusedArgs fa{};
        fa.g[0] = g1;
        fa.g[1] = g2;
        fa.g[2] = g3;
        fa.g[3] = g4;
        for (int k = 0; k < 4; ++k) fa.split[k] = split[k];
        fa.t0t32 = st->t0t32;
        fa.rows = Y;
        fa.len = X;
        fa.ld = BXc;
        fa.t0t_s = pl.t0t_s;
        fa.plane_stride = static_cast<int64_t>(Y) * BXc;
        fa.sum_t = sum_t;
        fa.bar = st->bar;
        fa.err = st->err;
        launch_fused(mp, fa, s);
        return;
    }
    const CUtensorMap* maps[4][3] = {{&st->cy, &st->rho_b, &st->rho_w}, {&st->cx, &st->t0t_b, &st->t0t_w},
                                     {&st->bcat, &st->p_b, &st->p_w}, {&st->acat, &st->t12t_b, &st->t12t_w}};
    const TcArgs* gs[4] = {&g1, &g2, &g3, &g4};
    const int batches[4] = {1, batch, 1, batch};
    if (st->wide[0] < 0) tc_tune(st, maps, gs, batches, tiles, s);
    launch_tc(st->cy, st->rho_b, st->rho_w, g1, 1, tiles[0], st->wide[0] > 0, s);
    prep_split(st->t0t32, Y, static_cast<int>(BX), BXc, X, 1, pl.t0t_s, static_cast<int64_t>(Y) * BXc, sum_t, s);
    launch_tc(st->cx, st->t0t_b, st->t0t_w, g2, batch, tiles[1], st->wide[1] > 0, s);
    launch_tc(st->bcat, st->p_b, st->p_w, g3, 1, tiles[2], st->wide[2] > 0, s);
    launch_tc(st->acat, st->t12t_b, st->t12t_w, g4, batch, tiles[3], st->wide[3] > 0, s);
}

}  // namespace spg
