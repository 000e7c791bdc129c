// Weighted-average wirelength, its gradient, and HPWL on sm_100a
// (WaWirelength::compute, src/gp/wa_wirelength.cpp:46-180; computeHPWL, src/db/hpwl.cpp:13-39).
//
// Pass 1 sorts nets by degree and cuts them into classes: a net of at most
// kWaThreadNetDegree pins is owned by one thread (its pins in registers, its sums in the
// reference's pin order), a larger one by a group of 8, 16 or 32 lanes, and a net above 32
// pins by a whole warp that loops over its pins. A warp's lanes stay converged and the pin
// loads of a net are issued together. Per net it
// forms the extrema, the shifted exponentials a+- = exp(+-(x - x_ext)/gamma), b+- and the
// centred c'+- sums (wa_wirelength.cpp:73-127), the WA value and the HPWL term, and every
// lane writes its pin's gradient contribution termMax - termMin (wa_wirelength.cpp:192-221)
// to a per-pin array.
// Pass 2 (wl_cells_kernel in optimizer.cu, on the same stream after this pass; the assembly
// reads its sums) adds those contributions per node in node->pin CSR order, which is exactly
// the reference's accumulation order, so the node gradient equals the reference's whenever the
// exponentials agree.
// HPWL is fused into pass 1 (the reference re-walks all pins for it every evaluation).
#include <algorithm>
#include <cfloat>
#include <cstdlib>

#include "engine.h"

namespace spg {

namespace {

// WA blocks per SM (0: one full wave, 5 at 48 registers); SPG_WA_BLOCKS_PER_SM overrides it.
// WA's blocks are resident before the fillers' step that runs beside it, so the registers they
// leave decide how many of the step's blocks fit: three blocks of 48 registers leave room for
// two (6822-6857 iter/s at 211k cells, against 6661-6668 at 64 registers, which left room for
// one; 2 blocks of 48: 6545-6576, 4: 6756-6788; 40 registers spill: 6457-6498).
constexpr int kWaBlocksPerSm = 3;

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_sum_d(double v, double* ws) {
    v = warp_sum_d(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < static_cast<int>(blockDim.x >> 5) ? ws[lane] : 0.0;
        r = warp_sum_d(r);
    }
    __syncthreads();
    return r;
}

// One coordinate axis of the WA gradient of pin with offset d+ = x - x_max, d- = x - x_min.
__device__ __forceinline__ float wa_pin_term(float dp, float dn, float ap, float an, float bp,
                                             float bn, float cp, float cn, float invG) {
    // termMax = ap * (bp + (dp*bp - cp)*invG) / (bp*bp)
    const float tmax = fdiv(fmul(ap, fadd(bp, fmul(fsub(fmul(dp, bp), cp), invG))), fmul(bp, bp));
    // termMin = an * (bn + (cn - dn*bn)*invG) / (bn*bn)
    const float tmin = fdiv(fmul(an, fadd(bn, fmul(fsub(cn, fmul(dn, bn)), invG))), fmul(bn, bn));
    return fsub(tmax, tmin);
}

// Width-G lane-group reductions (xor butterfly inside aligned groups of G lanes).
__device__ __forceinline__ float group_max(float v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v = fmax_(v, __shfl_xor_sync(0xffffffffu, v, o, G));
    return v;
}
__device__ __forceinline__ float group_min(float v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v = fmin_(v, __shfl_xor_sync(0xffffffffu, v, o, G));
    return v;
}
__device__ __forceinline__ float group_sum(float v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v = fadd(v, __shfl_xor_sync(0xffffffffu, v, o, G));
    return v;
}

// Position and gradient slot of entry q of the sorted WA pin order (pinX/pinY: node position
// plus pin offset).
__device__ __forceinline__ void wa_pin(const DevPtrs& p, int q, float& px, float& py, int& slot) {
    const int2 ns = __ldg(p.wa_node_slot + q);
    const float2 o = __ldg(p.wa_off + q);
    px = fadd(__ldg(p.x + ns.x), o.x);
    py = fadd(__ldg(p.y + ns.x), o.y);
    slot = ns.y;
}

// WA value of one net from its extrema and sums (wa_wirelength.cpp:122-126).
__device__ __forceinline__ double wa_value(float mxX, float mnX, float mxY, float mnY,
                                           const float* s) {
    return static_cast<double>(fsub(fadd(fsub(mxX, mnX), fdiv(s[1], s[0])), fdiv(s[3], s[2]))) +
           static_cast<double>(fsub(fadd(fsub(mxY, mnY), fdiv(s[5], s[4])), fdiv(s[7], s[6])));
}

// One net of more than 32 pins (sorted position t), owned by a whole warp that loops over
// its pins.
__device__ void wa_warp_net(const DevPtrs& p, int t, float invG, double& wl, double& hp) {
    const int lane = threadIdx.x & 31;
    const int b = p.wa_start[t], e = p.wa_start[t + 1];
    float mxX = -FLT_MAX, mnX = FLT_MAX, mxY = -FLT_MAX, mnY = FLT_MAX;
    for (int q = b + lane; q < e; q += 32) {
        float px, py;
        int sl;
        wa_pin(p, q, px, py, sl);
        mxX = fmax_(mxX, px);
        mnX = fmin_(mnX, px);
        mxY = fmax_(mxY, py);
        mnY = fmin_(mnY, py);
    }
    mxX = group_max(mxX, 32);
    mnX = group_min(mnX, 32);
    mxY = group_max(mxY, 32);
    mnY = group_min(mnY, 32);
    if (lane == 0) hp += static_cast<double>(fsub(mxX, mnX)) + static_cast<double>(fsub(mxY, mnY));
    if (e - b > p.ignore_net_degree) {
        for (int q = b + lane; q < e; q += 32) {
            const int sl = __ldg(p.wa_node_slot + q).y;
            p.gpx[sl] = 0.f;
            p.gpy[sl] = 0.f;
        }
        return;
    }
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int q = b + lane; q < e; q += 32) {
        float px, py;
        int sl;
        wa_pin(p, q, px, py, sl);
        const float dxp = fsub(px, mxX), dxn = fsub(px, mnX), dyp = fsub(py, mxY), dyn = fsub(py, mnY);
        const float ap = expf(fmul(dxp, invG)), an = expf(fmul(-dxn, invG));
        const float bp = expf(fmul(dyp, invG)), bn = expf(fmul(-dyn, invG));
        s[0] = fadd(s[0], ap);
        s[1] = fadd(s[1], fmul(dxp, ap));
        s[2] = fadd(s[2], an);
        s[3] = fadd(s[3], fmul(dxn, an));
        s[4] = fadd(s[4], bp);
        s[5] = fadd(s[5], fmul(dyp, bp));
        s[6] = fadd(s[6], bn);
        s[7] = fadd(s[7], fmul(dyn, bn));
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) s[i] = group_sum(s[i], 32);
    if (lane == 0) wl += wa_value(mxX, mnX, mxY, mnY, s);
    for (int q = b + lane; q < e; q += 32) {
        float px, py;
        int sl;
        wa_pin(p, q, px, py, sl);
        const float dxp = fsub(px, mxX), dxn = fsub(px, mnX), dyp = fsub(py, mxY), dyn = fsub(py, mnY);
        const float ap = expf(fmul(dxp, invG)), an = expf(fmul(-dxn, invG));
        const float bp = expf(fmul(dyp, invG)), bn = expf(fmul(-dyn, invG));
        p.gpx[sl] = wa_pin_term(dxp, dxn, ap, an, s[0], s[2], s[1], s[3], invG);
        p.gpy[sl] = wa_pin_term(dyp, dyn, bp, bn, s[4], s[6], s[5], s[7], invG);
    }
}

// One net of D pins (2 <= D <= kWaThreadNetDegree), owned by one thread: the extrema, the
// exponentials and the sums in pin order, as wa_wirelength.cpp:84-127 forms them, then the
// pins' gradient terms.
template <int D>
__device__ __forceinline__ void wa_thread_net(const DevPtrs& p, int b, float invG, double& wl, double& hp) {
    float px[D], py[D];
    int sl[D];
#pragma unroll
    for (int j = 0; j < D; ++j) wa_pin(p, b + j, px[j], py[j], sl[j]);
    float mxX = -FLT_MAX, mnX = FLT_MAX, mxY = -FLT_MAX, mnY = FLT_MAX;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        mxX = fmax_(mxX, px[j]);
        mnX = fmin_(mnX, px[j]);
        mxY = fmax_(mxY, py[j]);
        mnY = fmin_(mnY, py[j]);
    }
    hp += static_cast<double>(fsub(mxX, mnX)) + static_cast<double>(fsub(mxY, mnY));
    if (D > p.ignore_net_degree) {
#pragma unroll
        for (int j = 0; j < D; ++j) {
            p.gpx[sl[j]] = 0.f;
            p.gpy[sl[j]] = 0.f;
        }
        return;
    }
    float ap[D], an[D], bp[D], bn[D];
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int j = 0; j < D; ++j) {
        const float dxp = fsub(px[j], mxX), dxn = fsub(px[j], mnX);
        const float dyp = fsub(py[j], mxY), dyn = fsub(py[j], mnY);
        ap[j] = expf(fmul(dxp, invG));
        an[j] = expf(fmul(-dxn, invG));
        bp[j] = expf(fmul(dyp, invG));
        bn[j] = expf(fmul(-dyn, invG));
        s[0] = fadd(s[0], ap[j]);
        s[1] = fadd(s[1], fmul(dxp, ap[j]));
        s[2] = fadd(s[2], an[j]);
        s[3] = fadd(s[3], fmul(dxn, an[j]));
        s[4] = fadd(s[4], bp[j]);
        s[5] = fadd(s[5], fmul(dyp, bp[j]));
        s[6] = fadd(s[6], bn[j]);
        s[7] = fadd(s[7], fmul(dyn, bn[j]));
    }
    wl += wa_value(mxX, mnX, mxY, mnY, s);
#pragma unroll
    for (int j = 0; j < D; ++j) {
        p.gpx[sl[j]] = wa_pin_term(fsub(px[j], mxX), fsub(px[j], mnX), ap[j], an[j], s[0], s[2], s[1], s[3], invG);
        p.gpy[sl[j]] = wa_pin_term(fsub(py[j], mxY), fsub(py[j], mnY), bp[j], bn[j], s[4], s[6], s[5], s[7], invG);
    }
}

// A net of degree D (1..kWaThreadNetDegree, the same for the whole warp) whose pins start at
// entry b of the sorted pin order, in the one-thread class. A 1-pin net has no WA term and
// no HPWL; its gradient slot is written 0.
__device__ __forceinline__ void wa_thread_class_net(const DevPtrs& p, int D, int b, float invG, double& wl, double& hp) {
    switch (D) {
        case 1: {
            const int sl = __ldg(p.wa_node_slot + b).y;
            p.gpx[sl] = 0.f;
            p.gpy[sl] = 0.f;
            break;
        }
        case 2: wa_thread_net<2>(p, b, invG, wl, hp); break;
        case 3: wa_thread_net<3>(p, b, invG, wl, hp); break;
        case 4: wa_thread_net<4>(p, b, invG, wl, hp); break;
        case 5: wa_thread_net<5>(p, b, invG, wl, hp); break;
        default: break;
    }
}
static_assert(kWaThreadNetDegree == 5, "wa_thread_class_net covers degrees up to 5");

// Pass 1 of the WA model and HPWL. Nets of the one-thread class are formed in pin order
// (wa_thread_net). Other nets of degree <= 32 are owned by aligned groups of G = 2..32 lanes
// (G >= degree), one pin per lane: extrema, exponentials and the b+-/c'+- sums are group
// butterflies, and every lane writes its own pin's gradient term. Those sums are formed in
// butterfly order rather than the reference's pin order, so values differ from the
// reference's sequential float sums in the last bits only.
__global__ void __launch_bounds__(RED_THREADS, 5) wa_net_kernel(DevPtrs p, WaClasses wa, const float* gamma_dev,
                                                                float gamma_host, int use_dev) {
    pdl_wait();
    pdl_trigger();
    __shared__ double ws[32];
    const float gam = use_dev ? *gamma_dev : gamma_host;
    const float g = fmax_(gam, 1e-4f);  // kMinGamma, wa_wirelength.cpp:14
    const float invG = fdiv(1.0f, g);
    const int lane = threadIdx.x & 31;
    const int warps_total = wa.warp_begin[wa.n];
    const int wstride = gridDim.x * (blockDim.x >> 5);
    double wl = 0.0, hp = 0.0;
    int c = 0;  // the class of warp w (w only grows)
    for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < warps_total; w += wstride) {
        while (c + 1 < wa.n && w >= wa.warp_begin[c + 1]) ++c;
        const int G = wa.group[c], D = wa.deg[c];
        const int wi = w - wa.warp_begin[c];
        if (G == 0) {
            wa_warp_net(p, wa.net_begin[c] + wi, invG, wl, hp);
            continue;
        }
        if (G == 1) {
            const int i = wi * 32 + lane;
            if (wa.net_begin[c] + i < wa.net_end[c]) wa_thread_class_net(p, D, wa.pin_begin[c] + i * D, invG, wl, hp);
            continue;
        }
        const int sh = wa.shift[c];
        const int gi = lane >> sh, gl = lane & (G - 1);
        const int i = (wi << (5 - sh)) + gi;
        const int deg = wa.net_begin[c] + i < wa.net_end[c] ? D : 0;
        const int b = wa.pin_begin[c] + i * D;
        const bool act = gl < deg;
        float px = 0.f, py = 0.f;
        int sl = 0;
        if (act) wa_pin(p, b + gl, px, py, sl);
        const float mxX = group_max(act ? px : -FLT_MAX, G), mnX = group_min(act ? px : FLT_MAX, G);
        const float mxY = group_max(act ? py : -FLT_MAX, G), mnY = group_min(act ? py : FLT_MAX, G);
        if (gl == 0 && deg >= 2)  // computeHPWL counts every net of degree >= 2 (hpwl.cpp:18-32)
            hp += static_cast<double>(fsub(mxX, mnX)) + static_cast<double>(fsub(mxY, mnY));
        const bool wa_on = deg >= 2 && deg <= p.ignore_net_degree;
        const bool live = act && wa_on;
        const float dxp = fsub(px, mxX), dxn = fsub(px, mnX), dyp = fsub(py, mxY), dyn = fsub(py, mnY);
        const float ap = live ? expf(fmul(dxp, invG)) : 0.f, an = live ? expf(fmul(-dxn, invG)) : 0.f;
        const float bp = live ? expf(fmul(dyp, invG)) : 0.f, bn = live ? expf(fmul(-dyn, invG)) : 0.f;
        float s[8] = {ap, live ? fmul(dxp, ap) : 0.f, an, live ? fmul(dxn, an) : 0.f,
                      bp, live ? fmul(dyp, bp) : 0.f, bn, live ? fmul(dyn, bn) : 0.f};
#pragma unroll
        for (int i = 0; i < 8; ++i) s[i] = group_sum(s[i], G);
        if (act) {
            p.gpx[sl] = live ? wa_pin_term(dxp, dxn, ap, an, s[0], s[2], s[1], s[3], invG) : 0.f;
            p.gpy[sl] = live ? wa_pin_term(dyp, dyn, bp, bn, s[4], s[6], s[5], s[7], invG) : 0.f;
        }
        if (gl == 0 && wa_on) wl += wa_value(mxX, mnX, mxY, mnY, s);
    }
    wl = block_sum_d(wl, ws);
    hp = block_sum_d(hp, ws);
    put_partial(p, SLOT_WL, wl);
    put_partial(p, SLOT_HPWL, hp);
}

__global__ void wa_node_grad_kernel(DevPtrs p, float* grad) {
    pdl_wait();
    pdl_trigger();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.num_movable) return;
    float gx = 0.f, gy = 0.f;
    for (int t = p.slot_start[i]; t < p.slot_start[i + 1]; ++t) {
        gx = fadd(gx, p.gpx[t]);
        gy = fadd(gy, p.gpy[t]);
    }
    grad[i] = gx;
    grad[p.num_movable + i] = gy;
}

}  // namespace

void launch_wa_nets(const DevPtrs& p, const WaClasses& wa, const float* gamma_dev, float gamma_host, int use_dev,
                    cudaStream_t s) {
    // A fixed grid per device, so the FP64 partials keep a fixed owner per block. WA runs
    // beside the fillers' step and the rho -> Poisson chain; at most kWaBlocksPerSm blocks per
    // SM leave each SM room for the step's blocks and a Poisson GEMM block.
    int per_sm = kWaBlocksPerSm;
    if (const char* e = std::getenv("SPG_WA_BLOCKS_PER_SM")) per_sm = std::atoi(e);
    int dev = 0, sms = 0;
    SPG_CUDA(cudaGetDevice(&dev));
    SPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // one warp per lane group of nets: the grid the work fills, at most one wave
    const int full = work_grid(reinterpret_cast<const void*>(wa_net_kernel), wa.warp_begin[wa.n], RED_THREADS / 32);
    const int grid = per_sm > 0 ? std::min(full, std::min(per_sm * sms, RED_CAP)) : full;
    launch_prio(false, wa_net_kernel, dim3(grid), dim3(RED_THREADS), 0, s, p, wa, gamma_dev, gamma_host, use_dev);
}

void launch_wa_node_grad(const DevPtrs& p, float* grad, cudaStream_t s) {
    if (p.num_movable <= 0) return;
    launch_pdl(wa_node_grad_kernel, dim3(ceil_div(p.num_movable, 256)), dim3(256), 0, s, p, grad);
}

}  // namespace spg
