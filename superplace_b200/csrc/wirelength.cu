// Weighted-average wirelength, its gradient, and HPWL on sm_100a
// (WaWirelength::compute, src/gp/wa_wirelength.cpp:46-180; computeHPWL, src/db/hpwl.cpp:13-39).
//
// Pass 1 runs one thread per net over a degree-sorted net order (so a warp's nets have
// similar degrees and the pin loops stay converged). Per net it forms the extrema, the
// shifted exponentials a+- = exp(+-(x - x_ext)/gamma), b+- and the centred c'+- sums
// (wa_wirelength.cpp:73-127), the WA value and the HPWL term, then writes every pin's
// gradient contribution termMax - termMin (wa_wirelength.cpp:192-221) to a per-pin array.
// Pass 2 (fused into the gradient assembly) sums those contributions per node in
// node->pin CSR order, which is exactly the reference's accumulation order, so the node
// gradient equals the reference's whenever the exponentials agree.
// HPWL is fused into pass 1 (the reference re-walks all pins for it every evaluation).
#include <cfloat>

#include "engine.h"

namespace spg {

namespace {

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

__global__ void __launch_bounds__(RED_THREADS) wa_net_kernel(DevPtrs p, const float* gamma_dev,
                                                             float gamma_host, int use_dev) {
    __shared__ double ws[32];
    const float gam = use_dev ? *gamma_dev : gamma_host;
    const float g = fmax_(gam, 1e-4f);  // kMinGamma, wa_wirelength.cpp:14
    const float invG = fdiv(1.0f, g);
    double wl = 0.0, hp = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < p.num_nets;
         t += gridDim.x * blockDim.x) {
        const int k = p.net_order[t];
        const int b = p.net_start[k], e = p.net_start[k + 1];
        const int deg = e - b;
        if (deg < 2) {  // no WA, no HPWL; pass 2 skips these pins (bPos = 0 marker)
            for (int q = b; q < e; ++q) {
                p.gpx[p.net_pins[q]] = 0.f;
                p.gpy[p.net_pins[q]] = 0.f;
            }
            continue;
        }
        float mxX = -FLT_MAX, mnX = FLT_MAX, mxY = -FLT_MAX, mnY = FLT_MAX;
        for (int q = b; q < e; ++q) {
            const int pin = p.net_pins[q];
            const int nd = p.pin2node[pin];
            const float px = fadd(p.x[nd], p.pox[pin]);
            const float py = fadd(p.y[nd], p.poy[pin]);
            mxX = fmax_(mxX, px);
            mnX = fmin_(mnX, px);
            mxY = fmax_(mxY, py);
            mnY = fmin_(mnY, py);
        }
        // computeHPWL: every net of degree >= 2 (hpwl.cpp:18-32)
        hp += static_cast<double>(fsub(mxX, mnX)) + static_cast<double>(fsub(mxY, mnY));
        if (deg > p.ignore_net_degree) {
            for (int q = b; q < e; ++q) {
                const int pin = p.net_pins[q];
                p.gpx[pin] = 0.f;
                p.gpy[pin] = 0.f;
            }
            continue;
        }
        float bpx = 0.f, bnx = 0.f, cpx = 0.f, cnx = 0.f;
        float bpy = 0.f, bny = 0.f, cpy = 0.f, cny = 0.f;
        for (int q = b; q < e; ++q) {
            const int pin = p.net_pins[q];
            const int nd = p.pin2node[pin];
            const float px = fadd(p.x[nd], p.pox[pin]);
            const float py = fadd(p.y[nd], p.poy[pin]);
            const float dxp = fsub(px, mxX), dxn = fsub(px, mnX);
            const float ap = expf(fmul(dxp, invG));
            const float an = expf(fmul(-dxn, invG));
            bpx = fadd(bpx, ap);
            cpx = fadd(cpx, fmul(dxp, ap));
            bnx = fadd(bnx, an);
            cnx = fadd(cnx, fmul(dxn, an));
            const float dyp = fsub(py, mxY), dyn = fsub(py, mnY);
            const float bp = expf(fmul(dyp, invG));
            const float bn = expf(fmul(-dyn, invG));
            bpy = fadd(bpy, bp);
            cpy = fadd(cpy, fmul(dyp, bp));
            bny = fadd(bny, bn);
            cny = fadd(cny, fmul(dyn, bn));
        }
        // WA_x = (x_max - x_min) + c'+/b+ - c'-/b-   (wa_wirelength.cpp:122-126)
        wl += static_cast<double>(fsub(fadd(fsub(mxX, mnX), fdiv(cpx, bpx)), fdiv(cnx, bnx))) +
              static_cast<double>(fsub(fadd(fsub(mxY, mnY), fdiv(cpy, bpy)), fdiv(cny, bny)));
        for (int q = b; q < e; ++q) {
            const int pin = p.net_pins[q];
            const int nd = p.pin2node[pin];
            const float px = fadd(p.x[nd], p.pox[pin]);
            const float py = fadd(p.y[nd], p.poy[pin]);
            const float dxp = fsub(px, mxX), dxn = fsub(px, mnX);
            const float dyp = fsub(py, mxY), dyn = fsub(py, mnY);
            const float ap = expf(fmul(dxp, invG)), an = expf(fmul(-dxn, invG));
            const float bp = expf(fmul(dyp, invG)), bn = expf(fmul(-dyn, invG));
            p.gpx[pin] = wa_pin_term(dxp, dxn, ap, an, bpx, bnx, cpx, cnx, invG);
            p.gpy[pin] = wa_pin_term(dyp, dyn, bp, bn, bpy, bny, cpy, cny, invG);
        }
    }
    wl = block_sum_d(wl, ws);
    hp = block_sum_d(hp, ws);
    if (threadIdx.x == 0) {
        p.partials[SLOT_WL * RED_BLOCKS + blockIdx.x] = wl;
        p.partials[SLOT_HPWL * RED_BLOCKS + blockIdx.x] = hp;
    }
}

__global__ void wa_node_grad_kernel(DevPtrs p, float* grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.num_movable) return;
    float gx = 0.f, gy = 0.f;
    for (int t = p.node_start[i]; t < p.node_start[i + 1]; ++t) {
        const int pin = p.node_pins[t];
        if (p.pin2net[pin] < 0) continue;
        gx = fadd(gx, p.gpx[pin]);
        gy = fadd(gy, p.gpy[pin]);
    }
    grad[i] = gx;
    grad[p.num_movable + i] = gy;
}

}  // namespace

void launch_wa_nets(const DevPtrs& p, const float* gamma_dev, float gamma_host, int use_dev,
                    cudaStream_t s) {
    wa_net_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(p, gamma_dev, gamma_host, use_dev);
    count_launch();
    SPG_CHECK_LAUNCH();
}

void launch_wa_node_grad(const DevPtrs& p, float* grad, cudaStream_t s) {
    if (p.num_movable <= 0) return;
    wa_node_grad_kernel<<<ceil_div(p.num_movable, 256), 256, 0, s>>>(p, grad);
    count_launch();
    SPG_CHECK_LAUNCH();
}

}  // namespace spg
