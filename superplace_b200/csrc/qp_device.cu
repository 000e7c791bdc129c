// BiCGSTAB with a Jacobi preconditioner on the device, for the B2B quadratic placement: the
// host solver of qp.cpp (Eigen 3.4.0's BiCGSTAB iteration and restart rule) moved to HBM.
//
// One solve: an init kernel (r = b - A x, r0 = r, the two norms, the diagonal's inverse), a
// host read of its scalars, then a CUDA graph whose WHILE node runs one iteration per pass:
//   rho    rho_old = rho, rho = r0 . r, restart flag = |rho| < eps^2 |r0|^2
//   restart (only when flagged) r = b - A x, r0 = r, rho = |r0|^2, the first restart resets i
//   p      beta = (rho / rho_old)(alpha / w), p = r + beta (p - w v), y = p / diag
//   v      v = A y, alpha = rho / (r0 . v)
//   s      s = r - alpha v, z = s / diag
//   t      t = A z, w = (t . s) / |t|^2 (0 when |t| = 0)
//   x      x += alpha y + w z, r = s - w t, i += 1, continue while |r|^2 > tol^2 |b|^2 and
//          i < max_iter (the last block sets the WHILE node's condition)
// All kernels run on a fixed 1024 x 256 grid, thread g owning rows g, g + 262144, ...; the
// products and sums are __fmul_rn / __fadd_rn (never contracted to FMA), the SpMV sums each
// row in column order, and the dot products follow the order qp_device.h gives the host, so
// the device and host solvers produce the same bits. Scalars live in device memory; each
// reduction's last block (a ticket counter) finalises them.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "qp_device.h"
#include "spgpu.h"

namespace {

int64_t g_qp_launches = 0;

void cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw QpDeviceError(SPG_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct Scalars {
    float rho, rho_old, alpha, w, r0_sq, b_sq, tol2, rr, err, tol;
    int32_t it, restarts, max_iter, restart, cond, passes;
};

struct Vecs {
    int32_t n;
    const int32_t* start;
    const int32_t* col;
    const float* val;
    const float* b;
    float *x, *r, *r0, *v, *p, *y, *z, *s, *t, *inv;
    float* part;        // 3 x kQpBlocks block partials
    uint32_t* ticket;   // one counter per reduction kernel
    Scalars* sc;
    cudaGraphConditionalHandle cond;  // 0 outside the graph
};

__device__ __forceinline__ float row_dot(const Vecs& V, int32_t i, const float* x) {
    float acc = 0.f;
    for (int32_t k = V.start[i]; k < V.start[i + 1]; ++k) acc = __fadd_rn(acc, __fmul_rn(V.val[k], x[V.col[k]]));
    return acc;
}

// Halving tree over the block's 256 values in sh; returns the sum in thread 0.
__device__ __forceinline__ float block_tree(float* sh) {
    for (int h = kQpThreads / 2; h > 0; h >>= 1) {
        __syncthreads();
        if (threadIdx.x < h) sh[threadIdx.x] = __fadd_rn(sh[threadIdx.x], sh[threadIdx.x + h]);
    }
    __syncthreads();
    return sh[0];
}

// Writes this block's sums of the K thread values, and returns true in the last block to
// finish, whose sums[] then hold the K totals in the host's order.
template <int K>
__device__ bool reduce_last(const Vecs& V, int slot, const float (&mine)[K], float (&sums)[K]) {
    __shared__ float sh[kQpThreads];
    __shared__ bool last;
    for (int k = 0; k < K; ++k) {
        sh[threadIdx.x] = mine[k];
        const float v = block_tree(sh);
        if (threadIdx.x == 0) V.part[k * kQpBlocks + blockIdx.x] = v;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&V.ticket[slot], 1u) == kQpBlocks - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    for (int k = 0; k < K; ++k) {
        const volatile float* pk = V.part + k * kQpBlocks;
        const int t = threadIdx.x;
        sh[t] = __fadd_rn(__fadd_rn(__fadd_rn(pk[t], pk[t + 256]), pk[t + 512]), pk[t + 768]);
        sums[k] = block_tree(sh);
        __syncthreads();
    }
    if (threadIdx.x == 0) V.ticket[slot] = 0;
    return true;
}

__device__ __forceinline__ int64_t first_row() { return int64_t(blockIdx.x) * kQpThreads + threadIdx.x; }

__global__ void __launch_bounds__(kQpThreads) k_init(Vecs V) {
    float mine[2] = {0.f, 0.f};
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        float d = 1.f;
        for (int32_t k = V.start[i]; k < V.start[i + 1]; ++k)
            if (V.col[k] == i && V.val[k] != 0.f) d = __fdiv_rn(1.f, V.val[k]);
        V.inv[i] = d;
        const float r = __fsub_rn(V.b[i], row_dot(V, static_cast<int32_t>(i), V.x));
        V.r[i] = r;
        V.r0[i] = r;
        V.v[i] = 0.f;
        V.p[i] = 0.f;
        mine[0] = __fadd_rn(mine[0], __fmul_rn(r, r));
        mine[1] = __fadd_rn(mine[1], __fmul_rn(V.b[i], V.b[i]));
    }
    float sums[2];
    if (reduce_last(V, 0, mine, sums) && threadIdx.x == 0) {
        Scalars& S = *V.sc;
        S.r0_sq = sums[0];
        S.rr = sums[0];
        S.b_sq = sums[1];
        S.tol2 = __fmul_rn(__fmul_rn(S.tol, S.tol), S.b_sq);
        S.rho = S.alpha = S.w = 1.f;
        S.it = 0;
        S.restarts = 0;
        S.cond = (S.b_sq != 0.f && S.rr > S.tol2 && 0 < S.max_iter) ? 1 : 0;
        S.err = S.b_sq != 0.f ? __fsqrt_rn(__fdiv_rn(S.rr, S.b_sq)) : S.tol;
    }
}

__global__ void __launch_bounds__(kQpThreads) k_rho(Vecs V) {
    float mine[1] = {0.f};
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) mine[0] = __fadd_rn(mine[0], __fmul_rn(V.r0[i], V.r[i]));
    float sums[1];
    if (reduce_last(V, 1, mine, sums) && threadIdx.x == 0) {
        Scalars& S = *V.sc;
        const float eps = 1.1920928955078125e-07f;  // float epsilon, 2^-23
        S.rho_old = S.rho;
        S.rho = sums[0];
        S.restart = fabsf(S.rho) < __fmul_rn(__fmul_rn(eps, eps), S.r0_sq) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(kQpThreads) k_restart(Vecs V) {
    if (!V.sc->restart) return;  // every block reads the same flag
    float mine[1] = {0.f};
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        const float r = __fsub_rn(V.b[i], row_dot(V, static_cast<int32_t>(i), V.x));
        V.r[i] = r;
        V.r0[i] = r;
        mine[0] = __fadd_rn(mine[0], __fmul_rn(r, r));
    }
    float sums[1];
    if (reduce_last(V, 2, mine, sums) && threadIdx.x == 0) {
        Scalars& S = *V.sc;
        S.rho = S.r0_sq = sums[0];
        if (S.restarts++ == 0) S.it = 0;
        S.restart = 0;
    }
}

__global__ void __launch_bounds__(kQpThreads) k_p(Vecs V) {
    const Scalars S = *V.sc;
    const float beta = __fmul_rn(__fdiv_rn(S.rho, S.rho_old), __fdiv_rn(S.alpha, S.w));
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        const float p = __fadd_rn(V.r[i], __fmul_rn(beta, __fsub_rn(V.p[i], __fmul_rn(S.w, V.v[i]))));
        V.p[i] = p;
        V.y[i] = __fmul_rn(V.inv[i], p);
    }
}

__global__ void __launch_bounds__(kQpThreads) k_v(Vecs V) {
    float mine[1] = {0.f};
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        const float v = row_dot(V, static_cast<int32_t>(i), V.y);
        V.v[i] = v;
        mine[0] = __fadd_rn(mine[0], __fmul_rn(V.r0[i], v));
    }
    float sums[1];
    if (reduce_last(V, 3, mine, sums) && threadIdx.x == 0) V.sc->alpha = __fdiv_rn(V.sc->rho, sums[0]);
}

__global__ void __launch_bounds__(kQpThreads) k_s(Vecs V) {
    const float alpha = V.sc->alpha;
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        const float s = __fsub_rn(V.r[i], __fmul_rn(alpha, V.v[i]));
        V.s[i] = s;
        V.z[i] = __fmul_rn(V.inv[i], s);
    }
}

__global__ void __launch_bounds__(kQpThreads) k_t(Vecs V) {
    float mine[2] = {0.f, 0.f};
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        const float t = row_dot(V, static_cast<int32_t>(i), V.z);
        V.t[i] = t;
        mine[0] = __fadd_rn(mine[0], __fmul_rn(t, t));
        mine[1] = __fadd_rn(mine[1], __fmul_rn(t, V.s[i]));
    }
    float sums[2];
    if (reduce_last(V, 4, mine, sums) && threadIdx.x == 0) V.sc->w = sums[0] > 0.f ? __fdiv_rn(sums[1], sums[0]) : 0.f;
}

__global__ void __launch_bounds__(kQpThreads) k_x(Vecs V) {
    const float alpha = V.sc->alpha, w = V.sc->w;
    float mine[1] = {0.f};
    for (int64_t i = first_row(); i < V.n; i += kQpGrid) {
        V.x[i] = __fadd_rn(V.x[i], __fadd_rn(__fmul_rn(alpha, V.y[i]), __fmul_rn(w, V.z[i])));
        const float r = __fsub_rn(V.s[i], __fmul_rn(w, V.t[i]));
        V.r[i] = r;
        mine[0] = __fadd_rn(mine[0], __fmul_rn(r, r));
    }
    float sums[1];
    if (reduce_last(V, 5, mine, sums) && threadIdx.x == 0) {
        Scalars& S = *V.sc;
        S.it += 1;
        S.passes += 1;
        S.rr = sums[0];
        S.err = __fsqrt_rn(__fdiv_rn(S.rr, S.b_sq));
        S.cond = (S.rr > S.tol2 && S.it < S.max_iter) ? 1 : 0;
        if (V.cond) cudaGraphSetConditional(V.cond, S.cond ? 1u : 0u);
    }
}

void launch_body(const Vecs& V, cudaStream_t s) {
    const dim3 g(kQpBlocks), b(kQpThreads);
    k_rho<<<g, b, 0, s>>>(V);
    k_restart<<<g, b, 0, s>>>(V);
    k_p<<<g, b, 0, s>>>(V);
    k_v<<<g, b, 0, s>>>(V);
    k_s<<<g, b, 0, s>>>(V);
    k_t<<<g, b, 0, s>>>(V);
    k_x<<<g, b, 0, s>>>(V);
}

constexpr int kBodyKernels = 7;

template <typename T>
void grow(T*& p, size_t& cap, size_t need) {
    if (need <= cap) return;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cu(cudaMalloc(&p, need * sizeof(T)), "cudaMalloc");
    cap = need;
}

}  // namespace

struct QpDevice {
    cudaStream_t stream = nullptr;
    int32_t *start = nullptr, *col = nullptr;
    float *val = nullptr, *vec = nullptr, *part = nullptr;
    uint32_t* ticket = nullptr;
    Scalars* sc = nullptr;
    size_t cap_start = 0, cap_nnz = 0, cap_nnz_v = 0, cap_vec = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    Vecs graph_vecs{};  // the pointers and size the graph was captured with
};

QpDevice* qp_device_create() {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw QpDeviceError(SPG_E_NO_DEVICE, "no CUDA device for the QP solve");
    }
    auto* d = new QpDevice;
    try {
        cu(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cu(cudaMalloc(&d->part, 3 * kQpBlocks * sizeof(float)), "cudaMalloc");
        cu(cudaMalloc(&d->ticket, 8 * sizeof(uint32_t)), "cudaMalloc");
        cu(cudaMemset(d->ticket, 0, 8 * sizeof(uint32_t)), "cudaMemset");
        cu(cudaMalloc(&d->sc, sizeof(Scalars)), "cudaMalloc");
    } catch (...) {
        qp_device_destroy(d);
        throw;
    }
    return d;
}

void qp_device_destroy(QpDevice* d) {
    if (!d) return;
    if (d->exec) cudaGraphExecDestroy(d->exec);
    if (d->graph) cudaGraphDestroy(d->graph);
    for (void* p : {static_cast<void*>(d->start), static_cast<void*>(d->col), static_cast<void*>(d->val),
                    static_cast<void*>(d->vec), static_cast<void*>(d->part), static_cast<void*>(d->ticket),
                    static_cast<void*>(d->sc)})
        if (p) cudaFree(p);
    if (d->stream) cudaStreamDestroy(d->stream);
    delete d;
}

int64_t qp_device_launches() { return g_qp_launches; }

static bool same_vecs(const Vecs& a, const Vecs& b) {
    return a.n == b.n && a.start == b.start && a.col == b.col && a.val == b.val && a.x == b.x && a.sc == b.sc;
}

void qp_device_solve(QpDevice* d, int32_t n, int64_t nnz, const int32_t* row_start, const int32_t* col,
                     const float* val, const float* rhs, float* x, int32_t max_iter, float tol, int32_t* iters,
                     float* err) {
    if (n <= 0) {
        *iters = 0;
        *err = 0.f;
        return;
    }
    grow(d->start, d->cap_start, static_cast<size_t>(n) + 1);
    grow(d->col, d->cap_nnz, static_cast<size_t>(nnz));
    grow(d->val, d->cap_nnz_v, static_cast<size_t>(nnz));
    grow(d->vec, d->cap_vec, static_cast<size_t>(n) * 12);
    cudaStream_t s = d->stream;
    Vecs V{};
    V.n = n;
    V.start = d->start;
    V.col = d->col;
    V.val = d->val;
    float* base = d->vec;
    V.b = base;
    float** slots[] = {&V.x, &V.r, &V.r0, &V.v, &V.p, &V.y, &V.z, &V.s, &V.t, &V.inv};
    for (int k = 0; k < 10; ++k) *slots[k] = base + static_cast<size_t>(k + 1) * n;
    V.part = d->part;
    V.ticket = d->ticket;
    V.sc = d->sc;
    V.cond = 0;
    cu(cudaMemcpyAsync(d->start, row_start, (static_cast<size_t>(n) + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s),
       "upload row_start");
    cu(cudaMemcpyAsync(d->col, col, static_cast<size_t>(nnz) * sizeof(int32_t), cudaMemcpyHostToDevice, s), "upload col");
    cu(cudaMemcpyAsync(d->val, val, static_cast<size_t>(nnz) * sizeof(float), cudaMemcpyHostToDevice, s), "upload val");
    cu(cudaMemcpyAsync(const_cast<float*>(V.b), rhs, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice, s),
       "upload rhs");
    cu(cudaMemcpyAsync(V.x, x, static_cast<size_t>(n) * sizeof(float), cudaMemcpyHostToDevice, s), "upload x");
    Scalars init{};
    init.tol = tol;
    init.max_iter = max_iter;
    cu(cudaMemcpyAsync(d->sc, &init, sizeof(Scalars), cudaMemcpyHostToDevice, s), "upload scalars");
    k_init<<<kQpBlocks, kQpThreads, 0, s>>>(V);
    ++g_qp_launches;
    cu(cudaGetLastError(), "k_init");
    Scalars out{};
    cu(cudaMemcpyAsync(&out, d->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s), "read scalars");
    cu(cudaStreamSynchronize(s), "init");
    if (out.b_sq == 0.f) {  // b = 0: x = 0
        for (int32_t i = 0; i < n; ++i) x[i] = 0.f;
        *iters = max_iter;
        *err = tol;
        return;
    }
    if (out.cond) {
        if (!d->exec || !same_vecs(d->graph_vecs, V)) {
            if (d->exec) cudaGraphExecDestroy(d->exec);
            if (d->graph) cudaGraphDestroy(d->graph);
            d->exec = nullptr;
            d->graph = nullptr;
            cu(cudaGraphCreate(&d->graph, 0), "cudaGraphCreate");
            cudaGraphConditionalHandle h;
            cu(cudaGraphConditionalHandleCreate(&h, d->graph, 1, cudaGraphCondAssignDefault), "conditional handle");
            cudaGraphNodeParams wp{};
            wp.type = cudaGraphNodeTypeConditional;
            wp.conditional.handle = h;
            wp.conditional.type = cudaGraphCondTypeWhile;
            wp.conditional.size = 1;
            cudaGraphNode_t node;
            cu(cudaGraphAddNode(&node, d->graph, nullptr, 0, &wp), "while node");
            Vecs G = V;
            G.cond = h;
            cu(cudaStreamBeginCaptureToGraph(s, wp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal),
               "capture");
            launch_body(G, s);
            cudaGraph_t captured = nullptr;
            const cudaError_t e1 = cudaGetLastError();
            const cudaError_t e2 = cudaStreamEndCapture(s, &captured);
            cu(e1, "capture body");
            cu(e2, "end capture");
            cu(cudaGraphInstantiate(&d->exec, d->graph, 0), "cudaGraphInstantiate");
            d->graph_vecs = V;
        }
        cu(cudaGraphLaunch(d->exec, s), "cudaGraphLaunch");
        cu(cudaMemcpyAsync(&out, d->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s), "read scalars");
        cu(cudaMemcpyAsync(x, V.x, static_cast<size_t>(n) * sizeof(float), cudaMemcpyDeviceToHost, s), "download x");
        cu(cudaStreamSynchronize(s), "solve");
        g_qp_launches += static_cast<int64_t>(out.passes) * kBodyKernels;
    }
    *iters = out.it;
    *err = out.err;
}
