// Gradient assembly, Nesterov update with deferred backtracking, and the per-iteration
// schedule logic of ePlace, all on the device:
//   objAndGrad assembly       src/gp/eplace.cpp:136-203
//   NesterovOptimizer::step   src/numeric/cpu/nesterov.cpp:51-122
//   redoIfOvershot            nesterov.cpp:146-169
//   estimateInitialStep       nesterov.cpp:190-218
//   estimateStep              nesterov.cpp:221-240
//   EPlace::run loop body     eplace.cpp:356-474 (lambda/gamma schedule, stop test,
//                             stagnation snapshots and rollback)
//
// One loop pass is the step kernel, the evaluation, and the assembly that closes it:
//   step_kernel     v' = u - alpha g, u' = v' + m (v' - v), clamp (or the re-evaluation step
//                   when the last decisions asked for one), u' into the node positions and
//                   its fixed-point charge into the density maps; stagnation snapshot copy
//   wl_cells_kernel WA pass 2 of the opt cells (per-cell sum of its pin terms), on the WA
//                   stream after the nets pass, beside the density -> Poisson chain
//   assemble_kernel cell gather + gradient assembly (pass 2's sums read back) and, in the
//                   same pass, the norms |u-uPrev|, |g-gPrevTmp|, their dot and |g|^2; its last
//                   block applies
//                   the step's role rotation, finalizes the evaluation (tau, HPWL, WA value,
//                   force sums) and runs the backtracking test and every per-iteration decision
//                   of the reference (step size, momentum, lambda/gamma, metrics row, stop test,
//                   stagnation and snapshot choice)
// Vector work runs on fixed grids with grid-stride loops, so every FP64 partial sum has a
// fixed owner; the "last block" (an atomic ticket) reduces the partials in a fixed tree, so
// every reduction is deterministic. The host never computes a schedule value.
#include <cfloat>
#include <climits>

#include "engine.h"

namespace spg {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < static_cast<int>(blockDim.x >> 5) ? ws[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Sum of one slot's RED_CAP partials in a fixed order (valid on thread 0). The loads bypass
// L1 so a last block sees the partials other blocks of the same launch wrote.
__device__ __forceinline__ double finalize(const DevPtrs& p, int slot) {
    double v = 0.0;
    for (int j = threadIdx.x; j < RED_CAP; j += blockDim.x) v += __ldcg(p.partials + slot * RED_CAP + j);
    return block_sum(v);
}

// block_sum of N values at once (RED_THREADS-thread blocks), each in block_sum's tree, with
// one pair of barriers for all N; results on thread 0.
template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N]) {
    __shared__ double ws[N][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        v[i] = warp_sum(v[i]);
        if (lane == 0) ws[i][wid] = v[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double r = 0.0;
        if (wid == 0) {
            r = lane < RED_THREADS / 32 ? ws[i][lane] : 0.0;
            r = warp_sum(r);
        }
        v[i] = r;
    }
    __syncthreads();
}

// finalize of N slots at once, each in finalize's tree: all the partial loads are issued
// together and the N block reductions share their barriers.
template <int N>
__device__ __forceinline__ void finalize_n(const DevPtrs& p, const int (&slots)[N], double (&out)[N]) {
    static_assert(RED_CAP % RED_THREADS == 0, "partials must split evenly over the block");
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = 0.0;
#pragma unroll
    for (int j = 0; j < RED_CAP / RED_THREADS; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i)
            out[i] += __ldcg(p.partials + slots[i] * RED_CAP + j * RED_THREADS + threadIdx.x);
    block_sums(out);
}

// Whole-state copies between global and shared memory (all threads of the block). The
// serial decision code of a last block is a chain of dependent reads and writes of the
// state; on a shared copy each link costs a shared-memory access instead of an L2 trip.
__device__ __forceinline__ void state_copy_in(DevState* dst, const DevState* src) {
    static_assert(sizeof(DevState) % 8 == 0, "DevState is copied as 8-byte words");
    const auto* s = reinterpret_cast<const unsigned long long*>(src);
    auto* d = reinterpret_cast<unsigned long long*>(dst);
    for (int j = threadIdx.x; j < static_cast<int>(sizeof(DevState) / 8); j += blockDim.x) d[j] = __ldcg(s + j);
    __syncthreads();
}
__device__ __forceinline__ void state_copy_out(DevState* dst, const DevState* src) {
    __syncthreads();
    const auto* s = reinterpret_cast<const unsigned long long*>(src);
    auto* d = reinterpret_cast<unsigned long long*>(dst);
    for (int j = threadIdx.x; j < static_cast<int>(sizeof(DevState) / 8); j += blockDim.x) d[j] = s[j];
}

// True in exactly one block of the launch: the last to finish its partial sums.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
    __shared__ int is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (is_last) __threadfence();
    return is_last != 0;
}

__device__ __forceinline__ void raise_error(DevState* st, int code) { atomicCAS(&st->error, 0, code); }

// clamp into [lo, hi] with std::min(std::max(v, lo), hi) semantics (eplace.cpp:130-131)
__device__ __forceinline__ float clamp_box(float v, float lo, float hi) {
    const float a = (v < lo) ? lo : v;
    return (hi < a) ? hi : a;
}

// computeGamma (wa_wirelength.cpp:18-29)
__device__ float compute_gamma(float tau, float bin_step) {
    float gamma = fmul(8.0f, bin_step);
    if (tau > 1.0f) gamma = fmul(gamma, 10.0f);
    else if (tau < 0.1f) gamma = fmul(gamma, 0.1f);
    else gamma = fmul(gamma, powf(10.0f, fsub(fmul(20.0f / 9.0f, fsub(tau, 0.1f)), 1.0f)));
    return fmax_(gamma, 1e-4f);
}

// lambdaMultiplier (src/gp/lambda_schedule.h:22-25)
__device__ float lambda_multiplier(double dh, double ref) {
    const double mu = pow(1.1, -dh / ref + 1.0);
    return static_cast<float>(fmin(1.05, fmax(0.95, mu)));
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ float* snap_ptr(const DevPtrs& p, int slot) {
    return p.pool + static_cast<size_t>(NUM_ROLES + slot) * p.vec_stride;
}

// Step size and momentum of this step (nesterov.cpp:87-96, estimateStep :221-240), from
// the norms of the last evaluation.
__device__ void decide_step(const DevPtrs& p, DevState* st) {
    st->grad_norm = static_cast<float>(sqrt(st->gn));
    if (st->iter == 0) {
        st->alpha = st->alpha0;
    } else {
        const double dx = st->dx, dg = st->dg;
        if (dx > 0.0 && dg > 0.0) {
            const double lip = dx / dg;
            float a = static_cast<float>(lip);
            if (p.use_bb) {
                const double yy = dg * dg;
                bool bb_ok = false;
                if (yy > 0.0) {
                    const double bb = st->sy / yy;
                    if (bb > 0.0 && isfinite(bb)) {
                        a = static_cast<float>(bb);
                        bb_ok = true;
                    }
                }
                if (!bb_ok) a = static_cast<float>(fmin(dx / dg, lip));
            }
            st->alpha = a;
        }
    }
    const float an = st->a;
    const float a_next = fmul(0.5f, fadd(1.f, __fsqrt_rn(fadd(fmul(fmul(4.f, an), an), 1.f))));
    st->momentum = fdiv(fsub(an, 1.f), a_next);
    st->a = a_next;
}

// EPlace loop body for iteration st->iter after its last evaluation (eplace.cpp:362-473):
// lambda/gamma schedule, metrics row, stop test, stagnation guard with snapshots. These
// depend only on the evaluated point's tau and HPWL, so they are decided before the update
// is applied; the update of a converged or rolled-back iteration is skipped because the
// delivered point is the evaluated one (or a snapshot).
__device__ void decide_iteration(const DevPtrs& p, DevState* st) {
    const int iter = st->iter;
    if (!(isfinite(st->hpwl) && isfinite(st->tau) && isfinite(st->alpha))) {
        raise_error(st, SPG_E_NON_FINITE);
        st->done = 1;
        return;
    }
    const float eval_lambda = st->lambda, eval_gamma = st->gamma;
    const double dh = st->have_prev ? st->hpwl - st->prev_hpwl : 0.0;
    const bool schedule = st->have_prev && !p.freeze_lambda;
    const float mu = schedule ? lambda_multiplier(dh, st->hpwl_ref) : 1.f;
    if (schedule) st->lambda = fmul(st->lambda, mu);
    st->prev_hpwl = st->hpwl;
    st->have_prev = 1;
    if (!p.freeze_gamma) st->gamma = compute_gamma(st->tau, p.step_x_gamma);
    if (!isfinite(st->lambda) || !isfinite(st->gamma)) {
        raise_error(st, SPG_E_NON_FINITE);
        st->done = 1;
        return;
    }
    if (iter < st->max_iter) {
        spg_iter_metrics& m = p.metrics[iter];
        m.iter = iter;
        m.hpwl = st->hpwl;
        m.overflow = st->tau;
        m.lambda = st->lambda;
        m.gamma = st->gamma;
        m.step_size = st->alpha;
        m.grad_norm_wl = static_cast<float>(st->sum_wl);
        m.grad_norm_den = static_cast<float>(st->sum_den);
        m.eval_lambda = eval_lambda;
        m.eval_gamma = eval_gamma;
        m.delta_hpwl = dh;
        m.lambda_mu = mu;
        m.evaluations = st->evals;
        m.max_displacement = 0.f;  // not set by the reference's GP either
        m.elapsed_ms = static_cast<double>(global_ns() - st->t0_ns) * 1e-6;
    }
    st->rows = iter + 1;
    const bool filler_only = st->stage == SPG_STAGE_FILLER_ONLY;
    // stop test: deliver the evaluated point u (eplace.cpp:412-419)
    if (!filler_only && st->tau < st->target_tau) {
        st->converged = 1;
        st->deliver = 1;
        st->done = 1;
        return;
    }
    if (!filler_only && p.stagnation_window > 0) {
        const float g = p.min_gain;
        if (st->tau < fmul(st->ref_tau, fsub(1.f, g))) {
            st->ref_tau = st->tau;
            st->since_improve = 0;
        } else {
            st->since_improve += 1;
        }
        st->best_tau = fmin_(st->best_tau, st->tau);
        // the stagnation_mid diagnostic point (eplace.cpp:428-433)
        if (st->diag_mid && !st->diag_mid_hit && st->since_improve >= max(1, p.stagnation_window / 2))
            st->diag_mid_hit = 1;
        const float tol = fmul(st->best_tau, fadd(1.f, g));
        while (st->snap_count > 0 && st->snap_tau[st->snap_head] > tol) {
            st->snap_head = (st->snap_head + 1) % SNAP_MAX;
            st->snap_count -= 1;
        }
        const int last = (st->snap_head + st->snap_count - 1 + SNAP_MAX) % SNAP_MAX;
        if (st->snap_count == 0 || fmul(st->tau, fadd(1.f, fmul(0.5f, g))) <= st->snap_tau[last]) {
            if (st->snap_count == SNAP_MAX) {
                raise_error(st, SPG_E_CAPACITY);
                st->done = 1;
                return;
            }
            const int slot = (st->snap_head + st->snap_count) % SNAP_MAX;
            st->snap_tau[slot] = st->tau;
            st->snap_hpwl[slot] = st->hpwl;
            st->snap_iter[slot] = iter;
            st->snap_count += 1;
            st->snap_copy_to = slot;  // copied from u by the next update (or by deliver)
        }
        if (st->since_improve >= p.stagnation_window) {
            int pick = st->snap_head;
            for (int j = 1; j < st->snap_count; ++j) {
                const int s = (st->snap_head + j) % SNAP_MAX;
                if (st->snap_hpwl[s] < st->snap_hpwl[pick]) pick = s;
            }
            st->stagnated = 1;
            st->rollback_iter = st->snap_iter[pick];
            st->deliver = 2;
            st->deliver_slot = pick;
            st->done = 1;
            return;
        }
    }
    // the loop runs max_iter steps and delivers v after the last update (eplace.cpp:356,484)
    if (iter + 1 >= st->max_iter) st->last = 1;
}

// ------------------------------------------------------------------ vector kernels

__global__ void scatter_kernel(DevPtrs p, int role) {
    pdl_wait();
    pdl_trigger();
    const float* u = role_ptr(p, role);
    const int n = p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float x = u[k], y = u[n + k];
        // objAndGrad rejects non-finite coordinates (eplace.cpp:140-142)
        if (!isfinite(x) || !isfinite(y)) raise_error(p.st, SPG_E_NON_FINITE);
        const int i = p.opt_idx[k];
        p.x[i] = x;
        p.y[i] = y;
    }
}

// force = sum over the footprint of q * xi, bx outer, by inner, as gatherForce sums it
// (bin_grid.cpp:287-318), for a node at (x, y) with smoothed half extents hw, hh and charge
// weight w. Footprints of at most 2x2 bins (every cell no wider than one bin) issue their
// eight field loads before the sums, which keep the reference's order.
__device__ __forceinline__ void gather_at(const DevPtrs& p, float x, float y, float hw, float hh,
                                          float w, float& fx, float& fy) {
    const GridGeom& g = p.geom;
    const Footprint f = footprint(g, x, y, hw, hh);
    fx = 0.f;
    fy = 0.f;
    if (f.bx1 - f.bx0 <= 1 && f.by1 - f.by0 <= 1) {
        float q[4], ex[4], ey[4];
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int bx = f.bx0 + a, by = f.by0 + b;
                const bool in = bx <= f.bx1 && by <= f.by1;
                const size_t o = static_cast<size_t>(in ? bx : f.bx0) * g.dim + (in ? by : f.by0);
                q[2 * a + b] = in ? bin_contribution(g, bx, by, f, w) : 0.f;
                ex[2 * a + b] = __ldg(p.ex + o);
                ey[2 * a + b] = __ldg(p.ey + o);
            }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (q[j] <= 0.f) continue;
            fx = fadd(fx, fmul(q[j], ex[j]));
            fy = fadd(fy, fmul(q[j], ey[j]));
        }
        return;
    }
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

// Physical pool slot of a logical role while a step's role rotation is pending: uPrev <- u
// <- u' ; vPrev <- v <- v' ; gPrevTmp <- g <- (old gPrevTmp buffer) (nesterov.cpp:110-119).
__device__ __forceinline__ int role_slot(const DevState* st, int role, int pending) {
    const int* r = st->role;
    if (pending != 2) return r[role];
    switch (role) {
        case R_U: return r[R_UNEW];
        case R_UPREV: return r[R_U];
        case R_UNEW: return r[R_UPREV];
        case R_V: return r[R_VNEW];
        case R_VPREV: return r[R_V];
        case R_VNEW: return r[R_VPREV];
        case R_G: return r[R_GPREVTMP];
        case R_GPREVTMP: return r[R_G];
        default: return r[role];
    }
}
__device__ __forceinline__ float* role_ptr_pending(const DevPtrs& p, int role, int pending) {
    return p.pool + static_cast<size_t>(role_slot(p.st, role, pending)) * p.vec_stride;
}

// The end of the last step kernel (nesterov.cpp:110-119 and the loop counter): the snapshot
// copy it made is done; when it applied a step, the roles rotate, momentumPrev takes the
// step's momentum, the iteration advances, and max_iter marks the stage done.
__device__ void apply_pending_step(DevState* st) {
    const int pending = st->step_pending;
    if (pending == 0) return;
    st->step_pending = 0;
    st->snap_copy_to = -1;
    if (pending != 2) return;
    int* r = st->role;
    const int ru = r[R_U], rup = r[R_UPREV], run = r[R_UNEW];
    r[R_UPREV] = ru;
    r[R_U] = run;
    r[R_UNEW] = rup;
    const int rv = r[R_V], rvp = r[R_VPREV], rvn = r[R_VNEW];
    r[R_V] = rvn;
    r[R_VPREV] = rv;
    r[R_VNEW] = rvp;
    const int rg = r[R_G], rgp = r[R_GPREVTMP];
    r[R_GPREVTMP] = rg;
    r[R_G] = rgp;
    st->momentum_prev = st->momentum;
    st->iter += 1;
    st->tries = 1;
    if (st->last) st->done = 1;
}

// The finalized evaluation (eplace.cpp:149,154-155,190-197) into the state: tau from the
// overflow sum, HPWL, WA value and the two gradient-norm sums; s = {overflow, WA, HPWL,
// sum|dWL|, sum|q xi|}.
__device__ void finish_evaluation(const DevPtrs& p, DevState* st, const double* s, int count_eval) {
    st->tk_assemble = 0;
    st->tau = p.movable_area_scaled > 0.0 ? static_cast<float>(s[0] / p.movable_area_scaled) : 0.f;
    st->hpwl = s[2];
    st->wl_obj = s[1];
    st->sum_wl = s[3];
    st->sum_den = s[4];
    if (!(isfinite(s[2]) && isfinite(st->tau) && isfinite(s[1]) && isfinite(s[3]) && isfinite(s[4])))
        raise_error(st, SPG_E_NON_FINITE);
    if (count_eval && !st->done) st->evals += 1;
}

// The decisions after a counted evaluation, on the state `st` (a shared-memory copy): the
// redo test and, when no re-evaluation is due, the step decisions and then, for the EPlace
// loop (EPLACE), the iteration decisions of eplace.cpp; a plain optimizer run (the quadratic
// test objective) only marks its last step.
template <bool EPLACE = true>
__device__ void decide(const DevPtrs& p, DevState* st, double dx2, double dg2, double sy2, double gn2) {
    st->tk_reduce = 0;
    st->dx = sqrt(dx2);
    st->dg = sqrt(dg2);
    st->sy = sy2;
    st->gn = gn2;
    st->redo = 0;
    if (!st->done && !st->error) {
        if (p.backtrack && st->iter > 0 && st->tries < p.max_backtrack) {
            const double ddx = st->dx, ddg = st->dg;
            if (ddx > 0.0 && ddg > 0.0 && isfinite(ddg)) {
                const double lip = ddx / ddg;
                if (!(lip > 0.95 * static_cast<double>(st->alpha))) {
                    st->alpha = static_cast<float>(lip);
                    st->redo = 1;
                    st->tries += 1;
                    st->redos += 1;
                }
            }
        }
        if (!st->redo) {
            decide_step(p, st);
            if (EPLACE) decide_iteration(p, st);
            else if (st->iter + 1 >= st->max_iter) st->last = 1;
        }
    }
}

// WA pass 2 of the opt cells (k < filler_k0): wlg[k], wlg[n + k] = the sums of cell k's pin
// terms in node->pin order (wa_wirelength.cpp:137-179), the fadd sequence the assembly would
// run itself. It runs on the WA stream after the nets pass, beside the density -> Poisson
// chain, so the assembly on that chain reads two values per cell instead of walking its pins.
__global__ void __launch_bounds__(RED_THREADS) wl_cells_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const int n = p.n_opt;
    const int k0 = p.filler_k0 < n ? p.filler_k0 : n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < k0; k += gridDim.x * blockDim.x) {
        const int4 meta = p.opt_meta[k];
        float gx = 0.f, gy = 0.f;
        for (int t = meta.x; t < meta.y; ++t) {
            gx = fadd(gx, p.gpx[t]);
            gy = fadd(gy, p.gpy[t]);
        }
        p.wlg[k] = gx;
        p.wlg[n + k] = gy;
    }
}

// One node of the assembly (see assemble_kernel). FILL: a filler, whose attributes are the
// shared constants (no pins, so no WA term).
// precondition 1 / max(1, deg + lambda * area) (eplace.cpp:166-189) of one node.
__device__ __forceinline__ float precondition(int deg, float lambda, double area) {
    const double den = __dadd_rn(static_cast<double>(deg), __dmul_rn(static_cast<double>(lambda), area));
    return static_cast<float>(__ddiv_rn(1.0, fmax(1.0, den)));
}

// filler_pre: the fillers' common preconditioner (their degree and area are the shared
// constants), formed once per thread.
template <bool FUSE, bool FILL>
__device__ __forceinline__ void assemble_node(const DevPtrs& p, int k, float lambda, float filler_pre,
                                              const float* __restrict__ pos,
                                              float* __restrict__ grad, const float* __restrict__ up,
                                              const float* __restrict__ gp, double& acc_wl, double& acc_den,
                                              double& dx, double& dg, double& sy, double& gn) {
    const int n = p.n_opt;
    const int4 meta = FILL ? p.filler_meta : p.opt_meta[k];
    const float4 geo = FILL ? p.filler_geom : p.opt_geom[k];
    const float x = pos[k], y = pos[n + k];
    const double area = FILL ? p.filler_area : p.opt_area[k];
    float upx = 0.f, upy = 0.f, gpx = 0.f, gpy = 0.f;
    if (FUSE) {
        upx = up[k];
        upy = up[n + k];
        gpx = gp[k];
        gpy = gp[n + k];
    }
    float gx = 0.f, gy = 0.f;
    if (!FILL) {
        if (p.wlg) {
            gx = p.wlg[k];
            gy = p.wlg[n + k];
        } else {
            for (int t = meta.x; t < meta.y; ++t) {
                gx = fadd(gx, p.gpx[t]);
                gy = fadd(gy, p.gpy[t]);
            }
        }
    }
    float fx, fy;
    if (meta.w & K_LARGE) {
        fx = p.force[k];
        fy = p.force[n + k];
    } else {
        gather_at(p, x, y, geo.x, geo.y, geo.z, fx, fy);
    }
    const float precond = FILL ? filler_pre : precondition(meta.z, lambda, area);
    const float ox = fmul(precond, fsub(gx, fmul(lambda, fx)));
    const float oy = fmul(precond, fsub(gy, fmul(lambda, fy)));
    grad[k] = ox;
    grad[n + k] = oy;
    if (!isfinite(ox) || !isfinite(oy)) raise_error(p.st, SPG_E_NON_FINITE);
    if (!FILL && (meta.w & OPT_HAS_WL)) acc_wl += static_cast<double>(fadd(fabsf(gx), fabsf(gy)));
    acc_den += static_cast<double>(fadd(fabsf(fx), fabsf(fy)));
    if (FUSE) {
        // l2Diff, dotDiff, l2Norm terms (nesterov.cpp:25-45), x then y
        const double sxd = static_cast<double>(x) - static_cast<double>(upx);
        const double syd = static_cast<double>(y) - static_cast<double>(upy);
        const double yx = static_cast<double>(ox) - static_cast<double>(gpx);
        const double yy = static_cast<double>(oy) - static_cast<double>(gpy);
        dx += __dmul_rn(sxd, sxd) + __dmul_rn(syd, syd);
        dg += __dmul_rn(yx, yx) + __dmul_rn(yy, yy);
        sy += __dmul_rn(sxd, yx) + __dmul_rn(syd, yy);
        gn += __dmul_rn(static_cast<double>(ox), static_cast<double>(ox)) +
              __dmul_rn(static_cast<double>(oy), static_cast<double>(oy));
    }
}

// grad_k = precond * (dWL - lambda * q*xi), precond = 1 / max(1, deg + lambda*area)
// (eplace.cpp:166-189), with the field gather of cells fused in (large nodes' force comes from
// gather_opt_large) and the cells' WA gradient read from wl_cells_kernel's sums (WA pass 2:
// per-node sum of per-pin contributions in node->pin order, wa_wirelength.cpp:137-179; with
// SPG_WL_AHEAD=0 the assembly forms those sums itself). The last block finalizes the evaluation
// (eplace.cpp:149,154-155,190-197).
//
// FUSE (the iteration loop's evaluations, at u = R_U into g = R_G): the same pass also forms
// the four norms |u-uPrev|^2, |g-gPrevTmp|^2, (u-uPrev).(g-gPrevTmp), |g|^2 (l2Diff, dotDiff,
// l2Norm: nesterov.cpp:25-45) from the values it holds, and its last block runs the redo test
// (nesterov.cpp:148-157) and the decisions after the evaluation's finalize.
template <bool FUSE>
// loop_cond (graph mode, FUSE): the enclosing WHILE node's handle; the last block sets it
// from the decisions (continue while the stage is neither done nor failed). 0: host loop.
__global__ void __launch_bounds__(RED_THREADS) assemble_kernel(DevPtrs p, int pos_role, int grad_role,
                                                              int count_eval, cudaGraphConditionalHandle loop_cond) {
    pdl_wait();
    pdl_trigger();
    // the evaluated positions, by opt index: the role the update (or scatter) wrote the
    // node coordinates from, so pos[k] == x[opt_idx[k]] bit for bit
    // (through a step's pending role rotation, which the last block then applies)
    const int pending = p.st->step_pending;
    const float* __restrict__ pos = role_ptr_pending(p, pos_role, pending);
    float* __restrict__ grad = role_ptr_pending(p, grad_role, pending);
    const float* __restrict__ up = FUSE ? role_ptr_pending(p, R_UPREV, pending) : nullptr;
    const float* __restrict__ gp = FUSE ? role_ptr_pending(p, R_GPREVTMP, pending) : nullptr;
    const float lambda = p.st->lambda;
    const int n = p.n_opt;
    double acc_wl = 0.0, acc_den = 0.0;
    double dx = 0.0, dg = 0.0, sy = 0.0, gn = 0.0;
    // cells, then the fillers (their attributes the shared constants); every thread keeps the
    // nodes k = t0 (mod stride) of a single grid-stride pass, in increasing k
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const int k0 = p.filler_k0 < n ? p.filler_k0 : n;
    int k = t0;
    for (; k < k0; k += stride)
        assemble_node<FUSE, false>(p, k, lambda, 0.f, pos, grad, up, gp, acc_wl, acc_den, dx, dg, sy, gn);
    if (k < n) {
        const float filler_pre = precondition(p.filler_meta.z, lambda, p.filler_area);
        for (; k < n; k += stride)
            assemble_node<FUSE, true>(p, k, lambda, filler_pre, pos, grad, up, gp, acc_wl, acc_den, dx, dg, sy, gn);
    }
    if (FUSE) {
        double v6[6] = {acc_wl, acc_den, dx, dg, sy, gn};
        block_sums(v6);
        put_partial(p, SLOT_SUM_WL, v6[0]);
        put_partial(p, SLOT_SUM_DEN, v6[1]);
        put_partial(p, SLOT_DX, v6[2]);
        put_partial(p, SLOT_DG, v6[3]);
        put_partial(p, SLOT_SY, v6[4]);
        put_partial(p, SLOT_GN, v6[5]);
    } else {
        double v2[2] = {acc_wl, acc_den};
        block_sums(v2);
        put_partial(p, SLOT_SUM_WL, v2[0]);
        put_partial(p, SLOT_SUM_DEN, v2[1]);
    }
    if (!last_block(&p.st->tk_assemble)) return;
    if (!FUSE) {
        constexpr int kSlots[5] = {SLOT_OVERFLOW, SLOT_WL, SLOT_HPWL, SLOT_SUM_WL, SLOT_SUM_DEN};
        double sums[5];
        finalize_n(p, kSlots, sums);
        if (threadIdx.x == 0) {
            apply_pending_step(p.st);
            finish_evaluation(p, p.st, sums, count_eval);
        }
        return;
    }
    constexpr int kSlots[9] = {SLOT_OVERFLOW, SLOT_WL, SLOT_HPWL, SLOT_SUM_WL, SLOT_SUM_DEN,
                               SLOT_DX, SLOT_DG, SLOT_SY, SLOT_GN};
    double sums[9];
    finalize_n(p, kSlots, sums);
    __shared__ DevState sst;
    state_copy_in(&sst, p.st);
    if (threadIdx.x == 0) {
        apply_pending_step(&sst);
        finish_evaluation(p, &sst, sums, count_eval);
        decide(p, &sst, sums[5], sums[6], sums[7], sums[8]);
        // continue while the stage is neither done nor failed nor at a pause (filler reorder,
        // iteration callback, stagnation-midpoint callback)
        if (loop_cond)
            cudaGraphSetConditional(loop_cond, (sst.done || sst.error || sst.iter >= sst.pause_iter ||
                                                sst.rows > sst.pause_row || (sst.diag_mid && sst.diag_mid_hit))
                                                   ? 0u
                                                   : 1u);
    }
    state_copy_out(p.st, &sst);
}

// One coordinate of the Nesterov point (nesterov.cpp:97-107, and the redoIfOvershot body
// :158-163 with uPrev, gPrevTmp, vPrev and momentumPrev in place of u, g, v and momentum):
//   v' = u - alpha g ; u' = v' + m (v' - v) ; both clamped into [lo, hi] afterwards.
__device__ __forceinline__ void nesterov_point(float u, float v, float g, float alpha, float m, float lo,
                                               float hi, float& vn, float& un) {
    const float vk = fsub(u, fmul(alpha, g));
    const float uk = fadd(vk, fmul(m, fsub(vk, v)));
    vn = clamp_box(vk, lo, hi);
    un = clamp_box(uk, lo, hi);
}

// The loop's position step with the density scatter of the new positions fused in. One
// launch per loop pass, one node per thread; the pass applies whichever step the last
// decisions asked for:
//
//   a re-evaluation (st->redo; redoIfOvershot body, nesterov.cpp:158-163):
//     v = uPrev - alpha gPrevTmp ; u = v + momentumPrev (v - vPrev) ; clamp v, u.
//   otherwise the next step (NesterovOptimizer::step, nesterov.cpp:97-119):
//     v' = u - alpha g ; u' = v' + momentum (v' - v) ; clamp both (nesterov.cpp:97-107); when
//     the iteration decided a stagnation snapshot, the evaluated u is copied into its slot.
//     The role rotation uPrev <- u <- u' ; vPrev <- v <- v' ; gPrevTmp <- g and the loop
//     counter follow in the next assembly's last block (apply_pending_step).
//
// PLACE (the GP loop): the new u is written into the node positions (for the WA pass) and
// its fixed-point charge is added to the density maps right here (BinGrid::accumulate,
// bin_grid.cpp:191-251), so the evaluation needs no separate pass over the cells; nodes whose
// footprint may exceed 16 bins are left to the block-per-node kernel of the rest list. When
// no step applies (the stage is done) the current u is rasterized unchanged. Without PLACE
// (a plain optimizer run over a test objective) only the optimizer vectors are written, with
// the per-coordinate clamp bounds opt_lo / opt_hi.
// 6 blocks of 256 per SM: the kernel is latency-bound, so occupancy is what hides its loads
// and atomics. The grid covers the opt set (node_blocks), one node per thread.
// One launch covers the opt positions [k_begin, k_end): the whole set, or the cells and the
// fillers as two launches (the WA pass, which reads only cell positions, then starts after the
// cells' launch).
template <bool PLACE>
__global__ void __launch_bounds__(RED_THREADS, 6) step_kernel(DevPtrs p, int k_begin, int k_end) {
    pdl_wait();
    pdl_trigger();
    DevState* st = p.st;
    const bool redo = st->redo != 0;
    const int apply = redo ? 1 : !st->done;
    const int slot = (redo || !PLACE) ? -1 : st->snap_copy_to;
    const float* u = role_ptr(p, redo ? R_UPREV : R_U);
    const float* v = role_ptr(p, redo ? R_VPREV : R_V);
    const float* g = role_ptr(p, redo ? R_GPREVTMP : R_G);
    float* vn = role_ptr(p, redo ? R_V : R_VNEW);
    float* un = role_ptr(p, redo ? R_U : R_UNEW);
    const float* cur = role_ptr(p, R_U);
    float* snap = slot >= 0 ? snap_ptr(p, slot) : nullptr;
    const float alpha = st->alpha, m = redo ? st->momentum_prev : st->momentum;
    const int n = p.n_opt;
    const int k = k_begin + blockIdx.x * blockDim.x + threadIdx.x;
    const bool have = k < k_end;
    const bool fill = PLACE && k >= p.filler_k0;  // a filler: attributes are the shared constants
    int4 meta{};
    float4 geo{};
    float nu[2] = {0.f, 0.f};
    if (have) {
        if (PLACE) {
            meta = fill ? p.filler_meta : p.opt_meta[k];
            geo = fill ? p.filler_geom : p.opt_geom[k];
        }
        if (apply) {
            // every load first (the stores below go to other vectors, so both coordinates'
            // loads are in flight together), then the two Nesterov points, then the stores
            float uq[2], vq[2], gq[2], lo[2], hi[2], vk[2];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int q = c * n + k;
                uq[c] = u[q];
                vq[c] = v[q];
                gq[c] = g[q];
                lo[c] = fill ? (c ? p.filler_lo_y : p.filler_lo_x) : p.opt_lo[q];
                hi[c] = fill ? (c ? p.filler_hi_y : p.filler_hi_x) : p.opt_hi[q];
            }
            // the node arrays: read inside the loop only for cells (WA) and large nodes (their
            // gather); the fillers' entries are rewritten from R_POS when the stage ends
            const int node = (PLACE && (!fill || (meta.w & K_LARGE))) ? p.opt_idx[k] : -1;
#pragma unroll
            for (int c = 0; c < 2; ++c) nesterov_point(uq[c], vq[c], gq[c], alpha, m, lo[c], hi[c], vk[c], nu[c]);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int q = c * n + k;
                if (snap) snap[q] = uq[c];
                vn[q] = vk[c];
                un[q] = nu[c];
            }
            if (!isfinite(nu[0]) || !isfinite(nu[1])) raise_error(st, SPG_E_NON_FINITE);
            if (node >= 0) {
                p.x[node] = nu[0];
                p.y[node] = nu[1];
            }
        } else {
            nu[0] = cur[k];
            nu[1] = cur[n + k];
            if (snap) {
                snap[k] = nu[0];
                snap[n + k] = nu[1];
            }
        }
    }
    if (PLACE && have && !(meta.w & K_LARGE))
        rasterize(p, nu[0], nu[1], geo.x, geo.y, geo.z, (meta.w & K_FILLER) != 0);
    // the rest of the step (apply_pending_step) runs in the next assembly's last block; every
    // block read the state above before this store can matter to anyone
    if (!redo && blockIdx.x == 0 && threadIdx.x == 0) st->step_pending = apply ? 2 : 1;
}

// ------------------------------------------------------------------ quadratic test objective
// f(x) = 0.5 * sum_i c_i (x_i - t_i)^2 over the 2*nOpt optimizer coordinates, with gradient
// (float)(c_i (x_i - t_i)) and the objective summed in FP64: the objective of the reference's
// optimizer tests (test/test_nesterov.cpp:14-27). It drives the loop's own step kernel,
// redo test and step decisions without a placement, so the optimizer can be checked against
// the reference's NesterovOptimizer on its known answers.
//
// FUSE: an evaluation of the iteration (at u = R_U into g = R_G, counted) with the step's four
// norms, whose last block applies the pending step, records the objective and decides;
// otherwise an uncounted evaluation of pos_role into grad_role (estimateInitialStep).
template <bool FUSE>
__global__ void __launch_bounds__(RED_THREADS) quad_eval_kernel(DevPtrs p, const float* __restrict__ coef,
                                                                const float* __restrict__ target, int pos_role,
                                                                int grad_role) {
    pdl_wait();
    pdl_trigger();
    const int pending = p.st->step_pending;
    const float* __restrict__ pos = role_ptr_pending(p, FUSE ? R_U : pos_role, pending);
    float* __restrict__ grad = role_ptr_pending(p, FUSE ? R_G : grad_role, pending);
    const float* __restrict__ up = FUSE ? role_ptr_pending(p, R_UPREV, pending) : nullptr;
    const float* __restrict__ gp = FUSE ? role_ptr_pending(p, R_GPREVTMP, pending) : nullptr;
    const int n = 2 * p.n_opt;
    double obj = 0.0, dx = 0.0, dg = 0.0, sy = 0.0, gn = 0.0;
    bool bad = false;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float x = pos[k];
        const double c = static_cast<double>(coef[k]);
        const double d = static_cast<double>(x) - static_cast<double>(target[k]);
        obj += __dmul_rn(__dmul_rn(0.5 * c, d), d);
        const float gk = static_cast<float>(__dmul_rn(c, d));
        grad[k] = gk;
        bad |= !isfinite(x) || !isfinite(gk);
        if (FUSE) {
            const double sd = static_cast<double>(x) - static_cast<double>(up[k]);
            const double yd = static_cast<double>(gk) - static_cast<double>(gp[k]);
            dx += __dmul_rn(sd, sd);
            dg += __dmul_rn(yd, yd);
            sy += __dmul_rn(sd, yd);
            gn += __dmul_rn(static_cast<double>(gk), static_cast<double>(gk));
        }
    }
    if (bad) raise_error(p.st, SPG_E_NON_FINITE);
    if (!FUSE) return;
    double v5[5] = {obj, dx, dg, sy, gn};
    block_sums(v5);
    put_partial(p, SLOT_WL, v5[0]);
    put_partial(p, SLOT_DX, v5[1]);
    put_partial(p, SLOT_DG, v5[2]);
    put_partial(p, SLOT_SY, v5[3]);
    put_partial(p, SLOT_GN, v5[4]);
    if (!last_block(&p.st->tk_assemble)) return;
    constexpr int kSlots[5] = {SLOT_WL, SLOT_DX, SLOT_DG, SLOT_SY, SLOT_GN};
    double sums[5];
    finalize_n(p, kSlots, sums);
    __shared__ DevState sst;
    state_copy_in(&sst, p.st);
    if (threadIdx.x == 0) {
        DevState* q = &sst;
        apply_pending_step(q);
        q->tk_assemble = 0;
        if (!isfinite(sums[0])) raise_error(q, SPG_E_NON_FINITE);
        // the objective of the last counted evaluation (NesterovOptimizer::objective)
        if (!q->done) {
            q->evals += 1;
            q->wl_obj = sums[0];
        }
        decide<false>(p, q, sums[1], sums[2], sums[3], sums[4]);
    }
    state_copy_out(p.st, &sst);
}

__global__ void copy_role_kernel(DevPtrs p, int dst, int src) {
    pdl_wait();
    pdl_trigger();
    float* d = role_ptr(p, dst);
    const float* s = role_ptr(p, src);
    const int n = 2 * p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) d[k] = s[k];
}

__global__ void clamp_role_kernel(DevPtrs p, int role) {
    pdl_wait();
    pdl_trigger();
    float* d = role_ptr(p, role);
    const int n = 2 * p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        d[k] = clamp_box(d[k], p.opt_lo[k], p.opt_hi[k]);
}

// Delivered solution into R_POS (eplace.cpp:412-485): v after the last update, the last
// evaluated point u (converged), or the picked snapshot (stagnated; when the pick is the
// snapshot decided in the final iteration, its copy is still pending and u is it).
__global__ void deliver_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const DevState* st = p.st;
    const float* s = role_ptr(p, R_V);
    if (st->deliver == 1) s = role_ptr(p, R_U);
    if (st->deliver == 2)
        s = (st->deliver_slot == st->snap_copy_to) ? role_ptr(p, R_U) : snap_ptr(p, st->deliver_slot);
    float* d = role_ptr(p, R_POS);
    const int n = 2 * p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        d[k] = clamp_box(s[k], p.opt_lo[k], p.opt_hi[k]);
}

// |u|^2 -> SLOT_PN and |gA|^2 -> SLOT_GN for estimateInitialStep (nesterov.cpp:196-198)
__global__ void __launch_bounds__(RED_THREADS) init_norms_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const float* u = role_ptr(p, R_U);
    const float* ga = role_ptr(p, R_GA);
    const int n = 2 * p.n_opt;
    double pn = 0.0, gn = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double a = u[k], b = ga[k];
        pn += __dmul_rn(a, a);
        gn += __dmul_rn(b, b);
    }
    pn = block_sum(pn);
    gn = block_sum(gn);
    put_partial(p, SLOT_PN, pn);
    put_partial(p, SLOT_GN, gn);
}

// probe = clamp(u - (float)scale * gA) (nesterov.cpp:200-205); scale is in st->pn.
__global__ void init_perturb_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const float* u = role_ptr(p, R_U);
    const float* ga = role_ptr(p, R_GA);
    float* pr = role_ptr(p, R_PROBE);
    const float sc = static_cast<float>(p.st->pn);
    const int n = 2 * p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        pr[k] = clamp_box(fsub(u[k], fmul(sc, ga[k])), p.opt_lo[k], p.opt_hi[k]);
}

// dx^2 = |probe - u|^2 -> SLOT_DX, dg^2 = |gB - gA|^2 -> SLOT_DG (nesterov.cpp:207-208)
__global__ void __launch_bounds__(RED_THREADS) init_diff_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const float* u = role_ptr(p, R_U);
    const float* pr = role_ptr(p, R_PROBE);
    const float* ga = role_ptr(p, R_GA);
    const float* gb = role_ptr(p, R_GB);
    const int n = 2 * p.n_opt;
    double dx = 0.0, dg = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double a = static_cast<double>(pr[k]) - static_cast<double>(u[k]);
        const double b = static_cast<double>(gb[k]) - static_cast<double>(ga[k]);
        dx += __dmul_rn(a, a);
        dg += __dmul_rn(b, b);
    }
    dx = block_sum(dx);
    dg = block_sum(dg);
    put_partial(p, SLOT_DX, dx);
    put_partial(p, SLOT_DG, dg);
}

// ------------------------------------------------------------------ control kernels

// lambda_0 = sum|dWL| / sum|q xi|, gamma = computeGamma(tau) (eplace.cpp:254-258)
__global__ void ctl_lambda_init_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    DevState* st = p.st;
    st->gamma = compute_gamma(st->tau, p.step_x_gamma);
    float lam = st->sum_den > 0.0 ? static_cast<float>(st->sum_wl / st->sum_den) : 1.f;
    if (!isfinite(lam) || lam <= 0.f) lam = 1.f;
    st->lambda = lam;
}

// estimateInitialStep, first half: perturbation scale into st->pn, or alpha0 = 1.
__global__ void ctl_init_scale_kernel(DevPtrs p, float init_perturb) {
    pdl_wait();
    pdl_trigger();
    const double pn2 = finalize(p, SLOT_PN);
    const double gn2 = finalize(p, SLOT_GN);
    if (threadIdx.x != 0) return;
    DevState* st = p.st;
    const double pos_norm = sqrt(pn2), g_norm = sqrt(gn2);
    st->redo = 0;
    if (!(g_norm > 0.0) || !isfinite(g_norm)) {
        st->alpha0 = 1.f;
        st->redo = 1;  // marks "alpha0 decided"
        st->pn = 0.0;
        return;
    }
    st->pn = static_cast<double>(init_perturb) * (pos_norm > 0.0 ? pos_norm : 1.0) / g_norm;
}

// estimateInitialStep, second half: alpha0 = |probe-u| / |gB-gA| (nesterov.cpp:207-217).
__global__ void ctl_init_finish_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    const double dx2 = finalize(p, SLOT_DX);
    const double dg2 = finalize(p, SLOT_DG);
    if (threadIdx.x != 0) return;
    DevState* st = p.st;
    if (st->redo) {  // decided in the first half
        st->redo = 0;
        return;
    }
    const double dx = sqrt(dx2), dg = sqrt(dg2);
    if (!(dx > 0.0) || !(dg > 0.0) || !isfinite(dg)) {
        st->alpha0 = 1.f;
        return;
    }
    const double L = dg / dx;
    const double step = 1.0 / L;
    st->alpha0 = (isfinite(step) && step > 0.0) ? static_cast<float>(step) : 1.f;
}

__global__ void ctl_stage_start_kernel(DevPtrs p) {
    pdl_wait();
    pdl_trigger();
    p.st->t0_ns = global_ns();
}

__global__ void check_geometry_kernel(DevPtrs p, float lx, float ly, float hx, float hy,
                                      const float* w, const float* h) {
    pdl_wait();
    pdl_trigger();
    const int n = p.n_opt;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = p.opt_idx[k];
        const float x = p.x[i], y = p.y[i];
        if (!isfinite(x) || !isfinite(y)) {
            raise_error(p.st, SPG_E_NON_FINITE);
            continue;
        }
        const float hw = fmul(0.5f, w[i]), hh = fmul(0.5f, h[i]);
        // checkGeometry bounds (src/util/invariant.h:24-30)
        if (!(fsub(x, hw) >= fsub(lx, .01f) && fsub(y, hh) >= fsub(ly, .01f) &&
              fadd(x, hw) <= fadd(hx, .01f) && fadd(y, hh) <= fadd(hy, .01f)))
            raise_error(p.st, SPG_E_OUT_OF_CORE);
    }
}

__global__ void finalize_slots_kernel(DevPtrs p, int first, int count, double* out) {
    pdl_wait();
    pdl_trigger();
    for (int s = 0; s < count; ++s) {
        const double v = finalize(p, first + s);
        if (threadIdx.x == 0) out[s] = v;
    }
}

// One full wave of RED_THREADS-thread blocks (reducing kernels: the partials' owners).
template <typename K>
inline int wave(K kernel) {
    return wave_grid(reinterpret_cast<const void*>(kernel), RED_THREADS, RED_CAP);
}

// Element-wise kernels over 2*nOpt values: one thread per value up to one full wave.
template <typename K>
inline int vec_blocks(const DevPtrs& p, K kernel) {
    const int64_t b = ceil_div(2 * static_cast<int64_t>(p.n_opt), RED_THREADS);
    const int w = wave(kernel);
    return b < 1 ? 1 : (b > w ? w : static_cast<int>(b));
}

}  // namespace

#define LAUNCH(kernel, grid, block, ...) launch_pdl(kernel, dim3(grid), dim3(block), 0, s, __VA_ARGS__)

void launch_scatter(const DevPtrs& p, int role, cudaStream_t s) {
    LAUNCH(scatter_kernel, vec_blocks(p, scatter_kernel), RED_THREADS, p, role);
}
void launch_wl_cells(const DevPtrs& p, cudaStream_t s) {
    const int k0 = p.filler_k0 < p.n_opt ? p.filler_k0 : p.n_opt;
    if (!p.wlg || k0 <= 0) return;
    // no programmatic early start: blocks resident ahead of the WA pass's end would only wait
    // there, holding SM room the chain's kernels need; the WA stream's low priority
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ceil_div(k0, RED_THREADS));
    cfg.blockDim = dim3(RED_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = launch_priority(false);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SPG_CUDA(cudaLaunchKernelEx(&cfg, wl_cells_kernel, p));
    count_launch();
}
void launch_assemble(const DevPtrs& p, int pos_role, int grad_role, int count_eval, cudaStream_t s) {
    LAUNCH(assemble_kernel<false>, work_grid(reinterpret_cast<const void*>(assemble_kernel<false>), p.n_opt, RED_THREADS),
           RED_THREADS, p, pos_role, grad_role,
           count_eval, cudaGraphConditionalHandle{0});
}
void launch_assemble_reduce(const DevPtrs& p, cudaStream_t s, cudaGraphConditionalHandle loop_cond) {
    LAUNCH(assemble_kernel<true>, work_grid(reinterpret_cast<const void*>(assemble_kernel<true>), p.n_opt, RED_THREADS),
           RED_THREADS, p, static_cast<int>(R_U),
           static_cast<int>(R_G), 1, loop_cond);
}
// One opt node per thread: the step ends in four fixed-point atomics per node, and a grid
// of many short blocks keeps enough of them in flight (the step writes no partial sums, so
// its grid need not be one wave).
inline int node_blocks(const DevPtrs& p) {
    const int b = ceil_div(static_cast<int64_t>(p.n_opt), RED_THREADS);
    return b < 1 ? 1 : b;
}
void launch_update(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(step_kernel<true>, node_blocks(p), RED_THREADS, p, 0, p.n_opt);
}
void launch_update_range(const DevPtrs& p, int k_begin, int k_end, cudaStream_t s) {
    const int b = ceil_div(static_cast<int64_t>(k_end - k_begin), RED_THREADS);
    LAUNCH(step_kernel<true>, b < 1 ? 1 : b, RED_THREADS, p, k_begin, k_end);
}
void launch_quad_step(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(step_kernel<false>, node_blocks(p), RED_THREADS, p, 0, p.n_opt);
}
void launch_quad_eval(const DevPtrs& p, const float* coef, const float* target, int pos_role, int grad_role,
                      int fused, cudaStream_t s) {
    const int64_t n = 2 * static_cast<int64_t>(p.n_opt);
    if (fused)
        LAUNCH(quad_eval_kernel<true>, work_grid(reinterpret_cast<const void*>(quad_eval_kernel<true>), n, RED_THREADS),
               RED_THREADS, p, coef, target, pos_role, grad_role);
    else
        LAUNCH(quad_eval_kernel<false>, work_grid(reinterpret_cast<const void*>(quad_eval_kernel<false>), n, RED_THREADS),
               RED_THREADS, p, coef, target, pos_role, grad_role);
}
void launch_ctl_lambda_init(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(ctl_lambda_init_kernel, 1, 1, p);
}
void launch_init_norms(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(init_norms_kernel, work_grid(reinterpret_cast<const void*>(init_norms_kernel), 2 * static_cast<int64_t>(p.n_opt), RED_THREADS),
           RED_THREADS, p);
}
void launch_ctl_init_scale(const DevPtrs& p, float init_perturb, cudaStream_t s) {
    LAUNCH(ctl_init_scale_kernel, 1, RED_THREADS, p, init_perturb);
}
void launch_init_perturb(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(init_perturb_kernel, vec_blocks(p, init_perturb_kernel), RED_THREADS, p);
}
void launch_init_diff(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(init_diff_kernel, work_grid(reinterpret_cast<const void*>(init_diff_kernel), 2 * static_cast<int64_t>(p.n_opt), RED_THREADS),
           RED_THREADS, p);
}
void launch_ctl_init_finish(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(ctl_init_finish_kernel, 1, RED_THREADS, p);
}
void launch_copy_role(const DevPtrs& p, int dst, int src, cudaStream_t s) {
    LAUNCH(copy_role_kernel, vec_blocks(p, copy_role_kernel), RED_THREADS, p, dst, src);
}
void launch_clamp_role(const DevPtrs& p, int role, cudaStream_t s) {
    LAUNCH(clamp_role_kernel, vec_blocks(p, clamp_role_kernel), RED_THREADS, p, role);
}
void launch_deliver(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(deliver_kernel, vec_blocks(p, deliver_kernel), RED_THREADS, p);
}
void launch_stage_clock(const DevPtrs& p, cudaStream_t s) {
    LAUNCH(ctl_stage_start_kernel, 1, 1, p);
}
void launch_check_geometry(const DevPtrs& p, float lx, float ly, float hx, float hy, const float* w,
                           const float* h, cudaStream_t s) {
    LAUNCH(check_geometry_kernel, vec_blocks(p, check_geometry_kernel), RED_THREADS, p, lx, ly, hx, hy, w, h);
}
void launch_finalize_slots(const DevPtrs& p, int first, int count, double* out, cudaStream_t s) {
    LAUNCH(finalize_slots_kernel, 1, RED_THREADS, p, first, count, out);
}

}  // namespace spg
