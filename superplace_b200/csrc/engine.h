// Internal interfaces of the sm_100a GP engine (not part of the C ABI).
//
// Layout in HBM (one context):
//   node SoA      x, y, hw, hh, wgt (f32) and kind (u8) over all nodes; hw/hh/wgt/kind are
//                 rebuilt per stage (local smoothing and charge weight are stage-static)
//   pins          offsets (f32 x2), pin2node, pin2net, and both CSR directions (i32)
//   bin maps      node/filler fixed-point maps (i64, M^2 each), terminal, base, rho, phi,
//                 xi_x, xi_y (f32, M^2 each)
//   optimizer     a pool of 12 vectors of 2*nOpt f32 whose roles (u, v, uPrev, ...) rotate
//                 through a role table in DevState, so every launch has fixed arguments
//   reductions    RED_SLOTS x RED_CAP FP64 partial sums (fixed grid => deterministic)
//   DevState      every scalar of the Nesterov / lambda / gamma / stagnation logic
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace spg {

// Partial sums per slot: a reducing kernel writes one per block (at most RED_CAP blocks)
// and clears the entries past its grid; the finalizing code always sums all RED_CAP in a
// fixed tree. The vector and reducing kernels run one full wave (wave_grid), so no SM
// idles behind a partial second wave.
constexpr int RED_CAP = 1024;
constexpr int RED_THREADS = 256;

// Blocks of `threads` threads that fill every SM once at the kernel's occupancy, at most
// `cap`; cached per kernel and device (engine.cu).
int wave_grid(const void* kernel, int threads, int cap);
// The grid of a grid-stride kernel over `items` work items, `per_block` per block and pass:
// enough blocks for one item per thread, at most one wave (wave_grid). Small problems launch
// only the blocks they fill, so concurrent contexts share the device; the grid is fixed per
// device and problem size, so reductions keep their fixed order.
inline int work_grid(const void* kernel, int64_t items, int per_block, int threads = RED_THREADS) {
    const int64_t need = (items + per_block - 1) / per_block;
    const int w = wave_grid(kernel, threads, RED_CAP);
    return need < 1 ? 1 : (need < w ? static_cast<int>(need) : w);
}

enum RedSlot : int {
    SLOT_OVERFLOW = 0,
    SLOT_WL,
    SLOT_HPWL,
    SLOT_SUM_WL,
    SLOT_SUM_DEN,
    SLOT_DX,
    SLOT_DG,
    SLOT_SY,
    SLOT_GN,
    SLOT_PN,
    SLOT_CHARGE,
    RED_SLOTS
};

// node kind bits (stage-static)
constexpr uint8_t K_DENSITY = 1;  // contributes density (not fixed, not NI)
constexpr uint8_t K_FILLER = 2;
constexpr uint8_t K_LARGE = 4;    // footprint may exceed 16 bins: block-per-node kernels
constexpr int OPT_HAS_WL = 0x100;  // opt_meta flag: a movable node (it owns the WA gradient)

// optimizer vector roles
enum Role : int {
    R_U = 0, R_V, R_UPREV, R_VPREV, R_UNEW, R_VNEW, R_G, R_GPREVTMP, R_PROBE, R_GA, R_GB, R_POS,
    NUM_ROLES
};

constexpr int SNAP_MAX = 6;  // stagnation snapshots kept (at most ~4 are ever live)

// Every scalar of one stage run. Written by the control kernels, read by the vector
// kernels and (once per iteration) by the host.
struct DevState {
    // schedule (src/gp/eplace.cpp:59-68)
    float lambda, gamma, tau;
    float eval_lambda, eval_gamma;
    double hpwl, wl_obj, sum_wl, sum_den;
    // Nesterov (src/numeric/cpu/nesterov.cpp:315-324)
    float a, alpha, alpha0, momentum, momentum_prev, grad_norm;
    int iter;
    int64_t evals;
    double dx, dg, sy, gn, pn;
    int redo;       // redoIfOvershot decision for the current evaluation
    int tries;
    // lambda schedule (eplace.cpp:312-313)
    double prev_hpwl;
    int have_prev;
    double hpwl_ref;
    // stop / stagnation (eplace.cpp:339-353)
    float target_tau;
    float best_tau, ref_tau;
    int since_improve;
    int snap_count, snap_head;
    float snap_tau[SNAP_MAX];
    double snap_hpwl[SNAP_MAX];
    int snap_iter[SNAP_MAX];
    int snap_copy_to;   // slot the snapshot kernel copies lastEval into, or -1
    int deliver;        // 0 = v, 1 = lastEval (converged), 2 = snapshot slot deliver_slot
    int deliver_slot;
    int done, converged, stagnated, rollback_iter;
    int last;           // max_iter reached: apply this update, then stop
    int rows;           // iterations whose loop body ran (metrics rows)
    int error;          // SPG_E_* raised on the device (non-finite values)
    int64_t redos;      // backtracking re-evaluations
    unsigned int tk_update, tk_assemble, tk_reduce;  // last-block tickets
    // bookkeeping of the last step kernel, applied by the next assembly's last block (the step
    // kernel has no last block: a fence per block would wait on its atomics): 0 none,
    // 1 clear the snapshot copy, 2 also rotate the roles and advance the iteration
    int step_pending;
    int step_pending_pad;
    int stage;
    int max_iter;
    int role[NUM_ROLES];
    unsigned long long t0_ns;
    // the loop stops (without finishing the stage) once iter reaches pause_iter, so the host
    // can reorder the fillers between two passes (filler_order.cu), and once the metrics row
    // of iteration pause_row is written (rows > pause_row), so the host can run the iteration
    // callback at that evaluation point; INT_MAX: never
    int pause_iter;
    int pause_row;
    // diag_mid = 1: the loop also stops once, when the stagnation counter first reaches half
    // the window (the reference's stagnation_mid diagnostic point); diag_mid_hit records it
    int diag_mid;
    int diag_mid_hit;
};

// Nets of at most this degree get one thread each in WA pass 1 (SPG_WA_THREAD_DEGREE
// lowers it; 0 gives every net a lane group).
constexpr int kWaThreadNetDegree = 5;

// Degree classes of the WA kernel over the degree-sorted net order. Class i owns the nets at
// sorted positions [net_begin[i], net_end[i]), all of degree deg[i] (the last class, of the
// nets above 32 pins, has mixed degrees: deg -1), whose pins start at entry pin_begin[i] of
// the sorted pin order, with group[i] lanes per net (1: one thread; 2..32: a lane group,
// shift = log2 of it; 0: one warp that loops over the pins) and warps
// [warp_begin[i], warp_begin[i+1]). Passed by value to the WA kernel only.
constexpr int WA_MAX_CLASSES = 40;
struct WaClasses {
    int n;
    int group[WA_MAX_CLASSES];
    int shift[WA_MAX_CLASSES];
    int deg[WA_MAX_CLASSES];
    int net_begin[WA_MAX_CLASSES], net_end[WA_MAX_CLASSES];
    int pin_begin[WA_MAX_CLASSES];
    int warp_begin[WA_MAX_CLASSES + 1];
};

// Everything a kernel needs to address the device data, passed by value.
struct DevPtrs {
    int num_movable, num_nodes, num_fillers, total, num_pins, num_nets;
    float *x, *y;
    float *hw, *hh, *wgt;
    uint8_t* kind;
    const float *pox, *poy;
    const int *pin2node, *pin2net;
    const int *net_start, *net_pins;
    const int *node_start, *node_pins;
    const int* net_order;  // nets sorted by degree (ascending)
    // WA pass 1 pin data in the degree-sorted net order: the pins of net net_order[t] are
    // entries [wa_start[t], wa_start[t+1]) in net-CSR order, each with its node and gradient
    // slot (wa_node_slot) and its pin offset (wa_off)
    const int* wa_start;
    const int2* wa_node_slot;
    const float2* wa_off;
    // per-pin WA gradient contributions (x, y), stored in node order: the pins of node i
    // that belong to a net own slots [slot_start[i], slot_start[i+1]) in node->pin order;
    // net_slot[q] is the slot of net-CSR entry q
    float *gpx, *gpy;
    const int *slot_start, *net_slot;
    // grid
    GridGeom geom;
    unsigned long long *node_fix, *filler_fix;
    float *terminal, *base, *rho, *phi, *ex, *ey, *node_map, *filler_map;
    double movable_area_scaled;
    // stage / optimizer
    int n_opt;
    const int* opt_idx;
    const float* opt_lo;   // clamp bounds, 2*nOpt (x then y)
    const float* opt_hi;
    const double* opt_area;
    // stage-static attributes of opt node k packed for one load each:
    //   opt_geom[k] = {hw, hh, wgt, 0} of its node (smoothed half extents, charge weight)
    //   opt_meta[k] = {first pin slot, end pin slot, nodeDegree, kind | OPT_HAS_WL}
    const float4* opt_geom;
    const int4* opt_meta;
    // Fillers (opt indices k >= filler_k0, nodes filler_node0 + k) all share one size and
    // carry no pins, so their per-node attributes are these constants instead of loads;
    // filler_k0 = n_opt when the fillers differ (then every node reads the arrays).
    int filler_k0, filler_node0;
    float4 filler_geom;
    int4 filler_meta;
    double filler_area;
    float filler_lo_x, filler_hi_x, filler_lo_y, filler_hi_y;
    float* force;          // 2*nOpt, density force q*xi (not gradient)
    // 2*nOpt: the opt cells' WA gradient (pass 2, wl_cells_kernel) formed beside the density
    // chain; null when the assembly sums the pin terms itself (SPG_WL_AHEAD=0)
    float* wlg;
    float* pool;           // NUM_ROLES + SNAP_MAX vectors of 2*nOpt
    size_t vec_stride;
    // density work lists (node ids): every density node, and the "rest" the loop's step
    // kernel does not rasterize itself (density nodes outside the opt set, and every node
    // whose footprint may exceed 16 bins)
    const int* dens_large;  // the large density nodes (the small ones are found by kind)
    int n_dens_small, n_dens_large;
    const int *rest_small, *rest_large;
    int n_rest_small, n_rest_large;
    const int* opt_large;  // opt positions k of the large nodes
    int n_opt_large;
    double* partials;      // RED_SLOTS * RED_CAP
    DevState* st;
    spg_iter_metrics* metrics;
    int ignore_net_degree;
    int use_bb, backtrack, max_backtrack;
    float min_gain;
    int stagnation_window;
    float step_x_gamma;   // grid.stepX() used by computeGamma
    int freeze_lambda, freeze_gamma;  // GpRunOptions diagnostics (eplace.cpp:374-380)
};

__device__ __forceinline__ float* role_ptr(const DevPtrs& p, int role) {
    return p.pool + static_cast<size_t>(p.st->role[role]) * p.vec_stride;
}

// Fixed-point charge of one node with at most 16 footprint bins (BinGrid::accumulate,
// bin_grid.cpp:191-251): every overlap x weight formed with the reference's float
// operations, rounded once to 64-bit fixed point and added with an integer atomic, so the
// maps do not depend on the order of the adds.
__device__ __forceinline__ void rasterize(const DevPtrs& p, float x, float y, float hw, float hh, float w,
                                          bool filler) {
    const GridGeom& g = p.geom;
    const Footprint f = footprint(g, x, y, hw, hh);
    unsigned long long* map = filler ? p.filler_fix : p.node_fix;
    if (f.bx1 - f.bx0 <= 1 && f.by1 - f.by0 <= 1) {
        // at most 2 x 2 bins (a node no larger than a bin after smoothing): unrolled, so the
        // bins' corners are formed once per column and row; the same contributions
        const bool x2 = f.bx1 > f.bx0, y2 = f.by1 > f.by0;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                if ((a && !x2) || (b && !y2)) continue;
                const int bx = f.bx0 + a, by = f.by0 + b;
                const float c = bin_contribution(g, bx, by, f, w);
                if (c > 0.f) atomicAdd(map + static_cast<size_t>(bx) * g.dim + by, to_fixed(c, g));
            }
        }
        return;
    }
    for (int bx = f.bx0; bx <= f.bx1; ++bx) {
        unsigned long long* row = map + static_cast<size_t>(bx) * g.dim;
        for (int by = f.by0; by <= f.by1; ++by) {
            const float c = bin_contribution(g, bx, by, f, w);
            if (c <= 0.f) continue;
            atomicAdd(row + by, to_fixed(c, g));
        }
    }
}

// Thread 0 of every block stores the block's partial of `slot`; block 0 also clears the
// entries past the grid, so the slot sums exactly this launch's partials.
__device__ __forceinline__ void put_partial(const DevPtrs& p, int slot, double v) {
    double* d = p.partials + static_cast<size_t>(slot) * RED_CAP;
    if (threadIdx.x == 0) d[blockIdx.x] = v;
    if (blockIdx.x == 0)
        for (int j = gridDim.x + threadIdx.x; j < RED_CAP; j += blockDim.x) d[j] = 0.0;
}

// ---- density.cu
void launch_density_accumulate(const DevPtrs& p, cudaStream_t s);
// the density nodes the loop's step kernel does not rasterize (rest_small, rest_large)
void launch_density_rest(const DevPtrs& p, cudaStream_t s);
// rho + tau partials; write_maps also stores the float maps, zero clears the fixed maps
void launch_rho_overflow(const DevPtrs& p, int write_maps, int zero, cudaStream_t s);
// rho + tau partials (clearing the fixed maps) and the first operand of a one-grid
// tensor-core Poisson solve: the split planes of rho's rows minus their means, and the sums
void launch_rho_prep(const DevPtrs& p, uint16_t* planes, int64_t plane_stride, int64_t ld, float* sums,
                     cudaStream_t s);
// force of the large (block-per-node) opt nodes; cells are gathered inside the assembly
void launch_gather_opt_large(const DevPtrs& p, cudaStream_t s);
// gather for every density node into a node-indexed 2*total array (parity hook)
void launch_gather_all(const DevPtrs& p, float* force_nodes, cudaStream_t s);
// the float quotients int(a[i] / step) and bin_index's form of them, for the self-check
void launch_bin_index_check(const float* a, int n, float step, double inv, int* q_div, int* q_mul, cudaStream_t s);

// ---- filler_order.cu
// Device buffers of the fillers' spatial reorder: n_keys = filler_order_keys(dim) tile keys,
// nf fillers, NUM_ROLES + SNAP_MAX pool vectors.
struct FillerOrderBufs {
    int *key_of, *tmp, *perm, *fid, *fid_tmp;  // nf each; fid = filler id of each filler slot
    int *count, *offset, *cursor;               // n_keys each
    int* skip;                                  // 1 when a tile exceeds the segment capacity
    float* scratch;                             // 2 * nf * filler_order_vectors()
    int* opt_idx;                               // the opt set's node ids (the fillers' are rewritten)
};
int filler_order_keys(int dim);
int filler_order_vectors();
// Reorders the filler segment of the opt set by tile of the current u (see filler_order.cu).
void launch_filler_order(const DevPtrs& p, const FillerOrderBufs& b, cudaStream_t s);

// ---- wirelength.cu
void launch_wa_nets(const DevPtrs& p, const WaClasses& wa, const float* gamma_dev, float gamma_host, int use_dev_gamma,
                    cudaStream_t s);
// node-indexed WA gradient for movable nodes (parity hook)
void launch_wa_node_grad(const DevPtrs& p, float* grad, cudaStream_t s);

// ---- optimizer.cu
void launch_scatter(const DevPtrs& p, int role, cudaStream_t s);
// WA pass 2 of the opt cells into p.wlg (after the WA nets pass, before the assembly)
void launch_wl_cells(const DevPtrs& p, cudaStream_t s);
// cell gather + gradient assembly (with wl_cells_kernel's WA sums); its last block finalizes
// the evaluation
void launch_assemble(const DevPtrs& p, int pos_role, int grad_role, int count_eval, cudaStream_t s);
// the loop's evaluation tail: the assembly at u = R_U into g = R_G with the step's norms
// and the per-iteration decisions in the same launch
// the loop's fused assembly; in graph mode it also sets the WHILE node's condition
void launch_assemble_reduce(const DevPtrs& p, cudaStream_t s, cudaGraphConditionalHandle loop_cond = 0);
// the loop pass's position step (the Nesterov step, or the re-evaluation step when the last
// decisions asked for one) with the density scatter of the new positions fused in; the
// evaluation that follows accumulates only the rest list
void launch_update(const DevPtrs& p, cudaStream_t s);
// the same step over the opt positions [k_begin, k_end) only
void launch_update_range(const DevPtrs& p, int k_begin, int k_end, cudaStream_t s);
// the same step over the optimizer vectors alone (no node arrays, no density), clamped into
// opt_lo / opt_hi: the optimizer run on the quadratic test objective
void launch_quad_step(const DevPtrs& p, cudaStream_t s);
// the quadratic test objective 0.5 sum c (x - t)^2 over the 2*nOpt coordinates: fused = the
// counted evaluation of the iteration with its norms and decisions, else an uncounted one of
// pos_role into grad_role
void launch_quad_eval(const DevPtrs& p, const float* coef, const float* target, int pos_role, int grad_role,
                      int fused, cudaStream_t s);
void launch_ctl_lambda_init(const DevPtrs& p, cudaStream_t s);
void launch_init_norms(const DevPtrs& p, cudaStream_t s);
void launch_ctl_init_scale(const DevPtrs& p, float init_perturb, cudaStream_t s);
void launch_init_perturb(const DevPtrs& p, cudaStream_t s);
void launch_init_diff(const DevPtrs& p, cudaStream_t s);
void launch_ctl_init_finish(const DevPtrs& p, cudaStream_t s);
void launch_copy_role(const DevPtrs& p, int dst_role, int src_role, cudaStream_t s);
void launch_clamp_role(const DevPtrs& p, int role, cudaStream_t s);
void launch_deliver(const DevPtrs& p, cudaStream_t s);
void launch_stage_clock(const DevPtrs& p, cudaStream_t s);
void launch_check_geometry(const DevPtrs& p, float lx, float ly, float hx, float hy, const float* w,
                           const float* h, cudaStream_t s);
void launch_finalize_slots(const DevPtrs& p, int first, int count, double* out, cudaStream_t s);

}  // namespace spg
