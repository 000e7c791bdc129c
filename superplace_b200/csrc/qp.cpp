// Bound2Bound (Kraftwerk2) quadratic initial placement, on the host.
//
// Restates QuadraticPlacer::place (src/init/quadratic_placer.cpp:153-228) with its pair rule
// forEachB2BPair (src/init/b2b_model.h:57-82):
//   every outer iteration finds each net's bound pins (leftmost/rightmost, lowest/highest; a
//   tie keeps the earlier pin, src/db/hpwl.cpp:70-103), then per axis
//   - assembles A x = b from the pairs (p, q) of every net of degree 2..ignore_net_degree with
//     at least one bound pin and the two pins on different nodes, weight
//     w = net_weight / (deg - 1) / max(|pos_p - pos_q|, max(1e-6, min_distance)):
//       both nodes movable   A_ii += w, A_jj += w, A_ij -= w, A_ji -= w,
//                            b_i += -w (off_i - off_j), b_j += -w (off_j - off_i)
//       one node fixed       A_ii += w, b_i += w (pos of the fixed pin - off_i)
//     a movable node without any entry gets A_ii = 1e-6, b_i += 1e-6 * its position;
//   - solves it by BiCGSTAB with a Jacobi preconditioner from the previous solution;
//   - clamps each movable centre into the core (the core centre when the node is wider).
// It stops after max_iter iterations, or once HPWL moves by less than outer_tol of itself
// after the fifth.
//
// The reference solves with Eigen 3.4.0 (a dependency, not shipped with it):
// SparseMatrix::setFromTriplets sums equal (row, column) triplets in the order they were
// emitted, and Eigen's BiCGSTAB is van der Vorst's algorithm (1992) with one restart rule:
// when |r0 . r| < eps^2 |r0|^2 the residual is recomputed and taken as the new r0. Here the
// matrix is built in compressed rows by a two-level bucket sort that keeps every entry's
// summation in emission order, so A and b are the reference's bit for bit. The solver's
// vector updates are the same float expressions; its dot products sum 64 fixed chunks of
// rows, in float, so the result does not depend on the thread count (Eigen's own dot products
// sum SIMD lanes, so the solver's float rounding is not the reference's).
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "qp_device.h"
#include "spgpu.h"

namespace {

thread_local std::string g_qp_error;

constexpr int kChunks = 64;  // fixed reduction and assembly chunks

inline int64_t chunk_lo(int64_t n, int c) { return n * c / kChunks; }

struct Axis {
    const float* pos;     // node centres along the axis
    const float* off;     // pin offsets along the axis
    const float* size;    // node sizes along the axis
    float core_lo, core_hi;
};

struct Problem {
    const spg_db_view* db;
    const float* weight;  // per net, or null for 1
    int32_t num_movable;
    float min_dist;
    int32_t ignore_degree;
};

inline float pin_pos(const Axis& a, const spg_db_view* db, int32_t p) {
    return a.pos[db->pin2node[p]] + a.off[p];
}

// Bound pins of every net along both axes (computeNetBoundPins, src/db/hpwl.cpp:70-103).
void bound_pins(const spg_db_view* db, const float* x, const float* y, std::vector<int32_t>& bx_lo,
                std::vector<int32_t>& bx_hi, std::vector<int32_t>& by_lo, std::vector<int32_t>& by_hi) {
    const int32_t nets = db->num_nets;
    bx_lo.assign(nets, -1);
    bx_hi.assign(nets, -1);
    by_lo.assign(nets, -1);
    by_hi.assign(nets, -1);
#pragma omp parallel for schedule(static)
    for (int32_t k = 0; k < nets; ++k) {
        const int32_t b = db->net2pin_start[k], e = db->net2pin_start[k + 1];
        if (b == e) continue;
        int32_t p0 = db->flat_net2pin[b];
        int32_t ixl = p0, ixh = p0, iyl = p0, iyh = p0;
        float xl = x[db->pin2node[p0]] + db->pin_offset_x[p0], xh = xl;
        float yl = y[db->pin2node[p0]] + db->pin_offset_y[p0], yh = yl;
        for (int32_t t = b + 1; t < e; ++t) {
            const int32_t p = db->flat_net2pin[t];
            const float px = x[db->pin2node[p]] + db->pin_offset_x[p];
            const float py = y[db->pin2node[p]] + db->pin_offset_y[p];
            if (px < xl) { xl = px; ixl = p; }
            if (px > xh) { xh = px; ixh = p; }
            if (py < yl) { yl = py; iyl = p; }
            if (py > yh) { yh = py; iyh = p; }
        }
        bx_lo[k] = ixl;
        bx_hi[k] = ixh;
        by_lo[k] = iyl;
        by_hi[k] = iyh;
    }
}

// One contribution in emission order: a matrix entry (col >= 0) or a right-hand side term.
struct Entry {
    int32_t row, col;
    float val;
};

constexpr int32_t kRhs = -1;

// The B2B pairs of net k in the reference's (s, t) order, each as its matrix and rhs entries.
template <typename Emit>
void net_entries(const Problem& P, const Axis& a, int32_t k, int32_t lo, int32_t hi, Emit&& emit) {
    const spg_db_view* db = P.db;
    const int32_t b = db->net2pin_start[k], e = db->net2pin_start[k + 1];
    const int32_t deg = e - b;
    if (deg < 2 || deg > P.ignore_degree) return;
    const float coef = (P.weight ? P.weight[k] : 1.f) / static_cast<float>(deg - 1);
    const float min_d = std::max(1e-6f, P.min_dist);
    // slots of the bound pins in the net: a pair needs one of them, so a pin that is not bound
    // pairs only with the bound pins after it (visited in slot order, as the (s, t) loops do)
    int32_t t_lo = -1, t_hi = -1;
    for (int32_t t = b; t < e; ++t) {
        if (db->flat_net2pin[t] == lo && t_lo < 0) t_lo = t;
        if (db->flat_net2pin[t] == hi && t_hi < 0) t_hi = t;
    }
    const int32_t bound_slot[2] = {std::min(t_lo, t_hi), std::max(t_lo, t_hi)};
    auto pair = [&](int32_t p, int32_t q) {
        const int32_t ni = db->pin2node[p], nj = db->pin2node[q];
        if (ni == nj) return;
        const float w = coef / std::max(std::fabs(pin_pos(a, db, p) - pin_pos(a, db, q)), min_d);
        const float off_i = a.off[p], off_j = a.off[q];
        const bool mi = ni < P.num_movable, mj = nj < P.num_movable;
        if (mi && mj) {
            emit(Entry{ni, ni, w});
            emit(Entry{nj, nj, w});
            emit(Entry{ni, nj, -w});
            emit(Entry{nj, ni, -w});
            emit(Entry{ni, kRhs, -w * (off_i - off_j)});
            emit(Entry{nj, kRhs, -w * (off_j - off_i)});
        } else if (mi) {
            emit(Entry{ni, ni, w});
            emit(Entry{ni, kRhs, w * (pin_pos(a, db, q) - off_i)});
        } else if (mj) {
            emit(Entry{nj, nj, w});
            emit(Entry{nj, kRhs, w * (pin_pos(a, db, p) - off_j)});
        }
    };
    for (int32_t s = b; s < e; ++s) {
        const int32_t p = db->flat_net2pin[s];
        if (p == lo || p == hi) {
            for (int32_t t = s + 1; t < e; ++t) pair(p, db->flat_net2pin[t]);
        } else {
            for (int j = 0; j < 2; ++j) {
                const int32_t t = bound_slot[j];
                if (t > s && !(j == 1 && t == bound_slot[0])) pair(p, db->flat_net2pin[t]);
            }
        }
    }
}

struct Csr {
    std::vector<int32_t> start, col;
    std::vector<float> val, rhs;
};

// A and b of one axis. Nets are cut into kChunks ranges and rows into kChunks blocks: each
// net range sorts its entries into per-block buckets (in emission order), then each row block
// reads its buckets range by range, so every row sees its entries in emission order. A row's
// entries are ordered by column stably and equal columns summed left to right, from the
// zero diagonal the reference seeds first.
void assemble(const Problem& P, const Axis& a, const std::vector<int32_t>& lo, const std::vector<int32_t>& hi,
              Csr& m) {
    const spg_db_view* db = P.db;
    const int32_t n = P.num_movable;
    const int32_t nets = db->num_nets;
    const int32_t rows_per_block = std::max<int32_t>(1, (n + kChunks - 1) / kChunks);
    std::vector<std::vector<Entry>> bucket(static_cast<size_t>(kChunks) * kChunks);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < kChunks; ++c) {
        std::vector<Entry>* mine = &bucket[static_cast<size_t>(c) * kChunks];
        for (int32_t k = static_cast<int32_t>(chunk_lo(nets, c)); k < static_cast<int32_t>(chunk_lo(nets, c + 1)); ++k)
            net_entries(P, a, k, lo[k], hi[k], [&](const Entry& en) { mine[en.row / rows_per_block].push_back(en); });
    }
    std::vector<std::vector<Entry>> block_rows(kChunks);  // reduced entries of each block, row-major
    std::vector<int32_t> row_nnz(n, 0);
    m.rhs.assign(n, 0.f);
#pragma omp parallel for schedule(dynamic, 1)
    for (int rb = 0; rb < kChunks; ++rb) {
        const int32_t r0 = std::min(n, rb * rows_per_block), r1 = std::min(n, r0 + rows_per_block);
        if (r0 >= r1) continue;
        std::vector<int32_t> cnt(static_cast<size_t>(r1 - r0) + 1, 0);
        size_t total = 0;
        for (int c = 0; c < kChunks; ++c) {
            const std::vector<Entry>& v = bucket[static_cast<size_t>(c) * kChunks + rb];
            total += v.size();
            for (const Entry& en : v) ++cnt[en.row - r0 + 1];
        }
        for (int32_t r = 0; r < r1 - r0; ++r) cnt[r + 1] += cnt[r];
        std::vector<Entry> sorted(total);
        std::vector<int32_t> next(cnt.begin(), cnt.end() - 1);
        for (int c = 0; c < kChunks; ++c)
            for (const Entry& en : bucket[static_cast<size_t>(c) * kChunks + rb]) sorted[next[en.row - r0]++] = en;
        std::vector<Entry>& out = block_rows[rb];
        out.resize(total + static_cast<size_t>(r1 - r0));  // at most every entry plus a diagonal per row
        size_t o = 0;
        std::vector<Entry> off;
        for (int32_t r = r0; r < r1; ++r) {
            const Entry* row = sorted.data() + cnt[r - r0];
            const size_t len = static_cast<size_t>(cnt[r - r0 + 1] - cnt[r - r0]);
            // the right-hand side and the diagonal are summed in emission order as they come
            // (the diagonal from the zero the reference seeds first); only the off-diagonal
            // entries need ordering by column (stable, so equal columns keep emission order)
            float rhs = 0.f, diag = 0.f;
            off.clear();
            for (size_t j = 0; j < len; ++j) {
                if (row[j].col == kRhs) rhs += row[j].val;
                else if (row[j].col == r) diag += row[j].val;
                else off.push_back(row[j]);
            }
            for (size_t j = 1; j < off.size(); ++j) {  // stable insertion sort by column
                const Entry en = off[j];
                size_t h = j;
                for (; h > 0 && off[h - 1].col > en.col; --h) off[h] = off[h - 1];
                off[h] = en;
            }
            if (diag == 0.f) {  // a movable node with no connection: a tiny pull to where it is
                diag = 1e-6f;
                rhs += 1e-6f * a.pos[r];
            }
            const size_t before = o;
            bool diag_out = false;
            for (size_t i = 0; i < off.size();) {
                const int32_t c = off[i].col;
                if (!diag_out && c > r) {
                    out[o++] = Entry{r, r, diag};
                    diag_out = true;
                }
                float v = off[i].val;
                for (++i; i < off.size() && off[i].col == c; ++i) v += off[i].val;
                out[o++] = Entry{r, c, v};
            }
            if (!diag_out) out[o++] = Entry{r, r, diag};
            m.rhs[r] = rhs;
            row_nnz[r] = static_cast<int32_t>(o - before);
        }
        out.resize(o);
    }
    m.start.assign(static_cast<size_t>(n) + 1, 0);
    for (int32_t r = 0; r < n; ++r) m.start[r + 1] = m.start[r] + row_nnz[r];
    m.col.resize(m.start[n]);
    m.val.resize(m.start[n]);
#pragma omp parallel for schedule(static)
    for (int rb = 0; rb < kChunks; ++rb) {
        const std::vector<Entry>& v = block_rows[rb];
        if (v.empty()) continue;
        size_t at = static_cast<size_t>(m.start[v.front().row]);
        for (const Entry& en : v) {
            m.col[at] = en.col;
            m.val[at] = en.val;
            ++at;
        }
    }
}

// ------------------------------------------------------------------ BiCGSTAB
void spmv(const Csr& m, const std::vector<float>& x, std::vector<float>& y) {
    const int32_t n = static_cast<int32_t>(m.rhs.size());
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
        float s = 0.f;
        for (int32_t k = m.start[i]; k < m.start[i + 1]; ++k) s += m.val[k] * x[m.col[k]];
        y[i] = s;
    }
}

// u . v in the device solver's summation order (qp_device.cu): 1024 x 256 threads, thread g
// summing rows g, g + 262144, ... in float; a halving tree over each block's 256 partials; the
// 1024 block sums folded four to a slot, ((b[t] + b[t+256]) + b[t+512]) + b[t+768], and a last
// halving tree. The same order on the host makes the two solvers agree bit for bit.
float dot(const std::vector<float>& u, const std::vector<float>& v) {
    const int64_t n = static_cast<int64_t>(u.size());
    float blk[kQpBlocks];
#pragma omp parallel for schedule(static)
    for (int b = 0; b < kQpBlocks; ++b) {
        float s[kQpThreads];
        for (int t = 0; t < kQpThreads; ++t) {
            float acc = 0.f;
            for (int64_t i = int64_t(b) * kQpThreads + t; i < n; i += kQpGrid) acc += u[i] * v[i];
            s[t] = acc;
        }
        blk[b] = qp_tree(s);
    }
    return qp_fold_blocks(blk);
}

struct SolveInfo {
    int32_t iters;
    float error;
};

// BiCGSTAB, Jacobi-preconditioned, from the guess in x (the restart rule as described above).
SolveInfo bicgstab(const Csr& m, std::vector<float>& x, int32_t max_iter, float tol) {
    const int32_t n = static_cast<int32_t>(m.rhs.size());
    const std::vector<float>& b = m.rhs;
    std::vector<float> inv(n, 1.f);
    for (int32_t i = 0; i < n; ++i)
        for (int32_t k = m.start[i]; k < m.start[i + 1]; ++k)
            if (m.col[k] == i && m.val[k] != 0.f) inv[i] = 1.f / m.val[k];
    std::vector<float> r(n), r0, v(n, 0.f), p(n, 0.f), y(n), z(n), s(n), t(n), ax(n);
    auto residual = [&]() {
        spmv(m, x, ax);
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) r[i] = b[i] - ax[i];
    };
    residual();
    r0 = r;
    float r0_sq = dot(r0, r0);
    const float b_sq = dot(b, b);
    if (b_sq == 0.f) {
        std::fill(x.begin(), x.end(), 0.f);
        return {max_iter, tol};
    }
    float rho = 1.f, alpha = 1.f, w = 1.f;
    const float tol2 = tol * tol * b_sq;
    const float eps = std::numeric_limits<float>::epsilon();
    const float eps2 = eps * eps;
    int32_t it = 0, restarts = 0;
    while (dot(r, r) > tol2 && it < max_iter) {
        const float rho_old = rho;
        rho = dot(r0, r);
        if (std::fabs(rho) < eps2 * r0_sq) {
            residual();
            r0 = r;
            rho = r0_sq = dot(r, r);
            if (restarts++ == 0) it = 0;
        }
        const float beta = (rho / rho_old) * (alpha / w);
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            p[i] = r[i] + beta * (p[i] - w * v[i]);
            y[i] = inv[i] * p[i];
        }
        spmv(m, y, v);
        alpha = rho / dot(r0, v);
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            s[i] = r[i] - alpha * v[i];
            z[i] = inv[i] * s[i];
        }
        spmv(m, z, t);
        const float tt = dot(t, t);
        w = tt > 0.f ? dot(t, s) / tt : 0.f;
#pragma omp parallel for schedule(static)
        for (int32_t i = 0; i < n; ++i) {
            x[i] += alpha * y[i] + w * z[i];
            r[i] = s[i] - w * t[i];
        }
        ++it;
    }
    return {it, std::sqrt(dot(r, r) / b_sq)};
}

// computeHPWL (src/db/hpwl.cpp:13-39): per-net float bounding boxes summed as doubles over 64
// fixed chunks of nets.
double hpwl(const spg_db_view* db, const float* x, const float* y) {
    const int64_t nets = db->num_nets;
    double part[kChunks];
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < kChunks; ++c) {
        double s = 0.0;
        for (int64_t k = chunk_lo(nets, c); k < chunk_lo(nets, c + 1); ++k) {
            const int32_t b = db->net2pin_start[k], e = db->net2pin_start[k + 1];
            if (e - b < 2) continue;
            float xl = std::numeric_limits<float>::max(), xh = -std::numeric_limits<float>::max();
            float yl = xl, yh = xh;
            for (int32_t t = b; t < e; ++t) {
                const int32_t p = db->flat_net2pin[t];
                const float px = x[db->pin2node[p]] + db->pin_offset_x[p];
                const float py = y[db->pin2node[p]] + db->pin_offset_y[p];
                xl = std::min(xl, px);
                xh = std::max(xh, px);
                yl = std::min(yl, py);
                yh = std::max(yh, py);
            }
            s += static_cast<double>(xh - xl) + static_cast<double>(yh - yl);
        }
        part[c] = s;
    }
    double total = 0.0;
    for (int c = 0; c < kChunks; ++c) total += part[c];
    return total;
}

void check_view(const spg_db_view* db) {
    if (!db || db->num_movable < 0 || db->num_nodes < db->num_movable || db->num_nets < 0 || db->num_pins < 0)
        throw std::invalid_argument("bad spg_db_view");
    if (db->num_nets > 0 && (!db->net2pin_start || !db->flat_net2pin || !db->pin2node || !db->pin_offset_x ||
                             !db->pin_offset_y))
        throw std::invalid_argument("spg_db_view without nets/pins arrays");
}

Problem problem(const spg_db_view* db, const float* weight, const spg_qp_params* p) {
    return Problem{db, weight, db->num_movable, p->min_distance, p->ignore_net_degree};
}

Axis axis_of(const spg_db_view* db, int32_t ax, const float* x, const float* y) {
    return ax == 0 ? Axis{x, db->pin_offset_x, db->node_w, db->core_lx, db->core_hx}
                   : Axis{y, db->pin_offset_y, db->node_h, db->core_ly, db->core_hy};
}

struct Threads {  // the caller's OpenMP thread count, restored on exit
    int saved;
    explicit Threads(int n) : saved(omp_get_max_threads()) {
        if (n > 0) omp_set_num_threads(n);
    }
    ~Threads() { omp_set_num_threads(saved); }
};

int qp_fail(const std::exception& e) {
    g_qp_error = e.what();
    if (const auto* d = dynamic_cast<const QpDeviceError*>(&e)) return d->code;
    return SPG_E_INVALID;
}

}  // namespace

extern "C" {

const char* spg_qp_last_error(void) { return g_qp_error.c_str(); }

void spg_qp_default_params(spg_qp_params* p) {
    if (!p) return;
    p->max_iter = 20;
    p->tol = 1e-6f;
    p->solver_max_iter = 100;
    p->outer_tol = 1e-4f;
    p->min_distance = 1.0f;
    p->ignore_net_degree = 100;
    p->threads = 0;
    p->device = 0;
}

int spg_qp_place(const spg_db_view* db, const float* net_weight, const spg_qp_params* prm, float* x, float* y,
                 spg_qp_row* rows, int32_t cap, int32_t* num_rows) {
    try {
        check_view(db);
        if (!prm || !x || !y || (cap > 0 && !rows)) throw std::invalid_argument("null argument");
        const Threads threads(prm->threads);
        if (num_rows) *num_rows = 0;
        const int32_t n = db->num_movable;
        if (n == 0) return SPG_OK;
        const Problem P = problem(db, net_weight, prm);
        const float cx = 0.5f * (db->core_lx + db->core_hx);
        const float cy = 0.5f * (db->core_ly + db->core_hy);
        for (int32_t i = 0; i < n; ++i) {
            x[i] = cx;
            y[i] = cy;
        }
        std::vector<float> sol_x(x, x + n), sol_y(y, y + n);
        struct DeviceSolver {  // the GPU's BiCGSTAB, when asked for
            QpDevice* d = nullptr;
            ~DeviceSolver() { qp_device_destroy(d); }
        } gpu;
        if (prm->device) gpu.d = qp_device_create();
        std::vector<int32_t> bxl, bxh, byl, byh;
        Csr m;
        double last = 0.0;
        for (int32_t iter = 0;; ++iter) {
            using clock = std::chrono::steady_clock;
            auto ms = [](clock::time_point a, clock::time_point b) {
                return std::chrono::duration<double, std::milli>(b - a).count();
            };
            const auto t0 = clock::now();
            double t_asm = 0.0, t_solve = 0.0;
            bound_pins(db, x, y, bxl, bxh, byl, byh);
            t_asm += ms(t0, clock::now());
            SolveInfo info[2];
            for (int32_t ax = 0; ax < 2; ++ax) {
                const Axis a = axis_of(db, ax, x, y);
                const auto ta = clock::now();
                assemble(P, a, ax == 0 ? bxl : byl, ax == 0 ? bxh : byh, m);
                const auto tb = clock::now();
                t_asm += ms(ta, tb);
                std::vector<float>& sol = ax == 0 ? sol_x : sol_y;
                if (gpu.d) {
                    qp_device_solve(gpu.d, n, static_cast<int64_t>(m.col.size()), m.start.data(), m.col.data(),
                                    m.val.data(), m.rhs.data(), sol.data(), prm->solver_max_iter, prm->tol,
                                    &info[ax].iters, &info[ax].error);
                } else {
                    info[ax] = bicgstab(m, sol, prm->solver_max_iter, prm->tol);
                }
                t_solve += ms(tb, clock::now());
                float* pos = ax == 0 ? x : y;
#pragma omp parallel for schedule(static)
                for (int32_t i = 0; i < n; ++i) {
                    float v = sol[i];
                    if (!std::isfinite(v)) v = pos[i];
                    const float half = 0.5f * a.size[i];
                    const float lo = a.core_lo + half, hi = a.core_hi - half;
                    v = lo <= hi ? std::min(std::max(v, lo), hi) : 0.5f * (lo + hi);
                    pos[i] = v;
                    sol[i] = v;
                }
                if (!std::isfinite(info[ax].error)) info[ax].error = 0.f;
            }
            const double h = hpwl(db, x, y);
            if (num_rows && *num_rows < cap) {
                spg_qp_row& r = rows[(*num_rows)++];
                r.iter = iter;
                r.solver_iters_x = info[0].iters;
                r.solver_iters_y = info[1].iters;
                r.err = std::max(info[0].error, info[1].error);
                r.hpwl = h;
                r.elapsed_ms = ms(t0, clock::now());
                r.assemble_ms = t_asm;
                r.solve_ms = t_solve;
            }
            const bool stalled = iter > 4 && last > 0.0 && std::fabs(h - last) < prm->outer_tol * last;
            last = h;
            if (stalled || iter + 1 >= prm->max_iter) break;
        }
        return SPG_OK;
    } catch (const std::exception& e) {
        return qp_fail(e);
    }
}

int spg_qp_assemble(const spg_db_view* db, const float* net_weight, const spg_qp_params* prm, int32_t axis,
                    const float* x, const float* y, int32_t* row_start, int32_t* col, float* val, float* rhs,
                    int64_t cap, int64_t* nnz) {
    try {
        check_view(db);
        if (!prm || !x || !y || !nnz || (axis != 0 && axis != 1)) throw std::invalid_argument("bad argument");
        const Threads threads(prm->threads);
        std::vector<int32_t> bxl, bxh, byl, byh;
        bound_pins(db, x, y, bxl, bxh, byl, byh);
        Csr m;
        assemble(problem(db, net_weight, prm), axis_of(db, axis, x, y), axis == 0 ? bxl : byl,
                 axis == 0 ? bxh : byh, m);
        *nnz = static_cast<int64_t>(m.col.size());
        if (cap < *nnz) return SPG_OK;  // sizes only
        if (!row_start || !col || !val || !rhs) throw std::invalid_argument("null output array");
        std::copy(m.start.begin(), m.start.end(), row_start);
        std::copy(m.col.begin(), m.col.end(), col);
        std::copy(m.val.begin(), m.val.end(), val);
        std::copy(m.rhs.begin(), m.rhs.end(), rhs);
        return SPG_OK;
    } catch (const std::exception& e) {
        return qp_fail(e);
    }
}

int spg_host_hpwl(const spg_db_view* db, const float* x, const float* y, double* out) {
    try {
        check_view(db);
        if (!x || !y || !out) throw std::invalid_argument("null argument");
        *out = hpwl(db, x, y);
        return SPG_OK;
    } catch (const std::exception& e) {
        return qp_fail(e);
    }
}

}  // extern "C"
