// Abacus row legalisation of the standard cells, on the host (no device code).
//
// The algorithm is Abacus (Spindler, Schlichtmann, Johannes, ISPD 2008), as the reference's
// LegalizeStage runs it (legalizeCells, src/lg/abacus.cpp:155-284; segments,
// buildAbacusSegments, src/lg/abacus.cpp:107-153):
//   - cells are the movable, non-macro, non-fixed, non-filler, non-NI nodes of positive size;
//     any movable macro that is not fixed yet makes the call a no-op (precondition_ok = 0);
//   - each row is cut into segments by the fixed obstacles (positive-area overlap only; NI,
//     filler and zero-size nodes are not obstacles) and clipped to the core; segment ends snap
//     inwards to the row's sites, and a segment narrower than the narrowest cell is dropped;
//   - cells are taken in order of their lower-left x (index on ties); a cell's width is a whole
//     number of sites (rounded when within 1e-5 of one, else up);
//   - rows are visited outwards from the cell's lower-left y, nearer first (below on ties),
//     until the squared row distance reaches the best cost; in a row the segment with room
//     whose clamped position is nearest is tried: the cell joins the segment's last cluster
//     (or opens one), clusters collapse to their optimal x and merge leftwards while they
//     overlap; cost = dx^2 + dy^2 of the cell's resulting position, strict improvement wins;
//   - finally each cluster's x is rounded to the row's sites, clamped into its segment and kept
//     right of the previous cluster, and the cells are laid out left to right.
// Cluster arithmetic is in double (e weight, q weighted position sum, w width, x position).
#include <algorithm>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "spgpu.h"

namespace {

thread_local std::string g_lg_error;

struct Db {
    const spg_db_view* v;
    float* x;  // centres, updated in place
    float* y;
    float llx(int i) const { return x[i] - 0.5f * v->node_w[i]; }
    float lly(int i) const { return y[i] - 0.5f * v->node_h[i]; }
    float urx(int i) const { return x[i] + 0.5f * v->node_w[i]; }
    float ury(int i) const { return y[i] + 0.5f * v->node_h[i]; }
    bool flag(int i, uint8_t f) const { return (v->node_flags[i] & f) != 0; }
    float row_hx(int r) const { return v->row_lx[r] + v->row_step[r] * static_cast<float>(v->row_num_sites[r]); }
    float row_hy(int r) const { return v->row_ly[r] + v->row_height[r]; }
};

bool is_cell(const Db& d, int i) {
    return i < d.v->num_movable &&
           !(d.v->node_flags[i] & (SPG_F_MACRO | SPG_F_FIXED | SPG_F_FILLER | SPG_F_NI)) &&
           d.v->node_w[i] > 0.f && d.v->node_h[i] > 0.f;
}

double sites_width(float width, float step) {
    const double sites = static_cast<double>(width) / step;
    const double whole = std::round(sites);
    return (std::abs(sites - whole) < 1e-5 ? whole : std::ceil(sites)) * step;
}

// std::clamp's expression, defined for lo > hi as well
inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }

struct Segment {
    int row;
    float lx, hx;
};

struct Cluster {
    int first = 0, last = 0;
    double e = 0.0, q = 0.0, w = 0.0, x = 0.0;
};

struct Lane {  // one segment's state
    Segment seg;
    double used = 0.0;
    std::vector<int> cells;
    std::vector<Cluster> clusters;
};

void place_cluster(Cluster& c, const Segment& s) { c.x = clampd(c.q / c.e, s.lx, static_cast<double>(s.hx) - c.w); }

void absorb(Cluster& c, int slot, double want, double width, double weight) {
    c.last = slot;
    c.e += weight;
    c.q += weight * (want - c.w);
    c.w += width;
}

Cluster join(const Cluster& left, const Cluster& right) {
    Cluster m = left;
    m.last = right.last;
    m.q += right.q - right.e * m.w;
    m.e += right.e;
    m.w += right.w;
    return m;
}

// The lane's last cluster after appending a cell at `want`, without touching the lane:
// clusters [0, keep) stay as they are and the returned one replaces the rest.
Cluster try_append(const Lane& lane, double want, double width, double weight, int& keep) {
    keep = static_cast<int>(lane.clusters.size());
    const int slot = static_cast<int>(lane.cells.size());
    Cluster c;
    if (keep > 0 && lane.clusters[keep - 1].x + lane.clusters[keep - 1].w > want) {
        c = lane.clusters[--keep];
    } else {
        c.first = slot;
    }
    absorb(c, slot, want, width, weight);
    place_cluster(c, lane.seg);
    while (keep > 0 && lane.clusters[keep - 1].x + lane.clusters[keep - 1].w > c.x) {
        c = join(lane.clusters[--keep], c);
        place_cluster(c, lane.seg);
    }
    return c;
}

std::vector<Segment> segments(const Db& d) {
    const spg_db_view* v = d.v;
    float min_w = std::numeric_limits<float>::infinity();
    for (int i = 0; i < v->num_movable; ++i)
        if (is_cell(d, i)) min_w = std::min(min_w, v->node_w[i]);
    if (!std::isfinite(min_w)) min_w = 0.f;
    std::vector<int> blocks;
    for (int i = 0; i < v->num_nodes; ++i)
        if (d.flag(i, SPG_F_FIXED) && !d.flag(i, SPG_F_NI) && !d.flag(i, SPG_F_FILLER) && v->node_w[i] > 0.f &&
            v->node_h[i] > 0.f)
            blocks.push_back(i);
    std::vector<Segment> out;
    std::vector<std::pair<double, double>> cut;
    for (int r = 0; r < v->num_rows; ++r) {
        const float lx = v->row_lx[r], ly = v->row_ly[r], step = v->row_step[r], h = v->row_height[r];
        if (!std::isfinite(lx) || !std::isfinite(ly) || !std::isfinite(step) || !std::isfinite(h) || step <= 0.f ||
            h <= 0.f || v->row_num_sites[r] <= 0)
            throw std::invalid_argument("invalid site row for Abacus");
        if (ly < v->core_ly || d.row_hy(r) > v->core_hy) continue;
        const double lo = std::max(lx, v->core_lx), hi = std::min(d.row_hx(r), v->core_hx);
        if (lo >= hi) continue;
        cut.clear();
        for (int i : blocks) {
            if (d.lly(i) >= d.row_hy(r) || d.ury(i) <= ly) continue;
            const double a = std::max(lo, static_cast<double>(d.llx(i)));
            const double b = std::min(hi, static_cast<double>(d.urx(i)));
            if (a < b) cut.emplace_back(a, b);
        }
        std::sort(cut.begin(), cut.end());
        auto open = [&](double a, double b) {
            if (a >= b) return;
            const double s = lx + std::ceil((a - lx) / step) * step;
            const double e = lx + std::floor((b - lx) / step) * step;
            if (e > s && e - s >= min_w) out.push_back({r, static_cast<float>(s), static_cast<float>(e)});
        };
        double at = lo;
        for (const auto& c : cut) {
            open(at, c.first);
            at = std::max(at, c.second);
        }
        open(at, hi);
    }
    return out;
}

spg_abacus_result legalize(Db& d, bool area_weight) {
    const spg_db_view* v = d.v;
    spg_abacus_result res{};
    res.precondition_ok = 1;
    res.rows = v->num_rows;
    for (int i = 0; i < v->num_movable; ++i)
        if (d.flag(i, SPG_F_MACRO) && !d.flag(i, SPG_F_FIXED)) {
            res.precondition_ok = 0;
            return res;
        }
    std::vector<int> order;
    for (int i = 0; i < v->num_nodes; ++i) {
        if (!std::isfinite(d.x[i]) || !std::isfinite(d.y[i]) || !std::isfinite(v->node_w[i]) ||
            !std::isfinite(v->node_h[i]))
            throw std::invalid_argument("non-finite node geometry for Abacus");
        if (is_cell(d, i)) order.push_back(i);
    }
    res.cells = static_cast<int>(order.size());
    if (order.empty()) return res;
    std::vector<float> x0(v->num_movable), y0(v->num_movable);  // lower-left targets
    for (int i : order) {
        x0[i] = d.llx(i);
        y0[i] = d.lly(i);
    }
    std::sort(order.begin(), order.end(), [&](int a, int b) { return x0[a] < x0[b] || (x0[a] == x0[b] && a < b); });
    const std::vector<Segment> segs = segments(d);
    res.segments = static_cast<int>(segs.size());
    std::vector<Lane> lanes(segs.size());
    std::vector<std::vector<int>> row_lanes(v->num_rows);
    for (size_t s = 0; s < segs.size(); ++s) {
        lanes[s].seg = segs[s];
        row_lanes[segs[s].row].push_back(static_cast<int>(s));
    }
    std::vector<int> rows_by_y(v->num_rows);
    for (int r = 0; r < v->num_rows; ++r) rows_by_y[r] = r;
    std::sort(rows_by_y.begin(), rows_by_y.end(), [&](int a, int b) {
        return v->row_ly[a] < v->row_ly[b] || (v->row_ly[a] == v->row_ly[b] && a < b);
    });
    const double inf = std::numeric_limits<double>::infinity();
    const int nrows = v->num_rows;
    for (int i : order) {
        const double want_x = x0[i], want_y = y0[i];
        const double weight = area_weight ? static_cast<double>(v->node_w[i]) * v->node_h[i] : 1.0;
        int best = -1;
        double best_cost = inf;
        int up = static_cast<int>(std::lower_bound(rows_by_y.begin(), rows_by_y.end(), want_y,
                                                   [&](int r, double yv) { return v->row_ly[r] < yv; }) -
                                  rows_by_y.begin());
        int down = up - 1;
        while (down >= 0 || up < nrows) {
            const double dd = down >= 0 ? std::abs(v->row_ly[rows_by_y[down]] - want_y) : inf;
            const double du = up < nrows ? std::abs(v->row_ly[rows_by_y[up]] - want_y) : inf;
            const double dist = std::min(dd, du);
            if (dist * dist >= best_cost) break;
            const int r = dd <= du ? rows_by_y[down--] : rows_by_y[up++];
            if (v->node_h[i] > v->row_height[r] + 1e-5f) continue;
            const double width = sites_width(v->node_w[i], v->row_step[r]);
            int pick = -1;
            double nearest = inf;
            for (int s : row_lanes[r]) {
                const Lane& ln = lanes[s];
                if (ln.used + width > static_cast<double>(ln.seg.hx) - ln.seg.lx + 1e-7) continue;
                const double dx = std::abs(clampd(want_x, ln.seg.lx, static_cast<double>(ln.seg.hx) - width) - want_x);
                if (dx < nearest) {
                    nearest = dx;
                    pick = s;
                }
            }
            if (pick < 0) continue;
            int keep;
            const Cluster c = try_append(lanes[pick], want_x, width, weight, keep);
            const double dx = c.x + c.w - width - want_x;
            const double cost = dx * dx + dist * dist;
            if (cost < best_cost) {
                best_cost = cost;
                best = pick;
            }
        }
        if (best < 0) {
            ++res.failed;
            continue;
        }
        Lane& ln = lanes[best];
        const float step = v->row_step[ln.seg.row];
        const double width = sites_width(v->node_w[i], step);
        if (std::abs(width - v->node_w[i]) > 1e-5) ++res.rounded_widths;
        int keep;
        const Cluster c = try_append(ln, want_x, width, weight, keep);
        ln.clusters.resize(keep);
        ln.clusters.push_back(c);
        ln.cells.push_back(i);
        ln.used += width;
    }

    double disp_sum = 0.0;
    for (Lane& ln : lanes) {
        const int r = ln.seg.row;
        const float rlx = v->row_lx[r], rly = v->row_ly[r], step = v->row_step[r];
        double prev_right = ln.seg.lx;
        for (const Cluster& c : ln.clusters) {
            double at = rlx + std::round((c.x - rlx) / step) * step;
            at = clampd(at, ln.seg.lx, static_cast<double>(ln.seg.hx) - c.w);
            at = std::max(at, prev_right);
            for (int slot = c.first; slot <= c.last; ++slot) {
                const int i = ln.cells[slot];
                d.x[i] = static_cast<float>(at) + 0.5f * v->node_w[i];
                d.y[i] = rly + 0.5f * v->node_h[i];
                const double disp = std::hypot(static_cast<double>(d.llx(i)) - x0[i],
                                               static_cast<double>(d.lly(i)) - y0[i]);
                disp_sum += disp;
                res.disp_max = std::max(res.disp_max, disp);
                at += sites_width(v->node_w[i], step);
            }
            prev_right = at;
        }
        float right = ln.seg.lx;
        for (int i : ln.cells) {
            if (d.llx(i) < right - 1e-3f) ++res.selfcheck_overlaps;
            const double sites = (static_cast<double>(d.llx(i)) - rlx) / step;
            if (std::abs(sites - std::round(sites)) * step > 1e-3 || std::abs(d.lly(i) - rly) > 1e-3 ||
                d.urx(i) > ln.seg.hx + 1e-3f)
                ++res.selfcheck_off_site;
            right = d.urx(i);
        }
    }
    const int placed = res.cells - res.failed;
    res.disp_mean = placed ? disp_sum / placed : 0.0;
    return res;
}

void check(const spg_db_view* v, const float* x, const float* y) {
    if (!v || !x || !y || v->num_movable < 0 || v->num_nodes < v->num_movable || v->num_rows < 0)
        throw std::invalid_argument("bad argument");
    if (v->num_nodes > 0 && (!v->node_w || !v->node_h || !v->node_flags))
        throw std::invalid_argument("spg_db_view without node arrays");
    if (v->num_rows > 0 && (!v->row_ly || !v->row_height || !v->row_lx || !v->row_step || !v->row_num_sites))
        throw std::invalid_argument("spg_db_view without row arrays");
}

}  // namespace

extern "C" {

const char* spg_abacus_last_error(void) { return g_lg_error.c_str(); }

int spg_abacus_legalize(const spg_db_view* db, int32_t area_weight, float* x, float* y, spg_abacus_result* out) {
    try {
        check(db, x, y);
        if (!out) throw std::invalid_argument("null result");
        Db d{db, x, y};
        *out = legalize(d, area_weight != 0);
        return SPG_OK;
    } catch (const std::exception& e) {
        g_lg_error = e.what();
        return SPG_E_INVALID;
    }
}

int spg_abacus_segments(const spg_db_view* db, const float* x, const float* y, int32_t* row, float* lx, float* hx,
                        int32_t cap, int32_t* count) {
    try {
        check(db, x, y);
        if (!count) throw std::invalid_argument("null count");
        Db d{db, const_cast<float*>(x), const_cast<float*>(y)};
        const std::vector<Segment> segs = segments(d);
        *count = static_cast<int32_t>(segs.size());
        for (int32_t k = 0; k < std::min<int32_t>(cap, *count); ++k) {
            row[k] = segs[k].row;
            lx[k] = segs[k].lx;
            hx[k] = segs[k].hx;
        }
        return SPG_OK;
    } catch (const std::exception& e) {
        g_lg_error = e.what();
        return SPG_E_INVALID;
    }
}

}  // extern "C"
