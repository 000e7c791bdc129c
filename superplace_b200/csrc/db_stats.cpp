// The parse stage's design summary, on the host: DbStats::compute and DbStats::toString
// (src/db/db_stats.cpp:9-118, fields src/db/db_stats.h:17-86). Areas are summed in double in
// node order; a fixed node's area inside the core is its box clipped to the core; net degrees
// are binned 1 / 2 / 3-9 / 10-99 / >= 100, with exact counts up to 100.
#include <algorithm>
#include <cstdio>
#include <string>

#include "spgpu.h"

namespace {

void compute(const spg_db_view* v, spg_db_stats* s) {
    *s = spg_db_stats{};
    s->core_lx = v->core_lx;
    s->core_ly = v->core_ly;
    s->core_hx = v->core_hx;
    s->core_hy = v->core_hy;
    s->row_height = v->row_height_mode;
    s->row_count = v->num_rows;
    s->site_step = v->num_rows > 0 ? v->row_step[0] : 0.0;
    s->core_area = (s->core_hx - s->core_lx) * (s->core_hy - s->core_ly);
    s->total_row_area = v->total_row_area;
    for (int i = 0; i < v->num_nodes; ++i) {
        const float w = v->node_w[i], h = v->node_h[i];
        const double a = static_cast<double>(w) * static_cast<double>(h);
        if (v->node_flags[i] & SPG_F_FIXED) {
            s->fixed_area += a;
            ++s->fixed_count;
            const float lx = v->node_x[i] - 0.5f * w, hx = v->node_x[i] + 0.5f * w;
            const float ly = v->node_y[i] - 0.5f * h, hy = v->node_y[i] + 0.5f * h;
            const double dx = std::min<double>(hx, s->core_hx) - std::max<double>(lx, s->core_lx);
            const double dy = std::min<double>(hy, s->core_hy) - std::max<double>(ly, s->core_ly);
            if (dx > 0.0 && dy > 0.0) s->fixed_area_in_core += dx * dy;
        } else {
            s->movable_area += a;
            ++s->node_count;
            if (v->node_flags[i] & SPG_F_MACRO) ++s->macro_count;
        }
    }
    s->object_count = v->num_nodes;
    s->net_count = v->num_nets;
    s->pin_count = v->num_pins;
    for (int k = 0; k < v->num_nets; ++k) {
        const int d = v->net2pin_start[k + 1] - v->net2pin_start[k];
        s->max_net_degree = std::max(s->max_net_degree, d);
        if (d <= 100) ++s->degree_count[d];
        else ++s->degree_over;
        if (d == 1) ++s->degree_histogram[0];
        else if (d == 2) ++s->degree_histogram[1];
        else if (d >= 3 && d <= 9) ++s->degree_histogram[2];
        else if (d >= 10 && d <= 99) ++s->degree_histogram[3];
        else if (d >= 100) ++s->degree_histogram[4];
    }
}

std::string text(const spg_db_stats& s) {
    auto ratio = [&](double a) { return s.core_area > 0 ? a / s.core_area : 0.0; };
    const double free_sites = s.total_row_area - s.fixed_area_in_core;
    const double util = free_sites > 0 ? s.movable_area / free_sites : 0.0;
    const double density = s.core_area > 0 ? (s.movable_area + s.fixed_area_in_core) / s.core_area : 0.0;
    std::string out = "\n<<<< DATABASE SUMMARY >>>>\n\n";
    char b[512];
    auto add = [&](int len) { out.append(b, static_cast<size_t>(std::min<int>(len, sizeof b - 1))), out += '\n'; };
    add(std::snprintf(b, sizeof b, "       Core region: (%.0f, %.0f) - (%.0f, %.0f)", s.core_lx, s.core_ly, s.core_hx,
                      s.core_hy));
    add(std::snprintf(b, sizeof b, "Row height / count: %.0f / %d  (site step %.6f)", s.row_height, s.row_count,
                      s.site_step));
    add(std::snprintf(b, sizeof b, "         Core area: %.0f", s.core_area));
    add(std::snprintf(b, sizeof b, "         Cell area: %.0f  (%.2f%%)", s.movable_area, ratio(s.movable_area) * 100.0));
    add(std::snprintf(b, sizeof b, "      Movable area: %.0f  (%.2f%%)", s.movable_area, ratio(s.movable_area) * 100.0));
    add(std::snprintf(b, sizeof b, "        Fixed area: %.0f  (%.2f%%)", s.fixed_area, ratio(s.fixed_area) * 100.0));
    add(std::snprintf(b, sizeof b, " Fixed area in core: %.0f  (%.2f%%)", s.fixed_area_in_core,
                      ratio(s.fixed_area_in_core) * 100.0));
    add(std::snprintf(b, sizeof b, "   Placement util.: %.2f%%  (= move / freeSites)", util * 100.0));
    add(std::snprintf(b, sizeof b, "      Core density: %.2f%%  (= usedArea / core)", density * 100.0));
    add(std::snprintf(b, sizeof b, "             Nodes: %d", s.node_count));
    add(std::snprintf(b, sizeof b, "           Objects: %d  (fixed: %d, macro: %d)", s.object_count, s.fixed_count,
                      s.macro_count));
    add(std::snprintf(b, sizeof b, "              Nets: %d", s.net_count));
    add(std::snprintf(b, sizeof b, "              Pins: %d", s.pin_count));
    add(std::snprintf(b, sizeof b, "    Max net degree: %d", s.max_net_degree));
    const int* h = s.degree_histogram;
    add(std::snprintf(b, sizeof b, "   Pin degree dist: 2:(%d)  3-10:(%d)  11-100:(%d)  100-:(%d)   [reference bins]",
                      h[1], h[0] + h[2], h[3], h[4]));
    add(std::snprintf(b, sizeof b, "   Exact degree   : 1:(%d)  2:(%d)  3-9:(%d)  10-99:(%d)  >=100:(%d)", h[0], h[1],
                      h[2], h[3], h[4]));
    out += '\n';
    return out;
}

}  // namespace

extern "C" {

int spg_db_stats_compute(const spg_db_view* db, spg_db_stats* out) {
    if (!db || !out || db->num_nodes < 0 || db->num_nets < 0) return SPG_E_INVALID;
    if ((db->num_nodes > 0 && (!db->node_w || !db->node_h || !db->node_x || !db->node_y || !db->node_flags)) ||
        (db->num_nets > 0 && !db->net2pin_start) || (db->num_rows > 0 && !db->row_step))
        return SPG_E_INVALID;
    compute(db, out);
    return SPG_OK;
}

int64_t spg_db_stats_text(const spg_db_stats* s, char* buf, int64_t cap) {
    if (!s) return SPG_E_INVALID;
    const std::string t = text(*s);
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>(t.size(), static_cast<size_t>(cap - 1));
        t.copy(buf, n);
        buf[n] = '\0';
    }
    return static_cast<int64_t>(t.size());
}

}  // extern "C"
