// The other initial placers of the reference's init stage, on the host (no device code):
// "random" (RandomPlacer::place, src/init/random_placer.cpp:15-38) and "cluster_fc" /
// "cluster_bc" (ClusterPlacer::place, src/init/cluster_common.cpp; matchers in
// src/init/cluster_fc.cpp and src/init/cluster_bc.cpp). The "quadratic" one is qp.cpp.
//
// random: each movable centre uniform in the range that keeps the node inside the core (the
//   core centre when the node is wider), x then y, from std::mt19937(seed) through
//   std::uniform_real_distribution<float>, the reference's Rng.
// cluster: the movable nodes are coarsened into about n / 25 clusters (or a given count) by
//   repeated matching on the net hypergraph (nets of degree 2..ignore_net_degree, fixed pins
//   left out, a net counted once per cluster; the weight of a neighbour is the sum over shared
//   nets of 1 / (clusters on the net - 1), heaviest wins, lower index on ties):
//     first choice  visit clusters in index order, pair each free one with its best free
//                   neighbour;
//     best choice   a max-heap of (weight, cluster, neighbour) (ties: lower cluster, lower
//                   neighbour); a popped pair whose neighbour is taken is re-scored up to 3
//                   times;
//   a level stops early when it merges fewer than 1 in 50 clusters, and after 128 levels.
//   Clusters are then ordered breadth-first over shared nets (seeds in index order, neighbours
//   in index order), cut into round(sqrt(count)) shelves of equal area laid bottom-up across
//   the core in boustrophedon order, each cluster given a box of its area share, and its
//   nodes spread on a ceil(sqrt(m)) x ceil(sqrt(m)) grid in the box, clamped into the core.
#include <algorithm>
#include <cmath>
#include <memory>
#include <queue>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "spgpu.h"

namespace {

thread_local std::string g_init_error;

struct Hypergraph {  // nets over clusters, and each cluster's nets
    int clusters = 0;
    std::vector<int> net_start{0}, members, clu_start, clu_nets;
    int nets() const { return static_cast<int>(net_start.size()) - 1; }
    int size(int k) const { return net_start[k + 1] - net_start[k]; }
    void index() {
        clu_start.assign(static_cast<size_t>(clusters) + 1, 0);
        for (int m : members) ++clu_start[m + 1];
        for (int c = 0; c < clusters; ++c) clu_start[c + 1] += clu_start[c];
        clu_nets.resize(members.size());
        std::vector<int> at(clu_start.begin(), clu_start.end() - 1);
        for (int k = 0; k < nets(); ++k)
            for (int t = net_start[k]; t < net_start[k + 1]; ++t) clu_nets[at[members[t]]++] = k;
    }
};

struct Scratch {
    std::vector<float> weight;
    std::vector<int> touched;
    std::vector<char> taken;
    void reset(int n) {
        weight.assign(n, 0.f);
        taken.assign(n, 0);
        touched.clear();
    }
};

// The heaviest free neighbour of cluster c (-1 when none), its weight in *w.
int best_neighbour(const Hypergraph& g, int c, Scratch& s, float* w) {
    s.touched.clear();
    for (int t = g.clu_start[c]; t < g.clu_start[c + 1]; ++t) {
        const int k = g.clu_nets[t];
        const int m = g.size(k);
        if (m < 2) continue;
        const float share = 1.0f / static_cast<float>(m - 1);
        for (int q = g.net_start[k]; q < g.net_start[k + 1]; ++q) {
            const int o = g.members[q];
            if (o == c || s.taken[o]) continue;
            if (s.weight[o] == 0.f) s.touched.push_back(o);
            s.weight[o] += share;
        }
    }
    int best = -1;
    float best_w = 0.f;
    for (int o : s.touched) {
        const float v = s.weight[o];
        if (v > best_w || (v == best_w && best >= 0 && o < best)) {
            best_w = v;
            best = o;
        }
    }
    for (int o : s.touched) s.weight[o] = 0.f;
    if (w) *w = best_w;
    return best;
}

int match_first_choice(const Hypergraph& g, int max_merges, std::vector<int>& partner, Scratch& s) {
    partner.assign(g.clusters, -1);
    int merges = 0;
    for (int c = 0; c < g.clusters && merges < max_merges; ++c) {
        if (s.taken[c]) continue;
        const int b = best_neighbour(g, c, s, nullptr);
        if (b < 0) continue;
        partner[c] = b;
        s.taken[c] = s.taken[b] = 1;
        ++merges;
    }
    return merges;
}

struct Candidate {
    float w;
    int from, to;
    bool operator<(const Candidate& o) const {  // heap order: heavier, then lower from, lower to
        if (w != o.w) return w < o.w;
        if (from != o.from) return from > o.from;
        return to > o.to;
    }
};

int match_best_choice(const Hypergraph& g, int max_merges, std::vector<int>& partner, Scratch& s) {
    partner.assign(g.clusters, -1);
    if (max_merges <= 0) return 0;
    std::priority_queue<Candidate> heap;
    for (int c = 0; c < g.clusters; ++c) {
        float w = 0.f;
        const int b = best_neighbour(g, c, s, &w);
        if (b >= 0) heap.push({w, c, b});
    }
    std::vector<int> rescored(g.clusters, 0);
    int merges = 0;
    while (!heap.empty() && merges < max_merges) {
        const Candidate e = heap.top();
        heap.pop();
        if (s.taken[e.from]) continue;
        if (s.taken[e.to]) {
            if (rescored[e.from]++ >= 3) continue;
            float w = 0.f;
            const int b = best_neighbour(g, e.from, s, &w);
            if (b >= 0) heap.push({w, e.from, b});
            continue;
        }
        partner[e.from] = e.to;
        s.taken[e.from] = s.taken[e.to] = 1;
        ++merges;
    }
    return merges;
}

// Nets of degree 2..max_degree over the movable nodes (each node once per net).
Hypergraph level0(const spg_db_view* v, int max_degree) {
    Hypergraph g;
    g.clusters = v->num_movable;
    std::vector<int> seen(v->num_movable, -1), mem;
    for (int k = 0; k < v->num_nets; ++k) {
        const int b = v->net2pin_start[k], e = v->net2pin_start[k + 1];
        if (e - b < 2 || e - b > max_degree) continue;
        mem.clear();
        for (int t = b; t < e; ++t) {
            const int node = v->pin2node[v->flat_net2pin[t]];
            if (node >= v->num_movable || seen[node] == k) continue;
            seen[node] = k;
            mem.push_back(node);
        }
        if (mem.size() < 2) continue;
        g.members.insert(g.members.end(), mem.begin(), mem.end());
        g.net_start.push_back(static_cast<int>(g.members.size()));
    }
    g.index();
    return g;
}

Hypergraph coarsen(const Hypergraph& g, const std::vector<int>& id, int count) {
    Hypergraph h;
    h.clusters = count;
    std::vector<int> seen(count, -1), mem;
    for (int k = 0; k < g.nets(); ++k) {
        mem.clear();
        for (int t = g.net_start[k]; t < g.net_start[k + 1]; ++t) {
            const int c = id[g.members[t]];
            if (seen[c] == k) continue;
            seen[c] = k;
            mem.push_back(c);
        }
        if (mem.size() < 2) continue;
        h.members.insert(h.members.end(), mem.begin(), mem.end());
        h.net_start.push_back(static_cast<int>(h.members.size()));
    }
    h.index();
    return h;
}

void clamp_to_core(const spg_db_view* v, int i, float* x, float* y) {  // PlaceDB::clampToCore
    const float eps = 1e-4f, hw = 0.5f * v->node_w[i], hh = 0.5f * v->node_h[i];
    float px = x[i], py = y[i];
    if (px - hw < v->core_lx) px = v->core_lx + hw + eps;
    if (px + hw > v->core_hx) px = v->core_hx - hw - eps;
    if (py - hh < v->core_ly) py = v->core_ly + hh + eps;
    if (py + hh > v->core_hy) py = v->core_hy - hh - eps;
    x[i] = px;
    y[i] = py;
}

void cluster_place(const spg_db_view* v, bool best_choice, int target, int max_degree, float* x, float* y,
                   int* out_clusters, int* out_levels) {
    const int n = v->num_movable;
    if (n == 0) return;
    if (target <= 0) target = std::max(1, n / 25);
    target = std::min(target, n);
    Hypergraph g = level0(v, max_degree);
    std::vector<int> node_cluster(n);
    for (int i = 0; i < n; ++i) node_cluster[i] = i;
    Scratch s;
    std::vector<int> partner, id;
    int level = 0;
    while (g.clusters > target) {
        s.reset(g.clusters);
        const int want = g.clusters - target;
        const int merges = best_choice ? match_best_choice(g, want, partner, s) : match_first_choice(g, want, partner, s);
        if (merges == 0) break;
        const bool slow = merges * 50 < g.clusters;
        id.assign(g.clusters, -1);
        int count = 0;
        for (int c = 0; c < g.clusters; ++c) {
            if (id[c] >= 0) continue;
            id[c] = count;
            if (partner[c] >= 0) id[partner[c]] = count;
            ++count;
        }
        for (int i = 0; i < n; ++i) node_cluster[i] = id[node_cluster[i]];
        g = coarsen(g, id, count);
        ++level;
        if (slow || level > 128) break;
    }
    const int nc = g.clusters;
    if (out_clusters) *out_clusters = nc;
    if (out_levels) *out_levels = level;

    std::vector<int> first(nc + 1, 0), nodes(n);
    for (int i = 0; i < n; ++i) ++first[node_cluster[i] + 1];
    for (int c = 0; c < nc; ++c) first[c + 1] += first[c];
    {
        std::vector<int> at(first.begin(), first.end() - 1);
        for (int i = 0; i < n; ++i) nodes[at[node_cluster[i]]++] = i;
    }
    std::vector<double> area(nc, 0.0);
    for (int i = 0; i < n; ++i) area[node_cluster[i]] += static_cast<double>(v->node_w[i]) * static_cast<double>(v->node_h[i]);

    // breadth-first order over shared nets
    std::vector<int> order, next;
    std::vector<char> seen(nc, 0);
    order.reserve(nc);
    for (int seed = 0; seed < nc; ++seed) {
        if (seen[seed]) continue;
        std::queue<int> q;
        q.push(seed);
        seen[seed] = 1;
        while (!q.empty()) {
            const int c = q.front();
            q.pop();
            order.push_back(c);
            next.clear();
            for (int t = g.clu_start[c]; t < g.clu_start[c + 1]; ++t) {
                const int k = g.clu_nets[t];
                for (int u = g.net_start[k]; u < g.net_start[k + 1]; ++u) {
                    const int o = g.members[u];
                    if (o != c && !seen[o]) next.push_back(o);
                }
            }
            std::sort(next.begin(), next.end());
            next.erase(std::unique(next.begin(), next.end()), next.end());
            for (int o : next)
                if (!seen[o]) {
                    seen[o] = 1;
                    q.push(o);
                }
        }
    }

    double total = 0.0;
    for (int c : order) total += area[c];
    if (total <= 0.0) total = 1.0;
    const float core_w = v->core_hx - v->core_lx, core_h = v->core_hy - v->core_ly;
    const int shelves = std::max(1, static_cast<int>(std::round(std::sqrt(static_cast<double>(order.size())))));
    const double per_shelf = total / shelves;
    struct Box {
        int c;
        float lx, ly, hx, hy;
    };
    std::vector<Box> boxes;
    boxes.reserve(order.size());
    size_t at = 0;
    float y0 = v->core_ly;
    for (int sh = 0; sh < shelves && at < order.size(); ++sh) {
        const bool last = sh == shelves - 1;
        const size_t from = at;
        double shelf_area = 0.0;
        while (at < order.size() && (last || shelf_area < per_shelf)) shelf_area += area[order[at++]];
        if (shelf_area <= 0.0) shelf_area = 1.0;
        const float h = last ? (v->core_hy - y0) : static_cast<float>(shelf_area / total) * core_h;
        std::vector<size_t> seq;
        for (size_t t = from; t < at; ++t) seq.push_back(t);
        if (sh % 2 == 1) std::reverse(seq.begin(), seq.end());
        float x0 = v->core_lx;
        for (size_t j = 0; j < seq.size(); ++j) {
            const int c = order[seq[j]];
            const float w = j + 1 == seq.size() ? (v->core_hx - x0) : static_cast<float>(area[c] / shelf_area) * core_w;
            boxes.push_back({c, x0, y0, x0 + w, y0 + h});
            x0 += w;
        }
        y0 += h;
    }
    for (const Box& bx : boxes) {
        const int b = first[bx.c], m = first[bx.c + 1] - b;
        if (m == 0) continue;
        const int side = std::max(1, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(m)))));
        const float cw = std::max(1e-3f, (bx.hx - bx.lx) / static_cast<float>(side));
        const float ch = std::max(1e-3f, (bx.hy - bx.ly) / static_cast<float>(side));
        for (int t = 0; t < m; ++t) {
            const int node = nodes[b + t];
            const int gx = t % side, gy = std::min(t / side, side - 1);
            x[node] = bx.lx + (static_cast<float>(gx) + 0.5f) * cw;
            y[node] = bx.ly + (static_cast<float>(gy) + 0.5f) * ch;
            clamp_to_core(v, node, x, y);
        }
    }
}

void check(const spg_db_view* v, const float* x, const float* y) {
    if (!v || !x || !y || v->num_movable < 0 || v->num_nodes < v->num_movable || v->num_nets < 0)
        throw std::invalid_argument("bad argument");
    if (v->num_movable > 0 && (!v->node_w || !v->node_h)) throw std::invalid_argument("spg_db_view without node sizes");
    if (v->num_nets > 0 && (!v->net2pin_start || !v->flat_net2pin || !v->pin2node))
        throw std::invalid_argument("spg_db_view without nets");
}

}  // namespace

extern "C" {

const char* spg_init_last_error(void) { return g_init_error.c_str(); }

int spg_random_place(const spg_db_view* db, uint64_t seed, float* x, float* y) {
    try {
        check(db, x, y);
        std::mt19937 eng(static_cast<std::mt19937::result_type>(seed));
        const float cx = 0.5f * (db->core_lx + db->core_hx), cy = 0.5f * (db->core_ly + db->core_hy);
        for (int i = 0; i < db->num_movable; ++i) {
            const float hw = 0.5f * db->node_w[i], hh = 0.5f * db->node_h[i];
            const float lx = db->core_lx + hw, hx = db->core_hx - hw, ly = db->core_ly + hh, hy = db->core_hy - hh;
            x[i] = hx > lx ? std::uniform_real_distribution<float>(lx, hx)(eng) : cx;
            y[i] = hy > ly ? std::uniform_real_distribution<float>(ly, hy)(eng) : cy;
        }
        return SPG_OK;
    } catch (const std::exception& e) {
        g_init_error = e.what();
        return SPG_E_INVALID;
    }
}

int spg_cluster_place(const spg_db_view* db, int32_t best_choice, int32_t target_count, int32_t ignore_net_degree,
                      float* x, float* y, int32_t* clusters, int32_t* levels) {
    try {
        check(db, x, y);
        cluster_place(db, best_choice != 0, target_count, ignore_net_degree, x, y, clusters, levels);
        return SPG_OK;
    } catch (const std::exception& e) {
        g_init_error = e.what();
        return SPG_E_INVALID;
    }
}

}  // extern "C"
