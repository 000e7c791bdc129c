// BookShelf placement files <-> the PlaceDB layout, on the host (no device code).
//
// Reading follows BookshelfReader::read (src/io/bookshelf_reader.cpp:433-463):
//   .aux   the file names, recognised by extension
//   .scl   CoreRow ... End blocks: Coordinate (row bottom), Height, Sitewidth, Sitespacing
//          (the site step is the spacing when positive, else the width), SubrowOrigin and
//          NumSites (on the same line); a last block without End still counts
//   .nodes name w h [terminal | terminal_NI] (fixed, fixed + not-in-image)
//   .nets  NetDegree : d [name] then d pin lines "node [dir] : ox oy" (offsets from the centre)
//   .pl    name llx lly [: orient] [/FIXED]: centre = lower-left + half size; /FIXED fixes
//   .wts   "net weight" lines (weights default to 1)
// then marks macros (movable and taller than 1.5 row heights), reorders the nodes stably to
// [movable | fixed] and builds the two CSR directions by counting (pins in ascending order).
// Lines are split on '\n'; ' ', '\t' and '\r' separate tokens; empty lines, '#' comments and
// "UCLA ..." headers are skipped. Numbers are parsed with std::from_chars (floats rounded once
// to float; an integer field written as "12.000000" is read through a double and truncated).
//
// Writing a .pl follows BookshelfWriter::writePl (src/io/bookshelf_writer.cpp:16-37): node
// order, lower-left corners as "%.6f" of the double centre minus half the size, the
// orientation after ':' and " /FIXED" for fixed nodes.
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "spgpu.h"

namespace {

thread_local std::string g_bs_error;

struct BookshelfDb {
    // nodes in file order until finish(), then in [movable | fixed] order
    std::vector<std::string> node_name;
    std::vector<float> x, y, w, h;
    std::vector<uint8_t> flags, orient;
    int num_movable = 0;
    // pins in file order; pin_net in file order
    std::vector<float> ox, oy;
    std::vector<int32_t> pin2node, pin_net;
    std::vector<int32_t> net2pin_start, flat_net2pin, node2pin_start, flat_node2pin;
    std::vector<std::string> net_name;
    std::vector<float> net_weight;
    // rows
    std::vector<float> row_ly, row_height, row_lx, row_step;
    std::vector<int32_t> row_sites;
};

std::string slurp(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open: " + path);
    return std::string(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
}

bool blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Calls fn(tokens) for every line that is not empty, a '#' comment or a "UCLA " header.
template <typename F>
void for_each_line(const std::string& text, F&& fn) {
    std::vector<std::string_view> tok;
    size_t pos = 0;
    const size_t n = text.size();
    while (pos < n) {
        size_t end = text.find('\n', pos);
        if (end == std::string::npos) end = n;
        std::string_view line(text.data() + pos, end - pos);
        pos = end + 1;
        while (!line.empty() && blank(line.back())) line.remove_suffix(1);  // trailing blanks
        size_t a = 0;
        while (a < line.size() && blank(line[a])) ++a;
        if (a == line.size() || line[a] == '#' || line.substr(a, 5) == "UCLA ") continue;
        tok.clear();
        size_t i = a;
        while (i < line.size()) {
            while (i < line.size() && blank(line[i])) ++i;
            if (i == line.size()) break;
            const size_t b = i;
            while (i < line.size() && !blank(line[i])) ++i;
            tok.push_back(line.substr(b, i - b));
        }
        if (!tok.empty()) fn(tok);
    }
}

float parse_float(std::string_view s) {
    float v = 0.f;
    const auto r = std::from_chars(s.data(), s.data() + s.size(), v);
    if (r.ec != std::errc()) throw std::runtime_error("bad float: " + std::string(s));
    return v;
}

int parse_int(std::string_view s) {
    int v = 0;
    if (std::from_chars(s.data(), s.data() + s.size(), v).ec == std::errc()) return v;
    double d = 0.0;  // "12.000000"
    if (std::from_chars(s.data(), s.data() + s.size(), d).ec != std::errc())
        throw std::runtime_error("bad integer: " + std::string(s));
    return static_cast<int>(d);
}

// The value of "Key : value" (or "Key:value", "Key :value") starting at token `from`.
bool value_after_colon(const std::vector<std::string_view>& tok, size_t from, std::string_view& out) {
    for (size_t i = from; i + 1 < tok.size(); ++i) {
        if (tok[i] == ":") {
            out = tok[i + 1];
            return true;
        }
        const size_t c = tok[i].find(':');
        if (c != std::string_view::npos && c + 1 < tok[i].size()) {
            out = tok[i].substr(c + 1);
            return true;
        }
    }
    return false;
}

// A "NumNodes : n"-style count: only its syntax is checked (a bad integer is an error); the
// arrays are sized by what the file lists.
void check_declared(const std::vector<std::string_view>& tok) {
    std::string_view v;
    if (value_after_colon(tok, 0, v)) parse_int(v);
}

const char* const kOrient[8] = {"N", "E", "S", "W", "FN", "FE", "FS", "FW"};

uint8_t orient_code(std::string_view s) {
    for (uint8_t i = 0; i < 8; ++i)
        if (s == kOrient[i]) return i;
    return 0;
}

std::string dir_of(const std::string& p) {
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string(".") : (s == 0 ? std::string("/") : p.substr(0, s));
}

std::string ext_of(std::string_view name) {
    const size_t slash = name.find_last_of('/');
    const std::string_view base = slash == std::string_view::npos ? name : name.substr(slash + 1);
    const size_t dot = base.find_last_of('.');
    if (dot == std::string_view::npos || dot == 0) return std::string();
    return std::string(base.substr(dot));
}

struct Files {
    std::string nodes, nets, wts, pl, scl;
};

Files read_aux(const std::string& aux) {
    Files f;
    const std::string dir = dir_of(aux);
    for_each_line(slurp(aux), [&](const std::vector<std::string_view>& tok) {
        for (std::string_view t : tok) {
            if (t == ":" || t.find('.') == std::string_view::npos) continue;
            const std::string full = t[0] == '/' ? std::string(t)
                                     : dir.back() == '/' ? dir + std::string(t) : dir + "/" + std::string(t);
            const std::string e = ext_of(t);
            if (e == ".nodes") f.nodes = full;
            else if (e == ".nets") f.nets = full;
            else if (e == ".wts") f.wts = full;
            else if (e == ".pl") f.pl = full;
            else if (e == ".scl") f.scl = full;
        }
    });
    if (f.nodes.empty() || f.nets.empty() || f.pl.empty() || f.scl.empty())
        throw std::runtime_error("aux file missing required entries: " + aux);
    return f;
}

void read_scl(const std::string& path, BookshelfDb& db) {
    bool open = false;
    float ly = 0.f, height = 0.f, lx = 0.f, site_w = 1.f, site_sp = 0.f;
    int sites = 0;
    auto close_row = [&]() {
        db.row_ly.push_back(ly);
        db.row_height.push_back(height);
        db.row_lx.push_back(lx);
        db.row_step.push_back(site_sp > 0.f ? site_sp : site_w);
        db.row_sites.push_back(sites);
    };
    for_each_line(slurp(path), [&](const std::vector<std::string_view>& tok) {
        const std::string_view key = tok[0];
        if (key == "CoreRow") {
            open = true;
            ly = height = lx = 0.f;
            site_w = 1.f;
            site_sp = 0.f;
            sites = 0;
            return;
        }
        if (key == "End") {
            if (open) close_row();
            open = false;
            return;
        }
        if (!open) return;
        std::string_view v;
        if (key == "Coordinate") {
            if (value_after_colon(tok, 0, v)) ly = parse_float(v);
        } else if (key == "Height") {
            if (value_after_colon(tok, 0, v)) height = parse_float(v);
        } else if (key == "Sitewidth") {
            if (value_after_colon(tok, 0, v)) site_w = parse_float(v);
        } else if (key == "Sitespacing") {
            if (value_after_colon(tok, 0, v)) site_sp = parse_float(v);
        } else if (key == "SubrowOrigin") {
            if (value_after_colon(tok, 0, v)) lx = parse_float(v);
            for (size_t i = 1; i < tok.size(); ++i)
                if (tok[i].substr(0, 8) == "NumSites") {
                    if (value_after_colon(tok, i, v)) sites = parse_int(v);
                    break;
                }
        }
    });
    if (open) close_row();
    if (db.row_ly.empty()) throw std::runtime_error("no CoreRow found in " + path);
}

float mode_row_height(const BookshelfDb& db) {
    std::map<float, int> count;  // ascending heights: the smallest wins a tie
    for (float h : db.row_height) ++count[h];
    float best_h = 0.f;
    int best = -1;
    for (const auto& [h, c] : count)
        if (c > best) {
            best = c;
            best_h = h;
        }
    return best_h;
}

void read_nodes(const std::string& path, BookshelfDb& db) {
    for_each_line(slurp(path), [&](const std::vector<std::string_view>& tok) {
        if (tok[0] == "NumNodes" || tok[0] == "NumTerminals") return check_declared(tok);
        if (tok.size() < 3) return;
        uint8_t f = 0;
        if (tok.size() >= 4) {
            if (tok[3] == "terminal") f = SPG_F_FIXED;
            else if (tok[3] == "terminal_NI") f = SPG_F_FIXED | SPG_F_NI;
        }
        db.node_name.emplace_back(tok[0]);
        db.w.push_back(parse_float(tok[1]));
        db.h.push_back(parse_float(tok[2]));
        db.flags.push_back(f);
    });
    const size_t n = db.node_name.size();
    db.x.assign(n, 0.f);
    db.y.assign(n, 0.f);
    db.orient.assign(n, 0);
}

void read_nets(const std::string& path, BookshelfDb& db) {
    std::unordered_map<std::string_view, int32_t> index;
    index.reserve(db.node_name.size() * 2);
    for (size_t i = 0; i < db.node_name.size(); ++i) index.emplace(db.node_name[i], static_cast<int32_t>(i));
    int remaining = 0;
    for_each_line(slurp(path), [&](const std::vector<std::string_view>& tok) {
        if (tok[0] == "NumNets" || tok[0] == "NumPins") return check_declared(tok);
        if (tok[0] == "NetDegree") {
            std::string_view v;
            if (!value_after_colon(tok, 0, v)) throw std::runtime_error("malformed NetDegree line");
            remaining = parse_int(v);
            std::string name = "n" + std::to_string(db.net_name.size());
            for (size_t i = 0; i + 2 < tok.size(); ++i)
                if (tok[i] == ":") {
                    name = std::string(tok[i + 2]);
                    break;
                }
            db.net_name.push_back(std::move(name));
            return;
        }
        if (db.net_name.empty() || remaining <= 0) return;
        const auto it = index.find(tok[0]);
        if (it == index.end()) throw std::runtime_error("net references unknown node: " + std::string(tok[0]));
        float px = 0.f, py = 0.f;
        for (size_t i = 1; i < tok.size(); ++i)
            if (tok[i] == ":") {
                if (i + 2 < tok.size()) {
                    px = parse_float(tok[i + 1]);
                    py = parse_float(tok[i + 2]);
                }
                break;
            }
        db.pin2node.push_back(it->second);
        db.ox.push_back(px);
        db.oy.push_back(py);
        db.pin_net.push_back(static_cast<int32_t>(db.net_name.size() - 1));
        --remaining;
    });
}

void read_pl(const std::string& path, BookshelfDb& db) {
    std::unordered_map<std::string_view, int32_t> index;
    index.reserve(db.node_name.size() * 2);
    for (size_t i = 0; i < db.node_name.size(); ++i) index.emplace(db.node_name[i], static_cast<int32_t>(i));
    for_each_line(slurp(path), [&](const std::vector<std::string_view>& tok) {
        if (tok.size() < 3) return;
        const auto it = index.find(tok[0]);
        if (it == index.end()) return;
        const int32_t i = it->second;
        db.x[i] = parse_float(tok[1]) + 0.5f * db.w[i];
        db.y[i] = parse_float(tok[2]) + 0.5f * db.h[i];
        for (size_t k = 3; k < tok.size(); ++k) {
            if (tok[k] == ":") {
                if (k + 1 < tok.size()) db.orient[i] = orient_code(tok[k + 1]);
            } else if (tok[k].find("FIXED") != std::string_view::npos) {
                db.flags[i] |= SPG_F_FIXED;
            }
        }
    });
}

void read_wts(const std::string& path, BookshelfDb& db) {
    db.net_weight.assign(db.net_name.size(), 1.f);
    if (path.empty()) return;
    std::ifstream probe(path);
    if (!probe) return;  // a missing .wts means unit weights
    std::unordered_map<std::string_view, int32_t> index;
    index.reserve(db.net_name.size() * 2);
    for (size_t k = 0; k < db.net_name.size(); ++k) index.emplace(db.net_name[k], static_cast<int32_t>(k));
    for_each_line(slurp(path), [&](const std::vector<std::string_view>& tok) {
        if (tok.size() < 2) return;
        const auto it = index.find(tok[0]);
        if (it != index.end()) db.net_weight[it->second] = parse_float(tok[1]);
    });
}

template <typename T>
void reorder(std::vector<T>& v, const std::vector<int32_t>& order) {
    std::vector<T> out;
    out.reserve(v.size());
    for (int32_t i : order) out.push_back(std::move(v[i]));
    v.swap(out);
}

// [movable | fixed] in file order within each segment, pins renumbered; then the two CSR
// directions by counting (each net's and each node's pins in ascending pin order).
void finish(BookshelfDb& db) {
    const float rh = mode_row_height(db);
    const int32_t n = static_cast<int32_t>(db.node_name.size());
    for (int32_t i = 0; i < n; ++i)
        if (!(db.flags[i] & SPG_F_FIXED) && db.h[i] > rh * 1.5f) db.flags[i] |= SPG_F_MACRO;
    std::vector<int32_t> order;
    order.reserve(n);
    for (int32_t i = 0; i < n; ++i)
        if (!(db.flags[i] & SPG_F_FIXED)) order.push_back(i);
    db.num_movable = static_cast<int>(order.size());
    for (int32_t i = 0; i < n; ++i)
        if (db.flags[i] & SPG_F_FIXED) order.push_back(i);
    std::vector<int32_t> new_index(n);
    for (int32_t k = 0; k < n; ++k) new_index[order[k]] = k;
    reorder(db.node_name, order);
    reorder(db.x, order);
    reorder(db.y, order);
    reorder(db.w, order);
    reorder(db.h, order);
    reorder(db.flags, order);
    reorder(db.orient, order);
    for (int32_t& v : db.pin2node) v = new_index[v];

    const int32_t pins = static_cast<int32_t>(db.pin2node.size());
    const int32_t nets = static_cast<int32_t>(db.net_name.size());
    auto csr = [pins](const std::vector<int32_t>& owner, int32_t m, std::vector<int32_t>& start,
                      std::vector<int32_t>& flat) {
        start.assign(static_cast<size_t>(m) + 1, 0);
        for (int32_t p = 0; p < pins; ++p) ++start[owner[p] + 1];
        std::partial_sum(start.begin(), start.end(), start.begin());
        flat.assign(pins, 0);
        std::vector<int32_t> next(start.begin(), start.end() - 1);
        for (int32_t p = 0; p < pins; ++p) flat[next[owner[p]]++] = p;
    };
    csr(db.pin_net, nets, db.net2pin_start, db.flat_net2pin);
    csr(db.pin2node, n, db.node2pin_start, db.flat_node2pin);
}

int bs_fail(const std::exception& e) {
    g_bs_error = e.what();
    return SPG_E_INVALID;
}

void copy_names(const std::vector<std::string>& names, char* out) {
    for (const std::string& s : names) {
        std::memcpy(out, s.c_str(), s.size() + 1);
        out += s.size() + 1;
    }
}

int64_t names_bytes(const std::vector<std::string>& names) {
    int64_t b = 0;
    for (const std::string& s : names) b += static_cast<int64_t>(s.size()) + 1;
    return b;
}

}  // namespace

struct spg_bookshelf {
    BookshelfDb db;
};

extern "C" {

const char* spg_bookshelf_last_error(void) { return g_bs_error.c_str(); }

int spg_bookshelf_read(const char* aux_path, spg_bookshelf** out) {
    try {
        if (!aux_path || !out) throw std::invalid_argument("null argument");
        auto b = std::make_unique<spg_bookshelf>();
        const Files f = read_aux(aux_path);
        read_scl(f.scl, b->db);
        read_nodes(f.nodes, b->db);
        read_nets(f.nets, b->db);
        read_pl(f.pl, b->db);
        read_wts(f.wts, b->db);
        finish(b->db);
        *out = b.release();
        return SPG_OK;
    } catch (const std::exception& e) {
        return bs_fail(e);
    }
}

int spg_bookshelf_counts(const spg_bookshelf* b, int64_t* counts) {
    if (!b || !counts) return SPG_E_INVALID;
    const BookshelfDb& d = b->db;
    counts[0] = d.num_movable;
    counts[1] = static_cast<int64_t>(d.node_name.size());
    counts[2] = static_cast<int64_t>(d.pin2node.size());
    counts[3] = static_cast<int64_t>(d.net_name.size());
    counts[4] = static_cast<int64_t>(d.row_ly.size());
    counts[5] = names_bytes(d.node_name);
    counts[6] = names_bytes(d.net_name);
    return SPG_OK;
}

int spg_bookshelf_nodes(const spg_bookshelf* b, float* x, float* y, float* w, float* h, uint8_t* flags,
                        uint8_t* orient, char* names) {
    if (!b) return SPG_E_INVALID;
    const BookshelfDb& d = b->db;
    const size_t n = d.node_name.size();
    if (x) std::memcpy(x, d.x.data(), n * sizeof(float));
    if (y) std::memcpy(y, d.y.data(), n * sizeof(float));
    if (w) std::memcpy(w, d.w.data(), n * sizeof(float));
    if (h) std::memcpy(h, d.h.data(), n * sizeof(float));
    if (flags) std::memcpy(flags, d.flags.data(), n);
    if (orient) std::memcpy(orient, d.orient.data(), n);
    if (names) copy_names(d.node_name, names);
    return SPG_OK;
}

int spg_bookshelf_pins(const spg_bookshelf* b, float* ox, float* oy, int32_t* pin2node, int32_t* pin2net,
                       int32_t* net2pin_start, int32_t* flat_net2pin, int32_t* node2pin_start,
                       int32_t* flat_node2pin) {
    if (!b) return SPG_E_INVALID;
    const BookshelfDb& d = b->db;
    const size_t p = d.pin2node.size();
    if (ox) std::memcpy(ox, d.ox.data(), p * sizeof(float));
    if (oy) std::memcpy(oy, d.oy.data(), p * sizeof(float));
    if (pin2node) std::memcpy(pin2node, d.pin2node.data(), p * sizeof(int32_t));
    if (pin2net) std::memcpy(pin2net, d.pin_net.data(), p * sizeof(int32_t));
    if (net2pin_start) std::memcpy(net2pin_start, d.net2pin_start.data(), d.net2pin_start.size() * sizeof(int32_t));
    if (flat_net2pin) std::memcpy(flat_net2pin, d.flat_net2pin.data(), p * sizeof(int32_t));
    if (node2pin_start) std::memcpy(node2pin_start, d.node2pin_start.data(), d.node2pin_start.size() * sizeof(int32_t));
    if (flat_node2pin) std::memcpy(flat_node2pin, d.flat_node2pin.data(), p * sizeof(int32_t));
    return SPG_OK;
}

int spg_bookshelf_nets(const spg_bookshelf* b, float* weight, char* names) {
    if (!b) return SPG_E_INVALID;
    const BookshelfDb& d = b->db;
    if (weight) std::memcpy(weight, d.net_weight.data(), d.net_weight.size() * sizeof(float));
    if (names) copy_names(d.net_name, names);
    return SPG_OK;
}

int spg_bookshelf_rows(const spg_bookshelf* b, float* ly, float* height, float* lx, float* step, int32_t* sites) {
    if (!b) return SPG_E_INVALID;
    const BookshelfDb& d = b->db;
    const size_t r = d.row_ly.size();
    if (ly) std::memcpy(ly, d.row_ly.data(), r * sizeof(float));
    if (height) std::memcpy(height, d.row_height.data(), r * sizeof(float));
    if (lx) std::memcpy(lx, d.row_lx.data(), r * sizeof(float));
    if (step) std::memcpy(step, d.row_step.data(), r * sizeof(float));
    if (sites) std::memcpy(sites, d.row_sites.data(), r * sizeof(int32_t));
    return SPG_OK;
}

int spg_bookshelf_destroy(spg_bookshelf* b) {
    delete b;
    return SPG_OK;
}

int spg_bookshelf_write_pl(const char* path, int32_t num_nodes, const char* names, const float* x, const float* y,
                           const float* w, const float* h, const uint8_t* flags, const uint8_t* orient) {
    try {
        if (!path || num_nodes < 0 || (num_nodes > 0 && (!names || !x || !y || !w || !h || !flags)))
            throw std::invalid_argument("null argument");
        std::FILE* f = std::fopen(path, "wb");
        if (!f) throw std::runtime_error(std::string("cannot write: ") + path);
        std::fputs("UCLA pl 1.0\n# Generated by superPlace\n\n", f);
        const char* name = names;
        for (int32_t i = 0; i < num_nodes; ++i) {
            const double llx = static_cast<double>(x[i]) - 0.5 * w[i];
            const double lly = static_cast<double>(y[i]) - 0.5 * h[i];
            const uint8_t o = orient && orient[i] < 8 ? orient[i] : 0;
            std::fprintf(f, "%s\t%.6f\t%.6f\t: %s%s\n", name, llx, lly, kOrient[o],
                         (flags[i] & SPG_F_FIXED) ? " /FIXED" : "");
            name += std::strlen(name) + 1;
        }
        if (std::fclose(f) != 0) throw std::runtime_error(std::string("write failed: ") + path);
        return SPG_OK;
    } catch (const std::exception& e) {
        return bs_fail(e);
    }
}

}  // extern "C"
