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
#include <exception>
#include <filesystem>
#include <map>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <string_view>
#include <thread>
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
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open: " + path);
    std::string text;
    if (std::fseek(f, 0, SEEK_END) == 0) {
        const long n = std::ftell(f);
        if (n > 0) text.resize(static_cast<size_t>(n));
        std::fseek(f, 0, SEEK_SET);
    }
    text.resize(text.empty() ? 0 : std::fread(text.data(), 1, text.size(), f));
    char buf[1 << 16];
    for (size_t k; (k = std::fread(buf, 1, sizeof buf, f)) > 0;) text.append(buf, k);  // unsized files
    std::fclose(f);
    return text;
}

bool blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// Calls fn(tokens) for every line that is not empty, a '#' comment or a "UCLA " header.
template <typename F>
void for_each_line(std::string_view text, F&& fn) {
    std::vector<std::string_view> tok;
    size_t pos = 0;
    const size_t n = text.size();
    while (pos < n) {
        size_t end = text.find('\n', pos);
        if (end == std::string_view::npos) end = n;
        std::string_view line = text.substr(pos, end - pos);
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

// ------------------------------------------------------------------ parallel pieces
// Large files are parsed in line-aligned pieces on several threads; each piece's results are
// joined in file order, so the arrays and the first error reported are those of one pass.
constexpr size_t kPieceBytes = size_t(1) << 20;

int piece_count(size_t bytes) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return static_cast<int>(std::max<size_t>(1, std::min<size_t>({bytes / kPieceBytes, hw, 32})));
}

// The first token of `line` (a view into a larger text, starting at a line start).
std::string_view first_token(std::string_view text, size_t pos) {
    while (pos < text.size() && blank(text[pos])) ++pos;
    size_t e = pos;
    while (e < text.size() && !blank(text[e]) && text[e] != '\n') ++e;
    return text.substr(pos, e - pos);
}

// `parts` pieces covering `text`; every piece after the first starts at a line start (at or
// after an even split point) whose first token satisfies `opens` (any line when null).
std::vector<std::string_view> split_pieces(std::string_view text, int parts, bool (*opens)(std::string_view)) {
    std::vector<size_t> cut{0};
    const size_t n = text.size();
    for (int k = 1; k < parts; ++k) {
        size_t pos = std::max(cut.back(), n / static_cast<size_t>(parts) * static_cast<size_t>(k));
        while (pos < n) {
            if (pos > 0 && text[pos - 1] != '\n') {
                const size_t nl = text.find('\n', pos);
                pos = nl == std::string_view::npos ? n : nl + 1;
                continue;
            }
            if (!opens || opens(first_token(text, pos))) break;
            const size_t nl = text.find('\n', pos);
            pos = nl == std::string_view::npos ? n : nl + 1;
        }
        if (pos >= n) break;
        if (pos > cut.back()) cut.push_back(pos);
    }
    cut.push_back(n);
    std::vector<std::string_view> out;
    for (size_t k = 0; k + 1 < cut.size(); ++k) out.push_back(text.substr(cut[k], cut[k + 1] - cut[k]));
    return out;
}

// Runs fn(k) for k in [0, count) on `count` threads and rethrows the lowest k's exception.
template <typename F>
void run_pieces(int count, F&& fn) {
    std::vector<std::exception_ptr> err(static_cast<size_t>(count));
    auto body = [&](int k) {
        try {
            fn(k);
        } catch (...) {
            err[static_cast<size_t>(k)] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    for (int k = 1; k < count; ++k) pool.emplace_back(body, k);
    body(0);
    for (std::thread& t : pool) t.join();
    for (const std::exception_ptr& e : err)
        if (e) std::rethrow_exception(e);
}

// ------------------------------------------------------------------ name index
// Open-addressing table from a name to the FIRST index that carries it (the reference's
// unordered_map::emplace keeps the first). Slots hold 32 bits of the hash beside the index so
// that most probes compare no string.
class NameIndex {
public:
    explicit NameIndex(const std::vector<std::string>& names) : names_(names) {
        size_t cap = 16;
        while (cap < names.size() * 2) cap <<= 1;
        slots_.assign(cap, 0);
        mask_ = cap - 1;
        for (size_t i = 0; i < names.size(); ++i) {
            const uint64_t h = hash(names[i]);
            size_t s = h & mask_;
            for (;; s = (s + 1) & mask_) {
                const uint64_t v = slots_[s];
                if (v == 0) {
                    slots_[s] = (h >> 32 << 32) | (static_cast<uint64_t>(i) + 1);
                    break;
                }
                if ((v >> 32) == (h >> 32) && names_[(v & 0xffffffffu) - 1] == names[i]) break;  // duplicate
            }
        }
    }
    int32_t find(std::string_view name) const {
        const uint64_t h = hash(name);
        for (size_t s = h & mask_;; s = (s + 1) & mask_) {
            const uint64_t v = slots_[s];
            if (v == 0) return -1;
            if ((v >> 32) == (h >> 32)) {
                const int32_t i = static_cast<int32_t>((v & 0xffffffffu) - 1);
                if (names_[static_cast<size_t>(i)] == name) return i;
            }
        }
    }

private:
    // 8 bytes per multiply-xorshift round, then a final avalanche (a splitmix64-style mixer)
    static uint64_t hash(std::string_view s) {
        uint64_t h = 0x9e3779b97f4a7c15ull ^ (s.size() * 0xff51afd7ed558ccdull);
        size_t i = 0;
        for (; i + 8 <= s.size(); i += 8) {
            uint64_t w;
            std::memcpy(&w, s.data() + i, 8);
            h = (h ^ w) * 0xbf58476d1ce4e5b9ull;
            h ^= h >> 31;
        }
        uint64_t w = 0;
        std::memcpy(&w, s.data() + i, s.size() - i);
        h = (h ^ w) * 0x94d049bb133111ebull;
        h ^= h >> 29;
        h *= 0xbf58476d1ce4e5b9ull;
        return h ^ (h >> 32);
    }
    const std::vector<std::string>& names_;
    std::vector<uint64_t> slots_;
    size_t mask_ = 0;
};

// ------------------------------------------------------------------ numbers
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

void read_scl(const std::string& text, const std::string& path, BookshelfDb& db) {
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
    for_each_line(text, [&](const std::vector<std::string_view>& tok) {
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

void read_nodes(const std::string& text, BookshelfDb& db) {
    struct Part {
        std::vector<std::string> name;
        std::vector<float> w, h;
        std::vector<uint8_t> flags;
    };
    const std::vector<std::string_view> pieces = split_pieces(text, piece_count(text.size()), nullptr);
    std::vector<Part> parts(pieces.size());
    run_pieces(static_cast<int>(pieces.size()), [&](int k) {
        Part& p = parts[static_cast<size_t>(k)];
        for_each_line(pieces[static_cast<size_t>(k)], [&](const std::vector<std::string_view>& tok) {
            if (tok[0] == "NumNodes" || tok[0] == "NumTerminals") return check_declared(tok);
            if (tok.size() < 3) return;
            uint8_t f = 0;
            if (tok.size() >= 4) {
                if (tok[3] == "terminal") f = SPG_F_FIXED;
                else if (tok[3] == "terminal_NI") f = SPG_F_FIXED | SPG_F_NI;
            }
            p.name.emplace_back(tok[0]);
            p.w.push_back(parse_float(tok[1]));
            p.h.push_back(parse_float(tok[2]));
            p.flags.push_back(f);
        });
    });
    for (Part& p : parts) {
        db.node_name.insert(db.node_name.end(), std::make_move_iterator(p.name.begin()),
                            std::make_move_iterator(p.name.end()));
        db.w.insert(db.w.end(), p.w.begin(), p.w.end());
        db.h.insert(db.h.end(), p.h.begin(), p.h.end());
        db.flags.insert(db.flags.end(), p.flags.begin(), p.flags.end());
    }
    const size_t n = db.node_name.size();
    db.x.assign(n, 0.f);
    db.y.assign(n, 0.f);
    db.orient.assign(n, 0);
}

bool opens_net(std::string_view first) { return first == "NetDegree"; }

// Pieces of a .nets file start at NetDegree lines, so every piece holds whole nets; a piece's
// nets are numbered locally and shifted when the pieces are joined.
void read_nets(const std::string& text, const NameIndex& index, BookshelfDb& db) {
    struct Part {
        std::vector<int32_t> pin2node, pin_net;
        std::vector<float> ox, oy;
        std::vector<std::string> name;  // empty: unnamed, "n<global index>"
    };
    const std::vector<std::string_view> pieces = split_pieces(text, piece_count(text.size()), opens_net);
    std::vector<Part> parts(pieces.size());
    run_pieces(static_cast<int>(pieces.size()), [&](int k) {
        Part& p = parts[static_cast<size_t>(k)];
        int remaining = 0;
        for_each_line(pieces[static_cast<size_t>(k)], [&](const std::vector<std::string_view>& tok) {
            if (tok[0] == "NumNets" || tok[0] == "NumPins") return check_declared(tok);
            if (tok[0] == "NetDegree") {
                std::string_view v;
                if (!value_after_colon(tok, 0, v)) throw std::runtime_error("malformed NetDegree line");
                remaining = parse_int(v);
                std::string name;
                for (size_t i = 0; i + 2 < tok.size(); ++i)
                    if (tok[i] == ":") {
                        name = std::string(tok[i + 2]);
                        break;
                    }
                p.name.push_back(std::move(name));
                return;
            }
            if (p.name.empty() || remaining <= 0) return;
            const int32_t node = index.find(tok[0]);
            if (node < 0) throw std::runtime_error("net references unknown node: " + std::string(tok[0]));
            float px = 0.f, py = 0.f;
            for (size_t i = 1; i < tok.size(); ++i)
                if (tok[i] == ":") {
                    if (i + 2 < tok.size()) {
                        px = parse_float(tok[i + 1]);
                        py = parse_float(tok[i + 2]);
                    }
                    break;
                }
            p.pin2node.push_back(node);
            p.ox.push_back(px);
            p.oy.push_back(py);
            p.pin_net.push_back(static_cast<int32_t>(p.name.size() - 1));
            --remaining;
        });
    });
    for (Part& p : parts) {
        const int32_t base = static_cast<int32_t>(db.net_name.size());
        for (size_t k = 0; k < p.name.size(); ++k)
            db.net_name.push_back(p.name[k].empty() ? "n" + std::to_string(base + static_cast<int32_t>(k))
                                                    : std::move(p.name[k]));
        db.pin2node.insert(db.pin2node.end(), p.pin2node.begin(), p.pin2node.end());
        db.ox.insert(db.ox.end(), p.ox.begin(), p.ox.end());
        db.oy.insert(db.oy.end(), p.oy.begin(), p.oy.end());
        for (int32_t v : p.pin_net) db.pin_net.push_back(v + base);
    }
}

// .pl lines are parsed in pieces into records and applied in file order (a later line for the
// same node wins, as in one pass).
void read_pl(const std::string& text, const NameIndex& index, BookshelfDb& db) {
    struct Rec {
        int32_t node;
        float llx, lly;
        int8_t orient;  // -1: the line sets none
        uint8_t fixed;
    };
    const std::vector<std::string_view> pieces = split_pieces(text, piece_count(text.size()), nullptr);
    std::vector<std::vector<Rec>> parts(pieces.size());
    run_pieces(static_cast<int>(pieces.size()), [&](int k) {
        std::vector<Rec>& out = parts[static_cast<size_t>(k)];
        for_each_line(pieces[static_cast<size_t>(k)], [&](const std::vector<std::string_view>& tok) {
            if (tok.size() < 3) return;
            const int32_t i = index.find(tok[0]);
            if (i < 0) return;
            Rec r{i, parse_float(tok[1]), parse_float(tok[2]), -1, 0};
            for (size_t k2 = 3; k2 < tok.size(); ++k2) {
                if (tok[k2] == ":") {
                    if (k2 + 1 < tok.size()) r.orient = static_cast<int8_t>(orient_code(tok[k2 + 1]));
                } else if (tok[k2].find("FIXED") != std::string_view::npos) {
                    r.fixed = 1;
                }
            }
            out.push_back(r);
        });
    });
    for (const std::vector<Rec>& part : parts)
        for (const Rec& r : part) {
            db.x[r.node] = r.llx + 0.5f * db.w[r.node];
            db.y[r.node] = r.lly + 0.5f * db.h[r.node];
            if (r.orient >= 0) db.orient[r.node] = static_cast<uint8_t>(r.orient);
            if (r.fixed) db.flags[r.node] |= SPG_F_FIXED;
        }
}

void read_wts(const std::string& text, BookshelfDb& db) {
    db.net_weight.assign(db.net_name.size(), 1.f);
    if (text.empty()) return;
    const NameIndex index(db.net_name);
    for_each_line(text, [&](const std::vector<std::string_view>& tok) {
        if (tok.size() < 2) return;
        const int32_t k = index.find(tok[0]);
        if (k >= 0) db.net_weight[static_cast<size_t>(k)] = parse_float(tok[1]);
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

// One .pl line, "%s\t%.6f\t%.6f\t: %s%s\n" of BookshelfWriter::writePl; std::to_chars with a
// precision prints what printf prints for the same conversion.
void pl_line(std::string& out, const char* name, double llx, double lly, const char* orient, bool fixed) {
    char num[400];
    out += name;
    for (double v : {llx, lly}) {
        out += '\t';
        const auto r = std::to_chars(num, num + sizeof num, v, std::chars_format::fixed, 6);
        out.append(num, r.ptr);
    }
    out += "\t: ";
    out += orient;
    if (fixed) out += " /FIXED";
    out += '\n';
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
        BookshelfDb& db = b->db;
        const Files f = read_aux(aux_path);
        // The files are loaded on a second thread while the earlier ones parse; a load error
        // surfaces when its file's turn comes, so the error reported is that of one pass.
        struct Loaded {
            std::string text;
            std::exception_ptr err;
        };
        Loaded nodes, nets, pl, wts;
        auto load = [](const std::string& path, Loaded& out) {
            try {
                out.text = slurp(path);
            } catch (...) {
                out.err = std::current_exception();
            }
        };
        std::thread loader([&] {
            load(f.nodes, nodes);
            load(f.nets, nets);
            load(f.pl, pl);
            std::error_code ec;
            if (!f.wts.empty() && std::filesystem::exists(f.wts, ec)) load(f.wts, wts);  // none: unit weights
        });
        auto take = [&](Loaded& l) -> const std::string& {
            if (l.err) std::rethrow_exception(l.err);
            return l.text;
        };
        try {
            read_scl(slurp(f.scl), f.scl, db);
            loader.join();
        } catch (...) {
            loader.join();
            throw;
        }
        read_nodes(take(nodes), db);
        const NameIndex index(db.node_name);
        read_nets(take(nets), index, db);
        read_pl(take(pl), index, db);
        read_wts(take(wts), db);
        finish(db);
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

int spg_bookshelf_apply_pl(const char* path, int32_t num_nodes, const char* names, const float* w, const float* h,
                           float* x, float* y, uint8_t* flags, uint8_t* orient) {
    try {
        if (!path || num_nodes < 0 || (num_nodes > 0 && (!names || !w || !h || !x || !y || !flags || !orient)))
            throw std::invalid_argument("null argument");
        BookshelfDb db;
        const char* name = names;
        for (int32_t i = 0; i < num_nodes; ++i) {
            db.node_name.emplace_back(name);
            name += db.node_name.back().size() + 1;
        }
        const size_t n = static_cast<size_t>(num_nodes);
        db.w.assign(w, w + n);
        db.h.assign(h, h + n);
        db.x.assign(x, x + n);
        db.y.assign(y, y + n);
        db.flags.assign(flags, flags + n);
        db.orient.assign(orient, orient + n);
        read_pl(slurp(path), NameIndex(db.node_name), db);
        std::copy(db.x.begin(), db.x.end(), x);
        std::copy(db.y.begin(), db.y.end(), y);
        std::copy(db.flags.begin(), db.flags.end(), flags);
        std::copy(db.orient.begin(), db.orient.end(), orient);
        return SPG_OK;
    } catch (const std::exception& e) {
        return bs_fail(e);
    }
}

int spg_bookshelf_write_pl(const char* path, int32_t num_nodes, const char* names, const float* x, const float* y,
                           const float* w, const float* h, const uint8_t* flags, const uint8_t* orient) {
    try {
        if (!path || num_nodes < 0 || (num_nodes > 0 && (!names || !x || !y || !w || !h || !flags)))
            throw std::invalid_argument("null argument");
        std::vector<const char*> name(static_cast<size_t>(num_nodes));
        size_t bytes = 0;
        for (int32_t i = 0; i < num_nodes; ++i) {
            name[static_cast<size_t>(i)] = names + bytes;
            bytes += std::strlen(names + bytes) + 1;
        }
        // node ranges formatted on several threads, written in node order
        const int parts = piece_count(static_cast<size_t>(num_nodes) * 48);
        std::vector<std::string> text(static_cast<size_t>(parts));
        run_pieces(parts, [&](int k) {
            const int32_t a = static_cast<int32_t>(int64_t(num_nodes) * k / parts);
            const int32_t b = static_cast<int32_t>(int64_t(num_nodes) * (k + 1) / parts);
            std::string& out = text[static_cast<size_t>(k)];
            out.reserve(static_cast<size_t>(b - a) * 48);
            for (int32_t i = a; i < b; ++i) {
                const double llx = static_cast<double>(x[i]) - 0.5 * w[i];
                const double lly = static_cast<double>(y[i]) - 0.5 * h[i];
                const uint8_t o = orient && orient[i] < 8 ? orient[i] : 0;
                pl_line(out, name[static_cast<size_t>(i)], llx, lly, kOrient[o], (flags[i] & SPG_F_FIXED) != 0);
            }
        });
        std::FILE* f = std::fopen(path, "wb");
        if (!f) throw std::runtime_error(std::string("cannot write: ") + path);
        static const char kHead[] = "UCLA pl 1.0\n# Generated by superPlace\n\n";
        bool ok = std::fwrite(kHead, 1, sizeof kHead - 1, f) == sizeof kHead - 1;
        for (const std::string& t : text) ok = ok && std::fwrite(t.data(), 1, t.size(), f) == t.size();
        if (std::fclose(f) != 0 || !ok) throw std::runtime_error(std::string("write failed: ") + path);
        return SPG_OK;
    } catch (const std::exception& e) {
        return bs_fail(e);
    }
}

}  // extern "C"
