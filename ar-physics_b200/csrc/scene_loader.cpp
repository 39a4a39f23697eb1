// scene_loader.cpp -- scene files in the reference's TOML schema.
//
// Restates examples/test_mods/config.rs:62-474 (the schema and its defaults),
// src/soft_body/material_region/region.rs:21-272 (AABB, AABE, Transformed,
// Difference, Union, Intersection) and material_region/mod.rs:56-155
// (hex/HCP lattice seeding and the mass rule) on top of a small TOML reader.
// Tables iterate in sorted key order as toml 0.5's BTreeMap does, which fixes
// the material order: boundaries by name, then objects by name.  Arithmetic
// follows the Rust code's f32/f64 choices; this file is compiled without
// floating-point contraction so lattice coordinates accumulate exactly as
// there.  STL regions ("model", examples/test_mods/mesh.rs) are read as
// stl_io 0.4 reads them, from paths relative to the working directory as the
// reference opens them.  "on_click" objects are interactive additions and are
// not part of the initial scene.
#include "scene_loader.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace arp {

// ---- TOML subset -----------------------------------------------------------

struct TVal {
    enum Kind { Str, Int, Float, Bool, Arr, Tab } kind = Tab;
    std::string s;
    double num = 0;
    bool b = false;
    std::vector<TVal> arr;
    std::map<std::string, TVal> tab;
    bool is_num() const { return kind == Int || kind == Float; }
};

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// Valid input that this loader does not implement (ARP_ERR_UNSUPPORTED).
struct Unsupported : ParseError {
    using ParseError::ParseError;
};

class TomlReader {
public:
    explicit TomlReader(const std::string& text) : t_(text) {}

    TVal parse() {
        TVal root;
        TVal* cur = &root;
        for (;;) {
            skip_ws_nl();
            if (p_ >= t_.size()) break;
            if (t_[p_] == '[') {
                ++p_;
                if (p_ < t_.size() && t_[p_] == '[') throw Unsupported(where() + "arrays of tables are not supported");
                std::vector<std::string> path = key_path(']');
                expect(']');
                cur = &root;
                for (const auto& k : path) cur = &table_child(*cur, k);
            } else {
                std::vector<std::string> path = key_path('=');
                expect('=');
                TVal v = value();
                TVal* t = cur;
                for (size_t i = 0; i + 1 < path.size(); ++i) t = &table_child(*t, path[i]);
                if (t->tab.count(path.back())) fail("duplicate key " + path.back());
                t->tab[path.back()] = std::move(v);
            }
            skip_ws();
            if (p_ < t_.size() && t_[p_] == '#') skip_comment();
            if (p_ < t_.size() && t_[p_] != '\n' && t_[p_] != '\r') fail("expected end of line");
        }
        return root;
    }

private:
    const std::string& t_;
    size_t p_ = 0;

    std::string where() const {
        size_t line = 1;
        for (size_t i = 0; i < p_ && i < t_.size(); ++i) line += t_[i] == '\n';
        return "line " + std::to_string(line) + ": ";
    }
    [[noreturn]] void fail(const std::string& m) { throw ParseError(where() + m); }
    void skip_ws() {
        while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\t')) ++p_;
    }
    void skip_comment() {
        while (p_ < t_.size() && t_[p_] != '\n') ++p_;
    }
    void skip_ws_nl() {
        for (;;) {
            while (p_ < t_.size() && std::isspace((unsigned char)t_[p_])) ++p_;
            if (p_ < t_.size() && t_[p_] == '#') {
                skip_comment();
                continue;
            }
            break;
        }
    }
    void expect(char c) {
        skip_ws();
        if (p_ >= t_.size() || t_[p_] != c) fail(std::string("expected '") + c + "'");
        ++p_;
    }
    TVal& table_child(TVal& t, const std::string& k) {
        if (t.kind != TVal::Tab) fail("key " + k + " is not a table");
        TVal& c = t.tab[k];
        return c;
    }
    std::string bare_or_quoted_key() {
        skip_ws();
        if (p_ < t_.size() && t_[p_] == '"') return basic_string();
        size_t b = p_;
        while (p_ < t_.size() && (std::isalnum((unsigned char)t_[p_]) || t_[p_] == '_' || t_[p_] == '-')) ++p_;
        if (b == p_) fail("expected a key");
        return t_.substr(b, p_ - b);
    }
    std::vector<std::string> key_path(char end) {
        std::vector<std::string> path;
        for (;;) {
            path.push_back(bare_or_quoted_key());
            skip_ws();
            if (p_ < t_.size() && t_[p_] == '.') {
                ++p_;
                continue;
            }
            if (p_ < t_.size() && t_[p_] == end) return path;
            fail("unexpected character in key");
        }
    }
    std::string basic_string() {
        ++p_;  // opening quote
        std::string out;
        while (p_ < t_.size() && t_[p_] != '"') {
            char c = t_[p_++];
            if (c == '\\' && p_ < t_.size()) {
                char e = t_[p_++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    default: out += e;
                }
            } else {
                if (c == '\n') fail("newline in string");
                out += c;
            }
        }
        if (p_ >= t_.size()) fail("unterminated string");
        ++p_;
        return out;
    }
    TVal value() {
        skip_ws();
        if (p_ >= t_.size()) fail("expected a value");
        TVal v;
        char c = t_[p_];
        if (c == '"') {
            v.kind = TVal::Str;
            v.s = basic_string();
        } else if (c == '\'') {
            ++p_;
            size_t b = p_;
            while (p_ < t_.size() && t_[p_] != '\'') ++p_;
            if (p_ >= t_.size()) fail("unterminated string");
            v.kind = TVal::Str;
            v.s = t_.substr(b, p_ - b);
            ++p_;
        } else if (c == '[') {
            ++p_;
            v.kind = TVal::Arr;
            for (;;) {
                skip_ws_nl();
                if (p_ < t_.size() && t_[p_] == ']') {
                    ++p_;
                    break;
                }
                v.arr.push_back(value());
                skip_ws_nl();
                if (p_ < t_.size() && t_[p_] == ',') {
                    ++p_;
                    continue;
                }
                skip_ws_nl();
                if (p_ < t_.size() && t_[p_] == ']') {
                    ++p_;
                    break;
                }
                fail("expected ',' or ']' in array");
            }
        } else if (c == '{') {
            ++p_;
            v.kind = TVal::Tab;
            skip_ws();
            if (p_ < t_.size() && t_[p_] == '}') {
                ++p_;
                return v;
            }
            for (;;) {
                std::vector<std::string> path = key_path('=');
                expect('=');
                TVal x = value();
                TVal* t = &v;
                for (size_t i = 0; i + 1 < path.size(); ++i) t = &table_child(*t, path[i]);
                t->tab[path.back()] = std::move(x);
                skip_ws();
                if (p_ < t_.size() && t_[p_] == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < t_.size() && t_[p_] == '}') {
                    ++p_;
                    break;
                }
                fail("expected ',' or '}' in inline table");
            }
        } else if (t_.compare(p_, 4, "true") == 0) {
            v.kind = TVal::Bool;
            v.b = true;
            p_ += 4;
        } else if (t_.compare(p_, 5, "false") == 0) {
            v.kind = TVal::Bool;
            v.b = false;
            p_ += 5;
        } else {
            size_t b = p_;
            while (p_ < t_.size() && (std::isalnum((unsigned char)t_[p_]) || std::strchr("+-._", t_[p_]))) ++p_;
            std::string tok;
            for (size_t i = b; i < p_; ++i)
                if (t_[i] != '_') tok += t_[i];
            if (tok.empty()) fail("expected a value");
            const bool is_float = tok.find_first_of(".eE") != std::string::npos || tok == "inf" ||
                                  tok == "+inf" || tok == "-inf" || tok == "nan";
            char* end = nullptr;
            if (is_float) {
                v.kind = TVal::Float;
                v.num = std::strtod(tok.c_str(), &end);
            } else {
                v.kind = TVal::Int;
                v.num = (double)std::strtoll(tok.c_str(), &end, 10);
            }
            if (!end || *end != '\0') fail("bad number " + tok);
        }
        return v;
    }
};

// ---- values with the schema's defaults (config.rs:62-118) ------------------

using Table = std::map<std::string, TVal>;

const TVal* get(const Table& t, const char* k) {
    auto it = t.find(k);
    return it == t.end() ? nullptr : &it->second;
}
double num_or(const Table& t, const char* k, double def) {
    const TVal* v = get(t, k);
    if (!v) return def;
    if (!v->is_num()) throw ParseError(std::string("key ") + k + " must be a number");
    return v->num;
}
std::string str_or(const Table& t, const char* k, const std::string& def) {
    const TVal* v = get(t, k);
    if (!v) return def;
    if (v->kind != TVal::Str) throw ParseError(std::string("key ") + k + " must be a string");
    return v->s;
}
// to_vec4 (config.rs:62-66): missing components are zero
void to_vec4(const TVal& a, float out[4]) {
    for (int i = 0; i < 4; ++i) out[i] = 0.0f;
    if (a.kind != TVal::Arr) throw ParseError("expected an array of numbers");
    for (size_t i = 0; i < 4 && i < a.arr.size(); ++i) {
        if (!a.arr[i].is_num()) throw ParseError("expected an array of numbers");
        out[i] = (float)a.arr[i].num;
    }
}
void vec4_or(const Table& t, const char* k, const float def[4], float out[4]) {
    const TVal* v = get(t, k);
    if (!v) {
        for (int i = 0; i < 4; ++i) out[i] = def[i];
        return;
    }
    to_vec4(*v, out);
}
// get_packing (config.rs:107-109)
float packing_of(const Table& t, float h) {
    return (float)num_or(t, "packing", num_or(t, "spacing", 0.5 * (double)h) / (double)h);
}

// ---- regions (region.rs) -----------------------------------------------------

struct Box4 {
    float min[4], dim[4];
};

struct Region {
    virtual ~Region() = default;
    virtual Box4 bound() const = 0;
    virtual bool contains(const float p[4]) const = 0;
};
using RegionP = std::shared_ptr<Region>;

struct RAABB : Region {
    Box4 b;
    Box4 bound() const override { return b; }
    bool contains(const float p[4]) const override {  // region.rs:68-75
        for (int i = 0; i < 4; ++i)
            if (p[i] < b.min[i] || p[i] - b.min[i] > b.dim[i]) return false;
        return true;
    }
};

struct RAABE : Region {
    float center[4], radii[4];
    Box4 bound() const override {  // region.rs:80-86
        Box4 r;
        for (int i = 0; i < 4; ++i) {
            r.min[i] = center[i] - radii[i];
            r.dim[i] = 2.0f * radii[i];
        }
        return r;
    }
    bool contains(const float p[4]) const override {  // region.rs:88-107, in f64
        double lhs = 0.0;
        for (int i = 0; i < 4; ++i) {
            const double d = (double)(p[i] - center[i]);
            const double r = (double)radii[i];
            if (r > 0.0) {
                double coeff = 1.0;
                for (int j = 0; j < 4; ++j)
                    if (radii[j] > 0.0f && j != i) coeff = coeff * (double)radii[j];
                lhs = lhs + d * d * coeff * coeff;
            }
        }
        double rhs = 1.0;
        for (int i = 0; i < 4; ++i)
            if (radii[i] > 0.0f) rhs = rhs * (double)radii[i];
        return lhs <= rhs * rhs;
    }
};

struct RTransformed : Region {  // region.rs:125-217
    RegionP base;
    float a[4][4];  // column-major: a[col][row]
    float t[4];
    Box4 bound() const override {
        const Box4 bb = base->bound();
        float mn[4], mx[4];
        for (int i = 0; i < 4; ++i) {
            mn[i] = t[i];
            mx[i] = t[i];
        }
        for (int i = 0; i < 4; ++i) {
            float a_min = 0.0f;
            for (int j = 0; j < 4; ++j) a_min += a[j][i] * bb.min[j];
            mn[i] += a_min;
            mx[i] += a_min;
            for (int j = 0; j < 4; ++j) mn[i] += std::fmin(a[j][i] * bb.dim[j], 0.0f);
            for (int j = 0; j < 4; ++j) mx[i] += std::fmax(a[j][i] * bb.dim[j], 0.0f);
        }
        Box4 r;  // AABB::from_min_max
        for (int i = 0; i < 4; ++i) {
            r.min[i] = mn[i];
            r.dim[i] = mx[i] - mn[i];
        }
        return r;
    }
    bool contains(const float p[4]) const override {
        float v[4], m[4][4];
        for (int i = 0; i < 4; ++i) v[i] = p[i] - t[i];
        std::memcpy(m, a, sizeof(m));
        auto row_mul = [&](int row, int col, float f) {
            for (int k = col; k < 4; ++k) m[k][row] *= f;
            v[row] *= f;
        };
        auto row_sum = [&](int row, int col, float f, int dest) {
            for (int k = col; k < 4; ++k) m[k][dest] += f * m[k][row];
            v[dest] += f * v[row];
        };
        auto swap_rows = [&](int r1, int r2, int col) {
            for (int k = col; k < 4; ++k) std::swap(m[k][r1], m[k][r2]);
            std::swap(v[r1], v[r2]);
        };
        int i = 0, j = 0;  // Gauss-Jordan elimination as region.rs:175-203
        while (i < 4 && j < 4) {
            if (m[j][i] != 0.0f) {
                const float pivot = m[j][i];
                if (pivot != 1.0f) row_mul(i, j, 1.0f / pivot);
                for (int k = 0; k < 4; ++k) {
                    if (k != i && m[j][k] != 0.0f) row_sum(i, j, -m[j][k], k);
                }
                ++i;
                ++j;
            } else {
                bool cont = false;
                for (int k = i + 1; k < 4; ++k) {
                    if (m[j][k] != 0.0f) {
                        swap_rows(i, k, j);
                        cont = true;
                    }
                }
                if (!cont) ++j;
            }
        }
        return base->contains(v);
    }
};

struct RDifference : Region {
    RegionP l, r;
    Box4 bound() const override { return l->bound(); }
    bool contains(const float p[4]) const override { return l->contains(p) && !r->contains(p); }
};

struct RUnion : Region {
    RegionP l, r;
    Box4 bound() const override {  // region.rs:232-242
        const Box4 a = l->bound(), b = r->bound();
        Box4 o;
        for (int i = 0; i < 4; ++i) {
            const float m1 = a.min[i] + a.dim[i], m2 = b.min[i] + b.dim[i];
            o.min[i] = std::fmin(a.min[i], b.min[i]);
            o.dim[i] = std::fmax(m1, m2) - o.min[i];
        }
        return o;
    }
    bool contains(const float p[4]) const override { return l->contains(p) || r->contains(p); }
};

struct RIntersection : Region {
    RegionP l, r;
    Box4 bound() const override {  // region.rs:250-266
        const Box4 a = l->bound(), b = r->bound();
        Box4 o;
        for (int i = 0; i < 4; ++i) {
            const float m1 = a.min[i] + a.dim[i], m2 = b.min[i] + b.dim[i];
            o.min[i] = std::fmax(a.min[i], b.min[i]);
            o.dim[i] = std::fmin(m1, m2) - o.min[i];
        }
        return o;
    }
    bool contains(const float p[4]) const override { return l->contains(p) && r->contains(p); }
};

RegionP aabb_border(const Box4& b, float depth) {  // region.rs:37-46
    auto outer = std::make_shared<RAABB>();
    outer->b = b;
    auto inner = std::make_shared<RAABB>();
    for (int i = 0; i < 4; ++i) {
        const float c = b.min[i] + 0.5f * b.dim[i];
        inner->b.min[i] = std::fmin(b.min[i] + depth, c);
        inner->b.dim[i] = std::fmax(b.dim[i] - 2.0f * depth, 0.0f);
    }
    auto d = std::make_shared<RDifference>();
    d->l = outer;
    d->r = inner;
    return d;
}

RegionP aabe_border(const RAABE& e, float depth) {  // region.rs:54-63
    auto outer = std::make_shared<RAABE>(e);
    auto inner = std::make_shared<RAABE>(e);
    for (int i = 0; i < 4; ++i) inner->radii[i] = std::fmax(e.radii[i] - depth, 0.0f);
    auto d = std::make_shared<RDifference>();
    d->l = outer;
    d->r = inner;
    return d;
}

// ---- STL regions (examples/test_mods/mesh.rs) ------------------------------------

// An indexed triangle mesh as `stl_io::read_stl` (stl_io 0.4) returns it:
// vertices shared by exact value, each face with the normal stored in the file.
struct IndexedMesh {
    std::vector<std::array<float, 3>> vertices;
    struct Face {
        float normal[3];
        uint32_t v[3];
    };
    std::vector<Face> faces;
};

IndexedMesh read_stl(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw ParseError("cannot open STL file " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string data = ss.str();
    struct Tri {
        float n[3], v[3][3];
    };
    std::vector<Tri> tris;
    bool binary = data.size() >= 84;
    uint32_t count = 0;
    if (binary) {
        std::memcpy(&count, data.data() + 80, 4);
        binary = data.size() == 84 + 50ull * count;  // a binary file has exactly this size
    }
    if (binary) {
        tris.resize(count);
        for (uint32_t i = 0; i < count; ++i) {
            const char* r = data.data() + 84 + 50ull * i;
            std::memcpy(tris[i].n, r, 12);
            std::memcpy(tris[i].v, r + 12, 36);
        }
    } else {
        if (data.compare(0, 5, "solid") != 0) throw ParseError("not an STL file: " + path);
        std::istringstream in(data);
        std::string w;
        Tri t{};
        int nv = 0;
        while (in >> w) {
            if (w == "normal") {
                in >> t.n[0] >> t.n[1] >> t.n[2];
            } else if (w == "vertex") {
                if (nv >= 3) throw ParseError("STL facet with more than 3 vertices: " + path);
                in >> t.v[nv][0] >> t.v[nv][1] >> t.v[nv][2];
                ++nv;
            } else if (w == "endfacet") {
                if (nv != 3) throw ParseError("STL facet without 3 vertices: " + path);
                tris.push_back(t);
                nv = 0;
            }
        }
    }
    IndexedMesh m;
    std::map<std::array<uint32_t, 3>, uint32_t> index;  // by bit pattern
    for (const Tri& t : tris) {
        IndexedMesh::Face fc;
        std::memcpy(fc.normal, t.n, 12);
        for (int k = 0; k < 3; ++k) {
            std::array<uint32_t, 3> key;
            std::memcpy(key.data(), t.v[k], 12);
            auto it = index.find(key);
            if (it == index.end()) {
                it = index.emplace(key, (uint32_t)m.vertices.size()).first;
                m.vertices.push_back({t.v[k][0], t.v[k][1], t.v[k][2]});
            }
            fc.v[k] = it->second;
        }
        m.faces.push_back(fc);
    }
    if (m.vertices.empty()) throw ParseError("STL file without triangles: " + path);
    return m;
}

Box4 point_bound(const IndexedMesh& m) {  // mesh.rs:12-24
    float mn[3] = {m.vertices[0][0], m.vertices[0][1], m.vertices[0][2]};
    float mx[3] = {mn[0], mn[1], mn[2]};
    for (const auto& v : m.vertices)
        for (int i = 0; i < 3; ++i) {
            mn[i] = std::fmin(v[i], mn[i]);
            mx[i] = std::fmax(v[i], mx[i]);
        }
    Box4 b;
    for (int i = 0; i < 3; ++i) {
        b.min[i] = mn[i];
        b.dim[i] = mx[i] - mn[i];
    }
    b.min[3] = 0.0f;
    b.dim[3] = 0.0f;
    return b;
}

// f32::signum: 1 for +0 and positives, -1 for -0 and negatives, NaN for NaN
inline float signum(float x) { return std::isnan(x) ? x : std::copysign(1.0f, x); }

// Uniform grid over a box listing the items whose (margin-grown) boxes
// overlap each cell: a query visits only the items that can pass the exact
// test, so the result equals a walk over every item.
struct CullGrid {
    float lo[3] = {0, 0, 0}, inv[3] = {0, 0, 0};
    int n[3] = {1, 1, 1};
    std::vector<uint32_t> start, items;
    // cell of the scaled coordinate t = (p - lo) * inv along an axis of n
    // cells, clamped to [0, n - 1] in float before the conversion (a NaN or a
    // point far outside the grid would not fit in an int)
    static int axis_cell(float t, int n) {
        if (!(t >= 1.0f)) return 0;
        if (t >= (float)n) return n - 1;
        return std::min(n - 1, (int)t);
    }
    void build(const float mn[3], const float mx[3], int dims, size_t count,
               const std::function<void(size_t, float*, float*)>& box) {
        const int g = std::max(1, std::min(dims == 2 ? 512 : 96, (int)std::cbrt((double)count) * (dims == 2 ? 4 : 2)));
        for (int a = 0; a < 3; ++a) {
            n[a] = a < dims ? g : 1;
            lo[a] = mn[a];
            const float ext = mx[a] - mn[a];
            inv[a] = ext > 0.0f ? (float)n[a] / ext : 0.0f;
        }
        const size_t cells = (size_t)n[0] * n[1] * n[2];
        std::vector<uint32_t> cnt(cells + 1, 0);
        auto range = [&](const float* b0, const float* b1, int* c0, int* c1) {
            for (int a = 0; a < 3; ++a) {
                c0[a] = axis_cell((b0[a] - lo[a]) * inv[a], n[a]);
                c1[a] = axis_cell((b1[a] - lo[a]) * inv[a], n[a]);
            }
        };
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) {
                start.assign(cells + 1, 0);
                for (size_t c = 0; c < cells; ++c) start[c + 1] = start[c] + cnt[c];
                items.assign(start[cells], 0);
                std::fill(cnt.begin(), cnt.end(), 0);
            }
            for (size_t i = 0; i < count; ++i) {
                float b0[3], b1[3];
                box(i, b0, b1);
                int c0[3], c1[3];
                range(b0, b1, c0, c1);
                for (int z = c0[2]; z <= c1[2]; ++z)
                    for (int y = c0[1]; y <= c1[1]; ++y)
                        for (int x = c0[0]; x <= c1[0]; ++x) {
                            const size_t c = ((size_t)z * n[1] + y) * n[0] + x;
                            if (pass == 1) items[start[c] + cnt[c]] = (uint32_t)i;
                            ++cnt[c];
                        }
            }
        }
    }
    // items of the cell holding p (points outside the grid clamp to its border cells)
    std::pair<const uint32_t*, const uint32_t*> query(const float* p) const {
        size_t c = 0, mul = 1;
        for (int a = 0; a < 3; ++a) {
            const int i = axis_cell((p[a] - lo[a]) * inv[a], n[a]);
            c += (size_t)i * mul;
            mul *= (size_t)n[a];
        }
        return {items.data() + start[c], items.data() + start[c + 1]};
    }
};

struct RMesh : Region {  // mesh.rs:26-77: parity of the faces above the point whose xy triangle holds it
    IndexedMesh mesh;
    CullGrid grid;  // over xy: a face is visited only when p lies in its xy box
    Box4 bound() const override { return point_bound(mesh); }
    void index() {
        const Box4 b = point_bound(mesh);
        const float margin = 1e-4f * std::max(b.dim[0], b.dim[1]) + 1e-6f;
        const float mn[3] = {b.min[0] - margin, b.min[1] - margin, 0.0f};
        const float mx[3] = {b.min[0] + b.dim[0] + margin, b.min[1] + b.dim[1] + margin, 0.0f};
        grid.build(mn, mx, 2, mesh.faces.size(), [&](size_t i, float* b0, float* b1) {
            const auto& f = mesh.faces[i];
            for (int a = 0; a < 2; ++a) {
                float lo = mesh.vertices[f.v[0]][a], hi = lo;
                for (int k = 1; k < 3; ++k) {
                    lo = std::fmin(lo, mesh.vertices[f.v[k]][a]);
                    hi = std::fmax(hi, mesh.vertices[f.v[k]][a]);
                }
                b0[a] = lo - margin;
                b1[a] = hi + margin;
            }
            b0[2] = b1[2] = 0.0f;
        });
    }
    bool contains(const float p[4]) const override {
        if (p[3] != 0.0f) return false;
        bool inside = false;
        const float q[3] = {p[0], p[1], 0.0f};
        const auto span = grid.query(q);
        for (const uint32_t* it = span.first; it != span.second; ++it) {
            const auto& f = mesh.faces[*it];
            const auto& v0 = mesh.vertices[f.v[0]];
            const auto& v1 = mesh.vertices[f.v[1]];
            const auto& v2 = mesh.vertices[f.v[2]];
            const bool above = v0[2] >= p[2] || v1[2] >= p[2] || v2[2] >= p[2];
            if (!above) continue;
            const float s1[2] = {v1[0] - v0[0], v1[1] - v0[1]};
            const float s2[2] = {v2[0] - v0[0], v2[1] - v0[1]};
            const float d[2] = {p[0] - v0[0], p[1] - v0[1]};
            float a = s1[0] * s2[1] - s1[1] * s2[0];
            const float sg = signum(a);
            const float s = sg * (d[0] * s2[1] - d[1] * s2[0]);
            const float t = sg * (s1[0] * d[1] - s1[1] * d[0]);
            a = std::fabs(a);
            if (s >= 0.0f && s <= a && t >= 0.0f && t <= a && s + t <= a) inside = !inside;
        }
        return inside;
    }
};

struct RSurface : Region {  // mesh.rs:79-138: within `border` of a vertex or of a face
    IndexedMesh mesh;
    float border = 0.0f;
    // a vertex or a face is visited only when p lies in its box grown by the border
    CullGrid vgrid, fgrid;
    void index() {
        Box4 b = bound();
        const float ext = std::max({b.dim[0], b.dim[1], b.dim[2]});
        const float margin = border + 1e-4f * ext + 1e-6f;
        const float mn[3] = {b.min[0] - margin, b.min[1] - margin, b.min[2] - margin};
        const float mx[3] = {b.min[0] + b.dim[0] + margin, b.min[1] + b.dim[1] + margin,
                             b.min[2] + b.dim[2] + margin};
        vgrid.build(mn, mx, 3, mesh.vertices.size(), [&](size_t i, float* b0, float* b1) {
            for (int a = 0; a < 3; ++a) {
                b0[a] = mesh.vertices[i][a] - margin;
                b1[a] = mesh.vertices[i][a] + margin;
            }
        });
        fgrid.build(mn, mx, 3, mesh.faces.size(), [&](size_t i, float* b0, float* b1) {
            const auto& f = mesh.faces[i];
            for (int a = 0; a < 3; ++a) {
                float lo = mesh.vertices[f.v[0]][a], hi = lo;
                for (int k = 1; k < 3; ++k) {
                    lo = std::fmin(lo, mesh.vertices[f.v[k]][a]);
                    hi = std::fmax(hi, mesh.vertices[f.v[k]][a]);
                }
                b0[a] = lo - margin;
                b1[a] = hi + margin;
            }
        });
    }
    Box4 bound() const override {
        Box4 b = point_bound(mesh);
        for (int i = 0; i < 3; ++i) {
            b.min[i] -= border;
            b.dim[i] += border * 2.0f;
        }
        return b;
    }
    static float dot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
    static void cross3(const float* a, const float* b, float* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    }
    static void sub3(const float* a, const float* b, float* o) {
        o[0] = a[0] - b[0];
        o[1] = a[1] - b[1];
        o[2] = a[2] - b[2];
    }
    bool contains(const float p[4]) const override {
        const auto vs = vgrid.query(p);
        for (const uint32_t* it = vs.first; it != vs.second; ++it) {
            float d[3];
            sub3(p, mesh.vertices[*it].data(), d);
            if (dot3(d, d) <= border * border) return true;
        }
        const auto fs = fgrid.query(p);
        for (const uint32_t* it = fs.first; it != fs.second; ++it) {
            const auto& f = mesh.faces[*it];
            const float* n = f.normal;
            const float* a = mesh.vertices[f.v[0]].data();
            const float* b = mesh.vertices[f.v[1]].data();
            const float* c = mesh.vertices[f.v[2]].data();
            float d[3];
            sub3(p, a, d);
            if (std::fabs(dot3(d, n)) <= std::sqrt(dot3(n, n)) * border) {
                float s1[3], s2[3], s3[3], s4[3], d2[3], n1[3], n2[3], n3[3];
                sub3(b, a, s1);
                sub3(c, a, s2);
                sub3(c, b, s3);
                sub3(a, b, s4);
                sub3(p, b, d2);
                cross3(s1, n, n1);
                cross3(s2, n, n2);
                cross3(s3, n, n3);
                if (signum(dot3(d, n1)) == signum(dot3(s2, n1)) && signum(dot3(d, n2)) == signum(dot3(s1, n2)) &&
                    signum(dot3(d2, n3)) == signum(dot3(s4, n3)))
                    return true;
            }
        }
        return false;
    }
};

RegionP parse_region_from_mat(const Table& t);

RegionP parse_base(const Table& t) {  // config.rs:180-239
    if (const TVal* mv = get(t, "model"); mv && mv->kind == TVal::Str) {
        const TVal* bv = get(t, "border");
        if (bv && bv->kind == TVal::Float) {  // .and_then(as_float): an integer border is no border
            auto r = std::make_shared<RSurface>();
            r->mesh = read_stl(mv->s);
            r->border = (float)bv->num;
            r->index();
            return r;
        }
        auto r = std::make_shared<RMesh>();
        r->mesh = read_stl(mv->s);
        r->index();
        return r;
    }
    const TVal* border_v = get(t, "border");
    if (border_v && !border_v->is_num()) throw ParseError("border must be a number");
    float dim[4] = {0, 0, 0, 0}, mn[4] = {0, 0, 0, 0};
    bool boxed;
    if (const TVal* d = get(t, "dim"); d && d->kind == TVal::Arr) {
        boxed = true;
        to_vec4(*d, dim);
    } else if (const TVal* r = get(t, "radii"); r && r->kind == TVal::Arr) {
        boxed = false;
        to_vec4(*r, dim);
        for (int i = 0; i < 4; ++i) dim[i] *= 2.0f;
    } else if (const TVal* dd = get(t, "diameters"); dd && dd->kind == TVal::Arr) {
        boxed = false;
        to_vec4(*dd, dim);
    } else {
        return parse_region_from_mat(t);
    }
    if (const TVal* m = get(t, "min"); m && m->kind == TVal::Arr) {
        to_vec4(*m, mn);
    } else if (const TVal* c = get(t, "center"); c && c->kind == TVal::Arr) {
        to_vec4(*c, mn);
        for (int i = 0; i < 4; ++i) mn[i] -= 0.5f * dim[i];
    }
    if (boxed) {
        Box4 b;
        for (int i = 0; i < 4; ++i) {
            b.min[i] = mn[i];
            b.dim[i] = dim[i];
        }
        if (border_v) return aabb_border(b, (float)border_v->num);
        auto r = std::make_shared<RAABB>();
        r->b = b;
        return r;
    }
    RAABE e;
    for (int i = 0; i < 4; ++i) {
        dim[i] *= 0.5f;
        mn[i] += dim[i];
        e.center[i] = mn[i];
        e.radii[i] = dim[i];
    }
    if (border_v) return aabe_border(e, (float)border_v->num);
    return std::make_shared<RAABE>(e);
}

RegionP parse_region(const Table& t) {  // config.rs:130-178
    RegionP base = parse_base(t);
    if (!get(t, "translation") && !get(t, "scale") && !get(t, "rotation")) return base;
    const float zero[4] = {0, 0, 0, 0}, zaxis[4] = {0, 0, 1, 0};
    float trans[4], rot[4], scale[4] = {1, 1, 1, 1};
    vec4_or(t, "translation", zero, trans);
    const TVal* rv = get(t, "rotation");
    if (rv && rv->kind == TVal::Float) {
        rot[0] = 0;
        rot[1] = 0;
        rot[2] = 1;
        rot[3] = (float)rv->num;
    } else {
        vec4_or(t, "rotation", zaxis, rot);
    }
    const TVal* sv = get(t, "scale");
    if (sv && sv->kind == TVal::Float) {
        for (int i = 0; i < 4; ++i) scale[i] = (float)sv->num;
    } else if (sv && sv->kind == TVal::Arr) {
        for (size_t i = 0; i < sv->arr.size() && i < 4; ++i) {
            if (!sv->arr[i].is_num()) throw ParseError("scale must hold numbers");
            scale[i] = (float)sv->arr[i].num;
        }
    }
    const float pi = 3.14159265358979323846f;
    const float ang = rot[3] * (pi / 180.0f);  // f32::to_radians
    const float c = std::cos(ang), s = std::sin(ang);
    const float u_l = std::sqrt(rot[0] * rot[0] + rot[1] * rot[1] + rot[2] * rot[2]);
    const float u[3] = {rot[0] / u_l, rot[1] / u_l, rot[2] / u_l};
    float m[4][4] = {
        {c + u[0] * u[0] * (1.0f - c), u[0] * u[1] * (1.0f - c) + u[2] * s, u[0] * u[2] * (1.0f - c) - u[1] * s, 0.0f},
        {u[1] * u[2] * (1.0f - c) - u[1] * s, c + u[1] * u[1] * (1.0f - c), u[1] * u[2] * (1.0f - c) + u[0] * s, 0.0f},
        {u[0] * u[2] * (1.0f - c) + u[1] * s, u[1] * u[2] * (1.0f - c) - u[0] * s, c + u[2] * u[2] * (1.0f - c), 0.0f},
        {0.0f, 0.0f, 0.0f, 1.0f}};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) m[i][j] *= scale[i];
    auto r = std::make_shared<RTransformed>();
    r->base = base;
    std::memcpy(r->a, m, sizeof(m));
    std::memcpy(r->t, trans, sizeof(trans));
    return r;
}

template <class Node>
RegionP fold(const TVal& arr) {  // config.rs:124-128
    if (arr.kind != TVal::Arr || arr.arr.empty()) throw ParseError("region list must be a non-empty array");
    RegionP acc;
    for (const TVal& e : arr.arr) {
        if (e.kind != TVal::Tab) throw ParseError("region list entries must be tables");
        RegionP r = parse_region(e.tab);
        if (!acc) {
            acc = r;
        } else {
            auto n = std::make_shared<Node>();
            n->l = acc;
            n->r = r;
            acc = n;
        }
    }
    return acc;
}

RegionP parse_region_from_mat(const Table& t) {  // config.rs:242-252
    if (const TVal* a = get(t, "union"); a && a->kind == TVal::Arr) return fold<RUnion>(*a);
    if (const TVal* a = get(t, "difference"); a && a->kind == TVal::Arr) return fold<RDifference>(*a);
    if (const TVal* a = get(t, "intersection"); a && a->kind == TVal::Arr) return fold<RIntersection>(*a);
    if (const TVal* r = get(t, "region"); r && r->kind == TVal::Tab) return parse_region(r->tab);
    throw ParseError("material has no region table and no union, difference or intersection array");
}

// ---- seeding (material_region/mod.rs:56-155) --------------------------------

struct Velocity {
    float vel[4] = {0, 0, 0, 0};
    float w[6] = {0, 0, 0, 0, 0, 0};
    float center[4] = {0, 0, 0, 0};
    void at(const float p[4], float out[4]) const {  // config.rs:412-423
        const float r[4] = {p[0] - center[0], p[1] - center[1], p[2] - center[2], p[3] - center[3]};
        out[0] = w[1] * r[2] - w[2] * r[1] - w[3] * r[3] + vel[0];
        out[1] = w[2] * r[0] - w[0] * r[2] + w[4] * r[3] + vel[1];
        out[2] = w[0] * r[1] - w[1] * r[0] - w[5] * r[3] + vel[2];
        out[3] = w[3] * r[0] - w[4] * r[1] + w[5] * r[3] + vel[3];
    }
};

// Candidates of the staggered lattice with pitch packing*h inside the
// region's bound; returns the particles inside the region and sets the mass.
void gen_particles(const Region& region, float packing, float kernel_h, arp_material& mat, uint32_t mat_id,
                   const Velocity* velf, std::vector<arp_particle>& out) {
    const float h = packing * kernel_h;
    if (!(h > 0.0f) || !std::isfinite(h)) throw ParseError("particle spacing (packing * kernel_radius) must be positive");
    const Box4 bound = region.bound();
    uint64_t num_in_box = 0;
    float pos[4] = {bound.min[0], bound.min[1], bound.min[2], bound.min[3]};
    const float start_density = mat.start_den;
    const float sq2 = std::sqrt(2.0f), sq3 = std::sqrt(3.0f), sq8 = std::sqrt(8.0f);
    float offset2 = 0.0f;
    const uint64_t kLimit = 1ull << 28;
    std::vector<std::array<float, 4>> sites;  // every lattice site of the bound, in walk order
    for (;;) {
        float offset = 0.0f;
        pos[1] = bound.min[1] + offset2;
        for (;;) {
            pos[0] = bound.min[0] + (offset + offset2);
            for (;;) {
                if (++num_in_box > kLimit) throw ParseError("a region spans more than 2^28 lattice sites");
                sites.push_back({pos[0], pos[1], pos[2], pos[3]});
                pos[0] += h;
                if (pos[0] - bound.min[0] > bound.dim[0] || bound.dim[0] == 0.0f) break;
            }
            pos[1] += h / sq2;
            offset = offset == 0.0f ? h / 2.0f : 0.0f;
            if (pos[1] - bound.min[1] > bound.dim[1] || bound.dim[1] == 0.0f) break;
        }
        pos[2] += h / sq3;
        offset2 = offset2 == 0.0f ? h / sq8 : 0.0f;
        if (pos[2] - bound.min[2] > bound.dim[2] || bound.dim[2] == 0.0f) break;
    }
    // the region test of every site, on all host threads (the reference tests
    // its sites on worker threads too, material_region/mod.rs:79-103)
    std::vector<uint8_t> keep(sites.size(), 0);
    const size_t nt = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(),
                                                           (sites.size() + 4095) / 4096));
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (size_t k = t; k < sites.size(); k += nt) keep[k] = region.contains(sites[k].data()) ? 1 : 0;
        });
    for (auto& th : pool) th.join();
    for (size_t k = 0; k < sites.size(); ++k) {
        if (!keep[k]) continue;
        arp_particle p{};
        for (int i = 0; i < 4; ++i) p.pos[i] = sites[k][i];
        if (velf) velf->at(sites[k].data(), p.vel);
        p.den = start_density;
        p.mat = mat_id;
        p.solid_id = 0xFFFFFFFFu;
        out.push_back(p);
    }
    double content = 1.0;  // the f64 product of the nonzero extents, then times the density
    for (int i = 0; i < 4; ++i)
        if (bound.dim[i] > 0.0f) content = content * (double)bound.dim[i];
    const double box_mass = (double)start_density * content;
    mat.mass = (float)(box_mass / (double)num_in_box);
}

// ---- the schema (config.rs:296-474) ----------------------------------------------

struct Obj {
    std::string name;
    const Table* table;
    bool boundary;
};

arp_interaction parse_interaction(const Table& t, double h) {  // config.rs:255-277
    arp_interaction it{};
    it.strength = (float)num_or(t, "contact_strength", 10000.0);
    it.radius = (float)num_or(t, "contact_radius", num_or(t, "contact_factor", 2.0) * h);
    it.friction = (float)num_or(t, "friction", 0.0);
    it.dampening = (float)num_or(t, "dampening", 0.0);
    const std::string pot = str_or(t, "potential", "");
    if (pot == "Zero" || pot == "zero") it.potential = ARP_CONTACT_ZERO;
    else if (pot == "Constant" || pot == "constant") it.potential = ARP_CONTACT_CONSTANT;
    else if (pot == "Linear" || pot == "linear") it.potential = ARP_CONTACT_LINEAR;
    else if (pot == "Tait" || pot == "tait") it.potential = ARP_CONTACT_TAIT;
    else if (pot == "Hertz" || pot == "hertz") it.potential = ARP_CONTACT_HERTZ;
    else if (pot == "LennardJones" || pot == "Lennard-Jones" || pot == "Lennard Jones" || pot == "lennard jones" ||
             pot == "lennard-jones")
        it.potential = ARP_CONTACT_LENNARD_JONES;
    else it.potential = ARP_CONTACT_LINEAR;
    return it;
}

int integrator_id(const std::string& s) {  // examples/test.rs:165-180
    std::string l = s;
    std::transform(l.begin(), l.end(), l.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    if (l == "verlet") return ARP_INT_VERLET;
    if (l == "euler" || l == "rk1") return ARP_INT_EULER;
    if (l == "midpoint" || l == "rk2") return ARP_INT_MIDPOINT;
    if (l == "heun2" || l == "heun") return ARP_INT_HEUN2;
    if (l == "ralston") return ARP_INT_RALSTON;
    if (l == "rk3") return ARP_INT_RK3;
    if (l == "heun3") return ARP_INT_HEUN3;
    if (l == "rk4") return ARP_INT_RK4;
    if (l == "rk_3_8") return ARP_INT_RK_3_8;
    throw ParseError("invalid integrator " + s);
}

void build_scene(const TVal& root, LoadedScene& out) {
    const Table& top = root.tab;
    out.name = str_or(top, "name", "Fluid Test");
    out.subticks = (uint32_t)num_or(top, "subticks", 1);
    out.h = (float)num_or(top, "kernel_radius", 1.0 / 64.0);
    out.dt = (float)num_or(top, "time_step", 0.01);
    out.alpha = (float)num_or(top, "artificial_viscocity", 50.0);
    out.gravity = (float)num_or(top, "gravity", 1.0);
    const float dmin[4] = {-1, -1, 0, 0}, ddim[4] = {2, 2, 0, 0};
    vec4_or(top, "min", dmin, out.bounds.min);
    vec4_or(top, "dim", ddim, out.bounds.dim);
    out.integrator = integrator_id(str_or(top, "integrator", "verlet"));
    const float h = out.h;
    const float alpha = out.alpha;
    // renderer settings (config.rs:302-323, 466-470)
    {
        const TVal* lv = get(top, "lighting");
        if (lv && lv->kind != TVal::Bool) throw ParseError("lighting must be a boolean");
        out.lighting = lv ? lv->b : get(top, "light_pos") != nullptr;
        out.render_h = h * (float)num_or(top, "particle_render_factor", 1.0);
        float lp[4], lc[4];
        const float dlp[4] = {-3, 3, -3, 0}, dlc[4] = {1, 1, 1, 0};
        vec4_or(top, "light_pos", dlp, lp);
        vec4_or(top, "light_color", dlc, lc);
        for (int i = 0; i < 3; ++i) {
            out.light_pos[i] = lp[i];
            out.light_color[i] = lc[i];
        }
        out.ambient = (float)num_or(top, "ambient_brightness", 1.0);
        out.diffuse = (float)num_or(top, "diffuse_brightness", 10.0);
        out.specular = (float)num_or(top, "specular_brightness", 0.0);
        out.view_pos[0] = out.view_pos[1] = 0.0;
        if (const TVal* vp = get(top, "view_pos")) {
            if (vp->kind != TVal::Arr) throw ParseError("view_pos must be an array");
            for (size_t i = 0; i < vp->arr.size() && i < 2; ++i) {
                if (!vp->arr[i].is_num()) throw ParseError("view_pos must hold numbers");
                out.view_pos[i] = vp->arr[i].num;
            }
        }
        out.view_scale = num_or(top, "view_scale", 1.0);
        out.view_angle = num_or(top, "view_angle", 0.0) * (3.14159265358979323846 / 180.0);  // f64::to_radians
    }
    // get_colors (config.rs:111-118): color, color_low_density, color_high_density
    auto colors_of = [&](const Table& t, float* c12) {
        const float black[4] = {0, 0, 0, 1};
        vec4_or(t, "color", black, c12);
        vec4_or(t, "color_low_density", c12, c12 + 4);
        vec4_or(t, "color_high_density", c12, c12 + 8);
    };

    std::vector<Obj> objs;
    std::map<std::pair<std::string, std::string>, arp_interaction> inter_map;
    auto collect_interactions = [&](const std::string& name, const Table& t) {  // config.rs:279-294
        for (const auto& kv : t) {
            if (kv.second.kind != TVal::Tab) continue;
            if (kv.first == "region" || kv.first == "union" || kv.first == "intersection" || kv.first == "difference")
                continue;
            inter_map[{name, kv.first}] = parse_interaction(kv.second.tab, (double)h);
        }
    };
    if (const TVal* b = get(top, "boundaries"); b && b->kind == TVal::Tab)
        for (const auto& kv : b->tab) {
            if (kv.second.kind != TVal::Tab) throw ParseError("boundary " + kv.first + " must be a table");
            objs.push_back({kv.first, &kv.second.tab, true});
        }
    std::vector<Obj> clicks;
    if (const TVal* o = get(top, "objects"); o && o->kind == TVal::Tab)
        for (const auto& kv : o->tab) {
            if (kv.second.kind != TVal::Tab) throw ParseError("object " + kv.first + " must be a table");
            // objects with "on_click" are interactive additions (config.rs:426-446)
            (get(kv.second.tab, "on_click") ? clicks : objs).push_back({kv.first, &kv.second.tab, false});
        }

    // one material and its seeded particles, as config.rs:328-424 and
    // MaterialRegion::gen_particles build them
    auto seed = [&](const Obj& ob, uint32_t idx, arp_material& m, std::vector<arp_particle>& ps) {
        const Table& t = *ob.table;
        m = arp_material{};
        Velocity vel;
        const bool moving = !ob.boundary;
        if (ob.boundary) {  // config.rs:330-348, Material::new_immobile
            m.visc = (float)num_or(t, "friction", 0.0);
            m.start_den = 1.0f;
            m.target_den = 1.0f;
            m.immobile = 1;
        } else {  // config.rs:352-424
            m.start_den = (float)num_or(t, "start_density", num_or(t, "density", 1.0));
            m.target_den = (float)num_or(t, "target_density", num_or(t, "density", 1.0));
            m.sound_speed = (float)num_or(t, "speed_of_sound", 0.0);
            m.visc = (float)num_or(t, "viscocity", num_or(t, "friction", 0.0));
            m.bulk_visc = (float)num_or(t, "bulk_viscocity", (double)(alpha * h * m.sound_speed));
            const TVal* st = get(t, "state");
            if (!st) st = get(t, "state_equation");
            if (!st) {
                if (get(t, "speed_of_sound"))
                    m.state_eq = (get(t, "start_density") || get(t, "target_density")) ? ARP_EOS_IDEAL_GAS
                                                                                       : ARP_EOS_TAIT;
                else m.state_eq = ARP_EOS_ZERO;
            } else {
                if (st->kind != TVal::Str) throw ParseError("state must be a string");
                const std::string& v = st->s;
                if (v == "Tait" || v == "tait" || v == "Liquid" || v == "liquid") m.state_eq = ARP_EOS_TAIT;
                else if (v == "Ideal_Gas" || v == "ideal_gas" || v == "gas" || v == "Gas") m.state_eq = ARP_EOS_IDEAL_GAS;
                else if (v == "Constant" || v == "constant") m.state_eq = ARP_EOS_CONSTANT;
                else throw ParseError("Invalid state equation: " + v);
            }
            m.strain_order = (int32_t)num_or(t, "strain_order", 2);
            m.normal_stiffness = (float)num_or(t, "normal_stiffness", 0.0);
            m.shear_stiffness = (float)num_or(t, "shear_stiffness", 0.0);
            m.normal_damp = (float)num_or(t, "normal_dampening", 0.0);
            m.shear_damp = (float)num_or(t, "shear_dampening", 0.0);
            if (get(t, "yield_strength") || get(t, "relaxation_time")) {
                m.plastic = 1;
                m.yield_strength = (float)num_or(t, "yield_strength", 0.0);
                m.work_hardening = (float)num_or(t, "work_hardening", 0.0);
                m.work_hardening_exp = (float)num_or(t, "work_hardening_exp", 2.0);
                m.kinematic_hardening = (float)num_or(t, "kinematic_hardening", 0.0);
                m.thermal_softening = (float)num_or(t, "thermal_softening", 0.0);
                m.relaxation_time = (float)num_or(t, "relaxation_time", 1.0);
            }
            const float zero[4] = {0, 0, 0, 0};
            vec4_or(t, "velocity", zero, vel.vel);
            if (const TVal* av = get(t, "angular_velocity")) {
                if (av->kind != TVal::Arr) throw ParseError("angular_velocity must be an array");
                for (size_t i = 0; i < av->arr.size() && i < 6; ++i) {
                    if (!av->arr[i].is_num()) throw ParseError("angular_velocity must hold numbers");
                    vel.w[i] = (float)av->arr[i].num;
                }
            }
        }
        RegionP region = parse_region_from_mat(t);
        if (moving) {
            const Box4 b = region->bound();  // AABB::center
            for (int i = 0; i < 4; ++i) vel.center[i] = b.min[i] + 0.5f * b.dim[i];
        }
        gen_particles(*region, packing_of(t, h), h, m, idx, moving ? &vel : nullptr, ps);
    };
    for (uint32_t idx = 0; idx < objs.size(); ++idx) {
        arp_material m{};
        std::vector<arp_particle> ps;
        seed(objs[idx], idx, m, ps);
        out.materials.push_back(m);
        float c12[12];
        colors_of(*objs[idx].table, c12);
        out.colors.insert(out.colors.end(), c12, c12 + 12);
        auto& dst = m.immobile ? out.boundary : out.particles;
        dst.insert(dst.end(), ps.begin(), ps.end());
        collect_interactions(objs[idx].name, *objs[idx].table);
    }
    // FluidSim::add_particles seeds with material id 0 (mod.rs:182)
    for (const Obj& ob : clicks) {
        LoadedScene::Addition add;
        add.name = ob.name;
        const TVal* oc = get(*ob.table, "on_click");
        add.relative = oc->kind == TVal::Str && oc->s == "Relative";
        seed(ob, 0, add.material, add.particles);
        out.on_click.push_back(std::move(add));
    }
    // config.rs:453-466 then FluidSim::new's resolution (done by arp_sim_create)
    const size_t M = objs.size();
    out.interactions.assign(M * M, arp_interaction{});
    out.given.assign(M * M, 0);
    for (size_t i = 0; i < M; ++i)
        for (size_t j = 0; j < M; ++j) {
            auto it = inter_map.find({objs[i].name, objs[j].name});
            if (it == inter_map.end()) it = inter_map.find({objs[j].name, objs[i].name});
            if (it != inter_map.end()) {
                out.interactions[i * M + j] = it->second;
                out.given[i * M + j] = 1;
            }
        }
}

arp_status load_scene_toml(const char* path, LoadedScene& out, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = std::string("cannot open ") + path;
        return ARP_ERR_IO;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    try {
        TomlReader r(text);
        TVal root = r.parse();
        out = LoadedScene{};
        build_scene(root, out);
    } catch (const Unsupported& e) {
        err = std::string(path) + ": " + e.what();
        return ARP_ERR_UNSUPPORTED;
    } catch (const ParseError& e) {
        err = std::string(path) + ": " + e.what();
        return ARP_ERR_PARSE;
    } catch (const std::exception& e) {
        err = std::string(path) + ": " + e.what();
        return ARP_ERR_PARSE;
    }
    return ARP_OK;
}

}  // namespace arp
