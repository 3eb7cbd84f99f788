// RadFoam / PowerFoam PLY reader behind the C ABI (host code only): the walk
// subset of the reference's loader, blade-volume/src/io/radfoam_ply.rs
// (try_load :1141-1213, header :452-596, schema :122-372, decode_binary
// :728-859, decode_ascii :861-1109, validate_csr :1111-1139), so that a host
// in the reference's language loads a model file without a Python runtime.
//
// File layout: PLY 1.0, binary little-endian or ASCII, exactly two elements,
// `vertex` then `adjacency`.  A vertex row carries x, y, z, density (float),
// adjacency_offset (uint: the CSR end offset of that point), the DC colour as
// blade_sh_dc_0..2 (float) or as a red/green/blue preview (uchar, DC = (c /
// 255 - 0.5) / 0.2820948, :722-726), the higher SH coefficients color_sh_<k>
// (float, contiguous k; their count fixes the degree) and optionally radius
// (float, PowerFoam).  The adjacency element holds one uint per CSR entry.
// Oriented-surface, surface-detail, surface-colour and spherical-Voronoi
// properties are rejected: the walk has no such terms.

#include <algorithm>
#include <cctype>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "bv_internal.h"

namespace {

constexpr size_t kMaxHeaderBytes = 1024 * 1024;
constexpr size_t kMaxAsciiRowBytes = 64 * 1024;

enum class Ty { F32, U32, U8 };

struct Prop {
    std::string name;
    Ty ty;
    size_t offset;  // byte offset in a binary row
};

struct Element {
    std::string name;
    uint64_t count = 0;
    std::vector<Prop> props;
    size_t row_bytes = 0;
};

struct Header {
    bool ascii = false;
    std::vector<Element> elements;
    long body_offset = 0;
};

struct Schema {
    int x = -1, y = -1, z = -1, density = -1, adjacency_offset = -1, radius = -1;
    int dc[3] = {-1, -1, -1}, preview[3] = {-1, -1, -1};
    bool exact = false;
    std::vector<int> rest;  // property index of color_sh_<k>, k = 0, 1, ...
    uint32_t degree = 0;
};

bv_status ply_fail(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    bv::set_last_error(buf);
    return BV_ERR_INVALID_MODEL;
}

bv_status arg_fail(const char *msg) {
    bv::set_last_error(msg);
    return BV_ERR_INVALID_ARGUMENT;
}

size_t ty_size(Ty t) { return t == Ty::U8 ? 1 : 4; }

bool parse_type(const std::string &s, Ty *t) {
    if (s == "float" || s == "float32") {
        *t = Ty::F32;
    } else if (s == "uint" || s == "uint32") {
        *t = Ty::U32;
    } else if (s == "uchar" || s == "uint8") {
        *t = Ty::U8;
    } else {
        return false;
    }
    return true;
}

std::vector<std::string> words(const std::string &line) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && isspace((unsigned char)line[i])) ++i;
        size_t j = i;
        while (j < line.size() && !isspace((unsigned char)line[j])) ++j;
        if (j > i) out.push_back(line.substr(i, j - i));
        i = j;
    }
    return out;
}

// One line including its '\n'; false at the end of the file.  too_long: the
// line exceeds limit bytes (reading stops there).
bool read_line(FILE *f, std::string &line, size_t limit, bool *too_long) {
    line.clear();
    *too_long = false;
    int c;
    while ((c = fgetc(f)) != EOF) {
        line.push_back((char)c);
        if (line.size() > limit) {
            *too_long = true;
            return true;
        }
        if (c == '\n') break;
    }
    return !line.empty();
}

bool starts_with(const std::string &s, const char *p) { return s.compare(0, strlen(p), p) == 0; }

bv_status read_header(FILE *f, Header *h) {
    std::string line;
    size_t total = 0;
    bool first = true, saw_end = false, have_fmt = false, too_long = false;
    while (read_line(f, line, kMaxHeaderBytes, &too_long)) {
        total += line.size();
        if (too_long || total > kMaxHeaderBytes)
            return ply_fail("RadFoam PLY header exceeds %zu bytes", kMaxHeaderBytes);
        const auto w = words(line);
        if (first) {
            if (w.size() != 1 || w[0] != "ply") return ply_fail("RadFoam PLY is missing the 'ply' magic");
            first = false;
            continue;
        }
        if (w.empty()) continue;
        const std::string &head = w[0];
        if (head == "format") {
            if (have_fmt) return ply_fail("duplicate RadFoam PLY format line");
            if (w.size() < 3 || w[2] != "1.0")
                return ply_fail("unsupported RadFoam PLY version '%s'", w.size() > 2 ? w[2].c_str() : "");
            if (w[1] == "ascii") {
                h->ascii = true;
            } else if (w[1] == "binary_little_endian") {
                h->ascii = false;
            } else {
                return ply_fail("unsupported RadFoam PLY format '%s'", w[1].c_str());
            }
            have_fmt = true;
        } else if (head == "comment" || head == "obj_info") {
            continue;
        } else if (head == "element") {
            if (w.size() < 3) return ply_fail("RadFoam PLY element needs a name and a count");
            for (auto &e : h->elements)
                if (e.name == w[1]) return ply_fail("duplicate RadFoam PLY element '%s'", w[1].c_str());
            char *end = nullptr;
            const unsigned long long n = strtoull(w[2].c_str(), &end, 10);
            if (!end || *end || w[2][0] == '-')
                return ply_fail("invalid count for element '%s'", w[1].c_str());
            Element e;
            e.name = w[1];
            e.count = n;
            h->elements.push_back(e);
        } else if (head == "property") {
            if (h->elements.empty()) return ply_fail("RadFoam PLY property appears before an element");
            Element &e = h->elements.back();
            if (w.size() > 1 && w[1] == "list")
                return ply_fail("RadFoam PLY list properties are unsupported in element '%s'",
                                e.name.c_str());
            Ty t;
            if (w.size() < 3 || !parse_type(w[1], &t))
                return ply_fail("unsupported RadFoam PLY scalar type '%s'", w.size() > 1 ? w[1].c_str() : "");
            for (auto &p : e.props)
                if (p.name == w[2])
                    return ply_fail("duplicate RadFoam PLY property '%s.%s'", e.name.c_str(), w[2].c_str());
            e.props.push_back(Prop{w[2], t, e.row_bytes});
            e.row_bytes += ty_size(t);
        } else if (head == "end_header") {
            saw_end = true;
            break;
        } else {
            return ply_fail("unexpected RadFoam PLY header token '%s'", head.c_str());
        }
    }
    if (first) return ply_fail("RadFoam PLY is missing the 'ply' magic");
    if (!saw_end) return ply_fail("RadFoam PLY header has no end_header");
    if (!have_fmt) return ply_fail("RadFoam PLY has no format line");
    h->body_offset = ftell(f);
    return BV_OK;
}

bv_status make_schema(const Header &h, Schema *s) {
    if (h.elements.size() != 2 || h.elements[0].name != "vertex" || h.elements[1].name != "adjacency")
        return ply_fail("RadFoam PLY elements must be exactly 'vertex' followed by 'adjacency'");
    const Element &v = h.elements[0], &a = h.elements[1];
    if (v.count > 0xfffffffeull || a.count > 0xffffffffull)
        return ply_fail("RadFoam PLY element count exceeds 32 bits");
    auto find = [&](const char *name) {
        for (size_t i = 0; i < v.props.size(); ++i)
            if (v.props[i].name == name) return (int)i;
        return -1;
    };
    struct Req {
        const char *name;
        int *slot;
        Ty ty;
    };
    const Req req[] = {{"x", &s->x, Ty::F32},
                       {"y", &s->y, Ty::F32},
                       {"z", &s->z, Ty::F32},
                       {"density", &s->density, Ty::F32},
                       {"adjacency_offset", &s->adjacency_offset, Ty::U32}};
    for (const Req &r : req) {
        *r.slot = find(r.name);
        if (*r.slot < 0) return ply_fail("RadFoam PLY element 'vertex' is missing property '%s'", r.name);
        if (v.props[*r.slot].ty != r.ty)
            return ply_fail("RadFoam PLY property 'vertex.%s' has the wrong type", r.name);
    }
    if (a.props.size() != 1 || a.props[0].name != "adjacency" || a.props[0].ty != Ty::U32)
        return ply_fail("RadFoam PLY adjacency element must hold one uint 'adjacency'");
    static const char *unsupported[] = {"nx", "ny", "nz", "surface_offset", "blade_surface_detail_",
                                        "blade_surface_color_", "blade_spherical_voronoi_"};
    for (auto &p : v.props)
        for (const char *u : unsupported)
            if (starts_with(p.name, u))
                return ply_fail("RadFoam PLY property '%s' (oriented-surface / detail terms) is not "
                                "supported on this path",
                                p.name.c_str());
    int n_exact = 0, n_preview = 0;
    const char *exact[3] = {"blade_sh_dc_0", "blade_sh_dc_1", "blade_sh_dc_2"};
    const char *preview[3] = {"red", "green", "blue"};
    for (int c = 0; c < 3; ++c) {
        s->dc[c] = find(exact[c]);
        s->preview[c] = find(preview[c]);
        n_exact += s->dc[c] >= 0;
        n_preview += s->preview[c] >= 0;
    }
    if (n_exact > 0 && n_exact < 3) return ply_fail("RadFoam PLY needs all of blade_sh_dc_0..2");
    s->exact = n_exact == 3;
    if (!s->exact && n_preview < 3)
        return ply_fail("RadFoam PLY vertex needs exact blade_sh_dc_0..2 or red/green/blue preview DC");
    for (int c = 0; c < 3; ++c) {
        if (s->exact && v.props[s->dc[c]].ty != Ty::F32)
            return ply_fail("RadFoam PLY blade_sh_dc_* must be float32");
        if (!s->exact && v.props[s->preview[c]].ty != Ty::U8)
            return ply_fail("RadFoam PLY preview colours must be uchar");
    }
    std::vector<std::pair<long, int>> rest;
    for (size_t i = 0; i < v.props.size(); ++i) {
        const std::string &nm = v.props[i].name;
        if (!starts_with(nm, "color_sh_")) continue;
        if (v.props[i].ty != Ty::F32) return ply_fail("RadFoam PLY property '%s' must be float32", nm.c_str());
        const std::string k = nm.substr(9);
        char *end = nullptr;
        const long idx = strtol(k.c_str(), &end, 10);
        if (k.empty() || !end || *end || idx < 0)
            return ply_fail("invalid RadFoam PLY property '%s'", nm.c_str());
        rest.emplace_back(idx, (int)i);
    }
    std::sort(rest.begin(), rest.end());
    for (size_t i = 0; i < rest.size(); ++i)
        if (rest[i].first != (long)i) return ply_fail("RadFoam PLY color_sh indices must be contiguous");
    if (rest.size() % 3)
        return ply_fail("RadFoam PLY color_sh property count %zu is not divisible by three", rest.size());
    const size_t comps = rest.size() / 3 + 1;
    if (comps == 1) {
        s->degree = 0;
    } else if (comps == 4) {
        s->degree = 1;
    } else if (comps == 9) {
        s->degree = 2;
    } else if (comps == 16) {
        s->degree = 3;
    } else {
        return ply_fail("RadFoam PLY has %zu SH components, expected a complete degree up to 3", comps);
    }
    for (auto &r : rest) s->rest.push_back(r.second);
    s->radius = find("radius");
    if (s->radius >= 0 && v.props[s->radius].ty != Ty::F32)
        return ply_fail("RadFoam PLY vertex radius must be float32");
    return BV_OK;
}

struct OpenPly {
    FILE *f = nullptr;
    Header h;
    Schema s;
    ~OpenPly() {
        if (f) fclose(f);
    }
};

bv_status open_ply(const char *path, OpenPly *o) {
    if (!path) return arg_fail("null path");
    o->f = fopen(path, "rb");
    if (!o->f) return arg_fail("cannot open the RadFoam PLY file");
    const bv_status st = read_header(o->f, &o->h);
    if (st != BV_OK) return st;
    return make_schema(o->h, &o->s);
}

float load_f32(const unsigned char *p) {
    float v;
    std::memcpy(&v, p, 4);
    return v;
}

uint32_t load_u32(const unsigned char *p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

// One property value parsed from an ASCII token (the reference's
// str::parse::<f32 | u32 | u8>); false for an invalid token.
bool parse_token(const std::string &tok, Ty ty, double *out) {
    const char *s = tok.c_str();
    char *end = nullptr;
    if (ty == Ty::F32) {
        *out = (double)strtof(s, &end);
        return end && !*end;
    }
    if (s[0] == '-' || s[0] == '+') return false;
    const unsigned long long v = strtoull(s, &end, 10);
    if (!end || *end || end == s) return false;
    if (ty == Ty::U8 && v > 255ull) return false;
    if (ty == Ty::U32 && v > 0xffffffffull) return false;
    *out = (double)v;
    return true;
}

}  // namespace

extern "C" {

bv_status bv_radfoam_ply_info(const char *path, bv_ply_info *out) {
    if (!out) return arg_fail("null argument");
    OpenPly o;
    const bv_status st = open_ply(path, &o);
    if (st != BV_OK) return st;
    std::memset(out, 0, sizeof(*out));
    out->num_points = (uint32_t)o.h.elements[0].count;
    out->num_adjacency = (uint32_t)o.h.elements[1].count;
    out->sh_degree = o.s.degree;
    out->has_radii = o.s.radius >= 0 ? 1u : 0u;
    return BV_OK;
}

bv_status bv_radfoam_ply_read(const char *path, float *points, float *sh, uint32_t *offsets,
                              uint32_t *neighbors, float *radii) {
    if (!points || !sh || !offsets) return arg_fail("null argument");
    OpenPly o;
    bv_status st = open_ply(path, &o);
    if (st != BV_OK) return st;
    const Element &ve = o.h.elements[0], &ae = o.h.elements[1];
    const uint32_t n = (uint32_t)ve.count, m = (uint32_t)ae.count;
    if (m > 0 && !neighbors) return arg_fail("null neighbors with a non-empty adjacency");
    if (o.s.radius >= 0 && !radii) return arg_fail("the file carries radii: pass a radii array");
    const Schema &s = o.s;
    const uint32_t K = (s.degree + 1) * (s.degree + 1);
    const size_t nprop = ve.props.size();
    std::vector<double> val(nprop);
    std::vector<uint32_t> adj(m);
    offsets[0] = 0;
    auto store = [&](uint32_t i) {
        points[4 * (size_t)i + 0] = (float)val[s.x];
        points[4 * (size_t)i + 1] = (float)val[s.y];
        points[4 * (size_t)i + 2] = (float)val[s.z];
        points[4 * (size_t)i + 3] = (float)val[s.density];
        offsets[i + 1] = (uint32_t)val[s.adjacency_offset];
        float *row = sh + (size_t)i * 3 * K;
        for (int c = 0; c < 3; ++c) {
            if (s.exact) {
                row[c] = (float)val[s.dc[c]];
            } else {  // set_preview_dc (radfoam_ply.rs:722-726), FP32 operations
                const float cf = (float)val[s.preview[c]];
                row[c] = (cf / 255.0f - 0.5f) / 0.2820948f;
            }
        }
        for (size_t k = 0; k < s.rest.size(); ++k) row[3 + k] = (float)val[s.rest[k]];
        if (radii && s.radius >= 0) radii[i] = (float)val[s.radius];
    };
    FILE *f = o.f;
    if (!o.h.ascii) {
        // decode_binary: the body is exactly n vertex rows then m uints
        if (fseek(f, 0, SEEK_END) != 0) return ply_fail("cannot size the RadFoam PLY body");
        const long end = ftell(f);
        const unsigned long long want = (unsigned long long)n * ve.row_bytes + (unsigned long long)m * 4;
        if (end < o.h.body_offset || (unsigned long long)(end - o.h.body_offset) != want)
            return ply_fail("RadFoam PLY binary body is %lld bytes, expected %llu",
                            (long long)(end - o.h.body_offset), want);
        fseek(f, o.h.body_offset, SEEK_SET);
        std::vector<unsigned char> buf(ve.row_bytes);
        for (uint32_t i = 0; i < n; ++i) {
            if (fread(buf.data(), 1, ve.row_bytes, f) != ve.row_bytes)
                return ply_fail("RadFoam PLY binary body is truncated");
            for (size_t p = 0; p < nprop; ++p) {
                const unsigned char *q = buf.data() + ve.props[p].offset;
                switch (ve.props[p].ty) {
                    case Ty::F32: val[p] = load_f32(q); break;
                    case Ty::U32: val[p] = load_u32(q); break;
                    case Ty::U8: val[p] = *q; break;
                }
            }
            store(i);
        }
        for (uint32_t k = 0; k < m; ++k) {
            unsigned char q[4];
            if (fread(q, 1, 4, f) != 4) return ply_fail("RadFoam PLY binary body is truncated");
            adj[k] = load_u32(q);
        }
    } else {
        // decode_ascii / read_ascii_data_line: blank and "comment" lines are
        // skipped; a row gives one token per declared property in order
        // (columns past them are ignored, too few is an error); data after
        // the last adjacency row is an error
        std::string line;
        bool too_long = false;
        auto next_row = [&]() -> int {  // 1 row, 0 end of file, -1 row too long
            while (read_line(f, line, kMaxAsciiRowBytes, &too_long)) {
                if (too_long) return -1;
                const auto w = words(line);
                if (!w.empty() && !starts_with(w[0], "comment")) return 1;
            }
            return 0;
        };
        for (uint32_t i = 0; i < n; ++i) {
            const int r = next_row();
            if (r < 0) return ply_fail("RadFoam PLY ASCII row exceeds %zu bytes", kMaxAsciiRowBytes);
            if (r == 0) return ply_fail("RadFoam PLY is missing ASCII vertex row %u", i);
            const auto w = words(line);
            if (w.size() < nprop) return ply_fail("RadFoam PLY ASCII vertex row %u has too few columns", i);
            for (size_t p = 0; p < nprop; ++p)
                if (!parse_token(w[p], ve.props[p].ty, &val[p]))
                    return ply_fail("invalid RadFoam PLY value for '%s'", ve.props[p].name.c_str());
            store(i);
        }
        for (uint32_t k = 0; k < m; ++k) {
            const int r = next_row();
            if (r < 0) return ply_fail("RadFoam PLY ASCII row exceeds %zu bytes", kMaxAsciiRowBytes);
            if (r == 0) return ply_fail("RadFoam PLY is missing ASCII adjacency row %u", k);
            double v = 0.0;
            if (!parse_token(words(line)[0], Ty::U32, &v)) return ply_fail("invalid RadFoam PLY adjacency row");
            adj[k] = (uint32_t)v;
        }
        const int r = next_row();
        if (r != 0) return ply_fail("unexpected trailing RadFoam PLY ASCII data");
    }
    // validate_csr (radfoam_ply.rs:1111-1139)
    for (uint32_t i = 0; i < n; ++i)
        if (offsets[i + 1] < offsets[i]) return ply_fail("invalid RadFoam PLY CSR offsets");
    if (n && offsets[n] != m) return ply_fail("invalid RadFoam PLY CSR offsets");
    for (uint32_t k = 0; k < m; ++k) {
        if (adj[k] >= n) return ply_fail("RadFoam PLY adjacency references a missing point");
        neighbors[k] = adj[k];
    }
    return BV_OK;
}

}  // extern "C"
