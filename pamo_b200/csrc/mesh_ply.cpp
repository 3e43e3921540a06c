// Stanford PLY in and out on the host (pamo_ply_parse / pamo_ply_format): the
// second mesh format of the ingest step beside OBJ.  The reader takes ASCII,
// binary little-endian and binary big-endian files with any elements and
// properties: it needs an element `vertex` with properties x, y, z and reads
// the list property `vertex_indices` (or `vertex_index`) of an element `face`,
// splitting polygons into fans (c0, c_k, c_k+1); everything else is skipped.
// Coordinates are read as double, so `verts_f64` holds them exactly as stored
// (a float property widened) and `verts` rounds them to float once.  The
// writer emits binary little-endian: float x, y, z and `list uchar int`.
#include <charconv>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "pamo_b200.h"

namespace {

enum Type { T_NONE, T_I8, T_U8, T_I16, T_U16, T_I32, T_U32, T_F32, T_F64 };

Type type_of(const std::string &s)
{
    if (s == "char" || s == "int8") return T_I8;
    if (s == "uchar" || s == "uint8") return T_U8;
    if (s == "short" || s == "int16") return T_I16;
    if (s == "ushort" || s == "uint16") return T_U16;
    if (s == "int" || s == "int32") return T_I32;
    if (s == "uint" || s == "uint32") return T_U32;
    if (s == "float" || s == "float32") return T_F32;
    if (s == "double" || s == "float64") return T_F64;
    return T_NONE;
}

int size_of(Type t)
{
    switch (t) {
    case T_I8: case T_U8: return 1;
    case T_I16: case T_U16: return 2;
    case T_I32: case T_U32: case T_F32: return 4;
    case T_F64: return 8;
    default: return 0;
    }
}

struct Prop {
    std::string name;
    Type type = T_NONE, count_type = T_NONE;  // count_type set for a list
};

struct Element {
    std::string name;
    long long count = 0;
    std::vector<Prop> props;
};

enum Format { F_ASCII, F_LE, F_BE };

// Reads values in the file's encoding; every read is bounds-checked.
struct Reader {
    const char *p, *e;
    Format fmt;
    bool ok = true;

    bool next_token(const char *&b, const char *&t)
    {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
        if (p >= e) return false;
        b = p;
        while (p < e && !(*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
        t = p;
        return true;
    }

    double read(Type t)
    {
        if (!ok) return 0.0;
        if (fmt == F_ASCII) {
            const char *b, *q;
            if (!next_token(b, q)) {
                ok = false;
                return 0.0;
            }
            if (*b == '+') ++b;
            double v = 0.0;
            if (t == T_F32 || t == T_F64) {
                auto r = std::from_chars(b, q, v);
                ok = r.ec == std::errc() && r.ptr == q;
            } else {
                long long iv = 0;
                auto r = std::from_chars(b, q, iv);
                ok = r.ec == std::errc() && r.ptr == q;
                v = (double)iv;
            }
            return v;
        }
        const int n = size_of(t);
        if (n == 0 || e - p < n) {
            ok = false;
            return 0.0;
        }
        unsigned char b[8];
        memcpy(b, p, (size_t)n);
        p += n;
        if (fmt == F_BE)
            for (int i = 0; i < n / 2; ++i) std::swap(b[i], b[n - 1 - i]);
        switch (t) {
        case T_I8: { int8_t v; memcpy(&v, b, 1); return v; }
        case T_U8: return b[0];
        case T_I16: { int16_t v; memcpy(&v, b, 2); return v; }
        case T_U16: { uint16_t v; memcpy(&v, b, 2); return v; }
        case T_I32: { int32_t v; memcpy(&v, b, 4); return v; }
        case T_U32: { uint32_t v; memcpy(&v, b, 4); return v; }
        case T_F32: { float v; memcpy(&v, b, 4); return v; }
        case T_F64: { double v; memcpy(&v, b, 8); return v; }
        default: ok = false; return 0.0;
        }
    }
};

bool header(const char *data, long long len, Format &fmt, std::vector<Element> &els, long long &body)
{
    const char *p = data, *e = data + len;
    auto line = [&](std::string &out) {
        const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
        if (!nl) return false;
        out.assign(p, nl);
        if (!out.empty() && out.back() == '\r') out.pop_back();
        p = nl + 1;
        return true;
    };
    auto words = [](const std::string &s) {
        std::vector<std::string> w;
        size_t i = 0;
        while (i < s.size()) {
            while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) ++i;
            size_t j = i;
            while (j < s.size() && s[j] != ' ' && s[j] != '\t') ++j;
            if (j > i) w.emplace_back(s, i, j - i);
            i = j;
        }
        return w;
    };
    std::string l;
    if (!line(l) || l != "ply") return false;
    bool have_format = false;
    while (line(l)) {
        auto w = words(l);
        if (w.empty() || w[0] == "comment" || w[0] == "obj_info") continue;
        if (w[0] == "end_header") {
            body = p - data;
            return have_format;
        }
        if (w[0] == "format" && w.size() >= 2) {
            if (w[1] == "ascii") fmt = F_ASCII;
            else if (w[1] == "binary_little_endian") fmt = F_LE;
            else if (w[1] == "binary_big_endian") fmt = F_BE;
            else return false;
            have_format = true;
        } else if (w[0] == "element" && w.size() == 3) {
            Element el;
            el.name = w[1];
            auto r = std::from_chars(w[2].data(), w[2].data() + w[2].size(), el.count);
            if (r.ec != std::errc() || el.count < 0) return false;
            els.push_back(el);
        } else if (w[0] == "property" && !els.empty()) {
            Prop pr;
            if (w.size() == 5 && w[1] == "list") {
                pr.count_type = type_of(w[2]);
                pr.type = type_of(w[3]);
                pr.name = w[4];
                if (pr.count_type == T_NONE || pr.count_type == T_F32 || pr.count_type == T_F64) return false;
            } else if (w.size() == 3) {
                pr.type = type_of(w[1]);
                pr.name = w[2];
            } else {
                return false;
            }
            if (pr.type == T_NONE) return false;
            els.back().props.push_back(pr);
        } else {
            return false;
        }
    }
    return false;
}

// Walks the body; with `verts` / `tris` null only counts.  Returns false on a
// malformed or truncated body or an index outside the vertices.
bool body_pass(const char *data, long long len, long long body, Format fmt, const std::vector<Element> &els,
               long long &n_verts, long long &n_tris, float *verts, double *verts64, int *tris)
{
    Reader rd{data + body, data + len, fmt};
    long long nv = -1, nt = 0;
    for (const Element &el : els)
        if (el.name == "vertex") nv = el.count;
    if (nv < 0) return false;
    for (const Element &el : els) {
        const bool is_v = el.name == "vertex", is_f = el.name == "face";
        int ix = -1, iy = -1, iz = -1, il = -1;
        for (int k = 0; k < (int)el.props.size(); ++k) {
            const Prop &pr = el.props[k];
            if (is_v && pr.count_type == T_NONE) {
                if (pr.name == "x") ix = k;
                if (pr.name == "y") iy = k;
                if (pr.name == "z") iz = k;
            }
            if (is_f && pr.count_type != T_NONE && (pr.name == "vertex_indices" || pr.name == "vertex_index")) il = k;
        }
        if (is_v && (ix < 0 || iy < 0 || iz < 0)) return false;
        // an element without properties occupies no bytes: nothing to walk (and
        // a huge count must not spin the loop below)
        if (el.props.empty()) continue;
        long long t = 0;
        for (long long i = 0; i < el.count; ++i) {
            double xyz[3] = {0, 0, 0};
            for (int k = 0; k < (int)el.props.size(); ++k) {
                const Prop &pr = el.props[k];
                if (pr.count_type == T_NONE) {
                    const double v = rd.read(pr.type);
                    if (k == ix) xyz[0] = v;
                    if (k == iy) xyz[1] = v;
                    if (k == iz) xyz[2] = v;
                    continue;
                }
                const double cnt_d = rd.read(pr.count_type);
                if (!rd.ok || cnt_d < 0 || cnt_d > (double)(1 << 20)) return false;
                const long long cnt = (long long)cnt_d;
                if (k != il) {
                    for (long long j = 0; j < cnt; ++j) rd.read(pr.type);
                    continue;
                }
                if (cnt < 3) return false;
                long long first = 0, last = 0;
                for (long long j = 0; j < cnt; ++j) {
                    const double vd = rd.read(pr.type);
                    if (!rd.ok || vd < 0 || vd >= (double)nv || vd != (double)(long long)vd) return false;
                    const long long v = (long long)vd;
                    if (j == 0) first = v;
                    else if (j >= 2) {
                        if (tris) {
                            tris[3 * (nt + t)] = (int)first;
                            tris[3 * (nt + t) + 1] = (int)last;
                            tris[3 * (nt + t) + 2] = (int)v;
                        }
                        ++t;
                    }
                    last = v;
                }
            }
            if (!rd.ok) return false;
            if (is_v) {
                if (verts)
                    for (int a = 0; a < 3; ++a) verts[3 * i + a] = (float)xyz[a];
                if (verts64)
                    for (int a = 0; a < 3; ++a) verts64[3 * i + a] = xyz[a];
            }
        }
        if (is_f) nt += t;
    }
    n_verts = nv;
    n_tris = nt;
    return true;
}

}  // namespace

int pamo_ply_parse(const char *data, long long len, float *verts, double *verts_f64, long long cap_verts, int *tris,
                   long long cap_tris, long long *out_n_verts, long long *out_n_tris)
{
    if (len < 0 || (len && !data) || !out_n_verts || !out_n_tris || cap_verts < 0 || cap_tris < 0 ||
        (cap_verts && !verts && !verts_f64) || (cap_tris && !tris))
        return PAMO_ERR_INVALID_ARG;
    Format fmt = F_ASCII;
    std::vector<Element> els;
    long long body = 0, nv = 0, nt = 0;
    if (!header(data, len, fmt, els, body)) return PAMO_ERR_INVALID_ARG;
    if (!body_pass(data, len, body, fmt, els, nv, nt, nullptr, nullptr, nullptr)) return PAMO_ERR_INVALID_ARG;
    *out_n_verts = nv;
    *out_n_tris = nt;
    if (nv > cap_verts || nt > cap_tris || nv > 0x7fffffffLL) return PAMO_ERR_CAPACITY;
    if (!body_pass(data, len, body, fmt, els, nv, nt, verts, verts_f64, tris)) return PAMO_ERR_INVALID_ARG;
    return PAMO_OK;
}

int pamo_ply_format(const float *verts, long long n_verts, const int *tris, long long n_tris, char *out, long long cap,
                    long long *out_len)
{
    if (n_verts < 0 || n_tris < 0 || (n_verts && !verts) || (n_tris && !tris) || cap < 0 || (cap && !out) ||
        !out_len)
        return PAMO_ERR_INVALID_ARG;
    for (long long i = 0; i < 3 * n_tris; ++i)
        if (tris[i] < 0 || tris[i] >= n_verts) return PAMO_ERR_INVALID_ARG;
    const std::string head = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n_verts) +
                             "\nproperty float x\nproperty float y\nproperty float z\nelement face " +
                             std::to_string(n_tris) + "\nproperty list uchar int vertex_indices\nend_header\n";
    const long long total = (long long)head.size() + 12 * n_verts + 13 * n_tris;
    *out_len = total;
    if (total > cap) return PAMO_ERR_CAPACITY;
    // little-endian hosts only (x86-64, aarch64 as configured here)
    char *w = out;
    memcpy(w, head.data(), head.size());
    w += head.size();
    memcpy(w, verts, (size_t)(12 * n_verts));
    w += 12 * n_verts;
    for (long long t = 0; t < n_tris; ++t) {
        *w++ = 3;
        memcpy(w, tris + 3 * t, 12);
        w += 12;
    }
    return PAMO_OK;
}
