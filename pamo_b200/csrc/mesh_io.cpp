// Mesh ingest and egress on the host: Wavefront OBJ text to the flat float /
// int arrays the C ABI takes (pamo_obj_parse), and back (pamo_obj_format).
// The reference's example.py:24-43 loads and saves meshes with trimesh; this is
// the same step without it.  Both run over line-aligned chunks of the text on
// all host threads; the result does not depend on the thread count.
//
// Reading follows the OBJ specification: `v x y z [w]` vertices (extra values
// ignored), `f` polygons whose corners are `i`, `i/t`, `i//n` or `i/t/n` (only
// the vertex index is used; 1-based, negative = relative to the vertices read
// so far), split into the fan (c0, c_k, c_k+1); every other statement is
// skipped.  Coordinates are read as doubles and rounded to float, as loading
// into float64 and then calling `.float()` does.  Line continuations (a
// trailing backslash) are not supported: such a `v` line reports an error.
#include <algorithm>
#include <charconv>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pamo_b200.h"

namespace {

struct Chunk {
    const char *b = nullptr, *e = nullptr;
    long long nv = 0, nt = 0;  // vertices and triangles in the chunk
    long long v0 = 0, t0 = 0;  // before it
    long long err = -1;        // byte offset of the first bad line
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r'; }

inline const char *skip_space(const char *p, const char *e)
{
    while (p < e && is_space(*p)) ++p;
    return p;
}

// a statement keyword of one letter ("v", "f") followed by a blank
inline bool keyword(const char *p, const char *e, char k)
{
    return p + 1 < e && p[0] == k && (p[1] == ' ' || p[1] == '\t');
}

int thread_count(long long len, int requested)
{
    int hw = (int)std::thread::hardware_concurrency();
    if (hw < 1) hw = 1;
    int n = requested > 0 ? requested : hw;
    long long by_size = len / (1 << 20) + 1;  // at least ~1 MB of text per thread
    if (n > by_size) n = (int)by_size;
    return n < 1 ? 1 : n;
}

std::vector<Chunk> split_lines(const char *text, long long len, int n)
{
    std::vector<Chunk> c(n);
    const char *end = text + len;
    const char *prev = text;
    for (int k = 0; k < n; ++k) {
        const char *cut = k + 1 == n ? end : text + len * (k + 1) / n;
        if (cut < prev) cut = prev;
        if (k + 1 < n) {
            const void *nl = memchr(cut, '\n', (size_t)(end - cut));
            cut = nl ? (const char *)nl + 1 : end;
        }
        c[k].b = prev;
        c[k].e = cut;
        prev = cut;
    }
    return c;
}

template <class F>
void run_threads(int n, F &&f)
{
    if (n == 1) {
        f(0);
        return;
    }
    std::vector<std::thread> t;
    t.reserve(n);
    for (int k = 0; k < n; ++k) t.emplace_back(f, k);
    for (auto &x : t) x.join();
}

// Counts the corners of the face statement starting at p (after "f"); -1 on a
// corner without a vertex index.
int count_corners(const char *p, const char *e)
{
    int k = 0;
    while (true) {
        p = skip_space(p, e);
        if (p >= e || *p == '#') break;
        const char *q = p;
        while (q < e && !is_space(*q)) ++q;
        if (*p == '/') return -1;
        ++k;
        p = q;
    }
    return k;
}

void scan_chunk(Chunk &c)
{
    const char *p = c.b;
    while (p < c.e) {
        const char *nl = (const char *)memchr(p, '\n', (size_t)(c.e - p));
        const char *le = nl ? nl : c.e;
        const char *s = skip_space(p, le);
        if (keyword(s, le, 'v')) {
            ++c.nv;
        } else if (keyword(s, le, 'f')) {
            int k = count_corners(s + 1, le);
            if (k < 3) {
                if (c.err < 0) c.err = s - c.b;
            } else {
                c.nt += k - 2;
            }
        }
        p = le + 1;
    }
}

bool parse_double(const char *&p, const char *e, double &out)
{
    p = skip_space(p, e);
    if (p < e && *p == '+') ++p;  // accepted by strtod, not by from_chars
    auto r = std::from_chars(p, e, out);
    if (r.ec != std::errc() || (r.ptr < e && !is_space(*r.ptr) && *r.ptr != '#')) return false;
    p = r.ptr;
    return true;
}

void parse_chunk(Chunk &c, long long total_v, float *verts, double *verts64, int *tris)
{
    const char *p = c.b;
    long long nv = c.v0, nt = c.t0;
    while (p < c.e) {
        const char *nl = (const char *)memchr(p, '\n', (size_t)(c.e - p));
        const char *le = nl ? nl : c.e;
        const char *s = skip_space(p, le);
        if (keyword(s, le, 'v')) {
            const char *q = s + 1;
            double x, y, z;
            if (!parse_double(q, le, x) || !parse_double(q, le, y) || !parse_double(q, le, z)) {
                c.err = s - c.b;
                return;
            }
            if (verts) {
                verts[3 * nv] = (float)x;
                verts[3 * nv + 1] = (float)y;
                verts[3 * nv + 2] = (float)z;
            }
            if (verts64) {
                verts64[3 * nv] = x;
                verts64[3 * nv + 1] = y;
                verts64[3 * nv + 2] = z;
            }
            ++nv;
        } else if (keyword(s, le, 'f')) {
            const char *q = s + 1;
            long long first = -1, last = -1;
            int k = 0;
            while (true) {
                q = skip_space(q, le);
                if (q >= le || *q == '#') break;
                long long idx = 0;
                auto r = std::from_chars(q, le, idx);
                if (r.ec != std::errc() || idx == 0) {
                    c.err = s - c.b;
                    return;
                }
                const long long v = idx > 0 ? idx - 1 : nv + idx;
                if (v < 0 || v >= total_v || v > 0x7fffffffLL) {
                    c.err = s - c.b;
                    return;
                }
                q = r.ptr;
                if (q < le && *q != '/' && !is_space(*q) && *q != '#') {
                    c.err = s - c.b;
                    return;
                }
                while (q < le && !is_space(*q)) ++q;  // "/t/n"
                if (k == 0) {
                    first = v;
                } else if (k >= 2) {
                    tris[3 * nt] = (int)first;
                    tris[3 * nt + 1] = (int)last;
                    tris[3 * nt + 2] = (int)v;
                    ++nt;
                }
                last = v;
                ++k;
            }
        }
        p = le + 1;
    }
}

}  // namespace

int pamo_obj_parse(const char *text, long long len, float *verts, double *verts_f64, long long cap_verts, int *tris,
                   long long cap_tris, int n_threads, long long *out_n_verts, long long *out_n_tris,
                   long long *out_err_offset)
{
    if (len < 0 || (len && !text) || !out_n_verts || !out_n_tris || cap_verts < 0 || cap_tris < 0 ||
        (cap_verts && !verts && !verts_f64) || (cap_tris && !tris))
        return PAMO_ERR_INVALID_ARG;
    if (out_err_offset) *out_err_offset = -1;
    const int n = thread_count(len, n_threads);
    std::vector<Chunk> c = split_lines(text, len, n);
    run_threads(n, [&](int k) { scan_chunk(c[k]); });
    long long nv = 0, nt = 0;
    for (auto &x : c) {
        if (x.err >= 0) {
            if (out_err_offset) *out_err_offset = (x.b - text) + x.err;
            return PAMO_ERR_INVALID_ARG;
        }
        x.v0 = nv;
        x.t0 = nt;
        nv += x.nv;
        nt += x.nt;
    }
    *out_n_verts = nv;
    *out_n_tris = nt;
    if (nv > cap_verts || nt > cap_tris) return PAMO_ERR_CAPACITY;
    run_threads(n, [&](int k) { parse_chunk(c[k], nv, verts, verts_f64, tris); });
    for (auto &x : c)
        if (x.err >= 0) {
            if (out_err_offset) *out_err_offset = (x.b - text) + x.err;
            return PAMO_ERR_INVALID_ARG;
        }
    return PAMO_OK;
}

int pamo_obj_format(const float *verts, long long n_verts, const int *tris, long long n_tris, char *out,
                    long long cap, int n_threads, long long *out_len)
{
    if (n_verts < 0 || n_tris < 0 || (n_verts && !verts) || (n_tris && !tris) || cap < 0 || (cap && !out) ||
        !out_len)
        return PAMO_ERR_INVALID_ARG;
    for (long long i = 0; i < 3 * n_tris; ++i)
        if (tris[i] < 0 || tris[i] >= n_verts) return PAMO_ERR_INVALID_ARG;
    const long long items = n_verts + n_tris;
    const int n = thread_count(items * 24, n_threads);
    std::vector<std::string> part(n);
    // thread k formats items [items k / n, items (k+1) / n): vertices first, then faces
    run_threads(n, [&](int k) {
        const long long lo = items * k / n, hi = items * (k + 1) / n;
        std::string &s = part[k];
        s.reserve((size_t)(hi - lo) * 40);
        char buf[96];
        for (long long i = lo; i < hi; ++i) {
            char *w = buf;
            if (i < n_verts) {
                *w++ = 'v';
                for (int a = 0; a < 3; ++a) {
                    *w++ = ' ';
                    w = std::to_chars(w, buf + sizeof(buf), verts[3 * i + a]).ptr;  // shortest exact form
                }
            } else {
                const long long t = i - n_verts;
                *w++ = 'f';
                for (int a = 0; a < 3; ++a) {
                    *w++ = ' ';
                    w = std::to_chars(w, buf + sizeof(buf), (long long)tris[3 * t + a] + 1).ptr;
                }
            }
            *w++ = '\n';
            s.append(buf, (size_t)(w - buf));
        }
    });
    long long total = 0;
    for (auto &s : part) total += (long long)s.size();
    *out_len = total;
    if (total > cap) return PAMO_ERR_CAPACITY;
    long long off = 0;
    for (auto &s : part) {
        memcpy(out + off, s.data(), s.size());
        off += (long long)s.size();
    }
    return PAMO_OK;
}
