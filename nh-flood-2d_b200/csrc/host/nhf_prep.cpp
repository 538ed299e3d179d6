// NE/NS mesh preprocessing on the host, in C++ (no CUDA): the text parser
// and the table builder of the reference's preprocess/domain.py, for meshes
// of millions of cells where the reference's per-line Python loops take
// minutes.
//
//   filter   _filter_ne_ns          (domain.py:221-347): drop NE rows whose
//            bed is -9999, renumber the kept cells 1.., drop NS rows left
//            without a neighbour across their orientation, renumber the kept
//            sides 1.., and rewrite both files' references;
//   cells    create_ne_fdb_compact  (domain.py:83-174): index, x, y, z, land
//            type, per-face side counts, face CSR pointers, side list;
//   sides    create_ns_fdb_parallel (domain.py:439-470): index, length, x, y,
//            z, attribute, topology (orient, lower, higher).
//
// Numbers parse as the reference parses them (Python int / float, i.e.
// correctly rounded doubles) and are stored as its tables store them (F32
// coordinates, u32 indices, u8 types).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../../include/nhf_prep.h"

struct nhp_mesh {
    std::vector<uint32_t> c_index, counts, ptr, isl;
    std::vector<float> cx, cy, cz;
    std::vector<uint8_t> ctype;
    std::vector<uint32_t> s_index, topo;
    std::vector<float> slen, sx, sy, sz;
    std::vector<uint8_t> sattr;
};

namespace {

thread_local std::string g_error;

int fail(const std::string &why)
{
    g_error = why;
    return -1;
}

struct Line {
    const char *b, *e;
};

std::vector<Line> split_lines(const char *text, size_t n)
{
    std::vector<Line> out;
    size_t i = 0;
    while (i < n) {
        size_t j = i;
        while (j < n && text[j] != '\n') ++j;
        size_t k = j;
        if (k > i && text[k - 1] == '\r') --k;
        out.push_back({text + i, text + k});
        i = j + 1;
    }
    return out;
}

// Fields of one line, split at commas (surrounding blanks belong to the field,
// as Python's int()/float() accept them).
void split_fields(const Line &l, std::vector<Line> &f)
{
    f.clear();
    const char *p = l.b;
    const char *start = p;
    for (; p < l.e; ++p)
        if (*p == ',') { f.push_back({start, p}); start = p + 1; }
    f.push_back({start, l.e});
}

bool parse_int(const Line &f, long long &v)
{
    std::string s(f.b, f.e);
    char *end = nullptr;
    errno = 0;
    v = strtoll(s.c_str(), &end, 10);
    if (end == s.c_str() || errno) return false;
    while (*end == ' ' || *end == '\t' || *end == '\r' || *end == '\n') ++end;
    return *end == 0;
}

bool parse_double(const Line &f, double &v)
{
    std::string s(f.b, f.e);
    char *end = nullptr;
    v = strtod(s.c_str(), &end);
    if (end == s.c_str()) return false;
    while (*end == ' ' || *end == '\t' || *end == '\r' || *end == '\n') ++end;
    return *end == 0;
}

bool blank(const Line &l)
{
    for (const char *p = l.b; p < l.e; ++p)
        if (*p != ' ' && *p != '\t') return false;
    return true;
}

}  // namespace

extern "C" {

const char *nhp_error(void) { return g_error.c_str(); }

int nhp_prepare(const char *ne_text, size_t ne_len, const char *ns_text, size_t ns_len, nhp_mesh **out)
{
    if (!out || (!ne_text && ne_len) || (!ns_text && ns_len)) return fail("null argument");
    *out = nullptr;
    std::vector<Line> ne = split_lines(ne_text, ne_len), ns = split_lines(ns_text, ns_len);
    while (!ne.empty() && blank(ne.back())) ne.pop_back();
    while (!ns.empty() && blank(ns.back())) ns.pop_back();
    std::vector<Line> f;
    // pass 1: kept cells
    std::unordered_map<long long, uint32_t> ne_map;
    ne_map.reserve(ne.size() * 2);
    std::vector<uint32_t> kept;
    kept.reserve(ne.size());
    for (size_t r = 0; r < ne.size(); ++r) {
        split_fields(ne[r], f);
        long long old;
        double z;
        if (f.size() < 9 || !parse_int(f[0], old) || !parse_double(f[f.size() - 2], z))
            return fail("NE line " + std::to_string(r + 1) + " is malformed");
        if (z != -9999.0) {
            ne_map[old] = (uint32_t)(kept.size() + 1);
            kept.push_back((uint32_t)r);
        }
    }
    // pass 2: kept sides
    nhp_mesh *m = new nhp_mesh();
    std::unordered_map<long long, uint32_t> ns_map;
    ns_map.reserve(ns.size() * 2);
    m->s_index.push_back(0); m->slen.push_back(0); m->sx.push_back(0); m->sy.push_back(0); m->sz.push_back(0);
    m->sattr.push_back(0); m->topo.insert(m->topo.end(), {0, 0, 0});
    for (size_t r = 0; r < ns.size(); ++r) {
        split_fields(ns[r], f);
        if (f.size() < 6) continue;
        long long old, orient, nb[4];
        bool ok = parse_int(f[0], old) && parse_int(f[1], orient);
        for (int k = 0; k < 4 && ok; ++k) ok = parse_int(f[2 + k], nb[k]);
        if (!ok) { delete m; return fail("NS line " + std::to_string(r + 1) + " is malformed"); }
        uint32_t mapped[4];
        for (int k = 0; k < 4; ++k) {
            auto it = ne_map.find(nb[k]);
            mapped[k] = it == ne_map.end() ? 0u : it->second;
        }
        bool keep = orient == 1 ? (mapped[2] != 0 || mapped[3] != 0) : (mapped[0] != 0 || mapped[1] != 0);
        if (!keep) continue;
        if (f.size() < 11) { delete m; return fail("NS line " + std::to_string(r + 1) + " has too few fields"); }
        double v[4], attr;
        for (int k = 0; k < 4; ++k)
            if (!parse_double(f[6 + k], v[k])) { delete m; return fail("NS line " + std::to_string(r + 1) + " is malformed"); }
        if (!parse_double(f[10], attr)) { delete m; return fail("NS line " + std::to_string(r + 1) + " is malformed"); }
        uint32_t id = (uint32_t)m->s_index.size();
        ns_map[old] = id;
        m->s_index.push_back(id);
        m->slen.push_back((float)v[0]); m->sx.push_back((float)v[1]); m->sy.push_back((float)v[2]);
        m->sz.push_back((float)v[3]);
        m->sattr.push_back((uint8_t)(long long)attr);
        if (orient == 1) m->topo.insert(m->topo.end(), {(uint32_t)orient, mapped[2], mapped[3]});
        else m->topo.insert(m->topo.end(), {(uint32_t)orient, mapped[0], mapped[1]});
    }
    // pass 3: cell tables with renumbered side references
    const size_t e = kept.size() + 1;
    m->c_index.assign(e, 0); m->cx.assign(e, 0); m->cy.assign(e, 0); m->cz.assign(e, 0); m->ctype.assign(e, 0);
    m->counts.assign(e * 4, 0); m->ptr.assign(e * 4, 0);
    uint32_t offset = 0;
    for (size_t i = 1; i < e; ++i) {
        split_fields(ne[kept[i - 1]], f);
        long long c[4];
        bool ok = true;
        for (int k = 0; k < 4 && ok; ++k) ok = parse_int(f[1 + k], c[k]) && c[k] >= 0;
        long long total = ok ? c[0] + c[1] + c[2] + c[3] : 0;
        if (!ok || (long long)f.size() < 5 + total + 4) { delete m; return fail("NE line " + std::to_string(kept[i - 1] + 1) + " is malformed"); }
        for (long long k = 0; k < total; ++k) {
            long long sid;
            if (!parse_int(f[5 + k], sid)) { delete m; return fail("NE line " + std::to_string(kept[i - 1] + 1) + " is malformed"); }
            auto it = ns_map.find(sid);
            m->isl.push_back(it == ns_map.end() ? 0u : it->second);
        }
        double x, y, z;
        long long land;
        const size_t n = f.size();
        if (!parse_double(f[n - 4], x) || !parse_double(f[n - 3], y) || !parse_double(f[n - 2], z) ||
            !parse_int(f[n - 1], land)) { delete m; return fail("NE line " + std::to_string(kept[i - 1] + 1) + " is malformed"); }
        m->c_index[i] = (uint32_t)i;
        m->cx[i] = (float)x; m->cy[i] = (float)y; m->cz[i] = (float)z;
        m->ctype[i] = (uint8_t)land;
        for (int k = 0; k < 4; ++k) m->counts[4 * i + k] = (uint32_t)c[k];
        m->ptr[4 * i] = offset;
        m->ptr[4 * i + 1] = offset + (uint32_t)c[0];
        m->ptr[4 * i + 2] = offset + (uint32_t)(c[0] + c[1]);
        m->ptr[4 * i + 3] = offset + (uint32_t)(c[0] + c[1] + c[2]);
        offset += (uint32_t)total;
    }
    *out = m;
    return 0;
}

int nhp_sizes(const nhp_mesh *m, int64_t sizes[3])
{
    if (!m || !sizes) return fail("null argument");
    sizes[0] = (int64_t)m->c_index.size();
    sizes[1] = (int64_t)m->s_index.size();
    sizes[2] = (int64_t)m->isl.size();
    return 0;
}

int nhp_copy_cells(const nhp_mesh *m, uint32_t *index, float *x, float *y, float *z, uint8_t *type,
                   uint32_t *counts, uint32_t *ptr, uint32_t *isl)
{
    if (!m) return fail("null argument");
    const size_t e = m->c_index.size();
    if (index) memcpy(index, m->c_index.data(), e * 4);
    if (x) memcpy(x, m->cx.data(), e * 4);
    if (y) memcpy(y, m->cy.data(), e * 4);
    if (z) memcpy(z, m->cz.data(), e * 4);
    if (type) memcpy(type, m->ctype.data(), e);
    if (counts) memcpy(counts, m->counts.data(), e * 16);
    if (ptr) memcpy(ptr, m->ptr.data(), e * 16);
    if (isl && !m->isl.empty()) memcpy(isl, m->isl.data(), m->isl.size() * 4);
    return 0;
}

int nhp_copy_sides(const nhp_mesh *m, uint32_t *index, float *length, float *x, float *y, float *z, uint8_t *attr,
                   uint32_t *topo)
{
    if (!m) return fail("null argument");
    const size_t s = m->s_index.size();
    if (index) memcpy(index, m->s_index.data(), s * 4);
    if (length) memcpy(length, m->slen.data(), s * 4);
    if (x) memcpy(x, m->sx.data(), s * 4);
    if (y) memcpy(y, m->sy.data(), s * 4);
    if (z) memcpy(z, m->sz.data(), s * 4);
    if (attr) memcpy(attr, m->sattr.data(), s);
    if (topo) memcpy(topo, m->topo.data(), s * 12);
    return 0;
}

void nhp_free(nhp_mesh *m) { delete m; }

}  // extern "C"
