// objio.cpp -- Wavefront OBJ reading and writing on the host, in parallel.
//
// The reference reads meshes with OBJ::read (include/obj.h:107-257) into
// GPU::CSCMesh (include/Mesh.h:153-176): face offsets, 0-based corner vertex
// indices (negative OBJ indices count back from the vertices read so far),
// vals = the corner's 1-based position in its face, positions (x, y, z, 1),
// type TRI / QUAD / POLY from the face sizes.  This file produces the same
// arrays.  The file is split into newline-aligned chunks parsed by one thread
// each: a first pass counts each chunk's "v" lines, so a chunk knows how many
// vertices precede it and can resolve negative indices; a second pass parses.
// Writing formats chunks of lines in parallel and writes them in order.
//
// Crease tags.  OBJ::read keeps every "t" line as a Tag {type, intargs,
// floatargs} (include/obj.h:92-99, 202-229: "t <type> <ni>/<nf>/<ns>" then ni
// ints and nf floats); the reference never uses them.  slak_obj_read_creased
// turns "t crease" tags into crease pairs: the ni >= 2 ints are a chain of
// 0-based vertex ids v0 v1 ... (edges {v_j, v_j+1}), with one sharpness for
// the whole chain (nf == 1) or one per edge (nf == ni - 1).  slak_obj_read_sharp
// also reads "t corner" tags: ni >= 1 vertex ids with one sharpness or one
// each.  Other tag types are skipped.
#include "slak_b200.h"

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

struct Chunk {
    const char* b;
    const char* e;
    int64_t nv = 0;            // "v" lines in the chunk (first pass)
    std::vector<float> v;      // x, y, z per vertex
    std::vector<int32_t> fo;   // face sizes
    std::vector<int32_t> fi;   // corner vertex indices, 0-based
    std::vector<int32_t> cv;   // crease pairs (2 ids each), when tags are read
    std::vector<float> cs;     // their sharpness
    std::vector<int32_t> kv;   // corner vertices ("t corner"), when tags are read
    std::vector<float> ks;     // their sharpness
    int err_line = 0;          // nonzero: 1-based line (within the chunk) of a malformed face or tag
    int64_t lines = 0;
};

inline const char* skip_ws(const char* p, const char* e)
{
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    return p;
}

inline const char* line_end(const char* p, const char* e)
{
    const void* q = std::memchr(p, '\n', (size_t)(e - p));
    return q ? static_cast<const char*>(q) : e;
}

inline bool is_v(const char* p, const char* le) { return le - p >= 2 && p[0] == 'v' && (p[1] == ' ' || p[1] == '\t'); }
inline bool is_f(const char* p, const char* le) { return le - p >= 2 && p[0] == 'f' && (p[1] == ' ' || p[1] == '\t'); }
inline bool is_t(const char* p, const char* le) { return le - p >= 2 && p[0] == 't' && (p[1] == ' ' || p[1] == '\t'); }

// One "t" line (after the "t"): appends a crease tag's edges; false if malformed.
bool parse_tag(const char* q, const char* le, Chunk& c, bool corners)
{
    std::string line(q, le);
    const char* p = line.c_str();
    const char* e = p + line.size();
    p = skip_ws(p, e);
    const char* tb = p;
    while (p < e && *p != ' ' && *p != '\t' && *p != '\r') ++p;
    const std::string type(tb, p);
    char* end = nullptr;
    long n[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        p = skip_ws(p, e);
        n[k] = std::strtol(p, &end, 10);
        if (end == p || n[k] < 0) return false;
        p = end;
        if (k < 2) {
            if (p >= e || *p != '/') return false;
            ++p;
        }
    }
    const bool corner = corners && type == "corner";
    if (type != "crease" && !corner) return true;
    const long ni = n[0], nf = n[1];
    if (corner ? (ni < 1 || (nf != 1 && nf != ni)) : (ni < 2 || (nf != 1 && nf != ni - 1))) return false;
    if (ni > e - p || nf > e - p) return false;     // every value takes a character of the line at least
    std::vector<long> v((size_t)ni);
    for (long k = 0; k < ni; ++k) {
        p = skip_ws(p, e);
        v[(size_t)k] = std::strtol(p, &end, 10);
        if (end == p || v[(size_t)k] < 0 || v[(size_t)k] > INT32_MAX) return false;
        p = end;
    }
    std::vector<float> f((size_t)nf);
    for (long k = 0; k < nf; ++k) {
        p = skip_ws(p, e);
        f[(size_t)k] = std::strtof(p, &end);
        if (end == p) return false;
        p = end;
    }
    if (corner) {
        for (long k = 0; k < ni; ++k) {
            c.kv.push_back((int32_t)v[(size_t)k]);
            c.ks.push_back(nf == 1 ? f[0] : f[(size_t)k]);
        }
        return true;
    }
    for (long k = 0; k + 1 < ni; ++k) {
        c.cv.push_back((int32_t)v[(size_t)k]);
        c.cv.push_back((int32_t)v[(size_t)k + 1]);
        c.cs.push_back(nf == 1 ? f[0] : f[(size_t)k]);
    }
    return true;
}

void count_pass(Chunk& c)
{
    for (const char* p = c.b; p < c.e;) {
        const char* le = line_end(p, c.e);
        const char* s = skip_ws(p, le);
        if (is_v(s, le)) ++c.nv;
        p = le + 1;
    }
}

// base: vertices defined before this chunk; tags: read "t crease" lines;
// corners: also "t corner" lines
void parse_pass(Chunk& c, int64_t base, bool tags, bool corners)
{
    int64_t nv = base;
    std::string tmp;
    for (const char* p = c.b; p < c.e;) {
        const char* le = line_end(p, c.e);
        ++c.lines;
        const char* s = skip_ws(p, le);
        if (is_v(s, le)) {
            tmp.assign(s + 2, le);
            char* q = &tmp[0];
            char* end = nullptr;
            for (int k = 0; k < 3; ++k) {
                float x = std::strtof(q, &end);
                if (end == q) x = 0.f;
                c.v.push_back(x);
                q = end;
            }
            ++nv;
        } else if (is_f(s, le)) {
            int32_t order = 0;
            const char* q = s + 2;
            while (true) {
                q = skip_ws(q, le);
                if (q >= le) break;
                // one corner: v, v/vt, v//vn or v/vt/vn; only v is kept
                char* end = nullptr;
                long vi = std::strtol(q, &end, 10);
                if (end == q) { c.err_line = (int)c.lines; break; }
                const int64_t idx = vi < 0 ? nv + vi : (int64_t)vi - 1;
                if (vi == 0 || idx < 0 || idx > INT32_MAX) { c.err_line = (int)c.lines; break; }
                c.fi.push_back((int32_t)idx);
                ++order;
                q = end;
                while (q < le && *q != ' ' && *q != '\t' && *q != '\r') ++q;
            }
            if (c.err_line) break;
            c.fo.push_back(order);
        } else if (tags && is_t(s, le)) {
            if (!parse_tag(s + 1, le, c, corners)) { c.err_line = (int)c.lines; break; }
        }
        p = le + 1;
    }
}

int nthreads_for(size_t bytes)
{
    unsigned hc = std::thread::hardware_concurrency();
    const size_t by_size = bytes / (size_t(1) << 20) + 1;     // about 1 MB per thread at least
    return (int)std::max<size_t>(1, std::min<size_t>(hc ? hc : 1, by_size));
}

int obj_read(const char* path, slak_mesh* out, slak_creases* cr, slak_corners* ko = nullptr)
{
    if (!path || !out) return SLAK_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    if (cr) std::memset(cr, 0, sizeof(*cr));
    if (ko) std::memset(ko, 0, sizeof(*ko));
    FILE* f = std::fopen(path, "rb");
    if (!f) return SLAK_ERR_INVALID_ARG;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)std::max(size, 0L));
    const size_t got = size > 0 ? std::fread(buf.data(), 1, buf.size(), f) : 0;
    std::fclose(f);
    if (got != buf.size()) return SLAK_ERR_INVALID_ARG;
    const char* b = buf.data();
    const char* e = b + buf.size();

    const int nt = nthreads_for(buf.size());
    std::vector<Chunk> ch(nt);
    for (int t = 0; t < nt; ++t) {
        // chunk t ends after the line holding its nominal end point
        const char* cb = t == 0 ? b : ch[t - 1].e;
        const char* ce = t + 1 == nt ? e : b + buf.size() * (size_t)(t + 1) / (size_t)nt;
        if (ce < cb) ce = cb;
        if (ce < e) {
            const char* q = line_end(ce, e);
            ce = q < e ? q + 1 : e;
        }
        ch[t].b = cb;
        ch[t].e = ce;
    }
    auto run = [&](auto fn) {
        std::vector<std::thread> th;
        for (int t = 1; t < nt; ++t) th.emplace_back(fn, t);
        fn(0);
        for (auto& x : th) x.join();
    };
    run([&](int t) { count_pass(ch[t]); });
    std::vector<int64_t> vbase(nt + 1, 0);
    for (int t = 0; t < nt; ++t) vbase[t + 1] = vbase[t] + ch[t].nv;
    run([&](int t) { parse_pass(ch[t], vbase[t], cr != nullptr, ko != nullptr); });

    int64_t F = 0, N = 0, V = vbase[nt];
    for (auto& c : ch) {
        if (c.err_line) return SLAK_ERR_BAD_MESH;
        F += (int64_t)c.fo.size();
        N += (int64_t)c.fi.size();
    }
    if (N >= (int64_t(1) << 31) || V >= (int64_t(1) << 31)) return SLAK_ERR_UNSUPPORTED;
    int32_t* ptr = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)(F + 1)));
    int32_t* ids = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(N, 1)));
    int32_t* vals = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(N, 1)));
    float* verts = static_cast<float*>(std::malloc(sizeof(float) * 4 * (size_t)std::max<int64_t>(V, 1)));
    if (!ptr || !ids || !vals || !verts) {
        std::free(ptr); std::free(ids); std::free(vals); std::free(verts);
        return SLAK_ERR_OOM;
    }
    std::vector<int64_t> fbase(nt + 1, 0), nbase(nt + 1, 0);
    for (int t = 0; t < nt; ++t) {
        fbase[t + 1] = fbase[t] + (int64_t)ch[t].fo.size();
        nbase[t + 1] = nbase[t] + (int64_t)ch[t].fi.size();
    }
    int min_order = INT32_MAX, max_order = 0;
    for (auto& c : ch)
        for (int32_t o : c.fo) { min_order = std::min(min_order, (int)o); max_order = std::max(max_order, (int)o); }
    bool bad = F > 0 && min_order < 3;
    run([&](int t) {
        const Chunk& c = ch[t];
        int64_t off = nbase[t];
        for (size_t k = 0; k < c.fo.size(); ++k) {
            ptr[fbase[t] + (int64_t)k] = (int32_t)off;
            for (int32_t j = 0; j < c.fo[k]; ++j) vals[off + j] = j + 1;
            off += c.fo[k];
        }
        std::memcpy(ids + nbase[t], c.fi.data(), sizeof(int32_t) * c.fi.size());
        for (int64_t k = 0; k < c.nv; ++k) {
            float* o = verts + 4 * (vbase[t] + k);
            o[0] = c.v[3 * k]; o[1] = c.v[3 * k + 1]; o[2] = c.v[3 * k + 2]; o[3] = 1.0f;
        }
    });
    ptr[F] = (int32_t)N;
    for (int64_t c = 0; c < N && !bad; ++c) bad = ids[c] < 0 || ids[c] >= V;
    int64_t C = 0, K = 0;
    for (auto& c : ch) {
        C += (int64_t)c.cs.size();
        K += (int64_t)c.ks.size();
        for (int32_t x : c.cv) bad |= x < 0 || x >= V;
        for (int32_t x : c.kv) bad |= x < 0 || x >= V;
    }
    int32_t* kverts = nullptr;
    float* ksharp = nullptr;
    if (!bad && ko && K > 0) {
        kverts = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (size_t)K));
        ksharp = static_cast<float*>(std::malloc(sizeof(float) * (size_t)K));
        if (!kverts || !ksharp) {
            std::free(kverts); std::free(ksharp);
            std::free(ptr); std::free(ids); std::free(vals); std::free(verts);
            return SLAK_ERR_OOM;
        }
        int64_t o = 0;
        for (auto& c : ch) {
            std::memcpy(kverts + o, c.kv.data(), sizeof(int32_t) * c.kv.size());
            std::memcpy(ksharp + o, c.ks.data(), sizeof(float) * c.ks.size());
            o += (int64_t)c.ks.size();
        }
    }
    int32_t* cverts = nullptr;
    float* csharp = nullptr;
    if (!bad && cr && C > 0) {
        cverts = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * 2 * (size_t)C));
        csharp = static_cast<float*>(std::malloc(sizeof(float) * (size_t)C));
        if (!cverts || !csharp) {
            std::free(cverts); std::free(csharp); std::free(kverts); std::free(ksharp);
            std::free(ptr); std::free(ids); std::free(vals); std::free(verts);
            return SLAK_ERR_OOM;
        }
        int64_t o = 0;
        for (auto& c : ch) {
            std::memcpy(cverts + 2 * o, c.cv.data(), sizeof(int32_t) * c.cv.size());
            std::memcpy(csharp + o, c.cs.data(), sizeof(float) * c.cs.size());
            o += (int64_t)c.cs.size();
        }
    }
    if (bad) {
        std::free(ptr); std::free(ids); std::free(vals); std::free(verts);
        return SLAK_ERR_BAD_MESH;
    }
    if (cr) {
        cr->count = C;
        cr->verts = cverts;
        cr->sharpness = csharp;
    }
    if (ko) {
        ko->count = K;
        ko->verts = kverts;
        ko->sharpness = ksharp;
    }
    out->type = (F > 0 && min_order == 3 && max_order == 3) ? SLAK_MESH_TRI
              : (F > 0 && min_order == 4 && max_order == 4) ? SLAK_MESH_QUAD : SLAK_MESH_POLY;
    out->is_reduced = 1;
    out->nfaces = F;
    out->nverts = V;
    out->nnz = N;
    out->max_face_order = max_order;
    out->ptr = ptr;
    out->ids = ids;
    out->vals = vals;
    out->verts = verts;
    return SLAK_OK;
}

int obj_write(const char* path, const slak_mesh* m, const slak_creases* cr, const slak_corners* ko = nullptr)
{
    if (cr && cr->count < 0) return SLAK_ERR_INVALID_ARG;
    if (cr && cr->count > 0 && (!cr->verts || !cr->sharpness)) return SLAK_ERR_INVALID_ARG;
    if (ko && ko->count < 0) return SLAK_ERR_INVALID_ARG;
    if (ko && ko->count > 0 && (!ko->verts || !ko->sharpness)) return SLAK_ERR_INVALID_ARG;
    if (!path || !m || m->nverts < 0 || m->nfaces < 0 || (m->nverts > 0 && !m->verts)) return SLAK_ERR_INVALID_ARG;
    const int fixed = m->type == SLAK_MESH_QUAD ? 4 : m->type == SLAK_MESH_TRI ? 3 : 0;
    if (m->nfaces > 0 && (!m->ids || (!fixed && !m->ptr))) return SLAK_ERR_INVALID_ARG;
    // the faces are read through ptr / nnz: offsets that leave ids are refused
    // before anything is written
    if (fixed && m->nnz != (int64_t)fixed * m->nfaces) return SLAK_ERR_BAD_MESH;
    if (!fixed && m->nfaces > 0) {
        if (m->ptr[0] != 0 || (int64_t)m->ptr[m->nfaces] != m->nnz) return SLAK_ERR_BAD_MESH;
        for (int64_t g = 0; g < m->nfaces; ++g)
            if (m->ptr[g + 1] < m->ptr[g]) return SLAK_ERR_BAD_MESH;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return SLAK_ERR_INVALID_ARG;
    const int64_t V = m->nverts, F = m->nfaces;
    const int nt = nthreads_for((size_t)(V + F) * 32);
    std::vector<std::string> part(nt);
    // vertices, then faces; each thread formats a contiguous range of lines
    auto fmt_range = [&](int t) {
        std::string& s = part[t];
        char line[160];
        const int64_t vb = V * t / nt, ve = V * (t + 1) / nt;
        for (int64_t i = vb; i < ve; ++i) {
            const float* p = m->verts + 4 * i;
            const int n = std::snprintf(line, sizeof line, "v %.9g %.9g %.9g\n", p[0], p[1], p[2]);
            s.append(line, (size_t)n);
        }
    };
    std::vector<std::string> fpart(nt);
    auto fmt_faces = [&](int t) {
        std::string& s = fpart[t];
        char num[16];
        const int64_t fb = F * t / nt, fe = F * (t + 1) / nt;
        for (int64_t g = fb; g < fe; ++g) {
            const int64_t b = fixed ? g * fixed : m->ptr[g];
            const int64_t e = fixed ? b + fixed : m->ptr[g + 1];
            s.push_back('f');
            for (int64_t c = b; c < e; ++c) {
                const int n = std::snprintf(num, sizeof num, " %d", m->ids[c] + 1);
                s.append(num, (size_t)n);
            }
            s.push_back('\n');
        }
    };
    {
        std::vector<std::thread> th;
        for (int t = 1; t < nt; ++t) th.emplace_back([&, t] { fmt_range(t); fmt_faces(t); });
        fmt_range(0);
        fmt_faces(0);
        for (auto& x : th) x.join();
    }
    bool ok = true;
    for (auto& s : part) ok &= std::fwrite(s.data(), 1, s.size(), f) == s.size();
    for (auto& s : fpart) ok &= std::fwrite(s.data(), 1, s.size(), f) == s.size();
    if (cr) {
        char line[96];
        for (int64_t k = 0; k < cr->count && ok; ++k) {
            const int n = std::snprintf(line, sizeof line, "t crease 2/1/0 %d %d %.9g\n", cr->verts[2 * k],
                                        cr->verts[2 * k + 1], cr->sharpness[k]);
            ok &= std::fwrite(line, 1, (size_t)n, f) == (size_t)n;
        }
    }
    if (ko) {
        char line[96];
        for (int64_t k = 0; k < ko->count && ok; ++k) {
            const int n = std::snprintf(line, sizeof line, "t corner 1/1/0 %d %.9g\n", ko->verts[k], ko->sharpness[k]);
            ok &= std::fwrite(line, 1, (size_t)n, f) == (size_t)n;
        }
    }
    ok &= std::fclose(f) == 0;
    return ok ? SLAK_OK : SLAK_ERR_INVALID_ARG;
}

}  // namespace

extern "C" {

int slak_obj_read(const char* path, slak_mesh* out) { return obj_read(path, out, nullptr); }

int slak_obj_read_creased(const char* path, slak_mesh* out, slak_creases* creases)
{
    if (!creases) return SLAK_ERR_INVALID_ARG;
    return obj_read(path, out, creases);
}

int slak_obj_write(const char* path, const slak_mesh* m) { return obj_write(path, m, nullptr); }

int slak_obj_write_creased(const char* path, const slak_mesh* m, const slak_creases* creases)
{
    if (!creases) return SLAK_ERR_INVALID_ARG;
    return obj_write(path, m, creases);
}

int slak_obj_read_sharp(const char* path, slak_mesh* out, slak_creases* creases, slak_corners* corners)
{
    if (!creases || !corners) return SLAK_ERR_INVALID_ARG;
    return obj_read(path, out, creases, corners);
}

int slak_obj_write_sharp(const char* path, const slak_mesh* m, const slak_creases* creases,
                         const slak_corners* corners)
{
    return obj_write(path, m, creases, corners);
}

int slak_obj_free_corners(slak_corners* c)
{
    if (!c) return SLAK_ERR_INVALID_ARG;
    std::free(c->verts);
    std::free(c->sharpness);
    std::memset(c, 0, sizeof(*c));
    return SLAK_OK;
}

int slak_obj_free_creases(slak_creases* c)
{
    if (!c) return SLAK_ERR_INVALID_ARG;
    std::free(c->verts);
    std::free(c->sharpness);
    std::memset(c, 0, sizeof(*c));
    return SLAK_OK;
}

int slak_obj_free(slak_mesh* m)
{
    if (!m) return SLAK_ERR_INVALID_ARG;
    std::free(m->ptr);
    std::free(m->ids);
    std::free(m->vals);
    std::free(m->verts);
    std::memset(m, 0, sizeof(*m));
    return SLAK_OK;
}

}  // extern "C"
