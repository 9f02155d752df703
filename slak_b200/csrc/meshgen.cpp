// meshgen.cpp -- seeded synthetic control meshes for the subdivision workloads.
//
// Host-side input generation only (no CUDA).  Every generator returns a
// closed, consistently oriented 2-manifold in the reference's input layout
// (include/Mesh.h:153-176 of GPUPeople/SLAK): face offsets `ptr` (F+1),
// corner vertex ids `ids` (N), 1-based corner positions `vals` (N) and
// float4 positions with w = 1.
//
//   torus            W x H quad torus, major radius R, minor radius r
//   icosphere        class-I geodesic sphere of frequency n (20 n^2 triangles)
//   mixed torus      torus with a seeded fraction of adjacent quad pairs merged
//                    (shared edge removed) and of quads split on a diagonal
//   capped cylinder  `segs` x `rings` quad cylinder closed by two triangle fans
//                    whose poles have valence `segs`
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unordered_map>
#include <vector>
#include <algorithm>
#include <tuple>
#include <array>

extern "C" {
typedef struct {
    int32_t type;            // 0 TRI, 1 QUAD, 2 POLY
    int32_t is_reduced;
    int64_t nfaces, nverts, nnz, max_face_order;
    int32_t* ptr;
    int32_t* ids;
    int32_t* vals;
    float* verts;
} mg_mesh;
}

namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed ^ 0x9E3779B97F4A7C15ull) {}
    uint64_t next()
    {   // splitmix64
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double sym(double a) { return (2.0 * uniform() - 1.0) * a; }
    double normal()
    {
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct Poly {
    std::vector<int32_t> ptr{0};
    std::vector<int32_t> ids;
    std::vector<double> pos;   // xyz per vertex
    void face(std::initializer_list<int32_t> f)
    {
        for (int32_t v : f) ids.push_back(v);
        ptr.push_back((int32_t)ids.size());
    }
    void face(const std::vector<int32_t>& f)
    {
        for (int32_t v : f) ids.push_back(v);
        ptr.push_back((int32_t)ids.size());
    }
};

int emit(const Poly& P, mg_mesh* out)
{
    std::memset(out, 0, sizeof(*out));
    const int64_t F = (int64_t)P.ptr.size() - 1, N = (int64_t)P.ids.size(), V = (int64_t)P.pos.size() / 3;
    int64_t maxo = 0, mino = 1 << 30;
    for (int64_t f = 0; f < F; ++f) {
        int64_t o = P.ptr[f + 1] - P.ptr[f];
        maxo = std::max(maxo, o);
        mino = std::min(mino, o);
    }
    out->type = (maxo == 4 && mino == 4) ? 1 : (maxo == 3 && mino == 3) ? 0 : 2;
    out->is_reduced = 1;
    out->nfaces = F; out->nverts = V; out->nnz = N; out->max_face_order = maxo;
    out->ptr = (int32_t*)std::malloc(sizeof(int32_t) * (F + 1));
    out->ids = (int32_t*)std::malloc(sizeof(int32_t) * (N ? N : 1));
    out->vals = (int32_t*)std::malloc(sizeof(int32_t) * (N ? N : 1));
    out->verts = (float*)std::malloc(sizeof(float) * 4 * (V ? V : 1));
    std::memcpy(out->ptr, P.ptr.data(), sizeof(int32_t) * (F + 1));
    std::memcpy(out->ids, P.ids.data(), sizeof(int32_t) * N);
    for (int64_t f = 0; f < F; ++f)
        for (int32_t c = P.ptr[f]; c < P.ptr[f + 1]; ++c) out->vals[c] = c - P.ptr[f] + 1;
    for (int64_t v = 0; v < V; ++v) {
        out->verts[4 * v + 0] = (float)P.pos[3 * v + 0];
        out->verts[4 * v + 1] = (float)P.pos[3 * v + 1];
        out->verts[4 * v + 2] = (float)P.pos[3 * v + 2];
        out->verts[4 * v + 3] = 1.0f;
    }
    return 0;
}

void torus_positions(Poly& P, int W, int H, double R, double r, double jitter, Rng& rng)
{
    P.pos.resize((size_t)3 * W * H);
    for (int i = 0; i < W; ++i)
        for (int j = 0; j < H; ++j) {
            double th = 6.283185307179586 * i / W, ph = 6.283185307179586 * j / H;
            double* p = &P.pos[3 * ((size_t)i * H + j)];
            p[0] = (R + r * std::cos(ph)) * std::cos(th) + rng.sym(jitter);
            p[1] = (R + r * std::cos(ph)) * std::sin(th) + rng.sym(jitter);
            p[2] = r * std::sin(ph) + rng.sym(jitter);
        }
}

}  // namespace

extern "C" {

void mg_free(mg_mesh* m)
{
    if (!m) return;
    std::free(m->ptr); std::free(m->ids); std::free(m->vals); std::free(m->verts);
    std::memset(m, 0, sizeof(*m));
}

// Quad torus: vertex (i,j) = i*H + j, face (i,j) = [v(i,j), v(i+1,j), v(i+1,j+1), v(i,j+1)].
int mg_torus(int W, int H, double R, double r, double jitter, uint64_t seed, mg_mesh* out)
{
    if (W < 3 || H < 3) return 1;
    Rng rng(seed);
    Poly P;
    torus_positions(P, W, H, R, r, jitter, rng);
    auto v = [&](int i, int j) { return (int32_t)(((i + W) % W) * H + ((j + H) % H)); };
    P.ids.reserve((size_t)4 * W * H);
    for (int i = 0; i < W; ++i)
        for (int j = 0; j < H; ++j) P.face({v(i, j), v(i + 1, j), v(i + 1, j + 1), v(i, j + 1)});
    return emit(P, out);
}

// Class-I geodesic sphere: every icosahedron face is cut into n^2 triangles,
// points are projected to the unit sphere and scaled radially by (1 + N(0, sigma)).
int mg_icosphere(int n, double sigma, uint64_t seed, mg_mesh* out)
{
    if (n < 1) return 1;
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    const double I[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                             {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    const int T[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                          {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                          {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    Poly P;
    // a grid point is identified exactly by its integer weights on the 12 icosahedron vertices
    std::map<std::tuple<int, int, int, int, int, int>, int32_t> key2id;
    auto vid = [&](int a, int wa, int b, int wb, int c, int wc) {
        std::array<std::pair<int, int>, 3> k = {{{a, wa}, {b, wb}, {c, wc}}};
        for (auto& e : k) if (e.second == 0) e.first = -1;
        std::sort(k.begin(), k.end());
        auto key = std::make_tuple(k[0].first, k[0].second, k[1].first, k[1].second, k[2].first, k[2].second);
        auto it = key2id.find(key);
        if (it != key2id.end()) return it->second;
        int32_t id = (int32_t)(P.pos.size() / 3);
        key2id.emplace(key, id);
        double p[3];
        for (int d = 0; d < 3; ++d) p[d] = (wa * I[a][d] + wb * I[b][d] + wc * I[c][d]) / n;
        double l = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        for (int d = 0; d < 3; ++d) P.pos.push_back(p[d] / l);
        return id;
    };
    for (int f = 0; f < 20; ++f) {
        int A = T[f][0], B = T[f][1], C = T[f][2];
        auto g = [&](int i, int j) { return vid(A, n - i - j, B, i, C, j); };
        for (int j = 0; j < n; ++j)
            for (int i = 0; i + j < n; ++i) {
                P.face({g(i, j), g(i + 1, j), g(i, j + 1)});
                if (i + j + 1 < n) P.face({g(i + 1, j), g(i + 1, j + 1), g(i, j + 1)});
            }
    }
    Rng rng(seed);
    for (size_t v = 0; v < P.pos.size() / 3; ++v) {
        double s = 1.0 + sigma * rng.normal();
        for (int d = 0; d < 3; ++d) P.pos[3 * v + d] *= s;
    }
    return emit(P, out);
}

// Torus with merged and split faces.  A seeded, shuffled walk over all 2WH
// adjacent face pairs removes the shared edge of a pair when neither end of the
// edge already lost an edge (valence stays >= 3 and merge groups stay straight
// chains) and the merged group stays within `max_group` quads (<= 8-gons for 3).
// Then a seeded fraction of the remaining single quads is split on a random
// diagonal.  Faces keep the order of their first quad.
int mg_mixed_torus(int W, int H, double R, double r, double merge_frac, double split_frac,
                   double jitter, int max_group, uint64_t seed, mg_mesh* out)
{
    if (W < 4 || H < 4) return 1;
    Rng rng(seed);
    Poly P;
    torus_positions(P, W, H, R, r, jitter, rng);
    const int64_t nf = (int64_t)W * H;
    auto v = [&](int i, int j) { return (int32_t)(((i + W) % W) * H + ((j + H) % H)); };
    auto fid = [&](int i, int j) { return (int64_t)((i + W) % W) * H + ((j + H) % H); };
    std::vector<std::array<int32_t, 4>> quad(nf);
    for (int i = 0; i < W; ++i)
        for (int j = 0; j < H; ++j) quad[fid(i, j)] = {v(i, j), v(i + 1, j), v(i + 1, j + 1), v(i, j + 1)};
    // candidate pairs: (face, dir) with dir 0 = (i+1,j) neighbour, 1 = (i,j+1)
    std::vector<int64_t> cand(2 * nf);
    for (int64_t k = 0; k < 2 * nf; ++k) cand[k] = k;
    for (int64_t k = 2 * nf - 1; k > 0; --k) std::swap(cand[k], cand[(int64_t)(rng.next() % (uint64_t)(k + 1))]);
    std::vector<uint8_t> vtouched((size_t)W * H, 0);
    std::vector<int64_t> grp(nf), gsize(nf, 1);
    for (int64_t f = 0; f < nf; ++f) grp[f] = f;
    auto root = [&](int64_t f) { while (grp[f] != f) f = grp[f] = grp[grp[f]]; return f; };
    std::vector<uint64_t> removed;   // undirected edge keys min*V+max
    const uint64_t VV = (uint64_t)W * H;
    int64_t target = (int64_t)std::llround(merge_frac * 2 * nf), merged = 0;
    for (int64_t k = 0; k < 2 * nf && merged < target; ++k) {
        int64_t f = cand[k] >> 1;
        int dir = (int)(cand[k] & 1);
        int i = (int)(f / H), j = (int)(f % H);
        int64_t g = dir == 0 ? fid(i + 1, j) : fid(i, j + 1);
        int32_t p = dir == 0 ? v(i + 1, j) : v(i, j + 1), q = v(i + 1, j + 1);
        if (vtouched[p] || vtouched[q]) continue;
        int64_t rf = root(f), rg = root(g);
        if (rf == rg || gsize[rf] + gsize[rg] > max_group) continue;
        vtouched[p] = vtouched[q] = 1;
        grp[rg] = rf; gsize[rf] += gsize[rg];
        removed.push_back((uint64_t)std::min(p, q) * VV + (uint64_t)std::max(p, q));
        ++merged;
    }
    std::sort(removed.begin(), removed.end());
    auto is_removed = [&](int32_t a, int32_t b) {
        uint64_t key = (uint64_t)std::min(a, b) * VV + (uint64_t)std::max(a, b);
        return std::binary_search(removed.begin(), removed.end(), key);
    };
    // members of each group, in face order
    std::vector<std::vector<int64_t>> members(nf);
    for (int64_t f = 0; f < nf; ++f) members[root(f)].push_back(f);
    // split candidates: single quads
    std::vector<int64_t> singles;
    for (int64_t f = 0; f < nf; ++f) if (gsize[root(f)] == 1) singles.push_back(f);
    for (int64_t k = (int64_t)singles.size() - 1; k > 0; --k)
        std::swap(singles[k], singles[(int64_t)(rng.next() % (uint64_t)(k + 1))]);
    int64_t nsplit = std::min<int64_t>((int64_t)std::llround(split_frac * nf), (int64_t)singles.size());
    std::vector<int8_t> split(nf, 0);
    for (int64_t k = 0; k < nsplit; ++k) split[singles[k]] = 1 + (int8_t)(rng.next() & 1);
    P.ids.reserve((size_t)4 * nf);
    std::vector<uint8_t> done(nf, 0);
    for (int64_t f = 0; f < nf; ++f) {
        if (done[f]) continue;
        const auto& m = members[root(f)];
        if (m.size() == 1) {
            const auto& Q = quad[f];
            if (split[f] == 1) { P.face({Q[0], Q[1], Q[2]}); P.face({Q[0], Q[2], Q[3]}); }
            else if (split[f] == 2) { P.face({Q[0], Q[1], Q[3]}); P.face({Q[1], Q[2], Q[3]}); }
            else P.face({Q[0], Q[1], Q[2], Q[3]});
            done[f] = 1;
            continue;
        }
        // boundary walk of the union of the group's quads
        std::unordered_map<int32_t, int32_t> nxt;
        for (int64_t g : m) {
            done[g] = 1;
            const auto& Q = quad[g];
            for (int k = 0; k < 4; ++k) {
                int32_t a = Q[k], b = Q[(k + 1) & 3];
                if (!is_removed(a, b)) nxt[a] = b;
            }
        }
        std::vector<int32_t> poly;
        int32_t start = quad[m[0]][0], cur = start;
        do {
            poly.push_back(cur);
            cur = nxt.at(cur);
        } while (cur != start && poly.size() <= nxt.size());
        if (cur != start) return 2;
        P.face(poly);
    }
    return emit(P, out);
}

// Capped cylinder: ring k (0..rings-1) at height -1 + 2k/(rings-1), radius 1;
// quads between rings, a triangle fan to a pole under ring 0 and over the last ring.
int mg_capped_cylinder(int segs, int rings, double jitter, uint64_t seed, mg_mesh* out)
{
    if (segs < 3 || rings < 2) return 1;
    Rng rng(seed);
    Poly P;
    auto v = [&](int k, int s) { return (int32_t)(k * segs + ((s + segs) % segs)); };
    for (int k = 0; k < rings; ++k)
        for (int s = 0; s < segs; ++s) {
            double a = 6.283185307179586 * s / segs;
            P.pos.push_back(std::cos(a) + rng.sym(jitter));
            P.pos.push_back(std::sin(a) + rng.sym(jitter));
            P.pos.push_back(-1.0 + 2.0 * k / (rings - 1) + rng.sym(jitter));
        }
    const int32_t pb = rings * segs, pt = pb + 1;
    P.pos.push_back(rng.sym(jitter)); P.pos.push_back(rng.sym(jitter)); P.pos.push_back(-1.0 + rng.sym(jitter));
    P.pos.push_back(rng.sym(jitter)); P.pos.push_back(rng.sym(jitter)); P.pos.push_back(1.0 + rng.sym(jitter));
    for (int s = 0; s < segs; ++s) P.face({pb, v(0, s + 1), v(0, s)});
    for (int k = 0; k + 1 < rings; ++k)
        for (int s = 0; s < segs; ++s) P.face({v(k, s), v(k, s + 1), v(k + 1, s + 1), v(k + 1, s)});
    for (int s = 0; s < segs; ++s) P.face({pt, v(rings - 1, s), v(rings - 1, s + 1)});
    return emit(P, out);
}

}  // extern "C"
