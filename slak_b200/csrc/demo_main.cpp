// demo_main.cpp -- a host program written against the drop-in headers
// include/CatmullClark.h and include/LAKCatmullClark.h, in the shape of the
// reference's driver (source/main.cpp:84-113): build a control mesh, hand its
// device arrays to <scheme>::subdivideIteratively, read the refined mesh back.
//
//   slak_demo <torus|icosphere|cylinder|mixed> <scheme 0=LAK 1=SLAK> <level> <out.bin>
//
// out.bin: int64 nfaces, nverts, nnz, has_ptr; int32 ids[nnz]; float verts[4*nverts];
//          (LAK) int32 ptr[nfaces+1], vals[nnz]
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "CatmullClark.h"
#include "LAKCatmullClark.h"

extern "C" {
typedef struct {
    int32_t type, is_reduced;
    int64_t nfaces, nverts, nnz, max_face_order;
    int32_t* ptr;
    int32_t* ids;
    int32_t* vals;
    float* verts;
} mg_mesh;
int mg_torus(int W, int H, double R, double r, double jitter, uint64_t seed, mg_mesh* out);
int mg_icosphere(int n, double sigma, uint64_t seed, mg_mesh* out);
int mg_mixed_torus(int W, int H, double R, double r, double merge_frac, double split_frac, double jitter,
                   int max_group, uint64_t seed, mg_mesh* out);
int mg_capped_cylinder(int segs, int rings, double jitter, uint64_t seed, mg_mesh* out);
void mg_free(mg_mesh* m);
}

template <class MI>
void upload(const mg_mesh& h, MI& m)
{
    using T = typename MI::MeshType;
    m.type = h.type == 0 ? T::TRI : (h.type == 1 ? T::QUAD : T::POLY);
    m.nfaces = h.nfaces; m.nverts = h.nverts; m.nnz = h.nnz; m.max_face_order = h.max_face_order;
    m.is_reduced = true;
    slak_b200_detail::succeed(cudaMalloc((void**)&m.ptr, sizeof(int) * (h.nfaces + 1)));
    slak_b200_detail::succeed(cudaMalloc((void**)&m.ids, sizeof(int) * h.nnz));
    slak_b200_detail::succeed(cudaMalloc((void**)&m.vals, sizeof(int) * h.nnz));
    slak_b200_detail::succeed(cudaMalloc((void**)&m.verts, sizeof(float) * 4 * h.nverts));
    cudaMemcpy(m.ptr, h.ptr, sizeof(int) * (h.nfaces + 1), cudaMemcpyHostToDevice);
    cudaMemcpy(m.ids, h.ids, sizeof(int) * h.nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(m.vals, h.vals, sizeof(int) * h.nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(m.verts, h.verts, sizeof(float) * 4 * h.nverts, cudaMemcpyHostToDevice);
}

template <class S>
int run(const mg_mesh& h, int level, const char* path)
{
    typename S::template MeshInfo<int, int, int, float> cmesh, rmesh;
    upload(h, cmesh);
    try {
        S::subdivideIteratively(cmesh, rmesh, level);
    } catch (const char* e) {
        std::fprintf(stderr, "subdivision failed: %s\n", e);
        return 2;
    }
    std::vector<int32_t> ids(rmesh.nnz);
    std::vector<float> verts(4 * rmesh.nverts);
    cudaMemcpy(ids.data(), rmesh.ids, sizeof(int) * rmesh.nnz, cudaMemcpyDeviceToHost);
    cudaMemcpy(verts.data(), rmesh.verts, sizeof(float) * 4 * rmesh.nverts, cudaMemcpyDeviceToHost);
    int64_t hdr[4] = {(int64_t)rmesh.nfaces, (int64_t)rmesh.nverts, (int64_t)rmesh.nnz, rmesh.ptr != nullptr};
    FILE* f = std::fopen(path, "wb");
    if (!f) return 3;
    std::fwrite(hdr, sizeof hdr, 1, f);
    std::fwrite(ids.data(), sizeof(int32_t), ids.size(), f);
    std::fwrite(verts.data(), sizeof(float), verts.size(), f);
    if (rmesh.ptr) {
        std::vector<int32_t> ptr(rmesh.nfaces + 1), vals(rmesh.nnz);
        cudaMemcpy(ptr.data(), rmesh.ptr, sizeof(int) * ptr.size(), cudaMemcpyDeviceToHost);
        cudaMemcpy(vals.data(), rmesh.vals, sizeof(int) * vals.size(), cudaMemcpyDeviceToHost);
        std::fwrite(ptr.data(), sizeof(int32_t), ptr.size(), f);
        std::fwrite(vals.data(), sizeof(int32_t), vals.size(), f);
    }
    std::fclose(f);
    std::printf("Ctrl. Mesh: nf %zu nv %zu  Subd. Mesh: nf %zu nv %zu\n", cmesh.nfaces, cmesh.nverts, rmesh.nfaces,
                rmesh.nverts);
    rmesh.freeAndReset();
    cmesh.freeAndReset();     // the caller owns the input, as in the reference
    return 0;
}

int main(int argc, char** argv)
{
    if (argc != 5) {
        std::fprintf(stderr, "usage: slak_demo <torus|icosphere|cylinder|mixed> <scheme> <level> <out.bin>\n");
        return 1;
    }
    std::string w = argv[1];
    int scheme = std::atoi(argv[2]), level = std::atoi(argv[3]);
    mg_mesh h;
    int rc;
    if (w == "torus") rc = mg_torus(32, 32, 1.0, 0.3, 0.01, 11, &h);
    else if (w == "icosphere") rc = mg_icosphere(8, 0.02, 12, &h);
    else if (w == "cylinder") rc = mg_capped_cylinder(64, 32, 0.001, 15, &h);
    else rc = mg_mixed_torus(64, 48, 1.0, 0.3, 0.05, 0.03, 0.005, 3, 8, &h);
    if (rc) return 1;
    rc = scheme == 0 ? run<LAKCatmullClark>(h, level, argv[4]) : run<CatmullClark>(h, level, argv[4]);
    mg_free(&h);
    return rc;
}
