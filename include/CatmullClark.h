// CatmullClark.h -- drop-in for GPUPeople/SLAK's LibInclude/CatmullClark.h
// (the SLAK scheme, "Specialized LAK").
//
// Same names and shapes: struct CatmullClark with the nested
// MeshInfo<OFFSET, INDEX, VALUE, VERTEX> (CatmullClark.h:69-130 of the
// reference, freeAndReset() and freeAndReset(MEM_MANAGER&) included),
// Context<MESH_INFO> (:38-59), ProfilinInfo<PROFILER, MEM_MANAGER> (:62-67)
// and the static template subdivideIteratively (CatmullClark.h:163-164),
// usable for MeshInfo<int, int, int, float> (the only instantiation the
// reference provides, CatmullClarkImpl.cu:520-522).  The
// work runs in libslak_b200.so through the C ABI of slak_b200.h.
//
// Behaviour kept from the reference: device-resident input that is never
// freed or modified; output arrays cudaMalloc'ed and owned by the caller
// (freeAndReset releases them); a non-QUAD input always runs one polygon
// level; SLAK output has ptr = vals = nullptr and is_reduced = true; errors
// are thrown as `const char*` (cuda_host_helpers.h:34-41).  The report the
// reference prints after every call is printed only when SLAK_B200_VERBOSE=1.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include <cuda_runtime_api.h>

#include "slak_b200.h"

namespace slak_b200_detail {

inline void succeed(cudaError_t e)
{
    if (e != cudaSuccess) {
        std::printf("CUDA ERROR: %s", cudaGetErrorString(e));
        throw(cudaGetErrorString(e));
    }
}

// MeshInfo::freeAndReset(mem): the manager frees what it allocated
// (freeMemory returns true); anything else came from cudaMalloc
template <class MEM, class T>
void release(MEM& mem, T*& p)
{
    if (p != nullptr && !mem.freeMemory(p)) succeed(cudaFree(p));
    p = nullptr;
}

template <class MI>
slak_mesh to_c(const MI& m)
{
    slak_mesh c{};
    c.type = m.type == MI::MeshType::TRI ? SLAK_MESH_TRI : (m.type == MI::MeshType::QUAD ? SLAK_MESH_QUAD : SLAK_MESH_POLY);
    c.is_reduced = m.is_reduced ? 1 : 0;
    c.nfaces = (int64_t)m.nfaces;
    c.nverts = (int64_t)m.nverts;
    c.nnz = (int64_t)m.nnz;
    c.max_face_order = (int64_t)m.max_face_order;
    c.ptr = m.ptr;
    c.ids = m.ids;
    c.vals = m.vals;
    c.verts = m.verts;
    return c;
}

template <class MI>
void run(const MI& cmesh, MI& rmesh, int target_level, int scheme, const char* banner)
{
    static_assert(std::is_same<typename MI::offset_t, int>::value && std::is_same<typename MI::index_t, int>::value &&
                      std::is_same<typename MI::value_t, int>::value && std::is_same<typename MI::vertex_t, float>::value,
                  "subdivideIteratively is provided for MeshInfo<int, int, int, float> only");
    slak_mesh cin = to_c(cmesh);
    slak_mesh cout = to_c(rmesh);
    int rc = slak_subdivide(&cin, &cout, target_level, scheme, nullptr);
    if (rc != SLAK_OK) {
        std::printf("SLAK ERROR: %s %s\n", slak_status_string(rc), slak_last_error_detail());
        throw(slak_status_string(rc));
    }
    if (cout.ids != nullptr) {       // a level ran: the refined mesh replaces rmesh's arrays
        rmesh.type = MI::MeshType::QUAD;
        rmesh.is_reduced = cout.is_reduced != 0;
        rmesh.nfaces = (size_t)cout.nfaces;
        rmesh.nverts = (size_t)cout.nverts;
        rmesh.nnz = (size_t)cout.nnz;
        rmesh.max_face_order = (size_t)cout.max_face_order;
        rmesh.ptr = cout.ptr;
        rmesh.ids = cout.ids;
        rmesh.vals = cout.vals;
        rmesh.verts = cout.verts;
    }
    const char* v = std::getenv("SLAK_B200_VERBOSE");
    if (v && v[0] == '1')
        std::printf("==========%s==========\nSubdivision to level %d\nCtrl. Mesh:  nf: %zu  nv: %zu \n"
                    "Subd. Mesh:  nf: %zu  nv: %zu\n\n",
                    banner, target_level, (size_t)cmesh.nfaces, (size_t)cmesh.nverts, (size_t)rmesh.nfaces,
                    (size_t)rmesh.nverts);
}

}  // namespace slak_b200_detail

// The reference declares MeshInfo inside each scheme struct as a distinct
// 4-parameter class template (so template-template helpers such as
// CSCMeshCCMeshInfoConversion, include/Mesh.h:96-126, deduce it); both
// schemes' structs expand the same member list.
#define SLAK_B200_MESHINFO                                                                         \
    template <typename OFFSET_TYPE, typename INDEX_TYPE, typename VALUE_TYPE, typename VERTEX_TYPE> \
    struct MeshInfo {                                                                              \
        enum class MeshType { TRI, QUAD, POLY };                                                   \
        MeshType type;                                                                             \
        size_t nfaces{0};                                                                          \
        size_t nverts{0};                                                                          \
        size_t nnz{0};                                                                             \
        size_t max_face_order{0};                                                                  \
        bool is_reduced{false};                                                                    \
        using offset_t = OFFSET_TYPE;                                                              \
        OFFSET_TYPE* ptr{nullptr};                                                                 \
        using index_t = INDEX_TYPE;                                                                \
        INDEX_TYPE* ids{nullptr};                                                                  \
        using value_t = VALUE_TYPE;                                                                \
        VALUE_TYPE* vals{nullptr};                                                                 \
        using vertex_t = VERTEX_TYPE;                                                              \
        VERTEX_TYPE* verts{nullptr};                                                               \
        void reset() { *this = MeshInfo(); }                                                       \
        void freeAndReset()                                                                        \
        {                                                                                          \
            if (ptr != nullptr) slak_b200_detail::succeed(cudaFree(ptr));                          \
            if (ids != nullptr) slak_b200_detail::succeed(cudaFree(ids));                          \
            if (vals != nullptr) slak_b200_detail::succeed(cudaFree(vals));                        \
            if (verts != nullptr) slak_b200_detail::succeed(cudaFree(verts));                      \
            *this = MeshInfo();                                                                    \
        }                                                                                          \
        /* each array goes to mem.freeMemory(p) first; one the manager did */                     \
        /* not hand out (it returns false) is cudaFree'd                    */                     \
        template <typename MEM_MANAGER>                                                            \
        void freeAndReset(MEM_MANAGER& mem)                                                        \
        {                                                                                          \
            slak_b200_detail::release(mem, ptr);                                                   \
            slak_b200_detail::release(mem, ids);                                                   \
            slak_b200_detail::release(mem, vals);                                                  \
            slak_b200_detail::release(mem, verts);                                                 \
            *this = MeshInfo();                                                                    \
        }                                                                                          \
    };

// The reference's per-scheme scratch record (Context) and its pairing of a
// profiler with a memory manager (ProfilinInfo) are public nested types of
// each scheme's struct.  This library keeps its scratch in a plan and never
// reads a Context; the types exist so that host code naming them compiles.
#define SLAK_B200_PROFILININFO                                                                     \
    template <typename PROFILER_TYPE, typename MEM_MANAGER_TYPE>                                   \
    struct ProfilinInfo {                                                                          \
        PROFILER_TYPE prof;                                                                        \
        MEM_MANAGER_TYPE mem;                                                                      \
    };

struct CatmullClark
{
    // field names and defaults of the reference's CatmullClark::Context
    // (CatmullClark.h:38-59): adjacency, ordering and mapping buffers and the
    // boundary bookkeeping of its implementation; unused here
    template <typename MESH_INFO>
    struct Context {
        using index_t = typename MESH_INFO::index_t;
        size_t block_dim{256};
        bool is_initialized{false};
        index_t* d_order_buffer{nullptr};
        index_t* d_S_buffer{nullptr};
        index_t* d_mapping_buffer{nullptr};
        index_t* d_face_adjacency{nullptr};
        bool has_boundary{true};
        index_t nextern{0};
        index_t* d_nextern{nullptr};
        index_t* d_vextern{nullptr};
    };

    SLAK_B200_PROFILININFO

    SLAK_B200_MESHINFO

    template<typename MESH_INFO>
    static void subdivideIteratively(MESH_INFO const& cmesh, MESH_INFO& rmesh, int target_level)
    {
        slak_b200_detail::run(cmesh, rmesh, target_level, SLAK_SCHEME_SLAK, "SLAK");
    }
};
