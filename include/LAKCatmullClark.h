// LAKCatmullClark.h -- drop-in for GPUPeople/SLAK's LibInclude/LAKCatmullClark.h
// (the LAK scheme, "Linear Algebra Kernels").
//
// Same names and shapes as the reference: struct LAKCatmullClark with the
// nested MeshInfo (LAKCatmullClark.h:95-156) and the static template
// subdivideIteratively (LAKCatmullClark.h:165-166), for
// MeshInfo<int, int, int, float> (LAKCatmullClarkImpl.cu:576-578).  LAK
// output carries ptr[i] = 4i, vals[i] = i%4 + 1, max_face_order = 4 and
// is_reduced = false.  Unlike the reference, the input's ids/vals are not
// sorted in place (LAKCatmullClarkImpl.cu:101,277,326): the input is read only.
#pragma once

#include "CatmullClark.h"

struct LAKCatmullClark
{
    // field names and defaults of the reference's LAKCatmullClark::Context
    // (LAKCatmullClark.h:38-76): value maps, the E and F matrices (CSC),
    // interior / boundary edge lists and the boundary bookkeeping of its
    // implementation; unused here
    template <typename MESH_INFO>
    struct Context {
        using offset_t = typename MESH_INFO::offset_t;
        using index_t = typename MESH_INFO::index_t;
        using value_t = typename MESH_INFO::value_t;
        size_t block_dim{256};
        bool is_initialized{false};
        value_t* d_map{nullptr};
        value_t* d_F_map{nullptr};
        value_t* d_map0{nullptr};
        value_t* d_map1{nullptr};
        index_t* d_order_buffer{nullptr};
        offset_t* d_E_ptr{nullptr};
        index_t* d_E_ids{nullptr};
        index_t* d_E_vals{nullptr};
        offset_t* d_F_ptr{nullptr};
        index_t* d_F_ids{nullptr};
        index_t* d_F_vals{nullptr};
        index_t* d_mapping_buffer{nullptr};
        index_t* d_face_adjacency{nullptr};
        index_t* d_internal0{nullptr};
        index_t* d_internal1{nullptr};
        index_t* d_intids{nullptr};
        index_t* d_external0{nullptr};
        index_t* d_external1{nullptr};
        index_t* d_extids{nullptr};
        index_t* d_f0{nullptr};
        index_t* d_f1{nullptr};
        bool has_boundary{true};
        index_t nextern{0};
        index_t nedges{0};
        index_t* d_nextern{nullptr};
        index_t* d_vextern{nullptr};
    };

    SLAK_B200_PROFILININFO

    SLAK_B200_MESHINFO

    template<typename MESH_INFO>
    static void subdivideIteratively(MESH_INFO const& cmesh, MESH_INFO& rmesh, int target_level)
    {
        slak_b200_detail::run(cmesh, rmesh, target_level, SLAK_SCHEME_LAK, "LAK");
    }
};
