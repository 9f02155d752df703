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
    SLAK_B200_MESHINFO

    template<typename MESH_INFO>
    static void subdivideIteratively(MESH_INFO const& cmesh, MESH_INFO& rmesh, int target_level)
    {
        slak_b200_detail::run(cmesh, rmesh, target_level, SLAK_SCHEME_LAK, "LAK");
    }
};
