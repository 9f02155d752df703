/*
 * slak_oracle.h -- CPU restatement of the SLAK and LAK Catmull-Clark schemes.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * The product path (slak_b200/, include/) never links or calls it.
 *
 * Semantics: every atomic of the reference is serialized in ascending thread
 * order (the order a single-threaded execution of the reference kernels would
 * produce).  That fixes the reference's run-to-run nondeterminism (edge
 * numbering by atomicAdd slot order, float atomics) to one deterministic
 * answer, which the CUDA path reproduces bit-for-bit.  See slak_oracle.c for
 * per-function citations of the reference (GPUPeople/SLAK).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_TRI = 0, OR_QUAD = 1, OR_POLY = 2 };   /* MeshInfo::MeshType order, CatmullClark.h:72 */
enum { OR_LAK = 0, OR_SLAK = 1 };                 /* scheme ids of source/main.cpp:89-104 */

typedef struct {
    int32_t type;              /* OR_TRI / OR_QUAD / OR_POLY */
    int32_t is_reduced;
    int64_t nfaces, nverts, nnz, max_face_order;
    int32_t* ptr;              /* nfaces+1 (NULL allowed for a SLAK quad level) */
    int32_t* ids;              /* nnz */
    int32_t* vals;             /* nnz, 1-based corner position (LAK) ; may be NULL */
    float*   verts;            /* 4*nverts (x,y,z,w) */
    double*  verts64;          /* optional FP64 shadow positions, 4*nverts */
} or_mesh;

/* One subdivision level following the reference's per-level functions.
 * `poly` selects the first-level (arbitrary polygon) functions, otherwise the
 * quad functions.  Output arrays are malloc'ed; free with or_mesh_free.
 * Returns 0 on success, nonzero on a malformed mesh. */
int  or_level(const or_mesh* in, or_mesh* out, int scheme, int poly, int with_fp64);

/* Multi-level driver mirroring {LAK,}CatmullClark::subdivideIteratively
 * (CatmullClarkImpl.cu:457-515, LAKCatmullClarkImpl.cu:512-571): a non-QUAD
 * input always runs one polygon level, then quad levels up to target_level.
 * With target_level==0 and a QUAD input, out is left empty (nfaces==0). */
int  or_subdivide(const or_mesh* in, or_mesh* out, int target_level, int scheme, int with_fp64);

void or_mesh_free(or_mesh* m);

/* Number of OpenMP threads the oracle uses (1 when built without OpenMP). */
int  or_num_threads(void);

/* Set the thread count of later calls (n <= 0: back to the OpenMP default);
 * returns the count in effect. */
int  or_set_threads(int n);

#ifdef __cplusplus
}
#endif
