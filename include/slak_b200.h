/*
 * slak_b200.h -- C ABI of the B200-native Catmull-Clark subdivision library.
 *
 * Each entry point names the interface of GPUPeople/SLAK it replaces
 * (path:line inside that project).  All mesh arrays passed here live in
 * device memory unless stated otherwise; sizes are element counts.
 *
 * Mesh layout (the reference's MeshInfo<int,int,int,float>,
 * LibInclude/CatmullClark.h:69-130 and LibInclude/LAKCatmullClark.h:95-156):
 *   ptr   nfaces+1 face offsets (may be NULL for a SLAK quad mesh)
 *   ids   nnz corner vertex ids, corners of a face in cyclic order
 *   vals  nnz 1-based corner positions (LAK input and output)
 *   verts 4*nverts floats (x, y, z, w)
 * A refined mesh is all quads; quad q is coarse corner q and holds
 * {v, V+F+edge(q), V+face(q), V+F+edge(prev(q))}; its vertices are laid out
 * [V updated originals | F face points | E edge points].
 */
#ifndef SLAK_B200_H
#define SLAK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLAK_B200_ABI_VERSION 1

/* ABI-compatible with cudaStream_t; NULL selects the legacy default stream. */
typedef struct CUstream_st* slak_stream_t;

enum slak_mesh_type { SLAK_MESH_TRI = 0, SLAK_MESH_QUAD = 1, SLAK_MESH_POLY = 2 };
enum slak_scheme { SLAK_SCHEME_LAK = 0, SLAK_SCHEME_SLAK = 1 };

enum slak_status {
    SLAK_OK = 0,
    SLAK_ERR_INVALID_ARG = 1,   /* null pointer, negative count, unknown scheme          */
    SLAK_ERR_CUDA = 2,          /* a CUDA runtime call failed                             */
    SLAK_ERR_OOM = 3,           /* device allocation failed                               */
    SLAK_ERR_BAD_MESH = 4,      /* index out of range, face order < 3, non-manifold edge  */
    SLAK_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up                     */
    SLAK_ERR_UNSUPPORTED = 6,   /* size beyond int32 indexing                             */
    SLAK_ERR_NOT_READY = 7      /* a plan was queried before it ran                       */
};

typedef struct slak_mesh {
    int32_t type;               /* enum slak_mesh_type */
    int32_t is_reduced;
    int64_t nfaces;
    int64_t nverts;
    int64_t nnz;
    int64_t max_face_order;
    int32_t* ptr;
    int32_t* ids;
    int32_t* vals;
    float* verts;
} slak_mesh;

/* Human-readable text of a status code (never NULL). */
const char* slak_status_string(int status);

/* SLAK_B200_ABI_VERSION of the loaded library. */
int slak_abi_version(void);

/* Detail of the last failure on the calling thread (the CUDA error text and,
 * with SLAK_DEBUG_SYNC=1 set when the plan was created, the kernel that
 * failed); empty if none.  The reference printed CUDA errors before throwing
 * (LibInclude/cuda_host_helpers.h:34-41). */
const char* slak_last_error_detail(void);

/*
 * Replaces CatmullClark::subdivideIteratively (LibSource/device/CatmullClarkImpl.cu:457-515)
 * and LAKCatmullClark::subdivideIteratively (LibSource/device/LAKCatmullClarkImpl.cu:512-571);
 * scheme SLAK_SCHEME_SLAK / SLAK_SCHEME_LAK as in source/main.cpp:89-104.
 * A non-QUAD input always runs one polygon level, then quad levels until
 * target_level; a QUAD input with target_level <= 0 leaves *rmesh zeroed.
 * The input is not modified.  The output arrays are cudaMalloc'ed and owned by
 * the caller (free them with slak_mesh_free or cudaFree, like
 * MeshInfo::freeAndReset, CatmullClark.h:99-106).  SLAK output: ptr = vals =
 * NULL, is_reduced = 1, max_face_order copied from the input; LAK output:
 * ptr[i] = 4i, vals[i] = i%4+1, max_face_order = 4, is_reduced = 0.
 * Work is ordered on `stream`; the call returns once the refined mesh is
 * complete (the reference is synchronous too).  Intermediate levels live in a
 * per-device workspace that is kept for the next call (the reference
 * allocates and frees them inside every call); a call made while another
 * holds the workspace allocates its own.  SLAK_WORKSPACE_CACHE=0 in the
 * environment turns the cache off.
 */
int slak_subdivide(const slak_mesh* cmesh, slak_mesh* rmesh, int target_level, int scheme,
                   slak_stream_t stream);

/*
 * Mesh files (host memory).  slak_obj_read replaces OBJ::read + the
 * GPU::CSCMesh(path) constructor (include/obj.h:107-257,
 * include/Mesh.h:153-176): it fills *out with host arrays (malloc) in the
 * MeshInfo layout -- face offsets ptr (F+1), 0-based corner ids (N), vals =
 * each corner's 1-based position in its face, verts = (x, y, z, 1) -- and the
 * type TRI / QUAD / POLY from the face sizes.  "v" and "f" lines are read
 * ("f" corners as v, v/vt, v//vn or v/vt/vn; negative indices count back from
 * the vertices read so far); other lines are skipped.  A face with fewer than
 * three corners or an index out of range gives SLAK_ERR_BAD_MESH.  The file is
 * parsed by several threads.  Release with slak_obj_free.
 * slak_obj_write replaces OBJ::write (include/obj.h:259-297) for a host mesh:
 * "v x y z" lines (9 significant digits, so float32 positions read back
 * exactly) and 1-based "f" lines (QUAD / TRI faces need no ptr).
 */
int slak_obj_read(const char* path, slak_mesh* out);
int slak_obj_write(const char* path, const slak_mesh* host_mesh);
int slak_obj_free(slak_mesh* host_mesh);

/* Crease pairs of a mesh (host or device memory, as the call says):
 * 2 * count vertex ids and count sharpness values. */
typedef struct slak_creases {
    int64_t count;
    int32_t* verts;
    float* sharpness;
} slak_creases;

/* As slak_obj_read, and also turns the file's "t crease" tags into host
 * crease pairs (malloc; release with slak_obj_free_creases).  OBJ::read keeps
 * every "t <type> <ni>/<nf>/<ns> ints... floats..." line as a Tag
 * (include/obj.h:92-99, 202-229) that the reference never uses.  Here a
 * crease tag's ni >= 2 ints are a chain of 0-based vertex ids (edges
 * {v_j, v_j+1}) with one sharpness (nf == 1) or one per edge (nf == ni - 1);
 * other tag types are skipped; a malformed crease tag or an id out of range
 * gives SLAK_ERR_BAD_MESH.  slak_obj_write_creased appends one
 * "t crease 2/1/0 a b s" line per pair. */
int slak_obj_read_creased(const char* path, slak_mesh* out, slak_creases* creases);
int slak_obj_write_creased(const char* path, const slak_mesh* host_mesh, const slak_creases* creases);
int slak_obj_free_creases(slak_creases* creases);

/* Corner vertices of a mesh: count vertex ids and count sharpness values. */
typedef struct slak_corners {
    int64_t count;
    int32_t* verts;
    float* sharpness;
} slak_corners;

/* As slak_obj_read_creased, and also reads "t corner" tags: ni >= 1 0-based
 * vertex ids with one sharpness (nf == 1) or one each (nf == ni) (host
 * arrays, malloc; release with slak_obj_free_corners).  slak_obj_write_sharp
 * appends the crease lines (creases may be NULL), then one
 * "t corner 1/1/0 v s" line per corner (corners may be NULL). */
int slak_obj_read_sharp(const char* path, slak_mesh* out, slak_creases* creases, slak_corners* corners);
int slak_obj_write_sharp(const char* path, const slak_mesh* host_mesh, const slak_creases* creases,
                         const slak_corners* corners);
int slak_obj_free_corners(slak_corners* corners);

/* Frees the current device's cached slak_subdivide workspace.  No counterpart
 * in the reference, whose calls keep nothing between them.  Returns
 * SLAK_ERR_NOT_READY while a call holds the workspace. */
int slak_workspace_release(void);

/* cudaFree of every non-NULL array, then zero the descriptor
 * (MeshInfo::freeAndReset, CatmullClark.h:99-106). */
int slak_mesh_free(slak_mesh* mesh);

/*
 * One subdivision level that allocates no device memory.  No counterpart in the
 * reference.  It is meant for callers that cannot call cudaMalloc: an
 * application whose device memory is owned by its own pool allocator, or a
 * latency-critical loop that must not hit cudaMalloc/cudaFree, since those can
 * synchronise the device and take unbounded time.
 *
 * Runs the reference's first-level functions for a non-QUAD cmesh (the quad
 * functions for a QUAD cmesh), exactly as slak_subdivide with target_level 1.
 * The caller allocates the outputs:
 *   rmesh->ids    4*nnz ints
 *   rmesh->verts  4*rmesh->nverts floats; on entry rmesh->nverts is the buffer's
 *                 capacity in vertices (nverts + nfaces + nnz always suffices)
 *   rmesh->ptr, rmesh->vals   nnz+1 and 4*nnz ints, LAK only
 * On success, the counts in *rmesh are set as slak_subdivide sets them.
 *
 * The scratch is a fixed 32 MiB device array inside this library.  Every GPU
 * that loads the library holds it until the process exits.  A level needs
 * 36 bytes of scratch per corner (40 for a non-QUAD cmesh) plus 16 per vertex,
 * each of its 13-14 arrays rounded up to 256 bytes, plus its scan tiles
 * (4 bytes per 2048 corners) and a status record; meshes whose scratch does
 * not fit are rejected with SLAK_ERR_UNSUPPORTED before anything runs.  That
 * is about 830k corners for a closed quad mesh (vertices = corners / 4).
 * All calls share that array:
 *   - calls that overlap on the GPU (two streams, or two host threads) race,
 *     so serialise them;
 *   - each call clears what must start at zero.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before
 * any stream capture.  The call waits for `stream` twice: for the level's edge
 * count and for its status.
 */
int slak_subdivide_level_noalloc(const slak_mesh* cmesh, slak_mesh* rmesh, int scheme, slak_stream_t stream);

/*
 * Plans: the same computation with every size fixed up front, all device
 * memory allocated at creation and nothing allocated or synchronised when it
 * runs, so one execution can be captured in a CUDA graph.  No reference
 * counterpart (the reference allocates inside every level,
 * LibInclude/profiling.h:37-162); slak_subdivide is built on it.
 *
 * slak_plan_create reads the input's topology once (one stream sync) to size
 * all levels.  slak_plan_execute re-runs every level from the current
 * contents of cmesh's arrays, which must keep the same topology.  The refined
 * mesh stays owned by the plan (slak_plan_output) until slak_plan_release_output
 * hands the arrays to the caller.
 */
typedef struct slak_plan slak_plan;

enum slak_plan_flags {
    SLAK_PLAN_GRAPH = 1,        /* capture one execution as a CUDA graph and replay it       */
    SLAK_PLAN_GENERAL = 2,      /* run every level through the general per-level path         */
    SLAK_PLAN_COMPENSATED = 4,  /* compensated (TwoSum) sums in high-valence vertex points    */
    SLAK_PLAN_TIMING = 8,       /* record a CUDA event after every launch (per-kernel times)  */
    SLAK_PLAN_AUTOTUNE = 16,    /* measure launch shapes of untuned keys at creation (below)  */
    SLAK_PLAN_GQ = 32,          /* grandparent-quad levels: k_g1 sums most of the parent's    */
                                /* vertex columns instead of k_g3 (same results)             */
    SLAK_PLAN_BULK_RECORDS = 64 /* closed levels: k_g3 stages its slot records in shared      */
                                /* memory by bulk copy (TMA) (same results; see below)        */
};
/* SLAK_PLAN_GQ and SLAK_PLAN_BULK_RECORDS are alternative kernel layouts kept
 * for comparison: both give the default path's results bit for bit, and both
 * measured slower on B200, so neither is the default.  A SLAK_PLAN_BULK_RECORDS
 * block waits on its copies at most SLAK_BULK_WAIT_POLLS mbarrier polls (read
 * from the environment when the plan is created, default 2^20); past that it
 * reports SLAK_ERR_TIMEOUT through slak_plan_status (0 forces that path). */

typedef struct slak_kernel_timing {
    const char* name;           /* kernel name (static string)                     */
    int32_t level;              /* subdivision level it belongs to                 */
    float ms;                   /* device time since the previous launch's event   */
    int64_t algorithmic_bytes;  /* compulsory bytes it moves, 0 when not defined    */
} slak_kernel_timing;

/* Launch shapes of one fast level (slak_plan_tuning). */
typedef struct slak_tuning {
    int32_t state;              /* -1 not a fast level, 0 default, 1 measured by this plan,
                                   2 taken from the tuning cache                         */
    int32_t block[3];           /* block size of k_g1, k_g2, k_g3                          */
    float ms[3][3];             /* state 1: median ms of each kernel at block 128/256/512  */
    char key[64];               /* tuning-cache key                                        */
} slak_tuning;

typedef struct slak_level_stats {
    int64_t nfaces, nverts, nnz, nedges, nboundary;   /* of the level's input mesh */
    int64_t out_faces, out_verts;
    int64_t algorithmic_bytes;                        /* compulsory input + output bytes */
} slak_level_stats;

int slak_plan_create(const slak_mesh* cmesh, int target_level, int scheme, int flags,
                     slak_stream_t stream, slak_plan** plan);
int slak_plan_execute(slak_plan* plan, slak_stream_t stream);
/* Waits for `stream`, then reports the device-side status of the last execution. */
int slak_plan_status(slak_plan* plan, slak_stream_t stream);
int slak_plan_output(const slak_plan* plan, slak_mesh* rmesh);
int slak_plan_release_output(slak_plan* plan, slak_mesh* rmesh);
int slak_plan_num_levels(const slak_plan* plan);
int slak_plan_level_stats(const slak_plan* plan, int level, slak_level_stats* stats);
/* Kernel launches one execution issues (the count a graph replays). */
int64_t slak_plan_launches(const slak_plan* plan);
/* Per-launch device times of the last execution of a SLAK_PLAN_TIMING plan
 * (waits for it); returns the number of launches, or -status. */
int slak_plan_kernel_timings(slak_plan* plan, slak_kernel_timing* out, int capacity);
int slak_plan_destroy(slak_plan* plan);

/*
 * Autotuner (no counterpart in the reference, whose launch shapes are fixed).
 * The block sizes of the three closed-form kernels of every fast level are
 * chosen by measurement, keyed on the scheme, the parent level's face type,
 * whether the level feeds another fast level, log2 of the level's quads and
 * the input's valence histogram (largest valence; share of valence 4).  Every
 * plan and batch applies cached choices; with SLAK_PLAN_AUTOTUNE, creation also
 * measures the keys not yet cached (block 128 / 256 / 512 per kernel, median of
 * three executions).  The cache lives in the process; with SLAK_TUNE_FILE set
 * in the environment it is also loaded from and saved to that file.
 */
int slak_plan_tuning(const slak_plan* plan, int level, slak_tuning* out);
int slak_autotune_reset(void);    /* forget the in-process cache (the file is kept) */

/*
 * Semi-sharp creases.  The reference declares this step but does not implement
 * it: "if (has_creases && !creases_decayed) time += handleCreases(...)" is
 * commented out in LibSource/device/CatmullClarkImpl.cu:94-96 and :296-298 and
 * LibSource/device/LAKCatmullClarkImpl.cu:240-242.  The rules are those of
 * DeRose, Kass and Truong (SIGGRAPH 1998), with sharpness decaying by one per
 * level.  Both schemes use the same rules.
 *  - Edge points. An edge of sharpness s >= 1 becomes the midpoint of its
 *    ends. For 0 < s < 1 the result is smooth * (1 - s) + midpoint * s.
 *  - Vertex points. Let k be the number of crease edges at a vertex and
 *    w = min(1, their mean sharpness). With k == 2 the vertex takes the crease
 *    rule (3/4 p + 1/8 p_o1) + 1/8 p_o2, other ends in ascending id. With
 *    k >= 3, or on a boundary, it is a corner (p unchanged). With k == 1 it
 *    stays smooth. The sharp result is blended with the smooth one by w.
 *  - Child edges. The two child edges of a crease edge carry s - 1.
 *
 * crease_verts holds 2 * ncreases vertex ids (the pairs {a, b}).
 * crease_sharpness holds ncreases floats. Both arrays are in device memory and
 * are copied into the plan at creation.
 *  - A pair on a boundary edge is ignored, since the boundary is already
 *    sharp. So is a pair with sharpness <= 0.
 *  - A pair that is not an edge of the input, or an edge named twice, makes
 *    the execution's status SLAK_ERR_BAD_MESH.
 *  - A sharpness that is not finite gives SLAK_ERR_INVALID_ARG.
 *
 * The crease pass runs after each level that has a live crease. It needs four
 * launches, and a mesh without creases pays nothing.
 * slak_subdivide_creased is slak_subdivide with creases. It uses no workspace
 * cache.
 */
int slak_plan_create_creased(const slak_mesh* cmesh, int target_level, int scheme, int flags,
                             const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                             slak_stream_t stream, slak_plan** plan);
int slak_subdivide_creased(const slak_mesh* cmesh, slak_mesh* rmesh, int target_level, int scheme,
                           const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                           slak_stream_t stream);

/*
 * Creases and corners (vertex sharpness, the "t corner" tags OBJ::read also
 * keeps unused).  A vertex of sharpness s takes the corner rule (it keeps its
 * position) while s - level > 0, blended with its smooth point by
 * max(min(1, s - level), min(1, mean sharpness of its crease edges)).
 * corner_verts holds ncorners vertex ids and corner_sharpness their sharpness,
 * both in device memory.  They are read at creation: an id out of range or a
 * vertex named twice gives SLAK_ERR_BAD_MESH, and a sharpness that is not
 * finite gives SLAK_ERR_INVALID_ARG.  The _creased calls are these with no
 * corners.
 */
int slak_plan_create_sharp(const slak_mesh* cmesh, int target_level, int scheme, int flags,
                           const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                           const int32_t* corner_verts, const float* corner_sharpness, int64_t ncorners,
                           slak_stream_t stream, slak_plan** plan);
int slak_subdivide_sharp(const slak_mesh* cmesh, slak_mesh* rmesh, int target_level, int scheme,
                         const int32_t* crease_verts, const float* crease_sharpness, int64_t ncreases,
                         const int32_t* corner_verts, const float* corner_sharpness, int64_t ncorners,
                         slak_stream_t stream);

/*
 * Batches: many meshes, each with its own target level, refined by one call
 * (what the reference's config-file loop does one mesh at a time,
 * source/main.cpp:84-113).  Each mesh's result is exactly slak_subdivide's on
 * that mesh alone.  All sizes are fixed at creation (one stream sync for all
 * meshes' level-0 topology); every output lives in one batch-owned buffer
 * (slak_batch_output returns views, valid until slak_batch_destroy).
 *
 * Meshes that refine to fewer than 2^19 quads (SLAK_BATCH_GROUP_QUADS in the
 * environment at creation overrides the bound; 0 turns groups off) run in
 * groups: meshes whose plans launch the same kernels with the same shapes in
 * the same order, each step one grouped launch over all of them (a block finds
 * its mesh in a table of block offsets).  A small mesh's ~18 launches become a
 * share of its group's, so a batch of many small meshes is no longer bound by
 * launches.  Each grouped mesh has its own scratch; together they take at
 * most half of the scratch budget.  The other meshes run in 16 concurrent
 * chains, dealt longest predicted time first to the least loaded chain; a
 * chain reuses one scratch slice for its meshes.  Only when the chains'
 * slices outgrow the budget (3/4 of the free memory after the outputs, at most
 * 24 GB; SLAK_BATCH_WAVE_BYTES overrides the cap) does the batch run in
 * several waves.  With SLAK_PLAN_GRAPH the whole batch is captured as one
 * CUDA graph on the first execution.
 */
typedef struct slak_batch slak_batch;
int slak_batch_create(const slak_mesh* meshes, const int* levels, int64_t count, int scheme, int flags,
                      slak_stream_t stream, slak_batch** batch);
int slak_batch_execute(slak_batch* batch, slak_stream_t stream);
/* Waits for `stream`, then reports the first failing mesh's device status. */
int slak_batch_status(slak_batch* batch, slak_stream_t stream);
/* The refined mesh of meshes[index]; left untouched when that mesh had nothing to refine. */
int slak_batch_output(const slak_batch* batch, int64_t index, slak_mesh* rmesh);
int slak_batch_num_waves(const slak_batch* batch);     /* waves of the chained meshes        */
int slak_batch_num_groups(const slak_batch* batch);    /* groups of small meshes              */
int64_t slak_batch_launches(const slak_batch* batch);  /* kernel launches of one execution    */
int slak_batch_destroy(slak_batch* batch);

/*
 * The batch in one call: rmeshes[i] receives meshes[i] refined to levels[i].
 * This is the batched counterpart of slak_subdivide, and of the reference's
 * per-mesh loop (source/main.cpp:84-113). Each output array has its own
 * cudaMalloc and belongs to the caller, who frees it with slak_mesh_free or
 * cudaFree, as after slak_subdivide. A mesh with nothing to refine leaves
 * rmeshes[i] zeroed. The call returns once every mesh is refined. All
 * outputs are resident at once; the scratch is shared as in slak_batch_create.
 */
int slak_subdivide_batched(const slak_mesh* meshes, const int* levels, int64_t count, int scheme,
                           slak_mesh* rmeshes, slak_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SLAK_B200_H */
