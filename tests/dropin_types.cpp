// Host code written against the reference's public nested types: each scheme's
// Context<MESH_INFO>, ProfilinInfo<PROFILER, MEM_MANAGER> and
// MeshInfo::freeAndReset(MEM_MANAGER&) (LibInclude/CatmullClark.h:38-67,108-129;
// LibInclude/LAKCatmullClark.h:38-83).  Compiled and run by
// tests/test_dropin_types.py, with no GPU: the fake manager below claims every
// array, so no CUDA call is made until the last check, whose cudaFree must fail
// without a device and surface as the reference's `const char*` throw.
#include <cstdio>
#include <set>

#include "CatmullClark.h"
#include "LAKCatmullClark.h"

namespace {

struct FakeManager {             // the shape of the reference's DeviceMemManager::freeMemory
    std::set<const void*> owned;
    int freed = 0;
    template <typename T>
    bool freeMemory(T*& p)
    {
        if (p == nullptr || owned.erase(p) == 0) return false;
        ++freed;
        return true;
    }
};

struct NoProfiler {
    int calls = 0;
};

template <class S>
int exercise(const char* name)
{
    using MI = typename S::template MeshInfo<int, int, int, float>;
    typename S::template Context<MI> ctx;
    typename S::template ProfilinInfo<NoProfiler, FakeManager> info;
    if (ctx.block_dim != 256 || ctx.is_initialized || !ctx.has_boundary || ctx.nextern != 0) {
        std::printf("%s: Context defaults differ\n", name);
        return 1;
    }
    static int a[4], b[4], c[4];
    static float v[4];
    MI m;
    m.type = MI::MeshType::QUAD;
    m.nfaces = 1;
    m.ptr = a;
    m.ids = b;
    m.vals = c;
    m.verts = v;
    info.mem.owned = {a, b, c, v};
    m.freeAndReset(info.mem);
    if (info.mem.freed != 4 || m.ptr || m.ids || m.vals || m.verts || m.nfaces != 0) {
        std::printf("%s: freeAndReset(mem) left state behind\n", name);
        return 1;
    }
    // an array the manager does not own falls back to cudaFree, which has no
    // device here: the failure is thrown as const char*, as the reference does
    m.ids = b;
    bool threw = false;
    try {
        m.freeAndReset(info.mem);
    } catch (const char*) {
        threw = true;
    }
    std::printf("%s: ok (fallback %s)\n", name, threw ? "threw" : "freed");
    return 0;
}

}  // namespace

int main()
{
    int rc = exercise<CatmullClark>("CatmullClark");
    rc |= exercise<LAKCatmullClark>("LAKCatmullClark");
    LAKCatmullClark::Context<LAKCatmullClark::MeshInfo<int, int, int, float>> lctx;
    rc |= lctx.d_E_ptr != nullptr || lctx.nedges != 0;
    return rc;
}
