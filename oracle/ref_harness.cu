// ref_harness.cu -- C entry points around the reference's own
// subdivideIteratively, compiled together with the reference's sources.
// TEST / BASELINE INFRASTRUCTURE ONLY: it runs GPUPeople/SLAK's unmodified CUDA
// path (LibSource/device/CatmullClarkImpl.cu, LAKCatmullClarkImpl.cu) so its
// output can pin the oracle and its speed can be measured on the same GPU.
#include "CatmullClark.h"
#include "LAKCatmullClark.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unistd.h>

extern "C" {
typedef struct {
    int32_t type, is_reduced;
    int64_t nfaces, nverts, nnz, max_face_order;
    int32_t* ptr;
    int32_t* ids;
    int32_t* vals;
    float* verts;
} ref_mesh;
}

namespace {

// Redirects stdout (the reference prints a report per call) into a temp file
// and returns what was printed.
struct StdoutCapture {
    int saved = -1;
    FILE* tmp = nullptr;
    explicit StdoutCapture(bool on)
    {
        if (!on) return;
        std::fflush(stdout);
        std::cout.flush();
        tmp = std::tmpfile();
        saved = dup(1);
        dup2(fileno(tmp), 1);
    }
    std::string finish()
    {
        std::string s;
        if (saved < 0) return s;
        std::cout.flush();
        std::fflush(stdout);
        dup2(saved, 1);
        close(saved);
        saved = -1;
        std::rewind(tmp);
        char buf[4096];
        size_t n;
        while ((n = std::fread(buf, 1, sizeof buf, tmp)) > 0) s.append(buf, n);
        std::fclose(tmp);
        return s;
    }
    ~StdoutCapture() { finish(); }
};

float parse_took(const std::string& s)
{
    auto k = s.rfind(" took ");
    if (k == std::string::npos) return -1.f;
    return std::strtof(s.c_str() + k + 6, nullptr);
}

template <class MI>
void to_info(const ref_mesh& h, int* d_ptr, int* d_ids, int* d_vals, float* d_verts, MI& m)
{
    using T = typename MI::MeshType;
    m.type = h.type == 0 ? T::TRI : (h.type == 1 ? T::QUAD : T::POLY);
    m.nfaces = h.nfaces; m.nverts = h.nverts; m.nnz = h.nnz; m.max_face_order = h.max_face_order;
    m.is_reduced = h.is_reduced != 0;
    m.ptr = d_ptr; m.ids = d_ids; m.vals = d_vals; m.verts = d_verts;
}

template <class MI>
int download(const MI& r, ref_mesh* o)
{
    std::memset(o, 0, sizeof(*o));
    o->type = r.type == MI::MeshType::QUAD ? 1 : (r.type == MI::MeshType::TRI ? 0 : 2);
    o->is_reduced = r.is_reduced;
    o->nfaces = r.nfaces; o->nverts = r.nverts; o->nnz = r.nnz; o->max_face_order = r.max_face_order;
    if (r.ids) {
        o->ids = (int32_t*)std::malloc(sizeof(int) * r.nnz);
        if (cudaMemcpy(o->ids, r.ids, sizeof(int) * r.nnz, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    }
    if (r.verts) {
        o->verts = (float*)std::malloc(sizeof(float) * 4 * r.nverts);
        if (cudaMemcpy(o->verts, r.verts, sizeof(float) * 4 * r.nverts, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    }
    if (r.ptr) {
        o->ptr = (int32_t*)std::malloc(sizeof(int) * (r.nfaces + 1));
        if (cudaMemcpy(o->ptr, r.ptr, sizeof(int) * (r.nfaces + 1), cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    }
    if (r.vals) {
        o->vals = (int32_t*)std::malloc(sizeof(int) * r.nnz);
        if (cudaMemcpy(o->vals, r.vals, sizeof(int) * r.nnz, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    }
    return 0;
}

struct DevInput {
    int *ptr = nullptr, *ids = nullptr, *vals = nullptr;
    float* verts = nullptr;
    int upload(const ref_mesh& h)
    {
        if (h.ptr && cudaMalloc(&ptr, sizeof(int) * (h.nfaces + 1)) != cudaSuccess) return 3;
        if (cudaMalloc(&ids, sizeof(int) * h.nnz) != cudaSuccess) return 3;
        if (h.vals && cudaMalloc(&vals, sizeof(int) * h.nnz) != cudaSuccess) return 3;
        if (cudaMalloc(&verts, sizeof(float) * 4 * h.nverts) != cudaSuccess) return 3;
        if (h.ptr) cudaMemcpy(ptr, h.ptr, sizeof(int) * (h.nfaces + 1), cudaMemcpyHostToDevice);
        cudaMemcpy(ids, h.ids, sizeof(int) * h.nnz, cudaMemcpyHostToDevice);
        if (h.vals) cudaMemcpy(vals, h.vals, sizeof(int) * h.nnz, cudaMemcpyHostToDevice);
        cudaMemcpy(verts, h.verts, sizeof(float) * 4 * h.nverts, cudaMemcpyHostToDevice);
        return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
    }
    ~DevInput()
    {
        if (ptr) cudaFree(ptr);
        if (ids) cudaFree(ids);
        if (vals) cudaFree(vals);
        if (verts) cudaFree(verts);
    }
};

template <class S>
int call(const ref_mesh& h, DevInput& d, int levels, typename S::template MeshInfo<int, int, int, float>& r)
{
    typename S::template MeshInfo<int, int, int, float> c;
    to_info(h, d.ptr, d.ids, d.vals, d.verts, c);
    try {
        S::subdivideIteratively(c, r, levels);
    } catch (...) {
        return 4;
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

}  // namespace

extern "C" {

// Runs the reference once on a host mesh and downloads the refined mesh
// (arrays malloc'ed; release with ref_free).  scheme 0 = LAK, 1 = SLAK.
int ref_run(int scheme, const ref_mesh* in, int levels, ref_mesh* out, float* self_ms, int quiet)
{
    DevInput d;
    int rc = d.upload(*in);
    if (rc) return rc;
    StdoutCapture cap(quiet != 0);
    if (scheme == 1) {
        CatmullClark::MeshInfo<int, int, int, float> r;
        rc = call<CatmullClark>(*in, d, levels, r);
        if (!rc) rc = download(r, out);
        r.freeAndReset();
    } else {
        LAKCatmullClark::MeshInfo<int, int, int, float> r;
        rc = call<LAKCatmullClark>(*in, d, levels, r);
        if (!rc) rc = download(r, out);
        r.freeAndReset();
    }
    std::string txt = cap.finish();
    if (self_ms) *self_ms = parse_took(txt);
    return rc;
}

// Times `reps` calls on device-resident input: ms_each[i] brackets one
// subdivideIteratively with CUDA events (output freed outside the bracket);
// self_ms[i] is the reference's own printed "took X ms".  Before every call,
// outside the bracket, 256 MiB are written to flush L2, as the repository's
// own timing does.
int ref_time(int scheme, const ref_mesh* in, int levels, int warmup, int reps, double* ms_each, float* self_ms,
             int quiet)
{
    DevInput d;
    int rc = d.upload(*in);
    if (rc) return rc;
    const size_t flush_bytes = size_t(256) << 20;
    void* flush = nullptr;
    if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) return 3;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    StdoutCapture cap(quiet != 0);      // one redirect around the whole loop
    for (int i = -warmup; i < reps && !rc; ++i) {
        float ms = 0.f;
        cudaMemsetAsync(flush, i & 0xff, flush_bytes);
        cudaEventRecord(a);
        if (scheme == 1) {
            CatmullClark::MeshInfo<int, int, int, float> r;
            rc = call<CatmullClark>(*in, d, levels, r);
            cudaEventRecord(b);
            cudaEventSynchronize(b);
            r.freeAndReset();
        } else {
            LAKCatmullClark::MeshInfo<int, int, int, float> r;
            rc = call<LAKCatmullClark>(*in, d, levels, r);
            cudaEventRecord(b);
            cudaEventSynchronize(b);
            r.freeAndReset();
        }
        cudaEventElapsedTime(&ms, a, b);
        if (i >= 0) ms_each[i] = ms;
    }
    std::string txt = cap.finish();
    if (self_ms) {     // the reference's own "took X ms", one per call, warm-up first
        size_t k = 0;
        int idx = -warmup;
        while ((k = txt.find(" took ", k)) != std::string::npos) {
            if (idx >= 0 && idx < reps) self_ms[idx] = std::strtof(txt.c_str() + k + 6, nullptr);
            ++idx;
            k += 6;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(flush);
    return rc;
}

// End-to-end time of `reps` calls with host buffers (ms_each, wall clock):
// per call, the input is copied from pinned host memory into the device
// arrays, subdivideIteratively runs, and the refined ids and positions are
// copied back into pinned host memory; the output is freed outside the bracket.
int ref_time_e2e(int scheme, const ref_mesh* in, int levels, int warmup, int reps, double* ms_each,
                 int64_t* h2d_bytes, int64_t* d2h_bytes, int quiet)
{
    DevInput d;
    int rc = d.upload(*in);
    if (rc) return rc;
    const size_t bp = in->ptr ? sizeof(int) * (in->nfaces + 1) : 0, bi = sizeof(int) * in->nnz;
    const size_t bv = in->vals ? sizeof(int) * in->nnz : 0, bx = sizeof(float) * 4 * in->nverts;
    char* hin = nullptr;
    if (cudaMallocHost(&hin, bp + bi + bv + bx) != cudaSuccess) return 3;
    if (bp) std::memcpy(hin, in->ptr, bp);
    std::memcpy(hin + bp, in->ids, bi);
    if (bv) std::memcpy(hin + bp + bi, in->vals, bv);
    std::memcpy(hin + bp + bi + bv, in->verts, bx);
    char* hout = nullptr;
    size_t out_cap = 0;
    *h2d_bytes = (int64_t)(bp + bi + bv + bx);
    StdoutCapture cap(quiet != 0);
    for (int i = -warmup; i < reps && !rc; ++i) {
        cudaDeviceSynchronize();
        auto t0 = std::chrono::steady_clock::now();
        if (bp) cudaMemcpyAsync(d.ptr, hin, bp, cudaMemcpyHostToDevice);
        cudaMemcpyAsync(d.ids, hin + bp, bi, cudaMemcpyHostToDevice);
        if (bv) cudaMemcpyAsync(d.vals, hin + bp + bi, bv, cudaMemcpyHostToDevice);
        cudaMemcpyAsync(d.verts, hin + bp + bi + bv, bx, cudaMemcpyHostToDevice);
        auto fetch = [&](auto& r) {
            const size_t oi = sizeof(int) * r.nnz, ox = sizeof(float) * 4 * r.nverts;
            if (!hout) {
                out_cap = oi + ox;
                if (cudaMallocHost(&hout, out_cap) != cudaSuccess) return 3;
            }
            if (oi + ox > out_cap) return 3;
            cudaMemcpyAsync(hout, r.ids, oi, cudaMemcpyDeviceToHost);
            cudaMemcpyAsync(hout + oi, r.verts, ox, cudaMemcpyDeviceToHost);
            *d2h_bytes = (int64_t)(oi + ox);
            return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
        };
        double ms = 0;
        if (scheme == 1) {
            CatmullClark::MeshInfo<int, int, int, float> r;
            rc = call<CatmullClark>(*in, d, levels, r);
            if (!rc) rc = fetch(r);
            ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            r.freeAndReset();
        } else {
            LAKCatmullClark::MeshInfo<int, int, int, float> r;
            rc = call<LAKCatmullClark>(*in, d, levels, r);
            if (!rc) rc = fetch(r);
            ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            r.freeAndReset();
        }
        if (i >= 0) ms_each[i] = ms;
    }
    cap.finish();
    cudaFreeHost(hin);
    if (hout) cudaFreeHost(hout);
    return rc;
}

void ref_free(ref_mesh* m)
{
    if (!m) return;
    std::free(m->ptr); std::free(m->ids); std::free(m->vals); std::free(m->verts);
    std::memset(m, 0, sizeof(*m));
}

}  // extern "C"
