/*
 * ref_shim.h -- force-included (nvcc -include) when compiling the reference's
 * own sources for sm_100a with CUDA 12.9.  TEST INFRASTRUCTURE ONLY.
 *
 * GPUPeople/SLAK's LibInclude/device/math/spgemm.cuh:44,57,168,235 uses a
 * legacy texture reference (texture<>, tex1Dfetch on it, cudaBindTexture),
 * which CUDA 12 removed.  It is only read by MappedMul::multiply, the
 * EXPLICIT_MAP_LOOKUP variant that the reference disables by default
 * (spgemm.cuh:114-118), so inert stand-ins let the file compile without
 * changing anything the default path executes.  The reference tree itself is
 * never modified or copied.
 */
#pragma once
#include <cuda_runtime.h>

template <class T, int Dim, enum cudaTextureReadMode Mode>
struct slak_ref_legacy_texture {
};

#define texture __device__ slak_ref_legacy_texture

template <class T, int Dim, enum cudaTextureReadMode Mode>
__device__ inline T tex1Dfetch(const slak_ref_legacy_texture<T, Dim, Mode>&, int)
{
    return T(0);
}

template <class T, int Dim, enum cudaTextureReadMode Mode>
inline cudaError_t cudaBindTexture(size_t*, const slak_ref_legacy_texture<T, Dim, Mode>*, const void*,
                                   const cudaChannelFormatDesc*, size_t)
{
    return cudaSuccess;
}
