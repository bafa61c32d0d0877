/*
 * ref_cuda_shim.h -- force-included (nvcc -include) when the reference's
 * V3D/CUDA/v3d_cudamatching.cu is compiled, unmodified, with CUDA 12.9.
 *
 * TEST INFRASTRUCTURE ONLY: it exists to run the reference's own matching kernels as a
 * parity pin for the oracle.  CUDA 12 removed texture references, which the reference
 * uses for one array of right-image positions (v3d_cudamatching.cu:275, :295-296,
 * :334-335, :586, :599, :657, :670).  This header supplies a texture stand-in with the same
 * call syntax: a __device__ struct holding the bound pointer, tex1Dfetch() as a plain
 * global load, cudaBindTexture() as a copy of the pointer to that symbol.  A plain load
 * returns the same float a 1-D element-type texture fetch returns.
 */
#pragma once
#include <cuda_runtime.h>

template <class T, int dim, enum cudaTextureReadMode mode>
struct v3dref_texref {
    const T* ptr;
};

template <class T, int dim, enum cudaTextureReadMode mode>
__device__ __forceinline__ T tex1Dfetch(const v3dref_texref<T, dim, mode>& t, int i) {
    return t.ptr[i];
}

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaBindTexture(size_t* offset, const v3dref_texref<T, dim, mode>& tex, const void* p,
                                          size_t) {
    v3dref_texref<T, dim, mode> h;
    h.ptr = (const T*)p;
    if (offset) *offset = 0;
    return cudaMemcpyToSymbol(tex, &h, sizeof(h));
}

template <class T, int dim, enum cudaTextureReadMode mode>
static inline cudaError_t cudaUnbindTexture(const v3dref_texref<T, dim, mode>&) {
    return cudaSuccess;
}

/* 'texture<float, 1, cudaReadModeElementType> rightPos_tex;' becomes a __device__ variable. */
#define texture __device__ v3dref_texref
