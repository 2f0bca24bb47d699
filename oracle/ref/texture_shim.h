/*
 * texture_shim.h -- TEST INFRASTRUCTURE ONLY (force-included by oracle/build_ref.sh).
 *
 * OpenCurrent's device solver binds its inputs to legacy texture references
 * (ocuequation/sol_mgpressure3ddevf.cu:32-35, sol_mgpressure3ddevd.cu:35-62,
 * sol_selfadvection3ddev.cu:116-133 and 227-247).  CUDA 12 removed texture references, so
 * those files no longer compile as shipped.  This header gives the three constructs they use
 * a meaning that reads the same memory:
 *
 *   texture<T, 1, mode> name;          -> a __device__ object holding a const T* (plus the
 *                                         host-only fields the reference assigns);
 *   cudaBindTexture(0, &name, p, ...)  -> stores p into that object with cudaMemcpyToSymbol;
 *   tex1Dfetch(name, i)                -> __ldg(p + i), a read through the same read-only,
 *                                         non-coherent path a 1-D texture fetch used;
 *   cudaUnbindTexture(&name)           -> nothing.
 *
 * The reference reads through the textures only values that the same kernel does not write
 * (the other colour of a red-black sweep, the coarse grid of a prolongation, the inputs of
 * the advection stencil), so the non-coherent load returns what the texture fetch returned.
 * The int2 textures of the FP64 kernels become int2 loads of the double buffers, which the
 * kernels reassemble with __hiloint2double exactly as before.
 */
#pragma once
#include <cuda_runtime.h>

template <class T, int dim = 1, enum cudaTextureReadMode mode = cudaReadModeElementType>
struct ocu_ref_texref {
  const T *ptr;                       /* device address bound by cudaBindTexture */
  cudaTextureFilterMode filterMode;   /* assigned by the reference's host code, unused */
  int normalized;                     /* idem */
  cudaChannelFormatDesc channelDesc;  /* idem */
};

#define texture __device__ ocu_ref_texref

template <class T, int d, enum cudaTextureReadMode m>
__device__ __forceinline__ T tex1Dfetch(const ocu_ref_texref<T, d, m> &t, int i) {
  return __ldg(t.ptr + i);
}

template <class T, int d, enum cudaTextureReadMode m>
static inline cudaError_t cudaBindTexture(size_t *offset, const ocu_ref_texref<T, d, m> *t,
                                          const void *p, const cudaChannelFormatDesc *,
                                          size_t) {
  if (offset) *offset = 0;
  /* t is the host shadow of the __device__ object; the runtime maps it to the symbol. */
  return cudaMemcpyToSymbol(*t, &p, sizeof(p));
}

template <class T, int d, enum cudaTextureReadMode m>
static inline cudaError_t cudaUnbindTexture(const ocu_ref_texref<T, d, m> *) {
  return cudaSuccess;
}
