// Test infrastructure only (the reference comparator build).
//
// Stand-in for quadmap/texture_memory.cuh of open_quadtree_mapping
// (include/quadmap/texture_memory.cuh:10-63).  The original declares legacy
// `texture<>` references, which CUDA 12 removed, so the reference kernels do
// not compile for sm_100a as shipped.  This header is found first on the
// include path of the comparator build and provides the same names with the
// same sampling semantics through texture OBJECTS:
//   * each name is a __device__ struct holding a cudaTextureObject_t,
//   * tex2D(name, x, y) forwards to tex2D<T>(object, x, y),
//   * bindTexture() builds a pitch-2D texture object with clamp addressing,
//     unnormalised coordinates and the requested filter mode (linear by
//     default, exactly as the original bindTexture), and copies it into the
//     __device__ symbol,
//   * cudaUnbindTexture() destroys that object.
// The texture unit does the sampling in both cases, so kernel arithmetic is
// unchanged.  Every texture read on the depth path is at a texel centre or
// point-filtered, so values are exact texels either way.
#pragma once

#include <cuda_runtime.h>
#include <quadmap/device_image.cuh>
#include <quadmap/cuda_exception.cuh>
#include <map>

namespace quadmap
{

template <typename T>
struct TexRef
{
  cudaTextureObject_t obj;
};

// Names used by the kernels of the depth path (and the semi-dense tracker).
__device__ TexRef<float> income_image_tex;
__device__ TexRef<float> pre_image_tex;
__device__ TexRef<float2> income_gradient_tex;
__device__ TexRef<float> keyframe_image_tex;
__device__ TexRef<float2> keyframe_gradient_tex;
__device__ TexRef<int> quadtree_tex;

template <typename T>
__device__ __forceinline__ T tex2D(const TexRef<T> &t, float x, float y)
{
  return ::tex2D<T>(t.obj, x, y);
}

inline std::map<const void *, cudaTextureObject_t> &shim_live_textures()
{
  static std::map<const void *, cudaTextureObject_t> m;
  return m;
}

template <typename ElementType>
inline void cudaUnbindTexture(TexRef<ElementType> &symbol)
{
  auto &live = shim_live_textures();
  auto it = live.find((const void *)&symbol);
  if (it != live.end())
  {
    cudaDestroyTextureObject(it->second);
    live.erase(it);
  }
}

template <typename ElementType>
inline void bindTexture(TexRef<ElementType> &symbol,
                        const DeviceImage<ElementType> &mem,
                        cudaTextureFilterMode filter_mode = cudaFilterModeLinear)
{
  cudaUnbindTexture(symbol);
  cudaResourceDesc res = {};
  res.resType = cudaResourceTypePitch2D;
  res.res.pitch2D.devPtr = mem.data;
  res.res.pitch2D.desc = mem.getCudaChannelFormatDesc();
  res.res.pitch2D.width = mem.width;
  res.res.pitch2D.height = mem.height;
  res.res.pitch2D.pitchInBytes = mem.pitch;
  cudaTextureDesc td = {};
  td.addressMode[0] = cudaAddressModeClamp;
  td.addressMode[1] = cudaAddressModeClamp;
  td.filterMode = filter_mode;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 0;
  TexRef<ElementType> ref;
  cudaError_t err = cudaCreateTextureObject(&ref.obj, &res, &td, nullptr);
  if (err != cudaSuccess)
    throw CudaException("Unable to bind texture: ", err);
  err = cudaMemcpyToSymbol(symbol, &ref, sizeof(ref));
  if (err != cudaSuccess)
    throw CudaException("Unable to bind texture: ", err);
  shim_live_textures()[(const void *)&symbol] = ref.obj;
}

} // namespace quadmap
