// Stand-in for the reference's base/CommonUtils.h (device-memory and texture
// helpers) for compiling the reference's header-only solver math on the host.
// TEST INFRASTRUCTURE.
#pragma once
#include <base/CommonTypes.h>

namespace SparseSurfelFusion {
template <class T> __host__ __device__ inline void swap(T& a, T& b) noexcept {
    T t = a;
    a = b;
    b = t;
}
}  // namespace SparseSurfelFusion

namespace SparseSurfelFusion {
// texture fetches the solver types name in their device-side dot products
template <class T> __device__ inline T fetch1DLinear(cudaTextureObject_t t, unsigned i) { return tex1Dfetch<T>(t, (int)i); }
template <class T> __device__ inline T fetch1DArray(cudaTextureObject_t t, unsigned i) { return tex1D<T>(t, (float)i); }
}  // namespace SparseSurfelFusion
