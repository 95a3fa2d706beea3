// Stand-in for the reference's base/DeviceReadWrite/DeviceArrayView.h (tied
// to its device containers) for compiling the reference's header-only solver
// math on the host: a non-owning pointer + size view. TEST INFRASTRUCTURE.
#pragma once
#include <base/CommonTypes.h>
#include <cstddef>
#include <vector>

namespace SparseSurfelFusion {
template <typename T> class DeviceArrayView {
public:
    __host__ __device__ DeviceArrayView() : p_(nullptr), n_(0) {}
    __host__ __device__ DeviceArrayView(const T* p, size_t n) : p_(p), n_(n) {}
    __host__ __device__ size_t Size() const { return n_; }
    __host__ __device__ const T* RawPtr() const { return p_; }
    __host__ __device__ const T& operator[](size_t i) const { return p_[i]; }
    // the views here point at host memory, so a download is a copy
    __host__ void Download(std::vector<T>& out) const { out.assign(p_, p_ + n_); }
private:
    const T* p_;
    size_t n_;
};
}  // namespace SparseSurfelFusion
