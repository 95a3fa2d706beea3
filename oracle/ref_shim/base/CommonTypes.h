// Stand-in for the reference's base/CommonTypes.h (which pulls in Eigen, PCL
// and the reference's device containers), written here so that the
// reference's header-only solver math (dual quaternions, mat34, the ICP and
// smooth-term Jacobians, the 6x6 Gauss-Jordan inverse, node-pair encoding)
// compiles on the host for pinning the oracle. Only what those headers name is
// provided: the Eigen types appear in declarations of conversions the solver
// math never calls. TEST INFRASTRUCTURE.
#pragma once
#include <cuda_runtime.h>
#include <vector_functions.h>
#include <cmath>
#include <cstdint>
#include <base/GlobalConfigs.h>  // the reference's own compile-time limits (MAX_NODE_COUNT, ...)

namespace Eigen {
// a 3x3 column-major matrix with the (row, col) accessor the headers use
struct Matrix3f {
    float v[9];
    __host__ __device__ float operator()(int r, int c) const { return v[3 * c + r]; }
    __host__ __device__ float& operator()(int r, int c) { return v[3 * c + r]; }
};
struct Matrix4f;
struct Vector3f;
struct Vector4f;
struct Isometry3f;
}  // namespace Eigen

namespace SparseSurfelFusion {
using Matrix3f = Eigen::Matrix3f;
using Vector3f = Eigen::Vector3f;
using Matrix4f = Eigen::Matrix4f;
using Vector4f = Eigen::Vector4f;
using Isometry3f = Eigen::Isometry3f;

// camera intrinsics in the reference's field order
struct Intrinsic {
    float principal_x, principal_y;
    float focal_x, focal_y;
};
}  // namespace SparseSurfelFusion
