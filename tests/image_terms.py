"""Independent numpy restatement of the reference's image-term Jacobian, for
checks of the oracle and the kernels (test infrastructure only).

computeImageDensityJacobainAndResidual (core/NonRigidSolver/
density_map_jacobian.cuh:12-79) warps a pixel's reference vertex by the
blended warp field, takes it to the observing camera (world2camera, then the
inverse of InitialCameraSE3), projects it with round-to-nearest-even, samples
the image and its gradient there, and chains the image gradient through the
pinhole projection and the two rotations to a twist gradient. The foreground
term (DensityForegroundJacobianResidual.cu:93-142) uses it with the filtered
foreground mask, its gradient and a geometry density of 0.

`frame0` selects where the reference vertex is warped: False warps it as it is
stored in its camera's frame, as density_map_jacobian.cuh:32-36 does (the
library's MVDR_COMPAT_REF_FOREGROUND_FRAME); True first moves it to frame 0
with InitialCameraSE3, as the dense-depth term does
(DenseDepthJacobianResidual.cu:43-50) and the library does by default.
"""
import numpy as np


def unpack34(m):
    """mat34 of the ABI (rotation columns, then translation) -> R, t."""
    m = np.asarray(m, np.float64)
    return m[:9].reshape(3, 3).T, m[9:12]


def dq_blend_se3(dq, knn, w):
    """averageDualQuaternion + se3_matrix (DualQuaternion.h:281-332,381-393)
    in double for one term: returns R, t."""
    q = np.zeros(8)
    for n, wi in zip(knn, w):
        q += float(wi) * dq[int(n)].astype(np.float64)
    q0, q1 = q[:4], q[4:]
    inv = 1.0 / np.sqrt(q0 @ q0)
    q0, q1 = q0 * inv, q1 * inv
    q1 = q1 - (q0 @ q1) * q0
    x, y, z, ww = q0
    R = np.array([[1 - 2 * y * y - 2 * z * z, 2 * x * y - 2 * z * ww, 2 * x * z + 2 * y * ww],
                  [2 * x * y + 2 * z * ww, 1 - 2 * x * x - 2 * z * z, 2 * y * z - 2 * x * ww],
                  [2 * x * z - 2 * y * ww, 2 * y * z + 2 * x * ww, 1 - 2 * x * x - 2 * y * y]])
    a = 2 * q1
    b = np.array([-x, -y, -z, ww])
    t = np.array([a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1],
                  a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0],
                  a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3]])
    return R, t


def _image_terms(scene, pixels, frame0, image, gradient, geometry):
    W, H = scene.width, scene.height
    out = np.zeros((len(pixels), 8))
    for k, (x, y, v, _) in enumerate(np.asarray(pixels, np.int64)):
        view = scene.views[v]
        s = int(view.index_map[y, x])
        Rw, tw = unpack34(view.world2camera)
        Ri, ti = unpack34(view.initial_camera_se3)
        ref = view.reference_vertex_map[y, x, :3].astype(np.float64)
        if frame0:
            ref = Ri @ ref + ti
        R, t = dq_blend_se3(scene.node_se3, scene.surfel_knn[s], scene.surfel_knn_weight[s])
        wv = R @ ref + t
        vc = Ri.T @ (Rw @ wv + tw - ti)
        cx, cy, fx, fy = (float(a) for a in view.intrinsic)
        u = int(np.rint(np.float32(vc[0] / (vc[2] + 1e-10) * fx + cx)))
        r = int(np.rint(np.float32(vc[1] / (vc[2] + 1e-10) * fy + cy)))
        out[k, 7] = -1
        if 0 <= u < W and 0 <= r < H:
            img = float(image(view)[r, u])
            gx, gy = (float(a) for a in gradient(view)[r, u])
            d = np.array([gx * fx / vc[2], gy * fy / vc[2],
                          -1.0 / (vc[2] * vc[2]) * (fx * vc[0] * gx + fy * vc[1] * gy)])
            d = Rw.T @ (Ri @ d)
            out[k, :3] = [-d[1] * wv[2] + d[2] * wv[1], d[0] * wv[2] - d[2] * wv[0],
                          -d[0] * wv[1] + d[1] * wv[0]]
            out[k, 3:6] = d
            out[k, 6] = img - geometry(view, x, y)
            out[k, 7] = r * W + u
    return out


def density_terms(scene, pixels, frame0):
    """The density term (computeDensityMapJacobian,
    DensityForegroundJacobianResidual.cu:41-91) at the dense pixels: the
    observed grey level and its gradient, minus rgb2density of the rendered
    normalised rgb at the pixel (ColorTypeTransfer.h:51-56). Rows as in
    foreground_terms."""
    def geometry(view, x, y):
        c = view.normalized_rgb_map[y, x].astype(np.float32)
        return float(np.float32(0.299) * c[0] + np.float32(0.587) * c[1] + np.float32(0.114) * c[2])
    return _image_terms(scene, pixels, frame0, lambda v: v.density_map, lambda v: v.density_gradient_map, geometry)


def foreground_terms(scene, pixels, frame0):
    """(T, 8) float64 rows of the foreground terms at the compacted `pixels`
    ((T, 4) x, y, view, 0): the twist gradient (6), the residual, and the
    projected pixel y*W+x (-1 when the projection leaves the image, where the
    gradient and residual are 0)."""
    W, H = scene.width, scene.height
    out = np.zeros((len(pixels), 8))
    for k, (x, y, v, _) in enumerate(np.asarray(pixels, np.int64)):
        view = scene.views[v]
        s = int(view.index_map[y, x])
        Rw, tw = unpack34(view.world2camera)
        Ri, ti = unpack34(view.initial_camera_se3)
        ref = view.reference_vertex_map[y, x, :3].astype(np.float64)
        if frame0:
            ref = Ri @ ref + ti
        R, t = dq_blend_se3(scene.node_se3, scene.surfel_knn[s], scene.surfel_knn_weight[s])
        wv = R @ ref + t
        vc = Ri.T @ (Rw @ wv + tw - ti)
        cx, cy, fx, fy = (float(a) for a in view.intrinsic)
        u = int(np.rint(np.float32(vc[0] / (vc[2] + 1e-10) * fx + cx)))
        r = int(np.rint(np.float32(vc[1] / (vc[2] + 1e-10) * fy + cy)))
        out[k, 7] = -1
        if 0 <= u < W and 0 <= r < H:
            img = float(view.filtered_foreground_mask[r, u])
            gx, gy = (float(a) for a in view.foreground_mask_gradient[r, u])
            d = np.array([gx * fx / vc[2], gy * fy / vc[2],
                          -1.0 / (vc[2] * vc[2]) * (fx * vc[0] * gx + fy * vc[1] * gy)])
            d = Rw.T @ (Ri @ d)
            out[k, :3] = [-d[1] * wv[2] + d[2] * wv[1], d[0] * wv[2] - d[2] * wv[0],
                          -d[0] * wv[1] + d[1] * wv[0]]
            out[k, 3:6] = d
            out[k, 6] = img
            out[k, 7] = r * W + u
    return out
