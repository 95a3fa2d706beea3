"""Python mirror of the reference's SurfelNodeDeformer over the C ABI.

    SurfelNodeDeformer::ForwardWarpSurfelsAndNodes -> forward_warp_surfels_and_nodes
    SurfelNodeDeformer::InverseWarpSurfels         -> inverse_warp_surfels

(core/Geometry/SurfelNodeDeformer.h:28-89.) The reference writes the moved
surfels into every view's copy of the geometry; here there is one copy, in
tensors the caller owns. Arrays are CUDA tensors: float32 (n, 4) for
vertices, normals, weights and nodes, uint16 stored as int16 (n, 4) for KNN,
float32 (N, 8) for the warp field.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import abi, check, lib
from .solver import _stream_handle


def _surfels(knn, weight, vertex, normal, out_vertex, out_normal):
    s = abi.DeformSurfels()
    s.num_surfels = vertex.shape[0]
    s.knn, s.knn_weight = knn.data_ptr(), weight.data_ptr()
    s.in_vertex, s.in_normal = vertex.data_ptr(), normal.data_ptr()
    s.out_vertex, s.out_normal = out_vertex.data_ptr(), out_normal.data_ptr()
    return s


class SurfelNodeDeformer:
    @staticmethod
    def forward_warp_surfels_and_nodes(node_se3, knn, weight, canonical_vertex, canonical_normal, node_knn=None,
                                       node_weight=None, canonical_nodes=None, stream=None):
        """Live surfels (vertex, normal) and, with the node arrays, live nodes."""
        lv, ln = torch.empty_like(canonical_vertex), torch.empty_like(canonical_normal)
        s = _surfels(knn, weight, canonical_vertex, canonical_normal, lv, ln)
        live_nodes = None
        n = None
        if canonical_nodes is not None:
            live_nodes = torch.empty_like(canonical_nodes)
            n = abi.DeformNodes()
            n.num_nodes = canonical_nodes.shape[0]
            n.knn, n.knn_weight = node_knn.data_ptr(), node_weight.data_ptr()
            n.canonical_nodes, n.live_nodes = canonical_nodes.data_ptr(), live_nodes.data_ptr()
        check(lib().mvdr_forward_warp(C.c_void_p(node_se3.data_ptr()), node_se3.shape[0], C.byref(s),
                                      C.byref(n) if n is not None else None, _stream_handle(stream)))
        return lv, ln, live_nodes

    @staticmethod
    def inverse_warp_surfels(node_se3, knn, weight, live_vertex, live_normal, correct_se3=None, stream=None):
        """Canonical (reference) surfels from live ones; `correct_se3` (S, 12)
        mat34 per surfel is undone after the warp when given."""
        rv, rn = torch.empty_like(live_vertex), torch.empty_like(live_normal)
        s = _surfels(knn, weight, live_vertex, live_normal, rv, rn)
        cs = None if correct_se3 is None else C.c_void_p(correct_se3.data_ptr())
        check(lib().mvdr_inverse_warp(C.c_void_p(node_se3.data_ptr()), node_se3.shape[0], cs, C.byref(s),
                                      _stream_handle(stream)))
        return rv, rn
