"""Python mirror of the renderer's solver-map interface over the C ABI.

    Renderer::DrawSolverMapsWithRecentObservation(num_vertex, vao, time, world2camera)
        -> SolverMapRenderer.draw_solver_maps_with_recent_observation(geometry, time, cameras)
    Renderer::DrawSolverMapsConfidentObservation(...)
        -> SolverMapRenderer.draw_solver_maps_confident_observation(geometry, time, cameras)
    Renderer::MapSolverMapsToCuda(SolverMaps*)  -> SolverMapRenderer.maps(view)

(render/Renderer.h:381-393, render/RendererDraw.cpp:355-480.) The reference
draws the surfels with OpenGL and maps the render targets into CUDA; here the
maps are device buffers written by mvdr_render_solver_maps, so there is no
map/unmap step. View 0 is drawn with the sized-point shader when
`sized_view0` is set (SolverMapSized.vert; the reference picks it at compile
time), every other view with one-pixel points (SolverMapIndexMap.vert).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi, check, lib
from .solver import _stream_handle


class SolverMapRenderer:
    """Device-resident solver maps of `num_views` views of width x height:
    reference/live vertex and normal maps (float4, in each view's camera
    frame), the surfel index map (uint32, 0xFFFFFFFF = empty), the normalised
    rgb map and the 64-bit depth-index scratch of the depth test."""

    def __init__(self, width, height, num_views, max_depth=3.0, confidence_threshold=10.0,
                 recent_time_threshold=3.0, sized_view0=False, device="cuda"):
        if not 1 <= num_views <= abi.MVDR_MAX_VIEWS:
            raise ValueError("num_views must be in [1, MVDR_MAX_VIEWS]")
        self.width, self.height, self.num_views = width, height, num_views
        self.max_depth = max_depth
        self.confidence_threshold = confidence_threshold
        self.recent_time_threshold = recent_time_threshold
        self.sized_view0 = sized_view0
        shape = (num_views, height, width)
        f4 = dict(dtype=torch.float32, device=device)
        self.reference_vertex = torch.empty(shape + (4,), **f4)
        self.reference_normal = torch.empty(shape + (4,), **f4)
        self.live_vertex = torch.empty(shape + (4,), **f4)
        self.live_normal = torch.empty(shape + (4,), **f4)
        self.normalized_rgb = torch.empty(shape + (4,), **f4)
        self.index = torch.empty(shape, dtype=torch.int32, device=device)
        self.depth_index = torch.empty(shape, dtype=torch.int64, device=device)

    def _views(self, cameras):
        out = (abi.SolverMapView * len(cameras))()
        for v, cam in enumerate(cameras):
            ptrs = {"reference_vertex_map": self.reference_vertex[v].data_ptr(),
                    "reference_normal_map": self.reference_normal[v].data_ptr(),
                    "live_vertex_map": self.live_vertex[v].data_ptr(),
                    "live_normal_map": self.live_normal[v].data_ptr(),
                    "index_map": self.index[v].data_ptr(),
                    "normalized_rgb_map": self.normalized_rgb[v].data_ptr(),
                    "depth_index": self.depth_index[v].data_ptr()}
            out[v] = abi.solver_map_view(cam, ptrs, sized_points=self.sized_view0 and v == 0)
        return out

    def _draw(self, geometry, current_time, cameras, time_threshold, stream):
        if len(cameras) != self.num_views:
            raise ValueError(f"expected {self.num_views} cameras, got {len(cameras)}")
        tensors = {k: geometry[k] for k in abi.SURFEL_ARRAYS}
        n = int(tensors["live_vertex_confid"].shape[0])
        for k, t in tensors.items():
            if t.dtype != torch.float32 or t.shape != (n, 4) or not t.is_contiguous() or not t.is_cuda:
                raise ValueError(f"{k}: expected a contiguous CUDA float32 tensor of shape ({n}, 4)")
        g = abi.surfel_geometry(n, {k: t.data_ptr() for k, t in tensors.items()})
        prm = abi.solver_map_params(self.width, self.height, self.max_depth, float(current_time),
                                    self.confidence_threshold, time_threshold)
        views = self._views(cameras)
        check(lib().mvdr_render_solver_maps(C.byref(g), C.byref(prm), views, self.num_views,
                                            _stream_handle(stream)))

    def draw_solver_maps_with_recent_observation(self, geometry, current_time, cameras, stream=None):
        """Unstable surfels observed within the recent-time threshold are drawn."""
        self._draw(geometry, current_time, cameras, self.recent_time_threshold, stream)

    def draw_solver_maps_confident_observation(self, geometry, current_time, cameras, stream=None):
        """Only surfels at or above the confidence threshold are drawn (the
        time threshold is -1, RendererDraw.cpp:414-417)."""
        self._draw(geometry, current_time, cameras, -1.0, stream)

    def maps(self, v):
        return {"reference_vertex_map": self.reference_vertex[v], "reference_normal_map": self.reference_normal[v],
                "live_vertex_map": self.live_vertex[v], "live_normal_map": self.live_normal[v],
                "index_map": self.index[v], "normalized_rgb_map": self.normalized_rgb[v]}

    def bind(self, device_scene):
        """Point a DeviceScene's per-view reference maps, index maps and rgb
        maps at these maps (the solver's inputs from the renderer,
        SolverMaps of Renderer.h:381-388)."""
        for v in range(device_scene.inputs.num_views):
            vi = device_scene.inputs.views[v]
            vi.reference_vertex_map = self.reference_vertex[v].data_ptr()
            vi.reference_normal_map = self.reference_normal[v].data_ptr()
            vi.index_map = self.index[v].data_ptr()
            if vi.normalized_rgb_map:
                vi.normalized_rgb_map = self.normalized_rgb[v].data_ptr()
            vi.pitch = 0
        device_scene._solver_maps = self
        return device_scene


def geometry_to_device(geometry, device="cuda"):
    """numpy surfel arrays -> contiguous device tensors."""
    return {k: torch.from_numpy(np.ascontiguousarray(geometry[k], np.float32)).to(device) for k in abi.SURFEL_ARRAYS}
