"""Python mirror of the reference NonRigidSolver interface over the C ABI.

    NonRigidSolver.SetSolverInput(...)      -> NonRigidSolver.set_solver_input(scene)
    NonRigidSolver.SolveNonRigidAlignment() -> NonRigidSolver.solve_non_rigid_alignment(gn, pcg)
    NonRigidSolver.SolvedNodeSE3()          -> NonRigidSolver.solved_node_se3()

(core/NonRigidSolver/NonRigidSolver.h:133-140, 254, 214.) Device memory and
streams come from torch; every computation runs in libmvdr.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi, check, lib

_NP_TO_TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.uint16): torch.int16,
                np.dtype(np.uint32): torch.int32, np.dtype(np.float64): torch.float64,
                np.dtype(np.int32): torch.int32}

# element type and per-item width of each exported array
ARRAY_SPEC = {
    abi.ARRAY_DENSE_PIXELS: (np.uint16, 4), abi.ARRAY_DENSE_KNN: (np.uint16, 4),
    abi.ARRAY_DENSE_KNN_WEIGHT: (np.float32, 4), abi.ARRAY_FOREGROUND_PIXELS: (np.uint16, 4),
    abi.ARRAY_NODE2TERM_OFFSET: (np.uint32, 1), abi.ARRAY_NODE2TERM_INDEX: (np.uint32, 1),
    abi.ARRAY_HALF_NODEPAIR_KEY: (np.uint32, 1), abi.ARRAY_NODEPAIR_TERM_INDEX: (np.uint32, 1),
    abi.ARRAY_NODEPAIR_KEY: (np.uint32, 1), abi.ARRAY_NODEPAIR_TERM_RANGE: (np.uint32, 2),
    abi.ARRAY_BLKROW_OFFSET: (np.uint32, 1), abi.ARRAY_BINBLOCK_ROWPTR: (np.int32, 1),
    abi.ARRAY_BINBLOCK_COLPTR: (np.int32, 1), abi.ARRAY_TERM_JACOBIAN: (np.float32, 8),
    abi.ARRAY_SMOOTH_TERMS: (np.float32, 12), abi.ARRAY_WARPED_CORRESPONDENCE: (np.float32, 8),
    abi.ARRAY_DIAG_BLOCKS: (np.float32, 36), abi.ARRAY_JTR: (np.float32, 6),
    abi.ARRAY_PRECONDITIONER: (np.float32, 36), abi.ARRAY_OFFDIAG_BLOCKS: (np.float32, 36),
    abi.ARRAY_BINBLOCK_DATA: (np.float32, 1), abi.ARRAY_INCREMENT: (np.float32, 6),
    abi.ARRAY_NODE_SE3: (np.float32, 8), abi.ARRAY_DENSITY_JACOBIAN: (np.float32, 8),
    abi.ARRAY_FEATURE_TERMS: (np.float32, 8), abi.ARRAY_PCG_RESIDUALS: (np.float64, abi.MVDR_PCG_HISTORY),
}


def _check_image_size(config, ds):
    """The library reads every map as image_height rows of image_width (or
    pitch) elements and cannot see a buffer's size: maps of another size would
    be read past their end."""
    if ds.image_size != (config.image_width, config.image_height):
        raise ValueError(f"scene maps are {ds.image_size[0]}x{ds.image_size[1]}, the solver was created for "
                         f"{config.image_width}x{config.image_height}")


def _stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class DeviceScene:
    """Device copies (torch tensors) of every array of a synthetic scene."""

    def __init__(self, scene, device="cuda", pin=False, density=False):
        self.tensors = {}
        self.device = device
        self.pin = pin
        self.image_size = (scene.width, scene.height)
        arrays = []

        def collect(name, arr):
            a = np.ascontiguousarray(arr)
            if a.size:
                arrays.append((name, a.view(np.uint8).reshape(-1)))
            return None

        abi.fill_inputs(scene, collect, density)
        if pin:
            # one pinned arena, arrays at 256-byte offsets in input order: the
            # library's owned device copy has the same layout, so the upload
            # of an instance is a single transfer
            offs, total = {}, 0
            for name, a in arrays:
                offs[name] = total
                total += (a.size + 255) & ~255
            arena = torch.empty(total, dtype=torch.uint8).pin_memory()
            view = arena.numpy()
            for name, a in arrays:
                view[offs[name]:offs[name] + a.size] = a
                self.tensors[name] = arena[offs[name]:offs[name] + a.size]
            self._arena = arena
        else:
            for name, a in arrays:
                self.tensors[name] = torch.from_numpy(a.copy()).to(device)

        def ptr(name, arr):
            t = self.tensors.get(name)
            return None if t is None else t.data_ptr()

        self.inputs = abi.fill_inputs(scene, ptr, density)

    @property
    def nbytes(self):
        return sum(t.numel() for t in self.tensors.values())


class NonRigidSolver:
    def __init__(self, config):
        self.config = config
        h = C.c_void_p()
        check(lib().mvdr_create(C.byref(config), C.byref(h)))
        self.h = h
        self._inputs = None
        self.num_nodes = 0

    def close(self):
        if getattr(self, "h", None):
            lib().mvdr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # SetSolverInput
    def set_solver_input(self, scene, stream=None):
        ds = scene if isinstance(scene, DeviceScene) else DeviceScene(scene, density=bool(self.config.use_density))
        _check_image_size(self.config, ds)
        self._inputs = ds
        self.num_nodes = ds.inputs.num_nodes
        check(lib().mvdr_set_inputs(self.h, C.byref(ds.inputs), _stream_handle(stream)))
        return ds

    def set_solver_input_host(self, host_scene, stream=None):
        """`host_scene`: a DeviceScene built with pin=True (host pointers)."""
        _check_image_size(self.config, host_scene)
        self._inputs = host_scene
        self.num_nodes = host_scene.inputs.num_nodes
        check(lib().mvdr_set_inputs_host(self.h, C.byref(host_scene.inputs), _stream_handle(stream)))

    def build_index(self, stream=None):
        check(lib().mvdr_build_index(self.h, _stream_handle(stream)))

    def gn_iteration(self, pcg_iterations, stream=None):
        check(lib().mvdr_gn_iteration(self.h, pcg_iterations, _stream_handle(stream)))

    # SolveNonRigidAlignment
    def solve_non_rigid_alignment(self, gn_iterations, pcg_iterations, stream=None):
        check(lib().mvdr_solve(self.h, gn_iterations, pcg_iterations, _stream_handle(stream)))

    # SolvedNodeSE3
    def solved_node_se3(self, stream=None):
        out = torch.empty((self.num_nodes, 8), dtype=torch.float32, device="cuda")
        check(lib().mvdr_get_node_se3(self.h, C.c_void_p(out.data_ptr()), _stream_handle(stream)))
        return out

    def solved_node_se3_async(self, out, stream=None):
        """Enqueue the warp-field copy into `out` (device or pinned host) and
        return without synchronising; device-side errors are read later with
        counts()."""
        check(lib().mvdr_copy_node_se3_async(self.h, C.c_void_p(out.data_ptr()), _stream_handle(stream)))
        return out

    def counts(self, stream=None):
        c = abi.Counts()
        check(lib().mvdr_get_counts(self.h, C.byref(c), _stream_handle(stream)))
        return c

    def energy(self, stream=None):
        e = C.c_double()
        check(lib().mvdr_get_energy(self.h, C.byref(e), _stream_handle(stream)))
        return e.value

    def get_array(self, which, stream=None):
        dt, width = ARRAY_SPEC[which]
        cap = 1 << 22
        while True:
            buf = np.empty(cap // np.dtype(dt).itemsize, dt)
            written = C.c_size_t()
            st = lib().mvdr_get_array(self.h, which, buf.ctypes.data_as(C.c_void_p), buf.nbytes, C.byref(written),
                                      _stream_handle(stream))
            if st == abi.MVDR_ECAPACITY and written.value > buf.nbytes:
                cap = written.value
                continue
            check(st)
            out = buf[: written.value // np.dtype(dt).itemsize]
            return out.reshape(-1, width) if width > 1 else out

    def node_se3_device(self):
        """Device address of the warp field (the SolvedNodeSE3() view)."""
        p = C.c_void_p()
        check(lib().mvdr_node_se3_device(self.h, C.byref(p)))
        return p.value

    def save_input_bundle(self, path, stream=None):
        check(lib().mvdr_save_input_bundle(self.h, str(path).encode(), _stream_handle(stream)))

    # NonRigidSolver::ComputeAlignmentErrorOnNodes (+ the error maps)
    def compute_alignment_error_on_nodes(self, threshold=0.2, maps=False, stream=None):
        """Node alignment errors of the bound inputs under the current warp
        field: a dict of device tensors (accumulated_error, accumulated_weight,
        united_error, large_error_mark; with `maps`, per-view
        alignment_error_map and node_error_map of (H, W))."""
        N = self.num_nodes
        dev = torch.device("cuda", torch.cuda.current_device())
        out = {k: torch.empty(N, dtype=torch.float32, device=dev)
               for k in ("accumulated_error", "accumulated_weight", "united_error")}
        out["large_error_mark"] = torch.empty(N, dtype=torch.int32, device=dev)
        ne = abi.NodeError()
        ne.accumulated_error = out["accumulated_error"].data_ptr()
        ne.accumulated_weight = out["accumulated_weight"].data_ptr()
        ne.united_error = out["united_error"].data_ptr()
        ne.large_error_mark = out["large_error_mark"].data_ptr()
        ne.threshold = threshold
        if maps:
            V, H, W = self._inputs.inputs.num_views, self.config.image_height, self.config.image_width
            out["alignment_error_map"] = torch.empty((V, H, W), dtype=torch.float32, device=dev)
            out["node_error_map"] = torch.empty((V, H, W), dtype=torch.float32, device=dev)
            for v in range(V):
                ne.alignment_error_map[v] = out["alignment_error_map"][v].data_ptr()
                ne.node_error_map[v] = out["node_error_map"][v].data_ptr()
        check(lib().mvdr_compute_node_error(self.h, C.byref(ne), _stream_handle(stream)))
        return out

    # NonRigidSolver::CorrectLargeErrorNode (correspondence form)
    def correct_large_error_node(self, guides, united_error, live_nodes, node_knn, node_weight, live_vertex,
                                 live_normal, surfel_knn, surfel_weight, threshold=0.2, node_se3=None, stream=None):
        """`guides`: per bound view (se3 map (H, W, 12), valid (H, W) uint8,
        previous vertex map (H, W, 4)) device tensors. live_* are corrected in
        place, node_se3 too (None: the solver's own warp field); the
        corrected field becomes the solver's current one. Returns the
        per-node corrections (N, 8)."""
        corr = torch.empty((self.num_nodes, 8), dtype=torch.float32, device=live_nodes.device)
        c = abi.Correction()
        H, W = guides[0][1].shape
        c.width, c.height = W, H
        for v, (se3, valid, prev) in enumerate(guides):
            c.views[v].se3_map, c.views[v].valid_map = se3.data_ptr(), valid.data_ptr()
            c.views[v].previous_vertex_map, c.views[v].pitch = prev.data_ptr(), 0
        c.united_error, c.error_threshold = united_error.data_ptr(), threshold
        c.node_se3 = None if node_se3 is None else node_se3.data_ptr()
        c.live_nodes, c.node_knn, c.node_knn_weight = live_nodes.data_ptr(), node_knn.data_ptr(), node_weight.data_ptr()
        c.num_surfels = live_vertex.shape[0]
        c.live_vertex, c.live_normal = live_vertex.data_ptr(), live_normal.data_ptr()
        c.surfel_knn, c.surfel_knn_weight = surfel_knn.data_ptr(), surfel_weight.data_ptr()
        c.correction = corr.data_ptr()
        check(lib().mvdr_correct_large_error_nodes(self.h, C.byref(c), _stream_handle(stream)))
        return corr

    def apply_jtj(self, x, stream=None):
        x = x.contiguous().float()
        y = torch.empty_like(x)
        check(lib().mvdr_apply_jtj(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                   _stream_handle(stream)))
        return y


class BatchSolver:
    """Many independent solves of uneven sizes, one launch per stage."""

    def __init__(self, config, count):
        self.config = config
        self.count = count
        h = C.c_void_p()
        check(lib().mvdr_batch_create(C.byref(config), count, C.byref(h)))
        self.h = h
        self._inputs = [None] * count

    def close(self):
        if getattr(self, "h", None):
            lib().mvdr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_input(self, i, scene, stream=None):
        ds = scene if isinstance(scene, DeviceScene) else DeviceScene(scene, density=bool(self.config.use_density))
        _check_image_size(self.config, ds)
        self._inputs[i] = ds
        check(lib().mvdr_batch_set_inputs(self.h, i, C.byref(ds.inputs), _stream_handle(stream)))
        return ds

    def set_input_host(self, i, host_scene, stream=None):
        _check_image_size(self.config, host_scene)
        self._inputs[i] = host_scene
        check(lib().mvdr_batch_set_inputs_host(self.h, i, C.byref(host_scene.inputs), _stream_handle(stream)))

    def solve(self, gn, pcg, use_graph=True, stream=None):
        check(lib().mvdr_batch_solve(self.h, gn, pcg, int(use_graph), _stream_handle(stream)))

    def node_se3(self, i, out=None, stream=None):
        n = self._inputs[i].inputs.num_nodes
        if out is None:
            out = torch.empty((n, 8), dtype=torch.float32, device="cuda")
        check(lib().mvdr_batch_get_node_se3(self.h, i, C.c_void_p(out.data_ptr()), _stream_handle(stream)))
        return out

    def node_se3_async(self, i, out, stream=None):
        """Enqueue instance i's warp-field copy into `out`; no synchronisation
        and no error check (see NonRigidSolver.solved_node_se3_async)."""
        check(lib().mvdr_batch_copy_node_se3_async(self.h, i, C.c_void_p(out.data_ptr()), _stream_handle(stream)))
        return out

    def autotune(self, stream=None):
        """Pick the SpMV tile shape for this batch (see mvdr_batch_autotune);
        the inputs must be bound again before the next solve. Returns
        ((rows, split, form), per-candidate ms), the shape as in
        abi.SPMV_SHAPES."""
        times = (C.c_double * 32)()
        rows, split, form = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().mvdr_batch_autotune(self.h, _stream_handle(stream), times, 32, C.byref(rows), C.byref(split),
                                        C.byref(form)))
        return (rows.value, split.value, form.value), [t for t in times[:abi.NUM_SPMV_SHAPES]]

    def set_pcg_persistent(self, on=True):
        """One persistent cooperative launch per PCG solve (materialised
        mode) instead of two (mixed precision) or three launches per
        iteration."""
        check(lib().mvdr_batch_set_pcg_persistent(self.h, 1 if on else 0))

    def set_wait_limit(self, limit_ns, extra_arrivals=0):
        """Limit of each bounded barrier wait of the persistent PCG;
        extra_arrivals > 0 makes every barrier wait for arrivals that never
        come (exercises the MVDR_ETIMEOUT path)."""
        check(lib().mvdr_batch_set_wait_limit(self.h, int(limit_ns), int(extra_arrivals)))

    def set_spmv_shape(self, index):
        """Use SpMV tile shape `index` of abi.SPMV_SHAPES for later solves."""
        check(lib().mvdr_batch_set_spmv_shape(self.h, index))

    def instance(self, i):
        """NonRigidSolver-like view of one member (for checks); not owned."""
        h = C.c_void_p()
        check(lib().mvdr_batch_instance(self.h, i, C.byref(h)))
        n = self._inputs[i].inputs.num_nodes if self._inputs[i] else 0
        return _InstanceView(h, n, self.config)


def lane_sizes(count, lanes):
    """Sizes of the member batches of a batch of `count` split into `lanes`
    (at most `count`, at least 1): equal, the first ones one larger when
    `count` does not divide."""
    lanes = max(1, min(int(lanes), int(count)))
    base, extra = divmod(int(count), lanes)
    return [base + (1 if k < extra else 0) for k in range(lanes)]


class StreamedBatch:
    """A batch of independent solves split into `lanes` member batches, each
    solved (as its own CUDA graph) on a stream of its own. The solve's kernels
    are latency-bound and one batch leaves the GPU partly idle at every kernel
    boundary and in its small kernels; a second batch's kernels run in those
    gaps. Instance i lives in lane k at position i - start[k] (lanes of equal
    size, the first ones one larger when `count` does not divide).

    The calls take the caller's stream as BatchSolver's do: inputs are bound
    on it, and solve() starts the lanes after the work already queued there
    and makes it wait for all of them, so results are read on it as usual.
    Each instance's arithmetic is the same as in one batch of `count` with
    the same SpMV tile shape; only the launch grids' instance dimension
    differs."""

    def __init__(self, config, count, lanes=2):
        self.config = config
        self.count = count
        self.sizes = lane_sizes(count, lanes)
        self.starts = [sum(self.sizes[:k]) for k in range(lanes)]
        self.lanes = [BatchSolver(config, n) for n in self.sizes]
        self.streams = [torch.cuda.Stream() for _ in self.lanes]

    def close(self):
        for b in getattr(self, "lanes", []):
            b.close()

    def lane_of(self, i):
        """(lane, position in the lane) of instance i."""
        if not 0 <= i < self.count:
            raise IndexError(f"instance {i} of a batch of {self.count}")
        k = max(k for k in range(len(self.lanes)) if self.starts[k] <= i)
        return k, i - self.starts[k]

    def set_input(self, i, scene, stream=None):
        k, j = self.lane_of(i)
        return self.lanes[k].set_input(j, scene, stream=stream)

    def set_input_host(self, i, host_scene, stream=None):
        k, j = self.lane_of(i)
        self.lanes[k].set_input_host(j, host_scene, stream=stream)

    def solve(self, gn, pcg, use_graph=True, stream=None):
        caller = stream if stream is not None else torch.cuda.current_stream()
        start = torch.cuda.Event()
        start.record(caller)
        done = []
        for b, s in zip(self.lanes, self.streams):
            s.wait_event(start)
            b.solve(gn, pcg, use_graph=use_graph, stream=s)
            e = torch.cuda.Event()
            e.record(s)
            done.append(e)
        for e in done:
            caller.wait_event(e)

    def node_se3(self, i, out=None, stream=None):
        k, j = self.lane_of(i)
        return self.lanes[k].node_se3(j, out=out, stream=stream)

    def node_se3_async(self, i, out, stream=None):
        k, j = self.lane_of(i)
        return self.lanes[k].node_se3_async(j, out, stream=stream)

    def autotune(self, stream=None):
        """Tune each lane's SpMV tile shape; returns lane 0's result."""
        return [b.autotune(stream=stream) for b in self.lanes][0]

    def set_spmv_shape(self, index):
        for b in self.lanes:
            b.set_spmv_shape(index)

    def set_pcg_persistent(self, on=True):
        for b in self.lanes:
            b.set_pcg_persistent(on)

    def instance(self, i):
        k, j = self.lane_of(i)
        return self.lanes[k].instance(j)


class _InstanceView(NonRigidSolver):
    """A batch member seen through the single-solver interface. Its handle
    belongs to the batch, so closing the view releases nothing."""

    def __init__(self, h, num_nodes, config):
        self.h = h
        self.num_nodes = num_nodes
        self.config = config
        self._inputs = None

    def close(self):
        self.h = None
