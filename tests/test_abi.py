"""The C-ABI library loads without a GPU, exports every function declared in
include/mvdr.h, and its struct layouts match the ctypes mirror."""
import ctypes as C
import os
import re

import pytest

import multiviewdynrecon_b200 as m
from multiviewdynrecon_b200 import abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "mvdr.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mvdr_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def L():
    if not os.path.exists(m.LIB_PATH):
        m.build()
    return m.lib()


def test_exports_every_declared_symbol(L):
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match(L):
    for name, cls in abi.STRUCTS.items():
        size = C.c_size_t()
        assert L.mvdr_abi_layout(name.encode(), C.byref(size)) == abi.MVDR_OK, name
        assert size.value == C.sizeof(cls), (name, size.value, C.sizeof(cls))


def test_config_default_and_errors_without_gpu(L):
    cfg = abi.Config()
    L.mvdr_config_default(C.byref(cfg), 4096, 3, 640, 480)
    assert cfg.abi_version == abi.MVDR_ABI_VERSION
    assert cfg.precision == abi.PRECISION_MIXED and cfg.max_nodes == 4096
    # invalid configurations are rejected on the host before any CUDA call
    bad = abi.Config()
    L.mvdr_config_default(C.byref(bad), 70000, 3, 640, 480)
    h = C.c_void_p()
    assert L.mvdr_create(C.byref(bad), C.byref(h)) == abi.MVDR_EINVAL
    assert b"max_nodes" in L.mvdr_last_error_string()
    bad.max_nodes = 10
    bad.abi_version = 99
    assert L.mvdr_create(C.byref(bad), C.byref(h)) == abi.MVDR_EINVAL
    assert L.mvdr_destroy(None) == abi.MVDR_OK
    assert L.mvdr_set_inputs(None, None, None) == abi.MVDR_EINVAL


def test_spmv_shape_count_matches_header(L):
    text = open(HEADER).read()
    n = int(re.search(r"#define MVDR_NUM_SPMV_SHAPES (\d+)u", text).group(1))
    assert n == abi.NUM_SPMV_SHAPES
    assert L.mvdr_batch_set_spmv_shape(None, 0) == abi.MVDR_EINVAL


def test_enum_constants_match_header():
    """Every MVDR_* enumerator of the header (status codes, precision, mode,
    stage and array ids) has the value the ctypes mirror uses."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    found = dict((k, int(v)) for k, v in re.findall(r"\b(MVDR_[A-Z0-9_]+)\s*=\s*(\d+)\b", text))
    mirror = {"MVDR_OK": abi.MVDR_OK, "MVDR_EINVAL": abi.MVDR_EINVAL, "MVDR_ECAPACITY": abi.MVDR_ECAPACITY,
              "MVDR_ECUDA": abi.MVDR_ECUDA, "MVDR_ETIMEOUT": abi.MVDR_ETIMEOUT,
              "MVDR_ENONFINITE": abi.MVDR_ENONFINITE, "MVDR_ESTATE": abi.MVDR_ESTATE,
              "MVDR_PRECISION_FP32": abi.PRECISION_FP32, "MVDR_PRECISION_MIXED": abi.PRECISION_MIXED,
              "MVDR_MODE_MATERIALIZED": abi.MODE_MATERIALIZED, "MVDR_MODE_MATRIX_FREE": abi.MODE_MATRIX_FREE}
    for name in dir(abi):
        if name.startswith(("STAGE_", "ARRAY_")):
            mirror["MVDR_" + name] = getattr(abi, name)
    stages = sorted(k for k in found if k.startswith("MVDR_STAGE_"))
    arrays = sorted(k for k in found if k.startswith("MVDR_ARRAY_"))
    assert stages == sorted(k for k in mirror if k.startswith("MVDR_STAGE_"))
    assert arrays == sorted(k for k in mirror if k.startswith("MVDR_ARRAY_"))
    for k, v in mirror.items():
        assert found.get(k) == v, k


def test_lane_sizes_split_a_batch_evenly():
    """StreamedBatch's member batches: equal sizes, the first ones one larger
    when the count does not divide; never more lanes than instances."""
    from multiviewdynrecon_b200.solver import lane_sizes
    assert lane_sizes(16, 2) == [8, 8]
    assert lane_sizes(16, 3) == [6, 5, 5]
    assert lane_sizes(3, 2) == [2, 1]
    assert lane_sizes(2, 4) == [1, 1]
    assert lane_sizes(5, 0) == [5]
    for n in range(1, 40):
        for k in range(1, 9):
            s = lane_sizes(n, k)
            assert sum(s) == n and max(s) - min(s) <= 1 and len(s) == min(n, k)
