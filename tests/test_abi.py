"""CPU tests of the C ABI library: it loads, exports every symbol include/gt.h declares, and fails
cleanly (status codes, no exit) where it can be exercised without a GPU."""
import ctypes as C
import os
import re

import pytest

import gizmo_shared_memory_b200 as g
from gizmo_shared_memory_b200 import _gt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gt.h")).read()
    return sorted(set(re.findall(r"^GT_API\s+[\w\s\*]+?\b(gt_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    L = g.load_library()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_gt.EXPORTS) == names


def test_version_and_status_strings():
    L = g.load_library()
    assert L.gt_version() == 1
    for code, name in _gt.STATUS.items():
        assert L.gt_status_string(code).decode() == name


def test_option_defaults_match_reference_constants():
    L = g.load_library()
    o = _gt.BuildOptions()
    L.gt_build_options_default(C.byref(o))
    assert (o.leaf_max, o.max_level, o.randomize_seed) == (16, 20, -1)  # shmem/tree.h:357-358
    w = _gt.WalkOptions()
    L.gt_walk_options_default(C.byref(w))
    assert w.group_mode == g.GT_GROUP_LEAF and w.mac == g.GT_MAC_PLAIN
    assert w.sink_direct_radius == 0.0  # accel_grouped's default (tree.h:440)


def test_null_arguments_are_rejected():
    L = g.load_library()
    assert L.gt_build(None, 0, None, None, None, None, None, 0, None, None) == 1
    assert L.gt_context_destroy(None) == 1
    assert L.gt_tree_free(None) == 1
    assert L.gt_synchronize(None) == 1


def test_context_without_gpu_reports_device_error():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(g.GTError) as e:
        g.Context(0)
    assert e.value.status == 8  # GT_ERR_DEVICE
