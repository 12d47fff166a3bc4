"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes as C
import glob
import os
import re

import pytest

from fastwarp_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names.update(re.findall(r"\b(fw_[a-z0-9_]+)\s*\(", open(h).read()))
    return sorted(names)


def test_the_library_is_built_in_tree_for_sm100a():
    assert os.path.exists(N.LIB_PATH), "build with `make -C fastwarp_b200/csrc`"


@pytest.mark.parametrize("name", declared())
def test_every_declared_entry_point_is_exported(name):
    lib = N.lib()
    assert hasattr(lib, name), f"{name} is declared in include/ but not exported"


def test_struct_layouts_match_the_header():
    # sizes follow from the C declarations (natural alignment on x86-64)
    assert C.sizeof(N.Grid) == 8 * 3 + 8 * 3 + 8 * 3 + 8 * 9
    assert C.sizeof(N.Affine) == 8 * 12
    assert C.sizeof(N.InvertParams) == 32
    assert C.sizeof(N.InvertStats) == 24
    assert C.sizeof(N.MiBinning) == 8 + 8 * 8
    assert C.sizeof(N.LinearTransform) == 8 * 15 + 8 + 8 * 15
    assert C.sizeof(N.SynIteration) == 8 * 6 + 24 * 4
    assert C.sizeof(N.Stats) == 8 * 7


def test_the_backend_name_and_error_reporting_work_without_a_device():
    lib = N.lib()
    assert lib.fw_backend_name().decode().startswith("cuda")
    out = (C.c_uint32 * 3)()
    assert lib.fw_shrink_factors(C.c_uint32(4), (C.c_double * 3)(1.0, 2.0, 1.0), out) == 0
    assert tuple(out) == (4, 2, 4)
    g = N.Grid()
    bad = N.Grid()
    assert lib.fw_shrink_grid(C.byref(bad), (C.c_uint32 * 3)(2, 2, 2), C.byref(g)) == N.FW_ERR_INVALID
    assert b"zero size" in lib.fw_last_error()


def test_every_mirrored_struct_has_the_library_layout_size():
    import ctypes as C

    from fastwarp_b200 import _native as N
    from fastwarp_b200 import serve as S
    pairs = {"fw_grid": N.Grid, "fw_affine": N.Affine, "fw_invert_params": N.InvertParams,
             "fw_invert_stats": N.InvertStats, "fw_mi_binning": N.MiBinning,
             "fw_linear_transform": N.LinearTransform, "fw_syn_recipe": N.SynRecipe,
             "fw_syn_iteration": N.SynIteration, "fw_stats": N.Stats,
             "fw_syn_request": S.SynRequest, "fw_syn_result": S.SynResultC,
             "fw_server_stats": S.ServerStats, "fw_cg_settings": N.CgSettings,
             "fw_cg_trace": N.CgTrace, "fw_transform_elem": N.TransformElem,
             "fw_linear_recipe": N.LinearRecipe, "fw_linear_level_trace": N.LinearLevelTrace,
             "fw_linear_request": S.LinearRequest, "fw_linear_result": S.LinearResultC,
             "fw_linear_chain_result": N.LinearChainResult, "fw_batch_subject": N.BatchSubject,
             "fw_batch_tuning": N.BatchTuning, "fw_batch_report": N.BatchReport}
    for name, cls in pairs.items():
        assert N.lib().fw_abi_struct_size(name.encode()) == C.sizeof(cls), name
    assert N.lib().fw_abi_struct_size(b"no such struct") == 0
