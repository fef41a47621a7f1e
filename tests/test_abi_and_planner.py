"""CPU checks of the C ABI surface and the host-side hierarchy planner."""
import ctypes
import os
import re

import pytest

from fluid_b200 import _abi, plan_uniform_cm11a_hierarchy
from oracle.oracle import plan_hierarchy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fluid_pp.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fluid_pp_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_abi.EXPORTS)


def test_library_links_no_torch_and_needs_no_gpu_to_load():
    lib = _abi.load()
    # host-only entry points work without a device
    assert lib.fluid_pp_kernel_launches() >= 0
    assert plan_uniform_cm11a_hierarchy((32, 32, 32))["levelCount"] == 5


# Lattices of the workloads plus edge cases of mg.ts:99-169.
DIMS = [(32, 32, 32), (128, 96, 128), (64, 32, 64), (24, 24, 24), (2, 2, 2), (2, 64, 64), (128, 128, 8),
        (16, 8, 8), (37, 50, 99), (24, 128, 77), (3, 3, 3), (4, 3, 4), (256, 1024, 256), (64, 64, 2),
        (160, 160, 160), (33, 33, 33), (100, 100, 100), (2, 3, 2), (48, 96, 200), (127, 31, 64)]


@pytest.mark.parametrize("dims", DIMS)
def test_planner_matches_oracle_bit_exact(dims):
    product = plan_uniform_cm11a_hierarchy(dims)
    ref = plan_hierarchy(*dims)
    assert (product["rejection"] is None) == ref["ok"]
    if not ref["ok"]:
        return
    assert product["levelDimensions"] == ref["levels"]
    assert product["coarsestCells"] == ref["coarsest_cells"]
    assert product["semiCoarsened"] == ref["semi"]
    assert product["extended"] == ref["extended"]


def _reference_rules(dims):
    """planUniformCM11aHierarchy restated literally (mg.ts:99-169); None = rejected."""
    import math
    if min(dims) < 2:
        return None
    haloed = lambda d: (d[0] + 2) * (d[1] + 2) * (d[2] + 2)
    m = min(dims)
    levels = None
    if m & (m - 1) == 0:
        count = int(math.floor(math.log2(m)))
        c = 2 ** (count - 1)
        if all(v % c == 0 for v in dims):
            lv = [tuple(v // 2 ** i for v in dims) for i in range(count)]
            if haloed(lv[-1]) <= 256:
                levels = lv
    if levels is None:
        levels = [tuple(dims)]
        while True:
            nxt = tuple(v // 2 if v % 2 == 0 and v > 2 else v for v in levels[-1])
            if nxt == levels[-1]:
                break
            levels.append(nxt)
    if haloed(levels[-1]) > 256:
        return None
    return levels


@pytest.mark.parametrize("dims", DIMS)
def test_planner_agrees_with_reference_rules_where_reference_accepts(dims):
    ref = _reference_rules(dims)
    product = plan_uniform_cm11a_hierarchy(dims)
    if ref is None:
        assert product["rejection"] is not None or product["extended"]
    else:
        assert not product["extended"]
        assert product["levelDimensions"] == ref


def test_planner_known_level_maps():
    assert plan_uniform_cm11a_hierarchy((32, 32, 32))["levelDimensions"] == [
        (32, 32, 32), (16, 16, 16), (8, 8, 8), (4, 4, 4), (2, 2, 2)]
    p = plan_uniform_cm11a_hierarchy((128, 96, 128))
    assert p["levelCount"] == 7 and p["coarsestCells"] == 4 * 5 * 4 and p["semiCoarsened"]
    assert plan_uniform_cm11a_hierarchy((1, 8, 8))["rejection"]


def test_create_rejects_bad_arguments_without_gpu():
    from fluid_b200 import PressureProjector
    with pytest.raises(ValueError):
        PressureProjector((1, 8, 8), 0.1)
    with pytest.raises(ValueError):
        PressureProjector((8, 8, 8), -1.0)


def test_noalloc_rejects_lattices_beyond_its_scratch():
    """The size check comes before any CUDA call (no GPU needed)."""
    L = _abi.load()
    one = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = L.fluid_pp_apply_operator_noalloc(4096, 4096, 64, one, one, one, one, one, None)
    assert rc == _abi.INVALID_ARG
    assert b"fixed scratch" in L.fluid_pp_last_error(None)


def test_noalloc_rejects_outputs_that_alias_inputs():
    """The allocation-free operator apply rejects out = p (an in-place call), a dot
    slot inside an input and partly overlapping buffers before any CUDA call; the
    pointers are never dereferenced, so this runs without a GPU."""
    L = _abi.load()
    n = 16 * 16 * 16
    base = 1 << 20
    lab, dg, p, out, dot = (ctypes.c_void_p(base + k * 4 * n + 256) for k in range(5))
    assert L.fluid_pp_apply_operator_noalloc(16, 16, 16, lab, dg, p, p, dot, None) == _abi.INVALID_ARG
    assert b"must not overlap" in L.fluid_pp_last_error(None)
    inside_p = ctypes.c_void_p(p.value + 64)
    assert L.fluid_pp_apply_operator_noalloc(16, 16, 16, lab, dg, p, out, inside_p, None) == _abi.INVALID_ARG
    half_over = ctypes.c_void_p(dg.value + 2 * n)
    assert L.fluid_pp_apply_operator_noalloc(16, 16, 16, lab, dg, p, half_over, dot, None) == _abi.INVALID_ARG
