"""Host-side logic that needs no GPU: argument checks of the C ABI, tuning
candidates, workload keys, truth tables and the bench's byte count."""

import ctypes
import os

import numpy as np
import pytest

from subsetix_b200 import _core, _lib, autotune


def _lib_or_skip():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")
    import torch

    if torch.cuda.is_available():
        # the calls below pass placeholder pointers and must fail their host checks; a
        # machine with a GPU is not the place to find out whether one ever stops doing so
        pytest.skip("host-check tests run only without a GPU")
    return _lib.load()


def _one_leaf():
    arr = (_lib.SxLeaf * 1)()
    arr[0].begin = 16
    arr[0].end = 16
    arr[0].row_offsets = 16  # never dereferenced: every call below fails its checks first
    return arr


@pytest.mark.parametrize("field,value", [("kernel", 8), ("kernel", -1), ("warps", 9), ("tile_rows", 33),
                                         ("tile_rows", -2), ("staging_cap", -5), ("blocks_per_sm", -1),
                                         ("wait_limit", -1), ("withhold_tile", -3)])
def test_bool_eval_rejects_bad_tuning_on_the_host(field, value):
    lib = _lib_or_skip()
    tun = _lib.SxTuning(0, 0, 0, 0, 0, 0, 0)
    setattr(tun, field, value)
    tab = (ctypes.c_uint32 * 8)(0b1110, 0, 0, 0, 0, 0, 0, 0)
    rows = 64
    ws = lib.sx_bool_workspace_bytes(rows)
    rc = lib.sx_bool_eval(_one_leaf(), 1, rows, tab, _lib.MODE_TABLE, 16, 16, 16, 100, 16, 16, ws,
                          ctypes.byref(tun), None)
    assert rc == _lib.SX_ERR_INVALID
    assert "tuning" in _lib.last_error()


def test_bool_eval_rejects_row_lane_tiles_of_other_heights_on_the_host():
    lib = _lib_or_skip()
    tun = _lib.SxTuning(7, 0, 0, 0, 12, 0, 0)
    tab = (ctypes.c_uint32 * 8)(0b1110, 0, 0, 0, 0, 0, 0, 0)
    rows = 64
    ws = lib.sx_bool_workspace_bytes(rows)
    rc = lib.sx_bool_eval(_one_leaf(), 1, rows, tab, _lib.MODE_TABLE, 16, 16, 16, 100, 16, 16, ws,
                          ctypes.byref(tun), None)
    assert rc == _lib.SX_ERR_INVALID
    assert "32 rows" in _lib.last_error()


def test_bool_eval_rejects_a_short_workspace_on_the_host():
    lib = _lib_or_skip()
    tab = (ctypes.c_uint32 * 8)(0b1110, 0, 0, 0, 0, 0, 0, 0)
    rc = lib.sx_bool_eval(_one_leaf(), 1, 1 << 20, tab, _lib.MODE_TABLE, 16, 16, 16, 100, 16, 16, 64, None, None)
    assert rc == _lib.SX_ERR_WORKSPACE


def test_explicit_tile_height_is_refused_when_its_state_does_not_fit():
    """An explicit tile_rows is never silently replaced by 32-row tiles: a short workspace is an error."""
    lib = _lib_or_skip()
    tab = (ctypes.c_uint32 * 8)(0b1110, 0, 0, 0, 0, 0, 0, 0)
    rows = 1 << 16
    ws32 = lib.sx_bool_workspace_bytes(rows // 32)  # enough for 32-row tiles only
    for kernel, tile_rows in ((5, 1), (6, 3), (4, 16)):
        tun = _lib.SxTuning(kernel, 0, 0, 0, tile_rows, 0, 0)
        rc = lib.sx_bool_eval(_one_leaf(), 1, rows, tab, _lib.MODE_TABLE, 16, 16, 16, 100, 16, 16, ws32,
                              ctypes.byref(tun), None)
        assert rc == _lib.SX_ERR_WORKSPACE, (kernel, tile_rows)
        assert f"{tile_rows}-row tiles" in _lib.last_error()


def test_workspace_for_small_tiles_covers_32_row_tiles():
    lib = _lib_or_skip()
    for rows in (1, 31, 32, 33, 1000, 1 << 20):
        assert lib.sx_bool_workspace_bytes(rows) >= lib.sx_bool_workspace_bytes(max(1, rows // 8))


@pytest.mark.parametrize("k,rows,a,b", [(0, 8, 8, 32), (1, -1, 8, 32), (1, 8, 0, 32), (1, 8, 8, 0)])
def test_tile_boundaries_max_rejects_bad_arguments(k, rows, a, b):
    lib = _lib_or_skip()
    rc = lib.sx_tile_boundaries_max(_one_leaf(), k, rows, a, b, 16, None)
    assert rc == _lib.SX_ERR_INVALID


def test_tile_boundaries_max_needs_offsets():
    lib = _lib_or_skip()
    arr = (_lib.SxLeaf * 1)()
    assert lib.sx_tile_boundaries_max(arr, 1, 8, 8, 32, 16, None) == _lib.SX_ERR_INVALID
    assert "offsets" in _lib.last_error()


def test_workload_key_buckets():
    assert _core.workload_key([100, 100], 64) == _core.workload_key([120, 90], 64)
    assert _core.workload_key([100, 100], 64) != _core.workload_key([100, 100, 100], 64)
    assert _core.workload_key([100], 64) != _core.workload_key([10000], 64)
    assert autotune.workload_key is _core.workload_key


def test_autotune_candidates_cover_every_kernel_kind():
    sizes = [40000] * 5
    cands = autotune.candidates(sizes, 4096, largest_tile=5000, largest_eighth_tile=1300, largest_half_tile=2600)
    kinds = {c["kernel"] for c in cands}
    assert {1, 3, 4, 5, 6, 7} <= kinds
    for c in cands:
        if c["kernel"] == 7:
            assert c["tile_rows"] in (16, 32) and c["staging_cap"] >= (2600 if c["tile_rows"] == 16 else 5000)
        if c["kernel"] in (5, 6):
            assert c["tile_rows"] == 8 and 1300 <= c["staging_cap"] <= 25000
        if c["kernel"] == 4:
            assert c["tile_rows"] == 32 and 5000 <= c["staging_cap"] <= 25000


def test_truth_tables_of_the_binary_operations():
    from subsetix_b200.subsetix_cupy import expressions as E

    words = {"union": 0b1110, "intersection": 0b1000, "difference": 0b0010, "symmetric_difference": 0b0110}
    for op, word in words.items():
        node = E._remap((op, ("leaf", 0), ("leaf", 1)), {0: 0, 1: 1})
        assert int(E.truth_table(node, 2)[0]) == word, op


def test_truth_table_of_eight_leaves_spans_words():
    from subsetix_b200.subsetix_cupy import expressions as E

    node = E._remap(("union", ("leaf", 7), ("intersection", ("leaf", 0), ("leaf", 1))), {i: i for i in range(8)})
    table = [int(x) for x in E.truth_table(node, 8)]
    for state in range(256):
        want = bool(state & 0x80) or (bool(state & 1) and bool(state & 2))
        assert bool((table[state >> 5] >> (state & 31)) & 1) == want, state


def test_algorithmic_bytes_counts_inputs_once_and_the_output_once():
    import bench

    leaf = (np.zeros(10, np.int32), np.zeros(10, np.int32), np.zeros(5, np.int32), np.zeros(4, np.int32))
    got = bench.algorithmic_bytes([leaf, leaf], n_out=7, r_out=4)
    want = 2 * (8 * 10 + 4 * 5 + 4 * 4) + 8 * 7 + 4 * 5 + 4 * 4
    assert got == want


def test_vtr_and_pvd_writers(tmp_path):
    """Rectilinear grids and collections are host files: their structure is checked without a GPU."""
    import xml.etree.ElementTree as ET

    from subsetix_b200.subsetix_cupy import export_vtk as vtk

    u = np.arange(12, dtype=np.float32).reshape(3, 4)
    vtk.write_rectilinear_grid_vtr(str(tmp_path / "a.vtr"), u, 0.5, 0.25, cell_arrays={"flag": u > 5})
    root = ET.parse(tmp_path / "a.vtr").getroot()
    arrays = {a.get("Name"): a for a in root.iter("DataArray")}
    assert [float(x) for x in arrays["u"].text.split()] == u.ravel().tolist()
    assert [int(x) for x in arrays["flag"].text.split()] == (u.ravel() > 5).astype(int).tolist()
    assert [float(x) for x in arrays["X_COORDINATES"].text.split()] == [0.0, 0.5, 1.0, 1.5, 2.0]
    names, entry = vtk.save_amr3_step_vtr(str(tmp_path), "s", 3, 0.5, u0=u, u1=u, u2=u, refine0=u > 6,
                                          L1_mask=u > 2, refine1_mid=u > 8, L2_mask=u > 9, dx0=1, dy0=1, dx1=0.5,
                                          dy1=0.5, dx2=0.25, dy2=0.25)
    assert names == ["s_step0003_L0.vtr", "s_step0003_L1.vtr", "s_step0003_L2.vtr"] and entry == (0.5, names)
    vtk.write_pvd(str(tmp_path / "c.pvd"), [entry])
    sets = list(ET.parse(tmp_path / "c.pvd").getroot().iter("DataSet"))
    assert [(d.get("part"), d.get("file")) for d in sets] == [("0", names[0]), ("1", names[1]), ("2", names[2])]
    q = vtk.mask_quads(u > 9, u, 2, 0.25, 0.25)
    assert q.cells == 2 and q.points.shape == (8, 3) and q.values.tolist() == [10.0, 11.0]
