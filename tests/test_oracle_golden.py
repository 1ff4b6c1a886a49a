"""The oracle against outputs of the reference package itself.

The fixtures come from ``tests/golden/make_golden.py``, which runs the
reference's own Python and kernel code.  Every interval output must match
exactly.  FP32 field outputs must match to within 2 ulp (see
``FP32_ULP``): the fixtures evaluate the reference formulas without FMA
contraction, and so does the oracle.
"""

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden_io import load, get_set, error

FP32_ULP = 2


def iset(host):
    return O.ISet(*[np.asarray(a, dtype=np.int32) for a in host])


def assert_set_equal(actual, expected, msg=""):
    for name, a, e in zip(("begin", "end", "row_offsets", "rows"), actual, expected):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(e), err_msg=f"{msg} {name}")


def ulp_diff32(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


BIN = ["union", "intersection", "difference", "symmetric_difference", "complement"]


def test_random_rows_256_setops():
    g = load("setops.npz")
    A, B = iset(get_set(g, "rows256/A")), iset(get_set(g, "rows256/B"))
    for op in BIN:
        assert_set_equal(O.BINARY[op](A, B), get_set(g, f"rows256/{op}"), op)
    assert_set_equal(O.dilate(A, 1, 1), get_set(g, "rows256/dilate11"), "dilate")


def test_random_binary_cases():
    g = load("setops.npz")
    for c in range(int(g["bin_count"])):
        A, B = iset(get_set(g, f"bin{c}/A")), iset(get_set(g, f"bin{c}/B"))
        for op in BIN:
            assert_set_equal(O.BINARY[op](A, B), get_set(g, f"bin{c}/{op}"), f"case {c} {op}")


EXPRS = {
    "e0": ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")), "E"),
    "e1": ("union", ("intersection", ("difference", "D", "A"), "B"), ("symmetric_difference", "C", "E")),
    "e2": ("complement", ("union", "D", "E"), ("intersection", "A", "B")),
    "e3": ("intersection", ("union", "A", ("intersection", "B", "C")), ("difference", "E", "D")),
}


def test_expression_cases():
    g = load("setops.npz")
    for c in range(int(g["expr_count"])):
        leaves = {n: iset(get_set(g, f"expr{c}/{n}")) for n in "ABCDE"}
        for name, spec in EXPRS.items():
            assert_set_equal(O.evaluate(spec, leaves), get_set(g, f"expr{c}/{name}"), f"expr {c} {name}")
    leaves = {n: iset(get_set(g, f"shape512/{n}")) for n in "ABCDE"}
    assert_set_equal(O.evaluate(EXPRS["e0"], leaves), get_set(g, "shape512/e0"), "shape512")


def test_morphology_cases():
    g = load("morph.npz")
    for c in range(int(g["morph_count"])):
        S = iset(get_set(g, f"m{c}/S"))
        for hx, hy in [(0, 0), (2, 0), (0, 1), (1, 1), (3, 2), (1, 4)]:
            assert_set_equal(O.dilate(S, hx, hy), get_set(g, f"m{c}/dilate_{hx}_{hy}"), f"m{c} dilate {hx} {hy}")
        for w, h in [(8, 6), (16, 12), (1, 3)]:
            assert_set_equal(O.clip(S, w, h), get_set(g, f"m{c}/clip_{w}_{h}"), f"m{c} clip")
            assert_set_equal(O.erode(S, 1, 1, width=w, height=h), get_set(g, f"m{c}/erode_{w}_{h}"), f"m{c} erode")
            assert_set_equal(O.ghost_zones(S, 1, 1, width=w, height=h), get_set(g, f"m{c}/ghost_{w}_{h}"), f"m{c} ghost")
    A = iset(get_set(g, "rows256/A"))
    for hx, hy in [(1, 1), (2, 2), (4, 4), (3, 0)]:
        assert_set_equal(O.dilate(A, hx, hy), get_set(g, f"rows256/dilate_{hx}_{hy}"))
        assert_set_equal(O.erode(A, hx, hy, width=256, height=256), get_set(g, f"rows256/erode_{hx}_{hy}"))


def test_multilevel_sets():
    g = load("multilevel.npz")
    for c in range(int(g["ml_count"])):
        S = iset(get_set(g, f"p{c}/S"))
        for r in (1, 2, 3, 4):
            assert_set_equal(O.prolong_set(S, r), get_set(g, f"p{c}/prolong_{r}"), f"p{c} prolong {r}")
            assert_set_equal(O.restrict_set(S, r), get_set(g, f"p{c}/restrict_{r}"), f"p{c} restrict {r}")


def test_multilevel_fields():
    g = load("multilevel.npz")
    for c in range(int(g["field_count"])):
        S = iset(get_set(g, f"f{c}/S"))
        f = O.Field(S, g[f"f{c}/values"], O.cell_offsets(S))
        for r in (2, 3):
            err = error(g, f"f{c}/fine_{r}")
            if err:
                with pytest.raises(ValueError):
                    O.prolong_field(f, r)
                continue
            fine = O.prolong_field(f, r)
            assert_set_equal(fine.iset, get_set(g, f"f{c}/fine_{r}"))
            np.testing.assert_array_equal(fine.values, g[f"f{c}/fine_{r}/values"])
            noisy = O.Field(fine.iset, g[f"f{c}/noisy_{r}"], fine.offsets)
            for red in ("mean", "sum", "min", "max"):
                out = O.restrict_field(noisy, r, red)
                assert_set_equal(out.iset, get_set(g, f"f{c}/restrict_{r}_{red}"))
                assert ulp_diff32(out.values, g[f"f{c}/restrict_{r}_{red}/values"]).max(initial=0) <= FP32_ULP


def test_upwind_cases():
    g = load("stencil_regrid.npz")
    for c in range(int(g["upwind_count"])):
        S = iset(get_set(g, f"u{c}/S"))
        w, h, a, b, dt, dx, dy = g[f"u{c}/params"].tolist()
        f = O.Field(S, g[f"u{c}/values"], O.cell_offsets(S))
        out = O.upwind(f, width=int(w), height=int(h), a=a, b=b, dt=dt, dx=dx, dy=dy)
        assert ulp_diff32(out, g[f"u{c}/out"]).max(initial=0) <= FP32_ULP, c


def test_regrid_cases():
    g = load("stencil_regrid.npz")
    for c in range(int(g["regrid_count"])):
        w, h, thr = g[f"g{c}/params"].tolist()
        w, h = int(w), int(h)
        data = g[f"g{c}/data"]
        grad = O.gradient_magnitude(data.ravel(), w, h)
        assert ulp_diff32(grad, g[f"g{c}/grad"]).max(initial=0) <= FP32_ULP
        tags = O.gradient_tag_threshold(data.ravel(), w, h, thr)
        assert_set_equal(tags, get_set(g, f"g{c}/tags"), f"g{c} tags")
        assert_set_equal(O.threshold_intervals(data.ravel(), w, h, max(thr, 1e-8)), get_set(g, f"g{c}/tset"))
        for pad, mode in [(1, "von_neumann"), (1, "moore"), (2, "von_neumann"), (0, "moore")]:
            assert_set_equal(O.grading(tags, pad, mode, width=w, height=h),
                             get_set(g, f"g{c}/grade_{pad}_{mode}"), f"g{c} grade {pad} {mode}")


@pytest.mark.parametrize("tag", ["sq32", "sq24", "gauss32"])
def test_amr_simulation(tag):
    g = load("amr.npz")
    res, steps, every, va, vb, dt = g[f"{tag}/params"].tolist()
    sim = O.AMR2(int(res), (va, vb), cfl=0.5, threshold=0.05, grading_pad=1)
    assert abs(sim.dt - dt) < 1e-15
    sim.init(g[f"{tag}/coarse0"])
    assert_set_equal(sim.actions.refine, get_set(g, f"{tag}/refine0"))
    np.testing.assert_array_equal(sim.fine.values, g[f"{tag}/fine0"])
    sim.run(int(steps), int(every))
    assert_set_equal(sim.actions.refine, get_set(g, f"{tag}/refine"))
    assert_set_equal(sim.coarse_only, get_set(g, f"{tag}/coarse_only"))
    assert_set_equal(sim.actions.fine_set(), get_set(g, f"{tag}/fine_set"))
    assert ulp_diff32(sim.coarse.values, g[f"{tag}/coarse"]).max() <= 8
    assert ulp_diff32(sim.fine.values, g[f"{tag}/fine"]).max() <= 8


def test_percentile_tagging():
    g = load("levels.npz")
    for c in range(int(g["tag_count"])):
        data = g[f"t{c}/data"]
        h, w = data.shape
        for j, frac in enumerate(g[f"t{c}/fracs"].tolist()):
            assert_set_equal(O.gradient_tag_set(data.ravel(), w, h, frac), get_set(g, f"t{c}/tag_{j}"), f"t{c} {j}")


def test_level_helpers():
    g = load("levels.npz")
    for c in range(int(g["hier_count"])):
        l0 = iset(get_set(g, f"h{c}/base"))
        l1 = O.prolong_set(l0, 2)
        l2 = O.prolong_set(l1, 2)
        assert_set_equal(l1, get_set(g, f"h{c}/l1"))
        assert_set_equal(l2, get_set(g, f"h{c}/l2"))
        covered = O.restrict_set(l1, 2)
        assert_set_equal(covered, get_set(g, f"h{c}/covered0"))
        assert_set_equal(O.difference(l0, covered), get_set(g, f"h{c}/coarse_only0"))
        assert_set_equal(O.restrict_set(l2, 2), get_set(g, f"h{c}/restricted1"))
        if error(g, f"h{c}/fields"):
            continue
        f0 = O.Field(l0, g[f"h{c}/f0"], O.cell_offsets(l0))
        p1 = O.prolong_field(f0, 2)
        np.testing.assert_array_equal(p1.values, g[f"h{c}/pf1"])
        p2 = O.prolong_field(p1, 2)
        np.testing.assert_array_equal(p2.values, g[f"h{c}/pf2"])
        f2 = O.Field(p2.iset, g[f"h{c}/f2"], p2.offsets)
        for red in ("mean", "max"):
            assert ulp_diff32(O.restrict_field(f2, 2, red).values, g[f"h{c}/rf1_{red}"]).max(initial=0) <= FP32_ULP


def test_amr_simulation_128_physical_threshold():
    """The two-level AMR loop at 128^2 with the physical threshold 0.05 dx (12 % refined), 40 steps."""
    g = load("amr_large.npz")
    res, steps, every, va, vb, dt, thr = g["g128/params"].tolist()
    sim = O.AMR2(int(res), (va, vb), cfl=0.5, threshold=thr, grading_pad=1)
    assert abs(sim.dt - dt) < 1e-15
    sim.init(g["g128/u0"])
    assert_set_equal(sim.actions.refine, get_set(g, "g128/refine0"))
    sim.run(int(steps), int(every))
    assert_set_equal(sim.actions.refine, get_set(g, "g128/refine"))
    assert_set_equal(sim.coarse_only, get_set(g, "g128/coarse_only"))
    assert ulp_diff32(sim.coarse.values, g["g128/coarse"]).max() <= 8
    assert ulp_diff32(sim.fine.values, g["g128/fine"]).max() <= 8
