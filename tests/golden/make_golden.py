"""Generate golden fixtures by running the reference package itself.

This script runs only in the build container, where the reference sources
are mounted.  It puts ``oracle/refshim`` (a NumPy-backed stand-in for
``cupy``) and the reference checkout at the front of ``sys.path``.  It then
imports the reference's own ``subsetix_cupy`` and ``subsetix_amr2`` modules
and records their outputs on seeded inputs.  The reference's CUDA-C kernel
strings run on the host through ``oracle/refshim/cpu_rawkernel.py``.

Integer and interval outputs are exactly what the reference computes.  Float
outputs come from the reference's own formulas, compiled without FMA
contraction.  The FP32 tolerances in the tests allow for that.

Usage::

    python tests/golden/make_golden.py [--reference /path/to/reference]

Outputs are written next to this script as ``*.npz`` files.  The fixtures
are committed; the GPU tests and the oracle tests read only those files.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _setup(reference: str):
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    sys.path.insert(0, os.path.join(REPO, "oracle", "refshim"))
    sys.path.insert(0, REPO)


class Recorder:
    def __init__(self):
        self.data = {}

    def put_set(self, key, s):
        self.data[f"{key}/begin"] = np.asarray(s.begin, dtype=np.int32).view(np.ndarray).copy()
        self.data[f"{key}/end"] = np.asarray(s.end, dtype=np.int32).view(np.ndarray).copy()
        self.data[f"{key}/row_offsets"] = np.asarray(s.row_offsets, dtype=np.int32).view(np.ndarray).copy()
        self.data[f"{key}/rows"] = np.asarray(s.rows, dtype=np.int32).view(np.ndarray).copy()

    def put_error(self, key, exc):
        self.data[f"{key}/error"] = np.array(type(exc).__name__)

    def put(self, key, arr):
        self.data[key] = np.asarray(arr).view(np.ndarray).copy()

    def save(self, name):
        path = os.path.join(HERE, name)
        np.savez_compressed(path, **self.data)
        print(f"wrote {path}: {len(self.data)} arrays, {os.path.getsize(path)} bytes")


def random_small_set(rng, *, row_lo=-4, row_hi=14, max_rows=10, max_per_row=5,
                     touching=False, empties=False, dense_rows=None, min_per_row=0):
    """Small random set with sparse rows, used for the exhaustive-style cases."""
    if dense_rows is not None:
        rows = np.arange(dense_rows, dtype=np.int32)
    else:
        nrows = int(rng.integers(0, max_rows + 1))
        rows = np.sort(rng.choice(np.arange(row_lo, row_hi), size=min(nrows, row_hi - row_lo), replace=False)).astype(np.int32)
    begins, ends, offsets = [], [], [0]
    for _ in rows:
        k = int(rng.integers(min_per_row, max_per_row + 1))
        x = int(rng.integers(-12, 6))
        for _ in range(k):
            gap = int(rng.integers(0 if touching else 1, 5))
            if not begins or offsets[-1] == len(begins):
                gap = int(rng.integers(0, 5))
            length = int(rng.integers(0 if empties else 1, 6))
            x += gap
            begins.append(x)
            x += length
            ends.append(x)
        offsets.append(len(begins))
    return (np.asarray(begins, np.int32), np.asarray(ends, np.int32),
            np.asarray(offsets, np.int32), rows)


def domain_set(rng, width, height, max_per_row=4):
    """Dense-row set whose intervals lie inside ``[0, width)``."""
    begins, ends, offsets = [], [], [0]
    for _ in range(height):
        k = int(rng.integers(0, max_per_row + 1))
        pts = np.sort(rng.choice(width + 1, size=min(2 * k, width + 1), replace=False))
        for i in range(0, len(pts) - 1, 2):
            begins.append(int(pts[i]))
            ends.append(int(pts[i + 1]))
        offsets.append(len(begins))
    return (np.asarray(begins, np.int32), np.asarray(ends, np.int32),
            np.asarray(offsets, np.int32), np.arange(height, dtype=np.int32))


FILES = ("setops", "morph", "multilevel", "stencil_regrid", "amr", "levels", "amr_large")


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default="/root/reference")
    parser.add_argument("--only", nargs="*", choices=FILES, default=list(FILES),
                        help="write only these fixture files (each file's inputs come from its own seeds)")
    args = parser.parse_args()
    _setup(args.reference)
    only = set(args.only)

    import cupy as cp  # the NumPy-backed stand-in
    import subsetix_cupy as sc
    from subsetix_cupy import expressions as sx_expr
    from subsetix_cupy import morphology as sx_morph
    from subsetix_cupy import multilevel as sx_ml
    from subsetix_cupy.interval_field import create_interval_field, IntervalField
    from subsetix_cupy.interval_stencil import step_upwind_interval
    from subsetix_amr2 import regrid as sx_regrid
    from subsetix_amr2 import fields as sx_fields
    from subsetix_amr2.geometry import TwoLevelGeometry
    from subsetix_amr2.simulation import AMR2Simulation, SimulationConfig, SquareSpec
    from subsetix_amr2.runner import SimulationArgs, run_two_level_simulation
    from subsetix_b200 import synth

    def mk(host):
        b, e, off, rows = host
        return sx_expr.IntervalSet(begin=cp.asarray(b, dtype=cp.int32), end=cp.asarray(e, dtype=cp.int32),
                                   row_offsets=cp.asarray(off, dtype=cp.int32), rows=cp.asarray(rows, dtype=cp.int32))

    def put_host(rec, key, host):
        rec.put(f"{key}/begin", host[0]); rec.put(f"{key}/end", host[1])
        rec.put(f"{key}/row_offsets", host[2]); rec.put(f"{key}/rows", host[3])

    binops = {
        "union": sc.make_union,
        "intersection": sc.make_intersection,
        "difference": sc.make_difference,
        "symmetric_difference": sc.make_symmetric_difference,
        "complement": sc.make_complement,
    }

    # ---------------------------------------------------------------- set ops
    rec = Recorder()
    a_host = synth.random_rows_set(0)
    b_host = synth.random_rows_set(1)
    put_host(rec, "rows256/A", a_host)
    put_host(rec, "rows256/B", b_host)
    A, B = mk(a_host), mk(b_host)
    for name, fn in binops.items():
        rec.put_set(f"rows256/{name}", sc.evaluate(fn(sc.make_input(A), sc.make_input(B))))
    rec.put_set("rows256/dilate11", sx_morph.dilate_interval_set(A, halo_x=1, halo_y=1))

    rng = np.random.default_rng(1234)
    kinds = ["canonical", "touching", "empties"]
    case = 0
    for kind in kinds:
        for _ in range(40):
            opts = dict(touching=kind != "canonical", empties=kind == "empties")
            lh = random_small_set(rng, **opts)
            rh = random_small_set(rng, **opts)
            L, R = mk(lh), mk(rh)
            put_host(rec, f"bin{case}/A", lh)
            put_host(rec, f"bin{case}/B", rh)
            rec.put(f"bin{case}/kind", np.array(kinds.index(kind)))
            for name, fn in binops.items():
                rec.put_set(f"bin{case}/{name}", sc.evaluate(fn(sc.make_input(L), sc.make_input(R))))
            case += 1
    rec.put("bin_count", np.array(case))

    # nested expressions over five operands: ((A|B)-(C&D))^E and two others
    exprs = {
        "e0": ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")), "E"),
        "e1": ("union", ("intersection", ("difference", "D", "A"), "B"), ("symmetric_difference", "C", "E")),
        "e2": ("complement", ("union", "D", "E"), ("intersection", "A", "B")),
        "e3": ("intersection", ("union", "A", ("intersection", "B", "C")), ("difference", "E", "D")),
    }

    def build(spec, leaves):
        if isinstance(spec, str):
            return sc.make_input(leaves[spec])
        return binops[spec[0]](build(spec[1], leaves), build(spec[2], leaves))

    ecase = 0
    for kind in kinds:
        for _ in range(12):
            opts = dict(touching=kind != "canonical", empties=kind == "empties")
            leaves_host = {name: random_small_set(rng, **opts) for name in "ABCDE"}
            leaves = {k: mk(v) for k, v in leaves_host.items()}
            for name, host in leaves_host.items():
                put_host(rec, f"expr{ecase}/{name}", host)
            rec.put(f"expr{ecase}/kind", np.array(kinds.index(kind)))
            for ename, spec in exprs.items():
                rec.put_set(f"expr{ecase}/{ename}", sc.evaluate(build(spec, leaves)))
            ecase += 1
    rec.put("expr_count", np.array(ecase))

    # the shape workload at 512x512 (same generators, scaled) for the fused expression
    shapes = synth.shape_operands(512)
    for name, host in zip("ABCDE", shapes):
        put_host(rec, f"shape512/{name}", host)
    leaves = {name: mk(h) for name, h in zip("ABCDE", shapes)}
    rec.put_set("shape512/e0", sc.evaluate(build(exprs["e0"], leaves)))
    if "setops" in only:
        rec.save("setops.npz")

    # ------------------------------------------------------------- morphology
    rec = Recorder()
    mcase = 0
    for kind in kinds:
        for _ in range(20):
            opts = dict(touching=kind != "canonical", empties=kind == "empties")
            sh = random_small_set(rng, **opts)
            S = mk(sh)
            put_host(rec, f"m{mcase}/S", sh)
            rec.put(f"m{mcase}/kind", np.array(kinds.index(kind)))
            for hx, hy in [(0, 0), (2, 0), (0, 1), (1, 1), (3, 2), (1, 4)]:
                rec.put_set(f"m{mcase}/dilate_{hx}_{hy}", sx_morph.dilate_interval_set(S, halo_x=hx, halo_y=hy))
            for w, h in [(8, 6), (16, 12), (1, 3)]:
                rec.put_set(f"m{mcase}/clip_{w}_{h}", sx_morph.clip_interval_set(S, width=w, height=h))
                rec.put_set(f"m{mcase}/erode_{w}_{h}", sx_morph.erode_interval_set(S, halo_x=1, halo_y=1, width=w, height=h))
                rec.put_set(f"m{mcase}/ghost_{w}_{h}", sx_morph.ghost_zones(S, halo_x=1, halo_y=1, width=w, height=h))
            mcase += 1
    rec.put("morph_count", np.array(mcase))
    # morphology of the 256 x 256 random-rows set
    for hx, hy in [(1, 1), (2, 2), (4, 4), (3, 0)]:
        rec.put_set(f"rows256/dilate_{hx}_{hy}", sx_morph.dilate_interval_set(A, halo_x=hx, halo_y=hy))
        rec.put_set(f"rows256/erode_{hx}_{hy}", sx_morph.erode_interval_set(A, halo_x=hx, halo_y=hy, width=256, height=256))
    put_host(rec, "rows256/A", a_host)
    if "morph" in only:
        rec.save("morph.npz")

    # ------------------------------------------------------------- multilevel
    rec = Recorder()
    pcase = 0
    for kind in kinds:
        for _ in range(20):
            opts = dict(touching=kind != "canonical", empties=kind == "empties")
            sh = random_small_set(rng, **opts)
            S = mk(sh)
            put_host(rec, f"p{pcase}/S", sh)
            rec.put(f"p{pcase}/kind", np.array(kinds.index(kind)))
            for r in (1, 2, 3, 4):
                rec.put_set(f"p{pcase}/prolong_{r}", sx_ml.prolong_set(S, r))
                rec.put_set(f"p{pcase}/restrict_{r}", sx_ml.restrict_set(S, r))
            pcase += 1
    rec.put("ml_count", np.array(pcase))
    # fields on canonical coarse sets: prolong then perturb then restrict
    fcase = 0
    for i in range(20):
        # rows with no intervals make the reference's fine-row alignment raise
        sh = random_small_set(rng, min_per_row=0 if i % 4 == 3 else 1)
        S = mk(sh)
        field = create_interval_field(S, fill_value=0.0, dtype=cp.float32)
        field.values[...] = cp.asarray(rng.standard_normal(int(field.values.size)).astype(np.float32))
        put_host(rec, f"f{fcase}/S", sh)
        rec.put(f"f{fcase}/values", field.values)
        for r in (2, 3):
            try:
                fine = sx_ml.prolong_field(field, r)
            except Exception as exc:  # the reference's own error path
                rec.put_error(f"f{fcase}/fine_{r}", exc)
                continue
            rec.put_set(f"f{fcase}/fine_{r}", fine.interval_set)
            rec.put(f"f{fcase}/fine_{r}/values", fine.values)
            noisy = IntervalField(interval_set=fine.interval_set,
                                  values=cp.asarray(rng.standard_normal(int(fine.values.size)).astype(np.float32)),
                                  interval_cell_offsets=fine.interval_cell_offsets)
            rec.put(f"f{fcase}/noisy_{r}", noisy.values)
            for red in ("mean", "sum", "min", "max"):
                try:
                    out = sx_ml.restrict_field(noisy, r, reducer=red)
                except Exception as exc:
                    rec.put_error(f"f{fcase}/restrict_{r}_{red}", exc)
                    continue
                rec.put_set(f"f{fcase}/restrict_{r}_{red}", out.interval_set)
                rec.put(f"f{fcase}/restrict_{r}_{red}/values", out.values)
        fcase += 1
    rec.put("field_count", np.array(fcase))
    if "multilevel" in only:
        rec.save("multilevel.npz")

    # ----------------------------------------------------- stencil and regrid
    rec = Recorder()
    ucase = 0
    for width, height in [(16, 16), (24, 20), (64, 64)]:
        for signs in [(1.0, 0.5), (-0.7, 0.3), (0.4, -0.9), (-1.0, -1.0), (0.0, 0.0)]:
            sh = domain_set(rng, width, height)
            S = mk(sh)
            field = create_interval_field(S, fill_value=0.0, dtype=cp.float32)
            field.values[...] = cp.asarray(rng.uniform(0.0, 1.0, int(field.values.size)).astype(np.float32))
            a_vel, b_vel = signs
            dx, dy = 1.0 / width, 1.0 / height
            dt = 0.25 * dx
            out = step_upwind_interval(field, width=width, height=height, a=a_vel, b=b_vel, dt=dt, dx=dx, dy=dy)
            put_host(rec, f"u{ucase}/S", sh)
            rec.put(f"u{ucase}/values", field.values)
            rec.put(f"u{ucase}/params", np.array([width, height, a_vel, b_vel, dt, dx, dy], dtype=np.float64))
            rec.put(f"u{ucase}/out", out)
            ucase += 1
    rec.put("upwind_count", np.array(ucase))

    gcase = 0
    for width, height in [(8, 8), (33, 17), (64, 48)]:
        for thr in (0.05, 0.2, 0.5):
            data = rng.uniform(0, 1, size=(height, width)).astype(np.float32)
            data = np.where(rng.uniform(size=(height, width)) < 0.6, 0.0, data).astype(np.float32)
            full = sx_morph.full_interval_set(width, height)
            field = create_interval_field(full, fill_value=0.0, dtype=cp.float32)
            field.values[...] = cp.asarray(data.ravel())
            grad = sx_regrid.gradient_magnitude_interval_field(field, width=width, height=height)
            tags = sx_regrid.gradient_tag_threshold_interval_field(field, width=width, height=height, threshold=thr)
            tset = sx_regrid.gradient_tag_threshold_set(field, width=width, height=height, threshold=thr)
            rec.put(f"g{gcase}/data", data)
            rec.put(f"g{gcase}/params", np.array([width, height, thr], dtype=np.float64))
            rec.put(f"g{gcase}/grad", grad.values)
            rec.put_set(f"g{gcase}/tags", tags)
            rec.put_set(f"g{gcase}/tset", tset)
            for pad, mode in [(1, "von_neumann"), (1, "moore"), (2, "von_neumann"), (0, "moore")]:
                rec.put_set(f"g{gcase}/grade_{pad}_{mode}", sx_regrid.enforce_two_level_grading_set(
                    tags, padding=pad, mode=mode, width=width, height=height))
            gcase += 1
    rec.put("regrid_count", np.array(gcase))
    if "stencil_regrid" in only:
        rec.save("stencil_regrid.npz")

    # ---------------------------------------------------------- AMR drivers
    rec = Recorder()
    for tag, res, init, steps, every, vel in [
        ("sq32", 32, "square", 12, 4, (1.0, 0.5)),
        ("sq24", 24, "square", 9, 3, (-0.6, 0.8)),
        ("gauss32", 32, "gauss", 10, 5, (1.0, 0.5)),
    ]:
        config = SimulationConfig(coarse_resolution=res, velocity=vel, cfl=0.5, refine_threshold=0.05, grading=1)
        sim = AMR2Simulation(config)
        if init == "square":
            sim.initialize_square(squares=[SquareSpec(center=(0.35, 0.4), half_width=(0.15, 0.1))])
        else:
            full = sx_morph.full_interval_set(res, res)
            field = create_interval_field(full, fill_value=0.0, dtype=cp.float32)
            xs = (np.arange(res) + 0.5) / res
            gx, gy = np.meshgrid(xs, xs)
            u0 = np.exp(-((gx - 0.5) ** 2 + (gy - 0.5) ** 2) / (2 * 0.1 ** 2)).astype(np.float32)
            field.values[...] = cp.asarray(u0.ravel())
            sim.set_initial_field(field)
        state = sim.state
        rec.put(f"{tag}/coarse0", state.coarse_field.values)
        rec.put(f"{tag}/fine0", state.fine_field.values)
        rec.put_set(f"{tag}/refine0", state.actions.refine_set())
        rec.put(f"{tag}/params", np.array([res, steps, every, vel[0], vel[1], sim.dt], dtype=np.float64))
        state, stats = sim.run(steps=steps, regrid_every=every)
        rec.put(f"{tag}/coarse", state.coarse_field.values)
        rec.put(f"{tag}/fine", state.fine_field.values)
        rec.put_set(f"{tag}/refine", state.actions.refine_set())
        rec.put_set(f"{tag}/coarse_only", state.geometry.coarse_only)
        rec.put_set(f"{tag}/fine_set", state.geometry.fine)

    def init_fn(f):
        f.coarse_field.values.fill(1.0)
        f.fine_field.values.fill(1.0)

    field = run_two_level_simulation(SimulationArgs(velocity=(0.1, 0.0), cfl=0.5, t0=0.0, tf=0.01,
                                                    min_level=2, max_level=3, refine_threshold=0.05, grading=1), init_fn)
    rec.put("runner/coarse", field.coarse_field.values)
    rec.put("runner/fine", field.fine_field.values)
    if "amr" in only:
        rec.save("amr.npz")

    # ------------------------------------------- percentile tagging and level helpers
    if "levels" in only:
        lrng = np.random.default_rng(4321)
        rec = Recorder()
        tcase = 0
        for width, height in [(4, 4), (16, 12), (40, 33)]:
            for kind in ("golden", "uniform", "signed", "zeros"):
                if kind == "golden" and (width, height) != (4, 4):
                    continue
                data = np.zeros((height, width), np.float32)
                if kind == "golden":  # test_regrid.py:58-66
                    data[1, 1], data[2, 2] = 0.5, 1.0
                elif kind == "uniform":
                    data = lrng.uniform(0, 1, (height, width)).astype(np.float32)
                elif kind == "signed":
                    data = lrng.standard_normal((height, width)).astype(np.float32)
                full = sx_morph.full_interval_set(width, height)
                field = create_interval_field(full, fill_value=0.0, dtype=cp.float32)
                field.values[...] = cp.asarray(data.ravel())
                rec.put(f"t{tcase}/data", data)
                fracs = (0.0, 0.01, 0.2, 0.5, 1.0, 1.5)
                rec.put(f"t{tcase}/fracs", np.array(fracs))
                for j, frac in enumerate(fracs):
                    rec.put_set(f"t{tcase}/tag_{j}", sx_regrid.gradient_tag_set(field, width=width, height=height,
                                                                               frac_high=frac))
                tcase += 1
        rec.put("tag_count", np.array(tcase))
        # three-level hierarchies: prolong / restrict of sets and fields, covered cells, coarse-only sets
        hcase = 0
        for _ in range(8):
            base = random_small_set(lrng, row_lo=0, row_hi=12, max_rows=8, min_per_row=1)
            put_host(rec, f"h{hcase}/base", base)
            ml = sx_ml.MultiLevel2D.create(3, base_ratio=2)
            ml.set_level(0, mk(base))
            rec.put_set(f"h{hcase}/l1", sx_ml.prolong_level_sets(ml, 0))
            rec.put_set(f"h{hcase}/l2", sx_ml.prolong_level_sets(ml, 1))
            rec.put_set(f"h{hcase}/covered0", sx_ml.covered_by_fine(ml, 0))
            rec.put_set(f"h{hcase}/coarse_only0", sx_ml.coarse_only(ml.get_level(0), ml, 0))
            rec.put_set(f"h{hcase}/restricted1", sx_ml.restrict_level_sets(ml, 1))
            mf = sx_ml.MultiLevelField2D.create_from_geometry(ml, fill_value=0.0, dtype=cp.float32)
            f0 = mf.get_level_field(0)
            f0.values[...] = cp.asarray(lrng.standard_normal(int(f0.values.size)).astype(np.float32))
            rec.put(f"h{hcase}/f0", f0.values)
            try:
                rec.put(f"h{hcase}/pf1", sx_ml.prolong_level_field(ml, mf, 0).values)
                rec.put(f"h{hcase}/pf2", sx_ml.prolong_level_field(ml, mf, 1).values)
                f2 = mf.get_level_field(2)
                f2.values[...] = cp.asarray(lrng.standard_normal(int(f2.values.size)).astype(np.float32))
                rec.put(f"h{hcase}/f2", f2.values)
                for red in ("mean", "max"):
                    rec.put(f"h{hcase}/rf1_{red}", sx_ml.restrict_level_field(ml, mf, 1, reducer=red).values)
            except Exception as exc:
                rec.put_error(f"h{hcase}/fields", exc)
            hcase += 1
        rec.put("hier_count", np.array(hcase))
        rec.save("levels.npz")

    # --------------------------------- two-level AMR at a stated size, physical threshold
    if "amr_large" in only:
        rec = Recorder()
        res, steps, every = 128, 40, 10
        thr = 0.05 / res  # the physical gradient threshold 0.05 on the reference's per-cell difference
        config = SimulationConfig(coarse_resolution=res, velocity=(1.0, 0.5), cfl=0.5, refine_threshold=thr,
                                  grading=1)
        sim = AMR2Simulation(config)
        full = sx_morph.full_interval_set(res, res)
        field = create_interval_field(full, fill_value=0.0, dtype=cp.float32)
        xs = (np.arange(res) + 0.5) / res
        gx, gy = np.meshgrid(xs, xs)
        u0 = np.exp(-((gx - 0.5) ** 2 + (gy - 0.5) ** 2) / (2 * 0.05 ** 2)).astype(np.float32)
        field.values[...] = cp.asarray(u0.ravel())
        sim.set_initial_field(field)
        rec.put("g128/u0", u0)
        rec.put("g128/params", np.array([res, steps, every, 1.0, 0.5, sim.dt, thr], dtype=np.float64))
        rec.put_set("g128/refine0", sim.state.actions.refine_set())
        state, _ = sim.run(steps=steps, regrid_every=every)
        rec.put("g128/coarse", state.coarse_field.values)
        rec.put("g128/fine", state.fine_field.values)
        rec.put_set("g128/refine", state.actions.refine_set())
        rec.put_set("g128/coarse_only", state.geometry.coarse_only)
        rec.save("amr_large.npz")


if __name__ == "__main__":
    main()
