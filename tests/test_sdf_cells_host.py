"""SDF cell tables on the host: the library's own table builder
(myrt_b200/csrc/sdf_skip.hpp) compiled with g++ next to a host restatement of
the device evaluator's float arithmetic (tests/sdf_cells_check.cpp). For left
folds, balanced trees, right folds with unions, clusters of coincident
spheres (where smooth unions lower the value the most) and mixed primitives,
every march point evaluates bit for bit the same as the device runs it (cell
segments and the per-point bounding-sphere test) as in full, every march (with
the escape sphere's early exit) returns the same hit and t, and every material
load returns the same distance, material and random state, also when a
left-out operator draws exactly 1 and the load falls back to the full
program. Programs outside the supported shape get no grid."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from myrt_b200 import sdf as S

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("sdfcells") / "sdf_cells_check"
    subprocess.run([gxx, "-O2", "-std=c++20", "-pthread", "-ffp-contract=off", "-I", "/usr/local/cuda/include",
                    "-o", str(exe), str(ROOT / "tests" / "sdf_cells_check.cpp")], check=True)
    return exe


def _programs():
    """(name, node, expect_grid) in library order."""
    out = []
    out.append(("chain256", S.random_sdf_field(256, k=0.1, seed=9, extent=0.8, chain=True), True))
    out.append(("tree128", S.random_sdf_field(128, k=0.1, seed=5, extent=0.8, chain=False), True))
    rng = np.random.default_rng(4)
    nodes = [S.translate(S.sphere(float(rng.uniform(0.03, 0.15))), rng.uniform(-0.7, 0.7, 3)) for _ in range(20)]
    acc = nodes[-1]
    for i, nd in enumerate(reversed(nodes[:-1])):
        acc = S.smooth_union(nd, acc, 0.08) if i % 4 else S.union(nd, acc)
    out.append(("right_fold", acc, True))
    for shape in ("chain", "tree"):
        cl = []
        centres = rng.uniform(-0.5, 0.5, (4, 3))
        for i in range(32):
            cl.append(S.translate(S.sphere(0.1 + float(rng.uniform(-1e-4, 1e-4))),
                                  centres[i % 4] + rng.uniform(-1e-3, 1e-3, 3)))
        if shape == "chain":
            acc = cl[0]
            for nd in cl[1:]:
                acc = S.smooth_union(acc, nd, 0.2)
        else:
            while len(cl) > 1:
                cl = [S.smooth_union(cl[i], cl[i + 1], 0.2) for i in range(0, len(cl), 2)]
            acc = cl[0]
        out.append((f"cluster_{shape}", acc, True))
    mixed = []
    for i in range(40):
        kind = i % 4
        if kind == 0:
            p = S.sphere(float(rng.uniform(0.03, 0.12)))
        elif kind == 1:
            p = S.box(tuple(rng.uniform(0.02, 0.1, 3)))
        elif kind == 2:
            p = S.torus(float(rng.uniform(0.05, 0.12)), float(rng.uniform(0.01, 0.04)))
        else:
            p = S.vertical_capsule(float(rng.uniform(0.0, 0.2)), float(rng.uniform(0.02, 0.05)))
        mixed.append(S.translate(p, rng.uniform(-0.8, 0.8, 3)))
    acc = mixed[0]
    for i, nd in enumerate(mixed[1:]):
        acc = S.union(acc, nd) if i % 3 == 0 else S.smooth_union(acc, nd, 0.1)
    out.append(("mixed", acc, True))
    # a subtraction makes the program unsupported: evaluated in full both ways
    sub = S.subtraction(S.translate(S.sphere(0.2), (0.1, 0.0, 0.0)), acc)
    out.append(("subtraction", sub, False))
    return out


@pytest.mark.parametrize("cells", [8, 32])
def test_cell_segments_and_early_exit_are_exact(checker, tmp_path, cells):
    progs = _programs()
    lib = S.SdfLibrary()
    for _, node, _ in progs:
        lib.add(node)
    np.asarray(lib.instrs, np.int32).tofile(tmp_path / "instrs.bin")
    np.asarray(lib.programs, np.int32).tofile(tmp_path / "programs.bin")
    np.asarray(lib.params, np.float32).tofile(tmp_path / "params.bin")
    res = subprocess.run([str(checker), str(tmp_path), str(cells), "600", "3"], check=True, capture_output=True,
                         text=True).stdout.split("\n")
    rows = [list(map(float, r.split())) for r in res if r.strip()]
    assert len(rows) == len(progs)
    for (name, _, expect_grid), r in zip(progs, rows):
        _, grid, points, bad_points, hits, bad_marches, full_i, cell_i, loads, bad_loads, bad_forced, redos = r
        assert bad_points == 0 and bad_marches == 0, name
        # material loads: distance, material and final random state; a draw of
        # exactly 1 planted at each of the first 64 positions makes some calls
        # fall back to the full evaluation
        assert loads >= 100 and bad_loads == 0 and bad_forced == 0, name
        assert redos > 0, name
        assert points > 3_000 and hits > 20, name
        assert (grid > 0) == expect_grid, name
        if expect_grid:
            assert cell_i < 0.5 * full_i, (name, cell_i, full_i)
        else:  # no grid: only the per-point bounding-sphere test of the inner groups
            assert cell_i <= full_i, name
