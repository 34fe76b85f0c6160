"""CPU tests: the C restatement of the oracle (oracle/hisq_oracle.c) against the golden fixtures that the reference
library itself produced (tests/golden/make_golden.py).  These pin the oracle even where the reference cannot be
built: bit-exact for the operators, same iteration count and solutions to 1e-11 for the multishift CG."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

G = np.load(Path(__file__).resolve().parent / "golden" / "golden.npz")
EPS, LINK_SEED = 0.3, 7


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def lat(name):
    return tuple(int(v) for v in name.split("x"))


@pytest.mark.parametrize("name", ["8x8x8x8", "6x4x2x8", "4x4x4x1", "2x3x5x4"])
@pytest.mark.parametrize("p", [0, 1])
def test_port_dslash_matches_golden(name, p):
    dims = lat(name)
    fat, lng = O.make_links(dims, EPS, LINK_SEED)
    src = O.make_source(dims, 1 - p, 11)
    assert sha(fat, lng, src) == str(G[f"dslash_{name}_p{p}_sha"]), "input generator changed"
    assert np.array_equal(O.dslash(dims, fat, lng, src, p), G[f"dslash_{name}_p{p}"])


def test_port_dslash_f32_matches_golden():
    dims = (6, 4, 2, 8)
    fat, lng = O.make_links(dims, EPS, LINK_SEED)
    f32 = (fat.astype(np.float32), lng.astype(np.float32), O.make_source(dims, 1, 11).astype(np.float32))
    assert sha(*f32) == str(G["dslash_f32_6x4x2x8_sha"])
    assert np.array_equal(O.dslash(dims, *f32, 0), G["dslash_f32_6x4x2x8"])


@pytest.mark.parametrize("name", ["4x4x4x8", "6x2x4x2"])
def test_port_full_lattice_dslash_matches_golden(name):
    dims = lat(name)
    fat, lng = O.make_links(dims, EPS, LINK_SEED)
    src = np.concatenate([O.make_source(dims, 0, 12), O.make_source(dims, 1, 13)])
    assert sha(fat, lng, src) == str(G[f"full_{name}_sha"])
    assert np.array_equal(O.dslash_full(dims, fat, lng, src), G[f"full_{name}"])


def test_port_mdaggm_matches_golden():
    dims = (4, 4, 4, 4)
    fat, lng = O.make_links(dims, EPS, LINK_SEED)
    src = O.make_source(dims, 0, 14)
    assert sha(fat, lng, src) == str(G["mdaggm_4x4x4x4_sha"])
    assert np.array_equal(O.mdagm(dims, fat, lng, src, 0), G["mdaggm_4x4x4x4"])


def test_port_cgm_matches_golden():
    dims = (4, 4, 4, 4)
    fat, lng = O.make_links(dims, EPS, 21)
    b = O.make_source(dims, 0, 5)
    assert sha(fat, lng, b) == str(G["cgm_4x4x4x4_sha"])
    refsh = list(G["cgm_4x4x4x4_shifts"])
    xs, it = O.cgm(dims, fat, lng, 0, refsh, b, float(G["cgm_4x4x4x4_tol"]), 5000)
    assert it == int(G["cgm_4x4x4x4_iter"])
    gx = G["cgm_4x4x4x4_x"]
    for k in range(len(refsh)):
        # the reference reduces with OpenMP; the restatement sums in order: equal to rounding
        assert np.abs(xs[k] - gx[k]).max() <= 1e-11 * np.abs(gx[k]).max()


def test_port_kat_matches_golden():
    dims = (4, 4, 4, 1)
    V = int(np.prod(dims))
    one = np.ones(V * 72, np.float32)
    xs, it = O.cgm(dims, one, one, 1, [3.671676313381e-05], np.ones(V // 2 * 6, np.float32), 1e-4, 6500)
    assert it == int(G["kat_test_solver_iter"]) == 1
    assert np.allclose(xs[0], G["kat_test_solver_x"], rtol=1e-6)
    assert abs(float(G["kat_test_solver_x"].mean()) - 0.007561) < 1e-4  # test_solver.cpp's expected value
