"""Synthetic input generators (seeded, no dataset)."""
import numpy as np

from hmfem_b200.problem import (config_problem, gaussian_field, make_problem,
                                random_walk_conduit)


def test_conduit_walk_properties():
    rng = np.random.default_rng(1)
    nx, ny, nz = 20, 9, 7
    for _ in range(20):
        c = random_walk_conduit(rng, nx, ny, nz)
        i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
        assert i.min() == 0 and i.max() == nx - 1
        assert j.min() >= 0 and j.max() < ny and k.min() >= 0 and k.max() < nz
        # every x-slab is visited (the walk only moves +x, never -x)
        assert set(i.tolist()) == set(range(nx))


def test_gaussian_field_moments():
    g = gaussian_field(np.random.default_rng(2), 32, 24, 16, 4.0)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.0) < 1e-12


def test_configs_shapes_and_seeds():
    p0 = config_problem(0)
    assert (p0.nx, p0.ny, p0.nz) == (32, 32, 32) and np.all(p0.KX == 1e-14)
    p1 = config_problem(1, size=16)
    assert p1.conduit_mask.sum() > 0 and p1.KX.max() == 1e-10
    p2a, p2b = config_problem(2, size=12), config_problem(2, size=12)
    np.testing.assert_array_equal(p2a.KX, p2b.KX)
    p3 = config_problem(3, realisation=5)
    assert 24 <= min(p3.nx, p3.ny, p3.nz) and max(p3.nx, p3.ny, p3.nz) <= 96
    assert abs(p3.hx - 1 / 64) < 1e-15


def test_make_problem_bc_override():
    p = make_problem(4, 3, 2, bc_type=(1,) * 6, bc_value=(0.5,) * 6)
    assert p.bc_type == (1,) * 6
    fa = p.face_arrays()
    assert [len(f) for f in fa] == [6, 6, 8, 8, 12, 12]
