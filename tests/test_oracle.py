"""The oracle's C restatement against the reference's own kernels (CPU only).

Pins: the golden vectors in tests/golden/ (made by the reference's OpenCL C
compiled on the host, tests/golden/make_golden.py), and, where the compiled
reference is present (oracle/_ref/), direct comparisons on further cases.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from cases import Case
from slm_b200 import params as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _golden(prefix):
    files = sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))
    assert files, "golden fixtures missing"
    return files


@pytest.mark.parametrize("path", _golden("fields_"))
def test_fields_golden(path):
    g = np.load(path)
    for tag in ("down", "up"):
        prm = P.params_from_options(list(g["options_" + tag]))
        slc, slt, steps, ntraj = O.integrate_fields(prm, g["seeds"], g["mask"], g["uv"])
        assert np.array_equal(slc.astype(np.uint32), g["slc_" + tag])
        assert np.array_equal((slt & 0xFFFFFFFF).astype(np.uint32), g["slt_" + tag])
        d = prm.subpixel_seed_point_density
        assert ntraj == prm.n_seed_points * d * d
        assert steps > 0


@pytest.mark.parametrize("path", _golden("traj_"))
def test_trajectory_golden(path):
    g = np.load(path)
    for tag in ("down", "up"):
        prm = P.params_from_options(list(g["options_" + tag]))
        n = prm.n_seed_points
        traj, nsteps, length, steps = O.integrate_trajectory(prm, n, g["seeds"], g["mask"], g["uv"])
        assert np.array_equal(nsteps, g["nsteps_" + tag])
        assert np.array_equal(length.view(np.uint32), g["length_" + tag].view(np.uint32))
        assert np.array_equal(traj, g["traj_" + tag])
        assert steps == int(nsteps.astype(np.int64).sum())


needs_ref = pytest.mark.skipif(not O.ref_available("integrate_fields"),
                               reason="reference kernels not compiled (oracle/_ref)")


@needs_ref
@pytest.mark.parametrize("kw", [
    dict(nx=40, ny=56, seed=3, density=2, jitter=1.0, step=0.5, max_length=100.0),
    dict(nx=33, ny=27, seed=5, density=3, jitter=0.5, step=0.1, max_length=30.0, holes=True),
    dict(nx=30, ny=30, seed=6, density=1, jitter=0.0, step=0.5, max_length=0.75),
])
def test_fields_vs_reference(kw):
    c = Case(**kw)
    for sign in (1.0, -1.0):
        prm = c.params("INTEGRATE_FIELDS", sign)
        rslc, rslt = O.ref_integrate_fields(prm, c.seeds, c.mask, c.uv)
        slc, slt, _, _ = O.integrate_fields(prm, c.seeds, c.mask, c.uv)
        assert np.array_equal(slc.astype(np.uint32), rslc)
        assert np.array_equal((slt & 0xFFFFFFFF).astype(np.uint32), rslt)


@needs_ref
def test_fields_threads_deterministic():
    c = Case(nx=36, ny=30, seed=8, density=2)
    prm = c.params()
    a = O.integrate_fields(prm, c.seeds, c.mask, c.uv, n_threads=1)
    b = O.integrate_fields(prm, c.seeds, c.mask, c.uv, n_threads=4)
    rslc, rslt = O.ref_integrate_fields(prm, c.seeds, c.mask, c.uv, n_threads=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert np.array_equal(a[0].astype(np.uint32), rslc)


@needs_ref
@pytest.mark.parametrize("kw", [
    dict(nx=40, ny=40, seed=21, step=0.5, max_length=200.0, n_traj_seeds=200, holes=True),
    dict(nx=50, ny=30, seed=22, step=0.1, max_length=40.0, n_traj_seeds=100),
])
def test_trajectory_vs_reference(kw):
    c = Case(**kw)
    n = int(c.info.n_seed_points)
    for sign in (np.float32(1.0), np.float32(-1.0)):
        prm = c.params("INTEGRATE_TRAJECTORY", sign)
        rt, rn, rl = O.ref_integrate_trajectory(prm, n, c.seeds, c.mask, c.uv)
        t, nn, ll, _ = O.integrate_trajectory(prm, n, c.seeds, c.mask, c.uv)
        assert np.array_equal(rn, nn)
        assert np.array_equal(rl.view(np.uint32), ll.view(np.uint32))
        assert np.array_equal(rt, t)


@needs_ref
def test_trajectory_chunk_offset():
    c = Case(nx=30, ny=30, seed=23, n_traj_seeds=90)
    c.info.seeds_chunk_offset = np.uint32(40)
    prm = c.params("INTEGRATE_TRAJECTORY", np.float32(1.0))
    rt, rn, rl = O.ref_integrate_trajectory(prm, 32, c.seeds, c.mask, c.uv)
    t, nn, ll, _ = O.integrate_trajectory(prm, 32, c.seeds, c.mask, c.uv)
    assert np.array_equal(rn, nn) and np.array_equal(rt, t)


def test_rk4_oracle_properties():
    """RK4 is this project's extension (parity unpinned by the reference):
    check what holds by construction -- visits equal steps plus starts minus
    the trajectories that stepped into a masked pixel, and determinism."""
    c = Case(nx=32, ny=28, seed=9, density=2)
    prm = c.params()
    slc, slt, steps, ntraj = O.integrate_fields(prm, c.seeds, c.mask, c.uv, integrator=4)
    slc2, slt2, steps2, _ = O.integrate_fields(prm, c.seeds, c.mask, c.uv, integrator=4, n_threads=3)
    assert np.array_equal(slc, slc2) and np.array_equal(slt, slt2) and steps == steps2
    assert int(slc.sum()) <= steps + ntraj
    assert int(slc.sum()) >= steps  # each step adds a visit unless it entered a masked pixel
