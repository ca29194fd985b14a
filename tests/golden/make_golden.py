#!/usr/bin/env python3
"""Generate the golden vectors in this folder from the reference's own kernels.

Runs the reference's OpenCL C kernels compiled on the host by
``oracle/build_ref.py`` (which needs the reference checkout) on small seeded
synthetic cases and stores inputs, the ``-D`` option list and outputs as
``.npz``.  The tests check the oracle's C restatement against these files
wherever the reference checkout is absent.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as O  # noqa: E402
from cases import Case  # noqa: E402
from slm_b200 import params as P  # noqa: E402

FIELD_CASES = {
    "fields_a": dict(nx=24, ny=20, seed=11, density=2, jitter=1.0, step=0.5, max_length=60.0),
    "fields_b": dict(nx=20, ny=28, seed=12, density=1, jitter=0.0, step=0.1, max_length=20.0,
                     holes=True),
    "fields_c": dict(nx=18, ny=18, seed=13, density=3, jitter=1.0, step=0.25, max_length=40.0,
                     pixel_size=2.0),
}
TRAJ_CASES = {
    "traj_a": dict(nx=30, ny=26, seed=14, step=0.5, max_length=40.0, n_traj_seeds=64, holes=True),
    "traj_b": dict(nx=22, ny=22, seed=15, step=0.1, max_length=15.0, n_traj_seeds=48),
}


def main():
    from build_ref import build_all
    build_all(only=["integrate_fields", "integrate_trajectory"])
    for name, kw in FIELD_CASES.items():
        c = Case(**kw)
        out = dict(uv=c.uv, mask=c.mask, seeds=c.seeds)
        for tag, sign in (("down", 1.0), ("up", -1.0)):
            opts = P.compile_options(c.info, "INTEGRATE_FIELDS", sign)
            prm = P.params_from_options(opts)
            slc, slt = O.ref_integrate_fields(prm, c.seeds, c.mask, c.uv)
            out["options_" + tag] = np.array(opts)
            out["slc_" + tag] = slc
            out["slt_" + tag] = slt
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "slc sums", int(out["slc_down"].sum()), int(out["slc_up"].sum()))
    for name, kw in TRAJ_CASES.items():
        c = Case(**kw)
        out = dict(uv=c.uv, mask=c.mask, seeds=c.seeds)
        ns = int(c.info.n_seed_points)
        for tag, sign in (("down", np.float32(1.0)), ("up", np.float32(-1.0))):
            opts = P.compile_options(c.info, "INTEGRATE_TRAJECTORY", sign)
            prm = P.params_from_options(opts)
            traj, nsteps, length = O.ref_integrate_trajectory(prm, ns, c.seeds, c.mask, c.uv)
            out["options_" + tag] = np.array(opts)
            out["traj_" + tag] = traj
            out["nsteps_" + tag] = nsteps
            out["length_" + tag] = length
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "nsteps means", out["nsteps_down"].mean(), out["nsteps_up"].mean())


if __name__ == "__main__":
    main()
