"""Seeded mapping-pipeline inputs and kernel runners for the mapping tests."""
import copy

import numpy as np

import oracle as O
from cases import Case
from slm_b200.useful import Data


class _OracleRunner:
    """The oracle as a mapping kernel runner; its ``fmm_solver`` is the
    oracle of the fast-marching kernel."""

    def __call__(self, name, params, seeds, arrays):
        status = O.map_kernel(name, params, seeds, arrays)
        assert status == 0, (name, status)

    @staticmethod
    def fmm_solver(*args, **kwargs):
        import eikonal
        return eikonal.solve_problems(*args, **kwargs)


oracle_runner = _OracleRunner()


class ComparingRunner:
    """Runs the reference's own kernel on copies of the buffers, then the
    oracle's restatement on the buffers themselves, and records any buffer
    that differs."""

    def __init__(self):
        self.mismatches = []
        self.calls = []

    def __call__(self, name, params, seeds, arrays):
        ref_arrays = [a.copy() for a in arrays]
        O.ref_map_kernel(name, params, seeds, ref_arrays)
        oracle_runner(name, params, seeds, arrays)
        self.calls.append((name, seeds.shape[0]))
        for k, (a, b) in enumerate(zip(arrays, ref_arrays)):
            if not np.array_equal(a.view(np.uint8), b.view(np.uint8)):
                self.mismatches.append((name, k, int(np.sum(a != b))))


def pipeline_case(nx=96, ny=80, seed=5, channel_pct=94.0, segmentation_threshold=10):
    """A Case with downstream/upstream fields (oracle), ready for mapping."""
    c = Case(nx=nx, ny=ny, seed=seed, density=1, jitter=0.0, step=0.5, max_length=200.0)
    nxp, nyp = c.mask.shape
    slc = np.zeros((nxp, nyp, 2), np.float64)
    slt = np.zeros((nxp, nyp, 2), np.float32)
    for d, sign in ((0, 1.0), (1, -1.0)):
        prm = c.params("INTEGRATE_FIELDS", sign)
        a, b, _, _ = O.integrate_fields(prm, c.seeds, c.mask, c.uv)
        slc[:, :, d] = a.reshape(nxp, nyp)
        slt[:, :, d] = np.sqrt(b.reshape(nxp, nyp).astype(np.float32) * np.float32(0.5))
    slc = np.sqrt(2.0) * np.power(slc, 2 / 3)
    info = c.info
    thr = np.float32(np.percentile(slt[:, :, 0][~c.mask], channel_pct))
    info.set_thresholds(segmentation_threshold=np.uint32(segmentation_threshold),
                        channel_threshold=thr)
    data = Data(info=info, mask_array=c.mask, uv_array=c.uv,
                mapping_array=np.zeros(c.mask.shape, np.uint32),
                slt_array=slt, slc_array=slc)
    return c, info, data


def midslope_case(data, info, seed=3, frac=0.05):
    """Flag a seeded random subset of hillslope pixels as midslope and size the
    hillslope-length output for them."""
    rng = np.random.default_rng(seed)
    hill = (~data.mask_array) & ((data.mapping_array & info.is_thinchannel) == 0)
    pick = hill & (rng.random(hill.shape) < frac)
    data.mapping_array[pick] |= info.is_midslope
    n = int(np.sum(~data.mask_array & ((data.mapping_array & info.is_midslope) > 0)))
    data.subsegment_hsl_array = np.zeros(n, dtype=np.float32)
    return n


def clone(data):
    return copy.deepcopy(data)


def incised_pipeline_case(n=128, seed=3, n_incisions=12, max_steps=300, channel_pct=94.0,
                          segmentation_threshold=10):
    """Mapping inputs on the incised relief of the 2048^2 workload at a small
    size.  Its V-shaped valley floors make count_downchannels walks oscillate
    to the 1000*MAX_N_STEPS bound and leave link cycles for
    flag_downchannels; max_steps keeps that bound small for the oracle."""
    from slm_b200 import synth
    from slm_b200.useful import Info, create_seeds, default_parameters
    d = default_parameters()
    d.trace.subpixel_seed_point_density = 1
    d.trace.jitter_magnitude = 0.0
    d.trace.integrator_step_factor = 0.1
    d.trace.max_length = max_steps * 0.1
    dtm = synth.incised_dtm(n, seed, n_incisions)
    uv, mask = synth.uv_from_dtm(dtm, 2.0, 2)
    info = Info(d.state, d.trace, 2.0)
    info.set_xy(n, n, 2)
    seeds, ns, npad = create_seeds(mask, 2, info.n_work_items, do_shuffle=True, rng_seed=1)
    info.n_seed_points, info.n_padded_seed_points = ns, npad
    nxp, nyp = mask.shape
    slc = np.zeros((nxp, nyp, 2), np.float64)
    slt = np.zeros((nxp, nyp, 2), np.float32)
    from slm_b200.params import kernel_params
    for k, sign in ((0, 1.0), (1, -1.0)):
        prm = kernel_params(info, "INTEGRATE_FIELDS", sign)
        a, b, _, _ = O.integrate_fields(prm, seeds, mask, uv)
        slc[:, :, k] = a.reshape(nxp, nyp)
        slt[:, :, k] = np.sqrt(b.reshape(nxp, nyp).astype(np.float32) * np.float32(1.0))
    slc = np.sqrt(2.0) * np.power(slc, 2 / 3)
    thr = np.float32(np.percentile(slt[:, :, 0][~mask], channel_pct))
    info.set_thresholds(segmentation_threshold=np.uint32(segmentation_threshold), channel_threshold=thr)
    data = Data(info=info, mask_array=mask, uv_array=uv, mapping_array=np.zeros(mask.shape, np.uint32),
                slt_array=slt, slc_array=slc)
    return info, data
