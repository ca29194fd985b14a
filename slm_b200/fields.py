"""Streamline length/count fields: drop-in for the reference's ``Fields`` stage.

Mirrors ``python/streamlines/fields.py`` (class ``Fields``, :37-310): same
constructor, same ``integrate()`` contract on ``data`` -- fills
``data.seed_point_array`` and ``data.slc_array`` / ``slt_array`` /
``sla_array`` of shape ``(nxp, nyp, 2)`` (index 0 downstream, 1 upstream) --
with the tracing done by the CUDA kernels of ``libslm_b200.so`` instead of
PyOpenCL.  ``integrate()`` runs the reference's post-processing on the GPU
(``slm_fields_finish``, NumPy's promotion order, the pow of slc through a
table computed with the reference expression) and copies back only the
finished arrays; ``gpu_integrate()`` alone leaves the reference's raw
intermediate arrays, converted on the host step for step.

Differences from the reference (none changes a result):
* one parameter block per pass instead of an OpenCL program rebuild per pass;
* no time-sliced chunked launches (pocl.py:394-445): one persistent launch per
  direction; ``max_time_per_kernel`` is not used;
* device accumulators are uint64; ``slc``/``slt`` returned to the caller are
  the low 32 bits (what the reference's uint32 atomics hold) unless
  ``exact=True``, which keeps the full sums;
* with ``process_group`` (one process per GPU) each rank traces its dealt
  share of the tracer's queue (chunks of 64 queue positions, round robin;
  slm_b200.distributed) and the uint64 accumulators are summed with one
  all-reduce; every rank then holds the full fields.
"""
from __future__ import annotations

import numpy as np
import torch

from . import kernels
from .device import cuda_device, download, host_copy, low32, pinned_staging, to_device, traced
from .distributed import allreduce_counts, shard_queue, shard_queue_params, sharded_field_pass
from .params import kernel_params
from .useful import create_seeds_device, create_seeds_device_state, vprint


_SLC_TABLES = {}


def _slc_table(dev, dd, n):
    """Device table of sqrt(2) * (count / d^2) ** (2/3) for counts 0..n-1,
    computed with the reference's NumPy expression (so looked-up values are
    the reference's bit for bit); kept per device and d^2, grown on demand."""
    key = (str(dev), int(dd))
    t = _SLC_TABLES.get(key)
    if t is None or t.numel() < n:
        m = max(n, 2 * t.numel() if t is not None else 0, 1 << 16)
        table = np.sqrt(2.0) * np.power(np.arange(m) / dd, 2 / 3)
        t = torch.from_numpy(table).to(dev)
        _SLC_TABLES[key] = t
    return t


def _staging(slot, t):
    """Pinned host tensor shaped like device tensor ``t`` (kept for reuse, one per slot)."""
    return pinned_staging(slot, t.shape, t.dtype)


_ROWS_POOL = None
_SEEDS_POOL = None


def _rows_to_host_behind(t, dev, after=None):
    """A future of a fresh NumPy copy of device tensor ``t``: the copy to
    pinned memory runs on a side stream behind the work queued so far (or
    behind the CUDA event ``after`` alone), the copy out of it on a worker
    thread, so both overlap what the caller queues next."""
    global _ROWS_POOL
    if _ROWS_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _ROWS_POOL = ThreadPoolExecutor(1)
    side = torch.cuda.Stream(dev)
    if after is None:
        side.wait_stream(torch.cuda.current_stream(dev))
    else:
        side.wait_event(after)
    stage = _staging("seed rows", t)
    with torch.cuda.stream(side):
        stage.copy_(t, non_blocking=True)
        t.record_stream(side)
        done = torch.cuda.Event()
        done.record(side)

    def finish():
        done.synchronize()
        return host_copy(stage.numpy())
    return _ROWS_POOL.submit(finish)


class Fields:
    def __init__(self, cl_platform, cl_device, cl_src_path=None, info=None, data=None,
                 verbose=False, gpu_verbose=False, schedule="persistent", integrator=2,
                 exact=False, process_group=None, seed_order="spatial"):
        self.device = cuda_device(cl_platform, cl_device)
        self.cl_src_path = cl_src_path  # unused: kernels are prebuilt
        self.info = info
        self.data = data
        self.verbose = verbose
        self.gpu_verbose = gpu_verbose
        self.vprogress = verbose
        self.schedule = schedule
        self.integrator = integrator
        self.exact = exact
        self.process_group = process_group
        # "spatial": trace seeds in pixel-block order (slm_order_spatial), which
        # keeps large grids' working set in L2; "shuffled": the seed array's
        # own order, as the reference.  The fields are identical either way.
        if seed_order not in ("spatial", "shuffled"):
            raise ValueError("seed_order must be 'spatial' or 'shuffled'")
        self.seed_order = seed_order
        self.n_steps = [0, 0]
        self.n_trajectories = [0, 0]
        self._prepared = None

    # largest slc count whose pow is looked up in a host-computed table
    SLC_TABLE_MAX = 1 << 22

    def prepare(self, trace=True):
        """Start the work of ``integrate`` that does not need the trajectory
        statistics -- the seed list and, with ``trace``, both tracing passes
        -- on a worker thread and a side stream, and return at once;
        ``integrate`` waits for it and finishes (the statistics scale only the
        post-processing).  The Trace stage calls this before it runs the
        trajectories, so this work overlaps them.  The results are those of
        ``integrate`` alone; NumPy's global generator is set where
        ``integrate`` would set it.  With a process group only the seed list
        is prepared (the passes' collectives stay on the caller's thread)."""
        global _SEEDS_POOL
        if _SEEDS_POOL is None:
            from concurrent.futures import ThreadPoolExecutor
            _SEEDS_POOL = ThreadPoolExecutor(1)
        info, dev, mask_array, verbose = self.info, self.device, self.data.mask_array, self.verbose
        trace = trace and self.process_group is None

        def build():
            with torch.cuda.device(dev):
                side = torch.cuda.Stream(dev)
                with torch.cuda.stream(side):
                    mask_d = to_device(mask_array, dev)
                    seeds_d, n, npad, state = create_seeds_device_state(
                        mask_array, info.pad_width, info.n_work_items, dev, do_shuffle=info.do_shuffle,
                        rng_seed=info.shuffle_rng_seed, verbose=verbose, mask_d=mask_d, stream=side)
                    acc = host_seeds = None
                    if trace:
                        info.n_seed_points, info.n_padded_seed_points = n, npad
                        acc, host_seeds = self._trace_and_rows(seeds_d, mask_d)
                    done = torch.cuda.Event()
                    done.record(side)
            return mask_d, seeds_d, n, npad, state, done, acc, host_seeds
        self._prepared = _SEEDS_POOL.submit(build)

    def prepare_seeds(self):
        """``prepare`` without the tracing passes: only the seed list."""
        self.prepare(trace=False)

    def _take_prepared(self, dev):
        mask_d, seeds_d, n, npad, state, done, acc, host_seeds = self._prepared.result()
        self._prepared = None
        cur = torch.cuda.current_stream(dev)
        cur.wait_event(done)
        for t in (mask_d, seeds_d, acc):
            if t is not None:
                t.record_stream(cur)
        if state is not None:
            np.random.set_state(state)
        return mask_d, seeds_d, n, npad, acc, host_seeds

    @traced("slm.Fields.integrate")
    def integrate(self):
        """Trace all seeds down and up, then post-process slt/slc/sla (fields.py:69-167)."""
        vprint(self.verbose, "Integrating streamline fields...")
        info = self.info
        mask_array = self.data.mask_array
        traj_stats_df = self.data.traj_stats_df
        pixel_size = info.pixel_size
        dds = traj_stats_df["ds"]["downstream", "mean"]
        uds = traj_stats_df["ds"]["upstream", "mean"]
        nxp, nyp = mask_array.shape
        dev = self.device
        with torch.cuda.device(dev):
            # the seed list is built on the device (the rows create_seeds
            # gives, in its order); its host copy for data.seed_point_array is
            # taken behind the trace
            acc = host_seeds = None
            if self._prepared is not None:
                mask_d, seeds_d, info.n_seed_points, info.n_padded_seed_points, acc, host_seeds = \
                    self._take_prepared(dev)
            else:
                mask_d = to_device(mask_array, dev)
                seeds_d, info.n_seed_points, info.n_padded_seed_points = create_seeds_device(
                    mask_array, info.pad_width, info.n_work_items, dev, do_shuffle=info.do_shuffle,
                    rng_seed=info.shuffle_rng_seed, verbose=self.verbose, mask_d=mask_d)
            if acc is None:
                acc, host_seeds = self._trace_and_rows(seeds_d, mask_d)
            self._finish(acc, float(dds / pixel_size), float(uds / pixel_size), nxp, nyp)
            self.data.seed_point_array = host_seeds.result()
        vprint(self.verbose, "...done")

    def _trace_and_rows(self, seeds_d, mask_d):
        """``_trace`` of the seed list ``seeds_d``, with its copy to the host
        (a future of it) queued once the first pass is: the copy runs beside
        the passes and its host-side call does not delay their launch."""
        dev = self.device
        seeds_ready = torch.cuda.Event()
        seeds_ready.record(torch.cuda.current_stream(dev))
        rows = []
        acc = self._trace(seeds_d, mask_d, on_launch=lambda: rows.append(
            _rows_to_host_behind(seeds_d, dev, after=seeds_ready)))
        return acc, rows[0]

    @traced("slm.Fields.finish")
    def _finish(self, acc, scale_down, scale_up, nxp, nyp):
        """slm_fields_finish on the device; finished arrays copied to the host."""
        from . import _lib
        from ._lib import check, ptr
        dev = self.device
        info = self.info
        nxy = nxp * nyp
        dd = info.subpixel_seed_point_density ** 2
        counts = acc[:, 0].reshape(-1).view(torch.int64)
        if not self.exact:
            counts = counts & 0xFFFFFFFF  # the uint32 wrap the kernel applies
        cmax = int(counts.max().item()) if nxy else 0
        n_tab = min(cmax, self.SLC_TABLE_MAX) + 1
        table_d = _slc_table(dev, dd, n_tab)
        slc = torch.empty((nxp, nyp, 2), dtype=torch.float64, device=dev)
        slt = torch.empty((nxp, nyp, 2), dtype=torch.float32, device=dev)
        sla = torch.empty((nxp, nyp, 2), dtype=torch.float32, device=dev)
        check(_lib.load().slm_fields_finish(
            ptr(acc), nxy, int(info.subpixel_seed_point_density), scale_down, scale_up,
            1 if self.exact else 0, ptr(table_d), n_tab, ptr(slc), ptr(slt), ptr(sla),
            kernels._stream(None)))
        # by DMA straight into page-locked arrays the caller owns
        self.data.slc_array, self.data.slt_array, self.data.sla_array = download(
            (slc, slt, sla), "fields", pinned=True)

    @traced("slm.Fields.trace")
    def _trace(self, seeds_d=None, mask_d=None, on_launch=None):
        """Both passes on the device; returns the uint64 accumulators [2, 2, nxy].
        The seeds and mask come from ``data`` unless given on the device;
        ``on_launch`` is called once the first pass is queued."""
        info = self.info
        dev = self.device
        mask_array = self.data.mask_array
        nxp, nyp = mask_array.shape
        nxy = nxp * nyp
        with torch.cuda.device(dev):
            if seeds_d is None:
                seeds_d = to_device(self.data.seed_point_array, dev, torch.float32)
            if mask_d is None:
                mask_d = to_device(mask_array, dev)
            uv_d = to_device(self.data.uv_array, dev, torch.float32)
            work = kernels.workspace(dev)
            acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=dev)  # [downup, slc/slt]
            order = None
            if self.seed_order == "spatial" and int(info.n_seed_points) > 0:
                from .scheduler import spatial_order
                order = spatial_order(seeds_d, info.n_seed_points, info.nx, info.ny)
            if self.schedule == "persistent":
                # both directions in one persistent launch: each one's tail
                # fills with the other's trajectories
                prm = [kernel_params(info, "INTEGRATE_FIELDS", sign) for sign in (+1.0, -1.0)]
                info.downup_sign = -1.0
                for d in (0, 1):
                    self.n_trajectories[d] = int(prm[d].n_seed_points) * int(prm[d].subpixel_seed_point_density) ** 2
                pg = self.process_group
                queue = order
                if pg is not None:
                    import torch.distributed as dist
                    queue = shard_queue(order, int(info.n_seed_points), dist.get_rank(pg),
                                        dist.get_world_size(pg), device=dev)
                    prm = [shard_queue_params(p, queue) for p in prm]
                kernels.integrate_fields_pair(prm[0], prm[1], seeds_d, mask_d, uv_d, acc[:, 0], acc[:, 1], work,
                                              integrator=self.integrator, order=queue)
                if on_launch is not None:
                    on_launch()
                counts = work[1:4].view(torch.int64).clone()
                if pg is not None:
                    allreduce_counts(acc, counts, group=pg)
                counts = counts.cpu().tolist()
                self.n_steps[0], self.n_steps[1] = counts[0] - counts[2], counts[2]
                return acc
            if on_launch is not None:
                on_launch()
            for downup_idx, downup_sign in ((0, +1.0), (1, -1.0)):
                info.downup_sign = downup_sign
                prm = kernel_params(info, "INTEGRATE_FIELDS", downup_sign)

                def trace(p, slc, slt, queue):
                    kernels.integrate_fields(p, seeds_d, mask_d, uv_d, slc, slt, work,
                                             schedule=self.schedule, integrator=self.integrator,
                                             order=queue)
                    return int(work[1].view(torch.int64).item())

                if self.process_group is None:
                    self.n_steps[downup_idx] = trace(prm, acc[downup_idx, 0], acc[downup_idx, 1], order)
                else:
                    _, self.n_steps[downup_idx] = sharded_field_pass(
                        prm, trace, acc[downup_idx, 0], acc[downup_idx, 1], self.process_group, order=order)
                self.n_trajectories[downup_idx] = int(prm.n_seed_points) * int(prm.subpixel_seed_point_density) ** 2
        return acc

    def gpu_integrate(self):
        """Both passes on the device; fills raw slc/slt/sla like fields.py:169-310."""
        info = self.info
        dev = self.device
        nxp, nyp = self.data.mask_array.shape
        nxy = nxp * nyp
        with torch.cuda.device(dev):
            acc = self._trace()
            if self.exact:
                raw = acc.cpu().numpy()
                slc_raw = raw[:, 0].astype(np.float64)
                slt_raw = raw[:, 1].astype(np.float64)
            else:
                raw = low32(acc.view(-1)).view(2, 2, nxy).cpu().numpy()
                slc_raw = raw[:, 0]
                slt_raw = raw[:, 1]
        self.data.slc_array = np.zeros((nxp, nyp, 2), dtype=np.uint32 if not self.exact else np.float64)
        self.data.slt_array = np.zeros((nxp, nyp, 2), dtype=np.float32)
        self.data.sla_array = np.zeros((nxp, nyp, 2), dtype=np.float32)
        for downup_idx in (0, 1):
            self.data.slc_array[:, :, downup_idx] += slc_raw[downup_idx].reshape(nxp, nyp)
            self.data.slt_array[:, :, downup_idx] += slt_raw[downup_idx].reshape(nxp, nyp).astype(np.float32)
        slc, sla, slt = self.data.slc_array, self.data.sla_array, self.data.slt_array
        sla[slc == 0] = 0.0
        sla[slc > 0] = np.sqrt(2.0) * slt[slc > 0] / slc[slc > 0]
        slt[slc > 0] = slt[slc > 0] / info.subpixel_seed_point_density ** 2
