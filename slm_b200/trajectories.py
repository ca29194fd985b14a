"""Recorded streamline trajectories: drop-in for the reference's ``Trajectories``.

Mirrors ``python/streamlines/trajectories.py`` (class ``Trajectories``,
:40-346): same constructor and ``integrate()`` contract -- fills
``data.seed_point_array``, ``data.streamline_arrays_list`` (per direction, one
int8 ``(n_steps, 2)`` array of steps in 1/trajectory_resolution px per seed),
``data.traj_nsteps_array`` uint16 ``[N, 2]``, ``data.traj_length_array``
float32 ``[N, 2]`` and ``data.traj_stats_df`` -- with the tracing done by the
CUDA kernel ``k_trajectory``.  Chunking by device memory follows
``Trajectories.choose_chunks`` (:166-194) with the device's total memory.
The per-direction lists are NumPy object arrays of the per-seed step arrays.
"""
from __future__ import annotations

import numpy as np
import torch

from . import kernels
from .device import cuda_device, to_device, traced
from .params import kernel_params
from .useful import compute_stats, create_seeds_device, vprint


class Trajectories:
    def __init__(self, cl_platform, cl_device, cl_src_path=None, info=None, data=None,
                 do_trace_downstream=True, do_trace_upstream=True, verbose=False,
                 gpu_verbose=False, integrator=2):
        self.device = cuda_device(cl_platform, cl_device)
        self.cl_src_path = cl_src_path
        self.info = info
        self.data = data
        self.do_trace_downstream = do_trace_downstream
        self.do_trace_upstream = do_trace_upstream
        self.verbose = verbose
        self.gpu_verbose = gpu_verbose
        self.integrator = integrator
        self.n_steps = 0

    @traced("slm.Trajectories.integrate")
    def integrate(self):
        vprint(self.verbose, "Integrating trajectories...")
        info = self.info
        mask_array = self.data.mask_array
        # the seed list on the device (create_seeds' rows in its order): the
        # full shuffle runs there, only the first n_trajectory_seed_points
        # rows come back
        with torch.cuda.device(self.device):
            self._mask_d = to_device(mask_array, self.device)
            seeds_d, n_seed_points, n_padded_seed_points = create_seeds_device(
                mask_array, info.pad_width, info.n_work_items, self.device,
                n_seed_points=info.n_trajectory_seed_points, do_shuffle=info.do_shuffle,
                rng_seed=info.shuffle_rng_seed, verbose=self.verbose, mask_d=self._mask_d)
            self.data.seed_point_array = seeds_d.cpu().numpy()
            del seeds_d
        info.n_seed_points = n_seed_points
        info.n_padded_seed_points = n_padded_seed_points
        if self.data.mapping_array is None:
            self.data.mapping_array = np.zeros_like(mask_array, dtype=np.uint32)
        total = torch.cuda.get_device_properties(self.device).total_memory
        limit = (total * int(info.gpu_memory_limit_pc)) // 100
        request = n_seed_points * np.dtype(np.uint8).itemsize * int(info.max_n_steps) * 2
        n_chunks = max(1, int(np.ceil(request / limit)))
        self.choose_chunks(n_chunks)
        self.gpu_compute_trajectories()
        self._mask_d = None
        self.data.traj_stats_df = compute_stats(self.data.traj_length_array,
                                                self.data.traj_nsteps_array,
                                                info.pixel_size, self.verbose)
        vprint(self.verbose, "...done")

    def choose_chunks(self, n_chunks):
        ns = int(self.info.n_seed_points)
        npad = int(self.info.n_padded_seed_points)
        self.chunk_size = int(np.round(npad / n_chunks))
        chunk_list = [[i, c, min(ns, c + self.chunk_size) - c, self.chunk_size]
                      for i, c in enumerate(range(0, npad, self.chunk_size))]
        trace_do_list = [[self.do_trace_downstream, "Downstream:", 0, np.float32(+1.0)],
                         [self.do_trace_upstream, "Upstream:  ", 1, np.float32(-1.0)]]
        self.trace_do_chunks = [td + chunk for td in trace_do_list for chunk in chunk_list]

    def gpu_compute_trajectories(self):
        info = self.info
        dev = self.device
        ns = int(info.n_seed_points)
        nl = int(info.max_n_steps)
        streamline_arrays_list = [[], []]
        traj_nsteps_array = np.zeros([ns, 2], dtype=np.uint16)
        traj_length_array = np.zeros([ns, 2], dtype=np.float32)
        with torch.cuda.device(dev):
            seeds_d = to_device(self.data.seed_point_array, dev, torch.float32)
            mask_d = getattr(self, "_mask_d", None)
            if mask_d is None:
                mask_d = to_device(self.data.mask_array, dev)
            uv_d = to_device(self.data.uv_array, dev, torch.float32)
            todo = [td[1:] for td in self.trace_do_chunks if td[0]]
            # one chunk per direction (the usual case): both directions run
            # at once on their own streams (each kernel is a few thousand
            # latency-bound threads); otherwise chunk after chunk
            concurrent = len(todo) == 2 and todo[0][1] != todo[1][1]
            n_buf = 2 if concurrent else 1
            trajs = [torch.zeros(self.chunk_size * nl * 2, dtype=torch.int8, device=dev) for _ in range(n_buf)]
            nsteps = [torch.zeros(self.chunk_size, dtype=torch.uint16, device=dev) for _ in range(n_buf)]
            lengths = [torch.zeros(self.chunk_size, dtype=torch.float32, device=dev) for _ in range(n_buf)]
            cur = torch.cuda.current_stream(dev)
            if concurrent:
                streams = [torch.cuda.Stream(dev) for _ in range(2)]
                for j, (_, downup_idx, downup_sign, _c, seeds_chunk_offset, _n, n_chunk_ki) in enumerate(todo):
                    info.downup_sign = downup_sign
                    info.seeds_chunk_offset = seeds_chunk_offset
                    prm = kernel_params(info, "INTEGRATE_TRAJECTORY", downup_sign)
                    streams[j].wait_stream(cur)
                    kernels.integrate_trajectory(prm, n_chunk_ki, seeds_d, mask_d, uv_d, trajs[j],
                                                 nsteps[j], lengths[j], integrator=self.integrator,
                                                 stream=streams[j])
                for st in streams:
                    cur.wait_stream(st)
            for j, (_, downup_idx, downup_sign, _chunk_idx, seeds_chunk_offset, n_chunk_seeds,
                    n_chunk_ki) in enumerate(todo):
                b = j if concurrent else 0
                traj_d, nsteps_d, length_d = trajs[b], nsteps[b], lengths[b]
                if not concurrent:
                    info.downup_sign = downup_sign
                    info.seeds_chunk_offset = seeds_chunk_offset
                    prm = kernel_params(info, "INTEGRATE_TRAJECTORY", downup_sign)
                    kernels.integrate_trajectory(prm, n_chunk_ki, seeds_d, mask_d, uv_d, traj_d,
                                                 nsteps_d, length_d, integrator=self.integrator)
                n = max(n_chunk_seeds, 0)
                chunk_nsteps = nsteps_d[:n].cpu().numpy()
                chunk_length = length_d[:n].cpu().numpy()
                # copy back only the recorded prefix of each seed's row
                rows = traj_d.view(self.chunk_size, nl, 2)[:n]
                maxn = int(chunk_nsteps.max()) if n else 0
                chunk_traj = rows[:, :maxn].cpu().numpy()
                for k in range(n):
                    streamline_arrays_list[downup_idx].append(chunk_traj[k, :chunk_nsteps[k]].copy())
                traj_nsteps_array[seeds_chunk_offset:seeds_chunk_offset + n, downup_idx] = chunk_nsteps
                traj_length_array[seeds_chunk_offset:seeds_chunk_offset + n, downup_idx] = chunk_length
                self.n_steps += int(chunk_nsteps.astype(np.int64).sum())
            info.seeds_chunk_offset = np.uint32(0)
        for downup_idx in (0, 1):
            arr = np.empty(len(streamline_arrays_list[downup_idx]), dtype=object)
            for k, a in enumerate(streamline_arrays_list[downup_idx]):
                arr[k] = a
            streamline_arrays_list[downup_idx] = arr
        self.data.streamline_arrays_list = streamline_arrays_list
        self.data.traj_nsteps_array = traj_nsteps_array[0:ns].copy()
        self.data.traj_length_array = traj_length_array[0:ns].copy()


def decode_streamlines(seed_point_array, streamline_arrays_list, trajectory_resolution, origin=(0.0, 0.0),
                       indexes=None):
    """Positions of recorded trajectories from their wire format: each is a
    char2 list of steps in units of 1/trajectory_resolution pixel from its
    seed.  The decoding is the reference's plotting code's (plot.py:1414-1423):
    a (0, 0) start, the steps as float32 over the resolution, a running
    float32 sum per axis, plus the ROI origin, plus the seed.  Returns a list
    of (x, y) float32 arrays, one per trajectory (all, or ``indexes``)."""
    res = np.float32(trajectory_resolution)
    ox, oy = np.float32(origin[0]), np.float32(origin[1])
    out = []
    for k in (range(len(streamline_arrays_list)) if indexes is None else indexes):
        steps = np.asarray(streamline_arrays_list[k]).reshape(-1, 2)
        t = np.concatenate((np.zeros((1, 2), np.float32), steps.astype(np.float32) / res))
        seed = seed_point_array[k, :]
        out.append((ox + np.cumsum(t.T[0]) + seed[0], oy + np.cumsum(t.T[1]) + seed[1]))
    return out
