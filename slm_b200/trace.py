"""The Trace stage: trajectories and fields of a DTM region on the GPU.

Mirrors ``streamlines.trace.Trace`` (python/streamlines/trace.py:31-170), the
caller of the two hot-path wrappers: ``do()`` runs ``compute_trajectories``
then ``compute_fields``, with the fields' seed list and tracing passes run
on a worker thread and a side stream while the trajectories run
(``Fields.prepare``; the trajectory statistics are needed only by the
fields' post-processing).  Each crops the merged active mask and the uv field
to the bounding box of the unmasked pixels (widened by the pad), runs
``slm_b200.trajectories.Trajectories`` / ``slm_b200.fields.Fields`` on the
crop, and writes the results back into full padded ROI arrays, as the
reference does:

- ``seed_point_array``: the trajectory seeds, offset back to the ROI frame;
- ``streamline_arrays_list``, ``traj_stats_df``;
- ``slc_array`` (uint32: the float field truncated on assignment, as
  trace.py:159-166 does), ``slt_array``, ``sla_array`` (float32),
  [nxp, nyp, 2], zero outside the crop.
"""
from __future__ import annotations

import numpy as np

from .device import traced
from .fields import Fields
from .trajectories import Trajectories
from .useful import Data, Info, default_parameters, get_bbox, vprint


class Trace:
    """``state``: the job state (``merge_active_masks()``, ``cl_platform``,
    ``cl_device`` and the state parameters Info reads); ``imported_parameters``:
    the job's parameters (its 'trace' section, or that section itself);
    ``geodata``: ``roi_nx``, ``roi_ny``, ``pad_width``, ``roi_pixel_size``;
    ``preprocess``: ``uv_array``.  ``integrator`` (2, the reference's RK2, or
    4) and ``schedule`` select this project's tracer options."""

    def __init__(self, state, imported_parameters, geodata, preprocess, integrator=2, schedule="persistent"):
        params = dict(vars(default_parameters().trace))
        if imported_parameters:
            params.update(imported_parameters.get("trace", imported_parameters))
        for k, v in params.items():
            setattr(self, k, v)
        self.state = state
        self.geodata = geodata
        self.preprocess = preprocess
        self.integrator = integrator
        self.schedule = schedule
        self.mapping_array = None
        self.seed_point_array = None

    def print(self, *args, **kwargs):
        vprint(getattr(self.state, "verbose", False), *args, **kwargs)

    @traced("slm.Trace.do")
    def do(self):
        self.print("\n**Trace begin**")
        # the fields' seed list and passes run while the trajectories run
        job = self._fields_job()
        job[0].prepare()
        self.compute_trajectories()
        self.compute_fields(job)
        self.print("**Trace end**\n")

    def _crop(self):
        mask_array = self.state.merge_active_masks()
        bbox, bnx, bny = get_bbox(~mask_array)
        pad = self.geodata.pad_width
        nxp = self.geodata.roi_nx + pad * 2
        nyp = self.geodata.roi_ny + pad * 2
        info = Info(self.state, self, self.geodata.roi_pixel_size)
        info.set_xy(bnx, bny, pad)
        return mask_array, bbox, pad, nxp, nyp, info

    def compute_trajectories(self):
        """trace.py:93-128: the recorded trajectories of the cropped region."""
        mask_array, bbox, pad, nxp, nyp, info = self._crop()
        data = Data(info=info, bbox=bbox, pad=pad, mapping_array=np.zeros((nxp, nyp), dtype=np.uint32),
                    mask_array=mask_array, uv_array=self.preprocess.uv_array)
        trajectories = Trajectories(self.state.cl_platform, self.state.cl_device,
                                    cl_src_path=getattr(self.state, "cl_src_path", None), info=info, data=data,
                                    do_trace_downstream=self.do_trace_downstream,
                                    do_trace_upstream=self.do_trace_upstream,
                                    verbose=getattr(self.state, "verbose", False),
                                    gpu_verbose=getattr(self.state, "gpu_verbose", False),
                                    integrator=self.integrator)
        trajectories.integrate()
        offset_xy = np.array((bbox[0] - pad, bbox[2] - pad))
        self.seed_point_array = trajectories.data.seed_point_array + offset_xy
        self.streamline_arrays_list = trajectories.data.streamline_arrays_list
        self.traj_stats_df = trajectories.data.traj_stats_df

    def _fields_job(self):
        """The Fields wrapper of the cropped region and its Data (the
        trajectory statistics are added when the fields are computed)."""
        mask_array, bbox, pad, nxp, nyp, info = self._crop()
        data = Data(info=info, bbox=bbox, pad=pad, mask_array=mask_array, uv_array=self.preprocess.uv_array,
                    mapping_array=np.zeros((nxp, nyp), dtype=np.uint32), traj_stats_df=None)
        fields = Fields(self.state.cl_platform, self.state.cl_device,
                        cl_src_path=getattr(self.state, "cl_src_path", None), info=info, data=data,
                        verbose=getattr(self.state, "verbose", False),
                        gpu_verbose=getattr(self.state, "gpu_verbose", False),
                        schedule=self.schedule, integrator=self.integrator)
        return fields, data, nxp, nyp

    def compute_fields(self, job=None):
        """trace.py:130-170: the slc / slt / sla fields of the cropped region,
        written back into full padded arrays.  ``job``: a ``_fields_job()``
        whose seed list may already be under way."""
        fields, data, nxp, nyp = job if job is not None else self._fields_job()
        data.traj_stats_df = self.traj_stats_df
        fields.integrate()
        self.slc_array = np.zeros((nxp, nyp, 2), dtype=np.uint32)
        self.slt_array = np.zeros((nxp, nyp, 2), dtype=np.float32)
        self.sla_array = np.zeros((nxp, nyp, 2), dtype=np.float32)
        bounds = data.bounds_slx
        self.slc_array[bounds] = fields.data.slc_array
        self.slt_array[bounds] = fields.data.slt_array
        self.sla_array[bounds] = fields.data.sla_array
