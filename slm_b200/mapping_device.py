"""The mapping sequence with every grid resident on the GPU.

``mapping.map_channels_segments`` keeps the reference's wrappers: each kernel
call copies its NumPy buffers to the device and back, and the steps between
kernels (picking seeds, flag updates, thinning, relabelling) run in NumPy, as
in the reference (mapping.py:627-775).  ``map_channels_segments_device``
runs the same sequence with the same results, but uploads the inputs once,
does the in-between steps with the device kernels of map_device.cu
(``slm_pick_seeds``, ``slm_flag_op``, ``slm_map_channels``, ``slm_thin``,
``slm_relabel``, ``slm_signed_labels``), and copies the grids back once at the
end.  ``DeviceMapping.hsl`` does the same for the hillslope lengths.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, map_kernels
from ._lib import check, ptr
from .device import cuda_device, download, upload
from .params import kernel_params


_TORCH = {np.dtype(np.uint8): torch.uint8, np.dtype(np.float32): torch.float32,
          np.dtype(np.uint32): torch.uint32, np.dtype(np.float64): torch.float64}


class DeviceMapping:
    """Device copies of the mapping grids of one ``data`` object."""

    def __init__(self, info, data, device=None):
        """``data``: NumPy arrays (uploaded once), or CUDA tensors already on
        ``device`` (used in place; ``mapping_array`` is then updated there):
        ``mask_array`` [nxp, nyp] bool/uint8, ``uv_array`` [nxp, nyp, 2],
        ``mapping_array`` uint32, ``slt_array`` / ``slc_array`` [nxp, nyp, 2]
        (only the downstream half is read).  Its kernels run on the CUDA
        stream that is current when it is made."""
        self.info, self.data = info, data
        self.dev = device if device is not None else cuda_device(0, 0)
        self.L = _lib.load()
        dev = self.dev
        nxp, nyp = data.mask_array.shape
        self.shape = (nxp, nyp)
        self.n = nxp * nyp

        def up(a, dt, slot):
            if isinstance(a, torch.Tensor):
                t = a if a.dtype != torch.bool else a.view(torch.uint8)
                return t.to(dev, _TORCH[np.dtype(dt)]).contiguous()
            return upload(a, dev, ("mapping", slot), dtype=np.dtype(dt))
        m = data.mask_array
        self.mask = up(m.view(np.uint8) if isinstance(m, np.ndarray) and m.dtype == np.bool_ else m, np.uint8,
                       "mask")
        self.uv = up(data.uv_array, np.float32, "uv")
        self.mapping = up(data.mapping_array, np.uint32, "flags").reshape(-1)
        self.slt_dn = up(data.slt_array[:, :, 0], np.float32, "slt")
        self.slc_dn = up(data.slc_array[:, :, 0], np.float64, "slc")
        # the staging buffers are free again once the copies have run
        torch.cuda.current_stream(dev).synchronize()
        self.count = torch.zeros(self.n, dtype=torch.uint32, device=dev)
        self.link = torch.zeros(self.n, dtype=torch.uint32, device=dev)
        self.label = torch.zeros(self.n, dtype=torch.uint32, device=dev)
        self.channel_label = None
        self.select = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.scratch = torch.empty(self.n, dtype=torch.uint8, device=dev)
        self.flag = torch.zeros(1, dtype=torch.uint32, device=dev)
        self.pick_ws = torch.empty(int(self.L.slm_pick_seeds_workspace(self.n)), dtype=torch.uint8, device=dev)
        self.seeds = torch.empty((max(1, self.n), 2), dtype=torch.float32, device=dev)
        # status words of the kernels that report one, read back once
        self._status = 0
        self._slots = torch.zeros(32, dtype=torch.uint32, device=dev)
        self._n_slots = 0
        self._no_status = torch.zeros(1, dtype=torch.uint32, device=dev)
        self._prm = None
        # its kernels run on the stream that was current when it was made
        self._st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)

    @property
    def status(self):
        """OR of the status words of the kernels run so far (1: a walk the
        reference leaves unbounded hit its cap; 2: a read the reference would
        make outside the grid was skipped)."""
        if self._n_slots:
            self._status |= int(np.bitwise_or.reduce(self._slots[:self._n_slots].cpu().numpy()))
            self._slots.zero_()
            self._n_slots = 0
        return self._status

    def _params(self, n):
        """The launch parameters with n seeds.  They are formed from ``info``
        once: the mapping sequence changes only the seed count."""
        info = self.info
        info.n_seed_points = np.uint32(n)
        if self._prm is None:
            self._prm = kernel_params(info, "MAPPING")
        prm = self._prm.copy()
        prm.n_seed_points = int(info.n_seed_points)
        return prm

    def _stream(self):
        return self._st

    # ------------------------------------------------------------ host-step kernels
    def pick(self, mask=True, map=None, flag=0, invert=False):
        """pick_seeds on the device: (seeds view, n)."""
        got = ctypes.c_uint32(0)
        check(self.L.slm_pick_seeds(ptr(self.mask) if mask else None, ptr(map), int(flag), 1 if invert else 0,
                                    self.shape[0], self.shape[1], int(self.info.pad_width), ptr(self.seeds),
                                    self.n, ctypes.byref(got), ptr(self.pick_ws), self.pick_ws.numel(),
                                    self._stream()))
        return self.seeds, int(got.value)

    def flag_op(self, op, a, b=0, select=None):
        check(self.L.slm_flag_op(ptr(self.mapping), ptr(select), self.n, int(op), int(a), int(b), self._stream()))

    def run(self, kernel, seeds, n, bufs):
        prm = self._params(n)
        if map_kernels.SPECS[kernel][2] == "status":
            if self._n_slots == self._slots.numel():
                self.status  # noqa: B018 - folds the words read so far
            slot = self._slots[self._n_slots:self._n_slots + 1]
            self._n_slots += 1
        else:
            slot = self._no_status
        map_kernels.run_device(kernel, prm, seeds, n, bufs, self.dev, self._stream(), status=slot)

    # ------------------------------------------------------------ the sequence
    def map_channels_segments(self, do_map_channels_from_scratch=True, do_map_segments=True):
        info, dev = self.info, self.dev
        m = self.mapping
        if do_map_channels_from_scratch:
            check(self.L.slm_map_channels(ptr(self.slt_dn), ptr(self.slc_dn), float(np.float32(info.channel_threshold)),
                                          self.n, int(info.is_channel), ptr(m), self._stream()))
        seeds, n = self.pick(mask=False, map=m, flag=info.is_channel)
        if n == 0:
            return False
        self.run("connect_channels", seeds, n, [self.mask, self.uv, m])
        # thinning of channel | interchannel pixels, then IS_THINCHANNEL on them
        self.flag_op(3, info.is_channel, info.is_interchannel, select=self.select)
        it = ctypes.c_uint32(0)
        check(self.L.slm_thin(ptr(self.select), ptr(self.scratch), self.shape[0], self.shape[1], 10000,
                              ptr(self.flag), ctypes.byref(it), self._stream()))
        self.flag_op(2, 0, info.is_thinchannel, select=self.select)
        # map_channel_heads
        self.flag_op(0, info.is_thinchannel, info.is_channelhead)
        seeds, n = self.pick(mask=True, map=None)
        if n == 0:
            return False
        self.run("map_channel_heads", seeds, n, [self.mask, self.uv, m])
        self.count.zero_()
        self.link.zero_()
        # count_downchannels
        self.flag_op(1, info.is_thinchannel)
        seeds, n = self.pick(mask=True, map=m, flag=info.is_channelhead)
        if n == 0:
            return False
        self.run("count_downchannels", seeds, n, [self.mask, self.uv, m, self.count, self.link])
        if not self._flag_downchannels(True):
            return False
        if not do_map_segments:
            return True
        # label_confluences, then flag_downchannels three times
        seeds, n = self.pick(mask=True, map=m, flag=info.is_thinchannel)
        if n == 0:
            return False
        self.run("label_confluences", seeds, n, [self.mask, self.uv, self.slt_dn, m, self.count, self.link])
        if not (self._flag_downchannels(True) and self._flag_downchannels(False)
                and self._flag_downchannels(False)):
            return False
        # segment_channels with the relabelling
        self.label.zero_()
        seeds, n = self.pick(mask=True, map=m, flag=info.is_channelhead)
        if n == 0:
            return False
        self.run("segment_downchannels", seeds, n, [self.mask, self.uv, m, self.count, self.link, self.label])
        ws = torch.empty(int(self.L.slm_relabel_workspace(self.n)), dtype=torch.uint8, device=dev)
        nl = ctypes.c_uint32(0)
        check(self.L.slm_relabel(ptr(self.label), self.n, ptr(ws), ws.numel(), ctypes.byref(nl), self._stream()))
        del ws
        if nl.value == 0:
            return False
        self.channel_label = self.label.clone()
        # link_hillslopes, segment_hillslopes (seeds: not thin channel)
        seeds, n = self.pick(mask=True, map=m, flag=info.is_thinchannel, invert=True)
        if n == 0:
            return False
        self.run("hillslopes", seeds, n, [self.mask, self.uv, m, self.count, self.link])
        seeds, n = self.pick(mask=True, map=m, flag=info.is_thinchannel, invert=True)
        if n == 0:
            return False
        self.run("segment_hillslopes", seeds, n, [self.mask, self.uv, m, self.count, self.link, self.label])
        # subsegment_flanks
        arrays = [self.mask, self.uv, m, self.channel_label, self.link, self.label]
        seeds, n = self.pick(mask=True, map=m, flag=info.is_subsegmenthead)
        if n == 0:
            return False
        self.run("subsegment_channel_edges", seeds, n, arrays)
        flag = int(info.is_leftflank) | int(info.is_thinchannel)
        for kernel in ("subsegment_flanks", "fix_right_flanks"):
            seeds, n = self.pick(mask=True, map=m, flag=flag, invert=True)
            if n == 0:
                return False
            self.run(kernel, seeds, n, arrays)
        seeds, n = self.pick(mask=True, map=m, flag=info.is_leftflank)
        if n == 0:
            return False
        self.run("fix_left_flanks", seeds, n, arrays)
        check(self.L.slm_signed_labels(ptr(self.label), self.n, int(info.left_flank_addition), self._stream()))
        return True

    def _flag_downchannels(self, reset_count):
        info = self.info
        self.flag_op(1, info.is_thinchannel)
        if reset_count:
            self.count.zero_()
        seeds, n = self.pick(mask=True, map=self.mapping, flag=info.is_channelhead)
        if n == 0:
            return False
        self.run("flag_downchannels", seeds, n, [self.mask, self.uv, self.mapping, self.count, self.link])
        return True

    def upload_mapping(self, mapping_array):
        """Replace the device mapping grid (e.g. after host-side midslope flags)."""
        self.mapping.copy_(torch.from_numpy(np.ascontiguousarray(mapping_array, dtype=np.uint32)).reshape(-1))

    def hsl(self, do_use_ridges=False):
        """Hillslope lengths of the midslope (or ridge) pixels; the float32
        array (doubled unless ridges), as ``mapping.hsl`` leaves it."""
        info = self.info
        flag = info.is_ridge if do_use_ridges else info.is_midslope
        seeds, n = self.pick(mask=True, map=self.mapping, flag=flag)
        out = torch.zeros(max(1, n), dtype=torch.float32, device=self.dev)
        if n:
            self.run("hillslope_lengths", seeds, n, [self.mask, self.uv, self.mapping, self.label, out])
        out = out[:n].cpu().numpy()
        if not do_use_ridges:
            out *= 2.0
        return out

    def download(self):
        """Copy the grids back into ``data`` (the arrays the host sequence fills)."""
        d, shape = self.data, self.shape
        grids = [self.mapping, self.count, self.link, self.label]
        if self.channel_label is not None:
            grids.append(self.channel_label)
        out = download(grids, "mapping")
        d.mapping_array = out[0].reshape(shape)
        d.count_array = out[1].reshape(shape)
        d.link_array = out[2].reshape(shape)
        d.label_array = out[3].view(np.int32).reshape(shape)
        if self.channel_label is not None:
            d.channel_label_array = out[4].reshape(shape)


def map_channels_segments_device(info, data, do_map_channels_from_scratch=True, do_map_segments=True,
                                 device=None):
    """``mapping.map_channels_segments`` with the grids resident on the GPU;
    same return value, same arrays in ``data``."""
    dm = DeviceMapping(info, data, device)
    with torch.cuda.device(dm.dev):
        ok = dm.map_channels_segments(do_map_channels_from_scratch, do_map_segments)
        dm.download()
    return ok, dm
