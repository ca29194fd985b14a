"""Learned trajectory-length scheduler for the field tracer.

The persistent field kernel hands trajectories to idle lanes in queue order.
A trajectory of a few thousand steps that starts near the end of the queue
keeps its warp (and the launch) running long after everything else has
finished; issuing the longest trajectories first removes that tail.  The
traced fields do not depend on the order (per-pixel sums are integers and each
trajectory's RNG stream follows its seed index), so any order is exact.

``LengthModel`` is a small BF16 CNN that predicts, from the 16x16 uv patch
around a seed pixel, log(1 + RK steps) of the seed's downstream and upstream
trajectories:

    conv1 4x4/4  2 -> 32 channels + ReLU   (16 tiles)
    conv2 2x2/2 32 -> 64 channels + ReLU   (4 positions)
    dense 256 -> 2

Operands are rounded to bfloat16 and accumulated in fp32.  Training runs on
the GPU through this library's GEMM / ReLU / MSE / Adam kernels on fp32
master weights (bf16-rounded working copies, straight-through rounding in the
backward pass); inference is one fused tensor-core kernel (``slm_cnn_infer``)
and ``slm_order_by_prediction`` bins the predictions into the ``seed_order``
of ``slm_integrate_fields_scheduled``.  The training targets are the per-
trajectory step counts the tracer itself records (``item_steps``).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib, kernels
from ._lib import check, ptr

# name -> shape, in the order of the flat parameter vector
SHAPES = (("w1", (32, 32)), ("b1", (32,)), ("w2", (128, 64)), ("b2", (64,)),
          ("w3", (256, 2)), ("b3", (2,)))
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
N_BINS = 1024


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _views(flat):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = flat[o:o + k].view(*shape)
        o += k
    return out


def bf16_round(x):
    """Round-to-nearest-even to bfloat16, returned as float32 (torch)."""
    return x.to(torch.bfloat16).to(torch.float32)


def init_params(seed=0):
    """He-normal weights and zero biases (fp32, NumPy), bfloat16-rounded."""
    rng = np.random.default_rng(seed)
    out = {}
    for name, shape in SHAPES:
        if name.startswith("w"):
            out[name] = (rng.standard_normal(shape) * math.sqrt(2.0 / shape[0])).astype(np.float32)
        else:
            out[name] = np.zeros(shape, np.float32)
    return out


def step_targets(item_steps, n_seeds, density, reduce="mean"):
    """Per-seed training target log(1 + RK steps) of its d*d trajectories
    (their mean or, ``reduce="max"``, the longest)."""
    dd = int(density) ** 2
    s = item_steps[: n_seeds * dd].view(n_seeds, dd).to(torch.float32)
    s = s.amax(dim=1) if reduce == "max" else s.mean(dim=1)
    return torch.log1p(s)


class LengthModel:
    """CNN weights on one device with their training state."""

    def __init__(self, device=None, params=None, seed=0):
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        p = params if params is not None else init_params(seed)
        flat = np.concatenate([np.asarray(p[n], np.float32).ravel() for n, _ in SHAPES])
        self.master = torch.from_numpy(flat).to(self.device)
        self.work = bf16_round(self.master)
        self.grad = torch.zeros_like(self.master)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.step_count = 0
        self.W = _views(self.work)
        self.G = _views(self.grad)
        self._bufs = {}
        self.L = _lib.load()
        # bit 0: a tensor-core GEMM's wait ran out (checked by check_status)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def check_status(self):
        """Raise if any training GEMM since the last check gave up waiting for
        its tensor-core work (its outputs are then incomplete)."""
        st = int(self.status.item())
        if st:
            self.status.zero_()
            raise RuntimeError("tensor-core GEMM status {:#x}: a wait for the MMAs ran out".format(st))

    # ------------------------------------------------------------ persistence
    def state(self):
        return {n: t.detach().cpu().numpy().copy() for n, t in _views(self.master).items()}

    def save(self, path):
        np.savez(path, **self.state())

    @classmethod
    def load(cls, path, device=None):
        with np.load(path) as z:
            return cls(device, {n: z[n] for n, _ in SHAPES})

    # ------------------------------------------------------------ buffers
    def _buf(self, name, shape):
        b = self._bufs.get(name)
        n = int(np.prod(shape))
        if b is None or b.numel() < n:
            b = torch.empty(n, dtype=torch.float32, device=self.device)
            self._bufs[name] = b
        return b[:n].view(*shape)

    def _gemm(self, ta, tb, M, N, K, A, B, C, Z=None, bias=None, relu=0, rnd=0, split=0, stream=None):
        partial = self._buf("split_k", (int(split) * int(M) * int(N),)) if split > 0 else None
        check(self.L.slm_gemm(int(ta), int(tb), int(M), int(N), int(K), ptr(A), ptr(B), ptr(C), ptr(Z),
                              ptr(bias), int(relu), int(rnd), int(split), ptr(partial), ptr(self.status),
                              _stream(stream)))

    @staticmethod
    def _split(M, N, K):
        tiles = ((M + 63) // 64) * ((N + 63) // 64)
        return int(max(1, min((K + 255) // 256, max(1, 296 // tiles))))

    # ------------------------------------------------------------ training
    def gather(self, uv, nxp, nyp, pad, seeds, index, n, stream=None):
        """conv1 input rows [n*16][32] for the seeds seeds[index[i]] (index may be None)."""
        x1 = self._buf("x1", (n * 16, 32))
        check(self.L.slm_cnn_gather(ptr(uv), int(nxp), int(nyp), int(pad), ptr(seeds), ptr(index), int(n),
                                    ptr(x1), _stream(stream)))
        return x1

    def forward(self, x1, n, stream=None):
        """Training forward pass (activations kept for backward); returns y [n][2]."""
        W = self.W
        z1, a1 = self._buf("z1", (n * 16, 32)), self._buf("a1", (n * 16, 32))
        self._gemm(0, 0, n * 16, 32, 32, x1, W["w1"], a1, z1, W["b1"], 1, 1, stream=stream)
        x2 = self._buf("x2", (n * 4, 128))
        check(self.L.slm_cnn_rearrange(ptr(a1), int(n), ptr(x2), 0, _stream(stream)))
        z2, a2 = self._buf("z2", (n * 4, 64)), self._buf("a2", (n * 4, 64))
        self._gemm(0, 0, n * 4, 64, 128, x2, W["w2"], a2, z2, W["b2"], 1, 1, stream=stream)
        y = self._buf("y", (n, 2))
        self._gemm(0, 0, n, 2, 256, a2, W["w3"], y, None, W["b3"], 0, 0, stream=stream)
        return y

    def backward(self, dy, x1, n, stream=None):
        """Gradients of the loss w.r.t. the (bf16-rounded) weights into self.grad."""
        W, G = self.W, self.G
        self.grad.zero_()
        a2, z2, x2, z1 = self._bufs["a2"], self._bufs["z2"], self._bufs["x2"], self._bufs["z1"]
        a2, z2 = a2[: n * 256].view(n, 256), z2[: n * 256].view(n * 4, 64)
        x2, z1 = x2[: n * 512].view(n * 4, 128), z1[: n * 512].view(n * 16, 32)
        s = _stream(stream)
        self._gemm(1, 0, 256, 2, n, a2, dy, G["w3"], split=self._split(256, 2, n), stream=stream)
        check(self.L.slm_bias_grad(ptr(dy), n, 2, ptr(G["b3"]), s))
        da2 = self._buf("da2", (n * 4, 64))
        self._gemm(0, 1, n, 256, 2, dy, W["w3"], da2, stream=stream)
        check(self.L.slm_relu_backward(ptr(da2), ptr(z2), n * 256, ptr(da2), s))
        self._gemm(1, 0, 128, 64, n * 4, x2, da2, G["w2"], split=self._split(128, 64, n * 4), stream=stream)
        check(self.L.slm_bias_grad(ptr(da2), n * 4, 64, ptr(G["b2"]), s))
        dx2 = self._buf("dx2", (n * 4, 128))
        self._gemm(0, 1, n * 4, 128, 64, da2, W["w2"], dx2, stream=stream)
        da1 = self._buf("da1", (n * 16, 32))
        check(self.L.slm_cnn_rearrange(ptr(dx2), int(n), ptr(da1), 1, s))
        check(self.L.slm_relu_backward(ptr(da1), ptr(z1), n * 512, ptr(da1), s))
        self._gemm(1, 0, 32, 32, n * 16, x1, da1, G["w1"], split=self._split(32, 32, n * 16), stream=stream)
        check(self.L.slm_bias_grad(ptr(da1), n * 16, 32, ptr(G["b1"]), s))
        return {k: t for k, t in G.items()}

    def loss_and_grad(self, x1, target, n, weight=None, stream=None):
        """(Weighted) MSE loss (device scalar) and gradients for one batch;
        ``weight`` [n][2] or None, normalised by the caller."""
        y = self.forward(x1, n, stream)
        dy = self._buf("dy", (n, 2))
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        check(self.L.slm_mse(ptr(y), ptr(target), ptr(weight), n * 2, ctypes.c_float(1.0 / (n * 2)), ptr(dy),
                             ptr(loss), _stream(stream)))
        self.backward(dy, x1, n, stream)
        return loss

    def adam(self, lr=2e-3, b1=0.9, b2=0.999, eps=1e-8, stream=None):
        self.step_count += 1
        check(self.L.slm_adam(ptr(self.master), ptr(self.work), ptr(self.grad), ptr(self.m), ptr(self.v),
                              N_PARAMS, ctypes.c_float(lr), ctypes.c_float(b1), ctypes.c_float(b2),
                              ctypes.c_float(eps), int(self.step_count), 1, _stream(stream)))

    def fit(self, uv, nxp, nyp, pad, seeds, targets, steps=600, batch=4096, lr=2e-3, seed=0,
            weights=None, stream=None):
        """Adam on random batches of (seed patch, targets [n][2], optional
        per-target weights [n][2] with mean 1); returns the loss history."""
        n = int(targets.shape[0])
        g = torch.Generator(device=self.device)
        g.manual_seed(int(seed))
        hist = []
        for it in range(int(steps)):
            idx = torch.randint(0, n, (batch,), device=self.device, generator=g, dtype=torch.int64)
            idx32 = idx.to(torch.int32)
            x1 = self.gather(uv, nxp, nyp, pad, seeds, idx32, batch, stream)
            t = targets.index_select(0, idx).contiguous()
            w = weights.index_select(0, idx).contiguous() if weights is not None else None
            loss = self.loss_and_grad(x1, t, batch, w, stream)
            frac = it / max(1, steps - 1)
            self.adam(lr * 0.5 * (1.0 + math.cos(math.pi * frac)), stream=stream)
            hist.append(loss)
        out = torch.cat(hist).cpu().numpy()
        self.check_status()
        return out

    # ------------------------------------------------------------ inference
    def predict(self, uv, nxp, nyp, pad, seeds, n, out=None, visit=None, stream=None):
        """Fused tensor-core inference: predictions [n][2] (down, up).
        ``visit`` (uint32 [n], optional): the order the seeds are processed
        in, e.g. ``spatial_order(...)``, for cache locality of the patches."""
        W = self.W
        if out is None:
            out = torch.empty((n, 2), dtype=torch.float32, device=self.device)
        check(self.L.slm_cnn_infer(ptr(uv), int(nxp), int(nyp), int(pad), ptr(seeds), ptr(visit), int(n),
                                   ptr(W["w1"]), ptr(W["b1"]), ptr(W["w2"]), ptr(W["b2"]), ptr(W["w3"]),
                                   ptr(W["b3"]), ptr(out), _stream(stream)))
        return out

    def order(self, pred, col, hi, out=None, bins=None, stream=None):
        """Seed order (uint32 [n]), longest predicted first, for direction ``col``."""
        n = int(pred.shape[0])
        if out is None:
            out = torch.empty(n, dtype=torch.uint32, device=self.device)
        if bins is None:
            bins = torch.empty(N_BINS, dtype=torch.uint32, device=self.device)
        check(self.L.slm_order_by_prediction(ptr(pred), 2, int(col), n, ctypes.c_float(0.0),
                                             ctypes.c_float(hi), N_BINS, ptr(bins), ptr(out),
                                             _stream(stream)))
        return out


SPATIAL_BLOCK = 64


def spatial_order(seeds, n, nx, ny, block=SPATIAL_BLOCK, pred=None, col=0, threshold=0.0, out=None,
                  bins=None, stream=None):
    """Seed order by ``block`` x ``block`` pixel block of the nx x ny grid
    (uint32 [n]); with ``pred`` [n][2], seeds predicted >= ``threshold`` first.

    Trajectories traced together then share cache lines of uv / mask /
    slc / slt: on grids larger than L2 this is what keeps the tracer
    compute-bound (the reference shuffles the seeds instead)."""
    L = _lib.load()
    dev = seeds.device
    n = int(n)
    nb = int(L.slm_order_spatial_bins(int(nx), int(ny), int(block), 1 if pred is not None else 0))
    if out is None:
        out = torch.empty(max(1, n), dtype=torch.uint32, device=dev)
    if bins is None or bins.numel() < nb:
        bins = torch.empty(max(1, nb), dtype=torch.uint32, device=dev)
    check(L.slm_order_spatial(ptr(seeds), n, int(nx), int(ny), int(block), ptr(pred), 2, int(col),
                              ctypes.c_float(threshold), ptr(bins), int(bins.numel()), ptr(out),
                              _stream(stream)))
    return out


def log_cap(params):
    """Upper end of the prediction range for a trace: log(1 + max_n_steps)."""
    return float(math.log1p(float(params.max_n_steps)))


def record_steps(params, seeds, mask, uv, work=None, schedule="persistent", integrator=2, stream=None):
    """Trace one direction and return per-trajectory RK step counts (uint16, queue order)."""
    nxy = int(params.nxy_padded)
    dev = seeds.device
    d = int(params.subpixel_seed_point_density)
    n_items = (int(params.n_seed_points) - int(params.seeds_chunk_offset)) * d * d
    slc = torch.zeros(nxy, dtype=torch.uint64, device=dev)
    slt = torch.zeros(nxy, dtype=torch.uint64, device=dev)
    work = work if work is not None else kernels.workspace(dev)
    work.zero_()
    steps = torch.zeros(n_items, dtype=torch.uint16, device=dev)
    kernels.integrate_fields(params, seeds, mask, uv, slc, slt, work, schedule=schedule,
                             integrator=integrator, item_steps=steps, stream=stream)
    return steps


def warp_cost(steps, order, width=32):
    """Cost model of the plain (one thread per trajectory) kernel: each warp
    of ``width`` consecutive queue positions runs as long as its longest
    trajectory; returns the sum over warps, in steps."""
    s = np.asarray(steps, np.int64)[np.asarray(order, np.int64)]
    pad = (-s.size) % width
    s = np.concatenate([s, np.zeros(pad, np.int64)]).reshape(-1, width)
    return int(s.max(axis=1).sum())


def makespan(steps, order, lanes):
    """Lane-level list-scheduling model of the persistent kernel: trajectories
    (lengths ``steps`` [n]) handed in ``order`` to the first idle of ``lanes``
    lanes; returns the finishing time in steps.  Deterministic CPU proxy for
    the kernel's tail."""
    import heapq
    s = np.asarray(steps, np.int64)[np.asarray(order, np.int64)]
    if s.size <= lanes:
        return int(s.max(initial=0))
    h = list(np.zeros(lanes, np.int64))
    heapq.heapify(h)
    for x in s:
        t = heapq.heappop(h)
        heapq.heappush(h, t + int(x) + 1)
    return int(max(h))
