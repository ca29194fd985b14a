#!/usr/bin/env python3
"""Benchmark: trajectory steps/s and DTM Mpx/s of the trace + fields stages.

One step = the reference's Trace stage on one synthetic DTM: record the
trajectory-seed subsample down and up (Trajectories), then trace every pixel's
d*d jittered sub-pixel trajectories down and up accumulating slc/slt
(Fields).  Default workload: the 8192^2 DTM @ 1 m (fBm mountains, an alluvial
cone of slope 0.03 with +-0.3 m radial ridges, 5000 unfilled pits), d=2,
jitter +-0.5 px, RK4, step 0.1 px, max 20000 steps: 268 M field trajectories
per direction.

  value  steps/s of the fastest shipped form (both directions in one
         persistent launch, seeds in spatial queue order, the trajectory
         recorder beside it) with inputs resident in HBM: CUDA events around
         each step; the inputs exceed L2 and a 256 MiB buffer is written
         between steps
  arms   the field trace in other forms, on identical fields, both
         directions: `plain` is the reference's form (one thread per
         trajectory, one launch per direction, the reference's shuffled
         order); `plain_learned` that kernel in the learned scheduler's order;
         `pair_spatial` the value's form; `pair_learned_spatial` and
         `pair_learned` the persistent pair launch in learned orders.  The
         learned arms' time includes inference and ordering.  The model is
         trained here, on the GPU, on step counts the tracer records on a
         held-out DTM of the same family (another seed).
  e2e    the same metric through the public API (Trajectories + Fields) with
         the inputs in pinned host memory and the results read back per step
  roofline  the field kernel is issue-bound: warp instructions per RK step
         (profiles/k_fields_pair_fan4096_rk4.md) x this launch's steps / its
         CUDA-event time, against 148 SMs x 4 schedulers x the sampled SM
         clock.  Beside it: the algorithmic bytes (RK2 75 B, RK4 139 B per
         step) against the measured HBM copy peak; the profiled launch's DRAM
         and L2 bytes per RK step, scaled to this launch's steps, the L2 rate
         against the L2 peak ncu reports, and an L2-resident copy timed here
  cpu_baseline  the reference's CPU path on this host's cores, over a fixed
         stride of the shuffled seed list
  parity  the GPU traces that same strided seed list of the full-size DTM:
         slc/slt must equal the oracle's C restatement (this workload's
         integrator) bit for bit, and, with RK2 on the same DTM, the
         reference's own kernel compiled for the host (low 32 bits, which is
         what the reference keeps)

N>1 (torchrun): the tracer's queue is dealt to the ranks in chunks of 64 queue
positions, round robin, so every rank sweeps the whole grid in spatial order;
each rank accumulates its own uint64 slc/slt, then one NCCL all-reduce (sum)
combines them (integer sums: identical to one GPU).  Total work is fixed
(strong scaling).

`--impl reference` times the reference's own CPU implementation instead
(rank 0 only) on the same config: the oracle's C restatement of the RK4
workloads (RK4 has no counterpart in the reference), with the reference's
own kernels compiled for the host (oracle/_ref) timed on RK2 of the same DTM
beside it.  That process builds the seed list with NumPy, as the reference
does, and loads none of this repository's libraries.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

BYTES_PER_STEP = {2: 75, 4: 139}
N_SMS, SCHEDULERS_PER_SM = 148, 4
FIELD_PROFILE = os.path.join(ROOT, "profiles", "k_fields_pair_fan4096_rk4.md")
METRIC = "trajectory steps/s (trace+fields)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fp:
            pk = json.load(fp)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def field_profile():
    """Per-RK-step counters of one profiled k_fields_pair launch: the
    ``per_rk_step:`` JSON line of the ncu summary in profiles/, or None."""
    try:
        with open(FIELD_PROFILE) as fp:
            for ln in fp:
                if ln.startswith("per_rk_step:"):
                    return json.loads(ln.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload_config(wl):
    """The ``config`` of both arms' lines: the workload alone."""
    spec = wl.spec
    return {"workload": spec.name, "key": wl.key,
            "trajectories_per_direction": int(wl.info.n_seed_points) * spec.density ** 2,
            "trajectory_seeds": int(wl.n_traj),
            "l2": "inputs larger than L2; 256 MiB buffer written between timed steps"}


def _cpu_sample(wl, stride, sign, cores, integrator=None):
    """Fields pass over every stride-th shuffled seed on the host cores.

    The sampled seeds form their own list (their RNG streams follow their
    position in it).  The oracle's restatement counts the RK steps of that
    list; with the reference's RK2 the timed run is the reference's own kernel
    on the same list (bit-identical trajectories), otherwise the restatement.
    Returns (steps, seconds, kind)."""
    import oracle as O
    from slm_b200 import params as P
    integ = integrator or wl.spec.integrator
    sub = np.ascontiguousarray(wl.seeds[::stride])
    prm = P.kernel_params(wl.info, "INTEGRATE_FIELDS", sign)
    prm.n_seed_points = sub.shape[0]
    t0 = time.perf_counter()
    _, _, steps, _ = O.integrate_fields(prm, sub, wl.mask, wl.uv, integ, n_threads=cores)
    t = time.perf_counter() - t0
    if integ == 2 and O.ref_available("integrate_fields"):
        t0 = time.perf_counter()
        O.ref_integrate_fields(prm, sub, wl.mask, wl.uv, n_threads=cores)
        return steps, time.perf_counter() - t0, "reference"
    return steps, t, "port"


def _cpu_stride(wl, cores, target_s, integrator=None):
    n = int(wl.info.n_seed_points)
    probe = max(1, n // 512)
    _, t, _ = _cpu_sample(wl, probe, 1.0, cores, integrator)
    return max(1, int(probe * max(t, 1e-3) / target_s))


def _sample_text(wl, stride):
    n = int(wl.info.n_seed_points)
    return "every {}th shuffled seed ({} of {} seeds, {} sub-pixel trajectories each)".format(
        stride, (n + stride - 1) // stride, n, wl.spec.density ** 2)


def run_reference(args):
    """The reference's CPU implementation on this host, a bounded sample per step."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from slm_b200.workloads import Workload
    # the seed list the reference's way (NumPy's shuffle): no library of this
    # repository is loaded in this process
    wl = Workload(args.workload, seed_list="numpy")
    cores = os.cpu_count() or 1
    stride = _cpu_stride(wl, cores, 3.0)
    for _ in range(args.warmup):
        _cpu_sample(wl, stride * 16, 1.0, cores)
    tot_steps, tot_t, kind = 0, 0.0, "port"
    for _ in range(args.steps):
        for sign in (1.0, -1.0):
            s, t, kind = _cpu_sample(wl, stride, sign, cores)
            tot_steps += s
            tot_t += t
    v = tot_steps / tot_t
    sample = "fields down+up over " + _sample_text(wl, stride)
    what = ("the reference's integrate_fields kernel compiled for the host" if kind == "reference"
            else "the oracle's C restatement (RK{} has no counterpart in the reference)".format(
                wl.spec.integrator))
    line = {
        "impl": "reference", "metric": METRIC, "value": v,
        "unit": "steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_t / max(args.steps, 1), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded DTM; no dataset)",
        "config": workload_config(wl),
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": cores, "kind": kind,
                         "sample": sample, "what": what},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if wl.spec.integrator != 2:
        # the reference's own kernel, on RK2 over the same DTM and seed list
        try:
            import oracle as O
            if not O.ref_available("integrate_fields"):
                raise FileNotFoundError("oracle/_ref was not built")
            s2 = _cpu_stride(wl, cores, 3.0, integrator=2)
            st, tt = 0, 0.0
            for sign in (1.0, -1.0):
                s, t, k2 = _cpu_sample(wl, s2, sign, cores, integrator=2)
                st += s
                tt += t
            line["rk2_reference"] = {"value": st / tt, "unit": "steps/s", "cores": cores, "kind": k2,
                                     "sample": "RK2 fields down+up over " + _sample_text(wl, s2),
                                     "what": "the reference's integrate_fields kernel compiled for the host"}
        except Exception as e:  # noqa: BLE001 -- reported in the line
            line["rk2_reference"] = {"unavailable": str(e)}
    print(json.dumps(line), flush=True)
    return 0


def l2_copy_peak(dev, mib=24, launches=200):
    """Read + write bandwidth of an elementwise copy whose two buffers
    (2 x ``mib`` MiB) stay resident in L2: a CUDA graph of ``launches``
    copies, timed with CUDA events.  GB/s."""
    import torch
    a = torch.ones(mib << 18, dtype=torch.float32, device=dev)
    b = torch.empty_like(a)
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(3):
            torch.neg(a, out=b)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(launches):
            torch.neg(a, out=b)
    g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    g.replay()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3
    del g
    return 2.0 * a.numel() * 4 * launches / t / 1e9


def roofline_block(integrator, pair, steps_per_launch, t_launch, clocks, l2_peak):
    """The field kernel's roofline: issue rate first (what binds), then
    algorithmic bytes, DRAM traffic and L2 bytes."""
    hbm_peak, peak_kind = _peaks()
    bps = BYTES_PER_STEP[integrator]
    alg = steps_per_launch * bps
    kernel = "k_fields_pair<{}>".format(integrator) if pair else "k_fields_persistent<{}>".format(integrator)
    hbm = {"achieved": alg / t_launch / 1e9, "peak": hbm_peak, "unit": "GB/s",
           "frac": alg / t_launch / 1e9 / hbm_peak, "peak_source": peak_kind,
           "bytes_per_step": bps, "algorithmic_bytes_per_launch": alg}
    prof = field_profile()
    out = {"kernel": kernel, "launch_ms": 1e3 * t_launch, "rk_steps_per_launch": steps_per_launch}
    if prof is not None and int(prof.get("integrator", 0)) == integrator:
        mhz = clocks.get("sm_mhz") or prof.get("sm_mhz") or 1965.0
        peak_issue = N_SMS * SCHEDULERS_PER_SM * mhz * 1e6
        inst = prof["warp_inst"] * steps_per_launch / t_launch
        traffic = prof["dram_bytes"] * steps_per_launch
        out.update({"bound": "issue", "achieved": inst, "peak": peak_issue, "unit": "warp-inst/s",
                    "frac": inst / peak_issue, "traffic": traffic,
                    "peak_note": "148 SMs x 4 warp schedulers x median sampled SM clock ({:.0f} MHz)".format(mhz),
                    "source": "warp instructions, DRAM and L2 bytes per RK step of one profiled launch "
                              "({}: {}), scaled by this launch's RK steps".format(
                                  os.path.relpath(FIELD_PROFILE, ROOT), prof.get("case", "")),
                    "thread_inst_per_step": prof.get("thread_inst"),
                    "hbm_algorithmic": hbm,
                    "dram": {"achieved": traffic / t_launch / 1e9, "peak": hbm_peak, "unit": "GB/s",
                             "frac": traffic / t_launch / 1e9 / hbm_peak,
                             "bytes_per_step": prof["dram_bytes"]}})
        if prof.get("lts_bytes"):
            l2 = prof["lts_bytes"] * steps_per_launch / t_launch / 1e9
            l2_hw = prof.get("lts_peak_gbs")
            out["l2"] = {"achieved": l2, "peak": l2_hw, "unit": "GB/s",
                         "frac": l2 / l2_hw if l2_hw else None, "bytes_per_step": prof["lts_bytes"],
                         "peak_note": "the L2 peak ncu measures against (the profiled launch's L2 rate over its "
                                      "lts__t_bytes pct_of_peak_sustained_elapsed)",
                         "copy_probe_gbs": l2_peak,
                         "copy_probe_note": "an elementwise copy of 2 x 24 MiB resident in L2, timed in this run: "
                                            "what a plain streaming kernel reaches through L2"}
    else:
        out.update({"bound": "hbm", "achieved": hbm["achieved"], "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm["frac"], "traffic": None, "peak_source": peak_kind,
                    "note": "no profile of this integrator's launch: algorithmic bytes against the HBM peak"})
        out["hbm_algorithmic"] = hbm
    return out


def run_b200(args):
    import torch
    import torch.distributed as dist

    from slm_b200 import kernels
    from slm_b200.params import kernel_params
    from slm_b200.workloads import Workload

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = Workload(args.workload)
    spec = wl.spec
    info = wl.info
    integrator = spec.integrator
    n_seeds = int(info.n_seed_points)
    nxy = int(info.nx_padded * info.ny_padded)

    seeds_d = torch.from_numpy(wl.seeds).to(dev)
    mask_d = torch.from_numpy(wl.mask.view(np.uint8)).to(dev)
    uv_d = torch.from_numpy(wl.uv).to(dev)
    acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=dev)
    work = [kernels.workspace(dev) for _ in range(2)]
    n_traj = wl.n_traj
    nl = int(info.max_n_steps)
    traj_d = torch.zeros(n_traj * nl * 2, dtype=torch.int8, device=dev)
    nsteps_d = torch.zeros((2, n_traj), dtype=torch.uint16, device=dev)
    length_d = torch.zeros((2, n_traj), dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    from slm_b200.distributed import allreduce_counts, shard_positions, shard_queue_params
    field_prm = [kernel_params(info, "INTEGRATE_FIELDS", s) for s in (1.0, -1.0)]
    queue_d = None
    if ws > 1:
        # this rank's dealt share of the queue: chunks of 64 queue positions,
        # round robin over the ranks
        mine = torch.from_numpy(shard_positions(n_seeds, rank, ws)).to(dev)
        field_prm = [shard_queue_params(p, int(mine.numel())) for p in field_prm]
        queue_d = mine.to(torch.int32).view(torch.uint32).contiguous()
    tinfo = wl.fresh_info()
    tinfo.n_seed_points = n_traj
    traj_prm = [kernel_params(tinfo, "INTEGRATE_TRAJECTORY", np.float32(s)) for s in (1.0, -1.0)]
    stream = torch.cuda.current_stream()
    sides = [torch.cuda.Stream(), torch.cuda.Stream()]
    traj_d2 = torch.zeros_like(traj_d)
    from slm_b200.scheduler import spatial_order
    spatial = args.seed_order == "spatial"
    pair = args.schedule == "persistent" and not args.no_pair
    order_d = torch.empty(max(1, n_seeds), dtype=torch.uint32, device=dev)
    bins_d = torch.empty(int(kernels._lib.load().slm_order_spatial_bins(
        int(info.nx), int(info.ny), 64, 0)), dtype=torch.uint32, device=dev)

    def device_step(ev=None):
        # the trajectory recorder (1000 seeds, latency-bound) runs on two side
        # streams, one per direction, concurrently with the field passes
        acc.zero_()
        fork = torch.cuda.Event()
        fork.record(stream)
        joins = []
        for d, side in enumerate(sides):
            side.wait_event(fork)
            kernels.integrate_trajectory(traj_prm[d], n_traj, seeds_d, mask_d, uv_d,
                                         traj_d if d == 0 else traj_d2, nsteps_d[d],
                                         length_d[d], integrator, stream=side)
            joins.append(torch.cuda.Event())
            joins[-1].record(side)
        if ev is not None:
            ev[0].record(stream)
        if spatial:
            spatial_order(seeds_d, n_seeds, info.nx, info.ny, out=order_d, bins=bins_d)
        queue = order_d if spatial else None
        if queue_d is not None:
            if spatial:
                torch.index_select(order_d.view(torch.int32), 0, mine, out=queue_d.view(torch.int32))
            queue = queue_d
        if pair:
            # acc[d, k]: rows of the [slc|slt] arrays; upstream 2*nxy further
            kernels.integrate_fields_pair(field_prm[0], field_prm[1], seeds_d, mask_d, uv_d, acc[:, 0],
                                          acc[:, 1], work[0], integrator=integrator,
                                          block_threads=args.block_threads, blocks_per_sm=args.blocks_per_sm,
                                          chunk=args.chunk, order=queue)
        else:
            for d in range(2):
                kernels.integrate_fields(field_prm[d], seeds_d, mask_d, uv_d, acc[d, 0], acc[d, 1],
                                         work[d], schedule=args.schedule, integrator=integrator,
                                         order=queue)
        if ev is not None:
            ev[1].record(stream)
        for join in joins:
            stream.wait_event(join)
        if ws > 1:
            allreduce_counts(acc)

    def count_steps():
        f = sum(int(w[1].view(torch.int64).item()) for w in work)
        t = int(nsteps_d.to(torch.int32).sum().item())
        return f, t

    for w in work:
        w.zero_()
    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    field_steps_rank, traj_steps = count_steps()
    times, ktimes = [], []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            if ws > 1:
                dist.barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            device_step((k0, k1))
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            ktimes.append(k0.elapsed_time(k1) / 1e3)
    step_t = float(np.sum(times))
    kern_t = float(np.sum(ktimes))
    if ws > 1:
        t = torch.tensor([step_t, kern_t], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_t, kern_t = float(t[0]), float(t[1])
        fs = torch.tensor([field_steps_rank], dtype=torch.int64, device=dev)
        dist.all_reduce(fs, op=dist.ReduceOp.SUM)
        field_steps = int(fs.item())
    else:
        field_steps = field_steps_rank
    steps_per_step = field_steps + traj_steps
    value = steps_per_step * args.steps / step_t
    ms = 1e3 * step_t / args.steps
    clk = clocks.summary()
    launches_per_step = 1 if pair else 2
    l2_peak = l2_copy_peak(dev) if ws == 1 else None
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded DTM; no dataset)",
        "config": workload_config(wl),
        "form": {"schedule": args.schedule,
                 "seed_order": "spatial (64 px blocks, ordered inside the timed step)"
                 if spatial else "shuffled (the reference's)",
                 "directions": "one launch for both" if pair else "one launch each",
                 "launch": {"block_threads": args.block_threads, "blocks_per_sm": args.blocks_per_sm,
                            "chunk": args.chunk},
                 "trajectory_recorder": "{} seeds down and up on side streams".format(n_traj),
                 "parallelism": "dealt seed shards + NCCL all-reduce" if ws > 1 else "1 GPU"},
        "mpx_per_s": wl.n_pixels / (step_t / args.steps) / 1e6,
        "rk_steps_per_step": steps_per_step,
        "field_rk_steps_per_step": field_steps,
        "roofline": roofline_block(integrator, pair, field_steps_rank // launches_per_step,
                                   kern_t / args.steps / launches_per_step, clk, l2_peak),
        "clocks": clk,
        "gpu_launches": args.steps * ((3 if spatial else 0) + 2 + launches_per_step),
    }
    if ws == 1 and not args.no_sched:
        line["arms"] = arms_compare(args, wl, dev, seeds_d, mask_d, uv_d, field_prm, flush)
    if ws == 1 and not args.no_e2e:
        line["e2e"] = run_e2e(args, wl, dev)
    if ws == 1 and args.stages:
        line["stages"] = run_stages(args, wl, dev)
    if rank == 0 and not args.no_cpu and ws == 1:
        line["cpu_baseline"], line["parity"] = cpu_and_parity(wl, args, dev, mask_d, uv_d)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def SPECS_NAME(key):
    from slm_b200.workloads import SPECS
    return SPECS[key].name


ARMS_DEFAULT = "plain,plain_learned,pair_spatial,pair_learned_spatial,pair_learned"
ARMS_ALL = ("plain", "plain_learned", "plain_spatial", "pair_shuffled", "pair_spatial",
            "pair_learned", "pair_learned_spatial")


def arms_compare(args, wl, dev, seeds_d, mask_d, uv_d, field_prm, flush):
    """The field trace of both directions in several forms on identical
    trajectories (the fields of every arm must equal the first arm's):

      plain                 k_fields_plain, one launch per direction, the
                            reference's shuffled order: the reference's form
      plain_learned         k_fields_plain, each direction in the learned
                            order (longest predicted first)
      plain_spatial         k_fields_plain, spatial order
      pair_shuffled         k_fields_pair (both directions, one persistent
                            launch), shuffled order
      pair_spatial          k_fields_pair, spatial order (the value's form)
      pair_learned          k_fields_pair, each direction longest predicted
                            first
      pair_learned_spatial  k_fields_pair, each direction's predicted-long
                            class first, then spatial order

    The length model is trained here, on the GPU, on the step counts the
    tracer records on a held-out DTM of the same family (another seed); the
    learned arms' time includes inference and ordering."""
    import torch

    from slm_b200 import kernels, scheduler as S
    from slm_b200.workloads import Workload

    t0 = time.time()
    spec = wl.spec
    d = spec.density
    from slm_b200.params import kernel_params
    arm_names = [a for a in args.arms.split(",") if a]
    for a in arm_names:
        if a not in ARMS_ALL:
            raise ValueError("unknown arm " + a)
    learned = any("learned" in a for a in arm_names)

    def recorded(w):
        """(uv, seeds, targets [n][2]) of workload w on the device."""
        sd = torch.from_numpy(w.seeds).to(dev)
        md = torch.from_numpy(w.mask.view(np.uint8)).to(dev)
        ud = torch.from_numpy(w.uv).to(dev)
        n_w = int(w.info.n_seed_points)
        cols = []
        for s in (1.0, -1.0):
            prm = kernel_params(w.info, "INTEGRATE_FIELDS", s)
            st = S.record_steps(prm, sd, md, ud, integrator=w.spec.integrator)
            cols.append(S.step_targets(st, n_w, w.spec.density))
        return w.uv, w.seeds[:n_w], torch.stack(cols, 1).contiguous()

    n = int(wl.info.n_seed_points)
    nxp, nyp = uv_d.shape[0], uv_d.shape[1]
    out = {"arms": arm_names, "ms": {}}
    model = pred = None
    long_thr = None
    if learned:
        if args.workload == "incised4096_d4":
            # 40 seeded 512^2 DTMs of the same family, 4x4 seeds: 10.5 M pairs.
            # Their uv grids are stacked along x with an 8 px edge-replicated
            # margin each, so a patch clamps exactly as on its own grid.
            train_keys = [("incised512_d4", 100 + i) for i in range(40)]
            held_keys = [("incised512_d4", 200 + i) for i in range(4)]
        else:
            train_keys = [(args.workload, args.sched_train_seed)]
            held_keys = []
        grids, seed_sets, tsets = [], [], []
        xoff = 0
        for key, seed in train_keys:
            g_uv, g_seeds, g_t = recorded(Workload(key, seed=seed))
            m = 8 if len(train_keys) > 1 else 0
            grids.append(np.pad(g_uv, ((m, m), (m, m), (0, 0)), mode="edge"))
            seed_sets.append(g_seeds + np.array([xoff + m, m], np.float32))
            tsets.append(g_t)
            xoff += grids[-1].shape[0]
        tr_uv = torch.from_numpy(np.ascontiguousarray(np.concatenate(grids, 0))).to(dev)
        tr_seeds = torch.from_numpy(np.ascontiguousarray(np.concatenate(seed_sets, 0))).to(dev)
        targets = torch.cat(tsets, 0).contiguous()
        del grids, seed_sets, tsets
        n_tr = int(targets.shape[0])
        # "predicted long" class of the learned+spatial order: the top 1% of
        # the training targets
        g = torch.Generator(device=dev)
        g.manual_seed(0)
        sub = targets[torch.randint(0, n_tr, (min(n_tr, 1 << 20),), device=dev, generator=g)]
        long_thr = [float(torch.quantile(sub[:, c], 0.99)) for c in (0, 1)]
        model = S.LengthModel(dev, seed=0)
        torch.cuda.synchronize()
        t1 = time.time()
        hist = model.fit(tr_uv, tr_uv.shape[0], tr_uv.shape[1], 2, tr_seeds, targets,
                         steps=args.sched_train_steps, batch=4096)
        torch.cuda.synchronize()
        t_train = time.time() - t1
        del tr_seeds, tr_uv, targets
        pred = model.predict(uv_d, nxp, nyp, 2, seeds_d, n)

        def error_of(p_all, truth_all):
            rank = lambda x: torch.argsort(torch.argsort(x)).double()
            out_e = {}
            for col in (0, 1):
                p, truth = p_all[:, col], truth_all[:, col]
                rho = float(torch.corrcoef(torch.stack([rank(p), rank(truth)]))[0, 1])
                out_e["down" if col == 0 else "up"] = {
                    "mae_log_steps": float((p - truth).abs().mean()), "spearman": rho}
            return out_e

        held = {}
        for key, seed in held_keys:
            h_uv, h_seeds, h_t = recorded(Workload(key, seed=seed))
            hu = torch.from_numpy(h_uv).to(dev)
            hs = torch.from_numpy(np.ascontiguousarray(h_seeds)).to(dev)
            hp = model.predict(hu, hu.shape[0], hu.shape[1], 2, hs, int(hs.shape[0]))
            held["{} seed {}".format(key, seed)] = error_of(hp, h_t)
        truth = torch.stack([S.step_targets(S.record_steps(field_prm[c], seeds_d, mask_d, uv_d,
                                                           integrator=spec.integrator), n, d)
                             for c in (0, 1)], 1)
        trained_on = ("40 x {} (seeds 100..139)".format(SPECS_NAME("incised512_d4"))
                      if args.workload == "incised4096_d4"
                      else "{} (seed {})".format(spec.name, args.sched_train_seed))
        out.update({"trained_on": trained_on, "held_out_dtms": held,
                    "train_pairs": n_tr, "train_steps": args.sched_train_steps, "train_batch": 4096,
                    "train_s": t_train, "prep_s": t1 - t0,
                    "loss_first": float(np.mean(hist[:10])), "loss_last": float(np.mean(hist[-50:])),
                    "held_out_error": error_of(pred, truth),
                    "long_class_threshold_log_steps": long_thr})
        del truth
    cap = S.log_cap(field_prm[0])
    orders = [torch.empty(n, dtype=torch.uint32, device=dev) for _ in range(2)]
    bins = torch.empty(S.N_BINS, dtype=torch.uint32, device=dev)
    nxy = int(field_prm[0].nxy_padded)
    acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=dev)
    work = [kernels.workspace(dev) for _ in range(2)]
    stream = torch.cuda.current_stream()
    sbins = torch.empty(int(kernels._lib.load().slm_order_spatial_bins(
        int(wl.info.nx), int(wl.info.ny), S.SPATIAL_BLOCK, 1)), dtype=torch.uint32, device=dev)
    visit = torch.empty(n, dtype=torch.uint32, device=dev)
    nx, ny = wl.info.nx, wl.info.ny

    def arm(name):
        acc.zero_()
        for w in work:
            w.zero_()
        if "learned" in name:
            # inference visits the seeds in spatial order (patch locality)
            S.spatial_order(seeds_d, n, nx, ny, out=visit, bins=sbins)
            model.predict(uv_d, nxp, nyp, 2, seeds_d, n, out=pred, visit=visit)
        if name.endswith("_learned"):
            for col in (0, 1):
                model.order(pred, col, cap, out=orders[col], bins=bins)
        elif name.endswith("_learned_spatial"):
            for col in (0, 1):
                S.spatial_order(seeds_d, n, nx, ny, pred=pred, col=col, threshold=long_thr[col],
                                out=orders[col], bins=sbins)
        elif name.endswith("_spatial"):
            S.spatial_order(seeds_d, n, nx, ny, out=orders[0], bins=sbins)
        if name in ("plain", "pair_shuffled"):
            o_dn = o_up = None
        elif "learned" in name:
            o_dn, o_up = orders[0], orders[1]
        else:
            o_dn = o_up = orders[0]
        if name.startswith("plain"):
            for col, o in ((0, o_dn), (1, o_up)):
                kernels.integrate_fields(field_prm[col], seeds_d, mask_d, uv_d, acc[col, 0], acc[col, 1],
                                         work[col], schedule="plain", integrator=spec.integrator, order=o)
        else:
            kernels.integrate_fields_pair(field_prm[0], field_prm[1], seeds_d, mask_d, uv_d, acc[:, 0],
                                          acc[:, 1], work[0], integrator=spec.integrator, order=o_dn,
                                          order_up=o_up)

    ref = None
    for name in arm_names:
        arm(name)
        torch.cuda.synchronize()
        res = (acc.clone(), int(work[0][1].item()) + int(work[1][1].item()))
        if ref is None:
            ref = res
        elif not (torch.equal(res[0], ref[0]) and res[1] == ref[1]):
            raise RuntimeError("the {} arm's fields differ from the {} arm's".format(name, arm_names[0]))
        ts = []
        for _ in range(args.arm_reps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            arm(name)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        out["ms"][name] = float(np.median(ts))
    f_steps = ref[1]
    out["field_steps"] = f_steps
    out["steps_per_s"] = {k: f_steps / (v / 1e3) for k, v in out["ms"].items()}
    if "plain" in out["ms"]:
        out["vs_plain"] = {k: out["ms"]["plain"] / v for k, v in out["ms"].items() if k != "plain"}
    learned_ms = {k: v for k, v in out["ms"].items() if "learned" in k}
    if learned_ms and "plain" in out["ms"]:
        best = min(learned_ms, key=learned_ms.get)
        out["learned_vs_plain"] = {"arm": best, "speedup": out["ms"]["plain"] / learned_ms[best]}
    if learned_ms and "pair_spatial" in out["ms"]:
        best = min(learned_ms, key=learned_ms.get)
        out["learned_vs_pair_spatial"] = {"arm": best,
                                          "speedup": out["ms"]["pair_spatial"] / learned_ms[best]}
    out["identical_fields"] = True
    out["l2"] = "256 MiB buffer written before each timed run"
    return out


def run_batched(args):
    """Batched form: ``--tiles`` fBm tiles of uneven sizes (edges log-uniform in
    256..3072 px), 2x2 jittered seeds, RK2, step 0.1 px, max 2000 steps, both
    directions.  Times, on identical fields: one plain (thread per trajectory)
    launch per tile and direction; one persistent launch per tile and
    direction; one batched persistent launch per direction with the
    autotuned shape; the same captured in a CUDA graph (the headline)."""
    import torch

    from slm_b200 import autotune, batch

    import torch.distributed as dist
    ws, rank, local = _dist()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    t0 = time.time()
    all_tiles = batch.uneven_tiles(args.tiles, 256, 3072, seed=3, density=2, jitter=1.0, step=0.1,
                                   max_steps=2000)
    t_gen = time.time() - t0
    # whole tiles per rank (no collective on the data path)
    sizes = [int(t.info.nx) * int(t.info.ny) for t in all_tiles]
    tiles = [all_tiles[i] for i in batch.shard_tiles(sizes, rank, ws)]
    b = batch.TileBatch(tiles, dev, integrator=2)
    n_px = sum(sizes)
    sample = batch.TileBatch(tiles[:12], dev, integrator=2)
    launch, table = autotune.tune(lambda L: sample.trace(L), "k_fields_batched", 2,
                                  "uneven fBm tiles, d=2, RK2, 12-tile sample",
                                  force=args.retune)
    del sample
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return ts

    b.trace(launch)
    torch.cuda.synchronize()
    ref = b.acc.clone()
    steps = b.field_steps()
    forms = {}
    for name, fn in (("per_tile_plain", lambda: b.trace_per_tile("plain")),
                     ("per_tile_persistent", lambda: b.trace_per_tile("persistent")),
                     ("batched", lambda: b.trace(launch))):
        fn()
        torch.cuda.synchronize()
        if not torch.equal(b.acc, ref):
            raise RuntimeError(name + " fields differ from the batched launch")
        forms[name] = float(np.median(timed(fn, max(1, args.steps // 2))))
    g = b.capture(launch)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    with ClockSampler(local) as clocks:
        times = timed(g.replay, args.steps)
    if not torch.equal(b.acc, ref):
        raise RuntimeError("graph replay differs from the eager trace")
    step_t = float(np.sum(times))
    if ws > 1:
        t = torch.tensor([step_t], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_t = float(t[0])
        st = torch.tensor([steps], dtype=torch.int64, device=dev)
        dist.all_reduce(st, op=dist.ReduceOp.SUM)
        steps = int(st.item())
        del g
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return 0
    forms["batched_graph"] = step_t / args.steps
    peak, peak_kind = _peaks()
    bps = BYTES_PER_STEP[2]
    line = {
        "metric": "trajectory steps/s (fields, batched tiles)", "value": steps * args.steps / step_t,
        "unit": "steps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * step_t / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fBm tiles; no dataset)",
        "config": {"workload": "{} fBm tiles, edges log-uniform 256..3072 px, d=2 jitter +-0.5, RK2, "
                               "step 0.1 px, max 2000 steps, both directions".format(args.tiles),
                   "tiles": args.tiles, "pixels": n_px, "trajectories_per_direction": b.n_seeds * 4,
                   "rk_steps_per_step": steps, "mpx_per_s": n_px / (step_t / args.steps) / 1e6,
                   "l2": "256 MiB buffer written between steps", "generation_s": t_gen,
                   "launch": {"block_threads": launch.block_threads,
                              "blocks_per_sm": launch.blocks_per_sm},
                   "autotune_ms": table,
                   "parallelism": "whole tiles per rank ({} ranks)".format(ws) if ws > 1 else "1 GPU"},
        "forms_ms": {k: 1e3 * v for k, v in forms.items()},
        "forms_steps_per_s": {k: steps / v for k, v in forms.items()},
        "batched_vs_per_tile_plain": forms["per_tile_plain"] / forms["batched_graph"],
        "roofline": {"bound": "hbm", "achieved": steps * bps / forms["batched_graph"] / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": steps * bps / forms["batched_graph"] / 1e9 / peak,
                     "traffic": None, "peak_source": peak_kind, "kernel": "k_fields_batched<2>",
                     "bytes_per_step": bps},
        "clocks": clocks.summary(),
        "gpu_launches": args.steps * 2,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_stages(args, wl, dev):
    """Every stage of the path on the workload DTM through the public API, each
    timed (wall clock, synchronised; the mapping wrappers copy their buffers
    per kernel call as the reference's do), then the same mapping and KDE
    with the oracle's CPU restatement on identical inputs: the CPU timing, and
    a full-size parity check (mapping bit-exact, KDE within the tests'
    tolerance)."""
    import copy

    import torch

    import oracle as O
    from slm_b200 import kde as K
    from slm_b200 import mapping
    from slm_b200.analysis import Bivariate_distribution, Univariate_distribution
    from slm_b200.fields import Fields
    from slm_b200.trajectories import Trajectories
    from slm_b200.useful import Data

    spec = wl.spec
    out = {}

    def timed(key, fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        out[key] = time.perf_counter() - t
        return r

    # preprocess: the workload's DTM -> conditioned uv through the public API
    from slm_b200.preprocess import conditioned_gradient_vector_field
    conditioned_gradient_vector_field(wl.dtm.astype(np.float32), spec.pixel_size, 2, device=dev)
    pre = timed("preprocess_s", lambda: conditioned_gradient_vector_field(wl.dtm.astype(np.float32),
                                                                           spec.pixel_size, 2, device=dev))
    out["preprocess_loop_pixels"] = int(pre.n_loops)

    info = wl.fresh_info()
    data = Data(info=info, mask_array=wl.mask, uv_array=wl.uv,
                mapping_array=np.zeros(wl.mask.shape, np.uint32))
    tr = Trajectories(0, dev.index, info=info, data=data, integrator=spec.integrator)
    timed("trajectories_s", tr.integrate)
    info2 = wl.fresh_info()
    data2 = Data(info=info2, mask_array=wl.mask, uv_array=wl.uv,
                 mapping_array=np.zeros(wl.mask.shape, np.uint32), traj_stats_df=tr.data.traj_stats_df)
    f = Fields(0, dev.index, info=info2, data=data2, integrator=spec.integrator)
    timed("fields_s", f.integrate)
    # the reference's channel-threshold search on the dslt pdf (reported; the
    # mapping below keeps the 94th percentile so its timings stay comparable)
    from slm_b200.analysis import estimate_channel_threshold
    thr_kde = timed("channel_threshold_s", lambda: estimate_channel_threshold(data2, pixel_size=spec.pixel_size))
    out["channel_threshold_kde"] = None if thr_kde is None else float(thr_kde)
    slt_dn = data2.slt_array[:, :, 0]
    thr = np.float32(np.percentile(slt_dn[~wl.mask], 94.0))
    out["channel_threshold_p94"] = float(thr)
    info2.set_thresholds(segmentation_threshold=np.uint32(50), channel_threshold=thr)
    cpu_data = copy.deepcopy(data2)
    cpu_info = copy.deepcopy(info2)

    from slm_b200.mapping_device import map_channels_segments_device
    resident = copy.deepcopy(data2)
    res_info = copy.deepcopy(info2)
    ok_res, _ = timed("mapping_device_resident_s",
                      lambda: map_channels_segments_device(res_info, resident, device=dev))
    runner = mapping.DeviceRunner(dev)
    ok = timed("mapping_s", lambda: mapping.map_channels_segments(None, info2, data2, runner=runner))
    out["mapping_device_resident_identical"] = bool(ok_res == ok) and all(
        np.array_equal(getattr(resident, k), getattr(data2, k))
        for k in ("mapping_array", "count_array", "link_array", "label_array", "channel_label_array"))
    del resident

    cpu_status = [0]

    def oracle_runner(name, params, seeds, arrays):
        # status bits (1: a loop the reference leaves unbounded hit its cap;
        # 2: an out-of-grid read skipped) are compared with the GPU's
        cpu_status[0] |= O.map_kernel(name, params, seeds, arrays)

    cpu = args.stages_cpu
    if cpu:
        t = time.perf_counter()
        ok_cpu = mapping.map_channels_segments(None, cpu_info, cpu_data, runner=oracle_runner)
        out["mapping_cpu_s"] = time.perf_counter() - t
        same = bool(ok == ok_cpu)
        for name in ("mapping_array", "count_array", "link_array", "label_array", "channel_label_array"):
            a, b = getattr(data2, name, None), getattr(cpu_data, name, None)
            if a is not None or b is not None:
                same = same and a is not None and b is not None and np.array_equal(a, b)
        out["mapping_identical"] = same
    out["mapping_status"] = {"gpu": int(runner.status), "cpu_oracle": int(cpu_status[0]) if cpu else None}
    out["mapping_kernels_s"] = {k: round(v, 4) for k, v in runner.seconds.items()}
    m = data2.mapping_array
    out["channel_pixels"] = int(np.sum((m & info2.is_thinchannel) > 0))
    out["segments"] = int(data2.label_array.max()) if ok else 0

    # hillslope lengths from a seeded 2 % of the hillslope pixels
    rng = np.random.default_rng(3)
    hill = (~wl.mask) & ((m & info2.is_thinchannel) == 0)
    pick = hill & (rng.random(hill.shape) < 0.02)
    for dd_, ii in ((data2, info2), (cpu_data, cpu_info)):
        dd_.mapping_array[pick] |= ii.is_midslope
        nmid = int(np.sum(~wl.mask & ((dd_.mapping_array & ii.is_midslope) > 0)))
        dd_.subsegment_hsl_array = np.zeros(nmid, dtype=np.float32)
    timed("hillslope_lengths_s", lambda: mapping.hsl(None, info2, data2, False, runner=runner))
    out["hillslope_lengths"] = int(data2.subsegment_hsl_array.size)
    if cpu:
        t = time.perf_counter()
        mapping.hsl(None, cpu_info, cpu_data, False, runner=oracle_runner)
        out["hillslope_lengths_cpu_s"] = time.perf_counter() - t
        out["hillslope_lengths_identical"] = bool(np.array_equal(
            data2.subsegment_hsl_array.view(np.uint32), cpu_data.subsegment_hsl_array.view(np.uint32)))

    # KDEs: hillslope lengths (univariate, 8192 bins -> 1024 points, gaussian,
    # bandwidth 2) and downstream vs upstream slt (bivariate)
    hsl = data2.subsegment_hsl_array
    logx = np.log(hsl[hsl > 0]).astype(np.float32)
    ud = Univariate_distribution(logx_array=logx, logy_array=logx, pixel_size=spec.pixel_size,
                                 n_hist_bins=8192, n_pdf_points=1024)
    timed("kde_univariate_s", lambda: ud.compute_kde_opencl(kernel="gaussian", bandwidth=2.0))
    prm = K.kde_params(ud, "pdf_univariate")
    dat = np.ascontiguousarray(ud.logx_data.reshape(-1), dtype=np.float32)
    t = time.perf_counter()
    h_o = O.histogram_univariate(prm, dat)
    p_o = O.pdf_univariate(prm, h_o)
    out["kde_univariate_cpu_s"] = time.perf_counter() - t
    h_o = h_o.reshape(-1, 1)
    p_o = p_o.reshape(-1, 1)
    out["kde_univariate_hist_identical"] = bool(np.array_equal(ud.histogram, h_o / (np.sum(h_o) * ud.bin_dx)))
    p_ref = p_o / (np.sum(p_o) * ud.bin_dx)
    out["kde_univariate_max_rel_err"] = float(np.max(np.abs(ud.pdf - p_ref)) / np.max(np.abs(p_ref)))
    sl = data2.slt_array
    sel = (~wl.mask) & (sl[:, :, 0] > 0) & (sl[:, :, 1] > 0)
    with np.errstate(divide="ignore"):  # log(0) outside the selection, replaced below
        lx, ly = np.log(sl[:, :, 0]), np.log(sl[:, :, 1])
    lx[~sel] = np.finfo(np.float32).min
    ly[~sel] = np.finfo(np.float32).min
    bd = Bivariate_distribution(logx_array=lx, logy_array=ly, mask_array=wl.mask,
                                pixel_size=spec.pixel_size, n_hist_bins=1024, n_pdf_points=256)
    timed("kde_bivariate_s", lambda: bd.compute_kde_opencl(kernel="gaussian", bandwidth=0.1))
    out["kde_bivariate_points"] = int(bd.n_data)

    # the Mapping stage's passes 1 and 2 with the grids on the GPU: the
    # coarse channels at the 94th-percentile threshold, then per coarse
    # subsegment its KDE threshold, fine channels, the hillslope lengths (by
    # fast marching, the reference's measurement; then, on a fresh stage,
    # traced along streamlines) and their statistics
    import types

    from slm_b200 import analysis as A
    from slm_b200.mapping_stage import Mapping
    from slm_b200.useful import default_parameters
    dflt = default_parameters()
    state = types.SimpleNamespace(**vars(dflt.state))
    state.reset_active_masks = lambda: None
    state.merge_active_masks = lambda: wl.mask.copy()
    state.add_active_mask = lambda item: None
    trace_ns = types.SimpleNamespace(**vars(wl.defaults.trace))
    trace_ns.slc_array, trace_ns.slt_array, trace_ns.sla_array = data2.slc_array, data2.slt_array, data2.sla_array
    geodata = types.SimpleNamespace(roi_nx=spec.n, roi_ny=spec.n, pad_width=2, roi_pixel_size=spec.pixel_size)
    def new_stage():
        return Mapping(state, {"mapping": dict(coarse_channel_threshold=float(thr),
                                               coarse_segmentation_threshold=200)},
                       geodata, types.SimpleNamespace(uv_array=wl.uv), trace_ns,
                       analysis=A.Analysis(state, None, geodata, None, trace_ns), device=dev)
    stage = new_stage()
    timed("mapping_pass1_s", stage.pass1)
    timed("mapping_pass2_s", lambda: stage.pass2(hsl_method="fmm"))
    out["mapping_coarse_subsegments"] = int(stage.n_coarse_subsegments)
    out["mapping_passes_status"] = int(stage.engine.status)
    out["mapping_pass2_subsegments_with_lengths"] = int(len(stage.hsl_mean_array))
    out["mapping_pass2_hsl_pixels"] = int((stage.hsl_array > 0).sum())
    traced = new_stage()
    traced.pass1()
    timed("mapping_pass2_traced_s", lambda: traced.pass2(hsl_method="traced"))
    out["mapping_pass2_traced_subsegments_with_lengths"] = int(len(traced.hsl_mean_array))
    out["ok"] = bool(ok)
    return out


PREPROCESS_BYTES_PER_PX = 4 + 8 + 4 + 1 + 1 + 1 + 1 + 1 + 4 + 4  # roi in; uv, slope, 2 masks, 3 codes, 2 gradients


def run_preprocess(args):
    """DTM -> conditioned uv (slm_preprocess) on the workload's DTM: kernel time
    with the ROI resident (CUDA events, L2 flushed between launches), the public
    API from a host ROI to host arrays, and the oracle's NumPy restatement on
    the host (full grid up to 2048^2, else a band of rows), checked identical."""
    import ctypes

    import torch

    import dtm_preprocess as DP
    from slm_b200 import _lib
    from slm_b200.preprocess import conditioned_gradient_vector_field as cgvf
    from slm_b200.workloads import SPECS, make_dtm

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    spec = SPECS[args.workload]
    roi = np.ascontiguousarray(make_dtm(spec), np.float32)
    nx, ny = roi.shape
    pad = 2
    L = _lib.load()
    roi_d = torch.from_numpy(roi).to(dev)
    f32, u8 = torch.float32, torch.uint8
    uv = torch.empty((nx + 2 * pad, ny + 2 * pad, 2), dtype=f32, device=dev)
    slope = torch.empty(uv.shape[:2], dtype=f32, device=dev)
    uvm, mask = (torch.empty(uv.shape[:2], dtype=u8, device=dev) for _ in range(2))
    blk, nbr, cells = (torch.empty((nx, ny), dtype=u8, device=dev) for _ in range(3))
    gx, gy = (torch.empty((nx, ny), dtype=f32, device=dev) for _ in range(2))
    ncell = torch.zeros(1, dtype=torch.int32, device=dev)
    prm = _lib.SlmPreprocessParams(spec.pixel_size, 0.95, -0.5, 0.0, pad, 1)
    stream = torch.cuda.current_stream(dev)
    P = _lib.ptr

    def launch():
        _lib.check(L.slm_preprocess(P(roi_d), 0, nx, ny, ctypes.byref(prm), P(uv), P(slope), P(uvm), P(mask),
                                    P(blk), P(nbr), P(cells), P(gx), P(gy), P(ncell),
                                    ctypes.c_void_p(stream.cuda_stream)))

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    for _ in range(max(3, args.warmup)):
        launch()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(0) as clocks:
        for _ in range(max(args.steps, 20)):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            launch()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
    kt = float(np.median(times))
    n_loops = 4 * int(ncell.item())
    # public API: host ROI in, host arrays out
    cgvf(roi, spec.pixel_size, pad, device=dev)
    t0 = time.perf_counter()
    for _ in range(3):
        r = cgvf(roi, spec.pixel_size, pad, device=dev)
    e2e_s = (time.perf_counter() - t0) / 3
    # the oracle on the host, and the identity check
    rows = nx if nx * ny <= 2048 * 2048 else 1024
    band = roi[:rows]
    t0 = time.perf_counter()
    o = DP.conditioned_uv(band, spec.pixel_size, pad)
    cpu_s = time.perf_counter() - t0
    keep = rows + pad - 2 if rows < nx else rows + 2 * pad  # band rows unaffected by its lower edge
    same = all(np.array_equal(np.asarray(a)[:keep].view(np.uint8), np.asarray(b)[:keep].view(np.uint8))
               for a, b in ((r.uv_array, o["uv_array"]), (r.uv_mask_array, o["uv_mask_array"])))
    same &= all(np.array_equal(getattr(r, k)[:rows - 2], o[k][:rows - 2])
                for k in ("blockages_array", "blocked_neighbors_array", "loop_cells"))
    peak, peak_kind = _peaks()
    bytes_launch = nx * ny * PREPROCESS_BYTES_PER_PX
    line = {
        "metric": "DTM preprocess (conditioned uv) Mpx/s", "value": nx * ny / kt / 1e6, "unit": "Mpx/s",
        "n_gpus": 1, "steps": len(times), "warmup": max(3, args.warmup), "ms_per_step": 1e3 * kt,
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded DTM; no dataset)",
        "config": {"workload": spec.name, "roi": [nx, ny], "pad_width": pad, "n_loops": n_loops,
                   "l2": "256 MiB buffer written between launches"},
        "roofline": {"bound": "hbm", "achieved": bytes_launch / kt / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bytes_launch / kt / 1e9 / peak, "traffic": None,
                     "algorithmic_bytes_per_launch": bytes_launch, "peak_source": peak_kind,
                     "kernel": "k_preprocess<float>"},
        "e2e": {"value": nx * ny / e2e_s / 1e6, "unit": "Mpx/s", "h2d_bytes_per_step": roi.nbytes,
                "d2h_bytes_per_step": int(r.uv_array.nbytes + r.slope_array.nbytes + 2 * r.mask_array.size
                                          + 3 * nx * ny + 2 * 4 * nx * ny)},
        "cpu_baseline": {"value": band.size / cpu_s / 1e6, "unit": "Mpx/s", "cores": 1, "kind": "port",
                         "sample": "{} of {} rows, the oracle's NumPy restatement".format(rows, nx)},
        "identical_to_oracle": bool(same),
        "gpu_launches": len(times),
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))
    return 0


def run_e2e(args, wl, dev):
    """Public-API step: Trajectories then Fields on pinned host arrays."""
    import torch

    from slm_b200.device import pinned_empty
    from slm_b200.fields import Fields
    from slm_b200.trajectories import Trajectories
    from slm_b200.useful import Data

    uv_h = pinned_empty(wl.uv.shape, np.float32)
    uv_h[...] = wl.uv
    mask_h = pinned_empty(wl.mask.shape, np.bool_)
    mask_h[...] = wl.mask
    integ = wl.spec.integrator

    def step():
        # as the Trace stage runs them: the fields' seed list and passes run
        # on a worker thread and a side stream (Fields.prepare) while the
        # trajectories run; integrate() then post-processes
        info2 = wl.fresh_info()
        data2 = Data(info=info2, mask_array=mask_h, uv_array=uv_h,
                     mapping_array=np.zeros(mask_h.shape, np.uint32))
        f = Fields(0, dev.index, info=info2, data=data2, schedule=args.schedule, integrator=integ)
        f.prepare()
        info = wl.fresh_info()
        data = Data(info=info, mask_array=mask_h, uv_array=uv_h,
                    mapping_array=np.zeros(mask_h.shape, np.uint32))
        tr = Trajectories(0, dev.index, info=info, data=data, integrator=integ)
        tr.integrate()
        data2.traj_stats_df = tr.data.traj_stats_df
        f.integrate()
        return tr.n_steps + sum(f.n_steps)

    step()
    torch.cuda.synchronize()
    k = max(1, args.e2e_steps)
    times = []
    n = 0
    for _ in range(k):
        t0 = time.perf_counter()
        n += step()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    t = float(np.sum(times))
    nxy = wl.mask.size
    n_seeds = int(wl.info.n_seed_points)
    # up: uv and mask for each stage, each stage's swap partners of the seed
    # shuffle (uint32 per seed; the lists themselves are built on the
    # device), the trajectory seeds
    h2d = wl.uv.nbytes * 2 + wl.mask.nbytes * 2 + 4 * n_seeds * 2 + wl.traj_seeds.nbytes
    # down: finished slc (float64), slt and sla (float32) per direction, the
    # field seed list (data.seed_point_array) and the trajectory seeds, the
    # trajectory step counts and lengths (recorded steps come back as well,
    # up to each trajectory's length)
    d2h = nxy * 2 * (8 + 4 + 4) + wl.seeds.nbytes + wl.traj_seeds.nbytes + wl.n_traj * 2 * (2 + 4)
    return {"value": n / t, "unit": "steps/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": k,
            "ms_per_step": 1e3 * t / k, "ms_min_max": [1e3 * min(times), 1e3 * max(times)],
            "mpx_per_s": wl.n_pixels * k / t / 1e6,
            "note": "Trajectories.integrate + Fields.prepare/integrate through the public API, as "
                    "the Trace stage runs them (the fields' seed list and passes on a worker thread "
                    "and a side stream while the trajectories run): seed creation and shuffle for "
                    "each (swap partners drawn on the host, swaps on the GPU), "
                    "uploads, tracing, the fields' post-processing (on the GPU), the seed list and "
                    "the finished arrays copied back, every step"}


def _trace_sub(prm, sub_d, mask_d, uv_d, integrator, dev):
    """Both directions of the seed list ``sub_d`` in one pair launch; returns
    (acc [2][2][nxy] uint64 on the host: direction, slc|slt; RK steps)."""
    import torch

    from slm_b200 import kernels
    nxy = int(prm[0].nxy_padded)
    acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=dev)
    work = kernels.workspace(dev)
    kernels.integrate_fields_pair(prm[0], prm[1], sub_d, mask_d, uv_d, acc[:, 0], acc[:, 1], work,
                                  integrator=integrator)
    torch.cuda.synchronize()
    return acc.cpu().numpy(), int(work[1].item())


def cpu_and_parity(wl, args, dev, mask_d, uv_d):
    """The reference's CPU path on a fixed stride of the shuffled seed list
    (the baseline), and the GPU's fields on that same list compared with the
    CPU's (parity at the workload's full DTM size).

    * restatement: both directions with the workload's integrator, the
      oracle's C restatement against one pair launch, slc and slt bit for bit
      (uint64) and the RK step count;
    * reference RK2: the same DTM with RK2, the reference's own
      integrate_fields kernel compiled for the host against the pair launch
      on a 4x sparser stride; the reference keeps uint32 sums, so the GPU's
      low 32 bits are compared."""
    import torch

    import oracle as O
    from slm_b200.params import kernel_params
    cores = os.cpu_count() or 1
    n = int(wl.info.n_seed_points)
    integ = wl.spec.integrator
    stride = wl.spec.cpu_stride or _cpu_stride(wl, cores, 10.0)

    def params_for(m):
        prm = [kernel_params(wl.info, "INTEGRATE_FIELDS", s) for s in (1.0, -1.0)]
        for p in prm:
            p.n_seed_points = m
        return prm

    sub = np.ascontiguousarray(wl.seeds[::stride])
    prm = params_for(sub.shape[0])
    cpu, t_dir = [], []
    for p in prm:
        t0 = time.perf_counter()
        cpu.append(O.integrate_fields(p, sub, wl.mask, wl.uv, integ, n_threads=cores))
        t_dir.append(time.perf_counter() - t0)
    base_steps, base_t, kind = cpu[0][2], t_dir[0], "port"
    if integ == 2 and O.ref_available("integrate_fields"):
        t0 = time.perf_counter()
        O.ref_integrate_fields(prm[0], sub, wl.mask, wl.uv, n_threads=cores)
        base_t, kind = time.perf_counter() - t0, "reference"
    baseline = {"value": base_steps / base_t, "unit": "steps/s", "cores": cores, "kind": kind,
                "sample": "downstream fields over {}, {:.1f} s".format(_sample_text(wl, stride), base_t)}

    sub_d = torch.from_numpy(sub).to(dev)
    g, g_steps = _trace_sub(prm, sub_d, mask_d, uv_d, integ, dev)
    same = all(np.array_equal(g[d, 0], cpu[d][0]) and np.array_equal(g[d, 1], cpu[d][1]) for d in (0, 1))
    parity = {"restatement": {
        "identical": bool(same and g_steps == cpu[0][2] + cpu[1][2]),
        "kind": "RK{}: pair launch vs the oracle's C restatement, slc and slt uint64 bit for bit, "
                "both directions, and the RK step count".format(integ),
        "stride": stride, "seeds": int(sub.shape[0]), "of_seeds": n,
        "trajectories": int(2 * sub.shape[0] * wl.spec.density ** 2), "rk_steps": g_steps,
        "pixels_compared": int(4 * g.shape[2])}}
    del sub_d
    if O.ref_available("integrate_fields"):
        s2 = stride * 4 if integ != 2 else stride
        sub2 = np.ascontiguousarray(wl.seeds[::s2])
        prm2 = params_for(sub2.shape[0])
        t0 = time.perf_counter()
        ref = [O.ref_integrate_fields(p, sub2, wl.mask, wl.uv, n_threads=cores) for p in prm2]
        t_ref = time.perf_counter() - t0
        sub2_d = torch.from_numpy(sub2).to(dev)
        g2, g2_steps = _trace_sub(prm2, sub2_d, mask_d, uv_d, 2, dev)
        low = (g2 & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        same2 = all(np.array_equal(low[d, 0], ref[d][0]) and np.array_equal(low[d, 1], ref[d][1])
                    for d in (0, 1))
        parity["reference_rk2"] = {
            "identical": bool(same2),
            "kind": "RK2 on the same DTM: pair launch vs the reference's own integrate_fields kernel "
                    "compiled for the host, slc and slt low 32 bits, both directions",
            "stride": s2, "seeds": int(sub2.shape[0]), "of_seeds": n,
            "trajectories": int(2 * sub2.shape[0] * wl.spec.density ** 2), "rk_steps": g2_steps,
            "reference_s": t_ref, "pixels_compared": int(4 * g2.shape[2])}
    else:
        parity["reference_rk2"] = {"identical": None,
                                   "unavailable": "oracle/_ref was not built (it needs the reference "
                                                  "checkout when the library is built)"}
    return baseline, parity


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fan8192")
    ap.add_argument("--schedule", default="persistent", choices=["plain", "persistent"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10, help="public-API steps timed for e2e")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and the parity check")
    ap.add_argument("--no-sched", action="store_true", help="skip the arms (plain / learned / spatial)")
    ap.add_argument("--arms", default=ARMS_DEFAULT,
                    help="comma-separated arms of the form comparison, from " + ",".join(ARMS_ALL))
    ap.add_argument("--arm-reps", type=int, default=2, help="timed runs per arm (median)")
    ap.add_argument("--seed-order", default="spatial", choices=["spatial", "shuffled"])
    ap.add_argument("--no-pair", action="store_true", help="one field launch per direction")
    ap.add_argument("--block-threads", type=int, default=0, help="pair launch: threads per block (0: default)")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="pair launch: resident blocks per SM (0: default)")
    ap.add_argument("--chunk", type=int, default=0, help="pair launch: refill threshold in idle lanes (0: default)")
    ap.add_argument("--preprocess", action="store_true",
                    help="time the DTM preprocessing (slm_preprocess) on the workload's DTM instead")
    ap.add_argument("--stages", action="store_true",
                    help="also time mapping, hillslope lengths and KDE on the GPU")
    ap.add_argument("--stages-cpu", action="store_true",
                    help="with --stages: the same stages with the CPU oracle, timed, and compared")
    ap.add_argument("--tiles", type=int, default=96, help="tiles96: number of tiles")
    ap.add_argument("--retune", action="store_true", help="tiles96: ignore the autotuner cache")
    ap.add_argument("--sched-train-seed", type=int, default=12)
    ap.add_argument("--sched-train-steps", type=int, default=1500)
    ap.add_argument("--profile-case", action="store_true",
                    help="run only the field pair launch of the workload --steps times and print its "
                         "RK steps per launch (the command profiled for the roofline counters)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.preprocess:
        return run_preprocess(args)
    if args.profile_case:
        return run_profile_case(args)
    if args.workload == "tiles96":
        return run_batched(args)
    return run_b200(args)


def run_profile_case(args):
    """The field pair launch alone (spatial order), --warmup + --steps times,
    for an ncu capture of one launch; prints RK steps per launch and the
    CUDA-event time of the last launch."""
    import torch

    from slm_b200 import kernels
    from slm_b200.params import kernel_params
    from slm_b200.scheduler import spatial_order
    from slm_b200.workloads import Workload
    dev = torch.device("cuda", 0)
    wl = Workload(args.workload)
    info = wl.info
    n = int(info.n_seed_points)
    nxy = int(info.nx_padded * info.ny_padded)
    seeds_d = torch.from_numpy(wl.seeds).to(dev)
    mask_d = torch.from_numpy(wl.mask.view(np.uint8)).to(dev)
    uv_d = torch.from_numpy(wl.uv).to(dev)
    acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=dev)
    work = kernels.workspace(dev)
    prm = [kernel_params(info, "INTEGRATE_FIELDS", s) for s in (1.0, -1.0)]
    order = spatial_order(seeds_d, n, info.nx, info.ny)
    steps, ms = [], []
    for _ in range(args.warmup + args.steps):
        acc.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        kernels.integrate_fields_pair(prm[0], prm[1], seeds_d, mask_d, uv_d, acc[:, 0], acc[:, 1], work,
                                      integrator=wl.spec.integrator, order=order)
        e1.record()
        torch.cuda.synchronize()
        steps.append(int(work[1].item()))
        ms.append(e0.elapsed_time(e1))
    print(json.dumps({"profile_case": wl.key, "workload": wl.spec.name, "launches": len(steps),
                      "rk_steps_per_launch": steps[-1], "steps_identical": len(set(steps)) == 1,
                      "ms": ms, "device_bytes": int(seeds_d.nbytes + mask_d.nbytes + uv_d.nbytes
                                                    + acc.nbytes + order.nbytes)}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
