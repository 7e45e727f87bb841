#!/usr/bin/env python
"""Benchmark of the orbit-and-action hot path on B200.

Headline workload (config 2): axisymmetric Staeckel-fudge actions through the action finder for
1e6 disk-like particles in the Miyamoto-Nagai + NFW Multipole (lmax 8, 60 radial nodes), FP64.
One step = one batched action-finder call over the whole set of particles.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Engine arm: inputs resident in HBM; each step is timed with CUDA events on the launching stream,
with the L2 cache flushed (256 MB write) between steps; the max over ranks is reported.
`e2e` repeats the measurement through the public Python API with pinned host buffers (host->device
copy of the particles and device->host copy of the actions inside the timed region).
Multi-GPU: replicas (every rank processes its own 1e6-particle shard; weak scaling; no collective
on the data path -- only a barrier and a max-reduction of the timings).

Reference arm (--impl reference): the reference's own ActionFinderAxisymFudge (built from its
sources under oracle/_ref) on all host cores, OpenMP dynamic chunks of 64 as in its Python
binding, on the same workload; rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
METRIC = "actions/s & orbit-steps/s on 1xB200: mixed+MLP vs plain FP64 at rel err<=1e-6"
WORKLOAD = "config 2: Staeckel-fudge actions, 1e6 disk particles, MN+NFW Multipole lmax 8 / 60 nodes (ActionFinder)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--particles", type=int, default=1000000)
    ap.add_argument("--no-baseline", action="store_true", help="skip the CPU baseline (profiling runs)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ------------------------------------------------------------------------------------------
class ClockSampler:
    """samples nvidia-smi SM clocks and throttle reasons while the timed region runs"""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self, index=None):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.samples if len(r) >= 9 and (index is None or r[0] == str(index))]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",")]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# ------------------------------------------------------------------------------------------
def make_particles(n, seed, vcirc):
    from agama_b200 import workloads
    return workloads.disk_particles(n, vcirc, seed=seed)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle needs the reference sources)"}))
        return
    pot = ref.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    vc = lambda R: np.sqrt(R * pot.eval(np.column_stack([R, 0 * R, 0 * R]))[1][:, 0])
    pts = make_particles(args.particles, 3, vc)
    af = ref.ActionFinder(pot)
    cores = os.cpu_count()
    sample = min(args.particles, 200000)       # bounded sample of the workload per step
    for _ in range(args.warmup):
        af.actions(pts[:sample // 10], nthreads=cores)
    times = []
    for k in range(args.steps):
        sl = pts[(k * sample) % args.particles:][:sample]
        t0 = time.perf_counter()
        af.actions(sl, nthreads=cores)
        times.append(time.perf_counter() - t0)
    ms = 1000 * float(np.mean(times))
    value = sample / (ms / 1000)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "actions/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "particles_per_step": sample, "threads": cores},
        "cpu_baseline": {"value": value, "unit": "actions/s", "cores": cores, "kind": "reference",
                         "sample": "%d of the %d config-2 particles per step" % (sample, args.particles)},
        "e2e": {"value": value, "unit": "actions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cpu_baseline_line(pts):
    """the reference's CPU action finder on the host cores, on a bounded sample"""
    try:
        from oracle import ref
        if not ref.available():
            return None
        pot = ref.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
        af = ref.ActionFinder(pot)
        cores = os.cpu_count()
        sample = min(len(pts), 200000)
        af.actions(pts[:2000], nthreads=cores)
        t0 = time.perf_counter()
        af.actions(pts[:sample], nthreads=cores)
        dt = time.perf_counter() - t0
        return {"value": sample / dt, "unit": "actions/s", "cores": cores, "kind": "reference",
                "sample": "first %d of the config-2 particles, reference ActionFinderAxisymFudge, OpenMP" % sample}
    except Exception as e:   # the baseline is reported, never required
        return {"value": None, "unit": "actions/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "failed: %s" % e}


def run_engine(args):
    import torch
    import agama_b200
    from agama_b200 import _native
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    pot = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg2.coef"))
    af = agama_b200.ActionFinder(pot)          # focal-distance table built on the device
    vc = lambda R: np.sqrt(-R * pot.force(np.column_stack([R, 0 * R, 0 * R]))[:, 0])
    n = args.particles
    pts = make_particles(n, 3 + rank, vc)
    dpts = torch.tensor(pts, device=dev)
    act = torch.empty((n, 3), dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2 (126 MB)
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes_stream(stream)
    lib = _native.lib()
    hpts = agama_b200._dev_ptr(dpts)
    hact = agama_b200._dev_ptr(act)

    def step():
        agama_b200._native.check(lib.agama_evalActionsManyDevice(af.handle, n, hpts, hact, None, sptr))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler()
    if rank == 0:
        sampler.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        step()
        ends[k].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop(physical_gpu_index(local)) if rank == 0 else None
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(np.sum(per))
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = n * world * args.steps / (total_ms / 1000)
    ms_per_step = total_ms / args.steps

    # ---- end to end through the public API, pinned host buffers
    hp = torch.from_numpy(pts).pin_memory().numpy()
    af(hp[:1000])
    e2e_times = []
    for k in range(max(2, min(args.steps, 5))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = af(hp)
        e2e_times.append(time.perf_counter() - t0)
    e2e_ms = 1000 * float(np.mean(e2e_times))
    e2e_val = n * world / (e2e_ms / 1000)
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_val = n * world / (float(t.item()) / 1000)
    if rank == 0:
        # ---- roofline of the action kernels (FP64-pipe bound): executed FP64 flops per action
        # from an ncu capture of this workload; peak measured on this device
        import ctypes
        pk = ctypes.c_double(0)
        _native.check(lib.agama_measureFP64Throughput(ctypes.byref(pk)))
        flops_per_action = FLOPS_PER_ACTION_CFG2
        achieved = flops_per_action * n / (ms_per_step / 1000) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "actions/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded disk particles)",
            "config": {"workload": WORKLOAD, "particles_per_gpu": n, "mode": "plain FP64",
                       "l2": "flushed between steps (256 MB write)", "parallelism": "replicas x%d" % world},
            "e2e": {"value": e2e_val, "unit": "actions/s", "h2d_bytes_per_step": int(pts.nbytes),
                    "d2h_bytes_per_step": int(n * 3 * 8)},
            "gpu_launches": ACTION_LAUNCHES_PER_STEP * args.steps,
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": pk.value, "unit": "TFLOP/s",
                         "frac": achieved / pk.value if pk.value else None, "traffic": TRAFFIC_PER_LAUNCH_CFG2,
                         "peak_source": "measured FP64 FMA throughput of this device (agama_measureFP64Throughput)",
                         "flops_per_action": flops_per_action},
            "clocks": clocks,
            "cpu_baseline": None if args.no_baseline else cpu_baseline_line(pts),
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# kernels per action step: prepare, three root-search kinds, integrals
ACTION_LAUNCHES_PER_STEP = 5
# executed FP64 flops per action (dadd + dmul + 2 dfma summed over the five kernels, ncu, config-2
# workload) and DRAM bytes of one step for 1e6 particles
FLOPS_PER_ACTION_CFG2 = 26206.0
# dram read + write of one 200 000-particle launch (9.89 MB + 0.22 MB), scaled to 1e6 particles
TRAFFIC_PER_LAUNCH_CFG2 = 5 * (9.888256e6 + 0.220416e6)


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
