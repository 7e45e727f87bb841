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
    ap.add_argument("--no-secondary", action="store_true", help="skip the force / orbit workloads")
    ap.add_argument("--profile-case", action="store_true",
                    help="run each workload's kernels once on a small case (for ncu instruction counts) and print "
                         "the units each launch processed")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(value, dist, device):
    """the largest of one value over all ranks (a step's time: the slowest replica sets the job's)"""
    if not dist:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
        "cpu_baseline": {"value": value, "unit": "actions/s", "cores": cores, "cpu_model": cpu_model(),
                         "kind": "reference",
                         "sample": "%d of the %d config-2 particles per step" % (sample, args.particles)},
        "e2e": {"value": value, "unit": "actions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "secondary": None if args.no_secondary else run_reference_secondary(),
    }))


def run_reference_secondary():
    """the secondary workloads on the reference's CPU code (bounded samples, all host cores)"""
    from oracle import ref

    class RefPot:
        def __init__(self, f):
            self.p = ref.Potential(file=f)

        def potential(self, x):
            return self.p.eval(x)[0]

        def force(self, x):
            return -self.p.eval(x)[1]
    from agama_b200 import workloads
    _, pts1, ic1, T1, _, ic3, T3 = secondary_workloads(RefPot, lambda c: os.path.join(GOLDEN, c + ".coef"))
    p5 = RefPot(os.path.join(GOLDEN, "cfg5.coef"))
    ic5, T5 = workloads.orbit_workload(5, p5.potential, p5.force, ORBIT5_ORBITS)
    names = [("force evals/s", "config 1 forces"), ("orbit-steps/s", "config 1 orbits"),
             ("orbit-steps/s", "config 3 orbits, at most %d steps per orbit" % ORBIT3_MAX_STEPS),
             ("orbit-steps/s", "config 5 orbits"), ("actions/s", "config 5 actions of the final snapshot")]
    return [dict(metric=m, value=b and b["value"], unit=b and b.get("unit"), config=c, cpu_baseline=b)
            for (m, c), (b, _) in zip(names, reference_secondary(pts1, ic1, T1, ic3, T3, ic5, T5))]


def cpu_baseline_line(pts, J=None):
    """the reference's CPU action finder on the host cores, on a bounded sample; with the engine's
    actions J of the same points, their largest relative difference from the reference's"""
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
        Jref = af.actions(pts[:sample], nthreads=cores)
        dt = time.perf_counter() - t0
        line = {"value": sample / dt, "unit": "actions/s", "cores": cores, "cpu_model": cpu_model(),
                "kind": "reference",
                "sample": "first %d of the config-2 particles, reference ActionFinderAxisymFudge, OpenMP" % sample}
        if J is not None:
            line["max_rel_err_vs_reference"] = rel_action_err(J[:sample], Jref)
        return line
    except Exception as e:   # the baseline is reported, never required
        return {"value": None, "unit": "actions/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "failed: %s" % e}


# ------------------------------------------------------------------------------------------
# Secondary workloads: the other headline throughputs of the path, measured in the same run.
#   config 1 forces:  1e5 points of the triaxial Dehnen Multipole (lmax 6, 50 nodes), potential
#                     and force per point                                   -> force evals/s
#   config 1 orbits:  1e4 orbits, T = 10 T_circ(E), DOP853 accuracy 1e-8     -> orbit-steps/s
#   config 3 orbits:  all 1e5 config-3 orbits (T = 10-1000 T_circ, Omega = 0.05), at most
#                     ORBIT3_MAX_STEPS accepted steps per orbit: the workload's tail (orbits near
#                     r ~ 1e3 whose T spans 1e4-1e6 turns of the rotating frame) needs up to 1e7
#                     steps per orbit, hours of integration on either arm   -> orbit-steps/s
ORBIT3_MAX_STEPS = 5000
#   config 5:         all 1e6 orbits (100 T_circ each) in the Spheroid + disk Multipole (lmax 12,
#                     80 nodes), then the actions of their final snapshot, plain FP64 and with
#                     learned root brackets
ORBIT5_ORBITS = 1000000
# bounded samples of each workload on which the reference's CPU code is timed and compared
REF_SAMPLE = {"orbits1": 2000, "orbits3": 400, "orbits5": 200, "actions5": 4000}


def cpu_model():
    """the host CPU's model name (for the cpu_baseline records)"""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def secondary_workloads(potential_cls, coef, n3=None):
    """inputs of the secondary workloads for a potential class with .potential / .force"""
    from agama_b200 import workloads
    pot1 = potential_cls(coef("cfg1"))
    pts1 = workloads.dehnen_positions(100000, 1.0, q=(0.8, 0.6), seed=workloads.SEEDS["points1"])
    ic1, T1 = workloads.orbit_workload(1, pot1.potential, pot1.force)
    pot3 = potential_cls(coef("cfg3"))
    ic3, T3 = workloads.orbit_workload(3, pot3.potential, pot3.force, n3)
    return pot1, pts1, ic1, T1, pot3, ic3, T3


def rel_action_err(J, Jref):
    """largest relative action error (the parity tests' measure: |dJ| / max(|J|, 1e-3 sum|J|)) and
    whether the NaN patterns (unbound points) agree"""
    J, Jref = np.asarray(J), np.asarray(Jref)
    ok = np.isfinite(Jref).all(1)
    tot = np.abs(Jref[ok]).sum(1, keepdims=True)
    e = np.abs(J[ok] - Jref[ok]) / np.maximum(np.abs(Jref[ok]), 1e-3 * tot)
    return {"max": float(e.max()) if e.size else 0.0, "q999": float(np.quantile(e, 0.999)) if e.size else 0.0,
            "points": int(len(Jref)), "nan_pattern_equal": bool(np.array_equal(np.isfinite(J), np.isfinite(Jref)))}


def orbit_deviation(final, status, final_ref, status_ref):
    """final points of the engine against the reference's on the same orbits: regular orbits agree
    to round-off growth (<= 1e-7 in the tests), chaotic ones diverge (that is their nature), so the
    distribution is given"""
    ok = (np.asarray(status) == 0) & (np.asarray(status_ref) == 0)
    d = np.linalg.norm(final[ok, :3] - final_ref[ok, :3], axis=1) / np.linalg.norm(final_ref[ok, :3], axis=1)
    return {"orbits": int(len(final)), "status_equal": float(np.mean(np.asarray(status) == np.asarray(status_ref))),
            "final_pos_rel_median": float(np.median(d)) if d.size else None,
            "final_pos_rel_p25": float(np.quantile(d, 0.25)) if d.size else None,
            "frac_le_1e-7": float(np.mean(d <= 1e-7)) if d.size else None}


def fp64_roofline(kernel, flops_per_unit, per, units, ms, peak, source):
    """roofline record of an FP64-pipe-bound workload: executed FP64 flops per unit (ncu count of
    dadd + dmul + 2 dfma of the kernel on this workload) x units / CUDA-event time"""
    achieved = flops_per_unit * units / (ms / 1000) / 1e12 if flops_per_unit else None
    return {"bound": "fp64", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak and achieved else None, "flops_per_unit": flops_per_unit, "per": per,
            "flops_source": source, "peak_source": "measured FP64 FMA throughput of this device"}


def run_engine_secondary(dev, flush, dist, cpu, peak64):
    """device-timed throughputs of the secondary workloads (max over ranks), with the reference
    on the host cores beside each when cpu is true"""
    import torch
    import agama_b200
    from agama_b200 import workloads

    class Pot(agama_b200.Potential):
        def __init__(self, f):
            super().__init__(file=f)
    pot1, pts1, ic1, T1, pot3, ic3, T3 = secondary_workloads(Pot, lambda c: os.path.join(GOLDEN, c + ".coef"))
    stream = torch.cuda.current_stream(dev)

    step_ms = {}

    def timed(fn, warmup, steps):
        import gc
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        gc.collect()            # no collection of the interpreter's heap inside a timed step
        gc.disable()
        try:
            for _ in range(steps):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                r = fn()
                b.record(stream)
                torch.cuda.synchronize()
                ms.append(a.elapsed_time(b))
        finally:
            gc.enable()
        step_ms["last"] = ms
        # the median of the steps: a single step held up outside the engine (a host stall of
        # ~10 ms was seen once in five steps on the config-5 snapshot) does not move it
        t = float(np.median(ms))
        t = max_over_ranks(t, dist, dev)
        return t, r

    out, mixed_lines, engine_res = [], [], {}
    d1 = torch.tensor(pts1, device=dev)
    t, (phi1, acc1) = timed(lambda: pot1.eval(d1, pot=True, acc=True), 3, 10)
    engine_res["forces1"] = (phi1.cpu().numpy(), acc1.cpu().numpy())
    out.append({"metric": "force evals/s", "value": len(pts1) / (t / 1000), "unit": "evals/s", "ms_per_step": t,
                "config": "config 1: 1e5 points, triaxial Dehnen Multipole lmax 6 / 50 nodes, potential + force",
                "steps": 10, "warmup": 3, "gpu_launches_per_step": 1,
                "roofline": fp64_roofline("evalPotentialKernel", FLOPS["forces1"], "evaluation", len(pts1), t, peak64,
                                          FLOPS_SOURCE)})
    for key, name, pot, ic, T, Om, mx, warm, steps in (
            ("orbits1", "config 1: 1e4 orbits x 10 T_circ, DOP853 1e-8", pot1, ic1, T1, 0.0, 0, 3, 5),
            ("orbits3", "config 3: all 1e5 orbits (10-1000 T_circ, Omega 0.05), DOP853 1e-8, at most %d steps per orbit"
             % ORBIT3_MAX_STEPS, pot3, ic3, T3, 0.05, ORBIT3_MAX_STEPS, 1, 2)):
        dic, dT = torch.tensor(ic, device=dev), torch.tensor(T, device=dev)
        # the batch is captured once in a CUDA graph (work-counter reset + persistent kernel, lanes
        # per orbit chosen by the autotuner before the capture) and replayed every step
        graph = agama_b200.OrbitGraph(pot, dic, dT, Omega=Om, maxNumSteps=mx)
        t, _ = timed(graph.launch, warm, steps)
        nst, nrej = int(graph.steps.sum().item()), int(graph.rejected.sum().item())
        status = graph.status.cpu().numpy()
        k = REF_SAMPLE[key]
        engine_res[key] = (graph.final[:k].cpu().numpy(), status[:k])
        line = {"metric": "orbit-steps/s", "value": nst / (t / 1000), "unit": "accepted DOP853 steps/s",
                "ms_per_step": t, "config": name, "steps": steps, "warmup": warm, "accepted_steps": nst,
                "rejected_attempts": nrej, "gpu_launches_per_step": 1, "launch": "CUDA graph",
                "lanes_per_orbit": graph.lanes, "block": graph.block,
                "roofline": fp64_roofline("dop853Kernel", FLOPS[key], "accepted step", nst, t, peak64, FLOPS_SOURCE)}
        if mx:
            line["orbits_at_step_cap"] = float(np.mean(status == 1))
        out.append(line)
        mixed_lines.append(mixed_orbit_entry(agama_b200, timed, pot, dic, dT, Om, mx, warm, steps, name, graph, t))
        del graph
    # config 5: all 1e6 orbits, then the actions of the final snapshot (plain and learned brackets)
    pot5 = Pot(os.path.join(GOLDEN, "cfg5.coef"))
    ic5, T5 = workloads.orbit_workload(5, pot5.potential, pot5.force, ORBIT5_ORBITS)
    dic5, dT5 = torch.tensor(ic5, device=dev), torch.tensor(T5, device=dev)
    graph5 = agama_b200.OrbitGraph(pot5, dic5, dT5)
    t5, _ = timed(graph5.launch, 1, 2)
    nst5 = int(graph5.steps.sum().item())
    engine_res["orbits5"] = (graph5.final[:REF_SAMPLE["orbits5"]].cpu().numpy(),
                             graph5.status[:REF_SAMPLE["orbits5"]].cpu().numpy())
    af5 = agama_b200.ActionFinder(pot5)
    snap = graph5.final.clone()
    lib = agama_b200._native.lib()
    import ctypes
    af5(snap)
    torch.cuda.synchronize()
    agama_b200._native.check(lib.agama_actionPhaseTiming(1, None, None))    # CUDA events around each phase
    ta, J5 = timed(lambda: af5(snap), 3, 5)
    ms5 = list(step_ms["last"])
    ph5, np5 = (ctypes.c_double * 4)(), ctypes.c_long(0)
    agama_b200._native.check(lib.agama_actionPhaseTiming(0, ph5, ctypes.byref(np5)))
    phase5 = {"prepare": ph5[0] / 8, "roots": ph5[2] / 8, "integrals": ph5[3] / 8}
    J5 = J5.clone()
    engine_res["actions5"] = (snap[:REF_SAMPLE["actions5"]].cpu().numpy(), J5[:REF_SAMPLE["actions5"]].cpu().numpy())
    out.append({"metric": "orbit-steps/s", "value": nst5 / (t5 / 1000), "unit": "accepted DOP853 steps/s",
                "ms_per_step": t5, "config": "config 5: all %d orbits x 100 T_circ, Spheroid + disk Multipole "
                "lmax 12 / 80 nodes, DOP853 1e-8 (FP64: one harmonic, so the FP32 m != 0 mode has nothing to do)"
                % ORBIT5_ORBITS, "steps": 2, "warmup": 1, "accepted_steps": nst5,
                "gpu_launches_per_step": 1, "launch": "CUDA graph", "lanes_per_orbit": graph5.lanes, "block": graph5.block,
                "roofline": fp64_roofline("dop853Kernel", FLOPS["orbits5"], "accepted step", nst5, t5, peak64,
                                          FLOPS_SOURCE)})
    line5 = {"metric": "actions/s", "value": ORBIT5_ORBITS / (ta / 1000), "unit": "actions/s", "ms_per_step": ta,
             "config": "config 5: actions of the final snapshot of those orbits (action finder, plain FP64)",
             "steps": 5, "warmup": 3, "gpu_launches_per_step": 3, "phase_ms": phase5, "ms_each_step": ms5,
             "roofline": fp64_roofline("fudge kernels (3)", FLOPS["actions5"], "action", ORBIT5_ORBITS, ta, peak64,
                                       FLOPS_SOURCE)}
    out.append(line5)
    # the mixed-precision and learned-bracket forms on the snapshot: the network trained on the
    # orbits' initial points (the same distribution, other points), then used on the final points
    t0 = time.perf_counter()
    af5.train_brackets(ic5[:1000000], epochs=20, batch=2048, lr=2e-3, seed=1)
    ttrain5 = time.perf_counter() - t0
    af5.use_brackets(False)

    def rel_err(J, Jref):
        e = rel_action_err(J.cpu().numpy(), Jref.cpu().numpy())
        return e["max"], e["q999"]
    out5 = action_mode_lines(agama_b200, timed_ms(timed), rel_err, af5, snap, J5,
                             "config 5: actions of the final snapshot of those orbits",
                             {"samples": 1000000, "epochs": 20, "seconds": ttrain5,
                              "points": "the orbits' initial points"})
    del graph5
    if cpu:
        for line, (base, parity) in zip(out, reference_secondary(pts1, ic1, T1, ic3, T3, ic5, T5, engine_res)):
            line["cpu_baseline"] = base
            if parity is not None:
                line["max_rel_err_vs_reference" if "max" in parity else "vs_reference"] = parity
    return out + out5 + mixed_lines


def timed_ms(timed):
    """the (time, result) timer of the secondary workloads as a time-only timer with 3 warm-up
    steps and 5 timed steps"""
    return lambda fn, warmup=3, steps=5: timed(fn, warmup, steps)[0]


def mixed_orbit_entry(agama_b200, timed, pot, dic, dT, Om, mx, warm, steps, name, graph64, t64):
    """the same orbit batch with the m != 0 harmonics of the force in FP32, with the error of
    every orbit stated: its Jacobi-energy error and its deviation from the FP64 batch"""
    import torch
    agama_b200.set_orbit_precision(True)
    try:
        graph = agama_b200.OrbitGraph(pot, dic, dT, Omega=Om, maxNumSteps=mx)
    finally:
        agama_b200.set_orbit_precision(False)
    t, _ = timed(graph.launch, warm, steps)
    nst = int(graph.steps.sum().item())
    ok = ((graph.status == 0) & (graph64.status == 0)).cpu().numpy()
    f32, f64 = graph.final.cpu().numpy()[ok], graph64.final.cpu().numpy()[ok]
    ic = dic.cpu().numpy()[ok]
    dev = np.linalg.norm(f32[:, :3] - f64[:, :3], axis=1) / np.linalg.norm(f64[:, :3], axis=1)
    e32 = agama_b200.jacobi_energy_error(pot, ic, f32, Om)
    e64 = agama_b200.jacobi_energy_error(pot, ic, f64, Om)
    q = lambda a: {"median": float(np.median(a)), "p90": float(np.quantile(a, 0.9)), "max": float(a.max())}
    line = {"metric": "orbit-steps/s", "value": nst / (t / 1000), "unit": "accepted DOP853 steps/s",
            "ms_per_step": t, "config": name + "; mixed precision (m != 0 harmonics in FP32)", "steps": steps,
            "warmup": warm, "accepted_steps": nst, "gpu_launches_per_step": 1, "launch": "CUDA graph",
            "lanes_per_orbit": graph.lanes, "fp64_ms_per_step": t64,
            "error_per_orbit": {"jacobi_energy_rel_mixed": q(e32), "jacobi_energy_rel_fp64": q(e64),
                                "position_rel_vs_fp64": q(dev), "orbits": int(ok.sum())}}
    del graph
    torch.cuda.synchronize()
    return line


def run_bracket_modes(dev, flush, dist, af2, dpts2, J2plain):
    """the actions with learned root brackets (BF16 tensor-core network choosing the brackets of
    the FP64 searches) beside the plain FP64 form, config 2 (same 1e6 particles as the headline)
    and config 4 (1e7 particles of the config-1 distribution in the config-1 potential made
    axisymmetric, network trained on 2e6 of the finder's own searches)"""
    import torch
    import agama_b200
    from agama_b200 import workloads
    stream = torch.cuda.current_stream(dev)

    def timed(fn, warmup=3, steps=5):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        t = float(np.mean(ms))
        t = max_over_ranks(t, dist, dev)
        return t

    def rel_err(J, Jref):
        J, Jref = J.cpu().numpy(), Jref.cpu().numpy()
        ok = np.isfinite(Jref).all(1)
        tot = np.abs(Jref[ok]).sum(1, keepdims=True)
        e = np.abs(J[ok] - Jref[ok]) / np.maximum(np.abs(Jref[ok]), 1e-3 * tot)
        return float(np.max(e)), float(np.quantile(e, 0.999))

    out = []
    vc2 = workloads.vcirc_from_force(lambda x: af2.potential.force(x))
    train2 = workloads.disk_particles(1000000, vc2, seed=33)
    t0 = time.perf_counter()
    af2.train_brackets(train2, epochs=20, batch=2048, lr=2e-3, seed=1)
    ttrain2 = time.perf_counter() - t0
    cases = [("config 2: 1e6 disk particles (the headline set)", af2, dpts2, J2plain, ttrain2, 1000000)]
    pot4 = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg4.coef"))
    af4 = agama_b200.ActionFinder(pot4)
    pos = workloads.dehnen_positions(2000000, 1.0, q=(0.8, 0.6), seed=workloads.SEEDS["particles4"])
    train4 = workloads.orbit_ics(pos, pot4.potential, seed=workloads.SEEDS["particles4"] + 1000)
    t0 = time.perf_counter()
    af4.train_brackets(train4, epochs=20, batch=2048, lr=2e-3, seed=1)
    ttrain4 = time.perf_counter() - t0
    pos = workloads.dehnen_positions(10000000, 1.0, q=(0.8, 0.6), seed=workloads.SEEDS["particles4"] + 1)
    ev4 = workloads.orbit_ics(pos, pot4.potential, seed=workloads.SEEDS["particles4"] + 2000)
    d4 = torch.tensor(ev4, device=dev)
    del pos, ev4
    af4.use_brackets(False)
    J4plain = af4(d4)
    cases.append(("config 4: 1e7 particles of the config-1 distribution, config-1 potential made axisymmetric "
                  "(lmax 6, 50 nodes)", af4, d4, J4plain, ttrain4, 2000000))
    for name, af, d, Jplain, ttrain, ntrain in cases:
        out += action_mode_lines(agama_b200, timed, rel_err, af, d, Jplain, name,
                                 {"samples": ntrain, "epochs": 20, "seconds": ttrain})
    return out


def action_mode_lines(agama_b200, timed, rel_err, af, d, Jplain, name, training):
    """the same action batch in its mixed-precision and learned-bracket forms beside the plain FP64
    one: mixed precision (FP32 integrand arithmetic and compensated sums), learned root brackets
    (BF16 tcgen05 network + FP64 searches), and both; each with its speed-up over plain FP64 and its error against it"""
    n = d.shape[0]
    out = []
    af.use_brackets(False)
    af.count_brackets(False)          # timings without the search counters (the plain kernel)
    tp = timed(lambda: af(d))
    af.count_brackets(True)
    af.bracket_stats(reset=True)
    af(d)
    plain = af.bracket_stats(reset=True)
    for mode, mixed, learned in (("mixed precision (FP32 integrands, compensated FP32 sums; FP64 potential and roots)",
                                  True, False),
                                 ("learned root brackets (BF16 tcgen05 network + FP64 searches)", False, True),
                                 ("mixed precision + learned root brackets", True, True)):
        agama_b200.set_action_precision(mixed)
        af.use_brackets(learned)
        try:
            af.count_brackets(False)
            tl = timed(lambda: af(d))
            af.count_brackets(True)
            af.bracket_stats(reset=True)
            J = af(d)
            st = af.bracket_stats(reset=True)
        finally:
            agama_b200.set_action_precision(False)
            af.use_brackets(False)
        emax, e999 = rel_err(J, Jplain)
        line = {"metric": "actions/s", "mode": mode, "value": n / (tl / 1000), "unit": "actions/s",
                "ms_per_step": tl, "config": name, "plain_fp64": {"value": n / (tp / 1000), "ms_per_step": tp},
                "speedup_vs_plain": tp / tl, "max_rel_err_vs_plain": emax, "rel_err_vs_plain_q999": e999,
                "steps": 5, "warmup": 3, "gpu_launches_per_step": 4 if learned else 3}
        if learned:
            line.update({"seeded_searches": st["narrowed"] / max(1, st["searches"]),
                         "fallback_rate": st["fallbacks"] / max(1, st["narrowed"]),
                         "root_iterations_vs_plain": st["iterations"] / max(1, plain["iterations"]),
                         "training": training})
        out.append(line)
    return out


def reference_secondary(pts1, ic1, T1, ic3, T3, ic5, T5, engine=None):
    """the reference's own CPU code on bounded samples of the secondary workloads, all host cores:
    (cpu_baseline, parity against the engine's results on the same sample) per workload, in the
    order forces, config-1 orbits, config-3 orbits, config-5 orbits, config-5 snapshot actions"""
    try:
        from oracle import ref
        if not ref.available():
            return [(None, None)] * 5
        cores, model = os.cpu_count(), cpu_model()
        base = lambda v, unit, sample: {"value": v, "unit": unit, "cores": cores, "cpu_model": model,
                                        "kind": "reference", "sample": sample}
        p1 = ref.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
        p3 = ref.Potential(file=os.path.join(GOLDEN, "cfg3.coef"))
        res = []
        p1.eval(pts1[:1000], nthreads=cores)
        t0 = time.perf_counter()
        phi, grad = p1.eval(pts1, nthreads=cores)
        dt = time.perf_counter() - t0
        parity = None
        if engine is not None:
            ephi, eacc = engine["forces1"]
            parity = {"max": float(max(np.max(np.abs(ephi - phi) / np.abs(phi)),
                                       np.max(np.linalg.norm(-eacc - grad, axis=1) / np.linalg.norm(grad, axis=1)))),
                      "of": "potential and force, relative", "points": len(pts1)}
        res.append((base(len(pts1) / dt, "evals/s", "all 1e5 config-1 points, potential + force, OpenMP"), parity))
        for key, pot, ic, T, Om, mx, what in (("orbits1", p1, ic1, T1, 0.0, 0, "config 1"),
                                              ("orbits3", p3, ic3, T3, 0.05, ORBIT3_MAX_STEPS, "config 3")):
            n = REF_SAMPLE[key]
            t0 = time.perf_counter()
            fin, steps, status = pot.orbits(ic[:n], T[:n], Omega=Om, maxSteps=mx, nthreads=cores)
            dt = time.perf_counter() - t0
            parity = orbit_deviation(*engine[key], fin, status) if engine is not None else None
            res.append((base(float(steps.sum()) / dt, "accepted DOP853 steps/s",
                             "first %d orbits of the %s workload, OpenMP dynamic 1" % (n, what)), parity))
        p5 = ref.Potential(file=os.path.join(GOLDEN, "cfg5.coef"))
        n = REF_SAMPLE["orbits5"]
        t0 = time.perf_counter()
        fin5, steps5, status5 = p5.orbits(ic5[:n], T5[:n], nthreads=cores)
        dt = time.perf_counter() - t0
        parity = orbit_deviation(*engine["orbits5"], fin5, status5) if engine is not None else None
        res.append((base(float(steps5.sum()) / dt, "accepted DOP853 steps/s",
                         "first %d orbits of the config 5 workload, OpenMP dynamic 1" % n), parity))
        af5 = ref.ActionFinder(p5)
        # the actions of the engine's own snapshot points (the same inputs on both sides), or of the
        # reference's final points when there is no engine run (reference arm)
        pts = engine["actions5"][0] if engine is not None else fin5
        t0 = time.perf_counter()
        J = af5.actions(pts, nthreads=cores)
        dt = time.perf_counter() - t0
        parity = rel_action_err(engine["actions5"][1], J) if engine is not None else None
        res.append((base(len(pts) / dt, "actions/s", "actions of %d final points of the config-5 orbits, reference "
                         "ActionFinderAxisymFudge, OpenMP" % len(pts)), parity))
        return res
    except Exception as e:   # the baseline is reported, never required
        return [({"value": None, "kind": "reference", "sample": "failed: %s" % e}, None)] * 5


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
    import ctypes
    _native.check(lib.agama_actionPhaseTiming(1, None, None))     # CUDA events around each phase
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        step()
        ends[k].record(stream)
    torch.cuda.synchronize()
    phase_ms, phase_passes = (ctypes.c_double * 4)(), ctypes.c_long(0)
    _native.check(lib.agama_actionPhaseTiming(0, phase_ms, ctypes.byref(phase_passes)))
    phase_ms = [phase_ms[k] / args.steps for k in range(4)]
    if dist:
        dist.barrier()
    clocks = sampler.stop(physical_gpu_index(local)) if rank == 0 else None
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(np.sum(per))
    total_ms = max_over_ranks(total_ms, dist, dev)
    value = n * world * args.steps / (total_ms / 1000)
    ms_per_step = total_ms / args.steps

    # ---- end to end through the public API, pinned host buffers
    hp = torch.from_numpy(pts).pin_memory().numpy()
    out = None
    for _ in range(3):      # warm-up at full size: the outputs' page-locked blocks (the previous result
        out = af(hp)        # is alive during the next call, as in the timed loop), the pool's chunk scratch
    e2e_times = []
    for k in range(max(2, min(args.steps, 5))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = af(hp)
        e2e_times.append(time.perf_counter() - t0)
    e2e_ms = 1000 * float(np.mean(e2e_times))
    e2e_val = n * world / (max_over_ranks(e2e_ms, dist, dev) / 1000)
    pk = ctypes.c_double(0)
    _native.check(lib.agama_measureFP64Throughput(ctypes.byref(pk)))
    if rank == 0:
        # ---- roofline (FP64-pipe bound): the dominant kernel (root searches), timed by CUDA events
        # around it during the timed steps, and the whole three-kernel step; executed FP64 flops
        # per action from an ncu capture of this workload; peak measured on this device
        achieved = FLOPS_ROOT_PER_ACTION_CFG2 * n / (phase_ms[2] / 1000) / 1e12
        step_achieved = FLOPS_PER_ACTION_CFG2 * n / (ms_per_step / 1000) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "actions/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded disk particles)",
            "config": {"workload": WORKLOAD, "particles_per_gpu": n, "mode": "plain FP64",
                       "l2": "flushed between steps (256 MB write)", "parallelism": "replicas x%d" % world},
            "e2e": {"value": e2e_val, "unit": "actions/s", "h2d_bytes_per_step": int(pts.nbytes),
                    "d2h_bytes_per_step": int(n * 3 * 8)},
            "gpu_launches": ACTION_LAUNCHES_PER_STEP * args.steps,
            "roofline": {"bound": "fp64", "kernel": "fudgeRootKernel", "achieved": achieved, "peak": pk.value,
                         "unit": "TFLOP/s", "frac": achieved / pk.value if pk.value else None,
                         "traffic": TRAFFIC_ROOT_PER_LAUNCH_CFG2, "ms_per_launch": phase_ms[2],
                         "flops_per_action": FLOPS_ROOT_PER_ACTION_CFG2,
                         "peak_source": "measured FP64 FMA throughput of this device (agama_measureFP64Throughput)",
                         "step": {"kernels": 3, "achieved": step_achieved,
                                  "frac": step_achieved / pk.value if pk.value else None,
                                  "flops_per_action": FLOPS_PER_ACTION_CFG2, "traffic": TRAFFIC_PER_STEP_CFG2,
                                  "phase_ms": {"prepare": phase_ms[0], "roots": phase_ms[2],
                                               "integrals": phase_ms[3]}}},
            "clocks": clocks,
            "cpu_baseline": None if args.no_baseline else cpu_baseline_line(pts, act.cpu().numpy()),
        }
    secondary = None if args.no_secondary else run_engine_secondary(dev, flush, dist, rank == 0 and not args.no_baseline,
                                                                    pk.value)
    if not args.no_secondary:
        secondary += run_bracket_modes(dev, flush, dist, af, dpts, act.clone())
    if rank == 0:
        if secondary is not None:
            line["secondary"] = secondary
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# kernels per action step: prepare, root searches, integrals
ACTION_LAUNCHES_PER_STEP = 3
# executed FP64 flops per action (dadd + dmul + 2 dfma, ncu, config-2 workload, 200 000 particles):
# prepare 3485, root searches 10463, integrals 8612
FLOPS_ROOT_PER_ACTION_CFG2 = 10463.0
FLOPS_PER_ACTION_CFG2 = 3485.0 + 10463.0 + 8612.0
# dram read + write of one 200 000-particle step (prepare 11.60 + 50.42 MB, roots 35.31 + 0.62 MB,
# integrals 26.08 + 0.00 MB), scaled to 1e6 particles (the traffic grows with the particles)
TRAFFIC_ROOT_PER_LAUNCH_CFG2 = 5 * 35.94e6
TRAFFIC_PER_STEP_CFG2 = 5 * 124.03e6
# executed FP64 flops (dadd + dmul + 2 dfma, ncu) per unit of the secondary workloads: per force
# evaluation, per accepted DOP853 step (the rejected attempts' work included), per action
# (bench.py --profile-case under ncu; profiles/secondary_workloads_flops.md): forces 1.704e8 / 1e5,
# orbits 1.022e11 / 3 307 982, 3.624e11 / 9 784 415, 7.621e11 / 68 712 155 accepted steps, actions of
# the config-5 snapshot (prepare + roots + integrals) 4.802e8 / 20 000
FLOPS = {"forces1": 1704.0, "orbits1": 30895.0, "orbits3": 37038.0, "orbits5": 11091.0, "actions5": 24009.0}
FLOPS_SOURCE = "ncu FP64 instruction counts of the kernel on a case of this workload (bench.py --profile-case)"


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


def run_profile_case():
    """one launch of each workload's kernels on a small case, in a fixed order, with the units
    each launch processed (force evaluations, accepted steps, actions) printed as one JSON line:
    the ncu instruction counts of these launches divided by these units give the FLOPS table.
    Lanes per orbit and the block size are fixed (1, 64: the autotuner's trial would add launches of
    its own; neither changes the arithmetic of an orbit)."""
    import torch
    import agama_b200
    from agama_b200 import workloads
    dev = torch.device("cuda", 0)
    agama_b200.set_orbit_lanes(1)
    agama_b200.set_orbit_block(64)
    units = {}
    pot1 = agama_b200.Potential(file=os.path.join(GOLDEN, "cfg1.coef"))
    pts1 = workloads.dehnen_positions(100000, 1.0, q=(0.8, 0.6), seed=workloads.SEEDS["points1"])
    d1 = torch.tensor(pts1, device=dev)
    pot1.eval(d1, pot=True, acc=True)
    torch.cuda.synchronize()
    units["forces1"] = len(pts1)
    for key, coef, cfg, n, Om, mx in (("orbits1", "cfg1", 1, 10000, 0.0, 0), ("orbits3", "cfg3", 3, 20000, 0.05, 500),
                                      ("orbits5", "cfg5", 5, 20000, 0.0, 0)):
        pot = pot1 if coef == "cfg1" else agama_b200.Potential(file=os.path.join(GOLDEN, coef + ".coef"))
        ic, T = workloads.orbit_workload(cfg, pot.potential, pot.force, n)
        fin, info = agama_b200.orbit(pot, torch.tensor(ic, device=dev), torch.tensor(T, device=dev), Omega=Om,
                                     maxNumSteps=mx, queue=True, info=True)
        torch.cuda.synchronize()
        units[key] = int(info["steps"].sum().item())
        if key == "orbits5":
            af5 = agama_b200.ActionFinder(pot)
            af5(fin)
            torch.cuda.synchronize()
            units["actions5"] = n
    agama_b200.set_orbit_lanes(0)
    agama_b200.set_orbit_block(0)
    print(json.dumps({"profile_case_units": units, "order": ["forces1", "orbits1", "orbits3", "orbits5", "actions5"]}))


def main():
    args = parse()
    if args.profile_case:
        run_profile_case()
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
