"""Benchmark: rod-steps/s of the plain GPU PSOR path (hard-contact workload).

Workload (default): nsc_dense - N=20000 capsules L=1, d=0.05 (aspect ratio
20) in a periodic cube, isotropic RSA packing, PSOR friction cone mu=0.3,
omega=1, residual tolerance 1e-6, max 500 sweeps, dt=5e-4, no gravity, no
damping.  Isotropic RSA jams near phi=0.12 at this aspect ratio, so the
packing is generated at phi=0.10 (the stated phi=0.20 is unreachable).

  python bench.py --gpus N --steps K --warmup W           # this framework
  python bench.py --impl reference --steps K --warmup W   # reference CPU path

Under torchrun each rank runs an independent replica (the path does not
shard: replicas only); timing is max over ranks.  One step = one
App::physicsStep of the NSC branch over all N rods.  'value' is device time
(CUDA events on the library's stream) with the state resident in HBM;
'e2e' runs the same steps through the C ABI with the state uploaded from
and read back to pinned host memory every step.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rod-dynamics-3d_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

WORKLOAD_PHI = {"nsc_dense": 0.10, "nsc_large": 0.10, "hm_small": 0.10, "hm_large": 0.05}
METRIC = "rod-steps/s at PSOR residual<=1e-6: learned warm-start vs plain GPU PSOR"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {"hbm_gbs": 6650.0, "fallback": True}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[2 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_scene(workload, n, seed):
    from rodgpu import scene
    w = scene.WORKLOADS[workload]
    nn = w["n"] if n is None else n
    sc = scene.make_rods(nn, w["L"], w["d"], phi=WORKLOAD_PHI[workload], seed=seed, max_attempts=20000)
    kw = dict(w["cfg"])
    kw.update(gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0)
    kw.update(scene.pbc_kwargs(sc))
    return kw, sc


def algorithmic_bytes(stage, st, n, steps):
    """Algorithmic bytes of a stage over the timed steps (FP64 SoA model)."""
    c = st["contacts"]
    if stage == "psor":
        return 568.0 * st["psor_row_sweeps"]          # row 328 + λ 48 + two bodies' v,ω 192
    if stage == "integrate":
        return 496.0 * n * steps                      # free flight + drift/damp/wrap
    if stage == "detect":
        return 2 * (72.0 * n + 8.0 * c) * steps       # two detections per step: x,q,r,h per rod + pair
    if stage == "manifolds":
        return 616.0 * c * steps
    if stage == "project":
        return 312.0 * c * steps
    return None


def run_ours(args, rank, world):
    import rodgpu
    from rodgpu import scene  # noqa: F401
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(dev)  # the C library uses the current device
    kw, sc = build_scene(args.workload, args.n, args.seed + rank)
    n = sc["n"]

    def make():
        cfg = rodgpu.default_config(n_bodies=n, **kw)
        s = rodgpu.System(cfg)
        s.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        s.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
        return s

    sys_ = make()
    sys_.step(args.warmup)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        st = sys_.step(args.steps)
    torch.cuda.synchronize()
    ms = st["device_ms"]
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        ms = float(t.item())
    value = n * args.steps * world / (ms / 1000.0)

    # end-to-end through the C ABI with host buffers: upload, step, read back
    state = sys_.get_state()
    k_e2e = max(3, min(args.steps, 50))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        sys_.set_state(state["x"], state["q"], state["v"], state["w"])
        sys_.step(1)
        state = sys_.get_state()
    t1 = time.perf_counter()
    e2e = n * k_e2e / (t1 - t0)

    # stage timers over a short run for the roofline of the dominant stage
    prof = make()
    prof.step(args.warmup)
    prof.set_profiling(True)
    pst = prof.step(max(5, min(args.steps, 50)))
    stages = prof.profile()
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms, dom_launches = stages[dom]
    psteps = pst["steps"]
    b = algorithmic_bytes(dom, pst, n, psteps)
    pk = peaks()
    peak = pk.get("hbm_gbs", 6650.0)
    roof = {"bound": "hbm", "kernel": dom, "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
            "traffic": None, "peak_source": "measured" if "fallback" not in pk else "fallback",
            "stage_ms_share": {k: round(v[0] / max(1e-9, sum(x[0] for x in stages.values())), 4)
                               for k, v in stages.items()}}
    if b is not None and dom_ms > 0:
        ach = b / (dom_ms / 1000.0) / 1e9
        roof.update(achieved=round(ach, 2), frac=round(ach / peak, 5),
                    bytes_per_launch=round(b / max(1, dom_launches), 1))
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "rod-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded RSA packing, Gaussian velocities)",
        "config": {"workload": f"{args.workload}: N={n}, L=1, d={sc['d']}, phi={round(sc['phi'], 4)}, "
                               f"box={round(sc['side'], 4)}, PSOR mu=0.3 omega=1 tol=1e-6 max 500 sweeps, "
                               f"dt=5e-4, warm start=cache (plain GPU PSOR)",
                   "rods": n, "parallelism": f"replicas x{world}",
                   "l2": "inputs resident; working set < L2 (no flush: state persists step to step)"},
        "e2e": {"value": round(e2e, 1), "unit": "rod-steps/s", "h2d_bytes_per_step": n * 13 * 8,
                "d2h_bytes_per_step": n * 19 * 8, "steps": k_e2e},
        "gpu_launches": int(st["kernel_launches"]),
        "psor": {"sweeps_per_step": round(st["psor_sweeps"] / args.steps, 2),
                 "contacts_last": st["contacts"], "max_residual": st["max_residual"],
                 "not_converged_steps": st["not_converged"], "colors_last": st["colors"],
                 "list_rebuilds": st["list_rebuilds"]},
        "roofline": roof,
        "clocks": clk.summary(),
    }
    return out


def run_reference(args, steps, warmup, threads=0):
    """The reference's own FP32 CPU path (oracle/_ref) on the same workload."""
    from oracle import Reference
    import rodgpu
    kw, sc = build_scene(args.workload, args.n, args.seed)
    n = sc["n"]
    cfg = rodgpu.default_config(n_bodies=n, **kw)
    r = Reference(cfg, threads=threads, spatial_hash=True)
    r.set_bodies(sc["radius"], sc["half_height"], np.full(n, 1.0), sc["restitution"])
    r.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
    if warmup:
        r.step(warmup)
    t0 = time.perf_counter()
    r.step(steps)
    dt = time.perf_counter() - t0
    return n * steps / dt, r.threads(), n, steps, dt


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="nsc_dense")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank != 0:
            return
        try:
            v, th, n, k, dt = run_reference(args, steps=max(1, min(args.steps, 3)), warmup=min(args.warmup, 1))
        except Exception as e:  # noqa: BLE001
            print(json.dumps({"impl": "reference", "unavailable": f"reference build not loadable: {e}"}))
            return
        line = {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": "rod-steps/s",
                "n_gpus": 0, "steps": k, "warmup": min(args.warmup, 1), "higher_is_better": True,
                "dtype": "f32", "config": {"workload": f"{args.workload}: N={n} (same packing)"},
                "cpu_baseline": {"value": round(v, 2), "unit": "rod-steps/s", "cores": th, "kind": "reference",
                                 "sample": f"{k} steps of the full N={n} system, spatial hash, OpenMP"},
                "e2e": {"value": round(v, 2), "unit": "rod-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    out = run_ours(args, rank, world)
    if rank == 0 and not args.no_cpu_baseline:
        try:
            v, th, n, k, dt = run_reference(args, steps=2, warmup=0)
            out["cpu_baseline"] = {"value": round(v, 2), "unit": "rod-steps/s", "cores": th, "kind": "reference",
                                   "sample": f"{k} steps of the full N={n} system ({dt:.1f} s), reference "
                                             f"src/physics compiled FP32 + OpenMP, spatial hash"}
        except Exception as e:  # noqa: BLE001
            out["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
