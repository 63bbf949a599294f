"""Benchmark: rod-steps/s at PSOR residual <= 1e-6, learned warm start vs
plain GPU PSOR.

Headline (default workload 'batch'): the NSC half of the uneven-batch
workload - 128 independent periodic systems, N log-uniform in [500, 20000]
(662,433 rods in total for seed 1), aspect ratio 5/10/20/40 (L=1, d=1/AR), phi ~
U[0.05, 0.25] capped at 1.6/AR (isotropic RSA limit), mu ~ U[0, 1], PSOR
omega=1, tol 1e-6, max 500 sweeps, dt=5e-4, no gravity, no damping - run as
ONE persistent CUDA-graph launch per call with the learned warm start
(network trained first, by the library's own kernels, on converged impulses
recorded from plain PSOR on 32 other seeded systems).  Compared with the
plain single-system GPU PSOR path on nsc_dense (N=20000, AR 20, phi 0.10;
isotropic RSA jams near phi=0.12 at this aspect ratio, so the stated 0.20 is
unreachable) and with the plain batched path.

  python bench.py --gpus N --steps K --warmup W           # this framework
  python bench.py --impl reference --steps K --warmup W   # reference CPU path

Under torchrun each rank runs an independent replica on its own packings
(the path does not shard: replicas only); 'value' counts the rods of all
ranks over the slowest rank's time.  'value' is device time
(CUDA events on the library's stream) with the state resident in HBM; 'e2e'
runs steps through the C ABI with every member's state uploaded from and
read back to host memory every step.
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


def nsc_bytes(rod_steps, contact_steps, row_sweeps):
    """Algorithmic bytes of NSC steps (FP64 SoA model): 496 B per rod-step
    (free flight, detection reads, drift/damp/wrap), 616 B per contact-step
    (manifold row build), 568 B per contact-sweep (row 328 + lambda 48 + two
    bodies' v, w 192).  Position projection is not counted."""
    return 496.0 * rod_steps + 616.0 * contact_steps + 568.0 * row_sweeps


def roofline(bytes_, ms, kernel, traffic=None):
    pk = peaks()
    peak = pk.get("hbm_gbs", 6650.0)
    ach = bytes_ / (ms / 1000.0) / 1e9 if ms > 0 else None
    return {"bound": "hbm", "kernel": kernel, "achieved": None if ach is None else round(ach, 2),
            "peak": peak, "unit": "GB/s", "frac": None if ach is None else round(ach / peak, 5),
            "traffic": traffic, "peak_source": "measured" if "fallback" not in pk else "fallback",
            "algorithmic_bytes_per_launch": round(bytes_, 1)}


def profile_traffic(name, rod_steps):
    """DRAM bytes of a launch of rod_steps rod-steps, from the DRAM bytes per
    rod-step that the committed ncu summary records (a capture of a smaller
    launch of the same kernel, scaled by the rods and steps processed)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_rod_step:"):
                return round(float(line.split(":", 1)[1].split()[0]) * rod_steps, 1)
    except OSError:
        pass
    return None


def load_system(rodgpu, cfg, sc):
    s = rodgpu.System(cfg)
    s.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
    s.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
    return s


def load_batch(rodgpu, items, warm):
    cfgs = []
    for cfg, _ in items:
        c = rodgpu.RgConfig.from_buffer_copy(cfg)
        c.nsc_warm_start = rodgpu.WARM[warm]
        cfgs.append(c)
    b = rodgpu.Batch(cfgs)
    for k, (_, sc) in enumerate(items):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, sc["x"], sc["q"], sc["v"], sc["w"])
    return b


def plain_single(rodgpu, args):
    """The plain single-system GPU PSOR path on nsc_dense."""
    kw, sc = build_scene("nsc_dense", None, args.seed)
    s = load_system(rodgpu, rodgpu.default_config(n_bodies=sc["n"], **kw), sc)
    s.step(args.warmup)
    st = s.step(args.steps)
    n = sc["n"]
    ms = st["device_ms"]
    b = nsc_bytes(n * args.steps, st["contact_steps"], st["psor_row_sweeps"])
    return {"value": round(n * args.steps / (ms / 1000.0), 1), "ms_per_step": round(ms / args.steps, 4),
            "rods": n, "phi": round(sc["phi"], 4),
            "sweeps_per_step": round(st["psor_sweeps"] / args.steps, 2),
            "contacts_per_step": round(st["contact_steps"] / args.steps, 1),
            "not_converged_steps": st["not_converged"], "max_residual": st["max_residual"],
            "roofline": roofline(b, ms, "k_nsc_run (single system)", None)}


def verlet_bytes(rod_steps, contact_evals):
    """Algorithmic bytes of soft / Hertz-Mindlin velocity-Verlet steps (FP64
    SoA model): 896 B per rod-step (half kick + drift, two force
    evaluations' body reads and force writes, second kick, cell keys) and
    72 B per contact and force evaluation (pair record 8 + history read 32
    + write 32), i.e. 144 B per contact-step at two evaluations per step.
    contact_evals = the sum over the force evaluations of their contacts."""
    return 896.0 * rod_steps + 72.0 * contact_evals


# Hertz-Mindlin workloads timed beside the headline: the small plain
# soft-contact configuration (N = 1000, d = 0.1, phi 0.10, E = 1e5, mu 0.5,
# dt 1e-4, 1000 steps) and the large single system (N = 1e6, d = 0.02,
# E = 1e6, e = 0.3, dt 2e-5, 100 steps; isotropic RSA of aspect-ratio-50
# rods jams near phi*AR ~ 2.4, so it runs at phi 0.045 instead of 0.15; the
# packing comes from the device generator).
HM_LINES = {
    "hm_small": dict(n=1000, d=0.1, phi=0.10, steps=1000, device_gen=False,
                     cfg=dict(model="hertz-mindlin", dt=1e-4, hm_youngs_modulus=1e5, hm_poisson_ratio=0.3,
                              hm_restitution=0.5, hm_friction=0.5)),
    "hm_large": dict(n=1000000, d=0.02, phi=0.045, steps=100, device_gen=True,
                     cfg=dict(model="hertz-mindlin", dt=2e-5, hm_youngs_modulus=1e6, hm_poisson_ratio=0.3,
                              hm_restitution=0.3, hm_friction=0.5)),
}


def hm_line(rodgpu, args, name, n=None):
    """One Hertz-Mindlin workload: device time of its steps with the state
    resident in HBM, with the roofline of the whole velocity-Verlet step."""
    from rodgpu import scene
    w = HM_LINES[name]
    nn = w["n"] if n is None else n
    t0 = time.perf_counter()
    if w["device_gen"]:
        sc = scene.make_rods_device(nn, 1.0, w["d"], phi=w["phi"], seed=args.seed, max_attempts=20000)
    else:
        sc = scene.make_rods(nn, 1.0, w["d"], phi=w["phi"], seed=args.seed, max_attempts=20000)
    t_gen = time.perf_counter() - t0
    kw = dict(w["cfg"], gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0)
    kw.update(scene.pbc_kwargs(sc))
    s = load_system(rodgpu, rodgpu.default_config(n_bodies=sc["n"], **kw), sc)
    steps = args.hm_steps or w["steps"]
    s.step(max(3, args.warmup))
    st = s.step(steps)
    ms = st["device_ms"]
    m = sc["n"]
    out = {"value": round(m * steps / (ms / 1000.0), 1), "unit": "rod-steps/s", "rods": m,
           "phi": round(sc["phi"], 4), "steps": steps, "ms_per_step": round(ms / steps, 5),
           "contacts_per_evaluation": round(st["contact_steps"] / (2.0 * steps), 1),
           "kernel_launches": int(st["kernel_launches"]),
           "launches_per_step": round(st["kernel_launches"] / steps, 1),
           "scene_s": round(t_gen, 2), "scene_generator": "device" if w["device_gen"] else "host",
           "roofline": roofline(verlet_bytes(m * steps, st["contact_steps"]), ms,
                                "velocity-Verlet step, all kernels (Hertz-Mindlin)", None)}
    s.close()
    return out


def secondary_gpu_baseline(rodgpu, args, sizes=(10000, 50000, 100000)):
    """The reference's own FP32 two-pass CUDA broad phase
    (cudaDetectCapsulePairsTwoPass: AABB kernel, O(N^2) AABB pair kernel,
    Lumelsky narrow phase; built for sm_100a from the reference's source)
    against rg_detect on the same packings: aspect ratio 20 (L = 1,
    d = 0.05) at phi 0.10, generated at 0.9 d so contacts exist.  Both are
    timed as whole calls from host arrays to host contact lists (wall
    clock, median of 3 after one untimed call); the reference's own stage
    timers are reported beside them.  'ours_first' is the first call on a
    system, which builds the neighbour lists; 'ours' is a repeated call
    (lists kept, as in a running simulation)."""
    from oracle import refcuda_detect
    from rodgpu import scene
    out = []
    for n in sizes:
        side = scene.box_side(n, 1.0, 0.05, 0.10)
        sc = scene.make_rods_device(n, 1.0, 0.045, side=side, seed=args.seed + 7)
        sc["radius"] = np.full(sc["n"], 0.025)
        kw = dict(model="nsc", gravity=(0.0, 0.0, 0.0))
        kw.update(scene.pbc_kwargs(sc))
        s = rodgpu.System(rodgpu.default_config(n_bodies=sc["n"], **kw))
        s.set_bodies(sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        s.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
        t0 = time.perf_counter()
        mine, _, _ = s.detect(0.0)
        first = (time.perf_counter() - t0) * 1e3
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            mine, _, _ = s.detect(0.0)
            ts.append((time.perf_counter() - t0) * 1e3)
        s.close()
        box = (side, side, side)
        refcuda_detect(sc, 0.0, box)
        walls, stages = [], []
        for _ in range(3):
            theirs, st, wall = refcuda_detect(sc, 0.0, box)
            walls.append(wall)
            stages.append(st)
        st = np.median(np.array(stages), axis=0)
        a = {tuple(p) for p in mine.tolist()}
        b = {tuple(p) for p in theirs.tolist()}
        out.append({"n": int(sc["n"]), "ours_first_ms": round(first, 3), "ours_ms": round(float(np.median(ts)), 3),
                    "reference_ms": round(float(np.median(walls)), 3),
                    "reference_kernels_ms": round(float(st[1] + st[2] + st[3]), 3),
                    "reference_stages_ms": {"upload": round(float(st[0]), 3), "aabb": round(float(st[1]), 3),
                                            "pair_test": round(float(st[2]), 3),
                                            "narrow": round(float(st[3]), 3), "download": round(float(st[4]), 3)},
                    "reference_candidates": int(st[5]),
                    "contacts": {"ours_fp64": len(a), "reference_fp32": len(b), "common": len(a & b)},
                    "speedup_call": round(float(np.median(walls)) / max(float(np.median(ts)), 1e-9), 2)})
    return out


def learned_line(rodgpu, args, train_runs=12, eval_runs=5, n=50000, steps=200, warm=100, chunk=12):
    """The learned-warm-start configuration: N = 50,000 rods (L = 1,
    d = 0.05, phi 0.10 - the isotropic RSA limit near phi*AR ~ 2.4 rules
    out the stated 0.20 - device packings), mu ~ U[0.1, 0.8] per run.  The
    network is trained by the library's kernels on the records of
    train_runs plain-PSOR runs (steps recorded after `warm` unrecorded
    steps, generated `chunk` runs at a time and merged through the record
    file format), then each of eval_runs held-out seeds runs warm + steps
    steps from the cache start and from the learned start (default scope
    and gate).  Reported: PSOR sweeps, device time and steps stopped at the
    sweep cap, in total and per held-out run."""
    import tempfile
    from rodgpu import records, scene
    t0 = time.perf_counter()
    parts = []
    with tempfile.TemporaryDirectory() as tmp:
        for c0 in range(0, train_runs, chunk):
            path = os.path.join(tmp, f"records_{c0}.npz")
            records.generate(min(chunk, train_runs - c0), steps, n=n, ar=20, phi=0.10, mu_range=(0.1, 0.8),
                             seed=1000 + c0, warmup=warm, path=path)
            parts.append(records.load(path))
    ds = records.merge(parts)
    t_rec = time.perf_counter() - t0
    trainer = rodgpu.System(rodgpu.default_config(n_bodies=16, model="nsc"))
    t0 = time.perf_counter()
    loss = trainer.mlp_train(ds["features"], ds["targets"], epochs=20, batch=4096, lr=1e-3, seed=3)
    t_train = time.perf_counter() - t0
    params = trainer.mlp_get_params()
    trainer.close()
    per_run = []
    for k in range(eval_runs):
        rng = np.random.default_rng(50000 + k)
        mu = float(rng.uniform(0.1, 0.8))
        sc = scene.make_rods_device(n, 1.0, 0.05, phi=0.10, seed=70000 + k, max_attempts=20000)
        row = {"mu": round(mu, 3)}
        for mode in ("cache", "mlp"):
            kw = dict(model="nsc", dt=5e-4, nsc_mu=mu, nsc_omega=1.0, nsc_tol=1e-6, nsc_velocity_iters=500,
                      gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0, nsc_warm_start=mode)
            kw.update(scene.pbc_kwargs(sc))
            s = load_system(rodgpu, rodgpu.default_config(n_bodies=sc["n"], **kw), sc)
            if mode == "mlp":
                s.mlp_set_params(params)
            s.step(warm)
            st = s.step(steps)
            row[mode] = {"sweeps": int(st["psor_sweeps"]), "ms": round(st["device_ms"], 2),
                         "capped_steps": int(st["not_converged"])}
            s.close()
        per_run.append(row)
    tot = {m: {"sweeps": sum(r[m]["sweeps"] for r in per_run), "ms": round(sum(r[m]["ms"] for r in per_run), 2),
               "capped_steps": sum(r[m]["capped_steps"] for r in per_run)} for m in ("cache", "mlp")}
    ratio_sw = [r["mlp"]["sweeps"] / max(r["cache"]["sweeps"], 1) for r in per_run]
    ratio_ms = [r["mlp"]["ms"] / max(r["cache"]["ms"], 1e-9) for r in per_run]
    return {"rods": n, "train": {"runs": train_runs, "steps": steps, "warmup": warm, "records": int(len(ds["features"])),
                                 "final_loss": round(loss, 4), "record_s": round(t_rec, 1), "train_s": round(t_train, 1)},
            "held_out": {"runs": eval_runs, "steps": steps, "after_warmup": warm, "total": tot, "per_run": per_run,
                         "sweeps_ratio_mean": round(float(np.mean(ratio_sw)), 3),
                         "sweeps_ratio_range": [round(min(ratio_sw), 3), round(max(ratio_sw), 3)],
                         "time_ratio_mean": round(float(np.mean(ratio_ms)), 3),
                         "time_ratio_range": [round(min(ratio_ms), 3), round(max(ratio_ms), 3)]}}


def train_network(rodgpu, args):
    """Records converged impulses of plain PSOR on separate seeded systems
    and trains the network with the library's kernels."""
    from rodgpu import scene
    specs = [s for s in scene.batch_members(2 * args.train_systems, seed=args.seed + 100) if s["model"] == "nsc"]
    items = scene.batch_scenes(specs)
    b = load_batch(rodgpu, items, "cache")
    cap = 1 << 16
    for k in range(len(items)):
        b.member(k).mlp_record(True, cap)
    b.step(args.train_steps)
    xs, ys = [], []
    for k in range(len(items)):
        x, y = b.member(k).mlp_records()
        xs.append(x)
        ys.append(y)
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    t0 = time.perf_counter()
    m = b.member(0)
    loss = m.mlp_train(x, y, epochs=args.epochs, batch=2048, lr=1e-3, seed=args.seed)
    t_train = time.perf_counter() - t0
    params = m.mlp_get_params()
    b.close()
    return params, {"records": int(len(x)), "systems": len(items), "steps": args.train_steps,
                    "epochs": args.epochs, "final_loss": round(loss, 5), "train_s": round(t_train, 2)}


def time_batch(b, n_total, args, clk=None):
    b.step(args.warmup)
    if clk is not None:
        with clk:
            st = b.step(args.steps)
    else:
        st = b.step(args.steps)
    ms = st[0]["device_ms"]
    rs = sum(x["psor_row_sweeps"] for x in st)
    cs = sum(x["contact_steps"] for x in st)
    sw = sum(x["psor_sweeps"] for x in st)
    return {"value": round(n_total * args.steps / (ms / 1000.0), 1), "ms": ms,
            "ms_per_step": round(ms / args.steps, 4),
            "sweeps_per_system_step": round(sw / (len(st) * args.steps), 3),
            "contacts_per_step": round(cs / args.steps, 1),
            "not_converged_steps": int(sum(x["not_converged"] for x in st)),
            "max_residual": max(x["max_residual"] for x in st),
            "kernel_launches": int(st[0]["kernel_launches"]),
            "bytes": nsc_bytes(n_total * args.steps, cs, rs)}


def job_totals(ms, rods, dist, device="cuda"):
    """Whole-job figures of N replicas: the slowest rank's time (max over
    ranks) and the rods all ranks stepped (sum).  Every rank calls it at the
    same point (one all-reduce each for the two figures)."""
    if not dist:
        return ms, rods
    import torch
    import torch.distributed as tdist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    r = torch.tensor([float(rods)], dtype=torch.float64, device=device)
    tdist.all_reduce(r, op=tdist.ReduceOp.SUM)
    return float(t.item()), int(round(r.item()))


def run_ours(args, rank, world):
    import rodgpu
    from rodgpu import scene
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(dev)  # the C library uses the current device
    if args.workload == "batch_only":
        return run_batch_only(args, rank, world)
    if args.workload != "batch":
        return run_single(args, rank, world)
    specs = [s for s in scene.batch_members(256, seed=args.seed + rank) if s["model"] == "nsc"]
    items = scene.batch_scenes(specs)
    n_total = sum(sc["n"] for _, sc in items)
    params, train = train_network(rodgpu, args)
    single = plain_single(rodgpu, args)

    # schedule candidates: the balanced plan, and multiples of the rods per
    # block of an even split
    r0 = n_total / 148.0
    cands = (-1, 0) + tuple(int(r0 * f) for f in (0.5, 0.75, 1.0, 1.5, 2.0, 3.0))
    plain = load_batch(rodgpu, items, "cache")
    best_plain, _ = plain.autotune(candidates=cands, trial_steps=20)
    res_plain = time_batch(plain, n_total, args)
    plain.close()

    learned = load_batch(rodgpu, items, "mlp")
    learned.set_mlp(params)
    best, tune = learned.autotune(candidates=cands, trial_steps=20)
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(dev)
    res = time_batch(learned, n_total, args, clk)
    torch.cuda.synchronize()
    # replicas step different packings (seed + rank): whole-job rods are the
    # sum over ranks, the time the slowest rank's
    ms, job_rods = job_totals(res["ms"], n_total, dist)
    value = job_rods * args.steps / (ms / 1000.0)

    # end to end through the C ABI: every step uploads all members' states
    # from page-locked host arrays (one bulk transfer per array), steps, and
    # reads all states back
    def pinned(cols):
        return torch.empty((n_total, cols), dtype=torch.float64, pin_memory=True).numpy()
    host = (pinned(3), pinned(4), pinned(3), pinned(3))
    learned.get_state_all(out=host)
    k_e2e = max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        learned.set_state_all(*host)
        learned.step(1, stats=False)
        learned.get_state_all(out=host)
    t1 = time.perf_counter()
    e2e_s, _ = job_totals(t1 - t0, n_total, dist)
    e2e = job_rods * k_e2e / e2e_s
    sched = learned.schedule()
    learned.close()

    roof = roofline(res["bytes"], res["ms"], "k_nsc_run (batched, learned warm start)",
                    profile_traffic("k_nsc_run_batch.md", n_total * args.steps))
    hm = {} if args.no_hm else {name: hm_line(rodgpu, args, name) for name in HM_LINES}
    try:
        second = secondary_gpu_baseline(rodgpu, args)
    except Exception as e:  # noqa: BLE001
        second = {"unavailable": str(e)}
    learned_n50k = {} if args.no_learned else learned_line(rodgpu, args, train_runs=args.learned_train_runs,
                                                           eval_runs=args.learned_eval_runs)
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "rod-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded RSA packings, Gaussian velocities)",
        "config": headline_config(n_total, len(items)),
        "parallelism": f"replicas x{world}",
        "tuning": {"schedule": sched, "autotune_ms": tune},
        "psor_compliance": compliance(res, len(items), args.steps),
        "comparison": {"plain_single_system": single,
                       "plain_batched": {k: v for k, v in res_plain.items() if k not in ("ms", "bytes")},
                       "learned_batched": {k: v for k, v in res.items() if k not in ("ms", "bytes")},
                       "speedup_learned_batched_vs_plain_single": round(value / world / single["value"], 3),
                       "speedup_learned_vs_plain_batched": round(res["value"] / res_plain["value"], 3),
                       "autotuned_rods_per_block": {"plain": best_plain, "learned": best},
                       "training": train},
        "e2e": {"value": round(e2e, 1), "unit": "rod-steps/s", "h2d_bytes_per_step": job_rods * 13 * 8,
                "d2h_bytes_per_step": job_rods * 13 * 8, "steps": k_e2e,
                "path": "rg_batch_set_state_all + rg_batch_step(1) + rg_batch_get_state_all, pinned host arrays"},
        "gpu_launches": res["kernel_launches"],
        "roofline": roof,
        "hertz_mindlin": hm,
        "secondary_gpu_baseline": second,
        "learned_warm_start_n50k": learned_n50k,
        "clocks": clk.summary(),
    }
    return out


def compliance(res, nsys, steps):
    """How many system-steps met the PSOR tolerance (residual <= 1e-6 by the
    reference's definition, nsc_contact.cpp:546-551) and how many stopped at
    the sweep cap; 'value' counts every rod-step, the capped ones included."""
    total = nsys * steps
    nc = int(res["not_converged_steps"])
    return {"system_steps": total, "met_tolerance": total - nc, "stopped_at_max_sweeps": nc,
            "fraction_met": round((total - nc) / total, 5) if total else None,
            "max_final_residual": res["max_residual"],
            "value_includes_capped_steps": True}


def run_batch_only(args, rank, world):
    """The first --systems members of the batch workload, plain PSOR, fixed
    schedule (4096 rods per block): one warm-up launch, then one timed
    launch of --steps steps (the launch that profiles capture)."""
    import rodgpu
    from rodgpu import scene
    import torch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    specs = [x for x in scene.batch_members(256, seed=args.seed + rank) if x["model"] == "nsc"][:args.systems]
    items = scene.batch_scenes(specs)
    n_total = sum(sc["n"] for _, sc in items)
    b = load_batch(rodgpu, items, "cache")
    b.set_schedule(4096, True)
    b.step(args.warmup, stats=False)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        res = time_batch_once(b, n_total, args.steps)
    return {"metric": METRIC, "value": res["value"], "unit": "rod-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded RSA packings)",
            "config": {"workload": f"batch_only: {len(items)} NSC systems, {n_total} rods, plain PSOR"},
            "gpu_launches": res["kernel_launches"], "clocks": clk.summary(),
            "roofline": roofline(res["bytes"], res["ms"], "k_nsc_run (batched)", None)}


def time_batch_once(b, n_total, steps):
    st = b.step(steps)
    ms = st[0]["device_ms"]
    rs = sum(x["psor_row_sweeps"] for x in st)
    cs = sum(x["contact_steps"] for x in st)
    return {"value": round(n_total * steps / (ms / 1000.0), 1), "ms": ms, "ms_per_step": round(ms / steps, 4),
            "kernel_launches": int(st[0]["kernel_launches"]), "bytes": nsc_bytes(n_total * steps, cs, rs)}


def run_single(args, rank, world):
    """One named single-system workload (profiling and replica runs)."""
    import rodgpu
    import torch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "learned_n50k":
        r = learned_line(rodgpu, args, train_runs=args.learned_train_runs, eval_runs=args.learned_eval_runs)
        tot = r["held_out"]["total"]
        n_rs = r["rods"] * r["held_out"]["runs"] * r["held_out"]["steps"]
        return {"metric": METRIC, "value": round(n_rs / (tot["mlp"]["ms"] / 1000.0), 1), "unit": "rod-steps/s",
                "n_gpus": world, "steps": r["held_out"]["steps"], "warmup": r["held_out"]["after_warmup"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded device RSA packings)",
                "config": {"workload": "learned_n50k: N=50000, AR 20, phi 0.10, mu U[0.1,0.8]"},
                "plain_value": round(n_rs / (tot["cache"]["ms"] / 1000.0), 1), "detail": r}
    if args.workload in HM_LINES:
        with ClockSampler(dev) as clk:
            r = hm_line(rodgpu, args, args.workload, args.n)
        return {"metric": "rod-steps/s (Hertz-Mindlin velocity Verlet)", "value": r["value"], "unit": "rod-steps/s",
                "n_gpus": world, "steps": r["steps"], "warmup": max(3, args.warmup),
                "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic (seeded RSA packing)",
                "config": {"workload": f"{args.workload}: N={r['rods']}"}, "gpu_launches": r["kernel_launches"],
                "clocks": clk.summary(), "roofline": r["roofline"], "detail": r}
    if args.workload.startswith("member:"):
        # one member of the batch workload, stepped by a single block (the
        # team the batch schedule gives a member of moderate size)
        from rodgpu import scene
        k = int(args.workload.split(":", 1)[1])
        specs = [x for x in scene.batch_members(256, seed=args.seed) if x["model"] == "nsc"]
        cfg, sc = scene.batch_member_scene(specs[k])
        cfg.team_blocks = 1
        kw = {"model": "nsc"}
        n = sc["n"]
        s = load_system(rodgpu, cfg, sc)
    else:
        kw, sc = build_scene(args.workload, args.n, args.seed + rank)
        n = sc["n"]
        s = load_system(rodgpu, rodgpu.default_config(n_bodies=n, **kw), sc)
    s.step(args.warmup)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        st = s.step(args.steps)
    ms = st["device_ms"]
    out = {"metric": METRIC, "value": round(n * args.steps / (ms / 1000.0), 1), "unit": "rod-steps/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded RSA packing)", "config": {"workload": f"{args.workload}: N={n}"},
           "gpu_launches": int(st["kernel_launches"]), "clocks": clk.summary(),
           "psor": {"sweeps_per_step": round(st["psor_sweeps"] / max(1, args.steps), 2),
                    "not_converged_steps": st["not_converged"], "max_residual": st["max_residual"]}}
    if kw.get("model") == "nsc":
        out["roofline"] = roofline(nsc_bytes(n * args.steps, st["contact_steps"], st["psor_row_sweeps"]), ms,
                                   "k_nsc_run", None)
    return out


def batch_workload(nsys):
    """The headline workload's name (both arms print it; the rod count is
    the separate 'rods' key)."""
    return (f"batch: {nsys} NSC systems, N log-uniform [500, 20000], AR 5/10/20/40, "
            f"phi U[0.05,0.25] capped 1.6/AR, mu U[0,1], PSOR omega=1 tol=1e-6 max 500 sweeps, dt=5e-4, "
            f"learned warm start")


def reference_scenes(args, every=1):
    """The batch members as (config, scene), built by the reference library
    oracle/_ref/librodref.so, which compiles this repository's scene
    generator and config defaults beside the reference's physics sources:
    the packings and configurations are bit-identical to the GPU arm's, and
    no library of this repository is loaded.  every=k keeps every k-th
    member by size (the bounded cpu_baseline sample)."""
    from oracle import ref_lib
    from rodgpu import abi, scene  # pure Python (ctypes mirrors, member specs): loads no library
    gen = abi.bind_scene_lib(ref_lib())
    specs = [s for s in scene.batch_members(256, seed=args.seed) if s["model"] == "nsc"]
    if every > 1:
        specs = sorted(specs, key=lambda s: s["n"])[::every]
    return scene.batch_scenes(specs, gen=gen)


def run_reference(items, steps, warmup, threads=0):
    """The reference's own FP32 CPU path (oracle/_ref: the reference's
    src/physics compiled with OpenMP, spatial hash, plain PSOR) on every
    given system, one after the other on all host threads: warmup untimed
    steps, then steps timed with a steady clock."""
    from oracle import Reference
    rod_steps = 0
    dt = 0.0
    th = 0
    for cfg, sc in items:
        n = sc["n"]
        r = Reference(cfg, threads=threads, spatial_hash=True)
        r.set_bodies(sc["radius"], sc["half_height"], np.full(n, 1.0), sc["restitution"])
        r.set_state(sc["x"], sc["q"], sc["v"], sc["w"])
        if warmup:
            r.step(warmup)
        t0 = time.perf_counter()
        r.step(steps)
        dt += time.perf_counter() - t0
        rod_steps += n * steps
        th = r.threads()
        del r
    return rod_steps / dt, th, dt


def loaded_native_libs():
    """Shared objects of this repository mapped into this process."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            p = line.split()[-1] if line.strip() else ""
            if p.endswith(".so") and p.startswith(ROOT):
                out.add(os.path.relpath(p, ROOT))
    except OSError:
        pass
    return sorted(out)


def headline_config(n_total, nsys):
    """The config both arms print (identical keys and values)."""
    return {"workload": batch_workload(nsys), "rods": n_total, "systems": nsys,
            "l2": "no flush: state persists step to step (inputs 133 MB > L2 across members)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--train-systems", type=int, default=32)
    ap.add_argument("--train-steps", type=int, default=40)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--systems", type=int, default=128, help="batch_only: number of batch members")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-hm", action="store_true", help="skip the Hertz-Mindlin workloads")
    ap.add_argument("--hm-steps", type=int, default=0, help="timed steps of a Hertz-Mindlin workload (0: its own)")
    ap.add_argument("--no-learned", action="store_true", help="skip the N=50,000 learned-warm-start line")
    ap.add_argument("--learned-train-runs", type=int, default=12)
    ap.add_argument("--learned-eval-runs", type=int, default=5)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank != 0:
            return
        try:
            items = reference_scenes(args)
            v, th, dt = run_reference(items, steps=args.steps, warmup=args.warmup)
        except Exception as e:  # noqa: BLE001
            print(json.dumps({"impl": "reference", "unavailable": f"reference build not loadable: {e}"}))
            return
        n_total = sum(sc["n"] for _, sc in items)
        sample = (f"all {len(items)} batch systems ({n_total} rods), {args.warmup} untimed + {args.steps} timed "
                  f"steps each, one system after the other; reference src/physics compiled FP32 + OpenMP, "
                  f"spatial hash, plain PSOR ({dt:.1f} s timed)")
        line = {"impl": "reference", "metric": METRIC, "value": round(v, 2), "unit": "rod-steps/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(1000.0 * dt / args.steps, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded RSA packings, Gaussian velocities)",
                "config": headline_config(n_total, len(items)),
                "cpu_baseline": {"value": round(v, 2), "unit": "rod-steps/s", "cores": th, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": round(v, 2), "unit": "rod-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "native_libs": loaded_native_libs()}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    out = run_ours(args, rank, world)
    if rank == 0 and not args.no_cpu_baseline and args.workload == "batch":
        try:
            items = reference_scenes(args, every=4)
            v, th, dt = run_reference(items, steps=4, warmup=1)
            out["cpu_baseline"] = {
                "value": round(v, 2), "unit": "rod-steps/s", "cores": th, "kind": "reference",
                "sample": (f"every 4th batch system by size ({len(items)} systems, "
                           f"{sum(sc['n'] for _, sc in items)} rods), 1 untimed + 4 timed steps each, reference "
                           f"src/physics compiled FP32 + OpenMP, spatial hash, plain PSOR ({dt:.1f} s timed)")}
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
