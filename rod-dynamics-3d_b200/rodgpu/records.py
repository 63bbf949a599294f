"""PSOR training records on disk: the data set of the learned warm start.

A record pairs one contact's features at the start of an NSC velocity solve
with the impulse that plain PSOR converged to for it:

  features  float32 [n, 8]  gap phi, v_n, v_t1, v_t2 before the solve, the
                            previous step's (lambda_n, lambda_t1, lambda_t2)
                            for the pair (0 when new), contact-graph degree
  targets   float32 [n, 3]  converged (lambda_n, lambda_t1, lambda_t2)
  run       int32   [n]     index into `runs` of the system that produced it
  step      int32   [n]     step of that run (0-based, in recording order)

File format (".npz", numpy's zip of arrays, readable without this library):
the four arrays above plus `format` = "rodgpu-psor-records/1" and `runs_json`,
a JSON list with one object per run (seed, rods, aspect ratio, volume
fraction, friction, dt, steps, ...).  Several files concatenate with merge().

generate() produces a data set with the library's own plain PSOR: many
seeded systems of the same generator, stepped together in one batch while
recording (the learned-warm-start configuration: N = 50,000, aspect ratio
20, mu ~ U[0.1, 0.8], 200 runs x 200 steps).
"""
import json

import numpy as np

FORMAT = "rodgpu-psor-records/1"


def save(path, features, targets, run, step, runs):
    """Writes one record file (see the module docstring for the layout)."""
    features = np.ascontiguousarray(features, np.float32)
    targets = np.ascontiguousarray(targets, np.float32)
    run = np.ascontiguousarray(run, np.int32)
    step = np.ascontiguousarray(step, np.int32)
    n = len(features)
    if features.shape != (n, 8) or targets.shape != (n, 3) or run.shape != (n,) or step.shape != (n,):
        raise ValueError("records need features [n,8], targets [n,3], run [n], step [n]")
    np.savez(path, format=np.array(FORMAT), features=features, targets=targets, run=run, step=step,
             runs_json=np.array(json.dumps(list(runs))))


def load(path):
    """Reads a record file; returns a dict with the four arrays and 'runs'."""
    with np.load(path, allow_pickle=False) as z:
        if str(z["format"]) != FORMAT:
            raise ValueError(f"{path}: not a {FORMAT} file")
        out = {k: z[k] for k in ("features", "targets", "run", "step")}
        out["runs"] = json.loads(str(z["runs_json"]))
    return out


def merge(datasets):
    """Concatenates loaded data sets, renumbering their runs."""
    feats, targs, runs_idx, steps, runs = [], [], [], [], []
    for d in datasets:
        feats.append(d["features"])
        targs.append(d["targets"])
        runs_idx.append(d["run"] + len(runs))
        steps.append(d["step"])
        runs.extend(d["runs"])
    return {"features": np.concatenate(feats), "targets": np.concatenate(targs), "run": np.concatenate(runs_idx),
            "step": np.concatenate(steps), "runs": runs}


def generate(n_runs, steps, n=50000, ar=20, phi=0.10, mu_range=(0.1, 0.8), seed=0, dt=5e-4, warmup=0,
             record_cap=None, path=None):
    """Records plain-PSOR runs: n_runs seeded systems of n rods (L = 1,
    d = 1/ar, volume fraction phi, packings from the device generator), mu
    drawn per run from U[mu_range], stepped together in one batch for
    `warmup` unrecorded and then `steps` recorded steps.  Returns the data
    set (and writes it when path is given)."""
    from . import Batch, RgConfig, default_config, scene  # noqa: F401
    rng = np.random.default_rng(seed)
    cfgs, scs, runs = [], [], []
    d = 1.0 / ar
    for k in range(n_runs):
        mu = float(rng.uniform(*mu_range))
        s = int(seed * 100003 + k + 1)
        sc = scene.make_rods_device(n, 1.0, d, phi=phi, seed=s, max_attempts=20000)
        kw = dict(model="nsc", dt=dt, nsc_mu=mu, nsc_omega=1.0, nsc_tol=1e-6, nsc_velocity_iters=500,
                  gravity=(0.0, 0.0, 0.0), lin_damp=0.0, ang_damp=0.0)
        kw.update(scene.pbc_kwargs(sc))
        cfgs.append(default_config(n_bodies=sc["n"], **kw))
        scs.append(sc)
        runs.append({"seed": s, "rods": int(sc["n"]), "aspect_ratio": ar, "phi": round(float(sc["phi"]), 5),
                     "mu": mu, "dt": dt, "steps": steps, "warmup": warmup, "generator": "device RSA"})
    b = Batch(cfgs)
    for k, sc in enumerate(scs):
        b.set_bodies(k, sc["radius"], sc["half_height"], sc["mass"], sc["inertia"], sc["restitution"])
        b.set_state(k, sc["x"], sc["q"], sc["v"], sc["w"])
    if warmup:
        b.step(warmup, stats=False)
    cap = record_cap or max(1 << 16, 8 * n * steps // 100)
    for k in range(n_runs):
        b.member(k).mlp_record(True, cap)
    # every NSC step appends one record per velocity-solve contact, in slot
    # order; the per-step contact counts assign each record its step
    per_step = np.zeros((steps, n_runs), np.int64)
    for t in range(steps):
        st = b.step(1)
        per_step[t] = [x["contacts"] for x in st]
    feats, targs, run_idx, step_idx = [], [], [], []
    for k in range(n_runs):
        x, y = b.member(k).mlp_records()
        want = int(per_step[:, k].sum())
        if len(x) != want:
            raise RuntimeError(f"run {k}: {len(x)} records for {want} contacts (raise record_cap)")
        feats.append(x)
        targs.append(y)
        run_idx.append(np.full(len(x), k, np.int32))
        step_idx.append(np.repeat(np.arange(steps, dtype=np.int32), per_step[:, k]))
    b.close()
    out = {"features": np.concatenate(feats), "targets": np.concatenate(targs), "run": np.concatenate(run_idx),
           "step": np.concatenate(step_idx), "runs": runs}
    if path:
        save(path, out["features"], out["targets"], out["run"], out["step"], out["runs"])
    return out
