#!/usr/bin/env python
"""Benchmark of the CAC per-timestep force path on B200.

Workload (default): the mixed-precision configuration at scale -- the EAM
system enlarged to 4,179,600 atoms (129 atomic layers of 32,400) between two
coarse regions of 100,000 8-node elements (9 lattice sites per edge, 2x2x2
Gauss points), 4,979,600 atom+IP sites, under a uniaxial 3 % strain along x
applied as an affine map to atoms, nodes and box; analytic EAM tabulated to
10,000 points, cutoff 5.0 A, skin 1.0 A, list rebuilt every 10 steps, velocity
Verlet at dt = 1 fs from 300 K Maxwell-Boltzmann velocities.  Seeded
synthetic input (no dataset exists for this path).

The line's ``value`` is the mixed form (FP32 pair arithmetic on cell-relative
fixed-point positions; FP64 integration, nodal assembly and energy/virial
sums).  The plain FP64 form runs on the same system in the same process with
the same steps (``fp64``), and the line carries their ratio
(``mixed_over_fp64``) and the mixed form's force error against FP64 on the
seeded state (``accuracy``: largest and RMS per-site force error relative to
the largest FP64 per-site force, nodal forces, energy and virial).  The EAM
workload of 1,049,760 atoms + 20,000 elements (1,209,760 sites) in FP64 is a
second entry (``secondary``).  ``--workload`` / ``--form`` select another
system or form alone (``eam_1m``, ``eam_small``, ``lj_small``, ``batch256``,
``serve``); ``--compare none`` and ``--secondary none`` drop the extra runs.

One step = one velocity-Verlet timestep of the whole system (force evaluation
with both EAM passes, nodal assembly, integration; a list rebuild every 10th
step).  value = atom+IP sites x steps / device time (max over ranks).

The K timed steps run as trajectories of at most ``--segment`` (50) steps,
each restarted from the seeded initial state on the device (state restore,
list build and a force evaluation).  Each trajectory's steps are timed on
the device between CUDA events and the K steps' time is their sum: every
set-up (the first before the timed region, the restarts between the
segments) stays outside, as the reference's "Loop time" of each run starts
after its Verlet::setup.  The reference's own dynamics on these systems gain energy without
bound (its total energy rises by thousands of eV within 300 steps, LJ and EAM
alike), so long trajectories stop being physical; the restarts keep the
timed work on physical configurations.

``--fix langevin`` / ``--fix deform`` time the same trajectories under the
reference's fix langevin (300 K, damp 0.1 ps) or fix deform (x erate 0.1/ps,
y volume; each restart also restores the seeded box); the default is fix nve
alone.  ``thermo_readout_ms`` is the host time of one device thermo read-out.

``--gpus N`` (launched under torchrun) runs N independent replicas, one per
GPU, with no collective on the data path ("replicas only"); value is the sum.

``--impl reference`` times the CAC reference's own CPU path (oracle/_ref/cac,
built from the reference sources with a single-rank MPI stand-in; one core)
on the same workload: ``run W`` then ``run K``, rate from its "Loop time".
At this size a reference step takes seconds, so the reference runs at most
``--ref-max-steps`` timed steps and ``--ref-max-warmup`` warm-up steps; the
line states the requested and the timed counts (``steps_requested``,
``steps``).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom+IP-steps/s"
UNIT = "atom+IP-steps/s"
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "cac")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def batch_share(specs, rank: int, ws: int):
    """Indices of a rank's replicas: greedy split by size (atoms + 8 x elements)."""
    from cac_b200 import shard
    return shard.balanced_partition([ta + 8 * te for ta, te, _, _, _ in specs], ws)[rank]


def build_workload(name: str, seed: int, rank: int = 0, ws: int = 1, replicas: int = 256):
    """A rank's workload.  Single systems: one replica per rank (seeded by
    rank).  Batches: one global set of `replicas` (256) replicas per GPU, split
    over the ranks by the size-balanced greedy rule (each rank builds its own
    share); a smaller set is the first replicas of the full one."""
    from cac_b200 import gen, shard
    if name == "batch256" and ws > 1:
        specs = gen.replica_specs(replicas * ws, seed=13)
        return [gen.replica_from_spec(specs[i]) for i in batch_share(specs, rank, ws)], "eam"
    if name == "eam_1m":
        return gen.eam_1m(seed=seed), "eam"
    if name == "lj_small":
        return gen.lj_small(seed=seed), "lj"
    if name == "eam_small":
        return gen.eam_small(seed=seed), "eam"
    if name == "eam_4m_strained":
        return gen.eam_4m_strained(seed=seed), "eam"
    if name == "batch256":
        return gen.replica_set(replicas, seed=11 + seed), "eam"
    raise SystemExit(f"unknown workload {name}")


def totals(s):
    """(atom+IP sites, atoms, elements) of a system or a list of replicas."""
    items = s if isinstance(s, list) else [s]
    return (sum(r.nsites for r in items), sum(r.natoms for r in items), sum(r.nelements for r in items))


class ClockSampler:
    """Clocks and throttle reasons during the timed region: one ``nvidia-smi
    -lms`` process started before the region and stopped after it."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int, period_ms: int = 100):
        self.gpu = gpu
        self.period_ms = period_ms
        self.samples = []
        self._proc = None
        self._file = None

    def __enter__(self):
        self._file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                           "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                          stdout=self._file, stderr=subprocess.DEVNULL)
        except Exception:
            self._proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.25)
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=10)
            except Exception:
                self._proc.kill()
        self._file.flush()
        self._file.seek(0)
        for line in self._file.read().splitlines():
            parts = [t.strip() for t in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)
        self._file.close()
        os.unlink(self._file.name)

    def summary(self):
        def num(t):
            try:
                return float(t)
            except ValueError:
                return None
        sm = sorted(v for v in (num(s[1]) for s in self.samples) if v is not None)
        mx = [v for v in (num(s[2]) for s in self.samples) if v is not None]
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if s[5 + k].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def max_over_ranks(value: float, dist, device=None) -> float:
    """The largest value over the ranks (the slowest rank's time); the value
    itself without a process group.  `device`: where the collective's tensor
    lives (a CUDA device for NCCL, None for gloo)."""
    if not dist:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, ws: int, seconds: float) -> float:
    """Units all ranks processed (each rank runs its own replica of the same
    size) per second of the slowest rank."""
    return units_per_rank * steps * ws / seconds


def rank_seed(base: int, rank: int) -> int:
    """Seed of a rank's replica: replicas differ, the work per rank does not."""
    return base + rank


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 0, 1, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return rank, local, ws, dist


# ----------------------------------------------------------------- reference arm

def reference_input(d: str, s, pair: str, steps: int, warmup: int) -> None:
    from cac_b200 import gen
    gen.write_data(s, os.path.join(d, "data.cac"))
    lines = ["units metal", "dimension 3", "boundary p p p", "atom_style atomic",
             "element_style cac 8 1 wscale 1 1 1 1", "read_data data.cac"]
    if pair == "eam":
        gen.write_setfl(gen.EamParams(), os.path.join(d, "cu.setfl"))
        lines += ["pair_style eam/alloy", "pair_coeff * * cu.setfl Cu"]
    else:
        lines += ["pair_style lj/cut 5.5", "pair_coeff 1 1 0.4093 2.338"]
    lines += ["neighbor 1.0 bin", "neigh_modify every 10 delay 0 check no", "timestep 0.001",
              "fix 1 all nve", "thermo 1000000"]
    if warmup > 0:
        lines.append(f"run {warmup}")
    lines.append(f"run {steps}")
    with open(os.path.join(d, "in.cac"), "w") as f:
        f.write("\n".join(lines) + "\n")


def run_reference_many(systems, pair: str, steps: int, warmup: int, procs: int, timeout: float = 1800.0):
    """Independent replicas as concurrent single-rank reference processes, at
    most `procs` at a time; returns (sites x steps / s summed over the
    processes, replicas timed)."""
    rate = 0.0
    with tempfile.TemporaryDirectory() as root:
        pending = list(enumerate(systems))
        running = []
        while pending or running:
            while pending and len(running) < procs:
                k, s = pending.pop(0)
                d = os.path.join(root, f"r{k}")
                os.makedirs(d)
                reference_input(d, s, pair, steps, warmup)
                pr = subprocess.Popen([REF_EXE, "-in", "in.cac"], cwd=d, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True)
                running.append((s, pr))
            s, pr = running.pop(0)
            out, _ = pr.communicate(timeout=timeout)
            if pr.returncode != 0:
                raise RuntimeError("reference run failed: " + out[-2000:])
            loops = re.findall(r"Loop time of ([0-9.eE+-]+) on", out)
            rate += s.nsites * steps / float(loops[-1])
    return rate, len(systems)


def run_reference(workload: str, steps: int, warmup: int, seed: int = 2, timeout: float = 1800.0):
    """Time the reference executable: `run warmup` then `run steps`; returns
    (units per step, loop seconds of the timed run, log)."""
    from cac_b200 import gen
    s, pair = build_workload(workload, seed)
    with tempfile.TemporaryDirectory() as d:
        reference_input(d, s, pair, steps, warmup)
        r = subprocess.run([REF_EXE, "-in", "in.cac"], cwd=d, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError("reference run failed: " + r.stdout[-2000:] + r.stderr[-2000:])
        loops = re.findall(r"Loop time of ([0-9.eE+-]+) on", r.stdout)
        return s.nsites, float(loops[-1]), r.stdout


def reference_arm(args, rank, ws):
    if rank != 0:
        return
    if not os.path.exists(REF_EXE):
        print(json.dumps({"impl": "reference", "unavailable": "reference executable oracle/_ref/cac was not built"}))
        return
    steps = min(args.steps, args.ref_max_steps)
    warmup = min(args.warmup, args.ref_max_warmup)
    cores, kind_sample = 1, (f"full workload, run {warmup} then run {steps} steps (of {args.steps} and "
                             f"{args.warmup} requested: at most --ref-max-steps / --ref-max-warmup); rate "
                             f"from Loop time")
    par = "1 core (reference CPU path, single MPI rank)"
    if args.workload.startswith("batch"):
        systems, pair = build_workload(args.workload, 2, replicas=args.replicas)
        cores = min(os.cpu_count() or 1, len(systems))
        sample = systems[:cores]
        value, nrep = run_reference_many(sample, pair, steps, warmup, cores)
        units = totals(systems)[0]
        secs = units * steps / value
        kind_sample = (f"{nrep} of the {len(systems)} replicas as concurrent single-rank processes on {cores} "
                       f"cores, run {warmup} then run {steps} steps each (of {args.steps} and {args.warmup} "
                       f"requested); rate = sum over processes of sites x steps / Loop time")
        par = f"{cores} concurrent single-rank reference processes (one replica each)"
    else:
        units, secs, _ = run_reference(args.workload, steps, warmup)
        value = units * steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warmup, "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": 1000.0 * secs / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator)",
        "config": {"workload": args.workload, "sites": units,
                   "pair": "lj/cut" if args.workload.startswith("lj") else "eam/alloy",
                   "precision": "fp64 (the reference has no other form)", "parallelism": par},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": kind_sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------- b200 arm

def alg_bytes_per_site(kernel: str) -> int:
    """Compulsory state traffic per site and launch (FP64): what the kernel
    must read and write at minimum, independent of the list representation."""
    return {
        "eam_force": 24 + 8 + 24,     # read x, F'; write f
        "eam_rho": 24 + 8,            # read x; write rho
        "pair_lj": 24 + 24,           # read x; write f
        "eam_force32": 16 + 24,       # read fixed-point x + F'; write f (FP64)
        "eam_rho32": 16 + 8 + 4,      # read fixed-point x; write rho, F'
        "pair_lj32": 16 + 24,         # read fixed-point x; write f
        "nve_initial": 72 + 48,       # read x, v, f; write x, v
        "nve_final": 48 + 24,         # read v, f; write v
    }.get(kernel, 0)


# DRAM bytes per site and launch of the dominant kernels, from one ncu capture
# each (dram__bytes_read.sum + dram__bytes_write.sum) on the 313,120-site EAM
# slab, where the whole working set exceeds L2; the list stream grows with the
# sites, so the per-site figure carries over to larger systems of the same
# lattice.
# ncu dram read + write per launch on the 313,120-site slab (profiles/):
# the FP64 force pass (SM-local form), the mixed force and density passes
TRAFFIC_PER_SITE = {"eam_force": 110.80e6 / 313120, "eam_force32": 92.55e6 / 313120,
                    "eam_rho32": 92.36e6 / 313120}


def stream_bytes(kernel: str, na: int, ne: int, nact: int, mixed: bool = False) -> int:
    """Compulsory HBM bytes per launch of the streaming kernels (FP64 state):
    what each must read and write once, with per-element node data counted
    once per element.  The mixed form's pair table is written as 16-byte
    fixed-point records."""
    nsi = na + 8 * ne
    if mixed and kernel == "interpolate":
        # read atom (32) + slot (4), Gauss-point node (24), site id (4) and
        # nodes once per element; write a 16-byte record per entry
        return 52 * na + 40 * 8 * ne + 20 * nact + 192 * ne
    return {
        "nve_initial": 120 * nsi,                       # read x, v, f; write x, v (atoms and nodes)
        "nve_final": 72 * nsi,                          # read v, f; write v
        "interpolate": 68 * na + 56 * 8 * ne + 36 * nact + 192 * ne,   # pair table: atoms, Gauss points, sites
        "assemble": 384 * ne,                           # read Gauss-point forces, write nodal forces
        "pack32": 52 * (nsi + nact),                    # read the pair table, write fixed-point records
        "eam_site_fp": 12 * nact + 64 * ne,             # site ids, nodal density, F'
        "eam_site_fp32": 12 * nact + 64 * ne,
    }.get(kernel, 0)


def alg_flops_per_site(kernel: str) -> int:
    """FP operations per site counted on the reference algorithm's Verlet-list
    candidates at the workloads' density: 78 candidates within cut + skin
    (8 operations each for the separation and r^2) and 42 within the force
    cutoff (12 operations for a density term, 42 for an EAM force term, 12 for
    an LJ term; LJ: 86 and 54)."""
    return {
        "eam_force": 78 * 8 + 42 * 42, "eam_force32": 78 * 8 + 42 * 42,
        "eam_rho": 78 * 8 + 42 * 12, "eam_rho32": 78 * 8 + 42 * 12,
        "pair_lj": 86 * 8 + 54 * 12, "pair_lj32": 86 * 8 + 54 * 12,
    }.get(kernel, 0)


def pipe_peak(fp64: bool, device: int) -> float:
    """Dense GEMM throughput (TFLOP/s) of this GPU in the kernel's arithmetic
    type, measured here through cuBLAS (torch.matmul, TF32 off): the ceiling
    for the pair kernels' FP64 or FP32 arithmetic."""
    import torch
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 4096 if fp64 else 8192
    dt = torch.float64 if fp64 else torch.float32
    a = torch.randn(n, n, dtype=dt, device=torch.device("cuda", device))
    b = torch.randn(n, n, dtype=dt, device=torch.device("cuda", device))
    best = 0.0
    for _ in range(4):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(device)
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) / 1000.0) / 1e12)
    del a, b
    return best


WORK_QUEUE = True   # --work-queue: persistent launches of the mixed EAM passes
PREFIX_MARGIN = None   # --prefix-margin: inner list prefix margin (A; default 0.5 x skin)


def make_engine(s, pair, form: str, local: int, setfl: str, fix: str):
    """A context holding the workload, set up at the seeded state (lists,
    forces) and snapshotted for the restarts."""
    from cac_b200 import api
    eng = api.Engine(local)
    if isinstance(s, list):
        eng.upload_batch(s)
    else:
        eng.upload(s)
    if pair == "eam":
        eng.pair_eam(setfl)
    else:
        eng.pair_lj(0.4093, 2.338, 5.5)
    eng.set_precision(api.MIXED if form == "mixed" else api.FP64)
    eng.neighbor(1.0, 10)
    eng.work_queue(WORK_QUEUE)
    if PREFIX_MARGIN is not None:
        eng.list_prefix(PREFIX_MARGIN)
    if fix == "langevin":
        eng.langevin(300.0, 300.0, 0.1, 4928459)
    elif fix == "deform":
        if isinstance(s, list):
            raise SystemExit("--fix deform times a single system")
        eng.deform(1, x=("erate", 0.1), y=("volume",))
    return eng


class Trajectories:
    """Velocity-Verlet steps as segments of at most `seg` steps, each from
    the seeded initial state (restore + list build + forces; with a deforming
    box, the seeded box too).  `prepare` sets a segment up (the reference's
    Verlet::setup, outside its Loop time); `run` starts from a prepared
    state and sets up every later segment itself."""

    def __init__(self, eng, seg: int, box0=None):
        self.eng, self.seg, self.box0 = eng, seg, box0

    def prepare(self):
        self.eng.restore()
        if self.box0 is not None:
            self.eng.set_box(*self.box0)
        self.eng.setup()

    def run(self, nsteps: int, stream=None):
        """nsteps in segments; with a stream, each segment's steps are
        bracketed by CUDA events on it and the summed device time (ms) is
        returned: the set-up of a later segment (restore, lists, forces) is
        left out, as the reference leaves Verlet::setup out of each run's
        Loop time."""
        import torch
        done, ms = 0, 0.0
        while done < nsteps:
            if done:
                self.prepare()
            k = min(self.seg, nsteps - done)
            if stream is not None:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            self.eng.run_nve(k, 0.001)
            if stream is not None:
                e1.record(stream)
                e1.synchronize()
                ms += e0.elapsed_time(e1)
            done += k
        return ms


def timed_region(eng, tr: Trajectories, steps: int, warmup: int, local: int, dist, clocks: bool):
    """W warm-up steps, then K steps between barriers and synchronisations,
    timed with CUDA events on the context's stream; (slowest rank's ms, clock
    summary or None).  Every segment starts from a state set up outside its
    timer (lists and forces of the seeded state), as the reference's Loop
    time of each run starts after Verlet::setup; the K steps' device time is
    the sum over the segments."""
    import torch
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", local))
    tr.run(warmup)
    tr.prepare()
    torch.cuda.synchronize(local)
    if dist:
        dist.barrier()
    clk = ClockSampler(local) if clocks else None
    if clk:
        clk.__enter__()
    try:
        torch.cuda.synchronize(local)
        if dist:
            dist.barrier()
        ms = tr.run(steps, stream)
        torch.cuda.synchronize(local)
        if dist:
            dist.barrier()
    finally:
        if clk:
            clk.__exit__(None, None, None)
    return max_over_ranks(ms, dist, torch.device("cuda", local)), (clk.summary() if clk else None)


def force_accuracy(ref, mix, nelements: int) -> dict:
    """Mixed against FP64 on the same state: largest and RMS per-site force
    error (atoms and Gauss points) relative to the largest FP64 per-site
    force, the same for nodal forces, and the relative energy and virial
    errors."""
    import numpy as np
    from cac_b200 import api
    for e in (ref, mix):
        e.compute(api.ENERGY_GLOBAL, api.VIRIAL_GLOBAL)
    f64, nf64, gf64 = ref.forces()
    f32, nf32, gf32 = mix.forces()
    site64 = np.concatenate([f64, gf64.reshape(-1, 3)])
    site32 = np.concatenate([f32, gf32.reshape(-1, 3)])
    err = np.linalg.norm(site32 - site64, axis=1) / np.linalg.norm(site64, axis=1).max()
    out = {"force_err_max": float(err.max()), "force_err_rms": float(np.sqrt(np.mean(err ** 2)))}
    if nelements:
        nerr = np.linalg.norm((nf32 - nf64).reshape(-1, 3), axis=1) / np.linalg.norm(nf64.reshape(-1, 3),
                                                                                      axis=1).max()
        out["node_force_err_max"] = float(nerr.max())
    e64, e32 = ref.energy(peratom=False), mix.energy(peratom=False)
    out["energy_rel_err"] = abs(e32["energy"] - e64["energy"]) / abs(e64["energy"])
    out["virial_rel_err"] = float(np.abs(e32["virial"] - e64["virial"]).max() / np.abs(e64["virial"]).max())
    out["against"] = "FP64 form on the same seeded state (same process)"
    return out


def b200_arm(args, rank, local, ws, dist):
    import numpy as np
    import torch
    from cac_b200 import gen, shard

    seed = rank_seed(2, rank)
    s, pair = build_workload(args.workload, seed, rank, ws, replicas=args.replicas)
    units, natoms, nelements = totals(s)
    dev = torch.device("cuda", local)
    units_all = shard.sum_over_ranks(units, dist, dev)
    batch = isinstance(s, list)
    tmp = tempfile.mkdtemp()
    setfl = os.path.join(tmp, "cu.setfl")
    gen.write_setfl(gen.EamParams(), setfl)
    box0 = None
    if args.fix == "deform":
        box0 = (np.asarray(s.boxlo, dtype=np.float64), np.asarray(s.boxhi, dtype=np.float64))
    seg = max(1, min(args.segment, args.steps))
    compare = args.compare == "fp64" and args.form == "mixed"

    # the FP64 form on the same system: accuracy of the mixed form on the
    # seeded state, then its own timed steps
    fp64_entry, accuracy = None, None
    eng = make_engine(s, pair, args.form, local, setfl, args.fix)
    if compare:
        ref = make_engine(s, pair, "fp64", local, setfl, args.fix)
        accuracy = force_accuracy(ref, eng, nelements)
        ref.setup()
        ref.snapshot()
        ms64, clk64 = timed_region(ref, Trajectories(ref, seg, box0), args.steps, args.warmup, local, dist, True)
        fp64_entry = {"value": units_all * args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps,
                      "steps": args.steps, "warmup": args.warmup, "clocks": clk64}
        ref.close()
        del ref
    eng.setup()
    eng.snapshot()
    tr = Trajectories(eng, seg, box0)
    ms_max, clocks = timed_region(eng, tr, args.steps, args.warmup, local, dist, True)
    value = units_all * args.steps / (ms_max / 1000.0)

    # per-kernel device times (CUDA events around every launch) for the roofline
    nprof = min(seg, 50)
    eng.restore()
    eng.setup()
    eng.profile(True)
    eng.run_nve(nprof, 0.001)
    prof = eng.profile_read()
    eng.profile(False)
    # thermo read-out on the device: reduction plus one small copy, host wall time
    eng.thermo()
    t_th = time.perf_counter()
    for _ in range(20):
        eng.thermo()
    thermo_ms = (time.perf_counter() - t_th) / 20 * 1000.0
    timed = {k: v for k, v in prof.items() if alg_bytes_per_site(k) > 0}
    top = max(prof.items(), key=lambda kv: kv[1][0])
    dom = max(timed.items(), key=lambda kv: kv[1][0]) if timed else top
    avg_ms = dom[1][0] / max(dom[1][1], 1)
    nsi = units
    alg = alg_bytes_per_site(dom[0]) * nsi
    hbm, hbm_kind = peaks()
    achieved = alg / (avg_ms / 1000.0) / 1e9
    launches_per_step = sum(v[1] for v in prof.values()) / nprof
    nact = eng.counts()[2]
    hbm_by_kernel = {}
    for k, (tot_ms, nl) in sorted(prof.items()):
        b = stream_bytes(k, natoms, nelements, nact, args.form == "mixed")
        if b and nl:
            gbs = b / (tot_ms / nl / 1000.0) / 1e9
            hbm_by_kernel[k] = {"gbs": gbs, "frac": gbs / hbm, "bytes_per_launch": b}
    traffic = TRAFFIC_PER_SITE[dom[0]] * nsi if dom[0] in TRAFFIC_PER_SITE else None
    pipe = None
    if alg_flops_per_site(dom[0]):
        fp64 = not dom[0].endswith("32")
        peak_tf = pipe_peak(fp64, local)
        got_tf = alg_flops_per_site(dom[0]) * nsi / (avg_ms / 1000.0) / 1e12
        pipe = {"bound": "fp64" if fp64 else "fp32", "kernel": dom[0], "achieved": got_tf, "peak": peak_tf,
                "unit": "TFLOP/s", "frac": got_tf / peak_tf,
                "peak_kind": "measured here: cuBLAS " + ("DGEMM" if fp64 else "SGEMM, TF32 off"),
                "flops_per_site": alg_flops_per_site(dom[0])}
    tuned = eng.pair_blocks()
    work_tiles = eng.work_queue() if batch else None
    eng.restore()
    eng.setup()

    # end to end through the C ABI with pinned host buffers: every step copies the
    # state in (x, v, nodes), runs one step, and reads the state back
    # (cacb200_run_nve_host: the position copy runs beside the step's forces)
    x_h = torch.empty((natoms, 3), dtype=torch.float64).pin_memory().numpy()
    v_h = torch.empty((natoms, 3), dtype=torch.float64).pin_memory().numpy()
    nx_h = torch.empty((nelements, 8, 3), dtype=torch.float64).pin_memory().numpy()
    nv_h = torch.empty((nelements, 8, 3), dtype=torch.float64).pin_memory().numpy()
    x0, v0, nx0, nv0 = eng.state()
    x_h[:] = x0
    v_h[:] = v0
    nx_h[:] = nx0
    nv_h[:] = nv0
    k_e2e = max(5, min(args.steps, seg))
    torch.cuda.synchronize(local)
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        eng.run_nve_host(1, x_h, v_h, nx_h, nv_h, 0.001)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, torch.device("cuda", local))
    e2e_value = units_all * k_e2e / e2e_s
    bytes_state = 8 * (6 * natoms + 48 * nelements)
    eng.close()
    del eng

    # second workloads, each timed alone the same way (value, ms per step)
    secondary = {}
    for spec in ([] if args.secondary == "none" else args.secondary.split(",")):
        wname, wform = spec.split(":")
        s2, pair2 = build_workload(wname, seed, rank, ws, replicas=args.replicas)
        u2 = shard.sum_over_ranks(totals(s2)[0], dist, dev)
        e2 = make_engine(s2, pair2, wform, local, setfl, "none")
        e2.setup()
        e2.snapshot()
        ms2, _ = timed_region(e2, Trajectories(e2, seg), args.steps, args.warmup, local, dist, False)
        secondary[spec] = {"workload": wname, "form": wform, "sites": int(u2),
                           "value": u2 * args.steps / (ms2 / 1000.0), "ms_per_step": ms2 / args.steps,
                           "steps": args.steps, "warmup": args.warmup}
        e2.close()
        del e2, s2

    # CPU baseline: the reference on a bounded sample of the same workload,
    # at N = 1 only (under torchrun the other ranks would wait for rank 0's
    # CPU run in their next collective)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        if os.path.exists(REF_EXE):
            try:
                if batch:
                    cores = min(os.cpu_count() or 1, len(s))
                    rate, nrep = run_reference_many(s[:cores], pair, 10, 0, cores)
                    cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                           "sample": f"{nrep} of the {len(s)} replicas as concurrent single-rank reference "
                                     f"processes, 10 steps each incl. one list rebuild; rate = sum of sites x "
                                     f"steps / Loop time"}
                else:
                    cu, secs, _ = run_reference(args.workload, 10, 0)
                    cpu = {"value": cu * 10 / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                           "sample": "reference executable on the same workload, 10 steps incl. one list "
                                     "rebuild, rate from its Loop time (setup excluded)"}
            except Exception as ex:  # reported, not fatal
                cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "reference executable not built on this host"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32/f64",
            "data": "synthetic (seeded generator; no dataset exists for this path)",
            "config": {"workload": args.workload, "sites": int(units_all), "sites_rank0": units,
                       "atoms_rank0": natoms, "elements_rank0": nelements,
                       "replicas_rank0": len(s) if batch else 1,
                       "pair": "eam/alloy" if pair == "eam" else "lj/cut", "precision": args.form,
                       "rebuild_every": 10,
                       "parallelism": (f"{ws} ranks, replicas split by size (greedy), no data-path collective"
                                       if batch and ws > 1 else f"replicas x{ws} (no data-path collective)"),
                       "fix": {"none": "nve", "langevin": "nve + langevin 300 300 0.1",
                               "deform": "nve + deform 1 x erate 0.1 y volume"}[args.fix],
                       "l2": "working set larger than L2 (site table + lists > 126 MB)",
                       "work_queue": WORK_QUEUE, "prefix_margin": PREFIX_MARGIN},
            "fp64": fp64_entry,
            "mixed_over_fp64": (value / fp64_entry["value"]) if fp64_entry else None,
            "accuracy": accuracy,
            "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": hbm,
                         "peak_kind": hbm_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "traffic_note": "ncu dram read+write per launch, per-site figure "
                                                             "of a 313,120-site capture scaled to this workload",
                         "avg_launch_ms": avg_ms, "alg_bytes_per_launch": alg},
            "pipe_roofline": pipe,
            "kernels_ms_per_launch": {k: v[0] / max(v[1], 1) for k, v in sorted(prof.items())},
            "kernels_ms_per_step": {k: v[0] / nprof for k, v in sorted(prof.items())},
            "hbm_by_kernel": hbm_by_kernel,
            "segment_steps": seg,
            "secondary": secondary,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_state,
                    "d2h_bytes_per_step": bytes_state, "steps": k_e2e},
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "tuned_blocks": dict(zip(("rho", "force"), tuned)),
            "work_queue_tiles": (dict(zip(("below_8192_sites", "below_32768_sites", "larger"), work_tiles))
                                 if work_tiles else None),
            "thermo_readout_ms": thermo_ms,
            "clocks": clocks,
        }
        print(json.dumps(line))


def serve_specs(n: int, seed: int):
    """The serving stream: job sizes (atoms log-uniform 1k-200k, elements
    20-5,000, x-strain U(0, 5 %)), kinds (70 % FIRE to fmax 1e-6 eV/A capped at
    5,000 iterations, from rest; 30 % 2,000-step NVE at 300 K) and Poisson
    arrival times at 50 jobs/s per GPU, all from one seeded generator:
    (arrival, atoms, elements, strain, fire, seed) per job."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for k in range(n):
        ta = int(round(np.exp(rng.uniform(np.log(1000), np.log(200000)))))
        te = int(round(np.exp(rng.uniform(np.log(20), np.log(5000)))))
        st = float(rng.uniform(0.0, 0.05))
        fire = bool(rng.uniform() < 0.7)
        js = int(rng.integers(1 << 30))
        t += float(rng.exponential(1.0 / 50.0))
        out.append((t, ta, te, st, fire, js))
    return out


def serve_jobs(n: int, seed: int, rank: int = 0, ws: int = 1):
    """A rank's share of a stream of n x ws jobs (arrival rate scaled by the
    ranks), split by the size-balanced greedy rule: (arrival, system, fire)."""
    from cac_b200 import gen, shard
    specs = serve_specs(n * ws, seed)
    if ws > 1:
        specs = [(sp[0] / ws,) + tuple(sp[1:]) for sp in specs]
        own = shard.balanced_partition([ta + 8 * te for _, ta, te, _, _, _ in specs], ws)[rank]
        specs = [specs[i] for i in own]
    return [(t, gen.replica(ta, te, temperature=0.0 if fire else 300.0, strain=st, seed=js), fire)
            for t, ta, te, st, fire, js in specs]


def merge_serving(parts):
    """Rank records (latencies, site-steps, FIRE stop codes, failures,
    makespan) merged: sums, the longest makespan, all latencies."""
    lat, site_steps, codes, failed, makespan = [], 0.0, {}, {}, 0.0
    for p in parts:
        lat += list(p["lat"])
        site_steps += p["site_steps"]
        makespan = max(makespan, p["makespan"])
        for k, v in p["codes"].items():
            codes[k] = codes.get(k, 0) + v
        for k, v in p["failed"].items():
            failed[k] = failed.get(k, 0) + v
    return lat, site_steps, codes, failed, makespan


def serve_stream(srv, api, stream, t_scale: float = 1.0):
    """Submit a stream's jobs at their arrival times (scaled by t_scale),
    wait for all; (latencies in arrival order, site-steps, FIRE stop codes,
    failures, makespan)."""
    t0 = time.perf_counter()
    ids = []
    for t_arr, s, fire in stream:
        delay = t_arr * t_scale - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        if fire:
            ids.append(srv.submit(s, api.JOB_FIRE, 5000, 0.001, 0.0, 1e-6))
        else:
            ids.append(srv.submit(s, api.JOB_NVE, 2000, 0.001))
    lat, site_steps, codes, failed = [], 0.0, {}, {}
    for j, (t_arr, s, fire) in zip(ids, stream):
        rc = srv.wait(j)
        if rc != 0:
            msg = srv.last_error()
            failed[msg] = failed.get(msg, 0) + 1
            lat.append(srv.times(j)[2])
            continue
        _, _, _, _, _, it, code, times = srv.result(j)
        lat.append(times[2])
        site_steps += s.nsites * it
        if fire:
            codes[str(code)] = codes.get(str(code), 0) + 1
        srv.release(j)
    return lat, site_steps, codes, failed, time.perf_counter() - t0


def serve_arm(args, rank: int = 0, local: int = 0, ws: int = 1, dist=None):
    """Serve a Poisson stream of jobs at the offered rate (50 jobs/s per GPU);
    report throughput, latency percentiles and the same jobs run one after
    another in FP64 through the single-system engine (on a bounded prefix of
    the stream).  The offered run measures the server's capacity when the
    offered rate exceeds it (saturated: the queue then grows with the stream
    and latencies measure its drain); a second stream at 70 % of that
    capacity gives the steady-state latencies, with the percentiles of its
    first and second halves (by arrival) to show they do not grow.  NVE jobs
    run as restarted trajectories of --segment steps (the reference's
    dynamics heat up without bound on longer runs)."""
    import numpy as np
    from cac_b200 import api, gen, shard
    stream = serve_jobs(args.jobs, 101, rank, ws)
    tmp = tempfile.mkdtemp()
    setfl = os.path.join(tmp, "cu.setfl")
    gen.write_setfl(gen.EamParams(), setfl)

    def set_pair(obj):
        if args.pair == "eam":
            obj.pair_eam(setfl)
        else:
            obj.pair_lj(0.4093, 2.338, 5.5)

    srv = api.Server(local, workers=args.workers, budget_gb=120.0,
                     precision=api.MIXED if args.form == "mixed" else api.FP64)
    set_pair(srv)
    srv.neighbor(1.0, 10)
    srv.segment(args.segment)
    srv.start()
    if dist:
        dist.barrier()
    lat, site_steps, codes, failed, makespan = serve_stream(srv, api, stream)
    parts = shard.gather_objects({"lat": lat, "site_steps": site_steps, "codes": codes, "failed": failed,
                                  "makespan": makespan, "jobs": len(stream)}, dist)
    njobs = sum(p["jobs"] for p in parts)
    lat, site_steps, codes, failed, makespan = merge_serving(parts)
    lat = np.array(lat)
    # capacity and saturation: the offered rate against the rate jobs were served
    offered = 50.0 * ws
    served = njobs / makespan
    saturated = offered > 1.05 * served
    # steady state: a second stream (its own seed) at 70 % of the capacity
    steady = None
    if args.steady_jobs > 0:
        srate = min(offered, 0.7 * served)
        sstream = serve_jobs(args.steady_jobs, 202, rank, ws)
        slat, ssteps, scodes, sfailed, smake = serve_stream(srv, api, sstream, t_scale=offered / srate)
        sparts = shard.gather_objects({"lat": slat, "site_steps": ssteps, "codes": scodes, "failed": sfailed,
                                       "makespan": smake, "jobs": len(sstream)}, dist)
        snj = sum(p["jobs"] for p in sparts)
        slat_all, ssteps, scodes, sfailed, smake = merge_serving(sparts)
        slat_all = np.array(slat_all)
        half = len(slat_all) // 2
        steady = {"arrival_rate_jobs_per_s": srate, "jobs": snj, "jobs_per_s": snj / smake,
                  "latency_p50_s": float(np.percentile(slat_all, 50)),
                  "latency_p99_s": float(np.percentile(slat_all, 99)),
                  "first_half_p50_s": float(np.percentile(slat_all[:half], 50)),
                  "second_half_p50_s": float(np.percentile(slat_all[half:], 50)),
                  "first_half_p99_s": float(np.percentile(slat_all[:half], 99)),
                  "second_half_p99_s": float(np.percentile(slat_all[half:], 99)),
                  "fire_stop_codes": scodes, "failed": sfailed,
                  "value": ssteps / smake}
    srv.close()
    if rank != 0:
        return

    # serial FP64: the same jobs one at a time through one context
    serial_s, nser = 0.0, min(args.serial_jobs, len(stream))
    e = api.Engine(local)
    for t_arr, s, fire in stream[:nser]:
        e.upload(s)
        set_pair(e)
        e.neighbor(1.0, 10)
        e.set_precision(api.FP64)
        a = time.perf_counter()
        try:
            if fire:
                e.minimize_fire(0.0, 1e-6, 5000, 0.001, norm="max")
            else:
                e.snapshot()
                done = 0
                while done < 2000:
                    if done:
                        e.restore()
                    e.setup()
                    k = min(args.segment, 2000 - done)
                    done += k
                    e.run_nve(k, 0.001, eflag=api.ENERGY_GLOBAL if done == 2000 else 0)
                e.energy(peratom=False)
        except api.CacB200Error:
            pass
        serial_s += time.perf_counter() - a
    e.close()
    line = {
        "metric": METRIC, "value": site_steps / makespan, "unit": UNIT, "n_gpus": ws, "steps": None,
        "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.form == "fp64" else "f32/f64",
        "data": "synthetic (seeded generator; no dataset exists for this path)",
        "config": {"workload": "serve", "jobs": njobs, "arrivals": f"Poisson {50 * ws}/s",
                   "parallelism": f"{ws} ranks, jobs split by size (greedy), one server per GPU",
                   "pair": "eam/alloy" if args.pair == "eam" else "lj/cut",
                   "mix": "70% FIRE (ftol 1e-6 max-norm, cap 5000), 30% NVE 2000 steps "
                          f"(restarted every {args.segment})",
                   "workers": args.workers, "budget_gb": 120.0, "precision": args.form},
        "serving": {"offered_jobs_per_s": offered, "saturated": bool(saturated),
                    "capacity_note": ("the offered rate exceeds the server's: jobs queue up and the latencies "
                                      "measure the drain of the stream" if saturated else
                                      "the server keeps up with the offered rate"),
                    "steady": steady,
                    "jobs_per_s": njobs / makespan, "makespan_s": makespan,
                    "latency_p50_s": float(np.percentile(lat, 50)),
                    "latency_p99_s": float(np.percentile(lat, 99)), "fire_stop_codes": codes,
                    "failed": failed,
                    "serial_fp64_jobs_per_s": nser / serial_s if serial_s > 0 else None,
                    "serial_fp64_sample_jobs": nser},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="eam_4m_strained")
    ap.add_argument("--form", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--compare", default="fp64", choices=["fp64", "none"],
                    help="mixed form: also time the FP64 form on the same system and report the ratio "
                         "and the force error")
    ap.add_argument("--secondary", default="eam_1m:fp64",
                    help="comma-separated workload:form entries timed after the main one ('none': skip)")
    ap.add_argument("--ref-max-steps", type=int, default=10,
                    help="reference arm: timed steps at most (a reference step takes seconds at this size)")
    ap.add_argument("--ref-max-warmup", type=int, default=1, help="reference arm: warm-up steps at most")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fix", default="none", choices=["none", "langevin", "deform"],
                    help="integrate with fix langevin or fix deform besides fix nve")
    ap.add_argument("--jobs", type=int, default=64, help="serve workload: jobs in the stream")
    ap.add_argument("--workers", type=int, default=8, help="serve workload: worker contexts")
    ap.add_argument("--steady-jobs", type=int, default=48,
                    help="serve workload: jobs of the second stream, at 70 %% of the measured capacity")
    ap.add_argument("--serial-jobs", type=int, default=8,
                    help="serve workload: jobs of the stream timed one at a time in FP64")
    ap.add_argument("--pair", default="lj", choices=["lj", "eam"], help="serve workload: pair style")
    ap.add_argument("--replicas", type=int, default=256,
                    help="batch workload: replicas per GPU (fewer = the first of the 256; profiling cases)")
    ap.add_argument("--segment", type=int, default=50,
                    help="steps per trajectory from the seeded initial state (the reference's CAC "
                         "dynamics heat up unboundedly after ~100 steps, so long runs restart)")
    ap.add_argument("--work-queue", default="on", choices=["on", "off"],
                    help="mixed EAM passes as persistent launches (batches: work items per replica; "
                         "single systems: SM-local runs of list slots) or one grid launch per pass")
    ap.add_argument("--prefix-margin", type=float, default=None,
                    help="margin of the lists' inner prefix in A (default: the library's, 0.5 x skin; 0: off)")
    args = ap.parse_args()
    global WORK_QUEUE, PREFIX_MARGIN
    WORK_QUEUE = args.work_queue == "on"
    PREFIX_MARGIN = args.prefix_margin
    rank, local, ws, dist = dist_init()
    try:
        if args.impl == "reference":
            reference_arm(args, rank, ws)
        elif args.workload == "serve":
            serve_arm(args, rank, local, ws, dist)
        else:
            b200_arm(args, rank, local, ws, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
