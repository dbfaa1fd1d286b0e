"""Benchmark of the DEM droplet step (direct O(N^2) path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 65536] [--precision mixed|fp64]

Workload (default): N = 65,536 water droplets in oil, radii lognormal (median
5 um, sigma_ln 0.35, clipped to [1, 30] um), periodic cube at 2 % volume
fraction, overlaps rejected, seed 0; E = 3e5 V/m, eps_oil 2.85, eta_oil 0.06,
eta_water 0.001, dt = 1e-4 s.  One step = collision detection (spatial hash)
+ coalescence when pairs exist + dipole forces + Oseen convection + Euler
update with the periodic wrap, all on the device.

Printed JSON (rank 0, one line):
  value        steps/s of the whole job, inputs resident in HBM (20 timed steps
               after 500 untimed ones and the warm-up, so coalescence happens)
  e2e          steps/s through the public numpy API (host buffers every step:
               detection + forces/convection uploads, results downloaded)
  roofline     the dominant kernel (the longer of the two mixed pair passes)
               against the FP32 pipe; traffic from profiles/traffic.json
  memory_bound hash detection against the measured HBM copy bandwidth
  fp64_gpu     the bit-exact FP64 GPU step on the same state, and the speed-up
  accuracy_mixed_vs_fp64  forces and convection, mixed against FP64
  cpu_baseline the CPU oracle (restatement of the reference kernels, all host
               threads) on a bounded row sample, extrapolated to a full step
Other workloads (--workload): batched (64 boxes), adjoint, tree (Barnes-Hut at
N = 2^20), parity_tree (the reference-parity FP64 tree), correction (Oseen pass
with the periodic-image correction), trajectory (mixed against FP64 over a run).
Multi-GPU (torchrun): every rank integrates its own independent box (replicas;
weak scaling); value sums the ranks' steps/s over the max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "particle-simulator_b200"))

FLOPS_FORCE_PAIR = 33  # algorithmic flops of one force pair (FMA = 2)
FLOPS_OSEEN_PAIR = 34  # algorithmic flops of one Oseen pair
SM_COUNT_B200 = 148
FP32_LANES_PER_SM = 128
PHYS = dict(eps_oil=2.85, eta_oil=0.06, eta_water=0.001, E=3e5)
DT = 1e-4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=65536)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--schedule", default="auto", choices=["auto", "split", "symmetric", "symmetric_plain"],
                    help="mixed passes: auto (default), or force a schedule (symmetric_plain: blocks in the caller's "
                         "droplet order)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="direct: skip the FP64 GPU step and the error report")
    ap.add_argument("--advance", type=int, default=500,
                    help="direct: untimed steps before the warm-up, so that the timed steps include coalescence")
    ap.add_argument("--workload", default="direct",
                    choices=["direct", "batched", "adjoint", "tree", "parity_tree", "correction", "trajectory"],
                    help="direct: one box of --n droplets (default); batched: 64 boxes, N ~ U[1024, 32768] (seed 1); "
                         "adjoint: gradients through 200 steps at N = 16,384; tree: Barnes-Hut at N = 2^20; "
                         "correction: Oseen convection with the periodic-image correction (48^3 grid) at --n; "
                         "trajectory: --traj-steps direct steps in FP64 and mixed from one state, compared")
    ap.add_argument("--traj-steps", type=int, default=1000)
    ap.add_argument("--adjoint-steps", type=int, default=200,
                    help="adjoint: Euler steps per gradient (200: the measured configuration; fewer for a profile)")
    ap.add_argument("--accuracy", action="store_true", help="tree: errors on 4,096 droplets against direct FP64 sums")
    ap.add_argument("--fd", type=int, default=0, help="adjoint: central-difference checks on this many coordinates")
    ap.add_argument("--boxes", type=int, default=64)
    ap.add_argument("--parity-n", default="", help="parity_tree: comma-separated droplet counts (default 100k,250k,500k)")
    ap.add_argument("--parity-mpl", default="", help="parity_tree: comma-separated leaf sizes (default 1,2,4,8,16)")
    return ap.parse_args()


def make_state(n, seed, device="auto"):
    """The seeded lognormal state.  ``device="host"`` runs the overlap search
    with scipy and never loads the CUDA library (the reference arm); the GPU
    search gives the same state."""
    from dem.particle_generator import LognormalDropletGenerator

    g = LognormalDropletGenerator(n, seed=seed, device=device)
    s = g.generate()
    return s.positions, s.radii, g.L


def direct_workload(n):
    """The workload string both arms print for the direct step."""
    return (f"direct DEM step (hash detection + merge + dipole force + Oseen convection + Euler), N={n}, "
            f"periodic, 2% volume fraction, dt=1e-4")


def mapped_libraries():
    """Shared objects under this repository that the process has mapped."""
    root = str(ROOT)
    seen = []
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                path = ln.split()[-1] if ln.strip() else ""
                if path.startswith(root) and path.endswith(".so") and path not in seen:
                    seen.append(path)
    except OSError:
        return None
    return [str(Path(p).relative_to(ROOT)) for p in seen]


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(mx)) if mx else None,
            "power_w_median": float(np.median(power)) if power else None,
            "samples": len(sm),
            "reasons": sorted(reasons),
        }


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
class DeviceStepper:
    """Device-resident direct DEM step through the library's C ABI."""

    def __init__(self, pos, r, L, precision, device, track=False, schedule="auto"):
        import torch

        from dem.collision_detector import SpatialHashCollisionDetector
        from dem.force_calculator import DirectDropletForceCalculator

        self.torch = torch
        n = len(r)
        self.fc = DirectDropletForceCalculator(num_particles=n, L=L, boundary_mode="periodic", precision=precision,
                                               device=device, **PHYS)
        self.det = SpatialHashCollisionDetector(num_particles=n, L=L, boundary_mode="periodic", device=device)
        self.ctx = self.fc._ctx
        if precision == "mixed" and schedule != "auto":
            self.fc.set_tuning(schedule=schedule)
        self.L = L
        eta_o, eta_w = PHYS["eta_oil"], PHYS["eta_water"]
        self.stokes = 2 * np.pi * eta_o * (2 * eta_o + 3 * eta_w) / (eta_o + eta_w)
        self.dev = self.ctx.device
        self.pos = [torch.empty((3, n), dtype=torch.float64, device=self.dev) for _ in range(2)]
        self.r = [torch.as_tensor(r, device=self.dev).clone(), torch.empty(n, dtype=torch.float64, device=self.dev)]
        self.ctx.aos_to_soa(n, torch.as_tensor(pos, device=self.dev), self.pos[0])
        self.cur, self.rc, self.n = 0, 0, n
        self.n_out = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.merges = 0
        self.launches_per_step = None
        # track: the detected pair sets per step and the droplets' original ids (merged droplets get new ids)
        self.track = track
        self.steps_done = 0
        self.pair_log = []
        self.ids = np.arange(n)
        self.next_id = n
        self.merged = torch.empty((max(n, 1), 2), dtype=torch.int32, device=self.dev) if track else None

    def step(self):
        n, pos, r = self.n, self.pos[self.cur], self.r[self.rc]
        k, pairs, counts = self.det.detect_device(n, pos, r, self.L, True)
        if k > 0:  # coalescence, then detect again at the same time (reference semantics)
            nxt = 1 - self.cur
            self.ctx.merge(n, pos, r, pairs, counts, self.pos[nxt], self.r[1 - self.rc], self.n_out, self.merged)
            self.n = int(self.n_out.item())
            if self.track:
                self.pair_log.append((self.steps_done, pairs.cpu().numpy().copy()))
                m = self.merged[: n - self.n].cpu().numpy()
                gone = np.zeros(n, dtype=bool)
                gone[m.ravel()] = True
                new = np.arange(self.next_id, self.next_id + len(m))
                self.next_id += len(m)
                self.ids = np.concatenate([self.ids[~gone], new])
            self.cur, self.rc = nxt, 1 - self.rc
            self.merges += 1
            return self.step()
        F, V = self.fc.forces_and_convection_soa(n, pos, r)
        nxt = 1 - self.cur
        self.ctx.euler_update(n, pos, r, F, V, self.stokes, DT, self.L, True, self.pos[nxt])
        self.cur = nxt
        self.steps_done += 1

    def positions(self):
        return self.pos[self.cur][:, : self.n].T.cpu().numpy()


def flush_l2(buf):
    buf.fill_(1)


HBM_FALLBACK_GBS = 6650.0  # an earlier STREAM-style copy on this pool's B200s, used when no measured file exists


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json when
    present, else the fallback figure."""
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        for k in ("hbm_gbs", "hbm_GBs", "hbm"):
            if k in d and d[k]:
                return float(d[k]), "measured (MEASURED_PEAKS.json)"
    except Exception:
        pass
    return HBM_FALLBACK_GBS, "fallback (no MEASURED_PEAKS.json)"


# Algorithmic bytes of the memory-bound kernels (what a kernel that touches
# every input and output once would move):
#   hash detection (csrc/hash.cu): per droplet its position and radius (32 B
#     read), its bucket id (4 B written, 4 B read) and bucket slot (4 B written,
#     4 B read); per table slot its start (4 B written, 4 B read); 8 B per pair.
#   Morton build (csrc/bh.cu): per droplet positions (24 B read), key (4 B
#     written), 4 radix passes over (key, index) (16 B each), the gather of
#     position and radius into key order (32 B read, 32 B written); per node its
#     records (~140 B written).
def hash_bytes(n, table, pairs):
    return 48 * n + 8 * table + 8 * pairs


def morton_build_bytes(n, nodes):
    return (24 + 4 + 4 * 16 + 64) * n + 140 * nodes


def hbm_entry(name, ms, nbytes, peak, src, formula):
    gbs = nbytes / (ms * 1e-3) / 1e9 if ms else None
    return {"kernel": name, "ms_per_launch": ms, "algorithmic_bytes": nbytes, "formula": formula,
            "achieved_gbs": gbs, "peak_gbs": peak, "peak_source": src,
            "frac": gbs / peak if gbs else None}


def time_steps(st, steps, flush, stream, sizes=None):
    """CUDA-event time of each of ``steps`` steps, L2 flushed before each one
    (outside the events); returns (per-step ms, merges inside the window).
    ``sizes`` (a list) receives each step's droplet count after its merges: the
    N of that step's pair passes."""
    import torch

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    m0 = st.merges
    torch.cuda.synchronize()
    for k in range(steps):
        flush_l2(flush)  # every step starts with a cold L2
        ev[k][0].record(stream)
        st.step()
        ev[k][1].record(stream)
        if sizes is not None:
            sizes.append(st.n)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev], st.merges - m0


def mixed_vs_fp64(st, device):
    """Forces and convection of the mixed and the FP64 GPU passes on the
    stepper's current state: norm-wise relative error and the reference's
    per-droplet metric |d|/(|ref| + 0.01 mean|ref|) (benchmarks/test.py:63-77)."""
    import torch

    from dem.force_calculator import DirectDropletForceCalculator

    n = st.n
    pos, r = st.pos[st.cur], st.r[st.rc]
    out = {}
    for prec in ("fp64", "mixed"):
        fc = DirectDropletForceCalculator(num_particles=n, L=st.L, boundary_mode="periodic", precision=prec,
                                          device=device, **PHYS)
        F, V = fc.forces_and_convection_soa(n, pos, r)
        out[prec] = (F[:, :n].T.cpu().numpy().copy(), V[:, :n].T.cpu().numpy().copy())
    torch.cuda.synchronize()

    def errs(a, b):
        d = np.linalg.norm(a - b, axis=1)
        nb = np.linalg.norm(b, axis=1)
        e = d / (nb + 0.01 * nb.mean())
        return {"rel_norm": float(np.linalg.norm(a - b) / np.linalg.norm(b)), "ref_metric_mean": float(e.mean()),
                "ref_metric_max": float(e.max())}

    return {"forces": errs(out["mixed"][0], out["fp64"][0]), "convection": errs(out["mixed"][1], out["fp64"][1]),
            "state": f"the state after the timed steps ({n} droplets)"}


def run_ours(args, rank, world, device):
    import torch

    torch.cuda.set_device(device)
    from dem.replicas import replica_seed

    pos, r, L = make_state(args.n, replica_seed(args.seed, rank))
    n = len(r)
    st = DeviceStepper(pos, r, L, args.precision, device, schedule=args.schedule)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)  # > 126 MB L2
    for _ in range(args.advance):  # untimed: the timed window lies where droplets have begun to coalesce
        st.step()
    merges_advance = st.merges
    for _ in range(args.warmup):
        st.step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.4)
    st.ctx.profile(True)
    st.det._ctx.profile(True)  # the detector has its own context
    from dem._native import launch_count

    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    launches0 = launch_count()
    n_timed = []
    step_ms, merges_timed = time_steps(st, args.steps, flush, stream, n_timed)
    launches = launch_count() - launches0
    total_ms = float(sum(step_ms))
    kern = {}
    for c, names in ((st.ctx, ("mixed_force_pass", "mixed_convection_pass", "fp64_force_pass", "fp64_convection_pass")),
                     (st.det._ctx, ("hash_detect",))):
        for name in names:
            ms, cnt = c.profile_read(name)
            if cnt:
                kern[name] = (ms, cnt)
    st.ctx.profile(False)
    st.det._ctx.profile(False)
    schedule = st.ctx.plan(st.n, True) if args.precision == "mixed" else "fp64"
    clocks = sampler.stop() if sampler else None
    from dem.replicas import job_time_ms

    job_ms = job_time_ms(total_ms, device)
    if world > 1:
        torch.distributed.barrier()
    res = dict(n=n, n_timed=n_timed, n_final=st.n, L=L, total_ms=job_ms, step_ms=step_ms, kern=kern, clocks=clocks,
               merges=st.merges, merges_advance=merges_advance, merges_timed=merges_timed, pos=pos, r=r,
               launches=launches, schedule=schedule)
    if args.precision == "mixed" and not args.no_fp64 and rank == 0:
        # the second half of the metric: the plain FP64 GPU step from the same state, timed the same way,
        # and the mixed passes' error against it on that state
        res["accuracy"] = mixed_vs_fp64(st, device)
        st64 = DeviceStepper(st.positions(), st.r[st.rc][: st.n].cpu().numpy(), L, "fp64", device)
        for _ in range(2):
            st64.step()
        k64 = max(3, min(args.steps, 10))
        ms64, m64 = time_steps(st64, k64, flush, stream)
        res["fp64"] = dict(steps=k64, ms_per_step=float(np.mean(ms64)), merges=m64)
    return res


def run_e2e(args, device, steps, warmup):
    """The reference's solver loop (euler_droplet_solver.py:97-131) driving the
    drop-in detector and calculator through their numpy API: host state,
    uploads and downloads on every step."""
    import torch

    from dem.collision_detector import SpatialHashCollisionDetector
    from dem.force_calculator import DirectDropletForceCalculator
    from dem.solution.droplet_solution import merge_droplets

    pos, r, L = make_state(args.n, args.seed)
    n = len(r)
    fc = DirectDropletForceCalculator(num_particles=n, L=L, boundary_mode="periodic", precision=args.precision,
                                      device=device, **PHYS)
    det = SpatialHashCollisionDetector(num_particles=n, L=L, boundary_mode="periodic", device=device)
    eta_o, eta_w = PHYS["eta_oil"], PHYS["eta_water"]
    stokes = 2 * np.pi * eta_o * (2 * eta_o + 3 * eta_w) / (eta_o + eta_w)

    def one(pos, r):
        while True:
            hit, pairs = det.detect(pos, r)
            if not hit:
                break
            pos, r = merge_droplets(pos, r, pairs)
        F, V = fc.calculate_forces_and_convection(pos, r)
        pos = pos + (F / (stokes * r[:, None]) + V) * DT
        pos %= L
        return pos, r

    for _ in range(warmup):
        pos, r = one(pos, r)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        pos, r = one(pos, r)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    n = len(r)
    return dict(steps_per_s=steps / dt, h2d=2 * n * 32, d2h=n * 48 + 16)


# ---------------------------------------------------------------------------
# CPU oracle (reference algorithm restated in C, all host threads)
# ---------------------------------------------------------------------------
def cpu_step_rate(pos, r, L, budget_s, threads=0):
    """Times hash detection (full) and the two O(N^2) passes on a row sample
    sized to ~budget_s, and extrapolates the time of one full step."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    m, eta, stokes = O.physics_constants(**PHYS)
    n = len(r)
    cores = O.max_threads() if threads <= 0 else threads
    t0 = time.perf_counter()
    O.hash_detect(pos, r, L, True, table_size=O.next_power_of_2(2 * n))
    t_hash = time.perf_counter() - t0
    # calibrate on a small sample, then size the timed sample
    rows = max(cores * 4, 64)
    t0 = time.perf_counter()
    F = O.direct_forces(pos, r, m, L, True, rows=(0, rows), threads=threads)
    O.direct_convection(pos, F, eta, L, True, rows=(0, rows), threads=threads)
    per_row = (time.perf_counter() - t0) / rows
    # timed sample: consecutive row chunks until the budget is spent (or every row is done)
    chunk = int(min(n, max(rows, 0.25 * budget_s / max(per_row, 1e-9))))
    rows, t_rows = 0, 0.0
    while rows < n and t_rows < budget_s:
        r1 = min(n, rows + chunk)
        t0 = time.perf_counter()
        F = O.direct_forces(pos, r, m, L, True, rows=(rows, r1), threads=threads)
        O.direct_convection(pos, F, eta, L, True, rows=(rows, r1), threads=threads)
        t_rows += time.perf_counter() - t0
        rows = r1
    t0 = time.perf_counter()
    O.euler_direct(pos, r, np.zeros((n, 3)), np.zeros((n, 3)), stokes, DT, L, True)
    t_euler = time.perf_counter() - t0
    t_step = t_hash + t_rows * (n / rows) + t_euler
    return dict(steps_per_s=1.0 / t_step, cores=cores, rows=rows, sample_s=t_rows + t_hash + t_euler,
                pairs_per_s=n * (n - 1) / t_step)


def cpu_full_step(pos, r, L, O, consts, table):
    """One whole step of the reference's loop (euler_droplet_solver.py:97-139)
    on the oracle kernels: detect, merge and detect again while pairs exist,
    then forces, convection and the Euler update with the periodic wrap."""
    m, eta, stokes = consts
    merges = 0
    while True:
        hit, pairs = O.hash_detect(pos, r, L, True, table_size=table)
        if not hit:
            break
        pos, r, _ = O.merge(pos, r, pairs)
        merges += 1
    F = O.direct_forces(pos, r, m, L, True)
    V = O.direct_convection(pos, F, eta, L, True)
    return O.euler_direct(pos, r, F, V, stokes, DT, L, True), r, merges


def run_reference(args, rank, world):
    """The reference's algorithm on the host cores: the C restatement of its
    kernels (oracle/dem_oracle.c, all host threads), whole steps of the direct
    loop on the same seeded state, timed one by one.  It loads no CUDA code of
    this repository (the state comes from the host overlap search)."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    pos, r, L = make_state(args.n, args.seed, device="host")
    n = len(r)
    consts = O.physics_constants(**PHYS)
    table = O.next_power_of_2(2 * n)
    merges = 0
    for _ in range(args.warmup):
        pos, r, k = cpu_full_step(pos, r, L, O, consts, table)
        merges += k
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        pos, r, k = cpu_full_step(pos, r, L, O, consts, table)
        times.append(time.perf_counter() - t0)
        merges += k
    total = float(sum(times))
    sps = args.steps / total
    cores = O.max_threads()
    line = {
        "impl": "reference",
        "metric": f"DEM steps/s (direct, N={n})",
        "value": sps,
        "unit": "steps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction)",
        "config": {"workload": direct_workload(n), "precision": "fp64 (the reference's arithmetic)",
                   "pairs_per_s": sps * n * (n - 1), "merges_in_timed_and_warmup": merges, "n_final": len(r),
                   "in_tree_libraries_mapped": mapped_libraries()},
        "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} whole steps (detection, merges, both O(N^2) passes over all {n} "
                                   f"droplets, Euler) of the C restatement of the reference kernels"},
        "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# ensembles of independent boxes (main_multi.py-style)
# ---------------------------------------------------------------------------
def make_ensemble_states(boxes, seed=1):
    """Box sizes N_b ~ U[1024, 32768] (seed 1); each box seeded lognormal droplets
    at 2 % volume fraction with its own side."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1024, 32768, size=boxes, endpoint=True)
    states, Ls = [], []
    for b, nb in enumerate(sizes):
        pos, r, L = make_state(int(nb), seed * 1000 + b)
        states.append((pos, r))
        Ls.append(L)
    return states, np.array(Ls)


def run_batched(args, rank, world, device):
    import torch

    from dem._native import launch_count
    from dem.ensemble import DropletEnsemble

    torch.cuda.set_device(device)
    from dem.replicas import replica_seed

    states, Ls = make_ensemble_states(args.boxes, replica_seed(1, rank))
    ens = DropletEnsemble(states, Ls, device=device, **PHYS)
    tune = ens.autotune(reps=2)
    K, W = args.steps, args.warmup
    stream = torch.cuda.current_stream()
    ens.step(DT, steps=W, graph=True)  # capture + warm-up replays
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.4)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0 = launch_count()
    e0.record(stream)
    ens.step(DT, steps=K, graph=True)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = launch_count() - c0
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop() if sampler else None
    # the same steps as 64 sequential chains of plain per-box launches
    seq = DropletEnsemble(states, Ls, device=device, **PHYS)
    seq.ctx.set_tuning(i_per_thread=tune["i_per_thread"], schedule="symmetric")
    seq.step_sequential(DT, steps=1)
    torch.cuda.synchronize()
    ks = max(1, min(K, 10))
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    seq.step_sequential(DT, steps=ks)
    s1.record(stream)
    torch.cuda.synchronize()
    seq_ms = s0.elapsed_time(s1) / ks
    from dem.replicas import job_time_ms

    sizes = np.diff(ens.offsets)
    return dict(ms=job_time_ms(ms, device), seq_ms=seq_ms, tune=tune, launches=launches, clocks=clocks, sizes=sizes,
                errors=ens.ctx.device_errors())


def report_batched(args, res, world):
    K = args.steps
    sizes = res["sizes"]
    pairs = float(np.sum(sizes * (sizes - 1)))
    step_ms = res["ms"] / K
    sps = K * world / (res["ms"] / 1000.0)
    flops = (FLOPS_FORCE_PAIR + FLOPS_OSEEN_PAIR) * pairs
    clocks = res["clocks"] or {}
    max_mhz = clocks.get("sm_max_mhz") or 1965.0
    peak = SM_COUNT_B200 * FP32_LANES_PER_SM * 2 * max_mhz * 1e6 / 1e12
    achieved = flops / (step_ms / 1000.0) / 1e12
    line = {
        "metric": f"DEM ensemble steps/s ({len(sizes)} boxes, direct mixed)",
        "value": sps,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 pair terms + f64 near pairs/sums",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction per box)",
        "config": {
            "workload": f"{len(sizes)} independent periodic boxes, N_b ~ U[1024, 32768] (seed 1), "
                        f"{int(sizes.sum())} droplets; one step = forces + convection + Euler of every box, "
                        "CUDA-graph replay",
            "pairs_per_s": sps * pairs,
            "sequential_ms_per_step": res["seq_ms"],
            "speedup_vs_sequential_per_box_launches": res["seq_ms"] / step_ms,
            "tuning": res["tune"],
            "l2": "not flushed: the step's partial sums and inputs exceed the 126 MB L2",
        },
        "roofline": {
            "kernel": "whole step (both pair passes dominate)",
            "bound": "fp32_pipe",
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved / peak,
            "traffic": ncu_traffic("batched_step_pair_passes"),
            "flops_per_pair": FLOPS_FORCE_PAIR + FLOPS_OSEEN_PAIR,
            "units_per_launch": f"sum_b N_b(N_b-1) = {int(pairs)} ordered pairs per step",
        },
        "clocks": clocks,
        "gpu_launches": res["launches"],
        "device_errors": res["errors"],
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# adjoint: gradients through the direct steps
# ---------------------------------------------------------------------------
def run_adjoint(args, device):
    """N = 16,384 mixed-precision forward, 200 Euler steps with collisions frozen,
    loss = mean squared z displacement + sum over pairs of
    softplus((2.5 (r_i + r_j) - |r_ij|) / 1 um); gradients with respect to the
    initial positions, the radii and |E| through the VJP kernel, a checkpoint
    every 20 steps.  Optionally checked against FP64 central differences."""
    import torch

    from dem.adjoint import DirectTrajectory, mean_squared_z_displacement, pair_softplus

    torch.cuda.set_device(device)
    n = 16384
    pos, r, L = make_state(n, 0)
    x0 = torch.tensor(pos, dtype=torch.float64, device=device)
    rr = torch.tensor(r, dtype=torch.float64, device=device)
    E0 = torch.tensor(PHYS["E"], dtype=torch.float64, device=device)
    steps = args.adjoint_steps
    phys = dict(eps_oil=PHYS["eps_oil"], eta_oil=PHYS["eta_oil"], eta_water=PHYS["eta_water"])

    def loss(sim, x, rad, E):
        xT, D = sim(x, rad, E)
        return mean_squared_z_displacement(D) + pair_softplus(xT, rad, L)

    sim = DirectTrajectory(L, steps, DT, checkpoint_every=20, precision="mixed", device=device, **phys)
    times = []
    for k in range(max(args.warmup, 1) + max(args.steps, 1)):
        xg, rg, Eg = x0.clone().requires_grad_(), rr.clone().requires_grad_(), E0.clone().requires_grad_()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t2 = torch.cuda.Event(enable_timing=True)
        t0.record()
        val = loss(sim, xg, rg, Eg)
        t1.record()
        gx, gr, gE = torch.autograd.grad(val, (xg, rg, Eg))
        t2.record()
        torch.cuda.synchronize()
        if k >= max(args.warmup, 1):
            times.append((t0.elapsed_time(t1), t1.elapsed_time(t2)))
        if k == max(args.warmup, 1) - 1:  # the timed gradients: per-kernel events on the trajectory's context
            sim._ctx.profile(True)
            sim._ctx.profile_reset()
    vjp_ms, vjp_launches = sim._ctx.profile_read("vjp_pass")
    sim._ctx.profile(False)
    fwd = float(np.median([a for a, _ in times]))
    bwd = float(np.median([b for _, b in times]))
    out = dict(n=n, steps=steps, forward_ms=fwd, backward_ms=bwd, loss=float(val.detach()),
               vjp_pass_ms_per_launch=vjp_ms / max(vjp_launches, 1), vjp_pass_launches=vjp_launches)
    if args.fd > 0:
        # Central differences need a smooth forward map.  In a periodic box the
        # minimum image of a pair switches when a separation crosses L/2 (about
        # 20 pairs per step at this N), a jump the adjoint treats as an event, so
        # the check runs in the open box, where the map is smooth away from the
        # contact cut; h = 1e-9 m and h / 2 must agree for the check to count.
        res = {}
        for prec in ("fp64", "mixed"):
            simo = DirectTrajectory(L, steps, DT, checkpoint_every=20, precision=prec, device=device,
                                    boundary_mode="open", **phys)

            def lossf(x, rad, E, simo=simo):
                xT, D = simo(x, rad, E)
                return mean_squared_z_displacement(D) + pair_softplus(xT, rad, L, periodic=False)

            xg = x0.clone().requires_grad_()
            res[prec] = (simo, lossf, torch.autograd.grad(lossf(xg, rr, E0), (xg,))[0])
        lossf64 = res["fp64"][1]
        rng = np.random.default_rng(7)
        fd, fd2, ad64, admx = [], [], [], []
        with torch.no_grad():
            for i, c in zip(rng.integers(0, n, args.fd), rng.integers(0, 3, args.fd)):
                vals = []
                for h in (1e-9, 5e-10):
                    xp, xm = x0.clone(), x0.clone()
                    xp[i, c] += h
                    xm[i, c] -= h
                    vals.append(float(lossf64(xp, rr, E0) - lossf64(xm, rr, E0)) / (2 * h))
                fd.append(vals[0])
                fd2.append(vals[1])
                ad64.append(float(res["fp64"][2][i, c]))
                admx.append(float(res["mixed"][2][i, c]))
        fd, fd2, ad64, admx = map(np.array, (fd, fd2, ad64, admx))

        def rel(a, b):
            return float(np.linalg.norm(a - b) / np.linalg.norm(b))

        out.update(fd_coordinates=args.fd, fd_h=1e-9, fd_boundary="open", fd_h_vs_half_h=rel(fd2, fd),
                   fd_rel_err_fp64_forward=rel(ad64, fd), fd_rel_err_mixed_forward=rel(admx, fd),
                   fd_max_err_over_max_fp64_forward=float(np.abs(ad64 - fd).max() / np.abs(fd).max()))
    return out


# FP64 operations of vjp_pair_kernel per ordered pair (adds and multiplies 1, FMA 2), counted
# from its source: separation and |d|^-1 (Newton) 20, force-term Hessian and radius terms 76,
# the two Oseen K terms 90
FLOPS_VJP_PAIR = 186
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12  # SMs x FP64 lanes x 2 flop x max SM clock


def ncu_traffic(kernel):
    """DRAM bytes (read + write) per launch of a kernel from one ncu capture
    (profiles/traffic.json, written from the captures summarised in profiles/), or None."""
    prof = ROOT / "profiles" / "traffic.json"
    try:
        return json.loads(prof.read_text()).get(kernel)
    except (OSError, ValueError):
        return None


def report_adjoint(args, res):
    total = res["forward_ms"] + res["backward_ms"]
    n, steps = res["n"], res["steps"]
    vjp_ms = res["vjp_pass_ms_per_launch"]
    achieved = FLOPS_VJP_PAIR * n * (n - 1) / (vjp_ms * 1e-3) / 1e12 if vjp_ms > 0 else 0.0
    line = {
        "metric": f"DEM adjoint: gradient evaluations/s (N={n}, {steps} steps)",
        "value": 1000.0 / total,
        "unit": "gradients/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "forward f32 pair terms + f64 near pairs/sums; VJP f64",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction)",
        "config": {"workload": f"adjoint: {steps} Euler steps at N={n}, collisions frozen, checkpoint every 20 "
                               "steps; loss = mean squared z displacement + pair softplus((2.5 (r_i+r_j) - |r_ij|) "
                               "/ 1 um); gradients w.r.t. initial positions, radii and |E|",
                   **res},
        "roofline": {"kernel": "vjp_pass (vjp_pair_kernel + its fixed-order finish)", "bound": "fp64_pipe",
                     "achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
                     "frac": achieved / FP64_PEAK_TFLOPS,
                     "peak_source": "148 SMs x 64 FP64 lanes x 2 flop x 1965 MHz (max SM clock); "
                                    "MEASURED_PEAKS.json holds no FP64 figure",
                     "flops_per_pair": FLOPS_VJP_PAIR, "units_per_launch": f"N(N-1) = {n * (n - 1)} ordered pairs",
                     "traffic": ncu_traffic("vjp_pass") if n == 16384 else None},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Barnes-Hut step (main_tree.py-style) at N = 2^20
# ---------------------------------------------------------------------------
TREE_THETA, TREE_LEAF = 0.5, 16
FLOPS_LEAF_PAIR = 33  # as a force pair
FLOPS_NODE_TERM = 33 + 70  # monopole + quadrupole correction (force walk)


def run_tree(args, device):
    import torch

    from dem.collision_detector import SpatialHashCollisionDetector
    from dem.octree import MortonTreeForceCalculator

    torch.cuda.set_device(device)
    n = 1 << 20
    pos, r, L = make_state(n, 0)
    tc = MortonTreeForceCalculator(num_particles=n, theta=TREE_THETA, mpl=TREE_LEAF, L=L, periodic=True,
                                   device=device, **PHYS)
    det = SpatialHashCollisionDetector(num_particles=n, L=L, boundary_mode="periodic", device=device)
    ctx = tc._ctx
    eta_o, eta_w = PHYS["eta_oil"], PHYS["eta_water"]
    stokes = 2 * np.pi * eta_o * (2 * eta_o + 3 * eta_w) / (eta_o + eta_w)
    p = [torch.empty((3, n), dtype=torch.float64, device=device) for _ in range(2)]
    rr = [torch.as_tensor(r, device=device).clone(), torch.empty(n, dtype=torch.float64, device=device)]
    ctx.aos_to_soa(n, torch.as_tensor(pos, device=device), p[0])
    n_out = torch.zeros(1, dtype=torch.int32, device=device)
    state = dict(cur=0, rc=0, n=n, merges=0)

    def step():
        cur, rc, m = state["cur"], state["rc"], state["n"]
        k, pairs, counts = det.detect_device(m, p[cur], rr[rc], L, True)
        while k > 0:  # coalescence, then detect again (euler_droplet_solver.py:97-110)
            ctx.merge(m, p[cur], rr[rc], pairs, counts, p[1 - cur], rr[1 - rc], n_out)
            m = int(n_out.item())
            cur, rc = 1 - cur, 1 - rc
            state["merges"] += 1
            k, pairs, counts = det.detect_device(m, p[cur], rr[rc], L, True)
        V = tc.forces_and_total_velocity_soa(m, p[cur], rr[rc], stokes)
        ctx.euler_update_total(m, p[cur], V, DT, L, True, p[1 - cur])
        state.update(cur=1 - cur, rc=rc, n=m)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.4)
    from dem._native import launch_count

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    c0 = launch_count()
    ctx.profile(True)
    det._ctx.profile(True)  # the detector has its own context
    for k in range(args.steps):
        ev[k][0].record()
        step()
        ev[k][1].record()
    torch.cuda.synchronize()
    launches = launch_count() - c0
    kern = {}
    for c, names in ((ctx, ("bh_build", "bh_force_walk", "bh_velocity_walk")), (det._ctx, ("hash_detect",))):
        for name in names:
            ms, cnt = c.profile_read(name)
            if cnt:
                kern[name] = ms / cnt
    ctx.profile(False)
    det._ctx.profile(False)
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    st = tc.stats()  # counters of the last walk (velocity); the force walk visits the same tree
    out = dict(n=n, n_final=state["n"], merges=state["merges"], total_ms=float(sum(step_ms)), kern=kern,
               clocks=clocks, launches=launches, stats=st, L=L)
    if args.accuracy:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        m_const, eta, _ = O.physics_constants(**PHYS)
        rows = (0, 4096)
        tc0 = MortonTreeForceCalculator(num_particles=n, theta=TREE_THETA, mpl=TREE_LEAF, L=L, periodic=True,
                                        device=device, **PHYS)
        F, V = tc0.calculate_forces_and_convection(pos, r)
        F_ref = O.direct_forces(pos, r, m_const, L, True, rows=rows)[: rows[1]]
        V_ref = O.direct_convection(pos, F, eta, L, True, rows=rows)[: rows[1]]
        d = np.linalg.norm(F[: rows[1]] - F_ref, axis=1)
        nb = np.linalg.norm(F_ref, axis=1)
        out["accuracy"] = {
            "sample": "droplets 0..4095 of the seeded state (i.i.d. positions), direct FP64 sums over all 2^20",
            "force_rel_norm": float(np.linalg.norm(F[: rows[1]] - F_ref) / np.linalg.norm(F_ref)),
            "force_ref_metric_mean": float(np.mean(d / (nb + 0.01 * nb.mean()))),
            "velocity_rel_norm_same_forces": float(np.linalg.norm(V[: rows[1]] - V_ref) / np.linalg.norm(V_ref)),
        }
    return out


def report_tree(args, res):
    K = args.steps
    st = res["stats"]
    n = res["n"]
    step_ms = res["total_ms"] / K
    inter = (st["leaf_pairs"] + st["node_terms"])  # per walk
    clocks = res["clocks"] or {}
    max_mhz = clocks.get("sm_max_mhz") or 1965.0
    peak = SM_COUNT_B200 * FP32_LANES_PER_SM * 2 * max_mhz * 1e6 / 1e12
    fw = res["kern"].get("bh_force_walk")
    achieved = (st["leaf_pairs"] * FLOPS_LEAF_PAIR + st["node_terms"] * FLOPS_NODE_TERM) / (fw / 1000.0) / 1e12 \
        if fw else None
    line = {
        "metric": "DEM Barnes-Hut steps/s (N=1048576, theta=0.5, leaf 16)",
        "value": 1000.0 / step_ms,
        "unit": "steps/s",
        "n_gpus": 1,
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 terms, f64 positions and separations",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction)",
        "config": {
            "workload": "Barnes-Hut step: hash detection + merge + Morton octree build + force walk + Stokeslet "
                        "walk (total velocity) + Euler, N=2^20, periodic, dt=1e-4",
            "interactions_per_walk": inter,
            "leaf_pairs_per_droplet": st["leaf_pairs"] / n,
            "node_terms_per_droplet": st["node_terms"] / n,
            "tree_nodes": st["node_count"],
            "tree_levels": st["levels"],
            "kernel_ms_per_launch": res["kern"],
            "merges": res["merges"],
            "n_final": res["n_final"],
            "l2": "not flushed: the step's inputs (2^20 droplets) and tree exceed the 126 MB L2",
            **({"accuracy": res["accuracy"]} if "accuracy" in res else {}),
        },
        "roofline": {
            "kernel": "bh_force_walk",
            "bound": "fp32_pipe (latency-limited walk)",
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None,
            "traffic": ncu_traffic("bh_force_walk"),
            "units_per_launch": "leaf pair terms x 33 flops + node terms x 103 flops (monopole + quadrupole)",
        },
        "clocks": clocks,
        "gpu_launches": res["launches"],
    }
    peak_b, src_b = hbm_peak()
    mb = []
    if "hash_detect" in res["kern"]:
        table = 1 << max(int(2 * n - 1).bit_length(), 0)
        mb.append(hbm_entry("hash detection", res["kern"]["hash_detect"], hash_bytes(n, table, 0), peak_b, src_b,
                            "48 N + 8 table + 8 pairs"))
    if "bh_build" in res["kern"]:
        mb.append(hbm_entry("Morton octree build (keys, radix sort, gather, levels, node moments)",
                            res["kern"]["bh_build"], morton_build_bytes(n, st["node_count"]), peak_b, src_b,
                            "156 N + 140 nodes"))
    line["memory_bound"] = mb
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the main_tree.py drop-in: the reference-parity FP64 octree, timed as the
# reference's own benchmark times it (benchmarks/test.py)
# ---------------------------------------------------------------------------
PARITY_N = (100_000, 250_000, 500_000)
PARITY_MPL = (1, 2, 4, 8, 16)
PARITY_RADII = (2.5e-6, 7.5e-6)  # benchmarks/test.py:26
PARITY_PHYS = dict(eps_oil=2.85, eta_oil=0.065, eta_water=0.001, E=3e5)  # benchmarks/test.py:29


def parity_box_side(n, radii=PARITY_RADII, wvc=0.02):
    """box_size_from_volume, benchmarks/test.py:79-88."""
    return float(np.cbrt(np.pi * n * np.sum(radii) * np.sum(np.square(radii)) / (3 * wvc)))


def run_parity_tree(args, device):
    """TreeDropletForceCalculator (the reference-parity FP64 octree, the class
    main_tree.py builds) at N = 100k / 250k / 500k, theta = 0.5, mpl 1 / 2 / 4 /
    8 / 16.  One step = calculate(pos, r) + calculate_convection(pos, r, F)
    through the numpy API with host arrays, each call building the tree, as
    benchmarks/test.py:127-164 times it (mean of --steps calls after --warmup).
    The state: uniform radii in [2.5, 7.5] um, box side from the volume
    formula, open box, overlaps rejected with a 1 um gap (benchmarks/test.py:
    104-118), seeded.  Velocity error: the reference's metric (:63-77) of the
    total velocity F / (gamma r) + V against the FP64 direct sums."""
    import torch

    from dem.force_calculator import DirectDropletForceCalculator
    from dem.octree import TreeDropletForceCalculator
    from dem.particle_generator import UniformDropletGenerator

    torch.cuda.set_device(device)
    eta_o, eta_w = PARITY_PHYS["eta_oil"], PARITY_PHYS["eta_water"]
    sf = 2 * np.pi * eta_o * (2 * eta_o + 3 * eta_w) / (eta_o + eta_w)
    ns = [int(x) for x in args.parity_n.split(",")] if args.parity_n else list(PARITY_N)
    rows = []
    for n in ns:
        L = parity_box_side(n)
        st = UniformDropletGenerator(coord_range=(0, L), radii_range=PARITY_RADII, num_particles=n,
                                     minimum_distance=1e-6, seed=args.seed, device=device).generate()
        pos, rad = st.positions, st.radii
        fd = DirectDropletForceCalculator(num_particles=n, L=L, boundary_mode="open", device=device, **PARITY_PHYS)
        F_d, V_d = fd.calculate_forces_and_convection(pos, rad)
        vt_d = V_d + F_d / (sf * rad[:, None])
        tc = TreeDropletForceCalculator(num_particles=n, theta=0.5, mpl=1, periodic=False, **PARITY_PHYS)
        mpls = [int(x) for x in args.parity_mpl.split(",")] if args.parity_mpl else list(PARITY_MPL)
        for mpl in mpls:
            tc.update_params(0.5, mpl)

            def step():
                f = tc.calculate(pos, rad)
                return f, tc.calculate_convection(pos, rad, f)

            for _ in range(max(args.warmup, 1)):
                step()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                f, v = step()
            torch.cuda.synchronize()
            ms = 1000.0 * (time.perf_counter() - t0) / args.steps
            vt = v + f / (sf * rad[:, None])
            dn = np.linalg.norm(vt - vt_d, axis=1)
            nr = np.linalg.norm(vt_d, axis=1)
            rel = dn / (nr + 0.01 * nr.mean())
            stats = tc.octree.get_tree_stats() if hasattr(tc.octree, "get_tree_stats") else {}
            rows.append(dict(n=n, theta=0.5, mpl=mpl, tree_ms=ms, mean_err_pct=100 * float(rel.mean()),
                             max_err_pct=100 * float(rel.max()), nodes=stats.get("node_count")))
    return rows


# benchmarks/data.txt:116-119, 344-347, 572-575: the reference's Taichi CPU tree step (ms), i7-11800H, 16 threads
PARITY_PUBLISHED_MS = {
    (100_000, 1): 570.3, (100_000, 2): 460.8, (100_000, 4): 444.0, (100_000, 8): 566.6, (100_000, 16): 662.4,
    (250_000, 1): 1702.7, (250_000, 2): 1597.4, (250_000, 4): 1571.4, (250_000, 8): 1984.0, (250_000, 16): 1944.8,
    (500_000, 1): 5055.6, (500_000, 2): 4625.8, (500_000, 4): 4839.6, (500_000, 8): 7610.1, (500_000, 16): 8316.9,
}


def report_parity_tree(args, rows):
    for row in rows:
        pub = PARITY_PUBLISHED_MS.get((row["n"], row["mpl"]))
        row["reference_published_ms"] = pub
        row["vs_published"] = pub / row["tree_ms"] if pub else None
    head = rows[0]
    line = {
        "metric": "DEM tree step ms (TreeDropletForceCalculator, theta=0.5)",
        "value": head["tree_ms"],
        "unit": "ms/step",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["tree_ms"],
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": head["vs_published"],
        "dtype": "f64",
        "data": "synthetic (seeded uniform radii 2.5-7.5 um, 2% water volume fraction, open box)",
        "config": {"workload": "main_tree.py drop-in: calculate + calculate_convection of the reference-parity FP64 "
                               "octree through the numpy API (host arrays, tree built per call), as "
                               "benchmarks/test.py times it",
                   "rows": rows},
    }
    print(json.dumps(line), flush=True)


CORR_GRID = 48  # points per axis of the periodic-image correction grid (the shipped COMSOL grid's size)


def synthetic_correction(n=CORR_GRID, L_comsol=1e-3, Fz_comsol=1.1126e-11, eta_comsol=0.065, seed=7):
    """A smooth seeded correction field on the regular grid (the COMSOL data are
    not shipped; the passes' cost does not depend on the values)."""
    from dem.periodic_correction import COMSOLLatticeCorrection

    rng = np.random.default_rng(seed)
    ax = np.linspace(-L_comsol / 2, L_comsol / 2, n) / L_comsol
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    grids = []
    for _ in range(3):
        a = rng.normal(size=(3, 4))
        grids.append(1e-9 * sum(a[m, 0] * np.sin((m + 1) * 5.3 * X + a[m, 1]) * np.cos((m + 2) * 3.1 * Y + a[m, 2])
                                * np.cos(m * 4.7 * Z + a[m, 3]) for m in range(3)))
    return COMSOLLatticeCorrection.from_grid(*grids, L_comsol=L_comsol, Fz_comsol=Fz_comsol, eta_comsol=eta_comsol)


def run_correction(args, device):
    import torch

    from dem._native import launch_count
    from dem.force_calculator import DirectDropletForceCalculator

    torch.cuda.set_device(device)
    n = args.n
    pos, r, L = make_state(n, args.seed)
    corr = synthetic_correction()
    calc = {}
    for prec in ("mixed", "fp64"):
        fc = DirectDropletForceCalculator(num_particles=n, L=L, boundary_mode="periodic",
                                          correction_grid_resolution=CORR_GRID, precision=prec, device=device, **PHYS)
        fc.load_periodic_correction(corr, L_sim=L)
        calc[prec] = fc
    fc = calc["mixed"]
    ctx = fc._ctx
    P = torch.as_tensor(pos, device=device)
    R = torch.as_tensor(r, device=device)
    F = fc.calculate(P, R)
    for _ in range(args.warmup):
        fc.calculate_convection(P, R, F)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    time.sleep(0.4)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    c0 = launch_count()
    ctx.profile(True)
    for k in range(args.steps):
        ev[k][0].record()
        fc.calculate_convection(P, R, F)
        ev[k][1].record()
    torch.cuda.synchronize()
    launches = launch_count() - c0
    kern = {}
    for name in ("corr_direct_pass", "mixed_convection_pass"):
        ms, cnt = ctx.profile_read(name)
        if cnt:
            kern[name] = ms / cnt
    ctx.profile(False)
    clocks = sampler.stop()
    total_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    # the table's random-gather bandwidth, on the same stream (the roofline of the FP32 pass)
    ctas, per_thread = 8 * SM_COUNT_B200, 4096
    out = torch.empty(ctas * 256, dtype=torch.float32, device=device)
    fc._corr.gather_probe(ctas, per_thread, out)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fc._corr.gather_probe(ctas, per_thread, out)
    e1.record()
    torch.cuda.synchronize()
    probe_gbs = ctas * 256 * per_thread * 96 / (e0.elapsed_time(e1) / 1000.0) / 1e9
    # the FP64 pass (bit-identical to the reference's order), timed once after a warm-up
    f64 = calc["fp64"]
    F64 = f64.calculate(P, R)
    f64.calculate_convection(P, R, F64)
    f64._ctx.profile(True)
    f64.calculate_convection(P, R, F64)
    torch.cuda.synchronize()
    fp64_ms, _ = f64._ctx.profile_read("fp64_convection_corr_pass")
    f64._ctx.profile(False)
    # end to end through the numpy API: host arrays in, velocities back
    Fh = F.cpu().numpy()
    fc.calculate_convection(pos, r, Fh)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(e2e_steps):
        fc.calculate_convection(pos, r, Fh)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    out = dict(n=n, L=L, total_ms=total_ms, kern=kern, clocks=clocks, launches=launches, probe_gbs=probe_gbs,
               fp64_ms=fp64_ms, e2e_s=e2e_s)
    if args.accuracy:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        _, eta, _ = O.physics_constants(**PHYS)
        d = corr.get_grid_data()
        w0 = float(corr.evaluate(np.zeros((1, 3)))[0, 2])
        eta_r = d["eta_comsol"] / PHYS["eta_oil"]
        oc = O.Correction(d["grid_u"], d["grid_v"], d["grid_w"], d["grid_min"], d["grid_dx"], d["Fz_comsol"],
                          d["L_comsol"], d["eta_comsol"], L, PHYS["eta_oil"],
                          w0 / d["Fz_comsol"] * eta_r * (d["L_comsol"] / L))
        Fh = F.cpu().numpy()
        V = fc.calculate_convection(pos, r, Fh)
        rows = (0, 1024)
        V_ref = O.direct_convection_corr(pos, Fh, eta, L, True, oc, rows=rows)[: rows[1]]
        err = np.linalg.norm(V[: rows[1]] - V_ref, axis=1)
        out["accuracy"] = {
            "sample": "droplets 0..1023 against the oracle's FP64 sums over all N (same forces)",
            "velocity_rel_norm": float(np.linalg.norm(V[: rows[1]] - V_ref) / np.linalg.norm(V_ref)),
            "velocity_max_err_over_mean": float(err.max() / np.linalg.norm(V_ref, axis=1).mean()),
        }
    return out


def run_trajectory(args, device):
    """Config 1's long run: --traj-steps direct steps (detection, coalescence,
    forces, convection, Euler) from one seeded state, FP64 and mixed, with the
    validated FP64 GPU path as the reference (bit-identical to the oracle per
    step).  Compares the colliding-pair sets of every detection, the merge
    counts, and the positions of the droplets that never merged."""
    import torch

    torch.cuda.set_device(device)
    pos0, r0, L = make_state(args.n, args.seed)
    K = args.traj_steps
    runs = {}
    for prec in ("fp64", "mixed"):
        st = DeviceStepper(pos0, r0, L, prec, device, track=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            st.step()
        torch.cuda.synchronize()
        runs[prec] = dict(seconds=time.perf_counter() - t0, pos=st.positions(), ids=st.ids.copy(), n=st.n,
                          merges=st.merges, pair_log=st.pair_log)
    a, b = runs["fp64"], runs["mixed"]
    same_pairs = len(a["pair_log"]) == len(b["pair_log"]) and all(
        sa == sb and np.array_equal(pa, pb) for (sa, pa), (sb, pb) in zip(a["pair_log"], b["pair_log"]))
    first_diff = None
    for k, ((sa, pa), (sb, pb)) in enumerate(zip(a["pair_log"], b["pair_log"])):
        if sa != sb or not np.array_equal(pa, pb):
            first_diff = int(min(sa, sb))
            break
    # droplets present from the start in both runs
    orig = np.intersect1d(a["ids"][a["ids"] < len(r0)], b["ids"][b["ids"] < len(r0)])
    ia = {v: k for k, v in enumerate(a["ids"])}
    ib = {v: k for k, v in enumerate(b["ids"])}
    xa = a["pos"][[ia[v] for v in orig]]
    xb = b["pos"][[ib[v] for v in orig]]
    mic = lambda d: d - L * np.rint(d / L)  # noqa: E731
    disp = mic(xa - pos0[orig])
    err = mic(xb - xa)
    return dict(n=len(r0), K=K, L=L, seconds={p: runs[p]["seconds"] for p in runs},
                merges={p: runs[p]["merges"] for p in runs}, n_final={p: runs[p]["n"] for p in runs},
                detections_with_pairs={p: len(runs[p]["pair_log"]) for p in runs},
                pair_sets_identical=bool(same_pairs), first_differing_step=first_diff, compared=int(len(orig)),
                disp_rms=float(np.sqrt((disp**2).sum(1).mean())),
                rel_err_norm=float(np.linalg.norm(err) / np.linalg.norm(disp)),
                max_err_over_rms_disp=float(np.sqrt((err**2).sum(1)).max() / np.sqrt((disp**2).sum(1).mean())))


def report_trajectory(args, res):
    K = res["K"]
    sec = res["seconds"]
    line = {
        "metric": f"DEM direct steps/s over a {K}-step trajectory (N={res['n']}), mixed vs FP64 GPU",
        "value": K / sec["mixed"],
        "unit": "steps/s",
        "n_gpus": 1,
        "steps": K,
        "warmup": 0,
        "ms_per_step": 1000.0 * sec["mixed"] / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 pair terms (mixed) against f64",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction)",
        "config": {
            "workload": "direct step with detection, coalescence and Euler update, wall clock over the whole run "
                        "(host syncs for the pair count included); FP64 GPU as the reference trajectory",
            "fp64_steps_per_s": K / sec["fp64"],
            "speedup_mixed_over_fp64": sec["fp64"] / sec["mixed"],
            "merges": res["merges"],
            "detections_with_pairs": res["detections_with_pairs"],
            "n_final": res["n_final"],
            "pair_sets_identical_every_detection": res["pair_sets_identical"],
            "first_differing_step": res["first_differing_step"],
            "droplets_compared": res["compared"],
            "rms_displacement_m": res["disp_rms"],
            "position_error_rel_to_displacement_norm": res["rel_err_norm"],
            "position_error_max_over_rms_displacement": res["max_err_over_rms_disp"],
        },
    }
    print(json.dumps(line), flush=True)


def report_correction(args, res):
    K = args.steps
    n = res["n"]
    pass_ms = res["total_ms"] / K
    pairs = n * (n - 1)
    corr_ms = res["kern"].get("corr_direct_pass")
    gbs = pairs * 288 / (corr_ms / 1000.0) / 1e9 if corr_ms else None  # 3 lookups x 96 bytes per pair
    line = {
        "metric": f"DEM corrected Oseen convection passes/s (N={n}, periodic-image correction, 48^3 grid)",
        "value": 1000.0 / pass_ms,
        "unit": "passes/s",
        "n_gpus": 1,
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": pass_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 correction terms and mixed Oseen pass, f64 sums",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction; seeded smooth 48^3 correction grid)",
        "config": {
            "workload": "one Oseen convection pass with the periodic-image correction of every pair and the self "
                        "term (direct_droplet_force_calculator.py:354-464), forces given, mixed precision",
            "pair_corrections_per_s": pairs / (corr_ms / 1000.0) if corr_ms else None,
            "kernel_ms_per_launch": res["kern"],
            "fp64_pass_ms": res["fp64_ms"],
            "l2": "not flushed: the 13 MB table is meant to stay in L2; positions and forces (3 MB) too",
            **({"accuracy": res["accuracy"]} if "accuracy" in res else {}),
        },
        "roofline": {
            "kernel": "corr_direct_pass",
            "bound": "l2 (random 96-byte cell gathers from the L2-resident table)",
            "achieved": gbs,
            "peak": res["probe_gbs"],
            "unit": "GB/s",
            "frac": gbs / res["probe_gbs"] if gbs else None,
            "traffic": None,
            "units_per_launch": "N (N - 1) pairs x 3 lookups x 96 bytes; peak = dem_corr_gather_probe on the same "
                                "table and stream (measured in this run)",
        },
        "e2e": {"value": 1.0 / res["e2e_s"], "unit": "passes/s", "h2d_bytes_per_step": n * 56,
                "d2h_bytes_per_step": n * 24},
        "clocks": res["clocks"],
        "gpu_launches": res["launches"],
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch

        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            torch.cuda.set_device(local)
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()
        return

    import torch

    device = torch.device("cuda", local)
    if args.workload == "tree":
        if rank == 0:
            report_tree(args, run_tree(args, device))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "parity_tree":
        if rank == 0:
            report_parity_tree(args, run_parity_tree(args, device))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "trajectory":
        if rank == 0:
            report_trajectory(args, run_trajectory(args, device))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "correction":
        if rank == 0:
            report_correction(args, run_correction(args, device))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "adjoint":
        if rank == 0:
            report_adjoint(args, run_adjoint(args, device))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload == "batched":
        res = run_batched(args, rank, world, device)
        if world > 1:
            torch.distributed.destroy_process_group()
        if rank == 0:
            report_batched(args, res, world)
        return
    res = run_ours(args, rank, world, device)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    n = res["n"]
    K = args.steps
    from dem.replicas import whole_job_rate

    steps_per_s = whole_job_rate(K, world, res["total_ms"])
    # ordered pairs per step: the timed steps' own droplet counts (merges during the untimed advance and the
    # window itself leave fewer than the seeded n)
    nt = res["n_timed"] or [n]
    pairs = sum(m * (m - 1) for m in nt) / len(nt)
    clocks = res["clocks"] or {}
    # roofline of the dominant kernel
    prec = args.precision
    fname = "mixed_force_pass" if prec == "mixed" else "fp64_force_pass"
    cname = "mixed_convection_pass" if prec == "mixed" else "fp64_convection_pass"
    kern = res["kern"]
    dom = max((fname, cname), key=lambda k: kern.get(k, (0, 1))[0])
    ms, cnt = kern.get(dom, (float("nan"), 1))
    # algorithmic work: every ordered pair of the reference's double loop; the symmetric schedule evaluates each
    # unordered pair once and adds its terms to both droplets, so it executes fewer pair evaluations than this
    flops = (FLOPS_FORCE_PAIR if dom == fname else FLOPS_OSEEN_PAIR) * pairs
    schedule = res["schedule"]
    achieved = flops / (ms / cnt / 1000.0) / 1e12
    max_mhz = clocks.get("sm_max_mhz") or 1965.0
    lanes = FP32_LANES_PER_SM if prec == "mixed" else FP32_LANES_PER_SM // 2
    peak = SM_COUNT_B200 * lanes * 2 * max_mhz * 1e6 / 1e12
    peak_at_clock = SM_COUNT_B200 * lanes * 2 * (clocks.get("sm_mhz") or max_mhz) * 1e6 / 1e12
    traffic = ncu_traffic(dom)
    line = {
        "metric": f"DEM steps/s (direct, N={n})",
        "value": steps_per_s,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": K,
        "warmup": args.warmup,
        "ms_per_step": res["total_ms"] / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 pair terms + f64 near pairs/sums" if prec == "mixed" else "f64",
        "data": "synthetic (seeded lognormal droplets, 2% volume fraction)",
        "config": {
            "workload": direct_workload(n),
            "precision": prec,
            "pairs_per_s": steps_per_s * pairs,
            "l2": "flushed between steps (256 MiB write outside the timed events)",
            "timed_window": f"steps {args.advance + args.warmup}..{args.advance + args.warmup + K - 1} of the "
                            f"trajectory from the seeded state ({args.advance} untimed steps, then the warm-up)",
            "merges_before_timed": res["merges_advance"],
            "merges_in_timed": res["merges_timed"],
            "n_final": res["n_final"],
            "kernel_ms_per_launch": {k: v[0] / v[1] for k, v in kern.items()},
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "roofline": {
            "kernel": dom,
            "bound": "fp32_pipe" if prec == "mixed" else "fp64_pipe",
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved / peak,
            "frac_at_sampled_clock": achieved / peak_at_clock,
            "traffic": traffic,
            "peak_source": f"{SM_COUNT_B200} SMs x {lanes} lanes x 2 flop x {max_mhz:.0f} MHz (max SM clock); "
                           "MEASURED_PEAKS.json holds no CUDA-core figure",
            "flops_per_pair": FLOPS_FORCE_PAIR if dom == fname else FLOPS_OSEEN_PAIR,
            "units_per_launch": f"N(N-1) averaged over the timed steps = {pairs:.0f} ordered pairs (the reference's "
                                f"pair evaluations; N = {min(nt)}..{max(nt)} after merges)",
            "schedule": schedule,
        },
        "clocks": clocks,
        "gpu_launches": None,
    }
    if not args.no_e2e:
        e = run_e2e(args, device, steps=max(3, min(K, 10)), warmup=1)
        line["e2e"] = {"value": e["steps_per_s"], "unit": "steps/s", "h2d_bytes_per_step": e["h2d"],
                       "d2h_bytes_per_step": e["d2h"]}
    if not args.no_cpu:
        c = cpu_step_rate(res["pos"], res["r"], res["L"], args.cpu_sample_seconds)
        line["cpu_baseline"] = {"value": c["steps_per_s"], "unit": "steps/s", "cores": c["cores"], "kind": "port",
                                "sample": f"hash + Euler on all {n} droplets; both O(N^2) passes on {c['rows']} rows "
                                          f"x {n} columns, extrapolated ({c['sample_s']:.1f} s of CPU work)"}
    if "hash_detect" in kern:
        peak_b, src_b = hbm_peak()
        table = 1 << max(int(2 * n - 1).bit_length(), 0)
        n_det = int(round(sum(nt) / len(nt)))  # droplets per detection in the timed window
        line["memory_bound"] = [hbm_entry("hash detection (assign, scans, scatter, bucket records, count, write)",
                                          kern["hash_detect"][0] / kern["hash_detect"][1], hash_bytes(n_det, table, 0),
                                          peak_b, src_b, "48 N + 8 table + 8 pairs")]
    if "fp64" in res:
        f64 = res["fp64"]
        fp64_sps = 1000.0 / f64["ms_per_step"]
        line["fp64_gpu"] = {
            "steps_per_s": fp64_sps,
            "ms_per_step": f64["ms_per_step"],
            "steps_timed": f64["steps"],
            "merges_in_timed": f64["merges"],
            "speedup_mixed_vs_fp64": steps_per_s / fp64_sps,
            "how": "the FP64 drop-in step (bit-exact with the oracle) on the state after the mixed timed steps, "
                   "same CUDA events and L2 flush",
        }
        line["accuracy_mixed_vs_fp64"] = res["accuracy"]
    # kernels of the library launched inside the timed region (its own launch counter); a step without a merge
    # is hash detection (12) + forces (4) + convection (6) + Euler (1)
    line["gpu_launches"] = res["launches"]
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
