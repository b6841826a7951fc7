#!/usr/bin/env python
"""Throughput benchmark: molecule-steps/s of the particle engine on B200.

Workload (one GPU): the scale-up configuration - periodic cube of side 1000,
10^7 molecules uniform at random (45% A, 45% B, 10% C), A+B->C kf=0.05,
C->A+B kr=0.1, 0->A at 1e-4 per unit volume per unit time, D = 1, 1, 0.5,
dt = 0.01.  A step is one simulated time step over all molecules.

  value     device time of K steps (graph replays), inputs resident in HBM
  e2e       the same work through the libsmoldyn C API with host buffers:
            upload of the molecules from host memory, K smolRunTimeStep calls
            each followed by a per-species smolGetMoleculeCount read-back
  roofline  the dominant kernel's algorithmic bytes per launch / its average
            CUDA-event duration, against the measured HBM copy bandwidth
  cpu_baseline  the reference Smoldyn binary (compiled from the reference's
            sources by oracle/Makefile) on a bounded sample of the same
            workload on this host's cores

With --impl reference the reference CPU engine itself is timed (all host
cores, one independent process per core).  Under torchrun each rank runs an
independent replica (the workload shards as independent replicas; no data
collective) and rank 0 prints the job total over the slowest rank's time.
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "molecule-steps/s"
L_SIDE = 1000.0
N_MOL = 10_000_000
FRAC = (0.45, 0.45, 0.10)
DIFC = (1.0, 1.0, 0.5)
KF, KR, K0 = 0.05, 0.1, 1e-4
DT = 0.01
# algorithmic bytes per molecule-step: read 16 B (position + packed species/state)
# and write 16 B in box order in the fused move/rebin pass, read 16 B again in
# the pair search
ALG_BYTES_PER_MOLSTEP = 48
# per-kernel share of those algorithmic bytes per molecule: the move pass
# reads each molecule, the scatter writes it in box order, the pair search
# reads it again
KERNEL_BYTES = {"k_move": 16, "k_scatter": 16, "k_pairs": 16}


def measured_traffic():
    """DRAM bytes per molecule per launch from the committed ncu capture
    (profiles/traffic_per_molecule.txt), or {} if absent."""
    out = {}
    path = os.path.join(ROOT, "profiles", "traffic_per_molecule.txt")
    if os.path.exists(path):
        for line in open(path):
            t = line.split()
            if len(t) == 2 and not t[0].startswith("#"):
                out[t[0]] = float(t[1])
    return out


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits", "-lms", "20"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi needs a moment before its first sample; wait for it so the
        # samples cover the timed region that follows
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0:
            time.sleep(0.01)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
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
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_sim(sb, n_mol, side, seed):
    s = sb.Sim(3, (0, 0, 0), (side, side, side))
    for nm, d in zip(("A", "B", "C"), DIFC):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, "p")
    s.set_times(0, 1e9, DT)
    s.seed(seed)
    s.add_reaction("fwd", "A", "B", ["C"], KF)
    s.add_reaction("rev", "C", None, ["A", "B"], KR)
    s.add_reaction("birth", None, None, ["A"], K0)
    counts = [int(round(n_mol * f)) for f in FRAC]
    counts[0] += n_mol - sum(counts)
    for nm, c in zip(("A", "B", "C"), counts):
        s.add_molecules(nm, c)
    return s


def reference_config(path, n_mol, side, steps, seed):
    counts = [int(round(n_mol * f)) for f in FRAC]
    with open(path, "w") as f:
        f.write("dim 3\nspecies A B C\n")
        for nm, d in zip(("A", "B", "C"), DIFC):
            f.write("difc %s %g\n" % (nm, d))
        for d in range(3):
            f.write("boundaries %d 0 %.10g p\n" % (d, side))
        f.write("time_start 0\ntime_stop %.10g\ntime_step %g\nrandom_seed %d\n" % (steps * DT, DT, seed))
        f.write("reaction fwd A + B -> C %g\nreaction rev C -> A + B %g\nreaction birth 0 -> A %g\n" % (KF, KR, K0))
        for nm, c in zip(("A", "B", "C"), counts):
            f.write("mol %d %s u u u\n" % (c, nm))
        f.write("end_file\n")


def time_reference_sample(n_mol, steps_lo, steps_hi, procs, seed0=1):
    """Per-step wall time of the reference binary on a same-density sample,
    from the difference of two runs (so setup is excluded)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "smoldyn")
    if not os.path.exists(exe):
        return None, "reference binary not built (make -C oracle ref)"
    side = L_SIDE * (n_mol / N_MOL) ** (1.0 / 3.0)
    tmp = tempfile.mkdtemp(prefix="smolref_")
    try:
        walls = {}
        for steps in (steps_lo, steps_hi):
            cfgs = []
            for p in range(procs):
                c = os.path.join(tmp, "s%d_%d.txt" % (steps, p))
                reference_config(c, n_mol, side, steps, seed0 + p)
                cfgs.append(c)
            t0 = time.perf_counter()
            ps = [subprocess.Popen([exe, c, "-qt"], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, cwd=tmp)
                  for c in cfgs]
            rcs = [p.wait() for p in ps]
            walls[steps] = time.perf_counter() - t0
            if any(rcs):
                return None, "reference exited with %s" % rcs
        per_step = (walls[steps_hi] - walls[steps_lo]) / (steps_hi - steps_lo)
        return dict(per_step_s=per_step, side=side, n_mol=n_mol, procs=procs, walls=walls), None
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    procs = os.cpu_count() or 1
    n_s = args.ref_sample
    res, why = time_reference_sample(n_s, 2, 2 + max(1, args.steps), procs)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    value = procs * n_s / res["per_step_s"]
    sample = ("%d independent reference processes, each %d molecules in a periodic cube of side %.1f (the "
              "workload's density and rates), per-step time from runs of 2 and %d steps" %
              (procs, n_s, res["side"], 2 + max(1, args.steps)))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["per_step_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": procs, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def combine_ranks(dist, torch, t_s, work, device):
    """Whole-job numbers over the ranks of a replicas run: the slowest rank's
    time (max) and the work of all ranks (sum)."""
    tmax = torch.tensor([t_s], device=device, dtype=torch.float64)
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = torch.tensor([work], device=device, dtype=torch.float64)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax.item()), float(tsum.item())


def workload_config(args):
    n = getattr(args, "molecules", N_MOL)
    side = L_SIDE * (n / N_MOL) ** (1.0 / 3.0)
    return {"workload": "scale-up: periodic cube %g, %g molecules (45%% A, 45%% B, 10%% C), A+B->C 0.05, "
                        "C->A+B 0.1, 0->A 1e-4, D=1,1,0.5, dt=0.01" % (side, n),
            "molecules": n, "box": side, "dt": DT, "l2": "inputs larger than L2 (>=240 MB per buffer)",
            "parallelism": "replicas" if args.gpus > 1 else "single"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-sample", type=int, default=100000)
    ap.add_argument("--molecules", type=int, default=N_MOL,
                    help="molecules of the plain workload at its density (smaller only for profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-batched", action="store_true", help="skip the ensemble and surrogate workloads")
    ap.add_argument("--no-tune", action="store_true", help="default launch shape and box width (no autotuner)")
    ap.add_argument("--kernel-tour", action="store_true",
                    help="run one small case of every kernel of the library (profiler captures) and exit")
    ap.add_argument("--batched-steps", type=int, default=2000, help="steps of the 4096-replicate ensemble leg")
    ap.add_argument("--surrogate-steps", type=int, default=5000,
                    help="steps of the 65,536-replicate surrogate sweep (rates redrawn every 100)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.kernel_tour:
        return kernel_tour(args)

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    import smoldyn_b200 as sb

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident throughput
    n_mol = args.molecules
    s = build_sim(sb, n_mol, L_SIDE * (n_mol / N_MOL) ** (1.0 / 3.0), 1 + rank)
    s.update()
    t_tune = time.perf_counter()
    tune_ms = s.autotune(20) if not args.no_tune else None
    t_tune = time.perf_counter() - t_tune
    tuning = s.tuning()
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    clocks = ClockSampler(local)
    clocks.start()
    s.run_steps(args.warmup)
    s.synchronize()
    n0 = s.total()
    barrier()
    torch.cuda.synchronize()
    l0 = s.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.run_steps(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = s.launches() - l0
    barrier()
    ck = clocks.stop()
    n1 = s.total()
    mol_steps = 0.5 * (n0 + n1) * args.steps
    t_s = ms / 1e3
    if dist is not None:
        t_s, mol_steps = combine_ranks(dist, torch, t_s, mol_steps, "cuda")
    value = mol_steps / t_s

    # ---- per-kernel breakdown (events between launches) for the roofline
    prof = s.profile_steps(max(4, min(20, args.steps)))
    s.synchronize()
    nprof = max(4, min(20, args.steps))
    tot_ms = sum(v[0] for v in prof.values())
    top = max(prof.items(), key=lambda kv: kv[1][0])
    hbm, peak_kind = peaks()
    nmol_avg = 0.5 * (n0 + n1)
    roof = None
    if top[0] in KERNEL_BYTES:
        per_launch_ms = top[1][0] / top[1][1]
        bytes_launch = KERNEL_BYTES[top[0]] * nmol_avg
        achieved = bytes_launch / (per_launch_ms / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_kind": peak_kind,
                "traffic": (measured_traffic()[top[0]] * nmol_avg if top[0] in measured_traffic() else None),
                "traffic_note": "bytes per launch: ncu DRAM read+write per molecule (4e6-molecule capture, "
                                "profiles/traffic_per_molecule.txt) x molecules of this run",
                "alg_bytes_per_molecule": KERNEL_BYTES[top[0]]}
    step_frac = (ALG_BYTES_PER_MOLSTEP * value / (world if world > 1 else 1)) / (hbm * 1e9)
    kernels = {k: {"ms_per_step": v[0] / nprof, "share": v[0] / tot_ms} for k, v in prof.items()}
    s.close()
    torch.cuda.synchronize()

    # ---- end to end through the C API with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(sb, args, rank, world, dist, barrier)

    # ---- batched ensemble and surrogate sweep (extra workloads, same GPU)
    batched = surrogate = surfaces = bound = rdf = None
    if not args.no_batched:
        batched = run_batched(sb, torch, args, rank)
        surrogate = run_surrogate(sb, torch, args, rank)
        surfaces = run_surfaces(sb, torch, args, rank)
        bound = run_surface_bound(sb, torch, args, rank)
        rdf = run_rdf_tables(sb, args, rank, world)

    # ---- CPU baseline (rank 0, single GPU run only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_s = args.ref_sample
        res, why = time_reference_sample(n_s, 2, 12, 1)
        if res is not None:
            cpu = {"value": n_s / res["per_step_s"], "unit": METRIC, "cores": 1, "kind": "reference",
                   "sample": "reference smoldyn binary, %d molecules in a periodic cube of side %.1f (same density "
                             "and rates), per-step time from runs of 2 and 12 steps" % (n_s, res["side"])}
        else:
            cpu = {"value": None, "unit": METRIC, "cores": 1, "kind": "reference", "sample": why}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(args), tuning=tuning, autotune_s=t_tune, autotune_best_trial_ms=tune_ms),
            "e2e": e2e, "gpu_launches": int(launches),
            "roofline": roof, "step_roofline_frac": step_frac, "kernels": kernels, "cpu_baseline": cpu,
            "clocks": ck, "batched": batched, "batched_surrogate": surrogate, "surfaces": surfaces,
            "surface_bound": bound,
            "rdf_tables": rdf,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


TOUR_CONFIG = """dim 3
species A B C
difc A 1
difc B 1
difc C 0.5
boundaries 0 0 60 p
boundaries 1 0 60 p
boundaries 2 0 60 p
time_start 0
time_stop 100
time_step 0.01
random_seed 3
start_surface ball
action both all transmit
panel sphere 30 30 30 12 20 20
end_surface
start_compartment core
surface ball
point 30 30 30
end_compartment
reaction fwd A + B -> C 0.5
reaction rev C -> A + B 0.1
mol 20000 A u u u
mol 20000 B u u u
output_files msd.txt cnt.txt
cmd N 5 meansqrdisp A all msd.txt
cmd N 5 molcountincmpt core cnt.txt
end_file
"""


# surface-bound states: adsorption onto / desorption from a sphere with bound
# diffusion, plus a bimolecular reaction (the bound-state form of the step
# kernels and k_bound)
TOUR_BOUND_CONFIG = """dim 3
species A B C
difc A 1
difc B 1
difc C 0.5
difc A(front) 0.5
boundaries 0 0 60
boundaries 1 0 60
boundaries 2 0 60
time_start 0
time_stop 100
time_step 0.01
random_seed 4
start_surface walls
action both all reflect
panel rect +0 0 0 0 60 60
panel rect -0 60 0 0 60 60
panel rect +1 0 0 0 60 60
panel rect -1 0 60 0 60 60
panel rect +2 0 0 0 60 60
panel rect -2 0 0 60 60 60
end_surface
start_surface cell
action both all reflect
rate A fsoln front 2
rate A front fsoln 1
panel sphere 30 30 30 12 20 20 s1
end_surface
reaction fwd A + B -> C 0.5
reaction rev C -> A + B 0.1
reaction bnd A(front) + B -> A(front) 0.2
reaction dim A(front) + A(front) -> A(front) 0.05
mol 20000 A u u u
mol 20000 B u u u
surface_mol 20000 A(front) cell sph all
end_file
"""


def kernel_tour(args):
    """One small case of every kernel of the library, for profiler captures
    (ncu -k selects the kernel): the step pipeline on the scale-up workload
    at 4e6 molecules (its density), the device upload path, meansqrdisp and
    molcountincmpt with a transmitting sphere compartment (surface form of the
    step kernels), adsorption, desorption and bound diffusion on a sphere
    with a bound-solution and a bound-bound reaction (k_bound, the bound-state
    form and the bound-pair kernels), the FP64 radius solvers, the surrogate's sampling,
    training, inference and radius kernels, the persistent ensemble kernel
    and its layout changes, and the radial-distribution solver."""
    import ctypes as C
    import torch
    torch.cuda.set_device(0)
    import smoldyn_b200 as sb
    lib = sb.load()
    n = 4_000_000
    s = build_sim(sb, n, L_SIDE * (n / N_MOL) ** (1.0 / 3.0), 1)
    s.update()
    s.run_steps(3)
    pos, sp, sn = s.molecules()
    s.set_molecules(pos, sp, sn)     # device upload path
    s.run_steps(2)
    s.synchronize()
    s.close()
    d = tempfile.mkdtemp(prefix="smoltour_")
    try:
        with open(os.path.join(d, "t.txt"), "w") as f:
            f.write(TOUR_CONFIG)
        simp = C.c_void_p()
        assert lib.smolLoadSimFromFile((d + "/").encode(), b"t.txt", C.byref(simp), b"") == 0, sb.last_error()
        t = sb.Sim(ptr=simp.value)
        t.run_until(0.1)
        t.close()
        with open(os.path.join(d, "b.txt"), "w") as f:
            f.write(TOUR_BOUND_CONFIG)
        b = sb.Sim.load_file(os.path.join(d, "b.txt"))
        b.update()
        b.run_steps(10)
        b.synchronize()
        b.close()
    finally:
        shutil.rmtree(d, ignore_errors=True)
    rng = np.random.default_rng(1)
    m = 65536
    rate, difc = 10 ** rng.uniform(-3, 0, m), np.full(m, 2.0)
    sb.solve_radii_device(0, rate, DT, difc, np.full(m, 1.5), rel=1)
    sb.solve_radii_prob_device(rate, DT, difc, np.full(m, -1.0), 0, np.full(m, -1.0), np.full(m, 0.5))
    sur = sb.Surrogate()
    sur.train(nsamples=16384, epochs=1, batch=512, lr=3e-3, seed=5)
    sur.pair_radii(rate, difc, DT, same=0, rev=1, rparamt=sb.RPratio, rparam=1.5)
    R = 1024
    nr, side = draw_replicates(rng, R, 1e2, 1e4)
    e = sb.Ensemble(ensemble_template(sb, placement=(sb.RPratio, 1.5)), R)
    e.set_boxes(np.zeros((R, 3)), np.repeat(side[:, None], 3, 1))
    e.set_rates("fwd", 10 ** rng.uniform(-3, 0, R))
    e.set_rates("rev", 10 ** rng.uniform(-3, 0, R))
    e.add_molecules("A", nr // 2 + nr % 2)
    e.add_molecules("B", nr // 2)
    e.radius_mode(1)
    e.engine(2)
    e.update()
    e.run_steps(10)
    e.counts(4)
    e.molecules()
    e.close()
    sb.rdf_table("i", 100, 1e-5, "d")
    torch.cuda.synchronize()
    print("kernel tour done")
    return 0


def ensemble_template(sb, placement=None):
    s = sb.Sim(3, (0, 0, 0), (1, 1, 1))
    for nm, d in zip(("A", "B", "C"), DIFC):
        s.add_species(nm, d)
    for d in range(3):
        s.boundary(d, -1, "r")
    s.set_times(0, 1e9, DT)
    s.seed(4242)
    s.add_reaction("fwd", "A", "B", ["C"], 0.05)
    s.add_reaction("rev", "C", None, ["A", "B"], 0.1)
    if placement is not None:
        s.set_products("rev", *placement)
    return s


def draw_replicates(rng, nrep, lo, hi):
    n = np.rint(10 ** rng.uniform(np.log10(lo), np.log10(hi), nrep)).astype(np.int64)
    side = (n / 0.01) ** (1.0 / 3.0)
    return n, side


def time_on_stream(torch, stream, fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def run_batched(sb, torch, args, rank):
    """Ensemble workload: 4096 replicates, N log-uniform in [1e2, 1e5] at
    density 0.01, kf and kr log-uniform in [1e-3, 1] per replicate, radii from
    the exact FP64 solver on the device, dt = 0.01, 2000 steps (the
    configuration's count; fewer with --batched-steps).  Stepped by the step
    pipeline (the ensemble default), with the persistent kernel timed beside
    it."""
    rng = np.random.default_rng(12345 + rank)
    R = 4096
    n, side = draw_replicates(rng, R, 1e2, 1e5)
    kf = 10 ** rng.uniform(-3, 0, R)
    kr = 10 ** rng.uniform(-3, 0, R)
    t = ensemble_template(sb)
    e = sb.Ensemble(t, R)
    e.set_boxes(np.zeros((R, 3)), np.repeat(side[:, None], 3, 1))
    e.set_rates("fwd", kf)
    e.set_rates("rev", kr)
    e.add_molecules("A", n // 2 + n % 2)
    e.add_molecules("B", n // 2)
    e.radius_mode(1)
    t0 = time.perf_counter()
    e.update()
    setup = time.perf_counter() - t0
    t_tune = time.perf_counter()
    tune_ms = e.autotune(10) if not args.no_tune else None
    t_tune = time.perf_counter() - t_tune
    stream = torch.cuda.Stream()
    e.set_stream(stream.cuda_stream)
    e.run_steps(args.warmup)
    steps = args.batched_steps
    l0 = e.launches()
    sec = time_on_stream(torch, stream, lambda: e.run_steps(steps))
    launches = int(e.launches() - l0)
    engine = {1: "step pipeline", 2: "persistent"}.get(e.engine(), "?")
    tot = float(n.sum())
    ev = e.events()
    # the same ensemble on the persistent kernel, fewer steps (per-step cost is flat)
    e.engine(2)
    e.run_steps(args.warmup)
    psteps = min(steps, 100)
    psec = time_on_stream(torch, stream, lambda: e.run_steps(psteps))
    out = {"workload": "4096 replicates, N log-uniform [1e2,1e5] at density 0.01, kf,kr log-uniform [1e-3,1], "
                       "reflective cubes, A+B<->C, dt=0.01, radii by the device FP64 solver",
           "engine": engine, "value": tot * steps / sec, "unit": METRIC, "molecules": int(tot), "replicates": R,
           "steps": steps, "ms_per_step": sec * 1e3 / steps, "setup_s": setup, "gpu_launches": launches,
           "tuning": e.tuning(), "autotune_s": t_tune, "autotune_best_trial_ms": tune_ms,
           "events": {"rxn1": ev[2], "rxn2": ev[3], "overflow": ev[6]},
           "persistent_kernel": {"value": tot * psteps / psec, "steps": psteps, "ms_per_step": psec * 1e3 / psteps,
                                 "note": "one thread block per replicate, up to 100 steps per launch"}}
    out["persistent_vs_pipeline"] = out["persistent_kernel"]["value"] / out["value"]
    e.close()
    return out


def run_surrogate(sb, torch, args, rank):
    """Surrogate sweep: 65,536 replicates, N log-uniform in [1e2, 1e4] at
    density 0.01, rates redrawn every 100 steps over 5000 steps (fewer with
    --surrogate-steps); radii from the MLP surrogate (exact fallback above
    1e-3 estimated rate error).  Compared with the plain form (each replicate
    its own simulation) on a sample of replicates; the solvers are timed
    alone on the sweep's 65,536 radius problems; the measured rate-constant
    error is taken over independent seeds."""
    rng = np.random.default_rng(777 + rank)
    R = 65536
    n, side = draw_replicates(rng, R, 1e2, 1e4)
    rho = 1.5
    sur = sb.Surrogate()
    t0 = time.perf_counter()
    loss, train_s = sur.train(nsamples=1_000_000, epochs=80, batch=512, lr=3e-3, seed=12345)
    t = ensemble_template(sb, placement=(sb.RPratio, rho))
    e = sb.Ensemble(t, R)
    e.set_boxes(np.zeros((R, 3)), np.repeat(side[:, None], 3, 1))

    def redraw():
        e.set_rates("fwd", 10 ** rng.uniform(-3, 0, R))
        e.set_rates("rev", 10 ** rng.uniform(-3, 0, R))

    redraw()
    e.add_molecules("A", n // 2 + n % 2)
    e.add_molecules("B", n // 2)
    e.attach(sur)
    e.radius_mode(2)
    e.update()
    setup = time.perf_counter() - t0
    stream = torch.cuda.Stream()
    e.set_stream(stream.cuda_stream)
    e.run_steps(args.warmup)
    steps = max(100, args.surrogate_steps // 100 * 100)
    fb = []
    upd = []

    def work():
        for blk in range(steps // 100):
            redraw()
            e.synchronize()  # the update's own cost, not the previous block's steps
            t1 = time.perf_counter()
            e.update()
            upd.append(time.perf_counter() - t1)
            fb.append(e.fallbacks())
            e.run_steps(100)

    sec = time_on_stream(torch, stream, work)
    tot = float(n.sum())
    engine = {1: "step pipeline", 2: "persistent"}.get(e.engine(), "?")
    # cost of one redraw's update by radius mode: surrogate vs exact device vs
    # exact host (median of 3 redraws each, after the engine is idle)
    solver = {}
    for mode, name in ((2, "surrogate"), (1, "exact_device"), (0, "exact_host")):
        e.radius_mode(mode)
        ts = []
        for _ in range(3):
            redraw()
            e.synchronize()
            t1 = time.perf_counter()
            e.update()
            ts.append(time.perf_counter() - t1)
        solver[name + "_s"] = float(np.median(ts))
    out = {"workload": "65536 replicates, N log-uniform [1e2,1e4] at density 0.01, A+B<->C with unbinding ratio "
                       "%.1f, kf,kr log-uniform [1e-3,1] redrawn every 100 steps, dt=0.01, radii from the MLP "
                       "surrogate with exact fallback" % rho,
           "engine": engine, "value": tot * steps / sec, "unit": METRIC, "molecules": int(tot), "replicates": R,
           "steps": steps, "redraws": len(fb), "ms_per_step": sec * 1e3 / steps, "setup_s": setup,
           "redraw_update_s_mean": float(np.mean(upd)), "surrogate_train_s": train_s,
           "surrogate_loss": loss, "fallbacks_per_redraw_mean": float(np.mean(fb)),
           "fallback_fraction": float(np.mean(fb)) / R, "update_seconds": solver}
    e.close()
    out["solver_throughput"] = solver_throughput(sb, sur, rng, R, rho)
    # plain form: sampled replicates run one at a time as ordinary simulations
    idx = rng.choice(R, 24, replace=False)
    mol_steps, secs = 0.0, 0.0
    for k in idx:
        s = sb.Sim(3, (0, 0, 0), (side[k],) * 3)
        for nm, d in zip(("A", "B", "C"), DIFC):
            s.add_species(nm, d)
        for d in range(3):
            s.boundary(d, -1, "r")
        s.set_times(0, 1e9, DT)
        s.add_reaction("fwd", "A", "B", ["C"], 10 ** rng.uniform(-3, 0))
        s.add_reaction("rev", "C", None, ["A", "B"], 10 ** rng.uniform(-3, 0))
        s.set_products("rev", sb.RPratio, rho)
        s.add_molecules("A", int(n[k] // 2 + n[k] % 2))
        s.add_molecules("B", int(n[k] // 2))
        s.update()
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        s.run_steps(3)
        secs += time_on_stream(torch, st, lambda: s.run_steps(100))
        mol_steps += float(n[k]) * 100
        s.close()
    out["plain_form"] = {"value": mol_steps / secs, "unit": METRIC, "sampled_replicates": len(idx),
                         "note": "each replicate run as its own simulation through the same engine"}
    out["speedup_vs_plain_form"] = out["value"] / out["plain_form"]["value"]
    out["rate_check"] = surrogate_rate_check(sb, sur, rng)
    return out


def solver_throughput(sb, sur, rng, R, rho, dt=DT):
    """Radius solves per second on the sweep's problem set (R binding radii
    of A+B with unbinding ratio rho, kf log-uniform [1e-3, 1], D_A + D_B = 2):
    the MLP surrogate with its secant correction and exact fallback
    (smolgpuSurrogatePairRadii) against the exact FP64 device solver
    (smolgpuSolveRadii, doubling plus 15 bisections per problem), each call
    timed alone (host arrays in and out, best of 5)."""
    kf = 10 ** rng.uniform(-3, 0, R)
    ds = np.full(R, DIFC[0] + DIFC[1])
    res = {}
    best = 1e30
    for _ in range(5):
        t0 = time.perf_counter()
        b_sur, _, nfb = sur.pair_radii(kf, ds, dt, same=0, rev=1, rparamt=sb.RPratio, rparam=rho)
        best = min(best, time.perf_counter() - t0)
    res["surrogate_solves_per_s"] = R / best
    res["surrogate_fallbacks"] = int(nfb)
    best = 1e30
    for _ in range(5):
        t0 = time.perf_counter()
        b_ex = sb.solve_radii_device(0, kf, dt, ds, np.full(R, rho), rel=1)
        best = min(best, time.perf_counter() - t0)
    res["exact_device_solves_per_s"] = R / best
    res["surrogate_vs_exact"] = res["surrogate_solves_per_s"] / res["exact_device_solves_per_s"]
    res["max_radius_rel_diff"] = float(np.max(np.abs(b_sur / b_ex - 1)))
    res["problems"] = R
    return res


def surrogate_rate_check(sb, sur, rng, R=65536, steps=500, every=25):
    """Measured rate-constant error of the surrogate radii against the exact
    FP64 solver over independent seeds, at the sweep's configuration
    (65,536 replicates, N log-uniform [1e2, 1e4], kf, kr log-uniform
    [1e-3, 1], unbinding ratio 1.5): the ensemble runs once with surrogate
    radii and once with exact device radii, each with its own seed and
    molecule placement.  For each run the measured forward rate constant,
    relative to each replicate's requested one, is
        (forward events) / sum_r kf_r * integral A_r B_r / V_r dt
    (counts sampled every 25 steps, trapezoid rule); the error is the
    surrogate's ratio over the exact run's, with its Poisson standard error."""
    n, side = draw_replicates(rng, R, 1e2, 1e4)
    kf = 10 ** rng.uniform(-3, 0, R)
    kr = 10 ** rng.uniform(-3, 0, R)
    vol = side ** 3
    res = {}
    for mode, seed in ((2, 101), (1, 202)):
        t = ensemble_template(sb, placement=(sb.RPratio, 1.5))
        t.seed(seed)
        e = sb.Ensemble(t, R)
        e.set_boxes(np.zeros((R, 3)), np.repeat(side[:, None], 3, 1))
        e.set_rates("fwd", kf)
        e.set_rates("rev", kr)
        e.add_molecules("A", n // 2 + n % 2)
        e.add_molecules("B", n // 2)
        if mode == 2:
            e.attach(sur)
        e.radius_mode(mode)
        e.update()
        ev0 = e.events()[3]
        c = e.counts(4)
        expo = np.zeros(R)
        prev = c[:, 1].astype(float) * c[:, 2] / vol
        for _ in range(steps // every):
            e.run_steps(every)
            c = e.counts(4)
            cur = c[:, 1].astype(float) * c[:, 2] / vol
            expo += 0.5 * (prev + cur) * every * DT
            prev = cur
        fwd = e.events()[3] - ev0
        res[mode] = (float(fwd), float(np.sum(kf * expo)))
        e.close()
    (f_s, x_s), (f_e, x_e) = res[2], res[1]
    r_s, r_e = f_s / x_s, f_e / x_e
    err = r_s / r_e - 1
    se = np.sqrt(1 / max(f_s, 1) + 1 / max(f_e, 1))
    return {"replicates": R, "steps": steps, "forward_events_surrogate": f_s, "forward_events_exact": f_e,
            "measured_over_requested_surrogate": r_s, "measured_over_requested_exact": r_e,
            "rate_constant_rel_error": err, "standard_error": se,
            "note": "independent seeds and placements; forward events over the exposure sum kf*A*B/V dt"}


SURF_CONFIG = """dim 3
species A B C
difc A 2
difc B 1
difc C 0.2
boundaries 0 0 200
boundaries 1 0 200
boundaries 2 0 200
time_start 0
time_stop 5
time_step 0.005
random_seed %d
start_surface walls
action both all reflect
panel rect +0 0 0 0 200 200
panel rect -0 200 0 0 200 200
panel rect +1 0 0 0 200 200
panel rect -1 0 200 0 200 200
panel rect +2 0 0 0 200 200
panel rect -2 0 0 200 200 200
end_surface
start_surface membrane
action both all reflect
panel sphere 100 100 100 80 30 30
end_surface
start_surface sink
action both all absorb
panel rect +0 190 0 0 200 200
end_surface
reaction fwd A + B -> C 0.05
reaction decay C -> 0 0.01
end_file
"""


def run_surfaces(sb, torch, args, rank):
    """Surfaces workload: cube of side 200 closed by reflective panels, a
    reflective sphere of radius 80 (cell membrane) at the centre, an absorbing
    plane at x = 190; 4e6 molecules in equal thirds A, B, C (D = 2, 1, 0.2),
    60% uniform inside the sphere and 40% outside; A + B -> C (0.05) and
    C -> 0 (0.01); dt = 0.005."""
    import ctypes as C
    rng = np.random.default_rng(31 + rank)
    n = 4_000_000
    nin = int(0.6 * n)
    c = np.array([100.0, 100.0, 100.0])
    # inside: uniform in the ball; outside: uniform in the cube minus the ball
    u = rng.normal(size=(nin, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    pin = c + u * (80.0 * (1 - 1e-6)) * rng.uniform(size=(nin, 1)) ** (1.0 / 3.0)
    pout = np.empty((0, 3))
    while len(pout) < n - nin:
        q = rng.uniform(1e-3, 200 - 1e-3, size=(2 * (n - nin), 3))
        q = q[(np.linalg.norm(q - c, axis=1) > 80.0 * (1 + 1e-6)) & (q[:, 0] < 190.0)]
        pout = np.concatenate([pout, q])[: n - nin]
    pos = np.concatenate([pin, pout])
    sp = rng.integers(1, 4, size=n).astype(np.int32)
    lib = sb.load()
    d = tempfile.mkdtemp(prefix="smolsurf_")
    try:
        with open(os.path.join(d, "surf.txt"), "w") as f:
            f.write(SURF_CONFIG % (5 + rank))
        simp = C.c_void_p()
        rc = lib.smolLoadSimFromFile((d + "/").encode(), b"surf.txt", C.byref(simp), b"")
        if rc != 0:
            return {"error": str(sb.last_error())}
        s = sb.Sim(ptr=simp.value)
        s.set_molecules(pos, sp)
        s.update()
        tune_ms = s.autotune(10) if not args.no_tune else None
        stream = torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        s.run_steps(args.warmup)
        n0 = s.total()
        steps = 200
        sec = time_on_stream(torch, stream, lambda: s.run_steps(steps))
        n1 = s.total()
        out = {"workload": "surfaces: cube 200 closed by reflective panels, reflective sphere r=80 at the centre, "
                           "absorbing plane x=190; 4e6 molecules A/B/C in thirds (D=2,1,0.2), 60% inside the "
                           "sphere; A+B->C 0.05, C->0 0.01; dt=0.005",
               "value": 0.5 * (n0 + n1) * steps / sec, "unit": METRIC, "molecules_start": int(n0),
               "molecules_end": int(n1), "steps": steps, "ms_per_step": sec * 1e3 / steps,
               "tuning": s.tuning(), "autotune_best_trial_ms": tune_ms}
        s.close()
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


BOUND_CONFIG = """dim 3
species A B
difc A 1
difc B 1
difc A(front) 0.1
boundaries 0 0 100
boundaries 1 0 100
boundaries 2 0 100
time_start 0
time_stop 1000
time_step 0.01
random_seed %d
start_surface walls
action both all reflect
panel rect +0 0 0 0 100 100
panel rect -0 100 0 0 100 100
panel rect +1 0 0 0 100 100
panel rect -1 0 100 0 100 100
panel rect +2 0 0 0 100 100
panel rect -2 0 0 100 100 100
end_surface
start_surface cell
action both all reflect
rate A fsoln front 2
rate A front fsoln 0.5
panel sph 50 50 50 30 20 20
end_surface
reaction bnd A(front) + B -> A(front) 0.5
reaction birth 0 -> B 0.005
mol 500000 A u u u
mol 500000 B u u u
surface_mol 200000 A(front) cell sph all
end_file
"""


def run_surface_bound(sb, torch, args, rank):
    """Surface-bound states: cube 100 closed by reflective panels, a sphere of
    radius 30 where A adsorbs (rate 2) and desorbs (0.5) and diffuses bound
    (D 0.1); bound A removes solution B (A(front) + B -> A(front), 0.5), B is
    born in the volume (0.005); 5e5 A and 5e5 B in solution, 2e5 A bound;
    dt = 0.01.  Molecule-steps count solution and bound molecules."""
    d = tempfile.mkdtemp(prefix="smolbound_")
    try:
        with open(os.path.join(d, "bound.txt"), "w") as f:
            f.write(BOUND_CONFIG % (9 + rank))
        s = sb.Sim.load_file(os.path.join(d, "bound.txt"))
        s.update()
        stream = torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        s.run_steps(args.warmup)
        count = lambda: sum(s.count(nm, sb.MSall) for nm in ("A", "B"))
        n0, b0 = count(), s.count("A", sb.MSfront)
        steps = 200
        sec = time_on_stream(torch, stream, lambda: s.run_steps(steps))
        n1, b1 = count(), s.count("A", sb.MSfront)
        out = {"workload": "surface-bound states: cube 100 closed by reflective panels, sphere r=30 with A "
                           "adsorbing (2) and desorbing (0.5), bound diffusion 0.1, A(front) + B -> A(front) 0.5, "
                           "0 -> B 0.005; 5e5 A, 5e5 B in solution, 2e5 A bound; dt=0.01",
               "value": 0.5 * (n0 + n1) * steps / sec, "unit": METRIC, "molecules_start": int(n0),
               "molecules_end": int(n1), "bound_start": int(b0), "bound_end": int(b1), "steps": steps,
               "ms_per_step": sec * 1e3 / steps}
        s.close()
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_rdf_tables(sb, args, rank, world):
    """Radial-distribution-function solver: regenerate the irreversible rate
    table (600 radial points, eps 1e-5, upward and downward sweeps averaged)
    and the reversible one (500 points, 16 unbinding radii) on the device.
    The work unit is one solver iteration (a diffusion step over the grid,
    n^2 Green's-function pairs, plus an absorption); the CPU baseline times
    the reference's own rdfsteadystate (compiled from rxnparam.c) on the first
    two solves of the upward 600-point sweep."""
    import ctypes as C
    import time
    out = {"unit": "rdf iterations/s (600-point grid)"}
    t0 = time.perf_counter()
    flux, iters = sb.rdf_table("i", 600, 1e-5, "a")
    t1 = time.perf_counter()
    yi = sb.rxn_table("yi")
    out.update({"value": float(iters.sum()) / (t1 - t0), "table_s": t1 - t0, "iterations": int(iters.sum()),
                "max_dev_vs_compiled_table": float(np.max(np.abs(flux.reshape(-1) - yi)))})
    t0 = time.perf_counter()
    flux_r, iters_r = sb.rdf_table("r", 500, 1e-5, "a")
    t1 = time.perf_counter()
    out["reversible_table"] = {"table_s": t1 - t0, "iterations": int(iters_r.sum()), "max_dev_vs_compiled_table":
                               float(np.max(np.abs(flux_r.reshape(-1) - sb.rxn_table("yr"))))}
    if rank != 0 or world != 1 or args.no_cpu_baseline:
        return out
    here = os.path.dirname(os.path.abspath(__file__))
    so = os.path.join(here, "oracle", "_ref", "librxnparam_ref.so")
    if not os.path.exists(so):
        out["cpu_baseline"] = {"value": None, "sample": "reference rxnparam library not built"}
        return out
    ref = C.CDLL(so)
    ref.rdfsteadystate.restype = C.c_double
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    n = 600
    r = np.zeros(n)
    i, dr = 1, 10.0 / n
    while r[i - 1] < 1:  # table grid, rxnparam.c:965-971
        r[i] = r[i - 1] + dr
        i += 1
    r[i - 1], r[i] = 0.9999, 1.0001
    for k in range(i + 1, n):
        r[k] = r[k - 1] + dr
    trial = np.where(r < 1, 0.0, 1.0 - 1.0 / np.maximum(r, 1e-9))
    steps = [np.exp(-3.0), np.exp(-3.0) * np.exp(0.2)]

    def sweep(fn, extra):
        g, d = np.ascontiguousarray(trial.copy()), np.zeros(n)
        for st in steps:
            fn(dp(r), dp(g), dp(d), n, C.c_double(st), C.c_double(1.0), C.c_double(-1.0), C.c_double(1e-5),
               C.c_double(1.0), *extra())
    t0 = time.perf_counter()
    sweep(ref.rdfsteadystate, lambda: ())
    secs = time.perf_counter() - t0
    # iteration counts from the oracle's restatement, bit-identical to the
    # reference's rdfsteadystate on these inputs
    ora = C.CDLL(os.path.join(here, "oracle", "_ref", "liboracle.so"))
    ora.ora_rdf_steady.restype = C.c_double
    counts = []

    def counted():
        it = C.c_int()
        counts.append(it)
        return (C.byref(it),)
    sweep(ora.ora_rdf_steady, counted)
    it_cpu = sum(c.value for c in counts)
    out["cpu_baseline"] = {"value": it_cpu / secs, "unit": out["unit"], "cores": 1, "kind": "reference",
                           "sample": "reference rdfsteadystate (rxnparam.c) on the first two solves of the upward "
                                     "600-point sweep: %d iterations in %.2f s" % (it_cpu, secs),
                           "table_s_extrapolated": out["iterations"] / (it_cpu / secs)}
    return out


def run_e2e(sb, args, rank, world, dist, barrier):
    import torch
    s2 = build_sim(sb, N_MOL, L_SIDE, 101 + rank)
    pos0, sp0, sn = s2.molecules()  # host arrays (pending molecules)
    # the inputs live in pinned host memory, as a caller streaming states to
    # the GPU would keep them
    pos_t = torch.empty(pos0.shape, dtype=torch.float64, pin_memory=True)
    sp_t = torch.empty(sp0.shape, dtype=torch.int32, pin_memory=True)
    pos, sp = pos_t.numpy(), sp_t.numpy()
    pos[:] = pos0
    sp[:] = sp0
    s2.update()
    if not args.no_tune:
        s2.autotune(20)
    s2.run_steps(args.warmup)
    s2.synchronize()
    barrier()
    t0 = time.perf_counter()
    s2.set_molecules(pos, sp)
    names = [b"A", b"B", b"C"]
    for _ in range(args.steps):
        s2.lib.smolRunTimeStep(s2.ptr)
        for nm in names:
            s2.lib.smolGetMoleculeCount(s2.ptr, nm, 0)
    e2e_s = time.perf_counter() - t0
    e2e_molsteps = len(sp) * args.steps
    if dist is not None:
        tt = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
        e2e_molsteps *= world
    e2e = {"value": e2e_molsteps / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": int((pos.nbytes + sp.nbytes) / args.steps),
           "d2h_bytes_per_step": 3 * 8 * 3,
           "note": "includes the host->device upload of all molecules from pinned host memory (amortised "
                   "over the steps) and a per-step species-count read-back"}
    s2.close()
    return e2e


if __name__ == "__main__":
    sys.exit(main())
