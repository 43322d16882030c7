"""Benchmark of the omegagene per-step MD hot path on B200.

Default workload (N=1): 333,334 rigid TIP3P waters (1,000,002 atoms) in a 215.5 A periodic box,
NVE, dt 2 fs, SHAKE trio per water, cutoff 12 A / pair-list 13 A (list rebuilt every 10 steps),
zero-dipole alpha 0.  Inputs are seeded synthetic (a jittered lattice, random orientations).

Prints ONE JSON line.  `value` is ns/day (simulated time per wall-clock day) from CUDA events on
the engine's stream around the timed og_step calls; `e2e` is the same metric through the C ABI
with the state in pinned host memory, copied host->device before and device->host after every
step (coordinates in; coordinates and energies out, as the reference GPU path moves coordinates
and work every step).  With --gpus N (torchrun) every rank advances its own replica (replicas only: the path has
no exchange step), `value` sums the replicas' simulated time and the time is the max over ranks.

--impl reference times the reference's CPU cell-list build (oracle/_ref/omegagene_ns, compiled
from the reference sources) on the host cores: one 9,000-atom water box per core, converted to
the same unit (atom-steps/s at 1M atoms).
"""
import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ns/day@1M atoms"
UNIT = "ns/day"
DT_FS = 2.0
INTVL = 10
VMCMD_TRANS_INTERVAL = 100  # V-McMD walkers: steps between virtual-state transition trials
EQUIL_STEPS = 2000  # 1M water: untimed relaxation (0.5 fs, 300 K velocity rescaling) before the NVE run
N_WATERS = 333334
# the step's pair kernel by autotuned variant; pair_kernel_ms brackets everything one launch
# issues (variant 10: its j-list build, which does work at the first step of a list)
PAIR_KERNELS = {9: "k_pair_ljzd_jq<0,0,5,128,0>",
                10: "k_pair_ljzd_jl<0,0,5,128,0> (+ k_jl_build at list builds)"}
BOX = 215.5
LATTICE = 70
FLOP_PER_PAIR = 40  # FP32 FLOP per interacting pair (sub 3, r2 5, rsqrt 1, powers 4, LJ 5, ZD 6, force 3, accum 6, energy 7)
WORKLOAD = ("333334 TIP3P waters (1000002 atoms), 215.5 A cubic box, NVE dt 2 fs, SHAKE-trio rigid water, "
            "cutoff 12 A, pair-list cutoff 13 A rebuilt every 10 steps, zero-dipole alpha 0; seeded lattice start "
            "relaxed for 2000 untimed steps at 0.5 fs with 300 K velocity rescaling")


def ns_per_day(steps_per_s, dt_fs=DT_FS):
    return dt_fs * steps_per_s * 86400.0 / 1e6


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


# ------------------------------------------------------------------ clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference CPU program

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "omegagene_ns")
REF_RUN = """--mode md
--integrator leapfrog-presto
--cutoff 12.0
--n-steps {n_steps}
--time-step 2.0
--electrostatic zero-dipole
--ele-alpha 0
--thermostat none
--temperature 300
--com-motion cancel
--com-cancel-group-name all
--print-interval-log 1
--print-interval-coord 100000
--fn-o-coord run.cod
--format-o-coord presto
--fn-o-log md.log
--fn-o-energy md.ene
--fn-o-restart run_o.restart
--nsgrid-cutoff 13.0
--nsgrid-update-intvl 10
--constraint shake
--const-max-loops 1000
--const-tolerance 0.0000001
--expected-num-density 1.0
"""


def reference_cpu(n_steps, warmup, cores=None, n_waters=3000, box=44.8):
    """Runs the reference cell-list CPU program, one process (one 9,000-atom box) per core.
    Per-step times come from its own "Comput Time" log lines (cumulative CPU seconds of the MD
    loop, DynamicsMode.cpp:339-340).  Returns atom-steps/s summed over processes."""
    from omegagene_b200 import cls_io, systems  # the generator and the .cls writer
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/omegagene_ns was not built (reference sources absent at build time)"
    cores = cores or os.cpu_count() or 1
    work = tempfile.mkdtemp(prefix="ogref_")
    procs = []
    n_atoms = 3 * n_waters
    for c in range(cores):
        d = os.path.join(work, "p%d" % c)
        os.makedirs(d)
        s = systems.water_system(n_waters, box=box, seed=100 + c, lattice_m=15)
        # empty restraint sections: the reference allocates the restraint arrays only while
        # loading them and frees them at exit (Read.cpp:86-95, DynamicsMode.cpp:178-179)
        s["raw"] = {"dist_restraint": b"\0\0\0\0", "pos_restraint": b"\0\0\0\0"}
        cls_io.write_cls(os.path.join(d, "md.inp.cls"), s)
        open(os.path.join(d, "md.inp.run"), "w").write(REF_RUN.format(n_steps=n_steps + warmup))
        procs.append(subprocess.Popen([REF_BIN, "--cfg", "md.inp.run", "--inp", "md.inp.cls"], cwd=d,
                                      stdout=open(os.path.join(d, "out.txt"), "w"), stderr=subprocess.STDOUT))
    per_step = []
    for c, p in enumerate(procs):
        p.wait()
        txt = open(os.path.join(work, "p%d" % c, "out.txt")).read()
        t = [float(x) for x in re.findall(r"Comput Time:\s+([0-9.eE+-]+)", txt)]
        if p.returncode != 0 or len(t) < n_steps + warmup:
            shutil.rmtree(work, ignore_errors=True)
            return None, "reference program failed (rc=%s, %d steps logged)" % (p.returncode, len(t))
        per_step.append((t[warmup + n_steps - 1] - t[warmup - 1]) / n_steps if warmup > 0 else t[n_steps - 1] / n_steps)
    shutil.rmtree(work, ignore_errors=True)
    atom_steps = sum(n_atoms / s for s in per_step)
    return {"atom_steps_per_s": atom_steps, "cores": cores, "s_per_step": statistics.median(per_step),
            "sample": "%d processes x %d-atom water box (44.8 A), %d timed steps after %d warm-up, reference "
                      "CPU cell-list build (oracle/_ref/omegagene_ns)" % (cores, n_atoms, n_steps, warmup)}, None


def cpu_ns_per_day_at_1m(atom_steps_per_s):
    return ns_per_day(atom_steps_per_s / 1e6)


# ------------------------------------------------------------------ distributed helpers

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def replica_value(steps, ms_max, world):
    """Whole-job ns/day of `world` independent replicas: each ran `steps` steps, the slowest in
    ms_max (max over ranks), and every replica's simulated time counts."""
    return ns_per_day(steps / (ms_max / 1e3)) * world


# ------------------------------------------------------------------ our arm

def run_ours(args, world, rank, local, pg):
    import torch
    from omegagene_b200 import engine, systems
    torch.cuda.set_device(local)
    s = systems.water_system(N_WATERS, box=BOX, seed=20 + rank, lattice_m=LATTICE)
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=INTVL, time_step=DT_FS, thermostat="none", com_cancel_groups=["all"])
    # the lattice start melts and heats: relax it (untimed) with velocity rescaling to 300 K at
    # 0.5 fs, so that the NVE run starts from liquid water
    if args.equil_steps > 0:
        eq = engine.Engine(local)
        eq.add_system(s, dict(p, thermostat="scaling", temperature=300.0, time_step=0.5))
        eq.finalize()
        eq.step(args.equil_steps)
        crd, vel = eq.get_state(0)
        eq.close()
        s = dict(s, crd=crd, vel=vel)
    eng = engine.Engine(local)
    eng.add_system(s, p)
    eng.finalize()
    tuning = eng.tuning()
    n_atoms = s["n_atoms"]
    n_dist = 3 * len(s["constraint"]["trio_atoms"]) + len(s["constraint"]["pair_atoms"])
    # warm-up (untimed)
    eng.step(args.warmup)
    # interacting pairs of the current configuration (roofline numerator)
    eng.compute_forces()
    n_int = eng.pair_count(0)
    n_cell_pairs = eng.grid_info(0)[2]
    # keep the trajectory phase aligned with the list rebuild interval
    rem = (-args.warmup) % INTVL
    if rem:
        eng.step(rem)
    builds0 = eng.jlist_builds()
    eng.set_timing(True)
    clocks = ClockSampler(local)
    barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    eng.step(args.steps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    st = eng.stats()
    jl_builds = eng.jlist_builds() - builds0
    barrier(pg)
    ms_total = max_over_ranks(pg, st["step_ms"])
    pair_ms = st["pair_kernel_ms"] / args.steps
    launches = st["kernel_launches"]
    value = replica_value(args.steps, ms_total, world)
    # ---- end to end through the C ABI with host state (pinned) copied every step
    eng.set_timing(False)
    crd_h = torch.empty(3 * n_atoms, dtype=torch.float64, pin_memory=True)
    vel_h = torch.empty(3 * n_atoms, dtype=torch.float64, pin_memory=True)
    ene_h = torch.empty(11, dtype=torch.float64, pin_memory=True)
    eng.get_state_async_ptr(0, crd_h.data_ptr(), vel_h.data_ptr(), ene_h.data_ptr())
    eng.synchronize()
    e2e_steps = max(10, min(args.steps, 100))
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        # the reference GPU path's per-step traffic: coordinates in; here coordinates and
        # energies out (velocities stay on the device with the integrator)
        eng.put_state_ptr(0, crd_h.data_ptr(), 0)
        eng.step_async(1)
        eng.get_state_async_ptr(0, crd_h.data_ptr(), 0, ene_h.data_ptr())
        eng.synchronize()
    t_e2e = max_over_ranks(pg, time.perf_counter() - t0)
    flags = eng.flags()
    # ---- NVE drift of the engine over 500 further steps (untimed), from its per-step energies,
    # in calls of 100 steps; a call that faults (the synthetic water's hydrogens carry no LJ term,
    # and very rarely one collapses onto a neighbour's oxygen at 2 fs) ends the segment
    n_drift, tot, drift_note = 500, [], ""
    eng.set_trace(100)
    for _ in range(n_drift // 100):
        try:
            eng.step(100)
        except engine.OgError as ex:
            if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                raise
            drift_note = "; a system fault ended the segment after %d steps" % len(tot)
            break
        tot.extend(eng.get_trace(100)[:, 0, engine.ENERGY_NAMES.index("total")])
        eng.set_trace(100)
    t_ns = np.arange(len(tot)) * DT_FS * 1e-6
    dof = 3 * n_atoms - 3 - n_dist
    drift = float(np.polyfit(t_ns, np.asarray(tot), 1)[0]) / dof if len(tot) >= 100 else None
    # forces and state of the last configuration, for the FP64 check in the CPU leg
    eng.set_trace(0)
    eng.compute_forces()
    acc_work, acc_ene, _ = eng.get_forces(0)
    acc_crd, _ = eng.get_state(0)
    e2e = {"value": ns_per_day(e2e_steps / t_e2e) * world, "unit": UNIT,
           "h2d_bytes_per_step": 8 * 3 * n_atoms, "d2h_bytes_per_step": 8 * 3 * n_atoms + 8 * 11,
           "protocol": "per step: og_put_state (coordinates, pinned host -> device), og_step_async(1), "
                       "og_get_state_async (coordinates and energies, device -> pinned host), og_synchronize",
           "steps": e2e_steps}
    eng.close()
    pk = peaks()
    sm_max = (pk or {}).get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s: SMs x FP32 lanes x FMA x max clock
    achieved = FLOP_PER_PAIR * n_int / (pair_ms / 1e3) / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "pair_kernel_traffic.json")
    if os.path.exists(tp):
        try:
            tj = json.load(open(tp))["variants"][str(tuning["pair_variant"])]
            traffic = tj["dram_bytes_per_launch_per_1M_atoms"] * n_atoms / 1e6
        except Exception:
            traffic = None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms_per_gpu": n_atoms, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (cell-pair list %.0f MB, slot arrays %.0f MB)" % (
                       n_cell_pairs * 16 / 1e6, n_atoms * 1.07 * 64 / 1e6),
                   "arithmetic": "pair forces FP32 with int64 fixed-point accumulation; FP64 integrator, SHAKE, "
                                 "energies"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak, "traffic": traffic,
                     "kernel": PAIR_KERNELS.get(tuning["pair_variant"], "k_pair_ljzd"), "pair_kernel_ms": pair_ms,
                     "interacting_pairs": n_int,
                     "flop_per_pair": FLOP_PER_PAIR, "autotune": tuning,
                     "cell_pairs": n_cell_pairs,
                     "cluster_efficiency": n_int / (64.0 * n_cell_pairs) if n_cell_pairs else None,
                     "jlist_builds": jl_builds,
                     "jlist_note": "pair variant 10: j-list builds in the timed steps (at every cell-pair list "
                                   "build and whenever an atom had moved past the 0.35 A skin); pair_kernel_ms "
                                   "includes them",
                     "peak_note": "FP32 CUDA-core peak = 148 SMs x 128 lanes x 2 x %.0f MHz (nominal at the "
                                  "measured max SM clock; MEASURED_PEAKS.json has no FP32 figure)" % sm_max},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk, "device_flags": flags,
        "accuracy": {"nve_drift_kcal_mol_ns_dof": drift, "nve_drift_sample": "%d NVE steps after the timed region "
                     "(total energy per step, least-squares slope / %d degrees of freedom)%s" % (len(tot), dof,
                                                                                          drift_note)},
    }
    out["_acc"] = (dict(s, crd=acc_crd), p, acc_work, acc_ene)
    return out


def accuracy_vs_oracle(system, params, work, ene):
    """The FP64 oracle (the cell-list evaluator of the same step in double precision) against the
    engine's forces and energies at the configuration the bench ended on: per-atom force RMS
    relative error and the potential's relative error.  Part of the CPU leg."""
    import time as _t
    from oracle import ogo
    t0 = _t.perf_counter()
    md = ogo.OracleMD(system, params)
    ref = md.forces()
    w64 = md.work.reshape(-1, 3)
    err = float(np.sqrt(((work - w64) ** 2).sum() / (w64 ** 2).sum()))
    return {"force_rms_rel_err": err, "potential_rel_err": abs(ene["potential"] - ref["potential"]) /
            abs(ref["potential"]), "vdw_rel_err": abs(ene["vdw"] - ref["vdw"]) / abs(ref["vdw"]),
            "ele_rel_err": abs(ene["ele"] - ref["ele"]) / abs(ref["ele"]),
            "oracle": "FP64 over the reference's cell-pair list, all %d atoms (%.0f s on the host)" % (
                len(w64), _t.perf_counter() - t0)}


# ------------------------------------------------------------------ serving workload

def run_serve(args):
    """Batched serving stream: jobs of 500-10,000 TIP3P waters (log-uniform, box at 0.997 g/cm^3),
    300 K velocity rescaling, SHAKE, dt 2 fs.  Two runs of the continuous-batching server over
    the same jobs: all jobs queued at t=0 (aggregate capacity, the `value`), then Poisson arrivals
    at 80% of that capacity (p50/p99 latency).  The plain path (one job at a time, one engine
    each) is timed on a sample of jobs across the size range, fitted as a + b*atoms, and queued
    first come first served on the same arrivals."""
    import torch
    from omegagene_b200 import engine, serve, systems
    torch.cuda.set_device(0)
    rng = np.random.default_rng(3)
    n_jobs, steps = args.jobs, args.job_steps
    counts = np.exp(rng.uniform(np.log(500), np.log(10000), n_jobs)).astype(int)
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=INTVL, time_step=DT_FS, thermostat="scaling", temperature=300.0)
    built = [systems.water_system(int(c), seed=1000 + k) for k, c in enumerate(counts)]

    def jobs_at(arrivals):
        return [serve.Job(k, built[k], p, steps, arrival_s=float(arrivals[k])) for k in range(n_jobs)]

    total = float(sum(3 * counts) * steps)
    sat = serve.Server(0, max_jobs=args.max_jobs, window=args.window).run(jobs_at(np.zeros(n_jobs)))
    cap = sat["atom_steps_per_s"]
    inter = total / n_jobs / (0.8 * cap)
    arrivals = np.cumsum(rng.exponential(inter, n_jobs))
    arrivals -= arrivals[0]
    stream = serve.Server(0, max_jobs=args.max_jobs, window=args.window).run(jobs_at(arrivals))
    # plain path: one engine per job; a sample across the size range, service time a + b*atoms
    order = np.argsort(counts)
    sample = order[np.linspace(0, n_jobs - 1, min(args.plain_sample, n_jobs)).astype(int)]
    ts, na = [], []
    for k in sample:
        dt, _, _, _ = serve.run_alone(serve.Job(int(k), built[int(k)], p, steps))
        ts.append(dt)
        na.append(3 * int(counts[k]))
    b, a = np.polyfit(na, ts, 1)
    service = a + b * 3 * counts
    plain_cap = total / float(service.sum())
    lat_plain, _ = serve.fifo_latencies(arrivals, service)
    return {
        "metric": "batch atom-steps/s", "value": cap, "unit": "atom-steps/s", "n_gpus": 1,
        "steps": steps, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": "%d TIP3P water jobs, 500-10000 waters log-uniform (seed 3), %d steps each, dt 2 fs, "
                               "SHAKE, 300 K rescaling" % (n_jobs, steps),
                   "max_jobs": args.max_jobs, "window_steps": args.window,
                   "timing": "wall clock from the first arrival to the last completion, engine creation, "
                             "graph capture and state hand-over included"},
        "saturated": {"span_s": sat["span_s"], "relayouts": sat["relayouts"], "relayout_s": sat["relayout_s"],
                      "mean_batch": sat["mean_batch"], "p50_latency_s": sat["latency_p50_s"],
                      "p99_latency_s": sat["latency_p99_s"]},
        "serving": {"arrivals": "Poisson, mean inter-arrival %.4f s (80%% of the saturated capacity)" % inter,
                    "atom_steps_per_s": stream["atom_steps_per_s"], "p50_latency_s": stream["latency_p50_s"],
                    "p99_latency_s": stream["latency_p99_s"], "span_s": stream["span_s"],
                    "relayouts": stream["relayouts"], "relayout_s": stream["relayout_s"],
                    "mean_batch": stream["mean_batch"]},
        "plain": {"atom_steps_per_s": plain_cap, "p50_latency_s": float(np.percentile(lat_plain, 50)),
                  "p99_latency_s": float(np.percentile(lat_plain, 99)),
                  "service_fit_s": {"a": float(a), "b_per_atom": float(b)},
                  "sample": "%d jobs run alone (one engine each, graph capture included)" % len(sample)},
        "speedup_vs_plain": cap / plain_cap,
    }


# ------------------------------------------------------------------ McMD workload

def run_walkers(walkers, params, polys, n_steps, chunk, trace=False, vs_logs=None):
    """Steps all walkers in one engine, `chunk` steps per og_step call.  A walker whose system
    faults is dropped: og_step undoes the chunk for every walker, the rest are re-formed into a
    new engine (same step number, so the same trajectories) and the chunk is redone.  Returns
    the surviving indices, their states, the per-step trace of the survivors (or None), the
    device time of every og_step call (failed ones included) and the atom-steps completed.
    With V-McMD sections in `polys`, walker k draws with random_seed + k; a re-formed engine
    gets each walker's virtual state and generator, and the virtual-state logs are collected into
    `vs_logs` (walker -> list of states) when given."""
    from omegagene_b200 import engine
    keep = list(range(len(walkers)))
    state = {k: (walkers[k]["crd"], walkers[k]["vel"]) for k in keep}
    polys = list(polys) if polys else None
    vm = bool(polys) and "states" in polys[0]

    def collect(eng):
        for i, k in enumerate(keep):
            cur, mt = eng.vmcmd_state(i)
            polys[k] = dict(polys[k], cur_vs=cur, mt_state=mt)
            if vs_logs is not None:
                vs_logs.setdefault(k, []).extend(eng.take_vs_log(i)[1].tolist())

    traces = {k: [] for k in keep}
    done, ms, atom_steps, dropped = 0, 0.0, 0, []
    variant = -1  # the first engine autotunes; a re-formed one keeps its choice
    while done < n_steps:
        eng = engine.Engine(0)
        eng.set_tuning(variant)
        for k in keep:
            s = dict(walkers[k])
            s["crd"], s["vel"] = state[k]
            pk = dict(params, random_seed=params.get("random_seed", 0) + k) if vm else params
            eng.add_system(s, pk, polys[k] if polys else None, first_step=done)
        eng.finalize()
        variant = eng.tuning()["pair_variant"]
        eng.set_timing("step")
        if trace:
            eng.set_trace(n_steps)
        faulted = False
        while done < n_steps:
            n = min(chunk, n_steps - done)
            try:
                eng.step(n)
            except engine.OgError as ex:
                if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                    raise
                ms += eng.stats()["step_ms"]
                f = eng.system_faults()
                for i, k in enumerate(keep):
                    state[k] = eng.get_state(i)
                if vm:
                    collect(eng)
                dropped += [k for i, k in enumerate(keep) if f[i]]
                keep = [k for i, k in enumerate(keep) if not f[i]]
                faulted = True
                break
            ms += eng.stats()["step_ms"]
            atom_steps += n * sum(walkers[k]["n_atoms"] for k in keep)
            done += n
            if trace:
                tr = eng.get_trace(n_steps)
                for i, k in enumerate(keep):
                    traces[k].extend(tr[:, i, :])
                eng.set_trace(n_steps)
            for i, k in enumerate(keep):
                state[k] = eng.get_state(i)
        if vm and not faulted:
            collect(eng)
        eng.close()
        if not faulted:
            break
    tr = np.array([traces[k] for k in keep]).transpose(1, 0, 2) if trace else None
    return keep, [state[k] for k in keep], tr, ms, atom_steps, dropped


def run_mcmd(args):
    """64 V-McMD walkers (a 300-atom synthetic chain in 2,500 TIP3P waters each, own seeds,
    hydrogens held by angle terms), 300 K velocity rescaling, in one engine.  Protocol: 400
    steps at 0.5 fs (the generator's contacts relax), a 100-step unscaled prerun at 2 fs whose
    potential energies give each walker's virtual-state ladder (four overlapping windows over
    mean +- 4 sd, each with its own order-6 polynomial, a transition trial every 100 steps and
    the lambda logged every step, as the reference's sample V-McMD run logs it), then the timed
    V-McMD run at 2 fs.  Compared with the same walkers run one at a time."""
    import torch
    from omegagene_b200 import engine, serve, systems
    torch.cuda.set_device(0)
    walkers = [systems.chain_water_system(300, 2500, seed=args.walker_seed0 + w, radius=12.0, h_angles=True)
               for w in range(args.walkers)]
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=INTVL, time_step=DT_FS, thermostat="scaling", temperature=300.0)
    warm_p = dict(p, time_step=0.5)
    keep, states, _, _, _, drop_warm = run_walkers(walkers, warm_p, None, 400, 400)
    walkers = [dict(walkers[k], crd=c, vel=v) for k, (c, v) in zip(keep, states)]
    keep, states, tr, _, _, drop_pre = run_walkers(walkers, p, None, 100, 100, trace=True)
    walkers = [dict(walkers[k], crd=c, vel=v) for k, (c, v) in zip(keep, states)]
    pot = tr[:, :, engine.ENERGY_NAMES.index("potential")]
    polys = [systems.vmcmd_ladder(pot[:, w].mean(), max(pot[:, w].std(), 1.0), seed=900 + w, n_vs=4,
                                  interval=VMCMD_TRANS_INTERVAL, e_start=pot[-1, w]) for w in range(len(walkers))]
    p = dict(p, random_seed=1000 * args.walker_seed0 + 1, print_intvl_extended_lambda=1)
    # timed run: whole list intervals, so og_step replays the captured graph
    vs_logs = {}
    keep, _, _, ms, atom_steps, drop_run = run_walkers(walkers, p, polys, args.steps, args.chunk, vs_logs=vs_logs)
    batched = atom_steps / (ms / 1e3)
    moves = [int(np.count_nonzero(np.diff([polys[k]["init_vs"] - 1] + vs_logs.get(k, [])))) for k in keep]
    ts = []
    for w, m in list(zip(walkers, polys))[:2]:
        job = serve.Job(0, w, p, min(args.steps, 2000), mcmd=m)
        dt, _, _, _ = serve.run_alone(job, warmup=INTVL)
        ts.append(job.n_atoms * job.n_steps / dt)
    plain = float(np.mean(ts))
    n_atoms = sum(w["n_atoms"] for w in walkers)
    return {"metric": "batch atom-steps/s", "value": batched, "unit": "atom-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": 500, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": "%d McMD walkers, 300-atom chain in 2500 TIP3P waters each (%d atoms total), "
                                   "dt 2 fs, 300 K velocity rescaling, V-McMD: 4 virtual states per walker "
                                   "(order-6 polynomials), a transition trial every %d steps, lambda logged every "
                                   "step" % (args.walkers, n_atoms, VMCMD_TRANS_INTERVAL),
                       "timing": "CUDA events around every og_step call of %d steps, engine re-forming after a "
                                 "fault excluded" % args.chunk},
            "walkers_dropped": {"warm_up": len(drop_warm), "prerun": len(drop_pre), "run": len(drop_run),
                                "note": "a walker whose system faults (og_get_system_faults) is retired; the "
                                        "others are re-stepped from the undone call"},
            "vstate_moves": {"mean_per_walker": float(np.mean(moves)) if moves else 0.0,
                             "trials_per_walker": args.steps // VMCMD_TRANS_INTERVAL},
            "plain": {"atom_steps_per_s": plain, "sample": "2 walkers run alone (wall clock around og_step)"},
            "speedup_vs_plain": batched / plain}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--equil-steps", type=int, default=EQUIL_STEPS,
                    help="water1m: untimed relaxation steps before the NVE run (0: start from the lattice, "
                         "e.g. for a short launch list under a profiler)")
    ap.add_argument("--workload", default="water1m", choices=["water1m", "serve", "mcmd"],
                    help="water1m: the 1M-atom step (default); serve: batched job stream; mcmd: McMD walkers")
    ap.add_argument("--jobs", type=int, default=256)
    ap.add_argument("--job-steps", type=int, default=5000)
    ap.add_argument("--max-jobs", type=int, default=64)
    ap.add_argument("--window", type=int, default=100)
    ap.add_argument("--plain-sample", type=int, default=8)
    ap.add_argument("--walkers", type=int, default=64)
    ap.add_argument("--walker-seed0", type=int, default=500)
    ap.add_argument("--chunk", type=int, default=100, help="McMD: steps per og_step call")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload in ("serve", "mcmd") and args.impl == "ours":
        if int(os.environ.get("RANK", "0")) == 0:
            out = run_serve(args) if args.workload == "serve" else run_mcmd(args)
            print(json.dumps(out))
        return
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        if rank != 0:
            return
        steps = min(args.steps, 60)
        res, why = reference_cpu(steps, min(args.warmup, 10))
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        v = cpu_ns_per_day_at_1m(res["atom_steps_per_s"])
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0, "steps": steps,
            "warmup": min(args.warmup, 10), "ms_per_step": res["s_per_step"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": WORKLOAD + " (measured on the bounded sample below, scaled by atom count)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": res["cores"], "kind": "reference",
                             "sample": res["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return
    out = run_ours(args, world, rank, local, pg)
    acc = out.pop("_acc", None)
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:  # the CPU leg runs at N = 1 only
            out["accuracy"].update(accuracy_vs_oracle(*acc))
            res, why = reference_cpu(args.cpu_steps, 3)
            if res is not None:
                out["cpu_baseline"] = {"value": cpu_ns_per_day_at_1m(res["atom_steps_per_s"]), "unit": UNIT,
                                       "cores": res["cores"], "kind": "reference", "sample": res["sample"]}
            else:
                out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": why}
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
