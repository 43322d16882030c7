"""Benchmark of the omegagene per-step MD hot path on B200.

Default workload (N=1): 333,334 rigid TIP3P waters (1,000,002 atoms) in a 215.5 A periodic box,
NVE, dt 2 fs, SHAKE trio per water, cutoff 12 A / pair-list 16 A, zero-dipole alpha 0.  Inputs are
seeded synthetic (a jittered lattice, random orientations).  The cell-pair list is rebuilt
whenever an atom has moved half the 4 A list margin since the last build (exact lists), not on
the reference's fixed 10-step schedule with its 13 A list, which loses pairs of this water's
fastest atoms.

Prints ONE JSON line.  `value` is ns/day (simulated time per wall-clock day) from CUDA events on
the engine's stream around the timed og_step calls (CUDA-graph replays); `e2e` is the same metric
through the C ABI with the state in pinned host memory, copied host->device before and
device->host after every step (coordinates in; coordinates and energies out, as the reference GPU
path moves coordinates and work every step).  With --gpus N (torchrun) every rank advances its
own replica (replicas only: the path has no exchange step), `value` sums the replicas' simulated
time and the time is the max over ranks.

At N = 1 the line also carries, untimed: the FP64 checks of every workload of the benchmark's
configurations (`accuracy`, `configs`), a bounded batched-serving stream against the plain path
run job by job (`batched`) and a bounded batched McMD run (`mcmd`).

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
# pair-list cutoff by list policy: the reference's 13 A with its fixed schedule; 16 A when the
# list is rebuilt on displacement (a 2 A trigger: 19 builds in 400 steps at 1M atoms against 54
# at 14 A; 2.04 ms per step against 2.17, the 29% more cell pairs included; 17 and 18 A measure
# within 0.5% of 16 A)
LIST_CUTOFF = {"fixed": 13.0, "displacement": 16.0}
PAIR_TIMING_STEPS = 10  # kernel-by-kernel steps whose pair launches are timed for the roofline
PAIRED_STEPS, PAIRED_GAP = 150, 150  # paired FP32-vs-FP64 drift: segment length, steps between starts
CHAIN_STEPS = 1000  # timed thermostatted steps of the solvated chain
CHAIN_RELAX = 2000  # its relaxation at 0.5 fs
FLOP_PER_PAIR = 40  # FP32 FLOP per interacting pair (sub 3, r2 5, rsqrt 1, powers 4, LJ 5, ZD 6, force 3, accum 6, energy 7)
WORKLOAD = ("333334 TIP3P waters (1000002 atoms), 215.5 A cubic box, NVE dt 2 fs, SHAKE-trio rigid water, "
            "cutoff 12 A, pair-list cutoff 16 A rebuilt whenever an atom has moved 2 A, zero-dipole alpha 0; "
            "seeded lattice start relaxed for 2000 untimed steps at 0.5 fs with 300 K velocity rescaling")


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
                                      "--format=csv,noheader,nounits", "-lms", "50"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if os.path.getsize(self.path) == 0:  # a timed region shorter than the sampling period
            with open(self.path, "w") as f:
                subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                "--format=csv,noheader,nounits"], stdout=f, stderr=subprocess.DEVNULL, timeout=30)
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


# ------------------------------------------------------------------ background CPU work
# Spawned worker processes (no CUDA in them): system generation and FP64 oracle checks run on
# host cores while the GPU works.

def w_walkers(seeds):
    from omegagene_b200 import systems
    return [systems.chain_water_system(300, 2500, seed=int(k), radius=12.0) for k in seeds]


def w_chain():
    from omegagene_b200 import systems
    return systems.chain_water_system(2000, 30000, seed=1, radius=30.0, n_sigma_bins=None)


def w_oracle(system, params, work, ene):
    return accuracy_vs_oracle(system, params, work, ene)


# ------------------------------------------------------------------ our arm

def _params(**kw):
    from omegagene_b200 import engine
    p = dict(engine.DEFAULT_PARAMS)
    p.update(kw)
    return p


def _engine(system, params, variant=-1, policy="displacement", device=0):
    from omegagene_b200 import engine
    eng = engine.Engine(device)
    eng.set_tuning(variant)
    eng.set_list_policy(policy)
    eng.add_system(system, params)
    eng.finalize()
    return eng


def _relax(system, device, n_steps, dt=0.5):
    """The configurations' relaxation: velocity rescaling to 300 K at 0.5 fs."""
    eng = _engine(system, _params(nsgrid_update_intvl=INTVL, time_step=dt, thermostat="scaling",
                                  temperature=300.0), device=device)
    eng.step(n_steps)
    crd, vel = eng.get_state(0)
    eng.close()
    return dict(system, crd=crd, vel=vel)


def _dof(system):
    c = system["constraint"]
    return 3 * system["n_atoms"] - 3 - 3 * len(c["trio_atoms"]) - len(c["pair_atoms"]) - 6 * len(c["quad_atoms"])


def nve_drift(eng, system, n_steps, dt_fs=DT_FS, chunk=100):
    """Least-squares slope of the total energy per degree of freedom over n_steps further steps
    of an engine (kcal/mol/ns/dof), from its per-step trace; a system fault ends the window."""
    from omegagene_b200 import engine
    tot, note = [], ""
    for _ in range(n_steps // chunk):
        eng.set_trace(chunk)
        try:
            eng.step(chunk)
        except engine.OgError as ex:
            if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                raise
            note = "a system fault ended the window after %d steps" % len(tot)
            break
        tot.extend(eng.get_trace(chunk)[:, 0, engine.ENERGY_NAMES.index("total")])
    eng.set_trace(0)
    t_ns = np.arange(len(tot)) * dt_fs * 1e-6
    drift = float(np.polyfit(t_ns, np.asarray(tot), 1)[0]) / _dof(system) if len(tot) >= 100 else None
    return drift, len(tot), note


def paired_drift(system, params, device, segments, seg_steps, gap_steps, variant=-1):
    """NVE drift of the engine against the FP64 evaluation along the same trajectory: from shared
    starting states, the production engine and the FP64 pair variant each run seg_steps steps,
    short enough that the two trajectories stay close (the FP32 force error seeds a separation
    that grows about e-fold per 25 steps), so both meet the same events; the slope of the
    difference of their total energies per degree of freedom is the drift the FP32 arithmetic
    adds.  Starting states are gap_steps apart along the production run.  Returns the mean over
    segments, its standard error, and each side's own mean drift."""
    from omegagene_b200 import engine
    names = engine.ENERGY_NAMES
    dof = _dof(system)
    t_ns = np.arange(seg_steps) * params["time_step"] * 1e-6
    diff, d32, d64 = [], [], []
    s = dict(system)
    note = ""
    for k in range(segments):
        runs = []
        for v in (variant, engine.PAIR_VARIANT_F64):
            eng = _engine(s, params, variant=v, device=device)
            eng.set_trace(seg_steps)
            try:
                eng.step(seg_steps)
            except engine.OgError as ex:
                if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                    raise
                note = "a system fault ended segment %d" % k
                eng.close()
                break
            runs.append(eng.get_trace(seg_steps)[:, 0, names.index("total")])
            if v != engine.PAIR_VARIANT_F64:
                crd, vel = eng.get_state(0)
            eng.close()
        if len(runs) < 2:
            break
        diff.append(float(np.polyfit(t_ns, (runs[0] - runs[1]) / dof, 1)[0]))
        d32.append(float(np.polyfit(t_ns, runs[0] / dof, 1)[0]))
        d64.append(float(np.polyfit(t_ns, runs[1] / dof, 1)[0]))
        if k + 1 < segments:
            eng = _engine(dict(s, crd=crd, vel=vel), params, variant=variant, device=device)
            try:
                eng.step(gap_steps)
            except engine.OgError as ex:
                if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                    raise
                note = "a system fault ended the run after segment %d" % k
                eng.close()
                break
            crd, vel = eng.get_state(0)
            eng.close()
            s = dict(s, crd=crd, vel=vel)
    if not diff:
        return {"drift_vs_fp64_kcal_mol_ns_dof": None, "paired_note": note}
    d = np.array(diff)
    return {"drift_vs_fp64_kcal_mol_ns_dof": float(d.mean()),
            "drift_vs_fp64_se": float(d.std(ddof=1) / np.sqrt(len(d))) if len(d) > 1 else None,
            "drift_fp32_segments_mean": float(np.mean(d32)), "drift_fp64_segments_mean": float(np.mean(d64)),
            "protocol": "%d segments of %d NVE steps from shared starts %d steps apart; FP32 engine vs the FP64 "
                        "pair variant (OG_PAIR_VARIANT_F64), exact lists; slope of (E_fp32 - E_fp64) per dof%s"
                        % (len(diff), seg_steps, gap_steps, "; " + note if note else "")}


def run_ours(args, world, rank, local, pg, pool):
    import torch
    from omegagene_b200 import engine, systems
    torch.cuda.set_device(local)
    bg = {}
    if pool is not None:  # CPU work for the extras, started before the first GPU call
        bg["chain"] = pool.submit(w_chain)
        seeds = list(range(args.walker_seed0, args.walker_seed0 + args.walkers))
        per = max(1, (len(seeds) + 7) // 8)
        bg["walkers"] = [pool.submit(w_walkers, seeds[i:i + per]) for i in range(0, len(seeds), per)]
    s = systems.water_system(N_WATERS, box=BOX, seed=20 + rank, lattice_m=LATTICE)
    p = _params(nsgrid_update_intvl=INTVL, time_step=DT_FS, thermostat="none", com_cancel_groups=["all"],
                nsgrid_cutoff=LIST_CUTOFF[args.list_policy])
    # the lattice start melts and heats: relax it (untimed) with velocity rescaling to 300 K at
    # 0.5 fs, so that the NVE run starts from liquid water
    if args.equil_steps > 0:
        s = _relax(s, local, args.equil_steps)
    eng = _engine(s, p, policy=args.list_policy, device=local)
    if args.no_graphs:  # every kernel a launch of its own (for a profiler's launch list)
        eng.set_graphs(False)
    tuning = eng.tuning()
    n_atoms = s["n_atoms"]
    eng.step(args.warmup)  # warm-up (untimed)
    # interacting pairs of the current configuration (roofline numerator)
    eng.compute_forces()
    n_int = eng.pair_count(0)
    n_cell_pairs = eng.grid_info(0)[2]
    rem = (-args.warmup) % INTVL  # whole list intervals in the timed region: graph replays
    if rem:
        eng.step(rem)
    builds0, jl0 = eng.list_builds(), eng.jlist_builds()
    eng.set_timing("step")
    clocks = ClockSampler(local)
    barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    eng.step(args.steps)
    torch.cuda.synchronize()
    st = eng.stats()
    list_builds, jl_builds = eng.list_builds() - builds0, eng.jlist_builds() - jl0
    # the pair kernel alone (roofline): CUDA events around each pair launch, kernel by kernel
    # (the clock samples run on through these steps)
    eng.set_timing(True)
    eng.step(PAIR_TIMING_STEPS)
    pair_ms = eng.stats()["pair_kernel_ms"] / PAIR_TIMING_STEPS
    clk = clocks.stop()
    barrier(pg)
    ms_total = max_over_ranks(pg, st["step_ms"])
    launches = st["kernel_launches"]
    value = replica_value(args.steps, ms_total, world)
    gi = eng.graph_info()
    # ---- end to end through the C ABI with host state (pinned) copied every step.  The loop is
    # driven from the host, so it waits for the background generators of the extras: run beside
    # them it measured 4.0 instead of 3.3 ms per step
    for f in ([bg["chain"]] if "chain" in bg else []) + bg.get("walkers", []):
        f.result()
    eng.set_timing(False)
    crd_h = torch.empty(3 * n_atoms, dtype=torch.float64, pin_memory=True)
    ene_h = torch.empty(engine.N_ENERGY, dtype=torch.float64, pin_memory=True)
    eng.get_state_async_ptr(0, crd_h.data_ptr(), 0, ene_h.data_ptr())
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
    e2e = {"value": ns_per_day(e2e_steps / t_e2e) * world, "unit": UNIT,
           "h2d_bytes_per_step": 8 * 3 * n_atoms, "d2h_bytes_per_step": 8 * 3 * n_atoms + 8 * engine.N_ENERGY,
           "protocol": "per step: og_put_state (coordinates, pinned host -> device), og_step_async(1), "
                       "og_get_state_async (coordinates and energies, device -> pinned host), og_synchronize",
           "steps": e2e_steps}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms_per_gpu": n_atoms, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (cell-pair list %.0f MB, slot arrays %.0f MB)" % (
                       n_cell_pairs * 16 / 1e6, n_atoms * 1.07 * 64 / 1e6),
                   "list_policy": args.list_policy,
                   "timing": "CUDA events around og_step on the engine's stream (graph replays: %s)" % (
                       "on" if gi["enabled"] else "off: " + gi["note"]),
                   "arithmetic": "pair forces FP32 with int64 fixed-point accumulation; FP64 integrator, SHAKE, "
                                 "energies"},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk, "device_flags": flags,
        "lists": {"cell_pair_list_builds": list_builds, "jlist_builds": jl_builds, "steps": args.steps,
                  "note": "builds in the timed steps (displacement policy: whenever an atom had moved half the "
                          "list margin since the last build; j lists also when one passed the 0.35 A skin)"},
    }
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
    out["roofline"] = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                       "frac": achieved / fp32_peak, "traffic": traffic,
                       "kernel": PAIR_KERNELS.get(tuning["pair_variant"], "k_pair_ljzd"), "pair_kernel_ms": pair_ms,
                       "pair_timing": "CUDA events around every pair-kernel launch over %d kernel-by-kernel steps "
                                      "(j-list builds included)" % PAIR_TIMING_STEPS,
                       "interacting_pairs": n_int, "flop_per_pair": FLOP_PER_PAIR, "autotune": tuning,
                       "cell_pairs": n_cell_pairs,
                       "cluster_efficiency": n_int / (64.0 * n_cell_pairs) if n_cell_pairs else None,
                       "peak_note": "FP32 CUDA-core peak = 148 SMs x 128 lanes x 2 x %.0f MHz (nominal at the "
                                    "measured max SM clock; MEASURED_PEAKS.json has no FP32 figure)" % sm_max}
    acc = {}
    if world == 1 and not args.no_extras:
        # ---- accuracy of the 1M run: absolute NVE drift, then the paired drift against FP64
        d, n_d, note = nve_drift(eng, s, args.drift_steps)
        acc.update({"nve_drift_kcal_mol_ns_dof": d,
                    "nve_drift_sample": "%d NVE steps after the timed region, exact lists (total energy per step, "
                                        "least-squares slope / %d degrees of freedom)%s" % (
                                            n_d, _dof(s), "; " + note if note else "")})
        crd, vel = eng.get_state(0)
        eng.close()
        acc.update(paired_drift(dict(s, crd=crd, vel=vel), p, local, args.paired_segments, PAIRED_STEPS,
                                PAIRED_GAP, variant=tuning["pair_variant"]))
        # forces and state of the last configuration, FP64-checked by a background process
        e = _engine(dict(s, crd=crd, vel=vel), p, device=local)
        e.compute_forces()
        work, ene, _ = e.get_forces(0)
        e.close()
        if pool is not None and not args.no_cpu_baseline:
            bg["acc1m"] = pool.submit(w_oracle, dict(s, crd=crd, vel=vel), p, work, ene)
        out["configs"] = run_configs(args, local, pool, bg)
        out["batched"] = run_batched(args, local)
        out["mcmd"] = run_mcmd_bounded(args, local, bg)
        if "acc1m" in bg:
            acc.update(bg["acc1m"].result())
    else:
        eng.close()
    out["accuracy"] = acc
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


# ------------------------------------------------------------------ the other configurations

def _force_check(system, params, device):
    """Engine forces at the system's state against the FP64 oracle (CPU, inline)."""
    e = _engine(system, params, device=device)
    e.compute_forces()
    work, ene, _ = e.get_forces(0)
    e.close()
    return accuracy_vs_oracle(system, params, work, ene)


def run_configs(args, device, pool, bg):
    """FP64 checks of the other configurations: the 9,000-atom water box (relaxed as specified,
    then NVE at 2 fs) and the solvated 2,000-atom chain (thermostatted run as specified, then
    NVE), each with force / energy errors against the FP64 oracle, the absolute NVE drift and
    the paired drift against the FP64 pair variant."""
    from omegagene_b200 import engine, systems
    out = {}
    t0 = time.perf_counter()
    s0 = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    s0 = _relax(s0, device, 2000)
    p0 = _params(nsgrid_update_intvl=INTVL, time_step=2.0)
    c0 = _force_check(s0, p0, device)
    eng = _engine(s0, p0, device=device)
    d, n_d, note = nve_drift(eng, s0, 3000)
    crd, vel = eng.get_state(0)
    eng.close()
    c0.update({"nve_drift_kcal_mol_ns_dof": d, "nve_steps": n_d, "note": note})
    c0.update(paired_drift(dict(s0, crd=crd, vel=vel), p0, device, 8, PAIRED_STEPS, PAIRED_GAP))
    c0["workload"] = ("3,000 TIP3P waters (9,000 atoms), 44.8 A box, 2,000 steps at 0.5 fs with 300 K rescaling, "
                      "then NVE at 2 fs, exact lists")
    c0["wall_s"] = time.perf_counter() - t0
    out["water9k"] = c0
    # the solvated chain
    t0 = time.perf_counter()
    s1 = bg["chain"].result() if "chain" in bg else w_chain()
    p1 = _params(nsgrid_update_intvl=INTVL, time_step=2.0, thermostat="scaling", temperature=300.0)
    s1 = _relax(s1, device, CHAIN_RELAX)  # the generator's start relaxes violently: 0.5 fs first
    eng = _engine(s1, p1, device=device)
    eng.set_timing("step")
    done, ms, fault = 0, 0.0, ""
    while done < CHAIN_STEPS:  # 2 fs with rescaling, in calls of 100 steps (graph replays)
        try:
            eng.step(100)
        except engine.OgError as ex:
            if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                raise
            fault = "a system fault (og_get_system_faults %s) ended the run after %d steps at 2 fs" % (
                eng.system_faults(), done)
            break
        ms += eng.stats()["step_ms"]
        done += 100
    crd, vel = eng.get_state(0)
    eng.close()
    s1 = dict(s1, crd=crd, vel=vel)
    c1 = _force_check(s1, p1, device)
    if done:
        c1.update({"atom_steps_per_s": s1["n_atoms"] * done / (ms / 1e3), "ns_per_day": ns_per_day(done / (ms / 1e3)),
                   "ms_per_step": ms / done})
    c1.update({"timed_steps": done, "note": fault})
    p1n = dict(p1, thermostat="none")
    eng = _engine(s1, p1n, device=device)
    d, n_d, note = nve_drift(eng, s1, 2000)
    eng.close()
    c1.update({"nve_drift_kcal_mol_ns_dof": d, "nve_steps": n_d, "nve_note": note})
    c1.update(paired_drift(s1, p1n, device, 6, PAIRED_STEPS, PAIRED_GAP))
    c1["workload"] = ("2,000-atom chain (per-atom LJ types, SHAKE'd X-H, 111 deg / 63 angles on every bonded "
                      "triple) in 30,000 TIP3P waters less overlaps "
                      "(%d atoms, 97.3 A box); %d steps at 0.5 fs, then up to %d timed steps at 2 fs with 300 K "
                      "rescaling; force check at their end; NVE drift with the thermostat off, exact lists" % (
                          s1["n_atoms"], CHAIN_RELAX, CHAIN_STEPS))
    c1["wall_s"] = time.perf_counter() - t0
    out["chain87k"] = c1
    return out


def run_batched(args, device):
    """Bounded batched-serving stream (the serving configuration at a size that fits the default
    run): jobs of 500-10,000 TIP3P waters (log-uniform), 300 K rescaling, 2 fs, served by the
    continuous-batching server, first all queued at t = 0 (capacity), then with Poisson arrivals
    at 80% of that capacity (p50/p99 latency); the plain path runs every job alone, one engine
    each, one after the other (its own measured time, not a fit), and is queued first come first
    served on the same arrivals."""
    from omegagene_b200 import serve, systems
    rng = np.random.default_rng(3)
    n_jobs, steps = args.batch_jobs, args.batch_job_steps
    counts = np.exp(rng.uniform(np.log(500), np.log(10000), n_jobs)).astype(int)
    p = _params(nsgrid_update_intvl=INTVL, time_step=DT_FS, thermostat="scaling", temperature=300.0)
    built = [systems.water_system(int(c), seed=1000 + k) for k, c in enumerate(counts)]

    def jobs_at(arrivals):
        return [serve.Job(k, built[k], p, steps, arrival_s=float(arrivals[k])) for k in range(n_jobs)]

    total = float(sum(3 * counts) * steps)
    srv = serve.Server(device, max_jobs=args.max_jobs, window=args.window)
    sat = srv.run(jobs_at(np.zeros(n_jobs)))
    variant = srv.pair_variant
    cap = sat["atom_steps_per_s"]
    inter = total / n_jobs / (0.8 * cap)
    arrivals = np.cumsum(rng.exponential(inter, n_jobs))
    arrivals -= arrivals[0]
    stream = serve.Server(device, max_jobs=args.max_jobs, window=args.window, pair_variant=variant).run(
        jobs_at(arrivals))
    service = np.array([serve.run_alone(serve.Job(k, built[k], p, steps), device=device, pair_variant=variant)[0]
                        for k in range(n_jobs)])
    plain_cap = total / float(service.sum())
    lat_plain, _ = serve.fifo_latencies(arrivals, service)
    return {"metric": "batch atom-steps/s", "value": cap, "unit": "atom-steps/s",
            "workload": "%d TIP3P water jobs, 500-10,000 waters log-uniform (seed 3), %d steps each, dt 2 fs, SHAKE, "
                        "300 K rescaling, at most %d jobs per batch, %d-step windows, pair variant %s" % (
                            n_jobs, steps, args.max_jobs, args.window, variant),
            "timing": "wall clock from the first arrival to the last completion: engine creation, graph capture "
                      "and state hand-over included",
            "saturated": {"atom_steps_per_s": cap, "span_s": sat["span_s"], "relayouts": sat["relayouts"],
                          "mean_batch": sat["mean_batch"]},
            "serving": {"arrivals": "Poisson, mean inter-arrival %.4f s (80%% of the saturated capacity)" % inter,
                        "atom_steps_per_s": stream["atom_steps_per_s"], "p50_latency_s": stream["latency_p50_s"],
                        "p99_latency_s": stream["latency_p99_s"], "span_s": stream["span_s"],
                        "relayouts": stream["relayouts"], "mean_batch": stream["mean_batch"]},
            "plain": {"atom_steps_per_s": plain_cap, "p50_latency_s": float(np.percentile(lat_plain, 50)),
                      "p99_latency_s": float(np.percentile(lat_plain, 99)),
                      "note": "every job run alone (one engine each, creation and graph capture included, wall "
                              "clock around og_step), queued first come first served on the same arrivals"},
            "speedup_vs_plain": cap / plain_cap}


def run_mcmd_bounded(args, device, bg):
    """Bounded batched McMD (the walkers configuration with a shorter timed run): 64 V-McMD
    walkers, each a 300-atom chain in 2,500 TIP3P waters, the protocol of run_mcmd with
    args.mcmd_steps timed steps; the plain path runs two walkers alone."""
    from omegagene_b200 import serve, systems, engine
    if "walkers" in bg:
        walkers = [w for f in bg["walkers"] for w in f.result()]
    else:
        walkers = w_walkers(range(args.walker_seed0, args.walker_seed0 + args.walkers))
    p = _params(nsgrid_update_intvl=INTVL, time_step=DT_FS, thermostat="scaling", temperature=300.0)
    keep, states, _, _, _, drop_warm = run_walkers(walkers, dict(p, time_step=0.5), None, 400, 400)
    walkers = [dict(walkers[k], crd=c, vel=v) for k, (c, v) in zip(keep, states)]
    keep, states, tr, _, _, drop_pre = run_walkers(walkers, p, None, 100, 100, trace=True)
    walkers = [dict(walkers[k], crd=c, vel=v) for k, (c, v) in zip(keep, states)]
    pot = tr[:, :, engine.ENERGY_NAMES.index("potential")]
    polys = [systems.vmcmd_ladder(pot[:, w].mean(), max(pot[:, w].std(), 1.0), seed=900 + w, n_vs=4,
                                  interval=VMCMD_TRANS_INTERVAL, e_start=pot[-1, w]) for w in range(len(walkers))]
    p = dict(p, random_seed=1000 * args.walker_seed0 + 1, print_intvl_extended_lambda=1)
    vs_logs = {}
    keep, _, _, ms, atom_steps, drop_run = run_walkers(walkers, p, polys, args.mcmd_steps, args.chunk,
                                                       vs_logs=vs_logs)
    batched = atom_steps / (ms / 1e3)
    ts = []
    for w, m in list(zip(walkers, polys))[:2]:
        job = serve.Job(0, w, p, args.mcmd_steps, mcmd=m)
        dt, _, _, _ = serve.run_alone(job, device=device, warmup=INTVL)
        ts.append(job.n_atoms * job.n_steps / dt)
    plain = float(np.mean(ts))
    moves = [int(np.count_nonzero(np.diff([polys[k]["init_vs"] - 1] + vs_logs.get(k, [])))) for k in keep]
    return {"metric": "batch atom-steps/s", "value": batched, "unit": "atom-steps/s",
            "workload": "%d V-McMD walkers (300-atom chain in 2,500 TIP3P waters each, %d atoms), 4 virtual states, "
                        "a transition trial every %d steps; 400 steps at 0.5 fs and a 100-step prerun, then %d timed "
                        "steps at 2 fs" % (len(walkers), sum(w["n_atoms"] for w in walkers), VMCMD_TRANS_INTERVAL,
                                           args.mcmd_steps),
            "timing": "CUDA events around every og_step call of %d steps" % args.chunk,
            "walkers_retired": {"warm_up": len(drop_warm), "prerun": len(drop_pre), "run": len(drop_run)},
            "vstate_moves_mean": float(np.mean(moves)) if moves else 0.0,
            "plain": {"atom_steps_per_s": plain, "sample": "2 walkers run alone (wall clock around og_step)"},
            "speedup_vs_plain": batched / plain}


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
    walkers = [systems.chain_water_system(300, 2500, seed=args.walker_seed0 + w, radius=12.0)
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
    global WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="water1m: skip the untimed accuracy, configuration, batched and McMD sections")
    ap.add_argument("--equil-steps", type=int, default=EQUIL_STEPS,
                    help="water1m: untimed relaxation steps before the NVE run (0: start from the lattice, "
                         "e.g. for a short launch list under a profiler)")
    ap.add_argument("--list-policy", default="displacement", choices=["displacement", "fixed"],
                    help="water1m: cell-pair list rebuilds when an atom has moved half the margin (exact), or every "
                         "%d steps (the reference's schedule)" % INTVL)
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch the timed steps kernel by kernel instead of replaying CUDA graphs (profiling)")
    ap.add_argument("--drift-steps", type=int, default=2000)
    ap.add_argument("--paired-segments", type=int, default=16)
    ap.add_argument("--batch-jobs", type=int, default=64)
    ap.add_argument("--batch-job-steps", type=int, default=1000)
    ap.add_argument("--mcmd-steps", type=int, default=1000)
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
    if args.list_policy == "fixed":
        WORKLOAD = WORKLOAD.replace("pair-list cutoff 16 A rebuilt whenever an atom has moved 2 A",
                                    "pair-list cutoff 13 A rebuilt every %d steps" % INTVL)
    pool = None
    if world == 1 and not args.no_extras:
        # CPU work beside the GPU's: spawned before the first GPU call
        import concurrent.futures as cf
        import multiprocessing as mp
        pool = cf.ProcessPoolExecutor(max_workers=max(1, min(9, (os.cpu_count() or 2) - 1)),
                                      mp_context=mp.get_context("spawn"))
    try:
        out = run_ours(args, world, rank, local, pg, pool)
    finally:
        if pool is not None:
            pool.shutdown(wait=True, cancel_futures=True)
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:  # the CPU leg runs at N = 1 only
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
