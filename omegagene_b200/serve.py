"""Continuous-batching MD job server on one GPU.

Jobs (a system, run parameters and a step count) arrive over time. The server keeps every running
job in one engine, so all their atoms advance in the same kernel launches. At each window
boundary (a multiple of the pair-list interval) it does the following:
* retires finished jobs;
* admits queued jobs, first come first served, while the device-memory budget and the job cap allow;
* re-creates the engine for the new batch. Each continuing job carries over its positions,
  velocities and its own step number, so its list-rebuild phase and heating schedule continue
  unchanged.

A V-McMD job also carries its virtual state and its generator (og_get_vmcmd_state), and its
virtual-state and lambda logs are collected into the job at every boundary.

A job's trajectory is therefore the one it would have had alone. The engine's forces are
fixed-point sums and its reductions are per system, so the match is exact;
tests/test_gpu_serve.py checks it.

The next batch is built while the current window runs (prepare_ahead): which jobs finish at the
window's end and which queued jobs the rules admit are known when the window starts, so a
background thread creates and finalizes that engine, with the continuing jobs' step numbers and
placeholder coordinates; when the window ends as planned, their positions and velocities are
set with og_set_state (the list is built from them at the first step) and the engine takes over.
The result is the same engine the boundary would have built.  A window that faults, a job
arriving that the rules would admit, a V-McMD job in the batch (its generator state is only
known at the boundary) or a build that failed (two handles at once may not fit) falls back to
building the batch at the boundary.

A job whose system faults (a coordinate leaves the box or turns non-finite) is retired as failed
with its state at the start of the window; og_step undoes the window for every job, and the
others are stepped again in a new engine, with the results they would have had anyway.

Latency of a job = completion time - arrival time (wall clock). Throughput = atom-steps of all
jobs / (last completion - first arrival).
"""
import collections
import concurrent.futures
import time

import numpy as np

from . import engine

# device footprint per atom assumed until the server has measured an engine: state, grid, cell
# pairs, list scratch and, for the j-list pair kernel, its entries (a 60-job water batch of 546k
# atoms holds 1,728 bytes per atom with the j-queue kernel, 4,054 with the j-list kernel).  Every
# engine the server builds then reports what it holds (og_get_footprint), and admission uses the
# largest measured bytes per atom so far, with a 10% margin.
BYTES_PER_ATOM = 4200
FOOTPRINT_MARGIN = 1.1


class Job:
    def __init__(self, job_id, system, params, n_steps, arrival_s=0.0, mcmd=None):
        self.id = job_id
        self.system = system
        self.params = dict(params)
        self.n_steps = int(n_steps)
        self.arrival_s = float(arrival_s)
        self.mcmd = mcmd
        self.n_atoms = int(system["n_atoms"])
        self.crd = np.asarray(system["crd"], np.float64).copy()
        self.vel = np.asarray(system["vel"], np.float64).copy()
        self.steps_done = 0
        self.failed = False
        self.fault = 0
        self.t_admit = None
        self.t_done = None
        self.energies = None
        self.vs_log, self.lambda_log = [], []  # (step, 0-based state) / (step, lambda) of a V-McMD job
        intvl = self.params.get("nsgrid_update_intvl", 1)
        if self.n_steps % intvl:
            raise ValueError("job %s: n_steps must be a multiple of nsgrid_update_intvl" % job_id)

    @property
    def vmcmd(self):
        return self.mcmd is not None and "states" in self.mcmd

    def collect_vmcmd(self, eng, i):
        """Moves this job's V-McMD logs out of engine slot i and keeps its virtual state and
        generator, so that the next engine continues the run."""
        st, vs = eng.take_vs_log(i)
        self.vs_log += list(zip(st.tolist(), vs.tolist()))
        st, lam = eng.take_lambda_log(i)
        self.lambda_log += list(zip(st.tolist(), lam.tolist()))
        cur, mt = eng.vmcmd_state(i)
        self.mcmd = dict(self.mcmd, cur_vs=cur, mt_state=mt)

    @property
    def bytes(self):
        return self.n_atoms * BYTES_PER_ATOM

    @property
    def latency_s(self):
        return None if self.t_done is None else self.t_done - self.arrival_s


class Server:
    def __init__(self, device=0, hbm_budget_bytes=None, max_jobs=64, window=100, pair_variant="auto",
                 clock=time.perf_counter, sleep=time.sleep, engine_factory=None, prepare_ahead=True,
                 bytes_per_atom=None):
        """pair_variant: a fixed pair-kernel variant, or "auto": the first engine autotunes and
        every later engine reuses its choice, so a job keeps one kernel (and bitwise results)
        across re-formed batches.  prepare_ahead: build the next batch's engine during the
        current window when the next batch is known (see the module docstring).  bytes_per_atom:
        a fixed admission estimate; None measures every engine built (og_get_footprint) and
        admits by the largest bytes per atom seen, starting from BYTES_PER_ATOM."""
        self.device = device
        if hbm_budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget_bytes = int(0.5 * free)
        self.budget = hbm_budget_bytes
        self.max_jobs = max_jobs
        self.window = window
        self.pair_variant = pair_variant
        self.clock = clock
        self.sleep = sleep
        self.n_relayouts = 0
        self.n_prepared = 0  # relayouts served by an engine built during the previous window
        self.relayout_s = 0.0
        self.prepare_ahead = prepare_ahead
        self.batch_sizes = []
        self.engine_factory = engine_factory or engine.Engine
        self.measure = bytes_per_atom is None
        self.bytes_per_atom = float(BYTES_PER_ATOM if bytes_per_atom is None else bytes_per_atom)
        self.measured_bytes_per_atom = 0.0
        self.batch_footprints = []  # (atoms, peak device bytes) of every engine built

    def job_bytes(self, j):
        """Device memory a job is expected to take (the admission estimate)."""
        return j.n_atoms * self.bytes_per_atom

    def _measured(self, eng, members):
        """Records the engine's footprint and, when measuring, raises the admission estimate to
        the largest bytes per atom seen (with the margin)."""
        if not hasattr(eng, "footprint"):
            return
        _, peak = eng.footprint()
        atoms = sum(j.n_atoms for j, *_ in members)
        self.batch_footprints.append((atoms, peak))
        if atoms and self.measure:
            self.measured_bytes_per_atom = max(self.measured_bytes_per_atom, peak / atoms)
            self.bytes_per_atom = FOOTPRINT_MARGIN * self.measured_bytes_per_atom

    def _build(self, active):
        eng = self._engine_for([(j, j.crd, j.vel, j.steps_done) for j in active])
        if self.pair_variant == "auto":
            self.pair_variant = eng.tuning()["pair_variant"]
        self.n_relayouts += 1
        return eng

    def _engine_for(self, members):
        """A finalized engine of (job, coordinates, velocities, first step) members, in order."""
        eng = self.engine_factory(self.device)
        if self.pair_variant != "auto":
            eng.set_tuning(self.pair_variant)
        for j, crd, vel, first in members:
            s = dict(j.system)
            s["crd"], s["vel"] = crd, vel
            eng.add_system(s, j.params, j.mcmd, first_step=first)
        eng.finalize()
        self._measured(eng, members)
        return eng

    def _admits(self, running, queue):
        """Queued jobs the rules admit next to the running ones, first come first served."""
        used = sum(self.job_bytes(j) for j in running)
        out = []
        for j in queue:
            n = len(running) + len(out)
            if n >= self.max_jobs or (used + self.job_bytes(j) > self.budget and n > 0):
                break
            out.append(j)
            used += self.job_bytes(j)
        return out

    def _prepare(self, pool, active, queue, w):
        """Starts building the batch that follows a window of w steps ending as planned: returns
        (continuing jobs, admitted jobs, future of the engine), or None."""
        if not self.prepare_ahead or self.pair_variant == "auto":
            return None
        cont = [j for j in active if j.steps_done + w < j.n_steps]
        admit = self._admits(cont, queue)
        if len(cont) == len(active) and not admit:
            return None  # no boundary after this window
        if not cont and not admit:
            return None
        if any(j.vmcmd for j in cont + admit):
            return None
        members = [(j, j.crd, j.vel, j.steps_done + w) for j in cont] + [(j, j.crd, j.vel, j.steps_done)
                                                                          for j in admit]
        return cont, admit, pool.submit(self._engine_for, members)

    @staticmethod
    def _discard(prep):
        if prep is not None:
            try:
                prep[2].result().close()
            except Exception:  # a build that failed left nothing to close
                pass

    def run(self, jobs):
        """Runs every job to completion; returns a summary dict (throughput, latencies)."""
        intvls = {j.params.get("nsgrid_update_intvl", 1) for j in jobs}
        if len(intvls) != 1:
            raise ValueError("all jobs of one server share nsgrid_update_intvl")
        intvl = intvls.pop()
        if self.window % intvl:
            raise ValueError("window must be a multiple of nsgrid_update_intvl")
        with concurrent.futures.ThreadPoolExecutor(max_workers=1) as pool:
            return self._run(jobs, pool)

    def _run(self, jobs, pool):
        future = collections.deque(sorted(jobs, key=lambda j: j.arrival_s))
        queue = collections.deque()
        active, done, failed = [], [], []
        eng = None
        prep = None  # (continuing, admitted, engine future) built during the last window
        t0 = self.clock()
        first_arrival = future[0].arrival_s if future else 0.0
        while future or queue or active:
            now = self.clock() - t0
            while future and future[0].arrival_s <= now:
                queue.append(future.popleft())
            finished = [j for j in active if j.steps_done >= j.n_steps]
            used = sum(self.job_bytes(j) for j in active if j.steps_done < j.n_steps)
            n_run = len(active) - len(finished)
            admit = []
            while queue and n_run + len(admit) < self.max_jobs and (
                    used + self.job_bytes(queue[0]) <= self.budget or n_run + len(admit) == 0):
                # (a job estimated above the whole budget still runs, alone)
                admit.append(queue.popleft())
                used += self.job_bytes(admit[-1])
            if finished or admit:
                t_re = self.clock()
                cont = [j for j in active if j.steps_done < j.n_steps]
                ahead = None  # the engine built during the window, when it is the one needed
                if prep is not None and prep[0] == cont and prep[1] == admit:
                    try:
                        ahead = prep[2].result()
                    except Exception:  # e.g. no room for two handles: build at the boundary
                        ahead = None
                    prep = None
                if eng is not None:
                    for i, j in enumerate(active):
                        j.crd, j.vel = eng.get_state(i)
                        j.energies = eng.get_energies(i)
                        if j.vmcmd:
                            j.collect_vmcmd(eng, i)
                    self._measured(eng, [(j,) for j in active])  # the peak includes any list growth
                    eng.close()
                    eng = None
                now = self.clock() - t0
                for j in finished:
                    j.t_done = now
                    done.append(j)
                active = cont + admit
                for j in admit:
                    j.t_admit = now
                if ahead is not None:
                    eng = ahead
                    for i, j in enumerate(cont):
                        eng.set_state(i, j.crd, j.vel)
                    self.n_relayouts += 1
                    self.n_prepared += 1
                    self.batch_sizes.append(len(active))
                else:
                    self._discard(prep)
                    if active:
                        eng = self._build(active)
                        self.batch_sizes.append(len(active))
                prep = None
                self.relayout_s += self.clock() - t_re
            else:
                self._discard(prep)  # (a window that ended as planned always has a boundary)
                prep = None
            if not active:
                if future:
                    wait = future[0].arrival_s - (self.clock() - t0)
                    if wait > 0:
                        self.sleep(wait)
                continue
            w = min(self.window, min(j.n_steps - j.steps_done for j in active))
            prep = self._prepare(pool, active, queue, w)
            try:
                eng.step(w)
            except engine.OgError as ex:
                if ex.status != engine.OG_ERR_SYSTEM_FAULT:
                    raise
                self._discard(prep)
                prep = None
                bad = eng.system_faults()
                t_re = self.clock()
                for i, j in enumerate(active):
                    j.crd, j.vel = eng.get_state(i)
                    if j.vmcmd:
                        j.collect_vmcmd(eng, i)  # the undone call's entries are gone already
                eng.close()
                eng = None
                now = self.clock() - t0
                for i, j in enumerate(active):
                    if bad[i]:
                        j.failed, j.fault, j.t_done = True, int(bad[i]), now
                        failed.append(j)
                active = [j for i, j in enumerate(active) if not bad[i]]
                if active:
                    eng = self._build(active)
                    self.batch_sizes.append(len(active))
                self.relayout_s += self.clock() - t_re
                continue
            for j in active:
                j.steps_done += w
        t_end = max(j.t_done for j in done + failed) if done or failed else 0.0
        lat = np.array([j.latency_s for j in done]) if done else np.zeros(1)
        atom_steps = sum(j.n_atoms * j.n_steps for j in done)
        span = t_end - first_arrival
        return {"n_jobs": len(done), "n_failed": len(failed), "failed": failed, "atom_steps": atom_steps, "span_s": span,
                "atom_steps_per_s": atom_steps / span if span > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "relayouts": self.n_relayouts, "prepared_relayouts": self.n_prepared, "relayout_s": self.relayout_s,
                "mean_batch": float(np.mean(self.batch_sizes)) if self.batch_sizes else 0.0,
                "jobs": done}


def run_alone(job, device=0, pair_variant="auto", warmup=0, logs=None):
    """The plain path: one job, one engine, start to finish; returns (seconds, final energies,
    final positions, final velocities).  `warmup` extra steps run first, untimed (a timing aid:
    the returned state is then `warmup` steps further on).  For a V-McMD job, `logs` (a dict)
    receives the "vs" and "lambda" logs as (step, value) lists."""
    eng = engine.Engine(device)
    if pair_variant != "auto":
        eng.set_tuning(pair_variant)
    s = dict(job.system)
    eng.add_system(s, job.params, job.mcmd)
    eng.finalize()
    if warmup:
        eng.step(warmup)
    t = time.perf_counter()
    eng.step(job.n_steps)
    dt = time.perf_counter() - t
    crd, vel = eng.get_state(0)
    ene = eng.get_energies(0)
    if logs is not None and job.vmcmd:
        st, vs = eng.take_vs_log(0)
        logs["vs"] = list(zip(st.tolist(), vs.tolist()))
        st, lam = eng.take_lambda_log(0)
        logs["lambda"] = list(zip(st.tolist(), lam.tolist()))
    eng.close()
    return dt, ene, crd, vel


def fifo_latencies(arrivals, service_s):
    """Latencies of a one-at-a-time server (first come first served) for the given arrival
    times and per-job service times; also returns the span from the first arrival to the last
    completion."""
    t = 0.0
    out = []
    for a, s in sorted(zip(arrivals, service_s)):
        start = max(t, a)
        t = start + s
        out.append(t - a)
    return np.array(out), t - min(arrivals)
