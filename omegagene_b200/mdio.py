"""The reference's run outputs, written from the engine's device-resident state.

File formats (byte for byte those of the reference's writers):
* restart (WriteRestart::write_restart, WriteTrr.cpp:256-313): Fortran-style records of the
  80-byte title, the atom and velocity counts, the step, time and energies, then FP64
  coordinates and velocities;
* presto trajectory (WriteTrrPresto::write_trr, WriteTrr.cpp:179-253): per frame a 44-marked
  header record (step, time and energies in FP32) and the group's FP32 coordinates;
* GROMACS trr (WriteTrrGromacs::write_trr, WriteTrr.cpp:36-177): the reference's "real" is
  double, so coordinates and box are FP64 in nm;
* V-McMD virtual-state log (WriteTTPVMcMDLog, Write.cpp:41-44) and lambda log
  (WriteTableLogBinary / WriteTableLogAscii, Write.cpp:97-160);
* the energy log blocks the reference prints (DynamicsMode::sub_output_log,
  DynamicsMode.cpp:302-357).

``run()`` follows DynamicsMode::main_stream (DynamicsMode.cpp:186-214): steps 0..n_steps-1, a
frame at the start of every step k > 0 that is a multiple of --print-interval-coord, a restart
after every step k that is a multiple of --print-interval-restart, then a frame and the restart
after the loop, and the loop's "last step" n_steps.  Frames are recorded on the device inside
og_step (og_set_trajectory); the host only writes them out.
"""
import struct

import numpy as np

from . import engine

MAGIC_NUMBER = 66261   # CelesteObject.cpp:28
REAL_BYTE = 8          # sizeof(real), CelesteObject.cpp:26
TITLE = b"omegagene_b200"


def write_restart(path, n_steps, time, e_potential, e_kinetic, crd, vel, title=TITLE):
    crd = np.ascontiguousarray(crd, "<f8").reshape(-1, 3)
    vel = np.ascontiguousarray(vel, "<f8").reshape(-1, 3)
    n = len(crd)
    t = bytes(title)[:80].ljust(80, b"\0")
    out = [struct.pack("<i", 80), t, struct.pack("<i", 80),
           struct.pack("<iiii", 8, n, n, 8),
           struct.pack("<iidddd", 36, int(n_steps), float(time), float(e_kinetic + e_potential), float(e_kinetic),
                       float(e_potential)),
           struct.pack("<i", 36),
           struct.pack("<i", n * 24), crd.tobytes(), struct.pack("<i", n * 24),
           struct.pack("<i", n * 24), vel.tobytes(), struct.pack("<i", n * 24)]
    with open(path, "wb") as f:
        f.write(b"".join(out))


def read_restart(path):
    """The fields of a restart file (the layout of kkpresto_restart.PrestoRestartReader)."""
    b = open(path, "rb").read()
    title = b[4:84]
    n_atoms, n_vel = struct.unpack_from("<ii", b, 92)
    n_steps, = struct.unpack_from("<i", b, 108)
    time, e_total, e_kin, e_pot = struct.unpack_from("<dddd", b, 112)
    o = 148
    crd = np.frombuffer(b, "<f8", 3 * n_atoms, o + 4).reshape(-1, 3).copy()
    o += 8 + 24 * n_atoms
    vel = np.frombuffer(b, "<f8", 3 * n_vel, o + 4).reshape(-1, 3).copy()
    return {"title": title, "n_atoms": n_atoms, "n_vel": n_vel, "n_steps": n_steps, "time": time,
            "e_total": e_total, "e_kinetic": e_kin, "e_potential": e_pot, "crd": crd, "vel": vel}


def apply_restart(system, restart):
    """The system with a restart's coordinates and velocities, as the reference's toolkit puts a
    restart into the next run's .cls (kkmmsystem.set_crd_vel_from_restart)."""
    if restart["n_atoms"] != int(system["n_atoms"]):
        raise ValueError("restart holds %d atoms, the system %d" % (restart["n_atoms"], system["n_atoms"]))
    return dict(system, crd=restart["crd"].copy(), vel=restart["vel"].copy())


def presto_frame(step, time, energies, crd, cpu_time=0.0):
    """One WriteTrrPresto frame: energies is the engine's energy dict of the step the frame's
    coordinates belong to.  The header record's leading marker is 44 and its trailing one 0, as
    the reference writes them."""
    e = energies
    hdr = struct.pack("<ii10fi", 44, int(step), time, cpu_time, e["potential"] + e["kinetic"], e["kinetic"],
                      e["temperature"], e["potential"], 0.0, e["vdw"], 0.0, 0.0, 0)
    c = np.ascontiguousarray(crd, "<f4").reshape(-1)
    return hdr + struct.pack("<i", 4 * len(c)) + c.tobytes() + struct.pack("<i", 4 * len(c))


def read_presto_frames(path):
    """[(step, time, header floats, crd[n][3] float32)] of a presto trajectory."""
    b = open(path, "rb").read()
    out, o = [], 0
    while o < len(b):
        _, step = struct.unpack_from("<ii", b, o)
        vals = struct.unpack_from("<10f", b, o + 8)
        nb, = struct.unpack_from("<i", b, o + 52)
        crd = np.frombuffer(b, "<f4", nb // 4, o + 56).reshape(-1, 3).copy()
        out.append((step, vals[0], vals, crd))
        o += 56 + nb + 4
    return out


def gromacs_frame(step, time, box, crd):
    """One WriteTrrGromacs frame with box and coordinates (no velocities or forces); "real" is
    double in the reference, so every real field is FP64 and lengths are in nm."""
    c = np.ascontiguousarray(crd, np.float64).reshape(-1, 3)
    n = len(c)
    hdr = struct.pack("<iii12s", 1993, 13, 12, b"GMX_trn_file")
    hdr += struct.pack("<13i", 0, 0, 9 * 8, 0, 0, 0, 0, n * 3 * 8, 0, 0, n, int(step), 0)
    hdr += struct.pack("<dd", time, 0.0)
    bx = np.zeros(9)
    bx[0], bx[4], bx[8] = box[0] * 0.1, box[1] * 0.1, box[2] * 0.1
    return hdr + bx.astype("<f8").tobytes() + (c * 0.1).astype("<f8").tobytes()


def lambda_log_header():
    return struct.pack("<iii", MAGIC_NUMBER, REAL_BYTE, 1)


def log_block(step, time, e, comput_time=0.0, extended=False):
    """The energy block DynamicsMode::sub_output_log prints for a step."""
    lines = ["Step: %8d    Time: %10.4f" % (step, time),
             "Total:     %14.10e" % e.get("total", e["potential"] + e["kinetic"]),
             "Potential: %14.10e    Kinetic:  %14.10e" % (e["potential"], e["kinetic"]),
             "Bond:      %14.10e    Angle:    %14.10e" % (e["bond"], e["angle"]),
             "Torsion:   %14.10e    Improper: %14.10e" % (e["torsion"], e["improper"]),
             "14-VDW:    %14.10e    14-Ele:   %14.10e" % (e["vdw14"], e["ele14"]),
             "VDW:       %14.10e    Ele:      %14.10e" % (e["vdw"], e["ele"])]
    if extended:
        lines.append("Extended:           %14.10e" % 0.0)  # the reference prints pote_pos_rest here
    lines += ["Temperature:       %14.10e" % e["temperature"], "Comput Time:       %14.10e" % comput_time]
    return "\n".join(lines) + "\n"


def _group_atoms(system, params):
    names = params.get("group_o_crd") or []
    if not names:
        return None
    g = system["groups"]
    return np.asarray(g["atoms"][g["names"].index(names[0])], np.int32)


def run(system, params, mcmd=None, device=0, log=None, pair_variant=None):
    """Runs the reference's MD loop for params["n_steps"] with its outputs: trajectory
    (fn_o_crd, print_intvl_crd, group_o_crd, format_o_crd presto | gromacs), restart
    (fn_o_restart, print_intvl_restart), V-McMD logs (fn_o_vmcmd_log, fn_o_extended_lambda,
    format_o_extended_lambda) and, when `log` is a file object, the energy blocks at
    print_intvl_log.  One trajectory output per run.  Returns the engine's energies of the last
    step (step n_steps)."""
    n = int(params["n_steps"])
    dt = float(params["time_step"])
    ci = (params.get("print_intvl_crd") or [0])[0]
    fn_crd = (params.get("fn_o_crd") or [None])[0]
    if len(params.get("print_intvl_crd") or []) > 1:
        raise ValueError("one trajectory output per run")
    ri = int(params.get("print_intvl_restart", 0) or 0)
    li = int(params.get("print_intvl_log", 0) or 0)
    vm = mcmd is not None and "states" in mcmd
    eng = engine.Engine(device)
    if pair_variant is not None:
        eng.set_tuning(pair_variant)
    eng.add_system(system, params, mcmd)
    group = _group_atoms(system, params)
    if ci > 0 and fn_crd:
        eng.set_trajectory(0, ci, group)
    eng.finalize()
    box = [float(system["pbc_val"][0]), float(system["pbc_val"][4]), float(system["pbc_val"][8])]
    traj = open(fn_crd, "wb") if ci > 0 and fn_crd else None
    vsf = lamf = None
    if vm:
        vsf = open(params["fn_o_vmcmd_log"], "w") if params.get("fn_o_vmcmd_log") else None
        if params.get("fn_o_extended_lambda"):
            binary = params.get("format_o_extended_lambda", "binary") == "binary"
            lamf = open(params["fn_o_extended_lambda"], "wb" if binary else "w")
            if binary:
                lamf.write(lambda_log_header())

    def flush(upto):
        if traj is not None:
            steps, crd, ene = eng.take_frames(0)
            for st, c, e in zip(steps, crd, ene):
                if st <= upto:
                    ed = dict(zip(engine.ENERGY_NAMES, e))
                    if params.get("format_o_crd", "presto") == "gromacs":
                        traj.write(gromacs_frame(st, st * dt, box, c))
                    else:
                        traj.write(presto_frame(st, st * dt, ed, c))
        if vm:
            st, vs = eng.take_vs_log(0)
            if vsf is not None:
                vsf.writelines("%d\t%d\n" % (a, b + 1) for a, b in zip(st, vs) if a <= upto)
            st, lam = eng.take_lambda_log(0)
            if lamf is not None:
                for a, x in zip(st, lam):
                    if a <= upto:
                        lamf.write(struct.pack("<d", x) if "b" in lamf.mode else "%14.10e\n" % x)

    def write_log(k):
        if log is not None:
            log.write(log_block(k, k * dt, eng.get_energies(0), extended=vm))

    done = 0
    stops = sorted({k + 1 for k in range(n) if (ri > 0 and k % ri == 0) or (li > 0 and k % li == 0)
                    or k == 0 or k == n - 1} | {n})
    for stop in stops:
        if stop > done:
            eng.step(stop - done)
            done = stop
        k = done - 1  # the step just computed
        if k < n and ((li > 0 and k % li == 0) or k == 0 or k == n - 1):
            write_log(k)
        if ri > 0 and k < n and k % ri == 0 and params.get("fn_o_restart"):
            _restart(eng, params["fn_o_restart"], k, k * dt)
    flush(n)
    if params.get("fn_o_restart"):
        _restart(eng, params["fn_o_restart"], n, n * dt)
    eng.step(1)  # the loop's last step (DynamicsMode.cpp:205-211)
    write_log(n)
    flush(n)
    ene = eng.get_energies(0)
    for f in (traj, vsf, lamf):
        if f is not None:
            f.close()
    eng.close()
    return ene


def _restart(eng, path, n_steps, time):
    crd, vel = eng.get_state(0)
    e = eng.get_energies(0)
    write_restart(path, n_steps, time, e["potential"], e["kinetic"], crd, vel)
