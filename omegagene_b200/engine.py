"""Python host mirror of the engine's C ABI (include/omegagene_b200.h).

The compute path is the CUDA library ``libomegagene_b200.so`` built in-tree for sm_100a; this
module only marshals arrays.  There is no fallback: loading fails loudly when the library is
missing or no CUDA device is present.

The run parameters use the reference's config keys (src/celeste/core/Config.cpp:37-367), so a
``.cls`` launch set plus an ``md.inp.run``-style option list describes a system exactly as it
does for ``omegagene --cfg md.inp.run --inp md.inp.cls``.
"""
import ctypes as C
import os

import numpy as np

from . import cls_io

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libomegagene_b200.so")

(OG_OK, OG_ERR_INVALID, OG_ERR_CUDA, OG_ERR_CAPACITY, OG_ERR_STATE, OG_ERR_NOMEM, OG_ERR_NOT_CONVERGED,
 OG_ERR_SYSTEM_FAULT) = range(8)
ENERGY_NAMES = ["vdw", "ele", "bond", "angle", "potential", "kinetic", "temperature", "total", "ele_excess",
                "ele_self", "mcmd_factor", "torsion", "improper", "vdw14", "ele14"]
N_ENERGY = len(ENERGY_NAMES)
N_PAIR_VARIANTS = 11  # OG_N_PAIR_VARIANTS
PAIR_VARIANT_F64 = 11  # OG_PAIR_VARIANT_F64: FP64 validation evaluation, chosen only by set_tuning


class OgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("og status %d: %s" % (status, msg))
        self.status = status


_p = C.POINTER


class SystemDesc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("pbc_val", C.c_double * 12),
        ("crd", _p(C.c_double)), ("vel", _p(C.c_double)), ("charge", _p(C.c_double)), ("mass", _p(C.c_double)),
        ("atom_type", _p(C.c_int32)), ("n_lj_types", C.c_int32), ("lj6", _p(C.c_double)), ("lj12", _p(C.c_double)),
        ("n_excl", C.c_int32), ("excl", _p(C.c_int32)),
        ("n_shake_pair", C.c_int32), ("shake_pair", _p(C.c_int32)), ("shake_pair_dist", _p(C.c_double)),
        ("n_shake_trio", C.c_int32), ("shake_trio", _p(C.c_int32)), ("shake_trio_dist", _p(C.c_double)),
        ("n_bonds", C.c_int32), ("bond", _p(C.c_int32)), ("bond_k", _p(C.c_double)), ("bond_r0", _p(C.c_double)),
        ("n_angles", C.c_int32), ("angle", _p(C.c_int32)), ("angle_k", _p(C.c_double)), ("angle_t0", _p(C.c_double)),
        ("n_com_groups", C.c_int32), ("com_group_start", _p(C.c_int32)), ("com_group_atoms", _p(C.c_int32)),
        ("cutoff", C.c_double), ("nsgrid_cutoff", C.c_double), ("nsgrid_update_intvl", C.c_int32),
        ("time_step", C.c_double), ("thermostat", C.c_int32), ("temperature", C.c_double),
        ("temperature_init", C.c_double), ("heating_steps", C.c_int32), ("berendsen_tau", C.c_double),
        ("const_max_loops", C.c_int32), ("const_tolerance", C.c_double),
        ("thermo_const_max_loops", C.c_int32), ("thermo_const_tolerance", C.c_double),
        ("mcmd_order", C.c_int32), ("mcmd_lambda_low", C.c_double), ("mcmd_lambda_high", C.c_double),
        ("mcmd_temperature", C.c_double), ("mcmd_coef", _p(C.c_double)),
        ("first_step", C.c_int64),
        ("n_torsions", C.c_int32), ("torsion", _p(C.c_int32)), ("torsion_ene", _p(C.c_double)),
        ("torsion_phase", _p(C.c_double)), ("torsion_overlaps", _p(C.c_int32)), ("torsion_symmetry", _p(C.c_int32)),
        ("n_impros", C.c_int32), ("impro", _p(C.c_int32)), ("impro_ene", _p(C.c_double)),
        ("impro_phase", _p(C.c_double)), ("impro_overlaps", _p(C.c_int32)), ("impro_symmetry", _p(C.c_int32)),
        ("n_nb14", C.c_int32), ("nb14", _p(C.c_int32)), ("nb14_type", _p(C.c_int32)),
        ("nb14_coeff_vdw", _p(C.c_double)), ("nb14_coeff_ele", _p(C.c_double)),
        ("n_shake_quad", C.c_int32), ("shake_quad", _p(C.c_int32)), ("shake_quad_dist", _p(C.c_double)),
        ("dof_extra", C.c_int32),
        ("n_vstates", C.c_int32), ("vmcmd_trans_interval", C.c_int32), ("vmcmd_init_vs", C.c_int32),
        ("vmcmd_lambda_log_interval", C.c_int32), ("vmcmd_seed", C.c_uint32),
        ("vs_order", _p(C.c_int32)), ("vs_lambda", _p(C.c_double)), ("vs_prob", _p(C.c_double)),
        ("vs_coef", _p(C.c_double)), ("vmcmd_mt_state", _p(C.c_uint32)),
        ("ele_mode", C.c_int32), ("ele_alpha", C.c_double), ("dh_dielectric", C.c_double),
        ("dh_ionic_strength", C.c_double), ("dh_temperature", C.c_double), ("hps", C.c_int32),
        ("hps_epsilon", C.c_double), ("lj_hps_cutoff", _p(C.c_double)), ("lj_hps_lambda", _p(C.c_double)),
    ]

OG_MT_WORDS = 625


_lib = None


def load_library():
    """Loads the in-tree CUDA library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OgError(OG_ERR_STATE, "%s is missing: run `python -c 'import __graft_entry__ as g; g.build()'`"
                      % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    E = C.c_void_p
    sig = {
        "og_create": [C.c_int, _p(E)], "og_destroy": [E], "og_add_system": [E, _p(SystemDesc), _p(C.c_int32)],
        "og_finalize": [E], "og_step": [E, C.c_int32], "og_compute_forces": [E],
        "og_set_state": [E, C.c_int32, C.c_void_p, C.c_void_p], "og_get_state": [E, C.c_int32, C.c_void_p, C.c_void_p],
        "og_get_forces": [E, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
        "og_get_energies": [E, C.c_int32, C.c_void_p],
        "og_get_grid_info": [E, C.c_int32, _p(C.c_int32), _p(C.c_int32), _p(C.c_int32)],
        "og_get_grid": [E, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
        "og_get_cell_pairs": [E, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "og_set_trace": [E, C.c_int32], "og_get_trace": [E, C.c_void_p, C.c_int32, _p(C.c_int32)],
        "og_get_stats": [E, _p(C.c_int64), _p(C.c_double), _p(C.c_double)],
        "og_get_sizes": [E, _p(C.c_int32), _p(C.c_int64)], "og_set_timing": [E, C.c_int32],
        "og_get_flags": [E, _p(C.c_int32)], "og_put_state": [E, C.c_int32, C.c_void_p, C.c_void_p],
        "og_get_state_async": [E, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
        "og_step_async": [E, C.c_int32], "og_synchronize": [E],
        "og_get_pair_count": [E, C.c_int32, _p(C.c_int64)],
        "og_get_tuning": [E, _p(C.c_int32), C.c_void_p], "og_set_tuning": [E, C.c_int32],
        "og_get_jlist_builds": [E, _p(C.c_int64)], "og_set_list_policy": [E, C.c_int32],
        "og_get_list_builds": [E, _p(C.c_int64)], "og_get_footprint": [E, _p(C.c_int64), _p(C.c_int64)],
        "og_set_graphs": [E, C.c_int32], "og_release_pool_memory": [C.c_int32],
        "og_get_system_faults": [E, C.c_void_p],
        "og_get_graph_info": [E, _p(C.c_int32), _p(C.c_int64), _p(C.c_int64), C.c_char_p],
        "og_get_vmcmd_state": [E, C.c_int32, _p(C.c_int32), C.c_void_p],
        "og_take_vs_log": [E, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, _p(C.c_int64)],
        "og_take_lambda_log": [E, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, _p(C.c_int64)],
        "og_set_trajectory": [E, C.c_int32, C.c_int32, C.c_void_p, C.c_int32],
        "og_take_frames": [E, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, _p(C.c_int32)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.og_last_error.argtypes = [E]
    L.og_last_error.restype = C.c_char_p
    _lib = L
    return L


def _ptr(a, ctype):
    return a.ctypes.data_as(_p(ctype)) if a is not None and a.size else None


DEFAULT_PARAMS = {
    "cutoff": 12.0, "nsgrid_cutoff": 13.0, "nsgrid_update_intvl": 1, "time_step": 2.0, "thermostat": "none",
    "temperature": 300.0, "temperature_init": -1.0, "heating_steps": 0, "berendsen_tau": 0.0,
    "const_max_loops": 1000, "const_tolerance": 1e-7, "thermo_const_max_loops": 100,
    "thermo_const_tolerance": 1e-5, "com_motion": "cancel", "com_cancel_groups": None, "constraint": "shake",
    "extended_ensemble": "none", "random_seed": -1, "print_intvl_extended_lambda": 0,
    "fn_o_vmcmd_log": None, "fn_o_extended_lambda": None, "format_o_extended_lambda": "binary",
    "n_steps": 0, "print_intvl_log": 0, "print_intvl_crd": [], "fn_o_crd": [], "format_o_crd": "presto",
    "group_o_crd": [], "fn_o_restart": "md_o.restart", "print_intvl_restart": 0,
    "electrostatic": "zero-dipole", "ele_alpha": 0.0, "dh_dielectric": 0.0, "dh_ionic_strength": 0.0,
    "dh_temperature": 0.0, "nonbond": "lennard-jones", "hps_epsilon": 0.0,
}

# --electrostatic values (Config.cpp:114-128) and their engine codes
ELECTROSTATIC = {"zero-dipole": 0, "zero-quadrupole": 1, "zero-octupole": 2, "zero-hexadecapole": 3, "debye-huckel": 4}


def parse_run_config(text):
    """Parses the hot-path keys of an ``md.inp.run`` file (Config.cpp:9-35 tokeniser: whitespace
    separated `--key value`, `;` and `#` start comments).  Keys this engine does not implement
    raise ValueError, as unknown keys do in the reference (Config.cpp:359-362)."""
    toks = []
    for line in text.splitlines():
        for c in ";#":
            line = line.split(c)[0]
        toks += line.split()
    p = dict(DEFAULT_PARAMS)
    groups = []
    accepted_ignored = {"--processor", "--gpu-device-id", "--mode", "--fn-o-log", "--fn-o-energy", "--integrator",
                        "--expected-num-density"}
    lists = {"print_intvl_crd": [], "fn_o_crd": [], "group_o_crd": []}
    i = 0
    while i < len(toks):
        k = toks[i]
        v = toks[i + 1] if i + 1 < len(toks) else None
        i += 2
        if k == "--cutoff":
            p["cutoff"] = float(v)
        elif k == "--nsgrid-cutoff":
            p["nsgrid_cutoff"] = float(v)
        elif k == "--nsgrid-update-intvl":
            p["nsgrid_update_intvl"] = int(v)
        elif k == "--time-step":
            p["time_step"] = float(v)
        elif k == "--thermostat":
            p["thermostat"] = v
        elif k == "--temperature":
            p["temperature"] = float(v)
        elif k == "--temperature-init":
            p["temperature_init"] = float(v)
        elif k == "--heating-steps":
            p["heating_steps"] = int(v)
        elif k == "--berendsen-tau":
            p["berendsen_tau"] = float(v) * 1000.0  # Config.cpp:162-164
        elif k == "--const-max-loops":
            p["const_max_loops"] = int(v)
        elif k == "--const-tolerance":
            p["const_tolerance"] = float(v)
        elif k == "--thermo-const-max-loops":
            p["thermo_const_max_loops"] = int(v)
        elif k == "--thermo-const-tolerance":
            p["thermo_const_tolerance"] = float(v)
        elif k == "--com-motion":
            p["com_motion"] = v
        elif k == "--com-cancel-group-name":
            groups.append(v)
        elif k == "--constraint":
            p["constraint"] = v
        elif k == "--electrostatic":
            if v not in ELECTROSTATIC:
                raise ValueError("--electrostatic %s (%s)" % (v, ", ".join(ELECTROSTATIC)))
            p["electrostatic"] = v
        elif k == "--ele-alpha":
            p["ele_alpha"] = float(v)
        elif k == "--debye-huckel-dielectric":
            p["dh_dielectric"] = float(v)
        elif k == "--debye-huckel-ionic-strength":
            p["dh_ionic_strength"] = float(v)
        elif k == "--debye-huckel-temperature":
            p["dh_temperature"] = float(v)
        elif k == "--nonbond":   # Config.cpp:334-339
            if v not in ("lennard-jones", "hydrophobicity-scale-lj"):
                raise ValueError("--nonbond %s (lennard-jones, hydrophobicity-scale-lj)" % v)
            p["nonbond"] = v
        elif k == "--hydrophobicity-scale-epsiron":
            p["hps_epsilon"] = float(v)
        elif k == "--extended-ensemble":
            # Config.cpp:145-157; V-AUS and VcMD are not on this path
            if v not in ("none", "v-mcmd"):
                raise ValueError("--extended-ensemble %s is not on the hot path (none, v-mcmd)" % v)
            p["extended_ensemble"] = v
        elif k == "--random-seed":
            p["random_seed"] = int(v)
        elif k == "--n-steps":
            p["n_steps"] = int(v)
        elif k == "--print-interval-log":
            p["print_intvl_log"] = int(v)
        elif k == "--print-interval-coord":   # Config.cpp:204-205, one entry per output
            lists["print_intvl_crd"].append(int(v))
        elif k == "--fn-o-coord":
            lists["fn_o_crd"].append(v)
        elif k == "--group-o-coord":
            lists["group_o_crd"].append(v)
        elif k == "--format-o-coord":
            if v not in ("presto", "gromacs"):
                raise ValueError("--format-o-coord %s (presto, gromacs)" % v)
            p["format_o_crd"] = v
        elif k == "--fn-o-restart":
            p["fn_o_restart"] = v
        elif k == "--print-interval-restart":
            p["print_intvl_restart"] = int(v)
        elif k == "--print-interval-extended-lambda":
            p["print_intvl_extended_lambda"] = int(v)
        elif k == "--fn-o-vmcmd-log":
            p["fn_o_vmcmd_log"] = v
        elif k == "--fn-o-extended-lambda":
            p["fn_o_extended_lambda"] = v
        elif k == "--format-o-extended-lambda":
            p["format_o_extended_lambda"] = v
        elif k in accepted_ignored:
            if k == "--integrator" and v != "leapfrog-presto":
                raise ValueError("only --integrator leapfrog-presto is on the hot path")
        else:
            raise ValueError("unsupported config key %s" % k)
    if groups:
        p["com_cancel_groups"] = groups
    for key, val in lists.items():
        if val:
            p[key] = val
    return p


class _Keep:
    """Holds the numpy arrays a SystemDesc points into."""


def make_desc(system, params=None, mcmd=None, first_step=0):
    """Builds an og_system_desc from a launch-set dict (cls_io.read_cls or systems.*)."""
    prm = dict(DEFAULT_PARAMS)
    prm.update(params or {})
    keep = _Keep()
    t = system["topol"]
    n = int(system["n_atoms"])
    keep.crd = np.ascontiguousarray(system["crd"], np.float64).reshape(-1)
    keep.vel = np.ascontiguousarray(system.get("vel", np.zeros((n, 3))), np.float64).reshape(-1)
    keep.charge = np.ascontiguousarray(t["charge"], np.float64)
    keep.mass = np.ascontiguousarray(t["mass"], np.float64)
    keep.type = np.ascontiguousarray(t["atom_type"], np.int32)
    c6, c12 = cls_io.lj_tables(t)
    keep.lj6 = np.ascontiguousarray(c6.reshape(-1))
    keep.lj12 = np.ascontiguousarray(c12.reshape(-1))
    keep.excl = np.ascontiguousarray(np.asarray(t["nb15off_pairs"], np.int32).reshape(-1))
    d = SystemDesc()
    d.n_atoms = n
    for i in range(12):
        d.pbc_val[i] = float(system["pbc_val"][i])
    d.crd, d.vel = _ptr(keep.crd, C.c_double), _ptr(keep.vel, C.c_double)
    d.charge, d.mass = _ptr(keep.charge, C.c_double), _ptr(keep.mass, C.c_double)
    d.atom_type = _ptr(keep.type, C.c_int32)
    d.n_lj_types = int(t["n_lj_types"])
    d.lj6, d.lj12 = _ptr(keep.lj6, C.c_double), _ptr(keep.lj12, C.c_double)
    d.n_excl = len(keep.excl) // 2
    d.excl = _ptr(keep.excl, C.c_int32)
    cons = system.get("constraint") if prm["constraint"] in ("shake", "shake-settle", "settle") else None
    if cons is not None:
        keep.sp = np.ascontiguousarray(np.asarray(cons["pair_atoms"], np.int32).reshape(-1))
        keep.spd = np.ascontiguousarray(np.asarray(cons["pair_dist"], np.float64).reshape(-1))
        keep.st = np.ascontiguousarray(np.asarray(cons["trio_atoms"], np.int32).reshape(-1))
        keep.std = np.ascontiguousarray(np.asarray(cons["trio_dist"], np.float64).reshape(-1))
        qa = np.asarray(cons.get("quad_atoms", np.zeros((0, 4))), np.int32).reshape(-1)
        if len(qa):
            keep.qa = np.ascontiguousarray(qa)
            keep.qd = np.ascontiguousarray(np.asarray(cons["quad_dist"], np.float64).reshape(-1))
            d.n_shake_quad, d.shake_quad, d.shake_quad_dist = len(qa) // 4, _ptr(keep.qa, C.c_int32), _ptr(keep.qd, C.c_double)
        d.n_shake_pair, d.shake_pair, d.shake_pair_dist = len(keep.spd), _ptr(keep.sp, C.c_int32), _ptr(keep.spd, C.c_double)
        d.n_shake_trio, d.shake_trio, d.shake_trio_dist = len(keep.st) // 3, _ptr(keep.st, C.c_int32), _ptr(keep.std, C.c_double)
    b = t.get("bonds")
    if b is not None and len(b):
        keep.bond = np.ascontiguousarray(np.stack([b["a1"], b["a2"]], 1).astype(np.int32).reshape(-1))
        keep.bk, keep.br0 = np.ascontiguousarray(b["k"], np.float64), np.ascontiguousarray(b["r0"], np.float64)
        d.n_bonds, d.bond, d.bond_k, d.bond_r0 = len(b), _ptr(keep.bond, C.c_int32), _ptr(keep.bk, C.c_double), _ptr(keep.br0, C.c_double)
    a = t.get("angles")
    if a is not None and len(a):
        keep.angle = np.ascontiguousarray(np.stack([a["a1"], a["a2"], a["a3"]], 1).astype(np.int32).reshape(-1))
        keep.ak, keep.at0 = np.ascontiguousarray(a["k"], np.float64), np.ascontiguousarray(a["t0"], np.float64)
        d.n_angles, d.angle, d.angle_k, d.angle_t0 = len(a), _ptr(keep.angle, C.c_int32), _ptr(keep.ak, C.c_double), _ptr(keep.at0, C.c_double)
    if prm["com_motion"] == "cancel" and "groups" in system:
        names = prm["com_cancel_groups"] or system["groups"]["names"]
        lists = [np.asarray(system["groups"]["atoms"][system["groups"]["names"].index(nm)], np.int32) for nm in names]
        keep.gstart = np.ascontiguousarray(np.concatenate([[0], np.cumsum([len(x) for x in lists])]).astype(np.int32))
        keep.gatoms = np.ascontiguousarray(np.concatenate(lists).astype(np.int32))
        d.n_com_groups, d.com_group_start, d.com_group_atoms = len(lists), _ptr(keep.gstart, C.c_int32), _ptr(keep.gatoms, C.c_int32)
    d.cutoff, d.nsgrid_cutoff = prm["cutoff"], prm["nsgrid_cutoff"]
    d.nsgrid_update_intvl, d.time_step = prm["nsgrid_update_intvl"], prm["time_step"]
    d.thermostat = 1 if prm["thermostat"] == "scaling" else 0
    d.temperature, d.temperature_init = prm["temperature"], prm["temperature_init"]
    d.heating_steps, d.berendsen_tau = prm["heating_steps"], prm["berendsen_tau"]
    d.const_max_loops, d.const_tolerance = prm["const_max_loops"], prm["const_tolerance"]
    d.thermo_const_max_loops, d.thermo_const_tolerance = prm["thermo_const_max_loops"], prm["thermo_const_tolerance"]
    for key, pre in (("torsions", "torsion"), ("impros", "impro")):
        recs = t.get(key)
        if recs is not None and len(recs):
            arrs = (np.ascontiguousarray(recs["a"], np.int32).reshape(-1), np.ascontiguousarray(recs["ene"], np.float64),
                    np.ascontiguousarray(recs["phase"], np.float64), np.ascontiguousarray(recs["overlaps"], np.int32),
                    np.ascontiguousarray(recs["symmetry"], np.int32))
            setattr(keep, key, arrs)
            setattr(d, "n_" + ("torsions" if pre == "torsion" else "impros"), len(recs))
            setattr(d, pre, _ptr(arrs[0], C.c_int32))
            setattr(d, pre + "_ene", _ptr(arrs[1], C.c_double))
            setattr(d, pre + "_phase", _ptr(arrs[2], C.c_double))
            setattr(d, pre + "_overlaps", _ptr(arrs[3], C.c_int32))
            setattr(d, pre + "_symmetry", _ptr(arrs[4], C.c_int32))
    n14 = t.get("nb14")
    if n14 is not None and len(n14["atoms"]):
        keep.n14 = (np.ascontiguousarray(n14["atoms"], np.int32).reshape(-1),
                    np.ascontiguousarray(n14["types"], np.int32).reshape(-1),
                    np.ascontiguousarray(n14["coeff_vdw"], np.float64), np.ascontiguousarray(n14["coeff_ele"], np.float64))
        d.n_nb14 = len(keep.n14[2])
        d.nb14, d.nb14_type = _ptr(keep.n14[0], C.c_int32), _ptr(keep.n14[1], C.c_int32)
        d.nb14_coeff_vdw, d.nb14_coeff_ele = _ptr(keep.n14[2], C.c_double), _ptr(keep.n14[3], C.c_double)
    d.dof_extra = int(system.get("dof_extra", 0))
    d.first_step = int(first_step)
    # electrostatics / nonbond model (ForceField.cpp:30-100)
    d.ele_mode = ELECTROSTATIC[prm.get("electrostatic", "zero-dipole")]
    d.ele_alpha = float(prm.get("ele_alpha", 0.0))
    d.dh_dielectric, d.dh_ionic_strength = float(prm.get("dh_dielectric", 0.0)), float(prm.get("dh_ionic_strength", 0.0))
    d.dh_temperature = float(prm.get("dh_temperature", 0.0))
    if prm.get("nonbond", "lennard-jones") == "hydrophobicity-scale-lj":
        cut, lam = cls_io.hps_tables(t)
        keep.hcut, keep.hlam = np.ascontiguousarray(cut.reshape(-1)), np.ascontiguousarray(lam.reshape(-1))
        d.hps, d.hps_epsilon = 1, float(prm.get("hps_epsilon", 0.0))
        d.lj_hps_cutoff, d.lj_hps_lambda = _ptr(keep.hcut, C.c_double), _ptr(keep.hlam, C.c_double)
    d.mcmd_order = -1
    if mcmd is not None and "states" in mcmd:
        _vmcmd_desc(d, keep, mcmd, prm)
    elif mcmd is not None:
        keep.mcoef = np.ascontiguousarray(mcmd["coef"], np.float64)
        d.mcmd_order = len(keep.mcoef) - 1
        d.mcmd_lambda_low, d.mcmd_lambda_high = mcmd["lambda_low"], mcmd["lambda_high"]
        d.mcmd_temperature = mcmd["temperature"]
        d.mcmd_coef = _ptr(keep.mcoef, C.c_double)
    return d, keep


def vmcmd_seed(params):
    """The generator seed of a V-McMD run: --random-seed, or, when it is negative, a fresh one
    from the OS (the reference seeds from std::random_device then, DynamicsMode.cpp:79-84)."""
    seed = int(params.get("random_seed", -1))
    if seed < 0:
        seed = int.from_bytes(os.urandom(4), "little") & 0x7FFFFFFF
    return seed & 0xFFFFFFFF


def _vmcmd_desc(d, keep, v, prm):
    """Fills the V-McMD fields from the .cls section dict (cls_io: states, interval, temperature,
    init_vs 1-based as in the file).  Optional keys: cur_vs (0-based) and mt_state, a run's state
    handed over from another engine (Engine.vmcmd_state)."""
    st = v["states"]
    keep.vs_order = np.ascontiguousarray([len(x["coef"]) - 1 for x in st], np.int32)
    keep.vs_lambda = np.ascontiguousarray([[x["lambda_low"], x["lambda_high"]] for x in st], np.float64).reshape(-1)
    keep.vs_prob = np.ascontiguousarray([[x["prob_low"], x["prob_high"]] for x in st], np.float64).reshape(-1)
    keep.vs_coef = np.ascontiguousarray(np.concatenate([np.asarray(x["coef"], np.float64) for x in st]))
    d.n_vstates = len(st)
    d.vmcmd_trans_interval = int(v["interval"])
    d.vmcmd_init_vs = int(v["cur_vs"]) if "cur_vs" in v else int(v["init_vs"]) - 1
    d.vmcmd_lambda_log_interval = int(prm.get("print_intvl_extended_lambda", 0) or 0)
    d.vmcmd_seed = vmcmd_seed(prm)
    d.mcmd_temperature = float(v["temperature"])
    d.vs_order, d.vs_lambda = _ptr(keep.vs_order, C.c_int32), _ptr(keep.vs_lambda, C.c_double)
    d.vs_prob, d.vs_coef = _ptr(keep.vs_prob, C.c_double), _ptr(keep.vs_coef, C.c_double)
    if v.get("mt_state") is not None:
        keep.mt = np.ascontiguousarray(v["mt_state"], np.uint32)
        if keep.mt.shape != (OG_MT_WORDS,):
            raise ValueError("mt_state needs %d words" % OG_MT_WORDS)
        d.vmcmd_mt_state = _ptr(keep.mt, C.c_uint32)


def release_pool_memory(device=0):
    """Returns the device memory that destroyed engines left in the per-device pool."""
    st = load_library().og_release_pool_memory(int(device))
    if st != OG_OK:
        raise OgError(st, "og_release_pool_memory")


class Engine:
    """One engine = one CUDA context user holding a batch of independent systems."""

    def __init__(self, device=0):
        self.L = load_library()
        self.h = C.c_void_p()
        self._check(self.L.og_create(int(device), C.byref(self.h)), "og_create")
        self.n_atoms = []
        self._keep = []

    def _check(self, status, what=""):
        if status != OG_OK:
            msg = self.L.og_last_error(self.h).decode() if self.h else ""
            raise OgError(status, "%s: %s" % (what, msg))

    def close(self):
        if self.h:
            self.L.og_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_system(self, system, params=None, mcmd=None, first_step=0):
        d, keep = make_desc(system, params, mcmd, first_step)
        sid = C.c_int32()
        self._check(self.L.og_add_system(self.h, C.byref(d), C.byref(sid)), "og_add_system")
        self._keep.append(keep)
        self.n_atoms.append(int(system["n_atoms"]))
        return sid.value

    def finalize(self):
        self._check(self.L.og_finalize(self.h), "og_finalize")
        self._keep = []

    def step(self, n=1):
        self._check(self.L.og_step(self.h, int(n)), "og_step")

    def compute_forces(self):
        self._check(self.L.og_compute_forces(self.h), "og_compute_forces")

    def set_state(self, sys, crd=None, vel_next=None):
        c = None if crd is None else np.ascontiguousarray(crd, np.float64).reshape(-1)
        v = None if vel_next is None else np.ascontiguousarray(vel_next, np.float64).reshape(-1)
        self._check(self.L.og_set_state(self.h, sys, c.ctypes.data if c is not None else None,
                                        v.ctypes.data if v is not None else None), "og_set_state")

    def get_state(self, sys):
        n = self.n_atoms[sys]
        crd, vel = np.zeros((n, 3)), np.zeros((n, 3))
        self._check(self.L.og_get_state(self.h, sys, crd.ctypes.data, vel.ctypes.data), "og_get_state")
        return crd, vel

    def get_forces(self, sys):
        n = self.n_atoms[sys]
        work, ene, vir = np.zeros((n, 3)), np.zeros(N_ENERGY), np.zeros(9)
        self._check(self.L.og_get_forces(self.h, sys, work.ctypes.data, ene.ctypes.data, vir.ctypes.data),
                    "og_get_forces")
        return work, dict(zip(ENERGY_NAMES, ene)), vir.reshape(3, 3)

    def get_energies(self, sys):
        ene = np.zeros(N_ENERGY)
        self._check(self.L.og_get_energies(self.h, sys, ene.ctypes.data), "og_get_energies")
        return dict(zip(ENERGY_NAMES, ene))

    def grid_info(self, sys):
        nc, ncol, npair = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.L.og_get_grid_info(self.h, sys, C.byref(nc), C.byref(ncol), C.byref(npair)), "grid_info")
        return nc.value, ncol.value, npair.value

    def get_grid(self, sys):
        nc, ncol, _ = self.grid_info(sys)
        sa = np.zeros(8 * nc, np.int32)
        sc = np.zeros((8 * nc, 3))
        ch = np.zeros(ncol + 1, np.int32)
        self._check(self.L.og_get_grid(self.h, sys, sa.ctypes.data, sc.ctypes.data, ch.ctypes.data), "og_get_grid")
        return {"n_cells": nc, "slot_atomid": sa, "slot_crd": sc, "col_head_cell": ch}

    def get_cell_pairs(self, sys):
        nc, _, npair = self.grid_info(sys)
        head = np.zeros(nc + 1, np.int32)
        c1, c2, img = (np.zeros(npair, np.int32) for _ in range(3))
        mask = np.zeros(npair, np.uint64)
        self._check(self.L.og_get_cell_pairs(self.h, sys, head.ctypes.data, c1.ctypes.data, c2.ctypes.data,
                                             img.ctypes.data, mask.ctypes.data), "og_get_cell_pairs")
        return {"idx_head": head, "cell1": c1, "cell2": c2, "image": img, "mask": mask, "n_pairs": npair}

    def set_trace(self, capacity):
        self._check(self.L.og_set_trace(self.h, int(capacity)), "og_set_trace")

    def get_trace(self, max_steps):
        n_sys = len(self.n_atoms)
        out = np.zeros((max_steps, n_sys, N_ENERGY))
        n = C.c_int32()
        self._check(self.L.og_get_trace(self.h, out.ctypes.data, int(max_steps), C.byref(n)), "og_get_trace")
        return out[:n.value]

    def set_timing(self, on=True):
        """on=True: per-pair-kernel and per-call events (kernel-by-kernel steps); "step": per-call
        events only (graph replays stay on); False: off."""
        mode = 2 if on == "step" else (1 if on else 0)
        self._check(self.L.og_set_timing(self.h, mode), "og_set_timing")

    def stats(self):
        k, p, s = C.c_int64(), C.c_double(), C.c_double()
        self._check(self.L.og_get_stats(self.h, C.byref(k), C.byref(p), C.byref(s)), "og_get_stats")
        return {"kernel_launches": k.value, "pair_kernel_ms": p.value, "step_ms": s.value}

    def set_list_policy(self, policy):
        """Cell-pair list schedule before finalize(): "fixed" (the reference's, every
        nsgrid_update_intvl steps) or "displacement" (rebuilt whenever an atom has moved half the
        list margin since the last build; exact lists)."""
        code = {"fixed": 0, "displacement": 1}[policy]
        self._check(self.L.og_set_list_policy(self.h, code), "og_set_list_policy")

    def footprint(self):
        """(device bytes held now, most held at once) by this engine."""
        held, peak = C.c_int64(), C.c_int64()
        self._check(self.L.og_get_footprint(self.h, C.byref(held), C.byref(peak)), "og_get_footprint")
        return held.value, peak.value

    def list_builds(self):
        n = C.c_int64()
        self._check(self.L.og_get_list_builds(self.h, C.byref(n)), "og_get_list_builds")
        return n.value

    def jlist_builds(self):
        """Pair variant 10: j-list builds since finalize (list builds plus skin rebuilds)."""
        n = C.c_int64()
        self._check(self.L.og_get_jlist_builds(self.h, C.byref(n)), "og_get_jlist_builds")
        return n.value

    def flags(self):
        f = C.c_int32()
        self._check(self.L.og_get_flags(self.h, C.byref(f)), "og_get_flags")
        return f.value

    # ---- stream-ordered calls for callers that keep state in (pinned) host memory
    def put_state_ptr(self, sys, crd_ptr, vel_ptr):
        self._check(self.L.og_put_state(self.h, sys, crd_ptr, vel_ptr), "og_put_state")

    def get_state_async_ptr(self, sys, crd_ptr, vel_ptr, ene_ptr):
        self._check(self.L.og_get_state_async(self.h, sys, crd_ptr, vel_ptr, ene_ptr), "og_get_state_async")

    def step_async(self, n=1):
        self._check(self.L.og_step_async(self.h, int(n)), "og_step_async")

    def synchronize(self):
        self._check(self.L.og_synchronize(self.h), "og_synchronize")

    def pair_count(self, sys):
        """Interacting pairs (r < cutoff, not excluded) of the last og_compute_forces."""
        n = C.c_int64()
        self._check(self.L.og_get_pair_count(self.h, sys, C.byref(n)), "og_get_pair_count")
        return n.value

    def tuning(self):
        v = C.c_int32()
        ms = np.zeros(N_PAIR_VARIANTS)
        self._check(self.L.og_get_tuning(self.h, C.byref(v), ms.ctypes.data), "og_get_tuning")
        return {"pair_variant": v.value, "variant_ms": ms.tolist()}

    def set_tuning(self, variant):
        """Fixes the pair-kernel variant (0..N_PAIR_VARIANTS-1, or PAIR_VARIANT_F64 for the FP64
        validation evaluation) before finalize(); -1 = autotune."""
        self._check(self.L.og_set_tuning(self.h, int(variant)), "og_set_tuning")

    def set_graphs(self, on=True):
        self._check(self.L.og_set_graphs(self.h, 1 if on else 0), "og_set_graphs")

    def graph_info(self):
        en, rep, k = C.c_int32(), C.c_int64(), C.c_int64()
        note = C.create_string_buffer(256)
        self._check(self.L.og_get_graph_info(self.h, C.byref(en), C.byref(rep), C.byref(k), note), "og_get_graph_info")
        return {"enabled": bool(en.value), "replays": rep.value, "kernels_per_replay": k.value,
                "note": note.value.decode()}

    def vmcmd_state(self, sys):
        """(current 0-based virtual state, generator words [625] or None for a one-state system)."""
        cur = C.c_int32()
        mt = np.zeros(OG_MT_WORDS, np.uint32)
        st = self.L.og_get_vmcmd_state(self.h, sys, C.byref(cur), mt.ctypes.data)
        if st == OG_ERR_INVALID:
            self._check(self.L.og_get_vmcmd_state(self.h, sys, C.byref(cur), None), "og_get_vmcmd_state")
            return cur.value, None
        self._check(st, "og_get_vmcmd_state")
        return cur.value, mt

    def _take(self, fn, sys, dtype):
        n = C.c_int64()
        self._check(fn(self.h, sys, 0, None, None, C.byref(n)), "V-McMD log")
        steps, vals = np.zeros(n.value, np.int64), np.zeros(n.value, dtype)
        if n.value:
            self._check(fn(self.h, sys, n.value, steps.ctypes.data, vals.ctypes.data, C.byref(n)), "V-McMD log")
        return steps[:n.value], vals[:n.value]

    def take_vs_log(self, sys):
        """(steps, 0-based virtual states) logged since the last take (WriteTTPVMcMDLog lines)."""
        return self._take(self.L.og_take_vs_log, sys, np.int32)

    def take_lambda_log(self, sys):
        """(steps, lambda) logged since the last take (ExtendedVMcMD::write_lambda rows)."""
        return self._take(self.L.og_take_lambda_log, sys, np.float64)

    def set_trajectory(self, sys, interval, group=None):
        """Frames every `interval` steps of the group's atoms (None: all), recorded on the device;
        call before finalize."""
        g = None if group is None else np.ascontiguousarray(group, np.int32)
        self._check(self.L.og_set_trajectory(self.h, sys, int(interval), None if g is None else g.ctypes.data,
                                             0 if g is None else len(g)), "og_set_trajectory")
        self._tr_n = getattr(self, "_tr_n", {})
        self._tr_n[sys] = len(g) if g is not None else None

    def take_frames(self, sys):
        """(steps, crd [frames][group][3] float32, energies [frames][N_ENERGY]) not yet taken."""
        n = C.c_int32()
        self._check(self.L.og_take_frames(self.h, sys, 0, None, None, None, C.byref(n)), "og_take_frames")
        g = self._tr_n.get(sys) or self.n_atoms[sys]
        steps = np.zeros(n.value, np.int64)
        crd = np.zeros((n.value, g, 3), np.float32)
        ene = np.zeros((n.value, N_ENERGY), np.float64)
        if n.value:
            self._check(self.L.og_take_frames(self.h, sys, n.value, steps.ctypes.data, crd.ctypes.data,
                                              ene.ctypes.data, C.byref(n)), "og_take_frames")
        return steps[:n.value], crd[:n.value], ene[:n.value]

    def system_faults(self):
        """Per-system fault bits of the last og_step that returned OG_ERR_SYSTEM_FAULT
        (4 = bad coordinate, 32 = one-step displacement beyond the list margin, 2 = column over
        capacity); all zero otherwise."""
        f = np.zeros(len(self.n_atoms), np.int32)
        self._check(self.L.og_get_system_faults(self.h, f.ctypes.data), "og_get_system_faults")
        return f
