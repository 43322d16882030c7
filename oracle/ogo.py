"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE; imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU legs).

``OracleSystem`` drives the C restatement (libogo.so) through the reference's per-step
sequence (DynamicsModePresto::calc_in_each_step, src/celeste/core/DynamicsMode.cpp:468-560).
``ref_minicell`` runs the reference's own MiniCell.cpp (oracle/_ref/libogref_minicell.so).
"""
import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_NB15OFF = 32

i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


class Pbc(C.Structure):
    _fields_ = [(k, C.c_float * 3) for k in ("L", "L_half", "L_inv", "L_half_inv", "lower", "upper")]


class Hps(C.Structure):
    _fields_ = [("on", C.c_int), ("eps", C.c_float), ("cut", C.POINTER(C.c_float)), ("lam", C.POINTER(C.c_float))]


class Hps64(C.Structure):
    _fields_ = [("on", C.c_int), ("eps", C.c_double), ("cut", C.POINTER(C.c_double)), ("lam", C.POINTER(C.c_double))]


class EleModel:
    """The electrostatics / nonbond model of a run (ogo_ele_init; engine.ELECTROSTATIC codes):
    float coefficients for the FP32 restatement, double ones for the FP64 oracle, HPS tables."""

    def __init__(self, params, topol):
        from omegagene_b200 import cls_io, engine
        self.mode = engine.ELECTROSTATIC[params.get("electrostatic", "zero-dipole")]
        self.alpha = float(params.get("ele_alpha", 0.0))
        self.hps_on = params.get("nonbond", "lennard-jones") == "hydrophobicity-scale-lj"
        self.default = self.mode == 0 and self.alpha < 1e-10 and not self.hps_on
        L = lib()
        dh = (float(params.get("dh_dielectric", 0.0)), float(params.get("dh_ionic_strength", 0.0)),
              float(params.get("dh_temperature", 0.0)))
        self.m32 = C.create_string_buffer(512)
        self.m64 = C.create_string_buffer(512)
        L.ogo_ele_init(self.m32, self.mode, self.alpha, float(params["cutoff"]), *dh)
        L.ogo_ele_init64(self.m64, self.mode, self.alpha, float(params["cutoff"]), *dh)
        cut, lam = cls_io.hps_tables(topol)
        self.cut64, self.lam64 = np.ascontiguousarray(cut.reshape(-1)), np.ascontiguousarray(lam.reshape(-1))
        self.cut32, self.lam32 = self.cut64.astype(np.float32), self.lam64.astype(np.float32)
        eps = float(params.get("hps_epsilon", 0.0))
        self.h32 = Hps(int(self.hps_on), eps, self.cut32.ctypes.data_as(C.POINTER(C.c_float)),
                       self.lam32.ctypes.data_as(C.POINTER(C.c_float)))
        self.h64 = Hps64(int(self.hps_on), eps, self.cut64.ctypes.data_as(C.POINTER(C.c_double)),
                         self.lam64.ctypes.data_as(C.POINTER(C.c_double)))


class Geom(C.Structure):
    _fields_ = [("n_atoms", C.c_int), ("cutoff_pair", C.c_float), ("cutoff_pair_half", C.c_float),
                ("cutoff_pair2", C.c_float), ("exbox_l", C.c_float * 3), ("box_lower", C.c_float * 3),
                ("n_cells_xy", C.c_int * 2), ("L_cell", C.c_float * 2), ("n_columns", C.c_int),
                ("n_neighbors", C.c_int * 2), ("n_uni_z", C.c_int), ("L_z_uni", C.c_float)]


class Grid(C.Structure):
    _fields_ = [("n_cells", C.c_int), ("n_slots", C.c_int), ("slot_atomid", C.POINTER(C.c_int)),
                ("slot_crd", C.POINTER(C.c_double)), ("atomids_rev", C.POINTER(C.c_int)),
                ("cell_column", C.POINTER(C.c_int)), ("cell_z", C.POINTER(C.c_int)),
                ("col_head_cell", C.POINTER(C.c_int)), ("col_n_atoms", C.POINTER(C.c_int))]


class CellPairs(C.Structure):
    _fields_ = [("n_pairs", C.c_int), ("idx_head", C.POINTER(C.c_int)), ("cell1", C.POINTER(C.c_int)),
                ("cell2", C.POINTER(C.c_int)), ("image", C.POINTER(C.c_int)),
                ("mask", C.POINTER(C.c_uint64))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        from . import build
        path = build.build_oracle()
        L = C.CDLL(path)
        L.ogo_pbc_init.argtypes = [C.POINTER(Pbc), f64p]
        L.ogo_minim_image_d.argtypes = [C.POINTER(Pbc), C.c_int, f64p, f64p, f64p]
        L.ogo_geom_init.argtypes = [C.POINTER(Geom), C.POINTER(Pbc), C.c_int, C.c_double]
        L.ogo_grid_build.argtypes = [C.POINTER(Geom), C.c_int, f64p, C.c_int, C.POINTER(Grid)]
        L.ogo_grid_free.argtypes = [C.POINTER(Grid)]
        L.ogo_enumerate_cell_pairs.argtypes = [C.POINTER(Geom), C.POINTER(Pbc), C.POINTER(Grid), i32p, C.c_int,
                                               C.c_int, C.POINTER(CellPairs)]
        L.ogo_cellpairs_free.argtypes = [C.POINTER(CellPairs)]
        L.ogo_zd_constants.argtypes = [C.c_double, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                       C.POINTER(C.c_float)]
        L.ogo_pair_cells_f32.argtypes = [C.POINTER(Pbc), C.POINTER(Grid), C.POINTER(CellPairs), f32p, i32p, C.c_int,
                                         f32p, f32p, C.c_double, C.c_float, C.c_float, C.c_float, f64p, f64p]
        L.ogo_pair_allpairs_f32.argtypes = [C.POINTER(Pbc), C.c_int, f64p, f32p, i32p, C.c_int, f32p, f32p, i32p,
                                            C.c_int, C.c_double, C.c_float, C.c_float, C.c_float, f64p, f64p]
        L.ogo_pair_allpairs_f64.argtypes = [f64p, C.c_int, f64p, f64p, i32p, C.c_int, f64p, f64p, i32p, C.c_int,
                                            C.c_double, f64p, f64p, f64p]
        L.ogo_pair_cells_f64.argtypes = [f64p, C.POINTER(Grid), C.POINTER(CellPairs), f64p, f64p, i32p, C.c_int,
                                         f64p, f64p, C.c_double, f64p, f64p, f64p]
        L.ogo_excess_f32.argtypes = [C.POINTER(Pbc), C.c_int, i32p, f64p, f32p, C.c_float, C.c_float, f64p]
        L.ogo_excess_f32.restype = C.c_double
        L.ogo_excess_f64.argtypes = [f64p, C.c_int, i32p, f64p, f64p, C.c_double, f64p, f64p]
        L.ogo_excess_f64.restype = C.c_double
        L.ogo_self_energy.argtypes = [C.c_int, C.c_int, i32p, f32p, C.c_float]
        L.ogo_self_energy.restype = C.c_double
        L.ogo_excess_pairs.argtypes = [C.c_int, i32p, C.c_int, i32p, C.c_int]
        L.ogo_bonds.argtypes = [C.POINTER(Pbc), C.c_int, i32p, f64p, f64p, f64p, f64p]
        L.ogo_bonds.restype = C.c_double
        L.ogo_angles.argtypes = [C.POINTER(Pbc), C.c_int, i32p, f64p, f64p, f64p, f64p]
        L.ogo_angles.restype = C.c_double
        L.ogo_dihedrals.argtypes = [C.POINTER(Pbc), C.c_int, i32p, f64p, i32p, i32p, f64p, f64p, f64p]
        L.ogo_dihedrals.restype = C.c_double
        L.ogo_nb14.argtypes = [C.POINTER(Pbc), C.c_int, i32p, i32p, C.c_int, f32p, f32p, f32p, f64p, f64p, f64p,
                               f64p, f64p, f64p]
        L.ogo_mcmd_scale.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, f64p, C.c_double, C.c_int, f64p]
        L.ogo_mcmd_scale.restype = C.c_double
        vp = C.c_void_p
        L.ogo_ele_init.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        L.ogo_ele_init64.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        L.ogo_pair_allpairs_f32_m.argtypes = [C.POINTER(Pbc), C.c_int, f64p, f32p, i32p, C.c_int, f32p, f32p, i32p,
                                              C.c_int, C.c_double, vp, C.POINTER(Hps), f64p, f64p]
        L.ogo_pair_cells_f64_m.argtypes = [f64p, C.POINTER(Grid), C.POINTER(CellPairs), f64p, f64p, i32p, C.c_int,
                                           f64p, f64p, C.c_double, vp, C.POINTER(Hps64), f64p, f64p, f64p]
        L.ogo_excess_f32_m.argtypes = [C.POINTER(Pbc), C.c_int, i32p, f64p, f32p, vp, f64p]
        L.ogo_excess_f32_m.restype = C.c_double
        L.ogo_excess_f64_m.argtypes = [f64p, C.c_int, i32p, f64p, f64p, vp, f64p, f64p]
        L.ogo_excess_f64_m.restype = C.c_double
        L.ogo_self_energy_m.argtypes = [C.c_int, C.c_int, i32p, f32p, vp]
        L.ogo_self_energy_m.restype = C.c_double
        L.ogo_mt_seed.argtypes = [u32p, C.c_uint32]
        L.ogo_mt_next.argtypes = [u32p]
        L.ogo_mt_next.restype = C.c_uint32
        L.ogo_vmcmd_transition.argtypes = [C.c_int, f64p, f64p, C.c_int, C.c_double, u32p]
        L.ogo_vmcmd_transition.restype = C.c_int
        _lib = L
    return _lib


def _arr(ptr, n, dtype):
    if n <= 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def make_pbc(pbc_val):
    p = Pbc()
    lib().ogo_pbc_init(C.byref(p), np.ascontiguousarray(pbc_val, np.float64))
    return p


def make_geom(pbc, n_atoms, nsgrid_cutoff):
    g = Geom()
    rc = lib().ogo_geom_init(C.byref(g), C.byref(pbc), int(n_atoms), float(nsgrid_cutoff))
    if rc != 0:
        raise ValueError("grid geometry rejected (%d)" % rc)
    return g


def geom_dict(g):
    return {"n_cells_x": g.n_cells_xy[0], "n_cells_y": g.n_cells_xy[1], "L_cell_x": g.L_cell[0],
            "L_cell_y": g.L_cell[1], "n_neighbors_x": g.n_neighbors[0], "n_neighbors_y": g.n_neighbors[1],
            "n_uni_z": g.n_uni_z, "L_z_uni": g.L_z_uni, "n_columns": g.n_columns}


def wrap_inbox(pbc, crd):
    """MmSystem::revise_crd_inbox (MmSystem.cpp:808-816) in numpy (while loops, float bounds)."""
    crd = np.array(crd, np.float64).reshape(-1, 3)
    lo = np.array(pbc.lower, np.float32).astype(np.float64)
    up = np.array(pbc.upper, np.float32).astype(np.float64)
    L = np.array(pbc.L, np.float32).astype(np.float64)
    for d in range(3):
        x = crd[:, d]
        while (x < lo[d]).any():
            x[x < lo[d]] += L[d]
        while (x >= up[d]).any():
            x[x >= up[d]] -= L[d]
    return crd


class CellList:
    """Grid assignment + cell-pair list computed by the oracle (copied to numpy).  reference=True
    keeps three faults of the reference's, which lose pairs within the cutoff: its column
    arithmetic wraps an in-box coordinate within float rounding of the upper x or y face into
    column 0 (MiniCell.cpp:329-335); its uniform grid registers a cell whose top lies within
    float rounding of the upper z face in the next column (:912-926); its bin scan hides the
    cells of a neighbour column beyond a z gap of a bin's height (:1062-1076).  The default is
    the engine's grid and list, equal to the reference's whenever none of these occurs."""

    def __init__(self, pbc, geom, crd, nb15off, reference=False):
        L = lib()
        grid = Grid()
        crd = np.ascontiguousarray(crd, np.float64).reshape(-1)
        n = len(crd) // 3
        L.ogo_grid_build(C.byref(geom), n, crd, 1 if reference else 0, C.byref(grid))
        cps = CellPairs()
        L.ogo_enumerate_cell_pairs(C.byref(geom), C.byref(pbc), C.byref(grid),
                                   np.ascontiguousarray(nb15off, np.int32).reshape(-1), MAX_NB15OFF,
                                   1 if reference else 0, C.byref(cps))
        self._grid, self._cps = grid, cps
        self.n_cells = grid.n_cells
        self.n_slots = grid.n_slots
        self.slot_atomid = _arr(grid.slot_atomid, grid.n_slots, np.int32)
        self.slot_crd = _arr(grid.slot_crd, 3 * grid.n_slots, np.float64).reshape(-1, 3)
        self.atomids_rev = _arr(grid.atomids_rev, n, np.int32)
        self.cell_column = _arr(grid.cell_column, grid.n_cells, np.int32)
        self.col_head_cell = _arr(grid.col_head_cell, geom.n_columns + 1, np.int32)
        self.n_pairs = cps.n_pairs
        self.idx_head = _arr(cps.idx_head, grid.n_cells + 1, np.int32)
        self.cell1 = _arr(cps.cell1, cps.n_pairs, np.int32)
        self.cell2 = _arr(cps.cell2, cps.n_pairs, np.int32)
        self.image = _arr(cps.image, cps.n_pairs, np.int32)
        self.mask = _arr(cps.mask, cps.n_pairs, np.uint64)

    def __del__(self):
        try:
            lib().ogo_grid_free(C.byref(self._grid))
            lib().ogo_cellpairs_free(C.byref(self._cps))
        except Exception:
            pass


def unmasked_pair_keys(slot_atomid, cell1, cell2, image, mask):
    """Order-free content of a cell-pair list: one int64 key per unmasked atom pair,
    (lo_id, hi_id, image seen from lo_id), sorted.  Two lists whose grids differ only in the
    order of atoms with equal float z (the reference's quicksort tie order) give equal keys."""
    slot_atomid = np.asarray(slot_atomid, np.int64)
    bits = ((np.asarray(mask, np.uint64)[:, None] >> np.arange(64, dtype=np.uint64)[None, :]) & np.uint64(1)) == 0
    cp, b = np.nonzero(bits)
    a1 = b % 8
    a2 = b // 8
    id1 = slot_atomid[np.asarray(cell1, np.int64)[cp] * 8 + a1]
    id2 = slot_atomid[np.asarray(cell2, np.int64)[cp] * 8 + a2]
    img = np.asarray(image, np.int64)[cp]
    neg = ((img & 1) << 1) | ((img & 2) >> 1) | ((img & 4) << 1) | ((img & 8) >> 1) | ((img & 16) << 1) | ((img & 32) >> 1)
    swap = id1 > id2
    lo = np.where(swap, id2, id1)
    hi = np.where(swap, id1, id2)
    im = np.where(swap, neg, img)
    return np.sort((lo << 32) | (hi << 6) | im)


def zd_constants(cutoff):
    z, b, f = C.c_float(), C.c_float(), C.c_float()
    lib().ogo_zd_constants(float(cutoff), C.byref(z), C.byref(b), C.byref(f))
    return z.value, b.value, f.value


def excess_pairs(n, nb15off):
    cap = int((np.asarray(nb15off) >= 0).sum()) + 1
    out = np.zeros(2 * cap, np.int32)
    ne = lib().ogo_excess_pairs(n, np.ascontiguousarray(nb15off, np.int32).reshape(-1), MAX_NB15OFF, out, cap)
    return out[:2 * ne].reshape(-1, 2)


# ------------------------------------------------------------------ reference MiniCell

_ref = None


class RefCapacityError(RuntimeError):
    pass


def ref_lib():
    """The reference's own MiniCell (None when oracle/_ref was not built)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libogref_minicell.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ogref_minicell.argtypes = [C.c_int, f64p, C.c_double, C.c_double, f64p, i32p, C.c_int, i32p, f32p,
                                     C.c_int, C.POINTER(C.c_int), i32p, f64p, C.c_int, i32p, C.c_int,
                                     C.POINTER(C.c_int), i32p, i32p, i32p, i32p, u32p]
        _ref = R
    return _ref


def ref_pair_capacity(geom, n_atoms, density=1.0):
    """MiniCell::set_grid_xy's cell-pair capacity (MiniCell.cpp:248-280).  The reference calls
    exit(0) from add_cell_pair (:1170-1173) when a list exceeds it, so callers check first."""
    f = np.float32
    nx, ny = geom.n_cells_xy[0], geom.n_cells_xy[1]
    mac = int(math.ceil(f(f(f(f(geom.exbox_l[2]) * f(geom.L_cell[0])) * f(geom.L_cell[1])) * f(density)) * 1.3))
    mac = min(mac, n_atoms)
    nz = (mac - 8 + 1) // 8
    max_cells = nx * ny * nz
    tmp1 = n_atoms // 8 + nx * ny
    if density > 0 and max_cells > tmp1:
        max_cells = tmp1
    nnx, nny = geom.n_neighbors[0], geom.n_neighbors[1]
    cap = int(((nnx * 2 + 1) * (nny * 2 + 1) * (nnx + nny + 2)) * 0.5 * max_cells * 2.5)
    return min(cap, (max_cells * max_cells) // 2)


def ref_minicell(pbc_val, crd, nb15off, nsgrid_cutoff, density=1.0, expected_pairs=None, geom=None):
    """Runs the reference MiniCell; returns None when it is not built.  With expected_pairs and
    geom given, raises RefCapacityError instead of letting the reference exit the process."""
    R = ref_lib()
    if R is None:
        return None
    if expected_pairs is not None and geom is not None:
        n_at = len(np.asarray(crd).reshape(-1)) // 3
        if expected_pairs > ref_pair_capacity(geom, n_at, density):
            raise RefCapacityError("the reference's cell-pair capacity is too small for this box")
    crd = np.ascontiguousarray(crd, np.float64).reshape(-1)
    n = len(crd) // 3
    cap_slots = n + 8 * 200000
    cap_cols = 200000
    cap_pairs = 600 * (n // 8 + 1000)
    gi = np.zeros(8, np.int32)
    gf = np.zeros(4, np.float32)
    slot_atomid = np.zeros(cap_slots, np.int32)
    slot_crd = np.zeros(3 * cap_slots, np.float64)
    col_head = np.zeros(cap_cols, np.int32)
    idx_head = np.zeros(cap_slots // 8 + 2, np.int32)
    c1 = np.zeros(cap_pairs, np.int32)
    c2 = np.zeros(cap_pairs, np.int32)
    img = np.zeros(cap_pairs, np.int32)
    mask = np.zeros(2 * cap_pairs, np.uint32)
    n_cells = C.c_int()
    n_pairs = C.c_int()
    rc = R.ogref_minicell(n, np.ascontiguousarray(pbc_val, np.float64), float(nsgrid_cutoff), float(density), crd,
                          np.ascontiguousarray(nb15off, np.int32).reshape(-1), MAX_NB15OFF, gi, gf, cap_slots,
                          C.byref(n_cells), slot_atomid, slot_crd, cap_cols, col_head, cap_pairs, C.byref(n_pairs),
                          idx_head, c1, c2, img, mask)
    if rc != 0:
        raise RuntimeError("reference MiniCell capacity exceeded")
    nc, npairs, ncol = n_cells.value, n_pairs.value, int(gi[5])
    m = mask[:2 * npairs].astype(np.uint64)
    return {
        "geom": {"n_cells_x": int(gi[0]), "n_cells_y": int(gi[1]), "n_neighbors_x": int(gi[2]),
                 "n_neighbors_y": int(gi[3]), "n_uni_z": int(gi[4]), "n_columns": ncol,
                 "L_cell_x": float(gf[0]), "L_cell_y": float(gf[1]), "L_z_uni": float(gf[2])},
        "n_cells": nc, "slot_atomid": slot_atomid[:8 * nc].copy(), "slot_crd": slot_crd[:24 * nc].reshape(-1, 3).copy(),
        "col_head_cell": col_head[:ncol + 1].copy(), "n_pairs": npairs, "idx_head": idx_head[:nc + 1].copy(),
        "cell1": c1[:npairs].copy(), "cell2": c2[:npairs].copy(), "image": img[:npairs].copy(),
        "mask": m[0::2] | (m[1::2] << np.uint64(32)),
    }


# ------------------------------------------------------------------ oracle MD driver

class Integ(C.Structure):
    _fields_ = [("n", C.c_int), ("dt", C.c_double),
                ("crd", C.POINTER(C.c_double)), ("crd_prev", C.POINTER(C.c_double)), ("vel", C.POINTER(C.c_double)),
                ("vel_next", C.POINTER(C.c_double)), ("work", C.POINTER(C.c_double)),
                ("mass", C.POINTER(C.c_float)), ("mass_inv", C.POINTER(C.c_float)),
                ("n_pair", C.c_int), ("n_trio", C.c_int), ("pair_atoms", C.POINTER(C.c_int)),
                ("pair_dist2", C.POINTER(C.c_double)), ("trio_atoms", C.POINTER(C.c_int)),
                ("trio_dist2", C.POINTER(C.c_double)), ("n_quad", C.c_int), ("quad_atoms", C.POINTER(C.c_int)),
                ("quad_dist2", C.POINTER(C.c_double)), ("shake_max_loops", C.c_int), ("shake_tol", C.c_double),
                ("n_com_groups", C.c_int), ("com_group_start", C.POINTER(C.c_int)),
                ("com_group_atoms", C.POINTER(C.c_int)), ("com_mass_inv", C.POINTER(C.c_float)),
                ("thermostat", C.c_int), ("temperature", C.c_double), ("temperature_coeff", C.c_double),
                ("tau_inv", C.c_double), ("thermo_max_loops", C.c_int), ("thermo_tol", C.c_double),
                ("buf_crd", C.POINTER(C.c_double))]


def _bind_integ(L):
    if getattr(L, "_integ_bound", False):
        return
    ip = C.POINTER(Integ)
    for name in ("ogo_update_velocities", "ogo_thermostat_scaling", "ogo_update_coordinates",
                 "ogo_set_velocity_from_crd"):
        getattr(L, name).argtypes = [ip]
    L.ogo_cancel_com.argtypes = [ip, C.POINTER(C.c_double)]
    L.ogo_shake.argtypes = [ip, C.POINTER(Pbc)]
    L.ogo_thermostat_with_shake.argtypes = [ip, C.POINTER(Pbc)]
    L.ogo_revise_pbc.argtypes = [C.POINTER(Pbc), C.c_int, f64p]
    L.ogo_kinetic.argtypes = [ip, C.c_void_p]
    L.ogo_kinetic.restype = C.c_double
    L._integ_bound = True


def _dihedral_arrays(recs):
    """Torsion or improper records (cls_io.DIHED) as the flat arrays ogo_dihedrals takes."""
    if recs is None or not len(recs):
        return None
    return (np.ascontiguousarray(recs["a"], np.int32).reshape(-1), np.ascontiguousarray(recs["ene"], np.float64),
            np.ascontiguousarray(recs["overlaps"], np.int32), np.ascontiguousarray(recs["symmetry"], np.int32),
            np.ascontiguousarray(recs["phase"], np.float64))


class OracleMD:
    """The reference's leapfrog-presto step (DynamicsModePresto::calc_in_each_step,
    DynamicsMode.cpp:468-560) on the C oracle.  Forces: pair LJ + ZD, excess ZD pairs, bonds,
    angles, torsions, impropers and 1-4 pairs.  ``pair_mode`` "cells_f64" (default) evaluates
    the pair terms in FP64 over the reference's cell-pair list on the list's (unwrapped) grid
    positions; "allpairs_f32" restates the reference's all-pairs build (FP32 pair and excess
    terms, ``-DF_WO_NS``), whose output the ala3 sample log records.  ``params`` uses
    engine.DEFAULT_PARAMS keys.  ``mcmd``: a one-state dict (coef, lambda_low, lambda_high,
    temperature) or the .cls V-McMD section (cls_io: states, interval, temperature, init_vs),
    whose transitions draw from std::mt19937 seeded with params["random_seed"]
    (ExtendedVMcMD::apply_bias, Extend.cpp:126-143)."""

    def __init__(self, system, params, mcmd=None, pair_mode="cells_f64"):
        from omegagene_b200 import cls_io  # local import: oracle stays importable alone
        self.L = L = lib()
        _bind_integ(L)
        t = system["topol"]
        self.n = n = int(system["n_atoms"])
        self.p = dict(params)
        self.pbc = make_pbc(system["pbc_val"])
        self.Ld = np.array(self.pbc.L, np.float32).astype(np.float64)
        self.geom = make_geom(self.pbc, n, self.p["nsgrid_cutoff"])
        self.nb = cls_io.nb15off_table(n, t["nb15off_pairs"])
        self.ep = excess_pairs(n, self.nb).reshape(-1).astype(np.int32)
        self.q64 = np.ascontiguousarray(t["charge"], np.float64)
        self.q32 = self.q64.astype(np.float32)
        self.ty = np.ascontiguousarray(t["atom_type"], np.int32)
        c6, c12 = cls_io.lj_tables(t)
        self.c6, self.c12, self.nt = c6.reshape(-1).copy(), c12.reshape(-1).copy(), int(t["n_lj_types"])
        z, b, f = zd_constants(self.p["cutoff"])
        self.zcore = z
        self.model = EleModel(self.p, t)
        if self.model.default:
            self.self_e = L.ogo_self_energy(n, len(self.ep) // 2, self.ep, self.q32, z)
        else:
            self.self_e = L.ogo_self_energy_m(n, len(self.ep) // 2, self.ep, self.q32, self.model.m32)
        self.mass = np.ascontiguousarray(t["mass"], np.float64).astype(np.float32)
        self.mass_inv = (1.0 / self.mass.astype(np.float64)).astype(np.float32)
        crd = wrap_inbox(self.pbc, system["crd"]).reshape(-1)
        self.crd = np.ascontiguousarray(crd)
        L.ogo_revise_pbc(C.byref(self.pbc), n, self.crd)
        self.crd_prev = np.zeros(3 * n)
        self.vel = np.zeros(3 * n)
        self.vel_next = np.ascontiguousarray(np.asarray(system["vel"], np.float64).reshape(-1)).copy()
        self.work = np.zeros(3 * n)
        self.buf = np.zeros(3 * n)
        b = t.get("bonds")
        self.bonds = None
        if b is not None and len(b):
            self.bonds = (np.ascontiguousarray(np.stack([b["a1"], b["a2"]], 1).astype(np.int32).reshape(-1)),
                          np.ascontiguousarray(b["k"], np.float64), np.ascontiguousarray(b["r0"], np.float64))
        a = t.get("angles")
        self.angles = None
        if a is not None and len(a):
            self.angles = (np.ascontiguousarray(np.stack([a["a1"], a["a2"], a["a3"]], 1).astype(np.int32).reshape(-1)),
                           np.ascontiguousarray(a["k"], np.float64), np.ascontiguousarray(a["t0"], np.float64))
        self.pair_mode = pair_mode
        self.torsions = _dihedral_arrays(t.get("torsions"))
        self.impros = _dihedral_arrays(t.get("impros"))
        n14 = t.get("nb14")
        self.nb14 = None
        if n14 is not None and len(n14["atoms"]):
            self.nb14 = (np.ascontiguousarray(n14["atoms"], np.int32).reshape(-1),
                         np.ascontiguousarray(n14["types"], np.int32).reshape(-1),
                         np.ascontiguousarray(n14["coeff_vdw"], np.float64),
                         np.ascontiguousarray(n14["coeff_ele"], np.float64))
        self.c6f, self.c12f = self.c6.astype(np.float32), self.c12.astype(np.float32)
        cons = system.get("constraint")
        use_cons = cons is not None and self.p.get("constraint", "shake") != "none"
        self.pa = np.asarray(cons["pair_atoms"], np.int32).reshape(-1) if use_cons else np.zeros(0, np.int32)
        self.pd2 = (np.asarray(cons["pair_dist"], np.float64) ** 2).reshape(-1) if use_cons else np.zeros(0)
        self.ta = np.asarray(cons["trio_atoms"], np.int32).reshape(-1) if use_cons else np.zeros(0, np.int32)
        self.td2 = (np.asarray(cons["trio_dist"], np.float64) ** 2).reshape(-1) if use_cons else np.zeros(0)
        qa = np.asarray(cons.get("quad_atoms", np.zeros((0, 4))), np.int32).reshape(-1) if use_cons else None
        self.qa = qa if qa is not None and len(qa) else np.zeros(0, np.int32)
        self.qd2 = ((np.asarray(cons["quad_dist"], np.float64) ** 2).reshape(-1) if len(self.qa)
                    else np.zeros(0))
        self.has_cons = len(self.pd2) + len(self.td2) + len(self.qd2) > 0
        n_cdist = len(self.pd2) + len(self.td2) + len(self.qd2)
        # a position-restraint section adds 3 (Read.cpp:90-93)
        self.d_free = 3 * n - 3 - n_cdist + int(system.get("dof_extra", 0))
        gs, ga, gmi = [0], [], []
        if self.p.get("com_motion", "cancel") == "cancel" and "groups" in system:
            names = self.p.get("com_cancel_groups") or system["groups"]["names"]
            for nm in names:
                atoms = np.asarray(system["groups"]["atoms"][system["groups"]["names"].index(nm)], np.int32)
                ga.extend(atoms.tolist())
                gs.append(len(ga))
                ms = np.float32(0)
                for x in atoms:
                    ms = np.float32(ms + self.mass[x])
                gmi.append(np.float32(1.0 / np.float64(ms)))
        self.gs, self.ga, self.gmi = (np.asarray(gs, np.int32), np.asarray(ga if ga else [0], np.int32),
                                      np.asarray(gmi if gmi else [1.0], np.float32))
        self.t0 = self.p["temperature"]
        self.tinit = self.p["temperature"] if self.p.get("temperature_init", -1) < 0 else self.p["temperature_init"]
        tau = self.p.get("berendsen_tau", 0.0)
        if self.p["time_step"] < tau:
            tau = self.p["time_step"]
        self.tau_inv = (1.0 / tau) if tau > 0 else float("inf")
        self.mcmd = mcmd
        self.vm = mcmd if mcmd is not None and "states" in mcmd else None
        if self.vm is not None:
            st = self.vm["states"]
            self.vs_lam = np.ascontiguousarray([[x["lambda_low"], x["lambda_high"]] for x in st], np.float64).reshape(-1)
            self.vs_prob = np.ascontiguousarray([[x["prob_low"], x["prob_high"]] for x in st], np.float64).reshape(-1)
            self.vs_cur = int(self.vm["init_vs"]) - 1
            self.mt = np.zeros(625, np.uint32)
            L.ogo_mt_seed(self.mt, int(self.p["random_seed"]) & 0xFFFFFFFF)
            self.vs_log, self.lambda_log = [], []
        self.step_i = 0
        self.cl = None
        self.slot_crd = None
        self.I = Integ()
        I = self.I
        I.n, I.dt = n, self.p["time_step"]
        for nm in ("crd", "crd_prev", "vel", "vel_next", "work"):
            setattr(I, nm, getattr(self, nm).ctypes.data_as(C.POINTER(C.c_double)))
        I.buf_crd = self.buf.ctypes.data_as(C.POINTER(C.c_double))
        I.mass = self.mass.ctypes.data_as(C.POINTER(C.c_float))
        I.mass_inv = self.mass_inv.ctypes.data_as(C.POINTER(C.c_float))
        I.n_pair, I.n_trio = len(self.pd2), len(self.td2) // 3
        I.pair_atoms = self.pa.ctypes.data_as(C.POINTER(C.c_int))
        I.pair_dist2 = self.pd2.ctypes.data_as(C.POINTER(C.c_double))
        I.trio_atoms = self.ta.ctypes.data_as(C.POINTER(C.c_int))
        I.trio_dist2 = self.td2.ctypes.data_as(C.POINTER(C.c_double))
        I.n_quad = len(self.qd2) // 6
        I.quad_atoms = self.qa.ctypes.data_as(C.POINTER(C.c_int))
        I.quad_dist2 = self.qd2.ctypes.data_as(C.POINTER(C.c_double))
        I.shake_max_loops, I.shake_tol = self.p["const_max_loops"], self.p["const_tolerance"]
        I.n_com_groups = len(self.gs) - 1
        I.com_group_start = self.gs.ctypes.data_as(C.POINTER(C.c_int))
        I.com_group_atoms = self.ga.ctypes.data_as(C.POINTER(C.c_int))
        I.com_mass_inv = self.gmi.ctypes.data_as(C.POINTER(C.c_float))
        I.thermostat = 1 if self.p["thermostat"] == "scaling" else 0
        I.temperature = self.t0
        I.temperature_coeff = (2.0 * 4.184 * 1e3) / (8.31451 * self.d_free) * ((1e7 / (4.184 * 1e3)) * 0.5)
        I.tau_inv = self.tau_inv
        I.thermo_max_loops, I.thermo_tol = self.p["thermo_const_max_loops"], self.p["thermo_const_tolerance"]
        self.energies = {}

    def rebuild(self):
        self.cl = CellList(self.pbc, self.geom, self.crd, self.nb)
        self.slot_crd = self.cl.slot_crd.copy()

    def forces(self, virial=False):
        """Forces at the current positions into self.work; returns energies."""
        n = self.n
        w = np.zeros(3 * n)
        e = np.zeros(2)
        vir = np.zeros(9)
        vexc = np.zeros(9)
        M = self.model
        if self.pair_mode == "allpairs_f32" and not M.default:
            self.L.ogo_pair_allpairs_f32_m(self.pbc, n, self.crd, self.q32, self.ty, self.nt, self.c6f, self.c12f,
                                           self.nb.reshape(-1), self.nb.shape[1], float(self.p["cutoff"]), M.m32,
                                           C.byref(M.h32), w, e)
            exc = self.L.ogo_excess_f32_m(self.pbc, len(self.ep) // 2, self.ep, self.crd, self.q32, M.m32, w)
        elif self.pair_mode == "allpairs_f32":
            z, b, f = zd_constants(self.p["cutoff"])
            self.L.ogo_pair_allpairs_f32(self.pbc, n, self.crd, self.q32, self.ty, self.nt, self.c6f, self.c12f,
                                         self.nb.reshape(-1), self.nb.shape[1], float(self.p["cutoff"]), z, b, f, w, e)
            exc = self.L.ogo_excess_f32(self.pbc, len(self.ep) // 2, self.ep, self.crd, self.q32, b, f, w)
        else:
            if self.cl is None or self.step_i % self.p["nsgrid_update_intvl"] == 0:
                self.rebuild()
            pos = np.ascontiguousarray(self.slot_crd[self.cl.atomids_rev].reshape(-1))
            if M.default:
                self.L.ogo_pair_cells_f64(self.Ld, self.cl._grid, self.cl._cps, pos, self.q64, self.ty, self.nt,
                                          self.c6, self.c12, float(self.p["cutoff"]), w, e, vir)
                exc = self.L.ogo_excess_f64(self.Ld, len(self.ep) // 2, self.ep, self.crd, self.q64,
                                            float(self.p["cutoff"]), w, vexc)
            else:
                self.L.ogo_pair_cells_f64_m(self.Ld, self.cl._grid, self.cl._cps, pos, self.q64, self.ty, self.nt,
                                            self.c6, self.c12, float(self.p["cutoff"]), M.m64, C.byref(M.h64), w, e,
                                            vir)
                exc = self.L.ogo_excess_f64_m(self.Ld, len(self.ep) // 2, self.ep, self.crd, self.q64, M.m64, w,
                                              vexc)
        eb = ea = 0.0
        if self.bonds is not None:
            eb = self.L.ogo_bonds(self.pbc, len(self.bonds[1]), self.bonds[0], self.bonds[1], self.bonds[2], self.crd, w)
        if self.angles is not None:
            ea = self.L.ogo_angles(self.pbc, len(self.angles[1]), self.angles[0], self.angles[1], self.angles[2],
                                   self.crd, w)
        et = ei = ev14 = ee14 = 0.0
        if self.torsions is not None:
            et = self.L.ogo_dihedrals(self.pbc, len(self.torsions[1]), *self.torsions, self.crd, w)
        if self.impros is not None:
            ei = self.L.ogo_dihedrals(self.pbc, len(self.impros[1]), *self.impros, self.crd, w)
        if self.nb14 is not None:
            o1, o2 = np.zeros(1), np.zeros(1)
            a, ty, cv, ce = self.nb14
            self.L.ogo_nb14(self.pbc, len(cv), a, ty, self.nt, self.c6f, self.c12f, self.q32, cv, ce, self.crd, w,
                            o1, o2)
            ev14, ee14 = float(o1[0]), float(o2[0])
        self.work[:] = w
        ene = {"vdw": e[0], "ele": e[1] + exc + self.self_e, "bond": eb, "angle": ea, "ele_excess": exc,
               "ele_self": self.self_e, "torsion": et, "improper": ei, "vdw14": ev14, "ele14": ee14}
        ene["potential"] = ene["vdw"] + ene["ele"] + eb + ea + et + ei + ev14 + ee14
        if virial:
            ene["virial"] = (vir + vexc).reshape(3, 3)
        return ene

    def step(self):
        L, I = self.L, self.I
        ene = self.forces()
        if self.vm is not None:
            # MmSystem::set_potential_e's order (MmSystem.cpp:738-742)
            lam = (ene["bond"] + ene["angle"] + ene["torsion"] + ene["improper"] + ene["vdw14"] + ene["ele14"] +
                   ene["vdw"] + ene["ele"])
            g = self.step_i
            if g > 0 and g % int(self.vm["interval"]) == 0:
                self.vs_cur = L.ogo_vmcmd_transition(len(self.vm["states"]), self.vs_lam, self.vs_prob, self.vs_cur,
                                                     lam, self.mt)
                self.vs_log.append((g, self.vs_cur))
            li = int(self.p.get("print_intvl_extended_lambda", 0) or 0)
            if g > 0 and li > 0 and g % li == 0:
                self.lambda_log.append((g, lam))
            v = self.vm["states"][self.vs_cur]
            coef = np.ascontiguousarray(v["coef"], np.float64)
            ene["mcmd_factor"] = L.ogo_mcmd_scale(lam, v["lambda_low"], v["lambda_high"], len(coef) - 1, coef,
                                                  float(self.vm["temperature"]), self.n, self.work)
        elif self.mcmd is not None:
            m = self.mcmd
            coef = np.ascontiguousarray(m["coef"], np.float64)
            ene["mcmd_factor"] = L.ogo_mcmd_scale(ene["potential"], m["lambda_low"], m["lambda_high"], len(coef) - 1,
                                                  coef, m["temperature"], self.n, self.work)
        L.ogo_update_velocities(C.byref(I))
        L.ogo_cancel_com(C.byref(I), I.vel_next)
        if I.thermostat == 1:
            hs = self.p.get("heating_steps", 0)
            I.temperature = (self.tinit + ((self.t0 - self.tinit) / hs) * self.step_i) if self.step_i < hs else self.t0
            if not self.has_cons:
                L.ogo_thermostat_scaling(C.byref(I))
        L.ogo_update_coordinates(C.byref(I))
        if self.has_cons:
            if I.thermostat == 1:
                L.ogo_thermostat_with_shake(C.byref(I), C.byref(self.pbc))
            else:
                L.ogo_shake(C.byref(I), C.byref(self.pbc))
                L.ogo_set_velocity_from_crd(C.byref(I))
        # MiniCell::move_atom, then the PBC wrap
        if self.cl is not None:
            self.slot_crd[self.cl.atomids_rev] += (self.crd - self.crd_prev).reshape(-1, 3)
        L.ogo_revise_pbc(C.byref(self.pbc), self.n, self.crd)
        kin = L.ogo_kinetic(C.byref(I), None)
        ene["kinetic"] = kin
        ene["temperature"] = kin * (1.0 / (8.31451 * self.d_free) * 4.184 * 1e3 * 2.0)
        ene["total"] = ene["potential"] + kin
        self.step_i += 1
        self.energies = ene
        return ene
