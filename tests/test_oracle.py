"""The CPU oracle against the reference: its own MiniCell (bit for bit) and the ala3
known answer printed by the reference all-pairs build."""
import json
import os

import numpy as np
import pytest

from omegagene_b200 import cls_io, systems
from oracle import build as obuild
from oracle import ogo

import cases

HERE = os.path.dirname(os.path.abspath(__file__))


def _cell_list_case(s, cutoff=13.0):
    nb = cls_io.nb15off_table(s["n_atoms"], s["topol"]["nb15off_pairs"])
    pbc = ogo.make_pbc(s["pbc_val"])
    crd = ogo.wrap_inbox(pbc, s["crd"])
    geom = ogo.make_geom(pbc, s["n_atoms"], cutoff)
    return nb, pbc, crd, geom


@pytest.fixture(scope="module")
def ref_built():
    """The reference's MiniCell built into oracle/_ref (rebuilt first when its sources are
    present; a prebuilt library is used as it is)."""
    obuild.build_ref()
    if ogo.ref_lib() is None:
        pytest.skip("oracle/_ref was not built (reference sources absent)")
    return True


@pytest.mark.parametrize("n_waters,box,seed", [(3000, 44.8, 0), (1500, None, 5), (1234, None, 7)])
def test_cell_list_matches_reference_minicell(ref_built, n_waters, box, seed):
    s = systems.water_system(n_waters, box=box, seed=seed)
    nb, pbc, crd, geom = _cell_list_case(s)
    ours = ogo.CellList(pbc, geom, crd, nb, reference=True)
    ref = ogo.ref_minicell(s["pbc_val"], crd, nb, 13.0, expected_pairs=ours.n_pairs, geom=geom)
    assert ogo.geom_dict(geom) == pytest.approx(ref["geom"])
    assert ours.n_cells == ref["n_cells"]
    for k in ("slot_atomid", "col_head_cell", "idx_head", "cell1", "cell2", "image", "mask"):
        np.testing.assert_array_equal(getattr(ours, k), ref[k], err_msg=k)
    np.testing.assert_array_equal(ours.slot_crd, ref["slot_crd"])


def _ala3_system():
    """The reference's ala3 launch set (samples/ala3/md.inp.cls), from the committed fixture."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(HERE, "golden",
                                                                                 "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.load_system()


def test_cell_list_matches_reference_on_ala3(ref_built):
    """ala3's coordinates come from a PDB (0.001 A grid), so atoms of one column can share a
    float z; the reference's quicksort orders such ties arbitrarily.  A seeded 1e-3 A
    perturbation removes the ties; both implementations get the same coordinates."""
    s = _ala3_system()
    s["crd"] = s["crd"] + np.random.default_rng(11).uniform(-1e-3, 1e-3, s["crd"].shape)
    nb, pbc, crd, geom = _cell_list_case(s)
    ours = ogo.CellList(pbc, geom, crd, nb, reference=True)
    ref = ogo.ref_minicell(s["pbc_val"], crd, nb, 13.0, expected_pairs=ours.n_pairs, geom=geom)
    for k in ("slot_atomid", "idx_head", "cell1", "cell2", "image", "mask"):
        np.testing.assert_array_equal(getattr(ours, k), ref[k], err_msg=k)
    np.testing.assert_array_equal(ours.slot_crd, ref["slot_crd"])


def test_reference_capacity_guard():
    """Small boxes overflow the reference's max_n_cells^2/2 pair buffer (it exits); the guard
    reports that instead of running it."""
    s = systems.water_system(700, seed=5)
    nb, pbc, crd, geom = _cell_list_case(s)
    ours = ogo.CellList(pbc, geom, crd, nb)
    assert ours.n_pairs > ogo.ref_pair_capacity(geom, s["n_atoms"])


def _ala3_energies():
    s = _ala3_system()
    n, t = s["n_atoms"], s["topol"]
    nb = cls_io.nb15off_table(n, t["nb15off_pairs"])
    pbc = ogo.make_pbc(s["pbc_val"])
    crd = ogo.wrap_inbox(pbc, s["crd"]).reshape(-1)
    c6, c12 = cls_io.lj_tables(t)
    q = t["charge"].astype(np.float32)
    ty = t["atom_type"].astype(np.int32)
    z, b, f = ogo.zd_constants(12.0)
    work, ene = np.zeros(3 * n), np.zeros(2)
    L = ogo.lib()
    L.ogo_pair_allpairs_f32(pbc, n, crd, q, ty, int(t["n_lj_types"]), c6.astype(np.float32).reshape(-1),
                            c12.astype(np.float32).reshape(-1), nb.reshape(-1), 32, 12.0, z, b, f, work, ene)
    ep = ogo.excess_pairs(n, nb).reshape(-1).astype(np.int32)
    exc = L.ogo_excess_f32(pbc, len(ep) // 2, ep, crd, q, b, f, np.zeros(3 * n))
    self_e = L.ogo_self_energy(n, len(ep) // 2, ep, q, z)
    return ene[0], ene[1] + exc + self_e


def test_oracle_reproduces_ala3_known_answer():
    gold = json.load(open(os.path.join(HERE, "golden", "ala3_step0.json")))["step0"]
    vdw, ele = _ala3_energies()
    assert float("%.10e" % vdw) == gold["VDW"]
    assert float("%.10e" % ele) == gold["Ele"]


def test_zd_constants_alpha0():
    z, b, f = ogo.zd_constants(12.0)
    assert z == pytest.approx(1.5 / 12.0, rel=1e-7)
    assert f == pytest.approx(1.0 / 12.0 ** 3, rel=1e-7)
    assert b == pytest.approx(0.5 / 12.0 ** 3, rel=1e-7)


def test_fp32_cell_path_close_to_fp64_oracle():
    s = systems.water_system(700, seed=2)
    nb, pbc, crd, geom = _cell_list_case(s)
    cl = ogo.CellList(pbc, geom, crd, nb)
    n, t = s["n_atoms"], s["topol"]
    c6, c12 = cls_io.lj_tables(t)
    q, ty = t["charge"], t["atom_type"].astype(np.int32)
    L = np.array(pbc.L, np.float32).astype(np.float64)
    w64, e64, v64 = np.zeros(3 * n), np.zeros(2), np.zeros(9)
    ogo.lib().ogo_pair_allpairs_f64(L, n, crd.reshape(-1), q, ty, int(t["n_lj_types"]), c6.reshape(-1),
                                    c12.reshape(-1), nb.reshape(-1), 32, 12.0, w64, e64, v64)
    w64c, e64c, v64c = np.zeros(3 * n), np.zeros(2), np.zeros(9)
    ogo.lib().ogo_pair_cells_f64(L, cl._grid, cl._cps, crd.reshape(-1), q, ty, int(t["n_lj_types"]),
                                 c6.reshape(-1), c12.reshape(-1), 12.0, w64c, e64c, v64c)
    # the cell list is complete: FP64 over the list equals FP64 over all pairs
    np.testing.assert_allclose(w64c, w64, rtol=0, atol=1e-9)
    np.testing.assert_allclose(e64c, e64, rtol=1e-12)
    np.testing.assert_allclose(v64c, v64, rtol=1e-10, atol=1e-7)


def _ala3_golden():
    sys_path = os.path.join(HERE, "golden")
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_ala3_golden", os.path.join(sys_path, "make_ala3_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    gold = json.load(open(os.path.join(sys_path, "ala3_log.json")))
    return mod.load_system(), gold


def test_oracle_reproduces_ala3_log_trajectory():
    """The oracle's all-pairs mode against every energy the reference printed for the first ten
    steps of its ala3 sample (bond, angle, torsion, improper, 1-4 VDW/Ele, VDW, Ele, kinetic,
    total, temperature): equal to the printed 11 significant digits.  This pins the integrator,
    SHAKE pair/trio/quad, COM cancel and the bonded terms, not only the pair energies."""
    s, gold = _ala3_golden()
    md = ogo.OracleMD(s, gold["params"], pair_mode="allpairs_f32")
    assert md.d_free == 12417
    for row in gold["steps"][:10]:
        got = md.step()
        for key, ref in row.items():
            if key == "step":
                continue
            assert float("%.10e" % got[key]) == ref, (row["step"], key, got[key], ref)


def test_oracle_reproduces_reference_thermostat_runs():
    """The velocity-scaling thermostat against the reference's own runs of its ala3 sample
    (tests/golden/ala3_thermo.json, made by make_thermo_golden.py with the reference's all-pairs
    program): the thermostat-with-SHAKE loop at 300 K (Thermostat.cpp:86-170), the same with a
    heating ramp 200 -> 300 K (SubBox.cpp:1745-1757), and the unconstrained scaling
    (Thermostat.cpp:57-84).  Every printed energy of the first eight steps, to the printed 11
    significant digits."""
    s, _ = _ala3_golden()
    gold = json.load(open(os.path.join(HERE, "golden", "ala3_thermo.json")))
    for name, run in gold["runs"].items():
        md = ogo.OracleMD(s, run["params"], pair_mode="allpairs_f32")
        for row in run["steps"][:8]:
            got = md.step()
            for key, ref in row.items():
                if key == "step":
                    continue
                assert float("%.10e" % got[key]) == ref, (name, row["step"], key, got[key], ref)


def test_cell_list_across_a_z_gap():
    """The reference's bin scan (MiniCell.cpp:1062-1076) stops at the first empty bin after a
    filled one, so cells of a neighbour column beyond the cavity are never paired and atom pairs
    within the cutoff are lost.  The engine's list (first to last filled bin) holds every pair
    within the cutoff, holds every pair of the reference's list, and its FP64 forces equal the
    all-pairs ones; the reference's list gives forces off by far more than rounding."""
    s = cases.void_water()
    nb, pbc, crd, geom = _cell_list_case(s)
    ref = ogo.CellList(pbc, geom, crd, nb, reference=True)
    ours = ogo.CellList(pbc, geom, crd, nb)
    k_ref = ogo.unmasked_pair_keys(ref.slot_atomid, ref.cell1, ref.cell2, ref.image, ref.mask)
    k_ours = ogo.unmasked_pair_keys(ours.slot_atomid, ours.cell1, ours.cell2, ours.image, ours.mask)
    assert np.isin(k_ref, k_ours).all() and len(k_ours) > len(k_ref)
    # every atom pair within 12 A (minimum image, exclusions aside) is in the engine's list;
    # pair codes (lo << 26 | hi) are the keys without their image bits
    from scipy.spatial import cKDTree
    L = float(pbc.L[0])
    x = np.mod(np.asarray(crd, np.float64).reshape(-1, 3) - np.array(pbc.lower, np.float64), L)
    close = cKDTree(x, boxsize=L).query_pairs(11.99, output_type="ndarray").astype(np.int64)
    close = np.sort(close, axis=1)
    ii = np.repeat(np.arange(s["n_atoms"], dtype=np.int64), nb.shape[1])
    jj = np.asarray(nb, np.int64).reshape(-1)
    excl = (ii[jj > ii] << 26) | jj[jj > ii]
    want = (close[:, 0] << 26) | close[:, 1]
    want = want[~np.isin(want, excl)]
    assert np.isin(want, k_ours >> 6).all()
    assert not np.isin(want, k_ref >> 6).all()
    # forces: FP64 over each list vs FP64 all pairs, both at the list's grid positions (the
    # coordinates rounded through float, MiniCell.cpp:413-470)
    n, t = s["n_atoms"], s["topol"]
    c6, c12 = cls_io.lj_tables(t)
    q, ty = t["charge"], t["atom_type"].astype(np.int32)
    Ld = np.array(pbc.L, np.float32).astype(np.float64)
    grid_pos = np.ascontiguousarray(ours.slot_crd[ours.atomids_rev].reshape(-1))
    wa, ea, va = np.zeros(3 * n), np.zeros(2), np.zeros(9)
    ogo.lib().ogo_pair_allpairs_f64(Ld, n, np.ascontiguousarray(ogo.wrap_inbox(pbc, grid_pos).reshape(-1)), q, ty,
                                    int(t["n_lj_types"]), c6.reshape(-1), c12.reshape(-1), nb.reshape(-1),
                                    nb.shape[1], 12.0, wa, ea, va)
    for cl, close_enough in ((ours, True), (ref, False)):
        pos = np.ascontiguousarray(cl.slot_crd[cl.atomids_rev].reshape(-1))
        w, e, v = np.zeros(3 * n), np.zeros(2), np.zeros(9)
        ogo.lib().ogo_pair_cells_f64(Ld, cl._grid, cl._cps, pos, q, ty, int(t["n_lj_types"]), c6.reshape(-1),
                                     c12.reshape(-1), 12.0, w, e, v)
        err = float(np.abs(w - wa).max())
        assert (err < 1e-6) == close_enough, err


@pytest.mark.parametrize("case", ["face", "top"])
def test_atom_at_an_upper_face_keeps_its_pairs(case):
    """face: the reference computes x = crd - lower in float and wraps x >= L
    (MiniCell.cpp:329-335); an in-box oxygen 1e-7 A below the upper x face goes into column 0, a
    box length from the grid coordinate it keeps.  top: the reference's uniform grid puts a cell
    whose top lies 2e-7 A below the upper z face in bin n_uni_z, which is the next column's bin 0
    (:912-926), so the cells of its own column do not find it.  Either way pairs within the
    cutoff go missing from the reference's list; FP64 forces over the engine's list equal the
    all-pairs ones."""
    s = cases.face_water() if case == "face" else cases.top_water()
    nb, pbc, crdw, geom = _cell_list_case(s)
    if case == "face":
        L = float(np.float32(pbc.L[0]))
        assert np.float32(crdw[0, 0] - np.float64(np.float32(pbc.lower[0]))) == np.float32(L)
    n, t = s["n_atoms"], s["topol"]
    c6, c12 = cls_io.lj_tables(t)
    q, ty = t["charge"], t["atom_type"].astype(np.int32)
    Ld = np.array(pbc.L, np.float32).astype(np.float64)
    errs = {}
    for ref_mode in (True, False):
        cl = ogo.CellList(pbc, geom, crdw, nb, reference=ref_mode)
        pos = np.ascontiguousarray(cl.slot_crd[cl.atomids_rev].reshape(-1))
        wa, ea, va = np.zeros(3 * n), np.zeros(2), np.zeros(9)
        ogo.lib().ogo_pair_allpairs_f64(Ld, n, np.ascontiguousarray(ogo.wrap_inbox(pbc, pos).reshape(-1)), q, ty,
                                        int(t["n_lj_types"]), c6.reshape(-1), c12.reshape(-1), nb.reshape(-1),
                                        nb.shape[1], 12.0, wa, ea, va)
        wc, ec, vc = np.zeros(3 * n), np.zeros(2), np.zeros(9)
        ogo.lib().ogo_pair_cells_f64(Ld, cl._grid, cl._cps, pos, q, ty, int(t["n_lj_types"]), c6.reshape(-1),
                                     c12.reshape(-1), 12.0, wc, ec, vc)
        errs[ref_mode] = float(np.abs(wc - wa).max())
    assert errs[True] > 1e-2 and errs[False] < 1e-6, errs
