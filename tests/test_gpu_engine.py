"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Integer / index results (grid assignment, cell-pair list, masks) must be bit-exact; forces,
energies and the virial are compared with the FP64 oracle within the stated tolerances:
  * force RMS relative error  sqrt(sum|F - F64|^2 / sum|F64|^2) <= 1e-5
  * potential energy terms    |E - E64| <= 1e-6 |E64| + 2e-3 kcal/mol
  * virial                    ||W - W64||_F <= 1e-5 ||W64||_F
"""
import numpy as np
import pytest

from omegagene_b200 import engine, systems
from oracle import ogo

import cases

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5


def _params(**kw):
    p = dict(engine.DEFAULT_PARAMS)
    p.update(kw)
    return p


def _oracle_cells(s, p):
    from omegagene_b200 import cls_io
    nb = cls_io.nb15off_table(s["n_atoms"], s["topol"]["nb15off_pairs"])
    pbc = ogo.make_pbc(s["pbc_val"])
    crd = ogo.wrap_inbox(pbc, s["crd"])
    geom = ogo.make_geom(pbc, s["n_atoms"], p["nsgrid_cutoff"])
    return ogo.CellList(pbc, geom, crd, nb)


def _engine(systems_and_params, variant=None):
    eng = engine.Engine(0)
    if variant is not None:
        eng.set_tuning(variant)
    for s, p, m in systems_and_params:
        eng.add_system(s, p, m)
    eng.finalize()
    return eng


def _rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


SMALL = [
    ("water3000", lambda: systems.water_system(3000, box=44.8, seed=0, lattice_m=15)),
    ("water1500", lambda: systems.water_system(1500, seed=5)),
    ("water700", lambda: systems.water_system(700, seed=9)),
    ("chain300", lambda: systems.chain_water_system(300, 2500, seed=4, radius=12.0)),
    # where the reference's list build loses pairs (tests/cases.py, test_oracle.py): a cavity
    # whose z gap its bin scan does not cross, oxygens at the upper x and z faces
    ("water_void", cases.void_water),
    ("water_face", cases.face_water),
    ("water_top", cases.top_water),
]


@pytest.mark.parametrize("name,make", SMALL, ids=[n for n, _ in SMALL])
def test_cell_list_bit_exact(name, make):
    s = make()
    p = _params()
    eng = _engine([(s, p, None)])
    ref = _oracle_cells(s, p)
    g = eng.get_grid(0)
    cp = eng.get_cell_pairs(0)
    assert g["n_cells"] == ref.n_cells
    np.testing.assert_array_equal(g["slot_atomid"], ref.slot_atomid)
    np.testing.assert_array_equal(g["slot_crd"], ref.slot_crd)
    np.testing.assert_array_equal(g["col_head_cell"], ref.col_head_cell)
    assert cp["n_pairs"] == ref.n_pairs
    for k in ("idx_head", "cell1", "cell2", "image", "mask"):
        np.testing.assert_array_equal(cp[k], getattr(ref, k), err_msg=k)


def test_batched_cell_lists_equal_single():
    ss = [make() for _, make in SMALL]
    p = _params()
    eng = _engine([(s, p, None) for s in ss])
    for i, s in enumerate(ss):
        ref = _oracle_cells(s, p)
        cp = eng.get_cell_pairs(i)
        g = eng.get_grid(i)
        np.testing.assert_array_equal(g["slot_atomid"], ref.slot_atomid)
        for k in ("idx_head", "cell1", "cell2", "image", "mask"):
            np.testing.assert_array_equal(cp[k], getattr(ref, k), err_msg="%d %s" % (i, k))


@pytest.mark.parametrize("variant", [0, 3, 5, 7])
@pytest.mark.parametrize("name,make", SMALL, ids=[n for n, _ in SMALL])
def test_forces_energies_virial_vs_fp64(name, make, variant):
    """The four pair-kernel families (0: warp per 8x8 cell pair, 3: j-major, 5: j-major with
    packed FP32x2 arithmetic, 7: packed j-major fed by a queue of j atoms near the i cell)."""
    s = make()
    p = _params()
    eng = _engine([(s, p, None)], variant)
    eng.compute_forces()
    work, ene, vir = eng.get_forces(0)
    md = ogo.OracleMD(s, p)
    e64 = md.forces(virial=True)
    err = _rel_rms(work, md.work.reshape(-1, 3))
    assert err <= FORCE_RTOL, err
    for k in ("vdw", "ele", "bond", "angle", "potential"):
        assert abs(ene[k] - e64[k]) <= 1e-6 * abs(e64[k]) + 2e-3, (k, ene[k], e64[k])
    w64 = e64["virial"]
    assert np.linalg.norm(vir - w64) <= 1e-5 * np.linalg.norm(w64), (vir, w64)


@pytest.mark.parametrize("name,make", SMALL, ids=[n for n, _ in SMALL])
def test_fp64_variant_matches_fp64_oracle(name, make):
    """The FP64 validation variant evaluates what the FP64 oracle evaluates (the same list, the
    same formulas in double precision): forces within 1e-9 RMS relative (the fixed-point
    accumulators resolve 2^-32 kcal/mol/A), energies within 1e-9 relative; the virial within
    1e-7 (its x (x) f part reads positions from the FP32 cell-relative offsets)."""
    s = make()
    p = _params()
    eng = _engine([(s, p, None)], engine.PAIR_VARIANT_F64)
    assert eng.tuning()["pair_variant"] == engine.PAIR_VARIANT_F64
    eng.compute_forces()
    work, ene, vir = eng.get_forces(0)
    md = ogo.OracleMD(s, p)
    e64 = md.forces(virial=True)
    assert _rel_rms(work, md.work.reshape(-1, 3)) <= 1e-9
    for k in ("vdw", "ele", "bond", "angle", "potential"):
        assert abs(ene[k] - e64[k]) <= 1e-9 * abs(e64[k]) + 1e-9, (k, ene[k], e64[k])
    # the virial's x (x) f part takes the positions from the FP32 cell-relative offsets
    assert np.linalg.norm(vir - e64["virial"]) <= 1e-7 * np.linalg.norm(e64["virial"])


def test_fp64_variant_refuses_other_models():
    s = systems.water_system(700, seed=9)
    eng = engine.Engine(0)
    eng.set_tuning(engine.PAIR_VARIANT_F64)
    eng.add_system(s, _params(electrostatic="zero-quadrupole"))
    with pytest.raises(engine.OgError) as ex:
        eng.finalize()
    assert ex.value.status == engine.OG_ERR_INVALID


def test_forces_bitwise_reproducible():
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    eng = _engine([(s, _params(), None)])
    eng.compute_forces()
    w1, e1, _ = eng.get_forces(0)
    eng.compute_forces()
    w2, e2, _ = eng.get_forces(0)
    assert np.array_equal(w1, w2)
    assert e1 == e2


def _run_both(s, p, n_steps, mcmd=None, variant=None):
    eng = _engine([(s, p, mcmd)], variant)
    eng.set_trace(n_steps)
    md = ogo.OracleMD(s, p, mcmd)
    ref = [md.step() for _ in range(n_steps)]
    eng.step(n_steps)
    tr = eng.get_trace(n_steps)[:, 0, :]
    return eng, md, ref, tr


@pytest.mark.parametrize("variant", range(engine.N_PAIR_VARIANTS))
def test_one_step_state_matches_oracle(variant):
    """Every pair-kernel variant: positions and velocities after one step."""
    s = systems.water_system(1500, seed=5)
    p = _params(nsgrid_update_intvl=10, time_step=2.0)
    eng, md, ref, tr = _run_both(s, p, 1, variant=variant)
    crd, vel = eng.get_state(0)
    assert np.max(np.abs(crd.reshape(-1) - md.crd)) < 1e-6
    assert np.max(np.abs(vel.reshape(-1) - md.vel_next)) < 1e-6


@pytest.mark.parametrize("thermostat,dt", [("none", 2.0), ("scaling", 0.5)])
def test_energy_trace_matches_oracle(thermostat, dt):
    s = systems.water_system(1500, seed=5)
    p = _params(nsgrid_update_intvl=10, time_step=dt, thermostat=thermostat, temperature=300.0)
    eng, md, ref, tr = _run_both(s, p, 12)
    names = engine.ENERGY_NAMES
    for i, r in enumerate(ref):
        for k in ("potential", "kinetic", "total", "vdw", "ele"):
            got = tr[i, names.index(k)]
            assert abs(got - r[k]) <= 1e-5 * abs(r[k]) + 5e-3, (i, k, got, r[k])


def test_chain_with_bonds_angles_shake_pairs_matches_oracle():
    s = systems.chain_water_system(300, 2500, seed=4, radius=12.0)
    p = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    eng, md, ref, tr = _run_both(s, p, 8)
    names = engine.ENERGY_NAMES
    for i, r in enumerate(ref):
        for k in ("potential", "kinetic", "bond", "angle"):
            got = tr[i, names.index(k)]
            assert abs(got - r[k]) <= 1e-5 * abs(r[k]) + 5e-3, (i, k, got, r[k])


def test_mcmd_scaling_matches_oracle():
    s = systems.chain_water_system(300, 2500, seed=6, radius=12.0)
    p = _params(nsgrid_update_intvl=10, time_step=2.0)
    md0 = ogo.OracleMD(s, p)
    e0 = md0.forces()["potential"]
    # d lnP / dE as a polynomial in E with RT dlnP/dE = O(1), as a McMD run uses it
    mcmd = {"coef": [1.678, 2e-5, 1e-9, 0, 0, 0, 1e-24], "lambda_low": e0 - 2000.0, "lambda_high": e0 + 2000.0,
            "temperature": 300.0}
    eng, md, ref, tr = _run_both(s, p, 6, mcmd)
    names = engine.ENERGY_NAMES
    for i, r in enumerate(ref):
        assert 0.5 < r["mcmd_factor"] < 2.0
        assert abs(tr[i, names.index("mcmd_factor")] - r["mcmd_factor"]) <= 1e-7 * abs(r["mcmd_factor"])
        assert abs(tr[i, names.index("potential")] - r["potential"]) <= 1e-5 * abs(r["potential"]) + 5e-3


@pytest.mark.parametrize("variant", [1, 6, 8, 9, 10])
def test_batch_invariance_bitwise(variant):
    """A system gives the same trajectory alone and batched with others (fixed-point forces,
    per-system fixed-order reductions), for a given pair-kernel variant (variants of different
    families add FP32 partial sums in different orders).  The mix holds a deliberately hot
    system (velocities x4, no thermostat): with the j-list kernel (variant 10) its atoms pass
    the skin far more often than the others', so the engine rebuilds j lists at steps where
    the system under test alone would not; only the hot system's lists may change then."""
    a = systems.water_system(1500, seed=5)
    hot = systems.water_system(700, seed=9)
    hot = dict(hot, vel=np.asarray(hot["vel"]) * 4.0)
    chain = systems.chain_water_system(300, 2500, seed=4, radius=12.0)
    p = _params(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    p_hot = _params(nsgrid_update_intvl=10, time_step=2.0)
    alone = _engine([(a, p, None)], variant)
    alone.set_trace(25)
    alone.step(25)
    mixed = _engine([(hot, p_hot, None), (a, p, None), (chain, p, None)], variant)
    mixed.set_trace(25)
    mixed.step(25)
    np.testing.assert_array_equal(alone.get_trace(25)[:, 0, :], mixed.get_trace(25)[:, 1, :])
    c1, v1 = alone.get_state(0)
    c2, v2 = mixed.get_state(1)
    assert np.array_equal(c1, c2) and np.array_equal(v1, v2)
    if variant == 10:
        # the hot system forced j-list builds that the system alone did not have
        assert mixed.jlist_builds() > alone.jlist_builds() >= 3, (mixed.jlist_builds(), alone.jlist_builds())


def test_jlist_put_state_of_other_system_keeps_bits():
    """Variant 10: moving a molecule of another system through og_put_state between steps marks
    only that system's j lists stale; the system under test keeps its trajectory bit for bit."""
    a = systems.water_system(1500, seed=5)
    b = systems.water_system(700, seed=9)
    p = _params(nsgrid_update_intvl=10, time_step=2.0)
    alone = _engine([(a, p, None)], 10)
    mixed = _engine([(a, p, None), (b, p, None)], 10)
    for k in range(3):
        alone.step(3)
        mixed.step(3)
        crd, _ = mixed.get_state(1)
        crd = crd.copy()
        crd[3 * (10 + k):3 * (11 + k)] += np.array([0.8, -0.5, 0.3])  # one water, 1 A
        mixed.put_state_ptr(1, crd.ctypes.data, None)
        mixed.synchronize()
    alone.step(7)
    mixed.step(7)
    c1, v1 = alone.get_state(0)
    c2, v2 = mixed.get_state(0)
    assert np.array_equal(c1, c2) and np.array_equal(v1, v2)
    assert mixed.jlist_builds() > alone.jlist_builds()


def test_nve_drift_small():
    """Config-0 water: short velocity-rescaled warm-up at 0.5 fs, then NVE at 2 fs; the total
    energy drift stays within 0.01 kcal/mol/ns per degree of freedom.  The pair variant is fixed
    (the j-list kernel) so that the trajectory is reproducible, and the slope is fitted over
    2,900 steps: over 900 steps the estimate scatters by +-0.016 with the FP32 summation order
    alone (measured over pair variants 6/9/10 and two seeds), over 2,900 by +-0.002."""
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    warm = _params(nsgrid_update_intvl=10, time_step=0.5, thermostat="scaling", temperature=300.0)
    eng = _engine([(s, warm, None)], variant=10)
    eng.step(2000)
    crd, vel = eng.get_state(0)
    s2 = dict(s)
    s2["crd"], s2["vel"] = crd, vel
    nve = _params(nsgrid_update_intvl=10, time_step=2.0)
    eng2 = _engine([(s2, nve, None)], variant=10)
    eng2.set_trace(3000)
    eng2.step(3000)
    tr = eng2.get_trace(3000)[:, 0, :]
    tot = tr[:, engine.ENERGY_NAMES.index("total")]
    t_ns = np.arange(len(tot)) * 2.0 * 1e-6
    slope = np.polyfit(t_ns[100:], tot[100:], 1)[0]
    dof = 3 * s["n_atoms"] - 3 - 3 * 3000
    assert abs(slope) / dof <= 0.01, slope / dof
