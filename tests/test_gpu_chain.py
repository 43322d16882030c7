"""The solvated-chain workload at its full size: a 2,000-atom self-avoiding chain (bonds, angles,
every third atom a SHAKE'd hydrogen, per-atom Lennard-Jones types with exact Lorentz-Berthelot
mixing: a 2,002-type table) in 30,000 TIP3P waters less those within 2.4 A of it (86,810 atoms,
a 97.3 A box), cutoff 12 A, zero-dipole alpha 0, velocity rescaling to 300 K, dt 2 fs.

Against the FP64 oracle (reference path: ForceField.cpp:108-177 for the bonds and angles,
ConstraintShake.cpp:18-49 for the SHAKE pairs, Thermostat.cpp:86-170 for the loop):
  * forces at the start: per-atom RMS relative error <= 1e-5; VDW within 1e-6 |E| + 2e-3
    kcal/mol, the pair part of Ele (a small net of ~1.6e7 pair energies of both signs) within
    1e-6 |E| + 1e-7 kcal/mol per atom; the excluded-pair and self parts of Ele, bonds and angles
    (FP64 on both sides) within 1e-9 relative;
    the virial within 1e-5 (Frobenius, relative);
  * the first five steps at 2 fs after a 400-step relaxation at 0.5 fs: potential, kinetic,
    bond and angle energies within 1e-5 |E| + 5e-3 kcal/mol per step.
"""
import numpy as np
import pytest

from omegagene_b200 import engine, systems
from oracle import ogo

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chain():
    s = systems.chain_water_system(2000, 30000, seed=1, radius=30.0, n_sigma_bins=None)
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    return s, p


def _engine(s, p):
    eng = engine.Engine(0)
    eng.add_system(s, p)
    eng.finalize()
    return eng


def test_chain_system_is_the_specified_one(chain):
    s, _ = chain
    assert s["meta"]["n_chain"] == 2000 and s["topol"]["n_lj_types"] == 2002
    assert len(s["constraint"]["pair_atoms"]) == 666 and len(s["constraint"]["trio_atoms"]) == s["meta"]["n_waters"]
    assert 28000 < s["meta"]["n_waters"] < 30000 and abs(s["pbc_val"][0] - 97.26) < 0.1


def test_chain_forces_match_fp64_oracle(chain):
    s, p = chain
    eng = _engine(s, p)
    eng.compute_forces()
    work, ene, vir = eng.get_forces(0)
    md = ogo.OracleMD(s, p)
    e64 = md.forces(virial=True)
    w64 = md.work.reshape(-1, 3)
    err = float(np.sqrt(((work - w64) ** 2).sum() / (w64 ** 2).sum()))
    assert err <= 1e-5, err
    assert abs(ene["vdw"] - e64["vdw"]) <= 1e-6 * abs(e64["vdw"]) + 2e-3, (ene["vdw"], e64["vdw"])
    # Ele = pair + excluded-pair + self terms.  The pair part (+1.9e3 kcal/mol) is itself a small
    # net of ~1.6e7 FP32 pair energies of both signs, so its bar adds 1e-7 kcal/mol per atom to the
    # relative one; the FP64 parts are held to 1e-9
    pair, pair64 = (e["ele"] - e["ele_excess"] - e["ele_self"] for e in (ene, e64))
    assert abs(pair - pair64) <= 1e-6 * abs(pair64) + 1e-7 * s["n_atoms"], (pair, pair64)
    for k in ("ele_excess", "ele_self"):
        assert abs(ene[k] - e64[k]) <= 1e-9 * abs(e64[k]), (k, ene[k], e64[k])
    for k in ("bond", "angle"):  # (the bonds start at their rest length: ~1e-24 kcal/mol)
        assert abs(ene[k] - e64[k]) <= 1e-9 * abs(e64[k]) + 1e-9, (k, ene[k], e64[k])
    assert np.linalg.norm(vir - e64["virial"]) <= 1e-5 * np.linalg.norm(e64["virial"])
    eng.close()


def test_chain_energy_trace_matches_oracle(chain):
    s, p = chain
    # the generator's start (a random walk dropped into a lattice of waters) relaxes violently:
    # 400 steps at 0.5 fs with the thermostat first, on the engine; both sides then start from
    # the relaxed state
    eq = _engine(s, dict(p, time_step=0.5))
    eq.step(400)
    crd, vel = eq.get_state(0)
    eq.close()
    s = dict(s, crd=crd, vel=vel)
    n = 5
    eng = _engine(s, p)
    eng.set_trace(n)
    eng.step(n)
    tr = eng.get_trace(n)[:, 0, :]
    md = ogo.OracleMD(s, p)
    names = engine.ENERGY_NAMES
    for i in range(n):
        r = md.step()
        for k in ("potential", "kinetic", "bond", "angle", "temperature"):
            got = tr[i, names.index(k)]
            assert abs(got - r[k]) <= 1e-5 * abs(r[k]) + 5e-3, (i, k, got, r[k])
    assert eng.flags() & (8 | 16) == 0  # SHAKE and the thermostat loop converged
    eng.close()
