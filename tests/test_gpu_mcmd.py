"""Batched V-McMD walkers against the FP64 oracle over their first 200 steps.

Three walkers (a 300-atom synthetic chain in 2,500 TIP3P waters each, own seeds, hydrogens held
by angle terms) relax together for 400 steps at 0.5 fs, then run in one engine with velocity
rescaling to 300 K, dt 2 fs, and each walker's order-6 polynomial.  The middle walker's per-step
energies are compared with the oracle's FP64 run from the same relaxed state:
  * steps 0-49: potential and kinetic energy within 1e-5 |E| + 5e-3 kcal/mol, as for the other
    trajectory tests;
  * every step: the engine's McMD factor equals the walker's polynomial evaluated in FP64 on the
    host at the engine's own potential energy (1e-7 relative: the raw-power form cancels);
  * steps 0-49: the McMD factor within 1e-7 relative of the oracle's;
  * steps 0-199: the McMD factor within 1e-5 relative, the kinetic energy within 1e-5, the
    potential energy within 5e-3 relative.  FP32 pair forces (RMS error ~1e-6) start a
    separation that an MD trajectory amplifies by roughly e every 25 steps, so the bound widens
    with the step count; the mean potential over steps 100-199 stays within 1e-3 relative.
"""
import numpy as np
import pytest

from omegagene_b200 import engine, systems
from oracle import ogo

pytestmark = pytest.mark.gpu


def test_mcmd_walkers_track_oracle_200_steps():
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=10, time_step=2.0, thermostat="scaling", temperature=300.0)
    walkers = [systems.chain_water_system(300, 2500, seed=500 + w, radius=12.0) for w in range(3)]
    warm = engine.Engine(0)
    for w in walkers:
        warm.add_system(w, dict(p, time_step=0.5))
    warm.finalize()
    warm.step(400)
    for i, w in enumerate(walkers):
        w["crd"], w["vel"] = warm.get_state(i)
    warm.close()
    e0 = [ogo.OracleMD(w, p).forces()["potential"] for w in walkers]
    polys = [systems.mcmd_polynomial(e, 300.0, seed=900 + k) for k, e in enumerate(e0)]
    eng = engine.Engine(0)
    for w, m in zip(walkers, polys):
        eng.add_system(w, p, m)
    eng.finalize()
    n = 200
    eng.set_trace(n)
    eng.step(n)
    tr = eng.get_trace(n)[:, 1, :]
    md = ogo.OracleMD(walkers[1], p, polys[1])
    ref = [md.step() for _ in range(n)]
    names = engine.ENERGY_NAMES
    got = {k: tr[:, names.index(k)] for k in ("potential", "kinetic", "mcmd_factor")}
    want = {k: np.array([r[k] for r in ref]) for k in got}
    assert np.all(np.abs(want["mcmd_factor"] - 1.0) < 0.2)
    for k in ("potential", "kinetic"):
        d = np.abs(got[k][:50] - want[k][:50])
        assert np.all(d <= 1e-5 * np.abs(want[k][:50]) + 5e-3), (k, d.max())
    poly = polys[1]
    e_cl = np.clip(got["potential"], poly["lambda_low"], poly["lambda_high"])
    own = systems.KB_KCAL * poly["temperature"] * sum(c * e_cl ** i for i, c in enumerate(poly["coef"]))
    assert np.all(np.abs(got["mcmd_factor"] - own) <= 1e-7 * np.abs(own))
    rel = np.abs(got["mcmd_factor"] - want["mcmd_factor"]) / np.abs(want["mcmd_factor"])
    assert np.all(rel[:50] <= 1e-7) and np.all(rel <= 1e-5), rel.max()
    assert np.all(np.abs(got["kinetic"] - want["kinetic"]) <= 1e-5 * np.abs(want["kinetic"]))
    assert np.all(np.abs(got["potential"] - want["potential"]) <= 5e-3 * np.abs(want["potential"]))
    m1, m2 = got["potential"][100:].mean(), want["potential"][100:].mean()
    assert abs(m1 - m2) <= 1e-3 * abs(m2)
