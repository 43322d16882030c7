"""The pair variant over j lists (variant 10) against the j-queue variant (9) and the oracle.

Variant 10 culls the j atoms of each cell's cell pairs once per list build, with a margin of
0.7 A (twice the 0.35 A skin), and rebuilds its lists whenever an atom has moved farther than
the skin since.  It must evaluate exactly the pairs variant 9 evaluates; the two differ only
in the order in which FP32 partial sums are added.
* Over three list intervals the two give the same trajectory and the oracle's energies.  The
  order of FP32 partial sums alone separates them by ~4e-7 A after 30 steps (measured), so
  positions are compared within 1e-5 A.
* One molecule moved by 1 A through og_put_state in the middle of an interval (no cell-pair
  list rebuild) brings pairs that were beyond cutoff + margin inside the cutoff: the j lists are
  rebuilt, and two steps later positions still agree with variant 9's to 1e-6 A.  The ~50 pairs
  per moved atom that stale lists would miss (11.5-12 A, ~0.1 kcal/mol/A each) would move its
  hydrogens by ~1e-3 A.
* An og_put_state of unchanged coordinates (the end-to-end protocol) keeps the lists, and the
  step after it matches variant 9's.
* Every atom translated by 0.7 A (9,000 and 18,000 atoms): the lists are rebuilt and the step
  matches variant 9, energies included.
"""
import numpy as np
import pytest

from omegagene_b200 import engine, systems
from oracle import ogo

pytestmark = pytest.mark.gpu


def _params(**kw):
    p = dict(engine.DEFAULT_PARAMS)
    p.update(nsgrid_update_intvl=10, time_step=2.0)
    p.update(kw)
    return p


def _engine(s, p, variant):
    eng = engine.Engine(0)
    eng.set_tuning(variant)
    eng.add_system(s, p)
    eng.finalize()
    return eng


def test_jlist_trajectory_matches_jqueue_and_oracle():
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    p = _params(thermostat="scaling", temperature=300.0)
    n = 30
    out = {}
    for v in (9, 10):
        eng = _engine(s, p, v)
        assert eng.tuning()["pair_variant"] == v
        eng.set_trace(n)
        eng.step(n)
        out[v] = (eng.get_state(0), eng.get_trace(n)[:, 0, :])
        eng.close()
    (c9, v9), t9 = out[9]
    (c10, v10), t10 = out[10]
    assert np.max(np.abs(c10 - c9)) < 1e-5
    assert np.max(np.abs(v10 - v9)) < 1e-3
    names = engine.ENERGY_NAMES
    for k in ("potential", "vdw", "ele"):
        i = names.index(k)
        assert np.max(np.abs(t10[:, i] - t9[:, i]) / np.abs(t9[:, i])) < 1e-6, k
    md = ogo.OracleMD(s, p)
    ref = [md.step() for _ in range(n)]
    for i, r in enumerate(ref):
        for k in ("potential", "vdw", "ele", "kinetic"):
            got = t10[i, names.index(k)]
            assert abs(got - r[k]) <= 1e-5 * abs(r[k]) + 5e-3, (i, k, got, r[k])


def _put(eng, crd):
    buf = np.ascontiguousarray(crd, np.float64).reshape(-1)
    eng.put_state_ptr(0, buf.ctypes.data, 0)
    eng.synchronize()


@pytest.mark.parametrize("shift", [0.0, 1.0])
def test_jlist_rebuilds_after_a_move_beyond_the_skin(shift):
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    p = _params(thermostat="none")
    res = {}
    for v in (9, 10):
        eng = _engine(s, p, v)
        eng.step(4)  # mid-interval: the next list build is at step 10
        crd, _ = eng.get_state(0)
        crd = crd.copy()
        crd[300:303, 0] += shift  # one water molecule
        b0 = eng.jlist_builds()
        _put(eng, crd)
        eng.step(2)
        res[v] = eng.get_state(0)
        if v == 10 and shift > 0.35:
            assert eng.jlist_builds() > b0  # the move beyond the skin rebuilt the j lists
        eng.close()
    assert np.max(np.abs(res[10][0] - res[9][0])) < 1e-6
    assert np.max(np.abs(res[10][1] - res[9][1])) < 1e-3


@pytest.mark.parametrize("n_waters", [3000, 6000])
def test_every_atom_moved_beyond_the_skin(n_waters):
    box = 44.8 * (n_waters / 3000) ** (1 / 3)
    s = systems.water_system(n_waters, box=box, seed=1, lattice_m=int(np.ceil(n_waters ** (1 / 3))) + 1)
    p = _params(thermostat="none")
    res = {}
    for v in (9, 10):
        eng = _engine(s, p, v)
        eng.step(4)
        crd, _ = eng.get_state(0)
        crd = crd + np.array([0.7, 0.3, -0.4]) * 0.7 / np.sqrt(0.74)  # every atom moves 0.7 A
        b0 = eng.jlist_builds()
        _put(eng, crd)
        eng.step(2)
        res[v] = eng.get_state(0) + (eng.get_energies(0),)
        if v == 10:
            assert eng.jlist_builds() > b0
        eng.close()
    assert np.max(np.abs(res[10][0] - res[9][0])) < 1e-6
    assert np.max(np.abs(res[10][1] - res[9][1])) < 1e-3
    for k in ("potential", "vdw", "ele"):
        assert abs(res[10][2][k] - res[9][2][k]) <= 1e-6 * abs(res[9][2][k]), k


def test_put_state_from_pinned_and_pageable_buffers_agree():
    """og_put_state from a pinned and from a pageable host buffer: the same state, bit for bit
    (a scatter kernel reading the pinned buffer over PCIe instead of a staging copy was tried:
    1.12 ms against 0.53 ms for 24 MB)."""
    import torch
    s = systems.water_system(1500, seed=5)
    p = _params(thermostat="none")
    out = []
    for pinned in (False, True):
        eng = _engine(s, p, 10)
        eng.step(3)
        crd, vel = eng.get_state(0)
        crd = crd + 0.01
        if pinned:
            c = torch.from_numpy(np.ascontiguousarray(crd).reshape(-1)).pin_memory()
            v = torch.from_numpy(np.ascontiguousarray(vel).reshape(-1)).pin_memory()
            eng.put_state_ptr(0, c.data_ptr(), v.data_ptr())
        else:
            c = np.ascontiguousarray(crd).reshape(-1)
            v = np.ascontiguousarray(vel).reshape(-1)
            eng.put_state_ptr(0, c.ctypes.data, v.ctypes.data)
        eng.synchronize()
        eng.step(2)
        out.append(eng.get_state(0))
        eng.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("age", [3, 6])
def test_aged_jlists_give_the_fresh_lists_forces(age):
    """Two identical runs; in one, an atom is moved 0.6 A and back through og_put_state, which
    marks the j lists stale, so its next step evaluates freshly built j lists while the other
    evaluates lists built up to `age` steps earlier (the same cell-pair list, the same
    coordinates).  A pair missing from the aged lists (one at 11.5-12 A moves a hydrogen by
    ~1e-5 A in a step) would separate the two; summation order alone leaves them within 1e-8 A."""
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    p = _params(thermostat="none", time_step=0.5)
    runs = []
    for fresh in (False, True):
        eng = _engine(s, p, 10)
        eng.step(10)  # one list interval, then `age` steps into the next
        last = 0
        for k in range(age):
            b = eng.jlist_builds()
            eng.step(1)
            if eng.jlist_builds() > b:
                last = k + 1
        if not fresh:
            assert age - last >= 2, "the lists were rebuilt %d steps ago" % (age - last)
        if fresh:
            crd, _ = eng.get_state(0)
            moved = crd.copy()
            moved[7, 0] += 0.6
            b0 = eng.jlist_builds()
            _put(eng, moved)
            _put(eng, crd)
        eng.step(1)
        if fresh:
            assert eng.jlist_builds() == b0 + 1
        runs.append(eng.get_state(0))
        eng.close()
    assert np.max(np.abs(runs[0][0] - runs[1][0])) < 1e-8
    assert np.max(np.abs(runs[0][1] - runs[1][1])) < 1e-5
