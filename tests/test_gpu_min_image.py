"""A water molecule split across opposite faces inside the reference minimum image's failure
window (see tests/test_min_image.py): in a 31.95 A box (window +-1.86e-6 A) a water at rest
has O near the upper x face and H1 through the face near the lower one, placed so that after
the first step's unconstrained update their x offset through the face is 1e-6 A: the two
truncating passes of PBC::diff_crd_minim_image (PBC.cpp:70-84) return that O-H1 vector one box
long, and the reference's SHAKE trio, solving for it, throws the molecule across the box.  With
the guarded pass the engine's SHAKE holds the molecule rigid, no step faults, and the positions
after one step agree with the FP64 oracle's."""
import math

import numpy as np
import pytest

from omegagene_b200 import engine, systems
from oracle import ogo

pytestmark = pytest.mark.gpu

BOX = 31.95


FORCE_VEL = 4.184e-4  # CelesteObject.cpp:36


def _assemble(w, vel):
    nw = len(w)
    mass = np.tile([systems.M_O, systems.M_H, systems.M_H], nw)
    return systems._assemble(w.reshape(-1, 3) + 0.5 * BOX, vel, BOX,
                             charge=np.tile([systems.Q_O, systems.Q_H, systems.Q_H], nw), mass=mass,
                             atom_type=np.tile([0, 1, 1], nw), lj_types=[(systems.SIGMA_O, systems.EPS_O), (0.0, 0.0)],
                             bonds=None, angles=None, excl=systems._water_exclusions(0, nw), pairs=None,
                             trios=systems._water_trios(0, nw))


def _split_water_system(params, seed=2, n_waters=1000, offset=1e-6):
    """Water 0 (at rest) straddles the x faces so that after the first step's unconstrained
    update its O - H1 x difference is +-(L - offset); the update's displacement F/m dt^2 is
    taken from the FP64 oracle's forces, placing the molecule by fixed-point iteration."""
    rng = np.random.default_rng(seed)
    w = systems.water_positions(rng, n_waters, BOX).reshape(n_waters, 3, 3) - 0.5 * BOX  # centred frame
    Lf = float(np.float32(BOX))
    lower = -float(np.float32(np.float32(BOX) * np.float32(0.5)))
    upper = float(np.float32(np.float32(lower) + np.float32(Lf)))
    th = math.radians(104.52)
    y0, z0 = 1.0, -2.0

    def molecule(t):
        """O and H1 through the x face with true x offset t (H1 - O), each |t|/2 inside its
        face; H2 beside O."""
        e = 0.5 * abs(t)
        ox = upper - e if t > 0 else lower + e
        o = np.array([ox, y0, z0])
        h1 = np.array([ox + t - (Lf if t > 0 else -Lf), y0 + math.sqrt(systems.R_OH ** 2 - t * t), z0])
        h2 = np.array([ox, y0 + systems.R_OH * math.cos(th), z0 + systems.R_OH * math.sin(th)])
        return np.stack([o, h1, h2])

    # clear room for the molecule whichever face O ends up at
    mols = np.concatenate([molecule(0.05), molecule(-0.05)])
    d = w.reshape(-1, 1, 3) - mols.reshape(1, 6, 3)
    d -= BOX * np.round(d / BOX)
    near = (np.sqrt((d * d).sum(-1)) < 3.2).reshape(n_waters, 18).any(1)
    rest = w[~near][1:]
    mass = np.tile([systems.M_O, systems.M_H, systems.M_H], 1 + len(rest))
    vel = systems._maxwell(rng, mass, 300.0)
    vel[:3] = 0.0
    dt2 = params["time_step"] ** 2
    delta = 0.0
    for _ in range(8):
        # after the update, O - H1 = (raw O - H1) + delta with raw = +-L - t: aim at +-(L - offset)
        t = offset + delta if offset + delta > 0 else delta - offset
        s = _assemble(np.concatenate([molecule(t)[None], rest]), vel)
        md = ogo.OracleMD(s, params)
        md.forces()
        wk = md.work.reshape(-1, 3)
        m_inv = np.float32(1.0) / np.asarray(s["topol"]["mass"], np.float32)
        dx = -FORCE_VEL * wk[:2, 0] * m_inv[:2].astype(np.float64) * dt2
        delta = dx[0] - dx[1]
    return s, Lf, dx


def _two_pass(d, pbc):
    lhi = np.float32(pbc.L_half_inv[0])
    for _ in range(2):
        d = d - float(np.float32(pbc.L[0]) * np.float32(int(d * float(lhi))))
    return d


def test_split_water_inside_the_window():
    p = dict(engine.DEFAULT_PARAMS)
    p.update(time_step=2.0, nsgrid_update_intvl=10, thermostat="none")
    s, L, dx = _split_water_system(p)
    c = np.asarray(s["crd"])
    pbc = ogo.make_pbc(s["pbc_val"])
    # the input really is the failing case: after the update, O - H1 is one box long by the
    # reference's two passes
    post = (c[0, 0] + dx[0]) - (c[1, 0] + dx[1])
    assert abs(abs(post) - L) < 1.5e-6 and abs(_two_pass(post, pbc)) > 0.75 * L
    eng = engine.Engine(0)
    eng.set_tuning(10)
    eng.add_system(s, p)
    eng.finalize()
    eng.step(1)
    c1, _ = eng.get_state(0)
    md = ogo.OracleMD(s, p)
    md.step()
    assert np.abs(c1 - md.crd.reshape(-1, 3)).max() < 1e-6
    eng.step(49)
    assert eng.flags() & 8 == 0  # SHAKE converged on every step
    c2, _ = eng.get_state(0)
    for i, j, r in ((0, 1, systems.R_OH), (0, 2, systems.R_OH), (1, 2, systems.R_HH)):
        v = c2[i] - c2[j]
        v -= L * np.round(v / L)
        assert abs(np.linalg.norm(v) - r) < 1e-6 * r, (i, j, np.linalg.norm(v))
    eng.close()
