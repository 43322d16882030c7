"""Constructed systems shared by the CPU and GPU tests: water boxes placed where the reference's
MiniCell list build loses pairs (see test_oracle.py)."""
import numpy as np

from omegagene_b200 import systems
from oracle import ogo


def void_water():
    """3,000-site water box (44.8 A) with the molecules inside a 10 x 10 x 18 A block removed: the
    columns through the block have empty uniform z bins (7.47 A) between filled ones, and the
    scan windows of cells beside the cavity reach across it (196,067 cell pairs by the
    reference's scan, 196,320 with the cells beyond the gap)."""
    return systems.water_system(3000, box=44.8, seed=0, lattice_m=15, void=((-5.0, -5.0, -9.0), (5.0, 5.0, 9.0)))


def face_water():
    """3,000-site water box (44.8 A) with molecule 0 moved so that its oxygen sits 1e-7 A below
    the upper x face, where float(x - lower) rounds to the box length; molecules within 2.6 A of
    its new place are removed.  Velocities zero."""
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    pbc = ogo.make_pbc(s["pbc_val"])
    crd = np.array(s["crd"], dtype=np.float64)
    upper = float(np.float32(pbc.upper[0]))
    crd[0:3, 0] += upper - 1e-7 - crd[0, 0]
    crd[0:3] = ogo.wrap_inbox(pbc, crd[0:3])
    d = crd.reshape(-1, 3, 3)[:, 0, :] - crd[0]
    d -= float(pbc.L[0]) * np.round(d / float(pbc.L[0]))
    keep = np.sqrt((d ** 2).sum(1)) > 2.6
    keep[0] = True
    w = crd.reshape(-1, 3, 3)[keep].reshape(-1, 3)
    nw = len(w) // 3
    mass = np.tile([systems.M_O, systems.M_H, systems.M_H], nw)
    return systems._assemble(w + 0.5 * 44.8, np.zeros((3 * nw, 3)), 44.8,
                             charge=np.tile([systems.Q_O, systems.Q_H, systems.Q_H], nw), mass=mass,
                             atom_type=np.tile([0, 1, 1], nw), lj_types=[(systems.SIGMA_O, systems.EPS_O), (0.0, 0.0)],
                             bonds=None, angles=None, excl=systems._water_exclusions(0, nw), pairs=None,
                             trios=systems._water_trios(0, nw))
