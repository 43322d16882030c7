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


def moved_water(mol, axis, delta):
    """3,000-site water box (44.8 A) with molecule `mol` moved so that its oxygen sits `delta` A
    below the box's upper face along `axis`; molecules within 2.6 A of its new place are
    removed.  Velocities zero."""
    s = systems.water_system(3000, box=44.8, seed=0, lattice_m=15)
    pbc = ogo.make_pbc(s["pbc_val"])
    crd = np.array(s["crd"], dtype=np.float64)
    upper = float(np.float32(pbc.upper[axis]))
    sl = slice(3 * mol, 3 * mol + 3)
    crd[sl, axis] += upper - delta - crd[3 * mol, axis]
    crd[sl] = ogo.wrap_inbox(pbc, crd[sl])
    d = crd.reshape(-1, 3, 3)[:, 0, :] - crd[3 * mol]
    d -= float(pbc.L[0]) * np.round(d / float(pbc.L[0]))
    keep = np.sqrt((d ** 2).sum(1)) > 2.6
    keep[mol] = True
    w = crd.reshape(-1, 3, 3)[keep].reshape(-1, 3)
    nw = len(w) // 3
    mass = np.tile([systems.M_O, systems.M_H, systems.M_H], nw)
    return systems._assemble(w + 0.5 * 44.8, np.zeros((3 * nw, 3)), 44.8,
                             charge=np.tile([systems.Q_O, systems.Q_H, systems.Q_H], nw), mass=mass,
                             atom_type=np.tile([0, 1, 1], nw), lj_types=[(systems.SIGMA_O, systems.EPS_O), (0.0, 0.0)],
                             bonds=None, angles=None, excl=systems._water_exclusions(0, nw), pairs=None,
                             trios=systems._water_trios(0, nw))


def face_water():
    """Molecule 0's oxygen 1e-7 A below the upper x face, where float(x - lower) rounds to the
    box length."""
    return moved_water(0, 0, 1e-7)


def top_water():
    """Molecule 9's oxygen 2e-7 A below the upper z face, where its cell's top divides out to
    the uniform bin n_uni_z (201,810 cell pairs by the reference's grid, 201,962 with the cell
    kept in its own column)."""
    return moved_water(9, 2, 2e-7)
