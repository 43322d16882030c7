"""The minimum image of the constraint, bonded and excluded-pair terms.

The reference's PBC::diff_crd_minim_image (PBC.cpp:70-84) truncates d * L_half_inv to int twice,
with L and L_half_inv = 1 / (L/2) in float.  Where float L * float L_half_inv rounds above 2, a
difference within L (L L_half_inv / 2 - 1) of +-L passes +L -> -L through the two truncations
and comes back one box long instead of ~0.  That is two atoms of one molecule on opposite faces
whose x agree to a few microangstroms; the reference's SHAKE then diverges and throws the
molecule across the box (a 2,000-atom chain in 29,000 waters, 97.26 A box, at 2 fs met it every
few thousand steps).  The oracle and the engine add one guarded pass that fires only on such a
result (|d| > 3L/4).  Here: the two-pass restatement fails inside the window, the guarded pass
returns the true offset there, and everywhere else the oracle's output is the two-pass result
bit for bit."""
import numpy as np
import pytest

from oracle import ogo


def _pbc(L):
    return ogo.make_pbc([L, 0, 0, 0, L, 0, 0, 0, L, 0, 0, 0])


def two_pass(d, L, lhi):
    """PBC.cpp:78-79 as the reference computes it: float L times the float of the truncated
    quotient, subtracted in double."""
    for _ in range(2):
        d = d - float(np.float32(L) * np.float32(int(d * float(lhi))))
    return d


def _oracle(p, a, b):
    a = np.ascontiguousarray(a, np.float64).reshape(-1, 3)
    b = np.ascontiguousarray(b, np.float64).reshape(-1, 3)
    d = np.zeros_like(a)
    ogo.lib().ogo_minim_image_d(p, len(a), a, b, d)
    return d


@pytest.mark.parametrize("box", [97.26438448, 31.95, 45.8])
def test_reference_minimum_image_fails_in_its_window_and_the_guard_fixes_it(box):
    p = _pbc(box)
    L, lhi = np.float32(p.L[0]), np.float32(p.L_half_inv[0])
    assert float(L) * float(lhi) > 2.0  # the boxes with a window
    window = float(L) * (float(L) * float(lhi) / 2 - 1)
    upper = float(np.float32(p.upper[0]))
    tested = 0
    for off in (3e-6, 1e-6, 2e-7, -2e-7, -1e-6, -3e-6):
        if abs(off) >= 0.9 * window:
            continue
        # a just inside the upper face, b one box below a plus `off`: the true x of a - b is -off
        a = np.array([upper - 1e-6, 0.3, -0.2])
        b = np.array([a[0] - float(L) + off, 1.25, 0.4])
        ref = two_pass(a[0] - b[0], L, lhi)
        assert abs(ref) > 0.75 * float(L), (box, off, ref)  # the reference's result: one box long
        got = _oracle(p, a, b)[0]
        assert abs(got[0] + off) < 1e-9, (box, off, got[0])
        assert got[1] == a[1] - b[1] and got[2] == a[2] - b[2]
        tested += 1
    assert tested >= 2


@pytest.mark.parametrize("box", [97.26438448, 31.95, 44.8, 215.5])
def test_guarded_minimum_image_is_the_reference_elsewhere(box):
    p = _pbc(box)
    L, lhi = float(np.float32(p.L[0])), np.float32(p.L_half_inv[0])
    rng = np.random.default_rng(11)
    n = 20000
    a = rng.uniform(-0.5 * L, 0.5 * L, (n, 3))
    b = a - rng.uniform(-1.4 * L, 1.4 * L, (n, 3))
    got = _oracle(p, a, b)
    diff = a - b
    for k in range(n):
        for q in range(3):
            ref = two_pass(diff[k, q], L, lhi)
            if abs(ref) <= 0.75 * L:
                assert got[k, q] == ref, (box, k, q, got[k, q], ref)
            else:  # only inside the window
                assert abs(abs(diff[k, q]) - L) < 1e-5 and abs(got[k, q]) < 1e-5


def test_box_of_the_million_atom_workload_has_no_window():
    """215.5 A: float L * float L_half_inv rounds below 2, so the two passes never cycle."""
    p = _pbc(215.5)
    L, lhi = np.float32(p.L[0]), np.float32(p.L_half_inv[0])
    assert float(L) * float(lhi) < 2.0
    for e in np.linspace(-1e-5, 1e-5, 201):
        for s in (-1.0, 1.0):
            assert abs(two_pass(s * float(L) + e, L, lhi)) < 1e-4
