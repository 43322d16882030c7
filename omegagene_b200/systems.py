"""Seeded synthetic systems for the benchmark workloads (no public dataset is used by the
reference or named for these workloads; these generators stand in for them).

All systems are returned as launch-set dicts with the keys of :mod:`cls_io` (so they can
be written as .cls files for the reference CPU programs) plus a few convenience arrays.

Water model: rigid TIP3P, O-H 0.9572 A, H-O-H 104.52 deg, q_O -0.834 e, q_H +0.417 e,
LJ on O only (sigma 3.15061 A, epsilon 0.1521 kcal/mol) written in the .cls convention
E = C12/r^12 - C6/r^6 with C12 = 4 eps sigma^12, C6 = 4 eps sigma^6.
"""
import math

import numpy as np

WATER_NUMBER_DENSITY = 0.997 * 6.02214076e23 / 18.01528 / 1e24  # molecules / A^3 at 0.997 g/cm^3
R_OH = 0.9572
THETA_HOH = math.radians(104.52)
R_HH = 2.0 * R_OH * math.sin(THETA_HOH / 2.0)
Q_O, Q_H = -0.834, 0.417
M_O, M_H = 15.9994, 1.008
SIGMA_O, EPS_O = 3.15061, 0.1521
KB_KCAL = 8.31451 / 4.184 * 1e-3  # GAS_CONST / JOULE_CAL * 1e-3 (kcal/mol/K)


def water_box_side(n_waters):
    return (n_waters / WATER_NUMBER_DENSITY) ** (1.0 / 3.0)


def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def _maxwell(rng, mass, temperature):
    """Velocities in A/fs drawn at the temperature (KINETIC_COEFF convention, kcal/mol)."""
    # KE[kcal/mol] = 0.5 m v^2 * 1e7/4184 with v in A/fs and m in amu (CelesteObject.cpp:39)
    sd = np.sqrt(KB_KCAL * temperature / (mass * (1e7 / 4184.0)))
    return rng.normal(size=(len(mass), 3)) * sd[:, None]


def water_positions(rng, n_waters, box, lattice_m=None, jitter=0.3, origin=0.0):
    """O on seeded-random sites of an m^3 lattice with uniform jitter, random orientations."""
    m = lattice_m or int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    spacing = box / m
    sites = rng.choice(m ** 3, size=n_waters, replace=False)
    ijk = np.stack([sites // (m * m), (sites // m) % m, sites % m], 1).astype(np.float64)
    o = origin + (ijk + 0.5) * spacing + rng.uniform(-jitter, jitter, size=(n_waters, 3))
    half = THETA_HOH / 2.0
    h_local = np.array([[R_OH * math.sin(half), 0.0, R_OH * math.cos(half)],
                        [-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)]])
    rot = _random_rotations(rng, n_waters)
    h = np.einsum("nij,kj->nki", rot, h_local) + o[:, None, :]
    xyz = np.empty((n_waters, 3, 3))
    xyz[:, 0] = o
    xyz[:, 1:] = h
    return xyz.reshape(-1, 3)


def _wrap(crd, lo, box):
    return lo + np.mod(crd - lo, box)


def water_system(n_waters, box=None, seed=0, temperature=300.0, lattice_m=None, jitter=0.3, void=None):
    """Rigid TIP3P box: one SHAKE trio per molecule, exclusions within molecules.  void = (lo, hi)
    corners of a block (box-centred coordinates): molecules with an atom inside it are removed,
    leaving a cavity."""
    rng = np.random.default_rng(seed)
    box = float(box if box is not None else water_box_side(n_waters))
    crd = water_positions(rng, n_waters, box, lattice_m=lattice_m, jitter=jitter)
    if void is not None:
        lo, hi = np.asarray(void[0], float), np.asarray(void[1], float)
        c = crd.reshape(-1, 3, 3) - 0.5 * box
        inside = np.all((c >= lo) & (c <= hi), axis=2).any(axis=1)
        crd = crd.reshape(-1, 3, 3)[~inside].reshape(-1, 3)
        n_waters = len(crd) // 3
    n = 3 * n_waters
    mass = np.tile([M_O, M_H, M_H], n_waters)
    vel = _maxwell(rng, mass, temperature)
    vel -= (mass[:, None] * vel).sum(0) / mass.sum()
    sys_ = _assemble(crd, vel, box,
                     charge=np.tile([Q_O, Q_H, Q_H], n_waters),
                     mass=mass,
                     atom_type=np.tile([0, 1, 1], n_waters),
                     lj_types=[(SIGMA_O, EPS_O), (0.0, 0.0)],
                     bonds=None, angles=None,
                     excl=_water_exclusions(0, n_waters),
                     pairs=None,
                     trios=_water_trios(0, n_waters))
    sys_["meta"] = {"kind": "water", "n_waters": n_waters, "seed": seed, "box": box}
    return sys_


def _water_exclusions(first_atom, n_waters):
    o = first_atom + 3 * np.arange(n_waters)
    return np.concatenate([np.stack([o, o + 1], 1), np.stack([o, o + 2], 1), np.stack([o + 1, o + 2], 1)])


def _water_trios(first_atom, n_waters):
    o = first_atom + 3 * np.arange(n_waters)
    atoms = np.stack([o, o + 1, o + 2], 1)
    dist = np.tile([R_OH, R_HH, R_OH], (n_waters, 1))
    return atoms, dist


def _lj_records(lj_types, mix="lb"):
    """LJ pair records with Lorentz-Berthelot mixing; types with eps 0 get zero terms."""
    nt = len(lj_types)
    sig = np.array([t[0] for t in lj_types], np.float64)
    eps = np.array([t[1] for t in lj_types], np.float64)
    i, j = np.triu_indices(nt)
    s = 0.5 * (sig[i] + sig[j])
    e = np.sqrt(eps[i] * eps[j])
    out = np.zeros(len(i), dtype=[("t1", "<i4"), ("t2", "<i4"), ("p6", "<f8"), ("p12", "<f8")])
    out["t1"], out["t2"] = i + 1, j + 1
    # powers through the C library's pow, one value at a time (numpy's vectorised pow may
    # round differently in the last bit)
    sl = s.tolist()
    out["p6"] = 4.0 * e * np.array([x ** 6 for x in sl])
    out["p12"] = 4.0 * e * np.array([x ** 12 for x in sl])
    return out


def _assemble(crd, vel, box, charge, mass, atom_type, lj_types, bonds, angles, excl, pairs, trios,
              groups=None):
    n = len(crd)
    lo = -0.5 * box
    # box centred on the origin (pbc_val[9..11] is the box centre, PBC.cpp:36)
    crd = _wrap(crd - 0.5 * box, lo, box)
    lj_pairs = _lj_records(lj_types)
    # Read::load_ls_tpl reads one HPS record per LJ type pair whatever the section size says
    # (Read.cpp:323-334), so the records are written (unused by the LJ model)
    hps = np.zeros(len(lj_pairs), dtype=[("t1", "<i4"), ("t2", "<i4"), ("cutoff", "<f8"), ("lambda", "<f8")])
    hps["t1"], hps["t2"] = lj_pairs["t1"], lj_pairs["t2"]
    topol = {
        "charge": np.asarray(charge, np.float64),
        "mass": np.asarray(mass, np.float64),
        "atom_type": np.asarray(atom_type, np.int32),
        "n_lj_types": len(lj_types),
        "lj_pairs": lj_pairs,
        "lj_hps_raw": hps.tobytes(),
        "bonds": bonds if bonds is not None else np.zeros(0, [("a1", "<i4"), ("a2", "<i4"), ("k", "<f8"), ("r0", "<f8")]),
        "angles": angles if angles is not None else np.zeros(0, [("a1", "<i4"), ("a2", "<i4"), ("a3", "<i4"), ("k", "<f8"), ("t0", "<f8")]),
        "torsions_raw": b"\0\0\0\0", "impros_raw": b"\0\0\0\0", "nb14_raw": b"\0\0\0\0",
        "nb15off_pairs": np.concatenate([excl, excl[:, ::-1]], 1).reshape(-1, 2).astype(np.int32),
    }
    cons = {"pair_atoms": np.zeros((0, 2), np.int32), "pair_dist": np.zeros(0),
            "trio_atoms": np.zeros((0, 3), np.int32), "trio_dist": np.zeros((0, 3)),
            "quad_atoms": np.zeros((0, 4), np.int32), "quad_dist": np.zeros((0, 6))}
    if pairs is not None:
        cons["pair_atoms"], cons["pair_dist"] = pairs
    if trios is not None:
        cons["trio_atoms"], cons["trio_dist"] = trios
    pbc_val = np.array([box, 0, 0, 0, box, 0, 0, 0, box, 0.0, 0.0, 0.0])
    out = {"n_atoms": n, "pbc_val": pbc_val, "crd": crd, "vel": vel, "topol": topol, "constraint": cons,
           "groups": groups or {"names": ["all"], "atoms": [np.arange(n, dtype=np.int32)]}}
    return out


def _saw_chain(rng, n_backbone, radius, bond=1.53, angle_deg=111.0, min_dist=3.2, max_tries=200):
    """Self-avoiding random walk with fixed bond length and bond angle, confined to a sphere."""
    theta = math.radians(angle_deg)
    pts = [np.zeros(3)]
    d0 = rng.normal(size=3)
    d0 /= np.linalg.norm(d0)
    pts.append(pts[0] + bond * d0)
    buf = np.zeros((n_backbone, 3))  # pts as an array (rows past len(pts) are stale)
    buf[:2] = pts
    restarts = 0
    while len(pts) < n_backbone:
        ok = False
        if restarts > 50:  # dense packing: relax the exclusion distance instead of looping
            min_dist *= 0.9
            restarts = 0
        for _ in range(max_tries):
            prev = pts[-1] - pts[-2]
            prev /= np.linalg.norm(prev)
            perp = np.cross(prev, rng.normal(size=3))
            perp /= np.linalg.norm(perp)
            phi = rng.uniform(0, 2 * math.pi)
            perp = perp * math.cos(phi) + np.cross(prev, perp) * math.sin(phi)
            d = math.cos(math.pi - theta) * prev + math.sin(math.pi - theta) * perp
            cand = pts[-1] + bond * d
            if np.linalg.norm(cand) > radius:
                continue
            arr = buf[:len(pts) - 2]
            if len(arr) and np.min(np.linalg.norm(arr - cand, axis=1)) < min_dist:
                continue
            buf[len(pts)] = cand
            pts.append(cand)
            ok = True
            break
        if not ok:  # restart the walk from a shorter prefix
            del pts[max(2, len(pts) - 20):]
            restarts += 1
    return np.asarray(pts)


def chain_water_system(n_chain=2000, n_waters=30000, seed=1, radius=30.0, box=None, temperature=300.0,
                       n_sigma_bins=8, n_eps_bins=8, h_angles=True):
    """Solvated synthetic chain: every third atom is a hydrogen bonded (SHAKE pair, 1.09 A) to
    the preceding backbone atom; backbone bonds 1.53 A / 310, angles 111 deg / 63 (E = k(x-x0)^2,
    ForceField.cpp:108-177), on every bonded triple: backbone ones and, with h_angles, both
    backbone neighbour - parent - H ones.  Without them a hydrogen is a free rotor on its
    constraint sphere that can swing onto its (LJ-excluded) 1-3 neighbours; at 2 fs such a
    chain blows up within tens of steps in FP64 as in FP32.  Charges ~ N(0, 0.25) shifted to zero net; sigma ~ U(2.5, 3.8),
    epsilon ~ U(0.02, 0.2) binned into n_sigma_bins x n_eps_bins LJ types with Lorentz-Berthelot
    mixing, or, with n_sigma_bins=None, one LJ type per chain atom with its own sigma and
    epsilon (exact Lorentz-Berthelot mixing over an (n_chain + 2)^2 table).  Waters within 2.4 A
    of the solute are removed.  Exclusions: 1-2, 1-3 and 1-4 pairs."""
    rng = np.random.default_rng(seed)
    n_h = n_chain // 3
    n_bb = n_chain - n_h
    bb = _saw_chain(rng, n_bb, radius)
    # atom order: for k-th H, insert after its parent backbone atom
    order = []
    parent_of_h = {}
    bb_index = []
    idx = 0
    for b in range(n_bb):
        bb_index.append(idx)
        idx += 1
        if len(parent_of_h) < n_h and (b % 2 == 1):
            parent_of_h[idx] = idx - 1
            idx += 1
    while len(parent_of_h) < n_h:  # if the chain is short, attach remaining H at the end
        parent_of_h[idx] = bb_index[len(parent_of_h) % n_bb]
        idx += 1
    n_c = idx
    crd_c = np.zeros((n_c, 3))
    crd_c[bb_index] = bb
    pos_of_bb = {idx: k for k, idx in enumerate(bb_index)}
    placed = list(bb_index)
    is_placed = np.zeros(n_c, bool)
    is_placed[bb_index] = True
    for h, p in parent_of_h.items():
        # start on the outer bisector of the parent's backbone angle; keep the direction that
        # leaves the H farthest from every other chain atom
        k = pos_of_bb[p]
        v0 = np.zeros(3)
        nbs = [kk for kk in (k - 1, k + 1) if 0 <= kk < n_bb]
        for kk in nbs:
            d = bb[k] - bb[kk]
            v0 += d / np.linalg.norm(d)
        if len(nbs) == 1:
            # a chain end: 111 deg from its one bond (along the bond the angle would be 180 deg,
            # where the angle force's 1 / sin(theta) turns rounding into force)
            d = v0 / np.linalg.norm(v0)
            u = np.cross(d, rng.normal(size=3))
            u /= np.linalg.norm(u)
            v0 = math.cos(math.radians(69.0)) * d + math.sin(math.radians(69.0)) * u
        if np.linalg.norm(v0) < 1e-6:
            v0 = rng.normal(size=3)
        best, best_d = None, -1.0
        # every candidate lies 1.09 A from the parent, so only placed atoms within 8 A of the
        # parent can be a candidate's nearest one (the backbone neighbours are ~2.5 A away)
        near = is_placed.copy()
        near[p] = False
        others = crd_c[near]
        others = others[np.einsum("ij,ij->i", others - crd_c[p], others - crd_c[p]) < 64.0]
        for t in range(64):
            v = v0 / np.linalg.norm(v0) if t == 0 else v0 / np.linalg.norm(v0) + 0.8 * rng.normal(size=3)
            v /= np.linalg.norm(v)
            cand = crd_c[p] + 1.09 * v
            dmin = math.sqrt(np.min(((others - cand) ** 2).sum(1))) if len(others) else 9.0
            if dmin > best_d:
                best, best_d = cand, dmin
            if dmin >= 2.6:
                break
        crd_c[h] = best
        placed.append(h)
        is_placed[h] = True
    sig = rng.uniform(2.5, 3.8, n_c)
    eps = rng.uniform(0.02, 0.2, n_c)
    lj_types = [(SIGMA_O, EPS_O), (0.0, 0.0)]
    if n_sigma_bins is None:
        lj_types += [(float(a), float(b)) for a, b in zip(sig, eps)]
        type_c = 2 + np.arange(n_c)
    else:
        sb = np.minimum((sig - 2.5) / 1.3 * n_sigma_bins, n_sigma_bins - 1).astype(int)
        eb = np.minimum((eps - 0.02) / 0.18 * n_eps_bins, n_eps_bins - 1).astype(int)
        for i in range(n_sigma_bins):
            for j in range(n_eps_bins):
                lj_types.append((2.5 + (i + 0.5) * 1.3 / n_sigma_bins, 0.02 + (j + 0.5) * 0.18 / n_eps_bins))
        type_c = 2 + sb * n_eps_bins + eb
    q = rng.normal(0.0, 0.25, n_c)
    q -= q.mean()
    mass_c = np.where(np.isin(np.arange(n_c), list(parent_of_h.keys())), M_H, 12.011)
    box = float(box if box is not None else water_box_side(n_waters + n_chain / 3.0))
    # waters on a lattice filling the box, solute at the centre, then overlap removal
    w = water_positions(rng, n_waters, box, jitter=0.3).reshape(n_waters, 3, 3) - 0.5 * box
    # a water goes when one of its atoms lies within 2.4 A of a solute atom; only the atom pairs
    # a k-d tree finds within 2.5 A can be that close, and those are measured exactly
    from scipy.spatial import cKDTree
    wa = w.reshape(-1, 3)
    hits = cKDTree(crd_c).query_ball_point(wa, 2.5)
    close = np.zeros(n_waters, bool)
    for k, js in enumerate(hits):
        if js and np.sqrt(((crd_c[js] - wa[k]) ** 2).sum(1)).min() < 2.4:
            close[k // 3] = True
    w = w[~close]
    nw = len(w)
    crd = np.concatenate([crd_c, w.reshape(-1, 3)]) + 0.5 * box
    n = len(crd)
    charge = np.concatenate([q, np.tile([Q_O, Q_H, Q_H], nw)])
    mass = np.concatenate([mass_c, np.tile([M_O, M_H, M_H], nw)])
    atom_type = np.concatenate([type_c, np.tile([0, 1, 1], nw)])
    bonds = [(bb_index[i], bb_index[i + 1], 310.0, 1.53) for i in range(n_bb - 1)]
    angles = [(bb_index[i], bb_index[i + 1], bb_index[i + 2], 63.0, math.radians(111.0)) for i in range(n_bb - 2)]
    if h_angles:  # hold each hydrogen's direction: backbone neighbour - parent - H
        for h, p in sorted(parent_of_h.items()):
            k = pos_of_bb[p]
            for kk in (k - 1, k + 1):
                if 0 <= kk < n_bb:
                    angles.append((bb_index[kk], p, h, 63.0, math.radians(111.0)))
    bonds = np.array(bonds, dtype=[("a1", "<i4"), ("a2", "<i4"), ("k", "<f8"), ("r0", "<f8")])
    angles = np.array(angles, dtype=[("a1", "<i4"), ("a2", "<i4"), ("a3", "<i4"), ("k", "<f8"), ("t0", "<f8")])
    # 1-2, 1-3 and 1-4 pairs are excluded from the pair list (the reference's "nb15off")
    adj = {i: set() for i in range(n_c)}
    for b in bonds:
        adj[int(b["a1"])].add(int(b["a2"]))
        adj[int(b["a2"])].add(int(b["a1"]))
    for h, p in parent_of_h.items():
        adj[h].add(p)
        adj[p].add(h)
    excl = set()
    for i in range(n_c):
        frontier, seen = {i}, {i}
        for _ in range(3):
            frontier = {j for f in frontier for j in adj[f]} - seen
            seen |= frontier
        for j in seen:
            if j > i:
                excl.add((i, j))
    excl = np.array(sorted(excl), np.int64).reshape(-1, 2)
    excl = np.concatenate([excl, _water_exclusions(n_c, nw)])
    pairs = (np.array([(p, h) for h, p in sorted(parent_of_h.items())], np.int32),
             np.full(len(parent_of_h), 1.09))
    trios = _water_trios(n_c, nw)
    vel = _maxwell(rng, mass, temperature)
    vel -= (mass[:, None] * vel).sum(0) / mass.sum()
    groups = {"names": ["solute", "solvent"],
              "atoms": [np.arange(n_c, dtype=np.int32), np.arange(n_c, n, dtype=np.int32)]}
    s = _assemble(crd, vel, box, charge, mass, atom_type, lj_types, bonds, angles, excl, pairs, trios, groups)
    s["meta"] = {"kind": "chain_water", "n_chain": n_c, "n_waters": nw, "seed": seed, "box": box}
    return s


def poisson_job_stream(n_jobs=256, seed=3, lo=500, hi=10000, mean_interarrival_s=0.05):
    """Serving workload: water counts log-uniform in [lo, hi], Poisson arrival times."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), n_jobs)).astype(int)
    arrivals = np.cumsum(rng.exponential(mean_interarrival_s, n_jobs))
    return [{"job": i, "n_waters": int(c), "seed": 1000 + i, "arrival_s": float(t)}
            for i, (c, t) in enumerate(zip(counts, arrivals))]


def mcmd_polynomial(e_mean, e_sd, seed, temperature=300.0, order=6):
    """V-McMD parameters for one walker: a seeded order-`order` polynomial for d lnP / dE over
    [mean - 4 sd, mean + 4 sd], in powers of E as the reference's virtual-state files give it
    (Extend.cpp:178-203, where the factor is R T * sum c_i E^i with E clamped to the range).
    In the scaled variable x = (E - mean) / (4 sd) the coefficients are 1/(R T) for x^0 and
    U(-0.02, 0.02)/(R T) for the others, so R T dlnP/dE stays near 1 over the range."""
    rng = np.random.default_rng(seed)
    const_k = KB_KCAL * temperature
    lo, hi = e_mean - 4.0 * e_sd, e_mean + 4.0 * e_sd
    half = 0.5 * (hi - lo)
    a = np.zeros(order + 1)
    a[0] = 1.0 / const_k
    a[1:] = rng.uniform(-0.02, 0.02, order) / const_k
    c = np.zeros(order + 1)
    for k in range(order + 1):
        for i in range(k + 1):
            c[i] += a[k] * math.comb(k, i) * (-e_mean) ** (k - i) / half ** k
    return {"coef": c.tolist(), "lambda_low": lo, "lambda_high": hi, "temperature": temperature}


def vmcmd_ladder(e_mean, e_sd, seed, n_vs=4, interval=10, temperature=300.0, order=6, prob=0.5, e_start=None):
    """A V-McMD section for one walker, in the layout of the .cls "extended" section (cls_io;
    Read::load_ls_vmcmd, Read.cpp:521-560): n_vs windows over [mean - 4 sd, mean + 4 sd], each
    2 / (n_vs + 1) of the range wide, so that neighbours overlap by half a window; each window has
    its own seeded polynomial (mcmd_polynomial over the window); moves to a neighbour are tried
    with probability `prob` (0 off the ends of the ladder).  init_vs (1-based, as in the file) is
    the window whose centre lies nearest e_start, or the middle one."""
    lo, hi = e_mean - 4.0 * e_sd, e_mean + 4.0 * e_sd
    width = 2.0 * (hi - lo) / (n_vs + 1)
    states = []
    for v in range(n_vs):
        a = lo + 0.5 * width * v
        b = a + width
        poly = mcmd_polynomial(0.5 * (a + b), width / 8.0, seed=seed * 31 + v, temperature=temperature, order=order)
        states.append(dict(order=order, lambda_low=a, lambda_high=b, prob_low=0.0 if v == 0 else prob,
                           prob_high=0.0 if v == n_vs - 1 else prob, coef=poly["coef"], alpha_low=0.0,
                           alpha_high=0.0))
    init = n_vs // 2
    if e_start is not None:
        init = int(np.argmin([abs(0.5 * (x["lambda_low"] + x["lambda_high"]) - e_start) for x in states]))
    return {"n_vs": n_vs, "interval": interval, "temperature": temperature, "states": states,
            "init_vs": 1 + init, "seed": seed}
