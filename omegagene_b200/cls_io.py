"""Reader / writer for omegagene's binary ".cls" launch-set input (format v.0.52).

The layout follows ``Read::load_launch_set`` and its section loaders
(src/celeste/core/Read.cpp:50-600): a magic number (66261), a version string, thirteen
section sizes in bytes, then the sections in header order.  Atom indices in the bond,
angle, torsion, 1-4, 1-5-exclusion and constraint sections are 0-based; atom types,
LJ type pairs and atom-group members are 1-based (Read.cpp:279, 306, 568).

Torsions, impropers and 1-4 pairs are parsed (``torsions``, ``impros``, ``nb14``) and also kept
as raw bytes; sections the MD path does not use (restraints, VcMD, group coordinates,
potential tables) are kept as raw bytes only, so that a file read and written back is
byte-identical.
"""
import struct

import numpy as np

MAGIC = 66261
VERSION = "v.0.52"
SECTIONS = ("box", "crd", "vel", "topol", "constraint", "settle", "extended", "groups",
            "dist_restraint", "pos_restraint", "extended_vcmd", "group_coord", "pote")


class ClsFormatError(ValueError):
    pass


class _Reader:
    def __init__(self, buf):
        self.b = buf
        self.o = 0

    def i(self, n=None):
        if n is None:
            v = struct.unpack_from("<i", self.b, self.o)[0]
            self.o += 4
            return v
        v = np.frombuffer(self.b, dtype="<i4", count=n, offset=self.o).astype(np.int32)
        self.o += 4 * n
        return v

    def d(self, n=None):
        if n is None:
            v = struct.unpack_from("<d", self.b, self.o)[0]
            self.o += 8
            return v
        v = np.frombuffer(self.b, dtype="<f8", count=n, offset=self.o).astype(np.float64)
        self.o += 8 * n
        return v

    def rec(self, dtype, n):
        v = np.frombuffer(self.b, dtype=dtype, count=n, offset=self.o).copy()
        self.o += np.dtype(dtype).itemsize * n
        return v

    def raw(self, n):
        v = bytes(self.b[self.o:self.o + n])
        self.o += n
        return v


BOND = np.dtype([("a1", "<i4"), ("a2", "<i4"), ("k", "<f8"), ("r0", "<f8")])
ANGLE = np.dtype([("a1", "<i4"), ("a2", "<i4"), ("a3", "<i4"), ("k", "<f8"), ("t0", "<f8")])
LJ = np.dtype([("t1", "<i4"), ("t2", "<i4"), ("p6", "<f8"), ("p12", "<f8")])
# Read::load_ls_tpl torsion / improper records (Read.cpp:379-420): 4 atoms, energy, overlaps,
# symmetry, phase, 1-4 flag; packed, 44 bytes
DIHED = np.dtype([("a", "<i4", 4), ("ene", "<f8"), ("overlaps", "<i4"), ("symmetry", "<i4"), ("phase", "<f8"),
                  ("flag14", "<i4")])
# 1-4 pair records (Read.cpp:428-439): 2 atoms, 2 atom types (1-based), two scale factors
NB14 = np.dtype([("a1", "<i4"), ("a2", "<i4"), ("t1", "<i4"), ("t2", "<i4"), ("f1", "<f8"), ("f2", "<f8")])


def _parse_records(raw, dtype, what):
    r = _Reader(raw)
    n = r.i() if len(raw) >= 4 else 0
    if len(raw) != 4 + dtype.itemsize * n:
        raise ClsFormatError("inconsistent %s section" % what)
    return r.rec(dtype, n)


def _parse_topol(b, n_atoms):
    r = _Reader(b)
    t = {}
    n = r.i()
    if n != n_atoms:
        raise ClsFormatError("topology atom count %d != %d" % (n, n_atoms))
    t["charge"] = r.d(n)
    t["mass"] = r.d(n)
    t["atom_type"] = r.i(n) - 1
    size_lj = r.i()
    t["n_lj_types"] = r.i()
    n_pairs = r.i()
    t["lj_pairs"] = r.rec(LJ, n_pairs)
    if size_lj != 8 + LJ.itemsize * n_pairs:
        raise ClsFormatError("inconsistent LJ section")
    size_hps = r.i()
    t["lj_hps_raw"] = r.raw(size_hps)
    size_bond = r.i()
    nb = r.i()
    t["bonds"] = r.rec(BOND, nb)
    size_angle = r.i()
    na = r.i()
    t["angles"] = r.rec(ANGLE, na)
    for key in ("torsions_raw", "impros_raw", "nb14_raw"):
        size = r.i()
        t[key] = r.raw(size)
    t["torsions"] = _parse_records(t["torsions_raw"], DIHED, "torsion")
    t["impros"] = _parse_records(t["impros_raw"], DIHED, "improper")
    nb14 = _parse_records(t["nb14_raw"], NB14, "1-4")
    # MmSystem::set_nb14_param takes (coeff_vdw, coeff_ele) but Read.cpp:438 passes the record's
    # second factor first: the factor the reference applies to the 1-4 van der Waals term is the
    # record's second one, and the one it applies to the 1-4 electrostatics the first.
    t["nb14"] = {"atoms": np.stack([nb14["a1"], nb14["a2"]], 1).astype(np.int32),
                 "types": (np.stack([nb14["t1"], nb14["t2"]], 1) - 1).astype(np.int32),
                 "coeff_vdw": nb14["f2"].copy(), "coeff_ele": nb14["f1"].copy()}
    size_15 = r.i()
    n15 = r.i()
    t["nb15off_pairs"] = r.i(2 * n15).reshape(n15, 2)
    if r.o != len(b):
        raise ClsFormatError("trailing bytes in topology section")
    return t


def _parse_constraint(b):
    r = _Reader(b)
    n2, n3, n4 = r.i(), r.i(), r.i()
    c = {}
    p = r.rec(np.dtype([("a", "<i4", 2), ("d", "<f8")]), n2)
    c["pair_atoms"], c["pair_dist"] = p["a"].copy(), p["d"].copy()
    t = r.rec(np.dtype([("a", "<i4", 3), ("d", "<f8", 3)]), n3)
    c["trio_atoms"], c["trio_dist"] = t["a"].copy(), t["d"].copy()
    q = r.rec(np.dtype([("a", "<i4", 4), ("d", "<f8", 6)]), n4)
    c["quad_atoms"], c["quad_dist"] = q["a"].copy(), q["d"].copy()
    return c


def _parse_vmcmd(b):
    r = _Reader(b)
    v = {"n_vs": r.i(), "interval": r.i(), "temperature": r.d(), "states": []}
    for _ in range(v["n_vs"]):
        order = r.i()
        lam_lo, lam_hi, p_lo, p_hi = r.d(), r.d(), r.d(), r.d()
        coef = r.d(order + 1)
        a_lo, a_hi = r.d(), r.d()
        v["states"].append(dict(order=order, lambda_low=lam_lo, lambda_high=lam_hi, prob_low=p_lo,
                                prob_high=p_hi, coef=coef, alpha_low=a_lo, alpha_high=a_hi))
    v["init_vs"] = r.i()
    v["seed"] = r.i()
    return v


def _parse_groups(b):
    r = _Reader(b)
    n = r.i()
    names, counts = [], []
    for _ in range(n):
        ln = r.i()
        names.append(r.raw(ln).split(b"\0")[0].decode())
        counts.append(r.i())
    groups = [r.i(c) - 1 for c in counts]
    return {"names": names, "atoms": groups}


def read_cls(path):
    """Returns a dict with numpy arrays; raises ClsFormatError on a malformed file."""
    with open(path, "rb") as f:
        buf = f.read()
    r = _Reader(buf)
    if len(buf) < 8 or r.i() != MAGIC:
        raise ClsFormatError("%s: bad magic number" % path)
    ln = r.i()
    version = r.raw(ln).split(b"\0")[0].decode()
    if version != VERSION:
        raise ClsFormatError("%s: version %s, %s required" % (path, version, VERSION))
    sizes = dict(zip(SECTIONS, [r.i() for _ in SECTIONS]))
    raw = {}
    for s in SECTIONS:
        if sizes[s] < 0 or r.o + sizes[s] > len(buf):
            raise ClsFormatError("%s: section %s runs past the end of the file" % (path, s))
        raw[s] = r.raw(sizes[s])
    if r.o != len(buf):
        raise ClsFormatError("%s: trailing bytes" % path)
    out = {"version_len": ln, "raw": raw}
    # Read::load_launch_set adds 3 degrees of freedom when a position-restraint section is
    # present, whatever it holds (Read.cpp:90-93)
    out["dof_extra"] = 3 if len(raw["pos_restraint"]) > 0 else 0
    if raw["box"]:
        out["pbc_val"] = np.frombuffer(raw["box"], dtype="<f8").copy()
    if raw["crd"]:
        rr = _Reader(raw["crd"])
        n = rr.i()
        out["n_atoms"] = n
        out["crd"] = rr.d(3 * n).reshape(n, 3)
    if raw["vel"]:
        rr = _Reader(raw["vel"])
        n = rr.i()
        out["vel"] = rr.d(3 * n).reshape(n, 3)
    if raw["topol"]:
        out["topol"] = _parse_topol(raw["topol"], out["n_atoms"])
    if raw["constraint"]:
        out["constraint"] = _parse_constraint(raw["constraint"])
    if raw["settle"]:
        out["settle"] = _parse_constraint(raw["settle"])
    if raw["extended"]:
        out["vmcmd"] = _parse_vmcmd(raw["extended"])
    if raw["groups"]:
        out["groups"] = _parse_groups(raw["groups"])
    return out


# ------------------------------------------------------------------ writer

def _pack_records(t, key, dtype):
    """A dihedral section: the parsed records when present, else the raw bytes (count 0 if none)."""
    if key in t and t[key] is not None:
        arr = np.asarray(t[key], dtype)
        return struct.pack("<i", len(arr)) + arr.tobytes()
    return t.get(key + "_raw", struct.pack("<i", 0))


def _pack_nb14(t):
    """The 1-4 section from the parsed pairs (the reader swapped the record's two factors into
    coeff_vdw = second, coeff_ele = first; they are written back in record order), else raw."""
    nb = t.get("nb14")
    if nb is None:
        return t.get("nb14_raw", struct.pack("<i", 0))
    atoms = np.asarray(nb["atoms"], np.int64).reshape(-1, 2)
    rec = np.zeros(len(atoms), NB14)
    rec["a1"], rec["a2"] = atoms[:, 0], atoms[:, 1]
    types = np.asarray(nb["types"], np.int64).reshape(-1, 2) + 1
    rec["t1"], rec["t2"] = types[:, 0], types[:, 1]
    rec["f1"], rec["f2"] = nb["coeff_ele"], nb["coeff_vdw"]
    return struct.pack("<i", len(rec)) + rec.tobytes()


def _pack_topol(t, n_atoms):
    parts = [struct.pack("<i", n_atoms),
             np.asarray(t["charge"], "<f8").tobytes(),
             np.asarray(t["mass"], "<f8").tobytes(),
             (np.asarray(t["atom_type"], np.int64) + 1).astype("<i4").tobytes()]
    lj = np.asarray(t["lj_pairs"], LJ)
    body = struct.pack("<ii", int(t["n_lj_types"]), len(lj)) + lj.tobytes()
    parts += [struct.pack("<i", len(body)), body]
    hps = t.get("lj_hps_raw", b"")
    parts += [struct.pack("<i", len(hps)), hps]
    for key, dt in (("bonds", BOND), ("angles", ANGLE)):
        arr = np.asarray(t.get(key, np.zeros(0, dt)), dt)
        body = struct.pack("<i", len(arr)) + arr.tobytes()
        parts += [struct.pack("<i", len(body)), body]
    for key, body in (("torsions", _pack_records(t, "torsions", DIHED)), ("impros", _pack_records(t, "impros", DIHED)),
                      ("nb14", _pack_nb14(t))):
        parts += [struct.pack("<i", len(body)), body]
    p15 = np.asarray(t["nb15off_pairs"], "<i4").reshape(-1, 2)
    body = struct.pack("<i", len(p15)) + p15.tobytes()
    parts += [struct.pack("<i", len(body)), body]
    return b"".join(parts)


def _pack_constraint(c):
    pa = np.asarray(c.get("pair_atoms", np.zeros((0, 2))), "<i4").reshape(-1, 2)
    ta = np.asarray(c.get("trio_atoms", np.zeros((0, 3))), "<i4").reshape(-1, 3)
    qa = np.asarray(c.get("quad_atoms", np.zeros((0, 4))), "<i4").reshape(-1, 4)
    pd = np.asarray(c.get("pair_dist", np.zeros(0)), "<f8").reshape(-1)
    td = np.asarray(c.get("trio_dist", np.zeros((0, 3))), "<f8").reshape(-1, 3)
    qd = np.asarray(c.get("quad_dist", np.zeros((0, 6))), "<f8").reshape(-1, 6)
    out = [struct.pack("<iii", len(pa), len(ta), len(qa))]
    rp = np.zeros(len(pa), np.dtype([("a", "<i4", 2), ("d", "<f8")]))
    rp["a"], rp["d"] = pa, pd
    rt = np.zeros(len(ta), np.dtype([("a", "<i4", 3), ("d", "<f8", 3)]))
    rt["a"], rt["d"] = ta, td
    rq = np.zeros(len(qa), np.dtype([("a", "<i4", 4), ("d", "<f8", 6)]))
    rq["a"], rq["d"] = qa, qd
    return b"".join(out + [rp.tobytes(), rt.tobytes(), rq.tobytes()])


def _pack_vmcmd(v):
    out = [struct.pack("<iid", len(v["states"]), int(v["interval"]), float(v["temperature"]))]
    for s in v["states"]:
        coef = np.asarray(s["coef"], "<f8")
        out.append(struct.pack("<idddd", len(coef) - 1, s["lambda_low"], s["lambda_high"],
                               s["prob_low"], s["prob_high"]))
        out.append(coef.tobytes())
        out.append(struct.pack("<dd", s.get("alpha_low", 0.0), s.get("alpha_high", 0.0)))
    out.append(struct.pack("<ii", int(v["init_vs"]), int(v["seed"])))
    return b"".join(out)


def _pack_groups(g):
    out = [struct.pack("<i", len(g["names"]))]
    for name, atoms in zip(g["names"], g["atoms"]):
        nb = name.encode() + b"\0"
        out += [struct.pack("<i", len(nb)), nb, struct.pack("<i", len(atoms))]
    for atoms in g["atoms"]:
        out.append((np.asarray(atoms, np.int64) + 1).astype("<i4").tobytes())
    return b"".join(out)


def write_cls(path, s):
    """Writes a launch set.  ``s`` uses the keys produced by read_cls (parsed sections win
    over their raw bytes)."""
    raw = dict(s.get("raw", {}))
    n = int(s["n_atoms"])
    if "pbc_val" in s:
        raw["box"] = np.asarray(s["pbc_val"], "<f8").tobytes()
    raw["crd"] = struct.pack("<i", n) + np.asarray(s["crd"], "<f8").reshape(-1).tobytes()
    if "vel" in s:
        raw["vel"] = struct.pack("<i", n) + np.asarray(s["vel"], "<f8").reshape(-1).tobytes()
    if "topol" in s:
        raw["topol"] = _pack_topol(s["topol"], n)
    if "constraint" in s:
        raw["constraint"] = _pack_constraint(s["constraint"])
    if "settle" in s:
        raw["settle"] = _pack_constraint(s["settle"])
    if "vmcmd" in s:
        raw["extended"] = _pack_vmcmd(s["vmcmd"])
    if "groups" in s:
        raw["groups"] = _pack_groups(s["groups"])
    ver = VERSION.encode() + b"\0"
    hdr = [struct.pack("<i", MAGIC), struct.pack("<i", len(ver)), ver]
    hdr += [struct.pack("<i", len(raw.get(k, b""))) for k in SECTIONS]
    with open(path, "wb") as f:
        f.write(b"".join(hdr))
        for k in SECTIONS:
            f.write(raw.get(k, b""))


HPS = np.dtype([("t1", "<i4"), ("t2", "<i4"), ("cut", "<f8"), ("lam", "<f8")])


def hps_tables(topol):
    """Dense n_types x n_types HPS cutoff and lambda tables from the topology's HPS records
    (Read.cpp:322-334 reads one record per LJ type pair; MmSystem::set_lj_pair_hps_param,
    MmSystem.cpp:320-325, sets both orders, so a later record of a pair wins)."""
    nt = int(topol["n_lj_types"])
    cut = np.zeros((nt, nt), np.float64)
    lam = np.zeros((nt, nt), np.float64)
    raw = topol.get("lj_hps_raw", b"")
    n = min(len(raw) // HPS.itemsize, len(topol["lj_pairs"]))
    rec = np.frombuffer(raw[:n * HPS.itemsize], HPS)
    i, j, k = _last_per_type_pair(rec["t1"], rec["t2"], nt)
    cut[i, j] = cut[j, i] = rec["cut"][k]
    lam[i, j] = lam[j, i] = rec["lam"][k]
    return cut, lam


def _last_per_type_pair(t1, t2, nt):
    """0-based (i, j) and record index of the last record of every unordered type pair among
    1-based records (t1, t2): the record a sequential fill of both orders leaves in place."""
    i = np.asarray(t1, np.int64) - 1
    j = np.asarray(t2, np.int64) - 1
    key = np.minimum(i, j) * nt + np.maximum(i, j)
    rev = key[::-1]
    _, first_in_rev = np.unique(rev, return_index=True)
    k = len(key) - 1 - first_in_rev
    return i[k], j[k], k


def pack_hps(t1, t2, cut, lam):
    """HPS records (1-based types) as the topology section holds them."""
    rec = np.zeros(len(t1), HPS)
    rec["t1"], rec["t2"], rec["cut"], rec["lam"] = t1, t2, cut, lam
    return rec.tobytes()


def lj_tables(topol):
    """Dense n_types x n_types C6/C12 tables from the LJ type-pair records
    (MmSystem::set_lj_pair_param, MmSystem.cpp:313-319)."""
    nt = int(topol["n_lj_types"])
    c6 = np.zeros((nt, nt), np.float64)
    c12 = np.zeros((nt, nt), np.float64)
    rec = topol["lj_pairs"]
    i, j, k = _last_per_type_pair(rec["t1"], rec["t2"], nt)
    c6[i, j] = c6[j, i] = rec["p6"][k]
    c12[i, j] = c12[j, i] = rec["p12"][k]
    return c6, c12


def nb15off_table(n_atoms, pairs, max_nb15off=32):
    """Padded exclusion table as MmSystem::set_nb15off builds it (MmSystem.cpp:478-525):
    each listed pair is entered in both rows unless already present; -1 pads."""
    tab = np.full((n_atoms, max_nb15off), -1, np.int32)
    p = np.asarray(pairs, np.int64).reshape(-1, 2)
    # entries in the sequential order (a1 -> a2, then a2 -> a1, record by record); a repeat of an
    # entry already in its row is skipped, so each row keeps its first occurrences in order
    x = np.stack([p[:, 0], p[:, 1]], 1).reshape(-1)
    y = np.stack([p[:, 1], p[:, 0]], 1).reshape(-1)
    _, first = np.unique(x * max(n_atoms, 1) + y, return_index=True)
    first.sort()
    x, y = x[first], y[first]
    order = np.argsort(x, kind="stable")
    x, y = x[order], y[order]
    start = np.searchsorted(x, np.arange(n_atoms))
    col = np.arange(len(x)) - start[x]
    if len(col) and col.max() >= max_nb15off:
        raise ClsFormatError("more than %d exclusions for atom %d" % (max_nb15off, int(x[np.argmax(col)])))
    tab[x, col] = y
    return tab
