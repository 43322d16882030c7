"""CPU-side checks of the C ABI library and of the host-side logic (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from omegagene_b200 import cls_io, engine, systems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\s*(?:og_status|const char \*)\s*(og_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import __graft_entry__
    __graft_entry__.build()
    lib = ctypes.CDLL(engine.LIB_PATH)
    names = _declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_create_fails_cleanly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = engine.load_library()
    h = ctypes.c_void_p()
    assert lib.og_create(0, ctypes.byref(h)) == engine.OG_ERR_CUDA


def test_parse_run_config_reference_sample():
    txt = """--processor single ;
--integrator leapfrog-presto ;
--cutoff 12.0 ;
--time-step 2.0
--electrostatic zero-dipole ;
--ele-alpha 0 ;
;--thermostat scaling
--thermostat none
--temperature 300 ;
--com-motion cancel ;
--com-cancel-group-name solute
--com-cancel-group-name solvent
--nsgrid-cutoff 13.0
--nsgrid-update-intvl 10
--constraint shake
--const-max-loops 1000
--const-tolerance 0.0000001
--berendsen-tau 0.1
"""
    p = engine.parse_run_config(txt)
    assert p["cutoff"] == 12.0 and p["nsgrid_cutoff"] == 13.0 and p["nsgrid_update_intvl"] == 10
    assert p["thermostat"] == "none" and p["com_cancel_groups"] == ["solute", "solvent"]
    assert p["berendsen_tau"] == pytest.approx(100.0)
    with pytest.raises(ValueError):
        engine.parse_run_config("--integrator langevin")
    with pytest.raises(ValueError):
        engine.parse_run_config("--unknown-key 3")


def test_make_desc_fields():
    s = systems.chain_water_system(300, 400, seed=2, radius=10.0)
    d, keep = engine.make_desc(s, {"nsgrid_update_intvl": 5})
    assert d.n_atoms == s["n_atoms"] and d.nsgrid_update_intvl == 5
    assert d.n_shake_trio == len(s["constraint"]["trio_atoms"])
    assert d.n_shake_pair == len(s["constraint"]["pair_atoms"])
    assert d.n_bonds == len(s["topol"]["bonds"]) and d.n_angles == len(s["topol"]["angles"])
    assert d.n_com_groups == 2


def test_cls_roundtrip_synthetic(tmp_path):
    s = systems.water_system(200, seed=1)
    path = str(tmp_path / "w.cls")
    cls_io.write_cls(path, s)
    r = cls_io.read_cls(path)
    np.testing.assert_array_equal(r["crd"], s["crd"])
    np.testing.assert_array_equal(r["topol"]["atom_type"], s["topol"]["atom_type"])
    np.testing.assert_array_equal(r["constraint"]["trio_atoms"], s["constraint"]["trio_atoms"])
    cls_io.write_cls(str(tmp_path / "w2.cls"), r)
    assert open(path, "rb").read() == open(str(tmp_path / "w2.cls"), "rb").read()


def test_cls_rejects_bad_magic(tmp_path):
    p = tmp_path / "bad.cls"
    p.write_bytes(b"\0" * 64)
    with pytest.raises(cls_io.ClsFormatError):
        cls_io.read_cls(str(p))


def test_celeste_library_exports_the_reference_entry_points():
    """libomegagene_celeste.so defines every cuda_* function include/omegagene_celeste.h declares
    (the reference's CELESTE_GPU entry points), with C linkage."""
    import __graft_entry__
    __graft_entry__.build()
    from omegagene_b200 import build as ogb
    txt = open(os.path.join(ROOT, "include", "omegagene_celeste.h")).read()
    names = re.findall(r"^\s*(?:int|void)\s+(cuda\w+)\s*\(", txt, re.M)
    assert len(names) >= 30
    lib = ctypes.CDLL(ogb.CELESTE_OUT)
    for n in names:
        assert hasattr(lib, n), n
