"""Host-side checks of the product that need no GPU: the C ABI library loads and
exports every function include/*.h declares, the binding declares prototypes
for all of them, and the Params layout round-trips through .dat files."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import sysmat_b200
from sysmat_b200 import configs
from sysmat_b200.params import Params

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return names


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    assert {"PESysMatGen", "scatter"} <= names
    assert {"sm_context_create", "sm_geometry_create", "sm_pe_compute", "sm_last_error"} <= names


def test_library_exports_every_declared_symbol():
    lib = sysmat_b200.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, "not exported: %s" % missing
    assert set(declared_functions()) <= set(sysmat_b200.PROTOTYPES)


def test_shim_libraries_export_scatter_variants():
    libdir = os.path.dirname(sysmat_b200.LIB_PATH)
    for name in ("libsysmat_b200_scatter_crystal.so", "libsysmat_b200_scatter_collimator.so"):
        path = os.path.join(libdir, name)
        if not os.path.exists(path):
            pytest.skip("scatter shim libraries not built")
        assert hasattr(ctypes.CDLL(path), "scatter")


def test_version_and_error_without_gpu():
    lib = sysmat_b200.lib()
    assert b"sm_100a" in lib.sm_version()
    h = ctypes.c_void_p()
    rc = lib.sm_context_create(9999, ctypes.byref(h))
    assert rc != 0 and lib.sm_last_error()


@pytest.mark.parametrize("factory", [configs.pe_small, configs.tiny, configs.two_plates_small])
def test_params_dat_roundtrip(tmp_path, factory):
    p = factory()
    p.write_dat(str(tmp_path))
    q = Params.read_dat(str(tmp_path))
    assert np.array_equal(p.collimator[:80000], q.collimator)
    assert np.array_equal(p.detector[:80000], q.detector[:80000])
    assert np.array_equal(p.image, q.image) and np.array_equal(p.physics, q.physics)
    assert q.n_crystals == p.n_crystals and q.n_holes == p.n_holes and q.grid == p.grid


def test_named_workload_shapes():
    s = configs.pe_small()
    assert (s.n_crystals, s.n_voxels, s.n_holes, s.rays_per_entry) == (1024, 4096, 49, 1024)
    l = configs.pe_large()
    assert (l.n_crystals, l.n_voxels, l.n_holes, l.n_plates) == (6400, 131072, 800, 2)
    c = configs.scatter_small()
    assert (c.n_crystals, c.n_voxels) == (2048, 16384)
    assert len(configs.sweep()) == 64
    # plate 0 box and its holes coincide in depth after the FOV shift
    col = s.collimator
    assert col[100 + 1] == -col[12] / 2 and col[100 + 2] == col[12] / 2


def test_seeded_generators_are_deterministic():
    a, b = configs.pe_large(), configs.pe_large()
    assert np.array_equal(a.collimator, b.collimator)
    assert not np.array_equal(configs.pe_large(seed=2).collimator, a.collimator)


# ---- table validation without a device (sm_tables_check) ---------------------

def test_tables_check_reports_the_geometry():
    p = configs.two_plates_small()
    info = sysmat_b200.tables_check(p.collimator, p.detector, p.image, p.physics)
    assert info == {"crystals": p.n_crystals, "holes": p.n_holes, "plates": 2, "grid": p.grid, "rotations": 1}


def test_tables_check_rejects_truncated_tables():
    p = configs.tiny()
    n = p.n_crystals
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.tables_check(p.collimator, p.detector[:1 + 12 * (n - 3)], p.image)
    assert e.value.code == -2 and "%d crystals need %d detector floats" % (n, 1 + 12 * n) in str(e.value)
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.tables_check(p.collimator[:100 + 9 * (p.n_holes - 1)], p.detector, p.image)
    assert e.value.code == -2 and "holes need" in str(e.value)
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.tables_check(p.collimator, p.detector, p.image[:8])
    assert e.value.code == -1 and "image table" in str(e.value)


def test_tables_check_names_bad_fields():
    p = configs.tiny()
    det = p.detector.copy()
    det[1 + 12 * 5 + 4] = 0.0              # crystal 5 width
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.tables_check(p.collimator, det, p.image)
    assert "crystal 5" in str(e.value)
    col = p.collimator.copy()
    col[12] = -1.0                          # plate 0 thickness
    with pytest.raises(sysmat_b200.SysmatError) as e:
        sysmat_b200.tables_check(col, p.detector, p.image)
    assert "plate 0" in str(e.value)


def test_cli_rejects_a_truncated_params_file(tmp_path):
    """The reference's CLI freads into a zeroed buffer and computes with the
    zeros; here a Params_*.dat whose counts need more floats than it holds is
    an error, reported before any device work."""
    p = configs.tiny()
    p.write_dat(str(tmp_path))
    n = p.n_crystals
    p.detector[:1 + 12 * (n - 2)].astype("<f4").tofile(tmp_path / "Params_Detector.dat")
    binary = os.path.join(os.path.dirname(sysmat_b200.LIB_PATH), "..", "..", "bin", "PEGen_CircularHole")
    import subprocess
    r = subprocess.run([binary], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "Params_*.dat" in r.stderr and "%d crystals need" % n in r.stderr
    assert not list(tmp_path.glob("*.sysmat"))
