"""The JSON front-end and the geometry sanity report (sysmat_b200.geometry_json)
against the reference's json_to_dat.py and check_geometry_sanity.py, whose
outputs on the same inputs are stored in tests/golden/geometry_json_reference.npz
(tests/golden/make_golden.py json runs the reference scripts)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import sysmat_b200
from helpers import GOLDEN
from sysmat_b200 import configs, geometry_json

CASES = ("annotated", "two_plates", "tiny_rot")


@pytest.fixture(scope="module")
def ref():
    return np.load(os.path.join(GOLDEN, "geometry_json_reference.npz"))


@pytest.mark.parametrize("case", CASES)
def test_tables_equal_the_reference_converter(ref, case):
    cfg = json.loads(str(ref["json_" + case]))
    got = geometry_json.tables_from_json(cfg)
    for key, arr in zip(("collimator", "detector", "image", "physics"), got):
        want = ref["%s_%s" % (key, case)]
        assert arr.dtype == np.float32 and arr.shape == want.shape and np.array_equal(arr, want), key


def test_broken_inputs_give_the_reference_messages(ref):
    for text, msg in zip(ref["broken_json"], ref["broken_msg"]):
        with pytest.raises(geometry_json.GeometryJsonError) as e:
            geometry_json.tables_from_json(json.loads(str(text)))
        assert "ERROR: " + str(e.value) == str(msg)


@pytest.mark.parametrize("case", CASES + ("shipped",))
def test_sanity_report_prints_what_the_reference_prints(ref, case):
    if case == "shipped":
        z = np.load(os.path.join(GOLDEN, "pe_shipped_params.npz"))
        col, det, img = z["collimator"], z["detector"], z["image"]
    else:
        col, det, img = (ref["%s_%s" % (k, case)] for k in ("collimator", "detector", "image"))
    text = geometry_json.sanity_text(geometry_json.sanity_report(col, det, img))
    want = str(ref["sanity_" + case])
    want = want[:want.index("=== Paper expectation")].rstrip("\n") + "\n"
    assert text == want


def test_seeded_workloads_round_trip_and_validate(tmp_path):
    for p in (configs.two_plates_small(), configs.pe_small(), configs.tiny(seed=4, rotated=True)):
        cfg = geometry_json.params_to_json(p)
        q = geometry_json.params_from_json(json.loads(json.dumps(cfg)), p.sv, p.sc)
        assert q.n_crystals == p.n_crystals and q.n_holes == p.n_holes and q.grid == p.grid
        n_col, n_det = 100 + 9 * p.n_holes, 1 + 12 * p.n_crystals
        assert np.array_equal(q.collimator[:n_col], p.collimator[:n_col])
        assert np.array_equal(q.detector[:n_det], p.detector[:n_det])
        assert np.array_equal(q.image[:12], p.image[:12]) and np.array_equal(q.physics[:10], p.physics[:10])


def test_command_line_writes_verifies_and_reports(tmp_path):
    p = configs.two_plates_small()
    path = tmp_path / "g.json"
    path.write_text(json.dumps(geometry_json.params_to_json(p)))
    env = dict(os.environ, PYTHONPATH=os.path.dirname(os.path.dirname(sysmat_b200.__file__)))
    r = subprocess.run([sys.executable, "-m", "sysmat_b200.geometry_json", str(path), "--outdir", str(tmp_path),
                        "--prefix", "Params", "--verify", "--sanity"], capture_output=True, text=True, env=env,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert "'crystals': 108" in r.stdout and "OK: FOV entirely in front of plate" in r.stdout
    back = sysmat_b200.params.Params.read_dat(str(tmp_path))
    assert back.n_crystals == p.n_crystals and back.n_holes == p.n_holes
    # a detector record that the library rejects: --verify reports it and exits 2
    cfg = geometry_json.params_to_json(p)
    cfg["detector"]["bins"][4]["width_mm"] = 0.0
    path.write_text(json.dumps(cfg))
    r = subprocess.run([sys.executable, "-m", "sysmat_b200.geometry_json", str(path), "--outdir", str(tmp_path),
                        "--verify"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 2 and "crystal 4" in r.stdout
    del cfg["image"]["num_voxel_z"]
    path.write_text(json.dumps(cfg))
    r = subprocess.run([sys.executable, "-m", "sysmat_b200.geometry_json", str(path), "--outdir", str(tmp_path)],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 1 and "ERROR: Missing key 'num_voxel_z' in image" in r.stderr
