"""The generator CLI: --mode getrates --language cuda emits compilable
sm_100a source and the blob the C ABI loads."""
import os
import subprocess
import sys

import pytest

from conftest import REPO, REFERENCE, reference_available
from chemgen_b200 import pack, synthetic
from oracle import oracle


def test_blob_mode_roundtrip(tmp_path):
    yaml_path = tmp_path / "mech.yaml"
    out = tmp_path / "mech.blob"
    # a mechanism file written from the package's own JSON form
    mech = synthetic.h2o2_10sp()
    (tmp_path / "mech.json").write_text(mech.to_json())
    r = subprocess.run([sys.executable, os.path.join(REPO, "generate_chemistry.py"), "--mode", "blob",
                        "--mech", str(tmp_path / "mech.json"), "--output", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.read_bytes() == pack.pack(mech).to_blob()
    assert oracle.check_blob(out.read_bytes()) == 0


@pytest.mark.skipif(not reference_available(), reason="reference mechanism files not present")
@pytest.mark.parametrize("src", [("GRI30/chem.inp", "GRI30/therm.dat"), ("H2_burke/chem.yaml", None)])
def test_getrates_cuda_emits_compilable_source(tmp_path, src):
    mech_file, therm = src
    out = tmp_path / "getrates.cu"
    cmd = [sys.executable, os.path.join(REPO, "generate_chemistry.py"), "--mode", "getrates", "--language", "cuda",
           "--mech", os.path.join(REFERENCE, "ck_files", mech_file), "--output", str(out)]
    if therm:
        cmd += ["--therm", os.path.join(REFERENCE, "ck_files", therm)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    assert "__global__" in text and "cg_gen_fp64" in text and "cg_gen_mixed" in text
    assert oracle.check_blob((tmp_path / "getrates.blob").read_bytes()) == 0
    from chemgen_b200.build import ARCH, FLAGS, nvcc
    obj = tmp_path / "g.o"
    r = subprocess.run([nvcc()] + ARCH + FLAGS + ["-I", os.path.join(REPO, "chemgen_b200", "csrc"), "-c",
                        str(out), "-o", str(obj)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def test_getrates_cuda_from_chemkin_input(tmp_path):
    """--mech chem.inp --therm therm.dat: the Chemkin reader feeds the emitter."""
    from test_chemkin import _inp_text, _species, _therm_text
    (tmp_path / "chem.inp").write_text(_inp_text())
    (tmp_path / "therm.dat").write_text(_therm_text(_species()))
    out = tmp_path / "getrates.cu"
    r = subprocess.run([sys.executable, os.path.join(REPO, "generate_chemistry.py"), "--mode", "getrates",
                        "--language", "cuda", "--mech", str(tmp_path / "chem.inp"), "--therm",
                        str(tmp_path / "therm.dat"), "--output", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    assert "cg_gen_fp64" in text and "cg_gen_mixed" in text
    from chemgen_b200.chemkin import mechanism_from_chemkin
    m = mechanism_from_chemkin(_inp_text(), _therm_text(_species()))
    assert (tmp_path / "getrates.blob").read_bytes() == pack.pack(m).to_blob()


@pytest.mark.parametrize("precision,has64,has32,mask", [("fp64", True, False, 1), ("mixed", False, True, 2),
                                                         ("both", True, True, 3)])
def test_precision_selects_the_generated_kernels(tmp_path, precision, has64, has32, mask):
    from chemgen_b200 import cli
    out = tmp_path / "k.cu"
    src_yaml = tmp_path / "m.json"
    from chemgen_b200 import synthetic
    src_yaml.write_text(synthetic.h2o2_10sp().to_json())
    assert cli.main(["--mode", "getrates", "--mech", str(src_yaml), "--output", str(out), "--language", "cuda",
                     "--precision", precision]) == 0
    text = out.read_text()
    assert ("cg_gen_fp64<<<" in text) == has64 and ("cg_gen_mixed<<<" in text) == has32
    assert f", {mask}u, &launch)" in text
    import json
    from chemgen_b200 import ops
    rec = json.loads((tmp_path / "k.ops.json").read_text())
    assert rec["ns"] == 10 and rec["nr"] == 27 and rec["hbm_bytes_per_point"] == 176
    assert rec["ops_per_point"] == ops.inventory(synthetic.h2o2_10sp())
