"""The committed kernel instantiation units are exactly what gen_inst.py
writes (one per kernel kind, quadrature type, bra class and ket class, plus a
dispatch unit per kind and bra class), so the build and its generator agree."""
import glob
import os
import shutil
import subprocess
import sys

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "iqcp_b200", "csrc")


def test_instantiation_units_match_generator(tmp_path):
    shutil.copy(os.path.join(CSRC, "gen_inst.py"), tmp_path)
    subprocess.run([sys.executable, "gen_inst.py"], cwd=tmp_path, check=True)
    made = sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / "eri_inst_*.cu")))
    have = sorted(os.path.basename(f) for f in glob.glob(os.path.join(CSRC, "eri_inst_*.cu")))
    assert made == have
    for name in made:
        with open(tmp_path / name) as a, open(os.path.join(CSRC, name)) as b:
            assert a.read() == b.read(), name
    # 21 class pairs x 2 kinds x 2 precisions + 6 dispatch x 2 kinds + 6 store units
    assert len(made) == 21 * 4 + 12 + 6


def test_rys_tables_match_generator(tmp_path):
    """rys_tables.inc is exactly what gen_rys_tables.cpp writes (binary128
    Rys rules and their Chebyshev fits, computed from the Boys moments)."""
    gxx = shutil.which("g++")
    if gxx is None:
        import pytest
        pytest.skip("no g++")
    exe = str(tmp_path / "gen_rys")
    subprocess.run([gxx, "-O2", "-o", exe, os.path.join(CSRC, "gen_rys_tables.cpp"), "-lquadmath"], check=True)
    out = tmp_path / "rys_tables.inc"
    subprocess.run([exe, str(out)], check=True, timeout=900)
    with open(out) as a, open(os.path.join(CSRC, "rys_tables.inc")) as b:
        assert a.read() == b.read()
