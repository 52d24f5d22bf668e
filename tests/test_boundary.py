"""The drop-in boundary, checked without a GPU.

* The B200 headers restate the reference Chunk/Settings/State structs at the
  same offsets (golden: the reference headers' own offsets, tests/golden/layout_*.txt).
* The ctypes mirror used by the Python host has the same offsets too.
* Every function declared in include/*.h is exported by the built library,
  and every reference kernel-interface function is among them.
"""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from tealeaf_b200 import abi

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"

REFERENCE_2D_API = """run_set_chunk_data run_set_chunk_state run_kernel_initialise run_kernel_finalise
run_local_halos run_pack_or_unpack run_store_energy run_field_summary run_cg_init run_cg_calc_w
run_cg_calc_ur run_cg_calc_p run_cheby_init run_cheby_iterate run_jacobi_init run_jacobi_iterate
run_ppcg_init run_ppcg_inner_iteration run_copy_u run_calculate_residual run_calculate_2norm
run_finalise""".split()   # 2d/kernel_interface.h:13-71 (22 run_* + diffuse_overload hook)
REFERENCE_3D_API = """run_set_chunk_data run_set_chunk_state run_kernel_initialise run_local_halos
run_pack_or_unpack run_store_energy run_field_summary run_cg_solver_init run_cg_solver_calc_w
run_cg_solver_calc_ur run_cg_solver_calc_p run_cheby_solver_init run_cheby_solver_iterate
run_jacobi_solver_init run_jacobi_solver_iterate run_ppcg_init run_ppcg_inner_iteration
run_solver_copy_u run_calculate_residual run_calculate_2norm run_solver_finalise""".split()  # 3d/kernel_interface.h


def _layout_of_header(dims, tmp_path):
    exe = tmp_path / ("layout%d" % dims)
    cmd = ["/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc", "-DTL_PROBE_B200",
           "-I%s" % (REPO / "include"), str(REPO / "oracle" / "layout_probe.c"), "-o", str(exe)]
    if dims == 3:
        cmd.insert(1, "-DTL3D")
    subprocess.run(cmd, check=True, capture_output=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout


def _parse(text):
    out = {}
    for line in text.splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[1] == "sizeof":
            out[parts[0] + ".sizeof"] = int(parts[2])
        elif len(parts) == 3:
            out[parts[0]] = (int(parts[1]), int(parts[2]))
    return out


@pytest.mark.parametrize("dims", [2, 3])
def test_header_struct_layout_matches_reference(dims, tmp_path):
    header = REPO / "include" / ("tealeaf_b200_%dd.h" % dims)
    if not header.exists():
        pytest.skip("header not present")
    want = _parse((GOLDEN / ("layout_%dd.txt" % dims)).read_text())
    got = _parse(_layout_of_header(dims, tmp_path))
    assert got == want


@pytest.mark.parametrize("dims", [2, 3])
def test_ctypes_mirror_layout_matches_reference(dims):
    want = _parse((GOLDEN / ("layout_%dd.txt" % dims)).read_text())
    types = {"Chunk": abi.Chunk2D if dims == 2 else abi.Chunk3D,
             "Settings": abi.Settings2D if dims == 2 else abi.Settings3D,
             "State": abi.State2D if dims == 2 else abi.State3D}
    for key, val in want.items():
        sname, fname = key.split(".")
        t = types[sname]
        if fname == "sizeof":
            assert C.sizeof(t) == val, key
        else:
            assert getattr(t, fname).offset == val[0], key
            assert getattr(t, fname).size == val[1], key


def _declared(header: Path):
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:void\*?|int)\s+\**(\w+)\s*\(", text, flags=re.M)))


@pytest.mark.parametrize("dims", [2, 3])
def test_library_exports_every_declared_symbol(dims):
    header = REPO / "include" / ("tealeaf_b200_%dd.h" % dims)
    if not header.exists() or not abi.lib_path(dims).exists():
        pytest.skip("suite %dD not built" % dims)
    lib = C.CDLL(str(abi.lib_path(dims)))
    names = _declared(header)
    ref = REFERENCE_2D_API if dims == 2 else REFERENCE_3D_API
    assert set(ref) <= set(names), set(ref) - set(names)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    if dims == 2:
        assert "diffuse_overload" in names


def test_python_loader_refuses_missing_library(tmp_path, monkeypatch):
    monkeypatch.setattr(abi, "LIB_DIR", tmp_path)
    monkeypatch.setattr(abi, "_loaded", {})
    with pytest.raises(FileNotFoundError, match="no CPU fallback"):
        abi.load(2)
