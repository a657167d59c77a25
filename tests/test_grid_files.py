"""Grid files in the reference's format, host side (no GPU): the headers of
the reference's own grid files (tests/golden/grid_files/, written by
MakeGrid through WriteVDWGrid / WriteCoulombGrid, src/grids.c:692-875) as
rgpu_grid_read_file_header reads them, the file paths the reference gives
them (src/grids.c:716-723, :841-853), and the checks that turn a damaged
file into an error code."""
import os
import shutil

import pytest

from raspa2_b200 import native

from golden_cases import HERE, load

FILES = os.path.join(HERE, "grid_files")


@pytest.fixture(scope="module")
def case():
    return load("grid_co2_files")


@pytest.mark.parametrize("kind", ["C_co2", "O_co2", "coulomb"])
def test_header_of_reference_file(case, kind):
    coulomb = kind == "coulomb"
    h = native.grid_file_header(os.path.join(FILES, case["files"][kind]), coulomb=coulomb).as_dict()
    ref = case["meta"][kind]
    for k in ("spacing", "n", "size", "shift", "delta", "cell", "ncell"):
        assert h[k] == ref[k], (k, h[k], ref[k])
    if coulomb:
        assert h["ewald_precision"] == ref["ewald_precision"]


def test_paths_are_the_reference_paths(case):
    m = case["meta"]["coulomb"]
    fw = case["files"]["C_co2"].split("_C_co2")[0]
    for kind, rel in case["reference_paths"].items():
        if kind == "coulomb":
            p = native.grid_file_path("/raspa", "Local", fw, case["spacing"], None, unit_cells=m["ncell"])
        else:
            p = native.grid_file_path("/raspa", "Local", fw, case["spacing"], kind, shifted=True)
        assert p == "/raspa/" + rel


def test_truncated_file_is_an_error(case, tmp_path):
    src = os.path.join(FILES, case["files"]["C_co2"])
    bad = tmp_path / "short.grid"
    with open(src, "rb") as fh:
        bad.write_bytes(fh.read()[:-4])
    with pytest.raises(native.NativeError, match="error -5"):
        native.grid_file_header(str(bad))


def test_kind_mismatch_is_an_error(case, tmp_path):
    # a VDW file read as a Coulomb file has 8 bytes of planes too few
    src = os.path.join(FILES, case["files"]["C_co2"])
    with pytest.raises(native.NativeError, match="error -5"):
        native.grid_file_header(src, coulomb=True)
    with pytest.raises(native.NativeError, match="error -5"):
        native.grid_file_header(str(tmp_path / "missing.grid"))


def test_path_buffer_too_small_is_an_error():
    import ctypes as C
    buf = C.create_string_buffer(16)
    rc = native.load().rgpu_grid_file_path(buf, C.c_size_t(16), b"/raspa", b"Local", b"fw", C.c_double(0.1),
                                           b"CH4_sp3", C.c_int(1), None)
    assert rc == native.RGPU_E_INVALID


def test_copied_file_reads_the_same(case, tmp_path):
    src = os.path.join(FILES, case["files"]["coulomb"])
    dst = tmp_path / "copy.grid"
    shutil.copyfile(src, dst)
    assert native.grid_file_header(str(dst), True).as_dict() == native.grid_file_header(src, True).as_dict()
