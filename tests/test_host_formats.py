"""The reference's host file formats behind the C ABI (no GPU needed):
parameters.txt lookup (src/admin/admin.cpp:53-88), SPS/RPS points
(src/geometry/geometry.cpp:3-47) and raw float32 binaries."""
import numpy as np
import pytest

from fwi3d_b200 import lib

PARAMS = """#------------------------------------------------------------
# Model parameters ------------------------------------------
#------------------------------------------------------------

x_samples = 201
y_samples = 201
z_samples = 81

model_spacing = 25.0                # [m]
 z_samples = 99
# z_samples = 77
time_samples = 2001
time_spacing = 1e-3                 # [s]
time = 5
inv_input_prefix = seismogram_nt2001_nr2601_1000us_shot_
mig_input_folder = ../inputs/data/input_RTM_
path with space = a b  c # comment
noequals
"""


@pytest.fixture()
def pfile(tmp_path):
    p = tmp_path / "parameters.txt"
    p.write_text(PARAMS)
    return p


def test_values_and_inline_comments(pfile):
    assert lib.catch_parameter(pfile, "x_samples") == "201"
    assert lib.catch_parameter(pfile, "model_spacing") == "25.0"
    assert lib.catch_parameter(pfile, "time_spacing") == "1e-3"
    assert lib.catch_parameter(pfile, "inv_input_prefix") == "seismogram_nt2001_nr2601_1000us_shot_"


def test_lines_starting_with_hash_or_space_are_skipped(pfile):
    # " z_samples = 99" starts with a space and "# z_samples" with '#'
    assert lib.catch_parameter(pfile, "z_samples") == "81"


def test_prefix_match_takes_the_first_line_that_starts_with_the_key(pfile):
    # "time" matches "time_samples = 2001" before the later "time = 5"
    assert lib.catch_parameter(pfile, "time") == "2001"


def test_spaces_are_removed_and_missing_keys_are_empty(pfile):
    assert lib.catch_parameter(pfile, "path") == "abc"
    assert lib.catch_parameter(pfile, "absent_key") == ""


def test_line_without_equals_sign(pfile):
    # find("=") is npos, npos + 2 wraps to 1: the value is the line from index 1
    assert lib.catch_parameter(pfile, "noequals") == "oequals"


def test_unreadable_file(tmp_path):
    with pytest.raises(lib.FwiError) as e:
        lib.catch_parameter(tmp_path / "missing.txt", "x")
    assert e.value.code == 6


def test_points(tmp_path):
    f = tmp_path / "SPS.txt"
    f.write_text("# header\n1000.00,1000.00,100.00\n1600.50,1000.00,100.00\n\n2200.00,1250.25,0.00\n")
    p = lib.read_points(f)
    assert p.shape == (3, 3)
    np.testing.assert_allclose(p[1], [1600.5, 1000.0, 100.0])
    np.testing.assert_allclose(p[2], [2200.0, 1250.25, 0.0])


def test_points_as_written_by_numpy(tmp_path):
    pts = np.array([[0.0, 0.0, 10.0], [20.0, 40.0, 10.0]], np.float32)
    f = tmp_path / "RPS.txt"
    np.savetxt(f, pts, fmt="%.2f", delimiter=",")
    np.testing.assert_array_equal(lib.read_points(f), pts)


def test_malformed_points(tmp_path):
    f = tmp_path / "bad.txt"
    f.write_text("1.0,2.0\n")
    with pytest.raises(lib.FwiError):
        lib.read_points(f)


def test_binary_round_trip(tmp_path):
    import ctypes as C
    so = lib.load()
    a = np.random.default_rng(0).standard_normal(1001).astype(np.float32)
    f = str(tmp_path / "x.bin").encode()
    assert so.fwi_write_binary(f, a.ctypes.data_as(C.POINTER(C.c_float)), a.size) == 0
    b = np.empty_like(a)
    assert so.fwi_read_binary(f, b.ctypes.data_as(C.POINTER(C.c_float)), b.size) == 0
    assert np.array_equal(a, b)
    assert np.array_equal(np.fromfile(tmp_path / "x.bin", np.float32), a)
    # asking for more samples than the file holds is an error
    c = np.empty(2000, np.float32)
    assert so.fwi_read_binary(f, c.ctypes.data_as(C.POINTER(C.c_float)), c.size) == 6
