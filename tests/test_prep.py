"""Pipeline preparation: the reference's RTM input preprocessing on the GPU
against its numpy restatement (oracle/prep_oracle.py), and the setup command
(acquisition files and start model) on CPU."""
import numpy as np
import pytest

import prep_oracle
from fwi3d_b200 import lib, prep


@pytest.mark.gpu
def test_rtm_input_matches_the_reference_script_semantics():
    rng = np.random.default_rng(0)
    nt, nrec = 2001, 2601
    rec = np.stack(np.meshgrid(np.linspace(0, 5000, 51), np.linspace(0, 5000, 51)), -1).reshape(-1, 2)
    rec = np.concatenate([rec, np.zeros((nrec, 1))], 1).astype(np.float32)
    seis = (rng.standard_normal((nrec, nt)) * 1e3).astype(np.float32)   # (nrec, nt) = Fortran [nt, nrec]
    got = lib.prepare_rtm_input(seis, rec, (1600.0, 2200.0), np.float32(1e-3))
    want = prep_oracle.rtm_input(seis.T, 1600.0, 2200.0, rec, 1e-3).T
    ulps = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
    assert ulps.max() <= 1 and np.mean(ulps == 0) > 0.999
    # the taper zeroes nothing after the direct-wave sample and scales by 1/max
    assert np.abs(got).max() <= 1.0 + 1e-6


def test_setup_writes_reference_files(tmp_path):
    nx, ny, nz, dh = 20, 18, 16, 25.0
    true = (1500 + 50 * np.arange(nz)[:, None, None] + np.zeros((nz, nx, ny))).astype(np.float32)
    model = tmp_path / "m_true_x.bin"
    true.flatten("F").tofile(model)
    params = tmp_path / "parameters.txt"
    params.write_text(f"x_samples = {nx}\ny_samples = {ny}\nz_samples = {nz}\nmodel_spacing = {dh}\n"
                      f"model_file = {model}\nSPS = {tmp_path}/SPS.txt\nRPS = {tmp_path}/RPS.txt\n"
                      f"depth_mask = 100\n")
    prep.setup(params)
    sps = lib.read_points(tmp_path / "SPS.txt")
    rps = lib.read_points(tmp_path / "RPS.txt")
    assert sps.shape == (36, 3) and rps.shape == (2601, 3)
    assert np.allclose(sps[:, 2], 100.0) and np.allclose(sps[1, :2], [1000.0, 1600.0])
    init = np.fromfile(tmp_path / "m_init_x.bin", np.float32).reshape([nz, nx, ny], order="F")
    assert np.array_equal(init[:4], true[:4])           # above depth_mask: the true model
    assert not np.array_equal(init[4:], true[4:])        # below: smoothed in slowness
