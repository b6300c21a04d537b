"""The drop-in executables (fwi3d_b200/bin/*.exe) on a small setup written in
the reference's formats: their output files against the library and the FP64
oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from cases import TOL_IMAGE, TOL_SEIS, oracle_wavelet, rel_l2
from fwi3d_b200 import lib, synth

pytestmark = pytest.mark.gpu
BIN = Path(__file__).resolve().parents[1] / "fwi3d_b200" / "bin"

NZ, NX, NY, DH, NT, DT, FMAX = 24, 28, 26, 10.0, 150, 1e-3, 60.0
ABC_LEN, ABC_F, RBC_LEN = 85.0, 0.02, 65.0  # nb = 9 and 7


def write_setup(d: Path, vp, fixes=0, max_iteration=1, batch=1):
    d.mkdir(parents=True, exist_ok=True)
    for sub in ("data", "models", "seismic", "residuo"):
        (d / sub).mkdir(exist_ok=True)
    src = synth.surface_grid([70.0, 190.0], [120.0], 20.0)
    rec = synth.surface_grid(np.arange(10.0, 270.0, 40.0), np.arange(10.0, 250.0, 60.0), 30.0)
    np.savetxt(d / "SPS.txt", src, fmt="%.2f", delimiter=",")
    np.savetxt(d / "RPS.txt", rec, fmt="%.2f", delimiter=",")
    vp.astype(np.float32).tofile(d / "models" / "model.bin")
    prefix = f"seismogram_nt{NT}_nr{len(rec)}_{int(1e6 * np.float32(DT))}us_shot_"
    text = f"""# small drop-in setup
x_samples = {NX}
y_samples = {NY}
z_samples = {NZ}
model_spacing = {DH}
model_file = {d}/models/model.bin
SPS = {d}/SPS.txt
RPS = {d}/RPS.txt
time_samples = {NT}
time_spacing = {DT}
max_frequency = {FMAX}
abc_length = {ABC_LEN}
abc_factor = {ABC_F}
mod_output_folder = {d}/data/
max_iteration = {max_iteration}
depth_mask = 30
inv_rbc_ratio = 30
inv_rbc_varVp = 300
inv_rbc_length = {RBC_LEN}
inv_input_folder = {d}/data/
inv_input_prefix = {prefix}
inv_output_folder = {d}/models/
inv_residuo_folder = {d}/residuo/
mig_rbc_ratio = 30
mig_rbc_varVp = 300
mig_rbc_length = {RBC_LEN}
mig_input_folder = {d}/data/
mig_input_prefix = {prefix}
mig_output_folder = {d}/seismic/
b200_seed = 5
b200_fixes = {fixes}
b200_batch = {batch}
"""
    (d / "parameters.txt").write_text(text)
    return d / "parameters.txt", src, rec, prefix


def run(exe, params):
    r = subprocess.run([str(BIN / exe), str(params)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


@pytest.fixture(scope="module")
def true_model():
    v = synth.layered(NZ, NX, NY, DH, [1500, 2100, 2700], tops=[0, 80, 160])
    return synth.add_gaussian(v, DH, (140.0, 130.0, 120.0), 40.0, 0.1)


def test_modeling_exe_matches_library_and_oracle(tmp_path, true_model):
    params, src, rec, prefix = write_setup(tmp_path, true_model)
    out = run("modeling.exe", params)
    assert "Run time" in out
    nb = int(ABC_LEN / DH) + 1
    ctx = lib.Context(NZ, NX, NY, nb, DH, NT, DT, FMAX, lib.BOUNDARY_ABC, ABC_F)
    ctx.set_geometry(src, rec)
    ctx.set_velocity(true_model)
    seis = ctx.model_shots([0, 1])
    vpp = ctx.get_padded_velocity()
    w = synth.Workload("t", NZ, NX, NY, DH, NT, DT, FMAX, nb, true_model, src, rec)
    w64, _ = oracle_wavelet(ctx, w)
    nzz, nxx = NZ + 2 * nb, NX + 2 * nb
    flat = lambda p: orc.flat_index(orc.grid_index(float(p[2]), DH, nb), orc.grid_index(float(p[0]), DH, nb),
                                    orc.grid_index(float(p[1]), DH, nb), nzz, nxx)
    recf = np.array([flat(r) for r in rec], np.int64)
    for s in range(2):
        f = tmp_path / "data" / f"{prefix}{s + 1}.bin"
        got = np.fromfile(f, np.float32).reshape(len(rec), NT)
        assert np.array_equal(got, seis[s])
        ref, _, _ = orc.forward(vpp, DH, DT, NT, ctx.tlag, w64, flat(src[s]), recf, abc=True, nb=nb, factor=ABC_F)
        assert rel_l2(got, ref) < TOL_SEIS


def test_migration_exe_matches_library_and_oracle(tmp_path, true_model):
    params, src, rec, prefix = write_setup(tmp_path, true_model)
    run("modeling.exe", params)
    out = run("migration.exe", params)
    img = np.fromfile(tmp_path / "seismic" / f"RTM_section_{int(FMAX)}Hz_{NZ}x{NX}x{NY}_{int(DH)}m.bin",
                      np.float32)
    assert img.size == NZ * NX * NY and np.isfinite(img).all() and np.abs(img).max() > 0
    nb = int(RBC_LEN / DH) + 1
    ctx = lib.Context(NZ, NX, NY, nb, DH, NT, DT, FMAX, lib.BOUNDARY_RBC)
    ctx.set_geometry(src, rec)
    ctx.set_velocity(true_model)
    w = synth.Workload("t", NZ, NX, NY, DH, NT, DT, FMAX, nb, true_model, src, rec)
    w64, _ = oracle_wavelet(ctx, w)
    nzz, nxx = NZ + 2 * nb, NX + 2 * nb
    flat = lambda p: orc.flat_index(orc.grid_index(float(p[2]), DH, nb), orc.grid_index(float(p[0]), DH, nb),
                                    orc.grid_index(float(p[1]), DH, nb), nzz, nxx)
    recf = np.array([flat(r) for r in rec], np.int64)
    oimg = oill = None
    for s in range(2):
        # shot s runs through the pad of seed b200_seed + s
        ctx.apply_random_boundary(kind=0, ratio=30.0, varVp=300.0, seed=5 + s)
        d = np.fromfile(tmp_path / "data" / f"{prefix}{s + 1}.bin", np.float32)
        ctx.rtm_shots([s], d)
        vpp = ctx.get_padded_velocity()
        _, P, Q = orc.forward(vpp, DH, DT, NT, ctx.tlag, w64, flat(src[s]), recf)
        oimg, oill, _, _ = orc.backward(vpp, DH, DT, NT, ctx.tlag, recf, d.reshape(len(rec), NT), P, Q, mode=0,
                                        image=oimg, illum=oill)
    assert np.array_equal(ctx.rtm_image().ravel(), img)
    want = orc.rtm_post(oimg, oill, NZ, NX, NY, nb, DH)
    assert rel_l2(img, want) < TOL_IMAGE, rel_l2(img, want)
    # two shots per launch, each through its own pad: the same image up to the
    # order of the sum over shots
    params2, *_ = write_setup(tmp_path / "b2", true_model, batch=2)
    for f in (tmp_path / "data").iterdir():
        (tmp_path / "b2" / "data" / f.name).write_bytes(f.read_bytes())
    run("migration.exe", params2)
    img2 = np.fromfile(tmp_path / "b2" / "seismic" / f"RTM_section_{int(FMAX)}Hz_{NZ}x{NX}x{NY}_{int(DH)}m.bin",
                       np.float32)
    assert rel_l2(img2, img) < 1e-5


@pytest.mark.parametrize("fixes,iters", [(0, 1), (1, 2)])
def test_inversion_exe_outputs(tmp_path, true_model, fixes, iters):
    """Compat mode runs one iteration: its unbounded parabolic step overshoots
    on this small problem, as the reference's would.  With b200_fixes the
    bounded step lets the misfit fall over two iterations."""
    params, src, rec, prefix = write_setup(tmp_path, true_model, fixes=fixes, max_iteration=iters)
    run("modeling.exe", params)
    start = synth.smooth_slowness(true_model, 30.0, DH)
    start.astype(np.float32).tofile(tmp_path / "models" / "model.bin")  # model_file now holds the start model
    run("inversion.exe", params)
    conv = (tmp_path / "residuo" / f"convergence_{iters}_iterations.txt").read_text().split()
    res = [float(x) for x in conv]
    assert len(res) == iters + 1 and all(r > 0 for r in res)
    sfx = f"{int(FMAX)}Hz_{NZ}x{NX}x{NY}_{int(DH)}m.bin"
    for it in range(1, iters + 1):
        m = np.fromfile(tmp_path / "models" / f"model_FWI_iteration_{it}_{sfx}", np.float32)
        assert m.size == NZ * NX * NY and np.isfinite(m).all()
    final = np.fromfile(tmp_path / "models" / f"final_model_FWI_{sfx}", np.float32)
    assert np.array_equal(final, m)
    # the first misfit is that of the start model: check it against the oracle
    nb = int(ABC_LEN / DH) + 1
    ctx = lib.Context(NZ, NX, NY, nb, DH, NT, DT, FMAX, lib.BOUNDARY_ABC, ABC_F)
    ctx.set_geometry(src, rec)
    ctx.set_velocity(start)
    cal = ctx.model_shots([0, 1])
    total = 0.0
    for s in range(2):
        obs = np.fromfile(tmp_path / "data" / f"{prefix}{s + 1}.bin", np.float32)
        total += orc.residual_f32(obs, cal[s])
    assert abs(res[0] - np.sqrt(total)) <= 1e-5 * np.sqrt(total)
    assert all(b < a for a, b in zip(res, res[1:]))
