"""ctypes wrapper of oracle/liboracle.so -- TEST INFRASTRUCTURE ONLY.

The FP64 CPU restatement of the reference's hot path (oracle/fwi_oracle.c).
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it, as
the checker; the product (fwi3d_b200) never imports it.

Arrays: volumes are float64 C-order (nyy, nxx, nzz) (z fastest, the
reference's Fortran [nzz, nxx, nyy]); seismograms are (nrec, nt).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_fwi3d.so"

_d = C.c_double
_i = C.c_int
_l = C.c_long
_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)
_fp = C.POINTER(C.c_float)
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE), str(LIB)], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        sig = {
            "orc_num_threads": (_i, []),
            "orc_set_threads": (None, [_i]),
            "orc_wavelet": (None, [_i, _d, _d, _dp, C.POINTER(_i)]),
            "orc_damper_tables": (None, [_i, _d, _dp, _dp, _dp]),
            "orc_damper_at": (_d, [_dp, _dp, _dp, _i, _i, _i, _i, _i, _i, _i]),
            "orc_expand": (None, [_dp, _i, _i, _i, _i, _dp]),
            "orc_reduce": (None, [_dp, _i, _i, _i, _i, _dp]),
            "orc_grid_index": (_i, [C.c_float, C.c_float, _i]),
            "orc_forward": (None, [_i, _i, _i, _d, _d, _i, _i, _dp, _dp, _l, _i, _lp, _i, _i,
                                   _dp, _dp, _dp, _dp, _dp, _dp]),
            "orc_backward": (None, [_i, _i, _i, _d, _d, _i, _i, _dp, _i, _lp, _dp, _i, _i, _i,
                                    _dp, _l, _dp, _dp, _dp, _dp]),
            "orc_rtm_post": (None, [_dp, _dp, _i, _i, _i, _i, _d, _dp]),
            "orc_gradient_post": (_d, [_dp, _dp, _i, _i, _i, _i, _d, _d, _dp]),
            "orc_residual": (_d, [_dp, _dp, _l, _dp]),
            "orc_residual_f32": (_d, [_fp, _fp, _l]),
            "orc_parabola_step": (_d, [_d, _d, _d, _d, _d, _d]),
            "orc_model_step": (None, [_dp, _dp, _l, _d, _dp]),
            "orc_step": (None, [_i, _i, _i, _d, _d, _dp, _dp, _dp]),
            "orc_laplacian": (None, [_i, _i, _i, _d, _dp, _dp]),
            "orc_image_adjoint": (_i, [_i, _i, _i, _d, _d, _i, _i, _dp, _i, _lp, _i, _dp, _l, _dp, _dp, _dp,
                                       _dp]),
        }
        for k, (r, a) in sig.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def _d64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def set_threads(n: int):
    load().orc_set_threads(n)


def num_threads() -> int:
    return load().orc_num_threads()


def wavelet(nt: int, dt: float, fmax: float):
    w = np.zeros(nt)
    tl = C.c_int()
    load().orc_wavelet(nt, dt, fmax, _p(w), C.byref(tl))
    return w, tl.value


def damper_tables(nb: int, factor: float):
    b1, b2, b3 = np.zeros(nb), np.zeros(nb * nb), np.zeros(nb ** 3)
    load().orc_damper_tables(nb, factor, _p(b1), _p(b2), _p(b3))
    return b1, b2, b3


def grid_index(coord: float, dh: float, nb: int) -> int:
    return load().orc_grid_index(coord, dh, nb)


def expand(vp, nz, nx, ny, nb):
    out = np.zeros((ny + 2 * nb, nx + 2 * nb, nz + 2 * nb))
    load().orc_expand(_p(_d64(vp)), nz, nx, ny, nb, _p(out))
    return out


def reduce(vpp, nz, nx, ny, nb):
    out = np.zeros((ny, nx, nz))
    load().orc_reduce(_p(_d64(vpp)), nz, nx, ny, nb, _p(out))
    return out


def flat_index(i, j, k, nzz, nxx):
    return int(i) + int(j) * nzz + int(k) * nzz * nxx


def forward(vpp, dh, dt, nt, tlag, w, src, rec, abc=False, nb=0, factor=0.0):
    """One shot. vpp (nyy,nxx,nzz); src flat index; rec flat indices.
    Returns seis (nrec, nt), P = u^N, Pold = u^{N-1}."""
    vpp = _d64(vpp)
    nyy, nxx, nzz = vpp.shape
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    seis = np.zeros((rec.size, nt))
    P = np.zeros_like(vpp)
    Q = np.zeros_like(vpp)
    if abc:
        b1, b2, b3 = damper_tables(nb, factor)
    else:
        b1 = b2 = b3 = np.zeros(1)
    load().orc_forward(nzz, nxx, nyy, dh, dt, nt, tlag, _p(vpp), _p(_d64(w)), int(src), rec.size,
                       rec.ctypes.data_as(_lp), int(abc), nb, _p(b1), _p(b2), _p(b3), _p(seis), _p(P), _p(Q))
    return seis, P, Q


def backward(vpp, dh, dt, nt, tlag, rec, data, Ps, Psold, mode=0, with_dy=False, subtract_src=False,
             w=None, src=0, image=None, illum=None):
    """Fused back-propagation of one shot; returns (image, illum, Ps, Psold)."""
    vpp = _d64(vpp)
    nyy, nxx, nzz = vpp.shape
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    data = _d64(data)
    Ps, Psold = _d64(Ps).copy(), _d64(Psold).copy()
    image = np.zeros_like(vpp) if image is None else _d64(image).copy()
    illum = np.zeros_like(vpp) if illum is None else _d64(illum).copy()
    w = np.zeros(max(nt, 1)) if w is None else _d64(w)
    load().orc_backward(nzz, nxx, nyy, dh, dt, nt, tlag, _p(vpp), rec.size, rec.ctypes.data_as(_lp),
                        _p(data), mode, int(with_dy), int(subtract_src), _p(w), int(src),
                        _p(Ps), _p(Psold), _p(image), _p(illum))
    return image, illum, Ps, Psold


def image_adjoint(vpp, dh, dt, nt, tlag, rec, Ps, Psold, m, subtract_src=True, w=None, src=0):
    """Adjoint of backward(..., mode=0) as a map data -> image for the source
    fields rebuilt from (Ps, Psold): returns data (nrec, nt) such that
    <backward image(d), m> = <d, image_adjoint(m)>."""
    vpp = _d64(vpp)
    nyy, nxx, nzz = vpp.shape
    rec = np.ascontiguousarray(rec, dtype=np.int64)
    out = np.zeros((rec.size, nt))
    w = np.zeros(max(nt, 1)) if w is None else _d64(w)
    st = load().orc_image_adjoint(nzz, nxx, nyy, dh, dt, nt, tlag, _p(vpp), rec.size, rec.ctypes.data_as(_lp),
                                  int(subtract_src), _p(w), int(src), _p(_d64(Ps)), _p(_d64(Psold)),
                                  _p(_d64(m)), _p(out))
    if st:
        raise MemoryError("orc_image_adjoint: out of memory")
    return out


def rtm_post(image_pad, illum_pad, nz, nx, ny, nb, dh):
    out = np.zeros((ny, nx, nz))
    load().orc_rtm_post(_p(_d64(image_pad)), _p(_d64(illum_pad)), nz, nx, ny, nb, dh, _p(out))
    return out


def gradient_post(grad_pad, illum_pad, nz, nx, ny, nb, dh, zmask):
    out = np.zeros((ny, nx, nz))
    g = load().orc_gradient_post(_p(_d64(grad_pad)), _p(_d64(illum_pad)), nz, nx, ny, nb, dh, zmask, _p(out))
    return out, g


def residual(obs, cal):
    o, c = _d64(obs).ravel(), _d64(cal).ravel()
    res = np.zeros_like(o)
    s = load().orc_residual(_p(o), _p(c), o.size, _p(res))
    return res, s


def residual_f32(obs, cal) -> float:
    o = np.ascontiguousarray(obs, np.float32).ravel()
    c = np.ascontiguousarray(cal, np.float32).ravel()
    return load().orc_residual_f32(o.ctypes.data_as(_fp), c.ctypes.data_as(_fp), o.size)


def parabola_step(a0, a1, a2, f0, f1, f2) -> float:
    return load().orc_parabola_step(a0, a1, a2, f0, f1, f2)


def model_step(m, g, alpha):
    m, g = _d64(m).ravel(), _d64(g).ravel()
    out = np.zeros_like(m)
    load().orc_model_step(_p(m), _p(g), m.size, alpha, _p(out))
    return out


def step(vpp, dh, dt, P, Pold):
    """One undamped leapfrog step in place on copies; returns (P, Pnew)."""
    vpp = _d64(vpp)
    nyy, nxx, nzz = vpp.shape
    P, Q = _d64(P).copy(), _d64(Pold).copy()
    load().orc_step(nzz, nxx, nyy, dh, dt, _p(vpp), _p(P), _p(Q))
    return P, Q


def laplacian(f, dh):
    f = _d64(f)
    nyy, nxx, nzz = f.shape
    out = np.zeros_like(f)
    load().orc_laplacian(nzz, nxx, nyy, dh, _p(f), _p(out))
    return out


# ---------------------------------------------------------------------------
# Reference build (oracle/_ref): the reference's own kernels, GPU only.
# ---------------------------------------------------------------------------
_ref = None


def ref_available() -> bool:
    return REF_LIB.exists()


def load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_LIB))
        lib.ref_dims.restype = _i
        lib.ref_dims.argtypes = [C.c_char_p, C.POINTER(_i)]
        lib.ref_run.restype = _i
        lib.ref_run.argtypes = [C.c_char_p, _fp, _i, _i, _i, _fp, _fp, _fp, _fp, _fp, _fp, _fp]
        _ref = lib
    return _ref


def write_reference_setup(folder, nz, nx, ny, dh, nt, dt, fmax, nb, src_xyz, rec_xyz, abc_factor=0.0):
    """Write the parameters.txt, SPS/RPS files and a placeholder model that the
    reference's Modeling::set_parameters() reads; abc_length is chosen so that
    int(abc_length/dh)+1 == nb."""
    folder = Path(folder)
    folder.mkdir(parents=True, exist_ok=True)
    sps, rps, model = folder / "SPS.txt", folder / "RPS.txt", folder / "model.bin"
    np.savetxt(sps, np.atleast_2d(src_xyz), fmt="%.4f", delimiter=",")
    np.savetxt(rps, np.atleast_2d(rec_xyz), fmt="%.4f", delimiter=",")
    np.full(nz * nx * ny, 2000.0, np.float32).tofile(model)
    abc_length = (nb - 0.5) * dh
    text = f"""x_samples = {nx}
y_samples = {ny}
z_samples = {nz}
model_spacing = {dh!r}
model_file = {model}
SPS = {sps}
RPS = {rps}
time_samples = {nt}
time_spacing = {dt!r}
max_frequency = {fmax!r}
abc_length = {abc_length!r}
abc_factor = {abc_factor!r}
mod_output_folder = {folder}/
"""
    p = folder / "parameters.txt"
    p.write_text(text)
    return p


def ref_run(params, vpp, shot=0, abc=True, backward=0, adj=None, want_fields=False, want_acc=False):
    """Run one shot through the reference build.  Returns a dict with seis
    (nrec, nt), optionally P/Pold and image/illum (nyy, nxx, nzz), and ms."""
    lib = load_ref()
    dims = (C.c_int * 7)()
    st = lib.ref_dims(str(params).encode(), dims)
    if st:
        raise RuntimeError(f"ref_dims failed ({st})")
    nzz, nxx, nyy, nb, nt, nrec, tlag = list(dims)
    vpp = np.ascontiguousarray(vpp, np.float32).reshape(-1)
    assert vpp.size == nzz * nxx * nyy
    seis = np.zeros((nrec, nt), np.float32)
    shape = (nyy, nxx, nzz)
    P = np.zeros(shape, np.float32) if want_fields else None
    Q = np.zeros(shape, np.float32) if want_fields else None
    img = np.zeros(shape, np.float32) if want_acc else None
    ill = np.zeros(shape, np.float32) if want_acc else None
    a = np.ascontiguousarray(adj, np.float32).reshape(-1) if adj is not None else None
    ms = np.zeros(2, np.float32)
    fp = lambda x: x.ctypes.data_as(_fp) if x is not None else None
    st = lib.ref_run(str(params).encode(), fp(vpp), shot, int(abc), backward, fp(a), fp(seis), fp(P), fp(Q),
                     fp(img), fp(ill), fp(ms))
    if st:
        raise RuntimeError(f"ref_run failed ({st})")
    return {"seis": seis, "P": P, "Pold": Q, "image": img, "illum": ill, "ms": ms, "tlag": tlag}
