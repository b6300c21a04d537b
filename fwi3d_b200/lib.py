"""ctypes binding of libfwi3d.so (include/fwi3d.h).

Array conventions follow the reference's binary layouts:
  volumes      numpy float32, z fastest: C-order shape (ny, nx, nz), which is the
               reference's Fortran [nz, nx, ny] (src/functions.py:23-25);
  seismograms  C-order shape (nrec, nt), the reference's Fortran [nt, nrec]
               (src/functions.py:19-21).

The library is the only compute path: when libfwi3d.so is missing or there is
no CUDA device, every entry point raises; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

# FWI3D_LIB selects another build of the library (e.g. a tuning variant).
LIB_PATH = Path(os.environ.get("FWI3D_LIB", Path(__file__).resolve().parent / "lib" / "libfwi3d.so"))

FWI_OK = 0
BOUNDARY_ABC = 0
BOUNDARY_RBC = 1
FLAG_GRAD_DY = 0x1
FLAG_SUBTRACT_SOURCE = 0x2
FLAG_PAD_ACCUMULATE = 0x4   # accumulate in the pad too (default: the physical box only)

STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "device allocation failed",
                4: "device wait timed out", 5: "call out of order", 6: "file could not be opened",
                7: "numerical check failed", 8: "no CUDA device"}

# every entry point the header declares, with its ctypes signature
_p = C.c_void_p
_i = C.c_int
_f = C.c_float
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_i64 = C.c_int64

SIGNATURES = {
    "fwi_create": (_i, [_p, _p, C.POINTER(_p)]),
    "fwi_destroy": (_i, [_p]),
    "fwi_status_string": (C.c_char_p, [_i]),
    "fwi_last_error": (_i, [_p, C.c_char_p, _i]),
    "fwi_set_stream": (_i, [_p, _p]),
    "fwi_get_dims": (_i, [_p, _ip, _ip, _ip, _ip, _ip]),
    "fwi_set_velocity": (_i, [_p, _fp]),
    "fwi_set_padded_velocity": (_i, [_p, _fp]),
    "fwi_get_padded_velocity": (_i, [_p, _fp]),
    "fwi_apply_random_boundary": (_i, [_p, _p, C.c_uint64]),
    "fwi_set_shot_random_boundary": (_i, [_p, _p, C.c_uint64]),
    "fwi_random_boundary_recipe": (_i, [_p, _p, C.c_uint64, _fp, _fp, _fp, _i, _ip]),
    "fwi_set_geometry": (_i, [_p, _i, _fp, _fp, _fp, _i, _fp, _fp, _fp, _ip, _ip]),
    "fwi_shot_nrec": (_i, [_p, _i, _ip]),
    "fwi_model_shots": (_i, [_p, _ip, _i, _fp]),
    "fwi_model_shots_dev": (_i, [_p, _ip, _i, _p]),
    "fwi_rtm_shots": (_i, [_p, _ip, _i, _fp]),
    "fwi_rtm_shots_dev": (_i, [_p, _ip, _i, _p]),
    "fwi_reset_accumulators": (_i, [_p]),
    "fwi_zero_image": (_i, [_p]),
    "fwi_get_accumulators": (_i, [_p, _fp, _fp]),
    "fwi_get_accumulators_dev": (_i, [_p, _p, _p]),
    "fwi_set_accumulators_dev": (_i, [_p, _p, _p]),
    "fwi_rtm_image": (_i, [_p, _fp]),
    "fwi_gradient_shots": (_i, [_p, _ip, _i, _fp]),
    "fwi_gradient_shots_dev": (_i, [_p, _ip, _i, _p]),
    "fwi_gradient_post": (_i, [_p, _f, _fp, _fp]),
    "fwi_residual": (_i, [_p, _fp, _fp, _i64, _fp, _dp]),
    "fwi_residual_dev": (_i, [_p, _p, _p, _i64, _p, _dp]),
    "fwi_residual_noalloc": (_i, [_p, _p, _i64, _p, _p, _p]),
    "fwi_dot_dev": (_i, [_p, _p, _p, _i64, _dp]),
    "fwi_cnn_create": (_i, [C.c_uint64, C.POINTER(_p)]),
    "fwi_cnn_destroy": (_i, [_p]),
    "fwi_cnn_last_error": (_i, [_p, C.c_char_p, _i]),
    "fwi_cnn_set_stream": (_i, [_p, _p]),
    "fwi_cnn_get_weights": (_i, [_p, _fp, _fp]),
    "fwi_cnn_set_weights": (_i, [_p, _fp, _fp]),
    "fwi_cnn_forward": (_i, [_p, _i, _i, _i, _p, _p]),
    "fwi_cnn_train_step": (_i, [_p, _i, _i, _i, _p, _p, _f, _dp, _fp, _fp]),
    "fwi_prepare_rtm_input": (_i, [_fp, _fp, _i, _i, _fp, _fp, _f, _f, _f, _f, _f, _f]),
    "fwi_catch_parameter": (_i, [C.c_char_p, C.c_char_p, C.c_char_p, _i]),
    "fwi_read_points": (_i, [C.c_char_p, _fp, _fp, _fp, _i, _ip]),
    "fwi_read_binary": (_i, [C.c_char_p, _fp, _i64]),
    "fwi_write_binary": (_i, [C.c_char_p, _fp, _i64]),
    "fwi_selftest_bounded_wait": (_i, [_p, _i]),
    "fwi_last_timing": (_i, [_p, _fp, _fp]),
    "fwi_launch_count": (_i, [_p, C.POINTER(C.c_int64)]),
    "fwi_get_tiles": (_i, [_p, _ip, _ip]),
    "fwi_set_tiles": (_i, [_p, _i, _i]),
    "fwi_autotune": (_i, [_p]),
    "fwi_num_tiles": (_i, [_ip]),
    "fwi_tile_shape": (_i, [_i, _ip, _ip]),
}


class FwiGrid(C.Structure):
    _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nb", C.c_int), ("dh", C.c_float)]


class FwiParams(C.Structure):
    _fields_ = [("nt", C.c_int), ("dt", C.c_float), ("fmax", C.c_float), ("boundary", C.c_int),
                ("abc_factor", C.c_float), ("max_batch", C.c_int), ("flags", C.c_int)]


class FwiRbc(C.Structure):
    _fields_ = [("kind", C.c_int), ("ratio", C.c_float), ("varVp", C.c_float), ("cfl_cap", C.c_float)]


class FwiError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_LIB = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libfwi3d.so and declare every entry point; raise if it is missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python -m fwi3d_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def _f32(a, n: int | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class Context:
    """One library context: a padded grid, a time axis and one boundary kind.

    Mirrors the reference workflow classes: ``model_shots`` is
    Modeling::forward_solver + get_seismogram, ``rtm_shots`` is
    Migration::forward_propagation + backward_propagation, ``rtm_image`` is
    Migration::export_seismic, ``gradient_shots`` + ``gradient_post`` is the
    device part of Inversion::compute_gradient.
    """

    def __init__(self, nz, nx, ny, nb, dh, nt, dt, fmax, boundary=BOUNDARY_ABC, abc_factor=0.0,
                 max_batch=1, flags=0):
        self.lib = load()
        self.grid = FwiGrid(nz, nx, ny, nb, dh)
        self.params = FwiParams(nt, dt, fmax, boundary, abc_factor, max_batch, flags)
        h = C.c_void_p()
        self._check(self.lib.fwi_create(C.byref(self.grid), C.byref(self.params), C.byref(h)), None)
        self.h = h
        self.nz, self.nx, self.ny, self.nb, self.nt = nz, nx, ny, nb, nt
        d = [C.c_int() for _ in range(5)]
        self.lib.fwi_get_dims(self.h, *[C.byref(x) for x in d])
        self.nzz, self.nxx, self.nyy, self.ldz, self.tlag = (x.value for x in d)
        self._nrec = None

    # -- plumbing ---------------------------------------------------------
    def _check(self, st: int, h=None):
        if st != FWI_OK:
            msg = ""
            hh = h if h is not None else getattr(self, "h", None)
            if hh:
                buf = C.create_string_buffer(512)
                self.lib.fwi_last_error(hh, buf, 512)
                msg = buf.value.decode(errors="replace")
            raise FwiError(st, msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.fwi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def padded_shape(self):
        return (self.nyy, self.nxx, self.nzz)

    @property
    def model_shape(self):
        return (self.ny, self.nx, self.nz)

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.fwi_set_stream(self.h, C.c_void_p(stream_ptr)))

    # -- model --------------------------------------------------------------
    def set_velocity(self, vp):
        a = _f32(vp, self.nz * self.nx * self.ny)
        self._check(self.lib.fwi_set_velocity(self.h, _fptr(a)))

    def set_padded_velocity(self, vpp):
        a = _f32(vpp, self.nzz * self.nxx * self.nyy)
        self._check(self.lib.fwi_set_padded_velocity(self.h, _fptr(a)))

    def get_padded_velocity(self) -> np.ndarray:
        out = np.empty(self.padded_shape, np.float32)
        self._check(self.lib.fwi_get_padded_velocity(self.h, _fptr(out)))
        return out

    def apply_random_boundary(self, kind=0, ratio=100.0, varVp=1000.0, cfl_cap=0.98, seed=1):
        r = FwiRbc(kind, ratio, varVp, cfl_cap)
        self._check(self.lib.fwi_apply_random_boundary(self.h, C.byref(r), C.c_uint64(seed)))

    def set_shot_random_boundary(self, kind=0, ratio=100.0, varVp=1000.0, cfl_cap=0.98, base_seed=1):
        """From now on shot s propagates through the random pad of seed
        base_seed + s, rebuilt for every batch (one velocity slot per batch
        slot)."""
        r = FwiRbc(kind, ratio, varVp, cfl_cap)
        self._check(self.lib.fwi_set_shot_random_boundary(self.h, C.byref(r), C.c_uint64(base_seed)))

    def clear_shot_random_boundary(self):
        """Back to one shared velocity: the clean padded model."""
        self._check(self.lib.fwi_set_shot_random_boundary(self.h, None, C.c_uint64(0)))

    def random_boundary_recipe(self, kind=0, ratio=100.0, varVp=1000.0, cfl_cap=0.98, seed=1):
        """(vlo, vhi, blobs) of one seed: the clamp bounds and an (n, 5) array
        of blobs (x, y, z, r, signed amplitude) in the order they are added."""
        r = FwiRbc(kind, ratio, varVp, cfl_cap)
        lo, hi, n = C.c_float(), C.c_float(), C.c_int()
        self._check(self.lib.fwi_random_boundary_recipe(self.h, C.byref(r), C.c_uint64(seed), C.byref(lo),
                                                        C.byref(hi), None, 0, C.byref(n)))
        blobs = np.zeros((n.value, 5), np.float32)
        if n.value:
            self._check(self.lib.fwi_random_boundary_recipe(self.h, C.byref(r), C.c_uint64(seed), None, None,
                                                            _fptr(blobs), n.value, C.byref(n)))
        return lo.value, hi.value, blobs

    # -- geometry -----------------------------------------------------------
    def set_geometry(self, src_xyz, rec_xyz, rec_first=None, rec_count=None):
        """src_xyz (ns, 3) and rec_xyz (nr, 3) in metres, columns x, y, z."""
        s = np.ascontiguousarray(src_xyz, np.float32).reshape(-1, 3)
        r = np.ascontiguousarray(rec_xyz, np.float32).reshape(-1, 3)
        cols = [np.ascontiguousarray(s[:, k]) for k in range(3)] + \
               [np.ascontiguousarray(r[:, k]) for k in range(3)]
        ns, nr = s.shape[0], r.shape[0]
        if rec_first is not None:
            f = np.ascontiguousarray(rec_first, np.int32)
            n = np.ascontiguousarray(rec_count, np.int32)
            fp, np_ = f.ctypes.data_as(_ip), n.ctypes.data_as(_ip)
            self._nrec = n.copy()
        else:
            fp = np_ = None
            self._nrec = np.full(ns, nr, np.int32)
        self._check(self.lib.fwi_set_geometry(self.h, ns, _fptr(cols[0]), _fptr(cols[1]), _fptr(cols[2]),
                                              nr, _fptr(cols[3]), _fptr(cols[4]), _fptr(cols[5]), fp, np_))
        self._keep = cols

    def shot_nrec(self, shot: int) -> int:
        return int(self._nrec[shot])

    def _shots(self, shots):
        s = np.ascontiguousarray(np.atleast_1d(shots), np.int32)
        return s, s.ctypes.data_as(_ip)

    # -- workflows ------------------------------------------------------------
    def model_shots(self, shots) -> list[np.ndarray]:
        s, sp = self._shots(shots)
        counts = [self.shot_nrec(int(k)) for k in s]
        out = np.empty(sum(counts) * self.nt, np.float32)
        self._check(self.lib.fwi_model_shots(self.h, sp, len(s), _fptr(out)))
        res, off = [], 0
        for n in counts:
            res.append(out[off:off + n * self.nt].reshape(n, self.nt))
            off += n * self.nt
        return res

    def model_shots_dev(self, shots, d_out_ptr: int):
        s, sp = self._shots(shots)
        self._check(self.lib.fwi_model_shots_dev(self.h, sp, len(s), C.c_void_p(d_out_ptr)))

    def _concat(self, shots, data):
        if isinstance(data, (list, tuple)):
            data = np.concatenate([_f32(d) for d in data])
        a = _f32(data)
        need = sum(self.shot_nrec(int(k)) for k in np.atleast_1d(shots)) * self.nt
        if a.size != need:
            raise ValueError(f"data holds {a.size} samples, shots need {need}")
        return a

    def rtm_shots(self, shots, data):
        s, sp = self._shots(shots)
        a = self._concat(s, data)
        self._check(self.lib.fwi_rtm_shots(self.h, sp, len(s), _fptr(a)))

    def rtm_shots_dev(self, shots, d_data_ptr: int):
        s, sp = self._shots(shots)
        self._check(self.lib.fwi_rtm_shots_dev(self.h, sp, len(s), C.c_void_p(d_data_ptr)))

    def gradient_shots(self, shots, residual):
        s, sp = self._shots(shots)
        a = self._concat(s, residual)
        self._check(self.lib.fwi_gradient_shots(self.h, sp, len(s), _fptr(a)))

    def gradient_shots_dev(self, shots, d_res_ptr: int):
        s, sp = self._shots(shots)
        self._check(self.lib.fwi_gradient_shots_dev(self.h, sp, len(s), C.c_void_p(d_res_ptr)))

    def reset_accumulators(self):
        self._check(self.lib.fwi_reset_accumulators(self.h))

    def zero_image(self):
        self._check(self.lib.fwi_zero_image(self.h))

    def get_accumulators(self):
        img = np.empty(self.padded_shape, np.float32)
        ill = np.empty(self.padded_shape, np.float32)
        self._check(self.lib.fwi_get_accumulators(self.h, _fptr(img), _fptr(ill)))
        return img, ill

    def get_accumulators_dev(self, d_img: int, d_ill: int):
        self._check(self.lib.fwi_get_accumulators_dev(self.h, C.c_void_p(d_img or None), C.c_void_p(d_ill or None)))

    def set_accumulators_dev(self, d_img: int, d_ill: int):
        """Replace the accumulators by caller device buffers (dense padded)."""
        self._check(self.lib.fwi_set_accumulators_dev(self.h, C.c_void_p(d_img or None), C.c_void_p(d_ill or None)))

    def rtm_image(self, out: np.ndarray | None = None) -> np.ndarray:
        """The post-processed image (model shape).  `out`, if given, is a
        C-contiguous float32 host array of the model's size (for example a view
        of pinned memory) that receives it without an extra copy."""
        if out is None:
            out = np.empty(self.model_shape, np.float32)
        elif (out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"] or not out.flags["WRITEABLE"]
              or out.size != int(np.prod(self.model_shape))):
            raise ValueError("out must be a writable, C-contiguous float32 array of the model's size")
        self._check(self.lib.fwi_rtm_image(self.h, _fptr(out)))
        return out

    def gradient_post(self, zmask: float):
        out = np.empty(self.model_shape, np.float32)
        g = C.c_float()
        self._check(self.lib.fwi_gradient_post(self.h, zmask, _fptr(out), C.byref(g)))
        return out, g.value

    def residual(self, obs, cal):
        o, c = _f32(obs), _f32(cal)
        if o.size != c.size:
            raise ValueError("obs and cal differ in size")
        res = np.empty_like(o)
        s = C.c_double()
        self._check(self.lib.fwi_residual(self.h, _fptr(o), _fptr(c), o.size, _fptr(res), C.byref(s)))
        return res, s.value

    def residual_dev(self, d_obs: int, d_cal: int, n: int, d_res: int = 0) -> float:
        s = C.c_double()
        self._check(self.lib.fwi_residual_dev(self.h, C.c_void_p(d_obs), C.c_void_p(d_cal), n,
                                              C.c_void_p(d_res or None), C.byref(s)))
        return s.value

    def dot_dev(self, d_a: int, d_b: int, n: int) -> float:
        s = C.c_double()
        self._check(self.lib.fwi_dot_dev(self.h, C.c_void_p(d_a), C.c_void_p(d_b), n, C.byref(s)))
        return s.value

    # -- diagnostics ----------------------------------------------------------
    def last_timing(self):
        f, b = C.c_float(), C.c_float()
        self.lib.fwi_last_timing(self.h, C.byref(f), C.byref(b))
        return f.value, b.value

    def launch_count(self) -> int:
        n = C.c_int64()
        self.lib.fwi_launch_count(self.h, C.byref(n))
        return n.value

    def autotune(self):
        self._check(self.lib.fwi_autotune(self.h))

    def tiles(self):
        f, b = C.c_int(), C.c_int()
        self.lib.fwi_get_tiles(self.h, C.byref(f), C.byref(b))
        return f.value, b.value

    def set_tiles(self, fwd: int, bwd: int):
        self._check(self.lib.fwi_set_tiles(self.h, fwd, bwd))


class Cnn:
    """The learned preconditioner network (fwi_cnn_*): BF16 tensor-core
    forward/backward, FP32 Adam.  Volumes are device pointers."""

    NL, TAPS, CH = 4, 27, 16

    def __init__(self, seed=0):
        self.lib = load()
        h = C.c_void_p()
        st = self.lib.fwi_cnn_create(C.c_uint64(seed), C.byref(h))
        if st != FWI_OK:
            raise FwiError(st, "fwi_cnn_create")
        self.h = h

    def _check(self, st):
        if st != FWI_OK:
            buf = C.create_string_buffer(512)
            self.lib.fwi_cnn_last_error(self.h, buf, 512)
            raise FwiError(st, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self.lib.fwi_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.fwi_cnn_set_stream(self.h, C.c_void_p(stream_ptr)))

    def get_weights(self):
        w = np.zeros((self.NL, self.TAPS, self.CH, self.CH), np.float32)
        b = np.zeros((self.NL, self.CH), np.float32)
        self._check(self.lib.fwi_cnn_get_weights(self.h, _fptr(w), _fptr(b)))
        return w, b

    def set_weights(self, w, b):
        w = np.ascontiguousarray(w, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        self._check(self.lib.fwi_cnn_set_weights(self.h, _fptr(w), _fptr(b)))

    def forward(self, shape_zxy, d_in: int, d_out: int):
        nz, nx, ny = shape_zxy
        self._check(self.lib.fwi_cnn_forward(self.h, nz, nx, ny, C.c_void_p(d_in), C.c_void_p(d_out)))

    def train_step(self, shape_zxy, d_in: int, d_target: int, lr: float, want_grads=False):
        nz, nx, ny = shape_zxy
        loss = C.c_double()
        gw = gb = None
        if want_grads:
            gw = np.zeros((self.NL, self.TAPS, self.CH, self.CH), np.float32)
            gb = np.zeros((self.NL, self.CH), np.float32)
        self._check(self.lib.fwi_cnn_train_step(self.h, nz, nx, ny, C.c_void_p(d_in), C.c_void_p(d_target), lr,
                                                C.byref(loss), _fptr(gw) if gw is not None else None,
                                                _fptr(gb) if gb is not None else None))
        return (loss.value, gw, gb) if want_grads else loss.value


def prepare_rtm_input(seis, rec_xy, src_xy, dt, velocity=3600.0, time_delay=0.18, gstd=30.0):
    """RTM input gather of one shot (fwi_prepare_rtm_input): seis (nrec, nt)."""
    a = np.ascontiguousarray(seis, np.float32)
    nrec, nt = a.shape
    rx = np.ascontiguousarray(np.asarray(rec_xy)[:, 0], np.float32)
    ry = np.ascontiguousarray(np.asarray(rec_xy)[:, 1], np.float32)
    out = np.empty_like(a)
    st = load().fwi_prepare_rtm_input(_fptr(a), _fptr(out), nt, nrec, _fptr(rx), _fptr(ry), float(src_xy[0]),
                                      float(src_xy[1]), velocity, time_delay, dt, gstd)
    if st != FWI_OK:
        raise FwiError(st, "fwi_prepare_rtm_input")
    return out


def catch_parameter(file, key: str) -> str:
    """The reference's parameters.txt lookup (prefix match, '#' comments)."""
    buf = C.create_string_buffer(4096)
    st = load().fwi_catch_parameter(str(file).encode(), key.encode(), buf, 4096)
    if st != FWI_OK:
        raise FwiError(st, f"cannot read {file}")
    return buf.value.decode()


def read_points(file) -> np.ndarray:
    """SPS/RPS file -> (n, 3) float32 x, y, z."""
    lib = load()
    n = C.c_int()
    st = lib.fwi_read_points(str(file).encode(), None, None, None, 0, C.byref(n))
    if st != FWI_OK:
        raise FwiError(st, f"cannot read {file}")
    cols = [np.zeros(n.value, np.float32) for _ in range(3)]
    st = lib.fwi_read_points(str(file).encode(), *[_fptr(c) for c in cols], n.value, C.byref(n))
    if st != FWI_OK:
        raise FwiError(st, f"malformed {file}")
    return np.stack(cols, axis=1)


NOALLOC_MAX_N = 268435456


def residual_noalloc(d_obs: int, d_cal: int, n: int, d_res: int, d_sum_sq: int, stream: int = 0) -> None:
    """fwi_residual_noalloc on caller device buffers (no context, no device
    allocation); the FP64 sum lands in the double at d_sum_sq."""
    st = load().fwi_residual_noalloc(C.c_void_p(d_obs), C.c_void_p(d_cal), n, C.c_void_p(d_res or None),
                                     C.c_void_p(d_sum_sq), C.c_void_p(stream or None))
    if st != FWI_OK:
        raise FwiError(st, "fwi_residual_noalloc failed (n above NOALLOC_MAX_N or a CUDA error)")


def tile_table() -> list[tuple[int, int]]:
    lib = load()
    n = C.c_int()
    lib.fwi_num_tiles(C.byref(n))
    out = []
    for t in range(n.value):
        tz, tx = C.c_int(), C.c_int()
        lib.fwi_tile_shape(t, C.byref(tz), C.byref(tx))
        out.append((tz.value, tx.value))
    return out
