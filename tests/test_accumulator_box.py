"""Accumulation over the physical box only (the default) against the
reference's accumulation over every updated cell (FWI_FLAG_PAD_ACCUMULATE).

The reference accumulates image, gradient and illumination over the whole
padded grid (src/migration/migration.cu:134-202,
src/inversion/inversion.cu:400-468) and then crops the pad away before it reads
them (reduce_boundary, migration.cu:90-97, inversion.cu:142-146).  The library
by default neither reads nor writes the accumulators of pad cells.  Inside the
box both modes run the same FP32 arithmetic, so the accumulators there, the
RTM image and the post-processed gradient are the same bit for bit, and the
pad keeps the zeros of the last reset."""
import numpy as np
import pytest

from cases import interior
from fwi3d_b200 import lib, synth

pytestmark = pytest.mark.gpu

RBC = dict(kind=0, ratio=40.0, varVp=400.0)


def _case():
    # an 8-cell pad around 30 x 34 x 32 cells: the box edges fall inside z and
    # x tiles of every tile shape, so the per-cell masks are exercised
    w = synth.small_case(n=30, nb=8, nt=90, seed=4)
    w.src = np.array([[60.0, 70.0, 20.0], [150.0, 120.0, 30.0], [220.0, 200.0, 20.0]], np.float32)
    return w


def _run(w, flags, B, tile=None):
    c = lib.Context(w.nz, w.nx, w.ny, w.nb, w.dh, w.nt, w.dt, w.fmax, lib.BOUNDARY_RBC, 0.0, B,
                    flags | lib.FLAG_SUBTRACT_SOURCE)
    c.set_geometry(w.src, w.rec)
    c.set_velocity(w.vp)
    if tile is not None:
        c.set_tiles(tile, tile)
    c.set_shot_random_boundary(base_seed=7, **RBC)
    data = np.random.default_rng(3).standard_normal((3 * len(w.rec), w.nt)).astype(np.float32)
    c.rtm_shots([0, 1, 2], data)
    img, ill = c.get_accumulators()
    image = c.rtm_image()
    c.reset_accumulators()
    c.gradient_shots([0, 1, 2], data)
    g, gill = c.get_accumulators()
    gpost, gmax = c.gradient_post(zmask=20.0)
    c.close()
    return dict(img=img, ill=ill, image=image, g=g, gill=gill, gpost=gpost, gmax=gmax)


@pytest.mark.parametrize("B", [1, 3])
def test_box_accumulation_equals_pad_accumulation_inside_the_box(B):
    w = _case()
    box = _run(w, 0, B)
    pad = _run(w, lib.FLAG_PAD_ACCUMULATE, B)
    inside = np.zeros(box["img"].shape, bool)
    inside[w.nb:-w.nb, w.nb:-w.nb, w.nb:-w.nb] = True
    for k in ("img", "ill", "g", "gill"):
        assert np.array_equal(interior(box[k], w.nb), interior(pad[k], w.nb)), k
        assert not box[k][~inside].any(), f"{k}: the pad was accumulated"
        assert np.abs(pad[k][~inside]).max() > 0, f"{k}: the flag did not accumulate the pad"
    assert np.array_equal(box["image"], pad["image"])
    assert np.array_equal(box["gpost"], pad["gpost"]) and box["gmax"] == pad["gmax"]


def test_box_accumulation_is_the_same_for_every_tile():
    w = _case()
    base = _run(w, 0, 1, tile=0)
    for t in range(1, len(lib.tile_table())):
        got = _run(w, 0, 1, tile=t)
        for k in ("img", "ill", "g", "gill"):
            assert np.array_equal(got[k], base[k]), f"tile {t}: {k} differs"
