"""Image and gradient post-processing where part of the volume was never
illuminated (a short time axis, a deep model): image / illumination is
defined as 0 there (the reference's 0/0 is NaN), and an all-zero gradient
stays zero instead of being scaled by 1/0."""
import numpy as np
import pytest

import oracle as orc

NZ, NX, NY, NB, DH = 20, 12, 10, 4, 10.0


def _accumulators(seed=0):
    rng = np.random.default_rng(seed)
    shape = (NY + 2 * NB, NX + 2 * NB, NZ + 2 * NB)
    img = rng.standard_normal(shape)
    ill = rng.uniform(0.5, 2.0, shape)
    ill[:, :, NB + NZ // 2:] = 0.0  # the deep half never saw the source field
    img[:, :, NB + NZ // 2:] = 0.0
    return img, ill


def test_oracle_post_processing_is_finite_without_illumination():
    img, ill = _accumulators()
    r = orc.rtm_post(img, ill, NZ, NX, NY, NB, DH)
    g, gmax = orc.gradient_post(img, ill, NZ, NX, NY, NB, DH, 0.0)
    assert np.all(np.isfinite(r)) and np.all(np.isfinite(g)) and gmax > 0
    assert np.all(r[:, :, NZ // 2 + 1:] == 0.0) and np.all(g[:, :, NZ // 2 + 1:] == 0.0)
    z, zmax = orc.gradient_post(np.zeros_like(img), np.zeros_like(ill), NZ, NX, NY, NB, DH, 0.0)
    assert zmax == 0.0 and np.all(z == 0.0)


def test_oracle_post_processing_reads_only_the_physical_box():
    """The reference crops the pad away before it reads the accumulators
    (src/migration/migration.cu:90-97, src/inversion/inversion.cu:142-146), so
    accumulators whose pad is zero (the library's default, which accumulates
    over the physical box only) give the same image and gradient bit for bit."""
    rng = np.random.default_rng(3)
    shape = (NY + 2 * NB, NX + 2 * NB, NZ + 2 * NB)
    img = rng.standard_normal(shape)
    ill = rng.uniform(0.5, 2.0, shape)
    box = np.zeros(shape, bool)
    box[NB:-NB, NB:-NB, NB:-NB] = True
    img_box, ill_box = np.where(box, img, 0.0), np.where(box, ill, 0.0)
    assert np.array_equal(orc.rtm_post(img, ill, NZ, NX, NY, NB, DH), orc.rtm_post(img_box, ill_box, NZ, NX, NY, NB, DH))
    for zmask in (0.0, 30.0):
        g, gmax = orc.gradient_post(img, ill, NZ, NX, NY, NB, DH, zmask)
        gb, gbmax = orc.gradient_post(img_box, ill_box, NZ, NX, NY, NB, DH, zmask)
        assert np.array_equal(g, gb) and gmax == gbmax


@pytest.mark.gpu
def test_library_post_processing_matches_the_oracle_without_illumination():
    import torch
    from fwi3d_b200 import lib
    ctx = lib.Context(NZ, NX, NY, NB, DH, 50, 1e-3, 30.0, lib.BOUNDARY_RBC, 0.0, 1, 0)
    # nothing accumulated yet: an all-zero gradient and image
    ctx.reset_accumulators()
    g0, gmax0 = ctx.gradient_post(0.0)
    assert gmax0 == 0.0 and np.all(g0 == 0.0)
    assert np.all(ctx.rtm_image() == 0.0)
    img, ill = _accumulators(1)
    d_img = torch.from_numpy(img.astype(np.float32)).cuda()
    d_ill = torch.from_numpy(ill.astype(np.float32)).cuda()
    ctx.set_accumulators_dev(d_img.data_ptr(), d_ill.data_ptr())
    torch.cuda.synchronize()
    got_r = ctx.rtm_image()
    got_g, gmax = ctx.gradient_post(0.0)
    want_r = orc.rtm_post(img.astype(np.float32), ill.astype(np.float32), NZ, NX, NY, NB, DH)
    want_g, wmax = orc.gradient_post(img.astype(np.float32), ill.astype(np.float32), NZ, NX, NY, NB, DH, 0.0)
    assert np.all(np.isfinite(got_r)) and np.all(np.isfinite(got_g))
    assert np.abs(got_r - want_r).max() <= 1e-5 * np.abs(want_r).max()
    assert np.abs(got_g - want_g).max() <= 1e-5
    assert abs(gmax - wmax) <= 1e-5 * wmax
