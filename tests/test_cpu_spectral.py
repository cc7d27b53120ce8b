"""Spectral mode pieces of the oracle against the reference's own code
(tests/golden/reference_queries.npz, from the reference's host build) and
against the reference's 100 self-test vectors (spectrum_basis.cuh:2472-2489).

The network weights and CIE / D65 tables are the reference's; the build reads
them from the reference sources into aperturerendererv3-optix-geometry_b200/
_data/spectral_tables.bin (git-ignored).  Tolerances: the encoders differ
from the reference's host build only by the fixed sin/cos (<= 3e-7 absolute);
wavelength samples by the fixed exp/log and the erfc approximation of the
Newton step (<= 2e-6 relative, pdf <= 1e-4 relative).
"""
import hashlib
import os

import numpy as np
import pytest

import oracle
import spectral_tables

HERE = os.path.dirname(os.path.abspath(__file__))
pytestmark = pytest.mark.skipif(not spectral_tables.available(), reason="spectral tables not built")


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(HERE, "golden", "reference_queries.npz"))


@pytest.fixture(scope="module")
def tabs():
    return spectral_tables.load()


def test_tables_are_the_fixture_tables(fx, tabs):
    assert np.array_equal(np.frombuffer(hashlib.sha256(tabs[0].tobytes()).digest(), np.uint8),
                          fx["spec_tables_sha256"])


def test_encoders_match_reference(fx, tabs):
    tab, it, gt = tabs
    rk, lk = oracle.spectral_encode(tab, it[:3].T.copy(), it[3].copy())
    np.testing.assert_allclose(rk, fx["spec_rgb_k"], rtol=0, atol=3e-7)
    np.testing.assert_allclose(lk, fx["spec_lam_k"], rtol=0, atol=3e-7)
    # the reference's self test: SpectralInteract(RGBEncode(rgb), LambdaEncode(lambda)) vs its gtTest
    pred = np.clip((rk * lk).sum(1), 0.0, 1.0)
    assert np.abs(pred - gt).max() < 5e-4


def test_wavelength_sampling_and_weights_match_reference(fx, tabs):
    lam, pdf = oracle.spectral_sample(fx["spec_u3"])
    np.testing.assert_allclose(lam, fx["spec_lambda"], rtol=2e-6)
    np.testing.assert_allclose(pdf, fx["spec_pdf"], rtol=1e-4)
    assert lam.min() >= 360.0 and lam.max() <= 780.0
    import scenes
    osc = oracle.OracleScene(scenes.box_scene())
    osc.set_spectral(tabs[0], 8)
    _, d65, xyz = osc.spectral_interact(fx["spec_lambda"], np.ones((len(lam), 3), np.float32))
    np.testing.assert_allclose(d65, fx["spec_d65"], rtol=1e-6)
    np.testing.assert_allclose(xyz, fx["spec_xyz"], rtol=1e-6, atol=1e-9)


def test_white_reflects_about_one_and_lut_is_smooth(tabs):
    """Sanity of the RGB table path: the reference model's white reflects
    0.75..1 across 400-700 nm and its black stays below 0.05."""
    import scenes
    osc = oracle.OracleScene(scenes.box_scene())
    osc.set_spectral(tabs[0], 32)
    lam = np.linspace(400, 700, 31).astype(np.float32)
    w, _, _ = osc.spectral_interact(lam, np.ones((31, 3), np.float32))
    b, _, _ = osc.spectral_interact(lam, np.zeros((31, 3), np.float32))
    assert np.all(w > 0.75) and np.all(w <= 1.0) and np.all(b < 0.05)
