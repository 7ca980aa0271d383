"""GPU parity of the CRLB curve and the z-centre search (SearchPSFcenter) against the oracle."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS, astig_zernike, tetrapod_zernike

pytestmark = pytest.mark.gpu


def pair(zpkg, ctx, N, zern, zfocus, n_wat):
    o = dict(OPTICS)
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=N, n_wat=n_wat, zfocus=zfocus, **o), zern)
    ref = O.OraclePSF(N, o["xystep"], o["na"], o["wavelength"], o["n_oil"], n_wat, o["sigma"], zern,
                      gauss_f32=False, zfocus=zfocus)
    return psf, ref


@pytest.mark.parametrize("N,R,h,ha", [(64, 64, 0.005, 0.5), (64, 32, 0.0005, 0.0005), (128, 128, 0.0005, 0.0005)])
def test_crlb_curve_matches_oracle(zpkg, ctx, N, R, h, ha):
    zern = astig_zernike() if N == 64 else tetrapod_zernike()
    psf, ref = pair(zpkg, ctx, N, zern, 0.3, 1.33)
    z = np.linspace(-1.2, 1.5, 7)
    got = psf.crlb_curve(R, z, 3000.0, 50.0, h, ha)
    want = ref.crlb_curve(R, z, 3000.0, 50.0, h, ha)
    assert np.all(np.isfinite(got))
    assert np.abs(got / want - 1).max() < 1e-7


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("zfocus,n_wat", [(0.4, 1.33), (0.0, 1.518), (-0.6, 1.40)])
def test_center_search_matches_oracle(zpkg, ctx, variant, zfocus, n_wat):
    psf, ref = pair(zpkg, ctx, 64, astig_zernike(), zfocus, n_wat)
    got = psf.center_search(1.0, R=64, variant=variant)
    want = ref.center_search(64, 1.0, variant)
    if got != want:
        # the scan picked a different grid point: only a near tie of the summed CRLB allows that
        lat = lambda zz: np.hypot(*ref.crlb_curve(64, [zz], 3000.0, 50.0, 0.005, 0.5)[0, :2])
        assert abs(lat(got) / lat(want) - 1) < 1e-6
    if variant == 1 and n_wat == 1.518:
        assert got == zfocus


def test_center_search_edge_arguments(zpkg, ctx):
    psf, _ = pair(zpkg, ctx, 64, astig_zernike(), 0.25, 1.33)
    assert psf.center_search(0.0, R=64) == 0.25  # non-positive range keeps zfocus
    with pytest.raises(zpkg.ZolaError):
        psf.center_search(1.0, R=65)
    with pytest.raises(zpkg.ZolaError):
        psf.center_search(1.0, R=64, variant=7)
