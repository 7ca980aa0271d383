"""GPU drift correction (DriftCorrection) against the oracle's restatement and a known drift."""
import numpy as np
import pytest

import oracle as O
from test_oracle import drift_data

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bins,seed", [(6, 0), (3, 2), (2, 3)])
def test_drift_matches_oracle(zpkg, ctx, bins, seed):
    xyz, fr, cr, dt, vel = drift_data(seed=seed)
    got_b, got_l, px = zpkg.drift(ctx, xyz, fr, cr, pixel_nm=20.0, bins=bins, max_drift_um=0.16)
    want_b, want_l, wpx = O.drift(xyz, fr, cr, pixel_nm=20.0, bins=bins, max_drift_um=0.16)
    assert px == wpx
    assert np.array_equal(got_b[:, 0], want_b[:, 0])
    # float FFTs here, double in the oracle: the peak centroids agree to a small fraction of a voxel
    assert np.abs(got_b[:, 1:] - want_b[:, 1:]).max() < 0.05 * px
    assert np.abs(got_l - want_l).max() < 0.1 * px


def test_drift_recovers_a_known_drift_at_full_size(zpkg, ctx):
    xyz, fr, cr, dt, vel = drift_data(seed=5, nf=5000, nbead=200, n_per=60, L=3000.0, Lz=500.0,
                                      vel=(0.01, -0.008, 0.004))
    b, l, px = zpkg.drift(ctx, xyz, fr, cr, pixel_nm=10.0, bins=20, max_drift_um=0.3)
    want = np.outer(b[:, 0] - b[0, 0], vel)
    assert np.abs(b[:, 1:] - want).max() < 4.0
    assert np.abs(l - (dt - np.outer(np.full(len(fr), b[0, 0]), vel))).max() < 6.0


def test_drift_rejects_bad_arguments(zpkg, ctx):
    xyz, fr, cr, dt, vel = drift_data()
    with pytest.raises(zpkg.ZolaError):
        zpkg.drift(ctx, xyz, fr, cr, pixel_nm=0.0)
    with pytest.raises(zpkg.ZolaError):
        zpkg.drift(ctx, xyz, fr, cr, bins=0)
