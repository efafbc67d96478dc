"""The learned start's smooth upsampling, restated on the host
(warmstart.upsample_component): interpolation weights, edges and cell means (CPU)."""
import numpy as np

from artefact_b200.warmstart import upsample_component


def test_identity_without_subsampling():
    p = np.arange(12, dtype=np.float32).reshape(3, 4)
    np.testing.assert_array_equal(upsample_component(p, 1, 1, 3, 4), p)


def test_weights_and_clamped_edges():
    p = np.array([[0.0, 4.0, 8.0]], np.float32)
    out = upsample_component(p, 2, 1, 1, 6)
    # cell 0: left edge clamps to itself; cell 1: 3/4 own + 1/4 neighbour; cell 2: right edge clamps
    np.testing.assert_array_equal(out[0], np.array([0.0, 1.0, 3.0, 5.0, 7.0, 8.0], np.float32))
    col = upsample_component(p.T.copy(), 1, 2, 6, 1)
    np.testing.assert_array_equal(col[:, 0], out[0])


def test_linear_ramps_are_reproduced_and_cell_means_kept():
    y, x = np.mgrid[0:8, 0:10].astype(np.float32)
    p = 3 * x + 2 * y  # cell values of a linear ramp sampled at cell centres
    out = upsample_component(p, 2, 2, 16, 20)
    Y, X = np.mgrid[0:16, 0:20].astype(np.float64)
    exact = 3 * (X - 0.5) / 2 + 2 * (Y - 0.5) / 2
    inner = (slice(1, -1), slice(1, -1))
    np.testing.assert_allclose(out[inner], exact[inner], atol=1e-5)
    means = out.reshape(8, 2, 10, 2).mean(axis=(1, 3))
    np.testing.assert_allclose(means[1:-1, 1:-1], p[1:-1, 1:-1], atol=1e-5)


def test_ragged_full_grid_clamps_the_cell_index():
    """Rows past twice the component's height take the last cell's rule, as the
    solver's nearest upsampling clamps the cell index."""
    p = np.random.default_rng(1).standard_normal((3, 5)).astype(np.float32)
    out = upsample_component(p, 2, 2, 8, 12)  # full grid larger than 2x the component
    assert out.shape == (8, 12)
    np.testing.assert_array_equal(out[6], out[4])
    np.testing.assert_array_equal(out[7], out[5])
    np.testing.assert_array_equal(out[:, 10:], out[:, 8:10])
