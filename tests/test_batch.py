"""Ragged batches (gmilos_b200.batch): ROIs grouped by wavelength grid, one
engine call per grid over the concatenated pixels, each ROI's outputs cut
back out in order, and the lane-occupancy figure.  A deterministic
stand-in replaces the engine, so this runs on CPU; the GPU side of the same
path is tests/test_gpu_ragged.py."""
import numpy as np
import pytest

from gmilos_b200 import batch


class FakeEngine:
    """Records each configure / invert; a pixel's "model" is a function of
    its own samples only, as for the real engine."""

    def __init__(self):
        self.calls = []
        self.cfg = None

    def configure(self, cfg):
        self.cfg = cfg

    def invert(self, iquv, fitted=False):
        self.calls.append((self.cfg, len(iquv)))
        model = np.stack([iquv[:, 0, :].sum(axis=1), iquv[:, 3, :].max(axis=1)], axis=1)
        return {"model": model, "chi2": iquv[:, 1, 0].copy(), "fitted": iquv.copy() if fitted else None}


def roi(rng, n, lam):
    return rng.normal(size=(n, 4, len(lam))).astype(np.float32), lam


def test_one_call_per_grid_and_outputs_in_roi_order():
    rng = np.random.default_rng(5)
    g30 = 6173.3356 + np.linspace(-0.35, 0.665, 30)
    g45 = 6173.3356 + np.linspace(-0.35, 1.19, 45)
    rois = [roi(rng, 16, g30), roi(rng, 300, g45), roi(rng, 7, g30), roi(rng, 1, g45), roi(rng, 512, g30)]
    eng = FakeEngine()
    out, summary = batch.invert_rois(eng, rois, lambda lam: ("cfg", len(lam)), fitted=True)
    # one configure + invert per distinct grid, over all its ROIs' pixels
    assert sorted(eng.calls) == [(("cfg", 30), 16 + 7 + 512), (("cfg", 45), 300 + 1)]
    assert summary["launches"] == 2 and summary["pixels"] == 836
    for (iquv, _), o in zip(rois, out):
        alone = eng.invert(iquv, fitted=True)
        for k in ("model", "chi2", "fitted"):
            np.testing.assert_array_equal(o[k], alone[k])


def test_lane_occupancy():
    """Samples over lane slots: a row of 32 lanes holds up to 32 samples, two
    rows (64 slots) up to 64."""
    rng = np.random.default_rng(6)
    g30 = np.linspace(0, 1, 30)
    g45 = np.linspace(0, 1, 45)
    _, s = batch.invert_rois(FakeEngine(), [roi(rng, 10, g30)], lambda lam: None)
    assert s["lane_occupancy"] == pytest.approx(30 / 32)
    _, s = batch.invert_rois(FakeEngine(), [roi(rng, 10, g30), roi(rng, 30, g45)], lambda lam: None)
    assert s["lane_occupancy"] == pytest.approx((10 * 30 + 30 * 45) / (10 * 32 + 30 * 64))
    _, s = batch.invert_rois(FakeEngine(), [], lambda lam: None)
    assert s == {"launches": 0, "pixels": 0, "lane_occupancy": 0.0}


def test_grids_equal_to_rounding_share_a_call():
    """Grids that differ below 1e-9 A (the same grid written twice) are one
    group; grids that differ by a sample spacing are two."""
    rng = np.random.default_rng(7)
    g = 6173.3356 + np.linspace(-0.35, 0.665, 30)
    eng = FakeEngine()
    _, s = batch.invert_rois(eng, [roi(rng, 4, g), roi(rng, 4, g + 1e-12), roi(rng, 4, g + 0.035)], lambda lam: None)
    assert s["launches"] == 2 and [n for _, n in eng.calls] == [8, 4]


def test_mismatched_roi_is_an_error():
    rng = np.random.default_rng(8)
    g = np.linspace(0, 1, 30)
    bad = (rng.normal(size=(4, 4, 29)).astype(np.float32), g)
    with pytest.raises(ValueError):
        batch.invert_rois(FakeEngine(), [roi(rng, 4, g), bad], lambda lam: None)


def test_grids_grouped_by_tolerance_not_rounding():
    """Grids that differ by far less than the tolerance share a group even
    where rounding to a fixed number of decimals would split them; grids
    that differ by more, or in length, do not."""
    base = 6173.3356 + np.linspace(-0.35, 0.665, 30)
    base[3] = 6173.0000000004999999   # rounds to ...000 at 9 decimals
    near = base.copy()
    near[3] = 6173.0000000005000001   # rounds to ...001 at 9 decimals
    far = base + 5e-9
    short = base[:29]
    idx = batch.group_grids([base, near, far, short, base.copy()])
    assert idx[0] == idx[1] == idx[4]
    assert len({idx[0], idx[2], idx[3]}) == 3
