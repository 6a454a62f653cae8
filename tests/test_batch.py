"""Ragged batches on the host side (gmilos_b200.batch): grids grouped by
tolerance, one PSF per grid, every ROI handed to the engine's single batch
call in order on its group's exact grid.  A stand-in engine records the
call, so this runs on CPU; the GPU side is tests/test_gpu_ragged.py."""
import numpy as np
import pytest

from gmilos_b200 import batch


class FakeEngine:
    """Records the batch handed to invert_rois; a pixel's "model" is a
    function of its own samples only, as for the real engine."""

    def __init__(self):
        self.calls = []

    def invert_rois(self, rois, use_graph=False, autotune=False):
        self.calls.append((rois, use_graph, autotune))
        outs = [{"model": np.stack([a[:, 0, :].sum(axis=1), a[:, 3, :].max(axis=1)], axis=1),
                 "chi2": a[:, 1, 0].copy()} for a, _, _ in rois]
        return outs, {"pixels": sum(len(a) for a, _, _ in rois), "grids": len({id(l) for _, l, _ in rois})}


def roi(rng, n, lam):
    return rng.normal(size=(n, 4, len(lam))).astype(np.float32), lam


def test_one_call_in_roi_order():
    rng = np.random.default_rng(5)
    g30 = 6173.3356 + np.linspace(-0.35, 0.665, 30)
    g45 = 6173.3356 + np.linspace(-0.35, 1.19, 45)
    rois = [roi(rng, 16, g30), roi(rng, 300, g45), roi(rng, 7, g30), roi(rng, 1, g45), roi(rng, 512, g30)]
    eng = FakeEngine()
    psf_calls = []
    out, summary = batch.invert_rois(eng, rois, lambda lam: psf_calls.append(len(lam)) or np.ones(len(lam)),
                                     use_graph=True, autotune=True)
    assert len(eng.calls) == 1
    handed, use_graph, autotune = eng.calls[0]
    assert use_graph and autotune
    # one PSF per distinct grid; every ROI in order with its own profiles
    assert sorted(psf_calls) == [30, 45]
    assert [len(a) for a, _, _ in handed] == [16, 300, 7, 1, 512]
    for (iquv, lam), (a, l, p) in zip(rois, handed):
        np.testing.assert_array_equal(a, iquv)
        np.testing.assert_array_equal(l, lam)
        assert len(p) == len(lam)
    assert summary["pixels"] == 836 and summary["grids"] == 2
    for (iquv, _), o in zip(rois, out):
        np.testing.assert_array_equal(o["chi2"], iquv[:, 1, 0])


def test_grids_equal_to_rounding_share_a_grid():
    """Grids that differ below 1e-9 A (the same grid written twice) are one
    group, inverted on the first member's exact wavelengths; grids that
    differ by a sample spacing are two."""
    rng = np.random.default_rng(7)
    g = 6173.3356 + np.linspace(-0.35, 0.665, 30)
    eng = FakeEngine()
    _, s = batch.invert_rois(eng, [roi(rng, 4, g), roi(rng, 4, g + 1e-12), roi(rng, 4, g + 0.035)])
    handed = eng.calls[0][0]
    assert handed[0][1] is handed[1][1] and handed[2][1] is not handed[0][1]
    assert handed[0][2] is None
    assert s["grids"] == 2


def test_mismatched_roi_is_an_error():
    rng = np.random.default_rng(8)
    g = np.linspace(0, 1, 30)
    bad = (rng.normal(size=(4, 4, 29)).astype(np.float32), g)
    with pytest.raises(ValueError):
        batch.invert_rois(FakeEngine(), [roi(rng, 4, g), bad])


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
    idx, firsts = batch.group_grids([base, near, far, short, base.copy()])
    assert idx[0] == idx[1] == idx[4]
    assert len({idx[0], idx[2], idx[3]}) == 3
    assert len(firsts) == 3
