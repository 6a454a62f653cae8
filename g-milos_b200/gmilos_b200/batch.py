"""Ragged batches: regions of interest of any size and wavelength grid.

Pixels are independent, so a batch of ROIs inverts as one engine call per
distinct wavelength grid over the concatenated pixels of the ROIs on that
grid: the kernels' work-stealing cursors take pixels of all of them alike,
so ROI sizes do not matter.  The reference inverts one cube per
run (gmilos.cu:1008-1249); this is the host-side loop a caller of it would
write, done once.
"""
import numpy as np


GRID_ATOL = 1e-9   # A: grids closer than this everywhere are the same grid


def group_grids(lams, atol=GRID_ATOL):
    """Group wavelength grids that agree to `atol` at every sample (same
    length).  Returns one group index per grid; a group is inverted on its
    first member's exact wavelengths."""
    firsts, idx = [], []
    for lam in lams:
        lam = np.asarray(lam, dtype=np.float64)
        for g, f in enumerate(firsts):
            if len(f) == len(lam) and np.allclose(lam, f, rtol=0.0, atol=atol):
                idx.append(g)
                break
        else:
            firsts.append(lam)
            idx.append(len(firsts) - 1)
    return idx


def invert_rois(engine, rois, config_for_grid, fitted=False):
    """Invert a ragged batch.  rois: list of (iquv [P_i][4][nl_i] float32,
    lambda [nl_i] absolute wavelengths); config_for_grid(lam) returns the
    engine configuration (make_config) for one grid.  Returns one output
    dict per ROI (engine.invert's keys) and a summary: engine calls
    ("launches", one per grid), pixels and
    the lane occupancy (wavelength samples over lane slots, 32 per lane row
    of up to 32 samples, 64 above)."""
    groups = {}
    gidx = group_grids([lam for _, lam in rois])
    for i, (iquv, lam) in enumerate(rois):
        a = np.ascontiguousarray(iquv, dtype=np.float32)
        if a.ndim != 3 or a.shape[1] != 4 or a.shape[2] != len(lam):
            raise ValueError("ROI %d: iquv must be [P][4][nl] on its own grid" % i)
        groups.setdefault(gidx[i], []).append((i, a, lam))
    out = [None] * len(rois)
    pixels = 0
    slots = 0.0
    samples = 0.0
    for members in groups.values():
        lam = members[0][2]
        nl = len(lam)
        cube = np.concatenate([a for _, a, _ in members], axis=0)
        engine.configure(config_for_grid(lam))
        res = engine.invert(cube, fitted=fitted)
        start = 0
        for i, a, _ in members:
            n = len(a)
            out[i] = {k: (None if v is None else v[start:start + n]) for k, v in res.items()}
            start += n
        pixels += len(cube)
        samples += len(cube) * nl
        slots += len(cube) * (32 if nl <= 32 else 64)
    summary = {"launches": len(groups), "pixels": pixels,
               "lane_occupancy": samples / slots if slots else 0.0}
    return out, summary
