"""Ragged batches: regions of interest of any size and wavelength grid.

invert_rois hands a whole batch to the engine's gm_invert_rois: one
persistent wave-synchronous launch sequence per samples-per-lane class (the
grids of <= 32 samples and those of 33..64 run concurrently), in which
every pixel carries its grid and a warp reloads the grid's constants when it
moves to another grid, optionally captured in a CUDA graph and with its
launch shape tuned on the first batch of a layout.  The reference inverts
one cube on one grid per run (gmilos.cu:1008-1249).
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
    return idx, firsts


def invert_rois(engine, rois, psf_for_grid=None, use_graph=False, autotune=False):
    """Invert a ragged batch.  rois: list of (iquv [P_i][4][nl_i] float32,
    lambda [nl_i] absolute wavelengths); psf_for_grid(lam) gives the PSF taps
    of a grid (None: no PSF).  The engine must be configured (line, weights,
    free parameters, stop rule; its grid is not used).  Grids that agree to
    GRID_ATOL share one configuration.  Returns one output dict per ROI
    (model, chi2, iters, status) and the batch statistics (pixels, grids,
    launches, lane_occupancy, device_ms, graph_replayed, tuned limits)."""
    idx, firsts = group_grids([lam for _, lam in rois])
    psfs = [None if psf_for_grid is None else psf_for_grid(f) for f in firsts]
    batch = []
    for i, (iquv, lam) in enumerate(rois):
        a = iquv if hasattr(iquv, "data_ptr") else np.ascontiguousarray(iquv, dtype=np.float32)
        if a.ndim != 3 or a.shape[1] != 4 or a.shape[2] != len(lam):
            raise ValueError("ROI %d: iquv must be [P][4][nl] on its own grid" % i)
        batch.append((a, firsts[idx[i]], psfs[idx[i]]))
    return engine.invert_rois(batch, use_graph=use_graph, autotune=autotune)
