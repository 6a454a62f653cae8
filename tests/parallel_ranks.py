"""One rank of the multi-process tests of gmilos_b200.parallel (CPU, gloo).

Run as two processes with RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT set;
argv[1] names the case.  Rank 0 prints one line starting with RESULT."""
import datetime
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "g-milos_b200"))

import torch.distributed as dist  # noqa: E402

from gmilos_b200 import parallel  # noqa: E402


class FakeEngine:
    """Stands in for the GPU engine: deterministic outputs per pixel."""

    def invert(self, iquv):
        s = iquv.reshape(len(iquv), -1).astype(np.float64).sum(axis=1)
        return {"model64": s[:, None] * np.arange(1, 12)[None, :], "chi2": (s * 0.5).astype(np.float32),
                "iters": (np.abs(s * 1000).astype(np.int64) % 7).astype(np.int32) + 1,
                "status": np.full(len(iquv), 2, np.uint32)}


def main():
    case = sys.argv[1]
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    if case == "gather":
        for npix in (11, 1, 0, 64):
            a, b = parallel.pixel_range(npix, rank, world)
            local = np.arange(a, b, dtype=np.float32)[:, None] * np.array([[1.0, -2.0, 3.0]], np.float32)
            full = parallel.gather_rows(local, npix)
            if rank == 0:
                want = np.arange(npix, dtype=np.float32)[:, None] * np.array([[1.0, -2.0, 3.0]], np.float32)
                assert full.shape == want.shape and np.array_equal(full, want), npix
            else:
                assert full is None
        if rank == 0:
            print("RESULT ok")
    elif case == "invert":
        rng = np.random.default_rng(3)
        cube = rng.normal(size=(37, 4, 30)).astype(np.float32)   # every rank holds the cube
        out = parallel.invert_sharded(FakeEngine(), cube)
        if rank == 0:
            ref = FakeEngine().invert(cube)
            for k, v in ref.items():
                assert np.array_equal(out[k], v), k
            print("RESULT ok")
        else:
            assert out is None
    elif case == "max":
        m = parallel.max_over_ranks(1.5 + rank)
        if rank == 0:
            print("RESULT %.3f" % m)
    elif case == "failure":
        # rank 1 leaves between steps, before the gather; rank 0 must learn it
        # from a short host-group timeout instead of waiting for ever
        group = parallel.host_group(timeout_s=3)
        if rank == 1:
            os._exit(0)
        try:
            parallel.gather_rows(np.zeros((6, 2), np.float32), 11, group=group)
            print("RESULT no-error")
        except Exception as e:   # gloo reports the lost peer or the timeout
            print("RESULT detected %s" % type(e).__name__)
        os._exit(0)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
