"""Several GPUs as replicas (gmilos_b200.parallel): the pixel partition, the
host-side gather in pixel order, the max-over-ranks timing rule, and a rank
that leaves before the gather.  Two gloo ranks on CPU stand in for two
GPUs; a deterministic stand-in replaces the engine."""
import os
import socket
import subprocess
import sys

import pytest

from gmilos_b200 import parallel

HERE = os.path.dirname(os.path.abspath(__file__))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(case, world=2, timeout=120):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "parallel_ranks.py"), case],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    try:
        for p in procs:
            o, e = p.communicate(timeout=timeout)
            outs.append((p.returncode, o, e))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    return outs


def result_of(outs):
    lines = [l for l in outs[0][1].splitlines() if l.startswith("RESULT")]
    assert lines, outs[0][2][-2000:]
    return lines[-1][len("RESULT "):]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_pixel_range_partitions_every_cube(world):
    for npix in (0, 1, 2, 5, 7, 100, 1001, 1048576):
        ranges = [parallel.pixel_range(npix, r, world) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == npix
        for (a, b), (c, d) in zip(ranges, ranges[1:]):
            assert b == c and a <= b
        sizes = [b - a for a, b in ranges]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        parallel.pixel_range(10, 2, 2)


def test_gather_in_pixel_order_with_uneven_and_empty_ranges():
    outs = run_ranks("gather")
    assert all(rc == 0 for rc, _, _ in outs), [e[-2000:] for _, _, e in outs]
    assert result_of(outs) == "ok"


def test_sharded_inversion_equals_one_process():
    outs = run_ranks("invert")
    assert all(rc == 0 for rc, _, _ in outs), [e[-2000:] for _, _, e in outs]
    assert result_of(outs) == "ok"


def test_max_over_ranks():
    outs = run_ranks("max")
    assert all(rc == 0 for rc, _, _ in outs)
    assert result_of(outs) == "2.500"


def test_a_rank_that_leaves_is_detected_on_the_host():
    outs = run_ranks("failure", timeout=90)
    assert result_of(outs).startswith("detected")
