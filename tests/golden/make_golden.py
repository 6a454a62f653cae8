"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run where the reference checkout exists (its path is the first argument, else
GM_REFERENCE_DIR, else a `reference` directory beside this repository); the
fixtures it writes are committed so that the tests never read the reference
at run time.

kat_synthesis.npz -- the reference's only shipped known-answer vector
(data/synthesis_gpu.per, produced by `gmilos run/synthesis.mtrol`) together
with the inputs that define it: the guess model run/init.mod, the grid of
run/malla.grid, the Fe I 6173.3356 line (run/LINES entry 1, 5P 1.0- 5D 0.0)
and the tabulated CRISP PSF run/CRISP_6173_1mA.psf.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_mod(path):
    keys = {"eta_0": 0, "magnetic field": 1, "LOS velocity": 2, "Doppler width": 3,
            "damping": 4, "gamma": 5, "phi": 6, "S_0": 7, "S_1": 8, "v_mac": 9,
            "filling factor": 10}
    m = np.zeros(11)
    for line in open(path):
        if ":" not in line:
            continue
        name, val = line.split(":", 1)
        val = float(re.match(r"\s*([-+0-9.eE]+)", val).group(1))
        for k, i in keys.items():
            if k in name:
                m[i] = val
    return m


def read_grid(path):
    lines = open(path).read().splitlines()
    for i, l in enumerate(lines):
        if l.startswith("------"):
            idx, rest = lines[i + 1].split(":", 1)
            a, b, c = [float(x) for x in rest.split(",")]
            return int(idx), a, b, c
    raise ValueError(path)


def main(ref):
    per = np.loadtxt(os.path.join(ref, "data", "synthesis_gpu.per"))
    model = read_mod(os.path.join(ref, "run", "init.mod"))
    idx, first, step, last = read_grid(os.path.join(ref, "run", "malla.grid"))
    psf = np.loadtxt(os.path.join(ref, "run", "CRISP_6173_1mA.psf"))
    line = [l for l in open(os.path.join(ref, "run", "LINES")) if l.startswith("%d=" % idx)][0]
    lambda0 = float(line.split()[2])
    np.savez_compressed(
        os.path.join(HERE, "kat_synthesis.npz"),
        per_offsets_mA=per[:, 1], per_iquv=per[:, 2:6].T.copy(), model=model,
        grid=np.array([first, step, last]), line_index=idx, lambda0=lambda0,
        quantum=np.array([2, 1, 1.0, 2, 2, 0.0]), mu=1.0,
        psf_x_mA=psf[:, 0], psf_y=psf[:, 1])
    print("wrote kat_synthesis.npz", per.shape, model, lambda0)


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
    from build_ref import locate_reference
    where = locate_reference(sys.argv[1] if len(sys.argv) > 1 else None)
    if where is None:
        sys.exit("reference checkout not found: pass its path or set GM_REFERENCE_DIR")
    main(where)
