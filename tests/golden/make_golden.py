"""Regenerate the golden fixtures in this folder from the reference's shipped
test decks (run in a container where the reference checkout is mounted).

    python tests/golden/make_golden.py /path/to/reference

Fixtures written (all are reference *outputs or inputs*, no reference code):
  fbr005/            input deck of 1d/Testcases/1dFBr005Bor/Input (input.txt,
                     initial.dat, gauges.dat)
  fbr005_breaking_head.txt   first 40 lines of Output/breaking.dat
  fbr005_gauge_head.txt      Output/Hawassi_eta_gauge.txt rows with t <= 13.0
  fbr005_constants.npz       x, t, depth, k, nu_peak of Output/Constants_01.dat
  irslope_constants.npz      x, k, depth, nu_peak of 1dB001IrSlope Constants_01.dat
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_constants(path):
    a = np.fromfile(path, dtype=np.float64)
    nx = int(a[0])
    x = a[1:1 + nx]
    nt = int(a[1 + nx])
    t = a[2 + nx:2 + nx + nt]
    rest = a[2 + nx + nt:]
    return dict(x=x, t=t, depth=rest[:nx], k=rest[nx:2 * nx], nu_peak=rest[2 * nx:2 * nx + 1])


def main(ref):
    src = os.path.join(ref, "1d", "Testcases", "1dFBr005Bor")
    dst = os.path.join(HERE, "fbr005")
    os.makedirs(dst, exist_ok=True)
    for f in ("input.txt", "initial.dat", "gauges.dat"):
        shutil.copyfile(os.path.join(src, "Input", f), os.path.join(dst, f))
    with open(os.path.join(src, "Output", "breaking.dat")) as fi, \
            open(os.path.join(HERE, "fbr005_breaking_head.txt"), "w") as fo:
        for i, line in enumerate(fi):
            if i >= 40:
                break
            fo.write(line)
    with open(os.path.join(src, "Output", "Hawassi_eta_gauge.txt")) as fi, \
            open(os.path.join(HERE, "fbr005_gauge_head.txt"), "w") as fo:
        for i, line in enumerate(fi):
            if i > 0 and float(line.split()[0]) > 13.0:
                break
            fo.write(line)
    c = read_constants(os.path.join(src, "Output", "Constants_01.dat"))
    np.savez_compressed(os.path.join(HERE, "fbr005_constants.npz"), **c)
    c = read_constants(os.path.join(ref, "1d", "Testcases", "1dB001IrSlope", "output", "Output", "Constants_01.dat"))
    np.savez_compressed(os.path.join(HERE, "irslope_constants.npz"),
                        x=c["x"], depth=c["depth"], k=c["k"], nu_peak=c["nu_peak"])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
