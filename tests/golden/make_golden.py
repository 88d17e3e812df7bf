"""Regenerate the golden fixtures in this folder from the reference's shipped
test decks (run in a container where the reference checkout is mounted).

    python tests/golden/make_golden.py /path/to/reference

The reference checkout is the first argument, or $HAWASSI_REFERENCE.

Fixtures written (all are reference *outputs or inputs*, no reference code):
  fbr005/            input deck of 1d/Testcases/1dFBr005Bor/Input (input.txt,
                     initial.dat, gauges.dat)
  fbr005_breaking_head.txt   first 40 lines of Output/breaking.dat
  fbr005_gauge_head.txt      Output/Hawassi_eta_gauge.txt rows with t <= 13.0
  fbr005_constants.npz       x, t, depth, k, nu_peak of Output/Constants_01.dat
  irslope_constants.npz      x, k, depth, nu_peak of 1dB001IrSlope Constants_01.dat
  harmbar/           input deck of 1d/Testcases/1dB002HarmBar (input.txt, bath.dat,
                     influx.dat, gauges.dat): HS2 over a submerged bar (varying
                     bathymetry through three reference depths), Area influx of a
                     user-defined signal, adjcoef 0.3
  harmbar_gauges.npz         output/Hawassi_eta_gauge.txt and Hawassi_dteta_gauge.txt
                             (gauge positions; all 5000 rows as printed with %f,
                             stored as integers of 1e-6)
  harmbar_constants.npz      x, t, depth, k, nu_peak of output/Constants_01.dat
  reference_decks.tar.gz     the input decks (input.txt and the .dat files it names) of
                             the reference's other 1D test cases that stay inside the
                             hot path: flat and barred bottoms, HS2 and HS3, breaking,
                             Area and AreaShort influx, an initial-value bore
                             (REFERENCE_DECKS below)
"""
import io
import os
import shutil
import sys
import tarfile

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
    harmbar(ref)
    reference_decks(ref)


# 1d/Testcases decks (input files only) for the deck-by-deck parity test
REFERENCE_DECKS = ("1dB003IrBar", "1dBBr002IrBar", "1dF001Foc", "1dF002Draup", "1dF003Irreg", "1dF006Bor",
                   "1dFBr001Foc", "1dFBr002Foc", "1dFBr003Bi", "1dFBr004Ir")


def reference_decks(ref):
    out = os.path.join(HERE, "reference_decks.tar.gz")
    with tarfile.open(out, "w:gz") as tar:
        for name in REFERENCE_DECKS:
            src = os.path.join(ref, "1d", "Testcases", name)
            for f in sorted(os.listdir(src)):
                if f == "input.txt" or f.endswith(".dat"):
                    with open(os.path.join(src, f), "rb") as fi:
                        data = fi.read()
                    info = tarfile.TarInfo(f"{name}/{f}")
                    info.size = len(data)
                    info.mtime = 0
                    tar.addfile(info, io.BytesIO(data))


def read_gauge_text(path):
    """A Hawassi_*_gauge.txt file: header '#0 x1 x2 ...' (or '0 x1 ...'), then rows t g1 g2 ..."""
    with open(path) as f:
        head = f.readline().replace("#", " ").split()
    rows = np.loadtxt(path, skiprows=1)
    return np.array([float(v) for v in head[1:]]), rows


def harmbar(ref):
    src = os.path.join(ref, "1d", "Testcases", "1dB002HarmBar")
    dst = os.path.join(HERE, "harmbar")
    os.makedirs(dst, exist_ok=True)
    for f in ("input.txt", "bath.dat", "influx.dat", "gauges.dat"):
        shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
    xg, eta = read_gauge_text(os.path.join(src, "output", "Hawassi_eta_gauge.txt"))
    _, dteta = read_gauge_text(os.path.join(src, "output", "Hawassi_dteta_gauge.txt"))
    # the files print %f: stored exactly as integers of 1e-6 (micro_eta / 1e6 is the printed value)
    assert np.abs(eta).max() < 2000 and np.abs(dteta).max() < 2000
    np.savez_compressed(os.path.join(HERE, "harmbar_gauges.npz"), xgauge=xg,
                        micro_t=np.rint(eta[:, 0] * 1e6).astype(np.int64),
                        micro_eta=np.rint(eta[:, 1:] * 1e6).astype(np.int32),
                        micro_dteta=np.rint(dteta[:, 1:] * 1e6).astype(np.int32))
    c = read_constants(os.path.join(src, "output", "Constants_01.dat"))
    np.savez_compressed(os.path.join(HERE, "harmbar_constants.npz"), **c)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HAWASSI_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set HAWASSI_REFERENCE)")
    main(ref)
