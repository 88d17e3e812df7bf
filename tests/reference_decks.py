"""The reference's own 1D test decks (1d/Testcases, input files only), unpacked from
tests/golden/reference_decks.tar.gz (made by tests/golden/make_golden.py).

WINDOW is how far each deck is run in the deck-by-deck parity test: long enough to
reach the waves' arrival over the bar or the breaking onset where the deck has one,
short enough for the oracle to finish in seconds."""
import os
import tarfile

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ARCHIVE = os.path.join(GOLDEN, "reference_decks.tar.gz")

# deck -> simulated seconds of the parity run
WINDOW = {
    "1dB003IrBar": 20.0,      # HS2, user-defined bar, AreaShort influx
    "1dBBr002IrBar": 15.0,    # HS2 over a bar with breaking (onset at 14.86 s), AreaShort
    "1dF001Foc": 20.0,        # HS2 flat, focusing wave group, Area
    "1dF002Draup": 20.0,      # HS2 flat, Draupner-type group, AreaShort
    "1dF003Irreg": 20.0,      # HS2 flat, irregular waves, AreaShort
    "1dF006Bor": 20.0,        # HS2 flat, initial-value bore (initial.dat)
    "1dFBr001Foc": 10.0,      # HS3 flat with breaking enabled, Nx 8192
    "1dFBr002Foc": 20.0,      # HS3 flat with breaking enabled
    "1dFBr003Bi": 20.0,       # HS3 flat, bichromatic group with breaking enabled, AreaShort
    "1dFBr004Ir": 20.0,       # HS2 flat, irregular waves with breaking enabled, AreaShort
}


def unpack(root):
    """Extract every deck under root; returns {name: deck directory}."""
    with tarfile.open(ARCHIVE) as tar:
        tar.extractall(root, filter="data")
        names = sorted({m.name.split("/")[0] for m in tar.getmembers()})
    return {n: os.path.join(str(root), n) + os.sep for n in names}
