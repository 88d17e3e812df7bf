"""The reference's own 1D test decks, run through the device engine and the oracle
with the reference's tolerances (1d/functions.c:529-541): the drop-in claim on the
decks a reference user already has.  Each deck runs through its output samples to
reference_decks.WINDOW (up to a few thousand steps, inside the range where two
roundings of the same arithmetic keep identical step sequences): identical accepted
and rejected counts, eta and u within 1e-9, and on the breaking deck the same
breaking.dat records."""
import concurrent.futures as cf

import numpy as np
import pytest

import oracle_lib as ol
from decks_util import rel_l2
from reference_decks import WINDOW, unpack

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")


def _physical(y):
    n = y.size // 4
    return np.fft.ifft(y[:n] + 1j * y[n:2 * n]).real, np.fft.ifft(y[2 * n:3 * n] + 1j * y[3 * n:]).real


def _oracle_run(deck, t_stop):
    o = ol.Oracle(deck)
    tt = o.table("ttrace")
    y = o.initial_state()
    t, h = float(tt[0]), 1e-4
    i = 1
    while i < tt.size and tt[i] <= tt[0] + t_stop:
        while t < tt[i]:
            t, h = o.evolve_apply(t, tt[i], h, y)
        i += 1
    out = (i, t, y, tuple(o.stats()), o.breaking_log())
    o.close()
    return out


def _log_lines(recs):
    return [[f"{t:f}", str(len(nodes))] + [str(n) for n in nodes] for t, nodes in recs]


def test_reference_decks_match_oracle(tmp_path):
    decks = unpack(tmp_path)
    names = sorted(WINDOW)
    with cf.ThreadPoolExecutor(8) as ex:   # ctypes releases the GIL
        refs = dict(zip(names, ex.map(lambda n: _oracle_run(decks[n], WINDOW[n]), names)))
    any_breaking = False
    for name in names:
        i_stop, t, y, (rhs, acc, rej), log = refs[name]
        e = hw.Engine(decks[name])
        e.run(i_stop=i_stop)
        tg, _, yg = e.state()
        st = e.stats()
        assert st["status"] == 0, name
        assert tg == pytest.approx(t, rel=1e-13), name
        assert (st["accepted"], st["rejected"]) == (acc, rej), (name, st, acc, rej)
        (eo, uo), (eg, ug) = _physical(y), _physical(yg)
        assert rel_l2(eg, eo) < 1e-9 and rel_l2(ug, uo) < 1e-9, (name, rel_l2(eg, eo), rel_l2(ug, uo))
        gold = [l.split() for l in log.splitlines()]
        assert _log_lines(e.breaking_log()) == gold, name
        any_breaking = any_breaking or bool(gold)
        e.close()
    assert any_breaking   # the barred breaking deck starts breaking inside its window

