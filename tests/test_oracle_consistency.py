"""Structural checks of the 1D oracle's RHS where no reference output pins it (HS3,
HS1, the varying-depth operator): with the aliasing mask fixed (cutfrac 4 for every
model), the models differ only by their nonlinear terms, so on the same state and
time -- source, damping, delta H1 and the adjustment mask identical -- HS3 minus HS2 is
homogeneous of degree three in the state and HS2 minus HS1 of degree two, and HS1 is
affine (linear plus the source)."""
import numpy as np
import pytest

import oracle_lib as ol
from decks_util import random_state, rel_l2, small_deck

NX = 512


def _rhs(deck, t, y):
    o = ol.Oracle(deck)
    r = o.rhs(t, y)
    o.close()
    return r


@pytest.mark.parametrize("varying", [False, True])
def test_hs3_minus_hs2_is_cubic(tmp_path, varying):
    d2 = small_deck(tmp_path, "h2", nx=NX, model="HS2", varying=varying, cutfrac=4)
    d3 = small_deck(tmp_path, "h3", nx=NX, model="HS3", varying=varying, cutfrac=4)
    y = random_state(NX, 5)
    diff = lambda s: _rhs(d3, 1.3, s * y) - _rhs(d2, 1.3, s * y)
    full, half = diff(1.0), diff(0.5)
    assert np.linalg.norm(full) > 0
    assert rel_l2(8 * half, full) < 1e-9


@pytest.mark.parametrize("varying", [False, True])
def test_hs2_minus_hs1_is_quadratic(tmp_path, varying):
    d1 = small_deck(tmp_path, "h1", nx=NX, model="HS1", varying=varying, cutfrac=4)
    d2 = small_deck(tmp_path, "h2", nx=NX, model="HS2", varying=varying, cutfrac=4)
    y = random_state(NX, 6)
    diff = lambda s: _rhs(d2, 0.9, s * y) - _rhs(d1, 0.9, s * y)
    full, half = diff(1.0), diff(0.5)
    assert np.linalg.norm(full) > 0
    assert rel_l2(4 * half, full) < 1e-9


@pytest.mark.parametrize("varying", [False, True])
def test_hs1_is_affine(tmp_path, varying):
    d1 = small_deck(tmp_path, "h1", nx=NX, model="HS1", varying=varying, cutfrac=4)
    y1, y2 = random_state(NX, 7), random_state(NX, 8)
    r0 = _rhs(d1, 2.1, np.zeros(4 * NX))
    lhs = _rhs(d1, 2.1, y1 + y2) - r0
    rhs_ = (_rhs(d1, 2.1, y1) - r0) + (_rhs(d1, 2.1, y2) - r0)
    assert rel_l2(lhs, rhs_) < 1e-12
