"""Renumbering of cells, edges and vertices (hexdyn.reorder).

A renumbered case steps exactly like the original: the oracle's step of the
renumbered 162-cell reference inputs, mapped back, equals the reference's
own step outputs word for word.  Renumbering twice with a permutation and
its inverse gives back every array; the Hilbert numbering of a scrambled
mesh restores neighbour locality.
"""

import numpy as np
import pytest

from fixtures import SIDE, STATE, differing_words, inputs, load_golden
from hexdyn import reorder
from oracle.dycore import OracleConfig, OracleDycore, State


def _same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.shape == y.shape and x.dtype == y.dtype, k
        assert np.array_equal(x, y), k


def test_permutation_and_inverse_restore_every_array():
    arr = inputs(load_golden("l2_L12"))
    ren = reorder.random_order(arr, seed=3)
    there = reorder.apply(arr, ren)
    assert not np.array_equal(there["mesh.cellsOnEdge"], arr["mesh.cellsOnEdge"])
    _same(reorder.apply(there, ren.inverse()), arr)


def test_unknown_arrays_are_refused():
    arr = inputs(load_golden("l2_L12"))
    ren = reorder.random_order(arr)
    with pytest.raises(ValueError):
        reorder.apply({**arr, "mystery": np.zeros(3)}, ren)
    bad = reorder.Renumbering(ren.cell[:-1], ren.edge, ren.vertex)
    with pytest.raises(ValueError):
        reorder.apply(arr, bad)


def test_connectivity_stays_consistent():
    arr = reorder.apply(inputs(load_golden("l2_L12")), reorder.random_order(inputs(load_golden("l2_L12")), seed=1))
    coe = arr["mesh.cellsOnEdge"]
    eoc = arr["mesh.edgesOnCell"]
    n = arr["mesh.nEdgesOnCell"]
    for c in range(eoc.shape[0]):
        for s in range(int(n[c])):
            assert c in coe[eoc[c, s]]
    adv = arr["adv_cells_for_edge"]
    nadv = arr["n_adv_cells_for_edge"]
    for e in range(adv.shape[0]):
        # the edge's own two cells lead its stencil
        assert set(coe[e]) <= set(adv[e, : int(nadv[e])])


def test_hilbert_order_restores_locality():
    arr = inputs(load_golden("l3_L20"))
    scrambled = reorder.apply(arr, reorder.random_order(arr, seed=5))
    ordered = reorder.apply(scrambled, reorder.hilbert_order(scrambled))
    s_bad, s_good = reorder.neighbour_spread(scrambled), reorder.neighbour_spread(ordered)
    assert s_good["edge"] < 0.25 * s_bad["edge"] and s_good["cell"] < 0.25 * s_bad["cell"], (s_bad, s_good)


@pytest.mark.parametrize("order", ["random", "hilbert"])
def test_renumbered_step_equals_reference(order):
    fx = load_golden("l2_L12")
    arr = inputs(fx)
    ren = reorder.random_order(arr, seed=11)
    if order == "hilbert":
        # scramble, then order along the curve: the composite renumbering
        hil = reorder.hilbert_order(reorder.apply(arr, ren))
        ren = reorder.Renumbering(ren.cell[hil.cell], ren.edge[hil.edge], ren.vertex[hil.vertex])
    moved = reorder.apply(arr, ren)
    orc = OracleDycore(moved, OracleConfig(dt=float(fx["config.dt"]), n_sub_steps=int(fx["config.n_sub_steps"]),
                                           moist="dry"))
    state, side = orc.step(State(*(moved[k].copy() for k in STATE)), None)
    back = ren.inverse()
    for k in STATE:
        got = reorder.field(getattr(state, k), k, back)
        assert differing_words(got, fx[f"dry.step1.{k}"]) == 0, k
    for k in SIDE:
        got = reorder.field(getattr(side, k), k, back)
        assert differing_words(got, fx[f"dry.step1.side.{k}"]) == 0, k
