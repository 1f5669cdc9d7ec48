"""The stages of Mode::evaluateNNP as separate C-ABI calls (Mode.h:298-378).

calculateNeighborList -> calculateSymmetryFunction[Groups] (derivatives) ->
calculateAtomicNeuralNetworks (derivatives) -> calculateEnergy ->
calculateForces must give the bits that one n2p2_batch_evaluate gives (same
kernels, same order), G and dE/dG must equal the reference library's (G
within 1e-12 of the largest |G|, dE/dG within 1e-10, the plain-FP64 bounds
of the other parity tests), and the reference's caching flags and stage
order hold.
"""
import numpy as np
import pytest

from n2p2_b200 import _lib
from n2p2_b200 import water
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.int64)


def _staged(m, boxes, derivatives=True):
    b = m.batch(boxes)
    b.setPositions(np.concatenate([s.positions for s in boxes]))
    b.calculateNeighborList()
    b.calculateSymmetryFunctionGroups(derivatives)
    b.calculateAtomicNeuralNetworks(True)
    b.calculateEnergy()
    b.calculateForces()
    return b


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stage_sequence_equals_evaluate(precision):
    boxes = water.water_batch(3, seed=31, n_min=32, n_max=96)
    m = H.gpu_mode(H.WATER40, precision=precision)
    full = H.gpu_batch(m, boxes)
    E0, F0, G0, D0 = full.energies(), full.forces(), full.symmetryFunctions(), full.dEdG()
    b = _staged(m, boxes)
    assert np.array_equal(_bits(b.energies()), _bits(E0))
    assert np.array_equal(_bits(b.forces()), _bits(F0))
    assert np.array_equal(_bits(b.symmetryFunctions()), _bits(G0))
    assert np.array_equal(_bits(b.dEdG()), _bits(D0))
    if precision == "fp64":
        G, D = b.symmetryFunctions(), b.dEdG()
        g0 = a0 = 0
        for s in boxes:
            snap = H.reference_snapshot(H.WATER40, s)
            g1 = g0 + snap["G"].size
            assert H.max_rel(H.unscaled(H.WATER40, s, G[g0:g1]), H.unscaled(H.WATER40, s, snap["G"])) <= 1e-12
            assert H.max_rel(D[g0:g1], snap["dEdG"]) <= 1e-10
            g0 = g1
            a0 += s.numAtoms


def test_stored_derivatives_stage():
    """derivatives = stored: Atom::dGdr / Atom::Neighbor::dGdr as the
    reference stores them (1e-11, as the stored-dG/dr parity test), and the
    forces contracted from them equal the stored-form evaluation's bits."""
    s = water.water_box(32, seed=1)
    m = H.gpu_mode(H.WATER40)
    full = m.batch([s])
    full.setPositions(s.positions)
    full.evaluate(forces=True, storeDGdr=True)
    F0 = full.forces()
    b = _staged(m, [s], derivatives="stored")
    assert np.array_equal(_bits(b.forces()), _bits(F0))
    snap = H.reference_snapshot(H.WATER40, s)
    selfd, nbr = b.dGdr(int(snap["row_offset"][-1]))
    assert H.max_rel(selfd, snap["dGdr_self"]) <= 1e-11
    assert H.max_rel(nbr, snap["dGdr_nbr"]) <= 1e-11


def test_stage_order_and_caching_flags():
    boxes = water.water_batch(2, seed=32, n_min=32, n_max=48)
    m = H.gpu_mode(H.WATER40)
    b = m.batch(boxes)
    pos = np.concatenate([s.positions for s in boxes])
    b.setPositions(pos)
    with pytest.raises(_lib.N2P2Error):
        b.calculateSymmetryFunctionGroups(True)          # no neighbour list yet
    b.calculateNeighborList()
    with pytest.raises(_lib.N2P2Error):
        b.calculateAtomicNeuralNetworks(True)            # no symmetry functions yet
    b.calculateSymmetryFunctionGroups(False)
    b.calculateAtomicNeuralNetworks(True)
    with pytest.raises(_lib.N2P2Error):
        b.calculateForces()                              # values only: no derivatives
    # hasSymmetryFunctions && !derivatives: the call returns at once, the
    # networks' results stay valid
    b.calculateSymmetryFunctionGroups(False)
    b.calculateEnergy()
    E_values = b.energies()
    # asking for derivatives recomputes (Mode.cpp:1634-1635) and invalidates the networks
    b.calculateSymmetryFunctionGroups(True)
    with pytest.raises(_lib.N2P2Error):
        b.calculateEnergy()
    b.calculateAtomicNeuralNetworks(True)
    b.calculateEnergy()
    b.calculateForces()
    assert np.array_equal(_bits(b.energies()), _bits(E_values))
    F = b.forces()
    # new positions clear every flag
    b.setPositions(pos)
    with pytest.raises(_lib.N2P2Error):
        b.calculateSymmetryFunctionGroups(True)
    # evaluate sets them: a symmetry-function call after it does nothing
    b.evaluate(forces=True)
    b.calculateSymmetryFunctionGroups(True)
    b.calculateForces()
    assert np.array_equal(_bits(b.forces()), _bits(F))
