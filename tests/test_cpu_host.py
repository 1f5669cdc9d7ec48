"""Host-side logic of the product without a GPU: input.nn set-up through the
C ABI (symmetry-function order, derivative tables, scaling, network
topology), error codes of the reference's failure modes, input.data I/O and
the seeded workload generator."""
import os
import tempfile

import numpy as np
import pytest

from n2p2_b200 import _lib, read_structures, water
from n2p2_b200.mode import Mode
from oracle import port
from oracle import ref as oref
from tests import helpers as H

MODELS = [os.path.join(H.GOLDEN, "examples", "H2O_RPBE-D3"), os.path.join(H.GOLDEN, "examples", "Cu2S_PBE"),
          H.WATER40, H.WATER56]


@pytest.mark.skipif(not port.available(), reason="C restatement not built")
@pytest.mark.parametrize("model", MODELS)
def test_setup_matches_restatement(model):
    """Sorted SF table, rows per neighbour element and scaling factors equal
    the oracle's independent set-up."""
    m = Mode(0)
    m.setupFromDirectory(model)
    pm = port.PortModel(model)
    a = pm.arrays
    assert m.numElements == len(pm.symbols)
    for e in range(m.numElements):
        assert m.elementSymbol(e) == pm.symbols[e]
        b0, b1 = a["sfBegin"][e], a["sfBegin"][e + 1]
        assert m.numSymmetryFunctions(e) == b1 - b0
        for i in range(b1 - b0):
            t, e1, e2, eta, rs, lam, zeta, rc, sf = m.symmetryFunction(e, i)
            s = b0 + i
            assert t == a["type"][s] and e1 == a["e1"][s]
            if t != 2:
                assert e2 == a["e2"][s] and lam == a["lambda_"][s] and zeta == a["zeta"][s]
            assert eta == a["eta"][s] and rs == a["rs"][s] and rc == a["rc"][s]
            assert sf == a["scalingFactor"][s]
        for en in range(m.numElements):
            assert m.numDerivativeRows(e, en) == a["numRows"][e * m.numElements + en]
    assert m.getMaxCutoffRadius() == pm.maxCutoff
    m.close()


def _settings(text):
    d = tempfile.mkdtemp()
    p = os.path.join(d, "input.nn")
    open(p, "w").write(text)
    return p


def test_duplicate_keyword_is_critical():
    m = Mode(0)
    p = _settings("number_of_elements 1\nelements H\nelements H\n")
    with pytest.raises(_lib.N2P2Error) as e:
        m.loadSettingsFile(p)
    assert e.value.code == _lib.ERR_RUNTIME
    assert "critical" in str(e.value)


def test_unsupported_generation_and_types_are_rejected():
    m = Mode(0)
    with pytest.raises(_lib.N2P2Error):
        m.loadSettingsFile(_settings("nnp_type 4G-HDNNP\nnumber_of_elements 1\nelements H\n"))
    m2 = Mode(0)
    m2.loadSettingsFile(_settings("number_of_elements 1\nelements H\ncutoff_type 2\n"
                                  "global_hidden_layers_short 1\nglobal_nodes_short 2\n"
                                  "global_activation_short t l\nsymfunction_short H 12 0.5 0.0 5.0\n"))
    with pytest.raises(_lib.N2P2Error) as e:
        m2.setupGeneric()
    assert "not supported" in str(e.value)


def test_invalid_cutoff_parameter_maps_to_invalid_argument():
    m = Mode(0)
    m.loadSettingsFile(_settings("number_of_elements 1\nelements H\ncutoff_type 6 1.5\n"
                                 "global_hidden_layers_short 1\nglobal_nodes_short 2\n"
                                 "global_activation_short t l\nsymfunction_short H 2 H 0.1 0.0 5.0\n"))
    with pytest.raises(_lib.InvalidArgumentError):
        m.setupGeneric()


def test_missing_weights_file_is_reported():
    m = Mode(0)
    m.loadSettingsFile(os.path.join(H.WATER40, "input.nn"))
    m.setupGeneric()
    with pytest.raises(_lib.N2P2Error) as e:
        m.setupNeuralNetworkWeights("/nonexistent/weights.%03zu.data")
    assert "Could not open" in str(e.value)


def test_structure_text_round_trip_is_exact():
    s = water.water_box(8, seed=2, sigma=0.1)
    t = read_structures(s.to_text(), is_text=True)[0]
    assert np.array_equal(t.positions.view(np.int64), s.positions.view(np.int64))
    assert np.array_equal(t.box, s.box)
    assert t.elements == s.elements


def test_water_generator_recipe():
    s = water.water_box(64, seed=0)
    assert s.numAtoms == 192
    assert abs(s.box[0, 0] - 23.47) < 0.01
    p = s.positions.reshape(-1, 3, 3)
    oh1 = np.linalg.norm(p[:, 1] - p[:, 0], axis=1)
    oh2 = np.linalg.norm(p[:, 2] - p[:, 0], axis=1)
    assert np.allclose(oh1, 1.81) and np.allclose(oh2, 1.81)
    cosang = np.einsum("ij,ij->i", p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]) / (oh1 * oh2)
    assert np.allclose(np.degrees(np.arccos(cosang)), 104.5)
    b1 = water.water_batch(16, seed=1)
    b2 = water.water_batch(16, seed=1)
    assert all(np.array_equal(x.positions, y.positions) for x, y in zip(b1, b2))
    n = np.array([x.numAtoms // 3 for x in water.water_batch(400, seed=9)])
    assert n.min() >= 32 and n.max() <= 512


@pytest.mark.skipif(not oref.available(), reason="reference library not built")
@pytest.mark.parametrize("name", ["examples/Anisole_SCAN", "examples/DMABN_SCAN", "examples/Ethylbenzene_SCAN",
                                  "models/qm9_weighted", "models/scan_narrow"])
def test_compact_models_set_up_like_the_reference(name):
    """Compact symmetry functions (types 20-25): per element the number of
    functions, the derivative rows per neighbour element (every element for
    the weighted types) and the largest cutoff equal the reference library's
    set-up of the same files."""
    d = os.path.join(H.GOLDEN, name)
    m = Mode(0)
    m.setupFromDirectory(d)
    r = oref.RefPrediction(d)
    try:
        ne = m.numElements
        assert ne == r.num_elements
        for e in range(ne):
            assert m.numSymmetryFunctions(e) == r.num_sf(e)
            for f in range(ne):
                assert m.numDerivativeRows(e, f) == r.num_rows(e, f)
        assert m.getMaxCutoffRadius() == r.max_cutoff
    finally:
        r.close()
        m.close()
