"""Every cutoff function and every activation function on the GPU against
the reference.

1. The device's CutoffFunction::fdf of all nine types at the reference's own
   known answers (test/cpp/test_CutoffFunction.cpp: r = 2.4, rc = 3,
   alpha = 0.2; committed in tests/golden/cutoff_functions.json), within the
   reference test's accuracy of 100 DBL_EPSILON, and the FP32 per-triplet
   form of the mixed kernels within FP32 rounding of the FP64 values over
   the whole range.  The cos type's derivative keeps the reference's
   sqrt(1 - cos^2) form (CutoffFunction.cpp:128-139), so the device agrees
   with the reference where that form loses digits (x near 0 and 1) too.
2. Whole models through the reference library: the water model with each
   cutoff type (inner cutoff alpha = 0.2 where the type has one) and with
   each activation in the hidden layers (NeuralNetwork.cpp:794-837), FP64
   energies within 1e-10 relative and forces within 1e-10 of the largest
   component (or twice the reference's own FMA/no-FMA spread, as in the other
   water parity tests); the cutoff variants also in the mixed form, within
   1 meV/atom and 30 meV/A.
"""
import ctypes
import json
import os
import shutil

import numpy as np
import pytest

from n2p2_b200 import _lib
from n2p2_b200 import water
from n2p2_b200.scaling import collect_statistics, write_scaling
from tests import helpers as H

pytestmark = pytest.mark.gpu

_P = ctypes.POINTER(ctypes.c_double)


def _device_cutoff(kind, rc, alpha, r, precision=0):
    lib = _lib.load()
    r = np.ascontiguousarray(r, dtype=np.float64)
    f, df = np.zeros_like(r), np.zeros_like(r)
    _lib.check(lib.n2p2_cutoff_function(0, kind, rc, alpha, precision, r.ctypes.data_as(_P), r.size,
                                        f.ctypes.data_as(_P), df.ctypes.data_as(_P)))
    return f, df


def test_cutoff_functions_known_answers():
    gold = json.load(open(os.path.join(H.GOLDEN, "cutoff_functions.json")))
    acc = 100.0 * np.finfo(np.float64).eps
    for k, t in enumerate(gold["types"]):
        f, df = _device_cutoff(t, gold["rc"], gold["alpha"], [gold["r"]])
        assert abs(f[0] - gold["f"][k]) <= acc, (t, f[0], gold["f"][k])
        assert abs(df[0] - gold["df"][k]) <= acc, (t, df[0], gold["df"][k])


def test_cutoff_function_fp32_form():
    """The mixed kernels' f_c(r_jk): the factored polynomials (types 5-8),
    the hard cutoff, and the FP64 function rounded for the others, against
    the FP64 device values from r = 0 to past r_c (inner cutoff 0 and 0.2)."""
    rc = 12.0
    r = np.concatenate([np.linspace(0.0, 12.5, 20001), rc - np.logspace(-6, -1, 200)])
    for alpha in (0.0, 0.2):
        for t in range(9):
            # the hard cutoff's step moves with r's rounding to FP32: compare where it does not cross r_c
            rr = r[(r.astype(np.float32) < rc) == (r < rc)] if t == 0 else r
            f64, d64 = _device_cutoff(t, rc, alpha, rr, 0)
            f32, d32 = _device_cutoff(t, rc, alpha, rr, 1)
            # r itself is rounded to FP32 first: the bound is that rounding times the slope, plus FP32
            # evaluation error (16 ulps of the value: poly4 raises u to the fifth power), plus the FP64
            # expanded polynomial's own cancellation error near r_c (DBL_EPSILON times the sum of the
            # coefficients' magnitudes, ~4e-13 for poly4, where the function itself is ~1e-30; the
            # factored FP32 form does not cancel)
            slope = np.abs(d64) * np.abs(rr) * 6e-8
            assert np.all(np.abs(f32 - f64) <= slope + 2e-6 * np.abs(f64) + 1e-12), (t, alpha)
            scale = np.abs(d64).max() + 1e-300
            assert np.abs(d32 - d64).max() <= 1e-5 * scale, (t, alpha)
    with pytest.raises(_lib.InvalidArgumentError):
        _device_cutoff(6, rc, 1.0, [1.0])


CUTOFFS = [(0, 0.0), (1, 0.2), (2, 0.0), (3, 0.0), (4, 0.2), (5, 0.2), (6, 0.2), (7, 0.2), (8, 0.2)]
ACTIVATIONS = ["t t l", "s s l", "r r l", "g g l", "c c l", "S S l", "e e l", "h h l", "l l l", "p t s"]


def _variant(tmp_path, name, cutoff=None, activations=None, structures=None, normalize=False):
    """The water model with another cutoff or activation line (or with
    normalize_nodes); a changed cutoff gets scaling statistics of its own
    (nnp-scaling on the device over `structures`)."""
    d = str(tmp_path / name)
    shutil.copytree(H.WATER40, d)
    p = os.path.join(d, "input.nn")
    lines = []
    for ln in open(p):
        w = ln.split()
        if w and w[0] == "cutoff_type" and cutoff is not None:
            ln = "cutoff_type %d %.1f\n" % cutoff
        if w and w[0] == "global_activation_short" and activations is not None:
            ln = "global_activation_short %s\n" % activations
        lines.append(ln)
    if normalize:
        lines.append("normalize_nodes\n")
    open(p, "w").write("".join(lines))
    if cutoff is not None:
        from n2p2_b200 import Mode
        m = Mode(0)
        m.initialize()
        m.loadSettingsFile(p)
        m.setupGeneric()
        m.setupSymmetryFunctionScalingNone()
        write_scaling(os.path.join(d, "scaling.data"), collect_statistics(m, structures))
        m.close()
    return d


def _structures():
    return [water.water_box(32, seed=41), water.water_box(48, seed=42, sigma=0.1)]


def _check(d, structures, precision="fp64"):
    m = H.gpu_mode(d, precision=precision)
    b = H.gpu_batch(m, structures)
    E, F = b.energies(), b.forces()
    a0 = 0
    for k, s in enumerate(structures):
        snap = H.reference_snapshot(d, s)
        f = F[a0:a0 + s.numAtoms]
        if precision == "fp64":
            e_noise, f_noise = H.reference_noise(d, s)
            assert abs(E[k] - snap["energy"]) <= max(1e-10, 2 * e_noise) * abs(snap["energy"]), k
            assert H.max_rel(f, snap["forces"]) <= max(1e-10, 2 * f_noise), k
        else:
            assert abs(E[k] - snap["energy"]) / s.numAtoms * H.HA_TO_MEV <= 1.0, k
            assert np.abs(f - snap["forces"]).max() * H.HA_PER_BOHR_TO_MEV_PER_A <= 30.0, k
        a0 += s.numAtoms
    m.close()


@pytest.mark.parametrize("cutoff", CUTOFFS, ids=["type%d" % c[0] for c in CUTOFFS])
def test_cutoff_type_models(tmp_path, cutoff):
    ss = _structures()
    d = _variant(tmp_path, "cut%d" % cutoff[0], cutoff=cutoff, structures=ss)
    _check(d, ss, "fp64")
    _check(d, ss, "mixed")


@pytest.mark.parametrize("act", ACTIVATIONS, ids=[a.replace(" ", "") for a in ACTIVATIONS])
def test_activation_models(tmp_path, act):
    ss = _structures()
    d = _variant(tmp_path, "act_" + act.replace(" ", "_"), activations=act)
    _check(d, ss, "fp64")


def test_normalize_nodes_model(tmp_path):
    """normalize_nodes: every neuron's weighted input sum divided by the
    number of neurons feeding it (NeuralNetwork::propagateLayer,
    NeuralNetwork.cpp:761-790), and the same divisions in dE/dG
    (calculateDEdG, NeuralNetwork.cpp:396-442).  The water model with the
    keyword, FP64 (the tiled network kernel) against the reference library;
    the mixed form runs its networks in FP64 for such models (the
    tensor-core kernel does not take them)."""
    ss = _structures()
    d = _variant(tmp_path, "normalize", normalize=True)
    _check(d, ss, "fp64")
    _check(d, ss, "mixed")


def test_one_hidden_layer_energies_only(tmp_path):
    """A network with one hidden layer (40-25-1: an even number of weight
    layers, so the tiled network kernel's output lands in the buffer the next
    tile loads) on 48 boxes of 128 molecules: more tiles than resident blocks,
    so blocks evaluate several tiles in turn.  Seeded weights; energies of an
    energy-only evaluation and energies and forces of a full one against the
    reference library."""
    d = str(tmp_path / "hidden1")
    shutil.copytree(H.WATER40, d)
    p = os.path.join(d, "input.nn")
    lines = []
    for ln in open(p):
        w = ln.split()
        if w and w[0] == "global_hidden_layers_short":
            ln = "global_hidden_layers_short 1\n"
        elif w and w[0] == "global_nodes_short":
            ln = "global_nodes_short 25\n"
        elif w and w[0] == "global_activation_short":
            ln = "global_activation_short p l\n"
        lines.append(ln)
    open(p, "w").write("".join(lines))
    rng = np.random.default_rng(17)
    for z in (1, 8):
        w = rng.normal(scale=0.3, size=40 * 25 + 25 + 25 + 1)
        with open(os.path.join(d, "weights.%03d.data" % z), "w") as f:
            f.write("# seeded weights of a 40-25-1 network\n")
            f.write("".join("%24.16E\n" % x for x in w))
    ss = [water.water_box(128, seed=200 + k) for k in range(48)]
    m = H.gpu_mode(d)
    b = m.batch(ss)
    b.setPositions(np.concatenate([s.positions for s in ss]))
    b.evaluate(forces=False)
    E0 = b.energies()
    b.evaluate(forces=True)
    E, F = b.energies(), b.forces()
    E_ref, F_ref = H.reference_energies_forces(d, ss)
    a0 = 0
    for k, s in enumerate(ss):
        e_ref, f_ref = E_ref[k], F_ref[k]
        assert abs(E0[k] - e_ref) <= 1e-10 * abs(e_ref), k
        assert abs(E[k] - e_ref) <= 1e-10 * abs(e_ref), k
        assert H.max_rel(F[a0:a0 + s.numAtoms], f_ref) <= 1e-10, k
        a0 += s.numAtoms
    m.close()
