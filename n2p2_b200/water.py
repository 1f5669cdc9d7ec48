"""Seeded synthetic water workloads and n2p2 model-file writers.

The benchmark configurations are water boxes at 1.0 g/cm^3 (0.0049534
molecules/bohr^3): molecules on a jittered simple-cubic lattice, random
orientations, O-H 1.81 bohr, H-O-H 104.5 degrees, optional Gaussian thermal
displacement.  Everything is generated from a numpy seed, so every consumer
(GPU path, CPU baselines, tests) sees bit-identical positions.
"""
import math

import numpy as np

from .structure import Structure

MOLECULE_DENSITY = 0.0049534       # H2O per bohr^3 at 1.0 g/cm^3
OH_BOND = 1.81                     # bohr
HOH_ANGLE = 104.5                  # degrees


def box_edge(n_mol):
    return (n_mol / MOLECULE_DENSITY) ** (1.0 / 3.0)


def _rotations(q):
    """Rotation matrices [n,3,3] from unnormalised quaternions [n,4]."""
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], axis=1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], axis=1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], axis=1)], axis=1)


def water_box(n_mol, seed, jitter=0.5, sigma=0.0):
    """One periodic cubic water box; atoms ordered O, H, H per molecule."""
    rng = np.random.default_rng(seed)
    L = box_edge(n_mol)
    m = max(1, int(round(n_mol ** (1.0 / 3.0))))
    while m ** 3 < n_mol:
        m += 1
    sites = np.sort(rng.permutation(m ** 3)[:n_mol])
    a = L / m
    half = math.radians(HOH_ANGLE) / 2.0
    h1 = OH_BOND * np.array([math.sin(half), 0.0, math.cos(half)])
    h2 = OH_BOND * np.array([-math.sin(half), 0.0, math.cos(half)])
    grid = np.stack([sites // (m * m), (sites // m) % m, sites % m], axis=1).astype(np.float64)
    o = (grid + 0.5) * a + rng.uniform(-jitter, jitter, (n_mol, 3))
    R = _rotations(rng.normal(size=(n_mol, 4)))
    pos = np.empty((n_mol, 3, 3))
    pos[:, 0] = o
    pos[:, 1] = o + R @ h1
    pos[:, 2] = o + R @ h2
    pos = pos.reshape(-1, 3)
    if sigma > 0.0:
        pos += rng.normal(0.0, sigma, pos.shape)
    elements = ["O", "H", "H"] * n_mol
    return Structure(pos, elements, np.diag([L, L, L]), comment=f"water n_mol={n_mol} seed={seed}")


def water_batch(num_boxes, seed, n_min=32, n_max=512, sigma=0.0, sigma_range=None):
    """Boxes with molecule counts log-uniform in [n_min, n_max]."""
    rng = np.random.default_rng(seed)
    counts = np.rint(np.exp(rng.uniform(math.log(n_min), math.log(n_max), num_boxes))).astype(int)
    out = []
    for b, n in enumerate(counts):
        sg = sigma if sigma_range is None else rng.uniform(*sigma_range)
        out.append(water_box(int(n), seed * 1000003 + b + 1, sigma=sg))
    return out


# ---------------------------------------------------------------------------
# model files (input.nn, weights.%03d.data, scaling.data)
# ---------------------------------------------------------------------------

G2_ETAS = [0.001, 0.01, 0.03, 0.06, 0.15, 0.3, 0.6, 1.5]
G3_ETAS = [0.01, 0.03]
G3_ZETAS = [1.0, 4.0]
G9_ETAS = [0.001, 0.01]
G9_ZETAS = [1.0, 2.0, 4.0, 16.0]
LAMBDAS = [-1.0, 1.0]
RC = 12.0


def symfunction_lines(g2_etas=G2_ETAS, g3_etas=G3_ETAS, g3_zetas=G3_ZETAS, g9=False, rc=RC,
                      g9_etas=G9_ETAS, g9_zetas=G9_ZETAS):
    out = []
    for ec in ("H", "O"):
        for e1 in ("H", "O"):
            for eta in g2_etas:
                out.append(f"symfunction_short {ec} 2 {e1} {eta:.6g} 0.0 {rc:.6g}")
        for e1, e2 in (("H", "H"), ("H", "O"), ("O", "O")):
            for eta in g3_etas:
                for lam in LAMBDAS:
                    for zeta in g3_zetas:
                        out.append(f"symfunction_short {ec} 3 {e1} {e2} {eta:.6g} {lam:.0f} {zeta:.6g} {rc:.6g}")
        if g9:
            for eta in g9_etas:
                for lam in LAMBDAS:
                    for zeta in g9_zetas:
                        out.append(f"symfunction_short {ec} 9 H O {eta:.6g} {lam:.0f} {zeta:.6g} {rc:.6g}")
    return out


def input_nn_text(sf_lines, nodes=(25, 25), activations="p p l", cutoff="6 0.0", scaling=True, comment=""):
    lines = [f"# {comment}" if comment else "# synthetic water HDNNP",
             "number_of_elements 2",
             "elements H O",
             f"cutoff_type {cutoff}"]
    if scaling:
        lines += ["scale_symmetry_functions", "center_symmetry_functions", "scale_min_short 0.0",
                  "scale_max_short 1.0"]
    lines += [f"global_hidden_layers_short {len(nodes)}",
              "global_nodes_short " + " ".join(str(n) for n in nodes),
              f"global_activation_short {activations}"]
    lines += sf_lines
    return "\n".join(lines) + "\n"


def random_weights(layer_sizes, rng):
    """Weights-file order (NeuralNetwork::setConnections): per layer, for each
    source neuron j, for each target k: w(k<-j); then the biases (zero).
    Weights ~ N(0, 1/fan_in)."""
    out = []
    for l in range(1, len(layer_sizes)):
        nin, nout = layer_sizes[l - 1], layer_sizes[l]
        w = rng.normal(0.0, math.sqrt(1.0 / nin), size=(nout, nin))
        for j in range(nin):
            for k in range(nout):
                out.append(w[k, j])
        out.extend([0.0] * nout)
    return np.array(out)


def write_weights(path, values):
    with open(path, "w") as f:
        f.write("#" + "#" * 79 + "\n# Neural network connection values (weights and biases).\n#" + "#" * 79 + "\n")
        for v in values:
            f.write("%24.16E\n" % v)


def write_scaling(path, stats):
    """stats: list over elements of arrays [numSF, 4] = min, max, mean, sigma."""
    with open(path, "w") as f:
        f.write("#" * 80 + "\n# Symmetry function scaling data.\n" + "#" * 80 + "\n")
        for e, st in enumerate(stats):
            for i, (mn, mx, mean, sg) in enumerate(st):
                f.write("%10d %10d %24.16E %24.16E %24.16E %24.16E\n" % (e + 1, i + 1, mn, mx, mean, sg))


def scaling_statistics(G_per_element):
    """min, max, mean and sigma with the n-1 denominator of
    Dataset::writeSymmetryFunctionScaling (Dataset.cpp:1065-1071)."""
    out = []
    for G in G_per_element:
        G = np.asarray(G, dtype=np.float64)
        n = G.shape[0]
        s = G.sum(axis=0)
        s2 = (G * G).sum(axis=0)
        mean = s / n
        sigma = np.sqrt((s2 - s * s / n) / (n - 1))
        out.append(np.stack([G.min(axis=0), G.max(axis=0), mean, sigma], axis=1))
    return out
