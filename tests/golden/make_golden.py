"""Generates the committed test fixtures under tests/golden/.

Run in the development container, where the reference tree is mounted:

    python tests/golden/make_golden.py [--reference DIR] [--examples-only]

DIR is the reference checkout ($N2P2_REFERENCE, else a directory named
"reference" beside this repository).

It writes
  examples/<name>/        the model and structure files of the reference's
                          prediction regression examples (H2O_RPBE-D3,
                          Cu2S_PBE, and the compact-function models
                          Anisole_SCAN, DMABN_SCAN, Ethylbenzene_SCAN;
                          reference examples/nnp-predict/<name>/)
                          plus golden.json with the energy and forces that the
                          reference's own regression test asserts
                          (test/cpp/ExamplePrediction.h, 1000 eps absolute).
  training/<name>/        the reference's nnp-train example H2O_RPBE-D3
                          (examples/nnp-train/<name>/) with golden.json: the
                          epoch-2 learning-curve RMSEs its regression test
                          asserts (test/cpp/Example_nnp_train.h, 1e-8 absolute).
  cutoff_functions.json   f and df of all cutoff types at r = 2.4, rc = 3,
                          alpha = 0.2 (test/cpp/test_CutoffFunction.cpp:17-52).
  models/water40/         the synthetic water model of the batched benchmark
                          (40 SFs per element, 40-25-25-1 softplus, poly2
                          cutoff, weights N(0, 1/fan_in) seeded), with
                          scaling statistics (the nnp-scaling recipe) over the
                          benchmark's single 64-molecule box plus 48 boxes of
                          the batched workload's recipe (32..128 molecules,
                          own seed) with 0.05 bohr Gaussian displacements,
                          computed by the reference library itself.  The
                          single box of rigid molecules alone gives several
                          functions a range of ~1e-8 (scaling factors up to
                          1e16): any two FP64 evaluations that round
                          differently, the reference's own FMA and non-FMA
                          builds included, then disagree far beyond the error
                          targets, and boxes with closer O-O pairs extrapolate
                          to forces of 1e4 Ha/bohr.
  models/water56/         the large-system model (+16 wide G9 on (H,O),
                          56-64-64-1 softplus), written here with scaling from
                          a 512-molecule box with 0.15 bohr displacements
                          (seed 3) plus 48 boxes of the student-training recipe
                          (64..128 molecules, 0.05..0.4 bohr displacements,
                          seed 777).  The committed scaling.data is then
                          rewritten on the GPU by
                            python -m n2p2_b200.student teacher-scaling \
                                --teacher tests/golden/models/water56
                          (nnp-scaling statistics of that box plus all 20,000
                          configurations of the student-training recipe,
                          seed 11: the teacher labels those configurations and
                          the held-out boxes come from the same recipe, so its
                          inputs stay inside its scaling range there).
  water40_box64.json      reference energy and forces of the 64-molecule box.
  models/qm9_weighted/    the reference's QM9 training settings
                          (examples/nnp-train/QM9/input.nn: weighted compact
                          types 23, 24, 25 on five elements) with its first 16
                          molecules and three more holding fluorine, seeded
                          random weights and scaling
                          statistics from the reference library over them
                          (functions constant over the sample get a unit
                          range and sigma).
  models/scan_narrow/     the Ethylbenzene_SCAN functions with every wide
                          angular function (22) turned narrow (21), plus two
                          "p1" members per group whose radial window equals
                          that of the first "p2" member (the reference then
                          carries the j-k radial part across the subtype
                          boundary); the example frame plus three copies with
                          0.02 displacements, seeded weights, reference
                          scaling.

The reference library is oracle/_ref/libnnpref.so (built by oracle/Makefile).
"""
import argparse
import json
import os
import re
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from n2p2_b200 import water  # noqa: E402
from oracle import ref  # noqa: E402

EXAMPLES = ["H2O_RPBE-D3", "Cu2S_PBE", "Anisole_SCAN", "DMABN_SCAN", "Ethylbenzene_SCAN"]


def parse_example_goldens(src, name):
    blk = src.split('ExamplePrediction("%s")' % name)[1].split("examples.push_back")[0]
    energy = float(re.search(r"e->energy = ([-0-9.E+]+);", blk).group(1))
    forces = [[float(x) for x in m] for m in
              re.findall(r"Vec3D\(\s*([-0-9.E+]+),\s*([-0-9.E+]+),\s*([-0-9.E+]+)\)", blk)]
    return energy, forces


def parse_cutoff_goldens(src):
    def arr(name):
        body = re.search(r"vector<double> const %s = \{(.*?)\};" % name, src, re.S).group(1)
        return [float(x) for x in re.findall(r"[-0-9.]+E[-+][0-9]+", body)]
    types = re.search(r"types = \{(.*?)\};", src, re.S).group(1)
    names = re.findall(r"CT_([A-Z0-9]+)", types)
    codes = {"HARD": 0, "COS": 1, "TANHU": 2, "TANH": 3, "EXP": 4, "POLY1": 5, "POLY2": 6, "POLY3": 7, "POLY4": 8}
    return {"rc": 3.0, "alpha": 0.2, "r": 2.4, "types": [codes[n] for n in names], "f": arr("f"), "df": arr("df"),
            "tolerance": "100 * DBL_EPSILON"}


def write_model(dirname, sf_lines, nodes, seed, stats_structures):
    os.makedirs(dirname, exist_ok=True)
    text = water.input_nn_text(sf_lines, nodes=nodes, activations=" ".join(["p"] * len(nodes) + ["l"]),
                               comment="synthetic water HDNNP, generated by tests/golden/make_golden.py")
    with open(os.path.join(dirname, "input.nn"), "w") as f:
        f.write(text)
    rng = np.random.default_rng(seed)
    nsf = len(sf_lines) // 2
    for z in (1, 8):
        water.write_weights(os.path.join(dirname, "weights.%03d.data" % z),
                            water.random_weights([nsf, *nodes, 1], rng))
    # unscaled G of the statistics structure, from the reference library
    with tempfile.TemporaryDirectory() as tmp:
        with open(os.path.join(tmp, "input.nn"), "w") as f:
            f.write(water.input_nn_text(sf_lines, nodes=nodes,
                                        activations=" ".join(["p"] * len(nodes) + ["l"]), scaling=False))
        for z in (1, 8):
            shutil.copy(os.path.join(dirname, "weights.%03d.data" % z), tmp)
        water.write_scaling(os.path.join(tmp, "scaling.data"), [np.zeros((nsf, 4)), np.zeros((nsf, 4))])
        p = ref.RefPrediction(tmp)
        GH, GO = [], []
        for st in stats_structures:
            p.predict(st.to_text(), use_forces=False)
            G = p.arrays()["G"].reshape(-1, nsf)
            el = np.array([0 if e == "H" else 1 for e in st.elements])
            GH.append(G[el == 0])
            GO.append(G[el == 1])
        stats = water.scaling_statistics([np.concatenate(GH), np.concatenate(GO)])
        p.close()
    water.write_scaling(os.path.join(dirname, "scaling.data"), stats)


SCALING_KEYS = ("scale_symmetry_functions", "center_symmetry_functions", "scale_symmetry_functions_sigma",
                "scale_min_short", "scale_max_short")


def _sf_counts(input_nn):
    """Symmetry functions per element symbol of a settings text."""
    counts = {}
    for line in input_nn.splitlines():
        w = line.split("#")[0].split()
        if w and w[0] == "symfunction_short":
            counts[w[1]] = counts.get(w[1], 0) + 1
    return counts


def _settings_value(input_nn, key):
    for line in input_nn.splitlines():
        w = line.split("#")[0].split()
        if w and w[0] == key:
            return w[1:]
    raise KeyError(key)


def write_derived_model(dirname, input_nn, structures, seed):
    """A model directory from a settings text: seeded random weights
    (N(0, 1/fan_in), zero biases), scaling.data from the reference library's
    unscaled G over `structures` (the nnp-scaling statistics), input.data with
    the structures."""
    os.makedirs(dirname, exist_ok=True)
    with open(os.path.join(dirname, "input.nn"), "w") as f:
        f.write(input_nn)
    with open(os.path.join(dirname, "input.data"), "w") as f:
        for st in structures:
            f.write(st.to_text())
    symbols = _settings_value(input_nn, "elements")
    nodes = [int(x) for x in _settings_value(input_nn, "global_nodes_short")]
    counts = _sf_counts(input_nn)
    z = {sym: atomic_number(sym) for sym in symbols}
    order = sorted(symbols, key=lambda e: z[e])
    rng = np.random.default_rng(seed)
    for sym in order:
        water.write_weights(os.path.join(dirname, "weights.%03d.data" % z[sym]),
                            water.random_weights([counts[sym], *nodes, 1], rng))
    with tempfile.TemporaryDirectory() as tmp:
        plain = "\n".join(l for l in input_nn.splitlines()
                          if not (l.split() and l.split()[0] in SCALING_KEYS)) + "\n"
        with open(os.path.join(tmp, "input.nn"), "w") as f:
            f.write(plain)
        for sym in order:
            shutil.copy(os.path.join(dirname, "weights.%03d.data" % z[sym]), tmp)
        water.write_scaling(os.path.join(tmp, "scaling.data"), [np.zeros((counts[e], 4)) for e in order])
        p = ref.RefPrediction(tmp)
        G = {e: [] for e in order}
        for st in structures:
            p.predict(st.to_text(), use_forces=False)
            g = p.arrays()["G"]
            k = 0
            for sym in st.elements:
                G[sym].append(g[k:k + counts[sym]])
                k += counts[sym]
        p.close()
    with np.errstate(invalid="ignore", divide="ignore"):   # QM9 holds a single F atom: no sigma
        stats = water.scaling_statistics([np.array(G[e]) for e in order])
    for st in stats:   # functions constant over the sample get a unit range and sigma (finite scaling)
        flat = ~(st[:, 1] > st[:, 0])
        st[flat, 1] = st[flat, 0] + 1.0
        bad = ~(np.isfinite(st[:, 3]) & (st[:, 3] > 0.0))
        st[bad, 3] = 1.0
    water.write_scaling(os.path.join(dirname, "scaling.data"), stats)


def atomic_number(symbol):
    return {"H": 1, "C": 6, "N": 7, "O": 8, "F": 9, "S": 16, "Cu": 29}[symbol]


def compact_models(refdir):
    """The weighted (QM9) and narrow (from Ethylbenzene_SCAN) compact models."""
    from n2p2_b200 import read_structures
    qdir = os.path.join(refdir, "examples/nnp-train/QM9")
    text = open(os.path.join(qdir, "input.nn")).read()
    allm = read_structures(os.path.join(qdir, "input.data"))
    mols = allm[:16]
    for sym in _settings_value(text, "elements"):   # every element present (F is rare)
        if not any(sym in m.elements for m in mols):
            mols += [m for m in allm[16:] if sym in m.elements][:3]
    write_derived_model(os.path.join(HERE, "models", "qm9_weighted"), text, mols, 2024)

    edir = os.path.join(HERE, "examples", "Ethylbenzene_SCAN")
    lines = []
    extra = []
    for line in open(os.path.join(edir, "input.nn")).read().splitlines():
        w = line.split()
        if w and w[0] == "symfunction_short" and w[2] == "22":
            w[2] = "21"
            line = " ".join(w)
            key = (w[1], w[3], w[4])
            if key not in [k for k, _ in extra]:
                for al, ar in (("-90.00", "90.00"), ("0.00", "180.00")):
                    extra.append((key, "symfunction_short %s 21 %s %s -1.50E+01 1.50E+01 %s %s p1"
                                  % (key[0], key[1], key[2], al, ar)))
        lines.append(line)
    text = "\n".join(lines + [x for _, x in extra]) + "\n"
    frame = read_structures(os.path.join(edir, "input.data"))[0]
    frames = [frame]
    for k in range(3):
        c = read_structures(os.path.join(edir, "input.data"))[0]
        c.positions = c.positions + np.random.default_rng(40 + k).normal(0.0, 0.02, c.positions.shape)
        frames.append(c)
    write_derived_model(os.path.join(HERE, "models", "scan_narrow"), text, frames, 2025)


TRAINING_EXAMPLES = ["H2O_RPBE-D3"]


def parse_training_goldens(src, name):
    """lastEpoch, RMSE values and accuracy of one Example_nnp_train entry."""
    blk = src.split('Example_nnp_train("%s")' % name)[1].split("examples.push_back")[0]
    def val(key):
        return float(re.search(r"e->%s\s*=\s*([-0-9.E+]+);" % key, blk).group(1))
    return {"last_epoch": int(val("lastEpoch")), "rmse_energy_train": val("rmseEnergyTrain"),
            "rmse_energy_test": val("rmseEnergyTest"), "rmse_forces_train": val("rmseForcesTrain"),
            "rmse_forces_test": val("rmseForcesTest"), "accuracy": val("accuracy")}


def training_examples(refdir):
    """examples/nnp-train/<name>/ (input.nn, input.data, scaling.data) with the
    learning-curve values the reference's regression test asserts
    (test/cpp/Example_nnp_train.h; BOOST_REQUIRE_SMALL of the difference)."""
    src = open(os.path.join(refdir, "test/cpp/Example_nnp_train.h")).read()
    for name in TRAINING_EXAMPLES:
        d_in = os.path.join(refdir, "examples/nnp-train", name)
        d_out = os.path.join(HERE, "training", name)
        os.makedirs(d_out, exist_ok=True)
        for fn in ("input.nn", "scaling.data", "input.data"):
            shutil.copy(os.path.join(d_in, fn), os.path.join(d_out, fn))
        g = parse_training_goldens(src, name)
        g["source"] = "test/cpp/Example_nnp_train.h (n2p2 reference regression test of nnp-train)"
        g["columns"] = "learning-curve.out: RMSEpa energy (train, test), RMSE forces (train, test), physical units"
        exe = os.path.join(ROOT, "oracle", "_ref", "nnp-train")
        if os.path.exists(exe):
            g["reference_run"] = run_reference_training(exe, d_out)
        with open(os.path.join(d_out, "golden.json"), "w") as fh:
            json.dump(g, fh, indent=1)


def read_learning_curve(path):
    """Epoch rows of learning-curve.out: {epoch: (RMSEpa E train, test, RMSE F train, test)}
    (physical units; columns 1, 2, 9, 10 as the reference's test reads them)."""
    out = {}
    for line in open(path):
        c = line.split()
        if c and not c[0].startswith("#"):
            out[int(c[0])] = [float(c[1]), float(c[2]), float(c[9]), float(c[10])]
    return out


def run_reference_training(exe, example_dir):
    """The reference's nnp-train (oracle/_ref/nnp-train, built from its own
    sources by oracle/Makefile) on the example in a scratch directory: its
    learning curve per epoch and its Kalman status lines (updater.000.out)."""
    import subprocess
    with tempfile.TemporaryDirectory() as tmp:
        for fn in ("input.nn", "scaling.data", "input.data"):
            shutil.copy(os.path.join(example_dir, fn), tmp)
        subprocess.run([exe], cwd=tmp, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        curve = read_learning_curve(os.path.join(tmp, "learning-curve.out"))
        status = [[float(x) for x in l.split()] for l in open(os.path.join(tmp, "updater.000.out"))
                  if l.split() and not l.startswith("#")]
    return {"source": "oracle/_ref/nnp-train (the reference's nnp-train from its own sources, one process)",
            "learning_curve": {str(k): v for k, v in sorted(curve.items())},
            "kalman_status_columns": "epoch nupdates Pdiag Poffdiag Pasym Kmean q eta",
            "kalman_status": status}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("N2P2_REFERENCE") or
                    os.path.join(os.path.dirname(ROOT), "reference"))
    ap.add_argument("--examples-only", action="store_true", help="copy the reference examples and their goldens only")
    ap.add_argument("--compact-only", action="store_true", help="write the derived compact-function models only")
    ap.add_argument("--training-only", action="store_true", help="copy the nnp-train examples and their goldens only")
    args = ap.parse_args()
    refdir = args.reference
    if not ref.available():
        sys.exit("oracle/_ref/libnnpref.so missing: run `make -C oracle`")

    if args.compact_only:
        compact_models(refdir)
        return
    if args.training_only:
        training_examples(refdir)
        return

    src = open(os.path.join(refdir, "test/cpp/ExamplePrediction.h")).read()
    for name in EXAMPLES:
        d_in = os.path.join(refdir, "examples/nnp-predict", name)
        d_out = os.path.join(HERE, "examples", name)
        os.makedirs(d_out, exist_ok=True)
        for fn in os.listdir(d_in):
            if fn in ("input.nn", "scaling.data", "input.data") or re.match(r"weights\.\d{3}\.data", fn):
                shutil.copy(os.path.join(d_in, fn), os.path.join(d_out, fn))
        e, f = parse_example_goldens(src, name)
        with open(os.path.join(d_out, "golden.json"), "w") as fh:
            json.dump({"source": "test/cpp/ExamplePrediction.h (n2p2 reference regression test)",
                       "tolerance": "1000 * DBL_EPSILON absolute", "energy": e, "forces": f}, fh)

    if args.examples_only:
        return
    training_examples(refdir)
    compact_models(refdir)

    csrc = open(os.path.join(refdir, "test/cpp/test_CutoffFunction.cpp")).read()
    with open(os.path.join(HERE, "cutoff_functions.json"), "w") as fh:
        json.dump(parse_cutoff_goldens(csrc), fh, indent=1)

    box64 = water.water_box(64, seed=0)
    samples = [box64]
    for k, s in enumerate(water.water_batch(48, seed=999, n_min=32, n_max=128)):
        s.positions = s.positions + np.random.default_rng(100 + k).normal(0.0, 0.05, s.positions.shape)
        samples.append(s)
    write_model(os.path.join(HERE, "models", "water40"), water.symfunction_lines(), (25, 25), 12345, samples)
    box512 = water.water_box(512, seed=3, sigma=0.15)
    train_like = water.water_batch(48, seed=777, n_min=64, n_max=128, sigma_range=(0.05, 0.4))
    write_model(os.path.join(HERE, "models", "water56"), water.symfunction_lines(g9=True), (64, 64), 23456,
                [box512] + train_like)

    p = ref.RefPrediction(os.path.join(HERE, "models", "water40"))
    p.predict(box64.to_text())
    a = p.arrays()
    with open(os.path.join(HERE, "water40_box64.json"), "w") as fh:
        json.dump({"source": "reference libnnp (oracle/_ref/libnnpref.so), water_box(64, seed=0)",
                   "energy": a["energy"], "forces": a["forces"].tolist(),
                   "num_neighbors": int(a["nbr_offset"][-1])}, fh)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
