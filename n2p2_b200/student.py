"""Distilled student HDNNP: a reduced descriptor (8 radial G2 + 6 angular G3
per element) and a 14-16-16-1 softplus network, trained on the GPU by the
library's own kernels (n2p2_trainer_*) on energies and forces that the full
HDNNP (the teacher) computes, and evaluated with the teacher as fallback.

The student is an ordinary n2p2 model directory (input.nn, scaling.data,
weights.%03d.data), so the same engine evaluates it.  Evaluation follows the
reference's extrapolation check (SymFnc scaling range, Mode.cpp:1172-1210):
every structure in which any student symmetry function leaves its scaling
range is re-evaluated by the teacher.  A small held-out sample of every
evaluation batch is also run through the teacher and the student's error on
it is recorded.

    python -m n2p2_b200.student train --teacher tests/golden/models/water56 --out student_dir
"""
import argparse
import json
import math
import os
import shutil
import time

import numpy as np

from . import water

HA_TO_MEV = 27211.386245988
BOHR_TO_A = 0.529177210903

STUDENT_G2_ETAS = (0.001, 0.01, 0.06, 0.3)     # x {H, O} neighbours = 8 radial
STUDENT_G3_ETA = 0.01                          # x {HH, HO, OO} x lambda +-1 = 6 angular
STUDENT_G3_ZETA = 1.0
STUDENT_NODES = (16, 16)


def student_sf_lines(rc=water.RC, rc_angular=None):
    rca = rc if rc_angular is None else rc_angular
    out = []
    for ec in ("H", "O"):
        for e1 in ("H", "O"):
            for eta in STUDENT_G2_ETAS:
                out.append(f"symfunction_short {ec} 2 {e1} {eta:.6g} 0.0 {rc:.6g}")
        for e1, e2 in (("H", "H"), ("H", "O"), ("O", "O")):
            for lam in (-1.0, 1.0):
                out.append(f"symfunction_short {ec} 3 {e1} {e2} {STUDENT_G3_ETA:.6g} {lam:.0f} "
                           f"{STUDENT_G3_ZETA:.6g} {rca:.6g}")
    return out


def teacher_sf_importance(teacher_mode, structs):
    """Per element: mean |dE_i/dG_is| over the atoms times the spread (sigma)
    of the scaled G_s -- how much each teacher symmetry function moves the
    teacher's atomic energies on these structures."""
    b = teacher_mode.batch(structs)
    b.setPositions(_positions(structs))
    b.evaluate(forces=True, graph=False)
    G, D = b.symmetryFunctions(), b.dEdG()
    ne = teacher_mode.numElements
    nsf = np.array([teacher_mode.numSymmetryFunctions(e) for e in range(ne)])
    off = np.concatenate([[0], np.cumsum(nsf[b.elements])])
    out = []
    for e in range(ne):
        rows = np.nonzero(b.elements == e)[0]
        ix = off[rows][:, None] + np.arange(nsf[e])[None, :]
        out.append(np.mean(np.abs(D[ix]), axis=0) * np.std(G[ix], axis=0))
    b.close()
    return out


def select_student_sfs(teacher_mode, importance, n_radial=8, n_angular=6, rc_angular=None):
    """symfunction_short lines of the n_radial radial (type 2) and n_angular
    narrow angular (type 3) teacher functions of highest importance, per
    element (angular ones with cutoff rc_angular when given)."""
    sym = [teacher_mode.elementSymbol(e) for e in range(teacher_mode.numElements)]
    lines = []
    for e in range(teacher_mode.numElements):
        sfs = [teacher_mode.symmetryFunction(e, i) for i in range(teacher_mode.numSymmetryFunctions(e))]
        for t, n in ((2, n_radial), (3, n_angular)):
            cand = [i for i, f in enumerate(sfs) if f[0] == t]
            cand.sort(key=lambda i: -importance[e][i])
            for i in sorted(cand[:n]):
                typ, e1, e2, eta, rs, lam, zeta, rc, _ = sfs[i]
                if t == 2:
                    lines.append(f"symfunction_short {sym[e]} 2 {sym[e1]} {eta:.10g} {rs:.10g} {rc:.10g}")
                else:
                    rca = rc if rc_angular is None else rc_angular
                    lines.append(f"symfunction_short {sym[e]} 3 {sym[e1]} {sym[e2]} {eta:.10g} {lam:.0f} "
                                 f"{zeta:.10g} {rca:.10g}")
    return lines


def _sf_line(sym, e, f, rc_angular=None):
    typ, e1, e2, eta, rs, lam, zeta, rc, _ = f
    if typ == 2:
        return f"symfunction_short {sym[e]} 2 {sym[e1]} {eta:.10g} {rs:.10g} {rc:.10g}"
    rca = rc if rc_angular is None else rc_angular
    return f"symfunction_short {sym[e]} 3 {sym[e1]} {sym[e2]} {eta:.10g} {lam:.0f} {zeta:.10g} {rca:.10g}"


def candidate_sf_lines(teacher_mode, rc_angular=None, angular_etas=(0.001, 0.003, 0.01, 0.03),
                       angular_zetas=(1.0, 2.0, 4.0, 16.0), extra_radial_etas=(1.0, 3.0)):
    """Descriptor candidates per element: the teacher's radial functions,
    radial functions of the extra widths (per neighbour element, teacher's
    radial cutoff), and narrow angular functions (type 3) over the grid of
    eta x zeta x lambda +-1 for every neighbour-element pair, with cutoff
    rc_angular (the teacher's largest cutoff when None)."""
    ne = teacher_mode.numElements
    sym = [teacher_mode.elementSymbol(e) for e in range(ne)]
    rca = teacher_mode.getMaxCutoffRadius() if rc_angular is None else rc_angular
    lines = []
    for e in range(ne):
        sfs = [teacher_mode.symmetryFunction(e, i) for i in range(teacher_mode.numSymmetryFunctions(e))]
        radial = [f for f in sfs if f[0] == 2]
        lines += [_sf_line(sym, e, f) for f in radial]
        rcr = max(f[7] for f in radial) if radial else rca
        for e1 in range(ne):
            for eta in extra_radial_etas:
                if not any(f[1] == e1 and f[3] == eta and f[4] == 0.0 for f in radial):
                    lines.append(f"symfunction_short {sym[e]} 2 {sym[e1]} {eta:.10g} 0 {rcr:.10g}")
        for e1 in range(ne):
            for e2 in range(e1, ne):
                for eta in angular_etas:
                    for zeta in angular_zetas:
                        for lam in (-1, 1):
                            lines.append(f"symfunction_short {sym[e]} 3 {sym[e1]} {sym[e2]} {eta:.10g} {lam} "
                                         f"{zeta:.10g} {rca:.10g}")
    return lines


def _derivative_tables(mode):
    """rows[e][en]: symmetry-function indices of element e that depend on a
    neighbour of element en, in the order of the per-neighbour dG/dr rows
    (Element::symmetryFunctionTable order: ascending index)."""
    ne = mode.numElements
    out = [[[] for _ in range(ne)] for _ in range(ne)]
    for e in range(ne):
        for i in range(mode.numSymmetryFunctions(e)):
            typ, e1, e2 = mode.symmetryFunction(e, i)[:3]
            for en in range(ne):
                if (en == e1) if typ == 2 else en in (e1, e2):
                    out[e][en].append(i)
    return out


def _contribution_vectors(mode, batch, dEdG=None):
    """Per atom in turn (a generator): the dG_is/dr_k vectors of its
    symmetry functions over k = the atom itself, then its neighbour entries in
    list order ([1 + n] x 3 x numSF) -- or, with per-atom dE/dG given, their
    contraction sum_s dE_i/dG_is dG_is/dr_k ([1 + n] x 3), atom i's
    contribution to the forces.  The batch was evaluated with stored dG/dr."""
    nb = batch.neighbors()
    off, idx = nb["offset"], nb["index"]
    el = batch.elements
    ne = mode.numElements
    rows = np.array([[mode.numDerivativeRows(e, en) for en in range(ne)] for e in range(ne)])
    row_count = rows[el[np.repeat(np.arange(batch.numAtoms), np.diff(off))], el[idx]]
    row_off = np.concatenate([[0], np.cumsum(row_count)])
    selfd, nbr = batch.dGdr(int(row_off[-1]))
    nsf = np.array([mode.numSymmetryFunctions(e) for e in range(ne)])
    sf_off = np.concatenate([[0], np.cumsum(nsf[el])])
    tab = _derivative_tables(mode)
    for i in range(batch.numAtoms):
        e = el[i]
        p0, p1 = off[i], off[i + 1]
        V = np.zeros((1 + p1 - p0, 3, nsf[e]))
        V[0] = selfd[sf_off[i]:sf_off[i + 1]].T
        for q, p in enumerate(range(p0, p1)):
            t = tab[e][el[idx[p]]]
            V[1 + q][:, t] = nbr[row_off[p]:row_off[p] + len(t)].T
        yield V if dEdG is None else V @ dEdG[sf_off[i]:sf_off[i + 1]]


def force_span_statistics(teacher_mode, candidate_mode, structs):
    """Per element: (M [atoms, C, C], B [atoms, C], c [atoms]) with, for each
    atom i, V_i the dG/dr vectors of the C candidate functions (columns) and
    f_i the teacher's force contributions of atom i (both over the atom and its
    neighbours): M_i = V_i^T V_i, B_i = V_i^T f_i, c_i = |f_i|^2.  Both modes
    must have the same largest cutoff (identical neighbour lists)."""
    pos = _positions(structs)
    bt = teacher_mode.batch(structs)
    bt.setPositions(pos)
    bt.evaluate(forces=True, storeDGdr=True, graph=False)
    f = [g.ravel() for g in _contribution_vectors(teacher_mode, bt, bt.dEdG())]
    nt = bt.neighbors()
    bc = candidate_mode.batch(structs)
    bc.setPositions(pos)
    bc.evaluate(forces=True, storeDGdr=True, graph=False)
    nc = bc.neighbors()
    if not (np.array_equal(nt["offset"], nc["offset"]) and np.array_equal(nt["index"], nc["index"])):
        raise ValueError("teacher and candidate descriptors need the same neighbour lists (same largest cutoff)")
    el = bt.elements
    acc = [([], [], []) for _ in range(teacher_mode.numElements)]
    for i, V in enumerate(_contribution_vectors(candidate_mode, bc)):
        V = V.reshape(-1, V.shape[-1])
        M, B, c = acc[el[i]]
        M.append(V.T @ V)
        B.append(V.T @ f[i])
        c.append(f[i] @ f[i])
    out = [tuple(np.array(x) for x in a) for a in acc]
    bt.close()
    bc.close()
    return out


def span_residual(M, B, c, subset, ridge=1e-10):
    """sum_i min_a |f_i - V_i[:, subset] a|^2 from the Gram statistics (a
    ridge of `ridge` x the mean diagonal keeps near-collinear sets solvable)."""
    S = list(subset)
    if not S:
        return float(c.sum())
    Mss = M[:, S][:, :, S]
    k = len(S)
    Mss = Mss + (ridge * np.trace(Mss, axis1=1, axis2=2) / k)[:, None, None] * np.eye(k)[None]
    b = B[:, S]
    x = np.linalg.solve(Mss, b[..., None])[..., 0]
    return float((c - (b * x).sum(axis=1)).sum())


def greedy_span_selection(M, B, c, types, budget, admissible=None):
    """Forward selection of candidate columns minimising span_residual, taking
    at most budget[t] candidates of type types[j] == t (and, with
    `admissible`, only j for which admissible(chosen, j) holds); returns the
    chosen indices in order and the relative residual after each choice."""
    left = dict(budget)
    chosen, trace = [], []
    total = float(c.sum())
    while any(left.get(t, 0) > 0 for t in set(types)):
        best = None
        for j, t in enumerate(types):
            if j in chosen or left.get(t, 0) <= 0 or (admissible is not None and not admissible(chosen, j)):
                continue
            r = span_residual(M, B, c, chosen + [j])
            if best is None or r < best[0]:
                best = (r, j)
        if best is None:
            break
        chosen.append(best[1])
        left[types[best[1]]] -= 1
        trace.append(best[0] / total)
    return chosen, trace


GAUSSIAN_PLAN_MAX_POWER = 16   # exp(-eta r^2) as an integer power <= 16 of a group's base Gaussian
GAUSSIAN_PLAN_MAX_BASES = 4    # base Gaussians of a radial group in the specialised kernels


def gaussian_bases(etas):
    """Base widths of the engine's Gaussian plan for one group's widths (in
    ascending order, each width an integer multiple <= 16 of an earlier base
    within 1e-9, else a new base)."""
    bases = []
    for eta in sorted(set(etas)):
        for b in bases:
            k = round(eta / b)
            if 1 <= k <= GAUSSIAN_PLAN_MAX_POWER and abs(eta / b - k) <= 1e-9 * eta / b:
                break
        else:
            bases.append(eta)
    return bases


def specialised_kernel_admissible(sfs):
    """admissible(chosen, j) for greedy_span_selection: adding candidate j
    keeps every group of the chosen set runnable by the model-specialised
    symmetry-function kernels -- radial groups (per neighbour element and
    cutoff) with at most GAUSSIAN_PLAN_MAX_BASES base Gaussians; angular
    groups (per element pair and cutoff) with one base Gaussian, at most two
    widths, two lambdas and four integer zetas <= 32.  A descriptor outside
    this runs on the generic kernels, several times slower per triplet.
    sfs: Mode.symmetryFunction tuples of the candidates."""
    def key(f):
        return (f[0], f[1], f[2] if f[0] != 2 else -1, f[7])

    def admissible(chosen, j):
        grp = [sfs[i] for i in chosen if key(sfs[i]) == key(sfs[j])] + [sfs[j]]
        etas = [f[3] for f in grp]
        if any(f[4] != 0.0 for f in grp):
            return False
        if sfs[j][0] == 2:
            return len(gaussian_bases(etas)) <= GAUSSIAN_PLAN_MAX_BASES
        zetas = {f[6] for f in grp}
        return (len(gaussian_bases(etas)) == 1 and len(set(etas)) <= 2 and len({f[5] for f in grp}) <= 2
                and len(zetas) <= 4 and all(float(z).is_integer() and 1 <= z <= 32 for z in zetas))
    return admissible


def select_by_force_span(teacher_mode, structs, candidate_dir, n_radial=8, n_angular=6, rc_angular=None,
                         device=0, log=None, specialised=True):
    """symfunction_short lines of the student's descriptor chosen from
    candidate_sf_lines: per element, the n_radial radial and n_angular angular
    candidates whose dG/dr vectors best span the teacher's per-atom force
    contributions on `structs` (greedy forward selection).

    For atom i the teacher's contribution to the forces is
    f_i = (sum_s dE_i/dG_is dG_is/dr_k)_k over k = i and its neighbours; a
    student on descriptor set S produces sum_{s in S} a_s dG'_is/dr_k with
    a_s its own dE_i/dG'_is.  The least-squares residual of f_i against the
    span of those vectors, summed over atoms, is the part of the teacher's
    forces that no network on S reproduces even with free per-atom
    coefficients; the selection minimises it.  With `specialised`, only
    sets the model-specialised kernels run are considered
    (specialised_kernel_admissible).  Returns (lines, report)."""
    sym = [teacher_mode.elementSymbol(e) for e in range(teacher_mode.numElements)]
    cand = candidate_sf_lines(teacher_mode, rc_angular)
    write_student_model(candidate_dir, structs, device=device, sf_lines=cand)
    cm = load_mode(candidate_dir, device)
    stats = force_span_statistics(teacher_mode, cm, structs)
    lines, report = [], {}
    for e, (M, B, c) in enumerate(stats):
        sfs = [cm.symmetryFunction(e, i) for i in range(cm.numSymmetryFunctions(e))]
        types = [f[0] for f in sfs]
        chosen, trace = greedy_span_selection(M, B, c, types, {2: n_radial, 3: n_angular},
                                              specialised_kernel_admissible(sfs) if specialised else None)
        every = span_residual(M, B, c, range(len(sfs))) / float(c.sum())
        lines += [_sf_line(sym, e, sfs[j]) for j in sorted(chosen)]
        report[sym[e]] = {"candidates": len(sfs), "atoms": int(c.size), "residual_all_candidates": every,
                          "residual_after_each_choice": trace,
                          "force_contribution_sq_sum": float(c.sum())}
        if log:
            log(f"{sym[e]}: relative span residual {trace[-1]:.4f} with {len(chosen)} of {len(sfs)} "
                f"candidates ({every:.5f} with all)")
    cm.close()
    return lines, report


def training_structures(num, seed, n_min=64, n_max=512, sigma_range=(0.05, 0.4)):
    """Water boxes of 192-1536 atoms with Gaussian displacements sigma in the range."""
    return water.water_batch(num, seed, n_min=n_min, n_max=n_max, sigma_range=sigma_range)


def _positions(structs):
    return np.ascontiguousarray(np.concatenate([s.positions for s in structs]))


def label(mode, structs, chunk=512, warnings=False):
    """Energies [S] and forces [N,3] (physical units) of `structs` by `mode`;
    with `warnings`, also per structure whether the mode's extrapolation check
    fired (the mode must collect extrapolation warnings)."""
    E, F, W = [], [], []
    b = None
    for c0 in range(0, len(structs), chunk):
        sub = structs[c0:c0 + chunk]
        if b is None:
            b = mode.batch(sub)
        else:
            b.setStructures(sub)
        b.setPositions(_positions(sub))
        b.evaluate(forces=True, graph=False)
        E.append(b.energies())
        F.append(b.forces())
        if warnings:
            _, per_atom = b.extrapolationWarnings()
            starts = np.concatenate([[0], np.cumsum([x.numAtoms for x in sub])[:-1]])
            W.append(np.add.reduceat(per_atom, starts) > 0)
    if warnings:
        return np.concatenate(E), np.concatenate(F), np.concatenate(W)
    return np.concatenate(E), np.concatenate(F)


def write_student_model(directory, scaling_structs, seed=7, device=0, rc=water.RC, rc_angular=None, sf_lines=None):
    """input.nn + N(0, 1/fan_in) weights + scaling.data of the student's
    symmetry functions (`sf_lines`, default student_sf_lines) over
    `scaling_structs` (evaluated on the GPU)."""
    from .mode import Mode
    os.makedirs(directory, exist_ok=True)
    lines = student_sf_lines(rc, rc_angular) if sf_lines is None else list(sf_lines)
    with open(os.path.join(directory, "input.nn"), "w") as f:
        f.write(water.input_nn_text(lines, nodes=STUDENT_NODES, activations="p p l",
                                    comment="distilled student: 8 G2 + 6 G3 per element, 14-16-16-1 softplus"))
    rng = np.random.default_rng(seed)
    nsf = len(lines) // 2
    for Z in (1, 8):
        water.write_weights(os.path.join(directory, "weights.%03d.data" % Z),
                            water.random_weights((nsf,) + STUDENT_NODES + (1,), rng))
    m = Mode(device)
    m.initialize()
    m.loadSettingsFile(os.path.join(directory, "input.nn"))
    m.setupGeneric()
    m.setupSymmetryFunctionScalingNone()
    m.setupNeuralNetworkWeights(os.path.join(directory, "weights.%03zu.data"))
    ne = m.numElements
    nsf = np.array([m.numSymmetryFunctions(e) for e in range(ne)])
    # running min, max, sum, sum of squares (the statistics of
    # water.scaling_statistics without holding every G in memory)
    acc = [dict(n=0, mn=np.full(nsf[e], np.inf), mx=np.full(nsf[e], -np.inf), s=np.zeros(nsf[e]),
                s2=np.zeros(nsf[e])) for e in range(ne)]
    b = None
    for c0 in range(0, len(scaling_structs), 512):
        sub = scaling_structs[c0:c0 + 512]
        if b is None:
            b = m.batch(sub)
        else:
            b.setStructures(sub)
        b.setPositions(_positions(sub))
        b.evaluate(forces=False, graph=False)
        G = b.symmetryFunctions()
        off = np.concatenate([[0], np.cumsum(nsf[b.elements])])
        for e in range(ne):
            rows = np.nonzero(b.elements == e)[0]
            Ge = G[off[rows][:, None] + np.arange(nsf[e])[None, :]]
            a = acc[e]
            a["n"] += Ge.shape[0]
            a["mn"] = np.minimum(a["mn"], Ge.min(axis=0))
            a["mx"] = np.maximum(a["mx"], Ge.max(axis=0))
            a["s"] += Ge.sum(axis=0)
            a["s2"] += (Ge * Ge).sum(axis=0)
    stats = []
    for a in acc:
        mean = a["s"] / a["n"]
        sigma = np.sqrt(np.maximum(a["s2"] - a["s"] * a["s"] / a["n"], 0.0) / (a["n"] - 1))
        stats.append(np.stack([a["mn"], a["mx"], mean, sigma], axis=1))
    water.write_scaling(os.path.join(directory, "scaling.data"), stats)
    m.close()
    return directory


def write_trained_weights(directory, mode, parameters):
    """Weight files of the mode's elements from a parameter vector in file order."""
    pos = 0
    for e in range(mode.numElements):
        nsf = mode.numSymmetryFunctions(e)
        sizes = (nsf,) + STUDENT_NODES + (1,)
        n = sum(sizes[l] * sizes[l - 1] + sizes[l] for l in range(1, len(sizes)))
        Z = {"H": 1, "O": 8}[mode.elementSymbol(e)]
        water.write_weights(os.path.join(directory, "weights.%03d.data" % Z), parameters[pos:pos + n])
        pos += n


def load_mode(directory, device=0, extrapolation=False, precision="fp64"):
    from .mode import Mode
    m = Mode(device)
    m.setupFromDirectory(directory)
    if extrapolation:
        m.setupSymmetryFunctionStatistics(False, True, False, False)
    m.setPrecision(precision)
    return m


class StudentTraining:
    """Mini-batch Adam training of the student on teacher labels."""

    def __init__(self, student_mode, structs, energies, forces, batch_size=64, eta=1e-3, force_weight=10.0,
                 seed=0):
        from .mode import Trainer
        self.mode = student_mode
        self.structs = structs
        self.E = np.asarray(energies)
        self.atom_begin = np.concatenate([[0], np.cumsum([s.numAtoms for s in structs])])
        self.F = np.asarray(forces).reshape(-1, 3)
        self.batch_size = batch_size
        self.rng = np.random.default_rng(seed)
        self.trainer = Trainer(student_mode, eta=eta, forceWeight=force_weight)
        self.batch = None
        self.history = []

    def _set(self, idx):
        sub = [self.structs[k] for k in idx]
        if self.batch is None:
            self.batch = self.mode.batch(sub)
        else:
            self.batch.setStructures(sub)
        self.batch.setPositions(_positions(sub))
        e = self.E[idx]
        f = np.concatenate([self.F[self.atom_begin[k]:self.atom_begin[k + 1]] for k in idx])
        return e, f

    def step(self, idx, update=True, gradient=False):
        e, f = self._set(idx)
        return self.trainer.step(self.batch, e, f, update=update, gradient=gradient)

    def epoch(self):
        order = self.rng.permutation(len(self.structs))
        losses = []
        for b0 in range(0, len(order) - self.batch_size + 1, self.batch_size):
            losses.append(self.step(order[b0:b0 + self.batch_size])[0])
        self.history.append(float(np.mean(losses)))
        return self.history[-1]


def errors(E, F, E_ref, F_ref, atoms_per_structure):
    """Energy error per atom (meV/atom) and per-component force error (meV/A)."""
    de = np.abs(np.asarray(E) - np.asarray(E_ref)) / np.asarray(atoms_per_structure) * HA_TO_MEV
    df = np.abs(np.asarray(F) - np.asarray(F_ref)).ravel() * HA_TO_MEV / BOHR_TO_A
    return {"energy_meV_per_atom_rms": float(np.sqrt(np.mean(de ** 2))), "energy_meV_per_atom_max": float(de.max()),
            "force_meV_per_A_rms": float(np.sqrt(np.mean(df ** 2))), "force_meV_per_A_max": float(df.max())}


class StudentEvaluator:
    """Student evaluation of a batch with teacher fallback and a held-out monitor."""

    def __init__(self, student_mode, teacher_mode, structs, monitor=2, seed=0):
        self.student = student_mode
        self.teacher = teacher_mode
        self.structs = structs
        self.batch = student_mode.batch(structs)
        self.pos = _positions(structs)
        self.batch.setPositions(self.pos)
        self.atom_begin = np.concatenate([[0], np.cumsum([s.numAtoms for s in structs])])
        self.monitor = monitor
        self.rng = np.random.default_rng(seed)
        self.fallback_batch = None
        self.monitor_batch = None
        self.monitor_log = []
        self.fallbacks = 0
        self.evaluations = 0

    def evaluate(self):
        """Energies [S] and forces [N,3]: student, or teacher where the
        student's extrapolation check fired."""
        b = self.batch
        b.evaluate(forces=True)
        E = b.energies()
        F = b.forces()
        _, per_atom = b.extrapolationWarnings()
        flagged = np.add.reduceat(per_atom, self.atom_begin[:-1]) > 0
        self.evaluations += len(self.structs)
        idx = np.nonzero(flagged)[0]
        if idx.size:
            self.fallbacks += idx.size
            sub = [self.structs[k] for k in idx]
            if self.fallback_batch is None:
                self.fallback_batch = self.teacher.batch(sub)
            else:
                self.fallback_batch.setStructures(sub)
            self.fallback_batch.setPositions(_positions(sub))
            self.fallback_batch.evaluate(forces=True, graph=False)
            Et, Ft = self.fallback_batch.energies(), self.fallback_batch.forces()
            E[idx] = Et
            a = 0
            for k in idx:
                n = self.structs[k].numAtoms
                F[self.atom_begin[k]:self.atom_begin[k + 1]] = Ft[a:a + n]
                a += n
        if self.monitor:
            self._judge(E, F)
        return E, F, flagged

    def _judge(self, E, F):
        idx = np.sort(self.rng.choice(len(self.structs), size=min(self.monitor, len(self.structs)), replace=False))
        sub = [self.structs[k] for k in idx]
        if self.monitor_batch is None:
            self.monitor_batch = self.teacher.batch(sub)
        else:
            self.monitor_batch.setStructures(sub)
        self.monitor_batch.setPositions(_positions(sub))
        self.monitor_batch.evaluate(forces=True, graph=False)
        Et, Ft = self.monitor_batch.energies(), self.monitor_batch.forces()
        Fs = np.concatenate([F[self.atom_begin[k]:self.atom_begin[k + 1]] for k in idx])
        self.monitor_log.append(errors(E[idx], Fs, Et, Ft, [s.numAtoms for s in sub]))

    def fallback_rate(self):
        return self.fallbacks / max(1, self.evaluations)


def _subset_errors(Es, Fs, Et, Ft, apa, starts, idx):
    if idx.size == 0:
        return None
    sel = np.concatenate([np.arange(starts[k], starts[k + 1]) for k in idx])
    return errors(Es[idx], Fs[sel], Et[idx], Ft[sel], np.asarray(apa)[idx])


def benchmark(student_dir, teacher_dir, num=2048, seed=97, steps=3, warmup=2, device=0, monitor=2):
    """Held-out throughput and error of the student (with fallback and the
    per-batch held-out monitor) against the plain FP64 teacher on `num` boxes
    of the training recipe (own seed).  Both forms are timed the same way:
    one evaluation plus the energies and forces read back, per step."""
    structs = training_structures(num, seed)
    natoms = sum(s.numAtoms for s in structs)
    apa = [s.numAtoms for s in structs]
    teacher = load_mode(teacher_dir, device, extrapolation=True)
    tb = teacher.batch(structs)
    tb.setPositions(_positions(structs))

    def teacher_step():
        tb.evaluate(forces=True)
        return tb.energies(), tb.forces()

    for _ in range(warmup):
        Et, Ft = teacher_step()
    t0 = time.perf_counter()
    for _ in range(steps):
        Et, Ft = teacher_step()
    t_teacher = (time.perf_counter() - t0) / steps
    _, per_atom = tb.extrapolationWarnings()
    starts = np.concatenate([[0], np.cumsum(apa)])
    teacher_in_range = np.add.reduceat(per_atom, starts[:-1]) == 0

    smode = load_mode(student_dir, device, extrapolation=True)
    ev = StudentEvaluator(smode, teacher, structs, monitor=monitor, seed=seed)
    for _ in range(warmup):
        Es, Fs, flagged = ev.evaluate()
    ev.fallbacks = ev.evaluations = 0
    ev.monitor_log = []
    t0 = time.perf_counter()
    for _ in range(steps):
        Es, Fs, flagged = ev.evaluate()
    t_student = (time.perf_counter() - t0) / steps
    mon = ev.monitor_log
    out = {"workload": "%d held-out water boxes, 64-512 molecules, displacements 0.05-0.4 bohr (%d atoms)"
                       % (num, natoms),
           "value": natoms / t_student, "unit": "atoms/s", "ms_per_step": 1e3 * t_student,
           "teacher_fp64": {"value": natoms / t_teacher, "unit": "atoms/s", "ms_per_step": 1e3 * t_teacher},
           "speedup_vs_fp64": t_teacher / t_student,
           "fallback_rate": ev.fallback_rate(),
           "err_vs_teacher_fp64_gpu": errors(Es, Fs, Et, Ft, apa),
           "err_vs_teacher_fp64_gpu_teacher_in_range": _subset_errors(Es, Fs, Et, Ft, apa, starts,
                                                                      np.nonzero(teacher_in_range)[0]),
           "teacher_in_range_fraction": float(teacher_in_range.mean()),
           "held_out_monitor": {"structures_per_batch": monitor, "batches": len(mon),
                                "energy_meV_per_atom_rms": float(np.mean([m["energy_meV_per_atom_rms"] for m in mon]))
                                if mon else None,
                                "force_meV_per_A_rms": float(np.mean([m["force_meV_per_A_rms"] for m in mon]))
                                if mon else None}}
    out["_predictions"] = (structs, Es, Fs)
    return out


def train(teacher_dir, out_dir, num_configs=20000, epochs=8, batch_size=64, eta=1e-3, seed=11, device=0, log=print,
          select="span", decay=(0.5, 0.3), rc_angular=None):
    """The full recipe: label, choose the descriptor (`select`: "span" --
    select_by_force_span, "importance" -- the teacher's functions of largest
    teacher_sf_importance, None -- student_sf_lines), fit the scaling, train (step size
    `eta`, times decay[1] after each further decay[0] fraction of the epochs);
    writes the trained model and returns a summary dict."""
    t0 = time.perf_counter()
    structs = training_structures(num_configs, seed)
    log(f"{len(structs)} training structures, {sum(s.numAtoms for s in structs)} atoms "
        f"({time.perf_counter() - t0:.1f} s)")
    teacher = load_mode(teacher_dir, device)
    E, F = label(teacher, structs)
    # Labels from far outside the teacher's scaling range (rare close
    # contacts at the largest displacements) reach forces of many Ha/bohr and
    # would dominate a squared-error fit; structures whose largest teacher
    # force exceeds ten times the median of that maximum are not trained on
    # (they remain the teacher's to answer).
    starts = np.concatenate([[0], np.cumsum([s.numAtoms for s in structs])])
    fmax = np.maximum.reduceat(np.abs(F).max(axis=1), starts[:-1])
    outlier = fmax > 10.0 * np.median(fmax)
    keep = np.nonzero(~outlier)[0]
    all_structs = structs
    F = np.concatenate([F[starts[k]:starts[k + 1]] for k in keep])
    E = E[keep]
    structs = [structs[k] for k in keep]
    log(f"teacher labels ({time.perf_counter() - t0:.1f} s); {int(outlier.sum())} structures with outlying "
        f"teacher forces left out")
    lines, span = None, None
    if select == "span":
        sample = [s for s in structs if s.numAtoms <= 300][:12]
        cdir = os.path.join(out_dir, "_candidates")
        lines, span = select_by_force_span(teacher, sample, cdir, rc_angular=rc_angular, device=device, log=log)
        shutil.rmtree(cdir)
    elif select == "importance":
        lines = select_student_sfs(teacher, teacher_sf_importance(teacher, structs[:256]), rc_angular=rc_angular)
    if lines is not None:
        log("descriptor: " + "; ".join(l.replace("symfunction_short ", "") for l in lines))
    # scaling statistics (and hence the extrapolation range) over every training configuration
    write_student_model(out_dir, all_structs, seed=seed, device=device, sf_lines=lines)
    student = load_mode(out_dir, device)
    tr = StudentTraining(student, structs, E, F, batch_size=batch_size, eta=eta, seed=seed)
    first_decay = int(math.ceil(decay[0] * epochs))
    for ep in range(epochs):
        t1 = time.perf_counter()
        lr = eta * decay[1] ** max(0, (ep - first_decay) // max(1, (epochs - first_decay) // 2) + 1) \
            if ep >= first_decay else eta
        tr.trainer.setLearningRate(lr)
        loss = tr.epoch()
        log(f"epoch {ep + 1}: lr {lr:.1e} mean loss {loss:.6e} ({time.perf_counter() - t1:.1f} s)")
    write_trained_weights(out_dir, student, tr.trainer.parameters())
    summary = {"configs": num_configs, "outlying_labels_left_out": int(outlier.sum()),
               "atoms": int(sum(s.numAtoms for s in structs)), "epochs": epochs,
               "descriptor": lines if lines is not None else student_sf_lines(rc_angular=rc_angular),
               "rc_angular": rc_angular, "selection": select, "force_span": span,
               "batch_size": batch_size, "eta": eta, "force_weight": 10.0, "loss_history": tr.history,
               "seconds": time.perf_counter() - t0}
    with open(os.path.join(out_dir, "training.json"), "w") as f:
        json.dump(summary, f, indent=1)
    return summary


def teacher_scaling(teacher_dir, num_configs=20000, seed=11, device=0, log=print):
    """Rewrites the teacher's scaling.data with nnp-scaling statistics
    (n2p2_b200.scaling, the library's GPU statistics) over the configurations
    of the student-training recipe (`num_configs`, `seed`: the structures the
    teacher labels) plus the 512-molecule large-system box, so that the
    teacher's own inputs stay inside its scaling range on that distribution."""
    from . import scaling
    from .mode import Mode
    t0 = time.perf_counter()
    structs = [water.water_box(512, seed=3, sigma=0.15)] + training_structures(num_configs, seed)
    m = Mode(device)
    m.initialize()
    m.loadSettingsFile(os.path.join(teacher_dir, "input.nn"))
    m.setupGeneric()
    m.setupSymmetryFunctionScalingNone()
    stats = scaling.collect_statistics(m, structs)
    scaling.write_scaling(os.path.join(teacher_dir, "scaling.data"), stats)
    m.close()
    log(f"teacher scaling over {len(structs)} structures ({time.perf_counter() - t0:.1f} s)")


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    ts = sub.add_parser("teacher-scaling", help="rewrite the teacher's scaling.data over the training recipe")
    ts.add_argument("--teacher", required=True)
    ts.add_argument("--configs", type=int, default=20000)
    ts.add_argument("--seed", type=int, default=11)
    t = sub.add_parser("train")
    t.add_argument("--teacher", required=True)
    t.add_argument("--out", required=True)
    t.add_argument("--configs", type=int, default=20000)
    t.add_argument("--epochs", type=int, default=8)
    t.add_argument("--batch-size", type=int, default=64)
    t.add_argument("--eta", type=float, default=1e-3)
    t.add_argument("--seed", type=int, default=11)
    t.add_argument("--rc-angular", type=float, default=None, help="cutoff of the angular functions (bohr)")
    t.add_argument("--select", choices=("span", "importance", "fixed"), default="span",
                   help="descriptor choice: force-span selection from a candidate grid, the teacher's most "
                        "important functions, or the fixed student_sf_lines set")
    a = ap.parse_args()
    if a.cmd == "teacher-scaling":
        teacher_scaling(a.teacher, a.configs, a.seed)
    if a.cmd == "train":
        s = train(a.teacher, a.out, a.configs, a.epochs, a.batch_size, a.eta, a.seed, rc_angular=a.rc_angular,
                  select=None if a.select == "fixed" else a.select)
        print(json.dumps({k: v for k, v in s.items() if k != "loss_history"}))


if __name__ == "__main__":
    main()
