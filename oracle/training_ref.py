"""CPU restatement of the reference's training updates -- test
infrastructure only: the checker of the GPU training path, never part of it.

Restated (reference files under src/):
  libnnptrain/KalmanFilter.cpp:126-197   KalmanFilter::update
  libnnptrain/KalmanFilter.cpp:199-238   setParametersStandard / FadingMemory
  libnnptrain/GradientDescent.cpp:81-118 GradientDescent::update (fixed, Adam)
  libnnp/NeuralNetwork.cpp:444-527       calculateDEdc / calculateDFdc (the
                                         derivatives of an atomic network's
                                         output and of its directional
                                         derivative along dG/dx w.r.t. all
                                         connections)
  libnnptrain/Training.cpp:2551-2923     Training::update error and Jacobian
                                         assembly (2G networks, combined
                                         update strategy, one candidate)

The symmetry functions G and dG/dr are the reference library's own
(oracle/_ref/libnnpref.so, one Prediction per structure, once): they do not
depend on the weights.  Arithmetic is FP64 numpy, the Kalman covariance a
full matrix read through its lower triangle as the reference does
(P.selfadjointView<Lower>()).
"""
import os

import numpy as np

from . import ref as oref
from .port import PortModel

EXP_LIMIT = 35.0


def activation(code, x):
    """f, f', f'' of NeuralNetwork::propagate's activations (l, t, s, p)."""
    if code == "l":
        return x, np.ones_like(x), np.zeros_like(x)
    if code == "t":
        t = np.tanh(x)
        d = 1.0 - t * t
        return t, d, -2.0 * t * d
    if code == "s":
        t = 1.0 / (1.0 + np.exp(-x))
        d = t * (1.0 - t)
        return t, d, d * (1.0 - 2.0 * t)
    if code == "p":
        f = np.empty_like(x)
        d = np.empty_like(x)
        d2 = np.empty_like(x)
        hi, lo = x > EXP_LIMIT, x < -EXP_LIMIT
        mid = ~(hi | lo)
        f[hi], d[hi], d2[hi] = x[hi], 1.0, 0.0
        f[lo], d[lo], d2[lo] = 0.0, 0.0, 0.0
        e = np.exp(x[mid])
        f[mid] = np.log(1.0 + e)
        s = 1.0 / (1.0 + 1.0 / e)
        d[mid] = s
        d2[mid] = s * (1.0 - s)
        return f, d, d2
    raise ValueError("activation %r not restated" % code)


class Networks:
    """The atomic networks of a model directory, connections in weight-file
    order (NeuralNetwork::setConnections: per layer, for every source neuron
    its weights to all targets, then the targets' biases), elements by
    atomic number, concatenated (the combined update strategy's state)."""

    def __init__(self, model_dir):
        kv = {}
        for line in open(os.path.join(model_dir, "input.nn")):
            w = line.split("#")[0].split()
            if w:
                kv.setdefault(w[0], w[1:])
        self.pm = PortModel(model_dir)
        self.symbols = self.pm.symbols
        nodes = [int(x) for x in kv["global_nodes_short"]]
        acts = kv["global_activation_short"]
        self.layers = []      # per element: [(nin, nout, activation)]
        for e, sym in enumerate(self.symbols):
            sizes = [len(self.pm.sfs[e])] + nodes + [1]
            self.layers.append([(sizes[l - 1], sizes[l], acts[l - 1]) for l in range(1, len(sizes))])
        self.offsets = [0]
        for lay in self.layers:
            self.offsets.append(self.offsets[-1] + sum(nin * nout + nout for nin, nout, _ in lay))
        self.numWeights = self.offsets[-1]
        w = []
        for sym in self.symbols:
            fn = os.path.join(model_dir, "weights.%03d.data" % oref_z(sym))
            w.append(np.loadtxt(fn, comments="#", usecols=0, ndmin=1))
        self.weights = np.concatenate(w)
        assert self.weights.size == self.numWeights

    def _unpack(self, e, w):
        out, p = [], self.offsets[e]
        for nin, nout, act in self.layers[e]:
            W = w[p:p + nin * nout].reshape(nin, nout).T    # W[k, j] = w(k <- j)
            p += nin * nout
            b = w[p:p + nout]
            p += nout
            out.append((W, b, act))
        return out

    def value_and_gradient(self, e, G, v, a):
        """L = a E + dE/dG . v of one atom of element e, and dL/dc over the
        element's connections (file order)."""
        net = self._unpack(e, self.weights)
        xs, xds, zs, zds, f1s, f2s = [G], [v], [], [], [], []
        for W, b, act in net:
            z = W @ xs[-1] + b
            zd = W @ xds[-1]
            f, f1, f2 = activation(act, z)
            zs.append(z)
            zds.append(zd)
            f1s.append(f1)
            f2s.append(f2)
            xs.append(f)
            xds.append(f1 * zd)
        L = a * xs[-1][0] + xds[-1][0]
        grads = []
        xb = np.array([a])
        xdb = np.array([1.0])
        for l in range(len(net) - 1, -1, -1):
            W = net[l][0]
            zb = xb * f1s[l] + xdb * f2s[l] * zds[l]
            zdb = xdb * f1s[l]
            gW = np.outer(zb, xs[l]) + np.outer(zdb, xds[l])
            grads.append((gW, zb))
            xb = W.T @ zb
            xdb = W.T @ zdb
        grads.reverse()
        flat = []
        for gW, gb in grads:
            flat.append(gW.T.ravel())   # source-major, as the file
            flat.append(gb)
        return L, np.concatenate(flat)


def oref_z(symbol):
    from .port import Z
    return Z[symbol]


class StructureData:
    """G, dG/dr and neighbour layout of one structure from the reference
    library (scaled G, derivatives of the scaled G)."""

    def __init__(self, model_dir, structure, pm):
        p = oref.RefPrediction(model_dir)
        try:
            p.predict(structure.to_text(), use_forces=True)
            a = p.arrays()
        finally:
            p.close()
        self.n = structure.numAtoms
        self.elem = np.array([pm.symbols.index(x) for x in structure.elements])
        so = a["sf_offset"]
        self.G = [a["G"][so[i]:so[i + 1]] for i in range(self.n)]
        self.dself = [a["dGdr_self"][so[i]:so[i + 1]] for i in range(self.n)]
        self.nbr_offset = a["nbr_offset"]
        self.nbr_index = a["nbr_index"]
        self.row_offset = a["row_offset"]
        self.dnbr = a["dGdr_nbr"]
        # rows of a neighbour of element en for a centre of element ec: the
        # SFs relevant to en in index order (Element::setupSymmetryFunctionMemory)
        self.table = []
        for ec in range(len(pm.symbols)):
            t = []
            for en in range(len(pm.symbols)):
                t.append([k for k, s in enumerate(pm.sfs[ec]) if en in (s["e1"], s["e2"])])
            self.table.append(t)

    def tangents(self, atom, comp, images=True):
        """v_i = dG_i/dx_(atom, comp) for every atom i (zero rows omitted),
        Training::collectDGdxia (Training.cpp:3586-3625).  images=False
        leaves out the atom's own periodic-image entries, as
        Mode::calculateForces does (Mode.cpp:1957: neighborsUnique from its
        second element)."""
        out = {atom: self.dself[atom][:, comp].copy()}
        for i in range(self.n):
            for e in range(self.nbr_offset[i], self.nbr_offset[i + 1]):
                if self.nbr_index[e] != atom or (not images and i == atom):
                    continue
                rows = self.table[self.elem[i]][self.elem[atom]]
                d = self.dnbr[self.row_offset[e]:self.row_offset[e] + len(rows), comp]
                v = out.setdefault(i, np.zeros(len(self.G[i])))
                v[rows] += d
        return out


class KalmanFilter:
    """KalmanFilter (standard: type 0, fading memory: type 1)."""

    def __init__(self, n, kind, epsilon, q0, qtau, qmin, eta0=0.0, etatau=0.0, etamax=0.0, lam=0.0, nu=0.0):
        self.kind = kind
        self.P = np.eye(n) / epsilon
        self.q, self.q0, self.qtau, self.qmin = q0, q0, qtau, qmin
        self.eta, self.etatau, self.etamax = eta0, etatau, etamax
        self.lam, self.nu, self.gamma = lam, nu, 1.0
        self.K = np.zeros(n)
        self.numUpdates = 0

    def update(self, w, H, xi):
        H = H if H.ndim == 2 else H.reshape(-1, 1)
        xi = np.atleast_1d(xi)
        Pl = np.tril(self.P)
        Psym = Pl + np.tril(self.P, -1).T
        X = Psym @ H
        A = H.T @ X
        if self.kind == 0 and self.eta < self.etamax:
            self.eta *= np.exp(self.etatau)
        A = A + np.eye(A.shape[0]) * (1.0 / self.eta if self.kind == 0 else self.lam)
        K = X @ np.linalg.inv(A)
        self.P = self.P - K @ X.T
        if self.kind == 1:
            self.P *= 1.0 / self.lam
        self.P[np.diag_indices_from(self.P)] += self.q
        w += (K @ xi).ravel()
        if self.q > self.qmin:
            self.q *= np.exp(-self.qtau)
        if self.kind == 1:
            self.lam = self.nu * self.lam + 1.0 - self.nu
            self.gamma = 1.0 / (1.0 + self.lam / self.gamma)
        self.K = K.ravel()
        self.numUpdates += 1


class GradientDescent:
    """GradientDescent (fixed: type 0, Adam: type 1)."""

    def __init__(self, n, kind, eta, beta1=0.9, beta2=0.999, epsilon=1e-8):
        self.kind, self.eta, self.eta0 = kind, eta, eta
        self.beta1, self.beta2, self.eps = beta1, beta2, epsilon
        self.beta1t, self.beta2t = beta1, beta2
        self.m = np.zeros(n)
        self.v = np.zeros(n)

    def update(self, w, H, xi):
        if self.kind == 0:
            w -= self.eta * xi * -H
            return
        g = xi * -H
        self.m = self.beta1 * self.m + (1.0 - self.beta1) * g
        self.v = self.beta2 * self.v + (1.0 - self.beta2) * g * g
        eta = self.eta0 * np.sqrt(1.0 - self.beta2t) / (1.0 - self.beta1t)
        w -= eta * self.m / (np.sqrt(self.v) + self.eps)
        self.beta1t *= self.beta1
        self.beta2t *= self.beta2


class Training:
    """Training::update for a list of structures with reference energies
    (physical, with offsets) and forces; `updater` a KalmanFilter or
    GradientDescent over all weights (combined strategy)."""

    def __init__(self, model_dir, structures, energies, forces, updater, force_weight=1.0):
        self.nets = Networks(model_dir)
        pm = self.nets.pm
        self.data = [StructureData(model_dir, s, pm) for s in structures]
        self.updater = updater
        self.force_weight = force_weight
        self.eref = []
        self.fref = []
        k = 0
        for s, E in zip(structures, energies):
            el = self.data[len(self.eref)].elem
            Ei = E - sum(pm.atomicEnergyOffset[x] for x in el)
            if pm.normalize:
                Ei = (Ei - s.numAtoms * pm.meanEnergy) * pm.convEnergy
            self.eref.append(Ei)
            f = np.asarray(forces[k:k + s.numAtoms], dtype=np.float64)
            self.fref.append(f * (pm.convEnergy / pm.convLength if pm.normalize else 1.0))
            k += s.numAtoms

    def observation(self, prop, s, atom=0, comp=0):
        """(error ref - prediction, Jacobian) of an energy or force observation."""
        d = self.data[s]
        nets = self.nets
        H = np.zeros(nets.numWeights)
        pred = 0.0
        if prop == 0:
            for i in range(d.n):
                e = d.elem[i]
                L, g = nets.value_and_gradient(e, d.G[i], np.zeros_like(d.G[i]), 1.0)
                pred += L
                H[nets.offsets[e]:nets.offsets[e + 1]] += g
            return self.eref[s] - pred, H
        # F = -sum_i dE_i/dG_i . dG_i/dx: the tangent carries the minus sign.
        # The prediction is Mode::calculateForces' force, the Jacobian
        # calculateDFdc over collectDGdxia's derivatives.
        for i, v in sorted(d.tangents(atom, comp).items()):
            e = d.elem[i]
            _, g = nets.value_and_gradient(e, d.G[i], -v, 0.0)
            H[nets.offsets[e]:nets.offsets[e + 1]] += g
        for i, v in sorted(d.tangents(atom, comp, images=False).items()):
            L, _ = nets.value_and_gradient(d.elem[i], d.G[i], -v, 0.0)
            pred += L
        return self.fref[s][atom, comp] - pred, H

    def update(self, prop, s, atom=0, comp=0):
        return self.update_batch(prop, [(s, atom, comp)])[0]

    def update_element(self, prop, s, atom=0, comp=0):
        """update_strategy 1: one updater per element (self.updater a list),
        each on its element's weights with the error times the element's
        fraction of the atoms (energy) or of the atom's neighbours (force),
        then the force weight (Training.cpp:2900-2922)."""
        err, H = self.observation(prop, s, atom, comp)
        d = self.data[s]
        ne = len(self.nets.symbols)
        if prop == 0:
            frac = [(np.sum(d.elem == e), d.n) for e in range(ne)]
        else:
            js = d.nbr_index[d.nbr_offset[atom]:d.nbr_offset[atom + 1]]
            frac = [(np.sum(d.elem[js] == e), js.size) for e in range(ne)]
        for e in range(ne):
            o0, o1 = self.nets.offsets[e], self.nets.offsets[e + 1]
            xi = err * float(frac[e][0]) / float(frac[e][1])
            He = H[o0:o1]
            if prop == 1:
                xi = xi * self.force_weight
                He = He * self.force_weight
            w = self.nets.weights[o0:o1]      # a view: the updater changes the weights in place
            self.updater[e].update(w, He, xi)
        return err

    def update_full(self, prop, candidates):
        """jacobian_mode 2: every candidate its own observation (columns of
        H, entries of xi), one updater step."""
        errs, cols = [], []
        for s, atom, comp in candidates:
            err, H = self.observation(prop, s, atom, comp)
            errs.append(err)
            cols.append(H * (self.force_weight if prop == 1 else 1.0))
        xi = np.array(errs) * (self.force_weight if prop == 1 else 1.0)
        self.updater.update(self.nets.weights, np.stack(cols, axis=1), xi)
        return errs

    def update_batch(self, prop, candidates):
        """One update from a task batch of candidates: errors and Jacobians
        summed at the same weights, then the force weight
        (Training.cpp:2879-2923, jacobian_mode 0/1 on one process)."""
        errs, Hs = 0.0, None
        out = []
        for s, atom, comp in candidates:
            err, H = self.observation(prop, s, atom, comp)
            out.append(err)
            errs = errs + err
            Hs = H if Hs is None else Hs + H
        if prop == 1:
            errs = errs * self.force_weight
            Hs = Hs * self.force_weight
        self.updater.update(self.nets.weights, Hs, errs)
        return out
