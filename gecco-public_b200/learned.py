"""Learned correction of the diagonal preconditioner: sampling, training and
the instance stream it is trained on (host driver of gccu_lp_*).

The reference's amplitude step is diavc, -R/D (baserout/diavc.f:31-35,
called from optc_diis_sbsp_add, solve/optc_diis_sbsp_add.f:125-145).  The
engine's learned step multiplies it per element by 1 + tanh(o), o the output
of a small perceptron over the element's denominator and the product of its
normalised current and previous steps (include/gccu.h, gccu_lp_*).  It is
trained on (state, converged step) pairs that the solver generates itself:
during plain diagonal + DIIS solves of earlier instances every step samples
elements of the amplitude lists (inputs, plain step, amplitude); after
convergence the targets are converged amplitude - sampled amplitude.  The
loss, the gradient and the Adam steps run on the device.

Instance stream: seeded synthetic closed-shell CCSD Hamiltonians with
n_occ ~ U[6,16], n_virt ~ U[30,120], a HOMO-LUMO gap ~ U[0.2,0.8] Eh and the
integral distribution of the benchmark family (n_aux = 160, B ~ N(0, 0.05^2)).
With that distribution the doubles coupling grows like sqrt(n_occ n_virt)
against fixed gaps and plain diagonal + DIIS stalls or diverges from about
n_virt = 60 on; scale_sigma draws B with the standard deviation
0.035 (180 / (n_occ n_virt))^(1/4) instead, which keeps every size of the
stream convergent.
"""
import numpy as np

import cc
import hamiltonian as hm

LP_SAMPLES = 2048  # sampled elements per amplitude list and step
TRAIN = dict(steps=3000, batch=8192, lr=3e-3)


def stream(n, seed=4000, nocc=(6, 16), nvir=(30, 120), gap=(0.2, 0.8), naux=160,
           sigma=0.05, scale_sigma=False):
    """instance parameters (nocc, nvir, naux, gap, sigma, seed), seeded"""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        o = int(rng.integers(nocc[0], nocc[1] + 1))
        v = int(rng.integers(nvir[0], nvir[1] + 1))
        sg = 0.035 * (180.0 / (o * v)) ** 0.25 if scale_sigma else sigma
        out.append(dict(nocc=o, nvir=v, naux=naux, gap=float(rng.uniform(*gap)), sigma=sg,
                        seed=seed + 1 + k))
    return out


def hamiltonian(inst):
    return hm.synthetic(inst["nocc"], inst["nvir"], inst["naux"], seed=inst["seed"],
                        gap=inst["gap"], sigma=inst.get("sigma", 0.05))


class Sampler:
    """records (inputs, plain step, amplitude) rows of LP_SAMPLES elements of
    every amplitude list before each step; targets() turns them into training
    rows once the solve has converged"""

    def __init__(self, seed=0, per_list=LP_SAMPLES):
        self.rng = np.random.default_rng(seed)
        self.per_list = per_list
        self.rows = {}

    def __call__(self, s):
        e = s.e
        for a in s.amps:
            n = s.lists[a][1]
            idx = self.rng.choice(n, min(n, self.per_list), replace=False)
            rows = e.lp_rows(s.lid(s.res[a]), s.lid("D" + a), s.lid("P" + a), s.lid(a), idx,
                             fac=-1.0, shift=s.shift)
            self.rows.setdefault(a, []).append((idx, rows))

    def targets(self, s):
        """(rows[n,5], target[n]) with target = converged - sampled amplitude"""
        out_r, out_t = [], []
        for a, recs in self.rows.items():
            tconv = s.e.download(s.lid(a), s.lists[a][1])
            for idx, rows in recs:
                out_r.append(rows)
                out_t.append(tconv[idx] - rows[:, 4])
        if not out_r:
            return np.zeros((0, 5)), np.zeros(0)
        return np.concatenate(out_r), np.concatenate(out_t)


def initial_weights(seed=1):
    """small random weights (output near 0: the plain step to start with)"""
    rng = np.random.default_rng(seed)
    nh, ni = 32, 3
    W1 = rng.normal(0.0, 1.0 / np.sqrt(ni), (nh, ni))
    W2 = rng.normal(0.0, 1.0 / np.sqrt(nh), (nh, nh))
    W3 = rng.normal(0.0, 0.01, nh)
    return np.concatenate([W1.ravel(), np.zeros(nh), W2.ravel(), np.zeros(nh), W3, [0.0]])


def train(engine, rows, target, seed=1, steps=None, batch=None, lr=None):
    """Adam on the device from initial_weights(seed); returns (weights,
    full-set loss before, after)"""
    engine.lp_set_weights(initial_weights(seed))
    engine.lp_load_samples(rows, target)
    _, l0 = engine.lp_gradient()
    engine.lp_train(steps or TRAIN["steps"], batch or TRAIN["batch"], lr or TRAIN["lr"],
                    seed=seed)
    _, l1 = engine.lp_gradient()
    return engine.lp_get_weights(), l0, l1


def solve(engine, inst, weights=None, sampler=None, maxiter=80, conv=1e-9, mixed=False,
          callback=None):
    """one CCSD solve of an instance (Hamiltonian generated on the device):
    plain diagonal + DIIS, or with the learned step when weights are given;
    returns the solver"""
    from devfill import TorchIntegrals
    sp, eps, B = hamiltonian(inst)
    s = cc.CCSolver(engine, hm.FactorizedIntegrals(sp, eps, B), method="ccsd", learned=weights)
    s.load_hamiltonian_device(TorchIntegrals(sp, eps, B))
    s.recorder = sampler
    if mixed:
        s.solve_mixed(maxiter=maxiter, conv=conv, callback=callback)
    else:
        s.solve(maxiter=maxiter, conv=conv, use_graph=True, callback=callback)
    return s


def iterations_to(history, e_ref, tol=1e-6):
    """first iteration whose energy is within tol of e_ref (None: never)"""
    return next((h[0] for h in history if abs(h[1] - e_ref) < tol), None)
