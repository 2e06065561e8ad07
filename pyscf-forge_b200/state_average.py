"""State-averaged CSF solver: the mcscf ``state_average_`` protocol as the
reference implements it for its GAS solver (pyscf/mcscf/addons_gas.py:
103-286), around the GPU solvers of this package.

``state_average(fcisolver, weights)`` returns a solver whose ``kernel``
solves ``len(weights)`` roots and returns the weighted energy (root energies
in ``e_states``), and whose ``make_rdm1/1s/12/12s`` return the weighted
RDMs (computed on the device by the adjoint kernel, csffci_rdm12 /
csffci_rdm12s).  These are the state-averaged densities a CASSCF orbital
gradient consumes; ``autograd.csf_fci_energy`` gives the same averaged RDMs
as the gradient of ``(w * E).sum()``.
"""
import numpy as np
import torch

from .fci import direct_spin1 as D


def validate_state_weights(weights):
    """Non-empty, finite, non-negative weights summing to one
    (addons_gas.py:103-114)."""
    weights = np.asarray(weights, dtype=np.float64)
    if weights.ndim != 1 or weights.size == 0:
        raise ValueError("weights must be a non-empty one-dimensional array")
    if not np.all(np.isfinite(weights)):
        raise ValueError("weights must be finite")
    if np.any(weights < 0.0):
        raise ValueError("weights must be non-negative")
    if abs(float(weights.sum()) - 1.0) > 1e-10:
        raise ValueError("weights must sum to one")
    return weights


class StateAverageFCISolver:
    """Weighted multi-root wrapper (addons_gas.py:116-210).  Attributes not
    defined here are those of the wrapped solver."""

    def __init__(self, fcisolver, weights=(0.5, 0.5), wfnsym=None):
        object.__setattr__(self, "_base", fcisolver)
        self.weights = validate_state_weights(weights)
        self.e_states = None
        if wfnsym is not None:
            fcisolver.wfnsym = wfnsym

    def __getattr__(self, name):
        return getattr(object.__getattribute__(self, "_base"), name)

    def __setattr__(self, name, value):
        if name in ("weights", "e_states"):
            object.__setattr__(self, name, value)
        else:
            setattr(self._base, name, value)

    @property
    def nroots(self):
        return len(self.weights)

    def kernel(self, h1e, eri, norb, nelec, ci0=None, **kwargs):
        self._base.nroots = len(self.weights)
        kwargs.pop("nroots", None)
        e, c = self._base.kernel(h1e, eri, norb, nelec, ci0=ci0, **kwargs)
        e = np.atleast_1d(np.asarray(e, dtype=np.float64))
        self.e_states = e
        c = c if isinstance(c, list) else [c]
        return float(np.dot(self.weights, e)), c

    @property
    def e_average(self):
        return float(np.dot(self.weights, self.e_states))

    # ---- per-state densities (device RDM kernels) ---------------------
    def states_make_rdm1(self, ci0, norb, nelec, *args, **kwargs):
        return [D.make_rdm1(c, norb, nelec) for c in ci0]

    def states_make_rdm1s(self, ci0, norb, nelec, *args, **kwargs):
        res = [D.make_rdm1s(c, norb, nelec) for c in ci0]
        return [r[0] for r in res], [r[1] for r in res]

    def states_make_rdm12(self, ci0, norb, nelec, *args, **kwargs):
        res = [D.make_rdm12(c, norb, nelec) for c in ci0]
        return [r[0] for r in res], [r[1] for r in res]

    def states_make_rdm12s(self, ci0, norb, nelec, *args, **kwargs):
        res = [D.make_rdm12s(c, norb, nelec) for c in ci0]
        dm1a = [r[0][0] for r in res]
        dm1b = [r[0][1] for r in res]
        return (dm1a, dm1b), ([r[1][0] for r in res], [r[1][1] for r in res], [r[1][2] for r in res])

    def states_trans_rdm12(self, ci1, ci0, norb, nelec, *args, **kwargs):
        res = [D.trans_rdm12(b, k, norb, nelec) for b, k in zip(ci1, ci0)]
        return [r[0] for r in res], [r[1] for r in res]

    def states_spin_square(self, ci0, norb, nelec, *args, **kwargs):
        from .csf_fci.spin_op import spin_square
        res = [spin_square(c, norb, nelec) for c in ci0]
        return [r[0] for r in res], [r[1] for r in res]

    # ---- weighted densities ---------------------------------------------
    def _avg(self, mats):
        out = None
        for w, m in zip(self.weights, mats):
            term = w * (m if isinstance(m, torch.Tensor) else np.asarray(m))
            out = term if out is None else out + term
        return out

    def make_rdm1(self, ci0, norb, nelec, *args, **kwargs):
        return self._avg(self.states_make_rdm1(ci0, norb, nelec))

    def make_rdm1s(self, ci0, norb, nelec, *args, **kwargs):
        a, b = self.states_make_rdm1s(ci0, norb, nelec)
        return self._avg(a), self._avg(b)

    def make_rdm12(self, ci0, norb, nelec, *args, **kwargs):
        d1, d2 = self.states_make_rdm12(ci0, norb, nelec)
        return self._avg(d1), self._avg(d2)

    def make_rdm12s(self, ci0, norb, nelec, *args, **kwargs):
        (a, b), (aa, ab, bb) = self.states_make_rdm12s(ci0, norb, nelec)
        return (self._avg(a), self._avg(b)), (self._avg(aa), self._avg(ab), self._avg(bb))

    def spin_square(self, ci0, norb, nelec, *args, **kwargs):
        """Weighted <S^2> and its multiplicity (addons_gas.py:193-198)."""
        ss = np.asarray(self.states_spin_square(ci0, norb, nelec)[0])
        ss_average = float(np.dot(self.weights, ss))
        return ss_average, np.sqrt(max(0.0, 4.0 * ss_average + 1.0))

    def undo_state_average(self):
        return self._base


def state_average(fcisolver, weights=(0.5, 0.5), wfnsym=None):
    """A state-averaged view of a solver (or of ``mc.fcisolver`` for an
    object that carries one, which is then updated in place as
    state_average_ does, addons_gas.py:249-283)."""
    if hasattr(fcisolver, "fcisolver"):
        return state_average_(fcisolver, weights, wfnsym)
    if isinstance(fcisolver, StateAverageFCISolver):
        fcisolver = fcisolver.undo_state_average()
    return StateAverageFCISolver(fcisolver, weights, wfnsym)


def state_average_(mc, weights=(0.5, 0.5), wfnsym=None):
    """In place on an MCSCF-like object: its fcisolver becomes the
    state-averaged wrapper."""
    mc.fcisolver = state_average(mc.fcisolver if not isinstance(mc.fcisolver, StateAverageFCISolver)
                                 else mc.fcisolver.undo_state_average(), weights, wfnsym)
    return mc


__all__ = ["StateAverageFCISolver", "state_average", "state_average_", "validate_state_weights"]
