"""Bind the B200 hot path into the reference's own SCF driver.

``bind(scf_module)`` rebinds, in the reference module ``qepy_pw.pw.scf``,
the three names its SCF loop looks up at call time:

  LocalPotentialWorkspace  (qepy_pw/pw/scf.py:379, 1417, 2310)
  PlaneWaveHamiltonian     (qepy_pw/pw/scf.py:3396-3411)
  davidson                 (qepy_pw/pw/scf.py:3510-3538)

so that the reference's run_scf, unmodified, runs its H|psi>, Davidson and
density accumulation on the GPU.  The reference's host code keeps NumPy
arrays, so the bound objects take and return NumPy at this edge:

* ``DropInWorkspace`` wraps the reference's own workspace.  Its
  ``accumulate_density`` (qepy_pw/basis.py:1210-1215) and ``apply``
  (:1354-1362) run on a lazily built GPU workspace; every other attribute
  and method (the charge-density grid transforms, the maps the memory
  report reads) is the wrapped reference workspace's.
* ``HostHamiltonian`` is the GPU PlaneWaveHamiltonian built from the
  reference's constructor arguments: it unwraps the workspace, converts the
  reference's projector term objects (qepy_pw/diagonalization.py:21-43)
  and keeps ``apply`` / ``apply_into`` NumPy in, NumPy out.
* ``host_davidson`` runs the GPU Davidson and returns its eigenvectors as
  a column-major NumPy array (the reference feeds them to NumPy code:
  qepy_pw/pw/scf.py:3554, 3632, 1423).

Arithmetic is the plain FP64 form, so the reference's SCF reproduces its
own results.  ``bound(scf_module)`` is the same as a context manager that
restores the reference's names on exit.
"""

from __future__ import annotations

from contextlib import contextmanager

import numpy as np
import torch

from .basis import LocalPotentialWorkspace
from .diagonalization import (
    FactorizedProjectorTerm,
    PackedProjectorTerm,
    PlaneWaveHamiltonian,
    davidson,
)

NAMES = ("LocalPotentialWorkspace", "PlaneWaveHamiltonian", "davidson")


def _miller(indices_or_basis) -> np.ndarray:
    indices = getattr(indices_or_basis, "indices", indices_or_basis)
    return np.ascontiguousarray(np.asarray(indices, dtype=np.int32))


class DropInWorkspace:
    """The reference's LocalPotentialWorkspace with its wave-function
    operations (apply, accumulate_density) on the GPU."""

    reference_class = None  # set by bind(): the reference's own workspace class

    def __init__(self, indices_or_basis, shape, **options) -> None:
        object.__setattr__(self, "_reference",
                           type(self).reference_class(indices_or_basis, shape, **options))
        object.__setattr__(self, "_miller", _miller(indices_or_basis))
        object.__setattr__(self, "_shape", tuple(int(v) for v in shape))
        object.__setattr__(self, "_gpu", None)

    def __getattr__(self, name):
        return getattr(object.__getattribute__(self, "_reference"), name)

    def __setattr__(self, name, value) -> None:
        setattr(object.__getattribute__(self, "_reference"), name, value)

    def gpu_workspace(self) -> LocalPotentialWorkspace:
        if self._gpu is None:
            object.__setattr__(self, "_gpu", LocalPotentialWorkspace(self._miller, self._shape,
                                                                     precision="f64"))
        return self._gpu

    def apply(self, real_potential, coefficients, *, native_potential_layout=False, out=None,
              diagonal=None):
        return self.gpu_workspace().apply(real_potential, coefficients,
                                          native_potential_layout=native_potential_layout,
                                          out=out, diagonal=diagonal)

    def accumulate_density(self, density, coefficients, band_weights) -> None:
        self.gpu_workspace().accumulate_density(density, coefficients, band_weights)


def convert_terms(terms) -> tuple:
    """The reference's projector term objects as this package's types."""
    out = []
    for term in terms:
        if hasattr(term, "phases"):
            out.append(FactorizedProjectorTerm(term.beta, term.phases, term.coupling))
        elif hasattr(term, "diagonal") and hasattr(term, "beta"):
            out.append(PackedProjectorTerm(term.beta, term.coupling, term.diagonal))
        else:
            beta, coupling = term
            out.append((beta, coupling))
    return tuple(out)


class HostHamiltonian(PlaneWaveHamiltonian):
    """GPU PlaneWaveHamiltonian from the reference's constructor arguments
    (qepy_pw/diagonalization.py:127-137); NumPy in, NumPy out."""

    def __init__(self, basis, potential_g, projector_terms=(), local_workspace=None, timers=None,
                 real_potential=None, native_potential_layout=False,
                 potential_average=None) -> None:
        if isinstance(local_workspace, DropInWorkspace):
            workspace = local_workspace.gpu_workspace()
        elif isinstance(local_workspace, LocalPotentialWorkspace):
            workspace = local_workspace
        else:
            shape = local_workspace.shape if local_workspace is not None else np.shape(potential_g)
            workspace = LocalPotentialWorkspace(_miller(basis), shape, precision="f64")
        super().__init__(basis, potential_g, convert_terms(projector_terms),
                         local_workspace=workspace, timers=timers, real_potential=real_potential,
                         native_potential_layout=native_potential_layout,
                         potential_average=potential_average)


def host_davidson(operator, diagonal, number_of_roots, **options):
    """The GPU Davidson with the reference's signature
    (qepy_pw/diagonalization.py:527-548); eigenvectors come back as a
    column-major complex128 NumPy array."""
    options.pop("mpi", None)
    result = davidson(operator, diagonal, number_of_roots, **options)
    vectors = result.eigenvectors
    if isinstance(vectors, torch.Tensor):
        vectors = np.asfortranarray(vectors.to(torch.complex128).cpu().numpy())
    return type(result)(np.asarray(result.eigenvalues), vectors, np.asarray(result.residual_norms),
                        result.iterations, result.converged, result.number_unconverged,
                        result.hamiltonian_applications)


def bind(scf_module) -> dict:
    """Rebind the reference SCF module's hot-path names; returns the
    originals (``unbind`` puts them back)."""
    saved = {name: getattr(scf_module, name) for name in NAMES}
    workspace = type("DropInWorkspace", (DropInWorkspace,),
                     {"reference_class": saved["LocalPotentialWorkspace"]})
    scf_module.LocalPotentialWorkspace = workspace
    scf_module.PlaneWaveHamiltonian = HostHamiltonian
    scf_module.davidson = host_davidson
    return saved


def unbind(scf_module, saved: dict) -> None:
    for name, value in saved.items():
        setattr(scf_module, name, value)


@contextmanager
def bound(scf_module):
    saved = bind(scf_module)
    try:
        yield scf_module
    finally:
        unbind(scf_module, saved)
