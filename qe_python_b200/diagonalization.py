"""GPU plane-wave Hamiltonian and block Davidson eigensolver.

Drop-in for qepy_pw/diagonalization.py: ``PlaneWaveHamiltonian`` keeps the
constructor and ``apply`` / ``apply_into`` / ``diagonal`` of :124-244 and the
projector term types of :21-43; ``davidson`` keeps the signature and result
type of :527-548 / :113-121 and follows the algorithm of :527-880 step by
step.  Vectors are column-major torch CUDA tensors; every contraction runs in
libqeb200.so (complex GEMMs, FFT passes, column kernels).  The reduced
Hermitian generalized eigenproblem is solved in FP64 on the device
(Cholesky reduction + Hermitian eigensolve, the same transformation as
LAPACK zhegv).
"""

from __future__ import annotations

import weakref
from contextlib import nullcontext
from dataclasses import dataclass

import numpy as np
import torch

from . import kernels as K
from .basis import FFTScratchPool, LocalPotentialWorkspace, PlaneWaveBasis, apply_local_multi
from .device import (
    COMPLEX_OF,
    REAL_OF,
    as_numpy,
    empty_f,
    leading_dimension,
    require_cuda,
    to_device_f,
    zeros_f,
)
from .eigensolver import ReducedSolve


@dataclass(frozen=True)
class FactorizedProjectorTerm:
    """Species beta functions plus per-atom phase columns (diagonalization.py:21-28);
    ``phases`` may be a host array or a device tensor."""

    beta: np.ndarray
    phases: "np.ndarray | torch.Tensor"
    coupling: np.ndarray


@dataclass(frozen=True)
class PackedProjectorTerm:
    """Atom-packed beta with a precomputed diagonal (diagonalization.py:31-37)."""

    beta: np.ndarray
    coupling: np.ndarray
    diagonal: np.ndarray


@dataclass(frozen=True)
class DavidsonResult:
    """Same fields as qepy_pw/diagonalization.py:113-121 (eigenvectors on the device)."""

    eigenvalues: np.ndarray
    eigenvectors: torch.Tensor
    residual_norms: np.ndarray
    iterations: float
    converged: bool
    number_unconverged: int = 0
    hamiltonian_applications: int = 0


class StreamPool:
    """Streams reused across Hamiltonians and Davidson solves.

    The caching allocator keeps one pool of blocks per stream, so work put on
    a stream created for one Hamiltonian or one solve allocated its buffers
    with new device allocations (which waited for the queued GPU work: 33 of
    them, 0.34 s, in the 216-atom mixed SCF after a warm-up run), and the
    split-K scratch kept per stream stayed alive with every such stream.
    ``shared(device)``: the side stream of the projector products;
    ``acquire(device)`` / ``release``: a stream that no other holder uses
    until it is released (the overlapped reduced solves of lockstep k
    points)."""

    def __init__(self) -> None:
        self._shared: dict = {}
        self._free: dict = {}

    @staticmethod
    def _key(device) -> int:
        device = torch.device(device)
        return device.index if device.index is not None else torch.cuda.current_device()

    def shared(self, device) -> torch.cuda.Stream:
        key = self._key(device)
        stream = self._shared.get(key)
        if stream is None:
            stream = self._shared[key] = torch.cuda.Stream(device=key)
        return stream

    def acquire(self, device) -> torch.cuda.Stream:
        free = self._free.setdefault(self._key(device), [])
        return free.pop() if free else torch.cuda.Stream(device=self._key(device))

    def release(self, stream: torch.cuda.Stream) -> None:
        self._free.setdefault(stream.device.index, []).append(stream)


STREAMS = StreamPool()


def _solver(device, overlap_solves: bool) -> ReducedSolve:
    """The reduced-problem solver of one Davidson run: on the current stream,
    or for overlapped solves on a pooled stream returned when the solver is
    collected (the generator that holds it finished)."""
    if not overlap_solves:
        return ReducedSolve(torch.cuda.current_stream(device))
    stream = STREAMS.acquire(device)
    solver = ReducedSolve(stream)
    weakref.finalize(solver, STREAMS.release, stream)
    return solver


def _timer(timers, name):
    return timers.measure(name) if timers is not None else nullcontext()


class _DeviceProjectors:
    """All projector terms packed into one device beta (npw, P) and a dense
    block-diagonal coupling (P, P).

    A factorized term (species beta, per-atom phases) becomes beta * phase per
    atom: (beta*phase)^H psi equals the reference's conj(beta^T (conj(psi)
    phase)) (diagonalization.py:294-310) and (beta*phase) D becp equals its
    (beta D becp) * phase (:362-367).  Packing costs npw*P complex values of
    HBM, which the GPU holds easily, and turns the per-atom loop into two
    GEMMs.
    """

    def __init__(self, terms, npw: int, dtype: torch.dtype, device: torch.device) -> None:
        self.npw, self.dtype = int(npw), dtype
        betas, couplings, diagonals = [], [], []
        self.host_diagonal = np.zeros(npw)
        self.device_diagonal = torch.zeros(npw, dtype=torch.float64, device=device)
        for term in terms:
            if isinstance(term, PackedProjectorTerm):
                beta = to_device_f(term.beta, torch.complex128, device)
                betas.append(beta)
                couplings.append(np.asarray(term.coupling))
                diagonals.append(("packed", term.diagonal))
            elif isinstance(term, FactorizedProjectorTerm):
                species = to_device_f(term.beta, torch.complex128, device)
                phases = to_device_f(term.phases, torch.complex128, device)
                natoms = phases.shape[1]
                c = species.shape[1]
                packed = empty_f(npw, natoms * c, torch.complex128, device)
                for atom in range(natoms):
                    packed[:, atom * c:(atom + 1) * c] = species * phases[:, atom:atom + 1]
                betas.append(packed)
                couplings.append(np.kron(np.eye(natoms), np.asarray(term.coupling)))
                diagonals.append(("factorized", species, np.asarray(term.coupling), natoms))
            else:
                beta, coupling = term
                beta = to_device_f(beta, torch.complex128, device)
                betas.append(beta)
                couplings.append(np.asarray(coupling))
                diagonals.append(("materialized", beta, np.asarray(coupling), 1))
        self.channels = sum(b.shape[1] for b in betas)
        if self.channels == 0:
            self.beta = None
            self.coupling = None
        else:
            beta = empty_f(npw, self.channels, torch.complex128, device)
            coupling = np.zeros((self.channels, self.channels), dtype=np.complex128)
            offset = 0
            for b, c in zip(betas, couplings):
                n = b.shape[1]
                beta[:, offset:offset + n] = b
                coupling[offset:offset + n, offset:offset + n] = c
                offset += n
            self.beta = to_device_f(beta, dtype, device) if dtype != torch.complex128 else beta
            self.coupling = to_device_f(coupling, dtype, device)
            self.block_coupling = K.BlockCoupling(coupling, dtype, device)
        self._packed_conj = None
        self._packed_plain = None
        self._diagonal_terms(diagonals, npw, device)

    # Packed split-TF32 copies of beta for qeb_tf32_gemm, made on first use:
    # only needed when the operands cannot go to cgemm_tf32x3 directly.
    @property
    def packed_conj(self):
        if self._packed_conj is None and self.beta is not None and self.beta.dtype == torch.complex64:
            self._packed_conj = K.tf32_pack(self.beta, K.PACK_RAW)
        return self._packed_conj

    @property
    def packed_plain(self):
        if self._packed_plain is None and self.beta is not None and self.beta.dtype == torch.complex64:
            self._packed_plain = K.tf32_pack(self.beta, K.PACK_RAW, transposed=True)
        return self._packed_plain

    def _diagonal_terms(self, diagonals, npw, device):
        # Preconditioner diagonal (diagonalization.py:205-229).
        for entry in diagonals:
            if entry[0] == "packed":
                self.device_diagonal += to_device_f(entry[1], torch.float64, device)
                continue
            _kind, beta, coupling, multiplicity = entry
            coupled = K.gemm(K.OP_N, beta, to_device_f(coupling.astype(np.complex128),
                                                       torch.complex128, device))
            K.accumulate_projector_diagonal(self.device_diagonal, coupled, beta,
                                            float(multiplicity))


class PlaneWaveHamiltonian:
    """H = T + V_loc + sum |beta> D <beta| applied on the GPU.

    Same constructor as qepy_pw/diagonalization.py:127-203 plus ``precision``
    ('f64' plain or 'f32' chosen form; taken from ``local_workspace`` when
    given).
    """

    def __init__(self, basis: PlaneWaveBasis, potential_g, projector_terms=(),
                 local_workspace: LocalPotentialWorkspace | None = None, timers=None,
                 real_potential=None, native_potential_layout: bool = False,
                 potential_average: float | None = None, precision: str | None = None,
                 device_projectors: "_DeviceProjectors | None" = None) -> None:
        """``device_projectors``: the device form of ``projector_terms`` built
        by an earlier Hamiltonian of the same basis and precision (its
        ``projectors`` attribute); the SCF reuses it across iterations because
        the projectors depend on the ions only."""
        self.basis = basis
        self.potential_g = potential_g
        if local_workspace is None:
            shape = np.asarray(potential_g).shape if np.ndim(potential_g) == 3 else None
            if shape is None:
                raise ValueError("a local workspace or a 3-D potential_g is required")
            local_workspace = LocalPotentialWorkspace(basis, shape, precision=precision or "f64")
        elif precision is not None and precision != local_workspace.precision:
            raise ValueError("precision disagrees with the local workspace")
        self.local_workspace = local_workspace
        self.precision = local_workspace.precision
        self.dtype = local_workspace.complex_dtype
        self.device = local_workspace.device
        self.timers = timers
        self.native_potential_layout = bool(native_potential_layout)
        if real_potential is None:
            real_potential = local_workspace.prepare_potential(potential_g)
            self.native_potential_layout = False
        self.real_potential = real_potential
        if potential_average is None:
            potential_average = float(np.real(np.asarray(potential_g).flat[0]))
        self.potential_average = float(potential_average)
        self.mpi = None
        self.local_rows = np.arange(len(basis), dtype=np.int32)
        kinetic = np.asarray(basis.kinetic, dtype=float)
        self.local_kinetic = kinetic
        self._kinetic = torch.from_numpy(kinetic).to(self.device)
        self._kinetic_kernel = self._kinetic.to(REAL_OF[self.dtype])
        self._potential = local_workspace.native_potential(real_potential, self.native_potential_layout)
        if device_projectors is not None:
            if device_projectors.dtype != self.dtype or device_projectors.npw != len(basis):
                raise ValueError("device_projectors were built for another basis or precision")
            self.projectors = device_projectors
        else:
            self.projectors = _DeviceProjectors(projector_terms, len(basis), self.dtype, self.device)
        # chosen form: projector GEMMs as split-TF32 tcgen05 products
        self.tensor_gemm = self.dtype == torch.complex64
        self.projector_terms = tuple(projector_terms)
        self._diagonal_device = self._kinetic + self.potential_average + self.projectors.device_diagonal

    # The three nonlocal stages (reference: diagonalization.py:280-368).
    def calbec(self, vectors: torch.Tensor) -> torch.Tensor:
        """becp = beta^H psi (projector_overlaps, _native_fft.pyx:694-731)."""
        p = self.projectors
        if self.tensor_gemm and not K.is_skinny(K.OP_C, p.beta.shape[1], vectors.shape[1]):
            out = K.cgemm_tf32x3(K.OP_C, p.beta, vectors)
            if out is not None:
                return out
            return K.gemm_tf32(K.OP_C, p.beta, vectors, a_packed=p.packed_conj)
        return K.gemm(K.OP_C, p.beta, vectors)

    def couple(self, becp: torch.Tensor) -> torch.Tensor:
        """coupled = D becp with the block-diagonal 0.5 D_Ry (diagonalization.py:348)."""
        return self.projectors.block_coupling.apply(becp)

    def add_projectors(self, coupled: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        """target += beta coupled (add_projector_product, _native_fft.pyx:782-836)."""
        p = self.projectors
        if self.tensor_gemm and not K.is_skinny(K.OP_N, p.beta.shape[0], coupled.shape[1]):
            out = K.cgemm_tf32x3(K.OP_N, p.beta, coupled, target, beta=1.0)
            if out is not None:
                return out
            return K.gemm_tf32(K.OP_N, p.beta, coupled, target, beta=1.0, a_packed=p.packed_plain)
        return K.gemm(K.OP_N, p.beta, coupled, target, beta=1.0)

    @property
    def diagonal(self) -> torch.Tensor:
        """T + v_of_0 + projector diagonal on the device (usnldiag; :205-229)."""
        return self._diagonal_device

    def apply(self, coefficients):
        with _timer(self.timers, "h_psi"):
            return self._apply(coefficients)

    def apply_into(self, coefficients, out):
        with _timer(self.timers, "h_psi"):
            return self._apply(coefficients, out=out)

    def _side_stream(self) -> torch.cuda.Stream:
        """The stream of the projector products that overlap the FFT passes:
        one per device, shared by the Hamiltonians (a captured graph sets its
        own on the Hamiltonian)."""
        stream = getattr(self, "_stream_side", None)
        if stream is None:
            stream = STREAMS.shared(self.device)
        return stream

    def add_nonlocal(self, vectors: torch.Tensor, target: torch.Tensor) -> None:
        """target += sum |beta> D <beta|vectors> (calbec, D, add)."""
        if self.projectors.beta is None or vectors.shape[1] == 0:
            return
        if self.tensor_gemm and (leading_dimension(vectors) % 2 or vectors.data_ptr() % 16):
            aligned = empty_f(vectors.shape[0], vectors.shape[1], self.dtype, self.device)
            aligned.copy_(vectors)
            vectors = aligned
        with _timer(self.timers, "h_psi:calbec"):
            becp = self.calbec(vectors)
        with _timer(self.timers, "add_vuspsi"):
            self.add_projectors(self.couple(becp), target)

    def _apply(self, coefficients, out=None):
        host = not isinstance(coefficients, torch.Tensor)
        vectors = to_device_f(coefficients, self.dtype, self.device)
        was_vector = vectors.dim() == 1
        if was_vector:
            vectors = vectors[:, None]
        if self.tensor_gemm and vectors.shape[1] > 0 and \
                (leading_dimension(vectors) % 2 or vectors.data_ptr() % 16):
            # the split-TF32 GEMM reads 16-byte aligned columns: one copy here
            # is cheaper than packing both projector operands
            aligned = empty_f(vectors.shape[0], vectors.shape[1], self.dtype, self.device)
            aligned.copy_(vectors)
            vectors = aligned
        target = None
        if out is not None and isinstance(out, torch.Tensor):
            target = out[:, None] if out.dim() == 1 else out
        if target is None:
            target = empty_f(vectors.shape[0], vectors.shape[1], self.dtype, self.device)
        nonlocal_part = self.projectors.beta is not None and vectors.shape[1] > 0
        if nonlocal_part and self.timers is None:
            # beta^H psi and D becp need only psi: they run on a side stream
            # while the FFT passes write the local part into target, and the
            # projector add joins after both
            main = torch.cuda.current_stream(self.device)
            side = self._side_stream()
            side.wait_stream(main)
            with torch.cuda.stream(side):
                coupled = self.couple(self.calbec(vectors))
            self.local_workspace._launch_apply(self._potential, vectors, self._kinetic_kernel, target)
            main.wait_stream(side)
            coupled.record_stream(main)
            self.add_projectors(coupled, target)
        else:
            with _timer(self.timers, "vloc_psi"):
                self.local_workspace._launch_apply(self._potential, vectors, self._kinetic_kernel,
                                                   target)
            if nonlocal_part:
                with _timer(self.timers, "h_psi:calbec"):
                    becp = self.calbec(vectors)
                with _timer(self.timers, "add_vuspsi"):
                    self.add_projectors(self.couple(becp), target)
        if host:
            result = as_numpy(target)
            if out is not None and not isinstance(out, torch.Tensor):
                out[...] = result.reshape(out.shape)
                result = out
            return result[:, 0] if was_vector and result.ndim == 2 else result
        return target[:, 0] if was_vector else target


class HpsiGraph:
    """H|psi> of a fixed band count captured once as a CUDA graph.

    Every kernel of the application (FFT passes, operand packing, projector
    GEMMs, coupling) is recorded on the capture stream; ``__call__`` copies
    the input into the captured buffer, replays the graph and copies the
    result out, so one host call issues the whole H|psi> with no per-kernel
    launch overhead.
    """

    def __init__(self, ham: PlaneWaveHamiltonian, nbands: int, private: bool = False) -> None:
        """``private``: the graph gets its own stick scratch, side stream and
        split-K scratch, so that it can replay concurrently with the other
        private graphs of the same Hamiltonian (by default the graphs of one
        Hamiltonian share them and must replay one after another)."""
        npw = len(ham.basis)
        self.ham = ham
        self.nbands = int(nbands)
        self.input = zeros_f(npw, self.nbands, ham.dtype, ham.device)
        self.output = zeros_f(npw, self.nbands, ham.dtype, ham.device)
        # the (nbands, ld) row-major storage behind the column-major buffers:
        # one contiguous block, so a host copy of the same shape is one DMA
        self.input_storage = self.input.T.as_strided(
            (self.nbands, leading_dimension(self.input)), (leading_dimension(self.input), 1))
        self.output_storage = self.output.T.as_strided(
            (self.nbands, leading_dimension(self.output)), (leading_dimension(self.output), 1))
        stream = torch.cuda.Stream(device=ham.device)
        workspace = ham.local_workspace
        shared_pool, shared_side = workspace.scratch_pool, getattr(ham, "_stream_side", None)
        if private:
            workspace.scratch_pool = FFTScratchPool()
            ham._stream_side = torch.cuda.Stream(device=ham.device)
        try:
            stream.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(stream):
                # warm-up outside the capture: workspaces, attributes, scratch
                for _ in range(2):
                    ham.apply_into(self.input, self.output)
            torch.cuda.current_stream().wait_stream(stream)
            torch.cuda.synchronize()
            self.graph = torch.cuda.CUDAGraph()
            # a private graph captures on its warm-up stream, whose split-K
            # scratch is its own
            with torch.cuda.graph(self.graph, stream=stream if private else None):
                ham.apply_into(self.input, self.output)
            torch.cuda.synchronize()
        finally:
            # the private scratch and side stream stay alive with the graph
            self._scratch_pool, self._side = workspace.scratch_pool, ham._side_stream()
            workspace.scratch_pool = shared_pool
            if shared_side is None:
                if hasattr(ham, "_stream_side"):
                    del ham._stream_side
            else:
                ham._stream_side = shared_side

    def replay(self) -> torch.Tensor:
        self.graph.replay()
        return self.output

    def __call__(self, vectors: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        if tuple(vectors.shape) != tuple(self.input.shape):
            raise ValueError("the captured graph has a fixed band count")
        self.input.copy_(vectors)
        self.graph.replay()
        if out is None:
            return self.output.clone()
        out.copy_(self.output)
        return out


class HostStreamedHpsi:
    """H|psi> of host-resident band blocks with the PCIe copies overlapped.

    The bands are cut into chunks; chunk c is copied in on one stream, its
    H|psi> replayed from a captured graph on one of the compute streams
    (alternating, so chunk c's projector GEMMs can overlap chunk c+1's FFT
    passes), and its result copied out on another stream, so chunk c's
    compute overlaps chunk c+1's input and chunk c-1's output copies (H|psi>
    is independent per band; each graph has its own scratch).  Host buffers
    are pinned, with the (nbands, ld) storage layout of the device buffers so
    that each copy is one contiguous DMA.

    ``capture(host_in, host_out)`` records that whole pipeline for one pair
    of host buffers — every copy, every chunk's kernels and the cross-stream
    waits — as one CUDA graph, and ``replay()`` runs it: the host issues one
    launch per application instead of a few dozen stream operations, which
    otherwise left the copy engines and the SMs waiting for the host.

    ``chunks`` (sizes summing to nbands) replaces the equal chunks of
    ``chunk`` bands, each chunk with a buffer of its own: small first and
    last chunks start the compute early and shorten the final output copy,
    large middle ones keep the projector GEMMs' tiles full.
    """

    def __init__(self, ham: PlaneWaveHamiltonian, nbands: int, chunk: int = 64,
                 buffers: int = 2, compute_streams: int = 2, chunks=None) -> None:
        self.ham = ham
        self.nbands = int(nbands)
        if chunks is not None:
            self.sizes = [int(c) for c in chunks]
            if min(self.sizes, default=0) < 1 or sum(self.sizes) != self.nbands:
                raise ValueError("chunks must be positive sizes summing to nbands")
            self.chunk = max(self.sizes)
            sizes = self.sizes
        else:
            self.chunk = max(1, min(int(chunk), self.nbands))
            self.sizes = [min(self.chunk, self.nbands - start)
                          for start in range(0, self.nbands, self.chunk)]
            sizes = [self.chunk] * max(1, int(buffers))
        # private graphs: consecutive chunks replay on alternating compute
        # streams, so one chunk's projector GEMMs overlap the next one's FFTs
        self.graphs = [HpsiGraph(ham, size, private=True) for size in sizes]
        self.ld = self.graphs[0].input_storage.shape[1]
        self.copy_in = torch.cuda.Stream(device=ham.device)
        self.copy_out = torch.cuda.Stream(device=ham.device)
        self.computes = [torch.cuda.Stream(device=ham.device)
                         for _ in range(max(1, int(compute_streams)))]
        self._pipeline = None

    def host_buffers(self) -> tuple[torch.Tensor, torch.Tensor]:
        """Pinned (nbands, ld) input and output storage; band b's plane-wave
        coefficients are row b, columns [0, npw)."""
        dtype = self.ham.dtype
        make = lambda: torch.zeros((self.nbands, self.ld), dtype=dtype).pin_memory()  # noqa: E731
        return make(), make()

    def _check(self, host_in: torch.Tensor, host_out: torch.Tensor) -> None:
        if tuple(host_in.shape) != (self.nbands, self.ld) or host_in.shape != host_out.shape:
            raise ValueError("use buffers of host_buffers()")

    def _enqueue(self, host_in: torch.Tensor, host_out: torch.Tensor, captured: bool) -> None:
        """The pipeline's stream operations on the current stream's timeline;
        ``captured``: each chunk's H|psi> runs its kernels (with the private
        scratch of its buffer's graph) instead of replaying that graph."""
        n = len(self.graphs)
        ready_in, done_compute, done_out = [], [], []
        current = torch.cuda.current_stream(self.ham.device)
        for stream in (self.copy_in, self.copy_out, *self.computes):
            stream.wait_stream(current)
        workspace = self.ham.local_workspace
        starts = np.cumsum([0] + self.sizes[:-1])
        for index, (start, size) in enumerate(zip(starts.tolist(), self.sizes)):
            stop = start + size
            graph = self.graphs[index % n]
            with torch.cuda.stream(self.copy_in):
                if index >= n:  # the buffer's previous result has left the device
                    self.copy_in.wait_event(done_out[index - n])
                graph.input_storage[:stop - start].copy_(host_in[start:stop], non_blocking=True)
                if stop - start < graph.nbands:
                    graph.input_storage[stop - start:].zero_()
                ready_in.append(torch.cuda.Event())
                ready_in[-1].record(self.copy_in)
            compute = self.computes[index % len(self.computes)]
            with torch.cuda.stream(compute):
                compute.wait_event(ready_in[-1])
                if captured:
                    workspace.scratch_pool, self.ham._stream_side = graph._scratch_pool, graph._side
                    self.ham.apply_into(graph.input, graph.output)
                else:
                    graph.replay()
                done_compute.append(torch.cuda.Event())
                done_compute[-1].record(compute)
            with torch.cuda.stream(self.copy_out):
                self.copy_out.wait_event(done_compute[-1])
                host_out[start:stop].copy_(graph.output_storage[:stop - start], non_blocking=True)
                done_out.append(torch.cuda.Event())
                done_out[-1].record(self.copy_out)
        for stream in (self.copy_in, *self.computes, self.copy_out):
            current.wait_stream(stream)

    def __call__(self, host_in: torch.Tensor, host_out: torch.Tensor) -> None:
        """host_out = H host_in (both from host_buffers()); returns once the
        copies are queued; synchronise the device (or copy_out) to read."""
        self._check(host_in, host_out)
        self._enqueue(host_in, host_out, captured=False)

    def capture(self, host_in: torch.Tensor, host_out: torch.Tensor) -> None:
        """Record the pipeline for these two pinned buffers as one CUDA graph
        (after one eager run that settles allocations and tuned choices)."""
        self._check(host_in, host_out)
        if not (host_in.is_pinned() and host_out.is_pinned()):
            raise ValueError("captured copies need pinned host buffers")
        self(host_in, host_out)
        torch.cuda.synchronize()
        ham, workspace = self.ham, self.ham.local_workspace
        shared_pool, shared_side = workspace.scratch_pool, getattr(ham, "_stream_side", None)
        pipeline = torch.cuda.CUDAGraph()
        stream = torch.cuda.Stream(device=ham.device)
        stream.wait_stream(torch.cuda.current_stream(ham.device))
        try:
            with torch.cuda.graph(pipeline, stream=stream):
                self._enqueue(host_in, host_out, captured=True)
            torch.cuda.synchronize()
        finally:
            workspace.scratch_pool = shared_pool
            if shared_side is None:
                if hasattr(ham, "_stream_side"):
                    del ham._stream_side
            else:
                ham._stream_side = shared_side
        self._pipeline = (pipeline, host_in, host_out)

    def replay(self) -> None:
        """Run the captured pipeline (``capture`` first) on the current
        stream: host_out = H host_in for the captured buffers."""
        if self._pipeline is None:
            raise RuntimeError("capture() the pipeline first")
        self._pipeline[0].replay()


# ---------------------------------------------------------------------------
# Davidson


def _hermitize(a: torch.Tensor) -> torch.Tensor:
    return 0.5 * (a + a.conj().T)


def lowest_generalized_eigh(h: torch.Tensor, s: torch.Tensor, roots: int):
    """Lowest ``roots`` pairs of H x = e S x in FP64 on the device.

    Cholesky S = L L^H, reduced L^-1 H L^-H, Hermitian eigensolve, back
    transform (the transformation of LAPACK zhegv; reference fallback
    qepy_pw/diagonalization.py:83-110), on the current stream
    (eigensolver.ReducedSolve).  A subspace built from FP32 vectors can make
    S numerically indefinite; the solve then falls back to the
    well-conditioned part of its range (canonical orthogonalisation).
    """
    solve = ReducedSolve(torch.cuda.current_stream(h.device))
    solve.launch(h, s, roots)
    return solve.result()


class _Overlap:
    """What a Davidson generator with ``overlap_solves`` yields after it has
    enqueued its reduced eigensolve on its own stream: the driver may resume
    the other problems (which then enqueue theirs) before this one, whose
    next step reads the eigenvalues back to the host."""

    __slots__ = ()

    def __repr__(self) -> str:
        return "OVERLAP"


OVERLAP = _Overlap()


def _canonical_generalized_eigh(h: torch.Tensor, s: torch.Tensor, roots: int,
                                threshold: float = 1.0e-10):
    """H x = e S x restricted to eigenvectors of S above threshold * max(s):
    X = U s^-1/2, eigh(X^H H X) = Z, x = X Z."""
    values, vectors = torch.linalg.eigh(_hermitize(s))
    keep = values > threshold * values.max()
    if int(keep.sum()) < roots:
        raise np.linalg.LinAlgError("overlap matrix has fewer independent directions than roots")
    x = vectors[:, keep] / torch.sqrt(values[keep])[None, :]
    reduced = _hermitize(x.conj().T @ h @ x)
    e, z = torch.linalg.eigh(reduced)
    return e[:roots], (x @ z)[:, :roots]


def _orthonormalize(block: torch.Tensor, threshold: float = 1.0e-12) -> torch.Tensor:
    """Rank-revealing orthonormal basis of the block's span (:370-472, serial)."""
    if block.shape[1] == 0:
        return block
    wide = block.to(torch.complex128)
    if block.shape[1] == 1:
        norm = float(torch.linalg.vector_norm(wide))
        if norm == 0.0:
            return block[:, :0]
        return (wide / norm).to(block.dtype)
    gram = _hermitize(K.gemm(K.OP_C, wide, wide))
    squared, rotation = torch.linalg.eigh(gram)
    order = torch.argsort(squared, descending=True)
    squared = torch.clamp(squared[order].real, min=0.0)
    if squared.numel() == 0 or float(squared[0]) == 0.0:
        return block[:, :0]
    rank = int(torch.count_nonzero(squared > threshold ** 2 * squared[0]))
    transform = rotation[:, order[:rank]] / torch.sqrt(squared[:rank])[None, :]
    result = K.gemm(K.OP_N, wide, transform.T.contiguous().T)
    return result.to(block.dtype) if block.dtype != torch.complex128 else result


def davidson(operator, diagonal, number_of_roots: int, *, initial_vectors=None,
             tolerance: float = 1.0e-8, max_iterations: int = 40, subspace_multiplier: int = 4,
             residual_factor: float | None = 10.0, residual_energy_scale: float | None = None,
             occupied_roots: int | None = None, initial_is_ritz: bool = False,
             initial_is_orthonormal: bool = False, initial_eigenvalues=None,
             initial_applied=None, mpi=None, global_dimension: int | None = None,
             global_row_indices=None, timers=None, operator_into=None,
             dtype: torch.dtype | None = None, lock_converged: bool = False) -> DavidsonResult:
    """Lowest eigenpairs by restarted block Davidson (diagonalization.py:527-880).

    ``operator(C)`` / ``operator_into(C, out)`` act on column-major device
    tensors.  ``dtype`` selects the basis precision (default complex128, or
    the dtype of ``initial_vectors`` when it is a tensor).
    """
    steps = davidson_steps(diagonal, number_of_roots, initial_vectors=initial_vectors,
                           tolerance=tolerance, max_iterations=max_iterations,
                           subspace_multiplier=subspace_multiplier,
                           residual_factor=residual_factor,
                           residual_energy_scale=residual_energy_scale,
                           occupied_roots=occupied_roots, initial_is_ritz=initial_is_ritz,
                           initial_is_orthonormal=initial_is_orthonormal,
                           initial_eigenvalues=initial_eigenvalues,
                           initial_applied=initial_applied, global_dimension=global_dimension,
                           global_row_indices=global_row_indices, timers=timers, dtype=dtype,
                           lock_converged=lock_converged)

    def apply_into(vectors, destination):
        if operator_into is not None:
            operator_into(vectors, destination)
        else:
            destination[...] = operator(vectors)

    try:
        request = next(steps)
        while True:
            if request is not OVERLAP:
                apply_into(*request)
            request = steps.send(None)
    except StopIteration as done:
        return done.value


def apply_hamiltonians(hamiltonians, requests, scratch_pool: FFTScratchPool | None = None,
                       potential: torch.Tensor | None = None, always_batched: bool = False) -> None:
    """destination = H_index vectors for every (index, vectors, destination)
    request: the local parts of all k points in one launch per FFT pass
    (basis.apply_local_multi, stick scratch from ``scratch_pool``, the
    native potential ``potential`` or the first Hamiltonian's), then each
    k point's projector products.  A single request goes through the
    Hamiltonian's own apply unless ``always_batched`` (which a captured
    graph needs: the batched path alone uses the given scratch and
    potential, and nothing in it synchronises or times launches)."""
    if not requests:
        return
    hams = [hamiltonians[index] for index, _, _ in requests]
    first = hams[0]
    batched = (len(requests) > 1 or always_batched) and all(
        h.local_workspace.precision == first.local_workspace.precision and
        h.local_workspace.shape == first.local_workspace.shape and
        h.dtype == first.dtype for h in hams)
    if not batched:
        for (_, vectors, destination), ham in zip(requests, hams):
            ham.apply_into(vectors, destination)
        return
    vectors = [to_device_f(v, first.dtype, first.device) for _, v, _ in requests]
    with _timer(first.timers, "h_psi"):
        with _timer(first.timers, "vloc_psi"):
            apply_local_multi([h.local_workspace for h in hams],
                              first._potential if potential is None else potential, vectors,
                              [h._kinetic_kernel for h in hams],
                              [destination for _, _, destination in requests],
                              scratch_pool=scratch_pool)
        for v, (_, _, destination), ham in zip(vectors, requests, hams):
            ham.add_nonlocal(v, destination)


class RoundGraphs:
    """The H applications of lockstep Davidson rounds as CUDA graphs.

    A round applies each k point's Hamiltonian to its pending block of
    vectors (``apply_hamiltonians``: one launch per FFT pass for all k
    points, then each k point's projector GEMMs).  The graph of a round is
    keyed by every requesting k point's block width rounded up to a bucket
    (16 up to 16 columns, else a multiple of ``bucket``), so that a few
    graphs cover all the rounds of an SCF.  A new key runs eagerly once
    (its results serve the round) and is then captured; later rounds with
    that key replay it.  Inputs and outputs live in per-k static buffers of
    the largest width (``max_width``), the local potential in a static
    buffer that ``set_potential`` refreshes each SCF iteration (the kinetic
    terms and projectors of the k points do not change).  Padded columns
    carry stale values whose results are discarded: every operation acts on
    each column on its own.  Scratch is private and sized for
    ``max_width`` before the first capture, so that no captured graph ever
    sees its scratch reallocated: the stick scratch in its own pool, the
    split-K partial tiles as the scratch of the graphs' own stream."""

    def __init__(self, hamiltonians, max_width: int, bucket: int = 32, max_graphs: int = 48):
        from . import _lib

        self.hams = list(hamiltonians)
        if any(h.timers is not None for h in self.hams):
            raise ValueError("timed Hamiltonians synchronise and cannot be captured")
        self.bucket = int(bucket)
        self.max_width = -(-int(max_width) // self.bucket) * self.bucket
        self.max_graphs = int(max_graphs)
        first = self.hams[0]
        self.device = first.device
        self.stream = torch.cuda.Stream(device=self.device)
        self.pool = FFTScratchPool()
        self.potential = first._potential.clone()
        self.inputs = [zeros_f(len(h.basis), self.max_width, h.dtype, self.device)
                       for h in self.hams]
        self.outputs = [zeros_f(len(h.basis), self.max_width, h.dtype, self.device)
                        for h in self.hams]
        self.graphs: dict = {}
        self.captures = self.replays = self.eager = 0
        lib = _lib.load()
        import ctypes

        for start in range(0, len(self.hams), 16):
            part = self.hams[start:start + 16]
            plans = (ctypes.c_void_p * len(part))(*[h.local_workspace._plan.value for h in part])
            bands = (ctypes.c_int64 * len(part))(*([self.max_width] * len(part)))
            need = int(lib.qeb_local_multi_scratch_bytes(len(part), plans, bands))
            self.pool.buffer("sticks", max(need, 256), self.device)
        need = 0
        for h in self.hams:
            p = h.projectors.beta.shape[1] if h.projectors.beta is not None else 0
            npw = len(h.basis)
            for width in [16] + list(range(self.bucket, self.max_width + 1, self.bucket)):
                if p == 0:
                    continue
                if h.dtype == torch.complex64:
                    need = max(need, int(lib.qeb_cgemm_tf32x3_scratch_bytes(K.OP_C, p, width, npw)),
                               int(lib.qeb_cgemm_tf32x3_scratch_bytes(K.OP_N, npw, width, p)))
                prec = _lib.QEB_F32 if h.dtype == torch.complex64 else _lib.QEB_F64
                need = max(need, int(lib.qeb_zgemm_scratch_bytes(K.OP_C, p, width, npw, prec)))
        with torch.cuda.stream(self.stream):
            if need > 0:
                K._SCRATCH.get(need, self.device)

    def set_potential(self, potential: torch.Tensor) -> None:
        """The local potential of the current SCF iteration (native layout,
        the Hamiltonians' precision)."""
        self.potential.copy_(potential)

    def width(self, n: int) -> int:
        if n <= 16:
            return 16
        return min(self.max_width, -(-n // self.bucket) * self.bucket)

    def _requests(self, key):
        return [(i, self.inputs[i][:, :w], self.outputs[i][:, :w]) for i, w in key]

    def _apply(self, key) -> None:
        apply_hamiltonians(self.hams, self._requests(key), scratch_pool=self.pool,
                           potential=self.potential, always_batched=True)

    def run_key(self, key) -> None:
        """H of the static inputs of ``key`` into the static outputs: the
        graph's replay, or for a new key an eager run and then its capture."""
        current = torch.cuda.current_stream(self.device)
        self.stream.wait_stream(current)
        graph = self.graphs.get(key)
        with torch.cuda.stream(self.stream):
            if graph is not None:
                graph.replay()
                self.replays += 1
            else:
                self._apply(key)
                self.eager += 1
        current.wait_stream(self.stream)
        if graph is None and len(self.graphs) < self.max_graphs:
            torch.cuda.synchronize(self.device)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=self.stream):
                self._apply(key)
            torch.cuda.synchronize(self.device)
            self.graphs[key] = graph
            self.captures += 1

    def __call__(self, requests) -> None:
        """destination = H_index vectors for every (index, vectors,
        destination) request, as ``apply_hamiltonians`` computes it."""
        if any(v.shape[1] > self.max_width or v.dtype != self.hams[i].dtype
               for i, v, _ in requests):
            raise ValueError("a request exceeds the graphs' width or precision")
        key = tuple(sorted((index, self.width(v.shape[1])) for index, v, _ in requests))
        for index, vectors, _ in requests:
            self.inputs[index][:, :vectors.shape[1]].copy_(vectors)
        self.run_key(key)
        for index, vectors, destination in requests:
            destination.copy_(self.outputs[index][:, :vectors.shape[1]])


def run_lockstep(problems, apply_batch) -> list:
    """Drive several ``davidson_steps`` generators together: every round
    collects each unfinished problem's pending H application and hands them
    to ``apply_batch([(index, vectors, destination), ...])`` at once (the
    chosen form's batching of all k points into one launch per FFT pass).
    A problem that yields OVERLAP (its reduced eigensolve enqueued on its own
    stream) is resumed after the others have advanced to their next request
    or OVERLAP, so the k points' eigensolves run side by side on the GPU.
    Each problem runs the same operations as alone; returns the results in
    order."""
    results = [None] * len(problems)

    def advance(indices, first: bool) -> dict:
        """Resume ``indices`` until each has an H request or has finished."""
        requests = {}
        waiting = list(indices)
        while waiting:
            again = []
            for index in waiting:
                try:
                    request = next(problems[index]) if first else problems[index].send(None)
                except StopIteration as done:
                    results[index] = done.value
                    continue
                if request is OVERLAP:
                    again.append(index)
                else:
                    requests[index] = request
            waiting, first = again, False
        return requests

    pending = advance(range(len(problems)), True)
    while pending:
        apply_batch([(index, vectors, destination)
                     for index, (vectors, destination) in pending.items()])
        pending = advance(list(pending), False)
    return results


def davidson_steps(diagonal, number_of_roots: int, *, initial_vectors=None,
                   tolerance: float = 1.0e-8, max_iterations: int = 40,
                   subspace_multiplier: int = 4, residual_factor: float | None = 10.0,
                   residual_energy_scale: float | None = None, occupied_roots: int | None = None,
                   initial_is_ritz: bool = False, initial_is_orthonormal: bool = False,
                   initial_eigenvalues=None, initial_applied=None,
                   global_dimension: int | None = None, global_row_indices=None, timers=None,
                   dtype: torch.dtype | None = None, lock_converged: bool = False,
                   overlap_solves: bool = False):
    """The Davidson algorithm of ``davidson`` as a generator: it yields
    ``(vectors, destination)`` whenever it needs destination = H vectors and
    returns the DavidsonResult (StopIteration.value).  With
    ``overlap_solves`` it runs its reduced eigensolves on a stream of its own
    and yields OVERLAP between enqueuing one and reading its eigenvalues
    (``run_lockstep`` overlaps the k points' solves).

    ``lock_converged`` (chosen form; the reference never locks): at each
    restart the roots already converged leave the reduced problem.  Their
    Ritz vectors are kept aside, later corrections are projected out of
    their span, and the restarted subspace holds only the unconverged roots,
    so the FP64 reduced eigensolve of the following iterations has the size
    of the unconverged set instead of all roots.  Results differ from the
    unlocked solve below the convergence threshold of the locked roots."""
    device = require_cuda()
    diag = to_device_f(diagonal, torch.float64, device).reshape(-1)
    local_dimension = diag.numel()
    dimension = int(global_dimension) if global_dimension is not None else local_dimension
    if not 1 <= number_of_roots <= dimension:
        raise ValueError("number_of_roots must be between 1 and the matrix size")
    if tolerance <= 0.0:
        raise ValueError("Davidson tolerance must be positive")
    if max_iterations < 1:
        raise ValueError("Davidson max_iterations must be at least 1")
    if subspace_multiplier < 2:
        raise ValueError("diago_david_ndim must be at least 2")
    if residual_factor is not None and residual_factor <= 0.0:
        raise ValueError("Davidson residual_factor must be positive or None")
    if residual_energy_scale is not None and residual_energy_scale <= 0.0:
        raise ValueError("Davidson residual_energy_scale must be positive or None")
    if occupied_roots is None:
        occupied_roots = number_of_roots
    if not 0 <= occupied_roots <= number_of_roots:
        raise ValueError("occupied_roots must be between zero and number_of_roots")
    root_tolerances = np.full(number_of_roots, max(5.0 * tolerance, 5.0e-6))
    root_tolerances[:occupied_roots] = tolerance
    if dtype is None:
        dtype = initial_vectors.dtype if isinstance(initial_vectors, torch.Tensor) and \
            initial_vectors.is_complex() else torch.complex128

    if initial_vectors is None:
        rows = np.arange(local_dimension) if global_row_indices is None else \
            np.asarray(global_row_indices, dtype=int)
        trial_host = np.zeros((local_dimension, number_of_roots), dtype=np.complex128, order="F")
        for column in range(number_of_roots):
            matches = np.flatnonzero(rows == column)
            if len(matches):
                trial_host[matches[0], column] = 1.0
        trial = to_device_f(trial_host, dtype, device)
    else:
        trial = to_device_f(initial_vectors, dtype, device)
        if trial.dim() != 2 or trial.shape[0] != local_dimension or trial.shape[1] < number_of_roots:
            raise ValueError("initial_vectors must have shape (matrix size, at least number_of_roots)")

    if initial_is_ritz or initial_is_orthonormal:
        basis0 = trial[:, :number_of_roots]
    else:
        with _timer(timers, "cegterg:over"):
            basis0 = _orthonormalize(trial)
    if basis0.shape[1] < number_of_roots:
        raise ValueError("initial Davidson vectors are linearly dependent")
    maximum_subspace = min(dimension, max(basis0.shape[1], 2 * number_of_roots,
                                          subspace_multiplier * number_of_roots))
    active = basis0.shape[1]
    basis_storage = empty_f(local_dimension, maximum_subspace, dtype, device)
    applied_storage = empty_f(local_dimension, maximum_subspace, dtype, device)
    basis_storage[:, :active] = basis0
    del basis0, trial

    if initial_applied is None:
        yield basis_storage[:, :active], applied_storage[:, :active]
        applications = active
    else:
        supplied = to_device_f(initial_applied, dtype, device)
        if tuple(supplied.shape) != (local_dimension, active):
            raise ValueError("initial_applied must match the initial Ritz block")
        applied_storage[:, :active] = supplied
        applications = 0
    projected = torch.zeros((maximum_subspace, maximum_subspace), dtype=torch.complex128, device=device)
    overlap = torch.zeros_like(projected)

    def update_projected(first_new: int) -> None:
        """New rows/columns of V^H H V and V^H V (:658-695)."""
        with _timer(timers, "cegterg:over"):
            new = basis_storage[:, first_new:active]
            h_rows = K.gemm(K.OP_C, new, applied_storage[:, :active]).to(torch.complex128)
            s_rows = K.gemm(K.OP_C, new, basis_storage[:, :active]).to(torch.complex128)
            projected[first_new:active, :active] = h_rows
            overlap[first_new:active, :active] = s_rows
            if first_new:
                projected[:first_new, first_new:active] = h_rows[:, :first_new].conj().T
                overlap[:first_new, first_new:active] = s_rows[:, :first_new].conj().T
            block = slice(first_new, active)
            projected[block, block] = _hermitize(projected[block, block])
            overlap[block, block] = _hermitize(overlap[block, block])

    nroot = number_of_roots  # roots of the reduced problem (fewer once some are locked)
    root_ids = np.arange(number_of_roots)  # their indices among all roots
    locked = {"vectors": None, "count": 0, "values": [], "ids": [], "norms": []}

    solver = _solver(device, overlap_solves)

    def ritz_values():
        """Lowest roots and coefficients of the reduced problem (:699-708)."""
        with _timer(timers, "cdiaghg"):
            solver.launch(projected[:active, :active], overlap[:active, :active], nroot)
        if overlap_solves:
            yield OVERLAP
        with _timer(timers, "cdiaghg"):
            roots, coefficients = solver.result()
        return roots.cpu().numpy(), roots, coefficients

    def ritz_columns(coefficients, roots, columns=None):
        """Ritz vectors V c and residuals HV c - e V c (:709-724) of the
        selected roots (all when ``columns`` is None)."""
        with _timer(timers, "cegterg:upda"):
            if columns is not None:
                coefficients = coefficients.index_select(1, columns)
                roots = roots.index_select(0, columns)
            coeff = empty_f(coefficients.shape[0], coefficients.shape[1], dtype, device)
            coeff.copy_(coefficients)
            vectors = K.gemm(K.OP_N, basis_storage[:, :active], coeff)
            residual = K.gemm(K.OP_N, applied_storage[:, :active], coeff)
            K.subtract_band_energies(residual, vectors, roots)
        return vectors, residual

    # The reference forms all Ritz vectors and residuals after every reduced
    # solve.  Only the residuals of the roots still unconverged feed the next
    # correction block, so those are formed each iteration and the full Ritz
    # block only where it is consumed (restart, return, residual-norm
    # tracking); the values are the same columns of the same products.
    update_projected(0)
    coefficients = None
    if initial_is_ritz:
        if initial_eigenvalues is None:
            values_dev = K.column_inner_products(
                basis_storage[:, :number_of_roots], applied_storage[:, :number_of_roots]).real
        else:
            values_dev = torch.as_tensor(np.asarray(initial_eigenvalues[:number_of_roots], dtype=float),
                                         device=device)
        values = values_dev.cpu().numpy()
        ritz_vectors = basis_storage[:, :number_of_roots].clone()
        residuals = applied_storage[:, :number_of_roots].clone()
        K.subtract_band_energies(residuals, ritz_vectors, values_dev)
    else:
        values, values_dev, coefficients = yield from ritz_values()
        ritz_vectors, residuals = ritz_columns(coefficients, values_dev)
    track = residual_factor is not None or residual_energy_scale is not None

    def residual_norms_of(block):
        return np.sqrt(np.maximum(K.column_squared_norms(block).cpu().numpy(), 0.0))

    def full_ritz():
        """(vectors, residuals) of every root for the current state."""
        if coefficients is None:  # still the initial Ritz block
            return ritz_vectors, residuals
        return ritz_columns(coefficients, values_dev)

    residual_norms = residual_norms_of(residuals) if track else np.empty(number_of_roots)
    completed = 0
    unconverged_count = number_of_roots
    unconverged = np.ones(number_of_roots, dtype=bool)
    # residual columns of the unconverged roots, in root order
    block, energies = residuals, values_dev

    for iteration in range(1, max_iterations + 1):
        completed = iteration
        previous = values
        with _timer(timers, "g_psi"):
            corrections = K.precondition(block, energies, diag)
        if locked["count"]:
            span = locked["vectors"][:, :locked["count"]]
            for _ in range(2):  # classical Gram-Schmidt, repeated once
                K.gemm(K.OP_N, span, K.gemm(K.OP_C, span, corrections), corrections,
                       alpha=-1.0, beta=1.0)
        # Normalise (cegterg), dropping columns below 1e-14 of the largest norm (:500-524).
        norms2 = K.column_squared_norms(corrections)
        norms_host = norms2.cpu().numpy()
        if not len(norms_host):
            break
        scale = max(float(np.max(norms_host)), 1.0e-300)
        keep = np.flatnonzero(norms_host > (1.0e-14 ** 2) * scale)
        if keep.size == 0:
            break
        old = active
        active += keep.size
        selected = torch.as_tensor(keep.astype(np.int64), device=device)
        K.normalize_columns(corrections, norms2, selected, basis_storage[:, old:active])
        del ritz_vectors, residuals, corrections, block
        yield basis_storage[:, old:active], applied_storage[:, old:active]
        applications += keep.size
        update_projected(old)
        values, values_dev, coefficients = yield from ritz_values()
        ritz_vectors = residuals = None
        if track:
            ritz_vectors, residuals = full_ritz()
            residual_norms = residual_norms_of(residuals)
        tolerances = root_tolerances[root_ids]
        converged = np.abs(values - previous) < tolerances
        if residual_factor is not None:
            converged &= residual_norms < residual_factor * tolerances
        if residual_energy_scale is not None:
            converged &= residual_norms ** 2 < residual_energy_scale * tolerances
        unconverged = ~converged
        unconverged_count = int(np.count_nonzero(unconverged))
        if unconverged_count == 0:
            if residuals is None:
                ritz_vectors, residuals = full_ritz()
            if not track:
                residual_norms = residual_norms_of(residuals)
            return DavidsonResult(*_with_locked(locked, root_ids, values, ritz_vectors,
                                                residual_norms),
                                  iteration, True, 0, applications)
        index = torch.as_tensor(np.flatnonzero(unconverged), device=device)
        lockable = None
        if lock_converged and active + unconverged_count > maximum_subspace:
            # Roots that may leave the reduced problem: converged, occupied
            # (tight threshold) and with |r|^2 below that threshold, so the
            # eigenvalue error of the frozen vector is below it as well.
            if residuals is None:
                ritz_vectors, residuals = full_ritz()
            norms_now = residual_norms if track else residual_norms_of(residuals)
            lockable = converged & (root_ids < occupied_roots) & (norms_now ** 2 < tolerance)
            if not lockable.any():
                lockable = None
        if lockable is not None:
            # Lock them and restart on the Ritz block of the others.
            with _timer(timers, "cegterg:last"):
                keep_roots = ~lockable
                done = torch.as_tensor(np.flatnonzero(lockable), device=device)
                rest = torch.as_tensor(np.flatnonzero(keep_roots), device=device)
                count = done.numel()
                if locked["vectors"] is None:
                    locked["vectors"] = empty_f(local_dimension, number_of_roots, dtype, device)
                first = locked["count"]
                locked["vectors"][:, first:first + count] = _select_columns(ritz_vectors, done)
                locked["count"] = first + count
                locked["values"].extend(values[lockable].tolist())
                locked["ids"].extend(root_ids[lockable].tolist())
                locked["norms"].extend(np.asarray(norms_now[lockable]).tolist())
                nroot = int(np.count_nonzero(keep_roots))
                root_ids = root_ids[keep_roots]
                values = values[keep_roots]
                values_dev = values_dev.index_select(0, rest)
                if track:
                    residual_norms = residual_norms[keep_roots]
                ritz_vectors = _select_columns(ritz_vectors, rest)
                residuals = _select_columns(residuals, rest)
                active = nroot
                basis_storage[:, :active] = ritz_vectors
                applied_storage[:, :active] = residuals
                K.subtract_band_energies(applied_storage[:, :active], ritz_vectors, -values_dev)
                projected[:active, :active] = torch.diag(values_dev.to(torch.complex128))
                overlap[:active, :active] = torch.eye(active, dtype=torch.complex128, device=device)
                unconverged = unconverged[keep_roots]
                index = torch.as_tensor(np.flatnonzero(unconverged), device=device)
            coefficients = None
        elif active + unconverged_count > maximum_subspace:
            # Restart on the Ritz block without a new H application (:843-868).
            if residuals is None:
                ritz_vectors, residuals = full_ritz()
            with _timer(timers, "cegterg:last"):
                active = nroot
                basis_storage[:, :active] = ritz_vectors
                # H psi = residual + e psi, rebuilt in place (:855-860).
                applied_storage[:, :active] = residuals
                K.subtract_band_energies(applied_storage[:, :active], ritz_vectors, -values_dev)
                projected[:active, :active] = torch.diag(values_dev.to(torch.complex128))
                overlap[:active, :active] = torch.eye(active, dtype=torch.complex128, device=device)
            coefficients = None  # the Ritz block is the basis itself now
        if residuals is not None:
            if unconverged.all():
                block = residuals
            else:
                block = residuals.index_select(1, index).T.contiguous().T
        else:
            _, block = ritz_columns(coefficients, values_dev, index)
        energies = values_dev.index_select(0, index)
    if residuals is None:
        ritz_vectors, residuals = full_ritz()
    if not track:
        residual_norms = residual_norms_of(residuals)
    return DavidsonResult(*_with_locked(locked, root_ids, values, ritz_vectors, residual_norms),
                          completed, False, unconverged_count, applications)


# Budget (Ha) of the FP32 rounding that the refined Davidson lets its
# carried residual R accumulate (over restarts and SCF iterations) before it
# redoes the FP64 Rayleigh-Ritz step (refined_davidson_steps ``budget``).
REFINED_ERROR_BUDGET = 1.0e-8
# relative rounding of an FP32 product-sum (a few units of 2^-24 for the
# accumulation depths of the residual products)
_FP32_ROUNDING = 2.4e-7


def refined_davidson_steps(diagonal, number_of_roots: int, *, initial_vectors,
                           tolerance: float = 1.0e-8, max_iterations: int = 20,
                           subspace_multiplier: int = 2, occupied_roots: int | None = None,
                           timers=None, initial_state=None, state_out: dict | None = None,
                           budget: float | None = None, overlap_solves: bool = False):
    """Chosen-form Davidson: an FP64 block of vectors with FP32 corrections.

    A generator like ``davidson_steps``; it yields ``(vectors, destination)``
    for destination = H vectors, with complex128 vectors when it needs the
    FP64 Hamiltonian (only to start without ``initial_state``) and complex64
    vectors for the chosen form's (FP32 FFT passes, split-TF32 projector
    GEMMs).  Same criteria as the reference's Davidson
    (qepy_pw/diagonalization.py:527-880): the lowest roots of the reduced
    problem, converged when |e - e_previous| is below the root's threshold
    (occupied roots ``tolerance``, the others max(5 tol, 5e-6)), restart when
    the subspace is full; returns a DavidsonResult with complex128
    eigenvectors.

    How FP64 accuracy comes out of FP32 work.  The block X (complex128,
    near orthonormal) comes with values lam and R = H X - X lam, so that
    H X = X lam + R exactly.  R is small once X is near the eigenvectors
    and is kept in FP32.  The subspace is [X, D_1, D_2, ...] with FP32
    correction blocks D_j and their chosen-form products H D_j; the reduced
    matrices take
      * the X-X block as S lam + X^H R (the second term, small, from an
        FP32 product) and the overlap as S = X^H X (1 after an FP64
        Rayleigh-Ritz step, else an FP64 product: a block formed from the
        reduced solution is orthonormal only to the FP32 accuracy of the
        reduced overlap, and that drift would build up over restarts);
      * the D-X blocks as S_DX = D^H X32 and H_DX = S_DX lam + D^H R, both
        from the same FP32-accurate S_DX: an error in S_DX is an exact
        Rayleigh-Ritz step on [X, D + X dS^H], which spans the same space,
        so it does not reach the Ritz values;
      * the D-D blocks from FP32 products, whose errors enter the Ritz
        values through the squared correction coefficients only.
    Residuals of the roots, X (lam - e) c_X + R c_X + (H D_j - e D_j) c_j,
    are formed in FP32 from terms that shrink as the roots converge; at a
    restart and at the end the vectors X c_X + D c_D are formed with the X
    part in FP64 and R of the new block is that residual (with lam = e,
    H X = X lam + R holds for any X, orthonormal or not).  That R carries
    the FP32 rounding of the H D_j c_j terms, which enters the next X-X
    block x^H R at first order: about 2.4e-7 (sum_j |c_ji|^2 |H D_j|^2)^(1/2)
    / sqrt(npw) for root i, the rounding being independent of the unit
    vector it is projected on (measured: with no refresh at all the mixed
    SCF's eigenvalues on the 216-atom cell were within 4e-11 Ry of a plain
    FP64 Davidson on the same potential).  Its running total (carried with
    the state) may grow to
    ``budget`` Ha (default REFINED_ERROR_BUDGET, 1e-8); a restart that would
    exceed it redoes the FP64 Rayleigh-Ritz step below instead, and an end
    that would exceed it leaves no state to carry (the next solve starts
    with that step).  Near convergence the corrections are small, no FP64
    Hamiltonian application is needed after the start, and the FP64 work of
    a restart is two GEMMs (npw x n x n: X c_X and X^H X), of the end one.

    Start: ``initial_state = (lam, R, error)`` (an FP64 tensor of n
    values, a complex64 (npw, n) residual and the rounding accumulated in
    it so far, Ha) gives H X = X lam + R for ``initial_vectors`` X; the SCF
    carries it from the previous iteration's end, adding (V_new - V_old) X
    for the change of the local potential.  Without it the start is an
    FP64 Rayleigh-Ritz step: one FP64 H application of the block, X^H H X
    and X^H X in FP64, the FP64 reduced eigensolve and the rotation.
    ``state_out`` (a dict) receives the final ``lam``, ``residual`` (None
    when the budget is spent) and ``error``.  ``overlap_solves``: as in
    ``davidson_steps`` (OVERLAP yielded around the reduced eigensolves)."""
    device = require_cuda()
    if budget is None:
        budget = REFINED_ERROR_BUDGET
    diag = to_device_f(diagonal, torch.float64, device).reshape(-1)
    npw = diag.numel()
    n = int(number_of_roots)
    if not 1 <= n <= npw:
        raise ValueError("number_of_roots must be between 1 and the matrix size")
    if tolerance <= 0.0:
        raise ValueError("Davidson tolerance must be positive")
    if max_iterations < 1:
        raise ValueError("Davidson max_iterations must be at least 1")
    if subspace_multiplier < 2:
        raise ValueError("diago_david_ndim must be at least 2")
    if occupied_roots is None:
        occupied_roots = n
    if not 0 <= occupied_roots <= n:
        raise ValueError("occupied_roots must be between zero and number_of_roots")
    root_tolerances = np.full(n, max(5.0 * tolerance, 5.0e-6))
    root_tolerances[:occupied_roots] = tolerance
    trial = to_device_f(initial_vectors, torch.complex128, device)
    if trial.dim() != 2 or trial.shape[0] != npw or trial.shape[1] < n:
        raise ValueError("initial_vectors must have shape (matrix size, at least number_of_roots)")
    maximum_subspace = min(npw, max(2 * n, subspace_multiplier * n))
    if maximum_subspace <= n:
        raise ValueError("the subspace has no room for corrections")
    f32 = torch.complex64
    basis32 = empty_f(npw, maximum_subspace, f32, device)
    applied32 = empty_f(npw, maximum_subspace, f32, device)
    projected = torch.zeros((maximum_subspace, maximum_subspace), dtype=torch.complex128,
                            device=device)
    overlap = torch.zeros_like(projected)
    eye = torch.eye(n, dtype=torch.complex128, device=device)
    x = empty_f(npw, n, torch.complex128, device)
    x.copy_(trial[:, :n])
    del trial
    counts = {"applications": 0}

    solver = _solver(device, overlap_solves)

    def solve(h, s):
        """Lowest n pairs of the pencil (h, s); OVERLAP between enqueuing
        the solve and reading it when ``overlap_solves``."""
        with _timer(timers, "cdiaghg"):
            solver.launch(h, s, n)
        if overlap_solves:
            yield OVERLAP
        with _timer(timers, "cdiaghg"):
            return solver.result()

    def ritz_block(vectors):
        """FP64 Rayleigh-Ritz of ``vectors``: returns (X, lam, R) with X the
        Ritz vectors, lam their values and R = H X - X lam."""
        hx = empty_f(npw, n, torch.complex128, device)
        yield vectors, hx
        counts["applications"] += n
        with _timer(timers, "cegterg:over"):
            a = _hermitize(K.gemm(K.OP_C, vectors, hx))
            s = _hermitize(K.gemm(K.OP_C, vectors, vectors))
        lam, rot = yield from solve(a, s)
        with _timer(timers, "cegterg:upda"):
            rot = rot.T.contiguous().T
            ritz = K.gemm(K.OP_N, vectors, rot)
            residual = K.gemm(K.OP_N, hx, rot)
            K.subtract_band_energies(residual, ritz, lam)
        return ritz, lam, residual

    def start_block(lam, residual, exact: bool = False) -> None:
        """X block of the basis: X32, R, and the X-X blocks of the reduced
        matrices, S lam + X^H R and S = X^H X.  S is the identity after an
        FP64 Rayleigh-Ritz step (``exact``); a block formed as X c_X + D c_D
        is orthonormal only to the FP32 accuracy of the reduced overlap, a
        drift that would build up over restarts, so S is then an FP64
        product."""
        basis32[:, :n].copy_(x)
        applied32[:, :n].copy_(residual)
        lam_c = lam.to(torch.complex128)
        with _timer(timers, "cegterg:over"):
            xr = K.gemm(K.OP_C, basis32[:, :n], applied32[:, :n]).to(torch.complex128)
            gram = eye if exact else _hermitize(K.gemm(K.OP_C, x, x))
        projected[:n, :n] = _hermitize(xr + gram * lam_c[None, :])
        overlap[:n, :n] = gram

    def update_projected(first_new: int, active: int, lam_dev) -> None:
        with _timer(timers, "cegterg:over"):
            new = basis32[:, first_new:active]
            h_rows = K.gemm(K.OP_C, new, applied32[:, :active]).to(torch.complex128)
            s_rows = K.gemm(K.OP_C, new, basis32[:, :active]).to(torch.complex128)
            h_rows[:, :n] += s_rows[:, :n] * lam_dev.to(torch.complex128)[None, :]
            projected[first_new:active, :active] = h_rows
            overlap[first_new:active, :active] = s_rows
            projected[:first_new, first_new:active] = h_rows[:, :first_new].conj().T
            overlap[:first_new, first_new:active] = s_rows[:, :first_new].conj().T
            block = slice(first_new, active)
            projected[block, block] = _hermitize(projected[block, block])
            overlap[block, block] = _hermitize(overlap[block, block])

    def composite_residuals(coefficients, roots, lam_dev, active):
        """FP32 residuals H V c - e V c of the selected roots."""
        with _timer(timers, "cegterg:upda"):
            shift = torch.empty_like(coefficients)
            shift[:n] = coefficients[:n] * (lam_dev[:, None] - roots[None, :])
            shift[n:] = -coefficients[n:] * roots[None, :]
            left = empty_f(active, coefficients.shape[1], f32, device)
            left.copy_(shift)
            right = empty_f(active, coefficients.shape[1], f32, device)
            right.copy_(coefficients)
            out = K.gemm(K.OP_N, basis32[:, :active], left)
            K.gemm(K.OP_N, applied32[:, :active], right, out, beta=1.0)
        return out

    def vectors_of(coefficients, active):
        """X c_X (FP64) + D c_D (FP32) of every root."""
        with _timer(timers, "cegterg:last"):
            out = K.gemm(K.OP_N, x, coefficients[:n].T.contiguous().T)
            if active > n:
                low = empty_f(active - n, coefficients.shape[1], f32, device)
                low.copy_(coefficients[n:active])
                out += K.gemm(K.OP_N, basis32[:, n:active], low).to(torch.complex128)
        return out

    hd_norms = torch.zeros(maximum_subspace, dtype=torch.float64, device=device)

    def rounding(coefficients, active) -> float:
        """Estimate of what the FP32 rounding of the H D c_D terms of the
        roots' residuals adds to an entry x^H R of the next X-X block:
        2.4e-7 max_i (sum_j |c_ji|^2 |H D_j|^2)^(1/2) / sqrt(npw) (the
        rounding errors of the terms independent of one another and of the
        unit vectors x they are projected on)."""
        if active <= n:
            return 0.0
        weights = coefficients[n:active].abs() * hd_norms[n:active, None]
        return _FP32_ROUNDING * float(torch.linalg.vector_norm(weights, dim=0).max()) / \
            float(np.sqrt(npw))

    def reduced_solve(active):
        return (yield from solve(projected[:active, :active], overlap[:active, :active]))

    error = 0.0  # rounding accumulated in the carried residual (Ha)
    exact = initial_state is None
    if initial_state is None:
        x, lam_dev, r = yield from ritz_block(x)
    else:
        lam_dev = torch.as_tensor(initial_state[0], dtype=torch.float64, device=device)
        r = initial_state[1]
        error = float(initial_state[2]) if len(initial_state) > 2 else 0.0
        if tuple(r.shape) != (npw, n) or lam_dev.numel() != n:
            raise ValueError("initial_state does not match the initial block")
    start_block(lam_dev, r, exact)
    del r
    active = n
    # Ritz values and residuals of the starting block (the reference's first
    # reduced solve, :699-724)
    values_dev, coefficients = yield from reduced_solve(active)
    values = values_dev.cpu().numpy()
    block = composite_residuals(coefficients, values_dev, lam_dev, active)
    energies = values_dev
    unconverged = np.ones(n, dtype=bool)
    completed = 0
    for iteration in range(1, max_iterations + 1):
        completed = iteration
        previous = values
        with _timer(timers, "g_psi"):
            corrections = K.precondition(block, energies, diag)
        norms2 = K.column_squared_norms(corrections)
        norms_host = norms2.cpu().numpy()
        scale = max(float(np.max(norms_host)), 1.0e-300) if len(norms_host) else 0.0
        keep = np.flatnonzero(norms_host > (1.0e-14 ** 2) * scale) if scale else np.empty(0, int)
        if keep.size == 0:
            break
        if active + keep.size > maximum_subspace:
            # restart on the current Ritz vectors (:843-868): X c_X + D c_D
            # in FP64 for the X part, R the FP32 residual of every root, or
            # a fresh FP64 Rayleigh-Ritz step while corrections are large
            x_new = vectors_of(coefficients, active)
            step = rounding(coefficients, active)
            exact = error + step > budget
            if exact:
                x, lam_dev, r = yield from ritz_block(x_new)
                error = 0.0
            else:
                r = composite_residuals(coefficients, values_dev, lam_dev, active)
                x, lam_dev = x_new, values_dev
                error += step
            start_block(lam_dev, r, exact)
            del r, x_new
            active = n
            coefficients = torch.eye(n, dtype=torch.complex128, device=device)
        old = active
        active += keep.size
        selected = torch.as_tensor(keep.astype(np.int64), device=device)
        K.normalize_columns(corrections, norms2, selected, basis32[:, old:active])
        del corrections, block
        yield basis32[:, old:active], applied32[:, old:active]
        counts["applications"] += keep.size
        hd_norms[old:active] = torch.sqrt(K.column_squared_norms(applied32[:, old:active]))
        update_projected(old, active, lam_dev)
        values_dev, coefficients = yield from reduced_solve(active)
        values = values_dev.cpu().numpy()
        converged = np.abs(values - previous) < root_tolerances
        unconverged = ~converged
        count = int(np.count_nonzero(unconverged))
        if count == 0:
            break
        index = torch.as_tensor(np.flatnonzero(unconverged), device=device)
        energies = values_dev.index_select(0, index)
        block = composite_residuals(coefficients.index_select(1, index), energies, lam_dev,
                                    active)
    vectors = vectors_of(coefficients, active)
    residual = composite_residuals(coefficients, values_dev, lam_dev, active)
    norms = np.sqrt(np.maximum(K.column_squared_norms(residual).cpu().numpy(), 0.0))
    if state_out is not None:
        error += rounding(coefficients, active)
        state_out["lam"] = values_dev
        state_out["residual"] = residual if error <= budget else None
        state_out["error"] = error
    count = int(np.count_nonzero(unconverged))
    return DavidsonResult(values, vectors, norms, completed, count == 0, count,
                          counts["applications"])


def _select_columns(matrix: torch.Tensor, index: torch.Tensor) -> torch.Tensor:
    """Columns ``index`` of a column-major matrix, column-major."""
    return matrix.T.index_select(0, index).T


def _with_locked(locked: dict, root_ids, values, vectors, norms):
    """(eigenvalues, eigenvectors, residual norms) of all roots: the locked
    ones and those of the reduced problem, in ascending eigenvalue order."""
    count = locked["count"]
    if not count:
        return values, vectors, norms
    all_values = np.concatenate([np.asarray(locked["values"]), np.asarray(values)])
    all_norms = np.concatenate([np.asarray(locked["norms"]), np.asarray(norms)])
    order = np.argsort(all_values, kind="stable")
    stacked = torch.cat([locked["vectors"][:, :count], vectors], dim=1)
    out = empty_f(stacked.shape[0], stacked.shape[1], stacked.dtype, stacked.device)
    out.copy_(_select_columns(stacked, torch.as_tensor(order, device=stacked.device)))
    return all_values[order], out, all_norms[order]
