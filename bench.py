"""Benchmark of the B200 Kohn-Sham H|psi> hot path (one JSON line on rank 0).

Workload (one "step"): one full H|psi> application
  H psi = T psi + FFT^-(V . FFT^+ psi) + beta D beta^H psi
on the H|psi> microbenchmark cell: cubic L = 15.8 bohr, 64^3 grid,
11 019 plane waves, 256 bands, 64 atoms x 8 projectors (P = 512); seeded
synthetic inputs (qe_python_b200/workloads.py).

  value      H|psi> bands/s of the mixed form (FP32 FFT passes and FP32
             projector GEMMs), inputs resident in HBM; L2 is flushed before
             every timed step (a 256 MiB write).
  fp64       the same for the plain FP64 form.
  e2e        bands/s through the public HostStreamedHpsi (the Hamiltonian
             applied to host-resident bands in chunks of 1/8, 3/8, 3/8 and
             1/8 of the bands, the pipeline captured once and replayed per
             step) with pinned host buffers: H2D of psi and D2H of H psi in
             the timed region.
  roofline   the dominant kernel's algorithmic bytes (FFT passes) or flops
             (GEMMs) per launch over its CUDA-event duration.
  cpu_baseline  the oracle (NumPy/SciPy restatement of the reference's
             serial apply_serial + ZGEMM projector path) on host cores.

Multi-GPU: the operator does not shard across GPUs in this tier, so N GPUs
run N independent replicas ("scaling": "weak"); value is the sum of bands
over the max-over-ranks time.

``--impl reference`` times the reference's own PlaneWaveHamiltonian.apply_into
(the staged reference package, its native module the oracle) on all host
threads, on the same workload, a bounded band sample per step; without the
staged package, the oracle's restatement of the same path.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "SCF time to 1e-8 Ry and H|psi> bands/s: mixed+batched vs FP64 plain, 1 B200"
WORKLOAD = ("H|psi> microbenchmark: cubic L=15.8 bohr, ecutwfc 30 Ry, 64^3 grid, "
            "11019 plane waves, 256 bands, 64 atoms x 8 projectors (P=512)")
L2_FLUSH_BYTES = 256 << 20
# host-streamed end-to-end leg: chunk sizes as fractions of the bands (small
# first and last chunks: the compute starts early and the last output copy is
# short; large middle ones keep the GEMM tiles full), compute streams.
# Measured on one box, 256 bands, interleaved medians: (32, 96, 96, 32) 0.892
# ms, (64, 128, 64) 0.903, 128-band chunks on two streams 0.952, 64-band
# chunks 1.001.
E2E_EIGHTHS, E2E_STREAMS = (1, 3, 3, 1), 1


def e2e_chunks(nbands: int) -> list[int]:
    """Chunk sizes of the end-to-end leg: E2E_EIGHTHS of nbands, the last
    taking the remainder."""
    eighth = nbands // 8
    if eighth == 0:
        return [nbands]
    sizes = [eighth * f for f in E2E_EIGHTHS[:-1]]
    return sizes + [nbands - sum(sizes)]


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--bands", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--apply-only", choices=("f32", "f64"), default=None,
                   help="profiling driver: build the workload, apply H|psi> --steps times "
                        "in the given precision, print a checksum, no timing")
    p.add_argument("--cpu-seconds", type=float, default=10.0,
                   help="approximate CPU time budget of the cpu_baseline sample")
    p.add_argument("--scf", default="scf-dia216,scf-dia64",
                   help="comma-separated benchmark cells whose SCF-to-1e-8 Ry times (plain "
                        "and mixed) are reported beside the H|psi> rate (scf-fcc2, "
                        "scf-fcc2-smear, scf-dia8-disp, scf-dia64, scf-dia216, or none); "
                        "run at N = 1 only")
    return p.parse_args()


# DRAM bytes (read + write) of one pass-B launch of the 256-band microbenchmark,
# from one ncu capture (--set full) of `bench.py --apply-only f32` (the pruned
# plane pass, two bands per block): 78.8 MB read + 22.0 MB written.
PASS_B_NCU_TRAFFIC = {("pass_b", 256): 100.83e6}


# How the SCF benchmark cells differ from the configurations they stand for:
# with the synthetic pseudopotential the diamond supercells are semimetals,
# which fixed filling and plain Broyden do not converge (qe_python_b200/configs.py).
SCF_CELL_CHANGES = {
    "scf-dia64": ["Gaussian smearing, degauss 0.02 Ry (configuration: fixed occupations)",
                  "Thomas-Fermi Broyden mixing (configuration: default plain Broyden)",
                  "unshifted 2x2x2 k mesh, 4 irreducible points (the shifted mesh reduces "
                  "to one point under the cubic group)"],
    "scf-dia216": ["Gaussian smearing, degauss 0.02 Ry (configuration: fixed occupations)",
                   "Thomas-Fermi Broyden mixing (configuration: default plain Broyden)"],
}


def scf_cell_config(name: str) -> dict:
    """The SCF cell's settings as run, with its changes from the named
    benchmark configuration."""
    from qe_python_b200.scf import benchmark_system

    system = benchmark_system(name)
    return {"atoms": len(system.positions), "ecutwfc_ry": system.ecutwfc,
            "ecutrho_ry": system.ecutrho, "nbnd": system.nbnd,
            "kpoints": int(len(system.kpoints)), "occupations": system.occupations,
            "smearing": system.smearing if system.occupations == "smearing" else None,
            "degauss_ry": system.degauss, "mixing_mode": system.mixing_mode,
            "mixing_beta": system.mixing_beta, "changes": SCF_CELL_CHANGES.get(name, [])}


def fixed_potential_error(name: str, result) -> float:
    """Max |e_mixed - e_FP64| (Ry) over the nbnd bands of every k point: a
    plain FP64 Davidson to 1e-10 Ha on the mixed SCF's last potential,
    started from its eigenvectors."""
    from qe_python_b200.basis import LocalPotentialWorkspace
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian, davidson
    from qe_python_b200.scf import benchmark_system, projector_terms, scf_setup

    system = benchmark_system(name)
    setup = scf_setup(system, result.potential.device)
    worst = 0.0
    for k, basis in enumerate(setup.bases):
        ws = LocalPotentialWorkspace(basis, setup.shape, precision="f64")
        ham = PlaneWaveHamiltonian(basis, None, projector_terms(system, setup.tables, basis),
                                   local_workspace=ws, real_potential=result.potential,
                                   potential_average=setup.v_ion_average)
        vectors = result.eigenvectors[k]
        check = davidson(ham.apply, ham.diagonal, vectors.shape[1], initial_vectors=vectors,
                         tolerance=1.0e-10, max_iterations=200,
                         subspace_multiplier=system.diago_david_ndim, residual_factor=None,
                         occupied_roots=system.nbnd, initial_is_orthonormal=True,
                         operator_into=ham.apply_into)
        diff = np.abs(np.asarray(check.eigenvalues)[:system.nbnd]
                      - np.asarray(result.eigenvalues_ha[k])[:system.nbnd])
        worst = max(worst, 2.0 * float(np.max(diff)))
    return worst


def scf_times(name: str) -> dict:
    """Wall time of the GPU SCF to conv_thr = 1e-8 Ry, plain FP64 and mixed,
    with the mixed form's energy, eigenvalue and force differences from the
    FP64 run.  A third run, FP64 with the mixed form's guard bands
    (``f64_guard_bands``), separates what the guard bands save from what the
    precision saves.

    Each SCF runs twice in this process and ``seconds`` is the second run:
    the first one (``first_run_seconds``) also pays the one-time costs of
    the process (module loads, library handles, the launch-shape timings of
    the autotuner for every new problem class)."""
    import torch

    from qe_python_b200.scf import MIXED_GUARD_BANDS, benchmark_system, run_scf

    out = {"cell": name, "conv_thr_ry": 1.0e-8, "config": scf_cell_config(name)}
    results = {}
    runs = (("f64", "f64", {}), ("mixed", "mixed", {}),
            ("f64_guard_bands", "f64", {"guard_bands": MIXED_GUARD_BANDS}))
    for label, precision, options in runs:
        walls = []
        for _ in range(2):
            system = benchmark_system(name)
            torch.cuda.synchronize()
            started = time.perf_counter()
            result = run_scf(system, precision=precision, **options)
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - started)
        results[label] = result
        out[label] = {
            "seconds": walls[-1],
            "first_run_seconds": walls[0],
            "inside_run_scf_seconds": result.wall_seconds,
            "converged": bool(result.converged),
            "iterations": result.iterations,
            "total_energy_ry": result.total_energy_ry,
            "precision_per_iteration": result.precision_log,
            "davidson_iterations": float(sum(result.davidson_iterations)),
            "phase_seconds": {k: round(v, 3) for k, v in result.timings.items()},
        }
    out["mixed_speedup"] = out["f64"]["seconds"] / out["mixed"]["seconds"]
    out["mixed_speedup_first_runs"] = (out["f64"]["first_run_seconds"]
                                       / out["mixed"]["first_run_seconds"])
    out["guard_bands"] = MIXED_GUARD_BANDS
    out["mixed_speedup_over_f64_guard_bands"] = (out["f64_guard_bands"]["seconds"]
                                                 / out["mixed"]["seconds"])
    out["energy_difference_ry"] = out["mixed"]["total_energy_ry"] - out["f64"]["total_energy_ry"]
    a, b = results["mixed"], results["f64"]
    out["max_eigenvalue_difference_ry"] = max(
        float(np.max(np.abs(2.0 * (np.asarray(x) - np.asarray(y)))))
        for x, y in zip(a.eigenvalues_ha, b.eigenvalues_ha))
    # the same difference between the two FP64 runs (no guard bands / with):
    # two converged SCFs along different mixing paths, no FP32 arithmetic
    out["max_eigenvalue_difference_f64_paths_ry"] = max(
        float(np.max(np.abs(2.0 * (np.asarray(x) - np.asarray(y)))))
        for x, y in zip(results["f64_guard_bands"].eigenvalues_ha, b.eigenvalues_ha))
    # the chosen form's arithmetic error alone: its eigenvalues against a
    # tight plain-FP64 Davidson on its own final potential
    out["max_eigenvalue_error_at_fixed_potential_ry"] = fixed_potential_error(name, a)
    if a.forces_ha_per_bohr is not None and b.forces_ha_per_bohr is not None:
        out["max_force_difference_ry_per_bohr"] = float(
            np.max(np.abs(2.0 * (a.forces_ha_per_bohr - b.forces_ha_per_bohr))))
    return out


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)

def init_distributed(backend: str):
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        from datetime import timedelta

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(value: float, world: int, device) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region

def smi_device_id(local: int) -> str:
    """The PCI bus id (domain:bus:device.function, hex) of torch device
    ``local``.  nvidia-smi numbers GPUs in its own (PCI) order and ignores
    CUDA_VISIBLE_DEVICES, so a torch index can name another GPU there; the
    bus id names the same physical device in both."""
    import torch

    props = torch.cuda.get_device_properties(local)
    return f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"


class ClockSampler:
    """SM clocks and slowdown reasons of one GPU around a timed region (read
    only), from ``nvidia-smi -lms 200``; ``device_id`` is what nvidia-smi's
    ``--id`` takes (the PCI bus id from ``smi_device_id``).  Entry waits (at most 3 s) until
    the sampler has printed its first line, so the samples of the region
    are not lost to its start-up; exit waits (at most 1 s) for one more
    line, so a region shorter than the 200 ms period still has the sample
    taken as it ends."""

    QUERY = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id) -> None:
        self.device_id = str(device_id)
        self.samples: list[list[str]] = []
        self._lines: list[list[str]] = []
        self._proc = None
        self._thread = None
        self._arrived = threading.Condition()

    def _wait_for(self, count: int, seconds: float) -> None:
        with self._arrived:
            self._arrived.wait_for(lambda: len(self._lines) >= count, timeout=seconds)

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_id}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=self._read, daemon=True)
            self._thread.start()
            self._wait_for(1, 3.0)
        except (OSError, ValueError):
            self._proc = None
        self._first = len(self._lines)
        return self

    def _read(self):
        for line in self._proc.stdout:
            with self._arrived:
                self._lines.append([v.strip() for v in line.split(",")])
                self._arrived.notify_all()

    def __exit__(self, *exc):
        if self._proc is not None:
            self._wait_for(len(self._lines) + 1, 1.0)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        # the samples from the last one before the region to the end
        self.samples = self._lines[max(0, self._first - 1):]
        return False

    def summary(self) -> dict:
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in self.samples:
            if len(row) < 6:
                continue
            try:
                sm.append(float(row[0]))
                smax.append(float(row[1]))
            except ValueError:
                continue
            for name, flag in zip(names, row[2:6]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def plane_fft_rate(shape, bands: int, seconds: float) -> dict:
    """Pass B's arithmetic rate by the usual FFT convention: 5 N log2 N flops
    per complex transform of a full nx x ny plane, two transforms (inverse
    and forward) and the real potential product (2 flops a point) for each
    (z plane, band), against the nominal FP32 FMA peak of the 148 SMs at
    1.965 GHz.  The kernel skips the x transforms of rows that hold no
    stick, so the convention counts more than it executes."""
    nx, ny, nz = (int(v) for v in shape)
    points = nx * ny
    per_plane = 2 * 5.0 * points * np.log2(points) + 2.0 * points
    achieved = float(per_plane * nz * bands / seconds / 1e12)
    peak = 148 * 128 * 2 * 1.965e9 / 1e12
    return {"achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "convention": "5 N log2 N per full-plane 2-D transform; nominal FP32 FMA peak"}


def measured_peaks() -> dict:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return {"hbm_gbs": float(data["hbm_gbs"]), "bf16_tflops": float(data["bf16_tflops"]),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# ---------------------------------------------------------------------------
# CPU side: the oracle (reference algorithm restated in NumPy/SciPy)

def cpu_hpsi_rate(work, bands: int, seconds: float, threads: int) -> dict:
    """Bands/s of the oracle H|psi> (apply_serial + projector ZGEMMs)."""
    from oracle import native_fft as oracle
    from qe_python_b200.basis import grid_slots

    oracle.set_workers(threads)
    try:
        from threadpoolctl import threadpool_limits
        limiter = threadpool_limits(limits=threads)
    except Exception:  # pragma: no cover - threadpoolctl is optional
        limiter = None
    linear, *_ = grid_slots(work.miller, work.shape)
    size = int(np.prod(work.shape))
    psi = np.asfortranarray(work.psi[:, :bands])
    grid = np.zeros((bands, size), dtype=np.complex128)
    plan = oracle.NativeFFTWPlan(grid, work.shape, bands, 1, size)
    result = np.zeros_like(psi)
    beta = np.asfortranarray(work.beta)
    coupling = work.coupling.astype(np.complex128)

    def one():
        oracle.apply_serial(grid, psi, work.potential, linear, plan, size, size, result, 0,
                            work.kinetic)
        becp = oracle.projector_overlaps(beta, psi)
        coupled = np.asfortranarray(coupling @ becp)
        oracle.add_projector_product(result, beta, coupled)

    one()  # warm
    done, start = 0, time.perf_counter()
    while True:
        one()
        done += 1
        elapsed = time.perf_counter() - start
        if elapsed >= seconds:
            break
    if limiter is not None:
        limiter.unregister() if hasattr(limiter, "unregister") else None
    return {"value": done * bands / elapsed, "repeats": done, "elapsed_s": elapsed}


def reference_hpsi_rate(work, bands: int, seconds: float, threads: int) -> dict:
    """Bands/s of the reference's own PlaneWaveHamiltonian.apply_into
    (qepy_pw/diagonalization.py:205-368, its local part through its
    LocalPotentialWorkspace.apply, qepy_pw/basis.py:1354-1455) on the
    microbenchmark operator, from the staged reference package
    (baseline/stage_reference.py) with the oracle as its native module."""
    from oracle import native_fft as oracle
    from oracle.reference_env import load_reference

    load_reference()
    from qepy_pw.basis import LocalPotentialWorkspace as RefWorkspace
    from qepy_pw.basis import PlaneWaveBasis as RefBasis
    from qepy_pw.diagonalization import PlaneWaveHamiltonian as RefHamiltonian

    oracle.set_workers(threads)
    try:
        from threadpoolctl import threadpool_limits
        limiter = threadpool_limits(limits=threads)
    except Exception:  # pragma: no cover - threadpoolctl is optional
        limiter = None
    basis = RefBasis(work.miller, work.vectors, work.kinetic)
    workspace = RefWorkspace(work.miller, work.shape)
    ham = RefHamiltonian(basis, np.zeros(work.shape, dtype=np.complex128),
                         ((np.asfortranarray(work.beta), work.coupling),),
                         local_workspace=workspace, real_potential=work.potential,
                         potential_average=0.0)
    psi = np.asfortranarray(work.psi[:, :bands])
    out = np.empty_like(psi, order="F")
    ham.apply_into(psi, out)  # warm: plans and scratch
    done, start = 0, time.perf_counter()
    while True:
        ham.apply_into(psi, out)
        done += 1
        elapsed = time.perf_counter() - start
        if elapsed >= seconds:
            break
    if limiter is not None and hasattr(limiter, "unregister"):
        limiter.unregister()
    return {"value": done * bands / elapsed, "repeats": done, "elapsed_s": elapsed}


def run_reference(args) -> None:
    world, rank, _local = init_distributed("gloo")
    if rank != 0:
        return
    from oracle.reference_env import reference_available
    from qe_python_b200.workloads import hpsi_microbench

    threads = os.cpu_count() or 1
    work = hpsi_microbench(nbands=args.bands)
    sample = min(32, args.bands)
    per_step = max(1.0, 60.0 / max(1, args.steps + args.warmup))
    if reference_available():
        rate = reference_hpsi_rate
        path = ("the reference's own PlaneWaveHamiltonian.apply_into (staged qepy_pw package) "
                "on the oracle native module (SciPy pocketfft, NumPy BLAS)")
    else:
        rate = cpu_hpsi_rate
        path = ("oracle restatement of apply_serial + projector ZGEMMs (SciPy pocketfft, "
                "NumPy BLAS); the reference package is not staged")
    for _ in range(args.warmup):
        rate(work, sample, 0.0, threads)
    rates = [rate(work, sample, per_step, threads)["value"] for _ in range(args.steps)]
    value = statistics.median(rates)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "bands/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * sample / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "complex128",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "parallelism": "host threads"},
        "cpu_baseline": {
            "value": value, "unit": "bands/s", "cores": threads, "kind": "port",
            "sample": f"{sample} of {args.bands} bands per step, repeated for ~{per_step:.0f} s; "
                      + path,
        },
        "e2e": {"value": value, "unit": "bands/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU side

def run_b200(args) -> None:
    import torch

    world, rank, local = init_distributed("nccl")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    from qe_python_b200 import _lib
    from qe_python_b200 import kernels as K
    from qe_python_b200.basis import LocalPotentialWorkspace, make_bases
    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian
    from qe_python_b200.workloads import hpsi_microbench

    lib = _lib.load()
    work = hpsi_microbench(nbands=args.bands)
    npw, nb = work.npw, work.nbands
    basis = make_bases(work.reciprocal, np.zeros(3), 30.0)[0]
    assert np.array_equal(basis.indices, work.miller)
    terms = ((work.beta, work.coupling),)
    forms = {}
    for name, precision in (("mixed", "f32"), ("fp64", "f64")):
        ws = LocalPotentialWorkspace(basis, work.shape, precision=precision, device=device)
        ham = PlaneWaveHamiltonian(basis, None, terms, local_workspace=ws,
                                   real_potential=torch.from_numpy(work.potential).to(device),
                                   potential_average=0.0)
        psi = to_device_f(work.psi, ham.dtype, device)
        out = torch.empty_like(psi.T).T
        forms[name] = (ws, ham, psi, out)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream()

    def timed_loop(name: str, steps: int, warmup: int, profile: bool):
        ws, ham, psi, out = forms[name]
        for _ in range(warmup):
            ham.apply_into(psi, out)
        torch.cuda.synchronize()
        times, stages = [], []
        launches = 0
        for _ in range(steps):
            passes = (float("nan"),) * 3
            if profile:
                # pass A/B/C split from a profiled local apply of its own: the
                # profiled entry point synchronises, which would leave the
                # device idle while the host launches the next stage
                flush.fill_(1.0)
                torch.cuda.synchronize()
                ws.pass_times = []
                ws._launch_apply(ham._potential, psi, ham._kinetic_kernel, out)
                passes = ws.pass_times[0]
                ws.pass_times = None
            flush.fill_(1.0)
            barrier(world)
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            launches0 = lib.qeb_launch_count()
            ev[0].record(stream)
            # same sequence as PlaneWaveHamiltonian._apply, with events between stages
            ws._launch_apply(ham._potential, psi, ham._kinetic_kernel, out)
            ev[1].record(stream)
            becp = ham.calbec(psi)
            ev[2].record(stream)
            coupled = ham.couple(becp)
            ev[3].record(stream)
            ham.add_projectors(coupled, out)
            ev[4].record(stream)
            torch.cuda.synchronize()
            launches += lib.qeb_launch_count() - launches0
            times.append(ev[0].elapsed_time(ev[4]))
            stages.append((*passes, ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3]),
                           ev[3].elapsed_time(ev[4])))
        return times, stages, launches

    # timed region of the headline value
    with ClockSampler(smi_device_id(local)) as clocks:
        barrier(world)
        torch.cuda.synchronize()
        times, stages, launches = timed_loop("mixed", args.steps, args.warmup, profile=True)
        barrier(world)
        torch.cuda.synchronize()
    staged_ms = max_over_ranks(statistics.mean(times), world, device)
    fp64_times, fp64_stages, _ = timed_loop("fp64", args.steps, args.warmup, profile=True)
    fp64_ms = max_over_ranks(statistics.mean(fp64_times), world, device)

    # headline: the whole mixed-form H|psi> captured as one CUDA graph
    from qe_python_b200.diagonalization import HpsiGraph

    def graph_loop(name: str):
        _ws, ham, psi, _out = forms[name]
        graph = HpsiGraph(ham, nb)
        graph.input.copy_(psi)
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()
        count0 = lib.qeb_launch_count()
        samples = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            barrier(world)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            graph.replay()
            b.record(stream)
            torch.cuda.synchronize()
            samples.append(a.elapsed_time(b))
        # a replayed graph launches the same kernels as the staged loop; the
        # library's launch counter only sees launches made through its API
        return max_over_ranks(statistics.mean(samples), world, device), graph

    with ClockSampler(smi_device_id(local)) as graph_clocks:
        step_ms, mixed_graph = graph_loop("mixed")
    fp64_graph_ms, fp64_graph = graph_loop("fp64")
    del fp64_graph

    # eigenvalue error of the chosen form's H|psi>: Rayleigh quotients
    # <psi|H|psi>/<psi|psi> per band, FP32/split-TF32 H against FP64 H on the
    # same (FP32-representable) vectors, reductions in FP64
    psi64 = forms["mixed"][2].to(torch.complex128)
    rq = {}
    for name in ("mixed", "fp64"):
        _ws, ham, _psi, _out = forms[name]
        hpsi = ham.apply(psi64.to(ham.dtype).T.contiguous().T).to(torch.complex128)
        num = torch.real(torch.sum(psi64.conj() * hpsi, dim=0))
        den = torch.real(torch.sum(psi64.conj() * psi64, dim=0))
        rq[name] = (num / den).cpu().numpy()
    rayleigh_error_ry = float(np.max(np.abs(2.0 * (rq["mixed"] - rq["fp64"]))))

    # end to end through the public API with pinned host buffers
    ws, ham, psi_dev, _ = forms["mixed"]
    # end to end from pinned host memory to pinned host memory through the
    # public HostStreamedHpsi: chunks of 1/8, 3/8, 3/8 and 1/8 of the bands,
    # copies overlapped with compute,
    # the whole pipeline (copies, kernels, cross-stream waits) one captured
    # CUDA graph replayed per step
    from qe_python_b200.diagonalization import HostStreamedHpsi

    streamed = HostStreamedHpsi(forms["mixed"][1], nb, chunks=e2e_chunks(nb),
                                compute_streams=E2E_STREAMS)
    host_in_storage, host_out_storage = streamed.host_buffers()
    host_in_storage[:, :npw] = torch.from_numpy(work.psi.T.astype(np.complex64))
    streamed.capture(host_in_storage, host_out_storage)
    e2e_times = []
    for i in range(args.warmup + args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        streamed.replay()
        b.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e_times.append(a.elapsed_time(b))
    e2e_ms = max_over_ranks(statistics.mean(e2e_times), world, device)
    # the bare copies of one step's bytes, to tell the link's share of e2e
    copy_dev = torch.empty_like(host_in_storage, device=device)
    copy_ms = {}
    for name, copy in (("h2d", lambda: copy_dev.copy_(host_in_storage, non_blocking=True)),
                       ("d2h", lambda: host_out_storage.copy_(copy_dev, non_blocking=True))):
        samples = []
        for _ in range(5):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            copy()
            b.record(stream)
            torch.cuda.synchronize()
            samples.append(a.elapsed_time(b))
        copy_ms[name] = statistics.median(samples)
    del copy_dev

    # roofline of the dominant kernel in the headline (mixed) form
    names = ["pass_a", "pass_b", "pass_c", "calbec_gemm", "coupling_gemm", "add_gemm"]
    # medians for the breakdown (one step held up by the host or a clock
    # sample would otherwise dominate a 10-microsecond stage); the roofline
    # of the dominant kernel uses its mean launch time
    mean_stage = [statistics.mean(s[i] for s in stages) for i in range(len(names))]
    median_stage = [statistics.median(s[i] for s in stages) for i in range(len(names))]
    total_stage = sum(median_stage)
    shares = {n: round(t / total_stage, 4) for n, t in zip(names, median_stage)}
    dominant = names[int(np.argmax(median_stage))]
    c = 8  # complex64 bytes
    nst = ws.stick_count
    nz = work.shape[2]
    n_r = int(np.prod(work.shape))
    P = work.beta.shape[1]
    algorithmic = {
        "pass_a": ("hbm", nb * (npw + nst * nz) * c + npw * 12),
        "pass_b": ("hbm", nb * 2 * nst * nz * c + n_r * 4),
        "pass_c": ("hbm", nb * (nst * nz + 2 * npw) * c + npw * (12 + 4)),
        "calbec_gemm": ("flops", 8.0 * npw * P * nb),
        "coupling_gemm": ("flops", 8.0 * P * P * nb),
        "add_gemm": ("flops", 8.0 * npw * P * nb),
    }
    peaks = measured_peaks()
    kind, amount = algorithmic[dominant]
    seconds = mean_stage[names.index(dominant)] / 1e3
    if kind == "hbm":
        achieved = amount / seconds / 1e9
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved,
                    "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"],
                    "traffic": PASS_B_NCU_TRAFFIC.get((dominant, nb)),
                    "algorithmic_bytes": amount,
                    "peak_source": peaks["source"],
                    "note": "pass B is bound by the shared-memory data path (ncu: L1/TEX "
                            "91 %, issue 70 % active), not by HBM"}
        if dominant == "pass_b":
            roofline["fp32_fft_rate"] = plane_fft_rate(work.shape, nb, seconds)
    elif dominant in ("calbec_gemm", "add_gemm") and forms["mixed"][1].tensor_gemm:
        # split TF32: three tcgen05 TF32 products per real product
        algorithmic_tflops = amount / seconds / 1e12
        achieved = 3.0 * algorithmic_tflops
        peak = peaks["bf16_tflops"] / 2.0
        roofline = {"bound": "tensor", "kernel": dominant, "achieved": achieved,
                    "achieved_algorithmic": algorithmic_tflops, "peak": peak,
                    "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                    "peak_source": f"dense TF32 = half the {peaks['source']} bf16 cuBLAS peak; "
                                   "achieved counts the 3 split-TF32 products"}
    else:
        achieved = amount / seconds / 1e12
        # FP32 SIMT pipes: 148 SMs x 128 FMA/clk x 2 flop x 1.965 GHz (nominal)
        peak = 148 * 128 * 2 * 1.965e9 / 1e12
        roofline = {"bound": "tensor", "kernel": dominant, "achieved": achieved,
                    "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "traffic": None,
                    "peak_source": "nominal FP32 FMA peak (this GEMM runs on FP32 pipes, "
                                   "not tensor cores)"}
    fft_ms = sum(median_stage[:3])
    fft_bytes = sum(algorithmic[n][1] for n in names[:3])
    line = {
        "metric": METRIC,
        "value": world * nb / (step_ms / 1e3),
        "unit": "bands/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "complex64 FFT/V*psi; projector GEMMs split-TF32 on tcgen05, FP32 accumulate",
        "data": "synthetic (seeded, qe_python_b200/workloads.py)",
        "config": {"workload": WORKLOAD, "global_batch": world * nb, "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "fp64": {"value": world * nb / (fp64_graph_ms / 1e3), "unit": "bands/s",
                 "ms_per_step": fp64_graph_ms, "staged_ms_per_step": fp64_ms},
        "staged": {"ms_per_step": staged_ms, "value": world * nb / (staged_ms / 1e3),
                   "note": "same kernels launched one by one with events between stages"},
        "graph": "value/ms_per_step time one CUDA-graph replay of the whole H|psi>",
        "rayleigh_quotient_error_ry": {
            "value": rayleigh_error_ry,
            "note": "max over the 256 bands of |<psi|H|psi>/<psi|psi>| mixed form minus FP64 form"},
        "stages_ms": {n: round(t, 5) for n, t in zip(names, median_stage)},
        "kernel_shares": shares,
        "fft_passes": {"ms": fft_ms, "algorithmic_bytes": fft_bytes,
                       "GBps": fft_bytes / (fft_ms / 1e3) / 1e9},
        "roofline": roofline,
        "gpu_launches": int(launches),
        "e2e": {"value": world * nb / (e2e_ms / 1e3), "unit": "bands/s",
                "h2d_bytes_per_step": host_in_storage.numel() * 8,
                "d2h_bytes_per_step": host_out_storage.numel() * 8,
                "ms_per_step": e2e_ms,
                "bare_copy_ms": {k: round(v, 4) for k, v in copy_ms.items()},
                "link_gbs": {k: round(host_in_storage.numel() * 8 / (v / 1e3) / 1e9, 1)
                             for k, v in copy_ms.items()},
                "note": f"chunks of {e2e_chunks(nb)} bands: input copy, H|psi> and output "
                        f"copy on copy and {E2E_STREAMS} compute streams, the whole pipeline "
                        "one captured CUDA graph; bounded by the host link, whose speed "
                        "varies between boxes"},
        "clocks": graph_clocks.summary(),
        "clocks_staged": clocks.summary(),
    }
    # the SCF legs are single-GPU runs: under torchrun (N > 1) every rank
    # would only repeat them, so they run at N = 1 alone
    if args.scf and args.scf != "none" and world == 1:
        legs = [scf_times(name) for name in args.scf.split(",") if name]
        line["scf"] = legs[0] if len(legs) == 1 else legs
        line["config"]["scf_cells"] = {leg["cell"]: leg["config"] for leg in legs}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = 16
        cpu = cpu_hpsi_rate(work, sample, args.cpu_seconds, threads)
        line["cpu_baseline"] = {
            "value": cpu["value"], "unit": "bands/s", "cores": threads, "kind": "port",
            "sample": f"{sample} bands x {cpu['repeats']} repeats ({cpu['elapsed_s']:.1f} s); "
                      "oracle restatement of apply_serial + projector ZGEMMs, FP64",
        }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def apply_only(args) -> None:
    """One workload, ``args.steps`` H|psi> applications, nothing timed: the
    command line the ncu captures under profiles/ use."""
    import torch

    from qe_python_b200.basis import LocalPotentialWorkspace, make_bases
    from qe_python_b200.device import to_device_f
    from qe_python_b200.diagonalization import PlaneWaveHamiltonian
    from qe_python_b200.workloads import hpsi_microbench

    work = hpsi_microbench(nbands=args.bands)
    basis = make_bases(work.reciprocal, np.zeros(3), 30.0)[0]
    ws = LocalPotentialWorkspace(basis, work.shape, precision=args.apply_only)
    ham = PlaneWaveHamiltonian(basis, None, ((work.beta, work.coupling),), local_workspace=ws,
                               real_potential=torch.from_numpy(work.potential).cuda(),
                               potential_average=0.0)
    psi = to_device_f(work.psi, ham.dtype, ham.device)
    out = None
    for _ in range(max(1, args.steps)):
        out = ham.apply(psi)
    torch.cuda.synchronize()
    print(json.dumps({"apply_only": args.apply_only, "applications": max(1, args.steps),
                      "checksum": float(out.abs().sum())}))


def main():
    args = parse_args()
    if args.apply_only is not None:
        apply_only(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
