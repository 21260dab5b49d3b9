"""Benchmark: close-coupling scattering solves per second on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload cfg2|cfg1|cfg0] [--precision mixed|fp64]

Default workload (cfg2): 512 He-4 beams (E, theta, phi drawn with a fixed
seed) over one corrugated-Morse square potential, 150 Lobatto nodes, each
beam keeping the channels with pkd <= (2m/hbar^2) 200 meV of a 32 x 32
torus (204-262 channels, uneven).  One step = the whole 512-beam batch
solved to ||b - A psi|| <= 1e-10 ||b|| per beam in ONE batched call.

- ``value``: solves/s of the mixed form (FP32 inner GMRES on tcgen05 BF16x3
  + FP32 coupling, FP64 iterative refinement), batched, inputs resident in
  HBM.  Working set: FP32 Krylov basis (21 vectors) 3.0 GB > the 126 MB L2.
- ``plain_fp64``: the plain FP64 form on the same beams, batched and one
  beam at a time (the drop-in's way of working), and the ratio.
- ``accuracy``: max |Delta |S|^2| mixed vs FP64 over the batch and flux error.
- ``e2e``: the same batch through the public API from host numpy arrays:
  plan build (H2D of V, T and every beam's arrays), solve, D2H of |S|^2.
- ``roofline``: the kernel with the largest device-time share, timed with
  CUDA events recorded inside the solve graphs during a timed pass.
- ``cpu_baseline``: the reference algorithm on one host core (the oracle, a
  C restatement of the reference Fortran solve), bounded sample.
Multi-GPU (torchrun): one seeded sweep of 512 x N beams split into N
contiguous slices, one per rank (weak scaling: 512 beams per GPU), time =
max over ranks; no collective on the data path.
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("solves/s (close-coupling S-matrix solves; mixed FP32/BF16x3 + FP64 refinement, "
          "batched; max|dS|^2 <= 1e-6 vs FP64)")
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
KERNEL_NAMES = {
    "block_inverse": "block-diagonal inverse D^-1",
    "coupling": "channel coupling (per-z 2-D convolution)",
    "arnoldi_project": "Arnoldi projection Q^H w",
    "arnoldi_update_project": "Arnoldi update + re-projection + Givens",
    "arnoldi_normalize": "Arnoldi normalisation",
}


def load_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return dict(PEAKS_FALLBACK), "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    QUERY = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples: list[list[str]] = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                     "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                line = out.stdout.strip().splitlines()
                if line:
                    self.samples.append([x.strip() for x in line[0].split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 2 + i and s[2 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def dist_env():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def build_workload(name: str, beams: int = 512, rank: int = 0, world: int = 1):
    """(case, systems) of this rank.  cfg2 on N ranks: one seeded sweep of
    beams x N beams split into N contiguous slices (``replicas.shard``), so
    every rank solves `beams` beams of its own; N = 1 is the headline batch
    ``cfg2_batch(beams, seed=0)``."""
    from multiscat_b200 import workloads as wl
    from multiscat_b200.replicas import shard
    if name == "cfg1":
        case = wl.cfg1_case()
        return case, [case.system()]
    if name == "cfg0":
        case = wl.cfg0_case()
        return case, [case.system()]
    if name == "cfg2":
        case, systems = wl.cfg2_batch(n_solves=beams * world)
        return case, shard(systems, rank, world)
    raise ValueError(name)


def oracle_fixture_error(res, workload: str, beams: int, world: int) -> dict | None:
    """max |Delta |S|^2| of a cfg2 result against the oracle on the 64 beams of
    tests/golden/oracle_cfg2_batch.npz (beams of cfg2_batch(512, seed=0))."""
    path = ROOT / "tests" / "golden" / "oracle_cfg2_batch.npz"
    if workload != "cfg2" or beams != 512 or world != 1 or not path.exists():
        return None
    fx = np.load(path)
    inten = res.intensities.cpu().numpy()
    err, flux = 0.0, 0.0
    for k, b in enumerate(fx["beams"]):
        want = fx["intensities"][fx["offsets"][k]:fx["offsets"][k + 1]]
        got = inten[res.row_offsets[b]:res.row_offsets[b + 1]]
        err = max(err, float(np.abs(got - want).max()))
        flux = max(flux, abs(float(got.sum()) - 1.0))
    return {"max_abs_dI": err, "max_flux_error": flux, "beams_checked": int(len(fx["beams"])),
            "oracle_eps": float(fx["eps"]),
            "fixture": "tests/golden/oracle_cfg2_batch.npz (oracle on 64 beams of this batch: "
                       "8 largest-theta, 8 lowest-E, 8 most-iterations, 40 random)"}


# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# of a kernel kind over the given number of channel rows, from the captures
# summarised in profiles/ (file named beside each entry).  Used as the
# `traffic` of a kernel's roofline line, scaled to the rows of an average
# launch of this run.
NCU_TRAFFIC = {
    # (workload, kind): (bytes, rows of the captured launch, profile)
    ("cfg2", "coupling"): (439.8e6 + 138.9e6, 119741, "k_coupling_halo_f32_cfg2.md"),
    ("cfg2", "coupling_sep"): (79.125e6 + 14.128e6, 30011, "kernels_cfg2_128beams.md"),
    ("cfg2", "block_inverse"): (148.2e6 + 94.3e6, 119741, "k_block_inverse_tc_cfg2.md"),
}


def measure_fma_peaks() -> dict:
    """FP32 and FP64 CUDA-core FMA throughput of this GPU (TFLOP/s), from the
    library's msc_measure_fma_peak kernel timed with CUDA events (best of 3)."""
    import ctypes
    from multiscat_b200 import _native as nat
    lib = nat.load()
    out = {}
    for name, prec in (("fp32", nat.PRECISION_MIXED), ("fp64", nat.PRECISION_FP64)):
        best = 0.0
        for _ in range(3):
            fl = ctypes.c_double(0.0)
            ms = ctypes.c_float(0.0)
            nat.check("msc_measure_fma_peak",
                      lib.msc_measure_fma_peak(prec, 200000, ctypes.byref(fl), ctypes.byref(ms), None))
            best = max(best, fl.value / (ms.value / 1e3) / 1e12)
        out[name] = best
    return out


def kernel_records(kt: dict, res, n: int, taps: int, mixed: bool, dcgs: bool, tensor: bool,
                   peaks: dict, fma: dict, workload: str, sep: tuple | None = None) -> dict:
    """Per timed kernel kind: its bound, algorithmic work of the rows it
    actually processed, achieved rate and fraction of the measured peak.

    block inverse: 8 n^2 flop per row (two real GEMMs of the complex row),
      x3 for the BF16x3 split on tcgen05 (bound: tensor; else the FMA pipe);
    coupling: 8 K n flop per row (K taps, one complex MAC each), ~27 flop per
      byte at K = 80, so the FMA pipe bounds it, not HBM; the separable form
      (sep = (hx, HY) of its window) does 8 ((2hx+1)(8+2HY)/8 + 2HY + 2) n
      flop per row, which leaves its FMA and HBM roofs close: the line names
      the tighter one;
    Arnoldi passes: HBM bytes, one read or write of a row of a Krylov vector
      per vector touched: DCGS2 reduction (j + 1) + 1 reads at step j, update
      (j + 1) + 1 reads and 2 writes; CGS2 first projection (j + 1) + 1 reads,
      update/re-projection and normalisation (j + 1) + 1 reads and 1 write.
    """
    es = 8 if mixed else 16
    rows = np.diff(res.row_offsets).astype(float)
    steps_rows = float(np.dot(rows, res.iterations))
    vec_rows = float(np.dot(rows, res.basis_vectors))
    cyc_rows = float(np.dot(rows, res.cycles))
    fma_peak = fma["fp32" if mixed else "fp64"]
    hbm = peaks["hbm_gbs"]
    bf16 = peaks.get("bf16_tflops_sustained", peaks["bf16_tflops"])
    total_ms = sum(v["ms"] for v in kt.values()) or 1.0
    names = dict(KERNEL_NAMES)
    if dcgs:
        names["arnoldi_project"] = "Arnoldi reduction (DCGS2: Q^H v, Q^H w, norms, coefficients)"
        names["arnoldi_update_project"] = "Arnoldi update (DCGS2: q_j, next candidate, norm, Givens)"
    out = {}
    for k, v in kt.items():
        if not v["launches"]:
            continue
        t_s = v["ms"] / 1e3
        rec = {"what": names[k], "launches": v["launches"], "avg_us": 1e6 * t_s / v["launches"],
               "share_of_timed_kernels": v["ms"] / total_ms}
        if k == "block_inverse":
            r_done = steps_rows + cyc_rows
            fl = 8.0 * n * n * r_done * (3 if tensor else 1)
            rec.update({"bound": "tensor" if tensor else "fma", "unit": "TFLOP/s",
                        "achieved": fl / t_s / 1e12, "peak": bf16 if tensor else fma_peak,
                        "algorithmic": f"{8 * n * n * (3 if tensor else 1)} flop per row",
                        "rows": r_done, "bytes": 2.0 * es * n * r_done})
        elif k == "coupling" and sep:
            hx, hy = sep
            per_row = 8.0 * ((2 * hx + 1) * (8 + 2 * hy) / 8.0 + 2 * hy + 2) * n
            fl = per_row * steps_rows
            nbytes = 3.0 * es * n * steps_rows
            if fl / (fma_peak * 1e12) >= nbytes / (hbm * 1e9):
                rec.update({"bound": "fma", "unit": "TFLOP/s", "achieved": fl / t_s / 1e12,
                            "peak": fma_peak})
            else:
                rec.update({"bound": "hbm", "unit": "GB/s", "achieved": nbytes / t_s / 1e9,
                            "peak": hbm})
            rec.update({"what": "channel coupling, separable form (x pass + y pass)",
                        "algorithmic": f"{per_row:.0f} flop and {3 * es * n} bytes per row",
                        "rows": steps_rows, "bytes": nbytes,
                        "direct_form_equivalent_tflops": 8.0 * taps * n * steps_rows / t_s / 1e12})
        elif k == "coupling":
            fl = 8.0 * taps * n * steps_rows
            rec.update({"bound": "fma", "unit": "TFLOP/s", "achieved": fl / t_s / 1e12,
                        "peak": fma_peak, "algorithmic": f"8 K n = {8 * taps * n} flop per row",
                        "rows": steps_rows, "bytes": 3.0 * es * n * steps_rows})
        else:
            if k == "arnoldi_project":
                vecs = vec_rows + steps_rows
            elif k == "arnoldi_update_project":
                vecs = vec_rows + (3 if dcgs else 2) * steps_rows
            else:
                vecs = vec_rows + 2 * steps_rows
            nbytes = vecs * n * es
            rec.update({"bound": "hbm", "unit": "GB/s", "achieved": nbytes / t_s / 1e9,
                        "peak": hbm, "algorithmic": "one pass per Krylov vector row touched",
                        "rows": steps_rows, "bytes": nbytes})
        rec["frac"] = rec["achieved"] / rec["peak"]
        tr = NCU_TRAFFIC.get((workload, k if not (k == "coupling" and sep) else "coupling_sep"))
        if tr and mixed and "bytes" in rec:
            per_row = tr[0] / tr[1]
            alg_per_row = (3.0 if k == "coupling" else 2.0) * es * n
            rec["traffic_over_algorithmic"] = per_row / alg_per_row
            rec["traffic_profile"] = f"profiles/{tr[2]}"
        out[k] = rec
    return out


def timed_steps(plan, steps: int, stream, torch) -> float:
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        plan.solve()
    stop.record(stream)
    torch.cuda.synchronize()
    return start.elapsed_time(stop)


def run_b200(args) -> None:
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from multiscat_b200 import ScatteringPlan

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        from multiscat_b200.replicas import max_over_ranks as mor
        return mor(x, device="cuda")

    case, systems = build_workload(args.workload, args.beams, rank, world)
    nsys = len(systems)
    stream = torch.cuda.current_stream()
    plan = ScatteringPlan(case.v, case.t, systems, rtol=args.rtol, restart=args.restart,
                          precision=args.precision, inner_restart=args.inner_restart,
                          inner_rtol=args.inner_rtol, preconditioner_order=args.precond_order,
                          gram_schmidt=args.gram_schmidt)
    for _ in range(args.warmup):
        res = plan.solve()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms = timed_steps(plan, args.steps, stream, torch)
    barrier()
    ms = max_over_ranks(ms)
    value = world * nsys * args.steps / (ms / 1e3)
    launches = plan.launches_per_solve() * args.steps
    iters = res.iterations
    inten = res.intensities.clone()
    vs_oracle = oracle_fixture_error(res, args.workload, args.beams, world)
    fallbacks = int(plan.info().fallbacks_last)

    # kernel shares from a separate pass with event pairs inside the graphs
    plan.enable_kernel_timing(True)
    timed_steps(plan, 1, stream, torch)
    kt = plan.kernel_timing()
    plan.enable_kernel_timing(False)
    tuning = plan.tuning_report()
    mixed = args.precision == "mixed"
    n = case.v.shape[2]
    rows = plan.total_rows
    taps = plan.n_taps
    peaks, peak_kind = load_peaks()
    fma = measure_fma_peaks()
    tensor = mixed and "tc_" in tuning.get("chosen", "")
    chosen = tuning.get("chosen", "")
    sep = None
    if ("coupling32=separable" if mixed else "coupling64=separable") in chosen:
        sep = (int(tuning.get("halo_hx", 0)), int(tuning.get("halo_hy", 0)))
    kernels = kernel_records(kt, res, n, taps, mixed, args.gram_schmidt == "dcgs2", tensor,
                             peaks, fma, args.workload, sep)
    roof = None
    if kernels:
        dom = max(kernels, key=lambda k: kernels[k]["share_of_timed_kernels"])
        kr = kernels[dom]
        nl = kr["launches"]
        traffic = None
        tr = NCU_TRAFFIC.get((args.workload, dom if not (dom == "coupling" and sep)
                              else "coupling_sep"))
        if tr and mixed:
            traffic = tr[0] / tr[1] * (kr["rows"] / nl)      # at this run's average rows per launch
        roof = {"kernel": f"{dom}: {kr['what']}", "bound": kr["bound"], "achieved": kr["achieved"],
                "peak": kr["peak"], "unit": kr["unit"], "frac": kr["frac"], "traffic": traffic,
                "peak_source": ("CUDA-core FMA throughput measured in this run "
                                "(msc_measure_fma_peak, best of 3)" if kr["bound"] == "fma" else
                                f"{peak_kind} (MEASURED_PEAKS.json)"),
                "avg_launch_us": kr["avg_us"], "launches_timed": nl,
                "per_launch_work": (f"{kr['rows'] / nl:.0f} channel rows per launch on average "
                                    f"({rows} in the batch; converged systems skip their rows) "
                                    f"x {kr['algorithmic']}"),
                "algorithmic_bytes_per_launch": kr["bytes"] / nl,
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                   f"launch (profiles/{tr[2]}), scaled to the average rows per "
                                   "launch") if traffic else None,
                "share": kr["share_of_timed_kernels"],
                "hbm_frac": kr["bytes"] / (kr["avg_us"] * nl / 1e6) / 1e9 / peaks["hbm_gbs"]}
        if traffic:
            roof["traffic_over_algorithmic"] = traffic / (kr["bytes"] / nl)

    extra = {}
    if not args.quick and rank == 0:
        extra = secondary_measurements(args, case, systems, plan, inten, value, torch, stream)

    e2e = None
    if not args.quick:
        e2e = e2e_measurement(args, case, systems, torch, stream, barrier, max_over_ranks, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_sample(args.workload, case, systems)

    krylov_m = (args.inner_restart or min(args.restart, 20)) if mixed else args.restart
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+bf16x3 (inner), f64 (refinement)" if mixed else "f64",
            "data": "synthetic: seeded corrugated-Morse potential and beams built in-process",
            "config": {"workload": case.name, "systems_per_step": nsys, "rows": rows,
                       "n_z": n, "taps": taps, "restart": args.restart, "rtol": args.rtol,
                       "precision": args.precision,
                       "l2": "inputs larger than L2: Krylov basis "
                             f"{(krylov_m + 1) * rows * n * (8 if mixed else 16) / 1e9:.2f} GB "
                             f"({krylov_m + 1} vectors of {rows} x {n} "
                             f"{'complex64' if mixed else 'complex128'})",
                       "parallelism": (f"beam-sharded sweep over {world} GPUs "
                                       f"({nsys} beams each)" if world > 1 else "1 GPU")},
            "iterations": {"mean": float(np.mean(iters)), "max": int(np.max(iters)),
                           "min": int(np.min(iters))},
            "accuracy_vs_oracle": vs_oracle,
            "fp64_fallbacks_per_step": fallbacks,
            "roofline": roof, "kernels": kernels, "autotune": tuning,
            "fma_peak_tflops": fma,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(),
            "gpu_launches": launches,
        }
        line.update(extra)
        print(json.dumps(line))
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def secondary_measurements(args, case, systems, plan, inten, value, torch, stream) -> dict:
    """Plain FP64 rates (batched and one beam at a time), accuracy, cfg1 solve rates."""
    from multiscat_b200 import ScatteringPlan
    out = {}
    fp64 = ScatteringPlan(case.v, case.t, systems, rtol=args.rtol, restart=args.restart)
    fp64.solve()
    r64 = fp64.solve()
    ms64 = timed_steps(fp64, args.steps, stream, torch) / args.steps
    d = (inten - r64.intensities).abs()
    flux_err = []
    for s in range(len(systems)):
        a, b = plan.row_offsets[s], plan.row_offsets[s + 1]
        flux_err.append(abs(float(inten[a:b].sum()) - 1.0))
    out["accuracy"] = {"max_abs_dI_vs_fp64": float(d.max()),
                       "max_flux_error": float(max(flux_err)),
                       "bar": "max|dS|^2 <= 1e-6 (mixed vs FP64); FP64 parity vs the oracle "
                              "<= 1e-8 is covered by the tests"}
    fp64.close()
    # one beam at a time (a plan per beam, prebuilt; solves timed back to back)
    sample = systems[:min(len(systems), 24)]
    singles = [ScatteringPlan(case.v, case.t, [s], rtol=args.rtol, restart=args.restart)
               for s in sample]
    for p in singles:
        p.solve()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for p in singles:
        p.solve()
    stop.record(stream)
    torch.cuda.synchronize()
    single_rate = len(sample) / (start.elapsed_time(stop) / 1e3)
    for p in singles:
        p.close()
    batched_rate = len(systems) / (ms64 / 1e3)
    out["plain_fp64"] = {
        "batched_solves_per_s": batched_rate,
        "batched_steps_timed": args.steps,
        "batched_vs_oracle": oracle_fixture_error(r64, args.workload, args.beams, 1),
        "one_beam_at_a_time_solves_per_s": single_rate,
        "one_beam_sample": f"{len(sample)} beams, one FP64 plan each, solved back to back",
        "mixed_batched_over_fp64_one_at_a_time": value / single_rate,
        "mixed_batched_over_fp64_batched": value / batched_rate,
    }
    if args.workload != "cfg1":
        from multiscat_b200.workloads import cfg1_case
        c1 = cfg1_case()
        res = {}
        for prec in ("fp64", "mixed"):
            p = ScatteringPlan(c1.v, c1.t, [c1.system()], rtol=args.rtol, precision=prec)
            for _ in range(3):
                p.solve()
            t = timed_steps(p, 5, stream, torch) / 5
            res[prec] = {"solves_per_s": 1e3 / t, "ms": t,
                         "iterations": int(p.solve().iterations[0])}
            p.close()
        out["cfg1_single_solve"] = {"workload": c1.name, **res}
    out["cfg3_adjoint"] = adjoint_measurement(torch, stream)
    out["cfg4_batch"] = cfg4_measurement(args, torch, stream)
    return out


def adjoint_measurement(torch, stream) -> dict:
    """cfg3: forward + adjoint backward of L = sum w |S|^2 w.r.t. (D, alpha, h)
    through the torch potential builder; gradient error vs the oracle's
    central finite differences (tests/golden/oracle_cfg3_fd.json)."""
    from multiscat_b200.adjoint import scattering_intensities
    from multiscat_b200.workloads import cfg3_problem
    pr = cfg3_problem()
    ref_path = ROOT / "tests" / "golden" / "oracle_cfg3_fd.json"
    ref = json.loads(ref_path.read_text()) if ref_path.exists() else None
    w = torch.as_tensor(pr.weights, device="cuda")
    out = {"workload": pr.case.name}
    for prec, rtol in (("fp64", 1e-12), ("mixed", 1e-12)):
        def step():
            p = {k: torch.tensor(v, dtype=torch.float64, device="cuda", requires_grad=True)
                 for k, v in pr.params.items()}
            v = pr.potential(p["depth"], p["alpha"], p["h"], device="cuda")
            loss = (w * scattering_intensities(v, pr.case.t, [pr.case.system()], rtol=rtol,
                                               precision=prec)).sum()
            loss.backward()
            return {k: float(t.grad) for k, t in p.items()}
        for _ in range(2):
            g = step()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(3):
            g = step()
        stop.record(stream)
        torch.cuda.synchronize()
        rec = {"forward_backward_ms": start.elapsed_time(stop) / 3, "grads": g}
        if ref:
            rec["max_rel_err_vs_oracle_fd"] = max(abs(g[k] / ref["params"][k]["dL"] - 1.0)
                                                  for k in g)
        out[prec] = rec
    out["what"] = ("plan build + forward solve + A^H solve + gradient kernel + torch builder "
                   "backward, per step; bar: 1e-5 relative vs finite differences")
    return out


def cfg4_measurement(args, torch, stream) -> dict:
    """cfg4: 16 azimuths of the 81 x 81 x 300 square system (288 taps), batched,
    mixed vs plain FP64; accuracy of the mixed form against FP64."""
    from multiscat_b200 import ScatteringPlan
    from multiscat_b200.workloads import cfg4_batch
    case, systems = cfg4_batch()
    out = {"workload": case.name, "systems": len(systems),
           "rows": int(sum(s.pkd.size for s in systems))}
    inten = {}
    for prec in ("mixed", "fp64"):
        p = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, restart=args.restart,
                           precision=prec)
        r = p.solve()
        steps = max(2, args.steps // 2)
        ms = timed_steps(p, steps, stream, torch) / steps
        inten[prec] = r.intensities
        out[prec] = {"solves_per_s": len(systems) / (ms / 1e3), "ms": ms, "steps_timed": steps,
                     "iterations_max": int(r.iterations.max()),
                     "all_converged": bool((r.status == 0).all()),
                     "autotune": p.tuning_report()}
        p.close()
    out["max_abs_dI_mixed_vs_fp64"] = float((inten["mixed"] - inten["fp64"]).abs().max())
    out["mixed_over_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    return out


def e2e_measurement(args, case, systems, torch, stream, barrier, max_over_ranks, world) -> dict:
    """Whole batch through the public API from host arrays (plan build + solve + D2H)."""
    from multiscat_b200 import ScatteringPlan
    h2d = int(case.v.nbytes + case.t.nbytes)
    for s in systems:
        h2d += int(s.channel_ix.nbytes + s.channel_iy.nbytes + s.pkd.nbytes + s.wave_b.nbytes +
                   s.wave_c.nbytes + 16)
    rows = sum(int(s.pkd.size) for s in systems)
    d2h = rows * 8

    def one():
        p = ScatteringPlan(case.v, case.t, systems, rtol=args.rtol, restart=args.restart,
                           precision=args.precision)
        r = p.solve()
        host = r.intensities.cpu().numpy()
        p.close()
        return host

    one()
    torch.cuda.synchronize()
    barrier()
    steps = args.steps
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        one()
    stop.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(stop))
    return {"value": world * len(systems) * steps / (ms / 1e3), "unit": "solves/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps_timed": steps,
            "path": "ScatteringPlan(host numpy V, T, beams).solve() -> |S|^2 to host, "
                    "plan built inside every step (eigen/autotune caches warm)"}


# ---------------------------------------------------------------------------
# reference (CPU) arm
# ---------------------------------------------------------------------------

def _oracle_time(case, system, maxiter: int) -> float:
    from oracle import solver as osol
    t0 = time.perf_counter()
    osol.solve_channels(case.v, system.channel_ix, system.channel_iy, system.pkd, system.wave_c,
                        system.specular, system.wave_b[system.specular], case.t, eps=0.5e-10,
                        maxiter=maxiter)
    return time.perf_counter() - t0


def _oracle_solve_seconds(case, system, full: int, samples: int) -> tuple[float, str]:
    """Seconds per oracle solve of `system`: timed whole solves when that is
    cheap (under ~5 s), else medians of 1- and 3-iteration runs extrapolated."""
    t1 = _oracle_time(case, system, 1)          # warm-up and estimate
    if t1 * full < 5.0:
        ts = [_oracle_time(case, system, 2000) for _ in range(max(1, samples))]
        return float(np.median(ts)), f"median of {len(ts)} whole oracle solves"
    a = [_oracle_time(case, system, 1) for _ in range(max(1, samples))]
    b = [_oracle_time(case, system, 3) for _ in range(max(1, samples))]
    t1m, t3m = float(np.median(a)), float(np.median(b))
    per_iter = max((t3m - t1m) / 2.0, 0.25 * t1m)
    return t1m + (full - 1) * per_iter, (f"medians of 1- and 3-iteration runs ({t1m:.2f} s, "
                                         f"{t3m:.2f} s) extrapolated to {full} iterations")


def _full_iterations(workload: str) -> int:
    name = {"cfg1": "oracle_cfg1.json", "cfg0": "oracle_cfg0.json"}.get(workload,
                                                                       "oracle_subsets.json")
    g = ROOT / "tests" / "golden" / name
    if g.exists():
        rec = json.loads(g.read_text())
        if isinstance(rec, list):
            return int(round(np.mean([r["iterations"] for r in rec])))
        return int(rec["iterations"])
    return 20


def cpu_reference_sample(workload: str, case, systems) -> dict:
    """Oracle on one host core, beam 0 of the workload."""
    from oracle import solver as osol
    osol.build()
    full = _full_iterations(workload)
    solve_s, how = _oracle_solve_seconds(case, systems[0], full, 3)
    return {"value": 1.0 / solve_s, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": (f"oracle (C restatement of the reference Fortran GMRES: block Gauss-Seidel "
                       f"+ Neumann, unrestarted MGS) on beam 0 of {workload}, one core: {how}"),
            "seconds_per_solve": solve_s}


def _worker_rate(job):
    """One host process: seconds per oracle solve of its own beam."""
    workload, beam, steps = job
    sys.path.insert(0, str(ROOT))
    case, systems = build_workload(workload)
    system = systems[beam % len(systems)]
    return _oracle_solve_seconds(case, system, _full_iterations(workload), steps)


def run_reference(args) -> None:
    """The reference algorithm (oracle) on every host core: one beam per process."""
    import multiprocessing as mp
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import solver as osol
    osol.build()
    cores = max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count())
    full = _full_iterations(args.workload)
    case, systems = build_workload(args.workload)
    nproc = min(cores, max(1, len(systems))) if len(systems) > 1 else 1
    ctx = mp.get_context("spawn")
    with ctx.Pool(nproc) as pool:
        res = pool.map(_worker_rate, [(args.workload, b, args.steps) for b in range(nproc)])
    per_solve = [r[0] for r in res]
    how = res[0][1]
    value = float(sum(1.0 / t for t in per_solve))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(per_solve)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": case.name, "systems_per_step": nproc},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nproc, "kind": "port",
                         "sample": (f"{nproc} host processes at once, one beam each "
                                    f"(beams 0..{nproc - 1}), all cores busy: {how}; the oracle "
                                    f"is the serial C restatement of the reference Fortran "
                                    f"solve")},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=["cfg2", "cfg1", "cfg0"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--restart", type=int, default=30)
    ap.add_argument("--inner-restart", type=int, default=0,
                    help="mixed form: inner FP32 restart (0 = the library default)")
    ap.add_argument("--beams", type=int, default=512,
                    help="cfg2: beams in the batch (the headline workload is 512; smaller "
                         "batches are for profiling captures)")
    ap.add_argument("--inner-rtol", type=float, default=0.0,
                    help="mixed form: inner FP32 reduction per refinement step (0 = the library default)")
    ap.add_argument("--precond-order", type=int, default=0,
                    help="von Neumann order of the preconditioner (0 = block-diagonal)")
    ap.add_argument("--gram-schmidt", default="dcgs2", choices=["dcgs2", "cgs2"],
                    help="Arnoldi orthogonalisation (dcgs2: two basis passes per step; cgs2: three)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="only the main timed steps (no secondary rates, no e2e)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
