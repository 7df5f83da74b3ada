"""Benchmark: pyheat3d's stencil hot path on B200 (one JSON line on rank 0).

Workload (per rank): the plain GPU path at roofline size — 3D 512^3 fp32, periodic, FTCS heat
with r = 0.95/6, uniform random [0, 1) field from seed 0, advanced by the single-step TMA
z-march kernel (``b200/zmarch``). One bench *step* is one solve of ``--time-steps`` updates
(1000 by default). The metric is GLUPS: site updates (every cell, periodic) per second.

- ``value``: device time of K solves with the field resident in HBM (CUDA events on the launching
  stream, max over ranks), inputs larger than L2 (512 MiB per field vs 126 MB L2).
- ``e2e``: the same K solves through the public stepper API with a host->device copy of the
  initial field from pinned memory before and a device->host copy of the result after each
  solve inside the timed region.
- ``roofline``: the z-march kernel's algorithmic bytes (8 B per fp32 update: one read and one
  write of every value) per launch over its average launch time, against the measured HBM copy
  bandwidth.
- ``variants``: the other kernels of the same workload (naive, tb2/3/4/8, 16-bit storage), the 2D
  16384^2 fp32 periodic grid (r = 0.95/4) and the 3D 1024^3 fp32 grid (4 GiB per field), one
  solve each, for the per-variant roofline figures.
- ``cpu_baseline``: the NumPy oracle (pyheat3d's reference algorithm restated) on this host, on a
  bounded sample of the same workload.
- ``precision``, ``batching``, ``serving``: the defect-correction solve of the 256^3 Poisson
  problem, the 512-grid batch and the 2000 req/s request stream (``--no-…`` flags skip them).
- ``zslab``: one (512 N) x 512 x 512 grid split in z over the N ranks (halo exchange + z-range
  z-march per step); on one GPU by default (halos by local copies), across ranks with
  ``--zslab on``.

``--impl reference`` times the reference's CPU path (the NumPy oracle, thread-chunked over
z-slabs with every host core) on the same workload and prints the same line with
``"impl": "reference"``. Multi-GPU (torchrun): every rank advances its own 512^3 field (replicas,
weak scaling); there is no data-path collective.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N3 = 512
N2 = 16384
R3 = 0.95 / 6
R2 = 0.95 / 4
FALLBACK_HBM_GBS = 6650.0
NVSMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5, help="timed solves")
    ap.add_argument("--warmup", type=int, default=3, help="untimed solves (>= 3)")
    ap.add_argument("--time-steps", type=int, default=1000, help="updates per solve")
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--no-variants", action="store_true", help="skip the per-variant table")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving measurement")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision measurement")
    ap.add_argument("--no-small", action="store_true",
                    help="skip the 128^3 Dirichlet case (GPU and NumPy GLUPS, oracle error)")
    ap.add_argument("--zslab", default="auto", choices=("auto", "on", "off"),
                    help="z-slab split measurement: auto runs it on one GPU only (halos by "
                         "local copies); on also runs it across ranks (NCCL halo exchange)")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="length of the Poisson request stream (2000 req/s; 60 s configured)")
    ap.add_argument("--batch-problems", type=int, default=512,
                    help="problems of the batching measurement (512 configured; fewer only for "
                         "profiling the batch kernel)")
    ap.add_argument("--precision-n", type=int, default=256,
                    help="grid edge of the precision measurement (256 configured; smaller only "
                         "for profiling the defect-correction kernels)")
    ap.add_argument("--variant", default="b200/zmarch",
                    help="kernel of the headline line (b200/zmarch; others for profiling)")
    ap.add_argument("--n", type=int, default=None,
                    help="grid edge of the headline field (512; other sizes only for profiling)")
    ap.add_argument("--dims", type=int, default=3, choices=(2, 3),
                    help="3 (the headline); 2 runs a 2D n^2 field (n = 16384) for profiling "
                         "the 2D kernels")
    a = ap.parse_args()
    if a.n is None:
        a.n = N3 if a.dims == 3 else N2
    return a


# ---------------------------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------------------------
def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload_config(dims: int, n: int, storage: str, ws: int) -> dict:
    """The `config` object of both arms' JSON lines: the same workload on both. How many
    updates one bench step covers is reported beside it (`time_steps_per_step`), since the CPU
    arm times a bounded sample of the same solve."""
    return {"workload": f"{dims}D {n}^{dims} {storage} periodic heat, r=0.95/{2 * dims}, "
                        "uniform[0,1) fields, seed 0 (rank r: seed r)",
            "grid": [n] * dims, "bc": "periodic", "storage": storage,
            "units": "site updates (all cells)",
            "l2": f"inputs larger than L2 ({n ** dims * (4 if storage == 'float32' else 2) >> 20}"
                  " MiB field vs 126 MB L2)",
            "parallelism": f"replicas x{ws}"}


def field(n: int, dims: int, seed: int = 0) -> np.ndarray:
    return np.random.default_rng(seed).random((n,) * dims, dtype=np.float32)


class Clocks:
    """nvidia-smi sampler (200 ms) running while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"ph3_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={NVSMI_FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict:
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[4:]))
            except ValueError:
                continue
        try:
            self.path.unlink()
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [r for r in rows if r[2] > 300.0] or rows
        names = ["active_mask", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = set()
        for r in load:
            for nm, v in zip(names[1:], r[3][1:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in load), "sm_max_mhz": rows[0][1],
                "samples": len(load), "power_w_max": max(r[2] for r in rows),
                "reasons": sorted(reasons)}


def profile_traffic(name: str) -> float | None:
    """DRAM bytes per launch from a committed ncu summary (``dram_bytes_per_launch: N`` line)."""
    p = ROOT / "profiles" / name
    if not name or not p.is_file():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def copy_bandwidth(torch, nbytes: int = 1 << 30, iters: int = 20, repeats: int = 5) -> float:
    """Device copy_ bandwidth in GB/s, read + write counted, median (pyheat3d roofline.py:8-29)."""
    n = nbytes // 4
    a = torch.empty(n, device="cuda", dtype=torch.float32).uniform_()
    b = torch.empty_like(a)
    for _ in range(3):
        b.copy_(a)
    torch.cuda.synchronize()
    out = []
    for _ in range(repeats):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(iters):
            b.copy_(a)
        e.record()
        e.synchronize()
        out.append(2.0 * 4 * n * iters / (s.elapsed_time(e) * 1e-3) / 1e9)
    del a, b
    torch.cuda.empty_cache()
    return float(np.median(out))


# ---------------------------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------------------------
def dist_init(torch):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(torch, ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(torch, ws, x: float) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------------------
# the b200 arm
# ---------------------------------------------------------------------------------------------
def time_solves(torch, st, nsolves: int, tsteps: int) -> float:
    """Device seconds of `nsolves` solves on the current stream (field resident)."""
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(nsolves):
        st.step(tsteps)
    e.record()
    e.synchronize()
    return s.elapsed_time(e) * 1e-3


def check_parity(st, u0: np.ndarray, stencil) -> dict:
    """Run the stepper's kernel for max(2, k) updates of the bench field (one pass and a
    remainder for tb<k>) and compare with the oracle (thread-chunked, bit-identical to
    pyheat3d's reference_step / emulated_reference) bit for bit."""
    from oracle import threaded_emulated

    k = st.steps_per_pass
    n = k + 1 if k > 1 else 2
    st.step(n)
    got = st.get()
    want = threaded_emulated(u0, stencil.c0, stencil.c1, stencil.bc, n, st.storage,
                             k if st.storage != "float32" else 1, threads=host_cores())
    diff = int(np.count_nonzero(got != want))
    err = float(np.abs(got.astype(np.float64) - want).max() / np.abs(want).max())
    return {"steps": n, "oracle": "NumPy restatement of pyheat3d reference_step, all host "
            "threads", "bitwise_equal": diff == 0, "mismatches": diff, "max_rel_err": err}


def variant_row(torch, key: str, u0: np.ndarray, stencil, tsteps: int, copy_bw: float) -> dict:
    from pyheat3d_b200.registry import VARIANTS, make_stepper

    from pyheat3d_b200.traffic import tb_model_bytes

    var = VARIANTS[key]
    st = make_stepper(key, u0, stencil)
    st.step(max(3 * var.steps_per_pass, 6))
    torch.cuda.synchronize()
    secs = time_solves(torch, st, 1, tsteps)
    ok = bool(np.isfinite(st.get_tensor().float().sum().item()))
    tile = dict(st.tile)
    st.close()
    cells = u0.size
    glups = cells * tsteps / secs / 1e9
    k = var.steps_per_pass
    bpu = 2.0 * var.bytes_per_value / k
    row = {"glups": round(glups, 2), "bytes_per_update": bpu,
           "effective_GBs": round(glups * bpu, 1), "frac_copy": round(glups * bpu / copy_bw, 4),
           "k": k, "storage": var.storage, "finite": ok}
    if k > 1 and "tx" in tile:  # pyheat3d's halo-aware estimate (benchmark.py:219-230)
        hb = tb_model_bytes(u0.ndim, k, var.bytes_per_value, tile["tx"], tile["ty"], tile["zch"])
        row.update({"halo_model_bytes_per_unit": round(hb, 4),
                    "halo_model_GBs": round(glups * hb, 1),
                    "tile": [tile["tx"], tile["ty"], tile["zch"]]})
    return row


def cpu_sample(u0: np.ndarray, c0: float, c1: float, threads: int, sweeps: int) -> float:
    """GLUPS of the NumPy oracle on `sweeps` updates of u0 (periodic) with `threads` workers."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import reference_step, threaded_step

    u = u0.copy()
    out = np.empty_like(u)
    if threads == 1:
        t0 = time.perf_counter()
        for _ in range(sweeps):
            u = reference_step(u, c0, c1, "periodic")
        dt = time.perf_counter() - t0
    else:
        with ThreadPoolExecutor(threads) as pool:
            threaded_step(u, out, c0, c1, "periodic", threads=threads, pool=pool)  # warm
            t0 = time.perf_counter()
            for _ in range(sweeps):
                threaded_step(u, out, c0, c1, "periodic", threads=threads, pool=pool)
                u, out = out, u
            dt = time.perf_counter() - t0
    return u0.size * sweeps / dt / 1e9


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_b200(a: argparse.Namespace) -> None:
    import torch

    from pyheat3d_b200 import _lib, heat_stencil
    from pyheat3d_b200.registry import make_stepper

    ws, rank, local = dist_init(torch)
    T, K, W = a.time_steps, a.steps, max(3, a.warmup)
    hbm_peak, peak_kind = peaks()
    copy_bw = copy_bandwidth(torch)
    stencil = heat_stencil(a.dims, R3 if a.dims == 3 else R2, "periodic")
    u0 = field(a.n, a.dims, seed=rank)
    cells = u0.size

    # ---- parity first: the measured kernel on the measured field against the oracle
    st = make_stepper(a.variant, u0, stencil)
    parity = check_parity(st, u0, stencil)
    if not parity["bitwise_equal"]:
        raise SystemExit(f"bench: {a.variant} differs from the oracle on the bench field: {parity}")

    # ---- value: K solves, field resident in HBM
    for _ in range(W):
        st.step(T)
    barrier(torch, ws)
    with Clocks(local) as clk:
        secs = time_solves(torch, st, K, T)
    barrier(torch, ws)
    secs = max_over_ranks(torch, ws, secs)
    clocks = clk.summary()
    from pyheat3d_b200.registry import VARIANTS

    var = VARIANTS[a.variant]
    kpass = var.steps_per_pass
    launches = K * (T // kpass + T % kpass)
    value = ws * cells * T * K / secs / 1e9
    launch_s = secs / launches
    # one read + one write of every value per launch (k fused updates per launch for tb<k>)
    alg_bytes = 2.0 * var.bytes_per_value * cells
    achieved = alg_bytes / launch_s / 1e9
    final_ok = bool(np.isfinite(st.get_tensor().sum().item()))

    # ---- e2e: pinned H2D of the initial field, K solves through the stepper API, D2H result
    pin_in = torch.from_numpy(u0).pin_memory()
    pin_out = torch.empty(u0.shape, dtype=torch.float32).pin_memory()
    st.set_state(pin_in)
    st.step(T)
    st.get(out=pin_out)
    barrier(torch, ws)
    t0 = time.perf_counter()
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_ev.record()
    for _ in range(K):
        st.set_state(pin_in)
        st.step(T)
        st.get(out=pin_out)
    e_ev.record()
    e_ev.synchronize()
    e2e_secs = max(s_ev.elapsed_time(e_ev) * 1e-3, 0.0)
    wall = time.perf_counter() - t0
    e2e_secs = max_over_ranks(torch, ws, max(e2e_secs, wall))
    st.close()
    del st
    torch.cuda.empty_cache()
    if _lib.device_status(clear=True) != 0:
        raise RuntimeError("kernel status word set during the bench")

    # ---- per-variant table (rank 0 of a 1-GPU run)
    variants = {}
    if ws == 1 and not a.no_variants:
        for key in ("b200/naive", "b200/tb2", "b200/tb3", "b200/tb4", "b200/tb8",
                    "b200/zmarch-bf16", "b200/tb4-bf16", "b200/zmarch-fp16"):
            try:
                variants["3d512_" + key.split("/")[1]] = variant_row(torch, key, u0, stencil, T,
                                                                     copy_bw)
            except Exception as e:  # pragma: no cover - reported, not fatal
                variants["3d512_" + key.split("/")[1]] = {"error": str(e)[:200]}
        u2 = field(N2, 2)
        st2 = heat_stencil(2, R2, "periodic")
        for key in ("b200/ymarch", "b200/naive", "b200/tb2", "b200/tb4", "b200/tb8",
                    "b200/ymarch-bf16", "b200/tb4-fp16"):
            try:
                variants["2d16384_" + key.split("/")[1]] = variant_row(torch, key, u2, st2, T,
                                                                       copy_bw)
            except Exception as e:  # pragma: no cover
                variants["2d16384_" + key.split("/")[1]] = {"error": str(e)[:200]}
        del u2
        # the largest configured grid: 3D 1024^3 fp32, 4 GiB per field
        u3 = field(2 * N3, 3)
        for key in ("b200/zmarch", "b200/tb4"):
            try:
                variants["3d1024_" + key.split("/")[1]] = variant_row(torch, key, u3, stencil,
                                                                      min(T, 200), copy_bw)
            except Exception as e:  # pragma: no cover
                variants["3d1024_" + key.split("/")[1]] = {"error": str(e)[:200]}
        del u3
        torch.cuda.empty_cache()

    # ---- CPU baseline (rank 0, N = 1)
    cpu = None
    if ws == 1 and rank == 0 and not a.no_cpu:
        cores = host_cores()
        one = cpu_sample(u0, stencil.c0, stencil.c1, 1, 4)
        allc = cpu_sample(u0, stencil.c0, stencil.c1, cores, 12)
        cpu = {"value": round(allc, 4), "unit": "GLUPS", "cores": cores, "kind": "port",
               "sample": f"NumPy oracle, 12 periodic updates of the same 512^3 fp32 field, "
                         f"thread-chunked over z-slabs ({cores} threads)",
               "value_1core": round(one, 4),
               "sample_1core": "NumPy oracle, 4 updates of the 512^3 field, 1 thread "
                               "(pyheat3d numpy/slicing)"}

    extra = {}
    if a.zslab == "on" or (a.zslab == "auto" and ws == 1):
        # every rank takes part (collectives in the same order on all ranks), no try/except
        extra["zslab"] = bench_zslab(torch, ws, rank, min(T, 200), value / ws)
        torch.cuda.empty_cache()
    if ws == 1:
        for name, flag, fn in (("dirichlet_128cubed", a.no_small, lambda: bench_small(torch)),
                               ("precision", a.no_precision,
                                lambda: bench_precision(torch, a.precision_n)),
                               ("batching", a.no_batch,
                                lambda: bench_batching(torch, a.batch_problems)),
                               ("serving", a.no_serve,
                                lambda: bench_serving(torch, a.serve_seconds))):
            if flag:
                continue
            try:
                extra[name] = fn()
            except Exception as e:  # reported in the line, the headline stands
                extra[name] = {"error": f"{type(e).__name__}: {e}"[:300]}
            torch.cuda.empty_cache()

    if rank == 0:
        headline = (a.dims, a.n, a.variant) == (3, N3, "b200/zmarch")
        traffic = profile_traffic("zmarch_tma_512cubed_fp32.md" if headline else "")
        metric = "GLUPS (3D 512^3 fp32 periodic FTCS, single-step TMA z-march)"
        if not headline:  # a profiling run
            metric = f"GLUPS ({a.dims}D {a.n}^{a.dims} {var.storage} periodic FTCS, {a.variant})"
        line = {
            "metric": metric,
            "value": round(value, 2), "kernel": a.variant, "unit": "GLUPS", "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": round(secs / K * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(a.dims, a.n, var.storage, ws),
            "time_steps_per_step": T,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind,
                         "copy_bw_same_run": round(copy_bw, 1),
                         "frac_of_copy_same_run": round(achieved / copy_bw, 4),
                         "alg_bytes_per_launch": alg_bytes,
                         "launch_ms": round(launch_s * 1e3, 5)},
            "e2e": {"value": round(ws * cells * T * K / e2e_secs / 1e9, 2), "unit": "GLUPS",
                    "h2d_bytes_per_step": int(u0.nbytes), "d2h_bytes_per_step": int(u0.nbytes)},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "parity": parity,
            **extra,
            "finite": final_ok,
            "variants": variants,  # last: the longest part of the line
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# z-slab split of one grid over the ranks
# ---------------------------------------------------------------------------------------------
def bench_zslab(torch, ws: int, rank: int, tsteps: int, per_rank_glups: float) -> dict:
    """One (512 N) x 512 x 512 fp32 periodic grid split in z over the N ranks (512 planes each):
    per step a halo exchange and the z-range z-march; device time of `tsteps` steps, max over
    ranks. With one rank the periodic halos are local plane copies."""
    from pyheat3d_b200 import heat_stencil
    from pyheat3d_b200.slab import SlabSplit, SlabStepper

    split = SlabSplit(N3 * ws, ws, True)
    slab = np.zeros((N3 + 2, N3, N3), dtype=np.float32)
    slab[1:-1] = field(N3, 3, seed=rank)  # halos arrive with the first exchange
    st = SlabStepper(slab, heat_stencil(3, R3, "periodic"), split, rank)
    del slab
    st.step(20)
    barrier(torch, ws)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    st.step(tsteps)
    e.record()
    e.synchronize()
    secs = max_over_ranks(torch, ws, s.elapsed_time(e) * 1e-3)
    barrier(torch, ws)
    glups = split.nz * N3 * N3 * tsteps / secs / 1e9
    finite = bool(torch.isfinite(st.owned()).all().item())
    del st
    return {"grid": [split.nz, N3, N3], "ranks": ws, "bc": "periodic", "storage": "float32",
            "time_steps": tsteps, "glups": round(glups, 2),
            "ms_per_update": round(secs / tsteps * 1e3, 4),
            "exchange": "local plane copies" if ws == 1 else "NCCL send/recv of halo planes",
            "vs_whole_grid_per_rank": round(glups / ws / per_rank_glups, 4),
            "finite": finite}


# ---------------------------------------------------------------------------------------------
# precision, batching and serving workloads (1-GPU runs; reported beside the headline)
# ---------------------------------------------------------------------------------------------
def bench_batching(torch, nprob: int = 512) -> dict:
    """512 uneven grids: one persistent launch in a CUDA graph vs per-grid launches."""
    import ctypes

    from oracle import run_reference
    from pyheat3d_b200 import _lib, tune
    from pyheat3d_b200.batch import Batch, synthetic_batch

    # 2D problems take the tuned temporal-block depth (k fused steps per pass); the plain path
    # below runs each grid with the same depth, so results must agree bit for bit
    probs = tune.with_batch_k(synthetic_batch(nprob, seed=0))
    batch = Batch(probs)
    upd = batch.updates
    g = batch.graph(with_reset=True)
    g.replay()
    torch.cuda.synchronize()
    times = []
    for _ in range(2):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        g.replay()
        e.record()
        e.synchronize()
        times.append(s.elapsed_time(e) * 1e-3)
    batched = min(times)
    outs = {i: batch.result_tensor(i).float().cpu().numpy() for i in range(len(probs))}
    # plain path: one ph3_advance per grid on the same buffers
    L = _lib.lib()
    ib = ctypes.c_int(0)

    def plain():
        st = torch.cuda.current_stream().cuda_stream
        for i, _ in enumerate(probs):
            d = batch.descs[i]
            variant = _lib.VARIANT["tb"] if d.k > 1 else _lib.VARIANT["march"]
            _lib.check(L.ph3_advance(d.dims, d.nz, d.ny, d.nx, d.storage, d.bc, d.c0, d.c1,
                                     variant, max(d.k, 1), d.a, d.b, d.src, d.steps, st,
                                     ctypes.byref(ib)))

    batch.reset()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain()
    torch.cuda.synchronize()
    plain_s = time.perf_counter() - t0
    same = all(np.array_equal(outs[i], batch.result_tensor(i).float().cpu().numpy())
               for i in range(0, len(probs), 37))
    # FP64-oracle error on the smallest problems of each storage type
    errs = {}
    order = sorted(range(len(probs)), key=lambda i: probs[i].cells * probs[i].steps)
    for st_name in ("float32", "bfloat16"):
        picked = [i for i in order if probs[i].storage == st_name][:4]
        worst = 0.0
        for i in picked:
            p = probs[i]
            ref = run_reference(p.u0.astype(np.float64), p.stencil.c0, p.stencil.c1,
                                p.stencil.bc, p.steps)
            worst = max(worst, float(np.abs(outs[i] - ref).max() / np.abs(ref).max()))
        errs[st_name] = worst
    cfg, chunk = ctypes.c_int(-1), ctypes.c_int(0)
    _lib.check(L.ph3_tune_get(_lib.KERNEL["batch"], 3, 0, 1, ctypes.byref(cfg),
                              ctypes.byref(chunk)))
    tiles = L.ph3_tune_name(_lib.KERNEL["batch"], 3, 1, max(cfg.value, 0)).decode()
    k2d = tune.batch_k2d()
    del batch, g
    torch.cuda.empty_cache()
    return {"problems": len(probs), "updates": upd, "tiles": tiles, "k_2d": k2d,
            "batched_s": round(batched, 4), "batched_solves_per_s": round(len(probs) / batched, 2),
            "batched_glups": round(upd / batched / 1e9, 2),
            "plain_s": round(plain_s, 4), "plain_solves_per_s": round(len(probs) / plain_s, 2),
            "plain_glups": round(upd / plain_s / 1e9, 2),
            "speedup": round(plain_s / batched, 3), "bitwise_equal_to_plain": bool(same),
            "fp64_oracle_rel_err_smallest4": errs, "graph": True}


def bench_serving(torch, seconds: float) -> dict:
    """Poisson stream, 2000 req/s for `seconds`: continuous batching vs one solve at a time.

    Latencies cover every request that arrived: completed ones by their latency, unfinished ones
    by their age when the stream ended (right-censored, lower bounds; counted in `censored`).
    The FP64-oracle error is measured on the smallest completed requests of each kind and
    storage (the oracle is NumPy on the host, FP64, the same steps or sweeps from the same
    initial field)."""
    from oracle import run_reference
    from pyheat3d_b200.serve import GpuExecutor, PlainServer, Server, poisson_stream

    reqs = poisson_stream(2000.0, seconds, seed=0)
    # the smallest requests of each kind and storage (their results are copied back)
    keep: set[int] = set()
    for kind in ("heat", "jacobi"):
        for storage in ("float32", "bfloat16"):
            group = sorted((r for r in reqs if r.kind == kind and r.storage == storage),
                           key=lambda r: r.cells)
            keep.update(r.rid for r in group[:60])
    ex = GpuExecutor()
    eng_stats = Server(ex, budget_bytes=150e9, max_active=256, quantum=128, keep_ids=keep).run(
        reqs, duration=seconds, drain=False)
    eng = eng_stats.summary()
    torch.cuda.synchronize()
    # FP64-oracle error of served results, up to 4 per (kind, storage)
    errs: dict[str, float] = {}
    picked: dict[str, int] = {}
    for o in sorted((o for o in eng_stats.outcomes if o.result is not None),
                    key=lambda o: reqs[o.rid].cells * o.steps_done):
        req = reqs[o.rid]
        tag = f"{req.kind}_{req.storage}"
        if picked.get(tag, 0) >= 4:
            continue
        picked[tag] = picked.get(tag, 0) + 1
        u, src = ex.init_fields(req)
        c0, c1 = req.coefficients()
        ref = run_reference(u.double().cpu().numpy(), c0, c1, req.bc, o.steps_done,
                            src.double().cpu().numpy() if src is not None else None)
        err = float(np.abs(o.result - ref).max() / max(np.abs(ref).max(), 1e-300))
        errs[tag] = max(errs.get(tag, 0.0), err)
    eng["fp64_oracle_rel_err"] = {k: float(f"{v:.3e}") for k, v in sorted(errs.items())}
    eng["fp64_oracle_sample"] = {k: picked[k] for k in sorted(picked)}
    torch.cuda.empty_cache()
    plain = PlainServer(ex, quantum=128).run(reqs, duration=seconds)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return {"rate_per_s": 2000.0, "stream_s": seconds, "budget_gb": 150.0,
            "engine": eng, "plain": plain.summary(),
            "note": "offered load exceeds one B200 (about 1.7e12 site updates/s of heat work "
                    "alone); both servers stop at the end of the stream; p50/p99 count the "
                    "unfinished requests by their age at that moment (censored, lower bounds); "
                    "Jacobi stops at relative residual <= tol or at max_sweeps"}


def bench_small(torch) -> dict:
    """The reference's CPU-runnable case: 3D 128^3 fp32 with Dirichlet walls (zero boundary
    layer), r = 0.15, uniform [0, 1) from seed 0, 100 steps. GPU GLUPS of the tuned single-grid
    path (``b200/auto``, CUDA events, field resident) beside the NumPy GLUPS of the oracle on one
    host thread (pyheat3d's numpy/slicing backend runs one update per call the same way), and the
    relative error of the GPU result against the oracle (stated bound 1e-6)."""
    from oracle import reference_step
    from pyheat3d_b200 import heat_stencil
    from pyheat3d_b200.registry import make_stepper

    n, steps = 128, 100
    u0 = np.random.default_rng(0).random((n, n, n), dtype=np.float32)
    u0[0] = u0[-1] = 0
    u0[:, 0] = u0[:, -1] = 0
    u0[:, :, 0] = u0[:, :, -1] = 0
    st = heat_stencil(3, 0.15, "dirichlet")
    cells = (n - 2) ** 3
    s = make_stepper("b200/auto", u0, st)
    s.step(steps)  # warm-up
    s.synchronize()
    best = None
    for _ in range(5):
        s.set_state(u0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        s.step(steps)
        b.record()
        b.synchronize()
        t = a.elapsed_time(b) * 1e-3
        best = t if best is None else min(best, t)
    got = s.get()
    s.close()
    ref = u0.copy()
    t0 = time.perf_counter()
    for _ in range(steps):
        ref = reference_step(ref, st.c0, st.c1, "dirichlet")
    cpu_s = time.perf_counter() - t0
    err = float(np.abs(got.astype(np.float64) - ref).max() / np.abs(ref).max())
    return {"grid": [n, n, n], "bc": "dirichlet", "r": 0.15, "steps": steps,
            "units": "interior site updates", "gpu_glups": round(cells * steps / best / 1e9, 2),
            "gpu_ms": round(best * 1e3, 3), "numpy_glups_1thread": round(cells * steps / cpu_s / 1e9, 4),
            "rel_err_vs_oracle": err, "bitwise_equal": bool(np.array_equal(got, ref)),
            "tolerance": 1e-6}


def bench_precision(torch, n: int = 256) -> dict:
    """3D Poisson 256^3 by FP64 defect correction around 16-bit Jacobi."""
    from oracle.precision import discrete_solution, manufactured
    from pyheat3d_b200.precision import DefectCorrection

    h = 1.0 / (n - 1)
    u_exact, f = manufactured(n, 3)
    u_h = discrete_solution(n, 3)
    out = {}
    for storage in ("bfloat16", "float16"):
        dc = DefectCorrection(f, h, storage, "march")
        res = dc.solve(tol=1e-10)
        u = res.host()
        out[storage] = {
            "converged": res.converged, "rel_residual": res.history[-1], "outer": res.outer,
            "inner_sweeps_per_outer": int(res.sweeps / max(res.outer, 1)),
            "sweeps": res.sweeps, "seconds": round(res.seconds, 3),
            "sweep_glups": round(res.sweeps * (n - 2) ** 3 / res.seconds / 1e9, 2),
            "err_vs_fp64_oracle": float(np.abs(u - u_h).max() / np.abs(u_h).max()),
            "err_vs_exact": float(np.abs(u - u_exact).max() / np.abs(u_exact).max()),
        }
        del dc, res
        torch.cuda.empty_cache()
    return {"grid": [n, n, n], "tol": 1e-10, "fp64_oracle": "exact discrete solution "
            "(the manufactured f is an eigenfunction of the 7-point Laplacian)", **out}


# ---------------------------------------------------------------------------------------------
# the reference arm: the reference's CPU path (NumPy oracle), all host threads
# ---------------------------------------------------------------------------------------------
def run_reference(a: argparse.Namespace) -> None:
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from concurrent.futures import ThreadPoolExecutor

    from oracle import threaded_step

    cores = host_cores()
    u = field(N3, 3)
    out = np.empty_like(u)
    c0, c1 = np.float32(1.0 - 6.0 * R3), np.float32(R3)
    sweeps = 1  # one update of the 512^3 field per bench step (bounded sample of a solve)
    W, K = max(3, a.warmup), a.steps
    with ThreadPoolExecutor(cores) as pool:
        for _ in range(W):
            threaded_step(u, out, c0, c1, "periodic", threads=cores, pool=pool)
            u, out = out, u
        t0 = time.perf_counter()
        for _ in range(K * sweeps):
            threaded_step(u, out, c0, c1, "periodic", threads=cores, pool=pool)
            u, out = out, u
        secs = time.perf_counter() - t0
    value = u.size * sweeps * K / secs / 1e9
    line = {
        "impl": "reference",
        "metric": "GLUPS (3D 512^3 fp32 periodic FTCS, single-step TMA z-march)",
        "value": round(value, 4), "unit": "GLUPS", "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": round(secs / K * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(3, N3, "float32", ws),
        "time_steps_per_step": sweeps,
        "cpu_baseline": {"value": round(value, 4), "unit": "GLUPS", "cores": cores,
                         "kind": "port",
                         "sample": f"{sweeps} update of the 512^3 field per step, NumPy oracle "
                                   f"(pyheat3d reference_step restated) chunked over z-slabs on "
                                   f"{cores} threads"},
        "e2e": {"value": round(value, 4), "unit": "GLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)
