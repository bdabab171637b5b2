"""Benchmark: geodesic solves/s on the jittered 512 x 256 torus (131 072 vertices).

Workload: the torus of R = 1, r = 0.3, every vertex moved by N(0, (0.1 h)^2) per coordinate
(h the clean torus's mean edge length, seed 0), and a stream of 64 single-source heat-geodesic
queries whose sources are 64 vertices drawn uniformly without replacement (seed 1). One step
answers all 64 queries on the resident mesh (its pattern, operators and solver states kept on
the device, as a served ``Trimesh`` keeps them). ``value`` is whole-job solves/s with the inputs
resident in HBM; ``e2e`` is the same stream through the public API from host sources to host
distances. Each run also checks a sample of answers against the float64 CPU oracle.

``--impl reference`` times the CPU restatement of the same path (``oracle/``, float64 direct
solves with the factorisations reused across the stream) on the host cores, as the reference arm.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "geodesic solves/s (torus 131k, single-source query stream)"
UNIT = "solves/s"
WORKLOAD = "jittered torus 512x256 (131072 V, 262144 F), 64 single-source queries"


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--queries", type=int, default=64)
    p.add_argument("--cols", type=int, default=512)
    p.add_argument("--rows", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def workload(args: argparse.Namespace) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    from ordito_b200 import creation

    vertices, faces = creation.jittered_torus(args.cols, args.rows, 1.0, 0.3, 0.1, seed=0)
    rng = np.random.default_rng(1)
    sources = rng.choice(vertices.shape[0], size=args.queries, replace=False).astype(np.int32)
    return vertices, faces, sources


# ---------------------------------------------------------------------------------------------
# Distributed plumbing: one process per GPU, replicas (every rank answers its own stream).
# ---------------------------------------------------------------------------------------------


class Dist:
    def __init__(self, gpus: int) -> None:
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            torch.cuda.set_device(self.local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
            self.pg = dist
            self.torch = torch

    def barrier(self) -> None:
        if self.pg is not None:
            self.pg.barrier(device_ids=[self.local_rank])

    def max(self, value: float) -> float:
        if self.pg is None:
            return value
        t = self.torch.tensor([value], dtype=self.torch.float64, device=f"cuda:{self.local_rank}")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.pg is not None:
            self.pg.destroy_process_group()


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    QUERY = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self) -> "Clocks":
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *exc) -> None:
        time.sleep(0.15)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, sm_max, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    sm_max = max(sm_max, float(parts[2]))
                except ValueError:
                    continue
                for name, flag in zip(names, parts[5:9]):
                    if flag.lower() == "active":
                        reasons.add(name)
            os.unlink(self.path)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": sm_max or None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ---------------------------------------------------------------------------------------------
# CPU restatement (the oracle): reference arm and the reported CPU baseline.
# ---------------------------------------------------------------------------------------------


def cpu_stream(vertices: np.ndarray, faces: np.ndarray, sources: np.ndarray) -> tuple[float, dict]:
    """Oracle solves/s over ``sources`` (one query each), factorisations built once and reused;
    returns (solves/s, detail). Setup time is reported separately."""
    from oracle import heat_path as hp

    t0 = time.perf_counter()
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    H = hp.csr_matrix(ops["pattern"], ops["H"])
    P = hp.csr_matrix(ops["pattern"], ops["P"])
    factors = (hp.HeatFactor(H), hp.PoissonFactor(P))
    setup = time.perf_counter() - t0
    t1 = time.perf_counter()
    for s in sources:
        hp.heat_geodesic(vertices, faces, np.array([s]), operators=ops, factors=factors)
    per_query = (time.perf_counter() - t1) / len(sources)
    return 1.0 / per_query, {"setup_s": setup, "per_query_s": per_query}


def run_reference(args: argparse.Namespace, dist: Dist) -> None:
    if dist.rank != 0:
        return
    vertices, faces, sources = workload(args)
    sample = sources[: max(2, min(8, len(sources)))]
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_stream(vertices, faces, sample[:1])
    values = []
    detail = {}
    for _ in range(args.steps):
        v, detail = cpu_stream(vertices, faces, sample)
        values.append(v)
    value = statistics.median(values)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * len(sources) / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "queries_per_step": len(sources)},
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": 1,
            "kind": "port",
            "sample": f"{len(sample)} of the {len(sources)} queries per step; factorisations "
                      f"(scipy SuperLU) built once per step, {detail.get('setup_s', 0):.2f} s",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# The B200 arm.
# ---------------------------------------------------------------------------------------------


def run_b200(args: argparse.Namespace, dist: Dist) -> None:
    from oracle import heat_path as hp
    from ordito_b200 import _lib
    from ordito_b200.device import DeviceArray, synchronize
    from ordito_b200.heat import heat_geodesic
    from ordito_b200.mesh import Trimesh

    _lib.call("ob_set_device", dist.local_rank)
    vertices, faces, sources = workload(args)
    n = vertices.shape[0]
    mesh = Trimesh(vertices, faces.reshape(-1))
    device_sources = [DeviceArray.from_host(np.array([s], dtype=np.int32)) for s in sources]

    def step(results: list) -> None:
        for k, src in enumerate(device_sources):
            results[k] = heat_geodesic(mesh, src)

    results: list = [None] * len(sources)
    for _ in range(max(args.warmup, 3)):
        step(results)
    synchronize()

    # Accuracy against the float64 oracle on a sample of the stream (outside the timed region).
    check = [0, len(sources) // 2, len(sources) - 1]
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    errors = []
    for k in check:
        ref = hp.heat_geodesic(vertices, faces, np.array([sources[k]]), operators=ops, factors=factors)
        errors.append(hp.relative_linf(results[k].numpy(), ref))

    start, end = _events()
    launches0 = _lib.launch_count()
    dist.barrier()
    synchronize()
    with Clocks(dist.local_rank) as clocks:
        _lib.call("ob_event_record", start, None)
        for _ in range(args.steps):
            step(results)
        _lib.call("ob_event_record", end, None)
        synchronize()
    ms = _elapsed(start, end) / args.steps
    launches = _lib.launch_count() - launches0
    dist.barrier()
    ms_max = dist.max(ms)
    value = dist.world * len(sources) / (ms_max / 1e3)

    # End to end through the public API: host sources in, host distances out, every step.
    host_sources = [np.array([s], dtype=np.int32) for s in sources]
    dist.barrier()
    synchronize()
    t0 = time.perf_counter()
    _lib.call("ob_event_record", start, None)
    for _ in range(args.steps):
        for k, src in enumerate(host_sources):
            results[k] = heat_geodesic(mesh, src).numpy()
    _lib.call("ob_event_record", end, None)
    synchronize()
    e2e_ms = max(_elapsed(start, end), (time.perf_counter() - t0) * 1e3) / args.steps
    e2e_ms = dist.max(e2e_ms)
    e2e_value = dist.world * len(sources) / (e2e_ms / 1e3)

    # Roofline of the dominant kernel: the heat system's round mat-vec with its three dots.
    heat_system = mesh.heat_solver(None, method="meshlab").operators.heat_system
    solver = next(iter(heat_system._solvers.values()))
    import ctypes

    info = (ctypes.c_longlong * 5)()
    _lib.call("ob_pcg_info", solver.handle, info)
    n_rows, k_cols, nnz, narrow = int(info[0]), int(info[1]), int(info[2]), int(info[3])
    kernel_ms = ctypes.c_float(0.0)
    _lib.call("ob_pcg_time_matvec", solver.handle, 200, ctypes.byref(kernel_ms), None)
    value_bytes = 4 if narrow else 8
    # Algorithmic bytes of one launch: the values and column indices once, the row offsets, the
    # vector u read once, w written once, and r read for the dots.
    algorithmic = nnz * (value_bytes + 4) + 4 * (n_rows + 1) + 3 * 8 * n_rows * k_cols
    achieved = algorithmic / (kernel_ms.value / 1e3) / 1e9
    peaks = _peaks()

    line = None
    if dist.rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": dist.world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "queries_per_step": len(sources),
                "path": "resident Trimesh; settled Jacobi CG heat solve (f32 values, f64 vectors), "
                        "Chebyshev-12 CG Poisson solve",
                "l2": "inputs resident; the 131k-vertex operators (~8 MB) are L2-resident, no flush",
                "parallelism": f"replicas{dist.world}",
            },
            "accuracy": {"max_rel_linf_vs_fp64_oracle": max(errors), "checked_queries": len(check)},
            "e2e": {
                "value": e2e_value,
                "unit": UNIT,
                "h2d_bytes_per_step": 4 * len(sources),
                "d2h_bytes_per_step": 8 * n * len(sources),
            },
            "gpu_launches": launches // max(args.steps, 1),
            "clocks": clocks.summary(),
            "roofline": {
                "bound": "hbm",
                "kernel": "matvec_dots_kernel<float> (heat system round)",
                "achieved": achieved,
                "peak": peaks["hbm_gbs"],
                "peak_source": peaks["source"],
                "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "traffic": None,
                "kernel_ms": kernel_ms.value,
                "algorithmic_bytes": algorithmic,
                "note": "operator and vectors fit in L2: the fraction is of HBM peak but the kernel "
                        "is L2-served",
            },
        }
        if not args.no_cpu_baseline and dist.world == 1:
            sample = sources[:4]
            cpu_value, detail = cpu_stream(vertices, faces, sample)
            line["cpu_baseline"] = {
                "value": cpu_value,
                "unit": UNIT,
                "cores": 1,
                "kind": "port",
                "sample": f"{len(sample)} single-source queries on the same torus, float64 scipy "
                          f"SuperLU factorisations reused (setup {detail['setup_s']:.2f} s excluded)",
            }
        print(json.dumps(line), flush=True)
    _lib.call("ob_event_destroy", start)
    _lib.call("ob_event_destroy", end)


def _events():
    import ctypes

    from ordito_b200 import _lib

    a, b = ctypes.c_void_p(0), ctypes.c_void_p(0)
    _lib.call("ob_event_create", ctypes.byref(a))
    _lib.call("ob_event_create", ctypes.byref(b))
    return a, b


def _elapsed(a, b) -> float:
    import ctypes

    from ordito_b200 import _lib

    ms = ctypes.c_float(0.0)
    _lib.call("ob_event_elapsed_ms", a, b, ctypes.byref(ms))
    return float(ms.value)


def _peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            data = json.load(f)
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def main() -> None:
    args = parse()
    dist = Dist(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
