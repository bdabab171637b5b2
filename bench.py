"""Benchmark: heat-geodesic solves/s on the jittered 512 x 256 torus (131 072 vertices).

Workload: the torus of R = 1, r = 0.3, every vertex moved by N(0, (0.1 h)^2) per coordinate
(h the clean torus's mean edge length, seed 0), and a stream of 64 single-source queries whose
sources are 64 vertices drawn uniformly without replacement (seed 1). One step answers all 64
queries on the resident mesh -- the served + batched path: the mesh's operators and both Cholesky
factors stay on the device, and the 64 queries run as one batched pass in the factors' ordering
(seeding, the two float64 factored solves over 64 right-hand sides, the gathered divergence and the
shift; ``--refine 1`` adds a float64 refinement step to each solve).
``value`` is whole-job solves/s with the sources resident on the device, four batches in flight
on four streams; ``e2e`` is the same stream through the public API (``heat.BatchPipeline``) from
host source lists to pinned host distances, copies included. The plain drop-in
(``heat_geodesic(vertices, faces, [s])``: assembly, solves and any
factorisation inside every call) and the resident single query are timed beside it. A sample of
the answers is checked against the float64 CPU oracle on every run.

``--impl reference`` times the CPU restatement of the same path (``oracle/``: float64 scipy direct
solves, factorisations reused across the stream) on the host cores, as the reference arm.
"""

from __future__ import annotations

import argparse
import ctypes
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "geodesic solves/s (torus 131k, 64 single-source queries, rel err <= 1e-5 vs FP64)"
UNIT = "solves/s"
WORKLOAD = "jittered torus 512x256 (131072 V, 262144 F), 64 single-source queries per step"
# DRAM bytes (read + write) of one triangular pass of this workload's heat factor at 64 columns,
# measured once by ncu (dram__bytes_read.sum + dram__bytes_write.sum over the pass's 14 launches).
PASS_TRAFFIC_BYTES = 626_995_968
# Timed windows of K steps each; the line's value is the median window's.
TIMED_WINDOWS = 3


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--queries", type=int, default=64)
    p.add_argument("--cols", type=int, default=512)
    p.add_argument("--rows", type=int, default=256)
    p.add_argument("--refine", type=int, default=0)
    # Batches in flight (work sets): 3 / 4 / 6 measured 86.2k / 87.2k / 87.2k solves/s.
    p.add_argument("--in-flight", type=int, default=4, choices=[1, 2, 3, 4, 5, 6])
    p.add_argument("--no-vector-heat", action="store_true", help="skip the transport / log map timings")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-precision", action="store_true")
    p.add_argument("--no-serving", action="store_true")
    p.add_argument("--no-reference-benchmarks", action="store_true")
    p.add_argument("--no-large-mesh", action="store_true")
    p.add_argument("--no-packed", action="store_true")
    p.add_argument("--no-kernel-rooflines", action="store_true")
    p.add_argument("--no-serving-full-range", action="store_true")
    p.add_argument("--no-tune", action="store_true")
    p.add_argument("--pass-schedule", default="", metavar="CHUNK/WAVES",
                   help="a fixed split schedule of the passes instead of the tuned one")
    # Only the per-kernel rooflines, on icosphere(LEVEL) with 1 % radial noise (a profiling case).
    p.add_argument("--kernels-only", type=int, default=0, metavar="LEVEL")
    p.add_argument("--serving-requests", type=int, default=300)
    p.add_argument("--serving-warmup", type=int, default=150)
    p.add_argument("--serving-rate", type=float, default=40.0)
    p.add_argument("--serving-vmax", type=float, default=2e5)
    return p.parse_args()


def workload(args: argparse.Namespace) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    from ordito_b200 import creation

    vertices, faces = creation.jittered_torus(args.cols, args.rows, 1.0, 0.3, 0.1, seed=0)
    rng = np.random.default_rng(1)
    sources = rng.choice(vertices.shape[0], size=args.queries, replace=False).astype(np.int32)
    return vertices, faces, sources


# ---------------------------------------------------------------------------------------------
# Distributed plumbing: one process per GPU; replicas (every rank answers its own stream).
# ---------------------------------------------------------------------------------------------


class Dist:
    """Replicas: every rank runs the whole workload on its own GPU; only the timing is reduced
    (max over ranks). NCCL on GPUs, gloo where no CUDA device is visible (CPU tests)."""

    def __init__(self, backend: str | None = None) -> None:
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.backend = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist
            self.torch = torch
            self.backend = backend

    def barrier(self) -> None:
        if self.pg is None:
            return
        if self.backend == "nccl":
            self.pg.barrier(device_ids=[self.local_rank])
        else:
            self.pg.barrier()

    def max(self, value: float) -> float:
        if self.pg is None:
            return value
        device = f"cuda:{self.local_rank}" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([value], dtype=self.torch.float64, device=device)
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
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None
        # The timed region starts only once nvidia-smi samples: its start-up (NVML
        # initialisation) takes driver locks that can stall this process's launches.
        deadline = time.perf_counter() + 5.0
        while (self.proc is not None and self.proc.poll() is None and time.perf_counter() < deadline
               and os.path.getsize(self.path) == 0):
            time.sleep(0.02)
        time.sleep(0.1)
        return self

    def __exit__(self, *exc) -> None:
        time.sleep(0.1)
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
    """Oracle solves/s over ``sources`` (one query each): factorisations built once (setup, timed
    separately) and reused; the per-query work is the two direct solves, the divergence and the
    shift, all float64."""
    from oracle import heat_path as hp

    t0 = time.perf_counter()
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    setup = time.perf_counter() - t0
    t1 = time.perf_counter()
    for s in sources:
        hp.heat_geodesic(vertices, faces, np.array([s]), operators=ops, factors=factors)
    per_query = (time.perf_counter() - t1) / len(sources)
    return 1.0 / per_query, {"setup_s": setup, "per_query_s": per_query}


_ORACLE_STATE = None


def _oracle_worker_init(cols: int, rows: int, queries: int) -> None:
    """A reference-arm worker: the workload and its two float64 factorisations, built once."""
    global _ORACLE_STATE
    from oracle import heat_path as hp

    vertices, faces, _ = workload(argparse.Namespace(cols=cols, rows=rows, queries=queries))
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    _ORACLE_STATE = (vertices, faces, ops, factors)


def _oracle_worker_solve(share: list[int]) -> tuple[int, float]:
    from oracle import heat_path as hp

    vertices, faces, ops, factors = _ORACLE_STATE
    t0 = time.perf_counter()
    for s in share:
        hp.heat_geodesic(vertices, faces, np.array([s]), operators=ops, factors=factors)
    return len(share), time.perf_counter() - t0


def run_reference(args: argparse.Namespace, dist: Dist) -> None:
    """The oracle port on every host core: one worker process a core (spawned), each holding its
    own factorisations (setup excluded), a step's queries shared among them; a step's time is
    the slowest worker's."""
    if dist.rank != 0:
        return
    import multiprocessing

    vertices, faces, sources = workload(args)
    workers = max(1, min(len(os.sched_getaffinity(0)), len(sources)))
    shares = [[int(s) for s in sources[w::workers]] for w in range(workers)]
    ctx = multiprocessing.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(workers, initializer=_oracle_worker_init,
                  initargs=(args.cols, args.rows, args.queries)) as pool:
        pool.map(_oracle_worker_solve, [[s[0]] for s in shares], chunksize=1)  # every worker set up
        setup = time.perf_counter() - t0
        values = []
        for _ in range(min(max(1, args.steps), 3)):
            done = pool.map(_oracle_worker_solve, shares, chunksize=1)
            values.append(sum(n for n, _ in done) / max(t for _, t in done))
    value = statistics.median(values)
    sample = sources
    detail = {"setup_s": setup}
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": len(values),
        "warmup": 0,
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
            "cores": workers,
            "kind": "port",
            "sample": f"all {len(sample)} queries of a step shared by {workers} worker processes, "
                      f"float64 scipy SuperLU factorisations reused (their {detail.get('setup_s', 0):.2f} s "
                      "setup excluded)",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
# The B200 arm.
# ---------------------------------------------------------------------------------------------


def _events():
    from ordito_b200 import _lib

    a, b = ctypes.c_void_p(0), ctypes.c_void_p(0)
    _lib.call("ob_event_create", ctypes.byref(a))
    _lib.call("ob_event_create", ctypes.byref(b))
    return a, b


def _elapsed(a, b) -> float:
    from ordito_b200 import _lib

    ms = ctypes.c_float(0.0)
    _lib.call("ob_event_elapsed_ms", a, b, ctypes.byref(ms))
    return float(ms.value)


def _peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            data = json.load(f)
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


# The reference's own published heat_geodesic timings (docs/benchmarks/heat.md:52-57; RTX 5090,
# pytest-benchmark medians, synchronised; single source vertex 0): full = assembly inside the
# call, amortized = a warm Trimesh holding both factors.
REFERENCE_HEAT_MS = {
    "sphere_small": (4, 3.47, 0.3243),
    "sphere_med": (6, 6.60, 0.6897),
    "sphere_large": (7, 21.63, 1.48),
}


def run_reference_benchmarks() -> dict:
    """The reference's headline benchmark on its own meshes: heat_geodesic full and amortized on
    icospheres of 2 562, 40 962 and 163 842 vertices, source 0, medians of timed calls each
    followed by a device synchronise, beside the published numbers (another GPU)."""
    from oracle import heat_path as hp
    from ordito_b200 import creation
    from ordito_b200 import heat as gheat
    from ordito_b200.device import synchronize
    from ordito_b200.mesh import Trimesh

    src = np.array([0], dtype=np.int32)
    out = {}
    for name, (level, ref_full, ref_amortized) in REFERENCE_HEAT_MS.items():
        v, f = creation.icosphere(level)
        flat = f.reshape(-1)
        full = []
        for _ in range(8):
            synchronize()
            t0 = time.perf_counter()
            gheat.heat_geodesic(v, flat, src)
            synchronize()
            full.append(time.perf_counter() - t0)
        mesh = Trimesh(v, flat)
        assert mesh.heat_solver(None, method="meshlab").factor()
        warm = gheat.heat_geodesic(mesh, src).numpy()
        amortized = []
        for _ in range(30):
            synchronize()
            t0 = time.perf_counter()
            gheat.heat_geodesic(mesh, src)
            synchronize()
            amortized.append(time.perf_counter() - t0)
        full_ms = 1e3 * statistics.median(full[1:])
        amortized_ms = 1e3 * statistics.median(amortized)
        out[name] = {
            "vertices": int(v.shape[0]),
            "full_ms": full_ms,
            "amortized_ms": amortized_ms,
            "reference_full_ms": ref_full,
            "reference_amortized_ms": ref_amortized,
            "speedup_full": ref_full / full_ms,
            "speedup_amortized": ref_amortized / amortized_ms,
            "max_rel_linf_vs_fp64_oracle": hp.relative_linf(warm, hp.heat_geodesic(v, f, src)),
        }
        mesh.dispose()
    out["note"] = ("reference numbers are ordito's published medians on an RTX 5090 "
                   "(docs/benchmarks/heat.md:52-57), not run here")
    return out


def _sell_entries(handle) -> int:
    """The sliced-ELL entries (padding included) a CG solver's mat-vecs read."""
    from ordito_b200 import _lib

    info = (ctypes.c_longlong * 6)()
    _lib.call("ob_pcg_info", handle, info)
    return int(info[5])


def _sell_bytes(n: int, entries: int, value_bytes: int) -> int:
    """Bytes of one CG mat-vec with its dots over one column: the slice starts, every sliced-ELL
    entry's column and value once, u and r in and w out (float64)."""
    return 8 * ((n + 31) // 32 + 1) + (4 + value_bytes) * entries + 3 * 8 * n


def kernel_rooflines(mesh, solver, columns: int = 64, reps: int = 10) -> dict:
    """Each kernel family of the path launched alone on this mesh, timed with CUDA events over
    ``reps`` launches after one warm-up: achieved = algorithmic bytes (every input read and every
    output written once, named per kernel) / average launch time, against the measured HBM copy
    peak. Multi-column kernels run ``columns`` right-hand sides."""
    from ordito_b200 import _lib
    from ordito_b200.device import DeviceArray, synchronize

    peak = _peaks()["hbm_gbs"]
    n, f = mesh.n_vertices, mesh.n_faces
    pattern = mesh.mesh_operator_pattern
    terms_face = mesh.face_terms
    ops = solver.operators
    nnz = ops.heat_system.nnz
    count = pattern.n_keys
    start, end = _events()
    out: dict = {"mesh": {"vertices": n, "faces": f, "stored_entries": nnz}, "columns": columns,
                 "peak_gbs": peak, "kernels": {}}

    def timed(name: str, nbytes: int, launch, what: str, launches: int = 1) -> None:
        launch()
        synchronize()
        _lib.call("ob_event_record", start, None)
        for _ in range(reps):
            launch()
        _lib.call("ob_event_record", end, None)
        ms = _elapsed(start, end) / reps
        record(name, ms, nbytes, what, launches)

    def record(name: str, ms: float, nbytes: int, what: str, launches: int = 1) -> None:
        gbs = nbytes / (ms / 1e3) / 1e9
        out["kernels"][name] = {"ms": ms, "algorithmic_bytes": int(nbytes), "achieved_gbs": gbs,
                                "frac": gbs / peak, "launches": launches, "bytes": what}

    # a1: the pattern build (key kernel, radix sort, run flags, scan, placement).
    offsets = DeviceArray.empty(n + 1, np.int32)
    cols = DeviceArray.empty(count, np.int32)
    run_start = DeviceArray.empty(count, np.int32)
    keys = DeviceArray.empty(count, np.uint64)
    order = DeviceArray.empty(count, np.int32)
    size = ctypes.c_size_t(0)
    _lib.call("ob_pattern_workspace", n, f, ctypes.byref(size))
    workspace = DeviceArray.empty(int(size.value), np.uint8)
    timed("pattern_build", 12 * f + 4 * (n + 1) + 20 * count,
          lambda: _lib.call("ob_pattern_build", mesh.faces.ptr, f, n, offsets.ptr, cols.ptr,
                            run_start.ptr, keys.ptr, order.ptr, workspace.ptr, int(size.value), None),
          "faces in; offsets, columns, run starts, sorted keys and corner order out (the radix "
          "sort's own passes are not counted)")
    del offsets, cols, run_start, keys, order, workspace

    # a2/a3: per-face cot table, normals, areas and the float64 corner sums.
    cot = DeviceArray.empty(3 * f, np.float32)
    normals = DeviceArray.empty(3 * f, np.float32)
    areas = DeviceArray.empty(f, np.float32)
    area_sums = DeviceArray.empty(n, np.float64)
    timed("face_terms", 12 * n + 12 * f + 28 * f + 8 * n,
          lambda: _lib.call("ob_face_terms", mesh.vertices.ptr, mesh.faces.ptr, f, n, cot.ptr,
                            normals.ptr, areas.ptr, area_sums.ptr, None),
          "positions and faces in; cot table, normals, areas and corner sums out")

    # a5: the operator rows L, H, P and the lumped mass.
    values = DeviceArray.empty(3 * count, np.float64)
    mass = DeviceArray.empty(n, np.float64)
    edge_sums = DeviceArray.empty(2, np.float64)
    _lib.call("ob_edge_sums", pattern.offsets.ptr, pattern.columns.ptr, pattern.run_start.ptr,
              pattern.keys.ptr, count, n, mesh.vertices.ptr, 1, edge_sums.ptr, None)
    timed("heat_rows", 4 * (n + 1) + 8 * nnz + 16 * count + 12 * f + 8 * n + 24 * nnz + 8 * n,
          lambda: _lib.call("ob_heat_rows", pattern.offsets.ptr, pattern.columns.ptr,
                            pattern.run_start.ptr, pattern.keys.ptr, count, pattern.order.ptr, n,
                            terms_face.cot.ptr, -1.0, edge_sums.ptr, 1, terms_face.area_sums.ptr,
                            3.0, values.ptr, values.ptr + 8 * count, values.ptr + 16 * count,
                            mass.ptr, None),
          "pattern (offsets, columns, run starts, keys, corner order), cot table and corner sums "
          "in; L, H, P values and mass out")
    del values, mass, cot, normals, areas, area_sums

    # a7/a9: the CG round's first node (y = A u and three column dots), float64 and float32 values.
    H = ops.heat_system
    for narrow in (0, 1):
        handle = ctypes.c_void_p(0)
        _lib.call("ob_pcg_create", n, H.offsets.ptr, H.columns.ptr, H.values.ptr, 1, 1, narrow,
                  ctypes.byref(handle), None)
        ms = ctypes.c_float(0.0)
        _lib.call("ob_pcg_time_matvec", handle, 1, ctypes.byref(ms), None)
        _lib.call("ob_pcg_time_matvec", handle, reps, ctypes.byref(ms), None)
        entries = _sell_entries(handle)
        _lib.lib.ob_pcg_destroy(handle)
        record("pcg_matvec_dots_" + ("f32_values" if narrow else "f64"), ms.value,
               _sell_bytes(n, entries, 4 if narrow else 8),
               "sliced-ELL operator once (slice starts, columns and values, padding included: "
               f"{entries} entries for {nnz} stored), u, r in and w out (float64), one column")
    # The same kernel on an operator of the same size in a local vertex order (a jittered torus
    # 2048 x 1280, row by row): the mat-vec's gathers of u follow the vertex order, and the
    # icosphere's subdivision order scatters each row's neighbours across the vector.
    from ordito_b200 import creation
    from ordito_b200.mesh import Trimesh

    tv, tf = creation.jittered_torus(2048, 1280, 1.0, 0.3, 0.1, seed=0)
    torus = Trimesh(tv, tf.reshape(-1))
    T = torus.heat_solver(None, method="meshlab").operators.heat_system
    handle = ctypes.c_void_p(0)
    _lib.call("ob_pcg_create", T.nrow, T.offsets.ptr, T.columns.ptr, T.values.ptr, 1, 1, 0,
              ctypes.byref(handle), None)
    ms = ctypes.c_float(0.0)
    _lib.call("ob_pcg_time_matvec", handle, 1, ctypes.byref(ms), None)
    _lib.call("ob_pcg_time_matvec", handle, reps, ctypes.byref(ms), None)
    entries = _sell_entries(handle)
    _lib.lib.ob_pcg_destroy(handle)
    record("pcg_matvec_dots_f64_torus_2048x1280", ms.value, _sell_bytes(T.nrow, entries, 8),
           "as pcg_matvec_dots_f64, on the heat system of a 2 621 440-vertex torus in row order")
    torus.dispose()

    # a10: the V-cycle kernels of the Poisson hierarchy on `columns` float32 columns.
    amg = solver.poisson_multigrid
    if not amg.is_jacobi:
        ms = (ctypes.c_float * 5)()
        nbytes = (ctypes.c_longlong * 5)()
        _lib.call("ob_amg_time_kernels", amg.handle, columns, reps, ms, nbytes, None)
        for i, name in enumerate(("amg_sweep", "amg_residual", "amg_restrict", "amg_prolong")):
            record(name, ms[i], nbytes[i], "finest level: offsets, columns, float32 values and "
                   "every vector row once (float32, the columns padded to a power of two)")
        out["amg_vcycle_ms"] = ms[4]
        out["amg_levels"] = amg.grid

    # a8: the divergence from the per-face terms, `columns` fields in and out (float64).
    terms = solver.gradient_terms
    corner_offsets, corner_slots, tile_faces, tile_counts, codes = mesh.corner_tiles
    # A field with a gradient on every face (a zero field skips the normalisation).
    u = DeviceArray.from_host(np.random.default_rng(0).random(n * columns))
    div = DeviceArray.empty(n * columns, np.float64)
    timed("grad_div_terms", 144 * f + 12 * f + 4 * (n + 1) + 12 * f + 2 * 8 * n * columns,
          lambda: _lib.call("ob_grad_div_terms", terms.ptr, mesh.faces.ptr, corner_offsets.ptr,
                            corner_slots.ptr, n, columns, u.ptr, columns, None, div.ptr, columns,
                            None, None, None),
          "per-corner form: per-face terms, faces and corner index in, u in and -div out (float64)")
    from ordito_b200.heat import corner_records

    records, ids = corner_records(terms, mesh.faces, corner_slots, f)
    timed("grad_div_records", 144 * f + 12 * f + 4 * (n + 1) + 12 * f + 2 * 8 * n * columns,
          lambda: _lib.call("ob_grad_div_records", records.ptr, ids.ptr, corner_offsets.ptr, n, columns, u.ptr,
                            columns, None, div.ptr, columns, None, None, None),
          "corner-record form (the served pass's): the per-corner form's algorithmic bytes (the records "
          "themselves hold 336 B a face against the terms' 144), u in and -div out (float64)")
    del records, ids
    timed("grad_div_tiled", 144 * f + 12 * f + 4 * (n + 1) + 2 * 12 * f + 2 * 8 * n * columns,
          lambda: _lib.call("ob_grad_div_tiled", terms.ptr, mesh.faces.ptr, corner_offsets.ptr,
                            corner_slots.ptr, tile_faces.ptr, tile_counts.ptr, codes.ptr, n, columns,
                            u.ptr, columns, None, div.ptr, columns, None, None, None),
          "face-major form (built, off): per-face terms, faces, corner index, tile lists and corner "
          "codes in, u in and -div out (float64)")

    # a13: the shift of `columns` fields to their sources, written transposed.
    sources = DeviceArray.from_host(np.arange(columns, dtype=np.int32) * (n // columns))
    source_offsets = DeviceArray.from_host(np.arange(columns + 1, dtype=np.int32))
    iperm = DeviceArray.from_host(np.arange(n, dtype=np.int32))
    timed("shift", 4 * n + 2 * 8 * n * columns,
          lambda: _lib.call("ob_shift_permuted", u.ptr, n, columns, iperm.ptr, sources.ptr,
                            source_offsets.ptr, columns, 1, div.ptr, None),
          "phi in (float64, once), the numbering in, the shifted fields out", launches=2)
    synchronize()
    _lib.call("ob_event_destroy", start)
    _lib.call("ob_event_destroy", end)
    return out


def run_kernels_only(level: int) -> None:
    """The per-kernel rooflines alone on icosphere(level) with 1 % radial noise (seed 0)."""
    from ordito_b200 import creation
    from ordito_b200.mesh import Trimesh

    v, f = creation.icosphere(level)
    mesh = Trimesh(creation.radial_noise(v, 0.01, 0), f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    result = kernel_rooflines(mesh, solver, reps=3)
    result["workload"] = f"icosphere({level}) + 1 % radial noise"
    print(json.dumps(result), flush=True)
    mesh.dispose()


def run_large_mesh(with_rooflines: bool = True) -> tuple[dict, dict | None]:
    """The large single mesh: icosphere(9) (2 621 442 vertices) with 1 % seeded radial noise, 8
    uniform sources, one query at a time on the resident mesh. Its factors (9.7 GB each) are over
    the factorisation budget, so the heat solve is the settled CG with the band march behind it
    and the Poisson solve the mixed-precision multigrid solve. The float64 host oracle cannot
    factor this mesh in a bench run (SuperLU: minutes and tens of GB), so the same path -- the
    budget forced below the factor's size -- is checked against the oracle on icosphere(6)."""
    import oracle.heat_path as hp
    from ordito_b200 import cholesky as gchol
    from ordito_b200 import creation
    from ordito_b200 import heat as gheat
    from ordito_b200.device import synchronize
    from ordito_b200.mesh import Trimesh

    v, f = creation.icosphere(9)
    v = creation.radial_noise(v, 0.01, 0)
    n = v.shape[0]
    sources = np.random.default_rng(5).choice(n, 8, replace=False).astype(np.int32)
    t0 = time.perf_counter()
    mesh = Trimesh(v, f.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    factored = solver.factor()
    synchronize()
    setup_s = time.perf_counter() - t0
    times = []
    for s in sources:
        synchronize()
        t1 = time.perf_counter()
        gheat.heat_geodesic(mesh, np.array([s], dtype=np.int32), method="meshlab").numpy()
        times.append(time.perf_counter() - t1)
    grid = solver.poisson_multigrid.grid if getattr(solver, "_poisson_multigrid", None) else None
    rooflines = kernel_rooflines(mesh, solver) if with_rooflines else None
    mesh.dispose()
    # The same path on icosphere(6), checked against the oracle.
    budget = gchol.CHOLESKY_MEMORY_BUDGET
    gchol.CHOLESKY_MEMORY_BUDGET = 1 << 10
    try:
        sv, sf = creation.icosphere(6)
        sv = creation.radial_noise(sv, 0.01, 0)
        small = Trimesh(sv, sf.reshape(-1))
        got = gheat.heat_geodesic(small, np.array([7], dtype=np.int32), method="meshlab").numpy()
        check = hp.relative_linf(got, hp.heat_geodesic(sv, sf, np.array([7])))
        small.dispose()
    finally:
        gchol.CHOLESKY_MEMORY_BUDGET = budget
    return {
        "workload": "icosphere(9) + 1 % radial noise (2 621 442 V), 8 single-source queries",
        "factored": factored,
        "setup_s": setup_s,
        "first_query_s": times[0],
        "value": (len(times) - 1) / sum(times[1:]),
        "unit": "solves/s",
        "query_s": times,
        "poisson_multigrid_levels": grid,
        "path": "settled CG (float32 values) + backward-error check + band march (float64) for "
                "the heat system; float32 CG + V-cycle inside float64 refinement (1e-8) for -L",
        "max_rel_linf_vs_fp64_oracle_same_path_ico6": check,
    }, rooflines


def run_packed() -> dict:
    """The batched uneven solve: 256 meshes from seed 0 (icospheres of level 2-6 and jittered tori
    of 16-256 x 8-128), 1-16 single-source queries each, packed as one block-diagonal system with
    both factors; one step = the recorded pass over every query (16 columns), timed with CUDA
    events on its stream after 3 warm-ups."""
    import oracle.heat_path as hp
    from ordito_b200 import _lib
    from ordito_b200.device import synchronize
    from ordito_b200.packed import PackedMeshes, packed_workload, total_queries

    work = packed_workload(0, 256)
    queries = total_queries(work.queries)
    synchronize()
    t0 = time.perf_counter()
    packed = PackedMeshes(work.meshes, max_columns=16)
    synchronize()
    setup_s = time.perf_counter() - t0
    k = packed.load(work.queries)
    stream = ctypes.c_void_p(0)
    _lib.call("ob_stream_create", ctypes.byref(stream))
    packed.record(k, stream)
    start, end = _events()
    for _ in range(3):
        packed.replay(k, stream)
    steps = 10
    _lib.call("ob_event_record", start, stream)
    for _ in range(steps):
        packed.replay(k, stream)
    _lib.call("ob_event_record", end, stream)
    ms = _elapsed(start, end) / steps
    _lib.call("ob_stream_synchronize", stream)
    out = packed.out.numpy()
    errors = []
    for m in (0, 7, 100, 200, 255):
        v, f = work.meshes[m]
        got = out[0, packed.vertex_offsets[m]:packed.vertex_offsets[m + 1]]
        errors.append(hp.relative_linf(got, hp.heat_geodesic(v, f, np.array([work.queries[m][0]]))))
    result = {
        "workload": "256 meshes (seed 0): icospheres level 2-6 and jittered tori 16-256 x 8-128, "
                    "1-16 single-source queries each",
        "meshes": len(work.meshes),
        "vertices": packed.n,
        "queries": queries,
        "columns": k,
        "setup_s": setup_s,
        "factor_bytes": packed.nbytes,
        "pass_schedule": {role: {"split": list(report["best"]), "narrow_waves": report["narrow_waves"]}
                          for role, report in packed.tuning.items()},
        "ms_per_step": ms,
        "value": queries / (ms / 1e3),
        "unit": "solves/s",
        "max_rel_linf_vs_fp64_oracle": max(errors),
        "checked_meshes": 5,
        "path": "one block-diagonal system over all meshes (per-mesh t), both factors resident, the "
                "whole pass recorded as one CUDA graph",
    }
    _lib.call("ob_event_destroy", start)
    _lib.call("ob_event_destroy", end)
    packed.close()
    _lib.call("ob_stream_destroy", stream)
    return result


def run_serving(rate: float, v_max: float, warmup: int, requests: int) -> dict:
    """The serving stream: Poisson arrivals, meshes log-uniform in size (icospheres and jittered
    tori), 70 % of requests on one of the last 50 meshes, 1-32 sources each, 150 GB HBM budget.
    The first ``warmup`` requests fill the cache untimed (the steady state the stream describes);
    the next ``requests`` are timed at their arrival times."""
    from ordito_b200.serving import GeodesicServer, mesh_for, serving_workload

    total = warmup + requests
    stream = serving_workload(2, total, rate, v_min=1e3, v_max=v_max)
    meshes = {spec: mesh_for(spec) for spec in {r.mesh for r in stream}}
    server = GeodesicServer(hbm_budget=150 << 30, max_columns=64, slots=4)
    try:
        for r in stream[:warmup]:
            server.submit(*meshes[r.mesh], r.sources)
        server.reset_stats()
        timed = stream[warmup:]
        futures = []
        origin = time.perf_counter() - timed[0].arrival
        for r in timed:
            delay = origin + r.arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            futures.append(server.submit(*meshes[r.mesh], r.sources))
        for f in futures:
            f.result(timeout=1800)
        stats = server.stats()
    finally:
        server.close()
    stats.update({
        "unit": "solves/s",
        "offered_rate_per_s": rate,
        "mesh_vertices": [1e3, v_max],
        "reuse": 0.7,
        "hbm_budget_gb": 150,
        "warmup_requests": warmup,
        "what": "GeodesicServer: continuous batching on 4 CUDA streams, resident factors keyed by "
                "mesh hash, LRU eviction under the budget; latency = arrival to host result",
    })
    return stats


def run_vector_heat(mesh, source: int) -> dict:
    """transport_tangent_vectors and log_map (both constructions) on a resident mesh: the first
    call (tables, vector system, settled solves) and the median of 5 warm calls, host wall time
    with a device synchronise around each call."""
    from ordito_b200 import heat as gheat
    from ordito_b200.device import synchronize

    def timed(fn) -> tuple[float, float]:
        times = []
        for _ in range(7):
            synchronize()
            t0 = time.perf_counter()
            fn()
            synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
        return times[0], statistics.median(times[2:])

    src = np.array([source], dtype=np.int32)
    vec = np.array([[0.6, 0.8]], dtype=np.float32)
    out = {"mesh_vertices": mesh.n_vertices}
    first, warm = timed(lambda: gheat.transport_tangent_vectors(mesh, src, vec))
    out["transport_tangent_vectors"] = {"first_ms": first, "warm_ms": warm}
    for method in gheat.LOG_MAP_METHODS:
        first, warm = timed(lambda: gheat.log_map(mesh, source, method=method))
        out[f"log_map_{method}"] = {"first_ms": first, "warm_ms": warm}
    out["what"] = ("warm = the vector heat system (2V rows) and the heat system factored on the "
                   "device, two solves a call plus the per-vertex kernels")
    return out


def run_b200(args: argparse.Namespace, dist: Dist) -> None:
    from oracle import heat_path as hp
    from ordito_b200 import _lib
    from ordito_b200 import heat as gheat
    from ordito_b200.device import DeviceArray, PinnedArray, synchronize
    from ordito_b200.mesh import Trimesh

    _lib.call("ob_set_device", dist.local_rank)
    vertices, faces, sources = workload(args)
    n = vertices.shape[0]
    k = len(sources)
    sets = [[int(s)] for s in sources]

    # Resident state: mesh, operators and both factors (timed once, reported as setup).
    synchronize()
    t0 = time.perf_counter()
    mesh = Trimesh(vertices, faces.reshape(-1))
    solver = mesh.heat_solver(None, method="meshlab")
    assert solver.factor(), "factorisation refused"
    # The passes' tile schedule tuned to this mesh's tree at the batch width (part of setup);
    # --no-tune keeps the default schedule (short launch lists for profiling).
    tuning = None if args.no_tune or args.pass_schedule else solver.tune(k)
    if args.pass_schedule:
        chunk, waves = (int(x) for x in args.pass_schedule.split("/"))
        for factor in (solver.heat_factor, solver.poisson_factor):
            _lib.call("ob_chol_tile", factor.handle, chunk, waves, None)
    synchronize()
    setup_s = time.perf_counter() - t0
    src, offsets, _ = gheat._source_columns(sets, n)

    # The numeric factorisations on the device, timed alone over the solver's analysis (the
    # ordering and symbolic structure, host work, timed once on its own).
    from ordito_b200.cholesky import CholeskyAnalysis, SparseCholesky

    synchronize()
    t_analysis = time.perf_counter()
    CholeskyAnalysis(solver.operators.heat_system, mesh.vertices).close()
    factorization = {"analysis_ms": (time.perf_counter() - t_analysis) * 1e3}
    for role, matrix, singular in (("heat", solver.operators.heat_system, False),
                                   ("poisson", solver.operators.poisson_system, True)):
        times = []
        for _ in range(3):
            synchronize()
            t_factor = time.perf_counter()
            SparseCholesky(matrix, solver.heat_factor.analysis, singular=singular).close()
            times.append((time.perf_counter() - t_factor) * 1e3)
        factorization[f"{role}_ms"] = statistics.median(times)
    factorization["what"] = ("ob_chol_factor on the device: multifrontal over the dissection tree, "
                             "float64 tensor-core panel and trailing products, the stored "
                             "[L11^-1; G] blocks formed alongside; host wall time with a device "
                             "synchronise, median of 3")

    # One step = the whole batched pass, recorded once as a CUDA graph (BatchStep) and replayed
    # with one launch on its own stream; with refinement steps, the eager pass instead.
    stream = ctypes.c_void_p(0)
    _lib.call("ob_stream_create", ctypes.byref(stream))
    in_flight = 1
    if args.refine == 0:
        # Several batches in flight: the factors' work sets, each pass recorded on its own stream,
        # consecutive steps taking them in turn (a served stream of batches).
        in_flight = args.in_flight
        streams = [stream]
        for _ in range(in_flight - 1):
            extra = ctypes.c_void_p(0)
            _lib.call("ob_stream_create", ctypes.byref(extra))
            streams.append(extra)
        graph_steps = [gheat.BatchStep(mesh, solver, src, offsets, k,
                                       DeviceArray.empty((k, n), np.float64), streams[w], work_set=w)
                       for w in range(in_flight)]
        turn = [0]

        def step():
            w = turn[0]
            turn[0] = (w + 1) % in_flight
            return graph_steps[w].launch(streams[w])
    else:
        stream = ctypes.c_void_p(0)  # the eager pass runs on the default stream

        def step():
            return gheat._batch_columns(mesh, solver, src, offsets, k, args.refine, True)

    out = None
    for _ in range(max(args.warmup, 3)):
        out = step()
    synchronize()

    # Accuracy against the float64 oracle on a sample of the batch (outside the timed region).
    result = out.numpy()
    t_eff, _ = hp.vertex_time(vertices, faces, None)
    ops = hp.heat_operators(vertices, faces, t_eff)
    factors = (hp.HeatFactor(hp.csr_matrix(ops["pattern"], ops["H"])),
               hp.PoissonFactor(hp.csr_matrix(ops["pattern"], ops["P"])))
    check = sorted({0, k // 2, k - 1})
    errors = [
        hp.relative_linf(result[c], hp.heat_geodesic(vertices, faces, np.array([sources[c]]),
                                                     operators=ops, factors=factors))
        for c in check
    ]

    start, end = _events()
    dist.barrier()
    synchronize()
    # No garbage collection inside the timed regions: a collection there pauses the launching
    # thread while the device drains (the setup above leaves much garbage behind).
    gc.collect()
    gc.disable()
    # Three windows of exactly K steps, each bracketed by a barrier and a device synchronise; the
    # line reports the median window and lists all three (a one-off stall of a few hundred
    # milliseconds inside a window was seen in some runs, cause not identified).
    windows = []
    launches0 = _lib.launch_count()
    with Clocks(dist.local_rank) as clocks:
        for _ in range(TIMED_WINDOWS):
            dist.barrier()
            synchronize()
            _lib.call("ob_event_record", start, stream)
            for other in streams[1:] if in_flight > 1 else []:
                _lib.call("ob_stream_wait_event", other, start)
            for _ in range(args.steps):
                out = step()
            for other in streams[1:] if in_flight > 1 else []:
                joined = ctypes.c_void_p(0)
                _lib.call("ob_event_create", ctypes.byref(joined))
                _lib.call("ob_event_record", joined, other)
                _lib.call("ob_stream_wait_event", stream, joined)
            _lib.call("ob_event_record", end, stream)
            synchronize()
            windows.append(_elapsed(start, end) / args.steps)
    launches = (_lib.launch_count() - launches0) // max(args.steps * TIMED_WINDOWS, 1)
    ms = statistics.median(windows)
    single_ms = None
    if in_flight > 1:
        # The same steps one at a time (one stream, one work set), for the record.
        synchronize()
        _lib.call("ob_event_record", start, stream)
        for _ in range(args.steps):
            graph_steps[0].launch(stream)
        _lib.call("ob_event_record", end, stream)
        synchronize()
        single_ms = _elapsed(start, end) / args.steps
    dist.barrier()
    ms_max = dist.max(ms)
    value = dist.world * k / (ms_max / 1e3)

    # End to end through the public API: host source lists in, host distances out. The serial
    # form (heat_geodesic_batch, then a copy to pinned memory, per batch) and the pipelined one
    # (BatchPipeline: batch i + 1's pass overlaps batch i's copy back), the headline e2e.
    host = PinnedArray((k, n), np.float64)
    dist.barrier()
    synchronize()
    t_wall = time.perf_counter()
    _lib.call("ob_event_record", start, None)
    for _ in range(args.steps):
        batch = gheat.heat_geodesic_batch(mesh, sets, refine=args.refine)
        host.copy_from_device(batch, sync=True)
    _lib.call("ob_event_record", end, None)
    synchronize()
    serial_ms = max(_elapsed(start, end), (time.perf_counter() - t_wall) * 1e3) / args.steps
    serial_ms = dist.max(serial_ms)
    e2e_ms = serial_ms
    e2e_path = "serial: heat_geodesic_batch + copy to pinned host memory per batch"
    if args.refine == 0:
        pipe = gheat.BatchPipeline(mesh, k)
        for _ in pipe.map([sets] * max(args.warmup, 3)):
            pass
        dist.barrier()
        synchronize()
        t_wall = time.perf_counter()
        for _ in pipe.map([sets] * args.steps):
            pass
        e2e_ms = dist.max((time.perf_counter() - t_wall) * 1e3 / args.steps)
        pipe.close()
        e2e_path = ("heat.BatchPipeline: host source lists in, pinned host distances out, the pass "
                    "of one batch overlapping the copy back of the one before")
    e2e_value = dist.world * k / (e2e_ms / 1e3)
    gc.enable()

    # Resident single query (the same factors, one right-hand side at a time).
    single = [[int(s)] for s in sources[:16]]
    synchronize()
    _lib.call("ob_event_record", start, None)
    for s in single:
        gheat.heat_geodesic_batch(mesh, [s], refine=args.refine)
    _lib.call("ob_event_record", end, None)
    synchronize()
    single_value = len(single) / (_elapsed(start, end) / 1e3)

    # The workload's other reading: one query whose source set is all 64 vertices (the distance
    # to the nearest of them), through heat_geodesic on the resident mesh, against the oracle.
    all_sources = np.asarray(sources, dtype=np.int32)
    multi = gheat.heat_geodesic(mesh, all_sources).numpy()
    synchronize()
    _lib.call("ob_event_record", start, None)
    for _ in range(10):
        gheat.heat_geodesic(mesh, all_sources)
    _lib.call("ob_event_record", end, None)
    synchronize()
    multi_ms = _elapsed(start, end) / 10
    multi_error = hp.relative_linf(multi, hp.heat_geodesic(vertices, faces, all_sources, operators=ops,
                                                            factors=factors))

    # Plain drop-in: heat_geodesic(vertices, faces, [s]) builds everything inside every call.
    plain = None
    plain_call_s = None
    if not args.no_plain:
        plain_times = []
        # The median of five calls: a call now and then takes a one-off host or pool cost.
        for s in sources[:5]:
            synchronize()
            t_plain = time.perf_counter()
            gheat.heat_geodesic(vertices, faces.reshape(-1), np.array([s], dtype=np.int32)).numpy()
            plain_times.append(time.perf_counter() - t_plain)
        plain = 1.0 / statistics.median(plain_times)
        plain_call_s = [round(x, 4) for x in plain_times]

    # The vector heat method on the same resident mesh (f3): transport of one tangent vector and
    # both log maps, warm (each call's systems factored by the calls before it).
    vector_heat = None
    if not args.no_vector_heat:
        vector_heat = run_vector_heat(mesh, int(sources[0]))

    # Roofline of the dominant kernel: the factored triangular passes (batched dense products over
    # 64 columns), timed standalone with CUDA events on the heat factor.
    heat_factor = solver.heat_factor
    info = (ctypes.c_longlong * 4)()
    _lib.call("ob_chol_info", heat_factor.handle, info)
    n_vals, levels, pass_launches = int(info[1]), int(info[2]), int(info[3])
    pass_ms = ctypes.c_float(0.0)
    _lib.call("ob_chol_time_solve", heat_factor.handle, k, 20, ctypes.byref(pass_ms), None)
    # One forward + backward pass reads every stored factor value twice (once per direction) and
    # moves the three n x k work vectors about four times; 2 flops per value, column and direction.
    algorithmic = 2 * 8 * n_vals + 4 * 3 * 8 * n * k
    # The bytes a pass cannot avoid: every stored factor value once a direction, the right-hand
    # sides read once and the solutions written once (the work vectors in between can stay in L2).
    compulsory = 2 * 8 * n_vals + 2 * 8 * n * k
    flops = 2 * 2 * n_vals * k
    seconds = pass_ms.value / 1e3
    achieved = algorithmic / seconds / 1e9
    fp64 = ctypes.c_float(0.0)
    _lib.call("ob_fp64_peak", ctypes.byref(fp64), None)
    peaks = _peaks()

    # Precision form: the same batch with the Poisson system on the mixed-precision multigrid solve
    # (float32 CG and V-cycle inside float64 refinement to 1e-10), the heat system factored.
    precision = None
    if not args.no_precision:
        def precise():
            return gheat.heat_geodesic_batch(mesh, sets, refine=0, poisson="multigrid")
        batch = precise()
        synchronize()
        _lib.call("ob_event_record", start, None)
        for _ in range(3):
            batch = precise()
        _lib.call("ob_event_record", end, None)
        synchronize()
        p_ms = _elapsed(start, end) / 3
        result = batch.numpy()
        p_errors = [
            hp.relative_linf(result[c], hp.heat_geodesic(vertices, faces, np.array([sources[c]]),
                                                         operators=ops, factors=factors))
            for c in check
        ]
        precision = {
            "value": k / (p_ms / 1e3),
            "unit": UNIT,
            "ms_per_step": p_ms,
            "max_rel_linf_vs_fp64_oracle": max(p_errors),
            "multigrid_levels": solver.poisson_multigrid.grid,
            "what": "heat_geodesic_batch(..., poisson='multigrid'): Poisson by float32 CG with the "
                    "float32 smoothed-aggregation V-cycle inside float64 refinement to a relative "
                    "residual of 1e-10; heat by the float64 factor (its far field is below float32)",
        }

    # The reference's own benchmark runs before the serving stream, whose hundred-odd resident
    # meshes and their teardown would otherwise sit under its host-bound full calls.
    reference_benchmarks = None
    if not args.no_reference_benchmarks and dist.world == 1:
        reference_benchmarks = run_reference_benchmarks()
    serving = None
    if not args.no_serving and dist.world == 1:
        # The earlier sections' meshes and factors freed now, not by a collection inside the
        # stream's window (a factor's release waits for the device).
        gc.collect()
        synchronize()
        serving = run_serving(args.serving_rate, args.serving_vmax, args.serving_warmup,
                              args.serving_requests)
        if not args.no_serving_full_range:
            # The stream's full size range (1e3 - 2e6 vertices): the largest meshes are past the
            # factorisation budget or take seconds to factor on the host, so at a lower rate.
            serving["full_range"] = run_serving(10.0, 2e6, 60, 120)
    packed = None
    if not args.no_packed and dist.world == 1:
        try:
            packed = run_packed()
        except Exception as exc:  # noqa: BLE001 -- reported on the line, not fatal to it
            packed = {"error": f"{type(exc).__name__}: {exc}"}
    large_mesh = rooflines = None
    if not args.no_large_mesh and dist.world == 1:
        try:
            large_mesh, rooflines = run_large_mesh(not args.no_kernel_rooflines)
        except Exception as exc:  # noqa: BLE001 -- reported on the line, not fatal to it
            large_mesh = {"error": f"{type(exc).__name__}: {exc}"}

    if dist.rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": dist.world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max,
            "timed_windows_ms_per_step": [round(w, 4) for w in windows],
            "batches_in_flight": in_flight,
            "one_in_flight": None if single_ms is None else {
                "value": dist.world * k / (single_ms / 1e3), "ms_per_step": single_ms},
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {
                "workload": WORKLOAD,
                "queries_per_step": k,
                "path": "served + batched: resident Trimesh, nested-dissection supernodal Cholesky "
                        "of M - tL and -L held on the device, 64 right-hand sides per pass, the "
                        "whole pass recorded once as a CUDA graph (one launch a step), "
                        f"{args.refine} float64 refinement step(s) per solve"
                        + (" (in-place passes in the factors' ordering)" if args.refine == 0 else ""),
                "l2": f"no flush; per step the two {8 * n_vals / 1e6:.0f} MB factors "
                      f"({2 * 8 * n_vals / 1e6:.0f} MB) exceed the 126 MB L2",
                "parallelism": f"replicas{dist.world}",
                "setup_s": setup_s,
                "pass_schedule": {role: {"best": list(report["best"]),
                                         "narrow_waves": report["narrow_waves"],
                                         "width_ms": {str(w): round(t, 4) for w, t in report["width_ms"].items()},
                                         "ms": {f"{c}/{w}": round(t, 4) for (c, w), t in report["ms"].items()}}
                                  for role, report in tuning.items()} if tuning else (args.pass_schedule or "default (not tuned)"),
            },
            "accuracy": {"max_rel_linf_vs_fp64_oracle": max(errors), "checked_queries": len(check)},
            "factorization": factorization,
            "vector_heat": vector_heat,
            "e2e": {
                "value": e2e_value,
                "unit": UNIT,
                "h2d_bytes_per_step": 4 * (2 * k + 1),
                "d2h_bytes_per_step": 8 * n * k,
                "path": e2e_path,
                "serial_value": dist.world * k / (serial_ms / 1e3),
            },
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "plain_single_query": {
                "value": plain,
                "unit": UNIT,
                "what": "heat_geodesic(vertices, faces, [s]) per query: assembly, settled CG, the "
                        "backward-error check and its factored fallback inside every call (median of 5)",
                "call_s": plain_call_s,
            },
            "multi_source_query": {"ms": multi_ms, "max_rel_linf_vs_fp64_oracle": multi_error,
                                   "what": "heat_geodesic(mesh, sources) with all 64 sources in one "
                                           "set: the distance to the nearest (factors resident)"},
            "resident_single_query": {"value": single_value, "unit": UNIT,
                                      "what": "heat_geodesic_batch(mesh, [[s]]): factors resident, k = 1"},
            "precision": precision,
            "serving": serving,
            "reference_benchmarks": reference_benchmarks,
            "large_mesh": large_mesh,
            "packed": packed,
            "kernel_rooflines": rooflines,
            "roofline": {
                "bound": "hbm",
                "kernel": "tile_product_kernel (Cholesky forward+backward pass, 64 columns)",
                "achieved": achieved,
                "peak": peaks["hbm_gbs"],
                "peak_source": peaks["source"],
                "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "compulsory_bytes": compulsory,
                "frac_compulsory": compulsory / seconds / 1e9 / peaks["hbm_gbs"],
                "frac_dram": PASS_TRAFFIC_BYTES / seconds / 1e9 / peaks["hbm_gbs"],
                "bar": "frac_compulsory (the factor once a direction, B in, X out) is the HBM "
                       "fraction the pass is judged by; frac counts the work vectors' L2-resident "
                       "moves too, frac_dram the ncu-measured DRAM bytes; the pass is bound by the "
                       "float64 math (fp64.frac)",
                "traffic": PASS_TRAFFIC_BYTES,
                "traffic_source": "one ncu capture: dram__bytes_read.sum + dram__bytes_write.sum "
                                  "over the 14 launches of one pass",
                "pass_ms": pass_ms.value,
                "launches_per_pass": pass_launches,
                "algorithmic_bytes": algorithmic,
                "fp64": {
                    "achieved_tflops": flops / seconds / 1e12,
                    "peak_tflops_measured": fp64.value,
                    "frac": (flops / seconds / 1e12) / fp64.value if fp64.value else None,
                    "intensity_flop_per_byte": flops / algorithmic,
                },
            },
        }
        if not args.no_cpu_baseline and dist.world == 1:
            cpu_value, detail = cpu_stream(vertices, faces, sources[:4])
            line["cpu_baseline"] = {
                "value": cpu_value,
                "unit": UNIT,
                "cores": 1,
                "kind": "port",
                "sample": f"4 single-source queries on the same torus, float64 scipy SuperLU "
                          f"factorisations reused (their {detail['setup_s']:.2f} s setup excluded)",
            }
        print(json.dumps(line), flush=True)
    _lib.call("ob_event_destroy", start)
    _lib.call("ob_event_destroy", end)


def main() -> None:
    args = parse()
    dist = Dist()
    try:
        if args.kernels_only:
            run_kernels_only(args.kernels_only)
        elif args.impl == "reference":
            run_reference(args, dist)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
