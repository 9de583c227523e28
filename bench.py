#!/usr/bin/env python
"""Benchmark: QBX-FMM node-applies/s on the 3D Helmholtz combined-field apply.

Workload (headline): 3D Helmholtz combined field D - i k S, k = 10, on the ellipsoid
(1, 1.5, 2) from an icosphere refined 5 times (20480 triangles), 15 nodes per triangle
(307200 nodes) upsampled to 45 (921600 sources), exterior limit on the surface,
16 plane-wave densities, qbx_order 5, fmm_order 15, complex128 (the plain FP64 form).
node-applies = user targets x densities.  One step = one apply of all 16 densities
(upsample, weight, reorder, every FMM stage, assembly) with the densities resident in
HBM; the L2 cache (126 MB) is flushed between steps by writing a 256 MB buffer outside
the per-step events.  Beside it: the same step in the mixed-precision form, the 3D
Laplace double-layer apply (icosphere-3, 57600 sources, q 3 / p 10) and the CPU
checker on a bounded sample.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (launched by torch.distributed.run): the 16 densities of the one job are split
over the ranks (each rank applies its share on its own GPU, no exchange inside the
apply) and the results are all-gathered in density order inside the timed step
(NCCL); total work is fixed (strong scaling), time is the max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QBX-FMM node-applies/s at stated rel. err"
UNIT = "node-applies/s"

H3 = dict(nrefine=5, k=10.0, nrhs=16, qbx_order=5, fmm_order=15, op="CF")
H3_SAMPLE = dict(nrefine=2, nrhs=1)   # CPU-checker sample: same operator and orders
L3 = dict(nrefine=3, qbx_order=3, fmm_order=10, op="D")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nrefine", type=int, default=H3["nrefine"],
                    help="icosphere refinements of the headline surface (5: full size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-laplace", action="store_true",
                    help="skip the 3D Laplace measurement reported beside the headline")
    ap.add_argument("--no-side-configs", action="store_true",
                    help="skip the batched 2D Helmholtz solve and the 3D Laplace adjoint "
                         "reported beside the headline")
    return ap.parse_args()


def h3_counts(nrefine):
    ntri = 20 * 4 ** nrefine
    return {"triangles": ntri, "nodes": 15 * ntri, "sources": 45 * ntri,
            "user_targets": 15 * ntri}


def config_dict(args, world):
    c = h3_counts(args.nrefine)
    name = ("3D Helmholtz combined field D - ik S, k 10, ellipsoid (1,1.5,2), "
            f"icosphere-{args.nrefine} ({c['triangles']} tri), {c['nodes']} nodes -> "
            f"{c['sources']} sources, 16 plane-wave densities, qbx_order 5, fmm_order 15")
    if args.nrefine != H3["nrefine"]:
        name += " (reduced)"
    return {"workload": name, "nodes": c["nodes"], "sources": c["sources"],
            "user_targets": c["user_targets"], "nrhs": H3["nrhs"], "k": H3["k"],
            "qbx_order": H3["qbx_order"], "fmm_order": H3["fmm_order"],
            "l2": "flushed between steps (256 MB write)",
            "parallelism": "single GPU" if world == 1 else f"densities sharded over {world} GPUs"}


def h3_workload(nrefine, nrhs=H3["nrhs"], seed=0):
    from pytential_b200.workloads import helmholtz3d_ellipsoid
    return helmholtz3d_ellipsoid(nrefine=nrefine, k=H3["k"], nrhs=nrhs, seed=seed, op=H3["op"],
                                 qbx_order=H3["qbx_order"], fmm_order=H3["fmm_order"])


# {{{ clocks

class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    Polls NVML (read-only queries) every 5 ms from a thread; falls back to
    ``nvidia-smi -lms 200`` when NVML is unavailable."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20),
               ("hw_thermal_slowdown", 0x40), ("sw_power_cap", 0x4),
               ("hw_power_brake_slowdown", 0x80))

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.thread = None
        self.samples = []          # (sm_mhz, reason bitmask)
        self.sm_max = None
        self.lines = []

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            idx = int(vis.split(",")[self.index]) if vis and vis.split(",")[self.index].isdigit() \
                else self.index
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _poll(self, pynvml, h):
        while not self.stop.is_set():
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), int(rs)))
            except Exception:
                pass
            self.stop.wait(0.005)

    def __enter__(self):
        import threading
        try:
            pynvml, h = self._nvml_handle()
            self.sm_max = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(pynvml, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join()
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        if self.samples:
            reasons = {nm for nm, bit in self.REASONS for _, rs in self.samples if rs & bit}
            return {"sm_mhz": statistics.median(s for s, _ in self.samples),
                    "sm_max_mhz": self.sm_max, "reasons": sorted(reasons),
                    "samples": len(self.samples), "source": "nvml, 5 ms"}
        if not self.lines:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}

# }}}

# {{{ helpers

def _events(torch, n):
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range(n)]


def time_calls(torch, fn, steps, flush):
    """ms of each of ``steps`` calls of fn(), CUDA events on the current stream, the L2
    flushed before each call outside the events."""
    ev = _events(torch, steps)
    for a, b in ev:
        flush.zero_()
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def kernel_nodes(torch, ap, dens, out):
    """Kernels of this library in one apply: the apply captured into a CUDA graph (not
    instantiated), its kernel nodes counted."""
    from cuda.bindings import runtime as rt
    s = torch.cuda.Stream(device=ap.device)
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph(keep_graph=True)
    with torch.cuda.graph(g, stream=s):
        ap.apply_into(dens, out, s)
    graph = rt.cudaGraph_t(init_value=g.raw_cuda_graph())
    err, _, n = rt.cudaGraphGetNodes(graph, 0)
    err, nodes, n = rt.cudaGraphGetNodes(graph, n)
    kinds = [rt.cudaGraphNodeGetType(nd)[1] for nd in nodes[:n]]
    del g
    return sum(1 for k in kinds if k == rt.cudaGraphNodeType.cudaGraphNodeTypeKernel)


def measure_fp64_peak(torch, dev):
    """Dense float64 GEMM (cuBLAS, 8192^3) on this GPU, best of 5: the FP64 roofline
    denominator (the driver's measured peaks hold the HBM copy and bf16 GEMM only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def ncu_traffic(workload, kernel, units):
    """DRAM bytes of one launch of ``kernel`` scaled from the committed ncu capture of a
    smaller case by the ratio of work units (``profiles/ncu_dram_bytes.json``)."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_dram_bytes.json")) as f:
            e = json.load(f)[workload][kernel]
        return e["bytes"] * units / e["units"], e["case"]
    except (OSError, ValueError, KeyError, ZeroDivisionError):
        return None, None


# stage entry -> (kernel symbol of its main launch, argument names)
STAGES = {
    "form_multipoles": ("k_h3_p2e<0>", ("strengths", "mpoles")),
    "coarsen_multipoles": ("k_trans_mv (M2M)", ("mpoles",)),
    "multipole_to_local": ("k_h3_m2l_bulk", ("mpoles", "locals", "err")),
    "form_locals": ("k_h3_p2e<1>", ("strengths", "locals", "err")),
    "refine_locals": ("k_trans_mv (L2L)", ("locals",)),
    "translate_box_multipoles_to_qbx_local": ("k_h3_m2qbxl_pair", ("mpoles", "qbx_exps", "err")),
    "translate_box_local_to_qbx_local": ("k_h3_l2qbxl", ("locals", "qbx_exps")),
    "eval_target_specific_qbx_locals": ("k_h3_tsqbx", ("strengths", "pot_tree", "err")),
    "eval_qbx_expansions": ("k_h3_qbxl2p", ("qbx_exps", "pot_tree")),
}


def stage_times(torch, ap, steps, flush, names=STAGES):
    """Each stage entry of the apply timed alone (CUDA events, L2 flushed), on the
    workspace the last apply left."""
    st = torch.cuda.current_stream()
    S = ctypes.c_void_p(st.cuda_stream)
    ws = ap.ws
    bufs = {"strengths": ctypes.c_void_p(ws.strengths), "mpoles": ctypes.c_void_p(ws.mpoles),
            "locals": ctypes.c_void_p(ws.locals), "qbx_exps": ctypes.c_void_p(ws.qbx_exps),
            "pot_tree": ctypes.c_void_p(ws.pot_tree), "err": ws.error_word}
    out = {}
    for name, (_, args) in names.items():
        fn = (lambda n=name, a=args: ap.plan.call("qbxfmm_" + n, *[bufs[x] for x in a], S))
        out[name] = statistics.mean(time_calls(torch, fn, steps, flush))
    return out

# }}}


def cpu_checker_sample(threads, reps=1):
    """The CPU checker (C/OpenMP float64, all host threads) on the bounded sample of
    the headline workload: the same operator, wave number and orders on the
    icosphere-2 surface (320 triangles, 4800 nodes, 14400 sources) with one of the
    densities; host-built geometry (no CUDA code is loaded)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle.oracle import Oracle
    wl = h3_workload(H3_SAMPLE["nrefine"], nrhs=H3_SAMPLE["nrhs"])
    geo = wl.geometry(builders="host")
    sp = wl.spec
    o = Oracle(geo, dim=3, qbx_order=wl.qbx_order, fmm_order=wl.fmm_order, nrhs=wl.nrhs,
               charge_coeff=sp.charge_coeff, dipole_coeff=sp.dipole_coeff,
               family=sp.kernel.family, k=sp.wave_number)
    s = wl.tree_strengths()
    out, times = None, []
    for _ in range(reps):
        t0 = time.perf_counter()
        out = o.apply(s)
        times.append(time.perf_counter() - t0)
    return wl, out, times


def reference_near_field_sample(wl, threads):
    """The reference's own compiled target-specific QBX module
    (pytential/qbx/target_specific, built from its sources into oracle/_ref) on the
    near field of the CPU sample: every (QBX target, list-1 source) pair of the
    icosphere-2 surface for D - ik S at the headline's k and qbx_order, one density, all
    host threads (its OpenMP loop).  That module truncates the 3D Helmholtz series in
    spherical waves (the reference's fmmlib form); the pair work is the same as the
    near field of the headline's sumpy truncation.  None when the module is not
    built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    try:
        import impl
    except ImportError:
        return None
    from pytential_b200 import abi, costs
    os.environ["OMP_NUM_THREADS"] = str(threads)
    geo = wl.geometry(builders="host")
    scal, A = abi.geometry_arrays(geo)
    s = wl.tree_strengths()[0].astype(complex)
    sp = wl.spec
    charges = complex(sp.charge_coeff) * s
    dipoles = complex(sp.dipole_coeff) * s
    pot = np.zeros(scal["ntargets"], complex)
    grad = np.zeros((3, scal["ntargets"]), complex)

    def run():
        pot[:] = 0
        impl.eval_target_specific_qbx_locals(
            1, 0, 1, 1, wl.qbx_order, A["sources"], A["targets"], A["centers"],
            A["global_qbx_centers"], A["qbx_center_to_target_box"],
            A["center_to_targets_starts"], A["center_to_targets_lists"], A["list1_starts"],
            A["list1_lists"], A["box_source_starts"], A["box_source_counts_nonchild"],
            complex(sp.wave_number), charges, dipoles, A["source_normals"], pot, grad)
    run()
    t0 = time.perf_counter()
    run()
    dt = time.perf_counter() - t0
    pairs = costs.tsqbx_pairs(A, scal)
    return {"kind": "reference", "cores": threads, "ms": 1e3 * dt, "pairs": int(pairs),
            "pairs_per_s": pairs / dt,
            "sample": "the 3D Helmholtz near field (D - ik S, k 10, qbx_order 5) of every "
                      "QBX target over its center's list-1 sources, icosphere-2 ellipsoid "
                      "(14400 sources), one density, by the reference's compiled "
                      "target-specific module (spherical-wave truncation)"}


SAMPLE_TEXT = ("the full apply of the same operator (D - ik S, k 10, qbx_order 5, fmm_order "
               "15) on the icosphere-2 ellipsoid (320 tri, 4800 nodes -> 14400 sources) with "
               "one of the 16 densities, scaled to node-applies/s")


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's apply (the reference's
    pyopencl/sumpy path cannot be installed here), all host threads, one bounded
    sample per step."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    threads = os.cpu_count() or 1
    wl, _, _ = cpu_checker_sample(threads, reps=max(args.warmup, 0))
    _, _, times = cpu_checker_sample(threads, reps=max(args.steps, 1))
    t = statistics.mean(times)
    value = wl.nuser_targets * wl.nrhs / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded analytic geometry and plane-wave densities)",
        "config": config_dict(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": SAMPLE_TEXT},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def laplace_leg(torch, dev, steps, warmup, flush, fp64_peak, cpu):
    """The 3D Laplace double-layer apply (ellipsoid, icosphere-3, 57600 sources, 19200
    surface + 2000 shell targets, q 3 / p 10), FP64 and mixed, timed like the headline."""
    from pytential_b200 import costs
    from pytential_b200.fmm import PRECISION_MIXED, QBXApply
    from pytential_b200.workloads import laplace3d_ellipsoid
    wl = laplace3d_ellipsoid(nrefine=L3["nrefine"], op=L3["op"], qbx_order=L3["qbx_order"],
                             fmm_order=L3["fmm_order"])
    geo = wl.geometry()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, device=dev, target_specific_qbx=True)
    apm = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, device=dev,
                   device_geometry=ap.dgeo, target_specific_qbx=True, precision=PRECISION_MIXED)
    dens = torch.from_numpy(wl.density).to(dev)
    out, outm = ap.new_output(), apm.new_output()
    for _ in range(warmup):
        ap.apply_into(dens, out)
        apm.apply_into(dens, outm)
    ms = statistics.mean(time_calls(torch, lambda: ap.apply_into(dens, out), steps, flush))
    msm = statistics.mean(time_calls(torch, lambda: apm.apply_into(dens, outm), steps, flush))
    ap.check_error_word()
    apm.check_error_word()
    # (its M2L runs as translation-class matrix products inside the apply, not through
    # the per-pair stage entry, so it is not timed alone here)
    names = {k: v for k, v in STAGES.items() if k in (
        "translate_box_multipoles_to_qbx_local", "form_locals",
        "eval_target_specific_qbx_locals")}
    kt = stage_times(torch, ap, steps, flush, names)
    ap.apply_into(dens, out)
    res, resm = out.cpu().numpy(), outm.cpu().numpy()
    scal, arr = ap.dgeo.scalars, ap.dgeo.host_arrays
    alg = costs.algorithmic_flops(arr, scal, 3, False, wl.fmm_order, wl.qbx_order, wl.nrhs)
    dom = max(kt, key=kt.get)
    nodes = wl.nuser_targets * wl.nrhs
    d = {"workload": "3D Laplace double layer, ellipsoid (1,1.5,2), icosphere-3 (1280 tri), "
                     "19200 nodes -> 57600 sources, 19200 surface + 2000 shell targets, "
                     "qbx_order 3, fmm_order 10, FP64, target-specific near field",
         "value": nodes * 1e3 / ms, "unit": UNIT, "ms_per_step": ms,
         "mixed": {"value": nodes * 1e3 / msm, "ms_per_step": msm, "speedup_vs_fp64": ms / msm,
                   "rel_err_vs_fp64_gpu": float(np.abs(resm - res).max() / np.abs(res).max())},
         "dominant_kernel": {"stage": dom, "ms": kt[dom], "algorithmic_flops": alg[dom],
                             "tflops": alg[dom] / (kt[dom] * 1e-3) / 1e12,
                             "frac_of_fp64_peak": alg[dom] / (kt[dom] * 1e-3) / 1e12 / fp64_peak},
         "stages_ms": {k: round(v, 4) for k, v in kt.items()}}
    if cpu:
        from oracle.oracle import Oracle
        sp = wl.spec
        o = Oracle(geo, dim=3, qbx_order=wl.qbx_order, fmm_order=wl.fmm_order, nrhs=wl.nrhs,
                   charge_coeff=sp.charge_coeff, dipole_coeff=sp.dipole_coeff)
        t0 = time.perf_counter()
        ref = o.apply(wl.tree_strengths())
        d["cpu_checker_value"] = nodes / (time.perf_counter() - t0)
        d["rel_err_vs_fp64_oracle"] = float(np.abs(res - ref).max() / np.abs(ref).max())
        d["mixed"]["rel_err_vs_fp64_oracle"] = float(np.abs(resm - ref).max() / np.abs(ref).max())
    return d


def solve2d_leg(torch, dev):
    """The batched 2D Helmholtz Brakhage-Werner exterior Dirichlet solve (starfish,
    2048 x 16 nodes, k 20, q 5 / p 20, 64 plane-wave right-hand sides, GMRES to 1e-8,
    restart 50, all densities through one apply per iteration): one warm-up solve,
    then a timed solve (CUDA events around the whole solve), one apply timed alone,
    and the largest true relative residual."""
    from pytential_b200.fmm import QBXApply
    from pytential_b200.gmres import gmres
    from pytential_b200.workloads import helmholtz2d_starfish
    wl = helmholtz2d_starfish(nelements=2048, nrhs=64)
    ap = QBXApply(wl.geometry(), wl.spec, wl.qbx_order, wl.fmm_order, nrhs=wl.nrhs, device=dev)
    b = torch.from_numpy(wl.density).to(dev)
    napply = [0]

    def op(X):
        napply[0] += 1
        return ap(X).clone()
    gmres(op, b, tol=1e-8, restart=50, maxiter=300)
    napply[0] = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    res = gmres(op, b, tol=1e-8, restart=50, maxiter=300)
    e1.record()
    torch.cuda.synchronize()
    solve_ms = e0.elapsed_time(e1)
    out = ap.new_output()
    apply_ms = statistics.mean(time_calls(torch, lambda: ap.apply_into(b, out), 5,
                                          torch.empty(64 * 1024 * 1024, dtype=torch.float32,
                                                      device=dev)))
    r = b - ap(res.solution)
    rel = float((torch.linalg.norm(r, dim=1) / torch.linalg.norm(b, dim=1)).max())
    ap.check_error_word()
    return {"workload": "2D Helmholtz k 20 Brakhage-Werner D - ik S, starfish 2048 x 16 nodes "
                        "(32768 unknowns), 64 plane-wave right-hand sides, qbx_order 5, "
                        "fmm_order 20, GMRES to 1e-8 (restart 50), complex128",
            "solve_ms": solve_ms, "iterations": int(res.iteration_count),
            "applies": napply[0], "apply_ms": apply_ms,
            "max_true_relative_residual": rel, "converged": bool(res.success)}


def adjoint_leg(torch, dev):
    """The 3D Laplace single-layer adjoint (ellipsoid icosphere-4, 76800 nodes, 5000
    targets on the sphere of radius 3, q 4 / p 12): forward apply, the exact transpose
    over the apply's tree, the target gradient from the FMM, and forward + backward of
    J = |S sigma - g|^2 / 2 (density and target-position gradients), FP64 and the
    mixed form (FP32 far field, exchanged-tree adjoint); CUDA events, 5 calls each."""
    from pytential_b200.adjoint import FarFieldSingleLayer, single_layer
    from pytential_b200.fmm import PRECISION_MIXED
    from pytential_b200.workloads import laplace3d_adjoint
    w = laplace3d_adjoint(nrefine=4, ntargets=5000)
    sig0 = torch.from_numpy(w.sigma).to(dev)
    X0 = torch.from_numpy(w.targets).to(dev)
    g = torch.from_numpy(w.g(w.targets)).to(dev)
    r0 = torch.ones(w.targets.shape[1], dtype=torch.float64, device=dev)

    def timed(f):
        for _ in range(2):
            f()
        ev = _events(torch, 5)
        for a, b in ev:
            a.record()
            f()
            b.record()
        torch.cuda.synchronize()
        return statistics.mean(a.elapsed_time(b) for a, b in ev)

    out = {"workload": "3D Laplace single layer with adjoint, ellipsoid (1,1.5,2) icosphere-4 "
                       "(5120 tri), 76800 nodes -> 230400 sources, 5000 targets on the sphere "
                       "of radius 3, qbx_order 4, fmm_order 12"}
    ref = None
    for name, kw in (("fp64", {}), ("mixed", {"precision": PRECISION_MIXED})):
        op = FarFieldSingleLayer(w.discr, w.targets, w.qbx_order, w.fmm_order, device=dev, **kw)

        def fwd_bwd():
            sigma = sig0.clone().requires_grad_(True)
            X = X0.clone().requires_grad_(True)
            J = 0.5 * ((single_layer(op, sigma, X) - g) ** 2).sum()
            J.backward()
            return sigma.grad, X.grad
        d = {"adjoint_form": op.adjoint_form,
             "forward_ms": timed(lambda: op.apply(sig0)),
             "adjoint_ms": timed(lambda: op.adjoint(r0))}
        op.apply(sig0)
        d["target_gradient_ms"] = timed(lambda: op.target_gradient(sig0))
        d["forward_backward_ms"] = timed(fwd_bwd)
        gs, gx = fwd_bwd()
        if ref is None:
            ref = (gs, gx)
        else:
            d["rel_err_vs_fp64"] = {
                "density_gradient": float((gs - ref[0]).abs().max() / ref[0].abs().max()),
                "target_gradient": float((gx - ref[1]).abs().max() / ref[1].abs().max())}
        out[name] = d
    return out


def run_b200(args):
    import torch
    import torch.distributed as dist

    from pytential_b200 import costs
    from pytential_b200.fmm import PRECISION_MIXED, QBXApply
    from pytential_b200.sharding import all_gather_rhs, rhs_split

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # one job: the same 16 densities on every rank, each rank applies its share
    wl = h3_workload(args.nrefine)
    nrhs = wl.nrhs
    start, count = rhs_split(nrhs, world, rank)
    t0 = time.perf_counter()
    geo = wl.geometry()
    geo.traversal()
    geo.center_to_tree_targets()
    t_geo = time.perf_counter() - t0
    t0 = time.perf_counter()
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=count, device=dev,
                  target_specific_qbx=True)
    torch.cuda.synchronize()
    t_plan = time.perf_counter() - t0
    dens_all = torch.from_numpy(wl.density).to(dev)
    dens = dens_all[start:start + count].contiguous()
    out = ap.new_output()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    nodes_total = ap.nuser_targets * nrhs

    def step():
        ap.apply_into(dens, out)
        if world > 1:
            return all_gather_rhs(out, nrhs)
        return out

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    K = args.steps
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        step_ms = time_calls(torch, step, K, flush)
    barrier()
    t_max = max_over_ranks(sum(step_ms) / 1e3)
    value = nodes_total * K / t_max
    full = step().cpu().numpy()
    ap.check_error_word()
    launches = kernel_nodes(torch, ap, dens, out)

    # end to end through the host-buffer entry (H2D of this rank's densities, apply,
    # D2H of its potentials, sync), device-timed around each call
    ap.alloc_host_buffers()
    ap.h_in.copy_(torch.from_numpy(wl.density[start:start + count]))
    for _ in range(2):
        ap.apply_host()
    barrier()
    ev = _events(torch, K)
    for a, b in ev:
        a.record()
        ap.apply_host()
        b.record()
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1e3)
    e2e_value = nodes_total * K / t_e2e

    # the mixed-precision form on the same job
    mixed = {}
    try:
        apm = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, nrhs=count, device=dev,
                       device_geometry=ap.dgeo, target_specific_qbx=True,
                       precision=PRECISION_MIXED)
    except Exception as e:   # noqa: BLE001  (reported, not hidden)
        apm = None
        mixed = {"status": f"not available: {e}"}
    if apm is not None:
        outm = apm.new_output()
        for _ in range(max(args.warmup, 3)):
            apm.apply_into(dens, outm)
        barrier()
        msm = time_calls(torch, lambda: apm.apply_into(dens, outm), K, flush)
        tm = max_over_ranks(sum(msm) / 1e3)
        apm.check_error_word()
        resm = outm.cpu().numpy()
        resd = out.cpu().numpy()
        mixed = {"value": nodes_total * K / tm, "unit": UNIT, "ms_per_step": 1e3 * tm / K,
                 "speedup_vs_fp64": t_max / tm,
                 "rel_err_vs_fp64_gpu": max_over_ranks(
                     float(np.abs(resm - resd).max() / np.abs(resd).max()))}

    line = None
    if rank == 0:
        # each stage alone, the dominant one gives the roofline entry
        kt = stage_times(torch, ap, K, flush)
        scal, arr = ap.dgeo.scalars, ap.dgeo.host_arrays
        alg = costs.algorithmic_flops(arr, scal, 3, True, wl.fmm_order, wl.qbx_order, count)
        dom = max(kt, key=kt.get)
        fp64_peak = measure_fp64_peak(torch, dev)
        achieved = alg[dom] / (kt[dom] * 1e-3) / 1e12
        units = costs.m2qbxl_pairs(arr, scal) if dom.startswith("translate_box_mult") else None
        traffic, tcase = ncu_traffic("helmholtz3d", STAGES[dom][0], units) if units else (None, None)
        peaks = measured_peaks()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t_max / K,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic (seeded analytic geometry and plane-wave densities)",
            "config": config_dict(args, world),
            "roofline": {
                "kernel": f"{STAGES[dom][0]} ({dom})", "bound": "fp64",
                "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak,
                "peak_source": ("of measured: cuBLAS float64 GEMM 8192^3 on this GPU, best of 5 "
                                "(MEASURED_PEAKS.json holds no FP64 entry)"),
                "algorithmic_flops_per_launch": alg[dom],
                "algorithmic_count": "pytential_b200/costs.py algorithmic_flops",
                "kernel_ms": kt[dom], "share_of_step": kt[dom] / (1e3 * t_max / K),
                "traffic": traffic, "traffic_source": tcase,
                "stages_ms": {k: round(v, 3) for k, v in kt.items()},
                "stages_tflops_algorithmic": {
                    k: round(alg[k] / (kt[k] * 1e-3) / 1e12, 3) for k in kt},
                # sum over the stages of their algorithmic bound over the step time; the
                # algorithmic M2L count is the dense C_f^2 product, more than the
                # rotation-based translation performs, so that stage can exceed 1
                "apply": costs.apply_roofline(
                    kt, alg, costs.stage_hbm_bytes(scal, 3, True, wl.fmm_order, count),
                    fp64_peak, peaks.get("hbm_gbs"), 1e3 * t_max / K)},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": ap.h2d_bytes * world,
                    "d2h_bytes_per_step": ap.d2h_bytes * world},
            "gpu_launches": launches * K,
            "clocks": clk.summary(),
            "geometry_s": t_geo, "plan_and_precompute_s": t_plan,
            "hbm_peak_gbs": peaks.get("hbm_gbs"),
            "mixed": mixed,
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        swl, ref, times = cpu_checker_sample(threads, reps=1)
        cpu_t = statistics.mean(times)
        line["cpu_baseline"] = {"value": swl.nuser_targets * swl.nrhs / cpu_t, "unit": UNIT,
                                "cores": threads, "kind": "port", "sample": SAMPLE_TEXT}
        nf = reference_near_field_sample(swl, threads)
        if nf is not None:
            # the GPU's near field at the headline size, per (target, source) pair and
            # density, beside it
            arr, scal = ap.dgeo.host_arrays, ap.dgeo.scalars
            gpu_pairs = costs.tsqbx_pairs(arr, scal) * count
            ms = line["roofline"]["stages_ms"].get("eval_target_specific_qbx_locals")
            if ms:
                nf["gpu_pairs_per_s"] = gpu_pairs / (ms * 1e-3)
            line["cpu_baseline"]["reference_near_field"] = nf
        # parity spot check on the sample: the GPU forms against the checker
        sap = QBXApply(swl.geometry(), swl.spec, swl.qbx_order, swl.fmm_order, nrhs=swl.nrhs,
                       device=dev, target_specific_qbx=True)
        got = sap(torch.from_numpy(swl.density).to(dev)).cpu().numpy()
        line["rel_err_vs_fp64_oracle_sample"] = float(np.abs(got - ref).max() / np.abs(ref).max())
        if "value" in mixed:
            sapm = QBXApply(swl.geometry(), swl.spec, swl.qbx_order, swl.fmm_order,
                            nrhs=swl.nrhs, device=dev, device_geometry=sap.dgeo,
                            target_specific_qbx=True, precision=PRECISION_MIXED)
            gotm = sapm(torch.from_numpy(swl.density).to(dev)).cpu().numpy()
            mixed["rel_err_vs_fp64_oracle_sample"] = float(np.abs(gotm - ref).max()
                                                           / np.abs(ref).max())
    if world == 1 and not args.no_laplace:
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        line["laplace3d"] = laplace_leg(torch, dev, 20, 5, flush, line["roofline"]["peak"],
                                        cpu=not args.no_cpu_baseline)
    if world == 1 and not args.no_side_configs:
        line["helmholtz2d_solve"] = solve2d_leg(torch, dev)
        line["laplace3d_adjoint"] = adjoint_leg(torch, dev)
    del full
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
