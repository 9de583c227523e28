#!/usr/bin/env python
"""Benchmark: QBX-FMM node-applies/s on the 3D Laplace double-layer ellipsoid apply.

Workload: ellipsoid (1, 1.5, 2) from an icosphere refined 3 times (1280 triangles),
15 nodes per triangle (19200 nodes) upsampled to 45 (57600 sources), double
layer, exterior limit on the surface plus 2000 targets in the shell
2.5 <= r <= 3.5, qbx_order 3, fmm_order 10, float64.  node-applies = user
targets x densities.  One step = one apply (upsample, weight, reorder, every FMM
stage, assembly) with the density resident in HBM; the L2 cache (126 MB) is
flushed between steps by writing a 256 MB buffer outside the per-step events.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 (launched by torch.distributed.run): every rank applies its own density on
its own GPU (weak scaling, no data-path collective); time is the max over ranks.
"""

from __future__ import annotations

import argparse
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
WORKLOAD = ("3D Laplace double-layer QBX apply, ellipsoid (1,1.5,2), icosphere-3 "
            "(1280 tri), 19200 nodes -> 57600 sources, 19200 surface + 2000 shell "
            "targets, qbx_order 3, fmm_order 10, FP64")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nrefine", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-helmholtz", action="store_true",
                    help="skip the 3D Helmholtz measurement reported beside the headline")
    return ap.parse_args()


def make_workload(nrefine, seed):
    from pytential_b200.workloads import laplace3d_ellipsoid
    return laplace3d_ellipsoid(nrefine=nrefine, op="D", seed=seed)


def config_dict(wl, args, extra=None):
    d = {"workload": WORKLOAD if args.nrefine == 3 else f"{wl.name} (reduced)",
         "nodes": wl.discr.ndofs, "sources": wl.discr.nquad,
         "user_targets": wl.nuser_targets, "nrhs": wl.nrhs,
         "qbx_order": wl.qbx_order, "fmm_order": wl.fmm_order,
         "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{args.gpus}"}
    if extra:
        d.update(extra)
    return d


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


KERNEL_SYMBOLS = {
    "target-specific near field (eval_target_specific_qbx_locals)": "k_tsqbx",
    "M2QBXL (translate_box_multipoles_to_qbx_local)": "k_m2qbxl",
    "P2L list 4 (form_locals)": "k_p2l",
    "P2QBXL (form_global_qbx_locals)": "k_p2qbxl",
}


def ncu_traffic(label):
    """DRAM bytes per launch of a kernel from the committed ncu capture summary
    (``profiles/ncu_dram_bytes.json``), or None."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                               "profiles", "ncu_dram_bytes.json")) as f:
            data = json.load(f)
        return data["bytes_per_launch"].get(KERNEL_SYMBOLS.get(label, ""))
    except (OSError, ValueError, KeyError):
        return None


def cpu_reference(wl, reps, threads):
    """The CPU checker's full apply (float64, OpenMP) on the host cores."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle.oracle import Oracle
    sp = wl.spec
    o = Oracle(wl.geometry(), dim=3, qbx_order=wl.qbx_order, fmm_order=wl.fmm_order,
               nrhs=wl.nrhs, charge_coeff=sp.charge_coeff, dipole_coeff=sp.dipole_coeff)
    s = wl.tree_strengths()
    o.apply(s)   # warm (page-in, thread pool)
    times = []
    out = None
    for _ in range(reps):
        t0 = time.perf_counter()
        out = o.apply(s)
        times.append(time.perf_counter() - t0)
    return out, times


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    wl = make_workload(args.nrefine, seed=0)
    _, times = cpu_reference(wl, max(args.steps, 1), threads)
    t = statistics.mean(times)
    value = wl.nuser_targets * wl.nrhs / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(wl, args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "full apply of the workload per step (C/OpenMP float64 "
                                   "restatement; the reference's pyopencl/sumpy apply is "
                                   "not installable here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    import torch.distributed as dist

    from pytential_b200 import costs
    from pytential_b200.fmm import QBXApply

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)

    wl = make_workload(args.nrefine, seed=rank)
    geo = wl.geometry()
    # fastest verified configuration: translation-class matrices on the FP64 tensor
    # cores and the target-specific near field (same truncation, tests/test_gpu_parity)
    ap = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, device=dev,
                  target_specific_qbx=True)
    dens = torch.from_numpy(wl.density).to(dev)
    out = ap.new_output()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    scal, arr = ap.dgeo.scalars, ap.dgeo.host_arrays
    launches_per_step = costs.apply_launch_count(
        scal, arr, matrices=ap.uses_translation_matrices, tsqbx=True)
    pairs = costs.p2qbxl_pairs(arr, scal)
    sp = wl.spec
    fpp = costs.p2qbxl_flops_per_pair(3, wl.qbx_order, sp.charge_coeff != 0,
                                      sp.dipole_coeff != 0)
    node_applies = wl.nuser_targets * wl.nrhs

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        ap.apply_into(dens, out)
    torch.cuda.synchronize()

    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(K):
            flush.zero_()
            ev[i][0].record()
            ap.apply_into(dens, out)
            ev[i][1].record()
        torch.cuda.synchronize()
    barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_local = sum(step_ms) / 1e3
    t_all = torch.tensor([t_local], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_all, op=dist.ReduceOp.MAX)
    t_max = float(t_all.item())
    value = world * node_applies * K / t_max

    # the main kernels timed alone on the same stream (flushed L2); the dominant one
    # gives the roofline entry
    import ctypes
    st = torch.cuda.current_stream()
    ws = ap.ws
    V = ctypes.c_void_p
    S = V(st.cuda_stream)
    ch, dp = sp.charge_coeff != 0, sp.dipole_coeff != 0
    kernels = {
        "target-specific near field (eval_target_specific_qbx_locals)": (
            lambda: ap.plan.call("qbxfmm_eval_target_specific_qbx_locals", V(ws.strengths),
                                 V(ws.pot_tree), ws.error_word, S),
            costs.tsqbx_pairs(arr, scal) * costs.tsqbx_flops_per_pair(3, wl.qbx_order, ch, dp)),
        "M2QBXL (translate_box_multipoles_to_qbx_local)": (
            lambda: ap.plan.call("qbxfmm_translate_box_multipoles_to_qbx_local", V(ws.mpoles),
                                 V(ws.qbx_exps), ws.error_word, S),
            costs.m2qbxl_pairs(arr, scal) * costs.m2qbxl_flops_per_pair(wl.fmm_order, wl.qbx_order)),
        "P2L list 4 (form_locals)": (
            lambda: ap.plan.call("qbxfmm_form_locals", V(ws.strengths), V(ws.locals),
                                 ws.error_word, S),
            costs.p2l_flops(arr, scal, wl.fmm_order, ch, dp)),
        "P2QBXL (form_global_qbx_locals)": (
            lambda: ap.plan.call("qbxfmm_form_global_qbx_locals", V(ws.strengths),
                                 V(ws.qbx_exps), ws.error_word, S),
            pairs * fpp),
    }
    ktimes = {}
    for name, (fn, fl) in kernels.items():
        kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(K)]
        for i in range(K):
            flush.zero_()
            kev[i][0].record()
            fn()
            kev[i][1].record()
        torch.cuda.synchronize()
        ktimes[name] = (statistics.mean(a.elapsed_time(b) for a, b in kev), fl)
    # P2QBXL is not part of this configuration's step (the target-specific kernel
    # replaces it); it is timed for reference only
    in_step = {k: v for k, v in ktimes.items() if not k.startswith("P2QBXL")}
    dom = max(in_step, key=lambda k: in_step[k][0])
    k_ms, k_flops = in_step[dom]
    traffic = ncu_traffic(dom)
    fp64_peak = measure_fp64_peak(torch, dev)

    # end to end through the public host-buffer entry (H2D + apply + D2H + sync)
    ap.alloc_host_buffers()
    ap.h_in.copy_(torch.from_numpy(wl.density))
    for _ in range(3):
        ap.apply_host()
    barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        ap.apply_host()
    t_e2e = time.perf_counter() - t0
    te = torch.tensor([t_e2e], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * node_applies * K / float(te.item())

    res_gpu = ap.h_out.numpy().copy()
    ap.check_error_word()

    # the mixed-precision form (FP32 far field, split-TF32 translations, FP64 QBX near
    # field) on the same workload, timed the same way
    from pytential_b200.fmm import PRECISION_MIXED
    apm = QBXApply(geo, wl.spec, wl.qbx_order, wl.fmm_order, device=dev,
                   device_geometry=ap.dgeo, target_specific_qbx=True, precision=PRECISION_MIXED)
    outm = apm.new_output()
    for _ in range(max(args.warmup, 3)):
        apm.apply_into(dens, outm)
    barrier()
    evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(K)]
    for i in range(K):
        flush.zero_()
        evm[i][0].record()
        apm.apply_into(dens, outm)
        evm[i][1].record()
    torch.cuda.synchronize()
    tm = torch.tensor([sum(a.elapsed_time(b) for a, b in evm) / 1e3], dtype=torch.float64,
                      device=dev)
    if world > 1:
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    tm = float(tm.item())
    res_mixed = outm.cpu().numpy()
    apm.check_error_word()

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t_max / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded analytic geometry and density)",
            "config": config_dict(wl, args, {
                "near_field": "target-specific (per target and list-1 source)",
                "translations": "translation-class matrices, FP64 tensor cores"}),
            "roofline": {
                "kernel": dom, "bound": "fp64",
                "achieved": k_flops / (k_ms * 1e-3) / 1e12,
                "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": (k_flops / (k_ms * 1e-3) / 1e12) / fp64_peak,
                "peak_source": "measured here: cuBLAS float64 GEMM 8192^3, best of 5",
                "algorithmic_flops_per_launch": k_flops, "kernel_ms": k_ms,
                "share_of_step": k_ms / (1e3 * t_max / K), "traffic": traffic,
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch, "
                                   "profiles/ncu_dram_bytes.json") if traffic else None,
                "kernels_ms": {k: round(v[0], 4) for k, v in ktimes.items()},
                "kernels_tflops": {k: round(v[1] / (v[0] * 1e-3) / 1e12, 3)
                                   for k, v in ktimes.items()}},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": ap.h2d_bytes, "d2h_bytes_per_step": ap.d2h_bytes},
            "gpu_launches": launches_per_step * K,
            "clocks": clk.summary(),
            "mixed": {
                "form": "FP32 P2M/P2L/M2QBXL, split-TF32 tensor-core M2L, FP64 M2M/L2L, "
                        "target-specific near field and point evaluations",
                "value": world * node_applies * K / tm, "unit": UNIT,
                "ms_per_step": 1e3 * tm / K, "speedup_vs_fp64": t_max / tm,
                "rel_err_vs_fp64_gpu": float(np.abs(res_mixed - res_gpu).max()
                                             / np.abs(res_gpu).max())},
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        ref, times = cpu_reference(wl, 2, threads)
        cpu_t = statistics.mean(times)
        line["cpu_baseline"] = {
            "value": node_applies / cpu_t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "2 full applies of the same workload (C/OpenMP float64 restatement)"}
        line["rel_err_vs_fp64_oracle"] = float(np.abs(res_gpu - ref).max() / np.abs(ref).max())
        line["mixed"]["rel_err_vs_fp64_oracle"] = float(np.abs(res_mixed - ref).max()
                                                        / np.abs(ref).max())
    if world == 1 and not args.no_helmholtz:
        line["helmholtz3d"] = helmholtz3d_leg(torch, dev)
    print(json.dumps(line), flush=True)


def helmholtz3d_leg(torch, dev, steps=3, warmup=3):
    """The 3D Helmholtz combined-field apply at full size (ellipsoid from an
    icosphere refined 5 times: 20480 triangles, 307200 nodes -> 921600 sources, k 10,
    16 plane-wave densities, qbx_order 5, fmm_order 15), timed like the headline step
    with CUDA events; its working set (several GB) exceeds the L2, so no flush.  The
    one-time geometry (host tree and traversal, target association on the GPU) and the
    plan with its translation tables are timed apart."""
    from pytential_b200.fmm import QBXApply
    from pytential_b200.workloads import helmholtz3d_ellipsoid
    w = helmholtz3d_ellipsoid(nrefine=5, nrhs=16)
    geo = w.geometry()
    t0 = time.perf_counter()
    geo.traversal()
    t_geo = time.perf_counter() - t0
    t0 = time.perf_counter()
    ap = QBXApply(geo, w.spec, w.qbx_order, w.fmm_order, nrhs=w.nrhs, device=dev,
                  target_specific_qbx=True)
    torch.cuda.synchronize()
    t_plan = time.perf_counter() - t0
    dens = torch.from_numpy(w.density).to(dev)
    out = ap.new_output()
    for _ in range(warmup):
        ap.apply_into(dens, out)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    for a, b in ev:
        a.record()
        ap.apply_into(dens, out)
        b.record()
    torch.cuda.synchronize()
    ap.check_error_word()
    ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    nodes = ap.nuser_targets * w.nrhs
    return {"workload": "3D Helmholtz combined field D - ik S, k 10, ellipsoid (1,1.5,2), "
                        "icosphere-5 (20480 tri), 307200 nodes -> 921600 sources, 16 RHS, "
                        "qbx_order 5, fmm_order 15, FP64, target-specific near field",
            "metric": METRIC, "unit": UNIT, "value": nodes * 1e3 / ms, "ms_per_step": ms,
            "steps": steps, "warmup": warmup, "node_applies_per_step": nodes,
            "tree_and_lists_s": t_geo, "plan_and_precompute_s": t_plan,
            "l2": "not flushed (working set several GB)"}


def measure_fp64_peak(torch, dev):
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


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
