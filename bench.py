#!/usr/bin/env python
"""Benchmark of the B200 projection-step hot path.

Headline workload (one "step" = one pressure solve from a zero initial guess):
  256^3 cell-centred Poisson, h = 1/256, homogeneous Neumann on all faces, RHS = sum of 16 cosine
  modes cos(kx pi x) cos(ky pi y) cos(kz pi z) at cell centres x = (i+1/2)h with integer
  wavenumbers in 1..16 and N(0,1) amplitudes (seeded), mean removed; solved to a 1e-10
  relative RMS residual by FP32 V-cycles inside FP64 iterative refinement.  The plain FP64
  multigrid solve of the same system is timed beside it.  Synthetic data (no dataset).
Secondary lines in the same JSON object: the 64^3 FP32 solve to 1e-6 and 100 steps of the
128x128x64 FP32 Boussinesq (Rayleigh-Benard) flow.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Prints one JSON line on rank 0.  --impl reference times the CPU restatement of the
reference algorithm (FP32 FMG warm start + FP64 FMG, sol_mgpressuremixed3ddevd.cpp:79-100) on
the host cores instead.
"""
import argparse
import ctypes as C
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms to 1e-10 rel residual @256^3 (mixed vs FP64 MG), HBM GB/s, NS steps/s"
N_CFG3 = 256
TOL_REL = 1e-10


from opencurrent_b200 import _capi  # noqa: E402
from opencurrent_b200.workloads import config1_rhs, ensemble_sizes, fourier_rhs, interior, padded, rayleigh_benard  # noqa: E402


# --------------------------------------------------------------------------- clocks -----
class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------- helpers ----
def ir_alg_bytes(n, cycles, outer, ramp_iters=4):
    """Compulsory HBM bytes of the refinement solve with the split-layout FP32 inner solver
    (s = 4).  Per refinement step: `cycles` level-0 V-cycles (12.57 N s each, as in
    solve_alg_bytes); the right-hand side restricted down from a zero correction (b read, the
    coarse b written and its u cleared: (1 + 1/4) N_l s per level); the nested-iteration ramp
    (a prolongation that assigns, (1 + 1/8) N_l s, + ramp_iters red-black iterations of 3 N_l s
    on each level >= 1, and the assigning prolongation into level 0); x += e fused into the last
    prolongation (x read and written, 2N*8, and e not written back: - N s).  Plus the FP64
    residual + FP32 right-hand side per step and the initial residual (2N*8 + N*4 each)."""
    N = float(n) ** 3
    s = 4
    coarse = N / 7.0  # sum over levels >= 1
    ramp = 1.25 * N * s + 1.25 * coarse * s + (1.125 + 3 * ramp_iters) * coarse * s + 1.125 * N * s
    b = outer * (cycles * 12.57 * N * s + ramp + 2 * N * 8 - N * s)
    b += (outer + 1) * (2 * N * 8 + N * 4)
    return b


def solve_alg_bytes(n, s, vcycles, outer):
    """Compulsory HBM bytes of a multigrid solve: 12.57 N s per level-0 V-cycle (nu1 = nu2 = 2,
    no post-smooth on level 0: 10.25 N s on level 0, 16.25 N_l s on each coarser level), one FMG
    ramp (the cycles from the coarser levels, 12.57/7 N s) per FMG, and for the refinement solver
    per outer step the FP64 residual + FP32 right-hand side (2N*8 + N*4) and the update
    (2N*8 + N*4), plus the initial residual."""
    N = float(n) ** 3
    cycle = 12.57 * N * s
    ramps = max(outer, 1)
    b = vcycles * cycle + ramps * cycle / 7.0
    if outer:
        b += (outer + 1) * (2 * N * 8 + N * 4) + outer * (2 * N * 8 + N * 4)
    return b


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(name):
    """DRAM bytes per launch recorded from an ncu capture in profiles/<name>.md."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        txt = open(p).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def dist_setup(gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        # NCCL between the GPUs; gloo where there is no GPU (the host-side logic's tests)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=180))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_done(world):
    """After the last collective: every rank leaves the process group (no graph holds NCCL work)."""
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------- GPU arm ----
def run_gpu(args):
    import torch
    import opencurrent_b200 as ocu
    from opencurrent_b200 import _capi

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    lib = ocu.load()
    stream = torch.cuda.Stream()
    sh = C.c_void_p(stream.cuda_stream)

    n = N_CFG3
    h = 1.0 / n
    L = ocu.layout(n, n, n)
    b = fourier_rhs(n)
    rms_b = float(np.sqrt(np.mean(b ** 2)))
    tol = TOL_REL * rms_b
    host_rhs = torch.from_numpy(padded(b, L, np.float64)).pin_memory()
    host_out = torch.empty(int(L.allocated), dtype=torch.float64).pin_memory()

    rhs = ocu.Grid3DDevice(ocu.F64)
    rhs.init(n, n, n)
    rhs.copy_from_host(host_rhs.numpy())

    def make_solver(kind, rhs_grid=None):
        s = ocu.Sol_MultigridPressureMixed3DDeviceD("ir") if kind == "ir" else ocu.Sol_MultigridPressure3DDevice(ocu.F64)
        s.bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_NEUMANN, 0.0))
        s.ir_inner_cycles = args.ir_inner
        s.sweep_cells = args.sweep_cells
        s.initialize_storage(n, n, n, h, h, h, rhs if rhs_grid is None else rhs_grid)
        _capi.check(lib.ocu_mg_set_stream(s._h, sh))
        return s

    mixed = make_solver("ir")
    fp64 = make_solver("fp64")

    def one_solve(s):
        _capi.check(lib.ocu_grid_clear(s.pressure().handle, 0.0, sh))
        ok, res = s.solve(tol, 30)
        if not ok:
            raise RuntimeError(f"solve did not reach tolerance: residual {res / rms_b:.3e}")
        return res

    def timed(fn, steps, warmup, sampler=None):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        if sampler:
            sampler.__enter__()
            time.sleep(0.25)  # let the sampler emit before the timed region starts
        n0 = ocu.kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        n1 = ocu.kernel_launch_count()
        if sampler:
            sampler.__exit__(None, None, None)
        barrier(world)
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms, world), n1 - n0

    sampler = ClockSampler(local)
    res_holder = {}

    def mixed_step():
        res_holder["mixed"] = one_solve(mixed)

    ms_mixed, launches = timed(mixed_step, args.steps, args.warmup, sampler)
    st_mixed = mixed.stats
    ms_fp64, _ = timed(lambda: res_holder.__setitem__("fp64", one_solve(fp64)), args.steps, args.warmup)
    st_fp64 = fp64.stats

    # errors against an FP64 multigrid solution driven past the tolerance (the FP64 solver here,
    # bit-identical to the oracle's restatement and within 1e-15 of the reference's own device
    # solver in the GPU tests), all mean-removed: max relative and relative L2
    x_mixed = mixed.pressure().copy_to_host()
    x_fp64 = fp64.pressure().copy_to_host()
    _capi.check(lib.ocu_grid_clear(fp64.pressure().handle, 0.0, sh))
    ok_ref, res_ref = fp64.solve(1e-12 * rms_b, 40)
    x_ref = interior(fp64.pressure().copy_to_host(), L).copy()
    x_ref -= x_ref.mean()

    def errs(x):
        d = interior(x, L).copy()
        d -= d.mean()
        return (float(np.abs(d - x_ref).max() / np.abs(x_ref).max()),
                float(np.linalg.norm(d - x_ref) / np.linalg.norm(x_ref)))

    err_mixed, err_fp64 = errs(x_mixed), errs(x_fp64)

    # end to end through the public API with host buffers: H2D rhs, solve, D2H pressure
    def e2e_step():
        _capi.check(lib.ocu_grid_upload_async(rhs.handle, C.c_void_p(host_rhs.data_ptr()), sh))
        one_solve(mixed)
        _capi.check(lib.ocu_grid_download_async(mixed.pressure().handle, C.c_void_p(host_out.data_ptr()), sh))
        stream.synchronize()

    ms_e2e_serial, _ = timed(e2e_step, max(1, args.steps // 2), 1)
    bytes_grid = int(L.allocated) * 8

    # The same steps pipelined through the same API: two solvers alternate, and while step k
    # solves, step k+1's rhs goes up on one copy stream and step k-1's pressure comes down on
    # another (PCIe carries both directions at once).  Every step still uploads its rhs from
    # pinned host memory and downloads its pressure; the timed region runs from before the first
    # upload to after the last download.
    rhs2 = ocu.Grid3DDevice(ocu.F64)
    rhs2.init(n, n, n)
    mixed2 = make_solver("ir", rhs2)
    host_out2 = torch.empty(int(L.allocated), dtype=torch.float64).pin_memory()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    h_in, h_out = C.c_void_p(s_in.cuda_stream), C.c_void_p(s_out.cuda_stream)
    solvers, rhs_dev, outs = [mixed, mixed2], [rhs, rhs2], [host_out, host_out2]

    def e2e_pipelined(K):
        ev = lambda: torch.cuda.Event()  # noqa: E731
        ev_in, ev_solved, ev_out = [ev(), ev()], [ev(), ev()], [ev(), ev()]
        start = ev()
        start.record(stream)
        s_in.wait_event(start)
        s_out.wait_event(start)
        for j in (0, 1):
            ev_solved[j].record(stream)
            ev_out[j].record(s_out)
        _capi.check(lib.ocu_grid_upload_async(rhs_dev[0].handle, C.c_void_p(host_rhs.data_ptr()), h_in))
        ev_in[0].record(s_in)
        for k in range(K):
            j = k % 2
            if k + 1 < K:
                s_in.wait_event(ev_solved[1 - j])  # solver 1-j has finished reading its rhs
                _capi.check(lib.ocu_grid_upload_async(rhs_dev[1 - j].handle, C.c_void_p(host_rhs.data_ptr()), h_in))
                ev_in[1 - j].record(s_in)
            stream.wait_event(ev_in[j])
            stream.wait_event(ev_out[j])  # this solver's previous pressure has been downloaded
            res_holder["e2e"] = one_solve(solvers[j])
            ev_solved[j].record(stream)
            s_out.wait_event(ev_solved[j])
            _capi.check(lib.ocu_grid_download_async(solvers[j].pressure().handle,
                                                    C.c_void_p(outs[j].data_ptr()), h_out))
            ev_out[j].record(s_out)
        stream.wait_event(ev_out[0])
        stream.wait_event(ev_out[1])

    e2e_pipelined(2)  # warm-up: the second solver's graphs
    torch.cuda.synchronize()
    k_e2e = max(2, args.steps)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_pipelined(k_e2e)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / k_e2e, world)
    dist_done(world)  # the rest of this arm is per rank (rank 0's secondary lines)
    # the last step's pressure, downloaded inside the timed region, is the solution
    e2e_ok = bool(np.array_equal(outs[(k_e2e - 1) % 2].numpy(), x_mixed))

    # dominant kernel: the level-0 colour sweep of the refinement solver's split FP32 hierarchy
    # (k_chq_relax), launched as the V-cycles launch it: one colour reads the other colour's
    # array and its own u and b and writes its own u -- 2N*4 bytes, N = 256^3
    iters = 20
    mixed.relax(0, 2, 0, core=2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0 = ocu.kernel_launch_count()
    e0.record(stream)
    mixed.relax(0, iters, 0, core=2)
    e1.record(stream)
    torch.cuda.synchronize()
    per_iter = (ocu.kernel_launch_count() - c0) // iters
    ncell = n ** 3
    kernel_name, alg_bytes = "k_chq_relax (FP32 split-layout colour sweep) level 0 (256^3)", 2.0 * ncell * 4
    sweep_ms = e0.elapsed_time(e1) / (iters * per_iter)
    achieved = alg_bytes / (sweep_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic("chq_relax_f32_256cube.md")

    secondary = {}
    if rank == 0 and not args.skip_secondary:
        secondary = run_secondary(torch, ocu, _capi, lib, stream, sh)

    clocks = sampler.summary()
    if rank != 0:
        return None
    cpu = cpu_baseline_sample(args) if not args.skip_cpu else None
    line = {
        "metric": METRIC,
        "value": round(ms_mixed, 4),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_mixed, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32 V-cycles in fp64 refinement",
        "data": "synthetic",
        "config": {"workload": "mixed-precision Poisson solve 256^3 Neumann, 16 cosine modes, to 1e-10 rel RMS residual",
                   "grid": [n, n, n], "tolerance_rel": TOL_REL, "ir_inner_cycles": args.ir_inner,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2_policy": "inputs larger than L2 (rhs 145 MB FP64, levels 217 MB)"},
        "fp64_mg_ms": round(ms_fp64, 4),
        "speedup_mixed_vs_fp64": round(ms_fp64 / ms_mixed, 3),
        "mixed": {"outer_iterations": st_mixed.outer_iterations, "fp32_vcycles": st_mixed.vcycles,
                  "rel_residual": res_holder["mixed"] / rms_b,
                  "max_rel_err_vs_fp64_reference": err_mixed[0], "rel_l2_err_vs_fp64_reference": err_mixed[1],
                  "alg_gbs": round(ir_alg_bytes(n, args.ir_inner, st_mixed.outer_iterations)
                                   / (ms_mixed * 1e-3) / 1e9, 1)},
        "fp64": {"vcycles": st_fp64.vcycles, "rel_residual": res_holder["fp64"] / rms_b,
                 "max_rel_err_vs_fp64_reference": err_fp64[0], "rel_l2_err_vs_fp64_reference": err_fp64[1],
                 "alg_gbs": round(solve_alg_bytes(n, 8, st_fp64.vcycles, 0) / (ms_fp64 * 1e-3) / 1e9, 1)},
        "fp64_reference": {"solver": "FP64 multigrid of this library driven to 1e-12 relative",
                           "rel_residual": res_ref / rms_b, "converged": bool(ok_ref)},
        "roofline": {"bound": "hbm", "kernel": kernel_name,
                     "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": round(sweep_ms, 5)},
        "e2e": {"value": round(ms_e2e, 4), "unit": "ms", "h2d_bytes_per_step": bytes_grid,
                "d2h_bytes_per_step": bytes_grid, "steps": k_e2e,
                "mode": "pipelined: two solvers alternate; step k+1's rhs upload and step k-1's pressure "
                        "download run on two copy streams during step k's solve; first upload and last "
                        "download inside the timed region",
                "downloaded_equals_device_solution": e2e_ok,
                "serial_ms": round(ms_e2e_serial, 4)},
        "gpu_launches": int(launches),
        "gpu_launches_per_step": round(launches / args.steps, 1),
        "clocks": clocks,
        "secondary": secondary,
        "cpu_baseline": cpu,
    }
    return line


def run_secondary(torch, ocu, _capi, lib, stream, sh):
    out = {}
    # 64^3 FP32 pressure solve to 1e-6 relative (U[-1,1] seed 0)
    n = 64
    L = ocu.layout(n, n, n)
    b = config1_rhs(n)
    buf = padded(b, L, np.float32)
    rms = float(np.sqrt(np.mean(b.astype(np.float32).astype(np.float64) ** 2)))
    g = ocu.Grid3DDevice(ocu.F32)
    g.init(n, n, n)
    g.copy_from_host(buf)
    s = ocu.Sol_MultigridPressure3DDevice(ocu.F32)
    s.bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_NEUMANN, 0.0))
    s.initialize_storage(n, n, n, 1 / n, 1 / n, 1 / n, g)
    _capi.check(lib.ocu_mg_set_stream(s._h, sh))

    def solve64():
        _capi.check(lib.ocu_grid_clear(s.pressure().handle, 0.0, sh))
        ok, res = s.solve(1e-6 * rms, 20)
        assert ok
    for _ in range(3):
        solve64()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 10
    e0.record(stream)
    for _ in range(reps):
        solve64()
    e1.record(stream)
    torch.cuda.synchronize()
    out["fp32_64cube_solve_ms"] = round(e0.elapsed_time(e1) / reps, 4)
    out["fp32_64cube_vcycles"] = s.stats.vcycles

    # 100 steps of the 128x128x64 FP32 Boussinesq flow: the reference's projection (FP32
    # multigrid, which cannot reach the 1e-5 divergence target at Ra = 1e6 and retries from zero
    # every step), and the library option solving the pressure by FP32 V-cycles in FP64
    # refinement (every projection converged)
    def ns_run(mixed):
        pp = rayleigh_benard(ocu, 128, 128, 64)
        pp.mixed_pressure = mixed
        eq = ocu.Eqn_IncompressibleNS3D(ocu.F32)
        eq.set_parameters(pp)
        _capi.check(lib.ocu_ns_set_stream(eq._h, sh))
        for _ in range(3):
            eq.advance_one_step(eq.get_max_stable_timestep())
        torch.cuda.synchronize()
        e0.record(stream)
        steps = 100
        unconverged = 0
        for _ in range(steps):
            unconverged += 0 if eq.advance_one_step(eq.get_max_stable_timestep()) else 1
        e1.record(stream)
        torch.cuda.synchronize()
        return steps, e0.elapsed_time(e1), unconverged

    steps, ms, unconverged = ns_run(False)
    out["ns_128x128x64_fp32_steps_per_s"] = round(steps / (ms * 1e-3), 2)
    out["ns_ms_per_step"] = round(ms / steps, 4)
    out["ns_steps_projection_above_tol"] = unconverged
    steps, ms, unconverged = ns_run(True)
    out["ns_128x128x64_fp32_fp64_pressure_steps_per_s"] = round(steps / (ms * 1e-3), 2)
    out["ns_fp64_pressure_steps_projection_above_tol"] = unconverged
    out.update(run_coarray(torch, ocu, _capi, lib, stream, sh))
    out.update(run_ensemble(torch, ocu, stream, sh))
    out.update(run_persistent_ensemble(torch, ocu, stream, sh))
    out.update(run_differentiable(torch, ocu))
    return out


def run_coarray(torch, ocu, _capi, lib, stream, sh, n=256, images=2):
    """The headline FP64 solve (256^3 Neumann, 16 modes, to 1e-10 relative RMS residual) through
    the multi-image solver: `images` x-slabs on this one device, halo planes copied device to
    device after every ghost refresh, levels of at most 64^3 cells on image 0."""
    L = ocu.layout(n // images, n, n)
    b = fourier_rhs(n)
    rms = float(np.sqrt(np.mean(b ** 2)))
    nxl = n // images
    rhs = []
    for i in range(images):
        g = ocu.Grid3DDevice(ocu.F64)
        g.init(nxl, n, n)
        g.copy_from_host(padded(b[i * nxl:(i + 1) * nxl], L, np.float64))
        rhs.append(g)
    s = ocu.Sol_MultigridPressure3DDeviceCo(ocu.F64, images)
    s.bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_NEUMANN, 0.0))
    s.initialize_storage(nxl, n, n, 1.0 / n, 1.0 / n, 1.0 / n, rhs)
    _capi.check(lib.ocu_mg_set_stream(s._h, sh))

    def solve():
        for i in range(images):
            _capi.check(lib.ocu_grid_clear(s.co_pressure(i).handle, 0.0, sh))
        ok, res = s.solve(TOL_REL * rms, 30)
        if not ok:
            raise RuntimeError(f"multi-image solve did not reach tolerance: {res / rms:.3e}")
        return res
    for _ in range(2):
        solve()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record(stream)
    for _ in range(reps):
        res = solve()
    e1.record(stream)
    torch.cuda.synchronize()
    return {"coarray_256_fp64_images": images, "coarray_256_fp64_solve_ms": round(e0.elapsed_time(e1) / reps, 4),
            "coarray_256_fp64_vcycles": s.stats.vcycles, "coarray_256_fp64_rel_residual": res / rms,
            "coarray_256_fp64_cutoff_level": s.cutoff_level}


def run_differentiable(torch, ocu, n=96, steps=32, every=8, directions=8):
    """96^3 periodic flow: velocity = projected curl of a low-passed (|k| <= 8) N(0,1) vector
    potential, scalar = Gaussian blob (sigma 0.1), 32 steps of upwind advection + projection at
    CFL 0.5, loss = 1/2 |phi_32 - target blob|^2.  Times the FP32 forward + adjoint (checkpoints
    every 8 steps); checks the FP64 adjoint against central differences on 8 seeded directions
    and the FP32 gradient against the FP64 one."""
    from opencurrent_b200.autograd import AdvectProjectChain
    from opencurrent_b200.workloads import divergence_free_velocity, gaussian_blob
    u, v, w = divergence_free_velocity(n, seed=5, kmax=8)
    dt = 0.5 / n  # max |velocity| = 1
    rng = np.random.default_rng(6)
    c0, c1 = rng.uniform(0.3, 0.7, 3), rng.uniform(0.3, 0.7, 3)
    phi0, target = gaussian_blob(n, c0, 0.1), gaussian_blob(n, c1, 0.1)

    def setup(dtype, tol):
        ch = AdvectProjectChain((n, n, n), (1 / n,) * 3, steps, dt, checkpoint_every=every, dtype=dtype,
                                proj_tol=tol)
        ins = []
        for which, x in zip("uvwt", (u, v, w, phi0)):
            t = ch.empty(which)
            ch.interior(t, which).copy_(torch.from_numpy(x).to(t.dtype))
            ins.append(t)
        tgt = ch.empty("t")
        ch.interior(tgt, "t").copy_(torch.from_numpy(target).to(tgt.dtype))
        return ch, ins, tgt

    def loss_grad(ch, ins, tgt, grad=True):
        out = ch.forward(*ins)
        d = ch.interior(out, "t") - ch.interior(tgt, "t")
        loss = 0.5 * float((d.double() ** 2).sum())
        if not grad:
            return loss, None
        lam = ch.empty("t")
        ch.interior(lam, "t").copy_(d)
        return loss, ch.backward(lam)

    # projection tolerance (L-infinity of the pressure residual): 3e-5 is the tightest this FP32
    # flow reaches; at 1e-5 every projection stops at max_iter and retries from zero (2 x 16
    # cycles, 4.4x the chain's time) for the same gradient (9.1e-8 against 9.6e-8 relative to FP64)
    proj_tol32 = 3e-5
    ch32, in32, t32 = setup(ocu.F32, proj_tol32)
    loss_grad(ch32, in32, t32)  # warm-up (records the graphs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    _, g32 = loss_grad(ch32, in32, t32)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ch64, in64, t64 = setup(ocu.F64, 1e-11)
    _, g64 = loss_grad(ch64, in64, t64)
    num = sum(float(((a.double() - b) ** 2).sum()) for a, b in zip(g32, g64))
    den = sum(float((b ** 2).sum()) for b in g64)
    worst = 0.0
    drng = np.random.default_rng(8)
    eps = 1e-6
    for _ in range(directions):
        dirs = []
        for which in "uvw":
            d = ch64.empty(which)
            ch64.interior(d, which).copy_(torch.from_numpy(drng.standard_normal((n, n, n))))
            dirs.append(d)
        dirs.append(ch64.empty("t"))  # the derivative with respect to the initial velocity
        lp, _ = loss_grad(ch64, [x + eps * d for x, d in zip(in64, dirs)], t64, grad=False)
        lm, _ = loss_grad(ch64, [x - eps * d for x, d in zip(in64, dirs)], t64, grad=False)
        fd = (lp - lm) / (2 * eps)
        ad = sum(float((g * d).sum()) for g, d in zip(g64, dirs))
        worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-300))
    return {"adjoint_96cube_32steps_fp32_ms": round(ms, 2), "adjoint_proj_tol_fp32": proj_tol32,
            "adjoint_fd_max_rel_err_fp64": float(f"{worst:.3e}"),
            "adjoint_fp32_vs_fp64_grad_rel_l2": float(f"{(num / den) ** 0.5:.3e}")}


def run_ensemble(torch, ocu, stream, sh, count=512):
    """512 independent FP32 Neumann solves, sizes from {32,48,64,96}^3 (seed 1), rhs U[-1,1]
    mean-removed (seed 1000 + index), each to 1e-6 relative L2, as one ensemble: autotuned
    first (not timed), then timed from a zero guess."""
    sizes = ensemble_sizes(count, 1)
    dims = [(n, n, n) for n in sizes]
    ens = ocu.PressureEnsemble(ocu.F32, dims, [(1.0 / n,) * 3 for n in sizes])
    ens.set_stream(stream.cuda_stream)
    tols = []
    for m, n in enumerate(sizes):
        b = np.random.default_rng(1000 + m).uniform(-1.0, 1.0, (n, n, n))
        b -= b.mean()
        L = ocu.layout(n, n, n)
        ens.rhs(m).copy_from_host(padded(b, L, np.float32))
        tols.append(1e-6 * float(np.sqrt(np.mean(b ** 2))))
    ens.autotune(tols, 30)
    pressures = [ens.pressure(m) for m in range(count)]

    def zero():
        for g in pressures:
            _capi.check(ocu.load().ocu_grid_clear(g.handle, 0.0, sh))

    zero()
    ens.solve(tols, 30)  # graphs recorded
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps, total = 3, 0.0
    for _ in range(reps):
        zero()
        torch.cuda.synchronize()
        e0.record(stream)
        conv = ens.solve(tols, 30)
        e1.record(stream)
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1)
    ms = total / reps
    stats = [ens.member_stats(m) for m in range(count)]
    cycles = [st.vcycles for st in stats]
    # members left above their tolerance: how far (FP32 residual floor of the larger grids)
    ratios = [st.last_l2 / t for st, t in zip(stats, tols) if st.last_l2 >= t]
    # per member: (cycles + FMG ramp ~ 1/7 cycle) x 12.57 N s (one V-cycle's compulsory bytes)
    alg = sum((c + 1.0 / 7.0) * 12.57 * n ** 3 * 4 for c, n in zip(cycles, sizes))
    return {"ensemble_512_ms": round(ms, 3), "ensemble_members_converged": conv,
            "ensemble_alg_gbs": round(alg / (ms * 1e-3) / 1e9, 1),
            "ensemble_vcycles_mean": round(float(np.mean(cycles)), 2),
            "ensemble_unconverged_l2_over_tol": [round(min(ratios), 3), round(max(ratios), 3)] if ratios else None,
            "ensemble_classes": [{"n": c["dims"][0], "members": c["members"], "nu": [c["nu1"], c["nu2"]],
                                  "relax_block": list(c["relax_block"]), "tuned_ms": round(c["ms"], 3)}
                                 for c in ens.classes()]}


def run_persistent_ensemble(torch, ocu, stream, sh, count=512):
    """The same 512 members (sizes from {32,48,64,96}^3, seed 1; rhs U[-1,1] mean-removed, seed
    1000 + index; each to 1e-6 relative L2) solved by the persistent refinement ensemble: ONE
    kernel launch in which each block runs whole member solves (FP64 residual, FP32 split-layout
    multigrid corrections), autotuned first (not timed), then timed from a zero guess."""
    sizes = ensemble_sizes(count, 1)
    dims = [(n, n, n) for n in sizes]
    ens = ocu.PersistentEnsemble(dims, [(1.0 / n,) * 3 for n in sizes])
    ens.set_stream(stream.cuda_stream)
    tols = []
    for m, n in enumerate(sizes):
        b = np.random.default_rng(1000 + m).uniform(-1.0, 1.0, (n, n, n))
        b -= b.mean()
        L = ocu.layout(n, n, n)
        ens.rhs(m).copy_from_host(padded(b, L, np.float64))
        tols.append(1e-6 * float(np.sqrt(np.mean(b ** 2))))
    ens.autotune(tols)
    pressures = [ens.pressure(m) for m in range(count)]

    def zero():
        for g in pressures:
            _capi.check(ocu.load().ocu_grid_clear(g.handle, 0.0, sh))

    zero()
    ens.solve(tols)  # graph recorded
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps, total = 3, 0.0
    for _ in range(reps):
        zero()
        torch.cuda.synchronize()
        e0.record(stream)
        conv = ens.solve(tols)
        e1.record(stream)
        torch.cuda.synchronize()
        total += e0.elapsed_time(e1)
    ms = total / reps
    p = ens.params()
    stats = [ens.member_stats(m) for m in range(count)]
    corr = [st.corrections for st in stats]
    # per member and correction: the FP32 V-cycles (cycles + the nested-iteration ramp ~ 1/7
    # cycle) at 12.57 N 4 bytes each, the FP64 residual (x, b read, float r written: 20 N) and
    # x += e fused into the last prolongation (x read and written: 16 N; e not written back:
    # - 4 N); plus the final residual check
    alg = sum((c * ((p.cycles + 1.0 / 7.0) * 12.57 * 4 + 32) + 20) * n ** 3 for c, n in zip(corr, sizes))
    blocks, threads, scratch = ens.launch_shape()
    return {"pens_512_ms": round(ms, 3), "pens_members_converged": conv,
            "pens_alg_gbs": round(alg / (ms * 1e-3) / 1e9, 1),
            "pens_corrections_mean": round(float(np.mean(corr)), 2),
            "pens_max_rel_residual": float(f"{max(st.l2 / t for st, t in zip(stats, tols)) * 1e-6:.3e}"),
            "pens_tuning": {"threads": p.threads, "cycles": p.cycles, "nu": [p.nu1, p.nu2], "blocks": blocks,
                            "scratch_mb": round(scratch / 2 ** 20, 1)}}


# --------------------------------------------------------------------------- CPU arms ---
def cpu_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()


def cpu_solve_once(kind="mixed", threads=None):
    """One 256^3 solve by the oracle's restatement of the reference algorithm (OpenMP over
    `threads` host threads, all of them by default)."""
    from oracle import oracle_ctypes as O
    n = N_CFG3
    L = O.layout(n, n, n)
    b = fourier_rhs(n)
    rms = float(np.sqrt(np.mean(b ** 2)))
    rhs = padded(b, L, np.float64)
    prm = O.MGParams()
    prm.bc = O.bcset_all(4, 0.0)
    prm.nu1 = prm.nu2 = 2
    prm.convergence = 0x05
    O.lib().orc_ns_set_omp_threads(threads or cpu_threads())
    m = O.OracleMG(kind, prm, n, n, n, 1 / n, 1 / n, 1 / n, rhs, L)
    t0 = time.perf_counter()
    ok, res = m.solve(TOL_REL * rms, 30)
    ms = (time.perf_counter() - t0) * 1e3
    return ms, ok, res / rms


def cpu_baseline_sample(args):
    """All host cores, and one core -- the reference's host code is single-threaded."""
    ms, ok, rel = cpu_solve_once("mixed")
    ms1, ok1, _ = cpu_solve_once("mixed", threads=1)
    return {"value": round(ms, 1), "unit": "ms", "cores": cpu_threads(), "kind": "port",
            "sample": f"one full 256^3 solve to 1e-10 by the oracle's restatement of the reference mixed "
                      f"solver (FP32 FMG warm start + FP64 FMG), OpenMP, converged={bool(ok)}, rel={rel:.2e}",
            "one_core": {"value": round(ms1, 1), "unit": "ms", "cores": 1, "converged": bool(ok1)}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    for _ in range(args.warmup):
        cpu_solve_once("mixed")
    times = []
    for _ in range(args.steps):
        ms, ok, rel = cpu_solve_once("mixed")
        times.append(ms)
    v = float(np.mean(times))
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(v, 1),
        "unit": "ms",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(v, 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32 warm start + fp64 FMG",
        "data": "synthetic",
        "config": {"workload": "mixed-precision Poisson solve 256^3 Neumann, 16 cosine modes, to 1e-10 rel RMS residual",
                   "grid": [N_CFG3] * 3, "tolerance_rel": TOL_REL},
        "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": cpu_threads(), "kind": "port",
                         "sample": "full 256^3 solve per step, oracle restatement of the reference mixed solver"},
        "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_kernel_case(args):
    """A few launches of one hot kernel on a 256^3 FP32 hierarchy, for focused profiler captures
    (ncu -k <kernel> -c 1..3).  Level 1 is filled by a restriction first, so no FMG runs."""
    import torch
    import opencurrent_b200 as ocu

    if args.kernel_case == "chequer":
        # the refinement solver's split FP32 hierarchy at 256^3: colour sweeps of level 0, the
        # residual + restriction into level 1, the prolongation back
        n = N_CFG3
        L = ocu.layout(n, n, n)
        rhs = ocu.Grid3DDevice(ocu.F64)
        rhs.init(n, n, n)
        rhs.copy_from_host(padded(fourier_rhs(n), L, np.float64))
        s = ocu.Sol_MultigridPressureMixed3DDeviceD("ir")
        s.bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_NEUMANN, 0.0))
        s.initialize_storage(n, n, n, 1.0 / n, 1.0 / n, 1.0 / n, rhs)
        s.relax(0, 2, 0, core=2)
        s.restrict_residuals(0, 1, core=2)
        s.prolong(1, 0, core=2)
        s.synchronize()
        rms = float(np.sqrt(np.mean(fourier_rhs(n) ** 2)))
        s.solve(1e-10 * rms, 30)   # one whole solve: its coarse end runs the single-CTA kernel
        torch.cuda.synchronize()
        print(json.dumps({"kernel_case": "chequer", "grid": [n] * 3, "ok": True}), flush=True)
        return

    if args.kernel_case == "flow":
        # two steps of the Rayleigh-Benard flow on a 256x256x128 FP32 grid (each field 33.5 MB,
        # a kernel reads 3-7 of them: more than L2 holds)
        eq = ocu.Eqn_IncompressibleNS3D(ocu.F32)
        eq.set_parameters(rayleigh_benard(ocu, 256, 256, 128))
        for _ in range(2):
            eq.advance_one_step(eq.get_max_stable_timestep())
        torch.cuda.synchronize()
        print(json.dumps({"kernel_case": "flow", "grid": [256, 256, 128], "ok": True}), flush=True)
        return

    n = N_CFG3
    h = 1.0 / n
    L = ocu.layout(n, n, n)
    rhs = ocu.Grid3DDevice(ocu.F32)
    rhs.init(n, n, n)
    rhs.copy_from_host(padded(fourier_rhs(n), L, np.float32))
    s = ocu.Sol_MultigridPressure3DDevice(ocu.F32)
    s.bc = ocu.BoundaryConditionSet(ocu.BoundaryCondition(ocu.BC_NEUMANN, 0.0))
    s.initialize_storage(n, n, n, h, h, h, rhs)
    if args.kernel_case == "relax":
        s.relax(0, 3, 0)          # one pair of two-colour passes + one iteration of colour launches
    elif args.kernel_case == "prolong":
        s.relax(1, 1, 0)
        s.prolong(1, 0)
    elif args.kernel_case == "restrict":
        s.restrict_residuals(0, 1, norms=True)
    elif args.kernel_case == "tail":
        s.run_vcycles(1)          # one V-cycle: its coarse end is one k_coarse_tail_smem launch
    s.synchronize()
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": args.kernel_case, "grid": [n] * 3, "ok": True}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ir-inner", type=int, default=4)
    ap.add_argument("--sweep-cells", type=int, default=0,
                    help="levels with at least this many cells use the two-colour TMA pass (0 = off)")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-secondary", action="store_true")
    ap.add_argument("--kernel-case", choices=["relax", "prolong", "restrict", "tail", "flow", "chequer"],
                    help="run a few launches of one kernel on the 256^3 FP32 hierarchy, or two "
                         "256x256x128 flow steps (profiling)")
    args = ap.parse_args()
    if args.kernel_case:
        run_kernel_case(args)
        return
    line = run_reference(args) if args.impl == "reference" else run_gpu(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
