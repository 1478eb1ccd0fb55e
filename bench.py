"""Benchmark: multigrid solves/s at 1e-6 relative residual on one B200 (per rank).

Workload (``--workload batch64``, default): 64 independent anisotropic potential problems
-div(sigma grad phi) = f on 64^3 cell-centred grids (seeded log-normal sigma per axis, log-std
1, 5^3 box-filtered; +1/-1 point dipole), each solved to ||b - A phi|| / ||b|| < 1e-6 by
conjugate gradients preconditioned with one V(2,2) weighted-Jacobi (omega = 2/3) cycle
(2x2x2 averaging restriction, nearest prolongation, coarsest 4^3), float32.  One step =
install the 64 operators (coefficient hierarchies), load, iterate to tolerance, fetch.

``value``  whole-job solves/s with inputs resident in HBM;
``e2e``    the same through the public API from pinned host buffers (sigma, f in; phi out);
``plain_solves_per_s``  the one-request-at-a-time float32 path (one slot, host polls);
``roofline``  the fine-level smoother kernel (dominant kernel), CUDA-event timed;
``cpu_baseline``  the multi-threaded CPU port of the same algorithm on a bounded sample.

``--impl reference`` times the CPU port (the stand-in for the reference's TensorFlow CPU
path, which cannot be installed here) on the same workload, rank 0 only.

Multi-GPU (torchrun): every rank solves its own 64 problems (replicas, no collective);
``value`` = all ranks' solves / max-over-ranks time.
"""
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

METRIC = "MG solves/s @1e-6 rel resid (64^3 anisotropic, batch of 64 per GPU)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="batch64")
    p.add_argument("--n", type=int, default=64)
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    return p.parse_args()


def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_inputs(pkg, n, batch, seed0):
    sig = np.empty((3, batch, n, n, n), np.float32)
    f = np.empty((batch, n, n, n), np.float32)
    for i in range(batch):
        s = pkg.problems.anisotropic_sigma((n, n, n), seed=seed0 + i, log_std=1.0)
        sig[:, i] = s
        f[i] = pkg.problems.dipole((n, n, n), seed=seed0 + i)
    return sig, f


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", "bench_clocks_%d.csv" % os.getpid())

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(pkg, sig, f, n, budget_s=20.0):
    """The CPU port on as many of the batch's problems as fit in ``budget_s``."""
    from oracle import cpu_port, mg as omg
    cores = cpu_port.threads()
    nl = len(omg.level_shapes((n, n, n)))
    done, t0 = 0, time.perf_counter()
    iters = []
    while done < f.shape[0]:
        ops = cpu_port.hierarchy(sig[:, done], nl)
        _, it = cpu_port.pcg_solve(ops, f[done], tol=1e-6)
        iters.append(it)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": "%d of the %d 64^3 problems (PCG-V(2,2), mean %.1f iterations), torch CPU "
                      "port of the oracle" % (done, f.shape[0], float(np.mean(iters)))}


def run_reference(args):
    rank, world, _ = dist_init(args)
    if rank != 0:
        return 0
    import __graft_entry__ as ge
    pkg = ge.load_package()
    n, batch = args.n, args.batch
    per_step = 4  # problems per step: a bounded sample of the workload
    sig, f = make_inputs(pkg, n, max(per_step, 1), 1000)
    from oracle import cpu_port, mg as omg
    cores = cpu_port.threads()
    nl = len(omg.level_shapes((n, n, n)))

    def step():
        for i in range(per_step):
            ops = cpu_port.hierarchy(sig[:, i], nl)
            cpu_port.pcg_solve(ops, f[i], tol=1e-6)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    v = per_step * args.steps / dt
    out = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "impl": "reference",
           "config": {"workload": "64^3 anisotropic PCG-V(2,2) to 1e-6", "n": n,
                      "sample_per_step": per_step},
           "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                            "sample": "%d problems per step" % per_step},
           "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import __graft_entry__ as ge
    rank, world, local = dist_init(args)
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    pkg = ge.load_package()
    L, M, ops = pkg._lib, pkg.multigrid, pkg.ops
    n, batch = args.n, args.batch
    dev = torch.device("cuda", local)
    sig_h, f_h = make_inputs(pkg, n, batch, 1000 + 100000 * rank)
    sig_pin = torch.from_numpy(sig_h).pin_memory()
    f_pin = torch.from_numpy(f_h).pin_memory()
    out_pin = torch.empty((batch, n, n, n), dtype=torch.float32).pin_memory()
    sig_d = sig_pin.to(dev)
    f_d = f_pin.to(dev)
    phi_d = torch.empty_like(f_d)
    cfg = M.SolverConfig(cycle="V", accel="cg", tol=1e-6, max_cycles=200, cycles_per_launch=4)
    h = M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=batch)
    stats_box = {}

    def solve_resident():
        h.set_operator(ops.Sigma7(sig_d[0], sig_d[1], sig_d[2]))
        st = L.lib().hfm_mg_solve(h._h, __import__("ctypes").c_void_p(f_d.data_ptr()),
                                  __import__("ctypes").c_void_p(phi_d.data_ptr()), h._stats,
                                  ops._stream())
        stats_box["st"] = st

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        if world > 1:
            t = torch.tensor([ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    for _ in range(args.warmup):
        solve_resident()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    l0 = L.lib().hfm_kernel_launch_count()
    ms = timed(solve_resident, args.steps)
    launches = (L.lib().hfm_kernel_launch_count() - l0) // max(args.steps, 1)
    clk = clocks.stop()
    st = [dict(status=s.status, cycles=s.cycles, rel=s.rel_resid) for s in h._stats]
    assert all(s["status"] == 0 for s in st), st
    value = batch * world / (ms / 1000.0)

    # end to end: pinned host sigma and f in, phi out, through the public API
    def solve_e2e():
        sig_d.copy_(sig_pin, non_blocking=True)
        f_d.copy_(f_pin, non_blocking=True)
        solve_resident()
        out_pin.copy_(phi_d, non_blocking=True)
    for _ in range(2):
        solve_e2e()
    ms_e2e = timed(solve_e2e, max(2, args.steps // 2))
    e2e = {"value": batch * world / (ms_e2e / 1000.0), "unit": "solves/s",
           "h2d_bytes_per_step": int(sig_pin.numel() * 4 + f_pin.numel() * 4),
           "d2h_bytes_per_step": int(out_pin.numel() * 4)}

    # plain path: one request at a time, one slot, float32
    hp = M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=1)
    n_plain = min(8, batch)

    def plain():
        for i in range(n_plain):
            hp.set_operator(ops.Sigma7(sig_d[0, i], sig_d[1, i], sig_d[2, i]))
            hp.solve(f_d[i:i + 1])
    plain()
    ms_plain = timed(plain, 1)
    plain_sps = n_plain / (ms_plain / 1000.0)
    hp.close()

    # roofline: the smoother on the batch's fine level (Sigma7 Jacobi, 24 B/cell), CUDA events
    op = ops.Sigma7(sig_d[0], sig_d[1], sig_d[2])
    x = torch.randn_like(f_d)
    y = torch.empty_like(f_d)
    s = op.struct()
    import ctypes as C
    stream = ops._stream()

    def sweep():
        L.call("hfm_op_jacobi", C.byref(s), C.c_void_p(x.data_ptr()), C.c_void_p(f_d.data_ptr()),
               C.c_void_p(y.data_ptr()), C.c_void_p(0), batch, n, n, n, 2.0 / 3.0, 1, 0, stream)
    for _ in range(5):
        sweep()
    reps = 20
    ms_sweep = timed(sweep, reps)
    cells = batch * n ** 3
    bytes_alg = 24 * cells
    achieved = bytes_alg / (ms_sweep / 1000.0) / 1e9
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak = float(peaks.get("hbm_gbs", 6650.0))
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": None,
                "kernel": "k_smooth<SIGMA7,float> (fine-level weighted Jacobi)",
                "bytes_per_launch": bytes_alg, "ms_per_launch": ms_sweep,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650"}
    h.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(pkg, sig_h, f_h, n)
    if rank == 0:
        out = {"metric": METRIC, "value": round(value, 3), "unit": "solves/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic",
               "config": {"workload": "batch of %d anisotropic %d^3 solves per GPU (log-std 1, dipole)" % (batch, n),
                          "solver": "PCG + V(2,2) Jacobi omega=2/3, avg restriction, nearest prolongation, coarsest 4^3",
                          "tol": 1e-6, "l2": "inputs larger than L2 (%.0f MB per GPU)" % (batch * n ** 3 * 40 / 1e6),
                          "parallelism": "replicas x%d" % world},
               "plain_solves_per_s": round(plain_sps, 3),
               "iterations": {"mean": float(np.mean([s["cycles"] for s in st])),
                              "max": int(max(s["cycles"] for s in st))},
               "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": int(launches),
               "clocks": clk}
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
