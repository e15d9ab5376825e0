#!/usr/bin/env python
"""Benchmark of the batched local Hamiltonian (BigDFT's locham hot path).

Workload (the batched configuration): 256 normalised orbitals on one periodic
48^3 coarse grid (96^3 fine / ISF grid), hgrid 0.45 bohr, every coarse cell
carrying 1 scaling + 7 wavelet coefficients, local potential a sum of 4
Gaussians; seeded synthetic inputs.  One step = Hpsi, E_kin and E_pot of all
orbitals (FP32 convolutions, FP64 energies), the inputs already resident in
HBM.  The metric is coarse grid points processed per second (one point = one
coarse cell of one orbital).

Reported beside it: the plain FP64 GPU path (one kernel per 1D pass, the
reference OpenCL backend's structure) and the fused FP64 path on the same
workload, the FP32 energy error against FP64, per-kernel CUDA-event times, the
HBM and FP32-FMA rooflines of the dominant kernel, an end-to-end number
through the C ABI with host buffers, and the CPU oracle on the host cores.

Multi-GPU (torchrun): each rank holds its own 256 orbitals (orbital sharding,
weak scaling, as the reference distributes orbitals over MPI ranks) and the
per-step energies are summed with an all-reduce, like
calculate_energy_and_gradient's fmpi_allreduce (hpsiortho.f90:1572).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "bigdft-suite_b200"))

METRIC = "Hψ coarse pts/s FP32-batched vs FP64 plain (≤1e-6 Ha); serve p50/p99 ms"
UNIT = "coarse pts/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="wvlh", choices=["wvlh", "reference"])
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--norb", type=int, default=256)
    ap.add_argument("--no-extras", action="store_true", help="skip comparator / e2e / cpu legs")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [l.split(",") for l in Path(self.f.name).read_text().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        load = [s for s in sm if smax and s > 0.3 * smax] or sm
        med = load[len(load) // 2] if load else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    import torch
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


def cpu_oracle_rate(n, budget_s=12.0, max_orb=32, seed=7):
    """Time the CPU oracle (the reference's Fortran chain restated in C, OpenMP
    on all host threads) on a bounded sample of orbitals of the same workload."""
    import numpy as np
    nthreads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    import oracle as O
    O.lib()
    from wvlh import workloads as W
    rng = np.random.default_rng(seed)
    lr = W.full_periodic(n, 0.45)
    pot = W.gaussian_potential(lr, rng)
    d = O.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    done, t0 = 0, time.perf_counter()
    while done < max_orb:
        psi = rng.uniform(-1, 1, lr.ncoeff)
        O.locham_per(d, lr.hgrid, psi[:lr.nvctr_c], psi[lr.nvctr_c:], pot)
        done += 1
        if time.perf_counter() - t0 > budget_s and done >= 2:
            break
    dt = time.perf_counter() - t0
    return done * lr.coarse_cells / dt, nthreads, "%d orbitals of %d^3 (periodic, FP64), %.1f s" % (done, n, dt)


def run_reference(args, ws, rank):
    """The reference arm: the reference's CPU algorithm (its Fortran
    convolution chain, restated in C as the oracle port; no Fortran compiler
    exists here) on the host cores, same metric and configuration."""
    if rank != 0:
        return
    n = args.n
    for _ in range(args.warmup):
        cpu_oracle_rate(n, budget_s=0.0, max_orb=1)
    t0 = time.perf_counter()
    rates = []
    for _ in range(args.steps):
        r, cores, sample = cpu_oracle_rate(n, budget_s=0.0, max_orb=2)
        rates.append(r)
    dt = time.perf_counter() - t0
    value = sum(rates) / len(rates)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded uniform coefficients, 4-Gaussian potential)",
            "config": {"workload": "batched periodic locham, %d^3 coarse, %d orbitals (each step: a 2-orbital "
                                   "sample scaled to coarse pts/s)" % (n, args.norb), "n_coarse": n,
                       "norb": args.norb, "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": "2 orbitals of %d^3 per step" % n},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    import torch
    ws, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import numpy as np

    from wvlh import workloads as W
    from wvlh._lib import lib
    from wvlh.batch import Batch, Context

    dev = torch.device("cuda", local)
    n, norb = args.n, args.norb
    lr = W.full_periodic(n, 0.45)
    rng = np.random.default_rng(1234 + rank)
    pot64 = torch.tensor(W.gaussian_potential(lr, rng), device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(1000 + rank)
    psi64 = torch.rand(norb, lr.ncoeff, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    psi64 /= psi64.norm(dim=1, keepdim=True)
    psi64 = psi64.reshape(-1).contiguous()
    psi32 = psi64.float()
    pot32 = pot64.float()
    ctx = Context(local)
    batch = Batch(ctx, [lr], np.zeros(norb, np.int32))
    hpsi32 = torch.empty_like(psi32)
    ek = torch.empty(norb, dtype=torch.float64, device=dev)
    ep = torch.empty(norb, dtype=torch.float64, device=dev)
    esum = torch.zeros(2, dtype=torch.float64, device=dev)
    pts_step = norb * lr.coarse_cells

    def step():
        batch.locham(psi32, pot32, hpsi32, ek, ep)
        if ws > 1:
            esum[0] = ek.sum()
            esum[1] = ep.sum()
            torch.distributed.all_reduce(esum)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(args.steps):
        step()
    e1.record(st)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if ws > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = t.item()
    value = ws * pts_step * args.steps / (ms * 1e-3)
    launches = 4 * args.steps

    extras = {}
    if rank == 0 and not args.no_extras:
        # per-kernel CUDA-event times on the library stream
        import ctypes as C
        lib().wvlh_ctx_enable_timing(ctx.h, 1)
        nt = 5
        for _ in range(nt):
            batch.locham(psi32, pot32, hpsi32, ek, ep)
        kms = (C.c_double * 4)()
        ncall = C.c_longlong()
        lib().wvlh_ctx_kernel_times(ctx.h, kms, C.byref(ncall))
        lib().wvlh_ctx_enable_timing(ctx.h, 0)
        kt = [kms[i] / ncall.value for i in range(4)]
        names = ["k1_plane_forward", "k2_zpencil", "k3_plane_backward", "k_reduce_energies"]
        npt = 8 * lr.coarse_cells  # fine points per orbital (96^3)
        B = 4
        kbytes = [3 * B * npt * norb, 4 * B * npt * norb + B * npt, 4 * B * npt * norb, 0]
        kflops = [128 * npt * norb, 252 * npt * norb, 254 * npt * norb, 0]
        dom = max(range(3), key=lambda i: kt[i])
        hbm, hbm_src = peaks()
        tf32 = C.c_double()
        lib().wvlh_measure_fma_peak(32, 20000, C.byref(tf32))
        ach = kbytes[dom] / (kt[dom] * 1e-3) / 1e9
        extras["roofline"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                              "traffic": None, "kernel": names[dom], "peak_source": hbm_src,
                              "algorithmic_bytes_per_launch": kbytes[dom]}
        fach = kflops[dom] / (kt[dom] * 1e-3) / 1e12
        extras["roofline_fma"] = {"bound": "fp32_fma", "achieved": fach, "peak": tf32.value, "unit": "TFLOP/s",
                                  "frac": fach / tf32.value, "kernel": names[dom],
                                  "peak_source": "measured (register FMA-chain probe)"}
        extras["kernels_ms"] = {nm: round(v, 4) for nm, v in zip(names, kt)}

        # comparators on the same workload: FP64 plain per-pass and FP64 fused
        h64 = torch.empty_like(psi64)
        ek64, ep64 = torch.empty_like(ek), torch.empty_like(ep)

        def timed(fn, reps):
            fn()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            for _ in range(reps):
                fn()
            b.record(st)
            torch.cuda.synchronize()
            return a.elapsed_time(b) / reps

        ms_plain = timed(lambda: batch.locham_plain(psi64, pot64, h64, ek64, ep64), 2)
        ekp, epp = ek64.clone(), ep64.clone()
        ms_f64 = timed(lambda: batch.locham(psi64, pot64, h64, ek64, ep64), 3)
        batch.locham(psi32, pot32, hpsi32, ek, ep)
        torch.cuda.synchronize()
        de = max((ek - ek64).abs().max().item(), (ep - ep64).abs().max().item())
        dplain = max((ekp - ek64).abs().max().item(), (epp - ep64).abs().max().item())
        extras["fp64_plain"] = {"value": pts_step / (ms_plain * 1e-3), "ms_per_step": ms_plain}
        extras["fp64_fused"] = {"value": pts_step / (ms_f64 * 1e-3), "ms_per_step": ms_f64}
        extras["speedup_vs_fp64_plain"] = (pts_step / (ms / args.steps * 1e-3)) / (pts_step / (ms_plain * 1e-3))
        extras["energy_err_ha"] = {"fp32_vs_fp64_max_per_orbital": de, "plain_vs_fused_fp64": dplain}
        del h64

        # end to end through the C ABI with pinned host buffers
        hp = torch.empty(psi32.numel(), dtype=torch.float32, pin_memory=True)
        hp.copy_(psi32.cpu())
        hv = torch.empty(pot32.numel(), dtype=torch.float32, pin_memory=True)
        hv.copy_(pot32.cpu())
        hh = torch.empty_like(hp).pin_memory()
        hek = torch.empty(norb, dtype=torch.float64).pin_memory()
        hep = torch.empty(norb, dtype=torch.float64).pin_memory()
        batch.locham_host(hp, hv, hh, hek, hep, 32)
        reps = max(2, min(args.steps, 5))
        t0 = time.perf_counter()
        for _ in range(reps):
            batch.locham_host(hp, hv, hh, hek, hep, 32)
        dt = (time.perf_counter() - t0) / reps
        extras["e2e"] = {"value": pts_step / dt, "unit": UNIT, "h2d_bytes_per_step": hp.numel() * 4 + hv.numel() * 4,
                         "d2h_bytes_per_step": hh.numel() * 4 + 2 * 8 * norb, "ms_per_step": dt * 1e3}
        if ws == 1:
            r, cores, sample = cpu_oracle_rate(n)
            extras["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded uniform(-1,1) coefficients normalised per orbital, 4-Gaussian potential)",
                "config": {"workload": "batched periodic locham: %d orbitals on one %d^3 coarse grid (%d^3 ISF), "
                                       "FP32 convolutions + FP64 energies" % (norb, n, 2 * n),
                           "n_coarse": n, "norb": norb, "hgrid": 0.45, "parallelism": "orbital shards x%d" % ws,
                           "l2": "inputs larger than L2 (%.0f MB of psi read + written per step)" %
                                 (psi32.numel() * 8 / 1e6)},
                "gpu_launches": launches, "clocks": clocks}
        line.update(extras)
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
