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
DATA = "synthetic (seeded uniform(-1,1) coefficients normalised per orbital, 4-Gaussian potential)"


def workload_config(n, norb, ngpu):
    """The workload both arms measure (the same dict in both lines)."""
    return {"workload": "batched periodic locham: %d orbitals on one %d^3 coarse grid (%d^3 ISF), hgrid 0.45, "
                        "4-Gaussian potential" % (norb, n, 2 * n),
            "n_coarse": n, "norb": norb, "hgrid": 0.45, "parallelism": "orbital shards x%d" % ngpu,
            "l2": "inputs larger than L2 (%.0f MB of FP32 psi read + written per step)" %
                  (norb * 8 * n ** 3 * 4 * 2 / 1e6)}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="wvlh", choices=["wvlh", "reference"])
    ap.add_argument("--n", type=int, default=48)
    ap.add_argument("--norb", type=int, default=256)
    ap.add_argument("--no-extras", action="store_true", help="skip comparator / e2e / cpu / other-row legs")
    ap.add_argument("--leg", default=None, choices=["free_bc", "precond", "overlap", "nlpsp", "psolver", "conv_check", "serve32", "serve64"],
                    help="run one extra leg alone (one GPU) and print its result as one JSON line")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region: samples
    every 50 ms with their timestamps; stop(window) keeps those taken between
    the host clock readings around the timed loop (all of them if none fall
    inside a very short region, which the result then says)."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
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
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self, window=None):
        import datetime
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
        rows = [[x.strip() for x in r] for r in rows]

        def stamp(r):
            try:
                return datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except (ValueError, IndexError):
                return None
        scope = "timed region"
        if window:
            inside = [r for r in rows if stamp(r) is not None and window[0] - 0.05 <= stamp(r) <= window[1] + 0.05]
            if inside:
                rows = inside
            else:
                scope = "whole run (timed region shorter than the sampling interval)"
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[2]))
                smax = float(r[3])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 6 + k and r[6 + k].lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm), "scope": scope}


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


def host_cpu():
    """Host CPU model, physical cores and usable hardware threads (from
    /proc/cpuinfo, as lscpu reports them)."""
    model, cores = None, set()
    phys = core = None
    try:
        for line in open("/proc/cpuinfo"):
            k, _, v = line.partition(":")
            k, v = k.strip(), v.strip()
            if k == "model name" and model is None:
                model = v
            elif k == "physical id":
                phys = v
            elif k == "core id":
                core = v
            elif not k and phys is not None:
                cores.add((phys, core))
                phys = core = None
        if phys is not None:
            cores.add((phys, core))
    except OSError:
        pass
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    ncores = min(len(cores), threads) if cores else threads
    return {"model": model, "physical_cores": ncores, "threads": threads}


def omp_threads():
    """OpenMP threads of the CPU legs: one per physical core (set before the
    oracle's OpenMP runtime starts)."""
    n = host_cpu()["physical_cores"]
    os.environ.setdefault("OMP_NUM_THREADS", str(n))
    return int(os.environ["OMP_NUM_THREADS"])


def cpu_oracle_rate(n, budget_s=12.0, max_orb=512, seed=7):
    """Time the CPU oracle (the reference's Fortran chain restated in C, OpenMP
    over one thread per physical core) on a bounded sample of orbitals of the
    same workload."""
    import numpy as np
    nthreads = omp_threads()
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
    cores = 1
    for _ in range(args.steps):
        r, cores, sample = cpu_oracle_rate(n, budget_s=0.0, max_orb=2)
        rates.append(r)
    dt = time.perf_counter() - t0
    value = sum(rates) / len(rates)
    cpu = host_cpu()
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": DATA, "config": workload_config(n, args.norb, args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "cpu_model": cpu["model"], "physical_cores": cpu["physical_cores"],
                             "sample": "each step: 2 orbitals of the %d-orbital %d^3 workload through the oracle "
                                       "(FP64, OpenMP over %d threads), coarse pts/s of the sample" %
                                       (args.norb, n, cores)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _timed(torch, fn, reps, stream=None):
    """Mean ms of fn over reps launches, CUDA events on the current stream, after one warm call."""
    fn()
    torch.cuda.synchronize()
    st = stream or torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        fn()
    b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def oracle_errors(lr_list, psi_rows, pot_rows, hpsi_rows, ekin, epot):
    """Error of sampled results against the CPU oracle (outside any timed
    region): Hpsi relative L2 (largest over the sample), largest |dE_kin| and
    |dE_pot| in Ha."""
    import numpy as np
    import oracle as O
    worst = {"hpsi_rel_l2": 0.0, "ekin_abs_ha": 0.0, "epot_abs_ha": 0.0}
    for lr, x, v, h, e1, e2 in zip(lr_list, psi_rows, pot_rows, hpsi_rows, ekin, epot):
        d = O.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
        hc, hf, rk, rp = O.locham(d, lr.hgrid, x[:lr.nvctr_c], x[lr.nvctr_c:], v)
        ref = np.concatenate([hc, hf])
        worst["hpsi_rel_l2"] = max(worst["hpsi_rel_l2"], float(np.linalg.norm(h - ref) / np.linalg.norm(ref)))
        worst["ekin_abs_ha"] = max(worst["ekin_abs_ha"], abs(float(e1) - rk))
        worst["epot_abs_ha"] = max(worst["epot_abs_ha"], abs(float(e2) - rp))
    worst["sample"] = len(psi_rows)
    return worst


def leg_exchanges(torch, ctx, batch, psi32, psi64, lr, norb, ws, dev, reps=5):
    """The two data-path exchanges of an SCF step on sharded orbitals, every
    rank taking part (NCCL): the density of this rank's orbitals summed over
    the ranks into z-slabs (reduce-scatter, communicate_density,
    sumrho.f90:219), and the overlap S of all orbitals through the
    orbital -> component all-to-all, the local FP64 tensor-core Gram matrix
    and the all-reduce of S (orthogonality.f90:2695).  Timed on the device
    with CUDA events, the max over ranks."""
    import torch.distributed as dist
    from wvlh.shard import overlap_sharded, reduce_density
    vol = (0.5 * lr.hgrid[0]) * (0.5 * lr.hgrid[1]) * (0.5 * lr.hgrid[2])
    hf = torch.full((norb,), 2.0 / vol, dtype=torch.float64, device=dev)
    rho = torch.zeros(lr.nisf, dtype=torch.float64, device=dev)
    P = psi64.view(norb, -1)
    res = {}
    for name, fn in (("density_reduce_scatter", lambda: (rho.zero_(), batch.locden(psi32, hf, rho),
                                                         reduce_density(rho, lr.isf, scatter=True))),
                     ("overlap_sharded", lambda: overlap_sharded(P, ctx=ctx))):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        t = torch.tensor([a.elapsed_time(b) / reps], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        res[name + "_ms"] = t.item()
    res["orbitals_per_rank"] = norb
    res["ranks"] = ws
    return res


def leg_free_regions(torch, ctx, dev, nlr=1024, seed=2):
    """Free-BC support functions of uneven size: nlr regions with coarse boxes
    uniform 20..40 per dimension (all cells coarse), fine ellipsoid of radius
    0.4 x the box, one normalised orbital and one Gaussian potential each, all
    in one fused launch sequence.  FP32 fused vs FP64 fused vs FP64 plain."""
    import numpy as np
    from wvlh import workloads as W
    from wvlh.batch import Batch
    rng = np.random.default_rng(seed)
    lrs = [W.free_sphere(tuple(int(v) for v in rng.integers(20, 41, 3)), 0.45) for _ in range(nlr)]
    off = np.cumsum([0] + [lr.nisf for lr in lrs[:-1]])
    b = Batch(ctx, lrs, np.arange(nlr, dtype=np.int32), off)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    psi64 = torch.rand(b.psi_size, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    lens = torch.tensor([lr.ncoeff for lr in lrs], device=dev)
    idx = torch.repeat_interleave(torch.arange(nlr, device=dev), lens)
    nrm = torch.zeros(nlr, dtype=torch.float64, device=dev).index_add_(0, idx, psi64 * psi64)
    psi64 /= nrm.sqrt()[idx]
    del idx
    pot64 = torch.cat([W.gaussian_potential_device(lr, rng, dev) for lr in lrs])
    psi32, pot32 = psi64.float(), pot64.float()
    cells = sum(lr.coarse_cells for lr in lrs)
    h32, h64 = torch.empty_like(psi32), torch.empty_like(psi64)
    e = torch.empty(4, nlr, dtype=torch.float64, device=dev)
    tuned = {nm: b.autotune(ps, pt, hh, e[0], e[1], reps=1)[0]
             for nm, ps, pt, hh in (("fp32", psi32, pot32, h32), ("fp64", psi64, pot64, h64))}
    ms32 = _timed(torch, lambda: b.locham(psi32, pot32, h32, e[0], e[1]), 5)
    # the same call captured once into a CUDA graph and replayed (one launch a step)
    gr = b.locham_graph(psi32, pot32, h32, e[0], e[1])
    ms32_graph = _timed(torch, gr.launch, 5)
    gr.close()
    ms64 = _timed(torch, lambda: b.locham(psi64, pot64, h64, e[2], e[3]), 3)
    de = max((e[0] - e[2]).abs().max().item(), (e[1] - e[3]).abs().max().item())
    ms_plain = _timed(torch, lambda: b.locham_plain(psi64, pot64, h64, e[2], e[3]), 1)
    # sampled regions against the oracle, both precisions
    err = {}
    sample = [0, nlr - 1]
    poff = np.concatenate([[0], np.cumsum([lr.nisf for lr in lrs])])
    rows = [psi64[b.psi_offset(o):b.psi_offset(o) + lrs[o].ncoeff].cpu().numpy() for o in sample]
    vrows = [pot64[poff[o]:poff[o + 1]].cpu().numpy() for o in sample]
    for nm, ps, pt, hh, k in (("fp32", psi32, pot32, h32, 0), ("fp64", psi64, pot64, h64, 2)):
        b.locham(ps, pt, hh, e[k], e[k + 1])
        torch.cuda.synchronize()
        hr = [hh[b.psi_offset(o):b.psi_offset(o) + lrs[o].ncoeff].double().cpu().numpy() for o in sample]
        err[nm] = oracle_errors([lrs[o] for o in sample], rows, vrows, hr, [e[k][o].item() for o in sample],
                                [e[k + 1][o].item() for o in sample])
    out = {"workload": "%d free-BC regions, coarse 20..40 per dim, fine ellipsoid 0.4, 1 orbital each" % nlr,
           "err_vs_oracle": err, "plane_threads_measured": tuned,
           "coarse_cells": int(cells), "fp32_fused": {"value": cells / (ms32 * 1e-3), "ms": ms32,
                                                      "graph_replay_ms": ms32_graph},
           "fp64_fused": {"value": cells / (ms64 * 1e-3), "ms": ms64},
           "fp64_plain": {"value": cells / (ms_plain * 1e-3), "ms": ms_plain},
           "speedup_fp32_vs_fp64_plain": ms_plain / ms32, "energy_err_ha_fp32_vs_fp64": de}
    b.close()
    return out


def leg_precond(torch, ctx, dev, n=40, norb=512, ncong=5, seed=3):
    """Preconditioner batch: norb orbitals on an n^3 periodic grid, ncong CG
    iterations of (T - eps_i + c) x = r_i (c = 0.5, eps_i uniform(-1, -0.1)),
    from x0 = b = r (seeded uniform); FP32 convolutions / FP64 dot products vs
    FP64, with the squared residual norms of both."""
    import numpy as np
    from wvlh import workloads as W
    from wvlh.batch import Batch
    lr = W.full_periodic(n, 0.45)
    b = Batch(ctx, [lr], np.zeros(norb, np.int32))
    rng = np.random.default_rng(seed)
    cprec = 0.5 - rng.uniform(-1.0, -0.1, norb)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    r64 = torch.rand(b.psi_size, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    r32 = r64.float()
    x64, x32 = torch.empty_like(r64), torch.empty_like(r32)
    res = {}

    def run(x, r):
        x.copy_(r)
        return b.precond(x, r, cprec, ncong)

    for nm, x, r in (("fp32", x32, r32), ("fp64", x64, r64)):
        # measured block size of the preconditioner's plane kernels (untimed)
        pick, by_size = b.autotune_precond(x, r, cprec, ncong, reps=1)
        zpick = b.block_sizes()["precond"]["z"][0 if nm == "fp32" else 1]
        ms = _timed(torch, lambda: run(x, r), 3)
        _, hist = run(x, r)
        torch.cuda.synchronize()
        res[nm] = {"ms": ms, "value": norb * lr.coarse_cells / (ms * 1e-3), "hist": hist.cpu().numpy(),
                   "plane_threads": pick, "z_threads": zpick, "ms_by_block_size": by_size}
    h32, h64 = res["fp32"].pop("hist"), res["fp64"].pop("hist")
    rel = np.abs(h32 - h64) / np.abs(h64)
    # two orbitals through the oracle's CG (x0 = b = r): x relative L2 and the
    # largest relative error of a squared residual norm, per precision
    import oracle as O
    d = O.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    hf = [0.5 * h for h in lr.hgrid]
    err = {"fp32": {"x_rel_l2": 0.0, "residual_norm2_rel": 0.0}, "fp64": {"x_rel_l2": 0.0, "residual_norm2_rel": 0.0}}
    for o in (0, norb - 1):
        sl = slice(b.psi_offset(o), b.psi_offset(o) + lr.ncoeff)
        rr = r64[sl].cpu().numpy()
        xr, rn = O.precond(d, hf, cprec[o], ncong, rr, rr)
        for nm, x, hist in (("fp32", x32, h32), ("fp64", x64, h64)):
            xo = x[sl].double().cpu().numpy()
            err[nm]["x_rel_l2"] = max(err[nm]["x_rel_l2"], float(np.linalg.norm(xo - xr) / np.linalg.norm(xr)))
            err[nm]["residual_norm2_rel"] = max(err[nm]["residual_norm2_rel"],
                                                float(np.max(np.abs(hist[:, o] - rn) / np.abs(rn))))
    out = {"workload": "%d orbitals, %d^3 periodic, %d CG iterations" % (norb, n, ncong),
           "fp32": res["fp32"], "fp64": res["fp64"],
           "speedup_fp32_vs_fp64": res["fp64"]["ms"] / res["fp32"]["ms"],
           "residual_norm2_mean_per_iter_fp64": [float(v) for v in h64.mean(axis=1)],
           "residual_norm2_max_rel_err_fp32_vs_fp64": float(rel.max()),
           "x_rel_l2_fp32_vs_fp64": float((x32.double() - x64).norm() / x64.norm()),
           "err_vs_oracle": err}
    b.close()
    return out


def leg_density(torch, batch, psi32, psi64, lr, norb, dev):
    """Density of the batched workload: rho(r) = sum_o 2/vol |psi_o(r)|^2 on the ISF grid."""
    vol = (0.5 * lr.hgrid[0]) * (0.5 * lr.hgrid[1]) * (0.5 * lr.hgrid[2])
    hf = torch.full((norb,), 2.0 / vol, dtype=torch.float64, device=dev)
    r32 = torch.zeros(lr.nisf, dtype=torch.float64, device=dev)
    r64 = torch.zeros_like(r32)

    def go(psi, rho):
        rho.zero_()
        batch.locden(psi, hf, rho)

    ms32 = _timed(torch, lambda: go(psi32, r32), 5)
    ms64 = _timed(torch, lambda: go(psi64, r64), 3)
    cells = norb * lr.coarse_cells
    q32, q64 = r32.sum().item() * vol, r64.sum().item() * vol
    # a 4-orbital density against the oracle, both precisions
    import numpy as np
    import oracle as O
    from wvlh.batch import Batch
    d = O.Desc(lr.n, lr.periodic, lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
    P64 = psi64.view(norb, -1)[:4]
    ref = np.zeros(lr.nisf)
    for o in range(4):
        x = P64[o].cpu().numpy()
        ref = O.locden(d, x[:lr.nvctr_c], x[lr.nvctr_c:], 2.0 / vol, ref)
    b4 = Batch(batch.ctx, [lr], np.zeros(4, np.int32))
    err = {}
    for nm, P in (("fp32", psi32.view(norb, -1)[:4]), ("fp64", P64)):
        r = torch.zeros(lr.nisf, dtype=torch.float64, device=dev)
        b4.locden(P.reshape(-1), hf[:4], r)
        torch.cuda.synchronize()
        err[nm] = {"rho_rel_l2": float(np.linalg.norm(r.cpu().numpy() - ref) / np.linalg.norm(ref)), "sample": 4}
    b4.close()
    return {"fp32": {"ms": ms32, "value": cells / (ms32 * 1e-3)}, "fp64": {"ms": ms64, "value": cells / (ms64 * 1e-3)},
            "err_vs_oracle": err,
            "rho_rel_l2_fp32_vs_fp64": ((r32 - r64).norm() / r64.norm()).item(), "charge_fp64": q64,
            "charge_err_fp32": abs(q32 - q64)}


def leg_overlap(torch, ctx, psi64, norb):
    """S = Psi Psi^T (norb x norb, FP64) on FP64 tensor cores vs cuBLAS DGEMM (torch.mm)."""
    from wvlh.ortho import overlap
    P = psi64.view(norb, -1)
    K = P.shape[1]
    S = torch.empty(norb, norb, dtype=torch.float64, device=P.device)
    ms = _timed(torch, lambda: overlap(ctx, P, S=S), 5)
    ms_cublas = _timed(torch, lambda: torch.mm(P, P.T), 5)
    ref = torch.mm(P, P.T)
    fl = norb * (norb + 1) * K
    out = {"ms": ms, "tflops": fl / (ms * 1e-3) / 1e12, "cublas_dgemm_ms": ms_cublas,
           "max_abs_vs_cublas": (S - ref).abs().max().item(), "flops_count": "norb(norb+1)K (SYRK)"}
    # the psi-sized products of the orthonormalisation on the panel apply,
    # against the cuBLAS calls they replace: Loewdin / subspace update (dense
    # M psi, 2 norb^2 K flop), Cholesky (L^-1 psi, triangular: norb^2 K flop;
    # cuBLAS TRSM with L through torch.linalg.solve_triangular)
    from wvlh.ortho import panel_apply
    g = torch.Generator(device=P.device)
    g.manual_seed(17)
    Mf = torch.rand(norb, norb, generator=g, dtype=torch.float64, device=P.device) - 0.5
    L = torch.linalg.cholesky(ref / K + torch.eye(norb, dtype=torch.float64, device=P.device))
    Linv = torch.linalg.solve_triangular(L, torch.eye(norb, dtype=torch.float64, device=P.device), upper=False)
    O = torch.empty_like(P)
    ms_dense = _timed(torch, lambda: panel_apply(ctx, Mf, P, out=O), 3)
    ms_dense_cublas = _timed(torch, lambda: torch.mm(Mf, P, out=O), 3)
    err_dense = (panel_apply(ctx, Mf, P, out=O) - torch.mm(Mf, P)).abs().max().item()
    ms_tri = _timed(torch, lambda: panel_apply(ctx, Linv, P, out=O, lower=True), 3)
    ms_trsm = _timed(torch, lambda: torch.linalg.solve_triangular(L, P, upper=False), 2)
    ms_sub = _timed(torch, lambda: panel_apply(ctx, Mf, P, out=O, alpha=-1.0, beta=1.0), 3)
    del O
    fd = 2.0 * norb * norb * K
    out["panel_apply"] = {"workload": "%d x %d FP64 matrix times the %d x %d orbital panel" % (norb, norb, norb, K),
                          "dense_ms": ms_dense, "dense_tflops": fd / (ms_dense * 1e-3) / 1e12,
                          "cublas_dgemm_ms": ms_dense_cublas, "max_abs_vs_cublas": err_dense,
                          "cholesky_trmm_ms": ms_tri, "cublas_trsm_ms": ms_trsm,
                          "subspace_update_ms": ms_sub}
    return out


def leg_nlpsp(torch, ctx, psi64, lr, norb, natoms=64, seed=21):
    """Nonlocal projectors on the batched workload's orbitals: natoms atoms at
    seeded positions, each with 4 projectors (one s, three p: the shape of an
    HGH pseudopotential with one radial function per l) on a coarse ball of
    radius 10 cells with a fine ball of radius 5 cells, symmetric seeded h.
    FP64, hpsi += V_nl psi and eproj per orbital; the oracle on a 2-orbital,
    8-atom sample is the CPU figure."""
    import numpy as np
    from wvlh.batch import Region
    from wvlh.keys import Locreg
    from wvlh.nlpsp import Projectors
    rng = np.random.default_rng(seed)
    N = tuple(lr.n)
    ax = [np.arange(n) for n in N[::-1]]
    z, y, x = np.meshgrid(*ax, indexing="ij")
    atoms = []
    for _ in range(natoms):
        c = rng.uniform(11, np.array(N) - 11)
        d2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
        plr = Locreg.from_masks(d2 <= 100.0, d2 <= 25.0, (0, 0, 0), (0.45, 0.45, 0.45))
        h = rng.uniform(-1, 1, (4, 4))
        atoms.append((plr, rng.uniform(-1, 1, (4, plr.ncoeff)), h + h.T))
    nl = Projectors(ctx, Region(ctx, lr), atoms)
    P = psi64.view(norb, -1)
    H = torch.zeros_like(P)
    ms = _timed(torch, lambda: nl.apply(P, H), 5)
    ncoef = sum(a[1].size for a in atoms)
    out = {"workload": "%d orbitals of 48^3, %d atoms x 4 projectors (ball radius 10 coarse / 5 fine)" % (norb, natoms),
           "ms": ms, "projector_values": int(ncoef),
           "orbital_atom_pairs_per_s": norb * natoms / (ms * 1e-3)}
    try:
        from oracle import nlpsp_apply
        sub = [((a[0].keyg_c, a[0].keyv_c, a[0].keyg_f, a[0].keyv_f), a[1], a[2]) for a in atoms[:8]]
        kw = (lr.keyg_c, lr.keyv_c, lr.keyg_f, lr.keyv_f)
        p2 = P[:2].cpu().numpy()
        t = time.perf_counter()
        nlpsp_apply(kw, p2, sub)
        dt = time.perf_counter() - t
        out["cpu_oracle_orbital_atom_pairs_per_s"] = 16 / dt
    except Exception as e:  # the oracle is optional on the bench box
        out["cpu_oracle"] = "unavailable: %s" % e
    nl.close()
    return out


def leg_psolver(torch, ctx, dev, n=96, h=0.225):
    """The potential step that follows the density, on the 96^3 ISF grid of
    the batched workload (seeded positive density, FP64): the Hartree
    potential, periodic (wvlh_psolver_periodic: cuFFT and the ISF kernel
    multiply) and free (wvlh_psolver_free: the density padded to 192^3, the
    kernel table built once and kept) and surface (x, z periodic, y free,
    padded to 192 along y) and wire (z periodic, x and y padded to 192), the
    Kohn-Sham potential V_H + V_ext +
    V_xc with its three energies (wvlh_ks_potential_periodic / _free) and the
    LDA alone (wvlh_xc_lda, 16 bytes a point), against the oracle's numpy
    restatement on the host."""
    import numpy as np
    from wvlh.psolver import (hartree_free, hartree_periodic, hartree_surface, hartree_wire, ks_potential_free,
                              ks_potential_periodic, xc_lda)
    rng = np.random.default_rng(5)
    rho_h = rng.uniform(1e-3, 1, (n, n, n))
    vext_h = rng.uniform(-1, 1, (n, n, n))
    rho = torch.tensor(rho_h, device=dev)
    vext = torch.tensor(vext_h, device=dev)
    pot = torch.empty_like(rho)
    hh = (h, h, h)
    ms = _timed(torch, lambda: hartree_periodic(ctx, rho, hh, pot=pot), 10)
    ks_ms = _timed(torch, lambda: ks_potential_periodic(ctx, rho, hh, vext=vext, pot=pot), 10)
    xc_ms = _timed(torch, lambda: xc_lda(ctx, rho, vxc=pot, dvol=h ** 3), 10)
    hartree_free(ctx, rho, hh, pot=pot)      # builds the free kernel and plans once
    free_ms = _timed(torch, lambda: hartree_free(ctx, rho, hh, pot=pot), 10)
    ks_free_ms = _timed(torch, lambda: ks_potential_free(ctx, rho, hh, vext=vext, pot=pot), 10)
    t = time.perf_counter()
    hartree_surface(ctx, rho, hh, pot=pot)   # builds the surface kernel table and plans once
    torch.cuda.synchronize()
    surf_setup_ms = (time.perf_counter() - t) * 1e3
    surf_ms = _timed(torch, lambda: hartree_surface(ctx, rho, hh, pot=pot), 10)
    t = time.perf_counter()
    hartree_wire(ctx, rho, hh, pot=pot)      # builds the wire kernel table and plans once
    torch.cuda.synchronize()
    wire_setup_ms = (time.perf_counter() - t) * 1e3
    wire_ms = _timed(torch, lambda: hartree_wire(ctx, rho, hh, pot=pot), 10)
    out = {"workload": "%d^3 grid, h %.3f bohr, FP64" % (n, h), "ms": ms,
           "ks_potential_ms": ks_ms, "xc_lda_ms": xc_ms,
           "xc_lda_gbs": 16.0 * n ** 3 / (xc_ms * 1e-3) / 1e9,
           "free_ms": free_ms, "ks_potential_free_ms": ks_free_ms,
           "surface_ms": surf_ms, "surface_setup_ms": surf_setup_ms,
           "wire_ms": wire_ms, "wire_setup_ms": wire_setup_ms}
    try:
        from oracle import ks_potential_periodic as ks_cpu
        from oracle import psolver_periodic
        t = time.perf_counter()
        psolver_periodic(rho_h, hh)
        out["cpu_oracle_ms"] = (time.perf_counter() - t) * 1e3
        t = time.perf_counter()
        ks_cpu(rho_h, hh, vext_h)
        out["cpu_oracle_ks_ms"] = (time.perf_counter() - t) * 1e3
        from oracle import psolver_free
        t = time.perf_counter()
        psolver_free(rho_h, hh)
        out["cpu_oracle_free_ms"] = (time.perf_counter() - t) * 1e3
    except Exception as e:  # the oracle is optional on the bench box
        out["cpu_oracle"] = "unavailable: %s" % e
    return out


# the reference's OpenCL conv_check run (bigdft/tests/libs/OpenCL/OpenCL.ref.yaml, fort.1 =
# "76 92 130 2", FP64): its published CPU / GPU milliseconds per operation, unnamed hardware
CONV_CHECK_REF = {
    "magicfilter1d 76 x 11960": (17.09, 3.82), "magicfilter1d_t 76 x 11960": (17.04, 3.80),
    "kinetic1d 76 x 11960": (151.47, 12.00), "ana1d 76 x 11960": (21.02, 4.48),
    "syn1d 76 x 11960": (21.99, 4.59), "magic_filter_3d 76x92x130": (48.25, 11.19),
    "magic_filter_t_3d 76x92x130": (50.33, 11.37), "potential_3d 76x92x130": (106.31, 23.76),
    "kinetic_3d 76x92x130": (149.56, 28.18), "ana_3d 76x92x130": (66.95, 13.50),
    "syn_3d 76x92x130": (67.50, 12.73),
}


def leg_conv_check(torch, reps=20):
    """The drop-in per-operation kernels (ocl_* ABI, FP64) on the sizes of the
    reference's conv_check benchmark, beside its published numbers."""
    import ctypes as C
    import numpy as np
    from wvlh import ocl
    q = ocl.OclQueue(0)
    n1, n2, n3 = 76, 92, 130
    npt = n1 * n2 * n3
    rng = np.random.default_rng(3)
    bufs = [q.buffer(8 * npt) for _ in range(6)]
    for b in bufs[:2]:
        q.write(b, rng.uniform(-1, 1, npt))
    a, b, t1, t2, w1, w2 = bufs
    dims = (ocl.u32 * 3)(n1 // 2, n2 // 2, n3 // 2)
    per = (ocl.u32 * 3)(1, 1, 1)
    h = (C.c_double * 3)(0.2, 0.2, 0.2)
    e = (C.c_double * 2)()
    c0 = C.c_double(0.0)
    h1 = C.c_double(0.2)
    ops = {
        "magicfilter1d 76 x 11960": ("magicfilter1d_d_", (ocl._u(n1), ocl._u(n2 * n3), a.ref, b.ref)),
        "magicfilter1d_t 76 x 11960": ("magicfilter1d_t_d_", (ocl._u(n1), ocl._u(n2 * n3), a.ref, b.ref)),
        "kinetic1d 76 x 11960": ("kinetic1d_d_", (ocl._u(n1), ocl._u(n2 * n3), C.byref(h1), C.byref(c0), a.ref,
                                                  b.ref, w1.ref, w2.ref, e)),
        "ana1d 76 x 11960": ("ana1d_d_", (ocl._u(n1 // 2), ocl._u(n2 * n3), a.ref, b.ref)),
        "syn1d 76 x 11960": ("syn1d_d_", (ocl._u(n1 // 2), ocl._u(n2 * n3), a.ref, b.ref)),
        "magic_filter_3d 76x92x130": ("magic_filter_3d_generic_", (dims, per, t1.ref, t2.ref, a.ref, b.ref)),
        "magic_filter_t_3d 76x92x130": ("magic_filter_t_3d_generic_", (dims, per, t1.ref, t2.ref, a.ref, b.ref)),
        "potential_3d 76x92x130": ("potential_application_d_generic_", (dims, per, t1.ref, t2.ref, a.ref, b.ref,
                                                                         w1.ref, e)),
        "kinetic_3d 76x92x130": ("kinetic_d_generic_", (dims, per, h, a.ref, b.ref, w1.ref, w2.ref)),
        "ana_3d 76x92x130": ("ana_self_d_generic_", (dims, per, a.ref, b.ref)),
        "syn_3d 76x92x130": ("syn_self_d_generic_", (dims, per, a.ref, b.ref)),
    }
    out = {}
    for name, (fn, args) in ops.items():
        for _ in range(3):
            q.call(fn, *args)
        q.finish()
        t = time.perf_counter()
        for _ in range(reps):
            q.call(fn, *args)
        q.finish()
        ms = (time.perf_counter() - t) * 1e3 / reps
        cpu, gpu = CONV_CHECK_REF[name]
        out[name] = {"ms": ms, "ref_cpu_ms": cpu, "ref_gpu_ms": gpu}
    q.close()
    return {"workload": "conv_check sizes, FP64, wall time per call over %d calls (launch included)" % reps,
            "ops": out}


def leg_serve(torch, dev, precision, nreq=300, loads=(0.3, 0.5, 0.7)):
    """Serving loop: 64 clients (coarse 16..64 per dim, periodic or free, 4..128
    orbitals), requests 50/50 Hpsi and density; capacity from a burst of one
    request of each kind per client, then Poisson arrivals swept over loads x
    capacity.  The headline p50/p99 are those of the highest load whose
    served rate kept up with the rate the sample's arrivals actually came at
    (requests over the last arrival time; within 5 %: the span of a few
    hundred Poisson arrivals varies by several per cent around the nominal
    rate, which a comparison with the nominal rate would read as falling
    behind)."""
    from wvlh import workloads as W
    from wvlh.serve import Server, latency_stats
    specs = W.serving_clients()
    srv = Server(device=dev.index or 0, precision=precision, hbm_budget=150e9, n_slots=2, scratch_per_slot=16e9)
    cl = [srv.register(lr, n, seed=s) for lr, n, s in specs]
    cells = {c.id: c.coarse_cells for c in cl}
    for _ in range(2):
        t = time.perf_counter()
        reqs = [srv.submit(c, k) for c in cl for k in ("H", "rho")]
        srv.drain()
        dt = time.perf_counter() - t
    cap = len(reqs) / dt
    cap_cells = sum(cells[r.client.id] for r in reqs) / dt
    # warm-up replay, not measured: the first Poisson replay of a process
    # meets first-use costs (batch tables, arena growth) in its latencies
    srv.replay(W.poisson_arrivals(0.3 * cap, 60, len(cl), seed=7))
    sweep = []
    n0, k0 = srv.launches, srv.kernel_launches
    for i, load in enumerate(loads):
        arrivals = W.poisson_arrivals(load * cap, nreq, len(cl), seed=11 + i)
        t = time.perf_counter()
        reqs = srv.replay(arrivals)
        dt = time.perf_counter() - t
        st = latency_stats(reqs)
        sweep.append({"load": load, "offered_req_s": load * cap, "arrival_req_s": len(arrivals) / arrivals[-1][0],
                      "served_req_s": len(reqs) / dt,
                      "served_cells_s": sum(cells[r.client.id] for r in reqs) / dt,
                      "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                      "queued_p50_ms": st["queued_p50_ms"], "queued_p99_ms": st["queued_p99_ms"],
                      "launched_p50_ms": st["launched_p50_ms"], "launched_p99_ms": st["launched_p99_ms"],
                      "tail": st["tail"]})
    kept = [w for w in sweep if w["served_req_s"] >= 0.95 * w["arrival_req_s"]]
    head = kept[-1] if kept else sweep[0]
    out = {"clients": len(cl), "resident_gb": srv.resident / 1e9, "capacity_req_s": cap,
           "capacity_cells_s": cap_cells, "sustained_load": head["load"], "offered_req_s": head["offered_req_s"],
           "arrival_req_s": head["arrival_req_s"],
           "served_req_s": head["served_req_s"], "served_cells_s": head["served_cells_s"],
           "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"], "mean_ms": head["mean_ms"],
           "queued_p99_ms": head["queued_p99_ms"], "launched_p99_ms": head["launched_p99_ms"], "tail": head["tail"],
           "sweep": sweep,
           "launches": srv.launches - n0, "kernel_launches": srv.kernel_launches - k0,
           "requests": nreq * len(loads)}
    srv.close()
    del srv, cl
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    omp_threads()
    import torch
    ws, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import numpy as np

    if args.leg:
        from wvlh.batch import Context
        dev = torch.device("cuda", local)
        ctx = Context(local)
        if args.leg == "free_bc":
            res = leg_free_regions(torch, ctx, dev)
        elif args.leg == "precond":
            res = leg_precond(torch, ctx, dev)
        elif args.leg == "conv_check":
            res = leg_conv_check(torch)
        elif args.leg == "psolver":
            res = leg_psolver(torch, ctx, dev)
        elif args.leg == "nlpsp":
            from wvlh import workloads as W
            lr = W.full_periodic(args.n, 0.45)
            g = torch.Generator(device=dev)
            g.manual_seed(1000)
            psi = torch.rand(args.norb * lr.ncoeff, generator=g, device=dev, dtype=torch.float64) * 2 - 1
            res = leg_nlpsp(torch, ctx, psi, lr, args.norb)
        elif args.leg == "overlap":
            from wvlh import workloads as W
            lr = W.full_periodic(args.n, 0.45)
            g = torch.Generator(device=dev)
            g.manual_seed(1000)
            psi = torch.rand(args.norb * lr.ncoeff, generator=g, device=dev, dtype=torch.float64) * 2 - 1
            res = leg_overlap(torch, ctx, psi, args.norb)
        else:
            res = leg_serve(torch, dev, 32 if args.leg == "serve32" else 64)
        print(json.dumps({"leg": args.leg, "result": res}), flush=True)
        ctx.close()
        return

    from wvlh import workloads as W
    from wvlh._lib import lib
    from wvlh.batch import Batch, Context

    dev = torch.device("cuda", local)
    n, norb = args.n, args.norb
    lr, psi64, pot64 = W.batched_periodic_device(torch, dev, n=n, norb=norb, seed=1000 + rank, pot_seed=1234 + rank)
    psi32 = psi64.float()
    pot32 = pot64.float()
    ctx = Context(local)
    batch = Batch(ctx, [lr], np.zeros(norb, np.int32))
    hpsi32 = torch.empty_like(psi32)
    ek = torch.empty(norb, dtype=torch.float64, device=dev)
    ep = torch.empty(norb, dtype=torch.float64, device=dev)
    esum = torch.zeros(2, dtype=torch.float64, device=dev)
    pts_step = norb * lr.coarse_cells

    # measured block size of the plane kernels for this batch (kept for the run)
    tuned = {}
    for nm, ps, pt in (("fp32", psi32, pot32), ("fp64", psi64, pot64)):
        hh = torch.empty_like(ps)
        pick, times = batch.autotune(ps, pt, hh, ek, ep, reps=2)
        tuned[nm] = {"plane_threads": pick, "ms_by_block_size": times,
                     "z_threads": batch.block_sizes()["locham"]["z"][0 if nm == "fp32" else 1]}
        del hh

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
    w0 = time.time()
    e0.record(st)
    for _ in range(args.steps):
        step()
    e1.record(st)
    torch.cuda.synchronize()
    w1 = time.time()
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop((w0, w1))
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if ws > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms = t.item()
    value = ws * pts_step * args.steps / (ms * 1e-3)
    launches = 4 * args.steps

    extras = {"autotune": tuned}
    if ws > 1 and not args.no_extras:
        extras["multi_gpu"] = leg_exchanges(torch, ctx, batch, psi32, psi64, lr, norb, ws, dev)
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
        # kernel I/O (what each kernel reads and writes, intermediates included)
        kio = [3 * B * npt * norb, 4 * B * npt * norb + B * npt, 4 * B * npt * norb, 0]
        kflops = [128 * npt * norb, 252 * npt * norb, 254 * npt * norb, 0]
        dom = max(range(3), key=lambda i: kt[i])
        # algorithmic bytes of the path per launch: 8 values in + 8 values out
        # per coarse cell of each orbital (64 B in FP32) plus the potential once
        alg = 64 * lr.coarse_cells * norb + 4 * npt
        hbm, hbm_src = peaks()
        tf32 = C.c_double()
        lib().wvlh_measure_fma_peak(32, 20000, C.byref(tf32))
        ach = alg / (kt[dom] * 1e-3) / 1e9
        # DRAM traffic of each kernel (dram__bytes_read.sum + dram__bytes_write.sum) from ncu
        # captures of one call over 48 orbitals of this 48^3 FP32 workload, scaled by the orbitals
        # of this launch (the traffic grows in proportion to them); z kernels: both chains
        traffic48 = [453.519104e6, 582.610688e6, 656.173312e6]
        traffic = traffic48[dom] / 48 * norb if (dom < 3 and n == 48) else None
        step_s = ms / args.steps * 1e-3
        extras["roofline"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                              "traffic": traffic, "kernel": names[dom], "peak_source": hbm_src,
                              "algorithmic_bytes_per_launch": alg,
                              "algorithmic_bytes_rule": "64 B per coarse cell of each orbital (FP32 psi in, "
                                                        "Hpsi out) + the potential once",
                              "kernel_io_bytes": kio[dom],
                              "kernel_ms": kt[dom],
                              "whole_step": {"achieved": alg / step_s / 1e9, "frac": alg / step_s / 1e9 / hbm}}
        fach = kflops[dom] / (kt[dom] * 1e-3) / 1e12
        extras["roofline_fma"] = {"bound": "fp32_fma", "achieved": fach, "peak": tf32.value, "unit": "TFLOP/s",
                                  "frac": fach / tf32.value, "kernel": names[dom],
                                  "peak_source": "measured (register FMA-chain probe)"}
        extras["kernels_ms"] = {nm: round(v, 4) for nm, v in zip(names, kt)}
        # the same step replayed as one captured CUDA graph
        graph = batch.locham_graph(psi32, pot32, hpsi32, ek, ep)
        ga, gb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        graph.launch()
        torch.cuda.synchronize()
        ga.record(st)
        for _ in range(args.steps):
            graph.launch()
        gb.record(st)
        torch.cuda.synchronize()
        extras["graph"] = {"ms_per_step": ga.elapsed_time(gb) / args.steps, "launches_per_step": 1}
        graph.close()

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
        extras["speedup_fp64_fused_vs_fp64_plain"] = ms_plain / ms_f64
        extras["energy_err_ha"] = {"fp32_vs_fp64_max_per_orbital": de, "plain_vs_fused_fp64": dplain}
        # sampled orbitals of this step against the CPU oracle (FP64), both precisions
        sample = [0, norb // 3, norb - 1]
        P64 = psi64.view(norb, -1)
        rows = [P64[o].cpu().numpy() for o in sample]
        vh = pot64.cpu().numpy()
        err = {}
        batch.locham(psi64, pot64, h64, ek64, ep64)
        for nm, H, e1, e2 in (("fp32", hpsi32, ek, ep), ("fp64", h64, ek64, ep64)):
            torch.cuda.synchronize()
            Hs = H.view(norb, -1)
            err[nm] = oracle_errors([lr] * len(sample), rows, [vh] * len(sample),
                                    [Hs[o].double().cpu().numpy() for o in sample],
                                    [e1[o].item() for o in sample], [e2[o].item() for o in sample])
        extras["err_vs_oracle"] = err
        del h64

        # FP64 fused end to end (host buffers, same call as below)
        hp64 = torch.empty(psi64.numel(), dtype=torch.float64, pin_memory=True)
        hp64.copy_(psi64.cpu())
        hv64 = torch.empty(pot64.numel(), dtype=torch.float64, pin_memory=True)
        hv64.copy_(pot64.cpu())
        hh64 = torch.empty_like(hp64).pin_memory()
        hek = torch.empty(norb, dtype=torch.float64).pin_memory()
        hep = torch.empty(norb, dtype=torch.float64).pin_memory()
        batch.locham_host(hp64, hv64, hh64, hek, hep, 64)
        t0 = time.perf_counter()
        for _ in range(3):
            batch.locham_host(hp64, hv64, hh64, hek, hep, 64)
        dt64 = (time.perf_counter() - t0) / 3
        e2e64 = {"value": pts_step / dt64, "ms_per_step": dt64 * 1e3,
                 "h2d_bytes_per_step": hp64.numel() * 8 + hv64.numel() * 8,
                 "d2h_bytes_per_step": hh64.numel() * 8 + 2 * 8 * norb}
        extras["fp64_fused"]["e2e"] = e2e64
        del hp64, hv64, hh64

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
                         "d2h_bytes_per_step": hh.numel() * 4 + 2 * 8 * norb, "ms_per_step": dt * 1e3,
                         "fp64_fused": {"value": e2e64["value"], "ms_per_step": e2e64["ms_per_step"]}}
        # the precision-matched comparators and the oracle errors, also inside
        # the roofline record (FP64 fused and plain on this workload)
        extras["roofline"]["same_workload"] = {
            "fp32_fused_ms": ms / args.steps, "fp64_fused_ms": ms_f64, "fp64_plain_ms": ms_plain,
            "fp64_fused_value": pts_step / (ms_f64 * 1e-3), "fp64_plain_value": pts_step / (ms_plain * 1e-3),
            "speedup_fp32_vs_fp64_plain": extras["speedup_vs_fp64_plain"],
            "speedup_fp64_fused_vs_fp64_plain": ms_plain / ms_f64,
            "fp64_fused_frac": 2 * alg / (ms_f64 * 1e-3) / 1e9 / hbm,
            "err_vs_oracle": err}
        # the other rows of the path on this GPU
        extras["density"] = leg_density(torch, batch, psi32, psi64, lr, norb, dev)
        extras["overlap"] = leg_overlap(torch, ctx, psi64, norb)
        extras["nlpsp"] = leg_nlpsp(torch, ctx, psi64, lr, norb)
        extras["psolver"] = leg_psolver(torch, ctx, dev)
        extras["conv_check"] = leg_conv_check(torch)
        del hp, hv, hh
        extras["free_bc"] = leg_free_regions(torch, ctx, dev)
        extras["precond"] = leg_precond(torch, ctx, dev)
        serve = {}
        for prec in (32, 64):
            serve["fp%d" % prec] = leg_serve(torch, dev, prec)
        extras["serve"] = serve
        if ws == 1:
            r, cores, sample = cpu_oracle_rate(n)
            cpu = host_cpu()
            extras["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                                      "cpu_model": cpu["model"], "physical_cores": cpu["physical_cores"]}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": DATA, "config": workload_config(n, norb, ws),
                "gpu_launches": launches, "clocks": clocks}
        line.update(extras)
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
