#!/usr/bin/env python
"""Benchmark: atom-steps/s of SIMOX's per-step force and charge path on B200.

Workload (the 128k bulk-oxide configuration): alpha-Al2O3 corundum supercell
of 20x14x8 orthohexagonal cells, 128,000 atoms after 4.8 % random vacancies
(Al:O = 2:3), PME 128^3 with order-6 B-splines, Rcut 10 A, NVT Berendsen at
600 K, dt = 1 fs, cell sort every step.  Charges are equilibrated by
CTIP_SOLVER at step 1 (TAG_SET with freq_new larger than the run, inside the
warm-up); the timed steps are VV_NVE1, CELL_SORT, FORCE, PME and
VV_NVT2_BEREND of main.f90:41-61 with the RDF accumulated every step, as the
reference does, and the energies (always FP64) evaluated on every 10th step,
the cadence at which TAG_SET's status rule prints them.  Synthetic seeded
input (no dataset exists).

One step = one pass of that loop over all 128,000 atoms.  ``value`` is the
mixed-precision path (FP32 pair and PME terms, FP64 sums) with device-resident
inputs; ``fp64`` reports the all-FP64 path on the same input.  ``e2e`` goes
through the C ABI with host buffers: per step simox_set_state from pinned host
memory, one step, simox_get_state back (x, v, f, q both ways).

Multi-GPU: replicas only (one independent system per rank, weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s @128k Al/O: mixed vs FP64 on B200 (force err≤1e-5), CPU ref"
UNIT = "atom-steps/s"
WORKLOAD = "corundum Al2O3 128000 atoms, PME 128^3 order 6, Rcut 10 A, NVT Berendsen 600 K, dt 1 fs"
FREQ_NEW = 1000000          # CTIP at step 1 only (warm-up)
FREQ_STAT = 10              # energies (FP64) every 10th step, as TAG_SET's status rule


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, backend):
    if world <= 1:
        return None
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=timedelta(seconds=300))
    return dist


def reduce_max(dist, v, device=None):
    """Max of a float over ranks (identity for one rank)."""
    if dist is None:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_value(world, n_atoms, steps, ms_max):
    """Whole-job atom-steps/s of `world` independent replicas of n_atoms,
    each timed over `steps` steps, from the slowest rank's milliseconds."""
    return world * n_atoms * steps / (ms_max / 1e3)


def barrier(dist, device=None):
    if dist is None:
        return
    if device is not None and str(device).startswith("cuda"):
        dist.barrier(device_ids=[int(str(device).split(":")[1])])
    else:
        dist.barrier()


# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.proc = None
        self.idx = gpu_index
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "of measured"
    except Exception:
        return 6650.0, "of fallback"


def profile_figure(kernel, key):
    """A figure recorded in the committed ncu summary of ``kernel``
    (profiles/<kernel>_corundum128k.md, a line "key: value")."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_corundum128k.md")
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":")[1])
    except (OSError, ValueError):
        pass
    return None


# Algorithmic bytes per atom-step of each kernel family: the path's cost model
# (FP64 sizes, the mixed path's FP32 grids halved; K grid points amortised over
# the N atoms).  integrate-1 124 B, integrate-2 72 B (+ 48 B for the Berendsen
# rescale's second sweep over v), cell binning 104 B in all, EAM pass 1 44 B,
# pair/force pass 2 68 B, spread 32 B + K grid values, FFT R2C + C2R two
# read+write sweeps of the real and the half-complex grid each, influence
# multiply 40 B per half-spectrum point (20 B in FP32), gather 56 B + K grid
# values.  The skin-list upkeep, the gather into pair order and the exact-list
# rows are this implementation's own traffic, not algorithmic.
def algorithmic_bytes(name, n, K, prec):
    g = 8 if prec == "fp64" else 4          # bytes per real grid value
    table = {
        "vv_nve1": 124 * n, "vv_nvt2_kick": 72 * n, "vv_nvt2_scale": 48 * n,
        "cell_bin": 104 * n,                  # the whole binning (bin, scan, scatter, order)
        "neighbor_filter_density": 44 * n, "pair_force": 68 * n,
        "pme_spread": 32 * n + g * K, "pme_gather_force": 56 * n + g * K,
        "pme_fft_r2c": 4 * g * K, "pme_fft_c2r": 4 * g * K,
        "pme_influence": 5 * g * (K // 2),
    }
    return table.get(name)


# --------------------------------------------------------------------------
def build_system(seed=2):
    from simox_b200 import systems as S
    return S.corundum(seed=seed)


def equilibrated_context(s, precision, device=0):
    """Context with PME_SELF, CELL_SORT, initial FORCE/PME and the step-1
    CTIP solve done (the first warm-up step)."""
    from simox_b200 import api
    g = api.from_system(s, precision=precision, device=device)
    g.pme_self()
    g.cell_sort()
    g.force()
    g.pme()
    return g


def force_error(s, device=0):
    """Mixed-precision FORCE + PME forces against the all-FP64 path on the
    same input: ||F_mixed - F_fp64|| / ||F_fp64|| over all components, and
    the largest per-atom |dF| relative to the RMS atom force; the same two
    figures for FORCE alone and PME alone (each relative to the total force's
    RMS), which locate the error."""
    from simox_b200 import api
    out, pair, rec = {}, {}, {}
    for prec in ("fp64", "mixed"):
        with api.from_system(s, precision=prec, device=device) as g:
            g.pme_self()
            g.cell_sort()
            g.force(energies=False)
            pair[prec] = g.get_state()["f"]
            g.pme(energies=False)
            out[prec] = g.get_state()["f"]
            g.set_state(f=np.zeros((s.n, 3)))
            g.pme(energies=False)
            rec[prec] = g.get_state()["f"]
    nrm = np.linalg.norm(out["fp64"])
    frms = nrm / np.sqrt(s.n)

    def fig(a):
        d = a["mixed"] - a["fp64"]
        return {"rel_norm": float(np.linalg.norm(d) / nrm),
                "max_atom_rel_rms": float(np.linalg.norm(d, axis=1).max() / frms)}

    res = fig(out)
    res["force_only"] = fig(pair)
    res["pme_only"] = fig(rec)
    return res


def run_md(g, s, first, nsteps, rdf):
    from simox_b200 import systems as S
    return g.md_run(nsteps, 1.0 / S.TFM, first_step=first, thermostat=True, T_given=600.0 * S.KB,
                    freq_new=FREQ_NEW, freq_sort=1, rdf=rdf, freq_stat=FREQ_STAT)


def time_device(g, s, steps, warmup, dist, device):
    """W warm-up steps (step 1 runs CTIP), then K steps between events."""
    from simox_b200 import _abi
    rdf = np.zeros(_abi.RDF_LEN, np.int32)
    t0 = time.perf_counter()
    run_md(g, s, 1, warmup, rdf)
    g.sync()
    warm_s = time.perf_counter() - t0
    barrier(dist, device)
    g.sync()
    l0 = g.launch_count()
    r0 = g.skin_rebuilds()
    g.timer_begin()
    e = run_md(g, s, warmup + 1, steps, rdf)
    ms = g.timer_end()
    g.sync()
    launches = g.launch_count() - l0
    time_device.rebuilds = g.skin_rebuilds() - r0
    barrier(dist, device)
    return ms, e, launches, warm_s


def time_e2e(g, s, steps, first):
    """Through the C ABI with host buffers: set_state (pinned host -> device),
    one step, get_state (device -> pinned host), every step."""
    import torch
    n = s.n
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    x, v, f, q = pin((n, 3)), pin((n, 3)), pin((n, 3)), pin((n,))
    st = g.get_state()
    x[:], v[:], f[:], q[:] = st["x"], st["v"], st["f"], st["q"]
    from simox_b200 import api
    L = api.lib()
    ctx = g._ctx
    dp = api._dp
    xs, vs, fs, qs = (a.ctypes.data_as(dp) for a in (x, v, f, q))
    from simox_b200 import _abi
    rdf = np.zeros(_abi.RDF_LEN, np.int32)
    g.sync()
    t0 = time.perf_counter()
    for k in range(steps):
        rc = L.simox_set_state(ctx, n, None, xs, vs, fs, qs)
        if rc:
            raise RuntimeError(f"set_state {rc}")
        run_md(g, s, first + k, 1, rdf)
        rc = L.simox_get_state(ctx, n, None, xs, vs, fs, qs)
        if rc:
            raise RuntimeError(f"get_state {rc}")
    dt = time.perf_counter() - t0
    nbytes = n * (3 + 3 + 3 + 1) * 8
    return dt, nbytes


def profile_steps(g, s, steps, first):
    """Per-kernel event spans of `steps` eager steps run like the timed ones
    (RDF accumulated every step, energies on the status steps)."""
    from simox_b200 import _abi
    g.profile(True)
    g.profile_reset()
    run_md(g, s, first, steps, np.zeros(_abi.RDF_LEN, np.int32))
    prof = g.profile_read()
    g.profile(False)
    return prof


def cpu_baseline_sample(s, timeout_s=120.0):
    """The oracle (FP64 C restatement, one thread) on one full MD step of the
    same system: VV_NVE1, CELL_SORT, FORCE, PME, VV_NVT2_BEREND."""
    from oracle import oracle as O
    from simox_b200 import systems as S
    o = O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=s.order, nnb_max=640)
    o.pme_self()
    o.cell_sort()
    f, *_ = o.force()
    f, _ = o.pme(f)
    dt = 1.0 / S.TFM
    t0 = time.perf_counter()
    v = o.vv_nve1(s.v, f, dt)
    o.cell_sort()
    f, *_ = o.force()
    f, _ = o.pme(f)
    v, _ = o.vv_nvt2_berend(v, f, dt, 600.0 * S.KB)
    el = time.perf_counter() - t0
    return el


def _reference_worker(nsteps, warm, barrier, out):
    """One copy of the reference's step (the oracle port, one thread): set-up
    and warm-up, then `nsteps` timed steps started together with the other
    copies (barrier); puts (timed seconds, peak RSS in bytes) on `out`."""
    import resource
    s = build_system()
    from oracle import oracle as O
    from simox_b200 import systems as S
    o = O.System(s.ids, s.x, s.q, s.box, s.rcut, s.fft, order=s.order, nnb_max=640)
    o.pme_self()
    o.cell_sort()
    f, *_ = o.force()
    f, _ = o.pme(f)
    dt = 1.0 / S.TFM
    v = s.v.copy()

    def step(v, f):
        v = o.vv_nve1(v, f, dt)
        o.cell_sort()
        f, *_ = o.force(rdf=True)
        f, _ = o.pme(f)
        v, _ = o.vv_nvt2_berend(v, f, dt, 600.0 * S.KB)
        return v, f

    for _ in range(warm):
        v, f = step(v, f)
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        v, f = step(v, f)
    el = time.perf_counter() - t0
    out.put((el, resource.getrusage(resource.RUSAGE_SELF).ru_maxrss * 1024))


def reference_processes(requested=0):
    """Copies of the serial reference that this host runs side by side: one
    per core, at most one per 3 GiB of available memory (a 128,000-atom copy
    peaks near 2.2 GiB), at most 64."""
    if requested > 0:
        return requested
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil
        mem = int(psutil.virtual_memory().available // (3 << 30))
    except Exception:
        mem = cores
    return max(1, min(cores, mem, 64))


def run_reference(args):
    """--impl reference: the reference's path on the host's cores.  The
    Fortran reference cannot be compiled here (no Fortran compiler), so this
    times the oracle port of it (FP64, statement by statement).  The reference
    is serial, so it uses the host's threads the only way it can: one copy of
    the same 128,000-atom step per core, all started together; the value is
    the copies' total atom-steps over the slowest copy's time."""
    import multiprocessing as mp
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    from simox_b200 import systems as S
    n_atoms = build_system().n
    nsteps = max(1, min(args.steps, 3))
    warm = 1 if args.warmup > 0 else 0
    procs = reference_processes(args.ref_procs)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    out = ctx.Queue()
    workers = [ctx.Process(target=_reference_worker, args=(nsteps, warm, barrier, out)) for _ in range(procs)]
    for w in workers:
        w.start()
    res = [out.get() for _ in workers]
    for w in workers:
        w.join()
    el = max(r[0] for r in res)
    val = procs * n_atoms * nsteps / el
    sample = (f"{nsteps} timed step(s) after {warm} warm-up of the full 128,000-atom step "
              f"(VV_NVE1, CELL_SORT, FORCE, PME, VV_NVT2_BEREND), {procs} copies side by side, one thread "
              f"each (the reference is serial); oracle port of the Fortran (no Fortran compiler on this image); "
              f"slowest copy {el / nsteps:.2f} s per step, peak memory "
              f"{max(r[1] for r in res) / 2 ** 30:.2f} GiB per copy")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": nsteps, "warmup": warm, "ms_per_step": el / nsteps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_atoms": n_atoms, "copies": procs},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": procs, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def batch_object(nsys, steps, sequential=True):
    """The batched-replica workload (independent Al/O systems of 500-8000
    atoms, O fraction 0-0.6, 300-1200 K, own box and PME grid 32^3-64^3,
    order 6; seed 7), mixed precision, NVT Berendsen at each system's
    temperature, energies every 10th step.  All systems advance together (one
    CUDA graph launch per step, each kernel of the step launched once for all
    systems) after the force pass's CTA split is autotuned on the batch.
    Reported beside the per-system graph and the systems stepped one after
    another."""
    from simox_b200 import api, systems as S
    systems = S.replica_batch(seed=7, nsys=nsys)
    natoms = sum(s.n for s in systems)
    dt = 1.0 / S.TFM
    members = []
    for s in systems:
        g = api.from_system(s, precision="mixed")
        g.pme_self()
        g.cell_sort()
        g.force()
        g.pme()
        members.append(g)
    opts = [api.md_opts(dt, thermostat=True, T_given=s.meta["T"] * S.KB, freq_stat=10) for s in systems]
    b = api.Batch(members)
    b.md_run(opts, 2, first_step=1)
    times, best = b.autotune(opts, first_step=3, trial_steps=5)
    step = 3 + 5 * 6
    b.md_run(opts, 20, first_step=step)          # both step graphs captured again
    step += 20
    n = max(steps, 20)
    l0 = b.launch_count()
    t0 = time.perf_counter()
    b.md_run(opts, n, first_step=step)
    el = time.perf_counter() - t0
    launches = (b.launch_count() - l0) / n
    mode = b.mode()
    step += n
    out = {"metric": "atom-steps/s, batched independent Al/O systems", "value": natoms * n / el,
           "unit": UNIT, "steps": n, "ms_per_step": el / n * 1e3,
           "workload": f"{nsys} systems of 500-8000 atoms (seed 7), {natoms} atoms in total, mixed precision, "
                       f"energies every 10th step",
           "timing": "wall clock around one batch md_run call (ends with a device sync)",
           "mode": mode,
           "autotune_ms_per_step": [round(t, 3) for t in times], "autotune_best_rule": int(best),
           "gpu_launches_per_step": launches}
    # the same batch as one graph of every system's own launches
    b.set_mode("per_system")
    b.md_run(opts, 10, first_step=step)          # captures both step graphs (untimed)
    step += 10
    l1 = b.launch_count()
    t2 = time.perf_counter()
    b.md_run(opts, n, first_step=step)
    el_ps = time.perf_counter() - t2
    out["per_system_graph"] = {"value": natoms * n / el_ps, "unit": UNIT, "ms_per_step": el_ps / n * 1e3,
                               "gpu_launches_per_step": (b.launch_count() - l1) / n,
                               "how": "one graph per step holding every system's own kernel launches"}
    step += n
    if sequential:
        # untimed: each context captures its own step graphs (energy step and plain step)
        for k, g in enumerate(members):
            g.md_run(10, dt, first_step=step, thermostat=True, T_given=systems[k].meta["T"] * S.KB, freq_stat=10)
            g.sync()
        step += 10
        t1 = time.perf_counter()
        for k, g in enumerate(members):
            g.md_run(10, dt, first_step=step, thermostat=True, T_given=systems[k].meta["T"] * S.KB, freq_stat=10)
            g.sync()
        el_seq = time.perf_counter() - t1
        out["sequential"] = {"value": natoms * 10 / el_seq, "unit": UNIT, "ms_per_step": el_seq / 10 * 1e3,
                             "how": "each system's own md_run (its step graphs), one after another"}
    b.close()
    for g in members:
        g.close()
    return out


def batch_profile(nsys, mode):
    """--batch N --ncu: the batch set up as in batch_object (no autotuning),
    its step graphs captured, then ONE step without energies between
    cudaProfilerStart and cudaProfilerStop (ncu --profile-from-start off)."""
    import torch
    from simox_b200 import api, systems as S
    systems = S.replica_batch(seed=7, nsys=nsys)
    dt = 1.0 / S.TFM
    members = []
    for s in systems:
        g = api.from_system(s, precision="mixed")
        g.pme_self()
        g.cell_sort()
        g.force()
        g.pme()
        members.append(g)
    opts = [api.md_opts(dt, thermostat=True, T_given=s.meta["T"] * S.KB, freq_stat=10) for s in systems]
    b = api.Batch(members)
    b.set_mode(mode)
    b.md_run(opts, 14, first_step=1)          # eager first step, both step graphs captured
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    b.md_run(opts, 1, first_step=15)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    b.close()
    for g in members:
        g.close()


def run_batch(args):
    """--batch N: the batched-replica workload alone (256 systems in its
    configuration).  Not the headline metric."""
    from simox_b200 import build
    build.build()
    if args.ncu:
        batch_profile(args.batch, args.batch_mode)
        return 0
    o = batch_object(args.batch, args.steps)
    line = {"metric": o.pop("metric"), "value": o.pop("value"), "unit": UNIT, "n_gpus": 1,
            "steps": o.pop("steps"), "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": o.pop("workload"), "timing": o.pop("timing")}}
    line.update(o)
    print(json.dumps(line), flush=True)
    return 0


def adjoint_object(nsnap, sequential=True):
    """The parameter-gradient workload: seeded snapshots of 2000-atom Al/O
    systems (O fraction 0.1-0.5, 300-1000 K), synthetic targets = the FP64
    model forces plus Gaussian noise (0.05 eV/A); per snapshot the charges,
    forces and the gradients of the energy and of the force-matching loss with
    respect to 3 x 64 spline coefficients and chi, J, Z, xi (FP64, one adjoint
    CG through the charge solve), all snapshots at once through
    simox_adjoint_eval_many."""
    from simox_b200 import api, spline, systems as S
    rng = np.random.default_rng(11)
    P = api.default_potential()
    spl = spline.fit(P)
    ctxs, targets = [], []
    for k in range(nsnap):
        s = S.replica(int(rng.integers(1 << 30)), 2000, float(rng.uniform(0.1, 0.5)), float(rng.uniform(300, 1000)))
        g = api.from_system(s, precision="fp64")
        g.pme_self()
        g.cell_sort()
        g.set_eam_spline(spl)
        _, f0, _, _ = g.adjoint_eval(gradients=False)
        targets.append(f0 + rng.normal(0.0, 0.05, f0.shape))
        ctxs.append(g)
    api.adjoint_eval_many(ctxs, targets)   # warm-up: charges converged at these parameters, threads started
    seq = None
    if sequential:
        t0 = time.perf_counter()
        seq = [g.adjoint_eval(t) for g, t in zip(ctxs, targets)]
        el_seq = time.perf_counter() - t0
    t0 = time.perf_counter()
    out = api.adjoint_eval_many(ctxs, targets)
    el = time.perf_counter() - t0
    reps = [o[0] for o in out]
    gE = np.sum([o[2] for o in out], axis=0)
    gL = np.sum([o[3] for o in out], axis=0)
    res = {"metric": "parameter-gradient snapshots/s (2000-atom Al/O, FP64 adjoint)", "value": len(ctxs) / el,
           "unit": "snapshots/s",
           "workload": f"{len(ctxs)} seeded snapshots of 2000 atoms, targets = model forces + N(0, 0.05)",
           "parameters": "3 x 64 spline coefficients + chi, J, Z, xi of 5 species (212)",
           "api": "simox_adjoint_eval_many (all snapshots concurrently, one host thread and stream per "
                  "snapshot, up to 16 threads)",
           "ms_per_snapshot": el / len(ctxs) * 1e3,
           "mean_adjoint_cg_iterations": float(np.mean([r["n_adjoint"] for r in reps])),
           "mean_newton_steps": float(np.mean([r["n_newton"] for r in reps])),
           "max_charge_residual": float(max(r["residual"] for r in reps)),
           "loss_total": float(sum(r["loss"] for r in reps)),
           "grad_L_norm": float(np.linalg.norm(gL)), "grad_E_norm": float(np.linalg.norm(gE))}
    if seq is not None:
        gL_seq = np.sum([o[3] for o in seq], axis=0)
        res["sequential"] = {"value": len(ctxs) / el_seq, "unit": "snapshots/s",
                             "api": "simox_adjoint_eval, one snapshot after another"}
        res["grad_L_rel_diff_concurrent_vs_sequential"] = float(np.linalg.norm(gL - gL_seq) / np.linalg.norm(gL_seq))
    # the same with FP32 pair terms in the forward passes (FP64 adjoint)
    for g in ctxs:
        g.adjoint_forward_precision("mixed")
    t0 = time.perf_counter()
    out32 = api.adjoint_eval_many(ctxs, targets)
    el32 = time.perf_counter() - t0
    gL32 = np.sum([o[3] for o in out32], axis=0)
    res["fp32_forward"] = {"value": len(ctxs) / el32, "unit": "snapshots/s",
                           "api": "simox_adjoint_forward_precision(SIMOX_MIXED) + simox_adjoint_eval_many",
                           "grad_L_rel_diff_vs_fp64_forward": float(np.linalg.norm(gL32 - gL) / np.linalg.norm(gL))}
    for g in ctxs:
        g.close()
    return res


def run_adjoint(args):
    """--adjoint N: the parameter-gradient workload alone (32 snapshots in its
    configuration).  Not the headline metric."""
    from simox_b200 import build
    build.build()
    o = adjoint_object(args.adjoint)
    line = {"metric": o.pop("metric"), "value": o.pop("value"), "unit": o.pop("unit"), "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": o.pop("workload"), "parameters": o.pop("parameters"), "api": o.pop("api")}}
    line.update(o)
    print(json.dumps(line), flush=True)
    return 0


def ctip_object(g, label):
    """One CTIP_SOLVER re-solve at the context's current positions (charges
    from the last solve), timed with CUDA events on the context's stream:
    CG iterations, line evaluations, ms per solve and per CG iteration; then
    the per-kernel split from up to 20 host-driven iterations from the same
    starting charges with every launch bracketed by events."""
    q0 = g.get_state()["q"]
    g.sync()
    g.timer_begin()
    _, rep = g.ctip_solver()
    ms = g.timer_end()
    q1 = g.get_state()["q"]
    out = {"precision": label, "n_cg": rep["n_cg"], "n_line": rep["n_line"], "ms_per_solve": ms,
           "ms_per_cg_iteration": ms / max(rep["n_cg"], 1), "final_error": rep["error"],
           "total_charge_change_e": float(abs(q1.sum() - q0.sum()))}
    g.set_state(q=q0)
    g.profile(True)
    g.profile_reset()
    _, rep2 = g.ctip_solver(max_cg=20)
    prof = g.profile_read()
    g.profile(False)
    it = max(rep2["n_cg"], 1)
    out["kernels_ms_per_cg_iteration"] = {k: round(v[0] / it, 4)
                                          for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    out["kernels_note"] = f"host-driven loop, {it} iterations, event span per launch family"
    g.set_state(q=q1)
    return out


def c3_object(steps=2, device=0):
    """The oxidation slab (fcc Al 60x60x30 = 432,000 atoms plus 40,000 O at
    0.02 A^-3 above, PME 256x256x384, order 6), mixed precision, NVE at
    dt = 0.5 fs with CTIP_SOLVER on every step (the driver flag): one charge
    solve from zero charges first (untimed), then `steps` timed loop steps,
    each VV_NVE1, CELL_SORT, CTIP_SOLVER, FORCE, PME, VV_NVE2."""
    from simox_b200 import api, systems as S
    s = S.oxidation_slab()
    g = api.from_system(s, precision="mixed", device=device)
    g.pme_self()
    g.cell_sort()
    t0 = time.perf_counter()
    _, rep0 = g.ctip_solver()
    first_s = time.perf_counter() - t0
    g.force(energies=False)
    g.pme(energies=False)
    q0 = g.get_state()["q"].sum()
    g.sync()
    g.timer_begin()
    e = g.md_run(steps, 0.5 / S.TFM, first_step=2, thermostat=False, freq_new=1000, charge_every_step=True,
                 freq_stat=1)
    ms = g.timer_end()
    q = g.get_state()["q"]
    g.close()
    return {"metric": "atom-steps/s, oxidation slab with CTIP_SOLVER every step", "value": s.n * steps / (ms / 1e3),
            "unit": UNIT, "n_atoms": s.n, "steps": steps, "ms_per_step": ms / steps,
            "first_solve": {"n_cg": rep0["n_cg"], "seconds": first_s, "from": "zero charges"},
            "total_charge_change_e": float(abs(q.sum() - q0)),
            "energies_last_status_step": e}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-procs", type=int, default=0,
                    help="copies of the serial reference run side by side by --impl reference "
                         "(default: one per core, memory permitting)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the all-FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--ncu", action="store_true",
                    help="profiling run: set-up, then --steps MD steps of the workload (charges as "
                         "generated, no CTIP, RDF every step, no comparison runs); prints nothing else")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"], help="precision of --ncu")
    ap.add_argument("--ncu-ctip", type=int, default=0,
                    help="--ncu: after the set-up run this many CTIP_SOLVER CG iterations (host-driven loop) "
                         "instead of MD steps")
    ap.add_argument("--freq-stat", type=int, default=FREQ_STAT,
                    help="--ncu: energies on steps with MOD(step, freq_stat) == 0 (1: every step)")
    ap.add_argument("--batch", type=int, default=0,
                    help="run the batched-replica workload with this many systems (256 in its configuration)")
    ap.add_argument("--batch-mode", default="per_pass", choices=["per_pass", "per_system"],
                    help="--batch with --ncu: the batch mode of the profiled step")
    ap.add_argument("--adjoint", type=int, default=0,
                    help="run the parameter-gradient workload with this many snapshots (32 in its configuration)")
    ap.add_argument("--no-ctip", action="store_true", help="skip the timed CTIP re-solves")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the 256-system batch and 32-snapshot adjoint objects of the default line")
    ap.add_argument("--c3", action="store_true",
                    help="add the 472k oxidation slab with the charge solve on every step")
    args = ap.parse_args()
    if args.adjoint:
        return run_adjoint(args)
    if args.batch:
        return run_batch(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.ncu:
        from simox_b200 import build
        build.build()
        s = build_system()
        g = equilibrated_context(s, args.precision)
        from simox_b200 import systems as S
        if args.ncu_ctip:
            g.profile(True)   # host-driven CG loop: every iteration's kernels are plain launches
            g.ctip_solver(max_cg=args.ncu_ctip)
            g.profile(False)
        else:   # as the timed steps: RDF accumulated every step
            from simox_b200 import _abi
            g.md_run(args.steps, 1.0 / S.TFM, first_step=2, thermostat=True, T_given=600.0 * S.KB,
                     freq_new=FREQ_NEW, freq_sort=1, freq_stat=args.freq_stat,
                     rdf=np.zeros(_abi.RDF_LEN, np.int32))
        g.sync()
        g.close()
        return 0
    args.warmup = max(args.warmup, 3)

    rank, world, local = dist_info()
    import torch
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    dist = init_dist(world, "nccl")

    from simox_b200 import build
    build.build()
    s = build_system(seed=2 + rank)

    # mixed path (the headline)
    g = equilibrated_context(s, "mixed", device=local)
    clocks = ClockSampler(local)
    ms, e, launches, warm_s = time_device(g, s, args.steps, args.warmup, dist, device)
    rebuilds = time_device.rebuilds
    clk = clocks.stop()
    ms_max = reduce_max(dist, ms, device)
    value = replicas_value(world, s.n, args.steps, ms_max)
    mx_nnb, tot_nnb = g.neighbor_stats()
    half = g.get_tuning().get("half_list", 0) == 1
    if half:   # the statistics count pairs: both atoms' rows would hold each once
        tot_nnb *= 2
    nnb = tot_nnb / s.n

    # e2e through the C ABI with host buffers
    e2e_s, nbytes = time_e2e(g, s, max(3, args.steps // 2), args.warmup + args.steps + 1)
    e2e_s = reduce_max(dist, e2e_s, device)
    e2e_val = replicas_value(world, s.n, max(3, args.steps // 2), e2e_s * 1e3)

    # per-kernel profile (separate pass; event-bracketed launches)
    nprof = min(args.steps, 5)
    prof = profile_steps(g, s, nprof, args.warmup + args.steps + 100)
    ctip_mixed = ctip_object(g, "mixed") if not args.no_ctip else None
    g.close()
    K = int(np.prod(s.fft))
    fam = {k: [v[0] / nprof, v[1] / nprof] for k, v in prof.items()}
    cell = [k for k in fam if k in ("cell_bin", "cell_scan", "cell_scatter", "cell_order")]
    if cell:   # the binning's cost model covers its four kernels together
        fam["cell_bin"] = [sum(fam[k][0] for k in cell), 1.0]
        for k in cell:
            if k != "cell_bin":
                fam.pop(k)
    peak, peak_kind = measured_peaks()
    per_kernel = {}
    for k, (ms_k, nl) in fam.items():
        by = algorithmic_bytes(k, s.n, K, "mixed")
        if by is None or ms_k <= 0:
            continue
        per_launch = ms_k / max(nl, 1)
        gbs = by / (per_launch / 1e3) / 1e9
        per_kernel[k] = {"ms_per_step": round(ms_k, 4), "algorithmic_mb_per_launch": round(by / 1e6, 2),
                         "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    dom = max(per_kernel, key=lambda k: per_kernel[k]["ms_per_step"])
    dom_ms = fam[dom][0] / max(fam[dom][1], 1)
    dom_bytes = algorithmic_bytes(dom, s.n, K, "mixed")
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = profile_figure(dom, "traffic_bytes_per_launch")
    step_bytes = sum(algorithmic_bytes(k, s.n, K, "mixed") or 0 for k in
                     ("vv_nve1", "vv_nvt2_kick", "vv_nvt2_scale", "cell_bin", "neighbor_filter_density",
                      "pair_force", "pme_spread", "pme_gather_force", "pme_fft_r2c", "pme_fft_c2r", "pme_influence"))
    # the pair passes are bound by instruction issue and the SFU, not by
    # memory: their rate in pair evaluations per second beside the issue
    # utilisation ncu measured
    evals = tot_nnb * (0.5 if half else 1.0)
    pair_rate = {}
    for k in ("neighbor_filter_density", "pair_force"):
        if k in fam:
            t = fam[k][0] / max(fam[k][1], 1)
            pair_rate[k] = {"pairs_per_launch": int(tot_nnb // 2), "evaluations_per_launch": int(evals),
                            "pair_evaluations_per_s": evals / (t / 1e3), "ms_per_launch": round(t, 4),
                            "issue_active_pct_ncu": profile_figure(k, "issue_active_pct"),
                            "sfu_pipe_pct_ncu": profile_figure(k, "xu_pipe_pct")}

    # all-FP64 path, same input
    fp64 = None
    ctip_fp64 = None
    if not args.no_fp64:
        g64 = equilibrated_context(s, "fp64", device=local)
        ms64, _, _, _ = time_device(g64, s, args.steps, args.warmup, dist, device)
        if not args.no_ctip:
            ctip_fp64 = ctip_object(g64, "fp64")
        g64.close()
        ms64 = reduce_max(dist, ms64, device)
        fp64 = {"value": replicas_value(world, s.n, args.steps, ms64), "unit": UNIT, "ms_per_step": ms64 / args.steps,
                "skin_rebuilds_in_timed_steps": time_device.rebuilds}

    ferr = force_error(s, device=local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        el = cpu_baseline_sample(s)
        cpu = {"value": s.n / el, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "one full 128,000-atom step (VV_NVE1, CELL_SORT, FORCE, PME, VV_NVT2_BEREND) "
                         "of the oracle port on 1 host thread"}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        # the headline is measured by now: a failing side workload is reported
        # in its object instead of costing the whole line
        jobs = [("batch", lambda: batch_object(256, 20, sequential=True)),
                ("adjoint", lambda: adjoint_object(32, sequential=False))]
        if args.c3:
            jobs.append(("slab_charges_every_step", lambda: c3_object(steps=2, device=local)))
        for key, job in jobs:
            try:
                extras[key] = job()
            except Exception as exc:   # noqa: BLE001 - reported, not hidden
                extras[key] = {"error": f"{type(exc).__name__}: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_atoms": s.n, "per_rank_replicas": 1,
                       "parallelism": "replicas" if world > 1 else "single",
                       "precision": "mixed: FP32 pair/PME terms, FP64 sums, energies, CG",
                       "charges": "CTIP at step 1 (warm-up), freq_new > run length; re-solve timed separately (ctip)",
                       "energies": "FP64 energies on steps with MOD(step, 10) == 0 (status rule); RDF every step",
                       "l2": "inputs larger than L2 (exact neighbour list %.0f MB rebuilt every step)" % (
                           tot_nnb * (2 if half else 4) / 1e6),
                       "mean_neighbours": round(nnb, 1),
                       "neighbour_list": ("half: each pair once, partner shares scattered into 64-bit fixed-point "
                                          "sums" if half else "full: each pair in both atoms' rows")},
            "fp64": fp64,
            "mixed_over_fp64": (value / fp64["value"]) if fp64 else None,
            "force_err_vs_fp64": ferr,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "gpu_launches": launches,
            "skin_rebuilds_in_timed_steps": rebuilds,
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "traffic_over_algorithmic": (traffic / dom_bytes) if traffic else None,
                         "avg_launch_ms": dom_ms, "algorithmic_bytes_per_launch": dom_bytes,
                         "bytes_model": "per-atom cost model of the path (EAM pass 1 44 B, pair pass 2 68 B, ...)"},
            "step_roofline": {"algorithmic_mb_per_step": round(step_bytes / 1e6, 1),
                              "achieved_gbs": step_bytes / (ms_max / args.steps / 1e3) / 1e9,
                              "frac": step_bytes / (ms_max / args.steps / 1e3) / 1e9 / peak},
            "kernel_roofline": per_kernel,
            "pair_rate": pair_rate,
            "kernels_note": "event spans per launch family from a separate eager pass with PME on the main "
                            "stream (the timed steps run it on a side stream, overlapped with the pair passes)",
            "kernels_ms_per_step": {k: round(v[0] / max(nprof, 1), 4) for k, v in
                                    sorted(prof.items(), key=lambda kv: -kv[1][0])},
            "ctip": {"mixed": ctip_mixed, "fp64": ctip_fp64},
            "cpu_baseline": cpu,
            "clocks": clk,
            "energies_last_status_step": e,
            "warmup_seconds": warm_s,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
