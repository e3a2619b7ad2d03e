#!/usr/bin/env python
"""TreePM force-evaluation benchmark.

One step = one full TreePM force evaluation (Morton sort, TSC deposit,
Poisson FFT, gradient + interpolation, tree build, tree walk, forces
scattered back to the caller's order) of the plain engine at scale: 512^3
particles on a 512^3 mesh, L = 500 Mpc/h, seeded Zel'dovich field with
P(k) ~ k^-2.5 and an rms displacement of 2 spacings (strongly clustered),
velocities 0.5 psi, softening 0.05 cells.

The metric is quoted at rms force error <= 1e-3 against the FP64 Ewald sum.
The reference's own split law (PMFITPARA residual, efold 0.9, rsphere 4)
stays near 3.5e-3 on these workloads, so the headline uses the engine's
Gaussian split (rs = 0.7 cells, short-range cut at 3.5 cells, interlaced
TSC grids with their optimal influence function, 8-point gradient, theta
0.4: rms 4.8e-4 at 512^3 and below 8e-4 on every workload the tests run);
the same line also carries the reference law's throughput and error
("reference_law"), ten KDK global steps ("kdk"), the clustered 256^3
workload ("clustered256"), cuFFT timed on the same transforms
("fft_check"), the whole-step roofline ("step_roofline"), the 64-box uneven
ensemble evaluated box by box and batched ("ensemble"), the served request
loop ("served") and the engine's error against the reference build on the
CPU sample ("parity_vs_reference").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

value: Mparticles/s over all ranks with the positions resident in HBM.
e2e:   the same metric through the public C ABI with pinned host buffers
       (positions uploaded and forces read back every step).
With N > 1 (torchrun), every rank evaluates its own independent box (replicas,
weak scaling); no collective is on the data path.
"""
from __future__ import annotations

import argparse
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

METRIC = "Mparticles/s per TreePM force eval (plain vs batched) at rms err≤1e-3; p50/p99 latency"
UNIT = "Mparticles/s"
EPS = 0.05
HEADLINE_LAW = {"law": "gaussian", "rs_split": 0.7, "rsphere": 3.5, "theta": 0.4, "efold": 0.9}
# weakly clustered boxes carry small net forces: the ensemble and the served
# requests open nodes more often to stay under the same error bar
BOX_LAW = {"law": "gaussian", "rs_split": 0.8, "rsphere": 4.0, "theta": 0.3, "efold": 0.9}
REFERENCE_LAW = {"law": "reference", "rs_split": 1.25, "rsphere": 4.0, "theta": 0.3, "efold": 0.9}
WORKLOADS = {
    "scale512": "scale512: 512^3 particles on a 512^3 mesh, L=500 Mpc/h, Zel'dovich field P(k)~k^-2.5, "
                "rms displacement 2 spacings, v=0.5 psi",
    "clustered256": "clustered256: 256^3 particles on a 256^3 mesh, L=200 Mpc/h, Zel'dovich field "
                    "P(k)~k^-2 exp(-(0.5k)^2), rms 1.5 spacings, plus 200 Plummer spheres (a=0.64 cells, "
                    "2000-20000 particles each)",
    "plain64": "plain64: 64^3 particles on a 64^3 mesh, L=100 Mpc/h, Zel'dovich field "
               "P(k)~k^-2 exp(-(0.5k)^2), rms 0.3 spacings",
}
FP32_LANES_PER_SM = 128
# FLOPs charged per evaluated interaction of the walk (the operations of
# AddPar and AddNode, OST/ost.ver2.c:247-293):
# particle-particle 20, particle-node (quadrupole) 65
FLOP_PP, FLOP_PC = 20, 65


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _clock_sampler(path):
    fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except (FileNotFoundError, OSError):
        return None


def _clock_summary(path, device):
    sms, maxs, reasons = [], [], set()
    try:
        for line in open(path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9 or parts[0] != str(device):
                continue
            try:
                sms.append(float(parts[1]))
                maxs.append(float(parts[2]))
            except ValueError:
                continue
            names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
    except OSError:
        pass
    if not sms:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
    return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
            "samples": len(sms)}


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def _ncu_traffic():
    """DRAM bytes per launch of the profiled kernels, from the committed ncu
    summary (profiles/ncu_traffic.txt: '<kernel> <bytes_per_launch> <units>')."""
    out = {}
    try:
        for line in open(os.path.join(ROOT, "profiles", "ncu_traffic.txt")):
            p = line.split()
            if len(p) < 3 or line.startswith("#"):
                continue
            try:
                out[p[0]] = (float(p[-2]), float(p[-1]))
            except ValueError:
                continue
    except OSError:
        pass
    return out


# ---------------------------------------------------------------- CPU arms
SAMPLE_N = 128


def reference_sample(workload):
    """The bounded CPU sample: the benchmark's workload generated at 128^3
    (2.1M particles; the 512^3 field's spectrum and displacement in lattice
    units, or the clustered field's Plummer spheres with the same particle
    counts and scale radius, so the same local densities), one PM +
    tree-correction evaluation through the reference's own
    pmmain/treecorrection."""
    from lageunha_b200 import ic
    return ic.workload(workload, scale=SAMPLE_N)


def sample_name(workload):
    return f"{workload} workload at {SAMPLE_N}^3"


def run_reference_eval(ps):
    from oracle import oracle as O
    t0 = time.perf_counter()
    O.ref_pm_force(ps.n_mesh, ps.indx, ps.offset, 0.9)
    O.ref_tree_force(ps.n_mesh, ps.indx, ps.offset, theta=0.3, rsphere=4.0, eps=EPS, variant=O.VARIANT_A)
    return time.perf_counter() - t0


def _quiet_stdout():
    """The reference prints its stage timers; keep the JSON line alone on stdout."""
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    os.close(devnull)
    return saved


def _restore_stdout(saved):
    sys.stdout.flush()
    os.dup2(saved, 1)
    os.close(saved)


def run_ic(E, ic, n, local):
    """Zel'dovich and second-order initial conditions of n^3 particles with a
    CAMB-like spectrum (sigma_8 = 0.8, 500 Mpc/h box, growth 1/50): noise,
    transforms and records in device memory; each call returns when its work
    is done, so it is timed by the host clock around the call (best of 3)."""
    import torch
    k = np.exp(np.linspace(np.log(1e-3), np.log(50), 400))
    p = 2e4 * (k / 0.02) / (1 + (k / 0.02) ** 3)
    vp = ic.velpot_table(n, 500.0, k, p, growth=1.0 / 50, sigma8=0.8)
    out = torch.empty(n ** 3 * E.DM_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{local}")
    res = {"workload": f"{n}^3 lattice, CAMB-like P(k) table, seed -7", "particles": n ** 3}
    for name, fn in (("zeldovich", lambda: E.ic_zeldovich(n, -7, vp, out=out)),
                     ("2lpt", lambda: E.ic_2lpt(n, -7, vp, vamp2=-0.6, out=out))):
        fn()
        ts = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            ts.append(1e3 * (time.perf_counter() - t0))
        res[name] = {"ms": min(ts), "Mparticles/s": n ** 3 / (min(ts) * 1e-3) / 1e6}
    return res


def cpu_baseline(workload):
    ps = reference_sample(workload)
    saved = _quiet_stdout()
    try:
        dt = run_reference_eval(ps)
    finally:
        _restore_stdout(saved)
    return {"value": ps.np / dt / 1e6, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": f"{sample_name(workload)} ({ps.np} particles), one "
                      f"pmmain + treecorrection of the reference built from its sources (variant A), "
                      f"OpenMP on {os.cpu_count()} host threads, {dt:.1f} s; its FFTs run on the harness's "
                      f"double-precision DFT (oracle/dft.c) in place of FFTW, which is not built",
            "ic_reference": reference_ic_time(128)}


def reference_ic_time(n):
    """The reference's Zel'dovich initial conditions at n^3 on the host: its
    gasdev/ran3 mode loop and its Zeldovich (FFTs through the oracle's double
    DFT in place of FFTW, which is not built)."""
    from oracle import oracle as O
    k2 = np.arange((n // 2) ** 2 + 1, dtype=np.float64)
    rk = 2 * np.pi * np.sqrt(np.maximum(k2, 1.0))
    vp = (0.05 * rk ** -1.0 / rk ** 2 * n ** 3).astype(np.float32)
    t0 = time.perf_counter()
    d = O.ref_ic_noise(n, -7, vp)
    t1 = time.perf_counter()
    O.ref_zeldovich(n, d)
    t2 = time.perf_counter()
    return {"particles": n ** 3, "noise_s": t1 - t0, "zeldovich_s": t2 - t1, "threads": 1}


def run_reference_arm(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import oracle as O
    if not O.ref_available(O.VARIANT_A):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_A.so was not built "
                          "(the reference tree was absent when the oracle was compiled)"}))
        return 0
    ps = reference_sample(args.workload)
    saved = _quiet_stdout()
    try:
        for _ in range(args.warmup):
            run_reference_eval(ps)
        times = [run_reference_eval(ps) for _ in range(args.steps)]
    finally:
        _restore_stdout(saved)
    tot = sum(times)
    value = ps.np * args.steps / tot / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Zel'dovich field" + (" + Plummer spheres" if args.workload == "clustered256" else "")
                + "; no dataset)",
        "config": {"workload": WORKLOADS[args.workload] + f"; bounded CPU sample: the same field at {SAMPLE_N}^3",
                   "n_mesh": ps.n_mesh, "particles": ps.np,
                   "theta": 0.3, "rsphere": 4.0, "epsilon": EPS, "efold": 0.9},
        "latency_ms": {"p50": 1e3 * float(np.percentile(times, 50)), "p99": 1e3 * float(np.percentile(times, 99))},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"{ps.np} particles ({sample_name(args.workload)}) per step, reference pmmain + "
                                   f"treecorrection (variant A) on {os.cpu_count()} host threads; FFTs on "
                                   f"the harness's double-precision DFT (oracle/dft.c), not FFTW"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- engine arm
def run_batched(args, E, ic, law, local, dist=None):
    """The 64-box uneven ensemble: every box through the plain engine one
    after another (each call synchronises, as a caller of the plain engine
    does), then the same boxes as one ensemble (one graph launch per
    evaluation). Both evaluate the same forces with the same law. With N
    ranks every rank takes its share of the boxes (longest processing time
    first); times are the max over ranks."""
    import torch
    from lageunha_b200 import shard
    ws = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    sizes = [ic.ensemble_spec(b)[0] ** 3 for b in range(args.ensemble_boxes)]
    mine = shard.assign_boxes(sizes, ws)[rank]
    t0 = time.time()
    boxes = [ic.ensemble_box(b) for b in mine]
    t_ic = time.time() - t0
    dev = f"cuda:{local}"
    engines = [E.Engine(b.n_mesh, epsilon=EPS, device=local, **law) for b in boxes]
    for e, b in zip(engines, boxes):
        e.load_fixed(b.pos, b.vel)
    # one autotuner run per mesh size (its largest box), shared by the boxes
    # of that size; both arms below use the same shapes
    if not args.no_autotune:
        by_mesh = {}
        for e, b in zip(engines, boxes):
            if b.n_mesh not in by_mesh or b.np > by_mesh[b.n_mesh][1].np:
                by_mesh[b.n_mesh] = (e, b)
        for m, (e, b) in by_mesh.items():
            e.autotune(E.TUNE_FFT | E.TUNE_GROUPS)
            t = e.tuning
            for e2, b2 in zip(engines, boxes):
                if b2.n_mesh == m and e2 is not e:
                    e2.tuning = t
    for e in engines:
        e.sync()
    total = sum(b.np for b in boxes)

    def plain():
        for e in engines:
            e.compute(E.PART_ALL)

    batch = E.Batch(engines)
    plain()
    batch.compute(E.PART_ALL)
    reps = 3
    tp = []
    for _ in range(reps):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        s = time.perf_counter()
        plain()
        tp.append(time.perf_counter() - s)
    tb, tbd = [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        s = time.perf_counter()
        batch.compute(E.PART_ALL)
        tb.append(time.perf_counter() - s)
        tbd.append(batch.last_ms * 1e-3)
    ms_step = None
    cosmo = E.cosmology()
    steps = [0.05 / (float(np.sqrt(np.mean(np.square(b.vel, dtype=np.float64)))) * b.n_mesh) for b in boxes]
    batch.step(cosmo, 5.0, steps)
    ms_step = batch.last_ms
    # accuracy: FP64 Ewald on 1024 targets of a small, a middle and the largest box
    order = sorted(range(len(boxes)), key=lambda i: boxes[i].np)
    errs = []
    batch.compute(E.PART_ALL)
    for i in (sorted({order[0], order[len(order) // 2], order[-1]}) if order else []):
        b, e = boxes[i], engines[i]
        f = e.forces()
        rng = np.random.Generator(np.random.PCG64(1024 + i))
        tg = np.sort(rng.choice(b.np, min(1024, b.np), replace=False)).astype(np.int64)
        few = e.ewald(tg)
        er = np.linalg.norm(f[tg].astype(np.float64) - few, axis=1) / np.linalg.norm(few, axis=1)
        errs.append({"n_lattice": b.n_lattice, "n_mesh": b.n_mesh, "rms": float(np.sqrt(np.mean(er * er))),
                     "p99": float(np.percentile(er, 99))})
    batch.close()
    for e in engines:
        e.close()
    plain_s = shard.max_over_ranks(min(tp), dist, dev)
    batch_s = shard.max_over_ranks(min(tb), dist, dev)
    tbd_max = shard.max_over_ranks(min(tbd), dist, dev)
    ms_step = shard.max_over_ranks(ms_step, dist, dev)
    total = int(shard.sum_over_ranks(float(total), dist, dev))
    return {
        "boxes": args.ensemble_boxes, "boxes_per_rank": len(boxes), "particles": total,
        "lattice_range": [min(ic.ensemble_spec(i)[0] for i in range(args.ensemble_boxes)),
                          max(ic.ensemble_spec(i)[0] for i in range(args.ensemble_boxes))],
        "meshes": sorted({ic.fft_friendly(ic.ensemble_spec(i)[0]) for i in range(args.ensemble_boxes)}),
        "plain_box_by_box": {"value": total / plain_s / 1e6, "ms": plain_s * 1e3},
        "batched": {"value": total / batch_s / 1e6, "ms": batch_s * 1e3, "device_ms": tbd_max * 1e3},
        "speedup": plain_s / batch_s,
        "kdk_step_ms": ms_step,
        "err_vs_ewald": errs,
        "ic_seconds": t_ic,
        "unit": UNIT,
        "timing": "wall clock around each whole-ensemble evaluation after a device synchronize (best of 3, "
                  "max over ranks); device_ms from CUDA events around the ensemble graph launch",
    }


def run_served(args, E, ic, law, local, dist=None):
    """Served solves: seeded Poisson arrivals (mean 200 requests/s) of boxes
    drawn log-uniform in 32^3..256^3 particles with 1-20 global steps each,
    submitted to the request loop at their arrival times; latency = done -
    arrival per request; throughput = particle-steps / (last done - first
    arrival)."""
    from lageunha_b200 import shard
    ws = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    dev = f"cuda:{local}"
    rng = np.random.Generator(np.random.PCG64(5))
    nreq = args.served_requests
    gaps = rng.exponential(1.0 / 200.0, nreq)
    arrivals_all = np.cumsum(gaps) - gaps[0]
    # request r goes to rank r mod N (one server per GPU)
    mine = [r for r in range(nreq) if r % ws == rank]
    arrivals = arrivals_all[mine]
    reqs = []
    t0 = time.time()
    for r in mine:
        rr = np.random.Generator(np.random.PCG64(5000 + r))
        nl = int(round(np.exp(rr.uniform(np.log(32), np.log(256)))))
        nsteps = int(rr.integers(1, 21))
        ns = float(rr.uniform(-2.5, -1.5))
        box = ic.lattice_box(nl, ic.fft_friendly(nl), 5000 + r, ns, 1.0, float(rr.uniform(50, 300)), vel_factor=0.5)
        reqs.append((box, nsteps))
    t_ic = time.time() - t0
    import torch
    pinned = []
    for box, _ in reqs:
        pos = torch.from_numpy(box.pos.view(np.int32)).pin_memory()
        vel = torch.from_numpy(box.vel).pin_memory()
        po = torch.empty((box.np, 3), dtype=torch.int32).pin_memory()
        vo = torch.empty((box.np, 3), dtype=torch.float32).pin_memory()
        pinned.append((pos, vel, po, vo))
    cosmo = E.cosmology()
    srv = E.Server(hbm_cap_bytes=150 * 10 ** 9, max_active=args.served_max_active, device=local)
    # the server claims its contexts' memory before the first arrival, as a
    # serving process does at start-up; not part of any request's latency
    t_res = time.perf_counter()
    if args.served_reserve_gb > 0:
        srv.reserve(int(args.served_reserve_gb * 2 ** 30))
    t_res = time.perf_counter() - t_res
    ids = []
    if dist is not None:
        dist.barrier()
    start = time.perf_counter()
    for r, ((box, nsteps), (pos, vel, po, vo)) in enumerate(zip(reqs, pinned)):
        delay = arrivals[r] - (time.perf_counter() - start)
        if delay > 0:
            time.sleep(delay)
        # steps sized for a 0.05-cell rms drift, as the KDK block does
        vrms = float(np.sqrt(np.mean(np.square(box.vel, dtype=np.float64))))
        ids.append(srv.submit(pos.numpy().view(np.uint32), vel.numpy(), n_mesh=box.n_mesh, nsteps=nsteps, anow=4.0,
                              astep=0.05 / (vrms * box.n_mesh), cosmo=cosmo, pos_out=po.numpy().view(np.uint32),
                              vel_out=vo.numpy(), epsilon=EPS, **law))
    srv.wait(-1, 3600.0)
    infos = [srv.info(i) for i in ids]
    stats = srv.stats()
    srv.close()
    lat = np.array([i.t_done - i.t_submit for i in infos])
    wait = np.array([i.t_admit - i.t_submit for i in infos])
    span = max(i.t_done for i in infos) - min(i.t_submit for i in infos)
    work = sum(box.np * ns for box, ns in reqs)
    failed = sum(1 for i in infos if i.state != E.REQ_DONE)
    if dist is not None and dist.get_world_size() > 1:
        gathered = [None] * dist.get_world_size()
        dist.all_gather_object(gathered, (lat.tolist(), wait.tolist()))
        lat = np.array([x for g in gathered for x in g[0]])
        wait = np.array([x for g in gathered for x in g[1]])
        span = shard.max_over_ranks(span, dist, dev)
        work = shard.sum_over_ranks(float(work), dist, dev)
        failed = int(shard.sum_over_ranks(float(failed), dist, dev))
    return {
        "requests": nreq, "failed": failed, "arrival_rate_per_s": 200,
        "particle_steps": int(work), "value": work / span / 1e6, "unit": "Mparticle-steps/s",
        "span_s": span,
        "latency_ms": {"p50": float(np.percentile(lat, 50) * 1e3), "p99": float(np.percentile(lat, 99) * 1e3)},
        "admission_wait_ms": {"p50": float(np.percentile(wait, 50) * 1e3), "p99": float(np.percentile(wait, 99) * 1e3)},
        "server": stats, "hbm_cap_bytes": 150 * 10 ** 9, "ic_seconds": t_ic,
        "max_active": args.served_max_active, "reserved_gib": args.served_reserve_gb, "reserve_seconds": t_res,
    }


def fft_check(n, grids, ms_engine, local):
    """cuFFT (through torch.fft) on the transforms the engine's FFT stage
    makes: per grid one r2c and one c2r of the n^3 mesh with the Green's
    function applied between them. Only a check: the engine never calls
    cuFFT. Timed with CUDA events, best of 5 after 2 warm-ups."""
    import torch
    dev = f"cuda:{local}"
    x = torch.randn((n, n, n), dtype=torch.float32, device=dev)
    g = torch.rand((n, n, n // 2 + 1), dtype=torch.float32, device=dev)

    def once():
        for _ in range(grids):
            torch.fft.irfftn(torch.fft.rfftn(x) * g, s=(n, n, n))

    for _ in range(2):
        once()
    best = None
    for _ in range(5):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        once()
        b.record()
        torch.cuda.synchronize()
        t = a.elapsed_time(b)
        best = t if best is None else min(best, t)
    del x, g
    torch.cuda.empty_cache()
    return {"ms_engine": ms_engine, "ms_cufft": best, "grids": grids, "mesh": n,
            "transforms": f"{grids} x (r2c + Green + c2r) of {n}^3 float32",
            "engine_over_cufft": (ms_engine / best) if (ms_engine and best) else None}


def step_roofline(npart, n, grids, counters, ms_step, hbm_gbs, fp32_tflops):
    """T_roof = minimal HBM bytes of the HBM-bound stages / measured copy
    bandwidth + walk flops / FP32 peak, against the measured step. Bytes per
    particle (Np = n^3): sort 28 (12 position read + 12 write + 4
    permutation), deposit 12 + 4 per grid, FFT 16 per grid (one read and one
    write per transform), gradient + interpolation 24 + 4 per grid; tree
    build 12 per particle + 64 per node."""
    mesh_pp = n ** 3 / npart
    b = npart * (28 + (12 + 4 * grids * mesh_pp) + 16 * grids * mesh_pp + (24 + 4 * grids * mesh_pp) + 12) + \
        64 * counters["nodes"]
    t_hbm = b / (hbm_gbs * 1e9) * 1e3
    flops = FLOP_PP * counters["pp"] + FLOP_PC * counters["pc"]
    t_fp32 = flops / (fp32_tflops * 1e12) * 1e3
    t_roof = t_hbm + t_fp32
    return {"ms_roofline": t_roof, "ms_hbm_part": t_hbm, "ms_fp32_part": t_fp32, "ms_measured": ms_step,
            "frac": t_roof / ms_step, "bytes": b, "walk_flops": flops,
            "peaks": f"HBM {hbm_gbs:.0f} GB/s (measured copy), FP32 {fp32_tflops:.1f} TFLOP/s (nominal)"}


def run_clustered(args, E, ic, local, dist=None):
    """The clustered 256^3 workload (200 Plummer spheres) with the headline
    law: throughput with positions resident in HBM and the error against
    the FP64 Ewald sum."""
    import torch
    ps = ic.workload("clustered256")
    pu = ps.positions_u32()
    eng = E.Engine(256, epsilon=EPS, device=local, **HEADLINE_LAW)
    stream = torch.cuda.ExternalStream(eng.stream, device=local)
    pos_dev = torch.from_numpy(pu.view(np.int32)).to(f"cuda:{local}")
    f_dev = torch.empty((ps.np, 3), dtype=torch.float32, device=f"cuda:{local}")
    eng.load_fixed(pos_dev)
    if not args.no_autotune:
        eng.autotune(E.TUNE_FFT | E.TUNE_GROUPS)
    for _ in range(3):
        eng.compute(E.PART_ALL)
        eng.forces(f_dev)
    steps = max(3, min(args.steps, 10))
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    stages = {k: 0.0 for k in E.STAGES}
    a.record(stream)
    for _ in range(steps):
        eng.compute(E.PART_ALL)
        eng.forces(f_dev)
        st = eng.stage_times()
        for k in stages:
            stages[k] += st.get(k, 0.0)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    out = {"workload": WORKLOADS["clustered256"], "law": HEADLINE_LAW, "steps": steps, "ms_per_step": ms,
           "value": ps.np / (ms * 1e-3) / 1e6, "unit": UNIT,
           "stage_ms": {k: v / steps for k, v in stages.items()}, "counters": eng.counters()}
    if not args.no_ewald:
        rng = np.random.Generator(np.random.PCG64(4096))
        tg = np.sort(rng.choice(ps.np, 4096, replace=False)).astype(np.int64)
        few = eng.ewald(tg)
        fh = f_dev.cpu().numpy()
        e = np.linalg.norm(fh[tg].astype(np.float64) - few, axis=1) / np.linalg.norm(few, axis=1)
        out["err_vs_ewald"] = {"rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99)),
                               "targets": 4096}
    eng.close()
    del pos_dev, f_dev
    torch.cuda.empty_cache()
    return out


def parity_vs_reference(E, local, workload):
    """The engine with the reference's law on the CPU sample (the workload at 128^3)
    against the reference's own pmmain + treecorrection built from its
    sources (variant B, the three one-line fixes): per-particle relative
    force error, every particle."""
    from oracle import oracle as O
    if not O.ref_available(O.VARIANT_B):
        return {"unavailable": "oracle/_ref/libref_B.so was not built"}
    ps = reference_sample(workload)
    with E.Engine(ps.n_mesh, epsilon=EPS, device=local, **REFERENCE_LAW) as eng:
        eng.load_fixed(ps.positions_u32())
        eng.compute(E.PART_ALL)
        f = eng.forces()
    saved = _quiet_stdout()
    try:
        fr = O.ref_pm_force(ps.n_mesh, ps.indx, ps.offset, 0.9).astype(np.float64) + \
            O.ref_tree_force(ps.n_mesh, ps.indx, ps.offset, theta=0.3, rsphere=4.0, eps=EPS, variant=O.VARIANT_B)
    finally:
        _restore_stdout(saved)
    e = O.rel_err(f, fr)
    return {"sample": f"{sample_name(workload)}, {ps.np} particles, reference law (theta 0.3, rsphere 4)",
            "oracle": "reference pmmain + treecorrection built from its sources (variant B)",
            "rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99)), "particles": ps.np}


def run_engine_arm(args):
    import torch
    from lageunha_b200 import engine as E
    from lageunha_b200 import ic

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    ps = ic.workload(args.workload, scale=args.scale,
                     device=f"cuda:{local}" if args.workload == "scale512" else None)
    n = ps.n_mesh
    pu = ps.positions_u32()
    npart = ps.np

    law = REFERENCE_LAW if args.law == "reference" else HEADLINE_LAW
    eng = E.Engine(n, epsilon=EPS, device=local, **law)
    stream = torch.cuda.ExternalStream(eng.stream, device=local)
    pos_dev = torch.from_numpy(pu.view(np.int32)).to(f"cuda:{local}")
    f_dev = torch.empty((npart, 3), dtype=torch.float32, device=f"cuda:{local}")
    eng.load_fixed(pos_dev)
    # launch shapes from the autotuner (untimed; forces are measured after it)
    tuning = eng.autotune(E.TUNE_FFT | E.TUNE_GROUPS) if not args.no_autotune else None

    def step_dev():
        eng.compute(E.PART_ALL)
        eng.forces(f_dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step_dev()
    launches = eng.launch_count() + 1  # compute + the scatter to caller order
    stages = {k: 0.0 for k in E.STAGES}

    clk_path = os.path.join(tempfile.gettempdir(), f"tpm_clocks_{rank}.csv")
    sampler = _clock_sampler(clk_path)
    time.sleep(0.3)
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    per_step = []
    t_start.record(stream)
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step_dev()
        b.record(stream)
        per_step.append((a, b))
        st = eng.stage_times()
        for k in stages:
            stages[k] += st.get(k, 0.0)
    t_end.record(stream)
    barrier()
    if sampler:
        sampler.terminate()
        sampler.wait()
    ms_total = t_start.elapsed_time(t_end)
    lat = [a.elapsed_time(b) for a, b in per_step]
    counters = eng.counters()
    ms_max = ms_total
    if dist is not None:
        t = torch.tensor([ms_total], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    ms_step = ms_max / args.steps
    value = ws * npart / (ms_step * 1e-3) / 1e6

    # ---- e2e: host buffers through the public API, copies in the timed region
    pos_host = torch.from_numpy(pu.view(np.int32).copy()).pin_memory()
    f_host = torch.empty((npart, 3), dtype=torch.float32).pin_memory()

    f_host2 = torch.empty((npart, 3), dtype=torch.float32).pin_memory()

    def step_e2e():
        eng.load_fixed(pos_host)
        eng.compute(E.PART_ALL)
        eng.forces(f_host)

    def timed(body):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        body()
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    def sync_steps():
        for _ in range(args.steps):
            step_e2e()

    def streamed_steps():
        # every step copies its positions in and its forces out; a step's
        # copies run during its neighbours' evaluations (two in flight)
        pos_np, outs, tickets = pos_host.numpy(), (f_host.numpy(), f_host2.numpy()), []
        for k in range(args.steps):
            tickets.append(eng.stream_submit(pos_np, outs[k % 2]))
            if k >= 1:
                eng.stream_wait(tickets[k - 1])
        eng.stream_wait(tickets[-1])

    step_e2e()
    ms_e2e_sync = timed(sync_steps)
    streamed_steps()
    ms_e2e = timed(streamed_steps)
    e2e_value = ws * npart * args.steps / (ms_e2e * 1e-3) / 1e6
    e2e_sync_value = ws * npart * args.steps / (ms_e2e_sync * 1e-3) / 1e6

    # ---- accuracy against the FP64 Ewald sum on a 4096-particle subsample (untimed)
    err = None
    if not args.no_ewald:
        fh = f_host.numpy()
        rng = np.random.Generator(np.random.PCG64(4096))
        tg = np.sort(rng.choice(npart, 4096, replace=False)).astype(np.int64)
        few = eng.ewald(tg)
        e = np.linalg.norm(fh[tg].astype(np.float64) - few, axis=1) / np.linalg.norm(few, axis=1)
        err = {"rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99)), "targets": 4096}

    clocks = _clock_summary(clk_path, local)
    peaks = _peaks()

    # ---- the reference's law in the same run (the drop-in parity mode)
    ref_law = None
    if args.law != "reference" and not args.no_reference_law:
        eng.set_params(law="reference", rsphere=REFERENCE_LAW["rsphere"])
        for _ in range(2):
            step_dev()
        barrier()
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        r0.record(stream)
        for _ in range(args.steps):
            step_dev()
        r1.record(stream)
        barrier()
        ms_ref = r0.elapsed_time(r1) / args.steps
        ref_law = {"value": ws * npart / (ms_ref * 1e-3) / 1e6, "ms_per_step": ms_ref, **REFERENCE_LAW}
        if err is not None:
            fr = f_dev.cpu().numpy()
            e = np.linalg.norm(fr[tg].astype(np.float64) - few, axis=1) / np.linalg.norm(few, axis=1)
            ref_law["err_vs_ewald"] = {"rms": float(np.sqrt(np.mean(e * e))), "p99": float(np.percentile(e, 99))}

    # ---- roofline of the dominant kernel
    per = {k: v / args.steps for k, v in stages.items()}
    dominant = max(per, key=per.get)
    sm_max = clocks.get("sm_max_mhz") or peaks.get("sm_max_mhz") or 1965.0
    nsm = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = nsm * FP32_LANES_PER_SM * 2 * sm_max * 1e6 / 1e12
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    traffic = _ncu_traffic()
    if dominant == "tree_walk":
        flops = FLOP_PP * counters["pp"] + FLOP_PC * counters["pc"]
        achieved = flops / (per["tree_walk"] * 1e-3) / 1e12
        tr = traffic.get("k_tree_walk")
        roofline = {"bound": "fp32", "kernel": "k_tree_walk", "achieved": achieved, "peak": fp32_peak,
                    "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                    "peak_source": f"nominal FP32 {nsm} SMs x 128 lanes x 2 x {sm_max:.0f} MHz "
                                   "(no measured FP32 figure; HBM peak of measured)",
                    "traffic": (tr[0] * npart / tr[1]) if tr else None,
                    "algorithmic": f"{FLOP_PP} flop per particle-particle and {FLOP_PC} per particle-node "
                                   f"interaction evaluated: {counters['pp']} and {counters['pc']} per launch"}
    else:
        roofline = {"bound": "hbm", "kernel": dominant, "achieved": None, "peak": hbm_peak, "unit": "GB/s"}
    # HBM-bound stages: algorithmic bytes per particle (each stage's minimal reads and
    # writes): positions read once and forces written once per stage that uses them, and
    # each of the PM's grids (two interlaced ones for the Gaussian law) written by the
    # deposit, read and written once per transform, read by fda4
    grids = 1 if args.law == "reference" else 2
    mesh_pp = 4 * n ** 3 / npart
    bytes_pp = {"sort": 28 + 5 * 32, "deposit": 12 + grids * mesh_pp, "fft": grids * 4 * mesh_pp,
                "fda4": 24 + grids * mesh_pp}
    hbm_stages = {}
    for k, b in bytes_pp.items():
        if per.get(k, 0) > 0:
            gbs = b * npart / (per[k] * 1e-3) / 1e9
            hbm_stages[k] = {"ms": per[k], "GB/s": gbs, "frac": gbs / hbm_peak}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Zel'dovich field" + (" + Plummer spheres" if args.workload == "clustered256" else "")
                + "; no dataset)",
        "config": {"workload": WORKLOADS[args.workload] + (f", at {n}^3" if args.scale else "") +
                               "; one TreePM force evaluation per step, plain engine",
                   "n_mesh": n, "particles_per_gpu": npart, "epsilon": EPS, **law,
                   "l2": f"inputs larger than L2: {12 * npart / 1e6:.0f} MB of positions, "
                         f"{4 * n ** 3 / 1e6:.0f} MB mesh",
                   "parallelism": f"replicas x{ws}"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "stage_ms": per,
        # the PM chain (deposit, fft, fda4) runs on a second stream beside the
        # tree build, so stage_ms' tree_build spans that whole phase (from the
        # deposit's start to the tree's end) and the stages do not add up
        "phase_ms": {"sort": per.get("sort", 0.0), "pm_chain_beside_tree_build": per.get("tree_build", 0.0),
                     "tree_walk": per.get("tree_walk", 0.0),
                     "finish_and_gaps": ms_step - per.get("sort", 0.0) - per.get("tree_build", 0.0)
                     - per.get("tree_walk", 0.0)},
        "hbm_stages": hbm_stages,
        "counters": counters,
        "err_vs_ewald": err,
        "reference_law": ref_law,
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 12 * npart,
                "d2h_bytes_per_step": 12 * npart,
                "api": "tpm_stream_submit / tpm_stream_wait from pinned host buffers, two steps in flight",
                "synchronous": {"value": e2e_sync_value, "unit": UNIT,
                                "api": "tpm_load_fixed + tpm_compute_forces + tpm_read_forces per step"}},
        "gpu_launches": launches * args.steps,
        "autotune": tuning,
        "clocks": {"sm_mhz": clocks.get("sm_mhz"), "sm_max_mhz": clocks.get("sm_max_mhz"),
                   "reasons": clocks.get("reasons", [])},
    }
    # ---- cuFFT on the same transforms, as a check of the hand-written FFT
    line["fft_check"] = fft_check(n, grids, per.get("fft"), local)
    # ---- the whole step against its roofline: the HBM time of the stages'
    # minimal bytes plus the FP32 time of the walk's counted flops
    line["step_roofline"] = step_roofline(npart, n, grids, counters, ms_step, hbm_peak, fp32_peak)
    # ---- KDK global steps of the same box (drag, forces, kicks, drift),
    # velocities of the workload, anow from 5; the step is sized so that the
    # first drift moves particles by 0.05 cells rms (0.02 for a cold start)
    cosmo = E.cosmology()
    eng.set_params(**law)
    vel_dev = torch.from_numpy(ps.vel).to(f"cuda:{local}")
    eng.load_fixed(pos_dev, vel_dev)
    vrms = float(np.sqrt(np.mean(np.square(ps.vel, dtype=np.float64))))
    astep = 0.05 / (vrms * n) if vrms > 0 else 0.02
    eng.step(cosmo, 5.0, astep, 0)
    nk = max(1, args.kdk_steps)
    barrier()
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for s in range(nk):
        eng.step(cosmo, 5.0 + astep * (1 + s), astep, 1 + s)
    k1.record(stream)
    barrier()
    line["kdk"] = {"steps": nk, "astep": astep, "anow": 5.0, "ms_per_step": k0.elapsed_time(k1) / nk,
                   "value": ws * npart * nk / (k0.elapsed_time(k1) * 1e-3) / 1e6, "unit": UNIT}
    if err is not None and nk >= 1:
        # accuracy after the steps, on the moved particles
        eng.compute(E.PART_ALL)
        fk = eng.forces()
        fe = eng.ewald(tg)
        ek = np.linalg.norm(fk[tg].astype(np.float64) - fe, axis=1) / np.linalg.norm(fe, axis=1)
        line["kdk"]["err_vs_ewald"] = {"rms": float(np.sqrt(np.mean(ek * ek))), "p99": float(np.percentile(ek, 99))}
    eng.close()
    del pos_dev, f_dev, vel_dev
    torch.cuda.empty_cache()
    if args.workload != "clustered256" and not args.no_clustered:
        line["clustered256"] = run_clustered(args, E, ic, local, dist)
    if not args.no_ic:
        line["ic"] = run_ic(E, ic, n, local)
    box_law = REFERENCE_LAW if args.law == "reference" else BOX_LAW
    if not args.no_batched:
        line["ensemble"] = {"law": box_law, **run_batched(args, E, ic, box_law, local, dist)}
    if not args.no_served:
        line["served"] = {"law": box_law, **run_served(args, E, ic, box_law, local, dist)}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
        line["parity_vs_reference"] = parity_vs_reference(E, local, args.workload)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="scale512", choices=["clustered256", "plain64", "scale512"])
    ap.add_argument("--scale", type=int, default=None,
                    help="mesh size of a smaller instance of the workload (profiling captures)")
    ap.add_argument("--law", default="gaussian", choices=["gaussian", "reference"],
                    help="force law of the headline (gaussian: rms <= 1e-3 vs Ewald)")
    ap.add_argument("--no-reference-law", action="store_true")
    ap.add_argument("--no-ewald", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ic", action="store_true", help="skip the initial-conditions block")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-box ensemble block")
    ap.add_argument("--no-served", action="store_true", help="skip the served request-loop block")
    ap.add_argument("--ensemble-boxes", type=int, default=64)
    ap.add_argument("--served-requests", type=int, default=32)
    ap.add_argument("--served-max-active", type=int, default=64,
                    help="requests the server runs at once (the rest wait in arrival order)")
    ap.add_argument("--served-reserve-gb", type=float, default=32.0,
                    help="device memory (GiB) the server claims before the first request arrives")
    ap.add_argument("--kdk-steps", type=int, default=None,
                    help="timed KDK global steps of the workload (default: 10 at scale, else 1)")
    ap.add_argument("--no-clustered", action="store_true", help="skip the clustered 256^3 block")
    ap.add_argument("--no-autotune", action="store_true", help="keep the built-in launch shapes")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.kdk_steps is None:
        args.kdk_steps = 10 if args.workload == "scale512" else 1
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_engine_arm(args)


if __name__ == "__main__":
    sys.exit(main())
