"""Benchmark: lensing maps of the 1000-halo, 4096x4096 workload on B200.

One step = kappa, gamma1, gamma2, mu and the potential (x D_LS/D_OS) of the 4096^2 grid
over 300"x300" for the seeded 1000-halo catalogue (4 cluster-scale + 996 galaxy-scale
cut-dPIE halos), computed by the fused lens-maps kernel (LT_FP32C by default).  Metric:
halo x pixel evaluations per second, counting the Hessian and the potential sum once each
per (halo, pixel) pair.  The same JSON line also carries LT_FP64 on the same step, the
posterior-batch workload (bayes rows applied on the device + one batch launch; maps/s
against the reference's loop of one launch per map and set), the serving workload
(p50/p99 latency, maps/s against one plain call per request) and the delensing + chi2
workload (models/s against the reference's CPU code).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp32c|fp64]
                  [--impl ours|reference] [--skip-batch] [--skip-serving] [--skip-chi2]
                  [--only-batch --batch-sets N]

--impl reference times the reference's own CPU code (oracle/_ref: gradient2_grid_CPU and
the reference potential kernel compiled for the host) on all host cores, on a bounded
band of rows of the same workload; its line also carries `reference_gpu`, the reference's
own GPU kernels built for sm_100a (type_t double and float) timed on the full workload on
this GPU.  Multi-GPU (torchrun): independent replicas, one per
GPU (the maps are independent; no collective on the data path); value = all ranks' evals
/ max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "maps_1000h_4096"
METRIC = "halo x pixel evals/s (Hessian + potential, lens maps kappa/gamma1/gamma2/mu/psi)"
# the metric of the single-kind runs (--maps), which are profiling cases, not the bench line
METRIC_OF_MAPS = {"all": METRIC, "hessian": "halo x pixel evals/s (Hessian, maps kappa/gamma1/gamma2/mu)",
                  "potential": "halo x pixel evals/s (potential)",
                  "deflection": "halo x pixel evals/s (deflection x/y)"}
# weighted flop census per pair of the reference's own formulas (fixed convention:
# +,-,* = 1, fma = 2, div = sqrt = 4, log = atan2 = 20): dPIE Hessian 182
# (src/gradient2.cpp:92-167, :54-83) + dPIE potential 760 (src/potential_GPU.cu:47-116 with
# src/lt_math_GPU.cuh).  The library's forms execute less than that (the potential goes
# through the deflection), so this census is the roofline only of the modes measured below.
FLOPS_PER_PAIR = 182 + 760
# Work per pair that the default step's dominant kernel (grid32c_kernel<OP_HESS|OP_POT>,
# FP32C, the 1000-halo catalogue) executes, from ncu's counters on the 1024^2 case of the
# same catalogue (summary under profiles/): issued thread instructions (warp instructions
# x 32 per pair) and FP32 flops (fadd + fmul + 2 ffma).  The kernel is issue-bound.  The
# figures hold for the build whose KERNEL_SOURCES hash to INST_SOURCES_SHA; the bench line
# says whether the timed build is that one.
KERNEL_SOURCES = ("lt_eval.cuh", "lt_profiles32.cuh", "lt_profiles64.cuh", "lt_bulk.cuh", "lt_grid32.cu",
                  "lt_grid.cuh", "lt_halo.h", "lt_pack.h")
INST_SOURCES_SHA = "8e3ea4f58e55c5d4"
INST_PER_PAIR_FP32C_LENS = 150.6
FP32_FLOPS_PER_PAIR_FP32C_LENS = 126.4
# DRAM bytes (read + write) of one launch of that kernel at 4096^2, from a single-pass ncu
# capture of this bench's own launch (summary under profiles/)
TRAFFIC_FP32C_LENS_4096 = 14311424 + 630767872


def _package():
    if "lenstool_hpc_b200" in sys.modules:
        return sys.modules["lenstool_hpc_b200"]
    pkg_dir = ROOT / "lenstool-hpc_b200"
    spec = importlib.util.spec_from_file_location("lenstool_hpc_b200", pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lenstool_hpc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", self.gpu_id], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
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
        sm, mx, reasons = [], 0., set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx = max(mx, float(p[1]))
            except ValueError:
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(p.read_text())
    except Exception:
        return {}


def reference_cpu(steps, warmup, rows=None):
    """Reference CPU code on bands of rows of the workload; returns (evals/s, info).

    gradient2_grid_CPU spreads its rows over the OpenMP threads (`#pragma omp for` over
    rows, src/grid_gradient2_CPU.cpp:68-70), so every band has as many rows as there are
    threads (each thread one row of 4096 pixels); the potential kernel runs over the same
    pixels with a dynamic schedule.  Two bands, at a quarter and three quarters of the
    field's height, so that the sample is not one strip through the centre."""
    import oracle
    lt = _package()
    from lenstool_hpc_b200 import catalog
    ref = oracle.RefLib()
    cat, g = catalog.workload(WORKLOAD)
    threads = os.cpu_count()
    rows = rows or threads
    bands = [catalog.Grid(g.xmin, g.xmax, g.ymin, g.ymax, g.nx, rows, 0, j0, dx=g.dx, dy=g.dy)
             for j0 in (g.ny // 4 - rows // 2, 3 * g.ny // 4 - rows // 2)]
    times, th, tp = [], [], []
    for it in range(warmup + steps):
        h = p = 0.
        for band in bands:
            t0 = time.perf_counter()
            ref.hess_grid(cat, band)
            t1 = time.perf_counter()
            px, py = band.coords()
            ref.pot81_points(cat, px, py)
            h += t1 - t0
            p += time.perf_counter() - t1
        if it >= warmup:
            times.append(h + p)
            th.append(h)
            tp.append(p)
    npix = sum(b.npix for b in bands)
    evals = 2 * npix * cat.n
    v = evals / float(np.mean(times))
    sample = (f"{len(bands)} bands of {rows} rows x {g.nx} px x {cat.n} halos of the workload (gradient2_grid_CPU "
              f"+ the reference potential kernel on the host), {threads} OpenMP threads, one row per thread")
    return v, {"value": v, "unit": "evals/s", "cores": threads, "kind": "reference", "sample": sample,
               "threads_busy": {"hessian": min(threads, rows), "potential": threads},
               "hessian_evals_per_s": npix * cat.n / float(np.mean(th)),
               "potential_evals_per_s": npix * cat.n / float(np.mean(tp)),
               "seconds_per_sample": float(np.mean(times))}


def reference_gpu(reps=1, band_rows=32):
    """The reference's own GPU kernels (src/gradient2_GPU.cu, src/potential_GPU.cu, built
    for sm_100a from its sources) on the full workload, one Hessian and one potential
    launch per step as its wrappers make them (32 x 16 threads, one pixel per thread);
    evals counted as for `value`.  Builds: fp64_stock (the flags of the reference's
    default build: -O3 -use_fast_math, type_t = double), fp32_stock (the same with
    type_t = float), and fp64 / fp32 with -O3 alone.  Each build's error is measured
    against the reference CPU FP64 code on a band of rows."""
    import oracle
    from lenstool_hpc_b200 import catalog
    cat, g = catalog.workload(WORKLOAD)
    band = catalog.Grid(g.xmin, g.xmax, g.ymin, g.ymax, g.nx, band_rows, 0, g.ny // 2, dx=g.dx, dy=g.dy)
    bgrid = catalog.Grid(g.xmin, g.xmax, g.ymin + (g.ny // 2) * g.dy, g.ymax, g.nx, band_rows, dx=g.dx, dy=g.dy)
    cpu_h = cpu_p = None
    out = {"workload": WORKLOAD, "launch": "reference kernels, 32x16 threads, one pixel per thread"}
    for build in ("fp64_stock", "fp32_stock", "fp64", "fp32"):
        try:
            lib = oracle.RefGpuLib(build)
            th, _ = lib.grid("hessian", cat, g, reps=reps, want=False)
            tp, _ = lib.grid("potential", cat, g, reps=reps, want=False)
            _, h = lib.grid("hessian", cat, bgrid, reps=1)
            _, p = lib.grid("potential", cat, bgrid, reps=1)
        except (FileNotFoundError, RuntimeError, OSError) as ex:
            out[build] = {"unavailable": str(ex)}
            continue
        if cpu_h is None:
            ref = oracle.RefLib()
            cpu_h = ref.hess_grid(cat, band)
            px, py = band.coords()
            cpu_p = ref.pot81_points(cat, px, py).reshape(band_rows, g.nx)

        def err(a, b):
            rms = np.sqrt(np.mean(b * b))
            return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), rms)))
        evals = 2. * g.nx * g.ny * cat.n
        out[build] = {"hessian_ms": th, "potential_ms": tp, "evals_per_s": evals / ((th + tp) / 1e3),
                      "max_rel_err_vs_reference_cpu_fp64": {"hessian": max(err(h[k], cpu_h[k]) for k in range(4)),
                                                            "potential": err(p[0], cpu_p)}}
    return out


def _percentile(xs, q):
    return float(np.percentile(np.asarray(xs, np.float64), q)) if len(xs) else None


def bench_posterior_batch(ctx, precision, steps, warmup, n_sets=512, plain_sample=48, e2e=True):
    """Posterior-batch workload: n_sets bayes.dat-style rows (seeded Gaussian 5% perturbations
    of every halo's x, y, emass, theta, rcore, vdisp, rcut) of the 200-halo model (2 cluster
    + 198 galaxy halos), each on a grid drawn from {512^2, 1024^2, 2048^2} over the
    200"x200" field; outputs mu and kappa per set.  One step: the rows (resident in HBM)
    applied to the sets' resident catalogues (lt_bayes_apply, one launch) and all sets in
    one graph-captured persistent launch (lt_batch).  Compared with the reference's
    bayes-map loop: one launch per map and set (upload, compute, copy back, release)."""
    import torch
    lt = _package()
    from lenstool_hpc_b200 import bayes, catalog
    rng = np.random.Generator(np.random.PCG64(20261203 + 2))
    model = bayes.model_from_parameters(catalog.cluster_galaxy_parameters(2, 198, 20261203))
    B = bayes
    cols = bayes.columns_from_free([{B.X, B.Y, B.EMASS, B.THETA, B.RCORE, B.VDISP, B.RCUT}] * model.n)
    sizes = rng.choice([512, 1024, 2048], n_sets)
    rows = bayes.synthetic_rows(model, cols, n_sets, rng)
    base = bayes.catalog_from_state(model, bayes.base_state(model))
    grids = {n: catalog.Grid.square(100., int(n)) for n in (512, 1024, 2048)}
    dls, dos, _ = lt.cosmo_distances(0.35, 1.5)
    D = dls / dos
    kinds = ("mu", "kappa")
    cats = [ctx.upload(base) for _ in range(n_sets)]
    post = ctx.bayes(model, cols)
    rows_dev = torch.tensor(rows, device="cuda")
    outs = [{k: torch.empty((int(n), int(n)), dtype=torch.float64, device="cuda") for k in kinds} for n in sizes]
    reqs = [lt.Request(c, grids[int(n)], o, dlsds=D) for c, n, o in zip(cats, sizes, outs)]
    tune = None
    if precision == "fp32c":
        # the Hessian kernel configuration tuned on the model's catalogue (the batch takes
        # its pixels per thread and CTAs per SM)
        ppt, cps, tms = ctx.autotune(cats[0], precision, "hessian", grid_n=512)
        tune = dict(ctx.kernel_config(precision, "hessian"), ms_at_512=tms)
    batch = ctx.batch(reqs, precision=precision)
    evals = float(sum(int(n) * int(n) for n in sizes)) * base.n
    stream = torch.cuda.Stream()
    for _ in range(warmup):
        post.apply(rows_dev, cats, stream)
        batch.launch(stream)
    ctx.synchronize(stream)
    ctx.recompute_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = lt.launch_count()
    e0.record(stream)
    for _ in range(steps):
        post.apply(rows_dev, cats, stream)
        batch.launch(stream)
    e1.record(stream)
    ctx.synchronize(stream)
    launches = lt.launch_count() - n0
    dt = e0.elapsed_time(e1) / 1e3 / steps
    recomputed = ctx.recompute_count()
    npix_all = float(sum(int(n) * int(n) for n in sizes)) * steps
    res = {"workload": f"posterior_batch: {n_sets} bayes rows x {base.n} halos, grids U{{512,1024,2048}}^2, "
                       f"mu+kappa", "precision": precision, "maps_per_s": 2 * n_sets / dt, "sets_per_s": n_sets / dt,
           "evals_per_s": evals / dt, "ms_per_step": dt * 1e3, "gpu_launches_per_step": launches / steps,
           "evals_per_step": evals, "l2": f"outputs {2 * 8 * evals / base.n / 1e9:.1f} GB per step > L2",
           "step": "lt_bayes_apply of the rows (HBM) + one lt_batch graph",
           "shape": dict(batch.config(), autotuned=tune),
           "pixels_recomputed_fp64": recomputed / npix_all}
    # the sets as host catalogues (the reference's host-side row update), for the plain loop
    plain_sample = min(plain_sample, n_sets)
    sets = [bayes.catalog_from_state(model, bayes.reference_state(model, (), cols, rows[i]))
            for i in range(plain_sample)]
    # the reference's bayes-map loop (utils/maps/main.cpp:428-587): one launch per map and
    # set, each with its own upload, Hessian sum, copy back to pageable host memory and
    # release; a sample of the sets, scaled to all sets by their halo x pixel evaluations.
    # Also timed: both maps from one call per set (the fused epilogue, same Hessian sum).
    plain, fused = {}, {}
    idx = list(range(plain_sample))
    sample_evals = float(sum(int(sizes[i]) ** 2 for i in idx)) * base.n
    for prec in ("fp64", precision):
        host = {i: {k: np.empty((int(sizes[i]), int(sizes[i]))) for k in kinds} for i in idx}
        c = ctx.upload(sets[0])
        ctx.hessian_maps(c, grids[int(sizes[0])], list(kinds), precision=prec, dlsds=D, out=list(host[0].values()))
        c.release()
        t0 = time.perf_counter()
        for k in kinds:
            for i in idx:
                c = ctx.upload(sets[i])
                ctx.hessian_maps(c, grids[int(sizes[i])], [k], precision=prec, dlsds=D, out=[host[i][k]])
                c.release()
        t = time.perf_counter() - t0
        plain[prec] = {"maps_per_s": 2 * n_sets / (t * evals / sample_evals), "sample_sets": len(idx),
                       "sample_s": t}
        t0 = time.perf_counter()
        for i in idx:
            c = ctx.upload(sets[i])
            ctx.hessian_maps(c, grids[int(sizes[i])], list(kinds), precision=prec, dlsds=D,
                             out=list(host[i].values()))
            c.release()
        t = time.perf_counter() - t0
        fused[prec] = {"maps_per_s": 2 * n_sets / (t * evals / sample_evals), "sample_s": t}
    res["one_map_per_launch"] = plain
    res["two_maps_per_call"] = fused
    res["speedup_vs_one_map_per_launch_fp64"] = res["maps_per_s"] / plain["fp64"]["maps_per_s"]
    res["speedup_vs_one_map_per_launch_same_precision"] = res["maps_per_s"] / plain[precision]["maps_per_s"]
    res["speedup_vs_two_maps_per_call_fp64"] = res["maps_per_s"] / fused["fp64"]["maps_per_s"]
    try:
        import psutil
        host_free = psutil.virtual_memory().available
    except Exception:
        host_free = 0
    if e2e and host_free < 3 * 2 * 8 * evals / base.n:
        res["e2e"] = {"skipped": f"host memory available {host_free / 1e9:.0f} GB < 3x the maps"}
        e2e = False
    if e2e:
        # end to end through the public API: the rows from host memory applied to the
        # resident catalogues (lt_bayes_apply), every set served by the serving loop with its
        # maps delivered to pinned host memory while later sets compute.  The catalogue
        # slots, the host buffers and the server are set up outside the timed region.
        batch.destroy()
        batch = None
        host = [{k: torch.empty((int(n), int(n)), dtype=torch.float64, pin_memory=True) for k in kinds}
                for n in sizes]
        with ctx.server(precision=precision, slots=64, window=8, output_bytes=8 << 30) as srv:
            srv.wait(srv.submit(lt.Request(cats[0], grids[512], {"kappa": host[0]["kappa"][:512, :512].contiguous()},
                                           dlsds=D)))
            t0 = time.perf_counter()
            post.apply(rows, cats)
            ctx.synchronize()
            tickets = [srv.submit(lt.Request(c, grids[int(n)], h, dlsds=D)) for c, n, h in zip(cats, sizes, host)]
            for t in tickets:
                srv.wait(t, 3600.)
            te = time.perf_counter() - t0
            for t in tickets:
                srv.release(t)
        ntheta = int(np.sum(cols[:, 0] == bayes.THETA))
        res["e2e"] = {"maps_per_s": 2 * n_sets / te,
                      "h2d_bytes_per_step": int(rows.nbytes + n_sets * (16 * ntheta + 24)),
                      "d2h_bytes_per_step": int(2 * 8 * evals / base.n),
                      "note": "bayes rows from host memory applied on the device (lt_bayes_apply) + every set "
                              "served (lt_server) with its maps copied to pinned host memory while later sets "
                              "compute"}
        res["e2e"]["speedup_vs_one_map_per_launch_fp64"] = res["e2e"]["maps_per_s"] / plain["fp64"]["maps_per_s"]
    if batch is not None:
        batch.destroy()
    post.destroy()
    for c in cats:
        c.release()
    return res


def bench_serving(ctx, precision, n_requests=96, rate=200.0, plain_sample=None, seed=20261203 + 4):
    """Serving workload: Poisson arrivals at `rate` req/s of requests drawn uniformly from
    {deflection map, kappa/gamma1/gamma2/mu maps, chi2}, grids U{512^2, 1024^2, 2048^2,
    4096^2}.  Map requests use catalogues with log-uniform(50, 5000) halos (1% cluster-scale)
    resident in HBM; chi2 requests one of 8 perturbed models of the 200-halo catalogue
    against 40 image systems (as the chi2 workload).  The serving loop's p50/p99 latency
    (submission to results in HBM) and throughput, against the same requests as one plain
    FP64 call each."""
    import torch
    lt = _package()
    from lenstool_hpc_b200 import catalog
    from lenstool_hpc_b200.images import generate_systems
    rng = np.random.Generator(np.random.PCG64(seed))
    pool = []
    for i in range(12):
        n = int(round(np.exp(rng.uniform(np.log(50.), np.log(5000.)))))
        nc = max(1, int(round(0.01 * n)))
        pool.append(catalog.cluster_galaxy_catalog(nc, n - nc, seed + 100 + i))
    dcats = [ctx.upload(c) for c in pool]
    frame = (-100., 100., -100., 100.)
    base = catalog.cluster_galaxy_catalog(2, 198, 20261203)
    dbase = ctx.upload(base)
    ic = int(np.argmax(base.b0))
    dls, dos, _ = lt.cosmo_distances(0.35, 1.5)
    D = dls / dos
    systems = generate_systems(lambda bx, by, dr: ctx.delense(dbase, frame, 2048, bx, by, dr), 40, 20261203 + 3,
                               dr=D, centre=(base.position_x[ic], base.position_y[ic]), source_radius=10.)
    models = [ctx.upload(catalog.perturb_catalog(base, rng)) for _ in range(8)]
    kinds_of = (("deflection_x", "deflection_y"), ("kappa", "gamma1", "gamma2", "mu"), ())
    reqs = []
    for i in range(n_requests):
        k = int(rng.integers(3))
        n = int(rng.choice([512, 1024, 2048, 4096]))
        c = int(rng.integers(len(pool) if k < 2 else len(models)))
        reqs.append((k, n, c))
    gaps = rng.exponential(1.0 / rate, n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    outs = [{kk: torch.empty((n, n), dtype=torch.float64, device="cuda") for kk in kinds_of[k]} for k, n, c in reqs]
    halos = lambda k, c: pool[c].n if k < 2 else base.n  # noqa: E731
    evals = float(sum(n * n * halos(k, c) for k, n, c in reqs))
    nmaps = sum(len(kinds_of[k]) for k, n, c in reqs)
    nchi = sum(1 for k, n, c in reqs if k == 2)

    def run(arr):
        with ctx.server(precision=precision, slots=64, window=8, output_bytes=8 << 30) as srv:
            # warm-up request (the loop kernel's first launch)
            w = {"kappa": torch.empty((64, 64), dtype=torch.float64, device="cuda")}
            srv.wait(srv.submit(lt.Request(dcats[0], catalog.Grid.square(100., 64), w, dlsds=D)))
            tickets = []
            t0 = time.perf_counter()
            for (k, n, c), o, ta in zip(reqs, outs, arr):
                now = time.perf_counter() - t0
                if ta > now:
                    time.sleep(ta - now)
                if k == 2:
                    tickets.append(srv.submit_chi2(models[c], frame, n, systems))
                else:
                    tickets.append(srv.submit(lt.Request(dcats[c], catalog.Grid.square(100., n), o, dlsds=D,
                                                         scale=D)))
            for t in tickets:
                srv.wait(t, 3600.)
            t_end = time.perf_counter() - t0
            lat = [srv.times(t)[2] for t in tickets]
            lat_chi = [x for x, (k, n, c) in zip(lat, reqs) if k == 2]
            lat_map = [x for x, (k, n, c) in zip(lat, reqs) if k != 2]
            st = srv.stats()
        return {"p50_ms": _percentile(lat, 50), "p99_ms": _percentile(lat, 99),
                "maps": {"p50_ms": _percentile(lat_map, 50), "p99_ms": _percentile(lat_map, 99)},
                "chi2": {"p50_ms": _percentile(lat_chi, 50), "p99_ms": _percentile(lat_chi, 99)},
                "requests_per_s": len(reqs) / t_end, "maps_per_s": nmaps / t_end, "chi2_per_s": nchi / t_end,
                "evals_per_s": evals / t_end, "seconds": t_end, "max_inflight": st["max_inflight"],
                "loop_launches": st["loop_launches"]}

    res = {"workload": f"serving: {n_requests} requests, Poisson {rate:g}/s, grids U{{512..4096}}^2, "
                       f"deflection or kappa/gamma/mu maps (halos log-U(50,5000)) or chi2 (200 halos, "
                       f"40 systems): {n_requests - nchi} map and {nchi} chi2 requests",
           "precision": precision}
    sat = run(arrivals)
    res["at_rate"] = dict(sat, rate_per_s=rate, offered_over_capacity=rate / sat["requests_per_s"])
    # a second pass at 70% of the measured capacity (the queue does not build up)
    r70 = 0.7 * sat["requests_per_s"]
    res["at_70pct_capacity"] = dict(run(arrivals * rate / r70), rate_per_s=r70)
    # one plain call per request (host outputs / host chi2, the reference's calling
    # pattern), in FP64 and in the server's own precision: every request by default (a
    # smaller sample is scaled to all requests by the halo x pixel evaluations of their grids).
    # The same-precision loop (a few seconds; its host-memory page faults vary from run to
    # run) is timed twice and the faster pass kept.
    idx = list(range(plain_sample or n_requests))
    sample_evals = float(sum(reqs[i][1] ** 2 * halos(reqs[i][0], reqs[i][2]) for i in idx))
    for prec in dict.fromkeys(("fp64", precision)):
        t = float("inf")
        for _ in range(1 if prec == "fp64" else 2):
            t0 = time.perf_counter()
            for i in idx:
                k, n, c = reqs[i]
                g = catalog.Grid.square(100., n)
                if k == 0:
                    ctx.gradient_grid(dcats[c], g, precision=prec, scale=D)
                elif k == 1:
                    ctx.hessian_maps(dcats[c], g, list(kinds_of[1]), precision=prec, dlsds=D)
                else:
                    ctx.chi2(models[c], frame, n, systems, precision=prec)
            t = min(t, time.perf_counter() - t0)
        t_all = t * evals / sample_evals
        key = "one_request_per_call_" + ("fp64" if prec == "fp64" else "same_precision")
        res[key] = {"precision": prec, "requests_per_s": len(reqs) / t_all, "maps_per_s": nmaps / t_all,
                    "sample_requests": len(idx), "sample_s": t}
    res["speedup_vs_one_request_per_call_fp64"] = (sat["requests_per_s"] /
                                                   res["one_request_per_call_fp64"]["requests_per_s"])
    if "one_request_per_call_same_precision" in res:
        res["speedup_vs_one_request_per_call_same_precision"] = (
            sat["requests_per_s"] / res["one_request_per_call_same_precision"]["requests_per_s"])
    for c in dcats + models + [dbase]:
        c.release()
    return res


def bench_chi2(ctx, n_models=64, n=2048, nsys=40, seed=20261203 + 3, cpu=True):
    """Delensing + chi2 workload: perturbed models (5% Gaussian, seeded) of the 200-halo
    catalogue against 40 multiple-image systems with 3-5 images each, generated by
    forward ray-shooting of seeded sources through the true model (delensing on a 2048^2
    grid) plus 0.05" Gaussian noise; per model a 2048^2 deflection grid, barycentric
    delensing and the FP64 chi2 (lt_chi2_batch).  A sample of n_models models is timed,
    each leg as the median of three runs (the 4096-model batch takes 4096 / models_per_s)."""
    lt = _package()
    from lenstool_hpc_b200 import catalog
    from lenstool_hpc_b200.images import generate_systems
    frame = (-100., 100., -100., 100.)
    base = catalog.cluster_galaxy_catalog(2, 198, 20261203)
    dls, dos, _ = lt.cosmo_distances(0.35, 1.5)
    D = dls / dos
    dbase = ctx.upload(base)
    ic = int(np.argmax(base.b0))
    systems = generate_systems(lambda bx, by, dr: ctx.delense(dbase, frame, n, bx, by, dr), nsys, seed, dr=D,
                               centre=(base.position_x[ic], base.position_y[ic]), source_radius=10.)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    models = [ctx.upload(catalog.perturb_catalog(base, rng)) for _ in range(n_models)]
    def timed(precision, runs=3):
        """median wall time of `runs` calls over all models (host-side work included)"""
        ctx.chi2(models[:2], frame, n, systems, precision=precision)  # warm-up
        ts = []
        for _ in range(runs):
            t0 = time.perf_counter()
            out = ctx.chi2(models, frame, n, systems, precision=precision)
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), out

    dt, (chi, found) = timed("fp64")
    true_chi, _ = ctx.chi2(dbase, frame, n, systems)
    res = {"workload": f"chi2_batch: {n_models} of 4096 perturbed models x {base.n} halos, {nsys} systems "
                       f"({systems.nimages} images), {n}^2 delensing grid, FP64",
           "models_per_s": n_models / dt, "ms_per_model": 1e3 * dt / n_models,
           "seconds_for_4096_models": 4096 * dt / n_models, "deflection_evals_per_s": n_models * n * n * base.n / dt,
           "chi2_true_model": true_chi, "chi2_median_perturbed": float(np.median(chi))}
    # the deflection grid in LT_FP64_FAST (within 2e-12 of the reference's arithmetic), then in
    # LT_FP32C; delensing and chi2 in FP64
    dtf, (chif, foundf) = timed("fp64fast")
    res["fp64fast_deflections"] = {
        "models_per_s": n_models / dtf, "ms_per_model": 1e3 * dtf / n_models,
        "same_images_found": bool(np.array_equal(foundf, found)),
        "max_rel_chi2_diff": float(np.max(np.abs(chif - chi) / np.maximum(np.abs(chi), 1.)))}
    dt32, (chi32, found32) = timed("fp32c")
    res["fp32c_deflections"] = {
        "models_per_s": n_models / dt32, "ms_per_model": 1e3 * dt32 / n_models,
        "same_images_found": bool(np.array_equal(found32, found)),
        "max_rel_chi2_diff": float(np.max(np.abs(chi32 - chi) / np.maximum(np.abs(chi), 1.)))}
    if cpu:
        try:
            import oracle
            ref = oracle.RefLib()
            t0 = time.perf_counter()
            r = ref.chi2(base, frame, n, systems.nimg, systems.x, systems.y, systems.dr)
            tc = time.perf_counter() - t0
            res["cpu_baseline"] = {"models_per_s": 1. / tc, "cores": os.cpu_count(), "kind": "reference",
                                   "sample": f"1 model: gradient_grid_CPU ({os.cpu_count()} threads) + "
                                             "delense_barycenter (1 thread, its serial order) + chi_computation",
                                   "chi2_true_model": r["chi2"]}
        except Exception as ex:
            res["cpu_baseline"] = {"unavailable": str(ex)}
    for m in models:
        m.release()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", default="fp32c", choices=["fp64", "fp32c", "fp64fast"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="--impl reference: skip timing the reference's GPU kernels beside its CPU code")
    ap.add_argument("--grid", type=int, default=0, help="smaller square grid (profiling cases)")
    ap.add_argument("--maps", default="all", choices=["all", "hessian", "potential", "deflection"],
                    help="all = kappa/gamma1/gamma2/mu/psi (the workload); the others time one sum")
    ap.add_argument("--breakdown", action="store_true", help="also time the Hessian-only and potential-only passes")
    ap.add_argument("--no-fp64-compare", action="store_true", help="skip timing LT_FP64 on the same workload")
    ap.add_argument("--skip-batch", action="store_true", help="skip the posterior-batch workload")
    ap.add_argument("--skip-serving", action="store_true", help="skip the serving workload")
    ap.add_argument("--skip-chi2", action="store_true", help="skip the delensing + chi2 workload")
    ap.add_argument("--batch-sets", type=int, default=512)
    ap.add_argument("--only-batch", action="store_true",
                    help="run only the posterior-batch workload (--batch-sets sets, --steps launches) and print it")
    ap.add_argument("--serving-requests", type=int, default=96)
    args = ap.parse_args()
    warmup = max(args.warmup, 3)
    rank, local_rank, world = dist_env()

    if args.impl == "reference":
        if rank != 0:
            return 0
        v, info = reference_cpu(args.steps, warmup)
        line = {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": warmup, "ms_per_step": 1e3 * info["seconds_per_sample"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "impl": "reference", "config": {"workload": WORKLOAD, "sample": info["sample"]},
                "cpu_baseline": info, "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0,
                                              "d2h_bytes_per_step": 0}}
        if not args.no_reference_gpu:
            try:
                line["reference_gpu"] = reference_gpu()
            except Exception as ex:  # no device here: the CPU arm stands alone
                line["reference_gpu"] = {"unavailable": str(ex)}
        print(json.dumps(line))
        return 0

    import torch
    lt = _package()
    from lenstool_hpc_b200 import build, catalog, replicas
    torch.cuda.set_device(local_rank)
    replicas.init("nccl", timeout_s=120.0)
    build.build()
    if args.only_batch:
        ctx = lt.Context(local_rank)
        res = bench_posterior_batch(ctx, args.precision, steps=args.steps, warmup=warmup, n_sets=args.batch_sets,
                                    e2e=not args.no_e2e)
        if rank == 0:
            print(json.dumps({"posterior_batch": res}))
        ctx.close()
        return 0
    cat, g = catalog.workload(WORKLOAD)
    if args.grid:
        g = catalog.Grid.square(150., args.grid)
    dls, dos, _ = lt.cosmo_distances(0.35, 1.5)
    D = dls / dos
    ctx = lt.Context(local_rank)
    dcat = ctx.upload(cat)
    stream = torch.cuda.Stream()
    names = {"all": ("kappa", "gamma1", "gamma2", "mu", "psi"), "hessian": ("kappa", "gamma1", "gamma2", "mu"),
             "potential": ("psi",), "deflection": ("deflection_x", "deflection_y")}[args.maps]
    sums_per_pair = (2 if args.maps == "all" else 1)
    outs = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda") for k in names}

    def maps_call(c, prec, o, stream=None, which=names):
        """the timed call: the lens maps in one fused pass, or the deflection grid"""
        if args.maps == "deflection":
            ctx.gradient_grid(c, g, precision=prec, out=(o["deflection_x"], o["deflection_y"]), stream=stream)
        else:
            ctx.lens_maps(c, g, precision=prec, dlsds=D, out=o, stream=stream, which=which)

    def step(which=names, o=outs):
        maps_call(dcat, args.precision, o, stream, which)

    for _ in range(warmup):
        step()
    ctx.synchronize(stream)

    def barrier():
        replicas.barrier(torch.cuda.synchronize)

    props = torch.cuda.get_device_properties(local_rank)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local_rank)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    t_all0 = torch.cuda.Event(enable_timing=True)
    t_all1 = torch.cuda.Event(enable_timing=True)
    # the library records CUDA events around its passes on the launching stream (pass 1:
    # the FP32C kernel, pass 2: the FP64 recomputation near critical curves)
    timing = args.precision == "fp32c"
    if timing:
        ctx.set_pass_timing(True)
        ctx.pass_times()
        ctx.recompute_count()
    barrier()
    n0 = lt.launch_count()
    with ClockSampler(gpu_id) as clocks:
        t_all0.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            step()
            ends[k].record(stream)
        t_all1.record(stream)
        ctx.synchronize(stream)
        barrier()
    launches = lt.launch_count() - n0
    elapsed = t_all0.elapsed_time(t_all1) / 1e3
    per_launch = float(np.mean([s.elapsed_time(e) for s, e in zip(starts, ends)])) / 1e3
    passes = None
    if timing:
        p1, p2, ncalls = ctx.pass_times()
        ctx.set_pass_timing(False)
        recomputed = ctx.recompute_count()
        passes = {"pass1_ms": p1 / max(ncalls, 1), "pass2_ms": p2 / max(ncalls, 1), "calls": ncalls,
                  "pixels_recomputed_fp64": recomputed / float(g.npix * args.steps)}
    evals_step = sums_per_pair * g.npix * cat.n
    value, elapsed, _ = replicas.throughput(evals_step * args.steps, elapsed, "cuda")

    breakdown = None
    if args.breakdown and rank == 0:
        breakdown = {}
        for label, which in (("hessian_maps", ("kappa", "gamma1", "gamma2", "mu")), ("potential", ("psi",))):
            o = {k: outs[k] for k in which}
            step(which, o)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                step(which, o)
            e1.record(stream)
            ctx.synchronize(stream)
            dt = e0.elapsed_time(e1) / 1e3 / args.steps
            breakdown[label] = {"ms": dt * 1e3, "evals_per_s": g.npix * cat.n / dt}

    # the same workload in LT_FP64 (the reference's FP64 arithmetic; Hessian bit-identical),
    # and the accuracy of the timed step's maps against it (max and RMS error per map,
    # pixels with |mu| > 100 apart)
    fp64_cmp = None
    errors = None
    if rank == 0 and args.precision != "fp64" and not args.no_fp64_compare:
        from lenstool_hpc_b200.accuracy import map_errors
        timed_maps = {k: v.clone() for k, v in outs.items()}  # the last timed step's output

        def time_precision(prec, k=2):
            maps_call(dcat, prec, outs, stream)
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record(stream)
            for _ in range(k):
                maps_call(dcat, prec, outs, stream)
            f1.record(stream)
            ctx.synchronize(stream)
            return f0.elapsed_time(f1) / 1e3 / k
        t64 = time_precision("fp64")
        errors = {"reference": "LT_FP64 on the same catalogue and grid (Hessian = the reference's CPU arithmetic "
                               "bit for bit, potential = the reference's pi05)",
                  "metric": "|got - fp64| / max(|fp64|, RMS of the map over |mu| <= 100)",
                  args.precision: map_errors(timed_maps, outs)}
        fp64_cmp = {"evals_per_s": evals_step / t64, "ms_per_step": t64 * 1e3, "steps": 2,
                    "speedup_of_" + args.precision: (evals_step * args.steps / elapsed) / (evals_step / t64)}
        if args.precision != "fp64fast":
            fp64_maps = {k: v.clone() for k, v in outs.items()}
            tf = time_precision("fp64fast")
            fp64_cmp["fp64fast"] = {"evals_per_s": evals_step / tf, "ms_per_step": tf * 1e3, "steps": 2}
            errors["fp64fast"] = map_errors(outs, fp64_maps)
            del fp64_maps
        del timed_maps

    # end to end through the public API with host buffers: catalogue upload from host
    # arrays and the maps copied back into pinned host memory, every step
    e2e = None
    if not args.no_e2e:
        host = {k: torch.empty((g.ny, g.nx), dtype=torch.float64, pin_memory=True) for k in names}
        hnp = {k: v.numpy() for k, v in host.items()}
        for _ in range(1):
            c2 = ctx.upload(cat)
            maps_call(c2, args.precision, hnp)
            c2.release()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            c2 = ctx.upload(cat)
            maps_call(c2, args.precision, hnp)
            c2.release()
        torch.cuda.synchronize()
        e2e_value, _, _ = replicas.throughput(evals_step * args.steps, time.perf_counter() - t0, "cuda")
        # FP64 records 256 B + FP32 records 160 B + index and type 8 B per halo, chunk tables
        h2d = (256 + 160 + 8) * cat.n + 4 * 16 * ((cat.n + 63) // 64)
        d2h = len(names) * g.npix * 8
        e2e = {"value": e2e_value, "unit": "evals/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "note": "host SoA -> lt_catalog_upload (packed records + chunk table) and 5 float64 maps -> pinned host"}

    if rank == 0:
        peaks = measured_peaks()
        pipe = "fp32" if args.precision == "fp32c" else "fp64"
        peak_tflops = fma_peak_tflops(pipe)
        fpp = {"all": FLOPS_PER_PAIR, "hessian": 182, "potential": 760}.get(args.maps)  # no census: deflection
        achieved = g.npix * cat.n * fpp / per_launch / 1e12 if fpp else None
        out_bytes = len(names) * g.npix * 8
        cat_bytes = (256 + 160) * cat.n  # FP64 records (256 B) + FP32C records (160 B) per halo, at most
        pairs = g.npix * cat.n
        issue = args.precision == "fp32c" and args.maps == "all"
        if issue:
            # pass 1 (the dominant kernel, grid32c_kernel<OP_HESS|OP_POT>) timed live by the
            # library's events; its issued thread instructions per pair from ncu on the build
            # whose sources KERNEL_SOURCES hash to INST_SOURCES_SHA.  Peak: every SMSP issues
            # one warp instruction (32 thread instructions) per cycle, at the SM clock sampled
            # during the timed region
            t1 = passes["pass1_ms"] / 1e3 if passes and passes["calls"] else per_launch
            sm_mhz = clocks.summary().get("sm_mhz") or 1965.0
            nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
            peak_inst = nsm * 4 * 32 * sm_mhz * 1e6 / 1e12
            achieved_inst = pairs * INST_PER_PAIR_FP32C_LENS / t1 / 1e12
            fp32_tflops = pairs * FP32_FLOPS_PER_PAIR_FP32C_LENS / t1 / 1e12
            sources_now = kernel_sources_sha()
        cpu = None
        if not args.no_cpu_baseline:
            try:
                _, cpu = reference_cpu(1, 1)
            except Exception as ex:  # the reference library is absent
                cpu = {"value": None, "unit": "evals/s", "kind": "reference", "cores": os.cpu_count(),
                       "sample": f"unavailable: {ex}"}
        line = {
            "metric": METRIC_OF_MAPS[args.maps], "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps,
            "warmup": warmup, "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "fp32c" else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if not args.grid else f"{WORKLOAD} at {g.nx}x{g.ny}",
                       "grid": f"{g.nx}x{g.ny} over 300\"x300\"", "halos": cat.n,
                       "maps": list(names), "precision": args.precision, "evals_per_step": evals_step,
                       "parallelism": f"replicas x{world}",
                       "l2": f"outputs {out_bytes / 1e6:.0f} MB per step > 126 MB L2 (no flush needed); catalogue "
                             f"{cat_bytes / 1e3:.0f} KB stays resident"},
            "gpu_launches": int(launches),
            "roofline": ({"bound": "issue", "achieved": achieved_inst, "peak": peak_inst,
                          "unit": "T thread-instructions/s",
                          "frac": achieved_inst / peak_inst if peak_inst else None,
                          "inst_per_pair": INST_PER_PAIR_FP32C_LENS,
                          "inst_per_pair_sources_sha": INST_SOURCES_SHA, "kernel_sources_sha": sources_now,
                          "inst_per_pair_current": INST_SOURCES_SHA == sources_now,
                          "fp32": {"flops_per_pair": FP32_FLOPS_PER_PAIR_FP32C_LENS, "achieved": fp32_tflops,
                                   "peak": peak_tflops, "unit": "TFLOP/s",
                                   "frac": fp32_tflops / peak_tflops if peak_tflops else None,
                                   "peak_source": "measured in-run: fp32 FMA-chain kernel"},
                          "peak_source": f"nominal issue rate: {nsm} SMs x 4 SMSPs x 32 lanes x the sampled "
                                         f"SM clock ({sm_mhz:.0f} MHz)",
                          "time_basis": "pass 1 alone, CUDA events on the launching stream over the timed "
                                        "region", "passes": passes} if issue else
                         {"bound": pipe, "achieved": achieved, "peak": peak_tflops, "unit": "TFLOP/s",
                          "frac": achieved / peak_tflops if (peak_tflops and achieved) else None,
                          "flops_per_pair": fpp, "flop_convention": "weighted census of the reference's formulas",
                          "peak_source": f"measured in-run: {pipe} FMA-chain kernel"}),
            "clocks": clocks.summary(),
        }
        line["roofline"].update({
            "traffic": TRAFFIC_FP32C_LENS_4096 if (issue and not args.grid) else None,
            "traffic_algorithmic": out_bytes,
            "kernel": ("lt::grid64_kernel" if args.precision in ("fp64", "fp64fast") else "lt::grid32c_kernel") +
                      {"all": "<OP_HESS|OP_POT>", "hessian": "<OP_HESS>", "potential": "<OP_POT>",
                       "deflection": "<OP_GRAD>"}[args.maps],
            "hbm_writeback_gbs": out_bytes / per_launch / 1e9, "hbm_peak_gbs": peaks.get("hbm_gbs")})
        if e2e:
            line["e2e"] = e2e
        if breakdown:
            line["breakdown"] = breakdown
        if cpu:
            line["cpu_baseline"] = cpu
        if fp64_cmp:
            line["fp64_same_workload"] = fp64_cmp
        if errors:
            line["errors"] = errors
        if world == 1 and not args.skip_batch:
            line["posterior_batch"] = bench_posterior_batch(ctx, args.precision, steps=2, warmup=3,
                                                            n_sets=args.batch_sets)
        if world == 1 and not args.skip_serving:
            line["serving"] = bench_serving(ctx, args.precision, n_requests=args.serving_requests)
        if world == 1 and not args.skip_chi2:
            line["chi2_batch"] = bench_chi2(ctx, cpu=not args.no_cpu_baseline)
        print(json.dumps(line))
    ctx.close()
    replicas.finalize()
    return 0


def kernel_sources_sha() -> str:
    """sha256 (16 hex digits) of the sources the FP32C lens-maps kernel is built from."""
    import hashlib
    h = hashlib.sha256()
    for name in KERNEL_SOURCES:
        h.update((ROOT / "lenstool-hpc_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def fma_peak_tflops(pipe: str) -> float:
    """Measured FMA throughput of this GPU (TFLOP/s, FMA = 2 flops) from the library's
    FMA-chain kernel."""
    lt = _package()
    L = lt.load_library()
    fn = getattr(L, "lt_measure_fma_peak", None)
    if fn is None:
        return None
    fn.restype = C.c_double
    fn.argtypes = [C.c_int, C.c_int]
    return float(fn(0 if pipe == "fp64" else 1, 0))


if __name__ == "__main__":
    sys.exit(main())
