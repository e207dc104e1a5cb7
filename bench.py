#!/usr/bin/env python
"""Headline benchmark: particle force evaluations per second of the tree code
(grow + traverse) on a clustered 4M-particle Plummer sphere.

Workload (the 4M clustered-gravity configuration): N = 4,194,304 equal charges
q = +1/N (gravity differs only by the sign of E), Plummer sphere with scale
radius 1 truncated at r = 20, seeded (numpy PCG64, seed 3), eps = 1e-3,
theta = 0.4, quadrupole, Hilbert keys, open boundaries.  Synthetic data.

One step = clear the results, grow the tree (bounding box, keys, sort, tree,
multipoles) and evaluate E and phi on every particle (the traversal), with the
particles already in HBM.  The timed form is the mixed-precision group walk;
the plain FP64 per-target walk (the drop-in form) is timed beside it.

Prints one JSON line (rank 0).  --impl reference times the CPU restatement
of the reference algorithm (the oracle) on the host cores instead.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle force evals/s at 4M, mixed vs FP64 GPU walk, at ≤1e-4 median force err"
UNIT = "force evals/s"
# DRAM bytes per particle of one mixed group-walk launch (k_walk_group64), from one
# ncu capture of the kernel (Plummer N = 1,048,576, theta = 0.4: 283.7 MB read +
# 57.1 MB written), scaled by the particle count: the tree the walk re-reads grows
# with N
WALK_DRAM_BYTES_PER_PARTICLE = (283.7e6 + 57.1e6) / 1048576
FLOPS_TWIG = 144  # counted from coulomb/module_coulomb_kernels.f90:60-145 + delta, dist2, MAC, sums
FLOPS_LEAF = 22   # counted from module_coulomb_kernels.f90:242-257 + delta, dist2, sums
SMS = 148


def plummer(n, seed=3, rmax=20.0):
    """Plummer sphere, a = 1: r = (u^(-2/3) - 1)^(-1/2), resampled above rmax."""
    rng = np.random.default_rng(seed)
    r = np.empty(0)
    while r.size < n:
        u = rng.random(2 * n)
        with np.errstate(divide="ignore"):
            rr = 1.0 / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[np.isfinite(rr) & (rr <= rmax)]])
    r = r[:n]
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    p = v * r[:, None]
    return (np.ascontiguousarray(p[:, 0]), np.ascontiguousarray(p[:, 1]),
            np.ascontiguousarray(p[:, 2]), np.full(n, 1.0 / n))


class Clocks:
    """nvidia-smi sampling during the timed region (50 ms period).  Entering waits
    for the sampler's first row (nvidia-smi takes a while to start) and drops
    it, so that the rows kept are the ones taken while the timed steps run."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0:
                time.sleep(0.01)
            self.rows = []
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(x, y, z, q, theta2, eps2, sample, threads, seed=11):
    """The oracle (CPU restatement of the reference path) on the host cores:
    grow of all N, traverse of a random sample of targets, scaled to N."""
    from oracle import oracle as O
    n = len(x)
    orc = O.Oracle(theta2=theta2, eps2=eps2, walk=0, num_threads=threads)
    t0 = time.perf_counter()
    g = orc.grow_tree(x, y, z, q)
    t1 = time.perf_counter()
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(n, min(sample, n), replace=False))
    orc.traverse_tree(g["x"][idx], g["y"][idx], g["z"][idx])
    t2 = time.perf_counter()
    orc.close()
    t_full = (t1 - t0) + (t2 - t1) * n / len(idx)
    return {"value": n / t_full, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"grow of all {n} particles ({t1 - t0:.2f} s) + per-target walk of "
                      f"{len(idx)} random targets ({t2 - t1:.2f} s), scaled to {n} targets",
            "t_grow_s": t1 - t0, "t_walk_sample_s": t2 - t1}


def run_reference(args, rank):
    """The reference arm: the oracle on all host threads.  Each step really runs
    the grow of all N particles and the walk of a random sample of targets
    (args.cpu_sample); the rate for all N targets is extrapolated from the
    sample's walk time, and the line says so (extrapolated, timed_targets).
    ms_per_step is the measured time of the step as run."""
    if rank != 0:
        return
    x, y, z, q = plummer(args.n)
    threads = os.cpu_count() or 1
    vals, step_ms = [], []
    t_run0 = time.perf_counter()
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(x, y, z, q, args.theta ** 2, args.eps ** 2, args.cpu_sample, threads,
                          seed=100 + i)
        if i >= args.warmup:
            vals.append(cb["value"])
            step_ms.append((cb["t_grow_s"] + cb["t_walk_sample_s"]) * 1e3)
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median(step_ms),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "extrapolated": True, "timed_targets": min(args.cpu_sample, args.n),
            "ms_per_step_extrapolated": args.n / v * 1e3,
            "run_s": time.perf_counter() - t_run0,
            "config": {"workload": workload_name(args), "implementation":
                       "CPU restatement of the reference tree code (oracle, per-target walk), "
                       "all host threads; the reference itself needs gfortran + MPI, absent here",
                       "step": f"grow of all {args.n} particles + per-target walk of "
                               f"{min(args.cpu_sample, args.n)} random targets; value = "
                               f"{args.n} / (grow time + sample walk time x {args.n} / sample)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def launch_ranks(args):
    """--gpus N without a launcher: run this script as N ranks under
    torch.distributed.run (one process per GPU, 127.0.0.1 rendezvous) and
    return its exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1",
           "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def hbm_peak_gbs():
    """The measured copy bandwidth of this pool's B200s, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def grow_roofline(st, n):
    """Achieved HBM bandwidth of the grow phases from their algorithmic bytes:
    bounding box 24 B and keys 32 B per particle; sort 24 B (one read and
    write of key + index) plus the permutation 64 B per particle; tree build
    8 B per particle + 40 B per node; upward pass 240 B per twig."""
    peak, src = hbm_peak_gbs()
    nodes = st["nleaf"] + st["ntwig"]
    phases = {"keys": (st["t_keys_ms"], 56 * n), "sort": (st["t_sort_ms"], 88 * n),
              "tree": (st["t_tree_ms"], 8 * n + 40 * nodes),
              "upward": (st["t_upward_ms"], 240 * st["ntwig"])}
    out = {"peak_gbs": peak, "peak_source": src}
    for k, (ms, b) in phases.items():
        gbs = b / (ms * 1e-3) / 1e9 if ms > 0 else None
        out[k] = {"bytes": b, "ms": ms, "gbs": gbs, "frac": (gbs / peak) if gbs else None}
    return out


def max_over_ranks(ms, dist, device):
    """The slowest rank's time: every rank's replica must finish for the job's step
    to end.  `dist` is torch.distributed (or None for one rank)."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(n_per_rank, world, ms):
    """Whole-job force evaluations per second: every rank's N over the slowest time."""
    return n_per_rank * world / (ms * 1e-3)


def uniform_sphere(n, seed=2):
    """Uniform in the unit sphere: radius u^(1/3), isotropic direction."""
    rng = np.random.default_rng(seed)
    r = rng.random(n) ** (1.0 / 3.0)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    p = v * r[:, None]
    return tuple(np.ascontiguousarray(p[:, k]) for k in range(3))


def rocksalt(n):
    """Rock-salt lattice: sites (i + 1/2)/n of the unit cube, q = (-1)^(i+j+k)."""
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return (((i + 0.5) / n).ravel(), ((j + 0.5) / n).ravel(), ((k + 0.5) / n).ravel(),
            ((-1.0) ** (i + j + k)).ravel())


def event_ms(torch, stream, fn):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def kaplan_sphere(n, seed=1234):
    """pepc-benchmark's 'test' setup (frontends/pepc-benchmark/module_helper.f90:194-227):
    particle k of n at radius s = (1/(1 - k/n) - 1)^(1/3) (Kaplan's Eq. 9, mu = 1) in a
    random direction (phi uniform, cos theta uniform).  The reference draws the angles
    from its own generator; numpy's PCG64 (seed) stands in for it."""
    rng = np.random.default_rng(seed)
    k = np.arange(n, dtype=np.float64)
    s = (1.0 / (1.0 - k / n) - 1.0) ** (1.0 / 3.0)
    phi = rng.random(n) * 2.0 * math.pi
    th = np.arccos(rng.random(n) * 2.0 - 1.0)
    return s * np.cos(phi) * np.sin(th), s * np.sin(phi) * np.sin(th), s * np.cos(th)


def benchmark_check(P, torch, dev, n, prec, walk, stream=None, seed=1234):
    """pepc-benchmark's correctness run (benchmark/benchmark.xml, tag check; the loop of
    frontends/pepc-benchmark/pepc.f90:49-93) on the device time loop: n electrons
    (q = -2/n, m = 1e-3, at rest) from kaplan_sphere, theta2 = 0.25, eps2 = 1e-4, dt =
    0.02.  Every step: results cleared, grow, traverse (the particles' own fields), push.
    Every diag_interval = 100 steps: the direct test on 1000 random particles
    (test_particles, module_helper.f90:455-524: L2 = sqrt(sum |E - E_direct|^2) / 1000)
    and the energies after the push (check_energies_local, :272-310: kinetic from v half
    a step back, relativistic; potential sum 0.5 q phi, here pepcg_potential_energy_device).
    The check step is the first diagnostic step at or after sqrt(n / 1000) * 210
    (pepc.f90:60): there the velocity histogram of the particles at 7 <= r <= 8.5
    (histogram_local, :342-376: 50 bins of v_max / 50) has its runs of occupied bins
    counted (test_histogram, :378-428), and the check passes with exactly 2.  egy_drop
    is the JUBE pattern's (max - min) / max of the total energy, in percent."""
    q = torch.full((n,), -2.0 / n, dtype=torch.float64, device=dev)
    m = torch.full((n,), 1e-3, dtype=torch.float64, device=dev)
    zeros = lambda: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    x0, y0, z0 = kaplan_sphere(n, seed)
    st = {"x": T(x0), "y": T(y0), "z": T(z0), "q": q, "m": m,
          "vx": zeros(), "vy": zeros(), "vz": zeros()}
    tc = P.TreeCode(theta2=0.25, eps2=1e-4, precision=prec, walk=walk)
    if stream is not None:
        tc.set_stream(stream.cuda_stream)
    key = torch.empty(n, dtype=torch.int64, device=dev)
    perm = torch.empty(n, dtype=torch.int64, device=dev)
    out = [zeros() for _ in range(5)]
    dt, diag, ndirect = 0.02, 100, 1000
    check_at = math.sqrt(n / 1000.0) * 210
    rng = np.random.default_rng(seed + 1)
    energies, l2 = [], []
    step = 0
    t0 = time.time()
    while True:
        do_diag = step % diag == 0
        do_check = step >= check_at and step > 0 and step < check_at + diag
        tc.grow_tree_device(st["x"], st["y"], st["z"], st["q"])
        nx, ny, nz, nq, nm, nvx, nvy, nvz = (torch.empty_like(q) for _ in range(8))
        tc.particles_device(key, perm, nx, ny, nz, nq)
        for src, dst in ((st["m"], nm), (st["vx"], nvx), (st["vy"], nvy), (st["vz"], nvz)):
            tc.gather_device(src, dst)
        for o in out:
            o.zero_()
        tc.traverse_self_device(*out)
        if do_diag:
            idx = np.sort((rng.random(ndirect) * (n - 1)).astype(np.int64))
            d = tc.direct(idx)
            E = torch.stack(out[:3]).cpu().numpy()[:, idx]
            dE = (E[0] - d["ex"]) ** 2 + (E[1] - d["ey"]) ** 2 + (E[2] - d["ez"]) ** 2
            Ed2 = d["ex"] ** 2 + d["ey"] ** 2 + d["ez"] ** 2
            l2.append((math.sqrt(dE.sum()) / ndirect, math.sqrt(dE.sum() / Ed2.sum())))
        tc.push_particles_device(dt, nq, nm, out[:3], (nvx, nvy, nvz), (nx, ny, nz))
        st.update(x=nx, y=ny, z=nz, q=nq, m=nm, vx=nvx, vy=nvy, vz=nvz)
        if do_diag:
            f = (dt * 0.5) * (nq / nm)
            vx_, vy_, vz_ = nvx - f * out[0], nvy - f * out[1], nvz - f * out[2]
            gam = torch.sqrt(1.0 + (vx_ * vx_ + vy_ * vy_ + vz_ * vz_))
            e_kin = float(((gam - 1.0) * nm).sum())
            e_pot = tc.potential_energy_device(nq, out[3])
            energies.append(e_kin + e_pot)
            if do_check:
                v = torch.sqrt(nvx * nvx + nvy * nvy + nvz * nvz)
                r = torch.sqrt(nx * nx + ny * ny + nz * nz)
                sel = (r >= 7.0) & (r <= 8.5)
                pos = (v[sel] / (float(v.max()) / 50)).long()
                hist = torch.bincount(pos, minlength=51).cpu().numpy()[:51]
                runs = int(sum(1 for b in range(51) if hist[b] > 0 and (b == 0 or hist[b - 1] == 0)))
                break
        step += 1
    seconds = time.time() - t0
    tc.close()
    e = np.array(energies)
    return {"n": n, "check_step": step, "steps": step + 1, "seconds": seconds,
            "histogram_peaks": runs, "check": "passed" if runs == 2 else "failed",
            "histogram": hist.tolist(),
            "egy_drop_pct": float((e.max() - e.min()) / abs(e.max()) * 100),
            "energy_first": float(e[0]), "energy_last": float(e[-1]),
            "l2_last": l2[-1][0], "l2_rel_max": max(v[1] for v in l2)}


def run_benchmark_check(args, P, torch, dev, stream):
    """the benchmark-check workload: benchmark_check at the reference's size (n = --n,
    1,048,576 unless given), one descriptive JSON line"""
    n = args.n if args.n != 4194304 else 1048576
    prec = {"mixed": P.PRECISION_MIXED, "plain": P.PRECISION_PLAIN,
            "strict": P.PRECISION_MIXED_STRICT}[args.precision]
    walk = {"group": P.WALK_GROUP, "target": P.WALK_PER_TARGET, "tile": P.WALK_PER_TILE}[args.walk]
    res = benchmark_check(P, torch, dev, n, prec, walk, stream)
    res["ms_per_step"] = res["seconds"] / res["steps"] * 1e3
    print(json.dumps({"workload": "pepc-benchmark correctness check (Kaplan Coulomb explosion)",
                      "precision": args.precision, "walk": args.walk, **res}), flush=True)


def run_explosion(args, P, torch, dev, stream):
    """Coulomb explosion: N = 1,048,576 uniform in the unit sphere (seed 2), q = m = 1/N,
    eps = 1e-3, theta = 0.3, Hilbert keys; 10 kick-drift steps, dt = 1e-3, in the
    pepc-mini pusher form (v += dt q/m E; x += dt v, module_helper.f90:205-222).
    Each precision runs its own trajectory from the same start; the force error is
    measured against the FP64 direct sum on 4,096 sampled targets (seed 22) at the
    first and the last step."""
    n = args.n if args.n != 4194304 else 1048576
    x0, y0, z0 = uniform_sphere(n)
    dt, nsteps = 1e-3, 10
    res = {}
    final = {}
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    for name, prec, walk in (("mixed", P.PRECISION_MIXED, P.WALK_GROUP),
                             ("plain", P.PRECISION_PLAIN, P.WALK_PER_TARGET)):
        q = torch.full((n,), 1.0 / n, dtype=torch.float64, device=dev)
        zeros = lambda: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
        st = {"x": T(x0), "y": T(y0), "z": T(z0), "q": q, "m": q.clone(),
              "vx": zeros(), "vy": zeros(), "vz": zeros()}
        tc = P.TreeCode(theta2=0.09, eps2=1e-6, precision=prec, walk=walk)
        tc.set_stream(stream.cuda_stream)
        key = torch.empty(n, dtype=torch.int64, device=dev)
        perm = torch.empty(n, dtype=torch.int64, device=dev)
        out = [zeros() for _ in range(5)]

        def step():
            # the whole step in the library: grow, the particle state carried
            # into key order (like pepc-mini's reordered particle records),
            # traverse, then the pusher in place
            tc.grow_tree_device(st["x"], st["y"], st["z"], st["q"])
            nx, ny, nz, nq, nm, nvx, nvy, nvz = (torch.empty_like(q) for _ in range(8))
            tc.particles_device(key, perm, nx, ny, nz, nq)
            for src, dst in ((st["m"], nm), (st["vx"], nvx), (st["vy"], nvy), (st["vz"], nvz)):
                tc.gather_device(src, dst)
            for o in out:
                o.zero_()
            tc.traverse_self_device(*out)
            tc.push_particles_device(dt, nq, nm, out[:3], (nvx, nvy, nvz), (nx, ny, nz))
            st.update(x=nx, y=ny, z=nz, q=nq, m=nm, vx=nvx, vy=nvy, vz=nvz)

        def error():
            # the field just computed, at the positions before the push (key order)
            idx = np.sort(np.random.default_rng(22).choice(n, 4096, replace=False))
            d = tc.direct(idx)
            E = torch.stack(out[:3]).cpu().numpy()[:, idx]
            Ed = np.stack([d["ex"], d["ey"], d["ez"]])
            rel = np.linalg.norm(E - Ed, axis=0) / np.linalg.norm(Ed, axis=0)
            return float(np.median(rel)), float(np.percentile(rel, 99))

        ms, errs = [], []
        for k in range(nsteps):
            ms.append(event_ms(torch, stream, step))
            if k in (0, nsteps - 1):
                errs.append(error())
        res[name] = {"ms_per_step_median": statistics.median(ms), "ms_first": ms[0],
                     "value": n / (statistics.median(ms) * 1e-3),
                     "walk_ms_last": tc.stats()["t_walk_ms"],
                     "force_err_first": {"median": errs[0][0], "p99": errs[0][1]},
                     "force_err_last": {"median": errs[1][0], "p99": errs[1][1]}}
        final[name] = st
        tc.close()
    # the two trajectories hold their particles in different orders (each is
    # re-sorted by key every step), so they are compared through the mean radius
    rm = {k: float(torch.sqrt(v["x"] ** 2 + v["y"] ** 2 + v["z"] ** 2).mean())
          for k, v in final.items()}
    line = {"workload": f"Coulomb explosion N={n} uniform sphere, q=m=1/N, eps=1e-3, theta=0.3, "
                        f"10 kick-drift steps dt=1e-3", "unit": UNIT, "mixed": res["mixed"],
            "plain": res["plain"],
            "mixed_over_plain": res["mixed"]["value"] / res["plain"]["value"],
            "mean_radius_after": rm,
            "step": "grow + key-order gather + traverse + push (library entry points), "
                    "particles resident in HBM"}
    print(json.dumps(line), flush=True)


def run_madelung(args, P, torch, dev, stream):
    """Periodic rock-salt lattice, FMM far-lattice term, eps = 0, theta = 0.3,
    one mirror-box layer: the Madelung constant at n = 64 (262,144 ions), then
    n = 80 (512,000 ions) perturbed by N(0, 1e-3) (seed 5), wrapped into the
    box, timed for the mixed group walk and the plain per-target walk."""
    out_line = {"workload": "rock-salt lattice, periodic, FMM lattice, eps=0, theta=0.3"}
    x, y, z, q = rocksalt(64)
    tc = P.TreeCode(theta2=0.09, eps2=0.0, periodicity=(1, 1, 1), walk=P.WALK_PER_TARGET)
    g = tc.pepc_grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z)
    tc.close()
    m_est = -float(np.mean(q[g.perm] * r["pot"])) / 64
    out_line["madelung_n64"] = {"estimate": m_est, "reference": 1.747565,
                                "abs_err": abs(m_est - 1.7475645946331822)}
    n = 80
    x, y, z, q = rocksalt(n)
    rng = np.random.default_rng(5)
    x, y, z = ((a + rng.normal(0.0, 1e-3, a.size)) % 1.0 for a in (x, y, z))
    N = x.size
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    tx, ty, tz, tq = T(x), T(y), T(z), T(q)
    out = [torch.zeros(N, dtype=torch.float64, device=dev) for _ in range(5)]
    for name, prec, walk in (("mixed", P.PRECISION_MIXED, P.WALK_GROUP),
                             ("plain", P.PRECISION_PLAIN, P.WALK_PER_TARGET)):
        tc = P.TreeCode(theta2=0.09, eps2=0.0, periodicity=(1, 1, 1), precision=prec, walk=walk)
        tc.set_stream(stream.cuda_stream)

        def step():
            for o in out:
                o.zero_()
            tc.grow_tree_device(tx, ty, tz, tq)
            tc.traverse_self_device(*out)

        for _ in range(3):
            step()
        ms = statistics.median(event_ms(torch, stream, step) for _ in range(3))
        st = tc.stats()
        # error against the FP64 direct sum over the mirror boxes plus the lattice term
        idx = np.sort(np.random.default_rng(55).choice(N, 2048, replace=False))
        d = tc.direct(idx)
        E = torch.stack(out[:3]).cpu().numpy()[:, idx]
        Ed = np.stack([d["ex"], d["ey"], d["ez"]])
        rel = np.linalg.norm(E - Ed, axis=0) / np.linalg.norm(Ed, axis=0)
        out_line[name] = {"ms_per_step": ms, "value": N / (ms * 1e-3), "walk_ms": st["t_walk_ms"],
                          "lattice_ms": st["t_lattice_ms"], "interactions": st["interactions"],
                          "force_err": {"median": float(np.median(rel)),
                                        "p99": float(np.percentile(rel, 99))}}
        tc.close()
    out_line["n_timed"] = N
    out_line["mixed_over_plain"] = out_line["mixed"]["value"] / out_line["plain"]["value"]
    print(json.dumps(out_line), flush=True)


def run_sharded(args, P, torch, dev, stream, dist, rank, world, local, emit=True):
    """Target sharding (strong scaling): rank 0's particles are broadcast, every
    rank grows the same tree from them, walks its shard_range share of the
    key-ordered targets (pepcg_traverse_range_device) and all-gathers the
    shares' fields (gather_shards), so that every rank ends the step with all
    N fields.  The step time is the slowest rank's; the job's rate is N per
    step."""
    x, y, z, q = plummer(args.n)
    n = args.n
    tx, ty, tz, tq = (torch.from_numpy(a).to(dev) for a in (x, y, z, q))
    t0, t1 = P.shard_range(n, rank, world)
    share = torch.zeros((5, t1 - t0), dtype=torch.float64, device=dev)
    walk = {"group": P.WALK_GROUP, "target": P.WALK_PER_TARGET, "tile": P.WALK_PER_TILE}[args.walk]
    prec = P.PRECISION_MIXED if args.precision == "mixed" else P.PRECISION_PLAIN
    tc = P.TreeCode(theta2=args.theta ** 2, eps2=args.eps ** 2, precision=prec, walk=walk,
                    device=local)
    tc.set_stream(stream.cuda_stream)
    full = [None]

    def step():
        # the particles as rank 0 holds them, broadcast to every rank (32 B per
        # particle over NVLink), then the same grow on every rank
        if dist:
            for a in (tx, ty, tz, tq):
                dist.broadcast(a, src=0)
        share.zero_()
        tc.grow_tree_device(tx, ty, tz, tq)
        tc.traverse_range_device(t0, t1, *share)
        full[0] = P.gather_shards(share, n, rank, world)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = P.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, dev)
    launches = P.kernel_launches() - l0
    # the gathered fields against one single-call traverse of all targets
    ref = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(5)]
    tc.traverse_self_device(*ref)
    torch.cuda.synchronize()
    same = all(bool(torch.equal(full[0][k], ref[k])) for k in range(5))
    tc.close()
    if not emit:
        return {"value": n / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "scaling": "strong",
                "n_gpus": world, "fields_equal_single_call": same, "gpu_launches": launches,
                "parallelism": f"target shards over {world} ranks: broadcast of the particles, "
                               "replicated tree, all-gather of the fields"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": n / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 interactions + f64 offsets/sums" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": workload_name(args), "precision": args.precision,
                       "walk": args.walk,
                       "parallelism": f"target shards over {world} ranks: broadcast of the "
                                      "particles, replicated tree, all-gather of the fields"},
            "fields_equal_single_call": same, "gpu_launches": launches}), flush=True)


def direct_gradient_torch(torch, x, y, z, q, tx, ty, tz, gphi, eps2, chunk=64):
    """FP64 direct-sum dL/dq, dL/dx for dL/dphi = gphi at the probes (torch on
    the GPU, chunked over the probes): the error reference of the adjoint."""
    dq = torch.zeros_like(q)
    dx, dy, dz = torch.zeros_like(x), torch.zeros_like(x), torch.zeros_like(x)
    for s in range(0, tx.numel(), chunk):
        e = slice(s, s + chunk)
        rx = tx[e, None] - x[None, :]
        ry = ty[e, None] - y[None, :]
        rz = tz[e, None] - z[None, :]
        rinv = torch.rsqrt(rx * rx + ry * ry + rz * rz + eps2)
        g = gphi[e, None]
        dq += (g * rinv).sum(0)
        w = g * q[None, :] * rinv ** 3
        dx += (w * rx).sum(0)
        dy += (w * ry).sum(0)
        dz += (w * rz).sum(0)
    return dq, dx, dy, dz


def adjoint_measure(P, torch, dev, stream, prec, walk, plummer_xyzq, theta):
    """The adjoint (pepcg_traverse_adjoint_device) against the forward of the
    same walk and precision, both timed with CUDA events on the library's
    stream.
      configuration: 262,144 sources U[0,1)^3 (seed 4), q ~ N(0,1) (seed 41),
        4,096 probes U[0.25,0.75]^3 (seed 42), L = sum (phi - phi_t)^2 with
        phi_t from a second charge set (seed 43), theta 0.4, eps 1e-3; the
        gradient against the FP64 direct-sum gradient (median over sources of
        |error| / max |gradient|, dL/dq and dL/dx);
      4M: the benchmark's particles as targets of themselves, random dL/dphi
        and dL/dE (the full gradient) and dL/dphi alone."""
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731

    def ev(fn, reps):
        ms = []
        for i in range(reps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if i >= 1:
                ms.append(e0.elapsed_time(e1))
        return statistics.median(ms)

    n, nt = 262144, 4096
    rng = np.random.default_rng(4)
    x, y, z = (T(rng.random(n)) for _ in range(3))
    q = T(np.random.default_rng(41).standard_normal(n))
    prng = np.random.default_rng(42)
    tx, ty, tz = (T(0.25 + 0.5 * prng.random(nt)) for _ in range(3))
    q_t = T(np.random.default_rng(43).standard_normal(n))
    kw = dict(theta2=0.16, eps2=1e-6, precision=prec, walk=walk)
    zero = torch.zeros(nt, dtype=torch.float64, device=dev)
    f = [torch.zeros(nt, dtype=torch.float64, device=dev) for _ in range(5)]
    tt = P.TreeCode(**kw)
    tt.set_stream(stream.cuda_stream)
    tt.grow_tree_device(x, y, z, q_t)
    tt.traverse_tree_device(tx, ty, tz, *f)
    phi_t = f[3].clone()
    tt.close()
    tc = P.TreeCode(**kw)
    tc.set_stream(stream.cuda_stream)
    tc.grow_tree_device(x, y, z, q)

    def fwd():
        for o in f:
            o.zero_()
        tc.traverse_tree_device(tx, ty, tz, *f)

    fwd_ms = ev(fwd, 3)
    gphi = 2.0 * (f[3] - phi_t)
    g = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(4)]
    adj_ms = ev(lambda: tc.traverse_adjoint_device(tx, ty, tz, [zero] * 3, gphi, *g), 3)
    gd = direct_gradient_torch(torch, x, y, z, q, tx, ty, tz, gphi, 1e-6)
    err = {}
    for name, a, b in (("q", g[0], gd[0]), ("x", g[1], gd[1])):
        err[name] = float(((a - b).abs() / b.abs().max()).median().item())
    tc.close()
    conf = {"forward_ms": fwd_ms, "adjoint_ms": adj_ms, "ratio": adj_ms / fwd_ms,
            "grad_err_median": err, "against": "FP64 direct-sum gradient (torch, on the GPU)"}

    # the benchmark's particles as their own targets
    px, py, pz, pq = (T(a) for a in plummer_xyzq)
    N = px.numel()
    tc = P.TreeCode(theta2=theta ** 2, eps2=1e-6, precision=prec, walk=walk)
    tc.set_stream(stream.cuda_stream)
    tc.grow_tree_device(px, py, pz, pq)
    key = torch.empty(N, dtype=torch.int64, device=dev)
    perm = torch.empty_like(key)
    kx, ky, kz, kq = (torch.empty(N, dtype=torch.float64, device=dev) for _ in range(4))
    tc.particles_device(key, perm, kx, ky, kz, kq)
    F = [torch.zeros(N, dtype=torch.float64, device=dev) for _ in range(5)]

    def fwd4():
        for o in F:
            o.zero_()
        tc.traverse_self_device(*F)

    f4 = ev(fwd4, 2)
    gen = torch.Generator(device=dev).manual_seed(7)
    gp4 = torch.randn(N, dtype=torch.float64, device=dev, generator=gen)
    gE4 = [torch.randn(N, dtype=torch.float64, device=dev, generator=gen) for _ in range(3)]
    z4 = torch.zeros(N, dtype=torch.float64, device=dev)
    G = [torch.zeros(N, dtype=torch.float64, device=dev) for _ in range(4)]
    a_phi = ev(lambda: tc.traverse_adjoint_device(kx, ky, kz, [z4] * 3, gp4, *G), 2)
    a_full = ev(lambda: tc.traverse_adjoint_device(kx, ky, kz, gE4, gp4, *G), 2)
    tc.close()
    return {"configuration": conf,
            "self_4m": {"forward_ms": f4, "adjoint_phi_ms": a_phi, "adjoint_full_ms": a_full,
                        "ratio_phi": a_phi / f4, "ratio_full": a_full / f4},
            "note": "forward and adjoint of the same walk and precision"}


def workload_name(args):
    return (f"Plummer sphere N={args.n} (a=1, r<=20, q=1/N), theta={args.theta}, "
            f"eps={args.eps}, quadrupole, Hilbert keys, open boundaries")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4194304)
    ap.add_argument("--theta", type=float, default=0.4)
    ap.add_argument("--eps", type=float, default=1e-3)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "plain", "strict"])
    ap.add_argument("--walk", default="group", choices=["group", "target", "tile"])
    ap.add_argument("--ntest", type=int, default=8192)
    ap.add_argument("--cpu-sample", type=int, default=32768)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-strict", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="target sharding across the ranks (strong scaling) instead of replicas")
    ap.add_argument("--workload", default="plummer",
                    choices=["plummer", "explosion", "madelung", "adjoint", "benchmark-check"],
                    help="plummer: the headline line; explosion / madelung: the other "
                         "configurations, one descriptive JSON line each; adjoint: the "
                         "adjoint measurements alone (the adjoint configuration, then the "
                         "Plummer particles of --n as their own targets); benchmark-check: "
                         "pepc-benchmark's correctness run (Kaplan Coulomb explosion, "
                         "histogram and energy checks) at n = 1,048,576 unless --n is given")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(launch_ranks(args))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but the launcher started {world} ranks")
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import pepc_b200 as P

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    if args.workload == "adjoint":
        dev = torch.device("cuda", local)
        stream = torch.cuda.Stream(device=dev)
        torch.cuda.set_stream(stream)
        prec = {"mixed": P.PRECISION_MIXED, "plain": P.PRECISION_PLAIN,
                "strict": P.PRECISION_MIXED_STRICT}[args.precision]
        walk = {"group": P.WALK_GROUP, "target": P.WALK_PER_TARGET, "tile": P.WALK_PER_TILE}[args.walk]
        res = adjoint_measure(P, torch, dev, stream, prec, walk, plummer(args.n), args.theta)
        print(json.dumps({"workload": "adjoint", "precision": args.precision, "walk": args.walk,
                          "n": args.n, **res}), flush=True)
        return
    if args.workload != "plummer":
        dev = torch.device("cuda", local)
        stream = torch.cuda.Stream(device=dev)
        torch.cuda.set_stream(stream)
        {"explosion": run_explosion, "madelung": run_madelung,
         "benchmark-check": run_benchmark_check}[args.workload](args, P, torch, dev, stream)
        return

    if args.shard:
        dev = torch.device("cuda", local)
        stream = torch.cuda.Stream(device=dev)
        torch.cuda.set_stream(stream)
        run_sharded(args, P, torch, dev, stream, dist, rank, world, local)
        if dist:
            dist.destroy_process_group()
        return

    x, y, z, q = plummer(args.n)
    n = args.n
    dev = torch.device("cuda", local)
    tx, ty, tz, tq = (torch.from_numpy(a).to(dev) for a in (x, y, z, q))
    out = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(5)]
    # a dedicated stream, current for torch as well, so the CUDA events that
    # time the steps sit on the stream the library launches on
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    walk = {"group": P.WALK_GROUP, "target": P.WALK_PER_TARGET, "tile": P.WALK_PER_TILE}[args.walk]
    prec = {"mixed": P.PRECISION_MIXED, "plain": P.PRECISION_PLAIN,
            "strict": P.PRECISION_MIXED_STRICT}[args.precision]
    tc = P.TreeCode(theta2=args.theta ** 2, eps2=args.eps ** 2, precision=prec, walk=walk,
                    device=local)
    tc.set_stream(stream.cuda_stream)

    def step(t):
        for o in out:
            o.zero_()
        t.grow_tree_device(tx, ty, tz, tq)
        t.traverse_self_device(*out)

    def timed(t, steps, warmup, clocks=None):
        for _ in range(warmup):
            step(t)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = P.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx = Clocks(local) if clocks else None
        if ctx:
            ctx.__enter__()
        e0.record(stream)
        for _ in range(steps):
            step(t)
        e1.record(stream)
        torch.cuda.synchronize()
        if ctx:
            ctx.__exit__()
        if dist:
            dist.barrier()
        ms = e0.elapsed_time(e1) / steps
        launches = (P.kernel_launches() - l0)
        ms = max_over_ranks(ms, dist, dev)
        return ms, launches, (ctx.summary() if ctx else None)

    ms, launches, clk = timed(tc, args.steps, args.warmup, clocks=True)
    st = tc.stats()
    fields_dev = (out[0].cpu().numpy(), out[3].cpu().numpy())  # for the host-path check
    value = job_rate(n, world, ms)

    # accuracy of this step's result against an FP64 direct sum on sampled targets
    rng = np.random.default_rng(33)
    tidx = np.sort(rng.choice(n, args.ntest, replace=False))
    E = torch.stack(out[:3]).cpu().numpy()[:, tidx]
    d = tc.direct(tidx)
    Ed = np.stack([d["ex"], d["ey"], d["ez"]])
    rel = np.linalg.norm(E - Ed, axis=0) / np.linalg.norm(Ed, axis=0)
    prel = np.abs(out[3].cpu().numpy()[tidx] - d["pot"]) / np.abs(d["pot"])

    # roofline of the dominant kernel (the walk)
    f_mhz = clk["sm_mhz"] if clk and clk["sm_mhz"] else 1965.0
    lanes = 64 if prec == P.PRECISION_PLAIN else 128  # FP64 / FP32 lanes per SM
    peak = SMS * lanes * 2 * f_mhz * 1e6 / 1e12
    flops = FLOPS_TWIG * st["twig_interactions"] + FLOPS_LEAF * st["leaf_interactions"]
    achieved = flops / (st["t_walk_ms"] * 1e-3) / 1e12
    roof = {"bound": "fp64-core" if prec == P.PRECISION_PLAIN else "fp32-core",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": (WALK_DRAM_BYTES_PER_PARTICLE * n
                        if prec == P.PRECISION_MIXED and args.walk == "group" and args.theta == 0.4
                        else None),
            "traffic_source": "ncu dram__bytes_read+write of one launch at N=1,048,576, scaled by "
                              "N (mixed group walk, theta 0.4 only; null otherwise)",
            "kernel": "walk", "kernel_ms": st["t_walk_ms"],
            "peak_source": f"{SMS} SMs x {lanes} lanes x 2 flop/FMA x median SM clock under load "
                           f"({f_mhz:.0f} MHz); no measured CUDA-core peak in MEASURED_PEAKS.json",
            "flops_per_launch": flops,
            "interactions": {"twig": st["twig_interactions"], "leaf": st["leaf_interactions"]}}
    phases = {k: st[k] for k in ("t_keys_ms", "t_sort_ms", "t_tree_ms", "t_upward_ms",
                                 "t_walk_ms", "t_lattice_ms")}
    grow_roof = grow_roofline(st, n)

    # the plain FP64 drop-in form (per-target walk) on the same input
    plain = None
    if not args.no_plain:
        tp = P.TreeCode(theta2=args.theta ** 2, eps2=args.eps ** 2, precision=P.PRECISION_PLAIN,
                        walk=P.WALK_PER_TARGET, device=local)
        tp.set_stream(stream.cuda_stream)
        pms, _, _ = timed(tp, max(1, min(args.steps, 3)), 3)
        pst = tp.stats()
        Ep = torch.stack(out[:3]).cpu().numpy()[:, tidx]
        prel_p = np.linalg.norm(Ep - Ed, axis=0) / np.linalg.norm(Ed, axis=0)
        pflops = FLOPS_TWIG * pst["twig_interactions"] + FLOPS_LEAF * pst["leaf_interactions"]
        plain = {"value": n * world / (pms * 1e-3), "ms_per_step": pms,
                 "walk_ms": pst["t_walk_ms"], "interactions": pst["interactions"],
                 "walk_tflops": pflops / (pst["t_walk_ms"] * 1e-3) / 1e12,
                 "force_err_median": float(np.median(prel_p)),
                 "force_err_p99": float(np.percentile(prel_p, 99))}
        tp.close()

    # the north star's precision form of the same group walk (FP64 offsets per
    # interaction, compensated FP32 sums, the FP64 walk's MAC decisions)
    strict = None
    if not args.no_strict and prec == P.PRECISION_MIXED and args.walk == "group":
        ts = P.TreeCode(theta2=args.theta ** 2, eps2=args.eps ** 2,
                        precision=P.PRECISION_MIXED_STRICT, walk=P.WALK_GROUP, device=local)
        ts.set_stream(stream.cuda_stream)
        sms, _, _ = timed(ts, max(1, min(args.steps, 3)), 3)
        sst = ts.stats()
        Es = torch.stack(out[:3]).cpu().numpy()[:, tidx]
        rel_s = np.linalg.norm(Es - Ed, axis=0) / np.linalg.norm(Ed, axis=0)
        strict = {"value": n * world / (sms * 1e-3), "ms_per_step": sms,
                  "walk_ms": sst["t_walk_ms"], "interactions": sst["interactions"],
                  "force_err_median": float(np.median(rel_s)),
                  "force_err_p99": float(np.percentile(rel_s, 99)),
                  "form": "offsets target minus node centre in FP64 per interaction, Kahan-"
                          "compensated FP32 sums, FP64 MAC decisions"}
        ts.close()

    # end to end through the host API (pinned host buffers, copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        hx, hy, hz, hq = pin(x), pin(y), pin(z), pin(q)
        hk = torch.zeros(n, dtype=torch.int64).pin_memory().numpy()
        hp = torch.zeros(n, dtype=torch.int64).pin_memory().numpy()
        hxo, hyo, hzo = (torch.zeros(n, dtype=torch.float64).pin_memory().numpy() for _ in range(3))
        res = [torch.zeros(n, dtype=torch.float64).pin_memory().numpy() for _ in range(5)]
        import ctypes as C
        L = P.lib()
        dp = lambda a: a.ctypes.data_as(P.D)  # noqa: E731
        ipp = lambda a: a.ctypes.data_as(P.I64)  # noqa: E731

        # the frontend's results clear folded into the traverse: the old values
        # are not uploaded, the fields come back in full
        tc.set_params(overwrite_results=1)

        def host_step():
            tc._check(L.pepcg_grow_tree(tc._h, n, dp(hx), dp(hy), dp(hz), dp(hq), ipp(hk), ipp(hp),
                                        dp(hxo), dp(hyo), dp(hzo)))
            tc._check(L.pepcg_traverse_tree(tc._h, n, dp(hxo), dp(hyo), dp(hzo), ipp(hk),
                                            *[dp(r_) for r_ in res]))

        for _ in range(3):
            host_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ksteps = max(1, min(args.steps, 3))
        e0.record(stream)
        for _ in range(ksteps):
            host_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / ksteps
        ems = max_over_ranks(ems, dist, dev)
        tc.set_params(overwrite_results=0)
        # the host path's fields against the device path's (same walk, same input)
        same = bool(np.array_equal(res[0], fields_dev[0]) and np.array_equal(res[3], fields_dev[1]))
        # grow: x y z q in; key, perm, x y z out.  traverse: x y z in (the
        # group walk does not read the keys, so they are not uploaded); e(3)
        # pot work out
        h2d = n * (4 * 8) + n * (3 * 8)
        d2h = n * (8 + 8 + 3 * 8) + n * (5 * 8)
        e2e = {"value": n * world / (ems * 1e-3), "unit": UNIT, "ms_per_step": ems,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": "pepcg_grow_tree + pepcg_traverse_tree (host arrays, pinned; "
                      "overwrite_results = 1)", "fields_equal_device_path": same}

    # the gradient against the forward of the same walk and precision
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = adjoint_measure(P, torch, dev, stream, prec, walk, (x, y, z, q), args.theta)

    # with several ranks, the same workload sharded over them (strong scaling)
    sharded = None
    if world > 1:
        sstream = torch.cuda.Stream(device=dev)
        with torch.cuda.stream(sstream):
            sharded = run_sharded(args, P, torch, dev, sstream, dist, rank, world, local,
                                  emit=False)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(x, y, z, q, args.theta ** 2, args.eps ** 2, args.cpu_sample,
                           os.cpu_count() or 1)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if prec == P.PRECISION_PLAIN else "f32 interactions + f64 offsets/sums",
        "data": "synthetic",
        "config": {"workload": workload_name(args), "precision": args.precision,
                   "walk": args.walk,
                   "group_size": (32 if prec == P.PRECISION_PLAIN else 64) if args.walk == "group"
                   else None,
                   "parallelism": "replicas only" if world > 1 else "single GPU",
                   "l2": "inputs (128 MB) and tree (~0.7 GB) exceed the 126 MB L2; no flush",
                   "step": "zero results + grow (box, keys, sort, tree, multipoles) + traverse"},
        "force_err": {"median": float(np.median(rel)), "p99": float(np.percentile(rel, 99)),
                      "pot_median": float(np.median(prel)), "ntest": args.ntest,
                      "against": "FP64 direct sum (pepcg_direct)"},
        "walk_only": {"value": n * world / (st["t_walk_ms"] * 1e-3), "unit": UNIT,
                      "ms": st["t_walk_ms"]},
        "roofline": roof, "phases_ms": phases, "grow_roofline": grow_roof,
        "gpu_launches": launches,
        "clocks": clk, "e2e": e2e, "plain": plain,
        "mixed_over_plain": (value / plain["value"]) if plain else None,
        "strict": strict,
        "adjoint": adjoint,
        "cpu_baseline": cpu,
        "sharded": sharded,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    tc.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
