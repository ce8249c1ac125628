#!/usr/bin/env python
"""Benchmark of the B200 face-loop path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--n 256] [--impl ours|reference]

Workload: MeshStructGenSource-equivalent structured hex mesh n^3 on the unit
cube (default 256^3: 16.8M cells, 50.1M interior + 393K boundary faces),
seeded synthetic fields. One step = the FP32-compensated forward
(GradientPhiGaussDolfyn with nGradient = 1 fused with the plain
FluxMassDolfynFaceLoop m_f = rho_f (u_f . S_f)) plus the hand-written adjoint
of L = sum_c V_c |grad_c|^2 + sum_f g_f m_f, on device-resident inputs.
Metric: Gfaces/s = (interior + boundary faces) / step time, summed over GPUs
(each GPU runs its own mesh: weak scaling, no data-path collective).

Also reported: the plain FP64 forward on the same mesh, the FP32-compensated
error against the FP64 path, the end-to-end host-buffer call (H2D + D2H
inside the timed region), the CPU baseline (the reference's own kernels)
and the HBM roofline of the dominant kernel.

--impl reference: the reference's own CPU kernels (compiled unchanged into
oracle/_ref, else the oracle restatement), all host cores as independent
processes on z-slabs of the mesh (what mpirun -n P with the naive
partitioner runs: the kernels have no communication).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "Gfaces/s and HBM GB/s, FP32-comp+adjoint vs FP64 plain on 1 B200, err vs FP64"
SEED = 20261203


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_cupcfd():
    name = "cupcfd_b200"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(ROOT, "cup-cfd_b200", "__init__.py")
    spec = importlib.util.spec_from_file_location(name, path, submodule_search_locations=[os.path.dirname(path)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def face_counts(n):
    nC = n ** 3
    nFi = 3 * n * n * (n - 1)
    nB = 6 * n * n
    return nC, nFi + nB, nFi, nB


def bytes_model(nC, nF, nFi, nB):
    """Algorithmic (compulsory) bytes: each distinct input read once, each
    output written once; int32 indices; FP64 volumes in both precisions."""
    return {
        # forward with the mass-flux adjoint (k_fwd_madj_f32_pf): phi 4 + rho,u,v,w 16 + V 8 + grad 12 +
        # statebar 16 per cell; S 12 + lambda 4 + cell1 4 per face; cell2 4 + g_f 4 + m_f 4 per interior
        # face; phiB 4 per boundary face
        "fwd_madj_f32": 56 * nC + 20 * nF + 12 * nFi + 4 * nB,
        # gradient adjoint (k_gadj_f32_pf): grad 12 + phibar 4 per cell; face geometry and connectivity
        # as above; phibBar 4 per boundary face
        "gadj_f32": 16 * nC + 20 * nF + 4 * nFi + 4 * nB,
        # fused forward, FP32: phi 4 + rho,u,v,w 16 + V 8 + grad 12 per cell;
        # S 12 + lambda 4 + cell1 4 per face; cell2 4 + m_f 4 per interior face; phiB 4 per boundary face
        "fwd_f32": 40 * nC + 20 * nF + 8 * nFi + 4 * nB,
        # adjoint, FP32: grad 12 + state 16 + phibar 4 + statebar 16 per cell; face geometry and
        # connectivity as above; g_f 4 per interior face; phibBar 4 per boundary face
        "adj_f32": 48 * nC + 20 * nF + 8 * nFi + 4 * nB,
        # whole forward+adjoint pipeline: face data and inputs counted once, grad written once and read once
        "pipeline_f32": 72 * nC + 20 * nF + 12 * nFi + 8 * nB,
        # fused forward, FP64: 8-byte reals
        "fwd_f64": 72 * nC + 32 * nF + 16 * nFi + 8 * nB,
    }


def max_over_ranks(x, dist=None, device="cpu"):
    """The largest x over all ranks (the job's time is its slowest rank's);
    x itself when there is one rank."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gfaces(world, faces_per_rank, seconds):
    """Whole-job throughput: every rank runs its own mesh (weak scaling)."""
    return world * faces_per_rank / seconds / 1e9


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM traffic per launch from the committed ncu summary, if present."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


class Clocks:
    """nvidia-smi sampler for the timed region, every 20 ms (SM and memory
    clocks, board power, throttle reasons). A sustained forward+adjoint loop
    reaches the board's power limit within 100-200 ms (sw_power_cap, SM clock
    down to about 1.56 GHz, memory clock unchanged), so the samples must be
    dense enough to see a timed region of a few hundred milliseconds."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,clocks.mem")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
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
        sm, mem, pw, mx, reasons = [], [], [], None, set()
        capped = 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for conv, dst, i in ((float, pw, 3), (float, mem, 9)):
                    try:
                        dst.append(conv(p[i]))
                    except (ValueError, IndexError):
                        pass
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
                        capped += nm == "sw_power_cap"
        os.unlink(self.path)
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
               "samples": len(sm)}
        if sm:
            out["sm_mhz_min"] = min(sm)
        if mem:
            out["mem_mhz"] = statistics.median(mem)
        if pw:
            out["power_w_max"] = max(pw)
        if "sw_power_cap" in reasons:
            out["sw_power_cap_samples"] = capped
        return out


def sustained_run(step, st, seconds, ms_guess, nF, world, index):
    """The step back to back for about `seconds`, with the clocks sampled:
    device time per step in 100 ms bins of device time. The board's power
    limit engages 100-200 ms into a sustained loop (sw_power_cap: the SM clock
    falls, the memory clock does not), so a long run settles at the rate of
    the last bins, below the first."""
    import torch
    n = max(10, int(seconds * 1e3 / max(ms_guess, 1e-3)))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    torch.cuda.synchronize()
    time.sleep(1.0)  # let the board cool back from the measurements before
    clocks = Clocks(index)
    clocks.start()
    time.sleep(0.1)
    for k in range(n):
        ev[k][0].record(st)
        step()
        ev[k][1].record(st)
    torch.cuda.synchronize()
    clk = clocks.stop()
    time.sleep(1.0)  # and again before the measurements after
    t = [a.elapsed_time(b) for a, b in ev]
    starts = [ev[0][0].elapsed_time(a) for a, _ in ev]
    span = starts[-1] + t[-1]
    bins = {}
    for s0, x in zip(starts, t):
        bins.setdefault(int(s0 // 100), []).append(x)
    per = [sum(v) / len(v) for _, v in sorted(bins.items())]
    last = [x for s0, x in zip(starts, t) if s0 >= span - 500.0]
    ms_last = sum(last) / len(last)
    return {"seconds": span / 1e3, "steps": n, "ms_per_step_per_100ms": [round(x, 4) for x in per],
            "ms_per_step_first_100ms": per[0], "ms_per_step_last_500ms": ms_last,
            "value_last_500ms": world * nF / (ms_last * 1e-3) / 1e9, "unit": "Gfaces/s", "clocks": clk}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own kernels on a bounded sample
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    n, nz_local, z0, reps, warmup = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    h = 1.0 / n
    # one z-slab of the n^3 mesh plus one ghost layer below and above (when present)
    lo = max(z0 - 1, 0)
    hi = min(z0 + nz_local + 1, n)
    m = O.structgen(n, n, hi - lo, bounds=(0.0, 1.0, 0.0, 1.0, lo * h, hi * h))
    f = O.fields(m, SEED)
    kind = "reference"
    if O.load_ref() is not None:
        R = O.RefKernels(m)
        if warmup:
            R.gradient(f["phi"], f["phiB"], 1, reps=warmup)
            R.flux_mass(f, reps=warmup)
        _, _, _, sg = R.gradient(f["phi"], f["phiB"], 1, reps=reps)
        _, _, sm = R.flux_mass(f, reps=reps)
        t = [a + b for a, b in zip(sg, sm)]
    else:
        kind = "port"
        t = []
        for i in range(warmup + reps):
            t0 = time.perf_counter()
            O.gradient(m, f["phi"], f["phiB"], 1)
            O.flux_mass_face_loop(m, f)
            if i >= warmup:
                t.append(time.perf_counter() - t0)
    return kind, m["nFaces"], t


def slab_faces(n, nz_local, top):
    """Faces a z-slab of nz_local planes of the n^3 mesh owns: its x- and
    y-faces and the z-faces below each of its planes (and above the top plane
    for the topmost slab), so that the slabs' counts add up to the mesh's."""
    return 2 * (n + 1) * n * nz_local + n * n * (nz_local + (1 if top else 0))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(n, procs, reps, warmup=0, slabs=None):
    """Gfaces/s of the reference's forward face loops (GradientPhiGaussDolfyn +
    FluxMassDolfynFaceLoop, FP64; the reference has no adjoint) on an n^3 mesh
    cut into `slabs` z-slabs (default: one per process), each slab with one
    ghost layer, as mpirun with NaivePartitioner cuts it. `procs` independent
    processes run the first `procs` slabs; with procs = slabs that is the
    whole mesh, and per repetition the slowest slab bounds the step."""
    import multiprocessing as mp
    slabs = slabs or procs
    assert 1 <= procs <= slabs <= n
    nz = [n // slabs + (1 if r < n % slabs else 0) for r in range(slabs)]
    z, jobs, faces = 0, [], 0
    for r in range(procs):
        jobs.append((n, nz[r], z, reps, warmup))
        faces += slab_faces(n, nz[r], r == slabs - 1)
        z += nz[r]
    if procs == 1:
        res = [_cpu_worker(jobs[0])]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            res = pool.map(_cpu_worker, jobs)
    kind = res[0][0]
    per_rep = [max(r[2][i] for r in res) for i in range(reps)]
    t = statistics.median(per_rep)
    part = "the whole mesh" if procs == slabs else f"{procs} of the {slabs} slabs ({faces} of its faces)"
    return {"value": faces / t / 1e9, "unit": "Gfaces/s", "cores": procs, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"{n}^3 structured mesh cut into {slabs} z-slab(s) with one ghost layer, {part}; reference "
                      f"GradientPhiGaussDolfyn + FluxMassDolfynFaceLoop compiled unchanged (FP64 forward; the "
                      f"reference has no adjoint); {warmup} warm-up and {reps} timed repetitions, median, "
                      f"faces owned / slowest slab",
            "ms_per_step": t * 1e3, "warmup": warmup, "reps": reps}


def cpu_uvw(n, reps):
    """Gfaces/s of the reference's FluxUVWDolfynFaceLoop1 (FP64, one core) on
    an n^3 generated mesh with its default region, as the reference's
    FluxUVWDolfynFaceLoop1Benchmark runs it (BenchmarkKernels.cpp:751-860)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    m = O.structgen(n, n, n)
    f = O.uvw_fields(m, SEED)
    if O.load_ref() is not None:
        kind = "reference"
        _, _, secs = O.RefKernels(m).uvw_geometry().uvw_face_loop1(f, reps=reps)
    else:
        kind = "port"
        secs = []
        for _ in range(reps):
            t0 = time.perf_counter()
            O.uvw_face_loop1(m, f)
            secs.append(time.perf_counter() - t0)
    t = statistics.median(secs)
    return {"value": m["nFaces"] / t / 1e9, "unit": "Gfaces/s", "cores": 1, "kind": kind, "ms_per_call": t * 1e3,
            "sample": f"{n}^3 generated mesh ({m['nFaces']} faces), default region; median of {reps} calls"}


def bench_uvw(cg, mesh, dev, st, g, steps, warmup, peak):
    """The momentum face loop (FluxUVWDolfynFaceLoop1, FP64) through the
    device-resident call on the bench mesh: the generated mesh with its
    default region and zero rlencos, the reference benchmark's configuration.
    Inputs drawn as that benchmark draws them (U[1e-6, 1e-2]), gradients
    1e-2 N(0,1). Algorithmic bytes per call: per cell u, v, w, visEff, nine
    gradient components, the cell centre (read) and su..aw (read and written)
    = 224; per interior face S, lambda, massFlux, two cell ids (read) and
    rFace (written) = 64; per boundary face its region id = 4."""
    import torch
    nC, nF, nFi, nB = mesh.nCells, mesh.nFaces, mesh.nInteriorFaces, mesh.nBoundaries
    D = dict(dtype=torch.float64, device=dev)

    def U(n):
        return torch.rand(n, generator=g, **D) * (1e-2 - 1e-6) + 1e-6

    c = {k: U(nC) for k in ("u", "v", "w", "visC", "su", "sv", "sw", "au", "av", "aw")}
    grads = torch.randn(9, nC, generator=g, **D) * 1e-2
    b = {k: U(nB) for k in ("uB", "vB", "wB", "visB")}
    mf = U(nF)
    rf = torch.zeros(2 * nF, **D)

    def call():
        cg.dev_uvw_face_loop1(mesh, 0.9, 1e-18, c["u"], c["v"], c["w"], b["uB"], b["vB"], b["wB"], c["visC"], b["visB"],
                              mf, grads, rf, c["su"], c["sv"], c["sw"], c["au"], c["av"], c["aw"], stream=st)

    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        call()
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    alg = 224 * nC + 64 * nFi + 4 * nB
    gbs = alg / (ms * 1e-3) / 1e9
    return {"call": "cupcfd_gpu_dev_uvw_face_loop1 (FP64, bit-identical to the reference)", "kernel": "k_uvw_f64_pf",
            "ms_per_call": ms, "value": nF / (ms * 1e-3) / 1e9, "unit": "Gfaces/s", "steps": steps,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "algorithmic_bytes_per_launch": alg},
            "config": "generated mesh, default region, rlencos 0 (the reference benchmark's case)"}


def host_link(dev, mb=256, reps=5):
    """Pinned host <-> device copy bandwidth of this box (GB/s): each
    direction alone, and each direction while the other runs on a second
    stream (the host call overlaps them). Bounds the e2e figure."""
    import torch
    n = mb * 2 ** 20 // 4
    h_in = torch.ones(n, dtype=torch.float32, pin_memory=True)
    h_out = torch.empty(n, dtype=torch.float32, pin_memory=True)
    d_a = torch.empty(n, dtype=torch.float32, device=dev)
    d_b = torch.ones(n, dtype=torch.float32, device=dev)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def run(h2d, d2h):
        if h2d:
            with torch.cuda.stream(s1):
                d_a.copy_(h_in, non_blocking=True)
        if d2h:
            with torch.cuda.stream(s2):
                h_out.copy_(d_b, non_blocking=True)
        torch.cuda.current_stream().wait_stream(s1)
        torch.cuda.current_stream().wait_stream(s2)

    def ms(h2d, d2h):
        run(h2d, d2h)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run(h2d, d2h)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    gb = n * 4 / 1e9
    both = ms(True, True)
    return {"h2d_gbs": gb / ms(True, False) * 1e3, "d2h_gbs": gb / ms(False, True) * 1e3,
            "each_way_concurrent_gbs": gb / both * 1e3, "bytes": n * 4, "unit": "GB/s"}


def _time_calls(st, fn, steps, warmup):
    """Mean device time (ms) of fn() over `steps` calls on stream st, CUDA events."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def bench_boundary_loops(cg, mesh, dev, st, steps):
    """The mass-flux boundary / region loops (FluxMassDolfynBoundaryLoop1-5,
    FluxMassDolfynRegionLoop; FP64, bit-identical to the reference) as a
    solver step chains them, device-resident, on the bench mesh with six
    regions (default, inlet, two outlets, symmetry, wall) assigned to its
    boundaries at random. Sums run in boundary order, so the chain is bound
    by its ordered reductions, not by bytes."""
    import numpy as np
    import torch
    nB, nC, nF = mesh.nBoundaries, mesh.nCells, mesh.nFaces
    rng = np.random.Generator(np.random.Philox(key=SEED + 7))
    rtype = np.array([0, 1, 2, 3, 4, 2], np.int32)
    check = mesh.set_regions(rtype, rng.standard_normal(18), rng.uniform(0.9, 1.1, 6), rng.integers(0, 6, nB))
    if check != cg.E_SUCCESS or mesh.set_region_split(rng.uniform(0.2, 0.8, 6)) != cg.E_SUCCESS:
        raise RuntimeError(cg.last_error())
    D = dict(dtype=torch.float64, device=dev)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(**D)
    mf = T(rng.uniform(1e-6, 1e-2, nF) * rng.choice([-1.0, 1.0], nF))
    su = T(rng.standard_normal(nC))
    u, v, w, den = (T(rng.uniform(1e-6, 1e-2, nB)) for _ in range(4))
    fr = T(rng.uniform(1e-6, 1e-2, 6))
    sc = torch.zeros(5, **D)
    ff = torch.zeros(6, **D)

    def chain():
        cg.dev_boundary_loop1(mesh, mf, sc[0:1], stream=st)
        cg.dev_boundary_loop3(mesh, sc[0:1], sc[1:2], stream=st)
        cg.dev_boundary_loop4(mesh, mf, u, v, w, den, sc[1:2], sc[2:3], stream=st)
        cg.dev_boundary_loop2(mesh, mf, fr, sc[3:4], stream=st)
        cg.dev_region_loop(mesh, ff, fr, sc[0:1], stream=st)
        cg.dev_boundary_loop5(mesh, mf, su, u, v, w, 1.3, (1, 1, 1), ff, sc[4:5], stream=st)

    ms = _time_calls(st, chain, steps, 3)
    return {"call": "cupcfd_gpu_dev_boundary_loop1..5 + cupcfd_gpu_dev_region_loop (FP64, bit-identical)",
            "us_per_chain": ms * 1e3, "boundaries": nB, "value": nB / (ms * 1e-3) / 1e9, "unit": "Gboundaries/s",
            "steps": steps, "config": "bench mesh, six regions assigned to the boundaries at random"}


def cpu_boundary_loops(n, reps):
    """Gboundaries/s of the reference's boundary-loop chain (its
    FluxMassDolfynBoundaryLoop1-5 and FluxMassDolfynRegionLoop templates,
    compiled unchanged, one core) on an n^3 generated mesh with the same six
    regions assigned at random."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    if O.load_ref() is None:
        return {"value": None, "sample": "reference build absent"}
    m = O.structgen(n, n, n)
    rng = np.random.Generator(np.random.Philox(key=SEED + 7))
    m.update(nRegions=6, regionType=np.array([0, 1, 2, 3, 4, 2], np.int32), regionUVW=rng.standard_normal(18),
             regionDen=rng.uniform(0.9, 1.1, 6), bndRegion=rng.integers(0, 6, m["nBnd"]).astype(np.int32))
    R = O.RefKernels(m).boundary_loops(rng.uniform(0.2, 0.8, 6))
    nF, nB, nC = m["nFaces"], m["nBnd"], m["nCells"]
    secs = R.boundary_chain(rng.uniform(1e-6, 1e-2, nF) * rng.choice([-1.0, 1.0], nF), rng.standard_normal(nC),
                            *[rng.uniform(1e-6, 1e-2, nB) for _ in range(4)], rng.uniform(1e-6, 1e-2, 6), reps)
    t = statistics.median(secs)
    return {"value": nB / t / 1e9, "unit": "Gboundaries/s", "cores": 1, "kind": "reference", "ms_per_chain": t * 1e3,
            "sample": f"{n}^3 generated mesh ({nB} boundaries), six random regions; median of {reps} chains"}


def bench_halo(cg, mesh, dev, st, steps, parts=8):
    """Halo pack / unpack (cupcfd_gpu_dev_halo_pack / _unpack) for one rank of
    the bench mesh cut into `parts` z-slabs (the reference's naive
    partition): the two cell planes its neighbours need, packed from phi,
    the float4 state and the three gradient components (32 bytes a cell),
    and as many ghost cells unpacked. The transfer between GPUs is NCCL's and
    needs more than one GPU; this times the two kernels around it."""
    import numpy as np
    import torch
    n = round(mesh.nCells ** (1 / 3))
    plane = n * n
    c2o, _ = mesh.numbering()
    o2c = np.empty_like(c2o)
    o2c[c2o] = np.arange(len(c2o), dtype=np.int32)
    z0 = n // parts * (parts // 2)                      # an interior slab [z0, z0 + n / parts)
    z1 = z0 + n // parts
    ref = lambda z: np.arange(z * plane, (z + 1) * plane, dtype=np.int64)
    send = torch.from_numpy(o2c[np.concatenate([ref(z0), ref(z1 - 1)])].astype(np.int32)).to(dev)
    ghost = torch.from_numpy(o2c[np.concatenate([ref(z0 - 1), ref(z1)])].astype(np.int32)).to(dev)
    nC, k = mesh.nCells, send.numel()
    phi = torch.rand(nC, device=dev)
    state = torch.rand(nC, 4, device=dev)
    grad = torch.rand(3, nC, device=dev)
    bp, bs, bg = torch.empty(k, device=dev), torch.empty(k, 4, device=dev), torch.empty(k, 3, device=dev)

    L, S = cg.lib(), cg._stream(st)
    fields = (cg.HaloField * 3)(cg.HaloField(phi.data_ptr(), 4, 1, 0, bp.data_ptr()),
                                cg.HaloField(state.data_ptr(), 16, 1, 0, bs.data_ptr()),
                                cg.HaloField(grad.data_ptr(), 4, 3, nC, bg.data_ptr()))

    def exchange():   # the three fields in one pack and one unpack launch
        cg.check(L.cupcfd_gpu_dev_halo_pack_fields(fields, 3, cg._p(send), k, S))
        cg.check(L.cupcfd_gpu_dev_halo_unpack_fields(fields, 3, cg._p(ghost), k, S))

    ms = _time_calls(st, exchange, steps, 3)
    return {"call": "cupcfd_gpu_dev_halo_pack_fields / _unpack_fields (phi, float4 state, 3 gradient components)",
            "us_per_exchange": ms * 1e3, "cells_packed": k, "cells_unpacked": k,
            "bytes_per_exchange": 2 * k * (32 + 4), "gbs": 2 * k * (32 + 4) / (ms * 1e-3) / 1e9, "steps": steps,
            "config": f"one rank of {parts} z-slabs of the bench mesh: 2 planes sent, 2 planes of ghosts"}


def bench_mesh_files(cg, n=128):
    """Mesh files: a generated n^3 mesh written and read back in the
    reference's HDF5 layout (cupcfd_gpu_mesh_save_hdf5 / _load_hdf5) and in
    the library's raw-binary format (cupcfd_gpu_mesh_save / _load), host
    clock, page cache warm."""
    import tempfile
    import torch
    mesh = cg.Mesh.structgen(n, n, n)
    out = {"mesh": f"{n}^3", "cells": mesh.nCells, "faces": mesh.nFaces}
    with tempfile.TemporaryDirectory() as d:
        for kind, save, load in (("hdf5", mesh.save_hdf5, cg.Mesh.load_hdf5),
                                 ("raw", mesh.save, cg.Mesh.load)):
            p = os.path.join(d, "m." + kind)
            t0 = time.perf_counter()
            save(p)
            t1 = time.perf_counter()
            m2 = load(p)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            size = os.path.getsize(p)
            m2.close()
            os.remove(p)
            out[kind] = {"bytes": size, "save_s": t1 - t0, "load_s": t2 - t1,
                         "load_gbs": size / (t2 - t1) / 1e9}
    mesh.close()
    return out


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def workload_config(n, order, world):
    """The `config` of a bench line for the n^3 workload (both arms print it)."""
    nC, nF, nFi, nB = face_counts(n)
    bm = bytes_model(nC, nF, nFi, nB)
    return {"workload": f"structgen {n}^3 unit cube, FP32-compensated forward+adjoint of "
                        f"GradientPhiGaussDolfyn + FluxMassDolfynFaceLoop",
            "mesh": f"{n}^3", "cells": nC, "faces": nF, "interior_faces": nFi, "boundary_faces": nB,
            "order": ["native", "morton", "owner", "rcm"][order], "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 ({bm['pipeline_f32'] / 1e9:.2f} GB compulsory traffic per step)"}


def run_reference(a):
    """The reference's own CPU kernels (oracle/_ref: GradientKernels.ipp and
    MassKernels.ipp compiled unchanged) on every host core, on the GPU arm's
    mesh: the n^3 mesh in one z-slab per core, as mpirun -n P with
    NaivePartitioner runs it (the kernels exchange nothing). The reference has
    no adjoint, so each step is its forward face loops."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    procs = min(os.cpu_count() or 1, a.cpu_n)
    n = a.cpu_n
    reps = max(3, min(a.steps, 30))
    warmup = min(a.warmup, 10)
    t0 = time.time()
    cb = cpu_baseline(n, procs, reps, warmup)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "Gfaces/s", "n_gpus": a.gpus,
            "steps": reps, "warmup": warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_config(n, a.order, a.gpus),
            "reference_step": "GradientPhiGaussDolfyn + FluxMassDolfynFaceLoop forward, FP64 (the reference has no "
                              "adjoint)",
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "Gfaces/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0},
            "wall_s": round(time.time() - t0, 1)}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(a):
    import numpy as np
    import torch
    cg = load_cupcfd()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = a.n
    t_build = time.time()
    mesh = cg.Mesh.structgen(n, n, n, order=a.order, device=local)
    torch.cuda.synchronize()
    t_build = time.time() - t_build
    nC, nF, nFi, nB = mesh.nCells, mesh.nFaces, mesh.nInteriorFaces, mesh.nBoundaries
    log(f"[rank {rank}] mesh {n}^3: {nC} cells, {nF} faces ({nFi} interior), built in {t_build:.2f} s, "
        f"{mesh.deviceBytes / 1e9:.2f} GB")
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + rank)
    # fields (internal numbering; i.i.d. so numbering does not change the distribution)
    phi = torch.rand(nC, generator=g, device=dev) * 2 - 1
    phiB = torch.rand(nB, generator=g, device=dev) * 2 - 1
    rho = torch.rand(nC, generator=g, device=dev) * 0.2 + 0.9
    uvw = torch.randn(3, nC, generator=g, device=dev)
    state = torch.stack([rho, uvw[0], uvw[1], uvw[2]], 1).contiguous()           # float4 per cell
    gface = torch.randn(nF, generator=g, device=dev)
    grad = torch.empty(3, nC, device=dev)
    mflux = torch.zeros(nF, device=dev)
    pbar = torch.empty(nC, device=dev)
    pbbar = torch.empty(nB, device=dev)
    sbar = torch.empty(nC, 4, device=dev)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream()
    F32 = cg.PREC_F32C

    def step():
        cg.dev_forward_adjoint(mesh, F32, phi, phiB, state, gface, grad, mflux, pbar, pbbar, sbar, loss, stream=st)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    K = a.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    vis = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    clocks = Clocks(vis[local] if local < len(vis) else local)
    clocks.start()
    time.sleep(0.3)
    launches0 = cg.launch_count()
    cg.timing_read()
    cg.timing_enable(True)        # per-kernel CUDA events on the launching stream, over the timed region
    t_start.record(st)
    for k in range(K):
        ev[k][0].record(st)
        step()
        ev[k][1].record(st)
    t_end.record(st)
    torch.cuda.synchronize()
    launches = cg.launch_count() - launches0
    cg.timing_enable(False)
    ktimes = cg.timing_read()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    status = mesh.check_status(st)
    if status != cg.E_SUCCESS:
        raise RuntimeError(f"forward+adjoint reported an error: {cg.last_error()}")
    total_ms = t_start.elapsed_time(t_end)
    total_ms = max_over_ranks(total_ms, dist, dev)
    ms_step = total_ms / K
    value = job_gfaces(world, nF, ms_step * 1e-3)
    sus = None
    if a.sustained_s > 0:
        # the same step for longer, after the timed region: the power-capped rate
        sus = sustained_run(step, st, a.sustained_s, ms_step, nF, world, vis[local] if local < len(vis) else local)

    # ---- the same work as the separate dev_forward and dev_adjoint calls, for comparison
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    K2p = max(1, K // 4)
    for _ in range(2):
        cg.dev_forward(mesh, F32, phi, phiB, state, grad, mflux, gface=gface, loss=loss, stream=st)
        cg.dev_adjoint(mesh, F32, grad, state, gface, pbar, pbbar, sbar, stream=st)
    fwd_t, adj_t = 0.0, 0.0
    for _ in range(K2p):
        e0.record(st)
        cg.dev_forward(mesh, F32, phi, phiB, state, grad, mflux, gface=gface, loss=loss, stream=st)
        e1.record(st)
        cg.dev_adjoint(mesh, F32, grad, state, gface, pbar, pbbar, sbar, stream=st)
        e2.record(st)
        torch.cuda.synchronize()
        fwd_t += e0.elapsed_time(e1)
        adj_t += e1.elapsed_time(e2)
    fwd_ms, adj_ms = fwd_t / K2p, adj_t / K2p
    step()
    torch.cuda.synchronize()

    # ---- plain FP64 forward on the same mesh
    phi64, phiB64 = phi.double(), phiB.double()
    st64 = state.double().t().contiguous()                                        # [4][nC] blocks
    grad64 = torch.empty(3, nC, dtype=torch.float64, device=dev)
    mf64 = torch.zeros(nF, dtype=torch.float64, device=dev)
    for _ in range(a.warmup):
        cg.dev_forward(mesh, cg.PREC_F64, phi64, phiB64, st64, grad64, mf64, stream=st)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    K64 = max(1, K // 2)
    e0.record(st)
    for _ in range(K64):
        cg.dev_forward(mesh, cg.PREC_F64, phi64, phiB64, st64, grad64, mf64, stream=st)
    e1.record(st)
    torch.cuda.synchronize()
    ms64 = e0.elapsed_time(e1) / K64

    # ---- the same forward + adjoint in FP64 (same work as the FP32 step)
    gf64 = gface.double()
    pbar64 = torch.empty(nC, dtype=torch.float64, device=dev)
    pbbar64 = torch.empty(nB, dtype=torch.float64, device=dev)
    sbar64 = torch.empty(4, nC, dtype=torch.float64, device=dev)
    loss64 = torch.zeros(1, dtype=torch.float64, device=dev)

    def step64():
        cg.dev_forward_adjoint(mesh, cg.PREC_F64, phi64, phiB64, st64, gf64, grad64, mf64, pbar64, pbbar64, sbar64,
                               loss64, stream=st)

    for _ in range(3):
        step64()
    e0.record(st)
    for _ in range(K64):
        step64()
    e1.record(st)
    torch.cuda.synchronize()
    ms64fa = e0.elapsed_time(e1) / K64

    # ---- FP32-compensated vs FP64 on the same inputs (forward + adjoint)
    cg.dev_forward(mesh, cg.PREC_F64, phi64, phiB64, st64, grad64, mf64, gface=gf64, loss=loss64, stream=st)
    cg.dev_adjoint(mesh, cg.PREC_F64, grad64, st64, gf64, pbar64, pbbar64, sbar64, stream=st)
    step()
    torch.cuda.synchronize()

    def err(x32, x64):
        rms_ref = float(torch.sqrt(torch.mean(x64 * x64)).item()) if x64.numel() else 0.0
        e = cg.error_norms(x32, x64, 1e-2 * rms_ref)
        return {"max_rel_normwise": e["max_rel_norm"], "rms_rel": e["rms_rel"], "max_rel_floor1e-2rms": e["max_rel_floor"]}

    errors = {
        "grad": err(grad.contiguous(), grad64),
        "massFlux": err(mflux.contiguous(), mf64),
        "phiBar": err(pbar, pbar64),
        "phiBBar": err(pbbar, pbbar64),
        "denBar": err(sbar[:, 0].contiguous(), sbar64[0].contiguous()),
        "uvwBar": err(sbar[:, 1:].t().contiguous(), sbar64[1:].contiguous()),
        "stateBar": err(sbar.t().contiguous(), sbar64),
        "loss_rel": abs(float(loss.item()) - float(loss64.item())) / abs(float(loss64.item())),
    }

    # ---- end to end through the reference-facing host-buffer call: float
    # host arrays (the FP32 path's own storage type, the reference's T = float
    # arrays), and for comparison the FP64 arrays of the T = double call
    K2 = max(1, min(K, a.e2e_steps))

    def host_call(dt, steps):
        hb = {}
        for nm, cnt in (("phi", nC), ("phiB", nB), ("den", nC), ("u", nC), ("v", nC), ("w", nC), ("gface", nF)):
            hb[nm] = torch.empty(cnt, dtype=dt, pin_memory=True)
        hb["phi"].copy_(phi.cpu()); hb["phiB"].copy_(phiB.cpu())
        hb["den"].copy_(rho.cpu()); hb["u"].copy_(uvw[0].cpu())
        hb["v"].copy_(uvw[1].cpu()); hb["w"].copy_(uvw[2].cpu()); hb["gface"].copy_(gface.cpu())
        out = {"grad": torch.empty(nC, 3, dtype=dt, pin_memory=True),
               "massFlux": torch.empty(nF, dtype=dt, pin_memory=True),
               "phiBar": torch.empty(nC, dtype=dt, pin_memory=True),
               "phiBBar": torch.empty(nB, dtype=dt, pin_memory=True),
               "denBar": torch.empty(nC, dtype=dt, pin_memory=True),
               "uBar": torch.empty(nC, dtype=dt, pin_memory=True),
               "vBar": torch.empty(nC, dtype=dt, pin_memory=True),
               "wBar": torch.empty(nC, dtype=dt, pin_memory=True),
               "loss": torch.empty(1, dtype=torch.float64, pin_memory=True)}
        hn = {k: v.numpy() for k, v in hb.items()}
        on = {k: v.numpy() for k, v in out.items()}
        args = (mesh, F32, hn["phi"], hn["phiB"], hn["den"], hn["u"], hn["v"], hn["w"], hn["gface"])
        cg.forward_adjoint(*args, out=on)   # warm (allocates the mesh's scratch buffers)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            cg.forward_adjoint(*args, out=on)
        te = (time.perf_counter() - t0) / steps
        te = max_over_ranks(te, dist, dev)
        es = torch.tensor([], dtype=dt).element_size()
        h2d = es * (5 * nC + nB + nF)
        d2h = es * (3 * nC + nF + 5 * nC + nB) + 8
        return {"value": job_gfaces(world, nF, te), "unit": "Gfaces/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": te * 1e3, "steps": steps}

    e2e = host_call(torch.float32, K2)
    e2e["call"] = ("cupcfd_gpu_forward_adjoint_f32 (pinned host float arrays in the reference's numbering: the "
                   "FP32 path's storage type, the reference's T = float arrays)")
    e2e_f64 = host_call(torch.float64, max(1, K2 // 2))
    e2e_f64["call"] = "cupcfd_gpu_forward_adjoint (pinned host FP64 arrays in the reference's numbering)"
    link = host_link(dev)

    # ---- roofline of the dominant kernel, from the device timers of the timed region
    bm = bytes_model(nC, nF, nFi, nB)
    peak, peak_src = measured_peaks()

    # ---- the momentum face loop (the next operator after the path), FP64, same mesh
    uvw = None
    if not a.no_uvw:
        uvw = bench_uvw(cg, mesh, dev, st, g, max(3, K // 4), 3, peak)
        uvw["roofline"]["peak_source"] = peak_src
        uvw["roofline"]["traffic"] = profile_traffic().get(f"k_uvw_f64_pf@{n}")
        if rank == 0 and world == 1 and not a.no_cpu:
            try:
                uvw["cpu_reference"] = cpu_uvw(min(a.cpu_n, 64), 5)
            except Exception as ex:
                uvw["cpu_reference"] = {"value": None, "sample": f"failed: {ex}"}
        torch.cuda.synchronize()
    # ---- the other rows either side of the path: boundary / region loops,
    # halo pack / unpack, mesh files (after the momentum loop, which wants
    # the mesh's default region)
    rows = None
    if not a.no_rows:
        rows = {"boundary_loops": bench_boundary_loops(cg, mesh, dev, st, max(3, K // 10)),
                "halo": bench_halo(cg, mesh, dev, st, max(3, K // 10))}
        if rank == 0 and world == 1:
            rows["mesh_files"] = bench_mesh_files(cg)
            if not a.no_cpu:
                try:
                    rows["boundary_loops"]["cpu_reference"] = cpu_boundary_loops(96, 20)
                except Exception as ex:
                    rows["boundary_loops"]["cpu_reference"] = {"value": None, "sample": f"failed: {ex}"}
        torch.cuda.synchronize()
    kbytes = {"k_fwd_madj_f32_pf": bm["fwd_madj_f32"], "k_gadj_f32_pf": bm["gadj_f32"], "k_fused_f32": bm["pipeline_f32"],
              "k_fwd_f32_pf": bm["fwd_f32"], "k_fwd_f32": bm["fwd_f32"], "k_adj_f32_pf": bm["adj_f32"],
              "k_adj_f32": bm["adj_f32"]}
    tot_ms = sum(v[1] for v in ktimes.values()) or 1.0
    kernels = {k: {"launches": v[0], "avg_ms": v[1] / max(v[0], 1), "share": v[1] / tot_ms,
                   "algorithmic_bytes": kbytes.get(k)} for k, v in ktimes.items()}
    kname = max(ktimes, key=lambda k: ktimes[k][1]) if ktimes else None
    kms = kernels[kname]["avg_ms"] if kname else float("nan")
    kb = kbytes.get(kname, 0)
    achieved = kb / (kms * 1e-3) / 1e9
    tr = profile_traffic().get(f"{kname}@{n}")
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr, "kernel": kname, "peak_source": peak_src, "algorithmic_bytes_per_launch": kb,
            "ms_per_launch": kms,
            "pipeline": {"algorithmic_bytes": bm["pipeline_f32"], "ms_per_step": ms_step,
                         "achieved": bm["pipeline_f32"] / (ms_step * 1e-3) / 1e9,
                         "frac": bm["pipeline_f32"] / (ms_step * 1e-3) / 1e9 / peak}}
    separate = {"fwd_ms": fwd_ms, "adj_ms": adj_ms, "value": world * nF / ((fwd_ms + adj_ms) * 1e-3) / 1e9,
                "fwd_gbs": bm["fwd_f32"] / (fwd_ms * 1e-3) / 1e9, "adj_gbs": bm["adj_f32"] / (adj_ms * 1e-3) / 1e9}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        try:
            cpu = cpu_baseline(a.cpu_n, 1, a.cpu_reps, 2, slabs=16)
        except Exception as ex:  # the baseline never blocks the GPU line
            cpu = {"value": None, "unit": "Gfaces/s", "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gfaces/s", "n_gpus": world, "steps": K, "warmup": a.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic, seeded: phi~U[-1,1], u,v,w~N(0,1), rho~U[0.9,1.1], phiB~U[-1,1], g_f~N(0,1)",
            "config": workload_config(n, a.order, world),
            "roofline": roof,
            "kernels": kernels,
            "separate_calls": separate,
            "mesh": {"order": ["native", "morton", "owner", "rcm"][a.order], "bandwidth": mesh.bandwidth,
                     "incidence_width": mesh.full_width or "general",
                     "forward_adjoint": ("two launches: forward with the mass-flux adjoint, then the gradient "
                                         "adjoint; the FP64 loss reduction on a second stream beside the second")},
            "fp64_plain_forward": {"value": world * nF / (ms64 * 1e-3) / 1e9, "unit": "Gfaces/s", "ms_per_step": ms64,
                                   "gbs": bm["fwd_f64"] / (ms64 * 1e-3) / 1e9,
                                   "frac": bm["fwd_f64"] / (ms64 * 1e-3) / 1e9 / peak},
            "fp64_forward_adjoint": {"value": world * nF / (ms64fa * 1e-3) / 1e9, "unit": "Gfaces/s",
                                     "ms_per_step": ms64fa},
            "error_vs_fp64": errors,
            "e2e": e2e,
            "e2e_fp64_host_arrays": e2e_f64,
            "host_link": link,
            "cpu_baseline": cpu,
            "uvw_face_loop1": uvw,
            "next_rows": rows,
            "gpu_launches": launches,
            "clocks": clk,
            "sustained": sus,
            "mesh_build_s": t_build,
        }
        print(json.dumps(line), flush=True)
    mesh.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--n", type=int, default=256, help="mesh is n^3 cells")
    ap.add_argument("--order", type=int, default=2, help="0 native, 1 morton, 2 owner, 3 rcm")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-n", type=int, default=None,
                    help="mesh of the CPU reference (default: the GPU arm's n); the reference arm cuts it into one "
                         "z-slab per host core, the 1-core baseline times one slab of 16")
    ap.add_argument("--cpu-reps", type=int, default=10)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-uvw", action="store_true", help="skip the momentum face loop measurement")
    ap.add_argument("--sustained-s", type=float, default=1.5,
                    help="after the timed region, run the step back to back this long and report its rate per "
                         "100 ms with the clocks (0: skip)")
    ap.add_argument("--no-rows", action="store_true",
                    help="skip the boundary-loop, halo and mesh-file measurements")
    a = ap.parse_args()
    if a.cpu_n is None:
        a.cpu_n = a.n
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        sys.exit(run_reference(a))
    sys.exit(run_gpu(a))


if __name__ == "__main__":
    main()
