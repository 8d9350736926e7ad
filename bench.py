#!/usr/bin/env python
"""LenseFlow throughput benchmark: 512^2 QU maps/s on B200 (one JSON line on rank 0).

Workload (one "step"): a batch of B = 64 independent (QU field, phi) pairs,
512 x 512, 2 arcmin pixels, forward LenseFlow with 7 RK4 steps in FP32,
including the float64 phi-derivative precompute (a new phi per map).
Inputs are seeded Gaussian random fields (8 distinct maps tiled to the batch)
with the workload's spectra; the batch's working set (~1.4 GB) is far larger
than the 126 MB L2, so no flush is needed between steps.

``value``  : maps/s with inputs resident in HBM, CUDA events on the launching
             stream, max over ranks.
``e2e``    : the same metric through the public host-buffer API
             (engine.HostPipeline): float64 fields and phi copied from pinned
             host memory, derivative precompute with the magnification check,
             lens, float64 result copied back, every step.
``roofline``: the dominant kernel's algorithmic bytes per launch over its
             average event-timed duration inside the timed region.
Multi-GPU: every rank lenses its own batch (no collective; weak scaling).
``--impl reference`` times the float64 CPU oracle on the host cores instead.
``--adjoint`` measures the adjoint lens (the transpose, run by every Wiener
filter iteration and gradient) on the same workload instead of the forward.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LenseFlow 512x512 QU maps/s (FP32, nsteps=7, incl. phi precompute)"
METRIC_ADJ = "LenseFlow 512x512 QU adjoint maps/s (FP32, nsteps=7, incl. phi precompute)"
UNIT = "maps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--nside", type=int, default=512)
    ap.add_argument("--ncomp", type=int, default=2)
    ap.add_argument("--nsteps", type=int, default=7)
    ap.add_argument("--theta", type=float, default=2.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="skip the gradient and Wiener-filter legs")
    ap.add_argument("--serving-seconds", type=float, default=1.5)
    ap.add_argument("--serving-requests", type=int, default=2000,
                    help="requests measured at 80%% of the measured capacity (0: skip that stream)")
    ap.add_argument("--serving-rate", type=float, default=200.0)
    ap.add_argument("--adjoint", action="store_true", help="time the adjoint lens instead of the forward lens")
    return ap.parse_args()


def metric_name(a):
    return METRIC_ADJ if a.adjoint else METRIC


def workload_config(a):
    kind = "adj" if a.adjoint else "fwd"
    return {"workload": f"lenseflow_{kind}_qu{a.nside}_b{a.batch}_n{a.nsteps}" if a.ncomp == 2 else
            f"lenseflow_{kind}_c{a.ncomp}_{a.nside}_b{a.batch}_n{a.nsteps}",
            "adjoint": bool(a.adjoint), "nside": a.nside, "ncomp": a.ncomp, "batch_per_gpu": a.batch, "rk4_steps": a.nsteps,
            "theta_pix_arcmin": a.theta,
            "phi_spectrum": "1/[l^2 (l+1)^2 (1+(l/60)^2)], 2.5' rms deflection (well-posed reading)",
            "fields": "QU from E ~ l^-2 exp(-(l/2000)^2), 5 uK rms, B=0" if a.ncomp == 2 else "T",
            "l2": "inputs larger than L2 (working set ~1.4 GB per GPU), no flush",
            "magnification_check": "det(I + t grad grad phi) > 0 checked once before the timed region; "
                                   "the e2e leg checks every call",
            "phi_path": "float64 phi precompute writing p = M(t)^-1 grad phi at the 2n+1 stage times "
                        "(lf_phi_precompute_pp), then lf_lense_flow_pp",
            "parallelism": f"replicas x{a.gpus} (independent batches, no collective)"}


# ------------------------------------------------------------------ CPU legs
def _cpu_lens_one(args):
    """One map through the float64 oracle (runs in a spawned worker)."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from oracle import lenseflow_ref as R
    from cmblensing_b200.simulate import lens_batch
    N, theta, C, n, seed, adjoint = args
    f, phis = lens_batch(N, theta, 1, C, seed0=seed)
    pw = R.pix_width_of(theta)
    d = R.phi_derivatives(phis[0], pw)
    t0 = time.perf_counter()
    for c in range(C):
        R.primal_lense_flow(f[0, c], phis[0], pw, n, 1, adjoint, d)
    return time.perf_counter() - t0


class CpuPool:
    """Spawned process pool, one single-threaded worker per host core."""

    def __init__(self):
        import multiprocessing as mp
        self.cores = os.cpu_count() or 1
        self.pool = mp.get_context("spawn").Pool(self.cores, initializer=_set_single_thread)

    def run(self, a, nmaps, seed=0):
        """(time, CPU seconds) to lens ``nmaps`` maps, one per worker in parallel.

        The time is the slowest worker's lens time: input generation, done in
        the workers before their clocks start, is excluded.
        """
        jobs = [(a.nside, a.theta, a.ncomp, a.nsteps, seed + i, bool(a.adjoint)) for i in range(nmaps)]
        per = self.pool.map(_cpu_lens_one, jobs, chunksize=1)
        waves = math.ceil(nmaps / self.cores)
        return max(per) * waves, sum(per)

    def close(self):
        self.pool.close()
        self.pool.join()


def _set_single_thread():
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"


def cpu_describe():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pool = CpuPool()
    nmaps = pool.cores
    for i in range(max(a.warmup, 0)):
        pool.run(a, nmaps, seed=100 * i)
    walls = []
    for i in range(a.steps):
        w, _ = pool.run(a, nmaps, seed=1000 + 100 * i)
        walls.append(w)
    pool.close()
    total = sum(walls)
    value = nmaps * a.steps / total
    sample = (f"{nmaps} maps per step ({a.nside}^2, C={a.ncomp}, n={a.nsteps}, float64 numpy oracle, "
              f"one map per process), {pool.cores} processes on {cpu_describe()}")
    line = {"impl": "reference", "metric": metric_name(a), "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000 * total / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": pool.cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference = float64 numpy restatement of cmb_lensing/lense_flow.py (jax is not installed)"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ multi-rank
def max_over_ranks(ms, dist=None, device="cpu"):
    """The slowest rank's time (every rank must call this, in the same order)."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(world, batch_per_rank, steps, ms):
    """Whole-job maps/s: every rank lenses its own batch; the job takes the slowest rank's time."""
    return world * batch_per_rank * steps / (ms / 1000.0)


# ----------------------------------------------------------- algorithmic bytes
def row_bytes_per_lens(C, n, P, in_bytes=4, out_bytes=4, p_planes=2, adjoint=False):
    """Bytes the row kernels of one lens must move per map (float32 state).

    Forward -- init: read f, write y0 and S.  Stage 1: read Gx, S, y0, the phi
    planes; write acc, S.  Stages 2-3: also read acc.  Stage 4: read Gx, S,
    y0, acc, phi planes; write y0 and S (the last stage writes the output
    instead and no S).  Adjoint -- the same with V read in place of S, and
    both U and V written (init: read f, the p planes; write y0, U, V).
    ``p_planes`` = 2 when p is read at the stage time, 5 when it is formed
    from the derivative planes.
    """
    ph = 4 * p_planes
    w = 8 if adjoint else 4  # next-stage spectra written per component
    init = (in_bytes + 4 + w) * C + (ph if adjoint else 0)
    s1 = 16 * C + w * C + ph
    s23 = 20 * C + w * C + ph
    s4 = 20 * C + w * C + ph
    last_adj = -(4 + w) * C + out_bytes * C  # last stage: no y0/spectra writes, one output write
    total = init + n * (s1 + 2 * s23 + s4) + last_adj
    return total * P


def row_kernel_name(N, C, adjoint=False):
    """The stage row-pass kernel the engine launches for a lens of this shape."""
    if N == 512 and C == 2:
        if adjoint:
            return ("k_row_pair_adj (adjoint RK4 row pass, both rates from one full-length complex transform, "
                    "update in registers)")
        return "k_row_pair (RK4 row pass, two components in full-length complex transforms, update in registers)"
    return "k_row (RK4 row pass + fused epilogue)"


def col_bytes_per_lens(C, n, P):
    """Column kernels: read and write one row-spectral array (N x N/2 complex64 = 4P bytes) per plane."""
    return 4 * n * 8 * C * P


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per map of one RK4
# stage-1 launch of the dominant row kernel, from one ncu capture each: the
# 21st launch of each kernel in a 32-map step (RK4 step 6, stage 1); the capture's
# traffic scales with the maps of the launch.  The algorithmic bytes of that
# launch are stage1_bytes_per_map(C) N^2; the reads equal them, the writes
# fall short by what is still in L2 when the launch ends.
NCU_STAGE1_TRAFFIC_PER_MAP = {
    ("k_row_pair", 512, 2): (268.50e6 + 96.53e6) / 32,
    ("k_row_pair_adj", 512, 2): (268.49e6 + 151.81e6) / 32,
}


def stage1_bytes_per_map(C, adjoint=False):
    """Algorithmic bytes per N^2 of one stage-1 row launch (see row_bytes_per_lens)."""
    return (24 if adjoint else 20) * C + 8


def p_plane_bytes_per_lens(n, P):
    """k_p_planes: read the five derivative planes, write p_x, p_y at the 2n+1 stage times."""
    return (20 + 8 * (2 * n + 1)) * P


def phi_pp_bytes_per_map(n, P):
    """The phi precompute with the p planes formed in its row pass (lf_phi_precompute_pp, no derivative
    planes requested), per map: row r2c (read phi 8, write the half spectrum 8), in-place column FFT
    (8 + 8), derivative columns (read 8, write five packed float32 spectra 20), fused row pass (read 20,
    write p at 2n+1 times 8 (2n+1))."""
    return (16 + 16 + 28 + 20 + 8 * (2 * n + 1)) * P


def survey_bytes_per_map(C, n, P):
    """Minimal-pass model: 4n(36C+20)P + 8CP + 140P (phi precompute)."""
    return (4 * n * (36 * C + 20) + 8 * C + 140) * P



# ----------------------------------------------------------------- serving
SERVE_SIZES = {128: 3.0, 256: 3.0, 512: 2.0, 1024: 2.0}


def _wf_problem(N, C, theta, seed):
    """A Wiener-filter request's problem: beam 1', noise 2 (QU) / 10 (T) uK', hole mask, data lensed by the engine."""
    import numpy as np
    import torch
    import cmblensing_b200 as cl
    from cmblensing_b200 import engine, matrix_operators as mo
    from cmblensing_b200.simulate import ARCMIN, hole_mask, inference_problem
    p = inference_problem(N, theta, beam_fwhm=1.0, noise_t=10.0, noise_p=2.0, seed=seed, bb_fraction=0.01)
    pw = theta * ARCMIN
    w = 2.0 * np.ones(N // 2 + 1, dtype=np.complex128)
    w[0] = w[-1] = 1.0
    kw = dict(nside=N, theta_pix=theta, pix_width=pw, fourier_weights=w)
    mask = mo.PixelMask(mask_map=hole_mask(N, theta), **kw)
    if C == 1:
        f = cl.FlatS0(scalar_matrix=p["t"], **kw)
        D = lambda a: mo.DiagonalScalar(scalar_matrix=a, **kw)
        Cf, Cn, B, noise = D(p["cf_tt"]), D(p["cn_t"]), D(p["beam"]), [p["n_t"]]
    else:
        f = cl.FlatS2(polar_matrix_1=p["e"], polar_matrix_2=p["b"], **kw)
        D = lambda a, b: mo.DiagonalEB(matrix_EE=a, matrix_BB=b, **kw)
        Cf, Cn, B, noise = D(p["cf_ee"], p["cf_bb"]), D(p["cn_p"], p["cn_p"]), D(p["beam"], p["beam"]), [p["n_e"], p["n_b"]]
    fmap = cl.map(cl.eb2qu(f))
    mats = np.stack([getattr(fmap, k) for k in fmap._matrix_names()])[None]
    lensed = engine.lense_flow_batch(torch.as_tensor(mats, device="cuda"),
                                     torch.as_tensor(np.fft.irfft2(p["phi"], s=(N, N))[None], device="cuda"), pw,
                                     n=7)[0].double().cpu().numpy()
    lf = cl.qu2eb(cl.fourier(fmap.replace(**{k: lensed[i] for i, k in enumerate(fmap._matrix_names())})))
    d = mask * (B * lf)
    data = d.replace(**{k: getattr(d, k) + noise[i] for i, k in enumerate(d._matrix_names())})
    return dict(phi=cl.FlatS0(scalar_matrix=p["phi"], **kw), data=data, Cf=Cf, Cn=Cn, M=mask, B=B)


def _event_ms(fn, reps=1):
    """Milliseconds of ``reps`` calls of fn on the current stream (CUDA events, synchronised on both sides)."""
    import torch
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_gradient(a, dev):
    """Config-2 workload: the LenseFlow part of grad_phi_logpdf at 256^2 IQU, 3' pixels, n = 7, FP32.

    One unit = one (f, phi) pair through the phi-derivative precompute, the
    forward lens and the reverse pass that yields (delta_f, delta_phi in the
    Fourier basis), batched 16 pairs per call; the reference scheme (forward
    lens + reverse ODE from Lf, lf_lense_flow_vjp) and the checkpointed exact
    scheme (lf_lense_flow_vjp_ckpt, forward included) side by side.
    """
    import numpy as np
    import torch
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import ARCMIN, lens_batch
    N, C, B, n, theta = 256, 3, 16, 7, 3.0
    pw = theta * ARCMIN
    f, phis = lens_batch(N, theta, B, C, seed0=600)
    plan = engine.get_plan(N, C, pw, "f32", device=dev)
    ft = torch.as_tensor(f, device=dev, dtype=torch.float32)
    phif = torch.as_tensor(np.fft.rfft2(phis), device=dev)
    cot = torch.as_tensor(np.random.default_rng(601).standard_normal(f.shape), device=dev, dtype=torch.float32)
    planes = torch.empty((B, 5, N, N), dtype=torch.float32, device=dev)
    phi_ws = torch.empty(plan.phi_workspace_bytes(B), dtype=torch.uint8, device=dev)

    def ref_scheme():
        plan.phi_planes(phif, check_det=False, out=planes, workspace=phi_ws)
        lensed = plan.lense_flow(ft, planes, n=n)
        return plan.lense_flow_vjp(lensed, cot, planes, n=n, phi_basis="fourier")

    def exact_scheme():
        plan.phi_planes(phif, check_det=False, out=planes, workspace=phi_ws)
        return plan.lense_flow_vjp_ckpt(ft, cot, planes, n=n, phi_basis="fourier")

    out = {"workload": "grad_lenseflow_iqu256_b16_n7", "nside": N, "ncomp": C, "batch": B, "rk4_steps": n,
           "theta_pix_arcmin": theta, "unit": "maps/s",
           "what": "phi precompute + forward lens + reverse pass (delta_f, Fourier delta_phi), FP32"}
    for name, fn in (("reference_scheme", ref_scheme), ("exact_scheme", exact_scheme)):
        for _ in range(3):
            fn()
        reps = 10
        ms = _event_ms(fn, reps)
        out[name] = {"maps_per_s": B * reps / (ms / 1000.0), "ms_per_call": ms / reps}
    _, dphi_r = ref_scheme()
    _, dphi_e = exact_scheme()
    torch.cuda.synchronize()
    out["rel_l2_exact_vs_reference_dphi"] = float((dphi_e - dphi_r).norm() / dphi_r.norm())
    out["note"] = ("the two schemes' delta-phi differ by the reference scheme's RK4 discretisation gap; "
                   "tests/test_configs_gpu.py checks the exact one against finite differences to 1e-6")
    return out


def run_wf(a, dev):
    """Config-3 workload: lensed Wiener filter at 512^2 QU, 2' pixels, 1' beam, 2 uK' pol noise, 30-hole mask.

    A batch of 8 problems solved together by the device PCG (FP32 operator,
    float64 dots, true residual from the FP64 engine every 10 iterations,
    CG blocks replayed from a CUDA graph) to ||r||/||b|| = 1e-6; one
    application of A for the batch timed alone; problem 0 solved again by the
    FP64 engine to 1e-10 as the reference solution.
    """
    import torch
    from cmblensing_b200.wf_engine import DeviceWienerFilter
    N, C, theta, B = 512, 2, 2.0, 8
    probs = [_wf_problem(N, C, theta, seed=700 + i) for i in range(B)]
    wf = DeviceWienerFilter(problems=probs, n=7)
    x0 = wf.b_vector()
    for _ in range(3):
        wf.apply_A(x0)
    reps = []
    for _ in range(9):
        reps.append(_event_ms(lambda: wf.apply_A(x0)))
    a_ms = sorted(reps)[len(reps) // 2]
    wf64 = DeviceWienerFilter(problems=probs[:1], n=7, precision="f64")
    x64, it64 = wf64.solve(rel_tol=1e-10, maxiter=3000)
    out = {"workload": "wf_qu512_masked_b8_n7", "nside": N, "ncomp": C, "batch": B, "rk4_steps": 7,
           "theta_pix_arcmin": theta, "beam_fwhm_arcmin": 1.0, "noise_pol_uk_arcmin": 2.0, "mask": "30 holes",
           "refine_every": 10, "apply_A_ms_batch": a_ms, "apply_A_ms_per_problem": a_ms / B,
           "fp64_solution": {"rel_tol": 1e-10, "iterations": it64, "engine": "FP64 operator"}}
    # to the workload's 1e-6 relative residual, and further, to a solution within 1e-6 of the FP64 one
    for key, tol in (("solve_rel_tol_1e-6", 1e-6), ("solve_rel_tol_1e-8", 1e-8)):
        kw = dict(rel_tol=tol, refine_every=10, maxiter=1000)
        wf.solve(**kw)  # warm: plans, graph capture path
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x, its = wf.solve(**kw)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out[key] = {"iterations": its, "solve_wall_s_batch": wall, "wall_s_per_solve": wall / B,
                    "graph_blocks_replayed": wf.graph_blocks,
                    "rel_l2_vs_fp64_solution": float((x[0] - x64).norm() / x64.norm())}
    return out


def _serve_stream(srv, make, rng, rate, nreq, warm=0):
    """Submit ``warm + nreq`` requests as a Poisson stream at ``rate`` (None: all at once), wait for all;
    return (the ``nreq`` measured requests, seconds from the first measured submission to the last
    completion)."""
    import numpy as np
    reqs = [make() for _ in range(warm + nreq)]
    gaps = rng.exponential(1.0 / rate, size=len(reqs)) if rate else np.zeros(len(reqs))
    tnext = time.perf_counter()
    for r, g in zip(reqs, gaps):
        tnext += g
        dt = tnext - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        srv.submit(r)
    t_wait = time.perf_counter()
    ok = all(r.done.wait(max(1.0, 900 - (time.perf_counter() - t_wait))) for r in reqs)
    meas = reqs[warm:]
    t_end = max((r.t_done for r in meas if r.t_done), default=time.perf_counter())
    return meas, t_end - meas[0].t_submit, ok


def _serve_summary(reqs, span, ok):
    from cmblensing_b200.serve import latency_summary, lens_tail_breakdown
    wsum = sum(r.nside * r.nside * r.ncomp for r in reqs if r.error is None) / (512.0 * 512.0 * 2)
    lat = [r for r in reqs if r.latency is not None]
    k = max(1, len(lat) // 10)
    return {"requests": len(reqs), "all_completed": bool(ok), "errors": sum(r.error is not None for r in reqs),
            "error_samples": sorted({f"{r.kind} N={r.nside} C={r.ncomp}: {r.error!r}"[:300]
                                     for r in reqs if r.error})[:4],
            "seconds": span, "requests_per_s": len(reqs) / span,
            "qu512_equivalent_maps_per_s": wsum / span,
            "latency": latency_summary(reqs),
            "latency_by_kind": {kd: latency_summary([r for r in reqs if r.kind == kd])
                                for kd in ("lens", "delens", "wf")},
            "lens_tail_1pct": lens_tail_breakdown(reqs),
            # a bounded queue: the last tenth of the stream waits no longer than the first
            "p50_first_tenth_ms": latency_summary(lat[:k]).get("p50_ms"),
            "p50_last_tenth_ms": latency_summary(lat[-k:]).get("p50_ms")}


def run_serving(a):
    """Config-4 stream: mixed kinds/sizes/components.  (1) capacity: a burst of requests submitted at once,
    completions per second; (2) a Poisson stream at 80% of that capacity, ``--serving-requests`` measured
    after a tenth as many warm-up requests; (3) the specified 200 req/s for ``--serving-seconds``; and the same
    mix one request at a time with plain engine calls."""
    import numpy as np
    import torch
    from cmblensing_b200.serve import Request, Server, run_alone
    from cmblensing_b200.simulate import lens_batch
    rng = np.random.default_rng(4242)
    pools, wf = {}, {}
    for N, th in SERVE_SIZES.items():
        for C in (1, 2):
            f, ph = lens_batch(N, th, 2, C, seed0=N + C)
            pools[(N, C)] = (f, ph)
            wf[(N, C)] = _wf_problem(N, C, th, seed=N + C)
    wf_kw = dict(rel_tol=1e-5, refine_every=10, maxiter=300)

    def make():
        kind = rng.choice(["lens", "delens", "wf"], p=[0.5, 0.2, 0.3])
        N = int(rng.choice(list(SERVE_SIZES), p=[0.4, 0.3, 0.2, 0.1]))
        C = int(rng.choice([1, 2]))
        th = SERVE_SIZES[N]
        if kind == "wf":
            return Request("wf", N, C, th, problem=wf[(N, C)], n=7, wf_kwargs=wf_kw)
        f, ph = pools[(N, C)]
        i = int(rng.integers(2))
        return Request(str(kind), N, C, th, f=f[i], phi=ph[i], n=7)

    # every lens shape's slots and batch-bucket graphs before the server starts, then one request of every
    # shape (plans, kernel attributes, the Wiener-filter path), all outside the measurement
    srv = Server(max_batch=16)
    for N, th in SERVE_SIZES.items():
        for C in (1, 2):
            srv.prepare(N, C, th)
    srv.start()
    warm = [srv.submit(Request(k, N, C, th, f=pools[(N, C)][0][0], phi=pools[(N, C)][1][0], n=7))
            for N, th in SERVE_SIZES.items() for C in (1, 2) for k in ("lens", "delens")]
    warm += [srv.submit(Request("wf", N, C, th, problem=wf[(N, C)], n=7, wf_kwargs=wf_kw))
             for N, th in SERVE_SIZES.items() for C in (1, 2)]
    for r in warm:
        r.done.wait(300)
    out = {"mix": "50% lens / 20% inverse / 30% Wiener filter; N 128/256/512/1024 at 0.4/0.3/0.2/0.1; "
                  "T or QU 50/50", "wf_stop": "||r||/||b|| < 1e-5, FP64 residual every 10 iterations",
           "weighting": "qu512_equivalent_maps_per_s counts a request as N^2 C / (512^2 * 2) maps"}
    burst, span, ok = _serve_stream(srv, make, rng, None, max(60, a.serving_requests // 8))
    cap = len(burst) / span
    out["capacity"] = {"requests_per_s": cap, "method": "a burst submitted at once, completions per second",
                       **{k: v for k, v in _serve_summary(burst, span, ok).items() if k != "latency_by_kind"}}
    if a.serving_requests > 0:
        reqs, span, ok = _serve_stream(srv, make, rng, 0.8 * cap, a.serving_requests,
                                       warm=max(1, a.serving_requests // 10))
        out["at_80pct_capacity"] = {"offered_per_s": 0.8 * cap, **_serve_summary(reqs, span, ok)}
    nreq = int(rng.poisson(a.serving_rate * a.serving_seconds))
    if nreq > 0:
        reqs, span, ok = _serve_stream(srv, make, rng, a.serving_rate, nreq)
        out["at_specified_rate"] = {"offered_per_s": a.serving_rate, "seconds_of_arrivals": a.serving_seconds,
                                    **_serve_summary(reqs, span, ok)}
    srv.stop()
    # one request at a time, plain engine calls, on a sample of the same mix
    sample = [make() for _ in range(40)]
    torch.cuda.synchronize()
    ts = time.perf_counter()
    for r in sample:
        run_alone(r)
    torch.cuda.synchronize()
    seq = (time.perf_counter() - ts) / len(sample)
    out["one_at_a_time"] = {"requests_per_s": 1.0 / seq, "sample_requests": len(sample)}
    out["capacity_over_one_at_a_time"] = cap * seq
    return out

# --------------------------------------------------------------------- main
def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pool = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        pool = CpuPool()  # spawn before any CUDA work

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from cmblensing_b200 import _native as nat
    from cmblensing_b200 import engine
    from cmblensing_b200.simulate import lens_batch, ARCMIN

    N, C, B, n = a.nside, a.ncomp, a.batch, a.nsteps
    P = N * N
    pw = a.theta * ARCMIN
    uniq = min(8, B)
    f_u, phi_u = lens_batch(N, a.theta, uniq, C, seed0=17 * rank)
    reps = [i % uniq for i in range(B)]
    f_host = np.ascontiguousarray(f_u[reps])
    phi_host = np.ascontiguousarray(phi_u[reps])

    plan = engine.get_plan(N, C, pw, "f32", device=dev)
    f_dev = torch.as_tensor(f_host, device=dev, dtype=torch.float32)
    phi_dev = torch.as_tensor(phi_host, device=dev)
    out_dev = torch.empty_like(f_dev)
    pp = torch.empty((B, 2 * n + 1, 2, N, N), dtype=torch.float32, device=dev)
    ws = torch.empty(plan.workspace_bytes(B, a.adjoint), dtype=torch.uint8, device=dev)
    phi_ws = torch.empty(plan.phi_workspace_bytes(B), dtype=torch.uint8, device=dev)

    def step():
        # the float64 phi precompute writes p = M(t)^-1 grad phi at the 2n+1 stage times directly
        plan.phi_pp(phi_dev, n, check_det=False, out=pp, workspace=phi_ws)
        plan.lense_flow_pp(f_dev, pp, n, adjoint=a.adjoint, out=out_dev, workspace=ws)

    # the magnification check once, outside the timed region (the e2e leg checks every call)
    plan.phi_pp(phi_dev[:uniq], n, check_det=True)
    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    plan.profile_reset()
    plan.profile(True)
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(a.steps):
        step()
    ev1.record()
    barrier()
    plan.profile(False)
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    row_ms, row_n = plan.profile_read(nat.LF_KIND_ROW)
    col_ms, col_n = plan.profile_read(nat.LF_KIND_COL)
    phi_ms, phi_n = plan.profile_read(nat.LF_KIND_PHI)
    pp_ms, pp_n = plan.profile_read(nat.LF_KIND_PP)
    ms = max_over_ranks(ms, dist, dev)
    value = aggregate_value(world, B, a.steps, ms)

    # parity spot check of this run's output (one map) against the first lens of the batch in FP64 engine
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    row_b = row_bytes_per_lens(C, n, P, 4, 4, adjoint=a.adjoint) * B / max(4 * n + 1, 1)  # per launch, all maps
    col_b = col_bytes_per_lens(C, n, P) * B / max(4 * n, 1)
    kinds = {"row": (row_ms, row_n, row_b), "col": (col_ms, col_n, col_b)}
    dom = max(kinds, key=lambda k: kinds[k][0])
    k_ms, k_n, k_b = kinds[dom]
    avg_s = (k_ms / max(k_n, 1)) / 1000.0
    achieved = k_b / avg_s / 1e9 if avg_s > 0 else 0.0
    kname = row_kernel_name(N, C, a.adjoint) if dom == "row" else "k_col (column FFT pass)"
    t_map = NCU_STAGE1_TRAFFIC_PER_MAP.get((kname.split()[0], N, C)) if dom == "row" else None
    traffic = t_map * B if t_map is not None else None
    step_gbs = survey_bytes_per_map(C, n, P) * (value / world) / 1e9
    # the bytes this engine's path moves per map: row + column passes, phi
    # precompute and the stage-time p planes
    path_b = (row_bytes_per_lens(C, n, P, adjoint=a.adjoint) + col_bytes_per_lens(C, n, P)
              + phi_pp_bytes_per_map(n, P))
    path_gbs = path_b * (value / world) / 1e9

    result = {"metric": metric_name(a), "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
              "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
              "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(a),
              "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm_peak,
                           "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": traffic,
                           "traffic_launch": "RK4 stage 1 (ncu capture of a 32-map step, scaled to the batch)"
                           if traffic is not None else None,
                           "traffic_launch_algorithmic_bytes": stage1_bytes_per_map(C, a.adjoint) * P * B
                           if traffic is not None else None,
                           "peak_source": peak_src,
                           "bytes_per_launch": k_b, "avg_launch_ms": avg_s * 1000.0,
                           "step_model_gbs": step_gbs, "step_model_frac": step_gbs / hbm_peak,
                           "step_model": "(4n(36C+20)+8C+140) N^2 bytes per map",
                           "step_path_bytes_per_map": path_b, "step_path_frac": path_gbs / hbm_peak},
              "kernel_ms_per_step": {"row": row_ms / a.steps, "col": col_ms / a.steps, "phi": phi_ms / a.steps,
                                     "p_planes": pp_ms / a.steps},
              "gpu_launches": (row_n + col_n + phi_n + pp_n) // a.steps * a.steps,
              "clocks": clk}

    # ------------------------------------------------------------ e2e leg
    if not a.no_e2e:
        pipe = engine.HostPipeline(plan, B, io_dtype=torch.float64)
        fh = torch.from_numpy(f_host).pin_memory()
        ph = torch.from_numpy(phi_host).pin_memory()
        ohs = [torch.empty_like(fh).pin_memory() for _ in range(2)]  # step k writes ohs[k % 2]
        # every step is one call (its own H2D, lens, D2H and magnification check); calls are queued
        # without waiting, so a step's first copies overlap the previous step's last chunks
        for k in range(max(a.warmup, 4)):  # eager + graph capture for both minima rings
            pipe(fh, ph, ohs[k % 2], n=n, adjoint=a.adjoint, wait=False)
        pipe.wait()
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(a.steps):
            pipe(fh, ph, ohs[k % 2], n=n, adjoint=a.adjoint, wait=False)
        pipe.wait()
        e1.record()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        result["e2e"] = {"value": aggregate_value(world, B, a.steps, ems), "unit": UNIT,
                         "h2d_bytes_per_step": pipe.h2d_bytes(), "d2h_bytes_per_step": pipe.d2h_bytes(),
                         "api": "engine.HostPipeline (float64 host I/O, pinned; calls queued with wait=False, "
                                "joined by wait() before the closing event)"}
        # parity of the bench output against the device-resident leg
        oh = ohs[(a.steps - 1) % 2]
        diff = float((torch.as_tensor(oh[:1], device=dev).float() - out_dev[:1]).norm() / out_dev[:1].norm())
        result["e2e"]["rel_l2_vs_device_leg"] = diff

    # ---------------------------------------------------- FP64 comparator
    if not a.no_fp64 and not a.adjoint and rank == 0:  # the float64 restatement is forward-only
        sys.path.insert(0, os.path.join(ROOT, "baseline"))
        from fp64_torch import lense_flow_fp64
        nb = 4
        f64 = torch.as_tensor(f_host[:nb], device=dev)
        p64 = torch.as_tensor(phi_host[:nb], device=dev)
        lense_flow_fp64(f64, p64, pw, n)
        torch.cuda.synchronize()
        reps = []
        for _ in range(7):  # the median of seven event-timed calls
            c0 = torch.cuda.Event(enable_timing=True)
            c1 = torch.cuda.Event(enable_timing=True)
            c0.record()
            ref64 = lense_flow_fp64(f64, p64, pw, n)
            c1.record()
            torch.cuda.synchronize()
            reps.append(c0.elapsed_time(c1) / 1000.0)
        dt = sorted(reps)[len(reps) // 2]
        ours = out_dev[:nb].double()
        rel = float((ours - ref64).norm() / ref64.norm())
        result["fp64_restatement"] = {"value": nb / dt, "unit": UNIT, "batch": nb, "repeats": len(reps),
                                      "spread_s": [min(reps), max(reps)],
                                      "what": "torch float64 restatement of the reference op sequence (cuFFT), "
                                              "not the reference; median of 7 CUDA-event-timed calls",
                                      "speedup_of_value": value / world / (nb / dt),
                                      "rel_l2_fp32_vs_fp64": rel}

    # ---------------------------------------------------- configs 2 and 3
    # the 1-GPU legs (gradient, Wiener filter, serving) run only in single-process runs: under torchrun the
    # other ranks would idle at the closing barrier meanwhile
    if rank == 0 and world == 1 and not a.no_workloads:
        for key, fn in (("gradient", run_gradient), ("wf", run_wf)):
            try:
                result[key] = fn(a, dev)
            except Exception as e:  # the headline numbers stand on their own
                result[key] = {"error": repr(e)}

    # ---------------------------------------------------- serving
    if rank == 0 and world == 1 and (a.serving_seconds > 0 or a.serving_requests > 0):
        try:
            result["serving"] = run_serving(a)
        except Exception as e:  # the headline numbers stand on their own
            result["serving"] = {"error": repr(e)}

    # ---------------------------------------------------- CPU baseline
    if pool is not None:
        nm = pool.cores
        pool.run(a, min(nm, 2))  # warm the workers (imports)
        wall, busy = pool.run(a, nm, seed=500)
        pool.close()
        result["cpu_baseline"] = {"value": nm / wall, "unit": UNIT, "cores": pool.cores, "kind": "port",
                                  "sample": f"{nm} maps ({N}^2, C={C}, n={n}) through the float64 numpy oracle, "
                                            f"one single-threaded process per core on {cpu_describe()}; "
                                            f"{busy:.1f} s of CPU work"}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
