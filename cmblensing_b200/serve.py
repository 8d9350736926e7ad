"""Device-resident continuous-batching service for lens, delens and Wiener-filter requests.

Requests of mixed grid sizes arrive as they like (``Server.submit``).  A
scheduler thread admits them against an HBM budget, groups lens and delens
requests by (N, components, direction) and launches each group as one
batched engine call into a *slot*: static device buffers plus a CUDA graph
of the phi-derivative precompute and the LenseFlow launch sequence,
captured once per batch-size bucket and replayed afterwards.  Every slot has
its own stream, so batches of different shapes run concurrently on the
device; while they run, newly arrived requests queue for the next batch of
their group.  A batch's completion event frees its slot and memory and
completes its requests.  Wiener-filter solves (data-dependent CG iteration
counts) wait per (N, components, pixel size); a free worker thread, each
with its own stream, takes the oldest group (up to ``wf_batch`` problems)
and solves it with the batched device-resident PCG of ``wf_engine``
(operators precomputed per problem, CG scalars on the device).

Each lensed map is computed by exactly the kernels and tiles it would use
alone, so a request's result is bit-identical whether it runs alone or in a
mix (tested).
"""
from __future__ import annotations

import collections
import queue
import sys
import threading
import time

import numpy as np
import torch

from . import _native as nat
from . import engine
from .simulate import ARCMIN

_req_ids = iter(range(1 << 62))


class Request:
    """One unit of work.  ``kind`` is "lens", "delens" or "wf".

    lens/delens: ``f`` [C, N, N] and ``phi`` [N, N] host float arrays.
    wf: ``problem`` = dict(field, phi, data, Cf, Cn, M, B) of reference-shaped
    containers (host arrays), solved with ``wf_kwargs``.
    """

    def __init__(self, kind, nside, ncomp, theta_pix, f=None, phi=None, problem=None, n=7, wf_kwargs=None):
        self.id = next(_req_ids)
        self.kind = kind
        self.nside = int(nside)
        self.ncomp = int(ncomp)
        self.theta_pix = float(theta_pix)
        self.f = f
        self.phi = phi
        self.problem = problem
        self.n = n
        self.wf_kwargs = wf_kwargs or {}
        self.t_submit = None
        self.t_done = None
        # lens / delens stages (host clock): admitted by the scheduler, batch launch begun, launch issued
        # (inputs staged, graph replayed), completion seen by the scheduler's poll
        self.t_admit = self.t_launch = self.t_issued = self.t_seen = None
        self.result = None
        self.error = None
        self.done = threading.Event()

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit

    def footprint(self):
        """Device bytes this request holds while in flight (inputs, outputs, planes, workspaces)."""
        N, C = self.nside, self.ncomp
        P = N * N
        if self.kind == "wf":
            return 64 * C * P + 120 * P  # fields, spectra and two lens workspaces in float64/float32
        return 8 * C * P * 2 + 8 * P + 20 * P + 20 * C * P + 48 * P


def _bucket(b):
    s = 1
    while s < b:
        s *= 2
    return s


class _LensSlot:
    """Static buffers, stream and captured graphs for batches of one (N, C, direction)."""

    def __init__(self, dev, nside, ncomp, theta_pix, direction, cap, n, use_graphs, priority=0):
        self.dev = dev
        self.nside, self.ncomp, self.direction, self.cap, self.n = nside, ncomp, direction, cap, n
        self.plan = engine.get_plan(nside, ncomp, theta_pix * ARCMIN, "f32", device=dev)
        N, C = nside, ncomp
        self.h_f = torch.empty((cap, C, N, N), dtype=torch.float32).pin_memory()
        self.h_phi = torch.empty((cap, N, N), dtype=torch.float64).pin_memory()
        self.h_out = torch.empty((cap, C, N, N), dtype=torch.float32).pin_memory()
        self.h_md = torch.empty(cap, dtype=torch.int32).pin_memory()
        self.d_f = torch.empty((cap, C, N, N), dtype=torch.float32, device=dev)
        self.d_phi = torch.empty((cap, N, N), dtype=torch.float64, device=dev)
        self.d_out = torch.empty_like(self.d_f)
        # p = M(t)^-1 grad phi at the 2n+1 stage times, written by the phi precompute itself
        self.pp = torch.empty((cap, 2 * n + 1, 2, N, N), dtype=torch.float32, device=dev)
        self.ws = torch.empty(max(self.plan.workspace_bytes(cap, True), 16), dtype=torch.uint8, device=dev)
        self.phi_ws = torch.empty(max(self.plan.phi_workspace_bytes(cap), 16), dtype=torch.uint8, device=dev)
        self.md = torch.empty(cap, dtype=torch.int32, device=dev)
        self.stream = torch.cuda.Stream(dev, priority=priority)
        self.graphs = {}
        self.use_graphs = use_graphs
        self.busy = False
        self.event = None
        self.reqs = []

    def _body(self, b):
        p, lib = self.plan, self.plan._lib
        st = engine._stream_ptr(self.dev)
        nat.check(lib.lf_min_det_init(engine._ptr(self.md), b, st), "lf_min_det_init")
        nat.check(lib.lf_phi_precompute_pp(p.handle, engine._ptr(self.d_phi), nat.LF_PHI_MAP, b, None,
                                           engine._ptr(self.pp), self.n, engine._ptr(self.md), engine._ptr(self.phi_ws),
                                           self.phi_ws.numel(), st), "lf_phi_precompute_pp")
        nat.check(lib.lf_lense_flow_pp(p.handle, engine._ptr(self.d_f), nat.LF_F32, engine._ptr(self.d_out),
                                       nat.LF_F32, engine._ptr(self.pp), b, self.n, self.direction, 0,
                                       engine._ptr(self.ws), self.ws.numel(), st), "lf_lense_flow_pp")

    def _graph(self, bb):
        """The captured graph for batch bucket ``bb`` (captured on first use, on this slot's stream)."""
        g = self.graphs.get(bb)
        if g is None:
            with torch.cuda.stream(self.stream):
                self._body(bb)  # eager warm-up: kernel attributes are set outside the capture
                # thread-local capture without a device-wide synchronisation: Wiener-filter
                # workers keep running, and capturing, on their own threads
                g = engine.capture_graph(lambda: self._body(bb), stream=self.stream)
            self.graphs[bb] = g
        return g

    def launch(self, reqs):
        """Copy inputs in, run (graph replay or eager) and copy outputs out, all on this slot's stream."""
        b = len(reqs)
        self.reqs = reqs
        self.busy = True
        t0 = time.perf_counter()
        for r in reqs:
            r.t_launch = t0
        for i, r in enumerate(reqs):
            # torch converts float64 -> float32 inside the copy, multi-threaded and without the GIL
            self.h_f[i].copy_(torch.from_numpy(np.ascontiguousarray(r.f)))
            self.h_phi[i].copy_(torch.from_numpy(np.ascontiguousarray(r.phi)))
        with torch.cuda.stream(self.stream):
            self.d_f[:b].copy_(self.h_f[:b], non_blocking=True)
            self.d_phi[:b].copy_(self.h_phi[:b], non_blocking=True)
            bb = _bucket(b) if self.use_graphs else b
            bb = min(bb, self.cap)
            if self.use_graphs:
                self._graph(bb).replay()
            else:
                self._body(b)
            self.h_out[:b].copy_(self.d_out[:b], non_blocking=True)
            self.h_md[:b].copy_(self.md[:b], non_blocking=True)
            self.event = torch.cuda.Event()
            self.event.record(self.stream)
        t1 = time.perf_counter()
        for r in reqs:
            r.t_issued = t1

    def poll(self):
        """Complete the batch's requests if its event has fired; return them."""
        if not self.busy or not self.event.query():
            return []
        lib = self.plan._lib
        now = time.perf_counter()
        timed_out = lib.lf_timeout_status() != nat.LF_OK
        out = self.h_out[:len(self.reqs)].numpy().copy()
        mds = self.h_md[:len(self.reqs)].tolist()
        done = self.reqs
        for i, r in enumerate(done):
            md = lib.lf_decode_min_det(int(mds[i]))
            if timed_out:
                r.error = nat.LenseFlowError(nat.LF_ERR_TIMEOUT, "lens batch")
            elif not md > 0.0:
                r.error = nat.SingularMagnificationError(nat.LF_ERR_SINGULAR_MAGNIFICATION, f"min det {md:.3g}")
            else:
                r.result = out[i]
            r.t_seen = r.t_done = now
            r.done.set()
        self.busy = False
        self.reqs = []
        return done


class Server:
    """Continuous-batching scheduler over the LenseFlow engine on one GPU."""

    def __init__(self, hbm_budget=32 << 30, max_batch=16, use_graphs=True, wf_workers=2, wf_batch=8, device=None,
                 lens_priority=-1, gil_switch_s=5e-4):
        self.dev = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index)
        self.budget = int(hbm_budget)
        self.max_batch = int(max_batch)
        self.use_graphs = use_graphs
        # CUDA stream priority of the lens slots (lower = higher priority; 0 = the Wiener filters' level).
        # Two Wiener-filter workers with the lens slots one level above them measured best for the
        # mixed stream: 41 maps/s, lens p99 ~0.5 s, WF p50 ~4 s, against 33 maps/s, 1.2 s and 5.1 s
        # with four workers at equal priority.
        self.lens_priority = int(lens_priority)
        self.gil_switch_s = gil_switch_s  # interpreter switch interval while serving (None: leave it)
        self.inbox = queue.Queue()
        self.pending = collections.defaultdict(collections.deque)  # group key -> requests
        self.slots = {}  # group key -> list of _LensSlot
        self.in_use = 0
        self.wf_batch = int(wf_batch)
        self.wf_pending = collections.defaultdict(collections.deque)  # (N, C, theta) -> waiting WF requests
        self.wf_cond = threading.Condition()
        self._wf_stop = False
        self.completed = []
        self._stop = threading.Event()
        self._lock = threading.Lock()
        self._thread = threading.Thread(target=self._loop, daemon=True)
        self._wf_threads = [threading.Thread(target=self._wf_loop, daemon=True) for _ in range(wf_workers)]

    # ------------------------------------------------------------ client
    def start(self):
        # The scheduler thread makes a few dozen short GIL-releasing calls per batch (copies, graph replays,
        # event queries) while the Wiener-filter workers keep the interpreter busy; each call must win the
        # GIL back, which under contention takes up to the switch interval.  A shorter interval while the
        # server runs bounds that wait (restored by stop()).
        self._switch = sys.getswitchinterval()
        if self.gil_switch_s is not None:
            sys.setswitchinterval(min(self._switch, self.gil_switch_s))
        self._thread.start()
        for t in self._wf_threads:
            t.start()
        return self

    def submit(self, req):
        req.t_submit = time.perf_counter()
        self.inbox.put(req)
        return req

    def stop(self):
        self._stop.set()
        self._thread.join()
        with self.wf_cond:
            self._wf_stop = True
            self.wf_cond.notify_all()
        for t in self._wf_threads:
            t.join()
        if getattr(self, "_switch", None) is not None:
            sys.setswitchinterval(self._switch)

    def prepare(self, nside, ncomp, theta_pix, kinds=("lens", "delens")):
        """Create the lens slots of one shape and capture the graphs of every batch bucket now, before
        ``start``.  Otherwise the scheduler thread does it the first time a shape or bucket arrives: pinned
        host and device buffers (about 3 GB per slot for 1024^2 QU at max_batch 16) and a capture, during
        which every queued lens batch waits."""
        if self._thread.is_alive():
            raise RuntimeError("Server.prepare must be called before start()")
        torch.cuda.set_device(self.dev)
        for kind in kinds:
            key = (int(nside), int(ncomp), float(theta_pix), nat_direction(kind))
            ss = self.slots.setdefault(key, [])
            while len(ss) < 2:
                N, C, th, direction = key
                ss.append(_LensSlot(self.dev, N, C, th, direction, self.max_batch, 7, self.use_graphs,
                                    self.lens_priority))
            if self.use_graphs:
                for s in ss:
                    bb = 1
                    while True:
                        s._graph(min(bb, s.cap))
                        if bb >= s.cap:
                            break
                        bb *= 2
        torch.cuda.synchronize(self.dev)
        return self

    # ---------------------------------------------------------- internal
    def _release(self, nbytes):
        with self._lock:
            self.in_use -= nbytes

    def _admit(self, nbytes):
        with self._lock:
            if self.in_use + nbytes > self.budget and self.in_use > 0:
                return False
            self.in_use += nbytes
            return True

    def _finish(self, reqs):
        for r in reqs:
            self._release(r.footprint())
        self.completed.extend(reqs)

    def _slot_for(self, key):
        for s in self.slots.setdefault(key, []):
            if not s.busy:
                return s
        if len(self.slots[key]) < 2:  # two slots per shape: one can fill while the other runs
            N, C, th, direction = key
            s = _LensSlot(self.dev, N, C, th, direction, self.max_batch, 7, self.use_graphs, self.lens_priority)
            self.slots[key].append(s)
            return s
        return None

    def _loop(self):
        torch.cuda.set_device(self.dev)
        waiting = collections.deque()  # admitted-later requests in arrival order
        while not self._stop.is_set() or any(self.pending.values()) or any(
                s.busy for ss in self.slots.values() for s in ss):
            # 1. retire finished batches
            for ss in self.slots.values():
                for s in ss:
                    self._finish(s.poll())
            # 2. take arrivals
            try:
                while True:
                    waiting.append(self.inbox.get_nowait())
            except queue.Empty:
                pass
            # 3. admit by footprint, in arrival order
            while waiting and self._admit(waiting[0].footprint()):
                r = waiting.popleft()
                r.t_admit = time.perf_counter()
                if r.kind == "wf":
                    with self.wf_cond:
                        self.wf_pending[(r.nside, r.ncomp, r.theta_pix)].append(r)
                        self.wf_cond.notify()
                else:
                    d = nat_direction(r.kind)
                    self.pending[(r.nside, r.ncomp, r.theta_pix, d)].append(r)
            # 4. launch every group that has work and a free slot
            launched = False
            for key, q in self.pending.items():
                if not q:
                    continue
                s = self._slot_for(key)
                if s is None:
                    continue
                batch = [q.popleft() for _ in range(min(len(q), self.max_batch))]
                try:
                    s.launch(batch)
                except Exception as e:  # surface errors per request, keep serving
                    for r in batch:
                        r.error = e
                        r.t_done = time.perf_counter()
                        r.done.set()
                    s.busy = False
                    self._finish(batch)
                launched = True
            if not launched:
                time.sleep(0.0002)

    def _take_wf_batch(self):
        """Block until Wiener-filter work is waiting; take up to wf_batch requests of the oldest group."""
        with self.wf_cond:
            while True:
                groups = [(q[0].t_submit, k) for k, q in self.wf_pending.items() if q]
                if groups:
                    _, key = min(groups)
                    q = self.wf_pending[key]
                    return [q.popleft() for _ in range(min(len(q), self.wf_batch))]
                if self._wf_stop:
                    return None
                self.wf_cond.wait(0.05)

    def _wf_loop(self):
        torch.cuda.set_device(self.dev)
        stream = torch.cuda.Stream(self.dev)
        while True:
            batch = self._take_wf_batch()
            if batch is None:
                return
            try:
                with torch.cuda.stream(stream):
                    results = _solve_wf_batch(batch)
                    torch.cuda.current_stream().synchronize()
                for r, x in zip(batch, results):
                    r.result = x
            except Exception as e:
                for r in batch:
                    r.error = e
            now = time.perf_counter()
            for r in batch:
                r.t_done = now
                r.done.set()
            self._finish(batch)


def _solve_wf_batch(reqs):
    """Wiener-filter requests of one (N, C, pixel size) solved together by the batched device PCG."""
    from .wf_engine import DeviceWienerFilter
    wf = DeviceWienerFilter(problems=[r.problem for r in reqs], n=reqs[0].n)
    x, its = wf.solve(**reqs[0].wf_kwargs)
    if len(reqs) == 1:
        reqs[0].iterations = its
        return [wf.to_field(x)]
    for r, it in zip(reqs, its):
        r.iterations = it
    return [wf.to_field(x, i) for i in range(len(reqs))]


def _solve_wf(req):
    """One Wiener-filter request by itself."""
    return _solve_wf_batch([req])[0]


def nat_direction(kind):
    return 1 if kind == "lens" else -1


def run_alone(req):
    """The same request executed by itself with plain engine calls (no batching, no graphs)."""
    if req.kind == "wf":
        return _solve_wf(req)
    plan = engine.get_plan(req.nside, req.ncomp, req.theta_pix * ARCMIN, "f32")
    f = torch.as_tensor(np.asarray(req.f, dtype=np.float32), device="cuda").unsqueeze(0)
    phi = torch.as_tensor(np.asarray(req.phi, dtype=np.float64), device="cuda").unsqueeze(0)
    pp = plan.phi_pp(phi, req.n, check_det=True)
    return plan.lense_flow_pp(f, pp, req.n, direction=nat_direction(req.kind))[0].cpu().numpy()


def lens_tail_breakdown(reqs, frac=0.01):
    """For the slowest ``frac`` of the completed lens / delens requests: mean ms spent waiting for admission,
    queued for a slot (admitted -> launch begun), staging and issuing the batch, and on the GPU until the
    scheduler saw the batch complete."""
    done = [r for r in reqs if r.kind in ("lens", "delens") and r.t_seen is not None and r.t_launch is not None]
    if not done:
        return {}
    done.sort(key=lambda r: r.latency)
    tail = done[-max(1, int(round(frac * len(done)))):]
    ms = lambda f: float(np.mean([f(r) for r in tail]) * 1e3)
    return {"n": len(tail), "latency_ms": ms(lambda r: r.latency),
            "admission_ms": ms(lambda r: r.t_admit - r.t_submit),
            "slot_wait_ms": ms(lambda r: r.t_launch - r.t_admit),
            "stage_and_issue_ms": ms(lambda r: r.t_issued - r.t_launch),
            "gpu_until_seen_ms": ms(lambda r: r.t_seen - r.t_issued)}


def latency_summary(reqs):
    lat = np.array([r.latency for r in reqs if r.latency is not None])
    if lat.size == 0:
        return {}
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "n": int(lat.size)}
