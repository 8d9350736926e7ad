"""Device-level LenseFlow API on torch CUDA tensors (batched, stream-aware).

torch only supplies device memory and the current stream; all arithmetic runs
in the CUDA kernels of liblenseflow.so, reached through the C ABI.
"""
from __future__ import annotations

import ctypes
import threading

import torch

from . import _native as nat
from .constants import FORWARD_LENSE, INVERSE_LENSE

_plans = {}
_plans_lock = threading.Lock()


def _stream_ptr(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Plan:
    """A plan for N x N maps with C components in float32 or float64 compute."""

    def __init__(self, nside, ncomp, pix_width, precision="f32", device=None):
        lib = nat.load()
        self.nside = int(nside)
        self.ncomp = int(ncomp)
        self.pix_width = float(pix_width)
        self.precision = precision
        self.prec_code = nat.LF_F64 if precision == "f64" else nat.LF_F32
        self.dtype = torch.float64 if precision == "f64" else torch.float32
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(lib.lf_plan_create(ctypes.byref(h), self.nside, self.ncomp, self.pix_width, self.prec_code),
                      "lf_plan_create")
        self.handle = h
        self._lib = lib

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                self._lib.lf_plan_destroy(self.handle)
        except Exception:
            pass

    # -------------------------------------------------------------- sizes
    def workspace_bytes(self, batch, adjoint, n=None):
        """Lens workspace; with ``n`` RK4 steps, the size that also holds the stage-time p planes."""
        if n is None:
            return int(self._lib.lf_workspace_bytes(self.handle, int(batch), int(bool(adjoint))))
        return int(self._lib.lf_workspace_bytes_n(self.handle, int(batch), int(bool(adjoint)), int(n)))

    def phi_planes_bytes(self, batch):
        return int(self._lib.lf_phi_planes_bytes(self.handle, int(batch)))

    def phi_workspace_bytes(self, batch):
        return int(self._lib.lf_phi_workspace_bytes(self.handle, int(batch)))

    # ------------------------------------------------------------ phi
    def phi_planes(self, phi, check_det=True, out=None, workspace=None):
        """phi: [B,N,N] float64 map or [B,N,N/2+1] complex128 Fourier (rfft2 layout), on this device.

        Returns the [B,5,N,N] derivative planes in the plan's precision.  With
        ``check_det`` the minimum over pixels and t in [0,1] of
        det(I + t grad grad phi) is read back and a SingularMagnificationError
        raised if it is not positive (one device sync).
        """
        N = self.nside
        if phi.dim() == 2:
            phi = phi.unsqueeze(0)
        if phi.shape[-2:] == (N, N):
            basis = nat.LF_PHI_MAP
            phi = phi.to(device=self.device, dtype=torch.float64).contiguous()
        elif phi.shape[-2:] == (N, N // 2 + 1):
            basis = nat.LF_PHI_FOURIER
            phi = phi.to(device=self.device, dtype=torch.complex128).contiguous()
        else:
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, f"phi shape {tuple(phi.shape)} for N={N}")
        B = phi.shape[0]
        planes = out if out is not None else torch.empty((B, 5, N, N), dtype=self.dtype, device=self.device)
        if planes.shape != (B, 5, N, N) or planes.dtype != self.dtype or not planes.is_contiguous():
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "phi plane buffer does not match")
        ws = workspace
        if ws is None or ws.numel() < self.phi_workspace_bytes(B):
            ws = torch.empty(max(self.phi_workspace_bytes(B), 16), dtype=torch.uint8, device=self.device)
        md = torch.empty(max(B, 1), dtype=torch.int32, device=self.device) if check_det else None
        with torch.cuda.device(self.device):
            st = _stream_ptr(self.device)
            if md is not None:
                nat.check(self._lib.lf_min_det_init(_ptr(md), B, st), "lf_min_det_init")
            nat.check(self._lib.lf_phi_precompute(self.handle, _ptr(phi), basis, B, _ptr(planes),
                                                  _ptr(md) if md is not None else None, _ptr(ws), ws.numel(), st),
                      "lf_phi_precompute")
        if md is not None:
            vals = [self._lib.lf_decode_min_det(int(v)) for v in md.cpu().tolist()[:B]]
            check_timeouts("lf_phi_precompute")
            self.last_min_det = vals
            if not all(v > 0.0 for v in vals):
                raise nat.SingularMagnificationError(nat.LF_ERR_SINGULAR_MAGNIFICATION,
                                                     f"min det(I + t grad grad phi) = {min(vals):.3g}")
        return planes

    def pp_bytes(self, batch, n):
        """Bytes of the stage-time p planes of ``batch`` maps for ``n`` RK4 steps (float32 plans)."""
        return int(self._lib.lf_pp_bytes(self.handle, int(batch), int(n)))

    def phi_pp(self, phi, n, check_det=True, out=None, planes_out=None, workspace=None, min_det=None):
        """p = M(t)^-1 grad(phi) at the 2n+1 times k/(2n) for [B,N,N] map / [B,N,N/2+1] Fourier phi
        (lf_phi_precompute_pp; float32 plans): a [B, 2n+1, 2, N, N] float32 tensor, formed in float64 in the
        derivative row pass.  ``planes_out`` optionally receives the five derivative planes.  With
        ``check_det`` the magnification minimum is read back as in ``phi_planes``; a caller-owned int32
        ``min_det`` buffer (initialised with lf_min_det_init) is filled without a readback instead."""
        if self.prec_code != nat.LF_F32:
            raise nat.LenseFlowError(nat.LF_ERR_BAD_DTYPE, "p planes need a float32 plan")
        N = self.nside
        if phi.dim() == 2:
            phi = phi.unsqueeze(0)
        if phi.shape[-2:] == (N, N):
            basis = nat.LF_PHI_MAP
            phi = phi.to(device=self.device, dtype=torch.float64).contiguous()
        elif phi.shape[-2:] == (N, N // 2 + 1):
            basis = nat.LF_PHI_FOURIER
            phi = phi.to(device=self.device, dtype=torch.complex128).contiguous()
        else:
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, f"phi shape {tuple(phi.shape)} for N={N}")
        B, K = phi.shape[0], 2 * int(n) + 1
        pp = out if out is not None else torch.empty((B, K, 2, N, N), dtype=torch.float32, device=self.device)
        if pp.shape != (B, K, 2, N, N) or pp.dtype != torch.float32 or not pp.is_contiguous():
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "p-plane buffer does not match")
        if planes_out is not None and (planes_out.shape != (B, 5, N, N) or planes_out.dtype != torch.float32):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "derivative plane buffer does not match")
        ws = workspace
        if ws is None or ws.numel() < self.phi_workspace_bytes(B):
            ws = torch.empty(max(self.phi_workspace_bytes(B), 16), dtype=torch.uint8, device=self.device)
        md = min_det
        if md is None and check_det:
            md = torch.empty(max(B, 1), dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            st = _stream_ptr(self.device)
            if md is not None and min_det is None:
                nat.check(self._lib.lf_min_det_init(_ptr(md), B, st), "lf_min_det_init")
            nat.check(self._lib.lf_phi_precompute_pp(self.handle, _ptr(phi), basis, B,
                                                     _ptr(planes_out) if planes_out is not None else None, _ptr(pp),
                                                     int(n), _ptr(md) if md is not None else None, _ptr(ws),
                                                     ws.numel(), st), "lf_phi_precompute_pp")
        if md is not None and min_det is None:
            vals = [self._lib.lf_decode_min_det(int(v)) for v in md.cpu().tolist()[:B]]
            check_timeouts("lf_phi_precompute_pp")
            self.last_min_det = vals
            if not all(v > 0.0 for v in vals):
                raise nat.SingularMagnificationError(nat.LF_ERR_SINGULAR_MAGNIFICATION,
                                                     f"min det(I + t grad grad phi) = {min(vals):.3g}")
        return pp

    def lense_flow_pp(self, f, pp, n, direction=FORWARD_LENSE, adjoint=False, out=None, workspace=None,
                      out_dtype=None):
        """LenseFlow with precomputed p planes (from ``phi_pp`` with the same n): lf_lense_flow_pp."""
        N, C = self.nside, self.ncomp
        if f.dim() != 4 or f.shape[1:] != (C, N, N):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, f"field shape {tuple(f.shape)} for C={C}, N={N}")
        if f.dtype not in (torch.float32, torch.float64):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_DTYPE, str(f.dtype))
        f = f.contiguous()
        B = f.shape[0]
        if pp.shape != (B, 2 * int(n) + 1, 2, N, N) or pp.dtype != torch.float32 or not pp.is_contiguous():
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "p planes do not match the field batch / n")
        odt = f.dtype if out_dtype is None else out_dtype
        if out is None:
            out = torch.empty((B, C, N, N), dtype=odt, device=self.device)
        if workspace is None or workspace.numel() < self.workspace_bytes(B, adjoint):
            workspace = torch.empty(max(self.workspace_bytes(B, adjoint), 16), dtype=torch.uint8, device=self.device)
        code = lambda t: nat.LF_F64 if t == torch.float64 else nat.LF_F32
        with torch.cuda.device(self.device):
            nat.check(self._lib.lf_lense_flow_pp(self.handle, _ptr(f), code(f.dtype), _ptr(out), code(out.dtype),
                                                 _ptr(pp), B, int(n), int(direction), int(bool(adjoint)),
                                                 _ptr(workspace), workspace.numel(), _stream_ptr(self.device)),
                      "lf_lense_flow_pp")
        return out

    # ------------------------------------------------------------ lens
    def lense_flow(self, f, planes, n=10, direction=FORWARD_LENSE, adjoint=False, out=None, workspace=None,
                   out_dtype=None):
        """f: [B,C,N,N] float32/float64 map-space fields on this device (C = plan's ncomp)."""
        N, C = self.nside, self.ncomp
        if f.dim() != 4 or f.shape[1:] != (C, N, N):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, f"field shape {tuple(f.shape)} for C={C}, N={N}")
        if f.dtype not in (torch.float32, torch.float64):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_DTYPE, str(f.dtype))
        f = f.contiguous()
        B = f.shape[0]
        if planes.shape != (B, 5, N, N) or planes.dtype != self.dtype or not planes.is_contiguous():
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "phi planes do not match the field batch / plan")
        odt = f.dtype if out_dtype is None else out_dtype
        if out is None:
            out = torch.empty((B, C, N, N), dtype=odt, device=self.device)
        # a caller's workspace of at least the minimum is used as given (the
        # engine reads the p planes only when it also has room for them)
        if workspace is None or workspace.numel() < self.workspace_bytes(B, adjoint):
            workspace = torch.empty(max(self.workspace_bytes(B, adjoint, n), 16), dtype=torch.uint8,
                                    device=self.device)
        code = lambda t: nat.LF_F64 if t == torch.float64 else nat.LF_F32
        with torch.cuda.device(self.device):
            nat.check(self._lib.lf_lense_flow(self.handle, _ptr(f), code(f.dtype), _ptr(out), code(out.dtype),
                                              _ptr(planes), B, int(n), int(direction), int(bool(adjoint)),
                                              _ptr(workspace), workspace.numel(), _stream_ptr(self.device)),
                      "lf_lense_flow")
        return out


    # ------------------------------------------------------------ FFTs
    def rfft2(self, maps):
        """float64 rfft2 of [B,N,N] float32/float64 maps -> [B,N,N/2+1] complex128 (jnp.fft.rfft2)."""
        N = self.nside
        maps = maps.contiguous()
        if maps.dim() == 2:
            maps = maps.unsqueeze(0)
        if maps.shape[-2:] != (N, N) or maps.dtype not in (torch.float32, torch.float64):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, f"maps {tuple(maps.shape)} {maps.dtype}")
        B = maps.shape[0]
        spec = torch.empty((B, N, N // 2 + 1), dtype=torch.complex128, device=self.device)
        code = nat.LF_F64 if maps.dtype == torch.float64 else nat.LF_F32
        with torch.cuda.device(self.device):
            nat.check(self._lib.lf_rfft2(self.handle, _ptr(maps), code, B, _ptr(spec), _stream_ptr(self.device)),
                      "lf_rfft2")
        return spec

    def irfft2(self, spec, out_dtype=torch.float64):
        """float64 irfft2 of [B,N,N/2+1] complex128 -> [B,N,N] maps (jnp.fft.irfft2 semantics)."""
        N = self.nside
        spec = spec.to(torch.complex128).contiguous()
        if spec.dim() == 2:
            spec = spec.unsqueeze(0)
        if spec.shape[-2:] != (N, N // 2 + 1):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, f"spectrum {tuple(spec.shape)}")
        B = spec.shape[0]
        maps = torch.empty((B, N, N), dtype=out_dtype, device=self.device)
        ws = torch.empty(max(int(self._lib.lf_fft_workspace_bytes(self.handle, B)), 16), dtype=torch.uint8,
                         device=self.device)
        code = nat.LF_F64 if out_dtype == torch.float64 else nat.LF_F32
        with torch.cuda.device(self.device):
            nat.check(self._lib.lf_irfft2(self.handle, _ptr(spec), B, _ptr(maps), code, _ptr(ws), ws.numel(),
                                          _stream_ptr(self.device)), "lf_irfft2")
        return maps

    # ------------------------------------------------------------ VJP
    def lense_flow_vjp(self, f_lensed, cotangent, planes, n=10, direction=FORWARD_LENSE, phi_basis="fourier",
                       return_f=False):
        """The reference's reverse pass (lense_flow.py:23-126) for [B,C,N,N] fields.

        Returns (delta_f, delta_phi[, f_back]) with delta_f before undo_inner_product and
        delta_phi [B,N,N/2+1] complex128 (phi_basis "fourier") or [B,N,N] float64 ("map").
        """
        N, C = self.nside, self.ncomp
        if f_lensed.shape != cotangent.shape or f_lensed.dim() != 4 or f_lensed.shape[1:] != (C, N, N):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "field/cotangent shapes")
        dt = torch.float64 if torch.float64 in (f_lensed.dtype, cotangent.dtype) else torch.float32
        fl = f_lensed.to(dt).contiguous()
        ct = cotangent.to(dt).contiguous()
        B = fl.shape[0]
        if planes.shape != (B, 5, N, N) or planes.dtype != self.dtype:
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "phi planes do not match")
        df = torch.empty_like(fl)
        fb = torch.empty_like(fl) if return_f else None
        fourier = phi_basis == "fourier"
        dphi = (torch.empty((B, N, N // 2 + 1), dtype=torch.complex128, device=self.device) if fourier
                else torch.empty((B, N, N), dtype=torch.float64, device=self.device))
        ws = torch.empty(max(int(self._lib.lf_vjp_workspace_bytes(self.handle, B)), 16), dtype=torch.uint8,
                         device=self.device)
        code = nat.LF_F64 if dt == torch.float64 else nat.LF_F32
        with torch.cuda.device(self.device):
            nat.check(self._lib.lf_lense_flow_vjp(self.handle, _ptr(fl), _ptr(ct), code, _ptr(planes), B, int(n),
                                                  int(direction), _ptr(df), _ptr(fb) if fb is not None else None,
                                                  _ptr(dphi), nat.LF_PHI_FOURIER if fourier else nat.LF_PHI_MAP,
                                                  _ptr(ws), ws.numel(), _stream_ptr(self.device)),
                      "lf_lense_flow_vjp")
        return (df, dphi, fb) if return_f else (df, dphi)

    def lense_flow_vjp_ckpt(self, f, cotangent, planes, n=10, direction=FORWARD_LENSE, phi_basis="fourier",
                            return_lensed=False):
        """Checkpointed exact reverse pass (lf_lense_flow_vjp_ckpt) from the UNLENSED fields f [B,C,N,N].

        The forward integration keeps one field per RK4 step; each step is
        recomputed from it on the way back, so delta_phi is the exact gradient
        of the discrete lens (the reference scheme of ``lense_flow_vjp``
        carries the RK4 discretisation error).  Returns (delta_f, delta_phi[,
        lensed]) in the conventions of ``lense_flow_vjp``.
        """
        N, C = self.nside, self.ncomp
        if f.shape != cotangent.shape or f.dim() != 4 or f.shape[1:] != (C, N, N):
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "field/cotangent shapes")
        dt = torch.float64 if torch.float64 in (f.dtype, cotangent.dtype) else torch.float32
        fi = f.to(dt).contiguous()
        ct = cotangent.to(dt).contiguous()
        B = fi.shape[0]
        if planes.shape != (B, 5, N, N) or planes.dtype != self.dtype:
            raise nat.LenseFlowError(nat.LF_ERR_BAD_SHAPE, "phi planes do not match")
        df = torch.empty_like(fi)
        lensed = torch.empty_like(fi) if return_lensed else None
        fourier = phi_basis == "fourier"
        dphi = (torch.empty((B, N, N // 2 + 1), dtype=torch.complex128, device=self.device) if fourier
                else torch.empty((B, N, N), dtype=torch.float64, device=self.device))
        ws = torch.empty(max(int(self._lib.lf_vjp_ckpt_workspace_bytes(self.handle, B, int(n))), 16),
                         dtype=torch.uint8, device=self.device)
        code = nat.LF_F64 if dt == torch.float64 else nat.LF_F32
        with torch.cuda.device(self.device):
            nat.check(self._lib.lf_lense_flow_vjp_ckpt(self.handle, _ptr(fi), _ptr(ct), code, _ptr(planes), B, int(n),
                                                       int(direction), _ptr(lensed) if lensed is not None else None,
                                                       _ptr(df), _ptr(dphi),
                                                       nat.LF_PHI_FOURIER if fourier else nat.LF_PHI_MAP, _ptr(ws),
                                                       ws.numel(), _stream_ptr(self.device)),
                      "lf_lense_flow_vjp_ckpt")
        return (df, dphi, lensed) if return_lensed else (df, dphi)

    # ---------------------------------------------------------- profiling
    def profile(self, enable=True):
        nat.check(self._lib.lf_profile_enable(self.handle, int(bool(enable))), "lf_profile_enable")

    def profile_reset(self):
        nat.check(self._lib.lf_profile_reset(self.handle), "lf_profile_reset")

    def profile_read(self, kind):
        """(total milliseconds, launch count) of the recorded launches of one kernel kind."""
        ms = ctypes.c_double()
        n = ctypes.c_int()
        nat.check(self._lib.lf_profile_read(self.handle, int(kind), ctypes.byref(ms), ctypes.byref(n)),
                  "lf_profile_read")
        return ms.value, n.value


def chunk_schedule(batch, chunks=8, chunk_sizes=None):
    """Chunk sizes of a HostPipeline call: ``chunk_sizes`` as given (positive, summing to ``batch``), else
    ``chunks`` near-equal chunks (the last may be shorter)."""
    if chunk_sizes is None:
        k = max(1, min(int(chunks), batch))
        step = max(1, -(-batch // k))
        chunk_sizes = [min(step, batch - lo) for lo in range(0, batch, step)]
    chunk_sizes = [int(c) for c in chunk_sizes]
    if any(c <= 0 for c in chunk_sizes) or sum(chunk_sizes) != batch:
        raise ValueError(f"chunk sizes {chunk_sizes} must be positive and sum to the batch {batch}")
    return chunk_sizes


class HostPipeline:
    """The reference-facing call with host buffers, for a fixed batch, pipelined.

    Each call copies f [B,C,N,N] and phi [B,N,N] (pinned host memory) to the
    device, computes the phi derivative planes (with the magnification check),
    lenses, and copies the result back into a pinned host buffer.  The batch
    is split into ``chunks`` that move through ``slots`` sets of device
    buffers: host-to-device copies on one stream, compute alternating between
    ``compute_streams`` streams, device-to-host copies on another.  A chunk's
    lens is a few dozen short launches; with two compute streams the kernels
    of neighbouring chunks fill each other's tail waves and launch gaps, so
    smaller chunks (better copy overlap) stop costing compute throughput.
    With ``use_graphs`` each chunk's phi precompute + lens (about 60 launches)
    is captured into a CUDA graph at the second call of a given shape (the
    first runs eagerly, which also sets the kernels' shared-memory limits) and
    replayed from then on (captured without a device-wide synchronisation).  For 64
    512^2 QU maps with float64 host I/O: 4,528 maps/s on one stream, 5,600
    with two compute streams, 6,411 with graphs, 7,240 with consecutive calls
    queued (``wait=False``) so that each call's fill and drain overlap its
    neighbours (same outputs bit for bit).  With calls queued, the neighbours
    also hide a larger chunk's longer fill, and 8 chunks of 8 maps (the
    default) beat 16 chunks of 4 (per-map compute is cheaper at 8 maps):
    7,818-7,940 against 7,415-7,424 maps/s in two sweeps on one box (4
    chunks 7,770-7,844, 32 chunks 6,133-6,136).
    The magnification minima are read back after the last chunk; a call
    whose phi is singular raises SingularMagnificationError (its outputs are
    then meaningless).  ``wait=False`` returns once the call is queued: the
    next call's first copies then overlap this call's last chunks (each
    slot's reuse waits for the events of its previous use), and ``wait()``
    joins the pipeline into the current stream, reads the pending minima and
    raises for a singular phi.  The minima of the two most recent calls are
    kept in a ring, so a third call first waits for the oldest.  Device
    buffers are allocated once (the lens workspace at the first call, when n
    is known).
    """

    def __init__(self, plan, batch, io_dtype=torch.float64, chunks=8, compute_streams=2, slots=4,
                 use_graphs=True, chunk_sizes=None):
        self.plan = plan
        N, C = plan.nside, plan.ncomp
        dev = plan.device
        self.batch = batch
        chunk_sizes = chunk_schedule(batch, chunks, chunk_sizes)
        self.sizes = chunk_sizes
        self.offsets = [sum(chunk_sizes[:i]) for i in range(len(chunk_sizes))]
        self.chunks = len(chunk_sizes)
        self.cb = max(chunk_sizes, default=1)  # device buffers hold the largest chunk
        cb = self.cb
        self.io_dtype = io_dtype
        self.nslots = max(2, int(slots))
        ns = self.nslots
        self.d_f = [torch.empty((cb, C, N, N), dtype=io_dtype, device=dev) for _ in range(ns)]
        self.d_out = [torch.empty((cb, C, N, N), dtype=io_dtype, device=dev) for _ in range(ns)]
        self.d_phi = [torch.empty((cb, N, N), dtype=torch.float64, device=dev) for _ in range(ns)]
        # float32 plans: the phi precompute writes the stage-time p planes directly (lf_phi_precompute_pp), one
        # set per slot and step count, kept while graphs that use them may replay; float64: derivative planes
        self.use_pp = plan.prec_code == nat.LF_F32
        self.pp = {}  # n -> per-slot p-plane buffers
        self.planes = [] if self.use_pp else [torch.empty((cb, 5, N, N), dtype=plan.dtype, device=dev)
                                              for _ in range(ns)]
        self.ws = [torch.empty(max(plan.workspace_bytes(cb, True), 16), dtype=torch.uint8, device=dev)
                   for _ in range(ns)]
        self.phi_ws = [torch.empty(max(plan.phi_workspace_bytes(cb), 16), dtype=torch.uint8, device=dev)
                       for _ in range(ns)]
        # magnification minima of the two most recent calls
        self.min_det = [torch.empty(max(batch, 1), dtype=torch.int32, device=dev) for _ in range(2)]
        self._ring = 0
        self._pending = {}  # ring index -> events that end the call's compute
        # per slot: the last compute that read its inputs, the last copy-out of its output
        self._slot_in_free = [None] * ns
        self._slot_out_free = [None] * ns
        self.s_in = torch.cuda.Stream(dev)
        self.s_cmp = [torch.cuda.Stream(dev) for _ in range(max(1, int(compute_streams)))]
        self.s_out = torch.cuda.Stream(dev)
        # per chunk and call shape: the captured phi precompute + lens (replayed from the third call on)
        self.use_graphs = bool(use_graphs)
        self.graphs = {}
        self._warm = set()

    def _compute(self, slot, lo, m, n, direction, adjoint, check_det, ring):
        plan, lib = self.plan, self.plan._lib
        st = _stream_ptr(plan.device)
        md = _ptr(self.min_det[ring][lo:]) if check_det else None
        code = nat.LF_F64 if self.io_dtype == torch.float64 else nat.LF_F32
        if self.use_pp:
            pp = self.pp[n][slot]
            nat.check(lib.lf_phi_precompute_pp(plan.handle, _ptr(self.d_phi[slot]), nat.LF_PHI_MAP, m, None, _ptr(pp),
                                               int(n), md, _ptr(self.phi_ws[slot]), self.phi_ws[slot].numel(), st),
                      "lf_phi_precompute_pp")
            nat.check(lib.lf_lense_flow_pp(plan.handle, _ptr(self.d_f[slot]), code, _ptr(self.d_out[slot]), code,
                                           _ptr(pp), m, int(n), int(direction), int(bool(adjoint)),
                                           _ptr(self.ws[slot]), self.ws[slot].numel(), st), "lf_lense_flow_pp")
            return
        nat.check(lib.lf_phi_precompute(plan.handle, _ptr(self.d_phi[slot]), nat.LF_PHI_MAP, m,
                                        _ptr(self.planes[slot]), md, _ptr(self.phi_ws[slot]),
                                        self.phi_ws[slot].numel(), st), "lf_phi_precompute")
        nat.check(lib.lf_lense_flow(plan.handle, _ptr(self.d_f[slot]), code, _ptr(self.d_out[slot]), code,
                                    _ptr(self.planes[slot]), m, int(n), int(direction), int(bool(adjoint)),
                                    _ptr(self.ws[slot]), self.ws[slot].numel(), st), "lf_lense_flow")

    def h2d_bytes(self):
        N, C = self.plan.nside, self.plan.ncomp
        return self.batch * (C * N * N * torch.tensor([], dtype=self.io_dtype).element_size() + N * N * 8)

    def d2h_bytes(self):
        N, C = self.plan.nside, self.plan.ncomp
        return self.batch * C * N * N * torch.tensor([], dtype=self.io_dtype).element_size()

    def _check(self, ring):
        """Read the minima of a finished call (synchronises on its compute) and raise if singular."""
        events = self._pending.pop(ring)
        for ev in events:
            ev.synchronize()
        check_timeouts("HostPipeline")
        lib = self.plan._lib
        vals = [lib.lf_decode_min_det(int(v)) for v in self.min_det[ring][:self.batch].cpu().tolist()]
        self.plan.last_min_det = vals
        if not all(v > 0.0 for v in vals):
            raise nat.SingularMagnificationError(nat.LF_ERR_SINGULAR_MAGNIFICATION,
                                                 f"min det(I + t grad grad phi) = {min(vals):.3g}")

    def wait(self):
        """Join the queued calls into the current stream; raise for a singular phi among them."""
        cur = torch.cuda.current_stream(self.plan.device)
        for st in [self.s_in, self.s_out] + self.s_cmp:
            cur.wait_stream(st)
        if not self._pending:  # calls without the magnification check: wait for the compute here
            for st in self.s_cmp:
                st.synchronize()
            check_timeouts("HostPipeline")
        err = None
        for ring in sorted(self._pending):
            try:
                self._check(ring)
            except nat.SingularMagnificationError as e:
                err = err or e
        if err is not None:
            raise err

    def __call__(self, f_host, phi_host, out_host, n=10, direction=FORWARD_LENSE, adjoint=False, check_det=True,
                 wait=True):
        plan, lib = self.plan, self.plan._lib
        if self.use_pp and n not in self.pp:
            N = plan.nside
            self.pp[n] = [torch.empty((self.cb, 2 * int(n) + 1, 2, N, N), dtype=torch.float32, device=plan.device)
                          for _ in range(self.nslots)]
        cur = torch.cuda.current_stream(plan.device)
        streams = [self.s_in, self.s_out] + self.s_cmp
        for st in streams:
            st.wait_stream(cur)
        ring = self._ring
        self._ring = 1 - ring
        if ring in self._pending:  # the call two back is still unread
            self._check(ring)
        first = self.s_cmp[0]
        if check_det:
            with torch.cuda.stream(first):
                nat.check(lib.lf_min_det_init(_ptr(self.min_det[ring]), self.min_det[ring].numel(),
                                              _stream_ptr(plan.device)), "lf_min_det_init")
            for st in self.s_cmp[1:]:
                st.wait_stream(first)
        ns = self.nslots
        for i in range(self.chunks):
            lo, m = self.offsets[i], self.sizes[i]
            hi = lo + m
            slot = i % ns
            ev_in, ev_cmp, ev_out = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
            with torch.cuda.stream(self.s_in):
                if self._slot_in_free[slot] is not None:
                    self.s_in.wait_event(self._slot_in_free[slot])  # the slot's previous chunk has been consumed
                self.d_f[slot][:m].copy_(f_host[lo:hi], non_blocking=True)
                self.d_phi[slot][:m].copy_(phi_host[lo:hi], non_blocking=True)
                ev_in.record(self.s_in)
            sc = self.s_cmp[i % len(self.s_cmp)]
            with torch.cuda.stream(sc):
                sc.wait_event(ev_in)
                if self._slot_out_free[slot] is not None:
                    sc.wait_event(self._slot_out_free[slot])  # the slot's previous output has been copied out
                args = (slot, lo, m, n, direction, adjoint, check_det, ring)
                key = (i,) + args[2:]
                g = self.graphs.get(key) if self.use_graphs else None
                if g is None and self.use_graphs and key in self._warm:
                    # thread-local capture on the compute stream: the copy streams keep running meanwhile
                    g = capture_graph(lambda: self._compute(*args), stream=sc)
                    self.graphs[key] = g
                if g is not None:
                    g.replay()
                else:
                    self._compute(*args)  # eager; also sets kernel attributes before any capture
                    self._warm.add(key)
                ev_cmp.record(sc)
            self._slot_in_free[slot] = ev_cmp
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(ev_cmp)
                out_host[lo:hi].copy_(self.d_out[slot][:m], non_blocking=True)
                ev_out.record(self.s_out)
            self._slot_out_free[slot] = ev_out
        if check_det:
            ends = []
            for st in self.s_cmp:
                ev = torch.cuda.Event()
                ev.record(st)
                ends.append(ev)
            self._pending[ring] = ends
        if wait:
            self.wait()
        return out_host


class LenseFlowFunction(torch.autograd.Function):
    """torch autograd for y = L(phi) f on device tensors.

    f: [B,C,N,N]; phi: [B,N,N] real map or [B,N,N/2+1] complex Fourier.
    ``scheme="reference"``: the reference's backward pass (lense_flow.py:
    23-126): the f-cotangent is the exact adjoint lens of the incoming
    gradient, the phi-cotangent the continuous adjoint integrated with RK4 (it
    matches the exact discrete gradient to the RK4 discretisation error).
    ``scheme="exact"``: the checkpointed reverse pass (lf_lense_flow_vjp_ckpt):
    same f-cotangent, and the exact gradient of the discrete lens for phi.
    For a complex Fourier phi the gradient follows torch's convention
    dL/dRe + i dL/dIm, i.e. the reference's delta-phi times w/N^2 (w = 1 on
    the DC/Nyquist columns, 2 elsewhere).
    """

    @staticmethod
    def forward(ctx, f, phi, pix_width, n, direction, precision, scheme="reference"):
        if scheme not in ("reference", "exact"):
            raise ValueError(f"unknown reverse-pass scheme {scheme!r}")
        plan = get_plan(f.shape[-1], f.shape[1], pix_width, precision, device=f.device)
        planes = plan.phi_planes(phi.detach(), check_det=False)
        out = plan.lense_flow(f.detach(), planes, n=n, direction=direction)
        ctx.save_for_backward(f.detach() if scheme == "exact" else out, planes)
        ctx.plan, ctx.n, ctx.direction, ctx.scheme = plan, n, direction, scheme
        ctx.fourier = phi.is_complex()
        ctx.phi_dtype, ctx.f_dtype = phi.dtype, f.dtype
        return out

    @staticmethod
    def backward(ctx, g):
        saved, planes = ctx.saved_tensors
        plan = ctx.plan
        basis = "fourier" if ctx.fourier else "map"
        if ctx.scheme == "exact":
            df, dphi = plan.lense_flow_vjp_ckpt(saved, g.contiguous(), planes, n=ctx.n, direction=ctx.direction,
                                                phi_basis=basis)
        else:
            df, dphi = plan.lense_flow_vjp(saved, g.contiguous(), planes, n=ctx.n, direction=ctx.direction,
                                           phi_basis=basis)
        if ctx.fourier:
            N = plan.nside
            w = torch.full((N // 2 + 1,), 2.0, dtype=torch.float64, device=dphi.device)
            w[0] = 1.0
            w[-1] = 1.0
            dphi = dphi * (w / (N * N))
        return df.to(ctx.f_dtype), dphi.to(ctx.phi_dtype), None, None, None, None, None


def lense_flow_ad(f, phi, pix_width, n=10, direction=FORWARD_LENSE, precision="f32", scheme="reference"):
    """Differentiable LenseFlow (torch autograd) on device tensors; ``scheme`` selects the reverse pass."""
    return LenseFlowFunction.apply(f, phi, pix_width, n, direction, precision, scheme)


def capture_graph(fn, stream=None):
    """Capture the launches of ``fn()`` into a CUDA graph on ``stream`` without synchronising the device.

    ``torch.cuda.graph`` synchronises the whole device and empties the
    allocator's cache before it begins; while another host thread is
    capturing, that synchronisation is an illegal operation on the capturing
    stream and invalidates its capture.  Here the capture begins on the
    given (non-default) stream directly, in thread-local mode, so threads
    that capture concurrently -- a server's lens slots and its Wiener-filter
    workers -- leave one another alone.  With ``stream`` None the current
    stream is used unless it is the default stream, in which case a side
    stream is.  Replay the returned graph on any stream."""
    dev = torch.cuda.current_device()
    if stream is None:
        cur = torch.cuda.current_stream(dev)
        stream = cur if cur != torch.cuda.default_stream(dev) else torch.cuda.Stream(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        g.capture_begin(capture_error_mode="thread_local")
        try:
            fn()
        finally:
            g.capture_end()
    return g


def wait_timeouts(reset=False):
    """1 if a kernel block gave up waiting for its bulk copies since the last reset (its results are invalid).

    Synchronises the device; ``reset`` clears the record, after which the entry points compute again."""
    count = ctypes.c_int(0)
    nat.check(nat.load().lf_wait_timeouts(ctypes.byref(count), int(bool(reset))), "lf_wait_timeouts")
    return count.value


def check_timeouts(what="LenseFlow"):
    """Raise LenseFlowError(LF_ERR_TIMEOUT) if a kernel block has recorded a timed-out wait.

    No synchronisation: call it after the work in question has been waited for
    (the synchronising paths -- HostPipeline.wait, the server's batch
    completion, the Wiener filter's convergence checks -- do)."""
    nat.check(nat.load().lf_timeout_status(), what)


def get_plan(nside, ncomp, pix_width, precision="f32", device=None):
    dev = torch.cuda.current_device() if device is None else torch.device(device).index
    key = (dev, int(nside), int(ncomp), float(pix_width), precision)
    with _plans_lock:
        p = _plans.get(key)
        if p is None:
            p = Plan(nside, ncomp, pix_width, precision, device=torch.device("cuda", dev))
            _plans[key] = p
        return p


_planes_cache = {}
_PLANES_CACHE_SIZE = 8


def cached_phi_planes(plan, phi, check_det=True):
    """Derivative planes of ``phi`` for ``plan``, reused while the same phi tensor is unmodified.

    The key is the tensor's storage pointer, shape, dtype and in-place version
    counter, so repeated lensing by one phi (CG iterations, gradients) skips
    the float64 precompute and the magnification-check readback.  The cache
    holds a reference to the tensor, so its storage (and address) cannot be
    reused by another tensor while the entry lives.
    """
    key = (id(plan), phi.data_ptr(), tuple(phi.shape), phi.dtype, phi._version)
    hit = _planes_cache.get(key)
    if hit is not None:
        return hit[1]
    planes = plan.phi_planes(phi, check_det=check_det)
    if len(_planes_cache) >= _PLANES_CACHE_SIZE:
        _planes_cache.pop(next(iter(_planes_cache)))
    _planes_cache[key] = (phi, planes)
    return planes


def lense_flow_batch(f, phi, pix_width, n=10, direction=FORWARD_LENSE, adjoint=False, precision="f32",
                     check_det=True):
    """Batched LenseFlow on device tensors: f [B,C,N,N], phi [B,N,N] map or [B,N,N/2+1] Fourier."""
    if f.dim() == 3:
        f = f.unsqueeze(0)
    plan = get_plan(f.shape[-1], f.shape[1], pix_width, precision, device=f.device)
    planes = cached_phi_planes(plan, phi, check_det=check_det)
    return plan.lense_flow(f, planes, n=n, direction=direction, adjoint=adjoint)


def lense_flow_dlpack(f, phi, pix_width, n=10, direction=FORWARD_LENSE, adjoint=False, precision="f32"):
    """Zero-copy LenseFlow on arrays of any DLPack producer (CuPy, JAX, numba, torch ...).

    ``f`` [B,C,N,N] and ``phi`` [B,N,N] (map) or [B,N,N/2+1] (Fourier) are
    imported with ``torch.from_dlpack`` -- device arrays are used in place --
    lensed on the engine, and the result is returned as a torch tensor, which
    is itself a DLPack producer (``jax.dlpack.from_dlpack(out)``,
    ``cupy.from_dlpack(out)``).  Host arrays are copied to the current device
    first."""
    ft = torch.from_dlpack(f)
    pt = torch.from_dlpack(phi)
    dev = ft.device if ft.is_cuda else torch.device("cuda", torch.cuda.current_device())
    ft = ft.to(dev)
    pt = pt.to(dev)
    if ft.dtype not in (torch.float32, torch.float64):
        ft = ft.to(torch.float64)
    return lense_flow_batch(ft, pt, pix_width, n=n, direction=direction, adjoint=adjoint, precision=precision)


__all__ = ["Plan", "HostPipeline", "LenseFlowFunction", "get_plan", "lense_flow_ad", "lense_flow_batch",
           "lense_flow_dlpack", "FORWARD_LENSE", "INVERSE_LENSE"]
