"""CPU float64 oracle for the LenseFlow path (TEST INFRASTRUCTURE ONLY).

This module is a numpy restatement of the reference's LenseFlow algorithm and
of the inference functions that call it.  It exists to check the CUDA engine:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The product path
(``cmblensing_b200``) never imports, calls or falls back to it.

Parity pin: the oracle reproduces the reference's Julia-generated golden
vectors (``tests/ground_truth_data`` of zaneblood1/CMBLensing.py, 256x256,
2.5 arcmin pixels, RK4 with 7 steps) to ~1e-12 relative L2; the committed
fixtures under ``tests/golden/`` and ``tests/test_oracle_golden.py`` check it.

Conventions restated from the reference (file:line in zaneblood1/CMBLensing.py):

* map basis: real ``(N, N)``; Fourier basis: unnormalised ``rfft2``
  ``(N, N//2+1)``; axis 0 is the full axis ("KX", ``fftfreq``), axis 1 the
  half axis ("KY", ``rfftfreq`` with the Nyquist entry negated) --
  ``cmb_lensing/util.py:103-107``.
* every function mirrors the reference function of the same name; numpy's
  pocketfft has the same unnormalised-forward / 1/N^2-inverse convention as
  ``jax.numpy.fft``.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# ---------------------------------------------------------------- constants
# cmb_lensing/constants.py:5-8, :18-21
ARCMIN_PER_DEGREE = 60
INVERSE_LENSE = -1
FORWARD_LENSE = +1
NSIDE_DEFAULT = 256
THETA_PIX_DEFAULT = 2.5


def pix_width_of(theta_pix: float) -> float:
    """Pixel width in radians (constants.py:20, util.py:165)."""
    return float(np.deg2rad(theta_pix / ARCMIN_PER_DEGREE))


PIX_WIDTH_DEFAULT = pix_width_of(THETA_PIX_DEFAULT)


def fourier_weights_default(nside: int) -> np.ndarray:
    """Weights 2 with 0.5 at DC/Nyquist columns (constants.py:21)."""
    w = 2.0 * np.ones(nside // 2 + 1, dtype=np.complex128)
    w[0] = 0.5
    w[-1] = 0.5
    return w


def get_fourier_weights(field_shape) -> np.ndarray:
    """Weights 2 with 1 at DC/Nyquist columns (util.py:90-96)."""
    rows, _ = field_shape
    w = 2.0 * np.ones(rows // 2 + 1, dtype=np.complex128)
    w[0] = 1.0
    w[-1] = 1.0
    return w


class Basis:
    MAP = 0
    FOURIER = 1


class Parametrization:
    T = 0
    QU = 1
    EB = 2


# ------------------------------------------------------------------- fields
@dataclasses.dataclass
class Field:
    """Minimal stand-in for the flax pytrees of cmb_lensing/fields.py:15-116."""

    nside: int = NSIDE_DEFAULT
    theta_pix: float = THETA_PIX_DEFAULT
    pix_width: float = PIX_WIDTH_DEFAULT
    basis: int = Basis.FOURIER
    fourier_weights: np.ndarray = None

    def __post_init__(self):
        if self.fourier_weights is None:
            self.fourier_weights = fourier_weights_default(self.nside)

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    def _matrix_names(self):
        raise NotImplementedError

    def _binop(self, other, op):
        if isinstance(other, self.__class__):
            upd = {n: op(getattr(self, n), getattr(other, n)) for n in self._matrix_names()}
        else:
            upd = {n: op(getattr(self, n), other) for n in self._matrix_names()}
        return self.replace(**upd)

    def __add__(self, o):
        return self._binop(o, lambda a, b: a + b)

    def __sub__(self, o):
        return self._binop(o, lambda a, b: a - b)

    def __rsub__(self, o):
        return self._binop(o, lambda a, b: b - a)

    def __mul__(self, o):
        return self._binop(o, lambda a, b: a * b)

    __rmul__ = __mul__

    def __truediv__(self, o):
        return self._binop(o, lambda a, b: a / b)


@dataclasses.dataclass
class FlatS0(Field):
    scalar_matrix: np.ndarray = None
    parametrization: int = Parametrization.T

    def _matrix_names(self):
        return ["scalar_matrix"]


@dataclasses.dataclass
class FlatS2(Field):
    polar_matrix_1: np.ndarray = None
    polar_matrix_2: np.ndarray = None
    parametrization: int = Parametrization.EB

    def _matrix_names(self):
        return ["polar_matrix_1", "polar_matrix_2"]


@dataclasses.dataclass
class FlatS02(Field):
    scalar_matrix: np.ndarray = None
    polar_matrix_1: np.ndarray = None
    polar_matrix_2: np.ndarray = None
    parametrization: int = Parametrization.EB

    def _matrix_names(self):
        return ["scalar_matrix", "polar_matrix_1", "polar_matrix_2"]


# ----------------------------------------------------------------- numerics
def get_k_meshgrid(N, pix_width):
    """util.py:103-107: KX on axis 0 (fftfreq), KY on axis 1 (rfftfreq, Nyquist negated)."""
    kx = 2 * np.pi * np.fft.fftfreq(N, pix_width)
    ky = 2 * np.pi * np.fft.rfftfreq(N, pix_width)
    ky[-1] = -ky[-1]
    return np.meshgrid(kx, ky, indexing="ij")


def get_primal_derivatives(field, pix_width):
    """util.py:110-120: (Fx, Fy, Fxx, Fxy, Fyy) of a real map."""
    N = field.shape[0]
    KX, KY = get_k_meshgrid(N, pix_width)
    F = np.fft.rfft2(field)
    irf = lambda X: np.fft.irfft2(X, s=(N, N))
    return (irf(1j * KX * F), irf(1j * KY * F), irf(-(KX ** 2) * F),
            irf(-(KX * KY) * F), irf(-(KY ** 2) * F))


def get_primal_derivatives_from_fourier(phi_fourier, pix_width):
    """util.py:125-130: derivatives of an rfft2-shaped array, returned in map space."""
    N = phi_fourier.shape[0]
    KX, KY = get_k_meshgrid(N, pix_width)
    F = phi_fourier
    irf = lambda X: np.fft.irfft2(X, s=(N, N))
    return (irf(1j * KX * F), irf(1j * KY * F), irf(-(KX ** 2) * F),
            irf(-(KX * KY) * F), irf(-(KY ** 2) * F))


def get_primal_derivatives_to_fourier(field, pix_width):
    """util.py:133-137: derivative multipliers applied to rfft2(field), kept in Fourier space."""
    N = field.shape[0]
    KX, KY = get_k_meshgrid(N, pix_width)
    F = np.fft.rfft2(field)
    return (1j * KX * F), (1j * KY * F), (-(KX ** 2) * F), (-(KX * KY) * F), (-(KY ** 2) * F)


def gen_mesh_grid(nside, theta_pix):
    """util.py:163-172: lx on the half axis (axis 1), ly on the full axis (axis 0)."""
    d = math.radians(theta_pix / ARCMIN_PER_DEGREE)
    lx = 2 * np.pi * np.fft.rfftfreq(nside, d)
    ly = 2 * np.pi * np.fft.fftfreq(nside, d)
    lx, ly = np.meshgrid(lx, ly)
    return lx, ly, d


def gen_ell_grid(nside, theta_pix):
    """util.py:174-179."""
    lx, ly, d = gen_mesh_grid(nside, theta_pix)
    return np.sqrt(lx ** 2 + ly ** 2), d


def _eb_angle(nside, theta_pix):
    lx, ly, _ = gen_mesh_grid(nside, theta_pix)
    lx = lx.copy()
    # util.py:143 / :155: half-axis Nyquist column negated for rows 0..nside//2 only
    lx[: nside // 2 + 1, -1] = -lx[: nside // 2 + 1, -1]
    return np.arctan2(lx, ly)


def primal_eb2qu(e_field, b_field, nside, theta_pix):
    """util.py:140-149."""
    a = _eb_angle(nside, theta_pix)
    q = -e_field * np.cos(2 * a) + b_field * np.sin(2 * a)
    u = -e_field * np.sin(2 * a) - b_field * np.cos(2 * a)
    return q, u


def primal_qu2eb(q_field, u_field, nside, theta_pix):
    """util.py:152-161."""
    a = _eb_angle(nside, theta_pix)
    e = -q_field * np.cos(2 * a) - u_field * np.sin(2 * a)
    b = q_field * np.sin(2 * a) - u_field * np.cos(2 * a)
    return e, b


def rk4_solve(F, y0, t0, t1, nsteps, args=()):
    """util.py:184-199: classic fixed-step RK4 on a tuple of arrays."""
    h = (t1 - t0) / nsteps
    h_half = h / 2.0
    y = tuple(y0)
    for i in range(nsteps):
        t = t0 + i * h
        k1 = F(t, y, args)
        k2 = F(t + h_half, tuple(yi + h_half * ki for yi, ki in zip(y, k1)), args)
        k3 = F(t + h_half, tuple(yi + h_half * ki for yi, ki in zip(y, k2)), args)
        k4 = F(t + h, tuple(yi + h * ki for yi, ki in zip(y, k3)), args)
        y = tuple(yi + h * (a + 2 * b + 2 * c + d) / 6
                  for yi, a, b, c, d in zip(y, k1, k2, k3, k4))
    return y


def primal_dot(field_1, field_2, fourier_weights, num_pixels):
    """util.py:100-101."""
    return float(np.real(np.sum(np.conj(field_1) * field_2 * fourier_weights * (1 / num_pixels))))


def reciprocal_matrix(matrix):
    """util.py:45-47 (0 -> 0)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(matrix != 0, 1.0 / np.where(matrix != 0, matrix, 1), 0.0)


def primal_log_det(matrix, fourier_weights):
    """util.py:39-42."""
    with np.errstate(divide="ignore"):
        val = np.sum(np.where(matrix != 0, np.log(np.abs(np.where(matrix != 0, matrix, 1))), 0) * fourier_weights)
    sign = np.prod(np.sign(np.where(matrix != 0, matrix, 1)))
    return sign * val


def block_matrix_logdet(a, b, c, d, fourier_weights):
    """util.py:51-53."""
    return primal_log_det(a, fourier_weights) + primal_log_det(d - c * reciprocal_matrix(a) * b, fourier_weights)


def invert_block_matrix(a, b, c, d):
    """util.py:59-69 (Schur complement)."""
    rd = reciprocal_matrix(d)
    s = reciprocal_matrix(a - b * rd * c)
    inv_11 = s
    inv_22 = rd + rd * c * s * b * rd
    inv_12 = -s * b * rd
    inv_21 = -rd * c * s
    return inv_11, inv_12, inv_21, inv_22


# ------------------------------------------------------------ field methods
def dot(field_1, field_2):
    """fields.py:137-142: weights and nside taken from the first field."""
    s = 0.0
    for n in field_1._matrix_names():
        s += primal_dot(getattr(field_1, n), getattr(field_2, n), field_1.fourier_weights, field_1.nside ** 2)
    return s


def fourier(field):
    """fields.py:159-163."""
    upd = {n: np.fft.rfft2(getattr(field, n)) for n in field._matrix_names()}
    return field.replace(basis=Basis.FOURIER, **upd)


def map_(field):
    """fields.py:168-172 (named ``map`` in the reference)."""
    upd = {}
    for n in field._matrix_names():
        m = getattr(field, n)
        upd[n] = np.fft.irfft2(m, s=(m.shape[0], m.shape[0]))
    return field.replace(basis=Basis.MAP, **upd)


def eb2qu(field):
    """fields.py:178-199."""
    if isinstance(field, FlatS0):
        return field
    q, u = primal_eb2qu(field.polar_matrix_1, field.polar_matrix_2, field.nside, field.theta_pix)
    return field.replace(polar_matrix_1=q, polar_matrix_2=u, parametrization=Parametrization.QU)


def qu2eb(field):
    """fields.py:203-226."""
    if isinstance(field, FlatS0):
        return field
    e, b = primal_qu2eb(field.polar_matrix_1, field.polar_matrix_2, field.nside, field.theta_pix)
    return field.replace(polar_matrix_1=e, polar_matrix_2=b, parametrization=Parametrization.EB)


def undo_inner_product(field):
    """fields.py:147-154: identity for Fourier-shaped arrays."""
    def _undo(m):
        if m.shape[0] != m.shape[1]:
            return m
        N = m.shape[0]
        return np.fft.irfft2(np.conj(np.fft.rfft2(m) / field.fourier_weights) * field.nside ** 2, s=(N, N))
    return field.replace(**{n: _undo(getattr(field, n)) for n in field._matrix_names()})


# --------------------------------------------------------------- operators
@dataclasses.dataclass
class FieldOperator:
    nside: int = NSIDE_DEFAULT
    theta_pix: float = THETA_PIX_DEFAULT
    pix_width: float = PIX_WIDTH_DEFAULT
    fourier_weights: np.ndarray = None

    def __post_init__(self):
        if self.fourier_weights is None:
            self.fourier_weights = fourier_weights_default(self.nside)

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    def __add__(self, other):
        if isinstance(other, self.__class__):
            return self.replace(**{n: getattr(self, n) + getattr(other, n) for n in self._matrix_names()})
        return self.replace(**{n: getattr(self, n) + other for n in self._matrix_names()})


@dataclasses.dataclass
class DiagonalScalar(FieldOperator):
    """matrix_operators.py:46-63."""
    scalar_matrix: np.ndarray = None

    def _matrix_names(self):
        return ["scalar_matrix"]

    def __mul__(self, other):
        if isinstance(other, DiagonalScalar):
            return self.replace(scalar_matrix=self.scalar_matrix * other.scalar_matrix)
        if isinstance(other, FlatS0):
            return other.replace(scalar_matrix=self.scalar_matrix * other.scalar_matrix)
        return self.replace(scalar_matrix=self.scalar_matrix * other)

    __rmul__ = __mul__


@dataclasses.dataclass
class DiagonalEB(FieldOperator):
    """matrix_operators.py:66-90."""
    matrix_EE: np.ndarray = None
    matrix_BB: np.ndarray = None

    def _matrix_names(self):
        return ["matrix_EE", "matrix_BB"]

    def __mul__(self, other):
        if isinstance(other, DiagonalEB):
            return self.replace(matrix_EE=self.matrix_EE * other.matrix_EE, matrix_BB=self.matrix_BB * other.matrix_BB)
        if isinstance(other, FlatS2):
            return other.replace(polar_matrix_1=self.matrix_EE * other.polar_matrix_1,
                                 polar_matrix_2=self.matrix_BB * other.polar_matrix_2)
        return self.replace(matrix_EE=self.matrix_EE * other, matrix_BB=self.matrix_BB * other)

    __rmul__ = __mul__


@dataclasses.dataclass
class BlockTEB(FieldOperator):
    """matrix_operators.py:93-148 ([TT TE 0; ET EE 0; 0 0 BB])."""
    matrix_TT: np.ndarray = None
    matrix_TE: np.ndarray = None
    matrix_ET: np.ndarray = None
    matrix_EE: np.ndarray = None
    matrix_BB: np.ndarray = None

    def _matrix_names(self):
        return ["matrix_TT", "matrix_TE", "matrix_ET", "matrix_EE", "matrix_BB"]

    def __mul__(self, other):
        s = self
        if isinstance(other, BlockTEB):
            o = other
            return s.replace(matrix_TT=s.matrix_TT * o.matrix_TT + s.matrix_TE * o.matrix_ET,
                             matrix_ET=s.matrix_ET * o.matrix_TT + s.matrix_EE * o.matrix_ET,
                             matrix_TE=s.matrix_TT * o.matrix_TE + s.matrix_TE * o.matrix_EE,
                             matrix_EE=s.matrix_ET * o.matrix_TE + s.matrix_EE * o.matrix_EE,
                             matrix_BB=s.matrix_BB * o.matrix_BB)
        if isinstance(other, FlatS02):
            return other.replace(scalar_matrix=s.matrix_TT * other.scalar_matrix + s.matrix_TE * other.polar_matrix_1,
                                 polar_matrix_1=s.matrix_ET * other.scalar_matrix + s.matrix_EE * other.polar_matrix_1,
                                 polar_matrix_2=s.matrix_BB * other.polar_matrix_2)
        return s.replace(**{n: getattr(s, n) * other for n in s._matrix_names()})

    def __rmul__(self, other):
        if isinstance(other, BlockTEB):
            return other.__mul__(self)
        return self.replace(**{n: getattr(self, n) * other for n in self._matrix_names()})


def pinv(op):
    """matrix_operators.py:205-234."""
    if isinstance(op, DiagonalScalar):
        return op.replace(scalar_matrix=reciprocal_matrix(op.scalar_matrix))
    if isinstance(op, DiagonalEB):
        return op.replace(matrix_EE=reciprocal_matrix(op.matrix_EE), matrix_BB=reciprocal_matrix(op.matrix_BB))
    if isinstance(op, BlockTEB):
        tt, te, et, ee = invert_block_matrix(op.matrix_TT, op.matrix_TE, op.matrix_ET, op.matrix_EE)
        return op.replace(matrix_TT=tt, matrix_TE=te, matrix_ET=et, matrix_EE=ee,
                          matrix_BB=reciprocal_matrix(op.matrix_BB))
    raise TypeError(type(op))


def log_det(op):
    """matrix_operators.py:175-200."""
    w = op.fourier_weights
    if isinstance(op, DiagonalScalar):
        return primal_log_det(op.scalar_matrix, w)
    if isinstance(op, DiagonalEB):
        return primal_log_det(op.matrix_EE, w) + primal_log_det(op.matrix_BB, w)
    if isinstance(op, BlockTEB):
        return (block_matrix_logdet(op.matrix_TT, op.matrix_TE, op.matrix_ET, op.matrix_EE, w)
                + primal_log_det(op.matrix_BB, w))
    raise TypeError(type(op))


# --------------------------------------------------------------- LenseFlow
def get_m_matrix_components_at_time(time, phi_xx, phi_xy, phi_yy):
    """lense_flow.py:398-405."""
    return 1 + time * phi_xx, time * phi_xy, time * phi_xy, 1 + time * phi_yy


def get_inverse_matrix_components(m_xx, m_xy, m_yy, eps=1e-12):
    """lense_flow.py:408-415 (det + 1e-12, no guard)."""
    det = m_xx * m_yy - m_xy * m_xy
    inv_det = 1.0 / (det + eps)
    return m_yy * inv_det, -m_xy * inv_det, m_xx * inv_det


def get_p_vector_components(phi_x, phi_y, phi_xx, phi_xy, phi_yy, time):
    """lense_flow.py:373-381: p = M^-1 grad(phi)."""
    m_xx, m_xy, _, m_yy = get_m_matrix_components_at_time(time, phi_xx, phi_xy, phi_yy)
    ixx, ixy, iyy = get_inverse_matrix_components(m_xx, m_xy, m_yy)
    return phi_x * ixx + phi_y * ixy, phi_x * ixy + phi_y * iyy


def get_v_vector_components(time, field, phi_xx, phi_xy, phi_yy, pix_width):
    """lense_flow.py:384-395: v = M^-1 grad(f)."""
    fx, fy, _, _, _ = get_primal_derivatives(field, pix_width)
    m_xx, m_xy, _, m_yy = get_m_matrix_components_at_time(time, phi_xx, phi_xy, phi_yy)
    ixx, ixy, iyy = get_inverse_matrix_components(m_xx, m_xy, m_yy)
    return fx * ixx + fy * ixy, fy * iyy + fx * ixy


def get_standard_lensing_term(field, phi_x, phi_y, phi_xx, phi_xy, phi_yy, t, pix_width):
    """lense_flow.py:365-370: df/dt = grad(phi)^T M^-1 grad(f)."""
    vx, vy = get_v_vector_components(t, field, phi_xx, phi_xy, phi_yy, pix_width)
    return phi_x * vx + phi_y * vy


def get_adjoint_lensing_term(field, phi_x, phi_y, phi_xx, phi_xy, phi_yy, t, pix_width):
    """lense_flow.py:355-362: df/dt = d/dx(p_x f) + d/dy(p_y f)."""
    px, py = get_p_vector_components(phi_x, phi_y, phi_xx, phi_xy, phi_yy, t)
    dx = get_primal_derivatives(px * field, pix_width)[0]
    dy = get_primal_derivatives(py * field, pix_width)[1]
    return dx + dy


def phi_derivatives(phi, pix_width):
    """lense_flow.py:299-302: map (N,N) or Fourier (N,N/2+1) phi."""
    if phi.shape[0] != phi.shape[1]:
        return get_primal_derivatives_from_fourier(phi, pix_width)
    return get_primal_derivatives(phi, pix_width)


def time_span(direction, adjoint):
    """lense_flow.py:304-322: forward time iff (direction == +1) XOR adjoint."""
    if (direction == FORWARD_LENSE) != bool(adjoint):
        return 0.0, 1.0
    return 1.0, 0.0


def primal_lense_flow(primal_field, phi, pix_width, n, direction, adjoint, derivs=None):
    """lense_flow.py:295-333 (``derivs`` lets callers reuse the phi derivatives)."""
    if derivs is None:
        derivs = phi_derivatives(phi, pix_width)
    t0, t1 = time_span(direction, adjoint)
    rhs = get_adjoint_lensing_term if adjoint else get_standard_lensing_term

    def step(t, y, args):
        return (rhs(y[0], *derivs, t, pix_width),)

    return rk4_solve(step, (np.asarray(primal_field, dtype=np.float64),), t0, t1, n)[0]


def lense_flow(field, phi, n=10, direction=1, adjoint=False):
    """lense_flow.py:289-292: each matrix of the field lensed independently."""
    derivs = phi_derivatives(phi.scalar_matrix, field.pix_width)
    upd = {name: primal_lense_flow(getattr(field, name), phi.scalar_matrix, field.pix_width, n, direction,
                                   adjoint, derivs) for name in field._matrix_names()}
    return field.replace(**upd)


# ------------------------------------------------- custom VJP (lense_flow.py:10-252)
def spin_vector_matrix_data(field):
    """lense_flow.py:254-284: pack to (T, Q, U) with zeros for missing components."""
    if isinstance(field, FlatS02):
        return field.scalar_matrix, field.polar_matrix_1, field.polar_matrix_2
    if isinstance(field, FlatS2):
        z = np.zeros_like(field.polar_matrix_1)
        return z, field.polar_matrix_1, field.polar_matrix_2
    if isinstance(field, FlatS0):
        z = np.zeros_like(field.scalar_matrix)
        return field.scalar_matrix, z, z
    raise TypeError(type(field))


def output_like_input(input_field, t, q, u):
    """lense_flow.py:128-152 -- note the reference writes polar_matrix_1=U, polar_matrix_2=Q."""
    if isinstance(input_field, FlatS02):
        return input_field.replace(scalar_matrix=t, polar_matrix_1=u, polar_matrix_2=q)
    if isinstance(input_field, FlatS2):
        return input_field.replace(polar_matrix_1=u, polar_matrix_2=q)
    if isinstance(input_field, FlatS0):
        return input_field.replace(scalar_matrix=t)
    raise TypeError(type(input_field))


def get_delta_phi_tqu_roc(t, q, u, dt_, dq, du, phi_x, phi_y, phi_xx, phi_xy, phi_yy, time, pix_width,
                          phi_fourier=False):
    """lense_flow.py:195-252: rate of change of delta-phi."""
    tx, ty = get_primal_derivatives(t, pix_width)[:2]
    qx, qy = get_primal_derivatives(q, pix_width)[:2]
    ux, uy = get_primal_derivatives(u, pix_width)[:2]
    fdf_x = dt_ * tx + dq * qx + du * ux
    fdf_y = dt_ * ty + dq * qy + du * uy
    m_xx, m_xy, _, m_yy = get_m_matrix_components_at_time(time, phi_xx, phi_xy, phi_yy)
    ixx, ixy, iyy = get_inverse_matrix_components(m_xx, m_xy, m_yy)
    a_x = ixx * fdf_x + ixy * fdf_y
    a_y = ixy * fdf_x + iyy * fdf_y
    p_x, p_y = get_p_vector_components(phi_x, phi_y, phi_xx, phi_xy, phi_yy, time)
    w_xx, w_xy, w_yx, w_yy = p_x * a_x, p_x * a_y, p_y * a_x, p_y * a_y
    if phi_fourier:
        D = lambda f: get_primal_derivatives_to_fourier(f, pix_width)
    else:
        D = lambda f: get_primal_derivatives(f, pix_width)
    div = D(a_x)[0] + D(a_y)[1]
    lap = D(time * w_xx)[2] + D(time * w_xy)[3] + D(time * w_yx)[3] + D(time * w_yy)[4]
    return lap + div


def get_lensing_operator_gradients(phi_matrix, pix_width, tqu_field, tqu_cotangent, direction, n):
    """lense_flow.py:54-126: integrate (f, delta_f, delta_phi) with RK4.

    ``tqu_field``/``tqu_cotangent`` are (T, Q, U) map-space arrays.  Returns
    the integrated (f', delta_f, delta_phi) arrays without the output
    repacking (the caller applies ``output_like_input``).
    """
    if direction == INVERSE_LENSE:
        t0, t1 = 1.0, 0.0
    else:
        t0, t1 = 0.0, 1.0
    phi_fourier = phi_matrix.shape[0] != phi_matrix.shape[1]
    derivs = phi_derivatives(phi_matrix, pix_width)
    if phi_fourier:
        dphi0 = np.zeros(phi_matrix.shape, dtype=np.complex128)
    else:
        dphi0 = np.zeros(phi_matrix.shape, dtype=np.float64)

    def step(time, y, args):
        t, q, u, dt_, dq, du, _ = y
        r = [get_standard_lensing_term(c, *derivs, time, pix_width) for c in (t, q, u)]
        r += [get_adjoint_lensing_term(c, *derivs, time, pix_width) for c in (dt_, dq, du)]
        r.append(get_delta_phi_tqu_roc(t, q, u, dt_, dq, du, *derivs, time, pix_width, phi_fourier))
        return tuple(r)

    y0 = tuple(np.asarray(a, dtype=np.float64) for a in (*tqu_field, *tqu_cotangent)) + (dphi0,)
    return rk4_solve(step, y0, t0, t1, n)


def lensing_operator_gradients_exact(phi_matrix, pix_width, tqu_field, tqu_cotangent, direction, n):
    """The exact transpose of the discrete forward RK4 lens (the engine's checkpointed reverse pass).

    No counterpart in the reference: this restates the engine's extension
    ``lf_lense_flow_vjp_ckpt`` so that the tests can check it.  ``tqu_field``
    is the UNLENSED (T, Q, U) map and ``direction`` the direction of the lens
    being differentiated.  The forward RK4 (util.py:184-199 with the standard
    RHS, lense_flow.py:365-370) keeps y_i at the start of every step; each
    step is recomputed backwards from it, one RK4 step of the adjoint RHS
    (lense_flow.py:355-362, with the negated step) carries the cotangent over
    it, and forward stage s pairs with adjoint stage 5 - s at the same time:
    delta-phi gains h_back/6 {1,2,2,1}_j get_delta_phi_tqu_roc(u_{5-j}, v_j)
    with u the forward stage inputs and v the adjoint ones.  Pinned by central
    finite differences of the discrete lens (tests/test_oracle_golden.py).
    Returns (t, q, u lensed, delta_t, delta_q, delta_u, delta_phi).
    """
    t0, t1 = time_span(direction, False)
    h = (t1 - t0) / n
    hb = -h
    phi_fourier = phi_matrix.shape[0] != phi_matrix.shape[1]
    derivs = phi_derivatives(phi_matrix, pix_width)
    A = lambda y, t: get_standard_lensing_term(y, *derivs, t, pix_width)
    G = lambda y, t: get_adjoint_lensing_term(y, *derivs, t, pix_width)

    def stage_inputs(y, t):
        k1 = [A(c, t) for c in y]
        u2 = [c + h / 2 * k for c, k in zip(y, k1)]
        k2 = [A(c, t + h / 2) for c in u2]
        u3 = [c + h / 2 * k for c, k in zip(y, k2)]
        k3 = [A(c, t + h / 2) for c in u3]
        u4 = [c + h * k for c, k in zip(y, k3)]
        k4 = [A(c, t + h) for c in u4]
        return [y, u2, u3, u4], [c + h / 6 * (a + 2 * b + 2 * cc + d) for c, a, b, cc, d in zip(y, k1, k2, k3, k4)]

    y = [np.asarray(c, dtype=np.float64) for c in tqu_field]
    checkpoints = []
    for i in range(n):
        checkpoints.append(y)
        y = stage_inputs(y, t0 + i * h)[1]
    lensed = y
    dphi = np.zeros(phi_matrix.shape, dtype=np.complex128 if phi_fourier else np.float64)
    v = [np.asarray(c, dtype=np.float64) for c in tqu_cotangent]
    weights = (1.0, 2.0, 2.0, 1.0)
    for i in reversed(range(n)):
        t = t0 + i * h
        us = stage_inputs(checkpoints[i], t)[0]
        taus = (t + h, t + h / 2, t + h / 2, t)
        vs, ks = [], []
        for j in range(4):
            vj = v if j == 0 else [a + (hb if j == 3 else hb / 2) * k for a, k in zip(v, ks[-1])]
            vs.append(vj)
            ks.append([G(c, taus[j]) for c in vj])
            dphi = dphi + hb / 6 * weights[j] * get_delta_phi_tqu_roc(*us[3 - j], *vj, *derivs, taus[j], pix_width,
                                                                      phi_fourier)
        v = [a + hb / 6 * (p + 2 * q + 2 * r + s) for a, p, q, r, s in zip(v, *ks)]
    return (*lensed, *v, dphi)


def lense_flow_backwards(transformed_field, phi, cotangent, n=10, direction=1):
    """lense_flow.py:23-46: (delta_field, delta_phi) after undo_inner_product."""
    tqu = spin_vector_matrix_data(transformed_field)
    cot = spin_vector_matrix_data(cotangent)
    res = get_lensing_operator_gradients(phi.scalar_matrix, phi.pix_width, tqu, cot, -direction, n)
    delta_field = output_like_input(transformed_field, res[3], res[4], res[5])
    delta_phi = phi.replace(scalar_matrix=res[6])
    return undo_inner_product(delta_field), undo_inner_product(delta_phi)


# ------------------------------------------------------------ statistics
def logpdf(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, n=10):
    """statistics.py:139-165 (``n`` exposes the reference's default of 10 RK4 steps)."""
    phi_logdet = log_det(phi_covariance)
    noise_logdet = log_det(noise_covariance)
    field_logdet = log_det(field_covariance)
    field_product = dot(field, pinv(field_covariance) * field)
    phi_product = dot(phi, pinv(phi_covariance) * phi)
    fmap = map_(eb2qu(field))
    lensed = qu2eb(fourier(lense_flow(fmap, phi, n=n)))
    diff = data - mask * beam * lensed
    data_product = dot(diff, pinv(noise_covariance) * diff)
    return -np.real(data_product + field_product + phi_product + noise_logdet + phi_logdet + field_logdet) / 2


def gradf_logpdf(field, phi, data, field_covariance, noise_covariance, mask, beam, n=10):
    """gradients.py:13-26: L^dag B M Cn^-1 (d - M B L f) - Cf^-1 f."""
    fmap = map_(eb2qu(field))
    phimap = map_(phi)
    lensed = qu2eb(fourier(lense_flow(fmap, phimap, n=n)))
    g = beam * mask * pinv(noise_covariance) * (data - mask * beam * lensed)
    g = map_(eb2qu(g))
    g = lense_flow(g, phimap, n=n, adjoint=True)
    # gradients.py:243 rebinds ``field`` to the QU map, so the prior term
    # round-trips the field through map space (this matters on the
    # DC/Nyquist columns, where rfft2(irfft2(x)) != x).
    return qu2eb(fourier(g)) - pinv(field_covariance) * qu2eb(fourier(fmap))


def _half_plane_weight_ratio(nside, fourier_weights):
    """w / w_std where w_std = (1, 2, ..., 2, 1) is the weighting implied by irfft2."""
    w_std = get_fourier_weights((nside, nside))
    return np.real(fourier_weights / w_std)


def grad_phi_logpdf(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, n=10,
                    scheme="reference"):
    """gradients.py:30-37: ``jax.grad(logpdf, argnums=1)`` restated by hand.

    The data term's cotangent w.r.t. the lensed QU/T map (a real array, so
    its JAX gradient is the ordinary partial derivative) is
    ``irfft2(eb2qu(B M Cn^-1 diff) * w / w_std)``; it is fed to the
    reference's custom VJP (lense_flow.py:23-46) with phi in Fourier space.
    The phi prior's custom VJP (statistics.py:199-209) contributes
    ``-1/2 * 2 Cphi^-1 phi``.  ``scheme="exact"`` replaces the reverse pass
    with ``lensing_operator_gradients_exact`` (the engine's checkpointed
    extension; no reference counterpart).
    """
    fmap = map_(eb2qu(field))
    lensed_map = lense_flow(fmap, phi, n=n)
    lensed = qu2eb(fourier(lensed_map))
    diff = data - mask * beam * lensed
    g = beam * mask * (pinv(noise_covariance) * diff)
    h = eb2qu(g)
    ratio = _half_plane_weight_ratio(data.nside, diff.fourier_weights)
    N = data.nside
    cot = h.replace(**{nm: np.fft.irfft2(getattr(h, nm) * ratio, s=(N, N)) for nm in h._matrix_names()},
                    basis=Basis.MAP)
    if scheme == "exact":
        res = lensing_operator_gradients_exact(phi.scalar_matrix, phi.pix_width, spin_vector_matrix_data(fmap),
                                               spin_vector_matrix_data(cot), FORWARD_LENSE, n)
        dphi = undo_inner_product(phi.replace(scalar_matrix=res[6]))
    else:
        _, dphi = lense_flow_backwards(lensed_map, phi, cot, n=n, direction=FORWARD_LENSE)
    prior = pinv(phi_covariance) * phi
    return dphi.scalar_matrix - prior.scalar_matrix


# ------------------------------------------------------------------ mixing
def mix(field, phi, mixing_d, mixing_g, n=10):
    """mixing.py:8-20: f_mixed = qu2eb(fourier(L(phi) map(eb2qu(D f)))), phi_mixed = G phi."""
    df = map_(eb2qu(mixing_d * field))
    mixed_field = qu2eb(fourier(lense_flow(df, map_(phi), n=n)))
    return mixed_field, mixing_g * phi


def unmix(mixed_field, mixed_phi, mixing_d, mixing_g, n=10):
    """mixing.py:23-36: phi = G^-1 phi_mixed, f = D^-1 qu2eb(fourier(L^-1(phi) map(eb2qu(f_mixed))))."""
    phi = pinv(mixing_g) * mixed_phi
    mmap = map_(eb2qu(mixed_field))
    field = qu2eb(fourier(lense_flow(mmap, map_(phi), n=n, direction=INVERSE_LENSE)))
    return pinv(mixing_d) * field, phi


def mixing_jacobian_phi_component(mixed_field, phi, grad_f, mixing_d, n=10):
    """gradients.py:63-85: the pullback of phi -> map(D^-1 qu2eb(fourier(L^-1(phi) f_mixed_map))).

    phi is Fourier-shaped, so the reference's custom VJP returns delta-phi in
    the Fourier basis.  The pullback of ``map`` applied to the cotangent
    map(grad_f) is w conj(rfft2(map(grad_f))) / N^2 (JAX's irfft2 transpose),
    D^-1 and qu2eb transpose to themselves / eb2qu (real coefficients per
    mode), and the transpose of ``fourier`` is N^2 irfft2(conj(.) / w).  The
    weights and conjugations cancel, so the cotangent of the inverse-lensed QU
    map is map(eb2qu(D^-1 fourier(map(grad_f)))).
    """
    mmap = map_(eb2qu(mixed_field))
    unlensed = lense_flow(mmap, phi, n=n, direction=INVERSE_LENSE)
    cot = map_(eb2qu(pinv(mixing_d) * fourier(map_(grad_f))))
    _, dphi = lense_flow_backwards(unlensed, phi, cot, n=n, direction=INVERSE_LENSE)
    return dphi.scalar_matrix


def mixed_grad_phi_logpdf(mixed_field, mixed_phi, data, noise_covariance, phi_covariance, field_covariance,
                          mask, beam, mixing_d, mixing_g, n=10):
    """gradients.py:41-60: G^-1 (grad_phi logpdf + J_phi^T grad_f logpdf) at the unmixed point."""
    field, phi = unmix(mixed_field, mixed_phi, mixing_d, mixing_g, n=n)
    grad_phi = grad_phi_logpdf(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                               n=n)
    grad_f = gradf_logpdf(field, phi, data, field_covariance, noise_covariance, mask, beam, n=n)
    chain = mixing_jacobian_phi_component(mixed_field, phi, grad_f, mixing_d, n=n)
    return (pinv(mixing_g) * phi.replace(scalar_matrix=grad_phi + chain)).scalar_matrix


# ---------------------------------------------------------- Wiener filter
def hessian_logpdf_preconditioner(field_covariance, beam, mask, noise_covariance):
    """wiener_filter.py:36-43."""
    return pinv(field_covariance) + beam * mask * pinv(noise_covariance) * mask * beam


def conjugate_gradient(x0, apply_A, b_vector, preconditioner, maxiter=500, tol=1e-1, rel_tol=None,
                       history=None):
    """wiener_filter.py:52-104: the reference PCG recurrence.

    Stops when r.z < tol (absolute, the reference rule) or, if ``rel_tol`` is
    given, when ||r|| / ||b|| < rel_tol (norms from ``dot``).
    """
    Pinv = pinv(preconditioner)
    x = x0
    r = b_vector - apply_A(x0)
    z = Pinv * r
    p = z
    res = dot(r, z)
    bnorm = math.sqrt(max(dot(b_vector, b_vector), 1e-300))
    it = 0
    while it < maxiter:
        if rel_tol is None:
            if not res >= tol:
                break
        elif math.sqrt(max(dot(r, r), 0.0)) / bnorm < rel_tol:
            break
        Ap = apply_A(p)
        alpha = res / dot(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = Pinv * r
        res_curr = dot(r, z)
        p = z + (res_curr / res) * p
        res = res_curr
        it += 1
        if history is not None:
            history.append(math.sqrt(max(dot(r, r), 0.0)) / bnorm)
    return x, it


def wiener_filter(field, phi, data, field_covariance, noise_covariance, mask, beam, n=10, maxiter=500,
                  tol=1e-1, rel_tol=None):
    """wiener_filter.py:11-49: b = -gradf(0, d), A = gradf(., d=0)."""
    zero = data * 0
    b = gradf_logpdf(zero, phi, data, field_covariance, noise_covariance, mask, beam, n=n) * -1
    P = hessian_logpdf_preconditioner(field_covariance, beam, mask, noise_covariance)

    def apply_A(f):
        return gradf_logpdf(f, phi, f * 0, field_covariance, noise_covariance, mask, beam, n=n)

    return conjugate_gradient(field, apply_A, b, P, maxiter=maxiter, tol=tol, rel_tol=rel_tol)


# --------------------------------------------------- simulation and sampling
def field_from_normals(nside, covar_matrix, real_normals, imag_normals):
    """simulate.py:106-113 with the two normal draws given: irfft2(sqrt(C/2) (a + i b), norm="ortho")."""
    field = np.sqrt(np.asarray(covar_matrix) / 2) * (real_normals + 1j * imag_normals)
    return np.fft.irfft2(field, s=(nside, nside), norm="ortho")


def mixed_logpdf(mixed_field, mixed_phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                 mixing_g, mixing_d, n=10):
    """statistics.py:168-181: logpdf at the unmixed point minus Re log det G and Re log det D."""
    field, phi = unmix(mixed_field, mixed_phi, mixing_d, mixing_g, n=n)
    value = logpdf(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, n=n)
    return value - np.real(log_det(mixing_g)) - np.real(log_det(mixing_d))


def get_mass_matrix(cphi, nphi, mixing_g):
    """sampling_ar.py:65-66: G^-1 G^-1 (Cphi^-1 + Nphi^-1)."""
    return pinv(mixing_g) * pinv(mixing_g) * (pinv(cphi) + pinv(nphi))


def symplectic_integrate(x0, p0, mixed_field, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                         mixing_d, mixing_g, mass_matrix, num_steps=30, step_size=0.01, n=10):
    """sampling_ar.py:104-135: the reference's leapfrog (gradient of +logpdf) and delta H."""
    def grad(x):
        return x.replace(scalar_matrix=mixed_grad_phi_logpdf(mixed_field, x, data, noise_covariance, phi_covariance,
                                                             field_covariance, mask, beam, mixing_d, mixing_g, n=n))

    def hamiltonian(x, p):
        lp = mixed_logpdf(mixed_field, x, data, noise_covariance, phi_covariance, field_covariance, mask, beam,
                          mixing_g, mixing_d, n=n)
        return lp - dot(p, (pinv(mass_matrix) * p) / 2)

    minv = pinv(mass_matrix)
    g = grad(x0)
    x, p = x0, p0
    for _ in range(num_steps):
        prev = g
        x = x - step_size * (minv * (p - 0.5 * step_size * g))
        g = grad(x)
        p = p - 0.5 * step_size * (g + prev)
    return hamiltonian(x, p) - hamiltonian(x0, p0), x, p


def hmc_step_from_draws(x, always_accept, mass_matrix, p_real, p_imag, log_u, mixed_field, data, noise_covariance,
                        phi_covariance, field_covariance, mask, beam, mixing_d, mixing_g, num_steps=30,
                        step_size=0.01, n=10):
    """sampling_ar.py:69-100 with the momentum normals and log(uniform) given.

    The momentum is a FlatS0 with the mixed field's Fourier weights (the
    reference writes it through ``mixed_field.replace(scalar_matrix=...)``).
    """
    nside = x.nside
    p = FlatS0(scalar_matrix=np.fft.rfft2(field_from_normals(nside, mass_matrix.scalar_matrix, p_real, p_imag)),
               fourier_weights=mixed_field.fourier_weights)
    delta_h, x_test, _ = symplectic_integrate(x, p, mixed_field, data, noise_covariance, phi_covariance,
                                              field_covariance, mask, beam, mixing_d, mixing_g, mass_matrix,
                                              num_steps=num_steps, step_size=step_size, n=n)
    accept = bool(always_accept or (log_u < delta_h))
    return (x_test if accept else x), delta_h, accept


def gibbs_sample_f_from_draws(field_start, data, phi, field_covariance, noise_covariance, mask, beam, f_draws,
                              n_draws, n=10, maxiter=500, tol=1e-1):
    """sampling_ar.py:15-46 for a T field with the two normal pairs given.

    f' = f_sim + WF(d - (M B L f_sim + n_sim)): a constrained realisation.
    """
    nside = data.nside
    new_field = field_start.replace(scalar_matrix=np.fft.rfft2(
        field_from_normals(nside, field_covariance.scalar_matrix, *f_draws)))
    new_noise = field_start.replace(scalar_matrix=np.fft.rfft2(
        field_from_normals(nside, noise_covariance.scalar_matrix, *n_draws)))
    lensed = qu2eb(fourier(lense_flow(map_(eb2qu(new_field)), map_(phi), n=n)))
    new_data = mask * beam * lensed + new_noise
    delta, _ = wiener_filter(field_start, phi, data - new_data, field_covariance, noise_covariance, mask, beam, n=n,
                             maxiter=maxiter, tol=tol)
    return new_field + delta


# ---------------------------------------------------------------- MAP joint
def get_scalar_identity(op):
    """matrix_operators.py:159-170."""
    shape = (op.nside, op.nside // 2 + 1)
    return DiagonalScalar(fourier_weights=get_fourier_weights(shape), nside=op.nside, theta_pix=op.theta_pix,
                          pix_width=op.pix_width, scalar_matrix=np.ones(shape, dtype=np.complex128))


def zero_scalar_field_like(field):
    """fields.py:123-133."""
    shape = (field.nside, field.nside // 2 + 1)
    return FlatS0(fourier_weights=get_fourier_weights(shape), nside=field.nside, theta_pix=field.theta_pix,
                  pix_width=field.pix_width, scalar_matrix=np.zeros(shape, dtype=np.complex128))


def phi_gradient_hessian(phi_covariance, quadratic_estimate):
    """map_joint.py:72-77: Cphi^-1 + Nphi^-1."""
    return pinv(phi_covariance) + pinv(quadratic_estimate)


def logpdf_at_phi_new(alpha, grad_phi, mixed_field, phi_predict, data, beam, mask, field_covariance, phi_covariance,
                      noise_covariance, mixing_d, mixing_g, hessian, n=10):
    """map_joint.py:79-98: -logpdf at unmix(f_mixed, phi + alpha H^-1 grad)."""
    test_phi = phi_predict + alpha * (hessian * grad_phi)
    field, phi = unmix(mixed_field, test_phi, mixing_d, mixing_g, n=n)
    return -logpdf(field, phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, n=n)


def map_joint(data, noise_covariance, mixing_d, field_covariance, phi_covariance, quadratic_estimate, mask, beam,
              num_steps=30, constant_step=False, n=10, wf_maxiter=500, wf_tol=1e-1):
    """map_joint.py:19-67 with the data set's members passed one by one.

    Each step: Wiener-filter f at the current phi (reference rule), mix with
    G = 1, the mixed phi gradient, a scipy BFGS search for the step length
    alpha (from 1; alpha = 1 throughout with ``constant_step``) and
    phi <- phi + alpha H^-1-preconditioned gradient, H = Cphi^-1 + Nphi^-1.
    """
    from scipy.optimize import minimize
    mixing_g = get_scalar_identity(mixing_d)
    field = data * 0
    phi = zero_scalar_field_like(data)
    hessian = pinv(phi_gradient_hessian(phi_covariance, quadratic_estimate))
    alpha = 1.0
    for _ in range(num_steps):
        field, _ = wiener_filter(field, phi, data, field_covariance, noise_covariance, mask, beam, n=n,
                                 maxiter=wf_maxiter, tol=wf_tol)
        mixed_field, mixed_phi = mix(field, phi, mixing_d, mixing_g, n=n)
        grad = mixed_phi.replace(scalar_matrix=mixed_grad_phi_logpdf(
            mixed_field, mixed_phi, data, noise_covariance, phi_covariance, field_covariance, mask, beam, mixing_d,
            mixing_g, n=n))
        if not constant_step:
            f = lambda a: logpdf_at_phi_new(float(np.asarray(a).ravel()[0]), grad, mixed_field, mixed_phi, data,
                                            beam, mask, field_covariance, phi_covariance, noise_covariance,
                                            mixing_d, mixing_g, hessian, n=n)
            alpha = float(minimize(f, 1.0, method="BFGS").x[0])
        phi = phi + alpha * (hessian * grad)
    return field, phi


# ----------------------------------------------- quadratic-estimate noise
def _qe_k_grid(N, pix_width):
    """simulate.py:213-228 / :254-258: KX = 2 pi fftfreq, KY = 2 pi rfftfreq (no Nyquist flip)."""
    kx = 2 * np.pi * np.fft.fftfreq(N, pix_width)
    ky = 2 * np.pi * np.fft.rfftfreq(N, pix_width)
    return np.meshgrid(kx, ky, indexing="ij")


def qe_leg(field, pix_width, encapsulated, isolated):
    """simulate.py:272-302: (i KX)^nx (i KY)^ny F / |K|^len(isolated), NaN -> 0 (index 0 = x, 1 = y)."""
    field = np.nan_to_num(np.asarray(field, dtype=np.complex128), nan=0)
    idx = list(encapsulated) + list(isolated)
    ny = sum(idx)
    nx = len(idx) - ny
    if nx == 0 and ny == 0:
        return field
    KX, KY = _qe_k_grid(field.shape[0], pix_width)
    lap = KX ** 2 + KY ** 2
    with np.errstate(divide="ignore", invalid="ignore"):
        res = (1j * KX) ** nx * (1j * KY) ** ny * field / np.sqrt(lap ** len(isolated))
    return np.nan_to_num(res, nan=0)


def get_specific_derivative(F, pix_width, i, j):
    """simulate.py:231-251 for two indices: d_i d_j in Fourier space (xx, yy or xy)."""
    KX, KY = _qe_k_grid(F.shape[0], pix_width)
    K = (KX, KY)
    return -(K[i] * K[j]) * F


def _indices(length):
    """simulate.py:198-213: every 0/1 tuple of ``length``, grouped by the number of zeros."""
    import itertools
    out = []
    for n0 in range(length + 1):
        for zeros in itertools.combinations(range(length), n0):
            p = [1] * length
            for z in zeros:
                p[z] = 0
            out.append(tuple(p))
    return out


def scalar_quadratic_estimate(cn_tt, cf_tt, cfl_tt, m_tt, b_tt, pix_width):
    """simulate.py:305-315 / :357-367: the T quadratic-estimate noise 1 / sum_ij |d_i d_j rfft2(internal_ij)|."""
    N = cf_tt.shape[0]
    irf = lambda X: np.fft.irfft2(X, s=(N, N))
    tf = m_tt * b_tt
    sigma = tf ** 2 * cfl_tt + cn_tt
    with np.errstate(divide="ignore", invalid="ignore"):
        a1, a0, a2 = tf ** 2 * cf_tt ** 2 / sigma, tf ** 2 / sigma, tf ** 2 * cf_tt / sigma
    total = np.zeros(cf_tt.shape)
    for i, j in _indices(2):
        internal = (irf(qe_leg(a1, pix_width, (i, j), ())) * irf(qe_leg(a0, pix_width, (), ()))
                    + irf(qe_leg(a2, pix_width, (i,), ())) * irf(qe_leg(a2, pix_width, (j,), ())))
        total = total + np.abs(get_specific_derivative(np.fft.rfft2(internal), pix_width, i, j))
    with np.errstate(divide="ignore"):
        return np.nan_to_num(1 / total, nan=0, posinf=0, neginf=0)


def levi_civita_3d():
    """simulate.py:265-269."""
    i, j, k = np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing="ij")
    return (i - j) * (j - k) * (k - i) / 2


def get_polar_qe_norm_at_position(tf2e, cf_ee, sigma_e, tf2b, cf_bb, sigma_b, pix_width, i, j, k, l, m, n, p, q):
    """simulate.py:370-385."""
    N = cf_ee.shape[0]
    irf = lambda X: np.fft.irfft2(X, s=(N, N))
    with np.errstate(divide="ignore", invalid="ignore"):
        e2, e1, e0 = tf2e * cf_ee ** 2 / sigma_e, tf2e * cf_ee / sigma_e, tf2e / sigma_e
        b2, b1, b0 = tf2b * cf_bb ** 2 / sigma_b, tf2b * cf_bb / sigma_b, tf2b / sigma_b
    klmn, klpq = (k, l, m, n), (k, l, p, q)
    return (irf(qe_leg(e2, pix_width, (i, j), klmn)) * irf(qe_leg(b0, pix_width, (), klpq))
            - 2 * irf(qe_leg(e1, pix_width, (i,), klmn)) * irf(qe_leg(b1, pix_width, (j,), klpq))
            + irf(qe_leg(e0, pix_width, (), klmn)) * irf(qe_leg(b2, pix_width, (i, j), klpq)))


def polar_quadratic_estimate(cf_ee, cf_bb, cfl_ee, cfl_bb, cn_ee, cn_bb, mask_ee, mask_bb, beam_ee, beam_bb,
                             pix_width):
    """simulate.py:318-354: the EB quadratic-estimate noise."""
    eps = levi_civita_3d()
    tf2e, tf2b = (mask_ee * beam_ee) ** 2, (mask_bb * beam_bb) ** 2
    sigma_e, sigma_b = tf2e * cfl_ee + cn_ee, tf2b * cfl_bb + cn_bb
    total = np.zeros(cf_ee.shape)
    for i, j in _indices(2):
        internal = np.zeros((cf_ee.shape[0],) * 2)
        for (k, l, m, n, p, q) in _indices(6):
            w = 4 * eps[m, p, 2] * eps[n, q, 2]
            if w == 0:
                continue
            internal = internal + w * get_polar_qe_norm_at_position(tf2e, cf_ee, sigma_e, tf2b, cf_bb, sigma_b,
                                                                    pix_width, i, j, k, l, m, n, p, q)
        total = total + np.abs(get_specific_derivative(np.fft.rfft2(internal), pix_width, i, j))
    with np.errstate(divide="ignore"):
        return np.nan_to_num(1 / total, nan=0, posinf=0, neginf=0)
