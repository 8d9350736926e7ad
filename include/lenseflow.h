/* LenseFlow engine for B200 (sm_100a): C ABI.
 *
 * Plain pointers and sizes only.  Every device pointer is caller-owned and
 * must be 16-byte aligned; the library never frees caller memory.  Every call
 * that launches work takes a cudaStream_t passed as ``void*`` (NULL = the
 * legacy default stream) and is asynchronous with respect to the host.
 *
 * Layouts (row-major, as in zaneblood1/CMBLensing.py):
 *   field  : [batch][ncomp][N][N]          map basis, float32 or float64
 *            (ncomp 1 = T, 2 = Q,U, 3 = T,Q,U -- the matrices of FlatS0 /
 *             FlatS2 / FlatS02, cmb_lensing/fields.py:81-116)
 *   phi    : [batch][N][N] float64 map, or [batch][N][N/2+1] complex128
 *            (interleaved re,im) Fourier = unnormalised rfft2 layout
 *   planes : [batch][5][N][N] in the plan's precision: d_x phi, d_y phi,
 *            d_xx phi, d_xy phi, d_yy phi (cmb_lensing/util.py:110-130)
 *
 * Status codes are returned, never raised; nothing aborts or traps.
 */
#ifndef LENSEFLOW_H
#define LENSEFLOW_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum lf_status {
  LF_OK = 0,
  LF_ERR_BAD_SHAPE = 1,
  LF_ERR_BAD_DTYPE = 2,
  LF_ERR_BAD_ARG = 3,
  LF_ERR_SINGULAR_MAGNIFICATION = 4,
  LF_ERR_OOM = 5,
  LF_ERR_TIMEOUT = 6,
  LF_ERR_CUDA = 7,
  LF_ERR_WORKSPACE = 8
};

enum lf_dtype { LF_F32 = 0, LF_F64 = 1 };
enum lf_phi_basis { LF_PHI_MAP = 0, LF_PHI_FOURIER = 1 };

/* Direction constants of cmb_lensing/constants.py:7-8. */
#define LF_FORWARD_LENSE 1
#define LF_INVERSE_LENSE (-1)

typedef struct lf_plan_s* lf_plan_t;

/* Library version (major*10000 + minor*100 + patch). */
int lf_version(void);

/* Human-readable name of a status code (static string). */
const char* lf_status_string(int status);

/* Create a plan for N x N maps with ``ncomp`` components, pixel width
 * ``pix_width`` in radians (fields.py:21, lense_flow.py:291) and compute
 * precision LF_F32 or LF_F64.  N must be one of 64, 128, 256, 512, 1024.
 * Allocates only the plan's twiddle tables on the current device.
 * Replaces the per-call setup of lense_flow (cmb_lensing/lense_flow.py:289-302). */
int lf_plan_create(lf_plan_t* plan, int nside, int ncomp, double pix_width, int precision);
int lf_plan_destroy(lf_plan_t plan);

/* Bytes of caller workspace needed by lf_lense_flow for ``batch`` maps. */
size_t lf_workspace_bytes(lf_plan_t plan, int batch, int adjoint);
/* Workspace with which lf_lense_flow of a float32 plan also precomputes
 * p = M(t)^-1 grad(phi) at the 2 nsteps + 1 RK4 stage times (lense_flow.py:
 * 373-381, :398-415; two planes per time and map) so that every row pass
 * reads two planes per pixel instead of five.  lf_lense_flow takes that path
 * whenever ws_bytes is at least this; with at least lf_workspace_bytes it
 * forms p from the derivative planes in every stage. */
size_t lf_workspace_bytes_n(lf_plan_t plan, int batch, int adjoint, int nsteps);
/* Bytes of the derivative-plane buffer for ``batch`` maps. */
size_t lf_phi_planes_bytes(lf_plan_t plan, int batch);
/* Bytes of float64 scratch needed by lf_phi_precompute for ``batch`` maps. */
size_t lf_phi_workspace_bytes(lf_plan_t plan, int batch);

/* d_x, d_y, d_xx, d_xy, d_yy of phi, computed in float64 and stored in the
 * plan's precision.  Replaces get_primal_derivatives /
 * get_primal_derivatives_from_fourier (cmb_lensing/util.py:110-130) as used
 * by primal_lense_flow (cmb_lensing/lense_flow.py:299-302).
 * If ``min_det`` (device, ``batch`` ints) is non-NULL it receives, per map,
 * min over pixels and t in [0,1] of det(I + t grad grad phi), encoded with
 * lf_decode_min_det; the caller must initialise it with lf_min_det_init. */
int lf_phi_precompute(lf_plan_t plan, const void* phi, int phi_basis, int batch, void* planes, int* min_det,
                      void* workspace, size_t workspace_bytes, void* stream);
int lf_min_det_init(int* min_det, int batch, void* stream);
float lf_decode_min_det(int encoded);

/* The phi precompute with the stage-time p planes formed in the same pass
 * (float32 plans only; LF_ERR_BAD_DTYPE otherwise): pp receives
 * p = M(t)^-1 grad(phi) (lense_flow.py:373-381, :398-415), computed in
 * float32 (the RK4 arithmetic) from the float64 derivatives, at the 2n+1 times
 * k / (2n), k = 0..2n, ascending: [batch][2n+1][2][N][N] (lf_pp_bytes).  One
 * set serves the forward, inverse and adjoint lens with n steps.  ``planes``
 * (optional, NULL to skip) receives the five derivative planes as
 * lf_phi_precompute writes them; ``min_det`` as in lf_phi_precompute.  Every
 * transform is float64; without ``planes`` the derivative spectra between the
 * column and row transforms are stored as float32 (the p planes differ from
 * those of the planes-requested call by float32 rounding, about 1e-7). 
 * Workspace: lf_phi_workspace_bytes.  Replaces get_primal_derivatives
 * (util.py:110-130) plus the per-RHS p computation of the reference. */
size_t lf_pp_bytes(lf_plan_t plan, int batch, int nsteps);
int lf_phi_precompute_pp(lf_plan_t plan, const void* phi, int phi_basis, int batch, void* planes, void* pp, int nsteps,
                         int* min_det, void* workspace, size_t workspace_bytes, void* stream);
/* lf_lense_flow reading precomputed p planes (from lf_phi_precompute_pp with
 * the same nsteps) instead of forming them: float32 plans; workspace of
 * lf_workspace_bytes.  Same results as lf_lense_flow on the p-plane path up
 * to the p planes' rounding (float32 arithmetic on float64 derivatives here,
 * float64 arithmetic on float32 derivative planes there).  Replaces lense_flow (lense_flow.py:289-352) as
 * lf_lense_flow does. */
int lf_lense_flow_pp(lf_plan_t plan, const void* f_in, int in_dtype, void* f_out, int out_dtype, const void* pp,
                     int batch, int nsteps, int direction, int adjoint, void* workspace, size_t workspace_bytes,
                     void* stream);

/* LenseFlow: RK4 with ``nsteps`` fixed steps of df/dt = grad(phi)^T M^-1 grad f
 * (adjoint = 0) or df/dt = div(M^-1 grad(phi) f) (adjoint = 1), time running
 * 0 -> 1 iff (direction == +1) XOR adjoint.  Replaces lense_flow /
 * primal_lense_flow / single_lense_flow_step (cmb_lensing/lense_flow.py:289-352)
 * for all ``ncomp`` components of ``batch`` maps.  f_in may equal f_out.
 * ``in_dtype``/``out_dtype`` select float32/float64 field I/O. */
int lf_lense_flow(lf_plan_t plan, const void* f_in, int in_dtype, void* f_out, int out_dtype, const void* planes,
                  int batch, int nsteps, int direction, int adjoint, void* workspace, size_t workspace_bytes,
                  void* stream);

/* float64 2-D real FFTs in the reference's layout (util.py:113, fields.py:159-172):
 * lf_rfft2: maps [batch][N][N] (float32/float64) -> spec [batch][N][N/2+1]
 * complex128, unnormalised (jnp.fft.rfft2).  lf_irfft2: spec -> maps,
 * 1/N^2 normalised, imaginary parts of the DC/Nyquist columns ignored after
 * the column transform (jnp.fft.irfft2).  lf_irfft2 needs
 * lf_fft_workspace_bytes of scratch.  Replace the rfft2/irfft2 calls of
 * fields.py:159-172 (map, fourier) and fields.py:147-154 (undo_inner_product). */
size_t lf_fft_workspace_bytes(lf_plan_t plan, int batch);
int lf_rfft2(lf_plan_t plan, const void* maps, int in_dtype, int batch, void* spec, void* stream);
int lf_irfft2(lf_plan_t plan, const void* spec, int batch, void* maps, int out_dtype, void* workspace,
              size_t workspace_bytes, void* stream);

/* Reverse-mode derivative of lf_lense_flow in the reference's scheme
 * (lense_flow_backwards / get_lensing_operator_gradients /
 * lensing_gradients_integration_step / get_delta_phi_tqu_roc,
 * cmb_lensing/lense_flow.py:23-126, :156-252): from the lensed field
 * ``f_lensed`` and the cotangent, integrate (f, delta_f, delta_phi) with RK4
 * in the opposite time direction.  Outputs: ``delta_f`` [batch][ncomp][N][N]
 * (before undo_inner_product), optional ``f_back`` (the re-integrated field),
 * and ``dphi``: [batch][N][N/2+1] complex128 if dphi_basis = LF_PHI_FOURIER
 * (accumulated in Fourier space, lense_flow.py:233-239) or [batch][N][N]
 * float64 if LF_PHI_MAP (lense_flow.py:240-248). */
size_t lf_vjp_workspace_bytes(lf_plan_t plan, int batch);
int lf_lense_flow_vjp(lf_plan_t plan, const void* f_lensed, const void* cotangent, int io_dtype, const void* planes,
                      int batch, int nsteps, int direction, void* delta_f, void* f_back, void* dphi, int dphi_basis,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Per-mode products of Fourier-diagonal C x C operators with fields, as the
 * Wiener filter's operator applies them (the products of
 * matrix_operators.py:54-141 and the EB<->QU rotations of util.py:140-161,
 * composed per mode):  out[b][i][m] = scale * sum_j W[b][i][j][m] X[b][j][m]
 * + yscale * Y[b][i][m].  W: real float64 [batch or 1][ncomp][ncomp][modes]
 * (w_batched = 0 broadcasts one operator); X, Y, out: complex128
 * [batch][ncomp][modes] (interleaved re, im); Y may be NULL.  Bit i*ncomp+j
 * of ``nonzero`` marks the blocks of W that are not identically zero (the
 * others are skipped).  out may alias X or Y. */
int lf_modes_apply(const void* W, int w_batched, unsigned nonzero, const void* X, const void* Y, void* out, int batch,
                   int ncomp, long modes, double scale, double yscale, void* stream);

/* Checkpointed exact reverse pass: the transpose of the discrete forward map
 * f -> L(phi) f that lf_lense_flow computes (direction +1 or -1, standard
 * RHS), for the cotangent ``cotangent`` and the UNLENSED field ``f_in`` -- the
 * residuals of the reference's custom VJP include f (lense_flow.py:10-51).
 * The forward integration stores one checkpoint (the field at the start of
 * every RK4 step) in the workspace; backwards, each step is recomputed from
 * its checkpoint and one RK4 step of the adjoint RHS carries the cotangent
 * over it, with delta-phi accumulated from the recomputed forward stage
 * inputs.  delta_f equals the reference's (the adjoint lens is already the
 * exact transpose); delta_phi is the exact gradient of the discrete map,
 * where the reference's reverse ODE (lf_lense_flow_vjp) differs from it by the
 * RK4 discretisation error.  Same conventions and layouts as
 * lf_lense_flow_vjp; ``f_out`` (optional) receives L(phi) f_in.  Extends the
 * reference's lense_flow_backwards (lense_flow.py:23-46); the reference has
 * no checkpointed scheme. */
size_t lf_vjp_ckpt_workspace_bytes(lf_plan_t plan, int batch, int nsteps);
int lf_lense_flow_vjp_ckpt(lf_plan_t plan, const void* f_in, const void* cotangent, int io_dtype, const void* planes,
                           int batch, int nsteps, int direction, void* f_out, void* delta_f, void* dphi, int dphi_basis,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free variant of lf_lense_flow (float32 compute), for callers
 * that cannot allocate device memory: a host framework that has already
 * reserved (nearly) all of the GPU's memory for its own pool, where one more
 * cudaMalloc can fail, and latency-critical loops where cudaMalloc/cudaFree
 * would synchronise the device.  No counterpart in the reference.
 * The caller passes the inputs and the output; there is no plan: the
 * geometry is passed directly.  ``planes`` must be the float32 derivative
 * planes [batch][5][N][N] that lf_phi_precompute wrote for a plan created
 * with LF_F32 and the same N and pix_width (the computation is float32; the
 * planes of a float64 plan would be misread).  Scratch lives in a file-scope device array of
 * LF_NOALLOC_SCRATCH_BYTES that every GPU which loads the library holds until
 * exit; a call needing more (4 bytes x N^2 x batch x ncomp x (4, or 5 when
 * adjoint)) returns LF_ERR_WORKSPACE (nsteps = 0 needs none: it copies the
 * input, as lf_lense_flow does).  The first call on each device resolves
 * the array's device address and fills twiddle tables with a synchronous
 * copy: make that first call before any stream capture.  Every call shares
 * the one array, so calls that overlap on the GPU (other streams, other host
 * threads) race; serialise them.  No scratch element needs to start at zero:
 * each is written before it is read within a call. */
#define LF_NOALLOC_SCRATCH_BYTES (24u * 1024u * 1024u)
int lf_lense_flow_noalloc(int nside, int ncomp, double pix_width, const void* f_in, int in_dtype, void* f_out,
                          int out_dtype, const void* planes, int batch, int nsteps, int direction, int adjoint,
                          void* stream);

/* Device-wait timeouts.  Every wait of a kernel block on its own bulk copies
 * into shared memory is bounded (about one second of polls).  A block whose
 * wait runs out records it, waits once more (bounded) for its copies in
 * flight and then skips or finishes its work: the results of that launch and
 * of everything computed from them are invalid.  The record is sticky: from
 * then on every computing entry point (lf_phi_precompute, lf_lense_flow,
 * lf_lense_flow_vjp, lf_rfft2, lf_irfft2, lf_lense_flow_noalloc) returns
 * LF_ERR_TIMEOUT without launching anything, until lf_wait_timeouts resets
 * it.  Because calls are asynchronous, the call whose kernels timed out has
 * usually returned LF_OK already; the next call, lf_timeout_status after the
 * caller has synchronised with the work, or lf_stream_check reports it.  (If
 * the second wait also ran out, the block may have exited with copies into
 * its shared memory still in flight; every result until the reset is
 * invalid in that case too.)  No counterpart in the reference (its XLA path
 * has no device-side waits).
 *
 * lf_wait_timeouts: synchronises the current device, sets *count to 1 if a
 * timeout was recorded (else 0) and, with reset != 0, clears the record.
 * lf_timeout_status: LF_ERR_TIMEOUT if a timeout has been recorded, else
 * LF_OK; no synchronisation (exact once the caller has synchronised with the
 * work in question).  The record lives in one mapped pinned host word that
 * lf_plan_create sets up; without a plan only lf_wait_timeouts and
 * lf_stream_check see timeouts.
 * lf_stream_check: synchronises ``stream`` and returns LF_ERR_TIMEOUT,
 * LF_ERR_CUDA (a failed launch or fault) or LF_OK.
 * lf_set_wait_polls: a test hook that sets the poll limit of every block's
 * first wait on the current device (polls < 0 restores the default).  With 0
 * the first wait runs out at once while the copies are still legitimately in
 * flight; the drain wait keeps its full limit, so nothing waits forever and
 * every copy lands before its block moves on.  Synchronises the device. */
int lf_wait_timeouts(int* count, int reset);
int lf_timeout_status(void);
int lf_stream_check(void* stream);
int lf_set_wait_polls(int polls);

/* Launch timing for benchmarks and profiling.  While enabled, every kernel
 * launched through ``plan`` is bracketed by a CUDA event pair on its stream.
 * lf_profile_read synchronises on the last event and returns the summed
 * duration and count of the recorded launches of one kind.  No counterpart
 * in the reference (its device work is XLA-generated). */

enum lf_kernel_kind { LF_KIND_ROW = 0, LF_KIND_COL = 1, LF_KIND_PHI = 2, LF_KIND_PP = 3 };
int lf_profile_enable(lf_plan_t plan, int enable);
int lf_profile_reset(lf_plan_t plan);
int lf_profile_read(lf_plan_t plan, int kind, double* total_ms, int* launches);

#ifdef __cplusplus
}
#endif

#endif /* LENSEFLOW_H */
