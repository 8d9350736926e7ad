// LenseFlow kernels: phi-derivative precompute and the two passes of one RK4 stage.
//
// Spectral conventions follow the reference exactly (cmb_lensing/util.py:103-137):
// KX = 2 pi fftfreq(N, d) on axis 0 ("columns" here), KY = 2 pi rfftfreq(N, d)
// on axis 1 ("rows") with the Nyquist entry negated, and every derivative is
// irfft2(multiplier * rfft2(.)), whose inverse real transform ignores the
// imaginary parts of the DC/Nyquist bins of axis 1.
//
// Row-spectral arrays ("S", "U", "V", "Gx") hold, for every map row, the
// packed half spectrum of that row only (axis-1 transform done, axis 0 not):
// N/2 complex values, slot 0 = (X[0], X[N/2]).  Their N/2 columns are the
// "lines" of the column pass.  Column 0 -- the packed pair of real sequences
// X[.,0] and X[.,N/2] -- is transformed as one complex line; multiplying it
// by the Hermitian-symmetrised multiplier i*KX (zero at KX's Nyquist row)
// reproduces exactly the real parts that irfft2 keeps for those two columns.
//
// d/dx (axis 0) needs the column pass; d/dy (axis 1) is row-local:
// irfft2(i KY rfft2 f) == per-row irfft(i KY rfft f) because the axis-0
// transforms cancel.  So one RK4 stage is one column pass + one row pass.
#pragma once

#include "lf_fft.cuh"

namespace lf {

// ----------------------------------------------------------- parameters
struct StageArgs {
  // field I/O (caller dtype: io_f64 ? double : float), [B][C][N][N]
  const void* f_in;
  void* f_out;
  int in_f64, out_f64;
  // phi derivative planes, [B][5][N][N] of T: phi_x, phi_y, phi_xx, phi_xy, phi_yy
  const void* phi;
  // workspace, each [B*C][N*N] T values
  void* y0;
  void* acc;
  void* s;   // standard: rfft_rows(y_s);   adjoint: U = rfft_rows(p_x y_s)
  void* v;   // adjoint: V = rfft_rows(p_y y_s)
  void* gx;  // column pass output
  const void* twN;  // N complex T, exp(-2 pi i k / N)
  const void* twP;  // pass table of length N (ptw_size(N) complex T): column pass, paired row pass
  const void* twC;  // column table of the two-pass column plan (ctw_size(N) complex T; N = 512)
  double kbase;     // 2 pi / (N d)
  double t_cur;     // time of the rate evaluated in this stage
  double t_next;    // time of the next stage input
  double h;         // signed step
  int stage;        // 1..4 (0 = init)
  int last;         // final stage of the integration
  int nplanes;      // B*C (column pass)
  // reverse-mode (VJP) extras
  void* grad;       // standard pass with SAVE: d_x y_s, d_y y_s, [B*C][2][N][N] T
  void* dsave;      // adjoint pass with SAVE: next stage input, [B*C][N][N] T
  // p = M(t)^-1 grad(phi) at the 2n+1 stage times t0 + k h/2 (row pass with PP):
  // [B][pp_k][2][N][N] T; this stage reads time index pp_idx
  const void* pp;
  int pp_k;
  int pp_idx;
};

// p = M(t)^-1 grad(phi) with M = I + t grad grad phi (lense_flow.py:373-381, :398-415)
template <typename T>
__device__ __forceinline__ void p_vector(T px, T py, T pxx, T pxy, T pyy, T t, T& ox, T& oy) {
  const T mxx = T(1) + t * pxx, mxy = t * pxy, myy = T(1) + t * pyy;
  const T inv = T(1) / (mxx * myy - mxy * mxy + T(1e-12));
  const T ixx = myy * inv, ixy = -mxy * inv, iyy = mxx * inv;
  ox = px * ixx + py * ixy;
  oy = px * ixy + py * iyy;
}

template <typename T>
__device__ __forceinline__ c2<T> load_io(const void* p, int f64, long i) {
  if (f64) {
    const double2 v = reinterpret_cast<const double2*>(p)[i];
    return mk<T>(T(v.x), T(v.y));
  }
  const float2 v = reinterpret_cast<const float2*>(p)[i];
  return mk<T>(T(v.x), T(v.y));
}

template <typename T>
__device__ __forceinline__ void store_io(void* p, int f64, long i, c2<T> v) {
  if (f64) {
    reinterpret_cast<double2*>(p)[i] = make_double2(double(v.x), double(v.y));
  } else {
    reinterpret_cast<float2*>(p)[i] = make_float2(float(v.x), float(v.y));
  }
}

// Two consecutive packed elements: one 16-byte access for float32.
template <typename T>
__device__ __forceinline__ void ld2(const c2<T>* p, c2<T>* v) {
  if constexpr (sizeof(c2<T>) == 8) {
    const float4 w = *reinterpret_cast<const float4*>(p);
    v[0] = mk<T>(T(w.x), T(w.y));
    v[1] = mk<T>(T(w.z), T(w.w));
  } else {
    v[0] = p[0];
    v[1] = p[1];
  }
}

template <typename T>
__device__ __forceinline__ void st2(c2<T>* p, const c2<T>* v) {
  if constexpr (sizeof(c2<T>) == 8) {
    *reinterpret_cast<float4*>(p) = make_float4(float(v[0].x), float(v[0].y), float(v[1].x), float(v[1].y));
  } else {
    p[0] = v[0];
    p[1] = v[1];
  }
}

template <typename T, int N, int NT>
__device__ __forceinline__ void load_twiddles(c2<T>* tw, const void* g, int tid) {
  const c2<T>* src = reinterpret_cast<const c2<T>*>(g);
  for (int i = tid; i < N; i += NT) tw[i] = src[i];
}

// Programmatic dependent launch.  A stage kernel lets the next kernel of the
// stream launch once all its blocks are running (its blocks then fill SMs as
// this grid drains), and waits for the previous kernel to complete, with its
// memory visible, before touching any buffer the two share.  Without the
// launch attribute both are no-ops.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// shared-memory entries reserved for the column pass's twiddle table (rounded
// up to an even count so that the tile after it stays 16-byte aligned); TWO:
// the column table of the two-pass plan
__host__ __device__ constexpr int col_tw_entries(int n, bool two = false) {
  return ((two ? ctw_size(n) : ptw_size(n)) + 1) & ~1;
}

// ============================================ bulk copies and bounded waits
constexpr int kWaitTries = 1 << 20;  // polls of a bounded wait: about one second

// Set (never cleared by the kernels) when a block gave up waiting for its
// bulk copies; the host reads it with lf_wait_timeouts().
__device__ int g_lf_wait_timeouts;
// Polls of a block's first wait on its bulk copies.  lf_set_wait_polls lowers
// it (a test hook) so that the first wait runs out while the copies are still
// legitimately in flight; the drain wait that follows always polls kWaitTries.
__device__ int g_lf_wait_polls = kWaitTries;
// Mapped pinned host word (set up per device by lf_plan_create, else null):
// a timed-out block also sets it, so that every later entry point can report
// LF_ERR_TIMEOUT without synchronising the device.
__device__ int* g_lf_timeout_host;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
  // make the initialised barrier visible to the bulk-copy (async) proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
               : "memory");
}

// One contiguous global -> shared copy of ``bytes`` (16-byte aligned, multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(mbar))
      : "memory");
}

// Wait for phase ``parity`` of the barrier, giving up after ``tries`` polls;
// each poll suspends for at most about 1 microsecond (the explicit time hint),
// so a wait is bounded by roughly tries microseconds.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, int tries) {
  const uint32_t addr = smem_addr(mbar);
  for (int i = 0; i < tries; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(addr), "r"(parity), "r"(1000u)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Record that a block stopped waiting: the device flag and, when set up, the
// mapped host word (a plain store made visible system-wide; host-memory
// atomics are not available over every interconnect).  Only the thread that
// flips the device flag writes the host word, so a launch whose every block
// times out sends one write over the interconnect, not one per thread.
__device__ __forceinline__ void record_timeout() {
  if (atomicExch(&g_lf_wait_timeouts, 1) != 0) return;
  int* h = g_lf_timeout_host;
  if (h) {
    *reinterpret_cast<volatile int*>(h) = 1;
    __threadfence_system();
  }
}

// Wait for phase ``parity``.  If the first bounded wait (g_lf_wait_polls
// polls) runs out, record the timeout -- this launch's results are then
// invalid -- and wait once more, bounded by kWaitTries polls, for the copies
// still in flight, so that they land before the block moves on or exits.
// Returns whether the first wait succeeded.
__device__ __forceinline__ bool wait_or_record(uint64_t* mbar, uint32_t parity) {
  if (mbar_wait(mbar, parity, g_lf_wait_polls)) return true;
  record_timeout();
  mbar_wait(mbar, parity, kWaitTries);
  return false;
}

// ======================================================== column pass
// Gx = IFFT_col( (i KX / N^2) * FFT_col(S) ) on tiles of LINES columns.
// grid: x = column tile (N/2/LINES), y = plane.  TWO: the plan N = 16 x 32
// (one shared-memory round trip per direction) instead of 8 x 8 x 8.
template <typename T, int N, int LINES, int NT, int MINB = 1, bool TWO = false>
__global__ void __launch_bounds__(NT, MINB) k_col(StageArgs a) {
  constexpr int H = N / 2;
  static_assert(!TWO || col2_plan(N), "no two-pass column plan for this length");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c2<T>* tw = reinterpret_cast<c2<T>*>(smem_raw);  // pass table or column table
  c2<T>* buf = tw + col_tw_entries(N, TWO);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + LINES * N);  // 16 bytes reserved after the tile
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * LINES;
  // planes in reverse launch order: the row pass before this one wrote S map by map in forward order, so
  // the last planes are still in L2 when this pass starts on them, and the first planes' Gx (and S) are
  // the freshest in L2 when the next row pass starts on map 0 (row passes 4.55 -> 4.45 ms, column passes
  // 1.90 -> 1.86 ms per 64-map 512^2 QU step, identical outputs)
  const long plane = gridDim.y - 1 - blockIdx.y;
  static_assert(H % LINES == 0, "column tiles must cover the packed spectrum");
  constexpr int NTW = TWO ? ctw_size(N) : ptw_size(N);
  static_assert(NTW * sizeof(c2<T>) % 16 == 0, "twiddle table: one bulk copy");
  pdl_launch_dependents();
  if (tid == 0) {  // the table by one bulk copy; the first pass, which reads none of it, runs meanwhile
    mbar_init(mbar, 1);
    mbar_expect_tx(mbar, uint32_t(NTW * sizeof(c2<T>)));
    bulk_g2s(tw, TWO ? a.twC : a.twP, NTW * sizeof(c2<T>), mbar);
  }
  pdl_wait();
  // after the first pass's barrier (which also orders the barrier's init before the waits)
  // (a timed-out table wait is recorded; the block goes on to its remaining barriers)
  auto wait_table = [=]() { wait_or_record(mbar, 0); };
  const c2<T>* in = reinterpret_cast<const c2<T>*>(a.s) + plane * (long)N * H + c0;
  c2<T>* out = reinterpret_cast<c2<T>*>(a.gx) + plane * (long)N * H + c0;
  // i KX / N^2 between the transforms; zero on KX's Nyquist row of the packed
  // DC/Nyquist line (column 0)
  const T scale = T(a.kbase / (double(N) * double(N)));
  auto kx_mul = [=](int m, int line, c2<T> v) {
    const int kx = (m < N / 2) ? m : m - N;
    const T f = (c0 + line == 0 && m == N / 2) ? T(0) : scale * T(kx);
    return mk<T>(-f * v.y, f * v.x);
  };
  // rows of LINES consecutive columns: each warp's accesses cover whole 128-byte lines
  auto src = [=](int m, int line) { return in[m * H + line]; };
  auto dst = [=](int m, int line, c2<T> x) { out[m * H + line] = x; };
  if constexpr (TWO)
    fft_mul_ifft_2p<T, N, col2_r1(N), col2_r2(N), LINES, NT>(buf, tw, tw + ctw_inv_offset(N), tid, src, kx_mul, dst,
                                                           wait_table);
  else
    fft_mul_ifft<T, N, LINES, NT>(buf, tw, tid, src, kx_mul, dst, wait_table);
}

// ========================================================= row pass
// One tile = LINES consecutive rows of one map, all C components at once, so
// each phi pixel is read once per stage and applied to every component.
// Shared memory holds 2C tiles: the "primary" tiles 0..C-1 and the
// "secondary" tiles C..2C-1.
// Standard RHS (lense_flow.py:365-370):  k = p_x d_x y + p_y d_y y
//   primary = Gx (column pass of S) -> d_x y;  secondary = S -> i KY S -> d_y y
// Adjoint RHS (lense_flow.py:355-362):   k = d_x(p_x y) + d_y(p_y y)
//   primary = Gx + i KY V (one inverse transform);  secondary = V
// RK4 (util.py:184-199): stages 1..3 accumulate k1 + 2 k2 + 2 k3 and form the
// next stage input; stage 4 forms y0 + h/6 (acc + k4).
// STAGE0: initialisation (copy the input field, transform the first stage
// input), no rate.  SAVE (reverse mode): the standard pass also stores
// d_x y_s and d_y y_s; the adjoint pass stores its next stage input.
// PP: p at the stage time is read from the precomputed p planes (two loads per
// pixel) instead of being formed from the five derivative planes.
template <typename T, int N, int C, bool ADJ, bool STAGE0, int LINES, int NT, bool SAVE = false, int MINB = 1,
          bool PP = false>
__global__ void __launch_bounds__(NT, MINB) k_row(StageArgs a) {
  constexpr int H = N / 2;
  constexpr long P = (long)N * N;
  constexpr int TILE = LINES * H;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c2<T>* tw = reinterpret_cast<c2<T>*>(smem_raw);
  c2<T>* buf = tw + N;  // tile t at buf + t * TILE
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * LINES;
  const long map = blockIdx.y;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + 2 * C * TILE);  // 16 bytes reserved after the tiles
  static_assert(N * sizeof(c2<T>) % 16 == 0, "twiddle table: one bulk copy");
  pdl_launch_dependents();
  if (tid == 0) {  // the table by one bulk copy while the rows load
    mbar_init(mbar, 1);
    mbar_expect_tx(mbar, uint32_t(N * sizeof(c2<T>)));
    bulk_g2s(tw, a.twN, N * sizeof(c2<T>), mbar);
  }
  pdl_wait();
  // after the barrier that follows the row loads (it also orders the init before the waits)
  // (a timed-out table wait is recorded; the block goes on to its remaining barriers)
  auto wait_table = [=]() { wait_or_record(mbar, 0); };
  const T* phi = reinterpret_cast<const T*>(a.phi) + map * 5 * P + (long)r0 * N;
  const T tnext = T(a.t_next);
  const T tcur = T(a.t_cur);
  const T hh = T(a.h);
  const T ky_scale = T(a.kbase / double(N));
  const long half_plane = N * (long)H;  // complex elements per row-spectral plane
  auto spec = [&](void* base, int c) {
    return reinterpret_cast<c2<T>*>(base) + (map * C + c) * half_plane + (long)r0 * H;
  };
  auto real_rows = [&](void* base, int c) {
    return reinterpret_cast<c2<T>*>(reinterpret_cast<T*>(base) + (map * C + c) * P + (long)r0 * N);
  };

  // --------------------------------------------------------------- inputs
  if constexpr (!STAGE0) {
#pragma unroll
    for (int c = 0; c < C; ++c) {
      load_rows<T, c2<T>, H, LINES, NT>(buf + c * TILE, spec(a.gx, c), H, tid);
      load_rows<T, c2<T>, H, LINES, NT>(buf + (C + c) * TILE, spec(ADJ ? a.v : a.s, c), H, tid);
    }
    __syncthreads();
    wait_table();
    // d_y in the row spectrum: i KY / N, folded into the pre-pass of the
    // inverse real transform (KY's DC and Nyquist bins contribute nothing
    // after it, so the (X0, XH) slot of a d_y spectrum is zero).
    auto dy = [=](const c2<T> w, int kk) {
      const T f = ky_scale * T(kk);
      return (kk == 0) ? mk<T>(T(0), T(0)) : mk<T>(-f * w.y, f * w.x);
    };
    constexpr int NTI = ADJ ? C : 2 * C;
    if constexpr (ADJ) {
      // primary = Gx + i KY V / N: one inverse transform per component
      auto in = [=](int tile, int kk, int row, c2<T> g) {
        return (kk == 0) ? g : cadd<T>(g, dy(buf[(C + tile) * TILE + sw<T, LINES>(kk, row)], kk));
      };
      c2r_pre<T, H, LINES, NTI, NT>(buf, tw, tid, in);
    } else {
      auto in = [=](int tile, int kk, int, c2<T> w) { return tile < C ? w : dy(w, kk); };
      c2r_pre<T, H, LINES, NTI, NT>(buf, tw, tid, in);
    }
    fft_tiles<T, H, LINES, NTI, NT, true, N>(buf, tw, tid);
  } else {
    for (int idx = tid; idx < H * LINES * C; idx += NT) {
      const int c = idx / (H * LINES), rem = idx % (H * LINES);
      const int row = rem / H, m = rem % H;
      const long fo = (map * C + c) * (P / 2) + (long)r0 * H + (long)row * H + m;
      buf[c * TILE + sw<T, LINES>(m, row)] = load_io<T>(a.f_in, a.in_f64, fo);
    }
    __syncthreads();
    wait_table();
  }

  // ---------------------------------------------------- pointwise epilogue
  // Two packed elements (four pixels) per iteration; phi once for all C.
  constexpr int E2 = H / 2;
  const bool live = STAGE0 || !a.last;  // a next stage input is formed
#pragma unroll 1
  for (int idx = tid; idx < E2 * LINES; idx += NT) {
    const int row = idx / E2, m0 = 2 * (idx % E2);
    const long e0 = (long)row * H + m0;  // packed-element index within the tile
    const bool need_phi = STAGE0 ? ADJ : (!ADJ || live);
    // p at the rate time (standard) and at the next stage time (adjoint)
    T prx[2][2], pry[2][2];
    if (need_phi) {
      if constexpr (PP) {
        const T* pp = reinterpret_cast<const T*>(a.pp) + (map * a.pp_k + a.pp_idx) * 2 * P + (long)r0 * N;
        c2<T> px[2], py[2];
        ld2<T>(reinterpret_cast<const c2<T>*>(pp) + e0, px);
        ld2<T>(reinterpret_cast<const c2<T>*>(pp + P) + e0, py);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          prx[q][0] = px[q].x;
          prx[q][1] = px[q].y;
          pry[q][0] = py[q].x;
          pry[q][1] = py[q].y;
        }
      } else {
        c2<T> fx[2], fy[2], fxx[2], fxy[2], fyy[2];
        ld2<T>(reinterpret_cast<const c2<T>*>(phi) + e0, fx);
        ld2<T>(reinterpret_cast<const c2<T>*>(phi + P) + e0, fy);
        ld2<T>(reinterpret_cast<const c2<T>*>(phi + 2 * P) + e0, fxx);
        ld2<T>(reinterpret_cast<const c2<T>*>(phi + 3 * P) + e0, fxy);
        ld2<T>(reinterpret_cast<const c2<T>*>(phi + 4 * P) + e0, fyy);
        const T tp = ADJ ? tnext : tcur;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          p_vector<T>(fx[q].x, fy[q].x, fxx[q].x, fxy[q].x, fyy[q].x, tp, prx[q][0], pry[q][0]);
          p_vector<T>(fx[q].y, fy[q].y, fxx[q].y, fxy[q].y, fyy[q].y, tp, prx[q][1], pry[q][1]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < C; ++c) {
      c2<T>* pri = buf + c * TILE;
      c2<T>* sec = buf + (C + c) * TILE;
      c2<T>* y0g = real_rows(a.y0, c);
      c2<T>* accg = real_rows(a.acc, c);
      c2<T> ynext[2];
      if constexpr (STAGE0) {
        ynext[0] = pri[sw<T, LINES>(m0, row)];
        ynext[1] = pri[sw<T, LINES>(m0 + 1, row)];
        st2<T>(y0g + e0, ynext);
      } else {
        c2<T> k[2], g0[2], g1[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          g0[q] = pri[sw<T, LINES>(m0 + q, row)];
          if constexpr (ADJ) {
            k[q] = g0[q];
          } else {
            g1[q] = sec[sw<T, LINES>(m0 + q, row)];
            k[q] = mk<T>(prx[q][0] * g0[q].x + pry[q][0] * g1[q].x, prx[q][1] * g0[q].y + pry[q][1] * g1[q].y);
          }
        }
        if constexpr (SAVE && !ADJ) {
          c2<T>* gs = reinterpret_cast<c2<T>*>(reinterpret_cast<T*>(a.grad) + (map * C + c) * 2 * P + (long)r0 * N);
          st2<T>(gs + e0, g0);
          st2<T>(gs + P / 2 + e0, g1);
        }
        c2<T> y0[2], ac[2];
        ld2<T>(y0g + e0, y0);
        if (a.stage > 1) ld2<T>(accg + e0, ac);
        if (a.stage == 1) {
#pragma unroll
          for (int q = 0; q < 2; ++q)
            ynext[q] = mk<T>(y0[q].x + T(0.5) * hh * k[q].x, y0[q].y + T(0.5) * hh * k[q].y);
          st2<T>(accg + e0, k);
        } else if (a.stage < 4) {
          const T cc = a.stage == 2 ? T(0.5) * hh : hh;
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            ynext[q] = mk<T>(y0[q].x + cc * k[q].x, y0[q].y + cc * k[q].y);
            ac[q] = mk<T>(ac[q].x + T(2) * k[q].x, ac[q].y + T(2) * k[q].y);
          }
          st2<T>(accg + e0, ac);
        } else {
          const T h6 = hh / T(6);
#pragma unroll
          for (int q = 0; q < 2; ++q)
            ynext[q] = mk<T>(y0[q].x + h6 * (ac[q].x + k[q].x), y0[q].y + h6 * (ac[q].y + k[q].y));
          if (a.last) {
            const long fo = (map * C + c) * (P / 2) + (long)r0 * H + e0;
            store_io<T>(a.f_out, a.out_f64, fo, ynext[0]);
            store_io<T>(a.f_out, a.out_f64, fo + 1, ynext[1]);
          } else {
            st2<T>(y0g + e0, ynext);
          }
        }
      }
      if constexpr (SAVE && ADJ) {
        if (live) st2<T>(real_rows(a.dsave, c) + e0, ynext);
      }
      if (live) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if constexpr (ADJ) {
            pri[sw<T, LINES>(m0 + q, row)] = mk<T>(prx[q][0] * ynext[q].x, prx[q][1] * ynext[q].y);
            sec[sw<T, LINES>(m0 + q, row)] = mk<T>(pry[q][0] * ynext[q].x, pry[q][1] * ynext[q].y);
          } else {
            pri[sw<T, LINES>(m0 + q, row)] = ynext[q];
          }
        }
      }
    }
  }
  if (!STAGE0 && a.last) return;  // uniform across the block
  __syncthreads();
  // ------------------------------------------------ next stage's spectra
  constexpr int NTO = ADJ ? 2 * C : C;
  fft_tiles<T, H, LINES, NTO, NT, false, N>(buf, tw, tid);
  r2c_post<T, H, LINES, NTO, NT>(buf, tw, tid);
#pragma unroll
  for (int c = 0; c < C; ++c) {
    store_rows<T, c2<T>, H, LINES, NT>(spec(a.s, c), H, buf + c * TILE, tid);
    if constexpr (ADJ) store_rows<T, c2<T>, H, LINES, NT>(spec(a.v, c), H, buf + (C + c) * TILE, tid);
  }
}

// ============================================ row pass, component pairs
// Standard RHS for two components (Q, U) with the p planes, N = 512, FP32.
// The general row pass inverse-transforms four packed half spectra per row
// (d_x and d_y of both components) and forward-transforms two, each as a
// half-length complex FFT with a real-FFT pre/post pass in shared memory.
// Here each component's two Hermitian derivative spectra are combined into
// one full-length spectrum Z = DX + i DY, whose inverse FFT is dx + i dy;
// after the RK4 update the two next stage inputs are combined into
// w = y_0 + i y_1, whose forward FFT W gives both packed row spectra:
// S_0[k] = (W[k] + conj W[N-k]) / 2, S_1[k] = (W[k] - conj W[N-k]) / 2i.
// The Hermitian expansion and the split are local in k, so they happen in the
// 16-byte global load and store phases, and the inverse transform's last
// radix-8 pass, the pointwise update and the forward transform's first pass
// run in registers: both passes see x[j + 64 r] of one row in one thread.
// The update's operands y0 and acc (the tile's rows: contiguous blocks) are
// fetched into shared memory by bulk copies issued at the start, and each
// thread loads its pixels' p_x, p_y into registers, so their latency overlaps
// the loads and the first inverse passes.
template <int LINES>
constexpr size_t row_pair_smem_bytes(int n) {  // paired row passes: p_x, p_y in registers, four staged planes
  return sizeof(float2) * (n + 2 * LINES * n) + sizeof(float) * 4 * LINES * n + 16;
}

template <int N, int LINES, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_row_pair(StageArgs a) {
  using T = float;
  constexpr int H = N / 2;
  constexpr long P = (long)N * N;
  constexpr int R = 8, NB = N / R;  // radix-8 passes: NB butterflies per row
  static_assert(N == 512, "three radix-8 passes");
  static_assert(NB * LINES == NT, "one (row, butterfly) per thread in the fused passes");
  constexpr int TILE = LINES * N;
  constexpr int RB = LINES * N;  // floats per staged row block
  constexpr int IT = 2 * LINES * (H / 2) / NT;  // packed element pairs per thread in the load phase
  static_assert(2 * LINES * (H / 2) % NT == 0, "whole load-phase iterations");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c2<T>* tw = reinterpret_cast<c2<T>*>(smem_raw);
  c2<T>* buf = tw + N;                                 // tile c at buf + c * TILE
  T* stg = reinterpret_cast<T*>(buf + 2 * TILE);       // y0_0, y0_1, acc_0, acc_1
  uint64_t* mbar = reinterpret_cast<uint64_t*>(stg + 4 * RB);  // [0]: staged update operands, [1]: spectra
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * LINES;
  const long map = blockIdx.y;
  const long prow0 = (long)r0 * N;
  const bool with_acc = a.stage > 1;
  const long half_plane = N * (long)H;
  auto spec = [&](void* base, int c) {
    return reinterpret_cast<c2<T>*>(base) + (map * 2 + c) * half_plane + (long)r0 * H;
  };
  static_assert(ptw_size(N) <= N && ptw_size(N) * sizeof(c2<T>) % 16 == 0, "pass table: one bulk copy");
  pdl_launch_dependents();
  if (tid == 0) {
    mbar_init(mbar, 1);
    mbar_init(mbar + 1, 1);
    // the pass table and the spectra first (the transforms wait for them)
    mbar_expect_tx(mbar + 1, uint32_t(ptw_size(N) * sizeof(c2<T>) + 4 * LINES * H * sizeof(c2<T>)));
    bulk_g2s(tw, a.twP, ptw_size(N) * sizeof(c2<T>), mbar + 1);
    pdl_wait();  // the other copies read what the previous kernel wrote
    // Gx_c and S_c rows, packed, into tile c
    for (int c = 0; c < 2; ++c) {
      bulk_g2s(buf + c * TILE, spec(a.gx, c), LINES * H * sizeof(c2<T>), mbar + 1);
      bulk_g2s(buf + c * TILE + LINES * H, spec(a.s, c), LINES * H * sizeof(c2<T>), mbar + 1);
    }
    mbar_expect_tx(mbar, uint32_t((with_acc ? 4 : 2) * RB * sizeof(T)));
    for (int c = 0; c < 2; ++c) {
      bulk_g2s(stg + c * RB, reinterpret_cast<const T*>(a.y0) + (map * 2 + c) * P + prow0, RB * sizeof(T), mbar);
      if (with_acc)
        bulk_g2s(stg + (2 + c) * RB, reinterpret_cast<const T*>(a.acc) + (map * 2 + c) * P + prow0, RB * sizeof(T),
                 mbar);
    }
  }
  pdl_wait();  // every thread, before its own global reads and writes
  // p_x, p_y of the thread's 8 update pixels straight into registers (coalesced; their latency hides under
  // the transforms): without their staging a block needs 36.9 instead of 45.1 KB of shared memory, so six
  // blocks fit on an SM instead of five (row passes 4.51-4.53 -> 4.48-4.49 ms per 64-map step)
  T preg[2][R];
  {
    const T* pq = reinterpret_cast<const T*>(a.pp) + (map * a.pp_k + a.pp_idx) * 2 * P + prow0 + (tid / NB) * N +
                  tid % NB;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      preg[0][r] = __ldg(pq + NB * r);
      preg[1][r] = __ldg(pq + P + NB * r);
    }
  }
  constexpr int O8 = ptw_offset(N, R, R), O64 = ptw_offset(N, R, R * R);
  const T ky_scale = T(a.kbase / double(N));
  __syncthreads();  // barriers initialised before anyone waits on them
  // the pass table and spectra: a timed-out wait is recorded and the block goes
  // on, so that every thread meets every barrier below
  wait_or_record(mbar + 1, 0);

  // ------------------------- load: Z_c = DX_c + i DY_c with DY = i KY S / N
  // (slot 0 of a packed spectrum holds the real DC and Nyquist bins; the d_y
  // spectrum has none: KY's DC and Nyquist terms vanish after irfft).  The
  // packed rows sit in tile c; all of them are read before Z overwrites it.
  c2<T> gv[IT][2], sv[IT][2];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * NT;
    const int t = idx % (H / 2), rest = idx / (H / 2);
    const int row = rest % LINES, c = rest / LINES;
    const c2<T>* pk = buf + c * TILE;
    ld2<T>(pk + row * H + 2 * t, gv[it]);
    ld2<T>(pk + LINES * H + row * H + 2 * t, sv[it]);
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * NT;
    const int t = idx % (H / 2), rest = idx / (H / 2);
    const int row = rest % LINES, c = rest / LINES;
    c2<T>* z = buf + c * TILE;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int k = 2 * t + q;
      const c2<T> g = gv[it][q], sq = sv[it][q];
      if (k == 0) {
        z[sw<T, LINES>(0, row)] = mk<T>(g.x, T(0));
        z[sw<T, LINES>(H, row)] = mk<T>(g.y, T(0));
      } else {
        const T f = ky_scale * T(k);
        const T dyx = -f * sq.y, dyy = f * sq.x;  // DY = i f S
        z[sw<T, LINES>(k, row)] = mk<T>(g.x - dyy, g.y + dyx);       // DX + i DY
        z[sw<T, LINES>(N - k, row)] = mk<T>(g.x + dyy, dyx - g.y);   // conj(DX) + i conj(DY)
      }
    }
  }
  __syncthreads();
  stockham_pass<T, N, R, 1, LINES, 2, NT, true, N, true>(buf, tw, tid);
  stockham_pass<T, N, R, R, LINES, 2, NT, true, N, true>(buf, tw + O8, tid);

  // ----------------- inverse pass 3 -> RK4 update -> forward pass 1, in registers
  const int j = tid % NB, row = tid / NB;
  c2<T> v[2][R];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[c][r] = buf[c * TILE + sw<T, LINES>(j + r * NB, row)];
  }
#pragma unroll
  for (int r = 1; r < R; ++r) {
    const c2<T> w = tw[O64 + (r - 1) * NB + j];  // W_N^(r j): NS = N / R
#pragma unroll
    for (int c = 0; c < 2; ++c) v[c][r] = twmul<T, true>(v[c][r], w);
  }
  dft<R, T, true>(v[0]);
  dft<R, T, true>(v[1]);
  // v[c][r] = dx + i dy of component c at pixel n = j + NB r of row r0 + row
  if (!wait_or_record(mbar, 0)) return;  // the staged operands: recorded, drained, leave
  const long prow = prow0 + (long)row * N;
  const T* sy0 = stg + row * N;
  const T* sacc = stg + 2 * RB + row * N;
  const T hh = T(a.h);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int n = j + NB * r;
    const T px = preg[0][r], py = preg[1][r];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const T k = px * v[c][r].x + py * v[c][r].y;
      const T y0 = sy0[c * RB + n];
      T* accg = reinterpret_cast<T*>(a.acc) + (map * 2 + c) * P + prow;
      T yn;
      if (a.stage == 1) {
        yn = y0 + T(0.5) * hh * k;
        accg[n] = k;
      } else if (a.stage < 4) {
        yn = y0 + (a.stage == 2 ? T(0.5) * hh : hh) * k;
        accg[n] = sacc[c * RB + n] + T(2) * k;
      } else {
        yn = y0 + hh / T(6) * (sacc[c * RB + n] + k);
        if (a.last) {
          const long fo = (map * 2 + c) * P + prow + n;
          if (a.out_f64) reinterpret_cast<double*>(a.f_out)[fo] = double(yn);
          else reinterpret_cast<float*>(a.f_out)[fo] = yn;
        } else {
          reinterpret_cast<T*>(a.y0)[(map * 2 + c) * P + prow + n] = yn;
        }
      }
      v[c][r].x = yn;
    }
  }
  if (a.last) return;  // uniform across the block
  c2<T> w[R];
#pragma unroll
  for (int r = 0; r < R; ++r) w[r] = mk<T>(v[0][r].x, v[1][r].x);
  dft<R, T, false>(w);  // forward pass 1 (NS = 1): outputs at 8 j + r
  __syncthreads();      // every thread has read its inverse-pass-3 inputs
#pragma unroll
  for (int r = 0; r < R; ++r) buf[sw<T, LINES>(R * j + r, row)] = w[r];
  __syncthreads();
  stockham_pass<T, N, R, R, LINES, 1, NT, false, N, true>(buf, tw + O8, tid);
  stockham_pass<T, N, R, R * R, LINES, 1, NT, false, N, true>(buf, tw + O64, tid);

  // ------------------------------ split W into the two packed row spectra
#pragma unroll
  for (int idx = tid; idx < LINES * (H / 2); idx += NT) {
    const int t = idx % (H / 2), rw = idx / (H / 2);
    c2<T> s0[2], s1[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int k = 2 * t + q;
      if (k == 0) {
        const c2<T> w0 = buf[sw<T, LINES>(0, rw)], wh = buf[sw<T, LINES>(H, rw)];
        s0[0] = mk<T>(w0.x, wh.x);
        s1[0] = mk<T>(w0.y, wh.y);
      } else {
        const c2<T> A = buf[sw<T, LINES>(k, rw)];
        const c2<T> B = cconj<T>(buf[sw<T, LINES>(N - k, rw)]);
        s0[q] = cscale<T>(cadd<T>(A, B), T(0.5));
        const c2<T> d = csub<T>(A, B);
        s1[q] = mk<T>(T(0.5) * d.y, T(-0.5) * d.x);  // (A - B) / 2i
      }
    }
    st2<T>(spec(a.s, 0) + rw * H + 2 * t, s0);
    st2<T>(spec(a.s, 1) + rw * H + 2 * t, s1);
  }
}

// ==================================== adjoint row pass, component pairs
// The adjoint RHS k_c = d_x(p_x y_c) + d_y(p_y y_c) for two components with
// the p planes, N = 512, FP32.  Each component's rate spectrum
// K_c = Gx_c + i KY V_c / N is Hermitian, so both rates come from one
// full-length inverse FFT of Z = K_0 + i K_1 (z = k_0 + i k_1).  After the
// RK4 update the next stage's four real inputs pair up as
// w_u = p_x y_0 + i p_x y_1 and w_v = p_y y_0 + i p_y y_1 (p at the next
// stage time): two forward FFTs, split into the packed spectra U_c (a.s) and
// V_c (a.v) as in k_row_pair.  Same staging, passes and bounded wait.
template <int N, int LINES, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_row_pair_adj(StageArgs a) {
  using T = float;
  constexpr int H = N / 2;
  constexpr long P = (long)N * N;
  constexpr int R = 8, NB = N / R;
  static_assert(N == 512, "three radix-8 passes");
  static_assert(NB * LINES == NT, "one (row, butterfly) per thread in the fused passes");
  constexpr int TILE = LINES * N;
  constexpr int RB = LINES * N;
  constexpr int IT = LINES * (H / 2) / NT;  // packed element pairs per thread in the load phase
  static_assert(LINES * (H / 2) % NT == 0, "whole load-phase iterations");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c2<T>* tw = reinterpret_cast<c2<T>*>(smem_raw);
  c2<T>* buf = tw + N;                            // Z (tile 0); then w_u (tile 0), w_v (tile 1)
  T* stg = reinterpret_cast<T*>(buf + 2 * TILE);  // y0_0, y0_1, acc_0, acc_1
  uint64_t* mbar = reinterpret_cast<uint64_t*>(stg + 4 * RB);  // [0]: staged update operands, [1]: spectra
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * LINES;
  const long map = blockIdx.y;
  const long prow0 = (long)r0 * N;
  const bool with_acc = a.stage > 1;
  const long half_plane = N * (long)H;
  auto spec = [&](void* base, int c) {
    return reinterpret_cast<c2<T>*>(base) + (map * 2 + c) * half_plane + (long)r0 * H;
  };
  static_assert(ptw_size(N) <= N && ptw_size(N) * sizeof(c2<T>) % 16 == 0, "pass table: one bulk copy");
  pdl_launch_dependents();
  if (tid == 0) {
    mbar_init(mbar, 1);
    mbar_init(mbar + 1, 1);
    // the pass table and the spectra first
    mbar_expect_tx(mbar + 1, uint32_t(ptw_size(N) * sizeof(c2<T>) + 4 * LINES * H * sizeof(c2<T>)));
    bulk_g2s(tw, a.twP, ptw_size(N) * sizeof(c2<T>), mbar + 1);
    pdl_wait();  // the other copies read what the previous kernel wrote
    // Gx_c and V_c rows, packed, into tile c
    for (int c = 0; c < 2; ++c) {
      bulk_g2s(buf + c * TILE, spec(a.gx, c), LINES * H * sizeof(c2<T>), mbar + 1);
      bulk_g2s(buf + c * TILE + LINES * H, spec(a.v, c), LINES * H * sizeof(c2<T>), mbar + 1);
    }
    mbar_expect_tx(mbar, uint32_t((with_acc ? 4 : 2) * RB * sizeof(T)));
    for (int c = 0; c < 2; ++c) {
      bulk_g2s(stg + c * RB, reinterpret_cast<const T*>(a.y0) + (map * 2 + c) * P + prow0, RB * sizeof(T), mbar);
      if (with_acc)
        bulk_g2s(stg + (2 + c) * RB, reinterpret_cast<const T*>(a.acc) + (map * 2 + c) * P + prow0, RB * sizeof(T),
                 mbar);
    }
  }
  pdl_wait();  // every thread, before its own global reads and writes
  // p_x, p_y (next stage's time) of the thread's 8 update pixels in registers, as in k_row_pair: six blocks fit
  T preg[2][R];
  {
    const T* pq = reinterpret_cast<const T*>(a.pp) + (map * a.pp_k + a.pp_idx) * 2 * P + prow0 + (tid / NB) * N +
                  tid % NB;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      preg[0][r] = __ldg(pq + NB * r);
      preg[1][r] = __ldg(pq + P + NB * r);
    }
  }
  constexpr int O8 = ptw_offset(N, R, R), O64 = ptw_offset(N, R, R * R);
  const T ky_scale = T(a.kbase / double(N));
  __syncthreads();  // barriers initialised before anyone waits on them
  // the pass table and spectra: a timed-out wait is recorded and the block goes
  // on, so that every thread meets every barrier below
  wait_or_record(mbar + 1, 0);

  // -------------------- load: Z = K_0 + i K_1, K_c = Gx_c + i KY V_c / N (Hermitian)
  // The packed rows sit in tiles 0 and 1; all are read before Z overwrites tile 0.
  c2<T> g0[IT][2], g1[IT][2], v0[IT][2], v1[IT][2];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * NT;
    const int t = idx % (H / 2), row = idx / (H / 2);
    ld2<T>(buf + row * H + 2 * t, g0[it]);
    ld2<T>(buf + LINES * H + row * H + 2 * t, v0[it]);
    ld2<T>(buf + TILE + row * H + 2 * t, g1[it]);
    ld2<T>(buf + TILE + LINES * H + row * H + 2 * t, v1[it]);
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * NT;
    const int t = idx % (H / 2), row = idx / (H / 2);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int k = 2 * t + q;
      if (k == 0) {  // real DC and Nyquist bins of each rate; i KY contributes nothing there
        buf[sw<T, LINES>(0, row)] = mk<T>(g0[it][0].x, g1[it][0].x);
        buf[sw<T, LINES>(H, row)] = mk<T>(g0[it][0].y, g1[it][0].y);
      } else {
        const T f = ky_scale * T(k);
        const c2<T> k0 = mk<T>(g0[it][q].x - f * v0[it][q].y, g0[it][q].y + f * v0[it][q].x);  // Gx + i f V
        const c2<T> k1 = mk<T>(g1[it][q].x - f * v1[it][q].y, g1[it][q].y + f * v1[it][q].x);
        buf[sw<T, LINES>(k, row)] = mk<T>(k0.x - k1.y, k0.y + k1.x);            // K_0 + i K_1
        buf[sw<T, LINES>(N - k, row)] = mk<T>(k0.x + k1.y, k1.x - k0.y);        // conj(K_0) + i conj(K_1)
      }
    }
  }
  __syncthreads();
  stockham_pass<T, N, R, 1, LINES, 1, NT, true, N, true>(buf, tw, tid);
  stockham_pass<T, N, R, R, LINES, 1, NT, true, N, true>(buf, tw + O8, tid);

  // ------------- inverse pass 3 -> RK4 update -> two forward first passes, in registers
  const int j = tid % NB, row = tid / NB;
  c2<T> z[R];
#pragma unroll
  for (int r = 0; r < R; ++r) z[r] = buf[sw<T, LINES>(j + r * NB, row)];
#pragma unroll
  for (int r = 1; r < R; ++r) z[r] = twmul<T, true>(z[r], tw[O64 + (r - 1) * NB + j]);
  dft<R, T, true>(z);
  // z[r] = (k_0, k_1) at pixel n = j + NB r of row r0 + row
  if (!wait_or_record(mbar, 0)) return;  // the staged operands: recorded, drained, leave
  const long prow = prow0 + (long)row * N;
  const T* sy0 = stg + row * N;
  const T* sacc = stg + 2 * RB + row * N;
  const T hh = T(a.h);
  c2<T> wu[R], wv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int n = j + NB * r;
    T yn[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const T k = c == 0 ? z[r].x : z[r].y;
      const T y0 = sy0[c * RB + n];
      T* accg = reinterpret_cast<T*>(a.acc) + (map * 2 + c) * P + prow;
      if (a.stage == 1) {
        yn[c] = y0 + T(0.5) * hh * k;
        accg[n] = k;
      } else if (a.stage < 4) {
        yn[c] = y0 + (a.stage == 2 ? T(0.5) * hh : hh) * k;
        accg[n] = sacc[c * RB + n] + T(2) * k;
      } else {
        yn[c] = y0 + hh / T(6) * (sacc[c * RB + n] + k);
        if (a.last) {
          const long fo = (map * 2 + c) * P + prow + n;
          if (a.out_f64) reinterpret_cast<double*>(a.f_out)[fo] = double(yn[c]);
          else reinterpret_cast<float*>(a.f_out)[fo] = yn[c];
        } else {
          reinterpret_cast<T*>(a.y0)[(map * 2 + c) * P + prow + n] = yn[c];
        }
      }
    }
    const T px = preg[0][r], py = preg[1][r];  // p at the next stage's time
    wu[r] = mk<T>(px * yn[0], px * yn[1]);
    wv[r] = mk<T>(py * yn[0], py * yn[1]);
  }
  if (a.last) return;  // uniform across the block
  dft<R, T, false>(wu);  // forward pass 1 (NS = 1) of both: outputs at 8 j + r
  dft<R, T, false>(wv);
  __syncthreads();       // every thread has read its inverse-pass-3 inputs
#pragma unroll
  for (int r = 0; r < R; ++r) {
    buf[sw<T, LINES>(R * j + r, row)] = wu[r];
    buf[TILE + sw<T, LINES>(R * j + r, row)] = wv[r];
  }
  __syncthreads();
  stockham_pass<T, N, R, R, LINES, 2, NT, false, N, true>(buf, tw + O8, tid);
  stockham_pass<T, N, R, R * R, LINES, 2, NT, false, N, true>(buf, tw + O64, tid);

  // ----------------- split W_u into U_0, U_1 (a.s) and W_v into V_0, V_1 (a.v)
#pragma unroll
  for (int idx = tid; idx < 2 * LINES * (H / 2); idx += NT) {
    const int t = idx % (H / 2), rest = idx / (H / 2);
    const int rw = rest % LINES, which = rest / LINES;
    const c2<T>* wb = buf + which * TILE;
    c2<T> s0[2], s1[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int k = 2 * t + q;
      if (k == 0) {
        const c2<T> w0 = wb[sw<T, LINES>(0, rw)], wh = wb[sw<T, LINES>(H, rw)];
        s0[0] = mk<T>(w0.x, wh.x);
        s1[0] = mk<T>(w0.y, wh.y);
      } else {
        const c2<T> A = wb[sw<T, LINES>(k, rw)];
        const c2<T> B = cconj<T>(wb[sw<T, LINES>(N - k, rw)]);
        s0[q] = cscale<T>(cadd<T>(A, B), T(0.5));
        const c2<T> d = csub<T>(A, B);
        s1[q] = mk<T>(T(0.5) * d.y, T(-0.5) * d.x);  // (A - B) / 2i
      }
    }
    void* dst = which == 0 ? a.s : a.v;
    st2<T>(spec(dst, 0) + rw * H + 2 * t, s0);
    st2<T>(spec(dst, 1) + rw * H + 2 * t, s1);
  }
}

// ====================================================== p planes
// p = M(t)^-1 grad(phi), M = I + t grad grad phi (lense_flow.py:373-381,
// :398-415), at the K = 2n+1 stage times t_k = t0 + k hh of an RK4
// integration, from the five derivative planes; float64 arithmetic, stored in
// T.  grid: x covers P/2 pixel pairs, y = map.
template <typename T>
__global__ void __launch_bounds__(256) k_p_planes(const T* __restrict__ planes, T* __restrict__ pp, long P, int K,
                                                  double t0, double hh) {
  const long map = blockIdx.y;
  const T* ph = planes + map * 5 * P;
  T* out = pp + map * (long)K * 2 * P;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P / 2; i += (long)gridDim.x * blockDim.x) {
    c2<T> f[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) f[j] = reinterpret_cast<const c2<T>*>(ph + j * P)[i];
    for (int k = 0; k < K; ++k) {
      const double t = t0 + k * hh;
      double ox[2], oy[2];
      p_vector<double>(f[0].x, f[1].x, f[2].x, f[3].x, f[4].x, t, ox[0], oy[0]);
      p_vector<double>(f[0].y, f[1].y, f[2].y, f[3].y, f[4].y, t, ox[1], oy[1]);
      reinterpret_cast<c2<T>*>(out + (2 * k) * P)[i] = mk<T>(T(ox[0]), T(ox[1]));
      reinterpret_cast<c2<T>*>(out + (2 * k + 1) * P)[i] = mk<T>(T(oy[0]), T(oy[1]));
    }
  }
}

// ================================================ phi precompute (FP64)
// Each block's float64 twiddle table arrives by one bulk copy (thread 0, on
// an mbarrier placed after the block's tile) while the block loads its data;
// table_wait follows a barrier and precedes the first pass that reads it.
template <int NTAB>
__device__ __forceinline__ void table_copy(double2* tw, const double2* src, uint64_t* mbar, int tid) {
  static_assert(NTAB * sizeof(double2) % 16 == 0, "twiddle table: one bulk copy");
  if (tid == 0) {
    mbar_init(mbar, 1);
    mbar_expect_tx(mbar, uint32_t(NTAB * sizeof(double2)));
    bulk_g2s(tw, src, NTAB * sizeof(double2), mbar);
  }
}

// (a timed-out wait is recorded; the block goes on to its remaining barriers)
__device__ __forceinline__ void table_wait(uint64_t* mbar) { wait_or_record(mbar, 0); }
// rfft along rows of a real map (N x N double) into the unpacked
// (N x (N/2+1)) complex layout of rfft2.   grid: x = row tile, y = map.
template <int N, int LINES, int NT, typename TI = double>
__global__ void __launch_bounds__(NT) k_phi_rows_r2c(const TI* __restrict__ phi, double2* __restrict__ out,
                                                      const double2* __restrict__ twN) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* buf = tw + N;
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * LINES;
  const long map = blockIdx.y;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + LINES * H);
  table_copy<N>(tw, twN, mbar, tid);
  const c2<TI>* src = reinterpret_cast<const c2<TI>*>(phi + map * (long)N * N + (long)r0 * N);
  load_rows<double, c2<TI>, H, LINES, NT>(buf, src, H, tid);
  __syncthreads();
  table_wait(mbar);
  fft_tiles<double, H, LINES, 1, NT, false, N>(buf, tw, tid);
  r2c_post<double, H, LINES, 1, NT>(buf, tw, tid);
  double2* dst = out + map * (long)N * (H + 1) + (long)r0 * (H + 1);
  for (int idx = tid; idx < (H + 1) * LINES; idx += NT) {
    const int row = idx / (H + 1), k = idx % (H + 1);
    double2 v;
    if (k == 0) {
      v = make_double2(buf[sw<double, LINES>(0, row)].x, 0.0);
    } else if (k == H) {
      v = make_double2(buf[sw<double, LINES>(0, row)].y, 0.0);
    } else {
      v = buf[sw<double, LINES>(k, row)];
    }
    dst[(long)row * (H + 1) + k] = v;
  }
}

// In-place forward column FFT of the N/2+1 columns of an (N x (N/2+1)) array.
template <int N, int LINES, int NT>
__global__ void __launch_bounds__(NT) k_phi_cols_fwd(double2* __restrict__ arr, const double2* __restrict__ twN) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* buf = tw + N;
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * LINES;
  // maps in reverse launch order: the row transform before it finished on the last maps, still in L2
  // (with the fused row pass below also reversed: phi precompute 1.044 -> 1.034 ms per 64 maps)
  double2* a = arr + (gridDim.y - 1 - blockIdx.y) * (long)N * (H + 1);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + LINES * N);
  table_copy<N>(tw, twN, mbar, tid);
  load_cols<double, N, LINES, NT>(buf, a, H + 1, c0, H + 1, tid);
  __syncthreads();
  table_wait(mbar);
  fft_tiles<double, N, LINES, 1, NT, false, N>(buf, tw, tid);
  store_cols<double, N, LINES, NT>(a, H + 1, c0, H + 1, buf, tid);
}

// Five derivative spectra j in {x, y, xx, xy, yy} (util.py:125-130), each
// written as a packed row spectrum (columns 0 and N/2 keep only their real
// parts, as irfft2 does).  KY is constant down a column, so it commutes with
// the inverse column FFT: three inverse transforms serve all five,
//   G0 = IFFT_col(F):           phi_y = i KY G0,  phi_yy = -KY^2 G0
//   G1 = IFFT_col(i KX F):      phi_x = G1,       phi_xy = i KY G1
//   G2 = IFFT_col(-KX^2 F):     phi_xx = G2
// (the 1/N^2 of irfft2 folded into the column multiplier).  ``spec`` is the
// unpacked rfft2 of phi; ``packed`` is [B][5][N][N/2] complex.
template <int N, int LINES, int NT, typename PK = double2>
__global__ void __launch_bounds__(NT) k_phi_cols_deriv(const double2* __restrict__ spec, PK* __restrict__ packed,
                                                        const double2* __restrict__ twN, double kbase) {
  using S = decltype(PK::x);  // storage precision of the packed derivative spectra
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* buf = tw + N;
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * LINES;
  const long map = blockIdx.y;
  const double2* a = spec + map * (long)N * (H + 1);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + LINES * N);
  table_copy<N>(tw, twN, mbar, tid);
  const double scale = 1.0 / (double(N) * double(N));
  // (G, output j, KY power): KY power 0 = G itself, 1 = i KY G, 2 = -KY^2 G
  constexpr int kOut[3][2][2] = {{{1, 1}, {4, 2}}, {{0, 0}, {3, 1}}, {{2, 0}, {-1, 0}}};
#pragma unroll 1
  for (int g = 0; g < 3; ++g) {
    load_cols<double, N, LINES, NT>(buf, a, H + 1, c0, H + 1, tid);
    __syncthreads();
    for (int idx = tid; idx < N * LINES; idx += NT) {
      const int m = idx / LINES, line = idx % LINES;
      const double kx = kbase * double(m < N / 2 ? m : m - N);
      const double2 v = buf[sw<double, LINES>(m, line)];
      double2 r;
      if (g == 0) r = make_double2(scale * v.x, scale * v.y);
      else if (g == 1) r = make_double2(-kx * v.y * scale, kx * v.x * scale);
      else r = make_double2(-kx * kx * scale * v.x, -kx * kx * scale * v.y);
      buf[sw<double, LINES>(m, line)] = r;
    }
    __syncthreads();
    if (g == 0) table_wait(mbar);
    fft_tiles<double, N, LINES, 1, NT, true, N>(buf, tw, tid);
    for (int o = 0; o < 2; ++o) {
      const int j = kOut[g][o][0], pw = kOut[g][o][1];
      if (j < 0) continue;
      PK* out = packed + (map * 5 + j) * (long)N * H;
      for (int idx = tid; idx < N * LINES; idx += NT) {
        const int m = idx / LINES, line = idx % LINES;
        const int col = c0 + line;
        if (col > H) continue;
        const double ky = (col == H) ? -kbase * double(H) : kbase * double(col);
        const double2 G = buf[sw<double, LINES>(m, line)];
        double2 v;
        if (pw == 0) v = G;
        else if (pw == 1) v = make_double2(-ky * G.y, ky * G.x);
        else v = make_double2(-ky * ky * G.x, -ky * ky * G.y);
        if (col == 0) reinterpret_cast<S*>(out + (long)m * H)[0] = S(v.x);
        else if (col == H) reinterpret_cast<S*>(out + (long)m * H)[1] = S(v.x);
        else out[(long)m * H + col] = PK{S(v.x), S(v.y)};
      }
    }
    __syncthreads();
  }
}

// Inverse real transform of the packed rows into the five derivative planes.
// grid: x = row tile, y = map * 5 + j.
template <typename TO, int N, int LINES, int NT>
__global__ void __launch_bounds__(NT) k_phi_rows_c2r(const double2* __restrict__ packed, TO* __restrict__ planes,
                                                      const double2* __restrict__ twN) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* buf = tw + N;
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * LINES;
  const long pl = blockIdx.y;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + LINES * H);
  table_copy<N>(tw, twN, mbar, tid);
  load_rows<double, double2, H, LINES, NT>(buf, packed + pl * (long)N * H + (long)r0 * H, H, tid);
  __syncthreads();
  table_wait(mbar);
  c2r_pre<double, H, LINES, 1, NT>(buf, tw, tid);
  fft_tiles<double, H, LINES, 1, NT, true, N>(buf, tw, tid);
  using O2 = c2<TO>;
  O2* dst = reinterpret_cast<O2*>(planes + pl * (long)N * N + (long)r0 * N);
  store_rows<double, O2, H, LINES, NT>(dst, H, buf, tid);
}

// Per-map minimum over pixels and t in [0, 1] of det(I + t grad grad phi).
__device__ __forceinline__ int ordered_int(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}

template <typename T>
__global__ void k_min_det(const T* __restrict__ planes, long P, int* __restrict__ out) {
  const long map = blockIdx.y;
  const T* pxx = planes + map * 5 * P + 2 * P;
  const T* pxy = pxx + P;
  const T* pyy = pxy + P;
  double best = 1.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < P; i += (long)gridDim.x * blockDim.x) {
    const double A = pxx[i], B = pxy[i], Cc = pyy[i];
    const double q = A * Cc - B * B, l = A + Cc;
    double d = 1.0 + l + q;  // t = 1
    if (q > 0.0) {
      const double ts = -l / (2.0 * q);
      if (ts > 0.0 && ts < 1.0) d = fmin(d, 1.0 + ts * l + ts * ts * q);
    }
    best = fmin(best, d);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMin(out + map, ordered_int(float(best)));
}

// ============================ fused: derivative rows -> p planes at the stage times
// The inverse real row transforms of all five derivative spectra of LINES
// rows (as k_phi_rows_c2r, float64), and in the same block, from the five
// derivatives of each pixel: p = M(t)^-1 grad(phi) (lense_flow.py:373-381,
// :398-415) at the K = 2n+1 times k / (2n), in float32 arithmetic and stored
// float32 ascending in time ([B][K][2][N][N]), and the per-map minimum of
// det(I + t grad grad phi) over pixels and t in [0, 1] (float64, as
// k_min_det).  The
// five derivative planes are written only when ``planes`` is non-null, so
// the forward lens's p planes no longer round-trip them through HBM.
// grid: x = row tile, y = map.  NT: about one first-pass butterfly per thread (a warp multiple); 2-row
// tiles, four blocks per SM (measured against 4-row tiles at two: 1.142 vs 1.153 ms of phi precompute per
// 64-map 512^2 step).
__host__ __device__ constexpr int pp_threads(int n) { return n <= 64 ? 64 : (n == 128 ? 96 : (n <= 512 ? 160 : 320)); }

template <int N, int LINES, int NT, typename PK = double2>
__global__ void __launch_bounds__(NT, N == 1024 ? 2 : 4) k_phi_rows_c2r_pp(const PK* __restrict__ packed, float* __restrict__ planes,
                                                         float* __restrict__ pp, int K, int* __restrict__ min_det,
                                                         const double2* __restrict__ twN) {
  constexpr int H = N / 2;
  constexpr long P = (long)N * N;
  constexpr int TILE = LINES * H;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* buf = tw + N;  // derivative j at buf + j * TILE
  __shared__ double warp_min[NT / 32];
  const int tid = threadIdx.x;
  const int r0 = blockIdx.x * LINES;
  // maps in reverse launch order: the derivative column pass before it finished on the last maps, still
  // in L2, and the lens's first kernel then starts on map 0, the freshest here
  const long map = gridDim.y - 1 - blockIdx.y;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + 5 * TILE);
  table_copy<N>(tw, twN, mbar, tid);
#pragma unroll
  for (int j = 0; j < 5; ++j)
    load_rows<double, PK, H, LINES, NT>(buf + j * TILE, packed + ((map * 5 + j) * N + r0) * (long)H, H, tid);
  __syncthreads();
  table_wait(mbar);
  c2r_pre<double, H, LINES, 5, NT>(buf, tw, tid);
  fft_tiles<double, H, LINES, 5, NT, true, N>(buf, tw, tid);
  // tile element m of a row holds pixels 2m (re) and 2m + 1 (im); two elements (four pixels) per item
  const double inv2n = 1.0 / double(K - 1);
  double best = 1.0;
  for (int idx = tid; idx < LINES * (H / 2); idx += NT) {
    const int row = idx / (H / 2), m0 = 2 * (idx % (H / 2));
    double d[5][4];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double2 a0 = buf[j * TILE + sw<double, LINES>(m0, row)];
      const double2 a1 = buf[j * TILE + sw<double, LINES>(m0 + 1, row)];
      d[j][0] = a0.x;
      d[j][1] = a0.y;
      d[j][2] = a1.x;
      d[j][3] = a1.y;
    }
    const long o = (long)(r0 + row) * N + 2 * m0;  // first of the four pixels
    if (planes) {
#pragma unroll
      for (int j = 0; j < 5; ++j)
        *reinterpret_cast<float4*>(planes + (map * 5 + j) * P + o) =
            make_float4(float(d[j][0]), float(d[j][1]), float(d[j][2]), float(d[j][3]));
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {  // min over t in [0, 1] of det(I + t H) = 1 + t l + t^2 qd
      const double A = d[2][q], B = d[3][q], Cc = d[4][q];
      const double qd = A * Cc - B * B, l = A + Cc;
      double dm = 1.0 + l + qd;
      if (qd > 0.0) {
        const double ts = -l / (2.0 * qd);
        if (ts > 0.0 && ts < 1.0) dm = fmin(dm, 1.0 + ts * l + ts * ts * qd);
      }
      best = fmin(best, dm);
    }
    float* out = pp + map * (long)K * 2 * P + o;
    // p = M(t)^-1 grad phi through the adjugate of the symmetric 2x2 M = I + t H (H = grad grad phi):
    //   p_x = (phi_x + t (H_yy phi_x - H_xy phi_y)) / D,  p_y = (phi_y + t (H_xx phi_y - H_xy phi_x)) / D,
    //   D = det M = 1 + t (H_xx + H_yy) + t^2 (H_xx H_yy - H_xy^2).
    // The time-independent coefficients are formed once per pixel in float64; each time then costs two
    // FMAs for D, one reciprocal and four FMA/multiplies in float32 (the RK4 right-hand side that reads
    // the planes is float32).  The reference's det + 1e-12 (lense_flow.py:408-411) is below float32
    // resolution for D >= 0.2 and is not added.
    float gx[4], gy[4], bx[4], by[4], lt[4], qt[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double A = d[2][q], Bx = d[3][q], Cc = d[4][q];
      gx[q] = float(d[0][q]);
      gy[q] = float(d[1][q]);
      bx[q] = float(Cc * d[0][q] - Bx * d[1][q]);
      by[q] = float(A * d[1][q] - Bx * d[0][q]);
      lt[q] = float(A + Cc);
      qt[q] = float(A * Cc - Bx * Bx);
    }
#pragma unroll 1
    for (int k = 0; k < K; ++k) {
      const float t = float(double(k) * inv2n);
      float ox[4], oy[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float r = __frcp_rn(fmaf(t, fmaf(t, qt[q], lt[q]), 1.0f));
        ox[q] = fmaf(t, bx[q], gx[q]) * r;
        oy[q] = fmaf(t, by[q], gy[q]) * r;
      }
      *reinterpret_cast<float4*>(out + (2 * k) * P) =
          make_float4(float(ox[0]), float(ox[1]), float(ox[2]), float(ox[3]));
      *reinterpret_cast<float4*>(out + (2 * k + 1) * P) =
          make_float4(float(oy[0]), float(oy[1]), float(oy[2]), float(oy[3]));
    }
  }
  if (min_det) {
    for (int w = 16; w > 0; w >>= 1) best = fmin(best, __shfl_xor_sync(0xffffffffu, best, w));
    if ((tid & 31) == 0) warp_min[tid / 32] = best;
    __syncthreads();
    if (tid == 0) {
      double b = warp_min[0];
      for (int w = 1; w < NT / 32; ++w) b = fmin(b, warp_min[w]);
      atomicMin(min_det + map, ordered_int(float(b)));
    }
  }
}

// ======================================================= reverse mode
// delta-phi accumulation for one RK4 stage (lense_flow.py:195-252).  With
// fdf = sum_c df_c grad f_c, a = M^-1 fdf, w = p (x) a, the stage rate is
//   D_x a_x + D_y a_y + t (D_xx w_xx + D_xy (w_xy + w_yx) + D_yy w_yy).
// delta-phi never feeds back into the ODE, so its RK4 sum is linear in the
// rates: the five pre-derivative fields are accumulated with the stage
// weight h/6 {1,2,2,1} here and the derivative multipliers are applied once
// at the end (k_dphi_combine).  Accumulators are float64, [B][5][N][N].
template <typename T, int C>
__global__ void k_dphi_accum(const T* __restrict__ grad, const T* __restrict__ dsave, const T* __restrict__ phi,
                             double* __restrict__ acc, int B, long P, double t, double wgt, int first) {
  const long total = (long)B * P;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long b = i / P, px = i % P;
    double fx = 0.0, fy = 0.0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const long pl = b * C + c;
      const double d = dsave[pl * P + px];
      fx += d * double(grad[pl * 2 * P + px]);
      fy += d * double(grad[pl * 2 * P + P + px]);
    }
    const T* ph = phi + b * 5 * P + px;
    const double gx = ph[0], gy = ph[P], gxx = ph[2 * P], gxy = ph[3 * P], gyy = ph[4 * P];
    const double mxx = 1.0 + t * gxx, mxy = t * gxy, myy = 1.0 + t * gyy;
    const double inv = 1.0 / (mxx * myy - mxy * mxy + 1e-12);
    const double ixx = myy * inv, ixy = -mxy * inv, iyy = mxx * inv;
    const double ax = ixx * fx + ixy * fy, ay = ixy * fx + iyy * fy;
    const double pxv = gx * ixx + gy * ixy, pyv = gx * ixy + gy * iyy;
    const double v[5] = {ax, ay, t * pxv * ax, t * (pxv * ay + pyv * ax), t * pyv * ay};
    double* o = acc + b * 5 * P + px;
#pragma unroll
    for (int j = 0; j < 5; ++j) o[j * P] = first ? wgt * v[j] : o[j * P] + wgt * v[j];
  }
}

// delta-phi in the rfft2 layout: sum_j m_j * rfft2(acc_j) with the raw
// multipliers of get_primal_derivatives_to_fourier (util.py:133-137):
// i KX, i KY, -KX^2, -KX KY, -KY^2 (KY's Nyquist entry negated).
// ``spec`` holds rfft2(acc_j) as [B][5][N][N/2+1].
__global__ void k_dphi_combine(const double2* __restrict__ spec, double2* __restrict__ out, int B, int N,
                               double kbase) {
  const int H = N / 2;
  const long per = (long)N * (H + 1);
  const long total = (long)B * per;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long b = i / per, r = i % per;
    const int k0 = (int)(r / (H + 1)), k1 = (int)(r % (H + 1));
    const double kx = kbase * double(k0 < N / 2 ? k0 : k0 - N);
    const double ky = (k1 == H) ? -kbase * double(H) : kbase * double(k1);
    const double2* s = spec + b * 5 * per + r;
    const double2 s0 = s[0], s1 = s[per], s2 = s[2 * per], s3 = s[3 * per], s4 = s[4 * per];
    double re = -kx * s0.y - ky * s1.y;
    double im = kx * s0.x + ky * s1.x;
    const double q2 = -kx * kx, q3 = -kx * ky, q4 = -ky * ky;
    re += q2 * s2.x + q3 * s3.x + q4 * s4.x;
    im += q2 * s2.y + q3 * s3.y + q4 * s4.y;
    out[i] = make_double2(re, im);
  }
}

// Inverse column FFT of an unpacked (N x (N/2+1)) spectrum, scaled by
// 1/N^2, into packed rows whose slot 0 keeps the real parts of columns 0 and
// N/2 (what irfft2 keeps).  grid: x = column tile, y = map.
template <int N, int LINES, int NT>
__global__ void __launch_bounds__(NT) k_spec_cols_inv(const double2* __restrict__ spec, double2* __restrict__ packed,
                                                       const double2* __restrict__ twN) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* tw = reinterpret_cast<double2*>(smem_raw);
  double2* buf = tw + N;
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * LINES;
  const long map = blockIdx.y;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(buf + LINES * N);
  table_copy<N>(tw, twN, mbar, tid);
  load_cols<double, N, LINES, NT>(buf, spec + map * (long)N * (H + 1), H + 1, c0, H + 1, tid);
  __syncthreads();
  table_wait(mbar);
  const double scale = 1.0 / (double(N) * double(N));
  for (int idx = tid; idx < N * LINES; idx += NT) {
    const int m = idx / LINES, line = idx % LINES;
    const double2 v = buf[sw<double, LINES>(m, line)];
    buf[sw<double, LINES>(m, line)] = make_double2(v.x * scale, v.y * scale);
  }
  __syncthreads();
  fft_tiles<double, N, LINES, 1, NT, true, N>(buf, tw, tid);
  double2* out = packed + map * (long)N * H;
  for (int idx = tid; idx < N * LINES; idx += NT) {
    const int m = idx / LINES, line = idx % LINES;
    const int col = c0 + line;
    const double2 v = buf[sw<double, LINES>(m, line)];
    if (col == 0) reinterpret_cast<double*>(out + (long)m * H)[0] = v.x;
    else if (col == H) reinterpret_cast<double*>(out + (long)m * H)[1] = v.x;
    else if (col < H) out[(long)m * H + col] = v;
  }
}

}  // namespace lf

namespace lf {

// ================================================ per-mode operator products
// out[b][i][m] = s * sum_j W[b or 0][i][j][m] * X[b][j][m] + t * Y[b][i][m]
// for the Fourier-diagonal C x C operators of the Wiener filter
// (matrix_operators.py:54-141, the EB<->QU rotation of util.py:140-161):
// W real float64 [Bw][C][C][M] (Bw = 1 broadcasts), X / Y / out complex128
// [B][C][M].  Bit (i C + j) of ``nz`` marks the blocks that are not
// identically zero; the others are neither read nor multiplied.  Every
// output of a mode is formed from registers before any is stored, so out may
// alias X or Y.
template <int C>
__global__ void __launch_bounds__(256) k_modes_apply(const double* __restrict__ W, int w_batched, unsigned nz,
                                                     const double2* X, const double2* Y, double2* out, int B, long M,
                                                     double s, double t) {
  const long total = (long)B * M;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long b = e / M, m = e % M;
    const double* w = W + (w_batched ? b : 0) * (long)C * C * M + m;
    double2 x[C], o[C];
#pragma unroll
    for (int j = 0; j < C; ++j) x[j] = X[(b * C + j) * M + m];
#pragma unroll
    for (int i = 0; i < C; ++i) {
      double re = 0.0, im = 0.0;
#pragma unroll
      for (int j = 0; j < C; ++j) {
        if (nz & (1u << (i * C + j))) {
          const double wij = w[(long)(i * C + j) * M];
          re += wij * x[j].x;
          im += wij * x[j].y;
        }
      }
      o[i] = make_double2(s * re, s * im);
      if (Y) {
        const double2 y = Y[(b * C + i) * M + m];
        o[i].x += t * y.x;
        o[i].y += t * y.y;
      }
    }
#pragma unroll
    for (int i = 0; i < C; ++i) out[(b * C + i) * M + m] = o[i];
  }
}

}  // namespace lf
