// Shared-memory FFT engine for the LenseFlow kernels (sm_100a).
//
// A thread block owns a *tile* of LINES independent 1-D transforms ("lines"),
// each of length L, held in shared memory as complex values.  Element
// (m, line) -- m the position along the transform axis -- has the linear
// index e = m * LINES + line and is stored at
//
//     tile[e ^ ((e / EPC) & (EPC - 1))],   EPC = 128 bytes / element size,
//
// i.e. every 128-byte chunk of the tile is permuted by an XOR with its chunk
// number.  These warp access patterns then touch each bank at most twice
// per 32 accesses (the minimum for 8-byte elements): the Stockham reads
// (consecutive threads = consecutive lines, then consecutive m), the
// Stockham writes at stride R in m, the row-major global loads and stores and
// the pointwise epilogues (consecutive threads = consecutive m); the
// descending H-k accesses of the real-FFT pre-pass reach three on some warps.
// Permuting whole chunks rather than the lines of one m matters for tiles of
// fewer than 16 lines, whose stride-R writes otherwise fall on LINES banks.
//
// The transforms are radix-R Stockham autosort passes (Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors",
// SC08): each pass reads R inputs at stride L/R, twiddles, applies a
// register-resident radix-R DFT and writes in natural order.  Every thread
// keeps its butterflies' inputs in registers across the pass barrier, so a
// single buffer suffices.  Twiddles come from a host-computed table
// tw[e] = exp(-2 pi i e / NTAB) (float64 on the host, rounded once).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>


namespace lf {

// Pure-arithmetic helpers and the register DFTs compile for the host as well
// (their unit test runs on the CPU).
#define LF_HD __host__ __device__ __forceinline__

template <typename T> struct V2;
template <> struct V2<float> { using type = float2; };
template <> struct V2<double> { using type = double2; };
template <typename T> using c2 = typename V2<T>::type;

template <typename T> LF_HD c2<T> mk(T x, T y) { c2<T> r; r.x = x; r.y = y; return r; }
// sm_100 packed float32 pairs (add/sub/fma.rn.f32x2): one instruction per complex
// add, subtract or a + s u with a real s, where scalar code needs two.  Device
// float code only; the host build (the DFT unit test) keeps the scalar form.
// Measured on the two-pass column pass (64-map 512^2 QU step): add/sub 1.81 ->
// 1.63 ms, with the butterflies' a +- s u as well 1.56 ms.
__device__ __forceinline__ float2 f2_add(float2 a, float2 b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<uint64_t*>(&a)), "l"(*reinterpret_cast<uint64_t*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<uint64_t*>(&a)), "l"(*reinterpret_cast<uint64_t*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
template <typename T> LF_HD c2<T> cadd(c2<T> a, c2<T> b) {
#ifdef __CUDA_ARCH__
  if constexpr (std::is_same<T, float>::value) return f2_add(a, b);
#endif
  return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T> LF_HD c2<T> csub(c2<T> a, c2<T> b) {
#ifdef __CUDA_ARCH__
  if constexpr (std::is_same<T, float>::value) return f2_sub(a, b);
#endif
  return mk<T>(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(r)
      : "l"(*reinterpret_cast<uint64_t*>(&a)), "l"(*reinterpret_cast<uint64_t*>(&b)),
        "l"(*reinterpret_cast<uint64_t*>(&c)));
  return *reinterpret_cast<float2*>(&r);
}
// a + s u for a real s
template <typename T> LF_HD c2<T> caxpy(T s, c2<T> u, c2<T> a) {
#ifdef __CUDA_ARCH__
  if constexpr (std::is_same<T, float>::value) return f2_fma(make_float2(s, s), u, a);
#endif
  return mk<T>(a.x + s * u.x, a.y + s * u.y);
}
template <typename T> LF_HD c2<T> cmul(c2<T> a, c2<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T> LF_HD c2<T> cmulc(c2<T> a, c2<T> b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T> LF_HD c2<T> cconj(c2<T> a) { return mk<T>(a.x, -a.y); }
template <typename T> LF_HD c2<T> cscale(c2<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
// multiply by i
template <typename T> LF_HD c2<T> cmul_i(c2<T> a) { return mk<T>(-a.y, a.x); }

// Twiddle multiply by exp(-+2 pi i e/NTAB): forward uses tw[e], inverse conj(tw[e]).
template <typename T, bool INV> LF_HD c2<T> twmul(c2<T> a, c2<T> w) {
  return INV ? cmulc<T>(a, w) : cmul<T>(a, w);
}

// x * (-i) for the forward transform, x * (+i) for the inverse.
template <typename T, bool INV> LF_HD c2<T> rot90(c2<T> a) {
  return INV ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

// ----------------------------------------------------------- small DFTs
// In-place, natural order in and out, unnormalised; forward kernel e^{-2 pi i jk/R}.
template <typename T, bool INV> LF_HD void dft2(c2<T>* a) {
  c2<T> t = a[0];
  a[0] = cadd<T>(t, a[1]);
  a[1] = csub<T>(t, a[1]);
}

template <typename T, bool INV> LF_HD void dft4(c2<T>* a) {
  c2<T> t0 = cadd<T>(a[0], a[2]), t1 = csub<T>(a[0], a[2]);
  c2<T> t2 = cadd<T>(a[1], a[3]), t3 = rot90<T, INV>(csub<T>(a[1], a[3]));
  a[0] = cadd<T>(t0, t2);
  a[2] = csub<T>(t0, t2);
  a[1] = cadd<T>(t1, t3);
  a[3] = csub<T>(t1, t3);
}

// sqrt(2)/2, cos(pi/8), sin(pi/8)
#define LF_C45 0.70710678118654752440
#define LF_C22 0.92387953251128675613
#define LF_S22 0.38268343236508977173

template <typename T, bool INV> LF_HD void dft8(c2<T>* a) {
  c2<T> e[4] = {a[0], a[2], a[4], a[6]};
  c2<T> o[4] = {a[1], a[3], a[5], a[7]};
  dft4<T, INV>(e);
  dft4<T, INV>(o);
  const T c = T(LF_C45);
  // o1 * W8^1 = c s1, W8^1 = (c, -c) forward / (c, c) inverse
  const c2<T> s1 = INV ? mk<T>(o[1].x - o[1].y, o[1].x + o[1].y) : mk<T>(o[1].x + o[1].y, o[1].y - o[1].x);
  c2<T> o2 = rot90<T, INV>(o[2]);
  // o3 * W8^3 = c s3, W8^3 = (-c, -c) forward / (-c, c) inverse
  const c2<T> s3 = INV ? mk<T>(-o[3].x - o[3].y, o[3].x - o[3].y) : mk<T>(o[3].y - o[3].x, -o[3].x - o[3].y);
  a[0] = cadd<T>(e[0], o[0]);
  a[4] = csub<T>(e[0], o[0]);
  a[1] = caxpy<T>(c, s1, e[1]);
  a[5] = caxpy<T>(-c, s1, e[1]);
  a[2] = cadd<T>(e[2], o2);
  a[6] = csub<T>(e[2], o2);
  a[3] = caxpy<T>(c, s3, e[3]);
  a[7] = caxpy<T>(-c, s3, e[3]);
}

// a <- a + w b, b <- a - w b for a constant twiddle w = (wr, wi), with FMAs: w b is written as
// wr (1 + i wi/wr) b when |wr| >= |wi|, else wi (wr/wi + i) b, so the scaled b costs two FMAs and
// each output two more (six instructions instead of eight for a multiply, then an add and a subtract).
template <typename T> LF_HD void bfly_w(c2<T>& a, c2<T>& b, double wr, double wi) {
  c2<T> u;
  T f;
  if (wr * wr >= wi * wi) {
    const T t = T(wi / wr);
    u = mk<T>(b.x - t * b.y, b.y + t * b.x);
    f = T(wr);
  } else {
    const T t = T(wr / wi);
    u = mk<T>(t * b.x - b.y, t * b.y + b.x);
    f = T(wi);
  }
  const c2<T> a0 = a;
  a = caxpy<T>(f, u, a0);
  b = caxpy<T>(-f, u, a0);
}

// Radix-2 split into two 8-point DFTs: X[k] = E[k] + W16^k O[k], X[k+8] = E[k] - W16^k O[k].
template <typename T, bool INV> LF_HD void dft16(c2<T>* a) {
  c2<T> e[8], o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    e[i] = a[2 * i];
    o[i] = a[2 * i + 1];
  }
  dft8<T, INV>(e);
  dft8<T, INV>(o);
  // W16^k forward = (cos(pi k/8), -sin(pi k/8)), k = 0..7
  const double wr[8] = {1.0, LF_C22, LF_C45, LF_S22, 0.0, -LF_S22, -LF_C45, -LF_C22};
  const double ws[8] = {0.0, LF_S22, LF_C45, LF_C22, 1.0, LF_C22, LF_C45, LF_S22};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k == 0 || k == 4) {
      const c2<T> t = (k == 0) ? o[k] : rot90<T, INV>(o[k]);
      a[k] = cadd<T>(e[k], t);
      a[k + 8] = csub<T>(e[k], t);
    } else {
      bfly_w<T>(e[k], o[k], wr[k], INV ? ws[k] : -ws[k]);
      a[k] = e[k];
      a[k + 8] = o[k];
    }
  }
}

// cos(pi/16), sin(pi/16), cos(3 pi/16), sin(3 pi/16)
#define LF_C11 0.98078528040323044913
#define LF_S11 0.19509032201612826785
#define LF_C33 0.83146961230254523708
#define LF_S33 0.55557023301960222474

// Radix-2 split into two 16-point DFTs: X[k] = E[k] + W32^k O[k], X[k+16] = E[k] - W32^k O[k].
template <typename T, bool INV> LF_HD void dft32(c2<T>* a) {
  c2<T> e[16], o[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    e[i] = a[2 * i];
    o[i] = a[2 * i + 1];
  }
  dft16<T, INV>(e);
  dft16<T, INV>(o);
  // W32^k forward = (cos(pi k/16), -sin(pi k/16)), k = 0..15
  const double wr[16] = {1.0,     LF_C11,  LF_C22,  LF_C33,  LF_C45,  LF_S33,  LF_S22,  LF_S11,
                         0.0,     -LF_S11, -LF_S22, -LF_S33, -LF_C45, -LF_C33, -LF_C22, -LF_C11};
  const double ws[16] = {0.0,    LF_S11, LF_S22, LF_S33, LF_C45, LF_C33, LF_C22, LF_C11,
                         1.0,    LF_C11, LF_C22, LF_C33, LF_C45, LF_S33, LF_S22, LF_S11};
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if (k == 0 || k == 8) {
      const c2<T> t = (k == 0) ? o[k] : rot90<T, INV>(o[k]);
      a[k] = cadd<T>(e[k], t);
      a[k + 16] = csub<T>(e[k], t);
    } else {
      bfly_w<T>(e[k], o[k], wr[k], INV ? ws[k] : -ws[k]);
      a[k] = e[k];
      a[k + 16] = o[k];
    }
  }
}

template <int R, typename T, bool INV> LF_HD void dft(c2<T>* a) {
  if constexpr (R == 2) dft2<T, INV>(a);
  else if constexpr (R == 4) dft4<T, INV>(a);
  else if constexpr (R == 8) dft8<T, INV>(a);
  else if constexpr (R == 16) dft16<T, INV>(a);
  else if constexpr (R == 32) dft32<T, INV>(a);
  else static_assert(R == 2 || R == 4 || R == 8 || R == 16 || R == 32, "unsupported radix");
}

// ------------------------------------------------------------ tile layout
// (0 <= line < LINES; the chunk number is written per case so that it costs
// no more than a shift)
template <typename T, int LINES> __device__ __forceinline__ int sw(int m, int line) {
  constexpr int EPC = 128 / int(sizeof(c2<T>));  // elements per 128-byte chunk
  static_assert(LINES % EPC == 0 || EPC % LINES == 0, "LINES must divide or be a multiple of a chunk");
  if constexpr (LINES == EPC) {
    return m * LINES + (line ^ (m & (EPC - 1)));
  } else if constexpr (LINES > EPC) {
    return (m * LINES + line) ^ ((m * (LINES / EPC) + line / EPC) & (EPC - 1));
  } else {
    return (m * LINES + line) ^ ((m / (EPC / LINES)) & (EPC - 1));
  }
}

// ------------------------------------------------------- plans and tables
// Radices of the length-L plan: R1 x R2 (x R3).  The inverse half of
// fft_mul_ifft runs them in reverse order.
__host__ __device__ constexpr int plan_r1(int L) { return (L == 256 || L == 1024) ? 16 : 8; }
__host__ __device__ constexpr int plan_r2(int L) { return L == 32 ? 4 : (L == 64 || L == 512 || L == 1024) ? 8 : 16; }
__host__ __device__ constexpr int plan_r3(int L) { return (L == 512 || L == 1024) ? 8 : 1; }

// Pass twiddle tables.  A pass of radix R after passes of total length NS
// multiplies input r of butterfly j by W_{R NS}^{r k}, k = j mod NS.  Read
// from one table tw[r k NTAB / (R NS)], the threads of a warp (consecutive k)
// hit addresses r NTAB / (R NS) apart -- the same bank for many of them.  A
// pass table stores W^{r k} at (r - 1) NS + k instead, so a warp's reads are
// consecutive.  The table of length L holds one block per distinct (R, NS)
// of the forward plan and of the reversed (inverse) plan.
struct PtwBlock {
  int R, NS;
};

__host__ __device__ constexpr PtwBlock ptw_candidate(int L, int b) {
  const int r1 = plan_r1(L), r2 = plan_r2(L), r3 = plan_r3(L);
  if (r3 > 1)  // forward (r2, r1), (r3, r1 r2); reversed (r2, r3), (r1, r3 r2)
    return b == 0 ? PtwBlock{r2, r1} : b == 1 ? PtwBlock{r3, r1 * r2} : b == 2 ? PtwBlock{r2, r3} : PtwBlock{r1, r3 * r2};
  return b == 0 ? PtwBlock{r2, r1} : b == 1 ? PtwBlock{r1, r2} : PtwBlock{0, 0};  // forward, reversed
}

__host__ __device__ constexpr bool ptw_repeats(int L, int b) {
  for (int c = 0; c < b; ++c) {
    const PtwBlock x = ptw_candidate(L, c), y = ptw_candidate(L, b);
    if (x.R == y.R && x.NS == y.NS) return true;
  }
  return false;
}

// offset of the (R, NS) block in the pass table of length L (-1: none)
__host__ __device__ constexpr int ptw_offset(int L, int R, int NS) {
  int off = 0;
  for (int b = 0; b < 4; ++b) {
    const PtwBlock x = ptw_candidate(L, b);
    if (x.R == 0 || ptw_repeats(L, b)) continue;
    if (x.R == R && x.NS == NS) return off;
    off += (x.R - 1) * x.NS;
  }
  return -1;
}

__host__ __device__ constexpr int ptw_size(int L) {
  int off = 0;
  for (int b = 0; b < 4; ++b) {
    const PtwBlock x = ptw_candidate(L, b);
    if (x.R == 0 || ptw_repeats(L, b)) continue;
    off += (x.R - 1) * x.NS;
  }
  return off;
}

// ------------------------------------------------------------ Stockham pass
// One radix-R pass over the LINES lines of NTILES consecutive tiles
// (TILE_ELEMS apart) of length L.  NS is the product of the radices of the
// previous passes.  ``tw`` holds NTAB entries.  ``pre(m, line, v)`` may
// transform each input element as it is loaded (used to fold a spectral
// multiplier into the first pass of a transform).
// Called by fft_mul_ifft once its first pass (which reads no twiddles) has
// been written to shared memory, before the second pass reads the table.
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};

struct NoPre {
  template <typename V> __device__ __forceinline__ V operator()(int, int, int, V v) const { return v; }
};

// PT: ``tw`` points at this pass's block of a pass table (see ptw_offset).
template <typename T, int L, int R, int NS, int LINES, int NTILES, int NT, bool INV, int NTAB, bool PT = false,
          class Pre = NoPre>
__device__ __forceinline__ void stockham_pass(c2<T>* __restrict__ buf, const c2<T>* __restrict__ tw, int tid,
                                              Pre pre = Pre()) {
  constexpr int NB = L / R;                   // butterflies per line
  constexpr int TOT = NB * LINES * NTILES;    // butterflies in the pass
  constexpr int PER = (TOT + NT - 1) / NT;
  constexpr int TILE_ELEMS = L * LINES;
  constexpr int TWS = NTAB / (NS * R);        // table stride for W_{NS*R}
  static_assert(NTAB % (NS * R) == 0, "twiddle table too small");
  c2<T> v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int idx = tid + b * NT;
    if (TOT % NT == 0 || idx < TOT) {
      const int line = idx % LINES;
      const int rest = idx / LINES;
      const int j = rest % NB;
      const int tile = rest / NB;
      const c2<T>* tb = buf + tile * TILE_ELEMS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = pre(tile, j + r * NB, line, tb[sw<T, LINES>(j + r * NB, line)]);
      if constexpr (NS > 1) {
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = twmul<T, INV>(v[b][r], PT ? tw[(r - 1) * NS + k] : tw[r * k * TWS]);
      }
      dft<R, T, INV>(v[b]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int idx = tid + b * NT;
    if (TOT % NT == 0 || idx < TOT) {
      const int line = idx % LINES;
      const int rest = idx / LINES;
      const int j = rest % NB;
      const int tile = rest / NB;
      c2<T>* tb = buf + tile * TILE_ELEMS;
      const int k = j % NS;
      const int base = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) tb[sw<T, LINES>(base + r * NS, line)] = v[b][r];
    }
  }
  __syncthreads();
}

// Full transform of length L on NTILES consecutive tiles (LINES lines each);
// ``pre`` is applied to the elements as the first pass loads them.
// Radix plans: 32 = 8x4, 64 = 8x8, 128 = 8x16, 256 = 16x16, 512 = 8x8x8, 1024 = 16x8x8.
template <typename T, int L, int LINES, int NTILES, int NT, bool INV, int NTAB, class Pre = NoPre>
__device__ __forceinline__ void fft_tiles(c2<T>* buf, const c2<T>* tw, int tid, Pre pre = Pre()) {
  if constexpr (L == 32) {
    stockham_pass<T, L, 8, 1, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid, pre);
    stockham_pass<T, L, 4, 8, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
  } else if constexpr (L == 64) {
    stockham_pass<T, L, 8, 1, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid, pre);
    stockham_pass<T, L, 8, 8, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
  } else if constexpr (L == 128) {
    stockham_pass<T, L, 8, 1, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid, pre);
    stockham_pass<T, L, 16, 8, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
  } else if constexpr (L == 256) {
    stockham_pass<T, L, 16, 1, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid, pre);
    stockham_pass<T, L, 16, 16, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
  } else if constexpr (L == 512) {
    stockham_pass<T, L, 8, 1, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid, pre);
    stockham_pass<T, L, 8, 8, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
    stockham_pass<T, L, 8, 64, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
  } else if constexpr (L == 1024) {
    stockham_pass<T, L, 16, 1, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid, pre);
    stockham_pass<T, L, 8, 16, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
    stockham_pass<T, L, 8, 128, LINES, NTILES, NT, INV, NTAB>(buf, tw, tid);
  } else {
    static_assert(L == 32, "unsupported transform length");
  }
}

// ------------------------------------------------ register-level passes
// The pieces of one Stockham pass over the LINES lines of a single tile, for
// callers that keep a pass's outputs in registers: ``sp_read`` gathers the R
// inputs of each of the thread's butterflies from ``src(m, line)`` (shared
// memory or global), twiddles and transforms them; ``sp_apply`` /
// ``sp_emit`` visit the outputs at their natural positions m; ``sp_write``
// stores them to the tile.  Butterfly b of a thread is (line, j) =
// (idx % LINES, idx / LINES) with idx = tid + b * NT, as in stockham_pass.
template <int L, int R, int LINES, int NT> struct SpGeom {
  static constexpr int NB = L / R;
  static constexpr int TOT = NB * LINES;
  static constexpr int PER = (TOT + NT - 1) / NT;
};

template <typename T, int L, int R, int NS, int LINES, int NT, bool INV, int NTAB, bool PT, class Src>
__device__ __forceinline__ void sp_read(c2<T> (&v)[SpGeom<L, R, LINES, NT>::PER][R], Src src,
                                        const c2<T>* tw, int tid) {
  using G = SpGeom<L, R, LINES, NT>;
  constexpr int TWS = NTAB / (NS * R);
  static_assert(NTAB % (NS * R) == 0, "twiddle table too small");
#pragma unroll
  for (int b = 0; b < G::PER; ++b) {
    const int idx = tid + b * NT;
    if (G::TOT % NT == 0 || idx < G::TOT) {
      const int line = idx % LINES, j = idx / LINES;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = src(j + r * G::NB, line);
      if constexpr (NS > 1) {
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = twmul<T, INV>(v[b][r], PT ? tw[(r - 1) * NS + k] : tw[r * k * TWS]);
      }
      dft<R, T, INV>(v[b]);
    }
  }
}

// f(m, line, x) -> x' for every output of the thread's butterflies (in place).
template <typename T, int L, int R, int NS, int LINES, int NT, class F>
__device__ __forceinline__ void sp_apply(c2<T> (&v)[SpGeom<L, R, LINES, NT>::PER][R], F f, int tid) {
  using G = SpGeom<L, R, LINES, NT>;
#pragma unroll
  for (int b = 0; b < G::PER; ++b) {
    const int idx = tid + b * NT;
    if (G::TOT % NT == 0 || idx < G::TOT) {
      const int line = idx % LINES, j = idx / LINES;
      const int base = (j / NS) * NS * R + j % NS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = f(base + r * NS, line, v[b][r]);
    }
  }
}

template <typename T, int L, int R, int NS, int LINES, int NT, class Dst>
__device__ __forceinline__ void sp_emit(c2<T> (&v)[SpGeom<L, R, LINES, NT>::PER][R], Dst dst, int tid) {
  sp_apply<T, L, R, NS, LINES, NT>(v, [=](int m, int line, c2<T> x) { dst(m, line, x); return x; }, tid);
}

template <typename T, int L, int R, int NS, int LINES, int NT>
__device__ __forceinline__ void sp_write(c2<T>* buf, c2<T> (&v)[SpGeom<L, R, LINES, NT>::PER][R], int tid) {
  sp_emit<T, L, R, NS, LINES, NT>(v, [=](int m, int line, c2<T> x) { buf[sw<T, LINES>(m, line)] = x; }, tid);
}

// Two-pass form of fft_mul_ifft for a plan L = R1 x R2: the forward pass 2
// (radix R2 after R1, twiddles ``twf``), ``mul``, the inverse pass 1 (radix
// R2, no twiddles) in registers, then the inverse pass 2 (radix R1 after R2,
// twiddles ``twi``).  Shared memory sees one store and one load of the tile
// per direction.  ``twf`` and ``twi`` are pass-table blocks: W^{r k} at
// (r - 1) NS + k.
template <typename T, int L, int R1, int R2, int LINES, int NT, class Src, class Mul, class Dst, class Hook = NoHook>
__device__ __forceinline__ void fft_mul_ifft_2p(c2<T>* buf, const c2<T>* twf, const c2<T>* twi, int tid, Src src,
                                                Mul mul, Dst dst, Hook hook = Hook()) {
  static_assert(R1 * R2 == L, "plan");
  auto smem = [=](int m, int line) { return buf[sw<T, LINES>(m, line)]; };
  c2<T> a[SpGeom<L, R1, LINES, NT>::PER][R1];
  c2<T> b[SpGeom<L, R2, LINES, NT>::PER][R2];
  sp_read<T, L, R1, 1, LINES, NT, false, L, true>(a, src, twf, tid);
  sp_write<T, L, R1, 1, LINES, NT>(buf, a, tid);
  __syncthreads();
  hook();
  sp_read<T, L, R2, R1, LINES, NT, false, L, true>(b, smem, twf, tid);
  sp_apply<T, L, R2, R1, LINES, NT>(b, mul, tid);
#pragma unroll
  for (int i = 0; i < SpGeom<L, R2, LINES, NT>::PER; ++i) {
    if (SpGeom<L, R2, LINES, NT>::TOT % NT == 0 || tid + i * NT < SpGeom<L, R2, LINES, NT>::TOT)
      dft<R2, T, true>(b[i]);
  }
  __syncthreads();
  sp_write<T, L, R2, 1, LINES, NT>(buf, b, tid);
  __syncthreads();
  sp_read<T, L, R1, R2, LINES, NT, true, L, true>(a, smem, twi, tid);
  sp_emit<T, L, R1, R2, LINES, NT>(a, dst, tid);
}

// Column table: the two-pass plan 512 = 16 x 32 of the column pass.  Block
// (R 32, NS 16) of the forward pass 2 at entry 0, block (R 16, NS 32) of the
// inverse pass 2 after it; lengths without a two-pass column plan have none.
__host__ __device__ constexpr bool col2_plan(int L) { return L == 512; }
__host__ __device__ constexpr int col2_r1(int) { return 16; }
__host__ __device__ constexpr int col2_r2(int) { return 32; }
__host__ __device__ constexpr int ctw_inv_offset(int L) { return col2_plan(L) ? (col2_r2(L) - 1) * col2_r1(L) : 0; }
__host__ __device__ constexpr int ctw_size(int L) {
  return col2_plan(L) ? ctw_inv_offset(L) + (col2_r1(L) - 1) * col2_r2(L) : 0;
}

// src -> FFT -> mul -> IFFT -> dst for the LINES lines of one tile, with the
// forward plan's last pass and the inverse plan's first pass fused in
// registers.  The inverse runs the forward radices in reverse order, so both
// fused passes have the same radix R and the same butterfly positions: the
// forward pass leaves x[j + r L/R] in a thread's registers, which is exactly
// the input set of the inverse pass's butterfly j.  The first pass reads
// ``src(m, line)`` directly and the last pass hands its outputs to
// ``dst(m, line, x)``, so shared memory sees 2 * (passes - 1) sweeps instead
// of 2 * (2 passes + 1).  ``mul(m, line, x)`` gets the spectrum at frequency m.
// Plans: 32 = 8x4, 64 = 8x8, 128 = 8x16, 256 = 16x16, 512 = 8x8x8, 1024 = 16x8x8.
// ``tw`` is the pass table of length L (ptw_size(L) entries).
template <typename T, int L, int LINES, int NT, class Src, class Mul, class Dst, class Hook = NoHook>
__device__ __forceinline__ void fft_mul_ifft(c2<T>* buf, const c2<T>* tw, int tid, Src src, Mul mul,
                                             Dst dst, Hook hook = Hook()) {
  auto smem = [=](int m, int line) { return buf[sw<T, LINES>(m, line)]; };
  constexpr int R1 = plan_r1(L), R2 = plan_r2(L), R3 = plan_r3(L);
  // pass-table blocks (``tw`` is the pass table of length L); first passes read no twiddles
  constexpr int OF2 = ptw_offset(L, R2, R1), OF3 = ptw_offset(L, R3, R1 * R2);
  constexpr int OI2 = ptw_offset(L, R3 == 1 ? R1 : R2, R3 == 1 ? R2 : R3);
  constexpr int OI3 = ptw_offset(L, R1, R3 * R2);
  static_assert(OF2 >= 0 && OI2 >= 0 && (R3 == 1 || (OF3 >= 0 && OI3 >= 0)), "pass table block missing");
  static_assert(L == 32 || L == 64 || L == 128 || L == 256 || L == 512 || L == 1024, "unsupported length");
  if constexpr (R3 == 1) {
    fft_mul_ifft_2p<T, L, R1, R2, LINES, NT>(buf, tw + OF2, tw + OI2, tid, src, mul, dst, hook);
  } else {
    static_assert(R1 * R2 * R3 == L, "plan");
    c2<T> a[SpGeom<L, R1, LINES, NT>::PER][R1];
    c2<T> b[SpGeom<L, R2, LINES, NT>::PER][R2];
    c2<T> c[SpGeom<L, R3, LINES, NT>::PER][R3];
    sp_read<T, L, R1, 1, LINES, NT, false, L, true>(a, src, tw, tid);
    sp_write<T, L, R1, 1, LINES, NT>(buf, a, tid);
    __syncthreads();
    hook();
    sp_read<T, L, R2, R1, LINES, NT, false, L, true>(b, smem, tw + OF2, tid);
    __syncthreads();
    sp_write<T, L, R2, R1, LINES, NT>(buf, b, tid);
    __syncthreads();
    sp_read<T, L, R3, R1 * R2, LINES, NT, false, L, true>(c, smem, tw + OF3, tid);
    sp_apply<T, L, R3, R1 * R2, LINES, NT>(c, mul, tid);
#pragma unroll
    for (int i = 0; i < SpGeom<L, R3, LINES, NT>::PER; ++i) {
      if (SpGeom<L, R3, LINES, NT>::TOT % NT == 0 || tid + i * NT < SpGeom<L, R3, LINES, NT>::TOT)
        dft<R3, T, true>(c[i]);
    }
    __syncthreads();
    sp_write<T, L, R3, 1, LINES, NT>(buf, c, tid);
    __syncthreads();
    sp_read<T, L, R2, R3, LINES, NT, true, L, true>(b, smem, tw + OI2, tid);
    __syncthreads();
    sp_write<T, L, R2, R3, LINES, NT>(buf, b, tid);
    __syncthreads();
    sp_read<T, L, R1, R3 * R2, LINES, NT, true, L, true>(a, smem, tw + OI3, tid);
    sp_emit<T, L, R1, R3 * R2, LINES, NT>(a, dst, tid);
  }
}

// ----------------------------------------------------- real-FFT packing
// Rows of N real samples are held as H = N/2 complex values z[m] = x[2m] + i x[2m+1].
// The packed half spectrum of a row keeps X[k] for 1 <= k < H in slot k and
// (X[0], X[H]) -- both real for a real row -- as (re, im) of slot 0.
// twN[k] = exp(-2 pi i k / N).

// After a forward length-H FFT of z: turn Y into the packed spectrum X, in place.
template <typename T, int H, int LINES, int NTILES, int NT>
__device__ __forceinline__ void r2c_post(c2<T>* buf, const c2<T>* twN, int tid) {
  constexpr int ITEMS = (H / 2 + 1) * LINES * NTILES;
  constexpr int TILE_ELEMS = H * LINES;
  for (int idx = tid; idx < ITEMS; idx += NT) {
    const int line = idx % LINES;
    const int rest = idx / LINES;
    const int k = rest % (H / 2 + 1);
    c2<T>* tb = buf + (rest / (H / 2 + 1)) * TILE_ELEMS;
    if (k == 0) {
      c2<T> y = tb[sw<T, LINES>(0, line)];
      tb[sw<T, LINES>(0, line)] = mk<T>(y.x + y.y, y.x - y.y);
    } else {
      const c2<T> yk = tb[sw<T, LINES>(k, line)];
      const c2<T> yc = cconj<T>(tb[sw<T, LINES>(H - k, line)]);
      const c2<T> e = cscale<T>(cadd<T>(yk, yc), T(0.5));
      // O = (yk - yc) / (2i) = -i/2 (yk - yc)
      const c2<T> d = csub<T>(yk, yc);
      const c2<T> o = mk<T>(T(0.5) * d.y, T(-0.5) * d.x);
      const c2<T> wo = cmul<T>(o, twN[k]);
      tb[sw<T, LINES>(k, line)] = cadd<T>(e, wo);
      if (k != H - k) tb[sw<T, LINES>(H - k, line)] = cconj<T>(csub<T>(e, wo));
    }
  }
  __syncthreads();
}

// Before an inverse length-H FFT: turn the packed spectrum X into Z, in place,
// so that IFFT_H(Z) = unnormalised inverse real DFT of X (x[2m] + i x[2m+1]).
// The imaginary parts of X[0] and X[H] are never used, exactly as irfft does.
// ``in(tile, k, line, x)`` may transform each packed input element X[k] as it
// is read (k = 0 is the (X0, XH) slot); it lets callers fold a spectral
// multiplier into this pass.
template <typename T, int H, int LINES, int NTILES, int NT, class In = NoPre>
__device__ __forceinline__ void c2r_pre(c2<T>* buf, const c2<T>* twN, int tid, In in = In()) {
  constexpr int ITEMS = (H / 2 + 1) * LINES * NTILES;
  constexpr int TILE_ELEMS = H * LINES;
  for (int idx = tid; idx < ITEMS; idx += NT) {
    const int line = idx % LINES;
    const int rest = idx / LINES;
    const int k = rest % (H / 2 + 1);
    const int tile = rest / (H / 2 + 1);
    c2<T>* tb = buf + tile * TILE_ELEMS;
    if (k == 0) {
      c2<T> x = in(tile, 0, line, tb[sw<T, LINES>(0, line)]);  // (X0, XH)
      tb[sw<T, LINES>(0, line)] = mk<T>(x.x + x.y, x.x - x.y);
    } else {
      const c2<T> a = in(tile, k, line, tb[sw<T, LINES>(k, line)]);
      const c2<T> bc = cconj<T>(in(tile, H - k, line, tb[sw<T, LINES>(H - k, line)]));
      const c2<T> p = cadd<T>(a, bc);
      // q = i * W^{-k} (a - bc), W^{-k} = conj(twN[k])
      const c2<T> q = cmul_i<T>(cmulc<T>(csub<T>(a, bc), twN[k]));
      tb[sw<T, LINES>(k, line)] = cadd<T>(p, q);
      if (k != H - k) tb[sw<T, LINES>(H - k, line)] = cconj<T>(csub<T>(p, q));
    }
  }
  __syncthreads();
}

// -------------------------------------------------- global <-> tile moves
// Row tile: rows [0, LINES) of a row-major array (row stride ``ld`` elements),
// elements [0, E) of each row.  Row-major thread mapping: coalesced.
template <typename T, typename G, int E, int LINES, int NT>
__device__ __forceinline__ void load_rows(c2<T>* tile, const G* __restrict__ g, long ld, int tid) {
  if constexpr (std::is_same<T, float>::value && std::is_same<G, float2>::value && E % 2 == 0) {
    // 16-byte loads of two consecutive elements (ld even, rows 16-byte aligned)
    constexpr int E2 = E / 2;
#pragma unroll 4
    for (int idx = tid; idx < E2 * LINES; idx += NT) {
      const int row = idx / E2, m2 = idx % E2;
      const float4 v = reinterpret_cast<const float4*>(g + row * ld)[m2];
      tile[sw<T, LINES>(2 * m2, row)] = make_float2(v.x, v.y);
      tile[sw<T, LINES>(2 * m2 + 1, row)] = make_float2(v.z, v.w);
    }
  } else {
#pragma unroll 4
    for (int idx = tid; idx < E * LINES; idx += NT) {
      const int row = idx / E, m = idx % E;
      const G v = g[row * ld + m];
      tile[sw<T, LINES>(m, row)] = mk<T>(T(v.x), T(v.y));
    }
  }
}

template <typename T, typename G, int E, int LINES, int NT>
__device__ __forceinline__ void store_rows(G* __restrict__ g, long ld, const c2<T>* tile, int tid) {
  if constexpr (std::is_same<T, float>::value && std::is_same<G, float2>::value && E % 2 == 0) {
    constexpr int E2 = E / 2;
#pragma unroll 4
    for (int idx = tid; idx < E2 * LINES; idx += NT) {
      const int row = idx / E2, m2 = idx % E2;
      const float2 a0 = tile[sw<T, LINES>(2 * m2, row)], a1 = tile[sw<T, LINES>(2 * m2 + 1, row)];
      reinterpret_cast<float4*>(g + row * ld)[m2] = make_float4(a0.x, a0.y, a1.x, a1.y);
    }
  } else {
#pragma unroll 4
    for (int idx = tid; idx < E * LINES; idx += NT) {
      const int row = idx / E, m = idx % E;
      const c2<T> v = tile[sw<T, LINES>(m, row)];
      G o;
      o.x = v.x;
      o.y = v.y;
      g[row * ld + m] = o;
    }
  }
}

// Column tile: lines [c0, c0+LINES) (clipped to ``ncols``) of an (L x ld)
// row-major complex array; line-major mapping: coalesced LINES-wide rows.
template <typename T, int L, int LINES, int NT>
__device__ __forceinline__ void load_cols(c2<T>* tile, const c2<T>* __restrict__ g, long ld, int c0, int ncols,
                                          int tid) {
  if constexpr (std::is_same<T, float>::value) {
    if ((ld & 1) == 0 && (c0 & 1) == 0 && c0 + LINES <= ncols) {
      // full tile of an even-width array: 16-byte loads of two adjacent lines
#pragma unroll 4
      for (int idx = tid; idx < L * (LINES / 2); idx += NT) {
        const int m = idx / (LINES / 2), lp = idx % (LINES / 2);
        const float4 v = *reinterpret_cast<const float4*>(g + m * ld + c0 + 2 * lp);
        tile[sw<T, LINES>(m, 2 * lp)] = make_float2(v.x, v.y);
        tile[sw<T, LINES>(m, 2 * lp + 1)] = make_float2(v.z, v.w);
      }
      return;
    }
  }
#pragma unroll 4
  for (int idx = tid; idx < L * LINES; idx += NT) {
    const int m = idx / LINES, line = idx % LINES;
    const int c = c0 + line;
    tile[sw<T, LINES>(m, line)] = (c < ncols) ? g[m * ld + c] : mk<T>(T(0), T(0));
  }
}

template <typename T, int L, int LINES, int NT>
__device__ __forceinline__ void store_cols(c2<T>* __restrict__ g, long ld, int c0, int ncols, const c2<T>* tile,
                                           int tid) {
  if constexpr (std::is_same<T, float>::value) {
    if ((ld & 1) == 0 && (c0 & 1) == 0 && c0 + LINES <= ncols) {
#pragma unroll 4
      for (int idx = tid; idx < L * (LINES / 2); idx += NT) {
        const int m = idx / (LINES / 2), lp = idx % (LINES / 2);
        const float2 a0 = tile[sw<T, LINES>(m, 2 * lp)], a1 = tile[sw<T, LINES>(m, 2 * lp + 1)];
        *reinterpret_cast<float4*>(g + m * ld + c0 + 2 * lp) = make_float4(a0.x, a0.y, a1.x, a1.y);
      }
      return;
    }
  }
#pragma unroll 4
  for (int idx = tid; idx < L * LINES; idx += NT) {
    const int m = idx / LINES, line = idx % LINES;
    const int c = c0 + line;
    if (c < ncols) g[m * ld + c] = tile[sw<T, LINES>(m, line)];
  }
}

}  // namespace lf
