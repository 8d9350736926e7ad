// C ABI of the LenseFlow engine: plans, launch sequencing, validation.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/lenseflow.h"
#include "lf_kernels.cuh"

using namespace lf;

// Launch timing: when enabled, an event pair brackets every launch on the
// launching stream, tagged with the kernel kind (LF_KIND_*).
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<int> kind;  // one per recorded launch
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      pool.push_back(e);
    }
    return pool[used++];
  }
};

struct lf_plan_s {
  Prof prof;
  int N;
  int C;
  int prec;
  double pix_width;
  int device;
  void* tw;        // N complex values in the compute precision
  double2* tw64;   // N complex float64 (phi precompute)
  void* twp;       // pass table of length N, then the column table, in the compute precision
  const void* twc() const {  // the column table inside twp
    return static_cast<const char*>(twp) + (prec == LF_F64 ? sizeof(double2) : sizeof(float2)) * ptw_size(N);
  }
};

// Pass table of length L (layout: ptw_offset / ptw_size): store(i, cos, sin)
// for every entry, values computed in float64.
template <class Store>
static void fill_pass_table(int L, Store store) {
  for (int b = 0; b < 4; ++b) {
    const PtwBlock x = ptw_candidate(L, b);
    if (x.R == 0 || ptw_repeats(L, b)) continue;
    const int off = ptw_offset(L, x.R, x.NS);
    for (int r = 1; r < x.R; ++r)
      for (int k = 0; k < x.NS; ++k) {
        const double ang = -2.0 * M_PI * (double)r * (double)k / ((double)x.R * (double)x.NS);
        store(off + (r - 1) * x.NS + k, std::cos(ang), std::sin(ang));
      }
  }
}

// Column table of the two-pass column plan (layout: ctw_inv_offset /
// ctw_size): the forward pass-2 block (R2 after R1), then the inverse pass-2
// block (R1 after R2); W^{r k} at (r - 1) NS + k of each, float64 values.
template <class Store>
static void fill_col_table(int L, Store store) {
  if (!col2_plan(L)) return;
  const int blocks[2][3] = {{col2_r2(L), col2_r1(L), 0}, {col2_r1(L), col2_r2(L), ctw_inv_offset(L)}};
  for (const auto& b : blocks) {
    const int R = b[0], NS = b[1], off = b[2];
    for (int r = 1; r < R; ++r)
      for (int k = 0; k < NS; ++k) {
        const double ang = -2.0 * M_PI * (double)r * (double)k / ((double)R * (double)NS);
        store(off + (r - 1) * NS + k, std::cos(ang), std::sin(ang));
      }
  }
}

namespace {

constexpr int kVersion = 100;

bool valid_n(int n) { return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024; }

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return LF_OK;
  if (e == cudaErrorMemoryAllocation) return LF_ERR_OOM;
  return LF_ERR_CUDA;
}

// Launch geometry per (precision, N).
template <typename T> struct Geo;
// FP32 stage kernels: enough warps per SM to keep ~50 KB of loads in flight;
// minb() caps registers at 64 per thread so that many blocks fit.  The row
// pass runs 4-row tiles in half-size blocks: four blocks per SM (32 warps)
// whose load, transform and epilogue phases drift apart keep HBM busier than
// two 8-row blocks (7.46 vs 7.76 ms per 64-map 512^2 QU step; 2-row tiles in
// eight blocks per SM: 8.73 ms).
template <> struct Geo<float> {
  static constexpr int LINES = 16;     // column-pass tile
  static constexpr int ROW_LINES = 4;  // row-pass tile (all C components at once)
  static constexpr int nt(int n) { return n <= 64 ? 128 : (n <= 256 ? 256 : (n <= 512 ? 512 : 1024)); }
  static constexpr int minb(int n) { return 65536 / (nt(n) * 64); }
  static constexpr int row_nt(int n) { return nt(n) / 2; }
  // three components keep more values live in the epilogue: up to 85 registers
  // (64 spilled 100-250 bytes per thread)
  static constexpr int row_minb(int n, int c = 1) { return 65536 / (row_nt(n) * (c >= 3 ? 80 : 64)); }
};
template <> struct Geo<double> {
  static constexpr int LINES = 8;
  static constexpr int ROW_LINES = 4;
  static constexpr int nt(int n) { return n <= 64 ? 64 : (n <= 128 ? 128 : (n <= 512 ? 256 : 512)); }
  static constexpr int minb(int) { return 1; }
  static constexpr int row_nt(int n) { return nt(n); }
  static constexpr int row_minb(int, int = 1) { return 1; }
};

// Opt in to > 48 KB of dynamic shared memory once per kernel and device.
// Host threads may launch concurrently (a plan per thread, the allocation-free
// entry point): the per-device high-water mark is an atomic, and a racing
// thread at worst sets the same attribute twice.
template <auto Kernel>
cudaError_t ensure_smem(size_t smem) {
  static std::atomic<size_t> done[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (done[dev].load(std::memory_order_relaxed) >= smem) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    size_t cur = done[dev].load(std::memory_order_relaxed);
    while (cur < smem && !done[dev].compare_exchange_weak(cur, smem, std::memory_order_relaxed)) {
    }
  }
  return e;
}

// ------------------------------------------------------ wait timeouts
// One mapped pinned host word per process; its device address goes to
// g_lf_timeout_host on every device that creates a plan.  Kernels whose
// bounded wait runs out set it; entry points read it (no synchronisation)
// and return LF_ERR_TIMEOUT while it is set.
std::mutex g_flag_mu;
std::atomic<int*> g_host_flag{nullptr};
bool g_flag_on_device[64] = {false};

cudaError_t ensure_timeout_flag() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_flag_mu);
  if (!g_host_flag.load()) {
    void* h = nullptr;
    e = cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) return e;
    *static_cast<volatile int*>(h) = 0;
    g_host_flag.store(static_cast<int*>(h));
  }
  if (!g_flag_on_device[dev]) {
    int* d = nullptr;
    e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&d), g_host_flag.load(), 0);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_lf_timeout_host, &d, sizeof(d));
    if (e != cudaSuccess) return e;
    g_flag_on_device[dev] = true;
  }
  return cudaSuccess;
}

// True once a kernel has recorded a timeout that no lf_wait_timeouts reset has cleared.
bool timeout_recorded() {
  const int* h = g_host_flag.load(std::memory_order_acquire);
  return h && *reinterpret_cast<const volatile int*>(h) != 0;
}

thread_local Prof* g_prof = nullptr;  // profiler of the plan whose call is running on this thread

// Set while a lens issues its stage kernels after the first one: those
// launches carry the programmatic-dependent-launch attribute (every stage
// kernel waits for its predecessor before touching shared buffers).
thread_local bool g_pdl = false;

struct PdlScope {
  bool on = false;
  void enable() { g_pdl = on = true; }
  ~PdlScope() {
    if (on) g_pdl = false;
  }
};

template <auto Kernel, typename... Args>
cudaError_t launch_k(int kind, dim3 grid, int nt, size_t smem, cudaStream_t st, Args... args) {
  cudaError_t e = ensure_smem<Kernel>(smem);
  if (e != cudaSuccess) return e;
  Prof* pf = (g_prof && g_prof->on) ? g_prof : nullptr;
  if (g_pdl && !pf) {  // events between the launches would serialise them anyway
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(nt);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, Kernel, args...);
  }
  cudaEvent_t e0 = pf ? pf->next() : nullptr, e1 = pf ? pf->next() : nullptr;
  if (e0) cudaEventRecord(e0, st);
  Kernel<<<grid, nt, smem, st>>>(args...);
  e = cudaGetLastError();
  if (e1) {
    cudaEventRecord(e1, st);
    pf->kind.push_back(kind);
  }
  return e;
}

template <auto Kernel, typename... Args>
cudaError_t launch(dim3 grid, int nt, size_t smem, cudaStream_t st, Args... args) {
  return launch_k<Kernel>(LF_KIND_PHI, grid, nt, smem, st, args...);
}

// One column pass over `planes` packed row-spectrum planes.  FP32 512: the
// two-pass plan 16 x 32 in 256-thread blocks; otherwise the pass-table plan.
template <typename T, int N>
cudaError_t launch_col(int planes, cudaStream_t st, const StageArgs& a) {
  constexpr int LINES = Geo<T>::LINES;
  const dim3 grid(N / 2 / LINES, planes);
  if constexpr (std::is_same<T, float>::value && col2_plan(N)) {
    // 16-line tiles (128-byte row segments), 256 threads (one radix-32 butterfly each), 2 blocks per SM
    constexpr int NT2 = 256;
    const size_t smem = sizeof(c2<T>) * (col_tw_entries(N, true) + LINES * N) + 16;  // + the table's mbarrier
    return launch_k<k_col<T, N, LINES, NT2, 2, true>>(LF_KIND_COL, grid, NT2, smem, st, a);
  } else {
    constexpr int NT = Geo<T>::nt(N);
    const size_t smem = sizeof(c2<T>) * (col_tw_entries(N) + LINES * N) + 16;  // + the table's mbarrier
    return launch_k<k_col<T, N, LINES, NT, Geo<T>::minb(N)>>(LF_KIND_COL, grid, NT, smem, st, a);
  }
}

// The p planes hold p = M(t)^-1 grad(phi) at the 2n+1 times k / (2n), k = 0..2n, ascending; an
// integration from t0 = 1 reads time t0 + k hh at index 2n - k.  ``pp_given``: the caller supplies
// them (lf_lense_flow_pp), otherwise k_p_planes forms them from the derivative planes first.
template <typename T, int N, int C, bool ADJ, bool PP>
cudaError_t run_lens_pp(const StageArgs& base, int B, int nsteps, double t0, double t1, cudaStream_t st,
                        bool pp_given = false) {
  constexpr int RL = Geo<T>::ROW_LINES;
  constexpr int RNT = Geo<T>::row_nt(N);
  constexpr int RMB = Geo<T>::row_minb(N, C);
  constexpr int H = N / 2;
  const size_t smem_row = sizeof(c2<T>) * (N + 2 * C * RL * H) + 16;  // + the table's mbarrier
  const dim3 grow(N / RL, B);
  StageArgs a = base;
  cudaError_t e;
  const double h = (t1 - t0) / nsteps;  // util.py:185
  const double hh = h / 2.0;
  if constexpr (PP) {
    a.pp_k = 2 * nsteps + 1;
    if (!pp_given) {  // p at the times k / (2n), ascending
      const long P = (long)N * N;
      const int gx = (int)std::min<long>((P / 2 + 255) / 256, 1024);
      e = launch_k<k_p_planes<T>>(LF_KIND_PP, dim3(gx, B), 256, 0, st, reinterpret_cast<const T*>(a.phi),
                                  reinterpret_cast<T*>(const_cast<void*>(a.pp)), P, a.pp_k, 0.0,
                                  0.5 / nsteps);
      if (e != cudaSuccess) return e;
    }
  }
  const bool rev = t0 != 0.0;  // time t0 + k hh sits at index 2n - k
  auto pidx = [=](int k) { return rev ? 2 * nsteps - k : k; };
  a.h = h;
  a.stage = 0;
  a.last = 0;
  a.t_cur = t0;
  a.t_next = t0;
  a.pp_idx = pidx(0);
  // Programmatic dependent launch for small batches (up to 2^23 pixels, 16 maps of 512^2 QU):
  // measured per 512^2 QU lens with the phi precompute, 4 maps 0.79 -> 0.66 ms, 16 maps 2.35 ->
  // 2.25 ms, but 64 maps 7.85 -> 8.13 ms.  The initial transform follows k_p_planes (which has no
  // dependency wait) or the caller's work and is launched plainly; every later stage kernel waits
  // for its predecessor itself.
  const bool use_pdl = (long)B * C * N * N <= (1L << 23);
  PdlScope pdl;
  if (PP && use_pdl) pdl.enable();
  e = launch_k<k_row<T, N, C, ADJ, true, RL, RNT, false, RMB, PP>>(LF_KIND_ROW, grow, RNT, smem_row, st, a);
  if (e != cudaSuccess) return e;
  if (use_pdl) pdl.enable();
  for (int i = 0; i < nsteps; ++i) {
    const double t = t0 + i * h;  // util.py:189
    const double tc[4] = {t, t + hh, t + hh, t + h};
    const double tn[4] = {t + hh, t + hh, t + h, t0 + (i + 1) * h};
    // the same times as indices k of t0 + k hh
    const int kc[4] = {2 * i, 2 * i + 1, 2 * i + 1, 2 * i + 2};
    const int kn[4] = {2 * i + 1, 2 * i + 1, 2 * i + 2, 2 * i + 2};
    for (int s = 0; s < 4; ++s) {
      a.stage = s + 1;
      a.t_cur = tc[s];
      a.t_next = tn[s];
      a.pp_idx = pidx(ADJ ? kn[s] : kc[s]);
      a.last = (i == nsteps - 1 && s == 3);
      e = launch_col<T, N>(B * C, st, a);
      if (e != cudaSuccess) return e;
      if constexpr (PP && C == 2 && !ADJ && N == 512 && std::is_same<T, float>::value) {
        // two components: full-length complex transforms, update fused in registers;
        // 2-row tiles, 128 threads (measured best of 1, 2 and 4 rows: 6.81, 5.48 and
        // 5.96 ms of row passes per 64-map step), six blocks per SM
        constexpr int PL = 2, PNT = (N / 8) * PL;
        e = launch_k<k_row_pair<N, PL, PNT, 6>>(LF_KIND_ROW, dim3(N / PL, B), PNT, row_pair_smem_bytes<PL>(N),
                                                st, a);
      } else if constexpr (PP && C == 2 && ADJ && N == 512 && std::is_same<T, float>::value) {
        // adjoint counterpart: one inverse transform for both rates, two forward
        // transforms (p_x y, p_y y) for the next stage; same tile shape
        constexpr int PL = 2, PNT = (N / 8) * PL;
        e = launch_k<k_row_pair_adj<N, PL, PNT, 6>>(LF_KIND_ROW, dim3(N / PL, B), PNT,
                                                    row_pair_smem_bytes<PL>(N), st, a);
      } else {
        e = launch_k<k_row<T, N, C, ADJ, false, RL, RNT, false, RMB, PP>>(LF_KIND_ROW, grow, RNT, smem_row, st, a);
      }
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

// The p-plane path (a.pp set) is built for float32 plans only.
template <typename T, int N, int C, bool ADJ>
cudaError_t run_lens_n(const StageArgs& a, int B, int nsteps, double t0, double t1, cudaStream_t st, bool pp_given) {
  if constexpr (std::is_same<T, float>::value) {
    if (a.pp) return run_lens_pp<T, N, C, ADJ, true>(a, B, nsteps, t0, t1, st, pp_given);
  }
  return run_lens_pp<T, N, C, ADJ, false>(a, B, nsteps, t0, t1, st);
}

template <typename T, int N>
cudaError_t run_lens_c(int C, bool adj, const StageArgs& a, int B, int nsteps, double t0, double t1,
                       cudaStream_t st, bool pp_given) {
  if (C == 1) return adj ? run_lens_n<T, N, 1, true>(a, B, nsteps, t0, t1, st, pp_given) : run_lens_n<T, N, 1, false>(a, B, nsteps, t0, t1, st, pp_given);
  if (C == 2) return adj ? run_lens_n<T, N, 2, true>(a, B, nsteps, t0, t1, st, pp_given) : run_lens_n<T, N, 2, false>(a, B, nsteps, t0, t1, st, pp_given);
  return adj ? run_lens_n<T, N, 3, true>(a, B, nsteps, t0, t1, st, pp_given) : run_lens_n<T, N, 3, false>(a, B, nsteps, t0, t1, st, pp_given);
}

template <typename T>
cudaError_t run_lens(int N, int C, bool adj, const StageArgs& a, int B, int nsteps, double t0, double t1,
                     cudaStream_t st, bool pp_given = false) {
  switch (N) {
    case 64: return run_lens_c<T, 64>(C, adj, a, B, nsteps, t0, t1, st, pp_given);
    case 128: return run_lens_c<T, 128>(C, adj, a, B, nsteps, t0, t1, st, pp_given);
    case 256: return run_lens_c<T, 256>(C, adj, a, B, nsteps, t0, t1, st, pp_given);
    case 512: return run_lens_c<T, 512>(C, adj, a, B, nsteps, t0, t1, st, pp_given);
    default: return run_lens_c<T, 1024>(C, adj, a, B, nsteps, t0, t1, st, pp_given);
  }
}

template <typename TO, int N>
cudaError_t run_phi_n(const void* phi, int basis, int B, TO* planes, int* min_det, void* ws, const double2* tw64,
                      double kbase, cudaStream_t st) {
  constexpr int LINES = 8;
  constexpr int NT = Geo<double>::nt(N);
  constexpr int H = N / 2;
  double2* spec = reinterpret_cast<double2*>(ws);            // [B][N][H+1]
  double2* packed = spec + (size_t)B * N * (H + 1);          // [B][5][N][H]
  const size_t smem_row = sizeof(double2) * (N + LINES * H) + 16;  // + the table's mbarrier
  const size_t smem_col = sizeof(double2) * (N + LINES * N) + 16;  // + the table's mbarrier
  const int ctiles = (H + 1 + LINES - 1) / LINES;
  cudaError_t e;
  if (basis == LF_PHI_MAP) {
    e = launch<k_phi_rows_r2c<N, LINES, NT>>(dim3(N / LINES, B), NT, smem_row, st,
                                             reinterpret_cast<const double*>(phi), spec, tw64);
    if (e != cudaSuccess) return e;
    e = launch<k_phi_cols_fwd<N, LINES, NT>>(dim3(ctiles, B), NT, smem_col, st, spec, tw64);
    if (e != cudaSuccess) return e;
  } else {
    e = cudaMemcpyAsync(spec, phi, sizeof(double2) * (size_t)B * N * (H + 1), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  e = launch<k_phi_cols_deriv<N, LINES, NT>>(dim3(ctiles, B), NT, smem_col, st, (const double2*)spec, packed,
                                             (const double2*)tw64, kbase);
  if (e != cudaSuccess) return e;
  e = launch<k_phi_rows_c2r<TO, N, LINES, NT>>(dim3(N / LINES, B * 5), NT, smem_row, st, (const double2*)packed,
                                               planes, (const double2*)tw64);
  if (e != cudaSuccess) return e;
  if (min_det) {
    const long P = (long)N * N;
    e = launch<k_min_det<TO>>(dim3(32, B), 256, 0, st, (const TO*)planes, P, min_det);
  }
  return e;
}

// The phi precompute with the p planes formed in the derivative row pass (float32 plans):
// rfft2 of phi (or its given spectrum), the three inverse column transforms of the five
// derivatives, then k_phi_rows_c2r_pp over 2-row tiles of all five.
template <int N>
cudaError_t run_phi_pp_n(const void* phi, int basis, int B, float* planes, float* pp, int K, int* min_det, void* ws,
                         const double2* tw64, double kbase, cudaStream_t st) {
  constexpr int LINES = 8, PL = 2;
  constexpr int NT = Geo<double>::nt(N);
  constexpr int H = N / 2;
  double2* spec = reinterpret_cast<double2*>(ws);
  double2* packed = spec + (size_t)B * N * (H + 1);
  const size_t smem_row = sizeof(double2) * (N + LINES * H) + 16;
  const size_t smem_col = sizeof(double2) * (N + LINES * N) + 16;
  const size_t smem_pp = sizeof(double2) * (N + 5 * PL * H) + 16;
  const int ctiles = (H + 1 + LINES - 1) / LINES;
  cudaError_t e;
  if (basis == LF_PHI_MAP) {
    e = launch<k_phi_rows_r2c<N, LINES, NT>>(dim3(N / LINES, B), NT, smem_row, st,
                                             reinterpret_cast<const double*>(phi), spec, tw64);
    if (e != cudaSuccess) return e;
    e = launch<k_phi_cols_fwd<N, LINES, NT>>(dim3(ctiles, B), NT, smem_col, st, spec, tw64);
    if (e != cudaSuccess) return e;
  } else {
    e = cudaMemcpyAsync(spec, phi, sizeof(double2) * (size_t)B * N * (H + 1), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  constexpr int NTP = pp_threads(N);
  if (planes) {  // derivative planes requested too: float64 spectra, so they equal lf_phi_precompute's
    e = launch<k_phi_cols_deriv<N, LINES, NT>>(dim3(ctiles, B), NT, smem_col, st, (const double2*)spec, packed,
                                               (const double2*)tw64, kbase);
    if (e != cudaSuccess) return e;
    return launch<k_phi_rows_c2r_pp<N, PL, NTP>>(dim3(N / PL, B), NTP, smem_pp, st, (const double2*)packed, planes,
                                                 pp, K, min_det, (const double2*)tw64);
  }
  // p planes only: the five derivative spectra cross HBM as float32 (the p planes are float32; every
  // transform stays float64): 40 N^2 bytes per map less, phi precompute 1.152 -> 1.078 ms per 64 maps
  float2* packed32 = reinterpret_cast<float2*>(packed);
  e = launch<k_phi_cols_deriv<N, LINES, NT, float2>>(dim3(ctiles, B), NT, smem_col, st, (const double2*)spec,
                                                     packed32, (const double2*)tw64, kbase);
  if (e != cudaSuccess) return e;
  return launch<k_phi_rows_c2r_pp<N, PL, NTP, float2>>(dim3(N / PL, B), NTP, smem_pp, st, (const float2*)packed32,
                                                       planes, pp, K, min_det, (const double2*)tw64);
}

cudaError_t run_phi_pp(int N, const void* phi, int basis, int B, float* planes, float* pp, int K, int* min_det,
                       void* ws, const double2* tw64, double kbase, cudaStream_t st) {
  switch (N) {
    case 64: return run_phi_pp_n<64>(phi, basis, B, planes, pp, K, min_det, ws, tw64, kbase, st);
    case 128: return run_phi_pp_n<128>(phi, basis, B, planes, pp, K, min_det, ws, tw64, kbase, st);
    case 256: return run_phi_pp_n<256>(phi, basis, B, planes, pp, K, min_det, ws, tw64, kbase, st);
    case 512: return run_phi_pp_n<512>(phi, basis, B, planes, pp, K, min_det, ws, tw64, kbase, st);
    default: return run_phi_pp_n<1024>(phi, basis, B, planes, pp, K, min_det, ws, tw64, kbase, st);
  }
}

template <typename TO>
cudaError_t run_phi(int N, const void* phi, int basis, int B, TO* planes, int* min_det, void* ws, const double2* tw64,
                    double kbase, cudaStream_t st) {
  switch (N) {
    case 64: return run_phi_n<TO, 64>(phi, basis, B, planes, min_det, ws, tw64, kbase, st);
    case 128: return run_phi_n<TO, 128>(phi, basis, B, planes, min_det, ws, tw64, kbase, st);
    case 256: return run_phi_n<TO, 256>(phi, basis, B, planes, min_det, ws, tw64, kbase, st);
    case 512: return run_phi_n<TO, 512>(phi, basis, B, planes, min_det, ws, tw64, kbase, st);
    default: return run_phi_n<TO, 1024>(phi, basis, B, planes, min_det, ws, tw64, kbase, st);
  }
}

// --------------------------------------------------- float64 rfft2 / irfft2
template <int N>
cudaError_t run_rfft2_n(const void* maps, int in_f64, int B, double2* spec, const double2* tw64, cudaStream_t st) {
  constexpr int LINES = 8;
  constexpr int NT = Geo<double>::nt(N);
  constexpr int H = N / 2;
  const size_t smem_row = sizeof(double2) * (N + LINES * H) + 16;  // + the table's mbarrier
  const size_t smem_col = sizeof(double2) * (N + LINES * N) + 16;  // + the table's mbarrier
  const int ctiles = (H + 1 + LINES - 1) / LINES;
  cudaError_t e;
  if (in_f64)
    e = launch<k_phi_rows_r2c<N, LINES, NT, double>>(dim3(N / LINES, B), NT, smem_row, st,
                                                     reinterpret_cast<const double*>(maps), spec, tw64);
  else
    e = launch<k_phi_rows_r2c<N, LINES, NT, float>>(dim3(N / LINES, B), NT, smem_row, st,
                                                    reinterpret_cast<const float*>(maps), spec, tw64);
  if (e != cudaSuccess) return e;
  return launch<k_phi_cols_fwd<N, LINES, NT>>(dim3(ctiles, B), NT, smem_col, st, spec, tw64);
}

template <int N>
cudaError_t run_irfft2_n(const double2* spec, int B, void* maps, int out_f64, double2* packed, const double2* tw64,
                         cudaStream_t st) {
  constexpr int LINES = 8;
  constexpr int NT = Geo<double>::nt(N);
  constexpr int H = N / 2;
  const size_t smem_row = sizeof(double2) * (N + LINES * H) + 16;  // + the table's mbarrier
  const size_t smem_col = sizeof(double2) * (N + LINES * N) + 16;  // + the table's mbarrier
  const int ctiles = (H + 1 + LINES - 1) / LINES;
  cudaError_t e = launch<k_spec_cols_inv<N, LINES, NT>>(dim3(ctiles, B), NT, smem_col, st, spec, packed, tw64);
  if (e != cudaSuccess) return e;
  if (out_f64)
    return launch<k_phi_rows_c2r<double, N, LINES, NT>>(dim3(N / LINES, B), NT, smem_row, st, (const double2*)packed,
                                                        reinterpret_cast<double*>(maps), tw64);
  return launch<k_phi_rows_c2r<float, N, LINES, NT>>(dim3(N / LINES, B), NT, smem_row, st, (const double2*)packed,
                                                     reinterpret_cast<float*>(maps), tw64);
}

cudaError_t run_rfft2(int N, const void* maps, int in_f64, int B, double2* spec, const double2* tw64, cudaStream_t st) {
  switch (N) {
    case 64: return run_rfft2_n<64>(maps, in_f64, B, spec, tw64, st);
    case 128: return run_rfft2_n<128>(maps, in_f64, B, spec, tw64, st);
    case 256: return run_rfft2_n<256>(maps, in_f64, B, spec, tw64, st);
    case 512: return run_rfft2_n<512>(maps, in_f64, B, spec, tw64, st);
    default: return run_rfft2_n<1024>(maps, in_f64, B, spec, tw64, st);
  }
}

cudaError_t run_irfft2(int N, const double2* spec, int B, void* maps, int out_f64, double2* packed,
                       const double2* tw64, cudaStream_t st) {
  switch (N) {
    case 64: return run_irfft2_n<64>(spec, B, maps, out_f64, packed, tw64, st);
    case 128: return run_irfft2_n<128>(spec, B, maps, out_f64, packed, tw64, st);
    case 256: return run_irfft2_n<256>(spec, B, maps, out_f64, packed, tw64, st);
    case 512: return run_irfft2_n<512>(spec, B, maps, out_f64, packed, tw64, st);
    default: return run_irfft2_n<1024>(spec, B, maps, out_f64, packed, tw64, st);
  }
}

// ------------------------------------------------------------------ VJP
// Workspace of lf_lense_flow_vjp, in order.
struct VjpLayout {
  size_t f_sys, d_sys, grad, dsave, fback, dacc, spec, dphi_f, total;
  VjpLayout(int N, int C, int B, size_t el) {
    const size_t bcp = (size_t)B * C * N * N, bp = (size_t)B * N * N, half = (size_t)B * N * (N / 2 + 1);
    f_sys = 4 * el * bcp;
    d_sys = 5 * el * bcp;
    grad = 2 * el * bcp;
    dsave = el * bcp;
    fback = 8 * bcp;
    dacc = 5 * 8 * bp;
    spec = 5 * 16 * half;
    dphi_f = 16 * half;
    total = f_sys + d_sys + grad + dsave + fback + dacc + spec + dphi_f;
  }
};

template <typename T, int N, int C>
cudaError_t run_vjp_n(const StageArgs& af0, const StageArgs& ad0, double* dacc, int B, int nsteps, double t0,
                      double t1, cudaStream_t st) {
  constexpr int RL = Geo<T>::ROW_LINES;
  constexpr int RNT = Geo<T>::row_nt(N);
  constexpr int RMB = Geo<T>::row_minb(N, C);
  constexpr int H = N / 2;
  const size_t smem_row = sizeof(c2<T>) * (N + 2 * C * RL * H) + 16;  // + the table's mbarrier
  const dim3 grow(N / RL, B);
  const long P = (long)N * N;
  const int gacc = (int)std::min<long>(((long)B * P + 255) / 256, 4096);
  StageArgs af = af0, ad = ad0;
  const double h = (t1 - t0) / nsteps;
  const double hh = h / 2.0;
  const double cw[4] = {1.0, 2.0, 2.0, 1.0};
  af.h = ad.h = h;
  af.stage = ad.stage = 0;
  af.last = ad.last = 0;
  af.t_cur = af.t_next = ad.t_cur = ad.t_next = t0;
  cudaError_t e = launch_k<k_row<T, N, C, false, true, RL, RNT, false, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, af);
  if (e != cudaSuccess) return e;
  e = launch_k<k_row<T, N, C, true, true, RL, RNT, true, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, ad);
  if (e != cudaSuccess) return e;
  for (int i = 0; i < nsteps; ++i) {
    const double t = t0 + i * h;
    const double tc[4] = {t, t + hh, t + hh, t + h};
    const double tn[4] = {t + hh, t + hh, t + h, t0 + (i + 1) * h};
    for (int s = 0; s < 4; ++s) {
      const int last = (i == nsteps - 1 && s == 3);
      af.stage = ad.stage = s + 1;
      af.t_cur = ad.t_cur = tc[s];
      af.t_next = ad.t_next = tn[s];
      af.last = ad.last = last;
      e = launch_col<T, N>(B * C, st, af);
      if (e != cudaSuccess) return e;
      e = launch_k<k_row<T, N, C, false, false, RL, RNT, true, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, af);
      if (e != cudaSuccess) return e;
      e = launch<k_dphi_accum<T, C>>(dim3(gacc), 256, 0, st, (const T*)af.grad, (const T*)ad.dsave,
                                     (const T*)af.phi, dacc, B, P, tc[s], h / 6.0 * cw[s], (int)(i == 0 && s == 0));
      if (e != cudaSuccess) return e;
      e = launch_col<T, N>(B * C, st, ad);
      if (e != cudaSuccess) return e;
      e = launch_k<k_row<T, N, C, true, false, RL, RNT, true, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, ad);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

template <typename T, int N>
cudaError_t run_vjp_c(int C, const StageArgs& af, const StageArgs& ad, double* dacc, int B, int nsteps, double t0,
                      double t1, cudaStream_t st) {
  if (C == 1) return run_vjp_n<T, N, 1>(af, ad, dacc, B, nsteps, t0, t1, st);
  if (C == 2) return run_vjp_n<T, N, 2>(af, ad, dacc, B, nsteps, t0, t1, st);
  return run_vjp_n<T, N, 3>(af, ad, dacc, B, nsteps, t0, t1, st);
}

template <typename T>
cudaError_t run_vjp(int N, int C, const StageArgs& af, const StageArgs& ad, double* dacc, int B, int nsteps,
                    double t0, double t1, cudaStream_t st) {
  switch (N) {
    case 64: return run_vjp_c<T, 64>(C, af, ad, dacc, B, nsteps, t0, t1, st);
    case 128: return run_vjp_c<T, 128>(C, af, ad, dacc, B, nsteps, t0, t1, st);
    case 256: return run_vjp_c<T, 256>(C, af, ad, dacc, B, nsteps, t0, t1, st);
    case 512: return run_vjp_c<T, 512>(C, af, ad, dacc, B, nsteps, t0, t1, st);
    default: return run_vjp_c<T, 1024>(C, af, ad, dacc, B, nsteps, t0, t1, st);
  }
}

// --------------------------------------------- checkpointed exact VJP
// Workspace of lf_lense_flow_vjp_ckpt, in order: the n step checkpoints, the
// forward state (y0, acc, S, Gx), the four stage gradients (d_x u_s, d_y u_s),
// the adjoint state (y0, acc, U, V, Gx), the saved adjoint stage input, an
// output sink, the delta-phi accumulators and the spectra of the final combine.
struct CkptLayout {
  size_t ckpt, f_sys, grads, d_sys, dsave, sink, dacc, spec, dphi_f, total;
  CkptLayout(int N, int C, int B, int n, size_t el) {
    const size_t bcp = (size_t)B * C * N * N, bp = (size_t)B * N * N, half = (size_t)B * N * (N / 2 + 1);
    ckpt = (size_t)n * el * bcp;
    f_sys = 4 * el * bcp;
    grads = 4 * 2 * el * bcp;
    d_sys = 5 * el * bcp;
    dsave = el * bcp;
    sink = 8 * bcp;
    dacc = 5 * 8 * bp;
    spec = 5 * 16 * half;
    dphi_f = 16 * half;
    total = ckpt + f_sys + grads + d_sys + dsave + sink + dacc + spec + dphi_f;
  }
};

// The exact transpose of the discrete forward RK4 (lense_flow.py:336-352 with
// util.py:184-199).  The forward integration stores y_i at the start of every
// step.  Backwards, step i is recomputed from y_i with its four stage
// inputs' gradients saved (d_x u_s, d_y u_s), and one RK4 step of the
// adjoint RHS carries the cotangent from t_{i+1} to t_i: for a linear RHS the
// transpose of an RK4 step is an RK4 step of the transposed RHS with the
// stages in reverse order (forward stage s pairs with adjoint stage 5 - s at
// the same time).  The stage cotangents are k_bar_s = (h/6) w_s v_{5-s},
// w = {1, 2, 2, 1}, with v_j the adjoint stage inputs, so
// p_bar(t_s) += k_bar_s . grad u_s, and the chain rule through
// p = M(t)^-1 grad(phi) is the same per-stage delta-phi rate as the
// reference's reverse ODE (get_delta_phi_tqu_roc, lense_flow.py:195-252) --
// evaluated on the forward stage inputs u_s instead of a field re-integrated
// backwards from Lf.  The result is the gradient of the discrete map, free of
// the reference scheme's O(h^4) gap.
template <typename T, int N, int C>
cudaError_t run_vjp_ckpt_n(const StageArgs& af0, const StageArgs& ad0, char* ckpt, char* grads, void* sink, double* dacc,
                           int B, int nsteps, double t0, double t1, cudaStream_t st) {
  constexpr int RL = Geo<T>::ROW_LINES;
  constexpr int RNT = Geo<T>::row_nt(N);
  constexpr int RMB = Geo<T>::row_minb(N, C);
  constexpr int H = N / 2;
  const size_t smem_row = sizeof(c2<T>) * (N + 2 * C * RL * H) + 16;  // + the table's mbarrier
  const dim3 grow(N / RL, B);
  const long P = (long)N * N;
  const size_t plane = sizeof(T) * (size_t)B * C * P;
  const int gacc = (int)std::min<long>(((long)B * P + 255) / 256, 4096);
  const double h = (t1 - t0) / nsteps, hh = h / 2.0;
  const double hb = -h, hhb = hb / 2.0;  // the adjoint integration runs t1 -> t0
  const double cw[4] = {1.0, 2.0, 2.0, 1.0};
  StageArgs af = af0, ad = ad0;
  cudaError_t e;
  // ---- forward integration, storing y_i at the start of each step
  af.h = h;
  af.stage = 0;
  af.last = 0;
  af.t_cur = af.t_next = t0;
  e = launch_k<k_row<T, N, C, false, true, RL, RNT, false, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, af);
  if (e != cudaSuccess) return e;
  for (int i = 0; i < nsteps; ++i) {
    e = cudaMemcpyAsync(ckpt + (size_t)i * plane, af.y0, plane, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    const double t = t0 + i * h;
    const double tc[4] = {t, t + hh, t + hh, t + h};
    const double tn[4] = {t + hh, t + hh, t + h, t0 + (i + 1) * h};
    for (int s = 0; s < 4; ++s) {
      af.stage = s + 1;
      af.t_cur = tc[s];
      af.t_next = tn[s];
      af.last = (i == nsteps - 1 && s == 3);
      e = launch_col<T, N>(B * C, st, af);
      if (e != cudaSuccess) return e;
      e = launch_k<k_row<T, N, C, false, false, RL, RNT, false, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, af);
      if (e != cudaSuccess) return e;
    }
  }
  // ---- adjoint initialisation from the cotangent (saves the first stage input)
  ad.h = hb;
  ad.stage = 0;
  ad.last = 0;
  ad.t_cur = ad.t_next = t1;
  e = launch_k<k_row<T, N, C, true, true, RL, RNT, true, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, ad);
  if (e != cudaSuccess) return e;
  // ---- reverse steps: recompute forward step i, then one adjoint RK4 step over it
  StageArgs ar = af0;  // the recomputation reads the checkpoint in the compute precision
  ar.in_f64 = ar.out_f64 = std::is_same<T, double>::value;
  ar.f_out = sink;  // the recomputed steps' last-stage updates are discarded
  ar.h = h;
  for (int ib = 0; ib < nsteps; ++ib) {
    const int i = nsteps - 1 - ib;
    const double t = t0 + i * h;
    const double tc[4] = {t, t + hh, t + hh, t + h};
    const double tn[4] = {t + hh, t + hh, t + h, t0 + (i + 1) * h};
    ar.f_in = ckpt + (size_t)i * plane;
    ar.stage = 0;
    ar.last = 0;
    ar.t_cur = ar.t_next = t;
    e = launch_k<k_row<T, N, C, false, true, RL, RNT, false, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, ar);
    if (e != cudaSuccess) return e;
    for (int s = 0; s < 4; ++s) {
      ar.stage = s + 1;
      ar.t_cur = tc[s];
      ar.t_next = tn[s];
      ar.last = (s == 3);  // stage 4's update goes to the sink; no next-stage spectrum
      ar.grad = grads + (size_t)s * 2 * plane;
      e = launch_col<T, N>(B * C, st, ar);
      if (e != cudaSuccess) return e;
      e = launch_k<k_row<T, N, C, false, false, RL, RNT, true, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, ar);
      if (e != cudaSuccess) return e;
    }
    const double tb = t0 + (i + 1) * h;  // = t1 + ib * hb
    const double tcb[4] = {tb, tb + hhb, tb + hhb, tb + hb};
    const double tnb[4] = {tb + hhb, tb + hhb, tb + hb, t0 + i * h};
    for (int j = 0; j < 4; ++j) {
      // adjoint stage j + 1 (input in dsave) pairs with forward stage 4 - j at the same time
      e = launch<k_dphi_accum<T, C>>(dim3(gacc), 256, 0, st, (const T*)(grads + (size_t)(3 - j) * 2 * plane),
                                     (const T*)ad.dsave, (const T*)af.phi, dacc, B, P, tcb[j], hb / 6.0 * cw[j],
                                     (int)(ib == 0 && j == 0));
      if (e != cudaSuccess) return e;
      ad.stage = j + 1;
      ad.t_cur = tcb[j];
      ad.t_next = tnb[j];
      ad.last = (ib == nsteps - 1 && j == 3);
      e = launch_col<T, N>(B * C, st, ad);
      if (e != cudaSuccess) return e;
      e = launch_k<k_row<T, N, C, true, false, RL, RNT, true, RMB>>(LF_KIND_ROW, grow, RNT, smem_row, st, ad);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

template <typename T, int N>
cudaError_t run_vjp_ckpt_c(int C, const StageArgs& af, const StageArgs& ad, char* ckpt, char* grads, void* sink,
                           double* dacc, int B, int nsteps, double t0, double t1, cudaStream_t st) {
  if (C == 1) return run_vjp_ckpt_n<T, N, 1>(af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
  if (C == 2) return run_vjp_ckpt_n<T, N, 2>(af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
  return run_vjp_ckpt_n<T, N, 3>(af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
}

template <typename T>
cudaError_t run_vjp_ckpt(int N, int C, const StageArgs& af, const StageArgs& ad, char* ckpt, char* grads, void* sink,
                         double* dacc, int B, int nsteps, double t0, double t1, cudaStream_t st) {
  switch (N) {
    case 64: return run_vjp_ckpt_c<T, 64>(C, af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
    case 128: return run_vjp_ckpt_c<T, 128>(C, af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
    case 256: return run_vjp_ckpt_c<T, 256>(C, af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
    case 512: return run_vjp_ckpt_c<T, 512>(C, af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
    default: return run_vjp_ckpt_c<T, 1024>(C, af, ad, ckpt, grads, sink, dacc, B, nsteps, t0, t1, st);
  }
}

// delta-phi from the five accumulator planes per map: sum_j m_j rfft2(acc_j)
// (the multipliers of get_primal_derivatives_to_fourier, util.py:133-137), in
// the Fourier layout or, for a map phi, summed through irfft2
// (lense_flow.py:233-248).  ``spec`` holds 5 B spectra, ``dphi_f`` B more.
cudaError_t finish_dphi(int N, int B, double* dacc, double2* spec, double2* dphi_f, void* dphi, int dphi_basis,
                        const double2* tw64, double kbase, cudaStream_t st) {
  cudaError_t e = run_rfft2(N, dacc, 1, B * 5, spec, tw64, st);
  if (e != cudaSuccess) return e;
  const long half = (long)B * N * (N / 2 + 1);
  double2* target = dphi_basis == LF_PHI_FOURIER ? reinterpret_cast<double2*>(dphi) : dphi_f;
  e = launch<k_dphi_combine>(dim3((unsigned)std::min<long>((half + 255) / 256, 4096)), 256, 0, st,
                             (const double2*)spec, target, B, N, kbase);
  if (e != cudaSuccess) return e;
  if (dphi_basis == LF_PHI_MAP) e = run_irfft2(N, dphi_f, B, dphi, 1, spec, tw64, st);
  return e;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" {

int lf_version(void) { return kVersion; }

const char* lf_status_string(int s) {
  switch (s) {
    case LF_OK: return "ok";
    case LF_ERR_BAD_SHAPE: return "bad shape (N must be 64, 128, 256, 512 or 1024; ncomp 1..3; batch >= 0)";
    case LF_ERR_BAD_DTYPE: return "bad dtype";
    case LF_ERR_BAD_ARG: return "bad argument (null or misaligned pointer, bad direction or step count)";
    case LF_ERR_SINGULAR_MAGNIFICATION: return "det(I + t grad grad phi) <= 0 for some pixel and t in [0,1]";
    case LF_ERR_OOM: return "out of device memory";
    case LF_ERR_TIMEOUT:
      return "timeout: a kernel block gave up waiting for its bulk copies; results since the last "
             "lf_wait_timeouts reset are invalid";
    case LF_ERR_CUDA: return "CUDA error";
    case LF_ERR_WORKSPACE: return "workspace too small";
    default: return "unknown status";
  }
}

int lf_plan_create(lf_plan_t* out, int nside, int ncomp, double pix_width, int precision) {
  if (!out) return LF_ERR_BAD_ARG;
  *out = nullptr;
  if (!valid_n(nside) || ncomp < 1 || ncomp > 3) return LF_ERR_BAD_SHAPE;
  if (precision != LF_F32 && precision != LF_F64) return LF_ERR_BAD_DTYPE;
  if (!(pix_width > 0.0) || !std::isfinite(pix_width)) return LF_ERR_BAD_ARG;
  lf_plan_s* p = new (std::nothrow) lf_plan_s();
  if (!p) return LF_ERR_OOM;
  p->N = nside;
  p->C = ncomp;
  p->prec = precision;
  p->pix_width = pix_width;
  cudaGetDevice(&p->device);
  if (cudaError_t fe = ensure_timeout_flag(); fe != cudaSuccess) {
    delete p;
    return cuda_status(fe);
  }
  // exp(-2 pi i k / N) in float64 on the host, rounded once to the compute precision
  std::vector<double2> t64(nside);
  std::vector<float2> t32(nside);
  for (int k = 0; k < nside; ++k) {
    const double ang = -2.0 * M_PI * (double)k / (double)nside;
    t64[k] = make_double2(std::cos(ang), std::sin(ang));
    t32[k] = make_float2((float)t64[k].x, (float)t64[k].y);
  }
  cudaError_t e = cudaMalloc(&p->tw64, sizeof(double2) * nside);
  if (e == cudaSuccess) e = cudaMemcpy(p->tw64, t64.data(), sizeof(double2) * nside, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (precision == LF_F64) {
      p->tw = p->tw64;
    } else {
      e = cudaMalloc(&p->tw, sizeof(float2) * nside);
      if (e == cudaSuccess) e = cudaMemcpy(p->tw, t32.data(), sizeof(float2) * nside, cudaMemcpyHostToDevice);
    }
  }
  if (e == cudaSuccess) {
    const size_t np = (size_t)ptw_size(nside) + (size_t)ctw_size(nside);
    std::vector<double2> pt(np);
    std::vector<float2> pt32(np);
    auto put = [&](int i, double c, double sn) {
      pt[i] = make_double2(c, sn);
      pt32[i] = make_float2((float)c, (float)sn);
    };
    fill_pass_table(nside, put);
    fill_col_table(nside, [&](int i, double c, double sn) { put(ptw_size(nside) + i, c, sn); });
    const bool f64 = precision == LF_F64;
    const size_t bytes = f64 ? sizeof(double2) * np : sizeof(float2) * np;
    e = cudaMalloc(&p->twp, bytes);
    if (e == cudaSuccess)
      e = cudaMemcpy(p->twp, f64 ? (const void*)pt.data() : (const void*)pt32.data(), bytes, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    lf_plan_destroy(p);
    return cuda_status(e);
  }
  *out = p;
  return LF_OK;
}

int lf_plan_destroy(lf_plan_t p) {
  if (!p) return LF_OK;
  if (p->tw && p->tw != p->tw64) cudaFree(p->tw);
  if (p->tw64) cudaFree(p->tw64);
  if (p->twp) cudaFree(p->twp);
  for (cudaEvent_t e : p->prof.pool) cudaEventDestroy(e);
  delete p;
  return LF_OK;
}

size_t lf_workspace_bytes(lf_plan_t p, int batch, int adjoint) {
  if (!p || batch < 0) return 0;
  const size_t el = p->prec == LF_F64 ? 8 : 4;
  return el * (size_t)p->N * p->N * (size_t)batch * p->C * (adjoint ? 5 : 4);
}

// p-plane region: 2 (2n+1) planes per map, float32 plans only
static size_t pp_bytes(lf_plan_t p, int batch, int nsteps) {
  if (p->prec != LF_F32 || nsteps <= 0) return 0;
  return 4 * (size_t)p->N * p->N * (size_t)batch * 2 * (2 * (size_t)nsteps + 1);
}

size_t lf_workspace_bytes_n(lf_plan_t p, int batch, int adjoint, int nsteps) {
  if (!p || batch < 0 || nsteps < 0) return 0;
  return lf_workspace_bytes(p, batch, adjoint) + pp_bytes(p, batch, nsteps);
}

size_t lf_phi_planes_bytes(lf_plan_t p, int batch) {
  if (!p || batch < 0) return 0;
  const size_t el = p->prec == LF_F64 ? 8 : 4;
  return el * 5 * (size_t)p->N * p->N * (size_t)batch;
}

size_t lf_phi_workspace_bytes(lf_plan_t p, int batch) {
  if (!p || batch < 0) return 0;
  const size_t N = p->N, H = N / 2;
  return sizeof(double2) * (size_t)batch * (N * (H + 1) + 5 * N * H);
}

int lf_min_det_init(int* min_det, int batch, void* stream) {
  if (batch <= 0) return LF_OK;
  if (!min_det) return LF_ERR_BAD_ARG;
  return cuda_status(cudaMemsetAsync(min_det, 0x7f, sizeof(int) * (size_t)batch, (cudaStream_t)stream));
}

float lf_decode_min_det(int i) {
  const int b = i >= 0 ? i : (i ^ 0x7fffffff);
  float f;
  std::memcpy(&f, &b, sizeof(f));
  return f;
}

int lf_phi_precompute(lf_plan_t p, const void* phi, int basis, int batch, void* planes, int* min_det, void* ws,
                      size_t ws_bytes, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if (batch == 0) return LF_OK;
  if (basis != LF_PHI_MAP && basis != LF_PHI_FOURIER) return LF_ERR_BAD_ARG;
  if (!phi || !planes || !ws || !aligned16(phi) || !aligned16(planes) || !aligned16(ws)) return LF_ERR_BAD_ARG;
  if (ws_bytes < lf_phi_workspace_bytes(p, batch)) return LF_ERR_WORKSPACE;
  const double kbase = 2.0 * M_PI / ((double)p->N * p->pix_width);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  g_prof = &p->prof;
  if (p->prec == LF_F64)
    e = run_phi<double>(p->N, phi, basis, batch, reinterpret_cast<double*>(planes), min_det, ws, p->tw64, kbase, st);
  else
    e = run_phi<float>(p->N, phi, basis, batch, reinterpret_cast<float*>(planes), min_det, ws, p->tw64, kbase, st);
  return cuda_status(e);
}

int lf_lense_flow(lf_plan_t p, const void* f_in, int in_dtype, void* f_out, int out_dtype, const void* planes,
                  int batch, int nsteps, int direction, int adjoint, void* ws, size_t ws_bytes, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if ((in_dtype != LF_F32 && in_dtype != LF_F64) || (out_dtype != LF_F32 && out_dtype != LF_F64))
    return LF_ERR_BAD_DTYPE;
  if (nsteps < 0 || (direction != LF_FORWARD_LENSE && direction != LF_INVERSE_LENSE)) return LF_ERR_BAD_ARG;
  if (batch == 0) return LF_OK;
  if (!f_in || !f_out || !planes || !aligned16(f_in) || !aligned16(f_out) || !aligned16(planes)) return LF_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t npix = (size_t)p->N * p->N * (size_t)batch * p->C;
  if (nsteps == 0) {  // rk4_solve with zero steps returns its input (util.py:199)
    if (in_dtype != out_dtype) return LF_ERR_BAD_DTYPE;
    if (f_in == f_out) return LF_OK;
    return cuda_status(cudaMemcpyAsync(f_out, f_in, npix * (in_dtype == LF_F64 ? 8 : 4), cudaMemcpyDeviceToDevice, st));
  }
  const bool adj = adjoint != 0;
  if (!ws || !aligned16(ws)) return LF_ERR_BAD_ARG;
  if (ws_bytes < lf_workspace_bytes(p, batch, adj)) return LF_ERR_WORKSPACE;
  // lense_flow.py:304-322: forward time iff (direction == +1) XOR adjoint
  const bool fwd_time = ((direction == LF_FORWARD_LENSE) != adj);
  const double t0 = fwd_time ? 0.0 : 1.0, t1 = fwd_time ? 1.0 : 0.0;
  const size_t el = p->prec == LF_F64 ? 8 : 4;
  const size_t plane_bytes = el * npix;
  StageArgs a;
  std::memset(&a, 0, sizeof(a));
  a.f_in = f_in;
  a.f_out = f_out;
  a.in_f64 = in_dtype == LF_F64;
  a.out_f64 = out_dtype == LF_F64;
  a.phi = planes;
  char* w = reinterpret_cast<char*>(ws);
  a.y0 = w;
  a.acc = w + plane_bytes;
  a.s = w + 2 * plane_bytes;
  a.gx = w + 3 * plane_bytes;
  a.v = adj ? (void*)(w + 4 * plane_bytes) : nullptr;
  // room for the p planes: read p at the stage times instead of forming it
  const size_t base_bytes = lf_workspace_bytes(p, batch, adj);
  const size_t ppb = pp_bytes(p, batch, nsteps);
  if (ppb && ws_bytes >= base_bytes + ppb) a.pp = w + base_bytes;
  a.twN = p->tw;
  a.twP = p->twp;
  a.twC = p->twc();
  a.kbase = 2.0 * M_PI / ((double)p->N * p->pix_width);
  a.nplanes = batch * p->C;
  cudaError_t e;
  g_prof = &p->prof;
  if (p->prec == LF_F64)
    e = run_lens<double>(p->N, p->C, adj, a, batch, nsteps, t0, t1, st);
  else
    e = run_lens<float>(p->N, p->C, adj, a, batch, nsteps, t0, t1, st);
  return cuda_status(e);
}

size_t lf_pp_bytes(lf_plan_t p, int batch, int nsteps) {
  if (!p || batch < 0 || nsteps < 1) return 0;
  return pp_bytes(p, batch, nsteps);
}

int lf_phi_precompute_pp(lf_plan_t p, const void* phi, int basis, int batch, void* planes, void* pp, int nsteps,
                         int* min_det, void* ws, size_t ws_bytes, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (p->prec != LF_F32) return LF_ERR_BAD_DTYPE;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if (basis != LF_PHI_MAP && basis != LF_PHI_FOURIER) return LF_ERR_BAD_ARG;
  if (nsteps < 1) return LF_ERR_BAD_ARG;
  if (batch == 0) return LF_OK;
  if (!phi || !pp || !ws || !aligned16(phi) || !aligned16(pp) || !aligned16(ws) || (planes && !aligned16(planes)))
    return LF_ERR_BAD_ARG;
  if (ws_bytes < lf_phi_workspace_bytes(p, batch)) return LF_ERR_WORKSPACE;
  const double kbase = 2.0 * M_PI / ((double)p->N * p->pix_width);
  g_prof = &p->prof;
  return cuda_status(run_phi_pp(p->N, phi, basis, batch, reinterpret_cast<float*>(planes), reinterpret_cast<float*>(pp),
                                2 * nsteps + 1, min_det, ws, p->tw64, kbase, (cudaStream_t)stream));
}

int lf_lense_flow_pp(lf_plan_t p, const void* f_in, int in_dtype, void* f_out, int out_dtype, const void* pp,
                     int batch, int nsteps, int direction, int adjoint, void* ws, size_t ws_bytes, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (p->prec != LF_F32) return LF_ERR_BAD_DTYPE;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if ((in_dtype != LF_F32 && in_dtype != LF_F64) || (out_dtype != LF_F32 && out_dtype != LF_F64))
    return LF_ERR_BAD_DTYPE;
  if (nsteps < 1 || (direction != LF_FORWARD_LENSE && direction != LF_INVERSE_LENSE)) return LF_ERR_BAD_ARG;
  if (batch == 0) return LF_OK;
  if (!f_in || !f_out || !pp || !ws || !aligned16(f_in) || !aligned16(f_out) || !aligned16(pp) || !aligned16(ws))
    return LF_ERR_BAD_ARG;
  const bool adj = adjoint != 0;
  if (ws_bytes < lf_workspace_bytes(p, batch, adj)) return LF_ERR_WORKSPACE;
  const bool fwd_time = ((direction == LF_FORWARD_LENSE) != adj);
  const double t0 = fwd_time ? 0.0 : 1.0, t1 = fwd_time ? 1.0 : 0.0;
  const size_t plane_bytes = 4 * (size_t)p->N * p->N * (size_t)batch * p->C;
  StageArgs a;
  std::memset(&a, 0, sizeof(a));
  a.f_in = f_in;
  a.f_out = f_out;
  a.in_f64 = in_dtype == LF_F64;
  a.out_f64 = out_dtype == LF_F64;
  a.phi = pp;  // not read on the p-plane path
  a.pp = pp;
  char* w = reinterpret_cast<char*>(ws);
  a.y0 = w;
  a.acc = w + plane_bytes;
  a.s = w + 2 * plane_bytes;
  a.gx = w + 3 * plane_bytes;
  a.v = adj ? (void*)(w + 4 * plane_bytes) : nullptr;
  a.twN = p->tw;
  a.twP = p->twp;
  a.twC = p->twc();
  a.kbase = 2.0 * M_PI / ((double)p->N * p->pix_width);
  a.nplanes = batch * p->C;
  g_prof = &p->prof;
  return cuda_status(run_lens<float>(p->N, p->C, adj, a, batch, nsteps, t0, t1, (cudaStream_t)stream, true));
}

int lf_wait_timeouts(int* count, int reset) {
  if (!count) return LF_ERR_BAD_ARG;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpyFromSymbol(count, g_lf_wait_timeouts, sizeof(int));
  if (e != cudaSuccess) return cuda_status(e);
  if (timeout_recorded()) *count = 1;
  if (reset) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_lf_wait_timeouts, &zero, sizeof(int));
    std::lock_guard<std::mutex> lock(g_flag_mu);
    if (int* h = g_host_flag.load()) *reinterpret_cast<volatile int*>(h) = 0;
  }
  return cuda_status(e);
}

int lf_timeout_status(void) { return timeout_recorded() ? LF_ERR_TIMEOUT : LF_OK; }

int lf_stream_check(void* stream) {
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_status(e);
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  int dev_flag = 0;
  e = cudaMemcpyFromSymbol(&dev_flag, g_lf_wait_timeouts, sizeof(int));
  if (e != cudaSuccess) return cuda_status(e);
  return dev_flag ? LF_ERR_TIMEOUT : LF_OK;
}

int lf_set_wait_polls(int polls) {
  const int v = polls < 0 ? kWaitTries : std::min(polls, kWaitTries);
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_lf_wait_polls, &v, sizeof(int));
  return cuda_status(e);
}

size_t lf_fft_workspace_bytes(lf_plan_t p, int batch) {
  if (!p || batch < 0) return 0;
  return sizeof(double2) * (size_t)batch * p->N * (p->N / 2);
}

int lf_rfft2(lf_plan_t p, const void* maps, int in_dtype, int batch, void* spec, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if (in_dtype != LF_F32 && in_dtype != LF_F64) return LF_ERR_BAD_DTYPE;
  if (batch == 0) return LF_OK;
  if (!maps || !spec || !aligned16(maps) || !aligned16(spec)) return LF_ERR_BAD_ARG;
  g_prof = &p->prof;
  return cuda_status(run_rfft2(p->N, maps, in_dtype == LF_F64, batch, reinterpret_cast<double2*>(spec), p->tw64,
                               (cudaStream_t)stream));
}

int lf_irfft2(lf_plan_t p, const void* spec, int batch, void* maps, int out_dtype, void* ws, size_t ws_bytes,
              void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if (out_dtype != LF_F32 && out_dtype != LF_F64) return LF_ERR_BAD_DTYPE;
  if (batch == 0) return LF_OK;
  if (!maps || !spec || !ws || !aligned16(maps) || !aligned16(spec) || !aligned16(ws)) return LF_ERR_BAD_ARG;
  if (ws_bytes < lf_fft_workspace_bytes(p, batch)) return LF_ERR_WORKSPACE;
  g_prof = &p->prof;
  return cuda_status(run_irfft2(p->N, reinterpret_cast<const double2*>(spec), batch, maps, out_dtype == LF_F64,
                                reinterpret_cast<double2*>(ws), p->tw64, (cudaStream_t)stream));
}

size_t lf_vjp_workspace_bytes(lf_plan_t p, int batch) {
  if (!p || batch < 0) return 0;
  return VjpLayout(p->N, p->C, batch, p->prec == LF_F64 ? 8 : 4).total;
}

int lf_lense_flow_vjp(lf_plan_t p, const void* f_lensed, const void* cotangent, int io_dtype, const void* planes,
                      int batch, int nsteps, int direction, void* delta_f, void* f_back, void* dphi, int dphi_basis,
                      void* ws, size_t ws_bytes, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if (io_dtype != LF_F32 && io_dtype != LF_F64) return LF_ERR_BAD_DTYPE;
  if (nsteps < 1 || (direction != LF_FORWARD_LENSE && direction != LF_INVERSE_LENSE)) return LF_ERR_BAD_ARG;
  if (dphi_basis != LF_PHI_MAP && dphi_basis != LF_PHI_FOURIER) return LF_ERR_BAD_ARG;
  if (batch == 0) return LF_OK;
  if (!f_lensed || !cotangent || !planes || !delta_f || !dphi || !ws) return LF_ERR_BAD_ARG;
  if (!aligned16(f_lensed) || !aligned16(cotangent) || !aligned16(planes) || !aligned16(delta_f) ||
      !aligned16(dphi) || !aligned16(ws) || (f_back && !aligned16(f_back)))
    return LF_ERR_BAD_ARG;
  const size_t el = p->prec == LF_F64 ? 8 : 4;
  const VjpLayout L(p->N, p->C, batch, el);
  if (ws_bytes < L.total) return LF_ERR_WORKSPACE;
  // lense_flow.py:30 integrates in the opposite direction; :54-74 maps it to the time span
  const int back = -direction;
  const double t0 = back == LF_INVERSE_LENSE ? 1.0 : 0.0, t1 = back == LF_INVERSE_LENSE ? 0.0 : 1.0;
  char* w = reinterpret_cast<char*>(ws);
  const size_t plane = el * (size_t)batch * p->C * p->N * p->N;
  char* fs = w;
  char* ds = fs + L.f_sys;
  char* grad = ds + L.d_sys;
  char* dsave = grad + L.grad;
  char* fback = dsave + L.dsave;
  double* dacc = reinterpret_cast<double*>(fback + L.fback);
  double2* spec = reinterpret_cast<double2*>(reinterpret_cast<char*>(dacc) + L.dacc);
  double2* dphi_f = reinterpret_cast<double2*>(reinterpret_cast<char*>(spec) + L.spec);
  StageArgs af, ad;
  std::memset(&af, 0, sizeof(af));
  af.f_in = f_lensed;
  af.f_out = f_back ? f_back : (void*)fback;
  af.in_f64 = af.out_f64 = io_dtype == LF_F64;
  af.phi = planes;
  af.y0 = fs;
  af.acc = fs + plane;
  af.s = fs + 2 * plane;
  af.gx = fs + 3 * plane;
  af.twN = p->tw;
  af.twP = p->twp;
  af.twC = p->twc();
  af.kbase = 2.0 * M_PI / ((double)p->N * p->pix_width);
  af.nplanes = batch * p->C;
  af.grad = grad;
  ad = af;
  ad.f_in = cotangent;
  ad.f_out = delta_f;
  ad.y0 = ds;
  ad.acc = ds + plane;
  ad.s = ds + 2 * plane;
  ad.v = ds + 3 * plane;
  ad.gx = ds + 4 * plane;
  ad.grad = nullptr;
  ad.dsave = dsave;
  cudaStream_t st = (cudaStream_t)stream;
  g_prof = &p->prof;
  cudaError_t e = p->prec == LF_F64 ? run_vjp<double>(p->N, p->C, af, ad, dacc, batch, nsteps, t0, t1, st)
                                    : run_vjp<float>(p->N, p->C, af, ad, dacc, batch, nsteps, t0, t1, st);
  if (e != cudaSuccess) return cuda_status(e);
  return cuda_status(finish_dphi(p->N, batch, dacc, spec, dphi_f, dphi, dphi_basis, p->tw64, af.kbase, st));
}

size_t lf_vjp_ckpt_workspace_bytes(lf_plan_t p, int batch, int nsteps) {
  if (!p || batch < 0 || nsteps < 1) return 0;
  return CkptLayout(p->N, p->C, batch, nsteps, p->prec == LF_F64 ? 8 : 4).total;
}

int lf_lense_flow_vjp_ckpt(lf_plan_t p, const void* f_in, const void* cotangent, int io_dtype, const void* planes,
                           int batch, int nsteps, int direction, void* f_out, void* delta_f, void* dphi, int dphi_basis,
                           void* ws, size_t ws_bytes, void* stream) {
  if (!p) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  if (batch < 0) return LF_ERR_BAD_SHAPE;
  if (io_dtype != LF_F32 && io_dtype != LF_F64) return LF_ERR_BAD_DTYPE;
  if (nsteps < 1 || (direction != LF_FORWARD_LENSE && direction != LF_INVERSE_LENSE)) return LF_ERR_BAD_ARG;
  if (dphi_basis != LF_PHI_MAP && dphi_basis != LF_PHI_FOURIER) return LF_ERR_BAD_ARG;
  if (batch == 0) return LF_OK;
  if (!f_in || !cotangent || !planes || !delta_f || !dphi || !ws) return LF_ERR_BAD_ARG;
  if (!aligned16(f_in) || !aligned16(cotangent) || !aligned16(planes) || !aligned16(delta_f) || !aligned16(dphi) ||
      !aligned16(ws) || (f_out && !aligned16(f_out)))
    return LF_ERR_BAD_ARG;
  const size_t el = p->prec == LF_F64 ? 8 : 4;
  const CkptLayout L(p->N, p->C, batch, nsteps, el);
  if (ws_bytes < L.total) return LF_ERR_WORKSPACE;
  // the lens being differentiated runs 0 -> 1 for direction +1 (lense_flow.py:304-322)
  const double t0 = direction == LF_FORWARD_LENSE ? 0.0 : 1.0, t1 = 1.0 - t0;
  const size_t plane = el * (size_t)batch * p->C * p->N * p->N;
  char* w = reinterpret_cast<char*>(ws);
  char* ckpt = w;
  char* fs = ckpt + L.ckpt;
  char* grads = fs + L.f_sys;
  char* ds = grads + L.grads;
  char* dsave = ds + L.d_sys;
  char* sink = dsave + L.dsave;
  double* dacc = reinterpret_cast<double*>(sink + L.sink);
  double2* spec = reinterpret_cast<double2*>(reinterpret_cast<char*>(dacc) + L.dacc);
  double2* dphi_f = reinterpret_cast<double2*>(reinterpret_cast<char*>(spec) + L.spec);
  StageArgs af, ad;
  std::memset(&af, 0, sizeof(af));
  af.f_in = f_in;
  af.f_out = f_out ? f_out : (void*)sink;
  af.in_f64 = af.out_f64 = io_dtype == LF_F64;
  af.phi = planes;
  af.y0 = fs;
  af.acc = fs + plane;
  af.s = fs + 2 * plane;
  af.gx = fs + 3 * plane;
  af.twN = p->tw;
  af.twP = p->twp;
  af.twC = p->twc();
  af.kbase = 2.0 * M_PI / ((double)p->N * p->pix_width);
  af.nplanes = batch * p->C;
  ad = af;
  ad.f_in = cotangent;
  ad.f_out = delta_f;
  ad.y0 = ds;
  ad.acc = ds + plane;
  ad.s = ds + 2 * plane;
  ad.v = ds + 3 * plane;
  ad.gx = ds + 4 * plane;
  ad.dsave = dsave;
  cudaStream_t st = (cudaStream_t)stream;
  g_prof = &p->prof;
  cudaError_t e;
  if (p->prec == LF_F64)
    e = run_vjp_ckpt<double>(p->N, p->C, af, ad, ckpt, grads, sink, dacc, batch, nsteps, t0, t1, st);
  else
    e = run_vjp_ckpt<float>(p->N, p->C, af, ad, ckpt, grads, sink, dacc, batch, nsteps, t0, t1, st);
  if (e != cudaSuccess) return cuda_status(e);
  return cuda_status(finish_dphi(p->N, batch, dacc, spec, dphi_f, dphi, dphi_basis, p->tw64, af.kbase, st));
}

int lf_modes_apply(const void* W, int w_batched, unsigned nonzero, const void* X, const void* Y, void* out, int batch,
                   int ncomp, long modes, double scale, double yscale, void* stream) {
  if (batch < 0 || modes < 0 || ncomp < 1 || ncomp > 3) return LF_ERR_BAD_SHAPE;
  if (batch == 0 || modes == 0) return LF_OK;
  if (!W || !X || !out || !aligned16(X) || !aligned16(out) || (Y && !aligned16(Y))) return LF_ERR_BAD_ARG;
  if (reinterpret_cast<uintptr_t>(W) & 7u) return LF_ERR_BAD_ARG;
  const long total = (long)batch * modes;
  const dim3 grid((unsigned)std::min<long>((total + 255) / 256, 148L * 16));
  cudaStream_t st = (cudaStream_t)stream;
  const double* w = static_cast<const double*>(W);
  const double2* x = static_cast<const double2*>(X);
  const double2* y = static_cast<const double2*>(Y);
  double2* o = static_cast<double2*>(out);
  cudaError_t e;
  g_prof = nullptr;
  if (ncomp == 1) e = launch<k_modes_apply<1>>(grid, 256, 0, st, w, w_batched, nonzero, x, y, o, batch, modes, scale, yscale);
  else if (ncomp == 2) e = launch<k_modes_apply<2>>(grid, 256, 0, st, w, w_batched, nonzero, x, y, o, batch, modes, scale, yscale);
  else e = launch<k_modes_apply<3>>(grid, 256, 0, st, w, w_batched, nonzero, x, y, o, batch, modes, scale, yscale);
  return cuda_status(e);
}

int lf_profile_enable(lf_plan_t p, int enable) {
  if (!p) return LF_ERR_BAD_ARG;
  p->prof.on = enable != 0;
  return LF_OK;
}

int lf_profile_reset(lf_plan_t p) {
  if (!p) return LF_ERR_BAD_ARG;
  p->prof.used = 0;
  p->prof.kind.clear();
  return LF_OK;
}

int lf_profile_read(lf_plan_t p, int kind, double* total_ms, int* launches) {
  if (!p || !total_ms || !launches) return LF_ERR_BAD_ARG;
  double tot = 0.0;
  int n = 0;
  const size_t nrec = p->prof.kind.size();
  if (nrec) {
    cudaError_t e = cudaEventSynchronize(p->prof.pool[2 * nrec - 1]);
    if (e != cudaSuccess) return cuda_status(e);
  }
  for (size_t i = 0; i < nrec; ++i) {
    if (p->prof.kind[i] != kind) continue;
    float ms = 0.f;
    cudaError_t e = cudaEventElapsedTime(&ms, p->prof.pool[2 * i], p->prof.pool[2 * i + 1]);
    if (e != cudaSuccess) return cuda_status(e);
    tot += ms;
    ++n;
  }
  *total_ms = tot;
  *launches = n;
  return LF_OK;
}

}  // extern "C"

// ------------------------------------------------ allocation-free entry point
// lf_lense_flow_noalloc keeps its scratch in file-scope device arrays instead
// of caller- or library-allocated memory.  In host code these symbols are
// host-side stand-ins, not device addresses: their device addresses come
// from cudaGetSymbolAddress, taken once per device (with that device current)
// on the first call on the device, and only those addresses reach kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LF_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) float2 g_noalloc_tw[64 + 128 + 256 + 512 + 1024];
// pass table + column table of every supported N, back to back
constexpr int twp_entries(int n) { return ptw_size(n) + ctw_size(n); }
constexpr int kNoAllocTwp = twp_entries(64) + twp_entries(128) + twp_entries(256) + twp_entries(512) + twp_entries(1024);
static __device__ __align__(256) float2 g_noalloc_twp[kNoAllocTwp];

namespace {

struct NoAllocDevice {
  bool ready = false;
  char* scratch = nullptr;  // device address of g_noalloc_scratch
  float2* tw = nullptr;     // device address of g_noalloc_tw
  float2* twp = nullptr;    // device address of g_noalloc_twp
};

constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

int noalloc_tw_offset(int n) {
  return n == 64 ? 0 : n == 128 ? 64 : n == 256 ? 192 : n == 512 ? 448 : 960;
}

int noalloc_twp_offset(int n) {
  int off = 0;
  for (int m = 64; m < n; m *= 2) off += twp_entries(m);
  return off;
}

// Once per device: resolve the arrays' device addresses and fill the twiddle
// tables (exp(-2 pi i k / N), float64 on the host, rounded once) with a
// synchronous copy.  No device or host heap allocation.
int noalloc_setup(NoAllocDevice** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) return LF_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    void* scratch = nullptr;
    void* tw = nullptr;
    e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaGetSymbolAddress(&tw, g_noalloc_tw);
    if (e != cudaSuccess) return cuda_status(e);
    static float2 host[64 + 128 + 256 + 512 + 1024];
    for (int n = 64; n <= 1024; n *= 2) {
      const int off = noalloc_tw_offset(n);
      for (int k = 0; k < n; ++k) {
        const double ang = -2.0 * M_PI * (double)k / (double)n;
        host[off + k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
      }
    }
    e = cudaMemcpyToSymbol(g_noalloc_tw, host, sizeof(host));
    if (e != cudaSuccess) return cuda_status(e);
    void* twp = nullptr;
    e = cudaGetSymbolAddress(&twp, g_noalloc_twp);
    if (e != cudaSuccess) return cuda_status(e);
    static float2 host_p[kNoAllocTwp];
    for (int n = 64; n <= 1024; n *= 2) {
      const int off = noalloc_twp_offset(n);
      fill_pass_table(n, [&](int i, double c, double sn) { host_p[off + i] = make_float2((float)c, (float)sn); });
      fill_col_table(n, [&](int i, double c, double sn) {
        host_p[off + ptw_size(n) + i] = make_float2((float)c, (float)sn);
      });
    }
    e = cudaMemcpyToSymbol(g_noalloc_twp, host_p, sizeof(host_p));
    if (e != cudaSuccess) return cuda_status(e);
    d.scratch = reinterpret_cast<char*>(scratch);
    d.tw = reinterpret_cast<float2*>(tw);
    d.twp = reinterpret_cast<float2*>(twp);
    d.ready = true;
  }
  *out = &d;
  return LF_OK;
}

}  // namespace

extern "C" int lf_lense_flow_noalloc(int nside, int ncomp, double pix_width, const void* f_in, int in_dtype,
                                     void* f_out, int out_dtype, const void* planes, int batch, int nsteps,
                                     int direction, int adjoint, void* stream) {
  if (!valid_n(nside) || ncomp < 1 || ncomp > 3 || batch < 0) return LF_ERR_BAD_SHAPE;
  if ((in_dtype != LF_F32 && in_dtype != LF_F64) || (out_dtype != LF_F32 && out_dtype != LF_F64))
    return LF_ERR_BAD_DTYPE;
  if (!(pix_width > 0.0) || !std::isfinite(pix_width)) return LF_ERR_BAD_ARG;
  if (nsteps < 0 || (direction != LF_FORWARD_LENSE && direction != LF_INVERSE_LENSE)) return LF_ERR_BAD_ARG;
  if (timeout_recorded()) return LF_ERR_TIMEOUT;
  const bool adj = adjoint != 0;
  const size_t npix = (size_t)nside * nside * (size_t)batch * ncomp;
  const size_t plane_bytes = 4 * npix;  // float32 compute
  if (batch == 0) return LF_OK;
  if (!f_in || !f_out || !planes || !aligned16(f_in) || !aligned16(f_out) || !aligned16(planes)) return LF_ERR_BAD_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (nsteps == 0) {  // as lf_lense_flow: the input, needing no scratch
    if (in_dtype != out_dtype) return LF_ERR_BAD_DTYPE;
    if (f_in == f_out) return LF_OK;
    return cuda_status(cudaMemcpyAsync(f_out, f_in, npix * (in_dtype == LF_F64 ? 8 : 4), cudaMemcpyDeviceToDevice, st));
  }
  if (plane_bytes * (adj ? 5 : 4) > (size_t)LF_NOALLOC_SCRATCH_BYTES) return LF_ERR_WORKSPACE;
  NoAllocDevice* d = nullptr;
  const int s = noalloc_setup(&d);
  if (s != LF_OK) return s;
  const bool fwd_time = ((direction == LF_FORWARD_LENSE) != adj);
  const double t0 = fwd_time ? 0.0 : 1.0, t1 = fwd_time ? 1.0 : 0.0;
  StageArgs a;
  std::memset(&a, 0, sizeof(a));
  a.f_in = f_in;
  a.f_out = f_out;
  a.in_f64 = in_dtype == LF_F64;
  a.out_f64 = out_dtype == LF_F64;
  a.phi = planes;
  a.y0 = d->scratch;
  a.acc = d->scratch + plane_bytes;
  a.s = d->scratch + 2 * plane_bytes;
  a.gx = d->scratch + 3 * plane_bytes;
  a.v = adj ? (void*)(d->scratch + 4 * plane_bytes) : nullptr;
  a.twN = d->tw + noalloc_tw_offset(nside);
  a.twP = d->twp + noalloc_twp_offset(nside);
  a.twC = d->twp + noalloc_twp_offset(nside) + ptw_size(nside);
  a.kbase = 2.0 * M_PI / ((double)nside * pix_width);
  a.nplanes = batch * ncomp;
  g_prof = nullptr;
  return cuda_status(run_lens<float>(nside, ncomp, adj, a, batch, nsteps, t0, t1, st));
}
