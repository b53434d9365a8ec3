// Host driver and C ABI (include/dualres_b200.h) of the B200 sampler.
//
// One translation unit holds every kernel (kernels.cu) so that template
// instantiation and the twiddle tables stay in one module.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <unordered_map>
#include <memory>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/dualres_b200.h"
#include "host_setup.h"
#include "kernels.cu"
#include "tc_products.cuh"
#include "mce.cuh"
#include "kriging.cuh"
#include "estimate.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace drb {

// ---------------------------------------------------------------- errors
static thread_local std::string g_err;
static thread_local int64_t g_launches = 0;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                                     \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      throw Error(DR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));                  \
  } while (0)

#define CK_LAUNCH()                                                                                  \
  do {                                                                                               \
    cudaError_t e_ = cudaGetLastError();                                                             \
    if (e_ != cudaSuccess) throw Error(DR_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
    g_launches++;                                                                                    \
  } while (0)

// Launches of the leapfrog kernels allow programmatic dependent launch: the next kernel's grid is set up while the
// previous one drains, and each of these kernels waits for its predecessor (grid_dep_wait) before touching memory.
// DRB_PDL=0 turns it off.
static bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("DRB_PDL");
    return !(e && std::string(e) == "0");
  }();
  return on;
}
template <typename... P, typename... A>
static void launch_k(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  CK(cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...));
}

static int cdiv_i(long long a, long long b) { return (int)((a + b - 1) / b); }

// An NVTX range for the enclosing scope (shown by Nsight tools; no cost without one attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// DRB_TRACE=1: the set-up phases (volume preparation, kriging, tile plans, tuning candidates) print their host
// wall time to stderr when their scope ends.
static bool trace_on() {
  static const bool on = [] {
    const char* e = std::getenv("DRB_TRACE");
    return e && *e && std::string(e) != "0";
  }();
  return on;
}
struct TraceScope {
  std::string name;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit TraceScope(std::string n) : name(std::move(n)) {}
  // ends the current phase and starts the next one
  void next(std::string n) {
    print();
    name = std::move(n);
    t0 = std::chrono::steady_clock::now();
  }
  ~TraceScope() { print(); }
  TraceScope(const TraceScope&) = delete;
  TraceScope& operator=(const TraceScope&) = delete;

 private:
  void print() const {
    if (trace_on())
      std::fprintf(stderr, "[drb] %s: %.2f ms\n", name.c_str(),
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  }
};

// ---------------------------------------------------------------- per-device set-up
struct DeviceTables {
  bool ready = false;
  // The library's stream-ordered allocations come from one memory pool per device that keeps freed memory (release
  // threshold unlimited): a volume's kriging scratch, the tuner's candidate chain sets and a chain set's arrays
  // reuse one another's memory instead of growing and shrinking a pool around every set-up.  The process's default
  // pool is left as it is.
  cudaMemPool_t pool = nullptr;
  int sms = 148;
  int tma_dyn_max = 0;  // dynamic shared memory available to the bulk-copy plane kernel
  bool tc = false;      // the tensor-core kriging products fit this device's shared memory
  const float2* tw_f = nullptr;
  const double2* tw_d = nullptr;
};
static std::mutex g_dev_mtx;
static DeviceTables g_dev[64];

template <int N, class C>
static void set_pass_attrs() {
  const int bytes = N * (TILE_LINES + 1) * (int)sizeof(C);
  CK(cudaFuncSetAttribute(k_pass<N, -1, PRO_LOAD, EPI_STORE, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CK(cudaFuncSetAttribute(k_pass<N, +1, PRO_LOAD, EPI_STORE, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  if constexpr (sizeof(C) == 8) {
    CK(cudaFuncSetAttribute(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaFuncSetAttribute(k_xline<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if constexpr (N == 64 || N == 128 || N == 256) {  // the alternative radix plan (fft_smem PLAN 1)
      CK(cudaFuncSetAttribute(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C, 1, 1>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      CK(cudaFuncSetAttribute(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C, 1, 1>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      CK(cudaFuncSetAttribute(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C, 8, 1>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      CK(cudaFuncSetAttribute(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C, 8, 1>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      CK(cudaFuncSetAttribute(k_xline<N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    }
  }
}

template <int E, bool PF>
static void set_plane_attr(int dyn_max) {
  const PlaneLayout Ly = plane_layout(E, PlaneGeom<E>::SIZE, PF);
  if (Ly.total <= dyn_max)
    CK(cudaFuncSetAttribute(k_xyplane<E, PF>, cudaFuncAttributeMaxDynamicSharedMemorySize, Ly.total));
}

template <class C>
static void set_all_attrs() {
  set_pass_attrs<2, C>(); set_pass_attrs<4, C>(); set_pass_attrs<8, C>(); set_pass_attrs<16, C>();
  set_pass_attrs<32, C>(); set_pass_attrs<64, C>(); set_pass_attrs<128, C>(); set_pass_attrs<256, C>();
  if constexpr (sizeof(C) == 8) set_pass_attrs<512, C>();
}

static DeviceTables& device_tables(int dev) {
  std::lock_guard<std::mutex> lk(g_dev_mtx);
  if (dev < 0 || dev >= 64) throw Error(DR_ERR_INVALID, "device ordinal out of range");
  DeviceTables& t = g_dev[dev];
  if (t.ready) return t;
  CK(cudaSetDevice(dev));
  {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    CK(cudaMemPoolCreate(&t.pool, &props));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(t.pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  std::vector<float2> hf(TW_TOTAL);
  std::vector<double2> hd(TW_TOTAL);
  for (int N = 2; N <= 512; N <<= 1)
    for (int m = 0; m < N; m++) {
      const double a = -2.0 * M_PI * (double)m / (double)N;
      hd[tw_offset(N) + m] = make_double2(std::cos(a), std::sin(a));
      hf[tw_offset(N) + m] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  CK(cudaMemcpyToSymbol(g_tw_f, hf.data(), sizeof(float2) * TW_TOTAL));
  CK(cudaMemcpyToSymbol(g_tw_d, hd.data(), sizeof(double2) * TW_TOTAL));
  void* p = nullptr;
  CK(cudaGetSymbolAddress(&p, g_tw_f));
  t.tw_f = (const float2*)p;
  CK(cudaGetSymbolAddress(&p, g_tw_d));
  t.tw_d = (const double2*)p;
  set_all_attrs<float2>();
  set_all_attrs<double2>();
  {
    int sms = 0, optin = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    t.sms = sms;
    t.tma_dyn_max = optin - 256;  // the plane kernels' static shared memory is at most 128 bytes
    set_plane_attr<4, false>(t.tma_dyn_max); set_plane_attr<8, false>(t.tma_dyn_max);
    set_plane_attr<16, false>(t.tma_dyn_max); set_plane_attr<32, false>(t.tma_dyn_max);
    set_plane_attr<64, false>(t.tma_dyn_max); set_plane_attr<128, false>(t.tma_dyn_max);
    set_plane_attr<4, true>(t.tma_dyn_max); set_plane_attr<8, true>(t.tma_dyn_max);
    set_plane_attr<16, true>(t.tma_dyn_max); set_plane_attr<32, true>(t.tma_dyn_max);
    set_plane_attr<64, true>(t.tma_dyn_max);
    CK(cudaFuncSetAttribute(k_kriging_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(KrigSmem)));
    int smax = 0;
    for (int n = 16; n <= 256; n *= 2) smax = std::max(smax, tc_smem_bytes(n));
    t.tc = optin >= smax;
    if (t.tc) {
      CK(cudaFuncSetAttribute(k_tc_product<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
      CK(cudaFuncSetAttribute(k_tc_product<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
    }
  }
  t.ready = true;
  return t;
}

// Stream-ordered allocation on the current device from the library's pool.
static cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
  int dev = 0;
  const cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, bytes, device_tables(dev).pool, st);
}

// ---------------------------------------------------------------- pass launcher
template <int N, class C>
static void launch_pass_n(int dir, int pro, int epi, const PassArgs& a, const DevVolume& v, const DevChains& ch,
                          const C* tw, int nch, cudaStream_t s) {
  const dim3 grid(cdiv_i((long long)a.A * a.B, TILE_LINES), a.chain_only >= 0 ? 1 : nch);
  const dim3 block(PassCfg<N>::NT);
  const size_t smem = (size_t)N * (TILE_LINES + 1) * sizeof(C);
  if (dir < 0 && pro == PRO_LOAD && epi == EPI_STORE)
    launch_k(k_pass<N, -1, PRO_LOAD, EPI_STORE, C>, grid, block, smem, s, a, v, ch, tw);
  else if (dir > 0 && pro == PRO_LOAD && epi == EPI_STORE)
    launch_k(k_pass<N, +1, PRO_LOAD, EPI_STORE, C>, grid, block, smem, s, a, v, ch, tw);
  else if constexpr (sizeof(C) == 8) {
    // the z passes touch the chain-minor arrays: with 8 or more chains, tiles of 4 lines x 8 chains unless the chain
    // set's tuning chose tiles of 32 lines of one chain (ch.ztile)
    const bool grouped = a.chain_only < 0 && nch >= 8 && a.B > 1 && ch.ztile != 1;
    const dim3 ggrid(cdiv_i((long long)a.A * a.B, TILE_LINES / 8), cdiv_i(nch, 8));
    // the radix plan the chain set's tuning chose (ch.fftplan) for the lengths that have two
    constexpr bool two_plans = N == 64 || N == 128 || N == 256;
    const bool alt = two_plans && (ch.fftplan & (dir > 0 ? FP_ZINV : FP_ZFWD)) != 0;
    if (dir > 0 && pro == PRO_DATAGRAD && epi == EPI_STORE) {
      if (alt && grouped) launch_k(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C, 8, 1>, ggrid, block, smem, s, a, v, ch, tw);
      else if (alt) launch_k(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C, 1, 1>, grid, block, smem, s, a, v, ch, tw);
      else if (grouped) launch_k(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C, 8>, ggrid, block, smem, s, a, v, ch, tw);
      else launch_k(k_pass<N, +1, PRO_DATAGRAD, EPI_STORE, C>, grid, block, smem, s, a, v, ch, tw);
    } else if (dir < 0 && pro == PRO_LOAD && epi == EPI_GATHER) {
      if (alt && grouped) launch_k(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C, 8, 1>, ggrid, block, smem, s, a, v, ch, tw);
      else if (alt) launch_k(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C, 1, 1>, grid, block, smem, s, a, v, ch, tw);
      else if (grouped) launch_k(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C, 8>, ggrid, block, smem, s, a, v, ch, tw);
      else launch_k(k_pass<N, -1, PRO_LOAD, EPI_GATHER, C>, grid, block, smem, s, a, v, ch, tw);
    } else {
      throw Error(DR_ERR_INVALID, "unsupported pass combination");
    }
  } else {
    throw Error(DR_ERR_INVALID, "unsupported pass combination");
  }
  CK_LAUNCH();
}

template <class C>
static void launch_pass(int n, int dir, int pro, int epi, const PassArgs& a, const DevVolume& v, const DevChains& ch,
                        const C* tw, int nch, cudaStream_t s) {
  switch (n) {
    case 2: launch_pass_n<2, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 4: launch_pass_n<4, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 8: launch_pass_n<8, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 16: launch_pass_n<16, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 32: launch_pass_n<32, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 64: launch_pass_n<64, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 128: launch_pass_n<128, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 256: launch_pass_n<256, C>(dir, pro, epi, a, v, ch, tw, nch, s); break;
    case 512:
      if constexpr (sizeof(C) == 8) {
        launch_pass_n<512, C>(dir, pro, epi, a, v, ch, tw, nch, s);
        break;
      }
      [[fallthrough]];
    default: throw Error(DR_ERR_UNSUPPORTED, "FFT length not supported: " + std::to_string(n));
  }
}

static PassArgs pass_args(const void* in, void* out, long long in_cs, long long out_cs, int A, int B, int n_in,
                          int n_out, double scale = 1.0, int step = -1, int sel = 0, int write_o = 0,
                          int chain_only = -1) {
  PassArgs a;
  a.in = in; a.out = out; a.in_cs = in_cs; a.out_cs = out_cs;
  a.A = A; a.B = B; a.n_in = n_in; a.n_out = n_out; a.scale = scale;
  a.step = step; a.sel = sel; a.write_o = write_o; a.chain_only = chain_only;
  return a;
}

// Unpruned in-place 3D FFT of one (or nch chain-strided) field(s).
template <class C>
static void fft3d(C* f, const int* E, int dir, long long cs, int nch, const C* tw, cudaStream_t s,
                  const DevVolume& v, const DevChains& ch, int chain_only = -1) {
  const int E0 = E[0], E1 = E[1], E2 = E[2];
  if (dir < 0) {
    launch_pass<C>(E0, -1, PRO_LOAD, EPI_STORE, pass_args(f, f, cs, cs, E1 * E2, 1, E0, E0, 1.0, -1, 0, 0, chain_only), v, ch, tw, nch, s);
    launch_pass<C>(E1, -1, PRO_LOAD, EPI_STORE, pass_args(f, f, cs, cs, E2, E0, E1, E1, 1.0, -1, 0, 0, chain_only), v, ch, tw, nch, s);
    launch_pass<C>(E2, -1, PRO_LOAD, EPI_STORE, pass_args(f, f, cs, cs, 1, E0 * E1, E2, E2, 1.0, -1, 0, 0, chain_only), v, ch, tw, nch, s);
  } else {
    launch_pass<C>(E0, +1, PRO_LOAD, EPI_STORE, pass_args(f, f, cs, cs, E1 * E2, 1, E0, E0, 1.0, -1, 0, 0, chain_only), v, ch, tw, nch, s);
    launch_pass<C>(E1, +1, PRO_LOAD, EPI_STORE, pass_args(f, f, cs, cs, E2, E0, E1, E1, 1.0, -1, 0, 0, chain_only), v, ch, tw, nch, s);
    launch_pass<C>(E2, +1, PRO_LOAD, EPI_STORE, pass_args(f, f, cs, cs, 1, E0 * E1, E2, E2, 1.0, -1, 0, 0, chain_only), v, ch, tw, nch, s);
  }
}

// ---------------------------------------------------------------- volume
struct Volume {
  int device = 0;
  cudaStream_t stream = nullptr;  // uploads, spectrum and stream-ordered frees
  // Chain sets bound to this volume; a volume released while some remain is
  // freed by the last of them (g_vol_mtx guards both fields).
  int n_chainsets = 0;
  bool released = false;
  HostVolume hv;
  DevVolume dv{};
  std::vector<void*> allocs;
  double* lam_re = nullptr;
  int n_S = 0;
  double max_eig = 0.0;
  double setup_seconds = 0.0;
  int64_t bytes = 0;
  const float2* tw_f = nullptr;
  const double2* tw_d = nullptr;
  // Dense-tile form of W and W^T for the tensor-core products, built on first use by a chain set that can use
  // it (tc_state 0: not built, 1: built, -1: unavailable).
  std::mutex tc_mtx;
  int tc_state = 0;
  DevTcMatrix tc_w{}, tc_wt{};
  int tc_max_segs = 0;
  double tc_seconds = 0.0;

  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    const cudaError_t e = dev_alloc(&p, n * sizeof(T), stream);
    if (e != cudaSuccess) throw Error(DR_ERR_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    bytes += (int64_t)(n * sizeof(T));
    return (T*)p;
  }
  template <class T, class A>
  T* upload(const std::vector<T, A>& h) {
    T* d = alloc<T>(h.size());
    if (!h.empty()) CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return d;
  }
  virtual ~Volume() {
    if (stream) {
      cudaSetDevice(device);
      for (void* p : allocs) cudaFreeAsync(p, stream);
      cudaStreamDestroy(stream);
      cudaGetLastError();  // a failed release must not surface in the caller's next launch check
    }
  }
};

static std::mutex g_vol_mtx;


// Kriging weights of a prepared volume on the device (k_kriging_rows), then
// the CSR, its transpose and the host copies.  Rows whose system is not
// numerically positive definite are solved on the host by the same rule as
// the host builder (QR).
static bool device_kriging_enabled() { return std::getenv("DRB_HOST_KRIGING") == nullptr; }

// S = K^-1 on the device by the blocked kernels of kriging.cuh (factor, triangular inverse, Gram product), all
// CTAs of the GPU taking part; dK (m x m) is left unchanged and dS receives S.  Returns false when K is not
// positive definite.  Scratch comes from dalloc.
template <class Alloc>
static bool device_spd_inverse(const double* dK, int m, double* dS, cudaStream_t st, Alloc&& dalloc) {
  const int nb = (m + KR_NB - 1) / KR_NB;
  double* dM = (double*)dalloc(sizeof(double) * (size_t)m * m);
  double* dX = (double*)dalloc(sizeof(double) * (size_t)m * m);
  double* dDinv = (double*)dalloc(sizeof(double) * (size_t)nb * KR_NB * KR_NB);
  int* dok = (int*)dalloc(sizeof(int));
  static const int one = 1;
  CK(cudaMemcpyAsync(dM, dK, sizeof(double) * (size_t)m * m, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpyAsync(dok, &one, sizeof(int), cudaMemcpyHostToDevice, st));
  TraceScope tr("K^-1: factor (" + std::to_string(nb) + " panels)");
  for (int k0 = 0; k0 < m; k0 += KR_NB) {
    k_chol_diag<<<1, KR_NT, 0, st>>>(dM, m, k0, dDinv, dok);
    CK_LAUNCH();
    const int r0 = std::min(m, k0 + KR_NB);
    if (r0 >= m) break;
    const int T = cdiv_i(m - r0, KR_TILE);
    k_chol_panel<<<T, KR_NT, 0, st>>>(dM, m, k0, dDinv, dok);
    CK_LAUNCH();
    k_chol_update<<<T * (T + 1) / 2, KR_NT, 0, st>>>(dM, m, k0, dok);
    CK_LAUNCH();
  }
  int ok = 0;
  CK(cudaMemcpyAsync(&ok, dok, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (!ok) return false;
  tr.next("K^-1: triangular inverse + Gram product");
  for (int bi = 0; bi < nb; bi++) {
    k_trinv_row<<<bi + 1, KR_NT, 0, st>>>(dM, m, bi, dDinv, dX, dok);
    CK_LAUNCH();
  }
  k_trinv_gram<<<nb * (nb + 1) / 2, KR_NT, 0, st>>>(dX, m, dS, dok);
  CK_LAUNCH();
  if (trace_on()) CK(cudaStreamSynchronize(st));
  return true;
}

static void kriging_solve_device(HostVolume& hv, int device, cudaStream_t st) {
  const auto t0 = std::chrono::steady_clock::now();
  KrigingPlan& P = hv.kplan;
  const int m = P.m, nrows = P.nrows;
  CK(cudaSetDevice(device));
  DeviceTables& dt = device_tables(device);
  std::vector<void*> bufs;
  auto dalloc = [&](size_t bytes) {
    void* p = nullptr;
    const cudaError_t e = dev_alloc(&p, std::max<size_t>(bytes, 16), st);
    if (e != cudaSuccess) throw Error(DR_ERR_NOMEM, std::string("device allocation (kriging): ") + cudaGetErrorString(e));
    bufs.push_back(p);
    return p;
  };
  auto upload = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  };
  fill_vector<double> w(P.col.size());  // every entry comes back from the device (zeroed there)
  std::vector<char> keep(nrows, 1);
  std::vector<int> status(nrows, KR_OK);
  std::vector<int> dup_of(nrows, -1);
  int ntasks = 0;
  bool have_inv = false;
  try {
    double* dK = (double*)dalloc(sizeof(double) * (size_t)m * m);
    upload(dK, P.K.data(), sizeof(double) * (size_t)m * m);
    double* dS = nullptr;
    if (!P.S.empty()) {  // computed on the host
      dS = (double*)dalloc(sizeof(double) * (size_t)m * m);
      upload(dS, P.S.data(), sizeof(double) * (size_t)m * m);
      have_inv = true;
    } else if (P.inverse_wanted && m > 0) {
      const TraceScope tr("kriging: K^-1 (m = " + std::to_string(m) + ")");
      dS = (double*)dalloc(sizeof(double) * (size_t)m * m);
      have_inv = device_spd_inverse(dK, m, dS, st, dalloc);
    }
    TraceScope tr_rows("kriging: row tasks");
    // tasks: every row with neighbours; complete rows with equal k' are solved once (grouped by a hash of k', then
    // compared in place)
    std::vector<uint64_t> kh(nrows, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int ri = 0; ri < nrows; ri++) {
      const int r0 = P.row_start[ri], cnt = P.row_start[ri + 1] - r0;
      if (cnt != m) continue;
      uint64_t h = 1469598103934665603ull;  // FNV-1a over the bytes of k'
      const unsigned char* b = reinterpret_cast<const unsigned char*>(P.kp.data() + r0);
      for (size_t i = 0; i < (size_t)cnt * sizeof(double); i++) h = (h ^ b[i]) * 1099511628211ull;
      kh[ri] = h;
    }
    std::unordered_map<uint64_t, std::vector<int>> rep;
    std::vector<std::pair<double, int>> order;
    std::vector<int> route(nrows, 0);
    int nmax = 1;
    for (int ri = 0; ri < nrows; ri++) {
      const int r0 = P.row_start[ri], cnt = P.row_start[ri + 1] - r0;
      if (cnt == 0) continue;
      if (cnt == m) {
        std::vector<int>& reps = rep[kh[ri]];
        int found = -1;
        for (int o : reps)
          if (std::memcmp(P.kp.data() + P.row_start[o], P.kp.data() + r0, sizeof(double) * (size_t)cnt) == 0) {
            found = o;
            break;
          }
        if (found >= 0) {
          dup_of[ri] = found;
          continue;
        }
        reps.push_back(ri);
      }
      const bool schur = kriging_schur_route(cnt, m, have_inv);
      route[ri] = schur ? KR_ROUTE_SCHUR : KR_ROUTE_DIRECT;
      const int n = schur ? m - cnt : cnt;
      nmax = std::max(nmax, n);
      const double cost = (double)n * n * n / 3.0 + (schur ? 2.0 * m * cnt : 0.0);
      order.emplace_back(-cost, ri);
    }
    std::sort(order.begin(), order.end());
    ntasks = (int)order.size();
    std::vector<int> task_row(std::max(ntasks, 1)), task_route(std::max(ntasks, 1));
    for (int t = 0; t < ntasks; t++) {
      task_row[t] = order[t].second;
      task_route[t] = route[order[t].second];
    }
    if (ntasks > 0) {
      const size_t slot = (size_t)nmax * (nmax + 1) / 2 + m + nmax + (m + 1) / 2 + 1;
      int grid = std::min(ntasks, 2 * dt.sms);
      const size_t budget = (size_t)2 << 30;  // scratch cap
      grid = std::max(1, std::min(grid, (int)(budget / (slot * sizeof(double)))));
      tr_rows.next("kriging: scratch + uploads (" + std::to_string(ntasks) + " tasks, n <= " + std::to_string(nmax) +
                   ", " + std::to_string(grid) + " blocks, " + std::to_string(slot * grid * sizeof(double) >> 20) +
                   " MiB scratch)");
      KrigArgs a{};
      a.m = m;
      a.K = dK;
      a.S = dS;
      int* d_rs = (int*)dalloc(sizeof(int) * (nrows + 1));
      upload(d_rs, P.row_start.data(), sizeof(int) * (nrows + 1));
      int* d_pid = (int*)dalloc(sizeof(int) * P.pid.size());
      upload(d_pid, P.pid.data(), sizeof(int) * P.pid.size());
      double* d_kp = (double*)dalloc(sizeof(double) * P.kp.size());
      upload(d_kp, P.kp.data(), sizeof(double) * P.kp.size());
      int* d_tr = (int*)dalloc(sizeof(int) * ntasks);
      upload(d_tr, task_row.data(), sizeof(int) * ntasks);
      int* d_tt = (int*)dalloc(sizeof(int) * ntasks);
      upload(d_tt, task_route.data(), sizeof(int) * ntasks);
      int* d_cnt = (int*)dalloc(sizeof(int));
      CK(cudaMemsetAsync(d_cnt, 0, sizeof(int), st));
      double* d_w = (double*)dalloc(sizeof(double) * w.size());
      CK(cudaMemsetAsync(d_w, 0, sizeof(double) * w.size(), st));
      int* d_status = (int*)dalloc(sizeof(int) * nrows);
      CK(cudaMemsetAsync(d_status, 0, sizeof(int) * nrows, st));
      double* d_scr = (double*)dalloc(sizeof(double) * slot * grid);
      a.row_start = d_rs;
      a.pid = d_pid;
      a.kp = d_kp;
      a.task_row = d_tr;
      a.task_route = d_tt;
      a.ntasks = ntasks;
      a.counter = d_cnt;
      a.w = d_w;
      a.status = d_status;
      a.scratch = d_scr;
      a.slot = slot;
      a.nmax = nmax;
      if (trace_on()) {
        CK(cudaStreamSynchronize(st));
        tr_rows.next("kriging: row-solve kernel + download");
      }
      k_kriging_rows<<<grid, KR_NT, sizeof(KrigSmem), st>>>(a);
      CK_LAUNCH();
      CK(cudaMemcpyAsync(w.data(), d_w, sizeof(double) * w.size(), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(status.data(), d_status, sizeof(int) * nrows, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
    // the host route of rows the device could not factor reads K^-1 when it chooses the Schur route
    bool any_redo = false;
    for (int ri = 0; ri < nrows; ri++) any_redo |= dup_of[ri] < 0 && status[ri] == KR_NOT_SPD;
    if (any_redo && have_inv && P.S.empty()) {
      P.S.resize((size_t)m * m);
      CK(cudaMemcpyAsync(P.S.data(), dS, sizeof(double) * (size_t)m * m, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
  } catch (...) {
    for (void* p : bufs) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaGetLastError();
    throw;
  }
  for (void* p : bufs) cudaFreeAsync(p, st);
  CK(cudaStreamSynchronize(st));
  const TraceScope tr_host("kriging: host rows, assemble, transpose");
  // rows the device could not factor: host route (Cholesky / QR)
  std::vector<int> redo;
  for (int ri = 0; ri < nrows; ri++) {
    if (dup_of[ri] >= 0) continue;
    if (status[ri] == KR_DROP) keep[ri] = 0;
    if (status[ri] == KR_NOT_SPD) redo.push_back(ri);
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < (int)redo.size(); i++) {
    std::vector<double> x;
    const int ri = redo[i];
    if (kriging_solve_row_host(P, ri, &x)) std::copy(x.begin(), x.end(), w.begin() + P.row_start[ri]);
    else keep[ri] = 0;
  }
  for (int ri = 0; ri < nrows; ri++) {
    const int src = dup_of[ri];
    if (src < 0) continue;
    keep[ri] = keep[src];
    std::copy(w.begin() + P.row_start[src], w.begin() + P.row_start[src + 1], w.begin() + P.row_start[ri]);
  }
  kriging_assemble(P, w.data(), keep, &hv.w_rowptr, &hv.w_col, &hv.w_val);
  hv.kplan = KrigingPlan();
  hv.kriging_pending = false;
  hv.kriging_device_rows = ntasks;
  hv.kriging_host_rows = (int)redo.size();
  build_transpose(&hv);
  const double dt_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  hv.kriging_solve_seconds = dt_s;
  hv.kriging_seconds += dt_s;
}

// Device part of a volume from an already prepared HostVolume (V->hv).
static void volume_build_device(Volume* V, const float* covariance, int covfun, int device) {
  const NvtxRange range("volume: device set-up (kriging solves, FP64 spectrum)");
  const auto t0 = std::chrono::steady_clock::now();
  V->device = device;
  DeviceTables& dt = device_tables(device);
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&V->stream, cudaStreamNonBlocking));
  V->tw_f = dt.tw_f;
  V->tw_d = dt.tw_d;
  HostVolume& hv = V->hv;
  if (hv.kriging_pending) kriging_solve_device(hv, device, V->stream);
  const TraceScope tr("volume: uploads + FP64 spectrum");
  DevVolume& dv = V->dv;
  cudaStream_t st = V->stream;
  dv.E0 = hv.E[0]; dv.E1 = hv.E[1]; dv.E2 = hv.E[2]; dv.N = hv.N;
  dv.bx = hv.box[0]; dv.by = hv.box[1]; dv.bz = hv.box[2];
  dv.n_h = (int)hv.Yh.size(); dv.n_s = (int)hv.Ys.size(); dv.n_o = (int)hv.o_flat.size();
  dv.box_to_d = V->upload(hv.box_to_d);
  dv.box_to_o = V->upload(hv.box_to_o);
  dv.d_flat = V->upload(hv.d_flat);
  dv.o_flat = V->upload(hv.o_flat);
  dv.Yh = V->upload(hv.Yh);
  dv.Ys = V->upload(hv.Ys);
  dv.w_rowptr = V->upload(hv.w_rowptr.empty() ? std::vector<int>{0} : hv.w_rowptr);
  dv.w_col = V->upload(hv.w_col);
  dv.w_val = V->upload(hv.w_val);
  dv.wt_rowptr = V->upload(hv.wt_rowptr);
  dv.wt_col = V->upload(hv.wt_col);
  dv.wt_val = V->upload(hv.wt_val);

  // eigenvalues in FP64: base -> 3 forward passes -> S, 1/lambda
  const long long N = hv.N;
  float* sinv = V->alloc<float>(N);
  V->lam_re = V->alloc<double>(N);
  double2* base = nullptr;
  int* nS = nullptr;
  CK(dev_alloc((void**)&base, sizeof(double2) * N, st));
  const cudaError_t e2 = dev_alloc((void**)&nS, sizeof(int), st);
  if (e2 != cudaSuccess) {
    cudaFreeAsync(base, st);
    throw Error(DR_ERR_NOMEM, "device allocation (spectrum scratch)");
  }
  try {
    CK(cudaMemsetAsync(nS, 0, sizeof(int), st));
    const float* Q = hv.Q;
    k_base<<<cdiv_i(N, 256), 256, 0, st>>>(base, hv.E[0], hv.E[1], hv.E[2], Q[0], Q[1], Q[2], Q[4], Q[5], Q[6], Q[8],
                                           Q[9], Q[10], (double)covariance[0], (double)covariance[1],
                                           (double)covariance[2], covfun);
    CK_LAUNCH();
    DevChains none{};
    fft3d<double2>(base, hv.E, -1, 0, 1, V->tw_d, st, dv, none);
    k_spectrum<<<cdiv_i(N, 256), 256, 0, st>>>(base, sinv, V->lam_re, N, nS);
    CK_LAUNCH();
    double2 l0;
    CK(cudaMemcpyAsync(&l0, base, sizeof(double2), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&V->n_S, nS, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    V->max_eig = l0.x / (double)N;
  } catch (...) {
    cudaFreeAsync(base, st);
    cudaFreeAsync(nS, st);
    throw;
  }
  cudaFreeAsync(base, st);
  cudaFreeAsync(nS, st);
  dv.sinv = sinv;
  if ((long long)V->n_S >= N / 2) throw Error(DR_ERR_DOMAIN, "Too many negative eigen values");
  CK(cudaStreamSynchronize(st));
  V->setup_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

static void volume_build(Volume* V, const dr_volume_desc* d) {
  const NvtxRange range("volume: create");
  const auto t0 = std::chrono::steady_clock::now();
  device_tables(d->device);
  std::string err;
  int rc;
  {
    const TraceScope tr("volume: host preparation (indices, kriging plan)");
    rc = host_prepare(d, &V->hv, &err, device_kriging_enabled());
  }
  if (rc != DR_OK) throw Error(rc, err);
  V->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  volume_build_device(V, d->covariance, d->covfun, d->device);
}

// ---------------------------------------------------------------- chainset
struct Chainset {
  Volume* vol = nullptr;
  int C = 0;
  dr_hmc_opts opts{};
  DevChains dc{};
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_nodes = 0;
  std::vector<void*> allocs;
  float2* tmp = nullptr;        // [N] scratch for evaluation calls
  int NR = 1;
  bool plane = false;           // fused xy-plane update (E0 == E1 <= 128)
  int path = 0;                 // 0 plane kernel, 1 plane kernel with bulk prefetch, 2 x-line kernel + y passes
  int grid = 8;                 // kriging-product blocks per SM
  double tuned_ms = 0.0;        // iteration time of the chosen configuration when it was tuned (0: not tuned)
  bool tcp = false;             // kriging products on the tensor cores (dense tiles of the volume)
  int tc_N = 0;                 // chains per tensor-core product (power of two >= C)
  float* tc_partial = nullptr;  // [segments][tc_N][128] partial products
  bool tc_tg = false;           // W^T rs: the chain vectors arrive by TMA row gathers over tc_map_wt
  CUtensorMap tc_map_w{}, tc_map_wt{};  // (tc_map_w unused: W mu_D gathers with its threads); rs as [n_s] rows
  bool tma = false;             // path 1
  int tma_smem = 0, tma_grid = 0;

  int64_t bytes = 0;
  cudaEvent_t done_event = nullptr;  // recorded after the last launched iteration (server)

  template <class T>
  T* alloc(size_t n, bool zero = true) {
    void* p = nullptr;
    if (n == 0) n = 1;
    const cudaError_t e = dev_alloc(&p, n * sizeof(T), stream);
    if (e != cudaSuccess) throw Error(DR_ERR_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    allocs.push_back(p);
    bytes += (int64_t)(n * sizeof(T));
    if (zero) CK(cudaMemsetAsync(p, 0, n * sizeof(T), stream));
    return (T*)p;
  }
  int device = 0;
  ~Chainset() {
    cudaSetDevice(device);
    // Drain the chain set's work before anything is freed: its kernels read the volume's arrays, and the volume
    // frees them on its own stream, which is not ordered after this one (a chain set destroyed on an error path
    // may still have work in flight).
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (done_event) cudaEventDestroy(done_event);
    if (stream) {
      for (void* p : allocs) cudaFreeAsync(p, stream);
      cudaStreamDestroy(stream);
    }
    cudaGetLastError();
    if (vol) {
      bool last = false;
      {
        std::lock_guard<std::mutex> lk(g_vol_mtx);
        last = --vol->n_chainsets == 0 && vol->released;
      }
      if (last) delete vol;
    }
  }
};

// Frees a volume now, or when its last chain set is destroyed.
static void volume_release(Volume* v) {
  if (!v) return;
  {
    std::lock_guard<std::mutex> lk(g_vol_mtx);
    v->released = true;
    if (v->n_chainsets > 0) return;
  }
  delete v;
}

template <int CG, int NR>
static void launch_spmv_t(const DevVolume& v, const DevChains& ch, int nb, int step, int sel, int chain_only, bool w,
                          cudaStream_t s) {
  // a block per row while a block gets few rows; with at most 8 chains per warp, a warp per row once a block would
  // take 8 or more of them in turn
  bool rows = false;
  if constexpr (CG <= 8) rows = w && v.n_s >= 8 * nb;
  if (rows) {
    if constexpr (CG <= 8) launch_k(k_spmv_w_rows<CG, NR>, nb, 256, 0, s, v, ch, step, sel, chain_only);
  } else if (w) {
    launch_k(k_spmv_w<CG, NR>, nb, 256, 0, s, v, ch, step, sel, chain_only);
  } else
    launch_k(k_spmv_wt<CG, NR>, nb, 256, 0, s, v, ch, step, sel, chain_only);
  CK_LAUNCH();
}

// Kriging products for `ch` (chain group width CG = ch.CG, rounds NR).
static void launch_spmv_dc(const DevVolume& v, const DevChains& ch, int NR, int step, int sel, int chain_only, bool w,
                           cudaStream_t s) {
  const int nb = w ? std::max(1, std::min(v.n_s, ch.nb_w)) : std::max(1, std::min(cdiv_i(v.n_h, 8), ch.nb_wt));
  if (nb > ch.maxblk || ch.part == nullptr) throw Error(DR_ERR_STATE, "partial-sum buffer smaller than the block count");
  switch (ch.CG) {
    case 1: launch_spmv_t<1, 1>(v, ch, nb, step, sel, chain_only, w, s); break;
    case 2: launch_spmv_t<2, 1>(v, ch, nb, step, sel, chain_only, w, s); break;
    case 4: launch_spmv_t<4, 1>(v, ch, nb, step, sel, chain_only, w, s); break;
    case 8: launch_spmv_t<8, 1>(v, ch, nb, step, sel, chain_only, w, s); break;
    case 16: launch_spmv_t<16, 1>(v, ch, nb, step, sel, chain_only, w, s); break;
    default:
      switch (NR) {
        case 1: launch_spmv_t<32, 1>(v, ch, nb, step, sel, chain_only, w, s); break;
        case 2: launch_spmv_t<32, 2>(v, ch, nb, step, sel, chain_only, w, s); break;
        case 4: launch_spmv_t<32, 4>(v, ch, nb, step, sel, chain_only, w, s); break;
        default: launch_spmv_t<32, 8>(v, ch, nb, step, sel, chain_only, w, s); break;
      }
  }
}

// W mu_D (w) or W^T rs on the tensor cores: the tile products into segment partials, then the per-tile sums and
// the same epilogue as the CSR kernels.
static void launch_tc(Chainset* S, int step, int sel, int chain_only, bool w) {
  const Volume* V = S->vol;
  const DevTcMatrix& M = w ? V->tc_w : V->tc_wt;
  const int N = S->tc_N;
  const int nfin = tc_finish_blocks(M.T);
  if (nfin > S->dc.maxblk || S->tc_partial == nullptr)
    throw Error(DR_ERR_STATE, "partial-sum buffer smaller than the finishing block count");
  if (M.G > 0) {
    const int n_h = V->dv.n_h, mode = w ? 0 : 1;
    const size_t sm = tc_smem_bytes(N);
    const CUtensorMap& xm = w ? S->tc_map_w : S->tc_map_wt;
    float* P = S->tc_partial;
    // TMA row gathers for W^T rs (one row set per chunk); W mu_D would need both halves of mu_D per chunk, twice
    // the gathered bytes in twice the operations, and measured faster with the threads' own loads
    const bool tg = S->tc_tg && !w;
#define DRB_TC_LAUNCH(NN)                                                                                 \
  if (tg) launch_k(k_tc_product<NN, true>, M.G, tc_threads(NN), sm, S->stream, M, S->dc, n_h, sel, mode, P, xm); \
  else launch_k(k_tc_product<NN, false>, M.G, tc_threads(NN), sm, S->stream, M, S->dc, n_h, sel, mode, P, xm);
    switch (N) {
      case 16: DRB_TC_LAUNCH(16) break;
      case 32: DRB_TC_LAUNCH(32) break;
      case 64: DRB_TC_LAUNCH(64) break;
      case 128: DRB_TC_LAUNCH(128) break;
      default: DRB_TC_LAUNCH(256) break;
    }
#undef DRB_TC_LAUNCH
    CK_LAUNCH();
  }
  const size_t fs = tc_finish_smem_bytes(N);
  const int fm = w ? 0 : 1;
  switch (N) {
    case 16: launch_k(k_tc_finish<16>, nfin, 256, fs, S->stream, M, S->tc_partial, V->dv, S->dc, step, sel, chain_only, fm); break;
    case 32: launch_k(k_tc_finish<32>, nfin, 256, fs, S->stream, M, S->tc_partial, V->dv, S->dc, step, sel, chain_only, fm); break;
    case 64: launch_k(k_tc_finish<64>, nfin, 256, fs, S->stream, M, S->tc_partial, V->dv, S->dc, step, sel, chain_only, fm); break;
    case 128: launch_k(k_tc_finish<128>, nfin, 256, fs, S->stream, M, S->tc_partial, V->dv, S->dc, step, sel, chain_only, fm); break;
    default: launch_k(k_tc_finish<256>, nfin, 256, fs, S->stream, M, S->tc_partial, V->dv, S->dc, step, sel, chain_only, fm); break;
  }
  CK_LAUNCH();
}

static void launch_spmv(Chainset* S, int step, int sel, int chain_only, bool w) {
  if (S->tcp) launch_tc(S, step, sel, chain_only, w);
  else launch_spmv_dc(S->vol->dv, S->dc, S->NR, step, sel, chain_only, w, S->stream);
}

// The update kernels' L2 prefetch of their state (XF_L2_PREFETCH); DRB_L2_PREFETCH=0 turns it off.
static int l2_prefetch_flag() {
  static const int f = [] {
    const char* e = std::getenv("DRB_L2_PREFETCH");
    return (e && std::string(e) == "0") ? 0 : (int)XF_L2_PREFETCH;
  }();
  return f;
}

static void launch_xline(Chainset* S, int step, int flags) {
  flags |= l2_prefetch_flag();
  const DevVolume& v = S->vol->dv;
  if (cdiv_i((long long)v.E1 * v.E2, TILE_LINES) > S->dc.maxblk)
    throw Error(DR_ERR_STATE, "partial-sum buffer smaller than the x-line block count");
  const dim3 grid(cdiv_i((long long)v.E1 * v.E2, TILE_LINES), S->C);
  const size_t smem = (size_t)v.E0 * (TILE_LINES + 1) * sizeof(float2);
  const float2* tw = S->vol->tw_f;
  switch (v.E0) {
    case 2: launch_k(k_xline<2>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw); break;
    case 4: launch_k(k_xline<4>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw); break;
    case 8: launch_k(k_xline<8>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw); break;
    case 16: launch_k(k_xline<16>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw); break;
    case 32: launch_k(k_xline<32>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw); break;
    case 64:
      if (S->dc.fftplan & FP_XLINE) launch_k(k_xline<64, 1>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw);
      else launch_k(k_xline<64>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw);
      break;
    case 128:
      if (S->dc.fftplan & FP_XLINE) launch_k(k_xline<128, 1>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw);
      else launch_k(k_xline<128>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw);
      break;
    case 256:
      if (S->dc.fftplan & FP_XLINE) launch_k(k_xline<256, 1>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw);
      else launch_k(k_xline<256>, grid, 256, smem, S->stream, v, S->dc, step, flags, tw);
      break;
    case 512: launch_k(k_xline<512>, grid, 512, smem, S->stream, v, S->dc, step, flags, tw); break;
    default: throw Error(DR_ERR_UNSUPPORTED, "E0 not supported");
  }
  CK_LAUNCH();
}

template <int E, bool PF>
static void launch_plane_t(Chainset* S, int step, int flags) {
  flags |= l2_prefetch_flag();
  const DevVolume& v = S->vol->dv;
  const dim3 grid(v.E2, S->C);
  const size_t smem = (size_t)plane_layout(E, PlaneGeom<E>::SIZE, PF).total;
  launch_k(k_xyplane<E, PF>, grid, PlaneCfg<E, PF>::NT, smem, S->stream, v, S->dc, step, flags, S->vol->tw_f);
  CK_LAUNCH();
}

static void launch_plane(Chainset* S, int step, int flags) {
  const DevVolume& v = S->vol->dv;
  if (v.E2 > S->dc.maxblk) throw Error(DR_ERR_STATE, "partial-sum buffer smaller than the plane count");
  if (S->tma) {
    switch (v.E0) {
      case 4: launch_plane_t<4, true>(S, step, flags); return;
      case 8: launch_plane_t<8, true>(S, step, flags); return;
      case 16: launch_plane_t<16, true>(S, step, flags); return;
      case 32: launch_plane_t<32, true>(S, step, flags); return;
      case 64: launch_plane_t<64, true>(S, step, flags); return;
      default: throw Error(DR_ERR_UNSUPPORTED, "plane size not supported by the bulk-copy kernel");
    }
  }
  switch (v.E0) {
    case 4: launch_plane_t<4, false>(S, step, flags); break;
    case 8: launch_plane_t<8, false>(S, step, flags); break;
    case 16: launch_plane_t<16, false>(S, step, flags); break;
    case 32: launch_plane_t<32, false>(S, step, flags); break;
    case 64: launch_plane_t<64, false>(S, step, flags); break;
    case 128: launch_plane_t<128, false>(S, step, flags); break;
    default: throw Error(DR_ERR_UNSUPPORTED, "plane size not supported");
  }
}

// The gradient/leapfrog sequence for steps 0..L (see kernels.cu header).
static void enqueue_steps(Chainset* S, int L, int flags) {
  const DevVolume& v = S->vol->dv;
  const DevChains& ch = S->dc;
  const float2* tw = S->vol->tw_f;
  const int C = S->C;
  for (int s = 0; s <= L; s++) {
    const NvtxRange range(s == 0 ? "leapfrog step 0 (momentum, half kick, drift)"
                                 : (s == L ? "leapfrog last step (half kick, energies)" : "leapfrog step"));
    const int sel = s == 0 ? 0 : 1;
    if (s > 0) {
      if (!S->plane)
        launch_pass<float2>(v.E1, -1, PRO_LOAD, EPI_STORE,
                            pass_args(ch.T1, ch.T2, ch.t1_stride, ch.t2_stride, v.E2, v.bx, v.E1, v.by, 1.0, s), v, ch,
                            tw, C, S->stream);
      // forward z (pruned to the box), gather mu at data / output voxels
      launch_pass<float2>(v.E2, -1, PRO_LOAD, EPI_GATHER,
                          pass_args(ch.T2, nullptr, ch.t2_stride, 0, 1, v.by * v.bx, v.E2, v.bz,
                                    1.0 / (double)v.N, s, 1, 2),
                          v, ch, tw, C, S->stream);
    }
    if (v.n_s > 0) launch_spmv(S, s, sel, -1, true);
    launch_spmv(S, s, sel, -1, false);
    // inverse z from the box back to spectral z
    launch_pass<float2>(v.E2, +1, PRO_DATAGRAD, EPI_STORE,
                        pass_args(nullptr, ch.T2, 0, ch.t2_stride, 1, v.by * v.bx, v.bz, v.E2, 1.0, s), v, ch, tw, C,
                        S->stream);
    if (S->plane) {
      launch_plane(S, s, flags);
    } else {
      launch_pass<float2>(v.E1, +1, PRO_LOAD, EPI_STORE,
                          pass_args(ch.T2, ch.T1, ch.t2_stride, ch.t1_stride, v.E2, v.bx, v.by, v.E1, 1.0, s), v, ch,
                          tw, C, S->stream);
      launch_xline(S, s, flags);
    }
  }
}

static void enqueue_iteration(Chainset* S) {
  const DevVolume& v = S->vol->dv;
  k_iter_begin<<<cdiv_i(S->C, 128), 128, 0, S->stream>>>(S->dc);
  CK_LAUNCH();
  enqueue_steps(S, S->opts.leapfrog, 0);
  k_accept<<<S->C, 256, 0, S->stream>>>(v, S->dc);
  CK_LAUNCH();
  k_summary_max<<<S->C, 256, 0, S->stream>>>(v, S->dc);
  CK_LAUNCH();
  k_summary_acc<<<std::max(1, cdiv_i((long long)v.n_o * S->dc.Cp, 256)), 256, 0, S->stream>>>(v, S->dc);
  CK_LAUNCH();
}

static void init_chain_states(Chainset* S) {
  std::vector<ChainState> st(S->C);
  const dr_hmc_opts& o = S->opts;
  for (int c = 0; c < S->C; c++) {
    ChainState h;
    std::memset(&h, 0, sizeof(h));
    // HMCParameters<float> constructor (HMCParameters.h:97-149)
    h.warmup = o.burnin > 0;
    h.eps_start_found = !h.warmup;
    h.burnin = o.burnin;
    h.integrator_steps = o.leapfrog;
    h.iteration = 0;
    h.n_save = o.nsave;
    h.thin = o.thin == 0 ? 1 : o.thin;
    h.A = 1;
    h.eps0 = 1e-5;
    const float e0 = o.starting_eps > 0 ? o.starting_eps : (float)(1.0 / o.leapfrog);
    h.eps = std::max((double)e0, h.eps0);
    h.eps_bar = 1;
    h.gamma = (double)0.05f;
    h.h_bar = 0;
    h.mh_running_sum = 0;
    h.mh_target = (double)o.mhtarget;
    h.t0 = 10;
    h.kappa = (double)0.75f;
    h.acc = 0;
    h.L_cur = -1;
    h.done = o.nsave <= 0 ? 1 : 0;
    st[c] = h;
  }
  CK(cudaMemcpyAsync(S->dc.st, st.data(), sizeof(ChainState) * S->C, cudaMemcpyHostToDevice, S->stream));
  CK(cudaStreamSynchronize(S->stream));
}

// ---------------------------------------------------------------- autotuning
// Candidate update paths for an embedding: the fused plane kernel (square x/y
// planes whose padded layout fits shared memory), the same with bulk prefetch
// of the state planes, and the x-line kernel with separate y passes (always).
// ---------------------------------------------------------------- tensor-core kriging products
static void tc_upload(Volume* V, const TcPlanHost& P, const float* dval, int nnz, int n_rows, int n_cols,
                      DevTcMatrix* M) {
  cudaStream_t st = V->stream;
  M->n_rows = n_rows;
  M->n_cols = n_cols;
  M->T = P.T;
  M->G = P.G;
  M->n_segs = (int)(P.segs.size() / 4);
  M->chunks = (int)P.chunks;
  M->tile_rows = V->upload(P.tile_rows);
  M->chunk_cols = V->upload(P.chunk_cols);
  M->segs = reinterpret_cast<const int4*>(V->upload(P.segs));
  M->cta_seg_ptr = V->upload(P.cta_seg_ptr);
  M->tile_seg_ptr = V->upload(P.tile_seg_ptr);
  const size_t nblob = (size_t)P.chunks * TC_BLK;
  float* blob = V->alloc<float>(nblob);
  CK(cudaMemsetAsync(blob, 0, sizeof(float) * std::max<size_t>(nblob, 1), st));
  if (nnz > 0) {
    int* dest = nullptr;
    const cudaError_t e = dev_alloc((void**)&dest, sizeof(int) * nnz, st);
    if (e != cudaSuccess) throw Error(DR_ERR_NOMEM, "device allocation (tile positions)");
    CK(cudaMemcpyAsync(dest, P.dest.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
    k_tc_fill<<<cdiv_i(nnz, 256), 256, 0, st>>>(dval, dest, nnz, blob);
    CK_LAUNCH();
    CK(cudaFreeAsync(dest, st));
  }
  M->blob = blob;
}

// Builds the volume's dense tiles once; false when the tensor-core products are not available for it (no std-res
// data, a device without the shared memory, or tiles that would take more than a quarter of the free memory).
static bool volume_tc(Volume* V) {
  std::lock_guard<std::mutex> lk(V->tc_mtx);
  if (V->tc_state != 0) return V->tc_state > 0;
  V->tc_state = -1;
  const HostVolume& hv = V->hv;
  const DevVolume& dv = V->dv;
  const DeviceTables& dt = device_tables(V->device);
  if (!dt.tc || dv.n_s == 0 || hv.w_col.empty() || hv.wt_col.empty()) return false;
  const auto t0 = std::chrono::steady_clock::now();
  TraceScope tr("tensor-core tiles: row keys");
  CK(cudaSetDevice(V->device));
  auto coords = [&](int flat, int* x, int* y, int* z) {
    *x = flat % hv.E[0];
    *y = (flat / hv.E[0]) % hv.E[1];
    *z = flat / (hv.E[0] * hv.E[1]);
  };
  // W's rows are ordered by the centroid of the data voxels each std-res voxel is kriged from, W^T's by voxel
  std::vector<uint32_t> kw(dv.n_s, 0), kt(dv.n_h, 0);
#pragma omp parallel for schedule(static)
  for (int r = 0; r < dv.n_s; r++) {
    double sx = 0, sy = 0, sz = 0;
    const int n = hv.w_rowptr[r + 1] - hv.w_rowptr[r];
    for (int k = hv.w_rowptr[r]; k < hv.w_rowptr[r + 1]; k++) {
      int x, y, z;
      coords(hv.d_flat[hv.w_col[k]], &x, &y, &z);
      sx += x;
      sy += y;
      sz += z;
    }
    if (n > 0) kw[r] = zorder_key((int)std::lround(sx / n), (int)std::lround(sy / n), (int)std::lround(sz / n));
  }
#pragma omp parallel for schedule(static)
  for (int j = 0; j < dv.n_h; j++) {
    int x, y, z;
    coords(hv.d_flat[j], &x, &y, &z);
    kt[j] = zorder_key(x, y, z);
  }
  tr.next("tensor-core tiles: tile plans");
  TcPlanHost pw, pt;
  if (!tc_plan(hv.w_rowptr, hv.w_col.data(), hv.w_col.size(), kw, dt.sms, &pw) ||
      !tc_plan(hv.wt_rowptr, hv.wt_col.data(), hv.wt_col.size(), kt, dt.sms, &pt))
    return false;
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  const double blob_bytes = (double)(pw.chunks + pt.chunks) * TC_BLK * 4;
  if (blob_bytes > 0.25 * (double)fr) return false;
  tr.next("tensor-core tiles: blob build");
  tc_upload(V, pw, dv.w_val, (int)hv.w_col.size(), dv.n_s, dv.n_h, &V->tc_w);
  tc_upload(V, pt, dv.wt_val, (int)hv.wt_col.size(), dv.n_h, dv.n_s, &V->tc_wt);
  V->tc_max_segs = std::max(V->tc_w.n_segs, V->tc_wt.n_segs);
  CK(cudaStreamSynchronize(V->stream));
  V->tc_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  V->tc_state = 1;
  return true;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (null when the driver does not provide it).
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    cudaGetLastError();
  });
  return fn;
}

// A 2D map of a chain-minor array (rows of Cp floats) whose box is one row of N chains, for tile::gather4 row
// gathers; false when the driver cannot encode it (the products then gather with their threads).
static bool encode_row_map(CUtensorMap* m, const float* base, int Cp, long long rows, int N) {
  const PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
  if (!fn || rows <= 0 || rows > 0x7fffffffLL || (Cp * 4) % 16 != 0 || N > 256) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Cp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Cp * 4};
  const cuuint32_t box[2] = {(cuuint32_t)N, 1};
  const cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Chains per tensor-core product: the smallest power of two >= C and >= 16 (0 when C is outside [16, 256]).
static int tc_chains(int C) {
  if (C < 16 || C > 256) return 0;
  int n = 16;
  while (n < C) n *= 2;
  return n;
}

static bool tc_env_off() {
  const char* e = std::getenv("DRB_TC_PRODUCTS");
  return e && std::string(e) == "0";
}

struct PathOptions {
  bool plane = false, prefetch = false;
};
static PathOptions path_options(const DevVolume& v, int device) {
  PathOptions po;
  if (!(v.E0 == v.E1 && v.E0 >= 4 && v.E0 <= 128)) return po;
  const DeviceTables& dt = device_tables(device);
  const int elems = v.E0 == 64 ? PlaneGeom<64>::SIZE : (v.E0 == 128 ? PlaneGeom<128>::SIZE : v.E0 * (v.E0 + 1));
  po.plane = plane_layout(v.E0, elems, false).total <= dt.tma_dyn_max;
  po.prefetch = po.plane && v.E0 <= 64 && plane_layout(v.E0, elems, true).total <= dt.tma_dyn_max;
  return po;
}

struct TuneChoice {
  int ztile = 8;     // chains per z-pass tile (8 or 1) for chain sets of 8 or more chains
  int path = 0;      // 0 plane, 1 plane + prefetch, 2 x-line
  int grid = 8;      // kriging-product blocks per SM (CSR products)
  double ms = 0.0;   // measured milliseconds per iteration
  int tc = 0;        // 1: kriging products on the tensor cores
  int fftplan = 0;   // FP_* bits: transforms on the second radix plan (fft_smem PLAN 1) for 64, 128, 256 points
};

static bool autotune_enabled() {
  const char* e = std::getenv("DRB_AUTOTUNE");
  return !(e && std::string(e) == "0");
}

struct TuneKey {
  int dev, E0, E1, E2, bx, by, bz, C, n_h, n_s, L;  // n_h, n_s as tune_bucket()s
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, E0, E1, E2, bx, by, bz, C, n_h, n_s, L) <
           std::tie(o.dev, o.E0, o.E1, o.E2, o.bx, o.by, o.bz, o.C, o.n_h, o.n_s, o.L);
  }
};
static std::mutex g_tune_mtx;
static std::map<TuneKey, TuneChoice> g_tune;

static void chainset_build(Chainset* S, Volume* V, int C, const dr_hmc_opts* o, const TuneChoice* forced = nullptr);
static void launch_iterations(Chainset* S, int iters);
static void read_states(Chainset* S, std::vector<ChainState>* st);
static void write_states(Chainset* S, const std::vector<ChainState>& st);


// Quarter-octave bucket of a voxel count: volumes of one shape whose data counts differ by less than about 19 %
// share a tuning result (it chooses a speed, not a result), so a stream of similar jobs tunes once.
static int tune_bucket(int n) { return n <= 0 ? -1 : (int)std::lround(4.0 * std::log2((double)n)); }

// Tunes in two rounds on scratch chain sets of the same shape, each candidate
// timed for one iteration after one untimed, forced past the step-size search
// (so that all of their leapfrog steps run, at most 6 of them): first the update paths, with
// the tensor-core products where the volume and chain count allow them (else
// CSR products at 8 blocks per SM); then, on the fastest path, the other
// product choices (CSR at 8 blocks/SM, and at 4 and 2 for chain sets of fewer
// than 32 chains) and the z-pass tile shape.  The fastest candidate is kept
// and cached per shape.
static TuneChoice autotune(Volume* V, int C, const dr_hmc_opts* o) {
  const NvtxRange range("chain set: tuning");
  const DevVolume& v = V->dv;
  const TuneKey key{V->device, v.E0, v.E1, v.E2, v.bx, v.by, v.bz, C, tune_bucket(v.n_h), tune_bucket(v.n_s),
                    o->leapfrog};
  {
    std::lock_guard<std::mutex> lk(g_tune_mtx);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  const PathOptions po = path_options(v, V->device);
  const bool tc = tc_chains(C) > 0 && !tc_env_off() && volume_tc(V);
  TuneChoice best;
  best.ms = 1e300;
  dr_hmc_opts to = *o;
  to.store_samples = 0;
  // candidates are timed on iterations of at most TUNE_STEPS leapfrog steps: every step runs the same kernels, so
  // the ranking holds, and a candidate costs a quarter of a full iteration at L = 25; the time kept for the choice
  // is scaled to the full L (steps + 1 gradient evaluations per iteration)
  constexpr int TUNE_STEPS = 6;
  to.leapfrog = std::min(o->leapfrog, TUNE_STEPS);
  const double to_full = (double)(o->leapfrog + 1) / (double)(to.leapfrog + 1);
  auto try_candidate = [&](TuneChoice c) {
    // a candidate that cannot be built or run (for instance out of device memory beside the caller's other
    // allocations) is skipped; if none can, the default configuration is used untuned
    const TraceScope tr("tuning candidate path " + std::to_string(c.path) + " tc " + std::to_string(c.tc) +
                        " grid " + std::to_string(c.grid) + " ztile " + std::to_string(c.ztile) + " fft plan " +
                        std::to_string(c.fftplan));
    try {
      auto T = std::make_unique<Chainset>();
      chainset_build(T.get(), V, C, &to, &c);
      std::vector<ChainState> st;
      read_states(T.get(), &st);
      for (auto& h : st) {
        h.eps_start_found = 1;  // integrator_steps() = L from the first iteration
        h.warmup = 1;
      }
      write_states(T.get(), st);
      launch_iterations(T.get(), 1);
      cudaEvent_t e0, e1;
      CK(cudaEventCreate(&e0));
      CK(cudaEventCreate(&e1));
      CK(cudaEventRecord(e0, T->stream));
      launch_iterations(T.get(), 1);
      CK(cudaEventRecord(e1, T->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      c.ms = ms * to_full;
      if (trace_on()) std::fprintf(stderr, "[drb]   measured %.3f ms per iteration (scaled to L)\n", c.ms);
      if (c.ms < best.ms) best = c;
    } catch (const Error&) {
      cudaGetLastError();
    }
  };
  for (int path : {0, 1, 2}) {
    if ((path == 0 && !po.plane) || (path == 1 && !po.prefetch)) continue;
    try_candidate(TuneChoice{8, path, 8, 0.0, tc ? 1 : 0});
  }
  if (best.ms < 1e300) {
    const int path = best.path;
    if (tc) try_candidate(TuneChoice{8, path, 8, 0.0, 0});
    // narrower chain sets may do better with fewer, longer-lived CSR product blocks
    if (C < 32)
      for (int grid : {4, 2}) try_candidate(TuneChoice{8, path, grid, 0.0, 0});
    // the z passes' tile shape on the best configuration: 32 lines of one chain instead of 4 lines x 8 chains
    if (C >= 8) {
      TuneChoice t = best;
      t.ztile = 1;
      try_candidate(t);
    }
    // the second radix plan, one transform at a time on the best configuration so far: the inverse and the forward
    // z passes, and the x transforms of the x-line kernel, where their length has two plans
    auto two_plans = [](int n) { return n == 64 || n == 128 || n == 256; };
    for (int bit : {(int)FP_ZINV, (int)FP_ZFWD, (int)FP_XLINE}) {
      if (bit == FP_XLINE ? !(best.path == 2 && two_plans(v.E0)) : !two_plans(v.E2)) continue;
      TuneChoice t = best;
      t.fftplan |= bit;
      try_candidate(t);
    }
  }
  if (!(best.ms < 1e300)) {  // nothing could be timed: default, not cached
    TuneChoice d;
    d.path = po.plane ? 0 : 2;
    return d;
  }
  std::lock_guard<std::mutex> lk(g_tune_mtx);
  g_tune[key] = best;
  return best;
}

static void chainset_build(Chainset* S, Volume* V, int C, const dr_hmc_opts* o, const TuneChoice* forced) {
  if (C <= 0 || C > 256) throw Error(DR_ERR_UNSUPPORTED, "n_chains must be in [1, 256]");
  if (!o) throw Error(DR_ERR_INVALID, "opts is NULL");
  if (o->burnin < 0) throw Error(DR_ERR_DOMAIN, "HMCParameters: burnin must be >= 0");
  if (o->nsave < 0) throw Error(DR_ERR_DOMAIN, "HMCParameters: n_save must be >= 0");
  if (o->thin < 0) throw Error(DR_ERR_DOMAIN, "HMCParameters: thin must be >= 0");
  if (o->leapfrog <= 0) throw Error(DR_ERR_DOMAIN, "HMCParameters: integrator_steps must be > 0");
  if (!(o->mhtarget > 0 && o->mhtarget < 1)) throw Error(DR_ERR_DOMAIN, "HMCParameters: mh_target should be within (0, 1)");
  {
    std::lock_guard<std::mutex> lk(g_vol_mtx);
    S->vol = V;
    V->n_chainsets++;
  }
  const TraceScope tr("chain set: build (" + std::to_string(C) + " chains" + (forced ? ", tuning candidate)" : ")"));
  S->device = V->device;
  S->C = C;
  S->opts = *o;
  CK(cudaSetDevice(V->device));
  CK(cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking));
  const DevVolume& v = V->dv;
  DevChains& ch = S->dc;
  ch.C = C;
  ch.Cp = C;
  int cg = 1;
  while (cg < C && cg < 32) cg <<= 1;
  ch.CG = cg;
  S->NR = cdiv_i(C, cg);
  if (S->NR > 8) throw Error(DR_ERR_UNSUPPORTED, "too many chains");
  if (S->NR == 3) S->NR = 4;
  if (S->NR > 4 && S->NR < 8) S->NR = 8;
  const long long N = v.N;
  const PathOptions po = path_options(v, V->device);
  int path = po.plane ? 0 : 2, grid = 8;
  // tensor-core products by default for 32 or more chains; the tuner, DRB_TC_PRODUCTS=0 / 1 and a forced choice
  // override the default
  int tc = C >= 32 ? 1 : 0;
  if (const char* e = std::getenv("DRB_TC_PRODUCTS")) tc = std::atoi(e) != 0;
  int ztile = 8;
  if (const char* e = std::getenv("DRB_ZTILE")) ztile = std::atoi(e) == 1 ? 1 : 8;
  int fftplan = 0;
  if (const char* e = std::getenv("DRB_FFT_PLAN")) fftplan = std::atoi(e) & (FP_ZINV | FP_ZFWD | FP_XLINE);
  if (forced) {
    path = forced->path;
    grid = forced->grid;
    tc = forced->tc;
    ztile = forced->ztile;
    fftplan = forced->fftplan;
  } else if (std::getenv("DRB_NO_PLANE")) {
    path = 2;
  } else if (std::getenv("DRB_PLANE_PREFETCH")) {
    path = po.prefetch ? 1 : path;
  } else if (autotune_enabled()) {
    const TuneChoice t = autotune(V, C, o);
    path = t.path;
    grid = t.grid;
    if (!std::getenv("DRB_ZTILE")) ztile = t.ztile;
    if (!std::getenv("DRB_FFT_PLAN")) fftplan = t.fftplan;
    if (!std::getenv("DRB_TC_PRODUCTS")) tc = t.tc;
    S->tuned_ms = t.ms;
  }
  if (!forced) {
    if (const char* g = std::getenv("DRB_PRODUCT_BLOCKS_PER_SM")) grid = std::max(1, std::min(16, std::atoi(g)));
  }
  if ((path == 0 && !po.plane) || (path == 1 && !po.prefetch)) path = po.plane ? 0 : 2;
  // the state arrays are allocated after the tuning, whose candidate chain sets then reuse the pool's memory
  // without this chain set's arrays held beside them
  ch.U = S->alloc<float2>((size_t)C * 2 * N);
  ch.Q = S->alloc<float2>((size_t)C * N);
  S->path = path;
  S->grid = grid;
  S->plane = path != 2;
  S->tma = path == 1;
  ch.t2_stride = (long long)v.E2 * v.by * v.bx;
  if (S->plane) {
    // T1 is only needed by the initial transforms: borrow the momentum buffer
    ch.t1_stride = N;
    ch.T1 = ch.Q;
  } else {
    ch.t1_stride = (long long)v.E2 * v.E1 * v.bx;
    ch.T1 = S->alloc<float2>((size_t)C * ch.t1_stride);
  }
  ch.T2 = S->alloc<float2>((size_t)C * ch.t2_stride);
  ch.muD = S->alloc<float>((size_t)2 * v.n_h * C);
  ch.muO = S->alloc<float>((size_t)2 * std::max(v.n_o, 1) * C);
  ch.gD = S->alloc<float>((size_t)v.n_h * C);
  ch.rs = S->alloc<float>((size_t)std::max(v.n_s, 1) * C);
  ch.nb_x = S->plane ? v.E2 : cdiv_i((long long)v.E1 * v.E2, TILE_LINES);
  const int wide = device_tables(V->device).sms * S->grid;
  ch.nb_w = std::max(1, std::min(v.n_s, wide));
  ch.nb_wt = std::max(1, std::min(cdiv_i(v.n_h, 8), wide));
  S->tcp = tc && tc_chains(C) > 0 && volume_tc(V);
  if (S->tcp) {
    S->tc_N = tc_chains(C);
    ch.nb_w = tc_finish_blocks(V->tc_w.T);
    ch.nb_wt = tc_finish_blocks(V->tc_wt.T);
    S->tc_partial = S->alloc<float>((size_t)std::max(V->tc_max_segs, 1) * S->tc_N * TC_M, false);
    const char* tg = std::getenv("DRB_TC_TMA_GATHER");
    S->tc_tg = !(tg && std::string(tg) == "0") && encode_row_map(&S->tc_map_wt, ch.rs, ch.Cp, (long long)v.n_s, S->tc_N);
  }
  ch.maxblk = std::max(ch.nb_x, std::max(ch.nb_w, ch.nb_wt));
  ch.part = S->alloc<double>((size_t)C * NSLOT * ch.maxblk);
  ch.st = S->alloc<ChainState>(C);
  ch.s1 = S->alloc<double>((size_t)std::max(v.n_o, 1) * C);
  ch.s2 = S->alloc<double>((size_t)std::max(v.n_o, 1) * C);
  ch.sa = S->alloc<double>((size_t)std::max(v.n_o, 1) * C);
  ch.samples = o->store_samples ? S->alloc<float>((size_t)std::max(o->nsave, 1) * std::max(v.n_o, 1) * C, false) : nullptr;
  ch.save_rec = o->store_samples ? S->alloc<double>((size_t)std::max(o->nsave, 1) * C * 3, true) : nullptr;
  ch.seed = o->seed;
  ch.chain0 = 0;
  ch.ztile = ztile;
  ch.fftplan = fftplan;
  ch.err = S->alloc<int>(1);
  S->tmp = S->alloc<float2>(N);
  init_chain_states(S);

  // initial state: sigma, then u0 = IFFT(scatter(Yh)) + sqrt(N lambda) w / 10, then mu at data/output voxels
  const float2* tw = V->tw_f;
  cudaStream_t s = S->stream;
  k_init_sigma<<<cdiv_i(C, 128), 128, 0, s>>>(ch, V->hv.theta[0] > 0 ? (float)V->hv.theta[0] : 1.0f, v.n_s > 0 ? 2 : 1);
  CK_LAUNCH();
  k_fill_gD<<<std::max(1, cdiv_i((long long)v.n_h * C, 256)), 256, 0, s>>>(v, ch);
  CK_LAUNCH();
  launch_pass<float2>(v.E2, +1, PRO_DATAGRAD, EPI_STORE, pass_args(nullptr, ch.T2, 0, ch.t2_stride, 1, v.by * v.bx, v.bz, v.E2), v, ch, tw, C, s);
  launch_pass<float2>(v.E1, +1, PRO_LOAD, EPI_STORE, pass_args(ch.T2, ch.T1, ch.t2_stride, ch.t1_stride, v.E2, v.bx, v.by, v.E1), v, ch, tw, C, s);
  launch_pass<float2>(v.E0, +1, PRO_LOAD, EPI_STORE, pass_args(ch.T1, ch.U, ch.t1_stride, 2 * N, v.E2 * v.E1, 1, v.bx, v.E0), v, ch, tw, C, s);
  k_init_prior<<<dim3(std::max(1, cdiv_i(N / 2, 256)), C), 256, 0, s>>>(v, ch);
  CK_LAUNCH();
  launch_pass<float2>(v.E0, -1, PRO_LOAD, EPI_STORE, pass_args(ch.U, ch.T1, 2 * N, ch.t1_stride, v.E2 * v.E1, 1, v.E0, v.bx), v, ch, tw, C, s);
  launch_pass<float2>(v.E1, -1, PRO_LOAD, EPI_STORE, pass_args(ch.T1, ch.T2, ch.t1_stride, ch.t2_stride, v.E2, v.bx, v.E1, v.by), v, ch, tw, C, s);
  launch_pass<float2>(v.E2, -1, PRO_LOAD, EPI_GATHER, pass_args(ch.T2, nullptr, ch.t2_stride, 0, 1, v.by * v.bx, v.E2, v.bz, 1.0 / (double)N, -1, 0, 1), v, ch, tw, C, s);
  CK(cudaStreamSynchronize(s));
}

static void read_states(Chainset* S, std::vector<ChainState>* st) {
  st->resize(S->C);
  CK(cudaMemcpyAsync(st->data(), S->dc.st, sizeof(ChainState) * S->C, cudaMemcpyDeviceToHost, S->stream));
  CK(cudaStreamSynchronize(S->stream));
}
static void write_states(Chainset* S, const std::vector<ChainState>& st) {
  CK(cudaMemcpyAsync(S->dc.st, st.data(), sizeof(ChainState) * S->C, cudaMemcpyHostToDevice, S->stream));
  CK(cudaStreamSynchronize(S->stream));
}

static void ensure_graph(Chainset* S) {
  if (S->graph) return;
  cudaGraph_t g = nullptr;
  const int64_t before = g_launches;
  CK(cudaStreamBeginCapture(S->stream, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue_iteration(S);
  } catch (...) {
    cudaStreamEndCapture(S->stream, &g);
    if (g) cudaGraphDestroy(g);
    g_launches = before;
    throw;
  }
  CK(cudaStreamEndCapture(S->stream, &g));
  S->graph_nodes = g_launches - before;
  g_launches = before;
  const cudaError_t e = cudaGraphInstantiate(&S->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error(DR_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
}

// Enqueues `iters` iterations without waiting (the server's round).
static void launch_iterations(Chainset* S, int iters) {
  ensure_graph(S);
  for (int i = 0; i < iters; i++) {
    const NvtxRange range("HMC iteration (graph)");
    CK(cudaGraphLaunch(S->graph, S->stream));
    g_launches += S->graph_nodes;
  }
  if (!S->done_event) CK(cudaEventCreateWithFlags(&S->done_event, cudaEventDisableTiming));
  CK(cudaEventRecord(S->done_event, S->stream));
}

static void check_device_error(Chainset* S) {
  int err = 0;
  CK(cudaMemcpyAsync(&err, S->dc.err, sizeof(int), cudaMemcpyDeviceToHost, S->stream));
  CK(cudaStreamSynchronize(S->stream));
  if (err == ERR_BOUNDS) throw Error(DR_ERR_STATE, "a bounds check failed: an index left its array (checked build)");
  if (err == 3) throw Error(DR_ERR_TIMEOUT, "a bounded device wait gave up (tensor-core kriging product pipeline)");
  if (err) throw Error(DR_ERR_TIMEOUT, "a bounded device wait gave up (bulk copy did not complete)");
}

static void step(Chainset* S, int iters, double* device_ms = nullptr) {
  CK(cudaSetDevice(S->vol->device));
  ensure_graph(S);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (device_ms) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, S->stream));
  }
  for (int i = 0; i < iters; i++) {
    const NvtxRange range("HMC iteration (graph)");
    CK(cudaGraphLaunch(S->graph, S->stream));
    g_launches += S->graph_nodes;
  }
  if (device_ms) CK(cudaEventRecord(e1, S->stream));
  CK(cudaStreamSynchronize(S->stream));
  if (device_ms) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  check_device_error(S);
}

// Posterior summary of mcmc_summary<T> (gaussian_process_model.h:191-316) over
// chain `chain`, or pooled over all chains when chain = -1.
static void summary_of(Chainset* s, int chain, float* mean, float* var, float* activation) {
  const DevVolume& v = s->vol->dv;
  const size_t n = (size_t)v.n_o * s->C;
  std::vector<double> s1(n), s2(n), sa(n);
  CK(cudaSetDevice(s->vol->device));
  CK(cudaMemcpyAsync(s1.data(), s->dc.s1, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(s2.data(), s->dc.s2, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(sa.data(), s->dc.sa, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
  std::vector<ChainState> st;
  read_states(s, &st);
  const int c0 = chain < 0 ? 0 : chain, c1 = chain < 0 ? s->C : chain + 1;
  double ns = 0.0;
  for (int c = c0; c < c1; c++) ns += st[c].saved;
  if (ns <= 0) ns = 1;  // mcmc_summary::samples() (gaussian_process_model.h:255-258)
  std::vector<double> act(v.n_o);
  double amax = -1e300;
  for (int o = 0; o < v.n_o; o++) {
    double a1 = 0, a2 = 0, aa = 0;
    for (int c = c0; c < c1; c++) {
      a1 += s1[(size_t)o * s->C + c];
      a2 += s2[(size_t)o * s->C + c];
      aa += sa[(size_t)o * s->C + c];
    }
    const double m = a1 / ns, vr = (a2 - a1 * a1 / ns) / ns;
    if (mean) mean[o] = (float)m;
    if (var) var[o] = (float)vr;
    act[o] = aa / (ns * std::sqrt(vr));
    amax = std::max(amax, act[o]);
  }
  if (activation)
    for (int o = 0; o < v.n_o; o++) activation[o] = (float)(act[o] / amax);
}

// Spectral state of chain c from a real-space field (host, 2N floats).
static void upload_field(Chainset* S, const float* mu) {
  CK(cudaMemcpyAsync(S->tmp, mu, sizeof(float2) * S->vol->dv.N, cudaMemcpyHostToDevice, S->stream));
}

static void gather_data(Chainset* S, const float2* field, int c, int half, bool with_output) {
  const DevVolume& v = S->vol->dv;
  k_gather_re<<<cdiv_i(v.n_h, 256), 256, 0, S->stream>>>(field, v.d_flat, v.n_h, S->dc.muD + (long long)half * v.n_h * S->C, S->C, c, v.N, S->dc.err);
  CK_LAUNCH();
  if (with_output && v.n_o > 0) {
    k_gather_re<<<cdiv_i(v.n_o, 256), 256, 0, S->stream>>>(field, v.o_flat, v.n_o, S->dc.muO + (long long)half * v.n_o * S->C, S->C, c, v.N, S->dc.err);
    CK_LAUNCH();
  }
}

static double part_sum(Chainset* S, int c, int slot, int nb) {
  std::vector<double> h(nb);
  CK(cudaMemcpyAsync(h.data(), S->dc.part + ((long long)c * NSLOT + slot) * S->dc.maxblk, sizeof(double) * nb,
                     cudaMemcpyDeviceToHost, S->stream));
  CK(cudaStreamSynchronize(S->stream));
  double s = 0.0;
  for (double x : h) s += x;
  return s;
}

// Log prior, log likelihood (lpll[0..1]) and gradient (grad, 2N floats) at mu through the sampler's own kernels:
// step 0 of the leapfrog sequence (kriging products on the chain set's path, the inverse z pass, then the plane or
// x-line kernel) from a zero momentum, with eps = 2 so that the half kick is exactly 1 and no drift, because the
// step is both the first and the last.  The momentum it leaves is q = IFFT(gradient) in the spectral basis, and
// its step-0 partial sums are the energies at mu.  It works in the proposal half of the chain's buffers and in the
// momentum, which hold nothing between iterations, so the chain's state is unchanged.
static void eval_sampler(Chainset* S, int chain, const float* mu, double* lpll, float* grad) {
  const NvtxRange range("evaluation (sampler step 0)");
  CK(cudaSetDevice(S->vol->device));
  const DevVolume& v = S->vol->dv;
  std::vector<ChainState> st, saved;
  read_states(S, &st);
  saved = st;
  const int half = st[chain].acc ^ 1;
  DevChains none{};
  upload_field(S, mu);
  gather_data(S, S->tmp, chain, half, false);
  fft3d<float2>(S->tmp, S->vol->hv.E, +1, 0, 1, S->vol->tw_f, S->stream, v, none);
  CK(cudaMemcpyAsync(S->dc.U + ((long long)chain * 2 + half) * v.N, S->tmp, sizeof(float2) * v.N,
                     cudaMemcpyDeviceToDevice, S->stream));
  CK(cudaMemsetAsync(S->dc.Q + (long long)chain * v.N, 0, sizeof(float2) * v.N, S->stream));
  for (int c = 0; c < S->C; c++) st[c].L_cur = -1;
  st[chain].L_cur = 0;
  st[chain].eps_cur = 2.0f;
  st[chain].acc = half;
  write_states(S, st);
  try {
    enqueue_steps(S, 0, XF_FIXED_MOMENTUM | XF_WRITE_Q_LAST);
    if (lpll) {
      const double lp = part_sum(S, chain, SL_LP0, S->dc.nb_x);
      const double Rh = part_sum(S, chain, SL_RH0, S->dc.nb_wt);
      const double Rs = v.n_s > 0 ? part_sum(S, chain, SL_RS0, S->dc.nb_w) : 0.0;
      lpll[0] = -0.5 * lp / (double)v.N;
      lpll[1] = -0.5 * ((double)st[chain].sh * Rh + (v.n_s > 0 ? (double)st[chain].ss * Rs : 0.0));
    }
    if (grad) {
      CK(cudaMemcpyAsync(S->tmp, S->dc.Q + (long long)chain * v.N, sizeof(float2) * v.N, cudaMemcpyDeviceToDevice,
                         S->stream));
      fft3d<float2>(S->tmp, S->vol->hv.E, -1, 0, 1, S->vol->tw_f, S->stream, v, none);
      k_scale<<<cdiv_i(v.N, 256), 256, 0, S->stream>>>(S->tmp, v.N, 1.0f / (float)v.N);
      CK_LAUNCH();
      CK(cudaMemcpyAsync(grad, S->tmp, sizeof(float2) * v.N, cudaMemcpyDeviceToHost, S->stream));
    }
    CK(cudaStreamSynchronize(S->stream));
  } catch (...) {
    cudaStreamSynchronize(S->stream);
    write_states(S, saved);
    throw;
  }
  write_states(S, saved);
  check_device_error(S);
}

}  // namespace drb

// ==================================================================== C ABI
using namespace drb;

struct dr_volume : Volume {};
struct dr_chainset : Chainset {};

#define API_BEGIN try {
#define API_END                                                     \
  }                                                                 \
  catch (const Error& e) {                                          \
    g_err = e.what();                                               \
    return e.code;                                                  \
  }                                                                 \
  catch (const std::bad_alloc&) {                                   \
    g_err = "host allocation failed";                               \
    return DR_ERR_NOMEM;                                            \
  }                                                                 \
  catch (const std::exception& e) {                                 \
    g_err = e.what();                                               \
    return DR_ERR_INVALID;                                          \
  }                                                                 \
  return DR_OK;

// Calls another entry point and rethrows its failure with its message.
#define CK_API(call)                                   \
  do {                                                 \
    const int rc_ = (call);                            \
    if (rc_ != DR_OK) throw Error(rc_, std::string(g_err)); \
  } while (0)

extern "C" {

const char* dr_last_error(void) { return g_err.c_str(); }
#ifdef DRB_BOUNDS_CHECK
const char* dr_version(void) { return "dualres_b200 0.1 (sm_100a, bounds-checked)"; }
#else
const char* dr_version(void) { return "dualres_b200 0.1 (sm_100a)"; }
#endif
int64_t dr_kernel_launches(int reset) {
  const int64_t n = g_launches;
  if (reset) g_launches = 0;
  return n;
}

int dr_volume_create(const dr_volume_desc* desc, dr_volume** out) {
  API_BEGIN
  if (!desc || !out) throw Error(DR_ERR_INVALID, "NULL argument");
  *out = nullptr;
  dr_volume* v = new dr_volume();
  try {
    volume_build(v, desc);
  } catch (...) {
    delete v;
    throw;
  }
  *out = v;
  API_END
}

int dr_volume_info_get(const dr_volume* v, dr_volume_info* info) {
  API_BEGIN
  if (!v || !info) throw Error(DR_ERR_INVALID, "NULL argument");
  std::memset(info, 0, sizeof(*info));
  for (int k = 0; k < 3; k++) { info->E[k] = v->hv.E[k]; info->box[k] = v->hv.box[k]; }
  info->N = v->hv.N;
  info->n_highres = v->dv.n_h;
  info->n_stdres = v->dv.n_s;
  info->n_output = v->dv.n_o;
  info->kriging_nnz = (int64_t)v->hv.w_col.size();
  info->n_nonpositive = v->n_S;
  info->kriging_plan_seconds = v->hv.kriging_plan_seconds;
  info->kriging_solve_seconds = v->hv.kriging_solve_seconds;
  info->kriging_device_rows = v->hv.kriging_device_rows;
  info->kriging_host_rows = v->hv.kriging_host_rows;
  info->max_eigenvalue = v->max_eig;
  info->setup_seconds = v->setup_seconds;
  info->kriging_seconds = v->hv.kriging_seconds;
  info->neighborhood = v->hv.radius;
  info->device_bytes = v->bytes;
  API_END
}

int dr_volume_kriging_get(const dr_volume* v, int* rowptr, int* col, float* val) {
  API_BEGIN
  if (!v) throw Error(DR_ERR_INVALID, "NULL volume");
  if (rowptr && !v->hv.w_rowptr.empty()) std::memcpy(rowptr, v->hv.w_rowptr.data(), sizeof(int) * v->hv.w_rowptr.size());
  if (col && !v->hv.w_col.empty()) std::memcpy(col, v->hv.w_col.data(), sizeof(int) * v->hv.w_col.size());
  if (val && !v->hv.w_val.empty()) std::memcpy(val, v->hv.w_val.data(), sizeof(float) * v->hv.w_val.size());
  API_END
}

int dr_volume_lambda_get(const dr_volume* v, double* lam) {
  API_BEGIN
  if (!v || !lam) throw Error(DR_ERR_INVALID, "NULL argument");
  CK(cudaSetDevice(v->device));
  CK(cudaMemcpy(lam, v->lam_re, sizeof(double) * v->hv.N, cudaMemcpyDeviceToHost));
  API_END
}

int dr_volume_indices_get(const dr_volume* v, int* data_idx, int* out_idx) {
  API_BEGIN
  if (!v) throw Error(DR_ERR_INVALID, "NULL volume");
  if (data_idx) std::memcpy(data_idx, v->hv.d_flat.data(), sizeof(int) * v->hv.d_flat.size());
  if (out_idx && !v->hv.o_flat.empty()) std::memcpy(out_idx, v->hv.o_flat.data(), sizeof(int) * v->hv.o_flat.size());
  API_END
}

int dr_volume_data_get(const dr_volume* v, float* Yh, float* Ys) {
  API_BEGIN
  if (!v) throw Error(DR_ERR_INVALID, "NULL volume");
  if (Yh) std::memcpy(Yh, v->hv.Yh.data(), sizeof(float) * v->hv.Yh.size());
  if (Ys && !v->hv.Ys.empty()) std::memcpy(Ys, v->hv.Ys.data(), sizeof(float) * v->hv.Ys.size());
  API_END
}

void dr_volume_destroy(dr_volume* v) { volume_release(v); }

int dr_chainset_create(dr_volume* v, int n_chains, const dr_hmc_opts* opts, dr_chainset** out) {
  API_BEGIN
  if (!v || !out) throw Error(DR_ERR_INVALID, "NULL argument");
  *out = nullptr;
  dr_chainset* s = new dr_chainset();
  try {
    chainset_build(s, v, n_chains, opts);
  } catch (...) {
    delete s;
    throw;
  }
  *out = s;
  API_END
}

void dr_chainset_destroy(dr_chainset* s) { delete s; }

int dr_chainset_config_get(const dr_chainset* s, int* path, int* blocks_per_sm, double* tuned_ms,
                           int* tensor_products) {
  API_BEGIN
  if (!s) throw Error(DR_ERR_INVALID, "NULL chain set");
  if (path) *path = s->path;
  if (blocks_per_sm) *blocks_per_sm = s->grid;
  if (tuned_ms) *tuned_ms = s->tuned_ms;
  if (tensor_products) *tensor_products = s->tcp ? (s->tc_tg ? 2 : 1) : 0;
  API_END
}

int dr_chainset_ztile_get(const dr_chainset* s, int* z_tile_chains) {
  API_BEGIN
  if (!s || !z_tile_chains) throw Error(DR_ERR_INVALID, "NULL argument");
  *z_tile_chains = s->C >= 8 && s->dc.ztile != 1 ? 8 : 1;
  API_END
}

int dr_chainset_fft_plan_get(const dr_chainset* s, int* plan) {
  API_BEGIN
  if (!s || !plan) throw Error(DR_ERR_INVALID, "NULL argument");
  *plan = s->dc.fftplan;
  API_END
}

int dr_step(dr_chainset* s, int iterations) {
  API_BEGIN
  if (!s || iterations < 0) throw Error(DR_ERR_INVALID, "bad argument");
  step(s, iterations);
  API_END
}

int dr_step_timed(dr_chainset* s, int iterations, double* device_ms) {
  API_BEGIN
  if (!s || iterations < 0 || !device_ms) throw Error(DR_ERR_INVALID, "bad argument");
  step(s, iterations, device_ms);
  API_END
}

int dr_run(dr_chainset* s) {
  API_BEGIN
  if (!s) throw Error(DR_ERR_INVALID, "NULL chainset");
  std::vector<ChainState> st;
  read_states(s, &st);
  const int total = s->opts.burnin + (s->opts.thin == 0 ? 1 : s->opts.thin) * s->opts.nsave;
  int it = 0;
  for (const auto& h : st) it = std::max(it, h.iteration);
  if (total > it) step(s, total - it);
  API_END
}

int dr_chain_stats_get(dr_chainset* s, dr_chain_stats* out) {
  API_BEGIN
  if (!s || !out) throw Error(DR_ERR_INVALID, "NULL argument");
  std::vector<ChainState> st;
  read_states(s, &st);
  for (int c = 0; c < s->C; c++) {
    const ChainState& h = st[c];
    dr_chain_stats& o = out[c];
    o.iteration = h.iteration;
    o.saved = h.saved;
    o.integrator_steps = h.eps_start_found ? h.integrator_steps : 1;
    o.eps = (float)h.eps;
    const int d = h.iteration - h.burnin;
    o.mh_rate = (float)(h.mh_running_sum / std::max(d, 1));
    o.sigma_hr = std::sqrt(1.0f / h.sh);
    o.sigma_sr = std::sqrt(1.0f / h.ss);
    o.last_log_ratio = h.last_log_ratio;
    o.accepted = h.accepted;
    o.grad_evals = h.grad_evals;
    o.done = h.done;
    o.last_eps = h.eps_cur;
    o.initial_energy = h.last_E0;
    o.proposed_energy = h.last_Ep;
  }
  API_END
}

int dr_summary_get(dr_chainset* s, int chain, float* mean, float* var, float* activation) {
  API_BEGIN
  if (!s || chain < -1 || chain >= s->C) throw Error(DR_ERR_INVALID, "bad chain");
  summary_of(s, chain, mean, var, activation);
  API_END
}

int dr_samples_get(dr_chainset* s, int chain, float* samples, int max_saved, int* n_saved) {
  API_BEGIN
  if (!s || chain < 0 || chain >= s->C || !n_saved) throw Error(DR_ERR_INVALID, "bad argument");
  if (!s->dc.samples) throw Error(DR_ERR_STATE, "samples were not stored (store_samples = 0)");
  std::vector<ChainState> st;
  read_states(s, &st);
  const int ns = std::min(st[chain].saved, max_saved);
  *n_saved = ns;
  const DevVolume& v = s->vol->dv;
  const size_t per = (size_t)v.n_o * s->C;
  std::vector<float> buf(per);
  for (int i = 0; i < ns; i++) {
    CK(cudaMemcpy(buf.data(), s->dc.samples + i * per, sizeof(float) * per, cudaMemcpyDeviceToHost));
    for (int o = 0; o < v.n_o; o++) samples[(size_t)i * v.n_o + o] = buf[(size_t)o * s->C + chain];
  }
  API_END
}

int dr_sample_records_get(dr_chainset* s, int chain, double* rec, int max_saved, int* n_saved) {
  API_BEGIN
  if (!s || !rec || chain < 0 || chain >= s->C || !n_saved) throw Error(DR_ERR_INVALID, "bad argument");
  if (!s->dc.save_rec) throw Error(DR_ERR_STATE, "samples were not stored (store_samples = 0)");
  std::vector<ChainState> st;
  read_states(s, &st);
  const int ns = std::min(std::min(st[chain].saved, max_saved), std::max(s->opts.nsave, 1));
  *n_saved = ns;
  std::vector<double> buf((size_t)std::max(ns, 1) * s->C * 3);
  if (ns > 0) CK(cudaMemcpy(buf.data(), s->dc.save_rec, sizeof(double) * ns * s->C * 3, cudaMemcpyDeviceToHost));
  for (int i = 0; i < ns; i++)
    for (int k = 0; k < 3; k++) rec[(size_t)i * 3 + k] = buf[((size_t)i * s->C + chain) * 3 + k];
  API_END
}

int dr_set_state(dr_chainset* s, int chain, const float* mu, float s_hr, float s_sr) {
  API_BEGIN
  if (!s || !mu || chain < 0 || chain >= s->C) throw Error(DR_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(s->vol->device));
  std::vector<ChainState> st;
  read_states(s, &st);
  const DevVolume& v = s->vol->dv;
  const int acc = st[chain].acc;
  upload_field(s, mu);
  gather_data(s, s->tmp, chain, acc, true);
  DevChains none{};
  fft3d<float2>(s->tmp, s->vol->hv.E, +1, 0, 1, s->vol->tw_f, s->stream, v, none);
  CK(cudaMemcpyAsync(s->dc.U + ((long long)chain * 2 + acc) * v.N, s->tmp, sizeof(float2) * v.N,
                     cudaMemcpyDeviceToDevice, s->stream));
  st[chain].sh = s_hr;
  st[chain].ss = s_sr;
  write_states(s, st);
  API_END
}

// Checkpoint layout: a header of eight int64 {magic, version, C, N, n_h, n_o, Cp, nsave_stored}, then per chain the
// accepted spectral state (N float2), mu_D [2][n_h][Cp] and mu_O [2][n_o][Cp] floats, the ChainState array, the
// summary sums s1, s2, sa [n_o][Cp] doubles, and with stored samples the samples [nsave][n_o][Cp] floats and the
// sample records [nsave][C][3] doubles.
struct CheckpointShape {
  int64_t C, N, n_h, n_o, Cp, nsave;  // nsave: saved-sample capacity when samples are stored, else 0
  int64_t bytes() const {
    const int64_t no = std::max<int64_t>(n_o, 1);
    int64_t b = 8 * (int64_t)sizeof(int64_t);
    b += C * N * (int64_t)sizeof(float2);
    b += 2 * n_h * Cp * (int64_t)sizeof(float) + 2 * no * Cp * (int64_t)sizeof(float);
    b += C * (int64_t)sizeof(ChainState);
    b += 3 * no * Cp * (int64_t)sizeof(double);
    if (nsave > 0) b += nsave * no * Cp * (int64_t)sizeof(float) + nsave * C * 3 * (int64_t)sizeof(double);
    return b;
  }
};
static constexpr int64_t CKPT_MAGIC = 0x44524232434b5054LL, CKPT_VERSION = 1;

static CheckpointShape checkpoint_shape(const Chainset* s) {
  const DevVolume& v = s->vol->dv;
  const int64_t nsave = s->opts.store_samples ? std::max(s->opts.nsave, 1) : 0;
  return CheckpointShape{s->C, v.N, v.n_h, v.n_o, s->dc.Cp, nsave};
}

// Copies between the chain set's device state and the checkpoint buffer (to_host: save; else restore).
static void checkpoint_copy(Chainset* s, unsigned char* buf, bool to_host) {
  const CheckpointShape sh = checkpoint_shape(s);
  const DevChains& ch = s->dc;
  const int64_t no = std::max<int64_t>(sh.n_o, 1);
  cudaStream_t st = s->stream;
  const cudaMemcpyKind kind = to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice;
  auto copy = [&](void* dev, size_t bytes, size_t& off) {
    if (bytes == 0) return;
    if (to_host) CK(cudaMemcpyAsync(buf + off, dev, bytes, kind, st));
    else CK(cudaMemcpyAsync(dev, buf + off, bytes, kind, st));
    off += bytes;
  };
  size_t off = 8 * sizeof(int64_t);
  // the chain states first: on restore they say which half of U is each chain's accepted state
  std::vector<ChainState> states(sh.C);
  const size_t u_off = off;
  off += (size_t)sh.C * sh.N * sizeof(float2);
  const size_t mu_off = off;
  off += (size_t)(2 * sh.n_h * sh.Cp + 2 * no * sh.Cp) * sizeof(float);
  if (to_host) {
    read_states(s, &states);
    std::memcpy(buf + off, states.data(), sizeof(ChainState) * sh.C);
  } else {
    std::memcpy(states.data(), buf + off, sizeof(ChainState) * sh.C);
    write_states(s, states);
  }
  const size_t st_end = off + sizeof(ChainState) * sh.C;
  size_t o = u_off;
  for (int c = 0; c < sh.C; c++)
    copy(ch.U + ((int64_t)c * 2 + (states[c].acc & 1)) * sh.N, sizeof(float2) * sh.N, o);
  o = mu_off;
  copy(ch.muD, sizeof(float) * 2 * sh.n_h * sh.Cp, o);
  copy(ch.muO, sizeof(float) * 2 * no * sh.Cp, o);
  o = st_end;
  copy(ch.s1, sizeof(double) * no * sh.Cp, o);
  copy(ch.s2, sizeof(double) * no * sh.Cp, o);
  copy(ch.sa, sizeof(double) * no * sh.Cp, o);
  if (sh.nsave > 0) {
    copy(ch.samples, sizeof(float) * sh.nsave * no * sh.Cp, o);
    copy(ch.save_rec, sizeof(double) * sh.nsave * sh.C * 3, o);
  }
  CK(cudaStreamSynchronize(st));
  if ((int64_t)o != sh.bytes()) throw Error(DR_ERR_STATE, "checkpoint layout mismatch");
}

static void checkpoint_save(Chainset* s, void* buf, int64_t bytes) {
  const CheckpointShape sh = checkpoint_shape(s);
  if (bytes < sh.bytes()) throw Error(DR_ERR_INVALID, "checkpoint buffer too small");
  CK(cudaSetDevice(s->vol->device));
  auto* b = static_cast<unsigned char*>(buf);
  const int64_t hdr[8] = {CKPT_MAGIC, CKPT_VERSION, sh.C, sh.N, sh.n_h, sh.n_o, sh.Cp, sh.nsave};
  std::memcpy(b, hdr, sizeof(hdr));
  checkpoint_copy(s, b, true);
}

static void checkpoint_restore(Chainset* s, const void* buf, int64_t bytes) {
  const CheckpointShape sh = checkpoint_shape(s);
  if (bytes < 8 * (int64_t)sizeof(int64_t)) throw Error(DR_ERR_INVALID, "checkpoint buffer too small");
  int64_t hdr[8];
  std::memcpy(hdr, buf, sizeof(hdr));
  if (hdr[0] != CKPT_MAGIC || hdr[1] != CKPT_VERSION) throw Error(DR_ERR_INVALID, "not a chain-set checkpoint");
  const int64_t want[6] = {sh.C, sh.N, sh.n_h, sh.n_o, sh.Cp, sh.nsave};
  for (int i = 0; i < 6; i++)
    if (hdr[2 + i] != want[i])
      throw Error(DR_ERR_INVALID, "checkpoint of a chain set of another shape (chains, volume or stored samples)");
  if (bytes < sh.bytes()) throw Error(DR_ERR_INVALID, "checkpoint buffer too small");
  CK(cudaSetDevice(s->vol->device));
  checkpoint_copy(s, const_cast<unsigned char*>(static_cast<const unsigned char*>(buf)), false);
}

int dr_chainset_checkpoint_size(const dr_chainset* s, int64_t* bytes) {
  API_BEGIN
  if (!s || !bytes) throw Error(DR_ERR_INVALID, "NULL argument");
  *bytes = checkpoint_shape(s).bytes();
  API_END
}

int dr_chainset_checkpoint_save(dr_chainset* s, void* buf, int64_t bytes) {
  API_BEGIN
  if (!s || !buf) throw Error(DR_ERR_INVALID, "NULL argument");
  checkpoint_save(s, buf, bytes);
  API_END
}

int dr_chainset_checkpoint_restore(dr_chainset* s, const void* buf, int64_t bytes) {
  API_BEGIN
  if (!s || !buf) throw Error(DR_ERR_INVALID, "NULL argument");
  checkpoint_restore(s, buf, bytes);
  API_END
}

int dr_get_state(dr_chainset* s, int chain, float* mu, float* s2inv) {
  API_BEGIN
  if (!s || chain < 0 || chain >= s->C) throw Error(DR_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(s->vol->device));
  std::vector<ChainState> st;
  read_states(s, &st);
  const DevVolume& v = s->vol->dv;
  if (mu) {
    CK(cudaMemcpyAsync(s->tmp, s->dc.U + ((long long)chain * 2 + st[chain].acc) * v.N, sizeof(float2) * v.N,
                       cudaMemcpyDeviceToDevice, s->stream));
    DevChains none{};
    fft3d<float2>(s->tmp, s->vol->hv.E, -1, 0, 1, s->vol->tw_f, s->stream, v, none);
    k_scale<<<cdiv_i(v.N, 256), 256, 0, s->stream>>>(s->tmp, v.N, 1.0f / (float)v.N);
    CK_LAUNCH();
    CK(cudaMemcpyAsync(mu, s->tmp, sizeof(float2) * v.N, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  }
  if (s2inv) { s2inv[0] = st[chain].sh; s2inv[1] = st[chain].ss; }
  API_END
}

int dr_log_posterior(dr_chainset* s, int chain, const float* mu, double* out) {
  API_BEGIN
  if (!s || !mu || !out || chain < 0 || chain >= s->C) throw Error(DR_ERR_INVALID, "bad argument");
  eval_sampler(s, chain, mu, out, nullptr);
  API_END
}

int dr_gradient(dr_chainset* s, int chain, const float* mu, float* grad) {
  API_BEGIN
  if (!s || !mu || !grad || chain < 0 || chain >= s->C) throw Error(DR_ERR_INVALID, "bad argument");
  eval_sampler(s, chain, mu, nullptr, grad);
  API_END
}

int dr_leapfrog_fixed(dr_chainset* s, int chain, const float* mu0, const float* p0, float eps, int L, float* mu_out,
                      float* p_out, double* energies) {
  API_BEGIN
  if (!s || !mu0 || !p0 || chain < 0 || chain >= s->C || L <= 0) throw Error(DR_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(s->vol->device));
  std::vector<ChainState> st, saved;
  read_states(s, &st);
  saved = st;
  const DevVolume& v = s->vol->dv;
  const int acc = st[chain].acc;
  DevChains none{};
  // u0 and the data values of mu0
  upload_field(s, mu0);
  gather_data(s, s->tmp, chain, acc, false);
  fft3d<float2>(s->tmp, s->vol->hv.E, +1, 0, 1, s->vol->tw_f, s->stream, v, none);
  CK(cudaMemcpyAsync(s->dc.U + ((long long)chain * 2 + acc) * v.N, s->tmp, sizeof(float2) * v.N,
                     cudaMemcpyDeviceToDevice, s->stream));
  // q0 = IFFT(p0)
  upload_field(s, p0);
  fft3d<float2>(s->tmp, s->vol->hv.E, +1, 0, 1, s->vol->tw_f, s->stream, v, none);
  CK(cudaMemcpyAsync(s->dc.Q + (long long)chain * v.N, s->tmp, sizeof(float2) * v.N, cudaMemcpyDeviceToDevice,
                     s->stream));
  for (int c = 0; c < s->C; c++) st[c].L_cur = -1;
  st[chain].L_cur = L;
  st[chain].eps_cur = eps;
  write_states(s, st);
  enqueue_steps(s, L, XF_FIXED_MOMENTUM | XF_WRITE_Q_LAST);
  CK(cudaStreamSynchronize(s->stream));
  const double N = (double)v.N;
  const double sh = st[chain].sh, ss = st[chain].ss;
  if (energies) {
    const double K0 = part_sum(s, chain, SL_E0, s->dc.nb_x), lp0 = part_sum(s, chain, SL_LP0, s->dc.nb_x);
    const double Rh0 = part_sum(s, chain, SL_RH0, s->dc.nb_wt), RhL = part_sum(s, chain, SL_RHL, s->dc.nb_wt);
    const double Rs0 = v.n_s > 0 ? part_sum(s, chain, SL_RS0, s->dc.nb_w) : 0.0;
    const double RsL = v.n_s > 0 ? part_sum(s, chain, SL_RSL, s->dc.nb_w) : 0.0;
    const double lpL = part_sum(s, chain, SL_LPL, s->dc.nb_x), KL = part_sum(s, chain, SL_KL, s->dc.nb_x);
    energies[0] = -0.5 * lp0 / N;
    energies[1] = -0.5 * (sh * Rh0 + ss * Rs0);
    energies[2] = -0.5 * K0 / N;
    energies[3] = -0.5 * lpL / N;
    energies[4] = -0.5 * (sh * RhL + ss * RsL);
    energies[5] = -0.5 * KL / N;
  }
  if (mu_out) {
    CK(cudaMemcpyAsync(s->tmp, s->dc.U + ((long long)chain * 2 + (acc ^ 1)) * v.N, sizeof(float2) * v.N,
                       cudaMemcpyDeviceToDevice, s->stream));
    fft3d<float2>(s->tmp, s->vol->hv.E, -1, 0, 1, s->vol->tw_f, s->stream, v, none);
    k_scale<<<cdiv_i(v.N, 256), 256, 0, s->stream>>>(s->tmp, v.N, 1.0f / (float)v.N);
    CK_LAUNCH();
    CK(cudaMemcpyAsync(mu_out, s->tmp, sizeof(float2) * v.N, cudaMemcpyDeviceToHost, s->stream));
  }
  if (p_out) {
    CK(cudaMemcpyAsync(s->tmp, s->dc.Q + (long long)chain * v.N, sizeof(float2) * v.N, cudaMemcpyDeviceToDevice,
                       s->stream));
    fft3d<float2>(s->tmp, s->vol->hv.E, -1, 0, 1, s->vol->tw_f, s->stream, v, none);
    k_scale<<<cdiv_i(v.N, 256), 256, 0, s->stream>>>(s->tmp, v.N, 1.0f / (float)v.N);
    CK_LAUNCH();
    CK(cudaMemcpyAsync(p_out, s->tmp, sizeof(float2) * v.N, cudaMemcpyDeviceToHost, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  // the chain keeps mu0 as its state; the other chains are untouched
  for (int c = 0; c < s->C; c++) saved[c].L_cur = -1;
  write_states(s, saved);
  check_device_error(s);
  API_END
}

int dr_kriging_matrix(const float* hr, int nx, int ny, int nz, const float* Qhr, const float* sr, int sx, int sy,
                      int sz, const float* Qsr, const float* theta, float radius, int* n_rows, int64_t* nnz,
                      int** rowptr, int** col, float** val) {
  API_BEGIN
  if (!hr || !Qhr || !sr || !Qsr || !theta || !n_rows || !nnz || !rowptr || !col || !val)
    throw Error(DR_ERR_INVALID, "NULL argument");
  if (nx <= 0 || ny <= 0 || nz <= 0 || sx <= 0 || sy <= 0 || sz <= 0) throw Error(DR_ERR_INVALID, "bad grid");
  std::vector<int> rp, cl;
  std::vector<float> vl;
  std::string err;
  int nofs = 0;
  const int rc = kriging_build(hr, nx, ny, nz, Qhr, sr, sx, sy, sz, Qsr, theta, radius, &rp, &cl, &vl, &nofs, &err);
  if (rc != DR_OK) throw Error(rc, err);
  *n_rows = (int)rp.size() - 1;
  *nnz = (int64_t)cl.size();
  *rowptr = (int*)std::malloc(sizeof(int) * rp.size());
  *col = (int*)std::malloc(sizeof(int) * std::max<size_t>(cl.size(), 1));
  *val = (float*)std::malloc(sizeof(float) * std::max<size_t>(vl.size(), 1));
  if (!*rowptr || !*col || !*val) {
    std::free(*rowptr); std::free(*col); std::free(*val);
    throw Error(DR_ERR_NOMEM, "host allocation failed");
  }
  std::memcpy(*rowptr, rp.data(), sizeof(int) * rp.size());
  if (!cl.empty()) std::memcpy(*col, cl.data(), sizeof(int) * cl.size());
  if (!vl.empty()) std::memcpy(*val, vl.data(), sizeof(float) * vl.size());
  API_END
}

void dr_free(void* p) { std::free(p); }

int dr_debug_tc_layout(int n_rows, int n_cols, const int* rowptr, const int* col, const float* val,
                       const uint32_t* keys, int g_max, float* dense, int64_t* stats) {
  API_BEGIN
  if (n_rows < 0 || n_cols < 0 || !rowptr || !keys || !dense || !stats || (rowptr[n_rows] > 0 && (!col || !val)))
    throw Error(DR_ERR_INVALID, "bad argument");
  const int nnz = rowptr[n_rows];
  std::vector<int> rp(rowptr, rowptr + n_rows + 1), cl(col, col + nnz);
  std::vector<uint32_t> ky(keys, keys + n_rows);
  TcPlanHost P;
  if (!tc_plan(rp, cl.data(), cl.size(), ky, g_max, &P)) throw Error(DR_ERR_INVALID, "matrix too large for the tile layout");
  std::vector<float> blob((size_t)P.chunks * TC_BLK, 0.f);
  for (int i = 0; i < nnz; i++) blob[P.dest[i]] = val[i];
  std::fill(dense, dense + (size_t)n_rows * n_cols, 0.f);
  const int nseg = (int)(P.segs.size() / 4);
  std::vector<int> chunk_seen(P.chunks, 0), row_seen(n_rows, 0);
  for (int g = 0; g < nseg; g++) {
    const int t = P.segs[4 * g];
    for (int c = P.segs[4 * g + 1]; c < P.segs[4 * g + 2]; c++) {
      chunk_seen[c]++;
      for (int m = 0; m < TC_M; m++) {
        const int row = P.tile_rows[(size_t)t * TC_M + m];
        for (int kk = 0; kk < TC_KC; kk++) {
          const int cc = P.chunk_cols[(size_t)c * TC_KC + kk];
          const size_t off = (size_t)c * TC_BLK + (kk / 4) * (TC_M * 4) + m * 4 + kk % 4;
          if (row >= 0 && cc >= 0) dense[(size_t)row * n_cols + cc] += blob[off];
          else if (blob[off] != 0.f) dense[0] = NAN;  // padding must stay zero
        }
      }
    }
  }
  for (int r : P.tile_rows)
    if (r >= 0) row_seen[r]++;
  bool consistent = P.tile_seg_ptr.size() == (size_t)P.T + 1 && P.tile_seg_ptr[P.T] == nseg &&
                    P.cta_seg_ptr.size() == (size_t)P.G + 1 && P.cta_seg_ptr[P.G] == nseg;
  for (int t = 0; consistent && t < P.T; t++)
    for (int g = P.tile_seg_ptr[t]; g < P.tile_seg_ptr[t + 1]; g++) consistent = consistent && P.segs[4 * g] == t;
  for (int b = 0; consistent && b < P.G; b++) consistent = P.cta_seg_ptr[b] < P.cta_seg_ptr[b + 1];
  stats[0] = P.T;
  stats[1] = P.chunks;
  stats[2] = nseg;
  stats[3] = P.G;
  stats[4] = std::count(chunk_seen.begin(), chunk_seen.end(), 1);
  stats[5] = std::count(row_seen.begin(), row_seen.end(), 1);
  stats[6] = consistent ? 1 : 0;
  API_END
}

int dr_debug_time_kernel(dr_chainset* s, int which, int stp, int reps, double* avg_ms, double* algo_bytes) {
  API_BEGIN
  if (!s || !avg_ms || reps <= 0 || stp < 1 || which < 0 || which > 6) throw Error(DR_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(s->vol->device));
  const DevVolume& v = s->vol->dv;
  const DevChains& ch = s->dc;
  const float2* tw = s->vol->tw_f;
  const int C = s->C;
  const double N = (double)v.N, t1 = (double)ch.t1_stride, t2 = (double)ch.t2_stride, z = (double)s->vol->hv.w_col.size();
  auto launch = [&]() {
    switch (which) {
      case 0: if (s->plane) launch_plane(s, stp, 0); else launch_xline(s, stp, 0); break;
      case 1: if (s->plane) break;
        launch_pass<float2>(v.E1, -1, PRO_LOAD, EPI_STORE, pass_args(ch.T1, ch.T2, ch.t1_stride, ch.t2_stride, v.E2, v.bx, v.E1, v.by, 1.0, stp), v, ch, tw, C, s->stream); break;
      case 2: launch_pass<float2>(v.E2, -1, PRO_LOAD, EPI_GATHER, pass_args(ch.T2, nullptr, ch.t2_stride, 0, 1, v.by * v.bx, v.E2, v.bz, 1.0 / N, stp, 1, 2), v, ch, tw, C, s->stream); break;
      case 3: if (v.n_s > 0) launch_spmv(s, stp, 1, -1, true); break;
      case 4: launch_spmv(s, stp, 1, -1, false); break;
      case 5: launch_pass<float2>(v.E2, +1, PRO_DATAGRAD, EPI_STORE, pass_args(nullptr, ch.T2, 0, ch.t2_stride, 1, v.by * v.bx, v.bz, v.E2, 1.0, stp), v, ch, tw, C, s->stream); break;
      default: if (s->plane) break;
        launch_pass<float2>(v.E1, +1, PRO_LOAD, EPI_STORE, pass_args(ch.T2, ch.T1, ch.t2_stride, ch.t1_stride, v.E2, v.bx, v.by, v.E1, 1.0, stp), v, ch, tw, C, s->stream); break;
    }
  };
  launch();  // warm-up
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaEventRecord(e0, s->stream));
  for (int i = 0; i < reps; i++) launch();
  CK(cudaEventRecord(e1, s->stream));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *avg_ms = (double)ms / reps;
  if (algo_bytes) {
    // bytes a launch must move (each array read or written once; shared arrays once per launch)
    const double box = (double)v.bx * v.by * v.bz;
    double b = 0.0;
    switch (which) {
      case 0: b = C * (2.0 * (s->plane ? t2 : t1) * 8 + 4.0 * N * 8) + N * 4; break;  // T in/out, U and q in/out, 1/lambda
      case 1: b = s->plane ? 0.0 : C * (t1 + t2) * 8; break;
      case 2: b = C * (t2 * 8 + (v.n_h + v.n_o) * 4.0) + box * 8; break;            // box maps (2 x int32)
      case 3: b = z * 8 + C * ((double)v.n_h * 4 + (double)v.n_s * 4) + v.n_s * 8.0; // W values + columns, mu_D, rs
        break;
      case 4: b = z * 8 + C * ((double)v.n_s * 4 + 2.0 * v.n_h * 4) + v.n_h * 12.0; break;
      case 5: b = C * ((double)v.n_h * 4 + t2 * 8) + box * 4; break;
      default: b = s->plane ? 0.0 : C * (t2 + t1) * 8; break;
    }
    if (s->tcp && (which == 3 || which == 4)) {
      // tensor-core products: the dense FP32 blob, the chain vectors of every chunk column, the segment partials
      // written and read back, and the epilogue's operands (rs; or mu_D in and gD out)
      const DevTcMatrix& M = which == 3 ? s->vol->tc_w : s->vol->tc_wt;
      b = (double)M.chunks * TC_BLK * 4 + (double)M.chunks * TC_KC * C * 4 +
          2.0 * M.n_segs * s->tc_N * TC_M * 4 + (which == 3 ? (double)v.n_s * C * 4 : 2.0 * v.n_h * C * 4);
    }
    *algo_bytes = b;
  }
  API_END
}

int dr_debug_pool_usage(int device, int reset_high, uint64_t* used, uint64_t* high) {
  API_BEGIN
  if (!used || !high) throw Error(DR_ERR_INVALID, "bad argument");
  cudaMemPool_t pool = device_tables(device).pool;
  if (reset_high) {
    uint64_t zero = 0;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
  }
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, used));
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, high));
  API_END
}

int dr_debug_bounded_wait(int device, double limit_ms, int* gave_up, double* waited_ms) {
  API_BEGIN
  if (!gave_up || !waited_ms || !(limit_ms > 0 && limit_ms <= 10000)) throw Error(DR_ERR_INVALID, "bad argument");
  device_tables(device);
  CK(cudaSetDevice(device));
  int* d_flag = nullptr;
  unsigned long long* d_ns = nullptr;
  CK(cudaMalloc(&d_flag, sizeof(int)));
  const cudaError_t e = cudaMalloc(&d_ns, sizeof(unsigned long long));
  if (e != cudaSuccess) {
    cudaFree(d_flag);
    throw Error(DR_ERR_NOMEM, "cudaMalloc");
  }
  k_debug_bounded_wait<<<1, 32>>>((uint64_t)(limit_ms * 1e6), d_flag, d_ns);
  const cudaError_t le = cudaGetLastError();
  unsigned long long ns = 0;
  int flag = -1;
  const cudaError_t c1 = le == cudaSuccess ? cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost) : le;
  const cudaError_t c2 = c1 == cudaSuccess ? cudaMemcpy(&ns, d_ns, sizeof(ns), cudaMemcpyDeviceToHost) : c1;
  cudaFree(d_flag);
  cudaFree(d_ns);
  CK(c2);
  *gave_up = flag;
  *waited_ms = (double)ns * 1e-6;
  API_END
}

int dr_debug_dual_averaging(int burnin, int nsave, int thin, int L, float starting_eps, float mhtarget, int n,
                            const float* rates, double* eps_out, int* steps_out, int device) {
  API_BEGIN
  if (n < 0 || !rates || !eps_out || !steps_out) throw Error(DR_ERR_INVALID, "bad argument");
  device_tables(device);
  CK(cudaSetDevice(device));
  ChainState h;
  std::memset(&h, 0, sizeof(h));
  h.warmup = burnin > 0;
  h.eps_start_found = !h.warmup;
  h.burnin = burnin;
  h.integrator_steps = L;
  h.n_save = nsave;
  h.thin = thin == 0 ? 1 : thin;
  h.A = 1;
  h.eps0 = 1e-5;
  h.eps = std::max((double)starting_eps, h.eps0);
  h.eps_bar = 1;
  h.gamma = (double)0.05f;
  h.mh_target = (double)mhtarget;
  h.t0 = 10;
  h.kappa = (double)0.75f;
  float* dr = nullptr;
  double* de = nullptr;
  int* ds = nullptr;
  CK(cudaMalloc(&dr, sizeof(float) * std::max(n, 1)));
  CK(cudaMalloc(&de, sizeof(double) * std::max(n, 1)));
  CK(cudaMalloc(&ds, sizeof(int) * std::max(n, 1)));
  cudaError_t e = cudaMemcpy(dr, rates, sizeof(float) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_debug_dual_averaging<<<1, 32>>>(h, n, dr, de, ds);
    e = cudaGetLastError();
    g_launches++;
  }
  if (e == cudaSuccess) e = cudaMemcpy(eps_out, de, sizeof(double) * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(steps_out, ds, sizeof(int) * n, cudaMemcpyDeviceToHost);
  cudaFree(dr);
  cudaFree(de);
  cudaFree(ds);
  if (e != cudaSuccess) throw Error(DR_ERR_CUDA, cudaGetErrorString(e));
  API_END
}


}  // extern "C"


// ==================================================================== server
namespace drb {

struct Job {
  uint64_t id = 0;
  std::vector<float> hr, hm, om, sr, sm;
  float qh[16], qs[16];
  dr_volume_desc desc{};
  dr_hmc_opts opts{};
  int C = 1;
  int state = DR_JOB_QUEUED;
  int error = 0;
  std::string msg;
  double t_submit = 0, t_admit = 0, t_finish = 0;
  std::unique_ptr<Volume> vol;
  std::unique_ptr<Chainset> cs;
  int64_t est_bytes = 0, bytes = 0;
  int iters_total = 0, iters_launched = 0;
  bool in_flight = false;
  std::atomic<bool> preempt_req{false};  // checkpoint and release at the next round boundary
  std::vector<unsigned char> ckpt;   // chain-set checkpoint of a preempted job, restored when it is rebuilt
  std::vector<float> mean, var, act;
  int64_t grads = 0;
  float mh = 0.f;
  int n_output = 0;
};

// Device bytes of a volume + chain set before creating them (admission).
static int64_t estimate_bytes(const HostVolume& hv, int C, const dr_hmc_opts& o) {
  const double N = (double)hv.N, box = (double)hv.box[0] * hv.box[1] * hv.box[2];
  const double nh = (double)hv.Yh.size(), ns = (double)hv.Ys.size(), no = (double)hv.o_flat.size();
  const double nnz = (double)hv.w_col.size();
  const double t2 = (double)hv.E[2] * hv.box[1] * hv.box[0];
  double vol = box * 8 + (nh + no) * 4 + (nh + ns) * 4 + (ns + nh + 2) * 4 + nnz * 16 + N * 12 + N * 16;
  double cs = C * (3 * N * 8 + t2 * 8 + (hv.E[0] == hv.E[1] ? 0.0 : (double)hv.E[2] * hv.E[1] * hv.box[0] * 8)) +
              C * (2 * (nh + no) * 4 + (nh + ns) * 4 + no * 24) + N * 8 + (double)C * 9 * 2048 * 8;
  if (o.store_samples) cs += (double)std::max(o.nsave, 1) * (no * 4 + 24) * C;
  if (tc_chains(C) > 0 && ns > 0) {
    // dense tiles of W and W^T for the tensor-core products (their column unions are a few times the nonzeros:
    // 5.8x and 3.1x on a 32^3 volume; 10x each is budgeted), index tables, and the segment partials
    vol += 2 * nnz * 10 * 4 + (nh + ns) * 8;
    cs += (double)((ns + nh) / TC_M + 2 + 2 * 148) * tc_chains(C) * TC_M * 4;
  }
  return (int64_t)(1.10 * (vol + cs)) + (16 << 20);
}

struct Server {
  dr_server_opts o{};
  std::mutex mtx;
  std::condition_variable cv_work, cv_done;
  std::map<uint64_t, std::shared_ptr<Job>> jobs;
  std::deque<std::shared_ptr<Job>> setup_q, ready_q;
  // admitted jobs whose device set-up (kriging solves, spectrum, chain set and its tuning) runs on a device-set-up
  // thread, so that the scheduler keeps launching the resident jobs' rounds meanwhile; then built, for the scheduler
  std::deque<std::shared_ptr<Job>> device_q, built_q;
  int in_device_setup = 0;
  int64_t reserved = 0;  // footprint estimates of the jobs in device set-up (admission counts them with in_use)
  std::vector<std::shared_ptr<Job>> active;  // scheduler thread only
  std::vector<std::thread> workers, device_workers;
  std::condition_variable cv_device;
  std::thread sched;
  bool stop = false;
  uint64_t next_id = 1;
  int64_t budget = 0, in_use = 0, peak_bytes = 0;
  int peak_running = 0;
  int64_t n_submitted = 0, n_done = 0, n_failed = 0, grads_done = 0, launches = 0;
  int64_t n_preempted = 0;  // jobs preempted and not resumed
  double last_finish = 0;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

  void fail(const std::shared_ptr<Job>& j, int code, const std::string& msg) {
    // caller holds mtx
    j->state = DR_JOB_FAILED;
    j->error = code;
    j->msg = msg;
    j->t_finish = now();
    n_failed++;
    cv_done.notify_all();
  }

  void worker_loop(int nthreads) {
#ifdef _OPENMP
    omp_set_num_threads(std::max(1, nthreads));
#endif
    for (;;) {
      std::shared_ptr<Job> j;
      {
        std::unique_lock<std::mutex> lk(mtx);
        cv_work.wait(lk, [&] { return stop || !setup_q.empty(); });
        if (stop) return;
        j = setup_q.front();
        setup_q.pop_front();
      }
      auto vol = std::make_unique<Volume>();
      std::string err;
      int rc = DR_OK;
      try {
        rc = host_prepare(&j->desc, &vol->hv, &err, device_kriging_enabled());
      } catch (const std::exception& e) {
        rc = DR_ERR_INVALID;
        err = e.what();
      }
      std::lock_guard<std::mutex> lk(mtx);
      j->hr.clear(); j->hr.shrink_to_fit();
      j->hm.clear(); j->om.clear(); j->sr.clear(); j->sm.clear();
      if (rc != DR_OK) {
        fail(j, rc, err);
        continue;
      }
      j->est_bytes = estimate_bytes(vol->hv, j->C, j->opts);
      j->vol = std::move(vol);
      j->state = DR_JOB_READY;
      ready_q.push_back(j);
      cv_work.notify_all();
    }
  }

  // Device set-up of admitted jobs (volume on the device, chain set with its tuning), each on the job's own streams,
  // concurrent with the scheduler's launches; the job's reserved estimate is then replaced by its allocated bytes.
  void device_worker_loop() {
    cudaSetDevice(o.device);
    for (;;) {
      std::shared_ptr<Job> j;
      {
        std::unique_lock<std::mutex> lk(mtx);
        cv_device.wait(lk, [&] { return stop || !device_q.empty(); });
        if (stop) return;
        j = device_q.front();
        device_q.pop_front();
      }
      int64_t bytes = 0;
      int code = DR_OK;
      std::string msg;
      try {
        volume_build_device(j->vol.get(), j->desc.covariance, j->desc.covfun, o.device);
        auto cs = std::make_unique<Chainset>();
        chainset_build(cs.get(), j->vol.get(), j->C, &j->opts);
        if (!j->ckpt.empty()) {  // a resumed job continues from its checkpoint
          checkpoint_restore(cs.get(), j->ckpt.data(), (int64_t)j->ckpt.size());
          j->ckpt.clear();
          j->ckpt.shrink_to_fit();
        }
        bytes = j->vol->bytes + cs->bytes;
        j->cs = std::move(cs);
        j->iters_total = j->opts.burnin + (j->opts.thin == 0 ? 1 : j->opts.thin) * j->opts.nsave;
      } catch (const Error& e) {
        code = e.code;
        msg = e.what();
      } catch (const std::bad_alloc&) {
        code = DR_ERR_NOMEM;
        msg = "host allocation failed";
      } catch (const std::exception& e) {
        code = DR_ERR_INVALID;
        msg = e.what();
      }
      if (code != DR_OK) {
        fail_resident(j, code, msg, false);
        std::lock_guard<std::mutex> lk(mtx);
        reserved -= j->est_bytes;
        in_device_setup--;
        cv_work.notify_all();
        continue;
      }
      std::lock_guard<std::mutex> lk(mtx);
      reserved -= j->est_bytes;
      in_use += bytes;
      peak_bytes = std::max(peak_bytes, in_use);
      j->bytes = bytes;
      in_device_setup--;
      built_q.push_back(j);
      cv_work.notify_all();
    }
  }

  // Saves a resident job's checkpoint (its round has completed), frees its device objects but keeps its host
  // set-up for the rebuild, and marks it preempted.
  void preempt(const std::shared_ptr<Job>& j) {
    Chainset* cs = j->cs.get();
    const int64_t n = checkpoint_shape(cs).bytes();
    std::vector<unsigned char> buf((size_t)n);
    checkpoint_save(cs, buf.data(), n);
    HostVolume hv = std::move(j->vol->hv);
    j->cs.reset();
    j->vol.reset();
    auto vol = std::make_unique<Volume>();
    vol->hv = std::move(hv);
    std::lock_guard<std::mutex> lk(mtx);
    j->ckpt = std::move(buf);
    j->vol = std::move(vol);
    j->preempt_req = false;
    j->in_flight = false;
    j->state = DR_JOB_PREEMPTED;
    in_use -= j->bytes;
    j->bytes = 0;
    n_preempted++;
    cv_done.notify_all();
  }

  // Reads a finished job's summary and frees its device objects; the fields that dr_server_status and
  // dr_server_result read are published under mtx together with the DONE state.
  void finalize(const std::shared_ptr<Job>& j) {
    Chainset* cs = j->cs.get();
    check_device_error(cs);
    const int n_output = cs->vol->dv.n_o;
    std::vector<float> mean(n_output), var(n_output), act(n_output);
    summary_of(cs, -1, mean.data(), var.data(), act.data());
    std::vector<ChainState> st;
    read_states(cs, &st);
    int64_t g = 0;
    double mh = 0;
    for (const auto& h : st) {
      g += h.grad_evals;
      const int d = h.iteration - h.burnin;
      mh += h.mh_running_sum / std::max(d, 1);
    }
    j->cs.reset();
    j->vol.reset();
    std::lock_guard<std::mutex> lk(mtx);
    j->n_output = n_output;
    j->mean = std::move(mean);
    j->var = std::move(var);
    j->act = std::move(act);
    j->grads = g;
    j->mh = (float)(mh / st.size());
    const int64_t b = j->bytes;
    j->state = DR_JOB_DONE;
    j->t_finish = now();
    in_use -= b;
    n_done++;
    grads_done += j->grads;
    last_finish = j->t_finish;
    cv_done.notify_all();
  }

  // Frees a failed job's device objects (the chain set drains its stream first) and records the failure.
  void fail_resident(const std::shared_ptr<Job>& j, int code, const std::string& msg, bool counted) {
    j->cs.reset();
    j->vol.reset();
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(mtx);
    if (counted) in_use -= j->bytes;
    fail(j, code, msg);
  }

  void scheduler_loop() {
    cudaSetDevice(o.device);
    for (;;) {
      // admit prepared jobs that fit: their estimated footprint is reserved and their device set-up handed to the
      // device-set-up threads; built jobs join the resident set
      {
        std::lock_guard<std::mutex> lk(mtx);
        while (!stop && !ready_q.empty() && (int)active.size() + in_device_setup < o.max_active) {
          std::shared_ptr<Job> j = ready_q.front();
          if (in_use + reserved + j->est_bytes > budget && !(active.empty() && in_device_setup == 0)) break;
          ready_q.pop_front();
          reserved += j->est_bytes;
          j->state = DR_JOB_RUNNING;
          j->t_admit = now();
          in_device_setup++;
          device_q.push_back(j);
          cv_device.notify_one();
        }
        if (!built_q.empty()) {
          while (!built_q.empty()) {
            active.push_back(built_q.front());
            built_q.pop_front();
          }
          // submission order: the in-flight budget favours the earliest jobs
          std::stable_sort(active.begin(), active.end(),
                           [](const std::shared_ptr<Job>& a, const std::shared_ptr<Job>& b) { return a->id < b->id; });
        }
        peak_running = std::max(peak_running, (int)active.size());
      }
      // advance resident jobs by one round, earliest admitted first while their chains fit the in-flight budget (a
      // job wider than the budget runs when nothing else is in flight); finalise finished ones
      bool launched = false, waiting = false;
      int chains_in_flight = 0;
      for (auto& j : active) {
        try {
          if (j->in_flight) {
            const cudaError_t q = cudaEventQuery(j->cs->done_event);
            if (q == cudaErrorNotReady) {
              waiting = true;
              chains_in_flight += j->C;
              continue;
            }
            if (q != cudaSuccess) throw Error(DR_ERR_CUDA, cudaGetErrorString(q));
            j->in_flight = false;
          }
          if (j->preempt_req) {
            preempt(j);
            continue;
          }
          if (j->iters_launched < j->iters_total) {
            if (chains_in_flight > 0 && chains_in_flight + j->C > o.max_chains_in_flight) {
              waiting = true;
              continue;
            }
            chains_in_flight += j->C;
            const int n = std::min(o.iterations_per_round, j->iters_total - j->iters_launched);
            launch_iterations(j->cs.get(), n);
            j->iters_launched += n;
            j->in_flight = true;
            launched = true;
          } else {
            finalize(j);
          }
        } catch (const Error& e) {
          fail_resident(j, e.code, e.what(), true);
        } catch (const std::bad_alloc&) {
          fail_resident(j, DR_ERR_NOMEM, "host allocation failed", true);
        } catch (const std::exception& e) {
          fail_resident(j, DR_ERR_INVALID, e.what(), true);
        }
      }
      active.erase(std::remove_if(active.begin(), active.end(),
                                  [](const std::shared_ptr<Job>& j) {
                                    return j->state == DR_JOB_DONE || j->state == DR_JOB_FAILED ||
                                           j->state == DR_JOB_PREEMPTED;
                                  }),
                   active.end());
      std::unique_lock<std::mutex> lk(mtx);
      launches = g_launches;
      if (stop) break;
      if (!launched) {
        if (waiting)
          cv_work.wait_for(lk, std::chrono::microseconds(50));
        else if (ready_q.empty())
          cv_work.wait_for(lk, std::chrono::milliseconds(2));
      }
    }
    // shutdown: wait for in-flight work, release device objects
    for (auto& j : active) {
      if (j->cs) cudaStreamSynchronize(j->cs->stream);
      j->cs.reset();
      j->vol.reset();
    }
    active.clear();
  }
};

}  // namespace drb

struct dr_server : Server {};

extern "C" {

int dr_server_create(const dr_server_opts* opts, dr_server** out) {
  API_BEGIN
  if (!opts || !out) throw Error(DR_ERR_INVALID, "NULL argument");
  *out = nullptr;
  device_tables(opts->device);
  CK(cudaSetDevice(opts->device));
  auto* sv = new dr_server();
  sv->o = *opts;
  if (sv->o.max_active <= 0) sv->o.max_active = 64;
  if (sv->o.iterations_per_round <= 0) sv->o.iterations_per_round = 8;
  if (sv->o.max_chains_in_flight <= 0) sv->o.max_chains_in_flight = 128;
  if (sv->o.host_threads <= 0) sv->o.host_threads = 4;
  if (sv->o.hbm_budget_bytes > 0) {
    sv->budget = sv->o.hbm_budget_bytes;
  } else {
    size_t fr = 0, tot = 0;
    CK(cudaMemGetInfo(&fr, &tot));
    sv->budget = (int64_t)(0.8 * (double)fr);
  }
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int per = std::max(1, hw / sv->o.host_threads);
  for (int i = 0; i < sv->o.host_threads; i++) sv->workers.emplace_back([sv, per] { sv->worker_loop(per); });
  // two device-set-up threads: one job's kriging solves and tuning overlap another's, and the resident jobs' rounds
  for (int i = 0; i < 2; i++) sv->device_workers.emplace_back([sv] { sv->device_worker_loop(); });
  sv->sched = std::thread([sv] { sv->scheduler_loop(); });
  *out = sv;
  API_END
}

void dr_server_destroy(dr_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mtx);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  sv->cv_device.notify_all();
  for (auto& t : sv->workers) t.join();
  for (auto& t : sv->device_workers) t.join();
  if (sv->sched.joinable()) sv->sched.join();
  delete sv;
}

int dr_server_submit(dr_server* sv, const dr_volume_desc* d, const dr_hmc_opts* opts, int n_chains, uint64_t* job_id) {
  API_BEGIN
  if (!sv || !d || !opts || !job_id || !d->highres || !d->qform_hr) throw Error(DR_ERR_INVALID, "NULL argument");
  if (n_chains <= 0 || n_chains > 256) throw Error(DR_ERR_UNSUPPORTED, "n_chains must be in [1, 256]");
  if (d->nx <= 0 || d->ny <= 0 || d->nz <= 0) throw Error(DR_ERR_INVALID, "bad high-res grid");
  auto j = std::make_shared<Job>();
  const size_t nh = (size_t)d->nx * d->ny * d->nz;
  j->hr.assign(d->highres, d->highres + nh);
  if (d->hmask) j->hm.assign(d->hmask, d->hmask + nh);
  if (d->omask) j->om.assign(d->omask, d->omask + nh);
  std::memcpy(j->qh, d->qform_hr, sizeof(j->qh));
  j->desc = *d;
  j->desc.highres = j->hr.data();
  j->desc.hmask = d->hmask ? j->hm.data() : nullptr;
  j->desc.omask = d->omask ? j->om.data() : nullptr;
  j->desc.qform_hr = j->qh;
  if (d->stdres) {
    if (!d->qform_sr || d->sx <= 0 || d->sy <= 0 || d->sz <= 0) throw Error(DR_ERR_INVALID, "bad std-res grid");
    const size_t ns = (size_t)d->sx * d->sy * d->sz;
    j->sr.assign(d->stdres, d->stdres + ns);
    if (d->smask) j->sm.assign(d->smask, d->smask + ns);
    std::memcpy(j->qs, d->qform_sr, sizeof(j->qs));
    j->desc.stdres = j->sr.data();
    j->desc.smask = d->smask ? j->sm.data() : nullptr;
    j->desc.qform_sr = j->qs;
  }
  j->desc.device = sv->o.device;
  j->opts = *opts;
  if (j->opts.leapfrog <= 0 || j->opts.burnin < 0 || j->opts.nsave < 0 || j->opts.thin < 0 ||
      !(j->opts.mhtarget > 0 && j->opts.mhtarget < 1))
    throw Error(DR_ERR_DOMAIN, "HMCParameters: invalid settings");
  j->C = n_chains;
  std::lock_guard<std::mutex> lk(sv->mtx);
  j->id = sv->next_id++;
  j->t_submit = sv->now();
  sv->jobs[j->id] = j;
  sv->setup_q.push_back(j);
  sv->n_submitted++;
  *job_id = j->id;
  sv->cv_work.notify_all();
  API_END
}

static std::shared_ptr<Job> find_job(dr_server* sv, uint64_t id) {
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) throw Error(DR_ERR_INVALID, "unknown job id");
  return it->second;
}

int dr_server_status(dr_server* sv, uint64_t job_id, dr_job_status* out) {
  API_BEGIN
  if (!sv || !out) throw Error(DR_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(sv->mtx);
  auto j = find_job(sv, job_id);
  std::memset(out, 0, sizeof(*out));
  out->state = j->state;
  out->error = j->error;
  out->submit_s = j->t_submit;
  out->admit_s = j->t_admit;
  out->finish_s = j->t_finish;
  out->grad_evals = j->grads;
  out->mh_rate = j->mh;
  out->n_output = j->n_output;
  out->device_bytes = j->bytes;
  API_END
}

int dr_server_result(dr_server* sv, uint64_t job_id, float* mean, float* var, float* activation) {
  API_BEGIN
  if (!sv) throw Error(DR_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(sv->mtx);
  auto j = find_job(sv, job_id);
  if (j->state == DR_JOB_FAILED) throw Error(j->error ? j->error : DR_ERR_STATE, "job failed: " + j->msg);
  if (j->state != DR_JOB_DONE) throw Error(DR_ERR_STATE, "job not finished");
  if (mean) std::memcpy(mean, j->mean.data(), sizeof(float) * j->mean.size());
  if (var) std::memcpy(var, j->var.data(), sizeof(float) * j->var.size());
  if (activation) std::memcpy(activation, j->act.data(), sizeof(float) * j->act.size());
  API_END
}

int dr_server_wait(dr_server* sv, uint64_t job_id, double timeout_s) {
  API_BEGIN
  if (!sv) throw Error(DR_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(sv->mtx);
  auto j = find_job(sv, job_id);
  const bool ok = sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    return j->state == DR_JOB_DONE || j->state == DR_JOB_FAILED;
  });
  if (!ok) throw Error(DR_ERR_TIMEOUT, "job still running");
  if (j->state == DR_JOB_FAILED) throw Error(j->error ? j->error : DR_ERR_STATE, "job failed: " + j->msg);
  API_END
}

int dr_server_preempt(dr_server* sv, uint64_t job_id, double timeout_s) {
  API_BEGIN
  if (!sv) throw Error(DR_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(sv->mtx);
  auto j = find_job(sv, job_id);
  if (j->state != DR_JOB_RUNNING) throw Error(DR_ERR_STATE, "only an admitted, unfinished job can be preempted");
  j->preempt_req = true;
  sv->cv_work.notify_all();
  const bool ok = sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    return j->state == DR_JOB_PREEMPTED || j->state == DR_JOB_DONE || j->state == DR_JOB_FAILED;
  });
  if (!ok) throw Error(DR_ERR_TIMEOUT, "job not preempted yet");
  if (j->state == DR_JOB_FAILED) throw Error(j->error ? j->error : DR_ERR_STATE, "job failed: " + j->msg);
  if (j->state == DR_JOB_DONE) throw Error(DR_ERR_STATE, "job finished before it could be preempted");
  API_END
}

int dr_server_resume(dr_server* sv, uint64_t job_id) {
  API_BEGIN
  if (!sv) throw Error(DR_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(sv->mtx);
  auto j = find_job(sv, job_id);
  if (j->state != DR_JOB_PREEMPTED) throw Error(DR_ERR_STATE, "job is not preempted");
  j->state = DR_JOB_READY;
  sv->n_preempted--;
  sv->ready_q.push_back(j);
  sv->cv_work.notify_all();
  API_END
}

int dr_server_drain(dr_server* sv, double timeout_s) {
  API_BEGIN
  if (!sv) throw Error(DR_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(sv->mtx);
  const bool ok = sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                       [&] { return sv->n_done + sv->n_failed + sv->n_preempted >= sv->n_submitted; });
  if (!ok) throw Error(DR_ERR_TIMEOUT, "jobs still running");
  API_END
}

int dr_server_stats_get(dr_server* sv, dr_server_stats* out) {
  API_BEGIN
  if (!sv || !out) throw Error(DR_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(sv->mtx);
  out->submitted = sv->n_submitted;
  out->done = sv->n_done;
  out->failed = sv->n_failed;
  out->running = sv->n_submitted - sv->n_done - sv->n_failed - sv->n_preempted;
  out->grad_evals = sv->grads_done;
  out->peak_device_bytes = sv->peak_bytes;
  out->peak_running = sv->peak_running;
  out->busy_s = sv->last_finish;
  out->kernel_launches = sv->launches;
  API_END
}

int dr_server_forget(dr_server* sv, uint64_t job_id) {
  API_BEGIN
  if (!sv) throw Error(DR_ERR_INVALID, "NULL server");
  std::lock_guard<std::mutex> lk(sv->mtx);
  auto j = find_job(sv, job_id);
  if (j->state != DR_JOB_DONE && j->state != DR_JOB_FAILED) throw Error(DR_ERR_STATE, "job not finished");
  sv->jobs.erase(job_id);
  API_END
}

}  // extern "C"

// ==================================================================== covariance estimation
extern "C" {

int dr_mce_offsets(int* offsets, int max_out, int* n) {
  API_BEGIN
  if (!n) throw Error(DR_ERR_INVALID, "NULL argument");
  const std::vector<int> P = mce_offsets();
  *n = (int)(P.size() / 3);
  if (offsets) std::memcpy(offsets, P.data(), sizeof(int) * 3 * std::min(*n, std::max(max_out, 0)));
  API_END
}

int dr_mce_summary(const float* img, int nx, int ny, int nz, const float* qform, int device, float* distance,
                   float* covariance, int* npairs, double* sums) {
  API_BEGIN
  if (!img || !qform || !distance || !covariance || !npairs) throw Error(DR_ERR_INVALID, "NULL argument");
  if (nx <= 0 || ny <= 0 || nz <= 0) throw Error(DR_ERR_INVALID, "bad grid");
  const std::vector<int> P = mce_offsets();
  const int n_off = (int)(P.size() / 3);
  const std::vector<float> d = mce_distances(P, qform);
  std::memcpy(distance, d.data(), sizeof(float) * n_off);
  device_tables(device);
  CK(cudaSetDevice(device));
  const long long nvox = (long long)nx * ny * nz;
  const int rows = ny * nz;
  int n_slabs = std::max(1, std::min(32, rows / 256));
  const int rows_per_slab = cdiv_i(rows, n_slabs);
  n_slabs = cdiv_i(rows, rows_per_slab);
  cudaStream_t st = nullptr;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  std::vector<void*> bufs;
  auto dalloc = [&](size_t bytes) {
    void* p = nullptr;
    const cudaError_t e = dev_alloc(&p, std::max<size_t>(bytes, 16), st);
    if (e != cudaSuccess) throw Error(DR_ERR_NOMEM, std::string("device allocation: ") + cudaGetErrorString(e));
    bufs.push_back(p);
    return p;
  };
  try {
    float* d_img = (float*)dalloc(sizeof(float) * nvox);
    int* d_P = (int*)dalloc(sizeof(int) * P.size());
    MceSums* d_part = (MceSums*)dalloc(sizeof(MceSums) * (size_t)n_slabs * n_off);
    float* d_cov = (float*)dalloc(sizeof(float) * n_off);
    int* d_np = (int*)dalloc(sizeof(int) * n_off);
    double* d_sums = sums ? (double*)dalloc(sizeof(double) * 3 * n_off) : nullptr;
    CK(cudaMemcpyAsync(d_img, img, sizeof(float) * nvox, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_P, P.data(), sizeof(int) * P.size(), cudaMemcpyHostToDevice, st));
    const dim3 grid(n_slabs, cdiv_i(n_off, MCE_OFFSETS_PER_CTA));
    k_mce_partial<<<grid, MCE_THREADS, 0, st>>>(d_img, nx, ny, nz, d_P, n_off, rows_per_slab, d_part);
    CK_LAUNCH();
    k_mce_finish<<<cdiv_i(n_off, 256), 256, 0, st>>>(d_part, n_slabs, n_off, d_cov, d_np, d_sums);
    CK_LAUNCH();
    CK(cudaMemcpyAsync(covariance, d_cov, sizeof(float) * n_off, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(npairs, d_np, sizeof(int) * n_off, cudaMemcpyDeviceToHost, st));
    if (sums) CK(cudaMemcpyAsync(sums, d_sums, sizeof(double) * 3 * n_off, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  } catch (...) {
    for (void* p : bufs) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    cudaGetLastError();
    throw;
  }
  for (void* p : bufs) cudaFreeAsync(p, st);
  CK(cudaStreamSynchronize(st));
  cudaStreamDestroy(st);
  API_END
}

int dr_fit_rbf_parameters(const float* distance, const float* covariance, const int* npairs, int n, double* theta) {
  API_BEGIN
  if (!distance || !covariance || !npairs || !theta) throw Error(DR_ERR_INVALID, "NULL argument");
  std::string err;
  if (fit_rbf_parameters(distance, covariance, npairs, n, theta, &err) != 0) throw Error(DR_ERR_DOMAIN, err);
  API_END
}

int dr_estimate_covariance(const float* img, int nx, int ny, int nz, const float* qform, int device, double* theta) {
  API_BEGIN
  if (!theta) throw Error(DR_ERR_INVALID, "NULL argument");
  int n = 0;
  CK_API(dr_mce_offsets(nullptr, 0, &n));
  std::vector<float> dist(n), cov(n);
  std::vector<int> np(n);
  CK_API(dr_mce_summary(img, nx, ny, nz, qform, device, dist.data(), cov.data(), np.data(), nullptr));
  CK_API(dr_fit_rbf_parameters(dist.data(), cov.data(), np.data(), n, theta));
  API_END
}

}  // extern "C"

// ==================================================================== allocation-free evaluation
namespace drb {

// Scratch of dr_log_posterior_noalloc: one array in the library's device
// image, so that the call itself never allocates.  Layout (bytes):
//   [0, 16 MiB)      complex field, N <= 2^21
//   [16, 24 MiB)     Re mu at data voxels, two halves of n_h <= 2^20
//   [24, 28 MiB)     Ys - W mu_D, n_s <= 2^20
//   [28, 32 MiB)     data gradient (written by the W^T kernel, not used)
//   [32 MiB, +256 KiB) partial sums, chain state, result
constexpr long long NA_MAX_N = 1LL << 21;
constexpr long long NA_MAX_ROWS = 1LL << 20;
constexpr size_t NA_FIELD = 0;
constexpr size_t NA_MUD = NA_FIELD + sizeof(float2) * NA_MAX_N;
constexpr size_t NA_RS = NA_MUD + 2 * sizeof(float) * NA_MAX_ROWS;
constexpr size_t NA_GD = NA_RS + sizeof(float) * NA_MAX_ROWS;
constexpr size_t NA_PART = NA_GD + sizeof(float) * NA_MAX_ROWS;
constexpr int NA_MAXBLK = 148 * 8;
constexpr int NA_EBLK = 296;
constexpr size_t NA_EPART = NA_PART + ((sizeof(double) * NSLOT * NA_MAXBLK + 255) / 256) * 256;
constexpr size_t NA_ST = NA_EPART + ((sizeof(double) * NA_EBLK + 255) / 256) * 256;
constexpr size_t NA_OUT = NA_ST + ((sizeof(ChainState) + 255) / 256) * 256;
constexpr size_t NA_BYTES = NA_OUT + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

static std::mutex g_na_mtx;
static unsigned char* g_na_ptr[64] = {nullptr};

// Device address of the scratch array on device `dev` (looked up once per
// device with that device current; the host-side symbol is not a device address).
static unsigned char* noalloc_scratch(int dev) {
  std::lock_guard<std::mutex> lk(g_na_mtx);
  if (dev < 0 || dev >= 64) throw Error(DR_ERR_INVALID, "device ordinal out of range");
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Error(DR_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_na_ptr[dev] = (unsigned char*)p;
  }
  return g_na_ptr[dev];
}

// Sums the partials of the prior (mode 0 spectral energy), the W product and
// the W^T product in a fixed order and forms (log prior, log likelihood).
__global__ void k_noalloc_finish(const double* epart, int neblk, const double* part, int maxblk, int nbw, int nbwt,
                                 const ChainState* st, double N, int n_s, double* out) {
  __shared__ double red[8];
  double e = 0.0, rh = 0.0, rs = 0.0;
  for (int i = threadIdx.x; i < neblk; i += blockDim.x) e += epart[i];
  e = block_sum(e, red);
  for (int i = threadIdx.x; i < nbwt; i += blockDim.x) rh += part[(long long)SL_RH0 * maxblk + i];
  rh = block_sum(rh, red);
  if (n_s > 0)
    for (int i = threadIdx.x; i < nbw; i += blockDim.x) rs += part[(long long)SL_RS0 * maxblk + i];
  rs = block_sum(rs, red);
  if (threadIdx.x == 0) {
    out[0] = -0.5 * e / N;
    out[1] = -0.5 * ((double)st->sh * rh + (n_s > 0 ? (double)st->ss * rs : 0.0));
  }
}

}  // namespace drb

// Makes `dev` current for its scope and gives the caller's current device back at the end, on success and on error.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    CK(cudaSetDevice(dev));
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

extern "C" int dr_log_posterior_noalloc(const dr_volume* v, const float* mu_device, float s_hr, float s_sr,
                                        double* out) {
  API_BEGIN
  if (!v || !mu_device || !out) throw Error(DR_ERR_INVALID, "dr_log_posterior_noalloc: NULL argument");
  const DevVolume& dv = v->dv;
  if (dv.N > NA_MAX_N)
    throw Error(DR_ERR_UNSUPPORTED, "dr_log_posterior_noalloc: embedding of " + std::to_string(dv.N) +
                                        " points exceeds the scratch limit of 2^21 (use dr_log_posterior)");
  if (dv.n_h > NA_MAX_ROWS || dv.n_s > NA_MAX_ROWS)
    throw Error(DR_ERR_UNSUPPORTED, "dr_log_posterior_noalloc: more than 2^20 data voxels (use dr_log_posterior)");
  const DeviceScope scope(v->device);
  unsigned char* base = noalloc_scratch(v->device);
  float2* field = (float2*)(base + NA_FIELD);
  ChainState* st = (ChainState*)(base + NA_ST);
  DevChains ch{};
  ch.C = 1;
  ch.Cp = 1;
  ch.CG = 1;
  ch.muD = (float*)(base + NA_MUD);
  ch.rs = (float*)(base + NA_RS);
  ch.gD = (float*)(base + NA_GD);
  ch.part = (double*)(base + NA_PART);
  ch.maxblk = NA_MAXBLK;
  ch.nb_w = std::max(1, std::min(dv.n_s, NA_MAXBLK));
  ch.nb_wt = std::max(1, std::min(cdiv_i(dv.n_h, 8), NA_MAXBLK));
  ch.st = st;
  ChainState h;
  std::memset(&h, 0, sizeof(h));
  h.sh = s_hr;
  h.ss = s_sr;
  h.acc = 0;
  h.L_cur = 0;
  cudaStream_t s = 0;
  CK(cudaMemcpyAsync(st, &h, sizeof(ChainState), cudaMemcpyHostToDevice, s));
  // Re mu at the data voxels, then the kriging residuals and their norms
  k_gather_re<<<cdiv_i(dv.n_h, 256), 256, 0, s>>>((const float2*)mu_device, dv.d_flat, dv.n_h, ch.muD, 1, 0, dv.N,
                                                   nullptr);
  CK_LAUNCH();
  if (dv.n_s > 0) launch_spmv_dc(dv, ch, 1, -1, 0, 0, true, s);
  launch_spmv_dc(dv, ch, 1, -1, 0, 0, false, s);
  // u = IFFT(mu) in the scratch field, then the prior's spectral sum
  CK(cudaMemcpyAsync(field, mu_device, sizeof(float2) * dv.N, cudaMemcpyDeviceToDevice, s));
  DevChains none{};
  fft3d<float2>(field, v->hv.E, +1, 0, 1, v->tw_f, s, dv, none);
  double* epart = (double*)(base + NA_EPART);
  k_spectral_energy<<<NA_EBLK, 256, 0, s>>>(field, dv.sinv, dv.N, s_hr, 0, epart);
  CK_LAUNCH();
  double* dout = (double*)(base + NA_OUT);
  k_noalloc_finish<<<1, 256, 0, s>>>(epart, NA_EBLK, ch.part, NA_MAXBLK, ch.nb_w, ch.nb_wt, st, (double)dv.N, dv.n_s,
                                     dout);
  CK_LAUNCH();
  CK(cudaMemcpyAsync(out, dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  API_END
}
