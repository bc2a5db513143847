// Host runtime and C ABI of the B200-native ERTM hot path.
//
// A Prop is one propagator (reference: Propagator2D and subclasses,
// ertm/propagation.py:190-980) whose fields, CPML strips and coefficients live
// in HBM.  The whole-loop drivers (ertm_forward, ertm_migrate) run the time
// loops in C++ and only enqueue kernels, so the Python host makes one call
// per shot instead of one per time step.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cufft.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ertm_b200.h"
#include "aux_kernels.cuh"
#include "line_fft.cuh"
#include "line_fft_plan.h"
#include "step_kernels.cuh"

using namespace ertm;

namespace {

thread_local std::string g_error;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      throw Error(ERTM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)
#define CKFFT(call)                                                                          \
  do {                                                                                       \
    cufftResult r_ = (call);                                                                 \
    if (r_ != CUFFT_SUCCESS) throw Error(ERTM_ERR_CUDA, std::string(#call) + " failed"); \
  } while (0)
#define REQUIRE(cond, msg)                                   \
  do {                                                       \
    if (!(cond)) throw Error(ERTM_ERR_ARG, std::string(msg)); \
  } while (0)

template <class F>
int32_t guarded(F&& f) {
  try {
    f();
    return ERTM_OK;
  } catch (const Error& e) {
    g_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_error = e.what();
    return ERTM_ERR_STATE;
  }
}

// Instrumentation: kernel launches issued by this library, and optional
// CUDA-event timing of the stencil phases (every `every`-th step) on the
// stream they run on.
std::atomic<int64_t> g_launches{0};
struct StencilProfile {
  bool on = false;
  int every = 8;
  int64_t counter = 0;
  struct Sample {
    cudaEvent_t e0, e1;
    double bytes;
  };
  std::vector<Sample> pending;
  std::vector<cudaEvent_t> pool;
  double total_ms = 0.0, total_bytes = 0.0;
  int64_t samples = 0;
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    return e;
  }
  void drain() {
    for (auto& pr : pending) {
      float ms = 0.f;
      CK(cudaEventSynchronize(pr.e1));
      CK(cudaEventElapsedTime(&ms, pr.e0, pr.e1));
      total_ms += ms;
      total_bytes += pr.bytes;
      ++samples;
      pool.push_back(pr.e0);
      pool.push_back(pr.e1);
    }
    pending.clear();
  }
  // Bracket the stencil launches of one step or tick (every `every`-th call).
  bool begin(cudaStream_t st, cudaEvent_t& e0) {
    if (!on || (counter++ % every) != 0) return false;
    e0 = get();
    CK(cudaEventRecord(e0, st));
    return true;
  }
  void end(cudaStream_t st, cudaEvent_t e0, double bytes) {
    cudaEvent_t e1 = get();
    CK(cudaEventRecord(e1, st));
    pending.push_back({e0, e1, bytes});
  }
};
StencilProfile g_prof;

struct FftPair {
  cufftHandle fwd = 0, inv = 0;
};
std::mutex g_fft_mutex;

// Batched 1-D plans of the short-time Q filter (L-point frames, `batch` of
// them), cached by frame length, batch and stream.
std::map<std::tuple<int, int64_t, cudaStream_t>, FftPair> g_stft_plans;

FftPair stft_fft(int L, int64_t batch, cudaStream_t st) {
  std::lock_guard<std::mutex> lock(g_fft_mutex);
  auto key = std::make_tuple(L, batch, st);
  auto it = g_stft_plans.find(key);
  if (it != g_stft_plans.end()) return it->second;
  const int F = L / 2 + 1;
  int dims[1] = {L};
  FftPair p;
  CKFFT(cufftPlanMany(&p.fwd, 1, dims, nullptr, 1, L, nullptr, 1, F, CUFFT_D2Z, (int)batch));
  CKFFT(cufftPlanMany(&p.inv, 1, dims, nullptr, 1, F, nullptr, 1, L, CUFFT_Z2D, (int)batch));
  CKFFT(cufftSetStream(p.fwd, st));
  CKFFT(cufftSetStream(p.inv, st));
  g_stft_plans[key] = p;
  return p;
}

size_t round64(size_t n) { return (n + 63) / 64 * 64; }

// Grid of the record kernels: x over traces (blocks of 128), y over samples
// (at most 65535 rows of blocks; the kernels stride over the rest).
dim3 records_grid(int64_t ntr, int64_t n_samples) {
  return dim3((unsigned)((ntr + 127) / 128), (unsigned)std::min<int64_t>(std::max<int64_t>(n_samples, 1), 65535));
}

// Device allocation that frees itself (stream-ordered).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(size_t b, cudaStream_t s) : bytes(b), st(s) {
    if (b) CK(cudaMallocAsync(&p, b, s));
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    std::swap(p, o.p);
    std::swap(bytes, o.bytes);
    std::swap(st, o.st);
    return *this;
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

void upload(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st));
}

// --------------------------------------------------------------------------
// Wavenumber low-pass with NumPy's FFT arithmetic (line_fft.cuh)
// --------------------------------------------------------------------------
// Plans per device and transform length: factors and twiddles from the host
// plan; for a Bluestein length, the kernel's forward transform is computed
// once by the device passes themselves and mirrored as the library mirrors
// it (the upper half of the spectrum reuses the lower half's values).
struct LineFftPlan {
  FftPlanDev dev{};
  DevBuf tables;
};
std::map<std::pair<int, int>, std::unique_ptr<LineFftPlan>> g_line_plans;
std::mutex g_line_mutex;

constexpr size_t kLineSmemMax = 227 * 1024;       // opt-in dynamic shared memory per CTA
// Resident CTAs per SM the 256-thread line transforms are compiled for (the
// register cap follows: 3 → 80 registers; 2 → 128 registers was 3 % slower
// on 811×2011 fields, 1 → 174–200 registers 26 % slower)
constexpr int kLineNarrowMinBlocks = 3;
constexpr size_t kLineSmemWide = 113 * 1024;      // above this only one CTA fits an SM: use 512 threads
constexpr int64_t kLineScratchCtas = 296;         // CTAs of a launch whose lines do not fit in shared memory

// Launch the line transforms of J (J.plan, load, sources, lines set by the
// caller): work buffers in shared memory when they fit, else per-CTA global
// scratch; 512 threads for lines that leave one CTA per SM, 256 otherwise.
// Threads per CTA of the line transforms: 0 = chosen per transform length,
// else forced (ertm_set_line_threads).  Results do not depend on it.
std::atomic<int> g_line_threads{0};

void launch_lines(LineJob J, bool fwd, cudaStream_t st) {
  static std::mutex attr_mutex;
  static std::map<int, bool> attr_set;
  {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(attr_mutex);
    if (!attr_set[dev]) {
      const int m = (int)kLineSmemMax;
      CK(cudaFuncSetAttribute(k_fft_lines<true, 256, true, kLineNarrowMinBlocks>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<false, 256, true, kLineNarrowMinBlocks>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<true, 512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<false, 512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<true, 768, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<false, 768, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<true, 1024, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      CK(cudaFuncSetAttribute(k_fft_lines<false, 1024, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m));
      attr_set[dev] = true;
    }
  }
  const size_t smem = (size_t)2 * J.plan.n2 * sizeof(double2);
  DevBuf scratch;
  unsigned grid;
  if (smem <= kLineSmemMax) {
    J.use_smem = 1;
    grid = (unsigned)std::min<int64_t>(J.lines, 1 << 20);
  } else {
    J.use_smem = 0;
    grid = (unsigned)std::min<int64_t>(J.lines, kLineScratchCtas);
    scratch = DevBuf((size_t)grid * smem, st);
    J.scratch = scratch.as<double2>();
  }
  const bool wide = smem > kLineSmemWide;
  const int forced = g_line_threads.load();
  // one CTA per SM (wide lines): 704 threads of the 768-thread build; else
  // 256 threads, three CTAs per SM (the fastest counts on 811×2011 fields)
  const int t = !J.use_smem ? 512 : forced > 0 ? forced : wide ? 704 : 256;
  if (!J.use_smem) {
    if (fwd) k_fft_lines<true, 512, false><<<grid, t, 0, st>>>(J);
    else k_fft_lines<false, 512, false><<<grid, t, 0, st>>>(J);
  } else if (fwd) {
    if (t > 768) k_fft_lines<true, 1024, true, 1><<<grid, t, smem, st>>>(J);
    else if (t > 512) k_fft_lines<true, 768, true, 1><<<grid, t, smem, st>>>(J);
    else if (t > 256) k_fft_lines<true, 512, true><<<grid, t, smem, st>>>(J);
    else k_fft_lines<true, 256, true, kLineNarrowMinBlocks><<<grid, t, smem, st>>>(J);
  } else {
    if (t > 768) k_fft_lines<false, 1024, true, 1><<<grid, t, smem, st>>>(J);
    else if (t > 512) k_fft_lines<false, 768, true, 1><<<grid, t, smem, st>>>(J);
    else if (t > 256) k_fft_lines<false, 512, true><<<grid, t, smem, st>>>(J);
    else k_fft_lines<false, 256, true, kLineNarrowMinBlocks><<<grid, t, smem, st>>>(J);
  }
  ++g_launches;
  CK(cudaGetLastError());
}

const FftPlanDev& line_plan(int n, cudaStream_t st) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_line_mutex);
  auto it = g_line_plans.find({dev, n});
  if (it != g_line_plans.end()) return it->second->dev;
  using namespace fftplan;
  REQUIRE(n >= 1, "FFT length must be positive");
  const bool blue = use_bluestein((size_t)n);
  const size_t n2 = blue ? good_size_cmplx(2 * (size_t)n - 1) : (size_t)n;
  const CooleyTukey ct(n2);
  REQUIRE(ct.fct.size() <= (size_t)kFftMaxFactors, "FFT length has too many factors");
  std::vector<CxH> bk, kernel;
  if (blue) bluestein_chirp((size_t)n, n2, bk, kernel);
  const size_t ntw = ct.tw.size(), nbk = bk.size(), nbkf = blue ? n2 : 0;
  auto L = std::make_unique<LineFftPlan>();
  L->tables = DevBuf(std::max<size_t>(1, ntw + nbk + nbkf) * sizeof(double2), st);
  double2* tw = L->tables.as<double2>();
  upload(tw, ct.tw.data(), ntw * sizeof(double2), st);
  upload(tw + ntw, bk.data(), nbk * sizeof(double2), st);
  FftPlanDev& d = L->dev;
  d.n = n;
  d.n2 = (int)n2;
  d.blue = blue ? 1 : 0;
  d.nfact = (int)ct.fct.size();
  for (size_t f = 0; f < ct.fct.size(); ++f) {
    d.fct[f] = ct.fct[f];
    d.twoff[f] = ct.twoff[f];
    d.twsoff[f] = ct.twsoff[f];
  }
  d.tw = tw;
  d.bk = tw + ntw;
  d.bkf = tw + ntw + nbk;
  if (blue) {
    // the kernel's transform: one line through the length-n2 Cooley-Tukey plan
    FftPlanDev inner = d;
    inner.n = (int)n2;
    inner.blue = 0;
    DevBuf line(n2 * sizeof(double2), st);
    upload(line.p, kernel.data(), n2 * sizeof(double2), st);
    LineJob J{};
    J.plan = inner;
    J.load = LINE_LOAD_C;
    J.lines = 1;
    J.seg_lines = 1;
    J.nseg = 1;
    J.cbuf[0] = line.as<double2>();
    J.fct = 1.0;
    launch_lines(J, true, st);
    std::vector<CxH> spec(n2), full(n2);
    CK(cudaMemcpyAsync(spec.data(), line.p, n2 * sizeof(double2), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (size_t m = 0; m < n2; ++m) full[m] = spec[std::min(m, n2 - m)];
    upload(const_cast<double2*>(d.bkf), full.data(), n2 * sizeof(double2), st);
  }
  CK(cudaStreamSynchronize(st));
  const FftPlanDev& out = L->dev;
  g_line_plans[{dev, n}] = std::move(L);
  return out;
}

// numerics.py:424-442 on nseg arrays of shape (nz, nx): each becomes
// Re(ifft2(fft2(a) · taper)), the transforms along x then z as
// numpy.fft.fft2/ifft2 take them.  Inputs: real float32 rows of pitch
// in_pitch (padded fields) or float64 (images); outputs likewise (float32
// rounded to nearest); srcs[s] == dsts[s] is allowed.  All segments go
// through the same launches; segment s works in A[s] and B[s], nz·nx complex
// values each.
void lowpass2d(int nz, int nx, double dz, double dx, double cutoff, int nseg, const void* const* srcs, bool in_f32,
               int64_t in_pitch, void* const* dsts, bool out_f32, int64_t out_pitch, double2* const* A,
               double2* const* B, cudaStream_t st) {
  REQUIRE(nseg >= 1 && nseg <= kLineMaxSegs, "low-pass batch of 1.." + std::to_string(kLineMaxSegs) + " arrays");
  const FftPlanDev& px = line_plan(nx, st);
  const FftPlanDev& pz = line_plan(nz, st);
  const dim3 tb(32, 8);
  auto tgrid = [nseg](int rows, int cols) { return dim3((cols + 31) / 32, (rows + 31) / 32, nseg); };
  auto job = [&](const FftPlanDev& p, int load, int seg_lines, double fct, double2* const* buf) {
    LineJob J{};
    J.plan = p;
    J.load = load;
    J.seg_lines = seg_lines;
    J.nseg = nseg;
    J.lines = (int64_t)nseg * seg_lines;
    for (int k = 0; k < nseg; ++k) J.cbuf[k] = buf[k];
    J.fct = fct;
    J.dz = dz;
    J.dx = dx;
    J.cutoff = cutoff;
    return J;
  };
  auto transpose = [&](double2* const* in, void* const* out) {
    TransposeArgs T{};
    for (int k = 0; k < nseg; ++k) {
      T.in[k] = in[k];
      T.out[k] = out[k];
    }
    return T;
  };
  void* const* Av = reinterpret_cast<void* const*>(A);
  void* const* Bv = reinterpret_cast<void* const*>(B);
  LineJob rows = job(px, in_f32 ? LINE_LOAD_F32 : LINE_LOAD_F64, nz, 1.0, A);
  for (int k = 0; k < nseg; ++k) rows.src[k] = srcs[k];
  rows.src_pitch = in_pitch;
  launch_lines(rows, true, st);
  k_transpose_lines<T_COMPLEX><<<tgrid(nz, nx), tb, 0, st>>>(transpose(A, Bv), nz, nx, 0);
  launch_lines(job(pz, LINE_LOAD_C, nx, 1.0, B), true, st);
  k_transpose_lines<T_COMPLEX><<<tgrid(nx, nz), tb, 0, st>>>(transpose(B, Av), nx, nz, 0);
  launch_lines(job(px, LINE_LOAD_C_TAPER, nz, 1.0 / (double)nx, A), false, st);
  k_transpose_lines<T_COMPLEX><<<tgrid(nz, nx), tb, 0, st>>>(transpose(A, Bv), nz, nx, 0);
  launch_lines(job(pz, LINE_LOAD_C, nx, 1.0 / (double)nz, B), false, st);
  if (out_f32) k_transpose_lines<T_REAL_F32><<<tgrid(nx, nz), tb, 0, st>>>(transpose(B, dsts), nx, nz, out_pitch);
  else k_transpose_lines<T_REAL_F64><<<tgrid(nx, nz), tb, 0, st>>>(transpose(B, dsts), nx, nz, out_pitch);
  g_launches += 4;
  CK(cudaGetLastError());
}

// One array through lowpass2d.
void lowpass2d_one(int nz, int nx, double dz, double dx, double cutoff, const void* in, bool in_f32, int64_t in_pitch,
                   void* out, bool out_f32, int64_t out_pitch, double2* A, double2* B, cudaStream_t st) {
  const void* srcs[1] = {in};
  void* dsts[1] = {out};
  double2* a[1] = {A};
  double2* b[1] = {B};
  lowpass2d(nz, nx, dz, dx, cutoff, 1, srcs, in_f32, in_pitch, dsts, out_f32, out_pitch, a, b, st);
}

int comp_offsets(int comp, double& xo, double& zo) {
  // propagation.py:341-345, 380-384, 922-926
  xo = 0.0;
  zo = 0.0;
  if (comp == ERTM_COMP_VX) xo = -0.5;
  if (comp == ERTM_COMP_VZ) zo = -0.5;
  if (comp == ERTM_COMP_SXZ) { xo = -0.5; zo = -0.5; }
  return 0;
}

struct SamplePlanHost {
  int kind = SAMPLE_FIELD, slot = 0;
  DevBuf cell, valid, w;
  int n = 0;
};

struct InjectTarget {
  int slot;
  int offset_comp;   // component whose offsets apply
  int scaled;        // 0: (v·w_z)·w_x; 1: v·((w_z·w_x)·1); 2: v·((w_z·w_x)·1/|K_R|)
};

struct InjectPlanHost {
  DevBuf cell_field, cell_index, start, src, wa, wb;
  int n_cells = 0;
  InjectPlanDev dev() const {
    InjectPlanDev d{};
    d.n_cells = n_cells;
    d.cell_field = cell_field.as<int32_t>();
    d.cell_index = cell_index.as<int32_t>();
    d.start = start.as<int32_t>();
    d.src = src.as<int32_t>();
    d.wa = wa.as<double>();
    d.wb = wb.as<double>();
    return d;
  }
};

struct Prop {
  ertm_prop_config cfg{};
  DevProp h{};
  DevBuf d_desc;
  cudaStream_t st = nullptr;
  int M = 4;
  int n_psi = 2;
  size_t field_elems = 0, state_floats = 0;
  DevBuf state, coefs, prof, qidx, relax, peak, stab, status;
  int64_t step_index = 0;
  int tiles_x = 0, tiles = 0, tz = 32;
  int lowpass_steps = 0;
  bool stab_pending = false;   // after_step left the stabilisation scale to launch_epilogue
  float k_src = 0.f;             // K_R at the source node (viscoacoustic)
  std::vector<double> rx, rz;
  std::map<int, std::unique_ptr<SamplePlanHost>> samples;
  std::map<std::vector<int>, std::unique_ptr<InjectPlanHost>> injects;
  std::vector<float> host_kr;    // K_R copy for the ε-injection weights (lazy)
  size_t fe = 0;                 // field pitch in the state and coefficient blocks (floats)
  int n_coef = 0;
  mutable std::map<int, std::array<CUtensorMap, 3>> tma;   // tensor maps per tile height (see prop_tma)
  DevBuf tma_dev;                // the same maps in device memory for tile heights 8, 16, 32
  // complex work arrays of the compensated viscoacoustic low-pass (nzp·nxp each)
  DevBuf lp_a, lp_b;

  DevProp* dp() const { return d_desc.as<DevProp>(); }
  int n_fields() const { return h.n_fields; }
  float* field(int slot) const { return h.f[slot]; }
  void sync_desc() { upload(d_desc.p, &h, sizeof(DevProp), st); }
};

int field_slot(const Prop& P, int comp) {
  // component → field slot for sampling/injection, −1 if absent
  switch (P.h.engine) {
    case ENGINE_ACOUSTIC:
    case ENGINE_VISCO:
      if (comp == ERTM_COMP_P) return A_P;
      if (comp == ERTM_COMP_VX) return A_VX;
      if (comp == ERTM_COMP_VZ) return A_VZ;
      return -1;
    default:
      if (comp == ERTM_COMP_VX) return E_VX;
      if (comp == ERTM_COMP_VZ) return E_VZ;
      if (comp == ERTM_COMP_SXX) return E_SXX;
      if (comp == ERTM_COMP_SZZ) return E_SZZ;
      if (comp == ERTM_COMP_SXZ) return E_SXZ;
      return -1;
  }
}

void fractional(const Prop& P, double x, double z, double xo, double zo, double& xf, double& zf) {
  // propagation.py:251-262
  xf = (x - P.cfg.x0) / P.cfg.dx + (double)P.h.pad + xo;
  zf = (z - P.cfg.z0) / P.cfg.dz + (double)P.h.pad + zo;
}

SamplePlanHost& sample_plan(Prop& P, int comp) {
  auto it = P.samples.find(comp);
  if (it != P.samples.end()) return *it->second;
  auto sp = std::make_unique<SamplePlanHost>();
  const int n = (int)P.rx.size();
  sp->n = n;
  if (P.h.engine == ENGINE_ELASTIC && comp == ERTM_COMP_P) {
    sp->kind = SAMPLE_PRESSURE;  // ½(σxx+σzz) at the σxx node (propagation.py:891-893)
  } else if (P.h.engine == ENGINE_ACOUSTIC && comp == ERTM_COMP_SXZ) {
    sp->kind = SAMPLE_ZERO;      // propagation.py:464-466
  } else {
    sp->slot = field_slot(P, comp);
    REQUIRE(sp->slot >= 0, "propagator has no component " + std::to_string(comp));
  }
  double xo, zo;
  comp_offsets(sp->kind == SAMPLE_PRESSURE ? ERTM_COMP_SXX : comp, xo, zo);
  std::vector<int32_t> cell(n);
  std::vector<uint8_t> valid(n);
  std::vector<double> w(4 * (size_t)n);
  for (int r = 0; r < n; ++r) {
    double xf, zf;
    fractional(P, P.rx[r], P.rz[r], xo, zo, xf, zf);
    const double z0 = std::floor(zf), x0 = std::floor(xf);
    const double tz = zf - z0, tx = xf - x0;
    const long long zi = (long long)z0, xi = (long long)x0;
    valid[r] = (zi >= 0 && zi < P.h.nzp - 1 && xi >= 0 && xi < P.h.nxp - 1) ? 1 : 0;
    const long long zc = std::min<long long>(std::max<long long>(zi, 0), P.h.nzp - 2);
    const long long xc = std::min<long long>(std::max<long long>(xi, 0), P.h.nxp - 2);
    cell[r] = (int32_t)(zc * P.h.ld + xc);
    w[4 * r + 0] = 1 - tz;
    w[4 * r + 1] = tz;
    w[4 * r + 2] = 1 - tx;
    w[4 * r + 3] = tx;
  }
  sp->cell = DevBuf(n * sizeof(int32_t), P.st);
  sp->valid = DevBuf(n, P.st);
  sp->w = DevBuf(w.size() * sizeof(double), P.st);
  upload(sp->cell.p, cell.data(), n * sizeof(int32_t), P.st);
  upload(sp->valid.p, valid.data(), n, P.st);
  upload(sp->w.p, w.data(), w.size() * sizeof(double), P.st);
  CK(cudaStreamSynchronize(P.st));  // host vectors go out of scope
  auto& ref = *sp;
  P.samples[comp] = std::move(sp);
  return ref;
}

std::vector<InjectTarget> inject_targets(const Prop& P, int comp) {
  // imaging.py:437-444 maps record names to these components; the per-engine
  // field lists follow propagation.py:472-494, 764-774, 900-942.
  std::vector<InjectTarget> t;
  if (P.h.engine == ENGINE_ELASTIC) {
    if (comp == ERTM_COMP_P) {
      t.push_back({E_SXX, ERTM_COMP_SXX, 0});
      t.push_back({E_SZZ, ERTM_COMP_SXX, 0});
    } else {
      const int s = field_slot(P, comp);
      REQUIRE(s >= 0, "elastic propagator cannot inject component " + std::to_string(comp));
      t.push_back({s, comp, 0});
    }
  } else if (P.h.engine == ENGINE_VISCO) {
    const int s = field_slot(P, comp);
    REQUIRE(s >= 0, "viscoacoustic propagator cannot inject component " + std::to_string(comp));
    t.push_back({s, comp, 1});
    if (comp == ERTM_COMP_P) t.push_back({V_EPS, comp, 2});
  } else {
    const int s = field_slot(P, comp);
    REQUIRE(s >= 0, "acoustic propagator cannot inject component " + std::to_string(comp));
    t.push_back({s, comp, 0});
  }
  return t;
}

// Build the contribution lists for injecting the record components `comps`
// (record layout comps × nt × nrec).  Order inside a target cell follows the
// reference: component, then target field, then corner (00, 01, 10, 11),
// then receiver — np.add.at applies duplicates in index order.
InjectPlanHost& inject_plan(Prop& P, const std::vector<int>& comps, int64_t nt) {
  std::vector<int> key = comps;
  key.push_back((int)nt);
  auto it = P.injects.find(key);
  if (it != P.injects.end()) return *it->second;
  const int n = (int)P.rx.size();
  struct Contrib { int32_t src; double wa, wb; };
  std::map<std::pair<int, int64_t>, std::vector<Contrib>> cells;
  std::vector<std::pair<int, int64_t>> order;
  for (size_t ci = 0; ci < comps.size(); ++ci) {
    for (const InjectTarget& tg : inject_targets(P, comps[ci])) {
      if (tg.scaled == 2 && P.host_kr.empty()) {
        P.host_kr.resize(P.field_elems);
        CK(cudaMemcpyAsync(P.host_kr.data(), P.h.coef[CV_KR], P.field_elems * sizeof(float),
                           cudaMemcpyDeviceToHost, P.st));
        CK(cudaStreamSynchronize(P.st));
      }
      double xo, zo;
      comp_offsets(tg.offset_comp, xo, zo);
      std::vector<int64_t> zc(n), xc(n);
      std::vector<double> tz(n), tx(n);
      std::vector<char> ok(n);
      for (int r = 0; r < n; ++r) {
        double xf, zf;
        fractional(P, P.rx[r], P.rz[r], xo, zo, xf, zf);
        const double z0 = std::floor(zf), x0 = std::floor(xf);
        tz[r] = zf - z0;
        tx[r] = xf - x0;
        const long long zi = (long long)z0, xi = (long long)x0;
        ok[r] = (zi >= 0 && zi < P.h.nzp - 1 && xi >= 0 && xi < P.h.nxp - 1);
        zc[r] = zi;
        xc[r] = xi;
      }
      for (int corner = 0; corner < 4; ++corner) {
        const int dz = corner >> 1, dx = corner & 1;
        for (int r = 0; r < n; ++r) {
          if (!ok[r]) continue;
          const double wz = dz ? tz[r] : 1 - tz[r];
          const double wx = dx ? tx[r] : 1 - tx[r];
          Contrib c{(int32_t)(ci * nt * n + r), wz, wx};
          if (tg.scaled) {
            double fac = 1.0;  // np.float32(1.0)
            if (tg.scaled == 2) {
              const float kr = P.host_kr[(size_t)zc[r] * P.h.ld + xc[r]];
              fac = (double)(1.0f / std::max(std::fabs(kr), 1e-20f));
            }
            c.wa = wz * wx * fac;
            c.wb = 1.0;
          }
          const std::pair<int, int64_t> k{tg.slot, (zc[r] + dz) * P.h.ld + (xc[r] + dx)};
          auto& v = cells[k];
          if (v.empty()) order.push_back(k);
          v.push_back(c);
        }
      }
    }
  }
  std::vector<int32_t> cf, cidx, start{0}, src;
  std::vector<double> wa, wb;
  for (const auto& k : order) {
    cf.push_back(k.first);
    cidx.push_back((int32_t)k.second);
    for (const Contrib& c : cells[k]) {
      src.push_back(c.src);
      wa.push_back(c.wa);
      wb.push_back(c.wb);
    }
    start.push_back((int32_t)src.size());
  }
  auto ip = std::make_unique<InjectPlanHost>();
  ip->n_cells = (int)cf.size();
  auto put = [&](DevBuf& b, const void* data, size_t bytes) {
    b = DevBuf(bytes, P.st);
    upload(b.p, data, bytes, P.st);
  };
  put(ip->cell_field, cf.data(), cf.size() * 4);
  put(ip->cell_index, cidx.data(), cidx.size() * 4);
  put(ip->start, start.data(), start.size() * 4);
  put(ip->src, src.data(), src.size() * 4);
  put(ip->wa, wa.data(), wa.size() * 8);
  put(ip->wb, wb.data(), wb.size() * 8);
  CK(cudaStreamSynchronize(P.st));
  auto& ref = *ip;
  P.injects[key] = std::move(ip);
  return ref;
}

// --------------------------------------------------------------------------
// stepping
// --------------------------------------------------------------------------
// Host-side access to the works of a WorkSet1 / WorkSetN.
inline StepWork& ws_work(WorkSet1& ws, int) { return ws.w; }
inline StepWork ws_work(const WorkSet1& ws, int) { return ws.w; }
template <int N>
inline StepWork& ws_work(WorkSetN<N>& ws, int k) { return ws.w[k]; }
inline void ws_count(WorkSet1&, int) {}
template <int N>
inline void ws_count(WorkSetN<N>& ws, int n) { ws.n = n; }

template <int M, int BZ, int R, int KIND, class WS, class TM = TmaNone>
void launch_phase(int engine, int phase, const DevProp* d, const WS& ws, int blocks, cudaStream_t st,
                  const TM& tm = TM{}) {
  if (blocks <= 0) return;
  const dim3 blk(XT, BZ);
  if (phase == 0) {
    if (engine == ENGINE_ELASTIC) k_elastic_velocity<M, BZ, R, KIND, WS, TM><<<blocks, blk, 0, st>>>(d, ws, tm);
    else k_pressure_velocity<M, BZ, R, KIND, WS, TM><<<blocks, blk, 0, st>>>(d, ws, tm);
  } else {
    if (engine == ENGINE_ACOUSTIC)
      k_pressure_stress<M, BZ, R, false, KIND, WS, TM><<<blocks, blk, 0, st>>>(d, ws, tm);
    else if (engine == ENGINE_VISCO)
      k_pressure_stress<M, BZ, R, true, KIND, WS, TM><<<blocks, blk, 0, st>>>(d, ws, tm);
    else k_elastic_stress<M, BZ, R, KIND, WS, TM><<<blocks, blk, 0, st>>>(d, ws, tm);
  }
  ++g_launches;
}

// Tensor maps of a propagator for tile height tz (TMA staging of interior
// tiles): the state block as a 3-D tensor (ld × nzp × fields, pitches ld and
// fe floats — both multiples of 16 bytes) with a 40 × (tz+8) halo box and a
// 32 × tz cell box, and the coefficient block with a cell box.  Encoded once
// per (propagator, tz); the buffers never move.
PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    REQUIRE(q == cudaDriverEntryPointSuccess && p, "cuTensorMapEncodeTiled is not available");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

const std::array<CUtensorMap, 3>& prop_tma(const Prop& P, int tz) {
  auto it = P.tma.find(tz);
  if (it != P.tma.end()) return it->second;
  std::array<CUtensorMap, 3> m{};
  const cuuint64_t ld = (cuuint64_t)P.h.ld, nzp = (cuuint64_t)P.h.nzp;
  const cuuint64_t strides[2] = {ld * 4, (cuuint64_t)P.fe * 4};
  const cuuint32_t halo[3] = {(cuuint32_t)(TILE_X + 8), (cuuint32_t)(tz + 2 * P.M), 1};
  const cuuint32_t cell[3] = {(cuuint32_t)TILE_X, (cuuint32_t)tz, 1};
  const cuuint32_t unit[3] = {1, 1, 1};
  const cuuint64_t dims_state[3] = {ld, nzp, (cuuint64_t)P.h.n_fields};
  const cuuint64_t dims_coef[3] = {ld, nzp, (cuuint64_t)P.n_coef};
  auto enc = [&](CUtensorMap* out, void* base, const cuuint64_t* dims, const cuuint32_t* box) {
    const CUresult r = tma_encode_fn()(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, unit,
                                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                       CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    REQUIRE(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  };
  enc(&m[0], P.state.p, dims_state, halo);
  enc(&m[1], P.state.p, dims_state, cell);
  enc(&m[2], P.coefs.p, dims_coef, cell);
  return P.tma.emplace(tz, m).first->second;
}

// Stage interior tiles with TMA (1) or cp.async (0).  Measured on the batched
// elastic tick: cp.async 72.7 µs, TMA with tensor maps in device memory
// 87.2 µs (with maps in the kernel parameters 78.9 µs), so cp.async is the
// default; the TMA path is kept, tested and selectable.
std::atomic<int> g_tma{0};


template <int M, int BZ, int R, class WS>
void launch_step_shape(int engine, const DevProp* d, const WS& ws, int blocks, cudaStream_t st) {
  launch_phase<M, BZ, R, TILES_ALL>(engine, 0, d, ws, blocks, st);
  launch_phase<M, BZ, R, TILES_ALL>(engine, 1, d, ws, blocks, st);
}

// A second stream (per device) and fork/join events for the boundary-tile
// launches, so that they run beside the interior launches.
struct SplitStreams {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// Per device: stream pairs for the lanes of a batched tick (lane 0 runs on
// the caller's stream; lane k > 0 on its own stream) and, per lane, the side
// stream of its boundary-frame launches.
constexpr int kLanes = 4;
struct LaneStreams {
  SplitStreams split[kLanes];          // frame-launch side streams, per lane
  cudaStream_t lane[kLanes] = {};      // lane streams (lane[0] unused: the caller's)
  cudaEvent_t fork[kLanes] = {}, join[kLanes] = {};
};

LaneStreams& lane_streams() {
  static std::mutex mu;
  static std::map<int, LaneStreams> per_device;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  LaneStreams& s = per_device[dev];
  if (!s.split[0].side) {
    for (int k = 0; k < kLanes; ++k) {
      CK(cudaStreamCreateWithFlags(&s.split[k].side, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&s.split[k].fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&s.split[k].join, cudaEventDisableTiming));
      if (k > 0) CK(cudaStreamCreateWithFlags(&s.lane[k], cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&s.fork[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&s.join[k], cudaEventDisableTiming));
    }
  }
  return s;
}

SplitStreams& split_streams(int lane = 0) { return lane_streams().split[lane]; }

// Interior tiles in their own launches: the straight-line kernels then carry
// none of the boundary code's registers (more resident warps per SM).  The
// boundary-frame launch of each phase runs on the side stream, concurrently
// with the interior launch; the two join before the next phase.
// Elastic velocity phase of 32-row interiors: 0 tiles; 2, 4 or 8 marching
// column strips in segments of at most that many 16-row chunks (4: measured
// fastest on the benchmark job, tick 78.3 → 75.9 µs).
std::atomic<int> g_march{4};
// Elastic stress phase of 32-row interiors marching as well (same segments): 0 off, 1 on.
std::atomic<int> g_march_stress{0};

// The frame launch may use a lower tile (BZF × RF rows) than the interior one:
// more, shorter blocks for the boundary work.
template <int M, int BZ, int R, int BZF = BZ, int RF = R, class WS>
void launch_step_split(int engine, const DevProp* d, const WS& inner, int n_in, const WS& frame, int n_fr,
                       cudaStream_t st, int lane, const TmaGlobal* tm, const WS* march = nullptr, int n_march = 0) {
  SplitStreams& ss = split_streams(lane);
  for (int phase = 0; phase < 2; ++phase) {
    CK(cudaEventRecord(ss.fork, st));
    CK(cudaStreamWaitEvent(ss.side, ss.fork, 0));
    launch_phase<M, BZF, RF, TILES_FRAME>(engine, phase, d, frame, n_fr, ss.side);
    if (phase == 0 && march) {
      if constexpr (M == 4) {
        if (n_march > 0) {
          const int seg = g_march.load();
          if (seg == 2) k_elastic_velocity_march<M, 2, WS><<<n_march, dim3(XT, MARCH_CH), 0, st>>>(d, *march);
          else if (seg == 4) k_elastic_velocity_march<M, 4, WS><<<n_march, dim3(XT, MARCH_CH), 0, st>>>(d, *march);
          else k_elastic_velocity_march<M, 8, WS><<<n_march, dim3(XT, MARCH_CH), 0, st>>>(d, *march);
          ++g_launches;
        }
      }
    } else if (phase == 1 && march && g_march_stress.load() == 1) {
      if constexpr (M == 4) {
        if (n_march > 0) {
          const int seg = g_march.load();
          if (seg == 2) k_elastic_stress_march<M, 2, WS><<<n_march, dim3(XT, MARCH_CH), 0, st>>>(d, *march);
          else if (seg == 4) k_elastic_stress_march<M, 4, WS><<<n_march, dim3(XT, MARCH_CH), 0, st>>>(d, *march);
          else k_elastic_stress_march<M, 8, WS><<<n_march, dim3(XT, MARCH_CH), 0, st>>>(d, *march);
          ++g_launches;
        }
      }
    } else if (tm) {
      launch_phase<M, BZ, R, TILES_INTERIOR>(engine, phase, d, inner, n_in, st, *tm);
    } else {
      launch_phase<M, BZ, R, TILES_INTERIOR>(engine, phase, d, inner, n_in, st);
    }
    CK(cudaEventRecord(ss.join, ss.side));
    CK(cudaStreamWaitEvent(st, ss.join, 0));
  }
}

// Both phases of one step for every work in ws (one tile height for all):
// TZ 8 = 8×8 threads, 16 = 8×16 threads, 32 = 8×16 threads × 2 rows.
template <class WS>
void launch_step(int M, int tz, int engine, const DevProp* d, const WS& ws, int blocks, cudaStream_t st) {
  if (M == 4) {
    if (tz == 32) launch_step_shape<4, 16, 2>(engine, d, ws, blocks, st);
    else if (tz == 16) launch_step_shape<4, 16, 1>(engine, d, ws, blocks, st);
    else launch_step_shape<4, 8, 1>(engine, d, ws, blocks, st);
  } else if (M == 3) {
    launch_step_shape<3, 16, 1>(engine, d, ws, blocks, st);
  } else if (M == 2) {
    launch_step_shape<2, 16, 1>(engine, d, ws, blocks, st);
  } else {
    launch_step_shape<1, 16, 1>(engine, d, ws, blocks, st);
  }
}

// The interior rectangle of a work for tile height tz, as Geo::interior
// decides it tile by tile: physical, clear of every CPML strip, below the
// free-surface row, with the verified float64-product division; the source
// node's tile becomes the hole.  Returns the number of interior tiles.
int plan_interior(const DevProp& h, int tz, StepWork& w) {
  w.ti0 = w.ti1 = w.tj0 = w.tj1 = 0;
  w.hole_i = w.hole_j = -1;
  if (!(h.fast_x == 1 && h.fast_z == 1)) return 0;
  const int lo_i = std::max(std::max(h.pad, h.npz_t), h.free_surface ? h.pad + 1 : 0);
  const int hi_i = std::min(h.pad + h.nz, h.nzp - h.npz_b);
  const int lo_j = std::max(h.pad, h.npx_l);
  const int hi_j = std::min(h.pad + h.nx, h.nxp - h.npx_r);
  const int ti0 = (lo_i + tz - 1) / tz, ti1 = hi_i / tz;
  const int tj0 = (lo_j + TILE_X - 1) / TILE_X, tj1 = hi_j / TILE_X;
  if (ti1 <= ti0 || tj1 <= tj0) return 0;
  w.ti0 = ti0;
  w.ti1 = ti1;
  w.tj0 = tj0;
  w.tj1 = tj1;
  int n = (ti1 - ti0) * (tj1 - tj0);
  if (h.src_iz >= 0) {
    const int si = h.src_iz / tz, sj = h.src_ix / TILE_X;
    if (si >= ti0 && si < ti1 && sj >= tj0 && sj < tj1) {
      w.hole_i = si;
      w.hole_j = sj;
      --n;
    }
  }
  return n;
}

// Split launches (twice the launches, a fork and a join per phase) pay off
// once the interior tiles alone fill the GPU several times over; below that
// (a single 401×601 grid, say) the single launch per phase is faster.
constexpr int64_t kSplitMinTiles = 148 * 16;
std::atomic<int> g_tile_split{0};   // 0 automatic, 1 never, 2 whenever there are interior tiles
std::atomic<int> g_frame_rows{0};   // frame tile height in split launches: 0 as the interior's, or 8 / 16
// Blocks of the marching velocity launch for an interior rectangle planned in
// 32-row tiles: strips × segments of at most seg 16-row chunks (the kernel's
// march_loc splits the same way).
int march_blocks(const StepWork& w, int seg) {
  const int chunks = 2 * (w.ti1 - w.ti0);
  const int nseg = (chunks + seg - 1) / seg;
  return (w.tj1 - w.tj0) * nseg;
}

// A frame work in tiles of tzf rows around an interior rectangle planned in
// tiles of tz rows (tz a multiple of tzf): the rectangle's rows and the hole
// scale by q = tz / tzf, and the hole becomes q frame tiles (the frame kernel
// numbers them after the side columns).  Returns the frame tile count.
int frame_work(const DevProp& h, int tz, int tzf, int interior_tiles, StepWork& b) {
  const int q = tz / tzf;
  b.tiles = ((h.nxp + TILE_X - 1) / TILE_X) * ((h.nzp + tzf - 1) / tzf);
  b.ti0 *= q;
  b.ti1 *= q;
  if (b.hole_i >= 0) b.hole_i *= q;
  return b.tiles - q * interior_tiles;
}

// One step of the works ws.w[0..n) (tile heights tz; tile0/tiles/tiles_x set):
// split into interior and boundary launches where that pays, else one launch
// per phase over every tile.
template <class WS>
void launch_works(int M, int tz, int engine, const DevProp* d, WS& ws, int n, const Prop* const* hosts,
                  cudaStream_t st, int lane = 0, int split_mode = -1) {
  int total = 0;
  for (int k = 0; k < n; ++k) total += ws_work(ws, k).tiles;
  if (split_mode < 0) split_mode = g_tile_split.load();
  if (split_mode != 1 && M == 4) {
    WS inner = ws, frame = ws;
    int n_in = 0, n_fr = 0, ki = 0, kf = 0;
    const Prop* inner_props[MAX_BATCH_WORKS];
    const int fr = g_frame_rows.load();
    const int tzf = (fr == 8 || fr == 16) && fr < tz ? fr : tz;
    for (int k = 0; k < n; ++k) {
      StepWork w = ws_work(ws, k);
      const int in = plan_interior(hosts[k]->h, tz, w);
      if (in > 0) {
        StepWork a = w;
        a.tile0 = n_in;
        a.slot = ki;
        inner_props[ki] = hosts[k];
        ws_work(inner, ki++) = a;
        n_in += in;
      }
      StepWork b = w;
      b.tile0 = n_fr;
      ws_work(frame, kf) = b;
      n_fr += frame_work(hosts[k]->h, tz, tzf, in, ws_work(frame, kf));
      ++kf;
    }
    if (n_in > 0 && (n_in >= kSplitMinTiles || split_mode == 2)) {
      ws_count(inner, ki);
      ws_count(frame, kf);
      // TMA staging when every interior work has its tensor maps on the device
      static const TmaGlobal tm_global{};
      bool maps = g_tma.load() != 0;
      for (int k = 0; k < ki && maps; ++k) maps = inner_props[k]->h.tmap != nullptr;
      const TmaGlobal* tm = maps ? &tm_global : nullptr;
      // the elastic velocity phase of 32-row interiors may march down column strips
      WS march = inner;
      int n_march = 0;
      const int seg = g_march.load();
      const bool use_march = seg != 0 && engine == ENGINE_ELASTIC && tz == 32 && !tm;
      if (use_march) {
        for (int k = 0; k < ki; ++k) {
          StepWork& m = ws_work(march, k);
          m.tile0 = n_march;
          n_march += march_blocks(m, seg);
        }
      }
      const WS* mp = use_march ? &march : nullptr;
      if (tz == 32 && tzf == 8)
        launch_step_split<4, 16, 2, 8, 1>(engine, d, inner, n_in, frame, n_fr, st, lane, tm, mp, n_march);
      else if (tz == 32 && tzf == 16)
        launch_step_split<4, 16, 2, 16, 1>(engine, d, inner, n_in, frame, n_fr, st, lane, tm, mp, n_march);
      else if (tz == 32) launch_step_split<4, 16, 2>(engine, d, inner, n_in, frame, n_fr, st, lane, tm, mp, n_march);
      else if (tz == 16 && tzf == 8) launch_step_split<4, 16, 1, 8, 1>(engine, d, inner, n_in, frame, n_fr, st, lane, tm);
      else if (tz == 16) launch_step_split<4, 16, 1>(engine, d, inner, n_in, frame, n_fr, st, lane, tm);
      else launch_step_split<4, 8, 1>(engine, d, inner, n_in, frame, n_fr, st, lane, tm);
      return;
    }
  }
  launch_step(M, tz, engine, d, ws, total, st);
}

// Division mode for a grid spacing h (see divh): the cheapest form that the
// device reproduces __fdiv_rn(a, h) with for all 2^32 inputs, checked once per
// float value of h and cached for the process.
std::map<uint32_t, int> g_div_mode;
std::mutex g_div_mutex;

// Reciprocal pieces of a spacing: RN64(1/h), RN32(1/h) and RN32(1/h − RN32(1/h))
// (the last from the float64 difference, accurate to far below one ulp of it).
void reciprocals(float h, double& r64, float& r32, float& rl) {
  r64 = 1.0 / (double)h;               // IEEE double division on the host
  r32 = 1.0f / h;                      // IEEE single division on the host
  rl = (float)(r64 - (double)r32);
}

unsigned long long division_mismatches(float h, int mode, cudaStream_t st) {
  double r64;
  float r32, rl;
  reciprocals(h, r64, r32, rl);
  DevBuf bad(8, st);
  CK(cudaMemsetAsync(bad.p, 0, 8, st));
  k_verify_division<<<148 * 8, 256, 0, st>>>(h, r64, r32, rl, mode, bad.as<unsigned long long>());
  ++g_launches;
  CK(cudaGetLastError());
  unsigned long long n = 1;
  CK(cudaMemcpyAsync(&n, bad.p, 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return n;
}

int division_mode(float h, cudaStream_t st) {
  uint32_t key;
  std::memcpy(&key, &h, 4);
  {
    std::lock_guard<std::mutex> lock(g_div_mutex);
    auto it = g_div_mode.find(key);
    if (it != g_div_mode.end()) return it->second;
  }
  int mode = 0;
  for (int m : {1, 3, 2}) {
    if (division_mismatches(h, m, st) == 0) {
      mode = m;
      break;
    }
  }
  std::lock_guard<std::mutex> lock(g_div_mutex);
  g_div_mode[key] = mode;
  return mode;
}

// Tile height for a launch: the tallest tile that still gives ≥ 4 blocks per
// SM, unless the autotuner pinned one (ertm_set_tile_rows).
std::atomic<int> g_tile_rows{0};
int choose_tz(int M, int nxp, int64_t rows_total_tiles32, int64_t rows16, int64_t rows8) {
  (void)nxp;
  (void)rows8;
  if (M != 4) return 16;
  const int forced = g_tile_rows.load();
  if (forced == 8 || forced == 16 || forced == 32) return forced;
  // 16-row tiles measured fastest for batched ticks and for most single grids;
  // 8-row tiles when 16 rows would leave fewer than four blocks per SM.
  (void)rows_total_tiles32;
  const int64_t want = 148 * 4;
  if (rows16 >= want) return 16;
  return 8;
}

int tiles_for(const DevProp& h, int tz) { return ((h.nxp + TILE_X - 1) / TILE_X) * ((h.nzp + tz - 1) / tz); }

template <int M>
void launch_epilogue_M(const Prop& P, const Epilogue& E);

// The compensated viscoacoustic low-pass (propagation.py:744-749): p and ε
// of every propagator in `items`, in place, each with its cutoff at this
// step.  Propagators of the same padded grid, spacing and cutoff share the
// launches (two segments each); each keeps its own complex work arrays.
struct LowpassItem {
  Prop* P;
  double cutoff;
};

void lowpass_props(const std::vector<LowpassItem>& items, cudaStream_t st) {
  std::map<std::tuple<int, int, double, double, double>, std::vector<Prop*>> groups;
  for (const LowpassItem& it : items)
    groups[std::make_tuple(it.P->h.nzp, it.P->h.nxp, it.P->cfg.dz, it.P->cfg.dx, it.cutoff)].push_back(it.P);
  for (auto& kv : groups) {
    const int nz = std::get<0>(kv.first), nx = std::get<1>(kv.first);
    const size_t cells = (size_t)nz * nx;
    const std::vector<Prop*>& props = kv.second;
    for (size_t c0 = 0; c0 < props.size(); c0 += kLineMaxSegs / 2) {
      std::vector<const void*> srcs;
      std::vector<void*> dsts;
      std::vector<double2*> A, B;
      for (size_t k = c0; k < std::min(props.size(), c0 + kLineMaxSegs / 2); ++k) {
        Prop& P = *props[k];
        if (!P.lp_a.p) {
          P.lp_a = DevBuf(2 * cells * sizeof(double2), P.st);
          P.lp_b = DevBuf(2 * cells * sizeof(double2), P.st);
        }
        const int fields[2] = {V_P, V_EPS};
        for (int f = 0; f < 2; ++f) {
          srcs.push_back(P.field(fields[f]));
          dsts.push_back(P.field(fields[f]));
          A.push_back(P.lp_a.as<double2>() + f * cells);
          B.push_back(P.lp_b.as<double2>() + f * cells);
        }
      }
      const Prop& P0 = *props[c0];
      lowpass2d(nz, nx, P0.cfg.dz, P0.cfg.dx, std::get<4>(kv.first), (int)srcs.size(), srcs.data(), true, P0.h.ld,
                dsts.data(), true, P0.h.ld, A.data(), B.data(), st);
    }
  }
}

// Algorithmic HBM bytes of one propagator step: each state array read and
// written once, each per-cell coefficient read once, CPML strips read and
// written (the viscoacoustic a_l count as per-cell coefficients although
// they are read from a per-Q table here).
double step_bytes(const Prop& P) {
  const double npad = (double)P.h.nzp * P.h.nxp;
  const int n_state = P.h.n_fields;
  const int n_coef = P.h.engine == ENGINE_ACOUSTIC ? 3 : (P.h.engine == ENGINE_ELASTIC ? 5 : 3 + 2 * P.h.L);
  const double strips = (double)P.n_psi * ((double)P.h.wx * P.h.nzp + (double)P.h.hz_rows * P.h.nxp);
  return npad * (8.0 * n_state + 4.0 * n_coef) + 8.0 * strips;
}

// Algorithmic bytes of a fused epilogue over the physical cells: each
// imaging accumulator is read and written once per step, 16 B; the replayed
// source field is written once and read once, 4 B each.
double epilogue_bytes(const Epilogue& e, size_t npix) {
  double per = 0.0;
  switch (e.kind) {
    case EPI_STORE:
      per = 4.0 * ((e.out[0] ? 1 : 0) + (e.out[1] ? 1 : 0));
      break;
    case EPI_IMAGE:
      for (int k = 0; k < e.n_images; ++k) {
        if (e.cross) per += 16.0;
        if (e.illum && e.ill[k]) per += 16.0;
        if (e.rillum && e.ril[k]) per += 16.0;
      }
      per += 4.0 * ((e.src[0] ? 1 : 0) + (e.src[1] ? 1 : 0));
      break;
    case EPI_EXC_TRACK:
      per = 8.0;   // running |P| read and (when larger) written
      break;
    case EPI_EXC_IMAGE:
      per = 4.0;   // peak-step read; the few matching cells add 24 B each
      break;
    default:
      break;
  }
  return per * (double)npix;
}

// The StepWork of one step.  Amplitude: wavelet[t] from device memory when
// `wave` is given, else amp64 (float32 for the field, float32(amp64/K_R) for
// the viscoacoustic strain).  `epi` is fused into the stress phase.
StepWork make_work(const Prop& P, double amp64, const float* wave, int t, const Epilogue* epi) {
  StepWork w{};
  w.prop = 0;
  w.tile0 = 0;
  w.tiles_x = P.tiles_x;
  w.tiles = P.tiles;
  w.wavelet = wave;
  w.t = t;
  if (!wave) {
    // `if source_amplitude != 0.0` on the float64 value, then float32 adds
    w.amp = amp64 != 0.0 ? (float)amp64 : 0.f;
    if (P.h.engine == ENGINE_VISCO && amp64 != 0.0) w.amp_eps = (float)(amp64 / (double)P.k_src);
  }
  const bool comp = P.h.engine == ENGINE_VISCO && P.cfg.compensation;
  w.flags = comp ? STEP_PEAK : 0;
  if (epi) w.epi = *epi;
  return w;
}

// What follows the stress phase of a step: the force_z source on vz, the
// compensated viscoacoustic amplitude cap / low-pass (propagation.py:726-749,
// evaluated with the step index before its increment), and the increment.
// With `defer`, a low-pass due at this step is appended there for the
// caller to run (together with other propagators' low-passes) before
// anything reads the fields again; otherwise it runs here.
// fuse_stab: the caller launches this propagator's stand-alone epilogue
// next (launch_epilogue), so on a step without a low-pass the stabilisation
// scale is left pending and runs inside that launch.
void after_step(Prop& P, double amp64, const float* wave, int t, std::vector<LowpassItem>* defer = nullptr,
                bool fuse_stab = false) {
  const bool force_z = P.h.engine == ENGINE_ELASTIC && P.h.mech == MECH_FORCE_Z && P.h.src_iz >= 0;
  if (force_z && (wave || amp64 != 0.0)) {
    const int64_t idx = (int64_t)P.h.src_iz * P.h.ld + P.h.src_ix;
    if (wave) k_point_add_wave<<<1, 32, 0, P.st>>>(P.field(E_VZ), idx, wave, t);
    else k_point_add<<<1, 32, 0, P.st>>>(P.field(E_VZ), idx, (float)amp64);
    ++g_launches;
  }
  if (P.h.engine == ENGINE_VISCO && P.cfg.compensation) {
    const int64_t s = P.step_index;
    const int every = P.cfg.lowpass_interval;
    const bool lowpass = s >= 30 && every > 1 && s % every == 0;
    if (s < 30) {
      k_stab_reference<<<1, 32, 0, P.st>>>(P.dp(), 0, P.stab.as<StabState>());
      ++g_launches;
    } else if (fuse_stab && !lowpass) {
      P.stab_pending = true;
    } else {
      k_stab_scale<<<296, 256, 0, P.st>>>(P.dp(), 0, P.stab.as<StabState>(), P.cfg.amplitude_cap);
      ++g_launches;
      if (lowpass) {
        ++P.lowpass_steps;
        const double time = (double)s * P.cfg.dt;
        const double ratio = std::max(0.9 - 0.4 * std::min(time / 1.0, 1.0), 0.35);
        if (defer) defer->push_back({&P, ratio});
        else lowpass_props({{&P, ratio}}, P.st);
      }
    }
  }
  CK(cudaGetLastError());
  ++P.step_index;
}

void step_once(Prop& P, double amp64, const float* wave = nullptr, int t = 0, const Epilogue* epi = nullptr,
               bool fuse_stab = false) {
  WorkSet1 ws{make_work(P, amp64, wave, t, epi)};
  cudaEvent_t e0 = nullptr;
  const bool timed = g_prof.begin(P.st, e0);
  const Prop* hosts[1] = {&P};
  launch_works(P.M, P.tz, P.h.engine, P.dp(), ws, 1, hosts, P.st);
  if (timed) g_prof.end(P.st, e0, step_bytes(P) + (epi ? epilogue_bytes(*epi, (size_t)P.h.nz * P.h.nx) : 0.0));
  after_step(P, amp64, wave, t, nullptr, fuse_stab);
}

void image_field(Prop& P, int wave, int sep, float* out) {
  const dim3 b2(32, 8), g2((P.h.nx + 31) / 32, (P.h.nz + 7) / 8);
  ++g_launches;
  switch (P.M) {
    case 1: k_image_field<1><<<g2, b2, 0, P.st>>>(P.dp(), 0, wave, sep, out); break;
    case 2: k_image_field<2><<<g2, b2, 0, P.st>>>(P.dp(), 0, wave, sep, out); break;
    case 3: k_image_field<3><<<g2, b2, 0, P.st>>>(P.dp(), 0, wave, sep, out); break;
    default: k_image_field<4><<<g2, b2, 0, P.st>>>(P.dp(), 0, wave, sep, out); break;
  }
}

Prop* create(const ertm_prop_config* cfg, const float* vp, const float* vs, const float* rho,
             const float* ax, const float* bx, const float* az, const float* bz, const uint8_t* qidx,
             const double* tau, const double* delta, const double* mref, const float* relax_a, void* stream) {
  REQUIRE(cfg, "null config");
  REQUIRE(cfg->order == 2 || cfg->order == 4 || cfg->order == 6 || cfg->order == 8, "order must be 2/4/6/8");
  REQUIRE(cfg->nx >= 2 && cfg->nz >= 2, "grid must be at least 2x2");
  REQUIRE(cfg->engine >= 0 && cfg->engine <= 2, "unknown engine");
  REQUIRE(vp && rho && ax && bx && az && bz, "null material or profile array");
  auto P = std::make_unique<Prop>();
  P->cfg = *cfg;
  P->st = static_cast<cudaStream_t>(stream);
  DevProp& h = P->h;
  h.engine = cfg->engine;
  h.M = cfg->order / 2;
  P->M = h.M;
  h.pad = h.M + 1;
  h.nz = cfg->nz;
  h.nx = cfg->nx;
  h.nzp = cfg->nz + 2 * h.pad;
  h.nxp = cfg->nx + 2 * h.pad;
  REQUIRE(h.nzp > 2 * h.M && h.nxp > 2 * h.M, "grid too small for the stencil");
  h.ld = (h.nxp + 31) / 32 * 32;
  static const double C8[4][4] = {{1.0, 0, 0, 0},
                                  {9.0 / 8.0, -1.0 / 24.0, 0, 0},
                                  {75.0 / 64.0, -25.0 / 384.0, 3.0 / 640.0, 0},
                                  {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0}};
  for (int k = 0; k < 4; ++k) h.c[k] = (float)C8[h.M - 1][k];
  h.hx = (float)cfg->dx;
  h.hz = (float)cfg->dz;
  h.dt = (float)cfg->dt;
  h.rx = 1.0 / (double)h.hx;
  h.rz = 1.0 / (double)h.hz;
  {
    double d;
    reciprocals(h.hx, d, h.rx32, h.rxl);
    reciprocals(h.hz, d, h.rz32, h.rzl);
  }
  h.fast_x = division_mode(h.hx, P->st);
  h.fast_z = division_mode(h.hz, P->st);
  h.npx_l = cfg->npml_x_left;
  h.npx_r = cfg->npml_x_right;
  h.npz_t = cfg->npml_z_top;
  h.npz_b = cfg->npml_z_bottom;
  REQUIRE(h.npx_l >= 0 && h.npx_r >= 0 && h.npx_l + h.npx_r <= h.nxp, "bad x strips");
  REQUIRE(h.npz_t >= 0 && h.npz_b >= 0 && h.npz_t + h.npz_b <= h.nzp, "bad z strips");
  h.wx = h.npx_l + h.npx_r;
  h.hz_rows = h.npz_t + h.npz_b;
  h.free_surface = (cfg->free_surface && h.engine != ENGINE_VISCO) ? 1 : 0;
  h.src_iz = h.src_ix = -1;
  h.L = h.engine == ENGINE_VISCO ? cfg->n_mech : 0;
  if (h.engine == ENGINE_VISCO) {
    REQUIRE(h.L >= 1 && h.L <= MAX_MECH, "n_mech must be 1..8");
    REQUIRE(cfg->n_q >= 1 && cfg->n_q <= 255, "n_q must be 1..255");
    REQUIRE(qidx && tau && delta && mref && relax_a, "viscoacoustic tables missing");
  }
  if (h.engine == ENGINE_ELASTIC) REQUIRE(vs, "elastic needs vs");
  h.n_fields = h.engine == ENGINE_ACOUSTIC ? 3 : (h.engine == ENGINE_ELASTIC ? 5 : 4 + h.L);
  P->n_psi = h.engine == ENGINE_ELASTIC ? 4 : 2;
  const int n_coef = h.engine == ENGINE_ACOUSTIC ? 3 : (h.engine == ENGINE_ELASTIC ? 5 : 3 + h.L);
  P->field_elems = (size_t)h.nzp * h.ld;
  const size_t fe = round64(P->field_elems);
  P->fe = fe;
  const size_t px = round64((size_t)h.nzp * h.wx), pz = round64((size_t)h.hz_rows * h.ld);
  P->state_floats = fe * h.n_fields + P->n_psi * (px + pz);
  P->state = DevBuf(P->state_floats * 4, P->st);
  CK(cudaMemsetAsync(P->state.p, 0, P->state_floats * 4, P->st));
  float* s = P->state.as<float>();
  for (int f = 0; f < h.n_fields; ++f) h.f[f] = s + f * fe;
  for (int t = 0; t < P->n_psi; ++t) {
    h.psix[t] = s + fe * h.n_fields + t * px;
    h.psiz[t] = s + fe * h.n_fields + P->n_psi * px + t * pz;
  }
  P->coefs = DevBuf(fe * n_coef * 4, P->st);
  P->n_coef = n_coef;
  CK(cudaMemsetAsync(P->coefs.p, 0, fe * n_coef * 4, P->st));
  for (int c = 0; c < n_coef; ++c) h.coef[c] = P->coefs.as<float>() + c * fe;
  P->prof = DevBuf((2 * (size_t)h.nxp + 2 * (size_t)h.nzp) * 4, P->st);
  float* pr = P->prof.as<float>();
  upload(pr, ax, h.nxp * 4, P->st);
  upload(pr + h.nxp, bx, h.nxp * 4, P->st);
  upload(pr + 2 * h.nxp, az, h.nzp * 4, P->st);
  upload(pr + 2 * h.nxp + h.nzp, bz, h.nzp * 4, P->st);
  h.ax = pr;
  h.bx = pr + h.nxp;
  h.az = pr + 2 * h.nxp;
  h.bz = pr + 2 * h.nxp + h.nzp;
  P->peak = DevBuf(64, P->st);
  CK(cudaMemsetAsync(P->peak.p, 0, 64, P->st));
  h.peak = P->peak.as<float>();
  P->status = DevBuf(sizeof(uint32_t), P->st);
  CK(cudaMemsetAsync(P->status.p, 0, sizeof(uint32_t), P->st));
  h.status = P->status.as<uint32_t>();
  P->stab = DevBuf(sizeof(StabState), P->st);
  CK(cudaMemsetAsync(P->stab.p, 0, sizeof(StabState), P->st));
  DevBuf tables;
  if (h.engine == ENGINE_VISCO) {
    // per-cell Q index on the padded grid (host layout nzp × nxp → pitch ld)
    P->qidx = DevBuf(P->field_elems, P->st);
    CK(cudaMemsetAsync(P->qidx.p, 0, P->field_elems, P->st));
    CK(cudaMemcpy2DAsync(P->qidx.p, h.ld, qidx, h.nxp, h.nxp, h.nzp, cudaMemcpyDefault, P->st));
    h.qidx = P->qidx.as<uint8_t>();
    const size_t nqL = (size_t)cfg->n_q * h.L;
    P->relax = DevBuf(nqL * 4, P->st);
    upload(P->relax.p, relax_a, nqL * 4, P->st);
    h.relax_a = P->relax.as<float>();
    tables = DevBuf((2 * nqL + cfg->n_q) * 8, P->st);
    upload(tables.as<double>(), tau, nqL * 8, P->st);
    upload(tables.as<double>() + nqL, delta, nqL * 8, P->st);
    upload(tables.as<double>() + 2 * nqL, mref, cfg->n_q * 8, P->st);
  }
  // physical materials → device
  const size_t nphys = (size_t)cfg->nz * cfg->nx;
  DevBuf mat(nphys * 3 * 4, P->st);
  upload(mat.as<float>(), vp, nphys * 4, P->st);
  upload(mat.as<float>() + nphys, rho, nphys * 4, P->st);
  if (vs) upload(mat.as<float>() + 2 * nphys, vs, nphys * 4, P->st);
  // tensor maps for TMA staging of interior tiles (order 8), in device memory
  h.tmap = nullptr;
  if (P->M == 4 && g_tma.load()) {
    std::array<CUtensorMap, 9> all{};
    for (int k = 0; k < 3; ++k) {
      const std::array<CUtensorMap, 3>& m = prop_tma(*P, 8 << k);
      for (int q = 0; q < 3; ++q) all[3 * k + q] = m[q];
    }
    P->tma_dev = DevBuf(sizeof(all), P->st);
    upload(P->tma_dev.p, all.data(), sizeof(all), P->st);
    h.tmap = P->tma_dev.p;
  }
  P->d_desc = DevBuf(sizeof(DevProp), P->st);
  P->sync_desc();
  SetupArgs A{};
  A.vp = mat.as<float>();
  A.rho = mat.as<float>() + nphys;
  A.vs = mat.as<float>() + 2 * nphys;
  if (h.engine == ENGINE_VISCO) {
    const size_t nqL = (size_t)cfg->n_q * h.L;
    A.tau = tables.as<double>();
    A.delta = tables.as<double>() + nqL;
    A.mref = tables.as<double>() + 2 * nqL;
    A.relax_a = h.relax_a;
  }
  A.dt = cfg->dt;
  const dim3 b2(32, 8), g2((h.nxp + 31) / 32, (h.nzp + 7) / 8);
  k_setup_materials<<<g2, b2, 0, P->st>>>(P->dp(), 0, A);
  CK(cudaGetLastError());
  P->tz = choose_tz(h.M, h.nxp, tiles_for(h, 32), tiles_for(h, 16), tiles_for(h, 8));
  P->tiles_x = (h.nxp + TILE_X - 1) / TILE_X;
  P->tiles = tiles_for(h, P->tz);
  CK(cudaStreamSynchronize(P->st));  // materials/tables staging buffers are freed next
  return P.release();
}

// --------------------------------------------------------------------------
// migrate
// --------------------------------------------------------------------------
template <int M>
void launch_epilogue_M(Prop& P, const Epilogue& E) {
  const dim3 b2(32, 8);
  if (P.stab_pending) {
    // the step's stabilisation scale with the epilogue (after_step left it)
    P.stab_pending = false;
    const dim3 g2((unsigned)((P.h.ld + 31 + 31) / 32), (unsigned)((P.h.nzp + 7) / 8));   // + the column shift
    k_stab_epilogue<M><<<g2, b2, 0, P.st>>>(P.dp(), 0, P.stab.as<StabState>(), P.cfg.amplitude_cap, E);
    return;
  }
  const dim3 g2((P.h.nx + 31) / 32, (P.h.nz + 7) / 8);
  k_epilogue<M><<<g2, b2, 0, P.st>>>(P.dp(), 0, E);
}

void launch_epilogue(Prop& P, const Epilogue& E) {
  switch (P.M) {
    case 1: launch_epilogue_M<1>(P, E); break;
    case 2: launch_epilogue_M<2>(P, E); break;
    case 3: launch_epilogue_M<3>(P, E); break;
    default: launch_epilogue_M<4>(P, E); break;
  }
  ++g_launches;
}

// Per-shot state of one migration: device buffers, epilogue template and
// the position in the schedule (used by the plain and the batched drivers).
struct ShotRun {
  Prop* F = nullptr;
  Prop* B = nullptr;
  cudaStream_t f_st0 = nullptr, b_st0 = nullptr;   // the propagators' streams before the run
  ertm_migrate_config cfg{};
  int fi = 0, bi = 0;          // indices of F and B in the launch's DevProp table
  int nt = 0, iv = 1, n_states = 0;
  int64_t nrec = 0;
  size_t npix = 0;
  bool excitation = false, kahan = false, want_ill = false, want_ril = false;
  bool need_src[2] = {false, false}, need_rcv_s = false;
  bool bwd_unfused = false, fwd_unfused = false;
  int n_src = 1;               // source image fields stored per replayed step (P and/or S)
  DevBuf wave, rec, acc, ck, rbuf[2], running, peak;
  std::vector<int64_t> ck_step;
  InjectPlanHost* plan = nullptr;
  double* num[MAX_EPI_IMAGES] = {};
  double* ril[MAX_EPI_IMAGES] = {};
  double* ill_slot[2] = {};
  Epilogue base{};
  double* out[3] = {};
  // schedule: 0 forward, 1 replay/backward, 2 excitation map, 3 excitation backward, 4 done
  int phase = 0;
  int t_f = 0, rp_block = -1, rp_t = 0, bk_block = -1, bk_t = 0, replayed_below = 0;
  int s_of(int b) const { return b * iv; }
  int e_of(int b) const { return std::min((b + 1) * iv, nt); }
};

void prepare_run(ShotRun& R, Prop& F, Prop& B, const ertm_migrate_config& cfg, const float* wavelet,
                 const float* record, double* num_out, double* illum_out, double* rillum_out, cudaStream_t st,
                 int n_buffers) {
  REQUIRE(F.h.engine == B.h.engine && F.h.nz == B.h.nz && F.h.nx == B.h.nx, "fwd/back mismatch");
  REQUIRE(cfg.nt >= 1 && cfg.interval >= 1 && cfg.nt_spec >= 1, "bad nt/interval");
  REQUIRE(cfg.n_images >= 1 && cfg.n_images <= MAX_EPI_IMAGES, "n_images must be 1..2");
  REQUIRE(cfg.n_comp >= 0 && cfg.n_comp <= 8, "n_comp must be 0..8");
  REQUIRE(!B.rx.empty() || cfg.n_comp == 0, "receivers must be set on the backward propagator");
  for (int k = 0; k < cfg.n_images; ++k)
    REQUIRE((cfg.src_wave[k] == 0 || cfg.src_wave[k] == 1) && (cfg.rcv_wave[k] == 0 || cfg.rcv_wave[k] == 1) &&
                (F.h.engine == ENGINE_ELASTIC || (cfg.src_wave[k] == 0 && cfg.rcv_wave[k] == 0)),
            "wave not available for this engine");
  R.f_st0 = F.st;
  R.b_st0 = B.st;
  for (Prop* P : {&F, &B})
    if (P->st != st) {
      CK(cudaStreamSynchronize(P->st));
      P->st = st;
    }
  R.F = &F;
  R.B = &B;
  CK(cudaMemsetAsync(F.status.p, 0, sizeof(uint32_t), st));
  CK(cudaMemsetAsync(B.status.p, 0, sizeof(uint32_t), st));
  R.cfg = cfg;
  R.nt = cfg.nt;
  R.iv = cfg.interval;
  R.n_states = (cfg.nt + cfg.interval - 1) / cfg.interval;
  R.npix = (size_t)F.h.nz * F.h.nx;
  R.excitation = cfg.condition == ERTM_COND_EXCITATION;
  R.kahan = cfg.accum == ERTM_ACCUM_KAHAN && !R.excitation;
  R.want_ill = (cfg.illumination & 1) && !R.excitation;
  R.want_ril = (cfg.illumination & 2) != 0;
  R.out[0] = num_out;
  R.out[1] = illum_out;
  R.out[2] = rillum_out;
  const size_t npix = R.npix;
  const int nimg = cfg.n_images;
  R.acc = DevBuf(npix * 8 * (2 * nimg + 2), st);
  CK(cudaMemsetAsync(R.acc.p, 0, R.acc.bytes, st));
  R.ill_slot[0] = R.acc.as<double>() + 2 * nimg * npix;
  R.ill_slot[1] = R.acc.as<double>() + (2 * nimg + 1) * npix;
  for (int k = 0; k < nimg; ++k) {
    R.num[k] = R.acc.as<double>() + k * npix;
    R.ril[k] = R.acc.as<double>() + (nimg + k) * npix;
  }
  R.wave = DevBuf((size_t)R.nt * 4, st);
  upload(R.wave.p, wavelet, (size_t)R.nt * 4, st);
  std::vector<int> comps(cfg.comp, cfg.comp + cfg.n_comp);
  R.nrec = (int64_t)B.rx.size();
  R.rec = DevBuf((size_t)cfg.n_comp * cfg.nt_spec * R.nrec * 4, st);
  upload(R.rec.p, record, R.rec.bytes, st);
  R.plan = comps.empty() ? nullptr : &inject_plan(B, comps, cfg.nt_spec);
  if (R.plan && R.plan->n_cells == 0) R.plan = nullptr;
  R.ck = DevBuf((size_t)R.n_states * F.state_floats * 4, st);
  R.ck_step.assign(R.n_states, 0);
  Epilogue& E = R.base;
  E = Epilogue{};
  E.sep = cfg.separation;
  E.n_images = nimg;
  E.kahan = R.kahan ? 1 : 0;
  for (int k = 0; k < nimg; ++k) {
    E.src_slot[k] = cfg.src_wave[k];
    E.rcv_wave[k] = cfg.rcv_wave[k];
    E.num[k] = R.num[k];
    E.ril[k] = R.want_ril ? R.ril[k] : nullptr;
    R.need_src[cfg.src_wave[k]] = true;
    R.need_rcv_s |= cfg.rcv_wave[k] == 1;
  }
  // each distinct source wave's illumination is accumulated once
  for (int k = 0; k < nimg; ++k) {
    bool first = true;
    for (int q = 0; q < k; ++q) first &= cfg.src_wave[q] != cfg.src_wave[k];
    E.ill[k] = (R.want_ill && first) ? R.ill_slot[cfg.src_wave[k]] : nullptr;
  }
  // The fused epilogue sees the fields right after the stress phase; it runs
  // stand-alone when something still changes them afterwards.
  R.bwd_unfused = B.h.engine == ENGINE_VISCO && B.cfg.compensation;
  R.fwd_unfused = F.h.engine == ENGINE_ELASTIC && F.h.mech == MECH_FORCE_Z && cfg.separation == 1;
  if (!R.excitation) {
    // only the source waves some image uses are stored: P, S or both per step
    R.n_src = (R.need_src[0] ? 1 : 0) + (R.need_src[1] ? 1 : 0);
    for (int k = 0; k < n_buffers; ++k) R.rbuf[k] = DevBuf((size_t)R.iv * R.n_src * npix * 4, st);
  } else {
    R.running = DevBuf(npix * 4, st);
    R.peak = DevBuf(npix * 4, st);
    CK(cudaMemsetAsync(R.running.p, 0, npix * 4, st));
    CK(cudaMemsetAsync(R.peak.p, 0xff, npix * 4, st));  // −1
  }
}

void save_checkpoint(ShotRun& R, int b, cudaStream_t st) {
  CK(cudaMemcpyAsync(R.ck.as<float>() + (size_t)b * R.F->state_floats, R.F->state.p, R.F->state_floats * 4,
                     cudaMemcpyDeviceToDevice, st));
  R.ck_step[b] = R.F->step_index;
}

void restore_checkpoint(ShotRun& R, int b, cudaStream_t st) {
  CK(cudaMemcpyAsync(R.F->state.p, R.ck.as<float>() + (size_t)b * R.F->state_floats, R.F->state_floats * 4,
                     cudaMemcpyDeviceToDevice, st));
  R.F->step_index = R.ck_step[b];
}

// Epilogues of the replay step at time t of block b and of the backward step at t.
Epilogue replay_epilogue(const ShotRun& R, int b, int t) {
  Epilogue e = R.base;
  if (R.excitation) {
    e.kind = EPI_EXC_TRACK;
    e.running = R.running.as<float>();
    e.peak_step = R.peak.as<int32_t>();
    e.step = t;
    return e;
  }
  float* slot = R.rbuf[b & (R.rbuf[1].p ? 1 : 0)].as<float>() + (size_t)(t - R.s_of(b)) * R.n_src * R.npix;
  e.kind = EPI_STORE;
  e.need_s = R.need_src[1] ? 1 : 0;
  e.out[0] = R.need_src[0] ? slot : nullptr;
  e.out[1] = R.need_src[1] ? slot + (R.need_src[0] ? R.npix : 0) : nullptr;
  return e;
}

Epilogue backward_epilogue(const ShotRun& R, int b, int t) {
  Epilogue e = R.base;
  if (R.excitation) {
    e.kind = t >= R.cfg.start_step ? EPI_EXC_IMAGE : EPI_NONE;
    e.need_s = R.need_rcv_s ? 1 : 0;
    e.running = R.running.as<float>();
    e.peak_step = R.peak.as<int32_t>();
    e.step = t;
    return e;
  }
  const float* slot = R.rbuf[b & (R.rbuf[1].p ? 1 : 0)].as<float>() + (size_t)(t - R.s_of(b)) * R.n_src * R.npix;
  e.kind = EPI_IMAGE;
  e.need_s = R.need_rcv_s ? 1 : 0;
  e.illum = R.want_ill ? 1 : 0;
  e.rillum = R.want_ril ? 1 : 0;
  e.src[0] = R.need_src[0] ? slot : nullptr;
  e.src[1] = R.need_src[1] ? slot + (R.need_src[0] ? R.npix : 0) : nullptr;
  e.cross = t >= R.cfg.start_step ? 1 : 0;
  if (!e.cross && !e.illum && !e.rillum) e.kind = EPI_NONE;
  return e;
}

void finish_run(ShotRun& R, cudaStream_t st) {
  const size_t npix = R.npix;
  DevBuf tmp(R.kahan ? npix * 8 : 0, st);
  auto copy_out = [&](double* dst, const double* src) {
    const double* from = src;
    if (R.kahan) {
      const float* s = reinterpret_cast<const float*>(src);
      k_kahan_to_f64<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(s, s + npix, tmp.as<double>(), (int64_t)npix);
      from = tmp.as<double>();
    }
    CK(cudaMemcpyAsync(dst, from, npix * 8, cudaMemcpyDefault, st));
  };
  for (int k = 0; k < R.cfg.n_images; ++k) {
    if (R.out[0]) copy_out(R.out[0] + (size_t)k * npix, R.num[k]);
    if (R.out[1]) copy_out(R.out[1] + (size_t)k * npix, R.ill_slot[R.cfg.src_wave[k]]);
    if (R.out[2]) copy_out(R.out[2] + (size_t)k * npix, R.ril[k]);
  }
  CK(cudaStreamSynchronize(st));
}

// Hand the propagators back to the streams they had before the run (a
// session's stream dies with the session; the propagators outlive it).
void release_streams(ShotRun& R, cudaStream_t st) {
  CK(cudaStreamSynchronize(st));
  R.F->st = R.f_st0;
  R.B->st = R.b_st0;
}

void inject_one(ShotRun& R, int t, cudaStream_t st) {
  if (!R.plan) return;
  ++g_launches;
  k_inject<<<(R.plan->n_cells + 127) / 128, 128, 0, st>>>(R.B->dp(), 0, R.plan->dev(), R.rec.as<float>(),
                                                            (int64_t)t * R.nrec);
}

// Status word of a propagator after the work queued on `st`.
uint32_t read_status(const Prop& P, cudaStream_t st) {
  uint32_t v = 0;
  CK(cudaMemcpyAsync(&v, P.status.p, sizeof(v), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return v;
}

// The error of a run whose propagators flagged non-finite values.
void require_finite(const ShotRun& R, cudaStream_t st, const std::string& what) {
  const uint32_t f = read_status(*R.F, st), b = read_status(*R.B, st);
  if ((f | b) & STATUS_NONFINITE)
    throw Error(ERTM_ERR_NONFINITE, what + ": the " + std::string(f ? "source (forward/replay)" : "backward") +
                                        " wavefield became non-finite (NaN or infinity)");
}

// Plain driver: one shot, steps one after the other (imaging.py:255-331).
void migrate(Prop& F, Prop& B, const ertm_migrate_config& cfg, const float* wavelet, const float* record,
             double* num_out, double* illum_out, double* rillum_out) {
  cudaStream_t st = F.st;
  ShotRun R;
  prepare_run(R, F, B, cfg, wavelet, record, num_out, illum_out, rillum_out, st, 1);
  const float* dw = R.wave.as<float>();
  auto fwd_step = [&](int t, const Epilogue& e) {
    if (R.fwd_unfused) {
      step_once(F, 0.0, dw, t);
      launch_epilogue(F, e);
    } else {
      step_once(F, 0.0, dw, t, &e);
    }
  };
  auto bwd_step = [&](const Epilogue& e) {
    if (e.kind == EPI_NONE) {
      step_once(B, 0.0);
    } else if (R.bwd_unfused) {
      step_once(B, 0.0, nullptr, 0, nullptr, true);
      launch_epilogue(B, e);
    } else {
      step_once(B, 0.0, nullptr, 0, &e);
    }
  };
  // forward with checkpoints (imaging.py:113-137)
  for (int t = 0; t < R.nt; ++t) {
    step_once(F, 0.0, dw, t);
    if (t % R.iv == 0) save_checkpoint(R, t / R.iv, st);
  }
  if (!R.excitation) {
    for (int b = R.n_states - 1; b >= 0; --b) {
      restore_checkpoint(R, b, st);
      for (int t = R.s_of(b); t < R.e_of(b); ++t) fwd_step(t, replay_epilogue(R, b, t));
      for (int t = R.e_of(b) - 1; t >= R.s_of(b); --t) {
        inject_one(R, t, st);
        bwd_step(backward_epilogue(R, b, t));
      }
    }
  } else {
    for (int b = 0; b < R.n_states; ++b) {
      restore_checkpoint(R, b, st);
      for (int t = R.s_of(b); t < R.e_of(b); ++t) fwd_step(t, replay_epilogue(R, b, t));
    }
    // backward over [0, nt_spec) (imaging.py:283-303); A² illumination is unused
    for (int t = cfg.nt_spec - 1; t >= 0; --t) {
      inject_one(R, t, st);
      bwd_step(backward_epilogue(R, 0, t));
    }
  }
  CK(cudaGetLastError());
  finish_run(R, st);
  require_finite(R, st, "migrate");
}

// --------------------------------------------------------------------------
// Batched driver (form (b)): many shots advance in lockstep ticks.  A tick
// gives every unfinished shot at most one forward/replay step and one
// backward step; all steps of a tick share one velocity and one stress launch
// per (engine, order) group.  During the replay/backward phase the replay of
// block b−1 (into one replay buffer) overlaps the backward pass over block b
// (reading the other), so a shot needs ≈ 2·nt ticks instead of 3·nt steps.
// Every propagator performs exactly the steps of the plain driver in the same
// order, so the results are identical.
// --------------------------------------------------------------------------
struct TickItem {
  ShotRun* run;
  bool fwd;          // replay/forward propagator (else backward)
  StepWork w;
  bool unfused;      // epilogue runs after after_step
  Epilogue epi;      // the epilogue (fused into w, or stand-alone)
};

std::atomic<int> g_tick_lanes{0};   // 0 automatic, 1 or 2 lanes
// Which works share a lane: 0 alternate works (a shot's replay step on one
// lane, its backward step on the other), 1 alternate shots (both steps of a
// shot on one lane, so the lanes carry equal mixes).
std::atomic<int> g_lane_assign{0};
std::atomic<int> g_autotune{1};     // tune batched tick launches online

// ---------------------------------------------------------------------------
// Online autotuner for batched ticks.  A tick group (engine, order, number of
// works, size class) runs its first ticks with each candidate launch shape in
// turn — tile height 8/16/32, interior/frame split off/on, one or two lanes —
// timed with CUDA events on the launching stream and read back as they
// complete (no synchronisation); once every candidate has kTuneSamples
// samples the fastest one is kept for the process.  Every candidate computes
// the same results, so switching shapes between ticks is safe.
// ---------------------------------------------------------------------------
struct TuneCfg {
  int tz, split, lanes;
};
constexpr int kTuneSamples = 3;

struct TuneState {
  std::vector<TuneCfg> cands;
  std::vector<double> sum_ms;
  std::vector<int> n;
  int best = -1, next = 0, pending = 0;
};

struct TuneSample {
  TuneState* ts;
  int cand;
  cudaEvent_t e0, e1;
};

std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int, int>, TuneState> g_tune;
std::vector<TuneSample> g_tune_pending;
std::vector<cudaEvent_t> g_tune_events;

cudaEvent_t tune_event() {
  if (!g_tune_events.empty()) {
    cudaEvent_t e = g_tune_events.back();
    g_tune_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  CK(cudaEventCreate(&e));
  return e;
}

// Fold in the samples whose events have completed.
void tune_collect() {
  for (size_t k = 0; k < g_tune_pending.size();) {
    TuneSample& t = g_tune_pending[k];
    const cudaError_t q = cudaEventQuery(t.e1);
    if (q == cudaErrorNotReady) {
      ++k;
      continue;
    }
    CK(q);
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, t.e0, t.e1));
    TuneState& ts = *t.ts;
    ts.sum_ms[t.cand] += ms;
    ++ts.n[t.cand];
    --ts.pending;
    g_tune_events.push_back(t.e0);
    g_tune_events.push_back(t.e1);
    g_tune_pending[k] = g_tune_pending.back();
    g_tune_pending.pop_back();
    bool all = ts.best < 0;
    for (size_t c = 0; all && c < ts.cands.size(); ++c) all = ts.n[c] >= kTuneSamples;
    if (all) {
      int b = 0;
      for (size_t c = 1; c < ts.cands.size(); ++c)
        if (ts.sum_ms[c] / ts.n[c] < ts.sum_ms[b] / ts.n[b]) b = (int)c;
      ts.best = b;
    }
  }
}

// One (engine, order) group of a tick.  Large groups may run as two or four
// lanes (the works taken in turn, each lane on its own stream): the stress
// phase of one lane, bound by the latency of its epilogue loads, then
// overlaps the velocity phase of another, bound by instruction issue.
void launch_group(std::vector<TickItem*>& items, const DevProp* table, cudaStream_t st, double& bytes) {
  if (items.empty()) return;
  const Prop& P0 = items[0]->fwd ? *items[0]->run->F : *items[0]->run->B;
  const int M = P0.M, engine = P0.h.engine;
  for (size_t c0 = 0; c0 < items.size(); c0 += MAX_BATCH_WORKS) {
    const size_t c1 = std::min(items.size(), c0 + MAX_BATCH_WORKS);
    int64_t t32 = 0, t16 = 0, t8 = 0, cells = 0;
    for (size_t k = c0; k < c1; ++k) {
      const Prop& P = items[k]->fwd ? *items[k]->run->F : *items[k]->run->B;
      t32 += tiles_for(P.h, 32);
      t16 += tiles_for(P.h, 16);
      t8 += tiles_for(P.h, 8);
      cells += (int64_t)P.h.nzp * P.h.nxp;
    }
    // heuristic shape, or the autotuner's choice
    TuneCfg cfg{choose_tz(M, 0, t32, t16, t8), g_tile_split.load(), 0};
    {
      const int lanes_mode = g_tick_lanes.load();
      const int64_t total = cfg.tz == 32 ? t32 : (cfg.tz == 16 ? t16 : t8);
      cfg.lanes = (lanes_mode == 2 || (lanes_mode == 0 && c1 - c0 >= 4 && total >= 3 * kSplitMinTiles)) ? 2 : 1;
    }
    TuneState* ts = nullptr;
    int cand = -1;
    const bool forced = g_tile_rows.load() != 0 || g_tile_split.load() != 0 || g_tick_lanes.load() != 0;
    if (M == 4 && g_autotune.load() && !forced && t16 >= kSplitMinTiles / 4) {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      tune_collect();
      int lg = 0;
      while ((int64_t(1) << (lg + 1)) <= cells) ++lg;
      ts = &g_tune[{engine, M, (int)(c1 - c0), lg, 0}];
      if (ts->cands.empty()) {
        for (int tz : {16, 32, 8})
          for (int split : {1, 2})
            for (int lanes : {1, 2}) {             // four lanes measured slower on the benchmark job
              if (lanes > 1 && (int)(c1 - c0) < lanes) continue;
              ts->cands.push_back({tz, split, lanes});
            }
        ts->sum_ms.assign(ts->cands.size(), 0.0);
        ts->n.assign(ts->cands.size(), 0);
      }
      if (ts->best >= 0) {
        cfg = ts->cands[ts->best];
      } else if (ts->pending < 8) {
        // the candidate with the fewest samples (counting those in flight)
        cand = ts->next;
        ts->next = (ts->next + 1) % (int)ts->cands.size();
        cfg = ts->cands[cand];
      }
    }
    const int tz = cfg.tz;
    const int lanes = cfg.lanes;
    WorkSetB ws[kLanes]{};
    int tile0[kLanes] = {};
    const Prop* hosts[kLanes][MAX_BATCH_WORKS];
    const bool by_shot = g_lane_assign.load() == 1;
    int shot_no = 0;
    for (size_t k = c0; k < c1; ++k) {
      const Prop& P = items[k]->fwd ? *items[k]->run->F : *items[k]->run->B;
      if (k > c0 && items[k]->run != items[k - 1]->run) ++shot_no;
      const int l = lanes > 1 ? (by_shot ? shot_no : (int)(k - c0)) % lanes : 0;
      StepWork w = items[k]->w;
      w.tile0 = tile0[l];
      w.tiles_x = (P.h.nxp + TILE_X - 1) / TILE_X;
      w.tiles = tiles_for(P.h, tz);
      tile0[l] += w.tiles;
      hosts[l][ws[l].n] = &P;
      ws[l].w[ws[l].n++] = w;
      bytes += step_bytes(P) + epilogue_bytes(w.epi, (size_t)P.h.nz * P.h.nx);
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cand >= 0) {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      e0 = tune_event();
      e1 = tune_event();
      CK(cudaEventRecord(e0, st));
    }
    if (lanes == 1) {
      launch_works(M, tz, engine, table, ws[0], ws[0].n, hosts[0], st, 0, cfg.split);
    } else {
      // every lane starts after what precedes the tick on the caller's stream
      // and the caller's stream waits for every lane; lanes without works are
      // skipped
      LaneStreams& ls = lane_streams();
      for (int l = 1; l < lanes; ++l) {
        if (ws[l].n == 0) continue;
        CK(cudaEventRecord(ls.fork[l], st));
        CK(cudaStreamWaitEvent(ls.lane[l], ls.fork[l], 0));
      }
      if (ws[0].n > 0) launch_works(M, tz, engine, table, ws[0], ws[0].n, hosts[0], st, 0, cfg.split);
      for (int l = 1; l < lanes; ++l) {
        if (ws[l].n == 0) continue;
        launch_works(M, tz, engine, table, ws[l], ws[l].n, hosts[l], ls.lane[l], l, cfg.split);
        CK(cudaEventRecord(ls.join[l], ls.lane[l]));
        CK(cudaStreamWaitEvent(st, ls.join[l], 0));
      }
    }
    if (cand >= 0) {
      std::lock_guard<std::mutex> lock(g_tune_mutex);
      CK(cudaEventRecord(e1, st));
      g_tune_pending.push_back({ts, cand, e0, e1});
      ++ts->pending;
    }
  }
}

// The stand-alone epilogues of a tick's items (all of stencil half-order M,
// all on stream st) in launches of up to MAX_BATCH_WORKS items; an item
// whose stabilisation scale after_step left pending gets it here.
template <int M>
void launch_epilogue_batch_M(const std::vector<TickItem*>& its, const DevProp* table, cudaStream_t st) {
  static_assert(sizeof(EpiBatch) < 30000, "kernel parameter block too large");
  for (size_t c0 = 0; c0 < its.size(); c0 += MAX_BATCH_WORKS) {
    EpiBatch B{};
    unsigned gx = 1, gy = 1;
    for (size_t k = c0; k < std::min(its.size(), c0 + MAX_BATCH_WORKS); ++k) {
      TickItem& it = *its[k];
      Prop& P = it.fwd ? *it.run->F : *it.run->B;
      EpiItem& I = B.it[B.n++];
      I.prop = it.w.prop;
      I.stab = P.stab_pending ? 1 : 0;
      P.stab_pending = false;
      I.cap = P.cfg.amplitude_cap;
      I.st = P.stab.as<StabState>();
      I.E = it.epi;
      gx = std::max(gx, (unsigned)((P.h.ld + 31 + 31) / 32));   // + the column shift (< 32)
      gy = std::max(gy, (unsigned)((P.h.nzp + 7) / 8));
    }
    k_epilogue_batch<M><<<dim3(gx, gy, (unsigned)B.n), dim3(32, 8), 0, st>>>(table, B);
    ++g_launches;
  }
}

void launch_epilogue_batch(int M, const std::vector<TickItem*>& its, const DevProp* table, cudaStream_t st) {
  switch (M) {
    case 1: launch_epilogue_batch_M<1>(its, table, st); break;
    case 2: launch_epilogue_batch_M<2>(its, table, st); break;
    case 3: launch_epilogue_batch_M<3>(its, table, st); break;
    default: launch_epilogue_batch_M<4>(its, table, st); break;
  }
}

// DevProp table of every propagator of `runs` (uploaded when the set changes).
void upload_table(std::vector<ShotRun*>& runs, std::vector<DevProp>& table, DevBuf& dtable, cudaStream_t st) {
  table.clear();
  for (ShotRun* R : runs) {
    R->fi = (int)table.size();
    table.push_back(R->F->h);
    R->bi = (int)table.size();
    table.push_back(R->B->h);
  }
  const size_t bytes = std::max<size_t>(1, table.size()) * sizeof(DevProp);
  if (dtable.bytes < bytes) dtable = DevBuf(bytes, st);
  upload(dtable.p, table.data(), table.size() * sizeof(DevProp), st);
}

// One tick of the batched schedule: every unfinished shot of `runs` gets at
// most one forward/replay step and one backward step.  Returns false when no
// shot had work left.
bool batch_tick(std::vector<ShotRun*>& runs, const DevProp* dt, cudaStream_t st) {
  static_assert(sizeof(WorkSetB) < 30000, "kernel parameter block too large");
  static_assert(sizeof(InjectBatch) < 30000, "kernel parameter block too large");
  std::vector<TickItem> items;
  items.reserve(2 * runs.size());
  std::vector<std::pair<ShotRun*, int>> restores, injections;
  for (ShotRun* Rp : runs) {
    ShotRun& R = *Rp;
    switch (R.phase) {
      case 0: {  // forward with checkpoints
        TickItem it{&R, true, make_work(*R.F, 0.0, R.wave.as<float>(), R.t_f, nullptr), false, {}};
        it.w.prop = R.fi;
        items.push_back(it);
        break;
      }
      case 1: {  // replay of block rp_block overlapped with the backward over bk_block
        const bool do_rp = R.rp_block >= 0 && R.bk_block <= R.rp_block + 1;
        const bool do_bk = R.bk_block >= 0 && R.replayed_below <= R.bk_block;
        if (do_rp) {
          if (R.rp_t == R.s_of(R.rp_block)) restores.push_back({&R, R.rp_block});
          Epilogue e = replay_epilogue(R, R.rp_block, R.rp_t);
          TickItem it{&R, true, make_work(*R.F, 0.0, R.wave.as<float>(), R.rp_t, R.fwd_unfused ? nullptr : &e),
                      R.fwd_unfused, e};
          it.w.prop = R.fi;
          items.push_back(it);
        }
        if (do_bk) {
          injections.push_back({&R, R.bk_t});
          Epilogue e = backward_epilogue(R, R.bk_block, R.bk_t);
          const bool unf = R.bwd_unfused && e.kind != EPI_NONE;
          TickItem it{&R, false, make_work(*R.B, 0.0, nullptr, 0, unf ? nullptr : &e), unf, e};
          it.w.prop = R.bi;
          items.push_back(it);
        }
        break;
      }
      case 2: {  // excitation map: replay every block forward
        if (R.rp_t == R.s_of(R.rp_block)) restores.push_back({&R, R.rp_block});
        Epilogue e = replay_epilogue(R, R.rp_block, R.rp_t);
        TickItem it{&R, true, make_work(*R.F, 0.0, R.wave.as<float>(), R.rp_t, R.fwd_unfused ? nullptr : &e),
                    R.fwd_unfused, e};
        it.w.prop = R.fi;
        items.push_back(it);
        break;
      }
      case 3: {  // excitation backward over [0, nt_spec)
        injections.push_back({&R, R.bk_t});
        Epilogue e = backward_epilogue(R, 0, R.bk_t);
        const bool unf = R.bwd_unfused && e.kind != EPI_NONE;
        TickItem it{&R, false, make_work(*R.B, 0.0, nullptr, 0, unf ? nullptr : &e), unf, e};
        it.w.prop = R.bi;
        items.push_back(it);
        break;
      }
      default:
        break;
    }
  }
  if (items.empty()) return false;
  for (auto& r : restores) restore_checkpoint(*r.first, r.second, st);
  // time-reversed record injection of this tick's backward steps
  for (size_t c0 = 0; c0 < injections.size(); c0 += MAX_BATCH_WORKS) {
    InjectBatch ib{};
    int cells = 0;
    for (size_t k = c0; k < std::min(injections.size(), c0 + MAX_BATCH_WORKS); ++k) {
      ShotRun& R = *injections[k].first;
      if (!R.plan) continue;
      InjectItem& I = ib.it[ib.n++];
      I.plan = R.plan->dev();
      I.prop = dt + R.bi;
      I.record = R.rec.as<float>();
      I.time_offset = (int64_t)injections[k].second * R.nrec;
      I.cell0 = cells;
      cells += R.plan->n_cells;
    }
    if (cells > 0) {
      k_inject_batch<<<(cells + 127) / 128, 128, 0, st>>>(ib);
      ++g_launches;
    }
  }
  // stencil launches, grouped by (engine, order)
  std::map<std::pair<int, int>, std::vector<TickItem*>> groups;
  for (TickItem& it : items) {
    const Prop& P = it.fwd ? *it.run->F : *it.run->B;
    groups[{P.h.engine, P.M}].push_back(&it);
  }
  cudaEvent_t e0 = nullptr;
  const bool timed = g_prof.begin(st, e0);
  double bytes = 0.0;
  for (auto& g : groups) launch_group(g.second, dt, st, bytes);
  if (timed) g_prof.end(st, e0, bytes);
  // after the stress phase: sources on vz, stabilisation (the tick's
  // low-passes in shared launches), stand-alone epilogues, checkpoints
  std::vector<LowpassItem> lowpasses;
  for (TickItem& it : items) {
    ShotRun& R = *it.run;
    Prop& P = it.fwd ? *R.F : *R.B;
    after_step(P, 0.0, it.fwd ? R.wave.as<float>() : nullptr, it.w.t, &lowpasses, it.unfused);
  }
  if (!lowpasses.empty()) lowpass_props(lowpasses, st);
  // stand-alone epilogues: one launch per stencil order (k_epilogue_batch)
  // when they share the tick's stream, else one launch each
  std::map<int, std::vector<TickItem*>> unfused;
  for (TickItem& it : items) {
    ShotRun& R = *it.run;
    Prop& P = it.fwd ? *R.F : *R.B;
    if (it.unfused) {
      if (P.st == st) unfused[P.M].push_back(&it);
      else launch_epilogue(P, it.epi);
    }
    if (R.phase == 0 && R.t_f % R.iv == 0) save_checkpoint(R, R.t_f / R.iv, st);
  }
  for (auto& g : unfused) launch_epilogue_batch(g.first, g.second, dt, st);
  CK(cudaGetLastError());
  // advance the schedules
  for (ShotRun* Rp : runs) {
    ShotRun& R = *Rp;
    switch (R.phase) {
      case 0:
        if (++R.t_f == R.nt) {
          if (!R.excitation) {
            R.phase = 1;
            R.rp_block = R.bk_block = R.n_states - 1;
            R.rp_t = R.s_of(R.rp_block);
            R.bk_t = R.e_of(R.bk_block) - 1;
            R.replayed_below = R.n_states;
          } else {
            R.phase = 2;
            R.rp_block = 0;
            R.rp_t = 0;
          }
        }
        break;
      case 1: {
        const bool did_rp = R.rp_block >= 0 && R.bk_block <= R.rp_block + 1;
        const bool did_bk = R.bk_block >= 0 && R.replayed_below <= R.bk_block;
        if (did_bk) {
          if (--R.bk_t < R.s_of(R.bk_block)) {
            --R.bk_block;
            if (R.bk_block >= 0) R.bk_t = R.e_of(R.bk_block) - 1;
          }
        }
        if (did_rp) {
          if (++R.rp_t == R.e_of(R.rp_block)) {
            R.replayed_below = R.rp_block;
            --R.rp_block;
            if (R.rp_block >= 0) R.rp_t = R.s_of(R.rp_block);
          }
        }
        if (R.bk_block < 0) R.phase = 4;
        break;
      }
      case 2:
        if (++R.rp_t == R.e_of(R.rp_block)) {
          if (++R.rp_block == R.n_states) {
            R.phase = 3;
            R.bk_t = R.cfg.nt_spec - 1;
          } else {
            R.rp_t = R.s_of(R.rp_block);
          }
        }
        break;
      case 3:
        if (--R.bk_t < 0) R.phase = 4;
        break;
      default:
        break;
    }
  }
  return true;
}

void migrate_batch(std::vector<ShotRun>& runs, cudaStream_t st) {
  std::vector<ShotRun*> ptrs;
  for (ShotRun& R : runs) ptrs.push_back(&R);
  std::vector<DevProp> table;
  DevBuf dtable;
  upload_table(ptrs, table, dtable, st);
  while (batch_tick(ptrs, dtable.as<DevProp>(), st)) {
  }
  for (ShotRun& R : runs) finish_run(R, st);
  std::string bad;
  for (size_t k = 0; k < runs.size(); ++k) {
    const uint32_t f = read_status(*runs[k].F, st), b = read_status(*runs[k].B, st);
    if ((f | b) & STATUS_NONFINITE) bad += (bad.empty() ? "" : ", ") + std::to_string(k);
  }
  if (!bad.empty())
    throw Error(ERTM_ERR_NONFINITE, "migrate_batch: the wavefields of shot(s) " + bad +
                                        " became non-finite (NaN or infinity); the other shots' images are complete");
}

// --------------------------------------------------------------------------
// Batch sessions (serving): shots join between ticks and leave when done, so
// shots that arrive while others run share their ticks (continuous batching).
// --------------------------------------------------------------------------
struct Session {
  cudaStream_t st = nullptr;
  std::vector<std::unique_ptr<ShotRun>> runs;
  std::vector<int64_t> tags;
  std::vector<int64_t> failed;   // tags of shots taken out for non-finite wavefields
  std::vector<DevProp> table;
  DevBuf dtable, status;
  bool dirty = true;
  int64_t ticks = 0;
};

// --------------------------------------------------------------------------
// Allocation-free stacking (ertm_stack_noalloc)
// --------------------------------------------------------------------------
// Callers that cannot allocate device memory — a serving process whose whole
// device memory is carved up by its own pool at start-up, a host framework
// that owns every allocation, or code that must not trigger the implicit
// device synchronisation cudaMalloc/cudaFree can cause — still need the
// per-shot-normalised stack.  This variant keeps its scratch in file-scope
// device arrays: one chunk of float64 sums (the image is stacked chunk by
// chunk) and one max|·| word per image.  Every GPU that loads this library
// holds these 2 MiB + 4 KiB until the process exits.
constexpr int64_t kStackChunk = 1 << 18;     // pixels per pass
constexpr int kStackMaxImages = 1024;
static __device__ __align__(256) double g_stack_sum[kStackChunk];
static __device__ __align__(256) unsigned int g_stack_scale[kStackMaxImages];

struct StackScratch {
  double* sum = nullptr;
  unsigned int* scale = nullptr;
};
std::map<std::pair<int, CUcontext>, StackScratch> g_stack_scratch;
std::mutex g_stack_mutex;

// The calling thread's current driver context (through the runtime's
// driver entry point, so the library needs no link against libcuda).
CUcontext current_context() {
  static PFN_cuCtxGetCurrent_v4000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    CK(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q));
    REQUIRE(q == cudaDriverEntryPointSuccess && p, "cuCtxGetCurrent is not available");
    return reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
  }();
  CUcontext c = nullptr;
  REQUIRE(fn(&c) == CUDA_SUCCESS, "cuCtxGetCurrent failed");
  return c;
}

// Device addresses of the scratch arrays for the current device; looked up
// once per device and context (the host-side names are not device
// addresses).  Keying on the context as well means a device reset, which
// gives the device a new primary context, leads to a fresh lookup instead of
// addresses in a context that no longer exists.
StackScratch stack_scratch() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaFree(nullptr));   // makes the device's primary context current (allocates nothing)
  const std::pair<int, CUcontext> key{dev, current_context()};
  std::lock_guard<std::mutex> lock(g_stack_mutex);
  auto it = g_stack_scratch.find(key);
  if (it != g_stack_scratch.end()) return it->second;
  StackScratch s;
  CK(cudaGetSymbolAddress(reinterpret_cast<void**>(&s.sum), g_stack_sum));
  CK(cudaGetSymbolAddress(reinterpret_cast<void**>(&s.scale), g_stack_scale));
  g_stack_scratch[key] = s;
  return s;
}

void require_device_pointer(const void* p, const char* what) {
  cudaPointerAttributes a{};
  CK(cudaPointerGetAttributes(&a, p));
  REQUIRE(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged,
          std::string(what) + " must be device memory");
}

// Host-or-device arrays for the record kernels: device pointers are used in
// place; host inputs are uploaded and host outputs downloaded at the end.
bool is_device_ptr(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

struct InArray {
  DevBuf buf;
  const void* d = nullptr;
  InArray(const void* p, size_t bytes, cudaStream_t st) {
    if (is_device_ptr(p)) {
      d = p;
    } else {
      buf = DevBuf(bytes, st);
      upload(buf.p, p, bytes, st);
      d = buf.p;
    }
  }
  template <class T>
  const T* as() const { return static_cast<const T*>(d); }
};

struct OutArray {
  DevBuf buf;
  void* host = nullptr;
  void* d = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  OutArray(void* p, size_t b, cudaStream_t s) : bytes(b), st(s) {
    if (is_device_ptr(p)) {
      d = p;
    } else {
      buf = DevBuf(b, s);
      d = buf.p;
      host = p;
    }
  }
  void finish() {
    if (host) CK(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, st));
  }
  template <class T>
  T* as() const { return static_cast<T*>(d); }
};

// The per-shot-normalised float64 stack of `n_images` images in two
// launches per group of images: every image's max|·|, then at each pixel the
// sum over the images in order onto `sum` (or from 0 without it) and, with
// `out`, the mean.  Device images are read in place; host images are
// uploaded first, in groups of at most 1 GiB.  The terms and their order are
// those of one k_absmax_f32 + k_stack_add pair per image.
void stack_group(int n_images, int64_t n, const float* const* images, bool normalize, double* sum, int count,
                 float* out, cudaStream_t st) {
  std::vector<const float*> ptrs(images, images + n_images);
  int n_host = 0;
  for (const float* q : ptrs) n_host += is_device_ptr(q) ? 0 : 1;
  DevBuf stage(n_host > 0 ? (size_t)n_host * n * 4 : 0, st);
  for (int k = 0, h = 0; k < n_images; ++k) {
    if (is_device_ptr(ptrs[k])) continue;
    float* dst = stage.as<float>() + (size_t)h++ * n;
    upload(dst, ptrs[k], n * 4, st);
    ptrs[k] = dst;
  }
  DevBuf table((size_t)n_images * (sizeof(float*) + sizeof(unsigned)), st);
  upload(table.p, ptrs.data(), (size_t)n_images * sizeof(float*), st);
  const float* const* dptrs = table.as<const float*>();
  unsigned* scales = reinterpret_cast<unsigned*>(table.as<char>() + (size_t)n_images * sizeof(float*));
  const unsigned g = (unsigned)((n + 255) / 256);
  if (normalize) {
    CK(cudaMemsetAsync(scales, 0, (size_t)n_images * sizeof(unsigned), st));
    const unsigned bx = std::max(1u, std::min<unsigned>(g, (2368u + n_images - 1) / n_images));
    k_absmax_images<<<dim3(bx, n_images), 256, 0, st>>>(dptrs, n, scales);
    ++g_launches;
  }
  k_stack_images<<<g, 256, 0, st>>>(dptrs, n_images, n, scales, normalize ? 1 : 0, sum, count, out);
  ++g_launches;
  CK(cudaGetLastError());
}

void stack_all(int n_images, int64_t n, const float* const* images, bool normalize, double* sum, int count,
               float* out, cudaStream_t st) {
  if (n_images <= 0) return;
  const int per = (int)std::max<int64_t>(1, std::min<int64_t>(65535, (int64_t(1) << 30) / (n * 4)));
  if (n_images <= per) {
    stack_group(n_images, n, images, normalize, sum, count, out, st);
    return;
  }
  DevBuf acc(sum ? 0 : (size_t)n * 8, st);
  double* s = sum;
  if (!s) {
    s = acc.as<double>();
    CK(cudaMemsetAsync(s, 0, (size_t)n * 8, st));
  }
  for (int k0 = 0; k0 < n_images; k0 += per) {
    const int nk = std::min(per, n_images - k0);
    stack_group(nk, n, images + k0, normalize, s, count, k0 + nk == n_images ? out : nullptr, st);
  }
}

}  // namespace

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

const char* ertm_last_error(void) { return g_error.c_str(); }

int32_t ertm_version(void) { return 1; }

int64_t ertm_launch_count(void) { return g_launches.load(); }

int32_t ertm_division_check(float h, int32_t mode, uint64_t* mismatches) {
  return guarded([&] {
    REQUIRE(mismatches && mode >= 0 && mode <= 3 && h > 0.f, "bad arguments");
    *mismatches = division_mismatches(h, mode, 0);
  });
}

int32_t ertm_set_tile_rows(int32_t rows) {
  return guarded([&] {
    REQUIRE(rows == 0 || rows == 8 || rows == 16 || rows == 32, "tile rows must be 0 (auto), 8, 16 or 32");
    g_tile_rows = rows;
  });
}

int32_t ertm_set_tile_split(int32_t mode) {
  return guarded([&] {
    REQUIRE(mode >= 0 && mode <= 2, "tile split mode must be 0 (automatic), 1 (never) or 2 (always)");
    g_tile_split.store(mode);
  });
}

int32_t ertm_set_tick_lanes(int32_t lanes) {
  return guarded([&] {
    REQUIRE(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4, "tick lanes must be 0 (automatic), 1, 2 or 4");
    g_tick_lanes.store(lanes);
  });
}

int32_t ertm_set_march(int32_t enable) {
  return guarded([&] {
    REQUIRE(enable == 0 || enable == 1 || enable == 2 || enable == 4 || enable == 8,
            "march must be 0 (tiles) or 2, 4, 8 chunks per segment (1: 8)");
    g_march.store(enable == 1 ? 8 : enable);
  });
}

int32_t ertm_set_march_stress(int32_t enable) {
  return guarded([&] {
    REQUIRE(enable == 0 || enable == 1, "march_stress must be 0 or 1");
    g_march_stress.store(enable);
  });
}

int32_t ertm_set_line_threads(int32_t threads) {
  return guarded([&] {
    REQUIRE(threads == 0 || (threads >= 64 && threads <= 1024 && threads % 32 == 0),
            "threads must be 0 (automatic) or a multiple of 32 in [64, 1024]");
    g_line_threads = threads;
  });
}

int32_t ertm_set_frame_rows(int32_t rows) {
  return guarded([&] {
    REQUIRE(rows == 0 || rows == 8 || rows == 16, "frame tile height must be 0 (the interior's), 8 or 16");
    g_frame_rows.store(rows);
  });
}

int32_t ertm_set_lane_assign(int32_t mode) {
  return guarded([&] {
    REQUIRE(mode == 0 || mode == 1, "lane assignment must be 0 (alternate works) or 1 (alternate shots)");
    g_lane_assign.store(mode);
  });
}

int32_t ertm_set_tma(int32_t enable) {
  return guarded([&] { g_tma.store(enable ? 1 : 0); });
}

int64_t ertm_stage_timeouts(void) {
  unsigned int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_stage_timeouts, sizeof v) != cudaSuccess) return -1;
  return (int64_t)v;
}

int32_t ertm_set_autotune(int32_t enable) {
  return guarded([&] {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_autotune.store(enable > 0 ? 1 : 0);
    if (enable < 0) {                 // forget earlier choices (and keep tuning off)
      for (TuneSample& t : g_tune_pending) {
        CK(cudaEventSynchronize(t.e1));
        g_tune_events.push_back(t.e0);
        g_tune_events.push_back(t.e1);
      }
      g_tune_pending.clear();
      g_tune.clear();
    }
  });
}

const char* ertm_autotune_report(void) {
  static std::string report;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  tune_collect();
  report.clear();
  for (auto& kv : g_tune) {
    const TuneState& ts = kv.second;
    char line[256];
    std::snprintf(line, sizeof line, "engine %d order %d works %d cells 2^%d:", std::get<0>(kv.first),
                  2 * std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first));
    report += line;
    for (size_t c = 0; c < ts.cands.size(); ++c) {
      std::snprintf(line, sizeof line, " %s%d/%d/%d=%.1fus", (int)c == ts.best ? "*" : "", ts.cands[c].tz,
                    ts.cands[c].split, ts.cands[c].lanes, ts.n[c] ? 1e3 * ts.sum_ms[c] / ts.n[c] : -1.0);
      report += line;
    }
    report += "\n";
  }
  return report.c_str();
}

int32_t ertm_profile_stencil(int32_t enable, int32_t every) {
  return guarded([&] {
    g_prof.drain();
    g_prof.on = enable != 0;
    g_prof.every = every > 0 ? every : 1;
    g_prof.counter = 0;
    g_prof.total_ms = 0.0;
    g_prof.total_bytes = 0.0;
    g_prof.samples = 0;
  });
}

int32_t ertm_profile_read(double* total_ms, int64_t* samples, double* total_bytes) {
  return guarded([&] {
    REQUIRE(total_ms && samples, "null argument");
    g_prof.drain();
    *total_ms = g_prof.total_ms;
    *samples = g_prof.samples;
    if (total_bytes) *total_bytes = g_prof.total_bytes;
  });
}

int32_t ertm_init(int32_t device) {
  return guarded([&] {
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    REQUIRE(device >= 0 && device < n, "no such CUDA device");
    CK(cudaSetDevice(device));
    // keep freed stream-ordered allocations in the pool between calls
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    cudaDeviceProp prop{};
    CK(cudaGetDeviceProperties(&prop, device));
    REQUIRE(prop.major == 10, "this library is built for sm_100a (B200); found sm_" +
                                  std::to_string(prop.major) + std::to_string(prop.minor));
  });
}

void* ertm_prop_create(const ertm_prop_config* cfg, const float* vp, const float* vs, const float* rho,
                       const float* pml_ax, const float* pml_bx, const float* pml_az, const float* pml_bz,
                       const uint8_t* qidx, const double* tau, const double* delta, const double* mref,
                       const float* relax_a, void* stream) {
  Prop* out = nullptr;
  int rc = guarded([&] { out = create(cfg, vp, vs, rho, pml_ax, pml_bx, pml_az, pml_bz, qidx, tau, delta, mref,
                                      relax_a, stream); });
  return rc == ERTM_OK ? out : nullptr;
}

void ertm_prop_destroy(void* prop) {
  if (!prop) return;
  Prop* P = static_cast<Prop*>(prop);
  cudaStreamSynchronize(P->st);
  delete P;
}

int32_t ertm_prop_info_get(void* prop, ertm_prop_info* info) {
  return guarded([&] {
    REQUIRE(prop && info, "null argument");
    Prop& P = *static_cast<Prop*>(prop);
    info->nzp = P.h.nzp;
    info->nxp = P.h.nxp;
    info->ld = P.h.ld;
    info->pad = P.h.pad;
    info->state_bytes = (int64_t)P.state_floats * 4;
    info->field_bytes = (int64_t)P.h.n_fields * P.h.nzp * P.h.nxp * 4;
    info->step_index = P.step_index;
    info->n_fields = P.h.n_fields;
    StabState s{};
    CK(cudaMemcpyAsync(&s, P.stab.p, sizeof(s), cudaMemcpyDeviceToHost, P.st));
    CK(cudaStreamSynchronize(P.st));
    info->clipped = s.clipped;
    info->lowpass_steps = P.lowpass_steps;
    info->n_receivers = (int32_t)P.rx.size();
    info->fast_div_x = P.h.fast_x;
    info->fast_div_z = P.h.fast_z;
    info->tile_rows = P.tz;
  });
}

int32_t ertm_prop_reset(void* prop) {
  return guarded([&] {
    REQUIRE(prop, "null propagator");
    Prop& P = *static_cast<Prop*>(prop);
    CK(cudaMemsetAsync(P.state.p, 0, P.state_floats * 4, P.st));
    CK(cudaMemsetAsync(P.stab.p, 0, sizeof(StabState), P.st));
    CK(cudaMemsetAsync(P.status.p, 0, sizeof(uint32_t), P.st));
    P.step_index = 0;
    P.lowpass_steps = 0;
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_set_source(void* prop, int32_t iz, int32_t ix, int32_t mechanism) {
  return guarded([&] {
    REQUIRE(prop, "null propagator");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(iz >= 0 && iz < P.h.nzp && ix >= 0 && ix < P.h.nxp, "source node outside the padded grid");
    REQUIRE(mechanism >= 0 && mechanism <= 2, "unknown mechanism");
    P.h.src_iz = iz;
    P.h.src_ix = ix;
    P.h.mech = mechanism;
    if (P.h.engine == ENGINE_VISCO) {
      CK(cudaMemcpyAsync(&P.k_src, P.h.coef[CV_KR] + (size_t)iz * P.h.ld + ix, 4, cudaMemcpyDeviceToHost, P.st));
    }
    P.sync_desc();
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_set_receivers(void* prop, int32_t n, const double* x, const double* z) {
  return guarded([&] {
    REQUIRE(prop && n >= 0 && (n == 0 || (x && z)), "bad receivers");
    Prop& P = *static_cast<Prop*>(prop);
    P.rx.assign(x, x + n);
    P.rz.assign(z, z + n);
    P.samples.clear();
    P.injects.clear();
  });
}

int32_t ertm_prop_step(void* prop, int32_t n_steps, const double* amps) {
  return guarded([&] {
    REQUIRE(prop && n_steps >= 0, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    for (int t = 0; t < n_steps; ++t) step_once(P, amps ? amps[t] : 0.0);
  });
}

int32_t ertm_prop_sample(void* prop, int32_t n_comp, const int32_t* comps, float* out) {
  return guarded([&] {
    REQUIRE(prop && n_comp >= 0 && (n_comp == 0 || comps), "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    const int n = (int)P.rx.size();
    if (n == 0 || n_comp == 0) return;
    DevBuf o((size_t)n_comp * n * 4, P.st);
    for (int c = 0; c < n_comp; ++c) {
      SamplePlanHost& sp = sample_plan(P, comps[c]);
      SampleSet S{};
      S.count = 1;
      S.plan[0] = SamplePlanDev{n, sp.kind, sp.slot, 0, sp.cell.as<int32_t>(), sp.valid.as<uint8_t>(),
                                sp.w.as<double>(), o.as<float>() + (size_t)c * n};
      k_sample<<<dim3((n + 127) / 128, 1), 128, 0, P.st>>>(P.dp(), 0, S, 0);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, o.p, o.bytes, cudaMemcpyDefault, P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_inject(void* prop, int32_t comp, const float* values) {
  return guarded([&] {
    REQUIRE(prop && values, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(!P.rx.empty(), "receivers must be set before injection");
    const int n = (int)P.rx.size();
    InjectPlanHost& plan = inject_plan(P, std::vector<int>{comp}, 1);
    DevBuf v((size_t)n * 4, P.st);
    upload(v.p, values, v.bytes, P.st);
    if (plan.n_cells)
      k_inject<<<(plan.n_cells + 127) / 128, 128, 0, P.st>>>(P.dp(), 0, plan.dev(), v.as<float>(), 0);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_image_field(void* prop, int32_t wave, int32_t separation, float* out) {
  return guarded([&] {
    REQUIRE(prop && out, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(wave == 0 || (wave == 1 && P.h.engine == ENGINE_ELASTIC), "wave not available for this engine");
    DevBuf o((size_t)P.h.nz * P.h.nx * 4, P.st);
    image_field(P, wave, separation, o.as<float>());
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, o.p, o.bytes, cudaMemcpyDefault, P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_read_field(void* prop, int32_t slot, float* out) {
  return guarded([&] {
    REQUIRE(prop && out, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(slot >= 0 && slot < P.h.n_fields, "bad field slot");
    CK(cudaMemcpy2DAsync(out, P.h.nxp * 4, P.field(slot), P.h.ld * 4, P.h.nxp * 4, P.h.nzp, cudaMemcpyDefault,
                         P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_write_field(void* prop, int32_t slot, const float* in) {
  return guarded([&] {
    REQUIRE(prop && in, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(slot >= 0 && slot < P.h.n_fields, "bad field slot");
    CK(cudaMemcpy2DAsync(P.field(slot), P.h.ld * 4, in, P.h.nxp * 4, P.h.nxp * 4, P.h.nzp, cudaMemcpyDefault,
                         P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

// ψ terms are stored as strips; these expand to / extract from full padded arrays.
int32_t ertm_prop_read_psi(void* prop, int32_t axis, int32_t term, float* out) {
  return guarded([&] {
    REQUIRE(prop && out, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(term >= 0 && term < P.n_psi && (axis == 0 || axis == 1), "bad psi term");
    const int nzp = P.h.nzp, nxp = P.h.nxp;
    std::vector<float> full((size_t)nzp * nxp, 0.f);
    if (axis == 1 && P.h.wx > 0) {
      std::vector<float> s((size_t)nzp * P.h.wx);
      CK(cudaMemcpyAsync(s.data(), P.h.psix[term], s.size() * 4, cudaMemcpyDeviceToHost, P.st));
      CK(cudaStreamSynchronize(P.st));
      for (int i = 0; i < nzp; ++i)
        for (int c = 0; c < P.h.wx; ++c) {
          const int j = c < P.h.npx_l ? c : nxp - P.h.npx_r + (c - P.h.npx_l);
          full[(size_t)i * nxp + j] = s[(size_t)i * P.h.wx + c];
        }
    }
    if (axis == 0 && P.h.hz_rows > 0) {
      std::vector<float> s((size_t)P.h.hz_rows * P.h.ld);
      CK(cudaMemcpyAsync(s.data(), P.h.psiz[term], s.size() * 4, cudaMemcpyDeviceToHost, P.st));
      CK(cudaStreamSynchronize(P.st));
      for (int r = 0; r < P.h.hz_rows; ++r) {
        const int i = r < P.h.npz_t ? r : nzp - P.h.npz_b + (r - P.h.npz_t);
        std::memcpy(&full[(size_t)i * nxp], &s[(size_t)r * P.h.ld], nxp * 4);
      }
    }
    CK(cudaMemcpy(out, full.data(), full.size() * 4, cudaMemcpyDefault));
  });
}

int32_t ertm_prop_write_psi(void* prop, int32_t axis, int32_t term, const float* in) {
  return guarded([&] {
    REQUIRE(prop && in, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    REQUIRE(term >= 0 && term < P.n_psi && (axis == 0 || axis == 1), "bad psi term");
    const int nzp = P.h.nzp, nxp = P.h.nxp;
    std::vector<float> full((size_t)nzp * nxp);
    CK(cudaMemcpy(full.data(), in, full.size() * 4, cudaMemcpyDefault));
    if (axis == 1 && P.h.wx > 0) {
      std::vector<float> s((size_t)nzp * P.h.wx);
      for (int i = 0; i < nzp; ++i)
        for (int c = 0; c < P.h.wx; ++c) {
          const int j = c < P.h.npx_l ? c : nxp - P.h.npx_r + (c - P.h.npx_l);
          s[(size_t)i * P.h.wx + c] = full[(size_t)i * nxp + j];
        }
      CK(cudaMemcpyAsync(P.h.psix[term], s.data(), s.size() * 4, cudaMemcpyHostToDevice, P.st));
      CK(cudaStreamSynchronize(P.st));
    }
    if (axis == 0 && P.h.hz_rows > 0) {
      std::vector<float> s((size_t)P.h.hz_rows * P.h.ld, 0.f);
      for (int r = 0; r < P.h.hz_rows; ++r) {
        const int i = r < P.h.npz_t ? r : nzp - P.h.npz_b + (r - P.h.npz_t);
        std::memcpy(&s[(size_t)r * P.h.ld], &full[(size_t)i * nxp], nxp * 4);
      }
      CK(cudaMemcpyAsync(P.h.psiz[term], s.data(), s.size() * 4, cudaMemcpyHostToDevice, P.st));
      CK(cudaStreamSynchronize(P.st));
    }
  });
}

int32_t ertm_prop_set_step_index(void* prop, int64_t step_index) {
  return guarded([&] {
    REQUIRE(prop && step_index >= 0, "bad arguments");
    static_cast<Prop*>(prop)->step_index = step_index;
  });
}

int32_t ertm_prop_save_state(void* prop, void* dst) {
  return guarded([&] {
    REQUIRE(prop && dst, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    CK(cudaMemcpyAsync(dst, P.state.p, P.state_floats * 4, cudaMemcpyDefault, P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_prop_load_state(void* prop, const void* src) {
  return guarded([&] {
    REQUIRE(prop && src, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    CK(cudaMemcpyAsync(P.state.p, src, P.state_floats * 4, cudaMemcpyDefault, P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_forward(void* prop, int32_t nt, const float* amps, int32_t n_comp, const int32_t* comps, float* out) {
  return guarded([&] {
    REQUIRE(prop && nt >= 0 && n_comp >= 0 && n_comp <= MAX_SAMPLE, "bad arguments");
    Prop& P = *static_cast<Prop*>(prop);
    const int n = (int)P.rx.size();
    const bool sampling = n > 0 && n_comp > 0;
    DevBuf o(sampling ? (size_t)n_comp * nt * n * 4 : 0, P.st);
    SampleSet S{};
    if (sampling) {
      S.count = n_comp;
      for (int c = 0; c < n_comp; ++c) {
        SamplePlanHost& sp = sample_plan(P, comps[c]);
        S.plan[c] = SamplePlanDev{n, sp.kind, sp.slot, 0, sp.cell.as<int32_t>(), sp.valid.as<uint8_t>(),
                                  sp.w.as<double>(), o.as<float>() + (size_t)c * nt * n};
      }
    }
    DevBuf dwave(amps ? (size_t)nt * 4 : 0, P.st);
    if (amps) upload(dwave.p, amps, (size_t)nt * 4, P.st);
    for (int t = 0; t < nt; ++t) {
      if (amps) step_once(P, 0.0, dwave.as<float>(), t);
      else step_once(P, 0.0);
      if (sampling) {
        k_sample<<<dim3((n + 127) / 128, n_comp), 128, 0, P.st>>>(P.dp(), 0, S, (int64_t)t * n);
        ++g_launches;
      }
    }
    CK(cudaGetLastError());
    if (sampling) CK(cudaMemcpyAsync(out, o.p, o.bytes, cudaMemcpyDefault, P.st));
    CK(cudaStreamSynchronize(P.st));
  });
}

int32_t ertm_migrate(void* fwd, void* back, const ertm_migrate_config* cfg, const float* wavelet,
                     const float* record, double* num, double* illum, double* rillum) {
  return guarded([&] {
    REQUIRE(fwd && back && cfg && wavelet, "bad arguments");
    REQUIRE(cfg->n_comp == 0 || record, "record missing");
    migrate(*static_cast<Prop*>(fwd), *static_cast<Prop*>(back), *cfg, wavelet, record, num, illum, rillum);
  });
}

int32_t ertm_migrate_batch(int32_t n_shots, const ertm_batch_shot* shots) {
  return guarded([&] {
    REQUIRE(n_shots >= 1 && shots, "bad arguments");
    cudaStream_t st = static_cast<Prop*>(shots[0].fwd)->st;
    std::vector<ShotRun> runs(n_shots);
    for (int k = 0; k < n_shots; ++k) {
      const ertm_batch_shot& S = shots[k];
      REQUIRE(S.fwd && S.back && S.wavelet, "shot " + std::to_string(k) + ": missing propagator or wavelet");
      REQUIRE(S.cfg.n_comp == 0 || S.record, "shot " + std::to_string(k) + ": record missing");
      for (int q = 0; q < k; ++q)
        REQUIRE(shots[q].fwd != S.fwd && shots[q].back != S.back && shots[q].fwd != S.back && shots[q].back != S.fwd,
                "every shot needs its own pair of propagators");
      prepare_run(runs[k], *static_cast<Prop*>(S.fwd), *static_cast<Prop*>(S.back), S.cfg, S.wavelet, S.record,
                  S.num, S.illum, S.rillum, st, 2);
    }
    migrate_batch(runs, st);
  });
}

int32_t ertm_session_create(void** out) {
  return guarded([&] {
    REQUIRE(out, "bad arguments");
    // The session works on the legacy default stream: work the caller queued
    // there (inputs, output buffers) is ordered before its ticks, and buffers
    // the session creates inside a propagator (injection and sampling plans)
    // are freed on a stream that outlives the session.
    auto S = std::make_unique<Session>();
    S->st = nullptr;
    *out = S.release();
  });
}

int32_t ertm_session_add(void* session, const ertm_batch_shot* shot, int64_t tag) {
  return guarded([&] {
    REQUIRE(session && shot, "bad arguments");
    Session& S = *static_cast<Session*>(session);
    const ertm_batch_shot& B = *shot;
    REQUIRE(B.fwd && B.back && B.wavelet, "missing propagator or wavelet");
    REQUIRE(B.fwd != B.back, "a shot needs two propagators");
    REQUIRE(B.cfg.n_comp == 0 || B.record, "record missing");
    for (auto& R : S.runs)
      REQUIRE(R->F != B.fwd && R->B != B.back && R->F != B.back && R->B != B.fwd,
              "the propagators are in use by another shot of the session");
    for (int64_t t : S.tags) REQUIRE(t != tag, "tag already in use");
    auto R = std::make_unique<ShotRun>();
    prepare_run(*R, *static_cast<Prop*>(B.fwd), *static_cast<Prop*>(B.back), B.cfg, B.wavelet, B.record, B.num,
                B.illum, B.rillum, S.st, 2);
    S.runs.push_back(std::move(R));
    S.tags.push_back(tag);
    S.dirty = true;
  });
}

int32_t ertm_session_advance(void* session, int32_t max_ticks, int64_t* done_tags, int32_t cap, int32_t* n_done) {
  return guarded([&] {
    REQUIRE(session && n_done && max_ticks >= 0 && cap >= 0 && (done_tags || cap == 0), "bad arguments");
    Session& S = *static_cast<Session*>(session);
    *n_done = 0;
    std::vector<ShotRun*> ptrs;
    for (auto& R : S.runs) ptrs.push_back(R.get());
    if (S.dirty) {
      upload_table(ptrs, S.table, S.dtable, S.st);
      S.dirty = false;
    }
    auto any_done = [&] {
      for (ShotRun* R : ptrs)
        if (R->phase == 4) return true;
      return false;
    };
    for (int k = 0; k < max_ticks && !any_done(); ++k) {
      if (!batch_tick(ptrs, S.dtable.as<DevProp>(), S.st)) break;
      ++S.ticks;
    }
    // shots whose wavefields became non-finite leave the session; the others run on
    const int n_tab = (int)S.table.size();
    if (n_tab > 0) {
      if (S.status.bytes < (size_t)n_tab * 4) S.status = DevBuf((size_t)n_tab * 4, S.st);
      k_gather_status<<<(n_tab + 127) / 128, 128, 0, S.st>>>(S.dtable.as<DevProp>(), n_tab, S.status.as<uint32_t>());
      ++g_launches;
      std::vector<uint32_t> flags(n_tab);
      CK(cudaMemcpyAsync(flags.data(), S.status.p, (size_t)n_tab * 4, cudaMemcpyDeviceToHost, S.st));
      CK(cudaStreamSynchronize(S.st));
      for (size_t i = 0; i < S.runs.size();) {
        const ShotRun& R = *S.runs[i];
        if (!((flags[R.fi] | flags[R.bi]) & STATUS_NONFINITE)) {
          ++i;
          continue;
        }
        release_streams(*S.runs[i], S.st);
        S.failed.push_back(S.tags[i]);
        S.runs.erase(S.runs.begin() + (std::ptrdiff_t)i);
        S.tags.erase(S.tags.begin() + (std::ptrdiff_t)i);
        S.dirty = true;
      }
    }
    for (size_t i = 0; i < S.runs.size() && *n_done < cap;) {
      if (S.runs[i]->phase != 4) {
        ++i;
        continue;
      }
      finish_run(*S.runs[i], S.st);
      release_streams(*S.runs[i], S.st);
      done_tags[(*n_done)++] = S.tags[i];
      S.runs.erase(S.runs.begin() + (std::ptrdiff_t)i);
      S.tags.erase(S.tags.begin() + (std::ptrdiff_t)i);
      S.dirty = true;
    }
  });
}

int32_t ertm_session_take_failed(void* session, int64_t* tags, int32_t cap, int32_t* n) {
  return guarded([&] {
    REQUIRE(session && n && cap >= 0 && (tags || cap == 0), "bad arguments");
    Session& S = *static_cast<Session*>(session);
    const int32_t k = (int32_t)std::min<size_t>((size_t)cap, S.failed.size());
    for (int32_t i = 0; i < k; ++i) tags[i] = S.failed[i];
    S.failed.erase(S.failed.begin(), S.failed.begin() + k);
    *n = k;
  });
}

int32_t ertm_prop_status(void* prop, uint32_t* status) {
  return guarded([&] {
    REQUIRE(prop && status, "bad arguments");
    const Prop& P = *static_cast<Prop*>(prop);
    *status = read_status(P, P.st);
  });
}

int32_t ertm_session_active(void* session) {
  return session ? (int32_t) static_cast<Session*>(session)->runs.size() : 0;
}

int64_t ertm_session_ticks(void* session) { return session ? static_cast<Session*>(session)->ticks : 0; }

int32_t ertm_session_destroy(void* session) {
  return guarded([&] {
    if (!session) return;
    std::unique_ptr<Session> S(static_cast<Session*>(session));
    cudaStreamSynchronize(S->st);
    for (auto& R : S->runs) {
      R->F->st = R->f_st0;
      R->B->st = R->b_st0;
    }
    S->runs.clear();
    S->dtable = DevBuf();
    CK(cudaStreamSynchronize(S->st));
  });
}

int32_t ertm_postprocess(int32_t nz, int32_t nx, double dx, double dz, const double* num, const double* illum,
                         const double* rillum, int32_t by_illum, int32_t by_rillum, double eps, int32_t laplacian,
                         double lowpass, int32_t npml, int32_t top_mask, float* out, void* stream) {
  return guarded([&] {
    REQUIRE(nz >= 1 && nx >= 1 && num && out, "bad arguments");
    REQUIRE(!by_illum || illum, "illumination missing");
    REQUIRE(!by_rillum || rillum, "receiver illumination missing");
    REQUIRE(lowpass > 0.0 && lowpass <= 1.0, "lowpass fraction must lie in (0, 1]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = (int64_t)nz * nx;
    DevBuf in(n * 8 * 3, st), a(n * 8, st), b(n * 8, st), o(n * 4, st);
    double* dn = in.as<double>();
    upload(dn, num, n * 8, st);
    if (by_illum) upload(dn + n, illum, n * 8, st);
    if (by_rillum) upload(dn + 2 * n, rillum, n * 8, st);
    NormArgs A{};
    A.num = dn;
    A.illum = dn + n;
    A.rillum = dn + 2 * n;
    A.by_illum = by_illum;
    A.by_rillum = by_rillum;
    A.eps = eps;
    A.out = a.as<double>();
    A.n = n;
    k_normalize<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A);
    const dim3 b2(32, 8), g2((nx + 31) / 32, (nz + 7) / 8);
    double* cur = a.as<double>();
    double* other = b.as<double>();
    if (laplacian) {
      k_laplacian<<<g2, b2, 0, st>>>(cur, other, nz, nx, dx, dz);
      std::swap(cur, other);
    }
    g_launches += 2 + (laplacian ? 1 : 0);
    if (lowpass < 1.0) {
      DevBuf wa((size_t)n * sizeof(double2), st), wb((size_t)n * sizeof(double2), st);
      lowpass2d_one(nz, nx, dz, dx, lowpass, cur, false, nx, other, false, nx, wa.as<double2>(), wb.as<double2>(),
                    st);
      std::swap(cur, other);
    }
    k_mask_cast<<<g2, b2, 0, st>>>(cur, o.as<float>(), nz, nx, npml, top_mask);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, o.p, n * 4, cudaMemcpyDefault, st));
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_lowpass_wavenumber(int32_t nz, int32_t nx, double dx, double dz, double cutoff, const double* in,
                                double* out, void* stream) {
  return guarded([&] {
    REQUIRE(nz >= 1 && nx >= 1 && in && out, "bad arguments");
    REQUIRE(cutoff > 0.0 && cutoff <= 1.0, "cutoff fraction must lie in (0, 1]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = (size_t)nz * nx;
    InArray a(in, n * 8, st);
    OutArray b(out, n * 8, st);
    DevBuf wa(n * sizeof(double2), st), wb(n * sizeof(double2), st);
    lowpass2d_one(nz, nx, dz, dx, cutoff, a.as<double>(), false, nx, b.d, false, nx, wa.as<double2>(),
              wb.as<double2>(), st);
    b.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_resample(const float* in, int64_t n_in, int64_t ntr, const double* w, const int64_t* off0, int32_t taps,
                      int64_t n_out, float* out, void* stream) {
  return guarded([&] {
    REQUIRE(in && w && off0 && out && n_in >= 1 && ntr >= 1 && n_out >= 1 && taps >= 1, "bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    InArray a(in, (size_t)n_in * ntr * 4, st), W(w, (size_t)n_out * taps * 8, st), O(off0, (size_t)n_out * 8, st);
    OutArray b(out, (size_t)n_out * ntr * 4, st);
    k_resample<<<records_grid(ntr, n_out), 128, 0, st>>>(a.as<float>(), n_in, ntr, W.as<double>(), O.as<int64_t>(),
                                                        taps, n_out, b.as<float>());
    ++g_launches;
    CK(cudaGetLastError());
    b.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_mute(const float* in, int64_t nt, int64_t ntr, const double* t, const double* start, const double* end,
                  float* out, void* stream) {
  return guarded([&] {
    REQUIRE(in && t && start && end && out && nt >= 1 && ntr >= 1, "bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    InArray a(in, (size_t)nt * ntr * 4, st), T(t, (size_t)nt * 8, st), S(start, (size_t)ntr * 8, st),
        E(end, (size_t)ntr * 8, st);
    OutArray b(out, (size_t)nt * ntr * 4, st);
    k_mute<<<records_grid(ntr, nt), 128, 0, st>>>(a.as<float>(), nt, ntr, T.as<double>(), S.as<double>(),
                                                 E.as<double>(), b.as<float>());
    ++g_launches;
    CK(cudaGetLastError());
    b.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_taper(const float* in, int64_t nt, int64_t ntr, const double* ramp, int64_t w, float* out,
                   void* stream) {
  return guarded([&] {
    REQUIRE(in && ramp && out && nt >= 1 && ntr >= 1 && w >= 1 && w <= nt, "bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    InArray a(in, (size_t)nt * ntr * 4, st), R(ramp, (size_t)w * 8, st);
    OutArray b(out, (size_t)nt * ntr * 4, st);
    k_taper<<<records_grid(ntr, nt), 128, 0, st>>>(a.as<float>(), nt, ntr, R.as<double>(), w, b.as<float>());
    ++g_launches;
    CK(cudaGetLastError());
    b.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_rotate(const float* vx, const float* vz, int64_t n, double c, double s, float* ox, float* oz,
                    void* stream) {
  return guarded([&] {
    REQUIRE(vx && vz && ox && oz && n >= 1, "bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    InArray a(vx, (size_t)n * 4, st), b(vz, (size_t)n * 4, st);
    OutArray x(ox, (size_t)n * 4, st), z(oz, (size_t)n * 4, st);
    k_rotate<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.as<float>(), b.as<float>(), n, c, s, x.as<float>(),
                                                          z.as<float>());
    ++g_launches;
    CK(cudaGetLastError());
    x.finish();
    z.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_stft_filter(const double* in, int64_t n, int64_t ntr, int32_t L, int32_t hop, int32_t S,
                         const double* window, const double* response, double* out, void* stream) {
  return guarded([&] {
    REQUIRE(in && window && response && out && n >= 1 && ntr >= 1 && L >= 8 && hop >= 1 && S >= 1,
            "bad arguments");
    REQUIRE((int64_t)(S - 1) * hop < n, "more frames than the record holds");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int F = L / 2 + 1;
    InArray a(in, (size_t)n * ntr * 8, st), W(window, (size_t)L * 8, st), R(response, (size_t)S * F * 16, st);
    OutArray o(out, (size_t)n * ntr * 8, st);
    const int64_t batch = (int64_t)S * ntr;
    DevBuf frames((size_t)batch * L * 8, st), spec((size_t)batch * F * 16, st);
    const int64_t nf = batch * L;
    k_stft_frames<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(a.as<double>(), n, ntr, L, hop, S, W.as<double>(),
                                                               frames.as<double>());
    REQUIRE(batch <= INT32_MAX, "too many frames for one batched transform");
    const FftPair plan = stft_fft(L, batch, st);
    CKFFT(cufftExecD2Z(plan.fwd, frames.as<cufftDoubleReal>(), spec.as<cufftDoubleComplex>()));
    const int64_t ns = batch * F;
    k_stft_response<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(spec.as<double2>(), ntr, F, S, R.as<double2>());
    CKFFT(cufftExecZ2D(plan.inv, spec.as<cufftDoubleComplex>(), frames.as<cufftDoubleReal>()));
    const int64_t no = n * ntr;
    k_stft_overlap_add<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(frames.as<double>(), n, ntr, L, hop, S,
                                                                    W.as<double>(), o.as<double>());
    g_launches += 3;
    CK(cudaGetLastError());
    o.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_segy_decode(const uint8_t* traces, int64_t n_traces, int64_t ns, int32_t fmt, int64_t ncols,
                         const int32_t* order, const int64_t* dest, const int32_t* width, float* out,
                         int64_t out_len, void* stream) {
  return guarded([&] {
    REQUIRE(traces && order && dest && width && out && n_traces >= 1 && ns >= 1 && ncols >= 1 && out_len >= 1,
            "bad arguments");
    REQUIRE(fmt == 1 || fmt == 5, "data sample format must be 1 (IBM float) or 5 (IEEE float)");
    REQUIRE(!is_device_ptr(order) && !is_device_ptr(dest) && !is_device_ptr(width),
            "column maps are host arrays");
    for (int64_t c = 0; c < ncols; ++c) {
      REQUIRE(order[c] >= 0 && order[c] < n_traces, "column reads a trace outside the file");
      REQUIRE(width[c] >= 1 && dest[c] >= 0 && dest[c] + (ns - 1) * (int64_t)width[c] < out_len,
              "column writes outside the output");
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t tb = 240 + 4 * ns;
    InArray t(traces, (size_t)(n_traces * tb), st);
    REQUIRE(reinterpret_cast<uintptr_t>(t.d) % 4 == 0, "trace section must be 4-byte aligned");
    InArray o_(order, (size_t)ncols * 4, st), d_(dest, (size_t)ncols * 8, st), w_(width, (size_t)ncols * 4, st);
    OutArray o(out, (size_t)out_len * 4, st);
    if (o.host) CK(cudaMemsetAsync(o.d, 0, o.bytes, st));
    const dim3 grid((unsigned)((ncols + 31) / 32), (unsigned)((ns + 31) / 32));
    REQUIRE(grid.y <= 65535u, "too many samples per trace");
    k_segy_decode<<<grid, dim3(32, 8), 0, st>>>(t.as<uint8_t>(), ns, tb, ncols, o_.as<int32_t>(),
                                               d_.as<int64_t>(), w_.as<int32_t>(), fmt, o.as<float>());
    ++g_launches;
    CK(cudaGetLastError());
    o.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_segy_encode(const float* rec, int64_t ns, int64_t ntr, int32_t fmt, const uint8_t* headers,
                         uint8_t* traces, void* stream) {
  return guarded([&] {
    REQUIRE(rec && headers && traces && ns >= 1 && ntr >= 1, "bad arguments");
    REQUIRE(fmt == 1 || fmt == 5, "data sample format must be 1 (IBM float) or 5 (IEEE float)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t tb = 240 + 4 * ns;
    InArray r(rec, (size_t)(ns * ntr) * 4, st), h(headers, (size_t)ntr * 240, st);
    REQUIRE(reinterpret_cast<uintptr_t>(h.d) % 4 == 0, "headers must be 4-byte aligned");
    OutArray o(traces, (size_t)(ntr * tb), st);
    REQUIRE(reinterpret_cast<uintptr_t>(o.d) % 4 == 0, "trace section must be 4-byte aligned");
    const dim3 grid((unsigned)((ntr + 31) / 32), (unsigned)((ns + 31) / 32));
    REQUIRE(grid.y <= 65535u, "too many samples per trace");
    const int64_t nh = ntr * 60;
    k_segy_headers<<<(unsigned)((nh + 255) / 256), 256, 0, st>>>(h.as<uint32_t>(), ntr, tb, o.as<uint8_t>());
    k_segy_encode<<<grid, dim3(32, 8), 0, st>>>(r.as<float>(), ns, ntr, tb, fmt, o.as<uint8_t>());
    g_launches += 2;
    CK(cudaGetLastError());
    o.finish();
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_stack(int32_t n_images, int64_t n, const float* const* images, int32_t normalize, float* out,
                   void* stream) {
  return guarded([&] {
    REQUIRE(n_images >= 1 && n >= 1 && images && out, "bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_images == 1) {
      CK(cudaMemcpyAsync(out, images[0], n * 4, cudaMemcpyDefault, st));
      CK(cudaStreamSynchronize(st));
      return;
    }
    const bool dev_out = is_device_ptr(out);
    DevBuf o(dev_out ? 0 : n * 4, st);
    stack_all(n_images, n, images, normalize != 0, nullptr, n_images, dev_out ? out : o.as<float>(), st);
    if (!dev_out) CK(cudaMemcpyAsync(out, o.p, n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_stack_partial(int32_t n_images, int64_t n, const float* const* images, int32_t normalize, double* sum,
                           void* stream) {
  return guarded([&] {
    REQUIRE(n_images >= 0 && n >= 1 && (images || n_images == 0) && sum, "bad arguments");
    require_device_pointer(sum, "sum");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    stack_all(n_images, n, images, normalize != 0, sum, 1, nullptr, st);
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_stack_finish(int64_t n, const double* sum, int64_t count, float* out, void* stream) {
  return guarded([&] {
    REQUIRE(n >= 1 && sum && out && count >= 1, "bad arguments");
    require_device_pointer(sum, "sum");
    require_device_pointer(out, "out");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_stack_finish<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(sum, n, (int)count, out);
    ++g_launches;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
  });
}

int32_t ertm_stack_noalloc(int32_t n_images, int64_t n, const float* const* images, int32_t normalize, float* out,
                           void* stream) {
  return guarded([&] {
    REQUIRE(n_images >= 1 && n >= 1 && images && out, "bad arguments");
    REQUIRE(n_images <= kStackMaxImages,
            "ertm_stack_noalloc stacks at most " + std::to_string(kStackMaxImages) + " images per call");
    require_device_pointer(out, "out");
    for (int k = 0; k < n_images; ++k) require_device_pointer(images[k], "every image");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_images == 1) {
      CK(cudaMemcpyAsync(out, images[0], n * 4, cudaMemcpyDeviceToDevice, st));
      return;
    }
    const StackScratch S = stack_scratch();
    // the scratch keeps the previous call's contents: clear what must start at zero
    CK(cudaMemsetAsync(S.scale, 0, sizeof(unsigned int) * n_images, st));
    if (normalize) {
      const unsigned g = (unsigned)std::min<int64_t>((n + 255) / 256, 1184);
      for (int k = 0; k < n_images; ++k) k_absmax_f32<<<g, 256, 0, st>>>(images[k], n, S.scale + k);
      g_launches += n_images;
    }
    for (int64_t off = 0; off < n; off += kStackChunk) {
      const int64_t len = std::min<int64_t>(kStackChunk, n - off);
      const unsigned g = (unsigned)((len + 255) / 256);
      CK(cudaMemsetAsync(S.sum, 0, sizeof(double) * len, st));
      for (int k = 0; k < n_images; ++k)
        k_stack_add<<<g, 256, 0, st>>>(images[k] + off, len, S.scale + k, normalize, S.sum);
      k_stack_finish<<<g, 256, 0, st>>>(S.sum, len, n_images, out + off);
      g_launches += n_images + 1;
    }
    CK(cudaGetLastError());
  });
}

}  // extern "C"
