// Device-side data structures and exact-order arithmetic helpers for the
// ERTM staggered-grid stencils on sm_100a.
//
// Every floating-point operation of the hot path is written with the
// round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, __dadd_rn …)
// so that nvcc never contracts a*b+c into an FMA.  The operation order
// follows the reference NumPy code (ertm/numerics.py, ertm/propagation.py,
// ertm/imaging.py), which makes the GPU fields equal to the reference's
// float32 fields bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ertm {

enum Engine : int32_t { ENGINE_ACOUSTIC = 0, ENGINE_ELASTIC = 1, ENGINE_VISCO = 2 };
enum Mechanism : int32_t { MECH_EXPLOSIVE = 0, MECH_SHEAR = 1, MECH_FORCE_Z = 2 };

// Field slots.  Acoustic: p vx vz.  Elastic: vx vz sxx szz sxz.
// Viscoacoustic: p vx vz eps r0..r(L-1).
constexpr int A_P = 0, A_VX = 1, A_VZ = 2;
constexpr int E_VX = 0, E_VZ = 1, E_SXX = 2, E_SZZ = 3, E_SXZ = 4;
constexpr int V_P = 0, V_VX = 1, V_VZ = 2, V_EPS = 3, V_R0 = 4;
constexpr int MAX_FIELDS = 12;   // visco with up to 8 mechanisms
constexpr int MAX_MECH = 8;
constexpr int MAX_PSI = 4;       // per axis (elastic: 4 x-terms + 4 z-terms)

// Per-cell coefficient slots.  Acoustic: kappa irx irz.  Elastic: lam l2m
// muxz irx irz.  Visco: kR irx irz b0..b(L-1) (the a_l come from a per-Q
// table indexed by qidx).
constexpr int CA_KAPPA = 0, CA_IRX = 1, CA_IRZ = 2;
constexpr int CE_LAM = 0, CE_L2M = 1, CE_MUXZ = 2, CE_IRX = 3, CE_IRZ = 4;
constexpr int CV_KR = 0, CV_IRX = 1, CV_IRZ = 2, CV_B0 = 3;
constexpr int MAX_COEF = 3 + MAX_MECH;

// x-strip ψ terms per engine (order of use inside the kernels)
//   acoustic/visco: 0 vx_dp_dx, 1 p_dvx_dx
//   elastic:        0 vx_dsxx, 1 vz_dsxz, 2 sxx_dvx, 3 sxz_dvz
// z-strip ψ terms
//   acoustic/visco: 0 vz_dp_dz, 1 p_dvz_dz
//   elastic:        0 vx_dsxz, 1 vz_dszz, 2 szz_dvz, 3 sxz_dvx

struct DevProp {
  int32_t engine;
  int32_t M;            // half stencil width (order/2); pad = M + 1
  int32_t nzp, nxp;     // padded grid (reference geometry)
  int32_t ld;           // row pitch in floats (multiple of 32)
  int32_t nz, nx, pad;  // physical grid
  int32_t L;            // visco mechanisms
  int32_t n_fields;
  float c[4];           // float32 stencil coefficients (unused ones = 0)
  float hx, hz, dt;     // float32 spacing and time step
  double rx, rz;        // RN64(1/hx), RN64(1/hz)
  float rx32, rz32;     // RN32(1/hx), RN32(1/hz)
  float rxl, rzl;       // RN32(1/h − RN32(1/h)) for the one-FMA form
  int32_t fast_x, fast_z;  // division mode by hx / hz (see divh)
  int32_t npx_l, npx_r; // x-strip widths (0 when absent)
  int32_t npz_t, npz_b; // z-strip widths (top is 0 under a free surface)
  int32_t wx;           // npx_l + npx_r
  int32_t hz_rows;      // npz_t + npz_b
  const float* ax; const float* bx;   // x profiles, length nxp
  const float* az; const float* bz;   // z profiles, length nzp
  float* f[MAX_FIELDS];
  float* psix[MAX_PSI];               // [nzp][wx]
  float* psiz[MAX_PSI];               // [hz_rows][ld]
  const float* coef[MAX_COEF];
  const uint8_t* qidx;                // visco: per-cell Q index into relax_a
  const float* relax_a;               // visco: [n_q][L] float32 a_l table
  int32_t src_iz, src_ix, mech;       // source node (padded indices), mechanism
  int32_t free_surface;               // 1: zero the free-surface row (acoustic/elastic)
  const void* tmap;                   // 9 tensor maps (tile heights 8/16/32 × halo/cell/coef) or null
  float* peak;                        // visco compensation: max|p| of the last step (float bits)
  uint32_t* status;                   // STATUS_* bits, set by the stress phase (see nonfinite4)
};

// Status bits of a propagator.  The stress phase sets STATUS_NONFINITE when
// it writes a NaN or an infinity (an unstable or overflowing run); hosts read
// the word between steps and fail that run alone.
constexpr uint32_t STATUS_NONFINITE = 1u;

__device__ __forceinline__ bool nonfinite4(const float4& v) {
  // NaN fails every comparison; |±inf| exceeds the largest finite float
  return !(fabsf(v.x) <= 3.402823466e38f && fabsf(v.y) <= 3.402823466e38f && fabsf(v.z) <= 3.402823466e38f &&
           fabsf(v.w) <= 3.402823466e38f);
}

// What the stress phase does with the finished fields of each physical cell
// (fused so the image fields are never re-read from HBM).
enum EpilogueKind : int32_t {
  EPI_NONE = 0,
  EPI_STORE = 1,       // write the P (and S) image fields to out[] (replay)
  EPI_IMAGE = 2,       // imaging condition against stored source fields (backward)
  EPI_EXC_TRACK = 3,   // excitation map: running argmax |P| (replay)
  EPI_EXC_IMAGE = 4,   // excitation imaging at this step (backward)
};

constexpr int MAX_EPI_IMAGES = 2;

struct Epilogue {
  int32_t kind;
  int32_t sep;                       // 0 stress, 1 divcurl (elastic)
  int32_t need_s;                    // S is needed (elastic)
  int32_t n_images;
  int32_t src_slot[MAX_EPI_IMAGES];  // stored source field per image (0 P, 1 S)
  int32_t rcv_wave[MAX_EPI_IMAGES];  // receiver wave per image (0 P, 1 S)
  int32_t cross, illum, rillum;      // which sums to accumulate at this step
  int32_t kahan;                     // accumulators are Kahan float pairs
  int32_t step;                      // time label (excitation)
  int32_t pad_;
  float* out[2];                     // EPI_STORE destinations (P, S), (nz, nx)
  const float* src[2];               // EPI_IMAGE stored source fields (P, S)
  double* num[MAX_EPI_IMAGES];       // FP64 accumulators, (nz, nx); Kahan: float pairs
  double* ill[MAX_EPI_IMAGES];       // source illumination S² (nullptr: shared with image 0 / unused)
  double* ril[MAX_EPI_IMAGES];       // receiver illumination R² (nullptr: unused)
  float* running;                    // excitation |P| running max
  int32_t* peak_step;                // excitation argmax step
};

// One propagator advance inside a (possibly batched) launch.
struct StepWork {
  int32_t prop;         // index into the DevProp table
  int32_t tile0;        // first block of this work in the launch
  int32_t tiles_x;      // tiles along x for this propagator
  int32_t tiles;        // total tiles for this propagator
  const float* wavelet; // source time series (device); nullptr → use amp/amp_eps
  int32_t t;            // index into wavelet
  float amp;            // source amplitude (when wavelet == nullptr)
  float amp_eps;        // viscoacoustic strain amplitude (when wavelet == nullptr)
  int32_t flags;        // STEP_* bits
  // Straight-line interior tiles: rows [ti0, ti1) × columns [tj0, tj1) of
  // tiles, less the source node's tile (hole_i, hole_j; −1 when none).  A
  // launch of interior tiles walks the rectangle; a launch of boundary tiles
  // walks the frame around it and then the hole.
  int32_t ti0, ti1, tj0, tj1, hole_i, hole_j;
  int32_t slot;         // index of this work's tensor maps in a TMA launch
  Epilogue epi;
};
constexpr int STEP_PEAK = 1;        // visco: reduce max|p| into DevProp::peak

// The works of one launch, passed by value in the kernel parameters: one work
// (plain stepping) or up to N (batched ticks; blocks find their work by binary
// search over the tile offsets).
struct WorkSet1 {
  StepWork w;
  __device__ __forceinline__ const StepWork& get(int) const { return w; }
};

template <int N>
struct WorkSetN {
  int32_t n;
  int32_t pad_;
  StepWork w[N];
  __device__ __forceinline__ const StepWork& get(int block) const {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (w[mid].tile0 <= block) lo = mid; else hi = mid - 1;
    }
    return w[lo];
  }
};
constexpr int MAX_BATCH_WORKS = 32;
using WorkSetB = WorkSetN<MAX_BATCH_WORKS>;

// ---------------------------------------------------------------------------
// exact-order float helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Forward staggered difference D⁺ at s[0] along a unit-stride (stride=1) or
// row (stride=ld) axis: Σ_k c_k (f[+k] − f[−k+1]), accumulated k = 1..M,
// then divided by h (numerics.py:96-116).
template <int M>
__device__ __forceinline__ float dplus(const float* s, int stride, const float* c, float h) {
  float acc = fmul(c[0], fsub(s[stride], s[0]));
#pragma unroll
  for (int k = 2; k <= M; ++k)
    acc = fadd(acc, fmul(c[k - 1], fsub(s[k * stride], s[(1 - k) * stride])));
  return fdiv(acc, h);
}

// Backward staggered difference D⁻: Σ_k c_k (f[k−1] − f[−k]).
template <int M>
__device__ __forceinline__ float dminus(const float* s, int stride, const float* c, float h) {
  float acc = fmul(c[0], fsub(s[0], s[-stride]));
#pragma unroll
  for (int k = 2; k <= M; ++k)
    acc = fadd(acc, fmul(c[k - 1], fsub(s[(k - 1) * stride], s[-k * stride])));
  return fdiv(acc, h);
}

// a / h rounded to nearest, in one of four forms; the host picks the first
// of forms 1, 3, 2 whose value equals __fdiv_rn(a, h) for all 2^32 float
// inputs a (+0 and −0 count as equal, NaN as equal to NaN; k_verify_division)
// and otherwise keeps form 0.
//   3: RN(a·z_h + RN(a·z_l)) with one FMA, z_h = RN32(1/h), z_l = RN32(1/h − z_h)
//      — division by a constant known in advance, Brisebarre, Muller & Raina,
//      "Accelerating correctly rounded floating-point division when the
//      divisor is known in advance", IEEE Trans. Computers 53(8), 2004;
//   2: q = RN(a·r), e = a − q·h (exact FMA residual), RN(q + e·r), r = RN32(1/h)
//      — the one-step correction of Markstein, IBM J. Res. Dev. 34(1), 1990;
//   1: float32(RN64(double(a)·R)) with R = RN64(1/h);
//   0: __fdiv_rn(a, h).
__device__ __forceinline__ float div_bmr(float a, float zh, float zl) { return __fmaf_rn(a, zh, __fmul_rn(a, zl)); }
__device__ __forceinline__ float div_fma(float a, float h, float r) {
  const float q = __fmul_rn(a, r);
  return __fmaf_rn(__fmaf_rn(-q, h, a), r, q);
}
__device__ __forceinline__ float divh(float a, float h, double r64, float r32, float rl, int mode) {
  if (mode == 3) return div_bmr(a, r32, rl);
  if (mode == 2) return div_fma(a, h, r32);
  if (mode == 1) return __double2float_rn(__dmul_rn((double)a, r64));
  return __fdiv_rn(a, h);
}

// CPML memory update and corrected derivative: ψ ← ψ·b + a·D; return D + ψ
// (numerics.py:221-227 with κ ≡ 1).
__device__ __forceinline__ float cpml(float d, float& psi, float a, float b) {
  psi = fadd(fmul(psi, b), fmul(a, d));
  return fadd(d, psi);
}

// Column index into the x-strip ψ array, or −1 outside the strips.
__device__ __forceinline__ int strip_x(const DevProp& P, int j) {
  if (j < P.npx_l) return j;
  if (j >= P.nxp - P.npx_r) return P.npx_l + (j - (P.nxp - P.npx_r));
  return -1;
}
// Row index into the z-strip ψ array, or −1 outside the strips.
__device__ __forceinline__ int strip_z(const DevProp& P, int i) {
  if (i < P.npz_t) return i;
  if (i >= P.nzp - P.npz_b) return P.npz_t + (i - (P.nzp - P.npz_b));
  return -1;
}


}  // namespace ertm
