// Auxiliary kernels around the stencil: material setup, receiver sampling,
// time-reversed injection, image fields, imaging conditions, viscoacoustic
// stabilisation and image post-processing.  All are HBM-bound elementwise or
// gather/scatter work.
#pragma once

#include "ertm_device.cuh"
#include "step_kernels.cuh"

namespace ertm {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// material setup on the padded grid (propagation.py:165-187, 411-421,
// 588-675, 858-871): edge padding, κ = ρ·v²·, 1/ρ averaged to faces,
// μ averaged to corners.  Inputs are the physical (nz, nx) float32 arrays.
// ---------------------------------------------------------------------------
struct SetupArgs {
  const float* vp; const float* vs; const float* rho;   // physical (nz, nx)
  // visco relaxation tables, per unique Q value
  const double* tau;     // [nq][L]
  const double* delta;   // [nq][L] (already −αΔ under compensation)
  const double* mref;    // [nq]
  const float* relax_a;  // [nq][L] float32 exp(−dt/τ)
  double dt;
};

__device__ __forceinline__ float padded_at(const float* a, int nz, int nx, int pad, int i, int j) {
  return a[(size_t)clampi(i - pad, 0, nz - 1) * nx + clampi(j - pad, 0, nx - 1)];
}

__global__ void k_setup_materials(DevProp* props, int pi, SetupArgs A) {
  const DevProp& P = props[pi];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= P.nzp || j >= P.nxp) return;
  const int nz = P.nz, nx = P.nx, pad = P.pad;
  const size_t g = (size_t)i * P.ld + j;
  auto inv_rho = [&](int ii, int jj) { return fdiv(1.0f, padded_at(A.rho, nz, nx, pad, ii, jj)); };
  const float ir = inv_rho(i, j);
  const float irx = (j < P.nxp - 1) ? fmul(0.5f, fadd(ir, inv_rho(i, j + 1))) : ir;
  const float irz = (i < P.nzp - 1) ? fmul(0.5f, fadd(ir, inv_rho(i + 1, j))) : ir;
  const float rho = padded_at(A.rho, nz, nx, pad, i, j);
  const float vp = padded_at(A.vp, nz, nx, pad, i, j);
  float* const* C = const_cast<float* const*>(reinterpret_cast<const float* const*>(P.coef));
  if (P.engine == ENGINE_ACOUSTIC) {
    C[CA_KAPPA][g] = fmul(fmul(rho, vp), vp);
    C[CA_IRX][g] = irx;
    C[CA_IRZ][g] = irz;
  } else if (P.engine == ENGINE_ELASTIC) {
    auto mu_at = [&](int ii, int jj) {
      const float r = padded_at(A.rho, nz, nx, pad, ii, jj), s = padded_at(A.vs, nz, nx, pad, ii, jj);
      return fmul(fmul(r, s), s);
    };
    auto mux_at = [&](int ii, int jj) {  // _mean_x(mu)
      return (jj < P.nxp - 1) ? fmul(0.5f, fadd(mu_at(ii, jj), mu_at(ii, jj + 1))) : mu_at(ii, jj);
    };
    const float vs = padded_at(A.vs, nz, nx, pad, i, j);
    const float mu = fmul(fmul(rho, vs), vs);
    const float lam = fmul(rho, fsub(fmul(vp, vp), fmul(fmul(2.0f, vs), vs)));
    C[CE_LAM][g] = lam;
    C[CE_L2M][g] = fadd(lam, fmul(2.0f, mu));
    C[CE_MUXZ][g] = (i < P.nzp - 1) ? fmul(0.5f, fadd(mux_at(i, j), mux_at(i + 1, j))) : mux_at(i, j);
    C[CE_IRX][g] = irx;
    C[CE_IRZ][g] = irz;
  } else {
    const float kappa = fmul(fmul(rho, vp), vp);
    const int q = P.qidx[g];
    const float kr = __double2float_rn(__ddiv_rn((double)kappa, A.mref[q]));
    C[CV_KR][g] = kr;
    C[CV_IRX][g] = irx;
    C[CV_IRZ][g] = irz;
    for (int l = 0; l < P.L; ++l) {
      const float one_minus_a = fsub(1.0f, A.relax_a[q * P.L + l]);
      double b = dmul(dmul(dmul((double)kr, A.delta[q * P.L + l]), (double)one_minus_a), A.tau[q * P.L + l]);
      C[CV_B0 + l][g] = __double2float_rn(__ddiv_rn(b, A.dt));
    }
  }
}

// Exhaustive check of divh() against __fdiv_rn for a fixed divisor h: all
// 2^32 float inputs; value mismatches are counted (+0 == −0, NaN == NaN).
__global__ void k_verify_division(float h, double r64, float r32, float rl, int mode,
                                  unsigned long long* mismatches) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  unsigned long long bad = 0;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < (1ull << 32); k += stride) {
    const float a = __uint_as_float((uint32_t)k);
    const float q = divh(a, h, r64, r32, rl, mode);
    const float ref = __fdiv_rn(a, h);
    const bool same = (q == ref) || (q != q && ref != ref);
    bad += same ? 0ull : 1ull;
  }
  if (bad) atomicAdd(mismatches, bad);
}

// ---------------------------------------------------------------------------
// receiver sampling (numerics.py:478-511, propagation.py:371-391)
// ---------------------------------------------------------------------------
enum SampleKind : int32_t { SAMPLE_FIELD = 0, SAMPLE_PRESSURE = 1, SAMPLE_ZERO = 2 };

struct SamplePlanDev {
  int32_t n;            // receivers
  int32_t kind;         // SampleKind
  int32_t field;        // field slot (SAMPLE_FIELD)
  int32_t pad_;
  const int32_t* cell;  // zc·ld + xc (clipped floor node)
  const uint8_t* valid;
  const double* w;      // [n][4]: 1−tz, tz, 1−tx, tx
  float* out;           // row base for this step (n floats)
};

constexpr int MAX_SAMPLE = 8;
struct SampleSet {
  int32_t count;
  SamplePlanDev plan[MAX_SAMPLE];
};

__device__ __forceinline__ double corner(const DevProp& P, int kind, int field, int32_t idx) {
  if (kind == SAMPLE_PRESSURE) return (double)fmul(0.5f, fadd(P.f[E_SXX][idx], P.f[E_SZZ][idx]));
  return (double)P.f[field][idx];
}

// One thread per (component, receiver); writes the float32 sample of this step.
__global__ void k_sample(const DevProp* props, int pi, SampleSet S, int64_t row_offset) {
  const DevProp& P = props[pi];
  const int comp = blockIdx.y;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (comp >= S.count) return;
  const SamplePlanDev& sp = S.plan[comp];
  if (r >= sp.n) return;
  float v = 0.f;
  if (sp.kind != SAMPLE_ZERO && sp.valid[r]) {
    const int32_t c0 = sp.cell[r];
    const double* w = sp.w + 4 * r;
    const double v00 = corner(P, sp.kind, sp.field, c0), v01 = corner(P, sp.kind, sp.field, c0 + 1);
    const double v10 = corner(P, sp.kind, sp.field, c0 + P.ld), v11 = corner(P, sp.kind, sp.field, c0 + P.ld + 1);
    double acc = dmul(dmul(v00, w[0]), w[2]);
    acc = dadd(acc, dmul(dmul(v01, w[0]), w[3]));
    acc = dadd(acc, dmul(dmul(v10, w[1]), w[2]));
    acc = dadd(acc, dmul(dmul(v11, w[1]), w[3]));
    v = __double2float_rn(acc);
  }
  sp.out[row_offset + r] = v;
}

// ---------------------------------------------------------------------------
// time-reversed injection with np.add.at semantics (propagation.py:331-369,
// 472-494, 916-942): every contribution is added in float64 and rounded to
// float32, in the reference order (component, corner, receiver).  The host
// groups contributions by target cell, so one thread owns one cell and the
// launch is deterministic without atomics.
// ---------------------------------------------------------------------------
struct InjectPlanDev {
  int32_t n_cells;
  int32_t pad_;
  const int32_t* cell_field;  // field slot per target cell
  const int32_t* cell_index;  // i·ld + j per target cell
  const int32_t* start;       // [n_cells + 1] into the contribution arrays
  const int32_t* src;         // record offset (component·nt·nrec + receiver) per contribution
  const double* wa;           // contribution = (value·wa)·wb
  const double* wb;
};

__global__ void k_inject(const DevProp* props, int pi, InjectPlanDev plan, const float* record,
                         int64_t time_offset) {
  const DevProp& P = props[pi];
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= plan.n_cells) return;
  float* f = P.f[plan.cell_field[u]] + plan.cell_index[u];
  float acc = *f;
  for (int k = plan.start[u]; k < plan.start[u + 1]; ++k) {
    const double v = (double)record[plan.src[k] + time_offset];
    acc = __double2float_rn(dadd((double)acc, dmul(dmul(v, plan.wa[k]), plan.wb[k])));
  }
  *f = acc;
}

// Injection for many propagators in one launch (batched ticks): item k owns
// global cells [cell0, cell0 + n_cells).
struct InjectItem {
  InjectPlanDev plan;
  const DevProp* prop;
  const float* record;
  int64_t time_offset;
  int32_t cell0;
  int32_t pad_;
};
struct InjectBatch {
  int32_t n;
  int32_t pad_;
  InjectItem it[MAX_BATCH_WORKS];
};

__global__ void k_inject_batch(InjectBatch B) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  int lo = 0, hi = B.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (B.it[mid].cell0 <= u) lo = mid; else hi = mid - 1;
  }
  const InjectItem& I = B.it[lo];
  const int v = u - I.cell0;
  if (v < 0 || v >= I.plan.n_cells) return;
  float* f = I.prop->f[I.plan.cell_field[v]] + I.plan.cell_index[v];
  float acc = *f;
  for (int k = I.plan.start[v]; k < I.plan.start[v + 1]; ++k) {
    const double val = (double)I.record[I.plan.src[k] + I.time_offset];
    acc = __double2float_rn(dadd((double)acc, dmul(dmul(val, I.plan.wa[k]), I.plan.wb[k])));
  }
  *f = acc;
}

// Single-cell add (elastic force_z source lands on vz after the stress phase,
// propagation.py:872-873).
__global__ void k_point_add(float* f, int64_t idx, float amp) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && amp != 0.f) f[idx] = fadd(f[idx], amp);
}
__global__ void k_point_add_wave(float* f, int64_t idx, const float* wave, int t) {
  const float amp = wave[t];
  if (threadIdx.x == 0 && blockIdx.x == 0 && amp != 0.f) f[idx] = fadd(f[idx], amp);
}

// ---------------------------------------------------------------------------
// image fields (propagation.py:500-501, 795-796, 945-977)
// ---------------------------------------------------------------------------
enum Wave : int32_t { WAVE_P = 0, WAVE_S = 1 };
enum Separation : int32_t { SEP_STRESS = 0, SEP_DIVCURL = 1 };

template <int M>
__device__ __forceinline__ float image_value(const DevProp& P, int wave, int sep, int i, int j) {
  const size_t g = (size_t)i * P.ld + j;
  if (P.engine != ENGINE_ELASTIC) return P.f[A_P][g];
  if (sep == SEP_STRESS) {
    if (wave == WAVE_P) return fmul(0.5f, fadd(P.f[E_SXX][g], P.f[E_SZZ][g]));
    return P.f[E_SXZ][g];
  }
  const float c[4] = {P.c[0], P.c[1], P.c[2], P.c[3]};
  const float* vx = P.f[E_VX] + g;
  const float* vz = P.f[E_VZ] + g;
  // Physical cells are ≥ M+1 from every padded edge, so each D⁻ is in range.
  if (wave == WAVE_P) return fadd(dminus<M>(vx, 1, c, P.hx), dminus<M>(vz, P.ld, c, P.hz));
  return fsub(dminus<M>(vx, P.ld, c, P.hz), dminus<M>(vz, 1, c, P.hx));
}

template <int M>
__global__ void k_image_field(const DevProp* props, int pi, int wave, int sep, float* out) {
  const DevProp& P = props[pi];
  const int jj = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= P.nz || jj >= P.nx) return;
  out[(size_t)ii * P.nx + jj] = image_value<M>(P, wave, sep, ii + P.pad, jj + P.pad);
}

// ---------------------------------------------------------------------------
// stand-alone epilogue: the imaging step when it cannot be fused into the
// stress phase (after the compensated viscoacoustic stabilisation, or when a
// force_z source lands on vz after the stress phase and divcurl is imaged)
// ---------------------------------------------------------------------------
template <int M>
__global__ void k_epilogue(const DevProp* props, int pi, Epilogue E) {
  const DevProp& P = props[pi];
  const int jj = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = blockIdx.y * blockDim.y + threadIdx.y;
  if (ii >= P.nz || jj >= P.nx) return;
  const size_t c = (size_t)ii * P.nx + jj;
  const float pv = image_value<M>(P, WAVE_P, E.sep, ii + P.pad, jj + P.pad);
  const float sv = (P.engine == ENGINE_ELASTIC && E.need_s) ? image_value<M>(P, WAVE_S, E.sep, ii + P.pad, jj + P.pad)
                                                             : 0.f;
  run_epilogue(E, c, (size_t)P.nz * P.nx, pv, sv);
}

// Status words of every propagator of a launch table (one small copy back).
__global__ void k_gather_status(const DevProp* table, int n, uint32_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = *table[i].status;
}

__global__ void k_kahan_to_f64(const float* s, const float* c, double* out, int64_t n) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = (double)s[k] - (double)c[k];
}

// ---------------------------------------------------------------------------
// viscoacoustic compensation safety net (propagation.py:726-749)
// ---------------------------------------------------------------------------
struct StabState {
  double ref_amp;   // reference amplitude: running max|p| over steps < 30
  int32_t clipped;  // amplitude-cap events
  int32_t pad_;
};

__global__ void k_stab_reference(const DevProp* props, int pi, StabState* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double peak = (double)*props[pi].peak;
    st->ref_amp = st->ref_amp > peak ? st->ref_amp : peak;
  }
}

// Scale p, ε, vx, vz, r_l by float32(limit/peak) when max|p| exceeds the cap.
__global__ void k_stab_scale(const DevProp* props, int pi, StabState* st, double cap) {
  const DevProp& P = props[pi];
  const double peak = (double)*P.peak;
  const double ref = st->ref_amp > 1e-30 ? st->ref_amp : 1e-30;
  const double limit = cap * ref;
  if (!(peak > limit)) return;
  const float s = __double2float_rn(__ddiv_rn(limit, peak));
  if (blockIdx.x == 0 && threadIdx.x == 0) st->clipped += 1;
  const size_t n = (size_t)P.nzp * P.ld;
  const int nf = 4 + P.L;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    for (int f = 0; f < nf; ++f) P.f[f][k] = fmul(P.f[f][k], s);
  }
}

// Column origin of the padded grid in k_epilogue_batch / k_stab_epilogue:
// thread column t handles padded column t − epi_col_shift(pad), so that the
// physical columns (and the accumulators' rows) start at a multiple of 32.
__device__ __forceinline__ int epi_col_shift(int pad) { return ((pad + 31) / 32) * 32 - pad; }

// k_stab_scale followed by k_epilogue in one pass, for a compensated
// viscoacoustic step with no low-pass between them: each thread owns one
// padded cell, scales every field there when the cap clips (the cells and
// the arithmetic of k_stab_scale), and a physical cell's epilogue images
// the p value of its own cell (image_value of a pressure engine), which the
// same thread has just scaled.
template <int M>
__global__ void k_stab_epilogue(const DevProp* props, int pi, StabState* st, double cap, Epilogue E) {
  const DevProp& P = props[pi];
  const int jj = (int)(blockIdx.x * blockDim.x + threadIdx.x) - epi_col_shift(P.pad);   // padded column
  const int ii = blockIdx.y * blockDim.y + threadIdx.y;                                   // padded row
  if (ii >= P.nzp || jj < 0 || jj >= P.ld) return;
  const size_t k = (size_t)ii * P.ld + jj;
  const double peak = (double)*P.peak;
  const double ref = st->ref_amp > 1e-30 ? st->ref_amp : 1e-30;
  const double limit = cap * ref;
  if (peak > limit) {
    const float s = __double2float_rn(__ddiv_rn(limit, peak));
    if (ii == 0 && jj == 0) st->clipped += 1;
    const int nf = 4 + P.L;
    for (int f = 0; f < nf; ++f) P.f[f][k] = fmul(P.f[f][k], s);
  }
  const int pz = ii - P.pad, px = jj - P.pad;
  if (pz < 0 || pz >= P.nz || px < 0 || px >= P.nx) return;
  run_epilogue(E, (size_t)pz * P.nx + px, (size_t)P.nz * P.nx, image_value<M>(P, WAVE_P, E.sep, ii, jj), 0.f);
}

// The stand-alone epilogues of a batched tick in one launch: blockIdx.z is
// the item, x and y cover its padded grid (blocks outside it exit).  An item
// with `stab` set first applies its step's stabilisation scale, as
// k_stab_epilogue does; every item images its physical cells as k_epilogue
// does (P and, for elastic S, from image_value).
struct EpiItem {
  int32_t prop;      // index into the launch's DevProp table
  int32_t stab;      // 1: the step's stabilisation scale runs here first
  double cap;        // amplitude cap (stab)
  StabState* st;     // stabilisation state (stab)
  Epilogue E;
};
struct EpiBatch {
  int32_t n;
  int32_t pad_;
  EpiItem it[MAX_BATCH_WORKS];
};

template <int M>
__global__ void k_epilogue_batch(const DevProp* table, const __grid_constant__ EpiBatch B) {
  const EpiItem& I = B.it[blockIdx.z];
  const DevProp& P = table[I.prop];
  const int jj = (int)(blockIdx.x * blockDim.x + threadIdx.x) - epi_col_shift(P.pad);   // padded column
  const int ii = blockIdx.y * blockDim.y + threadIdx.y;                                   // padded row
  if (ii >= P.nzp || jj < 0 || jj >= P.ld) return;
  if (I.stab) {
    const double peak = (double)*P.peak;
    const double ref = I.st->ref_amp > 1e-30 ? I.st->ref_amp : 1e-30;
    const double limit = I.cap * ref;
    if (peak > limit) {
      const float s = __double2float_rn(__ddiv_rn(limit, peak));
      if (ii == 0 && jj == 0) I.st->clipped += 1;
      const size_t k = (size_t)ii * P.ld + jj;
      const int nf = 4 + P.L;
      for (int f = 0; f < nf; ++f) P.f[f][k] = fmul(P.f[f][k], s);
    }
  }
  const int pz = ii - P.pad, px = jj - P.pad;
  if (pz < 0 || pz >= P.nz || px < 0 || px >= P.nx) return;
  const float pv = image_value<M>(P, WAVE_P, I.E.sep, ii, jj);
  const float sv = (P.engine == ENGINE_ELASTIC && I.E.need_s) ? image_value<M>(P, WAVE_S, I.E.sep, ii, jj) : 0.f;
  run_epilogue(I.E, (size_t)pz * P.nx + px, (size_t)P.nz * P.nx, pv, sv);
}

// ---------------------------------------------------------------------------
// image post-processing (imaging.py:326-331, 476-502; numerics.py:398-404)
// ---------------------------------------------------------------------------
struct NormArgs {
  const double* num; const double* illum; const double* rillum;
  const float* num_s; const float* illum_s; const float* rillum_s;   // Kahan sums (comp ignored)
  int32_t kahan;
  int32_t by_illum, by_rillum;
  double eps;
  double* out;
  int64_t n;
};

__global__ void k_normalize(NormArgs A) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= A.n) return;
  double v = A.kahan ? (double)A.num_s[k] : A.num[k];
  if (A.by_illum) v = __ddiv_rn(v, dadd(A.kahan ? (double)A.illum_s[k] : A.illum[k], A.eps));
  if (A.by_rillum) v = __ddiv_rn(v, dadd(A.kahan ? (double)A.rillum_s[k] : A.rillum[k], A.eps));
  A.out[k] = v;
}

__global__ void k_laplacian(const double* a, double* out, int nz, int nx, double dx, double dz) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nz || j >= nx) return;
  auto at = [&](int ii, int jj) { return a[(size_t)clampi(ii, 0, nz - 1) * nx + clampi(jj, 0, nx - 1)]; };
  const double c = at(i, j);
  const double d2x = __ddiv_rn(dadd(dsub(at(i, j + 1), dmul(2.0, c)), at(i, j - 1)), dmul(dx, dx));
  const double d2z = __ddiv_rn(dadd(dsub(at(i + 1, j), dmul(2.0, c)), at(i - 1, j)), dmul(dz, dz));
  out[(size_t)i * nx + j] = dadd(d2x, d2z);
}

__global__ void k_mask_cast(const double* a, float* out, int nz, int nx, int npml, int top) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nz || j >= nx) return;
  const bool zero = j < npml || j >= nx - npml || i >= nz - npml || (top && i < npml);
  const double v = a[(size_t)i * nx + j] * (zero ? 0.0 : 1.0);
  out[(size_t)i * nx + j] = __double2float_rn(v);
}

// stack_images (pipeline.py:133-161): per-image max|·| then normalised mean.
// The maximum propagates NaN as np.max does (pipeline.py:147): |NaN| has its
// sign bit clear and its bits order above +inf as unsigned words, so the
// atomicMax of the bit patterns keeps it, and k_stack_add then leaves the
// image undivided (`scale > 0` is false for NaN).
__device__ __forceinline__ float max_nan(float m, float v) { return (v > m || v != v) ? v : m; }

__global__ void k_absmax_f32(const float* a, int64_t n, unsigned int* out_bits) {
  float m = 0.f;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    m = max_nan(m, fabsf(a[k]));
  for (int o = 16; o > 0; o >>= 1) m = max_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));
}

__global__ void k_stack_add(const float* img, int64_t n, const unsigned int* scale_bits, int normalize,
                            double* acc) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double d = (double)img[k];
  if (normalize) {
    const double s = (double)__uint_as_float(*scale_bits);
    if (s > 0.0) d = __ddiv_rn(d, s);
  }
  acc[k] = dadd(acc[k], d);
}

// Every image's max|·| in one launch: blockIdx.y is the image.
__global__ void k_absmax_images(const float* const* imgs, int64_t n, unsigned int* out_bits) {
  const float* a = imgs[blockIdx.y];
  float m = 0.f;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    m = max_nan(m, fabsf(a[k]));
  for (int o = 16; o > 0; o >>= 1) m = max_nan(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits + blockIdx.y, __float_as_uint(m));
}

// The stack of all images at each pixel in one launch: the float64 sum runs
// over the images in order, each term the k_stack_add term (divided by its
// image's max|·| when normalising and that is > 0), starting from sum[k]
// (or 0 without `sum`); the total goes back to `sum` and, with `out`, the
// k_stack_finish mean to `out`.
__global__ void k_stack_images(const float* const* imgs, int n_images, int64_t n, const unsigned int* scale_bits,
                               int normalize, double* sum, int count, float* out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double acc = sum ? sum[k] : 0.0;
#pragma unroll 4
  for (int i = 0; i < n_images; ++i) {
    double d = (double)imgs[i][k];
    if (normalize) {
      const double s = (double)__uint_as_float(scale_bits[i]);
      if (s > 0.0) d = __ddiv_rn(d, s);
    }
    acc = dadd(acc, d);
  }
  if (sum) sum[k] = acc;
  if (out) out[k] = __double2float_rn(__ddiv_rn(acc, (double)count));
}

__global__ void k_stack_finish(const double* acc, int64_t n, int count, float* out) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = __double2float_rn(__ddiv_rn(acc[k], (double)count));
}

}  // namespace ertm

namespace ertm {

// ---------------------------------------------------------------------------
// Record preprocessing (preprocess.py:36-224, numerics.py:337-392).  Records
// are (nt, ntr) float32, time-major; arithmetic in float64 as the reference
// does, one float32 rounding at the end.
// ---------------------------------------------------------------------------
// Sinc resampling: out[o, s] = Σ_t w[o, t] · in[clamp(off0[o] + t), s] with the
// weights and first offsets computed on the host (numerics.py:371-384).
// Records kernels below: grid x over traces (128 per block), grid y over time
// samples (grid-stride), so no thread divides an index.
__global__ void k_resample(const float* __restrict__ in, int64_t n_in, int64_t ntr, const double* __restrict__ w,
                           const int64_t* __restrict__ off0, int taps, int64_t n_out, float* __restrict__ out) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ntr) return;
  const float* __restrict__ col = in + s;
  for (int64_t o = blockIdx.y; o < n_out; o += gridDim.y) {
    const int64_t k0 = off0[o];
    const double* __restrict__ wo = w + o * taps;
    double acc = 0.0;
#pragma unroll 4
    for (int t = 0; t < taps; ++t) {
      int64_t k = k0 + t;
      k = k < 0 ? 0 : (k >= n_in ? n_in - 1 : k);
      acc = dadd(acc, dmul(wo[t], (double)col[k * ntr]));
    }
    out[o * ntr + s] = __double2float_rn(acc);
  }
}

// Direct-wave mute (preprocess.py:121-173): weight 0.5 − 0.5·cos(π·ramp) with
// ramp = clip((t − start_r)/(end_r − start_r), 0, 1) per receiver r.
__global__ void k_mute(const float* __restrict__ in, int64_t nt, int64_t ntr, const double* __restrict__ t,
                       const double* __restrict__ start, const double* __restrict__ end, float* __restrict__ out) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ntr) return;
  const double s0 = start[r], span = dsub(end[r], start[r]);
  for (int64_t i = blockIdx.y; i < nt; i += gridDim.y) {
    double ramp = __ddiv_rn(dsub(t[i], s0), span);
    ramp = ramp < 0.0 ? 0.0 : (ramp > 1.0 ? 1.0 : ramp);
    const double wgt = dsub(0.5, dmul(0.5, cos(dmul(3.141592653589793, ramp))));
    out[i * ntr + r] = __double2float_rn(dmul((double)in[i * ntr + r], wgt));
  }
}

// End taper (preprocess.py:176-191): the first w samples times ramp[k], the
// last w times ramp[w−1−k], in that order (both when they overlap).
__global__ void k_taper(const float* __restrict__ in, int64_t nt, int64_t ntr, const double* __restrict__ ramp,
                        int64_t w, float* __restrict__ out) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ntr) return;
  for (int64_t i = blockIdx.y; i < nt; i += gridDim.y) {
    double x = (double)in[i * ntr + r];
    if (i < w) x = dmul(x, ramp[i]);
    if (i >= nt - w) x = dmul(x, ramp[nt - 1 - i]);
    out[i * ntr + r] = __double2float_rn(x);
  }
}

// Two-component rotation (preprocess.py:36-67): vx' = c·vx + s·vz,
// vz' = (−s)·vx + c·vz in float64.
__global__ void k_rotate(const float* __restrict__ vx, const float* __restrict__ vz, int64_t n, double c, double s,
                         float* __restrict__ ox, float* __restrict__ oz) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const double x = (double)vx[idx], z = (double)vz[idx];
  ox[idx] = __double2float_rn(dadd(dmul(c, x), dmul(s, z)));
  oz[idx] = __double2float_rn(dadd(dmul(-s, x), dmul(c, z)));
}

}  // namespace ertm

namespace ertm {

// ---------------------------------------------------------------------------
// Short-time Fourier filtering with overlap-add (qcomp.py:98-147): frames of
// L samples every hop samples, Hann-windowed, one complex response per frame
// and frequency, windowed overlap-add normalised by Σ window².  Records are
// (n, ntr) float64, time-major; frame s covers [s·hop, s·hop + L) ∩ [0, n).
// ---------------------------------------------------------------------------
__global__ void k_stft_frames(const double* __restrict__ x, int64_t n, int64_t ntr, int L, int hop, int S,
                              const double* __restrict__ win, double* __restrict__ frames) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)S * ntr * L) return;
  const int k = (int)(idx % L);
  const int64_t sr = idx / L;
  const int64_t s = sr / ntr, r = sr - s * ntr;
  const int64_t t = s * hop + k;
  frames[idx] = t < n ? dmul(x[t * ntr + r], win[k]) : 0.0;
}

// Frame spectra times the frame's response (complex, (a+ib)(c+id)).
__global__ void k_stft_response(double2* __restrict__ spec, int64_t ntr, int F, int S,
                                const double2* __restrict__ resp) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)S * ntr * F) return;
  const int f = (int)(idx % F);
  const int64_t s = idx / F / ntr;
  const double2 a = spec[idx], b = resp[s * F + f];
  spec[idx] = make_double2(dsub(dmul(a.x, b.x), dmul(a.y, b.y)), dadd(dmul(a.x, b.y), dmul(a.y, b.x)));
}

// Overlap-add in frame order: out(t) = Σ_s (filt_s(t − s·hop)/L)·win(t − s·hop),
// divided by Σ_s win(t − s·hop)² (1 where that sum is ≤ 1e-12).
__global__ void k_stft_overlap_add(const double* __restrict__ filt, int64_t n, int64_t ntr, int L, int hop, int S,
                                   const double* __restrict__ win, double* __restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * ntr) return;
  const int64_t t = idx / ntr, r = idx - t * ntr;
  const int64_t s0 = t >= L ? (t - L) / hop + 1 : 0;
  double acc = 0.0, wsum = 0.0;
  for (int64_t s = s0; s < S && s * hop <= t; ++s) {
    const int64_t k = t - s * hop;
    if (k >= L) continue;
    const double y = __ddiv_rn(filt[(s * ntr + r) * L + k], (double)L);
    acc = dadd(acc, dmul(y, win[k]));
    wsum = dadd(wsum, dmul(win[k], win[k]));
  }
  out[idx] = __ddiv_rn(acc, wsum > 1e-12 ? wsum : 1.0);
}

}  // namespace ertm

namespace ertm {

// ---------------------------------------------------------------------------
// SEG-Y rev 1 trace samples ↔ float32 records (segy.py:103-155 reads with
// segyio, segy.py:373-530 writes).  A trace block is 240 header bytes then ns
// big-endian 4-byte samples, data sample format 5 (IEEE single) or 1 (IBM
// System/360 hexadecimal single: sign, excess-64 base-16 exponent, 24-bit
// fraction 0.F).  Records are (ns, width) float32, sample-major, so the
// codec is a 32×32 shared-memory transpose: file reads run along samples,
// record writes along traces.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t bswap32(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

// IBM → float32: |x| = F·2^(4(e−64)−24) is exact in double (leading bit at
// most 2^227, least 2^−280); one round-to-nearest-even to float32 follows.
__device__ __forceinline__ float ibm_to_float(uint32_t w) {
  const uint32_t frac = w & 0x00ffffffu;
  if (frac == 0) return __uint_as_float(w & 0x80000000u);
  const int e16 = (int)((w >> 24) & 0x7fu);
  const int p = 31 - __clz(frac);                         // leading bit of F, 0..23
  const int e2 = p + 4 * (e16 - 64) - 24;                  // binary exponent of that bit
  uint64_t bits = ((uint64_t)(e2 + 1023) << 52) | (((uint64_t)frac << (52 - p)) & 0x000fffffffffffffull);
  bits |= (uint64_t)(w & 0x80000000u) << 32;
  return __double2float_rn(__longlong_as_double((long long)bits));
}

// float32 → IBM, fraction rounded to nearest (ties to even); ±inf and NaN map
// to the largest IBM magnitude; every finite float32 (denormals included) lies
// inside the IBM exponent range.
__device__ __forceinline__ uint32_t float_to_ibm(float x) {
  const uint32_t u = __float_as_uint(x);
  const uint32_t sign = u & 0x80000000u;
  const uint32_t be = (u >> 23) & 0xffu;
  uint32_t m = u & 0x7fffffu;
  if (be == 0xffu) return sign | 0x7fffffffu;
  int e2;
  if (be == 0) {
    if (m == 0) return sign;
    e2 = -149;
  } else {
    m |= 0x800000u;
    e2 = (int)be - 150;
  }
  const int lead = 31 - __clz(m) + e2;                     // |x| in [2^lead, 2^(lead+1))
  int q = (lead >= 0 ? lead / 4 : -((-lead + 3) / 4)) + 1; // |x| in [16^(q−1), 16^q)
  const int sh = e2 + 24 - 4 * q;                          // F = m·2^sh, F in [2^20, 2^24)
  uint32_t F;
  if (sh >= 0) {
    F = m << sh;
  } else {
    const int r = -sh;                                     // 1..3 for normal inputs
    const uint32_t rem = m & ((1u << r) - 1u), half = 1u << (r - 1);
    F = m >> r;
    if (rem > half || (rem == half && (F & 1u))) ++F;
    if (F == (1u << 24)) {
      F = 1u << 20;
      ++q;
    }
  }
  return sign | ((uint32_t)(q + 64) << 24) | F;
}

// Decode: output column c takes input trace order[c]; its samples go to
// out[dest[c] + s·width[c]] (a column of that shot's (ns, width) record).
// Grid: x over 32-column tiles, y over 32-sample tiles; block 32×8.
__global__ void k_segy_decode(const uint8_t* __restrict__ traces, int64_t ns, int64_t tb, int64_t ncols,
                              const int32_t* __restrict__ order, const int64_t* __restrict__ dest,
                              const int32_t* __restrict__ width, int fmt, float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int64_t c0 = (int64_t)blockIdx.x * 32, s0 = (int64_t)blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += 8) {
    const int64_t c = c0 + j, s = s0 + threadIdx.x;
    float v = 0.f;
    if (c < ncols && s < ns) {
      const uint32_t* w = reinterpret_cast<const uint32_t*>(traces + (int64_t)order[c] * tb + 240);
      const uint32_t word = bswap32(__ldg(w + s));
      v = fmt == 1 ? ibm_to_float(word) : __uint_as_float(word);
    }
    tile[j][threadIdx.x] = v;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t s = s0 + i, c = c0 + threadIdx.x;
    if (c < ncols && s < ns) out[dest[c] + s * (int64_t)width[c]] = tile[threadIdx.x][i];
  }
}

// Encode a (ns, ntr) record: trace k's samples from column k, big-endian.
__global__ void k_segy_encode(const float* __restrict__ rec, int64_t ns, int64_t ntr, int64_t tb, int fmt,
                              uint8_t* __restrict__ traces) {
  __shared__ uint32_t tile[32][33];
  const int64_t c0 = (int64_t)blockIdx.x * 32, s0 = (int64_t)blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t s = s0 + i, c = c0 + threadIdx.x;
    uint32_t word = 0;
    if (c < ntr && s < ns) {
      const float v = rec[s * ntr + c];
      word = bswap32(fmt == 1 ? float_to_ibm(v) : __float_as_uint(v));
    }
    tile[i][threadIdx.x] = word;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += 8) {
    const int64_t c = c0 + j, s = s0 + threadIdx.x;
    if (c < ntr && s < ns) reinterpret_cast<uint32_t*>(traces + c * tb + 240)[s] = tile[threadIdx.x][j];
  }
}

// The 240-byte trace headers, already big-endian, into their trace blocks.
__global__ void k_segy_headers(const uint32_t* __restrict__ hdr, int64_t ntr, int64_t tb,
                               uint8_t* __restrict__ traces) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ntr * 60) return;
  const int64_t k = idx / 60, w = idx - k * 60;
  reinterpret_cast<uint32_t*>(traces + k * tb)[w] = hdr[idx];
}

}  // namespace ertm
