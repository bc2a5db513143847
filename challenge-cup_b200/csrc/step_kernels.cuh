// Staggered-grid velocity / stress update kernels (sm_100a).
//
// One time step of a propagator is two launches: the velocity phase (reads
// the stresses with a halo, updates vx, vz and their ψ strips in place) and
// the stress phase (reads the new velocities with a halo, updates the
// stresses, injects the source, applies the free surface, then runs the
// fused epilogue: image-field store, imaging condition or excitation map).
// Each block owns a 32-column × TZ-row tile of one propagator and runs
// 8 × BZ threads; a thread owns 4 adjacent columns (one float4) of R rows
// (TZ = BZ·R).  The staged fields go to shared memory with an M-cell halo by
// 16-byte cp.async; x-stencils read three 128-bit words per row, z-stencils
// one 128-bit word per row offset; per-cell coefficients and the updated
// fields move as float4 with coalesced 128-byte warp accesses.  TZ (8, 16 or
// 32) is picked per launch so the grid fills the 148 SMs.  A launch may carry many
// propagators (the batched form): a block finds its propagator by binary
// search over the StepWork table.
//
// Arithmetic order follows ertm/propagation.py (acoustic :430-454,
// viscoacoustic :686-723, elastic :840-883), ertm/numerics.py (:68-117,
// :221-227) and ertm/imaging.py (:305-324) so fields and image sums match the
// reference bit for bit.
#pragma once

#include <cuda.h>

#include "ertm_device.cuh"

namespace ertm {

constexpr int TILE_X = 32;
constexpr int XT = 8;   // threads across a tile (4 columns each)

// Shared-memory tile of one staged field: rows [i0−M, i0+TZ+M), columns
// [j0−4, j0+36) — 40 floats per row for every order, so each row is ten
// 16-byte chunks aligned like the global rows (j0 is a multiple of 32, the
// row pitch a multiple of 32 floats).  Column j of the tile sits at OFF + j−j0.
template <int M, int TZ>
struct TileShape {
  static constexpr int W = TILE_X + 8;
  static constexpr int OFF = 4;
  static constexpr int H = TZ + 2 * M;
  static constexpr int N = W * H;
  static constexpr int CHUNKS = H * (W / 4);
};

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int src_size = valid ? 16 : 0;   // 0 → zero-fill, nothing is read
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_size) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Issue the asynchronous copy of one field tile; rows outside [0, nzp) and
// chunks outside [0, ld) are zero-filled (a valid stencil never reads them;
// columns in [nxp, ld) are the row padding, which stays zero).
template <int M, int TZ, int NT>
__device__ __forceinline__ void stage(float* s, const float* __restrict__ g, int nzp, int ld, int i0, int j0) {
  using T = TileShape<M, TZ>;
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < (T::CHUNKS + NT - 1) / NT; ++it) {
    const int idx = tid + it * NT;
    if (T::CHUNKS % NT != 0 && idx >= T::CHUNKS) break;
    const int r = idx / (T::W / 4);
    const int ch = idx - r * (T::W / 4);
    const int gi = i0 - M + r, gj = j0 - T::OFF + 4 * ch;
    const bool ok = gi >= 0 && gi < nzp && gj >= 0 && gj < ld;
    cp_async16(s + r * T::W + 4 * ch, ok ? g + (size_t)gi * ld + gj : g, ok);
  }
}

// Issue the asynchronous copy of one per-cell operand tile (no halo): rows
// [i0, i0+TZ) × columns [j0, j0+32) into a TZ × 32 shared array; rows past
// the grid are zero-filled (j0 + 32 ≤ ld always holds).
template <int TZ, int NT>
__device__ __forceinline__ void stage_cells(float* s, const float* __restrict__ g, int nzp, int ld, int i0, int j0) {
  constexpr int CH = TZ * 8;
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < (CH + NT - 1) / NT; ++it) {
    const int idx = tid + it * NT;
    if (CH % NT != 0 && idx >= CH) break;
    const int r = idx >> 3, ch = idx & 7;
    const int gi = i0 + r;
    const bool ok = gi < nzp;
    cp_async16(s + r * 32 + 4 * ch, ok ? g + (size_t)gi * ld + j0 + 4 * ch : g, ok);
  }
}

// Several arrays of one propagator staged together: they share the row pitch,
// so a thread computes each chunk's offset and bounds once and issues one copy
// per array.
template <int M, int TZ, int NT, int NF>
__device__ __forceinline__ void stage_n(float* const (&s)[NF], const float* const (&g)[NF], int nzp, int ld, int i0,
                                        int j0) {
  using T = TileShape<M, TZ>;
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < (T::CHUNKS + NT - 1) / NT; ++it) {
    const int idx = tid + it * NT;
    if (T::CHUNKS % NT != 0 && idx >= T::CHUNKS) break;
    const int r = idx / (T::W / 4);
    const int ch = idx - r * (T::W / 4);
    const int gi = i0 - M + r, gj = j0 - T::OFF + 4 * ch;
    const bool ok = gi >= 0 && gi < nzp && gj >= 0 && gj < ld;
    const size_t off = ok ? (size_t)gi * ld + gj : 0;
    const int so = r * T::W + 4 * ch;
#pragma unroll
    for (int f = 0; f < NF; ++f) cp_async16(s[f] + so, g[f] + off, ok);
  }
}

template <int TZ, int NT, int NF>
__device__ __forceinline__ void stage_cells_n(float* const (&s)[NF], const float* const (&g)[NF], int nzp, int ld,
                                              int i0, int j0) {
  constexpr int CH = TZ * 8;
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < (CH + NT - 1) / NT; ++it) {
    const int idx = tid + it * NT;
    if (CH % NT != 0 && idx >= CH) break;
    const int r = idx >> 3, ch = idx & 7;
    const int gi = i0 + r;
    const bool ok = gi < nzp;
    const size_t off = ok ? (size_t)gi * ld + j0 + 4 * ch : 0;
    const int so = r * 32 + 4 * ch;
#pragma unroll
    for (int f = 0; f < NF; ++f) cp_async16(s[f] + so, g[f] + off, ok);
  }
}

// Row ranges of the same copies (local tile rows: [RLO, RHI) of the halo tile,
// rows 0 … TZ+2M; of the cell tile, rows 0 … TZ), for tiles staged in two
// commit groups.
template <int M, int TZ, int NT, int NF, int RLO, int RHI>
__device__ __forceinline__ void stage_n_rows(float* const (&s)[NF], const float* const (&g)[NF], int nzp, int ld,
                                             int i0, int j0) {
  using T = TileShape<M, TZ>;
  constexpr int C0 = RLO * (T::W / 4), CH = (RHI - RLO) * (T::W / 4);
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < (CH + NT - 1) / NT; ++it) {
    const int idx = C0 + tid + it * NT;
    if (CH % NT != 0 && idx >= C0 + CH) break;
    const int r = idx / (T::W / 4);
    const int ch = idx - r * (T::W / 4);
    const int gi = i0 - M + r, gj = j0 - T::OFF + 4 * ch;
    const bool ok = gi >= 0 && gi < nzp && gj >= 0 && gj < ld;
    const size_t off = ok ? (size_t)gi * ld + gj : 0;
    const int so = r * T::W + 4 * ch;
#pragma unroll
    for (int f = 0; f < NF; ++f) cp_async16(s[f] + so, g[f] + off, ok);
  }
}

template <int TZ, int NT, int NF, int RLO, int RHI>
__device__ __forceinline__ void stage_cells_n_rows(float* const (&s)[NF], const float* const (&g)[NF], int nzp, int ld,
                                                   int i0, int j0) {
  constexpr int C0 = RLO * 8, CH = (RHI - RLO) * 8;
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < (CH + NT - 1) / NT; ++it) {
    const int idx = C0 + tid + it * NT;
    if (CH % NT != 0 && idx >= C0 + CH) break;
    const int r = idx >> 3, ch = idx & 7;
    const int gi = i0 + r;
    const bool ok = gi < nzp;
    const size_t off = ok ? (size_t)gi * ld + j0 + 4 * ch : 0;
    const int so = r * 32 + 4 * ch;
#pragma unroll
    for (int f = 0; f < NF; ++f) cp_async16(s[f] + so, g[f] + off, ok);
  }
}

__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Interior tiles of two row halves: the copies the first half needs (halo rows
// i0−M … i0+TZ/2+M, cell rows i0 … i0+TZ/2) form one commit group, the rest a
// second, so the first half computes while the second half's copies are in
// flight.  No wait here: the kernel waits for one group (cp_async_wait_one +
// __syncthreads) before the first half and for both before the second.
template <int M, int TZ, int NT, int NH, int NC>
__device__ __forceinline__ void stage_tile_halves(const DevProp& P, int i0, int j0, float* const (&hd)[NH],
                                                  const int (&hf)[NH], float* const (&cd)[NC], const int (&cf)[NC]) {
  constexpr int HALF = TZ / 2;
  const float* hg[NH];
  const float* cg[NC];
#pragma unroll
  for (int k = 0; k < NH; ++k) hg[k] = P.f[hf[k]];
#pragma unroll
  for (int k = 0; k < NC; ++k) cg[k] = cf[k] >= 0 ? P.f[cf[k]] : P.coef[~cf[k]];
  stage_n_rows<M, TZ, NT, NH, 0, HALF + 2 * M>(hd, hg, P.nzp, P.ld, i0, j0);
  stage_cells_n_rows<TZ, NT, NC, 0, HALF>(cd, cg, P.nzp, P.ld, i0, j0);
  cp_async_commit();
  stage_n_rows<M, TZ, NT, NH, HALF + 2 * M, TZ + 2 * M>(hd, hg, P.nzp, P.ld, i0, j0);
  stage_cells_n_rows<TZ, NT, NC, HALF, TZ>(cd, cg, P.nzp, P.ld, i0, j0);
  cp_async_commit();
}

// ---------------------------------------------------------------------------
// TMA staging (interior tiles): one thread issues a tiled bulk copy per array
// (halo boxes of 40 × (TZ+2M) floats at x = j0 − 4, cell boxes of 32 × TZ at
// x = j0: both x offsets are multiples of 4 floats, i.e. 16 bytes), all
// completing on one mbarrier; rows and columns outside the tensor read as
// zero, as the cp.async path zero-fills them.  Waits are bounded: a wait that
// runs out counts in g_stage_timeouts (the host reports it as an error) and
// the block skips its tile.
// ---------------------------------------------------------------------------
struct TmaNone {
  static constexpr bool kOn = false;
};
// The propagator's own tensor maps in device memory (DevProp::tmap, written
// by the host at creation): per tile height, [0] the state block with a halo
// box, [1] the state block with a cell box, [2] the coefficient block with a
// cell box.
struct TmaGlobal {
  static constexpr bool kOn = true;
  __device__ __forceinline__ const CUtensorMap* maps(int, const DevProp& P, int tz) const {
    return static_cast<const CUtensorMap*>(P.tmap) + 3 * (tz == 8 ? 0 : (tz == 16 ? 1 : 2));
  }
};

__device__ unsigned int g_stage_timeouts;
constexpr int kTmaSpinLimit = 1 << 22;   // try_wait rounds (each suspends briefly): seconds, not forever

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done = 0;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < kTmaSpinLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Stage one tile: NH halo arrays (state-block field slots hf) and NC cell
// arrays (cf ≥ 0: state-block field slot; cf < 0: coefficient ~cf).  Returns
// false (for the whole block) only when a bounded TMA wait ran out.
template <int M, int TZ, int NT, int NH, int NC, class TM>
__device__ __forceinline__ bool stage_tile(const TM& tm, int slot, const DevProp& P, int i0, int j0,
                                           float* const (&hd)[NH], const int (&hf)[NH], float* const (&cd)[NC],
                                           const int (&cf)[NC], uint64_t* bar) {
  using T = TileShape<M, TZ>;
  const int tid = threadIdx.y * XT + threadIdx.x;
  if constexpr (TM::kOn) {
    if (tid == 0) mbar_init(bar, 1);
    __syncthreads();
    if (tid == 0) {
      const CUtensorMap* m = tm.maps(slot, P, TZ);
#pragma unroll
      for (int q = 0; q < 3; ++q)
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(m + q) : "memory");
      mbar_expect_tx(bar, (uint32_t)((NH * T::N + NC * TZ * 32) * sizeof(float)));
#pragma unroll
      for (int k = 0; k < NH; ++k) tma_load_3d(hd[k], &m[0], j0 - T::OFF, i0 - M, hf[k], bar);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        if (cf[k] >= 0) tma_load_3d(cd[k], &m[1], j0, i0, cf[k], bar);
        else tma_load_3d(cd[k], &m[2], j0, i0, ~cf[k], bar);
      }
    }
    bool ok = mbar_wait_bounded(bar, 0);
    if (!ok) {
      atomicAdd(&g_stage_timeouts, 1u);
      ok = mbar_wait_bounded(bar, 0);   // the copies still write this block's shared memory
    }
    return __syncthreads_and(ok) != 0;
  } else {
    const float* hg[NH];
    const float* cg[NC];
#pragma unroll
    for (int k = 0; k < NH; ++k) hg[k] = P.f[hf[k]];
#pragma unroll
    for (int k = 0; k < NC; ++k) cg[k] = cf[k] >= 0 ? P.f[cf[k]] : P.coef[~cf[k]];
    stage_n<M, TZ, NT, NH>(hd, hg, P.nzp, P.ld, i0, j0);
    stage_cells_n<TZ, NT, NC>(cd, cg, P.nzp, P.ld, i0, j0);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    return true;
  }
}

struct TileLoc {
  int i0, j0;
};

__device__ __forceinline__ TileLoc tile_of(const StepWork& w, int block, int tz) {
  const int t = block - w.tile0;
  const int ti = t / w.tiles_x;
  return {ti * tz, (t - ti * w.tiles_x) * TILE_X};
}

// Tile kinds of a launch: 0 every tile of the propagators (each block picks
// the interior or the boundary form), 1 the interior rectangle only, 2 the
// boundary frame (and the hole) only.
constexpr int TILES_ALL = 0, TILES_INTERIOR = 1, TILES_FRAME = 2;

template <int KIND>
__device__ __forceinline__ TileLoc tile_loc(const StepWork& w, int block, int tz) {
  if constexpr (KIND == TILES_ALL) {
    return tile_of(w, block, tz);
  } else if constexpr (KIND == TILES_INTERIOR) {
    const int nx_r = w.tj1 - w.tj0;
    int k = block - w.tile0;
    if (w.hole_i >= 0 && k >= (w.hole_i - w.ti0) * nx_r + (w.hole_j - w.tj0)) ++k;
    const int q = k / nx_r;
    return {(w.ti0 + q) * tz, (w.tj0 + (k - q * nx_r)) * TILE_X};
  } else {
    int k = block - w.tile0;
    const int tx = w.tiles_x, rows = w.tiles / w.tiles_x;
    const int top = w.ti0 * tx;
    if (k < top) return {(k / tx) * tz, (k % tx) * TILE_X};
    k -= top;
    const int bottom = (rows - w.ti1) * tx;
    if (k < bottom) return {(w.ti1 + k / tx) * tz, (k % tx) * TILE_X};
    k -= bottom;
    const int side = w.tj0 + (tx - w.tj1);
    if (k < (w.ti1 - w.ti0) * side) {
      const int q = k / side, c = k - q * side;
      return {(w.ti0 + q) * tz, (c < w.tj0 ? c : w.tj1 + (c - w.tj0)) * TILE_X};
    }
    // the hole: one tile, or the several lower frame tiles of one interior tile
    k -= (w.ti1 - w.ti0) * side;
    return {(w.hole_i + k) * tz, w.hole_j * TILE_X};
  }
}

// Source amplitudes of this step: float32(amp) for the field and, for the
// viscoacoustic strain, float32(amp / K_R) computed in float64
// (propagation.py:707-713).
__device__ __forceinline__ void source_amps(const StepWork& w, const DevProp& P, float& amp, float& amp_eps) {
  if (w.wavelet == nullptr) {
    amp = w.amp;
    amp_eps = w.amp_eps;
    return;
  }
  amp = w.wavelet[w.t];
  amp_eps = 0.f;
  if (P.engine == ENGINE_VISCO && amp != 0.f && P.src_iz >= 0) {
    const float kr = P.coef[CV_KR][(size_t)P.src_iz * P.ld + P.src_ix];
    amp_eps = __double2float_rn(__ddiv_rn((double)amp, (double)kr));
  }
}

// ---------------------------------------------------------------------------
// fused epilogue on one physical cell
// ---------------------------------------------------------------------------
__device__ __forceinline__ void acc_term(double* base, int kahan, size_t c, size_t npix, float term) {
  if (!kahan) {
    base[c] = dadd(base[c], (double)term);
  } else {
    float* s = reinterpret_cast<float*>(base);
    float* comp = s + npix;
    const float y = fsub(term, comp[c]);
    const float sv = s[c];
    const float t = fadd(sv, y);
    comp[c] = fsub(fsub(t, sv), y);
    s[c] = t;
  }
}

__device__ __forceinline__ void run_epilogue(const Epilogue& E, size_t c, size_t npix, float pv, float sv) {
  switch (E.kind) {
    case EPI_STORE:
      if (E.out[0]) E.out[0][c] = pv;
      if (E.out[1]) E.out[1][c] = sv;
      break;
    case EPI_IMAGE: {
      // imaging.py:313-324: illum += S², rillum += R² (all steps); num += S·R (t ≥ start)
      const float s0 = E.src[0] ? E.src[0][c] : 0.f;
      const float s1 = E.src[1] ? E.src[1][c] : 0.f;
      if (!E.kahan) {
        // float64 sums: every accumulator value is loaded before any is
        // stored, so the loads are in flight together (the compiler cannot
        // move a load above a store to another accumulator by itself)
        double vi[MAX_EPI_IMAGES], vr[MAX_EPI_IMAGES], vn[MAX_EPI_IMAGES];
#pragma unroll
        for (int k = 0; k < MAX_EPI_IMAGES; ++k) {
          if (k >= E.n_images) break;
          if (E.illum && E.ill[k]) vi[k] = E.ill[k][c];
          if (E.rillum && E.ril[k]) vr[k] = E.ril[k][c];
          if (E.cross) vn[k] = E.num[k][c];
        }
#pragma unroll
        for (int k = 0; k < MAX_EPI_IMAGES; ++k) {
          if (k >= E.n_images) break;
          const float s = E.src_slot[k] ? s1 : s0;
          const float r = E.rcv_wave[k] ? sv : pv;
          if (E.illum && E.ill[k]) E.ill[k][c] = dadd(vi[k], (double)fmul(s, s));
          if (E.rillum && E.ril[k]) E.ril[k][c] = dadd(vr[k], (double)fmul(r, r));
          if (E.cross) E.num[k][c] = dadd(vn[k], (double)fmul(s, r));
        }
        break;
      }
#pragma unroll
      for (int k = 0; k < MAX_EPI_IMAGES; ++k) {
        if (k >= E.n_images) break;
        const float s = E.src_slot[k] ? s1 : s0;
        const float r = E.rcv_wave[k] ? sv : pv;
        if (E.illum && E.ill[k]) acc_term(E.ill[k], E.kahan, c, npix, fmul(s, s));
        if (E.rillum && E.ril[k]) acc_term(E.ril[k], E.kahan, c, npix, fmul(r, r));
        if (E.cross) acc_term(E.num[k], E.kahan, c, npix, fmul(s, r));
      }
      break;
    }
    case EPI_EXC_TRACK: {
      // imaging.py:466-473: strict '>' against the running |P| maximum
      const float a = fabsf(pv);
      if (a > E.running[c]) {
        E.running[c] = a;
        E.peak_step[c] = E.step;
      }
      break;
    }
    case EPI_EXC_IMAGE: {
      // imaging.py:295-303: num += A·R in float64, rillum += R² (float32 square)
      if (E.peak_step[c] != E.step) break;
      const double a = (double)E.running[c];
#pragma unroll
      for (int k = 0; k < MAX_EPI_IMAGES; ++k) {
        if (k >= E.n_images) break;
        const float r = E.rcv_wave[k] ? sv : pv;
        E.num[k][c] = dadd(E.num[k][c], dmul(a, (double)r));
        if (E.ril[k]) E.ril[k][c] = dadd(E.ril[k][c], (double)fmul(r, r));
      }
      break;
    }
    default:
      break;
  }
}

// The epilogue of one tile: the stress phase leaves P and S of its cells in
// shared memory (TZ rows × 32 columns); the block then walks the tile one cell
// per thread, so a warp covers 32 consecutive physical cells of a row and its
// accumulator, replay and excitation accesses coalesce whatever their
// alignment.  One copy of the epilogue code serves every cell.
//
// The imaging condition with float64 sums (the common case) gathers: a thread
// loads the replayed source values of all its cells, then, accumulator by
// accumulator, loads all its cells' sums before it adds and stores them, so
// several global loads are in flight per thread instead of one.
template <int IT>
struct ImageCells {
  uint32_t pc[IT];
  bool ok[IT];
  float s0[IT], s1[IT];
};

template <int IT, class TERM>
__device__ __forceinline__ void accumulate_cells(double* acc, const ImageCells<IT>& C, TERM term) {
  double a[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) a[it] = C.ok[it] ? acc[C.pc[it]] : 0.0;
#pragma unroll
  for (int it = 0; it < IT; ++it)
    if (C.ok[it]) acc[C.pc[it]] = dadd(a[it], (double)term(it));
}

template <int TZ, int NT, class GEO>
__device__ __forceinline__ void image_tile_f64(const Epilogue& E, const GEO& G, int i0, int j0, const float* e_p,
                                               const float* e_s) {
  constexpr int IT = TZ * 32 / NT;
  const int tid = threadIdx.y * XT + threadIdx.x;
  ImageCells<IT> C;
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int idx = tid + it * NT;
    size_t pc = 0;
    C.ok[it] = G.physical(i0 + (idx >> 5), j0 + (idx & 31), pc);
    C.pc[it] = (uint32_t)pc;
  }
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    C.s0[it] = (C.ok[it] && E.src[0]) ? E.src[0][C.pc[it]] : 0.f;
    C.s1[it] = (C.ok[it] && E.src[1]) ? E.src[1][C.pc[it]] : 0.f;
  }
#pragma unroll 1
  for (int k = 0; k < E.n_images; ++k) {
    const bool s_is_1 = E.src_slot[k] != 0;
    const bool r_is_s = E.rcv_wave[k] != 0;
    auto src = [&](int it) { return s_is_1 ? C.s1[it] : C.s0[it]; };
    auto rcv = [&](int it) { return r_is_s ? (e_s ? e_s[tid + it * NT] : 0.f) : e_p[tid + it * NT]; };
    // imaging.py:313-324: illum += S², rillum += R² (all steps); num += S·R (t ≥ start)
    if (E.illum && E.ill[k]) accumulate_cells(E.ill[k], C, [&](int it) { return fmul(src(it), src(it)); });
    if (E.rillum && E.ril[k]) accumulate_cells(E.ril[k], C, [&](int it) { return fmul(rcv(it), rcv(it)); });
    if (E.cross) accumulate_cells(E.num[k], C, [&](int it) { return fmul(src(it), rcv(it)); });
  }
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

// Before the stencil of an interior tile: pull into L2 the lines that the
// float64 imaging epilogue will read-modify-write at the end of the block (the
// tile's physical cells of every accumulator this step touches) and the stored
// source fields it reads, so those loads hit L2 instead of DRAM.  Only
// addresses of the tile's physical cells are touched.
template <int TZ, int NT, class GEO>
__device__ __forceinline__ void prefetch_image_tile(const Epilogue& E, const GEO& G, int i0, int j0) {
  if (E.kind != EPI_IMAGE || E.kahan) return;
  const int ja = max(j0, G.pad), jb = min(j0 + TILE_X, G.pad + G.nx);
  const int ia = max(i0, G.pad), ib = min(i0 + TZ, G.pad + G.nz);
  if (ja >= jb || ia >= ib) return;
  const void* arr[3 * MAX_EPI_IMAGES + 2];
  int esz[3 * MAX_EPI_IMAGES + 2];
  int na = 0;
  for (int k = 0; k < E.n_images && k < MAX_EPI_IMAGES; ++k) {
    if (E.illum && E.ill[k]) { arr[na] = E.ill[k]; esz[na++] = 8; }
    if (E.rillum && E.ril[k]) { arr[na] = E.ril[k]; esz[na++] = 8; }
    if (E.cross && E.num[k]) { arr[na] = E.num[k]; esz[na++] = 8; }
  }
  for (int q = 0; q < 2; ++q)
    if (E.src[q]) { arr[na] = E.src[q]; esz[na++] = 4; }
  const int tid = threadIdx.y * XT + threadIdx.x;
  const int rows = ib - ia;
  for (int w = tid; w < rows * na; w += NT) {
    const int a = w / rows, i = ia + w - a * rows;
    const char* row = static_cast<const char*>(arr[a]) + ((size_t)(i - G.pad) * G.nx + (ja - G.pad)) * esz[a];
    const int bytes = (jb - ja) * esz[a];
    for (int b = 0; b < bytes; b += 128) prefetch_l2(row + b);
    prefetch_l2(row + bytes - 1);
  }
}

template <int TZ, int NT, class GEO>
__device__ __forceinline__ void epilogue_tile(const Epilogue& E, const GEO& G, int i0, int j0, const float* e_p,
                                              const float* e_s, size_t npix) {
  if (E.kind == EPI_IMAGE && !E.kahan && (TZ * 32) % NT == 0) {
    image_tile_f64<TZ, NT>(E, G, i0, j0, e_p, e_s);
    return;
  }
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll 1
  for (int idx = tid; idx < TZ * 32; idx += NT) {
    size_t pc;
    if (G.physical(i0 + (idx >> 5), j0 + (idx & 31), pc)) run_epilogue(E, pc, npix, e_p[idx], e_s ? e_s[idx] : 0.f);
  }
}

// Scalars and pointers of one propagator, loaded once into registers at the
// top of a kernel (the kernels store through float pointers, so reading the
// DevProp in global memory after a store would force a reload).
struct Geo {
  int nzp, nxp, ld, wx, npx_l, npx_r, npz_t, npz_b, pad, nz, nx, src_iz, src_ix, free_surface, fast_x, fast_z;
  float c[4];
  float dt, hx, hz, rx32, rz32, rxl, rzl;
  double rx, rz;
  __device__ __forceinline__ explicit Geo(const DevProp& P)
      : nzp(P.nzp), nxp(P.nxp), ld(P.ld), wx(P.wx), npx_l(P.npx_l), npx_r(P.npx_r), npz_t(P.npz_t),
        npz_b(P.npz_b), pad(P.pad), nz(P.nz), nx(P.nx), src_iz(P.src_iz), src_ix(P.src_ix),
        free_surface(P.free_surface), fast_x(P.fast_x), fast_z(P.fast_z), c{P.c[0], P.c[1], P.c[2], P.c[3]},
        dt(P.dt), hx(P.hx), hz(P.hz), rx32(P.rx32), rz32(P.rz32), rxl(P.rxl), rzl(P.rzl), rx(P.rx), rz(P.rz) {}
  __device__ __forceinline__ float dx_(float a) const { return divh(a, hx, rx, rx32, rxl, fast_x); }
  __device__ __forceinline__ float dz_(float a) const { return divh(a, hz, rz, rz32, rzl, fast_z); }
  // Straight-line interior form (only used when the float64-product form was verified).
  __device__ __forceinline__ float dxf(float a) const { return __double2float_rn(__dmul_rn((double)a, rx)); }
  __device__ __forceinline__ float dzf(float a) const { return __double2float_rn(__dmul_rn((double)a, rz)); }
  // Boundary tiles of a split launch: the host splits only propagators whose
  // spacings passed the float64-product check, so that form is the only one.
  template <int KIND>
  __device__ __forceinline__ float dxk(float a) const { return KIND == 2 ? dxf(a) : dx_(a); }
  template <int KIND>
  __device__ __forceinline__ float dzk(float a) const { return KIND == 2 ? dzf(a) : dz_(a); }
  // A tile whose cells are all physical, away from every CPML strip, the
  // free-surface row and the source node, with the FMA division verified:
  // its stencils run without per-cell branches.
  __device__ __forceinline__ bool interior(int i0, int j0, int tz) const {
    const int i1 = i0 + tz, j1 = j0 + 32;
    const bool phys = i0 >= pad && i1 <= pad + nz && j0 >= pad && j1 <= pad + nx;
    const bool strips = i0 >= npz_t && i1 <= nzp - npz_b && j0 >= npx_l && j1 <= nxp - npx_r;
    const bool fs = !free_surface || i0 > pad;
    const bool src = !(src_iz >= i0 && src_iz < i1 && src_ix >= j0 && src_ix < j1);
    return phys && strips && fs && src && fast_x == 1 && fast_z == 1;
  }
  __device__ __forceinline__ int sx(int j) const {
    if (j < npx_l) return j;
    if (j >= nxp - npx_r) return npx_l + (j - (nxp - npx_r));
    return -1;
  }
  __device__ __forceinline__ int sz(int i) const {
    if (i < npz_t) return i;
    if (i >= nzp - npz_b) return npz_t + (i - (nzp - npz_b));
    return -1;
  }
  __device__ __forceinline__ bool physical(int i, int j, size_t& c) const {
    const int ii = i - pad, jj = j - pad;
    if (ii < 0 || ii >= nz || jj < 0 || jj >= nx) return false;
    c = (size_t)ii * nx + jj;
    return true;
  }
};

__device__ __forceinline__ bool physical(const DevProp& P, int i, int j, size_t& c) {
  const int ii = i - P.pad, jj = j - P.pad;
  if (ii < 0 || ii >= P.nz || jj < 0 || jj >= P.nx) return false;
  c = (size_t)ii * P.nx + jj;
  return true;
}

// ---------------------------------------------------------------------------
// register stencils on 4 adjacent columns
// ---------------------------------------------------------------------------
// Twelve consecutive values of one staged row, columns j−4 … j+7 of the
// thread's first column j (shared-memory column 4·tx … 4·tx+11).
__device__ __forceinline__ void row12(const float* p, float v[12]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  const float4 b = *reinterpret_cast<const float4*>(p + 4);
  const float4 c = *reinterpret_cast<const float4*>(p + 8);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  v[8] = c.x; v[9] = c.y; v[10] = c.z; v[11] = c.w;
}

// Column c (0..3) of rows −M … +M around the thread's row: z[c][M+k] = f[i+k].
template <int M>
__device__ __forceinline__ void col9(const float* p /* row i, column j */, float z[4][2 * M + 1]) {
#pragma unroll
  for (int k = 0; k <= 2 * M; ++k) {
    const float4 q = *reinterpret_cast<const float4*>(p + (k - M) * 40);
    z[0][k] = q.x; z[1][k] = q.y; z[2][k] = q.z; z[3][k] = q.w;
  }
}

// Σ_k c_k (f[o+k] − f[o−k+1]) (D⁺ numerator) on an array with static indices.
template <int M>
__device__ __forceinline__ float sum_plus(const float* f, int o, const float* c) {
  float acc = fmul(c[0], fsub(f[o + 1], f[o]));
#pragma unroll
  for (int k = 2; k <= M; ++k) acc = fadd(acc, fmul(c[k - 1], fsub(f[o + k], f[o - k + 1])));
  return acc;
}
// Σ_k c_k (f[o+k−1] − f[o−k]) (D⁻ numerator).
template <int M>
__device__ __forceinline__ float sum_minus(const float* f, int o, const float* c) {
  float acc = fmul(c[0], fsub(f[o], f[o - 1]));
#pragma unroll
  for (int k = 2; k <= M; ++k) acc = fadd(acc, fmul(c[k - 1], fsub(f[o + k - 1], f[o - k])));
  return acc;
}

__device__ __forceinline__ float comp(const float4& v, int c) {
  return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_comp(float4& v, int c, float x) {
  if (c == 0) v.x = x; else if (c == 1) v.y = x; else if (c == 2) v.z = x; else v.w = x;
}
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float4 ldg4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void st4(float* p, const float4& v) { *reinterpret_cast<float4*>(p) = v; }

// Per-column x information for the thread's 4 columns.
struct ColInfo {
  bool xin[4];   // x-stencil inside [M, nxp − M)
  bool ok[4];    // column inside the padded grid
  int sx[4];     // x-strip index or −1
  float ax[4], bx[4];
};
template <int M>
__device__ __forceinline__ ColInfo col_info(const Geo& G, int j, const float* axp, const float* bxp) {
  ColInfo C;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int jc = j + c;
    C.ok[c] = jc < G.nxp;
    C.xin[c] = jc >= M && jc < G.nxp - M;
    C.sx[c] = C.ok[c] ? G.sx(jc) : -1;
    C.ax[c] = C.sx[c] >= 0 ? axp[jc] : 0.f;
    C.bx[c] = C.sx[c] >= 0 ? bxp[jc] : 1.f;
  }
  return C;
}

// Viscoacoustic memory variables of one thread's 4 cells (propagation.py:
// 700-705): r_l ← r_l·a_l(Q) + b_l·Δε for l = 0 … L−1, total = Σ_l r_l in
// that order.  Each r_l and b_l row is one aligned 16-byte word, so a
// mechanism costs two vector loads and one vector store.  Columns with
// keep[c] set are left as they are.  Up to kRelaxUnroll mechanisms run
// unrolled.
constexpr int kRelaxUnroll = 4;
__device__ __forceinline__ void relax4(float* r0, const float* b0, size_t fstride, const uint8_t* qidx,
                                       const float* relax_a, int nL, size_t g, const float (&inc)[4],
                                       const bool (&keep)[4], float (&tot)[4]) {
  const uchar4 q4 = *reinterpret_cast<const uchar4*>(qidx + g);
  const int q[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
  for (int c = 0; c < 4; ++c) tot[c] = 0.f;
  if (nL <= kRelaxUnroll) {
    // every mechanism's memory and coefficient loaded before any memory is
    // stored, so all the loads are in flight together (the compiler cannot
    // move a load of r_{l+1} above the store of r_l by itself: it does not
    // know that the arrays are distinct)
    float4 r4[kRelaxUnroll], b4[kRelaxUnroll];
#pragma unroll
    for (int l = 0; l < kRelaxUnroll; ++l) {
      if (l < nL) {
        r4[l] = ld4(r0 + l * fstride + g);
        b4[l] = ldg4(b0 + l * fstride + g);
      }
    }
#pragma unroll
    for (int l = 0; l < kRelaxUnroll; ++l) {
      if (l < nL) {
        float4 o4;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float rv = fadd(fmul(comp(r4[l], c), __ldg(relax_a + q[c] * nL + l)), fmul(comp(b4[l], c), inc[c]));
          set_comp(o4, c, keep[c] ? comp(r4[l], c) : rv);
          tot[c] = (l == 0) ? rv : fadd(tot[c], rv);
        }
        st4(r0 + l * fstride + g, o4);
      }
    }
    return;
  }
  for (int l = 0; l < nL; ++l) {
    float* rl = r0 + l * fstride;
    const float4 r4 = ld4(rl + g);
    const float4 b4 = ldg4(b0 + l * fstride + g);
    float4 o4;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float rv = fadd(fmul(comp(r4, c), __ldg(relax_a + q[c] * nL + l)), fmul(comp(b4, c), inc[c]));
      set_comp(o4, c, keep[c] ? comp(r4, c) : rv);
      tot[c] = (l == 0) ? rv : fadd(tot[c], rv);
    }
    st4(rl + g, o4);
  }
}

// CPML memories of one thread's 4 cells in one x-strip and one z-strip
// array, loaded together before any is updated (the cells' memories are
// distinct, so the loads can all be in flight at once).  z-strip rows hold ld
// columns, so their 4 cells are one aligned 16-byte word.
struct PsiCells {
  float x[4];
  float4 z;
};
__device__ __forceinline__ PsiCells psi_cells(const ColInfo& C, const float* psx, int i, int wx, const float* psz,
                                              int sz, int ld, int j) {
  PsiCells q;
#pragma unroll
  for (int c = 0; c < 4; ++c) q.x[c] = (C.ok[c] && C.sx[c] >= 0) ? psx[(size_t)i * wx + C.sx[c]] : 0.f;
  q.z = sz >= 0 ? ld4(psz + (size_t)sz * ld + j) : make_float4(0.f, 0.f, 0.f, 0.f);
  return q;
}

// ---------------------------------------------------------------------------
// velocity phase
// ---------------------------------------------------------------------------
// Acoustic and viscoacoustic: vx += (dt·irx)·(D⁺ₓp + ψ), vz += (dt·irz)·(D⁺_z p + ψ).
template <int M, int BZ, int R, int KIND, class WS, class TM>
__global__ void __launch_bounds__(XT* BZ)
k_pressure_velocity(const DevProp* __restrict__ props, const WS ws, const __grid_constant__ TM tm) {
  constexpr int TZ = BZ * R;
  using T = TileShape<M, TZ>;
  __shared__ __align__(128) float sp[T::N];
  __shared__ __align__(128) float c_vx[TZ * 32];
  __shared__ __align__(128) float c_vz[TZ * 32];
  __shared__ __align__(128) float c_irx[TZ * 32];
  __shared__ __align__(128) float c_irz[TZ * 32];
  __shared__ uint64_t tma_bar;
  const StepWork& w = ws.get(blockIdx.x);
  const DevProp& P = props[w.prop];
  const Geo G(P);
  const TileLoc L = tile_loc<KIND>(w, blockIdx.x, TZ);
  float* const vx = P.f[A_VX];
  float* const vz = P.f[A_VZ];
  const float* const irx = P.coef[CA_IRX];
  const float* const irz = P.coef[CA_IRZ];
  float* const psx = P.psix[0];
  float* const psz = P.psiz[0];
  const float* const azp = P.az; const float* const bzp = P.bz;
  if ((w.flags & STEP_PEAK) && blockIdx.x == w.tile0 && threadIdx.x == 0 && threadIdx.y == 0)
    *P.peak = 0.f;  // the stress phase of this step reduces into it
  // interior 32-row tiles staged in two halves (see stage_tile_halves)
  constexpr bool HALVES = KIND == TILES_INTERIOR && !TM::kOn && R == 2;
  {
    float* const hd[1] = {sp};
    const int hf[1] = {A_P};
    float* const cd[4] = {c_vx, c_vz, c_irx, c_irz};
    const int cf[4] = {A_VX, A_VZ, ~CA_IRX, ~CA_IRZ};
    if constexpr (HALVES) {
      stage_tile_halves<M, TZ, XT * BZ>(P, L.i0, L.j0, hd, hf, cd, cf);
    } else {
      if (!stage_tile<M, TZ, XT * BZ>(tm, w.slot, P, L.i0, L.j0, hd, hf, cd, cf, &tma_bar)) return;
    }
  }
  (void)irx;
  (void)irz;
  const int j = L.j0 + 4 * threadIdx.x;
#define CELL(arr, rr) ld4(arr + (rr) * 32 + 4 * threadIdx.x)
  if (HALVES && (j >= G.nxp || !G.interior(L.i0, L.j0, TZ))) {
    cp_async_wait_all();   // never exit with copies into this block's shared memory in flight
    return;
  }
  if (j >= G.nxp) return;
  if (KIND == TILES_INTERIOR && !G.interior(L.i0, L.j0, TZ)) return;   // the host plans only interior tiles here
  if (KIND == TILES_INTERIOR || (KIND == TILES_ALL && G.interior(L.i0, L.j0, TZ))) {
    if constexpr (KIND != TILES_FRAME) {
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      if constexpr (HALVES) {
        if (r == 0) cp_async_wait_one();
        else cp_async_wait_all();
        __syncthreads();
      }
      const int rr = threadIdx.y + BZ * r;
      const float* row = sp + (rr + M) * T::W + 4 * threadIdx.x;
      const size_t g = (size_t)(L.i0 + rr) * G.ld + j;
      float v[12];
      row12(row, v);
      float z[4][2 * M + 1];
      col9<M>(row + 4, z);
      float4 ox, oz;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float dx = G.dxf(sum_plus<M>(v, 4 + c, G.c));
        const float dz = G.dzf(sum_plus<M>(z[c], M, G.c));
        set_comp(ox, c, fadd(comp(CELL(c_vx, rr), c), fmul(fmul(G.dt, comp(CELL(c_irx, rr), c)), dx)));
        set_comp(oz, c, fadd(comp(CELL(c_vz, rr), c), fmul(fmul(G.dt, comp(CELL(c_irz, rr), c)), dz)));
      }
      st4(vx + g, ox);
      st4(vz + g, oz);
    }
    }
    return;
  }
  if constexpr (KIND != TILES_INTERIOR) {
  const ColInfo C = col_info<M>(G, j, P.ax, P.bx);
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    const int rr = threadIdx.y + BZ * r;
    const int i = L.i0 + rr;
    if (i >= G.nzp) break;
    const float* row = sp + (rr + M) * T::W + 4 * threadIdx.x;
    const size_t g = (size_t)i * G.ld + j;
    const bool zin = (i >= M && i < G.nzp - M);
    const int sz = G.sz(i);
    const float azi = sz >= 0 ? azp[i] : 0.f, bzi = sz >= 0 ? bzp[i] : 1.f;
    PsiCells q = psi_cells(C, psx, i, G.wx, psz, sz, G.ld, j);
    float v[12];
    row12(row, v);
    float4 ox = CELL(c_vx, rr);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (!C.ok[c]) continue;
      float d = C.xin[c] ? G.template dxk<KIND>(sum_plus<M>(v, 4 + c, G.c)) : 0.f;
      if (C.sx[c] >= 0) {
        d = cpml(d, q.x[c], C.ax[c], C.bx[c]);
        psx[(size_t)i * G.wx + C.sx[c]] = q.x[c];
      }
      set_comp(ox, c, fadd(comp(CELL(c_vx, rr), c), fmul(fmul(G.dt, comp(CELL(c_irx, rr), c)), d)));
    }
    st4(vx + g, ox);
    float z[4][2 * M + 1];
    col9<M>(row + 4, z);
    float4 oz = CELL(c_vz, rr);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (!C.ok[c]) continue;
      float d = zin ? G.template dzk<KIND>(sum_plus<M>(z[c], M, G.c)) : 0.f;
      if (sz >= 0) {
        float psi = comp(q.z, c);
        d = cpml(d, psi, azi, bzi);
        set_comp(q.z, c, psi);
      }
      set_comp(oz, c, fadd(comp(CELL(c_vz, rr), c), fmul(fmul(G.dt, comp(CELL(c_irz, rr), c)), d)));
    }
    st4(vz + g, oz);
    if (sz >= 0) st4(psz + (size_t)sz * G.ld + j, q.z);
  }
  }
}

// Elastic: vx += (dt·irx)·(D⁺ₓσxx + D⁻_zσxz), vz += (dt·irz)·(D⁻ₓσxz + D⁺_zσzz).
template <int M, int BZ, int R, int KIND, class WS, class TM>
__global__ void __launch_bounds__(XT* BZ)
k_elastic_velocity(const DevProp* __restrict__ props, const WS ws, const __grid_constant__ TM tm) {
  constexpr int TZ = BZ * R;
  using T = TileShape<M, TZ>;
  __shared__ __align__(128) float sxx_s[T::N];
  __shared__ __align__(128) float szz_s[T::N];
  __shared__ __align__(128) float sxz_s[T::N];
  __shared__ __align__(128) float c_vx[TZ * 32];
  __shared__ __align__(128) float c_vz[TZ * 32];
  __shared__ __align__(128) float c_irx[TZ * 32];
  __shared__ __align__(128) float c_irz[TZ * 32];
  __shared__ uint64_t tma_bar;
  const StepWork& w = ws.get(blockIdx.x);
  const DevProp& P = props[w.prop];
  const Geo G(P);
  const TileLoc L = tile_loc<KIND>(w, blockIdx.x, TZ);
  float* const vx = P.f[E_VX];
  float* const vz = P.f[E_VZ];
  const float* const irx = P.coef[CE_IRX];
  const float* const irz = P.coef[CE_IRZ];
  float* const psx0 = P.psix[0]; float* const psx1 = P.psix[1];
  float* const psz0 = P.psiz[0]; float* const psz1 = P.psiz[1];
  const float* const azp = P.az; const float* const bzp = P.bz;
  // interior 32-row tiles staged in two halves (see stage_tile_halves)
  constexpr bool HALVES = KIND == TILES_INTERIOR && !TM::kOn && R == 2;
  {
    float* const hd[3] = {sxx_s, szz_s, sxz_s};
    const int hf[3] = {E_SXX, E_SZZ, E_SXZ};
    float* const cd[4] = {c_vx, c_vz, c_irx, c_irz};
    const int cf[4] = {E_VX, E_VZ, ~CE_IRX, ~CE_IRZ};
    if constexpr (HALVES) {
      stage_tile_halves<M, TZ, XT * BZ>(P, L.i0, L.j0, hd, hf, cd, cf);
    } else {
      if (!stage_tile<M, TZ, XT * BZ>(tm, w.slot, P, L.i0, L.j0, hd, hf, cd, cf, &tma_bar)) return;
    }
  }
  (void)irx;
  (void)irz;
  const int j = L.j0 + 4 * threadIdx.x;
  if (HALVES && (j >= G.nxp || !G.interior(L.i0, L.j0, TZ))) {
    cp_async_wait_all();   // never exit with copies into this block's shared memory in flight
    return;
  }
  if (j >= G.nxp) return;
  if (KIND == TILES_INTERIOR && !G.interior(L.i0, L.j0, TZ)) return;   // the host plans only interior tiles here
  if (KIND == TILES_INTERIOR || (KIND == TILES_ALL && G.interior(L.i0, L.j0, TZ))) {
    if constexpr (KIND != TILES_FRAME) {
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      if constexpr (HALVES) {
        if (r == 0) cp_async_wait_one();
        else cp_async_wait_all();
        __syncthreads();
      }
      const int rr = threadIdx.y + BZ * r;
      const int ro = (rr + M) * T::W + 4 * threadIdx.x;
      const size_t g = (size_t)(L.i0 + rr) * G.ld + j;
      float v[12], z[4][2 * M + 1];
      float4 ox, oz;
      row12(sxx_s + ro, v);
      col9<M>(sxz_s + ro + 4, z);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float a = G.dxf(sum_plus<M>(v, 4 + c, G.c));
        const float b = G.dzf(sum_minus<M>(z[c], M, G.c));
        set_comp(ox, c, fadd(comp(CELL(c_vx, rr), c), fmul(fmul(G.dt, comp(CELL(c_irx, rr), c)), fadd(a, b))));
      }
      st4(vx + g, ox);
      row12(sxz_s + ro, v);
      col9<M>(szz_s + ro + 4, z);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float a = G.dxf(sum_minus<M>(v, 4 + c, G.c));
        const float b = G.dzf(sum_plus<M>(z[c], M, G.c));
        set_comp(oz, c, fadd(comp(CELL(c_vz, rr), c), fmul(fmul(G.dt, comp(CELL(c_irz, rr), c)), fadd(a, b))));
      }
      st4(vz + g, oz);
    }
    }
    return;
  }
  if constexpr (KIND != TILES_INTERIOR) {
  const ColInfo C = col_info<M>(G, j, P.ax, P.bx);
#pragma unroll 1
  for (int r = 0; r < R; ++r) {
    const int rr = threadIdx.y + BZ * r;
    const int i = L.i0 + rr;
    if (i >= G.nzp) break;
    const int ro = (rr + M) * T::W + 4 * threadIdx.x;
    const size_t g = (size_t)i * G.ld + j;
    const bool zin = (i >= M && i < G.nzp - M);
    const int sz = G.sz(i);
    const float azi = sz >= 0 ? azp[i] : 0.f, bzi = sz >= 0 ? bzp[i] : 1.f;
    PsiCells q0 = psi_cells(C, psx0, i, G.wx, psz0, sz, G.ld, j);
    PsiCells q1 = psi_cells(C, psx1, i, G.wx, psz1, sz, G.ld, j);
    // vx: vx_dsxx (x, D⁺ of σxx) + vx_dsxz (z, D⁻ of σxz)
    float a[4], b[4];
    {
      float v[12];
      row12(sxx_s + ro, v);
#pragma unroll
      for (int c = 0; c < 4; ++c) a[c] = C.xin[c] ? G.template dxk<KIND>(sum_plus<M>(v, 4 + c, G.c)) : 0.f;
      float z[4][2 * M + 1];
      col9<M>(sxz_s + ro + 4, z);
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = zin ? G.template dzk<KIND>(sum_minus<M>(z[c], M, G.c)) : 0.f;
    }
    float4 ox = CELL(c_vx, rr);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (!C.ok[c]) continue;
      float av = a[c], bv = b[c];
      if (C.sx[c] >= 0) {
        av = cpml(av, q0.x[c], C.ax[c], C.bx[c]);
        psx0[(size_t)i * G.wx + C.sx[c]] = q0.x[c];
      }
      if (sz >= 0) {
        float psi = comp(q0.z, c);
        bv = cpml(bv, psi, azi, bzi);
        set_comp(q0.z, c, psi);
      }
      set_comp(ox, c, fadd(comp(CELL(c_vx, rr), c), fmul(fmul(G.dt, comp(CELL(c_irx, rr), c)), fadd(av, bv))));
    }
    st4(vx + g, ox);
    if (sz >= 0) st4(psz0 + (size_t)sz * G.ld + j, q0.z);
    // vz: vz_dsxz (x, D⁻ of σxz) + vz_dszz (z, D⁺ of σzz)
    {
      float v[12];
      row12(sxz_s + ro, v);
#pragma unroll
      for (int c = 0; c < 4; ++c) a[c] = C.xin[c] ? G.template dxk<KIND>(sum_minus<M>(v, 4 + c, G.c)) : 0.f;
      float z[4][2 * M + 1];
      col9<M>(szz_s + ro + 4, z);
#pragma unroll
      for (int c = 0; c < 4; ++c) b[c] = zin ? G.template dzk<KIND>(sum_plus<M>(z[c], M, G.c)) : 0.f;
    }
    float4 oz = CELL(c_vz, rr);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (!C.ok[c]) continue;
      float av = a[c], bv = b[c];
      if (C.sx[c] >= 0) {
        av = cpml(av, q1.x[c], C.ax[c], C.bx[c]);
        psx1[(size_t)i * G.wx + C.sx[c]] = q1.x[c];
      }
      if (sz >= 0) {
        float psi = comp(q1.z, c);
        bv = cpml(bv, psi, azi, bzi);
        set_comp(q1.z, c, psi);
      }
      set_comp(oz, c, fadd(comp(CELL(c_vz, rr), c), fmul(fmul(G.dt, comp(CELL(c_irz, rr), c)), fadd(av, bv))));
    }
    st4(vz + g, oz);
    if (sz >= 0) st4(psz1 + (size_t)sz * G.ld + j, q1.z);
  }
  }
}

// ---------------------------------------------------------------------------
// stress phase
// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_max_to(float v, float* dst) {
  // v ≥ 0: the float bit pattern orders like the integer.
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ float red[32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5;
  const int nw = (blockDim.x * blockDim.y + 31) >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < nw ? red[lane] : 0.f;
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) atomicMax(reinterpret_cast<int*>(dst), __float_as_int(v));
  }
}

// Resident blocks per SM the viscoacoustic interior stress kernel is
// compiled for.  Its relaxation loads are all issued before the stores,
// which uncapped takes 80 registers (6 blocks per SM); capped for 9 blocks
// (56 registers, no spills) a 4-shot tick of the 2001×801 job took 159 µs,
// against 171 µs uncapped and 170 µs with one mechanism loaded at a time.
template <bool VISCO, int KIND, int R>
constexpr int kStressMinBlocks = (VISCO && KIND == TILES_INTERIOR && R == 1) ? 9 : 1;

// Acoustic (VISCO=false): p += (dt·κ)·div.  Viscoacoustic (VISCO=true):
// ε += dt·div; r_l ← r_l·a_l + b_l·Δε; p = K_R·ε + Σ r_l.
template <int M, int BZ, int R, bool VISCO, int KIND, class WS, class TM>
__global__ void __launch_bounds__(XT* BZ, kStressMinBlocks<VISCO, KIND, R>)
k_pressure_stress(const DevProp* __restrict__ props, const WS ws, const __grid_constant__ TM tm) {
  constexpr int TZ = BZ * R;
  using T = TileShape<M, TZ>;
  __shared__ __align__(128) float svx[T::N];
  __shared__ __align__(128) float svz[T::N];
  __shared__ __align__(128) float c_a[TZ * 32];
  __shared__ __align__(128) float c_b[TZ * 32];
  __shared__ __align__(16) float e_p[TZ * 32];                   // P for the epilogue
  __shared__ uint64_t tma_bar;
  const StepWork& w = ws.get(blockIdx.x);
  const DevProp& P = props[w.prop];
  const Geo G(P);
  const TileLoc L = tile_loc<KIND>(w, blockIdx.x, TZ);
  float* const p = P.f[A_P];
  float* const eps = VISCO ? P.f[V_EPS] : nullptr;
  float* const r0 = VISCO ? P.f[V_R0] : nullptr;
  const float* const cA = VISCO ? P.coef[CV_KR] : P.coef[CA_KAPPA];   // κ or K_R
  const float* const b0 = VISCO ? P.coef[CV_B0] : nullptr;
  const size_t fstride = (size_t)(P.f[1] - P.f[0]);                   // field / coefficient pitch
  const int nL = VISCO ? P.L : 0;
  const uint8_t* const qidx = VISCO ? P.qidx : nullptr;
  const float* const relax_a = VISCO ? P.relax_a : nullptr;
  float* const psx = P.psix[1];
  float* const psz = P.psiz[1];
  const float* const azp = P.az; const float* const bzp = P.bz;
  constexpr bool HALVES = KIND == TILES_INTERIOR && !TM::kOn && R == 2;
  {
    float* const hd[2] = {svx, svz};
    const int hf[2] = {A_VX, A_VZ};
    float* const cd[2] = {c_a, c_b};
    const int cf[2] = {VISCO ? V_EPS : A_P, VISCO ? ~CV_KR : ~CA_KAPPA};
    if constexpr (HALVES) {
      stage_tile_halves<M, TZ, XT * BZ>(P, L.i0, L.j0, hd, hf, cd, cf);
      prefetch_image_tile<TZ, XT * BZ>(w.epi, G, L.i0, L.j0);
    } else {
      if (!stage_tile<M, TZ, XT * BZ>(tm, w.slot, P, L.i0, L.j0, hd, hf, cd, cf, &tma_bar)) return;
    }
  }
  (void)cA;
  const int j = L.j0 + 4 * threadIdx.x;
  const bool jok = j < G.nxp;
  float amp, amp_eps;
  source_amps(w, P, amp, amp_eps);
  const size_t npix = (size_t)G.nz * G.nx;
  float peak = 0.f;
  const bool valid = KIND != TILES_INTERIOR || G.interior(L.i0, L.j0, TZ);   // the host plans only interior tiles there
  const bool inner = KIND == TILES_INTERIOR || (KIND == TILES_ALL && G.interior(L.i0, L.j0, TZ));
  if (HALVES && !(jok && valid)) {
    cp_async_wait_all();   // never exit with copies into this block's shared memory in flight
    return;
  }
  if (jok && inner && valid) {
    if constexpr (KIND != TILES_FRAME) {
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      if constexpr (HALVES) {
        if (r == 0) cp_async_wait_one();
        else cp_async_wait_all();
        __syncthreads();
      }
      const int rr = threadIdx.y + BZ * r;
      const int i = L.i0 + rr;
      const int ro = (rr + M) * T::W + 4 * threadIdx.x;
      const size_t g = (size_t)i * G.ld + j;
      float v[12], z[4][2 * M + 1];
      row12(svx + ro, v);
      col9<M>(svz + ro + 4, z);
      float4 out, epsv;
      float inc[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float div = fadd(G.dxf(sum_minus<M>(v, 4 + c, G.c)), G.dzf(sum_minus<M>(z[c], M, G.c)));
        if constexpr (!VISCO) {
          set_comp(out, c, fadd(comp(CELL(c_a, rr), c), fmul(fmul(G.dt, comp(CELL(c_b, rr), c)), div)));
        } else {
          inc[c] = fmul(G.dt, div);
        }
      }
      if constexpr (VISCO) {
        const bool keep[4] = {false, false, false, false};
        float tot[4];
        relax4(r0, b0, fstride, qidx, relax_a, nL, g, inc, keep, tot);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float e = fadd(comp(CELL(c_a, rr), c), inc[c]);
          const float pv = fadd(fmul(comp(CELL(c_b, rr), c), e), tot[c]);
          set_comp(epsv, c, e);
          set_comp(out, c, pv);
          peak = fmaxf(peak, fabsf(pv));
        }
      }
      st4(p + g, out);
      if (nonfinite4(out)) atomicOr(P.status, STATUS_NONFINITE);
      if constexpr (VISCO) st4(eps + g, epsv);
      if (w.epi.kind != EPI_NONE) st4(e_p + rr * 32 + 4 * threadIdx.x, out);
    }
    }
  } else if (jok && !inner) {
    if constexpr (KIND != TILES_INTERIOR) {
    const ColInfo C = col_info<M>(G, j, P.ax, P.bx);
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      const int rr = threadIdx.y + BZ * r;
      const int i = L.i0 + rr;
      if (i >= G.nzp) break;
      const int ro = (rr + M) * T::W + 4 * threadIdx.x;
      const size_t g = (size_t)i * G.ld + j;
      const bool zin = (i >= M && i < G.nzp - M);
      const int sz = G.sz(i);
      const float azi = sz >= 0 ? azp[i] : 0.f, bzi = sz >= 0 ? bzp[i] : 1.f;
      float dx[4], dz[4];
      {
        float v[12];
        row12(svx + ro, v);
#pragma unroll
        for (int c = 0; c < 4; ++c) dx[c] = C.xin[c] ? G.template dxk<KIND>(sum_minus<M>(v, 4 + c, G.c)) : 0.f;
        float z[4][2 * M + 1];
        col9<M>(svz + ro + 4, z);
#pragma unroll
        for (int c = 0; c < 4; ++c) dz[c] = zin ? G.template dzk<KIND>(sum_minus<M>(z[c], M, G.c)) : 0.f;
      }
      float4 out = CELL(c_a, rr);
      float4 epsv = out;
      PsiCells q = psi_cells(C, psx, i, G.wx, psz, sz, G.ld, j);
      float inc[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        inc[c] = 0.f;
        if (!C.ok[c]) continue;
        const int jc = j + c;
        float ddx = dx[c], ddz = dz[c];
        if (C.sx[c] >= 0) {
          ddx = cpml(ddx, q.x[c], C.ax[c], C.bx[c]);
          psx[(size_t)i * G.wx + C.sx[c]] = q.x[c];
        }
        if (sz >= 0) {
          float psi = comp(q.z, c);
          ddz = cpml(ddz, psi, azi, bzi);
          set_comp(q.z, c, psi);
        }
        const float div = fadd(ddx, ddz);
        if constexpr (!VISCO) {
          const bool src = (i == G.src_iz && jc == G.src_ix && amp != 0.f);
          float pv = fadd(comp(CELL(c_a, rr), c), fmul(fmul(G.dt, comp(CELL(c_b, rr), c)), div));
          if (src) pv = fadd(pv, amp);
          if (G.free_surface && i == G.pad) pv = 0.f;
          set_comp(out, c, pv);
        } else {
          inc[c] = fmul(G.dt, div);
        }
      }
      if (sz >= 0) st4(psz + (size_t)sz * G.ld + j, q.z);
      if constexpr (VISCO) {
        const bool keep[4] = {!C.ok[0], !C.ok[1], !C.ok[2], !C.ok[3]};
        float tot[4];
        relax4(r0, b0, fstride, qidx, relax_a, nL, g, inc, keep, tot);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (!C.ok[c]) continue;
          float e = fadd(comp(CELL(c_a, rr), c), inc[c]);
          float pv = fadd(fmul(comp(CELL(c_b, rr), c), e), tot[c]);
          if (i == G.src_iz && j + c == G.src_ix && amp != 0.f) {
            e = fadd(e, amp_eps);
            pv = fadd(pv, amp);
          }
          set_comp(epsv, c, e);
          set_comp(out, c, pv);
          peak = fmaxf(peak, fabsf(pv));
        }
      }
      st4(p + g, out);
      if (nonfinite4(out)) atomicOr(P.status, STATUS_NONFINITE);
      if constexpr (VISCO) st4(eps + g, epsv);
      if (w.epi.kind != EPI_NONE) st4(e_p + rr * 32 + 4 * threadIdx.x, out);
    }
    }
  }
  if (valid && w.epi.kind != EPI_NONE) {
    __syncthreads();
    epilogue_tile<TZ, XT * BZ>(w.epi, G, L.i0, L.j0, e_p, nullptr, npix);
  }
  if constexpr (VISCO) {
    if (w.flags & STEP_PEAK) block_max_to(peak, P.peak);
  }
}

// Elastic stress phase:
//   σxx += dt·(λ2μ·εxx + λ·εzz), σzz += dt·(λ·εxx + λ2μ·εzz),
//   σxz += (dt·μxz)·(D⁺_z vx + D⁺ₓ vz); source; free surface σzz = σxz = 0;
// then the epilogue with P/S from the stresses (stress separation) or from
// the raw velocity divergence/curl (divcurl, propagation.py:953-976).
template <int M, int BZ, int R, int KIND, class WS, class TM>
__global__ void __launch_bounds__(XT* BZ)
k_elastic_stress(const DevProp* __restrict__ props, const WS ws, const __grid_constant__ TM tm) {
  constexpr int TZ = BZ * R;
  using T = TileShape<M, TZ>;
  __shared__ __align__(128) float svx[T::N];
  __shared__ __align__(128) float svz[T::N];
  __shared__ __align__(128) float c_xx[TZ * 32];
  __shared__ __align__(128) float c_zz[TZ * 32];
  __shared__ __align__(128) float c_xz[TZ * 32];
  __shared__ __align__(128) float c_lam[TZ * 32];
  __shared__ __align__(128) float c_l2m[TZ * 32];
  __shared__ __align__(128) float c_mu[TZ * 32];
  __shared__ __align__(16) float e_p[TZ * 32], e_s[TZ * 32];   // P and S for the epilogue
  __shared__ uint64_t tma_bar;
  const StepWork& w = ws.get(blockIdx.x);
  const DevProp& P = props[w.prop];
  const Geo G(P);
  const TileLoc L = tile_loc<KIND>(w, blockIdx.x, TZ);
  float* const sxx = P.f[E_SXX];
  float* const szz = P.f[E_SZZ];
  float* const sxz = P.f[E_SXZ];
  const float* const clam = P.coef[CE_LAM];
  const float* const cl2m = P.coef[CE_L2M];
  const float* const cmu = P.coef[CE_MUXZ];
  float* const psx2 = P.psix[2]; float* const psx3 = P.psix[3];
  float* const psz2 = P.psiz[2]; float* const psz3 = P.psiz[3];
  const float* const azp = P.az; const float* const bzp = P.bz;
  const int mech = P.mech;
  constexpr bool HALVES = KIND == TILES_INTERIOR && !TM::kOn && R == 2;
  {
    float* const hd[2] = {svx, svz};
    const int hf[2] = {E_VX, E_VZ};
    float* const cd[6] = {c_xx, c_zz, c_xz, c_lam, c_l2m, c_mu};
    const int cf[6] = {E_SXX, E_SZZ, E_SXZ, ~CE_LAM, ~CE_L2M, ~CE_MUXZ};
    if constexpr (HALVES) {
      stage_tile_halves<M, TZ, XT * BZ>(P, L.i0, L.j0, hd, hf, cd, cf);
      prefetch_image_tile<TZ, XT * BZ>(w.epi, G, L.i0, L.j0);
    } else {
      if (!stage_tile<M, TZ, XT * BZ>(tm, w.slot, P, L.i0, L.j0, hd, hf, cd, cf, &tma_bar)) return;
    }
  }
  (void)clam;
  (void)cl2m;
  (void)cmu;
  const int j = L.j0 + 4 * threadIdx.x;
  float amp, amp_eps;
  source_amps(w, P, amp, amp_eps);
  const size_t npix = (size_t)G.nz * G.nx;
  const Epilogue& E = w.epi;
  const bool epi = E.kind != EPI_NONE;
  const bool want_curl = epi && E.sep == 1 && E.need_s;
  const bool valid = KIND != TILES_INTERIOR || G.interior(L.i0, L.j0, TZ);   // the host plans only interior tiles there
  const bool inner = KIND == TILES_INTERIOR || (KIND == TILES_ALL && G.interior(L.i0, L.j0, TZ));
  if (HALVES && !(j < G.nxp && valid)) {
    cp_async_wait_all();   // never exit with copies into this block's shared memory in flight
    return;
  }
  if (j < G.nxp && inner && valid) {
    if constexpr (KIND != TILES_FRAME) {
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      if constexpr (HALVES) {
        if (r == 0) cp_async_wait_one();
        else cp_async_wait_all();
        __syncthreads();
      }
      const int rr = threadIdx.y + BZ * r;
      const int i = L.i0 + rr;
      const int ro = (rr + M) * T::W + 4 * threadIdx.x;
      const size_t g = (size_t)i * G.ld + j;
      float v[12], z[4][2 * M + 1];
      float exx[4], ezz[4], f1[4], f2[4], ca[4], cb[4];
      row12(svx + ro, v);
#pragma unroll
      for (int c = 0; c < 4; ++c) exx[c] = G.dxf(sum_minus<M>(v, 4 + c, G.c));
      row12(svz + ro, v);
#pragma unroll
      for (int c = 0; c < 4; ++c) f2[c] = G.dxf(sum_plus<M>(v, 4 + c, G.c));
      if (want_curl) {
#pragma unroll
        for (int c = 0; c < 4; ++c) cb[c] = G.dxf(sum_minus<M>(v, 4 + c, G.c));
      }
      col9<M>(svx + ro + 4, z);
#pragma unroll
      for (int c = 0; c < 4; ++c) f1[c] = G.dzf(sum_plus<M>(z[c], M, G.c));
      if (want_curl) {
#pragma unroll
        for (int c = 0; c < 4; ++c) ca[c] = G.dzf(sum_minus<M>(z[c], M, G.c));
      }
      col9<M>(svz + ro + 4, z);
#pragma unroll
      for (int c = 0; c < 4; ++c) ezz[c] = G.dzf(sum_minus<M>(z[c], M, G.c));
      float4 oxx, ozz, oxz;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float lam = comp(CELL(c_lam, rr), c), l2m = comp(CELL(c_l2m, rr), c);
        set_comp(oxx, c, fadd(comp(CELL(c_xx, rr), c), fmul(G.dt, fadd(fmul(l2m, exx[c]), fmul(lam, ezz[c])))));
        set_comp(ozz, c, fadd(comp(CELL(c_zz, rr), c), fmul(G.dt, fadd(fmul(lam, exx[c]), fmul(l2m, ezz[c])))));
        set_comp(oxz, c, fadd(comp(CELL(c_xz, rr), c), fmul(fmul(G.dt, comp(CELL(c_mu, rr), c)), fadd(f1[c], f2[c]))));
      }
      st4(sxx + g, oxx);
      st4(szz + g, ozz);
      st4(sxz + g, oxz);
      if (nonfinite4(oxx) || nonfinite4(ozz) || nonfinite4(oxz)) atomicOr(P.status, STATUS_NONFINITE);
      if (epi) {
        float4 pv4, sv4;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (E.sep == 0) {
            set_comp(pv4, c, fmul(0.5f, fadd(comp(oxx, c), comp(ozz, c))));
            set_comp(sv4, c, comp(oxz, c));
          } else {
            set_comp(pv4, c, fadd(exx[c], ezz[c]));
            set_comp(sv4, c, want_curl ? fsub(ca[c], cb[c]) : 0.f);
          }
        }
        st4(e_p + rr * 32 + 4 * threadIdx.x, pv4);
        st4(e_s + rr * 32 + 4 * threadIdx.x, sv4);
      }
    }
    }
  } else if (j < G.nxp && !inner) {
    if constexpr (KIND != TILES_INTERIOR) {
    const ColInfo C = col_info<M>(G, j, P.ax, P.bx);
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      const int rr = threadIdx.y + BZ * r;
      const int i = L.i0 + rr;
      if (i >= G.nzp) break;
      const int ro = (rr + M) * T::W + 4 * threadIdx.x;
      const size_t g = (size_t)i * G.ld + j;
      const bool zin = (i >= M && i < G.nzp - M);
      const int sz = G.sz(i);
      const float azi = sz >= 0 ? azp[i] : 0.f, bzi = sz >= 0 ? bzp[i] : 1.f;
      float exx[4], ezz[4], f1[4], f2[4], curl_a[4], curl_b[4];
      {
        float v[12];
        row12(svx + ro, v);        // vx along x: D⁻ (εxx)
#pragma unroll
        for (int c = 0; c < 4; ++c) exx[c] = C.xin[c] ? G.template dxk<KIND>(sum_minus<M>(v, 4 + c, G.c)) : 0.f;
        row12(svz + ro, v);        // vz along x: D⁺ (σxz) and D⁻ (curl)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          f2[c] = C.xin[c] ? G.template dxk<KIND>(sum_plus<M>(v, 4 + c, G.c)) : 0.f;
          curl_b[c] = want_curl ? G.template dxk<KIND>(sum_minus<M>(v, 4 + c, G.c)) : 0.f;
        }
        float z[4][2 * M + 1];
        col9<M>(svx + ro + 4, z);  // vx along z: D⁺ (σxz) and D⁻ (curl)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          f1[c] = zin ? G.template dzk<KIND>(sum_plus<M>(z[c], M, G.c)) : 0.f;
          curl_a[c] = want_curl ? G.template dzk<KIND>(sum_minus<M>(z[c], M, G.c)) : 0.f;
        }
        col9<M>(svz + ro + 4, z);  // vz along z: D⁻ (εzz)
#pragma unroll
        for (int c = 0; c < 4; ++c) ezz[c] = zin ? G.template dzk<KIND>(sum_minus<M>(z[c], M, G.c)) : 0.f;
      }
      float4 oxx = CELL(c_xx, rr), ozz = CELL(c_zz, rr), oxz = CELL(c_xz, rr);
      float4 pv4 = make_float4(0.f, 0.f, 0.f, 0.f), sv4 = pv4;
      PsiCells q2 = psi_cells(C, psx2, i, G.wx, psz2, sz, G.ld, j);
      PsiCells q3 = psi_cells(C, psx3, i, G.wx, psz3, sz, G.ld, j);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (!C.ok[c]) continue;
        const int jc = j + c;
        const float exx_raw = exx[c], ezz_raw = ezz[c];
        float ex = exx_raw, ez = ezz_raw, g1 = f1[c], g2 = f2[c];
        if (C.sx[c] >= 0) {
          const size_t xo = (size_t)i * G.wx + C.sx[c];
          ex = cpml(ex, q2.x[c], C.ax[c], C.bx[c]);
          psx2[xo] = q2.x[c];
          g2 = cpml(g2, q3.x[c], C.ax[c], C.bx[c]);
          psx3[xo] = q3.x[c];
        }
        if (sz >= 0) {
          float psi = comp(q2.z, c);
          ez = cpml(ez, psi, azi, bzi);
          set_comp(q2.z, c, psi);
          psi = comp(q3.z, c);
          g1 = cpml(g1, psi, azi, bzi);
          set_comp(q3.z, c, psi);
        }
        const float lam = comp(CELL(c_lam, rr), c), l2m = comp(CELL(c_l2m, rr), c);
        float vxx = fadd(comp(CELL(c_xx, rr), c), fmul(G.dt, fadd(fmul(l2m, ex), fmul(lam, ez))));
        float vzz = fadd(comp(CELL(c_zz, rr), c), fmul(G.dt, fadd(fmul(lam, ex), fmul(l2m, ez))));
        float vxz = fadd(comp(CELL(c_xz, rr), c), fmul(fmul(G.dt, comp(CELL(c_mu, rr), c)), fadd(g1, g2)));
        if (i == G.src_iz && jc == G.src_ix && amp != 0.f) {
          if (mech == MECH_SHEAR) {
            vxz = fadd(vxz, amp);
          } else if (mech == MECH_EXPLOSIVE) {
            vxx = fadd(vxx, amp);
            vzz = fadd(vzz, amp);
          }
          // force_z adds to vz after this launch (other blocks still read vz here).
        }
        if (G.free_surface && i == G.pad) {
          vzz = 0.f;
          vxz = 0.f;
        }
        set_comp(oxx, c, vxx);
        set_comp(ozz, c, vzz);
        set_comp(oxz, c, vxz);
        if (E.sep == 0) {
          set_comp(pv4, c, fmul(0.5f, fadd(vxx, vzz)));
          set_comp(sv4, c, vxz);
        } else {
          set_comp(pv4, c, fadd(exx_raw, ezz_raw));
          set_comp(sv4, c, E.need_s ? fsub(curl_a[c], curl_b[c]) : 0.f);
        }
      }
      st4(sxx + g, oxx);
      st4(szz + g, ozz);
      st4(sxz + g, oxz);
      if (nonfinite4(oxx) || nonfinite4(ozz) || nonfinite4(oxz)) atomicOr(P.status, STATUS_NONFINITE);
      if (sz >= 0) {
        st4(psz2 + (size_t)sz * G.ld + j, q2.z);
        st4(psz3 + (size_t)sz * G.ld + j, q3.z);
      }
      if (epi) {
        st4(e_p + rr * 32 + 4 * threadIdx.x, pv4);
        st4(e_s + rr * 32 + 4 * threadIdx.x, sv4);
      }
    }
    }
  }
  if (epi && valid) {
    __syncthreads();
    epilogue_tile<TZ, XT * BZ>(E, G, L.i0, L.j0, e_p, e_s, npix);
  }
}

#undef CELL

// ---------------------------------------------------------------------------
// Elastic velocity phase of the interior rectangle, marching down column
// strips.  A block (8 × 16 threads) owns 32 columns of the rectangle over a
// segment of 16-row chunks (the rectangle's rows in order, about MARCH_SEG
// chunks per block) and walks it top to bottom: while one chunk computes, the
// next chunk's rows are in flight (cp.async, two stages).  σxz and σzz, read
// with a z-halo, live in a 64-row ring, so every row is copied in once per
// segment instead of once per tile with its halo; σxx (x-halo only) and the
// per-cell operands are double-buffered per chunk.  The arithmetic is the
// interior tile kernel's, expression for expression.  The source node's
// 32-row tile (the hole) is left to the frame launch: its two chunks are
// skipped.
// ---------------------------------------------------------------------------
constexpr int MARCH_CH = 16;     // rows per chunk: one per thread row
constexpr int MARCH_RING = 64;   // ring rows (power of two ≥ 2·MARCH_CH + 2M + MARCH_CH)

struct MarchLoc {
  int j0, a0, n, hole_c;   // strip column, first row, chunks, first hole chunk (relative; out of range: none)
};

// Blocks of a work: (tj1 − tj0) strips × nseg segments of at most SEG
// chunks; the host counts them the same way (march_blocks).
template <int SEG>
__device__ __forceinline__ MarchLoc march_loc(const StepWork& w, int block) {
  const int ncols = w.tj1 - w.tj0;
  const int chunks = 2 * (w.ti1 - w.ti0);
  const int nseg = (chunks + SEG - 1) / SEG;
  const int len = (chunks + nseg - 1) / nseg;
  const int k = block - w.tile0;
  const int seg = k / ncols, col = k - seg * ncols;
  const int c0 = seg * len;
  MarchLoc L;
  L.j0 = (w.tj0 + col) * TILE_X;
  L.a0 = w.ti0 * 32 + c0 * MARCH_CH;
  L.n = min(len, chunks - c0);
  L.hole_c = (w.hole_i >= 0 && w.tj0 + col == w.hole_j) ? 2 * (w.hole_i - w.ti0) - c0 : -1000;
  return L;
}

// Rows [r_lo, r_hi) of one field with a 4-column halo each side into a ring
// of 40-float rows (slot = row mod MARCH_RING).
template <int NT>
__device__ __forceinline__ void march_ring_rows(float* s, const float* __restrict__ g, int nzp, int ld, int r_lo,
                                                int r_hi, int j0) {
  const int tid = threadIdx.y * XT + threadIdx.x;
  const int n = (r_hi - r_lo) * 10;
  for (int idx = tid; idx < n; idx += NT) {
    const int q = idx / 10;
    const int r = r_lo + q, ch = idx - q * 10;
    const int gj = j0 - 4 + 4 * ch;
    const bool ok = r >= 0 && r < nzp && gj >= 0 && gj < ld;
    cp_async16(s + (r & (MARCH_RING - 1)) * 40 + 4 * ch, ok ? g + (size_t)r * ld + gj : g, ok);
  }
}

// One chunk's σxx rows (x-halo, 16 × 40) and per-cell operands (16 × 32 each).
template <int NT>
__device__ __forceinline__ void march_chunk_rows(float* sx, float* const (&cd)[4], const float* __restrict__ gx,
                                                 const float* const (&cg)[4], int nzp, int ld, int a, int j0) {
  const int tid = threadIdx.y * XT + threadIdx.x;
  for (int idx = tid; idx < MARCH_CH * 10; idx += NT) {
    const int q = idx / 10;
    const int r = a + q, ch = idx - q * 10;
    const int gj = j0 - 4 + 4 * ch;
    const bool ok = r < nzp && gj >= 0 && gj < ld;
    cp_async16(sx + q * 40 + 4 * ch, ok ? gx + (size_t)r * ld + gj : gx, ok);
  }
  for (int idx = tid; idx < MARCH_CH * 8; idx += NT) {
    const int q = idx >> 3, ch = idx & 7;
    const int r = a + q;
    const bool ok = r < nzp;
    const size_t off = ok ? (size_t)r * ld + j0 + 4 * ch : 0;
#pragma unroll
    for (int f = 0; f < 4; ++f) cp_async16(cd[f] + q * 32 + 4 * ch, cg[f] + off, ok);
  }
}

template <int M, int SEG, class WS>
__global__ void __launch_bounds__(XT* MARCH_CH)
k_elastic_velocity_march(const DevProp* __restrict__ props, const WS ws) {
  static_assert(M == 4, "the march covers the 8th-order stencil");
  static_assert(MARCH_RING >= 2 * MARCH_CH + 2 * M + MARCH_CH, "ring too short for two chunks in flight");
  __shared__ __align__(128) float ring_xz[MARCH_RING * 40];
  __shared__ __align__(128) float ring_zz[MARCH_RING * 40];
  __shared__ __align__(128) float sxx_b[2][MARCH_CH * 40];
  __shared__ __align__(128) float cell_b[2][4][MARCH_CH * 32];
  constexpr int NT = XT * MARCH_CH;
  const StepWork& w = ws.get(blockIdx.x);
  const DevProp& P = props[w.prop];
  const Geo G(P);
  const MarchLoc L = march_loc<SEG>(w, blockIdx.x);
  if (L.n <= 0) return;
  float* const vx = P.f[E_VX];
  float* const vz = P.f[E_VZ];
  const float* const gxx = P.f[E_SXX];
  const float* const gzz = P.f[E_SZZ];
  const float* const gxz = P.f[E_SXZ];
  const float* const cg[4] = {P.f[E_VX], P.f[E_VZ], P.coef[CE_IRX], P.coef[CE_IRZ]};
  const int j0 = L.j0;
  // chunk 0: its ring rows with the top halo, its σxx and cell rows
  march_ring_rows<NT>(ring_xz, gxz, G.nzp, G.ld, L.a0 - M, L.a0 + MARCH_CH + M, j0);
  march_ring_rows<NT>(ring_zz, gzz, G.nzp, G.ld, L.a0 - M, L.a0 + MARCH_CH + M, j0);
  {
    float* const cd[4] = {cell_b[0][0], cell_b[0][1], cell_b[0][2], cell_b[0][3]};
    march_chunk_rows<NT>(sxx_b[0], cd, gxx, cg, G.nzp, G.ld, L.a0, j0);
  }
  cp_async_commit();
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = j0 + 4 * tx;
#pragma unroll 1
  for (int c = 0; c < L.n; ++c) {
    const int a = L.a0 + c * MARCH_CH;
    const int b = c & 1;
    if (c + 1 < L.n) {   // the next chunk: 16 new ring rows, its σxx and cell rows
      march_ring_rows<NT>(ring_xz, gxz, G.nzp, G.ld, a + MARCH_CH + M, a + 2 * MARCH_CH + M, j0);
      march_ring_rows<NT>(ring_zz, gzz, G.nzp, G.ld, a + MARCH_CH + M, a + 2 * MARCH_CH + M, j0);
      float* const cd[4] = {cell_b[b ^ 1][0], cell_b[b ^ 1][1], cell_b[b ^ 1][2], cell_b[b ^ 1][3]};
      march_chunk_rows<NT>(sxx_b[b ^ 1], cd, gxx, cg, G.nzp, G.ld, a + MARCH_CH, j0);
    }
    cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
    if (c != L.hole_c && c != L.hole_c + 1) {
      const int i = a + ty;
      const size_t g = (size_t)i * G.ld + j;
      const float4 cvx = ld4(cell_b[b][0] + ty * 32 + 4 * tx), cvz = ld4(cell_b[b][1] + ty * 32 + 4 * tx);
      const float4 cirx = ld4(cell_b[b][2] + ty * 32 + 4 * tx), cirz = ld4(cell_b[b][3] + ty * 32 + 4 * tx);
      float v[12], z[4][2 * M + 1];
      float4 ox, oz;
      row12(sxx_b[b] + ty * 40 + 4 * tx, v);
#pragma unroll
      for (int k = 0; k <= 2 * M; ++k) {
        const float4 q = ld4(ring_xz + ((i + k - M) & (MARCH_RING - 1)) * 40 + 4 + 4 * tx);
        z[0][k] = q.x; z[1][k] = q.y; z[2][k] = q.z; z[3][k] = q.w;
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const float da = G.dxf(sum_plus<M>(v, 4 + cc, G.c));
        const float db = G.dzf(sum_minus<M>(z[cc], M, G.c));
        set_comp(ox, cc, fadd(comp(cvx, cc), fmul(fmul(G.dt, comp(cirx, cc)), fadd(da, db))));
      }
      st4(vx + g, ox);
      row12(ring_xz + (i & (MARCH_RING - 1)) * 40 + 4 * tx, v);
#pragma unroll
      for (int k = 0; k <= 2 * M; ++k) {
        const float4 q = ld4(ring_zz + ((i + k - M) & (MARCH_RING - 1)) * 40 + 4 + 4 * tx);
        z[0][k] = q.x; z[1][k] = q.y; z[2][k] = q.z; z[3][k] = q.w;
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const float da = G.dxf(sum_minus<M>(v, 4 + cc, G.c));
        const float db = G.dzf(sum_plus<M>(z[cc], M, G.c));
        set_comp(oz, cc, fadd(comp(cvz, cc), fmul(fmul(G.dt, comp(cirz, cc)), fadd(da, db))));
      }
      st4(vz + g, oz);
    }
    __syncthreads();   // the next iteration refills this chunk's buffers
  }
  cp_async_wait_all();
}

// Six per-cell operand rows of one chunk (16 × 32 each).
template <int NT>
__device__ __forceinline__ void march_cells6(float (&cd)[6][MARCH_CH * 32], const float* const (&cg)[6], int nzp,
                                             int ld, int a, int j0) {
  const int tid = threadIdx.y * XT + threadIdx.x;
#pragma unroll
  for (int it = 0; it < MARCH_CH * 8 / NT; ++it) {
    const int idx = tid + it * NT;
    const int q = idx >> 3, ch = idx & 7;
    const int r = a + q;
    const bool ok = r < nzp;
    const size_t off = ok ? (size_t)r * ld + j0 + 4 * ch : 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) cp_async16(cd[f] + q * 32 + 4 * ch, cg[f] + off, ok);
  }
}

// Elastic stress phase of the interior rectangle, marching like the velocity
// kernel above: vx and vz (read with both halos) in 64-row rings, the six
// per-cell operands double-buffered per chunk, and the fused epilogue run per
// 16-row chunk (it works cell by cell, so chunks give the tile's result).  P
// and S for the epilogue reuse the chunk's σxx / σzz operand buffers: each
// thread has read its own old values before it writes there.  Interior
// rectangles hold neither the source node nor the free-surface row.
template <int M, int SEG, class WS>
__global__ void __launch_bounds__(XT* MARCH_CH, 5)
k_elastic_stress_march(const DevProp* __restrict__ props, const WS ws) {
  static_assert(M == 4, "the march covers the 8th-order stencil");
  __shared__ __align__(128) float ring_vx[MARCH_RING * 40];
  __shared__ __align__(128) float ring_vz[MARCH_RING * 40];
  __shared__ __align__(128) float cell_b[2][6][MARCH_CH * 32];
  constexpr int NT = XT * MARCH_CH;
  const StepWork& w = ws.get(blockIdx.x);
  const DevProp& P = props[w.prop];
  const Geo G(P);
  const MarchLoc L = march_loc<SEG>(w, blockIdx.x);
  if (L.n <= 0) return;
  float* const sxx = P.f[E_SXX];
  float* const szz = P.f[E_SZZ];
  float* const sxz = P.f[E_SXZ];
  const float* const gvx = P.f[E_VX];
  const float* const gvz = P.f[E_VZ];
  const float* const cg[6] = {P.f[E_SXX], P.f[E_SZZ], P.f[E_SXZ], P.coef[CE_LAM], P.coef[CE_L2M], P.coef[CE_MUXZ]};
  const int j0 = L.j0;
  const size_t npix = (size_t)G.nz * G.nx;
  const Epilogue& E = w.epi;
  const bool epi = E.kind != EPI_NONE;
  const bool want_curl = epi && E.sep == 1 && E.need_s;
  march_ring_rows<NT>(ring_vx, gvx, G.nzp, G.ld, L.a0 - M, L.a0 + MARCH_CH + M, j0);
  march_ring_rows<NT>(ring_vz, gvz, G.nzp, G.ld, L.a0 - M, L.a0 + MARCH_CH + M, j0);
  march_cells6<NT>(cell_b[0], cg, G.nzp, G.ld, L.a0, j0);
  cp_async_commit();
  prefetch_image_tile<MARCH_CH, NT>(E, G, L.a0, j0);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int j = j0 + 4 * tx;
#pragma unroll 1
  for (int c = 0; c < L.n; ++c) {
    const int a = L.a0 + c * MARCH_CH;
    const int b = c & 1;
    if (c + 1 < L.n) {
      march_ring_rows<NT>(ring_vx, gvx, G.nzp, G.ld, a + MARCH_CH + M, a + 2 * MARCH_CH + M, j0);
      march_ring_rows<NT>(ring_vz, gvz, G.nzp, G.ld, a + MARCH_CH + M, a + 2 * MARCH_CH + M, j0);
      march_cells6<NT>(cell_b[b ^ 1], cg, G.nzp, G.ld, a + MARCH_CH, j0);
    }
    cp_async_commit();
    if (c + 1 < L.n) prefetch_image_tile<MARCH_CH, NT>(E, G, a + MARCH_CH, j0);
    cp_async_wait_one();
    __syncthreads();
    const bool run = c != L.hole_c && c != L.hole_c + 1;
    if (run) {
      const int i = a + ty;
      const size_t g = (size_t)i * G.ld + j;
      const int co = ty * 32 + 4 * tx;
      const float4 cxx = ld4(cell_b[b][0] + co), czz = ld4(cell_b[b][1] + co), cxz = ld4(cell_b[b][2] + co);
      const float4 clam = ld4(cell_b[b][3] + co), cl2m = ld4(cell_b[b][4] + co), cmu = ld4(cell_b[b][5] + co);
      float v[12], z[4][2 * M + 1];
      float exx[4], ezz[4], f1[4], f2[4], ca[4], cb[4];
      row12(ring_vx + (i & (MARCH_RING - 1)) * 40 + 4 * tx, v);
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) exx[cc] = G.dxf(sum_minus<M>(v, 4 + cc, G.c));
      row12(ring_vz + (i & (MARCH_RING - 1)) * 40 + 4 * tx, v);
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) f2[cc] = G.dxf(sum_plus<M>(v, 4 + cc, G.c));
      if (want_curl) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) cb[cc] = G.dxf(sum_minus<M>(v, 4 + cc, G.c));
      }
#pragma unroll
      for (int k = 0; k <= 2 * M; ++k) {
        const float4 q = ld4(ring_vx + ((i + k - M) & (MARCH_RING - 1)) * 40 + 4 + 4 * tx);
        z[0][k] = q.x; z[1][k] = q.y; z[2][k] = q.z; z[3][k] = q.w;
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) f1[cc] = G.dzf(sum_plus<M>(z[cc], M, G.c));
      if (want_curl) {
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) ca[cc] = G.dzf(sum_minus<M>(z[cc], M, G.c));
      }
#pragma unroll
      for (int k = 0; k <= 2 * M; ++k) {
        const float4 q = ld4(ring_vz + ((i + k - M) & (MARCH_RING - 1)) * 40 + 4 + 4 * tx);
        z[0][k] = q.x; z[1][k] = q.y; z[2][k] = q.z; z[3][k] = q.w;
      }
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) ezz[cc] = G.dzf(sum_minus<M>(z[cc], M, G.c));
      float4 oxx, ozz, oxz;
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const float lam = comp(clam, cc), l2m = comp(cl2m, cc);
        set_comp(oxx, cc, fadd(comp(cxx, cc), fmul(G.dt, fadd(fmul(l2m, exx[cc]), fmul(lam, ezz[cc])))));
        set_comp(ozz, cc, fadd(comp(czz, cc), fmul(G.dt, fadd(fmul(lam, exx[cc]), fmul(l2m, ezz[cc])))));
        set_comp(oxz, cc, fadd(comp(cxz, cc), fmul(fmul(G.dt, comp(cmu, cc)), fadd(f1[cc], f2[cc]))));
      }
      st4(sxx + g, oxx);
      st4(szz + g, ozz);
      st4(sxz + g, oxz);
      if (nonfinite4(oxx) || nonfinite4(ozz) || nonfinite4(oxz)) atomicOr(P.status, STATUS_NONFINITE);
      if (epi) {
        float4 pv4, sv4;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          if (E.sep == 0) {
            set_comp(pv4, cc, fmul(0.5f, fadd(comp(oxx, cc), comp(ozz, cc))));
            set_comp(sv4, cc, comp(oxz, cc));
          } else {
            set_comp(pv4, cc, fadd(exx[cc], ezz[cc]));
            set_comp(sv4, cc, want_curl ? fsub(ca[cc], cb[cc]) : 0.f);
          }
        }
        st4(cell_b[b][0] + co, pv4);   // P over this thread's old σxx slot
        st4(cell_b[b][1] + co, sv4);   // S over its old σzz slot
      }
    }
    if (epi && run) {
      __syncthreads();
      epilogue_tile<MARCH_CH, NT>(E, G, a, j0, cell_b[b][0], cell_b[b][1], npix);
    }
    __syncthreads();   // the next iteration refills this chunk's buffers
  }
  cp_async_wait_all();
}

}  // namespace ertm
