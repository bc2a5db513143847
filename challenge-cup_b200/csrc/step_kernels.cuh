// Staggered-grid velocity / stress update kernels (sm_100a).
//
// One time step of a propagator is two launches: the velocity phase (reads
// the stresses with a halo, updates vx, vz and their ψ strips in place) and
// the stress phase (reads the new velocities with a halo, updates the
// stresses, injects the source, applies the free surface).  Each block owns
// a 32-column × TZ-row tile of one propagator; the staged fields are copied
// to shared memory with an M-cell halo on all sides, the per-cell
// coefficients and the field being updated are read straight from HBM with
// coalesced 128-byte warp accesses.  A launch may carry many propagators
// (the batched form): the block finds its propagator by binary search over
// the StepWork table.
//
// Arithmetic order follows ertm/propagation.py (acoustic :430-454,
// viscoacoustic :686-723, elastic :840-883) and ertm/numerics.py (:68-117,
// :221-227) so the fields match the reference float32 fields bit for bit.
#pragma once

#include "ertm_device.cuh"

namespace ertm {

constexpr int TILE_X = 32;

template <int M, int TZ>
struct TileShape {
  static constexpr int W = TILE_X + 2 * M;
  static constexpr int H = TZ + 2 * M;
  static constexpr int N = W * H;
};

// Copy rows [i0−M, i0+TZ+M) × cols [j0−M, j0+32+M) of a padded field into
// shared memory; cells outside the padded grid read as 0 (never used by a
// valid stencil, which stays inside [0, n)).
template <int M, int TZ, int NT>
__device__ __forceinline__ void stage(float* s, const float* __restrict__ g, int nzp, int nxp, int ld,
                                      int i0, int j0) {
  using T = TileShape<M, TZ>;
  const int tid = threadIdx.y * TILE_X + threadIdx.x;
#pragma unroll 4
  for (int idx = tid; idx < T::N; idx += NT) {
    const int r = idx / T::W;
    const int c = idx - r * T::W;
    const int gi = i0 - M + r, gj = j0 - M + c;
    float v = 0.f;
    if (gi >= 0 && gi < nzp && gj >= 0 && gj < nxp) v = __ldg(g + (size_t)gi * ld + gj);
    s[idx] = v;
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

// ---------------------------------------------------------------------------
// velocity phase
// ---------------------------------------------------------------------------
// Acoustic and viscoacoustic: vx += (dt·irx)·(D⁺ₓp + ψ), vz += (dt·irz)·(D⁺_z p + ψ).
template <int M, int TZ, int BY>
__global__ void __launch_bounds__(TILE_X* BY)
k_pressure_velocity(const DevProp* __restrict__ props, WorkSet ws) {
  using T = TileShape<M, TZ>;
  __shared__ float sp[T::N];
  const StepWork w = find_work(ws, blockIdx.x);
  const DevProp& P = props[w.prop];
  const TileLoc L = tile_of(w, blockIdx.x, TZ);
  const int nzp = P.nzp, nxp = P.nxp, ld = P.ld;
  if ((w.flags & STEP_PEAK) && blockIdx.x == w.tile0 && threadIdx.x == 0 && threadIdx.y == 0)
    *P.peak = 0.f;  // the stress phase of this step reduces into it
  stage<M, TZ, TILE_X * BY>(sp, P.f[A_P], nzp, nxp, ld, L.i0, L.j0);
  __syncthreads();
  const int j = L.j0 + threadIdx.x;
  if (j >= nxp) return;
  float* __restrict__ vx = P.f[A_VX];
  float* __restrict__ vz = P.f[A_VZ];
  const float* __restrict__ irx = P.coef[CA_IRX];
  const float* __restrict__ irz = P.coef[CA_IRZ];
  const float c[4] = {P.c[0], P.c[1], P.c[2], P.c[3]};
  const float dt = P.dt, hx = P.hx, hz = P.hz;
  const bool xin = (j >= M && j < nxp - M);
  const int sx = strip_x(P, j);
  const float axj = sx >= 0 ? P.ax[j] : 0.f, bxj = sx >= 0 ? P.bx[j] : 1.f;
#pragma unroll
  for (int k = 0; k < TZ / BY; ++k) {
    const int r = threadIdx.y + k * BY;
    const int i = L.i0 + r;
    if (i >= nzp) break;
    const float* s = sp + (r + M) * T::W + threadIdx.x + M;
    const size_t g = (size_t)i * ld + j;
    float d = xin ? dplus<M>(s, 1, c, hx) : 0.f;
    if (sx >= 0) {
      float* ps = P.psix[0] + (size_t)i * P.wx + sx;
      float psi = *ps;
      d = cpml(d, psi, axj, bxj);
      *ps = psi;
    }
    vx[g] = fadd(vx[g], fmul(fmul(dt, irx[g]), d));
    d = (i >= M && i < nzp - M) ? dplus<M>(s, T::W, c, hz) : 0.f;
    const int sz = strip_z(P, i);
    if (sz >= 0) {
      float* ps = P.psiz[0] + (size_t)sz * ld + j;
      float psi = *ps;
      d = cpml(d, psi, P.az[i], P.bz[i]);
      *ps = psi;
    }
    vz[g] = fadd(vz[g], fmul(fmul(dt, irz[g]), d));
  }
}

// Elastic: vx += (dt·irx)·(D⁺ₓσxx + D⁻_zσxz), vz += (dt·irz)·(D⁻ₓσxz + D⁺_zσzz).
template <int M, int TZ, int BY>
__global__ void __launch_bounds__(TILE_X* BY)
k_elastic_velocity(const DevProp* __restrict__ props, WorkSet ws) {
  using T = TileShape<M, TZ>;
  __shared__ float sxx_s[T::N];
  __shared__ float szz_s[T::N];
  __shared__ float sxz_s[T::N];
  const StepWork w = find_work(ws, blockIdx.x);
  const DevProp& P = props[w.prop];
  const TileLoc L = tile_of(w, blockIdx.x, TZ);
  const int nzp = P.nzp, nxp = P.nxp, ld = P.ld;
  stage<M, TZ, TILE_X * BY>(sxx_s, P.f[E_SXX], nzp, nxp, ld, L.i0, L.j0);
  stage<M, TZ, TILE_X * BY>(szz_s, P.f[E_SZZ], nzp, nxp, ld, L.i0, L.j0);
  stage<M, TZ, TILE_X * BY>(sxz_s, P.f[E_SXZ], nzp, nxp, ld, L.i0, L.j0);
  __syncthreads();
  const int j = L.j0 + threadIdx.x;
  if (j >= nxp) return;
  float* __restrict__ vx = P.f[E_VX];
  float* __restrict__ vz = P.f[E_VZ];
  const float* __restrict__ irx = P.coef[CE_IRX];
  const float* __restrict__ irz = P.coef[CE_IRZ];
  const float c[4] = {P.c[0], P.c[1], P.c[2], P.c[3]};
  const float dt = P.dt, hx = P.hx, hz = P.hz;
  const bool xin = (j >= M && j < nxp - M);
  const int sx = strip_x(P, j);
  const float axj = sx >= 0 ? P.ax[j] : 0.f, bxj = sx >= 0 ? P.bx[j] : 1.f;
#pragma unroll
  for (int k = 0; k < TZ / BY; ++k) {
    const int r = threadIdx.y + k * BY;
    const int i = L.i0 + r;
    if (i >= nzp) break;
    const int so = (r + M) * T::W + threadIdx.x + M;
    const size_t g = (size_t)i * ld + j;
    const bool zin = (i >= M && i < nzp - M);
    const int sz = strip_z(P, i);
    const float azi = sz >= 0 ? P.az[i] : 0.f, bzi = sz >= 0 ? P.bz[i] : 1.f;
    // vx_dsxx (x, D⁺) and vx_dsxz (z, D⁻)
    float a = xin ? dplus<M>(sxx_s + so, 1, c, hx) : 0.f;
    float b = zin ? dminus<M>(sxz_s + so, T::W, c, hz) : 0.f;
    if (sx >= 0) {
      float* ps = P.psix[0] + (size_t)i * P.wx + sx;
      float psi = *ps; a = cpml(a, psi, axj, bxj); *ps = psi;
    }
    if (sz >= 0) {
      float* ps = P.psiz[0] + (size_t)sz * ld + j;
      float psi = *ps; b = cpml(b, psi, azi, bzi); *ps = psi;
    }
    vx[g] = fadd(vx[g], fmul(fmul(dt, irx[g]), fadd(a, b)));
    // vz_dsxz (x, D⁻) and vz_dszz (z, D⁺)
    a = xin ? dminus<M>(sxz_s + so, 1, c, hx) : 0.f;
    b = zin ? dplus<M>(szz_s + so, T::W, c, hz) : 0.f;
    if (sx >= 0) {
      float* ps = P.psix[1] + (size_t)i * P.wx + sx;
      float psi = *ps; a = cpml(a, psi, axj, bxj); *ps = psi;
    }
    if (sz >= 0) {
      float* ps = P.psiz[1] + (size_t)sz * ld + j;
      float psi = *ps; b = cpml(b, psi, azi, bzi); *ps = psi;
    }
    vz[g] = fadd(vz[g], fmul(fmul(dt, irz[g]), fadd(a, b)));
  }
}

// ---------------------------------------------------------------------------
// stress phase
// ---------------------------------------------------------------------------
__device__ __forceinline__ void block_max_to(float v, float* dst) {
  // v ≥ 0: the float bit pattern orders like the integer.
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  __shared__ float red[32];
  const int lane = threadIdx.x, wid = threadIdx.y;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < blockDim.y ? red[lane] : 0.f;
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) atomicMax(reinterpret_cast<int*>(dst), __float_as_int(v));
  }
}

// Acoustic (VISCO=false): p += (dt·κ)·div.  Viscoacoustic (VISCO=true):
// ε += dt·div; r_l ← r_l·a_l + b_l·Δε; p = K_R·ε + Σ r_l.
template <int M, int TZ, int BY, bool VISCO>
__global__ void __launch_bounds__(TILE_X* BY)
k_pressure_stress(const DevProp* __restrict__ props, WorkSet ws) {
  using T = TileShape<M, TZ>;
  __shared__ float svx[T::N];
  __shared__ float svz[T::N];
  const StepWork w = find_work(ws, blockIdx.x);
  const DevProp& P = props[w.prop];
  const TileLoc L = tile_of(w, blockIdx.x, TZ);
  const int nzp = P.nzp, nxp = P.nxp, ld = P.ld;
  stage<M, TZ, TILE_X * BY>(svx, P.f[A_VX], nzp, nxp, ld, L.i0, L.j0);
  stage<M, TZ, TILE_X * BY>(svz, P.f[A_VZ], nzp, nxp, ld, L.i0, L.j0);
  __syncthreads();
  const int j = L.j0 + threadIdx.x;
  const bool jok = j < nxp;
  float* __restrict__ p = P.f[A_P];
  const float c[4] = {P.c[0], P.c[1], P.c[2], P.c[3]};
  const float dt = P.dt, hx = P.hx, hz = P.hz;
  const bool xin = (j >= M && j < nxp - M);
  const int sx = jok ? strip_x(P, j) : -1;
  const float axj = sx >= 0 ? P.ax[j] : 0.f, bxj = sx >= 0 ? P.bx[j] : 1.f;
  float peak = 0.f;
#pragma unroll
  for (int k = 0; k < TZ / BY; ++k) {
    const int r = threadIdx.y + k * BY;
    const int i = L.i0 + r;
    if (!jok || i >= nzp) break;
    const int so = (r + M) * T::W + threadIdx.x + M;
    const size_t g = (size_t)i * ld + j;
    float dx = xin ? dminus<M>(svx + so, 1, c, hx) : 0.f;
    if (sx >= 0) {
      float* ps = P.psix[1] + (size_t)i * P.wx + sx;
      float psi = *ps; dx = cpml(dx, psi, axj, bxj); *ps = psi;
    }
    float dz = (i >= M && i < nzp - M) ? dminus<M>(svz + so, T::W, c, hz) : 0.f;
    const int sz = strip_z(P, i);
    if (sz >= 0) {
      float* ps = P.psiz[1] + (size_t)sz * ld + j;
      float psi = *ps; dz = cpml(dz, psi, P.az[i], P.bz[i]); *ps = psi;
    }
    const float div = fadd(dx, dz);
    const bool src = (i == P.src_iz && j == P.src_ix && w.amp != 0.f);
    if constexpr (!VISCO) {
      float pv = fadd(p[g], fmul(fmul(dt, P.coef[CA_KAPPA][g]), div));
      if (src) pv = fadd(pv, w.amp);
      if (P.free_surface && i == P.pad) pv = 0.f;
      p[g] = pv;
    } else {
      const float inc = fmul(dt, div);
      float* __restrict__ eps = P.f[V_EPS];
      float e = fadd(eps[g], inc);
      float total = 0.f;
      const uint8_t q = P.qidx[g];
      for (int l = 0; l < P.L; ++l) {
        float* __restrict__ rl = P.f[V_R0 + l];
        const float rv = fadd(fmul(rl[g], P.relax_a[q * P.L + l]), fmul(P.coef[CV_B0 + l][g], inc));
        rl[g] = rv;
        total = (l == 0) ? rv : fadd(total, rv);
      }
      float pv = fadd(fmul(P.coef[CV_KR][g], e), total);
      if (src) {
        e = fadd(e, w.amp_eps);
        pv = fadd(pv, w.amp);
      }
      eps[g] = e;
      p[g] = pv;
      peak = fmaxf(peak, fabsf(pv));
    }
  }
  if constexpr (VISCO) {
    if (w.flags & STEP_PEAK) block_max_to(peak, P.peak);
  }
}

// Elastic stress phase:
//   σxx += dt·(λ2μ·εxx + λ·εzz), σzz += dt·(λ·εxx + λ2μ·εzz),
//   σxz += (dt·μxz)·(D⁺_z vx + D⁺ₓ vz); source; free surface σzz = σxz = 0.
template <int M, int TZ, int BY>
__global__ void __launch_bounds__(TILE_X* BY)
k_elastic_stress(const DevProp* __restrict__ props, WorkSet ws) {
  using T = TileShape<M, TZ>;
  __shared__ float svx[T::N];
  __shared__ float svz[T::N];
  const StepWork w = find_work(ws, blockIdx.x);
  const DevProp& P = props[w.prop];
  const TileLoc L = tile_of(w, blockIdx.x, TZ);
  const int nzp = P.nzp, nxp = P.nxp, ld = P.ld;
  stage<M, TZ, TILE_X * BY>(svx, P.f[E_VX], nzp, nxp, ld, L.i0, L.j0);
  stage<M, TZ, TILE_X * BY>(svz, P.f[E_VZ], nzp, nxp, ld, L.i0, L.j0);
  __syncthreads();
  const int j = L.j0 + threadIdx.x;
  if (j >= nxp) return;
  float* __restrict__ sxx = P.f[E_SXX];
  float* __restrict__ szz = P.f[E_SZZ];
  float* __restrict__ sxz = P.f[E_SXZ];
  const float c[4] = {P.c[0], P.c[1], P.c[2], P.c[3]};
  const float dt = P.dt, hx = P.hx, hz = P.hz;
  const bool xin = (j >= M && j < nxp - M);
  const int sx = strip_x(P, j);
  const float axj = sx >= 0 ? P.ax[j] : 0.f, bxj = sx >= 0 ? P.bx[j] : 1.f;
#pragma unroll
  for (int k = 0; k < TZ / BY; ++k) {
    const int r = threadIdx.y + k * BY;
    const int i = L.i0 + r;
    if (i >= nzp) break;
    const int so = (r + M) * T::W + threadIdx.x + M;
    const size_t g = (size_t)i * ld + j;
    const bool zin = (i >= M && i < nzp - M);
    const int sz = strip_z(P, i);
    const float azi = sz >= 0 ? P.az[i] : 0.f, bzi = sz >= 0 ? P.bz[i] : 1.f;
    float exx = xin ? dminus<M>(svx + so, 1, c, hx) : 0.f;   // sxx_dvx
    float ezz = zin ? dminus<M>(svz + so, T::W, c, hz) : 0.f; // szz_dvz
    float f1 = zin ? dplus<M>(svx + so, T::W, c, hz) : 0.f;   // sxz_dvx
    float f2 = xin ? dplus<M>(svz + so, 1, c, hx) : 0.f;      // sxz_dvz
    if (sx >= 0) {
      float* p0 = P.psix[2] + (size_t)i * P.wx + sx;
      float psi = *p0; exx = cpml(exx, psi, axj, bxj); *p0 = psi;
      float* p1 = P.psix[3] + (size_t)i * P.wx + sx;
      psi = *p1; f2 = cpml(f2, psi, axj, bxj); *p1 = psi;
    }
    if (sz >= 0) {
      float* p0 = P.psiz[2] + (size_t)sz * ld + j;
      float psi = *p0; ezz = cpml(ezz, psi, azi, bzi); *p0 = psi;
      float* p1 = P.psiz[3] + (size_t)sz * ld + j;
      psi = *p1; f1 = cpml(f1, psi, azi, bzi); *p1 = psi;
    }
    const float lam = P.coef[CE_LAM][g], l2m = P.coef[CE_L2M][g];
    float vxx = fadd(sxx[g], fmul(dt, fadd(fmul(l2m, exx), fmul(lam, ezz))));
    float vzz = fadd(szz[g], fmul(dt, fadd(fmul(lam, exx), fmul(l2m, ezz))));
    float vxz = fadd(sxz[g], fmul(fmul(dt, P.coef[CE_MUXZ][g]), fadd(f1, f2)));
    if (i == P.src_iz && j == P.src_ix && w.amp != 0.f) {
      if (P.mech == MECH_SHEAR) {
        vxz = fadd(vxz, w.amp);
      } else if (P.mech == MECH_EXPLOSIVE) {
        vxx = fadd(vxx, w.amp);
        vzz = fadd(vzz, w.amp);
      }
      // force_z adds to vz after this launch (other blocks still read vz here).
    }
    if (P.free_surface && i == P.pad) {
      vzz = 0.f;
      vxz = 0.f;
    }
    sxx[g] = vxx;
    szz[g] = vzz;
    sxz[g] = vxz;
  }
}

}  // namespace ertm
