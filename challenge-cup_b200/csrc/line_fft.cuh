// Complex FFTs along lines, with the operation order of the pocketfft C++
// library (the FFT inside NumPy 2.x, numpy.fft), so that the wavenumber
// low-pass of the reference (ertm/numerics.py:424-442: fft2, radial taper,
// ifft2, real part) comes out bit for bit the same on the device.
//
// Algorithm (restated from pocketfft's published design, BSD-licensed, by
// M. Reinecke): a length-n complex transform runs either as a mixed-radix
// Cooley-Tukey sequence of passes over the factors of n (8s first, then 4s,
// a 2 moved to the front, then odd primes; radix 2/3/4/5/7/8/11 have fixed
// butterflies, larger primes a generic O(p²) pass), or - when n has a large
// prime factor and the cost model says so - as Bluestein's chirp-z
// convolution over an 11-smooth length n2 ≥ 2n−1.  The host builds the plan
// (factors, twiddle tables from a two-level table of cos/sin values, the
// Bluestein chirp and its transformed kernel); the device runs the passes.
//
// Every floating-point operation below is an explicit round-to-nearest
// intrinsic in the order the library evaluates it: no FMA contraction, no
// reassociation.  Butterflies of a pass are independent, so a CTA spreads a
// line's butterflies over its threads and synchronises between passes.
#pragma once

#include "ertm_device.cuh"

namespace ertm {

struct Cx {
  double r, i;
};

__device__ __forceinline__ Cx cx_add(Cx a, Cx b) { return {dadd(a.r, b.r), dadd(a.i, b.i)}; }
__device__ __forceinline__ Cx cx_sub(Cx a, Cx b) { return {dsub(a.r, b.r), dsub(a.i, b.i)}; }
__device__ __forceinline__ Cx cx_scale(Cx a, double s) { return {dmul(a.r, s), dmul(a.i, s)}; }
// v·conj(w) (forward) or v·w (backward), as the library's special_mul
template <bool FWD>
__device__ __forceinline__ Cx cx_smul(Cx v, Cx w) {
  return FWD ? Cx{dadd(dmul(v.r, w.r), dmul(v.i, w.i)), dsub(dmul(v.i, w.r), dmul(v.r, w.i))}
             : Cx{dsub(dmul(v.r, w.r), dmul(v.i, w.i)), dadd(dmul(v.r, w.i), dmul(v.i, w.r))};
}
// multiplication by ∓i
template <bool FWD>
__device__ __forceinline__ Cx cx_rot90(Cx a) {
  return FWD ? Cx{a.i, -a.r} : Cx{-a.i, a.r};
}
__device__ __forceinline__ Cx cx_ld(const double2* p) {
  const double2 v = __ldg(p);
  return {v.x, v.y};
}

// Butterfly constants: the library's long-double literals rounded to double.
constexpr double kHsqt2 = 0x1.6a09e667f3bcdp-1;     // √½
constexpr double kTw3 = 0x1.bb67ae8584caap-1;       // sin(2π/3)
constexpr double kTw5[4] = {0x1.3c6ef372fe950p-2, 0x1.e6f0e134454ffp-1, -0x1.9e3779b97f4a8p-1,
                            0x1.2cf2304755a5ep-1};
constexpr double kTw7[6] = {0x1.3f3a0e28bedd1p-1,  0x1.904c37505de4bp-1, -0x1.c7b90e3024582p-3,
                            0x1.f329c0558e969p-1,  -0x1.cd4bca9cb5c71p-1, 0x1.bc4c04d71abc1p-2};
constexpr double kTw11[10] = {0x1.aeb8c8764f0bap-1,  0x1.14cedf8bb580bp-1, 0x1.a9628d9c712b6p-2,
                              0x1.d1bb48eee2c13p-1,  -0x1.2375f640f44dbp-3, 0x1.fac9e043842efp-1,
                              -0x1.4f49e7f775887p-1, 0x1.82f19bb3a28a1p-1, -0x1.eb42a9bcd5057p-1,
                              0x1.207e7fd768dbfp-2};

template <bool FWD>
__device__ __forceinline__ Cx cx_rot45(Cx a) {
  return FWD ? Cx{dmul(kHsqt2, dadd(a.r, a.i)), dmul(kHsqt2, dsub(a.i, a.r))}
             : Cx{dmul(kHsqt2, dsub(a.r, a.i)), dmul(kHsqt2, dadd(a.i, a.r))};
}
template <bool FWD>
__device__ __forceinline__ Cx cx_rot135(Cx a) {
  return FWD ? Cx{dmul(kHsqt2, dsub(a.i, a.r)), dmul(kHsqt2, dsub(-a.r, a.i))}
             : Cx{dmul(kHsqt2, dsub(-a.r, a.i)), dmul(kHsqt2, dsub(a.r, a.i))};
}

// ---------------------------------------------------------------------------
// fixed-radix butterflies: c[0..IP) in, h[0..IP) out (before twiddles)
// ---------------------------------------------------------------------------
template <bool FWD, int IP>
struct Butterfly;

template <bool FWD>
struct Butterfly<FWD, 2> {
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    h[0] = cx_add(c[0], c[1]);
    h[1] = cx_sub(c[0], c[1]);
  }
};

template <bool FWD>
struct Butterfly<FWD, 3> {
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    const double twr = -0.5, twi = (FWD ? -1.0 : 1.0) * kTw3;
    const Cx t0 = c[0], t1 = cx_add(c[1], c[2]), t2 = cx_sub(c[1], c[2]);
    h[0] = cx_add(t0, t1);
    const Cx ca{dadd(t0.r, dmul(t1.r, twr)), dadd(t0.i, dmul(t1.i, twr))};
    const Cx cb{dmul(-t2.i, twi), dmul(t2.r, twi)};
    h[1] = cx_add(ca, cb);
    h[2] = cx_sub(ca, cb);
  }
};

template <bool FWD>
struct Butterfly<FWD, 4> {
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    const Cx t2 = cx_add(c[0], c[2]), t1 = cx_sub(c[0], c[2]);
    const Cx t3 = cx_add(c[1], c[3]);
    const Cx t4 = cx_rot90<FWD>(cx_sub(c[1], c[3]));
    h[0] = cx_add(t2, t3);
    h[2] = cx_sub(t2, t3);
    h[1] = cx_add(t1, t4);
    h[3] = cx_sub(t1, t4);
  }
};

template <bool FWD>
struct Butterfly<FWD, 8> {
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    Cx a1 = cx_add(c[1], c[5]), a5 = cx_sub(c[1], c[5]);
    Cx a3 = cx_add(c[3], c[7]), a7 = cx_sub(c[3], c[7]);
    {
      const Cx t = a1;
      a1 = cx_add(a1, a3);
      a3 = cx_sub(t, a3);
    }
    a3 = cx_rot90<FWD>(a3);
    a7 = cx_rot90<FWD>(a7);
    {
      const Cx t = a5;
      a5 = cx_add(a5, a7);
      a7 = cx_sub(t, a7);
    }
    a5 = cx_rot45<FWD>(a5);
    a7 = cx_rot135<FWD>(a7);
    const Cx a0 = cx_add(c[0], c[4]), a4 = cx_sub(c[0], c[4]);
    const Cx a2 = cx_add(c[2], c[6]);
    const Cx a6 = cx_rot90<FWD>(cx_sub(c[2], c[6]));
    const Cx s02 = cx_add(a0, a2), d02 = cx_sub(a0, a2);
    h[0] = cx_add(s02, a1);
    h[4] = cx_sub(s02, a1);
    h[2] = cx_add(d02, a3);
    h[6] = cx_sub(d02, a3);
    const Cx s46 = cx_add(a4, a6), d46 = cx_sub(a4, a6);
    h[1] = cx_add(s46, a5);
    h[5] = cx_sub(s46, a5);
    h[3] = cx_add(d46, a7);
    h[7] = cx_sub(d46, a7);
  }
};

// Odd prime radix P ∈ {5, 7, 11}: t⁺_m = c_m + c_{P−m}, t⁻_m = c_m − c_{P−m};
// h_u = ca ± cb with ca = c_0 + Σ_m cos-term·t⁺_m and cb from the sin-terms
// of t⁻_m, each sum taken left to right.  xr[u][m] is the 1-based index of
// the cosine constant, ys[u][m] that of the sine constant with its sign (the
// signs of the library's macro arguments).
template <bool FWD, int P, int H>
__device__ __forceinline__ void odd_prime(const Cx* c, Cx* h, const double* tr, const double* ti,
                                          const int (&xr)[H][H], const int (&ys)[H][H]) {
  Cx tp[H + 1], tm[H + 1];
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    tp[m] = cx_add(c[m], c[P - m]);
    tm[m] = cx_sub(c[m], c[P - m]);
  }
  double h0r = c[0].r, h0i = c[0].i;
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    h0r = dadd(h0r, tp[m].r);
    h0i = dadd(h0i, tp[m].i);
  }
  h[0] = {h0r, h0i};
  const double sg = FWD ? -1.0 : 1.0;
#pragma unroll
  for (int u = 1; u <= H; ++u) {
    double car = c[0].r, cai = c[0].i;
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      const double x = tr[xr[u - 1][m - 1] - 1];
      car = dadd(car, dmul(x, tp[m].r));
      cai = dadd(cai, dmul(x, tp[m].i));
    }
    double cbi = 0.0, cbr = 0.0;
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      const int s = ys[u - 1][m - 1];
      const double y = sg * ti[(s < 0 ? -s : s) - 1];
      const double pr = dmul(y, tm[m].r), pi = dmul(y, tm[m].i);
      if (m == 1) {
        cbi = pr;
        cbr = pi;
      } else if (s > 0) {
        cbi = dadd(cbi, pr);
        cbr = dadd(cbr, pi);
      } else {
        cbi = dsub(cbi, pr);
        cbr = dsub(cbr, pi);
      }
    }
    const Cx ca{car, cai}, cb{-cbr, cbi};
    h[u] = cx_add(ca, cb);
    h[P - u] = cx_sub(ca, cb);
  }
}

// The same butterfly handing each output to `out(j, value)` as soon as it is
// formed, so that a pass can twiddle and store it at once instead of holding
// all P outputs in registers.
template <bool FWD, int P, int H, class Out>
__device__ __forceinline__ void odd_prime_out(const Cx* c, const double* tr, const double* ti, const int (&xr)[H][H],
                                          const int (&ys)[H][H], Out out) {
  Cx tp[H + 1], tm[H + 1];
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    tp[m] = cx_add(c[m], c[P - m]);
    tm[m] = cx_sub(c[m], c[P - m]);
  }
  double h0r = c[0].r, h0i = c[0].i;
#pragma unroll
  for (int m = 1; m <= H; ++m) {
    h0r = dadd(h0r, tp[m].r);
    h0i = dadd(h0i, tp[m].i);
  }
  const Cx c0 = c[0];
  out(0, Cx{h0r, h0i});
  const double sg = FWD ? -1.0 : 1.0;
#pragma unroll
  for (int u = 1; u <= H; ++u) {
    double car = c0.r, cai = c0.i;
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      const double x = tr[xr[u - 1][m - 1] - 1];
      car = dadd(car, dmul(x, tp[m].r));
      cai = dadd(cai, dmul(x, tp[m].i));
    }
    double cbi = 0.0, cbr = 0.0;
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      const int s = ys[u - 1][m - 1];
      const double y = sg * ti[(s < 0 ? -s : s) - 1];
      const double pr = dmul(y, tm[m].r), pi = dmul(y, tm[m].i);
      if (m == 1) {
        cbi = pr;
        cbr = pi;
      } else if (s > 0) {
        cbi = dadd(cbi, pr);
        cbr = dadd(cbr, pi);
      } else {
        cbi = dsub(cbi, pr);
        cbr = dsub(cbr, pi);
      }
    }
    const Cx ca{car, cai}, cb{-cbr, cbi};
    out(u, cx_add(ca, cb));
    out(P - u, cx_sub(ca, cb));
  }
}

// run() fills h with the P outputs; run_out() hands each one to `out` as
// it is formed.  The constants are local arrays indexed by compile-time
// indices only, so they fold into immediates.
template <bool FWD>
struct Butterfly<FWD, 5> {
  template <class Out>
  __device__ __forceinline__ static void run_out(const Cx* c, Out out) {
    const double tr[2] = {kTw5[0], kTw5[2]}, ti[2] = {kTw5[1], kTw5[3]};
    constexpr int xr[2][2] = {{1, 2}, {2, 1}};
    constexpr int ys[2][2] = {{1, 2}, {2, -1}};
    odd_prime_out<FWD, 5, 2>(c, tr, ti, xr, ys, out);
  }
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    const double tr[2] = {kTw5[0], kTw5[2]}, ti[2] = {kTw5[1], kTw5[3]};
    constexpr int xr[2][2] = {{1, 2}, {2, 1}};
    constexpr int ys[2][2] = {{1, 2}, {2, -1}};
    odd_prime<FWD, 5, 2>(c, h, tr, ti, xr, ys);
  }
};

template <bool FWD>
struct Butterfly<FWD, 7> {
  template <class Out>
  __device__ __forceinline__ static void run_out(const Cx* c, Out out) {
    const double tr[3] = {kTw7[0], kTw7[2], kTw7[4]}, ti[3] = {kTw7[1], kTw7[3], kTw7[5]};
    constexpr int xr[3][3] = {{1, 2, 3}, {2, 3, 1}, {3, 1, 2}};
    constexpr int ys[3][3] = {{1, 2, 3}, {2, -3, -1}, {3, -1, 2}};
    odd_prime_out<FWD, 7, 3>(c, tr, ti, xr, ys, out);
  }
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    const double tr[3] = {kTw7[0], kTw7[2], kTw7[4]}, ti[3] = {kTw7[1], kTw7[3], kTw7[5]};
    constexpr int xr[3][3] = {{1, 2, 3}, {2, 3, 1}, {3, 1, 2}};
    constexpr int ys[3][3] = {{1, 2, 3}, {2, -3, -1}, {3, -1, 2}};
    odd_prime<FWD, 7, 3>(c, h, tr, ti, xr, ys);
  }
};

template <bool FWD>
struct Butterfly<FWD, 11> {
  template <class Out>
  __device__ __forceinline__ static void run_out(const Cx* c, Out out) {
    const double tr[5] = {kTw11[0], kTw11[2], kTw11[4], kTw11[6], kTw11[8]};
    const double ti[5] = {kTw11[1], kTw11[3], kTw11[5], kTw11[7], kTw11[9]};
    constexpr int xr[5][5] = {{1, 2, 3, 4, 5}, {2, 4, 5, 3, 1}, {3, 5, 2, 1, 4}, {4, 3, 1, 5, 2}, {5, 1, 4, 2, 3}};
    constexpr int ys[5][5] = {{1, 2, 3, 4, 5}, {2, 4, -5, -3, -1}, {3, -5, -2, 1, 4}, {4, -3, 1, 5, -2},
                              {5, -1, 4, -2, 3}};
    odd_prime_out<FWD, 11, 5>(c, tr, ti, xr, ys, out);
  }
  __device__ __forceinline__ static void run(const Cx* c, Cx* h) {
    const double tr[5] = {kTw11[0], kTw11[2], kTw11[4], kTw11[6], kTw11[8]};
    const double ti[5] = {kTw11[1], kTw11[3], kTw11[5], kTw11[7], kTw11[9]};
    constexpr int xr[5][5] = {{1, 2, 3, 4, 5}, {2, 4, 5, 3, 1}, {3, 5, 2, 1, 4}, {4, 3, 1, 5, 2}, {5, 1, 4, 2, 3}};
    constexpr int ys[5][5] = {{1, 2, 3, 4, 5}, {2, 4, -5, -3, -1}, {3, -5, -2, 1, 4}, {4, -3, 1, 5, -2},
                              {5, -1, 4, -2, 3}};
    odd_prime<FWD, 11, 5>(c, h, tr, ti, xr, ys);
  }
};

// ---------------------------------------------------------------------------
// plans and passes
// ---------------------------------------------------------------------------
constexpr int kFftMaxFactors = 40;

// One transform length, as the device sees it.  For a Bluestein plan the
// factors and twiddles are those of the inner length n2.
struct FftPlanDev {
  int32_t n;                        // transform length
  int32_t n2;                       // inner Cooley-Tukey length (n unless Bluestein)
  int32_t blue;                     // 1: Bluestein
  int32_t nfact;
  int32_t fct[kFftMaxFactors];
  int32_t twoff[kFftMaxFactors];    // per pass: offset of its twiddles in tw
  int32_t twsoff[kFftMaxFactors];   // per generic pass: offset of its p roots in tw
  const double2* tw;
  const double2* bk;                // Bluestein chirp, n values
  const double2* bkf;               // transformed Bluestein kernel, n2 values (mirrored half spectrum)
};

// A fixed-radix pass: CC(i, j, k) = cc[i + ido·(j + IP·k)] → CH(i, k, j) =
// ch[i + ido·(k + l1·j)], output j ≥ 1 of butterfly i ≥ 1 twiddled by
// WA(j−1, i) = wa[i−1 + (j−1)·(ido−1)].
template <bool FWD, int IP, bool EAGER>
__device__ __forceinline__ void fft_pass(int ido, int l1, const Cx* cc, Cx* ch, const double2* wa) {
  const int nb = l1 * ido;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int k = b / ido, i = b - k * ido;
    Cx c[IP];
#pragma unroll
    for (int j = 0; j < IP; ++j) c[j] = cc[i + ido * (j + IP * k)];
    if constexpr (EAGER && (IP == 5 || IP == 7 || IP == 11)) {
      // odd primes: each output twiddled and stored as soon as it is formed
      // (fewer live registers where the launch caps them)
      Butterfly<FWD, IP>::run_out(c, [&](int j, Cx v) {
        if (j > 0 && i > 0) v = cx_smul<FWD>(v, cx_ld(wa + (i - 1) + (j - 1) * (ido - 1)));
        ch[i + ido * (k + l1 * j)] = v;
      });
    } else {
      Cx h[IP];
      Butterfly<FWD, IP>::run(c, h);
      ch[i + ido * k] = h[0];
#pragma unroll
      for (int j = 1; j < IP; ++j) {
        Cx v = h[j];
        if (i > 0) v = cx_smul<FWD>(v, cx_ld(wa + (i - 1) + (j - 1) * (ido - 1)));
        ch[i + ido * (k + l1 * j)] = v;
      }
    }
  }
}

// The generic pass for a prime ip > 11 (the library's passg).  Every (i, k)
// is independent once the inputs are read: phase 1 forms the sums and
// differences CH, phase 2 the ip outputs in place of the input (CX), with
// the library's loop order over l and j.  `wal` roots come from tws.
template <bool FWD>
__device__ __forceinline__ void fft_pass_generic(int ido, int ip, int l1, Cx* cc, Cx* ch, const double2* wa,
                                                 const double2* tws) {
  const int ipph = (ip + 1) / 2;
  const int idl1 = ido * l1;
  for (int ik = threadIdx.x; ik < idl1; ik += blockDim.x) {
    const int k = ik / ido, i = ik - k * ido;
    auto CC = [&](int j) { return cc[i + ido * (j + ip * k)]; };
    ch[ik] = CC(0);
    for (int j = 1, jc = ip - 1; j < ipph; ++j, --jc) {
      const Cx a = CC(j), b = CC(jc);
      ch[ik + idl1 * j] = cx_add(a, b);
      ch[ik + idl1 * jc] = cx_sub(a, b);
    }
  }
  __syncthreads();
  auto wal = [&](int q) {
    if (q == 0) return Cx{1.0, 0.0};
    const Cx w = cx_ld(tws + q);
    return Cx{w.r, FWD ? -w.i : w.i};
  };
  for (int ik = threadIdx.x; ik < idl1; ik += blockDim.x) {
    const Cx* H = ch + ik;     // H[idl1·j]
    Cx* X = cc + ik;           // X[idl1·j]
    Cx tmp = H[0];
    for (int j = 1; j < ipph; ++j) tmp = cx_add(tmp, H[idl1 * j]);
    X[0] = tmp;
    for (int l = 1, lc = ip - 1; l < ipph; ++l, --lc) {
      const Cx w1 = wal(l), w2 = wal(2 * l);
      const Cx h0 = H[0], h1 = H[idl1], h2 = H[2 * idl1], hm1 = H[idl1 * (ip - 1)], hm2 = H[idl1 * (ip - 2)];
      Cx xl{dadd(dadd(h0.r, dmul(w1.r, h1.r)), dmul(w2.r, h2.r)), dadd(dadd(h0.i, dmul(w1.r, h1.i)), dmul(w2.r, h2.i))};
      Cx xlc{-dadd(dmul(w1.i, hm1.i), dmul(w2.i, hm2.i)), dadd(dmul(w1.i, hm1.r), dmul(w2.i, hm2.r))};
      int iwal = 2 * l;
      int j = 3, jc = ip - 3;
      for (; j < ipph - 1; j += 2, jc -= 2) {
        iwal += l;
        if (iwal > ip) iwal -= ip;
        const Cx xw = wal(iwal);
        iwal += l;
        if (iwal > ip) iwal -= ip;
        const Cx xw2 = wal(iwal);
        const Cx hj = H[idl1 * j], hj1 = H[idl1 * (j + 1)], hc = H[idl1 * jc], hc1 = H[idl1 * (jc - 1)];
        xl.r = dadd(xl.r, dadd(dmul(hj.r, xw.r), dmul(hj1.r, xw2.r)));
        xl.i = dadd(xl.i, dadd(dmul(hj.i, xw.r), dmul(hj1.i, xw2.r)));
        xlc.r = dsub(xlc.r, dadd(dmul(hc.i, xw.i), dmul(hc1.i, xw2.i)));
        xlc.i = dadd(xlc.i, dadd(dmul(hc.r, xw.i), dmul(hc1.r, xw2.i)));
      }
      for (; j < ipph; ++j, --jc) {
        iwal += l;
        if (iwal > ip) iwal -= ip;
        const Cx xw = wal(iwal);
        const Cx hj = H[idl1 * j], hc = H[idl1 * jc];
        xl.r = dadd(xl.r, dmul(hj.r, xw.r));
        xl.i = dadd(xl.i, dmul(hj.i, xw.r));
        xlc.r = dsub(xlc.r, dmul(hc.i, xw.i));
        xlc.i = dadd(xlc.i, dmul(hc.r, xw.i));
      }
      X[idl1 * l] = xl;
      X[idl1 * lc] = xlc;
    }
    // shuffling and twiddling
    const int k = ik / ido, i = ik - k * ido;
    (void)k;
    for (int j = 1, jc = ip - 1; j < ipph; ++j, --jc) {
      const Cx a = X[idl1 * j], b = X[idl1 * jc];
      Cx x1 = cx_add(a, b), x2 = cx_sub(a, b);
      if (i > 0) {
        x1 = cx_smul<FWD>(x1, cx_ld(wa + (j - 1) * (ido - 1) + i - 1));
        x2 = cx_smul<FWD>(x2, cx_ld(wa + (jc - 1) * (ido - 1) + i - 1));
      }
      X[idl1 * j] = x1;
      X[idl1 * jc] = x2;
    }
  }
}

// All passes of a Cooley-Tukey plan over a (in) with b as the other buffer;
// returns the buffer that holds the result.  Callers synchronise before.
template <bool FWD, bool EAGER>
__device__ __forceinline__ Cx* fft_passes(const FftPlanDev& p, Cx* a, Cx* b) {
  Cx* p1 = a;
  Cx* p2 = b;
  int l1 = 1;
  for (int f = 0; f < p.nfact; ++f) {
    const int ip = p.fct[f];
    const int ido = p.n2 / (l1 * ip);
    const double2* wa = p.tw + p.twoff[f];
    bool swap = true;
    switch (ip) {
      case 2: fft_pass<FWD, 2, EAGER>(ido, l1, p1, p2, wa); break;
      case 3: fft_pass<FWD, 3, EAGER>(ido, l1, p1, p2, wa); break;
      case 4: fft_pass<FWD, 4, EAGER>(ido, l1, p1, p2, wa); break;
      case 5: fft_pass<FWD, 5, EAGER>(ido, l1, p1, p2, wa); break;
      case 7: fft_pass<FWD, 7, EAGER>(ido, l1, p1, p2, wa); break;
      case 8: fft_pass<FWD, 8, EAGER>(ido, l1, p1, p2, wa); break;
      case 11: fft_pass<FWD, 11, EAGER>(ido, l1, p1, p2, wa); break;
      default:
        fft_pass_generic<FWD>(ido, ip, l1, p1, p2, wa, p.tw + p.twsoff[f]);
        swap = false;   // the generic pass leaves its result in place
        break;
    }
    __syncthreads();
    if (swap) {
      Cx* t = p1;
      p1 = p2;
      p2 = t;
    }
    l1 *= ip;
  }
  return p1;
}

// ---------------------------------------------------------------------------
// the wavenumber taper of numerics.py:424-442 at (iz, jx) of an (nz, nx)
// spectrum: fftfreq, the Nyquist ratios, the radius and the clipped ramp, in
// NumPy's operation order
// ---------------------------------------------------------------------------
__device__ __forceinline__ double lowpass_taper(int iz, int jx, int nz, int nx, double dz, double dx, double cutoff) {
  const int kzi = iz < (nz + 1) / 2 ? iz : iz - nz;
  const int kxi = jx < (nx + 1) / 2 ? jx : jx - nx;
  const double kz = dmul((double)kzi, __ddiv_rn(1.0, dmul((double)nz, dz)));
  const double kx = dmul((double)kxi, __ddiv_rn(1.0, dmul((double)nx, dx)));
  const double rz = __ddiv_rn(kz, fmax(__ddiv_rn(0.5, dz), 1e-12));
  const double rx = __ddiv_rn(kx, fmax(__ddiv_rn(0.5, dx), 1e-12));
  const double rad = __dsqrt_rn(dadd(dmul(rz, rz), dmul(rx, rx)));
  const double h = dsub(1.0, __ddiv_rn(dsub(rad, cutoff), 0.15));
  return h < 0.0 ? 0.0 : (h > 1.0 ? 1.0 : h);
}

enum LineLoad : int32_t {
  LINE_LOAD_F32 = 0,    // real float32 lines, pitch `src_pitch` floats (a padded field), per segment
  LINE_LOAD_F64 = 1,    // real float64 lines, pitch `src_pitch` doubles (an image), per segment
  LINE_LOAD_C = 2,      // complex lines of the segment's work array, pitch n
  LINE_LOAD_C_TAPER = 3 // the same times the taper at (row, m) of a (seg_lines, n) spectrum
};

// Several arrays of the same shape ("segments", e.g. p and ε of every
// propagator that needs the low-pass at this step) go through one launch:
// line l is row l % seg_lines of segment l / seg_lines; every segment has its
// own real input and its own complex work array.
constexpr int kLineMaxSegs = 64;

struct LineJob {
  FftPlanDev plan;
  int32_t load;
  int32_t use_smem;      // 1: work buffers in dynamic shared memory, else in `scratch`
  int64_t lines;         // nseg · seg_lines
  int32_t seg_lines;
  int32_t nseg;
  const void* src[kLineMaxSegs];   // real loads: each segment's first row
  int64_t src_pitch;
  double2* cbuf[kLineMaxSegs];     // complex lines of each segment, pitch n: the input of complex loads and
                                   // the output of every transform (in place)
  double fct;            // output scale (1, or 1/n for an inverse transform)
  double2* scratch;      // 2·n2 values per CTA when not in shared memory
  double dz, dx, cutoff; // taper of LINE_LOAD_C_TAPER
};

__device__ __forceinline__ Cx line_load(const LineJob& J, int seg, int row, int m) {
  const int n = J.plan.n;
  switch (J.load) {
    case LINE_LOAD_F32:
      return {(double)static_cast<const float*>(J.src[seg])[(int64_t)row * J.src_pitch + m], 0.0};
    case LINE_LOAD_F64:
      return {static_cast<const double*>(J.src[seg])[(int64_t)row * J.src_pitch + m], 0.0};
    case LINE_LOAD_C: {
      const double2 v = J.cbuf[seg][(int64_t)row * n + m];
      return {v.x, v.y};
    }
    default: {
      // spectrum × taper as NumPy multiplies complex128 by float64: the taper
      // is the complex (h, 0)
      const double2 v = J.cbuf[seg][(int64_t)row * n + m];
      const double h = lowpass_taper(row, m, J.seg_lines, n, J.dz, J.dx, J.cutoff);
      return {dsub(dmul(v.x, h), dmul(v.y, 0.0)), dadd(dmul(v.x, 0.0), dmul(v.y, h))};
    }
  }
}

// One CTA per line (grid-stride over lines): load, transform, scale, store.
// A Bluestein line is multiplied by the chirp, zero-padded to n2, convolved
// with the kernel through a forward and a backward length-n2 transform and
// multiplied by the chirp again (fftblue::fft of the library).  The launch
// has at most MAXT threads; how many only sets how the butterflies of a pass
// are spread over them.  SMEM: the two work buffers in dynamic shared
// memory (shared loads and stores), else in per-CTA global scratch.  MINB:
// resident CTAs per SM the register allocation is capped for (0: none
// beyond MAXT's); where the cap is tight (several CTAs, or more than 512
// threads) the odd-prime passes store their outputs eagerly.
template <bool FWD, int MAXT, bool SMEM, int MINB = 0>
__global__ void __launch_bounds__(MAXT, MINB) k_fft_lines(const LineJob J) {
  constexpr bool EAGER = MINB > 1 || MAXT > 512;   // registers capped below ~110
  extern __shared__ double2 line_smem[];
  const FftPlanDev& P = J.plan;
  const int n = P.n, n2 = P.n2;
  Cx* a = SMEM ? reinterpret_cast<Cx*>(line_smem) : reinterpret_cast<Cx*>(J.scratch) + (size_t)blockIdx.x * 2 * n2;
  Cx* b = a + n2;
  for (int64_t line = blockIdx.x; line < J.lines; line += gridDim.x) {
    const int seg = (int)(line / J.seg_lines), row = (int)(line - (int64_t)seg * J.seg_lines);
    if (P.blue) {
      for (int m = threadIdx.x; m < n2; m += blockDim.x)
        a[m] = m < n ? cx_smul<FWD>(line_load(J, seg, row, m), cx_ld(P.bk + m)) : Cx{0.0, 0.0};
    } else {
      for (int m = threadIdx.x; m < n; m += blockDim.x) a[m] = line_load(J, seg, row, m);
    }
    __syncthreads();
    Cx* r;
    if (P.blue) {
      r = fft_passes<true, EAGER>(P, a, b);
      for (int m = threadIdx.x; m < n2; m += blockDim.x) r[m] = cx_smul<!FWD>(r[m], cx_ld(P.bkf + m));
      __syncthreads();
      r = fft_passes<false, EAGER>(P, r, r == a ? b : a);
    } else {
      r = fft_passes<FWD, EAGER>(P, a, b);
    }
    double2* out = J.cbuf[seg] + (int64_t)row * n;
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      Cx v = r[m];
      if (P.blue) v = cx_smul<FWD>(v, cx_ld(P.bk + m));
      v = cx_scale(v, J.fct);
      out[m] = make_double2(v.r, v.i);
    }
    __syncthreads();   // the buffers are reused by the next line
  }
}

// ---------------------------------------------------------------------------
// transposes between the two axes (32×32 tiles through shared memory), one
// segment per blockIdx.z: complex (rows × cols) → complex (cols × rows), or
// the real part back into each segment's own real array
// ---------------------------------------------------------------------------
enum TransposeOut : int32_t {
  T_COMPLEX = 0,    // out[z][c·rows + r] = in[z][r·cols + c]
  T_REAL_F32 = 1,   // out[z][c·ld + r] = float32(real part): back into a padded field
  T_REAL_F64 = 2    // out[z][c·ld + r] = real part: an image
};

struct TransposeArgs {
  const double2* in[kLineMaxSegs];
  void* out[kLineMaxSegs];
};

template <int MODE>
__global__ void k_transpose_lines(const __grid_constant__ TransposeArgs T, int rows, int cols, int64_t ld) {
  __shared__ double2 tile[32][33];
  const double2* in = T.in[blockIdx.z];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[y][threadIdx.x] = in[(int64_t)r * cols + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (r < rows && c < cols) {
      const double2 v = tile[threadIdx.x][y];
      if (MODE == T_COMPLEX) static_cast<double2*>(T.out[blockIdx.z])[(int64_t)c * rows + r] = v;
      else if (MODE == T_REAL_F32) static_cast<float*>(T.out[blockIdx.z])[(int64_t)c * ld + r] = __double2float_rn(v.x);
      else static_cast<double*>(T.out[blockIdx.z])[(int64_t)c * ld + r] = v.x;
    }
  }
}

}  // namespace ertm
