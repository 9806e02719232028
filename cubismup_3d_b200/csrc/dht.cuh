// Shared-memory FFT passes of the periodic Poisson solve
// (the device replacement of PoissonSolverPeriodic's FFTW r2c / _solve / c2r,
// source/poisson/PoissonSolverPeriodic.cpp:15-146).
//
// The solve is p = H(f . H(b)) with H the separable real Hartley transform
// H[k] = Re X[k] - Im X[k] (X the unnormalised DFT) applied along x, y and z,
// and f the reference's grid-consistent factor
//   f = 4 / (Nx h Ny Nz) / (2 (cos(4 pi kx/Nx) + cos(4 pi ky/Ny) + cos(4 pi kz/Nz)) - 6)
// with the 8 modes kx in {0, Nx/2}, ky in {0, Ny/2}, kz in {0, Nz/2} zeroed.
// Because the wide Laplacian is a sum of symmetric circulants, the cos/sin
// pair of each DFT mode is one eigenspace, so H diagonalises it exactly like
// the DFT does; H is its own inverse up to 1/N. Everything stays real, every
// pass is in place on an Nx*Ny*Nz array, and the data layout never changes.
//
// A length-N Hartley transform is one length-M = N/2 complex FFT of
// z[m] = x[2m] + i x[2m+1] (Stockham autosort, radix 8/4/2 stages, Govindaraju
// et al., SC'08) followed by the standard even/odd split to X[k], k <= M.
#pragma once

#include "common.cuh"

namespace cup {

template <typename R>
struct Cplx;
template <>
struct Cplx<double> {
  using T = double2;
};
template <>
struct Cplx<float> {
  using T = float2;
};

template <typename R2>
__device__ __forceinline__ R2 cmul(R2 a, R2 b) {
  R2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename R2>
__device__ __forceinline__ R2 cadd(R2 a, R2 b) {
  R2 r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename R2>
__device__ __forceinline__ R2 csub(R2 a, R2 b) {
  R2 r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
// -i * a
template <typename R2>
__device__ __forceinline__ R2 cmul_mi(R2 a) {
  R2 r;
  r.x = a.y;
  r.y = -a.x;
  return r;
}

// Forward (e^{-2 pi i/R}) R-point DFTs in registers.
template <int R, typename R2>
struct DFT;
template <typename R2>
struct DFT<2, R2> {
  __device__ __forceinline__ static void run(R2* v) {
    const R2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <typename R2>
struct DFT<4, R2> {
  __device__ __forceinline__ static void run(R2* v) {
    const R2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const R2 t2 = cadd(v[1], v[3]), t3 = cmul_mi(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};
template <typename R2>
struct DFT<8, R2> {
  __device__ __forceinline__ static void run(R2* v) {
    using S = decltype(v[0].x);
    const S c = (S)0.70710678118654752440084436210484904;  // sqrt(2)/2
    R2 e[4] = {v[0], v[2], v[4], v[6]};
    R2 o[4] = {v[1], v[3], v[5], v[7]};
    DFT<4, R2>::run(e);
    DFT<4, R2>::run(o);
    // twiddles W8^k, k = 0..3: 1, c(1-i), -i, -c(1+i)
    R2 w1, w3;
    w1.x = c * (o[1].x + o[1].y);
    w1.y = c * (o[1].y - o[1].x);
    const R2 w2 = cmul_mi(o[2]);
    w3.x = c * (o[3].y - o[3].x);
    w3.y = -c * (o[3].x + o[3].y);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], w1);
    v[5] = csub(e[1], w1);
    v[2] = cadd(e[2], w2);
    v[6] = csub(e[2], w2);
    v[3] = cadd(e[3], w3);
    v[7] = csub(e[3], w3);
  }
};

// 16-point forward DFT as 4 x 4: X[k1 + 4 k2] =
//   sum_n2 W4^(n2 k2) W16^(n2 k1) sum_n1 x[4 n1 + n2] W4^(n1 k1).
template <typename R2>
struct DFT<16, R2> {
  __device__ __forceinline__ static R2 cm(R2 a, double re, double im) {
    using S = decltype(a.x);
    R2 r;
    r.x = a.x * (S)re - a.y * (S)im;
    r.y = a.x * (S)im + a.y * (S)re;
    return r;
  }
  __device__ __forceinline__ static void run(R2* v) {
    constexpr double c1 = 0.92387953251128675613;  // cos(pi/8)
    constexpr double s1 = 0.38268343236508977173;  // sin(pi/8)
    constexpr double h = 0.70710678118654752440;   // sqrt(2)/2
    R2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      R2 t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      DFT<4, R2>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = t[k1];
    }
    // twiddles W16^(n2 k1) = cos(2 pi m / 16) - i sin(2 pi m / 16), m = n2 k1
    y[1][1] = cm(y[1][1], c1, -s1);
    y[1][2] = cm(y[1][2], h, -h);
    y[1][3] = cm(y[1][3], s1, -c1);
    y[2][1] = cm(y[2][1], h, -h);
    y[2][2] = cmul_mi(y[2][2]);
    y[2][3] = cm(y[2][3], -h, -h);
    y[3][1] = cm(y[3][1], s1, -c1);
    y[3][2] = cm(y[3][2], -h, -h);
    y[3][3] = cm(y[3][3], -c1, s1);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      R2 t[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      DFT<4, R2>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
    }
  }
};

// Radix plan of an M-point complex FFT: radix-8 stages then one 2 or 4.
template <int M>
struct FFTPlan {
  static constexpr int nstages = (M == 8) ? 1 : (M == 16 || M == 32 || M == 64) ? 2 : 3;
  static constexpr int radix(int s) {
    return s == 0 ? 8
           : s == 1 ? (M == 16 ? 2 : M == 32 ? 4 : 8)
                    : (M == 128 ? 2 : 4);
  }
  static constexpr int ns(int s) { return s == 0 ? 1 : s == 1 ? 8 : 64; }
  // offset of stage s's twiddle table (R*Ns entries) in the per-length table
  static constexpr int tw_off(int s) { return s <= 1 ? 0 : radix(1) * ns(1); }
  static constexpr int tw_stage_total() {
    return nstages == 1 ? 0 : nstages == 2 ? radix(1) * ns(1) : radix(1) * ns(1) + radix(2) * ns(2);
  }
  // post-processing table W_N^k, k = 0..M/2, follows the stage tables
  static constexpr int post_off() { return tw_stage_total(); }
  // M = 128 only: W128^(r j), r < 8, j < 16 (index 16 r + j) of the 8-thread
  // plan (radix 16, then radix 8 over Ns = 16), after the post table
  static constexpr int r16_off() { return tw_stage_total() + M / 2 + 1; }
  static constexpr int table_len() { return tw_stage_total() + M / 2 + 1 + (M == 128 ? 128 : 0); }
  // the row passes use the 16-thread plan only: stage and post tables
  static constexpr int rows_table_len() { return tw_stage_total() + M / 2 + 1; }
};

// ---- line accessors -------------------------------------------------------
// Row lines: line l starts at base + l*pitch (reals), complex m at reals 2m, 2m+1.
template <typename R>
struct RowLines {
  using elem = R;
  using R2 = typename Cplx<R>::T;
  R* base;
  int pitch;
  __device__ __forceinline__ R2 ld(int l, int m) const { return *reinterpret_cast<const R2*>(base + l * pitch + 2 * m); }
  __device__ __forceinline__ void st(int l, int m, R2 v) const { *reinterpret_cast<R2*>(base + l * pitch + 2 * m) = v; }
  __device__ __forceinline__ R ldr(int l, int n) const { return base[l * pitch + n]; }
  __device__ __forceinline__ void str(int l, int n, R v) const { base[l * pitch + n] = v; }
};
// Padded row lines (complex m stored at m + m/8) to keep the first Stockham
// stage's stride-8 stores free of bank conflicts.
template <typename R>
struct RowLinesPad {
  using elem = R;
  using R2 = typename Cplx<R>::T;
  R* base;
  int pitch;  // reals per line (>= 2*(M + M/8))
  __device__ __forceinline__ R2 ld(int l, int m) const {
    return *reinterpret_cast<const R2*>(base + l * pitch + 2 * (m + (m >> 3)));
  }
  __device__ __forceinline__ void st(int l, int m, R2 v) const {
    *reinterpret_cast<R2*>(base + l * pitch + 2 * (m + (m >> 3))) = v;
  }
};
// Column lines of a tile [n][W]: element n of line l at n*W + l.
template <typename R>
struct ColLines {
  using elem = R;
  using R2 = typename Cplx<R>::T;
  R* base;
  int W;
  __device__ __forceinline__ R2 ld(int l, int m) const {
    R2 v;
    v.x = base[(2 * m) * W + l];
    v.y = base[(2 * m + 1) * W + l];
    return v;
  }
  __device__ __forceinline__ void st(int l, int m, R2 v) const {
    base[(2 * m) * W + l] = v.x;
    base[(2 * m + 1) * W + l] = v.y;
  }
  __device__ __forceinline__ R ldr(int l, int n) const { return base[n * W + l]; }
  __device__ __forceinline__ void str(int l, int n, R v) const { base[n * W + l] = v; }
};

// One Stockham stage: each of the M/8 threads of a line does 8/R radix-R
// butterflies j = t + b*M/8, reading in[j + r*M/R], writing
// out[(j/Ns)*Ns*R + j%Ns + r*Ns]. All threads of the CTA take part
// (every line in parallel), so the barriers are block-wide.
template <int M, int R, int NS, bool INPLACE, typename R2, class In, class Out>
__device__ __forceinline__ void fft_stage(const In& in, const Out& out, const R2* tw, int l, int t, bool active) {
  constexpr int NB = 8 / R;
  constexpr int TPL = M / 8;
  R2 v[8];
  if (active) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + b * TPL;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b * R + r] = in.ld(l, j + r * (M / R));
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[b * R + r] = cmul(v[b * R + r], tw[r * NS + (j % NS)]);
      }
    }
  }
  if (INPLACE) __syncthreads();
  if (active) {
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const int j = t + b * TPL;
      DFT<R, R2>::run(&v[b * R]);
      const int idxD = (j / NS) * NS * R + (j % NS);
#pragma unroll
      for (int r = 0; r < R; ++r) out.st(l, idxD + r * NS, v[b * R + r]);
    }
  }
  __syncthreads();
}

// No scaling after the forward transform.
struct NoScale {
  using type = double;
  static constexpr bool kOn = false;
  __device__ double operator()(int) const { return 1.0; }
};

// Even/odd split of the packed M-point FFT Z into the Hartley transform H of
// the length-2M real line, in place (task k handles Z[k], Z[M-k] and writes
// H[k], H[N-k], H[M-k], H[M+k]). With a scaler, the four outputs of task k are
// multiplied by scale(k): for the wide Laplacian (eigenvalue a function of
// cos(4 pi k / N), which has period N/2 and is even) the four indices k, N-k,
// M-k, M+k share one eigenvalue, so the spectral divide costs one factor per
// four values.
// The outputs go to `ao`; all inputs are read before a block barrier and the
// outputs written after it, so `ao` may alias `a` even with a wider element
// type (the z pass of the mixed-precision solve reads FP32 lines and writes
// FP64 ones over the same bytes).
// Split task k of one line: Z[k] = A, Z[M-k] = B -> H[k], H[N-k], H[M-k],
// H[M+k] (task 0: H[0], H[M] from A = Z[0]), times scale(k).
template <int M, typename R, typename R2, class AccO, class Scale>
__device__ __forceinline__ void split_task(const AccO& ao, int l, int k, R2 A, R2 B, R2 W, const Scale& scale) {
  using RO = typename AccO::elem;
  constexpr int N = 2 * M;
  using SF = typename Scale::type;  // the factor's type, in which the product is formed
  if (k == 0) {
    RO h0, hM;
    if constexpr (Scale::kOn) {
      const SF f = scale(0);
      h0 = (RO)((SF)(A.x + A.y) * f);
      hM = (RO)((SF)(A.x - A.y) * f);
    } else {
      h0 = (RO)(A.x + A.y);
      hM = (RO)(A.x - A.y);
    }
    ao.str(l, 0, h0);
    ao.str(l, M, hM);
  } else {
    const R half = (R)0.5;
    const R Er = (A.x + B.x) * half, Ei = (A.y - B.y) * half;
    const R Or = (A.y + B.y) * half, Oi = (B.x - A.x) * half;
    const R Xr = Er + (W.x * Or - W.y * Oi), Xi = Ei + (W.x * Oi + W.y * Or);
    const R X2r = Er - W.x * Or + W.y * Oi, X2i = -Ei + W.x * Oi + W.y * Or;
    RO hk, hNk, hMk, hMpk;
    if constexpr (Scale::kOn) {
      const SF f = scale(k);
      hk = (RO)((SF)(Xr - Xi) * f);
      hNk = (RO)((SF)(Xr + Xi) * f);
      hMk = (RO)((SF)(X2r - X2i) * f);
      hMpk = (RO)((SF)(X2r + X2i) * f);
    } else {
      hk = (RO)(Xr - Xi);
      hNk = (RO)(Xr + Xi);
      hMk = (RO)(X2r - X2i);
      hMpk = (RO)(X2r + X2i);
    }
    ao.str(l, k, hk);
    ao.str(l, N - k, hNk);
    // k = M/2: M - k = k and M + k = N - k (same values); write each index
    // once, so that an accumulating accessor adds it once
    if (2 * k != M) {
      ao.str(l, M - k, hMk);
      ao.str(l, M + k, hMpk);
    }
  }
}

template <int M, typename R, typename R2, class Acc, class AccO, class Scale>
__device__ __forceinline__ void dht_post_to(const Acc& a, const AccO& ao, const R2* twp, int l, int t, bool active,
                                            const Scale& scale) {
  constexpr int TPL = M / 8;
  constexpr int NT = (M / 2 + 1 + TPL - 1) / TPL;
  R2 A_[NT], B_[NT];
  if (active) {
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      const int k = t + i * TPL;
      if (k <= M / 2) {
        A_[i] = a.ld(l, k);
        B_[i] = a.ld(l, (M - k) & (M - 1));
      }
    }
  }
  __syncthreads();
  if (active) {
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      const int k = t + i * TPL;
      if (k > M / 2) continue;
      split_task<M, R, R2>(ao, l, k, A_[i], B_[i], twp[k], scale);
    }
  }
  __syncthreads();
}

// 128-point FFT (256-long lines): its last Stockham stage (radix 2, Ns = 64)
// fused with the even/odd split. Butterfly j (0..63) takes Z'[j] and
// W128^j Z'[j+64] and gives Z[j] = a + b, Z[j+64] = a - b. Split task k
// (0..64) needs Z[k] and Z[128-k], which come from butterflies k and 64-k
// (mod 64), so a thread that owns both does the stage and both tasks in
// registers: one shared-memory round trip less per transform. Thread t < 15
// owns butterflies t+1, 63-t (tasks t+1, 63-t) and t+17, 47-t (tasks t+17,
// 47-t); thread 15 owns 16, 48 (tasks 16, 48), 0 (tasks 0 and 64) and 32
// (task 32). All inputs are read before a block barrier, all outputs
// written after it (`ao` may alias `a`, also with a wider element type).
template <typename R, typename R2, class Acc, class AccO, class Scale>
__device__ __forceinline__ void dht128_tail(const Acc& a, const AccO& ao, const R2* tw3, const R2* twp, int l, int t,
                                            bool active, const Scale& scale) {
  constexpr int M = 128;
  int bj[4];
  if (t < 15) {
    bj[0] = t + 1;
    bj[1] = 63 - t;
    bj[2] = t + 17;
    bj[3] = 47 - t;
  } else {
    bj[0] = 16;
    bj[1] = 48;
    bj[2] = 0;
    bj[3] = 32;
  }
  R2 lo[4], hi[4];
  if (active) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const R2 x0 = a.ld(l, bj[q]);
      const R2 x1 = cmul(a.ld(l, bj[q] + 64), tw3[64 + bj[q]]);
      lo[q] = cadd(x0, x1);  // Z[bj]
      hi[q] = csub(x0, x1);  // Z[bj + 64]
    }
  }
  __syncthreads();
  if (active) {
    // pair (bj[0], bj[1] = 64 - bj[0]): tasks bj[0] and bj[1]
    split_task<M, R, R2>(ao, l, bj[0], lo[0], hi[1], twp[bj[0]], scale);
    split_task<M, R, R2>(ao, l, bj[1], lo[1], hi[0], twp[bj[1]], scale);
    if (t < 15) {
      split_task<M, R, R2>(ao, l, bj[2], lo[2], hi[3], twp[bj[2]], scale);
      split_task<M, R, R2>(ao, l, bj[3], lo[3], hi[2], twp[bj[3]], scale);
    } else {
      split_task<M, R, R2>(ao, l, 0, lo[2], lo[2], twp[0], scale);     // Z[0]
      split_task<M, R, R2>(ao, l, 64, hi[2], hi[2], twp[64], scale);   // Z[64], Z[128 - 64]
      split_task<M, R, R2>(ao, l, 32, lo[3], hi[3], twp[32], scale);   // Z[32], Z[96]
    }
  }
  __syncthreads();
}

template <int M, typename R, typename R2, class Acc, class Scale = NoScale>
__device__ __forceinline__ void dht_post(const Acc& a, const R2* twp, int l, int t, bool active,
                                         const Scale& scale = Scale()) {
  dht_post_to<M, R, R2>(a, a, twp, l, t, active, scale);
}

// Full in-place Hartley transform of the lines of `a` (pad: scratch for the
// first stage's output when USE_PAD). Thread `t` of line `l`, M/8 per line.
// The packed complex FFT stages of dht_lines (for M = 128 all but the last,
// which dht_tail_to fuses with the even/odd split).
template <int M, bool USE_PAD, typename R, class Acc, class P>
__device__ __forceinline__ void fft_stages(const Acc& a, const P& pad, const typename Cplx<R>::T* tw, int l, int t,
                                           bool active) {
  using R2 = typename Cplx<R>::T;
  using Pl = FFTPlan<M>;
  if constexpr (Pl::nstages == 1) {
    fft_stage<M, 8, 1, true, R2>(a, a, tw, l, t, active);
  } else if constexpr (USE_PAD) {
    fft_stage<M, 8, 1, false, R2>(a, pad, tw, l, t, active);
    fft_stage<M, Pl::radix(1), 8, false, R2>(pad, a, tw + Pl::tw_off(1), l, t, active);
    if constexpr (Pl::nstages == 3 && M != 128)
      fft_stage<M, Pl::radix(2), 64, true, R2>(a, a, tw + Pl::tw_off(2), l, t, active);
  } else {
    fft_stage<M, 8, 1, true, R2>(a, a, tw, l, t, active);
    fft_stage<M, Pl::radix(1), 8, true, R2>(a, a, tw + Pl::tw_off(1), l, t, active);
    if constexpr (Pl::nstages == 3 && M != 128)
      fft_stage<M, Pl::radix(2), 64, true, R2>(a, a, tw + Pl::tw_off(2), l, t, active);
  }
}

// 256-long lines with 8 threads per line (t = 0..7), two shared-memory round
// trips per transform instead of three:
//   A: radix-16 over m = t + 8 r (r < 16), outputs to 16 t + r (Stockham, Ns = 1);
//   B: radix-8 butterflies j (inputs Z'[j + 16 r] times W128^(r j), outputs
//      Z[j + 16 r]) fused with the even/odd split. Split task k needs Z[k] and
//      Z[128 - k]; Z[j + 16 r] pairs with Z[(16 - j) + 16 (7 - r)], so thread t
//      owns butterflies t and 16 - t (t = 0: 0 and 8, each its own partner)
//      and does their split tasks in registers.
// Meant for column tiles (ColLines), where stage A's 16-strided writes fall in
// different columns across a warp. `ao` may alias `a` (see dht_post_to).
// Stage A writes to `pa` and stage B reads from it (column tiles: `a` itself).
// PA_APART: `pa` shares no bytes with `a`, so stage A writes without waiting
// for every thread's reads (one block barrier less).
template <typename R, bool PA_APART = false, class Acc, class PAcc, class AccO, class Scale>
__device__ __forceinline__ void dht128_t8_to(const Acc& a, const PAcc& pa, const AccO& ao,
                                             const typename Cplx<R>::T* tw, int l, int t, bool active,
                                             const Scale& scale) {
  using R2 = typename Cplx<R>::T;
  using Pl = FFTPlan<128>;
  constexpr int M = 128;
  const R2* twB = tw + Pl::r16_off();
  const R2* twp = tw + Pl::post_off();
  R2 v[16];
  // stage A (in place: all reads, barrier, all writes)
  if (active) {
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = a.ld(l, t + 8 * r);
    DFT<16, R2>::run(v);
  }
  if constexpr (!PA_APART) __syncthreads();
  if (active) {
#pragma unroll
    for (int r = 0; r < 16; ++r) pa.st(l, 16 * t + r, v[r]);
  }
  __syncthreads();
  // stage B + split
  const int j0 = t == 0 ? 0 : t, j1 = t == 0 ? 8 : 16 - t;
  R2 z0[8], z1[8];
  if (active) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      z0[r] = pa.ld(l, j0 + 16 * r);
      z1[r] = pa.ld(l, j1 + 16 * r);
      if (r > 0) {
        z0[r] = cmul(z0[r], twB[16 * r + j0]);
        z1[r] = cmul(z1[r], twB[16 * r + j1]);
      }
    }
    DFT<8, R2>::run(z0);
    DFT<8, R2>::run(z1);
  }
  __syncthreads();
  if (active) {
    if (t == 0) {
      // butterfly 0: Z[16 r] pairs with Z[16 (8 - r)]; tasks 0, 16, 32, 48, 64
      split_task<M, R, R2>(ao, l, 0, z0[0], z0[0], twp[0], scale);
#pragma unroll
      for (int r = 1; r <= 4; ++r) split_task<M, R, R2>(ao, l, 16 * r, z0[r], z0[8 - r], twp[16 * r], scale);
      // butterfly 8: Z[8 + 16 r] pairs with Z[8 + 16 (7 - r)]; tasks 8, 24, 40, 56
#pragma unroll
      for (int r = 0; r < 4; ++r) split_task<M, R, R2>(ao, l, 8 + 16 * r, z1[r], z1[7 - r], twp[8 + 16 * r], scale);
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        split_task<M, R, R2>(ao, l, j0 + 16 * r, z0[r], z1[7 - r], twp[j0 + 16 * r], scale);
        split_task<M, R, R2>(ao, l, j1 + 16 * r, z1[r], z0[7 - r], twp[j1 + 16 * r], scale);
      }
    }
  }
  __syncthreads();
}

// The rest of the transform after fft_stages: for M = 128 the last Stockham
// stage fused with the even/odd split, otherwise the split alone; outputs to
// `ao` (may alias `a`).
template <int M, typename R, class Acc, class AccO, class Scale>
__device__ __forceinline__ void dht_tail_to(const Acc& a, const AccO& ao, const typename Cplx<R>::T* tw, int l, int t,
                                            bool active, const Scale& scale) {
  using R2 = typename Cplx<R>::T;
  using Pl = FFTPlan<M>;
  if constexpr (M == 128) {
    static_assert(Pl::nstages == 3 && Pl::radix(2) == 2, "the fused tail needs a final radix-2 stage");
    dht128_tail<R, R2>(a, ao, tw + Pl::tw_off(2), tw + Pl::post_off(), l, t, active, scale);
  } else {
    dht_post_to<M, R, R2>(a, ao, tw + Pl::post_off(), l, t, active, scale);
  }
}

template <int M, bool USE_PAD, typename R, class Acc, class P, class Scale = NoScale>
__device__ __forceinline__ void dht_lines(const Acc& a, const P& pad, const typename Cplx<R>::T* tw, int l, int t,
                                          bool active, const Scale& scale = Scale()) {
  fft_stages<M, USE_PAD, R>(a, pad, tw, l, t, active);
  dht_tail_to<M, R>(a, a, tw, l, t, active, scale);
}

template <typename R2>
__device__ __forceinline__ void load_table(R2* dst, const R2* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// x pass: LPC consecutive rows of length N = 2M per CTA (rows are contiguous
// in the [z][y][x] layout: row r is (y, z) = (r % ny, r / ny)). A producer
// computes the rows in shared memory from other fields, the rows are
// transformed, and a consumer stores them (one bulk store).

// Consumer: rows stored to an array (one bulk store).
template <typename R>
struct RowsToArray {
  R* out;
  __device__ R* dst(int row0, int N) const { return out + (size_t)row0 * N; }
};

// Output accessor of the last step of a correction solve's last x pass
// (k_dht_rows_addp_pipe): element n of line l is added to the shared-memory p
// row, minus the parity-class mean of p measured by the preceding residual
// pass (row r is (y, z) = (r & (ny-1), r >> log2ny); ny is a power of two).
struct AddToPRows {
  using elem = double;
  double* prow;
  const double* cm;  // the 8 class means (shared memory)
  int N, row0, log2ny;
  __device__ __forceinline__ void str(int l, int n, double v) const {
    const int r = row0 + l;
    const int cls = (n & 1) | ((r & 1) << 1) | (((r >> log2ny) & 1) << 2);
    double* q = prow + l * N + n;
    *q = *q + v - cm[cls];
  }
};

template <int M, typename R, class Prod, class Cons>
__global__ void __launch_bounds__(256) k_dht_rows(const Prod prod, const Cons cons, int nrows, int lpc,
                                                  const typename Cplx<R>::T* tw_g, int* err, const int* skip) {
  pdl_entry();
  using R2 = typename Cplx<R>::T;
  if (skip && *skip) return;
  constexpr int N = 2 * M, TPL = M / 8;
  constexpr int TL = FFTPlan<M>::rows_table_len();
  constexpr bool PAD = FFTPlan<M>::nstages > 1;
  constexpr int PPITCH = 2 * (M + M / 8);
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  R* rows = reinterpret_cast<R*>(smem_raw);  // lpc * N
  R* padb = rows + (size_t)lpc * N;          // lpc * PPITCH
  R2* tw = reinterpret_cast<R2*>(padb + (PAD ? (size_t)lpc * PPITCH : 0));
  const int row0 = blockIdx.x * lpc;
  const int nr = min(lpc, nrows - row0);
  if (nr <= 0) return;
  const uint32_t bytes = (uint32_t)((size_t)nr * N * sizeof(R));
  load_table(tw, tw_g, TL);
  prod.fill(rows, row0, nr, N);
  __syncthreads();
  const int l = threadIdx.x / TPL, t = threadIdx.x % TPL;
  const bool active = l < nr;
  RowLines<R> A{rows, N};
  RowLinesPad<R> P{padb, PPITCH};
  dht_lines<M, PAD, R>(A, P, tw, l, t, active);
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    bulk_store(cons.dst(row0, N), rows, bytes);
    bulk_commit();
    bulk_wait_all();
  }
}

// Pipelined x pass: persistent CTAs walk tiles of lpc consecutive rows
// (tile i of a CTA: rows (blockIdx.x + i gridDim.x) lpc ...) through NB
// shared-memory buffers. The 1-D bulk loads of the next NB-1 tiles and the
// bulk store of the previous tile overlap the transform of the current one;
// the twiddle table is loaded once per CTA. (The 8-thread plan of the column
// passes measured slower on rows: 16-strided stage-A writes need a padded
// buffer and fewer threads share a row tile.)
template <int M, typename R, int NB>
__global__ void __launch_bounds__(256, 2) k_dht_rows_pipe(const R* __restrict__ in, R* __restrict__ out, int nrows,
                                                          int lpc, const typename Cplx<R>::T* tw_g, int* err,
                                                          const int* skip) {
  pdl_entry();
  using R2 = typename Cplx<R>::T;
  static_assert(NB >= 2, "need at least two tile buffers");
  if (skip && *skip) return;
  constexpr int N = 2 * M, TPL = M / 8;
  constexpr int TL = FFTPlan<M>::rows_table_len();
  constexpr bool PAD = FFTPlan<M>::nstages > 1;
  constexpr int PPITCH = 2 * (M + M / 8);
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  R* bufs = reinterpret_cast<R*>(smem_raw);                 // NB * lpc * N
  R* padb = bufs + (size_t)NB * lpc * N;                     // lpc * PPITCH
  R2* tw = reinterpret_cast<R2*>(padb + (PAD ? (size_t)lpc * PPITCH : 0));
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + TL);
  const int tid = threadIdx.x;
  const int ntiles = (nrows + lpc - 1) / lpc;
  const int my = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0) {
    for (int b = 0; b < NB; ++b) mbar_init(&bar[b], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto rows_of = [&](int i, int& row0, int& nr) {
    row0 = (blockIdx.x + i * gridDim.x) * lpc;
    nr = min(lpc, nrows - row0);
  };
  auto issue = [&](int i) {
    int row0, nr;
    rows_of(i, row0, nr);
    const int b = i % NB;
    const uint32_t bytes = (uint32_t)((size_t)nr * N * sizeof(R));
    mbar_arrive_expect_tx(&bar[b], bytes);
    bulk_load(bufs + (size_t)b * lpc * N, in + (size_t)row0 * N, bytes, &bar[b]);
  };
  int issued = 0;
  if (tid == 0)
    for (; issued < min(NB - 1, my); ++issued) issue(issued);
  load_table(tw, tw_g, TL);
  __syncthreads();
  const int l = tid / TPL, t = tid % TPL;
  RowLinesPad<R> P{padb, PPITCH};
  bool ok = true;
  int done = 0;
  for (int i = 0; i < my; ++i) {
    // refill: tile i + NB - 1 goes into the buffer of tile i - 1, once its
    // store has read it
    if (tid == 0 && ok && issued < my) {
      bulk_wait_read<0>();
      issue(issued++);
    }
    int row0, nr;
    rows_of(i, row0, nr);
    const int b = i % NB;
    ok = __syncthreads_and(ok && mbar_wait(&bar[b], (i / NB) & 1, err));
    if (!ok) break;
    R* rows = bufs + (size_t)b * lpc * N;
    RowLines<R> A{rows, N};
    dht_lines<M, PAD, R>(A, P, tw, l, t, l < nr);
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      bulk_store(out + (size_t)row0 * N, rows, (uint32_t)((size_t)nr * N * sizeof(R)));
      bulk_commit();
    }
    done = i + 1;
  }
  if (tid == 0) {
    bulk_wait_all();
    // after a timed-out wait: bounded drain of the loads still in flight
    if (!ok)
      for (int r = done; r < issued; ++r) mbar_wait(&bar[r % NB], (r / NB) & 1, nullptr);
  }
}

// Pipelined last x pass of a correction solve (FP64): persistent CTAs walk
// tiles of lpc rows through NB buffer pairs, each pair holding the tile's
// transform rows and its p rows, both filled by 1-D bulk copies on one
// barrier. The inverse transform's last step adds into the p rows (AddToPRows:
// p += rows - class means of p) and one bulk store writes them back. The loads
// of the next NB-1 tiles and the store of the previous one overlap the
// transform of the current tile; the twiddle table and the class means are
// loaded once per CTA.
template <int M, int NB>
__global__ void __launch_bounds__(256, 1) k_dht_rows_addp_pipe(const double* __restrict__ in, double* p,
                                                               const double* cmean, int log2ny, int nrows, int lpc,
                                                               const double2* tw_g, int* err, const int* skip) {
  pdl_entry();
  static_assert(NB >= 2, "need at least two buffer pairs");
  if (skip && *skip) return;
  constexpr int N = 2 * M, TPL = M / 8;
  constexpr int TL = FFTPlan<M>::rows_table_len();
  constexpr bool PAD = FFTPlan<M>::nstages > 1;
  constexpr int PPITCH = 2 * (M + M / 8);
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  double* bufs = reinterpret_cast<double*>(smem_raw);  // NB * lpc * N transform rows
  double* pbufs = bufs + (size_t)NB * lpc * N;         // NB * lpc * N p rows
  double* padb = pbufs + (size_t)NB * lpc * N;         // lpc * PPITCH
  double2* tw = reinterpret_cast<double2*>(padb + (PAD ? (size_t)lpc * PPITCH : 0));
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + TL);
  double* cms = reinterpret_cast<double*>(bar + NB);   // the 8 class means
  const int tid = threadIdx.x;
  const int ntiles = (nrows + lpc - 1) / lpc;
  const int my = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0) {
    for (int b = 0; b < NB; ++b) mbar_init(&bar[b], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto rows_of = [&](int i, int& row0, int& nr) {
    row0 = (blockIdx.x + i * gridDim.x) * lpc;
    nr = min(lpc, nrows - row0);
  };
  auto issue = [&](int i) {
    int row0, nr;
    rows_of(i, row0, nr);
    const int b = i % NB;
    const uint32_t bytes = (uint32_t)((size_t)nr * N * sizeof(double));
    mbar_arrive_expect_tx(&bar[b], 2 * bytes);
    bulk_load(bufs + (size_t)b * lpc * N, in + (size_t)row0 * N, bytes, &bar[b]);
    bulk_load(pbufs + (size_t)b * lpc * N, p + (size_t)row0 * N, bytes, &bar[b]);
  };
  int issued = 0;
  if (tid == 0)
    for (; issued < min(NB - 1, my); ++issued) issue(issued);
  load_table(tw, tw_g, TL);
  if (tid < 8) cms[tid] = cmean[tid];
  __syncthreads();
  const int l = tid / TPL, t = tid % TPL;
  RowLinesPad<double> P{padb, PPITCH};
  bool ok = true;
  int done = 0;
  for (int i = 0; i < my; ++i) {
    // refill: tile i + NB - 1 goes into the buffer pair of tile i - 1, once
    // the store of its p rows has read them
    if (tid == 0 && ok && issued < my) {
      bulk_wait_read<0>();
      issue(issued++);
    }
    int row0, nr;
    rows_of(i, row0, nr);
    const int b = i % NB;
    ok = __syncthreads_and(ok && mbar_wait(&bar[b], (i / NB) & 1, err));
    if (!ok) break;
    RowLines<double> A{bufs + (size_t)b * lpc * N, N};
    double* prow = pbufs + (size_t)b * lpc * N;
    const bool active = l < nr;
    fft_stages<M, PAD, double>(A, P, tw, l, t, active);
    dht_tail_to<M, double>(A, AddToPRows{prow, cms, N, row0, log2ny}, tw, l, t, active, NoScale());
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      bulk_store(p + (size_t)row0 * N, prow, (uint32_t)((size_t)nr * N * sizeof(double)));
      bulk_commit();
    }
    done = i + 1;
  }
  if (tid == 0) {
    bulk_wait_all();
    // after a timed-out wait: bounded drain of the loads still in flight
    if (!ok)
      for (int r = done; r < issued; ++r) mbar_wait(&bar[r % NB], (r / NB) & 1, nullptr);
  }
}

// Spectral factor of PoissonSolverPeriodic::_solve (grid-consistent branch,
// source/poisson/PoissonSolverPeriodic.cpp:23-61): cx/cy/cz hold
// cos(4 pi k / N) evaluated on the host exactly as the reference does.
struct SpectralParams {
  const double* cx;
  const double* cy;  // cos(4 pi ky / ny) for the global ky
  const double* cz;
  double norm_factor;
  int nx, ny, nz;  // ny: the global line length in y
  int y0;          // global y index of the handle's first y (a slab of a decomposed grid; 0 otherwise)
};

// Scaler of the z pass: the factor of column (kx, ky) at z index k,
// nf / (2 (cos_x + cos_y + cos_z) - 6), zero on the 8 null modes (kx in
// {0, Nx/2}, ky in {0, Ny/2}, kz in {0, Nz/2}); the z indices 0 and Nz/2 are
// both handled by task k = 0. cz: cos_z[0..Nz/4] (the tasks' k range), staged
// in shared memory by the pass. SF = double divides exactly (the direct FP64
// solve). SF = float is the correction solve of the defect-correction loop:
// the denominator is still formed in FP64 (it cancels to 2 (1 - cos(4 pi/N))
// at the lowest modes), then the FP32 quotient scales the FP32 forward
// transform's output. A factor with relative error e changes each mode of the
// correction by the factor 1 + e, which leaves a residual of relative size e:
// the same order as the FP32 forward transform's own rounding.
template <typename SF>
struct ZColumnFactor {
  using type = SF;
  double cxy;  // cos_x[kx] + cos_y[ky]
  const double* cz;
  double nf;
  bool null_col;
  static constexpr bool kOn = true;
  __device__ __forceinline__ SF operator()(int k) const {
    if (k == 0 && null_col) return (SF)0;
    const double den = 2 * (cxy + cz[k]) - 6;
    if constexpr (sizeof(SF) == 4) return __fdividef((float)nf, (float)den);
    else return nf / den;
  }
};

template <typename SF>
__device__ __forceinline__ ZColumnFactor<SF> z_column_factor(const SpectralParams& sp, const double* cz, int kx,
                                                             int ky) {
  ZColumnFactor<SF> f;
  const int gy = sp.y0 + ky;
  f.cxy = __ldg(sp.cx + kx) + __ldg(sp.cy + gy);
  f.cz = cz;
  f.nf = sp.norm_factor;
  f.null_col = (kx == 0 || kx == sp.nx / 2) && (gy == 0 || gy == sp.ny / 2);
  return f;
}

// Pipelined y / z pass: persistent CTAs walk the tiles (W consecutive x
// columns by the whole line; tile t is x0 = (t % ntiles_x) W and the other
// coordinate t / ntiles_x) through NB shared-memory tile buffers. The TMA
// loads of the next NB-1 tiles and the store of the previous tile overlap the
// transform of the current one; the twiddle table is loaded once per CTA.
//
// RIN = float with R = double (z pass of the mixed-precision correction
// solve): the FP32 tile lands in the upper half of its FP64 buffer; the
// forward transform runs in FP32 on it (like the x and y forward passes) and
// its even/odd split writes the divided spectrum in FP64 over the whole
// buffer (all reads before a barrier, all writes after it); the inverse runs
// in FP64 and the tile is stored in FP64. tw_in_g: the FP32 table.
template <int M, typename R, int AXIS, bool DIVIDE, int W, int NB, typename RIN = R, bool T8 = false>
__global__ void __launch_bounds__(W * (T8 ? 8 : M / 8)) k_dht_cols_pipe(const __grid_constant__ CUtensorMap map_in,
                                                       const __grid_constant__ CUtensorMap map_out, int ntiles_x,
                                                       int ntiles, const typename Cplx<R>::T* tw_g,
                                                       const typename Cplx<RIN>::T* tw_in_g, SpectralParams sp,
                                                       int* err, const int* skip) {
  pdl_entry();
  using R2 = typename Cplx<R>::T;
  using RI2 = typename Cplx<RIN>::T;
  static_assert(NB >= 2, "need at least two tile buffers");
  static_assert(sizeof(RIN) <= sizeof(R), "input may only be narrower than the transform type");
  static_assert(!T8 || M == 128, "the 8-thread plan is for 256-long lines");
  if (skip && *skip) return;
  constexpr int N = 2 * M, TPL = T8 ? 8 : M / 8;
  constexpr int TL = FFTPlan<M>::table_len();
  constexpr bool WIDEN = sizeof(RIN) < sizeof(R);
  constexpr uint32_t TILE_BYTES = (uint32_t)(N * W * sizeof(RIN));
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  R* tiles = reinterpret_cast<R*>(smem_raw);  // [NB][N][W]
  R2* tw = reinterpret_cast<R2*>(tiles + (size_t)NB * N * W);
  RI2* tw_in = reinterpret_cast<RI2*>(tw + TL);  // (WIDEN only)
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw_in + (WIDEN ? TL : 0));
  double* czs = reinterpret_cast<double*>(bar + NB);  // cos_z[0..M/2] (DIVIDE)
  const int tid = threadIdx.x;
  const int my = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0) {
    for (int b = 0; b < NB; ++b) mbar_init(&bar[b], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto coords = [&](int i, int& x0, int& other) {
    const int t = blockIdx.x + i * gridDim.x;
    x0 = (t % ntiles_x) * W;
    other = t / ntiles_x;  // z for AXIS 1, y for AXIS 2
  };
  auto issue = [&](int i) {
    int x0, other;
    coords(i, x0, other);
    const int b = i % NB;
    mbar_arrive_expect_tx(&bar[b], TILE_BYTES);
    // widening: the narrow tile occupies the upper half of the buffer
    unsigned char* dst = reinterpret_cast<unsigned char*>(tiles + (size_t)b * N * W) +
                         (WIDEN ? (size_t)N * W * (sizeof(R) - sizeof(RIN)) : 0);
    tma_load_3d(dst, &map_in, x0, AXIS == 1 ? 0 : other, AXIS == 1 ? other : 0, &bar[b]);
  };
  int issued = 0;
  if (tid == 0)
    for (; issued < min(NB - 1, my); ++issued) issue(issued);
  load_table(tw, tw_g, TL);
  if constexpr (WIDEN) load_table(tw_in, tw_in_g, TL);
  if constexpr (DIVIDE)
    for (int i = tid; i <= M / 2; i += blockDim.x) czs[i] = sp.cz[i];
  __syncthreads();
  const int l = tid % W, t = tid / W;
  const bool active = t < TPL;
  bool ok = true;
  int done = 0;
  for (int i = 0; i < my; ++i) {
    // refill: tile i + NB - 1 goes into the buffer of tile i - 1, once the
    // store of tile i - 1 has read it
    if (tid == 0 && ok && issued < my) {
      bulk_wait_read<0>();
      issue(issued++);
    }
    const int b = i % NB;
    ok = __syncthreads_and(ok && mbar_wait(&bar[b], (i / NB) & 1, err));
    if (!ok) break;
    int x0, other;
    coords(i, x0, other);
    R* tile = tiles + (size_t)b * N * W;
    ColLines<R> A{tile, W};
    if constexpr (T8) {
      if constexpr (WIDEN) {
        ColLines<RIN> An{reinterpret_cast<RIN*>(reinterpret_cast<unsigned char*>(tile) +
                                                (size_t)N * W * (sizeof(R) - sizeof(RIN))),
                         W};
        // the lower part of the buffer is free until the widened output:
        // stage A of the narrow transform writes there
        ColLines<RIN> Lo{reinterpret_cast<RIN*>(tile), W};
        if constexpr (DIVIDE) {
          dht128_t8_to<RIN, true>(An, Lo, A, tw_in, l, t, active, z_column_factor<RIN>(sp, czs, x0 + l, other));
          dht128_t8_to<R>(A, A, A, tw, l, t, active, NoScale());
        } else {
          dht128_t8_to<RIN, true>(An, Lo, A, tw_in, l, t, active, NoScale());
        }
      } else if constexpr (DIVIDE) {
        dht128_t8_to<R>(A, A, A, tw, l, t, active, z_column_factor<double>(sp, czs, x0 + l, other));
        dht128_t8_to<R>(A, A, A, tw, l, t, active, NoScale());
      } else {
        dht128_t8_to<R>(A, A, A, tw, l, t, active, NoScale());
      }
    } else if constexpr (WIDEN) {
      ColLines<RIN> An{reinterpret_cast<RIN*>(reinterpret_cast<unsigned char*>(tile) +
                                              (size_t)N * W * (sizeof(R) - sizeof(RIN))),
                       W};
      fft_stages<M, false, RIN>(An, An, tw_in, l, t, active);
      if constexpr (DIVIDE) {
        dht_tail_to<M, RIN>(An, A, tw_in, l, t, active, z_column_factor<RIN>(sp, czs, x0 + l, other));
        dht_lines<M, false, R>(A, A, tw, l, t, active);
      } else {
        dht_tail_to<M, RIN>(An, A, tw_in, l, t, active, NoScale());
      }
    } else if constexpr (DIVIDE) {
      // forward, spectral divide fused into the even/odd split, inverse
      dht_lines<M, false, R>(A, A, tw, l, t, active, z_column_factor<double>(sp, czs, x0 + l, other));
      dht_lines<M, false, R>(A, A, tw, l, t, active);
    } else {
      dht_lines<M, false, R>(A, A, tw, l, t, active);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tma_store_3d(&map_out, x0, AXIS == 1 ? 0 : other, AXIS == 1 ? other : 0, tile);
      bulk_commit();
    }
    done = i + 1;
  }
  if (tid == 0) {
    bulk_wait_all();
    // after a timed-out wait: bounded drain of the loads still in flight
    if (!ok)
      for (int r = done; r < issued; ++r) mbar_wait(&bar[r % NB], (r / NB) & 1, nullptr);
  }
}

// Mixed-precision z pass of the correction solve (256-long lines, the 8-thread
// plan) with a narrow input ring: the FP32 input tiles (W columns by the whole
// z line) arrive by TMA in NBN narrow buffers and each tile is transformed in
// one FP64 buffer. Stage A of the FP32 forward transform reads the narrow tile
// and writes into the lower half of the FP64 buffer, so once the forward
// transform is done the narrow buffer takes the load of tile i + NBN while the
// FP64 inverse runs; the FP64 buffer is reused once the store of the previous
// tile has read it. Only the post-split and radix-16 twiddles of the 8-thread
// plan are staged. At W = 32, NBN = 1 a CTA needs 101 KB of shared memory
// (two CTAs per SM) and its tile rows are 128 B in FP32 and 256 B in FP64;
// the ring of two FP64 buffers at W = 16 needed 70 KB (three CTAs per SM) for
// 64-B and 128-B rows. Same arithmetic, in the same order, as
// k_dht_cols_pipe<128, double, 2, true, W, NB, float, true>.
template <int W, int NBN>
__global__ void __launch_bounds__(W * 8) k_dht_z_mixed(const __grid_constant__ CUtensorMap map_in,
                                                      const __grid_constant__ CUtensorMap map_out, int ntiles_x,
                                                      int ntiles, const double2* tw_g, const float2* tw_in_g,
                                                      SpectralParams sp, int* err, const int* skip) {
  pdl_entry();
  if (skip && *skip) return;
  using Pl = FFTPlan<128>;
  constexpr int M = 128, N = 2 * M;
  constexpr int T0 = Pl::post_off(), TN = Pl::table_len() - Pl::post_off();  // staged part of the tables
  constexpr uint32_t IN_BYTES = (uint32_t)(N * W * sizeof(float));
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw = smem_align128(smem_dyn);
  double* wide = reinterpret_cast<double*>(smem_raw);         // [N][W]
  float* narrow = reinterpret_cast<float*>(wide + N * W);      // [NBN][N][W]
  double2* tws = reinterpret_cast<double2*>(narrow + NBN * N * W);
  float2* tws_in = reinterpret_cast<float2*>(tws + TN);
  uint64_t* bar = reinterpret_cast<uint64_t*>(tws_in + TN);
  double* czs = reinterpret_cast<double*>(bar + NBN);  // cos_z[0..M/2]
  // the transforms index the tables from their start; entries below T0 are never read
  const double2* tw = tws - T0;
  const float2* tw_in = tws_in - T0;
  const int tid = threadIdx.x;
  const int my = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  if (tid == 0) {
    for (int b = 0; b < NBN; ++b) mbar_init(&bar[b], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto coords = [&](int i, int& x0, int& y) {
    const int t = blockIdx.x + i * gridDim.x;
    x0 = (t % ntiles_x) * W;
    y = t / ntiles_x;
  };
  auto issue = [&](int i) {
    int x0, y;
    coords(i, x0, y);
    const int b = i % NBN;
    mbar_arrive_expect_tx(&bar[b], IN_BYTES);
    tma_load_3d(narrow + (size_t)b * N * W, &map_in, x0, y, 0, &bar[b]);
  };
  int issued = 0;
  if (tid == 0)
    for (; issued < min(NBN, my); ++issued) issue(issued);
  load_table(tws, tw_g + T0, TN);
  load_table(tws_in, tw_in_g + T0, TN);
  for (int i = tid; i <= M / 2; i += blockDim.x) czs[i] = sp.cz[i];
  __syncthreads();
  const int l = tid % W, t = tid / W;
  bool ok = true;
  int done = 0;
  for (int i = 0; i < my; ++i) {
    // the store of tile i - 1 must have read the FP64 buffer before stage A writes it
    if (tid == 0 && i > 0) bulk_wait_read<0>();
    const int b = i % NBN;
    ok = __syncthreads_and(ok && mbar_wait(&bar[b], (i / NBN) & 1, err));
    if (!ok) break;
    int x0, y;
    coords(i, x0, y);
    ColLines<float> An{narrow + (size_t)b * N * W, W};
    ColLines<float> Lo{reinterpret_cast<float*>(wide), W};
    ColLines<double> A{wide, W};
    dht128_t8_to<float, true>(An, Lo, A, tw_in, l, t, true, z_column_factor<float>(sp, czs, x0 + l, y));
    // every read of the narrow tile came before the barriers of the forward transform
    if (tid == 0 && issued < my) issue(issued++);
    dht128_t8_to<double>(A, A, A, tw, l, t, true, NoScale());
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tma_store_3d(&map_out, x0, y, 0, wide);
      bulk_commit();
    }
    done = i + 1;
  }
  if (tid == 0) {
    bulk_wait_all();
    // after a timed-out wait: bounded drain of the loads still in flight
    if (!ok)
      for (int r = done; r < issued; ++r) mbar_wait(&bar[r % NBN], (r / NBN) & 1, nullptr);
  }
}

}  // namespace cup
