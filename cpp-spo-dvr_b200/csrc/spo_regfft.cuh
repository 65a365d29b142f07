// Register-resident DFTs with compile-time sizes, and the two-level FFT passes built on them.
//
// A DFT of N = P Q values held in one thread's registers is split recursively (Cooley-Tukey,
// decimation in time): P sub-DFTs of length Q over x[p + P q], twiddles w_N^(p k1), then Q DFTs of
// length P. The base radices are 2, 4 and the odd primes 3, 5, 7, 11 (the factors of the reference's
// FFT sizes, src/fft/fft_sizes.cpp:9-34). Every index and every twiddle is a compile-time constant:
// the roots of unity are template constants evaluated by the compiler from cos/sin written here (a
// Taylor polynomial on |r| <= pi/4 after an exact quadrant reduction), so the unrolled butterflies
// are plain FMAs with immediate operands.
#pragma once

#include <type_traits>
#include <utility>

#include "spo_kernels.cuh"

namespace spo {

// ---------------------------------------------------------------------------------------------
// Compile-time roots of unity
// ---------------------------------------------------------------------------------------------
constexpr double kHalfPi = 1.57079632679489661923132169163975144;

// sin and cos of |r| <= pi/4 by their Taylor series (Horner form, terms to r^25 / 25!, below 1e-22).
constexpr double taylor_sin(double r) {
  const double r2 = r * r;
  double s = 0.0;
  for (int n = 12; n >= 1; --n) s = (1.0 - s * r2 / ((2.0 * n) * (2.0 * n + 1.0)));
  return r * s;
}
constexpr double taylor_cos(double r) {
  const double r2 = r * r;
  double s = 0.0;
  for (int n = 12; n >= 1; --n) s = (1.0 - s * r2 / ((2.0 * n - 1.0) * (2.0 * n)));
  return s;
}
// cos and sin of 2 pi k / n: q = the nearest quarter turn, r = 2 pi k / n - q pi / 2 computed from the
// exact integer 4k - q n, then the quarter turns applied exactly.
constexpr long quarter_of(long k, long n) { return (8 * k + n) / (2 * n); }
constexpr double reduced_angle(long k, long n) {
  return kHalfPi * static_cast<double>(4 * k - quarter_of(k, n) * n) / static_cast<double>(n);
}
constexpr double root_cos(long k, long n) {
  k = ((k % n) + n) % n;
  const double r = reduced_angle(k, n);
  switch (quarter_of(k, n) & 3) {
    case 0: return taylor_cos(r);
    case 1: return -taylor_sin(r);
    case 2: return -taylor_cos(r);
    default: return taylor_sin(r);
  }
}
constexpr double root_sin(long k, long n) {
  k = ((k % n) + n) % n;
  const double r = reduced_angle(k, n);
  switch (quarter_of(k, n) & 3) {
    case 0: return taylor_sin(r);
    case 1: return taylor_cos(r);
    case 2: return -taylor_sin(r);
    default: return -taylor_cos(r);
  }
}

// exp(S 2 pi i K / N) as a compile-time constant pair.
template <long K, long N, int S>
struct Root {
  static constexpr double re = root_cos(K, N);
  static constexpr double im = S * root_sin(K, N);
};

// The compile-time value of a static_for index.
#define SPO_CV(i) decltype(i)::value

template <int B, int E, typename F>
SPO_HD void static_for(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    static_for<B + 1, E>(f);
  }
}

template <typename V, long K, long N, int S>
SPO_HD V twiddle_mul(V a) {
  constexpr long k = ((K % N) + N) % N;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (4 * k == N) {  // S i
    return cimul(a, S);
  } else if constexpr (2 * k == N) {
    return cmake<V>(-a.x, -a.y);
  } else if constexpr (4 * k == 3 * N) {  // -S i
    return cimul(a, -S);
  } else {
    using R = decltype(V::x);
    constexpr R c = static_cast<R>(Root<k, N, S>::re);
    constexpr R s = static_cast<R>(Root<k, N, S>::im);
    if constexpr (sizeof(R) == 4) {  // mixed form: the root as c + cl, s + sl (see cmul2, cmul_comp)
      constexpr R cl = static_cast<R>(Root<k, N, S>::re - static_cast<double>(c));
      constexpr R sl = static_cast<R>(Root<k, N, S>::im - static_cast<double>(s));
      if constexpr ((N & (N - 1)) != 0) return cmul_comp(a, cmake<V>(c, s), cmake<V>(cl, sl));
      else return cmul2(a, cmake<V>(c, s), cmake<V>(cl, sl));
    } else {
      return cmake<V>(a.x * c - a.y * s, a.x * s + a.y * c);
    }
  }
}

// A runtime twiddle of a length-N transform: cmul_comp for lengths with an odd factor, else cmul2.
template <int N, typename V>
SPO_HD V tw_mul(V a, V w, V wl) {
  if constexpr ((N & (N - 1)) != 0) return cmul_comp(a, w, wl);
  else return cmul2(a, w, wl);
}

// ---------------------------------------------------------------------------------------------
// Register DFT, in place, natural order in and out: x[k] <- sum_n x[n] exp(S 2 pi i n k / N)
// ---------------------------------------------------------------------------------------------
constexpr int first_factor(int n) {
  if (n % 4 == 0 && n != 4) return 4;
  for (int p : {2, 3, 5, 7, 11})
    if (n % p == 0) return p;
  return n;
}
constexpr bool supported_size(int n) {
  while (n % 2 == 0) n /= 2;
  for (int p : {3, 5, 7, 11})
    while (n % p == 0) n /= p;
  return n == 1;
}

template <int N, int S, typename V>
SPO_HD void rdft(V (&x)[N]) {
  static_assert(supported_size(N), "register DFT sizes are products of 2, 3, 5, 7, 11");
  if constexpr (N == 1) {
  } else if constexpr (N == 2) {
    const V a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (N == 4) {
    const V s02 = cadd(x[0], x[2]), d02 = csub(x[0], x[2]);
    const V s13 = cadd(x[1], x[3]), d13 = csub(x[1], x[3]);
    const V jd = cimul(d13, S);
    x[0] = cadd(s02, s13);
    x[1] = cadd(d02, jd);
    x[2] = csub(s02, s13);
    x[3] = csub(d02, jd);
  } else if constexpr (N == 3 || N == 5 || N == 7 || N == 11) {
    // Odd prime: pairs (t, N - t) share the real part of the root and have opposite imaginary parts.
    // Mixed form: radix 3 (one term per output pair) holds its root as two FP32 values (see cmul2) and adds
    // the small part's product first; radices 5, 7 and 11 sum each output pair in FP64 from the FP32 sums and
    // differences and round once. With the roots rounded to FP32, a forward-inverse pass with a phase
    // between them drifts the norm by ~2e-8 (radix 3); with exact roots but partial sums rounded in FP32,
    // by ~7e-9 (radix 5) and ~1e-8 (radix 7), the same sign every pass.
    using R = decltype(V::x);
    constexpr int H = N / 2;
    using A = std::conditional_t<sizeof(R) == 4 && H >= 2, double, R>;  // accumulation type
    V s[H + 1], d[H + 1];
    static_for<1, H + 1>([&](auto t) {
      s[t] = cadd(x[t], x[N - t]);
      d[t] = csub(x[t], x[N - t]);
    });
    V out[N];
    V o0 = x[0];
    static_for<1, H + 1>([&](auto t) { o0 = cadd(o0, s[t]); });
    out[0] = o0;
    static_for<1, H + 1>([&](auto q) {
      A rex = x[0].x, rey = x[0].y, ir = 0, ii = 0;
      static_for<1, H + 1>([&](auto t) {
        constexpr long tq = static_cast<long>(SPO_CV(t)) * SPO_CV(q) % N;
        constexpr A c = static_cast<A>(Root<tq, N, S>::re);
        constexpr A sn = static_cast<A>(Root<tq, N, S>::im);
        if constexpr (sizeof(A) == 4) {  // mixed form, radix 3
          constexpr A cl = static_cast<A>(Root<tq, N, S>::re - static_cast<double>(c));
          constexpr A sl = static_cast<A>(Root<tq, N, S>::im - static_cast<double>(sn));
          rex = fmaf(c, s[t].x, fmaf(cl, s[t].x, rex));
          rey = fmaf(c, s[t].y, fmaf(cl, s[t].y, rey));
          ir = fmaf(sn, d[t].x, fmaf(sl, d[t].x, ir));
          ii = fmaf(sn, d[t].y, fmaf(sl, d[t].y, ii));
        } else {
          rex += c * static_cast<A>(s[t].x);
          rey += c * static_cast<A>(s[t].y);
          ir += sn * static_cast<A>(d[t].x);
          ii += sn * static_cast<A>(d[t].y);
        }
      });
      out[q] = cmake<V>(static_cast<R>(rex - ii), static_cast<R>(rey + ir));  // re + i * sum Im(w) d
      out[N - q] = cmake<V>(static_cast<R>(rex + ii), static_cast<R>(rey - ir));
    });
    static_for<0, N>([&](auto t) { x[t] = out[t]; });
  } else {
    constexpr int P = first_factor(N);
    constexpr int Q = N / P;
    V y[N];
    static_for<0, P>([&](auto p) {
      V sub[Q];
      static_for<0, Q>([&](auto q) { sub[q] = x[p + P * q]; });
      rdft<Q, S>(sub);
      static_for<0, Q>([&](auto k1) {
        y[p * Q + k1] = twiddle_mul<V, static_cast<long>(SPO_CV(p)) * SPO_CV(k1), N, S>(sub[k1]);
      });
    });
    static_for<0, Q>([&](auto k1) {
      V t[P];
      static_for<0, P>([&](auto p) { t[p] = y[p * Q + k1]; });
      rdft<P, S>(t);
      static_for<0, P>([&](auto k2) { x[k1 + Q * k2] = t[k2]; });
    });
  }
}

// ---------------------------------------------------------------------------------------------
// Two-level axis pass: FFT along an axis of length N = N1 N2 of an array (outer, N, inner), for TB
// consecutive inner elements per block; forward, times a factor f[k], inverse (the kinetic step
// exp(-i T dt) of one coordinate, with the FFT scales folded into f).
//   forward:  thread (b, n2) loads x[n2 + N2 n1] (n1 < N1) from global memory, DFT_N1 in registers,
//             times w_N^(n2 k1), into shared memory Y[n2][k1][b]; thread (b, k1) loads Y[.][k1][b],
//             DFT_N2: X[k1 + N1 k2].
//   factor:   X[k] *= f[k] in the same registers.
//   inverse:  the same two levels backwards (IDFT_N2, conjugate twiddle, shared memory, IDFT_N1),
//             stored straight to global memory.
// One shared-memory round trip per direction; each thread reads and writes only its own Y entries
// between the two halves, so one buffer serves both.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct Axis2Args {
  Vec<T>* data;
  long long inner;
  const Vec<T>* factor;  // N values, by k
  const Vec<T>* tw;      // N values: exp(-2 pi i j / N)
  int tile;              // launch choice: batch lanes per block (8, 16 or 32; 0: the default) for lines of
                         // more than 8 sub-rows
  // Lane windows (all zero: every lane of [outer][N][inner]). Otherwise block x serves lanes
  //   (x / blocks_per_group) * group_stride + lane_offset + (x % blocks_per_group) * TB + b,  b < TB,
  // of which those with (x % blocks_per_group) * TB + b < window exist; the line's points are line_stride
  // apart and block y's lines start y * outer_stride further.
  int blocks_per_group;
  long long group_stride, lane_offset, window, line_stride, outer_stride;
  long long groups;  // host side: lane groups per line set (the launch has groups * blocks_per_group blocks)
  int persistent;    // launch choice: the persistent form (axis2p_kernel) for whole passes
  int balanced;      // launch choice: the balanced form (axis2b_kernel, N2 = 2 N1) for whole passes
  // The factors in the prime-factor order (axis2pfa_kernel): factor_pfa[k1 + N1 k2] = factor[k(k1, k2)];
  // null: the two-level kernels with twiddles.
  const Vec<T>* factor_pfa;
};

// Dynamic shared memory: (N TB + 2 N) values (axis2_smem).
// Mixed form with at most 8 sub-rows: registers capped for SPO_AXIS2_SM_THREADS resident threads per SM
// (default 1536: r = 48 = 6 x 8 at 40 registers, six blocks of 256 threads instead of five, took 1.23 ->
// 1.12 ms on configuration 3).
#ifndef SPO_AXIS2_SM_THREADS
#define SPO_AXIS2_SM_THREADS 1536
#endif
template <typename T, int N1, int N2, int TB>
__global__ void __launch_bounds__(TB*(N1 > N2 ? N1 : N2), sizeof(T) == 4 && (N1 > N2 ? N1 : N2) <= 8 ? SPO_AXIS2_SM_THREADS / (TB*(N1 > N2 ? N1 : N2)) : 1) axis2_kernel(Axis2Args<T> a) {
  using V = Vec<T>;
  constexpr int N = N1 * N2;
  constexpr int NS = N1 > N2 ? N1 : N2;
  constexpr int kParts = sizeof(T) == 4 ? 2 : 1;         // twiddles: value (then low part)
  constexpr int kFParts = sizeof(T) == 4 ? kFactorParts : 1;  // factors: see fmul_t
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* Y = reinterpret_cast<V*>(smem_raw);
  V* f = Y + N * TB;       // N factors (the mixed form's parts, see fmul_t)
  V* tw = f + kFParts * N;  // N twiddles (then N low parts)
  const int b = threadIdx.x % TB;
  const int s = threadIdx.x / TB;
  long long base, stride;
  bool lane_ok;
  if (a.blocks_per_group == 0) {
    const long long i0 = static_cast<long long>(blockIdx.x) * TB;
    base = static_cast<long long>(blockIdx.y) * N * a.inner + i0 + b;
    stride = a.inner;
    lane_ok = i0 + b < a.inner;
  } else {
    const int grp = blockIdx.x / a.blocks_per_group;
    const long long in_group = static_cast<long long>(blockIdx.x - grp * a.blocks_per_group) * TB + b;
    base = static_cast<long long>(blockIdx.y) * a.outer_stride + grp * a.group_stride + a.lane_offset + in_group;
    stride = a.line_stride;
    lane_ok = in_group < a.window;
  }
  for (int k = threadIdx.x; k < kFParts * N; k += TB * NS) f[k] = a.factor[k];
  for (int k = threadIdx.x; k < kParts * N; k += TB * NS) tw[k] = a.tw[k];
  __syncthreads();
  // forward, level 1
  if (s < N2) {
    const int n2 = s;
    V x[N1];
    static_for<0, N1>([&](auto n1) {
      x[n1] = lane_ok ? a.data[base + static_cast<long long>(n2 + N2 * n1) * stride] : cmake<V>(0, 0);
    });
    rdft<N1, -1>(x);
    static_for<0, N1>([&](auto k1) { Y[(n2 * N1 + k1) * TB + b] = k1 == 0 ? x[k1] : tw_mul<N>(x[k1], tw[n2 * k1], lo_part(tw, N, n2 * k1)); });
  }
  __syncthreads();
  // forward level 2, factor, inverse level 2
  if (s < N1) {
    const int k1 = s;
    V y[N2];
    static_for<0, N2>([&](auto n2) { y[n2] = Y[(n2 * N1 + k1) * TB + b]; });
    rdft<N2, -1>(y);
    static_for<0, N2>([&](auto k2) { y[k2] = fmul_t(y[k2], f, N, k1 + N1 * k2); });
    rdft<N2, +1>(y);
    static_for<0, N2>([&](auto n2) {
      Y[(n2 * N1 + k1) * TB + b] = n2 == 0 ? y[n2] : tw_mul<N>(y[n2], cconj(tw[n2 * k1]), cconj(lo_part(tw, N, n2 * k1)));
    });
  }
  __syncthreads();
  // inverse level 1, store
  if (s < N2 && lane_ok) {
    const int n2 = s;
    V x[N1];
    static_for<0, N1>([&](auto k1) { x[k1] = Y[(n2 * N1 + k1) * TB + b]; });
    rdft<N1, +1>(x);
    static_for<0, N1>([&](auto n1) { a.data[base + static_cast<long long>(n2 + N2 * n1) * stride] = x[n1]; });
  }
}

}  // namespace spo

namespace spo {

// ---------------------------------------------------------------------------------------------
// xy pass with register DFTs: exp(-i T_xy dt) at one (Z, r) point for TB rotational states
// (src/propagation/kinetic_operators.cpp:134-172), the gas-phase potential step fused for
// Z >= zasymp (potential_operator.cpp:104-112).
//   y forward:  thread (b, ix) loads psi[ix, 0..NY) (times the momentum shift), DFT_NY, -> S[ix][ky][b]
//   x:          thread (b, ky) loads S[0..NX)[ky][b], DFT_NX, times the factor, IDFT_NX, back in place
//   y inverse:  thread (b, ix) loads S[ix][0..NY)[b], IDFT_NY, shift back, (gas W), stores psi.
// ---------------------------------------------------------------------------------------------
template <typename T, int NX, int NY, int TB>
__global__ void __launch_bounds__(TB*(NX > NY ? NX : NY)) xy2_kernel(XyArgs<T> a) {
  using V = Vec<T>;
  constexpr int NXY = NX * NY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kFParts = sizeof(T) == 4 ? kFactorParts : 1;  // the mixed form's factor parts (fmul_t)
  V* S = reinterpret_cast<V*>(smem_raw);  // NXY * TB
  V* f = S + NXY * TB;                     // NXY factors (the mixed form's parts)
  const int b = threadIdx.x % TB;
  const int s = threadIdx.x / TB;
  const long long izr = a.izr_offset + blockIdx.y;
  const int irot = blockIdx.x * TB + b;
  const bool lane_ok = irot < a.n_rot;
  const long long col0 = izr * NXY;
  for (int k = threadIdx.x; k < kFParts * NXY; k += blockDim.x) f[k] = a.factor[k];
  if (s < NX) {
    const int ix = s;
    V x[NY];
    static_for<0, NY>([&](auto iy) {
      V v = cmake<V>(0, 0);
      if (lane_ok) {
        v = a.psi[(col0 + ix * NY + iy) * a.n_rot + irot];
        if (a.shift_f) v = fmul_t(v, a.shift_f, NXY, ix * NY + iy);
      }
      x[iy] = v;
    });
    rdft<NY, -1>(x);
    static_for<0, NY>([&](auto ky) { S[(ix * NY + ky) * TB + b] = x[ky]; });
  }
  __syncthreads();
  if (s < NY) {
    const int ky = s;
    V x[NX];
    static_for<0, NX>([&](auto ix) { x[ix] = S[(ix * NY + ky) * TB + b]; });
    rdft<NX, -1>(x);
    static_for<0, NX>([&](auto kx) { x[kx] = fmul_t(x[kx], f, NXY, kx * NY + ky); });
    rdft<NX, +1>(x);
    static_for<0, NX>([&](auto ix) { S[(ix * NY + ky) * TB + b] = x[ix]; });
  }
  __syncthreads();
  if (s < NX && lane_ok) {
    const int ix = s;
    V x[NY];
    static_for<0, NY>([&](auto ky) { x[ky] = S[(ix * NY + ky) * TB + b]; });
    rdft<NY, +1>(x);
    const bool gas = a.apply_gas && izr >= a.izr_gas_first;
    const int ir = static_cast<int>(izr % a.nr);
    const long long n_gas = static_cast<long long>(a.nr) * a.n_rot, k_gas = ir * a.n_rot + irot;
    const T oz = gas ? a.opt_z[izr / a.nr] : T(1);
    static_for<0, NY>([&](auto iy) {
      V v = x[iy];
      if (a.shift_b) v = fmul_t(v, a.shift_b, NXY, ix * NY + iy);
      if (gas) v = cscale(fmul_t(v, a.gas_step, n_gas, k_gas), oz);
      a.psi[(col0 + ix * NY + iy) * a.n_rot + irot] = v;
    });
  }
}

// ---------------------------------------------------------------------------------------------
// Potential step of the interaction region with register phi transforms: one (Z, r) point per
// block, CB (x, y) columns per chunk, one thread per (column, theta) line.
//   load:     the CB columns (absorption, rot(dt/2), the specular wave into the initial channel)
//             into shared memory F[c][irot];
//   forward:  thread (c, theta) forms its line's phi slots by the theta contraction of every mJ block
//             straight into registers (slot p of mJ = p or p - NPHI), DFT_NPHI (sign +1);
//   exp(iA):  times exp(i A) of the column's representative at the mapped phi;
//   back:     IDFT_NPHI (sign -1), the line into shared memory D[c][theta][p];
//   transpose sums: thread j takes rotational states irot = j, j + blockDim.x, ... and sums over
//             theta for all CB columns at once (one matrix element reused CB times), times rot(dt/2);
//   projection: the initial channel of every column of the point is kept and projected onto the
//             specular grid at the end in a fixed order (src/propagation/potential_operator.cpp:129-135).
// The matrix is read as legendre (block, theta, J) from shared memory by the transposed sums and as
// legendre_t (block, J, theta) through the read-only cache by the forward sums.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct Pot2Args {
  PotArgs<T> p;
  const T* legendre_t;  // (block, J, theta)
  int cb;
  int identity_maps;    // no symmetry: representative = ixy and phi map = identity
  // Slot-major forms for the chunked kernel: phi slot p holds mJ = p or p - nphi; its FBR states are
  // slot_first[p] .. + slot_nj[p] (slot_nj = 0 for slots without basis functions); jp = max slot_nj.
  const int* slot_first;
  const int* slot_nj;
  const T* legendre_slot;  // (p, j, theta), zero for j >= slot_nj[p]
  int jp;
};

template <typename T, int NPHI, int CB>
__global__ void __launch_bounds__(128) potential2_kernel(Pot2Args<T> args) {
  using V = Vec<T>;
  const PotArgs<T>& a = args.p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n_rot = a.n_rot, nt = a.n_theta;
  constexpr int LD = NPHI + 1;
  V* F = reinterpret_cast<V*>(smem_raw);  // CB * n_rot
  V* D = F + CB * n_rot;                  // CB * nt * LD
  V* i0buf = D + CB * nt * LD;            // n_xy
  V* red = i0buf + a.n_xy;                // 32
  T* leg = reinterpret_cast<T*>(red + 32);  // nt * n_rot, (block, theta, J) (then, mixed form, their low parts)
  const long long n_leg = static_cast<long long>(nt) * n_rot;
  const int izr = blockIdx.x;
  const int ir = izr % a.nr;
  const int iz = izr / a.nr;
  const int i0 = a.initial_channel;
  const int mj_max = a.mj_max;
  for (int k = threadIdx.x; k < (sizeof(T) == 4 ? 2 : 1) * nt * n_rot; k += blockDim.x) leg[k] = a.legendre[k];
  const T oz = a.opt_z[iz];
  const V incoming = a.chi[ir + a.nr * iz];
  const long long n_scale = static_cast<long long>(a.nr) * n_rot;  // entries of the scaling tables
  const long long col_base = static_cast<long long>(izr) * a.n_xy;
  const long long e_base = static_cast<long long>(izr) * a.n_rep * nt * NPHI;
  const int line_c = threadIdx.x / nt;  // this thread's line: column line_c, theta line_t
  const int line_t = threadIdx.x % nt;
  __syncthreads();

  for (int c0 = 0; c0 < a.n_xy; c0 += CB) {
    const int ncol = min(CB, a.n_xy - c0);
    for (int e = threadIdx.x; e < ncol * n_rot; e += blockDim.x) {
      const int c = e / n_rot, irot = e - c * n_rot;
      const int ixy = c0 + c;
      V v = a.psi[(col_base + ixy) * n_rot + irot];
      v = cscale(fmul_t(v, a.before, n_scale, ir * n_rot + irot), oz);
      if (irot == i0) v = cadd(v, fmul_t(cmul_t(incoming, a.sp2sc, a.n_xy, ixy), a.rot_half, n_scale, ir * n_rot + i0));
      F[c * n_rot + irot] = v;
    }
    __syncthreads();
    if (line_c < ncol) {
      const int c = line_c, t = line_t;
      const int ixy = c0 + c;
      const V* f = F + c * n_rot;
      V x[NPHI];
      static_for<0, NPHI>([&](auto p) {
        constexpr int P = SPO_CV(p);
        const int m = P <= mj_max ? P : (P >= NPHI - mj_max ? P - NPHI : 1 << 20);
        Acc<V> s = acc_zero();
        if (m != (1 << 20)) {
          const int blk = mj_max + m;
          const int nj = a.block_size[blk];
          const int first = a.block_first[blk];
          const long long m0 = a.block_offset[blk] + t;  // (J, theta) within the block
          for (int j = 0; j < nj; ++j) {
            const long long k = m0 + j * nt;
            s = acc_add(s, f[first + j], __ldg(args.legendre_t + k), lo_real(args.legendre_t, n_leg, k));
          }
        }
        x[P] = acc_out<V>(s);
      });
      rdft<NPHI, +1>(x);
      if (args.identity_maps) {
        const long long e0 = e_base + (static_cast<long long>(ixy) * nt + t) * NPHI;
        static_for<0, NPHI>([&](auto p) { x[p] = exp_mul(x[p], __ldg(a.expia + e0 + p), a.exp_mod, e0 + p); });
      } else {
        const long long e0 = e_base + (static_cast<long long>(a.rep_of[ixy]) * nt + t) * NPHI;
        const int* map = a.phi_map + ixy * NPHI;
        static_for<0, NPHI>([&](auto p) {
          const long long ei = e0 + __ldg(map + p);
          x[p] = exp_mul(x[p], __ldg(a.expia + ei), a.exp_mod, ei);
        });
      }
      rdft<NPHI, -1>(x);
      static_for<0, NPHI>([&](auto p) { D[(c * nt + t) * LD + p] = x[p]; });
    }
    __syncthreads();
    for (int irot = threadIdx.x; irot < n_rot; irot += blockDim.x) {
      const int blk = a.irot_block[irot];
      const int nj = a.block_size[blk];
      const int jj = irot - a.block_first[blk];
      const int slot = a.block_slot[blk];
      const long long c0l = a.block_offset[blk] + jj;
      Acc<V> acc[CB];
#pragma unroll
      for (int c = 0; c < CB; ++c) acc[c] = acc_zero();
      for (int t = 0; t < nt; ++t) {
        const T w = leg[c0l + t * nj], wl = lo_real(leg, n_leg, c0l + t * nj);
        const V* d = D + t * LD + slot;
#pragma unroll
        for (int c = 0; c < CB; ++c) acc[c] = acc_add(acc[c], d[c * nt * LD], w, wl);
      }
#pragma unroll
      for (int c = 0; c < CB; ++c) {
        if (c < ncol) {
          const V s = fmul_t(acc_out<V>(acc[c]), a.rot_half, n_scale, ir * n_rot + irot);
          if (irot == i0) i0buf[c0 + c] = s;
          else a.psi[(col_base + c0 + c) * n_rot + irot] = s;
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < 32) {
    V s = cmake<V>(0, 0);
    for (int ixy = threadIdx.x; ixy < a.n_xy; ixy += 32) s = cadd(s, cmul_t(i0buf[ixy], a.sc2sp, a.n_xy, ixy));
    red[threadIdx.x] = s;
    __syncwarp();
    if (threadIdx.x == 0) {
      V p = cmake<V>(0, 0);
      for (int k = 0; k < 32; ++k) p = cadd(p, red[k]);
      red[0] = p;
      a.chi[ir + a.nr * iz] = p;
    }
  }
  __syncthreads();
  const V proj = red[0];
  for (int ixy = threadIdx.x; ixy < a.n_xy; ixy += blockDim.x)
    a.psi[(col_base + ixy) * n_rot + i0] = csub(i0buf[ixy], cmul_t(proj, a.sp2sc, a.n_xy, ixy));
}

}  // namespace spo

namespace spo {

// ---------------------------------------------------------------------------------------------
// Potential step of the interaction region, one block per (Z, r) point and chunk of CB (x, y)
// columns (grid: chunks x points), one thread per (column, theta) line, no loop over chunks:
//   load:    the chunk's columns (absorption, rot(dt/2), the specular wave into the initial channel),
//            gathered slot-major into shared memory F[c][p][j]: phi slot p of mJ, its j-th FBR state,
//            zero-padded to the longest mJ block (rows padded by 2 values against bank conflicts);
//   forward: thread (c, theta) forms all NPHI phi slots at once, j by j, as NPHI independent FMA chains
//            with the slot-major matrix (p, j, theta) through the read-only cache; DFT_NPHI (sign +1),
//            times exp(i A) at the mapped phi, IDFT_NPHI (sign -1), into D[c][theta][p] (D reuses F);
//   back:    thread j takes irot = j, j + blockDim.x, ...: theta sums for all CB columns with each matrix
//            element loaded once, times rot(dt/2), stored;
//   projection: projection_finalize_kernel, launched after this kernel, sums scattering_to_specular
//            times the initial channel over all (x, y) columns of each point in column order
//            (src/propagation/potential_operator.cpp:129-135) and subtracts the projection, so the
//            result does not depend on the chunking.
// ---------------------------------------------------------------------------------------------
template <typename T, int NPHI, int CB>
__global__ void __launch_bounds__(CB * 16) potential3_kernel(Pot2Args<T> args) {
  using V = Vec<T>;
  const PotArgs<T>& a = args.p;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n_rot = a.n_rot, nt = a.n_theta, jp = args.jp;
  constexpr int LD = NPHI + 1;
  const int FS = NPHI * jp + 2;                   // slot-major column stride, padded against bank conflicts
  V* F = reinterpret_cast<V*>(smem_raw);          // CB * FS: F[c][p][j]
  V* D = F;                                       // CB * nt * LD, after F is consumed
  const int izr = blockIdx.y;
  const int ir = izr % a.nr;
  const int iz = izr / a.nr;
  const int i0 = a.initial_channel;
  const int c0 = blockIdx.x * CB;
  const int ncol = min(CB, a.n_xy - c0);
  const T oz = a.opt_z[iz];
  const long long col_base = static_cast<long long>(izr) * a.n_xy + c0;
  const int per_col = NPHI * jp;
  for (int e = threadIdx.x; e < ncol * per_col; e += blockDim.x) {
    const int c = e / per_col;
    const int r = e - c * per_col;
    const int p = r / jp;
    const int j = r - p * jp;
    V v = cmake<V>(0, 0);
    if (j < __ldg(args.slot_nj + p)) {
      const int irot = __ldg(args.slot_first + p) + j;
      v = a.psi[(col_base + c) * n_rot + irot];
      const long long n_scale = static_cast<long long>(a.nr) * n_rot;  // entries of the scaling tables
      v = cscale(fmul_t(v, a.before, n_scale, ir * n_rot + irot), oz);
      if (irot == i0) {
        const V incoming = a.chi[ir + a.nr * iz];
        v = cadd(v, fmul_t(cmul_t(incoming, a.sp2sc, a.n_xy, c0 + c), a.rot_half, n_scale, ir * n_rot + i0));
      }
    }
    F[c * FS + r] = v;
  }
  __syncthreads();
  const int line_c = threadIdx.x / nt;
  const int line_t = threadIdx.x - line_c * nt;
  const bool has_line = line_c < ncol;
  V x[NPHI];
  if (has_line) {
    const V* f = F + line_c * FS;
    const T* mt = args.legendre_slot + line_t;
    const long long n_slot = static_cast<long long>(NPHI) * jp * nt;  // low parts follow (mixed form)
    Acc<V> xa[NPHI];
    static_for<0, NPHI>([&](auto p) { xa[p] = acc_zero(); });
    for (int j = 0; j < jp; ++j) {
      static_for<0, NPHI>([&](auto p) {
        constexpr int P = SPO_CV(p);
        const long long k = (P * jp + j) * nt;
        xa[P] = acc_add(xa[P], f[P * jp + j], __ldg(mt + k), lo_real(mt, n_slot, k));
      });
    }
    static_for<0, NPHI>([&](auto p) { x[p] = acc_out<V>(xa[p]); });
  }
  __syncthreads();  // F is consumed; D takes its memory
  if (has_line) {
    const int ixy = c0 + line_c;
    rdft<NPHI, +1>(x);
    if (args.identity_maps) {
      const long long e0 = (static_cast<long long>(izr) * a.n_rep + ixy) * nt * NPHI + line_t * NPHI;
      static_for<0, NPHI>([&](auto p) { x[p] = exp_mul(x[p], __ldg(a.expia + e0 + p), a.exp_mod, e0 + p); });
    } else {
      const long long e0 = (static_cast<long long>(izr) * a.n_rep + a.rep_of[ixy]) * nt * NPHI + line_t * NPHI;
      const int* map = a.phi_map + ixy * NPHI;
      static_for<0, NPHI>([&](auto p) {
        const long long ei = e0 + __ldg(map + p);
        x[p] = exp_mul(x[p], __ldg(a.expia + ei), a.exp_mod, ei);
      });
    }
    rdft<NPHI, -1>(x);
    static_for<0, NPHI>([&](auto p) { D[(line_c * nt + line_t) * LD + p] = x[p]; });
  }
  __syncthreads();
  for (int irot = threadIdx.x; irot < n_rot; irot += blockDim.x) {
    const int blk = __ldg(a.irot_block + irot);
    const int nj = __ldg(a.block_size + blk);
    const int jj = irot - __ldg(a.block_first + blk);
    const int slot = __ldg(a.block_slot + blk);
    const T* col = a.legendre + __ldg(a.block_offset + blk) + jj;  // (theta, J) within the block
    const long long n_leg = static_cast<long long>(nt) * n_rot;      // low parts follow (mixed form)
    Acc<V> acc[CB];
#pragma unroll
    for (int c = 0; c < CB; ++c) acc[c] = acc_zero();
    for (int t = 0; t < nt; ++t) {
      const T w = __ldg(col + t * nj), wl = lo_real(col, n_leg, t * nj);
      const V* d = D + t * LD + slot;
#pragma unroll
      for (int c = 0; c < CB; ++c) acc[c] = acc_add(acc[c], d[c * nt * LD], w, wl);
    }
    const long long n_scale = static_cast<long long>(a.nr) * n_rot;
#pragma unroll
    for (int c = 0; c < CB; ++c)
      if (c < ncol) a.psi[(col_base + c) * n_rot + irot] = fmul_t(acc_out<V>(acc[c]), a.rot_half, n_scale, ir * n_rot + irot);
  }
}

// The projection of each interaction-region point onto the specular grid
// (src/propagation/potential_operator.cpp:129-135): chi(ir, iz) = sum over the (x, y) columns, in column
// order, of scattering_to_specular times the initial channel, then specular_to_scattering times it
// subtracted from the initial channel of every column. One block per point; the initial channel of the
// point's columns is gathered into shared memory (n_xy values) and summed by one thread.
template <typename T>
__global__ void projection_finalize_kernel(Vec<T>* __restrict__ psi, Vec<T>* __restrict__ chi, int n_rot, int n_xy,
                                           int i0, const Vec<T>* __restrict__ sc2sp, const Vec<T>* __restrict__ sp2sc) {
  using V = Vec<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* col = reinterpret_cast<V*>(smem_raw);  // n_xy
  V& proj = col[n_xy];                      // dynamic shared memory: (n_xy + 1) values
  const long long base = static_cast<long long>(blockIdx.x) * n_xy;  // blockIdx.x = ir + nr iz
  for (int ixy = threadIdx.x; ixy < n_xy; ixy += blockDim.x) col[ixy] = psi[(base + ixy) * n_rot + i0];
  __syncthreads();
  if (threadIdx.x == 0) {
    if constexpr (sizeof(T) == 4) {  // mixed form: the sum in FP64, the coefficients with their low parts
      double px = 0.0, py = 0.0;
      for (int ixy = 0; ixy < n_xy; ++ixy) {
        const V w = sc2sp[ixy], wl = sc2sp[n_xy + ixy], v = col[ixy];
        const double wx = static_cast<double>(w.x) + wl.x, wy = static_cast<double>(w.y) + wl.y;
        px += wx * v.x - wy * v.y;
        py += wx * v.y + wy * v.x;
      }
      proj = cmake<V>(static_cast<T>(px), static_cast<T>(py));
    } else {
      V p = cmake<V>(0, 0);
      for (int ixy = 0; ixy < n_xy; ++ixy) p = cadd(p, cmul(sc2sp[ixy], col[ixy]));
      proj = p;
    }
    chi[blockIdx.x] = proj;
  }
  __syncthreads();
  const V p = proj;
  for (int ixy = threadIdx.x; ixy < n_xy; ixy += blockDim.x)
    psi[(base + ixy) * n_rot + i0] = csub(col[ixy], cmul_t(p, sp2sc, n_xy, ixy));
}

}  // namespace spo

namespace spo {

// ---------------------------------------------------------------------------------------------
// Axis pass for N = N1 N2 with N1, N2 coprime, by the prime-factor (Good-Thomas) mapping: no twiddles
// between the levels. Point n = (N2 n1 + N1 n2) mod N; the two DFT levels (over n1, then over n2) give
// X(k1, k2) = DFT_N(x)[k], k = (N2 u k1 + N1 v k2) mod N with u = N2^-1 mod N1, v = N1^-1 mod N2,
// because exp(-2 pi i n k / N) = exp(-2 pi i n1 k1 / N1) exp(-2 pi i n2 k2 / N2) under these maps. The
// factor is diagonal in k, so it is applied at (k1, k2) from a table permuted on the host (factor_pfa),
// and the inverse levels undo the forward ones with the same point map. For r = 48 = 3 x 16 this drops
// the length-48 twiddles, whose products must be nearly correctly rounded in the mixed form (cmul_comp,
// ~26 instructions each), and leaves radix 3 (two-part roots) and a power-of-two DFT.
//   TB batch lanes x LT threads per lane: thread (b, s) takes the first-level lines n2 = s, s + LT, ...
//   (DFT_N1 each) and, for s < N1, the second-level line k1 = s (DFT_N2, factor, IDFT_N2).
// Dynamic shared memory: N TB values (the tile) and the factors (mixed form: their parts, see fmul_t).
// ---------------------------------------------------------------------------------------------
constexpr int pfa_inverse(int a, int m) {  // a^-1 mod m (a, m coprime)
  for (int x = 1; x < m; ++x)
    if ((a * x) % m == 1) return x;
  return 1;
}
template <typename T, int N1, int N2, int TB, int LT>
__global__ void __launch_bounds__(TB * LT) axis2pfa_kernel(Axis2Args<T> a) {
  using V = Vec<T>;
  constexpr int N = N1 * N2;
  static_assert(LT >= N1, "every second-level line needs a thread");
  constexpr int kFParts = sizeof(T) == 4 ? kFactorParts : 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* Y = reinterpret_cast<V*>(smem_raw);  // [n2][k1][b]
  V* f = Y + N * TB;                       // N factors in (k1, k2) order (then their parts)
  const int b = threadIdx.x % TB;
  const int s = threadIdx.x / TB;
  long long base, stride;
  bool lane_ok;
  if (a.blocks_per_group == 0) {
    const long long i0 = static_cast<long long>(blockIdx.x) * TB;
    base = static_cast<long long>(blockIdx.y) * N * a.inner + i0 + b;
    stride = a.inner;
    lane_ok = i0 + b < a.inner;
  } else {
    const int grp = blockIdx.x / a.blocks_per_group;
    const long long in_group = static_cast<long long>(blockIdx.x - grp * a.blocks_per_group) * TB + b;
    base = static_cast<long long>(blockIdx.y) * a.outer_stride + grp * a.group_stride + a.lane_offset + in_group;
    stride = a.line_stride;
    lane_ok = in_group < a.window;
  }
  for (int k = threadIdx.x; k < kFParts * N; k += TB * LT) f[k] = a.factor_pfa[k];
  __syncthreads();
  // forward, level 1 (DFT_N1 over n1 for each n2)
  for (int n2 = s; n2 < N2; n2 += LT) {
    V x[N1];
    static_for<0, N1>([&](auto n1) {
      int n = N2 * SPO_CV(n1) + N1 * n2;
      n = n >= N ? n - N : n;
      x[n1] = lane_ok ? a.data[base + static_cast<long long>(n) * stride] : cmake<V>(0, 0);
    });
    rdft<N1, -1>(x);
    static_for<0, N1>([&](auto k1) { Y[(n2 * N1 + k1) * TB + b] = x[k1]; });
  }
  __syncthreads();
  // level 2: DFT_N2 over n2, the factor at (k1, k2), inverse DFT_N2
  if (s < N1) {
    const int k1 = s;
    V y[N2];
    static_for<0, N2>([&](auto n2) { y[n2] = Y[(SPO_CV(n2) * N1 + k1) * TB + b]; });
    rdft<N2, -1>(y);
    static_for<0, N2>([&](auto k2) { y[k2] = fmul_t(y[k2], f, N, k1 + N1 * SPO_CV(k2)); });
    rdft<N2, +1>(y);
    static_for<0, N2>([&](auto n2) { Y[(SPO_CV(n2) * N1 + k1) * TB + b] = y[n2]; });
  }
  __syncthreads();
  // inverse level 1, store
  if (lane_ok) {
    for (int n2 = s; n2 < N2; n2 += LT) {
      V x[N1];
      static_for<0, N1>([&](auto k1) { x[k1] = Y[(n2 * N1 + k1) * TB + b]; });
      rdft<N1, +1>(x);
      static_for<0, N1>([&](auto n1) {
        int n = N2 * SPO_CV(n1) + N1 * n2;
        n = n >= N ? n - N : n;
        a.data[base + static_cast<long long>(n) * stride] = x[n1];
      });
    }
  }
}

}  // namespace spo

