// Device code of the split-operator step: complex helpers, a shared-memory mixed-radix Stockham FFT,
// and the kernels of one sub-step. Templated on the real type T (double: FP64 form, float: mixed form).
//
// Device layout of psi (the reference's host layout, src/propagation/wave_function.hpp:14-39):
//   psi[irot + n_rot * (ixy + n_xy * izr)], ixy = iy + ny*ix, izr = ir + nr*iz.
// Every FFT pass therefore moves tiles whose innermost (contiguous) index is a batch index, so the
// global loads and stores of every kernel are coalesced, whatever axis is transformed.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

namespace spo {

// ---------------------------------------------------------------------------------------------
// Complex arithmetic on double2 / float2
// ---------------------------------------------------------------------------------------------
template <typename T> struct VecOf;
template <> struct VecOf<double> { using type = double2; };
template <> struct VecOf<float> { using type = float2; };
template <typename T> using Vec = typename VecOf<T>::type;

#define SPO_HD __host__ __device__ __forceinline__

template <typename V> SPO_HD V cmake(decltype(V::x) re, decltype(V::x) im) {
  V v;
  v.x = re;
  v.y = im;
  return v;
}
template <typename V> SPO_HD V cadd(V a, V b) { return cmake<V>(a.x + b.x, a.y + b.y); }
template <typename V> SPO_HD V csub(V a, V b) { return cmake<V>(a.x - b.x, a.y - b.y); }
template <typename V> SPO_HD V cmul(V a, V b) {
  return cmake<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> SPO_HD V cconj(V a) { return cmake<V>(a.x, -a.y); }
template <typename V> SPO_HD V cscale(V a, decltype(V::x) s) { return cmake<V>(a.x * s, a.y * s); }
// a * (w + wl) for a constant held as two values: w (its rounding) and wl (the rounding of the rest).
// The mixed form keeps every constant factor (FFT twiddles, kinetic, rotation and coupling factors) this
// way: an FP32 constant of modulus 1 is off by up to 2^-24 in modulus, and the same constant applied at
// every time step to the same components changes the norm systematically (~1e-7 per step); held as
// w + wl it is exact to ~2^-48, and only the unbiased rounding of the product remains. The small terms are
// summed first, then the large ones, each by a fused multiply-add.
SPO_HD float2 cmul2(float2 a, float2 w, float2 wl) {
  const float cr = fmaf(a.x, wl.x, -a.y * wl.y);
  const float ci = fmaf(a.x, wl.y, a.y * wl.x);
  return make_float2(fmaf(a.x, w.x, fmaf(-a.y, w.y, cr)), fmaf(a.x, w.y, fmaf(a.y, w.x, ci)));
}
// The FP64 form keeps its constants in one double each (wl is ignored).
SPO_HD double2 cmul2(double2 a, double2 w, double2) {
  return make_double2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
// FP32 products and sums that the compiler may not fuse into FMAs (an error-free transformation needs the
// rounded product and the rounded sum themselves).
SPO_HD float mul_rn(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
SPO_HD float add_rn(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
// a b + c d + tl, nearly correctly rounded, in FP32 only: each product split exactly into its rounding and
// its error by an FMA (TwoProduct), the two roundings added with the error of the sum kept (Knuth's
// TwoSum), the errors and tl added last (the compensated dot product of Ogita, Rump and Oishi, "Accurate
// sum and dot product", SIAM J. Sci. Comput. 26, 2005).
SPO_HD float dot2_comp(float a, float b, float c, float d, float tl) {
  const float p1 = mul_rn(a, b), e1 = fmaf(a, b, -p1);
  const float p2 = mul_rn(c, d), e2 = fmaf(c, d, -p2);
  const float s = add_rn(p1, p2), bb = add_rn(s, -p1);
  const float es = add_rn(add_rn(p1, -add_rn(s, -bb)), add_rn(p2, -bb));
  return add_rn(s, add_rn(add_rn(es, e1), add_rn(e2, tl)));
}
// a * (w + wl) with each component nearly correctly rounded (mixed form). Twiddles of transform lengths with
// an odd factor (48 = 6 x 8, ...) need it: rounded as cmul2 rounds, their products drift the norm of a
// forward-inverse pass by ~2.6e-9, the same sign every pass (powers of two do not: cmul2 suffices); summed
// this way the drift is ~1e-11, as with an FP64 product, without the conversions.
SPO_HD float2 cmul_comp(float2 a, float2 w, float2 wl) {
  return make_float2(dot2_comp(a.x, w.x, -a.y, w.y, fmaf(a.x, wl.x, -a.y * wl.y)),
                     dot2_comp(a.x, w.y, a.y, w.x, fmaf(a.x, wl.y, a.y * wl.x)));
}
SPO_HD double2 cmul_comp(double2 a, double2 w, double2) {
  return make_double2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// The low part of a table entry: complex tables of the mixed form hold n values followed by their n low
// parts (see cmul2); the FP64 form's tables hold the n values only and have no low part.
template <typename V>
__device__ __forceinline__ V lo_part(const V* table, long long n, long long k) {
  if constexpr (sizeof(V) == 8) return table[n + k];
  else return V{0.0, 0.0};
}
// a * table[k] with the table's low part (mixed form).
template <typename V>
__device__ __forceinline__ V cmul_t(V a, const V* table, long long n, long long k) {
  return cmul2(a, table[k], lo_part(table, n, k));
}

// The low part of a real matrix entry k of a table of n entries: the mixed form's Legendre tables of the
// small-grid potential kernels hold their n entries followed by the n roundings of the remainders
// (FP64 value - entry), so that a contraction and its transpose keep the norm of a state to ~2^-48 whatever
// the number of theta points; FP64 tables have no low part.
template <typename T>
__device__ __forceinline__ T lo_real(const T* table, long long n, long long k) {
  if constexpr (sizeof(T) == 4) return table[n + k];
  else return T(0);
}
// Accumulators of the small-grid potential kernels' theta contractions: FP64 in both forms. The mixed form's
// matrix entry w + wl enters as one FP64 value and the sum is rounded to FP32 once (acc_out). Summed in FP32,
// the low part wl is mostly lost (it lies below half an ulp of the running sum), and the round trip of the
// forward and the transposed contraction then gains ~1.4e-8 of the norm per step on a physical wave packet
// whose rotational phases turn (host emulation of these kernels on cu111_dailight_small); summed in FP64,
// ~1e-10.
template <typename V> struct AccOf { using type = double2; };
template <typename V> using Acc = typename AccOf<V>::type;
__device__ __forceinline__ double2 acc_zero() { return make_double2(0.0, 0.0); }
// s + (w + wl) f
template <typename V>
__device__ __forceinline__ double2 acc_add(double2 s, V f, decltype(V::x) w, decltype(V::x) wl) {
  const double ww = static_cast<double>(w) + static_cast<double>(wl);
  return make_double2(fma(ww, static_cast<double>(f.x), s.x), fma(ww, static_cast<double>(f.y), s.y));
}
template <typename V>
__device__ __forceinline__ V acc_out(double2 s) {
  return cmake<V>(static_cast<decltype(V::x)>(s.x), static_cast<decltype(V::x)>(s.y));
}

// x * exp(i A) from the exp(i A) table. The mixed form holds g = exp(i A) - 1 (FP32; applied as x + x g, see
// fmul_t) and, per entry, m = 1/|1 + g| - 1 (FP16, a multiple of 2^-24): x (1 + g)(1 + m) = x + x (g + m (1 + g)).
// Without m a point's norm would change by |1 + g|^2 - 1 (~1e-8) every step, for all points of equal V the same
// way. The FP64 form holds exp(i A) itself.
// The same with the correction given: m as stored (a multiple of 2^-24 times 2^24) in FP32.
template <typename V>
__device__ __forceinline__ V exp_mul_m(V x, V e, float m24) {
  if constexpr (sizeof(V) == 8) {
    const float m = m24 * 5.9604644775390625e-8f;  // 2^-24
    return cadd(x, cmul2(x, e, make_float2(m * (1.0f + e.x), m * e.y)));
  } else {
    return cmul(e, x);
  }
}
template <typename V>
__device__ __forceinline__ V exp_mul(V x, V e, const __half* mod, long long idx) {
  if constexpr (sizeof(V) == 8) return exp_mul_m(x, e, __half2float(__ldg(mod + idx)));
  else return cmul(e, x);
}
// The corrections of entries 2i and 2i + 1 of a row read as 32-bit words (one __half2 per word).
__device__ __forceinline__ float mod_lo(uint32_t w) { return __low2float(*reinterpret_cast<const __half2*>(&w)); }
__device__ __forceinline__ float mod_hi(uint32_t w) { return __high2float(*reinterpret_cast<const __half2*>(&w)); }

// x times entry k of a factor table: a factor s e^{i phi} with s >= 0 real (a kinetic or rotation phase, with an
// FFT scale or an absorber). The mixed form holds each factor as g = e^{i phi} - 1 (n values), the low parts of g
// (n values) and (s, the low part of s) (n pairs), and forms s (x + x g): a near-unity phase applied as x e^{i phi}
// in FP32 rounds its result with a bias (~4e-10 of the norm per product for the small phases of the low kinetic
// momenta), x + x g does not (the correction x g is small and carries its own precision). The FP64 form's tables
// hold the factors themselves.
template <typename V>
__device__ __forceinline__ V fmul_parts(V x, V g, V gl, V sc) {
  if constexpr (sizeof(V) == 8) {
    const float2 z = cadd(x, cmul2(x, g, gl));
    return make_float2(fmaf(z.x, sc.x, z.x * sc.y), fmaf(z.y, sc.x, z.y * sc.y));
  } else {
    return cmul(g, x);
  }
}
template <typename V>
__device__ __forceinline__ V fmul_t(V x, const V* table, long long n, long long k) {
  if constexpr (sizeof(V) == 8) return fmul_parts(x, table[k], table[n + k], table[2 * n + k]);
  else return cmul(table[k], x);
}
// Entries of a mixed-form factor table per value: g, its low part, the scale pair.
constexpr int kFactorParts = 3;

// i * s * a for s = +1 or -1.
template <typename V> SPO_HD V cimul(V a, int s) {
  return s > 0 ? cmake<V>(-a.y, a.x) : cmake<V>(a.y, -a.x);
}

// ---------------------------------------------------------------------------------------------
// FFT plan: the radices of one length, passed by value. Lengths are 2^h 3^i 5^j 7^k 11^m
// (i <= 2, j, k, m <= 1), the reference's valid FFT sizes (src/fft/fft_sizes.cpp:9-34).
// ---------------------------------------------------------------------------------------------
constexpr int kMaxStages = 20;
struct FftPlan {
  int n;
  int n_stages;
  int radix[kMaxStages];
};

// w^q for the r-th roots of unity, read from the length-n table tw[k] = exp(-2 pi i k / n), and its low
// part (mixed form: the n low parts follow the table in shared memory).
template <typename V>
__device__ __forceinline__ V root_of(const V* tw, int n, int r, int q, int sign) {
  V w = tw[(q % r) * (n / r)];
  return sign > 0 ? cconj(w) : w;
}
template <typename V>
__device__ __forceinline__ V root_lo_of(const V* tw, int n, int r, int q, int sign) {
  V w = lo_part(tw, n, (q % r) * (n / r));
  return sign > 0 ? cconj(w) : w;
}

// In-register DFT of R values with exponent sign `sign`.
template <typename V, int R>
__device__ __forceinline__ void small_dft(V (&v)[R], const V* tw, int n, int sign) {
  if constexpr (R == 2) {
    const V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const V s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    const V s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
    const V jd = cimul(d13, sign);
    v[0] = cadd(s02, s13);
    v[1] = cadd(d02, jd);
    v[2] = csub(s02, s13);
    v[3] = csub(d02, jd);
  } else {
    // Odd prime R: pairs (t, R - t) share the real part of the root and have opposite imaginary parts.
    constexpr int H = R / 2;
    V s[H + 1], d[H + 1];
#pragma unroll
    for (int t = 1; t <= H; ++t) {
      s[t] = cadd(v[t], v[R - t]);
      d[t] = csub(v[t], v[R - t]);
    }
    V out0 = v[0];
#pragma unroll
    for (int t = 1; t <= H; ++t) out0 = cadd(out0, s[t]);
    V res[R];
    res[0] = out0;
    // Each output pair summed in the accumulation type A (FP64 in the mixed form, see the register DFTs'
    // odd primes) from the sums and differences, rounded once.
    using Rl = decltype(V::x);
    using A = std::conditional_t<sizeof(Rl) == 4, double, Rl>;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      A rex = v[0].x, rey = v[0].y, im_re = 0, im_im = 0;
#pragma unroll
      for (int t = 1; t <= H; ++t) {
        const V w = root_of(tw, n, R, t * q, sign);
        const V wl = root_lo_of(tw, n, R, t * q, sign);  // zero in the FP64 form
        const A wx = static_cast<A>(w.x) + static_cast<A>(wl.x), wy = static_cast<A>(w.y) + static_cast<A>(wl.y);
        rex += wx * static_cast<A>(s[t].x);
        rey += wx * static_cast<A>(s[t].y);
        im_re += wy * static_cast<A>(d[t].x);
        im_im += wy * static_cast<A>(d[t].y);
      }
      res[q] = cmake<V>(static_cast<Rl>(rex - im_im), static_cast<Rl>(rey + im_re));  // re + i * sum Im(w) d
      res[R - q] = cmake<V>(static_cast<Rl>(rex + im_im), static_cast<Rl>(rey - im_re));
    }
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = res[t];
  }
}

// One Stockham stage of radix R for n_lines independent lines of length n stored in shared memory.
// Line l starts at base(l) = (l / L1) * S1 + (l % L1), element e of a line is at base + e * S.
// Consecutive threads take consecutive lines (conflict-free when lines are adjacent words).
template <typename V, int R>
__device__ __forceinline__ void fft_stage(const V* __restrict__ src, V* __restrict__ dst, const V* tw, int n, int ns,
                                          int sign, int n_lines, int L1, int S1, int S) {
  const int m = n / R;
  const int span = ns * R;
  const int twstep = n / span;
  const int total = n_lines * m;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int line = idx % n_lines;
    const int j = idx / n_lines;
    const int base = (line / L1) * S1 + (line % L1);
    const int k = j % ns;
    V v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = src[base + (j + t * m) * S];
#pragma unroll
    for (int t = 1; t < R; ++t) {
      V w = tw[t * k * twstep];
      V wl = lo_part(tw, n, t * k * twstep);
      if (sign > 0) {
        w = cconj(w);
        wl = cconj(wl);
      }
      v[t] = (n & (n - 1)) != 0 ? cmul_comp(v[t], w, wl) : cmul2(v[t], w, wl);  // see cmul_comp
    }
    small_dft<V, R>(v, tw, n, sign);
    const int o = (j / ns) * span + k;
#pragma unroll
    for (int t = 0; t < R; ++t) dst[base + (o + t * ns) * S] = v[t];
  }
}

// Complete transform of the lines (see fft_stage), ping-ponging between a and b. Returns the buffer
// that holds the result. Every stage ends with __syncthreads(); the caller must have synchronised
// before the call.
template <typename V>
__device__ V* smem_fft(V* a, V* b, const V* tw, const FftPlan& p, int sign, int n_lines, int L1, int S1, int S) {
  int ns = 1;
  for (int s = 0; s < p.n_stages; ++s) {
    const int r = p.radix[s];
    switch (r) {
      case 2: fft_stage<V, 2>(a, b, tw, p.n, ns, sign, n_lines, L1, S1, S); break;
      case 3: fft_stage<V, 3>(a, b, tw, p.n, ns, sign, n_lines, L1, S1, S); break;
      case 4: fft_stage<V, 4>(a, b, tw, p.n, ns, sign, n_lines, L1, S1, S); break;
      case 5: fft_stage<V, 5>(a, b, tw, p.n, ns, sign, n_lines, L1, S1, S); break;
      case 7: fft_stage<V, 7>(a, b, tw, p.n, ns, sign, n_lines, L1, S1, S); break;
      case 11: fft_stage<V, 11>(a, b, tw, p.n, ns, sign, n_lines, L1, S1, S); break;
      default: break;  // rejected at plan time
    }
    __syncthreads();
    V* t = a;
    a = b;
    b = t;
    ns *= r;
  }
  return a;
}

// ---------------------------------------------------------------------------------------------
// Axis pass: FFT along one axis of an array (outer, n, inner) with inner contiguous, for a tile of
// `tb` consecutive inner elements: forward (sign -1), multiply by a factor, inverse (sign +1).
// Used for T_Z and T_r of psi (src/propagation/kinetic_operators.cpp:77-111, separably) and for the
// specular grid (src/propagation/specular_operator.cpp:48-54).
// ---------------------------------------------------------------------------------------------
enum AxisDir : int { kFwdFactorInv = 0, kFwdFactor = 1, kFactorInv = 2 };
enum FactorMode : int { kNoFactor = 0, kFactorAxis = 1, kFactorAxisInner = 2 };

template <typename T>
struct AxisArgs {
  Vec<T>* data;
  long long inner;
  FftPlan plan;
  const Vec<T>* tw;      // exp(-2 pi i k / n), n values
  const Vec<T>* factor;  // by axis index (kFactorAxis) or by inner + inner_count * k (kFactorAxisInner)
  int factor_mode;
  int dir;
  const Vec<T>* post;    // pointwise factor by global element index after the pass, or null
  int tb;
};

template <typename T>
__global__ void __launch_bounds__(256) axis_pass_kernel(AxisArgs<T> a) {
  using V = Vec<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* buf0 = reinterpret_cast<V*>(smem_raw);
  const int n = a.plan.n;
  const int tb = a.tb;
  V* buf1 = buf0 + n * tb;
  V* tw = buf1 + n * tb;  // n values, then (mixed form) their n low parts
  const long long outer = blockIdx.y;
  const long long i0 = static_cast<long long>(blockIdx.x) * tb;
  const long long base = outer * n * a.inner + i0;
  for (int k = threadIdx.x; k < (sizeof(T) == 4 ? 2 : 1) * n; k += blockDim.x) tw[k] = a.tw[k];
  for (int e = threadIdx.x; e < n * tb; e += blockDim.x) {
    const int k = e / tb, b = e % tb;
    V v = cmake<V>(0, 0);
    if (i0 + b < a.inner) v = a.data[base + k * a.inner + b];
    buf0[e] = v;
  }
  __syncthreads();
  V* cur = buf0;
  V* oth = buf1;
  if (a.dir != kFactorInv) {
    cur = smem_fft(cur, oth, tw, a.plan, -1, tb, tb, 0, tb);
    oth = cur == buf0 ? buf1 : buf0;
  }
  if (a.factor_mode != kNoFactor) {
    for (int e = threadIdx.x; e < n * tb; e += blockDim.x) {
      const int k = e / tb, b = e % tb;
      cur[e] = a.factor_mode == kFactorAxis ? fmul_t(cur[e], a.factor, n, k)
                                            : fmul_t(cur[e], a.factor, a.inner * n, (i0 + b) + a.inner * k);
    }
    __syncthreads();
  }
  if (a.dir != kFwdFactor) {
    cur = smem_fft(cur, oth, tw, a.plan, +1, tb, tb, 0, tb);
  }
  for (int e = threadIdx.x; e < n * tb; e += blockDim.x) {
    const int k = e / tb, b = e % tb;
    if (i0 + b < a.inner) {
      const long long g = base + k * a.inner + b;
      V v = cur[e];
      if (a.post) v = fmul_t(v, a.post, static_cast<long long>(gridDim.y) * n * a.inner, g);
      a.data[g] = v;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// xy pass: exp(-i T_xy dt) at every (Z, r) point for a tile of `tb` rotational states: momentum
// shift, 2D (x, y) FFT, kinetic factor, inverse, shift back (src/propagation/kinetic_operators.cpp:
// 134-172). In the gas-phase region (izr >= izr_gas_first) the potential step of that region,
// optical_z * rot exp(-i vasy dt) rot (src/propagation/potential_operator.cpp:104-112), is applied
// in the same pass when `apply_gas` is set.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct XyArgs {
  Vec<T>* psi;
  int n_rot, nx, ny;
  FftPlan px, py;
  const Vec<T>* twx;
  const Vec<T>* twy;
  const Vec<T>* factor;   // nx*ny, FFT scales folded in
  const Vec<T>* shift_f;  // nx*ny or null (no momentum shift)
  const Vec<T>* shift_b;
  int tb;
  int apply_gas;
  long long izr_gas_first;
  int nr;
  const T* opt_z;          // nz
  const Vec<T>* gas_step;  // (ir, irot): opt_r rot gas rot
  int tile;                // launch choice of the register-DFT xy kernel: rotational states per block
                           // (8, 16 or 32; 0: the default) for grids of more than 8 points per axis
  long long izr_offset;    // register-DFT xy kernel: block y serves point izr = izr_offset + y
  int persistent;          // launch choice: the persistent form of the register-DFT xy kernel (xy2p_kernel)
};

template <typename T>
__global__ void __launch_bounds__(256) xy_pass_kernel(XyArgs<T> a) {
  using V = Vec<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nxy = a.nx * a.ny;
  const int tb = a.tb;
  V* buf0 = reinterpret_cast<V*>(smem_raw);
  V* buf1 = buf0 + nxy * tb;
  constexpr int kParts = sizeof(T) == 4 ? 2 : 1;  // the mixed form's tables carry their low parts
  V* twx = buf1 + nxy * tb;
  V* twy = twx + kParts * a.nx;
  const long long izr = blockIdx.y;
  const int r0 = blockIdx.x * tb;
  for (int k = threadIdx.x; k < kParts * a.nx; k += blockDim.x) twx[k] = a.twx[k];
  for (int k = threadIdx.x; k < kParts * a.ny; k += blockDim.x) twy[k] = a.twy[k];
  const long long col0 = izr * nxy;
  for (int e = threadIdx.x; e < nxy * tb; e += blockDim.x) {
    const int ixy = e / tb, b = e % tb;
    V v = cmake<V>(0, 0);
    if (r0 + b < a.n_rot) {
      v = a.psi[(col0 + ixy) * a.n_rot + r0 + b];
      if (a.shift_f) v = fmul_t(v, a.shift_f, nxy, ixy);
    }
    buf0[e] = v;
  }
  __syncthreads();
  // y: lines (ix, b), element stride tb; x: lines (iy, b), element stride ny*tb.
  V* cur = smem_fft(buf0, buf1, twy, a.py, -1, a.nx * tb, tb, a.ny * tb, tb);
  V* oth = cur == buf0 ? buf1 : buf0;
  cur = smem_fft(cur, oth, twx, a.px, -1, a.ny * tb, a.ny * tb, 0, a.ny * tb);
  oth = cur == buf0 ? buf1 : buf0;
  for (int e = threadIdx.x; e < nxy * tb; e += blockDim.x) cur[e] = fmul_t(cur[e], a.factor, nxy, e / tb);
  __syncthreads();
  cur = smem_fft(cur, oth, twx, a.px, +1, a.ny * tb, a.ny * tb, 0, a.ny * tb);
  oth = cur == buf0 ? buf1 : buf0;
  cur = smem_fft(cur, oth, twy, a.py, +1, a.nx * tb, tb, a.ny * tb, tb);
  const bool gas = a.apply_gas && izr >= a.izr_gas_first;
  const int ir = static_cast<int>(izr % a.nr);
  const T oz = gas ? a.opt_z[izr / a.nr] : T(1);
  for (int e = threadIdx.x; e < nxy * tb; e += blockDim.x) {
    const int ixy = e / tb, b = e % tb;
    if (r0 + b < a.n_rot) {
      V v = cur[e];
      if (a.shift_b) v = fmul_t(v, a.shift_b, nxy, ixy);
      if (gas) {
        v = fmul_t(v, a.gas_step, static_cast<long long>(a.nr) * a.n_rot, ir * a.n_rot + r0 + b);
        v = cscale(v, oz);
      }
      a.psi[(col0 + ixy) * a.n_rot + r0 + b] = v;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Potential step of the interaction region, one (Z, r) point per block, all its (x, y) columns
// (src/propagation/potential_operator.cpp:114-136, 158-201; src/propagation/angular_transform.cpp:
// 54-114): absorption and rot(dt/2), the specular wave added to the initial channel, FBR -> DVR
// (theta contraction per mJ block, phi FFT sign +1), exp(i A) through the symmetry maps, DVR -> FBR
// (phi FFT sign -1, transposed contraction), rot(dt/2), and the projection of the initial channel
// onto the specular grid with a fixed summation order.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct PotArgs {
  Vec<T>* psi;
  Vec<T>* chi;                // (ir, iz)
  int n_rot, n_xy, nr, n_theta, n_phi, ld, n_blocks, mj_max, initial_channel, n_rep;
  int cb;                     // columns per chunk
  FftPlan pphi;
  const Vec<T>* twphi;
  const T* legendre;          // (block, theta, J)
  const int* block_first;     // per mJ block: first irot
  const int* block_size;      // n_J
  const int* block_slot;      // phi slot
  const int* block_offset;    // offset into legendre
  const int* irot_block;      // block of each irot
  const T* opt_z;             // nz
  const Vec<T>* before;       // (ir, irot): opt_r rot(dt/2)
  const Vec<T>* rot_half;     // (ir, irot)
  const Vec<T>* sp2sc;        // n_xy
  const Vec<T>* sc2sp;        // n_xy
  const Vec<T>* expia;        // (izr, irep, theta, phi)
  const __half* exp_mod;      // mixed form: per expia entry, (1/|entry| - 1) * 2^24 (see exp_mul); FP64: null
  const int* rep_of;          // n_xy
  const int* phi_map;         // n_xy * n_phi: phi_index of the operation of each ixy
};

template <typename T>
__global__ void __launch_bounds__(256) potential_kernel(PotArgs<T> a) {
  using V = Vec<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n_rot = a.n_rot, nt = a.n_theta, nphi = a.n_phi, ld = a.ld, cb = a.cb;
  const int dvr_col = nt * ld;
  V* fbr = reinterpret_cast<V*>(smem_raw);   // cb * n_rot
  V* dvr0 = fbr + cb * n_rot;                // cb * nt * ld
  V* dvr1 = dvr0 + cb * dvr_col;             // cb * nt * ld
  constexpr int kParts = sizeof(T) == 4 ? 2 : 1;  // the mixed form's twiddles carry their low parts
  V* twp = dvr1 + cb * dvr_col;              // nphi (then nphi low parts)
  V* i0buf = twp + kParts * nphi;            // n_xy
  V* red = i0buf + a.n_xy;                   // 32
  T* leg = reinterpret_cast<T*>(red + 32);   // nt * n_rot (then, mixed form, their low parts)
  const long long n_leg = static_cast<long long>(nt) * n_rot;
  const int izr = blockIdx.x;
  const int ir = izr % a.nr;
  const int iz = izr / a.nr;
  const int i0 = a.initial_channel;
  for (int k = threadIdx.x; k < kParts * nphi; k += blockDim.x) twp[k] = a.twphi[k];
  for (int k = threadIdx.x; k < (sizeof(T) == 4 ? 2 : 1) * nt * n_rot; k += blockDim.x) leg[k] = a.legendre[k];
  const T oz = a.opt_z[iz];
  const V incoming = a.chi[ir + a.nr * iz];
  const long long n_scale = static_cast<long long>(a.nr) * n_rot;  // entries of the scaling tables
  const long long col_base = static_cast<long long>(izr) * a.n_xy;
  const long long e_base = static_cast<long long>(izr) * a.n_rep * nt * nphi;
  __syncthreads();

  for (int c0 = 0; c0 < a.n_xy; c0 += cb) {
    const int ncol = min(cb, a.n_xy - c0);
    // Load, absorb, rot(dt/2), add the specular wave to the initial channel.
    for (int e = threadIdx.x; e < ncol * n_rot; e += blockDim.x) {
      const int c = e / n_rot, irot = e % n_rot;
      const int ixy = c0 + c;
      V v = a.psi[(col_base + ixy) * n_rot + irot];
      v = cscale(fmul_t(v, a.before, n_scale, ir * n_rot + irot), oz);
      if (irot == i0) v = cadd(v, fmul_t(cmul_t(incoming, a.sp2sc, a.n_xy, ixy), a.rot_half, n_scale, ir * n_rot + i0));
      fbr[c * n_rot + irot] = v;
    }
    __syncthreads();
    // FBR -> DVR: theta sums per mJ block into the block's phi slot; other slots zero.
    for (int e = threadIdx.x; e < ncol * nt * nphi; e += blockDim.x) {
      const int p = e % nphi;
      const int t = (e / nphi) % nt;
      const int c = e / (nphi * nt);
      // slot p holds mJ = p (p <= mj_max) or mJ = p - nphi (p >= nphi - mj_max)
      int blk = -1;
      if (p <= a.mj_max) blk = a.mj_max + p;
      else if (p >= nphi - a.mj_max) blk = a.mj_max + (p - nphi);
      Acc<V> s = acc_zero();
      if (blk >= 0) {
        const int nj = a.block_size[blk];
        const long long r0 = a.block_offset[blk] + t * nj;
        const V* f = fbr + c * n_rot + a.block_first[blk];
        for (int j = 0; j < nj; ++j) s = acc_add(s, f[j], leg[r0 + j], lo_real(leg, n_leg, r0 + j));
      }
      dvr0[c * dvr_col + t * ld + p] = acc_out<V>(s);
    }
    __syncthreads();
    V* cur = smem_fft(dvr0, dvr1, twp, a.pphi, +1, ncol * nt, 1, ld, 1);
    V* oth = cur == dvr0 ? dvr1 : dvr0;
    // exp(i A) of the representative, at the mapped phi.
    for (int e = threadIdx.x; e < ncol * nt * nphi; e += blockDim.x) {
      const int p = e % nphi;
      const int t = (e / nphi) % nt;
      const int c = e / (nphi * nt);
      const int ixy = c0 + c;
      const int rep = a.rep_of[ixy];
      const int pm = a.phi_map[ixy * nphi + p];
      const long long ei = e_base + (static_cast<long long>(rep) * nt + t) * nphi + pm;
      cur[c * dvr_col + t * ld + p] = exp_mul(cur[c * dvr_col + t * ld + p], a.expia[ei], a.exp_mod, ei);
    }
    __syncthreads();
    cur = smem_fft(cur, oth, twp, a.pphi, -1, ncol * nt, 1, ld, 1);
    // DVR -> FBR: transposed theta sums, then rot(dt/2).
    for (int e = threadIdx.x; e < ncol * n_rot; e += blockDim.x) {
      const int c = e / n_rot, irot = e % n_rot;
      const int blk = a.irot_block[irot];
      const int nj = a.block_size[blk];
      const int jj = irot - a.block_first[blk];
      const int slot = a.block_slot[blk];
      const long long c0l = a.block_offset[blk] + jj;
      Acc<V> sa = acc_zero();
      for (int t = 0; t < nt; ++t)
        sa = acc_add(sa, cur[c * dvr_col + t * ld + slot], leg[c0l + t * nj], lo_real(leg, n_leg, c0l + t * nj));
      const V s = fmul_t(acc_out<V>(sa), a.rot_half, n_scale, ir * n_rot + irot);
      const int ixy = c0 + c;
      if (irot == i0) i0buf[ixy] = s;
      else a.psi[(col_base + ixy) * n_rot + irot] = s;
    }
    __syncthreads();
  }
  // Projection onto the specular grid: a fixed-order sum over (x, y) by warp 0.
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

// ---------------------------------------------------------------------------------------------
// Utilities
// ---------------------------------------------------------------------------------------------

// Potential step of the gas-phase region alone (izr >= izr_first): optical_z * gas_step(ir, irot)
// (src/propagation/potential_operator.cpp:104-112). The propagation fuses this into the xy pass;
// this kernel serves the stage-by-stage entry point.
template <typename T>
__global__ void gas_phase_kernel(Vec<T>* __restrict__ psi, long long izr_first, long long n_zr, int n_rot, int n_xy,
                                 int nr, const T* __restrict__ opt_z, const Vec<T>* __restrict__ gas_step) {
  const long long per_izr = static_cast<long long>(n_xy) * n_rot;
  const long long n = (n_zr - izr_first) * per_izr;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long izr = izr_first + i / per_izr;
    const int irot = static_cast<int>(i % n_rot);
    const int ir = static_cast<int>(izr % nr);
    const long long g = izr_first * per_izr + i;
    psi[g] = cscale(fmul_t(psi[g], gas_step, static_cast<long long>(nr) * n_rot, ir * n_rot + irot), opt_z[izr / nr]);
  }
}

// exp(i A), A = -V dt, formed in FP64 (src/propagation/potential_operator.cpp:55-65 with
// src/potential/potential_grid.cpp:164-167), then rounded to T.
template <typename T>
__global__ void exp_potential_kernel(const double* __restrict__ v, Vec<T>* __restrict__ out, __half* __restrict__ mod,
                                     long long n, double dt) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double a = -v[i] * dt;
    double s, c;
    sincos(a, &s, &c);
    if constexpr (sizeof(T) == 4) {  // g = exp(i A) - 1 and the modulus correction of 1 + g (see exp_mul)
      const double cm1 = -2.0 * sin(0.5 * a) * sin(0.5 * a);  // cos A - 1 without cancellation
      const float gx = static_cast<float>(cm1), gy = static_cast<float>(s);
      out[i] = cmake<Vec<T>>(gx, gy);
      const double rx = 1.0 + static_cast<double>(gx), ry = gy;
      mod[i] = __double2half((1.0 / sqrt(rx * rx + ry * ry) - 1.0) * 16777216.0);
    } else {
      out[i] = cmake<Vec<T>>(static_cast<T>(c), static_cast<T>(s));
    }
  }
}

// The norm budget of one analysis window on the device, FP64 (src/analysis/norm_budget.cpp:24-35, 75-111):
// the cell probabilities of the current state (block densities times the scattering cell volume, |chi|^2 times
// the specular one), the loss of every absorbing cell over the window from the previous call's cells
//   gamma = window exponent, F = exp(-gamma), 1 - F = -expm1(-gamma),
//   loss = rho_start (1 - F) + (rho_end - F rho_start) (gamma / (1 - F) - 1),
//   error = gamma^2 / 6 |rho_end - rho_start + loss|,
// shared between the cell's Z absorber (z_share) and its r absorber (the rest), and the norms at the window's
// start and end. One block, a fixed assignment of cells to threads and a fixed tree: the sums are repeatable
// (not in the reference's serial order; they agree to rounding). The current cells replace the previous ones.
constexpr int kBudgetMaxAbsorbers = 6;
struct BudgetGrid {
  const double* exponent;  // per cell: 2 n V_opt dt of the window (0: the cell does not absorb)
  const double* z_share;   // per cell: the Z absorber's share of the loss
  const int* z_absorber;   // per cell: index of the Z absorber, -1: none
  const int* r_absorber;   // per cell: index of the r absorber, -1: none
  double* previous;        // the cells of the previous call
  long long cells;
};
template <typename T>
__global__ void __launch_bounds__(256) norm_budget_kernel(const double* __restrict__ densities, double vol_scat,
                                                          const Vec<T>* __restrict__ chi, double vol_spec,
                                                          BudgetGrid scat, BudgetGrid spec, int n_absorbers,
                                                          int has_previous, double* __restrict__ out) {
  constexpr int NV = 2 * kBudgetMaxAbsorbers + 2;  // loss, error per absorber; norm at start, at end
  __shared__ double part[NV][256];
  double acc[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int grid = 0; grid < 2; ++grid) {
    const BudgetGrid& g = grid == 0 ? scat : spec;
    for (long long k = threadIdx.x; k < g.cells; k += blockDim.x) {
      double rho_end;
      if (grid == 0) {
        rho_end = densities[k] * vol_scat;
      } else {
        const Vec<T> c = chi[k];
        rho_end = (static_cast<double>(c.x) * c.x + static_cast<double>(c.y) * c.y) * vol_spec;
      }
      if (has_previous) {
        const double rho_start = g.previous[k];
        acc[NV - 2] += rho_start;
        acc[NV - 1] += rho_end;
        const int za = g.z_absorber[k], ra = g.r_absorber[k];
        if (za >= 0 || ra >= 0) {
          const double gamma = g.exponent[k];
          const double one_minus_f = -expm1(-gamma);
          const double f = exp(-gamma);
          const double loss = rho_start * one_minus_f + (rho_end - f * rho_start) * (gamma / one_minus_f - 1.0);
          const double err = gamma * gamma / 6.0 * fabs(rho_end - rho_start + loss);
          const double zs = g.z_share[k];
#pragma unroll
          for (int a = 0; a < kBudgetMaxAbsorbers; ++a) {
            if (a == za) {
              acc[a] += zs * loss;
              acc[kBudgetMaxAbsorbers + a] += zs * err;
            }
            if (a == ra) {
              acc[a] += (1.0 - zs) * loss;
              acc[kBudgetMaxAbsorbers + a] += (1.0 - zs) * err;
            }
          }
        }
      }
      g.previous[k] = rho_end;
    }
  }
#pragma unroll
  for (int k = 0; k < NV; ++k) part[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < NV; ++k) part[k][threadIdx.x] += part[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int a = 0; a < n_absorbers; ++a) {
      out[a] = part[a][0];
      out[n_absorbers + a] = part[kBudgetMaxAbsorbers + a][0];
    }
    out[2 * n_absorbers] = part[NV - 2][0];
    out[2 * n_absorbers + 1] = part[NV - 1][0];
  }
}

// sum |psi|^2 over one (Z, r) block (n_block values) in FP64, fixed order: strided per thread, then
// a fixed tree (src/propagation/averages.cpp:20-29).
template <typename T>
__global__ void block_density_kernel(const Vec<T>* __restrict__ psi, long long n_block, double* __restrict__ out) {
  __shared__ double part[256];
  const long long base = static_cast<long long>(blockIdx.x) * n_block;
  double s = 0.0;
  for (long long i = threadIdx.x; i < n_block; i += blockDim.x) {
    const Vec<T> v = psi[base + i];
    const double re = v.x, im = v.y;
    s += re * re + im * im;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = part[0];
}

// (izr, irot) column of one (x, y) point: out[izr + n_zr * irot] = psi[irot + n_rot*(ixy + n_xy*izr)].
template <typename T>
__global__ void site_column_kernel(const Vec<T>* __restrict__ psi, double2* __restrict__ out, int n_rot, int n_xy,
                                   long long n_zr, int ixy) {
  const long long n = n_zr * n_rot;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long izr = i % n_zr;
    const int irot = static_cast<int>(i / n_zr);
    const Vec<T> v = psi[(izr * n_xy + ixy) * n_rot + irot];
    out[i] = make_double2(v.x, v.y);
  }
}

// Balint-Kurti projection, one block per (v, irotana) (src/analysis/balint_kurti.cpp:53-74), FP64:
// overlap(ixy) = sum_ir shift(ixy) psi(iz_a, ir, ixy, irot) phi_vj(ir) dr in ir order, a 2D (x, y)
// DFT (sign -1, scale 1), the diffraction channels times xy_scale.
template <typename T>
struct BkArgs {
  const Vec<T>* psi;
  int n_rot, nx, ny, nr, iz_analysis;
  int n_v, n_rotation, n_diffraction, j_max_gas;
  const int* rotation_index;
  const int* rotation_j;
  const int* channel_ix;
  const int* channel_iy;
  const double* phi_vj;  // (ir, j, v)
  const double2* shift;  // nx*ny, FP64
  double dr, xy_scale;
  FftPlan px, py;
  const double2* twx;
  const double2* twy;
  double2* bk;           // (is, v)
};

template <typename T>
__global__ void __launch_bounds__(256) bk_kernel(BkArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nxy = a.nx * a.ny;
  double2* o0 = reinterpret_cast<double2*>(smem_raw);
  double2* o1 = o0 + nxy;
  double2* twx = o1 + nxy;
  double2* twy = twx + a.nx;
  const int v = blockIdx.x / a.n_rotation;
  const int irotana = blockIdx.x % a.n_rotation;
  const int irot = a.rotation_index[irotana];
  const double* phi = a.phi_vj + static_cast<long long>(a.nr) * (a.rotation_j[irotana] + (a.j_max_gas + 1) * v);
  for (int k = threadIdx.x; k < a.nx; k += blockDim.x) twx[k] = a.twx[k];
  for (int k = threadIdx.x; k < a.ny; k += blockDim.x) twy[k] = a.twy[k];
  const long long plane = static_cast<long long>(a.iz_analysis) * a.nr * nxy;
  for (int ixy = threadIdx.x; ixy < nxy; ixy += blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    const double2 sh = a.shift[ixy];
    for (int ir = 0; ir < a.nr; ++ir) {
      const Vec<T> p = a.psi[((plane + static_cast<long long>(ir) * nxy) + ixy) * a.n_rot + irot];
      const double w = phi[ir] * a.dr;
      const double2 t = cmul(sh, make_double2(p.x, p.y));
      s = make_double2(s.x + t.x * w, s.y + t.y * w);
    }
    o0[ixy] = s;
  }
  __syncthreads();
  double2* cur = smem_fft(o0, o1, twy, a.py, -1, a.nx, 1, a.ny, 1);    // along y: lines ix, stride 1
  double2* oth = cur == o0 ? o1 : o0;
  cur = smem_fft(cur, oth, twx, a.px, -1, a.ny, a.ny, 0, a.ny);         // along x: lines iy, stride ny
  const int n_states = a.n_rotation * a.n_diffraction;
  for (int idif = threadIdx.x; idif < a.n_diffraction; idif += blockDim.x) {
    const double2 c = cur[a.channel_ix[idif] * a.ny + a.channel_iy[idif]];
    a.bk[irotana * a.n_diffraction + idif + static_cast<long long>(n_states) * v] =
        make_double2(c.x * a.xy_scale, c.y * a.xy_scale);
  }
}

// The initial state's coefficients from the specular wave at the fixed analysis line iz
// (balint_kurti.cpp:76-84): sum_ir chi(ir, iz) phi_(v, jin)(ir), times dr, in ir order.
template <typename T>
__global__ void bk_specular_kernel(const Vec<T>* __restrict__ chi, int nr, int iz, const double* __restrict__ phi_vj,
                                   int j_max_gas, int j_in, int n_v, int n_states, int initial_state, double dr,
                                   double2* __restrict__ bk) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n_v) return;
  const double* phi = phi_vj + static_cast<long long>(nr) * (j_in + (j_max_gas + 1) * v);
  double2 s = make_double2(0.0, 0.0);
  for (int ir = 0; ir < nr; ++ir) {
    const Vec<T> c = chi[ir + static_cast<long long>(nr) * iz];
    s = make_double2(s.x + c.x * phi[ir], s.y + c.y * phi[ir]);
  }
  bk[initial_state + static_cast<long long>(n_states) * v] = make_double2(s.x * dr, s.y * dr);
}

// S-matrix sums (s_matrix.cpp:49-56): sums(k, ien) += bk(k) exp(i E_ien t) dt_analysis, FP64.
static __global__ void s_matrix_add_kernel(const double2* __restrict__ bk, int n, const double* __restrict__ energies,
                                    int n_energies, double time, double dt, double2* __restrict__ sums) {
  const long long total = static_cast<long long>(n) * n_energies;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(i % n);
    const int ien = static_cast<int>(i / n);
    double sn, cs;
    sincos(energies[ien] * time, &sn, &cs);
    const double2 t = cmul(bk[k], make_double2(cs, sn));
    sums[i] = make_double2(sums[i].x + t.x * dt, sums[i].y + t.y * dt);
  }
}

// Precision conversion of a complex array.
template <typename TO, typename TI>
__global__ void convert_kernel(const Vec<TI>* __restrict__ in, Vec<TO>* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const Vec<TI> v = in[i];
    out[i] = cmake<Vec<TO>>(static_cast<TO>(v.x), static_cast<TO>(v.y));
  }
}

// Norm and position averages of the scattering plus specular wave in one block of 256 threads, FP64
// (src/propagation/averages.cpp:37-80). grids = [z (nz) | z_specular (nzs) | r (nr)]; densities are
// the block densities (izr = ir + nr iz). Seven sums, each strided per thread and then added in a
// fixed tree: the scattering norm, Z and r moments, the same three on the specular grid, and the
// specular norm between the analysis line (exclusive) and the analysis surface (inclusive).
// out = {norm, <Z>, <r>, rest norm}.
template <typename T>
__global__ void __launch_bounds__(256) averages_kernel(const double* __restrict__ densities, const Vec<T>* __restrict__ chi,
                                                       const double* __restrict__ grids, int nz, int nr, int nzs,
                                                       int iz_analysis, int surface_index, double vol_scat,
                                                       double vol_spec, double* __restrict__ out) {
  __shared__ double part[7][256];
  const double* zg = grids;
  const double* zsg = grids + nz;
  const double* rg = grids + nz + nzs;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const int n_scat = nz * nr;
  for (int izr = threadIdx.x; izr < n_scat; izr += blockDim.x) {
    const double d = densities[izr];
    acc[0] += d;
    acc[1] += zg[izr / nr] * d;
    acc[2] += rg[izr % nr] * d;
  }
  const int n_spec = nzs * nr;
  for (int k = threadIdx.x; k < n_spec; k += blockDim.x) {
    const int iz = k / nr;
    const int ir = k - iz * nr;
    const Vec<T> c = chi[k];
    const double re = c.x, im = c.y;
    const double d = re * re + im * im;
    acc[3] += d;
    acc[4] += zsg[iz] * d;
    acc[5] += rg[ir] * d;
    if (iz > iz_analysis && iz <= surface_index) acc[6] += d;
  }
#pragma unroll
  for (int q = 0; q < 7; ++q) part[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int q = 0; q < 7; ++q) part[q][threadIdx.x] += part[q][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double norm = part[0][0] * vol_scat + part[3][0] * vol_spec;
    out[0] = norm;
    out[1] = (part[1][0] * vol_scat + part[4][0] * vol_spec) / norm;
    out[2] = (part[2][0] * vol_scat + part[5][0] * vol_spec) / norm;
    out[3] = part[6][0] * vol_spec;
  }
}

}  // namespace spo
