// Persistent forms of the register kinetic kernels: a grid of (SMs x resident blocks) loops over the
// passes' tiles, and each thread requests the first-level values of its next tile into registers before
// it transforms the current one, so the loads of tile k + 1 overlap the DFTs and the stores of tile k.
// A tile's lines go through the operations of axis2_kernel / xy2_kernel (spo_regfft.cuh) in the same
// order; the forms agree to rounding (the compiler may contract the products of a complex multiply into
// FMAs differently in each kernel), so which one a pass uses is a fixed choice, not a timed one.
#pragma once

#include "spo_regfft.cuh"

namespace spo {

// T_Z or T_r as axis2_kernel (whole passes, no lane windows): tiles (outer o, lanes i0 .. i0 + TB) in the
// order o * lane_blocks + i0 / TB.
template <typename T, int N1, int N2, int TB>
__global__ void __launch_bounds__(TB*(N1 > N2 ? N1 : N2)) axis2p_kernel(Axis2Args<T> a, long long lane_blocks,
                                                                       long long n_tiles) {
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
  const long long stride = a.inner;
  auto locate = [&](long long tile, long long& base, bool& ok) {
    const long long o = tile / lane_blocks;
    const long long i0 = (tile - o * lane_blocks) * TB;
    base = o * N * a.inner + i0 + b;
    ok = i0 + b < a.inner;
  };
  auto fetch = [&](long long base, bool ok, V (&x)[N1]) {
    if (s < N2) {
      const int n2 = s;
      static_for<0, N1>([&](auto n1) {
        x[n1] = ok ? a.data[base + static_cast<long long>(n2 + N2 * n1) * stride] : cmake<V>(0, 0);
      });
    }
  };
  for (int k = threadIdx.x; k < kFParts * N; k += TB * NS) f[k] = a.factor[k];
  for (int k = threadIdx.x; k < kParts * N; k += TB * NS) tw[k] = a.tw[k];
  __syncthreads();
  long long tile = blockIdx.x, base = 0;
  bool lane_ok = false;
  V x[N1];
  if (tile < n_tiles) {
    locate(tile, base, lane_ok);
    fetch(base, lane_ok, x);
  }
  for (; tile < n_tiles; tile += gridDim.x) {
    const long long next = tile + gridDim.x;
    long long nbase = 0;
    bool nok = false;
    V xn[N1];
    if (next < n_tiles) {
      locate(next, nbase, nok);
      fetch(nbase, nok, xn);
    }
    // forward, level 1
    if (s < N2) {
      const int n2 = s;
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
      V z[N1];
      static_for<0, N1>([&](auto k1) { z[k1] = Y[(n2 * N1 + k1) * TB + b]; });
      rdft<N1, +1>(z);
      static_for<0, N1>([&](auto n1) { a.data[base + static_cast<long long>(n2 + N2 * n1) * stride] = z[n1]; });
    }
    __syncthreads();  // Y is read before the next tile's first level writes it
    static_for<0, N1>([&](auto n1) { x[n1] = xn[n1]; });
    base = nbase;
    lane_ok = nok;
  }
}

// T_xy as xy2_kernel over the points izr_offset .. izr_offset + n_zr: tiles (point, rotational states
// r0 .. r0 + TB) in the order p * rot_tiles + r0 / TB.
template <typename T, int NX, int NY, int TB>
__global__ void __launch_bounds__(TB*(NX > NY ? NX : NY)) xy2p_kernel(XyArgs<T> a, long long rot_tiles,
                                                                     long long n_tiles) {
  using V = Vec<T>;
  constexpr int NXY = NX * NY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kFParts = sizeof(T) == 4 ? kFactorParts : 1;  // the mixed form's factor parts (fmul_t)
  V* S = reinterpret_cast<V*>(smem_raw);  // NXY * TB
  V* f = S + NXY * TB;                     // NXY factors (the mixed form's parts)
  const int b = threadIdx.x % TB;
  const int s = threadIdx.x / TB;
  auto locate = [&](long long tile, long long& izr, int& irot, bool& ok) {
    const long long p = tile / rot_tiles;
    izr = a.izr_offset + p;
    irot = static_cast<int>(tile - p * rot_tiles) * TB + b;
    ok = irot < a.n_rot;
  };
  auto fetch = [&](long long izr, int irot, bool ok, V (&x)[NY]) {
    if (s < NX) {
      const int ix = s;
      const long long col0 = izr * NXY;
      static_for<0, NY>([&](auto iy) { x[iy] = ok ? a.psi[(col0 + ix * NY + iy) * a.n_rot + irot] : cmake<V>(0, 0); });
    }
  };
  for (int k = threadIdx.x; k < kFParts * NXY; k += blockDim.x) f[k] = a.factor[k];
  __syncthreads();
  long long tile = blockIdx.x, izr = 0;
  int irot = 0;
  bool lane_ok = false;
  V x[NY];
  if (tile < n_tiles) {
    locate(tile, izr, irot, lane_ok);
    fetch(izr, irot, lane_ok, x);
  }
  for (; tile < n_tiles; tile += gridDim.x) {
    const long long next = tile + gridDim.x;
    long long nizr = 0;
    int nirot = 0;
    bool nok = false;
    V xn[NY];
    if (next < n_tiles) {
      locate(next, nizr, nirot, nok);
      fetch(nizr, nirot, nok, xn);
    }
    const long long col0 = izr * NXY;
    if (s < NX) {
      const int ix = s;
      if (a.shift_f)
        static_for<0, NY>([&](auto iy) {
          if (lane_ok) x[iy] = fmul_t(x[iy], a.shift_f, NXY, ix * NY + iy);
        });
      rdft<NY, -1>(x);
      static_for<0, NY>([&](auto ky) { S[(ix * NY + ky) * TB + b] = x[ky]; });
    }
    __syncthreads();
    if (s < NY) {
      const int ky = s;
      V y[NX];
      static_for<0, NX>([&](auto ix) { y[ix] = S[(ix * NY + ky) * TB + b]; });
      rdft<NX, -1>(y);
      static_for<0, NX>([&](auto kx) { y[kx] = fmul_t(y[kx], f, NXY, kx * NY + ky); });
      rdft<NX, +1>(y);
      static_for<0, NX>([&](auto ix) { S[(ix * NY + ky) * TB + b] = y[ix]; });
    }
    __syncthreads();
    if (s < NX && lane_ok) {
      const int ix = s;
      V z[NY];
      static_for<0, NY>([&](auto ky) { z[ky] = S[(ix * NY + ky) * TB + b]; });
      rdft<NY, +1>(z);
      const bool gas = a.apply_gas && izr >= a.izr_gas_first;
      const int ir = static_cast<int>(izr % a.nr);
      const long long n_gas = static_cast<long long>(a.nr) * a.n_rot, k_gas = ir * a.n_rot + irot;
      const T oz = gas ? a.opt_z[izr / a.nr] : T(1);
      static_for<0, NY>([&](auto iy) {
        V v = z[iy];
        if (a.shift_b) v = fmul_t(v, a.shift_b, NXY, ix * NY + iy);
        if (gas) v = cscale(fmul_t(v, a.gas_step, n_gas, k_gas), oz);
        a.psi[(col0 + ix * NY + iy) * a.n_rot + irot] = v;
      });
    }
    __syncthreads();  // S is read before the next tile's first level writes it
    static_for<0, NY>([&](auto iy) { x[iy] = xn[iy]; });
    izr = nizr;
    irot = nirot;
    lane_ok = nok;
  }
}

}  // namespace spo

namespace spo {

// T_Z or T_r as axis2_kernel for N2 = 2 N1 (whole passes, no lane windows), with every thread busy in
// both levels: TB x N1 threads; thread (b, s) takes the first-level lines n2 = s and s + N1 of lane b
// (two DFT_N1) and the second-level line k1 = s (one DFT_N2). In axis2_kernel (TB x N2 threads) half of
// the threads wait at the barrier during the second level. Dynamic shared memory as axis2_kernel.
// Mixed form: registers capped for SPO_AXIS2B_SM_THREADS resident threads per SM (default 1024: eight
// blocks of 128 threads; the pass waits on its global loads, and 64 registers with a 64-byte spill took
// Z = 128 from 1.38 to 1.29 ms on configuration 3).
#ifndef SPO_AXIS2B_SM_THREADS
#define SPO_AXIS2B_SM_THREADS 1024
#endif
template <typename T, int N1, int N2, int TB>
__global__ void __launch_bounds__(TB * N1, sizeof(T) == 4 ? SPO_AXIS2B_SM_THREADS / (TB * N1) : 1) axis2b_kernel(Axis2Args<T> a) {
  using V = Vec<T>;
  static_assert(N2 == 2 * N1, "the balanced form needs N2 = 2 N1");
  constexpr int N = N1 * N2;
  constexpr int kParts = sizeof(T) == 4 ? 2 : 1;         // twiddles: value (then low part)
  constexpr int kFParts = sizeof(T) == 4 ? kFactorParts : 1;  // factors: see fmul_t
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* Y = reinterpret_cast<V*>(smem_raw);
  V* f = Y + N * TB;       // N factors (the mixed form's parts, see fmul_t)
  V* tw = f + kFParts * N;  // N twiddles (then N low parts)
  const int b = threadIdx.x % TB;
  const int s = threadIdx.x / TB;
  const long long i0 = static_cast<long long>(blockIdx.x) * TB;
  const long long base = static_cast<long long>(blockIdx.y) * N * a.inner + i0 + b;
  const long long stride = a.inner;
  const bool lane_ok = i0 + b < a.inner;
  for (int k = threadIdx.x; k < kFParts * N; k += TB * N1) f[k] = a.factor[k];
  for (int k = threadIdx.x; k < kParts * N; k += TB * N1) tw[k] = a.tw[k];
  __syncthreads();
  // forward, level 1: lines n2 = s, s + N1
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int n2 = s + h * N1;
    V x[N1];
    static_for<0, N1>([&](auto n1) {
      x[n1] = lane_ok ? a.data[base + static_cast<long long>(n2 + N2 * n1) * stride] : cmake<V>(0, 0);
    });
    rdft<N1, -1>(x);
    static_for<0, N1>([&](auto k1) { Y[(n2 * N1 + k1) * TB + b] = k1 == 0 ? x[k1] : tw_mul<N>(x[k1], tw[n2 * k1], lo_part(tw, N, n2 * k1)); });
  }
  __syncthreads();
  // forward level 2, factor, inverse level 2: line k1 = s
  {
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
  // inverse level 1, store: lines n2 = s, s + N1
  if (lane_ok) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n2 = s + h * N1;
      V x[N1];
      static_for<0, N1>([&](auto k1) { x[k1] = Y[(n2 * N1 + k1) * TB + b]; });
      rdft<N1, +1>(x);
      static_for<0, N1>([&](auto n1) { a.data[base + static_cast<long long>(n2 + N2 * n1) * stride] = x[n1]; });
    }
  }
}

}  // namespace spo
