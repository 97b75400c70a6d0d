// Device-side ZFP block codec for sm_100a: one thread codes one 4^d block.
//
// The stream format and every arithmetic step follow zfp-rs 1.0.1:
//   lifting transforms        src/codec/transform.rs:74-233
//   cast, rounding, negabinary src/codec/encode/core.rs:53-423
//   embedded bit-plane coder  src/codec/bitplane.rs:509-790
//   block coders              src/codec/encode/{float,integer,reversible}.rs,
//                             src/codec/decode/{core,reversible}.rs
// The implementation is GPU-shaped: coefficients live in registers (all
// indices compile-time after unrolling), bit planes are produced by an
// in-register bit-matrix transpose and kept in a per-thread slice of shared
// memory for the data-dependent plane loop, and stream words are assembled in
// a 64-bit register before a single store.
#pragma once

#include <cstdint>
#include <type_traits>
#include <utility>

#include "zfpb_engine.h"

namespace zfpb {

typedef unsigned long long u64;
typedef unsigned int u32;
typedef long long i64;

#define ZFPB_DEV __device__ __forceinline__

// ---------------------------------------------------------------------------
// Scalar traits (zfp-rs src/types.rs:327-344, encode/core.rs:309-325)
// ---------------------------------------------------------------------------

template <class T> struct Traits;
template <> struct Traits<float> {
  typedef int I; typedef u32 U;
  static constexpr int EBITS = 8, EBIAS = 127, PREC = 32, PBITS = 5, MIN_CAST_EMAX = -97;
  static constexpr bool FLOAT = true;
};
template <> struct Traits<double> {
  typedef i64 I; typedef u64 U;
  static constexpr int EBITS = 11, EBIAS = 1023, PREC = 64, PBITS = 6, MIN_CAST_EMAX = -961;
  static constexpr bool FLOAT = true;
};
template <> struct Traits<int> {
  typedef int I; typedef u32 U;
  static constexpr int EBITS = 0, EBIAS = 0, PREC = 32, PBITS = 5, MIN_CAST_EMAX = 0;
  static constexpr bool FLOAT = false;
};
template <> struct Traits<i64> {
  typedef i64 I; typedef u64 U;
  static constexpr int EBITS = 0, EBIAS = 0, PREC = 64, PBITS = 6, MIN_CAST_EMAX = 0;
  static constexpr bool FLOAT = false;
};

// Parameters of one compress/decompress call (zfp-rs src/config.rs:163-174):
// minbits, maxbits, maxprec, minexp, rounding (0 never, 1 first, 2 last), tight.
typedef CodecParams Codec;

static constexpr int ZFP_MIN_EXP = -1074;

// ---------------------------------------------------------------------------
// Coefficient order (zfp-rs src/codec/encode/core.rs:12-39).  These tables
// are the stream format; they are evaluated at compile time after unrolling.
// ---------------------------------------------------------------------------

__host__ __device__ constexpr int perm2(int i) {
  constexpr unsigned char t[16] = {0, 1, 4, 5, 2, 8, 6, 9, 3, 12, 10, 7, 13, 11, 14, 15};
  return t[i];
}
__host__ __device__ constexpr int perm3(int i) {
  constexpr unsigned char t[64] = {
      0,  1,  4,  16, 20, 17, 5,  2,  8,  32, 21, 6,  18, 24, 9,  33, 36, 3,  12, 48, 22, 25,
      37, 40, 34, 10, 7,  19, 28, 13, 49, 52, 41, 38, 26, 23, 29, 53, 11, 35, 44, 14, 50, 56,
      42, 27, 39, 45, 30, 54, 57, 60, 51, 15, 43, 46, 58, 61, 55, 31, 62, 59, 47, 63};
  return t[i];
}
__device__ const unsigned char kPerm4[256] = {
    0,   1,   4,   16,  64,  5,   80,  17,  68,  65,  20,  2,   8,   32,  128, 84,  81,  69,  21,
    6,   18,  66,  24,  72,  9,   96,  33,  36,  129, 132, 144, 3,   12,  48,  192, 85,  82,  70,
    22,  73,  25,  88,  37,  100, 97,  148, 145, 133, 10,  160, 34,  136, 130, 40,  7,   19,  67,
    28,  76,  13,  112, 49,  52,  193, 196, 208, 86,  89,  101, 149, 161, 137, 41,  134, 38,  164,
    26,  152, 146, 104, 98,  74,  83,  71,  23,  77,  29,  92,  53,  116, 113, 212, 209, 197, 11,
    35,  131, 44,  140, 14,  176, 50,  56,  194, 200, 224, 90,  165, 102, 153, 150, 105, 168, 162,
    138, 42,  87,  93,  117, 213, 27,  75,  99,  39,  135, 147, 108, 45,  141, 156, 30,  78,  177,
    180, 54,  114, 120, 57,  198, 210, 216, 201, 225, 228, 15,  240, 51,  204, 195, 60,  169, 166,
    154, 106, 91,  103, 151, 109, 157, 94,  181, 118, 121, 214, 217, 229, 163, 139, 43,  142, 46,
    172, 58,  184, 178, 232, 226, 202, 241, 205, 61,  199, 55,  244, 31,  220, 211, 124, 115, 79,
    170, 167, 155, 107, 158, 110, 173, 122, 185, 182, 233, 230, 218, 95,  245, 119, 221, 215, 125,
    242, 206, 62,  203, 59,  248, 47,  236, 227, 188, 179, 143, 171, 174, 186, 234, 246, 222, 126,
    219, 123, 249, 111, 237, 231, 189, 183, 159, 252, 243, 207, 63,  175, 250, 187, 238, 235, 190,
    253, 247, 223, 127, 254, 251, 239, 191, 255};

template <class I> ZFPB_DEV typename Traits<I>::U int2uint(I x);
ZFPB_DEV int uint2int(u32 x);
ZFPB_DEV i64 uint2int(u64 x);

template <int N> ZFPB_DEV int perm_at(int i) {
  if constexpr (N == 4) return i;
  else if constexpr (N == 16) return perm2(i);
  else if constexpr (N == 64) return perm3(i);
  else return kPerm4[i];
}

// Compile-time loop: f(std::integral_constant<int, i>) for i in [0, N), so
// that table lookups indexed by i are constant expressions.
template <class F, int... Is>
ZFPB_DEV void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, class F> ZFPB_DEV void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// u[i] = int2uint(b[perm[i]]) (encode/core.rs:98-109) and its inverse
// b[perm[i]] = uint2int(u[i]) (decode/core.rs:40-51).
template <int N, class I, class U> ZFPB_DEV void fwd_order(U* u, const I* b) {
  if constexpr (N == 256) {
    for (int i = 0; i < N; i++) u[i] = int2uint(b[kPerm4[i]]);
  } else {
    static_for<N>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int p = N == 4 ? i : N == 16 ? perm2(i) : perm3(i);
      u[i] = int2uint(b[p]);
    });
  }
}
template <int N, class I, class U> ZFPB_DEV void inv_order(const U* u, I* b) {
  if constexpr (N == 256) {
    for (int i = 0; i < N; i++) b[kPerm4[i]] = uint2int(u[i]);
  } else {
    static_for<N>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int p = N == 4 ? i : N == 16 ? perm2(i) : perm3(i);
      b[p] = uint2int(u[i]);
    });
  }
}

// ---------------------------------------------------------------------------
// Exact powers of two by exponent-field construction (no libm): 2^n rounded
// to the format, i.e. subnormal below the normal range, 0 below half the
// smallest subnormal, infinity above the largest finite exponent.
// ---------------------------------------------------------------------------

ZFPB_DEV float pow2f(int n) {
  if (n > 127) return __int_as_float(0x7f800000);
  if (n >= -126) return __int_as_float((n + 127) << 23);
  if (n >= -149) return __int_as_float(1 << (n + 149));
  return 0.0f;
}
ZFPB_DEV double pow2d(int n) {
  if (n > 1023) return __longlong_as_double(0x7ff0000000000000ll);
  if (n >= -1022) return __longlong_as_double((i64)(n + 1023) << 52);
  if (n >= -1074) return __longlong_as_double(1ll << (n + 1074));
  return 0.0;
}
template <class T> ZFPB_DEV T pow2(int n);
template <> ZFPB_DEV float pow2<float>(int n) { return pow2f(n); }
template <> ZFPB_DEV double pow2<double>(int n) { return pow2d(n); }

ZFPB_DEV u32 bits_of(float f) { return (u32)__float_as_int(f); }
ZFPB_DEV u64 bits_of(double f) { return (u64)__double_as_longlong(f); }
ZFPB_DEV float float_of(u32 u) { return __int_as_float((int)u); }
ZFPB_DEV double float_of(u64 u) { return __longlong_as_double((i64)u); }

// x86-64 truncation (zfp-rs encode/core.rs:385-423): out of range or NaN gives
// the minimum integer.  Explicit round-toward-zero conversions after the range
// check, so the result does not depend on the hardware's saturation rule.
ZFPB_DEV int trunc_i(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? __float2int_rz(v) : (int)0x80000000;
}
ZFPB_DEV i64 trunc_i(double v) {
  return (v >= -9223372036854775808.0 && v < 9223372036854775808.0) ? __double2ll_rz(v)
                                                                       : (i64)0x8000000000000000ll;
}
// Round-to-nearest integer -> float conversions (decode/core.rs:162-175).
ZFPB_DEV float to_float(int i) { return __int2float_rn(i); }
ZFPB_DEV double to_float(i64 i) { return __ll2double_rn(i); }
ZFPB_DEV float mul_rn(float a, float b) { return __fmul_rn(a, b); }
ZFPB_DEV double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// ---------------------------------------------------------------------------
// Lifting transforms with two's-complement wraparound (transform.rs:74-142)
// ---------------------------------------------------------------------------

template <class I> ZFPB_DEV I wadd(I a, I b) {
  typedef typename Traits<I>::U U;
  return (I)((U)a + (U)b);
}
template <class I> ZFPB_DEV I wsub(I a, I b) {
  typedef typename Traits<I>::U U;
  return (I)((U)a - (U)b);
}

template <class I> ZFPB_DEV void fwd_lift(I& x, I& y, I& z, I& w) {
  x = wadd(x, w) >> 1; w = wsub(w, x);
  z = wadd(z, y) >> 1; y = wsub(y, z);
  x = wadd(x, z) >> 1; z = wsub(z, x);
  w = wadd(w, y) >> 1; y = wsub(y, w);
  w = wadd(w, (I)(y >> 1));
  y = wsub(y, (I)(w >> 1));
}
template <class I> ZFPB_DEV void inv_lift(I& x, I& y, I& z, I& w) {
  y = wadd(y, (I)(w >> 1));
  w = wsub(w, (I)(y >> 1));
  y = wadd(y, w);
  w = wsub(w, wsub(y, w));
  z = wadd(z, x);
  x = wsub(x, wsub(z, x));
  y = wadd(y, z);
  z = wsub(z, wsub(y, z));
  w = wadd(w, x);
  x = wsub(x, wsub(w, x));
}
template <class I> ZFPB_DEV void rev_fwd_lift(I& x, I& y, I& z, I& w) {
  w = wsub(w, z); z = wsub(z, y); y = wsub(y, x);
  w = wsub(w, z); z = wsub(z, y); w = wsub(w, z);
}
template <class I> ZFPB_DEV void rev_inv_lift(I& x, I& y, I& z, I& w) {
  w = wadd(w, z); z = wadd(z, y); w = wadd(w, z);
  y = wadd(y, x); z = wadd(z, y); w = wadd(w, z);
}

// Lift every line of stride S in a block of N values (transform.rs:151-170).
template <class I, int N, int S, int KIND> ZFPB_DEV void lift_axis(I* p) {
#pragma unroll
  for (int g = 0; g < N; g += 4 * S) {
#pragma unroll
    for (int i = g; i < g + S; i++) {
      if constexpr (KIND == 0) fwd_lift(p[i], p[i + S], p[i + 2 * S], p[i + 3 * S]);
      else if constexpr (KIND == 1) inv_lift(p[i], p[i + S], p[i + 2 * S], p[i + 3 * S]);
      else if constexpr (KIND == 2) rev_fwd_lift(p[i], p[i + S], p[i + 2 * S], p[i + 3 * S]);
      else rev_inv_lift(p[i], p[i + S], p[i + 2 * S], p[i + 3 * S]);
    }
  }
}
// Forward: axes x, y, z, w; inverse: w, z, y, x (transform.rs:174-233).
template <class I, int N, int KIND> ZFPB_DEV void fwd_axes(I* p) {
  lift_axis<I, N, 1, KIND>(p);
  if constexpr (N >= 16) lift_axis<I, N, 4, KIND>(p);
  if constexpr (N >= 64) lift_axis<I, N, 16, KIND>(p);
  if constexpr (N >= 256) lift_axis<I, N, 64, KIND>(p);
}
template <class I, int N, int KIND> ZFPB_DEV void inv_axes(I* p) {
  if constexpr (N >= 256) lift_axis<I, N, 64, KIND>(p);
  if constexpr (N >= 64) lift_axis<I, N, 16, KIND>(p);
  if constexpr (N >= 16) lift_axis<I, N, 4, KIND>(p);
  lift_axis<I, N, 1, KIND>(p);
}

// ---------------------------------------------------------------------------
// Negabinary and rounding (encode/core.rs:53-91, decode/core.rs:21-82)
// ---------------------------------------------------------------------------

template <class U> ZFPB_DEV U nbmask() { return (U)0xaaaaaaaaaaaaaaaaull; }

template <class I> ZFPB_DEV typename Traits<I>::U int2uint(I x) {
  typedef typename Traits<I>::U U;
  return (U)((U)x + nbmask<U>()) ^ nbmask<U>();
}
ZFPB_DEV int uint2int(u32 x) { return (int)((x ^ 0xaaaaaaaau) - 0xaaaaaaaau); }
ZFPB_DEV i64 uint2int(u64 x) { return (i64)((x ^ 0xaaaaaaaaaaaaaaaaull) - 0xaaaaaaaaaaaaaaaaull); }

template <class I, int N> ZFPB_DEV void fwd_round(I* b, u32 maxprec) {
  typedef typename Traits<I>::U U;
  constexpr u32 B = sizeof(U) * 8;
  if (maxprec < B) {
    I bias = (I)((U)(nbmask<U>() >> 2) >> maxprec);
    if (!(maxprec & 1)) bias = wsub((I)0, bias);
#pragma unroll
    for (int i = 0; i < N; i++) b[i] = wadd(b[i], bias);
  }
}

template <class U, int N> ZFPB_DEV void inv_round(U* d, u32 m, u32 prec) {
  constexpr u32 B = sizeof(U) * 8;
  if (prec < B - 1) {
    U hi = (U)(nbmask<U>() >> 2) >> prec;
    U lo = (U)(nbmask<U>() >> 1) >> prec;
#pragma unroll
    for (int i = 0; i < N; i++) d[i] += ((u32)i < m) ? hi : lo;
  }
}

ZFPB_DEV bool with_maxbits(u32 maxbits, u32 maxprec, u32 size) {
  return ((u64)maxprec + 1) * (u64)size > (u64)maxbits + 1;
}

// encode/core.rs:231-244
ZFPB_DEV u32 precision_f(int maxexp, u32 maxprec, int minexp, u32 dims, bool tight) {
  i64 raw = (i64)maxexp - (i64)minexp + 2 * (i64)dims + (tight ? 1 : 2);
  raw = raw < 0 ? 0 : raw;
  raw = raw > (i64)maxprec ? (i64)maxprec : raw;
  return (u32)raw;
}

ZFPB_DEV u32 sat_sub(u32 a, u32 b) { return a > b ? a - b : 0u; }

// ---------------------------------------------------------------------------
// Block-floating-point (encode/core.rs:251-380, decode/core.rs:162-175)
// ---------------------------------------------------------------------------

// frexp exponent of the largest |x|, NaNs skipped: fmax ignores a NaN operand.
template <class T, int N> ZFPB_DEV int exponent_block(const T* d) {
  T m = 0;
#pragma unroll
  for (int i = 0; i < N; i++) m = fmax(m, fabs(d[i]));
  auto b = bits_of(m);
  if constexpr (sizeof(T) == 4) {
    u32 e = b >> 23;
    return b == 0 ? -127 : (e == 0xff ? 0 : (int)e - 126);
  } else {
    u32 e = (u32)(b >> 52);
    return b == 0 ? -1023 : (e == 0x7ff ? 0 : (int)e - 1022);
  }
}

template <class T, int N>
ZFPB_DEV void fwd_cast(typename Traits<T>::I* ib, const T* fb, int emax) {
  constexpr int ip = Traits<T>::PREC;
  if (emax < Traits<T>::MIN_CAST_EMAX) {
    // Two exact steps for blocks whose one-step scale overflows.
    T s = pow2<T>(ip - 2 - 64 - emax);
    T two64 = pow2<T>(64);
#pragma unroll
    for (int i = 0; i < N; i++) ib[i] = trunc_i(mul_rn(mul_rn(fb[i], two64), s));
  } else {
    T s = pow2<T>(ip - 2 - emax);
#pragma unroll
    for (int i = 0; i < N; i++) ib[i] = trunc_i(mul_rn(s, fb[i]));
  }
}

template <class T, int N>
ZFPB_DEV void inv_cast(const typename Traits<T>::I* ib, T* fb, int emax) {
  constexpr int ip = Traits<T>::PREC;
  T s = pow2<T>(emax - (ip - 2));
#pragma unroll
  for (int i = 0; i < N; i++) fb[i] = mul_rn(s, to_float(ib[i]));
}

// ---------------------------------------------------------------------------
// Bit-matrix transposes (Hacker's Delight 7-3, as bitplane.rs:75-92): row i
// is a[i], column c is bit c.
// ---------------------------------------------------------------------------

// The stages that move whole bytes (J = 32, 16, 8) are byte permutations of
// each pair of rows: with rows (a, b) and J = 16, the new a takes the low
// halves of a and b and the new b their high halves (J = 8: the even and the
// odd bytes; J = 32: the low and high 32-bit words).  __byte_perm does one
// 32-bit word of that in one instruction.
ZFPB_DEV void bperm_pair(u32& a, u32& b, u32 sel_a, u32 sel_b) {
  const u32 x = __byte_perm(a, b, sel_a), y = __byte_perm(a, b, sel_b);
  a = x;
  b = y;
}
template <int J> ZFPB_DEV void byte_stage_pair(u32& a, u32& b) {
  if constexpr (J == 16) bperm_pair(a, b, 0x5410, 0x7632);
  else bperm_pair(a, b, 0x6240, 0x7351);
}
template <int J> ZFPB_DEV void byte_stage_pair(u64& a, u64& b) {
  u32 al = (u32)a, ah = (u32)(a >> 32), bl = (u32)b, bh = (u32)(b >> 32);
  if constexpr (J == 32) {
    a = (u64)al | ((u64)bl << 32);
    b = (u64)ah | ((u64)bh << 32);
  } else {
    byte_stage_pair<J>(al, bl);
    byte_stage_pair<J>(ah, bh);
    a = (u64)al | ((u64)ah << 32);
    b = (u64)bl | ((u64)bh << 32);
  }
}

template <class W, int J> ZFPB_DEV void transpose_stage(W* a, int R) {
  if constexpr (J >= 8) {
#pragma unroll
    for (int k = 0; k < 64; k += 2 * J) {
      if (k >= R) break;
#pragma unroll
      for (int i = k; i < k + J; i++) byte_stage_pair<J>(a[i], a[i + J]);
    }
    return;
  }
  W m;
  if constexpr (J == 32) m = (W)0x00000000ffffffffull;
  else if constexpr (J == 16) m = (W)0x0000ffff0000ffffull;
  else if constexpr (J == 8) m = (W)0x00ff00ff00ff00ffull;
  else if constexpr (J == 4) m = (W)0x0f0f0f0f0f0f0f0full;
  else if constexpr (J == 2) m = (W)0x3333333333333333ull;
  else m = (W)0x5555555555555555ull;
#pragma unroll
  for (int k = 0; k < 64; k += 2 * J) {
    if (k >= R) break;
#pragma unroll
    for (int i = k; i < k + J; i++) {
      W t = ((a[i] >> J) ^ a[i + J]) & m;
      a[i] ^= t << J;
      a[i + J] ^= t;
    }
  }
}

// Stages are separate instantiations so every index is a compile-time
// constant and the matrix stays in registers.
template <class W, int R> ZFPB_DEV void transpose(W* a) {
  if constexpr (R >= 64) transpose_stage<W, 32>(a, R);
  transpose_stage<W, 16>(a, R);
  transpose_stage<W, 8>(a, R);
  transpose_stage<W, 4>(a, R);
  transpose_stage<W, 2>(a, R);
  transpose_stage<W, 1>(a, R);
}

// Per-thread plane storage in shared memory: plane k, word c of thread t is
// at base[(k * W + c) * stride + t]; consecutive threads hit consecutive
// words, so a warp's accesses are bank-conflict free.
struct PlaneStore {
  u64* base;
  int stride;
  ZFPB_DEV u64& at(int k, int c, int W) const { return base[(size_t)(k * W + c) * stride]; }
};

// Coefficients -> bit planes k = 0..PREC-1 (plane k, bit i = bit k of u[i]).
template <class U, int N> ZFPB_DEV void store_planes(const U* u, PlaneStore ps) {
  constexpr int P = sizeof(U) * 8;
  constexpr int W = N <= 64 ? 1 : N / 64;
  if constexpr (N == 4) {
#pragma unroll
    for (int k = 0; k < P; k++) {
      u64 x = 0;
#pragma unroll
      for (int i = 0; i < 4; i++) x |= (u64)((u[i] >> k) & 1) << i;
      ps.at(k, 0, 1) = x;
    }
  } else if constexpr (sizeof(U) == 4 && N == 16) {
    u32 a[32];
#pragma unroll
    for (int i = 0; i < 32; i++) a[i] = i < 16 ? u[i] : 0u;
    transpose<u32, 32>(a);
#pragma unroll
    for (int k = 0; k < 32; k++) ps.at(k, 0, 1) = a[k];
  } else if constexpr (sizeof(U) == 4) {
    // 64 coefficients per chunk, as two 32x32 transposes.
#pragma unroll
    for (int c = 0; c < W; c++) {
      u32 lo[32], hi[32];
#pragma unroll
      for (int i = 0; i < 32; i++) {
        lo[i] = u[64 * c + i];
        hi[i] = u[64 * c + 32 + i];
      }
      transpose<u32, 32>(lo);
      transpose<u32, 32>(hi);
#pragma unroll
      for (int k = 0; k < 32; k++) ps.at(k, c, W) = (u64)lo[k] | ((u64)hi[k] << 32);
    }
  } else {
#pragma unroll
    for (int c = 0; c < W; c++) {
      u64 a[64];
#pragma unroll
      for (int i = 0; i < 64; i++) a[i] = (64 * c + i) < N ? (u64)u[64 * c + i] : 0ull;
      transpose<u64, 64>(a);
#pragma unroll
      for (int k = 0; k < 64; k++) ps.at(k, c, W) = a[k];
    }
  }
}

// Bit planes -> coefficients; planes outside [lo, hi] are zero.
template <class U, int N> ZFPB_DEV void load_planes(U* u, PlaneStore ps, int lo, int hi) {
  constexpr int P = sizeof(U) * 8;
  constexpr int W = N <= 64 ? 1 : N / 64;
  if constexpr (N == 4) {
#pragma unroll
    for (int i = 0; i < 4; i++) u[i] = 0;
#pragma unroll
    for (int k = 0; k < P; k++) {
      u64 x = (k >= lo && k <= hi) ? ps.at(k, 0, 1) : 0ull;
#pragma unroll
      for (int i = 0; i < 4; i++) u[i] |= (U)((x >> i) & 1) << k;
    }
  } else if constexpr (sizeof(U) == 4 && N == 16) {
    u32 a[32];
#pragma unroll
    for (int k = 0; k < 32; k++) a[k] = (k >= lo && k <= hi) ? (u32)ps.at(k, 0, 1) : 0u;
    transpose<u32, 32>(a);
#pragma unroll
    for (int i = 0; i < 16; i++) u[i] = a[i];
  } else if constexpr (sizeof(U) == 4) {
#pragma unroll
    for (int c = 0; c < W; c++) {
      u32 a[32], b[32];
#pragma unroll
      for (int k = 0; k < 32; k++) {
        u64 x = (k >= lo && k <= hi) ? ps.at(k, c, W) : 0ull;
        a[k] = (u32)x;
        b[k] = (u32)(x >> 32);
      }
      transpose<u32, 32>(a);
      transpose<u32, 32>(b);
#pragma unroll
      for (int i = 0; i < 32; i++) {
        u[64 * c + i] = a[i];
        u[64 * c + 32 + i] = b[i];
      }
    }
  } else {
#pragma unroll
    for (int c = 0; c < W; c++) {
      u64 a[64];
#pragma unroll
      for (int k = 0; k < 64; k++) a[k] = (k >= lo && k <= hi) ? ps.at(k, c, W) : 0ull;
      transpose<u64, 64>(a);
#pragma unroll
      for (int i = 0; i < 64; i++)
        if (64 * c + i < N) u[64 * c + i] = a[i];
    }
  }
}

// ---- narrow plane ranges of 64-bit blocks ----------------------------------
//
// A block of 64 coefficients of 64 bits codes only planes [kmin, top): those
// below kmin = 64 - precision are dropped and none at or above top (one above
// the highest one-bit) is set.  Fixed-precision streams of at most 32 planes
// (and low-precision blocks of fixed-accuracy streams) span at most 32 planes,
// so the 32-bit words u >> kmin hold every coded bit and two 32x32 transposes
// give the planes: about a third of the 64x64 transpose's work, in 32-bit
// instead of 64-bit operations.  The choice is made for a whole warp at once
// (every thread of it narrow, else all wide), so the warp runs one transpose.

// Planes kmin .. kmin + 31 (those below 64) of u, which has no bit at or
// above kmin + 32.
template <class U, int N> ZFPB_DEV void store_planes_narrow(const U* u, PlaneStore ps, u32 kmin) {
  static_assert(sizeof(U) == 8 && N == 64, "64 coefficients of 64 bits");
  u32 lo[32], hi[32];
#pragma unroll
  for (int i = 0; i < 32; i++) {
    lo[i] = (u32)(u[i] >> kmin);
    hi[i] = (u32)(u[32 + i] >> kmin);
  }
  transpose<u32, 32>(lo);
  transpose<u32, 32>(hi);
#pragma unroll
  for (int j = 0; j < 32; j++)
    if (kmin + j < 64) ps.at((int)kmin + j, 0, 1) = (u64)lo[j] | ((u64)hi[j] << 32);
}

// Bit planes of the coded range [kmin, top) into ps: the narrow form when
// every thread of the warp allows it.
template <class U, int N> ZFPB_DEV void store_coded_planes(const U* u, PlaneStore ps, u32 kmin, u32 top) {
  if constexpr (sizeof(U) == 8 && N == 64) {
    if (__all_sync(__activemask(), kmin < 64 && top <= kmin + 32)) {  // kmin 64: no plane coded
      store_planes_narrow<U, N>(u, ps, kmin);
      return;
    }
  }
  store_planes<U, N>(u, ps);
}

// Coefficients from the stored planes [lo, hi] (hi - lo < 32).
template <class U, int N> ZFPB_DEV void load_planes_narrow(U* u, PlaneStore ps, int lo, int hi) {
  static_assert(sizeof(U) == 8 && N == 64, "64 coefficients of 64 bits");
  u32 a[32], b[32];
#pragma unroll
  for (int k = 0; k < 32; k++) {
    const u64 x = lo + k <= hi ? ps.at(lo + k, 0, 1) : 0ull;
    a[k] = (u32)x;
    b[k] = (u32)(x >> 32);
  }
  transpose<u32, 32>(a);
  transpose<u32, 32>(b);
#pragma unroll
  for (int i = 0; i < 32; i++) {
    u[i] = (U)a[i] << lo;
    u[32 + i] = (U)b[i] << lo;
  }
}

// Coefficients from the stored planes [lo, hi] (planes outside it zero): the
// narrow form when every thread of the warp allows it.
template <class U, int N> ZFPB_DEV void load_coded_planes(U* u, PlaneStore ps, int lo, int hi) {
  if constexpr (sizeof(U) == 8 && N == 64) {
    if (__all_sync(__activemask(), hi - lo < 32)) {
      load_planes_narrow<U, N>(u, ps, lo, hi);
      return;
    }
  }
  load_planes<U, N>(u, ps, lo, hi);
}

// ---- register planes of 4-value blocks ------------------------------------
//
// A 1D block's P = bits-of-U planes are 4 bits each, so all of them fit in
// P / 16 registers as a nibble string: plane k is nibble P - 1 - k (bit i of
// the nibble is bit k of u[i]).  Planes are coded from the top down, so a run
// of planes is a contiguous run of nibbles, in the order the stream carries a
// verbatim run.  Word w of the string holds nibbles 16w .. 16w + 15.

// Swaps bits a and a + D of x for every position a in the mask.
template <int D> ZFPB_DEV u64 delta_swap(u64 x, u64 mask) {
  const u64 t = ((x >> D) ^ x) & mask;
  return x ^ t ^ (t << D);
}

// Nibble-major (bit 4j + i) to lane-major (bit 16i + j): the 6 index bits
// [j3 j2 j1 j0 i1 i0] rotate to [i1 i0 j3 j2 j1 j0], as two 3-cycles of index
// bits, each two transpositions (index bits p < q swap with D = 2^q - 2^p on
// the positions whose bit p is 1 and bit q is 0).
ZFPB_DEV u64 nibbles_to_lanes(u64 x) {
  x = delta_swap<15>(x, 0x0000AAAA0000AAAAull);  // index bits 0, 4
  x = delta_swap<3>(x, 0x0A0A0A0A0A0A0A0Aull);   // 0, 2
  x = delta_swap<30>(x, 0x00000000CCCCCCCCull);  // 1, 5
  x = delta_swap<6>(x, 0x00CC00CC00CC00CCull);   // 1, 3
  return x;
}

ZFPB_DEV u64 lanes_to_nibbles(u64 x) {
  x = delta_swap<6>(x, 0x00CC00CC00CC00CCull);
  x = delta_swap<30>(x, 0x00000000CCCCCCCCull);
  x = delta_swap<3>(x, 0x0A0A0A0A0A0A0A0Aull);
  x = delta_swap<15>(x, 0x0000AAAA0000AAAAull);
  return x;
}

ZFPB_DEV u32 rev32(u32 x) {
#ifdef __CUDA_ARCH__
  return __brev(x);
#else
  x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
  x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
  x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
  x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
  return (x >> 16) | (x << 16);
#endif
}

// Low 16 bits of a, then low 16 bits of b (LO) or the high halves (HI).
ZFPB_DEV u32 pair_lo16(u32 a, u32 b) { return (a & 0xffffu) | (b << 16); }
ZFPB_DEV u32 pair_hi16(u32 a, u32 b) { return (a >> 16) | (b & 0xffff0000u); }

// u[0..3] -> the nibble string q[0 .. P/16).
template <class U> ZFPB_DEV void store_nibbles(const U* u, u64* q) {
  if constexpr (sizeof(U) == 4) {
    // t_i = reversed u[i]: bit m of t_i is bit i of nibble m.
    const u32 t0 = rev32(u[0]), t1 = rev32(u[1]), t2 = rev32(u[2]), t3 = rev32(u[3]);
    q[0] = lanes_to_nibbles((u64)pair_lo16(t0, t1) | ((u64)pair_lo16(t2, t3) << 32));
    q[1] = lanes_to_nibbles((u64)pair_hi16(t0, t1) | ((u64)pair_hi16(t2, t3) << 32));
  } else {
    u32 lo[4], hi[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      lo[i] = rev32((u32)((u64)u[i] >> 32));  // nibbles 0..31 come from the high half
      hi[i] = rev32((u32)u[i]);
    }
    q[0] = lanes_to_nibbles((u64)pair_lo16(lo[0], lo[1]) | ((u64)pair_lo16(lo[2], lo[3]) << 32));
    q[1] = lanes_to_nibbles((u64)pair_hi16(lo[0], lo[1]) | ((u64)pair_hi16(lo[2], lo[3]) << 32));
    q[2] = lanes_to_nibbles((u64)pair_lo16(hi[0], hi[1]) | ((u64)pair_lo16(hi[2], hi[3]) << 32));
    q[3] = lanes_to_nibbles((u64)pair_hi16(hi[0], hi[1]) | ((u64)pair_hi16(hi[2], hi[3]) << 32));
  }
}

// The nibble string q -> u[0..3].
template <class U> ZFPB_DEV void load_nibbles(U* u, const u64* q) {
  if constexpr (sizeof(U) == 4) {
    const u64 a = nibbles_to_lanes(q[0]), b = nibbles_to_lanes(q[1]);
    u[0] = rev32(pair_lo16((u32)a, (u32)b));
    u[1] = rev32(pair_hi16((u32)a, (u32)b));
    u[2] = rev32(pair_lo16((u32)(a >> 32), (u32)(b >> 32)));
    u[3] = rev32(pair_hi16((u32)(a >> 32), (u32)(b >> 32)));
  } else {
    const u64 a = nibbles_to_lanes(q[0]), b = nibbles_to_lanes(q[1]);
    const u64 c = nibbles_to_lanes(q[2]), d = nibbles_to_lanes(q[3]);
    u[0] = ((u64)rev32(pair_lo16((u32)a, (u32)b)) << 32) | rev32(pair_lo16((u32)c, (u32)d));
    u[1] = ((u64)rev32(pair_hi16((u32)a, (u32)b)) << 32) | rev32(pair_hi16((u32)c, (u32)d));
    u[2] = ((u64)rev32(pair_lo16((u32)(a >> 32), (u32)(b >> 32))) << 32) |
           rev32(pair_lo16((u32)(c >> 32), (u32)(d >> 32)));
    u[3] = ((u64)rev32(pair_hi16((u32)(a >> 32), (u32)(b >> 32))) << 32) |
           rev32(pair_hi16((u32)(c >> 32), (u32)(d >> 32)));
  }
}

// The 64 bits of the nibble string from bit `pos` (zeros past its end).
template <int W> ZFPB_DEV u64 nibbles_at(const u64* q, u32 pos) {
  const u32 wi = pos >> 6, s = pos & 63;
  u64 a = 0, b = 0;
#pragma unroll
  for (int w = 0; w < W; w++) {
    if ((u32)w == wi) a = q[w];
    if ((u32)w == wi + 1) b = q[w];
  }
  return s ? (a >> s) | (b << (64 - s)) : a;
}

// OR x into the nibble string from bit `pos` (bits past its end dropped).
template <int W> ZFPB_DEV void nibbles_or(u64* q, u32 pos, u64 x) {
  const u32 wi = pos >> 6, s = pos & 63;
  const u64 a = x << s, b = s ? x >> (64 - s) : 0ull;
#pragma unroll
  for (int w = 0; w < W; w++) {
    if ((u32)w == wi) q[w] |= a;
    if ((u32)w == wi + 1) q[w] |= b;
  }
}

// ---------------------------------------------------------------------------
// Bit I/O.  Streams are 64-bit words, bits least-significant first
// (zfp-rs src/bitstream/core.rs).
// ---------------------------------------------------------------------------

ZFPB_DEV u64 low_mask(u32 n) { return n < 64 ? (1ull << n) - 1 : ~0ull; }

// Writes a block's bits from bit `pos` of `dst`.  With EDGE_ATOMIC the first
// and the last (partial) word are OR-ed in atomically, for words shared with
// the neighbouring blocks in a zeroed buffer; interior words are stored.
// Words at or past `limit` are dropped (a block longer than its slot).
template <bool EDGE_ATOMIC> struct Writer {
  u64* dst;
  u64 word;  // index of the word being filled
  u64 limit;
  u64 buf;
  u32 bits;
  bool first;

  ZFPB_DEV void init(u64* d, u64 pos, u64 lim) {
    dst = d;
    word = pos >> 6;
    limit = lim;
    bits = (u32)(pos & 63);
    buf = 0;
    first = true;
  }
  ZFPB_DEV void emit(u64 w) {
    if (word < limit) {
      if (EDGE_ATOMIC && first)
        atomicOr(dst + word, w);
      else
        dst[word] = w;
    }
    word++;
    first = false;
  }
  // Append n <= 64 bits of v (no bits set above them).
  ZFPB_DEV void put(u64 v, u32 n) {
    buf |= v << bits;  // bits < 64
    u32 total = bits + n;
    if (total >= 64) {
      emit(buf);
      buf = (v >> 1) >> (63 - bits);
      bits = total - 64;
    } else {
      bits = total;
    }
  }
  ZFPB_DEV void put_zeros(u64 n) {
    u64 total = bits + n;
    while (total >= 64) {
      emit(buf);
      buf = 0;
      total -= 64;
    }
    bits = (u32)total;
  }
  // Write out the partial last word.
  ZFPB_DEV void finish() {
    if (bits > 0 && word < limit) {
      if (EDGE_ATOMIC)
        atomicOr(dst + word, buf);
      else
        dst[word] = buf;
    }
  }
  ZFPB_DEV u64 pos() const { return (word << 6) + bits; }
};

// Reads from bit `pos` of a stream of `len` words; words past the end read as
// zero (core.rs:151-157).  Holds the current partial word and the next word.
struct Reader {
  const u64* src;
  u64 len;
  u64 word;  // index of the word after `nxt`
  u64 buf;   // unread bits of the current word, `bits` of them
  u64 nxt;   // the following word
  u32 bits;

  ZFPB_DEV u64 load(u64 i) const { return i < len ? __ldg(src + i) : 0ull; }
  ZFPB_DEV void init(const u64* s, u64 n, u64 pos) {
    src = s;
    len = n;
    u64 w = pos >> 6;
    u32 off = (u32)(pos & 63);
    if (off) {
      buf = load(w) >> off;
      bits = 64 - off;
      nxt = load(w + 1);
      word = w + 2;
    } else {
      buf = 0;
      bits = 0;
      nxt = load(w);
      word = w + 1;
    }
  }
  ZFPB_DEV u64 peek() const { return buf | (bits < 64 ? nxt << bits : 0ull); }
  ZFPB_DEV void consume(u32 n) {
    if (n <= bits) {
      buf = n < 64 ? buf >> n : 0ull;
      bits -= n;
    } else {
      u64 w = nxt;
      nxt = load(word++);
      bits = bits + 64 - n;
      buf = (w >> 1) >> (63 - bits);
    }
  }
  ZFPB_DEV u64 read(u32 n) {
    u64 v = peek();
    consume(n);
    return v & low_mask(n);
  }
  ZFPB_DEV u32 read_bit() {
    u32 b = (u32)(peek() & 1);
    consume(1);
    return b;
  }
  // Bit position of the cursor.
  ZFPB_DEV u64 pos() const { return ((word - 1) << 6) - bits; }
  // Skip n bits (n may exceed 64).
  ZFPB_DEV void skip(u64 n) {
    u64 p = pos() + n;
    init(src, len, p);
  }
};

// ---------------------------------------------------------------------------
// Embedded bit-plane coder (bitplane.rs:509-790)
// ---------------------------------------------------------------------------

// Plane value of N <= 64 coefficients in one word; N = 256 in four.
template <int N> struct PlaneOps {
  static constexpr int W = N <= 64 ? 1 : N / 64;
};

// Lowest one-bit at or above n of plane words x[0..W): returns false if none.
template <int W> ZFPB_DEV bool next_one(const u64* x, u32 n, u32* p) {
  if constexpr (W == 1) {
    u64 rest = n < 64 ? x[0] >> n : 0ull;
    if (rest) { *p = n + (u32)__ffsll((long long)rest) - 1; return true; }
    return false;
  } else {
#pragma unroll
    for (int j = 0; j < W; j++) {
      if ((u32)(64 * j + 64) <= n) continue;
      u64 v = x[j];
      if ((u32)(64 * j) < n) v >>= (n - 64 * j), v <<= (n - 64 * j);
      if (v) { *p = 64 * j + (u32)__ffsll((long long)v) - 1; return true; }
    }
    return false;
  }
}

template <int W, class Wr> ZFPB_DEV void write_low(Wr& w, const u64* x, u32 m) {
  if constexpr (W == 1) {
    w.put(x[0] & low_mask(m), m);
  } else {
    u32 full = m >> 6, rest = m & 63;
    for (u32 i = 0; i < full; i++) w.put(x[i], 64);
    if (rest) w.put(x[full] & low_mask(rest), rest);
  }
}

// encode_ints + encode_planes one group test at a time (bitplane.rs:509-610);
// used for 4-D blocks, whose planes are 256 bits wide.
template <class U, int N, class Wr>
ZFPB_DEV u32 encode_ints_loop(Wr& w, u32 maxbits, u32 maxprec, const U* u, PlaneStore ps) {
  constexpr u32 intprec = sizeof(U) * 8;
  constexpr u32 size = N;
  constexpr int W = PlaneOps<N>::W;
  const u32 budget = with_maxbits(maxbits, maxprec, size) ? maxbits : 0xffffffffu;
  const u32 kmin = intprec > maxprec ? intprec - maxprec : 0;
  U all = 0;
#pragma unroll
  for (int i = 0; i < N; i++) all |= u[i];
  u32 top;
  if constexpr (sizeof(U) == 4) top = 32 - __clz((int)all);
  else top = 64 - __clzll((long long)all);
  store_planes<U, N>(u, ps);

  u32 bits = budget;
  u32 n = 0;
  u32 tk = top > kmin ? top : kmin;
  u32 empty = intprec - tk;
  empty = empty < bits ? empty : bits;
  w.put_zeros(empty);
  bits -= empty;
  u32 k = intprec - empty;
  while (bits != 0 && k > kmin) {
    if (n == size) {
      while (bits > size && k > kmin) {
        k--;
        u64 x[W];
#pragma unroll
        for (int c = 0; c < W; c++) x[c] = ps.at(k, c, W);
        write_low<W>(w, x, size);
        bits -= size;
      }
      if (k == kmin) break;
    }
    k--;
    u64 x[W];
#pragma unroll
    for (int c = 0; c < W; c++) x[c] = ps.at(k, c, W);
    u32 m = n < bits ? n : bits;
    bits -= m;
    write_low<W>(w, x, m);
    while (bits != 0 && n < size) {
      u32 p;
      if (!next_one<W>(x, n, &p)) {
        w.put(0, 1);
        bits -= 1;
        break;
      }
      u32 zeros = p - n;
      bool last = p == size - 1;
      u32 len = zeros + 2 - (last ? 1 : 0);
      u32 take = len < bits ? len : bits;
      if (take <= 64) {
        u64 code = (last || zeros >= 63) ? 1ull : (1ull | (2ull << zeros));
        w.put(code & low_mask(take), take);
      } else {
        w.put(1, 1);
        w.put_zeros(zeros < take - 1 ? zeros : take - 1);
        if (take == len && !last) w.put(1, 1);
      }
      bits -= take;
      n = p + 1;
    }
  }
  return budget - bits;
}

// kOnesDoubled[b]: the bits of byte b, least significant first, with every
// one-bit written twice ("1" -> "11"); at most 16 bits.
__device__ const unsigned short kOnesDoubled[256] = {
    0x0000, 0x0003, 0x0006, 0x000f, 0x000c, 0x001b, 0x001e, 0x003f, 0x0018, 0x0033, 0x0036, 0x006f,
    0x003c, 0x007b, 0x007e, 0x00ff, 0x0030, 0x0063, 0x0066, 0x00cf, 0x006c, 0x00db, 0x00de, 0x01bf,
    0x0078, 0x00f3, 0x00f6, 0x01ef, 0x00fc, 0x01fb, 0x01fe, 0x03ff, 0x0060, 0x00c3, 0x00c6, 0x018f,
    0x00cc, 0x019b, 0x019e, 0x033f, 0x00d8, 0x01b3, 0x01b6, 0x036f, 0x01bc, 0x037b, 0x037e, 0x06ff,
    0x00f0, 0x01e3, 0x01e6, 0x03cf, 0x01ec, 0x03db, 0x03de, 0x07bf, 0x01f8, 0x03f3, 0x03f6, 0x07ef,
    0x03fc, 0x07fb, 0x07fe, 0x0fff, 0x00c0, 0x0183, 0x0186, 0x030f, 0x018c, 0x031b, 0x031e, 0x063f,
    0x0198, 0x0333, 0x0336, 0x066f, 0x033c, 0x067b, 0x067e, 0x0cff, 0x01b0, 0x0363, 0x0366, 0x06cf,
    0x036c, 0x06db, 0x06de, 0x0dbf, 0x0378, 0x06f3, 0x06f6, 0x0def, 0x06fc, 0x0dfb, 0x0dfe, 0x1bff,
    0x01e0, 0x03c3, 0x03c6, 0x078f, 0x03cc, 0x079b, 0x079e, 0x0f3f, 0x03d8, 0x07b3, 0x07b6, 0x0f6f,
    0x07bc, 0x0f7b, 0x0f7e, 0x1eff, 0x03f0, 0x07e3, 0x07e6, 0x0fcf, 0x07ec, 0x0fdb, 0x0fde, 0x1fbf,
    0x07f8, 0x0ff3, 0x0ff6, 0x1fef, 0x0ffc, 0x1ffb, 0x1ffe, 0x3fff, 0x0180, 0x0303, 0x0306, 0x060f,
    0x030c, 0x061b, 0x061e, 0x0c3f, 0x0318, 0x0633, 0x0636, 0x0c6f, 0x063c, 0x0c7b, 0x0c7e, 0x18ff,
    0x0330, 0x0663, 0x0666, 0x0ccf, 0x066c, 0x0cdb, 0x0cde, 0x19bf, 0x0678, 0x0cf3, 0x0cf6, 0x19ef,
    0x0cfc, 0x19fb, 0x19fe, 0x33ff, 0x0360, 0x06c3, 0x06c6, 0x0d8f, 0x06cc, 0x0d9b, 0x0d9e, 0x1b3f,
    0x06d8, 0x0db3, 0x0db6, 0x1b6f, 0x0dbc, 0x1b7b, 0x1b7e, 0x36ff, 0x06f0, 0x0de3, 0x0de6, 0x1bcf,
    0x0dec, 0x1bdb, 0x1bde, 0x37bf, 0x0df8, 0x1bf3, 0x1bf6, 0x37ef, 0x1bfc, 0x37fb, 0x37fe, 0x6fff,
    0x03c0, 0x0783, 0x0786, 0x0f0f, 0x078c, 0x0f1b, 0x0f1e, 0x1e3f, 0x0798, 0x0f33, 0x0f36, 0x1e6f,
    0x0f3c, 0x1e7b, 0x1e7e, 0x3cff, 0x07b0, 0x0f63, 0x0f66, 0x1ecf, 0x0f6c, 0x1edb, 0x1ede, 0x3dbf,
    0x0f78, 0x1ef3, 0x1ef6, 0x3def, 0x1efc, 0x3dfb, 0x3dfe, 0x7bff, 0x07e0, 0x0fc3, 0x0fc6, 0x1f8f,
    0x0fcc, 0x1f9b, 0x1f9e, 0x3f3f, 0x0fd8, 0x1fb3, 0x1fb6, 0x3f6f, 0x1fbc, 0x3f7b, 0x3f7e, 0x7eff,
    0x0ff0, 0x1fe3, 0x1fe6, 0x3fcf, 0x1fec, 0x3fdb, 0x3fde, 0x7fbf, 0x1ff8, 0x3ff3, 0x3ff6, 0x7fef,
    0x3ffc, 0x7ffb, 0x7ffe, 0xffff};

// The bits of y (at most N of them) with every one-bit doubled, as a
// 128-bit value (lo, hi); hb is y's highest one-bit, so bytes past hb / 8
// are zero and are skipped (a warp goes on while any of its threads has
// bytes left).
template <int N> ZFPB_DEV void double_ones(u64 y, u32 hb, u64& lo, u64& hi) {
  lo = 0;
  hi = 0;
  u32 r = 0;  // one-bits below the current byte
#pragma unroll
  for (int i = 0; i < (N + 7) / 8; i++) {
    if ((u32)i > (hb >> 3)) break;
    const u32 b = (u32)(y >> (8 * i)) & 0xffu;
    const u64 t = __ldg(kOnesDoubled + b);
    const u32 sh = 8 * i + r;  // at most 112
    if (sh < 64) {
      lo |= t << sh;
      if (sh > 48) hi |= t >> (64 - sh);
    } else {
      hi |= t << (sh - 64);
    }
    r += __popc(b);
  }
}

// Plane codes of 1D blocks (4 coefficients) as tables, built at compile time
// from the same rules as the loops below (bitplane.rs:509-620, 675-790).
//   kPlane4Enc[n * 16 + x]: the code of plane x with n < 4 significant
//     coefficients: bits 0-7 the code (verbatim n bits, then the group tests),
//     bits 8-11 its length, bits 12-14 the new n.
//   kPlane4Dec[n * 256 + b]: reading a plane from the 8 stream bits b with
//     n < 4: bits 0-3 the plane, bits 4-7 the code length (0 when the code
//     does not end within 8 bits), bits 8-10 the new n.
struct Plane4Tables {
  unsigned short enc[64];
  unsigned short dec[1024];
  constexpr Plane4Tables() : enc(), dec() {
    for (unsigned n = 0; n < 4; n++) {
      for (unsigned x = 0; x < 16; x++) {
        unsigned code = x & ((1u << n) - 1), len = n, nn = n;
        const unsigned y = x >> n;
        if (y == 0) {
          len += 1;  // "0"
        } else {
          code |= 1u << len;  // "1": a one follows
          len += 1;
          unsigned c = n;
          while (c < 4) {
            if (c == 3) {  // the last coefficient's one is implied
              c = 4;
              break;
            }
            const unsigned b = (x >> c) & 1u;
            code |= b << len;
            len += 1;
            c += 1;
            if (b) {
              if ((x >> c) == 0) {  // no more ones: group test "0"
                len += 1;
                break;
              }
              code |= 1u << len;  // group test "1"
              len += 1;
            }
          }
          nn = c;
        }
        enc[n * 16 + x] = (unsigned short)(code | len << 8 | nn << 12);
      }
      for (unsigned b = 0; b < 256; b++) {
        unsigned pos = n, x = b & ((1u << n) - 1), c = n;
        bool ok = true;
        while (c < 4) {
          if (pos >= 8) {
            ok = false;
            break;
          }
          const unsigned g = (b >> pos) & 1u;
          pos += 1;
          if (!g) break;
          while (c < 4) {
            if (c == 3) {
              x |= 1u << 3;
              c = 4;
              break;
            }
            if (pos >= 8) {
              ok = false;
              break;
            }
            const unsigned v = (b >> pos) & 1u;
            pos += 1;
            if (v) {
              x |= 1u << c;
              c += 1;
              break;
            }
            c += 1;
          }
          if (!ok) break;
        }
        dec[n * 256 + b] = ok ? (unsigned short)(x | pos << 4 | c << 8) : (unsigned short)0;
      }
    }
  }
};
__device__ constexpr Plane4Tables kPlane4{};

// encode_ints (bitplane.rs:509-610) one bit plane at a time.  A plane with
// n significant coefficients is coded as its low n bits verbatim followed by
// the group tests of the rest, y = x >> n.  That code is "0" when y == 0, and
// otherwise "1" followed by y's bits up to its highest one with every one-bit
// doubled, the highest one written "10"; when that one is the last
// coefficient it is implied and omitted with its marker.  This is bit for bit
// what the reference's group-test loop writes, so the block's stream is the
// concatenation of plane codes, cut at the budget.
// Planes above the highest one-bit of any coefficient: top = that bit + 1.
template <class U, int N> ZFPB_DEV u32 top_plane(const U* u) {
  U all = 0;
#pragma unroll
  for (int i = 0; i < N; i++) all |= u[i];
  if constexpr (sizeof(U) == 4) return 32 - __clz((int)all);
  else return 64 - __clzll((long long)all);
}

// The plane loop of encode_ints for blocks of at most 64 values, from planes
// already stored (ps; 4-value blocks: the nibble string q), top as above.
template <class U, int N, class Wr>
ZFPB_DEV u32 encode_stored_planes(Wr& w, u32 maxbits, u32 maxprec, u32 top, PlaneStore ps, const u64* q) {
  {
    constexpr u32 intprec = sizeof(U) * 8;
    constexpr u32 size = N;
    const u32 budget = with_maxbits(maxbits, maxprec, size) ? maxbits : 0xffffffffu;
    const u32 kmin = intprec > maxprec ? intprec - maxprec : 0;
    constexpr int QW = N == 4 ? (int)intprec / 16 : 1;

    u32 bits = budget;
    u32 n = 0;
    u32 tk = top > kmin ? top : kmin;
    u32 empty = intprec - tk;
    empty = empty < bits ? empty : bits;
    w.put_zeros(empty);
    bits -= empty;
    u32 k = intprec - empty;
    while (bits != 0 && k > kmin) {
      if (n == size) break;  // verbatim tail below
      k--;
      if constexpr (N == 4) {
        const u32 x = (u32)nibbles_at<QW>(q, 4 * (intprec - 1 - k)) & 15u;
        const u32 e = kPlane4.enc[n * 16 + x];
        const u32 len = (e >> 8) & 15u;
        const u32 take = len < bits ? len : bits;
        w.put(e & low_mask(take), take);
        bits -= take;
        n = e >> 12;
        continue;
      }
      const u64 x = ps.at(k, 0, 1);
      const u64 y = x >> n;  // n < size <= 64 (n == size leaves the loop)
      u64 glo = 0, ghi = 0;
      u32 glen = 1, nn = n;
      if (y != 0) {
        const u32 hb = 63 - (u32)__clzll((long long)y);
        const u32 c = (u32)__popcll((long long)y);
        u64 elo, ehi;
        double_ones<N>(y, hb, elo, ehi);
        const u32 p = hb + c;  // second copy of the highest one: written as 0
        if (p < 64) elo &= ~(1ull << p);
        else ehi &= ~(1ull << (p - 64));
        glo = 1ull | (elo << 1);
        ghi = (ehi << 1) | (elo >> 63);
        glen = hb + c + 2;
        if (hb == size - 1 - n) glen -= 2;  // the last coefficient's one is implied
        nn = n + hb + 1;
      }
      const u32 total = n + glen;
      const u32 take = total < bits ? total : bits;
      const u32 tv = n < take ? n : take;
      w.put(x & low_mask(tv), tv);
      const u32 tg = take - tv;
      if (tg <= 64) {
        w.put(glo & low_mask(tg), tg);
      } else {
        w.put(glo, 64);
        w.put(ghi & low_mask(tg - 64), tg - 64);
      }
      bits -= take;
      n = nn;
    }
    {
      // Every coefficient significant: the remaining planes go out verbatim,
      // 64 / size of them per write (one for 64-value blocks), cut at the
      // budget.  After the loop above so that a warp's threads run it
      // together instead of alternating with the group-test planes.
      constexpr u32 per = 64 / size;
      while (bits != 0 && k > kmin) {
        u64 chunk = 0;
        const u32 np = k - kmin < per ? k - kmin : per;
        if constexpr (N == 4) {
          chunk = nibbles_at<QW>(q, 4 * (intprec - k));  // planes k - 1, k - 2, ...
        } else {
#pragma unroll
          for (u32 j = 0; j < per; j++)
            if (j < np) chunk |= (ps.at(k - 1 - j, 0, 1) & low_mask(size)) << (j * size);
        }
        const u32 want = np * size;
        const u32 take = want < bits ? want : bits;
        w.put(chunk & low_mask(take), take);
        bits -= take;
        k -= np;
      }
    }
    return budget - bits;
  }
}

template <class U, int N, class Wr>
ZFPB_DEV u32 encode_ints(Wr& w, u32 maxbits, u32 maxprec, const U* u, PlaneStore ps) {
  if constexpr (N > 64) {
    return encode_ints_loop<U, N>(w, maxbits, maxprec, u, ps);
  } else {
    const u32 top = top_plane<U, N>(u);
    constexpr int QW = N == 4 ? (int)sizeof(U) * 8 / 16 : 1;
    constexpr u32 intprec = sizeof(U) * 8;
    u64 q[QW];
    if constexpr (N == 4) store_nibbles<U>(u, q);
    else store_coded_planes<U, N>(u, ps, intprec > maxprec ? intprec - maxprec : 0, top);
    return encode_stored_planes<U, N>(w, maxbits, maxprec, top, ps, q);
  }
}

ZFPB_DEV u32 ctz64(u64 x) { return x ? (u32)__ffsll((long long)x) - 1 : 64u; }

struct PlaneResult {
  u32 bits, m, prec;
  int low, high;  // stored planes are [low, high]; low = intprec if none
};

// decode_planes (bitplane.rs:675-790): planes go to the plane store.
template <int N>
ZFPB_DEV PlaneResult decode_planes(Reader& r, u32 budget, u32 kmin, u32 intprec, PlaneStore ps) {
  constexpr u32 size = N;
  constexpr int W = PlaneOps<N>::W;
  u32 bits = budget, n = 0, m = 0, k = intprec;
  int low = (int)intprec, high = -1;
  while (bits != 0) {
    m = 0;
    if (k <= kmin) { k = k - 1; break; }
    if (n == 0) {
      u32 empty = ctz64(r.peek());
      empty = empty < k - kmin ? empty : k - kmin;
      empty = empty < bits ? empty : bits;
      if (empty != 0) {
        r.consume(empty);
        bits -= empty;
        k -= empty;
        m = size;
        continue;
      }
    } else if (n == size) {
      while (bits > size && k > kmin) {
        k--;
#pragma unroll
        for (int c = 0; c < W; c++) ps.at(k, c, W) = r.read(64 > size ? size : 64);
        if (high < 0) high = (int)k;
        bits -= size;
        low = (int)k;
      }
      if (k == kmin) { k = k - 1; break; }
    }
    k--;
    m = n < bits ? n : bits;
    bits -= m;
    u64 x[W];
    if constexpr (W == 1) {
      x[0] = r.read(m);
    } else {
#pragma unroll
      for (int c = 0; c < W; c++) x[c] = 0;
      u32 full = m >> 6, rest = m & 63;
      for (u32 i = 0; i < full; i++) x[i] = r.read(64);
      if (rest) x[full] = r.read(rest);
    }
    while (bits != 0 && n < size) {
      u64 ahead = r.peek();
      bits -= 1;
      if ((ahead & 1) == 0) {
        r.consume(1);
        m = size;
        break;
      }
      u32 limit = size - 1 - n;
      limit = limit < bits ? limit : bits;
      u32 zeros = ctz64(ahead >> 1);
      u32 lim63 = limit < 63 ? limit : 63;
      if (zeros < lim63) {
        r.consume(zeros + 2);
        bits -= zeros + 1;
        n += zeros;
      } else if (limit <= 63) {
        r.consume(limit + 1);
        bits -= limit;
        n += limit;
      } else {
        r.consume(64);
        bits -= 63;
        n += 63;
        u32 lim = limit - 63;
        while (lim != 0) {  // scan_zeros, bitplane.rs:775-790
          u32 z = ctz64(r.peek());
          u32 span = lim < 64 ? lim : 64;
          if (z < span) {
            r.consume(z + 1);
            bits -= z + 1;
            n += z;
            break;
          }
          r.consume(span);
          bits -= span;
          n += span;
          lim -= span;
        }
      }
      if constexpr (W == 1) x[0] |= 1ull << n;
      else x[n >> 6] |= 1ull << (n & 63);
      n += 1;
      m = n;
    }
#pragma unroll
    for (int c = 0; c < W; c++) ps.at(k, c, W) = x[c];
    if (high < 0) high = (int)k;
    low = (int)k;
  }
  if (n == 0) low = (int)intprec;
  PlaneResult res;
  res.bits = budget - bits;
  res.m = m;
  res.prec = intprec - k;
  res.low = low;
  res.high = high;
  return res;
}

// ---------------------------------------------------------------------------
// Plane-at-a-time decoder for blocks of up to 64 values.
//
// decode_planes follows the reference loop, one group test per iteration, so
// the 32 blocks of a warp run through different branches and the warp issues
// the union of their paths.  This decoder does the same work in one iteration
// per bit plane with a bounded amount of work per plane, so that the threads of
// a warp stay together.  Facts it rests on (the code written by
// bitplane.rs:509-620 and read by bitplane.rs:675-790):
//
// * A plane is n verbatim bits (n = coefficients already significant) and then
//   the group-test code of the rest.  That code is a GT bit; while it is 1, a
//   run of zeros ended by a 1 (the next significant coefficient); then the next
//   GT bit.  So, past the verbatim bits, the code is "1 0^z1 1 1 0^z2 1 ... 0":
//   its ones pair up as (GT, coefficient), and a bit is a GT bit exactly when
//   the number of ones up to and including it is odd (a prefix XOR).
// * The code ends at the first group start holding a 0 (a group start is bit 0
//   or the bit after a coefficient one), or, once the scan reaches the last
//   coefficient, without its "1" (the one is implied), or where the budget
//   runs out.
// * A plane takes at most 2 * size - n - 1 bits, so a 128-bit window at its
//   start holds all of it.
// ---------------------------------------------------------------------------

ZFPB_DEV u64 prefix_xor64(u64 x) {
  x ^= x << 1;
  x ^= x << 2;
  x ^= x << 4;
  x ^= x << 8;
  x ^= x << 16;
  x ^= x << 32;
  return x;
}

ZFPB_DEV u32 popc64(u64 x) { return (u32)__popcll((long long)x); }

// Bits of (hi:lo) below position e, e in [0, 128].
ZFPB_DEV u32 popc_below128(u64 lo, u64 hi, u32 e) {
  u32 c = popc64(lo & low_mask(e < 64 ? e : 64));
  if (e > 64) c += popc64(hi & low_mask(e - 64));
  return c;
}

ZFPB_DEV u32 bit128(u64 lo, u64 hi, u32 i) { return (u32)((i < 64 ? lo >> i : hi >> (i & 63)) & 1); }

// Position of the r-th (from 0) set bit of x, which has more than r set bits.
ZFPB_DEV u32 select64(u64 x, u32 r) {
  u32 pos = 0, c;
#pragma unroll
  for (int w = 32; w >= 2; w >>= 1) {
    c = popc64(x & low_mask((u32)w));
    if (r >= c) {
      r -= c;
      x >>= w;
      pos += (u32)w;
    }
  }
  c = (u32)(x & 1);
  return r >= c ? pos + 1 : pos;
}

ZFPB_DEV u32 select128(u64 lo, u64 hi, u32 r) {
  const u32 c = popc64(lo);
  return r < c ? select64(lo, r) : 64 + select64(hi, r - c);
}

// Three consecutive stream words and a bit offset into the first: a window
// of 128 bits at the cursor.
struct Window {
  const Reader* rd;
  u64 w0, w1, w2, next;
  u32 off;

  ZFPB_DEV void init(const Reader* r, u64 pos) {
    rd = r;
    const u64 wi = pos >> 6;
    off = (u32)(pos & 63);
    w0 = r->load(wi);
    w1 = r->load(wi + 1);
    w2 = r->load(wi + 2);
    next = wi + 3;
  }
  ZFPB_DEV u64 lo() const { return (w0 >> off) | ((w1 << 1) << (63 - off)); }
  ZFPB_DEV u64 hi() const { return (w1 >> off) | ((w2 << 1) << (63 - off)); }
  ZFPB_DEV void advance(u32 n) {  // n <= 128
    off += n;
    if (off >= 64) {
      w0 = w1;
      w1 = w2;
      w2 = rd->load(next++);
      off -= 64;
    }
    if (off >= 64) {
      w0 = w1;
      w1 = w2;
      w2 = rd->load(next++);
      off -= 64;
    }
  }
  ZFPB_DEV u64 pos() const { return ((next - 3) << 6) + off; }
  // Any distance: re-reads the three words at the new position.
  ZFPB_DEV void advance_far(u64 n) {
    const u64 p = pos() + n;
    init(rd, p);
  }
};

// One plane's group-test code, from bit 0 of the 128-bit window (t0, t1)
// whose bit 0 is a 1 (at least one new significant coefficient), with n
// coefficients significant before the plane and a bits of budget left for
// the code.  Sets end (the code's length), n_new and m_new (n and m of the
// reference's reader after the plane) and, with NEED_Y, y: the plane's bits
// from coefficient n up, as the reader would set them.
template <int N, bool NEED_Y>
ZFPB_DEV void group_tests(u64 t0, u64 t1, u32 n, u32 a, u32& end, u32& n_new, u32& m_new, u64& y) {
  constexpr u32 size = N;
  constexpr bool WIDE = N == 64;
  const u64 p0 = prefix_xor64(t0);
  const u64 p1 = WIDE ? prefix_xor64(t1) ^ (0ull - (p0 >> 63)) : 0ull;
  const u64 s0 = t0 & ~p0, s1 = t1 & ~p1;  // coefficient ones
  const u64 g0 = t0 & p0, g1 = t1 & p1;    // GT ones
  const u64 b0 = (s0 << 1) | 1, b1 = (s1 << 1) | (s0 >> 63);  // group starts
  const u32 e = WIDE ? (((b0 & ~t0) != 0) ? ctz64(b0 & ~t0) : 64 + ctz64(b1 & ~t1)) : ctz64(b0 & ~t0);
  const u32 lim = WIDE ? 128 : 64;
  const u32 ce = n + e - popc_below128(g0, g1, e);  // coefficients read before bit e
  const bool regular = e < lim && ce <= size - 1;
  u32 extra = 64;
  if (regular && e < a) {
    end = e + 1;
    n_new = ce;
    m_new = size;
  } else {
    // Ended by the implied last one (not a terminator), or cut by the budget.
    u32 istar = lim;
    u32 bs = 0;
    if (!regular) {
      const u32 L = size - 1 - n;  // coefficient zeros before the implied one
      istar = L == 0 ? 0 : select128(~g0, WIDE ? ~g1 : 0ull, L - 1) + 1;
      bs = bit128(b0, b1, istar < lim ? istar : 0);
    }
    if (!regular && (bs ? istar < a : istar <= a)) {
      end = istar + bs;
      extra = size - 1 - n;
      n_new = size;
      m_new = size;
    } else {
      end = a;  // a < lim here
      const u32 ca = n + a - popc_below128(g0, g1, a);
      if (bit128(b0, b1, a)) {
        n_new = ca;
      } else {
        extra = ca - n;  // the reader's implied one at the cut
        n_new = ca + 1;
      }
      m_new = n_new;
    }
  }
  if constexpr (!NEED_Y) {
    y = 0;
    return;
  }
  // Coefficient ones before `end`, each moved down past the GT bits
  // before it: the j-th (from 1) at bit s goes to coefficient s - j.
  u64 q0 = s0 & low_mask(end < 64 ? end : 64);
  u64 q1 = (WIDE && end > 64) ? s1 & low_mask(end - 64) : 0ull;
  y = extra < 64 ? 1ull << extra : 0ull;
  u32 j = 1;
  while (q0) {
    y |= 1ull << (ctz64(q0) - j);
    j++;
    q0 &= q0 - 1;
  }
  if (WIDE) {
    while (q1) {
      y |= 1ull << (64 + ctz64(q1) - j);
      j++;
      q1 &= q1 - 1;
    }
  }
}

// Same contract and results as decode_planes, for N <= 64.  With QW != 0
// (4-value blocks of QW * 16 planes) the planes go to the nibble string q
// instead of the plane store.
template <int N, int QW = 0>
ZFPB_DEV PlaneResult decode_planes_sync(Reader& rd, u32 budget, u32 kmin, u32 intprec, PlaneStore ps,
                                        u64* q = nullptr) {
  static_assert(N <= 64, "one plane word per plane");
  static_assert(QW == 0 || N == 4, "nibble planes are for 4-value blocks");
  constexpr u32 size = N;
  // Plane kk (its bits and, with `np` planes, the ones below it) to the store.
  auto put = [&](u32 kk, u64 x, u32 np) {
    if constexpr (QW != 0) {
      nibbles_or<QW>(q, 4 * (QW * 16 - 1 - kk), x);
    } else {
#pragma unroll
      for (u32 j = 0; j < 64 / size; j++)
        if (j < np) ps.at(kk - j, 0, 1) = (x >> (j * size)) & low_mask(size);
    }
  };
  constexpr bool WIDE = N == 64;  // the window needs its second word
  Window r;
  r.init(&rd, rd.pos());
  u32 bits = budget, n = 0, m = 0, k = intprec;
  int low = (int)intprec, high = -1;
  bool done = false;
  while (bits != 0) {
    if (N <= 16 && n == size) break;  // verbatim tail below
    if constexpr (N == 64) {
      if (n == size) {
        // Every coefficient significant: the remaining planes are the
        // stream's next bits verbatim, a plane per 64 bits while more than a
        // plane of budget is left (m = 0), then the rest of the budget as a
        // last plane (m = those bits); out of planes, the read ends with
        // m = 0 and k one below kmin.  One tight loop instead of the
        // iterations above, so that a warp's threads run it together.
        const u32 full_left = (bits - 1) / size, planes_left = k - kmin;
        const u32 f = full_left < planes_left ? full_left : planes_left;
        for (u32 j = 0; j < f; j++) {
          k--;
          ps.at(k, 0, 1) = r.lo();
          r.advance(size);
        }
        bits -= f * size;
        if (f) low = (int)k;
        m = 0;
        if (k <= kmin) {
          k = k - 1;
        } else {
          k--;
          ps.at(k, 0, 1) = r.lo() & low_mask(bits);
          low = (int)k;
          m = bits;
          r.advance(bits);
          bits = 0;
        }
        done = true;
        break;
      }
    }
    m = 0;
    if (k <= kmin) {
      k = k - 1;
      done = true;
      break;
    }
    const u64 lo = r.lo();
    if (n == 0) {
      // Leading empty planes: one 0 bit each (bitplane.rs:700-712).
      u32 e = ctz64(lo);
      e = e < k - kmin ? e : k - kmin;
      e = e < bits ? e : bits;
      if (e != 0) {
        r.advance(e);
        bits -= e;
        k -= e;
        m = size;
        continue;
      }
    }
    k--;
    if constexpr (N == 16 || N == 64) {
      // At most 4 coefficients still insignificant: the plane's code is its
      // first size - 4 bits verbatim, then the code of a 4-value plane with
      // n - (size - 4) significant (the group tests depend only on how many
      // coefficients remain), which the 4-value table reads.  (The encoder
      // keeps its general path here: the table made it slower.)
      constexpr u32 P = size - 4;
      if (n >= P && n < size) {
        const u64 t = WIDE ? (lo >> P) | (r.hi() << (64 - P)) : lo >> P;
        const u32 e = kPlane4.dec[(n - P) * 256 + (u32)(t & 0xff)];
        const u32 len = (e >> 4) & 15u;
        if (len != 0 && P + len <= bits) {
          ps.at(k, 0, 1) = (lo & low_mask(P)) | ((u64)(e & 15u) << P);
          if (high < 0) high = (int)k;
          low = (int)k;
          n = P + (e >> 8);
          m = size;
          bits -= P + len;
          r.advance(P + len);
          continue;
        }
      }
    }
    if constexpr (N == 4) {
      const u32 e = kPlane4.dec[n * 256 + (u32)(lo & 0xff)];
      const u32 len = (e >> 4) & 15u;
      if (len != 0 && len <= bits) {
        put(k, e & 15u, 1);
        if (high < 0) high = (int)k;
        low = (int)k;
        n = e >> 8;
        m = size;
        bits -= len;
        r.advance(len);
        continue;
      }
    }
    u64 x;
    u32 used;
    if (n == size) {
      // Every coefficient significant: the plane is verbatim.
      used = bits > size ? size : bits;
      x = lo & low_mask(used);
      m = bits > size ? 0 : bits;
      bits -= used;
    } else {
      used = n < bits ? n : bits;
      x = lo & low_mask(used);
      m = used;
      bits -= used;
      if (bits != 0) {
        const u64 hi = WIDE ? r.hi() : 0ull;
        // The group-test code, from bit n of the window.
        const u64 t0 = n ? (lo >> n) | (hi << (64 - n)) : lo;
        const u64 t1 = n ? hi >> n : hi;
        if ((t0 & 1) == 0) {
          used += 1;
          bits -= 1;
          m = size;
        } else {
          u32 end, n_new, m_new;
          u64 y;
          group_tests<N, true>(t0, t1, n, bits, end, n_new, m_new, y);
          x |= y << n;
          used += end;
          bits -= end;
          n = n_new;
          m = m_new;
        }
      }
    }
    r.advance(used);
    if constexpr (N == 4) put(k, x, 1);
    else ps.at(k, 0, 1) = x;
    if (high < 0) high = (int)k;
    low = (int)k;
  }
  if constexpr (N <= 16) {
    // Every coefficient significant: verbatim planes, as many at once as the
    // window's 64 bits hold while more than a plane of budget is left (the
    // reference reads them one at a time while bits > size, m staying 0),
    // then a last partial plane.  After the loop above so that a warp's
    // threads run it together.
    constexpr u32 per = 64 / size;
    while (!done && bits != 0) {
      m = 0;
      if (k <= kmin) {
        k = k - 1;
        break;
      }
      const u64 lo = r.lo();
      k--;
      if (bits > size) {
        u32 np = (bits - 1) / size;
        np = np < per ? np : per;
        np = np < k + 1 - kmin ? np : k + 1 - kmin;
        put(k, lo & low_mask(np * size), np);
        if (high < 0) high = (int)k;
        k -= np - 1;
        low = (int)k;
        bits -= np * size;
        r.advance(np * size);
      } else {
        put(k, lo & low_mask(bits), 1);
        if (high < 0) high = (int)k;
        low = (int)k;
        m = bits;
        r.advance(bits);
        bits = 0;
      }
    }
  }
  if (n == 0) low = (int)intprec;
  rd.init(rd.src, rd.len, r.pos());
  PlaneResult res;
  res.bits = budget - bits;
  res.m = m;
  res.prec = intprec - k;
  res.low = low;
  res.high = high;
  return res;
}

// decode_ints (bitplane.rs:626-667) into u; returns bits read, sets *zero.
template <class U, int N>
ZFPB_DEV u32 decode_ints(Reader& r, u32 maxbits, u32 maxprec, int rounding, U* u, bool* zero,
                         PlaneStore ps) {
  constexpr u32 intprec = sizeof(U) * 8;
  const bool constrained = with_maxbits(maxbits, maxprec, N);
  const u32 budget = constrained ? maxbits : 0xffffffffu;
  const u32 kmin = intprec > maxprec ? intprec - maxprec : 0;
  PlaneResult pr;
  constexpr int QW = N == 4 ? (int)intprec / 16 : 0;
  u64 q[QW ? QW : 1];
#pragma unroll
  for (int w = 0; w < (QW ? QW : 1); w++) q[w] = 0;
  if constexpr (N <= 64) pr = decode_planes_sync<N, QW>(r, budget, kmin, intprec, ps, q);
  else pr = decode_planes<N>(r, budget, kmin, intprec, ps);
  bool z = pr.low == (int)intprec;
  if (z) {
#pragma unroll
    for (int i = 0; i < N; i++) u[i] = 0;
  } else if constexpr (QW != 0) {
    load_nibbles<U>(u, q);
  } else {
    load_coded_planes<U, N>(u, ps, pr.low, pr.high);
  }
  bool round = rounding == 2;
  if (round) {
    u32 m = pr.m, prec = pr.prec;
    if (!constrained) {
      m = 0;
      prec = intprec - (kmin - 1);
    }
    inv_round<U, N>(u, m, prec);
  }
  *zero = z && !round;
  return pr.bits;
}

// ---------------------------------------------------------------------------
// Block coders
// ---------------------------------------------------------------------------

template <int N> struct Dims { static constexpr u32 value = N == 4 ? 1 : N == 16 ? 2 : N == 64 ? 3 : 4; };

// encode/integer.rs:50-93: transform, optional bias, reorder, planes, pad.
template <class I, int N, class Wr>
ZFPB_DEV u32 encode_int_block(Wr& w, I* b, u32 minbits, u32 maxbits, u32 maxprec, int rounding,
                              PlaneStore ps) {
  typedef typename Traits<I>::U U;
  fwd_axes<I, N, 0>(b);
  if (rounding == 1) fwd_round<I, N>(b, maxprec);
  U u[N];
  fwd_order<N>(u, b);
  u32 bits = encode_ints<U, N>(w, maxbits, maxprec, u, ps);
  if (bits < minbits) {
    w.put_zeros(minbits - bits);
    bits = minbits;
  }
  return bits;
}

// encode/float.rs:22-113
template <class T, int N, class Wr>
ZFPB_DEV u32 encode_float_block(Wr& w, const T* fb, const Codec& c, PlaneStore ps) {
  typedef typename Traits<T>::I I;
  int emax = exponent_block<T, N>(fb);
  u32 prec = precision_f(emax, c.maxprec, c.minexp, Dims<N>::value, c.tight != 0);
  u32 e = prec != 0 ? (u32)(emax + Traits<T>::EBIAS) : 0u;
  if (e != 0) {
    constexpr u32 hb = Traits<T>::EBITS + 1;
    w.put(2 * (u64)e + 1, hb);
    I ib[N];
    fwd_cast<T, N>(ib, fb, emax);
    return hb + encode_int_block<I, N>(w, ib, sat_sub(c.minbits, hb), sat_sub(c.maxbits, hb), prec,
                                       c.rounding, ps);
  }
  w.put(0, 1);
  if (c.minbits > 1) {
    w.put_zeros(c.minbits - 1);
    return c.minbits;
  }
  return 1;
}

// The same float block coder in two halves, so that one thread can prepare
// a block (cast, transform, planes into the plane store) and another code it
// from the store: a CTA orders its blocks by the expected length of their
// sequential plane loop before coding them, so that the threads of a warp run
// loops of similar length.
struct BlockPrep {
  u32 head;  // header value 2 * e + 1 (written in EBITS + 1 bits), 0: an empty block
  u32 prec;  // precision of the integer coder
  u32 top;   // one above the highest one-bit of any coefficient
  u32 key;   // planes before the last coefficient turns significant
};

template <class T, int N>
ZFPB_DEV BlockPrep prep_float_block(const T* fb, const Codec& c, PlaneStore ps) {
  static_assert(N == 16 || N == 64, "plane-store blocks of one word per plane");
  typedef typename Traits<T>::I I;
  typedef typename Traits<T>::U U;
  BlockPrep p;
  const int emax = exponent_block<T, N>(fb);
  const u32 prec = precision_f(emax, c.maxprec, c.minexp, Dims<N>::value, c.tight != 0);
  const u32 e = prec != 0 ? (u32)(emax + Traits<T>::EBIAS) : 0u;
  p.head = e != 0 ? 2 * e + 1 : 0u;
  p.prec = prec;
  p.top = 0;
  p.key = 0;
  if (e != 0) {
    I ib[N];
    fwd_cast<T, N>(ib, fb, emax);
    fwd_axes<I, N, 0>(ib);
    if (c.rounding == 1) fwd_round<I, N>(ib, prec);
    U u[N];
    fwd_order<N>(u, ib);
    p.top = top_plane<U, N>(u);
    constexpr u32 intprec = sizeof(U) * 8;
    const u32 kmin = intprec > prec ? intprec - prec : 0;
    store_coded_planes<U, N>(u, ps, kmin, p.top);
    // The group-test phase of the plane loop ends with the plane in which
    // the last coefficient turns significant (its highest one-bit).
    const u32 last = top_plane<U, 1>(u + N - 1);
    const u32 stop = last > kmin + 1 ? last - 1 : kmin;
    p.key = p.top > stop ? p.top - stop : 0u;
  }
  return p;
}

// encode/float.rs:22-113 from a prepared block (same bits as encode_float_block).
template <class T, int N, class Wr>
ZFPB_DEV u32 code_float_block(Wr& w, const BlockPrep& p, const Codec& c, PlaneStore ps) {
  static_assert(N == 16 || N == 64, "plane-store blocks of one word per plane");
  typedef typename Traits<T>::U U;
  if (p.head != 0) {
    constexpr u32 hb = Traits<T>::EBITS + 1;
    w.put(p.head, hb);
    u32 bits = encode_stored_planes<U, N>(w, sat_sub(c.maxbits, hb), p.prec, p.top, ps, nullptr);
    const u32 mb = sat_sub(c.minbits, hb);
    if (bits < mb) {
      w.put_zeros(mb - bits);
      bits = mb;
    }
    return hb + bits;
  }
  w.put(0, 1);
  if (c.minbits > 1) {
    w.put_zeros(c.minbits - 1);
    return c.minbits;
  }
  return 1;
}

// encode/reversible.rs:89-137
template <class I, int N, class Wr>
ZFPB_DEV u32 rev_encode_int_block(Wr& w, const I* ib, u32 maxbits, u32 maxprec, PlaneStore ps) {
  typedef typename Traits<I>::U U;
  constexpr u32 PB = sizeof(U) == 4 ? 5 : 6;
  U u[N];
  fwd_order<N>(u, ib);
  U all = 0;
#pragma unroll
  for (int i = 0; i < N; i++) all |= u[i];
  u32 prec;
  if constexpr (sizeof(U) == 4) prec = all ? 32 - (u32)(__ffs((int)all) - 1) : 0;
  else prec = all ? 64 - (u32)(__ffsll((long long)all) - 1) : 0;
  prec = prec < maxprec ? prec : maxprec;
  prec = prec < 1 ? 1 : prec;
  w.put(prec - 1, PB);
  return PB + encode_ints<U, N>(w, sat_sub(maxbits, PB), prec, u, ps);
}

// encode/reversible.rs:172-313
template <class T, int N, class Wr>
ZFPB_DEV u32 rev_encode_block(Wr& w, T* fb, const Codec& c, PlaneStore ps) {
  typedef typename Traits<T>::I I;
  typedef typename Traits<T>::U U;
  u32 bits;
  if constexpr (!Traits<T>::FLOAT) {
    I* b = reinterpret_cast<I*>(fb);
    fwd_axes<I, N, 2>(b);
    bits = rev_encode_int_block<I, N>(w, b, c.maxbits, c.maxprec, ps);
  } else {
    int emax = exponent_block<T, N>(fb);
    u32 e = (u32)(emax + Traits<T>::EBIAS);
    bool tiny = e != 0 && emax < Traits<T>::MIN_CAST_EMAX;
    I ib[N];
#pragma unroll
    for (int i = 0; i < N; i++) ib[i] = 0;
    if (e != 0 && !tiny) fwd_cast<T, N>(ib, fb, emax);
    bool rev = !tiny;
    if (rev) {
      constexpr int ip = Traits<T>::PREC;
      T sc = pow2<T>(emax - (ip - 2));
#pragma unroll
      for (int i = 0; i < N; i++) rev = rev && (bits_of(mul_rn(sc, to_float(ib[i]))) == bits_of(fb[i]));
    }
    if (rev) {
      if (e != 0) {
        constexpr u32 hb = 2 + Traits<T>::EBITS;
        w.put(1, 2);
        w.put(e, Traits<T>::EBITS);
        fwd_axes<I, N, 2>(ib);
        bits = hb + rev_encode_int_block<I, N>(w, ib, sat_sub(c.maxbits, hb), c.maxprec, ps);
      } else {
        w.put(0, 1);
        bits = 1;
      }
    } else {
      const U tc = (U)(~(U)0) >> 1;
#pragma unroll
      for (int i = 0; i < N; i++) {
        U b = (U)bits_of(fb[i]);
        ib[i] = (b >> (sizeof(U) * 8 - 1)) ? (I)(b ^ tc) : (I)b;
      }
      w.put(3, 2);
      fwd_axes<I, N, 2>(ib);
      bits = 2 + rev_encode_int_block<I, N>(w, ib, sat_sub(c.maxbits, 2), c.maxprec, ps);
    }
  }
  if (bits < c.minbits) {
    w.put_zeros(c.minbits - bits);
    bits = c.minbits;
  }
  return bits;
}

// Code one gathered block (codec/block/strided.rs dispatch).
template <class T, int N, class Wr>
ZFPB_DEV u32 encode_block(Wr& w, T* blk, const Codec& c, PlaneStore ps) {
  if (c.minexp < ZFP_MIN_EXP) return rev_encode_block<T, N>(w, blk, c, ps);
  if constexpr (Traits<T>::FLOAT) {
    return encode_float_block<T, N>(w, blk, c, ps);
  } else {
    return encode_int_block<T, N>(w, blk, c.minbits, c.maxbits, c.maxprec, c.rounding, ps);
  }
}

// ---- decoding -------------------------------------------------------------

// decode/core.rs:97-131 (without the skip to minbits, which the caller does)
template <class I, int N>
ZFPB_DEV u32 decode_int_block(Reader& r, u32 maxbits, u32 maxprec, int rounding, I* ib, PlaneStore ps) {
  typedef typename Traits<I>::U U;
  U u[N];
  bool zero;
  u32 bits = decode_ints<U, N>(r, maxbits, maxprec, rounding, u, &zero, ps);
  if (zero) {
#pragma unroll
    for (int i = 0; i < N; i++) ib[i] = 0;
  } else {
    inv_order<N>(u, ib);
    inv_axes<I, N, 1>(ib);
  }
  return bits;
}

// decode/reversible.rs:46-82
template <class I, int N>
ZFPB_DEV u32 rev_decode_int_block(Reader& r, u32 maxbits, I* ib, PlaneStore ps) {
  typedef typename Traits<I>::U U;
  constexpr u32 PB = sizeof(U) == 4 ? 5 : 6;
  u32 prec = (u32)r.read(PB) + 1;
  U u[N];
  bool zero;
  u32 ub = decode_ints<U, N>(r, sat_sub(maxbits, PB), prec, 0, u, &zero, ps);
  inv_order<N>(u, ib);
  inv_axes<I, N, 3>(ib);
  return PB + ub;
}

// Decode one block into blk; returns the bits the block occupies (after the
// skip to minbits) and, in *read_bits, the bits actually read.
// LOSSY: lossy float streams only (minexp >= ZFP_MIN_EXP), no reversible path.
template <class T, int N, bool LOSSY = false>
ZFPB_DEV u32 decode_block(Reader& r, T* blk, const Codec& c, PlaneStore ps, u32* read_bits) {
  typedef typename Traits<T>::I I;
  typedef typename Traits<T>::U U;
  u32 bits;
  if (!LOSSY && c.minexp < ZFP_MIN_EXP) {
    if constexpr (!Traits<T>::FLOAT) {
      bits = rev_decode_int_block<I, N>(r, c.maxbits, reinterpret_cast<I*>(blk), ps);
    } else {
      // decode/reversible.rs:130-194
      if (r.read_bit() == 0) {
#pragma unroll
        for (int i = 0; i < N; i++) blk[i] = 0;
        bits = 1;
      } else {
        bits = 2;
        u32 reinterp = r.read_bit();
        I ib[N];
        if (reinterp) {
          bits += rev_decode_int_block<I, N>(r, sat_sub(c.maxbits, bits), ib, ps);
          const U tc = (U)(~(U)0) >> 1;
#pragma unroll
          for (int i = 0; i < N; i++) blk[i] = float_of(ib[i] < 0 ? (U)((U)ib[i] ^ tc) : (U)ib[i]);
        } else {
          int emax = (int)r.read(Traits<T>::EBITS) - Traits<T>::EBIAS;
          bits += Traits<T>::EBITS;
          bits += rev_decode_int_block<I, N>(r, sat_sub(c.maxbits, bits), ib, ps);
          inv_cast<T, N>(ib, blk, emax);
        }
      }
    }
    *read_bits = bits;
    return bits < c.minbits ? c.minbits : bits;
  }
  if constexpr (Traits<T>::FLOAT) {
    // decode/core.rs:184-237
    if (r.read_bit()) {
      constexpr u32 hb = 1 + Traits<T>::EBITS;
      int emax = (int)r.read(Traits<T>::EBITS) - Traits<T>::EBIAS;
      u32 prec = precision_f(emax, c.maxprec, c.minexp, Dims<N>::value, c.tight != 0);
      I ib[N];
      u32 ibits = decode_int_block<I, N>(r, sat_sub(c.maxbits, hb), prec, c.rounding, ib, ps);
      inv_cast<T, N>(ib, blk, emax);
      u32 mb = sat_sub(c.minbits, hb);
      *read_bits = hb + ibits;
      return hb + (ibits < mb ? mb : ibits);
    }
#pragma unroll
    for (int i = 0; i < N; i++) blk[i] = 0;
    *read_bits = 1;
    return c.minbits > 1 ? c.minbits : 1;
  } else {
    bits = decode_int_block<I, N>(r, c.maxbits, c.maxprec, c.rounding, blk, ps);
    *read_bits = bits;
    return bits < c.minbits ? c.minbits : bits;
  }
}

// Bits of the planes of one block, as decode_planes_sync reads them, without
// the planes: group-test planes one at a time, and once every coefficient is
// significant the verbatim planes left all at once (min(bits, planes * size)).
// For the offsets of streams that come without an index.
template <int N>
ZFPB_DEV u32 plane_bits(Reader& rd, u32 budget, u32 kmin, u32 intprec) {
  static_assert(N <= 64, "one plane word per plane");
  constexpr u32 size = N;
  constexpr bool WIDE = N == 64;
  Window r;
  r.init(&rd, rd.pos());
  u32 bits = budget, n = 0, k = intprec;
  while (bits != 0 && k > kmin) {
    if (n == size) {
      const u64 rest = (u64)(k - kmin) * size;
      const u32 take = rest < bits ? (u32)rest : bits;
      r.advance_far(take);
      bits -= take;
      break;
    }
    const u64 lo = r.lo();
    if (n == 0) {
      u32 e = ctz64(lo);
      e = e < k - kmin ? e : k - kmin;
      e = e < bits ? e : bits;
      if (e != 0) {
        r.advance(e);
        bits -= e;
        k -= e;
        continue;
      }
    }
    k--;
    if constexpr (N == 16 || N == 64) {
      constexpr u32 P = size - 4;  // as in decode_planes_sync
      if (n >= P) {
        const u64 t = WIDE ? (lo >> P) | (r.hi() << (64 - P)) : lo >> P;
        const u32 e = kPlane4.dec[(n - P) * 256 + (u32)(t & 0xff)];
        const u32 len = (e >> 4) & 15u;
        if (len != 0 && P + len <= bits) {
          n = P + (e >> 8);
          bits -= P + len;
          r.advance(P + len);
          continue;
        }
      }
    }
    if constexpr (N == 4) {
      const u32 e = kPlane4.dec[n * 256 + (u32)(lo & 0xff)];
      const u32 len = (e >> 4) & 15u;
      if (len != 0 && len <= bits) {
        n = e >> 8;
        bits -= len;
        r.advance(len);
        continue;
      }
    }
    u32 used = n < bits ? n : bits;
    bits -= used;
    if (bits != 0) {
      const u64 hi = WIDE ? r.hi() : 0ull;
      const u64 t0 = n ? (lo >> n) | (hi << (64 - n)) : lo;
      const u64 t1 = n ? hi >> n : hi;
      if ((t0 & 1) == 0) {
        used += 1;
        bits -= 1;
      } else {
        u32 end, n_new, m_new;
        u64 y;
        group_tests<N, false>(t0, t1, n, bits, end, n_new, m_new, y);
        used += end;
        bits -= end;
        n = n_new;
      }
    }
    r.advance(used);
  }
  rd.init(rd.src, rd.len, r.pos());
  return budget - bits;
}

// decode_ints' bits without the planes.
template <class U, int N>
ZFPB_DEV u32 ints_bits(Reader& r, u32 maxbits, u32 maxprec) {
  constexpr u32 intprec = sizeof(U) * 8;
  const bool constrained = with_maxbits(maxbits, maxprec, N);
  const u32 kmin = intprec > maxprec ? intprec - maxprec : 0;
  return plane_bits<N>(r, constrained ? maxbits : 0xffffffffu, kmin, intprec);
}

// The bits one block occupies (after the skip to minbits), read as
// decode_block reads them (same headers), without decoding its values.
template <class T, int N>
ZFPB_DEV u32 block_length(Reader& r, const Codec& c) {
  typedef typename Traits<T>::U U;
  constexpr u32 PB = sizeof(U) == 4 ? 5 : 6;
  u32 bits;
  if (c.minexp < ZFP_MIN_EXP) {
    if constexpr (!Traits<T>::FLOAT) {
      const u32 prec = (u32)r.read(PB) + 1;
      bits = PB + ints_bits<U, N>(r, sat_sub(c.maxbits, PB), prec);
    } else {
      if (r.read_bit() == 0) {
        bits = 1;
      } else {
        bits = 2;
        if (!r.read_bit()) {
          r.read(Traits<T>::EBITS);
          bits += Traits<T>::EBITS;
        }
        const u32 mb = sat_sub(c.maxbits, bits);
        const u32 prec = (u32)r.read(PB) + 1;
        bits += PB + ints_bits<U, N>(r, sat_sub(mb, PB), prec);
      }
    }
    return bits < c.minbits ? c.minbits : bits;
  }
  if constexpr (Traits<T>::FLOAT) {
    if (r.read_bit()) {
      constexpr u32 hb = 1 + Traits<T>::EBITS;
      const int emax = (int)r.read(Traits<T>::EBITS) - Traits<T>::EBIAS;
      const u32 prec = precision_f(emax, c.maxprec, c.minexp, Dims<N>::value, c.tight != 0);
      const u32 ibits = ints_bits<U, N>(r, sat_sub(c.maxbits, hb), prec);
      const u32 mb = sat_sub(c.minbits, hb);
      return hb + (ibits < mb ? mb : ibits);
    }
    return c.minbits > 1 ? c.minbits : 1;
  } else {
    bits = ints_bits<U, N>(r, c.maxbits, c.maxprec);
    return bits < c.minbits ? c.minbits : bits;
  }
}

// ---- two-kernel decoding ----------------------------------------------------
//
// The same decode as decode_block, cut in two: parse_block reads a block's
// bits (header and bit planes; the planes go to the plane store, which here is
// a plane-major scratch in global memory) and returns a BlockHead;
// finish_block turns the head and the planes into values.  The head carries
// the block's kind, its exponent and the decode_ints state the value half
// needs (bitplane.rs:626-667), packed into one word between the kernels.

enum : u32 { HEAD_ZERO = 0, HEAD_FLOAT = 1, HEAD_INT = 2, HEAD_REV_REINTERP = 3, HEAD_REV_FLOAT = 4, HEAD_REV_INT = 5 };

struct BlockHead {
  u32 kind;
  int emax;
  int low, high;  // stored planes [low, high]; low = intprec if none
  u32 m, prec;    // inverse-rounding arguments
  bool round;     // ROUND_LAST
  bool z;         // no plane stored

  // kind 3 bits, emax + 2048 12 bits, low 9, high + 1 9, m 9, prec 8, round, z.
  ZFPB_DEV u64 pack() const {
    return (u64)kind | ((u64)(u32)(emax + 2048) & 0xfff) << 3 | (u64)((u32)low & 0x1ff) << 15 |
           (u64)((u32)(high + 1) & 0x1ff) << 24 | (u64)(m & 0x1ff) << 33 | (u64)(prec & 0xff) << 42 |
           (u64)round << 50 | (u64)z << 51;
  }
  ZFPB_DEV static BlockHead unpack(u64 v) {
    BlockHead h;
    h.kind = (u32)(v & 7);
    h.emax = (int)((v >> 3) & 0xfff) - 2048;
    h.low = (int)((v >> 15) & 0x1ff);
    h.high = (int)((v >> 24) & 0x1ff) - 1;
    h.m = (u32)((v >> 33) & 0x1ff);
    h.prec = (u32)((v >> 42) & 0xff);
    h.round = (v >> 50) & 1;
    h.z = (v >> 51) & 1;
    return h;
  }
};

// decode_ints, stream half: read the planes into ps; returns bits read.
template <class U, int N>
ZFPB_DEV u32 parse_ints(Reader& r, u32 maxbits, u32 maxprec, int rounding, PlaneStore ps, BlockHead& h) {
  constexpr u32 intprec = sizeof(U) * 8;
  const bool constrained = with_maxbits(maxbits, maxprec, N);
  const u32 budget = constrained ? maxbits : 0xffffffffu;
  const u32 kmin = intprec > maxprec ? intprec - maxprec : 0;
  PlaneResult pr;
  if constexpr (N <= 64) pr = decode_planes_sync<N>(r, budget, kmin, intprec, ps);
  else pr = decode_planes<N>(r, budget, kmin, intprec, ps);
  h.low = pr.low;
  h.high = pr.high;
  h.z = pr.low == (int)intprec;
  h.round = rounding == 2;
  h.m = pr.m;
  h.prec = pr.prec;
  if (!constrained) {
    h.m = 0;
    h.prec = intprec - (kmin - 1);
  }
  return pr.bits;
}

// decode_ints, value half: planes -> coefficients, inverse rounding, then the
// inverse reorder and transform (decode/core.rs:97-131, KIND 1;
// decode/reversible.rs:46-82, KIND 3).
template <class I, int N, int KIND>
ZFPB_DEV void finish_int_block(const BlockHead& h, I* ib, PlaneStore ps) {
  typedef typename Traits<I>::U U;
  U u[N];
  if (h.z) {
#pragma unroll
    for (int i = 0; i < N; i++) u[i] = 0;
  } else {
    load_coded_planes<U, N>(u, ps, h.low, h.high);
  }
  if (h.round) inv_round<U, N>(u, h.m, h.prec);
  if (KIND == 1 && h.z && !h.round) {
#pragma unroll
    for (int i = 0; i < N; i++) ib[i] = 0;
  } else {
    inv_order<N>(u, ib);
    inv_axes<I, N, KIND>(ib);
  }
}

// decode/reversible.rs:46-82, stream half.
template <class U, int N>
ZFPB_DEV u32 parse_rev_int_block(Reader& r, u32 maxbits, PlaneStore ps, BlockHead& h) {
  constexpr u32 PB = sizeof(U) == 4 ? 5 : 6;
  u32 prec = (u32)r.read(PB) + 1;
  return PB + parse_ints<U, N>(r, sat_sub(maxbits, PB), prec, 0, ps, h);
}

// Stream half of decode_block: returns the bits the block occupies (after the
// skip to minbits) and, in *read_bits, the bits actually read.
template <class T, int N, bool LOSSY = false>
ZFPB_DEV u32 parse_block(Reader& r, const Codec& c, PlaneStore ps, BlockHead& h, u32* read_bits) {
  typedef typename Traits<T>::U U;
  h.emax = 0;
  h.low = h.high = 0;
  h.m = h.prec = 0;
  h.round = h.z = false;
  u32 bits;
  if (!LOSSY && c.minexp < ZFP_MIN_EXP) {
    if constexpr (!Traits<T>::FLOAT) {
      h.kind = HEAD_REV_INT;
      bits = parse_rev_int_block<U, N>(r, c.maxbits, ps, h);
    } else {
      if (r.read_bit() == 0) {
        h.kind = HEAD_ZERO;
        bits = 1;
      } else {
        bits = 2;
        if (r.read_bit()) {
          h.kind = HEAD_REV_REINTERP;
          bits += parse_rev_int_block<U, N>(r, sat_sub(c.maxbits, bits), ps, h);
        } else {
          h.kind = HEAD_REV_FLOAT;
          h.emax = (int)r.read(Traits<T>::EBITS) - Traits<T>::EBIAS;
          bits += Traits<T>::EBITS;
          bits += parse_rev_int_block<U, N>(r, sat_sub(c.maxbits, bits), ps, h);
        }
      }
    }
    *read_bits = bits;
    return bits < c.minbits ? c.minbits : bits;
  }
  if constexpr (Traits<T>::FLOAT) {
    if (r.read_bit()) {
      constexpr u32 hb = 1 + Traits<T>::EBITS;
      h.kind = HEAD_FLOAT;
      h.emax = (int)r.read(Traits<T>::EBITS) - Traits<T>::EBIAS;
      u32 prec = precision_f(h.emax, c.maxprec, c.minexp, Dims<N>::value, c.tight != 0);
      u32 ibits = parse_ints<U, N>(r, sat_sub(c.maxbits, hb), prec, c.rounding, ps, h);
      u32 mb = sat_sub(c.minbits, hb);
      *read_bits = hb + ibits;
      return hb + (ibits < mb ? mb : ibits);
    }
    h.kind = HEAD_ZERO;
    *read_bits = 1;
    return c.minbits > 1 ? c.minbits : 1;
  } else {
    h.kind = HEAD_INT;
    bits = parse_ints<U, N>(r, c.maxbits, c.maxprec, c.rounding, ps, h);
    *read_bits = bits;
    return bits < c.minbits ? c.minbits : bits;
  }
}

// Value half of decode_block.
template <class T, int N, bool LOSSY = false>
ZFPB_DEV void finish_block(const BlockHead& h, T* blk, PlaneStore ps) {
  typedef typename Traits<T>::I I;
  typedef typename Traits<T>::U U;
  if constexpr (LOSSY && Traits<T>::FLOAT) {
    // Lossy float streams: a block of zeros or a float block, nothing else.
    if (h.kind == HEAD_FLOAT) {
      I ib[N];
      finish_int_block<I, N, 1>(h, ib, ps);
      inv_cast<T, N>(ib, blk, h.emax);
    } else {
#pragma unroll
      for (int i = 0; i < N; i++) blk[i] = 0;
    }
    return;
  }
  if constexpr (!Traits<T>::FLOAT) {
    if (h.kind == HEAD_REV_INT) finish_int_block<I, N, 3>(h, reinterpret_cast<I*>(blk), ps);
    else finish_int_block<I, N, 1>(h, reinterpret_cast<I*>(blk), ps);
  } else {
    if (h.kind == HEAD_ZERO) {
#pragma unroll
      for (int i = 0; i < N; i++) blk[i] = 0;
      return;
    }
    I ib[N];
    if (h.kind == HEAD_FLOAT) {
      finish_int_block<I, N, 1>(h, ib, ps);
      inv_cast<T, N>(ib, blk, h.emax);
    } else {
      finish_int_block<I, N, 3>(h, ib, ps);
      if (h.kind == HEAD_REV_REINTERP) {
        const U tc = (U)(~(U)0) >> 1;
#pragma unroll
        for (int i = 0; i < N; i++) blk[i] = float_of(ib[i] < 0 ? (U)((U)ib[i] ^ tc) : (U)ib[i]);
      } else {
        inv_cast<T, N>(ib, blk, h.emax);
      }
    }
  }
}

}  // namespace zfpb
