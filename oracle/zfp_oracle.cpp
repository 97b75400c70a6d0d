// CPU oracle: a restatement of zfp-rs 1.0.1's compress/decompress path.
//
// TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU
// baseline of bench.py as the checker.  The GPU library does not use it.
//
// Each function names the zfp-rs file:line it follows (paths relative to the
// zfp-rs repository root).  Floating-point casts follow x86-64 semantics, as
// zfp-rs does (src/codec/encode/core.rs:385-423); build with -O2 and without
// -ffast-math so that every multiply rounds as IEEE single/double.

#include "zfp_oracle.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace orc {

typedef uint64_t u64;
typedef uint32_t u32;

// ---------------------------------------------------------------------------
// Bit stream: src/bitstream/core.rs:7-542
// ---------------------------------------------------------------------------

struct Stream {
  u64* words;
  size_t len;
  size_t word_pos = 0;
  u64 buffer = 0;
  u32 bits = 0;
  bool overflowed = false;
  bool overread = false;
  size_t seek_word = 0;
};

// core.rs:151-157
static inline u64 read_word_raw(Stream& s) {
  u64 w = s.word_pos < s.len ? s.words[s.word_pos] : 0;
  s.word_pos++;
  return w;
}

// core.rs:159-170
static inline void write_word_raw(Stream& s, u64 v) {
  if (s.word_pos < s.len)
    s.words[s.word_pos] = v;
  else
    s.overflowed = true;
  s.word_pos++;
}

// core.rs:192-229
static u64 read_bits(Stream& s, u32 n) {
  if (n > 64) n = 64;
  u64 value = s.buffer;
  if (s.bits < n) {
    u64 w = read_word_raw(s);
    s.buffer = w;
    value += w << s.bits;  // bits < n <= 64, and bits < 64 by invariant
    s.bits += 64;
    s.bits -= n;
    if (s.bits == 0) {
      s.buffer = 0;
    } else {
      s.buffer >>= (64 - s.bits);
      if (n < 64) value &= (2ull << (n - 1)) - 1;
    }
  } else {
    s.bits -= n;
    s.buffer = n < 64 ? s.buffer >> n : 0;
    if (n < 64) value &= (1ull << n) - 1;
  }
  return value;
}

// core.rs:235-247
static inline u32 read_bit(Stream& s) {
  if (s.bits == 0) {
    s.buffer = read_word_raw(s);
    s.bits = 64;
  }
  s.bits--;
  u32 bit = (u32)(s.buffer & 1);
  s.buffer >>= 1;
  return bit;
}

// core.rs:384-386
static inline bool loaded_since_seek(const Stream& s) {
  size_t m = s.len > s.seek_word ? s.len : s.seek_word;
  return s.word_pos > m;
}

// core.rs:265-284
static void seek_read(Stream& s, u64 offset) {
  u32 n = (u32)(offset % 64);
  s.overread |= loaded_since_seek(s);
  s.word_pos = (size_t)(offset / 64);
  s.seek_word = s.word_pos;
  if (n != 0) {
    u64 w = read_word_raw(s);
    s.buffer = w >> n;
    s.bits = 64 - n;
  } else {
    s.buffer = 0;
    s.bits = 0;
  }
}

// core.rs:296-326
static u64 write_bits(Stream& s, u64 value, u32 n) {
  if (n > 64) n = 64;
  s.buffer += value << s.bits;
  s.bits += n;
  if (s.bits >= 64) {
    u64 val = value >> 1;
    u32 remaining = n - 1;
    for (;;) {
      u32 after = s.bits - 64;
      u64 buf = s.buffer;
      s.bits = after;
      write_word_raw(s, buf);
      s.buffer = val >> (remaining - after);
      if (s.bits < 64) break;
    }
  }
  if (s.bits < 64) s.buffer &= (1ull << s.bits) - 1;
  return n < 64 ? value >> n : 0;
}

// core.rs:332-347
static inline u32 write_bit(Stream& s, u32 bit) {
  s.buffer += (u64)bit << s.bits;
  s.bits++;
  if (s.bits == 64) {
    write_word_raw(s, s.buffer);
    s.buffer = 0;
    s.bits = 0;
  }
  return bit;
}

// core.rs:354-375
static void seek_write(Stream& s, u64 offset) {
  u32 n = (u32)(offset % 64);
  s.word_pos = (size_t)(offset / 64);
  s.overflowed = false;
  if (n != 0) {
    s.buffer = s.word_pos < s.len ? (s.words[s.word_pos] & ((1ull << n) - 1)) : 0;
    s.bits = n;
  } else {
    s.buffer = 0;
    s.bits = 0;
  }
}

// core.rs:390-404
static inline bool overread(const Stream& s) { return s.overread || loaded_since_seek(s); }
static inline void reset_overread(Stream& s) {
  s.overread = false;
  s.seek_word = s.bits > 0 ? (s.word_pos > 0 ? s.word_pos - 1 : 0) : s.word_pos;
}

// core.rs:416-443
static inline u64 wtell(const Stream& s) { return (u64)s.word_pos * 64 + s.bits; }
static inline u64 rtell(const Stream& s) { return (u64)s.word_pos * 64 - s.bits; }
static inline void skip(Stream& s, u64 n) { seek_read(s, rtell(s) + n); }

// core.rs:460-478
static void pad(Stream& s, u64 n) {
  u64 bits = (u64)s.bits + n;
  while (bits >= 64) {
    if (s.word_pos >= s.len) {
      s.word_pos += (size_t)(bits / 64);
      s.buffer = 0;
      s.overflowed = true;
      bits %= 64;
      break;
    }
    write_word_raw(s, s.buffer);
    s.buffer = 0;
    bits -= 64;
  }
  s.bits = (u32)bits;
}

// core.rs:524-542
static u32 align(Stream& s) {
  u32 b = s.bits;
  if (b != 0) skip(s, b);
  return b;
}
static u32 flush(Stream& s) {
  u32 p = (64 - s.bits) % 64;
  if (p != 0) pad(s, p);
  return p;
}

// Register-cached reader with lookahead: core.rs:549-624.  Same effects as
// read_bits; the cursor is written back by sync().
struct Reader {
  Stream& s;
  size_t word_pos;
  u64 buffer;
  u32 bits;
  explicit Reader(Stream& st) : s(st), word_pos(st.word_pos), buffer(st.buffer), bits(st.bits) {}
  void sync() {
    s.word_pos = word_pos;
    s.buffer = buffer;
    s.bits = bits;
  }
  u64 next_word() const { return word_pos < s.len ? s.words[word_pos] : 0; }
  u64 peek() const { return buffer | (bits < 64 ? next_word() << bits : 0); }
  void consume(u32 n) {
    if (n <= bits) {
      buffer = n < 64 ? buffer >> n : 0;
      bits -= n;
    } else {
      u64 w = next_word();
      word_pos++;
      bits = bits + 64 - n;
      buffer = (w >> 1) >> (63 - bits);
    }
  }
  u64 read(u32 n) {
    u64 v = peek();
    consume(n);
    return n < 64 ? v & ((1ull << n) - 1) : v;
  }
};

// ---------------------------------------------------------------------------
// Scalar traits, constants: src/types.rs:327-344, encode/core.rs:309-325
// ---------------------------------------------------------------------------

template <class T> struct Tr;
template <> struct Tr<float> {
  typedef int32_t I; typedef uint32_t U;
  enum { EBITS = 8, EBIAS = 127, PREC = 32, PBITS = 5, FLOAT = 1, MIN_CAST_EMAX = -97 };
};
template <> struct Tr<double> {
  typedef int64_t I; typedef uint64_t U;
  enum { EBITS = 11, EBIAS = 1023, PREC = 64, PBITS = 6, FLOAT = 1, MIN_CAST_EMAX = -961 };
};
template <> struct Tr<int32_t> {
  typedef int32_t I; typedef uint32_t U;
  enum { EBITS = 0, EBIAS = 0, PREC = 32, PBITS = 5, FLOAT = 0, MIN_CAST_EMAX = 0 };
};
template <> struct Tr<int64_t> {
  typedef int64_t I; typedef uint64_t U;
  enum { EBITS = 0, EBIAS = 0, PREC = 64, PBITS = 6, FLOAT = 0, MIN_CAST_EMAX = 0 };
};

static const u32 ZFP_MIN_BITS = 1, ZFP_MAX_BITS = 16658, ZFP_MAX_PREC = 64;
static const int32_t ZFP_MIN_EXP = -1074;

template <class U> static inline U nbmask() { return (U)0xaaaaaaaaaaaaaaaaull; }

// Coefficient order tables: src/codec/encode/core.rs:12-39 (stream format).
static const unsigned char PERM_1[4] = {0, 1, 2, 3};
static const unsigned char PERM_2[16] = {0, 1, 4, 5, 2, 8, 6, 9, 3, 12, 10, 7, 13, 11, 14, 15};
static const unsigned char PERM_3[64] = {
    0,  1,  4,  16, 20, 17, 5,  2,  8,  32, 21, 6,  18, 24, 9,  33, 36, 3,  12, 48, 22, 25,
    37, 40, 34, 10, 7,  19, 28, 13, 49, 52, 41, 38, 26, 23, 29, 53, 11, 35, 44, 14, 50, 56,
    42, 27, 39, 45, 30, 54, 57, 60, 51, 15, 43, 46, 58, 61, 55, 31, 62, 59, 47, 63};
static const unsigned char PERM_4[256] = {
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

template <int N> static inline const unsigned char* perm_of() {
  return N == 4 ? PERM_1 : N == 16 ? PERM_2 : N == 64 ? PERM_3 : PERM_4;
}

// ---------------------------------------------------------------------------
// Transforms: src/codec/transform.rs:74-233
// ---------------------------------------------------------------------------

template <class I> static inline I wadd(I a, I b) {
  typedef typename std::make_unsigned<I>::type U;
  return (I)((U)a + (U)b);
}
template <class I> static inline I wsub(I a, I b) {
  typedef typename std::make_unsigned<I>::type U;
  return (I)((U)a - (U)b);
}

// transform.rs:74-86
template <class I> static inline void fwd_lift(I* p, int s) {
  I x = p[0], y = p[s], z = p[2 * s], w = p[3 * s];
  x = wadd(x, w) >> 1; w = wsub(w, x);
  z = wadd(z, y) >> 1; y = wsub(y, z);
  x = wadd(x, z) >> 1; z = wsub(z, x);
  w = wadd(w, y) >> 1; y = wsub(y, w);
  w = wadd(w, (I)(y >> 1));
  y = wsub(y, (I)(w >> 1));
  p[0] = x; p[s] = y; p[2 * s] = z; p[3 * s] = w;
}
// transform.rs:98-110
template <class I> static inline void inv_lift(I* p, int s) {
  I x = p[0], y = p[s], z = p[2 * s], w = p[3 * s];
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
  p[0] = x; p[s] = y; p[2 * s] = z; p[3 * s] = w;
}
// transform.rs:118-142
template <class I> static inline void rev_fwd_lift(I* p, int s) {
  I x = p[0], y = p[s], z = p[2 * s], w = p[3 * s];
  w = wsub(w, z); z = wsub(z, y); y = wsub(y, x);
  w = wsub(w, z); z = wsub(z, y); w = wsub(w, z);
  p[s] = y; p[2 * s] = z; p[3 * s] = w; (void)x;
}
template <class I> static inline void rev_inv_lift(I* p, int s) {
  I x = p[0], y = p[s], z = p[2 * s], w = p[3 * s];
  w = wadd(w, z); z = wadd(z, y); w = wadd(w, z);
  y = wadd(y, x); z = wadd(z, y); w = wadd(w, z);
  p[s] = y; p[2 * s] = z; p[3 * s] = w;
}

// transform.rs:151-170: lift every line along the axis of stride s.
template <class I, int N, void (*L)(I*, int)> static inline void lift_axis(I* p, int s) {
  for (int g = 0; g < N; g += 4 * s)
    for (int i = g; i < g + s; i++) L(p + i, s);
}
template <class I, int N> static void fwd_xform(I* p) {
  lift_axis<I, N, fwd_lift<I>>(p, 1);
  if (N >= 16) lift_axis<I, N, fwd_lift<I>>(p, 4);
  if (N >= 64) lift_axis<I, N, fwd_lift<I>>(p, 16);
  if (N >= 256) lift_axis<I, N, fwd_lift<I>>(p, 64);
}
template <class I, int N> static void inv_xform(I* p) {
  if (N >= 256) lift_axis<I, N, inv_lift<I>>(p, 64);
  if (N >= 64) lift_axis<I, N, inv_lift<I>>(p, 16);
  if (N >= 16) lift_axis<I, N, inv_lift<I>>(p, 4);
  lift_axis<I, N, inv_lift<I>>(p, 1);
}
template <class I, int N> static void rev_fwd_xform(I* p) {
  lift_axis<I, N, rev_fwd_lift<I>>(p, 1);
  if (N >= 16) lift_axis<I, N, rev_fwd_lift<I>>(p, 4);
  if (N >= 64) lift_axis<I, N, rev_fwd_lift<I>>(p, 16);
  if (N >= 256) lift_axis<I, N, rev_fwd_lift<I>>(p, 64);
}
template <class I, int N> static void rev_inv_xform(I* p) {
  if (N >= 256) lift_axis<I, N, rev_inv_lift<I>>(p, 64);
  if (N >= 64) lift_axis<I, N, rev_inv_lift<I>>(p, 16);
  if (N >= 16) lift_axis<I, N, rev_inv_lift<I>>(p, 4);
  lift_axis<I, N, rev_inv_lift<I>>(p, 1);
}

// ---------------------------------------------------------------------------
// Encode helpers: src/codec/encode/core.rs
// ---------------------------------------------------------------------------

// core.rs:53-74
template <class I> static void fwd_round(I* b, int n, u32 maxprec) {
  typedef typename std::make_unsigned<I>::type U;
  const u32 bits = sizeof(U) * 8;
  if (maxprec < bits) {
    I bias = (I)((U)(nbmask<U>() >> 2) >> maxprec);
    if (maxprec & 1)
      for (int i = 0; i < n; i++) b[i] = wadd(b[i], bias);
    else
      for (int i = 0; i < n; i++) b[i] = wsub(b[i], bias);
  }
}

// core.rs:82-109
template <class I> static inline typename std::make_unsigned<I>::type int2uint(I x) {
  typedef typename std::make_unsigned<I>::type U;
  return (U)((U)x + nbmask<U>()) ^ nbmask<U>();
}
template <class U> static inline typename std::make_signed<U>::type uint2int(U x) {
  typedef typename std::make_signed<U>::type I;
  return (I)((U)(x ^ nbmask<U>()) - nbmask<U>());
}

// core.rs:183-185
static inline bool with_maxbits(u32 maxbits, u32 maxprec, u32 size) {
  return ((u64)maxprec + 1) * (u64)size > (u64)maxbits + 1;
}

// core.rs:147-172
static inline u32 pad_to(Stream& s, u32 bits, u32 minbits) {
  if (bits < minbits) {
    pad(s, minbits - bits);
    return minbits;
  }
  return bits;
}
static inline u32 skip_to(Stream& s, u32 bits, u32 minbits) {
  if (bits < minbits) {
    skip(s, minbits - bits);
    return minbits;
  }
  return bits;
}

// core.rs:231-244
static inline u32 precision_f(int32_t maxexp, u32 maxprec, int32_t minexp, u32 dims, bool tight) {
  int64_t raw = (int64_t)maxexp - (int64_t)minexp + 2 * (int64_t)dims + (tight ? 1 : 2);
  if (raw < 0) raw = 0;
  if (raw > (int64_t)maxprec) raw = maxprec;
  return (u32)raw;
}

static inline u32 fbits(float f) { u32 u; memcpy(&u, &f, 4); return u; }
static inline u64 fbits(double f) { u64 u; memcpy(&u, &f, 8); return u; }
static inline float ffrom(u32 u) { float f; memcpy(&f, &u, 4); return f; }
static inline double ffrom(u64 u) { double f; memcpy(&f, &u, 8); return f; }

// core.rs:251-307: frexp exponent of the largest |x|, NaNs skipped.
template <class T> static int32_t exponent_block(const T* d, int n) {
  T m = 0;
  for (int i = 0; i < n; i++) {
    T a = std::fabs(d[i]);
    if (!(a <= (T)INFINITY)) a = 0;
    m = a > m ? a : m;
  }
  auto b = fbits(m);
  if (sizeof(T) == 4) {
    u32 e = (u32)(b >> 23);
    if (b == 0) return -127;
    if (e == 0xff) return 0;
    return (int32_t)e - 126;
  } else {
    u32 e = (u32)(b >> 52);
    if (b == 0) return -1023;
    if (e == 0x7ff) return 0;
    return (int32_t)e - 1022;
  }
}

// core.rs:385-423 (x86-64 truncation: out of range and NaN give the minimum)
static inline int32_t truncate(float v) {
  return (v >= -2147483648.0f && v < 2147483648.0f) ? (int32_t)v : INT32_MIN;
}
static inline int64_t truncate(double v) {
  return (v >= -9223372036854775808.0 && v < 9223372036854775808.0) ? (int64_t)v : INT64_MIN;
}

// core.rs:334-380
template <class T> static void fwd_cast(typename Tr<T>::I* ib, const T* fb, int n, int32_t emax) {
  const int ip = Tr<T>::PREC;
  if (emax < Tr<T>::MIN_CAST_EMAX) {
    T s = (T)std::ldexp((T)1, ip - 2 - 64 - emax);
    T two64 = (T)18446744073709551616.0;
    for (int i = 0; i < n; i++) {
      volatile T a = fb[i] * two64;
      ib[i] = truncate((T)(a * s));
    }
    return;
  }
  T s = (T)std::ldexp((T)1, ip - 2 - emax);
  for (int i = 0; i < n; i++) ib[i] = truncate((T)(s * fb[i]));
}

// decode/core.rs:162-175
template <class T> static void inv_cast(const typename Tr<T>::I* ib, T* fb, int n, int32_t emax) {
  const int ip = Tr<T>::PREC;
  T s = (T)std::ldexp((T)1, emax - (ip - 2));
  for (int i = 0; i < n; i++) fb[i] = s * (T)ib[i];
}

// ---------------------------------------------------------------------------
// Bit planes and the embedded coder: src/codec/bitplane.rs:75-790
// ---------------------------------------------------------------------------

// A plane of N <= 256 coefficients as W = ceil(N/64) words.
template <int N> struct Plane {
  enum { W = N <= 64 ? 1 : N / 64 };
  u64 w[W];
  void clear() { for (int i = 0; i < W; i++) w[i] = 0; }
  // bitplane.rs:125-128, :164-173
  bool next_one(u32 n, u32* p) const {
    u32 i = n / 64;
    if (i >= (u32)W) return false;
    u64 rest = w[i] >> (n % 64);
    if (rest) { *p = n + (u32)__builtin_ctzll(rest); return true; }
    for (u32 j = i + 1; j < (u32)W; j++)
      if (w[j]) { *p = 64 * j + (u32)__builtin_ctzll(w[j]); return true; }
    return false;
  }
  void set(u32 n) { w[n / 64] |= 1ull << (n % 64); }
};

static inline u64 low_mask(u32 n) { return n < 64 ? (1ull << n) - 1 : ~0ull; }

template <int N> static inline void write_low(Stream& s, const Plane<N>& x, u32 m) {
  u32 full = m / 64, rest = m % 64;
  for (u32 i = 0; i < full; i++) write_bits(s, x.w[i], 64);
  if (rest) write_bits(s, x.w[full] & low_mask(rest), rest);
}
template <int N> static inline Plane<N> read_low(Reader& r, u32 m) {
  Plane<N> x;
  x.clear();
  u32 full = m / 64, rest = m % 64;
  for (u32 i = 0; i < full; i++) x.w[i] = r.read(64);
  if (rest) x.w[full] = r.read(rest);
  return x;
}

static inline void put_zeros(Stream& s, u32 n) {
  while (n > 64) { write_bits(s, 0, 64); n -= 64; }
  write_bits(s, 0, n);
}

// Plane k of coefficients u: bit i = bit k of u[i].  64x64 bit transpose
// (Hacker's Delight 7-3, as bitplane.rs:75-92) one 64-coefficient chunk at a
// time.
static void transpose64(u64 a[64]) {
  static const u64 M[6] = {0x5555555555555555ull, 0x3333333333333333ull, 0x0f0f0f0f0f0f0f0full,
                           0x00ff00ff00ff00ffull, 0x0000ffff0000ffffull, 0x00000000ffffffffull};
  int s = 6;
  for (int j = 32; j != 0; j >>= 1) {
    s--;
    u64 m = M[s];
    for (int k = 0; k < 64; k += 2 * j)
      for (int i = k; i < k + j; i++) {
        u64 t = ((a[i] >> j) ^ a[i + j]) & m;
        a[i] ^= t << j;
        a[i + j] ^= t;
      }
  }
}

template <class U, int N> static void to_planes(const U* u, Plane<N>* planes) {
  const int P = sizeof(U) * 8;
  for (int k = 0; k < P; k++) planes[k].clear();
  if (N < 64) {
    for (int k = 0; k < P; k++) {
      u64 x = 0;
      for (int i = 0; i < N; i++) x |= (u64)((u[i] >> k) & 1) << i;
      planes[k].w[0] = x;
    }
    return;
  }
  for (int c = 0; c < N / 64; c++) {
    // Row r is coefficient r, column k its bit k; transposed, row k is plane k.
    u64 a[64];
    for (int r = 0; r < 64; r++) a[r] = (u64)u[64 * c + r];
    transpose64(a);
    for (int k = 0; k < P; k++) planes[k].w[c] = a[k];
  }
}

template <class U, int N> static void from_planes(const Plane<N>* planes, U* u) {
  const int P = sizeof(U) * 8;
  if (N < 64) {
    for (int i = 0; i < N; i++) {
      U v = 0;
      for (int k = 0; k < P; k++) v |= (U)((planes[k].w[0] >> i) & 1) << k;
      u[i] = v;
    }
    return;
  }
  for (int c = 0; c < N / 64; c++) {
    u64 a[64];
    for (int r = 0; r < 64; r++) a[r] = 0;
    for (int k = 0; k < P; k++) a[k] = planes[k].w[c];
    transpose64(a);
    for (int r = 0; r < 64; r++) u[64 * c + r] = (U)a[r];
  }
}

// bitplane.rs:509-610: encode one bit plane at a time from the MSB.
template <class U, int N> static u32 encode_ints(Stream& s, u32 maxbits, u32 maxprec, const U* u) {
  const u32 intprec = sizeof(U) * 8;
  const u32 size = N;
  u32 budget = with_maxbits(maxbits, maxprec, size) ? maxbits : 0xffffffffu;
  u32 kmin = intprec > maxprec ? intprec - maxprec : 0;
  Plane<N> planes[64];
  to_planes<U, N>(u, planes);
  U all = 0;
  for (int i = 0; i < N; i++) all |= u[i];
  u32 top = 0;
  for (u32 b = 0; b < intprec; b++)
    if ((all >> b) & 1) top = b + 1;

  u32 bits = budget;
  u32 n = 0;
  u32 tk = top > kmin ? top : kmin;
  u32 empty = intprec - tk;
  if (empty > bits) empty = bits;
  put_zeros(s, empty);
  bits -= empty;
  u32 k = intprec - empty;
  while (bits != 0 && k > kmin) {
    if (n == size) {
      while (bits > size && k > kmin) {
        k--;
        write_low(s, planes[k], size);
        bits -= size;
      }
      if (k == kmin) break;
    }
    k--;
    const Plane<N>& x = planes[k];
    u32 m = n < bits ? n : bits;
    bits -= m;
    write_low(s, x, m);
    while (bits != 0 && n < size) {
      u32 p;
      if (!x.next_one(n, &p)) {
        write_bits(s, 0, 1);
        bits -= 1;
        break;
      }
      u32 zeros = p - n;
      bool last = p == size - 1;
      u32 len = zeros + 2 - (last ? 1 : 0);
      u32 take = len < bits ? len : bits;
      if (take <= 64) {
        u64 code = (last || zeros >= 63) ? 1 : (1 | (2ull << zeros));
        write_bits(s, code & low_mask(take), take);
      } else {
        write_bits(s, 1, 1);
        put_zeros(s, zeros < take - 1 ? zeros : take - 1);
        if (take == len && !last) write_bits(s, 1, 1);
      }
      bits -= take;
      n = p + 1;
    }
  }
  return budget - bits;
}

static inline u32 ctz64(u64 x) { return x ? (u32)__builtin_ctzll(x) : 64; }

// bitplane.rs:775-790
static void scan_zeros(Reader& r, u32& bits, u32& n, u32 limit) {
  while (limit != 0) {
    u32 zeros = ctz64(r.peek());
    u32 span = limit < 64 ? limit : 64;
    if (zeros < span) {
      r.consume(zeros + 1);
      bits -= zeros + 1;
      n += zeros;
      return;
    }
    r.consume(span);
    bits -= span;
    n += span;
    limit -= span;
  }
}

struct PlaneResult { u32 bits, m, prec, low; };

// bitplane.rs:675-770
template <int N>
static PlaneResult decode_planes(Reader& r, u32 budget, u32 kmin, u32 intprec, Plane<N>* planes) {
  const u32 size = N;
  u32 bits = budget, n = 0, m = 0, k = intprec, low = intprec;
  while (bits != 0) {
    m = 0;
    if (k <= kmin) { k = k - 1; break; }
    if (n == 0) {
      u32 empty = ctz64(r.peek());
      if (empty > k - kmin) empty = k - kmin;
      if (empty > bits) empty = bits;
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
        planes[k] = read_low<N>(r, size);
        bits -= size;
        low = k;
      }
      if (k == kmin) { k = k - 1; break; }
    }
    k--;
    m = n < bits ? n : bits;
    bits -= m;
    Plane<N> x = read_low<N>(r, m);
    while (bits != 0 && n < size) {
      u64 ahead = r.peek();
      bits -= 1;
      if ((ahead & 1) == 0) {
        r.consume(1);
        m = size;
        break;
      }
      u32 limit = size - 1 - n;
      if (limit > bits) limit = bits;
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
        scan_zeros(r, bits, n, limit - 63);
      }
      x.set(n);
      n += 1;
      m = n;
    }
    planes[k] = x;
    low = k;
  }
  if (n == 0) low = intprec;
  PlaneResult res = {budget - bits, m, intprec - k, low};
  return res;
}

// decode/core.rs:62-82
template <class U> static void inv_round(U* d, int n, u32 m, u32 prec) {
  const u32 B = sizeof(U) * 8;
  if (prec < B - 1) {
    u32 mm = m < (u32)n ? m : (u32)n;
    U hi = (U)(nbmask<U>() >> 2) >> prec;
    U lo = (U)(nbmask<U>() >> 1) >> prec;
    for (u32 i = 0; i < mm; i++) d[i] += hi;
    for (u32 i = mm; i < (u32)n; i++) d[i] += lo;
  }
}

// The stream half of decode_ints: the planes and the reader's state, which
// finish_ints turns into coefficients (bitplane.rs:626-667; the pipeline's
// read stage keeps exactly this per block, decode/staged.rs:216-267).
template <class U, int N> struct IntsRead {
  Plane<N> planes[64];
  PlaneResult pr;
  bool constrained;
  u32 kmin;
  int rounding;
};

template <class U, int N>
static u32 read_ints(Stream& s, u32 maxbits, u32 maxprec, int rounding, IntsRead<U, N>& st) {
  const u32 intprec = sizeof(U) * 8;
  st.constrained = with_maxbits(maxbits, maxprec, N);
  u32 budget = st.constrained ? maxbits : 0xffffffffu;
  st.kmin = intprec > maxprec ? intprec - maxprec : 0;
  st.rounding = rounding;
  for (u32 k = 0; k < intprec; k++) st.planes[k].clear();
  Reader r(s);
  st.pr = decode_planes<N>(r, budget, st.kmin, intprec, st.planes);
  r.sync();
  return st.pr.bits;
}

// The value half of decode_ints: fills u; returns the `zero` flag.
template <class U, int N> static bool finish_ints(const IntsRead<U, N>& st, U* u) {
  const u32 intprec = sizeof(U) * 8;
  bool zero = st.pr.low == intprec;
  if (zero)
    for (int i = 0; i < N; i++) u[i] = 0;
  else
    from_planes<U, N>(st.planes, u);
  bool round = st.rounding == 2;
  if (round) {
    u32 m = st.pr.m, prec = st.pr.prec;
    if (!st.constrained) { m = 0; prec = intprec - (st.kmin - 1); }
    inv_round<U>(u, N, m, prec);
  }
  return zero && !round;
}

// bitplane.rs:626-667: returns bits read; fills u and *zero.
template <class U, int N>
static u32 decode_ints(Stream& s, u32 maxbits, u32 maxprec, int rounding, U* u, bool* zero_out) {
  IntsRead<U, N> st;
  u32 bits = read_ints<U, N>(s, maxbits, maxprec, rounding, st);
  *zero_out = finish_ints<U, N>(st, u);
  return bits;
}

// ---------------------------------------------------------------------------
// Block encoders/decoders: encode/{float,integer,reversible}.rs,
// decode/{core,reversible}.rs
// ---------------------------------------------------------------------------

struct Cfg {
  u32 minbits, maxbits, maxprec;
  int32_t minexp;
  int rounding;
  bool tight;
  bool reversible() const { return minexp < ZFP_MIN_EXP; }  // config.rs:533-535
};

static inline u32 sat_sub(u32 a, u32 b) { return a > b ? a - b : 0; }

// encode/integer.rs:50-93
template <class I, int N>
static u32 encode_int_block(Stream& s, const I* iblock, u32 minbits, u32 maxbits, u32 maxprec,
                            int rounding) {
  typedef typename std::make_unsigned<I>::type U;
  I b[N];
  memcpy(b, iblock, sizeof(b));
  fwd_xform<I, N>(b);
  if (rounding == 1) fwd_round(b, N, maxprec);
  U u[N];
  const unsigned char* perm = perm_of<N>();
  for (int i = 0; i < N; i++) u[i] = int2uint(b[perm[i]]);
  u32 bits = encode_ints<U, N>(s, maxbits, maxprec, u);
  return pad_to(s, bits, minbits);
}

// encode/float.rs:22-113
template <class T, int N> static u32 encode_float_block(Stream& s, const T* fb, const Cfg& c) {
  typedef typename Tr<T>::I I;
  const u32 dims = N == 4 ? 1 : N == 16 ? 2 : N == 64 ? 3 : 4;
  int32_t emax = exponent_block(fb, N);
  u32 prec = precision_f(emax, c.maxprec, c.minexp, dims, c.tight);
  u32 e = prec != 0 ? (u32)(emax + Tr<T>::EBIAS) : 0;
  if (e != 0) {
    const u32 hb = Tr<T>::EBITS + 1;
    u32 bmin = sat_sub(c.minbits, hb), bmax = sat_sub(c.maxbits, hb);
    write_bits(s, 2 * (u64)e + 1, hb);
    I ib[N];
    fwd_cast<T>(ib, fb, N, emax);
    return hb + encode_int_block<I, N>(s, ib, bmin, bmax, prec, c.rounding);
  }
  write_bit(s, 0);
  return pad_to(s, 1, c.minbits);
}

// encode/reversible.rs:35-45
template <class U> static u32 rev_precision(const U* d, int n) {
  U o = 0;
  for (int i = 0; i < n; i++) o |= d[i];
  if (o == 0) return 0;
  return (u32)(sizeof(U) * 8) - (u32)__builtin_ctzll((u64)o);
}

// encode/reversible.rs:89-137: fwd_order, precision header, planes.
template <class I, int N>
static u32 rev_encode_int_block(Stream& s, const I* ib, u32 maxbits, u32 maxprec) {
  typedef typename std::make_unsigned<I>::type U;
  const u32 PB = sizeof(U) == 4 ? 5 : 6;
  U u[N];
  const unsigned char* perm = perm_of<N>();
  for (int i = 0; i < N; i++) u[i] = int2uint(ib[perm[i]]);
  u32 prec = rev_precision(u, N);
  if (prec > maxprec) prec = maxprec;
  if (prec < 1) prec = 1;
  write_bits(s, prec - 1, PB);
  u32 mb = sat_sub(maxbits, PB);
  return PB + encode_ints<U, N>(s, mb, prec, u);
}

// encode/reversible.rs:279-313 (integers)
template <class I, int N> static u32 rev_encode_int(Stream& s, const I* in, const Cfg& c) {
  I b[N];
  memcpy(b, in, sizeof(b));
  rev_fwd_xform<I, N>(b);
  u32 bits = rev_encode_int_block<I, N>(s, b, c.maxbits, c.maxprec);
  return pad_to(s, bits, c.minbits);
}

// encode/reversible.rs:172-261 (floats)
template <class T, int N> static u32 rev_encode_float(Stream& s, const T* fb, const Cfg& c) {
  typedef typename Tr<T>::I I;
  typedef typename Tr<T>::U U;
  int32_t emax = exponent_block(fb, N);
  u32 e = (u32)(emax + Tr<T>::EBIAS);
  bool tiny = e != 0 && emax < Tr<T>::MIN_CAST_EMAX;
  I ib[N];
  for (int i = 0; i < N; i++) ib[i] = 0;
  if (e != 0 && !tiny) fwd_cast<T>(ib, fb, N, emax);
  bool rev = false;
  if (!tiny) {
    rev = true;
    const int ip = Tr<T>::PREC;
    T sc = (T)std::ldexp((T)1, emax - (ip - 2));
    for (int i = 0; i < N; i++) {
      T rec = sc * (T)ib[i];
      if (fbits(rec) != fbits(fb[i])) { rev = false; break; }
    }
  }
  u32 bits;
  if (rev) {
    if (e != 0) {
      write_bits(s, 1, 2);
      write_bits(s, e, Tr<T>::EBITS);
      u32 hb = 2 + Tr<T>::EBITS;
      rev_fwd_xform<I, N>(ib);
      bits = hb + rev_encode_int_block<I, N>(s, ib, sat_sub(c.maxbits, hb), c.maxprec);
    } else {
      write_bit(s, 0);
      bits = 1;
    }
  } else {
    const U tc = (U)(~(U)0) >> 1;
    for (int i = 0; i < N; i++) {
      U b = (U)fbits(fb[i]);
      ib[i] = (b >> (sizeof(U) * 8 - 1)) ? (I)(b ^ tc) : (I)b;
    }
    write_bits(s, 3, 2);
    rev_fwd_xform<I, N>(ib);
    bits = 2 + rev_encode_int_block<I, N>(s, ib, sat_sub(c.maxbits, 2), c.maxprec);
  }
  return pad_to(s, bits, c.minbits);
}

// decode/core.rs:97-131
template <class I, int N>
static void decode_int_block(Stream& s, u32 minbits, u32 maxbits, u32 maxprec, int rounding, I* ib) {
  typedef typename std::make_unsigned<I>::type U;
  U u[N];
  bool zero;
  u32 bits = decode_ints<U, N>(s, maxbits, maxprec, rounding, u, &zero);
  skip_to(s, bits, minbits);
  for (int i = 0; i < N; i++) ib[i] = 0;
  if (!zero) {
    const unsigned char* perm = perm_of<N>();
    for (int i = 0; i < N; i++) ib[perm[i]] = uint2int(u[i]);
    inv_xform<I, N>(ib);
  }
}

// decode/core.rs:184-237
template <class T, int N> static void decode_float_block(Stream& s, const Cfg& c, T* fb) {
  typedef typename Tr<T>::I I;
  const u32 dims = N == 4 ? 1 : N == 16 ? 2 : N == 64 ? 3 : 4;
  for (int i = 0; i < N; i++) fb[i] = 0;
  if (read_bit(s)) {
    const u32 hb = 1 + Tr<T>::EBITS;
    int32_t emax = (int32_t)read_bits(s, Tr<T>::EBITS) - Tr<T>::EBIAS;
    u32 prec = precision_f(emax, c.maxprec, c.minexp, dims, c.tight);
    I ib[N];
    decode_int_block<I, N>(s, sat_sub(c.minbits, hb), sat_sub(c.maxbits, hb), prec, c.rounding, ib);
    inv_cast<T>(ib, fb, N, emax);
  } else {
    skip_to(s, 1, c.minbits);
  }
}

// decode/reversible.rs:46-82
template <class I, int N> static u32 rev_decode_int_block(Stream& s, u32 maxbits, I* ib) {
  typedef typename std::make_unsigned<I>::type U;
  const u32 PB = sizeof(U) == 4 ? 5 : 6;
  u32 prec = (u32)read_bits(s, PB) + 1;
  u32 mb = sat_sub(maxbits, PB);
  U u[N];
  bool zero;
  u32 ub = decode_ints<U, N>(s, mb, prec, 0, u, &zero);
  const unsigned char* perm = perm_of<N>();
  for (int i = 0; i < N; i++) ib[perm[i]] = uint2int(u[i]);
  return PB + ub;
}

// decode/reversible.rs:212-228 (integers)
template <class I, int N> static void rev_decode_int(Stream& s, const Cfg& c, I* ib) {
  u32 bits = rev_decode_int_block<I, N>(s, c.maxbits, ib);
  skip_to(s, bits, c.minbits);
  rev_inv_xform<I, N>(ib);
}

// decode/reversible.rs:130-194 (floats)
template <class T, int N> static void rev_decode_float(Stream& s, const Cfg& c, T* fb) {
  typedef typename Tr<T>::I I;
  typedef typename Tr<T>::U U;
  if (read_bits(s, 1) == 0) {
    for (int i = 0; i < N; i++) fb[i] = 0;
    skip_to(s, 1, c.minbits);
    return;
  }
  u32 bits = 2;
  u64 reinterpret = read_bits(s, 1);
  I ib[N];
  if (reinterpret) {
    bits += rev_decode_int_block<I, N>(s, sat_sub(c.maxbits, bits), ib);
    rev_inv_xform<I, N>(ib);
    const U tc = (U)(~(U)0) >> 1;
    for (int i = 0; i < N; i++) {
      U x = ib[i] < 0 ? (U)((U)ib[i] ^ tc) : (U)ib[i];
      fb[i] = ffrom(x);
    }
  } else {
    int32_t emax = (int32_t)read_bits(s, Tr<T>::EBITS) - Tr<T>::EBIAS;
    bits += Tr<T>::EBITS;
    bits += rev_decode_int_block<I, N>(s, sat_sub(c.maxbits, bits), ib);
    rev_inv_xform<I, N>(ib);
    inv_cast<T>(ib, fb, N, emax);
  }
  skip_to(s, bits, c.minbits);
}

// ---------------------------------------------------------------------------
// Gather / scatter: encode/dim{1..4}.rs, encode/core.rs:194-219,
// decode/dim{1..4}.rs
// ---------------------------------------------------------------------------

// Pad a run of 4 at offset o, stride st, with n real values (C pad_block).
template <class T> static inline void pad_run(T* b, int o, int n, int st) {
  switch (n) {
    case 0: b[o] = 0; b[o + st] = b[o]; b[o + 2 * st] = b[o + st]; b[o + 3 * st] = b[o]; break;
    case 1: b[o + st] = b[o]; b[o + 2 * st] = b[o + st]; b[o + 3 * st] = b[o]; break;
    case 2: b[o + 2 * st] = b[o + st]; b[o + 3 * st] = b[o]; break;
    case 3: b[o + 3 * st] = b[o]; break;
    default: break;
  }
}

// Gather a (possibly partial) block of 4^D values; len[d] in 1..4.
template <class T, int D>
static void gather(const T* p, const ptrdiff_t* st, const size_t* len, T* b) {
  const int N = 1 << (2 * D);
  for (int i = 0; i < N; i++) b[i] = 0;
  int nx = (int)len[0], ny = D > 1 ? (int)len[1] : 1, nz = D > 2 ? (int)len[2] : 1,
      nw = D > 3 ? (int)len[3] : 1;
  ptrdiff_t sx = st[0], sy = D > 1 ? st[1] : 0, sz = D > 2 ? st[2] : 0, sw = D > 3 ? st[3] : 0;
  for (int w = 0; w < nw; w++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) b[x + 4 * y + 16 * z + 64 * w] = p[x * sx + y * sy + z * sz + w * sw];
  // Pad x in every filled row, then y, then z, then w (dim3.rs:57-77).
  if (D == 1) { pad_run(b, 0, nx, 1); return; }
  for (int w = 0; w < nw; w++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) pad_run(b, 4 * y + 16 * z + 64 * w, nx, 1);
  for (int w = 0; w < nw; w++)
    for (int z = 0; z < nz; z++)
      for (int x = 0; x < 4; x++) pad_run(b, 16 * z + 64 * w + x, ny, 4);
  if (D == 2) return;
  for (int w = 0; w < nw; w++)
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) pad_run(b, 64 * w + 4 * y + x, nz, 16);
  if (D == 3) return;
  for (int z = 0; z < 4; z++)
    for (int y = 0; y < 4; y++)
      for (int x = 0; x < 4; x++) pad_run(b, 16 * z + 4 * y + x, nw, 64);
}

template <class T, int D>
static void scatter(const T* b, T* p, const ptrdiff_t* st, const size_t* len) {
  int nx = (int)len[0], ny = D > 1 ? (int)len[1] : 1, nz = D > 2 ? (int)len[2] : 1,
      nw = D > 3 ? (int)len[3] : 1;
  ptrdiff_t sx = st[0], sy = D > 1 ? st[1] : 0, sz = D > 2 ? st[2] : 0, sw = D > 3 ? st[3] : 0;
  for (int w = 0; w < nw; w++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) p[x * sx + y * sy + z * sz + w * sw] = b[x + 4 * y + 16 * z + 64 * w];
}

// One block, gathered, encoded (codec/block/strided.rs:296-557).
template <class T, int D>
static u32 encode_block(Stream& s, const T* p, const ptrdiff_t* st, const size_t* len, const Cfg& c) {
  const int N = 1 << (2 * D);
  T b[N];
  gather<T, D>(p, st, len, b);
  if constexpr (Tr<T>::FLOAT) {
    if (c.reversible()) return rev_encode_float<T, N>(s, b, c);
    return encode_float_block<T, N>(s, b, c);
  } else {
    if (c.reversible()) return rev_encode_int<T, N>(s, b, c);
    return encode_int_block<T, N>(s, b, c.minbits, c.maxbits, c.maxprec, c.rounding);
  }
}

template <class T, int D>
static void decode_block(Stream& s, T* p, const ptrdiff_t* st, const size_t* len, const Cfg& c) {
  const int N = 1 << (2 * D);
  T b[N];
  if constexpr (Tr<T>::FLOAT) {
    if (c.reversible())
      rev_decode_float<T, N>(s, c, b);
    else
      decode_float_block<T, N>(s, c, b);
  } else {
    if (c.reversible())
      rev_decode_int<T, N>(s, c, b);
    else
      decode_int_block<T, N>(s, c.minbits, c.maxbits, c.maxprec, c.rounding, b);
  }
  scatter<T, D>(b, p, st, len);
}

// ---------------------------------------------------------------------------
// Field plan: src/field_plan.rs:41-206, src/field.rs:541-735
// ---------------------------------------------------------------------------

struct Plan {
  int dims;
  size_t n[4];
  ptrdiff_t s[4];
  size_t bx, by, bz, bw, blocks;
};

static bool make_plan(const orc_field* f, Plan& p) {
  size_t n[4] = {f->nx, f->ny, f->nz, f->nw};
  if (n[0] == 0) return false;
  p.dims = n[1] == 0 ? 1 : n[2] == 0 ? 2 : n[3] == 0 ? 3 : 4;
  for (int i = p.dims; i < 4; i++)
    if (n[i] != 0) return false;
  ptrdiff_t st[4] = {f->sx, f->sy, f->sz, f->sw};
  size_t nat = 1;
  for (int i = 0; i < 4; i++) {
    p.n[i] = i < p.dims ? n[i] : 0;
    p.s[i] = st[i] != 0 ? st[i] : (ptrdiff_t)nat;
    if (i < p.dims) nat *= n[i];
  }
  p.bx = (n[0] + 3) / 4;
  p.by = p.dims >= 2 ? (n[1] + 3) / 4 : 1;
  p.bz = p.dims >= 3 ? (n[2] + 3) / 4 : 1;
  p.bw = p.dims >= 4 ? (n[3] + 3) / 4 : 1;
  p.blocks = p.bx * p.by * p.bz * p.bw;
  return true;
}

static void block_geometry(const Plan& p, size_t idx, ptrdiff_t* off, size_t* len) {
  size_t c[4];
  c[0] = idx % p.bx; idx /= p.bx;
  c[1] = idx % p.by; idx /= p.by;
  c[2] = idx % p.bz; idx /= p.bz;
  c[3] = idx;
  *off = 0;
  for (int d = 0; d < 4; d++) {
    len[d] = 0;
    if (d < p.dims) {
      size_t o = 4 * c[d];
      *off += (ptrdiff_t)o * p.s[d];
      size_t r = p.n[d] - o;
      len[d] = r < 4 ? r : 4;
    }
  }
}

template <class T, int D>
static void run_blocks_enc(Stream& s, const Plan& p, const T* data, const Cfg& c, size_t b0, size_t b1) {
  for (size_t i = b0; i < b1; i++) {
    ptrdiff_t off;
    size_t len[4];
    block_geometry(p, i, &off, len);
    encode_block<T, D>(s, data + off, p.s, len, c);
  }
}
template <class T, int D>
static void run_blocks_dec(Stream& s, const Plan& p, T* data, const Cfg& c, size_t b0, size_t b1) {
  for (size_t i = b0; i < b1; i++) {
    ptrdiff_t off;
    size_t len[4];
    block_geometry(p, i, &off, len);
    decode_block<T, D>(s, data + off, p.s, len, c);
  }
}

template <class T>
static void enc_range(Stream& s, const Plan& p, const void* data, const Cfg& c, size_t b0, size_t b1) {
  switch (p.dims) {
    case 1: run_blocks_enc<T, 1>(s, p, (const T*)data, c, b0, b1); break;
    case 2: run_blocks_enc<T, 2>(s, p, (const T*)data, c, b0, b1); break;
    case 3: run_blocks_enc<T, 3>(s, p, (const T*)data, c, b0, b1); break;
    default: run_blocks_enc<T, 4>(s, p, (const T*)data, c, b0, b1); break;
  }
}
template <class T>
static void dec_range(Stream& s, const Plan& p, void* data, const Cfg& c, size_t b0, size_t b1) {
  switch (p.dims) {
    case 1: run_blocks_dec<T, 1>(s, p, (T*)data, c, b0, b1); break;
    case 2: run_blocks_dec<T, 2>(s, p, (T*)data, c, b0, b1); break;
    case 3: run_blocks_dec<T, 3>(s, p, (T*)data, c, b0, b1); break;
    default: run_blocks_dec<T, 4>(s, p, (T*)data, c, b0, b1); break;
  }
}

static void enc_any(int type, Stream& s, const Plan& p, const void* d, const Cfg& c, size_t b0, size_t b1) {
  switch (type) {
    case 1: enc_range<int32_t>(s, p, d, c, b0, b1); break;
    case 2: enc_range<int64_t>(s, p, d, c, b0, b1); break;
    case 3: enc_range<float>(s, p, d, c, b0, b1); break;
    default: enc_range<double>(s, p, d, c, b0, b1); break;
  }
}
static void dec_any(int type, Stream& s, const Plan& p, void* d, const Cfg& c, size_t b0, size_t b1) {
  switch (type) {
    case 1: dec_range<int32_t>(s, p, d, c, b0, b1); break;
    case 2: dec_range<int64_t>(s, p, d, c, b0, b1); break;
    case 3: dec_range<float>(s, p, d, c, b0, b1); break;
    default: dec_range<double>(s, p, d, c, b0, b1); break;
  }
}

// ---------------------------------------------------------------------------
// Staged block decoding: src/codec/decode/staged.rs.  read_block parses one
// block's headers and bit planes and leaves the cursor after its padding;
// reconstruct turns what it read into the block's values.  Together they do
// what decode_block does, split so that the halves can run on different
// threads.
// ---------------------------------------------------------------------------

enum { ST_ZERO, ST_FLOAT, ST_INT, ST_REV_INT, ST_REV_FLOAT, ST_REV_REINTERP };

template <class T, int N> struct StagedBlock {
  IntsRead<typename Tr<T>::U, N> ints;
  int kind;
  int32_t emax;
};

// staged.rs:216-267 (the grammar of decode/core.rs:97-237 and
// decode/reversible.rs:46-228).
template <class T, int N> static void read_block(Stream& s, const Cfg& c, StagedBlock<T, N>& b) {
  typedef typename Tr<T>::U U;
  const u32 dims = N == 4 ? 1 : N == 16 ? 2 : N == 64 ? 3 : 4;
  const u32 PB = sizeof(U) == 4 ? 5 : 6;
  b.emax = 0;
  if (c.reversible()) {
    if constexpr (Tr<T>::FLOAT) {
      if (read_bits(s, 1) == 0) {
        b.kind = ST_ZERO;
        skip_to(s, 1, c.minbits);
        return;
      }
      u32 bits = 2;
      if (read_bits(s, 1)) {
        b.kind = ST_REV_REINTERP;
      } else {
        b.kind = ST_REV_FLOAT;
        b.emax = (int32_t)read_bits(s, Tr<T>::EBITS) - Tr<T>::EBIAS;
        bits += Tr<T>::EBITS;
      }
      u32 mb = sat_sub(c.maxbits, bits);
      u32 prec = (u32)read_bits(s, PB) + 1;
      bits += PB + read_ints<U, N>(s, sat_sub(mb, PB), prec, 0, b.ints);
      skip_to(s, bits, c.minbits);
    } else {
      b.kind = ST_REV_INT;
      u32 prec = (u32)read_bits(s, PB) + 1;
      u32 bits = PB + read_ints<U, N>(s, sat_sub(c.maxbits, PB), prec, 0, b.ints);
      skip_to(s, bits, c.minbits);
    }
    return;
  }
  if constexpr (Tr<T>::FLOAT) {
    if (read_bit(s)) {
      const u32 hb = 1 + Tr<T>::EBITS;
      b.kind = ST_FLOAT;
      b.emax = (int32_t)read_bits(s, Tr<T>::EBITS) - Tr<T>::EBIAS;
      u32 prec = precision_f(b.emax, c.maxprec, c.minexp, dims, c.tight);
      u32 bits = read_ints<U, N>(s, sat_sub(c.maxbits, hb), prec, c.rounding, b.ints);
      skip_to(s, bits, sat_sub(c.minbits, hb));
    } else {
      b.kind = ST_ZERO;
      skip_to(s, 1, c.minbits);
    }
  } else {
    b.kind = ST_INT;
    u32 bits = read_ints<U, N>(s, c.maxbits, c.maxprec, c.rounding, b.ints);
    skip_to(s, bits, c.minbits);
  }
}

// staged.rs:52-144 (Scalar::reconstruct).
template <class T, int N> static void reconstruct(const StagedBlock<T, N>& b, T* fb) {
  typedef typename Tr<T>::I I;
  typedef typename Tr<T>::U U;
  if (b.kind == ST_ZERO) {
    for (int i = 0; i < N; i++) fb[i] = 0;
    return;
  }
  const unsigned char* perm = perm_of<N>();
  U u[N];
  I ib[N];
  bool zero = finish_ints<U, N>(b.ints, u);
  if (b.kind == ST_FLOAT || b.kind == ST_INT) {
    for (int i = 0; i < N; i++) ib[i] = 0;
    if (!zero) {
      for (int i = 0; i < N; i++) ib[perm[i]] = uint2int(u[i]);
      inv_xform<I, N>(ib);
    }
  } else {
    for (int i = 0; i < N; i++) ib[perm[i]] = uint2int(u[i]);
    rev_inv_xform<I, N>(ib);
  }
  if constexpr (Tr<T>::FLOAT) {
    if (b.kind == ST_REV_REINTERP) {
      const U tc = (U)(~(U)0) >> 1;
      for (int i = 0; i < N; i++) fb[i] = ffrom(ib[i] < 0 ? (U)((U)ib[i] ^ tc) : (U)ib[i]);
    } else {
      inv_cast<T>(ib, fb, N, b.emax);
    }
  } else {
    for (int i = 0; i < N; i++) fb[i] = ib[i];
  }
}

// field_plan.rs:92-118: whether two index tuples may address one element.
static bool strides_may_alias(const Plan& p) {
  size_t st[4], dm[4];
  int k = 0;
  for (int d = 0; d < p.dims; d++)
    if (p.n[d] >= 2) {
      st[k] = (size_t)(p.s[d] < 0 ? -p.s[d] : p.s[d]);
      dm[k] = p.n[d];
      k++;
    }
  for (int i = 1; i < k; i++)  // sort by (stride, dim)
    for (int j = i; j > 0 && (st[j] < st[j - 1] || (st[j] == st[j - 1] && dm[j] < dm[j - 1])); j--) {
      std::swap(st[j], st[j - 1]);
      std::swap(dm[j], dm[j - 1]);
    }
  size_t reach = 1;
  for (int i = 0; i < k; i++) {
    if (st[i] < reach) return true;
    unsigned __int128 r = (unsigned __int128)st[i] * (dm[i] - 1) + reach;
    reach = r > (unsigned __int128)SIZE_MAX ? SIZE_MAX : (size_t)r;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Variable-rate decode pipeline: src/decompress/pipeline.rs:15-229.  The
// calling thread is the only reader of the stream: it reads batches of
// blocks (64 KiB of staged blocks each) in stream order into a pool of at
// most 16 buffers, and `threads - 1` workers reconstruct finished batches
// and scatter them into disjoint blocks of the field.  Returns false,
// having read nothing, where the reference falls back to the serial
// decoder: 1-D fields, fewer than two threads, a field of one batch.
// ---------------------------------------------------------------------------

template <class T, int D>
static bool decode_pipelined(Stream& s, const Plan& p, T* data, const Cfg& c, int threads) {
  constexpr int N = 1 << (2 * D);
  typedef StagedBlock<T, N> B;
  if (D == 1 || threads < 2) return false;
  const size_t batch_len = std::max<size_t>(1, 65536 / sizeof(B));
  if (batch_len >= p.blocks) return false;
  const size_t depth = std::min<size_t>(16, (p.blocks + batch_len - 1) / batch_len);
  std::vector<std::vector<B>> bufs(depth, std::vector<B>(batch_len));
  std::vector<size_t> first(depth), count(depth);
  std::mutex mu;
  std::condition_variable cv_free, cv_work;
  std::deque<size_t> free_q, work_q;
  bool done = false;
  for (size_t i = 0; i < depth; i++) free_q.push_back(i);
  auto worker = [&]() {
    for (;;) {
      size_t id;
      {
        std::unique_lock<std::mutex> l(mu);
        cv_work.wait(l, [&] { return !work_q.empty() || done; });
        if (work_q.empty()) return;
        id = work_q.front();
        work_q.pop_front();
      }
      for (size_t j = 0; j < count[id]; j++) {
        ptrdiff_t off;
        size_t len[4];
        block_geometry(p, first[id] + j, &off, len);
        T vals[N];
        reconstruct<T, N>(bufs[id][j], vals);
        scatter<T, D>(vals, data + off, p.s, len);
      }
      {
        std::lock_guard<std::mutex> l(mu);
        free_q.push_back(id);
      }
      cv_free.notify_one();
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < threads - 1; t++) pool.emplace_back(worker);
  for (size_t start = 0; start < p.blocks;) {
    size_t id;
    {
      std::unique_lock<std::mutex> l(mu);
      cv_free.wait(l, [&] { return !free_q.empty(); });
      id = free_q.front();
      free_q.pop_front();
    }
    const size_t n = std::min(batch_len, p.blocks - start);
    for (size_t j = 0; j < n; j++) read_block<T, N>(s, c, bufs[id][j]);
    first[id] = start;
    count[id] = n;
    {
      std::lock_guard<std::mutex> l(mu);
      work_q.push_back(id);
    }
    cv_work.notify_one();
    start += n;
  }
  {
    std::lock_guard<std::mutex> l(mu);
    done = true;
  }
  cv_work.notify_all();
  for (auto& t : pool) t.join();
  return true;
}

template <class T>
static bool pipelined_any_dims(Stream& s, const Plan& p, void* d, const Cfg& c, int threads) {
  switch (p.dims) {
    case 2: return decode_pipelined<T, 2>(s, p, (T*)d, c, threads);
    case 3: return decode_pipelined<T, 3>(s, p, (T*)d, c, threads);
    case 4: return decode_pipelined<T, 4>(s, p, (T*)d, c, threads);
    default: return false;
  }
}
static bool pipelined_any(int type, Stream& s, const Plan& p, void* d, const Cfg& c, int threads) {
  switch (type) {
    case 1: return pipelined_any_dims<int32_t>(s, p, d, c, threads);
    case 2: return pipelined_any_dims<int64_t>(s, p, d, c, threads);
    case 3: return pipelined_any_dims<float>(s, p, d, c, threads);
    default: return pipelined_any_dims<double>(s, p, d, c, threads);
  }
}

// ---------------------------------------------------------------------------
// Config inspectors: src/config.rs:469-686
// ---------------------------------------------------------------------------

static bool valid_params(u32 minb, u32 maxb, u32 maxp) { return minb <= maxb && maxp > 0 && maxp <= 64; }

static int mode_of(const orc_config* c) {
  u32 minb = c->minbits, maxb = c->maxbits, maxp = c->maxprec;
  int32_t mine = c->minexp;
  if (!valid_params(minb, maxb, maxp)) return 0;
  if (minb == ZFP_MIN_BITS && maxb == ZFP_MAX_BITS && maxp == ZFP_MAX_PREC && mine == ZFP_MIN_EXP) return 1;
  if (minb == maxb && maxb >= 1 && maxb <= ZFP_MAX_BITS && maxp >= ZFP_MAX_PREC && mine == ZFP_MIN_EXP) return 2;
  if (minb <= ZFP_MIN_BITS && maxb >= ZFP_MAX_BITS && maxp >= 1 && mine == ZFP_MIN_EXP) return 3;
  if (minb <= ZFP_MIN_BITS && maxb >= ZFP_MAX_BITS && maxp >= ZFP_MAX_PREC && mine >= ZFP_MIN_EXP) return 4;
  if (minb <= ZFP_MIN_BITS && maxb >= ZFP_MAX_BITS && maxp >= ZFP_MAX_PREC && mine < ZFP_MIN_EXP) return 5;
  return 1;
}

static u32 header_bits_of(int type) { return type == 3 ? 9 : type == 4 ? 12 : 0; }

static u32 block_bits_of(const orc_config* c, int type, int dims) {
  u32 values = 1u << (2 * dims);
  u32 header;
  if (c->minexp < ZFP_MIN_EXP)
    header = type == 1 ? 5 : type == 2 ? 6 : type == 3 ? 15 : 19;
  else
    header = header_bits_of(type);
  u32 prec = (type == 1 || type == 3) ? 32 : 64;
  u32 mp = c->maxprec < prec ? c->maxprec : prec;
  u64 most = (u64)header + values - 1 + (u64)values * mp;
  if (most > c->maxbits) most = c->maxbits;
  if (most < header) most = header;
  if (most < c->minbits) most = c->minbits;
  return (u32)most;
}

static u64 encode_expert_mode(u32 minb, u32 maxb, u32 maxp, int32_t mine) {
  auto clampu = [](u32 v, u32 lo, u32 hi) { return v < lo ? lo : v > hi ? hi : v; };
  u64 a = clampu(minb, 1, 0x8000) - 1, b = clampu(maxb, 1, 0x8000) - 1, p = clampu(maxp, 1, 0x80) - 1;
  int64_t e = (int64_t)mine + 16495;
  if (e < 0) e = 0;
  if (e > 0x7fff) e = 0x7fff;
  u64 mode = 0;
  mode = (mode << 15) | (u64)e;
  mode = (mode << 7) | p;
  mode = (mode << 15) | b;
  mode = (mode << 15) | a;
  mode = (mode << 12) | 0xfffu;
  return mode;
}

static u64 mode_bits_of(const orc_config* c) {
  int m = mode_of(c);
  if (m == 2 && c->maxbits <= 2048) return c->maxbits - 1;
  if (m == 3 && c->maxprec <= 128) return (u64)(c->maxprec - 1) + 2048;
  if (m == 5) return 2048 + 128;
  if (m == 4 && c->minexp <= 843) return (u64)(c->minexp - ZFP_MIN_EXP) + (2048 + 128 + 1);
  return encode_expert_mode(c->minbits, c->maxbits, c->maxprec, c->minexp);
}

static Cfg to_cfg(const orc_config* c) {
  Cfg g;
  g.minbits = c->minbits; g.maxbits = c->maxbits; g.maxprec = c->maxprec; g.minexp = c->minexp;
  g.rounding = c->rounding; g.tight = c->tight != 0;
  return g;
}

}  // namespace orc

using namespace orc;

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------

extern "C" {

void* orc_stream_open(uint64_t* words, size_t nwords) {
  Stream* s = new Stream();
  s->words = words;
  s->len = nwords;
  return s;
}
void orc_stream_close(void* s) { delete (Stream*)s; }
void orc_stream_rewind(void* s) {
  Stream* st = (Stream*)s;
  u64* w = st->words;
  size_t l = st->len;
  *st = Stream();
  st->words = w;
  st->len = l;
}
uint64_t orc_stream_wtell(void* s) { return wtell(*(Stream*)s); }
uint64_t orc_stream_rtell(void* s) { return rtell(*(Stream*)s); }
void orc_stream_rseek(void* s, uint64_t o) { seek_read(*(Stream*)s, o); }
void orc_stream_wseek(void* s, uint64_t o) { seek_write(*(Stream*)s, o); }
uint64_t orc_stream_write_bits(void* s, uint64_t v, uint32_t n) { return write_bits(*(Stream*)s, v, n); }
uint64_t orc_stream_read_bits(void* s, uint32_t n) { return read_bits(*(Stream*)s, n); }
uint32_t orc_stream_flush(void* s) { return flush(*(Stream*)s); }
uint32_t orc_stream_align(void* s) { return align(*(Stream*)s); }
size_t orc_stream_size(void* s) { return ((Stream*)s)->word_pos * 8; }

uint32_t orc_block_bits(const orc_config* c, int type, int dims) { return block_bits_of(c, type, dims); }
int orc_mode(const orc_config* c) { return mode_of(c); }
uint64_t orc_mode_bits(const orc_config* c) { return mode_bits_of(c); }

size_t orc_maximum_size(const orc_config* c, const orc_field* f) {
  Plan p;
  if (!make_plan(f, p)) return 0;
  u64 bits = (u64)p.blocks * block_bits_of(c, f->type, p.dims) + 148;
  bits = (bits + 63) / 64 * 64;
  return (size_t)(bits / 8);
}

// compress.rs:22-245
long long orc_compress(void* sp, const orc_field* f, const orc_config* cfg, int threads) {
  Stream& s = *(Stream*)sp;
  Plan p;
  if (!make_plan(f, p) || f->data == nullptr) return -1;
  Cfg c = to_cfg(cfg);
  if (threads <= 1 || p.blocks < 2) {
    enc_any(f->type, s, p, f->data, c, 0, p.blocks);
  } else {
    // execution.rs:119-148 chunk split, compress.rs:164-245 per-chunk streams
    size_t chunks = (size_t)threads < p.blocks ? (size_t)threads : p.blocks;
    std::vector<size_t> start(chunks + 1);
    for (size_t i = 0; i <= chunks; i++) start[i] = (size_t)((unsigned __int128)p.blocks * i / chunks);
    u32 bb = block_bits_of(cfg, f->type, p.dims);
    std::vector<std::vector<u64>> bufs(chunks);
    std::vector<u64> nbits(chunks);
    std::vector<std::thread> pool;
    for (size_t ci = 0; ci < chunks; ci++) {
      pool.emplace_back([&, ci]() {
        size_t nb = start[ci + 1] - start[ci];
        bufs[ci].assign((size_t)((u64)nb * bb / 64 + 1), 0);
        Stream ls;
        ls.words = bufs[ci].data();
        ls.len = bufs[ci].size();
        enc_any(f->type, ls, p, f->data, c, start[ci], start[ci + 1]);
        nbits[ci] = wtell(ls);
        flush(ls);
      });
    }
    for (auto& t : pool) t.join();
    for (size_t ci = 0; ci < chunks; ci++) {  // compress.rs:205-216
      u64 full = nbits[ci] / 64;
      for (u64 i = 0; i < full; i++) write_bits(s, bufs[ci][i], 64);
      u32 rest = (u32)(nbits[ci] % 64);
      if (rest) write_bits(s, bufs[ci][full] & ((1ull << rest) - 1), rest);
    }
  }
  flush(s);  // compress.rs:44-53
  if (s.overflowed) return -1;
  return (long long)(s.word_pos * 8);
}

// decompress.rs:27-330
long long orc_decompress(void* sp, orc_field* f, const orc_config* cfg, int threads) {
  Stream& s = *(Stream*)sp;
  Plan p;
  if (!make_plan(f, p) || f->data == nullptr) return -1;
  Cfg c = to_cfg(cfg);
  bool fixed = mode_of(cfg) == 2 && block_bits_of(cfg, f->type, p.dims) == cfg->maxbits;
  // decompress.rs:165-185: aliasing strides decode serially; fixed-rate
  // streams in seek-parallel chunks, the others through the pipeline.
  const bool shared = !strides_may_alias(p);
  if (threads > 1 && shared && fixed && p.blocks >= 2) {
    u64 start_bit = rtell(s);
    u64 bpb = cfg->maxbits;
    u64 end = start_bit + (u64)p.blocks * bpb;
    size_t chunks = (size_t)threads < p.blocks ? (size_t)threads : p.blocks;
    std::vector<size_t> start(chunks + 1);
    for (size_t i = 0; i <= chunks; i++) start[i] = (size_t)((unsigned __int128)p.blocks * i / chunks);
    std::vector<char> over(chunks, 0);
    std::vector<std::thread> pool;
    for (size_t ci = 0; ci < chunks; ci++) {
      pool.emplace_back([&, ci]() {
        Stream ls;
        ls.words = s.words;
        ls.len = s.len;
        seek_read(ls, start_bit + (u64)start[ci] * bpb);
        dec_any(f->type, ls, p, f->data, c, start[ci], start[ci + 1]);
        over[ci] = overread(ls) ? 1 : 0;
      });
    }
    for (auto& t : pool) t.join();
    bool ov = false;
    for (char o : over) ov |= o != 0;
    // decompress.rs:190-196 (park)
    reset_overread(s);
    seek_read(s, end);
    if (ov) s.overread = true;
  } else {
    reset_overread(s);
    if (!(threads > 1 && shared && mode_of(cfg) != 2 && pipelined_any(f->type, s, p, f->data, c, threads)))
      dec_any(f->type, s, p, f->data, c, 0, p.blocks);
  }
  align(s);  // decompress.rs:66-74
  if (overread(s)) return -1;
  return (long long)(s.word_pos * 8);
}

// header.rs:72-173, field.rs:678-735
size_t orc_write_header(void* sp, const orc_field* f, const orc_config* cfg, unsigned mask) {
  Stream& s = *(Stream*)sp;
  u64 meta = 0;
  if (mask & 2) {
    Plan p;
    if (!make_plan(f, p)) return 0;
    u32 width = 48 / p.dims;
    u64 maxenc = (1ull << width) - 1;
    u32 shift = 0;
    for (int i = 0; i < p.dims; i++) {
      u64 e = (u64)p.n[i] - 1;
      if (e > maxenc) return 0;
      meta |= e << shift;
      shift += width;
    }
    meta = (meta << 2) | (u64)(p.dims - 1);
    meta = (meta << 2) | (u64)(f->type - 1);
  }
  u64 mode = mode_bits_of(cfg);
  u32 msize = mode > (1u << 12) - 2 ? 64 : 12;
  u32 bits = ((mask & 1) ? 32 : 0) + ((mask & 2) ? 52 : 0) + ((mask & 4) ? msize : 0);
  if (wtell(s) + bits > (u64)s.len * 64) return 0;
  if (mask & 1) {
    write_bits(s, 'z', 8); write_bits(s, 'f', 8); write_bits(s, 'p', 8); write_bits(s, 5, 8);
  }
  if (mask & 2) write_bits(s, meta, 52);
  if (mask & 4) write_bits(s, mode, msize);
  return bits;
}

size_t orc_read_header(void* sp, orc_field* f, orc_config* cfg, unsigned mask) {
  Stream& s = *(Stream*)sp;
  size_t bits = 0;
  if (mask & 1) {
    if (read_bits(s, 8) != 'z' || read_bits(s, 8) != 'f' || read_bits(s, 8) != 'p' || read_bits(s, 8) != 5)
      return 0;
    bits += 32;
  }
  if (mask & 2) {
    u64 meta = read_bits(s, 52);
    f->type = (int)(meta & 3) + 1;
    u64 m = meta >> 2;
    int d = (int)(m & 3) + 1;
    m >>= 2;
    u32 width = 48 / d;
    u64 msk = (1ull << width) - 1;
    size_t n[4] = {0, 0, 0, 0};
    for (int i = 0; i < d; i++) { n[i] = (size_t)((m & msk) + 1); m >>= width; }
    f->nx = n[0]; f->ny = n[1]; f->nz = n[2]; f->nw = n[3];
    f->sx = f->sy = f->sz = f->sw = 0;
    bits += 52;
  }
  if (mask & 4) {
    u64 mode = read_bits(s, 12);
    bits += 12;
    if (mode > (1u << 12) - 2) {
      mode |= read_bits(s, 52) << 12;
      bits += 52;
    }
    u32 minb, maxb, maxp;
    int32_t mine;
    if (mode <= (1u << 12) - 2) {
      if (mode < 2048) { minb = maxb = (u32)mode + 1; maxp = 64; mine = -1074; }
      else if (mode < 2048 + 128) { minb = 1; maxb = 16658; maxp = (u32)mode + 1 - 2048; mine = -1074; }
      else if (mode == 2048 + 128) { minb = 1; maxb = 16658; maxp = 64; mine = -1075; }
      else { minb = 1; maxb = 16658; maxp = 64; mine = (int32_t)mode - 1074 - (2048 + 128 + 1); }
    } else {
      u64 m = mode >> 12;
      minb = (u32)(m & 0x7fff) + 1; m >>= 15;
      maxb = (u32)(m & 0x7fff) + 1; m >>= 15;
      maxp = (u32)(m & 0x7f) + 1; m >>= 7;
      mine = (int32_t)(m & 0x7fff) - 16495;
    }
    if (!valid_params(minb, maxb, maxp)) return 0;
    cfg->minbits = minb; cfg->maxbits = maxb; cfg->maxprec = maxp; cfg->minexp = mine;
  }
  return bits;
}

size_t orc_encode_block(void* sp, int type, int dims, const void* data, const ptrdiff_t* st,
                        const size_t* lengths, const orc_config* cfg) {
  Stream& s = *(Stream*)sp;
  size_t full[4] = {4, 4, 4, 4};
  const size_t* len = lengths ? lengths : full;
  Cfg c = to_cfg(cfg);
  u64 before = wtell(s);
#define ORC_ENC(T)                                                      \
  switch (dims) {                                                       \
    case 1: encode_block<T, 1>(s, (const T*)data, st, len, c); break;   \
    case 2: encode_block<T, 2>(s, (const T*)data, st, len, c); break;   \
    case 3: encode_block<T, 3>(s, (const T*)data, st, len, c); break;   \
    default: encode_block<T, 4>(s, (const T*)data, st, len, c); break;  \
  }
  switch (type) {
    case 1: ORC_ENC(int32_t) break;
    case 2: ORC_ENC(int64_t) break;
    case 3: ORC_ENC(float) break;
    default: ORC_ENC(double) break;
  }
#undef ORC_ENC
  return (size_t)(wtell(s) - before);
}

size_t orc_decode_block(void* sp, int type, int dims, void* data, const ptrdiff_t* st,
                        const size_t* lengths, const orc_config* cfg) {
  Stream& s = *(Stream*)sp;
  size_t full[4] = {4, 4, 4, 4};
  const size_t* len = lengths ? lengths : full;
  Cfg c = to_cfg(cfg);
  u64 before = rtell(s);
#define ORC_DEC(T)                                                \
  switch (dims) {                                                 \
    case 1: decode_block<T, 1>(s, (T*)data, st, len, c); break;   \
    case 2: decode_block<T, 2>(s, (T*)data, st, len, c); break;   \
    case 3: decode_block<T, 3>(s, (T*)data, st, len, c); break;   \
    default: decode_block<T, 4>(s, (T*)data, st, len, c); break;  \
  }
  switch (type) {
    case 1: ORC_DEC(int32_t) break;
    case 2: ORC_DEC(int64_t) break;
    case 3: ORC_DEC(float) break;
    default: ORC_DEC(double) break;
  }
#undef ORC_DEC
  return (size_t)(rtell(s) - before);
}

}  // extern "C"
