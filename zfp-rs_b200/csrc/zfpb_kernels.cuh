// Field-level kernels: block tiling (zfp-rs src/field_plan.rs:41-206), the
// gather/scatter of 4^d tiles (encode/dim{1..4}.rs, decode/dim{1..4}.rs), and
// one thread per block driving the block codec of zfpb_block.cuh.
#pragma once

#include <cuda_runtime.h>

#include "zfpb_block.cuh"
#include "zfpb_engine.h"

namespace zfpb {

// Block index -> origin element offset and per-axis lengths (1..4), for
// blocks in row-major order with x fastest (field_plan.rs:128-200).
template <int D>
ZFPB_DEV i64 block_origin(const FieldGeom& f, u64 idx, int* len) {
  i64 off = 0;
  if (D <= 3 && f.nblocks <= 0xffffffffull) {
    // Block coordinates by multiply-high (fields of fewer than 2^32 blocks;
    // 4D fields keep the 64-bit division: the batched int32 4D encoder gave
    // streams that differ from the single-array one's with this path, cause
    // not found).
    u32 r = (u32)idx;
#pragma unroll
    for (int d = 0; d < D; d++) {
      u32 c = r;
      if (d < D - 1) {
        const u32 q = f.inv[d] ? (u32)__umul64hi((u64)r, f.inv[d]) : r;
        c = r - q * (u32)f.b[d];
        r = q;
      }
      const u64 o = 4 * (u64)c;
      off += (i64)o * f.s[d];
      const u64 rest = f.n[d] - o;
      len[d] = rest < 4 ? (int)rest : 4;
    }
    return off;
  }
#pragma unroll
  for (int d = 0; d < D; d++) {
    u64 nb = f.b[d];
    u64 c = (d == D - 1) ? idx : idx % nb;
    idx = (d == D - 1) ? 0 : idx / nb;
    u64 o = 4 * c;
    off += (i64)o * f.s[d];
    u64 r = f.n[d] - o;
    len[d] = r < 4 ? (int)r : 4;
  }
  return off;
}

// Load four values of a row at stride sx; vectorised when the row is a
// 16-byte aligned contiguous run.
template <class T> ZFPB_DEV void load_row(const T* p, i64 sx, bool vec, T* v) {
  if (vec) {
    if constexpr (sizeof(T) == 4) {
      int4 q = __ldg(reinterpret_cast<const int4*>(p));
      v[0] = *reinterpret_cast<const T*>(&q.x);
      v[1] = *reinterpret_cast<const T*>(&q.y);
      v[2] = *reinterpret_cast<const T*>(&q.z);
      v[3] = *reinterpret_cast<const T*>(&q.w);
    } else {
      longlong2 a = __ldg(reinterpret_cast<const longlong2*>(p));
      longlong2 b = __ldg(reinterpret_cast<const longlong2*>(p) + 1);
      v[0] = *reinterpret_cast<const T*>(&a.x);
      v[1] = *reinterpret_cast<const T*>(&a.y);
      v[2] = *reinterpret_cast<const T*>(&b.x);
      v[3] = *reinterpret_cast<const T*>(&b.y);
    }
  } else {
#pragma unroll
    for (int x = 0; x < 4; x++) v[x] = __ldg(p + x * sx);
  }
}

template <class T> ZFPB_DEV void store_row(T* p, i64 sx, bool vec, const T* v) {
  if (vec) {
    if constexpr (sizeof(T) == 4) {
      int4 q;
      q.x = *reinterpret_cast<const int*>(&v[0]);
      q.y = *reinterpret_cast<const int*>(&v[1]);
      q.z = *reinterpret_cast<const int*>(&v[2]);
      q.w = *reinterpret_cast<const int*>(&v[3]);
      *reinterpret_cast<int4*>(p) = q;
    } else {
      longlong2 a, b;
      a.x = *reinterpret_cast<const long long*>(&v[0]);
      a.y = *reinterpret_cast<const long long*>(&v[1]);
      b.x = *reinterpret_cast<const long long*>(&v[2]);
      b.y = *reinterpret_cast<const long long*>(&v[3]);
      reinterpret_cast<longlong2*>(p)[0] = a;
      reinterpret_cast<longlong2*>(p)[1] = b;
    }
  } else {
#pragma unroll
    for (int x = 0; x < 4; x++) p[x * sx] = v[x];
  }
}

// Gather a (possibly partial) block with C pad_block padding
// (encode/dim3.rs:44-78, encode/core.rs:194-219): x within filled rows, then
// y, then z, then w; a padded entry copies entry 0, 1, 0 of its run for
// positions 1, 2, 3.
template <class T, int D>
ZFPB_DEV void gather_block(const T* base, const FieldGeom& f, i64 off, const int* len, T* b) {
  constexpr int N = 1 << (2 * D);
  const T* p = base + off;
  bool full = true;
#pragma unroll
  for (int d = 0; d < D; d++) full = full && len[d] == 4;
  if (full) {
    const bool vec = f.vec_ok != 0;
#pragma unroll
    for (int r = 0; r < N / 4; r++) {
      i64 o = 0;
      if (D > 1) o += (i64)(r & 3) * f.s[1];
      if (D > 2) o += (i64)((r >> 2) & 3) * f.s[2];
      if (D > 3) o += (i64)(r >> 4) * f.s[3];
      load_row<T>(p + o, f.s[0], vec, b + 4 * r);
    }
    return;
  }
  const int nx = len[0], ny = D > 1 ? len[1] : 1, nz = D > 2 ? len[2] : 1, nw = D > 3 ? len[3] : 1;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const int x = i & 3, y = (i >> 2) & 3, z = (i >> 4) & 3, w = i >> 6;
    T v = 0;
    if (x < nx && y < ny && z < nz && w < nw) {
      i64 o = (i64)x * f.s[0];
      if (D > 1) o += (i64)y * f.s[1];
      if (D > 2) o += (i64)z * f.s[2];
      if (D > 3) o += (i64)w * f.s[3];
      v = __ldg(p + o);
    }
    b[i] = v;
  }
  // x within rows
#pragma unroll
  for (int r = 0; r < N / 4; r++) {
    T* q = b + 4 * r;
    if (nx <= 1) q[1] = q[0];
    if (nx <= 2) q[2] = q[1];
    if (nx <= 3) q[3] = q[0];
  }
  if constexpr (D >= 2) {
#pragma unroll
    for (int g = 0; g < N / 16; g++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        T* q = b + 16 * g + x;
        if (ny <= 1) q[4] = q[0];
        if (ny <= 2) q[8] = q[4];
        if (ny <= 3) q[12] = q[0];
      }
  }
  if constexpr (D >= 3) {
#pragma unroll
    for (int g = 0; g < N / 64; g++)
#pragma unroll
      for (int x = 0; x < 16; x++) {
        T* q = b + 64 * g + x;
        if (nz <= 1) q[16] = q[0];
        if (nz <= 2) q[32] = q[16];
        if (nz <= 3) q[48] = q[0];
      }
  }
  if constexpr (D >= 4) {
#pragma unroll
    for (int x = 0; x < 64; x++) {
      T* q = b + x;
      if (nw <= 1) q[64] = q[0];
      if (nw <= 2) q[128] = q[64];
      if (nw <= 3) q[192] = q[0];
    }
  }
}

// Store the in-field part of a block (decode/dim3.rs:221-260).  With an
// owner map, an element is stored only by the block that owns it.
template <class T, int D>
ZFPB_DEV void scatter_block(T* base, const FieldGeom& f, i64 off, const int* len, const T* b,
                            const u64* owner = nullptr, i64 imin = 0, u64 blk = 0) {
  constexpr int N = 1 << (2 * D);
  T* p = base + off;
  bool full = true;
#pragma unroll
  for (int d = 0; d < D; d++) full = full && len[d] == 4;
  if (owner) {
    const int nx = len[0], ny = D > 1 ? len[1] : 1, nz = D > 2 ? len[2] : 1, nw = D > 3 ? len[3] : 1;
#pragma unroll
    for (int i = 0; i < N; i++) {
      const int x = i & 3, y = (i >> 2) & 3, z = (i >> 4) & 3, w = i >> 6;
      if (x < nx && y < ny && z < nz && w < nw) {
        i64 o = (i64)x * f.s[0];
        if (D > 1) o += (i64)y * f.s[1];
        if (D > 2) o += (i64)z * f.s[2];
        if (D > 3) o += (i64)w * f.s[3];
        if (owner[off + o - imin] == blk + 1) p[o] = b[i];
      }
    }
    return;
  }
  if (full) {
    const bool vec = f.vec_ok != 0;
#pragma unroll
    for (int r = 0; r < N / 4; r++) {
      i64 o = 0;
      if (D > 1) o += (i64)(r & 3) * f.s[1];
      if (D > 2) o += (i64)((r >> 2) & 3) * f.s[2];
      if (D > 3) o += (i64)(r >> 4) * f.s[3];
      store_row<T>(p + o, f.s[0], vec, b + 4 * r);
    }
    return;
  }
  const int nx = len[0], ny = D > 1 ? len[1] : 1, nz = D > 2 ? len[2] : 1, nw = D > 3 ? len[3] : 1;
#pragma unroll
  for (int i = 0; i < N; i++) {
    const int x = i & 3, y = (i >> 2) & 3, z = (i >> 4) & 3, w = i >> 6;
    if (x < nx && y < ny && z < nz && w < nw) {
      i64 o = (i64)x * f.s[0];
      if (D > 1) o += (i64)y * f.s[1];
      if (D > 2) o += (i64)z * f.s[2];
      if (D > 3) o += (i64)w * f.s[3];
      p[o] = b[i];
    }
  }
}

template <class T, int D> struct KernelShape {
  static constexpr int N = 1 << (2 * D);
  static constexpr int W = N <= 64 ? 1 : N / 64;
  static constexpr int PREC = Traits<T>::PREC;
  // Shared-memory words of plane storage per thread (none for 4-value
  // blocks, whose planes stay in registers).
  static constexpr int PLANE_WORDS = D == 1 ? 0 : PREC * W;
  // CTAs of 128 threads per SM the register allocation must allow: 4 caps
  // 32-bit blocks at 128 registers (16 warps per SM), 3 caps 64-bit ones at
  // 168.  Occupancy hides the latency of the sequential bit-plane coding.
  static constexpr int MIN_CTAS = sizeof(T) == 4 ? 4 : 3;
  // The value half of the split 3D decoder holds a block's 64 values and its
  // transposed planes at once: 64-bit blocks run 2 CTAs per SM (255
  // registers, no spills), measured faster than 3 (168 registers and 740
  // bytes of spills per thread): 512^3 float64 k_finish 0.727 -> 0.660 ms
  // (fixed-accuracy), 0.598 -> 0.538 ms (fixed-precision 32).
  static constexpr int FINISH_CTAS = sizeof(T) == 4 ? 4 : 2;
  // Batch kernels of 1D and 2D blocks: a batch kernel also holds its tile's
  // item (geometry, codec parameters, buffers) and loops over the tile's
  // blocks, and left to itself the compiler gives it far more registers than
  // the single-array kernel of the same codec (1D float encode 63 instead of
  // 31, 2D float decode 112 instead of 63), halving the warps per SM.  These
  // bounds hold them to the single-array kernels' budgets.
  static constexpr int BATCH_ENC_CTAS = D == 1 ? 12 : D == 2 && sizeof(T) == 4 ? 5 : MIN_CTAS;
  static constexpr int BATCH_DEC_CTAS = D == 1 ? 8 : D == 2 ? (sizeof(T) == 4 ? 8 : 4) : MIN_CTAS;
};

// ---------------------------------------------------------------------------
// Coding order inside a CTA.  The plane loop of a block runs one iteration per
// plane until the last coefficient turns significant, a count that differs
// from block to block (zero blocks: none; blocks with a spike: many), and a
// warp runs as long as its longest block.  Lossy float blocks of 16 and 64
// values are therefore prepared by their own thread (planes into the plane
// store), ordered by that count across the CTA, and coded in that order, so
// that the threads of a warp run loops of similar length.
// ---------------------------------------------------------------------------
template <class T, int D> struct SortedCoder {
  static constexpr bool value = Traits<T>::FLOAT && (D == 2 || D == 3);
};

// Counting sort of the CTA's keys (clamped to 0..63; at most 256 threads,
// every thread calls): returns the CTA-local index of the block this thread
// codes.  Ends with a barrier.
ZFPB_DEV int order_by_key(u32 key, u32* cnt, unsigned char* order) {
  const int tid = threadIdx.x;
  for (int i = tid; i < 64; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  key = key < 63 ? key : 63;
  const u32 rank = atomicAdd(&cnt[key], 1u);
  __syncthreads();
  if (tid < 32) {
    const u32 c0 = cnt[2 * tid], c1 = cnt[2 * tid + 1];
    u32 sum = c0 + c1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 v = __shfl_up_sync(0xffffffffu, sum, o);
      if (tid >= o) sum += v;
    }
    const u32 ex = sum - c0 - c1;
    cnt[2 * tid] = ex;
    cnt[2 * tid + 1] = ex + c0;
  }
  __syncthreads();
  order[cnt[key] + rank] = (unsigned char)tid;
  __syncthreads();
  return order[tid];
}

// Shared memory of the sorted coder (CTAs of at most 128 threads).
struct SortSmem {
  BlockPrep prep[128];
  u32 cnt[64];
  unsigned char order[128];
};

// Gather and prepare block `blk` (if in the field) into the plane store column
// of this thread; returns its record.
template <class T, int D>
ZFPB_DEV BlockPrep prep_field_block(const void* data, const FieldGeom& f, const Codec& c, u64 blk, PlaneStore ps) {
  BlockPrep p{0u, 0u, 0u, 0u};
  if (blk < f.nblocks) {
    int len[4];
    const i64 off = block_origin<D>(f, blk, len);
    T b[KernelShape<T, D>::N];
    gather_block<T, D>(static_cast<const T*>(data), f, off, len, b);
    p = prep_float_block<T, KernelShape<T, D>::N>(b, c, ps);
  }
  return p;
}

// ---------------------------------------------------------------------------
// Fixed-size blocks (every block exactly maxbits bits): stage a CTA's bits in
// shared memory, then store the stream words the CTA owns.  CTA j codes blocks
// [jB, jB + B + X): the X extra blocks are the next CTA's first ones, which
// complete the last word this CTA owns.  A CTA owns the words whose first bit
// lies in its own bit range; CTA 0 also owns the word holding the start bit,
// into which it merges the bits already in the stream.
// ---------------------------------------------------------------------------
// LOSSY (lossy float 2D/3D fields): the sorted coder only.
template <class T, int D, bool LOSSY>
__global__ void __launch_bounds__(128, KernelShape<T, D>::MIN_CTAS) k_encode_fixed(EncodeFixedArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  PlaneStore ps{smem + tid, nthr};
  u64* stage = smem + (size_t)S::PLANE_WORDS * nthr;
  const u64 maxbits = a.c.maxbits;
  const u64 first = (u64)blockIdx.x * a.blocks_per_cta;
  const u64 g0 = a.start + first * maxbits;
  const u64 w0 = g0 >> 6;
  const u32 lb = (u32)(g0 & 63);
  const u32 stage_words = (u32)((lb + (u64)nthr * maxbits + 63) >> 6) + 1;
  for (u32 i = tid; i < stage_words; i += nthr) stage[i] = 0;
  __syncthreads();

  const u64 blk = first + tid;
  if constexpr (LOSSY) {
    static_assert(SortedCoder<T, D>::value, "lossy kernels are for float 2D/3D fields");
    __shared__ SortSmem ss;
    const BlockPrep p = prep_field_block<T, D>(a.data, a.f, a.c, blk, ps);
    ss.prep[tid] = p;
    const int j = order_by_key(p.key, ss.cnt, ss.order);
    if (first + j < a.f.nblocks) {
      Writer<true> w;
      w.init(stage, lb + (u64)j * maxbits, stage_words);
      code_float_block<T, S::N>(w, ss.prep[j], a.c, PlaneStore{smem + j, nthr});
      w.finish();
    }
  } else if (blk < a.f.nblocks) {
    int len[4];
    i64 off = block_origin<D>(a.f, blk, len);
    T b[S::N];
    gather_block<T, D>(static_cast<const T*>(a.data), a.f, off, len, b);
    Writer<true> w;
    w.init(stage, lb + (u64)tid * maxbits, stage_words);
    encode_block<T, S::N>(w, b, a.c, ps);
    w.finish();
  }
  __syncthreads();

  const u64 nb = a.f.nblocks - first < a.blocks_per_cta ? a.f.nblocks - first : a.blocks_per_cta;
  u64 lo = (g0 + 63) >> 6;
  const u64 hi = (g0 + nb * maxbits + 63) >> 6;
  if (blockIdx.x == 0 && lb != 0) lo = w0;
  for (u64 wi = lo + tid; wi < hi; wi += nthr) {
    u64 v = stage[wi - w0];
    if (blockIdx.x == 0 && wi == w0) v |= a.init_word;
    a.out[wi] = v;
  }
}

// ---------------------------------------------------------------------------
// Variable-size blocks, pass 1: each block coded into its own slot of the
// scratch buffer (slot i at word i * slot_words), its bit length recorded.
// ---------------------------------------------------------------------------
template <class T, int D, bool LOSSY>
__global__ void __launch_bounds__(128, KernelShape<T, D>::MIN_CTAS) k_encode_var(EncodeVarArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  const int tid = threadIdx.x;
  PlaneStore ps{smem + tid, (int)blockDim.x};
  const u64 base = (u64)blockIdx.x * blockDim.x;
  const u64 blk = base + tid;
  if constexpr (LOSSY) {
    static_assert(SortedCoder<T, D>::value, "lossy kernels are for float 2D/3D fields");
    __shared__ SortSmem ss;
    const BlockPrep p = prep_field_block<T, D>(a.data, a.f, a.c, blk, ps);
    ss.prep[tid] = p;
    const int j = order_by_key(p.key, ss.cnt, ss.order);
    const u64 bj = base + j;
    if (bj < a.f.nblocks) {
      Writer<false> w;
      w.init(a.slots + bj * a.slot_words, 0, a.slot_words);
      const u32 bits = code_float_block<T, S::N>(w, ss.prep[j], a.c, PlaneStore{smem + j, (int)blockDim.x});
      w.finish();
      a.lengths[bj] = bits;
    }
    return;
  }
  if (blk >= a.f.nblocks) return;
  int len[4];
  i64 off = block_origin<D>(a.f, blk, len);
  T b[S::N];
  gather_block<T, D>(static_cast<const T*>(a.data), a.f, off, len, b);
  Writer<false> w;
  w.init(a.slots + blk * a.slot_words, 0, a.slot_words);
  u32 bits = encode_block<T, S::N>(w, b, a.c, ps);
  w.finish();
  a.lengths[blk] = bits;
}

// Truncation rule (zfp-rs decompress.rs:57-74, bitstream/core.rs:377-404): a
// stream is truncated when decoding loaded a word past its end: a word holding
// a bit that was read, or the word a skip to a block's padded end landed in
// (when not at a word boundary).
ZFPB_DEV void check_loads(u64 start, u32 read_bits, u32 occupied, u64 len, unsigned* flags) {
  u64 last = 0;
  bool any = false;
  if (read_bits > 0) {
    last = (start + read_bits - 1) >> 6;
    any = true;
  }
  u64 end = start + occupied;
  if (occupied > read_bits && (end & 63) != 0) {
    u64 wv = end >> 6;
    last = any && last > wv ? last : wv;
    any = true;
  }
  if (any && last >= len) atomicOr(flags, FLAG_TRUNCATED);
}

// Fixed-size blocks: block i starts at start + i * maxbits (decompress.rs:205-330).
template <class T, int D, bool LOSSY>
__global__ void __launch_bounds__(128, KernelShape<T, D>::MIN_CTAS) k_decode_fixed(DecodeArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  const int tid = threadIdx.x;
  PlaneStore ps{smem + tid, (int)blockDim.x};
  const u64 blk = (u64)blockIdx.x * blockDim.x + tid;
  if (blk >= a.f.nblocks) return;
  const u64 pos = a.start + blk * (u64)a.c.maxbits;
  Reader r;
  r.init(a.stream, a.stream_len, pos);
  T b[S::N];
  u32 rb;
  u32 occ = decode_block<T, S::N, LOSSY>(r, b, a.c, ps, &rb);
  check_loads(pos, rb, occ, a.stream_len, a.flags);
  int len[4];
  i64 off = block_origin<D>(a.f, blk, len);
  scatter_block<T, D>(static_cast<T*>(a.data), a.f, off, len, b, a.owner, a.imin, blk);
}

// Variable-size blocks with known offsets: decode each block from its offset
// and check that it ends where the next begins, which makes the offsets
// exactly those of a serial decode (else FLAG_BAD_INDEX).
template <class T, int D, bool LOSSY>
__global__ void __launch_bounds__(128, KernelShape<T, D>::MIN_CTAS) k_decode_var(DecodeArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  const int tid = threadIdx.x;
  PlaneStore ps{smem + tid, (int)blockDim.x};
  const u64 blk = (u64)blockIdx.x * blockDim.x + tid;
  if (blk >= a.f.nblocks) return;
  const u64 o0 = a.offsets[blk], o1 = a.offsets[blk + 1];
  const u64 pos = a.start + o0;
  Reader r;
  r.init(a.stream, a.stream_len, pos);
  T b[S::N];
  u32 rb;
  u32 occ = decode_block<T, S::N, LOSSY>(r, b, a.c, ps, &rb);
  if (o1 < o0 || (u64)occ != o1 - o0) {
    atomicOr(a.flags, FLAG_BAD_INDEX);
    return;
  }
  check_loads(pos, rb, occ, a.stream_len, a.flags);
  int len[4];
  i64 off = block_origin<D>(a.f, blk, len);
  scatter_block<T, D>(static_cast<T*>(a.data), a.f, off, len, b, a.owner, a.imin, blk);
}

// Two-kernel decoder for 4^3 blocks.  k_parse reads each block's bits: its
// head goes to heads[i] and its bit planes to a plane-major scratch (plane k
// of block i at planes[k * stride + i], so a warp's stores coalesce).  It
// holds no values and no shared memory, so far more blocks are in flight than
// in k_decode_*, whose plane store and value registers bound their occupancy.
// k_finish rebuilds the values and scatters them.
template <class T, int D, bool VAR, bool LOSSY>
__global__ void __launch_bounds__(128, 8) k_parse(DecodeArgs a, SplitArgs sa) {
  typedef KernelShape<T, D> S;
  const u64 blk = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= a.f.nblocks) return;
  u64 o0 = 0, o1 = 0, pos;
  if (VAR) {
    o0 = a.offsets[blk];
    o1 = a.offsets[blk + 1];
    pos = a.start + o0;
  } else {
    pos = a.start + blk * (u64)a.c.maxbits;
  }
  Reader r;
  r.init(a.stream, a.stream_len, pos);
  PlaneStore ps{sa.planes + blk, (int)sa.stride};
  BlockHead h;
  u32 rb;
  u32 occ = parse_block<T, S::N, LOSSY>(r, a.c, ps, h, &rb);
  if (VAR && (o1 < o0 || (u64)occ != o1 - o0)) {
    atomicOr(a.flags, FLAG_BAD_INDEX);
    return;
  }
  check_loads(pos, rb, occ, a.stream_len, a.flags);
  sa.heads[blk] = h.pack();
}

template <class T, int D, bool LOSSY>
__global__ void __launch_bounds__(128, KernelShape<T, D>::FINISH_CTAS) k_finish(DecodeArgs a, SplitArgs sa) {
  typedef KernelShape<T, D> S;
  const u64 blk = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= a.f.nblocks || (*(volatile unsigned*)a.flags & FLAG_BAD_INDEX)) return;
  PlaneStore ps{sa.planes + blk, (int)sa.stride};
  const BlockHead h = BlockHead::unpack(sa.heads[blk]);
  T b[S::N];
  finish_block<T, S::N, LOSSY>(h, b, ps);
  int len[4];
  i64 off = block_origin<D>(a.f, blk, len);
  scatter_block<T, D>(static_cast<T*>(a.data), a.f, off, len, b, a.owner, a.imin, blk);
}

// Offsets of a stream without an index: one thread decodes block after block,
// as the serial reader does (decompress/pipeline.rs:139-171), recording where
// each starts.  offsets[i] is relative to the start bit; offsets[n] is the end.
template <class T, int D>
__global__ void __launch_bounds__(32) k_walk(DecodeArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  if (threadIdx.x != 0) return;
  PlaneStore ps{smem, 1};
  u64 rel = 0;
  for (u64 blk = 0; blk < a.f.nblocks; blk++) {
    a.offsets[blk] = rel;
    Reader r;
    r.init(a.stream, a.stream_len, a.start + rel);
    if constexpr (S::N <= 64) {
      rel += block_length<T, S::N>(r, a.c);
    } else {
      BlockHead h;
      u32 rb;
      rel += parse_block<T, S::N>(r, a.c, ps, h, &rb);
    }
  }
  a.offsets[a.f.nblocks] = rel;
}

// ---------------------------------------------------------------------------
// Speculative parallel walk.  A zfp stream has no block markers, but a walk
// begun at a wrong bit reads some garbage blocks (most one or a few bits
// long) and then lands on a true block start, after which it follows the
// true walk (measured on smooth fields: a median of 60 steps for 1D, 950 for
// 3D f64, never more than 7000).  So the stream is cut into segments; for
// each, one thread walks from `lead` bits before its first bit and lists the
// positions it visits inside the segment (k_spec_walk).  Then one fix pass
// (k_spec_fix): for each segment s >= 1, a walk from the exit of segment
// s - 1's list runs until it meets a position listed by s or by a later
// segment, recording the positions before it.  Segment 0's list is exact (it
// starts at the true start), so the true walk is segment 0's list, segment
// 1's fix, the tail of the list it joined (whose exit is exact), the fix of
// the segment after that one, and so on: a short chain the host follows
// before k_spec_write places the pieces.  Each walker has a warp to itself:
// walkers sharing a warp diverge on every block and run several times
// slower.
// ---------------------------------------------------------------------------

// The bits of the block at x.  4-D blocks (256 values) are measured by the
// stream half of the decoder, as the serial walk does, with a one-thread
// plane store in the CTA's dynamic shared memory (one walker per CTA).
template <class T, int D> ZFPB_DEV u64 spec_len(const SpecWalkArgs& a, u64 x) {
  Reader r;
  r.init(a.stream, a.stream_len, a.start + x);
  if constexpr (KernelShape<T, D>::N <= 64) {
    return block_length<T, KernelShape<T, D>::N>(r, a.c);
  } else {
    extern __shared__ u64 smem[];
    PlaneStore ps{smem, 1};
    BlockHead h;
    u32 rb;
    return parse_block<T, KernelShape<T, D>::N>(r, a.c, ps, h, &rb);
  }
}

ZFPB_DEV u64 seg_hi(const SpecWalkArgs& a, u64 sg) {
  const u64 hi = (sg + 1) * a.seg_bits;
  return hi < a.end_bits ? hi : a.end_bits;
}

template <class T, int D> __global__ void __launch_bounds__(32) k_spec_walk(SpecWalkArgs a) {
  const u64 sg = blockIdx.x;
  if (threadIdx.x != 0 || sg >= a.nseg) return;
  const u64 lo = sg * a.seg_bits, hi = seg_hi(a, sg);
  u32* list = a.list + sg * a.cap;
  u64 x = sg == 0 ? 0 : (lo > a.lead ? lo - a.lead : 0), k = 0;
  for (u64 steps = 0; x < lo && steps < a.cap; steps++) x += spec_len<T, D>(a, x);  // lead-in, not listed
  if (x < lo) x = lo;  // a lead-in that did not arrive: start at the segment
  while (x < hi) {
    if (k == a.cap) break;  // overflow: the caller walks serially
    list[k++] = (u32)(x - lo);
    x += spec_len<T, D>(a, x);
  }
  if (x < hi) atomicOr(a.flags, 1u);
  a.list_len[sg] = (u32)k;
  a.exit_spec[sg] = x;
}

template <class T, int D> __global__ void __launch_bounds__(32) k_spec_fix(SpecWalkArgs a) {
  const u64 sg = blockIdx.x;
  if (threadIdx.x != 0 || sg >= a.nseg) return;
  if (sg == 0) {  // exact: no fix, joins its own list at 0
    a.fix_len[0] = 0;
    a.sync_t[0] = 0;
    a.sync_j[0] = 0;
    a.fix_exit[0] = 0;
    return;
  }
  const u64 lo = sg * a.seg_bits;
  u32* fix = a.fix + sg * a.cap;
  u64 x = a.exit_spec[sg - 1], k = 0;
  u64 t = x / a.seg_bits;  // the segment x lies in
  u32 j = 0;
  bool joined = false;
  while (x < a.end_bits) {
    const u64 xt = x / a.seg_bits;
    if (xt != t) {
      t = xt;
      j = 0;
    }
    const u32* list = a.list + t * a.cap;
    const u32 len = a.list_len[t], rx = (u32)(x - t * a.seg_bits);
    while (j < len && list[j] < rx) j++;
    if (j < len && list[j] == rx) {
      joined = true;
      break;
    }
    // Overflow (a full fix list, or a position past 2^32 bits from the
    // segment's start, which the u32 entries cannot hold): the caller walks
    // serially.
    if (k == a.cap || x - lo > 0xffffffffull) {
      atomicOr(a.flags, 1u);
      break;
    }
    fix[k++] = (u32)(x - lo);
    x += spec_len<T, D>(a, x);
  }
  a.fix_len[sg] = (u32)k;
  a.sync_t[sg] = joined ? (u32)t : (u32)a.nseg;
  a.sync_j[sg] = joined ? j : 0u;
  a.fix_exit[sg] = x;
}

// Blocks idx .. n - 1 of the walk from x (past the segments: a stream cut
// short, or blocks read past its last word), and off[n].
template <class T, int D> __global__ void k_spec_tail(SpecWalkArgs a, u64* off, u64 idx, u64 n, u64 x) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (; idx < n; idx++) {
    off[idx] = x;
    x += spec_len<T, D>(a, x);
  }
  off[n] = x;
}

// ---------------------------------------------------------------------------
// Batches: one CTA per tile (up to 128 consecutive blocks of one array, which
// the CTA's threads take in turn), the arrays of one (type, dims) class in one
// launch.  The per-block work is that of the
// single-array kernels above, with the array's geometry, codec parameters and
// buffers read from its BatchItem.
// ---------------------------------------------------------------------------

template <class T, int D>
__global__ void __launch_bounds__(128, KernelShape<T, D>::BATCH_ENC_CTAS) k_encode_batch(BatchArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  const BatchTile t = a.tiles[blockIdx.x];
  const int tid = threadIdx.x;
  const BatchItem* it = a.items + t.item;
  PlaneStore ps{smem + tid, (int)blockDim.x};
  const CodecParams c = it->c;
  const u64 sw = it->slot_words;
  u32* lens = a.lengths + it->len_base;
  if constexpr (SortedCoder<T, D>::value) {
    // One block per thread: prepared, ordered across the CTA, then coded.
    if (c.minexp >= ZFP_MIN_EXP && t.count <= blockDim.x) {
      __shared__ SortSmem ss;
      const BlockPrep p = prep_field_block<T, D>(it->data, it->f, c, tid < t.count ? t.first + tid : ~0ull, ps);
      ss.prep[tid] = p;
      const int j = order_by_key(p.key, ss.cnt, ss.order);
      if ((u32)j < t.count) {
        const u64 blk = t.first + j;
        Writer<false> w;
        w.init(a.slots + it->slot_base + blk * sw, 0, sw);
        lens[blk] = code_float_block<T, S::N>(w, ss.prep[j], c, PlaneStore{smem + j, (int)blockDim.x});
        w.finish();
        if (blk + 1 == it->f.nblocks) lens[blk + 1] = 0;
      }
      return;
    }
  }
  for (u32 j = tid; j < t.count; j += blockDim.x) {
    const u64 blk = t.first + j;
    int len[4];
    i64 off = block_origin<D>(it->f, blk, len);
    T b[S::N];
    gather_block<T, D>(static_cast<const T*>(it->data), it->f, off, len, b);
    Writer<false> w;
    w.init(a.slots + it->slot_base + blk * sw, 0, sw);
    u32 bits = encode_block<T, S::N>(w, b, c, ps);
    w.finish();
    lens[blk] = bits;
    if (blk + 1 == it->f.nblocks) lens[blk + 1] = 0;
  }
}

// Where block `blk` of an item starts, and where the next one starts (from the
// item's index, the walker's offsets, or i * maxbits).
ZFPB_DEV const u64* batch_offsets(const BatchArgs& a, const BatchItem* it) {
  return it->walk ? a.offsets + it->len_base : it->index;
}

template <class T, int D>
__global__ void __launch_bounds__(128, KernelShape<T, D>::BATCH_DEC_CTAS) k_decode_batch(BatchArgs a) {
  typedef KernelShape<T, D> S;
  extern __shared__ u64 smem[];
  const BatchTile t = a.tiles[blockIdx.x];
  const int tid = threadIdx.x;
  const BatchItem* it = a.items + t.item;
  PlaneStore ps{smem + tid, (int)blockDim.x};
  const CodecParams c = it->c;
  const u64* offs = batch_offsets(a, it);
  for (u32 j = tid; j < t.count; j += blockDim.x) {
    const u64 blk = t.first + j;
    u64 o0, o1;
    if (it->fixed) {
      o0 = it->start + blk * (u64)c.maxbits;
      o1 = o0 + c.maxbits;
    } else {
      o0 = it->start + offs[blk];
      o1 = it->start + offs[blk + 1];
    }
    Reader r;
    r.init(it->stream, it->stream_words, o0);
    T b[S::N];
    u32 rb;
    u32 occ = decode_block<T, S::N>(r, b, c, ps, &rb);
    if (o1 < o0 || (u64)occ != o1 - o0) {
      atomicOr(a.flags + t.item, FLAG_BAD_INDEX);
      continue;
    }
    check_loads(o0, rb, occ, it->stream_words, a.flags + t.item);
    int len[4];
    i64 off = block_origin<D>(it->f, blk, len);
    scatter_block<T, D>(static_cast<T*>(it->data), it->f, off, len, b, nullptr, 0, blk);
  }
}

template <class T>
__global__ void __launch_bounds__(128, 8) k_parse_batch(BatchArgs a) {
  const BatchTile t = a.tiles[blockIdx.x];
  const BatchItem* it = a.items + t.item;
  const CodecParams c = it->c;
  const u64* offs = batch_offsets(a, it);
  for (u32 j = threadIdx.x; j < t.count; j += blockDim.x) {
    const u64 blk = t.first + j;
    u64 o0, o1;
    if (it->fixed) {
      o0 = it->start + blk * (u64)c.maxbits;
      o1 = o0 + c.maxbits;
    } else {
      o0 = it->start + offs[blk];
      o1 = it->start + offs[blk + 1];
    }
    Reader r;
    r.init(it->stream, it->stream_words, o0);
    const u64 col = it->plane_base + blk;
    PlaneStore ps{a.planes + col, (int)a.plane_stride};
    BlockHead h;
    u32 rb;
    u32 occ = parse_block<T, 64>(r, c, ps, h, &rb);
    if (o1 < o0 || (u64)occ != o1 - o0) {
      atomicOr(a.flags + t.item, FLAG_BAD_INDEX);
      continue;
    }
    check_loads(o0, rb, occ, it->stream_words, a.flags + t.item);
    a.heads[col] = h.pack();
  }
}

template <class T>
__global__ void __launch_bounds__(128, KernelShape<T, 3>::FINISH_CTAS) k_finish_batch(BatchArgs a) {
  const BatchTile t = a.tiles[blockIdx.x];
  if (*(volatile unsigned*)(a.flags + t.item) & FLAG_BAD_INDEX) return;
  const BatchItem* it = a.items + t.item;
  for (u32 j = threadIdx.x; j < t.count; j += blockDim.x) {
    const u64 blk = t.first + j;
    const u64 col = it->plane_base + blk;
    PlaneStore ps{a.planes + col, (int)a.plane_stride};
    const BlockHead h = BlockHead::unpack(a.heads[col]);
    T b[64];
    finish_block<T, 64>(h, b, ps);
    int len[4];
    i64 off = block_origin<3>(it->f, blk, len);
    scatter_block<T, 3>(static_cast<T*>(it->data), it->f, off, len, b, nullptr, 0, blk);
  }
}

// Offsets of the items listed in walk_items: one thread per item walks its
// stream block by block (the stream half of the decode only).
template <class T, int D>
__global__ void __launch_bounds__(64) k_walk_batch(BatchArgs a) {
  typedef KernelShape<T, D> S;
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nwalk) return;
  const BatchItem* it = a.items + a.walk_items[i];
  PlaneStore ps{a.walk_planes + i, (int)a.nwalk};
  const CodecParams c = it->c;
  u64* off = a.offsets + it->len_base;
  u64 rel = 0;
  const u64 n = it->f.nblocks;
  for (u64 blk = 0; blk < n; blk++) {
    off[blk] = rel;
    Reader r;
    r.init(it->stream, it->stream_words, it->start + rel);
    if constexpr (S::N <= 64) {
      rel += block_length<T, S::N>(r, c);
    } else {
      BlockHead h;
      u32 rb;
      rel += parse_block<T, S::N>(r, c, ps, h, &rb);
    }
  }
  off[n] = rel;
}

// Owner map for fields whose strides may alias: every element records the
// last block, in stream order, that holds it.
template <int D> __global__ void k_claim(FieldGeom f, u64* owner, i64 imin) {
  const u64 blk = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= f.nblocks) return;
  int len[4];
  i64 off = block_origin<D>(f, blk, len);
  const int nx = len[0], ny = D > 1 ? len[1] : 1, nz = D > 2 ? len[2] : 1, nw = D > 3 ? len[3] : 1;
  for (int w = 0; w < nw; w++)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          i64 o = (i64)x * f.s[0];
          if (D > 1) o += (i64)y * f.s[1];
          if (D > 2) o += (i64)z * f.s[2];
          if (D > 3) o += (i64)w * f.s[3];
          atomicMax(owner + (off + o - imin), blk + 1);
        }
}

}  // namespace zfpb
