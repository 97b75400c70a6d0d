// Orchestration of a compress or decompress call on the device: choice of the
// fixed-size or variable-size path, the device-wide scan of block bit lengths,
// the bit-exact concatenation of variable-size blocks, and the device
// workspace.  The stream layout follows zfp-rs src/compress.rs and
// src/decompress.rs.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <vector>

#include "zfpb_engine.h"
#include "zfpb_kernels.cuh"

namespace zfpb {

// ---------------------------------------------------------------------------
// Block budgets (zfp-rs src/config.rs:670-686)
// ---------------------------------------------------------------------------

u32 block_bits(const CodecParams& c, int type, int dims) {
  u32 values = 1u << (2 * dims);
  u32 header;
  if (c.minexp < ZFP_MIN_EXP)
    header = type == 1 ? 5 : type == 2 ? 6 : type == 3 ? 15 : 19;
  else
    header = type == 3 ? 9 : type == 4 ? 12 : 0;
  u32 prec = (type == 1 || type == 3) ? 32 : 64;
  u32 mp = c.maxprec < prec ? c.maxprec : prec;
  u64 most = (u64)header + values - 1 + (u64)values * mp;
  if (most > c.maxbits) most = c.maxbits;
  if (most < header) most = header;
  if (most < c.minbits) most = c.minbits;
  return (u32)most;
}

bool fixed_size_blocks(const Call& call) {
  return call.c.minbits == call.c.maxbits && call.c.maxbits > 0 &&
         block_bits(call.c, call.type, call.dims) == call.c.maxbits;
}

bool strides_may_alias(const FieldGeom& f, int dims) {
  u64 st[4], n[4];
  int k = 0;
  for (int d = 0; d < dims; d++) {
    if (f.n[d] >= 2) {
      st[k] = (u64)(f.s[d] < 0 ? -f.s[d] : f.s[d]);
      n[k] = f.n[d];
      k++;
    }
  }
  for (int i = 1; i < k; i++)  // sort axes by |stride|
    for (int j = i; j > 0 && st[j] < st[j - 1]; j--) {
      std::swap(st[j], st[j - 1]);
      std::swap(n[j], n[j - 1]);
    }
  u64 reach = 1;
  for (int i = 0; i < k; i++) {
    if (st[i] < reach) return true;
    reach += st[i] * (n[i] - 1);
  }
  return false;
}

// Element index span [imin, imax] of a field relative to element [0,0,0,0].
static void index_span(const FieldGeom& f, int dims, i64* imin, i64* imax) {
  *imin = *imax = 0;
  for (int d = 0; d < dims; d++) {
    if (f.n[d] == 0) continue;
    i64 e = f.s[d] * (i64)(f.n[d] - 1);
    if (e < 0) *imin += e; else *imax += e;
  }
}

size_t plane_bytes(int type, int dims) {
  size_t prec = (type == 1 || type == 3) ? 32 : 64;
  size_t w = dims == 4 ? 4 : 1;
  return prec * w * sizeof(u64);
}

// ---------------------------------------------------------------------------
// Optional per-kernel timing with CUDA events recorded on the launching
// stream (zfpb_timing_enable / zfpb_timing_read).
// ---------------------------------------------------------------------------

enum KernelKind { K_ENCODE_FIXED, K_ENCODE_VAR, K_SCAN, K_PACK, K_DECODE_FIXED, K_DECODE_VAR, K_WALK, K_CLAIM,
                  K_OFFSETS, K_PARSE, K_FINISH, K_COUNT };

struct PendingTimer {
  int kind;
  cudaEvent_t e0, e1;
};
static std::mutex g_timer_mu;
static bool g_timing = false;
static std::vector<PendingTimer> g_pending;
static double g_ms[K_COUNT];
static unsigned long long g_count[K_COUNT];

struct KernelTimer {
  int kind;
  cudaStream_t s;
  cudaEvent_t e0 = nullptr;
  KernelTimer(int k, cudaStream_t st) : kind(k), s(st) {
    if (g_timing && cudaEventCreate(&e0) == cudaSuccess) cudaEventRecord(e0, s);
  }
  ~KernelTimer() {
    if (!e0) return;
    cudaEvent_t e1;
    if (cudaEventCreate(&e1) != cudaSuccess) return;
    cudaEventRecord(e1, s);
    std::lock_guard<std::mutex> l(g_timer_mu);
    g_pending.push_back({kind, e0, e1});
  }
};

void timing_enable(bool on) {
  std::lock_guard<std::mutex> l(g_timer_mu);
  for (auto& p : g_pending) {
    cudaEventDestroy(p.e0);
    cudaEventDestroy(p.e1);
  }
  g_pending.clear();
  for (int i = 0; i < K_COUNT; i++) {
    g_ms[i] = 0;
    g_count[i] = 0;
  }
  g_timing = on;
}

int timing_read(double* ms, unsigned long long* counts, int n) {
  std::lock_guard<std::mutex> l(g_timer_mu);
  for (auto& p : g_pending) {
    float t = 0;
    if (cudaEventSynchronize(p.e1) == cudaSuccess && cudaEventElapsedTime(&t, p.e0, p.e1) == cudaSuccess) {
      g_ms[p.kind] += t;
      g_count[p.kind] += 1;
    }
    cudaEventDestroy(p.e0);
    cudaEventDestroy(p.e1);
  }
  g_pending.clear();
  for (int i = 0; i < n && i < K_COUNT; i++) {
    ms[i] = g_ms[i];
    counts[i] = g_count[i];
  }
  return K_COUNT;
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of u32 block lengths into u64 offsets:
// per-tile totals, a scan of the totals, then per-tile scans.
// ---------------------------------------------------------------------------

static constexpr int SCAN_THREADS = 256;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Block-wide inclusive scan of one u64 per thread (warp shuffles + smem).
__device__ __forceinline__ u64 block_inclusive_scan(u64 v, u64* warp_sums) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    u64 t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) warp_sums[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    u64 s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      u64 t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  if (wid > 0) v += warp_sums[wid - 1];
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const u32* len, u64 n, u64* partial) {
  __shared__ u64 ws[32];
  const u64 base = (u64)blockIdx.x * SCAN_TILE + (u64)threadIdx.x * SCAN_ITEMS;
  u64 s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++)
    if (base + i < n) s += len[base + i];
  u64 incl = block_inclusive_scan(s, ws);
  if (threadIdx.x == blockDim.x - 1) partial[blockIdx.x] = incl;
}

// One CTA scans the tile totals in place (exclusive), carrying across rounds,
// and writes the grand total to *total.
__global__ void __launch_bounds__(1024) k_scan_partials(u64* partial, u64 m, u64* total) {
  __shared__ u64 ws[32];
  u64 carry = 0;
  for (u64 base = 0; base < m; base += blockDim.x) {
    u64 i = base + threadIdx.x;
    u64 v = i < m ? partial[i] : 0;
    u64 incl = block_inclusive_scan(v, ws);
    if (i < m) partial[i] = carry + incl - v;
    __shared__ u64 last;
    if (threadIdx.x == blockDim.x - 1) last = incl;
    __syncthreads();
    carry += last;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(const u32* len, u64 n, const u64* partial,
                                                              u64* off) {
  __shared__ u64 ws[32];
  const u64 base = (u64)blockIdx.x * SCAN_TILE + (u64)threadIdx.x * SCAN_ITEMS;
  u64 v[SCAN_ITEMS];
  u64 s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = base + i < n ? len[base + i] : 0;
    s += v[i];
  }
  u64 incl = block_inclusive_scan(s, ws);
  u64 run = partial[blockIdx.x] + incl - s;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    if (base + i < n) off[base + i] = run;
    run += v[i];
  }
}

__global__ void k_set_u64(u64* p, u64 v) { *p = v; }

__global__ void k_fill_fixed_offsets(u64* off, u64 n, u64 bits) {
  u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= n) off[i] = i * bits;
}

// ---------------------------------------------------------------------------
// Bit-exact concatenation of variable-size blocks (the device counterpart of
// zfp-rs compress.rs:196-216 append_bits).  Block i owns the stream words
// whose first bit lies in its range [start + off[i], start + off[i+1]); block
// 0 also owns the word holding the start bit.  Each owned word is gathered
// from the slots of block i and the blocks after it.
// ---------------------------------------------------------------------------

struct PackArgs {
  const u64* slots;
  u64 slot_words;
  const u64* off;  // nblocks + 1
  u64 nblocks;
  u64 start;
  u64 init_word;
  u64* out;
};

__device__ __forceinline__ u64 slot_bits(const u64* slot, u64 local, u32 take) {
  if (take == 0) return 0;
  u64 wi = local >> 6;
  u32 sh = (u32)(local & 63);
  u64 x = slot[wi] >> sh;
  if (sh != 0 && take > 64 - sh) x |= slot[wi + 1] << (64 - sh);
  return take < 64 ? x & ((1ull << take) - 1) : x;
}

// One warp per 32 consecutive blocks.  The warp's blocks own a contiguous run
// of stream words; lane l assembles words l, l + 32, ... of that run, finding
// each word's owner among the warp's block offsets (kept in shared memory), so
// slot reads and stream writes are coalesced and the lanes' loads do not wait
// on one another.  A word that runs past its owner's end takes the rest of its
// bits from the blocks after it.
__global__ void __launch_bounds__(256) k_pack(PackArgs a) {
  __shared__ u64 soff[8][33];
  const u32 wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const u64 b0 = ((u64)blockIdx.x * 8 + wib) * 32;
  if (b0 >= a.nblocks) return;
  const u32 nb = (u32)(a.nblocks - b0 < 32 ? a.nblocks - b0 : 32);
  u64* po = soff[wib];
  for (u32 t = lane; t <= nb; t += 32) po[t] = a.start + a.off[b0 + t];
  __syncwarp();
  const u64 wbeg = b0 == 0 ? a.start >> 6 : (po[0] + 63) >> 6;
  const u64 wend = (po[nb] + 63) >> 6;
  u32 j = 0;
  for (u64 w = wbeg + lane; w < wend; w += 32) {
    u64 v = 0;
    u32 fill = 0;
    u64 pos = w << 6;
    if (b0 == 0 && w == (a.start >> 6)) {
      v = a.init_word;
      fill = (u32)(a.start & 63);
      pos = a.start;
    }
    while (j + 1 < nb && po[j + 1] <= pos) j++;  // the block holding bit `pos`
    u64 blk = b0 + j;
    u64 pj = po[j], qj = po[j + 1];
    while (fill < 64 && blk < a.nblocks) {
      u64 local = pos - pj;
      u64 avail = qj - pos;
      u32 take = (u32)(avail < (u64)(64 - fill) ? avail : (u64)(64 - fill));
      v |= slot_bits(a.slots + blk * a.slot_words, local, take) << fill;  // fill < 64
      fill += take;
      pos += take;
      if (pos == qj) {
        blk++;
        if (blk < a.nblocks) {
          pj = qj;
          qj = a.start + a.off[blk + 1];
        }
      }
    }
    a.out[w] = v;
  }
}

// ---------------------------------------------------------------------------
// Device workspace, grown on demand and kept per device.
// ---------------------------------------------------------------------------

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t grow = std::max(need, (size_t)1 << 16);
    cudaError_t e = cudaMalloc(&p, grow);
    if (e == cudaSuccess) bytes = grow;
    return e;
  }
};

struct Workspace {
  Buf slots, lengths, offsets, partial, small, owner, planes, heads;
  u64* h_pinned = nullptr;  // two words for totals and flags
};

static std::mutex g_mu;
static std::map<int, Workspace*> g_ws;

static Workspace& workspace() {
  int dev = 0;
  cudaGetDevice(&dev);
  auto it = g_ws.find(dev);
  if (it != g_ws.end()) return *it->second;
  Workspace* w = new Workspace();
  cudaMallocHost((void**)&w->h_pinned, 4 * sizeof(u64));
  g_ws[dev] = w;
  return *w;
}

template <class Fn> static cudaError_t for_type(int type, Fn fn) {
  switch (type) {
    case 1: return fn((int*)nullptr);
    case 2: return fn((long long*)nullptr);
    case 3: return fn((float*)nullptr);
    default: return fn((double*)nullptr);
  }
}

#define ZFPB_CHECK(x)                 \
  do {                                \
    cudaError_t e_ = (x);             \
    if (e_ != cudaSuccess) {          \
      return ERR_CUDA;                \
    }                                 \
  } while (0)

static cudaError_t scan_lengths(Workspace& ws, const u32* d_len, u64 n, u64* d_off, cudaStream_t s) {
  u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  cudaError_t e = ws.partial.ensure((tiles + 1) * sizeof(u64));
  if (e != cudaSuccess) return e;
  u64* part = (u64*)ws.partial.p;
  KernelTimer t(K_SCAN, s);
  k_scan_reduce<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(d_len, n, part);
  k_scan_partials<<<1, 1024, 0, s>>>(part, tiles, d_off + n);
  k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(d_len, n, part, d_off);
  return cudaGetLastError();
}

// Threads and shared memory for the fixed-size encoder: stage of the CTA's
// bits plus plane storage, within the opt-in shared-memory limit.
static bool fixed_shape(const Call& call, int* threads, u64* per_cta, size_t* smem) {
  const u64 maxbits = call.c.maxbits;
  const u64 extra = (64 + maxbits - 1) / maxbits;
  const int cands[3] = {128, 64, 32};
  for (int th : cands) {
    if ((u64)th < 2 * extra) continue;
    size_t stage = ((63 + (u64)th * maxbits + 63) / 64 + 1) * sizeof(u64);
    size_t bytes = stage + plane_bytes(call.type, call.dims) * th;
    if (bytes <= 200 * 1024) {
      *threads = th;
      *per_cta = th - extra;
      *smem = bytes;
      return true;
    }
  }
  return false;
}

Status compress(const Call& call, const void* d_field, u64* d_out, u64 cap, u64 start, u64 init_word,
                u64* end_bit, u64* d_offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_mu);
  Workspace& ws = workspace();
  const u64 n = call.f.nblocks;
  if (n == 0) {
    *end_bit = start;
    if ((start & 63) != 0) {
      if ((start >> 6) >= cap) return ERR_OVERFLOW;
      ZFPB_CHECK(cudaMemcpyAsync(d_out + (start >> 6), &init_word, sizeof(u64), cudaMemcpyHostToDevice, s));
      ZFPB_CHECK(cudaStreamSynchronize(s));
    }
    return OK;
  }
  if (fixed_size_blocks(call)) {
    const u64 maxbits = call.c.maxbits;
    const u64 end = start + n * maxbits;
    if ((end + 63) / 64 > cap) return ERR_OVERFLOW;
    int threads;
    u64 per_cta;
    size_t smem;
    if (fixed_shape(call, &threads, &per_cta, &smem)) {
      EncodeFixedArgs a;
      a.data = d_field;
      a.f = call.f;
      a.c = call.c;
      a.out = d_out;
      a.start = start;
      a.init_word = init_word;
      a.blocks_per_cta = per_cta;
      u64 ctas = (n + per_cta - 1) / per_cta;
      {
        KernelTimer t(K_ENCODE_FIXED, s);
        ZFPB_CHECK(for_type(call.type, [&](auto* tp) {
          using T = std::remove_pointer_t<decltype(tp)>;
          return Launch<T>::encode_fixed(call, a, ctas, threads, smem, s);
        }));
      }
      if (d_offsets) {
        KernelTimer t(K_OFFSETS, s);
        k_fill_fixed_offsets<<<(unsigned)((n + 256) / 256), 256, 0, s>>>(d_offsets, n, maxbits);
      }
      ZFPB_CHECK(cudaGetLastError());
      *end_bit = end;
      return OK;
    }
    // Budgets too large to stage fall through to the variable-size path.
  }
  // Variable-size blocks: code into slots, scan lengths, concatenate.
  const u64 bb = block_bits(call.c, call.type, call.dims);
  const u64 slot_words = (bb + 63) / 64 + 1;
  ZFPB_CHECK(ws.slots.ensure((n * slot_words + 1) * sizeof(u64)));
  ZFPB_CHECK(ws.lengths.ensure(n * sizeof(u32)));
  u64* off = d_offsets;
  if (!off) {
    ZFPB_CHECK(ws.offsets.ensure((n + 1) * sizeof(u64)));
    off = (u64*)ws.offsets.p;
  }
  EncodeVarArgs ea;
  ea.data = d_field;
  ea.f = call.f;
  ea.c = call.c;
  ea.slots = (u64*)ws.slots.p;
  ea.slot_words = slot_words;
  ea.lengths = (u32*)ws.lengths.p;
  {
    KernelTimer t(K_ENCODE_VAR, s);
    ZFPB_CHECK(for_type(call.type, [&](auto* tp) {
      using T = std::remove_pointer_t<decltype(tp)>;
      return Launch<T>::encode_var(call, ea, s);
    }));
  }
  ZFPB_CHECK(scan_lengths(ws, ea.lengths, n, off, s));
  ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned, off + n, sizeof(u64), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  const u64 total = ws.h_pinned[0];
  const u64 end = start + total;
  *end_bit = end;
  if ((end + 63) / 64 > cap) return ERR_OVERFLOW;
  PackArgs pa;
  pa.slots = ea.slots;
  pa.slot_words = slot_words;
  pa.off = off;
  pa.nblocks = n;
  pa.start = start;
  pa.init_word = init_word;
  pa.out = d_out;
  {
    KernelTimer t(K_PACK, s);
    k_pack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pa);
  }
  ZFPB_CHECK(cudaGetLastError());
  return OK;
}

// Decode every block, from i * maxbits (var false) or from a.offsets (var
// true).  3D fields use the two-kernel decoder (k_parse, k_finish), whose
// plane scratch is as large as the field.  Other fields, 3D fields whose
// scratch cannot be had, and every field while the environment variable
// ZFPB_ONE_KERNEL_DECODE is 1 use the one-kernel decoder.  Both give the
// same values.
static cudaError_t decode_blocks(Workspace& ws, const Call& call, const DecodeArgs& a, bool var, cudaStream_t s) {
  const u64 n = call.f.nblocks;
  const char* one = getenv("ZFPB_ONE_KERNEL_DECODE");
  if (call.dims == 3 && !(one && one[0] == '1')) {
    const u64 stride = (n + 31) & ~31ull;
    const u64 planes = (call.type == 1 || call.type == 3) ? 32 : 64;
    if (stride < (1ull << 31) && ws.planes.ensure(planes * stride * sizeof(u64)) == cudaSuccess &&
        ws.heads.ensure(n * sizeof(u64)) == cudaSuccess) {
      SplitArgs sa{(u64*)ws.planes.p, stride, (u64*)ws.heads.p};
      cudaError_t e;
      {
        KernelTimer t(K_PARSE, s);
        e = for_type(call.type, [&](auto* tp) {
          using T = std::remove_pointer_t<decltype(tp)>;
          return Launch<T>::parse(call, a, sa, var, s);
        });
      }
      if (e != cudaSuccess) return e;
      KernelTimer t(K_FINISH, s);
      return for_type(call.type, [&](auto* tp) {
        using T = std::remove_pointer_t<decltype(tp)>;
        return Launch<T>::finish(call, a, sa, s);
      });
    }
    cudaGetLastError();  // a failed scratch allocation: use the one-kernel decoder
  }
  KernelTimer t(var ? K_DECODE_VAR : K_DECODE_FIXED, s);
  return for_type(call.type, [&](auto* tp) {
    using T = std::remove_pointer_t<decltype(tp)>;
    return var ? Launch<T>::decode_var(call, a, s) : Launch<T>::decode_fixed(call, a, s);
  });
}

Status decompress(const Call& call, const u64* d_in, u64 len, u64 start, void* d_field, u64* end_bit,
                  const u64* d_offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_mu);
  Workspace& ws = workspace();
  const u64 n = call.f.nblocks;
  if (n == 0) {
    *end_bit = start;
    return OK;
  }
  ZFPB_CHECK(ws.small.ensure(64));
  unsigned* flags = (unsigned*)ws.small.p;
  ZFPB_CHECK(cudaMemsetAsync(flags, 0, sizeof(unsigned), s));
  DecodeArgs a;
  a.data = d_field;
  a.f = call.f;
  a.c = call.c;
  a.stream = d_in;
  a.stream_len = len;
  a.start = start;
  a.offsets = nullptr;
  a.flags = flags;
  a.owner = nullptr;
  a.imin = 0;
  if (strides_may_alias(call.f, call.dims)) {
    i64 imin, imax;
    index_span(call.f, call.dims, &imin, &imax);
    u64 span = (u64)(imax - imin) + 1;
    ZFPB_CHECK(ws.owner.ensure(span * sizeof(u64)));
    ZFPB_CHECK(cudaMemsetAsync(ws.owner.p, 0, span * sizeof(u64), s));
    a.owner = (u64*)ws.owner.p;
    a.imin = imin;
    unsigned g = (unsigned)((n + 127) / 128);
    KernelTimer t(K_CLAIM, s);
    switch (call.dims) {
      case 1: k_claim<1><<<g, 128, 0, s>>>(call.f, a.owner, imin); break;
      case 2: k_claim<2><<<g, 128, 0, s>>>(call.f, a.owner, imin); break;
      case 3: k_claim<3><<<g, 128, 0, s>>>(call.f, a.owner, imin); break;
      default: k_claim<4><<<g, 128, 0, s>>>(call.f, a.owner, imin); break;
    }
    ZFPB_CHECK(cudaGetLastError());
  }
  if (fixed_size_blocks(call)) {
    ZFPB_CHECK(decode_blocks(ws, call, a, false, s));
    ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    ZFPB_CHECK(cudaStreamSynchronize(s));
    *end_bit = start + n * (u64)call.c.maxbits;
    return (*(unsigned*)ws.h_pinned & FLAG_TRUNCATED) ? ERR_TRUNCATED : OK;
  }
  unsigned fl = FLAG_BAD_INDEX;
  u64* off = nullptr;
  if (d_offsets) {
    a.offsets = const_cast<u64*>(d_offsets);
    ZFPB_CHECK(decode_blocks(ws, call, a, true, s));
    ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    ZFPB_CHECK(cudaStreamSynchronize(s));
    fl = *(unsigned*)ws.h_pinned;
    off = const_cast<u64*>(d_offsets);
    if (fl & FLAG_BAD_INDEX) return ERR_BAD_INDEX;
  }
  if (fl & FLAG_BAD_INDEX) {
    ZFPB_CHECK(ws.offsets.ensure((n + 1) * sizeof(u64)));
    off = (u64*)ws.offsets.p;
    a.offsets = off;
    ZFPB_CHECK(cudaMemsetAsync(flags, 0, sizeof(unsigned), s));
    {
      KernelTimer t(K_WALK, s);
      ZFPB_CHECK(for_type(call.type, [&](auto* tp) {
        using T = std::remove_pointer_t<decltype(tp)>;
        return Launch<T>::walk(call, a, s);
      }));
    }
    ZFPB_CHECK(decode_blocks(ws, call, a, true, s));
    ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    ZFPB_CHECK(cudaStreamSynchronize(s));
    fl = *(unsigned*)ws.h_pinned;
  }
  ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned + 1, off + n, sizeof(u64), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  *end_bit = start + ws.h_pinned[1];
  if (fl & FLAG_BAD_INDEX) return ERR_CUDA;
  return (fl & FLAG_TRUNCATED) ? ERR_TRUNCATED : OK;
}

}  // namespace zfpb

// ---------------------------------------------------------------------------
// Compression without device allocation (zfpb_compress_device_noalloc).
//
// Its scratch (block slots, bit lengths, block offsets, scan totals) is this
// file-scope device array instead of cudaMalloc'd workspace.  Every device
// that loads the library holds the array until the process exits.  Calls
// share it and leave their contents in it; nothing in it needs to start at
// zero, because every word a call reads was written earlier in that same call.
// Two calls whose kernels overlap on the GPU (different host threads or
// streams) race on the array.
// ---------------------------------------------------------------------------

namespace zfpb {

static constexpr u64 NOALLOC_SCRATCH_WORDS = 1ull << 21;  // 16 MiB
static __device__ __align__(256) u64 g_noalloc_scratch[NOALLOC_SCRATCH_WORDS];

static std::mutex g_noalloc_mu;
static u64* g_noalloc_ptr[64];

u64 noalloc_scratch_bytes() { return NOALLOC_SCRATCH_WORDS * sizeof(u64); }

// The array's device address for the current device, looked up on the first
// call on that device.  In host code the array's name is only a host-side
// stand-in, never a device address.
static Status noalloc_scratch(u64** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ERR_CUDA;
  std::lock_guard<std::mutex> l(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
      cudaGetLastError();
      return ERR_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<u64*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return OK;
}

Status compress_noalloc(const Call& call, const void* d_field, u64* d_out, u64 cap, u64* end_bit,
                        cudaStream_t s) {
  const u64 n = call.f.nblocks;
  *end_bit = 0;
  if (n == 0) return OK;
  if (fixed_size_blocks(call)) {
    // Fixed-size blocks need no scratch: the same kernel as compress().
    const u64 maxbits = call.c.maxbits;
    const u64 end = n * maxbits;
    if ((end + 63) / 64 > cap) return ERR_OVERFLOW;
    int threads;
    u64 per_cta;
    size_t smem;
    if (fixed_shape(call, &threads, &per_cta, &smem)) {
      EncodeFixedArgs a;
      a.data = d_field;
      a.f = call.f;
      a.c = call.c;
      a.out = d_out;
      a.start = 0;
      a.init_word = 0;
      a.blocks_per_cta = per_cta;
      u64 ctas = (n + per_cta - 1) / per_cta;
      ZFPB_CHECK(for_type(call.type, [&](auto* tp) {
        using T = std::remove_pointer_t<decltype(tp)>;
        return Launch<T>::encode_fixed(call, a, ctas, threads, smem, s);
      }));
      ZFPB_CHECK(cudaStreamSynchronize(s));
      *end_bit = end;
      return OK;
    }
  }
  u64* scratch = nullptr;
  Status st = noalloc_scratch(&scratch);
  if (st != OK) return st;
  const u64 bb = block_bits(call.c, call.type, call.dims);
  const u64 slot_words = (bb + 63) / 64 + 1;
  const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  const u64 w_slots = n * slot_words + 1, w_len = (n + 1) / 2, w_off = n + 1, w_part = tiles + 1;
  if (w_slots + w_len + w_off + w_part > NOALLOC_SCRATCH_WORDS) return ERR_TOO_LARGE;
  u64* slots = scratch;
  u32* lengths = reinterpret_cast<u32*>(scratch + w_slots);
  u64* off = scratch + w_slots + w_len;
  u64* part = off + w_off;
  EncodeVarArgs ea;
  ea.data = d_field;
  ea.f = call.f;
  ea.c = call.c;
  ea.slots = slots;
  ea.slot_words = slot_words;
  ea.lengths = lengths;
  ZFPB_CHECK(for_type(call.type, [&](auto* tp) {
    using T = std::remove_pointer_t<decltype(tp)>;
    return Launch<T>::encode_var(call, ea, s);
  }));
  k_scan_reduce<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(lengths, n, part);
  k_scan_partials<<<1, 1024, 0, s>>>(part, tiles, off + n);
  k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(lengths, n, part, off);
  ZFPB_CHECK(cudaGetLastError());
  u64 total = 0;
  ZFPB_CHECK(cudaMemcpyAsync(&total, off + n, sizeof(u64), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  *end_bit = total;
  if ((total + 63) / 64 > cap) return ERR_OVERFLOW;
  PackArgs pa;
  pa.slots = slots;
  pa.slot_words = slot_words;
  pa.off = off;
  pa.nblocks = n;
  pa.start = 0;
  pa.init_word = 0;
  pa.out = d_out;
  k_pack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pa);
  ZFPB_CHECK(cudaGetLastError());
  ZFPB_CHECK(cudaStreamSynchronize(s));
  return OK;
}

}  // namespace zfpb
