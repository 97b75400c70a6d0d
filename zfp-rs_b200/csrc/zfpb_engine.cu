// Orchestration of a compress or decompress call on the device: choice of the
// fixed-size or variable-size path, the device-wide scan of block bit lengths,
// the bit-exact concatenation of variable-size blocks, and the device
// workspace.  The stream layout follows zfp-rs src/compress.rs and
// src/decompress.rs.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <cstring>
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
  if (dims == 1) return 0;  // 4-value blocks keep their planes in registers
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
static thread_local bool g_no_timers = false;  // set while a batch plan is being captured
static std::vector<PendingTimer> g_pending;
static double g_ms[K_COUNT];
static unsigned long long g_count[K_COUNT];

struct KernelTimer {
  int kind;
  cudaStream_t s;
  cudaEvent_t e0 = nullptr;
  KernelTimer(int k, cudaStream_t st) : kind(k), s(st) {
    if (g_timing && !g_no_timers && cudaEventCreate(&e0) == cudaSuccess) cudaEventRecord(e0, s);
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
static_assert(SCAN_ITEMS == 8, "scan_load reads two uint4");

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

// A thread's SCAN_ITEMS lengths: two 16-byte loads where the run is whole
// and aligned, else one at a time.
__device__ __forceinline__ void scan_load(const u32* len, u64 n, u64 base, u32* v) {
  const u32* p = len + base;
  if (base + SCAN_ITEMS <= n && ((uintptr_t)p & 15) == 0) {
    const uint4 a = reinterpret_cast<const uint4*>(p)[0], b = reinterpret_cast<const uint4*>(p)[1];
    v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) v[i] = base + i < n ? len[base + i] : 0u;
  }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const u32* len, u64 n, u64* partial) {
  __shared__ u64 ws[32];
  const u64 base = (u64)blockIdx.x * SCAN_TILE + (u64)threadIdx.x * SCAN_ITEMS;
  u32 v[SCAN_ITEMS];
  scan_load(len, n, base, v);
  u64 s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) s += v[i];
  u64 incl = block_inclusive_scan(s, ws);
  if (threadIdx.x == blockDim.x - 1) partial[blockIdx.x] = incl;
}

// One CTA scans the tile totals in place (exclusive), carrying across rounds,
// and writes the grand total to *total.
__global__ void __launch_bounds__(1024) k_scan_partials(u64* partial, u64 m, u64* total, const u64* carry_in) {
  __shared__ u64 ws[32];
  u64 carry = carry_in ? *carry_in : 0;
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
  u32 v[SCAN_ITEMS];
  scan_load(len, n, base, v);
  u64 s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) s += v[i];
  u64 incl = block_inclusive_scan(s, ws);
  u64 run = partial[blockIdx.x] + incl - s;
  u64 o[SCAN_ITEMS];
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    o[i] = run;
    run += v[i];
  }
  u64* q = off + base;
  if (base + SCAN_ITEMS <= n && ((uintptr_t)q & 15) == 0) {
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i += 2) reinterpret_cast<ulonglong2*>(q)[i / 2] = make_ulonglong2(o[i], o[i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
      if (base + i < n) q[i] = o[i];
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

__device__ __forceinline__ u64 slot_bits(const u64* slot, u32 local, u32 take) {
  if (take == 0) return 0;
  const u32 wi = local >> 6, sh = local & 63;
  u64 x = slot[wi] >> sh;
  if (sh != 0 && take > 64 - sh) x |= slot[wi + 1] << (64 - sh);
  return take < 64 ? x & ((1ull << take) - 1) : x;
}

// One warp per BW consecutive blocks.  The warp's blocks own a contiguous run
// of stream words; lane l assembles words l, l + 32, ... of that run, finding
// each word's owner among the warp's block offsets (kept in shared memory), so
// slot reads and stream writes are coalesced and the lanes' loads do not wait
// on one another.  A word that runs past its owner's end takes the rest of its
// bits from the blocks after it.  Block i's bits start at delta + off[i]; only
// words below `cap` are written.  Bit positions inside the warp's run are
// 32-bit, relative to its first block (BW blocks of at most ZFP's largest
// block, 4^4 doubles, span far less than 2^32 bits).  Small blocks (1D, 2D)
// use more blocks per warp so that a warp has enough words to share out.
template <int BW>
__device__ void pack_warp(const u64* slots, u64 slot_words, const u64* off, u64 delta, u64 nblocks, u64 start,
                          u64 init_word, u64* out, u64 cap, u64 b0, u32* po, u32 lane) {
  const u32 nb = (u32)(nblocks - b0 < BW ? nblocks - b0 : BW);
  const u64 base = delta + off[b0];  // bit of the warp's first block; == start when b0 == 0
  for (u32 t = lane; t <= nb; t += 32) po[t] = (u32)(delta + off[b0 + t] - base);
  __syncwarp();
  const u32 span = po[nb];
  const u64 wbeg = b0 == 0 ? start >> 6 : (base + 63) >> 6;
  const u64 wend = (base + span + 63) >> 6;
  // Blocks of 8 words or more on average: the owner of a lane's next word
  // (32 words on) is at most a few blocks ahead, so a short linear step finds
  // it.  Shorter blocks (1D, 2D, low rates) go straight to bisection.
  const u32 lin = span >= nb * 512u ? 4 : 0;
  u32 j = 0;
  for (u64 w = wbeg + lane; w < wend; w += 32) {
    u64 v = 0;
    u32 fill = 0, pos;
    if (b0 == 0 && w == wbeg) {
      v = init_word;
      fill = (u32)(start & 63);
      pos = 0;
    } else {
      pos = (u32)((w << 6) - base);
    }
    // The block holding bit `pos`: the largest j < nb with po[j] <= pos.  It
    // only moves forward, so step from the last one; a far owner is found by
    // bisection instead.
    u32 steps = 0;
    while (steps < lin && j + 1 < nb && po[j + 1] <= pos) j++, steps++;
    if (j + 1 < nb && po[j + 1] <= pos) {
      u32 hi = nb;
      while (hi - j > 1) {
        const u32 mid = (j + hi) >> 1;
        if (po[mid] <= pos) j = mid;
        else hi = mid;
      }
    }
    u32 jj = j;
    u32 pj = po[jj], qj = po[jj + 1];
    while (fill < 64 && jj < nb) {
      const u32 avail = qj - pos;
      const u32 take = avail < 64 - fill ? avail : 64 - fill;
      v |= slot_bits(slots + (b0 + jj) * slot_words, pos - pj, take) << fill;  // fill < 64
      fill += take;
      pos += take;
      if (pos == qj) {
        jj++;
        pj = qj;
        qj = po[jj + (jj < nb)];  // past the last block: loop ends
      }
    }
    // A word that runs past the warp's blocks takes the rest from the next
    // warp's (only the run's last word; never for the array's last block).
    if (fill < 64 && b0 + nb < nblocks) {
      u64 blk = b0 + nb;
      u64 pj64 = base + span, qj64 = delta + off[blk + 1];
      u64 pos64 = base + pos;
      while (fill < 64 && blk < nblocks) {
        const u64 avail = qj64 - pos64;
        const u32 take = (u32)(avail < (u64)(64 - fill) ? avail : (u64)(64 - fill));
        v |= slot_bits(slots + blk * slot_words, (u32)(pos64 - pj64), take) << fill;
        fill += take;
        pos64 += take;
        if (pos64 == qj64) {
          blk++;
          if (blk < nblocks) {
            pj64 = qj64;
            qj64 = delta + off[blk + 1];
          }
        }
      }
    }
    if (w < cap) out[w] = v;
  }
  __syncwarp();
}

// Blocks per warp of the pack: more for small blocks.
static inline int pack_blocks_per_warp(int dims) { return dims <= 2 ? 128 : 32; }

template <int BW> __global__ void __launch_bounds__(256) k_pack(PackArgs a) {
  __shared__ u32 soff[8][BW + 1];
  const u32 wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const u64 b0 = ((u64)blockIdx.x * 8 + wib) * BW;
  if (b0 >= a.nblocks) return;
  pack_warp<BW>(a.slots, a.slot_words, a.off, a.start, a.nblocks, a.start, a.init_word, a.out, ~0ull, b0, soff[wib],
                lane);
}

// Staged pack for small blocks (slots of at most STAGE_SLOT_WORDS words: 1D
// blocks, 2D blocks of 32-bit values).  A CTA takes STAGE_BLOCKS consecutive
// blocks; each thread ORs its blocks' bits into a shared copy of the stream
// words they cover, then the CTA stores the words it owns (those whose first
// bit lies in its blocks' range; the first CTA also owns the word holding
// `start`) in coalesced runs.  The last owned word takes the rest of its bits
// from the blocks after the CTA's.  Where a warp per word spends most of its
// time finding each word's owner among many short blocks, here a block costs
// a load and two shared-memory ORs per slot word.
static constexpr u32 STAGE_BLOCKS = 512;
static constexpr u64 STAGE_SLOT_WORDS = 10;

struct StageSmem {
  u64 buf[STAGE_BLOCKS * (STAGE_SLOT_WORDS - 1) + 2];  // a block has at most (slot_words - 1) * 64 bits
  u32 po[STAGE_BLOCKS + 1];
};

__device__ void pack_stage(const u64* slots, u64 slot_words, const u64* off, u64 delta, u64 nblocks, u64 start,
                           u64 init_word, u64* out, u64 cap, u64 b0, StageSmem& sm) {
  const u32 tid = threadIdx.x, nt = blockDim.x;
  const u32 nb = (u32)(nblocks - b0 < STAGE_BLOCKS ? nblocks - b0 : STAGE_BLOCKS);
  const u64 base = delta + off[b0];  // == start when b0 == 0
  for (u32 t = tid; t <= nb; t += nt) sm.po[t] = (u32)(delta + off[b0 + t] - base);
  const u32 s0 = (u32)(base & 63);
  const u64 wfirst = base >> 6;  // global index of buffer word 0
  __syncthreads();
  const u32 span = sm.po[nb];
  const u32 nwords = (s0 + span + 63) >> 6;
  for (u32 i = tid; i < nwords; i += nt) sm.buf[i] = (i == 0 && b0 == 0) ? init_word : 0ull;
  __syncthreads();
  for (u32 i = tid; i < nb; i += nt) {
    const u32 p = s0 + sm.po[i], len = sm.po[i + 1] - sm.po[i];
    const u64* slot = slots + (b0 + i) * slot_words;
    for (u32 k = 0; k * 64 < len; k++) {
      u64 x = slot[k];
      const u32 take = len - k * 64;
      if (take < 64) x &= (1ull << take) - 1;
      const u32 q = p + k * 64, wi = q >> 6, sh = q & 63;
      atomicOr(&sm.buf[wi], x << sh);
      if (sh != 0 && (x >> (64 - sh)) != 0) atomicOr(&sm.buf[wi + 1], x >> (64 - sh));
    }
  }
  __syncthreads();
  const u32 first = (b0 == 0 || s0 == 0) ? 0 : 1;  // else word 0 is the previous CTA's
  for (u32 wi = first + tid; wi < nwords; wi += nt) {
    u64 v = sm.buf[wi];
    u32 fill = (s0 + span) & 63;
    if (wi == nwords - 1 && fill != 0 && b0 + nb < nblocks) {
      // The rest of the word from the blocks after this CTA's.
      u64 blk = b0 + nb;
      u64 pj = base + span, qj = delta + off[blk + 1], pos = pj;
      while (fill < 64 && blk < nblocks) {
        const u64 avail = qj - pos;
        const u32 take = (u32)(avail < (u64)(64 - fill) ? avail : (u64)(64 - fill));
        v |= slot_bits(slots + blk * slot_words, (u32)(pos - pj), take) << fill;
        fill += take;
        pos += take;
        if (pos == qj) {
          blk++;
          if (blk < nblocks) {
            pj = qj;
            qj = delta + off[blk + 1];
          }
        }
      }
    }
    const u64 g = wfirst + wi;
    if (g < cap) out[g] = v;
  }
}

__global__ void __launch_bounds__(256) k_pack_stage(PackArgs a) {
  __shared__ StageSmem sm;
  pack_stage(a.slots, a.slot_words, a.off, a.start, a.nblocks, a.start, a.init_word, a.out, ~0ull,
             (u64)blockIdx.x * STAGE_BLOCKS, sm);
}

static cudaError_t launch_pack(const PackArgs& pa, int dims, cudaStream_t s) {
  if (pa.slot_words <= STAGE_SLOT_WORDS)
    k_pack_stage<<<(unsigned)((pa.nblocks + STAGE_BLOCKS - 1) / STAGE_BLOCKS), 256, 0, s>>>(pa);
  else if (pack_blocks_per_warp(dims) == 128)
    k_pack<128><<<(unsigned)((pa.nblocks + 1023) / 1024), 256, 0, s>>>(pa);
  else
    k_pack<32><<<(unsigned)((pa.nblocks + 255) / 256), 256, 0, s>>>(pa);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Device workspace, grown on demand and kept per device.
// ---------------------------------------------------------------------------

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t owner = nullptr;  // set: allocated stream-ordered on this stream
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
  // Grow in stream order on s from `pool` (no device-wide synchronisation),
  // by 1.5x steps.
  cudaError_t ensure_on(size_t need, cudaStream_t s, cudaMemPool_t pool) {
    if (need <= bytes) return cudaSuccess;
    if (p) cudaFreeAsync(p, owner);
    p = nullptr;
    bytes = 0;
    size_t grow = std::max(need + need / 2, (size_t)1 << 16);
    cudaError_t e = cudaMallocFromPoolAsync(&p, grow, pool, s);
    if (e == cudaSuccess) {
      bytes = grow;
      owner = s;
    }
    return e;
  }
  void release() {
    if (!p) return;
    if (owner) cudaFreeAsync(p, owner);
    else cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

struct Workspace {
  Buf slots, lengths, offsets, partial, small, owner, planes, heads;
  Buf spec_list, spec_fix, spec_seg, spec_pieces;  // speculative walk
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

// Exclusive scan of n lengths into off[0..n] (off[n] = total); `part` holds
// ceil(n / SCAN_TILE) + 1 words.  With carry_in (device, read before off is
// written; it may be off[0] itself) every offset is raised by *carry_in.
static cudaError_t scan_entries(const u32* d_len, u64 n, u64* d_off, u64* part, cudaStream_t s,
                                const u64* carry_in = nullptr) {
  u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  KernelTimer t(K_SCAN, s);
  k_scan_reduce<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(d_len, n, part);
  k_scan_partials<<<1, 1024, 0, s>>>(part, tiles, d_off + n, carry_in);
  k_scan_tiles<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(d_len, n, part, d_off);
  return cudaGetLastError();
}

static cudaError_t scan_lengths(Workspace& ws, const u32* d_len, u64 n, u64* d_off, cudaStream_t s) {
  u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  cudaError_t e = ws.partial.ensure((tiles + 1) * sizeof(u64));
  if (e != cudaSuccess) return e;
  return scan_entries(d_len, n, d_off, (u64*)ws.partial.p, s);
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
    ZFPB_CHECK(launch_pack(pa, call.dims, s));
  }
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

// One CTA per piece of the speculative walk's chain: its positions (relative
// to the segment they were listed in) to their places among the offsets.
__global__ void k_spec_write(SpecWalkArgs a, const SpecPiece* pieces, u64* off, u64 n) {
  const SpecPiece pc = pieces[blockIdx.x];
  const u32* src = (pc.kind == 0 ? a.list : a.fix) + (u64)pc.seg * a.cap + pc.from;
  const u64 lo = (u64)pc.seg * a.seg_bits;
  for (u32 i = threadIdx.x; i < pc.count; i += blockDim.x)
    if (pc.dst + i <= n) off[pc.dst + i] = lo + src[i];
}

// Offsets (relative to start) of a variable-rate stream without an index by
// the speculative parallel walk (k_spec_walk, k_spec_fix).  Sets *done when
// a.offsets holds them; else (short streams, a full list) the caller walks
// serially.  ZFPB_SERIAL_WALK=1 turns it off.
static Status spec_walk(Workspace& ws, const Call& call, const DecodeArgs& a, cudaStream_t s, bool* done) {
  *done = false;
  const char* env = getenv("ZFPB_SERIAL_WALK");
  if (env && env[0] == '1') return OK;
  const u64 n = call.f.nblocks;
  const u64 end_bits = a.stream_len * 64 > a.start ? a.stream_len * 64 - a.start : 0;
  if (n < 1024 || end_bits == 0) return OK;
  // Segments of G blocks on average, one walker per warp, about 4096 of them
  // or fewer; a lead-in of L blocks before each.  A walk takes L + G steps
  // plus its garbage start, and a fix about as many as the walks it meets
  // took to join the true walk: a few hundred bits for 1D (no lead-in), up
  // to a few thousand blocks for 2D and 3D.  Swept on 2D f32 1024^2 and 3D
  // f64 128^3 and 512^3: a lead-in of one segment for 2D; half a segment for
  // 3D (512^3 f64 fixed-accuracy: 26.9 ms at one segment, 20.3 ms at half,
  // 22.4 ms at a quarter; segments of 256 or 1024 blocks were slower).  4D
  // fields take the 3D sizes.
  const u64 avg = std::max<u64>(1, end_bits / n);
  const u64 G = std::max<u64>(call.dims == 1 ? 128 : call.dims == 2 ? 256 : 512, n / 4096);
  const u64 L = call.dims == 1 ? 0 : call.dims == 2 ? G : G / 2;
  const u64 seg_bits = G * avg;
  if (seg_bits >= (1ull << 31)) return OK;
  const u64 nseg = (end_bits + seg_bits - 1) / seg_bits;
  if (nseg < 4) return OK;
  const u64 cap = G + G / 2 + 8192;
  ZFPB_CHECK(ws.spec_list.ensure(nseg * cap * sizeof(u32)));
  ZFPB_CHECK(ws.spec_fix.ensure(nseg * cap * sizeof(u32)));
  ZFPB_CHECK(ws.spec_seg.ensure(nseg * (2 * sizeof(u64) + 4 * sizeof(u32)) + 64));
  ZFPB_CHECK(ws.spec_pieces.ensure(2 * nseg * sizeof(SpecPiece)));
  SpecWalkArgs sa;
  sa.stream = a.stream;
  sa.stream_len = a.stream_len;
  sa.start = a.start;
  sa.c = a.c;
  sa.nseg = nseg;
  sa.seg_bits = seg_bits;
  sa.end_bits = end_bits;
  sa.cap = cap;
  sa.lead = L * avg;
  sa.list = (u32*)ws.spec_list.p;
  sa.fix = (u32*)ws.spec_fix.p;
  u64* w64 = (u64*)ws.spec_seg.p;
  sa.exit_spec = w64;
  sa.fix_exit = w64 + nseg;
  u32* w32 = (u32*)(w64 + 2 * nseg);
  sa.list_len = w32;
  sa.fix_len = w32 + nseg;
  sa.sync_t = w32 + 2 * nseg;
  sa.sync_j = w32 + 3 * nseg;
  sa.flags = w32 + 4 * nseg;
  auto by_type = [&](auto launch) {
    return for_type(call.type, [&](auto* tp) { return launch(tp); });
  };
  ZFPB_CHECK(cudaMemsetAsync(sa.flags, 0, sizeof(unsigned), s));
  ZFPB_CHECK(by_type([&](auto* tp) { return Launch<std::remove_pointer_t<decltype(tp)>>::spec_walk(call.dims, sa, s); }));
  ZFPB_CHECK(by_type([&](auto* tp) { return Launch<std::remove_pointer_t<decltype(tp)>>::spec_fix(call.dims, sa, s); }));
  // The chain, on the host: segment 0's list; then for each segment entered
  // at the exit of the list before it, its fix and the tail of the list the
  // fix joined (whose exit leads into the next segment).
  std::vector<u64> h64(2 * nseg);
  std::vector<u32> h32(4 * nseg + 1);
  ZFPB_CHECK(cudaMemcpyAsync(h64.data(), w64, 2 * nseg * sizeof(u64), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaMemcpyAsync(h32.data(), w32, (4 * nseg + 1) * sizeof(u32), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  if (h32[4 * nseg]) return OK;  // a list or fix overflowed
  const u64* exit_spec = h64.data();
  const u64* fix_exit = h64.data() + nseg;
  const u32* list_len = h32.data();
  const u32* fix_len = h32.data() + nseg;
  const u32* sync_t = h32.data() + 2 * nseg;
  const u32* sync_j = h32.data() + 3 * nseg;
  std::vector<SpecPiece> pieces;
  pieces.push_back({0, 0, 0, list_len[0], 0});
  u64 total = list_len[0], last = exit_spec[0];
  for (u64 sg = 1; sg < nseg && total <= n;) {
    pieces.push_back({1, (u32)sg, 0, fix_len[sg], total});
    total += fix_len[sg];
    const u32 t = sync_t[sg];
    if (t >= nseg) {
      last = fix_exit[sg];
      break;
    }
    pieces.push_back({0, t, sync_j[sg], list_len[t] - sync_j[sg], total});
    total += list_len[t] - sync_j[sg];
    last = exit_spec[t];
    sg = (u64)t + 1;
  }
  ZFPB_CHECK(cudaMemcpyAsync(ws.spec_pieces.p, pieces.data(), pieces.size() * sizeof(SpecPiece),
                             cudaMemcpyHostToDevice, s));
  k_spec_write<<<(unsigned)pieces.size(), 128, 0, s>>>(sa, (const SpecPiece*)ws.spec_pieces.p, a.offsets, n);
  ZFPB_CHECK(cudaGetLastError());
  if (total <= n) {
    ZFPB_CHECK(by_type([&](auto* tp) {
      return Launch<std::remove_pointer_t<decltype(tp)>>::spec_tail(call.dims, sa, a.offsets, total, n, last, s);
    }));
  }
  ZFPB_CHECK(cudaStreamSynchronize(s));  // the host's piece table is freed on return
  *done = true;
  return OK;
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
    bool spec = false;
    {
      KernelTimer t(K_WALK, s);
      const Status st = spec_walk(ws, call, a, s, &spec);
      if (st != OK) return st;
    }
    if (spec) {
      ZFPB_CHECK(decode_blocks(ws, call, a, true, s));
      ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
      ZFPB_CHECK(cudaStreamSynchronize(s));
      fl = *(unsigned*)ws.h_pinned;
      if (fl & FLAG_BAD_INDEX) spec = false;  // not the serial walk's offsets: walk serially
    }
    if (!spec) {
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
  }
  ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned + 1, off + n, sizeof(u64), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  *end_bit = start + ws.h_pinned[1];
  if (fl & FLAG_BAD_INDEX) return ERR_CUDA;
  return (fl & FLAG_TRUNCATED) ? ERR_TRUNCATED : OK;
}

// ---------------------------------------------------------------------------
// Host-buffer pipelines (compress_host / decompress_host).
//
// A field with natural strides is cut along its slowest axis into chunks of
// whole block layers (contiguous in memory and in block order).  Three streams
// overlap the host->device copy of chunk k+1, the coding of chunk k and the
// device->host copy of chunk k-1's output, so a call takes about as long as
// the larger of its two PCIe transfers instead of their sum.
// ---------------------------------------------------------------------------

// Every word in [wa, wb) assembled from the block slots: each thread finds
// the block holding its word's first bit (binary search over the offsets)
// and gathers from there, like k_pack.
__global__ void __launch_bounds__(256) k_pack_range(PackArgs a, u64 wa, u64 wb) {
  const u64 w = wa + (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= wb) return;
  u64 v = 0;
  u32 fill = 0;
  u64 pos = w << 6;
  if (w == (a.start >> 6)) {
    v = a.init_word;
    fill = (u32)(a.start & 63);
    pos = a.start;
  }
  const u64 rel = pos - a.start;
  u64 lo = 0, hi = a.nblocks;  // largest j with off[j] <= rel
  while (hi - lo > 1) {
    const u64 mid = (lo + hi) >> 1;
    if (a.off[mid] <= rel) lo = mid;
    else hi = mid;
  }
  u64 blk = lo;
  u64 pj = a.start + a.off[blk], qj = a.start + a.off[blk + 1];
  while (fill < 64 && blk < a.nblocks) {
    const u64 local = pos - pj;
    const u64 avail = qj - pos;
    const u32 take = (u32)(avail < (u64)(64 - fill) ? avail : (u64)(64 - fill));
    v |= slot_bits(a.slots + blk * a.slot_words, (u32)local, take) << fill;  // local < a slot
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

namespace {

struct Pipe {
  cudaStream_t in = nullptr, out = nullptr;
  std::vector<cudaEvent_t> ev;
  u64* h_words = nullptr;  // pinned scratch for chunk boundaries
  u64 h_cap = 0;
  cudaEvent_t event(size_t i) {
    while (ev.size() <= i) {
      cudaEvent_t e;
      cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      ev.push_back(e);
    }
    return ev[i];
  }
  bool pinned(u64 n) {
    if (n <= h_cap) return true;
    if (h_words) cudaFreeHost(h_words);
    h_words = nullptr;
    h_cap = 0;
    if (cudaMallocHost((void**)&h_words, n * sizeof(u64)) != cudaSuccess) return false;
    h_cap = n;
    return true;
  }
};
Pipe g_pipe;

bool pipe_streams() {
  if (!g_pipe.in && cudaStreamCreateWithFlags(&g_pipe.in, cudaStreamNonBlocking) != cudaSuccess) return false;
  if (!g_pipe.out && cudaStreamCreateWithFlags(&g_pipe.out, cudaStreamNonBlocking) != cudaSuccess) return false;
  return true;
}

// Chunking of a natural-stride field along its slowest axis.
struct Layers {
  int axis;
  u64 per_layer;   // blocks per block layer
  u64 layers;      // block layers
  u64 per_chunk;   // layers per chunk
  u64 layer_elems; // elements per full block layer (4 rows)
};

Layers layers_of(const Call& c, u64 es) {
  Layers L;
  L.axis = c.dims - 1;
  L.layers = c.f.b[L.axis];
  L.per_layer = c.f.nblocks / L.layers;
  L.layer_elems = 4 * (u64)c.f.s[L.axis];
  const u64 layer_bytes = L.layer_elems * es;
  // Chunks of about 32 MB: swept at 16, 32 and 64 MB on the 512^3 float64
  // end-to-end leg (49.1, 50.05 and 49.5 GB/s): smaller chunks shorten the
  // copy-in of the first chunk and the copy-out of the last, which nothing
  // overlaps, until per-chunk launches and events cost more.
  L.per_chunk = std::max<u64>(1, (32ull << 20) / std::max<u64>(1, layer_bytes));
  return L;
}

// The sub-field of layers [j0, j1).
Call sub_call(const Call& c, const Layers& L, u64 j0, u64 j1) {
  Call s = c;
  const int a = L.axis;
  const u64 rows = std::min<u64>(c.f.n[a], 4 * j1) - 4 * j0;
  s.f.n[a] = rows;
  s.f.b[a] = j1 - j0;
  s.f.nblocks = L.per_layer * (j1 - j0);
  return s;
}

}  // namespace

bool natural_strides(const Call& c) {
  i64 want = 1;
  for (int d = 0; d < c.dims; d++) {
    if (c.f.s[d] != want) return false;
    want *= (i64)c.f.n[d];
  }
  return true;
}

Status compress_host(const Call& call, const void* h_field, void* d_field, u64* h_out, u64* d_out, u64 cap,
                     u64 start, u64 init_word, u64* end_bit, u64* d_offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_mu);
  Workspace& ws = workspace();
  const u64 n = call.f.nblocks;
  const u64 es = (call.type == 1 || call.type == 3) ? 4 : 8;
  if (n == 0 || !natural_strides(call) || !pipe_streams()) return ERR_ARGS;
  const Layers L = layers_of(call, es);
  const u64 nchunks = (L.layers + L.per_chunk - 1) / L.per_chunk;
  const u64 bb = block_bits(call.c, call.type, call.dims);
  const u64 slot_words = (bb + 63) / 64 + 1;
  ZFPB_CHECK(ws.slots.ensure((n * slot_words + 1) * sizeof(u64)));
  ZFPB_CHECK(ws.lengths.ensure(n * sizeof(u32)));
  u64* off = d_offsets;
  if (!off) {
    ZFPB_CHECK(ws.offsets.ensure((n + 1) * sizeof(u64)));
    off = (u64*)ws.offsets.p;
  }
  const u64 chunk_blocks = L.per_chunk * L.per_layer;
  ZFPB_CHECK(ws.partial.ensure(((chunk_blocks + SCAN_TILE - 1) / SCAN_TILE + 1) * sizeof(u64)));
  if (!g_pipe.pinned(nchunks)) return ERR_CUDA;
  // The first block starts at offset 0 (the carry of chunk 0).
  ZFPB_CHECK(cudaMemsetAsync(off, 0, sizeof(u64), s));
  u64 wdone = start >> 6;  // stream words already assembled and copied out
  const u64 total_words_cap = cap;
  Status result = OK;
  auto pack_upto = [&](u64 k, bool last) -> cudaError_t {
    cudaEventSynchronize(g_pipe.event(3 * k + 1));
    const u64 end = start + g_pipe.h_words[k];
    u64 wend = last ? (end + 63) / 64 : end / 64;
    if ((end + 63) / 64 > total_words_cap) {
      result = ERR_OVERFLOW;
      return cudaSuccess;
    }
    if (wend <= wdone) return cudaSuccess;
    PackArgs pa;
    pa.slots = (u64*)ws.slots.p;
    pa.slot_words = slot_words;
    pa.off = off;
    pa.nblocks = std::min<u64>(n, (k + 1) * chunk_blocks);
    pa.start = start;
    pa.init_word = init_word;
    pa.out = d_out;
    {
      KernelTimer t(K_PACK, s);
      k_pack_range<<<(unsigned)((wend - wdone + 255) / 256), 256, 0, s>>>(pa, wdone, wend);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cudaEvent_t ep = g_pipe.event(3 * k + 2);
    cudaEventRecord(ep, s);
    cudaStreamWaitEvent(g_pipe.out, ep, 0);
    e = cudaMemcpyAsync(h_out + wdone, d_out + wdone, (wend - wdone) * 8, cudaMemcpyDeviceToHost, g_pipe.out);
    wdone = wend;
    return e;
  };
  for (u64 k = 0; k < nchunks && result == OK; k++) {
    const u64 j0 = k * L.per_chunk, j1 = std::min(L.layers, j0 + L.per_chunk);
    const u64 e0 = j0 * L.layer_elems;
    const u64 rows = std::min<u64>(call.f.n[L.axis], 4 * j1) - 4 * j0;
    const u64 bytes = rows * (u64)call.f.s[L.axis] * es;
    ZFPB_CHECK(cudaMemcpyAsync((char*)d_field + e0 * es, (const char*)h_field + e0 * es, bytes,
                               cudaMemcpyHostToDevice, g_pipe.in));
    cudaEvent_t ei = g_pipe.event(3 * k);
    ZFPB_CHECK(cudaEventRecord(ei, g_pipe.in));
    ZFPB_CHECK(cudaStreamWaitEvent(s, ei, 0));
    const Call sub = sub_call(call, L, j0, j1);
    const u64 b0 = j0 * L.per_layer;
    EncodeVarArgs ea;
    ea.data = (const char*)d_field + e0 * es;
    ea.f = sub.f;
    ea.c = call.c;
    ea.slots = (u64*)ws.slots.p + b0 * slot_words;
    ea.slot_words = slot_words;
    ea.lengths = (u32*)ws.lengths.p + b0;
    {
      KernelTimer t(K_ENCODE_VAR, s);
      ZFPB_CHECK(for_type(call.type, [&](auto* tp) {
        using T = std::remove_pointer_t<decltype(tp)>;
        return Launch<T>::encode_var(sub, ea, s);
      }));
    }
    ZFPB_CHECK(scan_entries((u32*)ws.lengths.p + b0, sub.f.nblocks, off + b0, (u64*)ws.partial.p, s, off + b0));
    ZFPB_CHECK(cudaMemcpyAsync(g_pipe.h_words + k, off + b0 + sub.f.nblocks, sizeof(u64), cudaMemcpyDeviceToHost, s));
    ZFPB_CHECK(cudaEventRecord(g_pipe.event(3 * k + 1), s));
    if (k > 0) ZFPB_CHECK(pack_upto(k - 1, false));
  }
  if (result == OK) ZFPB_CHECK(pack_upto(nchunks - 1, true));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  ZFPB_CHECK(cudaStreamSynchronize(g_pipe.out));
  ZFPB_CHECK(cudaStreamSynchronize(g_pipe.in));
  if (result != OK) return result;
  *end_bit = start + g_pipe.h_words[nchunks - 1];
  return OK;
}

Status decompress_host(const Call& call, const u64* h_in, u64* d_in, u64 len, u64 start, void* h_field,
                       void* d_field, u64* end_bit, const u64* d_offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(g_mu);
  Workspace& ws = workspace();
  const u64 n = call.f.nblocks;
  const u64 es = (call.type == 1 || call.type == 3) ? 4 : 8;
  const bool fixed = fixed_size_blocks(call);
  if (n == 0 || !natural_strides(call) || (!fixed && !d_offsets) || !pipe_streams()) return ERR_ARGS;
  const Layers L = layers_of(call, es);
  const u64 nchunks = (L.layers + L.per_chunk - 1) / L.per_chunk;
  const u64 chunk_blocks = L.per_chunk * L.per_layer;
  if (!g_pipe.pinned(nchunks + 1)) return ERR_CUDA;
  // Chunk boundaries in the stream.
  for (u64 k = 0; k <= nchunks; k++) {
    const u64 b = std::min(n, k * chunk_blocks);
    if (fixed) g_pipe.h_words[k] = b * (u64)call.c.maxbits;
    else ZFPB_CHECK(cudaMemcpyAsync(g_pipe.h_words + k, d_offsets + b, sizeof(u64), cudaMemcpyDeviceToHost, s));
  }
  ZFPB_CHECK(ws.small.ensure(64));
  unsigned* flags = (unsigned*)ws.small.p;
  ZFPB_CHECK(cudaMemsetAsync(flags, 0, sizeof(unsigned), s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  u64 wcopied = 0;
  for (u64 k = 0; k < nchunks; k++) {
    const u64 j0 = k * L.per_chunk, j1 = std::min(L.layers, j0 + L.per_chunk);
    const u64 e0 = j0 * L.layer_elems;
    // Stream words of the chunk's blocks, and two more (the readers look ahead).
    u64 wb = std::min(len, (start + g_pipe.h_words[k + 1] + 63) / 64 + 2);
    if (wb > wcopied)
      ZFPB_CHECK(cudaMemcpyAsync(d_in + wcopied, h_in + wcopied, (wb - wcopied) * 8, cudaMemcpyHostToDevice,
                                 g_pipe.in));
    wcopied = std::max(wcopied, wb);
    cudaEvent_t ei = g_pipe.event(3 * k);
    ZFPB_CHECK(cudaEventRecord(ei, g_pipe.in));
    ZFPB_CHECK(cudaStreamWaitEvent(s, ei, 0));
    const Call sub = sub_call(call, L, j0, j1);
    const u64 b0 = j0 * L.per_layer;
    DecodeArgs a;
    a.data = (char*)d_field + e0 * es;
    a.f = sub.f;
    a.c = call.c;
    a.stream = d_in;
    a.stream_len = len;
    a.start = fixed ? start + b0 * (u64)call.c.maxbits : start;
    a.offsets = fixed ? nullptr : const_cast<u64*>(d_offsets) + b0;
    a.flags = flags;
    a.owner = nullptr;
    a.imin = 0;
    ZFPB_CHECK(decode_blocks(ws, sub, a, !fixed, s));
    cudaEvent_t ed = g_pipe.event(3 * k + 1);
    ZFPB_CHECK(cudaEventRecord(ed, s));
    ZFPB_CHECK(cudaStreamWaitEvent(g_pipe.out, ed, 0));
    const u64 rows = std::min<u64>(call.f.n[L.axis], 4 * j1) - 4 * j0;
    const u64 bytes = rows * (u64)call.f.s[L.axis] * es;
    ZFPB_CHECK(cudaMemcpyAsync((char*)h_field + e0 * es, (char*)d_field + e0 * es, bytes, cudaMemcpyDeviceToHost,
                               g_pipe.out));
  }
  ZFPB_CHECK(cudaMemcpyAsync(ws.h_pinned, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  ZFPB_CHECK(cudaStreamSynchronize(g_pipe.out));
  ZFPB_CHECK(cudaStreamSynchronize(g_pipe.in));
  const unsigned fl = *(unsigned*)ws.h_pinned;
  *end_bit = start + g_pipe.h_words[nchunks];
  if (fl & FLAG_BAD_INDEX) return ERR_BAD_INDEX;
  return (fl & FLAG_TRUNCATED) ? ERR_TRUNCATED : OK;
}

// ---------------------------------------------------------------------------
// Batches (compress_batch / decompress_batch).
//
// Planning: jobs are cut into tiles of up to 128 consecutive blocks of one
// array and grouped by (type, dims); per class one launch codes all its tiles.
// Scratch (block slots for compress, the plane scratch for 3D decompress) is
// bounded per round, and rounds run back to back on the stream.  A plan keeps
// its tables, scratch and a CUDA graph of its launches; a later call with the
// same jobs replays the graph.  Tuning: the first run of a (pass, type, dims)
// class times its kernel at 32, 64 and 128 threads per CTA (the tiles are the
// same, a CTA's threads take its blocks in turn) and keeps the fastest for
// every later plan.
// ---------------------------------------------------------------------------

static constexpr u32 BATCH_TILE = 128;
static constexpr u64 BATCH_ROUND_BYTES = 8ull << 30;  // slot or plane scratch per round

// A tile of at most STAGE_BLOCKS blocks of one array: the staged pack for
// small slots, else a warp per BW = STAGE_BLOCKS / 8 blocks.
__global__ void __launch_bounds__(256) k_pack_batch(BatchArgs a) {
  constexpr int BW = STAGE_BLOCKS / 8;
  __shared__ union {
    StageSmem stage;
    u32 soff[8][BW + 1];
  } sm;
  const BatchTile t = a.tiles[blockIdx.x];
  const BatchItem* it = a.items + t.item;
  const u64* off = a.offsets + it->len_base;
  const u64 n = it->f.nblocks;
  const u64 delta = 0ull - off[0];  // block offsets relative to the first block
  // The blocks follow the header: from bit it->start, whose word holds the
  // header's last bits (k_batch_ends writes its whole words).
  const u64 start = it->start, init_word = it->hdr[start >> 6];
  if (it->slot_words <= STAGE_SLOT_WORDS) {
    pack_stage(a.slots + it->slot_base, it->slot_words, off, delta + start, n, start, init_word, it->stream,
               it->stream_words, t.first, sm.stage);
  } else {
    const u32 wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 b0 = t.first + (u64)wib * BW;
    if (b0 < t.first + t.count)
      pack_warp<BW>(a.slots + it->slot_base, it->slot_words, off, delta + start, n, start, init_word, it->stream,
                    it->stream_words, b0, sm.soff[wib], lane);
  }
  if (it->index) {
    const u64 e = t.first + t.count;
    for (u64 i = t.first + threadIdx.x; i < e; i += blockDim.x) it->index[i] = off[i] + delta;
    if (e == n && threadIdx.x == 0) it->index[n] = off[n] + delta;
  }
}

// End bit of each item of [first, first + n): compress from the scanned
// lengths; decompress from i * maxbits, the walker's offsets or the index.
// Items with a header: compress writes its whole words (the pack wrote its
// last, partial one with the first blocks); decompress checks the stream
// holds it (else FLAG_BAD_HEADER).
__global__ void k_batch_ends(BatchArgs a, u32 first, u32 n, int compress, u64* ends) {
  const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BatchItem* it = a.items + first + i;
  const u64 nb = it->f.nblocks;
  u64 e;
  if (compress) e = a.offsets[it->len_base + nb] - a.offsets[it->len_base];
  else if (it->fixed) e = nb * (u64)it->c.maxbits;
  else if (it->walk) e = a.offsets[it->len_base + nb];
  else e = it->index[nb];
  ends[first + i] = it->start + e;
  const u64 hw = it->start >> 6, hb = it->start & 63;
  if (compress) {
    for (u64 w = 0; w < hw && w < it->stream_words; w++) it->stream[w] = it->hdr[w];
  } else if (it->start) {
    bool ok = true;
    for (u64 w = 0; w <= hw && w < 3; w++) {
      if (w == hw && hb == 0) break;
      const u64 v = w < it->stream_words ? it->stream[w] : 0ull;
      const u64 m = w < hw ? ~0ull : (1ull << hb) - 1;
      ok = ok && (v & m) == it->hdr[w];
    }
    if (!ok) atomicOr(a.flags + first + i, FLAG_BAD_HEADER);
  }
}

namespace {

enum BatchPass { PASS_ENCODE = 0, PASS_DECODE = 1, PASS_PARSE = 2, PASS_FINISH = 3 };

struct BatchLaunch {
  int pass, type, dims;
  u32 tile0, ntiles;
  int threads;  // 0: tune on first run
};

struct BatchRound {
  u32 item0, nitems;
  std::vector<BatchLaunch> launches;
  u32 ptile0 = 0, nptiles = 0;       // compress: pack tiles
  u64 entries = 0;                   // lengths / offsets entries
  std::vector<std::pair<int, std::pair<u32, u32>>> walks;  // (type*8+dims, (first, count) in walk list)
};

// Pinned host memory, grown on demand.
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    size_t grow = std::max(need, (size_t)4096);
    cudaError_t e = cudaMallocHost(&p, grow);
    if (e == cudaSuccess) bytes = grow;
    return e;
  }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

struct BatchPlan {
  bool compress;
  int device;
  std::vector<char> key;
  std::vector<BatchItem> items;
  std::vector<u32> job_of_item;
  std::vector<BatchTile> tiles;
  std::vector<u32> walk;
  std::vector<BatchRound> rounds;
  u64 max_entries = 0, max_slot_words = 0, max_cols = 0, max_walk = 0;
  Buf d_items, d_tiles, d_walk, slots, lengths, offsets, partial, flags, planes, heads, walk_planes, ends;
  PinnedBuf h_stage, h_ends_buf, h_flags_buf;
  u64* h_ends = nullptr;
  unsigned* h_flags = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool capture_tried = false;
  cudaMemPool_t pool = nullptr;  // set: device buffers grow stream-ordered from this pool
  void reset() {
    items.clear();
    job_of_item.clear();
    tiles.clear();
    walk.clear();
    rounds.clear();
    max_entries = max_slot_words = max_cols = max_walk = 0;
  }
  ~BatchPlan() {
    if (graph) cudaGraphExecDestroy(graph);
    for (Buf* b : {&d_items, &d_tiles, &d_walk, &slots, &lengths, &offsets, &partial, &flags, &planes, &heads,
                   &walk_planes, &ends})
      b->release();
  }
};

std::mutex g_batch_mu;
std::vector<std::unique_ptr<BatchPlan>> g_plans;  // most recently used last
std::mutex g_tune_mu;
std::map<int, int> g_tuned;                          // (pass, type, dims) -> threads

int tune_key(int pass, int type, int dims) { return (pass * 8 + type) * 8 + dims; }

std::vector<int> thread_candidates(int pass, int type, int dims) {
  if (pass == PASS_PARSE || pass == PASS_FINISH) return {128, 64, 32};
  std::vector<int> c;
  for (int th : {128, 64, 32})
    if (plane_bytes(type, dims) * th <= 200 * 1024) c.push_back(th);
  return c;
}

cudaError_t launch_pass(const BatchLaunch& L, const BatchArgs& a0, int threads, cudaStream_t s) {
  BatchArgs a = a0;
  a.tiles = a0.tiles + L.tile0;
  return for_type(L.type, [&](auto* tp) {
    using T = std::remove_pointer_t<decltype(tp)>;
    switch (L.pass) {
      case PASS_ENCODE: return Launch<T>::encode_batch(L.dims, a, L.ntiles, threads, s);
      case PASS_DECODE: return Launch<T>::decode_batch(L.dims, a, L.ntiles, threads, s);
      case PASS_PARSE: return Launch<T>::parse_batch(a, L.ntiles, threads, s);
      default: return Launch<T>::finish_batch(a, L.ntiles, threads, s);
    }
  });
}

int kind_of_pass(int pass) {
  return pass == PASS_ENCODE ? K_ENCODE_VAR : pass == PASS_DECODE ? K_DECODE_VAR : pass == PASS_PARSE ? K_PARSE
                                                                                                        : K_FINISH;
}

// Pick the CTA size of a class by timing each candidate on its real tiles
// (the kernels are idempotent: a rerun writes the same bytes).
cudaError_t tune_launch(const BatchLaunch& L, const BatchArgs& a, cudaStream_t s, int* best) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  *best = 128;
  cudaError_t err = cudaSuccess;
  for (int th : thread_candidates(L.pass, L.type, L.dims)) {
    err = launch_pass(L, a, th, s);  // warm
    if (err != cudaSuccess) break;
    cudaEventRecord(e0, s);
    err = launch_pass(L, a, th, s);
    cudaEventRecord(e1, s);
    if (err != cudaSuccess) break;
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      *best = th;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return err;
}

// Issue every launch of the plan on s (and, when tune is set, tune the
// classes not tuned yet), then copy the ends and flags to pinned memory.
cudaError_t run_plan(BatchPlan& P, cudaStream_t s, bool tune) {
  BatchArgs a{};
  a.items = (const BatchItem*)P.d_items.p;
  a.tiles = (const BatchTile*)P.d_tiles.p;
  a.slots = (u64*)P.slots.p;
  a.lengths = (u32*)P.lengths.p;
  a.offsets = (u64*)P.offsets.p;
  a.flags = (unsigned*)P.flags.p;
  a.planes = (u64*)P.planes.p;
  a.plane_stride = P.max_cols;
  a.heads = (u64*)P.heads.p;
  a.walk_planes = (u64*)P.walk_planes.p;
  const u32 nitems = (u32)P.items.size();
  cudaError_t e = cudaMemsetAsync(P.flags.p, 0, nitems * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  for (BatchRound& R : P.rounds) {
    if (!P.compress) {
      for (auto& w : R.walks) {
        BatchArgs aw = a;
        aw.walk_items = (const u32*)P.d_walk.p + w.second.first;
        aw.nwalk = w.second.second;
        KernelTimer t(K_WALK, s);
        e = for_type(w.first / 8, [&](auto* tp) {
          using T = std::remove_pointer_t<decltype(tp)>;
          return Launch<T>::walk_batch(w.first % 8, aw, s);
        });
        if (e != cudaSuccess) return e;
      }
    }
    for (BatchLaunch& L : R.launches) {
      int th = L.threads;
      if (!th) {
        int known = 0;
        {
          std::lock_guard<std::mutex> l(g_tune_mu);
          auto it = g_tuned.find(tune_key(L.pass, L.type, L.dims));
          if (it != g_tuned.end()) known = it->second;
        }
        if (known) {
          th = known;
        } else if (tune) {
          e = tune_launch(L, a, s, &th);
          if (e != cudaSuccess) return e;
          std::lock_guard<std::mutex> l(g_tune_mu);
          g_tuned[tune_key(L.pass, L.type, L.dims)] = th;
        } else {
          th = thread_candidates(L.pass, L.type, L.dims)[0];
        }
        L.threads = th;
      }
      KernelTimer t(kind_of_pass(L.pass), s);
      e = launch_pass(L, a, th, s);
      if (e != cudaSuccess) return e;
    }
    if (P.compress) {
      e = scan_entries(a.lengths, R.entries, a.offsets, (u64*)P.partial.p, s);
      if (e != cudaSuccess) return e;
      BatchArgs ap = a;
      ap.tiles = a.tiles + R.ptile0;
      {
        KernelTimer t(K_PACK, s);
        k_pack_batch<<<R.nptiles, 256, 0, s>>>(ap);
      }
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    k_batch_ends<<<(R.nitems + 127) / 128, 128, 0, s>>>(a, R.item0, R.nitems, P.compress ? 1 : 0, (u64*)P.ends.p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  e = cudaMemcpyAsync(P.h_ends, P.ends.p, nitems * sizeof(u64), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(P.h_flags, P.flags.p, nitems * sizeof(unsigned), cudaMemcpyDeviceToHost, s);
}

void append_tiles(BatchPlan& P, u32 item, u64 nblocks, u32 size) {
  for (u64 b = 0; b < nblocks; b += size) P.tiles.push_back({item, (u32)std::min<u64>(size, nblocks - b), b});
}

std::vector<char> plan_key(const BatchJob* jobs, size_t n, bool compress, int dev) {
  std::vector<char> k(sizeof(int) * 2 + n * sizeof(BatchJob));
  int hdr[2] = {compress ? 1 : 0, dev};
  memcpy(k.data(), hdr, sizeof(hdr));
  for (size_t i = 0; i < n; i++) {
    BatchJob j = jobs[i];
    j.end_bit = 0;
    j.status = OK;
    memcpy(k.data() + sizeof(hdr) + i * sizeof(BatchJob), &j, sizeof(BatchJob));
  }
  return k;
}

// Build a plan for the jobs that go through the batch kernels (batched[]),
// reusing P's buffers; its tables are copied to the device on s.
cudaError_t build_plan(BatchPlan& P, const BatchJob* jobs, const std::vector<u32>& batched, cudaStream_t s) {
  P.reset();
  auto grow = [&](Buf& b, size_t need) { return P.pool ? b.ensure_on(need, s, P.pool) : b.ensure(need); };
  // Order items by round; within a round, by class, so a class's tiles are contiguous.
  std::vector<std::vector<u32>> rounds;
  {
    std::vector<u32> cur;
    u64 bytes = 0;
    for (u32 j : batched) {
      const Call& c = jobs[j].call;
      u64 need;
      if (P.compress) {
        need = c.f.nblocks * ((block_bits(c.c, c.type, c.dims) + 63) / 64 + 1) * sizeof(u64);
      } else {
        need = c.dims == 3 ? c.f.nblocks * 64 * sizeof(u64) : 0;
      }
      if (!cur.empty() && bytes + need > BATCH_ROUND_BYTES) {
        rounds.push_back(cur);
        cur.clear();
        bytes = 0;
      }
      cur.push_back(j);
      bytes += need;
    }
    if (!cur.empty()) rounds.push_back(cur);
  }
  for (auto& rj : rounds) {
    BatchRound R;
    R.item0 = (u32)P.items.size();
    std::stable_sort(rj.begin(), rj.end(), [&](u32 x, u32 y) {
      return jobs[x].call.type * 8 + jobs[x].call.dims < jobs[y].call.type * 8 + jobs[y].call.dims;
    });
    u64 slot = 0, entries = 0, cols = 0;
    for (u32 j : rj) {
      const BatchJob& J = jobs[j];
      BatchItem it{};
      it.f = J.call.f;
      it.c = J.call.c;
      it.data = J.field;
      it.stream = J.stream;
      it.stream_words = J.stream_words;
      it.index = J.index;
      it.fixed = fixed_size_blocks(J.call) ? 1 : 0;
      it.start = J.start_bit;
      for (int w = 0; w < 3; w++) it.hdr[w] = J.hdr[w];
      it.len_base = entries;
      entries += J.call.f.nblocks + 1;
      if (P.compress) {
        it.slot_words = (block_bits(J.call.c, J.call.type, J.call.dims) + 63) / 64 + 1;
        it.slot_base = slot;
        slot += J.call.f.nblocks * it.slot_words;
      } else {
        it.walk = (!it.fixed && !J.index) ? 1 : 0;
        if (J.call.dims == 3) {
          it.plane_base = cols;
          cols += J.call.f.nblocks;
        }
      }
      P.job_of_item.push_back(j);
      P.items.push_back(it);
    }
    R.nitems = (u32)P.items.size() - R.item0;
    R.entries = entries;
    P.max_entries = std::max(P.max_entries, entries);
    P.max_slot_words = std::max(P.max_slot_words, slot);
    P.max_cols = std::max(P.max_cols, (cols + 31) & ~31ull);
    // Launches per class.
    u32 i = R.item0;
    while (i < R.item0 + R.nitems) {
      const int type = jobs[P.job_of_item[i]].call.type, dims = jobs[P.job_of_item[i]].call.dims;
      u32 e = i;
      while (e < R.item0 + R.nitems && jobs[P.job_of_item[e]].call.type == type &&
             jobs[P.job_of_item[e]].call.dims == dims)
        e++;
      u32 t0 = (u32)P.tiles.size();
      for (u32 k = i; k < e; k++) append_tiles(P, k, P.items[k].f.nblocks, BATCH_TILE);
      u32 nt = (u32)P.tiles.size() - t0;
      if (P.compress) {
        R.launches.push_back({PASS_ENCODE, type, dims, t0, nt, 0});
      } else if (dims == 3) {
        R.launches.push_back({PASS_PARSE, type, dims, t0, nt, 0});
        R.launches.push_back({PASS_FINISH, type, dims, t0, nt, 0});
      } else {
        R.launches.push_back({PASS_DECODE, type, dims, t0, nt, 0});
      }
      if (!P.compress) {
        u32 w0 = (u32)P.walk.size();
        for (u32 k = i; k < e; k++)
          if (P.items[k].walk) P.walk.push_back(k);
        u32 nw = (u32)P.walk.size() - w0;
        if (nw) {
          R.walks.push_back({type * 8 + dims, {w0, nw}});
          P.max_walk = std::max<u64>(P.max_walk, nw);
        }
      }
      i = e;
    }
    if (P.compress) {
      R.ptile0 = (u32)P.tiles.size();
      for (u32 k = R.item0; k < R.item0 + R.nitems; k++) append_tiles(P, k, P.items[k].f.nblocks, STAGE_BLOCKS);
      R.nptiles = (u32)P.tiles.size() - R.ptile0;
    }
    P.rounds.push_back(std::move(R));
  }
  const u64 nitems = P.items.size();
  cudaError_t e;
  if ((e = grow(P.d_items, nitems * sizeof(BatchItem))) != cudaSuccess) return e;
  if ((e = grow(P.d_tiles, std::max<size_t>(1, P.tiles.size()) * sizeof(BatchTile))) != cudaSuccess) return e;
  if ((e = grow(P.flags, nitems * sizeof(unsigned))) != cudaSuccess) return e;
  if ((e = grow(P.ends, nitems * sizeof(u64))) != cudaSuccess) return e;
  if ((e = grow(P.offsets, (P.max_entries + 1) * sizeof(u64))) != cudaSuccess) return e;
  if (P.compress) {
    if ((e = grow(P.slots, (P.max_slot_words + 1) * sizeof(u64))) != cudaSuccess) return e;
    if ((e = grow(P.lengths, (P.max_entries + 1) * sizeof(u32))) != cudaSuccess) return e;
    if ((e = grow(P.partial, ((P.max_entries + SCAN_TILE - 1) / SCAN_TILE + 1) * sizeof(u64))) != cudaSuccess)
      return e;
  } else {
    if (P.max_cols) {
      if ((e = grow(P.planes, 64 * P.max_cols * sizeof(u64))) != cudaSuccess) return e;
      if ((e = grow(P.heads, P.max_cols * sizeof(u64))) != cudaSuccess) return e;
    }
    if (!P.walk.empty()) {
      if ((e = grow(P.d_walk, P.walk.size() * sizeof(u32))) != cudaSuccess) return e;
      if ((e = grow(P.walk_planes, 256 * P.max_walk * sizeof(u64))) != cudaSuccess) return e;
    }
  }
  if ((e = P.h_ends_buf.ensure(nitems * sizeof(u64))) != cudaSuccess) return e;
  if ((e = P.h_flags_buf.ensure(nitems * sizeof(unsigned))) != cudaSuccess) return e;
  P.h_ends = (u64*)P.h_ends_buf.p;
  P.h_flags = (unsigned*)P.h_flags_buf.p;
  // Tables through pinned staging, copied asynchronously on s.
  const size_t bi = nitems * sizeof(BatchItem), bt = P.tiles.size() * sizeof(BatchTile),
               bw = P.walk.size() * sizeof(u32);
  if ((e = P.h_stage.ensure(bi + bt + bw)) != cudaSuccess) return e;
  char* st = (char*)P.h_stage.p;
  memcpy(st, P.items.data(), bi);
  if (bt) memcpy(st + bi, P.tiles.data(), bt);
  if (bw) memcpy(st + bi + bt, P.walk.data(), bw);
  if ((e = cudaMemcpyAsync(P.d_items.p, st, bi, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if (bt && (e = cudaMemcpyAsync(P.d_tiles.p, st + bi, bt, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if (bw && (e = cudaMemcpyAsync(P.d_walk.p, st + bi + bt, bw, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  return cudaSuccess;
}

// Split jobs into those the batch kernels take and those decoded alone:
// fields whose strides alias, and large variable-rate streams without an
// index, whose offsets the single-array decoder finds by the speculative
// parallel walk (the batch walks one thread per stream, about 1.5-3.5 us a
// block).  Empty fields are done.
static constexpr u64 BATCH_WALK_MAX_BLOCKS = 8192;
void classify(BatchJob* jobs, size_t n, bool compress, std::vector<u32>& batched, std::vector<u32>& single) {
  batched.clear();
  single.clear();
  for (size_t i = 0; i < n; i++) {
    BatchJob& J = jobs[i];
    J.status = OK;
    J.end_bit = 0;
    const Call& c = J.call;
    if (c.f.nblocks == 0) continue;
    const bool long_walk = !J.index && !fixed_size_blocks(c) && c.dims <= 3 && c.f.nblocks > BATCH_WALK_MAX_BLOCKS;
    if (!compress && (strides_may_alias(c.f, c.dims) || long_walk)) single.push_back((u32)i);
    else batched.push_back((u32)i);
  }
}

// After the plan's launches completed: each job's end bit and status; jobs
// whose index did not match join `single` to be walked alone.
void collect(const BatchPlan& P, BatchJob* jobs, bool compress, std::vector<u32>& single) {
  for (size_t k = 0; k < P.items.size(); k++) {
    BatchJob& J = jobs[P.job_of_item[k]];
    J.end_bit = P.h_ends[k];
    const unsigned fl = P.h_flags[k];
    if (compress) {
      if ((J.end_bit + 63) / 64 > J.stream_words) J.status = ERR_OVERFLOW;
    } else if (fl & FLAG_BAD_HEADER) {
      J.status = ERR_HEADER;
    } else if (fl & FLAG_BAD_INDEX) {
      single.push_back(P.job_of_item[k]);
    } else if (fl & FLAG_TRUNCATED) {
      J.status = ERR_TRUNCATED;
    }
  }
}

// Whether a job's stream begins with its header (for jobs decoded alone;
// batched ones are checked by k_batch_ends).
static bool header_matches(const BatchJob& J, cudaStream_t s) {
  if (J.start_bit == 0) return true;
  const u64 hw = (J.start_bit + 63) / 64;
  if (hw > J.stream_words) return false;
  u64 w[3] = {0, 0, 0};
  if (cudaMemcpyAsync(w, J.stream, hw * sizeof(u64), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return false;
  if (J.start_bit & 63) w[hw - 1] &= (1ull << (J.start_bit & 63)) - 1;
  for (u64 i = 0; i < hw; i++)
    if (w[i] != J.hdr[i]) return false;
  return true;
}

// Jobs run alone: decompress without an index (compress never needs it).
Status finish_jobs(BatchJob* jobs, size_t n, bool compress, const std::vector<u32>& single, cudaStream_t s) {
  for (u32 i : single) {
    BatchJob& J = jobs[i];
    u64 end = 0;
    Status st;
    if (compress) st = ERR_ARGS;
    else if (!header_matches(J, s)) st = ERR_HEADER;
    else st = decompress(J.call, J.stream, J.stream_words, J.start_bit, J.field, &end, nullptr, s);
    J.status = st;
    J.end_bit = end;
  }
  Status all = OK;
  for (size_t i = 0; i < n; i++)
    if (jobs[i].status != OK) all = jobs[i].status;
  return all;
}

// Run the jobs that the batch kernels can take, through a cached plan.
Status run_batch(BatchJob* jobs, size_t n, bool compress, cudaStream_t s) {
  std::vector<u32> batched, single;
  classify(jobs, n, compress, batched, single);
  if (!batched.empty()) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_batch_mu);
    std::vector<char> key = plan_key(jobs, n, compress, dev);
    BatchPlan* P = nullptr;
    for (size_t i = 0; i < g_plans.size(); i++)
      if (g_plans[i]->key == key) {
        std::unique_ptr<BatchPlan> keep = std::move(g_plans[i]);
        g_plans.erase(g_plans.begin() + i);
        g_plans.push_back(std::move(keep));
        P = g_plans.back().get();
        break;
      }
    if (P && P->graph) {
      if (cudaGraphLaunch(P->graph, s) != cudaSuccess) return ERR_CUDA;
    } else if (P && P->capture_tried) {
      if (run_plan(*P, s, true) != cudaSuccess) return ERR_CUDA;
    } else {
      if (!P) {
        while (g_plans.size() >= 4) g_plans.erase(g_plans.begin());
        auto np = std::make_unique<BatchPlan>();
        np->compress = compress;
        np->device = dev;
        np->key = key;
        if (build_plan(*np, jobs, batched, s) != cudaSuccess) {
          cudaGetLastError();
          return ERR_CUDA;
        }
        g_plans.push_back(std::move(np));
        P = g_plans.back().get();
      }
      if (run_plan(*P, s, true) != cudaSuccess) return ERR_CUDA;
      if (cudaStreamSynchronize(s) != cudaSuccess) return ERR_CUDA;
      // Capture the launches for the next call with the same jobs (once: a
      // stream that cannot be captured, like the legacy default stream, runs
      // the launches directly every time).
      cudaGraph_t g = nullptr;
      P->capture_tried = true;
      g_no_timers = true;
      bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        cudaError_t re = run_plan(*P, s, false);
        ok = cudaStreamEndCapture(s, &g) == cudaSuccess && re == cudaSuccess && g;
      }
      g_no_timers = false;
      if (ok && cudaGraphInstantiate(&P->graph, g, 0) != cudaSuccess) P->graph = nullptr;
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return ERR_CUDA;
    collect(*P, jobs, compress, single);
  }
  return finish_jobs(jobs, n, compress, single, s);
}

}  // namespace

Status compress_batch(BatchJob* jobs, size_t n, cudaStream_t s) { return run_batch(jobs, n, true, s); }
Status decompress_batch(BatchJob* jobs, size_t n, cudaStream_t s) { return run_batch(jobs, n, false, s); }

u64 batch_scratch_bytes(const Call& c, bool compress) {
  const u64 n = c.f.nblocks;
  if (compress) return n * ((block_bits(c.c, c.type, c.dims) + 63) / 64 + 1) * sizeof(u64) + (n + 1) * 12;
  return (c.dims == 3 ? n * 65 * sizeof(u64) : 0) + (n + 1) * sizeof(u64);
}

// Asynchronous batches (the serving loop): plan on the host, launch on s,
// return; the caller polls batch_ready and then calls batch_collect.  No
// tuning (classes use the CTA sizes tuned so far, else 128 threads) and no
// graph: each run is a different set of requests.
struct BatchRun {
  BatchPlan plan;
  std::vector<BatchJob> jobs;
  std::vector<u32> batched, single;
  bool compress = true;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool launched = false;
};

// The memory pool of asynchronous batch scratch, one per device: it keeps
// what it has mapped (release threshold at its maximum), so scratch that a
// run frees and the next run takes again is not unmapped and mapped anew.
static cudaMemPool_t batch_pool() {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> l(mu);
  auto it = pools.find(dev);
  if (it != pools.end()) return it->second;
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  unsigned long long keep = ~0ull;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[dev] = pool;
  return pool;
}

bool batch_reserve(u64 bytes, cudaStream_t s) {
  cudaMemPool_t pool = batch_pool();
  void* p = nullptr;
  if (!pool || cudaMallocFromPoolAsync(&p, bytes, pool, s) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cudaFreeAsync(p, s) == cudaSuccess;
}

BatchRun* batch_run_create() {
  BatchRun* r = new BatchRun();
  r->plan.pool = batch_pool();
  if (!r->plan.pool) {
    delete r;
    return nullptr;
  }
  r->plan.h_stage.ensure(1 << 20);
  r->plan.h_ends_buf.ensure(1 << 16);
  r->plan.h_flags_buf.ensure(1 << 16);
  if (cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming) != cudaSuccess) {
    delete r;
    return nullptr;
  }
  return r;
}

void batch_run_destroy(BatchRun* r) {
  if (!r) return;
  if (r->launched) cudaEventSynchronize(r->done);
  if (r->stream) cudaStreamSynchronize(r->stream);
  cudaEventDestroy(r->done);
  delete r;
}

Status batch_launch(BatchRun* r, const BatchJob* jobs, size_t n, bool compress, cudaStream_t s) {
  r->jobs.assign(jobs, jobs + n);
  r->compress = compress;
  r->stream = s;
  r->plan.compress = compress;
  classify(r->jobs.data(), n, compress, r->batched, r->single);
  if (!r->batched.empty()) {
    if (build_plan(r->plan, r->jobs.data(), r->batched, s) != cudaSuccess) return ERR_CUDA;
    if (run_plan(r->plan, s, false) != cudaSuccess) return ERR_CUDA;
  }
  if (cudaEventRecord(r->done, s) != cudaSuccess) return ERR_CUDA;
  r->launched = true;
  return OK;
}

bool batch_ready(BatchRun* r) { return !r->launched || cudaEventQuery(r->done) != cudaErrorNotReady; }

Status batch_collect(BatchRun* r, BatchJob* out) {
  if (!r->launched) return ERR_ARGS;
  if (cudaEventSynchronize(r->done) != cudaSuccess) return ERR_CUDA;
  r->launched = false;
  if (!r->batched.empty()) collect(r->plan, r->jobs.data(), r->compress, r->single);
  Status st = finish_jobs(r->jobs.data(), r->jobs.size(), r->compress, r->single, r->stream);
  if (!r->single.empty()) cudaStreamSynchronize(r->stream);
  std::copy(r->jobs.begin(), r->jobs.end(), out);
  return st;
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
  k_scan_partials<<<1, 1024, 0, s>>>(part, tiles, off + n, nullptr);
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
  ZFPB_CHECK(launch_pack(pa, call.dims, s));
  ZFPB_CHECK(cudaStreamSynchronize(s));
  return OK;
}

}  // namespace zfpb
