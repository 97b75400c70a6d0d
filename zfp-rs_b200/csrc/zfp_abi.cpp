// The zfp.h C ABI over the CUDA engine.
//
// Host-side parts follow zfp-rs 1.0.1 and its C ABI crate zfp-rs-ffi:
//   bit streams          zfp-rs-ffi/src/bitstream.rs:168-668, src/bitstream/core.rs
//   fields               zfp-rs-ffi/src/field.rs:126-480, src/field.rs:541-735
//   configs and modes    zfp-rs-ffi/src/header.rs:60-140, src/config.rs:85-686
//   streams, headers     zfp-rs-ffi/src/stream.rs, src/header.rs:72-173
//   compress/decompress  zfp-rs-ffi/src/stream.rs:321-367
// zfp_compress and zfp_decompress run on the GPU (zfpb_engine.cu); host
// buffers are staged through device memory.  There is no CPU codec here.

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/zfp.h"
#include "../../include/zfp_b200.h"
#include "../../include/zfp_block.h"
#include "zfpb_engine.h"
#include "zfpb_serve.h"

using zfpb::u32;
using zfpb::u64;

extern "C" {
const size_t stream_word_bits = 64;
const uint32_t zfp_codec_version = ZFP_CODEC;
const uint32_t zfp_library_version = ZFP_VERSION;
}

static thread_local int g_last_error = 0;

// ---------------------------------------------------------------------------
// Memory kinds
// ---------------------------------------------------------------------------

static bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------------------
// Bit streams: zfp-rs src/bitstream/core.rs semantics on 64-bit words that
// may live in host or device memory.
// ---------------------------------------------------------------------------

struct IndexCache {
  u64* d_off = nullptr;   // nblocks + 1 offsets relative to `start`
  size_t cap = 0;         // entries allocated
  bool valid = false;
  u64 start = 0, nblocks = 0;
  u64 end = 0;            // stream bit after the last block
  int type = 0, dims = 0;
  zfpb::CodecParams c{};
};

struct bitstream {
  u64* words = nullptr;
  size_t len = 0;      // capacity in words
  bool owned = false;  // words allocated here (host)
  bool device = false;
  size_t word_pos = 0;
  u64 buffer = 0;
  u32 bits = 0;
  bool overflowed = false;
  bool overread = false;
  size_t seek_word = 0;
  IndexCache index;
};

static u64 get_word(const bitstream* s, size_t i) {
  if (!s->device) return s->words[i];
  u64 v = 0;
  cudaMemcpy(&v, s->words + i, sizeof(u64), cudaMemcpyDeviceToHost);
  return v;
}
static void set_word(bitstream* s, size_t i, u64 v) {
  if (!s->device)
    s->words[i] = v;
  else
    cudaMemcpy(s->words + i, &v, sizeof(u64), cudaMemcpyHostToDevice);
}

static u64 read_word_raw(bitstream* s) {
  u64 w = s->word_pos < s->len ? get_word(s, s->word_pos) : 0;
  s->word_pos++;
  return w;
}
static void write_word_raw(bitstream* s, u64 v) {
  if (s->word_pos < s->len)
    set_word(s, s->word_pos, v);
  else
    s->overflowed = true;
  s->word_pos++;
}

static u64 bs_read_bits(bitstream* s, u32 n) {
  if (n > 64) n = 64;
  u64 value = s->buffer;
  if (s->bits < n) {
    u64 w = read_word_raw(s);
    s->buffer = w;
    value += w << s->bits;
    s->bits += 64;
    s->bits -= n;
    if (s->bits == 0) {
      s->buffer = 0;
    } else {
      s->buffer >>= (64 - s->bits);
      if (n < 64) value &= (2ull << (n - 1)) - 1;
    }
  } else {
    s->bits -= n;
    s->buffer = n < 64 ? s->buffer >> n : 0;
    if (n < 64) value &= (1ull << n) - 1;
  }
  return value;
}

static u64 bs_write_bits(bitstream* s, u64 value, u32 n) {
  if (n > 64) n = 64;
  s->buffer += value << s->bits;
  s->bits += n;
  if (s->bits >= 64) {
    u64 val = value >> 1;
    u32 remaining = n - 1;
    for (;;) {
      u32 after = s->bits - 64;
      u64 buf = s->buffer;
      s->bits = after;
      write_word_raw(s, buf);
      s->buffer = val >> (remaining - after);
      if (s->bits < 64) break;
    }
  }
  if (s->bits < 64) s->buffer &= (1ull << s->bits) - 1;
  return n < 64 ? value >> n : 0;
}

static bool loaded_since_seek(const bitstream* s) {
  size_t m = s->len > s->seek_word ? s->len : s->seek_word;
  return s->word_pos > m;
}

static void bs_seek_read(bitstream* s, u64 offset) {
  u32 n = (u32)(offset % 64);
  s->overread |= loaded_since_seek(s);
  s->word_pos = (size_t)(offset / 64);
  s->seek_word = s->word_pos;
  if (n) {
    u64 w = read_word_raw(s);
    s->buffer = w >> n;
    s->bits = 64 - n;
  } else {
    s->buffer = 0;
    s->bits = 0;
  }
}

static void bs_seek_write(bitstream* s, u64 offset) {
  u32 n = (u32)(offset % 64);
  s->word_pos = (size_t)(offset / 64);
  s->overflowed = false;
  if (n) {
    s->buffer = s->word_pos < s->len ? (get_word(s, s->word_pos) & ((1ull << n) - 1)) : 0;
    s->bits = n;
  } else {
    s->buffer = 0;
    s->bits = 0;
  }
}

static u64 bs_wtell(const bitstream* s) { return (u64)s->word_pos * 64 + s->bits; }
static u64 bs_rtell(const bitstream* s) { return (u64)s->word_pos * 64 - s->bits; }

static void bs_pad(bitstream* s, u64 n) {
  u64 bits = (u64)s->bits + n;
  while (bits >= 64) {
    if (s->word_pos >= s->len) {
      s->word_pos += (size_t)(bits / 64);
      s->buffer = 0;
      s->overflowed = true;
      bits %= 64;
      break;
    }
    write_word_raw(s, s->buffer);
    s->buffer = 0;
    bits -= 64;
  }
  s->bits = (u32)bits;
}

static u32 bs_flush(bitstream* s) {
  u32 p = (64 - s->bits) % 64;
  if (p) bs_pad(s, p);
  return p;
}

static u32 bs_align(bitstream* s) {
  u32 b = s->bits;
  if (b) bs_seek_read(s, bs_rtell(s) + b);
  return b;
}

static void bs_rewind(bitstream* s) {
  s->word_pos = 0;
  s->buffer = 0;
  s->bits = 0;
  s->overflowed = false;
  s->overread = false;
  s->seek_word = 0;
}

extern "C" {

bitstream* stream_open(void* buffer, size_t bytes) {
  bitstream* s = new (std::nothrow) bitstream();
  if (!s) return nullptr;
  if (buffer == nullptr) {
    s->len = (bytes + 7) / 8;
    s->words = (u64*)calloc(s->len ? s->len : 1, sizeof(u64));
    if (!s->words) {
      delete s;
      return nullptr;
    }
    s->owned = true;
  } else if (((uintptr_t)buffer % 8) != 0) {
    // A misaligned buffer is copied (zfp-rs-ffi/src/bitstream.rs:184-189).
    s->len = (bytes + 7) / 8;
    s->words = (u64*)calloc(s->len ? s->len : 1, sizeof(u64));
    if (!s->words) {
      delete s;
      return nullptr;
    }
    s->owned = true;
    if (is_device_ptr(buffer))
      cudaMemcpy(s->words, buffer, bytes, cudaMemcpyDeviceToHost);
    else
      memcpy(s->words, buffer, bytes);
  } else {
    s->words = (u64*)buffer;
    s->len = bytes / 8;
    s->device = is_device_ptr(buffer);
  }
  return s;
}

void stream_close(bitstream* s) {
  if (!s) return;
  if (s->owned) free(s->words);
  if (s->index.d_off) cudaFree(s->index.d_off);
  delete s;
}

bitstream* stream_clone(const bitstream* s) {
  if (!s) return nullptr;
  size_t committed = s->word_pos < s->len ? s->word_pos : s->len;
  bitstream* c = new (std::nothrow) bitstream();
  if (!c) return nullptr;
  c->len = committed;
  c->words = (u64*)calloc(committed ? committed : 1, sizeof(u64));
  c->owned = true;
  if (committed) {
    if (s->device)
      cudaMemcpy(c->words, s->words, committed * 8, cudaMemcpyDeviceToHost);
    else
      memcpy(c->words, s->words, committed * 8);
  }
  return c;
}

bitstream_count stream_alignment(void) { return 8; }
void* stream_data(const bitstream* s) { return s ? (void*)s->words : nullptr; }
size_t stream_size(const bitstream* s) { return s ? s->word_pos * 8 : 0; }
size_t stream_capacity(const bitstream* s) { return s ? s->len * 8 : 0; }
size_t stream_stride_block(const bitstream*) { return 8; }
ptrdiff_t stream_stride_delta(const bitstream*) { return -8; }

uint stream_read_bit(bitstream* s) {
  if (!s) return 0;
  if (s->bits == 0) {
    s->buffer = read_word_raw(s);
    s->bits = 64;
  }
  s->bits--;
  uint b = (uint)(s->buffer & 1);
  s->buffer >>= 1;
  return b;
}

uint stream_write_bit(bitstream* s, uint bit) {
  if (!s) return 0;
  s->buffer += (u64)(bit & 1) << s->bits;
  s->bits++;
  if (s->bits == 64) {
    write_word_raw(s, s->buffer);
    s->buffer = 0;
    s->bits = 0;
  }
  return bit;
}

uint64 stream_read_bits(bitstream* s, bitstream_count n) {
  return s ? bs_read_bits(s, n > 0xffffffffu ? 0xffffffffu : (u32)n) : 0;
}
uint64 stream_write_bits(bitstream* s, uint64 v, bitstream_count n) {
  return s ? bs_write_bits(s, v, n > 0xffffffffu ? 0xffffffffu : (u32)n) : 0;
}
bitstream_offset stream_rtell(const bitstream* s) { return s ? bs_rtell(s) : 0; }
bitstream_offset stream_wtell(const bitstream* s) { return s ? bs_wtell(s) : 0; }
void stream_rewind(bitstream* s) {
  if (s) bs_rewind(s);
}
void stream_rseek(bitstream* s, bitstream_offset o) {
  if (s) bs_seek_read(s, o);
}
void stream_wseek(bitstream* s, bitstream_offset o) {
  if (s) bs_seek_write(s, o);
}
void stream_skip(bitstream* s, bitstream_size n) {
  if (s) bs_seek_read(s, bs_rtell(s) + n);
}
void stream_pad(bitstream* s, bitstream_size n) {
  if (s) bs_pad(s, n);
}
bitstream_count stream_align(bitstream* s) { return s ? bs_align(s) : 0; }
bitstream_count stream_flush(bitstream* s) { return s ? bs_flush(s) : 0; }

// core.rs:490-522
void stream_copy(bitstream* dst, bitstream* src, bitstream_size n) {
  if (!dst || !src) return;
  u64 remaining = n;
  while (remaining > 64) {
    bool src_done = src->word_pos >= src->len && src->buffer == 0;
    bool dst_done = dst->word_pos >= dst->len;
    if (src_done && dst_done) {
      u64 skipped = (remaining - 1) / 64;
      src->word_pos += (size_t)skipped;
      dst->word_pos += (size_t)skipped;
      dst->buffer = 0;
      dst->overflowed = true;
      remaining -= skipped * 64;
      break;
    }
    u64 w = bs_read_bits(src, 64);
    bs_write_bits(dst, w, 64);
    remaining -= 64;
  }
  if (remaining > 0) {
    u64 w = bs_read_bits(src, (u32)remaining);
    bs_write_bits(dst, w, (u32)remaining);
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Fields (zfp-rs src/field.rs:541-735)
// ---------------------------------------------------------------------------

static size_t type_size(zfp_type t) {
  return (t == zfp_type_int32 || t == zfp_type_float) ? 4 : (t == zfp_type_int64 || t == zfp_type_double) ? 8 : 0;
}

struct Plan {
  int dims = 0;
  size_t n[4] = {0, 0, 0, 0};
  ptrdiff_t s[4] = {0, 0, 0, 0};  // effective
  size_t nblocks = 0, nelems = 0;
  ptrdiff_t imin = 0, imax = 0;  // element index span
  size_t span_bytes = 0;
  bool contiguous = false;
};

static int dims_of(const zfp_field* f) {
  return f->ny == 0 ? 1 : f->nz == 0 ? 2 : f->nw == 0 ? 3 : 4;
}

static bool plan_field(const zfp_field* f, Plan& p) {
  if (type_size(f->type) == 0) return false;
  p.dims = dims_of(f);
  size_t n[4] = {f->nx, f->ny, f->nz, f->nw};
  ptrdiff_t st[4] = {f->sx, f->sy, f->sz, f->sw};
  size_t nat = 1;
  bool nat_ok = true;
  p.nelems = 1;
  p.nblocks = 1;
  for (int i = 0; i < 4; i++) {
    p.n[i] = i < p.dims ? n[i] : 0;
    if (i < p.dims) {
      if (__builtin_mul_overflow(p.nelems, n[i], &p.nelems)) return false;
      if (__builtin_mul_overflow(p.nblocks, (n[i] + 3) / 4, &p.nblocks)) return false;
    }
    p.s[i] = st[i] != 0 ? st[i] : (nat_ok ? (ptrdiff_t)nat : PTRDIFF_MAX);
    if (i < p.dims && __builtin_mul_overflow(nat, n[i], &nat)) nat_ok = false;
  }
  if (p.nelems > (size_t)PTRDIFF_MAX) return false;
  p.imin = p.imax = 0;
  for (int i = 0; i < p.dims; i++) {
    if (p.n[i] == 0) continue;
    ptrdiff_t ext;
    if (__builtin_mul_overflow(p.s[i], (ptrdiff_t)(p.n[i] - 1), &ext)) return false;
    if (ext < 0) p.imin += ext; else p.imax += ext;
  }
  size_t span = (size_t)(p.imax - p.imin) + 1;
  if (__builtin_mul_overflow(span, type_size(f->type), &p.span_bytes)) return false;
  p.contiguous = true;
  size_t natural = 1;
  for (int i = 0; i < p.dims; i++) {
    if (p.s[i] != (ptrdiff_t)natural) p.contiguous = false;
    natural *= p.n[i];
  }
  return true;
}

static bool valid_dims(const zfp_field* f) {
  size_t n[4] = {f->nx, f->ny, f->nz, f->nw};
  if (n[0] == 0) return false;
  bool zero = false;
  for (int i = 1; i < 4; i++) {
    if (n[i] == 0) zero = true;
    else if (zero) return false;
  }
  return true;
}

static uint64 field_metadata(zfp_type t, const size_t* n, int d) {
  uint64 meta = 0;
  u32 width = 48 / d;
  uint64 maxenc = (1ull << width) - 1;
  u32 shift = 0;
  for (int i = 0; i < d; i++) {
    uint64 e = (uint64)n[i] - 1;
    if (n[i] == 0 || e > maxenc) return ZFP_META_NULL;
    meta |= e << shift;
    shift += width;
  }
  meta = (meta << 2) | (uint64)(d - 1);
  meta = (meta << 2) | (uint64)(t - 1);
  return meta;
}

static bool decode_metadata(uint64 meta, zfp_type* t, size_t* n) {
  if (meta >> 52) return false;
  *t = (zfp_type)((meta & 3) + 1);
  uint64 m = meta >> 2;
  int d = (int)(m & 3) + 1;
  m >>= 2;
  u32 width = 48 / d;
  uint64 mask = (1ull << width) - 1;
  for (int i = 0; i < 4; i++) n[i] = 0;
  for (int i = 0; i < d; i++) {
    n[i] = (size_t)((m & mask) + 1);
    m >>= width;
  }
  return true;
}

extern "C" {

zfp_field* zfp_field_alloc(void) {
  zfp_field* f = (zfp_field*)calloc(1, sizeof(zfp_field));
  return f;
}
static zfp_field* field_new(void* data, zfp_type t, size_t nx, size_t ny, size_t nz, size_t nw) {
  zfp_field* f = zfp_field_alloc();
  if (!f) return nullptr;
  f->type = t;
  f->nx = nx;
  f->ny = ny;
  f->nz = nz;
  f->nw = nw;
  f->data = data;
  return f;
}
zfp_field* zfp_field_1d(void* d, zfp_type t, size_t nx) { return field_new(d, t, nx, 0, 0, 0); }
zfp_field* zfp_field_2d(void* d, zfp_type t, size_t nx, size_t ny) { return field_new(d, t, nx, ny, 0, 0); }
zfp_field* zfp_field_3d(void* d, zfp_type t, size_t nx, size_t ny, size_t nz) {
  return field_new(d, t, nx, ny, nz, 0);
}
zfp_field* zfp_field_4d(void* d, zfp_type t, size_t nx, size_t ny, size_t nz, size_t nw) {
  return field_new(d, t, nx, ny, nz, nw);
}
void zfp_field_free(zfp_field* f) { free(f); }
void* zfp_field_pointer(const zfp_field* f) { return f ? f->data : nullptr; }
void* zfp_field_begin(const zfp_field* f) {
  if (!f || !f->data) return nullptr;
  Plan p;
  if (!plan_field(f, p)) return nullptr;
  return (char*)f->data + p.imin * (ptrdiff_t)type_size(f->type);
}
zfp_type zfp_field_type(const zfp_field* f) { return f ? f->type : zfp_type_none; }
uint zfp_field_precision(const zfp_field* f) {
  return (f && type_size(f->type)) ? (uint)(8 * type_size(f->type)) : 0;
}
uint zfp_field_dimensionality(const zfp_field* f) {
  if (!f) return 0;
  Plan p;
  return plan_field(f, p) ? (uint)p.dims : 0;
}
size_t zfp_field_size(const zfp_field* f, size_t* dims) {
  if (!f) return 0;
  if (dims) {
    dims[0] = f->nx;
    dims[1] = f->ny;
    dims[2] = f->nz;
    dims[3] = f->nw;
  }
  Plan p;
  return plan_field(f, p) ? p.nelems : 0;
}
size_t zfp_field_size_bytes(const zfp_field* f) {
  if (!f) return 0;
  Plan p;
  return plan_field(f, p) ? p.span_bytes : 0;
}
size_t zfp_field_blocks(const zfp_field* f) {
  if (!f) return 0;
  Plan p;
  return plan_field(f, p) ? p.nblocks : 0;
}
zfp_bool zfp_field_stride(const zfp_field* f, ptrdiff_t* strides) {
  if (!f) return zfp_false;
  if (strides) {
    strides[0] = f->sx;
    strides[1] = f->sy;
    strides[2] = f->sz;
    strides[3] = f->sw;
  }
  Plan p;
  return (plan_field(f, p) && p.contiguous) ? zfp_false : zfp_true;
}
zfp_bool zfp_field_is_contiguous(const zfp_field* f) {
  if (!f) return zfp_false;
  Plan p;
  return (plan_field(f, p) && p.contiguous) ? zfp_true : zfp_false;
}
uint64 zfp_field_metadata(const zfp_field* f) {
  if (!f) return 0;
  if (!type_size(f->type) || !valid_dims(f)) return ZFP_META_NULL;
  size_t n[4] = {f->nx, f->ny, f->nz, f->nw};
  return field_metadata(f->type, n, dims_of(f));
}
void zfp_field_set_pointer(zfp_field* f, void* p) {
  if (f) f->data = p;
}
zfp_type zfp_field_set_type(zfp_field* f, zfp_type t) {
  if (!f) return zfp_type_int32;
  if (!type_size(t)) return zfp_type_none;
  f->type = t;
  return t;
}
void zfp_field_set_size_1d(zfp_field* f, size_t nx) {
  if (f) { f->nx = nx; f->ny = 0; f->nz = 0; f->nw = 0; }
}
void zfp_field_set_size_2d(zfp_field* f, size_t nx, size_t ny) {
  if (f) { f->nx = nx; f->ny = ny; f->nz = 0; f->nw = 0; }
}
void zfp_field_set_size_3d(zfp_field* f, size_t nx, size_t ny, size_t nz) {
  if (f) { f->nx = nx; f->ny = ny; f->nz = nz; f->nw = 0; }
}
void zfp_field_set_size_4d(zfp_field* f, size_t nx, size_t ny, size_t nz, size_t nw) {
  if (f) { f->nx = nx; f->ny = ny; f->nz = nz; f->nw = nw; }
}
void zfp_field_set_stride_1d(zfp_field* f, ptrdiff_t sx) {
  if (f) { f->sx = sx; f->sy = 0; f->sz = 0; f->sw = 0; }
}
void zfp_field_set_stride_2d(zfp_field* f, ptrdiff_t sx, ptrdiff_t sy) {
  if (f) { f->sx = sx; f->sy = sy; f->sz = 0; f->sw = 0; }
}
void zfp_field_set_stride_3d(zfp_field* f, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz) {
  if (f) { f->sx = sx; f->sy = sy; f->sz = sz; f->sw = 0; }
}
void zfp_field_set_stride_4d(zfp_field* f, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw) {
  if (f) { f->sx = sx; f->sy = sy; f->sz = sz; f->sw = sw; }
}
zfp_bool zfp_field_set_metadata(zfp_field* f, uint64 meta) {
  if (!f) return zfp_false;
  zfp_type t;
  size_t n[4];
  if (!decode_metadata(meta, &t, n)) return zfp_false;
  f->type = t;
  f->nx = n[0]; f->ny = n[1]; f->nz = n[2]; f->nw = n[3];
  f->sx = f->sy = f->sz = f->sw = 0;
  return zfp_true;
}

// ---------------------------------------------------------------------------
// Configs (zfp-rs-ffi/src/header.rs:60-140)
// ---------------------------------------------------------------------------

zfp_config zfp_config_none(void) {
  zfp_config c;
  memset(&c, 0, sizeof(c));
  c.mode = zfp_mode_null;
  return c;
}
zfp_config zfp_config_rate(double rate, zfp_bool align) {
  zfp_config c = zfp_config_none();
  c.mode = zfp_mode_fixed_rate;
  c.arg.rate = (align == zfp_false && rate >= 0.0) ? -rate : rate;
  return c;
}
zfp_config zfp_config_precision(uint32_t p) {
  zfp_config c = zfp_config_none();
  c.mode = zfp_mode_fixed_precision;
  c.arg.precision = p;
  return c;
}
zfp_config zfp_config_accuracy(double t) {
  zfp_config c = zfp_config_none();
  c.mode = zfp_mode_fixed_accuracy;
  c.arg.tolerance = t;
  return c;
}
zfp_config zfp_config_reversible(void) {
  zfp_config c = zfp_config_none();
  c.mode = zfp_mode_reversible;
  return c;
}
zfp_config zfp_config_expert(uint32_t minbits, uint32_t maxbits, uint32_t maxprec, int32_t minexp) {
  zfp_config c = zfp_config_none();
  c.mode = zfp_mode_expert;
  c.arg.expert.minbits = minbits;
  c.arg.expert.maxbits = maxbits;
  c.arg.expert.maxprec = maxprec;
  c.arg.expert.minexp = minexp;
  return c;
}

size_t zfp_type_size(zfp_type t) { return type_size(t); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Streams and modes (zfp-rs src/config.rs, zfp-rs-ffi/src/stream.rs)
// ---------------------------------------------------------------------------

struct zfp_exec_params_omp {
  uint threads;
  uint chunk_size;
};

// zfp_stream_open allocates this; the public struct comes first.
struct StreamExt {
  zfp_stream pub;
  int rounding;  // 0 never, 1 first, 2 last
  int tight;
};
static StreamExt* ext_of(zfp_stream* s) { return reinterpret_cast<StreamExt*>(s); }
static const StreamExt* ext_of(const zfp_stream* s) { return reinterpret_cast<const StreamExt*>(s); }

static bool valid_params(u32 minb, u32 maxb, u32 maxp) { return minb <= maxb && maxp > 0 && maxp <= 64; }

static zfp_mode mode_of(u32 minb, u32 maxb, u32 maxp, int32_t mine) {
  if (!valid_params(minb, maxb, maxp)) return zfp_mode_null;
  if (minb == ZFP_MIN_BITS && maxb == ZFP_MAX_BITS && maxp == ZFP_MAX_PREC && mine == ZFP_MIN_EXP)
    return zfp_mode_expert;
  if (minb == maxb && maxb >= 1 && maxb <= ZFP_MAX_BITS && maxp >= ZFP_MAX_PREC && mine == ZFP_MIN_EXP)
    return zfp_mode_fixed_rate;
  if (minb <= ZFP_MIN_BITS && maxb >= ZFP_MAX_BITS && maxp >= 1 && mine == ZFP_MIN_EXP)
    return zfp_mode_fixed_precision;
  if (minb <= ZFP_MIN_BITS && maxb >= ZFP_MAX_BITS && maxp >= ZFP_MAX_PREC && mine >= ZFP_MIN_EXP)
    return zfp_mode_fixed_accuracy;
  if (minb <= ZFP_MIN_BITS && maxb >= ZFP_MAX_BITS && maxp >= ZFP_MAX_PREC && mine < ZFP_MIN_EXP)
    return zfp_mode_reversible;
  return zfp_mode_expert;
}
static zfp_mode mode_of(const zfp_stream* s) { return mode_of(s->minbits, s->maxbits, s->maxprec, s->minexp); }

static uint64 encode_expert_mode(u32 minb, u32 maxb, u32 maxp, int32_t mine) {
  auto clampu = [](u32 v, u32 lo, u32 hi) { return v < lo ? lo : v > hi ? hi : v; };
  uint64 a = clampu(minb, 1, 0x8000) - 1, b = clampu(maxb, 1, 0x8000) - 1, p = clampu(maxp, 1, 0x80) - 1;
  int64_t e = (int64_t)mine + 16495;
  e = e < 0 ? 0 : e > 0x7fff ? 0x7fff : e;
  uint64 m = 0;
  m = (m << 15) | (uint64)e;
  m = (m << 7) | p;
  m = (m << 15) | b;
  m = (m << 15) | a;
  m = (m << 12) | 0xfffu;
  return m;
}

static uint64 mode_bits(const zfp_stream* s) {
  zfp_mode m = mode_of(s);
  if (m == zfp_mode_fixed_rate && s->maxbits <= 2048) return s->maxbits - 1;
  if (m == zfp_mode_fixed_precision && s->maxprec <= 128) return (uint64)(s->maxprec - 1) + 2048;
  if (m == zfp_mode_reversible) return 2048 + 128;
  if (m == zfp_mode_fixed_accuracy && s->minexp <= 843) return (uint64)(s->minexp - ZFP_MIN_EXP) + (2048 + 128 + 1);
  return encode_expert_mode(s->minbits, s->maxbits, s->maxprec, s->minexp);
}

// config.rs:215-247; false for an invalid mode.
static bool params_of_mode(uint64 mode, u32* minb, u32* maxb, u32* maxp, int32_t* mine) {
  if (mode <= ZFP_MODE_SHORT_MAX) {
    if (mode < 2048) { *minb = *maxb = (u32)mode + 1; *maxp = 64; *mine = ZFP_MIN_EXP; }
    else if (mode < 2048 + 128) { *minb = 1; *maxb = ZFP_MAX_BITS; *maxp = (u32)mode + 1 - 2048; *mine = ZFP_MIN_EXP; }
    else if (mode == 2048 + 128) { *minb = 1; *maxb = ZFP_MAX_BITS; *maxp = 64; *mine = ZFP_MIN_EXP - 1; }
    else { *minb = 1; *maxb = ZFP_MAX_BITS; *maxp = 64; *mine = (int32_t)mode + ZFP_MIN_EXP - (2048 + 128 + 1); }
  } else {
    uint64 m = mode >> 12;
    *minb = (u32)(m & 0x7fff) + 1; m >>= 15;
    *maxb = (u32)(m & 0x7fff) + 1; m >>= 15;
    *maxp = (u32)(m & 0x7f) + 1; m >>= 7;
    *mine = (int32_t)(m & 0x7fff) - 16495;
  }
  return valid_params(*minb, *maxb, *maxp);
}

static void set_params(zfp_stream* s, u32 minb, u32 maxb, u32 maxp, int32_t mine) {
  s->minbits = minb;
  s->maxbits = maxb;
  s->maxprec = maxp;
  s->minexp = mine;
}

static u32 header_bits_of(zfp_type t) { return t == zfp_type_float ? 9 : t == zfp_type_double ? 12 : 0; }

static zfpb::CodecParams codec_of(const zfp_stream* s) {
  zfpb::CodecParams c;
  c.minbits = s->minbits;
  c.maxbits = s->maxbits;
  c.maxprec = s->maxprec;
  c.minexp = s->minexp;
  c.rounding = ext_of(s)->rounding;
  c.tight = ext_of(s)->tight;
  return c;
}

extern "C" {

zfp_stream* zfp_stream_open(bitstream* bs) {
  StreamExt* e = (StreamExt*)calloc(1, sizeof(StreamExt));
  if (!e) return nullptr;
  set_params(&e->pub, ZFP_MIN_BITS, ZFP_MAX_BITS, ZFP_MAX_PREC, ZFP_MIN_EXP);
  e->pub.stream = bs;
  e->pub.exec.policy = zfp_exec_serial;
  e->pub.exec.params = nullptr;
  return &e->pub;
}

void zfp_stream_close(zfp_stream* s) {
  if (!s) return;
  free(s->exec.params);
  free(ext_of(s));
}

bitstream* zfp_stream_bit_stream(const zfp_stream* s) { return s ? s->stream : nullptr; }
zfp_mode zfp_stream_compression_mode(const zfp_stream* s) { return s ? mode_of(s) : zfp_mode_null; }
double zfp_stream_rate(const zfp_stream* s, uint dims) {
  if (!s || dims < 1 || dims > 4 || mode_of(s) != zfp_mode_fixed_rate) return 0.0;
  return (double)s->maxbits / (double)(1u << (2 * dims));
}
uint zfp_stream_precision(const zfp_stream* s) {
  return (s && mode_of(s) == zfp_mode_fixed_precision) ? s->maxprec : 0;
}
double zfp_stream_accuracy(const zfp_stream* s) {
  return (s && mode_of(s) == zfp_mode_fixed_accuracy) ? std::ldexp(1.0, s->minexp) : 0.0;
}
uint64 zfp_stream_mode(const zfp_stream* s) { return s ? mode_bits(s) : 0; }
void zfp_stream_params(const zfp_stream* s, uint* minb, uint* maxb, uint* maxp, int32_t* mine) {
  if (!s || !minb || !maxb || !maxp || !mine) return;
  *minb = s->minbits;
  *maxb = s->maxbits;
  *maxp = s->maxprec;
  *mine = s->minexp;
}
size_t zfp_stream_compressed_size(const zfp_stream* s) { return (s && s->stream) ? stream_size(s->stream) : 0; }

// zfp-rs-ffi/src/stream.rs:173-205: header + values - 1 + values * precision.
size_t zfp_block_maximum_size(zfp_type t, uint dims, zfp_bool reversible) {
  if (!type_size(t) || dims < 1 || dims > 4) return 0;
  size_t values = (size_t)1 << (2 * dims);
  size_t prec = 8 * type_size(t);
  size_t header = reversible != zfp_false
                      ? (t == zfp_type_int32 ? 5 : t == zfp_type_int64 ? 6 : t == zfp_type_float ? 15 : 19)
                      : header_bits_of(t);
  return header + values - 1 + values * prec;
}

size_t zfp_stream_maximum_size(const zfp_stream* s, const zfp_field* f) {
  if (!s || !f || !type_size(f->type)) return 0;
  zfp_field g = *f;
  size_t* n[4] = {&g.nx, &g.ny, &g.nz, &g.nw};
  bool zero = false;
  for (int i = 0; i < 4; i++) {
    if (*n[i] == 0) zero = true;
    if (zero) *n[i] = 0;
  }
  if (!valid_dims(&g)) return 0;
  Plan p;
  if (!plan_field(&g, p)) return 0;
  u64 bb = zfpb::block_bits(codec_of(s), g.type, p.dims);
  u64 bits;
  if (__builtin_mul_overflow((u64)p.nblocks, bb, &bits)) return 0;
  if (__builtin_add_overflow(bits, (u64)(ZFP_HEADER_MAX_BITS + 63), &bits)) return 0;
  return (size_t)(bits / 64 * 8);
}

size_t zfp_write_header(zfp_stream* s, const zfp_field* f, uint mask) {
  if (!s || !f || !s->stream) return 0;
  bitstream* bs = s->stream;
  uint64 meta = 0;
  if (mask & ZFP_HEADER_META) {
    if (!type_size(f->type) || !valid_dims(f)) return 0;
    size_t n[4] = {f->nx, f->ny, f->nz, f->nw};
    meta = field_metadata(f->type, n, dims_of(f));
    if (meta == ZFP_META_NULL) return 0;
  }
  size_t bits = 0;
  if (mask & ZFP_HEADER_MAGIC) {
    bs_write_bits(bs, 'z', 8);
    bs_write_bits(bs, 'f', 8);
    bs_write_bits(bs, 'p', 8);
    bs_write_bits(bs, ZFP_CODEC, 8);
    bits += ZFP_MAGIC_BITS;
  }
  if (mask & ZFP_HEADER_META) {
    bs_write_bits(bs, meta, ZFP_META_BITS);
    bits += ZFP_META_BITS;
  }
  if (mask & ZFP_HEADER_MODE) {
    uint64 m = mode_bits(s);
    u32 size = m > ZFP_MODE_SHORT_MAX ? ZFP_MODE_LONG_BITS : ZFP_MODE_SHORT_BITS;
    bs_write_bits(bs, m, size);
    bits += size;
  }
  return bits;
}

size_t zfp_read_header(zfp_stream* s, zfp_field* f, uint mask) {
  if (!s || !f || !s->stream) return 0;
  bitstream* bs = s->stream;
  size_t bits = 0;
  if (mask & ZFP_HEADER_MAGIC) {
    if (bs_read_bits(bs, 8) != 'z' || bs_read_bits(bs, 8) != 'f' || bs_read_bits(bs, 8) != 'p' ||
        bs_read_bits(bs, 8) != ZFP_CODEC)
      return 0;
    bits += ZFP_MAGIC_BITS;
  }
  zfp_type t = zfp_type_none;
  size_t n[4];
  bool have_meta = false;
  if (mask & ZFP_HEADER_META) {
    if (!decode_metadata(bs_read_bits(bs, ZFP_META_BITS), &t, n)) return 0;
    have_meta = true;
    bits += ZFP_META_BITS;
  }
  u32 minb = 0, maxb = 0, maxp = 0;
  int32_t mine = 0;
  bool have_mode = false;
  if (mask & ZFP_HEADER_MODE) {
    uint64 m = bs_read_bits(bs, ZFP_MODE_SHORT_BITS);
    bits += ZFP_MODE_SHORT_BITS;
    if (m > ZFP_MODE_SHORT_MAX) {
      m |= bs_read_bits(bs, ZFP_MODE_LONG_BITS - ZFP_MODE_SHORT_BITS) << ZFP_MODE_SHORT_BITS;
      bits += ZFP_MODE_LONG_BITS - ZFP_MODE_SHORT_BITS;
    }
    if (!params_of_mode(m, &minb, &maxb, &maxp, &mine)) return 0;
    have_mode = true;
  }
  if (have_meta) {
    f->type = t;
    f->nx = n[0]; f->ny = n[1]; f->nz = n[2]; f->nw = n[3];
    f->sx = f->sy = f->sz = f->sw = 0;
  }
  if (have_mode) set_params(s, minb, maxb, maxp, mine);
  return bits;
}

void zfp_stream_rewind(zfp_stream* s) {
  if (s && s->stream) bs_rewind(s->stream);
}
void zfp_stream_set_bit_stream(zfp_stream* s, bitstream* bs) {
  if (s) s->stream = bs;
}
void zfp_stream_set_reversible(zfp_stream* s) {
  if (s) set_params(s, ZFP_MIN_BITS, ZFP_MAX_BITS, ZFP_MAX_PREC, ZFP_MIN_EXP - 1);
}

// config.rs:85-102 (rate_bits) and zfp-rs-ffi/src/stream.rs:399-429
double zfp_stream_set_rate(zfp_stream* s, double rate, zfp_type t, uint dims, zfp_bool align) {
  if (!s || dims < 1 || dims > 4 || !type_size(t)) return 0.0;
  double values = (double)(1u << (2 * dims));
  double rounded = std::floor(values * rate + 0.5);
  if (!(rounded >= 0.0 && rounded <= 4294967295.0)) return 0.0;
  u64 bits = (u64)rounded;
  if (bits < header_bits_of(t)) bits = header_bits_of(t);
  if (align == zfp_true) {
    bits = (bits + 63) / 64 * 64;
    if (bits > 0xffffffffull) return 0.0;
  }
  set_params(s, (u32)bits, (u32)bits, ZFP_MAX_PREC, ZFP_MIN_EXP);
  return (double)bits / values;
}

uint zfp_stream_set_precision(zfp_stream* s, uint precision) {
  if (!s) return 0;
  u32 p = precision > 0 ? (precision < ZFP_MAX_PREC ? precision : ZFP_MAX_PREC) : ZFP_MAX_PREC;
  set_params(s, ZFP_MIN_BITS, ZFP_MAX_BITS, p, ZFP_MIN_EXP);
  return p;
}

double zfp_stream_set_accuracy(zfp_stream* s, double tolerance) {
  if (!s) return 0.0;
  int32_t emin = ZFP_MIN_EXP;
  if (tolerance > 0.0) {
    int e = 0;
    std::frexp(tolerance, &e);
    emin = e - 1;
  }
  set_params(s, ZFP_MIN_BITS, ZFP_MAX_BITS, ZFP_MAX_PREC, emin);
  return tolerance > 0.0 ? std::ldexp(1.0, emin) : 0.0;
}

zfp_mode zfp_stream_set_mode(zfp_stream* s, uint64 mode) {
  if (!s) return zfp_mode_null;
  u32 a, b, p;
  int32_t e;
  if (!params_of_mode(mode, &a, &b, &p, &e)) return zfp_mode_null;
  set_params(s, a, b, p, e);
  return mode_of(s);
}

zfp_bool zfp_stream_set_params(zfp_stream* s, uint minb, uint maxb, uint maxp, int32_t mine) {
  if (!s || !valid_params(minb, maxb, maxp)) return zfp_false;
  set_params(s, minb, maxb, maxp, mine);
  return zfp_true;
}

zfp_exec_policy zfp_stream_execution(const zfp_stream* s) { return s ? s->exec.policy : zfp_exec_serial; }
uint zfp_stream_omp_threads(const zfp_stream* s) {
  return (s && s->exec.params) ? ((const zfp_exec_params_omp*)s->exec.params)->threads : 0;
}
uint zfp_stream_omp_chunk_size(const zfp_stream* s) {
  return (s && s->exec.params) ? ((const zfp_exec_params_omp*)s->exec.params)->chunk_size : 0;
}

// Every policy runs the same GPU path; cuda is accepted here, where
// zfp-rs-ffi rejects it (stream.rs:570-593).
zfp_bool zfp_stream_set_execution(zfp_stream* s, zfp_exec_policy policy) {
  if (!s) return zfp_false;
  switch (policy) {
    case zfp_exec_serial:
      free(s->exec.params);
      s->exec.params = nullptr;
      s->exec.policy = zfp_exec_serial;
      return zfp_true;
    case zfp_exec_omp:
    case zfp_exec_cuda:
      s->exec.policy = policy;
      return zfp_true;
    default:
      return zfp_false;
  }
}
zfp_bool zfp_stream_set_omp_threads(zfp_stream* s, uint threads) {
  if (!s) return zfp_false;
  free(s->exec.params);
  zfp_exec_params_omp* p = (zfp_exec_params_omp*)calloc(1, sizeof(zfp_exec_params_omp));
  if (!p) return zfp_false;
  p->threads = threads;
  s->exec.params = p;
  s->exec.policy = zfp_exec_omp;
  return zfp_true;
}
zfp_bool zfp_stream_set_omp_chunk_size(zfp_stream* s, uint chunk) {
  if (!s) return zfp_false;
  zfp_exec_params_omp* p = (zfp_exec_params_omp*)s->exec.params;
  if (!p) {
    p = (zfp_exec_params_omp*)calloc(1, sizeof(zfp_exec_params_omp));
    if (!p) return zfp_false;
    s->exec.params = p;
  }
  p->chunk_size = chunk;
  s->exec.policy = zfp_exec_omp;
  return zfp_true;
}
size_t zfp_stream_flush(zfp_stream* s) { return (s && s->stream) ? bs_flush(s->stream) : 0; }
size_t zfp_stream_align(zfp_stream* s) { return (s && s->stream) ? bs_align(s->stream) : 0; }

zfp_bool zfp_stream_set_rounding(zfp_stream* s, int rounding, zfp_bool tight) {
  if (!s) return zfp_false;
  int r;
  if (rounding == ZFP_ROUND_NEVER) r = 0;
  else if (rounding == ZFP_ROUND_FIRST) r = 1;
  else if (rounding == ZFP_ROUND_LAST) r = 2;
  else return zfp_false;
  ext_of(s)->rounding = r;
  ext_of(s)->tight = tight != zfp_false ? 1 : 0;
  return zfp_true;
}
int zfp_stream_rounding(const zfp_stream* s, zfp_bool* tight) {
  if (!s) return ZFP_ROUND_NEVER;
  if (tight) *tight = ext_of(s)->tight ? zfp_true : zfp_false;
  int r = ext_of(s)->rounding;
  return r == 1 ? ZFP_ROUND_FIRST : r == 2 ? ZFP_ROUND_LAST : ZFP_ROUND_NEVER;
}

int zfpb_last_error(void) { return g_last_error; }

void zfpb_timing_enable(int on) { zfpb::timing_enable(on != 0); }
int zfpb_timing_read(double* ms, unsigned long long* counts, int n) { return zfpb::timing_read(ms, counts, n); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Compress / decompress through the engine
// ---------------------------------------------------------------------------

namespace {

std::mutex g_abi_mu;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool ensure(size_t need) {
    if (need <= bytes) return true;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (cudaMalloc(&p, need < 4096 ? 4096 : need) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    bytes = need < 4096 ? 4096 : need;
    return true;
  }
};

DevBuf g_field_stage, g_stream_stage;
cudaStream_t g_stream = nullptr;

cudaStream_t lib_stream() {
  if (!g_stream) cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
  return g_stream;
}

zfpb::FieldGeom geom_of(const Plan& p, zfp_type t, const void* d_origin) {
  zfpb::FieldGeom g;
  for (int i = 0; i < 4; i++) {
    g.s[i] = i < p.dims ? p.s[i] : 0;
    g.n[i] = i < p.dims ? p.n[i] : 0;
    g.b[i] = i < p.dims ? (p.n[i] + 3) / 4 : 1;
  }
  g.nblocks = p.nblocks;
  size_t es = type_size(t);
  bool vec = p.s[0] == 1 && ((uintptr_t)d_origin % 16) == 0;
  for (int i = 1; i < p.dims; i++) vec = vec && ((p.s[i] * (ptrdiff_t)es) % 16) == 0;
  g.vec_ok = vec ? 1 : 0;
  zfpb::fill_block_inverses(g);
  return g;
}

bool index_matches(const IndexCache& ix, u64 start, const zfpb::Call& call) {
  return ix.valid && ix.start == start && ix.nblocks == call.f.nblocks && ix.type == call.type &&
         ix.dims == call.dims && ix.c.minbits == call.c.minbits && ix.c.maxbits == call.c.maxbits &&
         ix.c.maxprec == call.c.maxprec && ix.c.minexp == call.c.minexp && ix.c.rounding == call.c.rounding &&
         ix.c.tight == call.c.tight;
}

// Host fields from this size on go through the pipelined copy paths.
constexpr size_t kPipelineBytes = 32u << 20;

int fail(int code) {
  g_last_error = code;
  return 0;
}

}  // namespace

extern "C" size_t zfp_compress(zfp_stream* zs, const zfp_field* f) {
  if (!zs || !f || !zs->stream) return fail(zfpb::ERR_ARGS);
  bitstream* bs = zs->stream;
  Plan p;
  if (!f->data || !valid_dims(f) || !plan_field(f, p)) return fail(zfpb::ERR_ARGS);
  const size_t es = type_size(f->type);
  if (((uintptr_t)f->data % es) != 0) return fail(zfpb::ERR_ARGS);
  std::lock_guard<std::mutex> lock(g_abi_mu);
  cudaStream_t s = lib_stream();

  // Field: device pointer as is, host span staged.  A large host field with
  // natural strides into a host stream goes through the pipelined path, which
  // copies the field in chunk by chunk itself.
  const void* d_origin = f->data;
  const bool pipelined = !is_device_ptr(f->data) && !zs->stream->device && p.contiguous &&
                         p.span_bytes >= kPipelineBytes;
  if (!is_device_ptr(f->data)) {
    if (!g_field_stage.ensure(p.span_bytes)) return fail(zfpb::ERR_CUDA);
    const char* begin = (const char*)f->data + p.imin * (ptrdiff_t)es;
    if (!pipelined && cudaMemcpyAsync(g_field_stage.p, begin, p.span_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    d_origin = (const char*)g_field_stage.p - p.imin * (ptrdiff_t)es;
  }
  zfpb::Call call;
  call.type = f->type;
  call.dims = p.dims;
  call.f = geom_of(p, f->type, d_origin);
  call.c = codec_of(zs);

  // Stream: words from the cursor's word on, staged for a host buffer.
  const u64 start = bs_wtell(bs);
  const u64 w0 = start / 64;
  if (w0 > bs->len) return fail(zfpb::ERR_OVERFLOW);
  const u64 cap = bs->len - w0;
  u64* d_out;
  if (bs->device) {
    d_out = bs->words + w0;
  } else {
    if (!g_stream_stage.ensure((cap + 1) * 8)) return fail(zfpb::ERR_CUDA);
    d_out = (u64*)g_stream_stage.p;
  }
  const u64 init = bs->bits ? (bs->buffer & ((1ull << bs->bits) - 1)) : 0;

  IndexCache& ix = bs->index;
  ix.valid = false;
  u64* d_off = nullptr;
  if (!zfpb::fixed_size_blocks(call)) {
    size_t need = p.nblocks + 1;
    if (ix.cap < need) {
      if (ix.d_off) cudaFree(ix.d_off);
      ix.d_off = nullptr;
      ix.cap = 0;
      if (cudaMalloc((void**)&ix.d_off, need * sizeof(u64)) == cudaSuccess) ix.cap = need;
      else cudaGetLastError();
    }
    d_off = ix.d_off;
  }
  u64 end_rel = 0;
  zfpb::Status st = zfpb::ERR_ARGS;
  if (pipelined) {
    // Copies in and out overlap the coding, chunk by chunk.
    st = zfpb::compress_host(call, (const char*)f->data, (void*)d_origin, bs->words + w0, d_out, cap, start % 64, init,
                             &end_rel, d_off, s);
  }
  bool copied = pipelined && st != zfpb::ERR_ARGS;
  if (!copied) {
    if (pipelined && cudaMemcpyAsync(g_field_stage.p, f->data, p.span_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    st = zfpb::compress(call, d_origin, d_out, cap, start % 64, init, &end_rel, d_off, s);
  }
  if (st == zfpb::ERR_OVERFLOW) {
    bs->overflowed = true;
    return fail(zfpb::ERR_OVERFLOW);
  }
  if (st != zfpb::OK) return fail(st);
  const u64 end = w0 * 64 + end_rel;
  const u64 wend = (end + 63) / 64;
  if (!copied && !bs->device && wend > w0) {
    if (cudaMemcpyAsync(bs->words + w0, d_out, (wend - w0) * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zfpb::ERR_CUDA);
  if (d_off) {
    ix.valid = true;
    ix.start = start;
    ix.nblocks = p.nblocks;
    ix.type = call.type;
    ix.dims = call.dims;
    ix.c = call.c;
    ix.end = end;
  }
  // finish(): flush to a word (compress.rs:44-53).
  bs->word_pos = (size_t)wend;
  bs->buffer = 0;
  bs->bits = 0;
  return (size_t)(wend * 8);
}

extern "C" size_t zfp_decompress(zfp_stream* zs, zfp_field* f) {
  if (!zs || !f || !zs->stream) return fail(zfpb::ERR_ARGS);
  bitstream* bs = zs->stream;
  Plan p;
  if (!f->data || !valid_dims(f) || !plan_field(f, p) || p.span_bytes == 0) return fail(zfpb::ERR_ARGS);
  const size_t es = type_size(f->type);
  if (((uintptr_t)f->data % es) != 0) return fail(zfpb::ERR_ARGS);
  std::lock_guard<std::mutex> lock(g_abi_mu);
  cudaStream_t s = lib_stream();

  const bool host_field = !is_device_ptr(f->data);
  void* d_origin = f->data;
  char* begin = (char*)f->data + p.imin * (ptrdiff_t)es;
  const bool pipelined = host_field && !bs->device && p.contiguous && p.span_bytes >= kPipelineBytes;
  if (host_field) {
    if (!g_field_stage.ensure(p.span_bytes)) return fail(zfpb::ERR_CUDA);
    // Gaps between strided elements keep their values.
    if (p.span_bytes != p.nelems * es &&
        cudaMemcpyAsync(g_field_stage.p, begin, p.span_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    d_origin = (char*)g_field_stage.p - p.imin * (ptrdiff_t)es;
  }
  zfpb::Call call;
  call.type = f->type;
  call.dims = p.dims;
  call.f = geom_of(p, f->type, d_origin);
  call.c = codec_of(zs);

  const u64 start = bs_rtell(bs);
  const u64 w0 = start / 64;
  const u64 avail = bs->len > w0 ? bs->len - w0 : 0;
  const u64* d_in;
  if (bs->device) {
    d_in = bs->words + w0;
  } else {
    // Stage the words the blocks occupy when their end is known: fixed-size
    // blocks, or the end recorded with the index of this stream's last compress.
    u64 need = avail;
    u64 end_known = 0;
    if (zfpb::fixed_size_blocks(call))
      end_known = start + (u64)p.nblocks * call.c.maxbits;
    else if (index_matches(bs->index, start, call))
      end_known = bs->index.end;
    if (end_known) {
      u64 words = (end_known + 63) / 64 - w0 + 1;
      need = words < avail ? words : avail;
    }
    if (!g_stream_stage.ensure((avail + 1) * 8)) return fail(zfpb::ERR_CUDA);
    const bool chunked = pipelined && (zfpb::fixed_size_blocks(call) || index_matches(bs->index, start, call));
    if (!chunked && need &&
        cudaMemcpyAsync(g_stream_stage.p, bs->words + w0, need * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    d_in = (const u64*)g_stream_stage.p;
  }
  const u64* cand = index_matches(bs->index, start, call) ? bs->index.d_off : nullptr;
  u64 end_rel = 0;
  zfpb::Status st = zfpb::ERR_ARGS;
  bool done_host = false;
  if (pipelined && (cand || zfpb::fixed_size_blocks(call))) {
    // Copies in and out overlap the decoding, chunk by chunk.
    st = zfpb::decompress_host(call, bs->words + w0, (u64*)g_stream_stage.p, avail, start % 64, begin,
                               (void*)d_origin, &end_rel, cand, s);
    done_host = st == zfpb::OK || st == zfpb::ERR_TRUNCATED;
    if (!done_host && st != zfpb::ERR_BAD_INDEX && st != zfpb::ERR_ARGS) return fail(st);
    if (!done_host) {
      // Fall back: stage the whole stream for the one-pass path below (which
      // walks the stream when the index did not match).
      if (avail && cudaMemcpyAsync(g_stream_stage.p, bs->words + w0, avail * 8, cudaMemcpyHostToDevice, s) !=
                       cudaSuccess)
        return fail(zfpb::ERR_CUDA);
    }
  }
  if (!done_host && st != zfpb::ERR_BAD_INDEX)
    st = zfpb::decompress(call, d_in, avail, start % 64, d_origin, &end_rel, cand, s);
  if (st == zfpb::ERR_BAD_INDEX) {
    // The stream changed since its last compress: stage all of it and walk it.
    bs->index.valid = false;
    if (!bs->device && avail &&
        cudaMemcpyAsync(g_stream_stage.p, bs->words + w0, avail * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    st = zfpb::decompress(call, d_in, avail, start % 64, d_origin, &end_rel, nullptr, s);
  }
  if (st != zfpb::OK && st != zfpb::ERR_TRUNCATED) return fail(st);
  if (host_field && !done_host &&
      cudaMemcpyAsync(begin, g_field_stage.p, p.span_bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return fail(zfpb::ERR_CUDA);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zfpb::ERR_CUDA);
  // finish(): align the cursor after the last block (decompress.rs:66-74).
  const u64 end = w0 * 64 + end_rel;
  bs->word_pos = (size_t)((end + 63) / 64);
  bs->buffer = 0;
  bs->bits = 0;
  bs->seek_word = bs->word_pos;
  if (st == zfpb::ERR_TRUNCATED) return fail(zfpb::ERR_TRUNCATED);
  return bs->word_pos * 8;
}

// ---------------------------------------------------------------------------
// Device API (zfp_b200.h)
// ---------------------------------------------------------------------------

static bool call_of_desc(const zfpb_desc* d, Plan& p, zfpb::Call& call, const void* d_origin) {
  zfp_field f;
  memset(&f, 0, sizeof(f));
  f.type = d->type;
  f.nx = d->nx; f.ny = d->ny; f.nz = d->nz; f.nw = d->nw;
  f.sx = d->sx; f.sy = d->sy; f.sz = d->sz; f.sw = d->sw;
  if (!valid_dims(&f) || !plan_field(&f, p)) return false;
  call.type = d->type;
  call.dims = p.dims;
  call.f = geom_of(p, d->type, d_origin);
  call.c.minbits = d->minbits;
  call.c.maxbits = d->maxbits;
  call.c.maxprec = d->maxprec;
  call.c.minexp = d->minexp;
  call.c.rounding = d->rounding == ZFP_ROUND_FIRST ? 1 : d->rounding == ZFP_ROUND_LAST ? 2 : 0;
  call.c.tight = d->tight_error != zfp_false ? 1 : 0;
  return true;
}

extern "C" size_t zfpb_compress_device(const zfpb_desc* d, const void* d_field, void* d_stream, size_t capacity,
                                       uint64_t* d_block_offsets, void* cuda_stream) {
  if (!d || !d_field || !d_stream || ((uintptr_t)d_stream % 8) != 0) return fail(zfpb::ERR_ARGS);
  Plan p;
  zfpb::Call call;
  if (!call_of_desc(d, p, call, d_field)) return fail(zfpb::ERR_ARGS);
  cudaStream_t s = (cudaStream_t)cuda_stream;
  u64 end = 0;
  zfpb::Status st = zfpb::compress(call, d_field, (u64*)d_stream, capacity / 8, 0, 0, &end, (u64*)d_block_offsets, s);
  if (st != zfpb::OK) return fail(st);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zfpb::ERR_CUDA);
  return (size_t)((end + 63) / 64 * 8);
}

extern "C" size_t zfpb_decompress_device(const zfpb_desc* d, const void* d_stream, size_t bytes, void* d_field,
                                         const uint64_t* d_block_offsets, void* cuda_stream) {
  if (!d || !d_field || !d_stream || ((uintptr_t)d_stream % 8) != 0) return fail(zfpb::ERR_ARGS);
  Plan p;
  zfpb::Call call;
  if (!call_of_desc(d, p, call, d_field)) return fail(zfpb::ERR_ARGS);
  cudaStream_t s = (cudaStream_t)cuda_stream;
  u64 end = 0;
  zfpb::Status st = zfpb::decompress(call, (const u64*)d_stream, bytes / 8, 0, d_field, &end, (const u64*)d_block_offsets, s);
  if (st == zfpb::ERR_BAD_INDEX)
    st = zfpb::decompress(call, (const u64*)d_stream, bytes / 8, 0, d_field, &end, nullptr, s);
  if (st != zfpb::OK) return fail(st);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zfpb::ERR_CUDA);
  return (size_t)((end + 63) / 64 * 8);
}

// The header zfp_write_header(mask) writes for a description's field and mode:
// its words (zero past the last bit) and its length in bits.  False if the
// description has none (e.g. sizes the metadata cannot hold).
static bool header_of_desc(const zfpb_desc* d, uint mask, u64* hdr, u64* bits) {
  hdr[0] = hdr[1] = hdr[2] = 0;
  *bits = 0;
  if (!mask) return true;
  zfp_field f;
  memset(&f, 0, sizeof(f));
  f.type = d->type;
  f.nx = d->nx; f.ny = d->ny; f.nz = d->nz; f.nw = d->nw;
  zfp_stream zs;
  memset(&zs, 0, sizeof(zs));
  zs.minbits = d->minbits;
  zs.maxbits = d->maxbits;
  zs.maxprec = d->maxprec;
  zs.minexp = d->minexp;
  alignas(8) u64 buf[4] = {0, 0, 0, 0};
  bitstream* bs = stream_open(buf, sizeof(buf));
  if (!bs) return false;
  zs.stream = bs;
  const size_t n = zfp_write_header(&zs, &f, mask);
  stream_flush(bs);
  stream_close(bs);
  if (n == 0 || n > 3 * 64) return false;
  for (int w = 0; w < 3; w++) hdr[w] = buf[w];
  *bits = n;
  return true;
}

// An item's job: its call, buffers and header.
static bool job_of_item(const zfpb_batch_item& it, zfpb::BatchJob& J) {
  if (!it.d_field || !it.d_stream || ((uintptr_t)it.d_stream % 8) != 0) return false;
  Plan p;
  if (!call_of_desc(&it.desc, p, J.call, it.d_field)) return false;
  if (!header_of_desc(&it.desc, it.header_mask, J.hdr, &J.start_bit)) return false;
  J.field = it.d_field;
  J.stream = (u64*)it.d_stream;
  J.stream_words = it.stream_bytes / 8;
  J.index = (u64*)it.d_block_offsets;
  return true;
}

// Batches: every item converted to an engine job, coded together
// (zfpb::compress_batch / decompress_batch), results written back per item.
static size_t run_batch_abi(zfpb_batch_item* items, size_t n, void* cuda_stream, bool compress) {
  if (!items && n) return fail(zfpb::ERR_ARGS);
  std::vector<zfpb::BatchJob> jobs(n);
  std::vector<size_t> job_of(n, (size_t)-1);
  size_t m = 0;
  for (size_t i = 0; i < n; i++) {
    zfpb_batch_item& it = items[i];
    it.result = 0;
    it.status = zfpb::ERR_ARGS;
    if (!job_of_item(it, jobs[m])) continue;
    job_of[i] = m++;
  }
  cudaStream_t s = (cudaStream_t)cuda_stream;
  if (m) {
    zfpb::Status st = compress ? zfpb::compress_batch(jobs.data(), m, s) : zfpb::decompress_batch(jobs.data(), m, s);
    (void)st;
  }
  size_t ok = 0;
  for (size_t i = 0; i < n; i++) {
    if (job_of[i] == (size_t)-1) continue;
    const zfpb::BatchJob& J = jobs[job_of[i]];
    items[i].status = J.status;
    if (J.status == zfpb::OK) {
      items[i].result = (size_t)((J.end_bit + 63) / 64 * 8);
      ok++;
    }
  }
  g_last_error = 0;
  for (size_t i = 0; i < n; i++)
    if (items[i].status != 0) {
      g_last_error = items[i].status;  // the first failing item's reason
      break;
    }
  return ok;
}

extern "C" size_t zfpb_compress_batch(zfpb_batch_item* items, size_t n, void* cuda_stream) {
  return run_batch_abi(items, n, cuda_stream, true);
}

extern "C" size_t zfpb_decompress_batch(zfpb_batch_item* items, size_t n, void* cuda_stream) {
  return run_batch_abi(items, n, cuda_stream, false);
}

// Serving loop (zfpb_serve.cpp): items converted to engine jobs at submit.
extern "C" zfpb_server* zfpb_server_create(size_t budget_bytes, int lanes, size_t max_batch, size_t batch_bytes) {
  zfpb::Server* s = zfpb::server_create(budget_bytes, lanes, max_batch, batch_bytes);
  if (!s) fail(zfpb::ERR_CUDA);
  return reinterpret_cast<zfpb_server*>(s);
}

extern "C" int zfpb_server_submit(zfpb_server* srv, const zfpb_batch_item* it, int decompress, uint64_t tag) {
  if (!srv || !it) return fail(zfpb::ERR_ARGS);
  zfpb::BatchJob J{};
  if (!job_of_item(*it, J)) return fail(zfpb::ERR_ARGS);
  if (!zfpb::server_submit(reinterpret_cast<zfpb::Server*>(srv), J, decompress != 0, tag))
    return fail(zfpb::ERR_TOO_LARGE);
  return 1;
}

extern "C" size_t zfpb_server_poll(zfpb_server* srv, zfpb_request_done* out, size_t max, int wait_ms) {
  if (!srv || (!out && max)) return 0;
  std::vector<zfpb::ServeDone> d(max);
  size_t n = zfpb::server_poll(reinterpret_cast<zfpb::Server*>(srv), d.data(), max, wait_ms);
  for (size_t i = 0; i < n; i++) {
    out[i].tag = d[i].tag;
    out[i].result = (size_t)d[i].result;
    out[i].status = d[i].status;
    out[i].queue_ms = d[i].queue_ms;
    out[i].latency_ms = d[i].latency_ms;
  }
  return n;
}

extern "C" size_t zfpb_server_outstanding(zfpb_server* srv) {
  return srv ? zfpb::server_outstanding(reinterpret_cast<zfpb::Server*>(srv)) : 0;
}

extern "C" void zfpb_server_destroy(zfpb_server* srv) { zfpb::server_destroy(reinterpret_cast<zfpb::Server*>(srv)); }

// Same stream as zfpb_compress_device, with scratch from the library's static
// device array instead of cudaMalloc (see include/zfp_b200.h).  Allocates
// nothing: no cudaMalloc, cudaFree, cudaMallocHost or library allocator.
extern "C" size_t zfpb_compress_device_noalloc(const zfpb_desc* d, const void* d_field, void* d_stream,
                                               size_t capacity, void* cuda_stream) {
  if (!d || !d_field || !d_stream || ((uintptr_t)d_stream % 8) != 0) return fail(zfpb::ERR_ARGS);
  Plan p;
  zfpb::Call call;
  if (!call_of_desc(d, p, call, d_field)) return fail(zfpb::ERR_ARGS);
  u64 end = 0;
  zfpb::Status st = zfpb::compress_noalloc(call, d_field, (u64*)d_stream, capacity / 8, &end,
                                           (cudaStream_t)cuda_stream);
  if (st != zfpb::OK) return fail(st);
  return (size_t)((end + 63) / 64 * 8);
}

// ---------------------------------------------------------------------------
// Block-level calls (zfp-rs-ffi/src/block.rs:25-776, codec/block/strided.rs:
// 420-690): one 4^d block of a caller's array coded at the bit stream's
// cursor, on the GPU.  The block is a field of one block (lengths 1..4 per
// axis, the caller's element strides taken as given, 0 included), run
// through the same engine as zfp_compress / zfp_decompress; the cursor is
// left right after the block's bits, not flushed, so that calls append block
// after block as the reference's do.  Returns the block's bits (after the
// pad/skip to minbits), or 0 for a missing stream or pointer or an invalid
// length.  Each call is one small GPU round trip: for many blocks
// zfpb_encode_blocks / zfpb_decode_blocks code them in one call.
// ---------------------------------------------------------------------------

namespace {

DevBuf g_block_words;  // stream words of one block call (host bit streams)

size_t block_call(zfp_stream* zs, zfp_type t, int dims, void* data, const ptrdiff_t* st, const size_t* len,
                  bool encode) {
  if (!zs || !zs->stream || !data) return 0;
  for (int d = 0; d < dims; d++)
    if (len[d] < 1 || len[d] > 4) return 0;  // strided.rs check_lengths
  bitstream* bs = zs->stream;
  const size_t es = type_size(t);
  Plan p;
  p.dims = dims;
  p.nblocks = 1;
  p.nelems = 1;
  for (int d = 0; d < dims; d++) {
    p.n[d] = len[d];
    p.s[d] = st[d];
    p.nelems *= len[d];
    const ptrdiff_t ext = st[d] * (ptrdiff_t)(len[d] - 1);
    if (ext < 0) p.imin += ext; else p.imax += ext;
  }
  p.span_bytes = (size_t)(p.imax - p.imin + 1) * es;
  std::lock_guard<std::mutex> lock(g_abi_mu);
  cudaStream_t s = lib_stream();
  const bool host = !is_device_ptr(data);
  char* begin = (char*)data + p.imin * (ptrdiff_t)es;
  void* d_origin = data;
  if (host) {
    if (!g_field_stage.ensure(p.span_bytes)) return fail(zfpb::ERR_CUDA);
    // Encode reads the span; decode keeps the gaps between strided elements.
    if (cudaMemcpyAsync(g_field_stage.p, begin, p.span_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    d_origin = (char*)g_field_stage.p - p.imin * (ptrdiff_t)es;
  }
  zfpb::Call call;
  call.type = t;
  call.dims = dims;
  call.f = geom_of(p, t, d_origin);
  call.c = codec_of(zs);
  const u64 bb = zfpb::block_bits(call.c, t, dims);
  if (encode) {
    const u64 start = bs_wtell(bs);
    const u64 w0 = start / 64;
    if (w0 > bs->len) {
      bs->overflowed = true;
      return fail(zfpb::ERR_OVERFLOW);
    }
    const u64 need = (start % 64 + bb + 63) / 64 + 1;
    const u64 cap = bs->len - w0 < need ? bs->len - w0 : need;
    u64* d_out = bs->words + w0;
    if (!bs->device) {
      if (!g_block_words.ensure(need * 8)) return fail(zfpb::ERR_CUDA);
      d_out = (u64*)g_block_words.p;
    }
    const u64 init = bs->bits ? (bs->buffer & ((1ull << bs->bits) - 1)) : 0;
    u64 end_rel = 0;
    zfpb::Status stt = zfpb::compress(call, d_origin, d_out, cap, start % 64, init, &end_rel, nullptr, s);
    if (stt == zfpb::ERR_OVERFLOW) {
      bs->overflowed = true;
      return fail(stt);
    }
    if (stt != zfpb::OK) return fail(stt);
    const u64 end = w0 * 64 + end_rel;
    const u64 wend = (end + 63) / 64;
    if (!bs->device && wend > w0 &&
        cudaMemcpyAsync(bs->words + w0, d_out, (wend - w0) * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zfpb::ERR_CUDA);
    // The cursor after the block, its partial word still buffered.
    bs->word_pos = (size_t)(end / 64);
    bs->bits = (u32)(end % 64);
    bs->buffer = bs->bits ? get_word(bs, bs->word_pos) & ((1ull << bs->bits) - 1) : 0;
    bs->index.valid = false;
    return (size_t)(end - start);
  }
  const u64 start = bs_rtell(bs);
  const u64 w0 = start / 64;
  const u64 avail = bs->len > w0 ? bs->len - w0 : 0;
  const u64 need = (start % 64 + bb + 63) / 64 + 2;
  const u64 len_words = avail < need ? avail : need;
  const u64* d_in = bs->words + w0;
  if (!bs->device) {
    if (!g_block_words.ensure((len_words + 1) * 8)) return fail(zfpb::ERR_CUDA);
    if (len_words &&
        cudaMemcpyAsync(g_block_words.p, bs->words + w0, len_words * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return fail(zfpb::ERR_CUDA);
    d_in = (const u64*)g_block_words.p;
  }
  u64 end_rel = 0;
  zfpb::Status stt = zfpb::decompress(call, d_in, len_words, start % 64, d_origin, &end_rel, nullptr, s);
  if (stt != zfpb::OK && stt != zfpb::ERR_TRUNCATED) return fail(stt);
  if (host && cudaMemcpyAsync(begin, g_field_stage.p, p.span_bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return fail(zfpb::ERR_CUDA);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(zfpb::ERR_CUDA);
  const u64 end = w0 * 64 + end_rel;
  bs_seek_read(bs, end);
  if (stt == zfpb::ERR_TRUNCATED) bs->overread = true;
  return (size_t)(end - start);
}

// The contiguous layout of a whole block: x fastest, strides 1, 4, 16, 64.
const ptrdiff_t kContig[4] = {1, 4, 16, 64};
const size_t kWhole[4] = {4, 4, 4, 4};

}  // namespace

#define ZFPB_BLOCK_FNS(NAME, CT, ZT)                                                                              \
  extern "C" size_t zfp_encode_block_##NAME##_1(zfp_stream* s, const CT* b) {                                   \
    return block_call(s, ZT, 1, (void*)b, kContig, kWhole, true);                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_##NAME##_2(zfp_stream* s, const CT* b) {                                   \
    return block_call(s, ZT, 2, (void*)b, kContig, kWhole, true);                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_##NAME##_3(zfp_stream* s, const CT* b) {                                   \
    return block_call(s, ZT, 3, (void*)b, kContig, kWhole, true);                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_##NAME##_4(zfp_stream* s, const CT* b) {                                   \
    return block_call(s, ZT, 4, (void*)b, kContig, kWhole, true);                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_##NAME##_1(zfp_stream* s, CT* b) {                                         \
    return block_call(s, ZT, 1, b, kContig, kWhole, false);                                                       \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_##NAME##_2(zfp_stream* s, CT* b) {                                         \
    return block_call(s, ZT, 2, b, kContig, kWhole, false);                                                       \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_##NAME##_3(zfp_stream* s, CT* b) {                                         \
    return block_call(s, ZT, 3, b, kContig, kWhole, false);                                                       \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_##NAME##_4(zfp_stream* s, CT* b) {                                         \
    return block_call(s, ZT, 4, b, kContig, kWhole, false);                                                       \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_strided_##NAME##_1(zfp_stream* s, const CT* b, ptrdiff_t sx) {             \
    const ptrdiff_t st[4] = {sx, 0, 0, 0};                                                                        \
    return block_call(s, ZT, 1, (void*)b, st, kWhole, true);                                                      \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_strided_##NAME##_2(zfp_stream* s, const CT* b, ptrdiff_t sx, ptrdiff_t sy) { \
    const ptrdiff_t st[4] = {sx, sy, 0, 0};                                                                       \
    return block_call(s, ZT, 2, (void*)b, st, kWhole, true);                                                      \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_strided_##NAME##_3(zfp_stream* s, const CT* b, ptrdiff_t sx, ptrdiff_t sy,  \
                                                        ptrdiff_t sz) {                                           \
    const ptrdiff_t st[4] = {sx, sy, sz, 0};                                                                      \
    return block_call(s, ZT, 3, (void*)b, st, kWhole, true);                                                      \
  }                                                                                                               \
  extern "C" size_t zfp_encode_block_strided_##NAME##_4(zfp_stream* s, const CT* b, ptrdiff_t sx, ptrdiff_t sy,  \
                                                        ptrdiff_t sz, ptrdiff_t sw) {                             \
    const ptrdiff_t st[4] = {sx, sy, sz, sw};                                                                     \
    return block_call(s, ZT, 4, (void*)b, st, kWhole, true);                                                      \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_strided_##NAME##_1(zfp_stream* s, CT* b, ptrdiff_t sx) {                   \
    const ptrdiff_t st[4] = {sx, 0, 0, 0};                                                                        \
    return block_call(s, ZT, 1, b, st, kWhole, false);                                                            \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_strided_##NAME##_2(zfp_stream* s, CT* b, ptrdiff_t sx, ptrdiff_t sy) {       \
    const ptrdiff_t st[4] = {sx, sy, 0, 0};                                                                       \
    return block_call(s, ZT, 2, b, st, kWhole, false);                                                            \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_strided_##NAME##_3(zfp_stream* s, CT* b, ptrdiff_t sx, ptrdiff_t sy,        \
                                                        ptrdiff_t sz) {                                           \
    const ptrdiff_t st[4] = {sx, sy, sz, 0};                                                                      \
    return block_call(s, ZT, 3, b, st, kWhole, false);                                                            \
  }                                                                                                               \
  extern "C" size_t zfp_decode_block_strided_##NAME##_4(zfp_stream* s, CT* b, ptrdiff_t sx, ptrdiff_t sy,        \
                                                        ptrdiff_t sz, ptrdiff_t sw) {                             \
    const ptrdiff_t st[4] = {sx, sy, sz, sw};                                                                     \
    return block_call(s, ZT, 4, b, st, kWhole, false);                                                            \
  }                                                                                                               \
  extern "C" size_t zfp_encode_partial_block_strided_##NAME##_1(zfp_stream* s, const CT* b, size_t nx,           \
                                                                ptrdiff_t sx) {                                   \
    const ptrdiff_t st[4] = {sx, 0, 0, 0};                                                                        \
    const size_t n[4] = {nx, 0, 0, 0};                                                                            \
    return block_call(s, ZT, 1, (void*)b, st, n, true);                                                           \
  }                                                                                                               \
  extern "C" size_t zfp_encode_partial_block_strided_##NAME##_2(zfp_stream* s, const CT* b, size_t nx,           \
                                                                size_t ny, ptrdiff_t sx, ptrdiff_t sy) {          \
    const ptrdiff_t st[4] = {sx, sy, 0, 0};                                                                       \
    const size_t n[4] = {nx, ny, 0, 0};                                                                           \
    return block_call(s, ZT, 2, (void*)b, st, n, true);                                                           \
  }                                                                                                               \
  extern "C" size_t zfp_encode_partial_block_strided_##NAME##_3(zfp_stream* s, const CT* b, size_t nx,           \
                                                                size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, \
                                                                ptrdiff_t sz) {                                   \
    const ptrdiff_t st[4] = {sx, sy, sz, 0};                                                                      \
    const size_t n[4] = {nx, ny, nz, 0};                                                                          \
    return block_call(s, ZT, 3, (void*)b, st, n, true);                                                           \
  }                                                                                                               \
  extern "C" size_t zfp_encode_partial_block_strided_##NAME##_4(zfp_stream* s, const CT* b, size_t nx,           \
                                                                size_t ny, size_t nz, size_t nw, ptrdiff_t sx,    \
                                                                ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw) {       \
    const ptrdiff_t st[4] = {sx, sy, sz, sw};                                                                     \
    const size_t n[4] = {nx, ny, nz, nw};                                                                         \
    return block_call(s, ZT, 4, (void*)b, st, n, true);                                                           \
  }                                                                                                               \
  extern "C" size_t zfp_decode_partial_block_strided_##NAME##_1(zfp_stream* s, CT* b, size_t nx, ptrdiff_t sx) { \
    const ptrdiff_t st[4] = {sx, 0, 0, 0};                                                                        \
    const size_t n[4] = {nx, 0, 0, 0};                                                                            \
    return block_call(s, ZT, 1, b, st, n, false);                                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_decode_partial_block_strided_##NAME##_2(zfp_stream* s, CT* b, size_t nx, size_t ny,      \
                                                                ptrdiff_t sx, ptrdiff_t sy) {                     \
    const ptrdiff_t st[4] = {sx, sy, 0, 0};                                                                       \
    const size_t n[4] = {nx, ny, 0, 0};                                                                           \
    return block_call(s, ZT, 2, b, st, n, false);                                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_decode_partial_block_strided_##NAME##_3(zfp_stream* s, CT* b, size_t nx, size_t ny,      \
                                                                size_t nz, ptrdiff_t sx, ptrdiff_t sy,            \
                                                                ptrdiff_t sz) {                                   \
    const ptrdiff_t st[4] = {sx, sy, sz, 0};                                                                      \
    const size_t n[4] = {nx, ny, nz, 0};                                                                          \
    return block_call(s, ZT, 3, b, st, n, false);                                                                 \
  }                                                                                                               \
  extern "C" size_t zfp_decode_partial_block_strided_##NAME##_4(zfp_stream* s, CT* b, size_t nx, size_t ny,      \
                                                                size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, \
                                                                ptrdiff_t sz, ptrdiff_t sw) {                     \
    const ptrdiff_t st[4] = {sx, sy, sz, sw};                                                                     \
    const size_t n[4] = {nx, ny, nz, nw};                                                                         \
    return block_call(s, ZT, 4, b, st, n, false);                                                                 \
  }

ZFPB_BLOCK_FNS(int32, int32_t, zfp_type_int32)
ZFPB_BLOCK_FNS(int64, int64_t, zfp_type_int64)
ZFPB_BLOCK_FNS(float, float, zfp_type_float)
ZFPB_BLOCK_FNS(double, double, zfp_type_double)
#undef ZFPB_BLOCK_FNS

// ---------------------------------------------------------------------------
// Integer promotion and demotion of one block of 4^dims values
// (zfp-rs-ffi/src/promote.rs:11-59, src/codec/promote.rs): 8- and 16-bit
// values to the int32 range the codec works in and back, clamped.  Plain
// element maps on the caller's (host) arrays; dims outside 1..4 or a null
// pointer do nothing.
// ---------------------------------------------------------------------------

namespace {
template <class D, class S, class F> void map_block(D* out, const S* in, uint dims, F f) {
  if (!out || !in || dims < 1 || dims > 4) return;
  const size_t n = (size_t)1 << (2 * dims);
  for (size_t i = 0; i < n; i++) out[i] = f(in[i]);
}
template <class T> T clamp_to(int32_t v, int32_t lo, int32_t hi) { return (T)(v < lo ? lo : v > hi ? hi : v); }
}  // namespace

extern "C" void zfp_promote_int8_to_int32(int32_t* o, const int8_t* i, uint dims) {
  map_block(o, i, dims, [](int8_t x) { return (int32_t)((uint32_t)(int32_t)x << 23); });
}
extern "C" void zfp_promote_uint8_to_int32(int32_t* o, const uint8_t* i, uint dims) {
  map_block(o, i, dims, [](uint8_t x) { return (int32_t)((uint32_t)((int32_t)x - 0x80) << 23); });
}
extern "C" void zfp_promote_int16_to_int32(int32_t* o, const int16_t* i, uint dims) {
  map_block(o, i, dims, [](int16_t x) { return (int32_t)((uint32_t)(int32_t)x << 15); });
}
extern "C" void zfp_promote_uint16_to_int32(int32_t* o, const uint16_t* i, uint dims) {
  map_block(o, i, dims, [](uint16_t x) { return (int32_t)((uint32_t)((int32_t)x - 0x8000) << 15); });
}
extern "C" void zfp_demote_int32_to_int8(int8_t* o, const int32_t* i, uint dims) {
  map_block(o, i, dims, [](int32_t x) { return clamp_to<int8_t>(x >> 23, -0x80, 0x7f); });
}
extern "C" void zfp_demote_int32_to_uint8(uint8_t* o, const int32_t* i, uint dims) {
  map_block(o, i, dims, [](int32_t x) { return clamp_to<uint8_t>((x >> 23) + 0x80, 0, 0xff); });
}
extern "C" void zfp_demote_int32_to_int16(int16_t* o, const int32_t* i, uint dims) {
  map_block(o, i, dims, [](int32_t x) { return clamp_to<int16_t>(x >> 15, -0x8000, 0x7fff); });
}
extern "C" void zfp_demote_int32_to_uint16(uint16_t* o, const int32_t* i, uint dims) {
  map_block(o, i, dims, [](int32_t x) { return clamp_to<uint16_t>((x >> 15) + 0x8000, 0, 0xffff); });
}

// ---------------------------------------------------------------------------
// Many whole blocks in one GPU call (zfp_b200.h): `count` contiguous blocks
// of 4^dims values (block i at element 4^dims * i, in the layout of
// zfp_encode_block_*) are, to the codec, a field of 4 x .. x 4 x (4 * count)
// values with natural strides, whose blocks come in exactly that order; the
// stream is the one `count` calls of zfp_encode_block_<type>_<dims> on one
// stream write, flushed to a word.
// ---------------------------------------------------------------------------

static bool blocks_desc(const zfpb_desc* d, uint dims, size_t count, zfpb_desc* out) {
  if (!d || dims < 1 || dims > 4 || count == 0 || count > ((size_t)1 << 58)) return false;
  *out = *d;
  size_t* n[4] = {&out->nx, &out->ny, &out->nz, &out->nw};
  ptrdiff_t* st[4] = {&out->sx, &out->sy, &out->sz, &out->sw};
  for (uint i = 0; i < 4; i++) {
    *n[i] = i < dims - 1 ? 4 : i == dims - 1 ? 4 * count : 0;
    *st[i] = 0;
  }
  return true;
}

extern "C" size_t zfpb_encode_blocks(const zfpb_desc* d, uint dims, size_t count, const void* d_blocks,
                                     void* d_stream, size_t capacity, uint64_t* d_block_offsets, void* cuda_stream) {
  zfpb_desc f;
  if (!blocks_desc(d, dims, count, &f)) return fail(zfpb::ERR_ARGS);
  return zfpb_compress_device(&f, d_blocks, d_stream, capacity, d_block_offsets, cuda_stream);
}

extern "C" size_t zfpb_decode_blocks(const zfpb_desc* d, uint dims, size_t count, const void* d_stream,
                                     size_t stream_bytes, void* d_blocks, const uint64_t* d_block_offsets,
                                     void* cuda_stream) {
  zfpb_desc f;
  if (!blocks_desc(d, dims, count, &f)) return fail(zfpb::ERR_ARGS);
  return zfpb_decompress_device(&f, d_stream, stream_bytes, d_blocks, d_block_offsets, cuda_stream);
}
