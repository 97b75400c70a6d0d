// Host-side engine interface between the C ABI (zfp_abi.cpp) and the CUDA
// kernels.  Plain structs only; every pointer named d_* is device memory.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace zfpb {

typedef unsigned long long u64;
typedef unsigned int u32;
typedef long long i64;

// Field tiling in elements: data points at element [0,0,0,0] (field.rs:541-588).
struct FieldGeom {
  i64 s[4];    // effective strides
  u64 n[4];    // dimensions
  u64 b[4];    // blocks per axis
  u64 nblocks;
  int vec_ok;  // full-block rows are 16-byte aligned contiguous runs
  // ceil(2^64 / b[d]) for d < 3 (0 when b[d] == 1): the block index of a
  // field of fewer than 2^32 blocks splits into per-axis block coordinates
  // by multiply-high instead of 64-bit division (set by fill_block_inverses).
  u64 inv[3];
};

inline void fill_block_inverses(FieldGeom& g) {
  for (int d = 0; d < 3; d++) g.inv[d] = g.b[d] > 1 ? ~0ull / g.b[d] + 1 : 0ull;
}

enum : unsigned { FLAG_TRUNCATED = 1u, FLAG_BAD_INDEX = 2u, FLAG_BAD_HEADER = 4u };

struct CodecParams {
  u32 minbits, maxbits, maxprec;
  int minexp;
  int rounding;
  int tight;
};

struct EncodeFixedArgs {
  const void* data;
  FieldGeom f;
  CodecParams c;
  u64* out;
  u64 start;      // stream bit where the first block begins
  u64 init_word;  // stream bits already in the start word, below start % 64
  u64 blocks_per_cta;
};

struct EncodeVarArgs {
  const void* data;
  FieldGeom f;
  CodecParams c;
  u64* slots;
  u64 slot_words;
  u32* lengths;
};

// Speculative parallel walk of a variable-rate stream without an index (see
// k_spec_walk).  Positions are bits relative to `start`; segment s's list and
// fix hold them relative to the segment's first bit (a fix may run on into
// later segments; cap steps of at most a 4^4-double block stay below 2^32).
struct SpecWalkArgs {
  const u64* stream;
  u64 stream_len;  // words
  u64 start;
  CodecParams c;
  u64 nseg, seg_bits, end_bits, cap;
  u64 lead;         // bits walked before a segment's first bit, unlisted
  u32* list;        // nseg * cap: the speculative walk's positions in the segment
  u32* list_len;
  u64* exit_spec;   // first position at or past the segment's end, speculative walk
  u32* fix;         // nseg * cap: from the exit of segment s - 1 up to a listed position
  u32* fix_len;
  u32* sync_t;      // segment whose list the fix joined (nseg: none, the walk reached the end)
  u32* sync_j;      // index in that list
  u64* fix_exit;    // where a fix that joined no list stopped
  unsigned* flags;  // [0] a list or fix overflowed
};

// One run of true block positions: `count` entries of segment `seg`'s list
// (kind 0) or fix (kind 1) from index `from`, placed from off[dst].
struct SpecPiece {
  u32 kind, seg, from, count;
  u64 dst;
};

struct DecodeArgs {
  void* data;
  FieldGeom f;
  CodecParams c;
  const u64* stream;
  u64 stream_len;  // words
  u64 start;
  u64* offsets;    // nblocks + 1 entries, relative to start (variable path)
  unsigned* flags;
  // Fields whose strides may alias: owner[e - imin] is 1 + the last block (in
  // stream order) that holds element e, and only that block stores it, so the
  // result is that of a serial decode (zfp-rs decompress.rs:153-186).
  u64* owner;
  i64 imin;
};

// Scratch of the two-kernel decoder: plane k of block i at planes[k * stride + i].
struct SplitArgs {
  u64* planes;
  u64 stride;
  u64* heads;
};

// Whether two index tuples of the field can address the same element
// (zfp-rs field_plan.rs:92-118).
bool strides_may_alias(const FieldGeom& f, int dims);

// One compress or decompress call.
struct Call {
  int type;  // 1 int32, 2 int64, 3 float, 4 double
  int dims;  // 1..4
  FieldGeom f;
  CodecParams c;
};

// Result codes of the engine entry points.
enum Status : int { OK = 0, ERR_OVERFLOW = 1, ERR_TRUNCATED = 2, ERR_CUDA = 3, ERR_ARGS = 4,
                   // Candidate block offsets did not match the stream; call again without them.
                   ERR_BAD_INDEX = 5,
                   // The field needs more scratch than the no-allocation entry point has.
                   ERR_TOO_LARGE = 6,
                   // A batch item's stream does not begin with the header its description gives.
                   ERR_HEADER = 7 };

// Whether every block takes exactly c.maxbits bits (minbits == maxbits and no
// block can exceed the budget, zfp-rs config.rs:670-686).
bool fixed_size_blocks(const Call& call);
u32 block_bits(const CodecParams& c, int type, int dims);

// Compress a device-resident field into d_out (cap words), from bit `start`
// whose word already holds `init_word` below start % 64.  On OK, *end_bit is
// the bit after the last block.  d_offsets (optional, nblocks + 1 entries)
// receives each block's start relative to `start`.
Status compress(const Call& call, const void* d_field, u64* d_out, u64 cap, u64 start, u64 init_word,
                u64* end_bit, u64* d_offsets, cudaStream_t s);

// Decompress into a device-resident field from d_in (len words) at bit
// `start`.  d_offsets (optional) holds candidate block offsets; they are used
// only if they check out as exactly those of a serial decode, else the call
// returns ERR_BAD_INDEX (the field may be partly written).  Without them,
// variable-size streams are walked for their offsets.  On OK or
// ERR_TRUNCATED, *end_bit is the bit after the last block.
Status decompress(const Call& call, const u64* d_in, u64 len, u64 start, void* d_field, u64* end_bit,
                  const u64* d_offsets, cudaStream_t s);

// Host buffers, copies overlapped with coding (fields with natural strides).
// compress_host: h_field is the host field (element [0,0,0,0]), d_field a
// device buffer of the same size; the stream goes to the host words h_out
// (cap words) through d_out, from bit `start` (< 64) whose word holds
// init_word.  decompress_host: h_in / d_in (len words) hold / receive the
// stream; block offsets are needed unless blocks are fixed-size.  Both return
// ERR_ARGS when the field does not qualify (then use compress / decompress).
bool natural_strides(const Call& call);
Status compress_host(const Call& call, const void* h_field, void* d_field, u64* h_out, u64* d_out, u64 cap,
                     u64 start, u64 init_word, u64* end_bit, u64* d_offsets, cudaStream_t s);
Status decompress_host(const Call& call, const u64* h_in, u64* d_in, u64 len, u64 start, void* h_field,
                       void* d_field, u64* end_bit, const u64* d_offsets, cudaStream_t s);

// ---- batches ---------------------------------------------------------------
//
// A batch codes many arrays of mixed type, dimensionality, size and mode in a
// few launches over a flattened block work list.  Work is cut into tiles
// (up to one CTA's worth of consecutive blocks of one array); the arrays of one
// (type, dims) class share one launch per kernel.

// Device-side descriptor of one array of a batch.
struct BatchItem {
  FieldGeom f;
  CodecParams c;
  void* data;        // the field (compress: read, decompress: written)
  u64* stream;       // compress: written from bit 0; decompress: read from bit 0
  u64 stream_words;  // compress: capacity; decompress: stream length
  u64* index;        // optional block offsets (nblocks + 1): compress writes, decompress tries
  u64 slot_base;     // compress: first word of this array's block slots
  u64 slot_words;    // compress: words per block slot
  u64 len_base;      // this array's nblocks + 1 entries in the batch lengths / offsets
  u64 plane_base;    // 3D decompress: column of block 0 in the plane scratch
  u32 fixed;         // every block takes exactly maxbits bits
  u32 walk;          // decompress: offsets come from the batch walker
  u64 start;         // bit of the first block; the stream's words below it (and the bits of
  u64 hdr[3];        //   word start / 64 below start % 64) are the header hdr
};

// Blocks [first, first + count) of items[item].
struct BatchTile {
  u32 item;
  u32 count;
  u64 first;
};

struct BatchArgs {
  const BatchItem* items;
  const BatchTile* tiles;  // this launch's tiles, one per CTA
  u64* slots;
  u32* lengths;
  u64* offsets;
  unsigned* flags;         // per item: FLAG_TRUNCATED, FLAG_BAD_INDEX
  u64* planes;             // 3D decompress plane scratch, plane k of column j at planes[k * plane_stride + j]
  u64 plane_stride;
  u64* heads;
  const u32* walk_items;   // items whose offsets the walker finds
  u32 nwalk;
  u64* walk_planes;        // one plane store per walking thread
};

// One array of a batch call (host side).
struct BatchJob {
  Call call;
  void* field;
  u64* stream;
  u64 stream_words;
  u64* index;          // block offsets relative to start_bit
  u64 start_bit = 0;   // a zfp header of start_bit bits (<= 148) precedes the blocks:
  u64 hdr[3] = {};     //   compress writes hdr there, decompress checks it
  u64 end_bit;         // out: stream bits written / read
  Status status;       // out
};

// Compress / decompress every job; each job's status and end_bit are set.
// Returns OK when every job succeeded.  Plans (tables, scratch and a CUDA
// graph of the launches) are cached by the jobs' contents, so calling again
// with the same jobs replays the graph.
Status compress_batch(BatchJob* jobs, size_t n, cudaStream_t s);
Status decompress_batch(BatchJob* jobs, size_t n, cudaStream_t s);

// The same, asynchronous: batch_launch plans and launches on s and returns;
// once batch_ready, batch_collect writes every job's result to out (in the
// order given).  A BatchRun keeps its scratch for the next launch; one run
// at a time per BatchRun.
struct BatchRun;
BatchRun* batch_run_create();
void batch_run_destroy(BatchRun* r);
Status batch_launch(BatchRun* r, const BatchJob* jobs, size_t n, bool compress, cudaStream_t s);
bool batch_ready(BatchRun* r);
// Map `bytes` of batch scratch ahead of use (kept by the scratch pool).
bool batch_reserve(u64 bytes, cudaStream_t s);
Status batch_collect(BatchRun* r, BatchJob* out);

// Device scratch a job needs inside a batch beyond its own buffers (block
// slots for compress, plane scratch for a 3D decompress), for admission.
u64 batch_scratch_bytes(const Call& call, bool compress);

// Kernel launchers, one instantiation per scalar type (zfpb_inst_*.cu).
template <class T> struct Launch {
  static cudaError_t encode_fixed(const Call& call, const EncodeFixedArgs& a, u64 ctas, int threads,
                                  size_t smem, cudaStream_t s);
  static cudaError_t encode_var(const Call& call, const EncodeVarArgs& a, cudaStream_t s);
  static cudaError_t decode_fixed(const Call& call, const DecodeArgs& a, cudaStream_t s);
  static cudaError_t decode_var(const Call& call, const DecodeArgs& a, cudaStream_t s);
  static cudaError_t walk(const Call& call, const DecodeArgs& a, cudaStream_t s);
  // Passes of the speculative walk (dims 1-3): the walk, one fix pass, the
  // blocks past the last segment.
  static cudaError_t spec_walk(int dims, const SpecWalkArgs& a, cudaStream_t s);
  static cudaError_t spec_fix(int dims, const SpecWalkArgs& a, cudaStream_t s);
  static cudaError_t spec_tail(int dims, const SpecWalkArgs& a, u64* off, u64 idx, u64 n, u64 x, cudaStream_t s);
  // Batches: one launch over `ntiles` tiles of (T, dims) arrays.
  static cudaError_t encode_batch(int dims, const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s);
  static cudaError_t decode_batch(int dims, const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s);
  static cudaError_t parse_batch(const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s);
  static cudaError_t finish_batch(const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s);
  static cudaError_t walk_batch(int dims, const BatchArgs& a, cudaStream_t s);
  // Two-kernel decoder, 3D fields only.
  static cudaError_t parse(const Call& call, const DecodeArgs& a, const SplitArgs& sa, bool var, cudaStream_t s);
  static cudaError_t finish(const Call& call, const DecodeArgs& a, const SplitArgs& sa, cudaStream_t s);
};

// Compress from bit 0 of d_out (cap words) without allocating device memory:
// scratch is a fixed static device array of noalloc_scratch_bytes() bytes.
// Returns ERR_TOO_LARGE for a field whose scratch does not fit.  Synchronous.
Status compress_noalloc(const Call& call, const void* d_field, u64* d_out, u64 cap, u64* end_bit,
                        cudaStream_t s);
u64 noalloc_scratch_bytes();

// Per-kernel timing: events on the launching stream around every launch.
void timing_enable(bool on);
int timing_read(double* ms, unsigned long long* counts, int n);

// Shared-memory bytes of plane storage per thread for a scalar type/dims.
size_t plane_bytes(int type, int dims);

}  // namespace zfpb
