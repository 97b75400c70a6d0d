/*
 * zfp_b200.h -- extensions of libzfp_b200.so beyond the zfp.h ABI.
 *
 * None of these replaces a zfp.h function; each gives C callers something
 * zfp-rs offers only through its Rust API, or a device-memory entry point.
 */
#ifndef ZFP_B200_EXT_H
#define ZFP_B200_EXT_H

#include "zfp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Coefficient rounding of a stream opened with zfp_stream_open, as zfp-rs's
 * per-call ZfpRounding (src/config.rs:115-138), which zfp-rs-ffi instead fixes
 * at build time (zfp-rs-ffi/src/stream.rs:12-16).  rounding: ZFP_ROUND_NEVER,
 * ZFP_ROUND_FIRST or ZFP_ROUND_LAST.  Returns zfp_false for an invalid value.
 * New streams round ZFP_ROUND_NEVER without tight error. */
zfp_bool zfp_stream_set_rounding(zfp_stream* stream, int rounding, zfp_bool tight_error);
int zfp_stream_rounding(const zfp_stream* stream, zfp_bool* tight_error);

/* Status of the last failed call on this thread: 0 none, 1 buffer too small,
 * 2 truncated stream, 3 CUDA error, 4 invalid arguments, 6 field too large
 * for zfpb_compress_device_noalloc, 7 a batch item's stream lacks its header. */
int zfpb_last_error(void);

/* A field and codec parameters in one plain struct for the device API. */
typedef struct zfpb_desc {
  zfp_type type;
  size_t nx, ny, nz, nw;       /* zero past the dimensionality */
  ptrdiff_t sx, sy, sz, sw;    /* element strides, 0 = natural */
  uint minbits, maxbits, maxprec;
  int32_t minexp;
  int rounding;                /* ZFP_ROUND_NEVER / _FIRST / _LAST */
  zfp_bool tight_error;
} zfpb_desc;

/* Compress a device-resident field (d_field points at element [0,0,0,0]) into
 * the device buffer d_stream of `capacity` bytes (8-byte aligned), starting at
 * bit 0 with no header.  d_block_offsets, if not NULL, receives nblocks + 1
 * bit offsets: where each block starts and where the last one ends.
 * cuda_stream is a cudaStream_t (NULL: the default stream).  Returns the
 * stream size in bytes, or 0 on failure; the call returns once the stream is
 * complete. */
size_t zfpb_compress_device(const zfpb_desc* desc, const void* d_field, void* d_stream, size_t capacity,
                            uint64_t* d_block_offsets, void* cuda_stream);

/* Decompress `bytes` bytes of a headerless stream at d_stream into the
 * device-resident field d_field.  d_block_offsets (optional) are candidate
 * block offsets, e.g. from zfpb_compress_device; they are used only if they
 * match the stream, else the offsets are recomputed from the stream.
 * Returns the bytes consumed, or 0 on failure (e.g. a truncated stream). */
size_t zfpb_decompress_device(const zfpb_desc* desc, const void* d_stream, size_t bytes, void* d_field,
                              const uint64_t* d_block_offsets, void* cuda_stream);

/* Compress without allocating device memory.
 *
 * No counterpart in the reference: zfp-rs allocates its chunk buffers itself.
 * This entry point is for callers that cannot have the library call
 * cudaMalloc: a host application that has reserved all of its device memory
 * for its own pool (so an allocation would fail or evict its data), or a
 * latency-critical loop that cannot absorb cudaMalloc's implicit device-wide
 * synchronization.  It behaves as zfpb_compress_device (same stream bytes,
 * no header, no index) but takes its scratch from a fixed 16 MiB device array
 * inside the library, which every device that loads the library holds until
 * the process exits.  Limit: fields whose variable-rate scratch (one slot of
 * zfp_block_maximum_size bits per block, plus 12 bytes per block) exceeds
 * 16 MiB are rejected: the call returns 0 and zfpb_last_error() returns 6.
 * Fixed-size blocks (fixed-rate mode) need no scratch and have no limit.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  All calls share the array: calls
 * whose kernels overlap on the GPU (from several host threads or streams)
 * race and must be serialized by the caller.  The call returns once the
 * stream is complete. */
size_t zfpb_compress_device_noalloc(const zfpb_desc* desc, const void* d_field, void* d_stream,
                                    size_t capacity, void* cuda_stream);

/* ---- batches ------------------------------------------------------------
 *
 * No counterpart in the reference (zfp-rs codes one field per call).  Many
 * device-resident arrays of mixed type, dimensionality, size and mode are
 * coded in a few launches over one flattened list of blocks, instead of one
 * set of launches (and one synchronisation) per array.  Each array's stream
 * and decoded values are exactly those of zfpb_compress_device /
 * zfpb_decompress_device for that array alone.  The first call with a given
 * item list plans it (tables, scratch, per-class CTA sizes tuned by timing)
 * and records its launches as a CUDA graph; a later call with the same item
 * list (same descriptors and buffers) replays the graph.  Up to four plans are
 * kept per process. */
typedef struct zfpb_batch_item {
  zfpb_desc desc;
  void* d_field;              /* compress: read; decompress: written */
  void* d_stream;             /* 8-byte aligned; compress: written from bit 0; decompress: read */
  size_t stream_bytes;        /* compress: capacity; decompress: stream size */
  uint64_t* d_block_offsets;  /* optional nblocks + 1 block offsets, as for zfpb_compress_device:
                                 compress writes them, decompress uses them if they match;
                                 relative to the first block (after the header, if any) */
  uint header_mask;           /* ZFP_HEADER_* bits, 0 = none.  Compress: the stream begins with
                                 the zfp_write_header(mask) header of desc's field and mode;
                                 decompress: the stream must begin with that header (else
                                 status 7 and result 0), and the blocks follow it */
  size_t result;              /* out: stream bytes written / consumed (header included), 0 on failure */
  int status;                 /* out: 0, or the zfpb_last_error code of this item */
} zfpb_batch_item;

/* Compress / decompress every item (blocks from bit 0, or after the item's
 * header).  Returns the number of items that succeeded; the call returns once
 * all are done. */
size_t zfpb_compress_batch(zfpb_batch_item* items, size_t n, void* cuda_stream);
size_t zfpb_decompress_batch(zfpb_batch_item* items, size_t n, void* cuda_stream);

/* ---- serving ------------------------------------------------------------
 *
 * No counterpart in the reference.  A serving loop for streams of compress /
 * decompress requests on device-resident buffers.  Requests are admitted in
 * arrival order while the device bytes they hold (field, stream and batch
 * scratch) fit in the budget; admitted requests are coded together in the
 * next batch as soon as one of `lanes` CUDA streams is free, so requests that
 * arrive while others run join the next batch and overlap with the batches in
 * flight.  Each result equals that of the single-array device call.  The
 * caller keeps the buffers alive until the request is returned by poll. */
typedef struct zfpb_server zfpb_server;

typedef struct zfpb_request_done {
  uint64_t tag;       /* as given to zfpb_server_submit */
  size_t result;      /* stream bytes written / consumed, 0 on failure */
  int status;         /* 0, or a zfpb_last_error code */
  double queue_ms;    /* submit -> launch */
  double latency_ms;  /* submit -> result available */
} zfpb_request_done;

/* budget_bytes: device memory that admitted requests may hold at once;
 * lanes: batches in flight at once (0: 4); max_batch: requests per batch
 * (0: 4096); batch_bytes: uncompressed bytes per batch, a larger request
 * running alone (0: 64 MiB).  Returns NULL on failure. */
zfpb_server* zfpb_server_create(size_t budget_bytes, int lanes, size_t max_batch, size_t batch_bytes);
/* Queue one request (decompress = 0: compress item->d_field into
 * item->d_stream).  Returns 0 if the request is invalid or alone exceeds the
 * budget. */
int zfpb_server_submit(zfpb_server* s, const zfpb_batch_item* item, int decompress, uint64_t tag);
/* Finished requests, up to max, waiting up to wait_ms for the first one. */
size_t zfpb_server_poll(zfpb_server* s, zfpb_request_done* out, size_t max, int wait_ms);
/* Submitted requests not yet returned by zfpb_server_poll. */
size_t zfpb_server_outstanding(zfpb_server* s);
/* Finish all submitted work, then free the server. */
void zfpb_server_destroy(zfpb_server* s);

/* Per-kernel timing for profiling: when enabled, every kernel launch of the
 * library is bracketed by CUDA events on its stream.  zfpb_timing_enable
 * clears the totals.  zfpb_timing_read fills, per kernel kind, the summed
 * milliseconds and the launch count, and returns the number of kinds:
 * 0 encode_fixed, 1 encode_var, 2 scan, 3 pack, 4 decode_fixed,
 * 5 decode_var, 6 walk, 7 claim, 8 offsets, 9 parse, 10 finish (the two
 * halves of the decoder used for 3D fields). */
void zfpb_timing_enable(int on);
int zfpb_timing_read(double* ms, unsigned long long* counts, int n);

/* Many whole blocks in one call: the batched form of the block-level calls
 * of zfp_block.h (zfp-rs-ffi/src/block.rs:34-236, one block per call there).
 * d_blocks holds `count` blocks of 4^dims values back to back (block i at
 * element i * 4^dims, each laid out as zfp_encode_block_<type>_<dims> reads
 * it); desc gives the type and the codec parameters (its sizes and strides
 * are ignored).  zfpb_encode_blocks writes the stream that `count` calls of
 * zfp_encode_block_<type>_<dims> on one stream followed by a flush write,
 * from bit 0 of d_stream (capacity bytes), and returns its size in bytes
 * (0 on failure); d_block_offsets (optional, count + 1 entries) receives
 * each block's first bit.  zfpb_decode_blocks decodes such a stream back
 * into d_blocks and returns the bytes consumed.  All buffers are device
 * memory; the calls return once the work is done. */
size_t zfpb_encode_blocks(const zfpb_desc* desc, uint dims, size_t count, const void* d_blocks, void* d_stream,
                          size_t capacity, uint64_t* d_block_offsets, void* cuda_stream);
size_t zfpb_decode_blocks(const zfpb_desc* desc, uint dims, size_t count, const void* d_stream,
                          size_t stream_bytes, void* d_blocks, const uint64_t* d_block_offsets, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* ZFP_B200_EXT_H */
