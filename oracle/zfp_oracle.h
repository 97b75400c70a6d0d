/*
 * CPU oracle for the ZFP compress/decompress path: a restatement of
 * zfp-rs 1.0.1 (src/bitstream/core.rs, src/codec/, src/compress.rs,
 * src/decompress.rs, src/field_plan.rs, src/header.rs).
 *
 * TEST INFRASTRUCTURE ONLY.  The GPU library never links, loads or calls
 * anything declared here; only the tests, the smoke check and the
 * benchmark's CPU-baseline leg do, and only as the checker.
 */
#ifndef ZFP_ORACLE_H
#define ZFP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as zfp_field (zfp-rs-ffi/src/abi.rs:220-233); `data` points at
 * element [0,0,0,0], strides are in elements, 0 selects the natural stride. */
typedef struct {
  int type; /* 1 int32, 2 int64, 3 float, 4 double */
  size_t nx, ny, nz, nw;
  ptrdiff_t sx, sy, sz, sw;
  void* data;
} orc_field;

/* Expert parameters plus rounding (zfp-rs src/config.rs:163-174, :115-138). */
typedef struct {
  uint32_t minbits, maxbits, maxprec;
  int32_t minexp;
  int rounding; /* 0 never, 1 first, 2 last */
  int tight;    /* tight_error */
} orc_config;

void* orc_stream_open(uint64_t* words, size_t nwords);
void orc_stream_close(void* s);
void orc_stream_rewind(void* s);
uint64_t orc_stream_wtell(void* s);
uint64_t orc_stream_rtell(void* s);
void orc_stream_rseek(void* s, uint64_t offset);
void orc_stream_wseek(void* s, uint64_t offset);
uint64_t orc_stream_write_bits(void* s, uint64_t value, uint32_t n);
uint64_t orc_stream_read_bits(void* s, uint32_t n);
uint32_t orc_stream_flush(void* s);
uint32_t orc_stream_align(void* s);
size_t orc_stream_size(void* s); /* bytes up to the cursor's word */

/* Whole-field compression.  threads <= 1: serial (compress.rs:22-116);
 * threads > 1: chunked like C OpenMP then concatenated at bit granularity
 * (compress.rs:132-245).  Returns the stream size in bytes, or -1 when the
 * buffer overflowed. */
long long orc_compress(void* s, const orc_field* f, const orc_config* c, int threads);
/* Whole-field decompression (decompress.rs:27-196).  threads > 1 and
 * strides that cannot alias: fixed-rate streams decode in seek-parallel
 * chunks (decompress.rs:205-330), other streams of 2-4 dimensions through the
 * reader/worker pipeline (decompress/pipeline.rs:193-229); otherwise serial.
 * Returns bytes consumed, or -1 when the stream was truncated. */
long long orc_decompress(void* s, orc_field* f, const orc_config* c, int threads);

/* Header (header.rs:72-173).  mask: 1 magic, 2 meta, 4 mode.  Returns bits
 * written/read, or 0 on failure.  orc_read_header fills type and dims of f
 * and the four expert parameters of c when the mask asks for them. */
size_t orc_write_header(void* s, const orc_field* f, const orc_config* c, unsigned mask);
size_t orc_read_header(void* s, orc_field* f, orc_config* c, unsigned mask);

/* Block codec on one strided block (codec/block/strided.rs).  lengths may be
 * NULL for a whole block.  Returns the bits written or read. */
size_t orc_encode_block(void* s, int type, int dims, const void* data, const ptrdiff_t* strides,
                        const size_t* lengths, const orc_config* c);
size_t orc_decode_block(void* s, int type, int dims, void* data, const ptrdiff_t* strides,
                        const size_t* lengths, const orc_config* c);

/* Helpers shared with the tests. */
uint32_t orc_block_bits(const orc_config* c, int type, int dims);      /* config.rs:670-686 */
size_t orc_maximum_size(const orc_config* c, const orc_field* f);     /* config.rs:642-658 */
int orc_mode(const orc_config* c);                                    /* config.rs:469-527 */
uint64_t orc_mode_bits(const orc_config* c);                          /* config.rs:570-596 */

#ifdef __cplusplus
}
#endif

#endif
