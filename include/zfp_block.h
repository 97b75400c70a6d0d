/*
 * zfp_block.h -- block-level calls of libzfp_b200.so: one 4^d block coded at
 * a zfp_stream's bit-stream cursor, as zfp-rs-ffi exports them
 * (zfp-rs-ffi/src/block.rs:34-776; codec in src/codec/block/strided.rs:
 * 420-690) and C zfp declares them.  zfp-rs-ffi's cbindgen header leaves
 * these out; the symbols and signatures are the ones its library exports.
 *
 * Every call uses the stream's compression parameters and rounding, appends
 * (encode) or reads (decode) exactly the block's bits at the cursor without
 * flushing, and returns that number of bits, or 0 for a NULL stream, bit
 * stream or block pointer, or (partial calls) a length outside 1..4.  The
 * block is coded on the GPU: each call is one small device round trip, so
 * code many blocks with zfpb_encode_blocks / zfpb_decode_blocks
 * (zfp_b200.h).  Block data may be host or device memory.
 *
 * Layouts: a contiguous block holds its 4^d values x fastest (element
 * strides 1, 4, 16, 64); strided calls take the element strides of the
 * caller's array (any sign; 0 repeats one element); partial calls code the
 * first nx x ny x nz x nw values (each 1..4), padded as zfp pads partial
 * blocks, and decode writes only those values.
 *
 * zfp_promote_* / zfp_demote_* (zfp-rs-ffi/src/promote.rs:11-59) map one
 * block of 4^dims 8- or 16-bit integers to the int32 range and back
 * (clamped), on host arrays.
 */
#ifndef ZFP_B200_BLOCK_H
#define ZFP_B200_BLOCK_H

#include "zfp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Contiguous block encoders (block.rs:34-133). */
size_t zfp_encode_block_int32_1(zfp_stream* stream, const int32_t* block);
size_t zfp_encode_block_int32_2(zfp_stream* stream, const int32_t* block);
size_t zfp_encode_block_int32_3(zfp_stream* stream, const int32_t* block);
size_t zfp_encode_block_int32_4(zfp_stream* stream, const int32_t* block);
size_t zfp_encode_block_int64_1(zfp_stream* stream, const int64_t* block);
size_t zfp_encode_block_int64_2(zfp_stream* stream, const int64_t* block);
size_t zfp_encode_block_int64_3(zfp_stream* stream, const int64_t* block);
size_t zfp_encode_block_int64_4(zfp_stream* stream, const int64_t* block);
size_t zfp_encode_block_float_1(zfp_stream* stream, const float* block);
size_t zfp_encode_block_float_2(zfp_stream* stream, const float* block);
size_t zfp_encode_block_float_3(zfp_stream* stream, const float* block);
size_t zfp_encode_block_float_4(zfp_stream* stream, const float* block);
size_t zfp_encode_block_double_1(zfp_stream* stream, const double* block);
size_t zfp_encode_block_double_2(zfp_stream* stream, const double* block);
size_t zfp_encode_block_double_3(zfp_stream* stream, const double* block);
size_t zfp_encode_block_double_4(zfp_stream* stream, const double* block);

/* Contiguous block decoders (block.rs:135-236). */
size_t zfp_decode_block_int32_1(zfp_stream* stream, int32_t* block);
size_t zfp_decode_block_int32_2(zfp_stream* stream, int32_t* block);
size_t zfp_decode_block_int32_3(zfp_stream* stream, int32_t* block);
size_t zfp_decode_block_int32_4(zfp_stream* stream, int32_t* block);
size_t zfp_decode_block_int64_1(zfp_stream* stream, int64_t* block);
size_t zfp_decode_block_int64_2(zfp_stream* stream, int64_t* block);
size_t zfp_decode_block_int64_3(zfp_stream* stream, int64_t* block);
size_t zfp_decode_block_int64_4(zfp_stream* stream, int64_t* block);
size_t zfp_decode_block_float_1(zfp_stream* stream, float* block);
size_t zfp_decode_block_float_2(zfp_stream* stream, float* block);
size_t zfp_decode_block_float_3(zfp_stream* stream, float* block);
size_t zfp_decode_block_float_4(zfp_stream* stream, float* block);
size_t zfp_decode_block_double_1(zfp_stream* stream, double* block);
size_t zfp_decode_block_double_2(zfp_stream* stream, double* block);
size_t zfp_decode_block_double_3(zfp_stream* stream, double* block);
size_t zfp_decode_block_double_4(zfp_stream* stream, double* block);

/* Strided block encoders (block.rs:239-362). */
size_t zfp_encode_block_strided_int32_1(zfp_stream* stream, const int32_t* p, ptrdiff_t sx);
size_t zfp_encode_block_strided_int32_2(zfp_stream* stream, const int32_t* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_block_strided_int32_3(zfp_stream* stream, const int32_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_block_strided_int32_4(zfp_stream* stream, const int32_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_encode_block_strided_int64_1(zfp_stream* stream, const int64_t* p, ptrdiff_t sx);
size_t zfp_encode_block_strided_int64_2(zfp_stream* stream, const int64_t* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_block_strided_int64_3(zfp_stream* stream, const int64_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_block_strided_int64_4(zfp_stream* stream, const int64_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_encode_block_strided_float_1(zfp_stream* stream, const float* p, ptrdiff_t sx);
size_t zfp_encode_block_strided_float_2(zfp_stream* stream, const float* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_block_strided_float_3(zfp_stream* stream, const float* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_block_strided_float_4(zfp_stream* stream, const float* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_encode_block_strided_double_1(zfp_stream* stream, const double* p, ptrdiff_t sx);
size_t zfp_encode_block_strided_double_2(zfp_stream* stream, const double* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_block_strided_double_3(zfp_stream* stream, const double* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_block_strided_double_4(zfp_stream* stream, const double* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);

/* Partial strided block encoders (block.rs:365-506). */
size_t zfp_encode_partial_block_strided_int32_1(zfp_stream* stream, const int32_t* p, size_t nx, ptrdiff_t sx);
size_t zfp_encode_partial_block_strided_int32_2(zfp_stream* stream, const int32_t* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_partial_block_strided_int32_3(zfp_stream* stream, const int32_t* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_partial_block_strided_int32_4(zfp_stream* stream, const int32_t* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_encode_partial_block_strided_int64_1(zfp_stream* stream, const int64_t* p, size_t nx, ptrdiff_t sx);
size_t zfp_encode_partial_block_strided_int64_2(zfp_stream* stream, const int64_t* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_partial_block_strided_int64_3(zfp_stream* stream, const int64_t* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_partial_block_strided_int64_4(zfp_stream* stream, const int64_t* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_encode_partial_block_strided_float_1(zfp_stream* stream, const float* p, size_t nx, ptrdiff_t sx);
size_t zfp_encode_partial_block_strided_float_2(zfp_stream* stream, const float* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_partial_block_strided_float_3(zfp_stream* stream, const float* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_partial_block_strided_float_4(zfp_stream* stream, const float* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_encode_partial_block_strided_double_1(zfp_stream* stream, const double* p, size_t nx, ptrdiff_t sx);
size_t zfp_encode_partial_block_strided_double_2(zfp_stream* stream, const double* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_encode_partial_block_strided_double_3(zfp_stream* stream, const double* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_encode_partial_block_strided_double_4(zfp_stream* stream, const double* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);

/* Strided block decoders (block.rs:509-632). */
size_t zfp_decode_block_strided_int32_1(zfp_stream* stream, int32_t* p, ptrdiff_t sx);
size_t zfp_decode_block_strided_int32_2(zfp_stream* stream, int32_t* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_block_strided_int32_3(zfp_stream* stream, int32_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_block_strided_int32_4(zfp_stream* stream, int32_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_decode_block_strided_int64_1(zfp_stream* stream, int64_t* p, ptrdiff_t sx);
size_t zfp_decode_block_strided_int64_2(zfp_stream* stream, int64_t* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_block_strided_int64_3(zfp_stream* stream, int64_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_block_strided_int64_4(zfp_stream* stream, int64_t* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_decode_block_strided_float_1(zfp_stream* stream, float* p, ptrdiff_t sx);
size_t zfp_decode_block_strided_float_2(zfp_stream* stream, float* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_block_strided_float_3(zfp_stream* stream, float* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_block_strided_float_4(zfp_stream* stream, float* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_decode_block_strided_double_1(zfp_stream* stream, double* p, ptrdiff_t sx);
size_t zfp_decode_block_strided_double_2(zfp_stream* stream, double* p, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_block_strided_double_3(zfp_stream* stream, double* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_block_strided_double_4(zfp_stream* stream, double* p, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);

/* Partial strided block decoders (block.rs:635-776). */
size_t zfp_decode_partial_block_strided_int32_1(zfp_stream* stream, int32_t* p, size_t nx, ptrdiff_t sx);
size_t zfp_decode_partial_block_strided_int32_2(zfp_stream* stream, int32_t* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_partial_block_strided_int32_3(zfp_stream* stream, int32_t* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_partial_block_strided_int32_4(zfp_stream* stream, int32_t* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_decode_partial_block_strided_int64_1(zfp_stream* stream, int64_t* p, size_t nx, ptrdiff_t sx);
size_t zfp_decode_partial_block_strided_int64_2(zfp_stream* stream, int64_t* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_partial_block_strided_int64_3(zfp_stream* stream, int64_t* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_partial_block_strided_int64_4(zfp_stream* stream, int64_t* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_decode_partial_block_strided_float_1(zfp_stream* stream, float* p, size_t nx, ptrdiff_t sx);
size_t zfp_decode_partial_block_strided_float_2(zfp_stream* stream, float* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_partial_block_strided_float_3(zfp_stream* stream, float* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_partial_block_strided_float_4(zfp_stream* stream, float* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);
size_t zfp_decode_partial_block_strided_double_1(zfp_stream* stream, double* p, size_t nx, ptrdiff_t sx);
size_t zfp_decode_partial_block_strided_double_2(zfp_stream* stream, double* p, size_t nx, size_t ny, ptrdiff_t sx, ptrdiff_t sy);
size_t zfp_decode_partial_block_strided_double_3(zfp_stream* stream, double* p, size_t nx, size_t ny, size_t nz, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz);
size_t zfp_decode_partial_block_strided_double_4(zfp_stream* stream, double* p, size_t nx, size_t ny, size_t nz, size_t nw, ptrdiff_t sx, ptrdiff_t sy, ptrdiff_t sz, ptrdiff_t sw);

/* Promotion / demotion of one block (promote.rs:51-59). */
void zfp_promote_int8_to_int32(int32_t* oblock, const int8_t* iblock, uint dims);
void zfp_promote_uint8_to_int32(int32_t* oblock, const uint8_t* iblock, uint dims);
void zfp_promote_int16_to_int32(int32_t* oblock, const int16_t* iblock, uint dims);
void zfp_promote_uint16_to_int32(int32_t* oblock, const uint16_t* iblock, uint dims);
void zfp_demote_int32_to_int8(int8_t* oblock, const int32_t* iblock, uint dims);
void zfp_demote_int32_to_uint8(uint8_t* oblock, const int32_t* iblock, uint dims);
void zfp_demote_int32_to_int16(int16_t* oblock, const int32_t* iblock, uint dims);
void zfp_demote_int32_to_uint16(uint16_t* oblock, const int32_t* iblock, uint dims);

#ifdef __cplusplus
}
#endif

#endif /* ZFP_B200_BLOCK_H */
