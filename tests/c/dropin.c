/*
 * A C program written against include/zfp.h alone, linked with
 * libzfp_b200.so: what an existing user of the zfp-rs C ABI compiles.
 *
 * The _Static_asserts pin the struct layouts to those of zfp-rs-ffi
 * (src/abi.rs:122-155 zfp_execution / zfp_stream, :160-212 zfp_config,
 * :220-233 zfp_field) on an LP64 target, so a layout change fails the
 * build.  main() runs three round trips through zfp_compress /
 * zfp_decompress on host buffers (the library codes them on the GPU):
 * reversible int32 1-D (lossless), fixed-rate float 3-D, and fixed-accuracy
 * double 2-D with a full header written and read back.  Exit status 0 on
 * success; the first failure is printed.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "zfp.h"

_Static_assert(sizeof(zfp_type) == 4, "zfp_type is a C enum");
_Static_assert(offsetof(zfp_field, type) == 0, "zfp_field.type");
_Static_assert(offsetof(zfp_field, nx) == 8 && offsetof(zfp_field, nw) == 32, "zfp_field sizes");
_Static_assert(offsetof(zfp_field, sx) == 40 && offsetof(zfp_field, sw) == 64, "zfp_field strides");
_Static_assert(offsetof(zfp_field, data) == 72 && sizeof(zfp_field) == 80, "zfp_field.data");
_Static_assert(offsetof(zfp_execution, policy) == 0 && offsetof(zfp_execution, params) == 8,
               "zfp_execution");
_Static_assert(sizeof(zfp_execution) == 16, "zfp_execution size");
_Static_assert(offsetof(zfp_stream, minbits) == 0 && offsetof(zfp_stream, maxbits) == 4, "zfp_stream bits");
_Static_assert(offsetof(zfp_stream, maxprec) == 8 && offsetof(zfp_stream, minexp) == 12, "zfp_stream prec");
_Static_assert(offsetof(zfp_stream, stream) == 16 && offsetof(zfp_stream, exec) == 24, "zfp_stream ptrs");
_Static_assert(sizeof(zfp_stream) == 40, "zfp_stream size");
_Static_assert(offsetof(zfp_config, mode) == 0 && offsetof(zfp_config, arg) == 8, "zfp_config");
_Static_assert(sizeof(zfp_config) == 24, "zfp_config size");
_Static_assert(ZFP_HEADER_MAX_BITS == 148, "header bound");

static int failed(const char* what) {
  fprintf(stderr, "dropin: %s\n", what);
  return 1;
}

/* Compress `field` with the stream's current mode into a fresh buffer, then
 * decompress into `out_field`; returns 0 on success. */
static int round_trip(zfp_stream* zfp, zfp_field* field, zfp_field* out_field, int header,
                      size_t* bytes_out) {
  size_t cap = zfp_stream_maximum_size(zfp, field);
  if (cap == 0) return failed("zfp_stream_maximum_size returned 0");
  void* buf = calloc(cap, 1);
  if (!buf) return failed("calloc");
  bitstream* bs = stream_open(buf, cap);
  if (!bs) return failed("stream_open returned NULL");
  zfp_stream_set_bit_stream(zfp, bs);
  zfp_stream_rewind(zfp);
  if (header && zfp_write_header(zfp, field, ZFP_HEADER_FULL) == 0) return failed("zfp_write_header");
  size_t n = zfp_compress(zfp, field);
  if (n == 0 || n > cap) return failed("zfp_compress");
  if (stream_size(bs) != n) return failed("stream_size differs from zfp_compress's result");
  zfp_stream_rewind(zfp);
  if (header) {
    zfp_field* hdr = zfp_field_alloc();
    if (!hdr || zfp_read_header(zfp, hdr, ZFP_HEADER_FULL) == 0) return failed("zfp_read_header");
    if (zfp_field_type(hdr) != zfp_field_type(field) || hdr->nx != field->nx || hdr->ny != field->ny)
      return failed("header does not describe the field");
    zfp_field_free(hdr);
  }
  size_t m = zfp_decompress(zfp, out_field);
  if (m != n) return failed("zfp_decompress did not consume the stream");
  zfp_stream_set_bit_stream(zfp, NULL);
  stream_close(bs);
  free(buf);
  *bytes_out = n;
  return 0;
}

int main(void) {
  size_t bytes = 0;
  zfp_stream* zfp = zfp_stream_open(NULL);
  if (!zfp) return failed("zfp_stream_open returned NULL");
  if (!zfp_stream_set_execution(zfp, zfp_exec_cuda)) return failed("zfp_exec_cuda refused");

  /* Reversible int32, 1-D, 1000 values: exact. */
  enum { N1 = 1000 };
  int32_t* a = malloc(N1 * sizeof(int32_t));
  int32_t* b = calloc(N1, sizeof(int32_t));
  for (int i = 0; i < N1; i++) a[i] = (int32_t)(31 * i * i - 7000 * i + 12345);
  zfp_field* fa = zfp_field_1d(a, zfp_type_int32, N1);
  zfp_field* fb = zfp_field_1d(b, zfp_type_int32, N1);
  zfp_stream_set_reversible(zfp);
  if (zfp_stream_compression_mode(zfp) != zfp_mode_reversible) return failed("mode is not reversible");
  if (round_trip(zfp, fa, fb, 0, &bytes)) return 1;
  if (memcmp(a, b, N1 * sizeof(int32_t)) != 0) return failed("reversible round trip is not exact");
  printf("int32 1-D reversible: %d values -> %zu bytes, exact\n", N1, bytes);

  /* Fixed-rate 8 float, 3-D 40 x 33 x 21 (partial blocks). */
  const size_t nx = 40, ny = 33, nz = 21, n3 = nx * ny * nz;
  float* x = malloc(n3 * sizeof(float));
  float* y = calloc(n3, sizeof(float));
  for (size_t k = 0; k < nz; k++)
    for (size_t j = 0; j < ny; j++)
      for (size_t i = 0; i < nx; i++)
        x[i + nx * (j + ny * k)] = (float)(sin(0.1 * i) * cos(0.13 * j) * sin(0.07 * k));
  zfp_field* fx = zfp_field_3d(x, zfp_type_float, nx, ny, nz);
  zfp_field* fy = zfp_field_3d(y, zfp_type_float, nx, ny, nz);
  if (zfp_stream_set_rate(zfp, 8.0, zfp_type_float, 3, zfp_false) != 8.0) return failed("set_rate");
  if (round_trip(zfp, fx, fy, 0, &bytes)) return 1;
  if (bytes != ((nx + 3) / 4) * ((ny + 3) / 4) * ((nz + 3) / 4) * 64) return failed("fixed-rate stream is not 512 bits per block");
  double worst = 0;
  for (size_t i = 0; i < n3; i++) worst = fmax(worst, fabs((double)x[i] - (double)y[i]));
  if (!(worst < 1e-2)) return failed("fixed-rate error too large");
  printf("float 3-D rate 8: %zu values -> %zu bytes, max error %.2e\n", n3, bytes, worst);

  /* Fixed-accuracy 1e-6 double, 2-D 300 x 125, with a header. */
  const size_t mx = 300, my = 125, n2 = mx * my;
  double* u = malloc(n2 * sizeof(double));
  double* v = calloc(n2, sizeof(double));
  for (size_t j = 0; j < my; j++)
    for (size_t i = 0; i < mx; i++) u[i + mx * j] = 1e3 * sin(0.05 * i) * cos(0.09 * j);
  zfp_field* fu = zfp_field_2d(u, zfp_type_double, mx, my);
  zfp_field* fv = zfp_field_2d(v, zfp_type_double, mx, my);
  zfp_stream_set_accuracy(zfp, 1e-6);
  if (round_trip(zfp, fu, fv, 1, &bytes)) return 1;
  worst = 0;
  for (size_t i = 0; i < n2; i++) worst = fmax(worst, fabs(u[i] - v[i]));
  if (!(worst <= 1e-6)) return failed("fixed-accuracy error above the tolerance");
  printf("double 2-D accuracy 1e-6 + header: %zu values -> %zu bytes, max error %.2e\n", n2, bytes, worst);

  zfp_field_free(fa);
  zfp_field_free(fb);
  zfp_field_free(fx);
  zfp_field_free(fy);
  zfp_field_free(fu);
  zfp_field_free(fv);
  zfp_stream_close(zfp);
  free(a);
  free(b);
  free(x);
  free(y);
  free(u);
  free(v);
  printf("dropin ok\n");
  return 0;
}
