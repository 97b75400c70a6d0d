// Kernel launchers for one scalar type; included by zfpb_inst.cu, which the
// Makefile compiles once per (type, group of passes) in parallel.
#pragma once

#include "zfpb_kernels.cuh"

namespace zfpb {

template <class T, int D> static size_t plane_smem(int threads) {
  return (size_t)KernelShape<T, D>::PLANE_WORDS * threads * sizeof(u64);
}

template <class T, int D> static cudaError_t set_smem(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static inline unsigned grid_of(u64 n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Kernels compiled for lossy float streams only (no reversible path) serve
// 2D and 3D float fields whose minexp selects a lossy mode.
template <class T, int D> static constexpr bool has_lossy() { return SortedCoder<T, D>::value; }
template <class T, int D> static bool lossy(const CodecParams& c) { return has_lossy<T, D>() && c.minexp >= ZFP_MIN_EXP; }

template <class T, int D, bool L>
static cudaError_t encode_fixed_k(const EncodeFixedArgs& a, u64 ctas, int threads, size_t smem, cudaStream_t s) {
  cudaError_t e = set_smem<T, D>((const void*)k_encode_fixed<T, D, L>, smem);
  if (e != cudaSuccess) return e;
  k_encode_fixed<T, D, L><<<(unsigned)ctas, threads, smem, s>>>(a);
  return cudaGetLastError();
}
template <class T, int D>
static cudaError_t encode_fixed_d(const EncodeFixedArgs& a, u64 ctas, int threads, size_t smem, cudaStream_t s) {
  if constexpr (has_lossy<T, D>())
    if (lossy<T, D>(a.c)) return encode_fixed_k<T, D, true>(a, ctas, threads, smem, s);
  return encode_fixed_k<T, D, false>(a, ctas, threads, smem, s);
}

template <class T, int D> static int var_threads() { return D == 4 ? 32 : 128; }

template <class T, int D, bool L> static cudaError_t encode_var_k(const EncodeVarArgs& a, cudaStream_t s) {
  const int th = var_threads<T, D>();
  size_t smem = plane_smem<T, D>(th);
  cudaError_t e = set_smem<T, D>((const void*)k_encode_var<T, D, L>, smem);
  if (e != cudaSuccess) return e;
  k_encode_var<T, D, L><<<grid_of(a.f.nblocks, th), th, smem, s>>>(a);
  return cudaGetLastError();
}
template <class T, int D> static cudaError_t encode_var_d(const EncodeVarArgs& a, cudaStream_t s) {
  if constexpr (has_lossy<T, D>())
    if (lossy<T, D>(a.c)) return encode_var_k<T, D, true>(a, s);
  return encode_var_k<T, D, false>(a, s);
}

template <class T, int D, bool L> static cudaError_t decode_fixed_k(const DecodeArgs& a, cudaStream_t s) {
  const int th = var_threads<T, D>();
  size_t smem = plane_smem<T, D>(th);
  cudaError_t e = set_smem<T, D>((const void*)k_decode_fixed<T, D, L>, smem);
  if (e != cudaSuccess) return e;
  k_decode_fixed<T, D, L><<<grid_of(a.f.nblocks, th), th, smem, s>>>(a);
  return cudaGetLastError();
}
template <class T, int D> static cudaError_t decode_fixed_d(const DecodeArgs& a, cudaStream_t s) {
  if constexpr (has_lossy<T, D>())
    if (lossy<T, D>(a.c)) return decode_fixed_k<T, D, true>(a, s);
  return decode_fixed_k<T, D, false>(a, s);
}

template <class T, int D, bool L> static cudaError_t decode_var_k(const DecodeArgs& a, cudaStream_t s) {
  const int th = var_threads<T, D>();
  size_t smem = plane_smem<T, D>(th);
  cudaError_t e = set_smem<T, D>((const void*)k_decode_var<T, D, L>, smem);
  if (e != cudaSuccess) return e;
  k_decode_var<T, D, L><<<grid_of(a.f.nblocks, th), th, smem, s>>>(a);
  return cudaGetLastError();
}
template <class T, int D> static cudaError_t decode_var_d(const DecodeArgs& a, cudaStream_t s) {
  if constexpr (has_lossy<T, D>())
    if (lossy<T, D>(a.c)) return decode_var_k<T, D, true>(a, s);
  return decode_var_k<T, D, false>(a, s);
}

template <class T, int D> static cudaError_t walk_d(const DecodeArgs& a, cudaStream_t s) {
  size_t smem = plane_smem<T, D>(1);
  k_walk<T, D><<<1, 1, smem, s>>>(a);
  return cudaGetLastError();
}

#define ZFPB_DISPATCH(call, fn, ...)             \
  switch ((call).dims) {                         \
    case 1: return fn<T, 1>(__VA_ARGS__);        \
    case 2: return fn<T, 2>(__VA_ARGS__);        \
    case 3: return fn<T, 3>(__VA_ARGS__);        \
    default: return fn<T, 4>(__VA_ARGS__);       \
  }

template <class T>
cudaError_t Launch<T>::encode_fixed(const Call& call, const EncodeFixedArgs& a, u64 ctas, int threads,
                                    size_t smem, cudaStream_t s) {
  ZFPB_DISPATCH(call, encode_fixed_d, a, ctas, threads, smem, s)
}
template <class T> cudaError_t Launch<T>::encode_var(const Call& call, const EncodeVarArgs& a, cudaStream_t s) {
  ZFPB_DISPATCH(call, encode_var_d, a, s)
}
template <class T> cudaError_t Launch<T>::decode_fixed(const Call& call, const DecodeArgs& a, cudaStream_t s) {
  ZFPB_DISPATCH(call, decode_fixed_d, a, s)
}
template <class T> cudaError_t Launch<T>::decode_var(const Call& call, const DecodeArgs& a, cudaStream_t s) {
  ZFPB_DISPATCH(call, decode_var_d, a, s)
}
template <class T>
cudaError_t Launch<T>::parse(const Call& call, const DecodeArgs& a, const SplitArgs& sa, bool var, cudaStream_t s) {
  if (call.dims != 3) return cudaErrorInvalidValue;
  const unsigned g = grid_of(a.f.nblocks, 128);
  if (lossy<T, 3>(a.c)) {
    if (var) k_parse<T, 3, true, true><<<g, 128, 0, s>>>(a, sa);
    else k_parse<T, 3, false, true><<<g, 128, 0, s>>>(a, sa);
  } else {
    if (var) k_parse<T, 3, true, false><<<g, 128, 0, s>>>(a, sa);
    else k_parse<T, 3, false, false><<<g, 128, 0, s>>>(a, sa);
  }
  return cudaGetLastError();
}
template <class T>
cudaError_t Launch<T>::finish(const Call& call, const DecodeArgs& a, const SplitArgs& sa, cudaStream_t s) {
  if (call.dims != 3) return cudaErrorInvalidValue;
  if (lossy<T, 3>(a.c)) k_finish<T, 3, true><<<grid_of(a.f.nblocks, 128), 128, 0, s>>>(a, sa);
  else k_finish<T, 3, false><<<grid_of(a.f.nblocks, 128), 128, 0, s>>>(a, sa);
  return cudaGetLastError();
}
template <class T, int D>
static cudaError_t encode_batch_d(const BatchArgs& a, u32 ntiles, int th, cudaStream_t s) {
  size_t smem = plane_smem<T, D>(th);
  cudaError_t e = set_smem<T, D>((const void*)k_encode_batch<T, D>, smem);
  if (e != cudaSuccess) return e;
  k_encode_batch<T, D><<<ntiles, th, smem, s>>>(a);
  return cudaGetLastError();
}
template <class T, int D>
static cudaError_t decode_batch_d(const BatchArgs& a, u32 ntiles, int th, cudaStream_t s) {
  size_t smem = plane_smem<T, D>(th);
  cudaError_t e = set_smem<T, D>((const void*)k_decode_batch<T, D>, smem);
  if (e != cudaSuccess) return e;
  k_decode_batch<T, D><<<ntiles, th, smem, s>>>(a);
  return cudaGetLastError();
}
template <class T, int D> static cudaError_t walk_batch_d(const BatchArgs& a, cudaStream_t s) {
  k_walk_batch<T, D><<<(a.nwalk + 63) / 64, 64, 0, s>>>(a);
  return cudaGetLastError();
}
template <class T>
cudaError_t Launch<T>::encode_batch(int dims, const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s) {
  switch (dims) {
    case 1: return encode_batch_d<T, 1>(a, ntiles, threads, s);
    case 2: return encode_batch_d<T, 2>(a, ntiles, threads, s);
    case 3: return encode_batch_d<T, 3>(a, ntiles, threads, s);
    default: return encode_batch_d<T, 4>(a, ntiles, threads, s);
  }
}
template <class T>
cudaError_t Launch<T>::decode_batch(int dims, const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s) {
  switch (dims) {
    case 1: return decode_batch_d<T, 1>(a, ntiles, threads, s);
    case 2: return decode_batch_d<T, 2>(a, ntiles, threads, s);
    case 3: return decode_batch_d<T, 3>(a, ntiles, threads, s);
    default: return decode_batch_d<T, 4>(a, ntiles, threads, s);
  }
}
template <class T>
cudaError_t Launch<T>::parse_batch(const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s) {
  k_parse_batch<T><<<ntiles, threads, 0, s>>>(a);
  return cudaGetLastError();
}
template <class T>
cudaError_t Launch<T>::finish_batch(const BatchArgs& a, u32 ntiles, int threads, cudaStream_t s) {
  k_finish_batch<T><<<ntiles, threads, 0, s>>>(a);
  return cudaGetLastError();
}
template <class T> cudaError_t Launch<T>::walk_batch(int dims, const BatchArgs& a, cudaStream_t s) {
  switch (dims) {
    case 1: return walk_batch_d<T, 1>(a, s);
    case 2: return walk_batch_d<T, 2>(a, s);
    case 3: return walk_batch_d<T, 3>(a, s);
    default: return walk_batch_d<T, 4>(a, s);
  }
}
// One walker per warp: a CTA of 32 threads per segment (4-D: plus the
// walker's plane store in dynamic shared memory).
template <class T> cudaError_t Launch<T>::spec_walk(int dims, const SpecWalkArgs& a, cudaStream_t s) {
  const unsigned g = (unsigned)a.nseg;
  switch (dims) {
    case 1: k_spec_walk<T, 1><<<g, 32, 0, s>>>(a); break;
    case 2: k_spec_walk<T, 2><<<g, 32, 0, s>>>(a); break;
    case 3: k_spec_walk<T, 3><<<g, 32, 0, s>>>(a); break;
    case 4: k_spec_walk<T, 4><<<g, 32, plane_smem<T, 4>(1), s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
template <class T> cudaError_t Launch<T>::spec_fix(int dims, const SpecWalkArgs& a, cudaStream_t s) {
  const unsigned g = (unsigned)a.nseg;
  switch (dims) {
    case 1: k_spec_fix<T, 1><<<g, 32, 0, s>>>(a); break;
    case 2: k_spec_fix<T, 2><<<g, 32, 0, s>>>(a); break;
    case 3: k_spec_fix<T, 3><<<g, 32, 0, s>>>(a); break;
    case 4: k_spec_fix<T, 4><<<g, 32, plane_smem<T, 4>(1), s>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
template <class T>
cudaError_t Launch<T>::spec_tail(int dims, const SpecWalkArgs& a, u64* off, u64 idx, u64 n, u64 x, cudaStream_t s) {
  switch (dims) {
    case 1: k_spec_tail<T, 1><<<1, 32, 0, s>>>(a, off, idx, n, x); break;
    case 2: k_spec_tail<T, 2><<<1, 32, 0, s>>>(a, off, idx, n, x); break;
    case 3: k_spec_tail<T, 3><<<1, 32, 0, s>>>(a, off, idx, n, x); break;
    case 4: k_spec_tail<T, 4><<<1, 32, plane_smem<T, 4>(1), s>>>(a, off, idx, n, x); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
template <class T> cudaError_t Launch<T>::walk(const Call& call, const DecodeArgs& a, cudaStream_t s) {
  ZFPB_DISPATCH(call, walk_d, a, s)
}

#undef ZFPB_DISPATCH

}  // namespace zfpb
