// Explicit instantiations of the kernel launchers (Launch<T>, zfpb_inst.cuh)
// for one scalar type and one group of passes.  The Makefile compiles this
// file once per (type, group) with -DZFPB_INST_T=<float|double|int|i64> and
// -DZFPB_INST_GROUP=<0..3>, so that the heavy templates compile in parallel.
#include "zfpb_inst.cuh"

namespace zfpb {
typedef ZFPB_INST_T InstT;

#if ZFPB_INST_GROUP == 0  // single-array encoders
template cudaError_t Launch<InstT>::encode_fixed(const Call&, const EncodeFixedArgs&, u64, int, size_t, cudaStream_t);
template cudaError_t Launch<InstT>::encode_var(const Call&, const EncodeVarArgs&, cudaStream_t);
#elif ZFPB_INST_GROUP == 1  // single-array decoders
template cudaError_t Launch<InstT>::decode_fixed(const Call&, const DecodeArgs&, cudaStream_t);
template cudaError_t Launch<InstT>::decode_var(const Call&, const DecodeArgs&, cudaStream_t);
template cudaError_t Launch<InstT>::parse(const Call&, const DecodeArgs&, const SplitArgs&, bool, cudaStream_t);
template cudaError_t Launch<InstT>::finish(const Call&, const DecodeArgs&, const SplitArgs&, cudaStream_t);
#elif ZFPB_INST_GROUP == 2  // batches
template cudaError_t Launch<InstT>::encode_batch(int, const BatchArgs&, u32, int, cudaStream_t);
template cudaError_t Launch<InstT>::decode_batch(int, const BatchArgs&, u32, int, cudaStream_t);
template cudaError_t Launch<InstT>::parse_batch(const BatchArgs&, u32, int, cudaStream_t);
template cudaError_t Launch<InstT>::finish_batch(const BatchArgs&, u32, int, cudaStream_t);
template cudaError_t Launch<InstT>::walk_batch(int, const BatchArgs&, cudaStream_t);
#elif ZFPB_INST_GROUP == 3  // block walks of streams without an index
template cudaError_t Launch<InstT>::walk(const Call&, const DecodeArgs&, cudaStream_t);
template cudaError_t Launch<InstT>::spec_walk(int, const SpecWalkArgs&, cudaStream_t);
template cudaError_t Launch<InstT>::spec_fix(int, const SpecWalkArgs&, cudaStream_t);
template cudaError_t Launch<InstT>::spec_tail(int, const SpecWalkArgs&, u64*, u64, u64, u64, cudaStream_t);
#else
#error "ZFPB_INST_GROUP must be 0..3"
#endif
}  // namespace zfpb
