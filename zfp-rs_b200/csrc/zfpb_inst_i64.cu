// Kernel instantiations for long long fields.
#include "zfpb_inst.cuh"

namespace zfpb {
template struct Launch<long long>;
}
