// Kernel instantiations for float fields.
#include "zfpb_inst.cuh"

namespace zfpb {
template struct Launch<float>;
}
