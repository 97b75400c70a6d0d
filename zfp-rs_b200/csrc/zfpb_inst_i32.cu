// Kernel instantiations for int fields.
#include "zfpb_inst.cuh"

namespace zfpb {
template struct Launch<int>;
}
