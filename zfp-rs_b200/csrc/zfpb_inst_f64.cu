// Kernel instantiations for double fields.
#include "zfpb_inst.cuh"

namespace zfpb {
template struct Launch<double>;
}
