// Class kernels of the integral engine: (dp| d): one thread per aux component (eri_class.cuh).
#include "eri_class.cuh"

namespace rr {
namespace eri {

bool launch_class_dp2(int la, int lb, int lc, const ClassArgs& args, cudaStream_t s) {
  if (la == 2 && lb == 1 && lc == 2) {
    launch_class<2, 1, 2, true>(args, s);
    return true;
  }
  return false;
}

}  // namespace eri
}  // namespace rr
