// Class kernels of the integral engine: (dp| s, p): one thread per aux component (eri_class.cuh).
#include "eri_class.cuh"

namespace rr {
namespace eri {

bool launch_class_dp01(int la, int lb, int lc, const ClassArgs& args, cudaStream_t s) {
  if (la == 2 && lb == 1 && lc == 0) {
    launch_class<2, 1, 0, true>(args, s);
    return true;
  }
  if (la == 2 && lb == 1 && lc == 1) {
    launch_class<2, 1, 1, true>(args, s);
    return true;
  }
  return false;
}

}  // namespace eri
}  // namespace rr
