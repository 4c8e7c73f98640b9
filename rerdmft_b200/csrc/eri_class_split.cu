// Class kernels of the integral engine: (pp| d, f) and (ds| d, f): one thread per aux component (eri_class.cuh).
#include "eri_class.cuh"

namespace rr {
namespace eri {

bool launch_class_split(int la, int lb, int lc, const ClassArgs& args, cudaStream_t s) {
  if (la == 1 && lb == 1 && lc == 2) {
    launch_class<1, 1, 2, true>(args, s);
    return true;
  }
  if (la == 1 && lb == 1 && lc == 3) {
    launch_class<1, 1, 3, true>(args, s);
    return true;
  }
  if (la == 2 && lb == 0 && lc == 2) {
    launch_class<2, 0, 2, true>(args, s);
    return true;
  }
  if (la == 2 && lb == 0 && lc == 3) {
    launch_class<2, 0, 3, true>(args, s);
    return true;
  }
  return false;
}

}  // namespace eri
}  // namespace rr
