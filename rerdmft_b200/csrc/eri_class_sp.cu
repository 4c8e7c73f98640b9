// Class kernels of the integral engine: s and p pairs with aux s .. f, (pp| s, p), (ds| s, p): one thread per item (eri_class.cuh).
#include "eri_class.cuh"

namespace rr {
namespace eri {

bool launch_class_sp(int la, int lb, int lc, const ClassArgs& args, cudaStream_t s) {
  if (la == 0 && lb == 0 && lc == 0) {
    launch_class<0, 0, 0, false>(args, s);
    return true;
  }
  if (la == 0 && lb == 0 && lc == 1) {
    launch_class<0, 0, 1, false>(args, s);
    return true;
  }
  if (la == 0 && lb == 0 && lc == 2) {
    launch_class<0, 0, 2, false>(args, s);
    return true;
  }
  if (la == 0 && lb == 0 && lc == 3) {
    launch_class<0, 0, 3, false>(args, s);
    return true;
  }
  if (la == 1 && lb == 0 && lc == 0) {
    launch_class<1, 0, 0, false>(args, s);
    return true;
  }
  if (la == 1 && lb == 0 && lc == 1) {
    launch_class<1, 0, 1, false>(args, s);
    return true;
  }
  if (la == 1 && lb == 0 && lc == 2) {
    launch_class<1, 0, 2, false>(args, s);
    return true;
  }
  if (la == 1 && lb == 0 && lc == 3) {
    launch_class<1, 0, 3, false>(args, s);
    return true;
  }
  if (la == 1 && lb == 1 && lc == 0) {
    launch_class<1, 1, 0, false>(args, s);
    return true;
  }
  if (la == 1 && lb == 1 && lc == 1) {
    launch_class<1, 1, 1, false>(args, s);
    return true;
  }
  if (la == 2 && lb == 0 && lc == 0) {
    launch_class<2, 0, 0, false>(args, s);
    return true;
  }
  if (la == 2 && lb == 0 && lc == 1) {
    launch_class<2, 0, 1, false>(args, s);
    return true;
  }
  return false;
}

}  // namespace eri
}  // namespace rr
