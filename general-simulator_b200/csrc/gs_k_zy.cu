// gs_k_zy.cu -- instances and launchers of the z-forward and y passes.
#include "gs_launch.h"
#include "gs_passes.cuh"

namespace gs {

bool size_supported(int n) {
  switch (n) {
#define GS_C(N_) case N_:
    GS_SIZE_CASES(GS_C)
#undef GS_C
    return true;
    default:
      return false;
  }
}

int pick_tz(int h) {
  int tz = 16;
  while (tz > 1 && (h % tz) != 0) tz >>= 1;
  return tz;
}

}  // namespace gs
