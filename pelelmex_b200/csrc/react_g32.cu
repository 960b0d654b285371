// react_g32.cu -- group integrator variants with 32 lanes per cell.
#include "react_group.cuh"

namespace b200 {

const GroupVariant* group_variants_g32(int* count) {
  static const GroupVariant v[] = {
      make_variant<32, 1, float>(), make_variant<32, 1, double>(),
      make_variant<32, 2, float>(), make_variant<32, 2, double>(),
  };
  *count = (int)(sizeof(v) / sizeof(v[0]));
  return v;
}

}  // namespace b200
