// react_g16.cu -- group integrator variants with 16 lanes per cell.
#include "react_group.cuh"

namespace b200 {

const GroupVariant* group_variants_g16(int* count) {
  static const GroupVariant v[] = {
      make_variant<16, 1, float>(), make_variant<16, 1, double>(),
      make_variant<16, 2, float>(), make_variant<16, 2, double>(),
      make_variant<16, 4, float>(), make_variant<16, 4, double>(),
  };
  *count = (int)(sizeof(v) / sizeof(v[0]));
  return v;
}

}  // namespace b200
