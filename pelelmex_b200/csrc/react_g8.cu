// react_g8.cu -- group integrator variants with 8 lanes per cell.
#include "react_group.cuh"

namespace b200 {

const GroupVariant* group_variants_g8(int* count) {
  static const GroupVariant v[] = {
      make_variant<8, 2, float>(), make_variant<8, 2, double>(),
      make_variant<8, 3, float>(), make_variant<8, 3, double>(),
  };
  *count = (int)(sizeof(v) / sizeof(v[0]));
  return v;
}

}  // namespace b200
