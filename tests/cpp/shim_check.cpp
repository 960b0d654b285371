// Host check of the ReactorB200 shim against the test stand-in for AMReX:
// the factory finds the reactor by name, and the views it passes to
// b200chem_react address the same elements as the Array4s (ghost cells,
// a tile box inside the fab, component stride).  Needs no GPU.
#include <cstdio>
#include <vector>

#include "pele/ReactorB200.H"

b200chem_mech_desc b200chem_make_mech_desc() { return b200chem_mech_desc{}; }

using namespace pele::physics::reactions;

static int fails = 0;
#define CHECK(c)                                         \
  do {                                                   \
    if (!(c)) {                                          \
      std::fprintf(stderr, "check failed: %s\n", #c);   \
      ++fails;                                           \
    }                                                    \
  } while (0)

int main() {
  (void)ReactorB200::registered;  // the stand-in factory registers on first use
  auto r = ReactorBase::create("ReactorB200");
  CHECK(r != nullptr);
  CHECK(b200chem_version() == B200CHEM_VERSION);
  // a fab over [-1, 6] x [2, 7] x [4, 6] with 3 components, tile box [0, 5] x [3, 6] x [5, 5]
  const int nx = 8, ny = 6, nz = 3, nc = 3;
  std::vector<double> buf((size_t)nx * ny * nz * nc);
  for (size_t q = 0; q < buf.size(); ++q) buf[q] = (double)q;
  amrex::Array4<double> a;
  a.p = buf.data();
  a.jstride = nx;
  a.kstride = (long long)nx * ny;
  a.nstride = (long long)nx * ny * nz;
  a.begin = {-1, 2, 4};
  a.end = {-1 + nx, 2 + ny, 4 + nz};
  a.ncomp = nc;
  std::vector<int> mbuf((size_t)nx * ny * nz, 1);
  amrex::Array4<int> m;
  m.p = mbuf.data();
  m.jstride = nx;
  m.kstride = (long long)nx * ny;
  m.nstride = (long long)nx * ny * nz;
  m.begin = a.begin;
  m.end = a.end;
  amrex::Box box{{0, 3, 5}, {5, 6, 5}};
  const b200chem_box_view v = ReactorB200::box_view(box, a, a, a, a, a, a, m);
  for (int d = 0; d < 3; ++d) {
    CHECK(v.lo[d] == box.lo[d] && v.hi[d] == box.hi[d]);
    CHECK(v.rhoY.lo[d] == a.begin[d] && v.rhoY.hi[d] == a.end[d] - 1);
  }
  // the element formula of b200chem.h reaches the Array4 element
  for (int n = 0; n < nc; ++n)
    for (int k = box.lo[2]; k <= box.hi[2]; ++k)
      for (int j = box.lo[1]; j <= box.hi[1]; ++j)
        for (int i = box.lo[0]; i <= box.hi[0]; ++i) {
          const double* e = v.rhoY.p + (i - v.rhoY.lo[0]) + (j - v.rhoY.lo[1]) * v.rhoY.jstride +
                            (k - v.rhoY.lo[2]) * v.rhoY.kstride + n * v.rhoY.nstride;
          CHECK(e == &a(i, j, k, n));
          const int32_t* me = v.mask.p + (i - v.mask.lo[0]) + (j - v.mask.lo[1]) * v.mask.jstride +
                              (k - v.mask.lo[2]) * v.mask.kstride;
          CHECK(me == &m(i, j, k));
        }
  if (fails) return 1;
  std::printf("shim ok\n");
  return 0;
}
