// Device run of the ReactorB200 shim through the ReactorBase factory, as
// PeleLMeX drives it (Source/PeleLMeX_Setup.cpp:146-155,
// Source/PeleLMeX_Reactions.cpp:101-108): inputs-file keys, create, init,
// set_eos_parm, react on device Array4 fabs with ghost cells, close.
//
//   shim_react IN OUT [surrogate weights file]
//
// IN (binary): int32 N, nx, ny, nz, ghost; double dt; then for the box cells
// (i fastest) rhoY [N][cells], T, rhoH (CGS).  OUT: rhoY [N][cells], T, rhoH,
// fctCount, then int32 hybrid (1 when the surrogate was selected).
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "pele/ReactorB200.H"

using namespace pele::physics::reactions;

#define CK(x)                                                          \
  do {                                                                 \
    cudaError_t e_ = (x);                                              \
    if (e_ != cudaSuccess) {                                           \
      std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));    \
      return 2;                                                        \
    }                                                                  \
  } while (0)

int main(int argc, char** argv) {
  if (argc < 3) return 1;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 1;
  int32_t hdr[5];
  double dt;
  if (std::fread(hdr, sizeof(hdr), 1, f) != 1 || std::fread(&dt, sizeof(dt), 1, f) != 1) return 1;
  const int N = hdr[0], nx = hdr[1], ny = hdr[2], nz = hdr[3], g = hdr[4];
  const long long cells = (long long)nx * ny * nz;
  std::vector<double> rY((size_t)N * cells), T(cells), rH(cells);
  if (std::fread(rY.data(), 8, rY.size(), f) != rY.size() || std::fread(T.data(), 8, cells, f) != (size_t)cells ||
      std::fread(rH.data(), 8, cells, f) != (size_t)cells)
    return 1;
  std::fclose(f);

  // the inputs file
  auto& pp = amrex::ParmParse::table();
  pp["peleLM.chem_integrator"] = "ReactorB200";
  pp["ode.rtol"] = "1e-8";
  pp["ode.atol"] = "1e-12";
  pp["cvode.max_order"] = "5";
  pp["cvode.max_substeps"] = "10000";
  if (argc > 3) pp["b200.surrogate"] = argv[3];

  // fabs over [-g, n + g) in each direction, component-strided like amrex::FArrayBox
  const int fx = nx + 2 * g, fy = ny + 2 * g, fz = nz + 2 * g;
  const long long fcells = (long long)fx * fy * fz;
  auto make = [&](int ncomp, double** d) -> amrex::Array4<double> {
    cudaMalloc(d, sizeof(double) * ncomp * fcells);
    cudaMemset(*d, 0, sizeof(double) * ncomp * fcells);
    amrex::Array4<double> a;
    a.p = *d;
    a.jstride = fx;
    a.kstride = (long long)fx * fy;
    a.nstride = fcells;
    a.begin = {-g, -g, -g};
    a.end = {nx + g, ny + g, nz + g};
    a.ncomp = ncomp;
    return a;
  };
  double *d_rY, *d_fY, *d_T, *d_rH, *d_fH, *d_fc;
  auto a_rY = make(N, &d_rY), a_fY = make(N, &d_fY), a_T = make(1, &d_T), a_rH = make(1, &d_rH),
       a_fH = make(1, &d_fH), a_fc = make(1, &d_fc);
  int* d_m;
  CK(cudaMalloc(&d_m, sizeof(int) * fcells));
  std::vector<int> ones(fcells, 1);
  CK(cudaMemcpy(d_m, ones.data(), sizeof(int) * fcells, cudaMemcpyHostToDevice));
  amrex::Array4<int> a_m;
  a_m.p = d_m;
  a_m.jstride = fx;
  a_m.kstride = (long long)fx * fy;
  a_m.nstride = fcells;
  a_m.begin = a_rY.begin;
  a_m.end = a_rY.end;

  // box cells into the fab interiors
  std::vector<double> frY((size_t)N * fcells, 0.0), fT(fcells, 0.0), frH(fcells, 0.0);
  auto fidx = [&](int i, int j, int k) { return (long long)(i + g) + (long long)(j + g) * fx + (long long)(k + g) * fx * fy; };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long long c = i + (long long)nx * (j + (long long)ny * k), q = fidx(i, j, k);
        for (int n = 0; n < N; ++n) frY[(size_t)n * fcells + q] = rY[(size_t)n * cells + c];
        fT[q] = T[c];
        frH[q] = rH[c];
      }
  CK(cudaMemcpy(d_rY, frY.data(), 8 * frY.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_T, fT.data(), 8 * fcells, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_rH, frH.data(), 8 * fcells, cudaMemcpyHostToDevice));

  (void)ReactorB200::registered;  // the stand-in factory registers on first use
  std::string name;
  amrex::ParmParse("peleLM").query("chem_integrator", name);
  auto reactor = ReactorBase::create(name);
  reactor->init(2, 1);
  reactor->set_eos_parm(nullptr);
  amrex::Box box{{0, 0, 0}, {nx - 1, ny - 1, nz - 1}};
  amrex::Real dt_react = dt, time = 0.0;
  reactor->react(box, a_rY, a_fY, a_T, a_rH, a_fH, a_fc, a_m, dt_react, time, nullptr);
  CK(cudaDeviceSynchronize());
  const int hybrid = static_cast<ReactorB200*>(reactor.get())->hybrid() ? 1 : 0;
  reactor->close();

  std::vector<double> ffc(fcells);
  CK(cudaMemcpy(frY.data(), d_rY, 8 * frY.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fT.data(), d_T, 8 * fcells, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(frH.data(), d_rH, 8 * fcells, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ffc.data(), d_fc, 8 * fcells, cudaMemcpyDeviceToHost));
  std::vector<double> fc(cells);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long long c = i + (long long)nx * (j + (long long)ny * k), q = fidx(i, j, k);
        for (int n = 0; n < N; ++n) rY[(size_t)n * cells + c] = frY[(size_t)n * fcells + q];
        T[c] = fT[q];
        rH[c] = frH[q];
        fc[c] = ffc[q];
      }
  // ghost cells untouched
  for (int k = -g; k < nz + g; ++k)
    for (int j = -g; j < ny + g; ++j)
      for (int i = -g; i < nx + g; ++i) {
        const bool inside = i >= 0 && i < nx && j >= 0 && j < ny && k >= 0 && k < nz;
        if (!inside && (fT[fidx(i, j, k)] != 0.0 || ffc[fidx(i, j, k)] != 0.0)) {
          std::fprintf(stderr, "ghost cell written\n");
          return 3;
        }
      }
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 1;
  std::fwrite(rY.data(), 8, rY.size(), o);
  std::fwrite(T.data(), 8, cells, o);
  std::fwrite(rH.data(), 8, cells, o);
  std::fwrite(fc.data(), 8, cells, o);
  std::fwrite(&hybrid, 4, 1, o);
  std::fclose(o);
  for (double* p : {d_rY, d_fY, d_T, d_rH, d_fH, d_fc}) cudaFree(p);
  cudaFree(d_m);
  std::printf("shim react ok\n");
  return 0;
}
