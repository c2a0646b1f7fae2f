// ref_host_harness.cpp -- drives the reference's own host initialisation.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with FlowLB's
// src/initData.cpp (compiled where it lies in the reference tree) into
// oracle/_ref/libflbref_host.so.  It calls the reference functions that build
// the initial state of a case from its geometry flags:
//   FLB::initFields                 src/initData.h:125-165
//   FLB::initFreeSurfaceFlags       src/initData.cpp:13-37
//   FLB::initFreeSurfaceFields      src/initData.h:175-206
// in the order FLB::initData uses them (src/initData.h:256-332), so that the
// oracle's initial state can be compared with the reference's cell by cell.
#include <cstdint>
#include <cstring>
#include <vector>

#include "initData.h"

namespace {

template <typename P>
int run_init(int nx, int ny, const uint8_t* geometry_flags, int free_surface, double inlet_ux, double inlet_uy,
             P* f, P* u, P* rho, uint8_t* flags, P* phi, P* mass, P* excess) {
  const unsigned int Nx = (unsigned)nx, Ny = (unsigned)ny, N = Nx * Ny;
  std::vector<P> h_f(9u * N, 0), h_u(2u * N, 0), h_rho(N, 0);
  std::vector<P> h_phi(N, 0), h_mass(N, 0), h_excess(N, 0);
  std::vector<uint8_t> h_flags(geometry_flags, geometry_flags + N);
  std::vector<P> h_weights;
  if (sizeof(P) == 4)
    h_weights = {4.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f,
                 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};
  else
    h_weights = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  FLB::OptionsCalculation opts;
  opts.LBVelocity.x = inlet_ux;
  opts.LBVelocity.y = inlet_uy;
  opts.typeProblem = free_surface ? FLB::TypeProblem::FREE_SURFACE : FLB::TypeProblem::MONOFLUID;
  for (unsigned int y = 0; y < Ny; y++)
    for (unsigned int x = 0; x < Nx; x++) {
      const unsigned int idx = x + y * Nx;
      FLB::initFields<P>(h_f, h_u, h_weights, h_flags, h_rho, false, 9, idx, x, y, 0, N, Nx, Ny, &opts);
    }
  if (free_surface) {
    for (unsigned int y = 0; y < Ny; y++)
      for (unsigned int x = 0; x < Nx; x++) {
        const unsigned int idx = x + y * Nx;
        FLB::initFreeSurfaceFlags(h_flags, false, 9, idx, x, y, 0, Nx, Ny, 1);
        FLB::initFreeSurfaceFields<P>(h_flags, h_phi, h_mass, h_excess, idx);
      }
  }
  std::memcpy(f, h_f.data(), h_f.size() * sizeof(P));
  std::memcpy(u, h_u.data(), h_u.size() * sizeof(P));
  std::memcpy(rho, h_rho.data(), h_rho.size() * sizeof(P));
  std::memcpy(flags, h_flags.data(), N);
  std::memcpy(phi, h_phi.data(), N * sizeof(P));
  std::memcpy(mass, h_mass.data(), N * sizeof(P));
  std::memcpy(excess, h_excess.data(), N * sizeof(P));
  return 0;
}

}  // namespace

extern "C" int ref_host_init(int precision, int nx, int ny, const uint8_t* geometry_flags, int free_surface,
                             double inlet_ux, double inlet_uy, void* f, void* u, void* rho, uint8_t* flags, void* phi,
                             void* mass, void* excess) {
  if (nx < 3 || ny < 3 || !geometry_flags) return -1;
  if (precision == 32)
    return run_init<float>(nx, ny, geometry_flags, free_surface, inlet_ux, inlet_uy, (float*)f, (float*)u,
                           (float*)rho, flags, (float*)phi, (float*)mass, (float*)excess);
  if (precision == 64)
    return run_init<double>(nx, ny, geometry_flags, free_surface, inlet_ux, inlet_uy, (double*)f, (double*)u,
                            (double*)rho, flags, (double*)phi, (double*)mass, (double*)excess);
  return -1;
}
