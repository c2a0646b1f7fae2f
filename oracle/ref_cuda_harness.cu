// ref_cuda_harness.cu -- runs the reference's own CUDA kernels headless.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with FlowLB's
// src/cuda/lbmKernel2D.cu, src/cuda/cudaInitData.cu and src/utils.cpp
// (compiled where they lie in the reference tree, with --fmad=false so that
// every float operation rounds as written) into oracle/_ref/libflbref_cuda.so.
//
// The reference's headless loops (src/cuda/runCuda.cu:460-528) include the GUI
// and OpenGL headers and cannot be built here, so this file re-states their
// launch sequence: constants via FLB::h_initConstantDataCuda2D
// (cudaInitData.cu:57-108), buffers via FLB::h_initDataCuda2D
// (cudaInitData.cuh:90-125), 16x16 blocks and a ceil-divided grid
// (cudaUtils.cu:89-105), and per step FS_1, StreamCollide, FS_2, FS_3, FS_4
// (free surface) or StreamCollide alone (mono-fluid).
//
// It also runs the reference's headless-capable visualisation kernel
// d_CreateIsoSurfaceVector2D (src/cuda/cudaIsosurface.cuh:33-199,
// cudaIsosurface.cu:16-76; built from cudaIsosurface.cu in place) into a CUDA
// array through a surface object, as the viewer's texture would receive it
// (ref_cuda_isoline).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "cudaInitData.cuh"
#include "cudaIsosurface.cuh"
#include "lbmKernel2D.cuh"

namespace {

template <typename P>
int run_ref(int nx, int ny, int free_surface, int collision, int subgrid, int use_force, double tau, double fx,
            double fy, uint64_t t0, uint64_t nsteps, int kernel_id, void* f, void* rho, void* u, uint8_t* flags,
            void* mass, void* excess, void* phi, uint64_t warm = 0, double* ms = nullptr) {
  const unsigned int Nx = (unsigned)nx, Ny = (unsigned)ny, N = Nx * Ny;
  static float wf[9] = {4.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f,
                        1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};
  static double wd[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                         1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  FLB::OptionsCalculation opts;
  opts.graphicsAPI = FLB::API::NONE;
  opts.typeProblem = free_surface ? FLB::TypeProblem::FREE_SURFACE : FLB::TypeProblem::MONOFLUID;
  opts.collisionOperator = (uint8_t)collision;
  opts.useSubgridModel = subgrid != 0;
  opts.useVolumetricForce = use_force != 0;
  opts.relaxationTime = tau;
  opts.volumetricForce.x = fx;
  opts.volumetricForce.y = fy;
  opts.precision = sizeof(P) == 4 ? 32 : 64;
  FLB::Units units;  // unit parameters 1: lattice units pass through
  FLB::h_initConstantDataCuda2D<P>(opts, sizeof(P) == 4 ? (P*)(void*)wf : (P*)(void*)wd, Nx, Ny, N, units);

  P *d_f = nullptr, *d_u = nullptr, *d_rho = nullptr, *d_mass = nullptr, *d_excess = nullptr, *d_phi = nullptr;
  uint8_t* d_flags = nullptr;
  FLB::h_initDataCuda2D<P>(opts, N, 2, 9, &d_f, (P*)f, &d_u, (P*)u, &d_flags, flags, &d_mass, (P*)mass, &d_rho,
                           (P*)rho, &d_excess, (P*)excess, &d_phi, (P*)phi);
  dim3 block(16, 16);
  dim3 grid((Nx + block.x - 1) / block.x, (Ny + block.y - 1) / block.y);
  if (kernel_id >= 0) {
    const unsigned long t = (unsigned long)t0;
    switch (kernel_id) {
      case 0: FLB::d_StreamCollide2D<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, d_mass, t); break;
      case 1: FLB::d_FreeSurface2D_1<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, d_mass, d_excess, d_phi, t); break;
      case 2: FLB::d_FreeSurface2D_2<9><<<grid, block>>>(d_flags); break;
      case 3: FLB::d_FreeSurface2D_3<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, t); break;
      case 4: FLB::d_FreeSurface2D_4<P, 9><<<grid, block>>>(d_rho, d_flags, d_mass, d_excess, d_phi); break;
      default: break;
    }
  } else {
    // timing (ms != nullptr): `warm` untimed steps, then CUDA events around
    // the nsteps steps that follow
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const uint64_t total = ms ? warm + nsteps : nsteps;
    for (uint64_t k = 0; k < total; k++) {
      if (ms && k == warm) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
      }
      const unsigned long t = (unsigned long)(t0 + k);
      if (free_surface) {
        FLB::d_FreeSurface2D_1<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, d_mass, d_excess, d_phi, t);
        FLB::d_StreamCollide2D<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, d_mass, t);
        FLB::d_FreeSurface2D_2<9><<<grid, block>>>(d_flags);
        FLB::d_FreeSurface2D_3<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, t);
        FLB::d_FreeSurface2D_4<P, 9><<<grid, block>>>(d_rho, d_flags, d_mass, d_excess, d_phi);
      } else {
        FLB::d_StreamCollide2D<P, 9><<<grid, block>>>(d_f, d_rho, d_u, d_flags, d_mass, t);
      }
    }
    if (ms && e0) {
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float m = 0.0f;
      cudaEventElapsedTime(&m, e0, e1);
      *ms = m;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
  }
  cudaError_t err = cudaDeviceSynchronize();
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err == cudaSuccess) {
    cudaMemcpy(f, d_f, 9ull * N * sizeof(P), cudaMemcpyDeviceToHost);
    cudaMemcpy(rho, d_rho, (size_t)N * sizeof(P), cudaMemcpyDeviceToHost);
    cudaMemcpy(u, d_u, 2ull * N * sizeof(P), cudaMemcpyDeviceToHost);
    cudaMemcpy(flags, d_flags, N, cudaMemcpyDeviceToHost);
    if (free_surface) {
      cudaMemcpy(mass, d_mass, (size_t)N * sizeof(P), cudaMemcpyDeviceToHost);
      cudaMemcpy(excess, d_excess, (size_t)N * sizeof(P), cudaMemcpyDeviceToHost);
      cudaMemcpy(phi, d_phi, (size_t)N * sizeof(P), cudaMemcpyDeviceToHost);
    }
    err = cudaGetLastError();
  }
  cudaFree(d_f);
  cudaFree(d_rho);
  cudaFree(d_u);
  cudaFree(d_flags);
  if (free_surface) {
    cudaFree(d_mass);
    cudaFree(d_excess);
    cudaFree(d_phi);
  }
  return err == cudaSuccess ? 0 : (int)err;
}

}  // namespace

// kernel_id < 0: run nsteps full steps from t0; otherwise run that one kernel
// (0 StreamCollide, 1..4 FreeSurface_1..4) once at t0.  All buffers are host
// memory in the reference layout and are updated in place.
extern "C" int ref_cuda_run(int precision, int nx, int ny, int free_surface, int collision, int subgrid,
                            int use_force, double tau, double fx, double fy, uint64_t t0, uint64_t nsteps,
                            int kernel_id, void* f, void* rho, void* u, uint8_t* flags, void* mass, void* excess,
                            void* phi) {
  if (nx < 3 || ny < 3) return -1;
  if (precision == 32)
    return run_ref<float>(nx, ny, free_surface, collision, subgrid, use_force, tau, fx, fy, t0, nsteps, kernel_id, f,
                          rho, u, flags, mass, excess, phi);
  if (precision == 64)
    return run_ref<double>(nx, ny, free_surface, collision, subgrid, use_force, tau, fx, fy, t0, nsteps, kernel_id,
                           f, rho, u, flags, mass, excess, phi);
  return -1;
}

// Device time of the reference's headless step sequence: from the state in the
// buffers, `warm` steps from t0, then nsteps more timed with CUDA events
// (default stream, one launch per kernel and step as runCuda.cu issues them);
// *ms receives the timed milliseconds and the buffers the final state.
extern "C" int ref_cuda_time(int precision, int nx, int ny, int free_surface, int collision, int subgrid,
                             int use_force, double tau, double fx, double fy, uint64_t t0, uint64_t warm,
                             uint64_t nsteps, void* f, void* rho, void* u, uint8_t* flags, void* mass,
                             void* excess, void* phi, double* ms) {
  if (nx < 3 || ny < 3 || !ms || nsteps == 0) return -1;
  *ms = 0.0;
  if (precision == 32)
    return run_ref<float>(nx, ny, free_surface, collision, subgrid, use_force, tau, fx, fy, t0, nsteps, -1, f, rho,
                          u, flags, mass, excess, phi, warm, ms);
  if (precision == 64)
    return run_ref<double>(nx, ny, free_surface, collision, subgrid, use_force, tau, fx, fy, t0, nsteps, -1, f,
                           rho, u, flags, mass, excess, phi, warm, ms);
  return -1;
}

// The reference's iso-line kernel on a two-component field v (host, 2N values
// of the precision, v[c] and v[c + N]) into a width x height uint8 image
// (host, row-major, row 0 = the surface's row 0): 16x16 blocks over the
// lattice, as the viewer launches it.  Every pixel it writes lies inside the
// image for camera bounds b0 < b1 <= nx, b2 < b3 <= ny and finite values (the
// pixel mapping of drawLine, cudaIsosurface.cu:23-31, keeps both end points
// of a segment inside and Bresenham stays between them); other inputs are
// refused here (-2), because the kernel writes through a surface that traps
// out of range.
extern "C" int ref_cuda_isoline(int precision, int nx, int ny, const void* v, float iso, unsigned width,
                                unsigned height, const unsigned bounds[4], uint8_t* img) {
  if (nx < 3 || ny < 3 || width == 0 || height == 0 || !v || !img || !bounds) return -1;
  if (!(bounds[0] < bounds[1] && bounds[1] <= (unsigned)nx && bounds[2] < bounds[3] && bounds[3] <= (unsigned)ny))
    return -2;
  if (!std::isfinite(iso)) return -2;
  const unsigned Nx = (unsigned)nx, Ny = (unsigned)ny, N = Nx * Ny;
  const size_t es = precision == 64 ? 8 : 4;
  for (size_t k = 0; k < 2ull * N; k++) {
    const double x = precision == 64 ? static_cast<const double*>(v)[k] : static_cast<const float*>(v)[k];
    if (!std::isfinite(x)) return -2;
  }
  // __constant__ sizes of the kernels (d_Nx, d_Ny, d_N), as the solver set-up uploads them
  static float wf[9] = {4.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f, 1.0f / 9.0f,
                        1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f, 1.0f / 36.0f};
  static double wd[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                         1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  FLB::OptionsCalculation opts;
  opts.graphicsAPI = FLB::API::NONE;
  opts.typeProblem = FLB::TypeProblem::MONOFLUID;
  opts.relaxationTime = 0.6;
  opts.precision = precision == 64 ? 64 : 32;
  FLB::Units units;
  if (precision == 64) FLB::h_initConstantDataCuda2D<double>(opts, wd, Nx, Ny, N, units);
  else FLB::h_initConstantDataCuda2D<float>(opts, wf, Nx, Ny, N, units);
  void* d_v = nullptr;
  cudaArray_t arr = nullptr;
  cudaSurfaceObject_t surf = 0;
  cudaError_t e = cudaMalloc(&d_v, 2ull * N * es);
  if (e == cudaSuccess) e = cudaMemcpy(d_v, v, 2ull * N * es, cudaMemcpyHostToDevice);
  cudaChannelFormatDesc cd = cudaCreateChannelDesc<unsigned char>();
  if (e == cudaSuccess) e = cudaMallocArray(&arr, &cd, width, height, cudaArraySurfaceLoadStore);
  std::vector<uint8_t> zero((size_t)width * height, 0);
  if (e == cudaSuccess) e = cudaMemcpy2DToArray(arr, 0, 0, zero.data(), width, width, height, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    e = cudaCreateSurfaceObject(&surf, &rd);
  }
  if (e == cudaSuccess) {
    dim3 block(16, 16);
    dim3 grid((Nx + block.x - 1) / block.x, (Ny + block.y - 1) / block.y);
    if (precision == 64)
      FLB::d_CreateIsoSurfaceVector2D<double><<<grid, block>>>(static_cast<const double*>(d_v), surf, width, height,
                                                               iso, bounds[0], bounds[1], bounds[2], bounds[3]);
    else
      FLB::d_CreateIsoSurfaceVector2D<float><<<grid, block>>>(static_cast<const float*>(d_v), surf, width, height,
                                                              iso, bounds[0], bounds[1], bounds[2], bounds[3]);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
  }
  if (e == cudaSuccess) e = cudaMemcpy2DFromArray(img, width, arr, 0, 0, width, height, cudaMemcpyDeviceToHost);
  if (surf) cudaDestroySurfaceObject(surf);
  if (arr) cudaFreeArray(arr);
  if (d_v) cudaFree(d_v);
  return e == cudaSuccess ? 0 : (int)e;
}
