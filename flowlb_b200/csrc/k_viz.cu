// k_viz.cu -- headless visualisation: the CUDA side of FlowLB's OpenGL view,
// drawn into device buffers in place of the OpenGL interop surfaces.
//
//   k_viz_uv       save2DDataToOpenGL (src/cuda/cudaUtils.cu:107-118): the
//                  velocity field as an interleaved float2 image
//   k_viz_shade    the fragment stage of the texture*2D shaders
//                  (assets/shaders/*/texture{X,Y}Velocity2D.glsl,
//                  textureMagnitudeVelocity2D.glsl, texturePressure2D.glsl):
//                  normalise, clamp at 0, look up a 1D colour map with linear
//                  filtering and mirrored-repeat wrapping (OpenGLTexture1D,
//                  src/graphics/OpenGL/OpenGLTexture.cpp:44-53), one pixel per
//                  lattice node, RGBA8
//   k_viz_isoline  d_CreateIsoSurfaceVector2D (src/cuda/cudaIsosurface.cuh:33-199,
//                  cudaIsosurface.cu:16-76): marching squares over the
//                  camera window, each edge segment rasterised with
//                  Bresenham's algorithm into a uint8 image
//
// All three are HBM-light (a few bytes per node); they run once per frame.
// Magnitudes are sqrt(x*x + y*y) with IEEE rounding of each operation (the
// reference calls hypotf, whose result may differ in the last bits); every
// other float operation follows the reference's order, so a CPU restatement
// reproduces the images exactly.
#include <cstdint>

#include "launch.h"

namespace flb {

namespace {

constexpr uint32_t kVizBlock = 256;

template <class T>
__device__ __forceinline__ float magnitude(T a, T b) {
  const float x = (float)a, y = (float)b;
  return __fsqrt_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
}

template <class T>
__global__ void k_viz_uv(const T* __restrict__ u, float2* __restrict__ out, uint32_t N) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  out[i] = make_float2((float)u[i], (float)u[i + N]);
}

// OpenGL's texel index wrap for GL_MIRRORED_REPEAT on a texture of n texels.
__device__ __forceinline__ int mirrored(int i, int n) {
  const int two = 2 * n;
  int j = i % two;
  if (j < 0) j += two;
  return j < n ? j : two - 1 - j;
}

__device__ __forceinline__ uint8_t unorm8(float c) {
  c = fminf(fmaxf(c, 0.0f), 1.0f);
  return (uint8_t)__float2int_rn(__fmul_rn(c, 255.0f));
}

template <class T>
__global__ void k_viz_shade(const T* __restrict__ u, uint32_t N, int quantity, const float* __restrict__ cmap,
                            uint32_t n, float vmax, float vmin, uchar4* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float ux = (float)u[i], uy = (float)u[i + N];
  float v;
  if (quantity == FLB_VIZ_UX) v = ux;
  else if (quantity == FLB_VIZ_UY) v = uy;
  else v = magnitude(ux, uy);  // magnitude and pressure shaders: length(texture.xy)
  float s = __fdiv_rn(__fsub_rn(v, vmin), __fsub_rn(vmax, vmin));
  s = (s < 0.0f) ? 0.0f : s;       // GLSL max(s, 0)
  if (!(s == s)) s = 0.0f;         // NaN: no defined colour in GLSL; black-body start of the map
  s = fminf(s, 1024.0f);           // keeps the texel index in int range (values far above the map)
  const float coord = __fsub_rn(__fmul_rn(s, (float)n), 0.5f);
  const float fl = floorf(coord);
  const float a = __fsub_rn(coord, fl);
  const int i0 = mirrored((int)fl, (int)n), i1 = mirrored((int)fl + 1, (int)n);
  float c[3];
#pragma unroll
  for (int k = 0; k < 3; k++)
    c[k] = __fadd_rn(__fmul_rn(__fsub_rn(1.0f, a), cmap[3 * i0 + k]), __fmul_rn(a, cmap[3 * i1 + k]));
  out[i] = make_uchar4(unorm8(c[0]), unorm8(c[1]), unorm8(c[2]), 255);
}

struct IsoView {
  uint32_t nx, ny, N;
  uint32_t width, height;
  uint32_t bx0, bx1, by0, by1;  // camera window in lattice nodes: [bx0, bx1) x [by0, by1)
  float iso;
};

__device__ __forceinline__ float2 interp(float2 p0, float2 p1, float v0, float v1, float iso) {
  const float aux = __fdiv_rn(__fsub_rn(iso, v0), __fsub_rn(v1, v0));
  const float aux2 = __fsub_rn(1.0f, aux);
  return make_float2(__fadd_rn(__fmul_rn(aux2, p0.x), __fmul_rn(aux, p1.x)),
                     __fadd_rn(__fmul_rn(aux2, p0.y), __fmul_rn(aux, p1.y)));
}

// drawLine (cudaIsosurface.cu:23-66).  The reference writes through a surface
// that traps outside the image; here a pixel outside is skipped, and a segment
// whose end points are not finite or lie far outside the image is not drawn.
__device__ void draw_line(float2 p0, float2 p1, float2 ppn, float xo, float yo, uint8_t* img, const IsoView& v) {
  const float xp0 = __fadd_rn(p0.x, xo), xp1 = __fadd_rn(p1.x, xo);
  const float yp0 = __fadd_rn(p0.y, yo), yp1 = __fadd_rn(p1.y, yo);
  const float fx0 = __fadd_rn(__fsub_rn(__fmul_rn(ppn.x, xp0), 1.0f * (float)((int)xp0 != 0)), 0.5f);
  const float fx1 = __fadd_rn(__fsub_rn(__fmul_rn(ppn.x, xp1), 1.0f * (float)((int)xp1 != 0)), 0.5f);
  const float fy0 = __fsub_rn(__fsub_rn((float)v.height, __fmul_rn(ppn.y, yp0)), 0.5f);
  const float fy1 = __fsub_rn(__fsub_rn((float)v.height, __fmul_rn(ppn.y, yp1)), 0.5f);
  const float lim_x = (float)v.width + 2.0f, lim_y = (float)v.height + 2.0f;
  if (!(fabsf(fx0) <= lim_x && fabsf(fx1) <= lim_x && fabsf(fy0) <= lim_y && fabsf(fy1) <= lim_y)) return;
  int x0 = (int)fx0, y0 = (int)fy0;
  const int x1 = (int)fx1, y1 = (int)fy1;
  // Bresenham (Zingl 2016), as the reference: the last point is not drawn
  const int dx = abs(x1 - x0), dy = -abs(y1 - y0);
  int err = dx + dy;
  const int sx = 2 * (x0 < x1) - 1, sy = 2 * (y0 < y1) - 1;
  for (int guard = dx - dy + 1; (x0 != x1 || y0 != y1) && guard > 0; guard--) {
    if (x0 >= 0 && y0 >= 0 && (uint32_t)x0 < v.width && (uint32_t)y0 < v.height) img[(size_t)y0 * v.width + x0] = 255;
    const int e2 = 2 * err;
    if (e2 >= dy) {
      err += dy;
      x0 += sx;
    }
    if (e2 <= dx) {
      err += dx;
      y0 += sy;
    }
  }
}

// VEC: the node value is the magnitude of a two-component field (velocity);
// otherwise the field is scalar (the fill fraction).
template <class T, bool VEC>
__global__ void k_viz_isoline(const T* __restrict__ f, uint8_t* __restrict__ img, IsoView v) {
  const uint32_t x = threadIdx.x + blockIdx.x * blockDim.x;
  const uint32_t y = threadIdx.y + blockIdx.y * blockDim.y;
  if (x >= v.nx - 1 || y >= v.ny - 1) return;
  if (x < v.bx0 || x >= v.bx1 || y < v.by0 || y >= v.by1) return;
  const uint32_t idx = x + (v.ny - y - 1) * v.nx;  // the view's y runs downwards
  const uint32_t c[4] = {idx, idx + 1, idx - v.nx + 1, idx - v.nx};
  float val[4];
#pragma unroll
  for (int k = 0; k < 4; k++) val[k] = VEC ? magnitude(f[c[k]], f[c[k] + v.N]) : (float)f[c[k]];
  const uint32_t sq = (val[0] > v.iso) | ((val[1] > v.iso) << 1) | ((val[2] > v.iso) << 2) | ((val[3] > v.iso) << 3);
  if (sq == 0 || sq == 15) return;
  const float2 P[4] = {{0.0f, 0.0f}, {1.0f, 0.0f}, {1.0f, 1.0f}, {0.0f, 1.0f}};
  const float2 ppn = make_float2(__fdiv_rn((float)v.width, (float)(v.bx1 - v.bx0)),
                                 __fdiv_rn((float)v.height, (float)(v.by1 - v.by0)));
  const float xo = (float)(x - v.bx0), yo = (float)(y - v.by0);
  auto e = [&](int a, int b) { return interp(P[a], P[b], val[a], val[b], v.iso); };
  switch (sq) {  // the edge pairs of cudaIsosurface.cuh:74-196
    case 1:
    case 14: draw_line(e(0, 1), e(0, 3), ppn, xo, yo, img, v); break;
    case 2:
    case 13: draw_line(e(0, 1), e(1, 2), ppn, xo, yo, img, v); break;
    case 3:
    case 12: draw_line(e(0, 3), e(1, 2), ppn, xo, yo, img, v); break;
    case 4:
    case 11: draw_line(e(1, 2), e(3, 2), ppn, xo, yo, img, v); break;
    case 5:
      draw_line(e(0, 1), e(0, 3), ppn, xo, yo, img, v);
      draw_line(e(3, 2), e(1, 2), ppn, xo, yo, img, v);
      break;
    case 6:
    case 9: draw_line(e(0, 1), e(3, 2), ppn, xo, yo, img, v); break;
    case 7:
    case 8: draw_line(e(0, 3), e(3, 2), ppn, xo, yo, img, v); break;
    case 10:
      draw_line(e(0, 3), e(3, 2), ppn, xo, yo, img, v);
      draw_line(e(0, 1), e(1, 2), ppn, xo, yo, img, v);
      break;
    default: break;
  }
}

}  // namespace

template <class T>
void launch_viz_uv(const void* u, float* out, uint32_t N, cudaStream_t st) {
  k_viz_uv<T><<<(N + kVizBlock - 1) / kVizBlock, kVizBlock, 0, st>>>((const T*)u, (float2*)out, N);
}

template <class T>
void launch_viz_shade(const void* u, uint32_t N, int quantity, const float* cmap, uint32_t n, float vmax, float vmin,
                      uint8_t* rgba, cudaStream_t st) {
  k_viz_shade<T><<<(N + kVizBlock - 1) / kVizBlock, kVizBlock, 0, st>>>((const T*)u, N, quantity, cmap, n, vmax,
                                                                         vmin, (uchar4*)rgba);
}

template <class T>
void launch_viz_isoline(const void* f, bool vec, uint32_t nx, uint32_t ny, float iso, uint32_t width, uint32_t height,
                        const uint32_t bounds[4], uint8_t* img, cudaStream_t st) {
  IsoView v{nx, ny, nx * ny, width, height, bounds[0], bounds[1], bounds[2], bounds[3], iso};
  const dim3 block(16, 16);
  const dim3 grid((nx + 15) / 16, (ny + 15) / 16);
  if (vec) k_viz_isoline<T, true><<<grid, block, 0, st>>>((const T*)f, img, v);
  else k_viz_isoline<T, false><<<grid, block, 0, st>>>((const T*)f, img, v);
}

#define FLB_VIZ_INSTANTIATE(T)                                                                                  \
  template void launch_viz_uv<T>(const void*, float*, uint32_t, cudaStream_t);                                 \
  template void launch_viz_shade<T>(const void*, uint32_t, int, const float*, uint32_t, float, float, uint8_t*, \
                                    cudaStream_t);                                                              \
  template void launch_viz_isoline<T>(const void*, bool, uint32_t, uint32_t, float, uint32_t, uint32_t,         \
                                      const uint32_t[4], uint8_t*, cudaStream_t);
FLB_VIZ_INSTANTIATE(float)
FLB_VIZ_INSTANTIATE(double)

}  // namespace flb
