// Records cvt.rs.f16x2.f32 (binary32 pair -> binary16 pair, stochastic
// rounding with caller-supplied random bits) on the GPU for 65536 seeded
// vectors: values of magnitude 1e-6 (binary16 subnormal results), 1, 1000 and
// 60000, random bits per pair.  One thread per vector, every access in
// bounds.  Output: argv[1] (default f16_rs_probe.bin) = a, b, rbits, result as
// four arrays of 65536 uint32.  make_f16_rs_fixture.py compiles and runs it
// and keeps a subset as f16_rs_probe.npz.
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>
__global__ void k(const float* a, const float* b, const uint32_t* r, uint32_t* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t d;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a[i]), "f"(b[i]), "r"(r[i]));
  out[i] = d;
}
int main(int argc, char** argv) {
  const int n = 1 << 16;
  std::vector<float> a(n), b(n);
  std::vector<uint32_t> r(n), o(n);
  srand(1234);
  for (int i = 0; i < n; i++) {
    float s = (i % 4 == 0) ? 1e-6f : (i % 4 == 1 ? 1.0f : (i % 4 == 2 ? 1000.0f : 60000.0f));
    a[i] = s * ((rand() / (float)RAND_MAX) * 2.0f - 1.0f);
    b[i] = s * ((rand() / (float)RAND_MAX) * 2.0f - 1.0f);
    r[i] = ((uint32_t)rand() << 16) ^ (uint32_t)rand();
  }
  float *da, *db; uint32_t *dr, *dout;
  cudaMalloc(&da, n * 4); cudaMalloc(&db, n * 4); cudaMalloc(&dr, n * 4); cudaMalloc(&dout, n * 4);
  cudaMemcpy(da, a.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(db, b.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dr, r.data(), n * 4, cudaMemcpyHostToDevice);
  k<<<(n + 255) / 256, 256>>>(da, db, dr, dout, n);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { printf("error %s\n", cudaGetErrorString(e)); return 1; }
  cudaMemcpy(o.data(), dout, n * 4, cudaMemcpyDeviceToHost);
  FILE* f = fopen(argc > 1 ? argv[1] : "f16_rs_probe.bin", "wb");
  if (!f) return 1;
  fwrite(a.data(), 4, n, f); fwrite(b.data(), 4, n, f); fwrite(r.data(), 4, n, f); fwrite(o.data(), 4, n, f);
  fclose(f);
  printf("ok %d\n", n);
  return 0;
}
