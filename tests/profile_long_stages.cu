// Profiling utility (not part of the library build): the instruction cost
// of the long-line kernel's stage code on shared-memory data, with no HBM
// traffic in the loop.  Mode 0 runs ilv_fft (two radix-16 stages over 8
// interleaved 256-point columns) with every stage in shared memory; mode 1
// sends the last stage through the column epilogue (inter-pass twiddle and
// global store) into a scratch region per CTA (CTA b writes only
// [b*Nx*N2, (b+1)*Nx*N2)).  Build and run:
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        --expt-relaxed-constexpr -I include -I wgpufft_b200/csrc \
//        -o profile_long_stages tests/profile_long_stages.cu
//   ./profile_long_stages
#include <cstdio>
#include <vector>
#include "longpass.cuh"
using namespace b2f;

__global__ void __launch_bounds__(kLongThreads, 2)
    k_probe(LongSched sch, uint32_t lg, uint32_t nx, uint32_t cap, const c32* tab, c32* scratch,
            uint32_t N2, int reps, int mode, c32* out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c32* a = reinterpret_cast<c32*>(smem_raw);
  c32* b = a + cap;
  c32* T = b + cap;
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < cap; i += kLongThreads) a[i] = c32{1e-3f * (float)i, 0.5f};
  for (uint32_t i = tid; i < kLongTab; i += kLongThreads) T[i] = tab[i];
  __syncthreads();
  const uint32_t G = 1u << lg, l = tid & (G - 1);
  for (int r = 0; r < reps; ++r) {
    if (mode == 0) {
      c32* res = ilv_fft(a, b, sch, lg, tid, T, EpiNone());
      if (res != a) {
        b = a;
        a = res;
      }
    } else {
      EpiCol e;
      e.c = l;
      e.ok = true;
      e.dst = scratch + (uint64_t)blockIdx.x * nx * N2 + l;
      e.sh = 8;
      e.T = T;
      e.N2 = N2;
      ilv_fft(a, b, sch, lg, tid, T, e);
    }
    __syncthreads();
  }
  if (tid < cap) out[blockIdx.x * kLongThreads + tid] = a[tid];
}

int main() {
  const uint32_t nx = 256, lg = 3, G = 8, P = G + 1, cap = nx * P, N2 = 256;
  LongSched sch{};
  sch.nst = 2;
  sch.st[0] = StageDesc{16, 1, 16, 0, make_fastdiv(1), make_fastdiv(16)};
  sch.st[1] = StageDesc{16, 16, 16, 0, make_fastdiv(16), make_fastdiv(16)};
  std::vector<c32> htab(kLongTab);
  for (uint32_t i = 0; i < kLongTab; ++i) htab[i] = c32{0.6f, 0.8f};
  const int blocks = 296, reps = 200;
  c32 *dtab, *dscr, *dout;
  cudaMalloc(&dtab, kLongTab * sizeof(c32));
  cudaMalloc(&dscr, (size_t)blocks * nx * N2 * sizeof(c32));
  cudaMalloc(&dout, (size_t)blocks * kLongThreads * sizeof(c32));
  cudaMemcpy(dtab, htab.data(), kLongTab * sizeof(c32), cudaMemcpyHostToDevice);
  const size_t smem = (2 * cap + kLongTab) * sizeof(c32);
  cudaFuncSetAttribute(k_probe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  for (int mode = 0; mode < 2; ++mode) {
    for (int w = 0; w < 2; ++w)
      k_probe<<<blocks, kLongThreads, smem>>>(sch, lg, nx, cap, dtab, dscr, N2, reps, mode, dout);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    k_probe<<<blocks, kLongThreads, smem>>>(sch, lg, nx, cap, dtab, dscr, N2, reps, mode, dout);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double pts = (double)blocks * G * nx * reps;
    printf("mode %d: %.3f ms, %.3f ns per point per FFT, err %s\n", mode, ms, ms * 1e6 / pts,
           cudaGetErrorString(cudaGetLastError()));
  }
  return 0;
}
