// Microbenchmark behind the fixed-point p2g tile: shared-memory float vs int32 vs 64-bit integer
// atomicAdd, random and conflict-free addresses, on the current GPU.  Build: nvcc -gencode arch=compute_100a,code=sm_100a -O3
//   -o microbench_shared_atomics genesis_b200/csrc/microbench_shared_atomics.cu
#include <cstdio>
#include <cuda_runtime.h>
__device__ __forceinline__ unsigned hsh(unsigned x){ x ^= x >> 16; x *= 0x7feb352d; x ^= x >> 15; x *= 0x846ca68b; x ^= x >> 16; return x; }
template <int MODE>
__global__ void k(float* out, int iters) {
  __shared__ float sf[512]; __shared__ int si[512]; __shared__ unsigned long long su[256];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) { sf[i] = 0.f; si[i] = 0; }
  for (int i = threadIdx.x; i < 256; i += blockDim.x) su[i] = 0ull;
  __syncthreads();
  unsigned h = hsh(threadIdx.x + 7919u * blockIdx.x);
  float accf = 0.f;
  for (int it = 0; it < iters; ++it) {
    h = hsh(h);
    int a_rand = h & 511;             // 0..511, in bounds
    int a_cf = (threadIdx.x & 31) + ((it & 15) << 5);  // distinct banks within a warp, in bounds
    if (MODE == 0) atomicAdd(&sf[a_rand], 1.0f);
    if (MODE == 1) atomicAdd(&si[a_rand], 1);
    if (MODE == 2) atomicAdd(&sf[a_cf], 1.0f);
    if (MODE == 3) atomicAdd(&si[a_cf], 1);
    if (MODE == 4) { sf[a_cf] += 1.0f; }
    if (MODE == 5) atomicAdd(&su[h & 255], 0x100000001ull);                      // 0..255, in bounds
    if (MODE == 6) atomicAdd(&su[(threadIdx.x & 31) + ((it & 7) << 5)], 0x100000001ull);  // 0..255
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 512; i += blockDim.x) accf += sf[i] + (float)si[i];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) accf += (float)su[i];
  if (accf == -1.f) out[0] = accf;
}
int main() {
  float* d; cudaMalloc(&d, 4);
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  const int ctas = 148 * 4, thr = 256, iters = 4096;
  const char* names[] = {"f32 atomic random", "i32 atomic random", "f32 atomic conflict-free", "i32 atomic conflict-free",
                         "f32 plain RMW conflict-free", "u64 atomic random", "u64 atomic conflict-free"};
  for (int rep = 0; rep < 2; ++rep)
  for (int m = 0; m < 7; ++m) {
    cudaEventRecord(a);
    switch (m) { case 0: k<0><<<ctas,thr>>>(d, iters); break; case 1: k<1><<<ctas,thr>>>(d, iters); break;
                 case 2: k<2><<<ctas,thr>>>(d, iters); break; case 3: k<3><<<ctas,thr>>>(d, iters); break;
                 case 4: k<4><<<ctas,thr>>>(d, iters); break; case 5: k<5><<<ctas,thr>>>(d, iters); break;
                 case 6: k<6><<<ctas,thr>>>(d, iters); break; }
    cudaEventRecord(b); cudaEventSynchronize(b);
    float ms; cudaEventElapsedTime(&ms, a, b);
    double ops = (double)ctas * thr * iters;
    if (rep) printf("%-30s %8.3f ms  %8.2f Gop/s  %6.2f clk/warp-op/SM\n", names[m], ms, ops / ms / 1e6, (ms * 1e-3 * 1.9e9 * 148) / (ops / 32));
  }
  cudaError_t e = cudaGetLastError(); printf("err=%s\n", cudaGetErrorString(e));
  return 0;
}
