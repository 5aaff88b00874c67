// Microbenchmark: ceilings of streaming, random gathers and stream x gather for the
// large LP shape (21M nonzeros, 2M columns). Build and run:
//   nvcc -O3 -gencode arch=compute_100a,code=sm_100a -o /tmp/gather_ceiling vikalp_b200/microbench/gather_ceiling.cu && /tmp/gather_ceiling
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <random>
#include <cuda_runtime.h>
#define CK(x) do { cudaError_t e = (x); if (e != cudaSuccess) { printf("err %s line %d\n", cudaGetErrorString(e), __LINE__); exit(1);} } while (0)

template <int U, int MODE>  // MODE 0: stream only, 1: gather only (ci streamed), 2: stream*gather
__global__ void __launch_bounds__(256) k(const int* __restrict__ ci, const double* __restrict__ val, const double* __restrict__ x, long n, double* out) {
  double s = 0;
  long stride = (long)gridDim.x * blockDim.x * U;
  for (long base = (long)blockIdx.x * blockDim.x * U + threadIdx.x; base < n; base += stride) {
    int c[U]; double v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) { long i = base + (long)u * blockDim.x; c[u] = i < n ? __ldg(ci + i) : 0; if (MODE != 1) v[u] = i < n ? __ldg(val + i) : 0.0; }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      long i = base + (long)u * blockDim.x;
      if (i < n) {
        if (MODE == 0) s += v[u] + (double)c[u];
        else if (MODE == 1) s += __ldg(x + c[u]);
        else s += v[u] * __ldg(x + c[u]);
      }
    }
  }
  if (s == 12345.678) out[0] = s;
}

template <int U, int MODE>
float run(const int* ci, const double* val, const double* x, long n, double* out, int blocks) {
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  for (int w = 0; w < 3; ++w) k<U, MODE><<<blocks, 256>>>(ci, val, x, n, out);
  float best = 1e9;
  for (int r = 0; r < 10; ++r) {
    cudaEventRecord(a); k<U, MODE><<<blocks, 256>>>(ci, val, x, n, out); cudaEventRecord(b); cudaEventSynchronize(b);
    float ms; cudaEventElapsedTime(&ms, a, b); if (ms < best) best = ms;
  }
  CK(cudaGetLastError());
  return best;
}

int main() {
  const long n = 21000000; const int ncols = 2000000;
  std::vector<int> hci(n); std::mt19937 rng(1); for (long i = 0; i < n; ++i) hci[i] = rng() % ncols;
  int* ci; double *val, *x, *out;
  CK(cudaMalloc(&ci, n * 4)); CK(cudaMalloc(&val, n * 8)); CK(cudaMalloc(&x, ncols * 8)); CK(cudaMalloc(&out, 8));
  CK(cudaMemcpy(ci, hci.data(), n * 4, cudaMemcpyHostToDevice));
  CK(cudaMemset(val, 0, n * 8)); CK(cudaMemset(x, 0, ncols * 8));
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  for (int bps : {4, 8}) {
    int blocks = sms * bps;
    printf("blocks/SM %d\n", bps);
    printf(" stream(12B/nnz)  U4 %.3f ms %.0f GB/s | U8 %.3f ms\n", run<4,0>(ci,val,x,n,out,blocks), n*12.0/run<4,0>(ci,val,x,n,out,blocks)/1e6, run<8,0>(ci,val,x,n,out,blocks));
    float g4 = run<4,1>(ci,val,x,n,out,blocks), g8 = run<8,1>(ci,val,x,n,out,blocks), g16 = run<16,1>(ci,val,x,n,out,blocks);
    printf(" gather only      U4 %.3f U8 %.3f U16 %.3f ms  (%.0f Ggather/s best)\n", g4, g8, g16, n / (g4 < g8 ? (g4 < g16 ? g4 : g16) : (g8 < g16 ? g8 : g16)) / 1e6);
    float s4 = run<4,2>(ci,val,x,n,out,blocks), s8 = run<8,2>(ci,val,x,n,out,blocks), s16 = run<16,2>(ci,val,x,n,out,blocks);
    printf(" stream*gather    U4 %.3f U8 %.3f U16 %.3f ms\n", s4, s8, s16);
  }
  // gather from a small (L1/L2-friendly) range: 64K columns
  for (long i = 0; i < n; ++i) hci[i] = hci[i] % 65536;
  CK(cudaMemcpy(ci, hci.data(), n * 4, cudaMemcpyHostToDevice));
  printf("narrow x (64K cols): stream*gather U8 %.3f ms\n", run<8,2>(ci,val,x,n,out,sms*8));
  // sorted indices within blocks of 1024 (locality)
  return 0;
}
