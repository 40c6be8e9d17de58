// Test kernel: fb_quot (one shared reciprocal + Markstein's correction)
// against IEEE division, element by element.
#include <cuda_runtime.h>
#include "fb_dev.cuh"

__global__ void k_quot(int n, const double *a, const double *d, unsigned long long *mismatch, double *qa, double *qb)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double r = 1.0 / d[t];
  const double x = fb_quot(a[t], d[t], r), y = a[t] / d[t];
  qa[t] = x;
  qb[t] = y;
  if (__double_as_longlong(x) != __double_as_longlong(y)) atomicAdd(mismatch, 1ull);
}

extern "C" int quot_check(int n, const double *ha, const double *hd, double *hqa, double *hqb, unsigned long long *hmis)
{
  double *a, *d, *qa, *qb;
  unsigned long long *m;
  const size_t b = (size_t)n * sizeof(double);
  if (cudaMalloc(&a, b) || cudaMalloc(&d, b) || cudaMalloc(&qa, b) || cudaMalloc(&qb, b) ||
      cudaMalloc(&m, sizeof(*m)))
    return 1;
  cudaMemcpy(a, ha, b, cudaMemcpyHostToDevice);
  cudaMemcpy(d, hd, b, cudaMemcpyHostToDevice);
  cudaMemset(m, 0, sizeof(*m));
  k_quot<<<(n + 255) / 256, 256>>>(n, a, d, m, qa, qb);
  cudaMemcpy(hqa, qa, b, cudaMemcpyDeviceToHost);
  cudaMemcpy(hqb, qb, b, cudaMemcpyDeviceToHost);
  cudaMemcpy(hmis, m, sizeof(*m), cudaMemcpyDeviceToHost);
  const int rc = cudaGetLastError() != cudaSuccess;
  cudaFree(a); cudaFree(d); cudaFree(qa); cudaFree(qb); cudaFree(m);
  return rc;
}
