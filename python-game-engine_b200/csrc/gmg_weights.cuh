// Transfer weights and relaxation reciprocals shared by the multigrid kernels of gmg.cu and
// batch.cu (included inside namespace sg).
#pragma once

// 1-D prolongation weight of fine index i onto coarse index I (grid of n coarse cells).
__device__ __forceinline__ float w1(int i, int I, int n) {
  int h = i >> 1;
  int x = h + ((i & 1) ? 1 : -1);
  x = x < 0 ? 0 : (x > n - 1 ? n - 1 : x);
  return (h == I ? 0.75f : 0.0f) + (x == I ? 0.25f : 0.0f);
}

// 1 / (number of open faces), n in 1..4.
template <typename T>
__device__ __forceinline__ T rcp_open(int n) {
  return n == 4 ? (T)0.25 : (n == 3 ? (T)(1.0 / 3.0) : (n == 2 ? (T)0.5 : (T)1.0));
}
