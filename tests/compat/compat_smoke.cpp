// Caller written against the reference's host API (the shapes of
// test/slabunified_test.cu:42-89 and test/set_test.cu:40-81), compiled
// against include/lslab_compat.h and linked with liblsb.so.
#include <cstdio>
#include <vector>

#include <cuda_runtime.h>

#include "lslab_compat.h"

#define CK(x)                                                         \
  do {                                                                \
    cudaError_t e = (x);                                              \
    if (e != cudaSuccess) {                                           \
      std::printf("cuda error %s at %d\n", cudaGetErrorString(e), __LINE__); \
      return 2;                                                       \
    }                                                                 \
  } while (0)

int main() {
  const size_t n = 1024;
  std::vector<uint64_t> hk(n), hv(n);
  for (size_t i = 0; i < n; ++i) hk[i] = i + 1;
  uint64_t *keys, *vals, *old;
  cuda::std::pair<bool, uint64_t>* got;
  CK(cudaMalloc(&keys, n * 8));
  CK(cudaMalloc(&vals, n * 8));
  CK(cudaMalloc(&old, n * 8));
  CK(cudaMalloc(&got, n * sizeof(*got)));
  CK(cudaMemcpy(keys, hk.data(), n * 8, cudaMemcpyHostToDevice));
  {
    lslab::map<uint64_t, uint64_t> m(10);
    for (uint64_t rep = 0; rep < 20; ++rep) {
      for (size_t i = 0; i < n; ++i) hv[i] = rep;
      CK(cudaMemcpy(vals, hv.data(), n * 8, cudaMemcpyHostToDevice));
      m.put(keys, vals, old, n);
      m.get<128>(keys, got, n);
      CK(cudaDeviceSynchronize());
      std::vector<uint64_t> ho(n);
      std::vector<cuda::std::pair<bool, uint64_t>> hg(n);
      CK(cudaMemcpy(ho.data(), old, n * 8, cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(hg.data(), got, n * sizeof(*got), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < n; ++i) {
        if (rep && ho[i] != rep - 1) { std::printf("put old mismatch\n"); return 1; }
        if (!hg[i].first || hg[i].second != rep) { std::printf("get mismatch\n"); return 1; }
      }
    }
    if (m.buckets() != 1024) return 1;
  }
  uint32_t* sk;
  bool* sr;
  std::vector<uint32_t> hs(n);
  for (size_t i = 0; i < n; ++i) hs[i] = (uint32_t)(i + 1);
  CK(cudaMalloc(&sk, n * 4));
  CK(cudaMalloc(&sr, n));
  CK(cudaMemcpy(sk, hs.data(), n * 4, cudaMemcpyHostToDevice));
  {
    lslab::set<uint32_t> s(10);
    for (int rep = 0; rep < 20; ++rep) {
      std::vector<char> hr(n);
      s.insert(sk, sr, n);
      s.contains(sk, sr, n);
      CK(cudaMemcpy(hr.data(), sr, n, cudaMemcpyDeviceToHost));
      for (char b : hr) if (!b) { std::printf("contains after insert\n"); return 1; }
      s.remove(sk, sr, n);
      s.contains(sk, sr, n);
      CK(cudaMemcpy(hr.data(), sr, n, cudaMemcpyDeviceToHost));
      for (char b : hr) if (b) { std::printf("contains after remove\n"); return 1; }
    }
  }
  try {
    lslab::map<uint64_t, uint64_t> bad(0);  // invalid size: reported, not trapped
    std::printf("no error for a zero-bucket map\n");
    return 1;
  } catch (const lslab::lsb_error& e) {
  }
  std::printf("compat ok\n");
  return 0;
}
