// Host harness for the FP32 fused flux kernel's point function
// (canard::flux_visc_values, canard_b200/csrc/kernels.cuh): reads n, the
// viscous flag, the frame velocity (3 floats) and n x 28 float inputs from
// stdin, writes n x 16 float outputs to stdout. Calls no CUDA API, so it runs
// without a GPU.
#include <cstdio>
#include <vector>

#include "kernels.cuh"

int main() {
  int n = 0, visc = 0;
  float um[3];
  if (std::fread(&n, sizeof(int), 1, stdin) != 1 || std::fread(&visc, sizeof(int), 1, stdin) != 1 ||
      std::fread(um, sizeof(float), 3, stdin) != 3 || n <= 0)
    return 2;
  std::vector<float> in((size_t)n * 28), out((size_t)n * 16);
  if (std::fread(in.data(), sizeof(float), in.size(), stdin) != in.size()) return 2;
  for (int i = 0; i < n; ++i)
    canard::flux_visc_values(&in[(size_t)i * 28], visc != 0, um[0], um[1], um[2], &out[(size_t)i * 16]);
  return std::fwrite(out.data(), sizeof(float), out.size(), stdout) == out.size() ? 0 : 3;
}
