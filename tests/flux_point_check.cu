// Host harness for the flux kernels' point functions (canard_b200/csrc/kernels.cuh),
// run without a GPU (it calls no CUDA API). stdin: int32 mode, n, viscous flag,
// the frame velocity as 3 doubles, then the points' inputs; stdout: 16 values per
// point, the 15 flux components (field (m-1)*3 + d) and de(:,5).
//   mode 0: flux_visc_values, the FP32 pair kernel's point (k_flux_visc_pairs);
//           inputs n x 28 float: 12 gradients, 9 metric terms [d][c], mu, yaco,
//           p, 1/rho, u, v, w. Outputs float.
//   mode 1: visc_point + flux_point<double> with the state preloaded, as in
//           k_flux_visc<double>; mode 2: the same with flux_point reading p and
//           the state itself, as in k_flux (the phase API). Inputs n x 33 double:
//           the 28 of mode 0 (1/rho unused), then the five conserved values.
//           Outputs double.
#include <cstdio>
#include <vector>

#include "kernels.cuh"

namespace {

template <class T>
bool read_all(std::vector<T>& v) {
  return std::fread(v.data(), sizeof(T), v.size(), stdin) == v.size();
}

template <class T>
bool write_all(const std::vector<T>& v) {
  return std::fwrite(v.data(), sizeof(T), v.size(), stdout) == v.size();
}

int run_f32(int n, bool visc, const double um[3]) {
  std::vector<float> in((size_t)n * 28), out((size_t)n * 16);
  if (!read_all(in)) return 2;
  for (int i = 0; i < n; ++i)
    canard::flux_visc_values(&in[(size_t)i * 28], visc, float(um[0]), float(um[1]), float(um[2]),
                             &out[(size_t)i * 16]);
  return write_all(out) ? 0 : 3;
}

int run_f64(int n, bool visc, const double um[3], bool preload) {
  std::vector<double> in((size_t)n * 33);
  if (!read_all(in)) return 2;
  const size_t N = (size_t)n;
  // the block's fields, one point per input row
  std::vector<double> scr(15 * N), xim(3 * N), etm(3 * N), zem(3 * N), mu(N), yaco(N), p(N), de(5 * N), qa(5 * N);
  for (size_t l = 0; l < N; ++l) {
    const double* a = &in[l * 33];
    for (int k = 0; k < 12; ++k) scr[k * N + l] = a[k];
    for (int c = 0; c < 3; ++c) {
      xim[c * N + l] = a[12 + c];
      etm[c * N + l] = a[15 + c];
      zem[c * N + l] = a[18 + c];
    }
    mu[l] = a[21];
    yaco[l] = a[22];
    p[l] = a[23];
    de[l] = a[21];
    for (int c = 0; c < 3; ++c) de[(1 + c) * N + l] = a[25 + c];
    for (int c = 0; c < 5; ++c) qa[c * N + l] = a[28 + c];
  }
  const canard::Work<double> W{de.data(), p.data(), mu.data(), nullptr, scr.data(),
                               xim.data(), etm.data(), zem.data(), yaco.data()};
  canard::BlockDev B{};
  B.qa = qa.data();
  canard::StageParams S{};
  for (int c = 0; c < 3; ++c) S.umf[c] = um[c];
  std::vector<double> out(16 * N);
  for (long long l = 0; l < (long long)N; ++l) {
    double t[9] = {};
    if (visc) {
      double d5;
      canard::visc_point<double>(W, l, (long long)N, mu[l], t, d5);
    }
    if (preload) {
      double pre[6];
      pre[0] = p[l];
      for (int c = 0; c < 5; ++c) pre[1 + c] = qa[c * N + l];
      canard::flux_point<double>(W, B, S, visc, l, (long long)N, t, pre);
    } else {
      canard::flux_point<double>(W, B, S, visc, l, (long long)N, t);
    }
    for (int k = 0; k < 15; ++k) out[l * 16 + k] = scr[k * N + l];
    out[l * 16 + 15] = de[4 * N + l];
  }
  return write_all(out) ? 0 : 3;
}

}  // namespace

int main() {
  int head[3];
  double um[3];
  if (std::fread(head, sizeof(int), 3, stdin) != 3 || std::fread(um, sizeof(double), 3, stdin) != 3 || head[1] <= 0)
    return 2;
  const int mode = head[0], n = head[1];
  const bool visc = head[2] != 0;
  if (mode == 0) return run_f32(n, visc, um);
  if (mode == 1 || mode == 2) return run_f64(n, visc, um, mode == 1);
  return 2;
}
