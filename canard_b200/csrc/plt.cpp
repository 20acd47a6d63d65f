// Tecplot binary output in the reference's layout (write_output_file_mb /
// techead / strio / vminmax, src/mo_io.f90:275-562). Host code, no device
// work. One file holds every block of a case: block 0's part starts with the
// file header (every zone's header), then each block contributes its zone
// section (per-variable format flags and FP64 min/max of its FP32 values)
// followed by its data, FP32, variable by variable, i fastest.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "canard_gpu.h"

namespace {

struct Out {
  std::vector<unsigned char> b;
  void i32(int32_t v) { raw(&v, 4); }
  void f32(float v) { raw(&v, 4); }
  void f64(double v) { raw(&v, 8); }
  void raw(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    b.insert(b.end(), c, c + n);
  }
  // strio: one 4-byte integer per character, then 0 (src/mo_io.f90:517-530)
  void str(const std::string& s) {
    for (char ch : s) i32((int32_t)(unsigned char)ch);
    i32(0);
  }
};

// three digits, as the reference builds names (0..999)
std::string three(int v) {
  char buf[16];
  std::snprintf(buf, sizeof buf, "%03d", v);
  return buf;
}

}  // namespace

extern "C" int canard_plt_write(const char* path, int32_t n, int32_t nblocks, const int32_t* dims, double time,
                                const float* const* data) {
  if (!path || nblocks < 1 || nblocks > 1000 || !dims || !data || n < -1 || n > 999) return CANARD_ERR_ARG;
  const int mq = n == -1 ? 3 : 5;
  for (int mb = 0; mb < nblocks; ++mb)
    if (!data[mb] || dims[3 * mb] < 1 || dims[3 * mb + 1] < 1 || dims[3 * mb + 2] < 1) return CANARD_ERR_ARG;
  Out o;
  // techead for block 0: the file header (src/mo_io.f90:426-487)
  o.raw("#!TDV112", 8);
  o.i32(1);
  o.i32(std::min(n + 2, 2));  // 1 grid, 2 solution
  o.str(n == -1 ? std::string("grid") : "n" + three(n));
  o.i32(mq);
  if (n == -1) {
    for (const char* v : {"x", "y", "z"}) o.str(v);
  } else {
    for (const char* v : {"rho", "u", "v", "w", "p"}) o.str(v);
  }
  for (int mm = 0; mm < nblocks; ++mm) {
    o.f32(299.0f);
    o.str("z" + three(mm));
    o.i32(-1);
    o.i32(mm + 1);
    o.f64(time);
    o.i32(-1);
    o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(dims[3 * mm]);
    o.i32(dims[3 * mm + 1]);
    o.i32(dims[3 * mm + 2]);
    o.i32(0);
  }
  o.f32(357.0f);
  // every block: its zone section (src/mo_io.f90:488-509) and data
  for (int mb = 0; mb < nblocks; ++mb) {
    const int64_t npts = (int64_t)dims[3 * mb] * dims[3 * mb + 1] * dims[3 * mb + 2];
    o.f32(299.0f);
    for (int m = 0; m < mq; ++m) o.i32(1);
    o.i32(0);
    o.i32(0);
    o.i32(-1);
    for (int m = 0; m < mq; ++m) {
      const float* v = data[mb] + m * npts;
      const auto mm = std::minmax_element(v, v + npts);
      o.f64((double)*mm.first);   // vminmax: minval / maxval of the FP32 values
      o.f64((double)*mm.second);
    }
    o.raw(data[mb], (size_t)(mq * npts) * sizeof(float));
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return CANARD_ERR_IO;
  const bool ok = std::fwrite(o.b.data(), 1, o.b.size(), f) == o.b.size();
  return (std::fclose(f) == 0 && ok) ? CANARD_OK : CANARD_ERR_IO;
}
