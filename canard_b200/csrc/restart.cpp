// Restart files in the reference's record format, the comparer of two
// restart files (contrib/dcanard.f90), and grid files in the reference's
// record format. Host code, no device work.
//
// A restart file holds one block (misc/restartZZZ.dat, src/mo_io.f90:115-116),
// written as a Fortran direct-access unformatted file of 40-byte records
// (5 IEEE doubles, src/mo_io.f90:233-271):
//   record 1: n, ndt, dt, dts, dte      (n and ndt stored as reals)
//   record 2: timo, 0, 0, 0, 0
//   record 3 + l: qa(l, 1..5) of stored point l = i + (lxi+1)(j + (let+1)k)
// Direct access carries no record markers, so record r starts at byte 40(r-1).
// One process per block writes the whole block (lpos = 0 and lio(j,k) =
// j(lxi+1) + k(let+1)(lxi+1), src/mo_canard_driver.f90:153-161).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "canard_gpu.h"

namespace {

constexpr int kRec = 5;  // doubles per record

struct File {
  FILE* f = nullptr;
  explicit File(const char* path, const char* mode) : f(path ? std::fopen(path, mode) : nullptr) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// read_restart_file's reads (src/mo_io.f90:184-229) into qa(0:npts-1, 5)
int read_file(const char* path, double* time6, double* qa, int64_t npts) {
  File in(path, "rb");
  if (!in.f) return CANARD_ERR_IO;
  if (std::fseek(in.f, 0, SEEK_END) != 0) return CANARD_ERR_IO;
  const long size = std::ftell(in.f);
  if (size != (long)(8 * kRec * (npts + 2))) return CANARD_ERR_IO;  // another block size
  std::rewind(in.f);
  double head[2 * kRec];
  if (std::fread(head, sizeof(double), 2 * kRec, in.f) != (size_t)(2 * kRec)) return CANARD_ERR_IO;
  if (time6) {
    for (int k = 0; k < 5; ++k) time6[k] = head[k];
    time6[5] = head[kRec];
  }
  if (qa) {
    std::vector<double> rec((size_t)kRec * 4096);
    for (int64_t l0 = 0; l0 < npts; l0 += 4096) {
      const int64_t m = std::min<int64_t>(4096, npts - l0);
      if (std::fread(rec.data(), sizeof(double), (size_t)(kRec * m), in.f) != (size_t)(kRec * m)) return CANARD_ERR_IO;
      for (int64_t l = 0; l < m; ++l)
        for (int c = 0; c < kRec; ++c) qa[(l0 + l) + c * npts] = rec[(size_t)(kRec * l + c)];
    }
  }
  return CANARD_OK;
}

// Fortran Ew.d output of one value (round to nearest, mantissa in [0.1, 1)),
// right-justified: " 0.1234567E+01" style.
std::string fortran_e(double v, int w, int d) {
  auto rjust = [w](std::string s) { return (int)s.size() < w ? std::string(w - s.size(), ' ') + s : s; };
  if (std::isnan(v)) return rjust("NaN");
  if (std::isinf(v)) return rjust(v < 0 ? "-Infinity" : "Infinity");
  char buf[64];
  int e = 0;
  std::string mant;
  if (v == 0) {
    mant = "0." + std::string(d, '0');
  } else {
    // the d significant digits of |v| as d.dddE+x, then shift the point one left
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, std::fabs(v));
    std::string s(buf);
    const size_t p = s.find('e');
    std::string digits = s.substr(0, 1) + s.substr(2, p - 2);
    e = std::stoi(s.substr(p + 1)) + 1;
    mant = "0." + digits;
  }
  // a three-digit exponent takes the place of the E
  if (std::abs(e) > 99)
    std::snprintf(buf, sizeof buf, "%s%s%c%03d", v < 0 ? "-" : "", mant.c_str(), e < 0 ? '-' : '+', std::abs(e));
  else
    std::snprintf(buf, sizeof buf, "%s%sE%c%02d", v < 0 ? "-" : "", mant.c_str(), e < 0 ? '-' : '+', std::abs(e));
  return rjust(buf);
}

}  // namespace

extern "C" {

int canard_restart_write_file(const char* path, const double* time6, const double* qa, int64_t npts) {
  if (!path || !time6 || !qa || npts < 1) return CANARD_ERR_ARG;
  File out(path, "wb");
  if (!out.f) return CANARD_ERR_IO;
  // write_restart_file (src/mo_io.f90:233-271): cha = (n, ndt, dt, dts, dte), dha = (timo, 0, 0, 0, 0)
  const double head[2 * kRec] = {time6[0], time6[1], time6[2], time6[3], time6[4], time6[5], 0.0, 0.0, 0.0, 0.0};
  if (std::fwrite(head, sizeof(double), 2 * kRec, out.f) != (size_t)(2 * kRec)) return CANARD_ERR_IO;
  std::vector<double> rec((size_t)kRec * 4096);
  for (int64_t l0 = 0; l0 < npts; l0 += 4096) {
    const int64_t m = std::min<int64_t>(4096, npts - l0);
    for (int64_t l = 0; l < m; ++l)
      for (int c = 0; c < kRec; ++c) rec[(size_t)(kRec * l + c)] = qa[(l0 + l) + c * npts];
    if (std::fwrite(rec.data(), sizeof(double), (size_t)(kRec * m), out.f) != (size_t)(kRec * m)) return CANARD_ERR_IO;
  }
  return std::fflush(out.f) == 0 ? CANARD_OK : CANARD_ERR_IO;
}

int canard_restart_read_file(const char* path, double* time6, double* qa, int64_t npts) {
  if (!path || npts < 1) return CANARD_ERR_ARG;
  return read_file(path, time6, qa, npts);
}

// Grid files (misc/gridZZZ.dat): a Fortran direct-access file read one
// 24-byte record (x, y, z) per stored point l = i + (lxi+1)(j + (let+1)k)
// (read_grid_parallel, src/mo_io.f90:151-180, one sub-domain per block) and
// written one record per k plane holding the plane's (x, y, z) triplets, i
// fastest (gridtoy / gridtoy_multi / gridaerofoil, src/mo_gridgen.f90:536-570):
// the same bytes, 3 doubles per point with no markers. xyz is ss(0:npts-1, 3).
int canard_grid_write_file(const char* path, const double* xyz, int64_t npts) {
  if (!path || !xyz || npts < 1) return CANARD_ERR_ARG;
  File out(path, "wb");
  if (!out.f) return CANARD_ERR_IO;
  std::vector<double> rec((size_t)3 * 4096);
  for (int64_t l0 = 0; l0 < npts; l0 += 4096) {
    const int64_t m = std::min<int64_t>(4096, npts - l0);
    for (int64_t l = 0; l < m; ++l)
      for (int c = 0; c < 3; ++c) rec[(size_t)(3 * l + c)] = xyz[(l0 + l) + c * npts];
    if (std::fwrite(rec.data(), sizeof(double), (size_t)(3 * m), out.f) != (size_t)(3 * m)) return CANARD_ERR_IO;
  }
  return std::fflush(out.f) == 0 ? CANARD_OK : CANARD_ERR_IO;
}

int canard_grid_read_file(const char* path, double* xyz, int64_t npts) {
  if (!path || !xyz || npts < 1) return CANARD_ERR_ARG;
  File in(path, "rb");
  if (!in.f) return CANARD_ERR_IO;
  if (std::fseek(in.f, 0, SEEK_END) != 0) return CANARD_ERR_IO;
  if (std::ftell(in.f) != (long)(24 * npts)) return CANARD_ERR_IO;  // another block size
  std::rewind(in.f);
  std::vector<double> rec((size_t)3 * 4096);
  for (int64_t l0 = 0; l0 < npts; l0 += 4096) {
    const int64_t m = std::min<int64_t>(4096, npts - l0);
    if (std::fread(rec.data(), sizeof(double), (size_t)(3 * m), in.f) != (size_t)(3 * m)) return CANARD_ERR_IO;
    for (int64_t l = 0; l < m; ++l)
      for (int c = 0; c < 3; ++c) xyz[(l0 + l) + c * npts] = rec[(size_t)(3 * l + c)];
  }
  return CANARD_OK;
}

int canard_restart_compare(const char* path1, const char* path2, int64_t npts, double wtol, const char* report_path,
                           int64_t* nreported) {
  if (!path1 || !path2 || npts < 1 || !(wtol >= 0)) return CANARD_ERR_ARG;
  std::vector<double> q1((size_t)5 * npts), q2((size_t)5 * npts);
  int rc = read_file(path1, nullptr, q1.data(), npts);
  if (rc == CANARD_OK) rc = read_file(path2, nullptr, q2.data(), npts);
  if (rc != CANARD_OK) return rc;
  File rep(report_path, "w");
  if (report_path && !rep.f) return CANARD_ERR_IO;
  int64_t n = 0;
  // contrib/dcanard.f90:114-124: variable j outer, point i inner; the
  // difference relative to the first file's value (no line where that is
  // 0/0, i.e. both values zero)
  for (int j = 1; j <= 5; ++j)
    for (int64_t i = 0; i < npts; ++i) {
      const double a = q1[(size_t)(i + (j - 1) * npts)], b = q2[(size_t)(i + (j - 1) * npts)];
      const double ad = std::fabs(a - b), rel = std::fabs((a - b) / a);
      if (rel > wtol) {
        ++n;
        if (rep.f)
          std::fprintf(rep.f, " i=%8lld j=%8d v1=%s v2=%s abs=%s rel=%s\n", (long long)i, j,
                       fortran_e(a, 15, 7).c_str(), fortran_e(b, 15, 7).c_str(), fortran_e(ad, 15, 7).c_str(),
                       fortran_e(rel, 15, 7).c_str());
      }
    }
  if (nreported) *nreported = n;
  return CANARD_OK;
}

}  // extern "C"
