// hr_output.cpp — binary output: float64 arrays as NumPy .npy files (format
// version 1.0, little-endian, C order). The binary replacement of the
// reference's text dumps: the two-surface solution (vel1 / vel2,
// 2S/main.cpp:258-270) and the extend-to-grid mid-plane slices
// (E2G/main.cpp:115-118, 297-300, 546, 921).
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/highreg_b200.h"

extern "C" int hr_write_npy(const char* path, const double* data, int ndim, const long long* shape) {
  if (!path || ndim < 1 || ndim > 8 || !shape) return HR_ERR_ARG;
  long long count = 1;
  for (int d = 0; d < ndim; d++) {
    if (shape[d] < 0) return HR_ERR_ARG;
    count *= shape[d];
  }
  if (count > 0 && !data) return HR_ERR_ARG;
  std::string dict = "{'descr': '<f8', 'fortran_order': False, 'shape': (";
  for (int d = 0; d < ndim; d++) {
    dict += std::to_string(shape[d]);
    if (ndim == 1 || d + 1 < ndim) dict += ",";
    if (d + 1 < ndim) dict += " ";
  }
  dict += "), }";
  // magic (6) + version (2) + header length (2) + dict + padding + '\n' is a multiple of 64
  const size_t pre = 10;
  size_t total = pre + dict.size() + 1;
  total = (total + 63) / 64 * 64;
  dict.append(total - pre - dict.size() - 1, ' ');
  dict += '\n';
  FILE* f = fopen(path, "wb");
  if (!f) return HR_ERR_ARG;
  const unsigned char head[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  const uint16_t hl = (uint16_t)dict.size();
  const unsigned char hlb[2] = {(unsigned char)(hl & 0xff), (unsigned char)(hl >> 8)};
  bool ok = fwrite(head, 1, 8, f) == 8 && fwrite(hlb, 1, 2, f) == 2 &&
            fwrite(dict.data(), 1, dict.size(), f) == dict.size() &&
            (count == 0 || fwrite(data, sizeof(double), (size_t)count, f) == (size_t)count);
  ok = (fclose(f) == 0) && ok;
  return ok ? HR_OK : HR_ERR_ARG;
}
