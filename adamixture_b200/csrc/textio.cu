// Host-side writer of the ADMIXTURE-compatible .Q / .P text files: one row per line, values
// formatted "%.18e" and separated by single spaces -- byte for byte what the reference's
// np.savetxt(path, X, delimiter=' ') writes (adamixture/src/utils.py:252-273). Rows are
// formatted by several threads into per-block buffers (C printf's "%.18e" is correctly
// rounded, as Python's float formatting is) and written in order with one fwrite each.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace {

void format_rows(const double* X, int64_t r0, int64_t r1, int64_t cols, std::string& out) {
  char buf[40];
  out.clear();
  out.reserve((size_t)(r1 - r0) * (size_t)cols * 25);
  for (int64_t r = r0; r < r1; ++r) {
    for (int64_t c = 0; c < cols; ++c) {
      const int n = snprintf(buf, sizeof(buf), "%.18e", X[r * cols + c]);
      out.append(buf, (size_t)n);
      out.push_back(c + 1 < cols ? ' ' : '\n');
    }
  }
}

}  // namespace

extern "C" int adx_write_text_matrix(const char* path, const double* X, int64_t rows, int64_t cols, int threads) {
  if (!path || (!X && rows * cols > 0) || rows < 0 || cols < 1) {
    adx_set_message("adx_write_text_matrix: bad argument");
    return ADX_ERR_ARG;
  }
  FILE* f = fopen(path, "wb");
  if (!f) {
    adx_set_message("adx_write_text_matrix: cannot open the output file");
    return ADX_ERR_ARG;
  }
  const int64_t block = 4096;
  const int64_t n_blocks = (rows + block - 1) / block;
  int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = (int)std::min<int64_t>(nt, std::max<int64_t>(n_blocks, 1));
  int rc = ADX_OK;
  // rounds of nt blocks: format in parallel, write in order
  std::vector<std::string> bufs((size_t)nt);
  for (int64_t b0 = 0; b0 < n_blocks && rc == ADX_OK; b0 += nt) {
    const int64_t b1 = std::min(n_blocks, b0 + nt);
    std::vector<std::thread> pool;
    for (int64_t b = b0; b < b1; ++b)
      pool.emplace_back(format_rows, X, b * block, std::min(rows, (b + 1) * block), cols,
                        std::ref(bufs[(size_t)(b - b0)]));
    for (auto& t : pool) t.join();
    for (int64_t b = b0; b < b1; ++b) {
      const std::string& s = bufs[(size_t)(b - b0)];
      if (fwrite(s.data(), 1, s.size(), f) != s.size()) {
        adx_set_message("adx_write_text_matrix: write failed");
        rc = ADX_ERR_ARG;
        break;
      }
    }
  }
  if (fclose(f) != 0 && rc == ADX_OK) {
    adx_set_message("adx_write_text_matrix: close failed");
    rc = ADX_ERR_ARG;
  }
  return rc;
}
