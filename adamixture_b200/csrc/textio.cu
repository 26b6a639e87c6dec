// Host-side writer of the ADMIXTURE-compatible .Q / .P text files: one row per line, values
// separated by single spaces -- byte for byte what the reference's np.savetxt(path, X,
// delimiter=' ') writes: "%.18e" for the main command (adamixture/src/utils.py:252-273) and
// "%.6f" for the projection and supervised commands (adamixture/project_entry.py:289,
// adamixture/supervised_entry.py:386-389). Rows are formatted by several threads into
// per-block buffers (C printf is correctly rounded from the exact binary value, as Python's
// float formatting is) and written in order with one fwrite each.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace {

// decimals < 0: "%.18e"; otherwise "%.<decimals>f"
void format_rows(const double* X, int64_t r0, int64_t r1, int64_t cols, int decimals, std::string& out) {
  // "%.Nf" of a double needs at most 309 integer digits + sign + point + N decimals
  std::vector<char> buf((size_t)(decimals < 0 ? 40 : 320 + decimals));
  out.clear();
  out.reserve((size_t)(r1 - r0) * (size_t)cols * (decimals < 0 ? 25 : 4 + decimals));
  for (int64_t r = r0; r < r1; ++r) {
    for (int64_t c = 0; c < cols; ++c) {
      const double v = X[r * cols + c];
      const int n = decimals < 0 ? snprintf(buf.data(), buf.size(), "%.18e", v)
                                 : snprintf(buf.data(), buf.size(), "%.*f", decimals, v);
      out.append(buf.data(), (size_t)n);
      out.push_back(c + 1 < cols ? ' ' : '\n');
    }
  }
}

int write_matrix(const char* fn, const char* path, const double* X, int64_t rows, int64_t cols,
                 int decimals, int threads) {
  if (!path || (!X && rows * cols > 0) || rows < 0 || cols < 1 || decimals > 60) {
    adx_set_message((std::string(fn) + ": bad argument").c_str());
    return ADX_ERR_ARG;
  }
  FILE* f = fopen(path, "wb");
  if (!f) {
    adx_set_message((std::string(fn) + ": cannot open the output file").c_str());
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
      pool.emplace_back(format_rows, X, b * block, std::min(rows, (b + 1) * block), cols, decimals,
                        std::ref(bufs[(size_t)(b - b0)]));
    for (auto& t : pool) t.join();
    for (int64_t b = b0; b < b1; ++b) {
      const std::string& s = bufs[(size_t)(b - b0)];
      if (fwrite(s.data(), 1, s.size(), f) != s.size()) {
        adx_set_message((std::string(fn) + ": write failed").c_str());
        rc = ADX_ERR_ARG;
        break;
      }
    }
  }
  if (fclose(f) != 0 && rc == ADX_OK) {
    adx_set_message((std::string(fn) + ": close failed").c_str());
    rc = ADX_ERR_ARG;
  }
  return rc;
}

}  // namespace

extern "C" int adx_write_text_matrix(const char* path, const double* X, int64_t rows, int64_t cols, int threads) {
  return write_matrix("adx_write_text_matrix", path, X, rows, cols, -1, threads);
}

extern "C" int adx_write_text_matrix_fixed(const char* path, const double* X, int64_t rows, int64_t cols,
                                           int decimals, int threads) {
  if (decimals < 0) {
    adx_set_message("adx_write_text_matrix_fixed: decimals must be >= 0");
    return ADX_ERR_ARG;
  }
  return write_matrix("adx_write_text_matrix_fixed", path, X, rows, cols, decimals, threads);
}
