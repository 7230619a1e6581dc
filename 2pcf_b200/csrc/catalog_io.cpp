// catalog_io.cpp -- host file I/O of the driver around the pair sums:
//   * text catalogues (load_standard_shape_catalog, load_standard_kappa_map,
//     load_standard_lens_catalog, src/input_formats.f90:227-333), memory-
//     mapped and parsed by all host threads with std::from_chars (correctly
//     rounded to FP32, as a list-directed read into `real` is), the masks
//     applied while parsing and the rows scattered into columns in parallel;
//   * the per-bin result table the driver writes (src/main.f90:699-702);
//   * the binary marks stream (save_marks / load_survey_marks,
//     src/input_formats.f90:528-603).
// Plain C++ (no CUDA): these are file formats, not device work.

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "tpcf_b200.h"

namespace {

bool read_file(const char* path, std::string& buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  if (std::fseek(f, 0, SEEK_END) != 0) { std::fclose(f); return false; }
  const long sz = std::ftell(f);
  if (sz < 0) { std::fclose(f); return false; }
  std::rewind(f);
  buf.resize((size_t)sz);
  const size_t got = sz ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
  std::fclose(f);
  return got == (size_t)sz;
}

// A read-only view of a whole file: memory-mapped (no copy; the parser
// threads fault the pages in in parallel), or read into a buffer where
// mapping is not possible.
struct FileView {
  const char* b = "";
  size_t n = 0;
  void* map = nullptr;
  std::string buf;
  bool open(const char* path) {
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (::fstat(fd, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
      void* p = ::mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
      if (p != MAP_FAILED) {
        ::close(fd);
        map = p;
        n = (size_t)st.st_size;
        b = static_cast<const char*>(p);
        ::madvise(p, n, MADV_WILLNEED);
        return true;
      }
    }
    ::close(fd);
    if (!read_file(path, buf)) return false;
    b = buf.data();
    n = buf.size();
    return true;
  }
  ~FileView() {
    if (map) ::munmap(map, n);
  }
};

// [b, e) cut into nt pieces at line boundaries.
std::vector<std::pair<const char*, const char*>> split_lines(const char* b, const char* e, int nt) {
  std::vector<std::pair<const char*, const char*>> out(nt);
  const size_t n = (size_t)(e - b);
  const char* s = b;
  for (int t = 0; t < nt; ++t) {
    const char* cut = (t == nt - 1) ? e : b + (size_t)((double)n * (t + 1) / nt);
    if (cut < s) cut = s;
    if (cut < e && cut > b && cut[-1] != '\n') {
      const char* nl = static_cast<const char*>(std::memchr(cut, '\n', (size_t)(e - cut)));
      cut = nl ? nl + 1 : e;
    }
    out[t] = {s, cut};
    s = cut;
  }
  return out;
}

// Runs fn(t) on nt threads (the caller's thread takes t = 0).
template <class F>
void run_threads(int nt, F fn) {
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(fn, t);
  fn(0);
  for (auto& x : th) x.join();
}

inline bool is_sep(char c) { return c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\f' || c == '\v'; }

// A line holds data when its first non-blank character exists and is not '#'.
inline bool data_line(const char* p, const char* e) {
  while (p < e && is_sep(*p)) ++p;
  return p < e && *p != '#';
}

int64_t count_data_lines(const char* p, const char* e) {
  int64_t n = 0;
  while (p < e) {
    const char* le = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
    if (!le) le = e;
    if (data_line(p, le)) ++n;
    p = le + 1;
  }
  return n;
}

struct Chunk {
  const char* b;
  const char* e;
  std::vector<float> vals;  // row-major values of the kept rows of this chunk
  int64_t rows = 0;         // kept rows
  bool bad = false;
  int64_t bad_line = 0;     // 1-based line within the chunk
};

// Parses the data lines of [b, e), ncols values per line, and keeps the rows
// that pass the masks (keep_pos: value > 0, keep_nonneg: value >= 0; -1 = no
// mask) as row-major floats.
void parse_chunk(Chunk& c, int ncols, int keep_pos, int keep_nonneg) {
  const char* p = c.b;
  int64_t line = 0;
  float row[64];
  c.vals.reserve((size_t)(c.e - c.b) / 8);
  while (p < c.e) {
    const char* le = static_cast<const char*>(std::memchr(p, '\n', (size_t)(c.e - p)));
    if (!le) le = c.e;
    ++line;
    if (data_line(p, le)) {
      const char* q = p;
      int got = 0;
      while (q < le && got < ncols) {
        while (q < le && is_sep(*q)) ++q;
        if (q >= le) break;
        if (*q == '+') ++q;  // from_chars does not take a leading '+'
        float v;
        const auto r = std::from_chars(q, le, v);
        if (r.ec == std::errc::result_out_of_range) {
          // overflow / underflow: fall back to strtof's IEEE result
          std::string tok(q, (size_t)(std::find_if(q, le, [](char ch) { return is_sep(ch); }) - q));
          v = std::strtof(tok.c_str(), nullptr);
          q += tok.size();
        } else if (r.ec != std::errc()) {
          break;
        } else {
          q = r.ptr;
        }
        // Fortran exponent letters d/D are not accepted by from_chars
        if (q < le && !is_sep(*q)) break;
        row[got++] = v;
      }
      while (q < le && is_sep(*q)) ++q;
      if (got != ncols || q < le) {
        c.bad = true;
        c.bad_line = line;
        return;
      }
      const bool keep = (keep_pos < 0 || row[keep_pos] > 0.0f) &&        // w > 0 (input_formats.f90:250)
                        (keep_nonneg < 0 || row[keep_nonneg] >= 0.0f);  // z >= 0 (input_formats.f90:320)
      if (keep) {
        c.vals.insert(c.vals.end(), row, row + ncols);
        ++c.rows;
      }
    }
    p = le + 1;
  }
}

}  // namespace

extern "C" tpcf_status tpcf_read_table(const char* path, int32_t ncols, int32_t keep_pos_col,
                                       int32_t keep_nonneg_col, int32_t n_threads, float* cols, int64_t capacity,
                                       int64_t* n_rows) {
  if (!path || ncols < 1 || ncols > 64 || !n_rows || keep_pos_col >= ncols || keep_nonneg_col >= ncols)
    return TPCF_ERR_INVALID_ARG;
  FileView f;
  if (!f.open(path)) return TPCF_ERR_INVALID_ARG;
  const char* b = f.b;
  const char* e = b + f.n;
  int nt = n_threads > 0 ? n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
  nt = (int)std::min<int64_t>(nt, std::max<int64_t>(1, (int64_t)f.n / (1 << 16)));
  const auto parts = split_lines(b, e, nt);
  if (!cols) {  // upper bound: data lines
    std::vector<int64_t> cnt(nt, 0);
    run_threads(nt, [&](int t) { cnt[t] = count_data_lines(parts[t].first, parts[t].second); });
    int64_t n = 0;
    for (int64_t v : cnt) n += v;
    *n_rows = n;
    return TPCF_OK;
  }
  std::vector<Chunk> ch(nt);
  for (int t = 0; t < nt; ++t) {
    ch[t].b = parts[t].first;
    ch[t].e = parts[t].second;
  }
  run_threads(nt, [&](int t) { parse_chunk(ch[t], ncols, keep_pos_col, keep_nonneg_col); });
  std::vector<int64_t> off(nt + 1, 0);
  for (int t = 0; t < nt; ++t) {
    if (ch[t].bad) return TPCF_ERR_INVALID_ARG;
    off[t + 1] = off[t] + ch[t].rows;
  }
  if (off[nt] > capacity) return TPCF_ERR_OVERFLOW;
  // rows to columns, each chunk's rows at its offset (in file order)
  run_threads(nt, [&](int t) {
    const Chunk& c = ch[t];
    for (int k = 0; k < ncols; ++k) {
      float* dst = cols + (size_t)k * (size_t)capacity + (size_t)off[t];
      const float* src = c.vals.data() + k;
      for (int64_t r = 0; r < c.rows; ++r) dst[r] = src[(size_t)r * (size_t)ncols];
    }
  });
  *n_rows = off[nt];
  return TPCF_OK;
}

extern "C" tpcf_status tpcf_write_result_table(const char* path, int32_t n_bin, const float* theta,
                                               const float* g_t, const float* g_x, const float* weights,
                                               const int64_t* n_pairs, const float* mean_theta,
                                               int32_t to_degrees) {
  if (!path || n_bin < 1 || !theta || !g_t || !g_x || !weights || !n_pairs || !mean_theta) return TPCF_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "w");
  if (!f) return TPCF_ERR_INVALID_ARG;
  // rad2deg in FP32 as the driver applies it (src/utils.f90 rad2deg: rad*180/pi)
  const float pi = 3.141592653589793f;
  auto deg = [&](float v) { return to_degrees ? v * 180.0f / pi : v; };
  for (int i = 0; i < n_bin; ++i)
    std::fprintf(f, "%16.7E%16.7E%16.7E%16.7E%21lld%16.7E\n", (double)deg(theta[i]), (double)g_t[i], (double)g_x[i],
                 (double)weights[i], (long long)n_pairs[i], (double)deg(mean_theta[i]));
  const bool ok = std::fclose(f) == 0;
  return ok ? TPCF_OK : TPCF_ERR_INVALID_ARG;
}

// ------------------------------------------------------------ marks stream --
// Layout (save_marks, src/input_formats.f90:528-560): int64 header_size = 1024
// at byte 0, int64 n_field at byte 8, int64 header_size again at byte 1016;
// then per field int64 n, int64 n_bin, float32 x[n], y[n], w[n], then
// float32 xi_E[n][n_bin], xi_B[n][n_bin], K[n][n_bin].
namespace {
constexpr int64_t kHeader = 1024;

bool rd(FILE* f, void* p, size_t bytes) { return std::fread(p, 1, bytes, f) == bytes; }
bool wr(FILE* f, const void* p, size_t bytes) { return std::fwrite(p, 1, bytes, f) == bytes; }

bool read_header(FILE* f, int64_t& n_field) {
  int64_t h = 0, h2 = 0;
  if (!rd(f, &h, 8) || !rd(f, &n_field, 8) || h != kHeader) return false;
  if (std::fseek(f, kHeader - 8, SEEK_SET) != 0 || !rd(f, &h2, 8) || h2 != kHeader) return false;
  return n_field >= 0 && n_field <= 20;  // the reference's limit (input_formats.f90:586)
}
}  // namespace

extern "C" tpcf_status tpcf_marks_save(const char* path, int32_t n_field, const tpcf_marks_field* fields) {
  if (!path || n_field < 0 || n_field > 20 || (n_field > 0 && !fields)) return TPCF_ERR_INVALID_ARG;
  for (int i = 0; i < n_field; ++i) {
    const tpcf_marks_field& m = fields[i];
    if (m.n < 0 || m.n_bin < 1 || (m.n > 0 && (!m.x || !m.y || !m.w || !m.xi_E || !m.xi_B || !m.K)))
      return TPCF_ERR_INVALID_ARG;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return TPCF_ERR_INVALID_ARG;
  std::vector<char> head((size_t)kHeader, 0);
  const int64_t nf = n_field;
  std::memcpy(head.data(), &kHeader, 8);
  std::memcpy(head.data() + 8, &nf, 8);
  std::memcpy(head.data() + kHeader - 8, &kHeader, 8);
  bool ok = wr(f, head.data(), head.size());
  for (int i = 0; ok && i < n_field; ++i) {
    const tpcf_marks_field& m = fields[i];
    const size_t n = (size_t)m.n, nm = (size_t)m.n * (size_t)m.n_bin;
    ok = wr(f, &m.n, 8) && wr(f, &m.n_bin, 8) && wr(f, m.x, 4 * n) && wr(f, m.y, 4 * n) && wr(f, m.w, 4 * n) &&
         wr(f, m.xi_E, 4 * nm) && wr(f, m.xi_B, 4 * nm) && wr(f, m.K, 4 * nm);
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? TPCF_OK : TPCF_ERR_INVALID_ARG;
}

extern "C" tpcf_status tpcf_marks_info(const char* path, int32_t max_fields, int32_t* n_field, int64_t* n,
                                       int64_t* n_bin) {
  if (!path || !n_field || max_fields < 0 || (max_fields > 0 && (!n || !n_bin))) return TPCF_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return TPCF_ERR_INVALID_ARG;
  int64_t nf = 0;
  bool ok = read_header(f, nf);
  for (int64_t i = 0; ok && i < nf; ++i) {
    int64_t a = 0, b = 0;
    ok = rd(f, &a, 8) && rd(f, &b, 8) && a >= 0 && a <= 50000000 && b >= 1;  // input_formats.f90:594
    if (!ok) break;
    if (i < max_fields) { n[i] = a; n_bin[i] = b; }
    ok = std::fseek(f, (long)(4 * (3 * a + 3 * a * b)), SEEK_CUR) == 0;
  }
  std::fclose(f);
  if (!ok) return TPCF_ERR_INVALID_ARG;
  *n_field = (int32_t)nf;
  return TPCF_OK;
}

extern "C" tpcf_status tpcf_marks_load(const char* path, int32_t n_field, const tpcf_marks_field* fields) {
  if (!path || n_field < 0 || (n_field > 0 && !fields)) return TPCF_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "rb");
  if (!f) return TPCF_ERR_INVALID_ARG;
  int64_t nf = 0;
  bool ok = read_header(f, nf) && nf == n_field;
  for (int i = 0; ok && i < n_field; ++i) {
    const tpcf_marks_field& m = fields[i];
    int64_t a = 0, b = 0;
    ok = rd(f, &a, 8) && rd(f, &b, 8) && a == m.n && b == m.n_bin;
    if (!ok) break;
    if (a > 0 && (!m.x || !m.y || !m.w || !m.xi_E || !m.xi_B || !m.K)) { ok = false; break; }
    const size_t n = (size_t)a, nm = (size_t)a * (size_t)b;
    ok = rd(f, m.x, 4 * n) && rd(f, m.y, 4 * n) && rd(f, m.w, 4 * n) && rd(f, m.xi_E, 4 * nm) &&
         rd(f, m.xi_B, 4 * nm) && rd(f, m.K, 4 * nm);
  }
  std::fclose(f);
  return ok ? TPCF_OK : TPCF_ERR_INVALID_ARG;
}
