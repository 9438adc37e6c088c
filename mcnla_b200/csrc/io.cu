// Dense file formats of the reference's io module, on the host: MatrixMarket
// "array" text files (include/mcnla/core/io/matrix_market/dense_load.hpp:70-251,
// dense_load_block.hpp, dense_save.hpp) and the MCNLA dense binary format
// (include/mcnla/core/io/binary/dense_load.hpp:70-141, dense_save.hpp, def.hpp;
// layout in doxygen/tutorial/io/binary.dox:17-30).  No device code: these read
// the inputs of a solve into host memory (then pinned memory and HBM) and write
// its results.
//
// MatrixMarket array: lines starting with '%' (the banner first), then the
// sizes ("m n" for a matrix, "m n l" for a 3-D collection of l m x n
// matrices), then one value per line in column-major order, matrix after
// matrix.  Values are written as the reference writes them: scientific with 16
// digits after the point (17 significant digits: a double round-trips).
//
// Binary: a 128-byte header (magic line, comment line, storage "DEN", value
// type "R8" / "R4", two reserved fields), then int64 ndim, int64 dims[ndim] and
// the values, contiguous along dims[0].
#include "common.cuh"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace mb {
namespace {

constexpr int kBinHeader = 32, kBinComment = 64, kBinField = 8;
constexpr const char* kBinMagic = "##MCNLABinaryFileFormat";

int io_error(const std::string& what) {
  set_last_message(what);
  return MCNLA_B200_ERR_IO;
}

bool read_file(const char* path, std::string* text) {
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  text->resize(size > 0 ? size_t(size) : 0);
  const size_t got = size > 0 ? std::fread(&(*text)[0], 1, size_t(size), f) : 0;
  std::fclose(f);
  return got == text->size();
}

// A parser over the text of a MatrixMarket array file.
struct MmText {
  std::string text;
  size_t pos = 0;
  int64_t dims[3] = {1, 1, 1};
  int ndim = 0;

  int open(const char* path) {
    if (!path) return MCNLA_B200_ERR_ARG;
    if (!read_file(path, &text)) return io_error(std::string("cannot read ") + path);
    // '%' lines: the banner (array format only) and comments
    while (pos < text.size() && text[pos] == '%') {
      const size_t eol = text.find('\n', pos);
      const std::string line = text.substr(pos, eol == std::string::npos ? std::string::npos : eol - pos);
      if (line.rfind("%%MatrixMarket", 0) == 0 && line.find("coordinate") != std::string::npos)
        return io_error(std::string(path) + ": a coordinate (sparse) MatrixMarket file, not a dense array");
      pos = eol == std::string::npos ? text.size() : eol + 1;
    }
    // the sizes: every integer on the first non-comment line
    const size_t eol = text.find('\n', pos);
    const size_t end = eol == std::string::npos ? text.size() : eol;
    while (pos < end && ndim < 4) {
      while (pos < end && (text[pos] == ' ' || text[pos] == '\t' || text[pos] == '\r')) ++pos;
      if (pos >= end) break;
      int64_t v = 0;
      const auto r = std::from_chars(text.data() + pos, text.data() + end, v);
      if (r.ec != std::errc() || v < 0) return io_error(std::string(path) + ": bad size line");
      if (ndim == 3) return io_error(std::string(path) + ": more than three sizes");
      dims[ndim++] = v;
      pos = size_t(r.ptr - text.data());
    }
    if (ndim < 2) return io_error(std::string(path) + ": the size line needs at least two sizes");
    pos = end;
    return MCNLA_B200_OK;
  }

  // the next value; false at the end of the text or on a malformed number
  bool next(double* v) {
    while (pos < text.size() && (text[pos] == ' ' || text[pos] == '\n' || text[pos] == '\t' || text[pos] == '\r'))
      ++pos;
    if (pos >= text.size()) return false;
    const char* b = text.data() + pos;
    if (*b == '+') ++b;   // from_chars takes no leading '+'
    const auto r = std::from_chars(b, text.data() + text.size(), *v);
    if (r.ec != std::errc()) return false;
    pos = size_t(r.ptr - text.data());
    return true;
  }
};

struct BinHeader {
  int64_t dims[3] = {1, 1, 1};
  int ndim = 0;
  char val_type[kBinField + 1] = {0};
  long data_offset = 0;
};

int read_bin_header(std::FILE* f, const char* path, BinHeader* h) {
  char head[kBinHeader + kBinComment + 4 * kBinField];
  if (std::fread(head, 1, sizeof(head), f) != sizeof(head)) return io_error(std::string(path) + ": short header");
  if (std::strncmp(head, kBinMagic, std::strlen(kBinMagic)) != 0)
    return io_error(std::string(path) + ": not an MCNLA binary file");
  const char* storage = head + kBinHeader + kBinComment;
  if (std::strncmp(storage, "DEN", 3) != 0)
    return io_error(std::string(path) + ": not a dense (DEN) binary file");
  std::memcpy(h->val_type, storage + kBinField, kBinField);
  for (int i = kBinField - 1; i >= 0 && (h->val_type[i] == ' ' || h->val_type[i] == 0); --i) h->val_type[i] = 0;
  int64_t nd = 0;
  if (std::fread(&nd, sizeof(nd), 1, f) != 1 || nd < 1 || nd > 3)
    return io_error(std::string(path) + ": bad number of dimensions");
  h->ndim = int(nd);
  for (int i = 0; i < h->ndim; ++i)
    if (std::fread(&h->dims[i], sizeof(int64_t), 1, f) != 1 || h->dims[i] < 0)
      return io_error(std::string(path) + ": bad dimensions");
  h->data_offset = std::ftell(f);
  return MCNLA_B200_OK;
}

}  // namespace
}  // namespace mb

extern "C" {

int mcnla_b200_mm_size(const char* path, int64_t* dims, int* ndim) {
  if (!dims || !ndim) return MCNLA_B200_ERR_ARG;
  mb::MmText t;
  MB_CHECK(t.open(path));
  for (int i = 0; i < 3; ++i) dims[i] = t.dims[i];
  *ndim = t.ndim;
  return MCNLA_B200_OK;
}

int mcnla_b200_mm_load(const char* path, int64_t row0, int64_t rows, int64_t col0, int64_t cols, double* out,
                       int64_t ldo, int layout) {
  if (!out || (layout != MCNLA_B200_ROW_MAJOR && layout != MCNLA_B200_COL_MAJOR)) return MCNLA_B200_ERR_ARG;
  mb::MmText t;
  MB_CHECK(t.open(path));
  const int64_t m = t.dims[0], n = t.dims[1], l = t.dims[2], ncols = n * l;
  if (row0 < 0 || rows < 0 || col0 < 0 || cols < 0 || row0 + rows > m || col0 + cols > ncols)
    return MCNLA_B200_ERR_SHAPE;
  if (ldo < (layout == MCNLA_B200_ROW_MAJOR ? cols : rows)) return MCNLA_B200_ERR_SHAPE;
  // values in file order: matrix k, column j, row i -> unfolded column k n + j
  double v = 0.0;
  for (int64_t k = 0; k < l; ++k)
    for (int64_t j = 0; j < n; ++j) {
      const int64_t jj = k * n + j - col0;
      const bool want_col = jj >= 0 && jj < cols;
      for (int64_t i = 0; i < m; ++i) {
        if (!t.next(&v)) return mb::io_error(std::string(path) + ": fewer values than the sizes announce");
        const int64_t ii = i - row0;
        if (want_col && ii >= 0 && ii < rows) {
          if (layout == MCNLA_B200_ROW_MAJOR) out[ii * ldo + jj] = v;
          else out[jj * ldo + ii] = v;
        }
      }
    }
  return MCNLA_B200_OK;
}

int mcnla_b200_mm_save(const char* path, const double* a, int64_t m, int64_t n, int64_t nmat, int64_t lda,
                       int layout, const char* comment) {
  if (!path || (!a && m * n * nmat > 0) || (layout != MCNLA_B200_ROW_MAJOR && layout != MCNLA_B200_COL_MAJOR))
    return MCNLA_B200_ERR_ARG;
  if (m < 0 || n < 0 || nmat < 1 || lda < (layout == MCNLA_B200_ROW_MAJOR ? n * nmat : m)) return MCNLA_B200_ERR_SHAPE;
  if (comment && std::strchr(comment, '\n')) return MCNLA_B200_ERR_ARG;
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return mb::io_error(std::string("cannot write ") + path);
  std::string buf;
  buf += nmat > 1 ? "%%MatrixMarket 3D array real general\n" : "%%MatrixMarket matrix array real general\n";
  if (comment) buf += std::string("% ") + comment + "\n";
  buf += std::to_string(m) + " " + std::to_string(n) + (nmat > 1 ? " " + std::to_string(nmat) : std::string()) + "\n";
  char num[64];
  bool ok = true;
  for (int64_t k = 0; k < nmat && ok; ++k)
    for (int64_t j = 0; j < n && ok; ++j) {
      for (int64_t i = 0; i < m; ++i) {
        const int64_t c = k * n + j;
        const double v = layout == MCNLA_B200_ROW_MAJOR ? a[i * lda + c] : a[c * lda + i];
        const auto r = std::to_chars(num, num + sizeof(num), v, std::chars_format::scientific, 16);
        buf.append(num, r.ptr);
        buf += '\n';
      }
      if (buf.size() > (size_t(1) << 24)) {
        ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
        buf.clear();
      }
    }
  if (ok) ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? MCNLA_B200_OK : mb::io_error(std::string("write failed: ") + path);
}

int mcnla_b200_binary_size(const char* path, int64_t* dims, int* ndim, char* val_type) {
  if (!path || !dims || !ndim) return MCNLA_B200_ERR_ARG;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return mb::io_error(std::string("cannot read ") + path);
  mb::BinHeader h;
  const int st = mb::read_bin_header(f, path, &h);
  std::fclose(f);
  if (st != MCNLA_B200_OK) return st;
  for (int i = 0; i < 3; ++i) dims[i] = h.dims[i];
  *ndim = h.ndim;
  if (val_type) std::memcpy(val_type, h.val_type, mb::kBinField + 1);
  return MCNLA_B200_OK;
}

int mcnla_b200_binary_load(const char* path, int64_t first, int64_t count, double* out) {
  if (!path || (!out && count > 0)) return MCNLA_B200_ERR_ARG;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return mb::io_error(std::string("cannot read ") + path);
  struct Close { std::FILE* f; ~Close() { std::fclose(f); } } close{f};
  mb::BinHeader h;
  MB_CHECK(mb::read_bin_header(f, path, &h));
  const bool r8 = std::strcmp(h.val_type, "R8") == 0, r4 = std::strcmp(h.val_type, "R4") == 0;
  if (!r8 && !r4) return mb::io_error(std::string(path) + ": value type " + h.val_type + " is not R8 or R4");
  // slices along the last dimension, each the product of the others
  int64_t slice = 1;
  for (int i = 0; i + 1 < h.ndim; ++i) slice *= h.dims[i];
  const int64_t nslices = h.dims[h.ndim - 1];
  if (first < 0 || count < 0 || first + count > nslices) return MCNLA_B200_ERR_SHAPE;
  const size_t esz = r8 ? 8 : 4;
  if (std::fseek(f, h.data_offset + long(first * slice * int64_t(esz)), SEEK_SET) != 0)
    return mb::io_error(std::string(path) + ": seek failed");
  const size_t total = size_t(count * slice);
  if (r8) {
    if (std::fread(out, 8, total, f) != total) return mb::io_error(std::string(path) + ": fewer values than the dims");
  } else {
    std::vector<float> tmp(size_t(1) << 20);
    for (size_t done = 0; done < total;) {
      const size_t chunk = std::min(tmp.size(), total - done);
      if (std::fread(tmp.data(), 4, chunk, f) != chunk)
        return mb::io_error(std::string(path) + ": fewer values than the dims");
      for (size_t i = 0; i < chunk; ++i) out[done + i] = double(tmp[i]);
      done += chunk;
    }
  }
  return MCNLA_B200_OK;
}

int mcnla_b200_binary_save(const char* path, const double* a, int ndim, const int64_t* dims, const char* comment) {
  if (!path || !dims || ndim < 1 || ndim > 3) return MCNLA_B200_ERR_ARG;
  int64_t total = 1;
  for (int i = 0; i < ndim; ++i) {
    if (dims[i] < 0) return MCNLA_B200_ERR_SHAPE;
    total *= dims[i];
  }
  if (!a && total > 0) return MCNLA_B200_ERR_ARG;
  const std::string c = comment ? comment : "";
  if (c.size() > size_t(mb::kBinComment - 3) || c.find('\n') != std::string::npos) return MCNLA_B200_ERR_ARG;
  char head[mb::kBinHeader + mb::kBinComment + 4 * mb::kBinField];
  std::memset(head, ' ', sizeof(head));
  std::memcpy(head, mb::kBinMagic, std::strlen(mb::kBinMagic));
  head[mb::kBinHeader - 1] = '\n';
  head[mb::kBinHeader] = '#';
  std::memcpy(head + mb::kBinHeader + 2, c.data(), c.size());
  head[mb::kBinHeader + mb::kBinComment - 1] = '\n';
  char* fields = head + mb::kBinHeader + mb::kBinComment;
  std::memcpy(fields, "DEN", 3);
  std::memcpy(fields + mb::kBinField, "R8", 2);
  head[sizeof(head) - 1] = '\n';
  std::FILE* f = std::fopen(path, "wb");
  if (!f) return mb::io_error(std::string("cannot write ") + path);
  const int64_t nd = ndim;
  bool ok = std::fwrite(head, 1, sizeof(head), f) == sizeof(head);
  ok = ok && std::fwrite(&nd, sizeof(nd), 1, f) == 1;
  ok = ok && std::fwrite(dims, sizeof(int64_t), size_t(ndim), f) == size_t(ndim);
  ok = ok && (total == 0 || std::fwrite(a, 8, size_t(total), f) == size_t(total));
  ok = (std::fclose(f) == 0) && ok;
  return ok ? MCNLA_B200_OK : mb::io_error(std::string("write failed: ") + path);
}

}  // extern "C"
