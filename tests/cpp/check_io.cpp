// Round trips of the C++ file API (mcnla_b200::io over the C ABI); host only.
// Usage: check_io <scratch dir>.  Prints "OK" and returns 0 when every check holds.
#include <mcnla_b200/isvd.hpp>

#include <cmath>
#include <cstdio>
#include <string>

using mcnla_b200::io::HostMatrix;
namespace io = mcnla_b200::io;

static int failures = 0;
static void expect(bool ok, const char* what) {
  if (!ok) {
    std::printf("FAILED: %s\n", what);
    ++failures;
  }
}

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  const std::string dir = argv[1];
  HostMatrix a;
  a.nrow = 7;
  a.ncol = 12;
  a.layout = MCNLA_B200_ROW_MAJOR;
  for (int64_t i = 0; i < a.nrow * a.ncol; ++i) a.val.push_back(std::sin(double(i + 1)) * std::pow(10.0, double(i % 9) - 4));
  const std::string mtx = dir + "/a.mtx", bin = dir + "/a.bin", col = dir + "/c.mtx";
  io::saveMatrixMarket(a, mtx.c_str(), 1, "check_io");
  const std::vector<int64_t> d = io::loadMatrixMarketSize(mtx.c_str());
  expect(d[0] == 7 && d[1] == 12 && d[2] == 1, "size");
  const HostMatrix b = io::loadMatrixMarket(mtx.c_str());
  expect(b.val == a.val, "matrix market round trip");
  const HostMatrix rb = io::loadMatrixMarketRowBlock(mtx.c_str(), 2, 3);
  bool ok = rb.nrow == 3 && rb.ncol == 12;
  for (int64_t i = 0; ok && i < 3; ++i)
    for (int64_t j = 0; j < 12; ++j) ok = ok && rb.val[size_t(i * 12 + j)] == a.val[size_t((i + 2) * 12 + j)];
  expect(ok, "row block");
  const HostMatrix cb = io::loadMatrixMarketColBlock(mtx.c_str(), 5, 4);
  ok = cb.nrow == 7 && cb.ncol == 4 && cb.layout == MCNLA_B200_COL_MAJOR;
  for (int64_t j = 0; ok && j < 4; ++j)
    for (int64_t i = 0; i < 7; ++i) ok = ok && cb.val[size_t(j * 7 + i)] == a.val[size_t(i * 12 + j + 5)];
  expect(ok, "column block");
  // a 3-D collection of 3 matrices of 7 x 4
  io::saveMatrixMarket(a, col.c_str(), 3);
  const std::vector<int64_t> dc = io::loadMatrixMarketSize(col.c_str());
  expect(dc[0] == 7 && dc[1] == 4 && dc[2] == 3, "collection size");
  expect(io::loadMatrixMarket(col.c_str()).val == a.val, "collection round trip");
  io::saveBinary(a, bin.c_str(), "check_io");
  const HostMatrix c = io::loadBinary(bin.c_str());
  expect(c.nrow == 7 && c.ncol == 12 && c.val == a.val, "binary round trip");
  try {
    io::loadMatrixMarket((dir + "/missing.mtx").c_str());
    expect(false, "missing file throws");
  } catch (const mcnla_b200::Error& e) {
    expect(e.status() == MCNLA_B200_ERR_IO, "missing file status");
  }
  if (failures == 0) std::printf("OK\n");
  return failures == 0 ? 0 : 1;
}
