// Minimal PNG writer (RGBA8, filter 0, one zlib stream split into IDAT chunks) for the headless
// colour-map export.
#include <zlib.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "render.h"

namespace fip {

namespace {

void be32(std::vector<unsigned char>& v, uint32_t x) {
  v.push_back((unsigned char)(x >> 24));
  v.push_back((unsigned char)(x >> 16));
  v.push_back((unsigned char)(x >> 8));
  v.push_back((unsigned char)x);
}

bool chunk(FILE* f, const char* type, const unsigned char* data, size_t n) {
  std::vector<unsigned char> hdr;
  be32(hdr, (uint32_t)n);
  hdr.insert(hdr.end(), type, type + 4);
  uLong crc = crc32(0L, reinterpret_cast<const Bytef*>(type), 4);
  if (n) crc = crc32(crc, data, (uInt)n);
  std::vector<unsigned char> tail;
  be32(tail, (uint32_t)crc);
  return fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size() && (n == 0 || fwrite(data, 1, n, f) == n) &&
         fwrite(tail.data(), 1, 4, f) == 4;
}

}  // namespace

std::string write_png_rgba(const std::string& path, const unsigned char* rgba, int W, int H) {
  const size_t row = (size_t)W * 4;
  std::vector<unsigned char> raw((row + 1) * (size_t)H);
  for (int r = 0; r < H; ++r) {
    raw[(row + 1) * r] = 0;  // filter type None
    std::copy(rgba + row * r, rgba + row * (r + 1), raw.begin() + (row + 1) * r + 1);
  }
  uLongf zn = compressBound((uLong)raw.size());
  std::vector<unsigned char> z(zn);
  if (compress2(z.data(), &zn, raw.data(), (uLong)raw.size(), 6) != Z_OK) return "PNG: zlib compression failed";
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return "cannot open " + path;
  static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  std::vector<unsigned char> ihdr;
  be32(ihdr, (uint32_t)W);
  be32(ihdr, (uint32_t)H);
  ihdr.push_back(8);  // bit depth
  ihdr.push_back(6);  // colour type RGBA
  ihdr.push_back(0);
  ihdr.push_back(0);
  ihdr.push_back(0);
  bool ok = fwrite(sig, 1, 8, f) == 8 && chunk(f, "IHDR", ihdr.data(), ihdr.size());
  for (size_t off = 0; ok && off < zn; off += (1u << 20)) {
    const size_t n = std::min<size_t>(1u << 20, zn - off);
    ok = chunk(f, "IDAT", z.data() + off, n);
  }
  ok = ok && chunk(f, "IEND", nullptr, 0);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? std::string() : "write failed: " + path;
}

}  // namespace fip
