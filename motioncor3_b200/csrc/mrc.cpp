// Minimal MRC reader/writer (see mrc.h).
#include "mrc.h"

#include <cstdio>
#include <cstring>

namespace mc3 {
namespace mrc {

namespace {
uint32_t bswap32(uint32_t v) {
  return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}
uint16_t bswap16(uint16_t v) { return (uint16_t)((v >> 8) | (v << 8)); }
bool valid_mode(int m) { return m == 0 || m == 1 || m == 2 || m == 5 || m == 6 || m == 101; }
}  // namespace

int bytes_per_pixel(int mode) {
  switch (mode) {
    case 0: case 5: return 1;
    case 1: case 6: return 2;
    case 2: return 4;
    default: return 0;
  }
}

long long frame_bytes(int mode, int nx, int ny) {
  if (mode == 101) return (long long)((nx + 1) / 2) * ny;  // C4BitImage::GetImgBytes
  return (long long)nx * ny * bytes_per_pixel(mode);
}

bool read_header(const std::string& path, Header* h) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  unsigned char buf[1024];
  const size_t n = std::fread(buf, 1, 1024, f);
  std::fclose(f);
  if (n != 1024) return false;
  int32_t w[24];
  std::memcpy(w, buf, sizeof(w));
  bool sw = false;
  if (!valid_mode(w[3])) {
    int32_t m = (int32_t)bswap32((uint32_t)w[3]);
    if (!valid_mode(m)) return false;
    sw = true;
  }
  auto get = [&](int i) { return sw ? (int32_t)bswap32((uint32_t)w[i]) : w[i]; };
  h->nx = get(0);
  h->ny = get(1);
  h->nz = get(2);
  h->mode = get(3);
  h->nsymbt = get(23);
  h->swapped = sw;
  float xl, yl, zl;
  int32_t t[3] = {get(10), get(11), get(12)};
  std::memcpy(&xl, &t[0], 4);
  std::memcpy(&yl, &t[1], 4);
  std::memcpy(&zl, &t[2], 4);
  const int mx = get(7), my = get(8), mz = get(9);
  h->pix[0] = mx > 0 ? xl / mx : 0.f;
  h->pix[1] = my > 0 ? yl / my : 0.f;
  h->pix[2] = mz > 0 ? zl / mz : 0.f;
  return h->nx > 0 && h->ny > 0 && h->nz > 0 && h->nsymbt >= 0;
}

bool read_frames(const std::string& path, const Header& h, int z0, int nz, void* dst) {
  const int bpp = bytes_per_pixel(h.mode);
  const long long frame = frame_bytes(h.mode, h.nx, h.ny);
  if (!frame || z0 < 0 || z0 + nz > h.nz) return false;
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  const long long off = 1024LL + h.nsymbt + frame * z0;
  bool ok = fseeko(f, (off_t)off, SEEK_SET) == 0;
  if (ok) ok = std::fread(dst, 1, (size_t)(frame * nz), f) == (size_t)(frame * nz);
  std::fclose(f);
  if (ok && h.swapped && bpp > 1) {
    const long long n = (long long)h.nx * h.ny * nz;
    if (bpp == 2) {
      uint16_t* p = (uint16_t*)dst;
      for (long long i = 0; i < n; ++i) p[i] = bswap16(p[i]);
    } else {
      uint32_t* p = (uint32_t*)dst;
      for (long long i = 0; i < n; ++i) p[i] = bswap32(p[i]);
    }
  }
  return ok;
}

bool read_image_float(const std::string& path, std::vector<float>* img, int* nx, int* ny) {
  Header h;
  if (!read_header(path, &h)) return false;
  const int bpp = bytes_per_pixel(h.mode);
  if (!bpp) return false;  // images (gain) in packed modes are not read
  std::vector<unsigned char> raw((size_t)h.nx * h.ny * bpp);
  if (!read_frames(path, h, 0, 1, raw.data())) return false;
  img->resize((size_t)h.nx * h.ny);
  for (size_t i = 0; i < img->size(); ++i) {
    switch (h.mode) {
      case 0: case 5: (*img)[i] = raw[i]; break;
      case 1: (*img)[i] = ((const int16_t*)raw.data())[i]; break;
      case 2: (*img)[i] = ((const float*)raw.data())[i]; break;
      case 6: (*img)[i] = ((const uint16_t*)raw.data())[i]; break;
    }
  }
  *nx = h.nx;
  *ny = h.ny;
  return true;
}

// Header of a single float image as the reference's CSaveMrc writes it
// (CSaveMainHeader::mSetDefault + SetImgSize(size, 1, 1, pix) +
// SetExtHeader(0, 0, 0) + SetMinMaxMean).
bool write_float_image(const std::string& path, const float* img, int nx, int ny, float pix,
                       float amin, float amax, float amean) {
  return write_float_stack(path, img, nx, ny, 1, pix, amin, amax, amean, 0);
}

bool write_float_stack(const std::string& path, const float* img, int nx, int ny, int nz,
                       float pix, float amin, float amax, float amean, int ext_floats) {
  unsigned char hd[1024];
  std::memset(hd, 0, sizeof(hd));
  auto put_i = [&](int off, int32_t v) { std::memcpy(hd + off, &v, 4); };
  auto put_f = [&](int off, float v) { std::memcpy(hd + off, &v, 4); };
  auto put_s = [&](int off, int16_t v) { std::memcpy(hd + off, &v, 2); };
  put_i(0, nx);
  put_i(4, ny);
  put_i(8, nz);
  put_i(12, 2);
  put_i(16, 0);
  put_i(20, 0);
  put_i(24, 0);
  put_i(28, nx);
  put_i(32, ny);
  put_i(36, nz);
  put_f(40, nx * pix);
  put_f(44, ny * pix);
  put_f(48, nz * pix);
  put_f(52, 90.f);
  put_f(56, 90.f);
  put_f(60, 90.f);
  put_i(64, 1);
  put_i(68, 2);
  put_i(72, 3);
  put_f(76, amin);
  put_f(80, amax);
  put_f(84, amean);
  put_i(88, 0);
  const int nsymbt = ext_floats * 4 * nz;
  put_i(92, nsymbt);
  put_s(96, -16224);
  std::memcpy(hd + 104, "AGAR", 5);
  put_i(108, 2014 * 10);
  put_s(128, 0);
  put_s(130, (int16_t)ext_floats);
  put_s(132, 1);
  put_s(160, 5);
  put_f(184, 90.f);
  put_f(188, 90.f);
  put_f(192, 90.f);
  std::memcpy(hd + 208, "MAP", 4);
  hd[212] = 0x44;
  hd[213] = 0x44;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(hd, 1, 1024, f) == 1024;
  if (ok && nsymbt > 0) {
    // CSaveExtHeader: ext_floats per section, float 11 = pixel size
    // (LibSrc/Mrcfile/Header/CSaveExtHeader.cpp:28-46, 102-123)
    std::vector<float> ext((size_t)ext_floats * nz, 0.0f);
    if (ext_floats > 11)
      for (int z = 0; z < nz; ++z) ext[(size_t)z * ext_floats + 11] = pix;
    ok = std::fwrite(ext.data(), sizeof(float), ext.size(), f) == ext.size();
  }
  const size_t n = (size_t)nx * ny * nz;
  if (ok) ok = std::fwrite(img, sizeof(float), n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

}  // namespace mrc
}  // namespace mc3
