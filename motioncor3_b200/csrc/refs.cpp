// Gain / dark reference preparation on the host (done once per context, not
// on the hot path): the orientation post-processing of CLoadRefs::PostProcess
// (CLoadRefs.cpp:204-229) and the super-resolution augmentation of
// CLoadRefs::AugmentRefs (CLoadRefs.cpp:231-268).  Each step restates the
// index arithmetic of the reference's kernel so that the results are the
// same pixels.
#include <cstring>
#include <vector>

#include "../../include/mc3.h"

namespace {

// MrcUtil/G90Rotate2D.cu:14-33 and G90Rotate2D::Setup (:71-83): rotation by
// rot x 90 degrees about the image centre, nearest pixel, size swapped for odd
// factors.
void rotate90(const float* in, int nx, int ny, int rot, std::vector<float>& out, int* rx, int* ry) {
  const bool odd = (rot % 2) != 0;
  *rx = odd ? ny : nx;
  *ry = odd ? nx : ny;
  // cos / sin of 90*rot degrees rounded to -1, 0, 1 as the reference does
  const int c[4] = {1, 0, -1, 0}, s[4] = {0, 1, 0, -1};
  const int k = ((rot % 4) + 4) % 4;
  const int cs = c[k], sn = s[k];
  out.assign((size_t)(*rx) * (*ry), 0.0f);
  for (int y = 0; y < *ry; ++y)
    for (int x = 0; x < *rx; ++x) {
      const float fnx = x - (*rx - 1) * 0.5f;
      const float fny = y - (*ry - 1) * 0.5f;
      const float fx = fnx * cs + fny * sn;
      const float fy = -fnx * sn + fny * cs;
      const int ix = (int)(fx + (nx - 1) * 0.5f + 0.5f);
      const int iy = (int)(fy + (ny - 1) * 0.5f + 0.5f);
      out[(size_t)y * (*rx) + x] = in[(size_t)iy * nx + ix];
    }
}

// MrcUtil/GFlip2D.cu:9-40: 1 = upside down (rows y <-> ny-1-y), 2 = left-right.
void flip(std::vector<float>& img, int nx, int ny, int mode) {
  if (mode == 1) {
    for (int y = 0; y < ny / 2; ++y)
      for (int x = 0; x < nx; ++x)
        std::swap(img[(size_t)y * nx + x], img[(size_t)(ny - 1 - y) * nx + x]);
  } else if (mode == 2) {
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx / 2; ++x)
        std::swap(img[(size_t)y * nx + x], img[(size_t)y * nx + nx - 1 - x]);
  }
}

}  // namespace

extern "C" {

int mc3_ref_orient(const float* in, int nx, int ny, int rot, int flip_mode, int inverse,
                   float* out, int* out_nx, int* out_ny) {
  if (!in || !out || nx < 1 || ny < 1 || flip_mode < 0 || flip_mode > 2) return MC3_EINVAL;
  std::vector<float> img(in, in + (size_t)nx * ny);
  int w = nx, h = ny;
  if (rot != 0) {  // CLoadRefs::mRotate
    std::vector<float> r;
    rotate90(img.data(), nx, ny, rot, r, &w, &h);
    img.swap(r);
  }
  flip(img, w, h, flip_mode);  // CLoadRefs::mFlip
  if (inverse)                 // CLoadRefs::mInverse, MrcUtil/GInverse2D.cu:11-21
    for (float& v : img) v = (v == 0) ? 0.0f : 1.0f / v;
  std::memcpy(out, img.data(), sizeof(float) * img.size());
  if (out_nx) *out_nx = w;
  if (out_ny) *out_ny = h;
  return MC3_OK;
}

int mc3_ref_augment(const float* in, int nx, int ny, int fact, float* out) {
  if (!in || !out || nx < 1 || ny < 1 || fact < 1) return MC3_EINVAL;
  // MrcUtil/GAugmentRef.cu:10-23: each reference pixel covers fact x fact pixels
  const size_t ox = (size_t)nx * fact, oy = (size_t)ny * fact;
  for (size_t y = 0; y < oy; ++y)
    for (size_t x = 0; x < ox; ++x) out[y * ox + x] = in[(y / fact) * nx + x / fact];
  return MC3_OK;
}

}  // extern "C"
