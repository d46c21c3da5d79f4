// Minimal MRC (2014) reader/writer for the movie, gain and sum files.
// Header layout and the writer's default fields follow
// LibSrc/Mrcfile/Include/CMrcFileInc.h:52-122 and
// LibSrc/Mrcfile/Header/CSaveMainHeader.cpp:180-260.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mc3 {
namespace mrc {

struct Header {
  int nx = 0, ny = 0, nz = 0, mode = 0;
  int nsymbt = 0;
  float pix[3] = {0, 0, 0};
  bool swapped = false;
};

int bytes_per_pixel(int mode);  // 0 when unsupported (and for packed mode 101)
long long frame_bytes(int mode, int nx, int ny);  // 0 when unsupported
// Reads the header; returns false on failure.
bool read_header(const std::string& path, Header* h);
// Reads frames [z0, z0+nz) as raw bytes in the file's mode (byte-swapped
// to host order when needed).
bool read_frames(const std::string& path, const Header& h, int z0, int nz, void* dst);
// Reads a whole single-image file (gain) converted to float.
bool read_image_float(const std::string& path, std::vector<float>* img, int* nx, int* ny);
// Writes a single float image (mode 2) with min/max/mean in the header.
bool write_float_image(const std::string& path, const float* img, int nx, int ny, float pix,
                       float amin, float amax, float amean);
// Writes nz float images (mode 2) with `ext_floats` extended-header floats
// per section holding the pixel size at float 11 (the aligned stack of
// CSaveSerialCryoEM::mSaveStack, CSaveSerialCryoEM.cpp:146-211).
bool write_float_stack(const std::string& path, const float* img, int nx, int ny, int nz,
                       float pix, float amin, float amax, float amean, int ext_floats);

}  // namespace mrc
}  // namespace mc3
