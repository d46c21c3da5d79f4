// Host-side shift bookkeeping of the alignment path, in FP32 with the same
// operation order as the reference's host code, so that its discontinuous
// steps (0.01 px truncation, the 5/10 px spike tests, bad-patch tests)
// take the same branches.
#pragma once
#include <vector>

namespace mc3 {
namespace host {

// Rendered (integrated) frames of a movie (DataUtil/CFmIntParam.cpp): raw
// frames start[i] .. start[i]+size[i]-1 are summed into frame i, which
// carries dose[i] and the accumulated dose acc[i]; its time stamp is
// center[i] = start + (size - 1)/2 in raw frames.
struct FmInt {
  std::vector<int> start, size;
  std::vector<float> dose, acc, center;
  int count() const { return (int)start.size(); }
  // CFmIntParam::mSetup (:118-136): one raw frame per rendered frame.
  void plain(int n_raw, float fm_dose);
  // CFmIntParam::mCalcIntFms (:138-229) from frame-integration entries
  // (raw frames, raw frames per rendered frame, raw-frame dose).
  void integrate(const std::vector<int>& group_size, const std::vector<int>& int_size,
                 float raw_dose, int n_raw);
  void centers();  // CFmIntParam::mCalcIntFmCenters (:276-283)
  // -Throw / -Trunc on rendered frames (CFmIntParam::mThrowIntFrames,
  // :231-256): the first t0 and last t1 are dropped, the others keep their
  // raw-frame starts and accumulated doses; ignored (false) when 5 or fewer
  // frames would be left.
  bool drop(int t0, int t1);
};

// CReadFmIntFile::DoIt (DataUtil/CReadFmIntFile.cpp:104-170): the entries
// of a frame-integration file, with the reference's parsing (a line that
// does not scan repeats the previous entry in the three-column form; mixed
// doses discard the file).  Returns false when the file cannot be opened.
bool read_fmint_file(const char* path, float cli_fm_dose, std::vector<int>& group_size,
                     std::vector<int>& int_size, std::vector<float>& dose);

// Frame groups of -Group binZ (DataUtil/CFmGroupParam.cpp:26-78): runs of
// rendered frames holding binZ x (smallest rendered-frame size) raw frames;
// group centres are the mean time stamps of their frames.
struct FrameGroups {
  int binZ = 1;
  std::vector<int> start, size;
  std::vector<float> center;
  std::vector<float> fm_center;  // time stamp of every rendered frame
  void setup(int n_frames, int bin_z);  // one raw frame per rendered frame
  void setup(const FmInt& fi, int bin_z);
  int count() const { return (int)start.size(); }
};

// Per-frame shift pairs stored as [x0..xn-1][y0..yn-1] (Align/CStackShift.cpp).
struct StackShift {
  int n = 0;
  std::vector<float> v;
  void setup(int n_frames) { n = n_frames; v.assign(2 * (size_t)n_frames, 0.0f); }
  float& x(int i) { return v[i]; }
  float& y(int i) { return v[n + i]; }
  float x(int i) const { return v[i]; }
  float y(int i) const { return v[n + i]; }
  void add(const StackShift& d);
  void multiply(float fx, float fy);
  void truncate_decimal();          // CStackShift::TruncateDecimal
  void make_relative(int ref);      // CStackShift::MakeRelative
  void smooth(float w);             // CStackShift::Smooth
  void remove_spikes();             // CStackShift::RemoveSpikes(false)
};

// CInterpolateShift::DoIt: group shifts -> frame shifts.
StackShift interpolate(const StackShift& grp, const FrameGroups& g, int n_frames, bool nearest);

// Util_LinEqs::DoIt (Gauss-Jordan, full pivoting).  Returns false when
// singular.
bool lin_eqs(float* coeff, float* vals, int dim);
// CRemoveSpikes1D::DoIt(pfX, pfY, bSingle=false)
void remove_spikes(float* sx, float* sy, int n);
// CPeak2D::DoIt on a float window.
void peak2d(const float* win, int sx, int sy, float* shift);

// Iteration driver state of CIterativeAlign::mAlignStack for one stack.
struct IterState {
  StackShift tmp, grp, total;
  float bfactor = 0;
  float max_err = 0;
  int iterations = 0;
  bool done = false;
  std::vector<float> errors;
  void start(int n_frames, int n_groups, float bf);
  // start() from a first iterate of the per-frame shifts init[n_frames][2]:
  // tmp = init, each group's total = the mean of its frames' shifts.
  void start_from(const float* init, const FrameGroups& g, int n_frames, float bf);
  // Consumes the group shifts measured in iteration `it`; returns true when
  // the stack has finished iterating.
  bool step(const float* grp_xy, const FrameGroups& g, int it, int max_iter, float tol);
  // Final trajectory (linear interpolation, spike removal, two smoothings).
  StackShift finish(const FrameGroups& g, int n_frames) const;
};

// Patch bookkeeping (Align/CPatchShifts.cpp).  shifts: [N][P][2].
void patch_make_relative(std::vector<float>& shifts, int n_frames, int n_patches);
void patch_detect_bads(const float* shifts, const float* centers, int n_frames, int n_patches,
                       int W, int H, unsigned char* bad);

// CDetectFeatures + CPatchCenters: patch start pixels in the alignment
// (xcf) image from the normalised 128x128 feature map and its moments.
void patch_starts(const float* map, int bx, int by, float mean, float m2, int px, int py,
                  int xcf_x, int xcf_y, int pat_x, int pat_y, std::vector<int>& starts);

// Patch starts in the alignment image for given full-frame patch centres
// (mc3_set_patch_centers): each centre divided by the bin and rounded to the
// nearest pixel, minus half the patch (the inverse of the centre the engine
// reports, start + size/2 times the bin), kept inside the image.
void patch_starts_from_centers(const float* centers, int n_patches, float bin_x, float bin_y,
                               int xcf_x, int xcf_y, int pat_x, int pat_y,
                               std::vector<int>& starts);

// GStretch::Setup (Correct/GStretch.cu:53-72) with the stretch and axis of
// CAlignParam::GetMagStretch (Align/CAlignParam.cpp:55-72): the inverse of
// the stretch matrix along -angle, as three floats.  Returns false when the
// stretch is below 1e-5 (no correction).
bool mag_matrix(const float mag[3], float m[3]);

// Ring template of the defect detector (BadPixel/CTemplate.cpp:20-57).
void defect_template(int ms, float* tpl);

// kV factor of the critical-dose curve (Correct/GWeightFrame.cu:101-109).
float kv_factor(int kv);

}  // namespace host
}  // namespace mc3
