// MotionCor3-compatible command line over libmc3 (single-movie MRC mode).
//
// Tags, defaults and value parsing follow CInput::Parse (CInput.cpp:425-677)
// and Util::CParseArgs (Util/CParseArgs.cpp); output naming follows
// sGenOutputName (CSaveSerialCryoEM.cpp:13-31) and CAlnSums::Setup
// (DataUtil/CAlnSums.cpp:18-43); log files follow CFullAlign::LogShift
// (Align/CFullAlign.cpp:173-194) and CPatchShifts::Log* (Align/CPatchShifts.cpp:155-249);
// exit codes follow ERetCode (CMotionCor3.cpp:20-28).  Tags outside the
// implemented path are accepted and ignored with a warning.
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <strings.h>
#include <vector>

#include "../../include/mc3.h"
#include "mrc.h"

namespace {

enum RetCode { eSuccess = 0, eNoFreeGPUs = 1, eInputOutputSame = 2, eFailLoad = 3, eFailSave = 4,
               eNoValidGPUs = 5, eFailProcess = 6 };

struct Args {
  int argc;
  char** argv;
  // CParseArgs::FindVals: values follow the tag until a token "-<alpha>...".
  bool find(const char* tag, int* first, int* count) const {
    *first = -1;
    *count = 0;
    for (int i = 1; i < argc; ++i)
      if (strcasecmp(argv[i], tag) == 0) {
        *first = i + 1;
        break;
      }
    if (*first < 0) return false;
    for (int i = *first; i < argc; ++i) {
      const char* a = argv[i];
      if (a[0] == '-' && std::strlen(a) >= 2 && std::isalpha((unsigned char)a[1])) break;
      char buf[256];
      std::snprintf(buf, sizeof(buf), "%s", a);
      for (char* t = std::strtok(buf, ", "); t; t = std::strtok(nullptr, ", ")) *count += 1;
    }
    return *count > 0;
  }
  std::string str(const char* tag) const {
    int f, n;
    if (!find(tag, &f, &n) || f >= argc) return std::string();
    return argv[f];
  }
  int ints(const char* tag, int* v, int maxn) const {
    int f, n;
    if (!find(tag, &f, &n)) return 0;
    if (n > maxn) n = maxn;
    int c = 0;
    for (int i = 0; i < n && f + i < argc && c < n; ++i) {
      char buf[256];
      std::snprintf(buf, sizeof(buf), "%s", argv[f + i]);
      for (char* t = std::strtok(buf, ", "); t && c < n; t = std::strtok(nullptr, ", "))
        std::sscanf(t, "%d", v + c++);
    }
    return c;
  }
  int floats(const char* tag, float* v, int maxn) const {
    int f, n;
    if (!find(tag, &f, &n)) return 0;
    if (n > maxn) n = maxn;
    int c = 0;
    for (int i = 0; i < n && f + i < argc; ++i) std::sscanf(argv[f + i], "%f", v + c++);
    return c;
  }
};

std::string out_name(const std::string& out_mrc, const char* suffix, const char* ext) {
  std::string s = out_mrc;
  auto cut = [&](const char* pat) {
    const char* p = strcasestr(s.c_str(), pat);
    if (p) s.resize(p - s.c_str());
  };
  cut(".mrc");
  cut(".st");
  return s + suffix + ext;
}

std::string log_stem(const std::string& log_dir, const std::string& in_file) {
  if (log_dir.empty()) return std::string();
  const char* base = std::strrchr(in_file.c_str(), '/');
  base = base ? base + 1 : in_file.c_str();
  std::string s = log_dir + base;
  // CAlignMain::mCreateLogFile (Align/CAlignMain.cpp:77-107)
  for (const char* ext : {".mrc", ".tif", ".eer"}) {
    const char* p = strcasestr(s.c_str(), ext);
    if (p) {
      s.resize(p - s.c_str());
      return s;
    }
  }
  return std::string();
}

void stats(const float* img, size_t n, float* mn, float* mx, float* mean) {
  double s = 0;
  float a = img[0], b = img[0];
  for (size_t i = 0; i < n; ++i) {
    a = img[i] < a ? img[i] : a;
    b = img[i] > b ? img[i] : b;
    s += img[i];
  }
  *mn = a;
  *mx = b;
  *mean = (float)(s / n);
}

// Page-locked host buffer (mc3_host_alloc) so the movie and the sums cross
// the host link at full speed; ordinary memory when pinning is refused (the
// copies are then slower, the results the same).
struct HostBuf {
  void* p = nullptr;
  bool pinned = false;
  std::vector<unsigned char> plain;
  explicit HostBuf(size_t n) {
    if (mc3_host_alloc(n, &p) == MC3_OK) {
      pinned = true;
    } else {
      plain.resize(n);
      p = plain.data();
    }
  }
  ~HostBuf() {
    if (pinned) mc3_host_free(p);
  }
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  template <class T>
  T* as() { return static_cast<T*>(p); }
};

// Align/CLoadAlign.cpp:52-250: an -InAln alignment file, as -OutAln (and
// the reference) write it.  Keywords are searched in order ("setting",
// "stackSize", "patches", "throw"); the first nz lines that scan as
// "%d %f %f" are the full-frame shifts; in patch mode every later line
// that scans as "%d %f %f %f %f" is (frame, centre x, y, shift x, y), nz of
// them per patch.
struct LoadedAln {
  int stk[4] = {0, 0, 0, 0};
  int patches[3] = {0, 0, 0};
  int thr[2] = {0, 0};
  std::vector<float> global, patch, centers;  // [nz][2], [nz][P][2], [P][2]
};

bool load_aln(const std::string& path, LoadedAln* a) {
  FILE* f = std::fopen(path.c_str(), "rt");
  if (!f) return false;
  char line[256], buf[64];
  auto find = [&](const char* key) {
    while (std::fgets(line, sizeof(line), f))
      if (std::strstr(line, key)) return true;
    return false;
  };
  bool ok = find("setting") && find("stackSize") &&
            std::sscanf(line, "%63s %d %d %d %d", buf, a->stk, a->stk + 1, a->stk + 2, a->stk + 3) >= 4;
  ok = ok && find("patches") &&
       std::sscanf(line, "%63s %d %d %d", buf, a->patches, a->patches + 1, a->patches + 2) >= 4;
  ok = ok && find("throw") && std::sscanf(line, "%63s %d %d", buf, a->thr, a->thr + 1) >= 3;
  const int nz = a->stk[2] - a->thr[0] - a->thr[1];
  ok = ok && nz > 0;
  if (ok) {
    a->global.assign(2 * (size_t)nz, 0.0f);
    int n = 0, fr;
    float sx, sy;
    while (n < nz && std::fgets(line, sizeof(line), f))
      if (std::sscanf(line, "%d  %f  %f", &fr, &sx, &sy) == 3) {
        a->global[2 * n] = sx;
        a->global[2 * n + 1] = sy;
        ++n;
      }
    ok = n == nz;
  }
  const int P = a->patches[0] * a->patches[1];
  if (ok && P > 0) {
    a->patch.assign(2 * (size_t)nz * P, 0.0f);
    a->centers.assign(2 * (size_t)P, 0.0f);
    int fm = 0, pc = 0, fr;
    float cx, cy, sx, sy;
    while (pc < P && std::fgets(line, sizeof(line), f)) {
      if (line[0] == '#') continue;
      if (std::sscanf(line, "%d %f %f %f %f", &fr, &cx, &cy, &sx, &sy) != 5) continue;
      a->patch[((size_t)fm * P + pc) * 2] = sx;
      a->patch[((size_t)fm * P + pc) * 2 + 1] = sy;
      a->centers[2 * pc] = cx;
      a->centers[2 * pc + 1] = cy;
      if (++fm == nz) {
        fm = 0;
        ++pc;
      }
    }
    ok = pc == P;
  }
  std::fclose(f);
  return ok;
}

// CLoadAlign::Open(dir, stack) (Align/CLoadAlign.cpp:66-86) and
// CMain::mOpenOutAlnFile: <dir>/<movie file name> with its last extension
// replaced by .aln.
std::string aln_name(const std::string& dir_in, const std::string& movie) {
  std::string name = dir_in;
  if (name.empty() || name.back() != '/') name += "/";
  const size_t slash = movie.rfind('/');
  name += slash == std::string::npos ? movie : movie.substr(slash + 1);
  const size_t dot = name.rfind('.');
  if (dot == std::string::npos) name += ".aln";
  else name = name.substr(0, dot) + ".aln";
  return name;
}

// CLoadRefs::LoadGain / LoadDark (CLoadRefs.cpp:82-202): the gain must be a
// float (mode 2) MRC image; a dark image in another mode is converted as the
// reference's mToFloat does (mode 0 read as signed char).  Both must measure
// 32..32000 pixels per side (sCheckSize).
bool load_ref(const std::string& path, bool is_gain, std::vector<float>* img, int* nx, int* ny) {
  const char* what = is_gain ? "Gain" : "Dark";
  if (is_gain) {
    // CLoadRefs::mGetFileType (CLoadRefs.cpp:93-106): by the last extension
    const size_t dot = path.rfind('.');
    if (dot == std::string::npos) return false;
    const std::string ext = path.substr(dot);
    const bool mrc = strcasestr(ext.c_str(), "mrc") != nullptr;
    const bool tif = !mrc && (strcasestr(ext.c_str(), "tif") || strcasestr(ext.c_str(), "gain"));
    if (!mrc && !tif) return false;
    if (tif) {  // mLoadGainTiff (:125-147): a float TIFF, first directory
      int m = -1, nz = 0;
      if (mc3_tiff_info(path.c_str(), nx, ny, &nz, &m) != MC3_OK) return false;
      if (m != 2) {
        std::printf("Warning: invalid pixel type of %s reference: %d\n"
                    "   mode 2 (32-bit float) is expected.\n\n", what, m);
        return false;
      }
      if (!(*nx >= 32 && *nx <= 32000 && *ny >= 32 && *ny <= 32000)) return false;
      img->resize((size_t)(*nx) * (*ny));
      return mc3_tiff_read(path.c_str(), 0, 1, img->data(), 1) == MC3_OK;
    }
  }
  mc3::mrc::Header h;
  if (!mc3::mrc::read_header(path, &h)) return false;
  if (is_gain && h.mode != 2) {
    std::printf("Warning: invalid pixel type of %s reference: %d\n"
                "   mode 2 (32-bit float) is expected.\n\n%s reference will not be loaded.\n"
                "   %s correction will be skipped.\n\n", what, h.mode, what, what);
    return false;
  }
  if (is_gain && !(h.nx >= 32 && h.nx <= 32000 && h.ny >= 32 && h.ny <= 32000)) {
    std::printf("Warning: invalid size of %s reference: %d  %d\n\n", what, h.nx, h.ny);
    return false;
  }
  const int bpp = mc3::mrc::bytes_per_pixel(h.mode);
  if (!bpp) return false;
  std::vector<unsigned char> raw((size_t)h.nx * h.ny * bpp);
  if (!mc3::mrc::read_frames(path, h, 0, 1, raw.data())) return false;
  const size_t n = (size_t)h.nx * h.ny;
  img->resize(n);
  for (size_t i = 0; i < n; ++i) {
    switch (h.mode) {
      case 0: (*img)[i] = (float)(signed char)raw[i]; break;
      case 5: (*img)[i] = raw[i]; break;
      case 1: (*img)[i] = ((const int16_t*)raw.data())[i]; break;
      case 6: (*img)[i] = ((const uint16_t*)raw.data())[i]; break;
      case 2: (*img)[i] = ((const float*)raw.data())[i]; break;
      default: return false;
    }
  }
  *nx = h.nx;
  *ny = h.ny;
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 2 && strcasecmp(argv[1], "--version") == 0) {
    std::printf("MotionCor3 (mc3-b200) %s\n", mc3_version());
    return eSuccess;
  }
  if (argc <= 1 || (argc == 2 && strcasecmp(argv[1], "--help") == 0)) {
    std::printf("Usage: MotionCor3 -InMrc movie.mrc|-InTiff movie.tif|-InEer movie.eer "
                "[-EerSampling 1|2|3] -OutMrc sum.mrc [-Gain gain.mrc] "
                "[-Patch x y] [-Iter n] [-Tol px] [-Bft g p] [-FmDose d] [-PixSize a] "
                "[-kV kv] [-Group g p] [-FmRef f] [-SumRange lo hi] [-PhaseOnly 0|1] [-SplitSum 0|1] "
                "[-FtBin b] [-OutAln dir] [-InAln dir] [-OutStack 0|1 zbin] [-FmIntFile file] "
                "[-Dark dark.mrc] [-RotGain r] [-FlipGain f] [-InvGain 0|1] [-Mag major minor angle] [-InFmMotion 0|1] [-Throw n] [-Trunc n] [-CorrInterp 0|1] [-DefectFile f] [-DefectMap f] [-OutStar 0|1] "
                "[-LogDir dir] [-Gpu id] [-PatchCenters file (mc3 only: x y per line)]\n");
    return eSuccess;
  }
  Args A{argc, argv};
  mc3_params p;
  mc3_params_default(&p);
  // -InMrc or -InTiff (CInput::IsInTiff, CInput.cpp:697-700); `in_mrc` names
  // the input file either way (logs, .aln names)
  const std::string in_tiff = A.str("-InTiff");
  const std::string in_eer = A.str("-InEer");  // CInput::IsInEer (CInput.cpp:703-707)
  int eer_sampling = 1;
  A.ints("-EerSampling", &eer_sampling, 1);   // CInput.cpp:502-504
  const std::string in_mrc = !in_tiff.empty() ? in_tiff : (!in_eer.empty() ? in_eer : A.str("-InMrc"));
  const std::string out_mrc = A.str("-OutMrc");
  const std::string gain_mrc = A.str("-Gain");
  const std::string dark_mrc = A.str("-Dark");
  int rot_gain = 0, flip_gain = 0, inv_gain = 0;
  A.ints("-RotGain", &rot_gain, 1);    // CInput.cpp:604-614
  A.ints("-FlipGain", &flip_gain, 1);
  A.ints("-InvGain", &inv_gain, 1);
  std::string log_dir = A.str("-LogDir");
  if (!log_dir.empty() && log_dir.back() != '/') log_dir += "/";
  int pt[3] = {0, 0, 0};
  A.ints("-Patch", pt, 3);
  p.patch[0] = pt[0] <= 1 ? 0 : pt[0];
  p.patch[1] = pt[1] <= 1 ? 0 : pt[1];
  p.patch[2] = pt[2] < 0 ? 0 : (pt[2] > 100 ? 100 : pt[2]);  // CInput.cpp:507-511
  const std::string out_aln = A.str("-OutAln");
  A.ints("-Iter", &p.iter, 1);
  A.floats("-Tol", &p.tol, 1);
  A.floats("-Bft", p.bft, 2);
  A.ints("-PhaseOnly", &p.phase_only, 1);
  A.floats("-FtBin", &p.ft_bin, 1);
  A.floats("-InitDose", &p.init_dose, 1);
  A.floats("-FmDose", &p.fm_dose, 1);
  A.floats("-PixSize", &p.pix_size, 1);
  A.ints("-kV", &p.kv, 1);
  A.ints("-Align", &p.align, 1);
  if (A.floats("-SumRange", p.sum_range, 2) && p.sum_range[0] < 0) p.sum_range[0] = 0;
  A.ints("-Group", p.group, 2);
  if (p.group[0] < 1) p.group[0] = 1;
  if (p.group[1] < 1) p.group[1] = 1;
  A.ints("-FmRef", &p.fm_ref, 1);
  A.ints("-SplitSum", &p.split_sum, 1);  // CInput.cpp:657-663
  A.ints("-OutStack", p.out_stack, 2);    // CInput.cpp:590-592
  A.ints("-InFmMotion", &p.in_fm_motion, 1);
  A.ints("-CorrInterp", &p.corr_interp, 1);  // CInput.cpp:673-675
  p.cs = 2.7f;  // CInput::CInput (CInput.cpp:96-99): the command line estimates the CTF by default
  A.floats("-Cs", &p.cs, 1);
  A.floats("-AmpCont", &p.amp_cont, 1);
  A.floats("-ExtPhase", &p.ext_phase, 1);
  int out_star = 0;
  A.ints("-OutStar", &out_star, 1);
  {
    float mg[3];
    int f0, nmag;
    // CInput.cpp:640-644: all three values or none
    if (A.find("-Mag", &f0, &nmag) && nmag == 3 && A.floats("-Mag", mg, 3) == 3)
      for (int i = 0; i < 3; ++i) p.mag[i] = mg[i];
  }
  const std::string in_aln = A.str("-InAln");
  // mc3 extension: "x y" per line, full-frame pixels (mc3_set_patch_centers)
  const std::string patch_centers_file = A.str("-PatchCenters");
  const std::string fmint_file = A.str("-FmIntFile");
  int gpu[8];
  if (A.ints("-Gpu", gpu, 8) > 0) p.gpu = gpu[0];
  const char* ignored[] = { "-InSuffix", "-InSkips", "-ArcDir",
                           "-FullSum", "-TmpFile",
                           "-StackZ", "-Serial",
                           "-Tilt", "-Crop",
                           "-GpuMemUsage", "-UseGpus",
                           "-TiffOrder"};
  for (const char* t : ignored) {
    int f, n;
    A.find(t, &f, &n);
    if (f > 0) std::fprintf(stderr, "Warning: %s is outside the implemented path and is ignored.\n", t);
  }
  if (in_mrc.empty() || out_mrc.empty()) return eFailLoad;
  if (in_mrc == out_mrc) return eInputOutputSame;
  if (!(p.cs > 0.001f && p.kv != 0 && p.pix_size != 0)) {  // CFindCtfMain::bEstimate (:26-40)
    std::printf("Skip CTF estimation. Need the following parameters.\n");
    std::printf("High tension: %d\n", p.kv);
    std::printf("Cs value:     %f\n", p.cs);
    std::printf("Pixel size:   %f\n\n", p.pix_size);
  }

  mc3::mrc::Header h;
  int eer_bits = 0;
  if (!in_eer.empty()) {
    // EER: the raw frames are the electron-event frames; they are rendered
    // below at -EerSampling into 8-bit frames (CLoadEerMain / CRenderMrcStack)
    int cx = 0, cy = 0;
    if (eer_sampling < 1 || eer_sampling > 3 ||
        mc3_eer_info(in_eer.c_str(), &cx, &cy, &h.nz, &eer_bits) != MC3_OK) {
      std::fprintf(stderr, "Error: cannot load EER file %s\n", in_eer.c_str());
      return eFailLoad;
    }
    const int fact = eer_sampling == 2 ? 2 : (eer_sampling == 3 ? 4 : 1);
    h.nx = cx * fact;
    h.ny = cy * fact;
    h.mode = 0;
    std::printf("EER file size bits: %d  %d  %d  %d\n", cx, cy, h.nz, eer_bits);
  } else if (!in_tiff.empty()) {
    if (mc3_tiff_info(in_tiff.c_str(), &h.nx, &h.ny, &h.nz, &h.mode) != MC3_OK) {
      std::fprintf(stderr, "CLoadTiffStack: cannot open Tiff file, skip,\n   %s\n\n",
                   in_tiff.c_str());
      return eFailLoad;
    }
    std::printf("TIFF file size mode: %d  %d  %d  %d\n", h.nx, h.ny, h.nz, h.mode);
  } else {
    if (!mc3::mrc::read_header(in_mrc, &h) || mc3::mrc::frame_bytes(h.mode, h.nx, h.ny) == 0) {
      std::fprintf(stderr, "Error: cannot load %s\n", in_mrc.c_str());
      return eFailLoad;
    }
    std::printf("MRC file size mode: %d  %d  %d  %d\n", h.nx, h.ny, h.nz, h.mode);
  }
  // -Throw / -Trunc (CInput.cpp:567-573): frames dropped at the start / end
  int thr[2] = {0, 0};
  A.ints("-Throw", &thr[0], 1);
  A.ints("-Trunc", &thr[1], 1);
  thr[0] = thr[0] < 0 ? 0 : thr[0];
  thr[1] = thr[1] < 0 ? 0 : thr[1];
  if (h.nz - thr[0] - thr[1] < 3) {
    std::fprintf(stderr, "Error: -Throw %d -Trunc %d leave fewer than 3 of %d frames\n", thr[0],
                 thr[1], h.nz);
    return eFailLoad;
  }
  // -FmIntFile (CReadFmIntFile::DoIt, CFmIntParam::Setup): rendered-frame
  // tables for this movie's raw frames
  std::vector<int> fi_start, fi_size;
  std::vector<float> fi_acc;
  int fi_dose = 0;
  bool fi_on = false;
  if (!fmint_file.empty()) {
    const int maxe = 4096;
    std::vector<int> eg(maxe), en(maxe);
    std::vector<float> ed(maxe);
    int ne = 0;
    if (mc3_read_fmint_file(fmint_file.c_str(), p.fm_dose, maxe, eg.data(), en.data(), ed.data(),
                            &ne) == MC3_OK && ne > 0) {
      ne = ne < maxe ? ne : maxe;
      fi_start.resize(h.nz);
      fi_size.resize(h.nz);
      fi_acc.resize(h.nz);
      int nint = 0;
      if (mc3_frame_integration_tables(eg.data(), en.data(), ed.data(), ne, h.nz, p.fm_dose,
                                       thr[0], thr[1], h.nz, &nint, fi_start.data(),
                                       fi_size.data(), fi_acc.data(), &fi_dose) == MC3_OK &&
          nint > 0) {
        fi_start.resize(nint);
        fi_size.resize(nint);
        fi_acc.resize(nint);
        fi_on = true;
        std::printf("Rendered size mode: %d  %d  %d  %d\n", h.nx, h.ny, nint,
                    (nint != h.nz) ? 0 : h.mode);
      }
    }
  }
  if (!in_eer.empty() && !fi_on) {  // every kept EER frame rendered on its own
    const int keep = h.nz - thr[0] - thr[1];
    fi_start.resize(keep);
    fi_size.assign(keep, 1);
    fi_acc.resize(keep);
    for (int i = 0; i < keep; ++i) {
      fi_start[i] = i + thr[0];
      fi_acc[i] = p.fm_dose * (i + 1);  // CFmIntParam::mSetup
    }
    fi_dose = 0;
    fi_on = true;
  }
  // without rendered-frame tables the throws only select the raw frames read
  const mc3::mrc::Header h_file = h;  // the file's own frame count, for reading
  const int z_first = fi_on ? 0 : thr[0];
  if (!fi_on) h.nz -= thr[0] + thr[1];
  const int n_raw = h.nz;
  const int n_render = fi_on ? (int)fi_start.size() : h.nz;
  // -InAln (CMain::mOpenInAlnFile, CMain.cpp:382-398): the file's patch
  // grid and throws replace the command line's.
  LoadedAln la;
  bool aln_ok = false;
  if (!in_aln.empty()) {
    aln_ok = load_aln(aln_name(in_aln, in_mrc), &la);
    if (aln_ok && (la.thr[0] != 0 || la.thr[1] != 0)) {
      std::printf("Info: alignment files with thrown frames are not supported; "
                  "the movie is aligned.\n\n");
      aln_ok = false;
    } else if (aln_ok && la.stk[2] != n_render) {
      std::printf("Info: alignment file covers %d frames, the movie has %d; "
                  "the movie is aligned.\n\n", la.stk[2], n_render);
      aln_ok = false;
    } else if (!aln_ok) {
      std::printf("Info: Alignment file cannot be read.\n\n");
    }
    if (aln_ok) {
      p.patch[0] = la.patches[0] <= 1 ? 0 : la.patches[0];
      p.patch[1] = la.patches[1] <= 1 ? 0 : la.patches[1];
      p.patch[2] = la.patches[2];
      if (p.patch[0] == 0 || p.patch[1] == 0) la.patch.clear();
    }
  }
  const size_t frame_bytes = (size_t)mc3::mrc::frame_bytes(h.mode, h.nx, h.ny);
  if (!in_eer.empty()) h.nz = n_render;  // the movie handed over holds the rendered frames
  HostBuf frames(frame_bytes * h.nz);
  if (!in_eer.empty()) {
    if (mc3_eer_render(in_eer.c_str(), eer_sampling, n_render, fi_start.data(), fi_size.data(),
                       frames.as<unsigned char>(), 0) != MC3_OK) {
      std::fprintf(stderr, "Error: cannot decode EER frames of %s\n", in_eer.c_str());
      return eFailLoad;
    }
  } else if (!in_tiff.empty()) {
    if (mc3_tiff_read(in_tiff.c_str(), z_first, h.nz, frames.p, 0) != MC3_OK) {
      std::fprintf(stderr, "error: load tiff images of %s\n", in_tiff.c_str());
      return eFailLoad;
    }
  } else if (!mc3::mrc::read_frames(in_mrc, h_file, z_first, h.nz, frames.as<unsigned char>())) {
    return eFailLoad;
  }

  mc3_ctx* ctx = nullptr;
  int s = mc3_create(&p, &ctx);
  if (s != MC3_OK) {
    std::fprintf(stderr, "Error: %s\n", mc3_strerror(s));
    return eNoValidGPUs;
  }
  // ---- references: CMain::mLoadRefs (CMain.cpp:326-340), CLoadRefs::PostProcess
  //      and AugmentRefs (CLoadRefs.cpp:82-268), CProcessThread::mCheckGain ----
  {
    std::vector<float> gain, dark;
    int gx = 0, gy = 0, dx = 0, dy = 0;
    bool have_gain = !gain_mrc.empty() && load_ref(gain_mrc, true, &gain, &gx, &gy);
    bool have_dark = !dark_mrc.empty() && load_ref(dark_mrc, false, &dark, &dx, &dy);
    if (have_dark && (!have_gain || dx != gx || dy != gy)) {  // mCheckDarkRef
      std::printf("Warning: The sizes of Dark and gain references do not match.\n"
                  "   Dark reference has been removed.\n\n");
      have_dark = false;
    }
    if (have_gain && (rot_gain != 0 || flip_gain != 0 || inv_gain != 0)) {
      std::vector<float> t(gain.size());
      mc3_ref_orient(gain.data(), gx, gy, rot_gain, flip_gain, inv_gain, t.data(), &gx, &gy);
      gain.swap(t);
      // the reference orients the dark only when (rot != 0 || flip == 0), and never inverts it
      if (have_dark && (rot_gain != 0 || flip_gain == 0)) {
        std::vector<float> u(dark.size());
        mc3_ref_orient(dark.data(), dx, dy, rot_gain, flip_gain, 0, u.data(), &dx, &dy);
        dark.swap(u);
      }
    }
    // super-resolution frames: references repeated by the common integer factor
    if (have_gain && (gx != h.nx || gy != h.ny)) {
      const int fx = h.nx / gx, fy = h.ny / gy;
      if (fx == 0 || fy == 0 || fx != fy || h.nx % gx || h.ny % gy) {
        std::fprintf(stderr, "Error: cannot augment gain reference.\n   Frame size: %d  %d\n"
                             "   Ref size:   %d  %d\n\n", h.nx, h.ny, gx, gy);
      } else {
        std::vector<float> t((size_t)h.nx * h.ny);
        mc3_ref_augment(gain.data(), gx, gy, fx, t.data());
        gain.swap(t);
        if (have_dark) {
          std::vector<float> u((size_t)h.nx * h.ny);
          mc3_ref_augment(dark.data(), dx, dy, fx, u.data());
          dark.swap(u);
          dx *= fx;
          dy *= fx;
        }
        gx *= fx;
        gy *= fx;
      }
    }
    if (!have_gain) {
      std::printf("Warning: Gain ref not found.\n......   Gain correction will be skipped.\n\n");
    } else if (gx != h.nx || gy != h.ny) {
      std::fprintf(stderr, "Error: Gain and frame dimensions mismatch!\n"
                           "...... Gain size:  %d  %d\n...... Frame size: %d  %d\n"
                           "Motion correction skipped.\n\n", gx, gy, h.nx, h.ny);
      mc3_destroy(ctx);
      return eFailProcess;
    } else {
      mc3_set_gain(ctx, gain.data(), gx, gy, 0);
      if (have_dark) mc3_set_dark(ctx, dark.data(), dx, dy, 0);
    }
  }
  // ---- known camera defects: CDetectMain::mLoadDefectFile / mLoadDefectMap
  //      (BadPixel/CDetectMain.cpp:146-260) ----
  const std::string defect_file = A.str("-DefectFile");
  const std::string defect_map = A.str("-DefectMap");
  if (!defect_file.empty() || !defect_map.empty()) {
    std::vector<unsigned char> mask((size_t)h.nx * h.ny, 0);
    bool any = false;
    if (FILE* f = defect_file.empty() ? nullptr : std::fopen(defect_file.c_str(), "rt")) {
      std::printf("Load camera defects.\n");
      char line[256];
      while (std::fgets(line, sizeof(line), f)) {
        int e[4];
        if (std::sscanf(line, "%d  %d  %d  %d", e, e + 1, e + 2, e + 3) != 4) continue;
        std::printf("...... Defect: %6d  %6d  %6d  %6d\n", e[0], e[1], e[2], e[3]);
        if (e[0] < 0) e[0] = 0;
        if (e[1] < 0) e[1] = 0;
        const int ex = e[0] + e[2] > h.nx ? h.nx : e[0] + e[2];
        const int ey = e[1] + e[3] > h.ny ? h.ny : e[1] + e[3];
        for (int y = e[1]; y < ey; ++y)
          for (int x = e[0]; x < ex; ++x) mask[(size_t)y * h.nx + x] = 1;
        any = true;
      }
      std::fclose(f);
      std::printf("Load camera defects: done.\n\n");
    }
    if (!defect_map.empty()) {
      // an 8-bit MRC image of the frame size, else an 8-bit TIFF (read
      // bottom-up like every TIFF image); bit 0 marks a defect
      std::vector<unsigned char> dm((size_t)h.nx * h.ny);
      bool ok = false;
      mc3::mrc::Header dh;
      if (mc3::mrc::read_header(defect_map, &dh) && (dh.mode == 0 || dh.mode == 5) &&
          dh.nx == h.nx && dh.ny == h.ny)
        ok = mc3::mrc::read_frames(defect_map, dh, 0, 1, dm.data());
      int tx = 0, ty = 0, tz = 0, tm = -1;
      if (!ok && mc3_tiff_info(defect_map.c_str(), &tx, &ty, &tz, &tm) == MC3_OK && tm == 0 &&
          tx == h.nx && ty == h.ny)
        ok = mc3_tiff_read(defect_map.c_str(), 0, 1, dm.data(), 1) == MC3_OK;
      if (ok) {
        for (size_t i = 0; i < dm.size(); ++i) mask[i] |= dm[i] & 1;
        any = true;
      }
    }
    if (any) mc3_set_defects(ctx, mask.data(), h.nx, h.ny);
  }
  mc3_plan_info info;
  if (fi_on) {
    mc3_frame_integration fi{n_raw, (int)fi_start.size(), fi_start.data(), fi_size.data(),
                             fi_acc.data(), fi_dose, in_eer.empty() ? 0 : 1};
    if ((s = mc3_set_frame_integration(ctx, &fi)) != MC3_OK) {
      std::fprintf(stderr, "Error: %s\n", mc3_strerror(s));
      mc3_destroy(ctx);
      return eFailProcess;
    }
  }
  if ((s = mc3_plan(ctx, h.nx, h.ny, h.nz, &info)) != MC3_OK) {
    std::fprintf(stderr, "Error: %s\n", mc3_strerror(s));
    mc3_destroy(ctx);
    return eFailProcess;
  }
  const int N = n_render, P = info.n_patches;
  if (aln_ok) {
    mc3_alignment al{};
    al.nz = N;
    al.global_shifts = la.global.data();
    al.n_patches = la.patch.empty() ? 0 : P;
    al.patch_shifts = la.patch.empty() ? nullptr : la.patch.data();
    al.patch_centers = la.patch.empty() ? nullptr : la.centers.data();
    if ((s = mc3_set_alignment(ctx, &al)) != MC3_OK) {
      std::fprintf(stderr, "Error: %s\n", mc3_strerror(s));
      mc3_destroy(ctx);
      return eFailProcess;
    }
  }
  if (!patch_centers_file.empty() && P > 0) {
    std::vector<float> pcs;
    if (FILE* fp = std::fopen(patch_centers_file.c_str(), "r")) {
      float x, y;
      while (std::fscanf(fp, "%f %f", &x, &y) == 2) {
        pcs.push_back(x);
        pcs.push_back(y);
      }
      std::fclose(fp);
    }
    if ((int)pcs.size() != 2 * P || (s = mc3_set_patch_centers(ctx, pcs.data(), P)) != MC3_OK) {
      std::fprintf(stderr, "Error: -PatchCenters %s: %d patch centres needed\n",
                   patch_centers_file.c_str(), P);
      mc3_destroy(ctx);
      return eFailProcess;
    }
  }
  const int ox = info.out_size[0], oy = info.out_size[1];  // -FtBin output size
  HostBuf sums_buf(sizeof(float) * (size_t)info.n_sums * ox * oy);
  float* sums = sums_buf.as<float>();
  std::vector<float> gsh(2 * (size_t)N), psh(2 * (size_t)N * (P > 0 ? P : 1)), pc(2 * (P > 0 ? P : 1));
  std::vector<unsigned char> pb((size_t)N * (P > 0 ? P : 1));
  std::vector<int> iters(1 + P);
  std::vector<float> errs((size_t)p.iter * (1 + P));
  mc3_movie mv{frames.p, h.mode, h.nx, h.ny, h.nz, 0};
  mc3_result r{};
  r.sums = sums;
  r.global_shifts = gsh.data();
  r.patch_shifts = P ? psh.data() : nullptr;
  r.patch_centers = P ? pc.data() : nullptr;
  r.patch_bad = P ? pb.data() : nullptr;
  r.iterations = iters.data();
  r.errors = errs.data();
  std::vector<unsigned char> hot((size_t)h.nx * h.ny);
  if (out_star) r.hot_map = hot.data();
  std::vector<float> ctf_img((size_t)512 * 512);
  r.ctf_spectrum = ctf_img.data();
  std::unique_ptr<HostBuf> stack_buf;
  if (p.out_stack[0] != 0) {
    stack_buf.reset(new HostBuf(sizeof(float) * (size_t)N * ox * oy));
    r.stack = stack_buf->as<float>();
  }
  auto t0 = std::chrono::steady_clock::now();
  s = mc3_process_movie(ctx, &mv, &r);
  auto t1 = std::chrono::steady_clock::now();
  if (s != MC3_OK) {
    std::fprintf(stderr, "Error: processing failed: %s\n", mc3_strerror(s));
    mc3_destroy(ctx);
    return eFailProcess;
  }
  for (int i = 0; i < iters[0]; ++i)
    std::printf("Iteration %2d  Error: %9.3f\n", i + 1, errs[i]);
  if (r.ctf_done) {  // CFindCtfMain::DoIt (FindCtf/CFindCtfMain.cpp:65-78)
    std::printf("CTF estimate\n");
    std::printf("  Df_max [A]   Df_min [A]  Azimuth [d]  Phase [d]    Score       Res\n");
    std::printf("  %9.2f    %9.2f  %8.2f    %7.2f    %9.4f  %7.2f\n\n", r.ctf[0], r.ctf[1], r.ctf[2],
                r.ctf[3], r.ctf[4], r.ctf[5]);
  }
  std::printf("Computation time: %f sec\n\n", std::chrono::duration<double>(t1 - t0).count());
  // ---- sums ----
  // file name extensions in the order of CAlnSums::Setup (DataUtil/CAlnSums.cpp:18-43)
  std::vector<const char*> exts = {"", "_DW", "_DWS"};
  exts.resize(r.n_sums - (p.split_sum ? 2 : 0));
  if (p.split_sum) {
    exts.push_back("_ODD");
    exts.push_back("_EVN");
  }
  // CInput::GetFinalPixelSize (CInput.cpp:709-715)
  const float pix = p.pix_size * p.ft_bin / (p.mag[0] > p.mag[1] ? p.mag[0] : p.mag[1]);
  bool saved = true;
  for (int i = 0; i < r.n_sums; ++i) {
    const float* img = sums + (size_t)i * ox * oy;
    float mn, mx, me;
    stats(img, (size_t)ox * oy, &mn, &mx, &me);
    const std::string name = out_name(out_mrc, exts[i], ".mrc");
    saved = mc3::mrc::write_float_image(name, img, ox, oy, pix, mn, mx, me) && saved;
    std::printf("Corrected sum has been saved in:\n   %s\n\n", name.c_str());
  }
  // ---- aligned stack (CSaveSerialCryoEM::mSaveStack, CSaveSerialCryoEM.cpp:146-211):
  //      min/max over frames, mean of the frame means, 32 ext-header floats ----
  if (stack_buf && r.stack_frames > 0) {
    const size_t fpx = (size_t)ox * oy;
    float mn = 1e20f, mx = -1e20f;
    double mean = 0.0;
    for (int i = 0; i < r.stack_frames; ++i) {
      float a, b, m;
      stats(r.stack + i * fpx, fpx, &a, &b, &m);
      mn = a < mn ? a : mn;
      mx = b > mx ? b : mx;
      mean += m;
    }
    mean /= r.stack_frames;
    const std::string name = out_name(out_mrc, "_Stk", ".mrc");
    std::printf("Saving motion corrected stack ......\n");
    saved = mc3::mrc::write_float_stack(name, r.stack, ox, oy, r.stack_frames, pix, mn, mx,
                                        (float)mean, 32) && saved;
    std::printf("Motion corrected stack done.\n\n");
  }
  // ---- CTF outputs (CSaveSerialCryoEM::mSaveCtfStack / mSaveCtfFit,
  //      CSaveSerialCryoEM.cpp:243-297): the 512 x 512 spectrum (pixel size 1,
  //      header statistics left at their defaults) and the fit line ----
  if (r.ctf_done) {
    saved = mc3::mrc::write_float_image(out_name(out_mrc, "_Ctf", ".mrc"), ctf_img.data(), 512, 512, 1.0f,
                                        0.f, 0.f, 0.f) && saved;
    const std::string txt = out_name(out_mrc, "_Ctf", ".txt");
    if (FILE* fh = std::fopen(txt.c_str(), "w")) {
      std::fprintf(fh, "# Columns: #1 micrograph number; "
                       "#2 - defocus 1 [A]; #3 - defocus 2; "
                       "#4 - azimuth of astigmatism; "
                       "#5 - additional phase shift [radian]; "
                       "#6 - cross correlation; "
                       "#7 - spacing (in Angstroms) up to which CTF rings were "
                       "fit successfully\n");
      std::fprintf(fh, " %9.2f  %9.2f  %7.2f  %7.2f  %9.5f  %8.4f\n", r.ctf[0], r.ctf[1], r.ctf[2], r.ctf[3],
                   r.ctf[4], r.ctf[5]);
      std::fclose(fh);
    }
  }
  // ---- RELION star file (-OutStar; CGenStarFile, CGenStarFile.cpp:44-159):
  //      <OutMrc directory>/<movie name>.star, where the movie name is the
  //      -InTiff file's (CMain::mDoSingleCryoEM passes m_acInTifFile, empty for
  //      MRC and EER input, which therefore write "<OutMrc directory>/.star") ----
  if (out_star) {
    std::string name = out_mrc;
    const size_t sl = name.rfind('/');
    name = sl == std::string::npos ? std::string() : name.substr(0, sl + 1);
    const size_t ms = in_tiff.rfind('/');
    const std::string in_main = ms == std::string::npos ? in_tiff : in_tiff.substr(ms + 1);
    std::string main = in_main;
    const size_t dot = main.rfind('.');
    main = dot == std::string::npos ? main + ".star" : main.substr(0, dot) + ".star";
    if (FILE* f = std::fopen((name + main).c_str(), "wt")) {
      std::fprintf(f, "\n# version 30001\n\n");
      std::fprintf(f, "data_general\n\n");
      std::fprintf(f, "%40s %-16d\n", "_rlnImageSizeX", h.nx);
      std::fprintf(f, "%40s %-16d\n", "_rlnImageSizeY", h.ny);
      std::fprintf(f, "%40s %-16d\n", "_rlnImageSizeZ", N);
      std::fprintf(f, "%40s %s\n", "_rlnMicrographMovieName", in_main.c_str());
      if (gain_mrc.empty()) {
        std::fprintf(f, "%40s\n", "_rlnMicrographGainName");
      } else {
        const size_t gs = gain_mrc.rfind('/');
        std::fprintf(f, "%40s %s\n", "_rlnMicrographGainName",
                     (gs == std::string::npos ? gain_mrc : gain_mrc.substr(gs + 1)).c_str());
      }
      std::fprintf(f, "%40s %-16.6f\n", "_rlnMicrographOriginalPixelSize", p.pix_size);
      std::fprintf(f, "%40s %-16.6f\n", "rlnMicrographBinning", p.ft_bin);
      std::fprintf(f, "%40s %-16.6f\n", "_rlnMicrographDoseRate", p.fm_dose);
      std::fprintf(f, "%40s %-16.6f\n", "_rlnMicrographPreExposure", 0.0f);
      std::fprintf(f, "%40s %-16.6f\n", "_rlnVoltage", (float)p.kv);
      std::fprintf(f, "%40s %-16d\n", "_rlnMicrographStartFrame", thr[0] + 1);
      std::fprintf(f, "%40s %-16d\n", "_rlnMotionModelVersion", 0);
      std::fprintf(f, "\n");
      // SetHotPixels: the reference passes the row as an int to %f; the
      // intended value, ny - y, is written here
      std::fprintf(f, "data_hot_pixels\n\n");
      std::fprintf(f, "loop\n");
      std::fprintf(f, "_rlnCoordinateX #1\n");
      std::fprintf(f, "_rlnCoordinateY #2\n");
      for (int y = 0; y < h.ny; ++y)
        for (int x = 0; x < h.nx; ++x)
          if (hot[(size_t)y * h.nx + x])
            std::fprintf(f, "%13.6f  %13.6f\n", x + 1.0f, (double)(h.ny - y));
      std::fprintf(f, "\n\n");
      // SetGlobalShifts: frame shifts relative to the first frame
      std::fprintf(f, "# version 30001\n\n");
      std::fprintf(f, "data_global_shift\n\n");
      std::fprintf(f, "loop\n");
      std::fprintf(f, "_rlnMicrographFrameNumber #1\n");
      std::fprintf(f, "_rlnMicrographShiftX #2\n");
      std::fprintf(f, "_rlnMicrographShiftY #3\n");
      for (int i = 0; i < N; ++i)
        std::fprintf(f, "%13d %13.6f %13.6f\n", i + 1, gsh[2 * i] - gsh[0],
                     gsh[2 * i + 1] - gsh[1]);
      std::fprintf(f, "\n");
      std::fclose(f);
    }
  }
  // ---- logs ----
  const std::string stem = log_stem(log_dir, in_mrc);
  if (!stem.empty()) {
    const char* fmt = "%4d  %8.2f  %8.2f\n";
    if (P == 0) {
      FILE* f = std::fopen((stem + "-Full.log").c_str(), "wt");
      if (f) {
        std::fprintf(f, "# full frame alignment\n");
        for (int i = 0; i < N; ++i) std::fprintf(f, fmt, i + 1, gsh[2 * i], gsh[2 * i + 1]);
        std::fclose(f);
      }
    } else {
      FILE* f = std::fopen((stem + "-Patch-Full.log").c_str(), "wt");
      if (f) {
        std::fprintf(f, "# Patch based alignment\n");
        std::fprintf(f, "# Initial alignment based upon full frames\n\n");
        for (int i = 0; i < N; ++i) std::fprintf(f, fmt, i + 1, gsh[2 * i], gsh[2 * i + 1]);
        std::fclose(f);
      }
      f = std::fopen((stem + "-Patch-Patch.log").c_str(), "wt");
      if (f) {
        std::fprintf(f, "# Patch based alignment\n");
        std::fprintf(f, "# Number of patches: %d\n", P);
        std::fprintf(f, "# Shifts are listed per patch.\n");
        std::fprintf(f, "# Movie size: %d  %d  %d\n\n", h.nx, h.ny, N);
        for (int i = 0; i < P; ++i) {
          std::fprintf(f, "#Patch %03d raw and fit shifts\n", i + 1);
          for (int j = 0; j < N; ++j) {
            const size_t k = (size_t)j * P + i;
            std::fprintf(f, "%4d %8.2f %8.2f ", j + 1, pc[2 * i], pc[2 * i + 1]);
            std::fprintf(f, "%8.2f %8.2f %4d\n", psh[2 * k], psh[2 * k + 1], (int)pb[k]);
          }
          std::fprintf(f, "\n");
        }
        std::fclose(f);
      }
      f = std::fopen((stem + "-Patch-Frame.log").c_str(), "wt");
      if (f) {
        std::fprintf(f, "# Patch based alignment\n");
        std::fprintf(f, "# Number of patches: %d\n", P);
        std::fprintf(f, "# Shifts are listed per frame.\n");
        std::fprintf(f, "# Movie size: %d  %d  %d\n\n", h.nx, h.ny, N);
        for (int i = 0; i < N; ++i) {
          for (int j = 0; j < P; ++j) {
            const size_t k = (size_t)i * P + j;
            std::fprintf(f, "%4d %8.2f %8.2f ", i + 1, pc[2 * j], pc[2 * j + 1]);
            std::fprintf(f, "%8.2f %8.2f %4d\n", psh[2 * k], psh[2 * k + 1], (int)pb[k]);
          }
          std::fprintf(f, "\n");
        }
        std::fclose(f);
      }
    }
  }
  // ---- alignment file (-OutAln; Align/CSaveAlign.cpp:61-151, opened by
  //      CMain::mOpenOutAlnFile, CMain.cpp:367-380) ----
  if (!out_aln.empty()) {
    const std::string name = aln_name(out_aln, in_mrc);
    FILE* f = std::fopen(name.c_str(), "wt");
    if (!f) {
      std::printf("Info: %s\n%s\n\n", "      cannot be opened. Alignment wiil not be saved.",
                  name.c_str());
    } else {
      std::fprintf(f, "setting\n");
      std::fprintf(f, "   stackSize: %d %d %d %d\n", h.nx, h.ny, N, 1);
      std::fprintf(f, "   patches: %d %d %d\n", p.patch[0], p.patch[1], p.patch[2]);
      std::fprintf(f, "   throw: %d %d\n", thr[0], thr[1]);
      std::fprintf(f, "#    Global Shift\n");
      std::fprintf(f, "#---------------------\n");
      std::fprintf(f, "globalShift\n");
      std::fprintf(f, "   stackID %d\n", 0);
      for (int i = 0; i < N; ++i)
        std::fprintf(f, "%6d  %+8.3f  %+8.3f\n", i, gsh[2 * i], gsh[2 * i + 1]);
      if (P > 0) {
        std::fprintf(f, "#    Local Shift\n");
        std::fprintf(f, "#---------------------\n");
        std::fprintf(f, "localShift\n");
        for (int i = 0; i < P; ++i) {
          std::fprintf(f, "   patchID: %d\n", i);
          std::fprintf(f, "   Converge: %d\n", 1);
          for (int j = 0; j < N; ++j) {
            const size_t k = (size_t)j * P + i;
            std::fprintf(f, "%6d  %8.2f  %8.2f  %+8.3f  %+8.3f\n", j, pc[2 * i], pc[2 * i + 1],
                         psh[2 * k], psh[2 * k + 1]);
          }
          if (i < P - 1) std::fprintf(f, "\n");
        }
      }
      std::fclose(f);
    }
  }
  mc3_destroy(ctx);
  return saved ? eSuccess : eFailSave;
}
