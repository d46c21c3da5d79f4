// Kernel variants chosen per movie size by the autotuner (mc3_autotune).
//
// The launch wrappers read the variant to use from the calling thread's
// active Tuning; the engine makes its table's entry for the movie's size
// active for the duration of a movie.  Without an entry the defaults hold
// (set from MC3_FFT_R16, MC3_FFT_COL_WIDE, MC3_GATHER_PX and MC3_FFT_ROW_PIPE when
// present).
#pragma once
#include <string>
#include <vector>

namespace mc3 {

struct Tuning {
  int fft_r16 = 1;    // radix-16 register passes for power-of-two lengths (else radix 8)
  int col_wide = 1;   // 4096-point column passes: 0 two columns per CTA, 1 four columns
                      // per CTA, 2 persistent with the next columns prefetched
  int gather_px = 2;  // pixels per thread in the local-motion gather (1 or 2)
  int row_pipe = 0;   // 4096-real row R2C and C2R: persistent, next rows by bulk copies
};

// Defaults (environment) and the calling thread's active choices.
const Tuning& default_tuning();
Tuning& active_tuning();

// Makes `t` active on this thread for the lifetime of the scope.
struct TuningScope {
  Tuning saved;
  explicit TuningScope(const Tuning& t);
  ~TuningScope();
};

// One autotuned size: movie geometry and options key, the choice and the
// measured device time of every candidate.
struct TuningEntry {
  int nx = 0, ny = 0, nz = 0, px = 0, py = 0;
  Tuning best;
  double best_ms = 0.0;
  std::vector<Tuning> cand;
  std::vector<double> cand_ms;
};

// All variants the tuner tries.
std::vector<Tuning> tuning_candidates();
// JSON text of entries, one entry per line, and its reader.
std::string tuning_json(const std::vector<TuningEntry>& e, const char* device);
int parse_tuning_json(const std::string& text, std::vector<TuningEntry>* out);

}  // namespace mc3
