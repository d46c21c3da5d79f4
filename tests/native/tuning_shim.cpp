// Host build of libmc3's tuning-table code (csrc/tuning.cpp) for the CPU
// tests: a JSON text written by tuning_json is read back by
// parse_tuning_json.
#include "../../motioncor3_b200/csrc/tuning.cpp"

#include <cstring>

extern "C" {
// Writes two entries, reads them back; returns the number of fields that
// differ (0 = the round trip is exact), or -1 when parsing fails.
int shim_tuning_roundtrip(char* json_out, int cap) {
  using namespace mc3;
  std::vector<TuningEntry> es(2);
  es[0].nx = 4096, es[0].ny = 4096, es[0].nz = 60, es[0].px = 5, es[0].py = 5;
  es[0].best.fft_r16 = 1, es[0].best.col_wide = 1, es[0].best.gather_px = 1;
  es[0].best_ms = 41.25;
  es[0].cand = tuning_candidates();
  for (size_t i = 0; i < es[0].cand.size(); ++i) es[0].cand_ms.push_back(40.0 + i);
  es[1].nx = 5760, es[1].ny = 4092, es[1].nz = 8, es[1].px = 7, es[1].py = 5;
  es[1].best.fft_r16 = 0, es[1].best.col_wide = 0, es[1].best.gather_px = 2;
  es[1].best_ms = 9.5;
  const std::string js = tuning_json(es, "test device");
  std::snprintf(json_out, cap, "%s", js.c_str());
  std::vector<TuningEntry> back;
  if (parse_tuning_json(js, &back) != 0 || back.size() != 2) return -1;
  int bad = 0;
  for (int i = 0; i < 2; ++i) {
    const TuningEntry &a = es[i], &b = back[i];
    bad += a.nx != b.nx || a.ny != b.ny || a.nz != b.nz || a.px != b.px || a.py != b.py;
    bad += a.best.fft_r16 != b.best.fft_r16 || a.best.col_wide != b.best.col_wide ||
           a.best.gather_px != b.best.gather_px;
    bad += std::abs(a.best_ms - b.best_ms) > 1e-3;
    bad += a.cand.size() != b.cand.size();
    for (size_t k = 0; k < a.cand.size() && k < b.cand.size(); ++k)
      bad += a.cand[k].col_wide != b.cand[k].col_wide || a.cand[k].row_pipe != b.cand[k].row_pipe ||
             std::abs(a.cand_ms[k] - b.cand_ms[k]) > 1e-3;
    // the persistent row passes go with the persistent column pass
    bad += b.best.row_pipe != (b.best.col_wide == 2);
  }
  return bad;
}

int shim_tuning_parse(const char* text) {
  std::vector<mc3::TuningEntry> back;
  return mc3::parse_tuning_json(text, &back) != 0 ? -1 : (int)back.size();
}

int shim_tuning_candidates() { return (int)mc3::tuning_candidates().size(); }

// Candidates whose persistent row and column passes are not paired, and
// candidates that differ in nothing: both must be 0.
int shim_tuning_candidate_faults() {
  const std::vector<mc3::Tuning> c = mc3::tuning_candidates();
  int bad = 0;
  for (size_t i = 0; i < c.size(); ++i) {
    bad += c[i].row_pipe != (c[i].col_wide == 2);
    for (size_t k = 0; k < i; ++k)
      bad += c[i].fft_r16 == c[k].fft_r16 && c[i].col_wide == c[k].col_wide &&
             c[i].gather_px == c[k].gather_px && c[i].row_pipe == c[k].row_pipe;
  }
  return bad;
}
}
