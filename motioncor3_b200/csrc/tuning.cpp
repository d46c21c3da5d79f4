// Tuning table: defaults, the per-thread active choice, and the JSON form
// written by mc3_autotune and read by mc3_load_tuning.
#include "tuning.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace mc3 {

namespace {
int env_int(const char* name, int dflt) {
  const char* e = getenv(name);
  return (e && e[0]) ? atoi(e) : dflt;
}
thread_local bool t_init = false;
thread_local Tuning t_active;
}  // namespace

const Tuning& default_tuning() {
  static const Tuning d = [] {
    Tuning t;
    t.fft_r16 = env_int("MC3_FFT_R16", 1) != 0;
    t.col_wide = std::min(std::max(env_int("MC3_FFT_COL_WIDE", 1), 0), 2);
    t.gather_px = env_int("MC3_GATHER_PX", 2) == 1 ? 1 : 2;
    t.row_pipe = env_int("MC3_FFT_ROW_PIPE", 0) != 0;
    return t;
  }();
  return d;
}

Tuning& active_tuning() {
  if (!t_init) {
    t_active = default_tuning();
    t_init = true;
  }
  return t_active;
}

TuningScope::TuningScope(const Tuning& t) : saved(active_tuning()) { active_tuning() = t; }
TuningScope::~TuningScope() { active_tuning() = saved; }

std::vector<Tuning> tuning_candidates() {
  std::vector<Tuning> c;
  // the column variants differ only in the radix-16 passes
  for (int r16 = 1; r16 >= 0; --r16)
    for (int wide = 0; wide <= (r16 ? 2 : 0); ++wide)
      for (int px = 2; px >= 1; --px) {
        Tuning t;
        t.fft_r16 = r16;
        t.col_wide = wide;
        t.gather_px = px;
        t.row_pipe = wide == 2;  // the persistent passes go together
        c.push_back(t);
      }
  return c;
}

std::string tuning_json(const std::vector<TuningEntry>& es, const char* device) {
  std::string s = "{\"mc3_tuning\": 1, \"device\": \"";
  s += device ? device : "";
  s += "\", \"entries\": [\n";
  char buf[512];
  for (size_t i = 0; i < es.size(); ++i) {
    const TuningEntry& e = es[i];
    snprintf(buf, sizeof(buf),
             "{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"patch\": [%d, %d], \"fft_r16\": %d, "
             "\"col_wide\": %d, \"gather_px\": %d, \"ms\": %.4f, \"candidates\": [",
             e.nx, e.ny, e.nz, e.px, e.py, e.best.fft_r16, e.best.col_wide, e.best.gather_px,
             e.best_ms);
    s += buf;
    for (size_t k = 0; k < e.cand.size(); ++k) {
      snprintf(buf, sizeof(buf), "%s{\"fft_r16\": %d, \"col_wide\": %d, \"gather_px\": %d, \"ms\": %.4f}",
               k ? ", " : "", e.cand[k].fft_r16, e.cand[k].col_wide, e.cand[k].gather_px,
               e.cand_ms[k]);
      s += buf;
    }
    s += "]}";
    s += i + 1 < es.size() ? ",\n" : "\n";
  }
  s += "]}\n";
  return s;
}

namespace {
// Integer value of "key": in [p, end); false when absent.
bool find_int(const char* p, const char* end, const char* key, int* v) {
  char pat[64];
  snprintf(pat, sizeof(pat), "\"%s\": ", key);
  const char* q = strstr(p, pat);
  if (!q || q >= end) return false;
  *v = atoi(q + strlen(pat));
  return true;
}
}  // namespace

int parse_tuning_json(const std::string& text, std::vector<TuningEntry>* out) {
  if (text.find("\"mc3_tuning\": 1") == std::string::npos) return 1;
  out->clear();
  // entries: one per line, starting with {"nx":
  size_t pos = 0;
  while ((pos = text.find("{\"nx\": ", pos)) != std::string::npos) {
    size_t eol = text.find('\n', pos);
    if (eol == std::string::npos) eol = text.size();
    const char* p = text.c_str() + pos;
    // the entry's own keys come before its candidate list
    size_t cpos = text.find("\"candidates\"", pos);
    const char* end = text.c_str() + (cpos != std::string::npos && cpos < eol ? cpos : eol);
    TuningEntry e;
    int px = 0, py = 0;
    bool ok = find_int(p, end, "nx", &e.nx) && find_int(p, end, "ny", &e.ny) &&
              find_int(p, end, "nz", &e.nz) && find_int(p, end, "fft_r16", &e.best.fft_r16) &&
              find_int(p, end, "col_wide", &e.best.col_wide) &&
              find_int(p, end, "gather_px", &e.best.gather_px);
    const char* pp = strstr(p, "\"patch\": [");
    if (ok && pp && pp < end && sscanf(pp, "\"patch\": [%d, %d]", &px, &py) == 2) {
      e.px = px;
      e.py = py;
    } else {
      return 1;
    }
    const char* ms = strstr(p, "\"ms\": ");
    if (ms && ms < end) e.best_ms = atof(ms + 6);
    if (e.best.gather_px != 1) e.best.gather_px = 2;
    e.best.row_pipe = e.best.col_wide == 2;  // the persistent passes go together
    // the candidates: {"fft_r16": a, "col_wide": b, "gather_px": c, "ms": t} each
    if (cpos != std::string::npos && cpos < eol) {
      const char* q = text.c_str() + cpos;
      const char* qend = text.c_str() + eol;
      while ((q = strstr(q, "{\"fft_r16\": ")) && q < qend) {
        Tuning t;
        double tms = 0.0;
        if (sscanf(q, "{\"fft_r16\": %d, \"col_wide\": %d, \"gather_px\": %d, \"ms\": %lf}",
                   &t.fft_r16, &t.col_wide, &t.gather_px, &tms) != 4)
          return 1;
        t.row_pipe = t.col_wide == 2;
        e.cand.push_back(t);
        e.cand_ms.push_back(tms);
        ++q;
      }
    }
    out->push_back(e);
    pos = eol;
  }
  return 0;
}

}  // namespace mc3
