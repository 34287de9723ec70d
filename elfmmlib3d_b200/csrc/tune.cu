// tune.cu -- the autotuner (tune.h): per-key exploration of equivalent
// implementations from the timings of real passes, decisions kept for the
// process and optionally in a file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include "tune.h"
#include "../../include/elfmm3d_b200.h"

namespace efmm {

bool TuneKey::operator<(const TuneKey& o) const {
  const int a[6] = {knob, p, nbox, C, prec, kind}, b[6] = {o.knob, o.p, o.nbox, o.C, o.prec, o.kind};
  return std::lexicographical_compare(a, a + 6, b, b + 6);
}
bool TuneKey::operator==(const TuneKey& o) const { return !(*this < o) && !(o < *this); }

namespace {

struct Entry {
  std::vector<float> ms;   // fastest timed run per candidate (inf: untried)
  std::vector<int> visits;
  int decided = -1;
};

std::mutex g_mu;
std::map<TuneKey, Entry> g_map;
bool g_loaded = false;

const char* tune_file() {
  const char* f = getenv("ELFMM3D_TUNE_FILE");
  return (f && f[0]) ? f : nullptr;
}

Entry& entry(const TuneKey& k, int ncand) {
  Entry& e = g_map[k];
  if ((int)e.ms.size() < ncand) {
    e.ms.resize(ncand, std::numeric_limits<float>::infinity());
    e.visits.resize(ncand, 0);
  }
  return e;
}

// decisions from the file: lines "knob p nbox C prec kind decided"
void load_locked() {
  if (g_loaded) return;
  g_loaded = true;
  const char* f = tune_file();
  if (!f) return;
  FILE* fp = fopen(f, "r");
  if (!fp) return;
  TuneKey k;
  int d;
  while (fscanf(fp, "%d %d %d %d %d %d %d", &k.knob, &k.p, &k.nbox, &k.C, &k.prec, &k.kind, &d) == 7) {
    int c;
    while ((c = fgetc(fp)) != '\n' && c != EOF) {
    }
    if (d >= 0) entry(k, d + 1).decided = d;
  }
  fclose(fp);
}

void save_locked(const TuneKey& k, const Entry& e) {
  const char* f = tune_file();
  if (!f) return;
  FILE* fp = fopen(f, "a");
  if (!fp) return;
  fprintf(fp, "%d %d %d %d %d %d %d", k.knob, k.p, k.nbox, k.C, k.prec, k.kind, e.decided);
  for (float m : e.ms) fprintf(fp, " %.4f", std::isinf(m) ? -1.0f : m);
  fprintf(fp, "\n");
  fclose(fp);
}

}  // namespace

int tune_pick(const TuneKey& k, int ncand) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_locked();
  Entry& e = entry(k, ncand);
  if (e.decided >= 0 && e.decided < ncand) return e.decided;
  for (int c = 0; c < ncand; c++)
    if (e.visits[c] < TUNE_VISITS) return c;
  e.decided = (int)(std::min_element(e.ms.begin(), e.ms.begin() + ncand) - e.ms.begin());
  save_locked(k, e);
  return e.decided;
}

int tune_best(const TuneKey& k, int fallback) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_locked();
  auto it = g_map.find(k);
  return (it != g_map.end() && it->second.decided >= 0) ? it->second.decided : fallback;
}

void tune_report(const TuneKey& k, int ncand, int cand, float ms) {
  if (cand < 0 || cand >= ncand || !(ms >= 0.0f)) return;
  std::lock_guard<std::mutex> lk(g_mu);
  Entry& e = entry(k, ncand);
  e.visits[cand]++;
  e.ms[cand] = std::min(e.ms[cand], ms);
}

void tune_reset() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_map.clear();
  g_loaded = false;
}

std::vector<std::string> tune_dump() {
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<std::string> out;
  for (const auto& kv : g_map) {
    const TuneKey& k = kv.first;
    char buf[256];
    int w = snprintf(buf, sizeof(buf), "%d %d %d %d %d %d %d", k.knob, k.p, k.nbox, k.C, k.prec, k.kind,
                     kv.second.decided);
    for (float m : kv.second.ms)
      w += snprintf(buf + w, sizeof(buf) - w, " %.4f", std::isinf(m) ? -1.0f : m);
    out.push_back(buf);
  }
  return out;
}

}  // namespace efmm

// C ABI of the tuner (tests, inspection): pick / report / reset / dump.
extern "C" int efmm_tune_pick(int knob, int p, int nbox, int C, int prec, int kind, int ncand) {
  return efmm::tune_pick({knob, p, nbox, C, prec, kind}, ncand);
}
extern "C" void efmm_tune_report(int knob, int p, int nbox, int C, int prec, int kind, int ncand, int cand,
                                 float ms) {
  efmm::tune_report({knob, p, nbox, C, prec, kind}, ncand, cand, ms);
}
extern "C" void efmm_tune_reset(void) { efmm::tune_reset(); }
extern "C" int efmm_tune_dump(char* buf, int len) {
  std::string s;
  for (const std::string& l : efmm::tune_dump()) s += l + "\n";
  if (buf && len > 0) {
    const int n = std::min((int)s.size(), len - 1);
    memcpy(buf, s.data(), n);
    buf[n] = '\0';
  }
  return (int)s.size();
}
