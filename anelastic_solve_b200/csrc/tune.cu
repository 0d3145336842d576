// tune.cu -- process-wide registry of autotuned launch variants.
#include "tune.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

namespace anel {

namespace {
struct Entry {
  int chosen;
  std::vector<double> ms;
};
std::mutex g_mu;
std::map<std::string, Entry> g_entries;
bool g_loaded = false;

// ANEL_TUNE_CACHE=<file>: choices persist across processes as lines
// "key<TAB>variant<TAB>ms ms ...", read once before the first lookup and
// appended by every store (a profiler run can replay a timed run's choices)
const char* cache_path() {
  const char* p = std::getenv("ANEL_TUNE_CACHE");
  return p && *p ? p : nullptr;
}

void load_cache_locked() {
  if (g_loaded) return;
  g_loaded = true;
  const char* path = cache_path();
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char line[1024];
  while (std::fgets(line, sizeof(line), f)) {
    char* tab = std::strchr(line, '\t');
    if (!tab) continue;
    *tab = 0;
    char* rest = tab + 1;
    char* end = nullptr;
    const long v = std::strtol(rest, &end, 10);
    if (end == rest || v < 0) continue;
    Entry e{(int)v, {}};
    for (char* q = end; *q;) {
      char* e2 = nullptr;
      const double t = std::strtod(q, &e2);
      if (e2 == q) break;
      e.ms.push_back(t);
      q = e2;
    }
    g_entries[line] = e;
  }
  std::fclose(f);
}
}  // namespace

bool tune_enabled() {
  const char* v = std::getenv("ANEL_TUNE");
  return !(v && (std::strcmp(v, "0") == 0 || std::strcmp(v, "off") == 0));
}

int tune_lookup(const std::string& key) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_cache_locked();
  auto it = g_entries.find(key);
  return it == g_entries.end() ? -1 : it->second.chosen;
}

void tune_store(const std::string& key, int chosen, const std::vector<double>& ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  load_cache_locked();
  g_entries[key] = Entry{chosen, ms};
  if (const char* path = cache_path()) {
    if (FILE* f = std::fopen(path, "a")) {
      std::fprintf(f, "%s\t%d\t", key.c_str(), chosen);
      for (double t : ms) std::fprintf(f, " %.6f", t);
      std::fprintf(f, "\n");
      std::fclose(f);
    }
  }
}

std::string tune_report() {
  std::lock_guard<std::mutex> lk(g_mu);
  std::string out;
  char buf[64];
  for (const auto& kv : g_entries) {
    out += kv.first;
    std::snprintf(buf, sizeof(buf), ": variant %d (", kv.second.chosen);
    out += buf;
    for (size_t q = 0; q < kv.second.ms.size(); ++q) {
      std::snprintf(buf, sizeof(buf), q ? " %.4f" : "%.4f", kv.second.ms[q]);
      out += buf;
    }
    out += " ms)\n";
  }
  return out;
}

}  // namespace anel
