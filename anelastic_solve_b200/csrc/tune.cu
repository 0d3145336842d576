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
}  // namespace

bool tune_enabled() {
  const char* v = std::getenv("ANEL_TUNE");
  return !(v && (std::strcmp(v, "0") == 0 || std::strcmp(v, "off") == 0));
}

int tune_lookup(const std::string& key) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_entries.find(key);
  return it == g_entries.end() ? -1 : it->second.chosen;
}

void tune_store(const std::string& key, int chosen, const std::vector<double>& ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_entries[key] = Entry{chosen, ms};
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
