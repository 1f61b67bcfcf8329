// Launch-configuration autotuner (see tune.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <vector>

#include "tune.h"

namespace pmf {
namespace {

struct Entry {
  int choice = 0;
  std::vector<float> us;  // per-launch microseconds of each candidate (< 0: not applicable)
};

struct Table {
  std::mutex mu;
  std::map<std::string, Entry> rows;
  bool loaded = false;
  int enabled = -1;  // -1: from the environment
  std::string device;
};

Table& table() {
  static Table t;
  return t;
}

const char* tune_file() {
  const char* f = getenv("PMF_TUNE_FILE");
  return (f && *f) ? f : nullptr;
}

// File format: one line per key, "<key>\t<choice>\t<t0>,<t1>,..."
void load_locked(Table& t) {
  t.loaded = true;
  const char* path = tune_file();
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  char line[4096];
  while (fgets(line, sizeof(line), f)) {
    char* tab1 = strchr(line, '\t');
    if (!tab1) continue;
    *tab1 = 0;
    char* tab2 = strchr(tab1 + 1, '\t');
    Entry e;
    e.choice = atoi(tab1 + 1);
    if (tab2) {
      std::stringstream ss(tab2 + 1);
      std::string tok;
      while (std::getline(ss, tok, ',')) e.us.push_back((float)atof(tok.c_str()));
    }
    t.rows[line] = e;
  }
  fclose(f);
}

void save_locked(const Table& t) {
  const char* path = tune_file();
  if (!path) return;
  FILE* f = fopen(path, "w");
  if (!f) return;
  for (const auto& kv : t.rows) {
    fprintf(f, "%s\t%d\t", kv.first.c_str(), kv.second.choice);
    for (size_t i = 0; i < kv.second.us.size(); ++i) fprintf(f, "%s%.3f", i ? "," : "", kv.second.us[i]);
    fprintf(f, "\n");
  }
  fclose(f);
}

}  // namespace

void tune_set_enabled(bool on) {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  t.enabled = on ? 1 : 0;
}

bool tune_enabled() {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  if (t.enabled < 0) {
    const char* e = getenv("PMF_AUTOTUNE");
    t.enabled = (e && e[0] == '0') ? 0 : 1;
  }
  return t.enabled == 1;
}

const std::string& tune_device() {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  if (t.device.empty()) {
    int dev = 0;
    cudaDeviceProp p;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&p, dev) == cudaSuccess)
      t.device = p.name;
    else
      t.device = "unknown";
  }
  return t.device;
}

int tune_choose(const std::string& key0, int ncand, const std::function<bool(int)>& launch, cudaStream_t st,
                int reps) {
  if (ncand <= 1) return 0;
  if (const char* f = getenv("PMF_TUNE_FORCE")) {  // tests: run candidate f (clamped) without timing
    const int c = atoi(f);
    return c < 0 ? 0 : (c >= ncand ? ncand - 1 : c);
  }
  if (!tune_enabled()) return 0;
  const std::string key = key0 + "|" + tune_device();
  Table& t = table();
  {
    std::lock_guard<std::mutex> lk(t.mu);
    if (!t.loaded) load_locked(t);
    auto it = t.rows.find(key);
    if (it != t.rows.end() && it->second.choice >= 0 && it->second.choice < ncand) return it->second.choice;
  }
  // a capture in progress cannot be timed: use the default and tune on a later call
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  Entry ent;
  ent.us.assign(ncand, -1.0f);
  float best = 1e30f;
  for (int c = 0; c < ncand; ++c) {
    if (!launch(c)) continue;  // warm-up (and applicability)
    if (cudaGetLastError() != cudaSuccess) continue;
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch(c);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) continue;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ent.us[c] = 1e3f * ms / (float)reps;
    if (ent.us[c] < best) {
      best = ent.us[c];
      ent.choice = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lk(t.mu);
  t.rows[key] = ent;
  save_locked(t);
  return ent.choice;
}

int tune_online_pick(const std::string& key0, int ncand) {
  if (ncand <= 1) return 0;
  if (const char* f = getenv("PMF_TUNE_FORCE")) {
    const int c = atoi(f);
    return c < 0 ? 0 : (c >= ncand ? ncand - 1 : c);
  }
  if (!tune_enabled()) return 0;
  const std::string key = key0 + "|" + tune_device();
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  if (!t.loaded) load_locked(t);
  auto it = t.rows.find(key);
  if (it == t.rows.end()) return 0;
  Entry& e = it->second;
  if ((int)e.us.size() != ncand) return 0;
  for (int c = 0; c < ncand; ++c)
    if (e.us[c] < 0.0f) return c;  // not measured yet
  return e.choice;
}

void tune_online_report(const std::string& key0, int ncand, int cand, float us_per_unit) {
  if (ncand <= 1 || cand < 0 || cand >= ncand || getenv("PMF_TUNE_FORCE") || !tune_enabled()) return;
  const std::string key = key0 + "|" + tune_device();
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  Entry& e = t.rows[key];
  if ((int)e.us.size() != ncand) {
    e.us.assign(ncand, -1.0f);
    e.choice = 0;
  }
  const bool complete_before = [&] {
    for (float u : e.us)
      if (u < 0.0f) return false;
    return true;
  }();
  if (complete_before) return;  // decided: later steps do not move the choice
  e.us[cand] = us_per_unit;
  float best = 1e30f;
  bool complete = true;
  for (int c = 0; c < ncand; ++c) {
    if (e.us[c] < 0.0f) {
      complete = false;
      continue;
    }
    if (e.us[c] < best) {
      best = e.us[c];
      e.choice = c;
    }
  }
  if (complete) save_locked(t);
}

std::string tune_report() {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  std::ostringstream o;
  o << "{";
  bool first = true;
  for (const auto& kv : t.rows) {
    if (!first) o << ", ";
    first = false;
    o << "\"" << kv.first << "\": {\"choice\": " << kv.second.choice << ", \"us\": [";
    for (size_t i = 0; i < kv.second.us.size(); ++i) {
      if (i) o << ", ";
      char buf[32];
      snprintf(buf, sizeof(buf), "%.2f", kv.second.us[i]);
      o << buf;
    }
    o << "]}";
  }
  o << "}";
  return o.str();
}

}  // namespace pmf
