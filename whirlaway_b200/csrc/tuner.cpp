// Autotuner table (see tuner.h): process-wide, per device and shape.
#include "tuner.h"

#include <map>
#include <mutex>
#include <tuple>

namespace wl {

namespace {
struct Entry {
  int plan;
  std::vector<float> ms;
};
std::mutex g_mu;
std::map<std::tuple<int, int, uint64_t>, Entry> g_table;
int g_forced[TUNE_FAMILIES] = {-1, -1, -1, -1};
const char* const kNames[TUNE_FAMILIES] = {"lde", "leaf", "merkle", "inner"};
const int kPlans[TUNE_FAMILIES] = {6, 3, 3, 2};
const int kDefaults[TUNE_FAMILIES] = {2, 1, 1, 0};
}  // namespace

const char* tune_family_name(int f) { return f >= 0 && f < TUNE_FAMILIES ? kNames[f] : "?"; }
int tune_plan_count(int f) { return f >= 0 && f < TUNE_FAMILIES ? kPlans[f] : 0; }
int tune_default_plan(int f) { return f >= 0 && f < TUNE_FAMILIES ? kDefaults[f] : 0; }
int tune_family_from_name(const char* name) {
  if (!name) return -1;
  for (int f = 0; f < TUNE_FAMILIES; f++)
    if (std::string(name) == kNames[f]) return f;
  return -1;
}
void tune_force(int f, int plan) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (f >= 0 && f < TUNE_FAMILIES) g_forced[f] = plan >= 0 && plan < kPlans[f] ? plan : -1;
}
int tune_forced(int f) {
  std::lock_guard<std::mutex> lk(g_mu);
  return f >= 0 && f < TUNE_FAMILIES ? g_forced[f] : -1;
}
int tune_lookup(int device, int f, uint64_t key) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_table.find({device, f, key});
  return it == g_table.end() ? -1 : it->second.plan;
}
void tune_store(int device, int f, uint64_t key, int plan, const std::vector<float>& ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table[{device, f, key}] = Entry{plan, ms};
}
void tune_clear() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
}
std::string tune_json() {
  std::lock_guard<std::mutex> lk(g_mu);
  std::string o = "{";
  for (int f = 0; f < TUNE_FAMILIES; f++) {
    o += std::string(f ? ", " : "") + "\"" + kNames[f] + "\": [";
    bool first = true;
    for (const auto& kv : g_table) {
      if (std::get<1>(kv.first) != f) continue;
      o += std::string(first ? "" : ", ") + "{\"device\": " + std::to_string(std::get<0>(kv.first)) +
           ", \"key\": " + std::to_string(std::get<2>(kv.first)) + ", \"plan\": " + std::to_string(kv.second.plan) +
           ", \"ms\": [";
      for (size_t i = 0; i < kv.second.ms.size(); i++) o += (i ? ", " : "") + std::to_string(kv.second.ms[i]);
      o += "]}";
      first = false;
    }
    o += "]";
  }
  return o + "}";
}

}  // namespace wl
