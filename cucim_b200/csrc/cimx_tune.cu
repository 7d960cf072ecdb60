// cimx_tune.cu — the schedule autotuner of cimx_separable.
//
// A pass list can run on several kernel schedules that give bit-identical
// results: the single-launch volume kernel or stream + slab launches, the
// stream kernel or the generic kernel for leading axes, the row stream or
// the slab kernel for the last two axes, the volume kernel's z chunk, fused
// launches or one launch per pass. Which is fastest depends on the dtypes,
// the tap counts and the extents. (cuCIM makes the corresponding choice, its
// shared-memory or elementwise kernel, by a fixed rule:
// _vendored/_ndimage_filters.py:284-297.) With algorithm="tensor" the
// tuner also chooses between the tensor-core and the plain float32 pass per
// call (the caller has accepted the tensor path's tolerance), replacing the
// fixed 2048-sample line rule.
//
// Tuning happens per call signature: the dtypes, the shape, each pass's axis,
// taps count, mode and flags, and the caller's tensor flags. In mode
// CIMX_TUNE_ON an unseen signature is timed on the call's own arrays (each
// candidate once to warm up, then three times between CUDA events on the
// call's stream) and the fastest schedule is recorded; in CIMX_TUNE_USE
// (the default) recorded schedules are used and unseen signatures run the
// built-in rules. Tables are per device model (the device name), each
// behind its own mutex. CIMX_TUNE (0, 1, 2) sets the initial mode and
// CIMX_TUNE_CACHE names a JSON file that is read at first use and rewritten
// after every newly tuned signature.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "cimx_common.cuh"
#include "cimx_internal.h"

namespace cimx {
namespace {

struct Entry {
  int flags = 0;
  double ms = 0;
  std::vector<std::pair<int, double>> candidates;
};

constexpr int kMaxDev = 64;
std::mutex g_mode_mu;
int g_mode = -1;  // -1: not read from the environment yet
std::string g_cache_path;
bool g_cache_read = false;

// one table per device model; the mutex of a table guards it and its file I/O
struct DeviceTable {
  std::mutex mu;
  std::map<std::string, Entry> entries;
};
std::mutex g_tables_mu;
std::map<std::string, DeviceTable*> g_tables;  // never freed: lives until exit
std::atomic<long long> g_entries{0};           // entries in all tables
DeviceTable* g_dev_table[kMaxDev] = {};         // the current device's table, by index (g_tables_mu)

std::mutex g_name_mu;
std::string g_names[kMaxDev];

std::string device_name() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return "unknown";
  std::lock_guard<std::mutex> g(g_name_mu);
  if (g_names[dev].empty()) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "unknown";
    g_names[dev] = std::string(p.name) + " (" + std::to_string(p.multiProcessorCount) + " SMs)";
  }
  return g_names[dev];
}

DeviceTable& table_for(const std::string& device) {
  std::lock_guard<std::mutex> g(g_tables_mu);
  DeviceTable*& t = g_tables[device];
  if (!t) t = new DeviceTable();
  return *t;
}

// the current device's table, found by name once per device index
DeviceTable& current_table() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return table_for("unknown");
  {
    std::lock_guard<std::mutex> g(g_tables_mu);
    if (g_dev_table[dev]) return *g_dev_table[dev];
  }
  DeviceTable& t = table_for(device_name());
  std::lock_guard<std::mutex> g(g_tables_mu);
  g_dev_table[dev] = &t;
  return t;
}

// ------------------------------------------------------------------ JSON

std::string json_escape(const std::string& s) {
  std::string o;
  for (char c : s) {
    if (c == '"' || c == '\\') {
      o += '\\';
      o += c;
    } else if ((unsigned char)c < 0x20) {
      char b[8];
      snprintf(b, sizeof(b), "\\u%04x", (unsigned)(unsigned char)c);
      o += b;
    } else {
      o += c;
    }
  }
  return o;
}

std::string dump_all() {
  std::ostringstream o;
  o.precision(17);
  o << "{\"format\": \"cimx-tune-1\", \"entries\": [";
  bool first = true;
  std::lock_guard<std::mutex> g(g_tables_mu);
  for (auto& dt : g_tables) {
    std::lock_guard<std::mutex> gt(dt.second->mu);
    for (auto& kv : dt.second->entries) {
      o << (first ? "\n  " : ",\n  ");
      first = false;
      o << "{\"device\": \"" << json_escape(dt.first) << "\", \"key\": \""
        << json_escape(kv.first) << "\", \"flags\": " << kv.second.flags
        << ", \"ms\": " << kv.second.ms << ", \"candidates\": [";
      for (size_t i = 0; i < kv.second.candidates.size(); ++i)
        o << (i ? ", " : "") << "[" << kv.second.candidates[i].first << ", "
          << kv.second.candidates[i].second << "]";
      o << "]}";
    }
  }
  o << "\n]}\n";
  return o.str();
}

// A small JSON reader: values are objects, arrays, strings, numbers,
// true/false/null; objects become key -> value maps.
struct JVal {
  enum Kind { NUL, NUM, STR, ARR, OBJ, BOOL } kind = NUL;
  double num = 0;
  std::string str;
  std::vector<JVal> arr;
  std::map<std::string, JVal> obj;
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  explicit JParser(const std::string& text) : s(text) {}
  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  bool lit(const char* t) {
    const size_t n = strlen(t);
    if (s.compare(i, n, t) != 0) return false;
    i += n;
    return true;
  }
  bool str(std::string& out) {
    if (i >= s.size() || s[i] != '"') return false;
    ++i;
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\') {
        if (++i >= s.size()) return false;
        if (s[i] == 'u') {
          if (i + 4 >= s.size()) return false;
          out += (char)strtol(s.substr(i + 1, 4).c_str(), nullptr, 16);
          i += 5;
          continue;
        }
        const char e = s[i];
        out += e == 'n' ? '\n' : e == 't' ? '\t' : e;
        ++i;
      } else {
        out += s[i++];
      }
    }
    if (i >= s.size()) return false;
    ++i;
    return true;
  }
  bool value(JVal& v, int depth = 0) {
    if (depth > 32) return false;
    ws();
    if (i >= s.size()) return false;
    const char c = s[i];
    if (c == '{') {
      ++i;
      v.kind = JVal::OBJ;
      ws();
      if (i < s.size() && s[i] == '}') {
        ++i;
        return true;
      }
      for (;;) {
        ws();
        std::string k;
        if (!str(k)) return false;
        ws();
        if (i >= s.size() || s[i] != ':') return false;
        ++i;
        if (!value(v.obj[k], depth + 1)) return false;
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          ++i;
          return true;
        }
        return false;
      }
    }
    if (c == '[') {
      ++i;
      v.kind = JVal::ARR;
      ws();
      if (i < s.size() && s[i] == ']') {
        ++i;
        return true;
      }
      for (;;) {
        v.arr.emplace_back();
        if (!value(v.arr.back(), depth + 1)) return false;
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          ++i;
          return true;
        }
        return false;
      }
    }
    if (c == '"') {
      v.kind = JVal::STR;
      return str(v.str);
    }
    if (lit("true")) {
      v.kind = JVal::BOOL;
      v.num = 1;
      return true;
    }
    if (lit("false")) {
      v.kind = JVal::BOOL;
      return true;
    }
    if (lit("null")) return true;
    char* end = nullptr;
    v.num = strtod(s.c_str() + i, &end);
    if (end == s.c_str() + i) return false;
    i = end - s.c_str();
    v.kind = JVal::NUM;
    return true;
  }
};

int load_text(const std::string& text, const char* what) {
  JVal root;
  JParser p(text);
  if (!p.value(root) || root.kind != JVal::OBJ)
    return fail(CIMX_E_INVALID, std::string("tuning table ") + what + ": not a JSON object");
  auto fmt = root.obj.find("format");
  if (fmt == root.obj.end() || fmt->second.str != "cimx-tune-1")
    return fail(CIMX_E_INVALID, std::string("tuning table ") + what + ": unknown format");
  auto ents = root.obj.find("entries");
  if (ents == root.obj.end() || ents->second.kind != JVal::ARR)
    return fail(CIMX_E_INVALID, std::string("tuning table ") + what + ": no entries list");
  for (const JVal& e : ents->second.arr) {
    if (e.kind != JVal::OBJ) return fail(CIMX_E_INVALID, "tuning table: bad entry");
    auto dev = e.obj.find("device"), key = e.obj.find("key"), fl = e.obj.find("flags"),
         ms = e.obj.find("ms");
    if (dev == e.obj.end() || key == e.obj.end() || fl == e.obj.end() ||
        dev->second.kind != JVal::STR || key->second.kind != JVal::STR ||
        fl->second.kind != JVal::NUM)
      return fail(CIMX_E_INVALID, "tuning table: entry without device, key or flags");
    Entry en;
    en.flags = (int)fl->second.num;
    en.ms = ms != e.obj.end() ? ms->second.num : 0.0;
    auto cands = e.obj.find("candidates");
    if (cands != e.obj.end() && cands->second.kind == JVal::ARR)
      for (const JVal& c : cands->second.arr)
        if (c.kind == JVal::ARR && c.arr.size() == 2)
          en.candidates.emplace_back((int)c.arr[0].num, c.arr[1].num);
    DeviceTable& t = table_for(dev->second.str);
    std::lock_guard<std::mutex> g(t.mu);
    if (t.entries.insert_or_assign(key->second.str, en).second) ++g_entries;
  }
  return CIMX_OK;
}

int load_file(const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) return fail(CIMX_E_INVALID, std::string("cannot open tuning table ") + path);
  std::string text;
  char buf[65536];
  size_t n;
  while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  fclose(f);
  return load_text(text, path);
}

int save_file(const char* path) {
  const std::string text = dump_all();
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = fopen(tmp.c_str(), "wb");
  if (!f) return fail(CIMX_E_INVALID, std::string("cannot write tuning table ") + path);
  const bool ok = fwrite(text.data(), 1, text.size(), f) == text.size();
  if (fclose(f) != 0 || !ok || rename(tmp.c_str(), path) != 0)
    return fail(CIMX_E_INVALID, std::string("cannot write tuning table ") + path);
  return CIMX_OK;
}

// CIMX_TUNE and CIMX_TUNE_CACHE, read once
void init_from_env() {
  std::lock_guard<std::mutex> g(g_mode_mu);
  if (g_mode >= 0) return;
  g_mode = CIMX_TUNE_USE;
  if (const char* m = getenv("CIMX_TUNE")) {
    const int v = atoi(m);
    if (v >= CIMX_TUNE_OFF && v <= CIMX_TUNE_ON) g_mode = v;
  }
  if (const char* p = getenv("CIMX_TUNE_CACHE")) g_cache_path = p;
}

void read_cache_once() {
  std::string path;
  {
    std::lock_guard<std::mutex> g(g_mode_mu);
    if (g_cache_read || g_cache_path.empty()) return;
    g_cache_read = true;
    path = g_cache_path;
  }
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return;  // not written yet
  fclose(f);
  load_file(path.c_str());
}

constexpr int kScheduleBits = CIMX_L_NO_FUSION | CIMX_L_NO_VOLUME | CIMX_L_NO_STREAM |
                              CIMX_L_NO_ROWSTREAM | (3 << CIMX_L_ZCHUNK_SHIFT) |
                              (3 << CIMX_L_SLAB_SPAN_SHIFT);
constexpr int kTensorBits = CIMX_L_TENSOR_BF16X3 | CIMX_L_TENSOR_TF32X3;

}  // namespace

std::string tune_key(const CimxArray* in, const CimxArray* out, const PassDesc* ds,
                     int npasses, int lib_flags) {
  // built with plain appends: this runs on every call that may be tuned
  std::string o;
  o.reserve(48 + 24 * npasses);
  char b[24];
  auto num = [&](long long v) {
    const auto r = std::to_chars(b, b + sizeof(b), v);
    o.append(b, r.ptr);
  };
  o += (char)in->dtype;
  o += '>';
  o += (char)out->dtype;
  o += " [";
  for (int d = 0; d < in->ndim; ++d) {
    if (d) o += ',';
    num(in->shape[d]);
  }
  o += ']';
  for (int i = 0; i < npasses; ++i) {
    o += " a";
    num(ds[i].axis);
    o += 'k';
    num(ds[i].K);
    o += 'o';
    num(ds[i].anchor);
    o += 'm';
    num(ds[i].mode);
    if (ds[i].w64) o += 'd';
    if (ds[i].skip_zero) o += 'z';
    if (ds[i].cval_as_input) o += 'c';
  }
  o += " t";
  num(lib_flags & (kTensorBits | CIMX_L_TENSOR_ALL_LINES));
  return o;
}

bool tuning_needed(int lib_flags) {
  init_from_env();
  int mode;
  {
    std::lock_guard<std::mutex> g(g_mode_mu);
    mode = g_mode;
  }
  if (mode == CIMX_TUNE_OFF || (lib_flags & (kScheduleBits | CIMX_L_NO_TUNE))) return false;
  if (mode == CIMX_TUNE_ON) return true;
  read_cache_once();
  return g_entries.load(std::memory_order_relaxed) > 0;  // nothing recorded: nothing to apply
}

int tuned_flags(const std::string& key, int lib_flags, cudaStream_t st,
                const std::function<int(int)>& run) {
  init_from_env();
  int mode;
  {
    std::lock_guard<std::mutex> g(g_mode_mu);
    mode = g_mode;
  }
  // a caller that chose a schedule, or asked for none to be tuned, keeps it
  if (mode == CIMX_TUNE_OFF || (lib_flags & (kScheduleBits | CIMX_L_NO_TUNE))) return lib_flags;
  read_cache_once();
  DeviceTable& t = current_table();
  {
    std::lock_guard<std::mutex> g(t.mu);
    auto it = t.entries.find(key);
    if (it != t.entries.end()) return (lib_flags & ~kScheduleBits & ~kTensorBits &
                                       ~CIMX_L_TENSOR_ALL_LINES) | it->second.flags;
  }
  if (mode != CIMX_TUNE_ON) return lib_flags;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return lib_flags;  // no synchronising measurement inside a capture
  }

  // candidates: every bit-identical schedule; with a tensor bit also the
  // tensor cores on every eligible pass and the plain float32 passes
  std::vector<int> cands;
  const int base = lib_flags & ~(kScheduleBits | CIMX_L_NO_TUNE);
  const int sched[] = {0,
                       CIMX_L_NO_VOLUME,
                       CIMX_L_NO_ROWSTREAM,
                       CIMX_L_NO_VOLUME | CIMX_L_NO_ROWSTREAM,
                       CIMX_L_NO_STREAM,
                       CIMX_L_NO_STREAM | CIMX_L_NO_VOLUME,
                       CIMX_L_NO_FUSION,
                       1 << CIMX_L_ZCHUNK_SHIFT,
                       2 << CIMX_L_ZCHUNK_SHIFT,
                       3 << CIMX_L_ZCHUNK_SHIFT,
                       1 << CIMX_L_SLAB_SPAN_SHIFT,
                       2 << CIMX_L_SLAB_SPAN_SHIFT,
                       3 << CIMX_L_SLAB_SPAN_SHIFT};
  for (int s : sched) cands.push_back(base | s);
  if (base & kTensorBits) {
    cands.push_back(base | CIMX_L_TENSOR_ALL_LINES);
    cands.push_back(base & ~(kTensorBits | CIMX_L_TENSOR_ALL_LINES));
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return lib_flags;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return lib_flags;
  }
  Entry best;
  best.ms = INFINITY;
  best.flags = lib_flags & ~CIMX_L_NO_TUNE;
  for (int c : cands) {
    if (run(c | CIMX_L_NO_TUNE) != CIMX_OK) continue;  // warm-up; a schedule that fails is skipped
    cudaEventRecord(e0, st);
    bool ok = true;
    for (int r = 0; r < 3 && ok; ++r) ok = run(c | CIMX_L_NO_TUNE) == CIMX_OK;
    cudaEventRecord(e1, st);
    if (!ok || cudaEventSynchronize(e1) != cudaSuccess) continue;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const double per = ms / 3.0;
    best.candidates.emplace_back(c, per);
    if (per < best.ms) {
      best.ms = per;
      best.flags = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best.candidates.empty()) return lib_flags;
  best.flags &= kScheduleBits | kTensorBits | CIMX_L_TENSOR_ALL_LINES;
  {
    std::lock_guard<std::mutex> g(t.mu);
    if (t.entries.insert_or_assign(key, best).second) ++g_entries;
  }
  std::string path;
  {
    std::lock_guard<std::mutex> g(g_mode_mu);
    path = g_cache_path;
  }
  if (!path.empty()) save_file(path.c_str());
  return (lib_flags & ~kScheduleBits & ~kTensorBits & ~CIMX_L_TENSOR_ALL_LINES) | best.flags;
}

}  // namespace cimx

using namespace cimx;

extern "C" {

int cimx_tune_mode(int mode) {
  init_from_env();
  std::lock_guard<std::mutex> g(g_mode_mu);
  const int prev = g_mode;
  if (mode >= CIMX_TUNE_OFF && mode <= CIMX_TUNE_ON) g_mode = mode;
  else if (mode >= 0) return fail(CIMX_E_INVALID, "tuning mode must be 0, 1 or 2");
  return prev;
}

int cimx_tune_load(const char* path) {
  if (!path) return fail(CIMX_E_INVALID, "path is NULL");
  return load_file(path);
}

int cimx_tune_save(const char* path) {
  if (!path) return fail(CIMX_E_INVALID, "path is NULL");
  return save_file(path);
}

int cimx_tune_clear(void) {
  std::lock_guard<std::mutex> g(g_tables_mu);
  for (auto& dt : g_tables) {
    std::lock_guard<std::mutex> gt(dt.second->mu);
    dt.second->entries.clear();
  }
  g_entries = 0;
  return CIMX_OK;
}

long long cimx_tune_dump(char* buf, long long size) {
  const std::string text = dump_all();
  if (buf && size > 0) {
    const size_t n = std::min<size_t>(text.size(), (size_t)size - 1);
    memcpy(buf, text.data(), n);
    buf[n] = '\0';
  }
  return (long long)text.size() + 1;
}

}  // extern "C"
