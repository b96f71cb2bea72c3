// The tuner's persistent cache: a versioned JSON file of choices keyed by (GPU, shape
// class). The file holds
//   {"version": 1, "entries": [{"gpu": "...", "class": "...", "ms": 1.5,
//                               "choice": {"kind": "split", "a_mode": "smem"}}, ...]}
// and is read with a small JSON parser (objects, arrays, strings, numbers, literals).
#include "kg_tune.cuh"
#include "kyto_gpu.h"

#include <cuda_runtime.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <vector>

#include <sys/stat.h>
#include <unistd.h>

namespace kg {

namespace {

// ------------------------------------------------------------------ JSON values ----

struct Json {
  enum Type { Null, Bool, Number, String, Array, Object } type = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;

  const Json* get(const std::string& key) const {
    if (type != Object) return nullptr;
    for (const auto& kv : obj)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

// Recursive descent over the text; any error leaves ok false (the file is then ignored).
struct Parser {
  const std::string& t;
  size_t i = 0;
  bool ok = true;
  int depth = 0;

  explicit Parser(const std::string& text) : t(text) {}

  void ws() {
    while (i < t.size() && (t[i] == ' ' || t[i] == '\n' || t[i] == '\r' || t[i] == '\t')) ++i;
  }
  bool eat(char c) {
    ws();
    if (i < t.size() && t[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  bool literal(const char* word) {
    size_t n = std::char_traits<char>::length(word);
    if (t.compare(i, n, word) != 0) return false;
    i += n;
    return true;
  }
  std::string string() {
    std::string out;
    if (!eat('"')) {
      ok = false;
      return out;
    }
    while (i < t.size() && t[i] != '"') {
      char c = t[i++];
      if (c != '\\') {
        out += c;
        continue;
      }
      if (i >= t.size()) break;
      char e = t[i++];
      switch (e) {
        case 'n': out += '\n'; break;
        case 't': out += '\t'; break;
        case 'r': out += '\r'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'u': {
          // Basic-plane code points as UTF-8 (the cache writes none; read for safety).
          if (i + 4 > t.size()) {
            ok = false;
            return out;
          }
          unsigned cp = (unsigned)std::strtoul(t.substr(i, 4).c_str(), nullptr, 16);
          i += 4;
          if (cp < 0x80) {
            out += (char)cp;
          } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
          } else {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
          }
          break;
        }
        default: out += e;  // \" \\ \/
      }
    }
    if (i >= t.size()) ok = false;
    else ++i;  // the closing quote
    return out;
  }
  Json value() {
    Json v;
    ws();
    if (!ok || i >= t.size() || ++depth > 32) {
      ok = false;
      return v;
    }
    const char c = t[i];
    if (c == '{') {
      ++i;
      v.type = Json::Object;
      if (!eat('}')) {
        do {
          ws();
          std::string key = string();
          if (!ok || !eat(':')) {
            ok = false;
            break;
          }
          Json item = value();
          if (!ok) break;
          v.obj.emplace_back(std::move(key), std::move(item));
        } while (eat(','));
        if (ok && !eat('}')) ok = false;
      }
    } else if (c == '[') {
      ++i;
      v.type = Json::Array;
      if (!eat(']')) {
        do {
          Json item = value();
          if (!ok) break;
          v.arr.push_back(std::move(item));
        } while (eat(','));
        if (ok && !eat(']')) ok = false;
      }
    } else if (c == '"') {
      v.type = Json::String;
      v.str = string();
    } else if (literal("true")) {
      v.type = Json::Bool;
      v.b = true;
    } else if (literal("false")) {
      v.type = Json::Bool;
    } else if (literal("null")) {
      v.type = Json::Null;
    } else {
      const char* start = t.c_str() + i;
      char* end = nullptr;
      v.num = std::strtod(start, &end);
      if (end == start) ok = false;
      else {
        v.type = Json::Number;
        i += (size_t)(end - start);
      }
    }
    --depth;
    return v;
  }
};

std::string quoted(const std::string& s) {
  std::string out = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') {
      out += '\\';
      out += c;
    } else if ((unsigned char)c < 0x20) {
      char buf[8];
      std::snprintf(buf, sizeof buf, "\\u%04x", (unsigned)(unsigned char)c);
      out += buf;
    } else {
      out += c;
    }
  }
  return out + "\"";
}

// ------------------------------------------------------------------ the file -------

struct Entry {
  std::string gpu, cls;
  double ms = 0.0;
  TuneChoice choice;
};

std::mutex& file_mutex() {
  static std::mutex mu;
  return mu;
}

// The file's entries under kTuneVersion (none if missing, unreadable, malformed or of
// another version).
std::vector<Entry> read_entries(const std::string& path) {
  std::vector<Entry> out;
  std::ifstream in(path, std::ios::binary);
  if (!in) return out;
  std::stringstream ss;
  ss << in.rdbuf();
  const std::string text = ss.str();
  if (text.size() > (64u << 20)) return out;
  Parser p(text);
  Json root = p.value();
  if (!p.ok || root.type != Json::Object) return out;
  const Json* ver = root.get("version");
  if (!ver || ver->type != Json::Number || (int)ver->num != kTuneVersion) return out;
  const Json* entries = root.get("entries");
  if (!entries || entries->type != Json::Array) return out;
  for (const Json& e : entries->arr) {
    const Json *gpu = e.get("gpu"), *cls = e.get("class"), *choice = e.get("choice"),
               *ms = e.get("ms");
    if (!gpu || gpu->type != Json::String || !cls || cls->type != Json::String || !choice ||
        choice->type != Json::Object)
      continue;
    Entry en;
    en.gpu = gpu->str;
    en.cls = cls->str;
    en.ms = ms && ms->type == Json::Number ? ms->num : 0.0;
    for (const auto& kv : choice->obj)
      if (kv.second.type == Json::String) en.choice[kv.first] = kv.second.str;
    out.push_back(std::move(en));
  }
  return out;
}

bool make_dirs(const std::string& dir) {
  if (dir.empty()) return true;
  struct stat st;
  if (stat(dir.c_str(), &st) == 0) return S_ISDIR(st.st_mode);
  const size_t slash = dir.find_last_of('/');
  if (slash != std::string::npos && slash > 0 && !make_dirs(dir.substr(0, slash))) return false;
  return mkdir(dir.c_str(), 0755) == 0 || errno == EEXIST;
}

}  // namespace

std::string tune_cache_path() {
  if (const char* p = std::getenv("KYTO_GPU_TUNE_CACHE")) {
    if (std::string(p) == "off") return "";
    if (*p) return p;
  }
  if (const char* x = std::getenv("XDG_CACHE_HOME"))
    if (*x) return std::string(x) + "/kyto_b200/tune.json";
  if (const char* h = std::getenv("HOME"))
    if (*h) return std::string(h) + "/.cache/kyto_b200/tune.json";
  return "";
}

bool tune_lookup(const std::string& path, const std::string& gpu, const std::string& cls,
                 TuneChoice& out) {
  if (path.empty()) return false;
  std::lock_guard<std::mutex> lock(file_mutex());
  for (const Entry& e : read_entries(path))
    if (e.gpu == gpu && e.cls == cls) {
      out = e.choice;
      return true;
    }
  return false;
}

bool tune_store(const std::string& path, const std::string& gpu, const std::string& cls,
                const TuneChoice& choice, double ms) {
  if (path.empty()) return false;
  std::lock_guard<std::mutex> lock(file_mutex());
  std::vector<Entry> entries = read_entries(path);
  bool found = false;
  for (Entry& e : entries)
    if (e.gpu == gpu && e.cls == cls) {
      e.choice = choice;
      e.ms = ms;
      found = true;
    }
  if (!found) entries.push_back(Entry{gpu, cls, ms, choice});
  const size_t slash = path.find_last_of('/');
  if (slash != std::string::npos && !make_dirs(path.substr(0, slash))) return false;
  std::ostringstream os;
  os << "{\"version\": " << kTuneVersion << ", \"entries\": [";
  for (size_t i = 0; i < entries.size(); ++i) {
    const Entry& e = entries[i];
    char ms_buf[64];
    std::snprintf(ms_buf, sizeof ms_buf, "%.6g", e.ms);
    os << (i ? ",\n  " : "\n  ") << "{\"gpu\": " << quoted(e.gpu)
       << ", \"class\": " << quoted(e.cls) << ", \"ms\": " << ms_buf << ", \"choice\": {";
    size_t j = 0;
    for (const auto& kv : e.choice)
      os << (j++ ? ", " : "") << quoted(kv.first) << ": " << quoted(kv.second);
    os << "}}";
  }
  os << "\n]}\n";
  const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
  {
    std::ofstream out(tmp, std::ios::binary | std::ios::trunc);
    if (!out) return false;
    out << os.str();
    if (!out.good()) return false;
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) {
    std::remove(tmp.c_str());
    return false;
  }
  return true;
}

std::string tune_gpu_name() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return "unknown";
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
  return std::string(prop.name) + "/sm_" + std::to_string(prop.major) +
         std::to_string(prop.minor) + "/" + std::to_string(prop.multiProcessorCount) + " SMs";
}

}  // namespace kg

using namespace kg;

extern "C" {

// The C ABI (include/kyto_gpu.h): lookups and stores on an explicit file, for tools and
// tests; the library itself uses tune_cache_path().
int kg_tune_lookup(const char* path, const char* gpu, const char* cls, const char* field,
                   char* out, size_t out_len) {
  if (!path || !gpu || !cls || !field || !out || out_len == 0) return -1;
  TuneChoice c;
  if (!tune_lookup(path, gpu, cls, c)) return 0;
  auto it = c.find(field);
  if (it == c.end()) return 0;
  std::snprintf(out, out_len, "%s", it->second.c_str());
  return it->second.size() < out_len ? 1 : -1;
}

int kg_tune_store(const char* path, const char* gpu, const char* cls, const char* keys,
                  const char* values, double ms) {
  if (!path || !gpu || !cls || !keys || !values) return -1;
  // keys and values: ';'-separated, the same count.
  TuneChoice c;
  std::string k(keys), v(values);
  size_t a = 0, b = 0;
  for (;;) {
    const size_t ka = k.find(';', a), vb = v.find(';', b);
    c[k.substr(a, ka == std::string::npos ? std::string::npos : ka - a)] =
        v.substr(b, vb == std::string::npos ? std::string::npos : vb - b);
    if (ka == std::string::npos || vb == std::string::npos) {
      if ((ka == std::string::npos) != (vb == std::string::npos)) return -1;
      break;
    }
    a = ka + 1;
    b = vb + 1;
  }
  return tune_store(path, gpu, cls, c, ms) ? 1 : 0;
}

}  // extern "C"
