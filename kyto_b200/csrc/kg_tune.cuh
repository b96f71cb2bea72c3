// The tuner's persistent cache (kg_tune.cu): choices that cannot change a result (the
// kNN filter's operand kind and query-operand mode), keyed by (GPU, shape class) in a
// versioned JSON file.
#pragma once

#include <map>
#include <string>

namespace kg {

// Bumped whenever a kernel the cached choices pick between changes: entries written
// under another version are ignored (and dropped at the next store).
constexpr int kTuneVersion = 1;

using TuneChoice = std::map<std::string, std::string>;

// The cache file: KYTO_GPU_TUNE_CACHE, else $XDG_CACHE_HOME/kyto_b200/tune.json, else
// $HOME/.cache/kyto_b200/tune.json; empty when KYTO_GPU_TUNE_CACHE is "off" (no cache:
// every process tunes once in memory).
std::string tune_cache_path();

// The cached choice for (gpu, class) in the file at `path` (false: none, the file is
// missing or unreadable, or written under another version).
bool tune_lookup(const std::string& path, const std::string& gpu, const std::string& cls,
                 TuneChoice& out);

// Records (gpu, class) -> choice (with the measured cost, ms) in the file at `path`,
// replacing an earlier entry for the same key; the file is rewritten whole through a
// temporary and a rename, under a process-wide lock. Returns false if it could not be
// written (the choice then lives only in memory).
bool tune_store(const std::string& path, const std::string& gpu, const std::string& cls,
                const TuneChoice& choice, double ms);

// "<device name>/sm_<major><minor>/<SMs> SMs" of the current device.
std::string tune_gpu_name();

}  // namespace kg
