// Tuning table of libcucholesky.so: the replacement for the reference's build-time
// autotuner contract (blas/config.c times its kernels and writes include/config.h,
// whose block sizes the drivers compile in, e.g. DGEMM_N_NB in lapack/dpotrf.c:313).
//
// Here the tuned values are a versioned, process-wide table of rows
//   potrf <type S|D|C|Z> <n_min> <sub>
// meaning: ?potrf of order n >= n_min (the largest such n_min of the type wins) uses
// outer blocks of sub diagonal blocks (sub x 128 columns; x 64 for Z), i.e. the
// trailing update's k and the lookahead depth in columns.  The built-in rows below
// were measured on a B200 (sm_100a, 148 SMs) with cuda-cholesky_b200/cucholesky/tune.py,
// which writes the same text format; a file in that format replaces the table at run
// time (cuLAPACKLoadTuning, or the CUCHOLESKY_TUNING environment variable when the
// first handle is created).  The file's first non-comment line must be
// "cucholesky-tuning <version>" with the version this library reads (1).
#pragma once

#include <mutex>

namespace cuchol {

constexpr int kTuningVersion = 1;
constexpr int kMaxSub = 16;

struct TuneRow {
  char type;
  long long n_min;
  int sub;
};

// FP64, B200: outer blocks of 2 / 3 / 4 / 6 / 8 diagonal blocks, measured at
// n = 4096 / 8192 / 16384 / 32768 (best 4.25, 11.22, 56.55, 398.1 ms) and
// split at the geometric midpoints; the other types keep 2 (not measured).
inline std::vector<TuneRow>& tuning_rows() {
  static std::vector<TuneRow> rows = {
      {'D', 0, 2}, {'D', 6144, 3}, {'D', 12288, 4}, {'D', 24576, 6}, {'D', 49152, 8},
      {'S', 0, 2}, {'C', 0, 2}, {'Z', 0, 2},
  };
  return rows;
}

inline std::mutex& tuning_mutex() {
  static std::mutex m;
  return m;
}

// Outer-block size (in diagonal blocks) for ?potrf of order n; 2 when the table has
// no row for the type.
inline int tuned_potrf_sub(char type, long long n) {
  std::lock_guard<std::mutex> lock(tuning_mutex());
  int sub = 2;
  long long best = -1;
  for (const TuneRow& r : tuning_rows())
    if (r.type == type && r.n_min <= n && r.n_min > best) {
      best = r.n_min;
      sub = r.sub;
    }
  return sub;
}

// Parses a tuning file; false (table unchanged) on any malformed line, unknown
// version, or a value out of range.
inline bool load_tuning(const char* path) {
  FILE* f = fopen(path, "r");
  if (f == nullptr) return false;
  std::vector<TuneRow> rows;
  char line[256];
  bool have_version = false, ok = true;
  while (ok && fgets(line, sizeof(line), f) != nullptr) {
    char* p = line;
    while (*p == ' ' || *p == '\t') ++p;
    if (*p == '#' || *p == '\n' || *p == '\r' || *p == '\0') continue;
    if (!have_version) {
      int v = 0;
      ok = (sscanf(p, "cucholesky-tuning %d", &v) == 1 && v == kTuningVersion);
      have_version = true;
      continue;
    }
    char key[32], type = 0;
    long long n_min = -1;
    int sub = 0;
    if (sscanf(p, "%31s %c %lld %d", key, &type, &n_min, &sub) != 4 || strcmp(key, "potrf") != 0 ||
        strchr("SDCZ", type) == nullptr || n_min < 0 || sub < 1 || sub > kMaxSub) {
      ok = false;
      break;
    }
    rows.push_back({type, n_min, sub});
  }
  fclose(f);
  if (!ok || !have_version) return false;
  std::lock_guard<std::mutex> lock(tuning_mutex());
  tuning_rows() = rows;
  return true;
}

}  // namespace cuchol
