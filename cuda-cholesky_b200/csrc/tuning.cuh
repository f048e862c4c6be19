// Tuning table of libcucholesky.so: the replacement for the reference's build-time
// autotuner contract (blas/config.c times its kernels and writes include/config.h,
// whose block sizes the drivers compile in, e.g. DGEMM_N_NB in lapack/dpotrf.c:313).
//
// Here the tuned values are a versioned, process-wide table of rows
//   potrf <type S|D|C|Z> <n_min> <sub>
//   ozaki D <n_min> <sub>
// meaning: ?potrf (or cuDpotrfOzaki) of order n >= n_min (the largest such n_min of the
// routine and type wins) uses outer blocks of sub diagonal blocks (sub x 128 columns;
// x 64 for Z), i.e. the trailing update's k and the lookahead depth in columns.  The
// built-in rows below were measured on a B200 (sm_100a, 148 SMs); the ?potrf rows are
// what cuda-cholesky_b200/cucholesky/tune.py writes, in the same text format, and a
// file in that format replaces the table at run time (cuLAPACKLoadTuning, or the
// CUCHOLESKY_TUNING environment variable when the first handle is created).  The file's
// first non-comment line must be "cucholesky-tuning <version>" with the version this
// library reads (1).
#pragma once

#include <mutex>

namespace cuchol {

constexpr int kTuningVersion = 1;
constexpr int kMaxSub = 16;

enum TuneKey { TUNE_POTRF = 0, TUNE_OZAKI = 1 };

struct TuneRow {
  int key;
  char type;
  long long n_min;
  int sub;
};

// FP64 ?potrf, B200, rows from tune.py with the 64 x 64-tile DMMA updates: outer
// blocks of 2 / 2 / 5 / 8 diagonal blocks at n = 4096 / 8192 / 16384 / 32768 (best
// 3.99, 10.78, 54.33, 382.6 ms; at 16384 the other widths gave 57.1 (2), 55.3 (3),
// 54.8 (4), 54.4 (6), 54.9 (8)), split at the geometric midpoints.  C: the rows tune.py wrote from n = 4096 / 8192 / 16384 (best
// cpotrf 7.34 / 29.82 / 196.8 ms; outer block 2 gave 208.5 ms at n = 16384).  Z on
// the complex FP64 tensor-core engine: best 9.93 / 37.56 / 223.9 ms with 2 / 6 / 12
// (outer block 2 gave 293.5 ms at 16384).  S on the split TF32 tensor-core updates:
// flat in the width up to n = 8192 (2.78 / 6.09 ms), best 4 at 16384 (16.69 ms; 1
// gave 22.37) and within 1% of the best at 32768 (88.74 ms).
// cuDpotrfOzaki: 8 (1024 columns) below n = 49152, 16 from there on (n = 8192 / 32768 /
// 65536: 10.8 / 255 / 2028 ms with 8; 11.7 / 255 / 1926 ms with 16; 4 gave 282 ms and
// 2344 ms at the two larger orders).
inline std::vector<TuneRow>& tuning_rows() {
  static std::vector<TuneRow> rows = {
      {TUNE_POTRF, 'D', 0, 2}, {TUNE_POTRF, 'D', 11585, 5}, {TUNE_POTRF, 'D', 23170, 8},
      {TUNE_POTRF, 'S', 0, 2}, {TUNE_POTRF, 'S', 11585, 4},
      {TUNE_POTRF, 'C', 0, 2}, {TUNE_POTRF, 'C', 5793, 3}, {TUNE_POTRF, 'C', 11585, 6},
      {TUNE_POTRF, 'Z', 0, 2}, {TUNE_POTRF, 'Z', 5793, 6}, {TUNE_POTRF, 'Z', 11585, 12},
      {TUNE_OZAKI, 'D', 0, 8}, {TUNE_OZAKI, 'D', 49152, 16},
  };
  return rows;
}

inline std::mutex& tuning_mutex() {
  static std::mutex m;
  return m;
}

// Outer-block size (in diagonal blocks) for the routine `key` of order n; when the
// table has no row for it, 2 for ?potrf and 8 for the Ozaki factor.
inline int tuned_sub(int key, char type, long long n) {
  std::lock_guard<std::mutex> lock(tuning_mutex());
  int sub = (key == TUNE_OZAKI) ? 8 : 2;
  long long best = -1;
  for (const TuneRow& r : tuning_rows())
    if (r.key == key && r.type == type && r.n_min <= n && r.n_min > best) {
      best = r.n_min;
      sub = r.sub;
    }
  return sub;
}
inline int tuned_potrf_sub(char type, long long n) { return tuned_sub(TUNE_POTRF, type, n); }

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
    const bool ozaki = sscanf(p, "%31s", key) == 1 && strcmp(key, "ozaki") == 0;
    if (sscanf(p, "%31s %c %lld %d", key, &type, &n_min, &sub) != 4 ||
        (strcmp(key, "potrf") != 0 && !ozaki) || strchr(ozaki ? "D" : "SDCZ", type) == nullptr || n_min < 0 ||
        sub < 1 || sub > kMaxSub) {
      ok = false;
      break;
    }
    rows.push_back({ozaki ? TUNE_OZAKI : TUNE_POTRF, type, n_min, sub});
  }
  fclose(f);
  if (!ok || !have_version) return false;
  std::lock_guard<std::mutex> lock(tuning_mutex());
  tuning_rows() = rows;
  return true;
}

}  // namespace cuchol
