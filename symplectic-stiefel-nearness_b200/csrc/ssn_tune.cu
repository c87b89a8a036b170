// ssn_tune.cu -- the autotuned launch-parameter table (ssn_set_tuning).
//
// The table maps a problem class (precision form, m, ranges of n and batch) to
// launch parameters that replace the built-in rules: the FP64 Gram's row splits,
// the split-form Gram's row chunks, the split-form recovery's row-tile parts and
// the Newton kernels' CTAs per instance.  ssn_solve looks its class up once and
// makes the entry the calling thread's active tuning while it enqueues, so every
// rule consults the same entry (and ssn_workspace_bytes sizes with it).
#include <mutex>
#include <vector>

#include "ssn_internal.h"

namespace ssn {

namespace {

constexpr int kMaxEntries = 1024;

std::mutex& table_mutex() {
  static std::mutex mu;
  return mu;
}
std::vector<ssn_tuning>& table() {
  static std::vector<ssn_tuning> t;
  return t;
}

thread_local const ssn_tuning* t_active = nullptr;

bool entry_ok(const ssn_tuning& e) {
  const bool prec = e.precision == SSN_PRECISION_FP64 || e.precision == SSN_PRECISION_SPLIT;
  return prec && e.m >= 2 && e.m <= 128 && (e.m % 2) == 0 && e.n_min >= 1 && e.n_max >= e.n_min &&
         e.batch_min >= 1 && e.batch_max >= e.batch_min && e.gram_splits >= 0 && e.gram_splits <= 64 &&
         e.gram_chunks >= 0 && e.gram_chunks <= 32 && e.recover_parts >= 0 && e.recover_parts <= 1024 &&
         (e.cluster == 0 || e.cluster == 1 || (e.cluster == 2 && e.m > 32));
}

}  // namespace

const ssn_tuning* active_tuning() { return t_active; }

const ssn_tuning* find_tuning(int precision, int n, int m, int batch) {
  // entries are only replaced wholesale by ssn_set_tuning, which callers do not run
  // concurrently with solves; the returned pointer stays valid until the next call
  const std::vector<ssn_tuning>& t = table();
  for (const ssn_tuning& e : t)
    if (e.precision == precision && e.m == m && n >= e.n_min && n <= e.n_max && batch >= e.batch_min &&
        batch <= e.batch_max)
      return &e;
  return nullptr;
}

TuningScope::TuningScope(const ssn_tuning* t) : prev(t_active) { t_active = t; }
TuningScope::~TuningScope() { t_active = prev; }

}  // namespace ssn

extern "C" {

int ssn_set_tuning(const ssn_tuning* entries, int count) {
  if (count < 0 || count > ssn::kMaxEntries || (count > 0 && !entries)) return SSN_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < count; ++i)
    if (!ssn::entry_ok(entries[i])) return SSN_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ssn::table_mutex());
  ssn::table().assign(entries, entries + count);
  return SSN_OK;
}

int ssn_get_tuning(ssn_tuning* entries, int capacity) {
  std::lock_guard<std::mutex> lock(ssn::table_mutex());
  const std::vector<ssn_tuning>& t = ssn::table();
  const int n = static_cast<int>(t.size());
  if (entries)
    for (int i = 0; i < n && i < capacity; ++i) entries[i] = t[i];
  return n;
}

}  // extern "C"
