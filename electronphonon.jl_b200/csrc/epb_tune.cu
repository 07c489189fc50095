// Tuning table of the autotuner: measured choices keyed by shape, kept in the context and exportable
// as text so that a production run can skip the timing trials (load the table once, the pass then
// reads its choices instead of timing candidates).
//
// The choices replace the reference's fixed crossovers -- `_FUSED_ROT_MAX_NWNM`
// (src/wannier_to_bloch_batched.jl:406: fused rotation kernel below nw*nm = 24, two cuBLAS batched
// GEMMs above) and `_FUSED_RQKQ_MAX_NW2NM` (ext/ElectronPhononCUDAExt.jl:214) -- by timings of the
// candidates on the caller's own shapes:
//   pass_kb/<nw>/<nm>/<nq>/<prec>    inner k batch of epb_eph_pass (4, 8, 16, 32)
//   pass_rot/<nw>/<nm>/<nq>/<prec>   rotation kernel of the mixed pass (0 warp tensor cores, 1 FP32)
//   pass_kq/<nw>/<nm>/<nq>/<prec>    kR->kq GEMM form (1 A-resident, 0 streamed operands)
//   eigh_varlen/<lo>/<hi>/<prec>     kernel of the uneven-eigensolve class (lo, hi] (1 the L2-scratch
//                                    instance for the class, 0 the shared-memory / 512-thread solver)
// Text form: one "key value" pair per line; '#' starts a comment line; keys are printable ASCII without
// spaces, at most 120 characters.
#include <cctype>
#include <cstdio>
#include <cstring>
#include <string>

#include "epb_common.cuh"

struct epb_tune_table {
  std::vector<std::pair<std::string, int64_t>> kv;
};

namespace epb {

bool tune_lookup(const std::vector<std::pair<std::string, int64_t>>& kv, const std::string& key, int64_t* value) {
  for (const auto& e : kv)
    if (e.first == key) {
      *value = e.second;
      return true;
    }
  return false;
}

void tune_store(std::vector<std::pair<std::string, int64_t>>& kv, const std::string& key, int64_t value) {
  for (auto& e : kv)
    if (e.first == key) {
      e.second = value;
      return;
    }
  kv.emplace_back(key, value);
}

static bool valid_key(const char* k) {
  const size_t n = strlen(k);
  if (n == 0 || n > 120) return false;
  for (size_t i = 0; i < n; ++i)
    if (!isgraph((unsigned char)k[i])) return false;
  return true;
}

}  // namespace epb

using namespace epb;

extern "C" {

int epb_tune_table_create(epb_tune_table** out) {
  clear_error();
  EPB_CHECK_ARG(out, "epb_tune_table_create: NULL pointer");
  *out = new epb_tune_table();
  return EPB_OK;
}

int epb_tune_table_destroy(epb_tune_table* t) {
  delete t;
  return EPB_OK;
}

int epb_tune_table_set(epb_tune_table* t, const char* key, int64_t value) {
  clear_error();
  EPB_CHECK_ARG(t && key && valid_key(key), "epb_tune_table_set: bad table or key");
  tune_store(t->kv, key, value);
  return EPB_OK;
}

int epb_tune_table_get(const epb_tune_table* t, const char* key, int64_t* value, int* found) {
  clear_error();
  EPB_CHECK_ARG(t && key && value && found, "epb_tune_table_get: NULL argument");
  *found = tune_lookup(t->kv, key, value) ? 1 : 0;
  return EPB_OK;
}

int epb_tune_table_size(const epb_tune_table* t, int64_t* n) {
  clear_error();
  EPB_CHECK_ARG(t && n, "epb_tune_table_size: NULL argument");
  *n = (int64_t)t->kv.size();
  return EPB_OK;
}

// Text of the table into buf (cap bytes, NUL-terminated); *len = bytes needed without the NUL. With
// cap too small nothing is written and EPB_ERR_ARG is returned (call again with *len + 1 bytes).
int epb_tune_table_serialize(const epb_tune_table* t, char* buf, int64_t cap, int64_t* len) {
  clear_error();
  EPB_CHECK_ARG(t && len, "epb_tune_table_serialize: NULL argument");
  std::string s;
  for (const auto& e : t->kv) {
    char line[160];
    snprintf(line, sizeof(line), "%s %lld\n", e.first.c_str(), (long long)e.second);
    s += line;
  }
  *len = (int64_t)s.size();
  EPB_CHECK_ARG(buf && cap > *len, "epb_tune_table_serialize: buffer of %lld bytes, %lld needed", (long long)cap,
                (long long)(*len + 1));
  memcpy(buf, s.c_str(), s.size() + 1);
  return EPB_OK;
}

// Add the pairs of `text` (the serialize format) to the table; a malformed line rejects the whole
// text and leaves the table unchanged.
int epb_tune_table_parse(epb_tune_table* t, const char* text) {
  clear_error();
  EPB_CHECK_ARG(t && text, "epb_tune_table_parse: NULL argument");
  std::vector<std::pair<std::string, int64_t>> add;
  const char* p = text;
  int line_no = 0;
  while (*p) {
    const char* e = strchr(p, '\n');
    std::string line(p, e ? (size_t)(e - p) : strlen(p));
    p = e ? e + 1 : p + line.size();
    ++line_no;
    size_t a = line.find_first_not_of(" \t\r");
    if (a == std::string::npos || line[a] == '#') continue;
    char key[128];
    long long v = 0;
    char extra[2];
    const int got = sscanf(line.c_str() + a, "%127s %lld %1s", key, &v, extra);
    EPB_CHECK_ARG(got == 2 && valid_key(key), "epb_tune_table_parse: line %d is not 'key value'", line_no);
    add.emplace_back(key, (int64_t)v);
  }
  for (const auto& kv : add) tune_store(t->kv, kv.first, kv.second);
  return EPB_OK;
}

// The context's measured choices into `t` (added / overwritten), and a table's choices into the context
// (later passes of those shapes use them instead of timing).
int epb_tune_export(epb_ctx* ctx, epb_tune_table* t) {
  clear_error();
  EPB_CHECK_ARG(ctx && t, "epb_tune_export: NULL argument");
  for (const auto& kv : ctx->tuned) tune_store(t->kv, kv.first, kv.second);
  return EPB_OK;
}

int epb_tune_import(epb_ctx* ctx, const epb_tune_table* t) {
  clear_error();
  EPB_CHECK_ARG(ctx && t, "epb_tune_import: NULL argument");
  for (const auto& kv : t->kv) tune_store(ctx->tuned, kv.first, kv.second);
  return EPB_OK;
}

}  // extern "C"
