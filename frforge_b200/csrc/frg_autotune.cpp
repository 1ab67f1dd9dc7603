// Persisted autotune table of the 2D stage kernels' tile variants.
//
// frg_autotune times every tile variant of a solve's stage kernel on its own
// state and keeps the fastest.  The table remembers that choice per
// (P, flux, dissipation form, geometry) for the whole process, so solves
// created later start from it without re-timing, and the batched engine runs
// each group with the variant of its key.  It is saved to and loaded from a
// small JSON file:
//
//   {"format": "frforge_b200 autotune table", "version": 1,
//    "entries": [{"p": 3, "flux": "hllc", "av": "br0", "geometry": "affine",
//                 "variant": 0, "ms": 0.284}, ...]}
//
// The reader accepts exactly that shape (keys in any order, unknown keys
// ignored); an entry whose names or numbers are out of range is rejected
// with FRG_ERR_INVALID_ARG and nothing of that file is merged.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "frg_internal.h"

namespace frg {

namespace {

struct Entry {
  int variant;
  double ms;  // measured mean stage time (informational), or NaN
};
using Key = std::tuple<int, int, int, int>;  // p, flux, av (kAv*), curved

std::mutex g_mu;
std::map<Key, Entry> g_table;

const char* kFlux[] = {"rusanov", "hllc"};
const char* kAvName[] = {"none", "br0", "local_dd"};
const char* kGeom[] = {"affine", "curved"};

bool valid_key(int p, int flux, int av, int curved) {
  return p >= 1 && p <= FRG_MAX_NP - 1 && (flux == FRG_FLUX_RUSANOV || flux == FRG_FLUX_HLLC) && av >= kAvNone &&
         av <= kAvDD && (curved == 0 || curved == 1);
}

int name_index(const std::string& v, const char* const* names, int n) {
  for (int i = 0; i < n; ++i)
    if (v == names[i]) return i;
  return -1;
}

// Minimal reader for the table's JSON shape.
struct Reader {
  const char* s;
  size_t i = 0, n;
  explicit Reader(const std::string& t) : s(t.c_str()), n(t.size()) {}
  void ws() {
    while (i < n && std::isspace((unsigned char)s[i])) ++i;
  }
  bool eat(char c) {
    ws();
    if (i < n && s[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  bool str(std::string* out) {
    ws();
    if (i >= n || s[i] != '"') return false;
    ++i;
    out->clear();
    while (i < n && s[i] != '"') {
      if (s[i] == '\\') return false;  // no escapes in this format
      out->push_back(s[i++]);
    }
    if (i >= n) return false;
    ++i;
    return true;
  }
  bool num(double* out) {
    ws();
    char* end = nullptr;
    *out = std::strtod(s + i, &end);
    if (end == s + i) return false;
    i = (size_t)(end - s);
    return true;
  }
  // skip any value (string, number, literal, array, object)
  bool skip() {
    ws();
    if (i >= n) return false;
    if (s[i] == '"') {
      std::string t;
      return str(&t);
    }
    if (s[i] == '{' || s[i] == '[') {
      const char open = s[i], close = open == '{' ? '}' : ']';
      ++i;
      if (eat(close)) return true;
      for (;;) {
        if (open == '{') {
          std::string k;
          if (!str(&k) || !eat(':')) return false;
        }
        if (!skip()) return false;
        if (eat(close)) return true;
        if (!eat(',')) return false;
      }
    }
    while (i < n && (std::isalnum((unsigned char)s[i]) || s[i] == '-' || s[i] == '+' || s[i] == '.')) ++i;
    return true;
  }
};

bool parse_entry(Reader& r, Key* key, Entry* e) {
  if (!r.eat('{')) return false;
  int p = -1, flux = -1, av = -1, curved = -1, variant = -1;
  e->ms = NAN;
  if (!r.eat('}')) {
    for (;;) {
      std::string k;
      if (!r.str(&k) || !r.eat(':')) return false;
      std::string sv;
      double dv = 0.0;
      if (k == "p" || k == "variant" || k == "ms") {
        if (!r.num(&dv)) return false;
        if (k == "p") p = (int)dv;
        if (k == "variant") variant = (int)dv;
        if (k == "ms") e->ms = dv;
        if ((k == "p" || k == "variant") && dv != std::floor(dv)) return false;
      } else if (k == "flux" || k == "av" || k == "geometry") {
        if (!r.str(&sv)) return false;
        if (k == "flux") flux = name_index(sv, kFlux, 2);
        if (k == "av") av = name_index(sv, kAvName, 3);
        if (k == "geometry") curved = name_index(sv, kGeom, 2);
      } else if (!r.skip()) {
        return false;
      }
      if (r.eat('}')) break;
      if (!r.eat(',')) return false;
    }
  }
  if (!valid_key(p, flux, av, curved) || variant < 0 || variant >= stage2d_variants(p + 1)) return false;
  *key = Key{p, flux, av, curved};
  e->variant = variant;
  return true;
}

}  // namespace

int autotune_table_lookup(int p, int flux, int av, int curved, int* variant) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_table.find(Key{p, flux, av, curved});
  if (it == g_table.end()) return 0;
  *variant = it->second.variant;
  return 1;
}

void autotune_table_record(int p, int flux, int av, int curved, int variant, double ms) {
  if (!valid_key(p, flux, av, curved)) return;
  std::lock_guard<std::mutex> lock(g_mu);
  g_table[Key{p, flux, av, curved}] = Entry{variant, ms};
}

}  // namespace frg

using namespace frg;

extern "C" {

int frg_autotune_table_set(int p, int flux, int av, int curved, int variant) {
  if (!valid_key(p, flux, av, curved) || variant < 0 || variant >= stage2d_variants(p + 1))
    return FRG_ERR_INVALID_ARG;
  autotune_table_record(p, flux, av, curved, variant, NAN);
  return FRG_OK;
}

int frg_autotune_table_get(int p, int flux, int av, int curved, int* variant) {
  if (!variant || !valid_key(p, flux, av, curved)) return FRG_ERR_INVALID_ARG;
  return autotune_table_lookup(p, flux, av, curved, variant) ? FRG_OK : FRG_ERR_STATE;
}

int frg_autotune_table_clear(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_table.clear();
  return FRG_OK;
}

int frg_autotune_table_size(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  return (int)g_table.size();
}

int frg_autotune_table_save(const char* path) {
  if (!path) return FRG_ERR_INVALID_ARG;
  std::string out = "{\"format\": \"frforge_b200 autotune table\", \"version\": 1, \"entries\": [";
  {
    std::lock_guard<std::mutex> lock(g_mu);
    bool first = true;
    char buf[256];
    for (const auto& kv : g_table) {
      const Key& k = kv.first;
      const Entry& e = kv.second;
      if (std::isfinite(e.ms))
        std::snprintf(buf, sizeof(buf),
                      "%s\n {\"p\": %d, \"flux\": \"%s\", \"av\": \"%s\", \"geometry\": \"%s\", \"variant\": %d, "
                      "\"ms\": %.6g}",
                      first ? "" : ",", std::get<0>(k), kFlux[std::get<1>(k)], kAvName[std::get<2>(k)],
                      kGeom[std::get<3>(k)], e.variant, e.ms);
      else
        std::snprintf(buf, sizeof(buf),
                      "%s\n {\"p\": %d, \"flux\": \"%s\", \"av\": \"%s\", \"geometry\": \"%s\", \"variant\": %d}",
                      first ? "" : ",", std::get<0>(k), kFlux[std::get<1>(k)], kAvName[std::get<2>(k)],
                      kGeom[std::get<3>(k)], e.variant);
      out += buf;
      first = false;
    }
  }
  out += "\n]}\n";
  FILE* f = std::fopen(path, "w");
  if (!f) return FRG_ERR_INVALID_ARG;
  const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  return (std::fclose(f) == 0 && ok) ? FRG_OK : FRG_ERR_INVALID_ARG;
}

int frg_autotune_table_load(const char* path) {
  if (!path) return FRG_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return FRG_ERR_INVALID_ARG;
  std::string text;
  char buf[4096];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
  std::fclose(f);
  Reader r(text);
  std::vector<std::pair<Key, Entry>> parsed;
  bool have_entries = false;
  if (!r.eat('{')) return FRG_ERR_INVALID_ARG;
  if (!r.eat('}')) {
    for (;;) {
      std::string k;
      if (!r.str(&k) || !r.eat(':')) return FRG_ERR_INVALID_ARG;
      if (k == "entries") {
        have_entries = true;
        if (!r.eat('[')) return FRG_ERR_INVALID_ARG;
        if (!r.eat(']')) {
          for (;;) {
            Key key;
            Entry e;
            if (!parse_entry(r, &key, &e)) return FRG_ERR_INVALID_ARG;
            parsed.emplace_back(key, e);
            if (r.eat(']')) break;
            if (!r.eat(',')) return FRG_ERR_INVALID_ARG;
          }
        }
      } else if (!r.skip()) {
        return FRG_ERR_INVALID_ARG;
      }
      if (r.eat('}')) break;
      if (!r.eat(',')) return FRG_ERR_INVALID_ARG;
    }
  }
  if (!have_entries) return FRG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lock(g_mu);
  for (const auto& kv : parsed) g_table[kv.first] = kv.second;
  return FRG_OK;
}

}  // extern "C"
