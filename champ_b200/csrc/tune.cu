// tune.cu -- autotuning of the engine's launch shapes (host code).
//
// The options that change only the speed of a VMC sweep, never its results beyond rounding --
// "delay_rank", "staged_eval", "move_coop", "orb_coop", and for the tensor-core orbitals of FP32 contexts
// "orbital_tc" and "orbital_tc_chunk" -- are timed one at a time over a few sweeps of the context's own walkers
// (device time from CUDA events on the context's stream), and each keeps its fastest value.  The
// result can be stored in a text file under a key of the system's shape and reused.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/champ_b200.h"
#include "ctx.h"

int champ_fail(int code, const std::string &msg);

namespace {

struct Knob {
  const char *name;
  std::vector<int64_t> values;
};

std::string shape_key(const champ_ctx *c) {
  char b[256];
  snprintf(b, sizeof b, "N=%d C=%d B=%d norb=%d ndet=%d nordc=%d nloc=%d prec=%d W=%d", c->N, c->C, c->nbasis,
           c->norb, c->md.ndet, c->nordc, c->nloc, c->prec, c->W);
  return b;
}

// Device ms of nsweep sweeps, after one untimed sweep.
int time_sweeps(champ_ctx *c, int nsweep, uint64_t seed, uint64_t &sweep, double step, float &ms) {
  int rc = champ_vmc_sweeps(c, 1, seed, sweep++, step, nullptr);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return champ_fail(CHAMP_ECUDA, "cudaEventCreate failed");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return champ_fail(CHAMP_ECUDA, "cudaEventCreate failed");
  }
  cudaEventRecord(e0, c->stream);
  rc = champ_vmc_sweeps(c, nsweep, seed, sweep, step, nullptr);
  sweep += nsweep;
  cudaEventRecord(e1, c->stream);
  if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = champ_fail(CHAMP_ECUDA, "cudaEventSynchronize failed");
  if (!rc) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

bool read_cache(const char *path, const std::string &key, std::string &val) {
  if (!path) return false;
  FILE *f = fopen(path, "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof line, f)) {
    std::string s(line);
    const size_t bar = s.find(" | ");
    if (bar == std::string::npos || s.substr(0, bar) != key) continue;
    val = s.substr(bar + 3);
    while (!val.empty() && (val.back() == '\n' || val.back() == '\r')) val.pop_back();
    found = true;  // the last entry of a key wins
  }
  fclose(f);
  return found;
}

}  // namespace

extern "C" {

int champ_autotune(champ_ctx *c, int32_t nsweep, uint64_t seed, double step, const char *cache_path, char *report,
                   int32_t report_len) {
  if (!c) return champ_fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return champ_fail(CHAMP_ESTATE, "no walkers set");
  if (nsweep < 1) return champ_fail(CHAMP_EINVAL, "nsweep < 1");
  const std::vector<Knob> knobs = {{"delay_rank", {0, 4, 8, 16}}, {"staged_eval", {1, 0}}, {"move_coop", {1, 0}}, {"orb_coop", {1, 0}},
                                   {"orbital_tc", {1, 2}}, {"orbital_tc_chunk", {2, 4, 8}}};
  const std::string key = shape_key(c);
  std::string out, cached;
  if (read_cache(cache_path, key, cached)) {
    // "name=value name=value ...": apply what this context accepts
    size_t p = 0;
    while (p < cached.size()) {
      size_t q = cached.find(' ', p);
      if (q == std::string::npos) q = cached.size();
      const std::string tok = cached.substr(p, q - p);
      const size_t eq = tok.find('=');
      if (eq != std::string::npos) {
        char *end = nullptr;
        const long long v = strtoll(tok.c_str() + eq + 1, &end, 10);
        if (end && *end == '\0') champ_set_option(c, tok.substr(0, eq).c_str(), v);
      }
      p = q + 1;
    }
    out = "cached: " + cached;
  } else {
    uint64_t sweep = 1u << 20;  // sweep numbers away from those of a production run's start
    std::string chosen;
    for (const Knob &k : knobs) {
      int64_t cur;
      if (champ_get_option(c, k.name, &cur)) continue;
      if ((!strcmp(k.name, "orbital_tc") || !strcmp(k.name, "orbital_tc_chunk")) && !c->tc_on) continue;
      if (!strcmp(k.name, "delay_rank") && !c->std_.dly) continue;
      if (!strcmp(k.name, "staged_eval") && !c->std_.el_vj) continue;
      if (!strcmp(k.name, "move_coop") && !c->kfm.lay.coop) continue;
      if (!strcmp(k.name, "orb_coop") && !(c->orb_coop_ok && c->el_staged)) continue;
      int64_t best = cur;
      float best_ms = 1e30f;
      char line[160];
      std::string times;
      for (int64_t v : k.values) {
        if (champ_set_option(c, k.name, v)) continue;
        float ms = 0;
        int rc = time_sweeps(c, nsweep, seed, sweep, step, ms);
        if (rc) return rc;
        snprintf(line, sizeof line, "%s%lld:%.2f", times.empty() ? "" : ",", (long long)v, ms / nsweep);
        times += line;
        if (ms < best_ms) { best_ms = ms; best = v; }
      }
      int rc = champ_set_option(c, k.name, best);
      if (rc) return rc;
      snprintf(line, sizeof line, "%s%s=%lld", chosen.empty() ? "" : " ", k.name, (long long)best);
      chosen += line;
      out += std::string(out.empty() ? "" : "; ") + k.name + " ms/sweep {" + times + "}";
    }
    if (cache_path) {
      FILE *f = fopen(cache_path, "a");
      if (f) {
        fprintf(f, "%s | %s\n", key.c_str(), chosen.c_str());
        fclose(f);
      }
    }
    out = chosen + " (" + out + ")";
  }
  if (report && report_len > 0) {
    strncpy(report, out.c_str(), (size_t)report_len - 1);
    report[report_len - 1] = '\0';
  }
  return CHAMP_OK;
}

}  // extern "C"
