// tune.cu -- the autotuner's table of chosen FFT plans.
//
// Every transform length has one or more candidate plans (plans_gen.h:
// radix lists and, for the strided line pass, the column tile); candidate 0
// is the generator's heuristic choice.  The first job that needs a length on
// a device times the candidates of each pass kind on a synthetic volume of
// that length (engine.cu, tune_measure) and records the fastest here.  This
// is the analogue of deconwolf's FFTW planning by measurement (fft_train,
// src/fft.c:206-319, FFTW_MEASURE by default, src/dw.c:400) and of its
// wisdom files (fftwf_import/export_wisdom_from/to_filename, src/fft.c:
// 299-316 and 355): the table can be written to a text file and read back, so a
// later process skips the measurements.
//
// Selection: the fastest candidate wins only if it beats candidate 0 by
// more than the margin (2 %); within the margin the heuristic's plan stays,
// so run-to-run noise does not flip plans.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/dwcu.h"
#include "plans_gen.h"

namespace dwcu {
void record_error(const char *msg);

namespace {

struct Entry {
    int cand = 0;
    std::vector<float> ms;  // per candidate; empty when imported or forced
    int source = 0;         // 0 measured, 1 imported, 2 forced
};

std::mutex g_mu;
// (device, kind, n) -> entry; device -1: every device (imported or forced)
std::map<std::tuple<int, int, int>, Entry> g_table;
int g_mode = -1;  // -1: not yet read from the environment
constexpr float kMargin = 0.02f;

int mode_locked()
{
    if (g_mode < 0) {
        const char *e = std::getenv("DWCU_AUTOTUNE");
        g_mode = (e && e[0] == '0') ? DWCU_TUNE_OFF : DWCU_TUNE_MEASURE;
    }
    return g_mode;
}

int err(int code, const char *msg)
{
    record_error(msg);
    return code;
}

const char *kind_name(int kind) { return kind == DWCU_PLAN_LINES ? "lines" : kind == DWCU_PLAN_Y ? "y" : "x"; }

int kind_of(const char *s)
{
    if (!strcmp(s, "lines")) return DWCU_PLAN_LINES;
    if (!strcmp(s, "y")) return DWCU_PLAN_Y;
    if (!strcmp(s, "x")) return DWCU_PLAN_X;
    return -1;
}

}  // namespace

int tune_plan_count(int kind, int n)
{
    int c = 0;
    if (kind == DWCU_PLAN_LINES) {
        for (const auto &p : kLinesPlans) c += (p.n == n);
    } else if (kind == DWCU_PLAN_Y) {
        for (const auto &p : kYPlans) c += (p.n == n);
    } else if (kind == DWCU_PLAN_X) {
        for (const auto &p : kXPlans) c += (p.n == n);
    }
    return c;
}

int tune_mode()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return mode_locked();
}

float tune_margin() { return kMargin; }

// the chosen candidate of (device, kind, n), or -1 when none is recorded
int tune_lookup(int device, int kind, int n)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find({device, kind, n});
    if (it == g_table.end()) it = g_table.find({-1, kind, n});
    return it == g_table.end() ? -1 : it->second.cand;
}

void tune_record(int device, int kind, int n, const std::vector<float> &ms, int cand)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Entry &e = g_table[{device, kind, n}];
    e.cand = cand;
    e.ms = ms;
    e.source = 0;
}

// index of the fastest finite time; candidate 0 unless the fastest beats it
// by more than `margin` (relative).  Non-finite or negative times are
// candidates that could not run.
int tune_select_idx(const float *ms, int n, float margin)
{
    int best = -1;
    for (int i = 0; i < n; ++i) {
        if (!std::isfinite(ms[i]) || ms[i] < 0.f) continue;
        if (best < 0 || ms[i] < ms[best]) best = i;
    }
    if (best <= 0) return 0;
    if (std::isfinite(ms[0]) && ms[0] >= 0.f && !(ms[best] < ms[0] * (1.f - margin))) return 0;
    return best;
}

}  // namespace dwcu

using namespace dwcu;

extern "C" {

int dwcu_tune_set_mode(int32_t mode)
{
    if (mode != DWCU_TUNE_OFF && mode != DWCU_TUNE_MEASURE) return err(DWCU_ERROR_INVALID_VALUE, "bad tuning mode");
    std::lock_guard<std::mutex> lk(g_mu);
    g_mode = mode;
    return DWCU_SUCCESS;
}

int dwcu_tune_get_mode(int32_t *mode)
{
    if (!mode) return err(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    *mode = tune_mode();
    return DWCU_SUCCESS;
}

int dwcu_tune_select(const float *ms, int32_t n, float margin, int32_t *choice)
{
    if (!ms || !choice || n < 1) return err(DWCU_ERROR_INVALID_VALUE, "bad arguments");
    *choice = tune_select_idx(ms, n, margin);
    return DWCU_SUCCESS;
}

int dwcu_tune_plan_count(int32_t kind, int32_t n, int32_t *count)
{
    if (!count) return err(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (kind < DWCU_PLAN_LINES || kind > DWCU_PLAN_X) return err(DWCU_ERROR_INVALID_VALUE, "bad plan kind");
    *count = tune_plan_count(kind, n);
    return DWCU_SUCCESS;
}

int dwcu_tune_plan_info(int32_t kind, int32_t n, int32_t cand, int32_t *radices, int32_t *tile)
{
    if (!radices || !tile) return err(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    auto set = [&](int a, int b, int c, int t) {
        radices[0] = a;
        radices[1] = b;
        radices[2] = c;
        *tile = t;
        return DWCU_SUCCESS;
    };
    if (kind == DWCU_PLAN_LINES) {
        for (const auto &p : kLinesPlans)
            if (p.n == n && p.cand == cand) return set(p.ra, p.rb, p.rc, p.T);
    } else if (kind == DWCU_PLAN_Y) {
        for (const auto &p : kYPlans)
            if (p.n == n && p.cand == cand) return set(p.ra, p.rb, p.rc, KB);
    } else if (kind == DWCU_PLAN_X) {
        for (const auto &p : kXPlans)
            if (p.n == n && p.cand == cand) return set(p.ra, p.rb, p.rc, p.R);
    }
    return err(DWCU_ERROR_INVALID_VALUE, "no such plan");
}

int dwcu_tune_force(int32_t kind, int32_t n, int32_t cand)
{
    if (kind < DWCU_PLAN_LINES || kind > DWCU_PLAN_X) return err(DWCU_ERROR_INVALID_VALUE, "bad plan kind");
    std::lock_guard<std::mutex> lk(g_mu);
    if (cand < 0) {
        // forget this length everywhere: the next job measures again
        for (auto it = g_table.begin(); it != g_table.end();) {
            if (std::get<1>(it->first) == kind && std::get<2>(it->first) == n)
                it = g_table.erase(it);
            else
                ++it;
        }
        return DWCU_SUCCESS;
    }
    if (cand >= tune_plan_count(kind, n)) return err(DWCU_ERROR_INVALID_VALUE, "no such candidate");
    for (auto it = g_table.begin(); it != g_table.end();) {
        if (std::get<1>(it->first) == kind && std::get<2>(it->first) == n)
            it = g_table.erase(it);
        else
            ++it;
    }
    Entry &e = g_table[{-1, kind, n}];
    e.cand = cand;
    e.source = 2;
    return DWCU_SUCCESS;
}

int dwcu_tune_query(int32_t device, int32_t kind, int32_t n, int32_t *cand, float *ms, int32_t cap, int32_t *nms)
{
    if (!cand) return err(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_table.find({device, kind, n});
    if (it == g_table.end()) it = g_table.find({-1, kind, n});
    *cand = -1;
    if (nms) *nms = 0;
    if (it == g_table.end()) return DWCU_SUCCESS;
    *cand = it->second.cand;
    const int k = (int) it->second.ms.size();
    if (nms) *nms = k;
    for (int i = 0; ms && i < k && i < cap; ++i) ms[i] = it->second.ms[(size_t) i];
    return DWCU_SUCCESS;
}

int dwcu_tune_clear(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_table.clear();
    return DWCU_SUCCESS;
}

// text format, one line per length:  <kind> <n> <cand> [<ms of each candidate> ...]
int dwcu_tune_export(const char *path)
{
    if (!path) return err(DWCU_ERROR_INVALID_VALUE, "NULL path");
    std::lock_guard<std::mutex> lk(g_mu);
    FILE *f = fopen(path, "w");
    if (!f) return err(DWCU_ERROR_IO, "cannot open the tuning file for writing");
    fprintf(f, "# dwcu plan table v1: kind length candidate [ms per candidate]\n");
    // one line per (kind, n): a device's measurement, else the any-device entry
    std::map<std::pair<int, int>, const Entry *> rows;
    for (const auto &kv : g_table) {
        const auto key = std::make_pair(std::get<1>(kv.first), std::get<2>(kv.first));
        auto it = rows.find(key);
        if (it == rows.end() || (it->second->ms.empty() && !kv.second.ms.empty())) rows[key] = &kv.second;
    }
    for (const auto &kv : rows) {
        fprintf(f, "%s %d %d", kind_name(kv.first.first), kv.first.second, kv.second->cand);
        for (float v : kv.second->ms) fprintf(f, " %.6g", (double) v);
        fprintf(f, "\n");
    }
    const bool ok = ferror(f) == 0;
    fclose(f);
    return ok ? DWCU_SUCCESS : err(DWCU_ERROR_IO, "writing the tuning file failed");
}

int dwcu_tune_import(const char *path)
{
    if (!path) return err(DWCU_ERROR_INVALID_VALUE, "NULL path");
    FILE *f = fopen(path, "r");
    if (!f) return err(DWCU_ERROR_IO, "cannot open the tuning file");
    char line[1024];
    std::vector<std::tuple<int, int, int>> rows;
    int rc = DWCU_SUCCESS;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        char kind[16];
        int n = 0, cand = 0;
        if (sscanf(line, "%15s %d %d", kind, &n, &cand) != 3 || kind_of(kind) < 0) {
            rc = err(DWCU_ERROR_INVALID_VALUE, "malformed line in the tuning file");
            break;
        }
        const int k = kind_of(kind);
        if (cand < 0 || cand >= tune_plan_count(k, n)) {
            rc = err(DWCU_ERROR_INVALID_VALUE, "the tuning file names a plan this library does not have");
            break;
        }
        rows.emplace_back(k, n, cand);
    }
    fclose(f);
    if (rc != DWCU_SUCCESS) return rc;  // nothing applied
    std::lock_guard<std::mutex> lk(g_mu);
    for (const auto &r : rows) {
        Entry &e = g_table[{-1, std::get<0>(r), std::get<1>(r)}];
        e.cand = std::get<2>(r);
        e.ms.clear();
        e.source = 1;
    }
    return DWCU_SUCCESS;
}

}  // extern "C"
