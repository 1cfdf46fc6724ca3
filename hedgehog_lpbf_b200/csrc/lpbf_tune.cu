// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Autotuner of the batched process map and its JSON cache.
//
// The tunables are the rows per task of each size class (the tile is 120
// owned columns by `rows` rows), the temporal depth, the CTAs per SM of the
// persistent grid and the row staging (bulk copies or tensor maps).  They
// are chosen by timing short runs of the batch kernel, with CUDA events, on
// a subset of the caller's scenarios (their own grids and plans, fields
// filled with T_amb in scratch memory the tuner allocates and frees):
//   1. per size class present, rows in {12, 24, 48, 96, 192, 384}, timed on
//      all classes' subsets together (the classes share the launches, so a
//      class's best rows depend on the others' work beside it), one class
//      after another from (24, 48, 96, 192) at depth 2;
//   2. on all subsets together, depth in {2, 3, 4} x CTAs per SM in
//      {all, all - 1} x staging in {bulk, maps}, with the rows of step 1.
// The winner is stored in a JSON file under a key made of the GPU's name,
// its SM count and the batch's size-class histogram (counts rounded up to a
// power of two), so a later batch of the same shape reuses it:
//   {"version": 1, "entries": {"<key>": {"depth": 3, "ctas_per_sm": 0,
//     "staging": 1, "rows": [24, 48, 48, 96], "gcells": 241.5}, ...}}
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "lpbf_batch.hpp"
#include "lpbf_host.hpp"
#include "lpbf_b200.h"

namespace lpbf_b200 {
namespace {

__global__ void fill_kernel(double* p, size_t n, double v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// ---- JSON cache (the flat format above) ---------------------------------------

std::string read_file(const char* path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return std::string();
    std::stringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

size_t skip_ws(const std::string& s, size_t i) {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) ++i;
    return i;
}

// Parse a JSON string starting at s[i] == '"'; returns the index after it.
size_t parse_string(const std::string& s, size_t i, std::string* out) {
    if (i >= s.size() || s[i] != '"') return std::string::npos;
    std::string r;
    for (++i; i < s.size(); ++i) {
        if (s[i] == '\\' && i + 1 < s.size()) { r.push_back(s[++i]); continue; }
        if (s[i] == '"') { *out = r; return i + 1; }
        r.push_back(s[i]);
    }
    return std::string::npos;
}

// Index after the balanced {...} starting at s[i] == '{' (strings respected).
size_t match_object(const std::string& s, size_t i) {
    int depth = 0;
    for (; i < s.size(); ++i) {
        if (s[i] == '"') {
            std::string tmp;
            i = parse_string(s, i, &tmp);
            if (i == std::string::npos) return i;
            --i;
        } else if (s[i] == '{') {
            ++depth;
        } else if (s[i] == '}') {
            if (--depth == 0) return i + 1;
        }
    }
    return std::string::npos;
}

// key -> raw object text of the "entries" member; false on malformed text.
bool parse_entries(const std::string& s, std::map<std::string, std::string>* out) {
    out->clear();
    if (s.find_first_not_of(" \n\r\t") == std::string::npos) return true;   // empty file
    const size_t e = s.find("\"entries\"");
    if (e == std::string::npos) return false;
    size_t i = s.find(':', e);
    if (i == std::string::npos) return false;
    i = skip_ws(s, i + 1);
    if (i >= s.size() || s[i] != '{') return false;
    const size_t end = match_object(s, i);
    if (end == std::string::npos) return false;
    ++i;
    for (;;) {
        i = skip_ws(s, i);
        if (i >= end - 1) break;
        if (s[i] == ',') { ++i; continue; }
        std::string key;
        i = parse_string(s, i, &key);
        if (i == std::string::npos) return false;
        i = skip_ws(s, i);
        if (i >= s.size() || s[i] != ':') return false;
        i = skip_ws(s, i + 1);
        if (i >= s.size() || s[i] != '{') return false;
        const size_t oe = match_object(s, i);
        if (oe == std::string::npos || oe > end) return false;
        (*out)[key] = s.substr(i, oe - i);
        i = oe;
    }
    return true;
}

bool get_number(const std::string& obj, const char* name, double* v) {
    const std::string pat = std::string("\"") + name + "\"";
    const size_t k = obj.find(pat);
    if (k == std::string::npos) return false;
    size_t i = obj.find(':', k + pat.size());
    if (i == std::string::npos) return false;
    i = skip_ws(obj, i + 1);
    char* endp = nullptr;
    const double x = std::strtod(obj.c_str() + i, &endp);
    if (endp == obj.c_str() + i) return false;
    *v = x;
    return true;
}

bool get_rows(const std::string& obj, int rows[4]) {
    const size_t k = obj.find("\"rows\"");
    if (k == std::string::npos) return false;
    size_t i = obj.find('[', k);
    if (i == std::string::npos) return false;
    ++i;
    for (int c = 0; c < 4; ++c) {
        i = skip_ws(obj, i);
        char* endp = nullptr;
        const long x = std::strtol(obj.c_str() + i, &endp, 10);
        if (endp == obj.c_str() + i) return false;
        rows[c] = (int)x;
        i = skip_ws(obj, (size_t)(endp - obj.c_str()));
        if (c < 3) {
            if (i >= obj.size() || obj[i] != ',') return false;
            ++i;
        }
    }
    return true;
}

std::string escape(const std::string& k) {
    std::string r;
    for (char ch : k) {
        if (ch == '"' || ch == '\\') r.push_back('\\');
        r.push_back(ch);
    }
    return r;
}

std::string entry_text(const lpbf_b200_batch_opts& o, double gcells) {
    char buf[256];
    std::snprintf(buf, sizeof(buf),
                  "{\"depth\": %d, \"ctas_per_sm\": %d, \"staging\": %d, "
                  "\"rows\": [%d, %d, %d, %d], \"gcells\": %.3f}",
                  o.depth, o.ctas_per_sm, o.staging, o.rows[0], o.rows[1], o.rows[2], o.rows[3],
                  gcells);
    return buf;
}

bool write_entries(const char* path, const std::map<std::string, std::string>& ent) {
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) return false;
        f << "{\"version\": 1, \"entries\": {";
        bool first = true;
        for (const auto& kv : ent) {
            f << (first ? "\n  " : ",\n  ") << '"' << escape(kv.first) << "\": " << kv.second;
            first = false;
        }
        f << "\n}}\n";
        if (!f) return false;
    }
    return std::rename(tmp.c_str(), path) == 0;
}

// ---- trials -------------------------------------------------------------------

struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch() { for (void* p : ptrs) cudaFree(p); }
    void* get(size_t bytes) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return p;
    }
};

// GCell-updates/s of `sub` under `o` over `steps` steps (graph replay; the
// first run captures and warms up).  0 on failure.
double trial(const std::vector<lpbf_b200_scenario>& sub, int steps, const lpbf_b200_batch_opts& o,
             cudaStream_t s) {
    const size_t wb = lpbf_b200_batch_workspace_bytes(sub.data(), (int)sub.size(), steps, &o);
    if (wb == 0) return 0.0;
    void* work = nullptr;
    if (cudaMalloc(&work, wb) != cudaSuccess) return 0.0;
    lpbf_b200_batch* b = nullptr;
    double g = 0.0;
    if (lpbf_b200_batch_create(sub.data(), (int)sub.size(), steps, &o, work, wb, s, &b) ==
        LPBF_OK) {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        bool ok = lpbf_b200_batch_run(b, 0, steps, 1, s) == LPBF_OK;
        float best = 1e30f;
        for (int r = 0; r < 2 && ok; ++r) {
            cudaEventRecord(e0, s);
            ok = lpbf_b200_batch_run(b, 0, steps, 1, s) == LPBF_OK;
            cudaEventRecord(e1, s);
            ok = ok && cudaEventSynchronize(e1) == cudaSuccess;
            float ms = 0.f;
            if (ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) best = std::min(best, ms);
        }
        unsigned int err = 1;
        ok = ok && lpbf_b200_batch_read_error(b, s, &err) == LPBF_OK && err == 0;
        if (ok && best < 1e29f) {
            double cells = 0.0;
            for (const auto& sc : sub) cells += (double)sc.k->nx * sc.k->ny;
            g = cells * steps / (best * 1e-3) / 1e9;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        lpbf_b200_batch_destroy(b);
    }
    cudaFree(work);
    return g;
}

}  // namespace
}  // namespace lpbf_b200

using namespace lpbf_b200;

extern "C" {

int lpbf_b200_tune_cache_get(const char* path, const char* key, lpbf_b200_batch_opts* out) {
    if (!path || !key || !out) return LPBF_ERR_ARG;
    std::map<std::string, std::string> ent;
    if (!parse_entries(read_file(path), &ent)) return LPBF_ERR_ARG;
    const auto it = ent.find(key);
    if (it == ent.end()) return 1;
    double d = 0, c = 0, st = 0;
    int rows[4];
    if (!get_number(it->second, "depth", &d) || !get_number(it->second, "ctas_per_sm", &c) ||
        !get_number(it->second, "staging", &st) || !get_rows(it->second, rows))
        return LPBF_ERR_ARG;
    lpbf_b200_batch_opts o;
    std::memset(&o, 0, sizeof(o));
    o.depth = (int)d;
    o.ctas_per_sm = (int)c;
    o.staging = (int)st;
    for (int i = 0; i < 4; ++i) o.rows[i] = rows[i];
    if (o.depth < 0 || o.depth > 4 || o.ctas_per_sm < 0 || o.staging < 0 || o.staging > 2)
        return LPBF_ERR_ARG;
    for (int i = 0; i < 4; ++i)
        if (o.rows[i] < 0) return LPBF_ERR_ARG;
    *out = o;
    return LPBF_OK;
}

int lpbf_b200_tune_cache_put(const char* path, const char* key, const lpbf_b200_batch_opts* o,
                             double gcells) {
    if (!path || !key || !o) return LPBF_ERR_ARG;
    std::map<std::string, std::string> ent;
    if (!parse_entries(read_file(path), &ent)) ent.clear();   // unreadable cache: start anew
    ent[key] = entry_text(*o, gcells);
    return write_entries(path, ent) ? LPBF_OK : LPBF_ERR_ARG;
}

int lpbf_b200_batch_tune_key(const lpbf_b200_scenario* sc, int n_scen, char* buf, size_t len) {
    if (!sc || n_scen <= 0 || !buf || len == 0) return LPBF_ERR_ARG;
    int count[4] = {0, 0, 0, 0};
    for (int i = 0; i < n_scen; ++i) {
        if (!sc[i].k) return LPBF_ERR_ARG;
        ++count[size_class(sc[i].k->nx, sc[i].k->ny)];
    }
    char name[256] = "cpu";
    int sms = 0;
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
        std::snprintf(name, sizeof(name), "%s", prop.name);
        sms = prop.multiProcessorCount;
    } else {
        cudaGetLastError();
    }
    auto bucket = [](int c) { int b = 0; while ((1 << b) < c) ++b; return c == 0 ? 0 : (1 << b); };
    const int w = std::snprintf(buf, len, "%s|sm%d|classes %d,%d,%d,%d", name, sms,
                                bucket(count[0]), bucket(count[1]), bucket(count[2]),
                                bucket(count[3]));
    return (w > 0 && (size_t)w < len) ? LPBF_OK : LPBF_ERR_ARG;
}

int lpbf_b200_batch_autotune(const lpbf_b200_scenario* sc, int n_scen, int n_steps,
                             const char* cache_path, int trial_steps, lpbf_b200_batch_opts* out) {
    NvtxRange nvtx_range("lpbf_b200_batch_autotune");
    if (!sc || n_scen <= 0 || !out || trial_steps < 1 || n_steps < trial_steps)
        return LPBF_ERR_ARG;
    for (int i = 0; i < n_scen; ++i)
        if (!sc[i].k || !sc[i].plan || sc[i].k->nx < 2 || sc[i].k->ny < 1) return LPBF_ERR_ARG;
    char key[512];
    if (lpbf_b200_batch_tune_key(sc, n_scen, key, sizeof(key)) != LPBF_OK) return LPBF_ERR_ARG;
    if (cache_path && lpbf_b200_tune_cache_get(cache_path, key, out) == LPBF_OK) return LPBF_OK;

    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return LPBF_ERR_CUDA;
    Scratch scratch;
    // Subset: per class, scenarios in the caller's order up to 2^27 cells
    // (at least one), each on scratch fields filled with its T_amb.
    constexpr double CLASS_CELLS = 134217728.0;
    std::vector<lpbf_b200_scenario> by_class[4];
    double cls_cells[4] = {0, 0, 0, 0};
    for (int i = 0; i < n_scen; ++i) {
        const StepConst& k = *sc[i].k;
        const int c = size_class(k.nx, k.ny);
        const double cells = (double)k.nx * k.ny;
        if (!by_class[c].empty() && cls_cells[c] + cells > CLASS_CELLS) continue;
        lpbf_b200_scenario t = sc[i];
        const size_t bytes = (size_t)k.nx * k.ny * sizeof(double);
        t.T_a = static_cast<double*>(scratch.get(bytes));
        t.T_b = static_cast<double*>(scratch.get(bytes));
        t.ring = static_cast<Partial*>(scratch.get(sizeof(Partial) * trial_steps));
        if (!t.T_a || !t.T_b || !t.ring) { cudaStreamDestroy(s); return LPBF_ERR_CUDA; }
        fill_kernel<<<256, 256, 0, s>>>(t.T_a, (size_t)k.nx * k.ny, k.Tamb);
        by_class[c].push_back(t);
        cls_cells[c] += cells;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) { cudaStreamDestroy(s); return LPBF_ERR_CUDA; }

    std::vector<lpbf_b200_scenario> all;
    for (int c = 0; c < 4; ++c) all.insert(all.end(), by_class[c].begin(), by_class[c].end());
    lpbf_b200_batch_opts best;
    std::memset(&best, 0, sizeof(best));
    best.depth = 2;
    static const int START[4] = {24, 48, 96, 192};
    for (int c = 0; c < 4; ++c) best.rows[c] = START[c];
    static const int ROWS[] = {12, 24, 48, 96, 192, 384};
    for (int c = 0; c < 4; ++c) {
        if (by_class[c].empty()) continue;
        double bg = 0.0;
        int br = best.rows[c];
        for (int r : ROWS) {
            lpbf_b200_batch_opts o = best;
            o.rows[c] = r;
            const double g = trial(all, trial_steps, o, s);
            if (g > bg) { bg = g; br = r; }
        }
        best.rows[c] = br;
    }
    double bg = 0.0;
    lpbf_b200_batch_opts win = best;
    for (int d : {2, 3, 4}) {
        for (int less = 0; less < 2; ++less) {
            const int occ = batch_resident_per_sm(d, BATCH_STAGE_BULK);
            if (less && occ <= 1) continue;
            for (int st : {BATCH_STAGE_BULK, BATCH_STAGE_TMAP}) {
                lpbf_b200_batch_opts o = best;
                o.depth = d;
                o.ctas_per_sm = less ? occ - 1 : 0;
                o.staging = st;
                const double g = trial(all, std::min(n_steps, std::max(trial_steps, 2 * d)), o, s);
                if (g > bg) { bg = g; win = o; }
            }
        }
    }
    cudaStreamDestroy(s);
    if (bg <= 0.0) return LPBF_ERR_CUDA;
    *out = win;
    if (cache_path) lpbf_b200_tune_cache_put(cache_path, key, &win, bg);
    return LPBF_OK;
}

}  // extern "C"
