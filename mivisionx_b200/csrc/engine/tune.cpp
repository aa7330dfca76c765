// tune.cpp -- the launch-shape table the autotuner (mivisionx_b200/autotune.py) writes and
// vxVerifyGraph reads: per kernel and frame size, the parameters of its launch (rows per
// thread, warps or threads per block, resident blocks per SM, persistent or not).
//
// File: $AGO_B200_TUNE_FILE, else tune/b200.json beside this library's directory
// (mivisionx_b200/tune/b200.json).  Format:
//   {"device": "...", "sm_count": 148,
//    "entries": [{"kernel": "<name>", "width": W, "height": H, "params": [a, b, c, d], ...}, ...]}
// Lookup: the entry of the kernel with the same frame size, else the one with the closest
// pixel count; no entry (or no file) gives the caller's default.
#include <dlfcn.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "vx_internal.h"

namespace agovx {

struct TuneEntry {
    std::string kernel;
    uint32_t width = 0, height = 0;
    std::vector<uint32_t> params;
};

namespace {

std::mutex g_tune_mu;
bool g_tune_loaded = false;
std::vector<TuneEntry> g_tune;
std::string g_tune_path;

std::string library_dir()
{
    Dl_info info{};
    if (!dladdr((void *)&library_dir, &info) || !info.dli_fname) return ".";
    std::string p(info.dli_fname);
    const size_t k = p.rfind('/');
    return k == std::string::npos ? "." : p.substr(0, k);
}

// The value after "key": in an object's text (numbers, strings, or [n, n, ...] arrays).
const char *find_key(const std::string &obj, const char *key)
{
    const std::string k = std::string("\"") + key + "\"";
    size_t i = obj.find(k);
    if (i == std::string::npos) return nullptr;
    i = obj.find(':', i + k.size());
    if (i == std::string::npos) return nullptr;
    const char *p = obj.c_str() + i + 1;
    while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r') p++;
    return p;
}

void parse(const std::string &text)
{
    const size_t e = text.find("\"entries\"");
    if (e == std::string::npos) return;
    size_t i = text.find('[', e);
    if (i == std::string::npos) return;
    for (;;) {
        const size_t a = text.find('{', i), close = text.find(']', i);
        if (a == std::string::npos || (close != std::string::npos && close < a)) break;
        const size_t b = text.find('}', a);
        if (b == std::string::npos) break;
        const std::string obj = text.substr(a, b - a + 1);
        TuneEntry t;
        if (const char *p = find_key(obj, "kernel"); p && *p == '"') {
            const char *q = strchr(p + 1, '"');
            if (q) t.kernel.assign(p + 1, q - p - 1);
        }
        if (const char *p = find_key(obj, "width")) t.width = (uint32_t)strtoul(p, nullptr, 10);
        if (const char *p = find_key(obj, "height")) t.height = (uint32_t)strtoul(p, nullptr, 10);
        if (const char *p = find_key(obj, "params"); p && *p == '[') {
            p++;
            for (;;) {
                while (*p == ' ' || *p == ',') p++;
                if (*p == ']' || !*p) break;
                char *end = nullptr;
                const unsigned long v = strtoul(p, &end, 10);
                if (end == p) break;
                t.params.push_back((uint32_t)v);
                p = end;
            }
        }
        if (!t.kernel.empty() && t.width && t.height && !t.params.empty()) g_tune.push_back(t);
        i = b + 1;
    }
}

void load()
{
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char *env = getenv("AGO_B200_TUNE_FILE");
    g_tune_path = env && *env ? std::string(env) : library_dir() + "/../tune/b200.json";
    FILE *f = fopen(g_tune_path.c_str(), "rb");
    if (!f) return;
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    fclose(f);
    parse(text);
}

}  // namespace

// Parameters for `kernel` on frames of w x h, or `dflt` when the table has none.
std::vector<uint32_t> tune_lookup(const char *kernel, uint32_t w, uint32_t h, const std::vector<uint32_t> &dflt)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    load();
    const TuneEntry *best = nullptr;
    double bestd = 0;
    for (const TuneEntry &t : g_tune) {
        if (t.kernel != kernel || t.params.size() != dflt.size()) continue;
        if (t.width == w && t.height == h) return t.params;
        const double d = std::fabs(std::log((double)t.width * t.height / ((double)w * h)));
        if (!best || d < bestd) { best = &t; bestd = d; }
    }
    return best ? best->params : dflt;
}

// Forget the loaded table (the next lookup reads the file again): for the autotuner, which
// rewrites it, and for tests that point AGO_B200_TUNE_FILE elsewhere.
void tune_reload()
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    g_tune_loaded = false;
}

}  // namespace agovx

// Hooks for the autotuner and tests (not part of the OpenVX API): re-read the table, and look
// an entry up as the planner does (returns the number of parameters written to `out`).
extern "C" void agovx_tune_reload(void) { agovx::tune_reload(); }

extern "C" int agovx_tune_lookup(const char *kernel, uint32_t width, uint32_t height, uint32_t count, uint32_t *out)
{
    if (!kernel || !out || !count || count > 16) return 0;
    std::vector<uint32_t> dflt(count, 0);
    const std::vector<uint32_t> p = agovx::tune_lookup(kernel, width, height, dflt);
    for (uint32_t i = 0; i < count; i++) out[i] = p[i];
    return p == dflt ? 0 : (int)count;
}
