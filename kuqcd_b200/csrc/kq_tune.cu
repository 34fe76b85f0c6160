// Launch-shape autotuning cache: shapes measured on this GPU model are kept in a small text file so that the timing
// runs happen once per problem signature.  The measurements themselves are made by the callers (kq_batch.cu times
// windows of the real batch for every candidate shape).
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>

#include <cuda_runtime.h>
#include <sys/stat.h>

#include "kq_tune.h"

namespace kq {

namespace {

std::mutex g_mu;
std::map<std::string, std::string> g_cache;
bool g_loaded = false;

std::string cache_path()
{
    if (const char *p = getenv("KUQCD_TUNE_CACHE")) return p;
    const char *home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/kuqcd_b200/tunecache.txt";
}

std::string gpu_name()
{
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
    std::string n = prop.name;
    for (char &c : n)
        if (c == ' ' || c == '|') c = '_';
    return n;
}

void load_locked()
{
    if (g_loaded) return;
    g_loaded = true;
    std::ifstream f(cache_path());
    std::string line;
    while (std::getline(f, line)) {
        const size_t sp = line.find(' ');
        if (sp == std::string::npos) continue;
        g_cache[line.substr(0, sp)] = line.substr(sp + 1);
    }
}

void append_locked(const std::string &k, const std::string &v)
{
    g_cache[k] = v;
    const std::string path = cache_path();
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
        // create the directory chain if needed (best effort)
        std::string dir = path.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i)
            if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    std::ofstream f(path, std::ios::app);
    if (f) f << k << ' ' << v << '\n';
}

}  // namespace

bool tune_lookup(const std::string &key, BatchTune *out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_cache.find(gpu_name() + "|" + key);
    if (it == g_cache.end()) return false;
    std::istringstream is(it->second);
    BatchTune t;
    if (!(is >> t.bs >> t.ctas_per_sm >> t.rhs >> t.spt >> t.p64)) return false;
    if (t.p64 != 0 && t.p64 != 1 && t.p64 != 2 && t.p64 != 4) return false;  // 0: staged FP64 kernels
    if (t.bs != 128 && t.bs != 256) return false;
    if (t.ctas_per_sm < 1 || t.ctas_per_sm > 32) return false;
    if (t.rhs != 1 && t.rhs != 2 && t.rhs != 4 && t.rhs != 8) return false;
    if (t.spt != 1 && t.spt != 2) return false;
    *out = t;
    return true;
}

void tune_store(const std::string &key, const BatchTune &t)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    append_locked(gpu_name() + "|" + key, std::to_string(t.bs) + " " + std::to_string(t.ctas_per_sm) + " " +
                                               std::to_string(t.rhs) + " " + std::to_string(t.spt) + " " +
                                               std::to_string(t.p64));
}

bool tune_lookup_int(const std::string &key, int *out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_cache.find(gpu_name() + "|" + key);
    if (it == g_cache.end()) return false;
    *out = atoi(it->second.c_str());
    return *out > 0;
}

void tune_store_int(const std::string &key, int v)
{
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    append_locked(gpu_name() + "|" + key, std::to_string(v));
}

}  // namespace kq
