// Thread-local error state of the C ABI. The reference entry points return void and the
// reference reports failures through assert (ray_queue.h:248,270-271); here nothing aborts,
// the failing call records an error that the caller reads with imbart_last_error().
#include <atomic>
#include <string>

#include "imbart_internal.h"

namespace {
thread_local int g_code = 0;
thread_local std::string g_msg;
}

namespace imbart {
void set_error(int code, const std::string& msg) {
    g_code = code;
    g_msg = msg;
}

// Process-wide count of kernel launches issued by libimbart (a CUDA graph's kernels are
// counted when the graph is launched).
static std::atomic<long long> g_launches{0};
void note_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_total() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace imbart

extern "C" int imbart_last_error(void) { return g_code; }
extern "C" const char* imbart_last_error_string(void) { return g_msg.c_str(); }
extern "C" void imbart_clear_error(void) { g_code = 0; g_msg.clear(); }
extern "C" const char* imbart_version(void) { return "imbart 0.1 (sm_100a)"; }
