/* Minimal stand-in for the subset of Intel TBB the reference uses (parallel_for,
 * parallel_reduce, parallel_sort, enumerable_thread_specific, task_group, blocked_range,
 * cache_aligned_allocator). TBB is not installed here. Loops run serially by default, which
 * makes the reference's float accumulation order deterministic for parity runs; setting
 * imbart_ref_tbb_threads > 1 runs blocked_range<int> loops on OpenMP threads (used to time
 * the reference's CPU path). TEST INFRASTRUCTURE ONLY. */
#ifndef IMBART_REF_TBB_SHIM_CORE_H
#define IMBART_REF_TBB_SHIM_CORE_H
#include <algorithm>
#include <cstddef>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

extern int imbart_ref_tbb_threads;

namespace tbb {

template <typename T>
class blocked_range {
public:
    blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), grain_(grain) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    size_t size() const { return (size_t)(e_ - b_); }
    bool empty() const { return !(b_ < e_); }
    size_t grainsize() const { return grain_; }

private:
    T b_, e_;
    size_t grain_;
};

template <typename Body>
void parallel_for(const blocked_range<int>& r, const Body& body) {
    const int n = r.end() - r.begin();
    if (imbart_ref_tbb_threads <= 1 || n < 256) {
        body(r);
        return;
    }
    const int chunk = 256;
    const int nchunks = (n + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1) num_threads(imbart_ref_tbb_threads)
    for (int c = 0; c < nchunks; ++c) {
        const int b = r.begin() + c * chunk;
        body(blocked_range<int>(b, std::min(b + chunk, r.end())));
    }
}

template <typename Range, typename Body>
void parallel_for(const Range& r, const Body& body) {
    body(r);
}

template <typename Range, typename Value, typename RealBody, typename Reduction>
Value parallel_reduce(const Range& r, const Value& identity, const RealBody& body, const Reduction& reduce) {
    return reduce(identity, body(r, identity));
}

template <typename It>
void parallel_sort(It b, It e) { std::sort(b, e); }
template <typename It, typename Cmp>
void parallel_sort(It b, It e, const Cmp& c) { std::sort(b, e, c); }

template <typename T>
using cache_aligned_allocator = std::allocator<T>;

enum ets_key_usage_type { ets_key_per_instance, ets_no_key };

template <typename T, typename Alloc = cache_aligned_allocator<T>, ets_key_usage_type K = ets_no_key>
class enumerable_thread_specific {
public:
    T& local() {
        std::lock_guard<std::mutex> lk(m_);
        auto& p = items_[std::this_thread::get_id()];
        if (!p) p.reset(new T());
        return *p;
    }

private:
    std::mutex m_;
    std::unordered_map<std::thread::id, std::unique_ptr<T>> items_;
};

class task_group {
public:
    template <typename F>
    void run(const F& f) { f(); }
    void wait() {}
};

}  // namespace tbb
#endif
