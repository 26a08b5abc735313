// Test infrastructure only: a project-written stand-in for the subset of Intel
// oneTBB 2020.3 (pinned by the reference, conanfile.py:23) that the emerald SPH
// sources call: parallel_for, parallel_reduce, parallel_scan, parallel_sort,
// blocked_range and concurrent_unordered_map. Work runs on a persistent
// std::thread pool; with one thread everything runs serially in index order.
// The emerald loops are owner-writes with integer/max reductions, so results
// do not depend on the thread count (the reference's own repeatability test,
// emerald/sph2d_box/tests/test_repeatability.cpp:53-112, relies on this).
#pragma once

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstddef>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

namespace tbb_shim {

class Pool {
public:
    static Pool& get();
    void set_threads(int n);
    int threads() const { return threads_; }
    // Runs fn(c) for every c in [0, nchunks), on the pool.
    void run(size_t nchunks, std::function<void(size_t)> const& fn);
    ~Pool();

private:
    Pool();
    void worker_loop();
    void stop_workers();

    int threads_ = 1;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_;
    std::condition_variable done_cv_;
    std::function<void(size_t)> const* job_ = nullptr;
    size_t nchunks_ = 0;
    std::atomic<size_t> next_{0};
    size_t busy_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

bool in_worker();

}  // namespace tbb_shim

namespace tbb {

template <class T>
class blocked_range {
public:
    blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), g_(grain ? grain : 1) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    size_t size() const { return static_cast<size_t>(e_ - b_); }
    size_t grainsize() const { return g_; }
    bool empty() const { return !(b_ < e_); }

private:
    T b_;
    T e_;
    size_t g_;
};

namespace detail {
template <class T>
inline std::vector<blocked_range<T>> split(blocked_range<T> const& r) {
    std::vector<blocked_range<T>> parts;
    size_t const n = r.size();
    if (n == 0) { return parts; }
    size_t const threads = static_cast<size_t>(tbb_shim::Pool::get().threads());
    size_t chunk = r.grainsize();
    if (threads > 1 && !tbb_shim::in_worker()) {
        size_t const target = (n + threads * 8 - 1) / (threads * 8);
        chunk = std::max(chunk, target);
    } else {
        chunk = n;
    }
    for (size_t off = 0; off < n; off += chunk) {
        size_t const len = std::min(chunk, n - off);
        parts.emplace_back(r.begin() + off, r.begin() + (off + len), r.grainsize());
    }
    return parts;
}
}  // namespace detail

template <class T, class Body>
void parallel_for(blocked_range<T> const& range, Body const& body) {
    auto const parts = detail::split(range);
    if (parts.size() <= 1) {
        if (!parts.empty()) body(parts[0]);
        return;
    }
    tbb_shim::Pool::get().run(parts.size(), [&](size_t c) { body(parts[c]); });
}

template <class T, class Value, class Func, class Reduction>
Value parallel_reduce(blocked_range<T> const& range,
                      Value const& identity,
                      Func const& func,
                      Reduction const& reduction) {
    auto const parts = detail::split(range);
    if (parts.empty()) return identity;
    if (parts.size() == 1) return func(parts[0], identity);
    std::vector<Value> partial(parts.size(), identity);
    tbb_shim::Pool::get().run(parts.size(),
                              [&](size_t c) { partial[c] = func(parts[c], identity); });
    Value acc = partial[0];
    for (size_t c = 1; c < partial.size(); ++c) acc = reduction(acc, partial[c]);
    return acc;
}

template <class T, class Value, class Scan, class Combine>
Value parallel_scan(blocked_range<T> const& range,
                    Value const& identity,
                    Scan const& scan,
                    Combine const& combine) {
    auto const parts = detail::split(range);
    if (parts.empty()) return identity;
    if (parts.size() == 1) return scan(parts[0], identity, true);
    std::vector<Value> sums(parts.size(), identity);
    auto& pool = tbb_shim::Pool::get();
    pool.run(parts.size(), [&](size_t c) { sums[c] = scan(parts[c], identity, false); });
    std::vector<Value> prefix(parts.size() + 1, identity);
    for (size_t c = 0; c < parts.size(); ++c) prefix[c + 1] = combine(prefix[c], sums[c]);
    pool.run(parts.size(), [&](size_t c) { scan(parts[c], prefix[c], true); });
    return prefix.back();
}

template <class It>
void parallel_sort(It first, It last) {
    size_t const n = static_cast<size_t>(last - first);
    size_t const threads = static_cast<size_t>(tbb_shim::Pool::get().threads());
    if (threads <= 1 || n < 4096 || tbb_shim::in_worker()) {
        std::sort(first, last);
        return;
    }
    size_t const k = threads;
    std::vector<size_t> bounds(k + 1);
    for (size_t c = 0; c <= k; ++c) bounds[c] = n * c / k;
    auto& pool = tbb_shim::Pool::get();
    pool.run(k, [&](size_t c) { std::sort(first + bounds[c], first + bounds[c + 1]); });
    for (size_t width = 1; width < k; width *= 2) {
        std::vector<size_t> starts;
        for (size_t c = 0; c + width < k; c += 2 * width) starts.push_back(c);
        pool.run(starts.size(), [&](size_t s) {
            size_t const c = starts[s];
            size_t const mid = c + width;
            size_t const hi = std::min(c + 2 * width, k);
            std::inplace_merge(first + bounds[c], first + bounds[mid], first + bounds[hi]);
        });
    }
}

template <class K, class V, class H = std::hash<K>, class E = std::equal_to<K>>
class concurrent_unordered_map {
public:
    using map_type = std::unordered_map<K, V, H, E>;
    using iterator = typename map_type::iterator;
    using const_iterator = typename map_type::const_iterator;
    using value_type = typename map_type::value_type;

    concurrent_unordered_map() : mu_(new std::mutex) {}
    explicit concurrent_unordered_map(size_t buckets) : map_(buckets), mu_(new std::mutex) {}
    concurrent_unordered_map(concurrent_unordered_map const& o) : map_(o.map_), mu_(new std::mutex) {}
    concurrent_unordered_map(concurrent_unordered_map&& o) noexcept
      : map_(std::move(o.map_)), mu_(new std::mutex) {}
    concurrent_unordered_map& operator=(concurrent_unordered_map const& o) {
        map_ = o.map_;
        return *this;
    }
    concurrent_unordered_map& operator=(concurrent_unordered_map&& o) noexcept {
        map_ = std::move(o.map_);
        return *this;
    }

    void clear() { map_.clear(); }
    void rehash(size_t n) { map_.rehash(n); }
    size_t size() const { return map_.size(); }
    bool empty() const { return map_.empty(); }

    template <class... A>
    std::pair<iterator, bool> emplace(A&&... a) {
        std::lock_guard<std::mutex> lock(*mu_);
        return map_.emplace(std::forward<A>(a)...);
    }
    std::pair<iterator, bool> insert(value_type const& v) {
        std::lock_guard<std::mutex> lock(*mu_);
        return map_.insert(v);
    }
    iterator find(K const& k) { return map_.find(k); }
    const_iterator find(K const& k) const { return map_.find(k); }
    iterator begin() { return map_.begin(); }
    iterator end() { return map_.end(); }
    const_iterator begin() const { return map_.begin(); }
    const_iterator end() const { return map_.end(); }

private:
    map_type map_;
    std::unique_ptr<std::mutex> mu_;
};

}  // namespace tbb
