// Test infrastructure only: the std::thread pool behind the TBB stand-in
// (tbb/tbb_shim.h). Linked only into the oracle build of the reference.
#include <tbb/tbb_shim.h>

namespace tbb_shim {

static thread_local bool t_in_worker = false;

bool in_worker() { return t_in_worker; }

Pool& Pool::get() {
    static Pool pool;
    return pool;
}

Pool::Pool() {}

Pool::~Pool() { stop_workers(); }

void Pool::stop_workers() {
    {
        std::lock_guard<std::mutex> lock(m_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    workers_.clear();
    stop_ = false;
}

void Pool::set_threads(int n) {
    if (n < 1) n = 1;
    if (n == threads_) return;
    stop_workers();
    threads_ = n;
    for (int i = 1; i < n; ++i) workers_.emplace_back([this] { worker_loop(); });
}

void Pool::worker_loop() {
    t_in_worker = true;
    unsigned long long seen = 0;
    for (;;) {
        std::function<void(size_t)> const* job = nullptr;
        size_t n = 0;
        {
            std::unique_lock<std::mutex> lock(m_);
            cv_.wait(lock, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            job = job_;
            n = nchunks_;
            ++busy_;
        }
        for (size_t c = next_.fetch_add(1); c < n; c = next_.fetch_add(1)) (*job)(c);
        {
            std::lock_guard<std::mutex> lock(m_);
            --busy_;
        }
        done_cv_.notify_all();
    }
}

void Pool::run(size_t nchunks, std::function<void(size_t)> const& fn) {
    if (threads_ <= 1 || nchunks <= 1 || t_in_worker) {
        for (size_t c = 0; c < nchunks; ++c) fn(c);
        return;
    }
    {
        // A worker that woke late for the previous job may still hold that
        // job's chunk count; let it drain before the counter is reset.
        std::unique_lock<std::mutex> lock(m_);
        done_cv_.wait(lock, [&] { return busy_ == 0; });
        job_ = &fn;
        nchunks_ = nchunks;
        next_.store(0);
        ++gen_;
    }
    cv_.notify_all();
    bool const was_worker = t_in_worker;
    t_in_worker = true;
    for (size_t c = next_.fetch_add(1); c < nchunks; c = next_.fetch_add(1)) fn(c);
    t_in_worker = was_worker;
    std::unique_lock<std::mutex> lock(m_);
    done_cv_.wait(lock, [&] { return busy_ == 0; });
    job_ = nullptr;
}

}  // namespace tbb_shim
