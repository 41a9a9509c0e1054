/*
 * Minimal host-side stand-in for the Xilinx hls::stream FIFO, written for this
 * project (test infrastructure only).  Unbounded, thread safe; read() blocks;
 * empty() yields the CPU when it reports empty so the reference's busy-wait
 * loops do not starve the other dataflow threads.
 */
#pragma once
#include <deque>
#include <mutex>
#include <condition_variable>
#include <thread>

namespace hls {
template <typename T>
class stream {
    std::deque<T> q_;
    mutable std::mutex mu_;
    std::condition_variable cv_;
public:
    stream() {}
    explicit stream(const char *) {}
    stream(const stream &) = delete;
    bool empty() const {
        bool e;
        { std::lock_guard<std::mutex> g(mu_); e = q_.empty(); }
        if (e) std::this_thread::yield();
        return e;
    }
    bool full() const { return false; }
    void write(const T &v) {
        { std::lock_guard<std::mutex> g(mu_); q_.push_back(v); }
        cv_.notify_all();
    }
    T read() {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return !q_.empty(); });
        T v = q_.front();
        q_.pop_front();
        return v;
    }
    void read(T &v) { v = read(); }
    size_t size() const { std::lock_guard<std::mutex> g(mu_); return q_.size(); }
};
}  // namespace hls
