// Stand-in: tbb::concurrent_queue as a mutex-guarded std::queue (push / try_pop / empty).
#pragma once
#include <mutex>
#include <queue>
namespace tbb {
template <class T>
class concurrent_queue {
    std::queue<T> q_;
    mutable std::mutex m_;
public:
    void push(const T& v) { std::lock_guard<std::mutex> l(m_); q_.push(v); }
    bool try_pop(T& v) {
        std::lock_guard<std::mutex> l(m_);
        if (q_.empty()) return false;
        v = q_.front();
        q_.pop();
        return true;
    }
    bool empty() const { std::lock_guard<std::mutex> l(m_); return q_.empty(); }
};
}  // namespace tbb
