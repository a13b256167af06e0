/*
 * Stand-in for TBB's concurrent_bounded_queue, used ONLY to compile the
 * reference's VCFData.cpp into the writer harness of the test oracle: a
 * mutex-guarded deque with the member functions VCFData uses (push, pop,
 * try_pop, size, empty, clear, set_capacity).  The harness runs the writer
 * with one worker and drains the queues after the call, so pop never waits.
 */
#ifndef EIMP_WRITER_STUB_TBB_QUEUE_H
#define EIMP_WRITER_STUB_TBB_QUEUE_H

#include <condition_variable>
#include <cstddef>
#include <deque>
#include <mutex>

namespace tbb {

template <typename T> class concurrent_bounded_queue {
public:
    concurrent_bounded_queue() = default;
    concurrent_bounded_queue(const concurrent_bounded_queue &o) : q(o.q), cap(o.cap) {}
    concurrent_bounded_queue &operator=(const concurrent_bounded_queue &o) { q = o.q; cap = o.cap; return *this; }
    void push(const T &v) {
        std::lock_guard<std::mutex> lk(m);
        q.push_back(v);
        cv.notify_one();
    }
    void pop(T &v) {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return !q.empty(); });
        v = q.front();
        q.pop_front();
    }
    bool try_pop(T &v) {
        std::lock_guard<std::mutex> lk(m);
        if (q.empty()) return false;
        v = q.front();
        q.pop_front();
        return true;
    }
    std::ptrdiff_t size() const { std::lock_guard<std::mutex> lk(m); return (std::ptrdiff_t)q.size(); }
    bool empty() const { std::lock_guard<std::mutex> lk(m); return q.empty(); }
    void clear() { std::lock_guard<std::mutex> lk(m); q.clear(); }
    void set_capacity(std::ptrdiff_t c) { cap = c; }
    void abort() {}

private:
    std::deque<T> q;
    std::ptrdiff_t cap = 0;
    mutable std::mutex m;
    std::condition_variable cv;
};

}  // namespace tbb

#endif
