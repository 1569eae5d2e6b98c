/* Minimal stand-in for the parts of Intel TBB that the reference hot-path
 * translation units use (kernel.cpp, KernelOctree.cpp, KernelSampler.cpp).
 * TEST INFRASTRUCTURE ONLY: it exists so the unmodified reference sources can
 * be compiled into the CPU oracle.  TBB only schedules work in those files; it
 * carries no arithmetic, so a std::thread pool is behaviourally equivalent.
 *
 * Thread count: dr_tbbshim_threads (0 = all hardware threads, 1 = serial and
 * deterministic, which makes the reference's mt19937 seeding order fixed).
 */
#ifndef DR_TBB_SHIM_H
#define DR_TBB_SHIM_H

#include <cstddef>
#include <cstdlib>
#include <vector>
#include <tuple>
#include <functional>
#include <thread>
#include <mutex>
#include <atomic>
#include <map>
#include <memory>
#include <algorithm>

extern "C" int dr_tbbshim_threads;

namespace tbb {

template <typename T>
class blocked_range {
public:
    blocked_range() : b_(), e_() {}
    blocked_range(T b, T e) : b_(b), e_(e) {}
    T begin() const { return b_; }
    T end() const { return e_; }
    std::size_t size() const { return (std::size_t)(e_ - b_); }
private:
    T b_, e_;
};

template <typename T>
class blocked_range2d {
public:
    blocked_range2d(T r0, T r1, T c0, T c1) : rows_(r0, r1), cols_(c0, c1) {}
    const blocked_range<T> &rows() const { return rows_; }
    const blocked_range<T> &cols() const { return cols_; }
private:
    blocked_range<T> rows_, cols_;
};

class auto_partitioner {};

inline int shim_thread_count() {
    int n = dr_tbbshim_threads;
    if (n <= 0) {
        n = (int)std::thread::hardware_concurrency();
        if (n <= 0) n = 1;
    }
    return n;
}

/* Rows of a 2-D range are handed out one at a time from an atomic counter. */
template <typename T, typename F>
void parallel_for(const blocked_range2d<T> &r, const F &f, const auto_partitioner & = auto_partitioner()) {
    const T r0 = r.rows().begin(), r1 = r.rows().end();
    int nt = shim_thread_count();
    if (nt == 1 || r1 - r0 <= 1) {
        f(r);
        return;
    }
    std::atomic<T> next(r0);
    auto worker = [&]() {
        for (;;) {
            T y = next.fetch_add(1);
            if (y >= r1) break;
            blocked_range2d<T> sub(y, y + 1, r.cols().begin(), r.cols().end());
            f(sub);
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < nt; ++i) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

template <typename T, typename F>
void parallel_for(const blocked_range<T> &r, const F &f, const auto_partitioner & = auto_partitioner()) {
    int nt = shim_thread_count();
    if (nt == 1 || r.size() <= 1) {
        f(r);
        return;
    }
    std::atomic<T> next(r.begin());
    const T e = r.end();
    auto worker = [&]() {
        for (;;) {
            T y = next.fetch_add(1);
            if (y >= e) break;
            f(blocked_range<T>(y, y + 1));
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < nt; ++i) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
}

class spin_mutex {
public:
    void lock() { m_.lock(); }
    void unlock() { m_.unlock(); }
private:
    std::mutex m_;
};

template <typename T>
class enumerable_thread_specific {
public:
    T &local() {
        std::lock_guard<std::mutex> g(m_);
        auto &p = map_[std::this_thread::get_id()];
        if (!p) p.reset(new T());
        return *p;
    }
private:
    std::mutex m_;
    std::map<std::thread::id, std::unique_ptr<T>> map_;
};

/* Only indexing, size and growth are used by the hot path and the harness. */
template <typename T>
class concurrent_vector : public std::vector<T> {
public:
    void grow_to_at_least(std::size_t n) {
        if (this->size() < n) this->resize(n);
    }
};

} // namespace tbb

inline void *scalable_malloc(std::size_t n) { return std::malloc(n); }
inline void scalable_free(void *p) { std::free(p); }

#endif
