// Minimal stand-in for the few oneTBB entry points the hpHawkes CPU engine
// (src/NewHawkes.hpp:225-235, :812-848) and its benchmark CLI
// (src/benchmark.cpp:79-97) use.  TBB is not installed in this image, so this
// header lets the reference engine be compiled unmodified as the oracle and as
// the timed CPU baseline.
//
// Test infrastructure only: nothing in the product links it.
//
// parallel_reduce / parallel_for split the range into P contiguous blocks
// (P = the active global_control limit, else hardware_concurrency) and run one
// std::thread per block.  Partial results are combined left to right, so a
// given P always gives the same floating-point result.
#ifndef HAWKES_ORACLE_TBB_STUB_H
#define HAWKES_ORACLE_TBB_STUB_H

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <thread>
#include <vector>

namespace tbb {

namespace stub_detail {
inline std::atomic<size_t>& limit() {
    static std::atomic<size_t> value{0};
    return value;
}
inline size_t threads() {
    size_t v = limit().load();
    if (v == 0) v = std::thread::hardware_concurrency();
    return v == 0 ? 1 : v;
}
}  // namespace stub_detail

class global_control {
public:
    enum parameter { max_allowed_parallelism, thread_stack_size };
    global_control(parameter p, size_t value) : param(p) {
        if (p == max_allowed_parallelism) previous = stub_detail::limit().exchange(value);
    }
    ~global_control() {
        if (param == max_allowed_parallelism) stub_detail::limit().store(previous);
    }
    static size_t active_value(parameter p) {
        return p == max_allowed_parallelism ? stub_detail::threads() : 0;
    }

private:
    parameter param;
    size_t previous = 0;
};

namespace this_task_arena {
inline int max_concurrency() { return static_cast<int>(stub_detail::threads()); }
}  // namespace this_task_arena

class task_arena {
public:
    explicit task_arena(int = -1) {}
};

template <typename Value>
class blocked_range {
public:
    blocked_range(Value b, Value e, size_t = 1) : b_(b), e_(e) {}
    Value begin() const { return b_; }
    Value end() const { return e_; }
    size_t size() const { return static_cast<size_t>(e_ - b_); }
    bool empty() const { return !(b_ < e_); }

private:
    Value b_, e_;
};

template <typename Value>
std::vector<blocked_range<Value>> stub_split(const blocked_range<Value>& r) {
    std::vector<blocked_range<Value>> parts;
    const size_t n = r.size();
    size_t p = std::min(stub_detail::threads(), n == 0 ? size_t(1) : n);
    if (p == 0) p = 1;
    const size_t base = n / p, extra = n % p;
    Value start = r.begin();
    for (size_t k = 0; k < p; ++k) {
        const size_t len = base + (k < extra ? 1 : 0);
        parts.emplace_back(start, static_cast<Value>(start + len));
        start = static_cast<Value>(start + len);
    }
    return parts;
}

template <typename Value, typename Real, typename Body, typename Reduction>
Real parallel_reduce(const blocked_range<Value>& range, const Real& identity, const Body& body,
                     const Reduction& reduction) {
    auto parts = stub_split(range);
    std::vector<Real> partial(parts.size(), identity);
    if (parts.size() == 1) {
        partial[0] = body(parts[0], identity);
    } else {
        std::vector<std::thread> pool;
        for (size_t k = 0; k < parts.size(); ++k) {
            pool.emplace_back([&, k] { partial[k] = body(parts[k], identity); });
        }
        for (auto& t : pool) t.join();
    }
    Real total = identity;
    for (auto& v : partial) total = reduction(total, v);
    return total;
}

template <typename Value, typename Body>
void parallel_for(const blocked_range<Value>& range, const Body& body) {
    auto parts = stub_split(range);
    if (parts.size() == 1) {
        body(parts[0]);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t k = 0; k < parts.size(); ++k) {
        pool.emplace_back([&, k] { body(parts[k]); });
    }
    for (auto& t : pool) t.join();
}

}  // namespace tbb

#endif  // HAWKES_ORACLE_TBB_STUB_H
