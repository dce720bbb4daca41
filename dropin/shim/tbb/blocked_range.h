/* TBB shim: blocked_range. */
#pragma once
#include <stddef.h>
namespace tbb {
template <typename Value>
class blocked_range {
    Value b, e;
    size_t g;
public:
    typedef Value const_iterator;
    blocked_range() : b(), e(), g(1) {}
    blocked_range(Value begin_, Value end_, size_t grain = 1) : b(begin_), e(end_), g(grain ? grain : 1) {}
    const_iterator begin() const { return b; }
    const_iterator end() const { return e; }
    size_t size() const { return (size_t)(e - b); }
    size_t grainsize() const { return g; }
    bool empty() const { return !(b < e); }
    bool is_divisible() const { return g < size(); }
};
}
