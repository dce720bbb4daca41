/* TBB shim: wall-clock tick_count. */
#pragma once
#include <time.h>
namespace tbb {
class tick_count {
    double t;
public:
    class interval_t {
        double s;
    public:
        interval_t() : s(0) {}
        explicit interval_t(double s_) : s(s_) {}
        double seconds() const { return s; }
        interval_t &operator+=(const interval_t &o) { s += o.s; return *this; }
        interval_t &operator-=(const interval_t &o) { s -= o.s; return *this; }
    };
    tick_count() : t(0) {}
    static tick_count now()
    {
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        tick_count c;
        c.t = ts.tv_sec + 1e-9 * ts.tv_nsec;
        return c;
    }
    friend interval_t operator-(const tick_count &a, const tick_count &b)
    {
        return interval_t(a.t - b.t);
    }
};
}
