/* TBB shim: pipeline of filters.  run(ntokens) starts min(ntokens, workers)
 * threads; each repeatedly asks the first filter for a token (NULL ends the
 * stream) and passes it through the remaining filters in order.  This is
 * the behaviour of a TBB pipeline whose filters are all parallel
 * (filter(false)), which is how the reference's block pipeline builds it. */
#pragma once
#include "_pool.h"
#include <vector>
namespace tbb {
class filter {
protected:
    explicit filter(bool is_serial_) : serial(is_serial_) {}
public:
    const bool serial;
    virtual void *operator()(void *item) = 0;
    virtual ~filter() {}
};

class pipeline {
    std::vector<filter *> stages;
    static void worker(void *p, int)
    {
        pipeline *self = (pipeline *)p;
        for (;;) {
            void *tok = (*self->stages[0])(NULL);
            if (!tok) break;
            for (size_t i = 1; i < self->stages.size() && tok; i++) tok = (*self->stages[i])(tok);
        }
    }
public:
    pipeline() : stages() {}
    void add_filter(filter &f) { stages.push_back(&f); }
    void clear() { stages.clear(); }
    void run(size_t max_tokens)
    {
        if (stages.empty()) return;
        int nw = shim::thread_count();
        if ((size_t)nw > max_tokens) nw = (int)max_tokens;
        shim::run_workers(nw, &pipeline::worker, this);
    }
};
}
