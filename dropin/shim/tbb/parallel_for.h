/* TBB shim: parallel_for over a blocked_range, chunked by the range's grain
 * size (or about four chunks per worker with auto_partitioner), chunks taken
 * dynamically by the workers.  The body is copied for every chunk, as TBB
 * copies it when it splits a range. */
#pragma once
#include "_pool.h"
#include "blocked_range.h"
namespace tbb {
class auto_partitioner {};
class simple_partitioner {};

namespace shim {
template <typename Range, typename Body>
struct pfor_job {
    const Range *range;
    const Body *body;
    size_t chunk;
    ticket_counter *tickets;
};

template <typename Range, typename Body>
void pfor_worker(void *p, int)
{
    pfor_job<Range, Body> *j = (pfor_job<Range, Body> *)p;
    long t;
    while (j->tickets->take(t)) {
        typename Range::const_iterator b = j->range->begin() + (size_t)t * j->chunk;
        typename Range::const_iterator e = b + j->chunk;
        if (j->range->end() < e) e = j->range->end();
        Body copy(*j->body);
        copy(Range(b, e, j->range->grainsize()));
    }
}

template <typename Range, typename Body>
void pfor(const Range &r, const Body &body, size_t chunk)
{
    if (r.empty()) return;
    const size_t n = r.size();
    if (chunk == 0) chunk = 1;
    const long nchunks = (long)((n + chunk - 1) / chunk);
    ticket_counter tickets(nchunks);
    pfor_job<Range, Body> job;
    job.range = &r; job.body = &body; job.chunk = chunk; job.tickets = &tickets;
    int nw = thread_count();
    if (nw > nchunks) nw = (int)nchunks;
    run_workers(nw, &pfor_worker<Range, Body>, &job);
}
} // namespace shim

template <typename Range, typename Body>
void parallel_for(const Range &r, const Body &body)
{
    shim::pfor(r, body, r.grainsize());
}

template <typename Range, typename Body>
void parallel_for(const Range &r, const Body &body, const simple_partitioner &)
{
    shim::pfor(r, body, r.grainsize());
}

template <typename Range, typename Body>
void parallel_for(const Range &r, const Body &body, const auto_partitioner &)
{
    const size_t n = r.size();
    const size_t want = (size_t)shim::thread_count() * 4;
    size_t chunk = (n + want - 1) / (want ? want : 1);
    if (chunk < r.grainsize()) chunk = r.grainsize();
    shim::pfor(r, body, chunk);
}
}
