/*
 * Project-written stand-in for the parts of Intel TBB 4.0 that the reference's
 * MRAG library names (task_scheduler_init, tick_count, blocked_range,
 * parallel_for, pipeline/filter, concurrent_bounded_queue, allocators).
 * TBB is not installed in this image; this shim lets the reference's own
 * sources compile unmodified: for the oracle and the CPU baseline, and for
 * the drop-in driver whose block tree is the reference's own grid.
 *
 * Threads are POSIX threads (the reference compiles as gnu++98, so no
 * std::thread).  One global worker count is set by task_scheduler_init(n),
 * else by the environment variable GBFK_TBB_THREADS, else by the number
 * of online cores.
 */
#pragma once
#include <pthread.h>
#include <unistd.h>
#include <stdlib.h>
#include <stddef.h>

namespace tbb {
namespace shim {

inline int &thread_count_ref() { static int n = 0; return n; }

inline int thread_count()
{
    int &n = thread_count_ref();
    if (n <= 0) {
        const char *e = getenv("GBFK_TBB_THREADS");
        if (e && atoi(e) > 0) n = atoi(e);
        else {
            long c = sysconf(_SC_NPROCESSORS_ONLN);
            n = c > 0 ? (int)c : 1;
        }
    }
    return n;
}

/* Run fn(arg, worker_index) on nworkers threads (the caller is worker 0) and
 * join them all before returning. */
typedef void (*worker_fn)(void *arg, int worker);

struct worker_args { worker_fn fn; void *arg; int worker; };

inline void *worker_trampoline(void *p)
{
    worker_args *a = (worker_args *)p;
    a->fn(a->arg, a->worker);
    return NULL;
}

inline void run_workers(int nworkers, worker_fn fn, void *arg)
{
    if (nworkers <= 1) { fn(arg, 0); return; }
    pthread_t *tids = new pthread_t[nworkers];
    worker_args *args = new worker_args[nworkers];
    for (int i = 1; i < nworkers; i++) {
        args[i].fn = fn; args[i].arg = arg; args[i].worker = i;
        if (pthread_create(&tids[i], NULL, worker_trampoline, &args[i]) != 0) abort();
    }
    fn(arg, 0);
    for (int i = 1; i < nworkers; i++) pthread_join(tids[i], NULL);
    delete[] tids;
    delete[] args;
}

/* Hand out the integers [0, n) to concurrent callers, one at a time. */
struct ticket_counter {
    pthread_mutex_t m;
    long next, n;
    ticket_counter(long n_) : next(0), n(n_) { pthread_mutex_init(&m, NULL); }
    ~ticket_counter() { pthread_mutex_destroy(&m); }
    bool take(long &out)
    {
        pthread_mutex_lock(&m);
        bool ok = next < n;
        if (ok) out = next++;
        pthread_mutex_unlock(&m);
        return ok;
    }
};

} // namespace shim
} // namespace tbb
