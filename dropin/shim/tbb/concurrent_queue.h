/* TBB shim: concurrent_bounded_queue (mutex + condition variables). */
#pragma once
#include <pthread.h>
#include <deque>
#include <stddef.h>
namespace tbb {
template <typename T>
class concurrent_bounded_queue {
    std::deque<T> q;
    ptrdiff_t cap;
    pthread_mutex_t m;
    pthread_cond_t not_empty, not_full;
    concurrent_bounded_queue(const concurrent_bounded_queue &);
    concurrent_bounded_queue &operator=(const concurrent_bounded_queue &);
public:
    concurrent_bounded_queue() : q(), cap(-1)
    {
        pthread_mutex_init(&m, NULL);
        pthread_cond_init(&not_empty, NULL);
        pthread_cond_init(&not_full, NULL);
    }
    ~concurrent_bounded_queue()
    {
        pthread_cond_destroy(&not_full);
        pthread_cond_destroy(&not_empty);
        pthread_mutex_destroy(&m);
    }
    void set_capacity(ptrdiff_t c) { pthread_mutex_lock(&m); cap = c; pthread_mutex_unlock(&m); }
    void push(const T &v)
    {
        pthread_mutex_lock(&m);
        while (cap >= 0 && (ptrdiff_t)q.size() >= cap) pthread_cond_wait(&not_full, &m);
        q.push_back(v);
        pthread_cond_signal(&not_empty);
        pthread_mutex_unlock(&m);
    }
    void pop(T &v)
    {
        pthread_mutex_lock(&m);
        while (q.empty()) pthread_cond_wait(&not_empty, &m);
        v = q.front(); q.pop_front();
        pthread_cond_signal(&not_full);
        pthread_mutex_unlock(&m);
    }
    bool try_pop(T &v)
    {
        pthread_mutex_lock(&m);
        bool ok = !q.empty();
        if (ok) { v = q.front(); q.pop_front(); pthread_cond_signal(&not_full); }
        pthread_mutex_unlock(&m);
        return ok;
    }
    bool pop_if_present(T &v) { return try_pop(v); }
    ptrdiff_t size() const { return (ptrdiff_t)q.size(); }
    bool empty() const { return q.empty(); }
};
}
