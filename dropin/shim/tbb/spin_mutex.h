/* TBB shim: spin_mutex as a pthread mutex. */
#pragma once
#include <pthread.h>
namespace tbb {
class spin_mutex {
    pthread_mutex_t m;
public:
    spin_mutex() { pthread_mutex_init(&m, NULL); }
    ~spin_mutex() { pthread_mutex_destroy(&m); }
    class scoped_lock {
        spin_mutex *mx;
    public:
        scoped_lock() : mx(0) {}
        explicit scoped_lock(spin_mutex &x) : mx(&x) { pthread_mutex_lock(&mx->m); }
        void acquire(spin_mutex &x) { mx = &x; pthread_mutex_lock(&mx->m); }
        void release() { if (mx) pthread_mutex_unlock(&mx->m); mx = 0; }
        ~scoped_lock() { release(); }
    };
};
}
