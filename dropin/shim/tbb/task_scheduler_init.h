/* TBB shim: task_scheduler_init sets the worker count used by the shim. */
#pragma once
#include "_pool.h"
namespace tbb {
class task_scheduler_init {
public:
    static const int automatic = -1;
    explicit task_scheduler_init(int n = automatic)
    {
        if (n > 0) shim::thread_count_ref() = n;
    }
    static int default_num_threads() { return shim::thread_count(); }
};
}
