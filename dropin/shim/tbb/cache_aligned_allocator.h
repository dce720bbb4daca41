/* TBB shim: cache_aligned_allocator is a plain std::allocator here. */
#pragma once
#include <memory>
namespace tbb {
template <typename T>
class cache_aligned_allocator : public std::allocator<T> {
public:
    template <typename U> struct rebind { typedef cache_aligned_allocator<U> other; };
    cache_aligned_allocator() throw() {}
    cache_aligned_allocator(const cache_aligned_allocator &a) throw() : std::allocator<T>(a) {}
    template <typename U> cache_aligned_allocator(const cache_aligned_allocator<U> &) throw() {}
};
}
