/* TBB shim: scalable_allocator is a plain std::allocator here. */
#pragma once
#include <memory>
namespace tbb {
template <typename T>
class scalable_allocator : public std::allocator<T> {
public:
    template <typename U> struct rebind { typedef scalable_allocator<U> other; };
    scalable_allocator() throw() {}
    scalable_allocator(const scalable_allocator &a) throw() : std::allocator<T>(a) {}
    template <typename U> scalable_allocator(const scalable_allocator<U> &) throw() {}
};
}
