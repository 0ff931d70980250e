/* Oracle shim: minimal stand-in for boost::alignment::aligned_allocator<T, A>,
 * the only Boost.Align facility the reference's hot-path sources use. */
#pragma once
#include <cstddef>
#include <cstdlib>
#include <new>
namespace boost { namespace alignment {
template <class T, std::size_t A>
struct aligned_allocator {
  typedef T value_type;
  template <class U> struct rebind { typedef aligned_allocator<U, A> other; };
  aligned_allocator() noexcept {}
  template <class U> aligned_allocator(const aligned_allocator<U, A>&) noexcept {}
  T* allocate(std::size_t n) {
    std::size_t bytes = ((n * sizeof(T) + A - 1) / A) * A;
    if (bytes == 0) bytes = A;
    void* p = std::aligned_alloc(A, bytes);
    if (!p) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, std::size_t) noexcept { std::free(p); }
  template <class U> bool operator==(const aligned_allocator<U, A>&) const noexcept { return true; }
  template <class U> bool operator!=(const aligned_allocator<U, A>&) const noexcept { return false; }
};
}}
