/* Oracle shim: the hot path never serialises; these names only need to exist. */
#pragma once
#include <cstddef>
namespace boost { namespace serialization {
class access {};
template <class T> inline T* make_array(T* p, std::size_t) { return p; }
template <class B, class D> inline B& base_object(D& d) { return static_cast<B&>(d); }
}}
