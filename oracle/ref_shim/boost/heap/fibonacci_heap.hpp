// Shim: see indexed_heap_shim.hpp.
#pragma once
#include "indexed_heap_shim.hpp"
namespace boost { namespace heap {
template <class T> using fibonacci_heap = indexed_heap_shim<T>;
} }
