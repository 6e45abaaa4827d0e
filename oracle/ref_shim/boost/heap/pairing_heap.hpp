// Shim: see indexed_heap_shim.hpp.
#pragma once
#include "indexed_heap_shim.hpp"
namespace boost { namespace heap {
template <class T> using pairing_heap = indexed_heap_shim<T>;
} }
