// Minimal stand-in for the part of Boost.Heap that the reference's CPU
// programs use (push returning a handle, top, pop, update(handle, value),
// size, empty).  Boost is not installed here; this lets oracle/_ref compile
// the reference's own PrunedDP++ / HOP_cpu sources unchanged.  It is a
// binary max-heap (ordered by the element's operator<, as Boost orders its
// heaps) with position-tracked nodes; ties may pop in a different order than
// Boost's Fibonacci / pairing heaps.  Test infrastructure only.
#pragma once
#include <cstddef>
#include <utility>
#include <vector>

namespace boost {
namespace heap {

template <class T>
class indexed_heap_shim {
  struct node {
    T value;
    std::size_t idx;
  };
  std::vector<node*> h_;

  bool less(std::size_t a, std::size_t b) const { return h_[a]->value < h_[b]->value; }
  void swap_at(std::size_t a, std::size_t b) {
    std::swap(h_[a], h_[b]);
    h_[a]->idx = a;
    h_[b]->idx = b;
  }
  void sift_up(std::size_t i) {
    while (i > 0) {
      std::size_t p = (i - 1) / 2;
      if (!less(p, i)) break;
      swap_at(p, i);
      i = p;
    }
  }
  void sift_down(std::size_t i) {
    for (;;) {
      std::size_t l = 2 * i + 1, r = l + 1, m = i;
      if (l < h_.size() && less(m, l)) m = l;
      if (r < h_.size() && less(m, r)) m = r;
      if (m == i) break;
      swap_at(i, m);
      i = m;
    }
  }

 public:
  struct handle_type {
    node* p = nullptr;
    T& operator*() const { return p->value; }
  };
  indexed_heap_shim() = default;
  indexed_heap_shim(const indexed_heap_shim&) = delete;
  indexed_heap_shim& operator=(const indexed_heap_shim&) = delete;
  ~indexed_heap_shim() {
    for (node* n : h_) delete n;
  }
  handle_type push(const T& v) {
    node* n = new node{v, h_.size()};
    h_.push_back(n);
    sift_up(n->idx);
    return handle_type{n};
  }
  const T& top() const { return h_.front()->value; }
  void pop() {
    node* n = h_.front();
    swap_at(0, h_.size() - 1);
    h_.pop_back();
    if (!h_.empty()) sift_down(0);
    delete n;
  }
  void update(handle_type hd, const T& v) {
    hd.p->value = v;
    sift_up(hd.p->idx);
    sift_down(hd.p->idx);
  }
  std::size_t size() const { return h_.size(); }
  bool empty() const { return h_.empty(); }
};

}  // namespace heap
}  // namespace boost
