// TEST INFRASTRUCTURE ONLY: host stand-in for Kokkos::UnorderedMap<Key, void>
// (a set of keys in a fixed-capacity open-addressed table) as the reference's
// WENO cell selector uses it: insert (thread safe, fails when the table is
// full), capacity, valid_at / key_at over slots, clear, rehash.  Copies share one
// table, as Kokkos containers do.
#ifndef KFVM_REFSHIM_KOKKOS_UNORDEREDMAP_HPP
#define KFVM_REFSHIM_KOKKOS_UNORDEREDMAP_HPP

#include "Kokkos_Core.hpp"

namespace Kokkos {

struct UnorderedMapInsertResult {
  int code = 0;  // 0 success, 1 existing, 2 failed
  bool success() const { return code == 0; }
  bool existing() const { return code == 1; }
  bool failed() const { return code == 2; }
};

template <class Key, class Value, class Space = HostSpace>
class UnorderedMap {
  struct Table {
    std::vector<Key> keys;
    std::vector<unsigned char> used;
    uint32_t count = 0;
    std::mutex mtx;
  };
  std::shared_ptr<Table> m_track;
  Table *m_t = nullptr;

  // Capacity for a requested size, rounded up as Kokkos rounds it (7/6 of the
  // request in blocks of 128).
  static uint32_t capacity_for(uint32_t n) {
    if (n == 0) return 128u;
    return static_cast<uint32_t>(((7ull * n / 6) + 127u) / 128u * 128u);
  }

 public:
  explicit UnorderedMap(uint32_t capacity_hint = 0) {
    m_track = std::make_shared<Table>();
    m_t = m_track.get();
    reset(capacity_for(capacity_hint));
  }
  UnorderedMap(const UnorderedMap &o) : m_t(o.m_t) {
    if (!Impl::in_parallel()) m_track = o.m_track;
  }
  UnorderedMap &operator=(const UnorderedMap &o) {
    m_t = o.m_t;
    if (!Impl::in_parallel()) {
      m_track = o.m_track;
    } else {
      m_track.reset();
    }
    return *this;
  }

  void reset(uint32_t cap) {
    m_t->keys.assign(cap, Key());
    m_t->used.assign(cap, 0);
    m_t->count = 0;
  }

  uint32_t capacity() const { return static_cast<uint32_t>(m_t->keys.size()); }
  uint32_t size() const { return m_t->count; }
  void clear() {
    std::fill(m_t->used.begin(), m_t->used.end(), 0);
    m_t->count = 0;
  }
  bool rehash(uint32_t n) {
    uint32_t cap = capacity_for(std::max(n, m_t->count));
    std::vector<Key> old;
    for (uint32_t i = 0; i < capacity(); i++)
      if (m_t->used[i]) old.push_back(m_t->keys[i]);
    reset(cap);
    for (auto k : old) insert(k);
    return true;
  }

  UnorderedMapInsertResult insert(Key k) const {
    UnorderedMapInsertResult r;
    std::lock_guard<std::mutex> lock(m_t->mtx);
    const uint32_t cap = capacity();
    if (cap == 0) {
      r.code = 2;
      return r;
    }
    uint64_t h = static_cast<uint64_t>(k) * 0x9E3779B97F4A7C15ull;
    uint32_t s = static_cast<uint32_t>((h >> 17) % cap);
    for (uint32_t probe = 0; probe < cap; probe++) {
      uint32_t i = (s + probe) % cap;
      if (!m_t->used[i]) {
        m_t->used[i] = 1;
        m_t->keys[i] = k;
        m_t->count++;
        r.code = 0;
        return r;
      }
      if (m_t->keys[i] == k) {
        r.code = 1;
        return r;
      }
    }
    r.code = 2;
    return r;
  }

  bool valid_at(uint32_t i) const { return i < capacity() && m_t->used[i]; }
  Key key_at(uint32_t i) const { return m_t->keys[i]; }
  bool exists(Key k) const {
    for (uint32_t i = 0; i < capacity(); i++)
      if (m_t->used[i] && m_t->keys[i] == k) return true;
    return false;
  }
};

} // namespace Kokkos

#endif
