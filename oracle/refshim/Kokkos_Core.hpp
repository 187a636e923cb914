// TEST INFRASTRUCTURE ONLY: a host-only stand-in for the parts of Kokkos that the
// reference solver's src/ uses, so that the reference's own sources compile and
// run unchanged on the CPU (the reference build in oracle/_ref is the checker
// that pins the oracle restatement).  Written from Kokkos' documented semantics:
//  * View: reference-counted, zero-initialised arrays with mixed dynamic/static
//    extents (dynamic dimensions first), LayoutLeft / LayoutRight / strided;
//    copies alias the same memory; subview with integer, ALL and pair arguments.
//  * parallel_for / parallel_reduce over RangePolicy and MDRangePolicy (OpenMP
//    over the outermost index); reductions overwrite their result with the
//    reduction over all iterations (Sum / Max / Min, plain scalars are sums);
//    per-thread partial results are joined in thread order.
//  * reference counting is switched off inside parallel dispatch, as Kokkos
//    does, so per-iteration subviews do not contend on a shared counter.
// Nothing in the product library includes or links this file.
#ifndef KFVM_REFSHIM_KOKKOS_CORE_HPP
#define KFVM_REFSHIM_KOKKOS_CORE_HPP

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline __attribute__((always_inline))
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [ =, *this ]

namespace Kokkos {

// ---------------------------------------------------------------- spaces, layouts
struct HostSpace {};
struct SharedHostPinnedSpace {};
struct Serial {
  using memory_space = HostSpace;
  using execution_space = Serial;
};
struct OpenMP {
  using memory_space = HostSpace;
  using execution_space = OpenMP;
};
using DefaultHostExecutionSpace = OpenMP;
using DefaultExecutionSpace = OpenMP;

struct LayoutLeft {};
struct LayoutRight {};
struct LayoutStride {};

inline void initialize(int &, char **) {}
inline void initialize() {}
inline void finalize() {}
inline void fence() {}
inline void fence(const std::string &) {}

namespace Profiling {
inline void pushRegion(const std::string &) {}
inline void popRegion() {}
} // namespace Profiling

// ---------------------------------------------------------------- math, pairs, arrays
using std::abs;
using std::atan;
using std::cbrt;
using std::cos;
using std::exp;
using std::fabs;
using std::fmax;
using std::fmin;
using std::isinf;
using std::isnan;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;
using std::tanh;

template <class T1, class T2>
struct pair {
  T1 first;
  T2 second;
  pair() = default;
  pair(T1 a, T2 b) : first(a), second(b) {}
};
template <class T1, class T2>
inline pair<T1, T2> make_pair(T1 a, T2 b) {
  return pair<T1, T2>(a, b);
}

template <class T, std::size_t N>
struct Array {
  T m_data[N];
  KOKKOS_INLINE_FUNCTION T &operator[](std::size_t i) { return m_data[i]; }
  KOKKOS_INLINE_FUNCTION const T &operator[](std::size_t i) const { return m_data[i]; }
  static constexpr std::size_t size() { return N; }
  T *data() { return m_data; }
  const T *data() const { return m_data; }
};

struct ALL_t {};
inline constexpr ALL_t ALL{};

namespace Impl {
// Reference counting is suspended while a parallel dispatch runs.
inline bool &in_parallel() {
  static thread_local bool flag = false;
  return flag;
}
struct ParallelScope {
  bool prev;
  ParallelScope() : prev(in_parallel()) { in_parallel() = true; }
  ~ParallelScope() { in_parallel() = prev; }
};

template <class T>
struct ptr_count {
  static constexpr int n = 0;
  using base = T;
};
template <class T>
struct ptr_count<T *> {
  static constexpr int n = 1 + ptr_count<T>::n;
  using base = typename ptr_count<T>::base;
};

// Kokkos data type: "T**[A][B]" = dynamic dimensions (pointers) first, then the
// static ones in order.
template <class DT>
struct analyze {
  using noext = std::remove_all_extents_t<DT>;
  static constexpr int rank_static = std::rank_v<DT>;
  static constexpr int rank_dynamic = ptr_count<noext>::n;
  static constexpr int rank = rank_static + rank_dynamic;
  using value_type = typename ptr_count<noext>::base;
  template <std::size_t... I>
  static void fill_static(std::size_t *out, std::index_sequence<I...>) {
    ((out[I] = std::extent_v<DT, I>), ...);
  }
  static void static_extents(std::size_t *out) {
    fill_static(out, std::make_index_sequence<rank_static>{});
  }
};

template <class T, int N>
struct add_ptrs {
  using type = typename add_ptrs<T *, N - 1>::type;
};
template <class T>
struct add_ptrs<T, 0> {
  using type = T;
};

template <class... P>
struct pick_layout {
  using type = LayoutRight;
};
template <class... P>
struct pick_layout<LayoutLeft, P...> {
  using type = LayoutLeft;
};
template <class... P>
struct pick_layout<LayoutRight, P...> {
  using type = LayoutRight;
};
template <class... P>
struct pick_layout<LayoutStride, P...> {
  using type = LayoutStride;
};
template <class H, class... P>
struct pick_layout<H, P...> {
  using type = typename pick_layout<P...>::type;
};
} // namespace Impl

// ---------------------------------------------------------------- View
template <class DT, class... P>
class View {
 public:
  using A = Impl::analyze<DT>;
  using value_type = typename A::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using data_type = DT;
  using array_layout = typename Impl::pick_layout<P...>::type;
  using memory_space = HostSpace;
  using execution_space = OpenMP;
  using HostMirror = View<DT, array_layout, HostSpace>;
  static constexpr int Rank = A::rank;
  static constexpr int rank_dynamic = A::rank_dynamic;
  static constexpr unsigned rank = A::rank;

  value_type *m_ptr = nullptr;
  std::size_t m_ext[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::size_t m_str[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::shared_ptr<void> m_track;
  const char *m_label = "";

  View() = default;

  // Allocating constructor: label plus the dynamic extents.
  template <class... I, class = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  explicit View(const std::string &label, I... n) {
    static_assert(sizeof...(I) <= A::rank_dynamic || sizeof...(I) == A::rank,
                  "wrong extent count");
    std::size_t dyn[] = {static_cast<std::size_t>(n)..., 0};
    std::size_t st[8] = {0};
    A::static_extents(st);
    if constexpr (sizeof...(I) == A::rank && A::rank_static > 0 &&
                  A::rank_dynamic != A::rank) {
      for (int r = 0; r < A::rank; r++) m_ext[r] = dyn[r];
    } else {
      for (int r = 0; r < A::rank_dynamic; r++)
        m_ext[r] = r < int(sizeof...(I)) ? dyn[r] : 0;
      for (int r = 0; r < A::rank_static; r++) m_ext[A::rank_dynamic + r] = st[r];
    }
    allocate(label);
  }

  // Unmanaged view of existing memory.
  template <class... I, class = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  View(value_type *p, I... n) {
    std::size_t dyn[] = {static_cast<std::size_t>(n)..., 0};
    std::size_t st[8] = {0};
    A::static_extents(st);
    for (int r = 0; r < A::rank_dynamic; r++) m_ext[r] = dyn[r];
    for (int r = 0; r < A::rank_static; r++) m_ext[A::rank_dynamic + r] = st[r];
    set_contiguous_strides();
    m_ptr = p;
  }

  View(const View &o) { copy_from(o); }
  View &operator=(const View &o) {
    if (this != &o) copy_from(o);
    return *this;
  }
  // Any view of the same rank and element type converts (layout checks are not modelled).
  template <class DT2, class... P2,
            class = std::enable_if_t<Impl::analyze<DT2>::rank == A::rank &&
                                     std::is_convertible_v<
                                         typename Impl::analyze<DT2>::value_type *,
                                         value_type *>>>
  View(const View<DT2, P2...> &o) {
    copy_from(o);
  }
  template <class DT2, class... P2,
            class = std::enable_if_t<Impl::analyze<DT2>::rank == A::rank>>
  View &operator=(const View<DT2, P2...> &o) {
    copy_from(o);
    return *this;
  }

  template <class V>
  void copy_from(const V &o) {
    m_ptr = o.m_ptr;
    for (int r = 0; r < 8; r++) {
      m_ext[r] = o.m_ext[r];
      m_str[r] = o.m_str[r];
    }
    m_label = o.m_label;
    if (!Impl::in_parallel()) {
      m_track = o.m_track;
    } else {
      m_track.reset();
    }
  }

  void set_contiguous_strides() {
    if constexpr (std::is_same_v<array_layout, LayoutLeft>) {
      std::size_t s = 1;
      for (int r = 0; r < A::rank; r++) {
        m_str[r] = s;
        s *= m_ext[r];
      }
    } else {
      std::size_t s = 1;
      for (int r = A::rank - 1; r >= 0; r--) {
        m_str[r] = s;
        s *= m_ext[r];
      }
    }
  }

  void allocate(const std::string &label) {
    set_contiguous_strides();
    std::size_t n = span_count();
    auto *mem = new non_const_value_type[n > 0 ? n : 1]();
    m_track = std::shared_ptr<void>(mem, [](void *q) {
      delete[] static_cast<non_const_value_type *>(q);
    });
    m_ptr = mem;
    auto *lbl = new std::string(label);  // kept for the lifetime of the program
    m_label = lbl->c_str();
  }

  std::size_t span_count() const {
    std::size_t n = 1;
    for (int r = 0; r < A::rank; r++) n *= m_ext[r];
    return n;
  }

  template <class... I>
  KOKKOS_FORCEINLINE_FUNCTION value_type &operator()(I... idx) const {
    static_assert(sizeof...(I) == A::rank || (A::rank == 0 && sizeof...(I) == 0),
                  "wrong index count");
    std::size_t off = 0;
    int r = 0;
    ((off += static_cast<std::size_t>(idx) * m_str[r++]), ...);
    return m_ptr[off];
  }
  template <class I>
  KOKKOS_FORCEINLINE_FUNCTION value_type &operator[](I i) const {
    return m_ptr[static_cast<std::size_t>(i) * m_str[0]];
  }
  KOKKOS_INLINE_FUNCTION std::size_t extent(int r) const { return m_ext[r]; }
  KOKKOS_INLINE_FUNCTION int extent_int(int r) const { return int(m_ext[r]); }
  KOKKOS_INLINE_FUNCTION std::size_t stride(int r) const { return m_str[r]; }
  KOKKOS_INLINE_FUNCTION std::size_t size() const { return span_count(); }
  KOKKOS_INLINE_FUNCTION std::size_t span() const { return span_count(); }
  KOKKOS_INLINE_FUNCTION value_type *data() const { return m_ptr; }
  std::string label() const { return std::string(m_label); }
  bool is_allocated() const { return m_ptr != nullptr; }
  long use_count() const { return m_track.use_count(); }
};

template <class V>
using view_value_t = typename V::value_type;

// ---------------------------------------------------------------- subview
namespace Impl {
template <class T>
struct is_range : std::false_type {};
template <class A, class B>
struct is_range<Kokkos::pair<A, B>> : std::true_type {};
template <class A, class B>
struct is_range<std::pair<A, B>> : std::true_type {};
template <>
struct is_range<ALL_t> : std::true_type {};

template <class... Args>
constexpr int kept_dims() {
  return (0 + ... + (is_range<std::decay_t<Args>>::value ? 1 : 0));
}

template <class V>
struct sub_state {
  std::size_t off = 0;
  int out = 0;
  std::size_t ext[8];
  std::size_t str[8];
};

template <class V, class S>
void sub_arg(const V &v, S &s, int r, ALL_t) {
  s.ext[s.out] = v.m_ext[r];
  s.str[s.out] = v.m_str[r];
  s.out++;
}
template <class V, class S, class A, class B>
void sub_arg(const V &v, S &s, int r, const Kokkos::pair<A, B> &p) {
  s.off += static_cast<std::size_t>(p.first) * v.m_str[r];
  s.ext[s.out] = static_cast<std::size_t>(p.second - p.first);
  s.str[s.out] = v.m_str[r];
  s.out++;
}
template <class V, class S, class A, class B>
void sub_arg(const V &v, S &s, int r, const std::pair<A, B> &p) {
  s.off += static_cast<std::size_t>(p.first) * v.m_str[r];
  s.ext[s.out] = static_cast<std::size_t>(p.second - p.first);
  s.str[s.out] = v.m_str[r];
  s.out++;
}
template <class V, class S, class I, class = std::enable_if_t<std::is_integral_v<I>>>
void sub_arg(const V &v, S &s, int r, I i) {
  s.off += static_cast<std::size_t>(i) * v.m_str[r];
}
} // namespace Impl

template <class DT, class... P, class... Args>
auto subview(const View<DT, P...> &v, Args... args) {
  using V = View<DT, P...>;
  static_assert(sizeof...(Args) == V::Rank, "subview needs one argument per dimension");
  constexpr int R = Impl::kept_dims<Args...>();
  using T = typename V::value_type;
  using Out = View<typename Impl::add_ptrs<T, R>::type, LayoutStride, HostSpace>;
  Impl::sub_state<V> s;
  int r = 0;
  ((Impl::sub_arg(v, s, r++, args)), ...);
  Out o;
  o.m_ptr = v.m_ptr + s.off;
  for (int q = 0; q < R; q++) {
    o.m_ext[q] = s.ext[q];
    o.m_str[q] = s.str[q];
  }
  o.m_label = v.m_label;
  if (!Impl::in_parallel()) o.m_track = v.m_track;
  return o;
}

// ---------------------------------------------------------------- mirrors, copies
template <class DT, class... P>
auto create_mirror(const View<DT, P...> &v) {
  using V = View<DT, P...>;
  using L = std::conditional_t<std::is_same_v<typename V::array_layout, LayoutLeft>,
                               LayoutLeft, LayoutRight>;
  using T = typename V::non_const_value_type;
  using Out = View<typename Impl::add_ptrs<T, V::Rank>::type, L, HostSpace>;
  Out o;
  for (int r = 0; r < V::Rank; r++) o.m_ext[r] = v.m_ext[r];
  o.allocate(v.label());
  return o;
}
template <class DT, class... P>
auto create_mirror_view(const View<DT, P...> &v) {
  return create_mirror(v);
}
template <class Space, class DT, class... P>
auto create_mirror_view_and_copy(const Space &, const View<DT, P...> &v) {
  auto m = create_mirror(v);
  deep_copy(m, v);
  return m;
}

namespace Impl {
template <class F>
void for_each_index(const std::size_t *ext, int rank, F &&f) {
  std::size_t idx[8] = {0};
  std::size_t total = 1;
  for (int r = 0; r < rank; r++) total *= ext[r];
  if (total == 0) return;
  for (std::size_t n = 0; n < total; n++) {
    f(idx);
    for (int r = rank - 1; r >= 0; r--) {
      if (++idx[r] < ext[r]) break;
      idx[r] = 0;
    }
  }
}
} // namespace Impl

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...> &dst, const View<D2, P2...> &src) {
  using V1 = View<D1, P1...>;
  static_assert(V1::Rank == View<D2, P2...>::Rank, "deep_copy rank mismatch");
  for (int r = 0; r < V1::Rank; r++) {
    if (dst.m_ext[r] != src.m_ext[r]) {
      std::fprintf(stderr, "Kokkos shim: deep_copy extent mismatch\n");
      std::abort();
    }
  }
  if (dst.m_ptr == src.m_ptr) return;
  Impl::for_each_index(dst.m_ext, V1::Rank, [&](const std::size_t *i) {
    std::size_t od = 0, os = 0;
    for (int r = 0; r < V1::Rank; r++) {
      od += i[r] * dst.m_str[r];
      os += i[r] * src.m_str[r];
    }
    dst.m_ptr[od] = src.m_ptr[os];
  });
}
template <class D1, class... P1, class S,
          class = std::enable_if_t<std::is_arithmetic_v<S>>>
void deep_copy(const View<D1, P1...> &dst, const S &val) {
  using V1 = View<D1, P1...>;
  Impl::for_each_index(dst.m_ext, V1::Rank, [&](const std::size_t *i) {
    std::size_t od = 0;
    for (int r = 0; r < V1::Rank; r++) od += i[r] * dst.m_str[r];
    dst.m_ptr[od] = static_cast<typename V1::non_const_value_type>(val);
  });
}
template <class E, class D1, class... P1, class Src>
void deep_copy(const E &, const View<D1, P1...> &dst, const Src &src) {
  deep_copy(dst, src);
}

template <class DT, class... P, class... I>
void realloc(View<DT, P...> &v, I... n) {
  v = View<DT, P...>(v.label(), n...);
}
template <class DT, class... P, class... I>
void resize(View<DT, P...> &v, I... n) {
  View<DT, P...> w(v.label(), n...);
  // keep the overlapping part (rank-1 views only are resized by the solver)
  std::size_t m = std::min(v.m_ptr ? v.m_ext[0] : 0, w.m_ext[0]);
  for (std::size_t i = 0; i < m; i++) w.m_ptr[i * w.m_str[0]] = v.m_ptr[i * v.m_str[0]];
  v = w;
}

// ---------------------------------------------------------------- policies
template <class T>
struct IndexType {
  using type = T;
};
template <unsigned N>
struct Rank {
  static constexpr unsigned rank = N;
};

template <class... P>
struct RangePolicy {
  int64_t lo, hi;
  RangePolicy(int64_t l, int64_t h) : lo(l), hi(h) {}
  template <class E>
  RangePolicy(const E &, int64_t l, int64_t h) : lo(l), hi(h) {}
};

namespace Impl {
template <class... P>
struct md_rank {
  static constexpr unsigned value = 0;
};
template <unsigned N, class... P>
struct md_rank<Rank<N>, P...> {
  static constexpr unsigned value = N;
};
template <class H, class... P>
struct md_rank<H, P...> {
  static constexpr unsigned value = md_rank<P...>::value;
};
} // namespace Impl

template <class... P>
struct MDRangePolicy {
  static constexpr unsigned R = Impl::md_rank<P...>::value;
  int64_t lo[8] = {0}, hi[8] = {0};
  MDRangePolicy(std::initializer_list<int64_t> l, std::initializer_list<int64_t> h) {
    set(l, h);
  }
  MDRangePolicy(std::initializer_list<int64_t> l, std::initializer_list<int64_t> h,
                std::initializer_list<int64_t>) {
    set(l, h);
  }
  template <class T, std::size_t N>
  MDRangePolicy(const Array<T, N> &l, const Array<T, N> &h) {
    for (std::size_t r = 0; r < N; r++) {
      lo[r] = l[r];
      hi[r] = h[r];
    }
  }
  void set(std::initializer_list<int64_t> l, std::initializer_list<int64_t> h) {
    int r = 0;
    for (auto v : l) lo[r++] = v;
    r = 0;
    for (auto v : h) hi[r++] = v;
  }
};

// ---------------------------------------------------------------- reducers
template <class T>
struct reduction_identity {
  static T sum() { return T(0); }
  static T max() { return std::numeric_limits<T>::lowest(); }
  static T min() { return std::numeric_limits<T>::max(); }
};

template <class T>
struct Sum {
  using value_type = T;
  T &ref;
  explicit Sum(T &r) : ref(r) {}
  static T identity() { return reduction_identity<T>::sum(); }
  static void join(T &a, const T &b) { a += b; }
  T &reference() const { return ref; }
};
template <class T>
struct Max {
  using value_type = T;
  T &ref;
  explicit Max(T &r) : ref(r) {}
  static T identity() { return reduction_identity<T>::max(); }
  static void join(T &a, const T &b) {
    if (b > a) a = b;
  }
  T &reference() const { return ref; }
};
template <class T>
struct Min {
  using value_type = T;
  T &ref;
  explicit Min(T &r) : ref(r) {}
  static T identity() { return reduction_identity<T>::min(); }
  static void join(T &a, const T &b) {
    if (b < a) a = b;
  }
  T &reference() const { return ref; }
};

namespace Impl {
template <class T>
struct is_reducer : std::false_type {};
template <class T>
struct is_reducer<Sum<T>> : std::true_type {};
template <class T>
struct is_reducer<Max<T>> : std::true_type {};
template <class T>
struct is_reducer<Min<T>> : std::true_type {};

template <class R>
auto as_reducer(R &r) {
  if constexpr (is_reducer<std::remove_const_t<R>>::value) {
    return r;
  } else {
    return Sum<R>(r);
  }
}

inline int num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
inline int thread_id() {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

// Static partition of [lo, hi) over the threads of the team.
inline void share(int64_t lo, int64_t hi, int nt, int t, int64_t &a, int64_t &b) {
  int64_t n = hi - lo;
  int64_t q = n / nt, rem = n % nt;
  a = lo + t * q + std::min<int64_t>(t, rem);
  b = a + q + (t < rem ? 1 : 0);
}

template <unsigned R, class F, class... V>
void md_loop(const int64_t *lo, const int64_t *hi, int64_t a, int64_t b, const F &f,
             V &...vals) {
  if constexpr (R == 1) {
    for (int64_t i = a; i < b; i++) f(i, vals...);
  } else if constexpr (R == 2) {
    for (int64_t i = a; i < b; i++)
      for (int64_t j = lo[1]; j < hi[1]; j++) f(i, j, vals...);
  } else if constexpr (R == 3) {
    for (int64_t i = a; i < b; i++)
      for (int64_t j = lo[1]; j < hi[1]; j++)
        for (int64_t k = lo[2]; k < hi[2]; k++) f(i, j, k, vals...);
  } else if constexpr (R == 4) {
    for (int64_t i = a; i < b; i++)
      for (int64_t j = lo[1]; j < hi[1]; j++)
        for (int64_t k = lo[2]; k < hi[2]; k++)
          for (int64_t l = lo[3]; l < hi[3]; l++) f(i, j, k, l, vals...);
  } else {
    static_assert(R >= 1 && R <= 4, "MDRangePolicy rank not supported by the shim");
  }
}

template <class Pol>
struct range_of;
template <class... P>
struct range_of<RangePolicy<P...>> {
  static constexpr unsigned R = 1;
  static void get(const RangePolicy<P...> &p, int64_t *lo, int64_t *hi) {
    lo[0] = p.lo;
    hi[0] = p.hi;
  }
};
template <class... P>
struct range_of<MDRangePolicy<P...>> {
  static constexpr unsigned R = MDRangePolicy<P...>::R;
  static void get(const MDRangePolicy<P...> &p, int64_t *lo, int64_t *hi) {
    for (unsigned r = 0; r < R; r++) {
      lo[r] = p.lo[r];
      hi[r] = p.hi[r];
    }
  }
};

template <class Pol>
auto normalise(const Pol &p) {
  if constexpr (std::is_integral_v<Pol>) {
    return RangePolicy<>(0, int64_t(p));
  } else {
    return p;
  }
}

template <class Pol, class F>
void run_for(const Pol &pol0, const F &f) {
  auto pol = normalise(pol0);
  using RO = range_of<decltype(pol)>;
  int64_t lo[8], hi[8];
  RO::get(pol, lo, hi);
  for (unsigned r = 0; r < RO::R; r++)
    if (hi[r] <= lo[r]) return;
#pragma omp parallel
  {
    ParallelScope scope;
    int64_t a, b;
    share(lo[0], hi[0], num_threads(), thread_id(), a, b);
    md_loop<RO::R>(lo, hi, a, b, f);
  }
}

template <class Pol, class F, class... Red>
void run_reduce(const Pol &pol0, const F &f, Red... red) {
  auto pol = normalise(pol0);
  using RO = range_of<decltype(pol)>;
  int64_t lo[8], hi[8];
  RO::get(pol, lo, hi);
  using Vals = std::tuple<typename Red::value_type...>;
  const int nt = num_threads();
  std::vector<Vals> part(nt, Vals(Red::identity()...));
  bool empty = false;
  for (unsigned r = 0; r < RO::R; r++)
    if (hi[r] <= lo[r]) empty = true;
  if (!empty) {
#pragma omp parallel num_threads(nt)
    {
      ParallelScope scope;
      const int t = thread_id();
      int64_t a, b;
      share(lo[0], hi[0], nt, t, a, b);
      std::apply([&](auto &...v) { md_loop<RO::R>(lo, hi, a, b, f, v...); }, part[t]);
    }
  }
  Vals acc(Red::identity()...);
  for (int t = 0; t < nt; t++) {
    std::apply(
        [&](auto &...av) {
          std::apply(
              [&](const auto &...pv) {
                (Red::join(av, pv), ...);
              },
              part[t]);
        },
        acc);
  }
  std::apply([&](const auto &...av) { ((red.reference() = av), ...); }, acc);
}
} // namespace Impl

template <class Pol, class F>
void parallel_for(const std::string &, const Pol &pol, const F &f) {
  Impl::run_for(pol, f);
}
template <class Pol, class F>
void parallel_for(const Pol &pol, const F &f) {
  Impl::run_for(pol, f);
}

template <class Pol, class F, class... R>
void parallel_reduce(const std::string &, const Pol &pol, const F &f, R &&...r) {
  Impl::run_reduce(pol, f, Impl::as_reducer(r)...);
}
template <class Pol, class F, class R0, class... R,
          class = std::enable_if_t<!std::is_convertible_v<Pol, std::string>>>
void parallel_reduce(const Pol &pol, const F &f, R0 &&r0, R &&...r) {
  Impl::run_reduce(pol, f, Impl::as_reducer(r0), Impl::as_reducer(r)...);
}

} // namespace Kokkos

#include "Kokkos_UnorderedMap.hpp"

#endif
