// Kokkos_Core.hpp — a minimal host-only stand-in for the parts of the Kokkos
// API that the reference (euphoricpoptarts/UnitigCoarsening) uses, written
// from Kokkos's public documentation so the reference's own sources compile
// unmodified into a CPU program.  TEST INFRASTRUCTURE ONLY: it builds the
// reference driver for the parity pin and the CPU baseline; nothing in the
// product links it.
//
// Two modes: OpenMP (default; parallel_for/scan/reduce spread over threads)
// and serial (-DKSHIM_SERIAL; every loop in index order, so the reference's
// compare-and-swap races resolve deterministically).
#pragma once

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#if !defined(KSHIM_SERIAL)
#include <omp.h>
#endif

#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION

namespace Kokkos {

// ---------------------------------------------------------------- spaces
struct HostSpace {
  using memory_space = HostSpace;
};
struct OpenMP {
  using execution_space = OpenMP;
  using memory_space = HostSpace;
  using size_type = std::size_t;
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;

template <class Exec, class Mem>
struct Device {
  using execution_space = Exec;
  using memory_space = Mem;
};

enum MemoryTraitsFlags : unsigned { Unmanaged = 0x01, RandomAccess = 0x02, Atomic = 0x04, Restrict = 0x08 };
template <unsigned T>
struct MemoryTraits {};
template <class T>
struct IndexType {};

struct AUTO_t {};
constexpr AUTO_t AUTO{};

inline void initialize() {}
inline void initialize(int&, char**) {}
inline void finalize() {}

inline int shim_threads() {
#if defined(KSHIM_SERIAL)
  return 1;
#else
  return omp_get_max_threads();
#endif
}
inline int shim_thread_id() {
#if defined(KSHIM_SERIAL)
  return 0;
#else
  return omp_get_thread_num();
#endif
}

// ----------------------------------------------------------------- views
struct ViewAllocateWithoutInitializing {
  std::string label;
  ViewAllocateWithoutInitializing(const std::string& l) : label(l) {}
  ViewAllocateWithoutInitializing(const char* l) : label(l) {}
};

template <class D>
struct view_data;
template <class T>
struct view_data<T*> {
  using value_type = T;
  static constexpr int rank = 1;
};
template <class T>
struct view_data {
  using value_type = T;
  static constexpr int rank = 0;
};

template <class D, class... P>
class View;

template <class D, class... P>
class View {
 public:
  using data_type = D;
  using value_type = typename view_data<D>::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using reference_type = value_type&;
  static constexpr int Rank = view_data<D>::rank;
  using non_const_data_type = std::conditional_t<Rank == 1, non_const_value_type*, non_const_value_type>;
  using HostMirror = View<non_const_data_type, HostSpace>;
  using memory_space = HostSpace;
  using execution_space = OpenMP;
  using size_type = std::size_t;

  View() = default;
  // rank 1 allocation (zero filled) / without initialization
  View(const std::string& label, std::size_t n) { alloc(n, true); (void)label; }
  View(const char* label, std::size_t n) { alloc(n, true); (void)label; }
  View(const ViewAllocateWithoutInitializing& a, std::size_t n) { alloc(n, false); (void)a; }
  // rank 0 allocation
  explicit View(const std::string& label) { alloc(1, true); (void)label; }
  explicit View(const char* label) { alloc(1, true); (void)label; }
  // wrap existing memory (unmanaged)
  View(value_type* p, std::size_t n) : ptr_(const_cast<non_const_value_type*>(p)), n_(n) {}

  template <class D2, class... P2,
            class = std::enable_if_t<std::is_same<typename View<D2, P2...>::non_const_value_type,
                                                  non_const_value_type>::value &&
                                     View<D2, P2...>::Rank == Rank>>
  View(const View<D2, P2...>& o) : own_(o.owner()), ptr_(o.raw()), n_(o.extent(0)) {}

  template <class D2, class... P2>
  View& operator=(const View<D2, P2...>& o) {
    own_ = o.owner();
    ptr_ = o.raw();
    n_ = o.extent(0);
    return *this;
  }

  template <class I>
  inline reference_type operator()(I i) const {
    return ptr_[static_cast<std::size_t>(i)];
  }
  inline reference_type operator()() const { return ptr_[0]; }
  template <class I>
  inline reference_type operator[](I i) const {
    return ptr_[static_cast<std::size_t>(i)];
  }

  std::size_t extent(int r) const { return r == 0 ? (Rank == 1 ? n_ : 1) : 1; }
  std::size_t extent_int(int r) const { return extent(r); }
  std::size_t size() const { return Rank == 1 ? n_ : 1; }
  std::size_t span() const { return size(); }
  value_type* data() const { return ptr_; }
  bool is_allocated() const { return ptr_ != nullptr; }
  std::string label() const { return std::string(); }

  // internals shared by conversions and helpers
  const std::shared_ptr<void>& owner() const { return own_; }
  non_const_value_type* raw() const { return ptr_; }
  void rebind(std::shared_ptr<void> o, non_const_value_type* p, std::size_t n) {
    own_ = std::move(o);
    ptr_ = p;
    n_ = n;
  }

 private:
  void alloc(std::size_t n, bool zero) {
    const std::size_t cnt = n ? n : 1;
    non_const_value_type* p = static_cast<non_const_value_type*>(std::malloc(cnt * sizeof(non_const_value_type)));
    if (!p) throw std::bad_alloc();
    if (zero) std::memset(static_cast<void*>(p), 0, cnt * sizeof(non_const_value_type));
    own_ = std::shared_ptr<void>(p, [](void* q) { std::free(q); });
    ptr_ = p;
    n_ = n;
  }
  std::shared_ptr<void> own_;
  non_const_value_type* ptr_ = nullptr;
  std::size_t n_ = 0;
};

// subview(v, pair) -> rank 1 slice; subview(v, i) -> rank 0 element
template <class D, class... P, class A, class B>
View<D, P...> subview(const View<D, P...>& v, const std::pair<A, B>& r) {
  View<D, P...> s;
  const std::size_t b = static_cast<std::size_t>(r.first), e = static_cast<std::size_t>(r.second);
  s.rebind(v.owner(), v.raw() + b, e - b);
  return s;
}
template <class D, class... P, class I, class = std::enable_if_t<std::is_integral<I>::value>>
View<typename View<D, P...>::value_type, P...> subview(const View<D, P...>& v, I i) {
  View<typename View<D, P...>::value_type, P...> s;
  s.rebind(v.owner(), v.raw() + static_cast<std::size_t>(i), 1);
  return s;
}

// deep_copy: view <- view, view <- scalar (fill), scalar <- rank-0 view
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.raw() == src.raw()) return;
  const std::size_t n = std::min(dst.size(), src.size());
  std::memmove(static_cast<void*>(dst.raw()), static_cast<const void*>(src.raw()),
               n * sizeof(typename View<D1, P1...>::non_const_value_type));
}
template <class D, class... P, class T, class = std::enable_if_t<std::is_arithmetic<T>::value>>
void deep_copy(const View<D, P...>& dst, const T& v) {
  auto* p = dst.raw();
  const std::size_t n = dst.size();
  for (std::size_t i = 0; i < n; ++i) p[i] = static_cast<typename View<D, P...>::non_const_value_type>(v);
}
template <class T, class D, class... P, class = std::enable_if_t<std::is_arithmetic<T>::value>>
void deep_copy(T& dst, const View<D, P...>& src) {
  dst = static_cast<T>(src.raw()[0]);
}

template <class D, class... P>
typename View<D, P...>::HostMirror create_mirror(const View<D, P...>& v) {
  typename View<D, P...>::HostMirror m("mirror", v.size());
  return m;
}
template <class D, class... P>
typename View<D, P...>::HostMirror create_mirror_view(const View<D, P...>& v) {
  typename View<D, P...>::HostMirror m;
  m.rebind(v.owner(), v.raw(), v.size());
  return m;
}
template <class D, class... P>
void resize(View<D, P...>& v, std::size_t n) {
  View<D, P...> nv("resized", n);
  std::memcpy(static_cast<void*>(nv.raw()), static_cast<const void*>(v.raw()),
              std::min(n, v.size()) * sizeof(typename View<D, P...>::non_const_value_type));
  v = nv;
}

// --------------------------------------------------------------- atomics
template <class T>
inline bool atomic_compare_exchange_strong(T* p, T expected, T desired) {
  return __atomic_compare_exchange_n(p, &expected, desired, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline T atomic_fetch_add(T* p, U v) {
  return __atomic_fetch_add(p, static_cast<T>(v), __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline void atomic_add(T* p, U v) {
  __atomic_fetch_add(p, static_cast<T>(v), __ATOMIC_SEQ_CST);
}
template <class T>
inline void atomic_increment(T* p) {
  __atomic_fetch_add(p, static_cast<T>(1), __ATOMIC_SEQ_CST);
}
template <class T, class U>
inline void atomic_or(T* p, U v) {
  __atomic_fetch_or(p, static_cast<T>(v), __ATOMIC_SEQ_CST);
}

// --------------------------------------------------------------- policies
template <class... Args>
struct RangePolicy {
  using execution_space = OpenMP;
  std::int64_t begin_, end_;
  RangePolicy() : begin_(0), end_(0) {}
  template <class A, class B>
  RangePolicy(A b, B e) : begin_(static_cast<std::int64_t>(b)), end_(static_cast<std::int64_t>(e)) {}
};

struct TeamMember {
  std::int64_t league;
  std::int64_t league_rank() const { return league; }
  int team_rank() const { return 0; }
  int team_size() const { return 1; }
  void team_barrier() const {}
};

template <class... Args>
struct TeamPolicy {
  using execution_space = OpenMP;
  using member_type = TeamMember;
  std::int64_t league_;
  template <class L>
  TeamPolicy(L league, AUTO_t) : league_(static_cast<std::int64_t>(league)) {}
  template <class L>
  TeamPolicy(L league, int) : league_(static_cast<std::int64_t>(league)) {}
};

template <class B, class E>
struct TeamThreadRangeBoundaries {
  B b;
  E e;
};
template <class B, class E>
TeamThreadRangeBoundaries<std::common_type_t<B, E>, std::common_type_t<B, E>> TeamThreadRange(const TeamMember&,
                                                                                               B b, E e) {
  return {static_cast<std::common_type_t<B, E>>(b), static_cast<std::common_type_t<B, E>>(e)};
}
template <class C>
TeamThreadRangeBoundaries<C, C> TeamThreadRange(const TeamMember&, C n) {
  return {C(0), n};
}

// ------------------------------------------------------------ parallel_for
template <class F>
inline void shim_range_for(std::int64_t b, std::int64_t e, const F& f) {
#if defined(KSHIM_SERIAL)
  for (std::int64_t i = b; i < e; ++i) f(i);
#else
#pragma omp parallel for schedule(static)
  for (std::int64_t i = b; i < e; ++i) f(i);
#endif
}

template <class I, class F, class = std::enable_if_t<std::is_integral<I>::value>>
void parallel_for(const std::string&, I n, const F& f) {
  shim_range_for(0, static_cast<std::int64_t>(n), f);
}
template <class... A, class F>
void parallel_for(const std::string&, const RangePolicy<A...>& p, const F& f) {
  shim_range_for(p.begin_, p.end_, f);
}
template <class... A, class F>
void parallel_for(const RangePolicy<A...>& p, const F& f) {
  shim_range_for(p.begin_, p.end_, f);
}
template <class... A, class F>
void parallel_for(const std::string&, const TeamPolicy<A...>& p, const F& f) {
#if defined(KSHIM_SERIAL)
  for (std::int64_t i = 0; i < p.league_; ++i) f(TeamMember{i});
#else
#pragma omp parallel for schedule(dynamic, 64)
  for (std::int64_t i = 0; i < p.league_; ++i) f(TeamMember{i});
#endif
}
template <class B, class E, class F>
void parallel_for(const TeamThreadRangeBoundaries<B, E>& r, const F& f) {
  for (B j = r.b; j < r.e; ++j) f(j);
}

// ----------------------------------------------------------- scan / reduce
template <class F>
struct scan_value;
template <class C, class R, class I, class V>
struct scan_value<R (C::*)(I, V&, const bool) const> {
  using type = V;
};
template <class F>
using scan_value_t = typename scan_value<decltype(&F::operator())>::type;

template <class F>
scan_value_t<F> shim_scan(std::int64_t b, std::int64_t e, const F& f) {
  using V = scan_value_t<F>;
#if defined(KSHIM_SERIAL)
  V acc = V();
  for (std::int64_t i = b; i < e; ++i) f(i, acc, true);
  return acc;
#else
  // two passes: per-thread partial sums without side effects (final=false),
  // then each thread's slice again from its exclusive offset (final=true)
  const int nt = omp_get_max_threads();
  std::vector<V> part(nt + 1, V());
  int used = 1;
  const std::int64_t len = e - b;
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const int tn = omp_get_num_threads();
#pragma omp single
    used = tn;
    const std::int64_t lo = b + len * t / tn, hi = b + len * (t + 1) / tn;
    V acc = V();
    for (std::int64_t i = lo; i < hi; ++i) f(i, acc, false);
    part[t + 1] = acc;
#pragma omp barrier
#pragma omp single
    for (int q = 1; q <= tn; ++q) part[q] += part[q - 1];
    V acc2 = part[t];
    for (std::int64_t i = lo; i < hi; ++i) f(i, acc2, true);
  }
  return part[used];
#endif
}

template <class I, class F, class = std::enable_if_t<std::is_integral<I>::value>>
void parallel_scan(const std::string&, I n, const F& f) {
  shim_scan(0, static_cast<std::int64_t>(n), f);
}
template <class I, class F, class R, class = std::enable_if_t<std::is_integral<I>::value>>
void parallel_scan(const std::string&, I n, const F& f, R& result) {
  result = static_cast<R>(shim_scan(0, static_cast<std::int64_t>(n), f));
}
template <class... A, class F>
void parallel_scan(const std::string&, const RangePolicy<A...>& p, const F& f) {
  shim_scan(p.begin_, p.end_, f);
}
template <class... A, class F, class R>
void parallel_scan(const std::string&, const RangePolicy<A...>& p, const F& f, R& result) {
  result = static_cast<R>(shim_scan(p.begin_, p.end_, f));
}

template <class T>
struct reduction_identity {
  static T sum() { return T(); }
};

template <class F, class R>
void shim_reduce(std::int64_t b, std::int64_t e, const F& f, R& result) {
#if defined(KSHIM_SERIAL)
  R acc = reduction_identity<R>::sum();
  for (std::int64_t i = b; i < e; ++i) f(i, acc);
  result = acc;
#else
  R total = reduction_identity<R>::sum();
#pragma omp parallel
  {
    R acc = reduction_identity<R>::sum();
#pragma omp for schedule(static) nowait
    for (std::int64_t i = b; i < e; ++i) f(i, acc);
#pragma omp critical
    total += acc;
  }
  result = total;
#endif
}

template <class I, class F, class R, class = std::enable_if_t<std::is_integral<I>::value>>
void parallel_reduce(const std::string&, I n, const F& f, R& result) {
  shim_reduce(0, static_cast<std::int64_t>(n), f, result);
}
template <class... A, class F, class R>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, R& result) {
  shim_reduce(p.begin_, p.end_, f, result);
}
template <class... A, class F, class R>
void parallel_reduce(const RangePolicy<A...>& p, const F& f, R& result) {
  shim_reduce(p.begin_, p.end_, f, result);
}

// ------------------------------------------------------------------ timer
class Timer {
 public:
  Timer() { reset(); }
  void reset() { t0_ = std::chrono::steady_clock::now(); }
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

 private:
  std::chrono::steady_clock::time_point t0_;
};

}  // namespace Kokkos
