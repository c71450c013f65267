// Host-only SYCL subset used to compile the reference PMG path as a CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This header lets g++ build the reference's own
// PBE_pmgc_class.h + pmgc/{matvecd,gsd,buildPd,buildGd,mypdec}.cc unchanged,
// so that tests and the CPU baseline of bench.py can run the reference
// algorithm on host cores. Nothing in the product (multigrid_b200/) includes it.
//
// What it models (only what the reference's hot path uses):
//   queue: parallel_for over range<1..3> with 0..2 reductions, submit +
//          handler::parallel_for/single_task, memcpy, memset, fill, wait,
//          get_device; every call runs synchronously on the calling thread.
//   id<N>, item<N>, range<N>, reduction + plus, malloc_device/shared (zeroed),
//   free, fabs, selectors, property_list, printf.
//
// Execution order: the serial build walks a range in row-major order
// (dimension 0 outermost). Each reference kernel writes a single colour or an
// independent output per work-item, so this order gives the canonical result;
// reductions then sum in row-major order. With -DPMG_SHIM_OPENMP the outermost
// dimension is split across OpenMP threads (timing only: reduction order then
// depends on the thread count).
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#ifdef PMG_SHIM_OPENMP
#include <omp.h>
#endif

namespace sycl {

template <int N> struct id_storage {
  std::size_t v[N] = {};
};
// A one-dimensional id converts to size_t (a plain, non-template conversion
// so that it also works as a built-in pointer subscript).
template <> struct id_storage<1> {
  std::size_t v[1] = {};
  operator std::size_t() const { return v[0]; }
};

template <int N> struct id : id_storage<N> {
  id() = default;
  template <typename... I,
            typename = std::enable_if_t<sizeof...(I) == N &&
                                        (std::is_integral_v<I> && ...)>>
  id(I... i) : id_storage<N>{{static_cast<std::size_t>(i)...}} {}
  std::size_t &operator[](int d) { return this->v[d]; }
  const std::size_t &operator[](int d) const { return this->v[d]; }
  std::size_t get(int d) const { return this->v[d]; }
};

template <int N> struct range {
  std::size_t v[N] = {};
  range() = default;
  template <typename... I,
            typename = std::enable_if_t<sizeof...(I) == N &&
                                        (std::is_integral_v<I> && ...)>>
  range(I... i) : v{static_cast<std::size_t>(i)...} {}
  std::size_t &operator[](int d) { return v[d]; }
  const std::size_t &operator[](int d) const { return v[d]; }
  std::size_t get(int d) const { return v[d]; }
  std::size_t size() const {
    std::size_t s = 1;
    for (int d = 0; d < N; ++d)
      s *= v[d];
    return s;
  }
};
template <typename A> range(A) -> range<1>;
template <typename A, typename B> range(A, B) -> range<2>;
template <typename A, typename B, typename C> range(A, B, C) -> range<3>;

template <int N> struct item : id<N> {
  range<N> r;
  item(const id<N> &i, const range<N> &rr) : id<N>(i), r(rr) {}
  id<N> get_id() const { return *this; }
  std::size_t get_id(int d) const { return this->v[d]; }
  range<N> get_range() const { return r; }
  std::size_t get_linear_id() const {
    std::size_t l = 0;
    for (int d = 0; d < N; ++d)
      l = l * r[d] + this->v[d];
    return l;
  }
};

template <typename T = void> struct plus {
  T operator()(const T &a, const T &b) const { return a + b; }
};
template <> struct plus<void> {
  template <typename A, typename B> auto operator()(A a, B b) const {
    return a + b;
  }
};

template <typename T, typename Op> struct reduction_desc {
  T *ptr;
  Op op;
};
template <typename T, typename Op> reduction_desc<T, Op> reduction(T *p, Op op) {
  return {p, op};
}

// The object a kernel's reduction argument binds to ("auto &acc").
template <typename T> struct reducer {
  T value{};
  reducer &operator+=(const T &x) {
    value += x;
    return *this;
  }
  void combine(const T &x) { value += x; }
};

struct event {
  void wait() {}
  void wait_and_throw() {}
};

namespace info {
namespace device {
struct name {};
} // namespace device
} // namespace info

struct device {
  template <typename Info> std::string get_info() const {
    return std::string("host oracle shim");
  }
};

namespace property {
namespace queue {
struct in_order {};
} // namespace queue
} // namespace property

struct property_list {
  template <typename... P> property_list(P...) {}
};

struct cpu_selector {};
struct gpu_selector {};
struct default_selector {};

namespace detail {

// Calls k(item) for every index of r; row-major, dimension 0 outermost.
template <int N, typename K> inline void run_range(const range<N> &r, K &&k) {
  if constexpr (N == 1) {
#ifdef PMG_SHIM_OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (long a = 0; a < (long)r[0]; ++a)
      k(item<1>(id<1>((std::size_t)a), r));
  } else if constexpr (N == 2) {
#ifdef PMG_SHIM_OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (long a = 0; a < (long)r[0]; ++a)
      for (std::size_t b = 0; b < r[1]; ++b)
        k(item<2>(id<2>((std::size_t)a, b), r));
  } else {
#ifdef PMG_SHIM_OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (long a = 0; a < (long)r[0]; ++a)
      for (std::size_t b = 0; b < r[1]; ++b)
        for (std::size_t c = 0; c < r[2]; ++c)
          k(item<3>(id<3>((std::size_t)a, b, c), r));
  }
}

// Same walk with one or two reductions. Partial sums are kept per outermost
// index and added into the target in index order after the walk, so the
// serial and the OpenMP builds only differ in how partials are formed.
template <int N, typename K, typename... R>
inline void run_range_reduce(const range<N> &r, K &&k, R... reds) {
  constexpr std::size_t nred = sizeof...(R);
  auto ptrs = std::make_tuple(reds.ptr...);
  using T0 = std::remove_pointer_t<std::tuple_element_t<0, decltype(ptrs)>>;
  const long outer = (long)r[0];
  std::vector<std::array<T0, nred>> part((std::size_t)outer);
#ifdef PMG_SHIM_OPENMP
#pragma omp parallel for schedule(static)
#endif
  for (long a = 0; a < outer; ++a) {
    reducer<T0> acc[nred];
    if constexpr (N == 1) {
      item<1> it(id<1>((std::size_t)a), r);
      if constexpr (nred == 1)
        k(it, acc[0]);
      else
        k(it, acc[0], acc[1]);
    } else if constexpr (N == 2) {
      for (std::size_t b = 0; b < r[1]; ++b) {
        item<2> it(id<2>((std::size_t)a, b), r);
        if constexpr (nred == 1)
          k(it, acc[0]);
        else
          k(it, acc[0], acc[1]);
      }
    } else {
      for (std::size_t b = 0; b < r[1]; ++b)
        for (std::size_t c = 0; c < r[2]; ++c) {
          item<3> it(id<3>((std::size_t)a, b, c), r);
          if constexpr (nred == 1)
            k(it, acc[0]);
          else
            k(it, acc[0], acc[1]);
        }
    }
    for (std::size_t q = 0; q < nred; ++q)
      part[(std::size_t)a][q] = acc[q].value;
  }
  // Row-major combination: identical to a single running sum when serial
  // only up to the association of per-row partials, which the oracle accepts
  // (reductions are compared with a tolerance, never bit-exactly).
  std::size_t q = 0;
  auto add = [&](auto *p) {
    for (long a = 0; a < outer; ++a)
      *p += part[(std::size_t)a][q];
    ++q;
  };
  std::apply([&](auto *...p) { (add(p), ...); }, ptrs);
}

template <typename... A> inline void print(A &&...) {}

} // namespace detail

struct handler {
  template <int N, typename K> void parallel_for(range<N> r, K k) {
    detail::run_range(r, k);
  }
  template <int N, typename T, typename Op, typename K>
  void parallel_for(range<N> r, reduction_desc<T, Op> r0, K k) {
    detail::run_range_reduce(r, k, r0);
  }
  template <int N, typename T, typename Op, typename T1, typename Op1,
            typename K>
  void parallel_for(range<N> r, reduction_desc<T, Op> r0,
                    reduction_desc<T1, Op1> r1, K k) {
    detail::run_range_reduce(r, k, r0, r1);
  }
  template <typename K> void single_task(K k) { k(); }
};

struct queue {
  queue() = default;
  template <typename S> explicit queue(const S &) {}
  template <typename S> queue(const S &, const property_list &) {}

  template <int N, typename K> event parallel_for(range<N> r, K k) {
    detail::run_range(r, k);
    return {};
  }
  template <int N, typename T, typename Op, typename K>
  event parallel_for(range<N> r, reduction_desc<T, Op> r0, K k) {
    detail::run_range_reduce(r, k, r0);
    return {};
  }
  template <int N, typename T, typename Op, typename T1, typename Op1,
            typename K>
  event parallel_for(range<N> r, reduction_desc<T, Op> r0,
                     reduction_desc<T1, Op1> r1, K k) {
    detail::run_range_reduce(r, k, r0, r1);
    return {};
  }
  template <typename K> event single_task(K k) {
    k();
    return {};
  }
  template <typename F> event submit(F &&f) {
    handler h;
    f(h);
    return {};
  }
  event memcpy(void *dst, const void *src, std::size_t bytes) {
    if (bytes)
      std::memmove(dst, src, bytes);
    return {};
  }
  event memset(void *dst, int v, std::size_t bytes) {
    if (bytes)
      std::memset(dst, v, bytes);
    return {};
  }
  template <typename T, typename V>
  event fill(T *dst, const V &v, std::size_t count) {
    for (std::size_t i = 0; i < count; ++i)
      dst[i] = static_cast<T>(v);
    return {};
  }
  void wait() {}
  void wait_and_throw() {}
  device get_device() const { return {}; }
  bool operator==(const queue &o) const { return this == &o; }
  bool operator!=(const queue &o) const { return this != &o; }
};

template <typename T> T *malloc_device(std::size_t n, const queue &) {
  return static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
}
template <typename T> T *malloc_shared(std::size_t n, const queue &) {
  return static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
}
template <typename T> T *malloc_host(std::size_t n, const queue &) {
  return static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
}
inline void free(void *p, const queue &) { std::free(p); }

using std::fabs;
using std::sqrt;

namespace ext {
namespace oneapi {
namespace experimental {
template <typename... A> inline int printf(const char *fmt, A... a) {
  return std::printf(fmt, a...);
}
} // namespace experimental
} // namespace oneapi
} // namespace ext

} // namespace sycl
