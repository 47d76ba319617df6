// Kokkos-API host shim: test infrastructure for the oracle only.
//
// teuk-kokkos is header-only C++ written against Kokkos, whose submodule is
// not vendored with the reference sources. This header is a project-written,
// minimal host implementation of the *public* Kokkos API names the reference
// headers use (View up to rank 4 with LayoutRight / LayoutStride subviews,
// RangePolicy + parallel_for, deep_copy, mirrors, atomics, complex and the
// math wrappers). It lets the reference's own headers compile unchanged into
// the CPU oracle binaries under oracle/_ref. It is written from the API's
// documented names and semantics, not from Kokkos sources.
//
// Backends: Serial (default, deterministic) and, with TEUK_SHIM_THREADS
// defined, a persistent std::thread pool that splits every RangePolicy into
// one contiguous chunk per thread (TEUK_SHIM_NUM_THREADS, default: hardware
// concurrency). Declared arithmetic semantics (these are the points where a
// real Kokkos build could differ in the last bits):
//   * complex / complex uses the |c|+|d| scaled textbook division;
//   * abs(complex) is std::hypot(re, im);
//   * sin/cos/acos/sqrt/exp/pow forward to the C library.
// Nothing in the product library includes this file.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <condition_variable>
#include <cstdlib>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include <string>
#include <type_traits>
#include <utility>

#include "Kokkos_Complex.hpp"

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]
#define KOKKOS_VERSION_MAJOR 5
#define KOKKOS_VERSION_MINOR 1
#define KOKKOS_VERSION_PATCH 0
#define KOKKOS_VERSION 50100

namespace Kokkos {

// ---------------------------------------------------------------- spaces
class HostSpace {
 public:
  using memory_space = HostSpace;
  using size_type = std::size_t;
  static constexpr const char* name() { return "HostSpace"; }
};

class Serial {
 public:
  using execution_space = Serial;
  using memory_space = HostSpace;
  using device_type = Serial;
  using size_type = std::size_t;
  static constexpr const char* name() {
#if defined(TEUK_SHIM_THREADS)
    return "Threads";
#else
    return "Serial";
#endif
  }
  void fence(const std::string& = std::string()) const {}
  static void impl_static_fence(const std::string& = std::string()) {}
  int concurrency() const { return 1; }
};

using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;
using OpenMP = Serial;

inline void fence(const std::string& = std::string()) {}

template <class ExecSpace, class MemSpace>
struct SpaceAccessibility {
  static constexpr bool accessible = true;
  static constexpr bool assignable = true;
  static constexpr bool deepcopy = true;
};

inline bool& shim_initialized_flag() {
  static bool flag = false;
  return flag;
}
inline void initialize(int&, char**) { shim_initialized_flag() = true; }
inline void initialize() { shim_initialized_flag() = true; }
inline void finalize() { shim_initialized_flag() = false; }
inline bool is_initialized() { return shim_initialized_flag(); }

struct ScopeGuard {
  ScopeGuard(int& argc, char** argv) { initialize(argc, argv); }
  ScopeGuard() { initialize(); }
  ~ScopeGuard() { finalize(); }
};

// ---------------------------------------------------------------- layouts
struct LayoutRight {};
struct LayoutLeft {};
struct LayoutStride {};

enum MemoryTraitsFlags : unsigned {
  Unmanaged = 0x01,
  RandomAccess = 0x02,
  Atomic = 0x04,
  Restrict = 0x08,
  Aligned = 0x10
};
template <unsigned Flags>
struct MemoryTraits {
  static constexpr unsigned value = Flags;
};

struct ALL_t {};
inline constexpr ALL_t ALL{};

struct WithoutInitializing_t {};
inline constexpr WithoutInitializing_t WithoutInitializing{};

struct ViewCtorProp {
  std::string label;
  bool initialize = true;
};

namespace shim_detail {
inline void apply_prop(ViewCtorProp& prop, const std::string& label) {
  prop.label = label;
}
inline void apply_prop(ViewCtorProp& prop, const char* label) {
  prop.label = label;
}
inline void apply_prop(ViewCtorProp& prop, WithoutInitializing_t) {
  prop.initialize = false;
}
template <class Space>
inline void apply_prop(ViewCtorProp&, const Space&) {}
}  // namespace shim_detail

template <class... Args>
ViewCtorProp view_alloc(const Args&... args) {
  ViewCtorProp prop;
  (shim_detail::apply_prop(prop, args), ...);
  return prop;
}

// ---------------------------------------------------------------- View
namespace shim_detail {

template <class T>
struct data_analysis {
  using value_type = T;
  static constexpr unsigned rank = 0;
};
template <class T>
struct data_analysis<T*> {
  using value_type = typename data_analysis<T>::value_type;
  static constexpr unsigned rank = 1 + data_analysis<T>::rank;
};

template <class T, unsigned R>
struct add_pointers {
  using type = typename add_pointers<T*, R - 1>::type;
};
template <class T>
struct add_pointers<T, 0> {
  using type = T;
};

template <class... P>
struct layout_of {
  using type = LayoutRight;
};
template <class... P>
struct layout_of<LayoutStride, P...> {
  using type = LayoutStride;
};
template <class... P>
struct layout_of<LayoutRight, P...> {
  using type = LayoutRight;
};
template <class Head, class... P>
struct layout_of<Head, P...> {
  using type = typename layout_of<P...>::type;
};

template <class... P>
struct unmanaged_of {
  static constexpr bool value = false;
};
template <unsigned F, class... P>
struct unmanaged_of<MemoryTraits<F>, P...> {
  static constexpr bool value = (F & Unmanaged) != 0;
};
template <class Head, class... P>
struct unmanaged_of<Head, P...> {
  static constexpr bool value = unmanaged_of<P...>::value;
};

struct ViewAccess;

}  // namespace shim_detail

template <class DataType, class... Properties>
class View {
  using analysis = shim_detail::data_analysis<DataType>;

 public:
  using data_type = DataType;
  using value_type = typename analysis::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using const_value_type = const non_const_value_type;
  using pointer_type = value_type*;
  using reference_type = value_type&;
  using array_layout = typename shim_detail::layout_of<Properties...>::type;
  using memory_space = HostSpace;
  using execution_space = DefaultExecutionSpace;
  using device_type = DefaultExecutionSpace;
  using size_type = std::size_t;
  using traits = View;
  using HostMirror = View<DataType, array_layout, HostSpace>;
  using host_mirror_type = HostMirror;
  using non_const_type = View<typename shim_detail::add_pointers<
                                  non_const_value_type, analysis::rank>::type,
                              Properties...>;
  using const_type =
      View<typename shim_detail::add_pointers<const_value_type,
                                              analysis::rank>::type,
           Properties...>;
  static constexpr std::integral_constant<unsigned, analysis::rank> rank{};
  static constexpr std::integral_constant<unsigned, analysis::rank>
      rank_dynamic{};
  static constexpr bool is_unmanaged =
      shim_detail::unmanaged_of<Properties...>::value;

  View() = default;

  template <class... Extents,
            class = std::enable_if_t<(std::is_convertible_v<Extents, std::size_t> && ...)>>
  explicit View(const std::string& label, Extents... extents) {
    allocate(label, true, static_cast<std::size_t>(extents)...);
  }
  template <class... Extents,
            class = std::enable_if_t<(std::is_convertible_v<Extents, std::size_t> && ...)>>
  explicit View(const char* label, Extents... extents) {
    allocate(label, true, static_cast<std::size_t>(extents)...);
  }
  template <class... Extents,
            class = std::enable_if_t<(std::is_convertible_v<Extents, std::size_t> && ...)>>
  explicit View(const ViewCtorProp& prop, Extents... extents) {
    allocate(prop.label, prop.initialize,
             static_cast<std::size_t>(extents)...);
  }
  template <class... Extents,
            class = std::enable_if_t<(std::is_convertible_v<Extents, std::size_t> && ...)>>
  View(pointer_type pointer, Extents... extents) {
    set_extents(static_cast<std::size_t>(extents)...);
    data_ = pointer;
  }

  // Permissive conversion between views of the same rank and element type
  // (LayoutRight <-> LayoutStride, managed <-> unmanaged, non-const ->
  // const). Strides travel with the data.
  template <class OtherData, class... OtherProps,
            class = std::enable_if_t<
                View<OtherData, OtherProps...>::rank == analysis::rank &&
                std::is_convertible_v<
                    typename View<OtherData, OtherProps...>::pointer_type,
                    pointer_type>>>
  View(const View<OtherData, OtherProps...>& other)
      : owner_(other.owner_),
        data_(other.data_),
        label_(other.label_) {
    for (unsigned i = 0; i < 8; ++i) {
      extents_[i] = other.extents_[i];
      strides_[i] = other.strides_[i];
    }
  }

  [[nodiscard]] std::size_t extent(const unsigned dim) const {
    return dim < 8 ? extents_[dim] : 1;
  }
  [[nodiscard]] int extent_int(const unsigned dim) const {
    return static_cast<int>(extent(dim));
  }
  [[nodiscard]] std::size_t stride(const unsigned dim) const {
    return dim < 8 ? strides_[dim] : 0;
  }
  template <class Integer>
  void stride(Integer* out) const {
    for (unsigned i = 0; i < analysis::rank; ++i) out[i] = strides_[i];
  }
  [[nodiscard]] std::size_t stride_0() const { return strides_[0]; }
  [[nodiscard]] std::size_t stride_1() const { return strides_[1]; }
  [[nodiscard]] std::size_t stride_2() const { return strides_[2]; }
  [[nodiscard]] std::size_t stride_3() const { return strides_[3]; }
  [[nodiscard]] std::size_t size() const {
    std::size_t total = 1;
    for (unsigned i = 0; i < analysis::rank; ++i) total *= extents_[i];
    return total;
  }
  [[nodiscard]] std::size_t span() const {
    if (analysis::rank == 0) return data_ ? 1 : 0;
    std::size_t last = 0;
    for (unsigned i = 0; i < analysis::rank; ++i) {
      if (extents_[i] == 0) return 0;
      last += (extents_[i] - 1) * strides_[i];
    }
    return last + 1;
  }
  [[nodiscard]] bool span_is_contiguous() const { return span() == size(); }
  [[nodiscard]] pointer_type data() const { return data_; }
  [[nodiscard]] std::string label() const { return label_; }
  [[nodiscard]] bool is_allocated() const { return data_ != nullptr; }
  [[nodiscard]] long use_count() const { return owner_.use_count(); }

  template <class... Indices>
  reference_type operator()(const Indices... indices) const {
    static_assert(sizeof...(Indices) == analysis::rank ||
                      (analysis::rank == 0 && sizeof...(Indices) == 0),
                  "View index count must equal its rank");
    std::size_t offset = 0;
    unsigned dim = 0;
    ((offset += static_cast<std::size_t>(indices) * strides_[dim++]), ...);
    return data_[offset];
  }
  template <class Index>
  reference_type operator[](const Index index) const {
    return data_[static_cast<std::size_t>(index) * strides_[0]];
  }
  template <class Index>
  reference_type access(const Index index) const {
    return (*this)[index];
  }

 private:
  template <class, class...>
  friend class View;
  friend struct shim_detail::ViewAccess;

  template <class... Extents>
  void set_extents(const Extents... extents) {
    static_assert(sizeof...(Extents) <= 8, "shim View rank is at most 8");
    const std::size_t given[] = {static_cast<std::size_t>(extents)..., 0};
    for (unsigned i = 0; i < 8; ++i) {
      extents_[i] = 1;
      strides_[i] = 0;
    }
    for (unsigned i = 0; i < analysis::rank; ++i) {
      extents_[i] = i < sizeof...(Extents) ? given[i] : 0;
    }
    std::size_t stride = 1;
    for (int i = static_cast<int>(analysis::rank) - 1; i >= 0; --i) {
      strides_[i] = stride;
      stride *= extents_[i];
    }
  }

  template <class... Extents>
  void allocate(const std::string& label, const bool initialize,
                const Extents... extents) {
    set_extents(extents...);
    label_ = label;
    const std::size_t count = size();
    std::shared_ptr<non_const_value_type[]> storage(
        new non_const_value_type[count > 0 ? count : 1]());
    (void)initialize;
    owner_ = storage;
    data_ = storage.get();
  }

  std::shared_ptr<non_const_value_type[]> owner_;
  pointer_type data_ = nullptr;
  std::size_t extents_[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  std::size_t strides_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::string label_;
};

namespace shim_detail {

struct ViewAccess {
  template <class V>
  static auto& owner(V& v) {
    return v.owner_;
  }
  template <class V>
  static auto& data(V& v) {
    return v.data_;
  }
  template <class V>
  static auto* extents(V& v) {
    return v.extents_;
  }
  template <class V>
  static auto* strides(V& v) {
    return v.strides_;
  }
  template <class V>
  static auto& label(V& v) {
    return v.label_;
  }
};

template <class T>
constexpr unsigned all_count() {
  return std::is_same_v<std::decay_t<T>, ALL_t> ? 1U : 0U;
}

template <class SourceView>
void subview_apply(std::size_t& offset, std::size_t* extents,
                   std::size_t* strides, unsigned& out, const SourceView& v,
                   const unsigned dim, const ALL_t&) {
  extents[out] = v.extent(dim);
  strides[out] = v.stride(dim);
  ++out;
}
template <class SourceView, class Index,
          class = std::enable_if_t<std::is_integral_v<Index>>>
void subview_apply(std::size_t& offset, std::size_t*, std::size_t*,
                   unsigned&, const SourceView& v, const unsigned dim,
                   const Index index) {
  offset += static_cast<std::size_t>(index) * v.stride(dim);
}
template <class SourceView, class Index>
void subview_apply(std::size_t& offset, std::size_t* extents,
                   std::size_t* strides, unsigned& out, const SourceView& v,
                   const unsigned dim, const std::pair<Index, Index>& range) {
  offset += static_cast<std::size_t>(range.first) * v.stride(dim);
  extents[out] = static_cast<std::size_t>(range.second - range.first);
  strides[out] = v.stride(dim);
  ++out;
}

template <class T>
constexpr unsigned range_count() {
  using D = std::decay_t<T>;
  if constexpr (std::is_same_v<D, ALL_t>) {
    return 1U;
  } else if constexpr (std::is_integral_v<D>) {
    return 0U;
  } else {
    return 1U;  // std::pair range
  }
}

}  // namespace shim_detail

template <class DataType, class... Props, class... Args>
auto subview(const View<DataType, Props...>& view, const Args&... args) {
  using Source = View<DataType, Props...>;
  static_assert(sizeof...(Args) == Source::rank,
                "subview needs one argument per dimension");
  constexpr unsigned result_rank = (shim_detail::range_count<Args>() + ... + 0U);
  using Value = typename Source::value_type;
  using Result =
      View<typename shim_detail::add_pointers<Value, result_rank>::type,
           LayoutStride, HostSpace>;
  Result result;
  std::size_t offset = 0;
  std::size_t* extents = shim_detail::ViewAccess::extents(result);
  std::size_t* strides = shim_detail::ViewAccess::strides(result);
  for (unsigned i = 0; i < 8; ++i) {
    extents[i] = 1;
    strides[i] = 0;
  }
  unsigned out = 0;
  unsigned dim = 0;
  (shim_detail::subview_apply(offset, extents, strides, out, view, dim++,
                              args),
   ...);
  auto source = view;
  shim_detail::ViewAccess::owner(result) =
      shim_detail::ViewAccess::owner(source);
  shim_detail::ViewAccess::data(result) = view.data() + offset;
  shim_detail::ViewAccess::label(result) = view.label();
  return result;
}

// ---------------------------------------------------------------- policies
template <class... Args>
struct IndexType {};

template <class... Properties>
class RangePolicy {
 public:
  using execution_space = DefaultExecutionSpace;
  using index_type = std::int64_t;
  using member_type = std::int64_t;
  RangePolicy() = default;
  template <class B, class E,
            class = std::enable_if_t<std::is_integral_v<B> &&
                                     std::is_integral_v<E>>>
  RangePolicy(const B begin, const E end)
      : begin_(static_cast<std::int64_t>(begin)),
        end_(static_cast<std::int64_t>(end)) {}
  template <class Space, class B, class E,
            class = std::enable_if_t<!std::is_integral_v<Space> &&
                                     std::is_integral_v<B> &&
                                     std::is_integral_v<E>>>
  RangePolicy(const Space&, const B begin, const E end)
      : begin_(static_cast<std::int64_t>(begin)),
        end_(static_cast<std::int64_t>(end)) {}
  [[nodiscard]] std::int64_t begin() const { return begin_; }
  [[nodiscard]] std::int64_t end() const { return end_; }
  [[nodiscard]] execution_space space() const { return {}; }

 private:
  std::int64_t begin_ = 0;
  std::int64_t end_ = 0;
};

namespace shim_detail {

#if defined(TEUK_SHIM_THREADS)
// Persistent worker pool: thread t runs chunk t of every dispatched range;
// the calling thread runs chunk 0 and waits for the others.
class ThreadPool {
 public:
  static ThreadPool& instance() {
    static ThreadPool pool;
    return pool;
  }
  unsigned size() const { return count_; }

  void run(const std::int64_t begin, const std::int64_t end,
           const std::function<void(std::int64_t, std::int64_t)>& body) {
    const std::int64_t total = end - begin;
    if (total <= 0) return;
    if (count_ <= 1 || total < 2 * static_cast<std::int64_t>(count_)) {
      body(begin, end);
      return;
    }
    {
      std::unique_lock<std::mutex> lock(mutex_);
      body_ = &body;
      begin_ = begin;
      end_ = end;
      pending_ = count_ - 1;
      ++generation_;
    }
    wake_.notify_all();
    const auto [b0, e0] = chunk(0);
    body(b0, e0);
    std::unique_lock<std::mutex> lock(mutex_);
    done_.wait(lock, [&] { return pending_ == 0; });
    body_ = nullptr;
  }

  ~ThreadPool() {
    {
      std::unique_lock<std::mutex> lock(mutex_);
      stop_ = true;
      ++generation_;
    }
    wake_.notify_all();
    for (auto& worker : workers_) worker.join();
  }

 private:
  ThreadPool() {
    unsigned requested = std::thread::hardware_concurrency();
    if (const char* env = std::getenv("TEUK_SHIM_NUM_THREADS")) {
      const long value = std::strtol(env, nullptr, 10);
      if (value > 0) requested = static_cast<unsigned>(value);
    }
    count_ = requested > 0 ? requested : 1;
    for (unsigned t = 1; t < count_; ++t) {
      workers_.emplace_back([this, t] { work(t); });
    }
  }

  std::pair<std::int64_t, std::int64_t> chunk(const unsigned t) const {
    const std::int64_t total = end_ - begin_;
    const std::int64_t lo = begin_ + total * t / count_;
    const std::int64_t hi = begin_ + total * (t + 1) / count_;
    return {lo, hi};
  }

  void work(const unsigned t) {
    std::uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lock(mutex_);
      wake_.wait(lock, [&] { return generation_ != seen; });
      seen = generation_;
      if (stop_) return;
      const auto* body = body_;
      const auto [lo, hi] = chunk(t);
      lock.unlock();
      (*body)(lo, hi);
      lock.lock();
      if (--pending_ == 0) done_.notify_one();
    }
  }

  unsigned count_ = 1;
  std::vector<std::thread> workers_;
  std::mutex mutex_;
  std::condition_variable wake_;
  std::condition_variable done_;
  const std::function<void(std::int64_t, std::int64_t)>* body_ = nullptr;
  std::int64_t begin_ = 0;
  std::int64_t end_ = 0;
  unsigned pending_ = 0;
  std::uint64_t generation_ = 0;
  bool stop_ = false;
};

inline std::mutex& atomic_mutex() {
  static std::mutex mutex;
  return mutex;
}
#endif

template <class Functor>
void run_range(const std::int64_t begin, const std::int64_t end,
               const Functor& functor) {
#if defined(TEUK_SHIM_THREADS)
  const std::function<void(std::int64_t, std::int64_t)> body =
      [&functor](const std::int64_t lo, const std::int64_t hi) {
        for (std::int64_t i = lo; i < hi; ++i) {
          functor(static_cast<std::size_t>(i));
        }
      };
  ThreadPool::instance().run(begin, end, body);
#else
  for (std::int64_t i = begin; i < end; ++i) {
    functor(static_cast<std::size_t>(i));
  }
#endif
}
}  // namespace shim_detail

template <class... P, class Functor>
void parallel_for(const std::string&, const RangePolicy<P...>& policy,
                  const Functor& functor) {
  shim_detail::run_range(policy.begin(), policy.end(), functor);
}
template <class... P, class Functor>
void parallel_for(const RangePolicy<P...>& policy, const Functor& functor) {
  shim_detail::run_range(policy.begin(), policy.end(), functor);
}
template <class Integer, class Functor,
          class = std::enable_if_t<std::is_integral_v<Integer>>>
void parallel_for(const std::string&, const Integer count,
                  const Functor& functor) {
  shim_detail::run_range(0, static_cast<std::int64_t>(count), functor);
}
template <class Integer, class Functor,
          class = std::enable_if_t<std::is_integral_v<Integer>>>
void parallel_for(const Integer count, const Functor& functor) {
  shim_detail::run_range(0, static_cast<std::int64_t>(count), functor);
}

// Reductions run serially in index order so results are deterministic.
template <class... P, class Functor, class Result>
void parallel_reduce(const std::string&, const RangePolicy<P...>& policy,
                     const Functor& functor, Result& result) {
  Result accumulator{};
  for (std::int64_t i = policy.begin(); i < policy.end(); ++i) {
    functor(static_cast<std::size_t>(i), accumulator);
  }
  result = accumulator;
}
template <class... P, class Functor, class Result>
void parallel_reduce(const RangePolicy<P...>& policy, const Functor& functor,
                     Result& result) {
  parallel_reduce(std::string(), policy, functor, result);
}

// ---------------------------------------------------------------- copies
namespace shim_detail {
template <class Dst, class Src>
void copy_elements(const Dst& dst, const Src& src) {
  constexpr unsigned r = Dst::rank;
  static_assert(r == Src::rank, "deep_copy requires equal ranks");
  for (unsigned i = 0; i < r; ++i) {
    if (dst.extent(i) != src.extent(i)) {
      throw std::runtime_error("deep_copy extents do not match");
    }
  }
  const std::size_t total = dst.size();
  if (total == 0) return;
  if (dst.span_is_contiguous() && src.span_is_contiguous() &&
      std::is_trivially_copyable_v<typename Dst::non_const_value_type>) {
    bool same_strides = true;
    for (unsigned i = 0; i < r; ++i) {
      same_strides = same_strides && dst.stride(i) == src.stride(i);
    }
    if (same_strides) {
      if (dst.data() != src.data()) {
        std::memmove(static_cast<void*>(dst.data()),
                     static_cast<const void*>(src.data()),
                     total * sizeof(typename Dst::non_const_value_type));
      }
      return;
    }
  }
  for (std::size_t flat = 0; flat < total; ++flat) {
    std::size_t rem = flat;
    std::size_t dst_offset = 0;
    std::size_t src_offset = 0;
    for (int i = static_cast<int>(r) - 1; i >= 0; --i) {
      const std::size_t index = rem % dst.extent(static_cast<unsigned>(i));
      rem /= dst.extent(static_cast<unsigned>(i));
      dst_offset += index * dst.stride(static_cast<unsigned>(i));
      src_offset += index * src.stride(static_cast<unsigned>(i));
    }
    dst.data()[dst_offset] = src.data()[src_offset];
  }
}

template <class Dst, class Value>
void fill_elements(const Dst& dst, const Value& value) {
  constexpr unsigned r = Dst::rank;
  const std::size_t total = dst.size();
  for (std::size_t flat = 0; flat < total; ++flat) {
    std::size_t rem = flat;
    std::size_t offset = 0;
    for (int i = static_cast<int>(r) - 1; i >= 0; --i) {
      const std::size_t index = rem % dst.extent(static_cast<unsigned>(i));
      rem /= dst.extent(static_cast<unsigned>(i));
      offset += index * dst.stride(static_cast<unsigned>(i));
    }
    dst.data()[offset] = value;
  }
}
}  // namespace shim_detail

template <class DD, class... DP, class SD, class... SP>
void deep_copy(const View<DD, DP...>& dst, const View<SD, SP...>& src) {
  shim_detail::copy_elements(dst, src);
}
template <class Space, class DD, class... DP, class SD, class... SP>
void deep_copy(const Space&, const View<DD, DP...>& dst,
               const View<SD, SP...>& src) {
  shim_detail::copy_elements(dst, src);
}
template <class DD, class... DP, class Value,
          class = std::enable_if_t<!std::is_base_of_v<
              View<DD, DP...>, std::decay_t<Value>>>>
void deep_copy(const View<DD, DP...>& dst, const Value& value) {
  shim_detail::fill_elements(dst, value);
}
template <class Space, class DD, class... DP, class Value>
void deep_copy(const Space&, const View<DD, DP...>& dst, const Value& value) {
  shim_detail::fill_elements(dst, value);
}
template <class Value, class SD, class... SP,
          class = std::enable_if_t<std::is_arithmetic_v<Value>>>
void deep_copy(Value& dst, const View<SD, SP...>& src) {
  dst = src();
}

template <class D, class... P>
auto create_mirror_view(const View<D, P...>& view) {
  return view;
}
template <class D, class... P>
auto create_mirror_view(const HostSpace&, const View<D, P...>& view) {
  return view;
}
template <class D, class... P>
auto create_mirror_view(const WithoutInitializing_t&,
                        const View<D, P...>& view) {
  return view;
}
template <class D, class... P>
auto create_mirror_view_and_copy(const HostSpace&, const View<D, P...>& view) {
  return view;
}
template <class D, class... P>
auto create_mirror(const View<D, P...>& view) {
  using V = View<D, P...>;
  using Result = View<typename shim_detail::add_pointers<
                          typename V::non_const_value_type, V::rank>::type,
                      LayoutRight, HostSpace>;
  std::size_t e[8];
  for (unsigned i = 0; i < 8; ++i) e[i] = view.extent(i);
  if constexpr (V::rank == 1) {
    return Result(view.label(), e[0]);
  } else if constexpr (V::rank == 2) {
    return Result(view.label(), e[0], e[1]);
  } else if constexpr (V::rank == 3) {
    return Result(view.label(), e[0], e[1], e[2]);
  } else {
    return Result(view.label(), e[0], e[1], e[2], e[3]);
  }
}

// ---------------------------------------------------------------- atomics
#if defined(TEUK_SHIM_THREADS)
#define TEUK_SHIM_ATOMIC_LOCK \
  std::lock_guard<std::mutex> teuk_shim_guard(shim_detail::atomic_mutex())
#else
#define TEUK_SHIM_ATOMIC_LOCK (void)0
#endif
template <class T>
void atomic_add(T* destination, const T value) {
  TEUK_SHIM_ATOMIC_LOCK;
  *destination += value;
}
template <class T>
void atomic_max(T* destination, const T value) {
  TEUK_SHIM_ATOMIC_LOCK;
  *destination = std::max(*destination, value);
}
template <class T>
void atomic_min(T* destination, const T value) {
  TEUK_SHIM_ATOMIC_LOCK;
  *destination = std::min(*destination, value);
}
template <class T, class U>
T atomic_exchange(T* destination, const U value) {
  TEUK_SHIM_ATOMIC_LOCK;
  const T old = *destination;
  *destination = static_cast<T>(value);
  return old;
}

// ---------------------------------------------------------------- Array
template <class T, std::size_t N>
struct Array {
  T m_internal_implementation_detail_do_not_use_me[N > 0 ? N : 1];
  static constexpr std::size_t size() { return N; }
  T& operator[](const std::size_t i) {
    return m_internal_implementation_detail_do_not_use_me[i];
  }
  const T& operator[](const std::size_t i) const {
    return m_internal_implementation_detail_do_not_use_me[i];
  }
  T* data() { return m_internal_implementation_detail_do_not_use_me; }
  const T* data() const {
    return m_internal_implementation_detail_do_not_use_me;
  }
};

template <class T1, class T2>
struct pair {
  T1 first;
  T2 second;
};

}  // namespace Kokkos

#include "Kokkos_MathematicalFunctions.hpp"
