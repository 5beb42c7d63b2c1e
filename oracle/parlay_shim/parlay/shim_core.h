// shim_core.h -- a small parlay-compatible primitive layer, written for this
// project, so that the reference's own BFS sources (serialBFS, simpleBFS,
// backForwardBFS + common/ligraLight.h, deterministicBFS, bench/BFSTime.C,
// bench/BFSCheck.C) compile unmodified while the parlaylib submodule is absent.
//
// TEST INFRASTRUCTURE: used only to build oracle/_ref (the reference run as a
// checker and as the timed CPU baseline).  It covers exactly the calls made on
// the BFS path, with the semantics of parlaylib's published API (sequence,
// tabulate, map, reduce, scan, filter, pack, block_delayed::flatten/filter_map,
// write_max, internal::timer, file_map/tokens/chars_to_long).  parallel_for is
// an OpenMP loop when compiled with -fopenmp, sequential otherwise; every
// other primitive is built on parallel_for.  Order-preserving semantics are
// kept (filter/pack/flatten keep input order) so results match parlaylib's.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <limits>
#include <new>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace parlay {

inline int num_workers() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

inline bool in_parallel_region() {
#ifdef _OPENMP
  return omp_in_parallel();
#else
  return true;
#endif
}

// parallel_for(start, end, f[, granularity[, conservative]])
template <class F>
inline void parallel_for(long start, long end, F&& f, long granularity = 0,
                         bool /*conservative*/ = false) {
  long n = end - start;
  if (n <= 0) return;
#ifdef _OPENMP
  if (n >= 2048 && !omp_in_parallel()) {
    long chunk = granularity > 0 ? granularity : std::max<long>(64, n / (64L * num_workers()));
#pragma omp parallel for schedule(dynamic, chunk)
    for (long i = start; i < end; i++) f(i);
    return;
  }
  if (granularity == 1 && n > 1 && !omp_in_parallel()) {
#pragma omp parallel for schedule(dynamic, 1)
    for (long i = start; i < end; i++) f(i);
    return;
  }
#endif
  for (long i = start; i < end; i++) f(i);
}

template <class Lf, class Rf>
inline void par_do(Lf&& left, Rf&& right, bool = false) {
  left();
  right();
}

// ---------------------------------------------------------------- slice
template <class It, class S = It>
struct slice {
  It s;
  S e;
  using value_type = typename std::iterator_traits<It>::value_type;
  using iterator = It;
  slice(It b, S en) : s(b), e(en) {}
  size_t size() const { return (size_t)(e - s); }
  It begin() const { return s; }
  S end() const { return e; }
  decltype(auto) operator[](size_t i) const { return s[i]; }
  slice cut(size_t i, size_t j) const { return slice(s + i, s + j); }
};

template <class It>
inline slice<It, It> make_slice(It b, It e) {
  return slice<It, It>(b, e);
}
template <class R>
inline auto make_slice(R& r) {
  return make_slice(r.begin(), r.end());
}
template <class R>
inline auto make_slice(const R& r) {
  return make_slice(r.begin(), r.end());
}

// ------------------------------------------------------------- sequence
template <class T>
class sequence {
  T* d_ = nullptr;
  size_t n_ = 0;

  static T* alloc(size_t n) {
    if (n == 0) return nullptr;
    void* p = ::operator new(n * sizeof(T), std::align_val_t(64));
    return static_cast<T*>(p);
  }
  void release() {
    if (d_) {
      if (!std::is_trivially_destructible<T>::value)
        for (size_t i = 0; i < n_; i++) d_[i].~T();
      ::operator delete(d_, std::align_val_t(64));
    }
    d_ = nullptr;
    n_ = 0;
  }

 public:
  using value_type = T;
  using reference = T&;
  using const_reference = const T&;
  using iterator = T*;
  using const_iterator = const T*;
  using size_type = size_t;

  sequence() {}
  explicit sequence(size_t n) : d_(alloc(n)), n_(n) {
    T* d = d_;
    parallel_for(0, (long)n, [d](long i) { new (d + i) T(); });
  }
  sequence(size_t n, const T& v) : d_(alloc(n)), n_(n) {
    T* d = d_;
    parallel_for(0, (long)n, [d, &v](long i) { new (d + i) T(v); });
  }
  template <class It, class = typename std::iterator_traits<It>::value_type>
  sequence(It b, It e) : d_(alloc((size_t)(e - b))), n_((size_t)(e - b)) {
    T* d = d_;
    parallel_for(0, (long)n_, [d, b](long i) { new (d + i) T(b[i]); });
  }
  sequence(std::initializer_list<T> l) : d_(alloc(l.size())), n_(l.size()) {
    size_t i = 0;
    for (auto& x : l) new (d_ + i++) T(x);
  }
  sequence(const sequence& o) : d_(alloc(o.n_)), n_(o.n_) {
    T* d = d_;
    const T* s = o.d_;
    parallel_for(0, (long)n_, [d, s](long i) { new (d + i) T(s[i]); });
  }
  sequence(sequence&& o) noexcept : d_(o.d_), n_(o.n_) {
    o.d_ = nullptr;
    o.n_ = 0;
  }
  sequence& operator=(const sequence& o) {
    if (this != &o) {
      sequence t(o);
      swap(t);
    }
    return *this;
  }
  sequence& operator=(sequence&& o) noexcept {
    if (this != &o) {
      release();
      d_ = o.d_;
      n_ = o.n_;
      o.d_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  ~sequence() { release(); }

  void swap(sequence& o) {
    std::swap(d_, o.d_);
    std::swap(n_, o.n_);
  }

  // Storage only; elements are value-initialised for non-trivial types.
  static sequence uninitialized(size_t n) {
    sequence s;
    s.d_ = alloc(n);
    s.n_ = n;
    if (!std::is_trivially_default_constructible<T>::value) {
      T* d = s.d_;
      parallel_for(0, (long)n, [d](long i) { new (d + i) T(); });
    }
    return s;
  }
  template <class F>
  static sequence from_function(size_t n, F&& f) {
    sequence s;
    s.d_ = alloc(n);
    s.n_ = n;
    T* d = s.d_;
    parallel_for(0, (long)n, [d, &f](long i) { new (d + i) T(f(i)); });
    return s;
  }

  size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  T* data() { return d_; }
  const T* data() const { return d_; }
  T* begin() { return d_; }
  T* end() { return d_ + n_; }
  const T* begin() const { return d_; }
  const T* end() const { return d_ + n_; }
  const T* cbegin() const { return d_; }
  const T* cend() const { return d_ + n_; }
  T& operator[](size_t i) { return d_[i]; }
  const T& operator[](size_t i) const { return d_[i]; }
  T& at(size_t i) { return d_[i]; }
  T& front() { return d_[0]; }
  T& back() { return d_[n_ - 1]; }
  void clear() { release(); }
  auto head(size_t k) { return make_slice(d_, d_ + k); }
  auto head(size_t k) const { return make_slice((const T*)d_, (const T*)d_ + k); }
  auto cut(size_t i, size_t j) { return make_slice(d_ + i, d_ + j); }
  auto cut(size_t i, size_t j) const { return make_slice((const T*)d_ + i, (const T*)d_ + j); }
  void push_back(const T& v) {
    sequence t = sequence::uninitialized(n_ + 1);
    for (size_t i = 0; i < n_; i++) new (t.d_ + i) T(std::move(d_[i]));
    new (t.d_ + n_) T(v);
    swap(t);
  }
  bool operator==(const sequence& o) const {
    if (n_ != o.n_) return false;
    for (size_t i = 0; i < n_; i++)
      if (!(d_[i] == o.d_[i])) return false;
    return true;
  }
  bool operator!=(const sequence& o) const { return !(*this == o); }
};

template <class T>
using chars_t = sequence<T>;

// ------------------------------------------------------ delayed sequences
template <class F>
struct delayed_seq_t {
  size_t n;
  F f;
  using value_type = std::decay_t<decltype(std::declval<F>()(size_t(0)))>;
  size_t size() const { return n; }
  value_type operator[](size_t i) const { return f(i); }
};

template <class T, class F>
struct typed_delayed_seq_t {
  size_t n;
  F f;
  using value_type = T;
  size_t size() const { return n; }
  T operator[](size_t i) const { return (T)f(i); }
};

template <class T, class F>
inline auto delayed_seq(size_t n, F f) {
  return typed_delayed_seq_t<T, F>{n, std::move(f)};
}
template <class F>
inline auto delayed_tabulate(size_t n, F f) {
  return delayed_seq_t<F>{n, std::move(f)};
}
template <class R, class F>
inline auto delayed_map(const R& r, F f) {
  auto g = [&r, f](size_t i) { return f(r[i]); };
  return delayed_seq_t<decltype(g)>{r.size(), std::move(g)};
}

// --------------------------------------------------------------- monoids
template <class T>
struct addm {
  using value_type = T;
  T identity = (T)0;
  T f(T a, T b) const { return a + b; }
};
template <class T>
struct minm {
  using value_type = T;
  T identity = std::numeric_limits<T>::max();
  T f(T a, T b) const { return (a < b) ? a : b; }
};
// Pairs (as in MISCheck.C's minm<std::pair<size_t,size_t>>): the identity is
// both components at their maximum, the order lexicographic.
template <class A, class B>
struct minm<std::pair<A, B>> {
  using value_type = std::pair<A, B>;
  value_type identity = value_type(std::numeric_limits<A>::max(), std::numeric_limits<B>::max());
  value_type f(value_type a, value_type b) const { return (a < b) ? a : b; }
};
template <class T>
struct maxm {
  using value_type = T;
  T identity = std::numeric_limits<T>::lowest();
  T f(T a, T b) const { return (a < b) ? b : a; }
};
template <class F, class T>
struct monoid_t {
  using value_type = T;
  F op;
  T identity;
  T f(T a, T b) const { return op(a, b); }
};
template <class F, class T>
inline monoid_t<F, T> make_monoid(F f, T id) {
  return monoid_t<F, T>{f, id};
}

// ---------------------------------------------------------- primitives
template <class F>
inline auto tabulate(size_t n, F&& f, size_t = 0) {
  using T = std::decay_t<decltype(f(size_t(0)))>;
  return sequence<T>::from_function(n, f);
}

template <class R, class F>
inline auto map(const R& r, F&& f, size_t = 0) {
  using T = std::decay_t<decltype(f(r[0]))>;
  return sequence<T>::from_function(r.size(), [&](size_t i) { return f(r[i]); });
}

// Blocked, order-preserving reduction.
template <class R, class M>
inline auto reduce(const R& r, M m) {
  using T = typename M::value_type;
  size_t n = r.size();
  if (n < 4096) {
    T acc = m.identity;
    for (size_t i = 0; i < n; i++) acc = m.f(acc, (T)r[i]);
    return acc;
  }
  size_t nb = (size_t)std::max(1, num_workers()) * 8;
  size_t bs = (n + nb - 1) / nb;
  std::vector<T> part(nb, m.identity);
  parallel_for(0, (long)nb, [&](long b) {
    size_t s = b * bs, e = std::min(n, s + bs);
    T acc = m.identity;
    for (size_t i = s; i < e; i++) acc = m.f(acc, (T)r[i]);
    part[b] = acc;
  }, 1);
  T acc = m.identity;
  for (size_t b = 0; b < nb; b++) acc = m.f(acc, part[b]);
  return acc;
}
template <class R>
inline auto reduce(const R& r) {
  using T = std::decay_t<decltype(r[0])>;
  return reduce(r, addm<T>());
}

// Exclusive scan; returns (prefix sums, total).
template <class R, class M>
inline auto scan(const R& r, M m) {
  using T = typename M::value_type;
  size_t n = r.size();
  sequence<T> out = sequence<T>::uninitialized(n);
  T acc = m.identity;
  for (size_t i = 0; i < n; i++) {
    T x = (T)r[i];
    out[i] = acc;
    acc = m.f(acc, x);
  }
  return std::make_pair(std::move(out), acc);
}
template <class R>
inline auto scan(const R& r) {
  using T = std::decay_t<decltype(r[0])>;
  return scan(r, addm<T>());
}
template <class R>
inline auto scan_inplace(R&& r) {
  using T = std::decay_t<decltype(r[0])>;
  T acc = 0;
  for (size_t i = 0; i < r.size(); i++) {
    T x = r[i];
    r[i] = acc;
    acc += x;
  }
  return acc;
}

// Order-preserving parallel filter/map over [0, n): keep(i) decides, val(i)
// produces the value; keep is evaluated exactly once per index.
template <class T, class Keep>
inline sequence<T> blocked_collect(size_t n, Keep&& keep_and_emit) {
  size_t nb = (n < 4096) ? 1 : (size_t)std::max(1, num_workers()) * 16;
  size_t bs = (n + nb - 1) / (nb ? nb : 1);
  std::vector<std::vector<T>> bufs(nb);
  parallel_for(0, (long)nb, [&](long b) {
    size_t s = b * bs, e = std::min(n, s + bs);
    auto& out = bufs[b];
    for (size_t i = s; i < e; i++) keep_and_emit(i, out);
  }, 1);
  std::vector<size_t> off(nb + 1, 0);
  for (size_t b = 0; b < nb; b++) off[b + 1] = off[b] + bufs[b].size();
  sequence<T> r = sequence<T>::uninitialized(off[nb]);
  parallel_for(0, (long)nb, [&](long b) {
    std::copy(bufs[b].begin(), bufs[b].end(), r.begin() + off[b]);
  }, 1);
  return r;
}

template <class R, class P>
inline auto filter(const R& r, P&& pred) {
  using T = std::decay_t<decltype(r[0])>;
  return blocked_collect<T>(r.size(), [&](size_t i, std::vector<T>& out) {
    T x = r[i];
    if (pred(x)) out.push_back(x);
  });
}

template <class R, class Flags>
inline auto pack(const R& r, const Flags& fl) {
  using T = std::decay_t<decltype(r[0])>;
  return blocked_collect<T>(r.size(), [&](size_t i, std::vector<T>& out) {
    if (fl[i]) out.push_back(r[i]);
  });
}

template <class I, class Flags>
inline sequence<I> pack_index(const Flags& fl) {
  return blocked_collect<I>(fl.size(), [&](size_t i, std::vector<I>& out) {
    if (fl[i]) out.push_back((I)i);
  });
}

template <class R, class V>
inline size_t count(const R& r, const V& v) {
  auto d = delayed_tabulate(r.size(), [&](size_t i) -> size_t { return (r[i] == v) ? 1 : 0; });
  return reduce(d, addm<size_t>());
}

template <class R, class V>
inline auto find(R& r, const V& v) {
  size_t n = r.size();
  for (size_t i = 0; i < n; i++)
    if (r[i] == v) return r.begin() + i;
  return r.begin() + n;
}

template <class A, class B>
inline auto append(const A& a, const B& b) {
  using T = std::decay_t<decltype(a[0])>;
  size_t na = a.size(), nb = b.size();
  return sequence<T>::from_function(na + nb, [&](size_t i) -> T { return i < na ? (T)a[i] : (T)b[i - na]; });
}

template <class R>
inline auto to_sequence(const R& r) {
  using T = std::decay_t<decltype(r[0])>;
  return sequence<T>::from_function(r.size(), [&](size_t i) -> T { return r[i]; });
}

// write_max as a CAS loop (same rule as the helper in common/atomics.h:67-81).
template <class T, class F>
inline bool write_max(std::atomic<T>* a, T b, F less) {
  T c;
  bool r = false;
  do c = a->load();
  while (less(c, b) && !(r = a->compare_exchange_strong(c, b)));
  return r;
}
template <class T, class F>
inline bool write_min(std::atomic<T>* a, T b, F less) {
  T c;
  bool r = false;
  do c = a->load();
  while (less(b, c) && !(r = a->compare_exchange_strong(c, b)));
  return r;
}

// ------------------------------------------------------------ utilities
// 64-bit mixing hash (SplitMix64 output function).  Stands in for
// parlay::hash64, whose constants live in the missing parlaylib; only the
// graph generators use it and those are not built on the BFS path.
inline uint64_t hash64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline size_t log2_up(size_t i) {
  size_t a = 0, b = i - 1;
  while (b > 0) {
    b >>= 1;
    a++;
  }
  return a;
}

class random {
  size_t seed_;

 public:
  explicit random(size_t seed = 0) : seed_(seed) {}
  random fork(size_t i) const { return random(hash64(seed_ + i)); }
  random next() const { return fork(0); }
  size_t ith_rand(size_t i) const { return hash64(seed_ ^ hash64(i)); }
  size_t operator[](size_t i) const { return ith_rand(i); }
};

template <class R>
inline auto random_shuffle(const R& r, random rnd = random(0)) {
  using T = std::decay_t<decltype(r[0])>;
  sequence<T> s = to_sequence(r);
  for (size_t i = s.size(); i > 1; i--) std::swap(s[i - 1], s[rnd.ith_rand(i) % i]);
  return s;
}
template <class I>
inline sequence<I> random_permutation(size_t n, random rnd = random(0)) {
  auto s = tabulate(n, [](size_t i) -> I { return (I)i; });
  for (size_t i = n; i > 1; i--) std::swap(s[i - 1], s[rnd.ith_rand(i) % i]);
  return s;
}
template <class R, class Less>
inline auto remove_duplicates_ordered(const R& r, Less less) {
  using T = std::decay_t<decltype(r[0])>;
  std::vector<T> v(r.begin(), r.end());
  std::stable_sort(v.begin(), v.end(), less);
  std::vector<T> o;
  for (size_t i = 0; i < v.size(); i++)
    if (i == 0 || less(v[i - 1], v[i])) o.push_back(v[i]);
  return sequence<T>(o.begin(), o.end());
}

namespace internal {
// Stable counting sort by key in [0, num_buckets); returns (sorted, counts).
template <class R, class G>
inline auto integer_sort_with_counts(const R& r, G g, size_t num_buckets) {
  using T = std::decay_t<decltype(r[0])>;
  sequence<size_t> counts(num_buckets, 0);
  for (size_t i = 0; i < r.size(); i++) counts[g(r[i])]++;
  std::vector<size_t> pos(num_buckets + 1, 0);
  for (size_t b = 0; b < num_buckets; b++) pos[b + 1] = pos[b] + counts[b];
  sequence<T> out = sequence<T>::uninitialized(r.size());
  for (size_t i = 0; i < r.size(); i++) out[pos[g(r[i])]++] = r[i];
  return std::make_pair(std::move(out), std::move(counts));
}

// timer: name and a report switch; prints "<name>: [<label>: ]<seconds>",
// the line format PBBS's runTests.py parses ("Parlay time: ...").
struct timer {
  std::string name_;
  bool report_;
  bool on_ = false;
  double total_ = 0.0, last_ = 0.0;
  static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }
  explicit timer(std::string name = "Parlay time", bool report = true) : name_(name), report_(report) {
    start();
  }
  void start() {
    on_ = true;
    last_ = now();
  }
  double stop() {
    on_ = false;
    double d = now() - last_;
    total_ += d;
    return d;
  }
  void reset() {
    total_ = 0.0;
    on_ = false;
  }
  double total_time() const { return on_ ? total_ + now() - last_ : total_; }
  double next_time() {
    if (!on_) return 0.0;
    double t = now(), d = t - last_;
    total_ += d;
    last_ = t;
    return d;
  }
  void next(const std::string& label) {
    double d = next_time();
    if (report_ && on_) {
      std::ios::fmtflags f = std::cout.flags();
      auto p = std::cout.precision(4);
      std::cout << std::fixed << name_ << ": ";
      if (!label.empty()) std::cout << label << ": ";
      std::cout << d << std::endl;
      std::cout.flags(f);
      std::cout.precision(p);
    }
  }
  void total() {
    if (report_) std::cout << name_ << ": total: " << total_time() << std::endl;
  }
};
}  // namespace internal

// ------------------------------------------------------- block_delayed
namespace block_delayed {

// View of a sequence of ranges as one flat range; filter_map runs in
// parallel over the outer index and keeps the flat order.
template <class Outer>
struct flat_view {
  const Outer& outer;
};

template <class Outer>
inline flat_view<Outer> flatten(const Outer& o) {
  return flat_view<Outer>{o};
}

template <class Outer, class P, class F>
inline auto filter_map(const flat_view<Outer>& fv, P&& pred, F&& f) {
  using E = std::decay_t<decltype(fv.outer[0][0])>;
  using T = std::decay_t<decltype(f(std::declval<E>()))>;
  const Outer& o = fv.outer;
  size_t no = o.size();
  // Blocks are cut over the flat (edge) index so one long inner range is
  // still split across threads, as parlay's block_delayed does.
  std::vector<size_t> off(no + 1, 0);
  for (size_t i = 0; i < no; i++) off[i + 1] = off[i] + o[i].size();
  size_t total = off[no];
  size_t nb = (total < 4096) ? 1 : (size_t)std::max(1, num_workers()) * 16;
  size_t bs = (total + nb - 1) / nb;
  return blocked_collect<T>(nb, [&](size_t b, std::vector<T>& out) {
    size_t s = b * bs, e = std::min(total, s + bs);
    if (s >= e) return;
    size_t i = (size_t)(std::upper_bound(off.begin(), off.end(), s) - off.begin()) - 1;
    size_t j = s - off[i];
    for (size_t k = s; k < e; k++) {
      while (j >= o[i].size()) {
        i++;
        j = 0;
      }
      E x = o[i][j++];
      if (pred(x)) out.push_back(f(x));
    }
  });
}

template <class Outer, class P>
inline auto filter(const flat_view<Outer>& fv, P&& pred) {
  return filter_map(fv, pred, [](auto x) { return x; });
}

template <class R, class P, class F>
inline auto filter_map(const R& r, P&& pred, F&& f) {
  using E = std::decay_t<decltype(r[0])>;
  using T = std::decay_t<decltype(f(std::declval<E>()))>;
  return blocked_collect<T>(r.size(), [&](size_t i, std::vector<T>& out) {
    E x = r[i];
    if (pred(x)) out.push_back(f(x));
  });
}

template <class R, class P>
inline auto filter(const R& r, P&& pred) {
  return parlay::filter(r, pred);
}
}  // namespace block_delayed

// ------------------------------------------------------------------ io
using chars = sequence<char>;

inline sequence<char> chars_from_file(const std::string& fname) {
  FILE* f = fopen(fname.c_str(), "rb");
  if (!f) {
    std::cout << "Unable to open file: " << fname << std::endl;
    abort();
  }
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  sequence<char> s(n > 0 ? n : 0, (char)0);
  if (n > 0 && fread(s.data(), 1, (size_t)n, f) != (size_t)n) {
    std::cout << "read error: " << fname << std::endl;
    abort();
  }
  fclose(f);
  return s;
}
// file_map returns the file's bytes (read, not mapped).
inline sequence<char> file_map(const std::string& fname) { return chars_from_file(fname); }

template <class R, class Sp>
inline sequence<sequence<char>> tokens(const R& s, Sp is_space) {
  size_t n = s.size();
  std::vector<std::pair<size_t, size_t>> spans;
  size_t i = 0;
  while (i < n) {
    while (i < n && is_space(s[i])) i++;
    size_t b = i;
    while (i < n && !is_space(s[i])) i++;
    if (i > b) spans.push_back({b, i});
  }
  return sequence<sequence<char>>::from_function(spans.size(), [&](size_t k) {
    return sequence<char>(s.begin() + spans[k].first, s.begin() + spans[k].second);
  });
}

template <class R>
inline long chars_to_long(const R& r) {
  std::string t(r.begin(), r.end());
  return std::strtol(t.c_str(), nullptr, 10);
}
template <class R>
inline double chars_to_double(const R& r) {
  std::string t(r.begin(), r.end());
  return std::strtod(t.c_str(), nullptr);
}

}  // namespace parlay
