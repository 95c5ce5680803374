// Host-only stand-in for the small Kokkos / EKAT surface that the mam4xx
// microphysics headers use (View, subview, resize, team policies, math
// forwards, complex, numeric traits, kernel asserts).
//
// TEST INFRASTRUCTURE ONLY. This lets the reference's own headers compile
// unchanged with g++ so their outputs can pin the oracle restatement. It is
// never linked into the product library.
//
// Semantics follow Kokkos' documented host behaviour: LayoutRight storage,
// views are reference-counted handles, unmanaged views wrap a raw pointer,
// math functions forward to the C library (glibc libm), and team ranges run
// serially on one thread.
//
// Compiled by nvcc (__CUDACC__), the same surface is also available in
// device code, for the reference headers compiled for the GPU (one thread
// per grid cell, oracle/ref/ref_step_gpu.cu): the Kokkos function macros
// become __host__ __device__, math functions forward to CUDA's math
// library in device code (double arguments; integer arguments promoted to
// double as Kokkos does), views are plain pointer/extent/stride handles
// (their allocating constructor is host-only and never frees: the device
// driver allocates no views), and a failed kernel assert is counted in a
// device counter instead of stopping the kernel.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#ifdef __CUDACC__
#define MAM4SHIM_HD __host__ __device__
#else
#define MAM4SHIM_HD
#endif

#define KOKKOS_INLINE_FUNCTION MAM4SHIM_HD inline
#define KOKKOS_FUNCTION MAM4SHIM_HD inline
#define KOKKOS_FORCEINLINE_FUNCTION MAM4SHIM_HD inline
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]

namespace mam4shim {
// Counted host check used for EKAT_KERNEL_ASSERT*: a failed check is
// recorded (not fatal) so a test can inspect it.
inline long &assert_failures() {
  static thread_local long n = 0;
  return n;
}
#ifdef __CUDACC__
// the device-side count of failed kernel asserts (read by the driver)
static __device__ unsigned long long dev_assert_failures;
#endif
} // namespace mam4shim

#if defined(__CUDA_ARCH__)
#define MAM4SHIM_FAIL() atomicAdd(&mam4shim::dev_assert_failures, 1ull)
#else
#define MAM4SHIM_FAIL() (++mam4shim::assert_failures())
#endif

#define EKAT_KERNEL_ASSERT(cond)                                               \
  do {                                                                         \
    if (!(cond))                                                               \
      MAM4SHIM_FAIL();                                                         \
  } while (0)
#define EKAT_KERNEL_ASSERT_MSG(cond, msg) EKAT_KERNEL_ASSERT(cond)
#define EKAT_KERNEL_REQUIRE(cond) EKAT_KERNEL_ASSERT(cond)
#define EKAT_KERNEL_REQUIRE_MSG(cond, msg) EKAT_KERNEL_ASSERT(cond)
#define EKAT_REQUIRE(cond) EKAT_KERNEL_ASSERT(cond)
#define EKAT_REQUIRE_MSG(cond, msg) EKAT_KERNEL_ASSERT(cond)
#define EKAT_ASSERT(cond) EKAT_KERNEL_ASSERT(cond)
#define EKAT_ASSERT_MSG(cond, msg) EKAT_KERNEL_ASSERT(cond)
#define EKAT_KERNEL_ERROR_MSG(msg) MAM4SHIM_FAIL()
#define EKAT_ERROR_MSG(msg) MAM4SHIM_FAIL()

namespace Kokkos {

struct HostSpace {};
struct CudaSpace {};
struct Serial {
  using memory_space = HostSpace;
};
struct MemoryUnmanaged {};
struct LayoutRight {};
struct LayoutLeft {};
struct LayoutStride {};
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;

struct ALL_t {
  MAM4SHIM_HD constexpr const ALL_t &operator()() const { return *this; }
};
inline constexpr ALL_t ALL{};

template <class T1, class T2 = T1> struct pair {
  T1 first;
  T2 second;
  constexpr pair() = default;
  MAM4SHIM_HD constexpr pair(const T1 &a, const T2 &b) : first(a), second(b) {}
  template <class U1, class U2>
  constexpr pair(const std::pair<U1, U2> &p) : first(p.first), second(p.second) {}
};
template <class T1, class T2> MAM4SHIM_HD pair<T1, T2> make_pair(T1 a, T2 b) {
  return pair<T1, T2>(a, b);
}

#ifdef __CUDACC__
// host: print and stop; device: counted like a failed kernel assert (the
// device oracle never traps)
MAM4SHIM_HD inline void abort(const char *msg) {
#if defined(__CUDA_ARCH__)
  (void)msg;
  MAM4SHIM_FAIL();
#else
  std::fprintf(stderr, "Kokkos::abort: %s\n", msg);
  std::abort();
#endif
}
#else
[[noreturn]] inline void abort(const char *msg) {
  std::fprintf(stderr, "Kokkos::abort: %s\n", msg);
  std::abort();
}
#endif

// ---------------------------------------------------------------- math
#ifdef __CUDACC__
// double overloads forwarding to the global C functions, which nvcc maps to
// CUDA's math library in device code and to the C library in host code;
// float overloads to the f-suffixed functions; integers promoted to double
#define MAM4SHIM_MATH1(f, ff)                                                  \
  MAM4SHIM_HD inline double f(double x) { return ::f(x); }                     \
  MAM4SHIM_HD inline float f(float x) { return ::ff(x); }                      \
  template <class I, std::enable_if_t<std::is_integral_v<I>, int> = 0>         \
  MAM4SHIM_HD inline double f(I x) {                                           \
    return ::f(static_cast<double>(x));                                        \
  }
MAM4SHIM_MATH1(atan, atanf)
MAM4SHIM_MATH1(cbrt, cbrtf)
MAM4SHIM_MATH1(cos, cosf)
MAM4SHIM_MATH1(erf, erff)
MAM4SHIM_MATH1(erfc, erfcf)
MAM4SHIM_MATH1(exp, expf)
MAM4SHIM_MATH1(log, logf)
MAM4SHIM_MATH1(log10, log10f)
MAM4SHIM_MATH1(round, roundf)
MAM4SHIM_MATH1(sin, sinf)
MAM4SHIM_MATH1(sqrt, sqrtf)
#undef MAM4SHIM_MATH1
MAM4SHIM_HD inline double abs(double x) { return ::fabs(x); }
MAM4SHIM_HD inline float abs(float x) { return ::fabsf(x); }
MAM4SHIM_HD inline int abs(int x) { return x < 0 ? -x : x; }
MAM4SHIM_HD inline long abs(long x) { return x < 0 ? -x : x; }
MAM4SHIM_HD inline bool isnan(double x) { return ::isnan(x); }
MAM4SHIM_HD inline bool isnan(float x) { return ::isnan(x); }
MAM4SHIM_HD inline double pow(double x, double y) { return ::pow(x, y); }
MAM4SHIM_HD inline float pow(float x, float y) { return ::powf(x, y); }
// mixed or integer arguments: both promoted to double (std::pow's rule)
template <class A, class B,
          std::enable_if_t<std::is_arithmetic_v<A> && std::is_arithmetic_v<B> &&
                               !(std::is_same_v<A, double> && std::is_same_v<B, double>) &&
                               !(std::is_same_v<A, float> && std::is_same_v<B, float>),
                           int> = 0>
MAM4SHIM_HD inline double pow(A x, B y) {
  return ::pow(static_cast<double>(x), static_cast<double>(y));
}
MAM4SHIM_HD inline double nan(const char *s) { return ::nan(s); }
MAM4SHIM_HD inline double copysign(double x, double y) { return ::copysign(x, y); }
#else
using std::abs;
using std::atan;
using std::cbrt;
using std::cos;
using std::erf;
using std::erfc;
using std::exp;
using std::isnan;
using std::log;
using std::log10;
using std::pow;
using std::round;
using std::sin;
using std::sqrt;
using std::copysign;
inline double nan(const char *s) { return std::nan(s); }
#endif
template <class T> MAM4SHIM_HD constexpr const T &min(const T &a, const T &b) {
  return (b < a) ? b : a;
}
template <class T> MAM4SHIM_HD constexpr const T &max(const T &a, const T &b) {
  return (a < b) ? b : a;
}

// libm inside the complex arithmetic: std:: on the host build, the global
// functions (CUDA's math library in device code) under nvcc
#ifdef __CUDACC__
#define MAM4SHIM_M(f) ::f
#else
#define MAM4SHIM_M(f) std::f
#endif

// Kokkos::complex with Kokkos' own arithmetic (Kokkos_Complex.hpp, Kokkos
// 4.x): component-wise +,-; textbook product; quotient scaled by the
// 1-norm of the divisor; abs = hypot; sqrt by the half-angle formula;
// pow(z, real) = polar(pow(|z|, y), y*atan2(im, re)). These differ from
// libstdc++'s std::complex (which calls __divdc3 / csqrt / clog) in the
// last bits, and the water-uptake quartic goes through them.
template <class T> class complex {
  T re_ = T(0), im_ = T(0);

public:
  using value_type = T;
  constexpr complex() = default;
  MAM4SHIM_HD constexpr complex(const T &r) : re_(r), im_(T(0)) {}
  MAM4SHIM_HD constexpr complex(const T &r, const T &i) : re_(r), im_(i) {}
  MAM4SHIM_HD constexpr T real() const { return re_; }
  MAM4SHIM_HD constexpr T imag() const { return im_; }
  MAM4SHIM_HD complex &operator+=(const complex &o) {
    re_ += o.re_;
    im_ += o.im_;
    return *this;
  }
  MAM4SHIM_HD complex &operator-=(const complex &o) {
    re_ -= o.re_;
    im_ -= o.im_;
    return *this;
  }
  MAM4SHIM_HD complex &operator*=(const complex &o) {
    const T r = re_ * o.re_ - im_ * o.im_;
    im_ = re_ * o.im_ + im_ * o.re_;
    re_ = r;
    return *this;
  }
  MAM4SHIM_HD complex &operator/=(const T &s) {
    re_ /= s;
    im_ /= s;
    return *this;
  }
  MAM4SHIM_HD complex &operator*=(const T &s) {
    re_ *= s;
    im_ *= s;
    return *this;
  }
};
template <class T> MAM4SHIM_HD complex<T> operator-(const complex<T> &x) {
  return complex<T>(-x.real(), -x.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator+(const complex<T> &x, const complex<T> &y) {
  return complex<T>(x.real() + y.real(), x.imag() + y.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator+(const complex<T> &x, const T &y) {
  return complex<T>(x.real() + y, x.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator+(const T &x, const complex<T> &y) {
  return complex<T>(x + y.real(), y.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator-(const complex<T> &x, const complex<T> &y) {
  return complex<T>(x.real() - y.real(), x.imag() - y.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator-(const complex<T> &x, const T &y) {
  return complex<T>(x.real() - y, x.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator-(const T &x, const complex<T> &y) {
  return complex<T>(x - y.real(), -y.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator*(const complex<T> &x, const complex<T> &y) {
  return complex<T>(x.real() * y.real() - x.imag() * y.imag(),
                    x.real() * y.imag() + x.imag() * y.real());
}
template <class T> MAM4SHIM_HD complex<T> operator*(const complex<T> &x, const T &y) {
  return complex<T>(x.real() * y, x.imag() * y);
}
template <class T> MAM4SHIM_HD complex<T> operator*(const T &x, const complex<T> &y) {
  return complex<T>(x * y.real(), x * y.imag());
}
template <class T> MAM4SHIM_HD complex<T> operator/(const complex<T> &x, const complex<T> &y) {
  const T s = MAM4SHIM_M(fabs)(y.real()) + MAM4SHIM_M(fabs)(y.imag());
  if (s == 0.0)
    return complex<T>(x.real() / s, x.imag() / s);
  const complex<T> xs(x.real() / s, x.imag() / s);
  const complex<T> ycs(y.real() / s, -y.imag() / s);
  const T yabs2 = ycs.real() * ycs.real() + ycs.imag() * ycs.imag();
  complex<T> r = xs * ycs;
  r /= yabs2;
  return r;
}
template <class T> MAM4SHIM_HD complex<T> operator/(const complex<T> &x, const T &y) {
  return complex<T>(x.real() / y, x.imag() / y);
}
template <class T> MAM4SHIM_HD complex<T> operator/(const T &x, const complex<T> &y) {
  return complex<T>(x) / y;
}
template <class T> MAM4SHIM_HD bool operator==(const complex<T> &x, const complex<T> &y) {
  return x.real() == y.real() && x.imag() == y.imag();
}
template <class T> MAM4SHIM_HD bool operator!=(const complex<T> &x, const complex<T> &y) {
  return !(x == y);
}
template <class T> MAM4SHIM_HD T real(const complex<T> &x) { return x.real(); }
template <class T> MAM4SHIM_HD T imag(const complex<T> &x) { return x.imag(); }
template <class T> MAM4SHIM_HD T abs(const complex<T> &x) { return MAM4SHIM_M(hypot)(x.real(), x.imag()); }
template <class T> MAM4SHIM_HD complex<T> polar(const T &rho, const T &theta) {
  return complex<T>(rho * MAM4SHIM_M(cos)(theta), rho * MAM4SHIM_M(sin)(theta));
}
template <class T> MAM4SHIM_HD complex<T> sqrt(const complex<T> &x) {
  const T r = x.real(), i = x.imag();
  if (r == T(0)) {
    const T t = MAM4SHIM_M(sqrt)(MAM4SHIM_M(fabs)(i) / 2);
    return complex<T>(t, i < T(0) ? -t : t);
  }
  const T t = MAM4SHIM_M(sqrt)(2 * (abs(x) + MAM4SHIM_M(fabs)(r)));
  const T u = t / 2;
  return r > T(0) ? complex<T>(u, i / t)
                  : complex<T>(MAM4SHIM_M(fabs)(i) / t, i < T(0) ? -u : u);
}
template <class T, class U,
          std::enable_if_t<std::is_arithmetic_v<U>, int> = 0>
MAM4SHIM_HD complex<T> pow(const complex<T> &x, const U &y) {
  const T r = abs(x);
  const T theta = MAM4SHIM_M(atan2)(x.imag(), x.real());
  return polar(T(MAM4SHIM_M(pow)(r, T(y))), T(y) * theta);
}

namespace Experimental {
template <class T> inline constexpr T epsilon_v = std::numeric_limits<T>::epsilon();
template <class T> inline constexpr T finite_max_v = std::numeric_limits<T>::max();
template <class T> inline constexpr T finite_min_v = std::numeric_limits<T>::lowest();
template <class T> inline constexpr T infinity_v = std::numeric_limits<T>::infinity();
template <class T> inline constexpr T quiet_NaN_v = std::numeric_limits<T>::quiet_NaN();
} // namespace Experimental

template <class T, std::size_t N> struct Array {
  T m_data[N > 0 ? N : 1];
  MAM4SHIM_HD constexpr T &operator[](std::size_t i) { return m_data[i]; }
  MAM4SHIM_HD constexpr const T &operator[](std::size_t i) const { return m_data[i]; }
  MAM4SHIM_HD constexpr std::size_t size() const { return N; }
  MAM4SHIM_HD constexpr T *data() { return m_data; }
  MAM4SHIM_HD constexpr const T *data() const { return m_data; }
};
template <class T, std::size_t N>
MAM4SHIM_HD constexpr Array<T, N> to_array(const T (&a)[N]) {
  Array<T, N> out{};
  for (std::size_t i = 0; i < N; ++i)
    out.m_data[i] = a[i];
  return out;
}
template <class T, std::size_t N>
MAM4SHIM_HD constexpr Array<std::remove_cv_t<T>, N> to_array(T (&&a)[N]) {
  Array<std::remove_cv_t<T>, N> out{};
  for (std::size_t i = 0; i < N; ++i)
    out.m_data[i] = a[i];
  return out;
}

// ---------------------------------------------------------------- views
namespace impl {
// Decompose a Kokkos data type such as double**, const double*[3].
template <class D> struct data_traits {
  using value_type = D;
  static constexpr int rank = 0;
  static constexpr std::size_t static_extent[1] = {0};
};
template <class D> struct data_traits<D *> {
  using value_type = typename data_traits<D>::value_type;
  static constexpr int rank = data_traits<D>::rank + 1;
};
template <class D, std::size_t N> struct data_traits<D[N]> {
  using value_type = typename data_traits<D>::value_type;
  static constexpr int rank = data_traits<D>::rank + 1;
};
template <class D> struct data_traits<D[]> {
  using value_type = typename data_traits<D>::value_type;
  static constexpr int rank = data_traits<D>::rank + 1;
};
// static extents, outermost first (0 for runtime extents)
template <class D> struct static_extents {
  MAM4SHIM_HD static void fill(std::size_t *) {}
};
template <class D> struct static_extents<D *> {
  MAM4SHIM_HD static void fill(std::size_t *e) {
    e[0] = 0;
    static_extents<D>::fill(e + 1);
  }
};
template <class D, std::size_t N> struct static_extents<D[N]> {
  MAM4SHIM_HD static void fill(std::size_t *e) {
    e[0] = N;
    static_extents<D>::fill(e + 1);
  }
};
template <class D> struct static_extents<D[]> {
  MAM4SHIM_HD static void fill(std::size_t *e) {
    e[0] = 0;
    static_extents<D>::fill(e + 1);
  }
};
} // namespace impl

constexpr int VIEW_MAX_RANK = 8;

template <class DataType, class... Props> class View {
public:
  using traits = impl::data_traits<DataType>;
  using value_type = typename traits::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using pointer_type = value_type *;
  using reference_type = value_type &;
  using data_type = DataType;
  using HostMirror = View<std::remove_const_t<DataType>>;
  using host_mirror_type = HostMirror;
  using non_const_type = View<std::remove_const_t<DataType>>;
  using const_type = View<const DataType>;
  using memory_space = HostSpace;
  using execution_space = Serial;
  static constexpr int rank = traits::rank;
  static constexpr int Rank = traits::rank;

  value_type *m_ptr = nullptr;
  std::size_t m_ext[VIEW_MAX_RANK] = {};
  std::size_t m_str[VIEW_MAX_RANK] = {};
#ifdef __CUDACC__
  // nvcc build: a plain handle usable in device code; the allocating
  // constructor (host only) never frees
  const char *m_label = "";
#else
  std::shared_ptr<non_const_value_type> m_owner;
  std::string m_label;
#endif

  View() = default;

#ifdef __CUDACC__
  template <class... I,
            typename = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  View(const char *label, I... n) : m_label(label) {
    set_extents(n...);
    std::size_t sz = size();
    m_ptr = new non_const_value_type[sz > 0 ? sz : 1]();
  }
  template <class... I,
            typename = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  View(const std::string &label, I... n) : View("", n...) {}
#else
  // allocating: View(label, runtime extents...)
  template <class... I,
            typename = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  View(const std::string &label, I... n) : m_label(label) {
    set_extents(n...);
    std::size_t sz = size();
    m_owner = std::shared_ptr<non_const_value_type>(
        new non_const_value_type[sz > 0 ? sz : 1](),
        std::default_delete<non_const_value_type[]>());
    m_ptr = m_owner.get();
  }
  template <class... I,
            typename = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  View(const char *label, I... n) : View(std::string(label), n...) {}
#endif

  // unmanaged: View(ptr, runtime extents...)
  template <class... I,
            typename = std::enable_if_t<(std::is_integral_v<I> && ...)>>
  MAM4SHIM_HD View(value_type *p, I... n) : m_ptr(p) {
    set_extents(n...);
  }

  // conversion from compatible (e.g. non-const -> const, other props)
  template <class D2, class... P2,
            typename = std::enable_if_t<std::is_convertible_v<
                typename View<D2, P2...>::value_type *, value_type *>>>
#ifdef __CUDACC__
  MAM4SHIM_HD View(const View<D2, P2...> &o) : m_ptr(o.m_ptr), m_label(o.m_label) {
#else
  View(const View<D2, P2...> &o)
      : m_ptr(o.m_ptr), m_owner(o.m_owner), m_label(o.m_label) {
#endif
    for (int r = 0; r < VIEW_MAX_RANK; ++r) {
      m_ext[r] = o.m_ext[r];
      m_str[r] = o.m_str[r];
    }
  }

  template <class... I> MAM4SHIM_HD void set_extents(I... n) {
    std::size_t st[VIEW_MAX_RANK] = {};
    impl::static_extents<DataType>::fill(st);
    std::size_t dyn[] = {static_cast<std::size_t>(n)..., 0};
    std::size_t k = 0;
    for (int r = 0; r < rank; ++r) {
      if (st[r] != 0)
        m_ext[r] = st[r];
      else
        m_ext[r] = (k < sizeof...(I)) ? dyn[k++] : 1;
    }
    std::size_t s = 1;
    for (int r = rank - 1; r >= 0; --r) {
      m_str[r] = s;
      s *= m_ext[r];
    }
  }

  MAM4SHIM_HD std::size_t size() const {
    std::size_t s = 1;
    for (int r = 0; r < rank; ++r)
      s *= m_ext[r];
    return s;
  }
  MAM4SHIM_HD std::size_t span() const { return size(); }
  MAM4SHIM_HD std::size_t extent(int r) const { return r < rank ? m_ext[r] : 1; }
  MAM4SHIM_HD int extent_int(int r) const { return static_cast<int>(extent(r)); }
  MAM4SHIM_HD std::size_t stride(int r) const { return m_str[r]; }
  MAM4SHIM_HD value_type *data() const { return m_ptr; }
  MAM4SHIM_HD bool is_allocated() const { return m_ptr != nullptr; }
#ifdef __CUDACC__
  std::string label() const { return m_label; }
  long use_count() const { return 1; }
#else
  const std::string &label() const { return m_label; }
  long use_count() const { return m_owner.use_count(); }
#endif

  template <class... I> MAM4SHIM_HD value_type &operator()(I... i) const {
    std::size_t idx[] = {static_cast<std::size_t>(i)..., 0};
    std::size_t off = 0;
    for (std::size_t r = 0; r < sizeof...(I); ++r)
      off += idx[r] * m_str[r];
    return m_ptr[off];
  }
  template <class I> MAM4SHIM_HD value_type &operator[](I i) const {
    return m_ptr[static_cast<std::size_t>(i) * m_str[0]];
  }
};

template <class D, class... P, class... I>
void resize(View<D, P...> &v, I... n) {
  View<D, P...> nv(v.label(), n...);
  v = nv;
}
template <class D, class... P, class... I>
void realloc(View<D, P...> &v, I... n) {
  resize(v, n...);
}

template <class V> typename V::HostMirror create_mirror_view(const V &v) {
  return typename V::HostMirror(v);
}
template <class V> typename V::HostMirror create_mirror(const V &v) {
  typename V::HostMirror m(v.label(), 0);
  return m;
}
template <class V1, class V2> void deep_copy(const V1 &dst, const V2 &src) {
  if constexpr (std::is_arithmetic_v<V2>) {
    for (std::size_t i = 0; i < dst.size(); ++i)
      dst.data()[i] = src;
  } else {
    std::copy(src.data(), src.data() + src.size(), dst.data());
  }
}
inline void fence() {}
inline void fence(const char *) {}

namespace impl {
template <class T> struct is_index : std::is_integral<T> {};
// one subview argument: integer index, ALL, or [first, last) range
struct sv_arg {
  enum Kind { Index, All, Range } kind;
  std::size_t a, b;
};
MAM4SHIM_HD inline sv_arg mk(const ALL_t &) { return {sv_arg::All, 0, 0}; }
template <class T, std::enable_if_t<std::is_integral_v<T>, int> = 0>
MAM4SHIM_HD sv_arg mk(T i) {
  return {sv_arg::Index, static_cast<std::size_t>(i), 0};
}
template <class A, class B> MAM4SHIM_HD sv_arg mk(const pair<A, B> &p) {
  return {sv_arg::Range, static_cast<std::size_t>(p.first),
          static_cast<std::size_t>(p.second)};
}
template <class A, class B> sv_arg mk(const std::pair<A, B> &p) {
  return {sv_arg::Range, static_cast<std::size_t>(p.first),
          static_cast<std::size_t>(p.second)};
}
template <class T> struct is_idx_arg : std::is_integral<std::decay_t<T>> {};
template <class T> struct add_ptr { using type = T *; };
template <class T, int N> struct ptrs { using type = typename ptrs<T *, N - 1>::type; };
template <class T> struct ptrs<T, 0> { using type = T; };
} // namespace impl

template <class D, class... P, class... A>
MAM4SHIM_HD auto subview(const View<D, P...> &v, A... args) {
  constexpr int n_idx = (0 + ... + (std::is_integral_v<std::decay_t<A>> ? 1 : 0));
  constexpr int new_rank = View<D, P...>::rank - n_idx;
  using T = typename View<D, P...>::value_type;
  using R = View<typename impl::ptrs<T, new_rank>::type, LayoutStride>;
  impl::sv_arg sa[] = {impl::mk(args)...};
  R out;
  std::size_t off = 0;
  int k = 0;
  for (int r = 0; r < View<D, P...>::rank; ++r) {
    if (r < (int)sizeof...(A)) {
      const auto &s = sa[r];
      if (s.kind == impl::sv_arg::Index) {
        off += s.a * v.m_str[r];
        continue;
      }
      if (s.kind == impl::sv_arg::Range) {
        off += s.a * v.m_str[r];
        out.m_ext[k] = s.b - s.a;
        out.m_str[k] = v.m_str[r];
        ++k;
        continue;
      }
    }
    out.m_ext[k] = v.m_ext[r];
    out.m_str[k] = v.m_str[r];
    ++k;
  }
  out.m_ptr = v.m_ptr + off;
#ifndef __CUDACC__
  out.m_owner = v.m_owner;
#endif
  return out;
}

// ---------------------------------------------------------------- teams
struct TeamMember {
  int m_league_rank = 0;
  MAM4SHIM_HD int league_rank() const { return m_league_rank; }
  MAM4SHIM_HD int league_size() const { return 1; }
  MAM4SHIM_HD int team_rank() const { return 0; }
  MAM4SHIM_HD int team_size() const { return 1; }
  MAM4SHIM_HD void team_barrier() const {}
};
struct TeamPolicy {
  using member_type = TeamMember;
  int m_league = 1;
  TeamPolicy() = default;
  TeamPolicy(int league, int) : m_league(league) {}
  TeamPolicy(int league, int, int) : m_league(league) {}
  template <class A> TeamPolicy(int league, const A &) : m_league(league) {}
  int league_size() const { return m_league; }
};
template <class... P> struct RangePolicy {
  int b = 0, e = 0;
  RangePolicy(int begin, int end) : b(begin), e(end) {}
};
struct AUTO_t {};
inline constexpr AUTO_t AUTO{};

template <class I> struct IndexRange {
  I b, e;
};
template <class M, class I> MAM4SHIM_HD IndexRange<I> TeamVectorRange(const M &, I n) {
  return {I(0), n};
}
template <class M, class I, class J>
MAM4SHIM_HD IndexRange<std::common_type_t<I, J>> TeamVectorRange(const M &, I b, J e) {
  return {std::common_type_t<I, J>(b), std::common_type_t<I, J>(e)};
}
template <class M, class I> MAM4SHIM_HD IndexRange<I> TeamThreadRange(const M &, I n) {
  return {I(0), n};
}
template <class M, class I, class J>
MAM4SHIM_HD IndexRange<std::common_type_t<I, J>> TeamThreadRange(const M &, I b, J e) {
  return {std::common_type_t<I, J>(b), std::common_type_t<I, J>(e)};
}
template <class M, class I> MAM4SHIM_HD IndexRange<I> ThreadVectorRange(const M &, I n) {
  return {I(0), n};
}
template <class M, class I, class J>
MAM4SHIM_HD IndexRange<std::common_type_t<I, J>> ThreadVectorRange(const M &, I b, J e) {
  return {std::common_type_t<I, J>(b), std::common_type_t<I, J>(e)};
}

template <class I, class F> MAM4SHIM_HD void parallel_for(const IndexRange<I> &r, const F &f) {
  for (I i = r.b; i < r.e; ++i)
    f(i);
}
template <class F> void parallel_for(const TeamPolicy &p, const F &f) {
  for (int l = 0; l < p.league_size(); ++l) {
    TeamMember m;
    m.m_league_rank = l;
    f(m);
  }
}
template <class F> void parallel_for(const std::string &, const TeamPolicy &p, const F &f) {
  parallel_for(p, f);
}
template <class F> void parallel_for(int n, const F &f) {
  for (int i = 0; i < n; ++i)
    f(i);
}
template <class F, class... P> void parallel_for(const RangePolicy<P...> &r, const F &f) {
  for (int i = r.b; i < r.e; ++i)
    f(i);
}
template <class F, class... P>
void parallel_for(const std::string &, const RangePolicy<P...> &r, const F &f) {
  parallel_for(r, f);
}

template <class T> struct Sum {
  T &ref;
  MAM4SHIM_HD explicit Sum(T &r) : ref(r) {}
};
template <class T> struct Min {
  T &ref;
  MAM4SHIM_HD explicit Min(T &r) : ref(r) {}
};
template <class T> struct Max {
  T &ref;
  MAM4SHIM_HD explicit Max(T &r) : ref(r) {}
};
template <class I, class F, class T>
MAM4SHIM_HD void parallel_reduce(const IndexRange<I> &r, const F &f, T &result) {
  T acc{};
  for (I i = r.b; i < r.e; ++i)
    f(i, acc);
  result = acc;
}
template <class I, class F, class T>
MAM4SHIM_HD void parallel_reduce(const IndexRange<I> &r, const F &f, Sum<T> red) {
  T acc{};
  for (I i = r.b; i < r.e; ++i)
    f(i, acc);
  red.ref = acc;
}
template <class I, class F, class T>
MAM4SHIM_HD void parallel_reduce(const IndexRange<I> &r, const F &f, Min<T> red) {
  T acc = std::numeric_limits<T>::max();
  for (I i = r.b; i < r.e; ++i)
    f(i, acc);
  red.ref = acc;
}
template <class I, class F, class T>
MAM4SHIM_HD void parallel_reduce(const IndexRange<I> &r, const F &f, Max<T> red) {
  T acc = std::numeric_limits<T>::lowest();
  for (I i = r.b; i < r.e; ++i)
    f(i, acc);
  red.ref = acc;
}
// Serial inclusive scan: one pass with final = true, double accumulator
// (the only value type the headers scan).
template <class I, class F> MAM4SHIM_HD void parallel_scan(const IndexRange<I> &r, const F &f) {
  double acc = 0.0;
  for (I i = r.b; i < r.e; ++i)
    f(i, acc, true);
}
template <class M, class F> MAM4SHIM_HD void single(const M &, const F &f) { f(); }
struct PerTeamT {};
struct PerThreadT {};
template <class M> MAM4SHIM_HD PerTeamT PerTeam(const M &) { return {}; }
template <class M> MAM4SHIM_HD PerThreadT PerThread(const M &) { return {}; }
template <class M, class F> MAM4SHIM_HD void single(PerTeamT, const F &f) { f(); }
template <class M, class F> MAM4SHIM_HD void single(PerThreadT, const F &f) { f(); }

} // namespace Kokkos

// ---------------------------------------------------------------- ekat
namespace ekat {
struct DefaultDevice {};
struct HostDevice {};
template <class Dev> struct KokkosTypes {
  using ExeSpace = Kokkos::Serial;
  using MemSpace = Kokkos::HostSpace;
  using TeamPolicy = Kokkos::TeamPolicy;
  using MemberType = Kokkos::TeamMember;
  using RangePolicy = Kokkos::RangePolicy<>;
  template <class T> using view = Kokkos::View<T>;
  template <class T> using view_1d = Kokkos::View<T *>;
  template <class T> using view_2d = Kokkos::View<T **>;
  template <class T> using view_3d = Kokkos::View<T ***>;
  template <class T, int N>
  using view_ND = Kokkos::View<typename Kokkos::impl::ptrs<T, N>::type>;
};
template <class V> struct unmanaged_helper;
template <class D, class... P> struct unmanaged_helper<Kokkos::View<D, P...>> {
  using type = Kokkos::View<D, P..., Kokkos::MemoryUnmanaged>;
};
template <class V> using Unmanaged = typename unmanaged_helper<V>::type;

template <class T> MAM4SHIM_HD constexpr T invalid() {
  if constexpr (std::is_integral_v<T>)
    return std::numeric_limits<T>::max();
  else
    return std::numeric_limits<T>::quiet_NaN();
}
template <class V, class I> MAM4SHIM_HD auto subview(const V &v, I i) {
  return Kokkos::subview(v, i, Kokkos::ALL);
}
template <class V, class I, class J> MAM4SHIM_HD auto subview(const V &v, I i, J j) {
  return Kokkos::subview(v, i, j, Kokkos::ALL);
}
template <class T> struct is_single_precision : std::false_type {};
template <> struct is_single_precision<float> : std::true_type {};
template <class T> MAM4SHIM_HD T square(const T &x) { return x * x; }
template <class T> MAM4SHIM_HD T cube(const T &x) { return x * x * x; }

namespace logger {
enum class LogLevel { trace, debug, info, warn, err, critical, off };
}
template <class... A> struct LoggerT {
  template <class... B> LoggerT(B &&...) {}
  template <class... B> void info(B &&...) const {}
  template <class... B> void debug(B &&...) const {}
  template <class... B> void warn(B &&...) const {}
  template <class... B> void error(B &&...) const {}
};
using Logger = LoggerT<>;
} // namespace ekat
