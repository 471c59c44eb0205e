/* ORACLE PIN — test infrastructure only; never linked into the product.
 *
 * The reference calls the float overloads of std::cos / std::sin / std::pow / std::asin /
 * std::acos / atan2f, whose last bit depends on the C library it is linked against (glibc's cosf and
 * powf, for example, are not correctly rounded).  The oracle and the device both use the correctly
 * rounded value: the function evaluated in double and rounded once to float (pow(x, 5) as
 * (x*x)*(x*x)*x in double, the oracle's pow5_rn).  This file gives the pin library its own
 * definitions of those C functions, with hidden visibility, so that the reference's headers compiled
 * into the pin library call them instead of glibc's; ref_libm_glibc(1) makes them forward to the C
 * library's own functions instead, so a test can also measure how often glibc's last bit differs. */
#include <dlfcn.h>

#include <cmath>
#include <cstdint>

namespace {
int g_use_glibc = 0;

template<class F>
F glibc_fn(const char *name) {
  static_assert(sizeof(F) == sizeof(void *), "function pointer");
  return reinterpret_cast<F>(dlsym(RTLD_DEFAULT, name));
}
}  // namespace

extern "C" {

void ref_libm_glibc(int32_t use_glibc) { g_use_glibc = use_glibc; }

__attribute__((visibility("hidden"))) float cosf(float x) {
  if (g_use_glibc) {
    static auto f = glibc_fn<float (*)(float)>("cosf");
    return f(x);
  }
  return (float)std::cos((double)x);
}

__attribute__((visibility("hidden"))) float sinf(float x) {
  if (g_use_glibc) {
    static auto f = glibc_fn<float (*)(float)>("sinf");
    return f(x);
  }
  return (float)std::sin((double)x);
}

__attribute__((visibility("hidden"))) void sincosf(float x, float *s, float *c) {
  *s = sinf(x);
  *c = cosf(x);
}

__attribute__((visibility("hidden"))) float asinf(float x) {
  if (g_use_glibc) {
    static auto f = glibc_fn<float (*)(float)>("asinf");
    return f(x);
  }
  return (float)std::asin((double)x);
}

__attribute__((visibility("hidden"))) float acosf(float x) {
  if (g_use_glibc) {
    static auto f = glibc_fn<float (*)(float)>("acosf");
    return f(x);
  }
  return (float)std::acos((double)x);
}

__attribute__((visibility("hidden"))) float atan2f(float y, float x) {
  if (g_use_glibc) {
    static auto f = glibc_fn<float (*)(float, float)>("atan2f");
    return f(y, x);
  }
  return (float)std::atan2((double)y, (double)x);
}

__attribute__((visibility("hidden"))) float powf(float x, float y) {
  if (g_use_glibc) {
    static auto f = glibc_fn<float (*)(float, float)>("powf");
    return f(x, y);
  }
  if (y == 5.f) {
    const double d = (double)x, d2 = d * d;
    return (float)(d2 * d2 * d);
  }
  return (float)std::pow((double)x, (double)y);
}

}  // extern "C"
