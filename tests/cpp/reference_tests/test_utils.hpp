// The helpers the reference's own test headers expect from
// test/test_utils.hpp (test_random_engine, the ans_check overloads,
// get_type), written for this build.  The reference's file also covers
// tensors, dense and random-structure matrices and build queries, which are
// outside the CRS solve path; build_reference_tests.py places this file
// where the reference's test headers look for test_utils.hpp.
#pragma once
#include "monolish_blas.hpp"
#include "monolish_vml.hpp"

#include <cmath>
#include <iomanip>
#include <iostream>
#include <random>
#include <string>
#include <vector>

template <typename T> std::string get_type();
template <> inline std::string get_type<double>() { return "double"; }
template <> inline std::string get_type<float>() { return "float"; }

// the seeded engine the tests draw their vector seeds from (mt19937, 1234)
inline std::mt19937 test_random_engine(1234);

// |result - ans| relative to |ans| (absolute when |ans| <= tol) below tol
inline bool within(double result, double ans, double tol) {
  const double err =
      std::abs(ans) <= tol ? std::abs(result - ans) : std::abs((result - ans) / ans);
  return err < tol;
}

template <typename T>
bool ans_check(const std::string &func, double result, double ans, double tol) {
  if (within(result, ans, tol)) return true;
  std::cout << func << "(" << get_type<T>() << "): fail, result " << std::scientific
            << result << " ans " << ans << std::endl;
  return false;
}

template <typename T> bool ans_check(const T *result, const T *ans, int size, double tol) {
  int bad = 0;
  for (int i = 0; i < size; ++i) {
    // as the reference's array check: relative unless the expected value is small
    const double err = ans[i] <= tol ? std::abs(result[i] - ans[i])
                                     : std::abs((result[i] - ans[i]) / ans[i]);
    if (err >= tol) {
      if (bad < 10)
        std::cout << i << "\tresult: " << std::setprecision(15) << result[i]
                  << "\tans: " << ans[i] << std::endl;
      ++bad;
    }
  }
  return bad == 0;
}

template <typename T>
bool ans_check(const std::string &func, const T *result, const T *ans, int size,
               double tol) {
  if (ans_check<T>(result, ans, size, tol)) return true;
  std::cout << func << "(" << get_type<T>() << "): fail" << std::endl;
  return false;
}
