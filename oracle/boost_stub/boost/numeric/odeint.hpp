// Project-written stand-in for the few Boost.Odeint names that dynex.cc mentions.
//
// TEST INFRASTRUCTURE ONLY: used to compile the unmodified reference (dynex.cc) as
// the parity oracle and CPU baseline.  Boost is not installed in this image.  The
// reference's default integrator (ODE_CONSTANT_NOBOOST, dynex.cc:1381-1459) does not
// use odeint at all; the odeint-based modes (dynex.cc:1233-1379) are out of scope and
// abort if selected.
#pragma once
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <map>
#include <numeric>
#include <unistd.h>
#include <utility>
#include <vector>

namespace boost {
namespace numeric {
namespace odeint {

[[noreturn]] inline void odeint_stub_abort(const char* what) {
  std::fprintf(stderr, "odeint stub: %s is not available in this build\n", what);
  std::abort();
}

template <class State, class Value>
struct runge_kutta_cash_karp54 {};

template <class State, class Value>
struct bulirsch_stoer {
  template <class... A>
  explicit bulirsch_stoer(A&&...) {}
};

template <class State, class Value>
struct euler {
  template <class... A>
  void do_step(A&&...) { odeint_stub_abort("euler::do_step"); }
};

template <class A, class B, class Stepper>
Stepper make_controlled(A, B, Stepper s) {
  odeint_stub_abort("make_controlled");
  return s;
}

template <class... A>
std::size_t integrate_adaptive(A&&...) { odeint_stub_abort("integrate_adaptive"); }

template <class... A>
std::size_t integrate_n_steps(A&&...) { odeint_stub_abort("integrate_n_steps"); }

}  // namespace odeint
}  // namespace numeric
}  // namespace boost
