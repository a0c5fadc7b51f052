// Project-written stand-in for the few Boost.Odeint names that dynex.cc mentions.
//
// TEST INFRASTRUCTURE ONLY: used to compile the unmodified reference (dynex.cc) as
// the parity oracle and CPU baseline.  Boost is not installed in this image.  The
// reference's default integrator (ODE_CONSTANT_NOBOOST, dynex.cc:1381-1459) does not
// use odeint at all.  Its parameter tuner's initial objective (dynex.cc:1711-1716) takes
// one explicit Euler step through integrate_n_steps (dynex.cc:1260-1283), which is
// implemented here from Boost.Odeint's documented behaviour: the observer sees the
// start state at t0 and the state after each of the n steps; euler::do_step evaluates the
// system once at (x, t) and sets x = 1 * x + dt * dxdt element by element (odeint's
// scale_sum2).  The other odeint-based modes (dynex.cc:1233-1379) are out of scope and
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
  std::fprintf(stderr, "odeint stub: %s is not provided by this stub\n", what);
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
  // one explicit Euler step in place: x <- 1 * x + dt * f(x, t)
  template <class System, class Time>
  void do_step(System system, State& x, Time t, Time dt) {
    State dxdt(x.size());
    system(x, dxdt, t);
    for (std::size_t i = 0; i < x.size(); i++) x[i] = Value(1) * x[i] + dt * dxdt[i];
  }
};

template <class A, class B, class Stepper>
Stepper make_controlled(A, B, Stepper s) {
  odeint_stub_abort("make_controlled");
  return s;
}

template <class... A>
std::size_t integrate_adaptive(A&&...) { odeint_stub_abort("integrate_adaptive"); }

// n steps of size dt from (x, t0); the observer is called at t0 and after every step.
// Returns the end time.
template <class Stepper, class System, class State, class Time, class Observer>
Time integrate_n_steps(Stepper stepper, System system, State& x, Time t0, Time dt, std::size_t n,
                       Observer observer) {
  Time t = t0;
  observer(x, t);
  for (std::size_t k = 0; k < n; k++) {
    stepper.do_step(system, x, t, dt);
    t = t0 + Time(k + 1) * dt;
    observer(x, t);
  }
  return t;
}

}  // namespace odeint
}  // namespace numeric
}  // namespace boost
