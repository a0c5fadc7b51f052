// Project-written stand-in for boost::posix_time as used by dynex.cc
// (microsec_clock::local_time().time_of_day().total_milliseconds(), dynex.cc:335).
// TEST INFRASTRUCTURE ONLY.  Returns milliseconds of a monotonic clock instead of the
// wall-clock time of day; the reference only uses differences of these values.
#pragma once
#include <chrono>

namespace boost {
namespace posix_time {

struct time_duration {
  long long ms;
  long long total_milliseconds() const { return ms; }
};

struct ptime {
  long long ms;
  time_duration time_of_day() const { return time_duration{ms}; }
};

struct microsec_clock {
  static ptime local_time() {
    using namespace std::chrono;
    return ptime{(long long)duration_cast<milliseconds>(steady_clock::now().time_since_epoch()).count()};
  }
};

}  // namespace posix_time
}  // namespace boost
