// Stand-in for the boost::posix_time clock types the reference's src/RunControl/Time.cpp uses
// for its progress messages (test infrastructure): wall-clock points and durations in
// microseconds, printed as hh:mm:ss.ffffff.
#ifndef CAFFE_REFSHIM_DATE_TIME_HPP
#define CAFFE_REFSHIM_DATE_TIME_HPP

#include <chrono>
#include <cstdio>
#include <string>

namespace boost {
namespace posix_time {

class time_duration {
public:
    long long us = 0;
    time_duration() = default;
    time_duration(double h, double m, double s, double frac) : us((long long)((h * 3600. + m * 60. + s) * 1e6 + frac)) {}
    time_duration& operator+=(const time_duration& o) { us += o.us; return *this; }
    bool operator>(const time_duration& o) const { return us > o.us; }
    long long total_microseconds() const { return us; }
};

class ptime {
public:
    long long us = 0;
    time_duration operator-(const ptime& o) const { time_duration d; d.us = us - o.us; return d; }
};

struct microsec_clock {
    static ptime local_time() {
        ptime t;
        t.us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::system_clock::now().time_since_epoch()).count();
        return t;
    }
};
struct second_clock {
    static ptime local_time() {
        ptime t = microsec_clock::local_time();
        t.us -= t.us % 1000000;
        return t;
    }
};

inline std::string to_simple_string(const time_duration& d) {
    long long us = d.us < 0 ? -d.us : d.us;
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%s%02lld:%02lld:%02lld.%06lld", d.us < 0 ? "-" : "", us / 3600000000LL,
                  (us / 60000000LL) % 60, (us / 1000000LL) % 60, us % 1000000LL);
    return buf;
}
inline std::string to_simple_string(const ptime& t) {
    time_duration d;
    d.us = t.us;
    return to_simple_string(d);
}

}  // namespace posix_time
}  // namespace boost

#endif
