// gnuplot-iostream.h — a stand-in for the gnuplot-iostream header, which is not
// installed here (TEST INFRASTRUCTURE ONLY). lcurve_re's helpers include it for
// their plotting code; the solvers built by tests/solvers/Makefile run with
// plot_device "none", which never constructs a Gnuplot, so this type only has to
// accept the calls the sources make on one (stream insertion, manipulators
// and send1d) and
// does nothing with them.
#ifndef LCG_TEST_GNUPLOT_IOSTREAM_STUB_H
#define LCG_TEST_GNUPLOT_IOSTREAM_STUB_H

#include <ostream>

class Gnuplot {
public:
    Gnuplot() = default;
    explicit Gnuplot(const char *) {}
    template <class T>
    Gnuplot &operator<<(const T &) {
        return *this;
    }
    Gnuplot &operator<<(std::ostream &(*)(std::ostream &)) {  // std::flush, std::endl
        return *this;
    }
    template <class T>
    Gnuplot &send1d(const T &) {
        return *this;
    }
};

#endif
