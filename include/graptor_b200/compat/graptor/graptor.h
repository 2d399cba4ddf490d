// graptor/graptor.h for sources written against Graptor: maps the include
// onto the B200 library's operator surface (graptor_b200/api.h) and adds the
// small utilities the analytics use (commandLine, timer).
//
// Put include/graptor_b200/compat first on the include path; the analytics'
// own sources (bench/BFSLVLv.C, bench/BFSv.C, ...) then compile unchanged
// and run their edgemap / vertexmap steps on the GPU.
#ifndef GRAPTOR_B200_COMPAT_GRAPTOR_H
#define GRAPTOR_B200_COMPAT_GRAPTOR_H

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <type_traits>
#include <vector>

#include "graptor_b200/api.h"

// Command-line options with Graptor's accessors (legacy/parseCommandLine.h):
// getOption(flag) = flag present, getOptionValue(flag) = next argument,
// getOptionLongValue(flag, default).
struct commandLine {
    int argc;
    char **argv;
    std::string usage;
    commandLine(int c, char **v, std::string u = "") : argc(c), argv(v), usage(std::move(u)) {}
    int find(const std::string &flag) const {
        for (int i = 1; i < argc; ++i)
            if (flag == argv[i]) return i;
        return -1;
    }
    bool getOption(const std::string &flag) const { return find(flag) >= 0; }
    char *getOptionValue(const std::string &flag) const {
        int i = find(flag);
        return (i >= 0 && i + 1 < argc) ? argv[i + 1] : nullptr;
    }
    std::string getOptionValue(const std::string &flag, const std::string &dflt) const {
        char *v = getOptionValue(flag);
        return v ? std::string(v) : dflt;
    }
    long getOptionLongValue(const std::string &flag, long dflt) const {
        char *v = getOptionValue(flag);
        return v ? std::atol(v) : dflt;
    }
    double getOptionDoubleValue(const std::string &flag, double dflt) const {
        char *v = getOptionValue(flag);
        return v ? std::atof(v) : dflt;
    }
    char *getArgument(int i) const { return argv[argc - 1 - i]; }
};

// Wall-clock interval timer with Graptor's interface (timer.h): start(),
// next() = seconds since the previous start/next, total().
class timer {
public:
    timer() { start(); }
    void start() { last_ = now(); }
    double next() {
        double t = now(), d = t - last_;
        last_ = t;
        total_ += d;
        return d;
    }
    double stop() { next(); return total_; }
    double total() const { return total_; }

private:
    static double now() {
        return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
    }
    double last_ = 0, total_ = 0;
};

#endif
