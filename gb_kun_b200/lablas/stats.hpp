// Per-call statistics macros of the reference (src/helpers/stats/stats.h:11-117):
// SAVE_STATS, SAVE_TEPS, SAVE_TIME, SAVE_TIME_SEC and save_teps /
// save_time_in_ms / save_time_in_sec.  Each runs the call, times it and
// appends one line to perf_stats.txt in the working directory in the
// reference's line format ("<op> <time> (ms) <perf> (GFLOP/s|MTEPS/s) <bw>
// (GB/s) <nvals>"), so tooling that reads that file keeps working.
//
// The calls here are asynchronous device work, so the timer brackets the
// call with a synchronisation of the calling thread's lablas stream on both
// sides: the recorded time is the call's device time plus its host overhead.
// The macros open their own scope (the reference's declare my_* variables in
// the caller's scope); the call itself runs unchanged.
#pragma once

#include <chrono>
#include <cstdio>

#include "core.hpp"

namespace lablas {
namespace stats {

inline double now_ms() {
    cudaStreamSynchronize(current_stream());
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

inline void append(const char* op, double value, const char* time_unit, double perf, const char* perf_unit,
                   double bw, long long nvals) {
    FILE* f = std::fopen("perf_stats.txt", "a");
    if (!f) return;
    std::fprintf(f, "%s %lf (%s) %lf (%s) %lf (GB/s) %lld\n", op, value, time_unit, perf, perf_unit, bw, nvals);
    std::fclose(f);
}

}  // namespace stats
}  // namespace lablas

// GFLOP/s = 2 nvals / t, GB/s = nvals * bytes_per_flop / t (nvals of `matrix`).
#define SAVE_STATS(call_instruction, op_name, bytes_per_flop, iterations, matrix)                           \
    do {                                                                                                    \
        Index gbk_stats_nvals_ = 0;                                                                         \
        (matrix)->get_nvals(&gbk_stats_nvals_);                                                             \
        const double gbk_stats_t1_ = ::lablas::stats::now_ms();                                             \
        call_instruction;                                                                                   \
        const double gbk_stats_ms_ = ::lablas::stats::now_ms() - gbk_stats_t1_;                             \
        const double gbk_stats_s_ = gbk_stats_ms_ * 1e-3;                                                   \
        ::lablas::stats::append(op_name, gbk_stats_ms_, "ms", gbk_stats_nvals_ * 2.0 / (gbk_stats_s_ * 1e9), \
                                "GFLOP/s", gbk_stats_nvals_ * (double)(bytes_per_flop) / (gbk_stats_s_ * 1e9), \
                                (long long)gbk_stats_nvals_);                                               \
        (void)(iterations);                                                                                 \
    } while (0)

// MTEPS/s = iterations * nvals / t (nvals of `matrix`).
#define SAVE_TEPS(call_instruction, op_name, iterations, matrix)                                            \
    do {                                                                                                    \
        Index gbk_stats_nvals_ = 0;                                                                         \
        (matrix)->get_nvals(&gbk_stats_nvals_);                                                             \
        const double gbk_stats_t1_ = ::lablas::stats::now_ms();                                             \
        call_instruction;                                                                                   \
        const double gbk_stats_ms_ = ::lablas::stats::now_ms() - gbk_stats_t1_;                             \
        ::lablas::stats::append(op_name, gbk_stats_ms_, "ms",                                               \
                                (iterations) * (gbk_stats_nvals_ / (gbk_stats_ms_ * 1e3)), "MTEPS/s", 0.0,   \
                                (long long)gbk_stats_nvals_);                                               \
    } while (0)

#define SAVE_TIME(call_instruction, op_name)                                                                \
    do {                                                                                                    \
        const double gbk_stats_t1_ = ::lablas::stats::now_ms();                                             \
        call_instruction;                                                                                   \
        ::lablas::stats::append(op_name, ::lablas::stats::now_ms() - gbk_stats_t1_, "ms", 0.0, "GFLOP/s",   \
                                0.0, 0);                                                                    \
    } while (0)

#define SAVE_TIME_SEC(call_instruction, op_name)                                                            \
    do {                                                                                                    \
        const double gbk_stats_t1_ = ::lablas::stats::now_ms();                                             \
        call_instruction;                                                                                   \
        ::lablas::stats::append(op_name, (::lablas::stats::now_ms() - gbk_stats_t1_) * 1e-3, "s", 0.0,      \
                                "GFLOP/s", 0.0, 0);                                                         \
    } while (0)

// _time in ms; MTEPS/s = iterations * nvals / time.
inline void save_teps(const char* _op_name, double _time, size_t _nvals, int _iterations = 1) {
    ::lablas::stats::append(_op_name, _time, "ms", _iterations * (_nvals / (_time * 1e3)), "MTEPS/s", 0.0,
                            (long long)_nvals);
}
inline void save_time_in_ms(const char* _op_name, double _time) {
    ::lablas::stats::append(_op_name, _time * 1000, "ms", 0.0, "GFLOP/s", 0.0, 0);
}
inline void save_time_in_sec(const char* _op_name, double _time) {
    ::lablas::stats::append(_op_name, _time, "ms", 0.0, "GFLOP/s", 0.0, 0);
}
