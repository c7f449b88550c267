// Stand-in for the CUDA samples' helper_timer.h (src/main.cu:4): the
// wall-clock stopwatch the reference prints its ">>>>>>Simulation time" with
// (src/main.cu:713-747).
#ifndef OCTMPS_BASELINE_HELPER_TIMER_H
#define OCTMPS_BASELINE_HELPER_TIMER_H

#include <chrono>

struct StopWatchInterface {
    std::chrono::steady_clock::time_point start;
    double total_ms = 0.0;
    bool running = false;
};

inline bool sdkCreateTimer(StopWatchInterface **t) {
    *t = new StopWatchInterface();
    return true;
}
inline bool sdkStartTimer(StopWatchInterface **t) {
    (*t)->start = std::chrono::steady_clock::now();
    (*t)->running = true;
    return true;
}
inline bool sdkStopTimer(StopWatchInterface **t) {
    if (!(*t)->running) return false;
    (*t)->total_ms += std::chrono::duration<double, std::milli>(
                          std::chrono::steady_clock::now() - (*t)->start)
                          .count();
    (*t)->running = false;
    return true;
}
inline float sdkGetTimerValue(StopWatchInterface **t) { return (float)(*t)->total_ms; }
inline bool sdkDeleteTimer(StopWatchInterface **t) {
    delete *t;
    *t = nullptr;
    return true;
}

#endif
