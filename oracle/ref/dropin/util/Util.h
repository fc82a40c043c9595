/* ORACLE (test infrastructure): what the reference driver main/run.cpp takes
 * from util/Util.h - the standard headers it relies on and
 * Util::get_cur_time() in milliseconds (main/run.cpp:45, 73, 95). */
#pragma once
#include <chrono>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

class Util {
 public:
  static long get_cur_time() {
    return (long)std::chrono::duration_cast<std::chrono::milliseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
  }
};
