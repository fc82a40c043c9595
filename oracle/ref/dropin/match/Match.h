/* ORACLE (test infrastructure): resolves `#include "../match/Match.h"`
 * (main/run.cpp:12) to this library's drop-in Match. */
#pragma once
#include "gpsm_host/Match.h"
