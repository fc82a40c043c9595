/* ORACLE (test infrastructure): resolves `#include "../graph/Graph.h"`
 * (main/run.cpp:11) to this library's drop-in Graph. */
#pragma once
#include "gpsm_host/Graph.h"
