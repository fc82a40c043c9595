/* ORACLE (test infrastructure): resolves the reference driver's
 * `#include "../io/IO.h"` (main/run.cpp:10) to this library's drop-in IO. */
#pragma once
#include "gpsm_host/IO.h"
