// Test infrastructure only: see tbb_shim.h.
#pragma once
#include <tbb/tbb_shim.h>
