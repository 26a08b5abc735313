// Test infrastructure only: see format.h.
#pragma once
#include <fmt/format.h>
