// Test infrastructure only: the emerald sources name `half` in a typedef only.
#pragma once
#include <cstdint>
struct half { std::uint16_t bits; };
