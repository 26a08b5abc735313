// Test infrastructure only: Imath::Math lives in the ImathVec.h stand-in.
#pragma once
#include <OpenEXR/ImathVec.h>
