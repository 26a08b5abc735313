// Test infrastructure only: nothing from Alembic::Util is used on the SPH path.
#pragma once
#include <Alembic/AbcGeom/All.h>
