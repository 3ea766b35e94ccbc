// Project-written stand-in for the waLBerla header of the same name, so that the
// reference's generated kernels compile without the (absent) waLBerla submodule.
// Test infrastructure only: used solely to build the checker under oracle/_ref.
#pragma once
#define WALBERLA_RESTRICT __restrict__
