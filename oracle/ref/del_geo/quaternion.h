// Host shim for the del-geo C++ headers that del-splat's CUDA kernels
// include (TEST ONLY).  The del-geo crate is absent from the reference tree,
// so every function here forwards to this oracle's restatement in
// oracle/del_geo_restated.h; it exists only so that the reference's own
// kernel sources compile for the host unchanged.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include "../../del_geo_restated.h"

// (quaternion -> rotation is used inside mat2_sym::projected_spd_mat3)
