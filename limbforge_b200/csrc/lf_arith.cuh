// The limb arithmetic lives in include/limbforge/detail/arith.hpp, shared with the host-side scalar API.
#pragma once
#include "limbforge/detail/arith.hpp"
