// amgcl/adapter/crs_tuple.hpp -- oracle API shim (test infrastructure); see shim_amgcl.hpp.
#pragma once
#include "../../shim_amgcl.hpp"
