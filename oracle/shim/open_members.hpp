// open_members.hpp -- forced include (-include) for building the reference inside the
// oracle harness. TEST INFRASTRUCTURE ONLY. It pulls in every standard header the
// reference and the shim use (so their include guards are already set), then opens
// HO_2D's private members so the harness can set inputs and read stage arrays without
// editing src/HO_2D.hpp.
#pragma once
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>
#include "shim_linalg.hpp"
#define private public
