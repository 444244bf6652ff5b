// Project-written stand-in for the reference's external common.h.  The headers
// compiled in oracle/_ref need only the standard library from it.
#pragma once

#include <cassert>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <iostream>
#include <iomanip>
#include <sstream>
#include <string>
