// TEST INFRASTRUCTURE: GSL-API stand-in header, see gslshim.h.
#pragma once
#include "gslshim.h"
