// Stand-in for Arccore's <arccore/serialize/ISerializer.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
