// Stand-in for Arccore's <arccore/serialize/BasicSerializer.h>: see arccore_min.h.
#pragma once
#include "../../arccore_min.h"
